"""Generate the golden (T) fixtures from the reference's own C kernels.

The reference library (oracle/_ref/libcc_vjp_ref.so) is compiled unchanged
from pyscfadlib/pyscfadlib/vjp/cc/*.c by oracle/Makefile; it exists only
where the reference checkout does, so this script runs here and its
outputs are committed.  Each fixture holds the seeded inputs (reference
layouts), E(T), the gradients w.r.t. every input as an independent tensor
(ovvv unpacked), and the reference's packed-tril ovvv cotangent
(pyscfad/cc/ccsd_t.py:184-191).

    python tests/golden/make_golden.py          # all fixtures
    python tests/golden/make_golden.py --lno    # the LNO fixtures only
    python tests/golden/make_golden.py --df     # the DF-factor fixtures only

The LNO fixtures hold, in addition, the projector mat and its cotangent,
from the reference's lnoccsdt_contract / lnoccsdt_energy_vjp
(pyscfadlib/pyscfadlib/vjp/cc/lno_ccsd_t.c, lno_ccsd_t_vjp.c).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from pyscfad_b200.synthetic import make_inputs  # noqa: E402

# name: (nocc, nvir, naux, seed, fvo_sigma, scale)
CASES = {
    "o5v19_canonical": (5, 19, 80, 0, 0.0, 1.0),      # water/cc-pVDZ scale workload
    "o5v19_fvo": (5, 19, 80, 0, 1e-3, 1.0),
    "o4v9_fvo": (4, 9, 30, 1, 1e-3, 1.0),
    "o3v4_fvo": (3, 4, 20, 2, 1e-3, 1.0),
    "o1v1": (1, 1, 4, 3, 1e-3, 1.0),                   # smallest possible
    "o1v5": (1, 5, 8, 4, 1e-3, 1.0),
    "o6v2": (6, 2, 10, 5, 1e-3, 1.0),                  # nvir < nocc
    "o7v13_scaled": (7, 13, 40, 6, 1e-3, 0.05),        # |E| ~ 1e-6 variant
}


# LNO fragment cases, name: (nocc, nvir, naux, seed, nlo); the projector is
# mat = ulo^T ulo for a seeded ulo[nlo, nocc] (pyscfad/lno/ccsd_t.py:42)
LNO_CASES = {
    "lno_o3v5": (3, 5, 20, 11, 1),
    "lno_o4v9": (4, 9, 30, 12, 2),
    "lno_o5v19": (5, 19, 60, 13, 2),   # three virtual blocks (16, 2, 1): ragged chunks
    "lno_o6v2": (6, 2, 10, 14, 3),     # nvir < nocc
}


def lno_projector(nocc, nlo, seed):
    rng = np.random.default_rng(1000 + seed)
    ulo = np.linalg.qr(rng.normal(size=(nocc, nocc)))[0][:nlo]
    return ulo.T @ ulo


def main_lno():
    for name, (o, v, naux, seed, nlo) in LNO_CASES.items():
        inp = make_inputs(o, v, naux, seed=seed, fvo_sigma=1e-3)
        mat = lno_projector(o, nlo, seed)
        e, g = O.ref_lno_energy_vjp(inp, mat, ybar=1.0)
        cot = O.reference_cotangents(g, o, v)
        out = dict(nocc=o, nvir=v, naux=naux, seed=seed, nlo=nlo, e=e, in_mat=mat, grad_mat=g["mat"])
        for k in O.GRAD_KEYS:
            out["in_" + k] = getattr(inp, k)
            out["grad_" + k] = g[k]
        out["cot_ovvv_tril"] = cot["ovvv"]
        out["in_ovvv_tril"] = inp.ovvv_tril()
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{name}: E = {e:.15g}  -> {os.path.relpath(path, ROOT)}")


# DF cases, name: (nocc, nvir, naux, seed): inputs given as the DF factors
DF_CASES = {
    "df_o4v9": (4, 9, 30, 21),
    "df_o5v19": (5, 19, 60, 22),
}


def main_df():
    from pyscfad_b200.synthetic import make_df_inputs
    for name, (o, v, naux, seed) in DF_CASES.items():
        inp, Lov, Lvv = make_df_inputs(o, v, naux, seed=seed, fvo_sigma=1e-3)
        e, g = O.ref_energy_vjp(inp, ybar=1.0)
        cot = O.reference_cotangents(g, o, v)
        Lov_bar, Lvv_bar = O.df_factor_grads(cot["ovvv"], Lov, Lvv)
        out = dict(nocc=o, nvir=v, naux=naux, seed=seed, e=e, in_Lov=Lov, in_Lvv=Lvv, grad_Lov=Lov_bar,
                   grad_Lvv=Lvv_bar, cot_ovvv_tril=cot["ovvv"], in_ovvv_tril=inp.ovvv_tril())
        for k in O.GRAD_KEYS:
            if k != "ovvv":
                out["in_" + k] = getattr(inp, k)
                out["grad_" + k] = g[k]
        out["in_ovvv"] = inp.ovvv
        out["grad_ovvv"] = g["ovvv"]
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{name}: E = {e:.15g}  -> {os.path.relpath(path, ROOT)}")


def main():
    if not O.ref_available():
        O.build()
    assert O.ref_available(), "reference sources missing; fixtures cannot be regenerated"
    for name, (o, v, naux, seed, fs, scale) in CASES.items():
        inp = make_inputs(o, v, naux, seed=seed, fvo_sigma=fs, scale=scale)
        e, g = O.ref_energy_vjp(inp, ybar=1.0)
        cot = O.reference_cotangents(g, o, v)
        out = dict(nocc=o, nvir=v, naux=naux, seed=seed, fvo_sigma=fs, scale=scale, e=e)
        for k in O.GRAD_KEYS:
            out["in_" + k] = getattr(inp, k)
            out["grad_" + k] = g[k]
        out["cot_ovvv_tril"] = cot["ovvv"]
        out["in_ovvv_tril"] = inp.ovvv_tril()
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{name}: E = {e:.15g}  -> {os.path.relpath(path, ROOT)}")


if __name__ == "__main__":
    if "--lno" in sys.argv:
        main_lno()
    elif "--df" in sys.argv:
        main_df()
    else:
        main()
        main_lno()
        main_df()
