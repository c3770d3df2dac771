"""Golden vectors for one virtual slice of a BASELINE-size (T) problem, from
the reference's own C kernels (oracle/_ref/libcc_vjp_ref.so, compiled
unchanged from pyscfadlib/pyscfadlib/vjp/cc/*.c).

The reference slices its backward by job ranges (pyscfad/cc/ccsd_t.py:145-175):
for an a-range [a0, a1) it calls ccsd_t_energy_vjp once on the diagonal block
(a0, a1, a0, a1) and once per lower b-range (a0, a1, b0, b1) with b1 <= a0
(pyscfadlib/pyscfadlib/vjp/cc/ccsd_t_vjp.c:332-346, jobs from
_ccsd_t_gen_jobs, ccsd_t.c:6-72).  Together these cover every job
a >= b >= c with a in [a0, a1): with 16-wide virtual blocks, a in
[16A, 16A + 16) is exactly the chunk slice (A, A + 1) of triples_options.

A full o=20, v=180 gradient is far too large to commit, so the fixture holds
the slice energy, the small gradients in full (mo_energy, t1, fvo), seeded
samples of the large ones (t2, ovoo, ovov, packed ovvv) and the 2-norm of
every gradient.  The slice energy comes from the reference's gradients by
Euler's theorem: E(T) is homogeneous of degree 2 in (t1, t2) jointly (W and V
are linear in them), so E = (<t1, dE/dt1> + <t2, dE/dt2>) / 2; the script
checks that identity against our C restatement of the same slice.

    python tests/golden/make_slices.py      # writes tests/golden/slice_*.npz
"""
from __future__ import annotations

import ctypes
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from pyscfad_b200.synthetic import make_inputs  # noqa: E402

# name: (nocc, nvir, naux, seed, fvo_sigma, block A of 16 virtuals, samples per large gradient)
SLICES = {
    "slice_o20v180_a3": (20, 180, 600, 7, 1e-3, 3, 3000),
}
TV = 16


def ref_vjp_aslice(inp, a0, a1, ybar=1.0):
    """The reference's blocking for one a-range (ccsd_t.py:145-175) with one
    lower b-block [0, a0): gradients in the reference's internal layouts."""
    lib = O._lib("ref")
    o, v = inp.nocc, inp.nvir
    n = o + v
    t1T, t2T, vooo, vvop = O._ref_layouts(inp)
    mo_energy = np.ascontiguousarray(inp.mo_energy)
    fvo = np.ascontiguousarray(inp.fvo)
    bars = dict(mo_energy=np.zeros(n), t1T=np.zeros_like(t1T), t2T=np.zeros_like(t2T),
                vooo=np.zeros_like(vooo), fvo=np.zeros_like(fvo))
    vvop_bar = np.zeros_like(vvop)
    p = O._ptr

    def contract(b0, b1, row_a, col_a, row_b, col_b, bar):
        lib.ccsd_t_energy_vjp(
            p(mo_energy), p(t1T), p(t2T), p(vooo), p(fvo), ctypes.c_double(2.0 * ybar),
            ctypes.c_int(o), ctypes.c_int(v), ctypes.c_int(a0), ctypes.c_int(a1), ctypes.c_int(b0), ctypes.c_int(b1),
            p(row_a), p(col_a), p(row_b), p(col_b),
            p(bars["mo_energy"]), p(bars["t1T"]), p(bars["t2T"]), p(bars["vooo"]), p(bars["fvo"]),
            p(bar[0]), p(bar[1]), p(bar[2]), p(bar[3]))

    row_a = np.ascontiguousarray(vvop[a0:a1, :a1])
    row_a_bar = np.zeros_like(row_a)
    col_a = np.ascontiguousarray(vvop[:a0, a0:a1])
    col_a_bar = np.zeros_like(col_a)
    contract(a0, a1, row_a, col_a, row_a, col_a, (row_a_bar, col_a_bar, row_a_bar, col_a_bar))
    if a0 > 0:
        row_b = np.ascontiguousarray(vvop[0:a0, :a0])
        row_b_bar = np.zeros_like(row_b)
        contract(0, a0, row_a, col_a, row_b, row_b, (row_a_bar, col_a_bar, row_b_bar, row_b_bar))
        vvop_bar[0:a0, :a0] += row_b_bar
    vvop_bar[a0:a1, :a1] += row_a_bar
    vvop_bar[:a0, a0:a1] += col_a_bar
    g = dict(
        mo_energy=bars["mo_energy"],
        t1=np.ascontiguousarray(bars["t1T"].T),
        t2=np.ascontiguousarray(bars["t2T"].transpose(3, 2, 0, 1)),
        ovoo=np.ascontiguousarray(bars["vooo"].transpose(1, 0, 3, 2)),
        ovov=np.ascontiguousarray(vvop_bar[:, :, :, :o].transpose(2, 0, 3, 1)),
        ovvv=O.fold_ovvv_tril(vvop_bar[:, :, :, o:].transpose(2, 0, 3, 1)),
        fvo=bars["fvo"],
    )
    return g


def euler_energy(inp, g, ybar=1.0):
    return 0.5 * (float(np.vdot(inp.t1, g["t1"])) + float(np.vdot(inp.t2, g["t2"]))) / ybar


def make(name, check_oracle=True):
    o, v, naux, seed, fvo_sigma, A, nsamp = SLICES[name]
    t0 = time.time()
    inp = make_inputs(o, v, naux, seed=seed, fvo_sigma=fvo_sigma)
    a0, a1 = TV * A, min(v, TV * A + TV)
    g = ref_vjp_aslice(inp, a0, a1)
    e = euler_energy(inp, g)
    out = dict(nocc=o, nvir=v, naux=naux, seed=seed, fvo_sigma=fvo_sigma, block=A, tv=TV, a0=a0, a1=a1, e=e)
    for k in ("mo_energy", "t1", "fvo"):
        out["grad_" + k] = g[k]
    rng = np.random.default_rng(seed + 100)
    for k in ("t2", "ovoo", "ovov", "ovvv"):
        flat = g[k].reshape(-1)
        nz = np.flatnonzero(flat)
        idx = np.sort(rng.choice(nz, size=min(nsamp, nz.size), replace=False))
        out["idx_" + k] = idx.astype(np.int64)
        out["val_" + k] = flat[idx]
        out["norm_" + k] = float(np.linalg.norm(flat))
    for k in ("mo_energy", "t1", "fvo"):
        out["norm_" + k] = float(np.linalg.norm(g[k]))
    if check_oracle:
        e_or, _ = O.oracle_energy_vjp(inp, want_grad=False, a0=a0, a1=a1)
        out["e_oracle"] = e_or
        assert abs(e_or - e) <= 1e-11 * abs(e), (e_or, e)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: E(slice) = {e:.12e}  ({time.time() - t0:.0f} s)")


if __name__ == "__main__":
    for name in SLICES:
        make(name)
