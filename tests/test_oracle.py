"""The CPU oracle, pinned against the reference's own C kernels.

Golden fixtures come from the reference library compiled unchanged from
pyscfadlib/pyscfadlib/vjp/cc/*.c (tests/golden/make_golden.py).  Tolerances
are FP64 summation-order level.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from pyscfad_b200.synthetic import make_inputs
from tests import golden_util as G

HERE = os.path.dirname(os.path.abspath(__file__))


def _relerr(a, b):
    # exact cancellations (nocc == 1 gives E = 0) leave ~1e-22 rounding noise
    scale = max(np.abs(b).max(), 1e-7)
    return np.abs(a - b).max() / scale


@pytest.mark.parametrize("name", G.names())
def test_oracle_matches_reference_golden(name):
    inp, e_ref, g_ref, _ = G.load(name)
    e, g = O.oracle_energy_vjp(inp, ybar=1.0)
    assert abs(e - e_ref) <= 1e-12 * max(1.0, abs(e_ref))
    for k in G.KEYS:
        if np.abs(g_ref[k]).max() == 0:
            assert np.abs(g[k]).max() < 1e-14
        else:
            assert _relerr(g[k], g_ref[k]) < 1e-11, k


@pytest.mark.parametrize("name", ["o3v4_fvo", "o4v9_fvo", "o6v2"])
def test_numpy_restatement_matches_golden(name):
    inp, e_ref, _, _ = G.load(name)
    assert abs(O.np_energy(inp) - e_ref) <= 1e-12 * max(1.0, abs(e_ref))


@pytest.mark.parametrize("name", G.names())
def test_packed_ovvv_cotangent_fold(name):
    _, _, g_ref, z = G.load(name)
    assert np.allclose(O.fold_ovvv_tril(g_ref["ovvv"]), z["cot_ovvv_tril"], rtol=0, atol=1e-15)


def test_reference_library_reproduces_golden():
    if not O.ref_available():
        pytest.skip("reference library not built on this machine")
    inp, e_ref, g_ref, _ = G.load("o4v9_fvo")
    e, g = O.ref_energy_vjp(inp)
    assert abs(e - e_ref) < 1e-13
    for k in G.KEYS:
        assert _relerr(g[k], g_ref[k]) < 1e-12


def test_slices_sum_to_total():
    inp, e_ref, g_ref, _ = G.load("o5v19_fvo")
    parts = [O.oracle_energy_vjp(inp, a0=a0, a1=a1) for a0, a1 in [(0, 7), (7, 15), (15, 19)]]
    assert abs(sum(p[0] for p in parts) - e_ref) < 1e-12 * abs(e_ref)
    for k in G.KEYS:
        tot = sum(p[1][k] for p in parts)
        assert _relerr(tot, g_ref[k]) < 1e-11


def test_oracle_gradient_central_differences():
    """Central FD (h=1e-4, relative) on a few entries of every input."""
    inp = make_inputs(4, 7, 24, seed=11, fvo_sigma=1e-3)
    _, g = O.oracle_energy_vjp(inp)
    rng = np.random.default_rng(0)
    for k in G.KEYS:
        arr = getattr(inp, k)
        flat = arr.reshape(-1)
        for idx in rng.choice(flat.size, size=3, replace=False):
            x0 = flat[idx]
            h = 1e-4 * max(abs(x0), 1e-2)
            flat[idx] = x0 + h
            ep, _ = O.oracle_energy_vjp(inp, want_grad=False)
            flat[idx] = x0 - h
            em, _ = O.oracle_energy_vjp(inp, want_grad=False)
            flat[idx] = x0
            fd = (ep - em) / (2 * h)
            an = g[k].reshape(-1)[idx]
            assert abs(fd - an) <= 1e-6 * max(abs(an), np.abs(g[k]).max() * 1e-3), (k, idx, fd, an)


# ---- LNO fragment (T): projector mat on the first occupied index ----
_LNO_KEYS = ("mat",) + G.KEYS


@pytest.mark.parametrize("name", G.lno_names())
def test_lno_numpy_restatement_matches_reference_golden(name):
    inp, e_ref, g_ref, z = G.load(name)
    e, g = O.np_lno_energy_vjp(inp, z["in_mat"], ybar=1.0)
    assert abs(e - e_ref) <= 1e-12 * max(1e-3, abs(e_ref))
    for k in _LNO_KEYS:
        assert _relerr(g[k], g_ref[k]) < 1e-11, k
    assert np.allclose(O.fold_ovvv_tril(g_ref["ovvv"]), z["cot_ovvv_tril"], rtol=0, atol=1e-15)


def test_lno_identity_projector_is_canonical():
    inp, e_ref, g_ref, _ = G.load("o4v9_fvo")
    e, g = O.np_lno_energy_vjp(inp, np.eye(inp.nocc), ybar=1.0)
    assert abs(e - e_ref) <= 1e-12 * abs(e_ref)
    for k in G.KEYS:
        assert _relerr(g[k], g_ref[k]) < 1e-11, k


def test_lno_reference_library_reproduces_golden():
    if not O.ref_available():
        pytest.skip("reference library not built on this machine")
    inp, e_ref, g_ref, z = G.load("lno_o4v9")
    e, g = O.ref_lno_energy_vjp(inp, z["in_mat"], ybar=1.0)
    assert abs(e - e_ref) < 1e-15
    for k in _LNO_KEYS:
        assert _relerr(g[k], g_ref[k]) < 1e-13, k


def test_lno_projector_gradient_central_differences():
    """dE/dmat by central differences (E is linear in mat: exact up to rounding)."""
    inp, _, g_ref, z = G.load("lno_o3v5")
    mat = z["in_mat"].copy()
    for (l, i) in [(0, 0), (1, 2), (2, 1)]:
        h = 1e-3
        mat[l, i] += h
        ep, _ = O.np_lno_energy_vjp(inp, mat, want_grad=False)
        mat[l, i] -= 2 * h
        em, _ = O.np_lno_energy_vjp(inp, mat, want_grad=False)
        mat[l, i] += h
        assert abs((ep - em) / (2 * h) - g_ref["mat"][l, i]) < 1e-12 * max(1.0, abs(g_ref["mat"][l, i]))


# ---- DF factors: ovvv_tril = Lov^T Lvv_tril (dfccsd.py:77-88) ----
@pytest.mark.parametrize("name", ["df_o4v9"])
def test_df_factor_gradients_match_finite_differences(name):
    """Chain rule of the DF producer: central differences of E(T) (oracle) in a
    few Lov and packed-Lvv entries against the fixture's factor gradients."""
    from pyscfad_b200.synthetic import TriplesInputs
    _, e_ref, g_ref, z = G.load(name)
    Lov, Lvv = z["in_Lov"].copy(), z["in_Lvv"].copy()
    o, v = int(z["nocc"]), int(z["nvir"])
    il, jl = np.tril_indices(v)

    def energy(Lov_, Lvv_):
        tril = (Lov_.T @ Lvv_).reshape(o, v, -1)
        full = np.zeros((o, v, v, v))
        full[:, :, il, jl] = tril
        full[:, :, jl, il] = tril
        inp = TriplesInputs(z["in_mo_energy"], z["in_t1"], z["in_t2"], z["in_ovoo"], z["in_ovov"], full, z["in_fvo"])
        return O.oracle_energy_vjp(inp, want_grad=False)[0]

    assert abs(energy(Lov, Lvv) - e_ref) <= 1e-12 * abs(e_ref)
    rng = np.random.default_rng(3)
    for arr, gkey in ((Lov, "grad_Lov"), (Lvv, "grad_Lvv")):
        flat = arr.reshape(-1)
        for idx in rng.choice(flat.size, size=3, replace=False):
            x0 = flat[idx]
            h = 1e-4 * max(abs(x0), 1e-2)
            flat[idx] = x0 + h
            ep = energy(Lov, Lvv)
            flat[idx] = x0 - h
            em = energy(Lov, Lvv)
            flat[idx] = x0
            fd = (ep - em) / (2 * h)
            ref = z[gkey].reshape(-1)[idx]
            assert abs(fd - ref) <= 1e-6 * max(abs(ref), 1e-3 * np.abs(z[gkey]).max()), (gkey, idx, fd, ref)


@pytest.mark.parametrize("name", ["df_o4v9", "df_o5v19"])
def test_df_fixture_is_the_factor_chain_of_the_packed_cotangent(name):
    _, _, _, z = G.load(name)
    lb, vb = O.df_factor_grads(z["cot_ovvv_tril"], z["in_Lov"], z["in_Lvv"])
    assert np.allclose(lb, z["grad_Lov"], rtol=0, atol=1e-14 * np.abs(lb).max())
    assert np.allclose(vb, z["grad_Lvv"], rtol=0, atol=1e-14 * np.abs(vb).max())
    o, v = int(z["nocc"]), int(z["nvir"])
    assert np.allclose((z["in_Lov"].T @ z["in_Lvv"]).reshape(o, v, -1), z["in_ovvv_tril"], rtol=0, atol=1e-14)


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("A", [0, 1, 2])
def test_reference_aslice_blocking_matches_oracle_slice(A):
    """tests/golden/make_slices.py drives the reference's ccsd_t_energy_vjp
    the way pyscfad/cc/ccsd_t.py:145-175 blocks it for one a-range; that slice
    equals our C restatement's slice a in [16A, 16A+16), and its energy follows
    from the gradients by Euler's theorem."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_slices", os.path.join(HERE, "golden", "make_slices.py"))
    M = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(M)
    inp = make_inputs(5, 40, 60, seed=3, fvo_sigma=1e-3)
    a0, a1 = 16 * A, min(40, 16 * A + 16)
    g = M.ref_vjp_aslice(inp, a0, a1)
    e_or, g_or = O.oracle_energy_vjp(inp, a0=a0, a1=a1)
    g_or = dict(g_or, ovvv=O.fold_ovvv_tril(g_or["ovvv"]))
    assert abs(M.euler_energy(inp, g) - e_or) <= 1e-13 * abs(e_or)
    for k in g:
        assert np.abs(g[k] - g_or[k]).max() <= 1e-13 * np.abs(g_or[k]).max(), k


def test_slice_fixture_is_consistent():
    z = np.load(os.path.join(HERE, "golden", "slice_o20v180_a3.npz"))
    assert int(z["a0"]) == 16 * int(z["block"]) and int(z["a1"]) == int(z["a0"]) + 16
    assert abs(float(z["e"]) - float(z["e_oracle"])) <= 1e-11 * abs(float(z["e"]))
    for k in ("t2", "ovoo", "ovov", "ovvv"):
        assert z["idx_" + k].size == z["val_" + k].size > 1000
        assert np.all(np.diff(z["idx_" + k]) > 0)
        assert np.abs(z["val_" + k]).max() <= float(z["norm_" + k])
