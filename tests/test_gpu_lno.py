"""Parity of the CUDA LNO fragment (T) path (triples_lno_energy[_vjp]) with
the reference and the oracle, through the C ABI.

FP64 throughout: energies to 1e-12 relative, gradients (mat included) to
1e-10 relative (max abs error over max abs value).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from pyscfad_b200 import triples
from pyscfad_b200.synthetic import make_inputs
from tests import golden_util as G

pytestmark = pytest.mark.gpu

E_RTOL = 1e-12
G_RTOL = 1e-10
KEYS = ("mat",) + G.KEYS


def _relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-7))


def _run(inp, mat, packed=True, ybar=1.0, precision="fp64", block_size=0):
    ovvv = inp.ovvv_tril() if packed else inp.ovvv
    e, g = triples.lno_energy_vjp(mat, inp.mo_energy, inp.t1, inp.t2, inp.ovoo, inp.ovov, ovvv, inp.fvo,
                                  ybar=ybar, precision=precision, device="cuda", block_size=block_size)
    torch.cuda.synchronize()
    return float(e), {k: v.cpu().numpy() for k, v in g.items()}


@pytest.mark.parametrize("name", G.lno_names())
@pytest.mark.parametrize("packed", [True, False])
def test_lno_matches_reference_golden(name, packed):
    inp, e_ref, g_ref, z = G.load(name)
    e, g = _run(inp, z["in_mat"], packed)
    assert abs(e - e_ref) <= E_RTOL * max(1e-3, abs(e_ref))
    for k in KEYS:
        ref = z["cot_ovvv_tril"] if (k == "ovvv" and packed) else g_ref[k]
        assert _relerr(g[k], ref) < G_RTOL, k


# tensor-core contractions on 16-bit hi/lo splits, FP64 epilogue: the
# tolerances of the canonical mixed path
MIXED_TOL = {"mixed": (1e-6, 1e-5), "mixed_bf16": (1e-4, 1e-3)}


@pytest.mark.parametrize("name", ["lno_o4v9", "lno_o5v19"])
@pytest.mark.parametrize("precision", ["mixed", "mixed_bf16"])
def test_lno_mixed_matches_reference_golden(name, precision):
    inp, e_ref, g_ref, z = G.load(name)
    te, tg = MIXED_TOL[precision]
    e, g = _run(inp, z["in_mat"], packed=True, precision=precision)
    assert abs(e - e_ref) <= te * abs(e_ref), (e, e_ref)
    for k in KEYS:
        ref = z["cot_ovvv_tril"] if k == "ovvv" else g_ref[k]
        assert _relerr(g[k], ref) < tg, k


def test_lno_mixed_full_projector():
    """Mixed path with a full non-symmetric projector (scale bound with row/column sums != 1)."""
    inp = make_inputs(7, 24, 40, seed=3, fvo_sigma=1e-3)
    mat = np.random.default_rng(7).normal(size=(7, 7)) * 0.8
    e_ref, g_ref = _run(inp, mat, packed=False)
    e, g = _run(inp, mat, packed=False, precision="mixed")
    assert abs(e - e_ref) <= 1e-6 * abs(e_ref)
    for k in KEYS:
        assert _relerr(g[k], g_ref[k]) < 1e-5, k
    e0 = triples.lno_energy(mat, inp.mo_energy, inp.t1, inp.t2, inp.ovoo, inp.ovov, inp.ovvv, inp.fvo,
                            precision="mixed", device="cuda")
    assert abs(float(e0) - e) <= 1e-12 * abs(e)


def test_lno_energy_only_matches_vjp_energy():
    inp, e_ref, _, z = G.load("lno_o5v19")
    e = triples.lno_energy(z["in_mat"], inp.mo_energy, inp.t1, inp.t2, inp.ovoo, inp.ovov, inp.ovvv_tril(),
                           inp.fvo, device="cuda")
    assert abs(float(e) - e_ref) <= E_RTOL * abs(e_ref)


@pytest.mark.parametrize("tv", [1, 2, 4, 8])
def test_lno_block_sizes(tv):
    """Many chunks, degenerate (A == B, B == C) and ragged blocks."""
    inp, e_ref, g_ref, z = G.load("lno_o4v9")
    e, g = _run(inp, z["in_mat"], packed=False, block_size=tv)
    assert abs(e - e_ref) <= E_RTOL * abs(e_ref)
    for k in KEYS:
        assert _relerr(g[k], g_ref[k]) < G_RTOL, k


@pytest.mark.parametrize("o,v,ybar", [(2, 7, -1.7), (7, 12, 0.5)])
def test_lno_matches_numpy_oracle(o, v, ybar):
    """Full (non-symmetric, not PSD) projector and a non-unit seed."""
    inp = make_inputs(o, v, 30, seed=o + v, fvo_sigma=1e-3)
    mat = np.random.default_rng(o).normal(size=(o, o))
    e_ref, g_ref = O.np_lno_energy_vjp(inp, mat, ybar=ybar)
    e, g = _run(inp, mat, packed=False, ybar=ybar)
    assert abs(e - e_ref) <= E_RTOL * max(1e-3, abs(e_ref))
    for k in KEYS:
        assert _relerr(g[k], g_ref[k]) < G_RTOL, k


def test_lno_identity_projector_equals_canonical_path():
    """mat = I reproduces the canonical FP64 path on three virtual blocks (16, 16, 1)."""
    inp = make_inputs(6, 33, 60, seed=5, fvo_sigma=1e-3)
    e_l, g_l = _run(inp, np.eye(6))
    e_c, g_c = triples.energy_vjp(inp.mo_energy, inp.t1, inp.t2, inp.ovoo, inp.ovov, inp.ovvv_tril(), inp.fvo,
                                  device="cuda")
    assert abs(e_l - float(e_c)) <= E_RTOL * abs(float(e_c))
    for k in G.KEYS:
        assert _relerr(g_l[k], g_c[k].cpu().numpy()) < G_RTOL, k


def test_lno_mirror_kernel_autograd():
    """pyscfad_b200.lno.ccsd_t mirrors pyscfad.lno.ccsd_t: kernel() value and
    the autograd cotangents of _ccsd_t_energy in the reference layouts."""
    from pyscfad_b200.lno import ccsd_t as L

    inp, e_ref, g_ref, z = G.load("lno_o4v9")
    o, v = inp.nocc, inp.nvir
    dev = torch.device("cuda")
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev, requires_grad=True)
    mat, t1T, t2T = t(z["in_mat"]), t(inp.t1.T), t(inp.t2.transpose(2, 3, 1, 0))
    mo, fvo, ovoo, ovov, ovvv = t(inp.mo_energy), t(inp.fvo), t(inp.ovoo), t(inp.ovov), t(inp.ovvv_tril())
    e = L._ccsd_t_energy(mat, t1T, t2T, mo, fvo, ovoo, ovov, ovvv, 4000)
    (2.0 * e).backward()
    assert abs(float(e.detach()) - e_ref) <= E_RTOL * abs(e_ref)
    assert _relerr(mat.grad.cpu().numpy(), 2 * g_ref["mat"]) < G_RTOL
    assert _relerr(t1T.grad.cpu().numpy(), 2 * g_ref["t1"].T) < G_RTOL
    assert _relerr(t2T.grad.cpu().numpy(), 2 * g_ref["t2"].transpose(2, 3, 1, 0)) < G_RTOL
    assert _relerr(ovvv.grad.cpu().numpy(), 2 * z["cot_ovvv_tril"]) < G_RTOL
    assert _relerr(mo.grad.cpu().numpy(), 2 * g_ref["mo_energy"]) < G_RTOL
    bw = L._ccsd_t_energy_bwd(None, (z["in_mat"], inp.t1.T, inp.t2.transpose(2, 3, 1, 0), inp.mo_energy,
                                     inp.fvo, inp.ovoo, inp.ovov, inp.ovvv_tril()), 1.0)
    assert _relerr(bw[0], g_ref["mat"]) < G_RTOL and _relerr(bw[7], z["cot_ovvv_tril"]) < G_RTOL

    class _Eris:
        pass

    eris = _Eris()
    fock = np.zeros((o + v, o + v))
    fock[o:, :o] = inp.fvo
    eris.fock, eris.mo_energy, eris.ovoo, eris.ovov, eris.ovvv = fock, inp.mo_energy, inp.ovoo, inp.ovov, \
        inp.ovvv_tril()

    class _CC:
        t1, t2, max_memory = inp.t1, inp.t2, 4000

    # ulo with ulo^T ulo = mat: the fixture's projector is a rank-nlo orthogonal projector
    w, U = np.linalg.eigh(z["in_mat"])
    ulo = (U[:, w > 0.5]).T
    assert abs(L.kernel(_CC(), eris, ulo) - e_ref) <= 1e-11 * abs(e_ref)


@pytest.mark.parametrize("o,v", [(1, 1), (1, 6), (3, 1), (2, 2)])
def test_lno_smallest_shapes(o, v):
    """Degenerate sizes: one occupied or one virtual orbital (E vanishes
    analytically for nocc = 1 and the gradients are rounding noise there)."""
    inp = make_inputs(o, v, 8, seed=o * 10 + v, fvo_sigma=1e-3)
    mat = np.random.default_rng(o + v).normal(size=(o, o))
    e_ref, g_ref = O.np_lno_energy_vjp(inp, mat, ybar=1.3)
    e, g = _run(inp, mat, packed=True, ybar=1.3)
    assert abs(e - e_ref) <= 1e-12 * max(1e-3, abs(e_ref))
    scale = max(np.abs(g_ref["t2"]).max(), 1e-7)
    for k in KEYS:
        ref = O.fold_ovvv_tril(g_ref[k]) if k == "ovvv" else g_ref[k]
        assert np.abs(g[k] - ref).max() <= 1e-10 * max(np.abs(ref).max(), scale), k


def test_lno_zero_projector_and_zero_seed():
    """mat = 0: E = 0 and only mat_bar survives; ybar = 0: every gradient is zero."""
    inp, e_ref, g_ref, z = G.load("lno_o4v9")
    o = inp.nocc
    e, g = _run(inp, np.zeros((o, o)))
    assert e == 0.0
    _, g_np = O.np_lno_energy_vjp(inp, np.zeros((o, o)), ybar=1.0)
    assert _relerr(g["mat"], g_np["mat"]) < G_RTOL
    for k in G.KEYS:
        assert np.abs(g[k]).max() == 0.0, k
    e, g = _run(inp, z["in_mat"], ybar=0.0)
    assert abs(e - e_ref) <= E_RTOL * abs(e_ref)
    for k in KEYS:
        assert np.abs(g[k]).max() == 0.0, k


def test_lno_bf16_rank_one_projector():
    inp = make_inputs(5, 19, 40, seed=17, fvo_sigma=1e-3)
    u = np.random.default_rng(5).normal(size=5)
    mat = np.outer(u, u) / (u @ u)
    e_ref, g_ref = _run(inp, mat, packed=True)
    e, g = _run(inp, mat, packed=True, precision="mixed_bf16")
    assert abs(e - e_ref) <= 1e-4 * abs(e_ref)
    for k in KEYS:
        assert _relerr(g[k], g_ref[k]) < 1e-3, k


def test_lno_linear_in_projector_at_larger_size():
    """Size-independent checks where the oracle is too slow (o=12, v=64, several
    chunks per block edge): E is linear in mat, so E(a M1 + b M2) =
    a E(M1) + b E(M2) and mat_bar does not depend on mat; mat = I gives the
    canonical path's energy and gradients."""
    inp = make_inputs(12, 64, 120, seed=31, fvo_sigma=1e-3)
    rng = np.random.default_rng(12)
    m1, m2 = rng.normal(size=(12, 12)), rng.normal(size=(12, 12))
    e1, g1 = _run(inp, m1)
    e2, g2 = _run(inp, m2)
    e3, g3 = _run(inp, 0.5 * m1 - 2.0 * m2)
    assert abs(e3 - (0.5 * e1 - 2.0 * e2)) <= 1e-11 * (abs(e1) + 4 * abs(e2))
    assert _relerr(g3["mat"], g1["mat"]) < 1e-10 and _relerr(g2["mat"], g1["mat"]) < 1e-10
    for k in G.KEYS:
        assert _relerr(g3[k], 0.5 * g1[k] - 2.0 * g2[k]) < 1e-9, k
    e_i, g_i = _run(inp, np.eye(12))
    e_c, g_c = triples.energy_vjp(inp.mo_energy, inp.t1, inp.t2, inp.ovoo, inp.ovov, inp.ovvv_tril(), inp.fvo,
                                  device="cuda")
    assert abs(e_i - float(e_c)) <= 1e-12 * abs(float(e_c))
    for k in G.KEYS:
        assert _relerr(g_i[k], g_c[k].cpu().numpy()) < 1e-10, k


def test_lno_mirror_mixed_precision_keyword():
    from pyscfad_b200.lno import ccsd_t as L

    inp, e_ref, _, z = G.load("lno_o5v19")
    e = L._ccsd_t_energy(z["in_mat"], inp.t1.T, inp.t2.transpose(2, 3, 1, 0), inp.mo_energy, inp.fvo, inp.ovoo,
                         inp.ovov, inp.ovvv_tril(), None, precision="mixed")
    assert abs(float(e) - e_ref) <= 1e-6 * abs(e_ref)
