"""Parity of the CUDA (T) path with the oracle, through the C ABI.

FP64 path: energies to 1e-12 relative, gradients to 1e-10 relative (max
abs error over max abs value) -- FP64 summation-order level.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from pyscfad_b200 import triples
from pyscfad_b200.synthetic import make_inputs
from tests import golden_util as G

pytestmark = pytest.mark.gpu

FP64_E_RTOL = 1e-12
FP64_G_RTOL = 1e-10


def _relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-7))


def _run(inp, packed, precision="fp64", ybar=1.0, **opt):
    ovvv = inp.ovvv_tril() if packed else inp.ovvv
    e, g = triples.energy_vjp(inp.mo_energy, inp.t1, inp.t2, inp.ovoo, inp.ovov, ovvv, inp.fvo,
                              ybar=ybar, precision=precision, device="cuda", **opt)
    torch.cuda.synchronize()
    return float(e), {k: v.cpu().numpy() for k, v in g.items()}


@pytest.mark.parametrize("name", G.names())
@pytest.mark.parametrize("packed", [True, False])
def test_fp64_matches_reference_golden(name, packed):
    inp, e_ref, g_ref, z = G.load(name)
    e, g = _run(inp, packed)
    assert abs(e - e_ref) <= FP64_E_RTOL * max(1.0, abs(e_ref))
    for k in G.KEYS:
        ref = z["cot_ovvv_tril"] if (k == "ovvv" and packed) else g_ref[k]
        assert _relerr(g[k], ref) < FP64_G_RTOL, k


@pytest.mark.parametrize("tv", [1, 2, 4, 8, 16])
def test_fp64_block_sizes(tv):
    """Chunk decomposition with degenerate (A==B, B==C) and ragged blocks."""
    inp, e_ref, g_ref, _ = G.load("o4v9_fvo")
    e, g = _run(inp, packed=False, block_size=tv)
    assert abs(e - e_ref) <= FP64_E_RTOL * abs(e_ref)
    for k in G.KEYS:
        assert _relerr(g[k], g_ref[k]) < FP64_G_RTOL, k


def test_energy_only_entry_point_matches():
    inp, e_ref, _, _ = G.load("o5v19_fvo")
    e = triples.energy(inp.mo_energy, inp.t1, inp.t2, inp.ovoo, inp.ovov, inp.ovvv_tril(), inp.fvo,
                       device="cuda")
    assert abs(float(e) - e_ref) <= FP64_E_RTOL * abs(e_ref)


def test_ybar_scales_gradients():
    inp, _, g_ref, _ = G.load("o3v4_fvo")
    _, g = _run(inp, packed=False, ybar=-2.5)
    for k in G.KEYS:
        assert _relerr(g[k], -2.5 * g_ref[k]) < FP64_G_RTOL


@pytest.mark.parametrize("o,v,naux,seed", [(6, 23, 40, 7), (8, 12, 30, 8), (2, 40, 30, 9)])
def test_fp64_random_vs_oracle(o, v, naux, seed):
    inp = make_inputs(o, v, naux, seed=seed, fvo_sigma=1e-3)
    e_ref, g_ref = O.oracle_energy_vjp(inp)
    e, g = _run(inp, packed=True)
    assert abs(e - e_ref) <= FP64_E_RTOL * abs(e_ref)
    g_ref = dict(g_ref, ovvv=O.fold_ovvv_tril(g_ref["ovvv"]))
    for k in G.KEYS:
        assert _relerr(g[k], g_ref[k]) < FP64_G_RTOL, k


def test_repeated_calls_are_stable():
    inp, e_ref, _, _ = G.load("o4v9_fvo")
    es = [_run(inp, packed=True)[0] for _ in range(3)]
    assert max(es) - min(es) <= 1e-14 * abs(e_ref)


@pytest.mark.parametrize("tv", [4, 16])
def test_fp64_chunk_slices_partition_the_problem(tv):
    """Energies and gradients of chunk slices that partition the virtual
    blocks add up to the full result (the basis of slice timing)."""
    inp, e_ref, g_ref, _ = G.load("o5v19_fvo")
    nb = len(triples.block_sizes(inp.t1.shape[1], tv))
    cut = nb // 2
    parts = [_run(inp, packed=True, block_size=tv, chunk_range=(a0, a1)) for a0, a1 in ((0, cut), (cut, nb))]
    e = parts[0][0] + parts[1][0]
    assert abs(e - e_ref) <= FP64_E_RTOL * abs(e_ref)
    for k in G.KEYS:
        if k == "ovvv":
            continue
        assert _relerr(parts[0][1][k] + parts[1][1][k], g_ref[k]) < FP64_G_RTOL, k
    assert abs(parts[0][0]) > 0 and abs(parts[1][0]) > 0
