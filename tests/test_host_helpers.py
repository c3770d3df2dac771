"""Host-side helpers (no GPU): the chunk decomposition the Python side
mirrors, the DF synthetic inputs, and the bench's flop / byte accounting."""
import numpy as np
import pytest

import bench
from pyscfad_b200 import triples
from pyscfad_b200.synthetic import make_df_inputs, make_inputs


@pytest.mark.parametrize("v,tv", [(1, 16), (19, 16), (33, 16), (180, 16), (360, 16), (97, 8), (7, 4), (5, 1)])
def test_block_sizes_partition_the_virtual_range(v, tv):
    sizes = triples.block_sizes(v, tv)
    assert sum(sizes) == v
    assert sizes[: v // tv] == [tv] * (v // tv)
    rest = sizes[v // tv:]
    assert all(s & (s - 1) == 0 for s in sizes)            # powers of two
    assert rest == sorted(rest, reverse=True) and len(set(rest)) == len(rest)


@pytest.mark.parametrize("v", [19, 64, 180])
def test_chunk_fractions_partition_all_amplitudes(v):
    """Chunks A >= B >= C with all their distinct orderings hold every
    virtual triple exactly once: the fractions over a partition of the
    largest-block range add up to 1."""
    nb = len(triples.block_sizes(v))
    assert abs(triples.chunk_fraction(v, 0, nb) - 1.0) < 1e-12
    cut = nb // 2
    parts = triples.chunk_fraction(v, 0, cut) + triples.chunk_fraction(v, cut, nb)
    assert abs(parts - 1.0) < 1e-12


def test_df_inputs_are_the_factor_product_of_make_inputs():
    inp, Lov, Lvv = make_df_inputs(4, 9, 30, seed=5, fvo_sigma=1e-3)
    ref = make_inputs(4, 9, 30, seed=5, fvo_sigma=1e-3)
    assert Lov.shape == (30, 36) and Lvv.shape == (30, 45)
    assert np.allclose((Lov.T @ Lvv).reshape(4, 9, 45), ref.ovvv_tril(), rtol=0, atol=1e-15)
    for k in ("mo_energy", "t1", "t2", "ovoo", "ovov", "ovvv", "fvo"):
        assert np.array_equal(getattr(inp, k), getattr(ref, k)), k


def test_flop_and_byte_accounting():
    o, v = 40, 360
    f = bench.algorithmic_flops(o, v)
    assert f["step"] == 8.0 * o ** 3 * v ** 4
    # executed tensor work: W contraction + four adjoint contractions (no recompute)
    assert sum(f[k] for k in f if k != "step") == 6.0 * o ** 3 * v ** 4 + 6.0 * o ** 4 * v ** 3
    b64, b32 = bench.lno_pass_bytes(8), bench.lno_pass_bytes(4)
    assert b64["lno_tile_fwd"] == 24 and b32["lno_tile_fwd"] == 20
    assert b64["lno_tile_adj"] == 32 and b32["lno_tile_adj"] == 28
    assert b64["lno_projection"] == b32["lno_projection"] == 40
    assert b64["lno_vgrad"] == 16


@pytest.mark.parametrize("step_s", [0.5, 10.0, 40.0, 77.0, 300.0])
def test_step_plan_fits_the_wall_clock_budget(step_s):
    """The bench's plan: at least three warm-up steps when asked for >= 3, at
    least one timed and one e2e step, and no more steps than the budget holds."""
    budget, reserve, elapsed = 1450.0, 150.0, 60.0 + step_s
    warm, timed, e2e = bench.plan_steps(step_s, elapsed, 20, 5, budget, reserve)
    assert warm == 3 and 1 <= timed <= 20 and 1 <= e2e <= min(2, timed)
    if timed > 1:   # everything planned fits (one timed step is the floor)
        assert elapsed + (warm - 1 + timed + e2e) * step_s + reserve <= budget
    assert bench.plan_steps(step_s, 1.0, 4, 1, 1e9, 0.0) == (1, 4, 2)
