"""Batched mode: many uneven (T) problems replayed as one CUDA graph give the
same energies and gradients as one call per problem, with both engines (the
library's batched entry points, one launch per kernel kind and chunk step
over all problems; and one call per problem over several streams), and the
reference's own energies and gradients on the golden problems."""
import numpy as np
import pytest
import torch

from pyscfad_b200 import triples
from pyscfad_b200.batched import Autotuner, BatchedTriples
from pyscfad_b200.synthetic import make_inputs

pytestmark = pytest.mark.gpu

SHAPES = [(4, 20), (6, 27), (5, 33), (8, 24), (4, 41), (7, 20)]
# the batch engine takes every epilogue item through the generic kernel (single calls
# send the all-distinct ones to the persistent one): same math, FP32 rounding may differ
TOL = {"fp64": (1e-12, 1e-10), "mixed": (1e-10, 1e-6), "mixed_bf16": (1e-10, 1e-6)}


def _problems(seed0=100):
    out = []
    for i, (o, v) in enumerate(SHAPES):
        inp = make_inputs(o, v, 4 * (o + v), seed=seed0 + i, fvo_sigma=1e-3)
        out.append({"mo_energy": inp.mo_energy, "t1": inp.t1, "t2": inp.t2, "ovoo": inp.ovoo,
                    "ovov": inp.ovov, "ovvv": inp.ovvv_tril(), "fvo": inp.fvo})
    return out


def _relerr(a, b):
    a, b = a.cpu().numpy(), b.cpu().numpy()
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-7))


def _single(p, precision, tv):
    e, g = triples.energy_vjp(*(p[k] for k in triples.KEYS), precision=precision, device="cuda", block_size=tv)
    return float(e), g


@pytest.mark.parametrize("precision,engine", [("fp64", "lanes"), ("fp64", "batch"), ("mixed", "lanes"),
                                              ("mixed", "batch"), ("mixed_bf16", "batch")])
def test_graph_batch_matches_single_calls(precision, engine):
    probs = _problems()
    bt = BatchedTriples(probs, precision=precision, lanes=3, autotuner=Autotuner(), engine=engine)
    etol, gtol = TOL[precision]
    for _ in range(2):   # two replays of the same graph
        bt.run()
        bt.check()
        for p, prob, (e, g) in zip(probs, bt.problems, bt.results()):
            e_ref, g_ref = _single(p, precision, prob.tv)
            assert abs(e - e_ref) <= etol * abs(e_ref)
            for k in triples.KEYS:
                assert _relerr(g[k], g_ref[k]) < gtol, k


def test_graph_batch_update_inputs():
    probs = _problems()
    bt = BatchedTriples(probs, precision="fp64", lanes=2, tune=False)
    bt.run()
    e_old = bt.results()[2][0]
    new = _problems(seed0=500)[2]
    bt.update(2, new)
    bt.run()
    e_new = bt.results()[2][0]
    e_ref, _ = _single(new, "fp64", bt.problems[2].tv)   # fp64: the N tile does not apply
    assert abs(e_new - e_ref) <= 1e-12 * abs(e_ref)
    assert e_new != e_old


def test_autotuner_table_roundtrip(tmp_path):
    probs = _problems()[:2]
    path = str(tmp_path / "tune.json")
    at = Autotuner(path)
    BatchedTriples(probs, precision="fp64", lanes=1, autotuner=at)
    assert len(at.table) == 2
    assert all(tv in (4, 8, 16) and tn in (0, 128, 256) for tv, tn in at.table.values())
    at.save()
    assert Autotuner(path).table == at.table


@pytest.mark.parametrize("precision,etol,gtol", [("fp64", 1e-12, 1e-10), ("mixed", 1e-6, 1e-5)])
def test_batch_engine_matches_reference_golden(precision, etol, gtol):
    """The golden problems of the reference's own kernels (tests/golden), run as
    one batch: every problem's E(T) and gradients against the reference."""
    from tests import golden_util as G

    names = ["o5v19_fvo", "o4v9_fvo", "o3v4_fvo", "o1v5", "o6v2", "o7v13_scaled"]
    probs, refs = [], []
    for nm in names:
        inp, e_ref, g_ref, z = G.load(nm)
        probs.append({"mo_energy": inp.mo_energy, "t1": inp.t1, "t2": inp.t2, "ovoo": inp.ovoo,
                      "ovov": inp.ovov, "ovvv": inp.ovvv_tril(), "fvo": inp.fvo})
        refs.append((e_ref, g_ref, z))
    bt = BatchedTriples(probs, precision=precision, tune=False, engine="batch")
    bt.run()
    bt.check()
    for nm, (e, g), (e_ref, g_ref, z) in zip(names, bt.results(), refs):
        assert abs(e - e_ref) <= etol * max(abs(e_ref), 1.0), nm   # o1v5: E(T) is rounding noise (1e-21)
        assert _relerr(g["ovvv"], torch.as_tensor(z["cot_ovvv_tril"])) < gtol, nm
        for k in ("mo_energy", "t1", "t2", "ovoo", "ovov", "fvo"):
            assert _relerr(g[k], torch.as_tensor(g_ref[k])) < gtol, (nm, k)
