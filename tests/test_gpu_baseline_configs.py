"""Parity at the benchmark's own problem sizes (not only at golden-fixture
sizes):

* nocc=20, nvir=180 (naux 600): one 16-wide virtual slice of the E+VJP against
  the reference's own C kernels (tests/golden/slice_o20v180_a3.npz, made by
  tests/golden/make_slices.py), FP64 and mixed precision;
* nocc=20, nvir=180 in full: the mixed-precision gates against the FP64 path
  on the same inputs (relative dE and per-input gradient error <= 1e-6), and
  the absolute |dE| <= 1e-7 Eh gate on physically scaled factors
  (|E(T)| ~ 1e-2 Eh);
* nocc=40, nvir=360 (naux 1200): central finite differences (h = 1e-4) of the
  FP64 energy of one chunk slice on 64 t2 and 16 mo_energy entries against
  the FP64 and mixed-precision gradients of the same slice.
"""
import os

import numpy as np
import pytest

from pyscfad_b200 import triples
from pyscfad_b200.synthetic import make_inputs, make_inputs_torch

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
KEYS = triples.KEYS


def _packed(inp_dict):
    import torch

    v = inp_dict["t1"].shape[1]
    il, jl = torch.tril_indices(v, v, device=inp_dict["ovvv"].device)
    out = dict(inp_dict)
    out["ovvv"] = inp_dict["ovvv"][:, :, il, jl].contiguous()
    return out


@pytest.fixture(autouse=True)
def _release():
    yield
    triples.release_workspace()
    import torch

    torch.cuda.empty_cache()


@pytest.mark.parametrize("precision,etol,gtol", [("fp64", 1e-10, 1e-10), ("mixed", 1e-6, 1e-6)])
def test_c1_slice_matches_reference(precision, etol, gtol):
    import torch

    z = np.load(os.path.join(HERE, "golden", "slice_o20v180_a3.npz"))
    o, v, naux, seed = int(z["nocc"]), int(z["nvir"]), int(z["naux"]), int(z["seed"])
    A, tv = int(z["block"]), int(z["tv"])
    inp = make_inputs(o, v, naux, seed=seed, fvo_sigma=float(z["fvo_sigma"]))
    dev = torch.device("cuda")
    x = {k: torch.as_tensor(np.ascontiguousarray(getattr(inp, k)), device=dev) for k in KEYS if k != "ovvv"}
    x["ovvv"] = torch.as_tensor(inp.ovvv_tril(), device=dev)
    e, g = triples.energy_vjp(*(x[k] for k in KEYS), precision=precision, device=dev, block_size=tv,
                              chunk_range=(A, A + 1))
    e = float(e)
    e_ref = float(z["e"])
    assert abs(e - e_ref) <= etol * abs(e_ref), (e, e_ref)
    for k in ("mo_energy", "t1", "fvo"):
        ref = z["grad_" + k]
        got = g[k].cpu().numpy()
        assert np.abs(got - ref).max() <= gtol * np.abs(ref).max(), k
    for k in ("t2", "ovoo", "ovov", "ovvv"):
        flat = g[k].reshape(-1)
        idx = torch.as_tensor(z["idx_" + k], device=dev)
        got = flat[idx].cpu().numpy()
        ref = z["val_" + k]
        assert np.abs(got - ref).max() <= gtol * np.abs(ref).max(), k
        # size-independent: the 2-norm of the whole gradient
        nrm = float(torch.linalg.vector_norm(flat))
        assert abs(nrm - float(z["norm_" + k])) <= max(gtol, 1e-12) * float(z["norm_" + k]), k


def _full(precision, inp):
    e, g = triples.energy_vjp(*(inp[k] for k in KEYS), precision=precision)
    return float(e), g


def test_c1_precision_gates_mixed_vs_fp64():
    """The headline precision gates on the full o=20, v=180 problem: mixed
    precision against the FP64 path on the same inputs."""
    import torch

    inp = _packed(make_inputs_torch(20, 180, 600, seed=5, fvo_sigma=1e-3))
    e64, g64 = _full("fp64", inp)
    em, gm = _full("mixed", inp)
    assert abs(em - e64) <= 1e-6 * abs(e64), (em, e64)
    for k in KEYS:
        ref = g64[k]
        err = float((gm[k] - ref).abs().max() / ref.abs().max())
        assert err <= 1e-6, (k, err)
    del g64, gm
    torch.cuda.empty_cache()


def test_c1_scaled_absolute_energy_gate():
    """Factors scaled so that |E(T)| ~ 1e-2 Eh (the size of a real molecule's
    triples correction): the absolute gate |dE| <= 1e-7 Eh of mixed vs FP64."""
    inp = _packed(make_inputs_torch(20, 180, 600, seed=6, fvo_sigma=1e-3, scale=4.3e-3))
    e64 = float(triples.energy(*(inp[k] for k in KEYS), precision="fp64"))
    em = float(triples.energy(*(inp[k] for k in KEYS), precision="mixed"))
    assert 1e-3 < abs(e64) < 1e-1, e64
    assert abs(em - e64) <= 1e-7, (em, e64)


def test_c2_slice_gradients_match_central_differences():
    """nocc=40, nvir=360: the FP64 energy of chunk slice (0, 1) (virtual
    indices a in [0, 16), a >= b >= c) under central differences h = 1e-4 on
    64 t2 entries and 16 mo_energy entries, against the FP64 and the
    mixed-precision gradients of the same slice.  E is quadratic in t2, so
    its central differences are exact up to rounding."""
    import torch

    o, v = 40, 360
    inp = _packed(make_inputs_torch(o, v, 1200, seed=3))
    args = [inp[k] for k in KEYS]
    sl = dict(chunk_range=(0, 1), block_size=16)
    _, g64 = triples.energy_vjp(*args, precision="fp64", **sl)
    _, gmx = triples.energy_vjp(*args, precision="mixed", **sl)
    rng = np.random.default_rng(11)
    # t2[i, j, a, b] with a in the slice's first block (b anywhere)
    t2_idx = [(int(rng.integers(o)), int(rng.integers(o)), int(rng.integers(16)), int(rng.integers(v)))
              for _ in range(64)]
    mo_idx = [int(i) for i in rng.choice(o, 8, replace=False)] + [o + int(i) for i in rng.choice(16, 8, replace=False)]
    h = 1e-4

    def e_slice():
        return float(triples.energy(*args, precision="fp64", **sl))

    def fd(t, idx):
        old = float(t[idx])
        t[idx] = old + h
        ep = e_slice()
        t[idx] = old - h
        em = e_slice()
        t[idx] = old
        return (ep - em) / (2 * h)

    fd_t2 = np.array([fd(inp["t2"], i) for i in t2_idx])
    fd_mo = np.array([fd(inp["mo_energy"], i) for i in mo_idx])
    for g, tol in ((g64, 1e-6), (gmx, 1e-6)):
        an_t2 = np.array([float(g["t2"][i]) for i in t2_idx])
        an_mo = np.array([float(g["mo_energy"][i]) for i in mo_idx])
        assert np.abs(an_t2 - fd_t2).max() <= tol * np.abs(fd_t2).max()
        assert np.abs(an_mo - fd_mo).max() <= tol * np.abs(fd_mo).max()
    assert np.abs(fd_t2).max() > 0 and np.abs(fd_mo).max() > 0
    del g64, gmx
    torch.cuda.empty_cache()
