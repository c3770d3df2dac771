"""DF-factor entry points (triples_energy_df / triples_energy_vjp_df): ovvv
built on the device from Lov and the packed Lvv as pyscfad's DF ERIs build it
(dfccsd.py:77-88), gradients returned for the factors.  Against the reference
golden vectors (factor gradients by the chain rule of the reference's packed
ovvv cotangent) and against the ovvv-input path on the same inputs."""
import numpy as np
import pytest
import torch

from pyscfad_b200 import triples
from pyscfad_b200.synthetic import make_df_inputs
from tests import golden_util as G

pytestmark = pytest.mark.gpu

TOL = {"fp64": (1e-12, 1e-10), "mixed": (1e-6, 1e-5), "mixed_bf16": (1e-4, 1e-3)}
DF_KEYS = ("mo_energy", "t1", "t2", "ovoo", "ovov", "Lov", "Lvv", "fvo")


def _relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-7))


def _run_df(z, precision, ybar=1.0):
    args = [z["in_" + k] for k in ("mo_energy", "t1", "t2", "ovoo", "ovov", "Lov", "Lvv", "fvo")]
    e, g = triples.energy_vjp_df(*args, ybar=ybar, precision=precision, device="cuda")
    torch.cuda.synchronize()
    return float(e), {k: v.cpu().numpy() for k, v in g.items()}


@pytest.mark.parametrize("name", G.df_names())
@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed_bf16"])
def test_df_matches_reference_golden(name, precision):
    _, e_ref, g_ref, z = G.load(name)
    te, tg = TOL[precision]
    e, g = _run_df(z, precision)
    assert abs(e - e_ref) <= te * max(1.0, abs(e_ref)) if precision == "fp64" else abs(e - e_ref) <= te * abs(e_ref)
    for k in DF_KEYS:
        ref = z["grad_" + k]
        assert _relerr(g[k], ref) < tg, k


def test_df_equals_ovvv_input_path():
    """Same inputs through the ovvv path: energies and shared gradients agree, and
    the factor gradients are the chain rule of the packed ovvv cotangent."""
    inp, Lov, Lvv = make_df_inputs(6, 33, 70, seed=9, fvo_sigma=1e-3)
    e_d, g_d = _run_df({"in_mo_energy": inp.mo_energy, "in_t1": inp.t1, "in_t2": inp.t2, "in_ovoo": inp.ovoo,
                        "in_ovov": inp.ovov, "in_Lov": Lov, "in_Lvv": Lvv, "in_fvo": inp.fvo}, "fp64", ybar=-0.5)
    e_o, g_o = triples.energy_vjp(inp.mo_energy, inp.t1, inp.t2, inp.ovoo, inp.ovov, inp.ovvv_tril(), inp.fvo,
                                  ybar=-0.5, device="cuda")
    g_o = {k: v.cpu().numpy() for k, v in g_o.items()}
    assert abs(e_d - float(e_o)) <= 1e-12 * abs(float(e_o))
    for k in ("mo_energy", "t1", "t2", "ovoo", "ovov", "fvo"):
        assert _relerr(g_d[k], g_o[k]) < 1e-10, k
    G_ = g_o["ovvv"].reshape(Lov.shape[1], Lvv.shape[1])
    assert _relerr(g_d["Lov"], Lvv @ G_.T) < 1e-10
    assert _relerr(g_d["Lvv"], Lov @ G_) < 1e-10
    e0 = triples.energy_df(inp.mo_energy, inp.t1, inp.t2, inp.ovoo, inp.ovov, Lov, Lvv, inp.fvo, device="cuda")
    assert abs(float(e0) - e_d) <= 1e-12 * abs(e_d)


def test_df_single_auxiliary_function():
    """naux = 1: ovvv of rank one; the factor gradients are still the chain rule."""
    inp, Lov, Lvv = make_df_inputs(3, 7, 1, seed=4, fvo_sigma=1e-3)
    z = {"in_mo_energy": inp.mo_energy, "in_t1": inp.t1, "in_t2": inp.t2, "in_ovoo": inp.ovoo,
         "in_ovov": inp.ovov, "in_Lov": Lov, "in_Lvv": Lvv, "in_fvo": inp.fvo}
    e_d, g_d = _run_df(z, "fp64")
    e_o, g_o = triples.energy_vjp(inp.mo_energy, inp.t1, inp.t2, inp.ovoo, inp.ovov, inp.ovvv_tril(), inp.fvo,
                                  device="cuda")
    G_ = g_o["ovvv"].cpu().numpy().reshape(Lov.shape[1], Lvv.shape[1])
    assert abs(e_d - float(e_o)) <= 1e-12 * max(abs(float(e_o)), 1e-12)
    assert _relerr(g_d["Lov"], Lvv @ G_.T) < 1e-10
    assert _relerr(g_d["Lvv"], Lov @ G_) < 1e-10
