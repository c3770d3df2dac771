"""The canonical Python mirror of pyscfad.cc.ccsd_t (pyscfad/cc/ccsd_t.py:28-192):
``kernel(mycc, eris)``, ``_ccsd_t_energy_vjp`` and the autograd wrapper, on a
tiny ERI namespace holding the reference's golden inputs (o5 v19, non-canonical
fvo, packed DF-style ovvv).  Checked against the reference's own energy and
cotangents: fock_bar carries only the vo block (ccsd_t.py:181-182), ovvv_bar
is the packed tril fold (ccsd_t.py:184-191)."""
from types import SimpleNamespace

import numpy as np
import pytest

from pyscfad_b200.cc import ccsd_t
from tests import golden_util as G

pytestmark = pytest.mark.gpu

E_RTOL, G_RTOL = 1e-12, 1e-10


def _relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-7))


def _eris_and_cc(inp):
    o, v = inp.t1.shape
    n = o + v
    fock = np.zeros((n, n))
    fock[np.arange(n), np.arange(n)] = inp.mo_energy
    fock[o:, :o] = inp.fvo
    fock[:o, o:] = inp.fvo.T
    eris = SimpleNamespace(fock=fock, mo_energy=inp.mo_energy, ovoo=inp.ovoo, ovov=inp.ovov,
                           ovvv=inp.ovvv_tril(), oooo=np.zeros((o, o, o, o)))
    mycc = SimpleNamespace(t1=inp.t1, t2=inp.t2, max_memory=4000)
    return eris, mycc


def test_kernel_returns_the_reference_energy():
    inp, e_ref, _, _ = G.load("o5v19_fvo")
    eris, mycc = _eris_and_cc(inp)
    e = ccsd_t.kernel(mycc, eris)
    assert isinstance(e, float)
    assert abs(e - e_ref) <= E_RTOL * abs(e_ref)


@pytest.mark.parametrize("et_bar", [1.0, -0.75])
def test_energy_vjp_cotangents(et_bar):
    inp, _, g_ref, z = G.load("o5v19_fvo")
    eris, _ = _eris_and_cc(inp)
    o, v = inp.t1.shape
    t1_bar, t2_bar, fock_bar, mo_bar, ovoo_bar, ovov_bar, ovvv_bar = ccsd_t._ccsd_t_energy_vjp(
        eris, inp.t1, inp.t2, et_bar)
    assert fock_bar.shape == (o + v, o + v)
    assert _relerr(fock_bar[o:, :o], et_bar * g_ref["fvo"]) < G_RTOL
    rest = fock_bar.copy()
    rest[o:, :o] = 0.0
    assert not rest.any()                          # only the vo block is read by (T)
    assert ovvv_bar.shape == eris.ovvv.shape       # packed, like eris.ovvv
    assert _relerr(ovvv_bar, et_bar * z["cot_ovvv_tril"]) < G_RTOL
    for got, k in ((t1_bar, "t1"), (t2_bar, "t2"), (mo_bar, "mo_energy"), (ovoo_bar, "ovoo"),
                   (ovov_bar, "ovov")):
        assert _relerr(got, et_bar * g_ref[k]) < G_RTOL, k


@pytest.mark.parametrize("precision,etol,gtol", [("fp64", E_RTOL, G_RTOL), ("mixed", 1e-6, 1e-5)])
def test_autograd_through_kernel(precision, etol, gtol):
    import torch

    inp, e_ref, g_ref, z = G.load("o5v19_fvo")
    eris, mycc = _eris_and_cc(inp)
    dev = torch.device("cuda")
    leaves = {k: torch.tensor(np.ascontiguousarray(getattr(eris, k)), device=dev, requires_grad=True)
              for k in ("fock", "mo_energy", "ovoo", "ovov", "ovvv")}
    t1 = torch.tensor(inp.t1, device=dev, requires_grad=True)
    t2 = torch.tensor(inp.t2, device=dev, requires_grad=True)
    teris = SimpleNamespace(**leaves, oooo=torch.zeros((1,), device=dev))
    e = ccsd_t.kernel(mycc, teris, t1, t2, precision=precision)
    assert isinstance(e, torch.Tensor) and e.requires_grad
    assert abs(float(e) - e_ref) <= etol * abs(e_ref)
    seed = 0.5
    grads = torch.autograd.grad(seed * e, [leaves["fock"], leaves["mo_energy"], leaves["ovoo"], leaves["ovov"],
                                           leaves["ovvv"], t1, t2])
    fock_bar, mo_bar, ovoo_bar, ovov_bar, ovvv_bar, t1_bar, t2_bar = [g.cpu().numpy() for g in grads]
    o = inp.t1.shape[0]
    assert _relerr(fock_bar[o:, :o], seed * g_ref["fvo"]) < gtol
    assert not fock_bar[:o, :].any() and not fock_bar[o:, o:].any()
    assert _relerr(ovvv_bar, seed * z["cot_ovvv_tril"]) < gtol
    for got, k in ((t1_bar, "t1"), (t2_bar, "t2"), (mo_bar, "mo_energy"), (ovoo_bar, "ovoo"),
                   (ovov_bar, "ovov")):
        assert _relerr(got, seed * g_ref[k]) < gtol, k


def test_energy_without_gradients_takes_the_energy_only_call():
    import torch

    inp, e_ref, _, _ = G.load("o5v19_fvo")
    eris, _ = _eris_and_cc(inp)
    dev = torch.device("cuda")
    ts = [torch.tensor(np.ascontiguousarray(getattr(eris, k)), device=dev)
          for k in ("fock", "mo_energy", "ovoo", "ovov", "ovvv")]
    e = ccsd_t.ccsd_t_energy(*ts, torch.tensor(inp.t1, device=dev), torch.tensor(inp.t2, device=dev))
    assert not e.requires_grad
    assert abs(float(e) - e_ref) <= E_RTOL * abs(e_ref)


class _FakeCCSD:
    """The attributes pyscfad's CCSD.ccsd_t reads (ccsd.py:420-429)."""

    def __init__(self, inp, eris):
        self.t1, self.t2, self.mo_coeff, self.verbose, self.max_memory = inp.t1, inp.t2, "C", 0, 4000
        self._eris, self.ao2mo_calls = eris, []

    def ao2mo(self, mo_coeff):
        self.ao2mo_calls.append(mo_coeff)
        return self._eris


@pytest.mark.parametrize("precision,etol", [("fp64", E_RTOL), ("mixed", 1e-6)])
def test_ccsd_t_method_routes_to_the_gpu_kernel(precision, etol):
    from pyscfad_b200.cc import ccsd as gpu_ccsd

    inp, e_ref, _, _ = G.load("o5v19_fvo")
    eris, _ = _eris_and_cc(inp)

    class CC(_FakeCCSD):
        pass

    gpu_ccsd.install(CC, precision=precision)
    mycc = CC(inp, eris)
    e = mycc.ccsd_t()                      # defaults: self.t1, self.t2, self.ao2mo(self.mo_coeff)
    assert mycc.ao2mo_calls == ["C"]
    assert abs(e - e_ref) <= etol * abs(e_ref)
    e2 = mycc.ccsd_t(inp.t1, inp.t2, eris)  # explicit arguments: no ao2mo
    assert mycc.ao2mo_calls == ["C"] and e2 == e

    class CC2(gpu_ccsd.CCSDTriplesMixin, _FakeCCSD):
        triples_precision = precision

    assert abs(CC2(inp, eris).ccsd_t() - e_ref) <= etol * abs(e_ref)
