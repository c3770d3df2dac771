"""CCSD.ccsd_t routing (pyscfad/cc/ccsd.py:420-429) without a GPU: the
method fills its defaults from the CCSD object and hands the call to
pyscfad_b200.cc.ccsd_t.kernel with the object's verbosity and precision."""
import pytest

from pyscfad_b200.cc import ccsd as gpu_ccsd
from pyscfad_b200.cc import ccsd_t


class _CC:
    t1, t2, mo_coeff, verbose = "T1", "T2", "C", 4

    def ao2mo(self, mo_coeff):
        return ("ERIS", mo_coeff)


def test_defaults_and_routing(monkeypatch):
    calls = []
    monkeypatch.setattr(ccsd_t, "kernel", lambda mycc, eris, t1, t2, verbose, precision: calls.append(
        (eris, t1, t2, verbose, precision)) or -1.5)

    class CC(_CC):
        pass

    gpu_ccsd.install(CC, precision="mixed")
    assert CC().ccsd_t() == -1.5
    assert calls[-1] == (("ERIS", "C"), "T1", "T2", 4, "mixed")
    CC().ccsd_t(t1="a", t2="b", eris="E")
    assert calls[-1] == ("E", "a", "b", 4, "mixed")

    class CC2(gpu_ccsd.CCSDTriplesMixin, _CC):
        pass

    CC2().ccsd_t()
    assert calls[-1][-1] == "fp64"


def test_install_rejects_unknown_precision():
    class CC(_CC):
        pass

    with pytest.raises(ValueError):
        gpu_ccsd.install(CC, precision="fp32")
