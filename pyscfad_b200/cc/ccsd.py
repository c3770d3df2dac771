"""Routing of ``CCSD.ccsd_t`` to the B200 (T) kernel.

Mirrors the dispatch of pyscfad/cc/ccsd.py:420-429: ``ccsd_t(t1=None,
t2=None, eris=None)`` fills the defaults from the CCSD object (its
amplitudes, and ``self.ao2mo(self.mo_coeff)`` for the ERIs) and calls the
(T) kernel with ``self.verbose``.  The reference chooses between its
compiled path (``pyscfad.cc.ccsd_t.kernel``) and the JAX restatement
(``ccsd_t_slow.kernel``) on ``config.moleintor_opt``; here there is one
path, ``pyscfad_b200.cc.ccsd_t.kernel`` on the GPU, and no CPU fallback.

Two ways to use it:

* ``class MyCCSD(CCSDTriplesMixin, pyscfad.cc.ccsd.CCSD)``: the mixin's
  ``ccsd_t`` comes first in the method order;
* ``install(pyscfad.cc.ccsd.CCSD)``: replaces the method on an existing
  class, the edit a maintainer would otherwise make in ccsd.py.

The precision of the (T) contractions is the class or instance attribute
``triples_precision`` ("fp64", "mixed" or "mixed_bf16"; default "fp64", the
reference's arithmetic).
"""
from __future__ import annotations

from . import ccsd_t as _ccsd_t

__all__ = ["CCSDTriplesMixin", "install", "ccsd_t"]


def ccsd_t(self, t1=None, t2=None, eris=None):
    """E(T) of a CCSD object (pyscfad/cc/ccsd.py:420-429), on the GPU."""
    if t1 is None:
        t1 = self.t1
    if t2 is None:
        t2 = self.t2
    if eris is None:
        eris = self.ao2mo(self.mo_coeff)
    precision = getattr(self, "triples_precision", "fp64")
    return _ccsd_t.kernel(self, eris, t1, t2, getattr(self, "verbose", None), precision=precision)


class CCSDTriplesMixin:
    """Gives a CCSD class the GPU ``ccsd_t`` method."""

    triples_precision = "fp64"
    ccsd_t = ccsd_t


def install(cls, precision: str | None = None):
    """Make ``cls.ccsd_t`` the GPU (T) path; returns ``cls``.  With
    ``precision`` given it also sets ``cls.triples_precision``."""
    cls.ccsd_t = ccsd_t
    if precision is not None:
        if precision not in ("fp64", "mixed", "mixed_bf16"):
            raise ValueError(f"unknown precision {precision!r}")
        cls.triples_precision = precision
    return cls
