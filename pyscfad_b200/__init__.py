"""B200-native CCSD(T) perturbative-triples energy and adjoint.

Drop-in for the (T) hot path of pyscfad: ``pyscfad_b200.cc.ccsd_t.kernel``
mirrors ``pyscfad.cc.ccsd_t.kernel`` (pyscfad/cc/ccsd_t.py:28), backed by
hand-written sm_100a CUDA kernels behind the C ABI in include/pyscfad_b200.h.
"""
__version__ = "0.1.0"

from . import synthetic  # noqa: F401
