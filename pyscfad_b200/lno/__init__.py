"""Local-natural-orbital (LNO) fragment (T), mirroring pyscfad.lno."""
from . import ccsd_t  # noqa: F401
