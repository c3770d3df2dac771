from . import ccsd_t  # noqa: F401
