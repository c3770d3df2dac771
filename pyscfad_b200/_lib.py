"""ctypes binding of the C ABI in include/pyscfad_b200.h.

The CUDA library is mandatory: there is no CPU fallback.  Loading fails
loudly if pyscfad_b200/libpyscfad_b200.so is missing.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpyscfad_b200.so")

PRECISION = {"fp64": 0, "mixed": 1, "mixed_bf16": 2}
STATUS_OK = 0

_lib = None

_c_int, _c_size, _c_double, _vp = ctypes.c_int, ctypes.c_size_t, ctypes.c_double, ctypes.c_void_p


class Options(ctypes.Structure):
    """triples_options (include/pyscfad_b200.h): per-call settings."""
    _fields_ = [("block_size", _c_int), ("chunk_a0", _c_int), ("chunk_a1", _c_int),
                ("accumulation_segment", _c_int), ("tile_n", _c_int)]


def options(block_size=0, chunk_range=None, accumulation_segment=0, tile_n=0):
    """An Options value; chunk_range = (a0, a1) restricts the call to the chunks
    whose largest virtual block index lies in [a0, a1)."""
    a0, a1 = chunk_range if chunk_range is not None else (0, 0)
    return Options(int(block_size), int(a0), int(a1), int(accumulation_segment), int(tile_n))


class Problem(ctypes.Structure):
    """triples_problem (include/pyscfad_b200.h): one problem of a batch."""
    _fields_ = ([("nocc", _c_int), ("nvir", _c_int), ("ovvv_packed", _c_int), ("block_size", _c_int),
                 ("tile_n", _c_int)] +
                [(k, _vp) for k in ("mo_energy", "t1", "t2", "ovoo", "ovov", "ovvv", "fvo", "e_out",
                                    "mo_energy_bar", "t1_bar", "t2_bar", "ovoo_bar", "ovov_bar", "ovvv_bar",
                                    "fvo_bar")])


class TriplesError(RuntimeError):
    """A C-ABI entry point returned a non-zero triples_status."""

    def __init__(self, status: int, where: str):
        lib = load()
        msg = lib.triples_status_string(status).decode()
        if status == 3:
            msg += f" (cudaError {lib.triples_last_cuda_error()})"
        super().__init__(f"{where}: {msg}")
        self.status = status


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m pyscfad_b200.build` "
            "(the (T) path has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    lib.triples_workspace_size.restype = _c_size
    lib.triples_workspace_size.argtypes = [_c_int] * 5
    lib.triples_energy.restype = _c_int
    lib.triples_energy.argtypes = [_vp, _c_int, _c_int, _c_int, _c_int] + [_vp] * 7 + [_vp, _c_size, _vp]
    lib.triples_energy_vjp.restype = _c_int
    lib.triples_energy_vjp.argtypes = ([_vp, _c_int, _c_int, _c_int, _c_int] + [_vp] * 7 +
                                       [_c_double, _vp, _c_size, _vp] + [_vp] * 7)
    _opt = ctypes.POINTER(Options)
    lib.triples_workspace_size_ex.restype = _c_size
    lib.triples_workspace_size_ex.argtypes = [_c_int] * 5 + [_opt]
    lib.triples_energy_vjp_ex.restype = _c_int
    lib.triples_energy_vjp_ex.argtypes = ([_vp, _c_int, _c_int, _c_int, _c_int] + [_vp] * 7 +
                                          [_c_double, _c_int, _opt, _vp, _c_size, _vp] + [_vp] * 7)
    lib.triples_lno_workspace_size_ex.restype = _c_size
    lib.triples_lno_workspace_size_ex.argtypes = [_c_int] * 5 + [_opt]
    lib.triples_lno_energy_vjp_ex.restype = _c_int
    lib.triples_lno_energy_vjp_ex.argtypes = ([_vp, _c_int, _c_int, _c_int, _c_int] + [_vp] * 8 +
                                              [_c_double, _c_int, _opt, _vp, _c_size, _vp] + [_vp] * 8)
    lib.triples_static_check_device_status.restype = _c_int
    lib.triples_static_check_device_status.argtypes = [_vp]
    lib.triples_static_scratch.restype = _c_int
    lib.triples_static_scratch.argtypes = [ctypes.POINTER(_vp), ctypes.POINTER(_c_size)]
    lib.triples_lno_workspace_size.restype = _c_size
    lib.triples_lno_workspace_size.argtypes = [_c_int] * 5
    lib.triples_lno_energy.restype = _c_int
    lib.triples_lno_energy.argtypes = [_vp, _c_int, _c_int, _c_int, _c_int] + [_vp] * 8 + [_vp, _c_size, _vp]
    lib.triples_lno_energy_vjp.restype = _c_int
    lib.triples_lno_energy_vjp.argtypes = ([_vp, _c_int, _c_int, _c_int, _c_int] + [_vp] * 8 +
                                           [_c_double, _vp, _c_size, _vp] + [_vp] * 8)
    lib.triples_df_workspace_size.restype = _c_size
    lib.triples_df_workspace_size.argtypes = [_c_int] * 5
    lib.triples_energy_df.restype = _c_int
    lib.triples_energy_df.argtypes = [_vp] + [_c_int] * 4 + [_vp] * 8 + [_vp, _c_size, _vp]
    lib.triples_energy_vjp_df.restype = _c_int
    lib.triples_energy_vjp_df.argtypes = ([_vp] + [_c_int] * 4 + [_vp] * 8 + [_c_double, _vp, _c_size, _vp] +
                                          [_vp] * 8)
    _prob = ctypes.POINTER(Problem)
    lib.triples_batch_workspace_size.restype = _c_size
    lib.triples_batch_workspace_size.argtypes = [_c_int, _c_int, _prob]
    lib.triples_batch_create.restype = _c_int
    lib.triples_batch_create.argtypes = [_c_int, _c_int, _prob, _c_double, _vp, _c_size, ctypes.POINTER(_vp)]
    lib.triples_batch_run.restype = _c_int
    lib.triples_batch_run.argtypes = [_vp, _vp]
    lib.triples_batch_check_device_status.restype = _c_int
    lib.triples_batch_check_device_status.argtypes = [_vp, _vp]
    lib.triples_batch_destroy.restype = None
    lib.triples_batch_destroy.argtypes = [_vp]
    lib.triples_status_string.restype = ctypes.c_char_p
    lib.triples_status_string.argtypes = [_c_int]
    lib.triples_last_cuda_error.restype = _c_int
    lib.triples_version.restype = ctypes.c_char_p
    lib.triples_check_device_status.restype = _c_int
    lib.triples_check_device_status.argtypes = [_vp, _vp]
    lib.triples_profile_enable.restype = None
    lib.triples_profile_enable.argtypes = [_c_int]
    lib.triples_profile_read.restype = _c_int
    lib.triples_profile_read.argtypes = [_c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_c_int)]
    lib.triples_profile_name.restype = ctypes.c_char_p
    lib.triples_profile_name.argtypes = [_c_int]
    _lib = lib
    return lib


def check(status: int, where: str):
    if status != STATUS_OK:
        raise TriplesError(status, where)
