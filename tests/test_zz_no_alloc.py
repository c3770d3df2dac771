"""triples_energy_vjp_static: the entry point for callers that may not
allocate device memory (code inside another framework's memory pool, or a
host program that must keep its device footprint fixed).  It runs the same
computation as triples_energy_vjp on a fixed scratch array inside the
library instead of a caller-provided workspace.

This file is collected last on purpose: it checks the new entry point
against the workspace entry point and against the reference's golden
vectors, through the C ABI, on two calls in a row (the scratch keeps the
previous call's contents, so the second call shows that everything that
must start at zero is cleared), and checks that a device-side failure
recorded in the fixed scratch reaches the caller.
"""
import ctypes

import numpy as np
import pytest

from pyscfad_b200 import _lib
from pyscfad_b200.synthetic import make_inputs
from tests import golden_util as G

_c = ctypes.c_int
_d = ctypes.c_double
_vp = ctypes.c_void_p
STATIC_BYTES = 64 << 20   # TRIPLES_STATIC_SCRATCH_BYTES

# tolerances of the other GPU tests: FP64 summation order, and the mixed path
TOL = {"fp64": (1e-12, 1e-10), "mixed": (1e-6, 1e-5)}
KEYS = ("mo_energy", "t1", "t2", "ovoo", "ovov", "ovvv", "fvo")


def _static_fn():
    lib = _lib.load()
    fn = lib.triples_energy_vjp_static
    fn.restype = _c
    fn.argtypes = [_vp, _c, _c, _c, _c] + [_vp] * 7 + [_d, _vp] + [_vp] * 7
    return lib, fn


def _relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-7))


def test_static_rejects_problems_beyond_its_scratch():
    """Too large for the fixed scratch: refused before any GPU work (no device needed)."""
    lib, fn = _static_fn()
    o, v = 12, 80
    assert lib.triples_workspace_size(0, o, v, 1, 1) > STATIC_BYTES
    null = [None] * 7
    rc = fn(None, 0, o, v, 1, *null, 1.0, None, *null)
    assert rc == 2, lib.triples_status_string(rc)   # TRIPLES_ERR_WORKSPACE


@pytest.mark.gpu
@pytest.mark.parametrize("precision,o,v,naux", [("fp64", 5, 19, 80), ("fp64", 5, 40, 120), ("mixed", 6, 32, 100)])
def test_static_matches_workspace_entry_point(precision, o, v, naux):
    import torch

    from pyscfad_b200 import triples

    lib, fn = _static_fn()
    prec = _lib.PRECISION[precision]
    assert 0 < lib.triples_workspace_size(prec, o, v, 1, 1) <= STATIC_BYTES

    inp = make_inputs(o, v, naux, seed=11, fvo_sigma=1e-3)
    dev = torch.device("cuda")
    host = {"mo_energy": inp.mo_energy, "t1": inp.t1, "t2": inp.t2, "ovoo": inp.ovoo, "ovov": inp.ovov,
            "ovvv": inp.ovvv_tril(), "fvo": inp.fvo}
    x = {k: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev) for k, a in host.items()}

    # reference: the workspace entry point
    e_ref, g_ref = triples.energy_vjp(*(x[k] for k in KEYS), ybar=1.0, precision=precision, device=dev)
    torch.cuda.synchronize()
    e_ref = float(e_ref)
    g_ref = {k: t.cpu().numpy() for k, t in g_ref.items()}

    stream = torch.cuda.current_stream(dev).cuda_stream
    etol, gtol = TOL[precision]
    for call in range(2):
        e_out = torch.full((), float("nan"), dtype=torch.float64, device=dev)
        bars = {k: torch.full_like(x[k], float("nan")) for k in KEYS}
        rc = fn(stream, prec, o, v, 1, *(x[k].data_ptr() for k in KEYS), 1.0, e_out.data_ptr(),
                *(bars[k].data_ptr() for k in KEYS))
        assert rc == 0, (call, lib.triples_status_string(rc))
        torch.cuda.synchronize()
        e = float(e_out)
        assert abs(e - e_ref) <= etol * max(1.0, abs(e_ref)), (call, e, e_ref)
        for k in KEYS:
            assert _relerr(bars[k].cpu().numpy(), g_ref[k]) < gtol, (call, k)


def _static_call(fn, x, precision, o, v, stream, dev):
    import torch

    e_out = torch.full((), float("nan"), dtype=torch.float64, device=dev)
    bars = {k: torch.full_like(x[k], float("nan")) for k in KEYS}
    rc = fn(stream, _lib.PRECISION[precision], o, v, 1, *(x[k].data_ptr() for k in KEYS), 1.0, e_out.data_ptr(),
            *(bars[k].data_ptr() for k in KEYS))
    return rc, e_out, bars


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_static_matches_reference_golden(precision):
    """The static entry point against the reference's own outputs (o5 v19, non-canonical fvo)."""
    import torch

    lib, fn = _static_fn()
    inp, e_ref, g_ref, z = G.load("o5v19_fvo")
    dev = torch.device("cuda")
    host = {"mo_energy": inp.mo_energy, "t1": inp.t1, "t2": inp.t2, "ovoo": inp.ovoo, "ovov": inp.ovov,
            "ovvv": inp.ovvv_tril(), "fvo": inp.fvo}
    x = {k: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev) for k, a in host.items()}
    stream = torch.cuda.current_stream(dev).cuda_stream
    etol, gtol = TOL[precision]
    for call in range(2):
        rc, e_out, bars = _static_call(fn, x, precision, 5, 19, stream, dev)
        assert rc == 0, lib.triples_status_string(rc)
        assert lib.triples_static_check_device_status(stream) == 0
        e = float(e_out)
        assert abs(e - e_ref) <= etol * abs(e_ref), (call, e, e_ref)
        for k in KEYS:
            ref = z["cot_ovvv_tril"] if k == "ovvv" else g_ref[k]
            assert _relerr(bars[k].cpu().numpy(), ref) < gtol, (call, k)


@pytest.mark.gpu
def test_static_call_reports_device_side_failures():
    """A device-side failure bit in the fixed scratch's control block (what a
    bounded wait that gave up leaves) is reported by the status calls, and
    the next static call starts clean.  The bit is written from the host:
    nothing on the GPU is made to fail."""
    import torch
    from cuda.bindings import runtime as rt

    lib, fn = _static_fn()
    inp = make_inputs(4, 9, 30, seed=5, fvo_sigma=1e-3)
    dev = torch.device("cuda")
    host = {"mo_energy": inp.mo_energy, "t1": inp.t1, "t2": inp.t2, "ovoo": inp.ovoo, "ovov": inp.ovov,
            "ovvv": inp.ovvv_tril(), "fvo": inp.fvo}
    x = {k: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev) for k, a in host.items()}
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc, _, _ = _static_call(fn, x, "fp64", 4, 9, stream, dev)
    assert rc == 0
    assert lib.triples_static_check_device_status(stream) == 0
    ptr, nbytes = ctypes.c_void_p(), ctypes.c_size_t()
    assert lib.triples_static_scratch(ctypes.byref(ptr), ctypes.byref(nbytes)) == 0
    assert ptr.value and nbytes.value == STATIC_BYTES
    one = np.array([1], dtype=np.int32)
    err, = rt.cudaMemcpy(ptr.value, one.ctypes.data, 4, rt.cudaMemcpyKind.cudaMemcpyHostToDevice)
    assert int(err) == 0
    assert lib.triples_static_check_device_status(stream) == 5     # TRIPLES_ERR_DEVICE_TIMEOUT
    assert lib.triples_check_device_status(stream, ptr) == 5
    rc, _, _ = _static_call(fn, x, "fp64", 4, 9, stream, dev)
    assert rc == 0
    assert lib.triples_static_check_device_status(stream) == 0
