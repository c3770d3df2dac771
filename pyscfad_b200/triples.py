"""Device-level calls of the (T) energy and VJP on torch CUDA tensors.

Inputs use the reference's canonical layouts (FP64, C order):
mo_energy[n], t1[o,v], t2[o,o,v,v], ovoo[o,v,o,o], ovov[o,v,o,v],
ovvv[o,v,v(v+1)/2] (packed, DF ERIs) or ovvv[o,v,v,v], fvo[v,o].
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

KEYS = ("mo_energy", "t1", "t2", "ovoo", "ovov", "ovvv", "fvo")

# One cached workspace per (device, stream): calls on different streams never
# share scratch, so they may run concurrently.
_workspaces: dict = {}


def _workspace(nbytes: int, device: torch.device, stream) -> torch.Tensor:
    key = (device.type, device.index, int(stream.cuda_stream))
    buf = _workspaces.get(key)
    if buf is None or buf.numel() < nbytes:
        _workspaces.pop(key, None)
        buf = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=device)
        _workspaces[key] = buf
    return buf


def release_workspace():
    _workspaces.clear()


def _as_dev(x, device) -> torch.Tensor:
    t = torch.as_tensor(x)
    if t.dtype != torch.float64:
        raise TypeError(f"(T) inputs must be float64, got {t.dtype}")
    return t.to(device=device).contiguous()


def _shapes(t1, t2, ovoo, ovov, ovvv, fvo, mo_energy):
    if t1.dim() != 2:
        raise ValueError("t1 must be [nocc, nvir]")
    o, v = t1.shape
    packed = ovvv.dim() == 3
    exp = {
        "mo_energy": (o + v,), "t1": (o, v), "t2": (o, o, v, v), "ovoo": (o, v, o, o),
        "ovov": (o, v, o, v), "fvo": (v, o),
        "ovvv": (o, v, v * (v + 1) // 2) if packed else (o, v, v, v),
    }
    got = dict(mo_energy=mo_energy, t1=t1, t2=t2, ovoo=ovoo, ovov=ovov, ovvv=ovvv, fvo=fvo)
    for k, shp in exp.items():
        if tuple(got[k].shape) != shp:
            raise ValueError(f"{k} has shape {tuple(got[k].shape)}, expected {shp}")
    return o, v, packed


def block_sizes(nvir: int, tv: int = 16):
    """Virtual block sizes of the chunk decomposition: nvir // tv blocks of tv,
    then the remainder split into descending powers of two."""
    sizes = [tv] * (nvir // tv)
    rem, bit = nvir - tv * (nvir // tv), tv >> 1
    while bit:
        if rem & bit:
            sizes.append(bit)
        bit >>= 1
    return sizes


def chunk_fraction(nvir: int, a0: int, a1: int, tv: int = 16) -> float:
    """Fraction of all raw amplitudes o^3 v^3 that the chunks with largest block
    in [a0, a1) hold (each chunk holds o^3 * (distinct orderings) * nA nB nC)."""
    n = block_sizes(nvir, tv)
    tot = 0
    for A in range(a0, min(a1, len(n))):
        for B in range(A + 1):
            for C in range(B + 1):
                nperm = len({(A, B, C), (A, C, B), (B, A, C), (B, C, A), (C, A, B), (C, B, A)})
                tot += nperm * n[A] * n[B] * n[C]
    return tot / float(nvir) ** 3


def workspace_size(nocc, nvir, packed=True, want_grad=True, precision="fp64", block_size=0,
                   chunk_range=None, accumulation_segment=0) -> int:
    opt = _lib.options(block_size, chunk_range, accumulation_segment)
    return int(_lib.load().triples_workspace_size_ex(_lib.PRECISION[precision], nocc, nvir, int(packed),
                                                     int(want_grad), ctypes.byref(opt)))


def _device_of(device, t1):
    return torch.device(device or (t1.device if isinstance(t1, torch.Tensor) and t1.is_cuda else "cuda"))


def _run(mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, ybar, want_grad, precision, device, stream, check,
         block_size, chunk_range, accumulation_segment, tile_n=0):
    lib = _lib.load()
    device = _device_of(device, t1)
    args = [_as_dev(a, device) for a in (mo_energy, t1, t2, ovoo, ovov, ovvv, fvo)]
    o, v, packed = _shapes(*args[1:], args[0])
    prec = _lib.PRECISION[precision]
    opt = _lib.options(block_size, chunk_range, accumulation_segment, tile_n)
    nbytes = lib.triples_workspace_size_ex(prec, o, v, int(packed), int(want_grad), ctypes.byref(opt))
    if nbytes == 0:
        raise _lib.TriplesError(1, "triples_workspace_size_ex")
    st = stream if stream is not None else torch.cuda.current_stream(device)
    ws = _workspace(nbytes, device, st)
    e = torch.zeros((), dtype=torch.float64, device=device)
    grads = {k: torch.empty_like(a) for k, a in zip(KEYS, args)} if want_grad else {}
    gptr = [grads[k].data_ptr() for k in KEYS] if want_grad else [None] * len(KEYS)
    rc = lib.triples_energy_vjp_ex(st.cuda_stream, prec, o, v, int(packed), *[a.data_ptr() for a in args],
                                   float(ybar), int(want_grad), ctypes.byref(opt), ws.data_ptr(), ws.numel(),
                                   e.data_ptr(), *gptr)
    _lib.check(rc, "triples_energy_vjp_ex")
    if check:
        _lib.check(lib.triples_check_device_status(st.cuda_stream, ws.data_ptr()), "triples_energy_vjp_ex (device)")
    return e, grads


def energy(mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, precision="fp64", device=None,
           stream=None, check=True, block_size=0, chunk_range=None, accumulation_segment=0) -> torch.Tensor:
    """E(T) as a 0-dim FP64 tensor on the device.  With check=True the
    stream is synchronised and device-side failures raise TriplesError.
    block_size, chunk_range and accumulation_segment are the per-call
    settings of triples_options (0 / None: defaults)."""
    e, _ = _run(mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, 1.0, False, precision, device, stream, check,
                block_size, chunk_range, accumulation_segment)
    return e


def energy_vjp(mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, ybar=1.0, precision="fp64",
               device=None, stream=None, check=True, block_size=0, chunk_range=None, accumulation_segment=0,
               tile_n=0):
    """E(T) and dE/d(inputs) * ybar.  Gradients have the input layouts; for a
    packed ovvv the gradient is the reference's packed-tril fold
    (pyscfad/cc/ccsd_t.py:184-191).  Returns (e, dict)."""
    return _run(mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, ybar, True, precision, device, stream, check,
                block_size, chunk_range, accumulation_segment, tile_n)


def _check_mat(mat, o):
    if tuple(mat.shape) != (o, o):
        raise ValueError(f"mat has shape {tuple(mat.shape)}, expected {(o, o)}")


def lno_workspace_size(nocc, nvir, packed=True, want_grad=True, precision="fp64", block_size=0) -> int:
    opt = _lib.options(block_size)
    return int(_lib.load().triples_lno_workspace_size_ex(_lib.PRECISION[precision], nocc, nvir, int(packed),
                                                         int(want_grad), ctypes.byref(opt)))


def _run_lno(mat, mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, ybar, want_grad, precision, device, stream, check,
             block_size):
    lib = _lib.load()
    device = _device_of(device, t1)
    args = [_as_dev(a, device) for a in (mat, mo_energy, t1, t2, ovoo, ovov, ovvv, fvo)]
    o, v, packed = _shapes(*args[2:], args[1])
    _check_mat(args[0], o)
    prec = _lib.PRECISION[precision]
    opt = _lib.options(block_size)
    nbytes = lib.triples_lno_workspace_size_ex(prec, o, v, int(packed), int(want_grad), ctypes.byref(opt))
    if nbytes == 0:
        raise _lib.TriplesError(4 if o > 64 else 1, "triples_lno_workspace_size_ex")
    st = stream if stream is not None else torch.cuda.current_stream(device)
    ws = _workspace(nbytes, device, st)
    e = torch.zeros((), dtype=torch.float64, device=device)
    keys = ("mat",) + KEYS
    grads = {k: torch.empty_like(a) for k, a in zip(keys, args)} if want_grad else {}
    gptr = [grads[k].data_ptr() for k in keys] if want_grad else [None] * len(keys)
    rc = lib.triples_lno_energy_vjp_ex(st.cuda_stream, prec, o, v, int(packed), *[a.data_ptr() for a in args],
                                       float(ybar), int(want_grad), ctypes.byref(opt), ws.data_ptr(), ws.numel(),
                                       e.data_ptr(), *gptr)
    _lib.check(rc, "triples_lno_energy_vjp_ex")
    if check:
        _lib.check(lib.triples_check_device_status(st.cuda_stream, ws.data_ptr()),
                   "triples_lno_energy_vjp_ex (device)")
    return e, grads


def lno_energy(mat, mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, precision="fp64", device=None,
               stream=None, check=True, block_size=0) -> torch.Tensor:
    """LNO (T) energy with the occupied projector mat[o,o] (= ulo^T ulo,
    pyscfad/lno/ccsd_t.py:42); mat = identity gives E(T).  nocc <= 64."""
    e, _ = _run_lno(mat, mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, 1.0, False, precision, device, stream, check,
                    block_size)
    return e


def lno_energy_vjp(mat, mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, ybar=1.0, precision="fp64",
                   device=None, stream=None, check=True, block_size=0):
    """LNO (T) energy and its VJP; the dict holds "mat" next to the seven
    keys of energy_vjp, each in its input's layout.  Returns (e, dict)."""
    return _run_lno(mat, mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, ybar, True, precision, device, stream, check,
                    block_size)


DF_KEYS = ("mo_energy", "t1", "t2", "ovoo", "ovov", "Lov", "Lvv", "fvo")


def _df_args(mo_energy, t1, t2, ovoo, ovov, Lov, Lvv, fvo, device):
    args = [_as_dev(a, device) for a in (mo_energy, t1, t2, ovoo, ovov, Lov, Lvv, fvo)]
    o, v = args[1].shape
    naux = args[5].shape[0]
    if args[5].numel() != naux * o * v:
        raise ValueError(f"Lov has shape {tuple(args[5].shape)}, expected ({naux}, {o * v})")
    if tuple(args[6].shape) != (naux, v * (v + 1) // 2):
        raise ValueError(f"Lvv has shape {tuple(args[6].shape)}, expected ({naux}, {v * (v + 1) // 2})")
    return args, o, v, naux


def energy_df(mo_energy, t1, t2, ovoo, ovov, Lov, Lvv, fvo, precision="fp64", device=None, stream=None,
              check=True) -> torch.Tensor:
    """E(T) with ovvv built on the device from the DF factors as pyscfad's DF
    ERIs build it (dfccsd.py:77-88): Lov[naux, o*v], Lvv[naux, v(v+1)/2] packed."""
    lib = _lib.load()
    device = torch.device(device or (t1.device if isinstance(t1, torch.Tensor) and t1.is_cuda else "cuda"))
    args, o, v, naux = _df_args(mo_energy, t1, t2, ovoo, ovov, Lov, Lvv, fvo, device)
    prec = _lib.PRECISION[precision]
    nbytes = lib.triples_df_workspace_size(prec, o, v, naux, 0)
    if nbytes == 0:
        raise _lib.TriplesError(1, "triples_df_workspace_size")
    st = stream if stream is not None else torch.cuda.current_stream(device)
    ws = _workspace(nbytes, device, st)
    e = torch.zeros((), dtype=torch.float64, device=device)
    rc = lib.triples_energy_df(st.cuda_stream, prec, o, v, naux, *[a.data_ptr() for a in args], ws.data_ptr(),
                               ws.numel(), e.data_ptr())
    _lib.check(rc, "triples_energy_df")
    if check:
        _lib.check(lib.triples_check_device_status(st.cuda_stream, ws.data_ptr()), "triples_energy_df (device)")
    return e


def energy_vjp_df(mo_energy, t1, t2, ovoo, ovov, Lov, Lvv, fvo, ybar=1.0, precision="fp64", device=None,
                  stream=None, check=True):
    """E(T) and its VJP with respect to the DF factors instead of ovvv: the
    dict holds "Lov" [naux, o*v] and "Lvv" [naux, v(v+1)/2] (one entry per
    packed pair) next to the other inputs' cotangents."""
    lib = _lib.load()
    device = torch.device(device or (t1.device if isinstance(t1, torch.Tensor) and t1.is_cuda else "cuda"))
    args, o, v, naux = _df_args(mo_energy, t1, t2, ovoo, ovov, Lov, Lvv, fvo, device)
    prec = _lib.PRECISION[precision]
    nbytes = lib.triples_df_workspace_size(prec, o, v, naux, 1)
    if nbytes == 0:
        raise _lib.TriplesError(1, "triples_df_workspace_size")
    st = stream if stream is not None else torch.cuda.current_stream(device)
    ws = _workspace(nbytes, device, st)
    e = torch.zeros((), dtype=torch.float64, device=device)
    grads = {k: torch.empty_like(a) for k, a in zip(DF_KEYS, args)}
    rc = lib.triples_energy_vjp_df(st.cuda_stream, prec, o, v, naux, *[a.data_ptr() for a in args], float(ybar),
                                   ws.data_ptr(), ws.numel(), e.data_ptr(), *[grads[k].data_ptr() for k in DF_KEYS])
    _lib.check(rc, "triples_energy_vjp_df")
    if check:
        _lib.check(lib.triples_check_device_status(st.cuda_stream, ws.data_ptr()), "triples_energy_vjp_df (device)")
    return e, grads


def device_status(device=None, stream=None) -> int:
    """Synchronise and return the device-side status of the last call made
    on this stream (its cached workspace)."""
    device = torch.device(device or "cuda")
    st = stream if stream is not None else torch.cuda.current_stream(device)
    buf = _workspaces.get((device.type, device.index, int(st.cuda_stream)))
    if buf is None:
        return 0
    return int(_lib.load().triples_check_device_status(st.cuda_stream, buf.data_ptr()))
