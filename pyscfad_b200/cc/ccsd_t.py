"""Drop-in for pyscfad.cc.ccsd_t (pyscfad/cc/ccsd_t.py:28-192).

``kernel(mycc, eris, t1=None, t2=None, verbose=None)`` returns E(T) and is
differentiable w.r.t. the ERI leaves (fock, mo_energy, ovoo, ovov, ovvv) and
the amplitudes (t1, t2), with the reference's cotangent conventions:
fock_bar holds only the vo block (ccsd_t.py:181-182), ovvv_bar has the
layout of eris.ovvv (packed tril folded as in ccsd_t.py:184-191), and leaves
the (T) energy does not read get zero cotangents (ccsd_t.py:71-74).

The reference wraps its kernels in ``jax.custom_vjp``; here the same
forward/backward pair is a ``torch.autograd.Function`` over CUDA tensors
(JAX is not part of this runtime).  Because E(T) is a scalar, the forward
computes E and dE/d(inputs) in one pass when any input requires a
gradient, and the backward scales the stored gradient by the incoming
cotangent -- the reference instead recomputes W/V in its backward.
"""
from __future__ import annotations

import numpy
import torch

from .. import triples

__all__ = ["kernel", "ccsd_t_energy", "_ccsd_t_energy_vjp"]


def _fvo(fock, nocc):
    return fock[nocc:, :nocc]


class _TriplesEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, precision, fock, mo_energy, ovoo, ovov, ovvv, t1, t2):
        nocc = t1.shape[0]
        fvo = _fvo(fock, nocc).contiguous()
        need = any(ctx.needs_input_grad[1:])
        if need:
            e, g = triples.energy_vjp(mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, 1.0,
                                      precision=precision)
            ctx.grads = g
            ctx.fock_shape = fock.shape
        else:
            e = triples.energy(mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, precision=precision)
        return e

    @staticmethod
    def backward(ctx, ybar):
        g = ctx.grads
        nocc = g["t1"].shape[0]
        fock_bar = torch.zeros(ctx.fock_shape, dtype=torch.float64, device=ybar.device)
        fock_bar[nocc:, :nocc] = g["fvo"]
        s = ybar.to(torch.float64)
        return (None, fock_bar * s, g["mo_energy"] * s, g["ovoo"] * s, g["ovov"] * s,
                g["ovvv"] * s, g["t1"] * s, g["t2"] * s)


def ccsd_t_energy(fock, mo_energy, ovoo, ovov, ovvv, t1, t2, precision="fp64"):
    """Functional form: E(T) from tensors, differentiable through autograd."""
    dev = t1.device if isinstance(t1, torch.Tensor) and t1.is_cuda else torch.device("cuda")
    ts = [torch.as_tensor(x).to(dev) for x in (fock, mo_energy, ovoo, ovov, ovvv, t1, t2)]
    return _TriplesEnergy.apply(precision, *ts)


def kernel(mycc, eris, t1=None, t2=None, verbose=None, precision="fp64"):
    """E(T) for CCSD amplitudes (mirrors pyscfad/cc/ccsd_t.py:28).

    Host (numpy) inputs return a Python float, as the reference does;
    torch tensors return a 0-dim tensor that carries gradients."""
    if t1 is None:
        t1 = mycc.t1
    if t2 is None:
        t2 = mycc.t2
    leaves = (eris.fock, eris.mo_energy, eris.ovoo, eris.ovov, eris.ovvv, t1, t2)
    host = not any(isinstance(x, torch.Tensor) for x in leaves)
    _check_memory(mycc, t1, eris.ovvv, precision)
    e = ccsd_t_energy(*leaves, precision=precision)
    return float(e) if host else e


def _check_memory(mycc, t1, ovvv, precision):
    """Error behaviour of the reference's pre-flight budget check
    (ccsd_t.py:135-139): RuntimeError when the device cannot hold the
    workspace."""
    nocc, nvir = t1.shape
    packed = len(ovvv.shape) == 3
    need = triples.workspace_size(nocc, nvir, packed, True, precision)
    if torch.cuda.is_available():
        free, _ = torch.cuda.mem_get_info()
        if need > free:
            raise RuntimeError(f"_ccsd_t_energy_vjp: at least {need / 1e6:.0f} MB of device memory "
                               f"needed, {free / 1e6:.0f} MB free.")


def _ccsd_t_energy_vjp(eris, t1, t2, et_bar, max_memory=None, precision="fp64"):
    """Mirror of pyscfad/cc/ccsd_t.py:82: returns
    (t1_bar, t2_bar, fock_bar, mo_energy_bar, ovoo_bar, ovov_bar, ovvv_bar)
    for the cotangent et_bar of E(T), as numpy arrays."""
    nocc = t1.shape[0]
    fock = torch.as_tensor(eris.fock)
    fvo = fock[nocc:, :nocc].contiguous()
    _, g = triples.energy_vjp(eris.mo_energy, t1, t2, eris.ovoo, eris.ovov, eris.ovvv, fvo,
                              float(et_bar), precision=precision)
    fock_bar = numpy.zeros(tuple(fock.shape))
    fock_bar[nocc:, :nocc] = g["fvo"].cpu().numpy()
    cpu = {k: v.cpu().numpy() for k, v in g.items()}
    return (cpu["t1"], cpu["t2"], fock_bar, cpu["mo_energy"], cpu["ovoo"], cpu["ovov"], cpu["ovvv"])
