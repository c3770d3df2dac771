"""Drop-in for pyscfad.lno.ccsd_t (pyscfad/lno/ccsd_t.py:35-237): the (T)
energy of an LNO fragment, whose projected amplitudes carry the occupied
projector mat = ulo^T ulo on their first occupied index.

``kernel(mycc, eris, ulo, t1=None, t2=None)`` and
``_ccsd_t_energy(mat, t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv, max_memory)``
take the reference's arguments and layouts (t1T = t1.T,
t2T = t2.transpose(2,3,1,0), ovvv packed as eris.ovvv); the backward returns
the reference's cotangents (pyscfad/lno/ccsd_t.py:235), with ovvv_bar folded
to the packed layout.  The reference wraps lnoccsdt_contract /
lnoccsdt_energy_vjp in ``jax.custom_vjp``; here the pair is a
``torch.autograd.Function`` over the FP64 CUDA path of
triples_lno_energy(_vjp).
"""
from __future__ import annotations

import numpy
import torch

from .. import triples

__all__ = ["kernel", "_ccsd_t_energy", "_ccsd_t_energy_bwd"]


def _canonical(t1T, t2T):
    """t1[o,v], t2[o,o,v,v] from the reference's t1T[v,o], t2T[v,v,o,o]."""
    return t1T.transpose(0, 1), t2T.permute(3, 2, 0, 1)


class _LnoTriplesEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, precision, mat, t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv):
        t1, t2 = _canonical(t1T, t2T)
        if any(ctx.needs_input_grad[1:]):
            e, g = triples.lno_energy_vjp(mat, mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, 1.0, precision=precision)
            ctx.grads = g
        else:
            e = triples.lno_energy(mat, mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, precision=precision)
        return e

    @staticmethod
    def backward(ctx, ybar):
        g = ctx.grads
        s = ybar.to(torch.float64)
        return (None, g["mat"] * s, g["t1"].transpose(0, 1) * s, g["t2"].permute(2, 3, 1, 0) * s,
                g["mo_energy"] * s, g["fvo"] * s, g["ovoo"] * s, g["ovov"] * s, g["ovvv"] * s)


def _device_of(*xs):
    for x in xs:
        if isinstance(x, torch.Tensor) and x.is_cuda:
            return x.device
    return torch.device("cuda")


def _check_memory(nocc, nvir, packed, want_grad, precision="fp64"):
    """Error behaviour of the reference's memory checks
    (pyscfad/lno/ccsd_t.py:101-103 and 185-192): RuntimeError when the device
    cannot hold the workspace."""
    need = triples.lno_workspace_size(nocc, nvir, packed, want_grad, precision)
    if torch.cuda.is_available():
        free, _ = torch.cuda.mem_get_info()
        if need > free:
            raise RuntimeError(f"{need / 1e6:.0f} MB more memory is needed "
                               f"({free / 1e6:.0f} MB of device memory free).")


def _ccsd_t_energy(mat, t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv, max_memory=None, *, precision="fp64"):
    """Fragment (T) energy (pyscfad/lno/ccsd_t.py:71-112), differentiable
    through autograd in every argument but max_memory (kept for the
    signature; the device workspace is sized exactly).  ``precision`` (not in
    the reference) selects "fp64", "mixed" or "mixed_bf16" contractions."""
    dev = _device_of(mat, t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv)
    ts = [torch.as_tensor(x).to(dev) for x in (mat, t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv)]
    nvir, nocc = ts[1].shape
    _check_memory(nocc, nvir, ts[7].dim() == 3, any(t.requires_grad for t in ts), precision)
    return _LnoTriplesEnergy.apply(precision, *ts)


def _ccsd_t_energy_bwd(max_memory, res, et_bar):
    """Mirror of pyscfad/lno/ccsd_t.py:121-235: res = (mat, t1T, t2T,
    mo_energy, fvo, ovoo, ovov, ovvv); returns (mat_bar, t1T_bar, t2T_bar,
    mo_energy_bar, fvo_bar, ovoo_bar, ovov_bar, ovvv_bar) as numpy arrays."""
    mat, t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv = res
    dev = _device_of(*res)
    t1T, t2T = torch.as_tensor(t1T).to(dev), torch.as_tensor(t2T).to(dev)
    t1, t2 = _canonical(t1T, t2T)
    _, g = triples.lno_energy_vjp(mat, mo_energy, t1, t2, ovoo, ovov, ovvv, fvo, float(et_bar), device=dev)
    c = {k: v.cpu().numpy() for k, v in g.items()}
    return (c["mat"], c["t1"].T.copy(), c["t2"].transpose(2, 3, 1, 0).copy(), c["mo_energy"], c["fvo"],
            c["ovoo"], c["ovov"], c["ovvv"])


def kernel(mycc, eris, ulo, t1=None, t2=None, verbose=None, precision="fp64"):
    """Fragment (T) energy for the projector ulo (pyscfad/lno/ccsd_t.py:35-69).
    Host (numpy) inputs return a Python float, as the reference does; torch
    tensors return a 0-dim tensor that carries gradients."""
    if t1 is None:
        t1 = mycc.t1
    if t2 is None:
        t2 = mycc.t2
    leaves = (ulo, eris.fock, eris.mo_energy, eris.ovoo, eris.ovov, eris.ovvv, t1, t2)
    host = not any(isinstance(x, torch.Tensor) for x in leaves)
    dev = _device_of(*leaves)
    ulo_t = torch.as_tensor(ulo).to(dev)
    mat = ulo_t.transpose(0, 1) @ ulo_t
    t1_t = torch.as_tensor(t1).to(dev)
    t2_t = torch.as_tensor(t2).to(dev)
    if mat.shape[0] != t1_t.shape[0]:
        raise AssertionError("ulo does not span the occupied space of t1")
    nocc = t1_t.shape[0]
    fock = torch.as_tensor(eris.fock).to(dev)
    fvo = fock[nocc:, :nocc].contiguous()
    et = _ccsd_t_energy(mat, t1_t.transpose(0, 1), t2_t.permute(2, 3, 1, 0), eris.mo_energy, fvo,
                        eris.ovoo, eris.ovov, eris.ovvv, getattr(mycc, "max_memory", None), precision=precision)
    return float(et) if host else et
