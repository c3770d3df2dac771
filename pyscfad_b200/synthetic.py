"""Seeded synthetic (T) inputs with the shapes and distributions of the
benchmark workloads (no molecular data is available offline).

Distributions (one seed per workload):
  mo_energy  occupied ~U(-1.5,-0.3), virtual ~U(0.2,3.0), each sorted
  t1[o,v]    ~N(0, 1e-2)
  t2[o,o,v,v] ~N(0, 2e-2), symmetrised t2[i,j,a,b] = t2[j,i,b,a]
  L[P,p,q]   ~N(0, 0.1), symmetrised in (p,q)  (Cholesky-like factors)
  ovvv[i,a,b,c] = sum_P L[P,i,a] L[P,b,c]   (symmetric in b,c)
  ovoo[i,a,j,k] = sum_P L[P,i,a] L[P,j,k]   (ooov[j,k,i,a] = ovoo[i,a,j,k])
  ovov[i,a,j,b] = sum_P L[P,i,a] L[P,j,b]
  fvo[v,o]   zero (canonical orbitals) or ~N(0, 1e-3)
``scale`` multiplies L, giving a "physically scaled" variant whose |E(T)|
is small enough for an absolute error gate to be meaningful.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# Named workloads: (nocc, nvir, naux)
WORKLOADS = {
    "water_ccpvdz_o5v19": (5, 19, 80),
    "medium_o20v180": (20, 180, 600),
    "large_o40v360": (40, 360, 1200),
    "huge_o50v450": (50, 450, 1500),
}


@dataclass
class TriplesInputs:
    """Reference-layout (T) inputs, FP64, C order (pyscfad/cc/ccsd_t.py:86-105)."""
    mo_energy: np.ndarray   # [n]
    t1: np.ndarray          # [o,v]
    t2: np.ndarray          # [o,o,v,v]
    ovoo: np.ndarray        # [o,v,o,o]
    ovov: np.ndarray        # [o,v,o,v]
    ovvv: np.ndarray        # [o,v,v,v] (unpacked)
    fvo: np.ndarray         # [v,o]

    @property
    def nocc(self) -> int:
        return self.t1.shape[0]

    @property
    def nvir(self) -> int:
        return self.t1.shape[1]

    def ovvv_tril(self) -> np.ndarray:
        """Packed lower-triangle form [o,v,v(v+1)/2] (DF ERIs, dfccsd.py:88)."""
        v = self.nvir
        il, jl = np.tril_indices(v)
        return np.ascontiguousarray(self.ovvv[:, :, il, jl])


def make_inputs(nocc: int, nvir: int, naux: int, seed: int = 0,
                fvo_sigma: float = 0.0, scale: float = 1.0) -> TriplesInputs:
    return _make(nocc, nvir, naux, seed, fvo_sigma, scale)[0]


def make_df_inputs(nocc: int, nvir: int, naux: int, seed: int = 0, fvo_sigma: float = 0.0,
                   scale: float = 1.0):
    """make_inputs plus the DF factors its ERIs come from, in the layouts of
    pyscfad's DF ERIs (dfccsd.py:77-78): Lov[naux, o*v] and the packed
    Lvv[naux, v(v+1)/2] (pair f >= y at f(f+1)/2 + y).  Returns (inputs, Lov, Lvv)."""
    inp, Lov, Lvv = _make(nocc, nvir, naux, seed, fvo_sigma, scale)
    il, jl = np.tril_indices(nvir)
    Lvv_tril = np.ascontiguousarray(Lvv.reshape(naux, nvir, nvir)[:, il, jl])
    return inp, np.ascontiguousarray(Lov), Lvv_tril


def _make(nocc, nvir, naux, seed, fvo_sigma, scale):
    rng = np.random.default_rng(seed)
    o, v = nocc, nvir
    n = o + v
    eo = np.sort(rng.uniform(-1.5, -0.3, o))
    ev = np.sort(rng.uniform(0.2, 3.0, v))
    mo_energy = np.concatenate([eo, ev])
    t1 = rng.normal(0.0, 1e-2, (o, v))
    x = rng.normal(0.0, 2e-2, (o, o, v, v))
    t2 = 0.5 * (x + x.transpose(1, 0, 3, 2))
    L = rng.normal(0.0, 0.1, (naux, n, n)) * scale
    L = 0.5 * (L + L.transpose(0, 2, 1))
    Lov = L[:, :o, o:].reshape(naux, o * v)
    Lvv = L[:, o:, o:].reshape(naux, v * v)
    Loo = L[:, :o, :o].reshape(naux, o * o)
    ovvv = (Lov.T @ Lvv).reshape(o, v, v, v)
    ovoo = (Lov.T @ Loo).reshape(o, v, o, o)
    ovov = (Lov.T @ Lov).reshape(o, v, o, v)
    if fvo_sigma > 0:
        fvo = rng.normal(0.0, fvo_sigma, (v, o))
    else:
        fvo = np.zeros((v, o))
    inp = TriplesInputs(mo_energy, t1, t2, np.ascontiguousarray(ovoo),
                        np.ascontiguousarray(ovov), np.ascontiguousarray(ovvv), fvo)
    return inp, Lov, Lvv


def make_inputs_torch(nocc: int, nvir: int, naux: int, seed: int = 0,
                      fvo_sigma: float = 0.0, scale: float = 1.0,
                      device="cuda", dtype=None):
    """Same distributions, generated on a torch device (for sizes where the
    o*v^3 ERI block does not fit a host round trip).  Values differ from
    make_inputs for the same seed; shapes and distributions are identical.
    Returns a dict of reference-layout tensors."""
    import torch
    dtype = dtype or torch.float64
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    o, v = nocc, nvir
    n = o + v
    eo = torch.sort(torch.empty(o, device=device, dtype=dtype).uniform_(-1.5, -0.3, generator=g))[0]
    ev = torch.sort(torch.empty(v, device=device, dtype=dtype).uniform_(0.2, 3.0, generator=g))[0]
    mo_energy = torch.cat([eo, ev])
    t1 = torch.empty(o, v, device=device, dtype=dtype).normal_(0.0, 1e-2, generator=g)
    x = torch.empty(o, o, v, v, device=device, dtype=dtype).normal_(0.0, 2e-2, generator=g)
    t2 = 0.5 * (x + x.permute(1, 0, 3, 2))
    del x
    L = torch.empty(naux, n, n, device=device, dtype=dtype).normal_(0.0, 0.1, generator=g) * scale
    L = 0.5 * (L + L.transpose(1, 2))
    Lov = L[:, :o, o:].reshape(naux, o * v)
    Lvv = L[:, o:, o:].reshape(naux, v * v)
    Loo = L[:, :o, :o].reshape(naux, o * o)
    ovvv = (Lov.T @ Lvv).reshape(o, v, v, v)
    ovoo = (Lov.T @ Loo).reshape(o, v, o, o)
    ovov = (Lov.T @ Lov).reshape(o, v, o, v)
    del L, Lov, Lvv, Loo
    if fvo_sigma > 0:
        fvo = torch.empty(v, o, device=device, dtype=dtype).normal_(0.0, fvo_sigma, generator=g)
    else:
        fvo = torch.zeros(v, o, device=device, dtype=dtype)
    return dict(mo_energy=mo_energy, t1=t1, t2=t2.contiguous(), ovoo=ovoo.contiguous(),
                ovov=ovov.contiguous(), ovvv=ovvv.contiguous(), fvo=fvo)
