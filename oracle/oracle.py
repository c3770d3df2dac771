"""CPU oracle for the (T) energy and VJP -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs may import this module; the product path never does.

Three independent CPU implementations are exposed:

* ``ref_energy`` / ``ref_energy_vjp``: the reference's own C kernels
  (``_ref/libcc_vjp_ref.so``, compiled unchanged from
  pyscfadlib/pyscfadlib/vjp/cc/*.c by ``oracle/Makefile``), driven with the
  host-side layout preparation of pyscfad/cc/ccsd_t.py:82-192 and
  pyscfad/lno/ccsd_t.py:70-113.  The forward is ``lnoccsdt_contract`` with
  mat = I times 2/3, which equals the canonical forward that the reference
  delegates to pyscf (pyscf.cc.ccsd_t.kernel, third-party, pinned
  pyscf>=2.3,<2.12 by the reference and absent here).
* ``oracle_energy_vjp``: our plain-C FP64 restatement (triples_oracle.c).
* ``np_energy``: a NumPy restatement of pyscfad/cc/ccsd_t_slow.py:29-125 for
  tiny sizes.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(HERE, "lib", "libtriples_oracle.so")
_REF_SO = os.path.join(HERE, "_ref", "libcc_vjp_ref.so")
_libs = {}

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.c_void_p)


# where the reference checkout and the BLAS the reference library links live
# on the machine that builds the checker (override with REF / OPENBLAS_DIR)
_REF_DEFAULT = "/root/reference/pyscfadlib/pyscfadlib"


def _openblas_dir():
    """The folder of the OpenBLAS bundled with the opencv wheel of this image
    (it exports dgemm_/dgemv_), found through the installed package."""
    import importlib.util
    spec = importlib.util.find_spec("cv2")
    if spec is None or not spec.origin:
        return ""
    site = os.path.dirname(os.path.dirname(spec.origin))
    for name in sorted(os.listdir(site)):
        if name.startswith("opencv_python") and name.endswith(".libs"):
            return os.path.join(site, name)
    return ""


def build():
    """Compile the oracle (and the reference library when its sources exist)."""
    import subprocess
    env = dict(os.environ)
    if not env.get("REF") and os.path.isdir(_REF_DEFAULT):
        env["REF"] = _REF_DEFAULT
    if not env.get("OPENBLAS_DIR"):
        env["OPENBLAS_DIR"] = _openblas_dir()
    args = ["make", "-s", "-C", HERE]
    for k in ("REF", "OPENBLAS_DIR"):
        if env.get(k):
            args.append(f"{k}={env[k]}")
    subprocess.run(args, check=True, env=env)


def _lib(name):
    if name not in _libs:
        path = _ORACLE_SO if name == "oracle" else _REF_SO
        if not os.path.exists(path):
            build()
        _libs[name] = ctypes.CDLL(path)
    return _libs[name]


def ref_available() -> bool:
    return os.path.exists(_REF_SO)


GRAD_KEYS = ("mo_energy", "t1", "t2", "ovoo", "ovov", "ovvv", "fvo")


def _arrays(inp):
    return [np.ascontiguousarray(getattr(inp, k), dtype=np.float64) for k in GRAD_KEYS]


# --------------------------------------------------------------------------
# our C restatement
# --------------------------------------------------------------------------
def oracle_energy_vjp(inp, ybar=1.0, want_grad=True, a0=0, a1=None, nthreads=None):
    """E(T) and (optionally) gradients w.r.t. each reference-layout array
    treated as an independent tensor (ovvv gradient unpacked [o,v,v,v])."""
    lib = _lib("oracle")
    o, v = inp.nocc, inp.nvir
    a1 = v if a1 is None else a1
    arrs = _arrays(inp)
    grads = {k: np.zeros_like(a) for k, a in zip(GRAD_KEYS, arrs)}
    e = ctypes.c_double(0.0)
    if nthreads:
        os.environ["OMP_NUM_THREADS"] = str(nthreads)
    f = lib.triples_oracle_energy_vjp
    f.restype = ctypes.c_int
    gp = [_ptr(grads[k]) if want_grad else None for k in GRAD_KEYS]
    rc = f(ctypes.c_int(o), ctypes.c_int(v), *[_ptr(a) for a in arrs],
           ctypes.c_double(ybar), ctypes.c_int(int(want_grad)), ctypes.c_int(a0),
           ctypes.c_int(a1), ctypes.byref(e), *gp)
    if rc != 0:
        raise RuntimeError(f"triples_oracle_energy_vjp failed: {rc}")
    return e.value, (grads if want_grad else None)


# --------------------------------------------------------------------------
# the reference's own C kernels, with ccsd_t.py's host-side preparation
# --------------------------------------------------------------------------
def _ref_layouts(inp):
    """pyscfad/cc/ccsd_t.py:86-106 layouts."""
    o, v = inp.nocc, inp.nvir
    n = o + v
    t1T = np.ascontiguousarray(inp.t1.T)
    t2T = np.ascontiguousarray(inp.t2.transpose(2, 3, 1, 0))
    vooo = np.ascontiguousarray(inp.ovoo.transpose(1, 0, 3, 2))
    vvop = np.empty((v, v, o, n))
    vvop[:, :, :, :o] = inp.ovov.transpose(1, 3, 0, 2)
    vvop[:, :, :, o:] = inp.ovvv.transpose(1, 3, 0, 2)
    return t1T, t2T, vooo, np.ascontiguousarray(vvop)


def ref_energy(inp, a0=0, a1=None):
    """lnoccsdt_contract(mat=I) * 2/3 (pyscfad/lno/ccsd_t.py:76-113).  With
    (a0,a1) a slice, returns that slice's partial sum (jobs a in [a0,a1),
    all b, c<=b)."""
    lib = _lib("ref")
    o, v = inp.nocc, inp.nvir
    a1 = v if a1 is None else a1
    t1T, t2T, vooo, vvop = _ref_layouts(inp)
    mat = np.eye(o)
    mo_energy = np.ascontiguousarray(inp.mo_energy)
    fvo = np.ascontiguousarray(inp.fvo)
    et = np.zeros(1)
    lib.lnoccsdt_contract(_ptr(et), _ptr(mat), _ptr(mo_energy), _ptr(t1T), _ptr(t2T),
                          _ptr(vooo), _ptr(fvo), ctypes.c_int(o), ctypes.c_int(v),
                          ctypes.c_int(a0), ctypes.c_int(a1), _ptr(vvop))
    return float(et[0]) * 2.0 / 3.0


def ref_vjp_raw(inp, ybar=1.0, a0=0, a1=None):
    """One-block call of ccsd_t_energy_vjp (ccsd_t_vjp.c:332-497) over jobs
    a in [a0,a1), b in [a0,a], c<=b -- with a0=0, a1=v that is every a>=b>=c
    (the else-branch of _ccsd_t_gen_jobs, ccsd_t.c:41-70).  Returns the
    reference's internal-layout gradients."""
    lib = _lib("ref")
    o, v = inp.nocc, inp.nvir
    n = o + v
    a1 = v if a1 is None else a1
    t1T, t2T, vooo, vvop = _ref_layouts(inp)
    mo_energy = np.ascontiguousarray(inp.mo_energy)
    fvo = np.ascontiguousarray(inp.fvo)
    et_bar = 2.0 * ybar                                        # ccsd_t.py:88
    bars = dict(mo_energy=np.zeros(n), t1T=np.zeros_like(t1T), t2T=np.zeros_like(t2T),
                vooo=np.zeros_like(vooo), fvo=np.zeros_like(fvo))
    # cache_row_a = vvop[a0:a1,:a1]; with a0 == 0 the col cache aliases it
    row = np.ascontiguousarray(vvop[a0:a1, :a1])
    row_bar = np.zeros_like(row)
    if a0 == 0:
        col, col_bar = row, row_bar
    else:
        col = np.ascontiguousarray(vvop[:a0, a0:a1])
        col_bar = np.zeros_like(col)
    lib.ccsd_t_energy_vjp(
        _ptr(mo_energy), _ptr(t1T), _ptr(t2T), _ptr(vooo), _ptr(fvo), ctypes.c_double(et_bar),
        ctypes.c_int(o), ctypes.c_int(v), ctypes.c_int(a0), ctypes.c_int(a1),
        ctypes.c_int(a0), ctypes.c_int(a1),
        _ptr(row), _ptr(col), _ptr(row), _ptr(col),
        _ptr(bars["mo_energy"]), _ptr(bars["t1T"]), _ptr(bars["t2T"]), _ptr(bars["vooo"]),
        _ptr(bars["fvo"]), _ptr(row_bar), _ptr(col_bar), _ptr(row_bar), _ptr(col_bar))
    vvop_bar = np.zeros_like(vvop)
    vvop_bar[a0:a1, :a1] += row_bar
    if a0 != 0:
        vvop_bar[:a0, a0:a1] += col_bar
    return bars, vvop_bar


def ref_energy_vjp(inp, ybar=1.0):
    """E(T) and gradients w.r.t. the independent reference-layout arrays
    (same convention as oracle_energy_vjp; the ovvv gradient is unpacked)."""
    e = ref_energy(inp)
    bars, vvop_bar = ref_vjp_raw(inp, ybar)
    o = inp.nocc
    g = dict(
        mo_energy=bars["mo_energy"],
        t1=np.ascontiguousarray(bars["t1T"].T),
        t2=np.ascontiguousarray(bars["t2T"].transpose(3, 2, 0, 1)),
        ovoo=np.ascontiguousarray(bars["vooo"].transpose(1, 0, 3, 2)),
        ovov=np.ascontiguousarray(vvop_bar[:, :, :, :o].transpose(2, 0, 3, 1)),
        ovvv=np.ascontiguousarray(vvop_bar[:, :, :, o:].transpose(2, 0, 3, 1)),
        fvo=bars["fvo"],
    )
    return e, g


def ref_lno_energy(inp, mat, a0=0, a1=None):
    """lnoccsdt_contract with a projector mat[o,o] on the first occupied index,
    times 2/3 (pyscfad/lno/ccsd_t.py:76-113, lno_ccsd_t.c:96-138)."""
    lib = _lib("ref")
    o, v = inp.nocc, inp.nvir
    a1 = v if a1 is None else a1
    t1T, t2T, vooo, vvop = _ref_layouts(inp)
    mat = np.ascontiguousarray(mat, dtype=np.float64)
    mo_energy = np.ascontiguousarray(inp.mo_energy)
    fvo = np.ascontiguousarray(inp.fvo)
    et = np.zeros(1)
    lib.lnoccsdt_contract(_ptr(et), _ptr(mat), _ptr(mo_energy), _ptr(t1T), _ptr(t2T),
                          _ptr(vooo), _ptr(fvo), ctypes.c_int(o), ctypes.c_int(v),
                          ctypes.c_int(a0), ctypes.c_int(a1), _ptr(vvop))
    return float(et[0]) * 2.0 / 3.0


def ref_lno_energy_vjp(inp, mat, ybar=1.0):
    """E and gradients of the LNO (T) energy, from the reference's
    lnoccsdt_energy_vjp (lno_ccsd_t_vjp.c:400-566) called as one block over all
    jobs the way pyscfad/lno/ccsd_t.py:120-235 does for (a0, a1) = (0, nvir),
    mapped to the independent reference-layout arrays (ovvv gradient unpacked)
    plus mat."""
    lib = _lib("ref")
    o, v = inp.nocc, inp.nvir
    n = o + v
    e = ref_lno_energy(inp, mat)
    t1T, t2T, vooo, vvop = _ref_layouts(inp)
    mat = np.ascontiguousarray(mat, dtype=np.float64)
    mo_energy = np.ascontiguousarray(inp.mo_energy)
    fvo = np.ascontiguousarray(inp.fvo)
    bars = dict(mat=np.zeros_like(mat), mo_energy=np.zeros(n), t1T=np.zeros_like(t1T),
                t2T=np.zeros_like(t2T), vooo=np.zeros_like(vooo), fvo=np.zeros_like(fvo))
    vvop_bar = np.zeros_like(vvop)
    lib.lnoccsdt_energy_vjp(
        _ptr(mat), _ptr(mo_energy), _ptr(t1T), _ptr(t2T), _ptr(vooo), _ptr(fvo),
        ctypes.c_double(ybar * 2.0 / 3.0), ctypes.c_int(o), ctypes.c_int(v),
        ctypes.c_int(0), ctypes.c_int(v), ctypes.c_int(0), ctypes.c_int(v),
        _ptr(vvop), _ptr(vvop), _ptr(vvop), _ptr(vvop),
        _ptr(bars["mat"]), _ptr(bars["mo_energy"]), _ptr(bars["t1T"]), _ptr(bars["t2T"]),
        _ptr(bars["vooo"]), _ptr(bars["fvo"]),
        _ptr(vvop_bar), _ptr(vvop_bar), _ptr(vvop_bar), _ptr(vvop_bar))
    g = dict(
        mat=bars["mat"],
        mo_energy=bars["mo_energy"],
        t1=np.ascontiguousarray(bars["t1T"].T),
        t2=np.ascontiguousarray(bars["t2T"].transpose(3, 2, 0, 1)),
        ovoo=np.ascontiguousarray(bars["vooo"].transpose(1, 0, 3, 2)),
        ovov=np.ascontiguousarray(vvop_bar[:, :, :, :o].transpose(2, 0, 3, 1)),
        ovvv=np.ascontiguousarray(vvop_bar[:, :, :, o:].transpose(2, 0, 3, 1)),
        fvo=bars["fvo"],
    )
    return e, g


def fold_ovvv_tril(ovvv_bar):
    """ccsd_t.py:184-191: symmetrise over the last two indices, halve the
    diagonal, pack the lower triangle -> [o,v,v(v+1)/2]."""
    v = ovvv_bar.shape[-1]
    s = ovvv_bar + ovvv_bar.transpose(0, 1, 3, 2)
    idx = np.arange(v)
    s[:, :, idx, idx] *= 0.5
    il, jl = np.tril_indices(v)
    return np.ascontiguousarray(s[:, :, il, jl])


def reference_cotangents(grads, nocc, nvir):
    """The reference fast path's returned cotangents (ccsd_t.py:179-192):
    t1_bar, t2_bar, fock_bar (vo block only), mo_energy_bar, ovoo_bar,
    ovov_bar, ovvv_bar packed tril."""
    n = nocc + nvir
    fock_bar = np.zeros((n, n))
    fock_bar[nocc:, :nocc] = grads["fvo"]
    return dict(t1=grads["t1"], t2=grads["t2"], fock=fock_bar, mo_energy=grads["mo_energy"],
                ovoo=grads["ovoo"], ovov=grads["ovov"], ovvv=fold_ovvv_tril(grads["ovvv"]))


# --------------------------------------------------------------------------
# NumPy restatement of pyscfad/cc/ccsd_t_slow.py:29-125 (tiny sizes only)
# --------------------------------------------------------------------------
def np_energy(inp):
    o, v = inp.nocc, inp.nvir
    e_occ, e_vir = inp.mo_energy[:o], inp.mo_energy[o:]
    eijk = e_occ[:, None, None] + e_occ[None, :, None] + e_occ[None, None, :]
    vvov = inp.ovvv.transpose(1, 3, 0, 2)       # [a,b,i,f]
    vooo = inp.ovoo.transpose(1, 0, 3, 2)       # [a,i,j,m] = ovoo[i,a,m,j]
    vvoo = inp.ovov.transpose(1, 3, 0, 2)       # [a,b,i,j]
    t1T = inp.t1.T
    t2T = inp.t2.transpose(2, 3, 0, 1)          # [a,b,i,j] = t2[i,j,a,b]
    fvo = inp.fvo

    def get_w(a, b, c):
        w = np.einsum('if,fkj->ijk', vvov[a, b], t2T[c, :])
        w -= np.einsum('ijm,mk->ijk', vooo[a, :], t2T[b, c])
        return w

    def get_v(a, b, c):
        return (np.einsum('ij,k->ijk', vvoo[a, b], t1T[c])
                + np.einsum('ij,k->ijk', t2T[a, b], fvo[c]))

    def r3(w):
        return (4 * w + w.transpose(1, 2, 0) + w.transpose(2, 0, 1)
                - 2 * w.transpose(2, 1, 0) - 2 * w.transpose(0, 2, 1) - 2 * w.transpose(1, 0, 2))

    et = 0.0
    for a in range(v):
        for b in range(a + 1):
            for c in range(b + 1):
                fac = 6 if a == c else (2 if (a == b or b == c) else 1)
                d3 = (eijk - e_vir[a] - e_vir[b] - e_vir[c]) * fac
                WW = (get_w(a, b, c) + get_w(a, c, b).transpose(0, 2, 1)
                      + get_w(b, a, c).transpose(1, 0, 2) + get_w(b, c, a).transpose(2, 0, 1)
                      + get_w(c, a, b).transpose(1, 2, 0) + get_w(c, b, a).transpose(2, 1, 0))
                VV = (get_v(a, b, c) + get_v(a, c, b).transpose(0, 2, 1)
                      + get_v(b, a, c).transpose(1, 0, 2) + get_v(b, c, a).transpose(2, 0, 1)
                      + get_v(c, a, b).transpose(1, 2, 0) + get_v(c, b, a).transpose(2, 1, 0))
                ZZ = r3(WW + 0.5 * VV) / d3
                et += np.einsum('ijk,ijk', WW, ZZ)
    return 2.0 * et


# --------------------------------------------------------------------------
# NumPy restatement of the LNO (T) energy and its adjoint (tiny sizes only):
# the energy of lnoccsdt_contract (pyscfadlib/pyscfadlib/vjp/cc/lno_ccsd_t.c:6-29,
# job weights 73-94) times 2/3 (pyscfad/lno/ccsd_t.py:111), and the chain rule
# of lnoccsdt_energy_vjp (lno_ccsd_t_vjp.c:9-122 and 145-297), written over the
# full index range [p,q,r,x,y,z] instead of a >= b >= c jobs.
# --------------------------------------------------------------------------
_PERMS6 = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))
# r3 of pyscfad/cc/ccsd_t_slow.py:84-87 as (axis order, coefficient)
_R3 = (((0, 1, 2), 4.0), ((1, 2, 0), 1.0), ((2, 0, 1), 1.0),
       ((2, 1, 0), -2.0), ((0, 2, 1), -2.0), ((1, 0, 2), -2.0))


def _sym6(a):
    """sum over the six simultaneous permutations of (p,q,r) with (x,y,z)."""
    return sum(a.transpose(*s, *(3 + np.array(s))) for s in _PERMS6)


def _r3_virt(a, adjoint=False):
    out = np.zeros_like(a)
    for s, c in _R3:
        axes = np.argsort(s) if adjoint else np.array(s)
        out += c * a.transpose(0, 1, 2, *(3 + axes))
    return out


def np_lno_energy_vjp(inp, mat, ybar=1.0, want_grad=True):
    """(E, grads) of the LNO (T) energy with projector mat[o,o] on the first
    occupied index; grads in the layouts of ``ref_lno_energy_vjp`` (ovvv
    unpacked) plus "mat".  mat = identity gives the canonical E(T)."""
    o, v = inp.nocc, inp.nvir
    w = (np.einsum('pxfy,rqzf->pqrxyz', inp.ovvv, inp.t2)
         - np.einsum('pxmq,rmzy->pqrxyz', inp.ovoo, inp.t2))
    vv = (np.einsum('pxqy,rz->pqrxyz', inp.ovov, inp.t1)
          + np.einsum('qpyx,zr->pqrxyz', inp.t2, inp.fvo))
    WW, VV = _sym6(w), _sym6(vv)
    Z = _r3_virt(WW + 0.5 * VV)
    eo, ev = inp.mo_energy[:o], inp.mo_energy[o:]
    D = (eo[:, None, None, None, None, None] + eo[None, :, None, None, None, None]
         + eo[None, None, :, None, None, None] - ev[None, None, None, :, None, None]
         - ev[None, None, None, None, :, None] - ev[None, None, None, None, None, :])
    Q = Z / D
    Wt = np.einsum('li,ljkxyz->ijkxyz', mat, WW)
    e = float(np.einsum('ijkxyz,ijkxyz->', Wt, Q)) / 3.0
    if not want_grad:
        return e, None
    Qbar = ybar / 3.0 * Wt
    Wtbar = ybar / 3.0 * Q
    g = {"mat": np.einsum('ljkxyz,ijkxyz->li', WW, Wtbar)}
    Zbar = Qbar / D
    Dbar = -Qbar * Q / D
    Xbar = _r3_virt(Zbar, adjoint=True)
    wbar = _sym6(np.einsum('li,ijkxyz->ljkxyz', mat, Wtbar) + Xbar)
    vbar = _sym6(0.5 * Xbar)
    mob = np.zeros(o + v)
    for ax in range(6):
        part = Dbar.sum(axis=tuple(a for a in range(6) if a != ax))
        if ax < 3:
            mob[:o] += part
        else:
            mob[o:] -= part
    g["mo_energy"] = mob
    g["t1"] = np.einsum('pqrxyz,pxqy->rz', vbar, inp.ovov)
    g["fvo"] = np.einsum('pqrxyz,qpyx->zr', vbar, inp.t2)
    g["ovov"] = np.einsum('pqrxyz,rz->pxqy', vbar, inp.t1)
    g["t2"] = (np.einsum('pqrxyz,zr->qpyx', vbar, inp.fvo)
               + np.einsum('pqrxyz,pxfy->rqzf', wbar, inp.ovvv)
               - np.einsum('pqrxyz,pxmq->rmzy', wbar, inp.ovoo))
    g["ovvv"] = np.einsum('pqrxyz,rqzf->pxfy', wbar, inp.t2)
    g["ovoo"] = -np.einsum('pqrxyz,rmzy->pxmq', wbar, inp.t2)
    return e, g


# --------------------------------------------------------------------------
# DF factors (pyscfad/cc/dfccsd.py:77-88): ovvv_tril = Lov^T Lvv_tril, so the
# packed ovvv cotangent of pyscfad/cc/ccsd_t.py:184-191 maps to the factors
# by the chain rule.
# --------------------------------------------------------------------------
def df_factor_grads(ovvv_tril_bar, Lov, Lvv_tril):
    """(Lov_bar[naux, o*v], Lvv_bar[naux, v(v+1)/2]) from the packed ovvv
    cotangent [o, v, v(v+1)/2]."""
    G = ovvv_tril_bar.reshape(Lov.shape[1], Lvv_tril.shape[1])
    return Lvv_tril @ G.T, Lov @ G
