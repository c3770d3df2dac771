"""CPU baseline: the reference's own (T) C kernels timed on the host cores.

TEST / MEASUREMENT INFRASTRUCTURE ONLY (used by bench.py's CPU-baseline and
reference legs, never by the product).

Times, at the workload's real (nocc, nvir), bounded job slices of
  * the forward: lnoccsdt_contract (pyscfadlib/.../lno_ccsd_t.c:96-138) with
    mat = I over a in [0,1) -- every job of that slice costs what one
    canonical a>=b>=c job of pyscf's forward costs (same six get_wv calls and
    energy contraction);
  * the backward: ccsd_t_energy_vjp (pyscfadlib/.../ccsd_t_vjp.c:332-497) over
    the a>=b>=c jobs with a < A (one block, as ccsd_t.py:145-156 calls it);
and extrapolates both linearly in the number of canonical jobs
v(v+1)(v+2)/6 (per-job cost does not depend on the job's indices).
Input values do not affect the timing; arrays are filled with constants.

    OMP_NUM_THREADS=<cores> OPENBLAS_NUM_THREADS=1 python oracle/cpu_baseline.py 40 360 --target 8
prints one JSON object; --lno times the LNO (projected) kernels the same way.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import oracle as O  # noqa: E402


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def time_forward_slice(lib, o, v):
    n = o + v
    vvop = np.full((v, v, o, n), 1e-3)
    t1T = np.full((v, o), 1e-2)
    t2T = np.full((v, v, o, o), 1e-2)
    vooo = np.full((v, o, o, o), 1e-3)
    fvo = np.zeros((v, o))
    mat = np.eye(o)
    mo = np.concatenate([np.linspace(-1.5, -0.3, o), np.linspace(0.2, 3.0, v)])
    et = np.zeros(1)
    t0 = time.perf_counter()
    lib.lnoccsdt_contract(_p(et), _p(mat), _p(mo), _p(t1T), _p(t2T), _p(vooo), _p(fvo),
                          ctypes.c_int(o), ctypes.c_int(v), ctypes.c_int(0), ctypes.c_int(1), _p(vvop))
    dt = time.perf_counter() - t0
    return dt, v * (v + 1) // 2


def time_vjp_slice(lib, o, v, A):
    n = o + v
    row = np.full((A, A, o, n), 1e-3)
    row_bar = np.zeros_like(row)
    t1T = np.full((v, o), 1e-2)
    t2T = np.full((v, v, o, o), 1e-2)
    vooo = np.full((v, o, o, o), 1e-3)
    fvo = np.zeros((v, o))
    mo = np.concatenate([np.linspace(-1.5, -0.3, o), np.linspace(0.2, 3.0, v)])
    bars = [np.zeros(n), np.zeros_like(t1T), np.zeros_like(t2T), np.zeros_like(vooo), np.zeros_like(fvo)]
    t0 = time.perf_counter()
    lib.ccsd_t_energy_vjp(_p(mo), _p(t1T), _p(t2T), _p(vooo), _p(fvo), ctypes.c_double(2.0),
                          ctypes.c_int(o), ctypes.c_int(v), ctypes.c_int(0), ctypes.c_int(A),
                          ctypes.c_int(0), ctypes.c_int(A), _p(row), _p(row), _p(row), _p(row),
                          *[_p(b) for b in bars], _p(row_bar), _p(row_bar), _p(row_bar), _p(row_bar))
    dt = time.perf_counter() - t0
    return dt, A * (A + 1) * (A + 2) // 6


def measure(o, v, target_s=8.0):
    lib = O._lib("ref")
    # backward: grow the slice until it takes about target_s
    A = min(v, 6)
    dt_b, jobs_b = time_vjp_slice(lib, o, v, A)
    while dt_b < 0.25 * target_s and A < v:
        per = dt_b / jobs_b
        want = target_s / per
        A_new = A
        while A_new < v and A_new * (A_new + 1) * (A_new + 2) // 6 < want:
            A_new += 1
        if A_new == A:
            break
        A = A_new
        dt_b, jobs_b = time_vjp_slice(lib, o, v, A)
    dt_f, jobs_f = time_forward_slice(lib, o, v)
    n_canon = v * (v + 1) * (v + 2) // 6
    t_fwd = dt_f / jobs_f * n_canon
    t_bwd = dt_b / jobs_b * n_canon
    flops = 8.0 * o ** 3 * v ** 4
    return {
        "nocc": o, "nvir": v, "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())),
        "fwd_slice_jobs": jobs_f, "fwd_slice_s": dt_f, "bwd_slice_jobs": jobs_b, "bwd_slice_s": dt_b,
        "bwd_slice_a_max": A, "canonical_jobs": n_canon,
        "t_full_fwd_s": t_fwd, "t_full_bwd_s": t_bwd, "t_full_s": t_fwd + t_bwd,
        "tflops": flops / (t_fwd + t_bwd) / 1e12,
        "sample": (f"reference lnoccsdt_contract(mat=I) over a in [0,1) ({jobs_f} jobs) + "
                   f"ccsd_t_energy_vjp over a<{A} ({jobs_b} jobs), extrapolated to {n_canon} "
                   f"canonical jobs"),
    }


# ---------------------------------------------------------------------------
# LNO (T): lnoccsdt_contract / lnoccsdt_energy_vjp with a full projector.
# Both enumerate jobs a in all, b in [b0,b1), c <= b (lno_ccsd_t.c:73-94,
# lno_ccsd_t_vjp.c:355-397): v * v(v+1)/2 jobs for the whole problem.
# ---------------------------------------------------------------------------
def _lno_inputs(o, v):
    n = o + v
    t1T = np.full((v, o), 1e-2)
    t2T = np.full((v, v, o, o), 1e-2)
    vooo = np.full((v, o, o, o), 1e-3)
    fvo = np.zeros((v, o))
    mat = np.full((o, o), 0.05) + np.eye(o)
    mo = np.concatenate([np.linspace(-1.5, -0.3, o), np.linspace(0.2, 3.0, v)])
    return n, t1T, t2T, vooo, fvo, mat, mo


def time_lno_forward_slice(lib, o, v):
    n, t1T, t2T, vooo, fvo, mat, mo = _lno_inputs(o, v)
    vvop = np.full((v, v, o, n), 1e-3)
    et = np.zeros(1)
    t0 = time.perf_counter()
    lib.lnoccsdt_contract(_p(et), _p(mat), _p(mo), _p(t1T), _p(t2T), _p(vooo), _p(fvo),
                          ctypes.c_int(o), ctypes.c_int(v), ctypes.c_int(0), ctypes.c_int(1), _p(vvop))
    return time.perf_counter() - t0, v * (v + 1) // 2


def time_lno_vjp_slice(lib, o, v, B):
    """b, c in [0, B): the reference's diagonal block (lno/ccsd_t.py:195-205)."""
    n, t1T, t2T, vooo, fvo, mat, mo = _lno_inputs(o, v)
    row = np.full((B, v, o, n), 1e-3)
    col = np.full((v, B, o, n), 1e-3)
    row_bar, col_bar = np.zeros_like(row), np.zeros_like(col)
    bars = [np.zeros_like(mat), np.zeros(n), np.zeros_like(t1T), np.zeros_like(t2T), np.zeros_like(vooo),
            np.zeros_like(fvo)]
    t0 = time.perf_counter()
    lib.lnoccsdt_energy_vjp(_p(mat), _p(mo), _p(t1T), _p(t2T), _p(vooo), _p(fvo), ctypes.c_double(2.0 / 3.0),
                            ctypes.c_int(o), ctypes.c_int(v), ctypes.c_int(0), ctypes.c_int(B), ctypes.c_int(0),
                            ctypes.c_int(B), _p(row), _p(col), _p(row), _p(col), *[_p(b) for b in bars],
                            _p(row_bar), _p(col_bar), _p(row_bar), _p(col_bar))
    return time.perf_counter() - t0, v * B * (B + 1) // 2


def measure_lno(o, v, target_s=8.0):
    lib = O._lib("ref")
    B = min(v, 2)
    dt_b, jobs_b = time_lno_vjp_slice(lib, o, v, B)
    while dt_b < 0.25 * target_s and B < v:
        per = dt_b / jobs_b
        B_new = B
        while B_new < v and v * B_new * (B_new + 1) // 2 < target_s / per:
            B_new += 1
        if B_new == B:
            break
        B = B_new
        dt_b, jobs_b = time_lno_vjp_slice(lib, o, v, B)
    dt_f, jobs_f = time_lno_forward_slice(lib, o, v)
    n_jobs = v * v * (v + 1) // 2
    t_fwd = dt_f / jobs_f * n_jobs
    t_bwd = dt_b / jobs_b * n_jobs
    flops = 8.0 * o ** 3 * v ** 4
    return {
        "nocc": o, "nvir": v, "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())),
        "fwd_slice_jobs": jobs_f, "fwd_slice_s": dt_f, "bwd_slice_jobs": jobs_b, "bwd_slice_s": dt_b,
        "bwd_slice_b_max": B, "lno_jobs": n_jobs,
        "t_full_fwd_s": t_fwd, "t_full_bwd_s": t_bwd, "t_full_s": t_fwd + t_bwd,
        "tflops": flops / (t_fwd + t_bwd) / 1e12,
        "sample": (f"reference lnoccsdt_contract over a in [0,1) ({jobs_f} jobs) + lnoccsdt_energy_vjp over "
                   f"b,c < {B} ({jobs_b} jobs), extrapolated to {n_jobs} LNO jobs"),
    }


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("nocc", type=int)
    ap.add_argument("nvir", type=int)
    ap.add_argument("--target", type=float, default=8.0)
    ap.add_argument("--lno", action="store_true", help="the LNO (projected) kernels instead of the canonical ones")
    a = ap.parse_args()
    print(json.dumps(measure_lno(a.nocc, a.nvir, a.target) if a.lno else measure(a.nocc, a.nvir, a.target)))
