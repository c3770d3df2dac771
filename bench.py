"""Benchmark: CCSD(T) energy + VJP throughput on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision mixed|mixed_bf16|fp64] [--workload NAME]

One step = E(T) plus its full VJP (ybar = 1) for one (T) problem of the
workload's shape (default large_o40v360: nocc=40, nvir=360, naux=1200),
seeded synthetic inputs with the reference benchmark's distributions.
Metric: TFLOP/s at the algorithmic count 8*o^3*v^4 per step (forward
2*o^3*v^4 + backward with recompute 6*o^3*v^4).

Multi-GPU: the (T) problem of this workload fits one GPU, so --gpus N runs N
independent replicas (one process per GPU under torchrun); value = N
problems / max-over-ranks time ("weak" scaling).  No data-path collective.

--impl reference times the reference's own CPU kernels (compiled from its
sources into oracle/_ref) on the host cores on a bounded job sample and
extrapolates to the full workload; rank 0 alone runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "(T) E+VJP TFLOP/s (o=40,v=360): mixed-prec vs FP64 on B200 at |dE|<=1e-7 Eh"
WORKLOADS = {
    "water_ccpvdz_o5v19": (5, 19, 80),
    "small_o14v96": (14, 96, 400),
    "medium_o20v180": (20, 180, 600),
    "large_o40v360": (40, 360, 1200),
    "huge_o50v450": (50, 450, 1500),
}
DATA = ("synthetic: seeded mo_energy occ~U(-1.5,-0.3) vir~U(0.2,3.0) sorted, t1~N(0,1e-2), "
        "t2~N(0,2e-2) symmetrised, ERIs from Cholesky-like factors L~N(0,0.1) (naux), fvo=0, "
        "packed ovvv")


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def max_over_ranks(x, device=None):
    """Largest value of x over all ranks (the slowest replica sets the job time)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t)


def job_throughput(world, steps, flops_per_step, t_max):
    """Whole-job TFLOP/s: every replica ran `steps` steps; the job took t_max seconds."""
    return world * steps * flops_per_step / t_max / 1e12


# Wall-clock plan of one bench run.  A headline step (E+VJP at o=40, v=360)
# takes tens of seconds, so the requested --steps/--warmup may not fit the
# run's wall-clock budget; the plan keeps at least MIN_WARMUP warm-up steps
# (the first one carries the library's one-time set-up) and times as many of
# the requested steps as the budget allows, reporting the count it timed.
MIN_WARMUP = 3


def plan_steps(step_s, elapsed_s, steps, warmup, budget_s, reserve_s, e2e_max=2):
    """(warm-up steps in total, timed steps, e2e steps) for a step of step_s
    seconds, elapsed_s seconds already spent (one warm-up step included),
    `steps`/`warmup` requested, budget_s for the whole run and reserve_s kept
    for the CPU leg and the output.  Never fewer than one timed and one e2e
    step; warm-up min(warmup, MIN_WARMUP) when warmup >= 1."""
    step_s = max(float(step_s), 1e-6)
    warm = max(1, min(int(warmup), MIN_WARMUP)) if warmup >= 1 else 1
    left = budget_s - elapsed_s - reserve_s - (warm - 1) * step_s
    e2e = max(1, min(e2e_max, int(steps)))
    timed = int(max(0.0, left - e2e * step_s * 1.1) // step_s)
    timed = max(1, min(int(steps), timed))
    if timed < e2e:
        e2e = timed
    return warm, timed, e2e


def algorithmic_flops(o, v):
    """Per step and per kernel class (the tensor contractions only)."""
    main = 2.0 * o ** 3 * v ** 4
    ooov = 2.0 * o ** 4 * v ** 3
    return {
        "step": 8.0 * o ** 3 * v ** 4,
        "f1_contract": main + ooov,
        "b1a_ovvv_grad": main,
        "b1b_t2_grad": main,
        "b1c_ovoo_grad": ooov,
        "b1d_t2_ooov_grad": ooov,
    }


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        loaded = [x for x in sm if x > 0.5 * (smax or max(sm))] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU legs (reference kernels from oracle/_ref)
# ---------------------------------------------------------------------------
def cpu_reference_measure(o, v, target_s=8.0):
    cores = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(cores), OPENBLAS_NUM_THREADS="1")
    env.pop("CUDA_VISIBLE_DEVICES", None)
    try:
        out = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "cpu_baseline.py"), str(o), str(v),
                              "--target", str(target_s)], env=env, capture_output=True, text=True,
                             timeout=900, check=True)
        return json.loads(out.stdout.strip().splitlines()[-1])
    except Exception as exc:  # noqa: BLE001 - reported, not fatal for the GPU line
        return {"error": f"{type(exc).__name__}: {exc}"[:300]}


def run_reference(args, o, v, rank):
    """The reference's CPU kernels on the host cores, measured ONCE: a full
    step at o=40, v=360 would take hours on the CPU, so the step time is
    extrapolated from one bounded job sample (forward slice + backward slice,
    both the reference's own C code).  Repeating an extrapolation adds
    nothing, so --steps/--warmup do not repeat it; the line says so."""
    if rank != 0:
        return
    t_start = time.perf_counter()
    res = cpu_reference_measure(o, v, args.cpu_target)
    if "error" in res:
        print(json.dumps({"impl": "reference", "unavailable": res["error"]}))
        return
    t = res["t_full_s"]
    flops = algorithmic_flops(o, v)["step"]
    val = flops / t / 1e12
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "TFLOP/s", "n_gpus": 0,
        "steps": 1, "warmup": 0, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
        "config": {"workload": args.workload, "nocc": o, "nvir": v, "naux": WORKLOADS[args.workload][2],
                   "path": "reference CPU C kernels (ccsd_t_energy_vjp + LNO forward with mat=I)",
                   "timing": ("one bounded job sample extrapolated to the full step (measured once; "
                              "warm-up does not apply to an extrapolation)"),
                   "sample_wall_s": round(time.perf_counter() - t_start, 1)},
        "cpu_baseline": {"value": val, "unit": "TFLOP/s", "cores": res["cores"], "kind": "reference",
                         "sample": res["sample"]},
        "e2e": {"value": val, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU leg
# ---------------------------------------------------------------------------
def load_traffic(workload, precision):
    path = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get(f"{workload}:{precision}", {})
    except (OSError, ValueError):
        return {}


def run_batched(args):
    """Many small uneven problems: the batch engine (one launch per kernel kind
    and chunk step over all problems) replayed as one CUDA graph, against one
    E+VJP call per problem on one stream and against the per-problem calls
    spread over 8 streams and captured as one graph."""
    import numpy as np
    import torch

    from pyscfad_b200 import triples
    from pyscfad_b200.batched import Autotuner, BatchedTriples
    from pyscfad_b200.synthetic import make_inputs_torch

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(args.seed)
    probs = []
    for i in range(args.instances):
        o = int(rng.integers(4, 13))
        v = int(rng.integers(20, 81))
        inp = make_inputs_torch(o, v, 4 * (o + v), seed=args.seed + 1000 + i, device=dev)
        il, jl = torch.tril_indices(v, v, device=dev)
        inp["ovvv"] = inp["ovvv"][:, :, il, jl].contiguous()
        probs.append({k: inp[k] for k in triples.KEYS})
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, reps):
        for _ in range(max(args.warmup, 1)):
            fn()
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(reps):
            fn()
        ev[1].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / 1e3 / reps

    t0 = time.perf_counter()
    bt = BatchedTriples(probs, precision=args.precision, tune=False, engine="batch")
    t_create = time.perf_counter() - t0
    t0 = time.perf_counter()
    bt.capture()
    t_cap = time.perf_counter() - t0
    lib = bt.lib
    lib.triples_profile_enable(1)
    t_graph = timed(bt.run, max(args.steps, 3))
    e_graph = np.array([e for e, _ in bt.results()])
    bt.check()
    t_eager = timed(bt.run_eager, 1)
    import ctypes
    ncat = 16
    ms, cnt = (ctypes.c_double * ncat)(), (ctypes.c_int * ncat)()
    ncat = lib.triples_profile_read(ncat, ms, cnt)
    lib.triples_profile_enable(0)
    launches_eager = int(sum(cnt[i] for i in range(ncat)))   # profiled: the eager runs (warm-up + timed)
    nrun = max(args.warmup, 1) + 1
    kernel_ms = {lib.triples_profile_name(i).decode(): round(ms[i] / nrun, 3) for i in range(ncat) if cnt[i]}
    flops = sum(8.0 * p["t1"].shape[0] ** 3 * p["t1"].shape[1] ** 4 for p in probs)

    def one_by_one():
        for p in probs:
            triples.energy_vjp(*(p[k] for k in triples.KEYS), precision=args.precision, device=dev, check=False)

    t_single = timed(one_by_one, 1)
    del bt
    torch.cuda.empty_cache()
    lanes = BatchedTriples(probs, precision=args.precision, lanes=8, tune=False, engine="lanes")
    lanes.capture()
    t_lanes = timed(lanes.run, max(args.steps, 3))
    n = len(probs)
    line = {"metric": "(T) E+VJP instances/s, batched uneven problems", "impl": "ours",
            "config": {"workload": "batched_c3", "instances": n, "nocc": "U{4..12}", "nvir": "U{20..80}",
                       "naux": "4(o+v)", "precision": args.precision, "engine": "batch (one launch per kernel "
                       "kind and chunk step over all problems), one CUDA graph"},
            "unit": "instances/s", "higher_is_better": True,
            "value": n / t_graph,
            "graph_instances_per_s": n / t_graph, "graph_ms_per_batch": t_graph * 1e3,
            "tflops_at_8o3v4": flops / t_graph / 1e12,
            "eager_batch_instances_per_s": n / t_eager,
            "launches_per_batch": launches_eager // nrun, "kernel_ms_per_batch_eager": kernel_ms,
            "one_call_per_instance_per_s": n / t_single,
            "lanes_graph_instances_per_s": n / t_lanes,
            "speedup_vs_one_call_per_instance": t_single / t_graph,
            "speedup_vs_lanes_graph": t_lanes / t_graph,
            "create_s": t_create, "capture_s": t_cap,
            "e_sum": float(e_graph.sum())}
    print(json.dumps(line))


def run_accuracy(args, o, v, naux):
    """Precision report: the mixed modes against the FP64 path on the same seeded
    inputs, with the FP64-vs-FP64 difference of two summation orders (block
    sizes 16 and 8) as the noise floor."""
    import numpy as np
    import torch

    from pyscfad_b200 import triples
    from pyscfad_b200.synthetic import make_inputs_torch

    dev = torch.device("cuda", 0)
    inp = make_inputs_torch(o, v, naux, seed=args.seed, device=dev, fvo_sigma=1e-3, scale=args.scale)
    il, jl = torch.tril_indices(v, v, device=dev)
    inp["ovvv"] = inp["ovvv"][:, :, il, jl].contiguous()
    xs = [inp[k] for k in triples.KEYS]

    a0, a1 = args.slice if args.slice else (0, 0)
    stream = torch.cuda.current_stream(dev)

    # The FP64 form may run with a smaller virtual block (--fp64-block) so its
    # FP64 staging fits next to the inputs at the largest sizes (likewise
    # --mixed-block); a slice of 16-wide blocks [a0, a1) is the slice
    # [a0 16/tv, a1 16/tv) of tv-wide blocks (the same virtual triples
    # a >= b >= c with a in [16 a0, 16 a1)).  Gradients stay on the device and
    # are compared there, one input at a time.
    tv64 = args.fp64_block

    def run(prec, tv=0):
        s = 16 // (tv or 16)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        e, g = triples.energy_vjp(*xs, ybar=1.0, precision=prec, device=dev, block_size=tv,
                                  chunk_range=(a0 * s, a1 * s),
                                  accumulation_segment=0 if prec == "fp64" else args.accumulation_segment)
        t1.record(stream)
        torch.cuda.synchronize()
        out = float(e), g, t0.elapsed_time(t1) / 1e3
        triples.release_workspace()
        torch.cuda.empty_cache()
        return out

    precs = ("mixed",) if args.no_bf16 else ("mixed", "mixed_bf16")
    tvm = args.mixed_block if args.mixed_block != 16 else 0
    if args.slice:   # one-time set-up of both paths outside the timed calls
        for prec in ("fp64",) + precs:
            tvp = tv64 if prec == "fp64" else (tvm or 16)
            triples.energy_vjp(*xs, ybar=1.0, precision=prec, device=dev, chunk_range=(0, 16 // tvp),
                               block_size=tvp)
            torch.cuda.synchronize()
            triples.release_workspace()
            torch.cuda.empty_cache()
    e64, g64, t64 = run("fp64", tv64)
    e64b = e64 if args.slice else run("fp64", 8 if tv64 == 16 else 16)[0]

    def relerr(a, b):
        return float((a - b).abs().max() / max(float(b.abs().max()), 1e-300))

    out = {"workload": args.workload, "nocc": o, "nvir": v, "naux": naux, "scale": args.scale,
           "accumulation_segment": args.accumulation_segment,
           "e_fp64": e64, "fp64_seconds": t64, "fp64_block": tv64, "mixed_block": tvm or 16}
    if args.slice:
        frac = triples.chunk_fraction(v, a0, a1)
        out.update({"slice_blocks": [a0, a1], "slice_fraction_of_amplitudes": frac,
                    "fp64_seconds_full_extrapolated": t64 / frac})
    else:
        out.update({"fp64_noise_abs": abs(e64 - e64b), "fp64_noise_rel": abs(e64 - e64b) / abs(e64)})
    for prec in precs:
        e, g, tm = run(prec, tvm)
        out[prec] = {"e": e, "abs_dE": abs(e - e64), "rel_dE": abs(e - e64) / abs(e64), "seconds": tm,
                     "speedup_vs_fp64": t64 / tm,
                     "grad_rel_err": {k: relerr(g[k], g64[k]) for k in g64}}
        del g
        torch.cuda.empty_cache()
    print(json.dumps(out))


# ---------------------------------------------------------------------------
# LNO fragment (T): projector on the first occupied index
# ---------------------------------------------------------------------------
LNO_METRIC = "LNO (T) E+VJP TFLOP/s (projected first occupied index), B200 vs reference CPU kernels"
# algorithmic bytes per raw amplitude position of each LNO epilogue pass
# (sz = staging element size: 8 FP64, 4 mixed): tile forward reads w, writes
# WW and Q; the projection reads WW, Q and writes Zbar, Dbar, P^T(Wtbar);
# tile adjoint reads Zbar, P^T(Wtbar), writes vbar and the Wbar operand
# (FP64, or two 16-bit halves); V gradients read vbar, Dbar.
def lno_pass_bytes(sz):
    return {"lno_tile_fwd": sz + 16, "lno_projection": 40, "lno_tile_adj": 16 + 8 + (8 if sz == 8 else 4),
            "lno_vgrad": 16}


def run_lno(args, o, v, naux):
    import ctypes

    import numpy as np
    import torch

    from pyscfad_b200 import _lib, triples
    from pyscfad_b200.synthetic import make_inputs_torch

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    inp = make_inputs_torch(o, v, naux, seed=args.seed, device=dev)
    il, jl = torch.tril_indices(v, v, device=dev)
    inp["ovvv"] = inp["ovvv"][:, :, il, jl].contiguous()
    # projector of a fragment with half the occupied orbitals: mat = ulo^T ulo
    rng = np.random.default_rng(1000 + args.seed)
    ulo = np.linalg.qr(rng.normal(size=(o, o)))[0][: max(1, o // 2)]
    mat = torch.tensor(ulo.T @ ulo, dtype=torch.float64, device=dev)
    dev_args = [mat] + [inp[k] for k in triples.KEYS]

    def step(a):
        return triples.lno_energy_vjp(*a, ybar=1.0, precision=args.precision, device=dev, check=False)

    for _ in range(args.warmup):
        e, g = step(dev_args)
    torch.cuda.synchronize()
    _lib.check(triples.device_status(dev), "warm-up")
    e_val = float(e)
    del g
    clocks = ClockSampler(0)
    torch.cuda.synchronize()
    clocks.start()
    lib.triples_profile_enable(1)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    for _ in range(args.steps):
        e, g = step(dev_args)
    s1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ncat = 16
    ms, cnt = (ctypes.c_double * ncat)(), (ctypes.c_int * ncat)()
    ncat = lib.triples_profile_read(ncat, ms, cnt)
    lib.triples_profile_enable(0)
    prof = {lib.triples_profile_name(i).decode(): (ms[i], cnt[i]) for i in range(ncat)}
    t_dev = s0.elapsed_time(s1) / 1e3
    _lib.check(triples.device_status(dev), "timed steps")
    del g
    flops = algorithmic_flops(o, v)["step"]
    value = args.steps * flops / t_dev / 1e12

    host_in = [a.cpu().pin_memory() for a in dev_args]
    h2d = sum(a.numel() * a.element_size() for a in host_in)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    grads_host, d2h = None, 0
    for _ in range(args.steps):
        dev_in = [a.to(dev, non_blocking=True) for a in host_in]
        ee, gg = step(dev_in)
        if grads_host is None:
            grads_host = {k: torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for k, t in gg.items()}
            e_host = torch.empty((), dtype=torch.float64, pin_memory=True)
        e_host.copy_(ee, non_blocking=True)
        for k, t in gg.items():
            grads_host[k].copy_(t, non_blocking=True)
        d2h = 8 + sum(t.numel() * t.element_size() for t in gg.values())
        del dev_in, gg
    e1.record()
    torch.cuda.synchronize()
    t_e2e = e0.elapsed_time(e1) / 1e3

    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        pass
    hpeak, hnote = (float(peaks["hbm_gbs"]), "of measured (copy)") if "hbm_gbs" in peaks else (6650.0, "of fallback")
    positions = float(o) ** 3 * float(v) ** 3
    pbytes = lno_pass_bytes(8 if args.precision == "fp64" else 4)
    total_ms = sum(m for m, _ in prof.values()) or 1.0
    classes = {}
    for k, b in pbytes.items():
        m, c = prof.get(k, (0.0, 0))
        if c <= 0 or m <= 0:
            continue
        ach = b * positions * args.steps / (m / 1e3) / 1e9
        classes[k] = {"bound": "hbm", "achieved": ach, "peak": hpeak, "unit": "GB/s", "frac": ach / hpeak,
                      "kernel": k, "launches": c, "avg_launch_ms": m / c, "share": m / total_ms,
                      "bytes_per_position": b}
    roof = None
    if classes:
        dom = max(classes, key=lambda k: prof[k][0])
        roof = dict(classes[dom])
        roof["traffic"] = load_traffic("lno_" + args.workload, args.precision).get(dom)
        roof["peak_note"] = hnote
        roof["classes"] = {k: {kk: (round(vv, 4) if isinstance(vv, float) else vv) for kk, vv in c.items()
                               if kk in ("achieved", "frac", "share")} for k, c in classes.items()}
    line = {
        "metric": LNO_METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_dev / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else (
            "fp16x3-split f32acc, f64 LNO epilogue" if args.precision == "mixed" else "bf16x3-split f32acc, f64 LNO epilogue"),
        "data": DATA + "; projector mat = ulo^T ulo, ulo = o/2 orthonormal rows (seeded)",
        "config": {"workload": "lno_" + args.workload, "nocc": o, "nvir": v, "naux": naux,
                   "precision": args.precision, "nlo": max(1, o // 2), "l2": "chunk work arrays larger than L2",
                   "e_t": e_val},
        "e2e": {"value": args.steps * flops / t_e2e / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(sum(c for _, c in prof.values())),
        "kernel_ms": {k: round(m, 3) for k, (m, _) in prof.items()},
        "roofline": roof,
        "clocks": clk,
    }
    if not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        env = dict(os.environ, OMP_NUM_THREADS=str(cores), OPENBLAS_NUM_THREADS="1")
        try:
            out = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "cpu_baseline.py"), str(o), str(v),
                                  "--target", str(args.cpu_target), "--lno"], env=env, capture_output=True,
                                 text=True, timeout=900, check=True)
            res = json.loads(out.stdout.strip().splitlines()[-1])
            line["cpu_baseline"] = {"value": res["tflops"], "unit": "TFLOP/s", "cores": res["cores"],
                                    "kind": "reference", "sample": res["sample"], "t_full_s": res["t_full_s"]}
        except Exception as exc:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "unit": "TFLOP/s", "error": f"{exc}"[:300]}
    print(json.dumps(line))


def main():
    t_start = time.perf_counter()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "mixed_bf16", "fp64"])
    ap.add_argument("--workload", default=None, choices=sorted(WORKLOADS),
                    help="default large_o40v360 (medium_o20v180 with --lno)")
    ap.add_argument("--shape", type=int, nargs=3, metavar=("NOCC", "NVIR", "NAUX"), default=None,
                    help="a custom (nocc, nvir, naux) instead of --workload (small cases for profiler captures)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-target", type=float, default=8.0, help="seconds per CPU backward sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--budget", type=float, default=1450.0,
                    help="wall-clock seconds the whole run may take; timed steps beyond it are not run "
                         "(the line reports the count timed)")
    ap.add_argument("--e2e-host-gb", type=float, default=32.0,
                    help="largest pinned host buffers (inputs + gradients) the e2e leg may allocate; the "
                         "headline workload needs 22 GB")
    ap.add_argument("--cpu-reserve", type=float, default=150.0,
                    help="seconds of the budget kept for the CPU-baseline leg")
    ap.add_argument("--accuracy", action="store_true",
                    help="instead of timing: mixed modes vs FP64 on the same inputs (|dE|, relative "
                         "errors, FP64 summation-order noise floor), one JSON line")
    ap.add_argument("--slice", type=int, nargs=2, metavar=("A0", "A1"), default=None,
                    help="with --accuracy: only the chunks whose largest virtual block is in [A0, A1), "
                         "timed in both precisions (FP64 vs mixed on identical work)")
    ap.add_argument("--fp64-block", type=int, default=16, choices=[4, 8, 16],
                    help="with --accuracy: virtual block size of the FP64 run (8 or 4 shrink its FP64 staging)")
    ap.add_argument("--accumulation-segment", type=int, default=0,
                    help="mixed precision: 64-wide K blocks per FP32 tensor-core accumulation segment (0: library default)")
    ap.add_argument("--mixed-block", type=int, default=16, choices=[4, 8, 16],
                    help="with --accuracy: virtual block size of the mixed-precision runs")
    ap.add_argument("--no-bf16", action="store_true", help="with --accuracy: skip the bf16 mode")
    ap.add_argument("--batched", action="store_true",
                    help="instead of the headline: 256 uneven problems (nocc 4-12, nvir 20-80, naux 4(o+v)) "
                         "as one CUDA-graph launch vs one call per problem; one JSON line")
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--lno", action="store_true",
                    help="instead of the headline: the LNO fragment (T) (projector on the first occupied "
                         "index, pyscfad/lno/ccsd_t.py) E+VJP on --workload (default medium_o20v180)")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="scale of the Cholesky-like factors (a small value gives a physically sized E(T))")
    args = ap.parse_args()

    if args.workload is None:
        args.workload = "medium_o20v180" if args.lno else "large_o40v360"
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.shape:
        o, v, naux = args.shape
        args.workload = "shape_o%dv%d" % (o, v)
        WORKLOADS[args.workload] = (o, v, naux)
    o, v, naux = WORKLOADS[args.workload]

    if args.impl == "reference":
        run_reference(args, o, v, rank)
        return
    if args.accuracy:
        run_accuracy(args, o, v, naux)
        return
    if args.batched:
        run_batched(args)
        return
    if args.lno:
        if rank == 0:
            run_lno(args, o, v, naux)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)

    from pyscfad_b200 import _lib, triples
    from pyscfad_b200.synthetic import make_inputs_torch

    lib = _lib.load()
    inp = make_inputs_torch(o, v, naux, seed=args.seed + rank, device=dev)
    il, jl = torch.tril_indices(v, v, device=dev)
    inp["ovvv"] = inp["ovvv"][:, :, il, jl].contiguous()   # packed DF layout (dfccsd.py:88)
    keys = triples.KEYS
    dev_args = [inp[k] for k in keys]
    ovvv_gb = inp["ovvv"].numel() * 8 / 1e9
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()

    def step():
        e, g = triples.energy_vjp(*dev_args, ybar=1.0, precision=args.precision, device=dev, check=False,
                                  accumulation_segment=args.accumulation_segment)
        return e, g

    # first warm-up step (one-time set-up included) sizes the plan; every rank
    # takes the same plan (the slowest rank's step time)
    w0 = time.perf_counter()
    e, g = step()
    torch.cuda.synchronize()
    step_s = max_over_ranks(time.perf_counter() - w0, dev)
    del g
    reserve = 0.0 if (args.no_cpu_baseline or world > 1) else args.cpu_reserve
    n_warm, n_steps, n_e2e = plan_steps(step_s, time.perf_counter() - t_start, args.steps, args.warmup,
                                        args.budget, reserve)
    for _ in range(n_warm - 1):
        e, g = step()
        del g
    torch.cuda.synchronize()
    _lib.check(triples.device_status(dev), "warm-up")
    e_val = float(e)

    # timed region: inputs resident in HBM
    clocks = ClockSampler(local_rank)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    lib.triples_profile_enable(1)
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record()
    torch.cuda.nvtx.range_push("timed_steps")   # lets a profiler select exactly the timed launches
    for _ in range(n_steps):
        e, g = step()
        del g
    torch.cuda.nvtx.range_pop()
    s1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    import ctypes
    ncat = 16
    ms = (ctypes.c_double * ncat)()
    cnt = (ctypes.c_int * ncat)()
    ncat = lib.triples_profile_read(ncat, ms, cnt)
    lib.triples_profile_enable(0)
    prof = {lib.triples_profile_name(i).decode(): (ms[i], cnt[i]) for i in range(ncat)}
    t_dev = s0.elapsed_time(s1) / 1e3
    t_dev = max_over_ranks(t_dev, dev)
    _lib.check(triples.device_status(dev), "timed steps")
    peak_mem = torch.cuda.max_memory_allocated(dev)   # inputs + gradients + workspace, input generation included

    flops = algorithmic_flops(o, v)
    value = job_throughput(world, n_steps, flops["step"], t_dev)

    # end-to-end through the public API with host buffers: pinned host inputs
    # copied in and E plus every gradient copied out, inside the timed region.
    # The device-resident inputs are dropped first (the e2e call copies its
    # own); pinned host buffers above --e2e-host-gb (inputs + gradients) are
    # not attempted, and the line says so.
    in_bytes = sum(a.numel() * a.element_size() for a in dev_args)
    h2d = in_bytes
    d2h = 8 + in_bytes
    e2e_value, e2e_note = None, None
    if (h2d + d2h) / 1e9 > args.e2e_host_gb:
        e2e_note = ("not run: %.1f GB of pinned host buffers exceed the %.0f GB allowed by --e2e-host-gb"
                    % ((h2d + d2h) / 1e9, args.e2e_host_gb))
    else:
        host_in = []
        for a in dev_args:
            hb = torch.empty(a.shape, dtype=a.dtype, pin_memory=True)
            hb.copy_(a)
            host_in.append(hb)
        grads_host = {k: torch.empty(a.shape, dtype=a.dtype, pin_memory=True) for k, a in zip(keys, dev_args)}
        e_host = torch.empty((), dtype=torch.float64, pin_memory=True)
        del dev_args, inp
        triples.release_workspace()
        torch.cuda.empty_cache()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n_e2e):
            dev_in = [a.to(dev, non_blocking=True) for a in host_in]
            ee, gg = triples.energy_vjp(*dev_in, ybar=1.0, precision=args.precision, device=dev, check=False,
                                        accumulation_segment=args.accumulation_segment)
            e_host.copy_(ee, non_blocking=True)
            for k in keys:
                grads_host[k].copy_(gg[k], non_blocking=True)
            del dev_in, gg
        e1.record()
        torch.cuda.synchronize()
        barrier()
        t_e2e = e0.elapsed_time(e1) / 1e3
        t_e2e = max_over_ranks(t_e2e, dev)
        e2e_value = job_throughput(world, n_e2e, flops["step"], t_e2e)
        del host_in, grads_host

    # roofline of the dominant kernel class
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        pass
    # per kernel class: tensor classes against the GEMM peak (algorithmic flops),
    # the epilogue against HBM bandwidth (algorithmic bytes: each raw amplitude
    # W read once, its adjoint Wbar written once); the dominant class by time
    # is the headline roofline
    elem = float(o) ** 3 * float(v) ** 3
    sz = 8 if args.precision == "fp64" else 4
    algo_bytes = {"f2_epilogue": elem * 2 * sz}
    if args.precision == "fp64":
        tpeak, tnote = 40.0, "nominal B200 FP64 (no measured FP64 peak on this pool)"
    elif "bf16_tflops_sustained" in peaks:
        tpeak, tnote = float(peaks["bf16_tflops_sustained"]), "of measured (cuBLAS bf16, sustained)"
    else:
        tpeak, tnote = 1400.0, "of fallback (sustained)"
    if "hbm_gbs" in peaks:
        hpeak, hnote = float(peaks["hbm_gbs"]), "of measured (copy)"
    else:
        hpeak, hnote = 6650.0, "of fallback"
    traffic_tab = load_traffic(args.workload, args.precision)
    total_ms = sum(m for m, _ in prof.values()) or 1.0
    classes = {}
    for k, (ms, cnt) in prof.items():
        if cnt <= 0 or ms <= 0:
            continue
        avg_s = ms / 1e3 / cnt
        if k in flops and k != "step":
            ach = flops[k] * n_steps / cnt / avg_s / 1e12
            ent = {"bound": "tensor", "achieved": ach, "peak": tpeak, "unit": "TFLOP/s", "frac": ach / tpeak}
            if args.precision != "fp64":
                ent["frac_emulated"] = ach / (tpeak / 3)   # 3 split products per FP32-level product
        elif k in algo_bytes:
            ach = algo_bytes[k] * n_steps / cnt / avg_s / 1e9
            ent = {"bound": "hbm", "achieved": ach, "peak": hpeak, "unit": "GB/s", "frac": ach / hpeak}
        else:
            continue
        ent.update({"kernel": k, "launches": cnt, "avg_launch_ms": avg_s * 1e3, "share": ms / total_ms})
        classes[k] = ent
    roof = None
    if classes:
        dom = max(classes, key=lambda k: prof[k][0])
        roof = dict(classes[dom])
        roof["traffic"] = traffic_tab.get(dom)
        bpa = traffic_tab.get(dom + "_bytes_per_amplitude")
        if roof["traffic"] is None and bpa is not None:
            # measured DRAM bytes per raw amplitude (ncu, smaller chunk) x this step's amplitudes, per launch
            roof["traffic"] = bpa * elem * n_steps / roof["launches"]
            roof["traffic_note"] = "%.1f DRAM bytes per raw amplitude (ncu) scaled to this launch" % bpa
        roof["peak_note"] = hnote if roof["bound"] == "hbm" else tnote
        roof["classes"] = {k: {kk: (round(vv, 4) if isinstance(vv, float) else vv) for kk, vv in c.items()
                               if kk in ("bound", "achieved", "frac", "frac_emulated", "share")}
                           for k, c in classes.items()}

    line = {
        "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": n_steps,
        "warmup": n_warm, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": t_dev / n_steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else (
            "fp16x3-split f32acc, f64 epilogue" if args.precision == "mixed" else "bf16x3-split f32acc, f64 epilogue"),
        "data": DATA,
        "config": {"workload": args.workload, "nocc": o, "nvir": v, "naux": naux, "precision": args.precision,
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (packed ovvv %.1f GB)" % (ovvv_gb),
                   "e_t": e_val,
                   "step_plan": ("warm-up %d, timed %d of %d requested, e2e %d: the steps that fit a %d s "
                                 "wall-clock budget at %.1f s per step" % (n_warm, n_steps, args.steps, n_e2e,
                                                                           args.budget, step_s))},
        "e2e": {"value": e2e_value, "unit": "TFLOP/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": n_e2e if e2e_value is not None else 0, **({"note": e2e_note} if e2e_note else {})},
        "gpu_launches": int(sum(c for _, c in prof.values())),
        "triplets_per_s": world * n_steps * (o * (o + 1) * (o + 2) // 6) / t_dev,
        "device_peak_gb": round(peak_mem / 1e9, 2),
        "kernel_ms": {k: round(m, 3) for k, (m, _) in prof.items()},
        "roofline": roof,
        "clocks": clk,
    }
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        res = cpu_reference_measure(o, v, args.cpu_target)
        if "error" in res:
            line["cpu_baseline"] = {"value": None, "unit": "TFLOP/s", "error": res["error"]}
        else:
            line["cpu_baseline"] = {"value": res["tflops"], "unit": "TFLOP/s", "cores": res["cores"],
                                    "kind": "reference", "sample": res["sample"]}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
