"""Many (T) problems of uneven size in one CUDA-graph launch.

The reference evaluates one molecule per call (pyscfad/cc/ccsd_t.py:28-192);
a screening or training workload has hundreds of small, differently sized
problems, each far too small to fill a B200.  ``BatchedTriples`` runs E(T)
and its VJP for all of them with one of two engines:

* ``engine="batch"`` (default in the mixed modes): the library's batched
  entry points (``triples_batch_*``).  Each problem keeps its own workspace;
  chunk step c launches every kernel kind (W contraction, Wbar scale,
  epilogue, energy sum, the four adjoint contractions) ONCE over the c-th
  chunk of every problem, the persistent kernels pulling tiles from a job
  table built when the batch is created.  A batch of 256 small problems is
  a few hundred launches instead of tens of thousands.
* ``engine="lanes"``: one ``triples_energy_vjp_ex`` call per problem, spread
  over ``lanes`` CUDA streams (largest first, each to the least-loaded
  lane), one workspace per lane.

Either way ``capture()`` records the whole batch as ONE CUDA graph and
``run()`` replays it with a single launch and no host work per problem.
``Autotuner`` picks, per problem shape (nocc, nvir, precision), the chunk
block size Tv and, in the mixed modes, the N tile of the tensor-core W
contraction (128 or 256 columns) by timing each candidate once (results are
cached per process and can be saved to / loaded from a JSON file); the batch
engine uses the tuned N tile with Tv = 16, which keeps the number of chunk
steps smallest.

Inputs are copied once into device buffers owned by the batch; ``update()``
refreshes their values in place (same shapes) before the next ``run()``.
"""
from __future__ import annotations

import ctypes
import json
import os
import time
from dataclasses import dataclass

import torch

from . import _lib, triples

KEYS = triples.KEYS
TV_CANDIDATES = (4, 8, 16)
TILE_N_CANDIDATES = (128, 256)   # tensor-core W contraction (mixed precision only)


@dataclass
class _Problem:
    nocc: int
    nvir: int
    packed: bool
    inputs: list      # device tensors in KEYS order
    grads: dict       # device tensors, KEYS -> gradient
    energy: torch.Tensor
    tv: int = 16
    tile_n: int = 0
    lane: int = 0


class Autotuner:
    """(block size Tv, W-contraction N tile) per (nocc, nvir, precision,
    packed), chosen by timing every candidate pair once."""

    def __init__(self, path: str | None = None):
        self.path = path
        self.table: dict = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.table = {tuple(json.loads(k)): v for k, v in json.load(f).items()}

    def save(self):
        if self.path:
            with open(self.path, "w") as f:
                json.dump({json.dumps(list(k)): v for k, v in self.table.items()}, f, indent=1)

    def best(self, prob: _Problem, precision: str, ws: torch.Tensor, stream: torch.cuda.Stream):
        key = (prob.nocc, prob.nvir, precision, int(prob.packed))
        if key in self.table:
            return _choice(self.table[key])
        lib = _lib.load()
        prec = _lib.PRECISION[precision]
        times = {}
        tile_ns = TILE_N_CANDIDATES if precision != "fp64" else (0,)
        for tv in TV_CANDIDATES:
            if prob.nocc * tv > 1024:
                continue
            for tn in tile_ns:
                for rep in range(2):      # first call: one-time set-up; second: timed
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    _call(lib, prec, prob, ws, stream, tv, tn)
                    torch.cuda.synchronize()
                    dt = time.perf_counter() - t0
                times[(tv, tn)] = dt
        tv, tn = min(times, key=times.get)
        self.table[key] = [tv, tn]
        return tv, tn


def _choice(entry):
    """A table entry: [Tv, N tile] (a bare Tv from older tables means the default N tile)."""
    if isinstance(entry, (list, tuple)):
        return int(entry[0]), int(entry[1])
    return int(entry), 0


def _call(lib, prec, prob: _Problem, ws: torch.Tensor, stream: torch.cuda.Stream, tv: int, tile_n: int = 0):
    opt = _lib.options(block_size=tv, tile_n=tile_n)
    rc = lib.triples_energy_vjp_ex(stream.cuda_stream, prec, prob.nocc, prob.nvir, int(prob.packed),
                                   *[a.data_ptr() for a in prob.inputs], 1.0, 1, ctypes.byref(opt), ws.data_ptr(),
                                   ws.numel(), prob.energy.data_ptr(), *[prob.grads[k].data_ptr() for k in KEYS])
    _lib.check(rc, "triples_energy_vjp_ex")


class BatchedTriples:
    """E(T) + VJP (adjoint seed 1) for a list of problems, replayed as one graph.

    ``problems``: iterable of dicts with the KEYS arrays (reference layouts,
    FP64; ovvv packed or full) -- numpy arrays or tensors.
    """

    def __init__(self, problems, precision: str = "mixed", lanes: int = 8, device=None,
                 autotuner: Autotuner | None = None, tune: bool = True, engine: str | None = None):
        self.device = torch.device(device or "cuda")
        self.precision = precision
        self.lib = _lib.load()
        self.prec = _lib.PRECISION[precision]
        self.engine = engine or ("batch" if precision != "fp64" else "lanes")
        if self.engine not in ("batch", "lanes"):
            raise ValueError(f"unknown engine {self.engine!r}")
        self.problems: list[_Problem] = []
        for p in problems:
            ins = [torch.as_tensor(p[k], dtype=torch.float64).to(self.device).contiguous() for k in KEYS]
            o, v, packed = _shape_of(ins)
            grads = {k: torch.empty_like(a) for k, a in zip(KEYS, ins)}
            self.problems.append(_Problem(o, v, packed, ins, grads,
                                          torch.zeros((), dtype=torch.float64, device=self.device)))
        self.lanes = max(1, min(int(lanes), len(self.problems)))
        self.streams = [torch.cuda.Stream(self.device) for _ in range(self.lanes)]
        self.autotuner = autotuner or Autotuner()
        self._tune(tune)
        self._assign_lanes()
        self.graph = None
        self.handle = None
        if self.engine == "batch":
            for prob in self.problems:
                prob.tv = 16 if prob.nocc * 16 <= 1024 else 8
            self._create_batch()
            self.workspaces = []
        else:
            self.workspaces = [torch.empty(max(self._ws_bytes(l), 256), dtype=torch.uint8, device=self.device)
                               for l in range(self.lanes)]

    def _create_batch(self):
        n = len(self.problems)
        arr = (_lib.Problem * n)()
        for i, prob in enumerate(self.problems):
            q = arr[i]
            q.nocc, q.nvir, q.ovvv_packed = prob.nocc, prob.nvir, int(prob.packed)
            q.block_size, q.tile_n = prob.tv, prob.tile_n
            for k, a in zip(KEYS, prob.inputs):
                setattr(q, k, a.data_ptr())
            q.e_out = prob.energy.data_ptr()
            for k in KEYS:
                setattr(q, k + "_bar", prob.grads[k].data_ptr())
        self._problem_array = arr
        nbytes = int(self.lib.triples_batch_workspace_size(self.prec, n, arr))
        if nbytes == 0:
            raise _lib.TriplesError(1, "triples_batch_workspace_size")
        self.batch_workspace = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        handle = ctypes.c_void_p()
        torch.cuda.synchronize(self.device)
        _lib.check(self.lib.triples_batch_create(self.prec, n, arr, 1.0, self.batch_workspace.data_ptr(), nbytes,
                                                 ctypes.byref(handle)), "triples_batch_create")
        self.handle = handle

    def __del__(self):
        handle = getattr(self, "handle", None)
        if handle is not None and handle.value:
            self.lib.triples_batch_destroy(handle)
            self.handle = None

    # -- set-up ---------------------------------------------------------------
    def _size(self, prob: _Problem, tv: int) -> int:
        opt = _lib.options(block_size=tv)
        return int(self.lib.triples_workspace_size_ex(self.prec, prob.nocc, prob.nvir, int(prob.packed), 1,
                                                      ctypes.byref(opt)))

    def _tune(self, tune: bool):
        stream = self.streams[0]
        scratch = None
        for prob in self.problems:
            if not tune:
                prob.tv = 16 if prob.nocc * 16 <= 1024 else 8
                prob.tile_n = 0
                continue
            key = (prob.nocc, prob.nvir, self.precision, int(prob.packed))
            if key not in self.autotuner.table:
                need = max(self._size(prob, tv) for tv in TV_CANDIDATES if prob.nocc * tv <= 1024)
                if scratch is None or scratch.numel() < need:
                    scratch = torch.empty(need, dtype=torch.uint8, device=self.device)
                with torch.cuda.stream(stream):
                    self.autotuner.best(prob, self.precision, scratch, stream)
            prob.tv, prob.tile_n = _choice(self.autotuner.table[key])
        torch.cuda.synchronize()

    def _cost(self, prob: _Problem) -> float:
        return float(prob.nocc) ** 3 * float(prob.nvir) ** 4

    def _assign_lanes(self):
        load = [0.0] * self.lanes
        for i in sorted(range(len(self.problems)), key=lambda i: -self._cost(self.problems[i])):
            lane = min(range(self.lanes), key=lambda l: load[l])
            self.problems[i].lane = lane
            load[lane] += self._cost(self.problems[i])

    def _ws_bytes(self, lane: int) -> int:
        return max([self._size(p, p.tv) for p in self.problems if p.lane == lane] or [0])

    def _enqueue(self):
        """The whole batch on the current stream (batch engine), or all calls of all
        lanes on their streams, forked from / joined into the current stream."""
        main = torch.cuda.current_stream(self.device)
        if self.engine == "batch":
            _lib.check(self.lib.triples_batch_run(self.handle, main.cuda_stream), "triples_batch_run")
            return
        fork = torch.cuda.Event()
        fork.record(main)
        for lane, st in enumerate(self.streams):
            st.wait_event(fork)
            for prob in self.problems:
                if prob.lane != lane:
                    continue
                _call(self.lib, self.prec, prob, self.workspaces[lane], st, prob.tv, prob.tile_n)
            join = torch.cuda.Event()
            join.record(st)
            main.wait_event(join)

    def capture(self):
        """Record the whole batch as one CUDA graph (after one eager warm-up pass)."""
        self._enqueue()
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(self.device)
        with torch.cuda.graph(self.graph, stream=cap):
            self._enqueue()
        torch.cuda.synchronize()
        return self

    # -- execution ------------------------------------------------------------
    def run(self):
        """One graph launch for all problems (captures on first use)."""
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def run_eager(self):
        """The same calls, one launch sequence per problem, no graph."""
        self._enqueue()

    def update(self, i: int, problem: dict):
        """New input values (same shapes) for problem i, used by the next run()."""
        for a, k in zip(self.problems[i].inputs, KEYS):
            a.copy_(torch.as_tensor(problem[k], dtype=torch.float64))

    def results(self):
        """[(E, {key: gradient})] in input order (synchronises)."""
        torch.cuda.synchronize()
        return [(float(p.energy), p.grads) for p in self.problems]

    def check(self):
        """Device-side status of the last run (synchronises)."""
        if self.engine == "batch":
            _lib.check(self.lib.triples_batch_check_device_status(
                self.handle, torch.cuda.current_stream(self.device).cuda_stream), "batched run")
            return
        for lane, st in enumerate(self.streams):
            _lib.check(self.lib.triples_check_device_status(st.cuda_stream, self.workspaces[lane].data_ptr()),
                       f"batched lane {lane}")


def _shape_of(ins):
    mo_energy, t1, t2, ovoo, ovov, ovvv, fvo = ins
    return triples._shapes(t1, t2, ovoo, ovov, ovvv, fvo, mo_energy)
