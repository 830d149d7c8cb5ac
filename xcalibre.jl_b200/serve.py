"""Serving: continuous batching of steady cases on one GPU.

A request is a steady case (a lid-driven cavity or a channel with its mesh,
Reynolds number and solver settings) that must be solved to a scaled residual
(1e-6 by default).  The server keeps every admitted case resident on the
device (fields, matrices, Krylov workspaces) inside one :class:`api.Batch`
and advances all of them one SIMPLE iteration per step: each Krylov solve is
one batched launch sequence over the block-diagonal system of all resident
cases.  Between steps it

* retires the cases that converged (or hit their iteration cap), freeing
  their slot and device memory, and
* admits queued requests in arrival order while the device-memory budget
  (from :func:`api.footprint_estimate`, known before the case is created) and
  the slot count allow -- requests that arrive while others run join the next
  step, so their work overlaps on the device with the cases already running.

Reported: per-request time-to-converged (finish - arrival, queueing
included), p50/p99, throughput in cases/s and Mcell-iterations/s.  A case's
arithmetic does not depend on what it shares the batch with, so each result
is the same alone and in the mix.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import api as A
from . import cases as K
from .foam import Mesh3, build_mesh3
from .meshgen import cavity_polymesh, channel_polymesh


@dataclass
class Request:
    rid: int
    kind: str          # "cavity" or "channel"
    dims: tuple        # cells per axis
    aspect: float      # box length / height
    Re: float
    arrival: float     # seconds after the start of the stream
    mesh: Mesh3 | None = None

    @property
    def n_cells(self) -> int:
        return int(np.prod(self.dims))

    def build(self) -> Mesh3:
        if self.mesh is None:
            if self.kind == "cavity":
                nx, ny = self.dims[0], self.dims[1]
                pm = cavity_polymesh(ny, nx=nx, lx=self.aspect, seed=self.rid)
            else:
                pm = channel_polymesh(*self.dims, seed=self.rid, length=self.aspect)
            self.mesh = build_mesh3(pm)
        return self.mesh

    def config(self, precision: str, max_iters: int, convergence: float):
        mesh = self.build()
        # Re = U L / nu with U = 1 (lid / peak inlet speed) and L = 1 (height)
        nu = 1.0 / self.Re
        if self.kind == "cavity":
            model, config = K.cavity_case(mesh, iterations=max_iters, precision=precision, nu=nu)
            pref = 0.0
        else:
            model, config = K.channel_case(mesh, iterations=max_iters, precision=precision, nu=nu,
                                           convergence=convergence)
            pref = None
        for s in ("U", "p"):
            config.solvers[s].convergence = convergence
        return model, config, pref


def make_requests(count: int, seed: int = 0, n_min: float = 1e3, n_max: float = 5e5, rate: float = 4.0,
                  re_range=(100.0, 2000.0), aspect_range=(1.0, 4.0)) -> list[Request]:
    """A seeded request stream: cavity or channel (50/50), N log-uniform in
    [n_min, n_max], box aspect uniform in aspect_range, Re uniform in
    re_range, Poisson arrivals at `rate` per second."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count))
    out = []
    for i in range(count):
        kind = "cavity" if rng.random() < 0.5 else "channel"
        N = float(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        aspect = float(rng.uniform(*aspect_range))
        Re = float(rng.uniform(*re_range))
        if kind == "cavity":  # 2D slab aspect x 1
            ny = max(4, int(round(np.sqrt(N / aspect))))
            nx = max(4, int(round(N / ny)))
            dims = (nx, ny, 1)
        else:                 # 3D box aspect x 1 x 1
            ny = max(4, int(round((N / aspect) ** (1.0 / 3.0))))
            nx = max(4, int(round(N / (ny * ny))))
            dims = (nx, ny, ny)
        out.append(Request(i, kind, dims, aspect, Re, float(t[i])))
    return out


@dataclass
class Result:
    rid: int
    n_cells: int
    arrival: float
    admitted: float
    finished: float
    iterations: int
    converged: bool
    residuals: np.ndarray
    U: np.ndarray | None = None
    p: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class _Done:
    """A finished result with the interface of a future."""

    def __init__(self, value):
        self.value = value

    def result(self):
        return self.value


@dataclass
class _Active:
    req: Request
    case: A.Case
    dmesh: A.DeviceMesh
    keep: object
    charge: int
    admitted: float
    iters: int = 0


@dataclass
class Server:
    ctx: A.Context
    budget_bytes: int
    max_cases: int = 64
    precision: str = "mixed"
    max_iters: int = 3000
    convergence: float = 1e-6
    keep_fields: bool = False
    timeline: list = field(default_factory=list)  # (t, active, queued, used bytes)
    phase_ms: dict = field(default_factory=dict)  # batch phase times (host wall, ms)
    admit_s: float = 0.0    # wall time spent admitting (mesh build, case set-up, batch.add)
    iterate_s: float = 0.0  # wall time spent in batch iterations
    retire_s: float = 0.0   # wall time spent retiring finished cases (batch.remove, freeing)
    idle_s: float = 0.0     # wall time waiting for arrivals with nothing to run
    cleanup_s: float = 0.0  # wall time freeing what is left at the end
    # finished cases leave the batch at once; freeing their device memory
    # (which waits for the device) is deferred until this many are pending,
    # or the run ends, so it does not stall the running batch every time
    free_every: int = 16
    # the last case of a drained stream leaves the batch and finishes alone
    # in graph mode (device-driven Krylov loops, no host round trip per
    # chunk; its iterates are the same bit for bit)
    solo_tail: bool = True
    # cases (mesh, configuration, device mesh, case, initial fields) are set
    # up on this many host threads for the first `prepare_ahead` queued
    # requests, overlapping the batch iterations (0 threads: at admission);
    # the budget check and batch.add stay on this thread
    build_threads: int = 2
    prepare_ahead: int = 4

    def _prepare(self, req: Request):
        """A request's case ready for batch.add: (footprint, case, device
        mesh, configuration kept alive); case None when it exceeds the budget."""
        mesh = req.build()
        est = A.footprint_estimate(mesh, self.precision, dilu_U=True, dilu_p=False)
        if est > self.budget_bytes:
            return est, None, None, None
        model, config, pref = req.config(self.precision, self.max_iters, self.convergence)
        cfg, keep = A.build_config(model, config, pref=pref)
        dm = A.DeviceMesh(self.ctx, mesh)
        case = A.Case(dm, cfg)
        case.set_field(A._abi.FIELD_U, model.momentum.U)
        case.set_field(A._abi.FIELD_P, model.momentum.p)
        return est, case, dm, (cfg, keep)

    def run(self, requests: list[Request], realtime: bool = True) -> list[Result]:
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        queue: deque = deque()
        active: list[_Active] = []
        results: list[Result] = []
        retired: list = []  # (case, device mesh) out of the batch, not yet freed
        pool = ThreadPoolExecutor(self.build_threads) if self.build_threads > 0 else None
        builds: dict = {}
        batch = A.Batch(self.ctx, self.max_cases, self.budget_bytes)
        used = 0
        t0 = time.perf_counter()
        try:
            while pending or queue or active:
                now = time.perf_counter() - t0
                while pending and (pending[0].arrival <= now or not realtime):
                    queue.append(pending.popleft())
                if pool is not None:
                    for req in list(queue)[: self.prepare_ahead]:
                        if req.rid not in builds:
                            builds[req.rid] = pool.submit(self._prepare, req)
                # admission, in arrival order, by device-memory footprint
                ta = time.perf_counter()
                while queue and len(active) < self.max_cases:
                    req = queue[0]
                    fut = builds.get(req.rid)
                    if fut is None:
                        fut = builds[req.rid] = _Done(self._prepare(req))
                    est, case, dm, keep = fut.result()
                    if case is None:
                        raise ValueError(f"request {req.rid} needs {est} bytes, more than the budget")
                    if used + est > self.budget_bytes or not batch.add(case, est):
                        break  # stays prepared until it fits
                    builds.pop(req.rid)
                    used += est
                    queue.popleft()
                    active.append(_Active(req, case, dm, keep, est, time.perf_counter() - t0))
                self.admit_s += time.perf_counter() - ta
                self.timeline.append((time.perf_counter() - t0, len(active), len(queue), used))
                if not active:
                    if pending and realtime:
                        tw = time.perf_counter()
                        time.sleep(max(0.0, min(0.05, pending[0].arrival - (time.perf_counter() - t0))))
                        self.idle_s += time.perf_counter() - tw
                    continue
                if self.solo_tail and len(active) == 1 and not queue and not pending:
                    a = active[0]
                    ti = time.perf_counter()
                    batch.remove(a.case)
                    a.case.set_graph_mode(True)
                    r, ok = a.case.simple_iterate(max(0, self.max_iters - a.iters))
                    self.iterate_s += time.perf_counter() - ti
                    a.iters += len(r)
                    done_t = time.perf_counter() - t0
                    U = a.case.get_field(A._abi.FIELD_U) if self.keep_fields else None
                    p = a.case.get_field(A._abi.FIELD_P) if self.keep_fields else None
                    last = r[-1].copy() if len(r) else np.zeros(4)
                    results.append(Result(a.req.rid, a.req.n_cells, a.req.arrival, a.admitted, done_t, a.iters, ok,
                                          last, U, p))
                    retired.append((a.case, a.dmesh))
                    used -= a.charge
                    active.remove(a)
                    continue
                ti = time.perf_counter()
                res, conv = batch.simple_iterate()
                self.iterate_s += time.perf_counter() - ti
                self.phase_ms = batch.timings()
                done_t = time.perf_counter() - t0
                finished = []
                for k, a in enumerate(active):
                    a.iters += 1
                    if conv[k] or a.iters >= self.max_iters:
                        finished.append((a, bool(conv[k]), res[k].copy()))
                tr = time.perf_counter()
                for a, ok, r in finished:
                    U = a.case.get_field(A._abi.FIELD_U) if self.keep_fields else None
                    p = a.case.get_field(A._abi.FIELD_P) if self.keep_fields else None
                    results.append(Result(a.req.rid, a.req.n_cells, a.req.arrival, a.admitted, done_t, a.iters, ok,
                                          r, U, p))
                    batch.remove(a.case)
                    retired.append((a.case, a.dmesh))
                    used -= a.charge
                    active.remove(a)
                if len(retired) >= self.free_every or (not active and not queue and not pending):
                    for case, dm in retired:
                        case.close()
                        dm.close()
                    retired.clear()
                self.retire_s += time.perf_counter() - tr
        finally:
            tc = time.perf_counter()
            if pool is not None:
                pool.shutdown(wait=True)
            for fut in builds.values():  # set up but never admitted
                est, case, dm, keep = fut.result()
                if case is not None:
                    case.close()
                    dm.close()
            for case, dm in retired:
                case.close()
                dm.close()
            for a in active:
                try:
                    batch.remove(a.case)
                except Exception:
                    pass
                a.case.close()
                a.dmesh.close()
            batch.close()
            self.cleanup_s += time.perf_counter() - tc
        self.wall = time.perf_counter() - t0
        return sorted(results, key=lambda r: r.rid)


def summarize(results: list[Result], wall: float) -> dict:
    lat = np.array([r.latency for r in results]) * 1e3
    cell_iters = sum(r.n_cells * r.iterations for r in results)
    return {
        "cases": len(results),
        "converged": int(sum(r.converged for r in results)),
        "wall_s": wall,
        "cases_per_s": len(results) / wall if wall > 0 else None,
        "mcell_iters_per_s": cell_iters / wall / 1e6 if wall > 0 else None,
        "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
        "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
        "mean_iterations": float(np.mean([r.iterations for r in results])) if results else None,
    }
