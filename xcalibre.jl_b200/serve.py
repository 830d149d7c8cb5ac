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

Failures stay with their request: a request larger than the budget is
rejected, one whose set-up raises is failed, and one whose residual becomes
NaN/Inf leaves the batch as diverged (the library retires it without
touching the other cases); each gets a Result with that status and the
stream goes on.  Device memory stays within the budget: a case set up ahead
of admission holds a reservation of its footprint from the moment its set-up
is submitted, and a finished case keeps its charge until its memory is
actually freed.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import api as A
from ._lib import XcalError
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
    # "converged", "max_iters" (cap reached first), "diverged" (NaN/Inf
    # residual), "rejected" (footprint above the budget), "failed" (set-up
    # raised); error: the message of the last two
    status: str = "converged"
    error: str | None = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class _Done:
    """A finished result with the interface of a future."""

    def __init__(self, value):
        self.value = value

    def result(self):
        return self.value


class _Failed:
    """A failed set-up with the interface of a future."""

    def __init__(self, exc):
        self.exc = exc

    def result(self):
        raise self.exc


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

    def footprint(self, req: Request) -> int:
        """Device bytes the request's case will hold (an upper bound, from
        the mesh sizes, before anything is allocated)."""
        return A.footprint_estimate(req.build(), self.precision, dilu_U=True, dilu_p=False)

    def _prepare(self, req: Request):
        """A request's case ready for batch.add: (case, device mesh,
        configuration kept alive).  Frees what it made if a step fails."""
        model, config, pref = req.config(self.precision, self.max_iters, self.convergence)
        cfg, keep = A.build_config(model, config, pref=pref)
        dm = A.DeviceMesh(self.ctx, req.build())
        try:
            case = A.Case(dm, cfg)
        except Exception:
            dm.close()
            raise
        try:
            case.set_field(A._abi.FIELD_U, model.momentum.U)
            case.set_field(A._abi.FIELD_P, model.momentum.p)
        except Exception:
            case.close()
            dm.close()
            raise
        return case, dm, (cfg, keep)

    @staticmethod
    def _free(case, dm):
        """Close a case and its device mesh; a failure to close one is not
        allowed to leak the other or to end the stream."""
        for h in (case, dm):
            try:
                if h is not None:
                    h.close()
            except Exception:
                pass

    def run(self, requests: list[Request], realtime: bool = True) -> list[Result]:
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        queue: deque = deque()
        active: list[_Active] = []
        results: list[Result] = []
        retired: list = []  # (case, device mesh, charge) out of the batch, not yet freed
        pool = ThreadPoolExecutor(self.build_threads) if self.build_threads > 0 else None
        builds: dict = {}   # rid -> (future of _prepare, reserved bytes)
        batch = A.Batch(self.ctx, self.max_cases, self.budget_bytes)
        # device bytes: `used` = admitted cases plus finished ones not yet
        # freed; `reserved` = cases being set up or set up ahead of admission
        used = 0
        reserved = 0
        t0 = time.perf_counter()

        def now():
            return time.perf_counter() - t0

        def fail_request(req, status, msg):
            t = now()
            results.append(Result(req.rid, req.n_cells, req.arrival, t, t, 0, False, np.full(4, np.nan),
                                  status=status, error=msg))

        def free_retired():
            nonlocal used
            for case, dm, charge in retired:
                self._free(case, dm)
                used -= charge
            retired.clear()

        def finish(a, status, r, U=None, p=None):
            nonlocal used
            results.append(Result(a.req.rid, a.req.n_cells, a.req.arrival, a.admitted, now(), a.iters,
                                  status == "converged", r, U, p, status=status))
            retired.append((a.case, a.dmesh, a.charge))
            active.remove(a)

        try:
            while pending or queue or active:
                while pending and (pending[0].arrival <= now() or not realtime):
                    queue.append(pending.popleft())
                # set-up ahead of admission, each under a reservation of its
                # footprint, never past the budget
                if pool is not None:
                    for req in list(queue)[: self.prepare_ahead]:
                        if req.rid in builds:
                            continue
                        est = self.footprint(req)
                        if est > self.budget_bytes:
                            continue  # rejected at admission
                        if used + reserved + est > self.budget_bytes:
                            break
                        reserved += est
                        builds[req.rid] = (pool.submit(self._prepare, req), est)
                # admission, in arrival order, by device-memory footprint;
                # a request not set up ahead is reserved and set up here
                ta = time.perf_counter()
                while queue and len(active) < self.max_cases:
                    req = queue[0]
                    if req.rid not in builds:
                        est = self.footprint(req)
                        if est > self.budget_bytes:
                            queue.popleft()
                            fail_request(req, "rejected",
                                         f"needs {est} bytes, more than the budget {self.budget_bytes}")
                            continue
                        if used + reserved + est > self.budget_bytes:
                            if retired:
                                free_retired()
                                continue
                            break
                        reserved += est
                        try:
                            builds[req.rid] = (_Done(self._prepare(req)), est)
                        except Exception as e:
                            builds[req.rid] = (_Failed(e), est)
                    fut, est = builds[req.rid]
                    try:
                        case, dm, keep = fut.result()
                    except Exception as e:  # this request's set-up failed; the stream goes on
                        builds.pop(req.rid)
                        reserved -= est
                        queue.popleft()
                        fail_request(req, "failed", f"{type(e).__name__}: {e}")
                        continue
                    if not batch.add(case, est):
                        break  # stays set up, under its reservation, until it fits
                    builds.pop(req.rid)
                    reserved -= est
                    used += est
                    queue.popleft()
                    active.append(_Active(req, case, dm, keep, est, now()))
                self.admit_s += time.perf_counter() - ta
                self.timeline.append((now(), len(active), len(queue), used))
                if not active:
                    if pending and realtime:
                        tw = time.perf_counter()
                        time.sleep(max(0.0, min(0.05, pending[0].arrival - now())))
                        self.idle_s += time.perf_counter() - tw
                    elif queue and retired:
                        free_retired()
                    continue
                if self.solo_tail and len(active) == 1 and not queue and not pending:
                    a = active[0]
                    ti = time.perf_counter()
                    batch.remove(a.case)
                    a.case.set_graph_mode(True)
                    try:
                        r, ok = a.case.simple_iterate(max(0, self.max_iters - a.iters))
                    except XcalError as e:
                        if e.code != A._abi.XCAL_ERR_DIVERGED:
                            raise
                        self.iterate_s += time.perf_counter() - ti
                        finish(a, "diverged", np.full(4, np.nan))
                        results[-1].error = str(e)
                        continue
                    self.iterate_s += time.perf_counter() - ti
                    a.iters += len(r)
                    U = a.case.get_field(A._abi.FIELD_U) if self.keep_fields else None
                    p = a.case.get_field(A._abi.FIELD_P) if self.keep_fields else None
                    last = r[-1].copy() if len(r) else np.zeros(4)
                    finish(a, "converged" if ok else "max_iters", last, U, p)
                    continue
                ti = time.perf_counter()
                members = list(batch.cases)
                res, conv = batch.simple_iterate()
                self.iterate_s += time.perf_counter() - ti
                self.phase_ms = batch.timings()
                tr = time.perf_counter()
                by_case = {id(a.case): a for a in active}
                for k, c in enumerate(members):
                    a = by_case[id(c)]
                    a.iters += 1
                    if c in batch.last_diverged:  # already out of the batch
                        finish(a, "diverged", res[k].copy())
                        results[-1].error = "residual became NaN/Inf"
                    elif conv[k] or a.iters >= self.max_iters:
                        U = a.case.get_field(A._abi.FIELD_U) if self.keep_fields else None
                        p = a.case.get_field(A._abi.FIELD_P) if self.keep_fields else None
                        batch.remove(a.case)
                        finish(a, "converged" if conv[k] else "max_iters", res[k].copy(), U, p)
                if len(retired) >= self.free_every or (not active and not queue and not pending):
                    free_retired()
                self.retire_s += time.perf_counter() - tr
        finally:
            tc = time.perf_counter()
            if pool is not None:
                pool.shutdown(wait=True)
            for fut, _ in builds.values():  # set up but never admitted
                try:
                    case, dm, keep = fut.result()
                except Exception:
                    continue
                self._free(case, dm)
            free_retired()
            for a in active:
                try:
                    batch.remove(a.case)
                except Exception:
                    pass
                self._free(a.case, a.dmesh)
            try:
                batch.close()
            except Exception:
                pass
            self.cleanup_s += time.perf_counter() - tc
        self.wall = time.perf_counter() - t0
        return sorted(results, key=lambda r: r.rid)


def shard_requests(requests: list[Request], rank: int, world: int) -> list[Request]:
    """The requests one of `world` servers takes (one process per GPU, each
    with its own Server): request i goes to rank i mod world, arrival times
    unchanged, so every rank sees the same stream rate divided by world."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    return [r for r in requests if r.rid % world == rank]


def result_record(r: Result) -> tuple:
    """A Result without its field arrays, for gathering across ranks."""
    return (r.rid, r.n_cells, r.arrival, r.admitted, r.finished, r.iterations, bool(r.converged), r.status,
            r.error)


def merge_records(parts: list[list[tuple]]) -> list[Result]:
    """Every rank's result records as Results, in request order; each request
    must appear exactly once."""
    out = [Result(rid=t[0], n_cells=t[1], arrival=t[2], admitted=t[3], finished=t[4], iterations=t[5],
                  converged=t[6], residuals=np.zeros(0), status=t[7], error=t[8]) for part in parts for t in part]
    out.sort(key=lambda r: r.rid)
    rids = [r.rid for r in out]
    if len(set(rids)) != len(rids):
        raise ValueError("a request was served by more than one rank")
    return out


def summarize(results: list[Result], wall: float) -> dict:
    """Throughput and time-to-result over the solved requests (rejected and
    failed ones are counted, not timed)."""
    solved = [r for r in results if r.status in ("converged", "max_iters", "diverged")]
    lat = np.array([r.latency for r in solved]) * 1e3
    cell_iters = sum(r.n_cells * r.iterations for r in solved)
    return {
        "cases": len(results),
        "converged": int(sum(r.converged for r in results)),
        "status_counts": {st: sum(r.status == st for r in results)
                          for st in ("converged", "max_iters", "diverged", "rejected", "failed")},
        "wall_s": wall,
        "cases_per_s": len(results) / wall if wall > 0 else None,
        "mcell_iters_per_s": cell_iters / wall / 1e6 if wall > 0 else None,
        "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
        "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
        "mean_iterations": float(np.mean([r.iterations for r in solved])) if solved else None,
    }
