#!/usr/bin/env python
"""Headline benchmark: SIMPLE outer iterations of the 128^3 (2,097,152-cell)
steady laminar channel with randomly permuted cell/face numbering, FP64,
through libxcal_b200 on one B200 per process.

A "step" is one SIMPLE outer iteration of the whole case (momentum
assembly + 3 BiCGSTAB/DILU solves, pressure assembly + CG/Jacobi solve,
gradients, flux and velocity corrections).  Metric: Mcell-iters/s =
cells x iterations / device seconds.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--size 128] [--precision fp64|mixed] [--no-second-precision]

The line's `value` is the FP64 plain path (or --precision's mode);
`second_precision` carries the same measurement in the other mode (mixed:
FP32 Krylov inner solves inside FP64 defect correction).

--impl reference times the CPU restatement of the reference's path (the
oracle; the Julia reference cannot run in this image) on the host cores.
Multi-GPU: replicas only (independent cases, no collective in the path);
rank 0 prints the line, `value` is the sum over ranks / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-iters/s (FP64 vs mixed, resid 1e-6) at 2M cells; serve p50/p99 ms"
UNIT = "Mcell-iters/s"
L2_NOTE = "working set (matrices + face arrays, >1 GB) larger than the GPU's L2; no flush between steps"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-iters", type=int, default=1, help="SIMPLE iterations in the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-second-precision", action="store_true",
                    help="skip the second timed run in the other precision mode")
    ap.add_argument("--les-size", type=int, default=96, help="periodic LES box: cells per side (0 = skip)")
    ap.add_argument("--les-steps", type=int, default=200)
    ap.add_argument("--serve-cases", type=int, default=16, help="serving stream: requests (0 = skip)")
    ap.add_argument("--serve-nmax", type=float, default=3e4)
    ap.add_argument("--serve-rate", type=float, default=8.0)
    ap.add_argument("--serve-iters", type=int, default=1500, help="serving: SIMPLE iteration cap per request")
    ap.add_argument("--serve-budget-gb", type=float, default=40.0, help="serving: device-memory budget (GB)")
    ap.add_argument("--serve-max-cases", type=int, default=64, help="serving: most requests resident at once")
    ap.add_argument("--converge-cap", type=int, default=1200,
                    help="time-to-convergence block: SIMPLE iteration cap per precision (0 = skip)")
    ap.add_argument("--only", choices=["les", "serving", "batch", "converge", "step-window", "les-window"],
                    default=None,
                    help="run one secondary workload alone and print its block as the line (profiling); "
                         "step-window: --steps SIMPLE iterations of the channel case after --warmup, between "
                         "cudaProfilerStart/Stop (for ncu --profile-from-start off); les-window: the same for "
                         "--steps host-polled PISO steps of the --les-size LES box")
    ap.add_argument("--inner-cg", type=int, default=None,
                    help="mixed precision: form of the FP32 inner CG (xcal_case_set_inner_cg; default: the "
                         "library's)")
    ap.add_argument("--ncu-table", default=None, metavar="CSV",
                    help="print the per-kernel table (launches, time, share, DRAM bytes) of an ncu --csv "
                         "per-launch metrics file and exit (no GPU)")
    return ap.parse_args()


def ncu_table(path):
    """Per-kernel sums of an ncu --csv log of gpu__time_duration.sum and
    dram__bytes_read/write.sum, one line per kernel, by total time."""
    import collections
    import csv
    import re
    rows = list(csv.reader(ln for ln in open(path) if not ln.startswith("==")))
    ix = {h: i for i, h in enumerate(rows[0])}
    scale = {"ns": 1e-9, "nsecond": 1e-9, "us": 1e-6, "usecond": 1e-6, "ms": 1e-3, "msecond": 1e-3,
             "second": 1.0, "byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}
    agg = collections.OrderedDict()
    for r in rows[1:]:
        if len(r) < len(ix):
            continue
        name = re.sub(r"\(.*", "", r[ix["Kernel Name"]]).replace("void ", "").replace("xcal::", "")
        a = agg.setdefault(name, {"ids": set(), "t": 0.0, "rd": 0.0, "wr": 0.0})
        a["ids"].add(r[ix["ID"]])
        v = float(r[ix["Metric Value"]].replace(",", "")) * scale.get(r[ix["Metric Unit"]], 1.0)
        key = {"gpu__time_duration.sum": "t", "dram__bytes_read.sum": "rd", "dram__bytes_write.sum": "wr"}
        if r[ix["Metric Name"]] in key:
            a[key[r[ix["Metric Name"]]]] += v
    tot = sum(a["t"] for a in agg.values())
    print(f"{'kernel':44s} {'launches':>8s} {'time ms':>9s} {'share':>6s} {'DRAM MB/launch':>14s} {'DRAM GB/s':>9s}")
    for name, a in sorted(agg.items(), key=lambda kv: -kv[1]["t"]):
        k = len(a["ids"])
        gbs = (a["rd"] + a["wr"]) / a["t"] / 1e9 if a["t"] else 0.0
        print(f"{name[:44]:44s} {k:8d} {a['t'] * 1e3:9.3f} {a['t'] / tot:6.1%} {(a['rd'] + a['wr']) / k / 1e6:14.2f} "
              f"{gbs:9.0f}")
    print(f"total device time {tot * 1e3:.3f} ms over {sum(len(a['ids']) for a in agg.values())} launches")
    return 0


def workload_name(n):
    return f"channel {4}x1x1 box, {n}^3 hex = {n ** 3} cells, permuted numbering (seed 0), FP64 SIMPLE"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            import tempfile
            fd, self.path = tempfile.mkstemp(prefix=f"xcal_clocks_gpu{self.gpu}_", suffix=".csv")
            self.f = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for ln in f:
                p = [s.strip() for s in ln.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        try:
            os.unlink(self.path)
        except OSError:
            pass
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def max_over_ranks(v: float, world: int, device=None) -> float:
    """The largest of the ranks' values (every rank takes part; 1 rank: v)."""
    if world <= 1:
        return v
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_throughput(cells_per_rank: int, world: int, steps: int, seconds: float) -> float:
    """Whole-job Mcell-iters/s of `world` replicas, each advancing its own
    `cells_per_rank`-cell case `steps` iterations, timed by the slowest rank."""
    return cells_per_rank * world * steps / seconds / 1e6


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args):
    """CPU restatement of the reference's path (the oracle), all host threads."""
    world, rank, local = dist_setup(args)
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    import __graft_entry__ as ge
    x = ge.load_package()
    n = args.size
    pm = x.channel_polymesh(n, n, n, seed=0)
    om = orc.OracleMesh.from_polymesh(pm)
    e = om.export()
    mesh = x.Mesh3(patch_names=list(pm.patch_names), **e)
    model, config = x.cases.channel_case(mesh, iterations=args.steps + args.warmup)
    cfg, keep = x.build_config(model, config)
    oc = orc.OracleCase(om, cfg)
    cores = orc.threads()
    # W untimed warm-up iterations (at most 3: the CPU path has no JIT or
    # caches to warm, more would only lengthen the run), then K timed ones
    W = min(args.warmup, 3)
    oc.simple_iterate(W)
    t0 = time.perf_counter()
    res, _ = oc.simple_iterate(args.steps)
    dt = time.perf_counter() - t0
    value = mesh.n_cells * args.steps / dt / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": W, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(n), "cells": mesh.n_cells, "precision": "fp64", "l2": L2_NOTE},
            "implementation": "CPU restatement of XCALibre.jl's path (C++/OpenMP oracle)",
            "parallelism": f"{cores} host threads",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"SIMPLE iterations {W + 1}..{W + args.steps} of the full case"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_sample(x, pm, mesh, iters):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    om = orc.OracleMesh.from_mesh3(mesh)
    model, config = x.cases.channel_case(mesh, iterations=iters + 1)
    cfg, keep = x.build_config(model, config)
    oc = orc.OracleCase(om, cfg)
    # as the reference arm (--impl reference): one untimed iteration from
    # rest, then the timed ones
    oc.simple_iterate(1)
    t0 = time.perf_counter()
    oc.simple_iterate(iters)
    dt = time.perf_counter() - t0
    return {"value": mesh.n_cells * iters / dt / 1e6, "unit": UNIT, "cores": orc.threads(), "kind": "port",
            "sample": f"SIMPLE iterations 2..{iters + 1} of the same {mesh.n_cells}-cell case (iteration 1 from "
                      f"U=0, p=0 untimed; {dt:.1f} s wall, C++ oracle with OpenMP over all host threads)"}


def spmv_bytes(nnz, n, fp32):
    """Algorithmic bytes of one CG SpMV launch (k >= 1): matrix slots (value +
    column index) once, row length (1 byte) and slice offsets (4 bytes per 32
    rows), z and p_{k-1} read once, p_k and q written once."""
    s = 4 if fp32 else 8
    return nnz * (s + 4) + n * (1 + 4 * s) + 4 * ((n + 31) // 32)


def measure(x, A, mesh, precision, args, local, world, stream_cls):
    """Warm up, then time args.steps SIMPLE iterations of a fresh case on the
    device (CUDA events on the case stream, barrier + synchronize around)."""
    import torch
    model, config = x.cases.channel_case(mesh, iterations=args.steps + args.warmup, precision=precision,
                                         device=local)
    cfg, keep = x.build_config(model, config)
    ctx = x.Context(local)
    t_setup = time.perf_counter()
    dm = x.DeviceMesh(ctx, mesh)
    case = x.Case(dm, cfg)
    if args.inner_cg is not None and precision == "mixed":
        case.set_inner_cg(args.inner_cg)
    case.set_field(A.FIELD_U, model.momentum.U)
    case.set_field(A.FIELD_P, model.momentum.p)
    t_setup = time.perf_counter() - t_setup
    nnz_p = case.nnz(A.EQN_P)
    stream = stream_cls(case.stream(), device=torch.device("cuda", local))
    case.simple_iterate(args.warmup)
    torch.cuda.synchronize()
    case.set_profiling(True)
    prof0 = [case.profile(k) for k in range(6)]
    l0 = x.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    res, _ = case.simple_iterate(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    launches = x.launch_count() - l0
    prof1 = [case.profile(k) for k in range(6)]
    case.set_profiling(False)
    ms = max_over_ranks(ms, world, "cuda")
    fp32 = precision == "mixed"
    n = mesh.n_cells
    # roofline of the dominant kernel: the CG SpMV fused with p = z + beta p
    # and <p, Ap> (pressure solve), timed by CUDA events on sampled launches
    spmv_ms = prof1[0][0] - prof0[0][0]
    spmv_n = prof1[0][1] - prof0[0][1]
    spmv_all = prof1[4][1] - prof0[4][1]  # every CG SpMV launch that did work
    bytes_spmv = spmv_bytes(nnz_p, n, fp32)
    peak, peak_kind = measured_peak_hbm()
    avg_s = spmv_ms / max(spmv_n, 1) / 1e3
    achieved = bytes_spmv / avg_s / 1e9 if spmv_n else None
    traffic = None
    tr_all = {}
    tp = os.path.join(ROOT, "profiles", "spmv_traffic.json")
    if os.path.exists(tp):
        try:
            tr_all = json.load(open(tp))
        except Exception:
            tr_all = {}
    if os.path.exists(tp):
        try:
            tr = json.load(open(tp))
            key = "bytes_per_launch_128_fp32" if fp32 else "bytes_per_launch_128"
            traffic = tr.get(key) if args.size == 128 else None
        except Exception:
            traffic = None
    prec_name = "FP32" if fp32 else "FP64"
    roof = {"bound": "hbm", "kernel": f"k_cg_spmv<{prec_name}> (SELL-32 SpMV fused with p = z + beta p and <p,Ap>)",
            "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "traffic": traffic, "bytes_per_launch": bytes_spmv,
            "launches_timed": spmv_n, "launches_total": spmv_all, "avg_launch_us": avg_s * 1e6,
            "share_of_step": avg_s * 1e3 * spmv_all / ms if ms else None}
    # persistent CG: one cooperative launch per solve runs every iteration
    # (SpMV phase + update phase, q on chip); per iteration it moves the
    # matrix slots, row lengths and slice offsets, gathers z and p_{k-1},
    # writes p_k, then reads x, r, P, p_k and writes x, r, z
    pers_ms = prof1[5][0] - prof0[5][0]
    pers_it = prof1[5][1] - prof0[5][1]
    if pers_it and fp32:
        # folded FP32 CG (Jacobi-scaled system, implicit unit diagonal): per
        # iteration the off-diagonal slots (value + column) and row lengths
        # stream once, the (r, p_{k-1}) pairs are gathered (8 B per row), and
        # phase 2 reads the row's pair and writes the next (r, p_k) pair (x
        # and q stay in shared memory)
        nnz_off = nnz_p - n
        bpi = nnz_off * 8 + n * (1 + 8 + 8 + 8)
        t_it = pers_ms / pers_it / 1e3
        ach = bpi / t_it / 1e9
        roof = {"bound": "hbm", "kernel": "k_cgf_persist (FP32 CG on the Jacobi-scaled system, whole solve in one "
                                          "cooperative launch, one block per SM: gathered SpMV of the off-diagonal "
                                          "slots with p = r + beta p from (r, p) pairs, grid barrier, x/r update, "
                                          "grid barrier)",
                "achieved": ach, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": ach / peak,
                "traffic": (tr_all.get("fold_bytes_per_iteration_128") if args.size == 128 else None),
                "traffic_unit": "bytes per CG iteration (ncu DRAM read + write of one launch / its iterations)",
                "bytes_per_iteration": bpi, "iterations": pers_it, "us_per_iteration": t_it * 1e6,
                "share_of_step": pers_ms / ms if ms else None}
    elif pers_it:
        s_ = 4 if fp32 else 8
        bpi = nnz_p * (s_ + 4) + n * (1 + 10 * s_) + 4 * ((n + 31) // 32)
        t_it = pers_ms / pers_it / 1e3
        ach = bpi / t_it / 1e9
        roof = {"bound": "hbm", "kernel": f"k_cg_persist<{'FP32' if fp32 else 'FP64'}> (whole CG solve in one "
                                          "cooperative launch: SELL-32 SpMV with p = z + beta p and <p,Ap>, grid "
                                          "barrier, x/r/z update with <r,z>, grid barrier)",
                "achieved": ach, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": ach / peak,
                "traffic": (tr_all.get("persist_bytes_per_iteration_128")
                            if (not fp32 and args.size == 128) else None),
                "traffic_unit": "bytes per CG iteration (ncu DRAM read + write of one launch / its iterations)",
                "bytes_per_iteration": bpi, "iterations": pers_it,
                "us_per_iteration": t_it * 1e6,
                "share_of_step": pers_ms / ms if ms else None}
    # second kernel of each CG iteration: x += alpha p; r -= alpha q; z = P r;
    # <r,z> -- reads x, p, r, q, P and writes x, r, z (8 vectors)
    upd_ms = prof1[3][0] - prof0[3][0]
    upd_n = prof1[3][1] - prof0[3][1]
    if upd_n and not pers_it:
        upd_s = upd_ms / upd_n / 1e3
        ub = 8 * (4 if fp32 else 8) * n
        roof["cg_update"] = {"avg_launch_us": upd_s * 1e6, "bytes_per_launch": ub, "achieved": ub / upd_s / 1e9,
                             "launches_timed": upd_n, "share_of_step": upd_s * 1e3 * spmv_all / ms if ms else None}
    tm = case.timings()
    out = {"value": job_throughput(n, world, args.steps, ms / 1e3), "ms_per_step": ms / args.steps, "roofline": roof,
           "gpu_launches": launches, "clocks": clk, "setup_s": round(t_setup, 2), "nnz_p": nnz_p,
           "residuals_last": [float(v) for v in res[-1]] if len(res) else None,
           "phases_ms_total": {"U_solve": tm[1], "p_solve": tm[2], "other": tm[3], "total": tm[5]}}
    return out, case, dm, model


def les_measure(x, A, args, local):
    """Transient LES (PISO + Smagorinsky Cs = 0.17) on the periodic 2*pi cube:
    seeded divergence-free Fourier initial field (k^4 exp(-2 (k/4)^2), rms 1),
    nu = 1e-4, dt from CFL 0.5, 2 correctors; mixed precision; every time step
    one CUDA graph (device-driven Krylov loops).  Steps timed with CUDA
    events on the case stream after 3 warm-up steps."""
    import torch
    n = args.les_size
    mesh = x.build_mesh3(x.periodic_box_polymesh(n, seed=0), device=local)
    U0 = x.cases.fourier_field(mesh, seed=0)
    out = {"workload": f"periodic LES box 2pi^3, {n}^3 hex = {mesh.n_cells} cells, PISO x2 correctors, "
                       f"Smagorinsky 0.17, nu 1e-4, CFL 0.5, mixed precision, graph per step"}
    model, config = x.cases.periodic_les_case(mesh, steps=args.les_steps, U0=U0, precision="mixed", device=local)
    cfg, keep = x.build_config(model, config, pref=0.0)
    ctx = x.Context(local)
    dm = x.DeviceMesh(ctx, mesh)
    case = x.Case(dm, cfg)
    case.set_field(A.FIELD_U, model.momentum.U)
    case.set_field(A.FIELD_P, model.momentum.p)
    case.set_graph_mode(True)
    stream = torch.cuda.ExternalStream(case.stream(), device=torch.device("cuda", local))
    case.piso_step(3)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    l0 = x.launch_count()
    e0.record(stream)
    res, co = case.piso_step(args.les_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out.update({"value": mesh.n_cells * args.les_steps / (ms / 1e3) / 1e6, "unit": UNIT,
                "ms_per_step": ms / args.les_steps, "steps": args.les_steps, "dt": config.runtime.time_step,
                "courant_last": float(co[-1]), "residuals_last": [float(v) for v in res[-1]],
                "gpu_launches": x.launch_count() - l0})
    case.close()
    dm.close()
    return out


def serve_measure(x, args, local):
    """Serving stream: steady cavity/channel requests (50/50), N log-uniform
    in [1e3, serve_nmax], aspect U[1,4], Re U[100,2000], Poisson arrivals at
    serve_rate per second, mixed precision, each to a 1e-6 scaled residual
    (cap 1500 SIMPLE iterations); continuous batching with admission by
    device-memory footprint (serve_budget_gb).  Meshes are built before the
    stream starts (they are the requests' payload).  serve_iters caps each
    request's SIMPLE iterations.  With several ranks (one process per GPU)
    the stream is sharded: rank r serves requests r, r + N, ... with its own
    Server, the ranks start together, and the line reports every request
    (throughput over the slowest rank's wall time, p50/p99 over all)."""
    from importlib import import_module
    serve = import_module(x.__name__ + ".serve")
    world, rank = (torch_world() if args.gpus > 1 else (1, 0))
    reqs = serve.make_requests(args.serve_cases, seed=0, n_min=1e3, n_max=args.serve_nmax, rate=args.serve_rate)
    mine = serve.shard_requests(reqs, rank, world)
    for r in mine:
        r.build()
    ctx = x.Context(local)
    budget = int(args.serve_budget_gb * (1 << 30))
    srv = serve.Server(ctx, budget_bytes=budget, max_cases=args.serve_max_cases, precision="mixed",
                       max_iters=args.serve_iters,
                       convergence=1e-6)
    l0 = x.launch_count()
    if world > 1:
        import torch
        torch.distributed.barrier()
    res = srv.run(mine, realtime=True)
    wall = srv.wall
    if world > 1:
        res, wall = gather_served(res, wall, world, serve)
    s = serve.summarize(res, wall)
    s["sharding"] = f"{world} ranks, request i on rank i mod {world}" if world > 1 else "1 GPU"
    s.update({"workload": f"{len(reqs)} steady cavity/channel requests, N log-uniform [1e3, {args.serve_nmax:g}], "
                          f"Re U[100,2000], aspect U[1,4], Poisson {args.serve_rate:g}/s, mixed, resid 1e-6, "
                          f"cap {args.serve_iters} iterations",
              "rate_per_s": args.serve_rate, "budget_bytes": budget, "max_cases": args.serve_max_cases,
              "converged_ge_1e5_cells": "%d/%d" % (sum(r.converged for r in res if r.n_cells >= 1e5),
                                                    sum(1 for r in res if r.n_cells >= 1e5)),
              "max_active": max((t[1] for t in srv.timeline), default=0),
              "admission_s": srv.admit_s, "iterate_s": srv.iterate_s, "retire_s": srv.retire_s,
              "idle_s": srv.idle_s, "cleanup_s": srv.cleanup_s,
              "gpu_launches": x.launch_count() - l0})
    return s


def torch_world():
    """(world size, rank) of the running process group, or (1, 0)."""
    import torch
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        return torch.distributed.get_world_size(), torch.distributed.get_rank()
    return 1, 0


def gather_served(results, wall, world, serve):
    """Every rank's served requests (records without field arrays) and the
    slowest rank's wall time, on every rank."""
    import torch
    parts = [None] * world
    torch.distributed.all_gather_object(parts, ([serve.result_record(r) for r in results], wall))
    return serve.merge_records([p[0] for p in parts]), max(p[1] for p in parts)


def batch_measure(x, args, local):
    """Batching: the serving sample's requests (same seed and sizes) resident
    as one fixed batch, mixed precision; W warm-up batch iterations, then K
    timed ones (each one SIMPLE iteration of every case: batched Krylov
    solves over all cases, per-case face loops on the cases' own streams).
    Host wall time around xcal_batch_simple_iterate, which ends in a device
    synchronisation (it returns the residuals)."""
    from importlib import import_module
    serve = import_module(x.__name__ + ".serve")
    reqs = serve.make_requests(args.serve_cases, seed=0, n_min=1e3, n_max=args.serve_nmax, rate=args.serve_rate)
    ctx = x.Context(local)
    batch = x.api.Batch(ctx, max(64, len(reqs)), 40 << 30)
    keep = []
    for r in reqs:
        model, config, pref = r.config("mixed", 1500, 1e-6)
        cfg, k = x.build_config(model, config, pref=pref)
        dm = x.DeviceMesh(ctx, r.build())
        c = x.Case(dm, cfg)
        c.set_field(x._abi.FIELD_U, model.momentum.U)
        c.set_field(x._abi.FIELD_P, model.momentum.p)
        if not batch.add(c):
            raise RuntimeError("batch admission refused")
        keep.append((c, dm, k))
    for _ in range(args.warmup):
        batch.simple_iterate()
    p0 = batch.timings()
    l0 = x.launch_count()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        batch.simple_iterate()
    dt = time.perf_counter() - t0
    p1 = batch.timings()
    launches = x.launch_count() - l0
    cells = sum(r.n_cells for r in reqs)
    out = {"workload": f"{len(reqs)} steady cavity/channel cases (the serving sample's requests) as one batch, "
                       f"mixed", "cases": len(reqs), "cells": cells, "steps": args.steps, "warmup": args.warmup,
           "value": cells * args.steps / dt / 1e6, "unit": UNIT, "ms_per_iter": dt / args.steps * 1e3,
           "phase_ms_per_iter": {k: (p1[k] - p0[k]) / args.steps for k in p1},
           "gpu_launches_per_iter": launches / args.steps}
    batch.close()
    for c, dm, _ in keep:
        c.close()
        dm.close()
    return out


def converge_measure(x, A, mesh, args, local):
    """Time to the 1e-6 scaled residual: the same case from rest in FP64 and
    in mixed precision, each run until the SIMPLE convergence test passes
    (Solvers_1_SIMPLE.jl:222-240) or the cap; CUDA events on the case
    stream; then U and p of the two end states compared (relative L2)."""
    import torch
    out = {"workload": workload_name(args.size).replace(", FP64 SIMPLE", "") + ", SIMPLE from rest to 1e-6",
           "cap": args.converge_cap}
    ends = {}
    for prec in ("fp64", "mixed"):
        model, config = x.cases.channel_case(mesh, iterations=args.converge_cap, precision=prec, device=local)
        cfg, keep = x.build_config(model, config)
        ctx = x.Context(local)
        dm = x.DeviceMesh(ctx, mesh)
        case = x.Case(dm, cfg)
        if args.inner_cg is not None and prec == "mixed":
            case.set_inner_cg(args.inner_cg)
        case.set_field(A.FIELD_U, model.momentum.U)
        case.set_field(A.FIELD_P, model.momentum.p)
        stream = torch.cuda.ExternalStream(case.stream(), device=torch.device("cuda", local))
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res, conv = case.simple_iterate(args.converge_cap)
        e1.record(stream)
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        ends[prec] = (case.get_field(A.FIELD_U), case.get_field(A.FIELD_P))
        out[prec] = {"iterations": len(res), "converged": bool(conv), "seconds": sec,
                     "value": mesh.n_cells * len(res) / sec / 1e6, "unit": UNIT,
                     "residuals_last": [float(v) for v in res[-1]]}
        case.close()
        dm.close()
    out["time_ratio_fp64_over_mixed"] = out["fp64"]["seconds"] / out["mixed"]["seconds"]
    (U64, p64), (U32, p32) = ends["fp64"], ends["mixed"]
    out["mixed_vs_fp64_rel_l2"] = {"U": float(np.linalg.norm(U32 - U64) / np.linalg.norm(U64)),
                                   "p": float(np.linalg.norm(p32 - p64) / np.linalg.norm(p64))}
    return out


def step_window(x, A, args, local):
    """--warmup SIMPLE iterations of the --size channel case in --precision,
    then --steps more between cudaProfilerStart/Stop, so that an ncu capture
    with --profile-from-start off sees exactly those steps' launches."""
    import torch
    n = args.size
    mesh = x.build_mesh3(x.channel_polymesh(n, n, n, seed=0), device=local)
    model, config = x.cases.channel_case(mesh, iterations=100, precision=args.precision)
    cfg, keep = x.build_config(model, config)
    ctx = x.Context(local)
    dm = x.DeviceMesh(ctx, mesh)
    case = x.Case(dm, cfg)
    if args.inner_cg is not None and args.precision == "mixed":
        case.set_inner_cg(args.inner_cg)
    case.set_field(A.FIELD_U, model.momentum.U)
    case.set_field(A.FIELD_P, model.momentum.p)
    case.simple_iterate(args.warmup)
    torch.cuda.synchronize()
    l0 = x.launch_count()
    torch.cuda.profiler.start()
    res, _ = case.simple_iterate(args.steps)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    rep = case.solve_report()
    out = {"workload": workload_name(n), "precision": args.precision, "warmup": args.warmup, "steps": args.steps,
           "launches": x.launch_count() - l0, "residuals_last": [float(v) for v in res[-1]],
           "krylov_iterations_last": [int(v) for v in rep["iterations"]]}
    case.close()
    dm.close()
    return out


def les_window(x, A, args, local):
    """--warmup PISO steps of the --les-size LES box (the les block's case),
    then --steps more between cudaProfilerStart/Stop.  Host-polled, not graph
    mode: ncu profiles no kernel node of a graph with conditional nodes (the
    graph's device-driven Krylov loops); the kernels are the same."""
    import torch
    n = args.les_size
    mesh = x.build_mesh3(x.periodic_box_polymesh(n, seed=0), device=local)
    U0 = x.cases.fourier_field(mesh, seed=0)
    model, config = x.cases.periodic_les_case(mesh, steps=args.steps, U0=U0, precision="mixed", device=local)
    cfg, keep = x.build_config(model, config, pref=0.0)
    ctx = x.Context(local)
    dm = x.DeviceMesh(ctx, mesh)
    case = x.Case(dm, cfg)
    case.set_field(A.FIELD_U, model.momentum.U)
    case.set_field(A.FIELD_P, model.momentum.p)
    case.piso_step(args.warmup)
    torch.cuda.synchronize()
    l0 = x.launch_count()
    torch.cuda.profiler.start()
    res, _ = case.piso_step(args.steps)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    out = {"workload": f"periodic LES box {n}^3 = {mesh.n_cells} cells, mixed, host-polled",
           "warmup": args.warmup, "steps": args.steps, "launches": x.launch_count() - l0,
           "residuals_last": [float(v) for v in res[-1]]}
    case.close()
    dm.close()
    return out


def e2e_measure(x, A, case, mesh, args, world):
    """Same metric through the public API with host buffers: every step copies
    U and p host->device, runs one SIMPLE iteration and reads them back."""
    import torch
    nC = mesh.n_cells
    hU = torch.empty((3, nC), dtype=torch.float64, pin_memory=True).numpy()
    hp = torch.empty(nC, dtype=torch.float64, pin_memory=True).numpy()
    hU[:] = case.get_field(A.FIELD_U)
    hp[:] = case.get_field(A.FIELD_P)
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        case.set_field(A.FIELD_U, hU)
        case.set_field(A.FIELD_P, hp)
        r, _ = case.simple_iterate(1)
        case.get_field(A.FIELD_U, out=hU)
        case.get_field(A.FIELD_P, out=hp)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, "cuda")
    return {"value": job_throughput(nC, world, args.e2e_steps, e2e_s), "unit": UNIT,
            "h2d_bytes_per_step": 4 * nC * 8, "d2h_bytes_per_step": 4 * nC * 8 + 4 * 8, "steps": args.e2e_steps}


def main():
    args = parse()
    if args.ncu_table:
        return ncu_table(args.ncu_table)
    if args.impl == "reference":
        return run_reference(args)
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local))
    import __graft_entry__ as ge
    x = ge.load_package()
    A = x._abi
    if args.only is not None:
        def conv_only():
            m = x.build_mesh3(x.channel_polymesh(args.size, args.size, args.size, seed=0), device=local)
            return converge_measure(x, A, m, args, local)
        blk = {"les": lambda: les_measure(x, A, args, local), "serving": lambda: serve_measure(x, args, local),
               "batch": lambda: batch_measure(x, args, local), "converge": conv_only,
               "step-window": lambda: step_window(x, A, args, local),
               "les-window": lambda: les_window(x, A, args, local)}[args.only]()
        if rank == 0:
            print(json.dumps({"only": args.only, **blk}), flush=True)
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0
    n = args.size
    t_mesh = time.perf_counter()
    pm = x.channel_polymesh(n, n, n, seed=0)
    mesh = x.build_mesh3(pm, device=local)  # geometry on the GPU (identical to the host build)
    t_mesh = time.perf_counter() - t_mesh
    primary = args.precision
    r, case, dm, model = measure(x, A, mesh, primary, args, local, world, torch.cuda.ExternalStream)
    e2e = e2e_measure(x, A, case, mesh, args, world) if args.e2e_steps > 0 else None
    case.close()
    dm.close()
    other = None
    if not args.no_second_precision:
        sec = "mixed" if primary == "fp64" else "fp64"
        r2, case2, dm2, _ = measure(x, A, mesh, sec, args, local, world, torch.cuda.ExternalStream)
        case2.close()
        dm2.close()
        other = {"precision": sec, "value": r2["value"], "ms_per_step": r2["ms_per_step"],
                 "ratio_mixed_over_fp64": (r2["value"] / r["value"]) if sec == "mixed" else (r["value"] / r2["value"]),
                 "roofline": r2["roofline"], "residuals_last": r2["residuals_last"],
                 "phases_ms_total": r2["phases_ms_total"], "gpu_launches": r2["gpu_launches"]}
    converge = converge_measure(x, A, mesh, args, local) if args.converge_cap > 0 else None
    les = les_measure(x, A, args, local) if args.les_size > 0 else None
    serving = serve_measure(x, args, local) if args.serve_cases > 0 else None
    batched = batch_measure(x, args, local) if args.serve_cases > 0 else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(x, pm, mesh, args.cpu_iters)
    if rank == 0:
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if primary == "fp64" else "f32/f64",
                "data": "synthetic",
                "config": {"workload": workload_name(n), "cells": mesh.n_cells, "precision": primary,
                           "l2": L2_NOTE},
                "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                "setup": {"nnz_p": r["nnz_p"], "mesh_build_s": round(t_mesh, 2), "setup_s": r["setup_s"]},
                "roofline": r["roofline"], "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": r["gpu_launches"],
                "clocks": r["clocks"], "residuals_last": r["residuals_last"],
                "phases_ms_total": r["phases_ms_total"], "second_precision": other, "to_convergence": converge,
                "les": les,
                "serving": serving, "batch": batched}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
