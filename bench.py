#!/usr/bin/env python
"""Benchmark: occluded pair-integrals/s of the element-pair view-factor assembly.

Workload (one step = one full assembly of the closed-cube configuration):
closed unit cube, edge 1, inward normals, each face a 60 x 60 grid split into
Tri3 with face-interior nodes jittered by +-0.3 h (seed 2) -> 43,200 elements,
933,098,400 unordered pairs; a centred box of edge 0.3 (12 x 12 Tri3 per face,
1,728 triangles) passed as the obstruction group; Dunavant 7-point rule
(nquad = 3); dense 43,200^2 FP64 F matrix.

`value`  -- pairs / s with the mesh resident in HBM (device-timed, CUDA events
            on the library's stream, max over ranks).
`e2e`    -- the same metric through the C ABI with host buffers: mesh upload
            (host -> device) and the full F matrix back to pinned host memory
            inside the timed region.
`--impl reference` times the reference's CPU path (its C++ restatement in
oracle/, all host threads) on a bounded sample of rows of the same workload.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "radiativeviewfactor.jl_b200"
METRIC = "occluded pair-integrals/s"
UNIT = "pair-integrals/s"
NQUAD = 3
OBSTRUCTION = [7]
# algorithmic work constants (flop): 3-D point pair, slab test, Moller-Trumbore
FLOP_POINT_PAIR = 23
FLOP_SLAB = 12
FLOP_TRI = 51
# Reference-order traversal counts of the bench workloads: node (box) tests
# and triangle tests of the reference's stackless walk (src/GPUBVH.jl:202-285)
# ray by ray, from the oracle's instrumented FP64 traversal
# (oracle/ref_counts.py, which prints these numbers).  Every
# cast ray's first box test (the root) runs in the generation kernel, so the
# traversal kernels' algorithmic work is 12 (node_visits - n_rays) + 51 prim_tests.
REF_COUNTS = {
    "medium": {"n_rays": 975146106, "node_visits": 5688464541, "prim_tests": 3647097481},
    "full": {"n_rays": 38102400000, "node_visits": 222278703194, "prim_tests": 142516108216},
}
# DRAM bytes per traced ray of the traversal phase, pair lists included
# (dram__bytes_read.sum + dram__bytes_write.sum of k_trace32 / k_trace64 and
# k_plist in one ncu capture of the medium workload divided by the rays it
# traced; the capture is summarized under profiles/).
TRAFFIC_PER_TRACED_RAY = {"mixed": (0.987216e9 + 0.019866e9 + 0.039880e9 + 0.225654e9) / 75262173,
                          "fp64": (0.990203e9 + 0.017742e9 + 0.039880e9 + 0.225654e9) / 75267549}


def load_pkg():
    if "rvf_b200" in sys.modules:
        return sys.modules["rvf_b200"]
    spec = importlib.util.spec_from_file_location("rvf_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["rvf_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


class Workload:
    """One bench configuration: mesh, obstruction groups and solve options."""

    def __init__(self, md, desc, obs, nquad, method="quadrature", use_duffy=False, n_samples=64, seed=1,
                 precisions=("fp64", "mixed")):
        self.md, self.desc, self.obs, self.nquad = md, desc, list(obs), nquad
        self.method, self.use_duffy, self.n_samples, self.seed = method, use_duffy, n_samples, seed
        self.precisions = list(precisions)

    def options(self, rvf, prec):
        return rvf.make_options(self.nquad, monte_carlo=self.method == "mc", n_samples=self.n_samples,
                                use_duffy=self.use_duffy, seed=self.seed, precision=prec)


def workload(rvf, size: str) -> Workload:
    M = rvf.meshes
    if size == "small":  # quick check of the same shape at m = 12
        return Workload(M.cube_enclosure(12, box_m=4), "cube 12x12/face Tri3 (1,728 elements) + box", OBSTRUCTION,
                        NQUAD)
    if size == "medium":  # profiling size: F = 382 MB > L2, same box
        return Workload(M.cube_enclosure(24, jitter=0.3, seed=2, box=True, box_edge=0.3, box_m=12),
                        "cube 24x24/face jittered Tri3 (6,912 elements) + centred 0.3 box (1,728 tris), nquad=3",
                        OBSTRUCTION, NQUAD)
    if size == "c1":  # the CPU-runnable plain case: coaxial plates, analytic F12 = 0.19982
        return Workload(M.parallel_plates(20, "quad4"),
                        "two coaxial unit squares 1 apart, 20x20 Quad4 each (800 elements), Gauss-Legendre nquad=4, "
                        "no obstruction", [], 4, precisions=("fp64",))
    if size == "c3":  # precision form with Duffy
        return Workload(M.cylinder(nc=64, na=32, caps=True, cap_rings=8, jitter=0.01, seed=3),
                        "open cylinder r=0.5 h=1, 64x32 Quad8 wall + two 64x8 Quad8 annular caps sharing the end "
                        "rings (3,072 elements), +-1% radial jitter, use_duffy, nquad=5, no obstruction", [], 5,
                        use_duffy=True)
    if size == "c4":  # Monte Carlo 2-D
        return Workload(M.cavity_2d(n_wall=800, n_circle=200, n_circles=4, seed=4),
                        "1x1 cavity, 4 x 800 Line3 walls + 4 circles r=0.1 x 200 Line3 (4,000 elements), circles "
                        "as obstruction, stratified Monte Carlo 64 samples (8x8), seed 4", [5, 6, 7, 8], 3,
                        method="mc", n_samples=64, seed=4, precisions=("fp64",))
    return Workload(M.cube_enclosure(60, jitter=0.3, seed=2, box=True, box_edge=0.3, box_m=12),
                    "closed cube 60x60/face jittered Tri3 (43,200 elements) + centred 0.3 box (1,728 tris), "
                    "Dunavant 7-pt (nquad=3), dense FP64 F", OBSTRUCTION, NQUAD)


class Clocks:
    """nvidia-smi sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3] not in ("", "[N/A]"))}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def allreduce_max(x: float, ws: int) -> float:
    """Max over ranks (the slowest replica's time), on the process group's
    own device: CUDA for NCCL, the host for gloo."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, seconds_max: float, ws: int) -> float:
    """Whole-job throughput of ws replicas that each processed units_per_rank
    units, timed as the slowest rank (weak scaling: per-rank work is fixed)."""
    return ws * units_per_rank / seconds_max


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline(rvf, W: Workload, seconds: float, offset: int = 0):
    """The reference's CPU path (src/Assembly.jl:102-225, restated in
    oracle/; Monte Carlo: the restated src/GPUMCKernels.jl streams) on every
    `stride`-th row, all host threads; pairs/s."""
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    from oracle import pyoracle as orc
    md = W.md
    m = orc.Mesh(md, W.obs)
    N = md.n_elems
    cores = os.cpu_count() or 1

    def run(begin, stride):
        if W.method == "mc":
            orc.solve_mc(m, W.n_samples, W.seed, row_begin=begin, row_stride=stride, threads=cores)
        else:
            orc.solve_cpu(m, W.nquad, use_duffy=W.use_duffy, row_begin=begin, row_stride=stride, threads=cores)

    # calibrate on 2 rows per thread
    probe = max(2 * cores, 8)
    stride0 = max(1, N // probe)
    t0 = time.perf_counter()
    run(offset % stride0, stride0)
    dt = time.perf_counter() - t0
    pairs0 = sum(N - 1 - i for i in range(offset % stride0, N, stride0))
    rate = pairs0 / max(dt, 1e-9)
    stride = max(1, int(N * (N / 2) / max(rate * seconds, 1.0)))
    begin = offset % stride
    t0 = time.perf_counter()
    run(begin, stride)
    dt = time.perf_counter() - t0
    pairs = sum(N - 1 - i for i in range(begin, N, stride))
    what = ("Monte Carlo streams of the GPU path" if W.method == "mc" else
            "CPU path with one BVH per active obstruction subset" + (", Duffy pairs" if W.use_duffy else ""))
    return {"value": pairs / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"rows {begin}::{stride} of {N} ({pairs:,} pairs, {dt:.1f} s), {what}, OpenMP over rows"}


def run_reference(args):
    # a host-only run: rank 0 measures and prints, the other ranks exit at once
    # (no process group, no GPU)
    if int(os.environ.get("RANK", "0")) != 0:
        return
    rvf = load_pkg()
    W = workload(rvf, args.size)
    md, desc = W.md, W.desc
    # each step is a bounded row sample, sized so that the whole run (warm-up
    # included) takes about ref_total seconds
    per_step = min(args.ref_seconds, args.ref_total / max(1, args.warmup + args.steps))
    samples, step_s = [], []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        r = cpu_baseline(rvf, W, per_step, offset=k * 7919)
        if k >= args.warmup:
            samples.append(r)
            step_s.append(time.perf_counter() - t0)
    v = statistics.median(s["value"] for s in samples)
    N = md.n_elems
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.mean(step_s),
            "step": "one bounded row sample of the workload (calibration rows, then the timed rows)",
            "ms_full_workload_projected": 1000.0 * (N * (N - 1) / 2) / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "n_elems": N, "nquad": W.nquad},
            "cpu_baseline": {**samples[-1], "value": v},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def timed_solves(dm, opts, steps, warmup, flush, ws, local):
    """W untimed + K timed resident solves; returns per-step stats and clocks."""
    import torch
    for _ in range(warmup):
        dm.solve(opts)
    barrier(ws)
    torch.cuda.synchronize()
    stats = []
    with Clocks(local) as clk:
        for _ in range(steps):
            flush.zero_()  # 256 MB write between steps (L2 flush)
            torch.cuda.synchronize()
            stats.append(dm.solve(opts).as_dict())
    torch.cuda.synchronize()
    barrier(ws)
    return stats, clk.summary()


def roofline(stats, peak, bound, kernel, prec, size):
    """Roofline of the dominant phase, the traversal (pair lists, FP32 rays and
    the FP64 re-traversal in mixed mode): the reference-order traversal work
    of the step / CUDA-event time of the phase."""
    s0 = stats[-1]
    trace_ms = statistics.mean(s["ms_trace"] + s["ms_trace_fp64"] for s in stats)
    chunks = max(1, int(s0["n_chunks"]))
    ref = REF_COUNTS.get(size)
    if ref:
        flops = FLOP_SLAB * (ref["node_visits"] - ref["n_rays"]) + FLOP_TRI * ref["prim_tests"]
        src = "reference-order box and triangle tests (oracle traversal of this workload)"
    else:
        flops = FLOP_SLAB * (s0["node_visits"] - s0["n_rays_traced"]) + FLOP_TRI * s0["prim_tests"]
        src = "box and triangle tests as executed (no reference-order counts for this size)"
    achieved = flops / (trace_ms / 1e3) / 1e12
    # the same time against the tests the kernels actually ran (pair lists and
    # tile masks skip most of the reference's tests: executed < algorithmic)
    ex_flops = FLOP_SLAB * (s0["node_visits"] - s0["n_rays_traced"]) + FLOP_TRI * s0["prim_tests"]
    ex = ex_flops / (trace_ms / 1e3) / 1e12
    tpr = TRAFFIC_PER_TRACED_RAY.get(prec)
    traffic = tpr * s0["n_rays_traced"] / chunks if tpr else None
    return {"bound": bound, "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "executed": {"achieved": ex, "frac": ex / peak, "flop_per_launch": ex_flops / chunks,
                         "box_tests": int(s0["node_visits"]), "triangle_tests": int(s0["prim_tests"]),
                         "rays_traced": int(s0["n_rays_traced"])},
            "traffic": traffic, "peak_source": "measured by rvf_fma_peak (FMA microbenchmark) in this run",
            "kernel": kernel, "kernel_ms_per_launch": trace_ms / chunks, "launches_per_step": chunks,
            "algorithmic_flop_per_launch": flops / chunks, "work_counts": src,
            "traffic_source": "ncu capture of the medium workload scaled by traced rays" if tpr else None}


# Monte Carlo sample pair on Line3 curves: two element evaluations (45 flop
# each), the 2-D kernel (26) and the accumulation (2); a 2-D segment test is
# 14 flop, a box test 12.
FLOP_MC_LINE3 = 45 + 45 + 26 + 2
FLOP_SEG = 14


def roof_for(W: Workload, stats, prec, size, peak64, peak32):
    """Roofline of the workload's dominant kernel."""
    peak, bound = (peak32, "fp32_fma") if prec == "mixed" else (peak64, "fp64_fma")
    s0 = stats[-1]
    if W.method == "mc":
        ms = statistics.mean(s["ms_pairs"] for s in stats)
        flops = FLOP_MC_LINE3 * s0["n_point_pairs"] + FLOP_SLAB * s0["node_visits"] + FLOP_SEG * s0["prim_tests"]
        achieved = flops / (ms / 1e3) / 1e12
        return {"bound": bound, "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": None, "peak_source": "measured by rvf_fma_peak (FMA microbenchmark) in this run",
                "kernel": "k_pairs_mc<DIM3=0,OCC=1> (+ k_mc_area)", "kernel_ms_per_launch": ms,
                "launches_per_step": 1, "algorithmic_flop_per_launch": flops,
                "work_counts": "sample pairs, box and segment tests as executed"}
    if not W.obs:
        ms = statistics.mean(s["ms_gen"] for s in stats)
        flops = FLOP_POINT_PAIR * s0["n_point_pairs"]
        achieved = flops / (ms / 1e3) / 1e12
        return {"bound": bound, "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": None, "peak_source": "measured by rvf_fma_peak (FMA microbenchmark) in this run",
                "kernel": "k_gen_mixed<OCC=0>" if prec == "mixed" else "k_gen_fp64<DIM3=1,OCC=0>",
                "kernel_ms_per_launch": ms, "launches_per_step": 1, "algorithmic_flop_per_launch": flops,
                "work_counts": "23 flop per quadrature point pair (Duffy pairs run in k_duffy, timed in phases)"}
    kernel = "k_plist + k_trace32 (+ k_trace64 re-traversal)" if prec == "mixed" else "k_plist + k_trace64<DIM3=1>"
    return roofline(stats, peak, bound, kernel, prec, size)


def phases(stats):
    keys = ("ms_cull", "ms_gen", "ms_trace", "ms_lists", "ms_trace_fp64", "ms_resolve", "ms_duffy", "ms_pairs",
            "ms_prep", "ms_reduce")
    d = {k: statistics.mean(s[k] for s in stats) for k in keys}
    for k in ("n_chunks", "n_rays_traced", "n_list_pairs", "n_walk_pairs", "n_tiles_culled", "n_pairs_masked",
              "n_tiles_unclassified"):
        d[k] = int(stats[-1][k])
    return d


# ---------------------------------------------------------------------------
# Serving stream (C5): seeded requests with Poisson arrivals through rvf_server
# ---------------------------------------------------------------------------
SERVE_SIZES = {
    # requests, element count range (log-uniform), admission budget
    "small": (32, 2000, 8000, 150 << 30),
    "medium": (128, 2000, 20000, 150 << 30),
    "full": (512, 2000, 40000, 150 << 30),
}


def serve_requests(rvf, n_req, n_lo, n_hi, seed=5):
    """Random geometry (plates / cube enclosure / cylinder), element count
    log-uniform in [n_lo, n_hi], Tri3 / Quad4 / Quad8, nquad 2..5, 30% with
    an obstruction box, 20% Monte Carlo (64 samples); quadrature requests in
    mixed precision."""
    import math
    import numpy as np
    rng = np.random.default_rng(seed)
    M = rvf.meshes
    out = []
    for k in range(n_req):
        n = math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))
        geo = rng.choice(["plates", "cube", "cylinder"])
        fam = rng.choice(["tri3", "quad4", "quad"])
        box = rng.uniform() < 0.3
        mc = rng.uniform() < 0.2
        nquad = int(rng.integers(2, 6))
        obs = []
        if geo == "cylinder":
            nc = max(8, int(round(math.sqrt(n / 0.75) / 4)) * 4)
            md = M.cylinder(nc=nc, na=nc // 2, cap_rings=max(2, nc // 8), seed=int(rng.integers(1 << 30)))
            fam = "quad"
            center = (0.0, 0.0, 0.5)
        elif geo == "cube":
            per = 12 if fam == "tri3" else 6
            md = M.cube_enclosure(max(2, int(round(math.sqrt(n / per)))), family=fam, box=False,
                                  seed=int(rng.integers(1 << 30)))
            center = (0.5, 0.5, 0.5)
        else:
            per = 4 if fam == "tri3" else 2
            md = M.parallel_plates(max(2, int(round(math.sqrt(n / per)))), fam)
            center = (0.5, 0.5, 0.5)
        if box:
            md.group_tri_soup[99] = M.obstruction_box(center=center, edge=0.3, m=8)
            obs = [99]
        o = rvf.make_options(nquad, monte_carlo=bool(mc), n_samples=64, seed=int(rng.integers(1 << 62)),
                             precision="fp64" if mc else "mixed")
        out.append({"md": md, "obs": obs, "opts": o, "geo": str(geo), "family": fam, "nquad": nquad,
                    "box": bool(box), "mc": bool(mc), "N": md.n_elems})
    return out


def serve_work(r) -> int:
    """Work of one request for the service-time estimate: quadrature point
    pairs (points per element from the family and nquad: nquad^2 on quads,
    the 1/3/7/13-point triangle rules), or sample pairs for Monte Carlo."""
    N = r["N"]
    P = N * (N - 1) // 2
    if r["mc"]:
        return P * 64
    nq = r["nquad"]
    pts = nq * nq if r["family"] in ("quad4", "quad") else (1 if nq <= 1 else 3 if nq == 2 else 7 if nq == 3 else 13)
    return P * pts * pts


def run_serve(rvf, sess, size: str, local: int):
    """p50/p99 latency and throughput of a Poisson request stream through the
    serving loop, offered at 80% of the server's measured capacity; the
    capacity (a burst of the stream's first 32 requests) is set beside the
    same 32 requests solved one at a time, and a fixed sample of the served
    results is compared with plain FP64 one-at-a-time solves."""
    import math
    import queue
    import threading
    import numpy as np
    from rvf_b200 import _abi
    n_req, n_lo, n_hi, admit = SERVE_SIZES[size]
    reqs = serve_requests(rvf, n_req, n_lo, n_hi)
    arrays = [rvf.mesh_desc_arrays(r["md"], r["obs"]) for r in reqs]
    pairs = [r["N"] * (r["N"] - 1) // 2 for r in reqs]
    burst = list(range(min(n_req, 32)))
    # the burst's requests one at a time through the public API: mesh upload,
    # solve with the request's options (result left on the device), release --
    # the work the server does per request; each after one warm-up solve of
    # its own mesh (session buffers and launch graphs warm, as in a service)
    t_alone, t_solve_only = [], []
    clk_alone = Clocks(local).__enter__()
    for k in burst:
        r = reqs[k]
        dm = _abi.DeviceMesh(sess, arrays[k])
        dm.solve(r["opts"])
        t0 = time.perf_counter()
        dm.solve(r["opts"])
        t_solve_only.append(time.perf_counter() - t0)
        dm.release()
        t0 = time.perf_counter()
        dm = _abi.DeviceMesh(sess, arrays[k])
        dm.solve(r["opts"])
        dm.release()
        t_alone.append(time.perf_counter() - t0)
    clk_alone.__exit__(None, None, None)
    # the burst: the same requests submitted at once to a server of their own,
    # each released when done; timed on its second pass, when the session's
    # buffer cache holds F buffers for the burst's concurrent requests (as the
    # one-at-a-time solves above reuse theirs: a service in steady state)
    for rep in range(2):
        sv = _abi.Server(sess, admit_bytes=admit)
        clk_burst = Clocks(local).__enter__()
        t0 = time.perf_counter()
        rids = {sv.submit(arrays[k], reqs[k]["opts"]) for k in burst}
        while rids:  # release in completion order
            rid = sv.wait_any(3_600_000)
            if rid in rids:
                sv.release(rid)
                rids.discard(rid)
        t_burst = time.perf_counter() - t0
        clk_burst.__exit__(None, None, None)
        st_burst = sv.stats()
        sv.close()
    # Offered load: each request's cost is its work (quadrature point pairs or
    # Monte Carlo sample pairs) at the burst's measured rate for its kind;
    # the arrival rate puts the stream at 80% of that capacity.
    work = [serve_work(r) for r in reqs]
    t_kind = {kind: sum(t_alone[n] for n, k in enumerate(burst) if reqs[k]["mc"] == kind) for kind in (False, True)}
    sec_per_unit = {}
    for kind in (False, True):
        units = sum(work[k] for k in burst if reqs[k]["mc"] == kind)
        sec_per_unit[kind] = t_kind[kind] / units if units else 0.0
    if not sec_per_unit[True]:
        sec_per_unit[True] = sec_per_unit[False]
    cost = [work[k] * sec_per_unit[reqs[k]["mc"]] for k in range(n_req)]
    est_service = sum(cost) * t_burst / sum(cost[k] for k in burst)
    mean_service = est_service / n_req
    lam = 0.8 / mean_service
    rng = np.random.default_rng(7)
    arrivals = np.cumsum(rng.exponential(1.0 / lam, size=n_req))
    # a fixed sample of the quadrature requests (10% of the stream, at least
    # 50 on the full one), evenly spread: 64 rows and columns of each served
    # F against a plain FP64 one-at-a-time solve of the same mesh
    quad = [k for k in range(n_req) if not reqs[k]["mc"]]
    n_check = min(len(quad), max(math.ceil(0.1 * n_req), 50 if size == "full" else 4))
    check = sorted({quad[int(c * len(quad) / n_check)] for c in range(n_check)})
    ref_rows = {}
    for k in check:
        r = reqs[k]
        N = r["N"]
        dm = _abi.DeviceMesh(sess, arrays[k])
        dm.solve(rvf.make_options(r["nquad"], seed=0, precision="fp64"))
        idx = np.unique(np.linspace(0, N - 1, min(N, 64)).astype(np.int64))
        ref_rows[k] = (idx,) + device_rows_cols(dm.result_device(), N, idx, local)
        dm.release()
    sv = _abi.Server(sess, admit_bytes=admit)
    submitted = queue.Queue()
    err = []
    dF, n_checked = 0.0, 0

    def submitter():
        t0 = time.perf_counter()
        for k in range(n_req):
            dt = arrivals[k] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            submitted.put((k, sv.submit(arrays[k], reqs[k]["opts"])))

    th = threading.Thread(target=submitter)
    t_start = time.perf_counter()
    th.start()
    # The client takes each request as it finishes (rvf_wait_any), reads the
    # checked results on the device and releases every request at once: a
    # finished request keeps its device memory and its admission charge
    # until rvf_release, so releasing in submission order would hold finished
    # results behind a long request and stall admission.
    id2k = {}
    for _ in range(n_req):
        rid = sv.wait_any(3_600_000)
        while rid not in id2k:  # the submitter thread hands over (k, id) after rvf_submit returns
            k, r = submitted.get()
            id2k[r] = k
        k = id2k.pop(rid)
        try:
            state, status, _ = sv.poll(rid)
            if status != 0:
                raise _abi.RVFError(status, f"request {k}: {state}")
            if k in ref_rows:
                idx, rr, cc = ref_rows.pop(k)
                rows, cols = device_rows_cols(sv.result_device(rid), reqs[k]["N"], idx, local)
                dF = max(dF, float(np.nanmax(np.abs(rows - rr))), float(np.nanmax(np.abs(cols - cc))))
                n_checked += 1
        except _abi.RVFError as e:
            err.append(str(e))
        try:
            sv.release(rid)
        except _abi.RVFError:
            pass
    wall = time.perf_counter() - t_start
    th.join()
    st = sv.stats()
    sv.close()
    total_pairs = sum(pairs)
    burst_pairs = sum(pairs[k] for k in burst)
    return {
        "metric": "serve latency and throughput", "requests": n_req, "failed": len(err),
        "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
        "throughput_pairs_per_s": total_pairs / wall, "wall_s": wall,
        "burst_pairs_per_s": burst_pairs / t_burst, "burst_s": t_burst, "burst_requests": len(burst),
        "one_at_a_time_pairs_per_s": burst_pairs / sum(t_alone),
        "one_at_a_time_s": sum(t_alone),
        "one_at_a_time": "the burst's requests, each alone through the public API after a warm-up solve of its "
                         "mesh: mesh upload, solve with the request's options (result left on the device), "
                         "release -- the work the server does per request",
        "one_at_a_time_solve_only_pairs_per_s": burst_pairs / sum(t_solve_only),
        "burst_over_one_at_a_time": sum(t_alone) / t_burst,
        "clocks_one_at_a_time": clk_alone.summary(), "clocks_burst": clk_burst.summary(),
        "lambda_per_s": lam, "offered_load": 0.8, "estimated_service_s": est_service,
        "max_abs_dF_vs_fp64_solo": dF, "checked_requests": n_checked,
        "check": "64 rows and columns of each checked served F against a plain FP64 one-at-a-time solve",
        "chunks": st["chunks"], "batched_requests": st["batched_requests"], "graph_replays": st["graph_replays"],
        "admit_bytes": admit, "admitted_bytes_peak": st["admitted_bytes_peak"],
        "burst_worker_ms": {"admit": st_burst["ms_admit"], "quad_chunks": st_burst["ms_quad_chunks"],
                            "mc_chunks": st_burst["ms_mc_chunks"], "free": st_burst["ms_free"],
                            "idle": st_burst["ms_idle"]},
        "one_at_a_time_ms": {"quad": 1e3 * sum(t for n, t in enumerate(t_alone) if not reqs[burst[n]]["mc"]),
                             "mc": 1e3 * sum(t for n, t in enumerate(t_alone) if reqs[burst[n]]["mc"]),
                             "solve_only": 1e3 * sum(t_solve_only)},
        "tuned_shapes": st["tuned"], "tuned_shapes_burst": st_burst["tuned"],
        "config": {"stream": f"{n_req} seeded requests (seed 5), Poisson arrivals, N log-uniform {n_lo}-{n_hi}, "
                             "plates / cube / cylinder, Tri3 / Quad4 / Quad8, nquad 2-5, 30% obstruction box, "
                             "20% Monte Carlo (64 samples), quadrature in mixed precision",
                   "mix": {"mc": sum(r["mc"] for r in reqs), "box": sum(r["box"] for r in reqs),
                           "elements_total": sum(r["N"] for r in reqs)}},
    }


class _DeviceMatrix:
    """A column-major N x N FP64 matrix at a device address, seen by torch
    through the CUDA array interface (no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n, n), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": (8, 8 * n)}


def device_rows_cols(ptr, N, idx, local):
    """Rows F[i, :] and columns F[:, i] of the device F for the sampled i."""
    import ctypes
    import torch
    addr = ctypes.cast(ptr, ctypes.c_void_p).value
    F = torch.as_tensor(_DeviceMatrix(addr, N), device=f"cuda:{local}")
    ii = torch.as_tensor(idx, dtype=torch.int64, device=f"cuda:{local}")
    rows = F.index_select(0, ii).cpu().numpy()
    cols = F.index_select(1, ii).cpu().numpy().T.copy()
    return rows, cols


def oracle_sample(W: Workload, stride: int):
    """The oracle's raw values on sampled rows of the workload (the rows
    i = 0, stride, 2 stride, ...): (rows, raw[rows, :] as rows x N, areas,
    seconds).  Quadrature: every pair of the row as the reference's GPU path
    integrates it, Duffy pairs replaced by the oracle's Sauter-Schwab
    integrals; Monte Carlo: the reference's streams for the pairs (i, j > i)."""
    import numpy as np
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    from oracle import pyoracle as orc
    m = orc.Mesh(W.md, W.obs)
    N = W.md.n_elems
    rows = np.arange(0, N, stride, dtype=np.int64)
    t0 = time.perf_counter()
    if W.method == "mc":
        raw, area, _, _ = orc.solve_mc(m, W.n_samples, W.seed, row_stride=stride, threads=os.cpu_count() or 1)
        out = raw[rows, :].copy()
        del raw
    else:
        out, area, _ = orc.solve_rows(m, W.nquad, rows, threads=os.cpu_count() or 1)
        if W.use_duffy:
            for r, i in enumerate(rows):
                for j in range(N):
                    if j == i:
                        continue
                    a, b = (int(i), j) if i < j else (j, int(i))
                    if orc.singularity_type(m, a, b)[0] > 0:
                        out[r, j] = orc.pair_duffy(m, a, b, W.nquad, None, gpu_semantics=True)[0]
    return rows, out, area, time.perf_counter() - t0


def compare_with_oracle(rows, raw, area, Frows, Fcols, mc):
    """The device F against the oracle on the sampled rows (F[i, :] = raw / A_i)
    and columns (F[:, i] = raw / A_j): largest absolute and relative element
    difference, whether they are identical, the row-sum deviation and the
    reciprocity A_i F_ij = A_j F_ji."""
    import numpy as np
    N = raw.shape[1]
    with np.errstate(invalid="ignore", divide="ignore"):
        Fo_r = raw / area[rows][:, None]
        Fo_c = raw / area[None, :]
    if mc:  # Monte Carlo rows hold the pairs j > i only
        mask = np.arange(N)[None, :] > rows[:, None]
    else:
        mask = np.arange(N)[None, :] != rows[:, None]
    d_r = np.abs(Frows - Fo_r)[mask]
    d_c = np.abs(Fcols - Fo_c)[mask]
    ref_r = np.abs(Fo_r)[mask]
    ref_c = np.abs(Fo_c)[mask]
    rel = max(float(np.max(d_r / np.maximum(ref_r, 1e-300))), float(np.max(d_c / np.maximum(ref_c, 1e-300))))
    out = {"max_abs_dF": max(float(d_r.max()), float(d_c.max())), "max_rel_dF": rel,
           "identical": bool(np.array_equal(Frows[mask], Fo_r[mask]) and np.array_equal(Fcols[mask], Fo_c[mask]))}
    if not mc:
        out["max_row_sum_dev"] = float(np.max(np.abs(np.where(mask, Frows, 0.0).sum(axis=1) -
                                                     np.where(mask, Fo_r, 0.0).sum(axis=1))))
        lhs, rhs = area[rows][:, None] * Frows, area[None, :] * Fcols
        rec = np.abs(lhs - rhs)[mask] / np.maximum(np.abs(lhs)[mask], 1e-30)
        out["max_reciprocity_err"] = float(rec.max())
    return out


def run_ours(args):
    ws, rank, local = dist_setup()
    rvf = load_pkg()
    import numpy as np
    import torch
    from rvf_b200 import _abi
    if not _abi.LIB_PATH.exists():
        raise SystemExit("librvf_b200.so is not built (run __graft_entry__.build())")
    W = workload(rvf, args.size)
    md, desc = W.md, W.desc
    N = md.n_elems
    G = len(md.group_tags)
    pairs = N * (N - 1) // 2
    sess = _abi.Session(local)
    arrays = rvf.mesh_desc_arrays(md, W.obs)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    precisions = W.precisions if args.precision == "both" else [p for p in W.precisions if p == args.precision]
    if not precisions:
        raise SystemExit(f"--precision {args.precision} is not available for --size {args.size}")
    head = precisions[-1]
    runs, meshes = {}, {}
    for prec in precisions:
        opts = W.options(rvf, prec)
        dm = _abi.DeviceMesh(sess, arrays)
        stats, clocks = timed_solves(dm, opts, args.steps, args.warmup, flush, ws, local)
        total_ms = allreduce_max(sum(s["ms_total"] for s in stats), ws)
        runs[prec] = {"stats": stats, "clocks": clocks, "ms": total_ms / args.steps,
                      "value": job_rate(pairs * args.steps, total_ms / 1e3, ws)}
        meshes[prec] = dm
    accuracy = None
    if len(precisions) == 2:
        d = _abi.max_abs_diff(meshes["fp64"].result_device(), meshes["mixed"].result_device(), N * N)
        accuracy = {"max_abs_dF_mixed_vs_fp64": d,
                    "max_row_sum_dev_fp64": runs["fp64"]["stats"][-1]["max_row_sum_dev"],
                    "max_row_sum_dev_mixed": runs["mixed"]["stats"][-1]["max_row_sum_dev"],
                    "rays_fp64_retraced_mixed": runs["mixed"]["stats"][-1]["n_rays_fp64"],
                    "pairs_fp64_mixed": runs["mixed"]["stats"][-1]["n_pairs_fp64"],
                    "unsure_rays": {k: runs["mixed"]["stats"][-1][k] for k in
                                    ("unsure_rays", "unsure_slab", "unsure_prim", "unsure_direction")},
                    "graze_point_pairs": runs["mixed"]["stats"][-1]["graze_point_pairs"]}
    vs_oracle = None
    if rank == 0 and args.oracle_stride > 0:
        stride = args.oracle_stride if args.size == "full" else max(1, min(args.oracle_stride, N // 32))
        rows, raw, area, t_orc = oracle_sample(W, stride)
        vs_oracle = {"rows": int(rows.size), "row_stride": int(stride), "oracle_s": t_orc,
                     "pairs_checked": int(sum(N - 1 - i for i in rows) if W.method == "mc" else rows.size * (N - 1)),
                     "what": "every stride-th row and column of the device F against the oracle's restatement of "
                             "the reference's GPU path (Duffy pairs: its Sauter-Schwab integrals; Monte Carlo: "
                             "its streams, pairs j > i)"}
        for prec, dm in meshes.items():
            Fr, Fc = device_rows_cols(dm.result_device(), N, rows, local)
            vs_oracle[prec] = compare_with_oracle(rows, raw, area, Fr, Fc, W.method == "mc")
        del raw
    for dm in meshes.values():
        dm.release()
    peak64 = _abi.fma_peak(local, True)
    peak32 = _abi.fma_peak(local, False)
    H = runs[head]
    roof = roof_for(W, H["stats"], head, args.size, peak64, peak32)

    # ---- e2e: through the C ABI with host buffers, every precision ----
    e2e_all = {}
    if not args.no_e2e:
        h2d = sum(a.nbytes for k, a in arrays.items() if hasattr(a, "nbytes")) + sum(t.nbytes for t in arrays["nodes"])
        d2h = 8 * (N * N + N + G * G + G)
        try:
            Fh = _abi.PinnedArray((N, N), order="F")
            F, pinned = Fh.array, True
        except Exception:
            F, pinned = np.empty((N, N), order="F"), False
        A = np.empty(N)
        Fg = np.empty((G, G), order="F")
        Ag = np.empty(G)
        for prec in precisions:
            opts = W.options(rvf, prec)
            times = []
            for k in range(args.e2e_warmup + args.e2e_steps):
                barrier(ws)
                t0 = time.perf_counter()
                mesh_arrays = rvf.mesh_desc_arrays(md, W.obs)
                ta = time.perf_counter()
                d = _abi.DeviceMesh(sess, mesh_arrays)
                tb = time.perf_counter()
                st = d.solve(opts, F, A, Fg, Ag).as_dict()
                tc = time.perf_counter()
                d.release()
                t1 = time.perf_counter()
                if k >= args.e2e_warmup:
                    times.append(t1 - t0)
                    # where the last step's time went (host clock, and the
                    # solve's own event-timed phases)
                    brk = {"flatten_ms": 1e3 * (ta - t0), "upload_ms": 1e3 * (tb - ta),
                           "solve_ms": 1e3 * (tc - tb), "release_ms": 1e3 * (t1 - tc),
                           "solve_phases_ms": {key: round(st[key], 2) for key in
                                               ("ms_prep", "ms_cull", "ms_pairs", "ms_reduce", "ms_download",
                                                "ms_total")}}
            t = allreduce_max(sum(times), ws)
            e2e_all[prec] = {"value": job_rate(pairs * len(times), t, ws), "unit": UNIT,
                             "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                             "host_buffer": "pinned" if pinned else "pageable", "steps": len(times),
                             "s_per_step": t / len(times), "precision": prec, "last_step": brk}
        if pinned:
            Fh.free()
    e2e = e2e_all.get(head)

    s0 = H["stats"][-1]
    line = {"metric": METRIC, "value": H["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": H["ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if head == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": desc, "n_elems": N, "pairs_per_step": pairs, "nquad": W.nquad,
                       "method": W.method, "use_duffy": W.use_duffy,
                       "precision": head, "parallelism": f"replicas x{ws} (independent meshes)",
                       "l2": "each step writes the dense F matrix (C2: 14.9 GB >> 126 MB L2); a 256 MB "
                             "buffer is also written between steps"},
            "e2e": e2e,
            "gpu_launches": int(sum(s["gpu_kernels"] for s in H["stats"])),
            "roofline": roof,
            "clocks": H["clocks"],
            "phases": phases(H["stats"]),
            "counts": {k: s0[k] for k in ("n_point_pairs", "n_rays", "n_rays_fp64", "n_pairs_fp64", "node_visits",
                                          "prim_tests", "n_rays_traced")}}
    if len(precisions) == 2:
        line["fp64"] = {"value": runs["fp64"]["value"], "ms_per_step": runs["fp64"]["ms"],
                        "e2e": e2e_all.get("fp64"),
                        "roofline": roof_for(W, runs["fp64"]["stats"], "fp64", args.size, peak64, peak32),
                        "phases": phases(runs["fp64"]["stats"]),
                        "clocks": runs["fp64"]["clocks"]}
        line["mixed_over_fp64"] = runs["mixed"]["value"] / runs["fp64"]["value"]
        line["accuracy"] = accuracy
    if vs_oracle is not None:
        line["accuracy"] = dict(line.get("accuracy") or {}, vs_oracle=vs_oracle)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(rvf, W, args.ref_seconds)
    if rank == 0 and args.serve != "none":
        line["serve"] = run_serve(rvf, sess, args.serve, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    del flush
    sess.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed", "both"], default="both")
    ap.add_argument("--size", choices=["full", "medium", "small", "c1", "c3", "c4"], default="full",
                    help="full: the headline workload (closed cube, 43,200 Tri3, occluded); c1: 20x20 Quad4 plates; "
                         "c3: cylinder with Duffy pairs; c4: 2-D Monte Carlo cavity; medium / small: the headline "
                         "shape at m = 24 / 12")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--e2e-warmup", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-seconds", type=float, default=15.0)
    ap.add_argument("--ref-total", type=float, default=150.0,
                    help="--impl reference: seconds for the whole run (warm-up and timed samples)")
    ap.add_argument("--oracle-stride", type=int, default=97,
                    help="compare every stride-th row and column of the device F with the oracle (0: off)")
    ap.add_argument("--serve", choices=["none", "small", "medium", "full"], default="small",
                    help="serving stream reported beside the main line (small: 32 requests, 2k-8k elements; "
                         "medium: 128, 2k-20k; full: 512, 2k-40k)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
