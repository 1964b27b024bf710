#!/usr/bin/env python
"""bench.py -- time to an FP64 relative residual of 1e-10 for the plain nested
F3R solve on one B200.

Workload: the nonsymmetric 27-point stencil on a 192^3 grid (7,077,888 rows,
189,119,224 nonzeros; diagonal 26, neighbours at a positive linear offset
-1+beta, negative -1-beta, beta = 0.5), symmetrically diagonal-scaled as the
reference drivers do, stored SELL-32 in natural row order (sigma = 1) with
offset-aligned slices (no stored column index), SDAINV
(tol 0.1, acc 1.0) innermost, F3R(m2=8, m3=4, m4=2, c=64) under an fp64
FGMRES(100), b = A x* with x* ~ U(-1, 1) from mt19937_64(seed = rank).
Synthetic data (the reference publishes no dataset for this configuration).

One step = one full solve from x0 = 0 to ||b - Ax|| / ||b|| < 1e-10 (the
implicit Givens estimate, checked against the explicit fp64 residual).  With
N GPUs every rank solves its own system (replicas, no collective on the data
path); the time is the max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

The SELL layout is a tuning choice: `--layout aligned` (the default, the
fastest the SELL autotuner found: 144 us per fp16 product at 192^3) or
`--layout sigma256` (SELL-C-sigma with C = 32, sigma = 256 and explicit
32-bit indices, 212 us).  Every run also times a few solves in the other
layout and reports them under config.alt_layout.

Other preconditioners on the same workload (not the headline configuration):
  --precond ilu-bj      block-Jacobi ILU(0), exact level-scheduled solves
  --precond ilu-jacobi  ILU(0) solved by --trsv-iters Jacobi sweeps (trsv/jacobi.hpp)
  --precond ilu-baj     ILU(0) solved by --trsv-iters BAJ sweeps (trsv/baj.hpp)
with --ilu-blocks B (112, the reference's; 1 = one global ILU(0)).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = 192
BETA = 0.5
SIGMA = 1
ALIGN = 1
SELL_C = 64
LAYOUTS = {"aligned": dict(sell_sigma=1, sell_align=1, format=0, sell_c=32),
           "aligned64": dict(sell_sigma=1, sell_align=1, format=0, sell_c=64),
           "sigma256": dict(sell_sigma=256, sell_align=0, format=0, sell_c=32),
           "csr": dict(sell_sigma=1, sell_align=0, format=1, sell_c=32),
           "auto": dict(sell_sigma=1, sell_align=0, format=0, sell_autotune=1, sell_c=32)}
TOL = 1e-10
PARAMS = dict(m_outer=100, max_restarts=20, m2=8, m3=4, m4=2, c=64, sdainv_tol=0.1, acc=1.0, sell_sigma=SIGMA,
              sell_align=ALIGN, format=0, sell_c=SELL_C,
              rel_tol=TOL, use_graphs=1)
METRIC = "time to 1e-10 FP64 relative residual, plain F3R (fp64/fp32/fp16 nested FGMRES), 192^3 27-pt nonsymmetric"
WORKLOAD = "F3R-SDAINV-SELL64al stencil27-halfspace beta0.5 192^3 (n=7077888, nnz=189119224), tol 1e-10"


PRECONDS = {"sdainv": 0, "ilu-bj": 1, "ilu-jacobi": 2, "ilu-baj": 3, "ilu-level": 4}
PRECOND_DESC = "SDAINV(tol=0.1, acc=1.0)"


def set_size(nx):
    global NX, WORKLOAD
    NX = nx
    nnz = 27 * nx ** 3 - 54 * nx ** 2 + 36 * nx - 8
    WORKLOAD = (f"F3R-SDAINV-{layout_tag()} stencil27-halfspace beta0.5 {nx}^3 (n={nx ** 3}, nnz={nnz}), tol 1e-10")


def layout_tag():
    if PARAMS.get("format"):
        return "CSR"
    c = PARAMS.get("sell_c", 32)
    return f"SELL{c}al" if PARAMS["sell_align"] else f"SELL{c}s{PARAMS['sell_sigma']}"


def set_layout(name):
    PARAMS.update(LAYOUTS[name])


AUTOTUNED = {}


def layout_desc(p=None):
    p = PARAMS if p is None else p
    if p.get("sell_autotune"):
        return {"autotuned": True}
    if AUTOTUNED and p is PARAMS:
        return dict(AUTOTUNED["chosen"], autotuned=True)
    if p.get("format"):
        return {"format": "CSR", "index": "explicit int32"}
    return {"C": p.get("sell_c", 32), "sigma": p["sell_sigma"],
            "index": "offset-aligned (no stored column index)" if p["sell_align"] else "explicit int32"}


def set_precond(name, blocks, iters):
    """Switches the innermost preconditioner (PARAMS, workload name, config)."""
    global WORKLOAD, PRECOND_DESC
    if name == "sdainv":
        return
    PARAMS.update(precond=PRECONDS[name], ilu_blocks=blocks, trsv_iters=iters)
    label = {"ilu-bj": f"BJILU0x{blocks}-levels", "ilu-jacobi": f"ILU0x{blocks}-jacobi{iters}",
             "ilu-baj": f"ILU0x{blocks}-baj{iters}", "ilu-level": "ILU0-global-levels"}[name]
    WORKLOAD = WORKLOAD.replace("F3R-SDAINV", "F3R-" + label)
    PRECOND_DESC = {"ilu-bj": f"block-Jacobi ILU(0), {blocks} blocks, exact level-scheduled triangular solves",
                    "ilu-jacobi": f"ILU(0) over {blocks} block(s), {iters} Jacobi sweeps per triangular solve",
                    "ilu-baj": f"ILU(0) over {blocks} block(s), BAJ max_iter {iters}",
                    "ilu-level": "one global ILU(0), exact triangular solves level-scheduled over the whole GPU"}[name]


def config_dict(extra=None):
    d = {"workload": WORKLOAD, "grid": [NX, NX, NX], "n": NX ** 3, "nnz": 27 * NX ** 3 - 54 * NX ** 2 + 36 * NX - 8, "sell": layout_desc(),
         "f3r": {"m_outer": 100, "m2": 8, "m3": 4, "m4": 2, "c": 64, "restarts": 20},
         "precond": PRECOND_DESC, "rhs": "b = A x*, x* ~ U(-1,1) mt19937_64(rank)",
         "l2": "inputs larger than L2 (fp16+fp32+fp64 matrix copies 4.6 GB, vectors 12 GB)",
         "parallelism": "replicas (one independent system per GPU)"}
    if extra:
        d.update(extra)
    return d


def replica_seed(rank: int) -> int:
    """With N GPUs each rank solves its own system (replicas, no collective on
    the data path): x* ~ U(-1, 1) from mt19937_64(seed = rank)."""
    return rank


def max_over_ranks(value: float, world: int, device=None) -> float:
    """The job's time is the slowest rank's (all_reduce MAX; identity at N=1)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_problem(seed: int):
    import f3r_b200 as F
    A = F.stencil27(NX, NX, NX, 2, BETA).scale()
    n = A.shape[0]
    xs = F.random_uniform(seed, -1.0, 1.0, n)
    b = A.spmv(xs)
    return A, b, xs


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(aligned=False, height=32):
    """dram bytes per launch of the dominant kernel from the committed ncu summary"""
    if aligned and height == 64:
        name = "spmv_f16_aligned64_c2_traffic.txt"
    else:
        name = "spmv_f16_aligned_c2_traffic.txt" if aligned else "spmv_f16_c2_traffic.txt"
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("bytes_per_launch"):
                    return float(line.split("=")[1])
    except (OSError, ValueError, IndexError):
        pass
    return None


def spmv_roofline(solver, A, torch, F):
    """Dominant kernel: the fp16-matrix SELL SpMV of level 3 on the solver's
    own matrix, as the solve runs it (fp16 values, x from level 3's fp16 Z
    basis, fp32 y; the Richardson step, the largest share, is the same
    product with a fused epilogue), timed with CUDA events on the stream the
    library launches on.  `achieved` / `frac` use the CSR-equivalent
    algorithmic bytes, nnz * (2 + 4) + 4 (n + 1) + 2 n + 4 n, whatever the
    stored layout; the offset-aligned layout stores no column index, so there
    they are an effective rate that can exceed the copy peak, and `stored_*`
    give the rate over the bytes the layout actually holds (padded values,
    slice-column bases, row pointers, x and y)."""
    n, nnz = A.shape[0], A.nnz
    info, _ = solver.info()
    x = torch.randn(n, dtype=torch.float32, device="cuda").to(torch.float16)
    y = torch.empty(n, dtype=torch.float32, device="cuda")
    for _ in range(5):
        solver.operate(x, y, val_t=F.F16)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 50
    e0.record(torch.cuda.current_stream())
    for _ in range(reps):
        solver.operate(x, y, val_t=F.F16)
    e1.record(torch.cuda.current_stream())
    torch.cuda.synchronize()
    dt = e0.elapsed_time(e1) * 1e-3 / reps
    alg = nnz * (2 + 4) + 4 * (n + 1) + n * 2 + n * 4
    aligned = info.index_bits == 0
    csr = info.slice_height == 0
    h = info.slice_height or 32
    nslices = (n + h - 1) // h
    idx_bytes = (info.nnz_padded // h) * 4 if aligned else info.nnz_padded * 4
    stored = alg if csr else info.nnz_padded * 2 + idx_bytes + 4 * (nslices + 1) + n * 2 + n * 4
    peak, src = measured_peak()
    achieved = alg / dt / 1e9
    if csr:
        kern = "k_csr_cfg<__half,__half,EpiStore<float>,24> (CSR, fp16 A, fp16 x, fp32 y)"
    elif h == 64:
        kern = "k_sell64<__half,__half,EpiStore<float>,32,1,32> (64-row offset-aligned slices, fp16 A, fp16 x, fp32 y)"
    elif aligned:
        kern = ("k_sell_cfg<__half,__half,EpiStore<float>,32,2,32,AllAlignedIdx> (SELL-32 sigma=1, offset-aligned, "
                "fp16 A, fp16 x, fp32 y)")
    else:
        kern = (f"k_sell_cfg<__half,__half,EpiStore<float>,24,2,16,int> (SELL-32 sigma={info.sigma}, fp16 A, fp16 x, "
                "fp32 y)")
    return {"kernel": kern, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "peak_source": src,
            "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None if csr else profiled_traffic(aligned, h),
            "algorithmic_bytes": alg, "effective_rate": aligned, "stored_bytes": stored,
            "stored_achieved": round(stored / dt / 1e9, 1), "stored_frac": round(stored / dt / 1e9 / peak, 4),
            "launch_us": round(dt * 1e6, 2)}


def time_alt_layout(F, torch, ctx, A, b_d, stream, steps=3):
    """The same solve in the other SELL layout (a few solves, device time),
    reported beside the headline so the layout choice can be checked."""
    other = "sigma256" if PARAMS["sell_align"] else "aligned"
    p = dict(PARAMS)
    p.update(LAYOUTS[other])
    S = F.Solver(ctx, A, **p)
    x = torch.zeros_like(b_d)
    for _ in range(2):
        x.zero_()
        S.solve(b_d, x)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        x.zero_()
        r = S.solve(b_d, x)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    roof = spmv_roofline(S, A, torch, F)
    S.close()
    return {"layout": layout_desc(p), "ms_per_solve": round(ms, 3), "steps": steps, "outer_iters": r.res_iter,
            "expl_rel_res": r.expl_rel_res, "spmv_f16_us": roof["launch_us"]}


def cpu_baseline(A, b, iters_gpu, sample_steps=2):
    """The reference's own CPU F3R (oracle/_ref, compiled from the reference
    sources) on this host's cores: a bounded sample of `sample_steps` outer
    FGMRES steps of the same solve, scaled to the outer-step count of the GPU
    solve."""
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    from oracle import oracle as O
    try:
        ref = O.Ref("fast")
    except FileNotFoundError as e:
        return {"value": None, "unit": "ms", "cores": cores, "kind": "reference", "sample": f"unavailable: {e}"}
    rptr, idx, val = A.arrays()
    # the reference's SDAINV + SELL-32 method (f3r-gpu.cpp) or, for the ILU
    # preconditioners, its block-Jacobi ILU(0) + CSR method (f3r.cpp)
    config = 0 if PARAMS.get("precond", 0) == 0 else 1
    r = ref.f3r_solve(config, rptr, idx, val, b, tol=TOL, stop_after=sample_steps)
    per_step = r["time_s"] / max(r["iters"], 1)
    return {"value": round(per_step * iters_gpu * 1e3, 1), "unit": "ms", "cores": int(os.environ["OMP_NUM_THREADS"]),
            "kind": "reference",
            "sample": f"{r['iters']} outer FGMRES steps of the same {NX}^3 solve on the host "
                      f"({ref.name}, {'SELL-32 + SDAINV' if config == 0 else 'CSR + BJ-ILU(0) x112'}, fp16 as "
                      f"_Float16; {per_step:.2f} s/step), "
                      f"scaled by the GPU solve's {iters_gpu} outer steps"}


def run_ours(args):
    import torch
    import torch.distributed as dist
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    import f3r_b200 as F

    A, b, xs = make_problem(seed=replica_seed(rank))
    n = A.shape[0]
    ctx = F.Context(local)
    stream = torch.cuda.Stream()          # one non-default stream for torch and the library
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    solver = F.Solver(ctx, A, **PARAMS)
    if PARAMS.get("sell_autotune"):
        # the layout the autotuner chose, in the config's terms
        info, _ = solver.info()
        PARAMS.update(format=1 if info.slice_height == 0 else 0, sell_sigma=info.sigma,
                      sell_align=1 if info.index_bits == 0 else 0, sell_autotune=0,
                      sell_c=info.slice_height if info.slice_height else 32)
        AUTOTUNED["chosen"] = layout_desc()
    b_d = torch.from_numpy(b).cuda()
    x_d = torch.zeros_like(b_d)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(max(args.warmup, 3)):
        x_d.zero_()
        r = solver.solve(b_d, x_d)
    barrier()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    results = []
    torch.cuda.nvtx.range_push("timed")
    e0.record(stream)
    for _ in range(args.steps):
        x_d.zero_()
        results.append(solver.solve(b_d, x_d))
    e1.record(stream)
    torch.cuda.nvtx.range_pop()
    barrier()
    ck = clocks.stop()
    t = max_over_ranks(e0.elapsed_time(e1) * 1e-3, world, "cuda")
    ms_per = t / args.steps * 1e3
    r = results[-1]
    err = float(torch.linalg.norm(x_d.cpu() - torch.from_numpy(xs)) / np.linalg.norm(xs))

    # end to end through the public API with pinned host buffers: b and x0
    # copied in, x copied out, every step
    b_h = torch.from_numpy(b).pin_memory()
    x_h = torch.zeros(n, dtype=torch.float64).pin_memory()
    x_h.zero_()
    solver.solve(b_h, x_h)
    barrier()
    w0 = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        x_h.zero_()
        re = solver.solve(b_h, x_h)
    e1.record(stream)
    barrier()
    t_e2e = max(e0.elapsed_time(e1) * 1e-3, 0.0)
    wall_e2e = max_over_ranks(time.perf_counter() - w0, world, "cuda")
    e2e_ms = wall_e2e / args.steps * 1e3

    roof = spmv_roofline(solver, A, torch, F) if rank == 0 else None
    alt = time_alt_layout(F, torch, ctx, A, b_d, stream) if (rank == 0 and not args.no_alt_layout) else None
    cpu = cpu_baseline(A, b, r.res_iter) if (rank == 0 and world == 1 and not args.no_cpu_baseline) else None
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(ms_per, 3), "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": round(ms_per, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "mixed: f16 storage/f32 accumulate, f32, f64",
            "data": "synthetic (seeded 192^3 stencil, b = A x*)",
            "config": config_dict({"solves_per_s_all_gpus": round(world * args.steps / t, 3), "alt_layout": alt}),
            "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": 2 * n * 8,
                    "d2h_bytes_per_step": n * 8, "timed_with": "host wall clock around solve() on pinned buffers",
                    "device_ms": round(t_e2e / args.steps * 1e3, 3)},
            "gpu_launches": int(sum(x.kernel_launches for x in results)),
            "solve": {"outer_iters": r.res_iter, "inner_applications": r.inner_applications,
                      "impl_rel_res": r.impl_rel_res, "expl_rel_res": r.expl_rel_res, "x_rel_err": err,
                      "restarts": r.restarts, "device_ms_per_solve": round(r.solve_seconds * 1e3, 3),
                      "kernels_per_solve": r.kernel_launches},
            "roofline": roof, "cpu_baseline": cpu, "clocks": ck,
        }
    solver.close()
    ctx.close()
    if rank == 0:
        if world == 1 and not args.no_extra and NX == 192:  # the configurations' own sizes, headline runs only
            line["extra"] = extra_block(args, A)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    """The reference's own CPU F3R (compiled in place from its sources into
    oracle/_ref) on this host's cores, same metric and workload.  Warm-up 1 is
    a full solve (its outer-step count is kept); every timed step is a bounded
    sample of 1 outer step, scaled by that count.  Rank 0 only."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    from oracle import oracle as O
    try:
        ref = O.Ref("fast")
    except FileNotFoundError as e:
        print(json.dumps({"impl": "reference", "unavailable": str(e)}))
        return
    A, b, _ = make_problem(seed=0)
    rptr, idx, val = A.arrays()
    full = ref.f3r_solve(0, rptr, idx, val, b, tol=TOL)
    iters = full["iters"]
    samples = []
    for i in range(max(args.warmup - 1, 0) + args.steps):
        r = ref.f3r_solve(0, rptr, idx, val, b, tol=TOL, stop_after=1)
        if i >= max(args.warmup - 1, 0):
            samples.append(r["time_s"] / max(r["iters"], 1))
    per_step = statistics.mean(samples)
    value = per_step * iters * 1e3
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": "ms", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(per_step * 1e3, 1),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "mixed: _Float16 storage/arith, f32, f64", "data": "synthetic (seeded 192^3 stencil, b = A x*)",
            "config": config_dict({"sell": {"C": 32, "sigma": 1, "index": "explicit int32 (the reference's SELL<32>)"}}),
            "cpu_baseline": {"value": round(value, 1), "unit": "ms", "cores": int(os.environ["OMP_NUM_THREADS"]),
                             "kind": "reference",
                             "sample": f"each step = 1 outer FGMRES step of the 192^3 solve ({ref.name}); value = "
                                       f"mean step time x {iters} outer steps of a full solve run in warm-up "
                                       f"({full['time_s']:.2f} s measured, expl res {full['expl_res']:.2e})"},
            "full_solve_s": round(full["time_s"], 3), "outer_iters": iters,
            "e2e": {"value": round(value, 1), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def make_c4(seed=4, count=96):
    """The batched configuration: `count` systems from one master seed; each a
    7-point variable-coefficient diffusion (sigma 1.0, correlation length 4
    cells) or the 27-point half-space stencil, edge ~ U{16..112}, nrhs ~
    U{1..16}, right-hand sides ~ N(0, 1)."""
    import f3r_b200 as F
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        kind = 7 if rng.integers(2) == 0 else 27
        e = int(rng.integers(16, 113))
        k = int(rng.integers(1, 17))
        A = F.diffusion7(e, e, e, 1.0, 4.0, seed * 1000 + i) if kind == 7 else F.stencil27(e, e, e, 2, BETA)
        A.scale()
        B = np.ascontiguousarray(rng.standard_normal((k, e ** 3)))
        out.append((kind, e, A, B))
    return out


def run_c4(args):
    print(json.dumps(c4_line(args)), flush=True)


def c4_line(args):
    """C4: the batch solved at once (f3r_solve_batch: each system's
    right-hand sides in lockstep blocks, systems on their own contexts
    concurrently) against one right-hand side at a time; wall time around the
    whole batch with the device synchronised on both sides."""
    import torch
    import f3r_b200 as F
    torch.cuda.set_device(0)
    t_setup = time.perf_counter()
    systems = make_c4()
    ctxs, solvers = [], []
    for kind, e, A, B in systems:
        ctxs.append(F.Context(0))
        # lockstep blocks take 32-row slices (64-row slices would solve the columns one after another)
        solvers.append(F.Solver(ctxs[-1], A, **{**PARAMS, **LAYOUTS["aligned"]}))
    Bd = [torch.from_numpy(B).cuda() for _, _, _, B in systems]
    Xd = [torch.zeros_like(b) for b in Bd]
    batch = [(S, b, x) for S, b, x in zip(solvers, Bd, Xd)]
    t_setup = time.perf_counter() - t_setup

    def batched():
        for x in Xd:
            x.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = F.solve_batch(batch)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, res

    def sequential():
        """one right-hand side at a time, system after system"""
        for x in Xd:
            x.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = [[S.solve(b[k], x[k]) for k in range(b.shape[0])] for S, b, x in batch]
        torch.cuda.synchronize()
        return time.perf_counter() - t0, res

    def blocks():
        """each system's right-hand sides in lockstep blocks, system after system"""
        for x in Xd:
            x.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = [S.solve_multi(b, x) for S, b, x in batch]
        torch.cuda.synchronize()
        return time.perf_counter() - t0, res

    for _ in range(max(args.warmup, 1)):
        batched()
        blocks()
        sequential()
    tb = min(batched()[0] for _ in range(args.steps))
    tk = min(blocks()[0] for _ in range(args.steps))
    ts, res = min((sequential() for _ in range(args.steps)), key=lambda t: t[0])
    _, resb = batched()
    nrhs = sum(B.shape[0] for _, _, _, B in systems)
    rows = sum(A.shape[0] * B.shape[0] for _, _, A, B in systems)
    worst = max(r.expl_rel_res for rs in resb for r in rs)
    line = {"metric": "time to 1e-10 FP64 relative residual for the whole batch (C4: 96 systems, 1-16 RHS each)",
            "value": round(tb * 1e3, 2), "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": False, "dtype": "mixed: f16 storage/f32 accumulate, f32, f64",
            "data": "synthetic (seeded C4 batch)",
            "config": {"workload": "C4 batched: 96 systems, 7-pt diffusion / 27-pt stencil, edge U{16..112}, "
                                   "nrhs U{1..16}, RHS N(0,1), tol 1e-10",
                       "systems": len(systems), "rhs": nrhs, "rows_x_rhs": rows,
                       "sell": layout_desc({**PARAMS, **LAYOUTS["aligned"]}),
                       "timing": "host wall clock, device synchronised on both sides"},
            "batched_ms": round(tb * 1e3, 2), "sequential_ms": round(ts * 1e3, 2),
            "blocks_one_system_at_a_time_ms": round(tk * 1e3, 2),
            "speedup_batched_vs_sequential": round(ts / tb, 2), "speedup_blocks_vs_sequential": round(ts / tk, 2),
            "solves_per_s": round(nrhs / tb, 1),
            "modes": "batched: f3r_solve_batch (each system's right-hand sides in lockstep blocks of up to 16, "
                     "systems on their own contexts concurrently); blocks: the same blocks, one system after "
                     "another; sequential: one right-hand side at a time",
            "all_solved": all(r.is_solved for rs in resb for r in rs), "worst_expl_rel_res": worst,
            "outer_iters_total": sum(r.res_iter for rs in resb for r in rs), "setup_s": round(t_setup, 1)}
    for S in solvers:
        S.close()
    for c in ctxs:
        c.close()
    return line


def level_errors(F, torch, solver, A_unscaled_range, A, xs):
    """Error of every precision level against fp64, on the solved (scaled)
    system: the value copies' rounding (max relative entry error) and the
    products w = A z at each level's types against the fp64 product, all on
    z = x* (the exact solution)."""
    rptr, idx, val = A.arrays()
    e16 = np.abs(val.astype(np.float16).astype(np.float64) - val) / np.abs(val)
    e32 = np.abs(val.astype(np.float32).astype(np.float64) - val) / np.abs(val)
    n = A.shape[0]
    z64 = torch.from_numpy(xs).cuda()
    y64 = torch.empty_like(z64)
    solver.operate(z64, y64, val_t=F.F64)
    z32 = z64.float()
    y32 = torch.empty_like(z32)
    solver.operate(z32, y32, val_t=F.F32)
    y16 = torch.empty_like(z32)
    solver.operate(z32, y16, val_t=F.F16)           # level 3: fp16 matrix, fp32 vectors
    z16 = z64.half()
    y16h = torch.empty(n, dtype=torch.float16, device="cuda")
    solver.operate(z16, y16h, val_t=F.F16)           # level 4: fp16 matrix, fp16 vectors
    torch.cuda.synchronize()
    ref = y64.double()
    nr = float(torch.linalg.norm(ref))
    rel = lambda y: float(torch.linalg.norm(y.double() - ref)) / nr
    return {"raw_entry_range": A_unscaled_range,
            "scaled_entry_range": [float(np.abs(val).min()), float(np.abs(val).max())],
            "value_rounding_max_rel": {"fp32": float(e32.max()), "fp16": float(e16.max())},
            "spmv_rel_err_vs_fp64": {"level2_fp32": rel(y32), "level3_fp16A_fp32x": rel(y16),
                                     "level4_fp16A_fp16x": rel(y16h)}}


def run_c3(args):
    print(json.dumps(c3_line(args)), flush=True)


def c3_line(args):
    """C3, precision stress: 7-point diffusion with coefficients exp(g) (g a
    seeded Gaussian field, sigma 2.5, correlation length 8 cells) on an
    nx^3 grid (256 by default), diagonally scaled into fp16 range; time to
    1e-10 and the error of every precision level against fp64."""
    import torch
    import f3r_b200 as F
    torch.cuda.set_device(0)
    nx = args.nx if args.nx != NX else 256
    A = F.diffusion7(nx, nx, nx, 2.5, 8.0, 3)
    raw = np.abs(A.arrays()[2])
    raw_range = [float(raw.min()), float(raw.max())]
    A.scale()
    n = A.shape[0]
    xs = F.random_uniform(0, -1.0, 1.0, n)
    b = A.spmv(xs)
    ctx = F.Context(0)
    t0 = time.perf_counter()
    S = F.Solver(ctx, A, **PARAMS)
    setup = time.perf_counter() - t0
    b_d = torch.from_numpy(b).cuda()
    x_d = torch.zeros_like(b_d)
    for _ in range(max(args.warmup, 1)):
        x_d.zero_()
        S.solve(b_d, x_d)
    torch.cuda.synchronize()
    times, r = [], None
    for _ in range(args.steps):
        x_d.zero_()
        r = S.solve(b_d, x_d)
        times.append(r.solve_seconds)
    err = float(torch.linalg.norm(x_d.cpu() - torch.from_numpy(xs)) / np.linalg.norm(xs))
    lv = level_errors(F, torch, S, raw_range, A, xs)
    line = {"metric": "time to 1e-10 FP64 relative residual, plain F3R, C3 precision stress", "value":
            round(min(times) * 1e3, 2), "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": False, "dtype": "mixed: f16 storage/f32 accumulate, f32, f64",
            "data": "synthetic (seeded log-normal coefficient field)",
            "config": {"workload": f"C3: 7-pt diffusion exp(g), sigma 2.5, corr 8, {nx}^3 (n={n}, nnz={A.nnz}), "
                                   "SDAINV, tol 1e-10", "sell": layout_desc(), "setup_s": round(setup, 1)},
            "solve": {"outer_iters": r.res_iter, "inner_applications": r.inner_applications,
                      "impl_rel_res": r.impl_rel_res, "expl_rel_res": r.expl_rel_res,
                      "x_rel_err_vs_exact": err, "solved": r.is_solved},
            "levels": lv}
    S.close()
    ctx.close()
    return line


def run_c1(args):
    """C1, the reference's own CPU configuration (work/src/f3r.cpp:44-58,
    195-248): the hpcg 27-point matrix on a 64^3 grid (diagonal 26,
    neighbours -1), scaled, b = A_s 1, x0 = 0, tol 1e-10, F3R(8, 4, 2, c 64)
    with a restart cap of 3, acc 1.0, block-Jacobi ILU(0) over 112 blocks,
    CSR storage.  Our GPU solve in exactly that configuration (format CSR,
    exact level-scheduled block solves), the same preconditioner in the
    offset-aligned SELL layout, and the reference's compiled CPU solve on all
    host cores (oracle/_ref, config 1 = f3r.cpp's solver)."""
    import torch
    import f3r_b200 as F
    torch.cuda.set_device(0)
    nx = args.nx if args.nx != NX else 64
    A = F.stencil27(nx, nx, nx, 0, 0.0).scale()
    n = A.shape[0]
    b = A.spmv(np.ones(n))
    kw = dict(m_outer=100, max_restarts=3, m2=8, m3=4, m4=2, c=64, precond=F.PRECOND_ILU0_BJ, ilu_blocks=112,
              acc=1.0, rel_tol=TOL, use_graphs=1)
    ctx = F.Context(0)

    def gpu(layout):
        S = F.Solver(ctx, A, **kw, **layout)
        x = np.zeros(n)
        for _ in range(max(args.warmup, 1)):
            x[:] = 0
            S.solve(b, x)
        best, wall = None, []
        for _ in range(args.steps):
            x[:] = 0
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = S.solve(b, x)
            wall.append(time.perf_counter() - t0)
            best = r if best is None or r.solve_seconds < best.solve_seconds else best
        S.close()
        return best, min(wall), float(np.max(np.abs(x - 1.0)))

    r_csr, w_csr, e_csr = gpu(dict(format=1, sell_sigma=1, sell_align=0))
    r_al, w_al, _ = gpu(dict(format=0, sell_sigma=1, sell_align=1))
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    ref_line = None
    try:
        from oracle import oracle as O
        ref = O.Ref("fast")
        rptr, idx, val = A.arrays()
        runs = [ref.f3r_solve(1, rptr, idx, val, b, m2=8, m3=4, m4=2, c=64, restarts=3, tol=TOL, acc=1.0, blocks=112)
                for _ in range(2)]
        rr = min(runs, key=lambda d: d["time_s"])
        ref_line = {"ms": round(rr["time_s"] * 1e3, 1), "outer_iters": rr["iters"], "expl_rel_res": rr["expl_res"],
                    "solved": rr["solved"], "cores": int(os.environ["OMP_NUM_THREADS"]), "build": ref.name}
    except FileNotFoundError as e:
        ref_line = {"unavailable": str(e)}
    line = {"metric": "time to 1e-10 FP64 relative residual, F3R in the reference's CPU configuration (C1)",
            "value": round(r_csr.solve_seconds * 1e3, 2), "unit": "ms", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False, "dtype": "mixed: f16 storage/f32 accumulate, f32, f64",
            "data": "synthetic (hpcg 27-point matrix, b = A 1)",
            "config": {"workload": f"C1: hpcg 27-pt {nx}^3 (n={n}, nnz={A.nnz}), BJ-ILU(0) x112 exact, CSR, "
                                   "F3R(8,4,2,c=64), restart cap 3, tol 1e-10",
                       "timing": "device solve time (CUDA events), best of steps"},
            "e2e": {"value": round(w_csr * 1e3, 2), "unit": "ms", "h2d_bytes_per_step": 16 * n,
                    "d2h_bytes_per_step": 8 * n},
            "solve": {"outer_iters": r_csr.res_iter, "expl_rel_res": r_csr.expl_rel_res, "solved": r_csr.is_solved,
                      "max_abs_err_vs_ones": e_csr},
            "aligned_sell_same_precond": {"ms": round(r_al.solve_seconds * 1e3, 2), "outer_iters": r_al.res_iter,
                                          "e2e_ms": round(w_al * 1e3, 2)},
            "reference_cpu": ref_line}
    if ref_line and "ms" in ref_line:
        line["reference_cpu_over_gpu_e2e"] = round(ref_line["ms"] / (w_csr * 1e3), 1)
    print(json.dumps(line), flush=True)


C5_BATCH = 8  # held-out systems kept for the batched comparison (two solvers each)


def c2_block_line(args, A):
    """K right-hand sides of the headline 192^3 system solved as one
    lockstep block (f3r_solver_solve_multi) against the same K solved one at a
    time on the same solver, in the bench's layout; device time (CUDA events)
    of each, and whether every block column is bit for bit its single solve."""
    import torch
    import f3r_b200 as F
    K = args.block_k
    torch.cuda.set_device(0)
    ctx = F.Context(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    kw = {**PARAMS, "sell_autotune": 0}
    S = F.Solver(ctx, A, **kw)
    n = A.shape[0]
    B = np.stack([A.spmv(F.random_uniform(100 + k, -1.0, 1.0, n)) for k in range(K)])
    B_d = torch.from_numpy(B).cuda()
    Xb, Xs = torch.zeros_like(B_d), torch.zeros_like(B_d)
    S.solve_multi(B_d, Xb)      # warm-up: the block's work buffers and graphs
    S.solve(B_d[0], Xs[0])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, tag):
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push(tag)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    Xb.zero_()
    tb, rb = timed(lambda: S.solve_multi(B_d, Xb), "block")
    Xs.zero_()
    ts, rs = timed(lambda: [S.solve(B_d[k], Xs[k]) for k in range(K)], "singles")
    line = {"workload": f"C2 192^3 27-point stencil, {K} right-hand sides b_k = A x*_k, x*_k ~ U(-1, 1)",
            "rhs": K, "sell": layout_desc(kw),
            "timing": "device time, CUDA events on the solver's stream",
            "block_ms": round(tb, 2), "singles_ms": round(ts, 2),
            "block_ms_per_rhs": round(tb / K, 2), "single_ms_per_rhs": round(ts / K, 2),
            "per_rhs_time_ratio_block_vs_single": round(tb / ts, 3),
            "all_solved": all(r.is_solved for r in rb), "outer_iters": [r.res_iter for r in rb],
            "columns_bit_identical_to_single_solves": bool(torch.equal(Xb, Xs)),
            "worst_expl_rel_res": max(r.expl_rel_res for r in rb)}
    S.close()
    ctx.close()
    return line


def extra_block(args, A=None):
    """The learned / batched / precision-stress half of the metric, measured
    after the headline solve and outside its timed region, at the sizes of
    their configurations: C2 block (K right-hand sides of the headline system
    in one lockstep block), C5 (learned vs plain SDAINV, held-out 128^3
    fields), C4 (the 96-system batch), C3 (the 256^3 precision stress).  Each
    is timed with its own clock (stated in its config) and reported in full;
    a part that fails is reported as an error string instead."""
    import copy
    import torch
    out = {}
    sub = copy.copy(args)
    sub.steps, sub.warmup, sub.nx = 2, 1, NX
    sub.c5_eval = max(args.c5_eval, 8)
    saved = dict(PARAMS)
    parts = [("c5", c5_line), ("c4", c4_line), ("c3", c3_line)]
    if A is not None:
        parts.insert(0, ("c2_block", lambda a: c2_block_line(a, A)))
    for key, fn in parts:
        t0 = time.perf_counter()
        try:
            PARAMS.clear()
            PARAMS.update(saved)
            out[key] = fn(sub)
        except Exception as e:  # noqa: BLE001 -- reported in the line, the headline stands
            out[key] = {"error": f"{type(e).__name__}: {e}"}
        out[key]["wall_s"] = round(time.perf_counter() - t0, 1)
        torch.cuda.empty_cache()
    PARAMS.clear()
    PARAMS.update(saved)
    return out


def run_c5(args):
    print(json.dumps(c5_line(args)), flush=True)


def c5_line(args):
    """C5, the learned preconditioner: the network trained on the GPU on
    residual / error pairs of 256 seeded 7-point log-normal fields (sigma
    1.5, correlation length 6; 24^3 each, stacked), then held-out 128^3
    fields solved to 1e-10:
      * one at a time (device time of each solve, best of steps), with plain
        SDAINV and with the learned correction (BF16 tensor-core inference),
        in the headline's layout (offset-aligned SELL);
      * batched: groups of C5_BATCH fields of the one 7-point pattern solved
        together (f3r_batch: one lockstep solve, each column its own system
        with its own values and factors), plain and learned; wall time of the
        group's solve with the device synchronised on both sides.
    learned+batched is compared with plain solves one after another."""
    import torch
    import f3r_b200 as F
    from f3r_b200.learned import Learned, training_set
    torch.cuda.set_device(0)
    nx = args.nx if args.nx != NX else 128
    ctx = F.Context(0)
    t0 = time.perf_counter()
    ts = training_set(ctx, range(args.c5_train), nt=args.c5_train_grid, **PARAMS)
    t_data = time.perf_counter() - t0
    L = Learned(ctx, seed=0)
    L.set_data(**ts.data())
    t0 = time.perf_counter()
    losses = L.train(args.c5_steps, 2e-3)
    t_train = time.perf_counter() - t0
    final_loss = L.evaluate()
    n_train, n_pairs = ts.A.shape[0], ts.r.shape[0]
    del ts
    rows, held = [], []
    fallbacks = {"single": 0, "plain": 0, "learned": 0}
    inference_us = {}
    for s in range(10000, 10000 + args.c5_eval):
        A = F.diffusion7(nx, nx, nx, 1.5, 6.0, s).scale()
        n = A.shape[0]
        Z, Wt = A.sdainv()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Zc, Wc = L.correct(A, nx, nx, Z, Wt)
        t_inf = time.perf_counter() - t0
        b = A.spmv(F.random_uniform(s, -1.0, 1.0, n))
        Sp = F.Solver(ctx, A, factors=(Z, Wt), **PARAMS)
        Sl = F.Solver(ctx, A, factors=(Zc, Wc), **PARAMS)
        b_d = torch.from_numpy(b).cuda()
        x_d = torch.zeros_like(b_d)
        rec = {"seed": s, "correct_call_ms": round(t_inf * 1e3, 1)}
        if not held:  # the network alone on the first field's features, both tensor-core engines
            inference_us = {e: round(L.time_inference(A, nx, nx, Z, Wt, engine=e, reps=20), 2)
                            for e in ("tcgen05", "mma.sync")}
        for name, S in (("plain", Sp), ("learned", Sl)):
            for _ in range(max(args.warmup, 1)):
                x_d.zero_()
                S.solve(b_d, x_d)
            best = None
            for _ in range(args.steps):
                x_d.zero_()
                r = S.solve(b_d, x_d)
                best = r if best is None or r.solve_seconds < best.solve_seconds else best
            rec[name] = {"ms": round(best.solve_seconds * 1e3, 2), "outer_iters": best.res_iter,
                         "expl_rel_res": best.expl_rel_res, "solved": bool(best.is_solved)}
        if not (rec["learned"]["solved"] and rec["learned"]["expl_rel_res"] < 1e-10):
            # the learned solve fell short: plain SDAINV solves the field again, and its time counts
            fallbacks["single"] += 1
            rec["learned"]["fell_back"] = True
            rec["learned"]["ms"] = round(rec["learned"]["ms"] + rec["plain"]["ms"], 2)
        # residual after a fixed number of outer steps (one fewer than plain needs): the
        # convergence gain that the whole-iteration count can hide
        k = max(1, rec["plain"]["outer_iters"] - 1)
        for name, S in (("plain", Sp), ("learned", Sl)):
            x_d.zero_()
            r = S.solve(b_d, x_d, cond=lambda i, e, k=k: i >= k)
            rec[name][f"expl_rel_res_after_{k}"] = r.expl_rel_res
        Sp.close()
        Sl.close()
        rows.append(rec)
        held.append((A, b, (Z, Wt), (Zc, Wc)))

    # batched: the held-out fields in groups of C5_BATCH, one f3r_batch each
    bp = dict(PARAMS)
    bp.update(sell_align=0)
    bat = {"plain": [], "learned": []}
    solved = True
    for g0 in range(0, len(held), C5_BATCH):
        grp = held[g0:g0 + C5_BATCH]
        bs = [torch.from_numpy(b).cuda() for _, b, _, _ in grp]
        xs = [torch.zeros_like(b) for b in bs]
        for name, fi in (("plain", 2), ("learned", 3)):
            B = F.Batch(ctx, [h[0] for h in grp], factors=[h[fi] for h in grp], **bp)
            best = None
            for it in range(max(args.warmup, 1) + args.steps):
                for x in xs:
                    x.zero_()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                res = B.solve(bs, xs)
                torch.cuda.synchronize()
                dt = time.perf_counter() - t0
                if it >= max(args.warmup, 1) and (best is None or dt < best[0]):
                    best = (dt, res)
            # a system the batch leaves unsolved is solved again alone with plain SDAINV, and that
            # solve's time is added to the batch's
            fb_s = 0.0
            for (A, b, pf, _), r in zip(grp, best[1]):
                if r.is_solved and r.expl_rel_res < 1e-10:
                    continue
                fallbacks[name] += 1
                Sf = F.Solver(ctx, A, factors=pf, **PARAMS)
                xf = torch.zeros(A.shape[0], dtype=torch.float64, device="cuda")
                rf = Sf.solve(torch.from_numpy(b).cuda(), xf)
                fb_s += rf.solve_seconds
                solved = solved and rf.is_solved
                Sf.close()
            bat[name].append({"systems": len(grp), "wall_ms": round((best[0] + fb_s) * 1e3, 2),
                              "outer_iters": [r.res_iter for r in best[1]]})
            B.close()
    mean = lambda key: float(np.mean([r[key]["ms"] for r in rows]))
    per_sys = {k: sum(g["wall_ms"] for g in v) / len(held) for k, v in bat.items()}
    gains = [r["plain"][k] / r["learned"][k] for r in rows for k in r["plain"] if k.startswith("expl_rel_res_after")]
    plain_ms = mean("plain")
    line = {"metric": "time to 1e-10 FP64 relative residual per system, learned / batched vs plain SDAINV (C5)",
            "value": round(per_sys["learned"], 2), "unit": "ms", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "dtype": "mixed: f16 storage/f32 accumulate, f32, f64; MLP bf16 inference, f32 training",
            "data": "synthetic (seeded log-normal coefficient fields)",
            "config": {"workload": f"C5: 7-pt diffusion, log-normal sigma 1.5, corr 6, {nx}^3 held-out "
                                   f"(n={nx ** 3}), SDAINV vs learned SDAINV, tol 1e-10",
                       "train_fields": args.c5_train, "train_grid": f"{args.c5_train_grid}^3 each, stacked", "train_rows": n_train,
                       "eval_fields": args.c5_eval, "batch": C5_BATCH, "sell_single": layout_desc(),
                       "sell_batched": "packed SELL-32, int32 indices, values of the batch interleaved",
                       "timing": "single: device solve time (CUDA events), best of steps; batched: host wall "
                                 "clock around one batch solve, device synchronised on both sides, best of steps, "
                                 "divided by the systems"},
            "plain_ms": round(plain_ms, 2),
            "learned_ms": round(mean("learned"), 2),
            "plain_batched_ms_per_system": round(per_sys["plain"], 2),
            "learned_batched_ms_per_system": round(per_sys["learned"], 2),
            "learned_over_plain_time": round(mean("learned") / plain_ms, 3),
            "speedup_learned_batched_vs_plain": round(plain_ms / per_sys["learned"], 3),
            "speedup_plain_batched_vs_plain": round(plain_ms / per_sys["plain"], 3),
            "outer_iters": {"plain": [r["plain"]["outer_iters"] for r in rows],
                            "learned": [r["learned"]["outer_iters"] for r in rows]},
            "residual_gain_at_fixed_outer_steps": {"min": round(min(gains), 2), "max": round(max(gains), 2),
                                                   "geomean": round(float(np.exp(np.mean(np.log(gains)))), 2)},
            "batched": bat, "all_solved": solved and all(r[k]["solved"] for r in rows for k in ("plain", "learned")),
            "fallbacks_to_plain": {"learned_single": fallbacks["single"], "plain_batched": fallbacks["plain"],
                                   "learned_batched": fallbacks["learned"]},
            "inference_us_first_field": inference_us,
            "training": {"pairs": n_pairs, "steps": args.c5_steps, "train_s": round(t_train, 2),
                         "data_s": round(t_data, 1), "loss_first": float(losses[0]), "loss_final": final_loss},
            "systems": rows}
    L.close()
    ctx.close()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nx", type=int, default=NX, help="grid edge (the benchmark is 192; smaller sizes for profiling)")
    ap.add_argument("--precond", default="sdainv", choices=sorted(PRECONDS),
                    help="innermost preconditioner of our arm (the headline is sdainv)")
    ap.add_argument("--ilu-blocks", type=int, default=112)
    ap.add_argument("--trsv-iters", type=int, default=2)
    ap.add_argument("--layout", default="aligned64", choices=sorted(LAYOUTS),
                    help="matrix layout of our arm: offset-aligned SELL sigma=1 with 64-row slices (default) or "
                         "32-row slices (aligned), packed SELL sigma=256, CSR, or auto (the library's layout "
                         "autotuner picks at set-up)")
    ap.add_argument("--no-alt-layout", action="store_true", help="skip timing the other layout")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the C2-block / C5 / C4 / C3 measurements the default C2 line carries under `extra`")
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c2block", "c3", "c4", "c5"],
                    help="c2: the headline solve; c2block: --block-k right-hand sides of the c2 system as one "
                         "lockstep block against one at a time; "
                         "c3: the precision stress (256^3 diffusion, per-level errors); "
                         "c4: the batched configuration (96 systems, 1-16 RHS each); "
                         "c5: the learned preconditioner (training, then held-out 128^3 solves); "
                         "c1: the reference's CPU configuration (64^3 hpcg, BJ-ILU(0) x112, CSR) on the GPU and, "
                         "beside it, the reference's CPU solve")
    ap.add_argument("--block-k", type=int, default=8, help="right-hand sides of the C2 block measurement")
    ap.add_argument("--c5-train", type=int, default=256, help="C5 training fields")
    ap.add_argument("--c5-train-grid", type=int, default=24, help="C5 training field edge")
    ap.add_argument("--c5-eval", type=int, default=4, help="C5 held-out fields solved (32 for the full set)")
    ap.add_argument("--c5-steps", type=int, default=500, help="C5 Adam steps")
    args = ap.parse_args()
    if args.impl == "ours":
        set_layout(args.layout)
    set_size(args.nx)
    if args.impl == "ours":
        set_precond(args.precond, args.ilu_blocks, args.trsv_iters)
    if args.config == "c1":
        run_c1(args)
    elif args.config == "c5":
        run_c5(args)
    elif args.config == "c4":
        run_c4(args)
    elif args.config == "c3":
        run_c3(args)
    elif args.config == "c2block":
        A, _, _ = make_problem(seed=replica_seed(0))
        print(json.dumps(c2_block_line(args, A)), flush=True)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
