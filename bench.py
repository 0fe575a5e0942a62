"""Benchmark of the B200 Jacobi-PCG hot path on the 1108x1108 2D P1-FEM system.

Workload: interior grid 1108 x 1108 (n = 1,227,664, ~7 nnz/row), jittered nodes (0.3h),
log-normal per-element conductivity sigma = 2.0, random symmetric permutation (seed 1) then
reverse Cuthill-McKee, SELL-C-sigma C=32 sigma=256 chunk 4, b = A x_true with x_true ~ U(-1,1), x0 = 0,
tolerance 1e-8 FP64 true relative residual.  Synthetic (generated here; the reference's
SuiteSparse thermal2 of the same shape class is not available offline).

A step is one full solve to tolerance.  `value` is solves/s over all ranks; the line also
carries time-to-tolerance, SpMV GB/s (L2-flushed and warm), the roofline of the persistent
kernel, an end-to-end number through the public host-array API, and the reference's own CPU
code timed on a bounded sample (cpu_baseline).  With --gpus N > 1 every rank solves its own
replica (the single-system solve does not shard; no collective on the data path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--grid G]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "time-to-1e-8 rel. residual: learned/mixed vs plain Jacobi-PCG; SpMV HBM GB/s"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
# Iterations the reference's run_jacobi_pcg (src/CgSolverGolden.hpp:42-124, built from its
# sources) takes on the 1108x1108 system to ||r|| <= 1e-8 ||b||: one full solve, 170 s on one
# core (the reference arm times a bounded sample of it per step).
GOLDEN_ITERATIONS_1108 = 5569
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the SM-resident kernel per
# iteration on the 1108x1108 system: 349.1 MB over a captured launch of 100 iterations
# (ncu --set full of `python -m project_xplus_b200.profile_case --grid 1108 --iters 100 --spmv 0`).
RESIDENT1_DRAM_BYTES_PER_ITER = 349.1e6 / 100


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--grid", type=int, default=1108, help="interior grid side (n = grid^2)")
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--cpu-sample-iters", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the plain-FP32 and FP64 comparison solves")
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-system batched solve")
    ap.add_argument("--no-spmv3d", action="store_true", help="skip the SpMV on the 128^3 3D system")
    ap.add_argument("--no-config0", action="store_true", help="skip the n = 1024 system's GPU/CPU comparison")
    ap.add_argument("--clocks-dir", default=None,
                    help="directory for the nvidia-smi clock samples (default: a temporary directory)")
    a = ap.parse_args()
    if a.clocks_dir:
        Clocks.out_dir = Path(a.clocks_dir)
    return a


def peaks():
    if PEAKS_FILE.exists():
        p = json.loads(PEAKS_FILE.read_text())
        return float(p["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def workload_config(args, extra=None):
    c = {"workload": f"2d-p1fem-{args.grid}x{args.grid}-sigma2-perm1-rcm", "n": args.grid * args.grid,
         "tol_rel_true": args.tol, "format": "sell-c32-sigma256 chunk4, row-sum form, int16 column offsets",
         "precision": "fp32 values+vectors, fp64 x accumulation and fp64 residual replacement",
         "l2": "flushed between timed solves (256 MiB write)", "parallelism": f"replicas x{args.gpus}"}
    if extra:
        c.update(extra)
    return c


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    out_dir = None  # --clocks-dir, else a fresh temporary directory per process

    def __init__(self, device_index, append=False):
        self.dev = device_index
        self.proc = None
        self.append = append
        if Clocks.out_dir is None:
            import tempfile
            Clocks.out_dir = Path(tempfile.mkdtemp(prefix="xplus_bench_clocks_"))
        self.path = Path(Clocks.out_dir) / f"clocks_rank{device_index}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            self.f = open(self.path, "a" if self.append else "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl" if args.impl == "b200" else "gloo",
                                timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, value, device):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, device=None):
    if pg is not None:
        if device is not None:
            pg.barrier(device_ids=[device.index])
        else:
            pg.barrier()


# --------------------------------------------------------------------------------------
# reference arm: the reference's own CPU code (oracle/_ref, built from its sources)
# --------------------------------------------------------------------------------------
def cpu_model():
    """The host CPU's model name (for the CPU baselines' tables)."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cuper_reference_sample(d, iters):
    """Times the reference's own FP32-SpMV software PCG (run_cuper_pcg_solver,
    host/cuper_pcg_solver.hpp:311, oracle/_ref) on this host, one thread: `iters` and
    iters / 4 iterations, the per-iteration cost as the slope.  Returns (seconds per iteration,
    plan build in ms) or None without the reference build."""
    from oracle import oracle as O
    if O.reflib() is None:
        return None
    t0 = time.perf_counter()
    r = O.cuper_pcg_ref(d, 1e-300, iters)
    dt = time.perf_counter() - t0
    t1 = time.perf_counter()
    O.cuper_pcg_ref(d, 1e-300, max(1, iters // 4))
    dt2 = time.perf_counter() - t1
    return (dt - dt2) / (iters - max(1, iters // 4)), r["plan_ms"]


def cpu_reference_sample(d, iters):
    """Times `iters` iterations of the reference's run_jacobi_pcg on this host (1 thread: the
    reference has no threading).  Returns (seconds per iteration, kind, label)."""
    from oracle import oracle as O
    use_ref = O.reflib() is not None
    t0 = time.perf_counter()
    O.golden(d, 1e-300, iters, use_ref=use_ref)
    dt = time.perf_counter() - t0
    # one SpMV + setup are inside; per-iteration cost is the slope: time a second, shorter run
    t1 = time.perf_counter()
    O.golden(d, 1e-300, max(1, iters // 4), use_ref=use_ref)
    dt2 = time.perf_counter() - t1
    per_it = (dt - dt2) / (iters - max(1, iters // 4))
    setup = max(0.0, dt - per_it * iters)
    kind = "reference" if use_ref else "port"
    return per_it, setup, kind


def run_reference(args):
    world, rank, local, pg = dist_init(args)
    if rank != 0:
        return 0
    from project_xplus_b200 import generators as g
    d, _ = g.system_2d_large(args.grid)
    # iterations the reference's own solve needs on this system to reach 1e-8 (measured once in
    # full); other grids: the FP64 CG count scales with the grid side
    iters_needed = GOLDEN_ITERATIONS_1108 if args.grid == 1108 else round(GOLDEN_ITERATIONS_1108 * args.grid / 1108)
    samples = []
    for k in range(args.warmup + args.steps):
        per_it, setup, kind = cpu_reference_sample(d, args.cpu_sample_iters)
        if k >= args.warmup:
            samples.append(per_it * iters_needed + setup)
    t = statistics.median(samples)
    value = 1.0 / t
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args), "solver": "reference run_jacobi_pcg (FP64 CSR, 1 thread)",
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": 1, "kind": kind, "cpu_model": cpu_model(),
                             "sample": f"{args.cpu_sample_iters} iterations of run_jacobi_pcg per step on the full "
                                       f"system, extrapolated to {iters_needed} iterations"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------------------
# B200 arm
# --------------------------------------------------------------------------------------
def run_b200(args):
    import ctypes as C

    import torch

    world, rank, local, pg = dist_init(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import project_xplus_b200 as xp
    from project_xplus_b200 import _lib
    from project_xplus_b200 import generators as g

    d, xt = g.system_2d_large(args.grid)
    n = d.n
    # the library's first call in a process brings up its CUDA runtime and context (a one-time
    # cost, reported apart as first_call_ms); the first create of this system size then loads
    # the builder's kernels and grows the allocator (setup_first_ms); setup_ms is the create of
    # a process that has made one before, as a service that sees a new matrix per call runs it
    t_first = time.perf_counter()
    d0, _ = g.system_2d_small()
    xp.PcgSolver.from_dataset(d0, device=local).close()
    first_call_ms = (time.perf_counter() - t_first) * 1e3
    t_setup = time.perf_counter()
    # the workload's own storage: SELL-C-sigma with C = 32, sigma = 256 (compare.sort_window_1
    # times the same solve with sigma = 1)
    headline = dict(values_dtype="f32", vector_dtype="f32", chunk=4, sigma=256, device=local)
    xp.PcgSolver.from_dataset(d, **headline).close()
    setup_first_ms = (time.perf_counter() - t_setup) * 1e3
    # checks, SELL build and every device array, on the GPU: three creates, the fastest reported
    # (one create has read far above the others in a process now and then; all three are listed)
    setup_warm = []
    for k in range(3):
        t_setup = time.perf_counter()
        solver = xp.PcgSolver.from_dataset(d, **headline)
        setup_warm.append((time.perf_counter() - t_setup) * 1e3)
        if k < 2:
            solver.close()
    setup_ms = min(setup_warm)
    info = solver.info()
    # a real (non-default) stream: the library enqueues on exactly the stream the events see
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sp = C.c_void_p(stream.cuda_stream)
    b_dev = torch.from_numpy(d.b).to(dev)
    x_dev = torch.zeros(n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    hbm, hbm_kind = peaks()

    def one_solve():
        x_dev.zero_()
        _lib.check(_lib.lib.xplus_pcg_solve_device(solver.handle, b_dev.data_ptr(), x_dev.data_ptr(),
                                                   args.tol, _lib.XPLUS_TAU_REL_TRUE, 20000, sp))

    def metrics():
        m = _lib.XplusMetrics()
        _lib.check(_lib.lib.xplus_pcg_last_metrics(solver.handle, C.byref(m)))
        return m

    for _ in range(args.warmup):
        flush.fill_(1.0)
        one_solve()
        torch.cuda.synchronize()
    m0 = metrics()
    kernel_name = xp.solver.KERNEL_NAMES.get(int(m0.reserved[2]), "unknown")
    barrier(pg, dev)
    torch.cuda.synchronize()
    step_ms, kern_ms, iters, repls, relres = [], [], [], [], []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            one_solve()
            e1.record(stream)
            e1.synchronize()
            m = metrics()
            step_ms.append(e0.elapsed_time(e1))
            kern_ms.append(m.kernel_ms)
            iters.append(m.iterations)
            repls.append(m.replacements)
            relres.append(m.true_rel_residual)
            if m.status != 0:
                raise SystemExit(f"solve did not converge: status {m.status} res {m.true_rel_residual}")
    torch.cuda.synchronize()
    barrier(pg, dev)
    total_ms = sum(step_ms)
    total_ms_max = max_over_ranks(pg, total_ms, dev)
    value = world * args.steps / (total_ms_max / 1e3)
    ms_per_step = total_ms_max / args.steps

    # roofline of the persistent kernel: algorithmic bytes per launch / launch time
    nnz = info["nnz"]
    it_mean = statistics.mean(iters)
    rp_mean = statistics.mean(repls)
    bytes_iter = 8 * nnz + 52 * n
    bytes_repl = 12 * nnz + 28 * n
    bytes_launch = it_mean * bytes_iter + (rp_mean + 2) * bytes_repl
    kern_mean = statistics.mean(kern_ms)
    achieved = bytes_launch / (kern_mean / 1e3) / 1e9
    # the resident kernel keeps the matrix in L2 and the vectors in shared memory, so its bound
    # is per-iteration latency: microseconds per iteration and the phase clock of the last
    # timed solve (median CTA) say where they go
    us_per_iter = 1e3 * kern_mean / max(1.0, it_mean + rp_mean)
    ph = solver.phase_times()
    phase_us = [round(1e3 * v / max(1, iters[-1]), 2) for v in ph["median_ms"]]

    # SpMV alone: cold (L2 flushed before every launch) and warm (back to back), for the product
    # layout (row-sum form, FP32 off-diagonals, int16 offsets) and for the plain layout (FP32
    # values with the diagonal, int32 columns, 128-bit value and column loads)
    def measure_spmv(handle):
        xs = C.c_void_p()
        ys = C.c_void_p()
        _lib.check(_lib.lib.xplus_pcg_scratch_vectors(handle, C.byref(xs), C.byref(ys)))

        def spmv():
            _lib.check(_lib.lib.xplus_pcg_spmv_device(handle, xs, ys, sp))

        cold = []
        for k in range(23):
            flush.fill_(1.0)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            spmv()
            b.record(stream)
            b.synchronize()
            if k >= 3:
                cold.append(a.elapsed_time(b))
        for _ in range(5):
            spmv()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(100):
            spmv()
        b.record(stream)
        b.synchronize()
        return statistics.median(cold), a.elapsed_time(b) / 100

    spmv_bytes = info["spmv_bytes"]
    cold_ms, warm_ms = measure_spmv(solver.handle)
    spmv_cold_gbs = spmv_bytes / (cold_ms / 1e3) / 1e9
    spmv_warm_gbs = spmv_bytes / (warm_ms / 1e3) / 1e9
    plain = xp.PcgSolver.from_dataset(d, values_dtype="f32", vector_dtype="f32", chunk=4, row_sum_form=False,
                                      index16=False, keep_fp64=False, device=local)
    plain_bytes = plain.info()["spmv_bytes"]
    p_cold_ms, p_warm_ms = measure_spmv(plain.handle)
    plain.close()
    spmv_plain = {"cold_gbs": plain_bytes / (p_cold_ms / 1e3) / 1e9, "warm_gbs": plain_bytes / (p_warm_ms / 1e3) / 1e9,
                  "cold_ms": p_cold_ms, "warm_ms": p_warm_ms, "bytes": plain_bytes,
                  "frac_cold": plain_bytes / (p_cold_ms / 1e3) / 1e9 / hbm,
                  "layout": "fp32 values incl. diagonal, int32 columns, chunk 4 (128-bit value and column loads)"}

    # The same SpMV on the 128^3 3D system (n = 2.1M, ~15 nnz/row), whose matrix is larger than
    # L2 (126 MB), so back-to-back launches stream it from HBM: the kernel's bandwidth without
    # the fixed launch cost that dominates a single ~60 MB launch.
    spmv_large = None
    if not args.no_spmv3d:
        d3, _ = g.system_3d(128)
        spmv_large = {"workload": "3d-p1fem-128^3-sigma1.5", "n": d3.n, "nnz": d3.nnz}
        for name, kw in (("rowsum_int16", dict(values_dtype="f32", chunk=4)),
                         ("plain_int32", dict(values_dtype="f32", chunk=4, row_sum_form=False, index16=False))):
            s3 = xp.PcgSolver.from_dataset(d3, vector_dtype="f32", keep_fp64=False, device=local, **kw)
            b3 = s3.info()["spmv_bytes"]
            c_ms, w_ms = measure_spmv(s3.handle)
            spmv_large[name] = {"bytes": b3, "cold_ms": c_ms, "stream_ms": w_ms,
                                "cold_gbs": b3 / (c_ms / 1e3) / 1e9, "stream_gbs": b3 / (w_ms / 1e3) / 1e9,
                                "frac_stream": b3 / (w_ms / 1e3) / 1e9 / hbm}
            s3.close()
    # The 3D system as a mixed-precision workload: values in FP32, BF16 or FP16 (power-of-two
    # scale), FP32 inner PCG, FP64 residual replacement every 50 iterations or at a 1e-4 drop
    # of the recurrence residual, to 1e-10 FP64 true relative residual; FP64 for comparison.
    # 16-bit values run with the library defaults: two-term entries in cancelling rows and
    # flexible re-conjugation of the search direction at replacements.
    mixed_3d = None
    if not args.no_spmv3d and not args.no_compare:
        mixed_3d = {"workload": "3d-p1fem-128^3-sigma1.5, tol 1e-10 rel. FP64 true residual", "n": d3.n}
        for name, kw in (("f32_values", dict(values_dtype="f32", vector_dtype="f32")),
                         ("bf16_values", dict(values_dtype="bf16", vector_dtype="f32")),
                         ("f16_values", dict(values_dtype="f16", vector_dtype="f32")),
                         ("fp64", dict(values_dtype="f64", vector_dtype="f64", chunk=2))):
            s3 = xp.PcgSolver.from_dataset(d3, replace_every=50, replace_drop=1e-4, device=local, **kw)
            runs = []
            for _ in range(2):
                flush.fill_(1.0)
                torch.cuda.synchronize()
                runs.append(s3.solve(d3.b, None, tau=1e-10, tau_mode=_lib.XPLUS_TAU_REL_TRUE, max_iters=20000))
            r3 = runs[-1]
            mixed_3d[name] = {"time_to_tol_ms": r3.kernel_ms, "iterations": r3.iterations, "status": r3.status,
                              "replacements": r3.replacements, "true_rel_residual": r3.residual_rel,
                              "stagnated": r3.metrics["stagnated"], "kernel": r3.metrics["kernel"],
                              "slots": s3.info()["slots"]}
            s3.close()
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            # the reference's golden on this system, sampled on one core and extrapolated to the
            # FP64 GPU solve's iteration count (the golden's own count here was not measured)
            per_it3, setup3, kind3 = cpu_reference_sample(d3, 10)
            it3 = mixed_3d["fp64"]["iterations"]
            mixed_3d["cpu_reference"] = {
                "value_ms": (per_it3 * it3 + setup3) * 1e3, "cores": 1, "kind": kind3, "cpu_model": cpu_model(),
                "sample": f"10 iterations of run_jacobi_pcg (FP64, 1 thread) on the full system, "
                          f"{per_it3 * 1e3:.1f} ms/iteration, extrapolated to {it3} iterations (the FP64 GPU "
                          f"solve's count to 1e-10)"}
    if not args.no_spmv3d:
        del d3

    # end to end through the public host-array API (pinned host buffers)
    e2e = None
    if not args.no_e2e:
        b_host = torch.from_numpy(d.b).pin_memory()
        x_host = torch.empty(n, dtype=torch.float64).pin_memory()
        iters_c = C.c_int()
        mm = _lib.XplusMetrics()
        e2e_ms = []
        clk_e2e = Clocks(local, append=True).__enter__()
        for k in range(args.warmup + args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _lib.check(_lib.lib.xplus_pcg_solve(solver.handle, b_host.data_ptr(), None, args.tol,
                                                _lib.XPLUS_TAU_REL_TRUE, 20000, x_host.data_ptr(),
                                                C.byref(iters_c), None, 0, C.byref(mm)))
            dt = (time.perf_counter() - t0) * 1e3
            if k >= args.warmup:
                e2e_ms.append(dt)
        clk_e2e.__exit__(None, None, None)
        e2e_tot = max_over_ranks(pg, sum(e2e_ms), dev)
        e2e = {"value": world * args.steps / (e2e_tot / 1e3), "unit": "solves/s",
               "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n + 128,
               "ms_per_step": e2e_tot / args.steps}

    # The same solve with the straightforward FP32 kernel (a_ij rounded to FP32, int32 columns)
    # and in FP64: "plain Jacobi-PCG" of the metric, and the iteration count FP64 CG needs.
    compare = None
    fp64_iters = None
    if not args.no_compare:
        compare = {}
        for name, kw in (("plain_fp32", dict(values_dtype="f32", vector_dtype="f32", chunk=1, row_sum_form=False,
                                               index16=False)),
                         ("fp64", dict(values_dtype="f64", vector_dtype="f64", chunk=2))):
            s2 = xp.PcgSolver.from_dataset(d, device=local, **kw)
            flush.fill_(1.0)
            torch.cuda.synchronize()
            r2 = s2.solve(d.b, None, tau=args.tol, tau_mode=_lib.XPLUS_TAU_REL_TRUE, max_iters=40000)
            compare[name] = {"time_to_tol_ms": r2.kernel_ms, "iterations": r2.iterations, "status": r2.status,
                             "true_rel_residual": r2.residual_rel}
            if name == "fp64":
                fp64_iters = r2.iterations
            s2.close()
        # the headline solve with SELL sort window 1 instead of 256: on this matrix the window
        # saves no padding and scatters the rows of a slice, which costs the resident kernel's
        # shared-memory gathers bank conflicts (second of two solves)
        s2 = xp.PcgSolver.from_dataset(d, **dict(headline, sigma=1))
        for _ in range(2):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            r2 = s2.solve(d.b, None, tau=args.tol, tau_mode=_lib.XPLUS_TAU_REL_TRUE)
        compare["sort_window_1"] = {"time_to_tol_ms": r2.kernel_ms, "iterations": r2.iterations,
                                    "status": r2.status, "true_rel_residual": r2.residual_rel,
                                    "us_per_iteration": 1e3 * r2.kernel_ms / max(1, r2.iterations),
                                    "slots": s2.info()["slots"], "slots_sigma256": info["slots"]}
        s2.close()
        # M^-1 = G^T G: G from the learned network (shipped weights, inference on the GPU) and
        # the exact FSAI of the same pattern (host), both with the in-kernel Jacobi fallback
        from project_xplus_b200.learned import fsai_lower, load_weights
        params, _ = load_weights()
        for name in ("learned_gtg", "learned_gtg_bf16", "fsai_gtg"):
            # learned_gtg_bf16: the same learned G with the matrix values in BF16 (two-term
            # entries in cancelling rows), FP32 vectors, FP64 residual replacement
            kw3 = dict(values_dtype="bf16") if name == "learned_gtg_bf16" else {}
            s3 = xp.PcgSolver.from_dataset(d, device=local, **kw3)
            t0 = time.perf_counter()
            if name.startswith("learned_gtg"):
                s3.set_gnn(params, refine_sweeps=4)  # inference, refinement sweeps, rows normalized: on the GPU
            else:
                s3.set_gtg(fsai_lower(d.row_ptr, d.col_idx, d.values))
            pre_ms = (time.perf_counter() - t0) * 1e3  # preconditioner set-up on this handle
            runs = []
            for _ in range(2):
                flush.fill_(1.0)
                torch.cuda.synchronize()
                runs.append(s3.solve(d.b, None, tau=args.tol, tau_mode=_lib.XPLUS_TAU_REL_TRUE, max_iters=40000))
            r3 = runs[-1]
            compare[name] = {"time_to_tol_ms": r3.kernel_ms, "iterations": r3.iterations, "status": r3.status,
                             "refine_sweeps": 4 if name.startswith("learned_gtg") else None,
                             "true_rel_residual": r3.residual_rel, "setup_ms": pre_ms,
                             "time_to_tol_incl_setup_ms": r3.kernel_ms + pre_ms,
                             "jacobi_fallback_at": r3.metrics["jacobi_fallback_at"]}
            s3.close()
        compare["speedup_vs_plain_fp32"] = compare["plain_fp32"]["time_to_tol_ms"] / kern_mean
        compare["speedup_vs_fp64"] = compare["fp64"]["time_to_tol_ms"] / kern_mean
        for name in ("learned_gtg", "learned_gtg_bf16", "fsai_gtg"):
            compare[name]["speedup_vs_plain_fp32"] = compare["plain_fp32"]["time_to_tol_ms"] / compare[name]["time_to_tol_ms"]
        # the learned preconditioner against the headline Jacobi kernel in the same layout (row-sum
        # form, FP32, int16 columns: this line's own solve) and against FSAI of the same pattern
        compare["learned_vs_jacobi_same_layout"] = kern_mean / compare["learned_gtg"]["time_to_tol_ms"]
        compare["learned_vs_fsai"] = compare["fsai_gtg"]["time_to_tol_ms"] / compare["learned_gtg"]["time_to_tol_ms"]

    # CPU baseline: the reference's own golden on a bounded sample, rank 0 only, N=1 only
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        per_it, setup, kind = cpu_reference_sample(d, args.cpu_sample_iters)
        # the golden's own iteration count on this system (one full run, recorded beside
        # GOLDEN_ITERATIONS_1108), else the FP64 GPU solve's as a stand-in
        ref_iters = GOLDEN_ITERATIONS_1108 if args.grid == 1108 else (fp64_iters or it_mean)
        t_cpu = per_it * ref_iters + setup
        cup = cuper_reference_sample(d, 8)
        cpu = {"value": 1.0 / t_cpu, "unit": "solves/s", "cores": 1, "kind": kind, "cpu_model": cpu_model(),
               "cuper_pcg": None if cup is None else {
                   "ms_per_iteration": cup[0] * 1e3, "plan_ms": cup[1],
                   "note": "the reference's FP32-SpMV software PCG (run_cuper_pcg_solver), 8- and 2-iteration "
                           "samples on one core; per iteration only (its iteration count to 1e-8 not measured)"},
               "sample": f"{args.cpu_sample_iters} iterations of the reference run_jacobi_pcg (FP64, 1 thread) on "
                         f"the full system, extrapolated to {ref_iters:.0f} iterations (the golden's own "
                         f"iteration count to 1e-8 on this system); {per_it * 1e3:.1f} ms/iteration"}

    config0 = run_config0(args, local) if rank == 0 and not args.no_config0 else None

    # the batch runs after the single-system handle is gone: that handle keeps its matrix
    # persisting in L2, which the L2-resident batch would otherwise lose
    solver.close()
    batch = None if args.no_batch else run_batch(args, world, rank, pg, dev, stream, flush)

    clocks = clk.summary()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args, {"nnz": nnz}),
            "time_to_tol_ms": ms_per_step,
            "setup_ms": setup_ms, "time_to_tol_incl_setup_ms": ms_per_step + setup_ms,
            "first_call_ms": first_call_ms, "setup_first_ms": setup_first_ms, "setup_warm_ms_all": setup_warm,
            "iterations": it_mean, "replacements": rp_mean, "true_rel_residual": max(relres),
            "spmv": {"cold_gbs": spmv_cold_gbs, "warm_gbs": spmv_warm_gbs, "cold_ms": cold_ms, "warm_ms": warm_ms,
                     "bytes": spmv_bytes, "frac_cold": spmv_cold_gbs / hbm, "peak_kind": hbm_kind,
                     "layout": "row-sum form: fp32 off-diagonals + row sums, int16 column offsets, chunk 4",
                     "plain": spmv_plain, "large_3d": spmv_large},
            "mixed_3d": mixed_3d,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm,
                         "traffic": (RESIDENT1_DRAM_BYTES_PER_ITER * it_mean
                                     if kernel_name == "pcg_resident1_kernel" and args.grid == 1108 else None),
                         "traffic_note": "ncu DRAM bytes of a 100-iteration capture of this kernel on this system, "
                                         "scaled by the iterations of one launch; the matrix stays in L2 and the "
                                         "vectors in shared memory, so traffic is ~5% of the streaming model",
                         "memory_level": "L2-resident, not HBM: frac is the streaming model's bytes over "
                                         "the HBM copy peak; the kernel is bound by per-iteration latency",
                         "us_per_iteration": us_per_iter,
                         "phase_us_per_iteration": dict(zip(
                             ["publish_partials", "grid_barrier_and_totals", "update_and_halo", "spmv_and_records"]
                             if kernel_name == "pcg_resident1_kernel" else ["a", "b", "c", "d"], phase_us)),
                         "kernel": f"{kernel_name}<float,4,short> (FP32 values + vectors, row-sum form)",
                         "bytes_model": "8*nnz + 52*n per iteration (FP32 PCG) + 12*nnz + 28*n per FP64 residual",
                         "peak_kind": hbm_kind,
                         "bytes_per_launch": bytes_launch, "launch_ms": kern_mean},
            "compare": compare,
            "config0": config0,
            "batch": batch,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": 4 * args.steps,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


def run_config0(args, device):
    """The n = 1024 system (32x32 interior grid, sigma 1.0, x_true ~ U(-1,1) seed 0, x0 = 0) at
    the reference's own defaults (tau = 1e-10 on r.r, max_iters 0 -> max(4n, 1000),
    host/run_defaults.hpp:12-13), through three paths:
      gpu_persistent   xplus_pcg_solve: host arrays in and out, FP64 values and vectors, one
                       persistent launch per solve
      gpu_multikernel  the reference's host loop (archived/host/multi_kernel_solver.hpp:100-234)
                       driving this library's five C entry points (blocking calls, staged host arrays)
      cpu_reference    the reference's run_local_multi_kernel_solver and run_jacobi_pcg built from
                       its sources (oracle/_ref), one host thread (the reference has no threading)
    Each is timed over repeated full solves; x is checked against the golden's."""
    import project_xplus_b200 as xp
    from oracle import oracle as O
    from project_xplus_b200 import generators as g
    from project_xplus_b200 import kernels as K
    d, _ = g.system_2d_small()
    n, tau = d.n, 1e-10
    ref_lib = O.reflib()
    gold = O.golden(d, tau, use_ref=ref_lib is not None)
    out = {"workload": "2d-p1fem-32x32-sigma1 (n=1024), tau 1e-10 on r.r (the reference's run defaults)",
           "n": n, "nnz": d.nnz, "golden_iterations": gold["iterations"]}

    def timed(fn, reps, warm=3):
        for _ in range(warm):
            fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            r = fn()
        return (time.perf_counter() - t0) / reps, r

    s = xp.PcgSolver.from_dataset(d, values_dtype="f64", vector_dtype="f64", device=device)
    dt, r = timed(lambda: s.solve(d.b, d.x0, tau=tau), 50)
    s.close()
    out["gpu_persistent"] = {"solves_per_s": 1.0 / dt, "ms_per_solve": dt * 1e3, "iterations": r.iterations,
                             "kernel_ms": r.kernel_ms, "max_abs_diff_vs_golden": float(np.abs(r.solution - gold["x"]).max())}
    m_inv = 1.0 / d.extract_jacobi_diag()

    def mk_gpu():
        x = d.x0.copy()
        rr_, z, p, y = (np.zeros(n) for _ in range(4))
        met, dot = np.zeros(2), np.zeros(1)
        K.spmv_csr_kernel(d.row_ptr, d.col_idx, d.values, x, y, n)
        K.init_pcg_kernel(d.b, y, m_inv, rr_, z, p, met, n)
        rz, rr = met
        it = 0
        while it < max(4 * n, 1000) and rr > tau:
            K.spmv_csr_kernel(d.row_ptr, d.col_idx, d.values, p, y, n)
            K.dot_kernel(p, y, dot, n)
            alpha = rz / dot[0]
            K.update_xrz_kernel(x, p, rr_, y, m_inv, z, met, alpha, n)
            beta = met[0] / rz
            K.update_p_kernel(z, p, beta, n)
            rz, rr = met
            it += 1
        return it, x
    dt, (it, x) = timed(mk_gpu, 5, warm=1)
    out["gpu_multikernel"] = {"solves_per_s": 1.0 / dt, "ms_per_solve": dt * 1e3, "iterations": it,
                              "max_abs_diff_vs_golden": float(np.abs(x - gold["x"]).max()),
                              "calls_per_iteration": 5}
    if ref_lib is not None:
        import ctypes as C
        rp, ci, v = (np.ascontiguousarray(a) for a in (d.row_ptr, d.col_idx, d.values))
        xo = np.empty(n)
        it_c, st_c = C.c_int(), C.c_int()
        frr, res = C.c_double(), C.c_double()
        P = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731

        def mk_cpu():
            ref_lib.ref_multi_kernel(n, P(rp), P(ci), P(v), P(d.b), P(d.x0), C.c_double(tau), 0, P(xo),
                                     C.byref(it_c), C.byref(frr), C.byref(st_c), C.byref(res), None)
            return it_c.value
        dt, it = timed(mk_cpu, 200)
        dt_g, _ = timed(lambda: O.golden(d, tau, use_ref=True), 200)
        out["cpu_reference"] = {"multi_kernel": {"solves_per_s": 1.0 / dt, "ms_per_solve": dt * 1e3, "iterations": it,
                                                 "max_abs_diff_vs_golden": float(np.abs(xo - gold["x"]).max())},
                                "golden": {"solves_per_s": 1.0 / dt_g, "ms_per_solve": dt_g * 1e3},
                                "cores": 1, "kind": "reference", "cpu_model": cpu_model()}
    return out


def _golden_solve(payload):
    """One system solved by the reference's run_jacobi_pcg (oracle/_ref when built, else the
    port), tolerance on ||r|| relative to ||b||; returns (seconds, iterations)."""
    rp, ci, v, b, tol = payload
    from oracle import oracle as O
    from project_xplus_b200.solver import CsrDataset
    d = CsrDataset(rp, ci, v, b, np.zeros(len(b)))
    tau_rr = (tol * float(np.linalg.norm(b))) ** 2
    t0 = time.perf_counter()
    r = O.golden(d, tau_rr, 0, use_ref=O.reflib() is not None)
    return time.perf_counter() - t0, int(r["iterations"])


def batch_cpu_baseline(systems, works, tol, sample=24):
    """The reference's CPU solver on the batch, as independent single-thread processes on all
    host cores: a bounded sample of systems spread over the work range is solved in full and
    the total is extrapolated by the work estimate nnz * sqrt(n) of every system."""
    import multiprocessing as mp
    order = np.argsort(works)
    pick = [int(order[int(i)]) for i in np.linspace(0, len(order) - 1, min(sample, len(order)))]
    cores = os.cpu_count() or 1
    payloads = [(systems[k].row_ptr, systems[k].col_idx, systems[k].values, systems[k].b, tol) for k in pick]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(min(cores, len(payloads))) as pool:
        res = pool.map(_golden_solve, payloads)
    wall = time.perf_counter() - t0
    per_work = sum(t for t, _ in res) / sum(works[k] for k in pick)
    total_cpu_s = per_work * sum(works)
    est_wall = total_cpu_s / cores
    return {"value": len(systems) / est_wall, "unit": "systems/s", "cores": cores, "kind": "reference",
            "cpu_model": cpu_model(),
            "sample": f"{len(pick)} of {len(systems)} systems (spread over the work range) solved by the reference "
                      f"run_jacobi_pcg, one process per core; total CPU time {total_cpu_s:.1f} s extrapolated by "
                      f"nnz*sqrt(n), divided over {cores} cores (sample wall {wall:.1f} s)"}


def run_batch(args, world, rank, pg, dev, stream, flush):
    """The batched workload: 512 2D P1-FEM systems, grid side log-uniform in [45, 256] and
    conductivity sigma log-uniform in [0.5, 2.5] (seeded), FP32 values and vectors, 1e-8 FP64
    true relative residual each, one graph-captured persistent launch per step.  With N ranks
    the systems are split by estimated work (no collective); the time is the max over ranks."""
    import torch

    from project_xplus_b200 import generators as g
    from project_xplus_b200.batch import BatchSolver, shard_systems, system_work
    sides, sigmas = g.batch_sides(512, 45, 256, seed=3)
    works = [system_work(int(sd) ** 2, 7 * int(sd) ** 2) for sd in sides]
    mine = shard_systems(works, world, rank)
    systems = [g.fem2d(int(sides[k]), sigma=float(sigmas[k]), seed=1000 + k, x_seed=1000 + k)[0] for k in mine]
    s = BatchSolver([(d.row_ptr, d.col_idx, d.values) for d in systems], values_dtype="f32")
    b = torch.from_numpy(np.concatenate([d.b for d in systems])).to(dev)
    x = torch.zeros_like(b)
    torch.cuda.synchronize()
    # one solve, then the launch shape tuned on this right-hand side (full solves)
    s.solve_device(b, x, tau=args.tol, stream=stream)
    stream.synchronize()
    tune = s.autotune(iters=0, tau=args.tol)
    info = s.info()
    for _ in range(args.warmup):
        x.zero_()
        s.solve_device(b, x, tau=args.tol, stream=stream)
        stream.synchronize()
    barrier(pg, dev)
    ms = []
    clk = Clocks(dev.index, append=True).__enter__()
    for _ in range(args.steps):
        flush.fill_(1.0)
        x.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.solve_device(b, x, tau=args.tol, stream=stream)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    clk.__exit__(None, None, None)
    r = s.results()
    if not np.all(r["status"] == 0):
        raise SystemExit(f"batch: {int((r['status'] != 0).sum())} systems did not converge")
    tot = max_over_ranks(pg, sum(ms), dev)
    staged = s.staged()
    # the same launch shape with every band's matrix read from global memory (one step; the
    # same x bit for bit)
    unstaged_ms = None
    if info["resident"]["on"]:
        s.set_stage_matrix(False)
        x.zero_()
        s.solve_device(b, x, tau=args.tol, stream=stream)
        stream.synchronize()
        flush.fill_(1.0)
        x.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.solve_device(b, x, tau=args.tol, stream=stream)
        e1.record(stream)
        e1.synchronize()
        unstaged_ms = max_over_ranks(pg, e0.elapsed_time(e1), dev)
    s.close()
    # the same batch with BF16 values (the other value type of the batched workload), with its
    # own tuned kernel and launch shapes
    s16 = BatchSolver([(d.row_ptr, d.col_idx, d.values) for d in systems], values_dtype="bf16")
    x.zero_()
    s16.solve_device(b, x, tau=args.tol, stream=stream)
    stream.synchronize()
    tune16 = s16.autotune(iters=0, tau=args.tol)
    info16 = s16.info()
    for _ in range(args.warmup):
        x.zero_()
        s16.solve_device(b, x, tau=args.tol, stream=stream)
        stream.synchronize()
    ms16 = []
    clk = Clocks(dev.index, append=True).__enter__()
    for _ in range(args.steps):
        flush.fill_(1.0)
        x.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s16.solve_device(b, x, tau=args.tol, stream=stream)
        e1.record(stream)
        e1.synchronize()
        ms16.append(e0.elapsed_time(e1))
    clk.__exit__(None, None, None)
    r16 = s16.results()
    tot16 = max_over_ranks(pg, sum(ms16), dev)
    staged16 = s16.staged()
    s16.close()
    bf16 = {"value": len(sides) * args.steps / (tot16 / 1e3), "unit": "systems/s", "ms_per_step": tot16 / args.steps,
            "converged": int((r16["status"] == 0).sum()), "iterations_total": int(r16["iterations"].sum()),
            "max_true_rel_residual": float(r16["true_rel"].max()),
            "system_ms_max": float(r16["system_ms"].max()),
            "launch": {"cluster": info16["cluster"], "block_threads": info16["block_threads"],
                       "grid": info16["grid"], "autotune_ms": tune16["ms"],
                       "largest_systems_lane": info16["split_lane"], "resident": info16["resident"],
                       "matrix_staged_systems": staged16["all"], "matrix_staged_partly": staged16["some"]}}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = batch_cpu_baseline(systems, [works[k] for k in mine], args.tol)
    return {"cpu_baseline": cpu, "workload": "512 x 2d-p1fem, side log-uniform [45,256], sigma log-uniform [0.5,2.5], fp32, tol 1e-8",
            "systems": len(sides), "sum_n": int(sum(int(sd) ** 2 for sd in sides)),
            "value": len(sides) * args.steps / (tot / 1e3), "unit": "systems/s", "ms_per_step": tot / args.steps,
            "scaling": "strong (systems split over ranks)", "iterations_total": int(r["iterations"].sum()),
            "iterations_max": int(r["iterations"].max()), "max_true_rel_residual": float(r["true_rel"].max()),
            "system_ms": {"max": float(r["system_ms"].max()), "median": float(np.median(r["system_ms"])),
                          "sum": float(r["system_ms"].sum())},
            "launch": {"cluster": info["cluster"], "block_threads": info["block_threads"], "grid": info["grid"],
                       "autotune_ms": tune["ms"], "largest_systems_lane": info["split_lane"],
                       "resident": info["resident"], "matrix_staged_systems": staged["all"],
                       "matrix_staged_partly": staged["some"], "ms_matrix_not_staged": unstaged_ms},
            "graph": True, "bf16_values": bf16}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
