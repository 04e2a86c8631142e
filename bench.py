#!/usr/bin/env python
"""Benchmark: unwrapped Mpx/s of the B200 DCT+IRLS L1 unwrapper.

Workload (one "step" = one full unwrap, function-default iteration parameters
max_iter=50, tol=1e-3, cg_max_iter=20, cg_tol=1e-4, epsilon=1e-2):
  g2_4096   4096 x 4096 float32 grid, G2 generator (Gaussian + ramp truth, 3*pi
            fault, noise 0.6 rad, Beta(2,2) coherence, 5% NaN ellipses), seed 0.
            Seeded synthetic input standing in for the reference's benchmark data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
    torchrun --nproc-per-node N bench.py --gpus N ...   (one replica per GPU)

Printed JSON (rank 0, one line):
  value      Mpx/s with inputs resident in HBM (C ABI on device pointers),
             K solves timed with CUDA events, max over ranks, barrier both sides;
  e2e        same metric through the public API irls_unwrap_2d with numpy input
             and numpy output (H2D + D2H inside the timed region);
  roofline   dominant kernel's algorithmic bytes / its mean CUDA-event launch
             time inside the timed region, against MEASURED_PEAKS.json hbm_gbs;
  cpu_baseline  the numpy oracle on the GPU host's cores, bounded sample;
  clocks     nvidia-smi samples taken during the timed region;
  accuracy   cycle-map match and RMS of the output against the reference's own
             FP64 and FP32 runs of the bench grid (committed fixtures).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

FN = dict(max_iter=50, tol=1e-3, cg_max_iter=20, cg_tol=1e-4, epsilon=1e-2, conncomp_size=30)
METRIC = "unwrapped Mpx/s (4096^2 fault grid, function-default iterations)"


def metric_name(shape_arg):
    """The metric label of the workload run: the 4096^2 fault grid by default, else the
    --shape grid of the smooth generator."""
    if shape_arg is None:
        return METRIC
    return f"unwrapped Mpx/s ({int(shape_arg[0])}x{int(shape_arg[1])} smooth grid, function-default iterations)"
UNIT = "Mpx/s"

# Algorithmic HBM bytes per pixel per launch of each kernel family (float32 words,
# halo re-reads and reduction partials not counted).
ALG_BYTES = {
    "matvec": 16.0,    # read p, wIx, wIy; write Ap
    "row_upd": 28.0,   # read x, p, r, Ap; write x, r, T
    "col": 8.0,        # read T; write T
    "row_inv": 12.0,   # read T, p; write p (p = z + beta p in place)
    "head": 40.0,      # read u, gx, gy, wx, wy; write u, wIx, wIy, b (+ halo)
    "row_r0": 24.0,    # read b, x, wIx, wIy; write r, T
}


def load_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms (background process)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus):
    """torchrun env -> (rank, world, local_rank); initialises NCCL when world > 1."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier_max(x, world, local):
    """Barrier, then the max of a float over ranks."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=torch.device("cuda", local))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def make_input(seed=0, shape=None):
    """The 4096^2 G2 fault grid, or a G1 grid of the given (H, W) (seed + 1)."""
    if shape:
        from core_b200.synthetic import gen_g1
        p, c, _ = gen_g1(int(shape[0]), int(shape[1]), seed=seed + 1)
        return p, c
    from core_b200.synthetic import gen_g2
    p, c, _ = gen_g2(4096, seed=seed)
    return p, c


def workload_name(shape):
    return f"g1_{shape[0]}x{shape[1]} fn-defaults" if shape else "g2_4096 fn-defaults"


# --------------------------------------------------------------------------- CPU baseline
def cpu_sample(p, c, n_irls, workers):
    """The oracle on a bounded sample of the workload: the setup + DCT initial
    solve + post-processing (max_iter=0) and one IRLS iteration of 20 PCG steps;
    the full-solve time is extrapolated as t0 + n_irls * (t1 - t0), n_irls being
    the IRLS count of the same solve (identical algorithm)."""
    from oracle.irls_oracle import irls_unwrap_2d as oracle
    kw = dict(FN)
    t = time.perf_counter()
    oracle(p, c, workers=workers, **dict(kw, max_iter=0))
    t0 = time.perf_counter() - t
    t = time.perf_counter()
    oracle(p, c, workers=workers, **dict(kw, max_iter=1, tol=0.0))
    t1 = time.perf_counter() - t
    full = t0 + n_irls * max(t1 - t0, 0.0)
    return t0, t1, full


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_irls_count(p, c, shape, workers):
    """IRLS iterations of the full solve of this workload: the reference function's own
    float32 run of the 4096^2 fault grid (stored with its cycle map in
    tests/golden/L_g2_4096_fn_fp32.npz); for other shapes, one full oracle solve."""
    if shape is None:
        f = os.path.join(REPO, "tests", "golden", "L_g2_4096_fn_fp32.npz")
        if os.path.exists(f):
            return int(np.load(f)["iters"]), "the reference function's own float32 run of this grid"
    from oracle.irls_oracle import OracleStats, irls_unwrap_2d as oracle
    st = OracleStats()
    oracle(p, c, workers=workers, stats=st, **FN)
    return int(st.irls_iters), "a full oracle solve of this grid"


def run_reference(args):
    """--impl reference: the reference's CPU path, restated by the oracle, on the host cores.

    One step = one IRLS iteration (20 PCG iterations, the same array work as every IRLS
    iteration of the full solve) of the workload's solve, timed on the host clock; the
    setup + DCT initial solve + post-processing is timed once beforehand.  `ms_per_step`
    is that measured step time.  `value` is in the GPU arm's unit, Mpx of full solves per
    second: grid pixels / (setup-and-post time + IRLS count x median step time), the IRLS
    count being that of the reference's own run of the same grid."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import scipy.fft
    workers = os.cpu_count()
    p, c = make_input(shape=args.shape)
    npx = p.size
    n_irls, n_src = reference_irls_count(p, c, args.shape, workers)
    from oracle.irls_oracle import irls_unwrap_2d as oracle
    t = time.perf_counter()
    oracle(p, c, workers=workers, **dict(FN, max_iter=0))
    t0 = time.perf_counter() - t
    samples = []
    for i in range(args.warmup + args.steps):
        t = time.perf_counter()
        oracle(p, c, workers=workers, **dict(FN, max_iter=1, tol=0.0))
        dt = time.perf_counter() - t
        if i >= args.warmup:
            samples.append(max(dt - t0, 1e-9))
    t_irls = float(np.median(samples))
    full = t0 + n_irls * t_irls
    value = npx / 1e6 / full
    sample = (f"per step: one IRLS iteration (20 PCG) of the {p.shape[0]}x{p.shape[1]} solve, measured "
              f"{t_irls:.2f} s (median of {args.steps}); setup + DCT init + post measured once {t0:.2f} s; "
              f"full solve = {t0:.1f} + {n_irls} x {t_irls:.2f} = {full:.0f} s, {n_irls} IRLS iterations "
              f"from {n_src}")
    cpu = {"value": value, "unit": UNIT, "cores": workers, "kind": "port", "sample": sample,
           "cpu_model": cpu_model(), "os_cpu_count": os.cpu_count(), "scipy_fft_workers": workers,
           "numpy_threads_note": "the oracle's FFTs run on scipy.fft with workers=cores; its elementwise "
                                 "numpy work is single-threaded"}
    out = {"metric": metric_name(args.shape), "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": t_irls * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
           "config": workload_config(p.shape, args.shape, args.gpus),
           "full_solve_s_extrapolated": full, "irls_iters_full_solve": n_irls,
           "step_definition": "one IRLS iteration of the full solve (ms_per_step is measured; value "
                              "extrapolates to the full solve)",
           "cpu_baseline": cpu,
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


def workload_config(grid_shape, shape_arg, n_gpus):
    """The `config` both arms print (identical for the same workload)."""
    return {"workload": workload_name(shape_arg), "grid": [int(grid_shape[0]), int(grid_shape[1])],
            "params": FN, "parallelism": f"replicas x{n_gpus}"}


# --------------------------------------------------------------------------- GPU arm
def run_b200(args):
    import torch

    import core_b200
    from core_b200 import _lib
    from core_b200.irls import make_params, precision_flags

    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    p, c = make_input(seed=rank, shape=args.shape)
    H, W = p.shape
    npx = H * W

    ph = torch.from_numpy(p).to(dev)
    wt = torch.from_numpy(c).to(dev)
    out_u = torch.empty((H, W), dtype=torch.float32, device=dev)
    out_cc = torch.empty((H, W), dtype=torch.int16, device=dev)
    ws = torch.empty(lib.unw_workspace_bytes(H, W), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    base_flags = precision_flags(args.precision, args.col_pass)

    def solve(flags=0, **over):
        prm = make_params(**dict(FN, **over))
        prm.flags |= flags | base_flags
        st = _lib.UnwStats()
        rc = lib.unw_solve_f32(ph.data_ptr(), W, wt.data_ptr(), W, H, W, C.byref(prm), out_u.data_ptr(), W,
                               out_cc.data_ptr(), W, ws.data_ptr(), ws.numel(), C.byref(st), stream.cuda_stream)
        _lib.check(rc, "unw_solve_f32")
        return st

    for _ in range(args.warmup):
        solve()
    torch.cuda.synchronize()

    # ---- device-resident timed region: the product path, no per-launch events
    clocks = ClockSampler(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    stats = None
    for _ in range(args.steps):
        stats = solve().as_dict()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    t_dev = ev0.elapsed_time(ev1) / 1e3
    t_dev = barrier_max(t_dev, world, local)
    value = world * npx * args.steps / 1e6 / t_dev

    # ---- the mixed-precision form on the same grid (BASELINE's "mixed vs plain" metric), and
    # the plain form without CUDA graphs (every launch issued from the host, as the
    # reference's eager loop does); same K steps, CUDA events
    def timed(flags, k):
        for _ in range(2):
            solve(flags)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(k):
            st_ = solve(flags)
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / 1e3 / k, st_
    k_alt = max(1, min(args.steps, 5))
    t_mixed, st_mixed = timed(_lib.UNW_F_MIXED, k_alt)
    t_nograph, _ = timed(_lib.UNW_F_NO_GRAPH, k_alt)
    mixed = {"value": round(npx / 1e6 / t_mixed, 3), "unit": UNIT, "ms_per_step": round(t_mixed * 1e3, 3),
             "col_path": int(st_mixed.col_path), "resid_rel": float(f"{st_mixed.resid_rel:.3g}"),
             "ratio_mixed_over_plain": round(t_dev / args.steps / t_mixed, 4),
             "plain_no_graph": {"value": round(npx / 1e6 / t_nograph, 3), "ms_per_step": round(t_nograph * 1e3, 3)},
             "note": (f"H = {H} > 1024: the mixed form keeps the float32 FFT column pass (the tensor-core "
                      "pass covers grids of at most 1024 rows); see mixed_1024 for where it applies")
             if H > 1024 else "H <= 1024: the autotuner chose col_path (0 FFT, 1 tensor cores)"}

    # ---- per-kernel CUDA-event times (UNW_F_PROFILE brackets every launch with an event
    # pair on the solve stream; the events add about 10 us per launch, so this timed pass
    # is kept apart from the one that gives `value`)
    prof_steps = max(1, min(args.steps, 2))
    prof_ms = np.zeros(_lib.PROF_N)
    prof_n = np.zeros(_lib.PROF_N, dtype=np.int64)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(prof_steps):
        st = solve(_lib.UNW_F_PROFILE)
        prof_ms += np.array(st.prof_ms[:_lib.PROF_N])
        prof_n += np.array(st.prof_launches[:_lib.PROF_N])
    ev1.record(stream)
    torch.cuda.synchronize()
    t_prof = ev0.elapsed_time(ev1) / 1e3 / prof_steps

    # ---- end to end through the public API as a numpy caller uses it: numpy (pageable)
    # input copied to the device (through the API's pinned staging) and numpy output copied
    # back inside the timed region
    # warm-up in the timed loop's own pattern: a caller that keeps the previous
    # result while the next call runs holds two pinned output blocks
    pkw = dict(precision=args.precision, col_pass=args.col_pass)
    for _ in range(2):
        u_np, cc_np = core_b200.irls_unwrap_2d(p, c, device=dev, **FN, **pkw)
    torch.cuda.synchronize()
    barrier(world)
    e2e_steps = max(1, min(args.steps, 3))
    t = time.perf_counter()
    ev0.record(stream)
    for _ in range(e2e_steps):
        u_np, cc_np = core_b200.irls_unwrap_2d(p, c, device=dev, **FN, **pkw)
    ev1.record(stream)
    torch.cuda.synchronize()
    t_e2e = max(ev0.elapsed_time(ev1) / 1e3, time.perf_counter() - t)
    barrier(world)
    t_e2e = barrier_max(t_e2e, world, local)
    e2e = world * npx * e2e_steps / 1e6 / t_e2e

    # ---- accuracy of this run's output against the reference's own runs of the same grid
    # (committed fixtures: full 2-pi cycle map + unwrapped phase on a sub-sampled lattice)
    accuracy = accuracy_vs_reference(p, u_np) if (rank == 0 and args.shape is None) else None
    if accuracy:
        # the same grid at the reference run's own IRLS count (tol = 0, max_iter = that count;
        # cg_tol and the numerical breaks as usual): on this grid rel_change at the 29th
        # iteration is within about 1% of tol, so the natural stop can differ by one iteration
        n_ref = reference_irls_count(p, c, None, 1)[0]
        st_same = solve(0, max_iter=n_ref, tol=0.0)
        torch.cuda.synchronize()
        acc_same = accuracy_vs_reference(p, out_u.cpu().numpy())
        accuracy["natural_stop_irls_iters"] = stats["irls_iters"]
        accuracy["reference_irls_iters"] = n_ref
        accuracy["same_irls_iters"] = {"irls_iters": st_same.irls_iters, **(acc_same or {})}

    # ---- roofline of the dominant kernel (live event times from the timed region)
    names = _lib.PROF_NAMES
    peak, peak_kind = load_peaks()
    fam = {names[i]: (prof_ms[i], prof_n[i]) for i in range(len(names))}
    dom = max(ALG_BYTES, key=lambda k: fam[k][0])
    ms, n = fam[dom]
    per_launch_s = ms / 1e3 / max(n, 1)
    achieved = ALG_BYTES[dom] * npx / per_launch_s / 1e9
    kernels = {}
    for k in ALG_BYTES:
        kms, kn = fam[k]
        if kn:
            kernels[k] = {"launches": int(kn), "ms_total": round(float(kms), 3),
                          "us_per_launch": round(float(kms) / kn * 1e3, 2),
                          "gbs": round(ALG_BYTES[k] * npx / (kms / 1e3 / kn) / 1e9, 1)}
    pcg_ms = sum(fam[k][0] for k in ("matvec", "row_upd", "col", "row_inv"))
    pcg_bpx = sum(ALG_BYTES[k] for k in ("matvec", "row_upd", "col", "row_inv"))
    n_pcg = max(int(fam["matvec"][1]), 1)
    traffic = None
    tf = os.path.join(REPO, "profiles", "traffic.json")
    if os.path.exists(tf):
        traffic = json.load(open(tf)).get(dom)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "kernel": dom,
                "peak_source": peak_kind,
                "alg_bytes_per_launch": ALG_BYTES[dom] * npx,
                "pcg_iteration": {"us": round(pcg_ms / n_pcg * 1e3, 1), "alg_bytes_per_px": pcg_bpx,
                                  "gbs": round(pcg_bpx * npx / (pcg_ms / 1e3 / n_pcg) / 1e9, 1)},
                "kernels": kernels,
                "timing": f"per-launch CUDA events on the solve stream over a separate timed pass of "
                          f"{prof_steps} step(s) ({t_prof * 1e3:.1f} ms/step with the events)"}

    # column pass: bound by instruction issue, not memory -> also its issue-rate roofline
    # (warp instructions per launch from the ncu capture in profiles/, peak = 4 issue slots
    # per SM per cycle at the sampled SM clock)
    if os.path.exists(tf):
        inst = json.load(open(tf)).get("inst", {}).get("col")
        if inst and fam["col"][1]:
            col_s = fam["col"][0] / 1e3 / fam["col"][1]
            sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
            peak_i = 148 * 4 * sm_mhz * 1e6 / 1e9
            roofline["col_issue"] = {"bound": "issue", "kernel": "col", "unit": "Ginst/s (warp)",
                                     "inst_per_launch": inst, "achieved": round(inst / col_s / 1e9, 1),
                                     "peak": round(peak_i, 1), "frac": round(inst / col_s / 1e9 / peak_i, 4)}

    # ---- the 64-grid uneven stack (the other workload of the headline metric), sharded by grid
    stack = None
    if not args.no_stack_line:
        mine, sph, swt, s_npx = stack_grids(64, rank, world)
        pos = [mine.index(m) for m in (0, 1, 2) if m in mine]
        s_prof = {}
        s_val, s_t, s_iters, s_out, _ = stack_measure(sph, swt, 3, 2, world, local, s_npx, keep_out=pos,
                                                      profile_out=s_prof)
        m_val, m_t, _, _, m_paths = stack_measure(sph, swt, 1, 2, world, local, s_npx, flags=_lib.UNW_F_MIXED)
        # equal work per pixel on both workloads: 3 IRLS x 20 PCG iterations, every stop test off
        f_val, f_t, _, _, _ = stack_measure(sph, swt, 1, 2, world, local, s_npx, flags=_lib.UNW_F_FIXED_ITERS,
                                            over={"max_iter": 3})
        for _ in range(2):
            solve(_lib.UNW_F_FIXED_ITERS, max_iter=3)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(3):
            solve(_lib.UNW_F_FIXED_ITERS, max_iter=3)
        ev1.record(stream)
        torch.cuda.synchronize()
        g_fixed = npx / 1e6 / (ev0.elapsed_time(ev1) / 1e3 / 3)
        stack = {"value": round(s_val, 3), "unit": UNIT, "ms_per_step": round(s_t * 1e3, 1), "steps": 2,
                 "warmup": 3, "grids": 64, "total_mpx": round(s_npx / 1e6, 1),
                 "workload": "64 G1 grids, rows U[1500,2600] x cols U[4000,7000], noise U[0.2,0.8], "
                             "function defaults, one batched solve per step, inputs resident in HBM",
                 "parallelism": f"grids sharded over {world} GPU(s)",
                 "mixed": {"value": round(m_val, 3), "ms_per_step": round(m_t * 1e3, 1),
                           "ratio_mixed_over_plain": round(m_val / s_val, 4),
                           "tensor_core_grids": int(sum(m_paths)),
                           "note": "every stack grid has more than 1024 rows, so the mixed form keeps the "
                                   "float32 FFT column pass (the tensor-core pass covers H <= 1024)"},
                 "kernels": {"note": "per-launch CUDA-event times of one separately profiled batched solve of "
                                     "this rank's grids (launch groups one after another; the timed steps run "
                                     "them concurrently)", **s_prof},
                 "fixed_iters_3x20": {"stack_mpx_s": round(f_val, 3), "stack_ms_per_step": round(f_t * 1e3, 1),
                                      "single_grid_mpx_s": round(g_fixed, 3),
                                      "note": "both workloads at exactly 3 IRLS x 20 PCG iterations (stop tests "
                                              "off): per-pixel work is equal, so the two Mpx/s compare the "
                                              "launch shapes (Bluestein stack grids vs the power-of-two 4096^2 "
                                              "grid) rather than iteration counts"},
                 "accuracy": stack_accuracy({mine[k]: s_out[k] for k in s_out}, sph, mine) if rank == 0 else None}
        del sph, swt

    # ---- component linking after the unwrap (Stack.unwrap2d's default path)
    link = None
    if not args.no_link_line:
        link = link_measure(local, 5, 2)

    # ---- CPU baseline (rank 0, N=1 only): the oracle on a bounded sample
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        workers = os.cpu_count()
        t0, t1, full = cpu_sample(p, c, stats["irls_iters"], workers)
        cpu = {"value": round(npx / 1e6 / full, 5), "unit": UNIT, "cores": workers, "kind": "port",
               "sample": (f"oracle (numpy/scipy.fft, {workers} threads) on the same 4096^2 input: "
                          f"max_iter=0 run {t0:.1f}s + one IRLS iteration (20 PCG) {t1 - t0:.1f}s, "
                          f"extrapolated to {stats['irls_iters']} IRLS iterations = {full:.0f}s")}

    launches = int(prof_n.sum()) // prof_steps * args.steps  # same deterministic launch sequence per step
    out = {"metric": metric_name(args.shape), "value": round(value, 3), "unit": UNIT, "n_gpus": world,
           "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(t_dev / args.steps * 1e3, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": dict(workload_config((H, W), args.shape, world),
                          step="one full unwrap per step, one replica per GPU",
                          precision=args.precision, col_pass=args.col_pass,
                          irls_iters=stats["irls_iters"], pcg_iters=stats["cg_iters_total"],
                          l2="inputs 134 MB and solver working set ~1.1 GB exceed the 126 MB L2"),
           "e2e": {"value": round(e2e, 3), "unit": UNIT, "h2d_bytes_per_step": int(npx * 8),
                   "d2h_bytes_per_step": int(npx * 6),
                   "path": "core_b200.irls_unwrap_2d(numpy phase, numpy weight) -> numpy (u, conncomp); "
                           "pageable numpy input sent through chunked pinned staging, pinned staging "
                           "for the output"},
           "roofline": roofline, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches // 1,
           "stack": stack, "link": link, "accuracy": accuracy, "mixed": mixed,
           "mixed_1024": mixed_small(local) if not args.no_mixed_small else None,
           "diff": diff_measure(local, args.diff_large) if not args.no_diff_line else None}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def accuracy_vs_reference(p, u):
    """Cycle-map match and RMS (after mean removal, on the fixture's lattice) of the
    4096^2 fault-grid output against the reference function's FP64 and FP32 runs of
    the same input (tests/golden/L_g2_4096_fn_fp64.npz, L_g2_4096_fn_fp32.npz)."""
    out = {}
    v = np.isfinite(p)
    k = np.zeros(p.shape, np.int16)
    k[v] = np.round((u[v].astype(np.float64) - p[v].astype(np.float64)) / (2 * np.pi)).astype(np.int16)
    for prec in ("fp64", "fp32"):
        f = os.path.join(REPO, "tests", "golden", f"L_g2_4096_fn_{prec}.npz")
        if not os.path.exists(f):
            continue
        d = np.load(f)
        if tuple(d["cycles"].shape) != p.shape:
            continue
        s = int(d["step"])
        vs = v[::s, ::s]
        e = (u[::s, ::s].astype(np.float64) - d["u_sub"].astype(np.float64))[vs]
        out[f"vs_reference_{prec}"] = {
            "cycle_match": round(float((k == d["cycles"])[v].mean()), 6),
            "rms_rad": float(f"{np.sqrt(np.mean((e - e.mean()) ** 2)):.3g}"),
            "lattice": f"every {s}th row and column ({int(vs.sum())} valid pixels)"}
    return out or None


def stack_accuracy(outs, phases, mine):
    """Stack members 0-2 against the reference function's FP32 (cycle map) and FP64 runs
    (tests/golden/L_stack{m}_fn_fp{32,64}.npz)."""
    res = {}
    for m, u in sorted(outs.items()):
        p = phases[mine.index(m)]
        f32 = os.path.join(REPO, "tests", "golden", f"L_stack{m}_fn_fp32.npz")
        f64 = os.path.join(REPO, "tests", "golden", f"L_stack{m}_fn_fp64.npz")
        if not (os.path.exists(f32) and os.path.exists(f64)):
            continue
        d32, d64 = np.load(f32), np.load(f64)
        v = np.isfinite(p)
        k = np.zeros(p.shape, np.int16)
        k[v] = np.round((u[v].astype(np.float64) - p[v].astype(np.float64)) / (2 * np.pi)).astype(np.int16)
        s = int(d32["step"])
        vs = v[::s, ::s]
        e = {}
        for nm, d in (("fp64", d64), ("fp32", d32)):
            x = (u[::s, ::s].astype(np.float64) - d["u_sub"].astype(np.float64))[vs]
            e[nm] = float(f"{np.sqrt(np.mean((x - x.mean()) ** 2)):.3g}")
        res[f"grid{m}"] = {"shape": list(p.shape), "cycle_match_vs_fp32": round(float((k == d32["cycles"])[v].mean()), 6),
                           "rms_rad_vs_fp64": e["fp64"], "rms_rad_vs_fp32": e["fp32"]}
    return res or None


def mixed_small(local):
    """The mixed-precision form where it applies (grids of <= 1024 rows): the 1024^2 G1 grid
    of the reference's fixtures, a batch of 16 such grids (the differentiable-unwrap batch
    shape) and 64 tiles of 256^2 (a tiled unwrap), plain vs mixed (autotuned) vs mixed with
    the tensor-core pass forced, device-resident inputs, CUDA events; error of the 1024^2
    grid against the reference's FP64 run."""
    import torch

    from core_b200 import _lib
    from core_b200.irls import make_params
    from core_b200.synthetic import gen_g1
    lib = _lib.load()
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    out = {}
    d64 = os.path.join(REPO, "tests", "golden", "L_g1_1024_fn_fp64.npz")
    for label, count, side in (("g1_1024", 1, 1024), ("batch16_g1_1024", 16, 1024), ("tiles64_g1_256", 64, 256)):
        grids = [gen_g1(side, side, seed=k) for k in range(count)]
        n = len(grids)
        arr = (_lib.UnwGrid * n)()
        keep = []
        Hs, Ws = (C.c_int64 * n)(), (C.c_int64 * n)()
        for k, (p, c, _) in enumerate(grids):
            ph, wt = torch.from_numpy(p).to(dev), torch.from_numpy(c).to(dev)
            ou = torch.empty((side, side), dtype=torch.float32, device=dev)
            oc = torch.empty((side, side), dtype=torch.int16, device=dev)
            keep += [ph, wt, ou, oc]
            arr[k] = _lib.UnwGrid(ph.data_ptr(), side, wt.data_ptr(), side, side, side, ou.data_ptr(), side,
                                  oc.data_ptr(), side)
            Hs[k] = Ws[k] = side
        ws = torch.empty(lib.unw_batch_workspace_bytes(n, Hs, Ws), dtype=torch.uint8, device=dev)
        sts = (_lib.UnwStats * n)()
        row = {}
        for mode, flags in (("plain", 0), ("mixed", _lib.UNW_F_MIXED),
                            ("mixed_tc", _lib.UNW_F_MIXED | _lib.UNW_F_COL_TC)):
            prm = make_params(**FN)
            prm.flags |= flags

            def solve():
                _lib.check(lib.unw_solve_batch(n, arr, C.byref(prm), ws.data_ptr(), ws.numel(), sts,
                                               stream.cuda_stream))
            for _ in range(3):
                solve()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(5):
                solve()
            e1.record(stream)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / 1e3 / 5
            r = {"mpx_s": round(n * side * side / 1e6 / t, 2), "ms_per_step": round(t * 1e3, 3),
                 "col_path": int(sts[0].col_path), "resid_rel": float(f"{sts[0].resid_rel:.3g}")}
            if flags & _lib.UNW_F_MIXED:
                r["tune_ms_fft_tc"] = [round(float(x), 4) for x in sts[0].tune_ms]
            if side == 1024 and os.path.exists(d64):
                d = np.load(d64)
                p = grids[0][0]
                u = keep[2].cpu().numpy()
                sl = int(d["step"])
                vs = np.isfinite(p[::sl, ::sl])
                x = (u[::sl, ::sl].astype(np.float64) - d["u_sub"])[vs]
                r["rms_rad_vs_fp64_grid0"] = float(f"{np.sqrt(np.mean((x - x.mean()) ** 2)):.3g}")
            row[mode] = r
        row["ratio_mixed_over_plain"] = round(row["mixed"]["mpx_s"] / row["plain"]["mpx_s"], 4)
        row["ratio_tc_over_plain"] = round(row["mixed_tc"]["mpx_s"] / row["plain"]["mpx_s"], 4)
        out[label] = row
        del keep, ws
        torch.cuda.empty_cache()
    return out


def diff_measure(local, large=False):
    """The differentiable unwrap: a batch of 16 G1 grids of 1024^2 through
    core_b200.irls_unwrap_2d_diff (function-default forward, adjoint at a 1e-6 relative
    tolerance), loss = L2 distance to the true phase, forward (solve + loss) and backward
    (frozen-weight adjoint: refinement, adjoint PCG, gradients for phase and weight) timed
    separately with CUDA events on device-resident inputs; with large=True also one
    20000^2 G1 grid (the adjoint re-derives the frozen system from phase, weight and u, so
    no forward state is kept for the backward pass)."""
    import torch

    import core_b200
    from core_b200.synthetic import gen_g1
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    out = {}
    cases = [("batch16_g1_1024", 16, 1024, 1, 2)] + ([("g1_20000", 1, 20000, 0, 1)] if large else [])
    for label, count, side, warm, steps in cases:
        grids = [gen_g1(side, side, seed=k) for k in range(count)]
        p = torch.from_numpy(np.stack([g[0] for g in grids])).to(dev)
        c = torch.from_numpy(np.stack([g[1] for g in grids])).to(dev)
        t = torch.from_numpy(np.stack([g[2] for g in grids]).astype(np.float32)).to(dev)
        del grids
        if count == 1:
            p, c, t = p[0], c[0], t[0]
        torch.cuda.reset_peak_memory_stats(dev)

        def step():
            pt = p.detach().requires_grad_(True)
            ct = c.detach().requires_grad_(True)
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            torch.cuda.synchronize()
            e[0].record(stream)
            u, _ = core_b200.irls_unwrap_2d_diff(pt, ct)
            v = torch.isfinite(u)
            loss = 0.5 * (u[v] - t[v]).pow(2).sum()
            e[1].record(stream)
            loss.backward()
            e[2].record(stream)
            torch.cuda.synchronize()
            ok = bool(torch.isfinite(pt.grad).all()) and bool(torch.isfinite(ct.grad).all())
            return e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2]), ok
        for _ in range(warm):
            step()
        fw, bw, oks = [], [], []
        for _ in range(steps):
            a, b, ok = step()
            fw.append(a)
            bw.append(b)
            oks.append(ok)
        npx = count * side * side
        f_ms, b_ms = float(np.median(fw)), float(np.median(bw))
        out[label] = {"forward_ms": round(f_ms, 2), "backward_ms": round(b_ms, 2),
                      "fwd_bwd_mpx_s": round(npx / 1e6 / ((f_ms + b_ms) / 1e3), 3), "steps": steps,
                      "warmup": warm, "finite_gradients": all(oks),
                      "peak_device_gb": round(torch.cuda.max_memory_allocated(dev) / 1e9, 1)}
        del p, c, t
        torch.cuda.empty_cache()
    return out


# --------------------------------------------------------------------------- stack workload
def _gen_stack_entry(m):
    from core_b200.synthetic import gen_stack_grid
    p, c, _ = gen_stack_grid(m)
    return p, c


def stack_grids(n, rank, world):
    """This rank's share of the n-grid stack (grid indices, phases, weights), generated
    in a spawned process pool (safe after CUDA is initialised); shapes come from the
    seeded metadata, so every rank computes the same shard without communicating."""
    import multiprocessing as mproc
    from core_b200.stack import shard_stack
    from core_b200.synthetic import gen_stack_meta
    meta = gen_stack_meta(n, seed=0)
    shapes = [(m[0], m[1]) for m in meta]
    mine = shard_stack(shapes, world)[rank]
    with mproc.get_context("spawn").Pool(min(16, os.cpu_count() or 1, max(1, len(mine)))) as pool:
        grids = pool.map(_gen_stack_entry, [meta[i] for i in mine])
    return mine, [g[0] for g in grids], [g[1] for g in grids], sum(h * w for h, w in shapes)


def link_measure(local, steps, warmup):
    """Component linking on a 4096^2 scene of ~640 components >= 1000 px (the default conncomp_size of
    Stack.unwrap2d): device-resident input, then pinned host input and host output (H2D + D2H inside)."""
    import torch

    import core_b200
    from core_b200.synthetic import gen_link_scene
    dev = torch.device("cuda", local)
    ph, cc = gen_link_scene(4096, 4096, 2500, seed=110, holes=True, rmax=60)
    tp = torch.from_numpy(ph).to(dev)
    tc = torch.from_numpy(cc.view(np.int16)).to(dev)
    kw = dict(conncomp_size=1000)
    for _ in range(warmup):
        core_b200.link_components(tp, tc, **kw)
    torch.cuda.synchronize()
    times, parts = [], []
    for _ in range(steps):
        t = time.perf_counter()
        _, info = core_b200.link_components(tp, tc, return_info=True, **kw)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t)
        parts.append(info["timing_ms"])
    t_dev = float(np.median(times))
    # end to end as the main e2e line: pinned host input, host output
    hp = torch.from_numpy(ph).pin_memory()
    hc = torch.from_numpy(cc.view(np.int16)).pin_memory()
    core_b200.link_components(hp, hc, **kw)
    e2e_times = []
    for _ in range(steps):
        t = time.perf_counter()
        core_b200.link_components(hp, hc, **kw)
        e2e_times.append(time.perf_counter() - t)
    t_e2e = float(np.median(e2e_times))
    npx = ph.size
    return {"metric": "linked Mpx/s (4096^2, component linking)", "value": round(npx / 1e6 / t_dev, 2),
            "unit": UNIT, "ms_per_step": round(t_dev * 1e3, 2), "steps": steps, "warmup": warmup,
            "e2e": {"value": round(npx / 1e6 / t_e2e, 2), "unit": UNIT, "h2d_bytes_per_step": int(npx * 6),
                    "d2h_bytes_per_step": int(npx * 4)},
            "components": int(len(info["components"])), "connections": int(len(info["connections"])),
            "ms_parts": {k: round(float(np.median([p[k] for p in parts])), 2) for k in parts[0]},
            "timing": "median host wall clock over the calls (each call synchronises its stream; the offset "
                      "solver runs on the host)",
            "workload": "gen_link_scene(4096, 4096, 2500 ellipses r<=60, holes, seed 110), conncomp_size 1000, "
                        "linksize 5, linkcount 30, IRLS-style labels given"}


def stack_measure(phases, weights, warmup, steps, world, local, npx_all, flags=0, keep_out=(), over=None,
                  profile_out=None):
    """Batched solves of this rank's grids, inputs resident in HBM: (Mpx/s over the whole
    stack, seconds per step (max over ranks), per-grid IRLS counts, {position: u} of the
    positions in `keep_out` copied to the host, per-grid column paths).  `flags` are extra
    UNW_F_* bits (e.g. the mixed-precision form)."""
    import torch

    from core_b200 import _lib
    from core_b200.irls import make_params

    dev = torch.device("cuda", local)
    lib = _lib.load()
    n = len(phases)
    grids = (_lib.UnwGrid * max(n, 1))()
    keep = []
    Hs, Ws = (C.c_int64 * max(n, 1))(), (C.c_int64 * max(n, 1))()
    for k in range(n):
        H, W = phases[k].shape
        ph = torch.from_numpy(phases[k]).to(dev)
        wt = torch.from_numpy(weights[k]).to(dev)
        ou = torch.empty((H, W), dtype=torch.float32, device=dev)
        oc = torch.empty((H, W), dtype=torch.int16, device=dev)
        keep += [ph, wt, ou, oc]
        grids[k] = _lib.UnwGrid(ph.data_ptr(), W, wt.data_ptr(), W, H, W, ou.data_ptr(), W, oc.data_ptr(), W)
        Hs[k], Ws[k] = H, W
    ws = torch.empty(lib.unw_batch_workspace_bytes(n, Hs, Ws) if n else 1, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sts = (_lib.UnwStats * max(n, 1))()
    prm = make_params(**dict(FN, **(over or {})))
    prm.flags |= flags

    def solve():
        if n:
            _lib.check(lib.unw_solve_batch(n, grids, C.byref(prm), ws.data_ptr(), ws.numel(), sts,
                                           stream.cuda_stream))

    for _ in range(warmup):
        solve()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        solve()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    t = barrier_max(ev0.elapsed_time(ev1) / 1e3, world, local)
    iters = [sts[k].irls_iters for k in range(n)]
    paths = [sts[k].col_path for k in range(n)]
    outs = {k: keep[4 * k + 2].cpu().numpy() for k in keep_out if k < n}
    if profile_out is not None and n:
        # one more solve with every launch bracketed by CUDA events (groups one after
        # another); the sums of grid 0's stats cover all groups
        prm.flags |= _lib.UNW_F_PROFILE
        solve()
        torch.cuda.synchronize()
        st0 = sts[0]
        for i, name in enumerate(_lib.PROF_NAMES):
            if st0.prof_launches[i]:
                profile_out[name] = {"launches": int(st0.prof_launches[i]), "ms_total": round(float(st0.prof_ms[i]), 3),
                                     "us_per_launch": round(float(st0.prof_ms[i]) * 1e3 / st0.prof_launches[i], 2)}
    del keep, ws
    torch.cuda.empty_cache()
    return npx_all * steps / 1e6 / t, t / steps, iters, outs, paths


def run_stack(args):
    """K batched solves of this rank's share of the stack, inputs resident in HBM."""
    import torch

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(torch.device("cuda", local))
    mine, phases, weights, npx_all = stack_grids(args.stack, rank, world)
    clocks = ClockSampler(local)
    clocks.start()
    value, t_step, iters, _, _ = stack_measure(phases, weights, args.warmup, args.steps, world, local, npx_all)
    clk = clocks.stop()
    out = {"metric": "unwrapped Mpx/s (64-interferogram uneven stack, function-default iterations)",
           "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(t_step * 1e3, 3), "higher_is_better": True, "scaling": "strong",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": f"stack of {args.stack} G1 grids, rows U[1500,2600] x cols U[4000,7000]",
                      "total_mpx": round(npx_all / 1e6, 1), "params": FN, "irls_iters_rank0": iters,
                      "l2": "working set tens of GB, far above the 126 MB L2",
                      "parallelism": f"grids sharded over {world} GPU(s)"},
           "clocks": clk}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--stack", type=int, default=0,
                    help="measure the uneven SBAS stack of this many grids instead of the 4096^2 grid")
    ap.add_argument("--shape", type=int, nargs=2, default=None, metavar=("H", "W"),
                    help="time a G1 grid of this shape instead of the 4096^2 fault grid")
    ap.add_argument("--no-stack-line", action="store_true",
                    help="leave the 64-grid stack sub-measurement out of the default line")
    ap.add_argument("--no-link-line", action="store_true",
                    help="leave the component-linking sub-measurement out of the default line")
    ap.add_argument("--precision", default="plain", choices=["plain", "mixed"],
                    help="precision form of the main line's solves (default: plain float32)")
    ap.add_argument("--col-pass", default="auto", choices=["auto", "tc", "fft"],
                    help="with --precision mixed: column pass chosen by the autotuner, or forced")
    ap.add_argument("--no-mixed-small", action="store_true",
                    help="leave the 1024^2 mixed-precision sub-measurement out of the default line")
    ap.add_argument("--no-diff-line", action="store_true",
                    help="leave the differentiable-unwrap (16 x 1024^2 forward + backward) sub-measurement out")
    ap.add_argument("--diff-large", action="store_true",
                    help="also time forward + backward of one 20000^2 grid in the differentiable-unwrap line")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.stack:
        return run_stack(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
