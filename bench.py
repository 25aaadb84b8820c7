"""Benchmark: batched rigid motion correction of a 64x64x33x200 series.

One step = registering volumes 1..199 of a synthetic fMRI-like series to
volume 0 (199 rigid registrations, up to 20 iterations each, per-volume
early exit at a 1e-3-voxel update), all instances in one batched launch
sequence replayed from a CUDA graph.  Metric: registrations per second.

  value   inputs resident in HBM (device-pointer entry point)
  e2e     the host-buffer entry point brc_motion_correct: pinned host
          series in, corrected series and motion parameters out, copies
          inside the timed region
  --impl reference   the reference's CPU implementation of the path
          (oracle/_ref: its OpenCL C kernels compiled for the CPU with the
          host loops restated; else the C restatement) on a bounded sample
          of the same workload, all host threads

Multi-GPU (torchrun, --gpus N): replicas -- every rank corrects its own
series (weak scaling); no data-path collective; time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPE = (33, 64, 64)  # D, H, W
T = 200  # series length (--series overrides, e.g. for small profiling runs)
ITERS = 20
TOL = 1e-3
VOXEL = (3.0, 3.0, 3.0)
METRIC = "registrations/sec at <=0.05-voxel RMS err (batched rigid motion correction)"
UNIT = "registrations/s"
FLOP_PER_VOXEL_FILTER = 1372  # per complex 7^3 filter (343 taps x 2 real MACs x 2)


def workload_config(n_gpus: int, extra: dict | None = None, cert_sigma: float = 1.0) -> dict:
    c = {
        "workload": "batched rigid motion correction, 64x64x33x200 series to volume 0",
        "volume": [64, 64, 33],
        "series_length": T,
        "registrations_per_step_per_gpu": T - 1,
        "max_iterations": ITERS,
        "early_exit_voxels": TOL,
        "filters": "3 complex 7x7x7 quadrature filters (lognormal, u0=pi/3, 2 octaves)",
        "noise": "Rician, SNR 50",
        "certainty_smoothing": (f"separable 3x3x3 Gaussian, sigma {cert_sigma:g} voxel" if cert_sigma > 0
                                else "off"),
        "parallelism": f"replicas x{n_gpus}",
        "l2": "flushed between timed steps (256 MiB write)",
    }
    if extra:
        c.update(extra)
    return c


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_series(rank: int = 0):
    from broccoli_b200 import synthetic as S
    vols, truth = S.motion_series(T=T, shape=SHAPE, base_seed=rank, snr=50.0)
    return vols, truth


def filters():
    from broccoli_b200 import filters as F
    return F.linear_registration_filters()


def symmetric_bank(flt) -> bool:
    """Whether the library takes the even/odd half-tap filter kernel for
    this bank (even real, odd imaginary parts to 1e-6 of the largest tap)."""
    f = np.asarray(flt, np.float32)
    for k in range(f.shape[0]):
        mx = np.abs(f[k]).max()
        re, im = f[k, 0], f[k, 1]
        if (np.abs(re - re[::-1, ::-1, ::-1]).max() > 1e-6 * mx or
                np.abs(im + im[::-1, ::-1, ::-1]).max() > 1e-6 * mx):
            return False
    return True


def accuracy(vols, truth, params, flt, n_oracle: int = 2, cert_sigma: float = 0.0) -> dict:
    """RMS displacement error of the GPU results against the FP64 oracle on
    a sample of volumes, and against the known motion on all volumes."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from broccoli_b200 import synthetic as S
    vs_truth = []
    for i in range(params.shape[0]):
        rel = S.relative_params(truth[0], truth[i + 1])
        vs_truth.append(S.rms_displacement_error(params[i], rel, SHAPE))
    vs_oracle = []
    for i in range(n_oracle):
        p64, _, _ = oracle.align_linear(vols[0], vols[i + 1], flt, ITERS, oracle.RIGID, prec="f64",
                                        cert_sigma=cert_sigma)
        vs_oracle.append(S.rms_displacement_error(params[i], p64, SHAPE))
    return {"rms_vs_fp64_oracle_max": float(max(vs_oracle)) if vs_oracle else None,
            "oracle_sample": n_oracle,
            "rms_vs_truth_mean": float(np.mean(vs_truth)),
            "rms_vs_truth_max": float(np.max(vs_truth))}


def cpu_reference_rate(vols, flt, n_regs: int, iters: int = ITERS):
    """Registrations/s of the reference's CPU path on n_regs volumes of the
    series.  Returns (rate, kind, threads, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    kind = "reference" if oracle.ref_available() else "port"
    fn = oracle.ref_align_linear if kind == "reference" else oracle.align_linear
    t0 = time.perf_counter()
    for i in range(n_regs):
        fn(vols[0], vols[1 + i], flt, iters, oracle.RIGID)
    dt = time.perf_counter() - t0
    return n_regs / dt, kind, oracle.num_threads(), dt


def normalisation_rates(ctx, prec) -> dict:
    """T1-to-template normalisation (affine, then nonlinear over the scales
    8, 4, 2, 1 with the six nonlinear filters; 10 + 10 iterations) timed with
    CUDA events: one subject of 256 x 256 x 170 1-mm voxels (a head phantom
    warped by a smooth 6-mm field) and a cohort of 64 subjects with per-axis
    sizes U{160..256} (seeds 300 + i, crops of one 256^3 phantom), both onto a
    182 x 218 x 182 1-mm template phantom.  Filters: the reference's shipped
    linear and nonlinear banks (tests/golden/filters)."""
    import torch
    from broccoli_b200 import filters as F
    from broccoli_b200 import synthetic as S
    bank = F.load_filter_dir(os.path.join(ROOT, "tests", "golden", "filters"))
    tpl = torch.from_numpy(S.head_phantom((182, 218, 182), seed=2)).cuda()
    subj_np = S.warp_with_field(S.head_phantom((170, 256, 256), seed=1),
                                S.smooth_field((170, 256, 256), seed=200, max_mm=6.0))
    subj = torch.from_numpy(np.ascontiguousarray(subj_np, np.float32)).cuda()
    one = (1.0, 1.0, 1.0)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    two = lambda: ctx.register_two_volumes(subj, one, tpl, one, bank, 10, 10, 8, precision=prec)  # noqa: E731
    timed(two)
    # the first timed registration is the range a profiler started with
    # --profile-from-start off records (no effect without a profiler)
    torch.cuda.profiler.start()
    ms1 = timed(two)
    torch.cuda.profiler.stop()
    ms1 = min([ms1] + [timed(two) for _ in range(2)])
    big = S.head_phantom((256, 256, 256), seed=3)
    subjects, sizes = [], []
    for i in range(64):
        rng = np.random.Generator(np.random.PCG64(300 + i))
        d, h, w = (int(v) for v in rng.integers(160, 257, 3))
        z0, y0, x0 = (256 - d) // 2, (256 - h) // 2, (256 - w) // 2
        subjects.append(torch.from_numpy(np.ascontiguousarray(big[z0:z0 + d, y0:y0 + h, x0:x0 + w])).cuda())
        sizes.append((w, h, d))
    coh = lambda: ctx.register_cohort(subjects, [one] * 64, tpl, one, bank, 10, 10, 8, precision=prec)  # noqa: E731
    timed(coh)
    ms64 = min(timed(coh) for _ in range(2))
    return {
        "t1_to_template": {"value": 1000.0 / ms1, "unit": "subjects/s", "ms_per_subject": ms1,
                           "config": {"subject": [256, 256, 170], "template": [182, 218, 182], "voxel_mm": 1.0,
                                      "linear_iterations": 10, "nonlinear_iterations": 10,
                                      "scales": [8, 4, 2, 1]}},
        "cohort": {"value": 64 * 1000.0 / ms64, "unit": "subjects/s", "ms": ms64,
                   "config": {"subjects": 64, "sizes": "U{160..256} per axis (seeds 300 + i)",
                              "template": [182, 218, 182], "linear_iterations": 10,
                              "nonlinear_iterations": 10, "scales": [8, 4, 2, 1]}},
    }


def run_reference(args, rank, world):
    if rank != 0:
        return
    vols, _ = make_series(0)
    flt = filters()
    n_regs = 2
    rates = []
    for _ in range(args.warmup):
        cpu_reference_rate(vols, flt, 1)
    secs = 0.0
    for _ in range(args.steps):
        r, kind, thr, dt = cpu_reference_rate(vols, flt, n_regs)
        rates.append(r)
        secs += dt
    value = float(np.median(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(args.gpus, {"certainty_smoothing": "none: the reference path has no certainty "
                                                                     "smoothing (raw certainties)"}),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": thr, "kind": kind,
                         "sample": f"{n_regs} of the {T - 1} registrations per step, {ITERS} iterations "
                                   "each (the reference runs every iteration; no early exit)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_gpu(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from broccoli_b200 import _lib as L
    from broccoli_b200.api import Context

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = Context(local_rank)
    flt = filters()
    prec = L.PREC_BF16X3 if args.precision == "bf16x3" else L.PREC_FP32
    vols, truth = make_series(rank)
    D, H, W = SHAPE
    V = D * H * W
    d_series = torch.from_numpy(vols).to(dev)
    ref = d_series[0]
    moving = d_series[1:]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    cs = args.certainty_sigma

    def step(precision=None):
        return ctx.register_linear(ref, moving, flt, ITERS, L.RIGID, tolerance=TOL,
                                   precision=prec if precision is None else precision, certainty_sigma=cs)

    def barrier():
        if world > 1:
            dist.barrier()

    # clocks are sampled from the warm-up through the end of the timed
    # region (nvidia-smi needs ~0.2 s per sample; the timed region is short)
    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    for _ in range(args.warmup):
        out = step()
    torch.cuda.synchronize()

    # ---- device-resident timed region ----
    launches0 = ctx.kernel_launches
    st = torch.cuda.current_stream()
    times = []
    barrier()
    torch.cuda.synchronize()
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        out = step()
        e1.record(st)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    barrier()
    launches = ctx.kernel_launches - launches0
    if sampler:
        time.sleep(0.25)
    clocks = sampler.stop() if sampler else None
    ms = float(np.sum(times))
    iters_used = out["iterations"].cpu().numpy()
    if args.only_steps:
        # the timed step alone (for launch lists and profiles of the step)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": (T - 1) * args.steps / (ms / 1000.0), "unit": UNIT,
                              "steps": args.steps, "warmup": args.warmup, "only_steps": True,
                              "precision": args.precision, "gpu_launches": int(launches)}))
        return

    # ---- end-to-end through the host-buffer entry point ----
    host = torch.from_numpy(vols).pin_memory()
    motion = np.zeros(6 * T, np.float32)
    e2e_times = []
    import ctypes
    opts = L.LinearOpts()
    L.lib().brc_linear_opts_default(ctypes.byref(opts), ITERS)
    opts.type = L.RIGID
    opts.tolerance = TOL
    opts.precision = prec
    opts.certainty_sigma_x100 = int(round(cs * 100))
    vs = np.asarray(VOXEL, np.float32)
    fl = np.ascontiguousarray(flt, np.float32)
    work = torch.empty_like(host).pin_memory()
    ctx._bind_stream()
    for k in range(args.warmup + args.steps):
        work.copy_(host)
        flush.fill_(1.0)
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        s = L.lib().brc_motion_correct(ctx.handle, ctypes.c_void_p(work.data_ptr()), W, H, D, T,
                                       vs.ctypes.data_as(ctypes.c_void_p), fl.ctypes.data_as(ctypes.c_void_p),
                                       ctypes.byref(opts), None, motion.ctypes.data_as(ctypes.c_void_p))
        dt = time.perf_counter() - t0
        if s != 0:
            raise RuntimeError(f"brc_motion_correct failed: {s}")
        if k >= args.warmup:
            e2e_times.append(dt * 1000.0)
    e2e_ms = float(np.sum(e2e_times))

    # ---- the plain FP32 GPU path: the same registrations one volume at a
    # time (batch 1, eager launches, no graph), on a sample of the series ----
    n_serial = min(24, T - 1)
    for i in range(2):
        ctx.register_linear(ref, moving[i:i + 1], flt, ITERS, L.RIGID, tolerance=TOL, use_graph=False,
                            certainty_sigma=cs)
    torch.cuda.synchronize()
    se0 = torch.cuda.Event(enable_timing=True)
    se1 = torch.cuda.Event(enable_timing=True)
    se0.record(st)
    for i in range(n_serial):
        ctx.register_linear(ref, moving[i:i + 1], flt, ITERS, L.RIGID, tolerance=TOL, use_graph=False,
                            certainty_sigma=cs)
    se1.record(st)
    se1.synchronize()
    serial_rate = n_serial / (se0.elapsed_time(se1) / 1000.0)

    # ---- the same batched step with FP32 filtering (when timing BF16X3) ----
    fp32_batched = None
    if prec != L.PREC_FP32:
        for _ in range(2):
            step(L.PREC_FP32)
        torch.cuda.synchronize()
        b_times = []
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            step(L.PREC_FP32)
            e1.record(st)
            e1.synchronize()
            b_times.append(e0.elapsed_time(e1))
        fp32_batched = (T - 1) * args.steps / (float(np.sum(b_times)) / 1000.0)

    # ---- dominant kernel alone: 7^3 filtering of the 199 moving volumes
    # (inputs 107 MB + responses 640 MB per launch, larger than L2) ----
    q = torch.empty((T - 1, 3, D, H, W, 2), dtype=torch.float32, device=dev)

    def time_filter(precision, nrep=20):
        for _ in range(3):
            L.lib().brc_filter3d(ctx.handle, ctypes.c_void_p(moving.data_ptr()), W, H, D, T - 1, V,
                                 fl.ctypes.data_as(ctypes.c_void_p), 3, precision, ctypes.c_void_p(q.data_ptr()))
        torch.cuda.synchronize()
        fe0 = torch.cuda.Event(enable_timing=True)
        fe1 = torch.cuda.Event(enable_timing=True)
        fe0.record(st)
        for _ in range(nrep):
            L.lib().brc_filter3d(ctx.handle, ctypes.c_void_p(moving.data_ptr()), W, H, D, T - 1, V,
                                 fl.ctypes.data_as(ctypes.c_void_p), 3, precision, ctypes.c_void_p(q.data_ptr()))
        fe1.record(st)
        fe1.synchronize()
        return fe0.elapsed_time(fe1) / nrep

    f_ms = time_filter(prec)
    f32_ms = time_filter(L.PREC_FP32) if prec != L.PREC_FP32 else f_ms
    ctx.synchronize()
    f_flop = FLOP_PER_VOXEL_FILTER * 3 * V * (T - 1)

    # ---- reduce over ranks ----
    t_max = ms
    e_max = e2e_ms
    if world > 1:
        tt = torch.tensor([ms, e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max, e_max = float(tt[0]), float(tt[1])
    if rank != 0:
        return
    regs = (T - 1) * world * args.steps
    value = regs / (t_max / 1000.0)
    e2e_value = regs / (e_max / 1000.0)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    sm_max = clocks.get("sm_max_mhz") if clocks else None
    fp32_peak = 148 * 128 * 2 * (sm_max or 1965.0) * 1e6 / 1e12
    # DRAM bytes (read + write) per filtered volume of 64x64x33 from one ncu
    # capture of each kernel on 63 volumes (profiles/filter3d_tc_motion_
    # correction.md, profiles/filter3d_sym_motion_correction.md), scaled to
    # this launch by the volume count (traffic grows with the volumes).  The
    # tensor-core figure is below the algorithmic bytes: the input comes
    # partly from L2 (written by the preceding resampling) and part of the
    # output is still in L2 when the kernel ends.
    tc_bytes_per_vol = (17850368 + 48461056) / 63
    sym_bytes_per_vol = (34094848 + 147386624) / 63
    traffic = sym_bytes_per_vol * (T - 1) if symmetric_bank(fl) and tuple(SHAPE) == (33, 64, 64) else None
    tc_traffic = tc_bytes_per_vol * (T - 1) if tuple(SHAPE) == (33, 64, 64) else None
    achieved = f_flop / (f_ms / 1000.0) / 1e12
    if prec == L.PREC_BF16X3:
        peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
        tc_peak = peaks.get("bf16_tflops", 1590.0)
        # the split form issues 3 BF16 products per tap: 3x the convolution FLOPs
        tc_achieved = 3 * f_flop / (f_ms / 1000.0) / 1e12
        roofline = {"kernel": "filter3d_tc_kernel (tcgen05.mma kind::f16, split BF16 x3, FP32 accumulate in TMEM)",
                    "bound": "tensor", "achieved": tc_achieved, "peak": tc_peak, "unit": "TFLOP/s",
                    "frac": tc_achieved / tc_peak,
                    "peak_source": ("MEASURED_PEAKS.json bf16_tflops (burst, measured)" if "bf16_tflops" in peaks
                                    else "fallback 1.59 PFLOP/s"),
                    "flop_per_launch": 3 * f_flop,
                    "flop_note": "3 split products x the 343-tap convolution of 3 complex filters; "
                                 "the banded-Toeplitz zeros the GEMMs also issue are not counted",
                    "launch_ms": f_ms, "fp32_equiv_tflops": achieved,
                    "fp32_filter_launch_ms": f32_ms, "traffic": tc_traffic,
                    "traffic_note": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch on 63 "
                                    "volumes, scaled by the volume count; algorithmic: 4 B in + 24 B out "
                                    "per voxel"}
    else:
        roofline = {"kernel": ("filter3d_sym_kernel<3,8,3> (even/odd half-tap form; FLOP counted "
                               "as the full 343-tap convolution)") if symmetric_bank(fl) else
                    "filter3d_fp32_kernel<3,8,3>", "bound": "fp32",
                    "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                    "frac": achieved / fp32_peak,
                    "peak_source": "nominal FP32 FMA rate 148 SMs x 128 lanes x 2 at the sampled max SM clock "
                                   "(MEASURED_PEAKS.json has no FP32 figure)",
                    "flop_per_launch": f_flop, "launch_ms": f_ms, "traffic": traffic}
    acc = (accuracy(vols, truth, out["params"].cpu().numpy(), flt, cert_sigma=cs)
           if not args.skip_accuracy else None)
    cpu = None
    if not args.skip_cpu:
        r, kind, thr, dt = cpu_reference_rate(vols, flt, 8)
        cpu = {"value": r, "unit": UNIT, "cores": thr, "kind": kind,
               "sample": f"8 of the {T - 1} registrations of one series, {ITERS} iterations each, "
                         f"{dt:.1f} s (the reference path: raw certainties, no early exit)"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3" if prec == L.PREC_BF16X3 else "f32",
        "data": "synthetic",
        "config": workload_config(world, {"mean_iterations": float(iters_used.mean()),
                                          "precision": args.precision}, cert_sigma=cs),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(4 * V * T),
                "d2h_bytes_per_step": int(4 * V * (T - 1) + 4 * 15 * (T - 1))},
        "gpu_launches": int(launches),
        "roofline": roofline,
        "accuracy": acc,
        "plain_fp32_serial": {"value": serial_rate, "unit": UNIT,
                              "sample": f"{n_serial} volumes of the series registered one at a time "
                                        "(batch 1, eager launches)",
                              "batched_over_serial": value / serial_rate},
        "fp32_batched": ({"value": fp32_batched, "unit": UNIT,
                          "sample": "the same batched step with FP32 filtering"} if fp32_batched else None),
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if not args.skip_normalisation:
        line.update(normalisation_rates(ctx, prec))
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-accuracy", action="store_true")
    ap.add_argument("--skip-normalisation", action="store_true",
                    help="skip the T1-to-template and cohort timings (configs 2 and 4)")
    ap.add_argument("--series", type=int, default=T, help="series length (volumes)")
    ap.add_argument("--precision", default="bf16x3", choices=["fp32", "bf16x3"],
                    help="filtering precision of the timed path (bf16x3: tensor-core split BF16)")
    ap.add_argument("--certainty-sigma", type=float, default=1.0,
                    help="sigma (voxels) of the 3x3x3 certainty smoothing; 0 = off")
    ap.add_argument("--only-steps", action="store_true",
                    help="time the device-resident steps only (no e2e, baselines or kernel timing)")
    args = ap.parse_args()
    globals()["T"] = args.series
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_gpu(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
