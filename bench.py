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

The line also carries: the same batched step in the reference arm's own
configuration (like_for_like), one FP32 AFFINE registration of 64x64x33
(config0_plain_fp32_affine), the forward and backward times of the
differentiable objective at 128x128x96 (differentiable), T1-to-template
normalisation and a 64-subject cohort in mixed precision and in FP32
(t1_to_template, cohort), RMS displacement errors against the FP64 oracle,
and clocks sampled through every section.

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
    """nvidia-smi clock/throttle sampling (every 200 ms) from the warm-up to
    the end of the last GPU section; each sample is time-stamped so that
    every section gets its own median clock."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.samples = []  # (monotonic time, sm MHz, max MHz, active reasons)
        self.sections = {}

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
            parts = [p.strip() for p in line.strip().split(",")]
            if len(parts) < 7:
                continue
            try:
                sm, smax = float(parts[0]), float(parts[1])
            except ValueError:
                continue
            reasons = [n for n, v in zip(self.NAMES, parts[3:7]) if v.lower() == "active"]
            self.samples.append((time.monotonic(), sm, smax, reasons))

    def section(self, name: str, t0: float, t1: float):
        self.sections[name] = (t0, t1)

    def stop(self):
        if self.proc is None:
            return
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()

    def summary(self, t0: float = None, t1: float = None) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sel = [s for s in self.samples if (t0 is None or s[0] >= t0) and (t1 is None or s[0] <= t1)]
        if not sel and t0 is not None:  # a section shorter than the sampling period
            mid = 0.5 * (t0 + t1)
            sel = sorted(self.samples, key=lambda s: abs(s[0] - mid))[:1]
        reasons = sorted({r for s in sel for r in s[3]})
        return {"sm_mhz": float(np.median([s[1] for s in sel])) if sel else None,
                "sm_max_mhz": max(s[2] for s in sel) if sel else None,
                "reasons": reasons, "samples": len(sel)}

    def section_summary(self, name: str) -> dict:
        t0, t1 = self.sections[name]
        return self.summary(t0, t1)


class Section:
    """Context manager that records a named section's wall interval with
    the sampler (for its median clock)."""

    def __init__(self, sampler, name):
        self.sampler, self.name = sampler, name

    def __enter__(self):
        self.t0 = time.monotonic()
        return self

    def __exit__(self, *exc):
        if self.sampler:
            self.sampler.section(self.name, self.t0, time.monotonic())
        return False


def clocked(entry: dict, sampler, name: str, ms: float) -> dict:
    """Adds the section's clock record and time x median SM clock (millions
    of SM cycles, comparable across runs at different clocks)."""
    if sampler and name in sampler.sections:
        c = sampler.section_summary(name)
        entry["clocks"] = c
        if c.get("sm_mhz"):
            entry["sm_mcycles"] = ms * c["sm_mhz"] / 1000.0
    return entry


def cuda_ms(fn, stream=None) -> float:
    """Device time of fn() in ms (CUDA events on the current stream)."""
    import torch
    st = stream or torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    fn()
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1)


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


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def accuracy(vols, truth, params, flt, n_oracle: int = 16, cert_sigma: float = 0.0) -> dict:
    """RMS displacement error of the GPU results against the FP64 oracle on
    the first n_oracle volumes (all 20 iterations, the same certainty
    smoothing), and against the known motion on all volumes."""
    oracle = _oracle()
    from broccoli_b200 import synthetic as S
    vs_truth = []
    for i in range(params.shape[0]):
        rel = S.relative_params(truth[0], truth[i + 1])
        vs_truth.append(S.rms_displacement_error(params[i], rel, SHAPE))
    vs_oracle = []
    for i in range(min(n_oracle, params.shape[0])):
        p64, _, _ = oracle.align_linear(vols[0], vols[i + 1], flt, ITERS, oracle.RIGID, prec="f64",
                                        cert_sigma=cert_sigma)
        vs_oracle.append(S.rms_displacement_error(params[i], p64, SHAPE))
    return {"rms_vs_fp64_oracle_max": float(max(vs_oracle)) if vs_oracle else None,
            "rms_vs_fp64_oracle_mean": float(np.mean(vs_oracle)) if vs_oracle else None,
            "oracle_sample": len(vs_oracle),
            "rms_vs_truth_mean": float(np.mean(vs_truth)),
            "rms_vs_truth_max": float(np.max(vs_truth))}


def cpu_reference_rate(vols, flt, n_regs: int, iters: int = ITERS, type_: int = 1):
    """Registrations/s of the reference's CPU path on n_regs volumes of the
    series.  Returns (rate, kind, threads, seconds)."""
    oracle = _oracle()
    kind = "reference" if oracle.ref_available() else "port"
    fn = oracle.ref_align_linear if kind == "reference" else oracle.align_linear
    t0 = time.perf_counter()
    for i in range(n_regs):
        fn(vols[0], vols[1 + i], flt, iters, type_)
    dt = time.perf_counter() - t0
    return n_regs / dt, kind, oracle.num_threads(), dt


def cpu_baseline_protocol(vols, flt) -> dict:
    """The reference's CPU path (oracle/_ref: its OpenCL C kernels compiled
    for the host, else the restatement) on the host cores: the median of 5
    runs of 2 registrations each after 1 warm-up registration, all threads;
    plus one registration on 1 thread."""
    oracle = _oracle()
    cpu_reference_rate(vols, flt, 1)
    runs = [cpu_reference_rate(vols, flt, 2) for _ in range(5)]
    kind, thr = runs[0][1], runs[0][2]
    rate = float(np.median([r[0] for r in runs]))
    n = oracle.num_threads()
    oracle.set_num_threads(1)
    try:
        r1, _, _, dt1 = cpu_reference_rate(vols, flt, 1)
    finally:
        oracle.set_num_threads(n)
    return {"value": rate, "unit": UNIT, "cores": thr, "kind": kind,
            "sample": (f"median of 5 runs of 2 of the {T - 1} registrations (after 1 warm-up), {ITERS} "
                       "iterations each, RIGID, FP32, raw certainties, no early exit (the reference path)"),
            "runs": [float(r[0]) for r in runs],
            "one_thread": {"value": float(r1), "unit": UNIT, "cores": 1,
                           "sample": f"1 registration, {dt1:.1f} s"}}


def config0_rates(ctx, L, dev, cpu: bool) -> dict:
    """One plain FP32 AFFINE registration of a 64 x 64 x 33 volume (3 mm
    EPI-like base volume and a copy under a seeded affine), 20 iterations,
    single scale, no early exit, lognormal u0 = pi/3 / 2-octave filters:
    batch 1 through the library's linear-registration entry point (graph
    replay), median of 20 registrations; and the reference's CPU path on the
    same registration."""
    import torch
    from broccoli_b200 import synthetic as S
    base, moved, truth = S.affine_pair(SHAPE)
    flt = filters()
    b, m = torch.from_numpy(base).to(dev), torch.from_numpy(moved).to(dev)[None]

    def one():
        return ctx.register_linear(b, m, flt, ITERS, L.AFFINE, tolerance=0.0, precision=L.PREC_FP32)
    for _ in range(3):
        r = one()
    ms = float(np.median([cuda_ms(one) for _ in range(20)]))
    p = r["params"].cpu().numpy()[0]
    out = {"value": 1000.0 / ms, "unit": "registrations/s", "ms_per_registration": ms,
           "config": {"workload": "one FP32 AFFINE registration, 64x64x33, 20 iterations, no early exit",
                      "precision": "fp32", "batch": 1, "filters": "lognormal u0=pi/3, 2 octaves"}}
    oracle = _oracle()
    p64, _, _ = oracle.align_linear(base, moved, flt, ITERS, oracle.AFFINE, prec="f64")
    out["rms_vs_fp64_oracle"] = S.rms_displacement_error(p, p64, SHAPE)
    out["rms_vs_truth"] = S.rms_displacement_error(p, truth, SHAPE)
    if cpu:
        kind = "reference" if oracle.ref_available() else "port"
        fn = oracle.ref_align_linear if kind == "reference" else oracle.align_linear
        t0 = time.perf_counter()
        fn(base, moved, flt, ITERS, oracle.AFFINE)
        dt = time.perf_counter() - t0
        out["cpu_reference"] = {"value": 1.0 / dt, "unit": "registrations/s", "kind": kind,
                                "cores": oracle.num_threads(), "sample": "the same registration, once"}
    return out


def differentiable_rates(dev) -> dict:
    """Config 3: the filter-response SSD of a 128 x 128 x 96 pair (head
    phantoms as in the T1 workload, the moving one warped by a smooth field),
    smoothed at sigma 2, warped by 12 affine parameters or a 3 x 128 x 128 x
    96 displacement field, filtered by the 3 lognormal filters; forward and
    backward (adjoint kernels) device times, median of 10."""
    import torch
    from broccoli_b200 import autograd as AG
    from broccoli_b200 import synthetic as S
    shape = (96, 128, 128)
    ref = torch.from_numpy(S.head_phantom(shape, seed=2)).to(dev)
    mov = torch.from_numpy(np.ascontiguousarray(
        S.warp_with_field(S.head_phantom(shape, seed=1), S.smooth_field(shape, seed=200, max_mm=4.0)),
        np.float32)).to(dev)
    flt = filters()
    q_ref = AG.reference_responses(ref, flt, 2.0)
    out = {}
    for name in ("params", "field"):
        if name == "params":
            x = torch.zeros(12, device=dev, requires_grad=True)
            kw = {"params": x}
        else:
            x = torch.zeros((3,) + shape, device=dev, requires_grad=True)
            kw = {name: x}
        holder = {}

        def fwd():
            holder["L"] = AG.registration_objective(mov, q_ref, flt, 2.0, **kw)

        def bwd():
            holder["L"].backward()
        for _ in range(3):
            fwd()
            bwd()
        f_ms, b_ms = [], []
        for _ in range(10):
            x.grad = None
            f_ms.append(cuda_ms(fwd))
            b_ms.append(cuda_ms(bwd))
        out[name] = {"forward_ms": float(np.median(f_ms)), "backward_ms": float(np.median(b_ms))}
    out["config"] = {"volume": [128, 128, 96], "sigma": 2.0, "filters": 3,
                     "gradient_check": "tests/test_gpu_autograd.py (FP64 central differences, 1e-3 voxel)"}
    return out


def normalisation_rates(ctx, L, prec, sampler, accuracy_on: bool, reps: int = 5) -> dict:
    """T1-to-template normalisation (affine, then nonlinear over the scales
    8, 4, 2, 1 with the six nonlinear filters; 10 + 10 iterations) timed with
    CUDA events: one subject of 256 x 256 x 170 1-mm voxels (a head phantom
    warped by a smooth 6-mm field) and a cohort of 64 subjects with per-axis
    sizes U{160..256} (seeds 300 + i, crops of one 256^3 phantom), both onto a
    182 x 218 x 182 1-mm template phantom.  Filters: the reference's shipped
    linear and nonlinear banks (tests/golden/filters).  The mixed-precision
    form (tensor-core filtering in the timed precision, TF32 or BF16X3, FP64
    per-voxel 3x3 solves, FP64 12x12 solves) and
    the plain FP32 form (FP32 filtering, the reference's FP32 cofactor
    solves); medians of `reps` runs; the cohort also one subject at a time in
    plain FP32."""
    import torch
    from broccoli_b200 import filters as F
    from broccoli_b200 import synthetic as S
    bank = F.load_filter_dir(os.path.join(ROOT, "tests", "golden", "filters"))
    tpl_np = S.head_phantom((182, 218, 182), seed=2)
    tpl = torch.from_numpy(tpl_np).cuda()
    subj_np = np.ascontiguousarray(S.warp_with_field(S.head_phantom((170, 256, 256), seed=1),
                                                     S.smooth_field((170, 256, 256), seed=200, max_mm=6.0)),
                                   np.float32)
    subj = torch.from_numpy(subj_np).cuda()
    one = (1.0, 1.0, 1.0)
    mixed = prec in (L.PREC_BF16X3, L.PREC_TF32)
    pname = {L.PREC_BF16X3: "bf16x3", L.PREC_TF32: "tf32"}.get(prec, "fp32")
    forms = [("mixed" if mixed else "fp32", prec, mixed)] + ([("fp32", L.PREC_FP32, False)] if mixed else [])

    def two(p, fp64):
        return ctx.register_two_volumes(subj, one, tpl, one, bank, 10, 10, 8, precision=p, solve_fp64=fp64)

    t1 = {}
    results = {}
    for name, p, fp64 in forms:
        results[name] = two(p, fp64)
        with Section(sampler, "t1_" + name):
            if name == forms[0][0]:
                # the first timed registration is the range a profiler started
                # with --profile-from-start off records (no effect without one)
                torch.cuda.profiler.start()
                ms = [cuda_ms(lambda: two(p, fp64))]
                torch.cuda.profiler.stop()
            else:
                ms = [cuda_ms(lambda: two(p, fp64))]
            ms += [cuda_ms(lambda: two(p, fp64)) for _ in range(reps - 1)]
        med = float(np.median(ms))
        t1[name] = clocked({"value": 1000.0 / med, "unit": "subjects/s", "ms_per_subject": med,
                            "runs_ms": [float(v) for v in ms], "precision": pname + " + fp64 solves" if fp64 else
                            "fp32"}, sampler, "t1_" + name, med)

    big = S.head_phantom((256, 256, 256), seed=3)
    subjects = []
    for i in range(64):
        rng = np.random.Generator(np.random.PCG64(300 + i))
        d, h, w = (int(v) for v in rng.integers(160, 257, 3))
        z0, y0, x0 = (256 - d) // 2, (256 - h) // 2, (256 - w) // 2
        subjects.append(torch.from_numpy(np.ascontiguousarray(big[z0:z0 + d, y0:y0 + h, x0:x0 + w])).cuda())
    coh = {}
    coh_res = {}
    for name, p, fp64 in forms:
        def run(p=p, fp64=fp64):
            return ctx.register_cohort(subjects, [one] * 64, tpl, one, bank, 10, 10, 8, precision=p, solve_fp64=fp64)
        coh_res[name] = run()
        with Section(sampler, "cohort_" + name):
            ms = [cuda_ms(run) for _ in range(reps)]
        med = float(np.median(ms))
        coh[name] = clocked({"value": 64 * 1000.0 / med, "unit": "subjects/s", "ms": med,
                             "runs_ms": [float(v) for v in ms], "precision": pname + " + fp64 solves" if fp64 else
                             "fp32"}, sampler, "cohort_" + name, med)

    def serial():
        for sub in subjects:
            ctx.register_two_volumes(sub, one, tpl, one, bank, 10, 10, 8, precision=L.PREC_FP32)
    serial()
    with Section(sampler, "cohort_serial_fp32"):
        ms = [cuda_ms(serial) for _ in range(3)]
    med = float(np.median(ms))
    coh["serial_fp32"] = clocked({"value": 64 * 1000.0 / med, "unit": "subjects/s", "ms": med,
                                  "runs_ms": [float(v) for v in ms],
                                  "sample": "the 64 subjects one at a time through brc_register_two_volumes, "
                                            "FP32, median of 3"}, sampler, "cohort_serial_fp32", med)

    head = forms[0][0]
    out_t1 = {"value": t1[head]["value"], "unit": "subjects/s", "ms_per_subject": t1[head]["ms_per_subject"],
              "forms": t1,
              "config": {"subject": [256, 256, 170], "template": [182, 218, 182], "voxel_mm": 1.0,
                         "linear_iterations": 10, "nonlinear_iterations": 10, "scales": [8, 4, 2, 1]}}
    if "fp32" in t1 and head != "fp32":
        out_t1["mixed_over_fp32"] = t1[head]["value"] / t1["fp32"]["value"]
    out_coh = {"value": coh[head]["value"], "unit": "subjects/s", "ms": coh[head]["ms"], "forms": coh,
               "batched_over_serial_fp32": coh[head]["value"] / coh["serial_fp32"]["value"],
               "config": {"subjects": 64, "sizes": "U{160..256} per axis (seeds 300 + i)",
                          "template": [182, 218, 182], "linear_iterations": 10,
                          "nonlinear_iterations": 10, "scales": [8, 4, 2, 1]}}
    if accuracy_on:
        # RMS over the template grid of the length of the difference between
        # the combined (affine + nonlinear) displacement fields and those of
        # the FP64 oracle, on the single subject and on cohort subject 0
        oracle = _oracle()
        sub0 = subjects[0].cpu().numpy()

        def rms(f, ref):
            d = np.asarray(f, np.float64) - ref
            return float(np.sqrt((d * d).sum(0).mean()))
        t0 = time.perf_counter()
        o1 = oracle.register_two_volumes(subj_np, one, tpl_np, one, bank, 10, 10, 8, prec="f64")
        acc1 = {k: rms(v["field"].cpu().numpy(), o1["field"]) for k, v in results.items()}
        o2 = oracle.register_two_volumes(sub0, one, tpl_np, one, bank, 10, 10, 8, prec="f64")
        acc2 = {k: rms(v["fields"][0].cpu().numpy(), o2["field"]) for k, v in coh_res.items()}
        dt = time.perf_counter() - t0
        out_t1["accuracy"] = {"rms_field_vs_fp64_oracle_voxels": acc1, "bar": 0.05}
        out_coh["accuracy"] = {"rms_field_vs_fp64_oracle_voxels": acc2, "bar": 0.05,
                               "sample": "cohort subject 0", "oracle_seconds_both": dt}
    return {"t1_to_template": out_t1, "cohort": out_coh}


def max_over_ranks(values, world: int, device) -> list:
    """Each value's maximum over the ranks: the slowest rank's time.  One
    all_reduce (MAX) of a float64 tensor on `device` (the rank's GPU under
    NCCL); on one rank the values themselves."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def whole_job_rate(world: int, steps: int, slowest_ms: float) -> float:
    """Registrations per second of the whole job: each of the `world`
    replicas registers T - 1 volumes per step, and the job lasts as long as
    its slowest rank."""
    return (T - 1) * world * steps / (slowest_ms / 1000.0)


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
    import ctypes
    import torch
    import torch.distributed as dist
    from broccoli_b200 import _lib as L
    from broccoli_b200.api import Context

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = Context(local_rank)
    flt = filters()
    prec = {"bf16x3": L.PREC_BF16X3, "tf32": L.PREC_TF32}.get(args.precision, L.PREC_FP32)
    vols, truth = make_series(rank)
    D, H, W = SHAPE
    V = D * H * W
    d_series = torch.from_numpy(vols).to(dev)
    ref = d_series[0]
    moving = d_series[1:]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream()
    cs = args.certainty_sigma

    def step(precision=None, tol=TOL, cert=cs):
        return ctx.register_linear(ref, moving, flt, ITERS, L.RIGID, tolerance=tol,
                                   precision=prec if precision is None else precision, certainty_sigma=cert)

    def barrier():
        if world > 1:
            dist.barrier()

    def timed_steps(fn, n):
        """n steps, each timed with CUDA events on the launching stream,
        the L2 flushed (256 MiB write) before each."""
        out, times = None, []
        for _ in range(n):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            out = fn()
            e1.record(st)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        return out, times

    # clocks are sampled from the warm-up through the last GPU section
    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    t_main0 = time.monotonic()
    for _ in range(args.warmup):
        out = step()
    torch.cuda.synchronize()

    # ---- device-resident timed region ----
    launches0 = ctx.kernel_launches
    barrier()
    torch.cuda.synchronize()
    out, times = timed_steps(step, args.steps)
    torch.cuda.synchronize()
    barrier()
    launches = ctx.kernel_launches - launches0
    if sampler:
        sampler.section("main", t_main0, time.monotonic())
    ms = float(np.sum(times))
    iters_used = out["iterations"].cpu().numpy()
    if args.only_steps:
        # the timed step alone (for launch lists and profiles of the step)
        if sampler:
            sampler.stop()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": (T - 1) * args.steps / (ms / 1000.0), "unit": UNIT,
                              "steps": args.steps, "warmup": args.warmup, "only_steps": True,
                              "precision": args.precision, "gpu_launches": int(launches)}))
        return

    # ---- end-to-end through the host-buffer entry point ----
    host = torch.from_numpy(vols).pin_memory()
    motion = np.zeros(6 * T, np.float32)
    e2e_times = []
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
    with Section(sampler, "e2e"):
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

    # ---- the GPU path run exactly as the reference arm runs: FP32
    # filtering, no early exit (all 20 iterations), raw certainties, RIGID,
    # batched over the series ----
    with Section(sampler, "like_for_like"):
        for _ in range(2):
            step(L.PREC_FP32, 0.0, 0.0)
        _, lfl_times = timed_steps(lambda: step(L.PREC_FP32, 0.0, 0.0), args.steps)
    lfl_ms = float(np.median(lfl_times))

    # ---- the plain FP32 GPU path: the same registrations one volume at a
    # time (batch 1, eager launches, no graph), on a sample of the series ----
    n_serial = min(24, T - 1)
    for i in range(2):
        ctx.register_linear(ref, moving[i:i + 1], flt, ITERS, L.RIGID, tolerance=TOL, use_graph=False,
                            certainty_sigma=cs)

    def serial():
        for i in range(n_serial):
            ctx.register_linear(ref, moving[i:i + 1], flt, ITERS, L.RIGID, tolerance=TOL, use_graph=False,
                                certainty_sigma=cs)
    with Section(sampler, "serial"):
        serial_rate = n_serial / (cuda_ms(serial, st) / 1000.0)

    # ---- the same batched step with the other filtering precisions ----
    other_arms = {}
    for name, p2 in (("fp32_batched", L.PREC_FP32), ("bf16x3_batched", L.PREC_BF16X3), ("tf32_batched", L.PREC_TF32)):
        if p2 == prec:
            continue
        with Section(sampler, name):
            for _ in range(2):
                step(p2)
            o2, b_times = timed_steps(lambda: step(p2), args.steps)
        other_arms[name] = {"value": (T - 1) * args.steps / (float(np.sum(b_times)) / 1000.0), "unit": UNIT,
                            "mean_iterations": float(o2["iterations"].float().mean()),
                            "sample": f"the same batched step with {name.split('_')[0].upper()} filtering"}

    # ---- dominant kernel alone: 7^3 filtering of the 199 moving volumes
    # (inputs 107 MB + responses 640 MB per launch, larger than L2) ----
    q = torch.empty((T - 1, 3, D, H, W, 2), dtype=torch.float32, device=dev)

    def time_filter(precision, nrep=20):
        def launch():
            L.lib().brc_filter3d(ctx.handle, ctypes.c_void_p(moving.data_ptr()), W, H, D, T - 1, V,
                                 fl.ctypes.data_as(ctypes.c_void_p), 3, precision, ctypes.c_void_p(q.data_ptr()))
        for _ in range(3):
            launch()

        def many():
            for _ in range(nrep):
                launch()
        return cuda_ms(many, st) / nrep

    with Section(sampler, "filter"):
        f_ms = time_filter(prec)
        filter_ms = {n: (time_filter(p2) if p2 != prec else f_ms)
                     for n, p2 in (("fp32", L.PREC_FP32), ("bf16x3", L.PREC_BF16X3), ("tf32", L.PREC_TF32))}
    ctx.synchronize()
    del q
    f_flop = FLOP_PER_VOXEL_FILTER * 3 * V * (T - 1)

    # ---- the other configurations (rank 0; single-GPU figures) ----
    extra = {}
    if rank == 0 and not args.skip_configs:
        with Section(sampler, "config0"):
            extra["config0_plain_fp32_affine"] = config0_rates(ctx, L, dev, cpu=not args.skip_cpu)
        with Section(sampler, "config3"):
            extra["differentiable"] = differentiable_rates(dev)
    if rank == 0 and not args.skip_normalisation:
        extra.update(normalisation_rates(ctx, L, prec, sampler, accuracy_on=not args.skip_accuracy))
    if sampler:
        sampler.stop()

    # ---- reduce over ranks ----
    t_max, e_max = max_over_ranks([ms, e2e_ms], world, dev)
    if rank != 0:
        return
    value = whole_job_rate(world, args.steps, t_max)
    e2e_value = whole_job_rate(world, args.steps, e_max)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
    clocks = sampler.section_summary("main") if sampler else None
    sm_max = clocks.get("sm_max_mhz") if clocks else None
    fp32_peak = 148 * 128 * 2 * (sm_max or 1965.0) * 1e6 / 1e12
    # DRAM bytes (read + write) per filtered volume of 64x64x33 from one ncu
    # capture of each kernel on 63 volumes, scaled to this launch by the
    # volume count (traffic grows with the volumes).  The tensor-core figure
    # is below the algorithmic bytes: the input comes partly from L2 (written
    # by the preceding resampling) and part of the output is still in L2
    # when the kernel ends.
    tc_bytes_per_vol = ((34503168 + 148295936) if prec == L.PREC_TF32 else (17850368 + 48461056)) / 63
    sym_bytes_per_vol = (34094848 + 147386624) / 63
    traffic = sym_bytes_per_vol * (T - 1) if symmetric_bank(fl) and tuple(SHAPE) == (33, 64, 64) else None
    tc_traffic = tc_bytes_per_vol * (T - 1) if tuple(SHAPE) == (33, 64, 64) else None
    achieved = f_flop / (f_ms / 1000.0) / 1e12
    bf16_peak = peaks.get("bf16_tflops", 1590.0)
    peak_src = "MEASURED_PEAKS.json bf16_tflops (burst, measured)" if "bf16_tflops" in peaks else "fallback 1.59 PFLOP/s"
    alg_note = ("algorithmic: 1,372 FLOP per voxel per complex filter (343 taps x 2 real MACs x 2) x 3 filters x the "
                "voxels of the 199 volumes; the split products and the banded-Toeplitz, row and halo padding the "
                "GEMMs also issue are not counted")
    if prec == L.PREC_TF32:
        tf32_peak = bf16_peak / 2.0
        roofline = {"kernel": "filter3d_tc_kernel<TF32> (tcgen05.mma.sp kind::tf32, 1:2 structured-sparse "
                              "banded taps, FP32 accumulate in TMEM)",
                    "bound": "tensor", "achieved": achieved, "peak": tf32_peak, "unit": "TFLOP/s",
                    "frac": achieved / tf32_peak,
                    "peak_source": peak_src + " / 2: the dense kind::tf32 rate is half the kind::f16 rate (a "
                                   "sparse K = 16 MMA multiplies the 8 stored values of each row: the useful "
                                   "rate stays bounded by the dense one)",
                    "frac_of_bf16_peak": achieved / bf16_peak,
                    "flop_per_launch": f_flop, "flop_note": alg_note, "launch_ms": f_ms,
                    "filter_launch_ms": filter_ms, "traffic": tc_traffic,
                    "traffic_note": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch on 63 "
                                    "volumes, scaled by the volume count; algorithmic: 4 B in + 24 B out "
                                    "per voxel"}
    elif prec == L.PREC_BF16X3:
        roofline = {"kernel": "filter3d_tc_kernel<BF16X3> (tcgen05.mma kind::f16, split BF16 x3, FP32 accumulate "
                              "in TMEM)",
                    "bound": "tensor", "achieved": achieved, "peak": bf16_peak, "unit": "TFLOP/s",
                    "frac": achieved / bf16_peak, "peak_source": peak_src,
                    "flop_per_launch": f_flop, "flop_note": alg_note,
                    "split_products": {"achieved": 3 * achieved, "frac": 3 * achieved / bf16_peak,
                                       "note": "the 3 BF16 products per tap the split form executes"},
                    "launch_ms": f_ms, "filter_launch_ms": filter_ms, "traffic": tc_traffic,
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
                    "flop_per_launch": f_flop, "launch_ms": f_ms, "filter_launch_ms": filter_ms, "traffic": traffic}
    acc = (accuracy(vols, truth, out["params"].cpu().numpy(), flt, cert_sigma=cs)
           if not args.skip_accuracy else None)
    cpu = cpu_baseline_protocol(vols, flt) if not args.skip_cpu else None
    lfl_rate = (T - 1) / (lfl_ms / 1000.0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": {L.PREC_BF16X3: "bf16x3", L.PREC_TF32: "tf32"}.get(prec, "f32"),
        "data": "synthetic",
        "config": workload_config(world, {"mean_iterations": float(iters_used.mean()),
                                          "precision": args.precision}, cert_sigma=cs),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(4 * V * T),
                "d2h_bytes_per_step": int(4 * V * (T - 1) + 4 * 15 * (T - 1))},
        "gpu_launches": int(launches),
        "roofline": roofline,
        "accuracy": acc,
        "like_for_like": {"value": lfl_rate, "unit": UNIT, "ms_per_step": lfl_ms,
                          "config": "the reference arm's configuration: FP32 filtering, all 20 iterations (no "
                                    "early exit), raw certainties, RIGID, the 199 registrations batched",
                          "over_cpu_baseline": (lfl_rate / cpu["value"]) if cpu else None},
        "plain_fp32_serial": {"value": serial_rate, "unit": UNIT,
                              "sample": f"{n_serial} volumes of the series registered one at a time "
                                        "(batch 1, eager launches)",
                              "batched_over_serial": value / serial_rate},
        "other_precisions": other_arms,
        "clocks": clocks,
        "clocks_all_sections": sampler.summary() if sampler else None,
        "cpu_baseline": cpu,
    }
    line.update(extra)
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
    ap.add_argument("--skip-configs", action="store_true",
                    help="skip the single FP32 affine registration and the differentiable objective "
                         "(configs 0 and 3)")
    ap.add_argument("--series", type=int, default=T, help="series length (volumes)")
    ap.add_argument("--precision", default="tf32", choices=["fp32", "bf16x3", "tf32"],
                    help="filtering precision of the timed path (tf32: tensor-core TF32; bf16x3: tensor-core "
                         "split BF16)")
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
