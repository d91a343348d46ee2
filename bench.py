#!/usr/bin/env python
"""Benchmark of the FWI2D wave-propagation hot path on B200.

Workload (one "step"): forward modeling of the whole plain-modeling survey -
151 x 501 cells at 10 m padded by a 100-cell absorbing boundary (351 x 701),
11 shots, 251 receivers, Ricker 30 Hz, dt 1 ms, nt 3001 (+119 delay samples) -
through libfwi2d's C ABI.  Metric: FD grid-point updates per second
(padded points x time steps x shots), whole job over all ranks.

  value     device-resident: model already in HBM, seismograms written to a
            device buffer; L2 flushed between timed steps (256 MiB write).
  e2e       fwi_set_model from pinned host memory + fwi_model_survey into a
            pinned host buffer, both inside the timed region.
  roofline  the forward-step kernel: 16 algorithmic bytes per grid-point
            update (read v, Q^t, Q^{t-1}; write Q^{t+1}) x points per launch,
            over the average launch time in the timed region.
  cpu_baseline  the oracle's float restatement of compute_pressure +
            compute_seismogram (OpenMP over all host cores) on the survey.
  batched_survey  RTM of the 240-shot windowed survey: forward and backward
            kernels' algorithmic GB/s against the HBM peak.
  rtm_benchmark_geometry  RTM and FWI-gradient kernels on the survey's
            geometry (100-cell random boundary), updates/s.
  fwi       FWI of the 81-shot and of the 240-shot windowed surveys: seconds
            per iteration, misfit and model error per iteration.

--impl reference runs the reference's own CUDA build (oracle/_ref/modeling.exe,
compiled from the reference sources for sm_100a) on the same survey and reports
updates / its own "Run time" (without that build it times the CPU port), and
times the reference's own forward, migration and adjoint loops on the same
geometry (oracle/_ref/ref_harness --time).

Multi-GPU (torchrun): every rank models its own copy of the survey (shots are
independent; no data-path collective) -> weak scaling; time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

HBM_FALLBACK_GBS = 6650.0
BYTES_PER_UPDATE = 16
WORKLOAD = ("plain modeling survey: 151x501 @10 m + 100-cell ABC (351x701), 11 shots, 251 receivers, "
            "30 Hz Ricker, dt 1 ms, nt 3001")


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


def traffic_from_profiles(plan: str):
    """DRAM bytes per launch of the forward kernel variant `plan` uses, from the
    committed ncu summaries of the benchmark survey (lines
    'dram_bytes_per_launch[<variant>]: <bytes>', <variant> as the plan string
    starts, e.g. 'loop TX=16 S=3' or 'resident').  Returns (bytes, source):
    the profile file the figure comes from, or (None, why) when no capture of
    this variant is committed, so a missing figure is reported as missing."""
    for f in sorted((ROOT / "profiles").glob("fwd_*_modeling_survey.md")):
        for m in re.finditer(r"dram_bytes_per_launch\[([^\]]+)\]:\s*([0-9.eE+]+)", f.read_text()):
            if plan.startswith(m.group(1)):
                return float(m.group(2)), f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of " \
                                          f"'{m.group(1)}' on this survey, {f.relative_to(ROOT)}"
    variant = plan.split("|")[0].strip()
    print(f"bench: no committed ncu capture of the forward variant '{variant}': roofline.traffic is null",
          file=sys.stderr)
    return None, f"missing: no ncu capture of '{variant}' in profiles/"


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(tempfile.mkstemp(suffix=".csv")[1])

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            t = [x.strip() for x in line.split(",")]
            if len(t) < 9:
                continue
            try:
                sm.append(float(t[1]))
                smax = float(t[2])
            except ValueError:
                continue
            for n, v in zip(names, t[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def make_case():
    from fwi2d_b200 import synth
    d = Path(tempfile.mkdtemp(prefix="fwi2d_bench_"))
    case, vp = synth.modeling_survey(d, seed=0)
    return case, vp


def updates_per_step(ctx):
    d = ctx.dims
    return d.nsrc * d.nzz * d.nxx * (d.nt + d.tlag)


def cpu_baseline(case, vp, budget_s: float = 15.0):
    """Oracle float restatement of the reference's stencil loop on all host
    cores: shots of the survey in order until all are done or budget_s passed."""
    from oracle import oracle as O
    nb = 100
    wav, tlag = O.wavelet(case.nt, case.dt, case.fmax)
    vel = O.expand(vp, nb)
    tab = O.b1d(nb, 0.004)
    rx = O.indices(case.rx, case.dh, nb)
    rz = O.indices(case.rz, case.dh, nb)
    nshots = len(case.sx)
    t0 = time.perf_counter()
    done = 0
    while done < nshots and (time.perf_counter() - t0) < budget_s:
        sx = O.indices(case.sx[done:done + 1], case.dh, nb)[0]
        sz = O.indices(case.sz[done:done + 1], case.dh, nb)[0]
        O.forward(vel, nb, tab, wav, case.nt, tlag, case.dt, case.dh, (sx, sz), rx, rz, bits=32)
        done += 1
    t = time.perf_counter() - t0
    ups = done * vel.size * (case.nt + tlag)
    return {"value": ups / t, "unit": "grid-pt updates/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{done} of {nshots} shots, full {case.nt + tlag} steps each on 351x701, float fields with the "
                      f"reference's double stencil sums, OpenMP over columns; {t:.2f} s"}


def run_reference(args, rank, world):
    case, vp = make_case()
    exe = ROOT / "oracle" / "_ref" / "modeling.exe"
    ups = 11 * 351 * 701 * (3001 + 119)
    line = {"metric": "FD grid-pt updates/s", "unit": "grid-pt updates/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded layered model)",
            "config": {"workload": WORKLOAD}}
    if rank != 0:
        return None
    if exe.exists():
        times = []
        for k in range(args.warmup + args.steps):
            r = subprocess.run([str(exe), str(case.params)], capture_output=True, text=True, cwd=str(case.root),
                               env=dict(os.environ, TERM=os.environ.get("TERM", "dumb")), timeout=900)
            if r.returncode != 0:
                print(json.dumps({"impl": "reference", "unavailable": f"reference modeling.exe failed: rc={r.returncode}"}))
                return None
            m = re.search(r"Run time:\s*([0-9.eE+-]+)", r.stdout)
            if k >= args.warmup:
                times.append(float(m.group(1)))
        t = max(times)
        value = ups / (sum(times) / len(times))
        line.update(value=value, ms_per_step=1e3 * sum(times) / len(times),
                    cpu_baseline={"value": value, "unit": "grid-pt updates/s", "cores": os.cpu_count(),
                                  "kind": "reference",
                                  "sample": "the reference's own CUDA build (oracle/_ref/modeling.exe: reference "
                                            "sources, FFTW via cuFFTW, sm_100a) on the full 11-shot survey, its "
                                            "'Run time' (shot loop incl. per-shot file writes); runs on the B200"},
                    e2e={"value": value, "unit": "grid-pt updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                    reference_build="oracle/_ref/modeling.exe", slowest_step_s=t,
                    note="the reference's 'Run time' covers its shot loop including a terminal clear and one "
                         "3 MB seismogram file write per shot; the other arm's e2e includes the host copies "
                         "but no file writes")
        if not args.no_batched:
            back = reference_backward(case, vp)
            if back:
                line["backward_loops"] = back
            fwi = reference_fwi_iteration()
            if fwi:
                line["fwi_iteration"] = fwi
    else:
        cb = cpu_baseline(case, vp)
        line.update(value=cb["value"], ms_per_step=None, cpu_baseline=dict(cb, kind="port"),
                    e2e={"value": cb["value"], "unit": cb["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    return line


def profile_case(which: str = "large"):
    """Forward surveys for ncu captures.  large: the FWI survey's grid
    (301x1701 + 100-cell ABC = 501x1901) with all 81 shots, nt 40 (277 steps),
    fields ~630 MB > L2.  small: the benchmark survey once (L2-resident)."""
    from fwi2d_b200 import api, synth
    d = Path(tempfile.mkdtemp(prefix="fwi2d_prof_"))
    if which == "unet":
        # the CNN preconditioner on one 301x1701 image: forward, MSE, backward
        import torch
        from fwi2d_b200 import cnn
        net = cnn.UNet(seed=0)
        H, W = 1701, 301
        x = torch.zeros(H * W * 16, dtype=torch.bfloat16, device="cuda")
        x.view(-1, 16)[:, :3] = torch.randn(H * W, 3, device="cuda").to(torch.bfloat16)
        t = torch.randn(H * W, device="cuda")
        for _ in range(2):
            net.forward(x, 1, H, W)
            net.mse(t)
            net.backward(x, net.dout)
        torch.cuda.synchronize()
        print("profile case done: unet", float(net.loss.item()))
        return
    if which == "unet-time":
        return unet_timing()
    if which == "batch-sweep":
        # RTM of the 240-shot survey with 240, 120 and 80 shots per batch
        peak, _ = peaks()
        out = {}
        for bs in (240, 120, 80):
            for nt in (300, 4001):
                r = batched_survey(peak, nt=nt, reps=2 if nt == 300 else 1, batch_shots=bs)
                out[f"{bs}_shots_nt{nt}"] = {
                    "forward_frac": r["forward"]["frac"], "backward_frac": r["backward"]["frac"],
                    "rtm_s": (r["forward"]["ms"] + r["backward"]["ms"]) / (2 if nt == 300 else 1) / 1e3,
                    "launches": r["forward"]["launches"], "peak_gbs": peak}
        print(json.dumps(out))
        return
    if which == "batched":
        # 60 of the 240 windowed shots (every 4th), nt 40: one RTM = one
        # forward and one backward multi-level launch, fields ~1.9 GB > L2
        case, _ = synth.aperture_survey(d, every=4, nt=40)
        with api.Context(case.params, api.MODE_MIGRATION) as ctx:
            dims = ctx.dims
            ctx.rtm_reset()
            ctx.rtm_survey_raw(np.zeros(dims.nsrc * dims.nrec * dims.nt, np.float32))
            print("profile case done:", ctx.describe())
        return
    if which == "small":
        case, _ = synth.modeling_survey(d, seed=0)
    elif which == "resident":
        # the benchmark survey with the shared-memory-resident kernel, nt 200
        case, _ = synth.modeling_survey(d, seed=0, nt=200, fwd_kernel="resident")
    else:
        case, _ = synth.fwi_survey(d, seed=2, nt=40)
    with api.Context(case.params, api.MODE_MODELING) as ctx:
        ctx.model_survey_raw()
        print("profile case done:", ctx.describe())


def unet_timing(reps: int = 20) -> None:
    """CUDA-event timing of the CNN preconditioner's kernels: one forward + MSE
    + backward pass on a 1701 x 301 image (the FWI model), one training step
    (pass + Adam) on 4 images of 501 x 151 (the training models), and each
    layer's forward, data-gradient and weight-gradient convolution alone.
    Prints one JSON line."""
    import torch

    from fwi2d_b200 import api, cnn
    L = api.lib()

    def timed(fn, n=reps):
        for _ in range(3):
            fn()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n * 1e3  # us

    def image(N, H, W):
        x = torch.zeros(N * H * W * cnn.IN_CH, dtype=torch.bfloat16, device="cuda")
        x.view(-1, cnn.IN_CH)[:, :3] = torch.randn(N * H * W, 3, device="cuda").to(torch.bfloat16)
        return x, torch.randn(N * H * W, device="cuda")

    out = {}
    for key, (N, H, W, adam) in {"pass_1701x301_us": (1, 1701, 301, False),
                                 "train_step_4x501x151_us": (4, 501, 151, True)}.items():
        net = cnn.UNet(seed=0)
        x, t = image(N, H, W)

        def step():
            net.forward(x, N, H, W)
            net.mse(t)
            net.backward(x, net.dout)
            if adam:
                net.adam()
        out[key] = round(timed(step), 1)
    net = cnn.UNet(seed=0)
    N, H, W = 1, 1701, 301
    x, t = image(N, H, W)
    net.forward(x, N, H, W)
    layers = {}
    for c in net.layers:
        h, w = net.dims[net.level[c.name]]
        src = net._input_of(c.name, x)
        y = torch.empty(N * h * w * c.cout, dtype=torch.bfloat16, device="cuda")
        gx = torch.empty(N * h * w * c.cin, dtype=torch.float32, device="cuda")
        dy = torch.randn(N * h * w * c.cout, device="cuda").to(torch.bfloat16)
        flop = 2.0 * N * h * w * 9 * c.cin * c.cout
        calls = {
            "fwd": lambda: L.fwi_nn_conv3x3(src.data_ptr(), N, h, w, c.cin, c.w16.data_ptr(), c.b.data_ptr(), c.cout,
                                            1, y.data_ptr(), None, None),
            "dgrad": lambda: L.fwi_nn_conv3x3(dy.data_ptr(), N, h, w, c.cout, c.wt16.data_ptr(), None, c.cin, 0, None,
                                              gx.data_ptr(), None),
            "wgrad": lambda: L.fwi_nn_conv3x3_wgrad(src.data_ptr(), dy.data_ptr(), N, h, w, c.cin, c.cout,
                                                    net.partial.data_ptr(), c.gw.data_ptr(), c.gb.data_ptr(), None),
        }
        row = {"size": f"{h}x{w}", "cin": c.cin, "cout": c.cout}
        for kind, fn in calls.items():
            us = timed(fn)
            row[kind + "_us"] = round(us, 1)
            row[kind + "_tflops"] = round(flop / us / 1e6, 1)
        layers[c.name] = row
    out["layers"] = layers
    if L.fwi_nn_check() != 0:
        raise RuntimeError("a bounded wait of the tensor-core kernels gave up")
    print(json.dumps(out))


def batched_survey(peak: float, nt: int = 300, reps: int = 2, batch_shots: int | None = None) -> dict:
    """HBM-bound companion measurement: the batched uneven-aperture survey
    (240 shots of the 301x1701 FWI model, each on its own window; the engine's
    default batches, or batch_shots per batch), RTM through the random boundary
    with nt time samples; forward and backward kernels timed by CUDA events on
    the engine stream."""
    from fwi2d_b200 import api, synth
    d = Path(tempfile.mkdtemp(prefix="fwi2d_batched_"))
    extra = {"batch_shots": batch_shots} if batch_shots else {}
    case, _ = synth.aperture_survey(d, nt=nt, **extra)
    with api.Context(case.params, api.MODE_MIGRATION) as ctx:
        dims = ctx.dims
        widths = [ctx.window(s)[1] for s in range(dims.nsrc)]
        data = np.zeros(dims.nsrc * dims.nrec * dims.nt, np.float32)
        ctx.rtm_reset()
        ctx.rtm_survey_raw(data)  # autotune + warm-up
        ctx.fwd_timing(True)
        for _ in range(reps):
            ctx.rtm_survey_raw(data)
        fms, fn, fu = ctx.fwd_timing_read()
        bms, bn, bu = ctx.bwd_timing_read()
        ctx.fwd_timing(False)
        plan = ctx.describe()
    fwd_gbs = 16 * fu / (fms * 1e-3) / 1e9
    bwd_gbs = 44 * bu / (bms * 1e-3) / 1e9
    return {
        "workload": f"{dims.nsrc} shots of the 301x1701 FWI model, aperture windows {min(widths)}-{max(widths)} "
                    f"columns (mean {np.mean(widths):.0f}) + 2x{dims.rbc_nb} boundary, {dims.nzz} rows, "
                    f"{dims.nt + dims.tlag} levels, RTM through the random boundary",
        "forward": {"updates_per_s": fu / (fms * 1e-3), "algorithmic_gbs": fwd_gbs, "frac": fwd_gbs / peak,
                    "bytes_per_update": 16, "launches": fn, "ms": fms},
        "backward": {"updates_per_s": bu / (bms * 1e-3), "algorithmic_gbs": bwd_gbs, "frac": bwd_gbs / peak,
                     "bytes_per_update": 44, "launches": bn, "ms": bms},
        "plans": plan,
    }


def rtm_benchmark_geometry(reps: int = 2) -> dict:
    """RTM and FWI-gradient back-propagation on the benchmark survey's geometry
    (11 shots, 351 x 701 padded, nt 3001 + 119 levels; migration in the
    Gaussian-smoothed model, as configuration 1), timed per kernel with CUDA
    events on the engine stream.  The reference arm times its own loops on the
    same geometry (oracle/_ref/ref_harness --time): forward_solver without ABC
    (modeling.cu:286-299), inject_seismogram + cross_correlation
    (migration.cu:61-81) and inject_adjoint + build_gradient
    (inversion.cu:230-248).  The input traces are seeded noise: the timing does
    not depend on their values."""
    from fwi2d_b200 import api, synth
    d = Path(tempfile.mkdtemp(prefix="fwi2d_rtm_"))
    case, vp = synth.modeling_survey(d, seed=0)
    smooth = synth.smooth_model(vp, case.dh, 150.0)
    out = {"workload": "RTM / FWI gradient of the plain modeling survey's geometry: 11 shots, 351x701 padded "
                       "(100-cell random boundary), 251 receivers, nt 3001 + 119 levels"}
    for mode, key in ((api.MODE_MIGRATION, "rtm"), (api.MODE_INVERSION, "gradient")):
        with api.Context(case.params, mode) as ctx:
            dims = ctx.dims
            data = (np.random.default_rng(1).standard_normal(dims.nsrc * dims.nrec * dims.nt) * 1e-3).astype(
                np.float32)
            ctx.set_model(smooth)
            if mode == api.MODE_MIGRATION:
                run = lambda: (ctx.rtm_reset(), ctx.rtm_survey_raw(data))
            else:
                ctx.set_observed_raw(data)
                run = lambda: ctx.compute_gradient(True)
            run()  # autotune + warm-up
            ctx.fwd_timing(True)
            t0 = time.perf_counter()
            for _ in range(reps):
                run()
            wall = (time.perf_counter() - t0) / reps
            fms, fn, fu = ctx.fwd_timing_read()
            bms, bn, bu = ctx.bwd_timing_read()
            ctx.fwd_timing(False)
            out[key] = {"backward_updates_per_s": bu / (bms * 1e-3), "backward_ms": bms / reps,
                        "forward_updates_per_s": fu / (fms * 1e-3), "forward_ms": fms / reps,
                        "survey_wall_s": wall, "plans": ctx.describe()}
    return out


FWI_VMIN, FWI_VMAX = 1400.0, 4800.0  # bounds of the FWI companion's velocity update (m/s)


def fwi_measure(case, vp_true: np.ndarray, iterations: int) -> dict:
    """The reference's FWI iteration (inversion_main.cpp:13-22: compute_gradient,
    optimization = two line-search modelings + the parabola, update_model;
    inversion.cu:111-358) from the 1-D depth-gradient model, through the C ABI;
    observed data modeled in the true model by the same engine.  The update is
    the reference's parabola step with the velocity bounded to [FWI_VMIN,
    FWI_VMAX] (fwi_update_model_bounded): the reference's unbounded update
    made the 81-shot survey's model unstable at its 4th iteration (non-finite
    misfit at the 5th).  Reports the wall time per iteration and the misfit
    and relative model RMS error after each."""
    import torch

    from fwi2d_b200 import api, synth
    init = synth.gradient_model(vp_true, case.dh)
    vt = vp_true.astype(np.float64)
    err = lambda v: float(np.sqrt(np.mean((v.astype(np.float64) - vt) ** 2)) / np.sqrt(np.mean(vt ** 2)))
    with api.Context(case.params, api.MODE_INVERSION) as ctx:
        dims = ctx.dims
        seis = torch.empty(dims.nsrc * dims.nrec * dims.nt, dtype=torch.float32, device="cuda")
        ctx.set_model(vp_true)
        ctx.model_survey_dev(seis.data_ptr())
        ctx.set_model(init)
        ctx.set_observed_dev(seis.data_ptr())
        torch.cuda.synchronize()
        res = {"shots": dims.nsrc, "grid": [dims.nzz, dims.nxx], "levels": dims.nt + dims.tlag,
               "iterations": iterations, "misfit": [], "model_error": [err(init)], "step": [], "seconds": []}
        for _ in range(iterations):
            t0 = time.perf_counter()
            sum_res = ctx.compute_gradient(True)
            f0 = float(np.sqrt(np.float32(sum_res)))
            step = ctx.optimization(f0)
            v = ctx.update_model_bounded(step, FWI_VMIN, FWI_VMAX)
            res["seconds"].append(time.perf_counter() - t0)
            res["misfit"].append(f0)
            res["step"].append(float(step))
            res["model_error"].append(err(v))
        res["update"] = f"the reference's parabola step, velocity bounded to [{FWI_VMIN:g}, {FWI_VMAX:g}] m/s"
        res["s_per_iteration"] = float(np.mean(res["seconds"]))
        res["shots_per_s"] = dims.nsrc / res["s_per_iteration"]
        res["plans"] = ctx.describe()
    return res


def fwi_surveys(iters_plain: int = 5, iters_batched: int = 1) -> dict:
    """Configurations 2 and 3 as FWI: the 81-shot survey on the 301x1701 dipping
    model (501x1901 padded, nt 4001) and the 240-shot survey of per-shot
    aperture windows on the same model."""
    from fwi2d_b200 import synth
    out = {}
    d = Path(tempfile.mkdtemp(prefix="fwi2d_fwi_"))
    for key, make, iters in (("plain_fwi", synth.fwi_survey, iters_plain),
                             ("batched_fwi", synth.aperture_survey, iters_batched)):
        if iters <= 0:
            continue
        try:
            case, vp = make(d / key)
            out[key] = fwi_measure(case, vp, iters)
        except Exception as e:  # report, never lose the headline line
            out[key] = {"error": f"{type(e).__name__}: {e}"}
    out["plain_fwi_workload"] = ("81 shots every 200 m, 851 receivers, 301x1701 @10 m dipping model + 100-cell "
                                 "boundaries, 15 Hz, dt 1 ms, nt 4001, 1-D depth-gradient start")
    out["batched_fwi_workload"] = ("240 shots every 70 m with aperture windows 300-1700 columns, same model, "
                                   "receivers and time axis, all shots of a propagation in one launch per batch")
    return out


def _harness_time(exe, case, vp, reps: int, seed: int = 1):
    """Run oracle/_ref/ref_harness --time on `case` (boundary velocity: the
    oracle's random boundary of the Gaussian-smoothed model, traces: seeded
    noise) and return its per-repetition rows."""
    from fwi2d_b200 import synth
    from oracle import oracle as O
    nb = 100
    smooth = synth.smooth_model(vp, case.dh, 150.0)
    base = O.expand(smooth, nb)
    bt = O.bumps(base.shape[1], base.shape[0], nb, case.dh, 200.0, 500.0, 0, 0)
    vel = O.rbc(base, nb, case.dh, 500.0, float(smooth.min()), float(smooth.max()), 0, 0, bt)
    vfile = case.root / "ref_vel.bin"
    np.ascontiguousarray(vel.T, dtype=np.float32).tofile(vfile)
    rng = np.random.default_rng(seed)
    for k in range(len(case.sx)):
        (rng.standard_normal(case.nt * len(case.rx)) * 1e-3).astype(np.float32).tofile(
            case.root / f"ref_data_{k + 1}.bin")
    r = subprocess.run([str(exe), "--time", str(case.params), str(vfile), str(case.root / "ref_data_"), str(reps)],
                       capture_output=True, text=True, cwd=str(case.root), timeout=900,
                       env=dict(os.environ, TERM=os.environ.get("TERM", "dumb")))
    if r.returncode != 0:
        raise RuntimeError(f"ref_harness --time rc={r.returncode}: {r.stderr[-300:]}")
    return [dict(kv.split("=") for kv in ln.split()[1:]) for ln in r.stdout.splitlines() if ln.startswith("time ")]


def reference_fwi_iteration() -> dict | None:
    """The reference's FWI iteration on the 81-shot survey (301 x 1701 + 100-cell
    boundaries, nt 4001), composed from its own loops timed once by
    ref_harness: per shot the residual modeling and the two line-search
    modelings (forward_solver, absorbing boundary on), the random-boundary
    forward and the adjoint back-propagation (inversion.cu:111-166, 286-342).
    Host work (file reads, the residual loop) is not included."""
    from fwi2d_b200 import synth
    exe = ROOT / "oracle" / "_ref" / "ref_harness"
    if not exe.exists():
        return None
    d = Path(tempfile.mkdtemp(prefix="fwi2d_ref_fwi_"))
    case, vp = synth.fwi_survey(d)
    try:
        row = _harness_time(exe, case, synth.gradient_model(vp, case.dh), reps=1)[0]
    except (RuntimeError, subprocess.TimeoutExpired) as e:
        return {"error": str(e)}
    ms = 3 * float(row["fwd_abc_ms"]) + float(row["fwd_ms"]) + float(row["grad_bwd_ms"])
    return {"workload": "the reference's loops on the 81-shot FWI survey: 501x1901 padded, nt 4001 + 237 levels",
            "s_per_iteration": ms * 1e-3, "shots_per_s": len(case.sx) / (ms * 1e-3),
            "composition": "3 x modeling forward (ABC) + random-boundary forward + adjoint back-propagation per "
                           "shot, the reference's kernels only",
            "modeling_forward_ms": float(row["fwd_abc_ms"]), "rbc_forward_ms": float(row["fwd_ms"]),
            "adjoint_ms": float(row["grad_bwd_ms"]), "reference_build": "oracle/_ref/ref_harness"}


def reference_backward(case, vp, reps: int = 3) -> dict | None:
    """The reference's own forward, migration and adjoint loops on the benchmark
    geometry, run by oracle/_ref/ref_harness --time (built from the reference
    sources; the boundary velocity is an input because the reference's
    random-boundary kernels index out of bounds), CUDA events per loop."""
    exe = ROOT / "oracle" / "_ref" / "ref_harness"
    if not exe.exists():
        return None
    try:
        rows = _harness_time(exe, case, vp, reps)
    except (RuntimeError, subprocess.TimeoutExpired) as e:
        return {"error": str(e)}
    rows = rows[1:] if len(rows) > 1 else rows  # the first repetition warms up
    ups = float(rows[0]["updates"])
    mean = lambda k: float(np.mean([float(x[k]) for x in rows]))
    return {"workload": "the reference's loops on the plain modeling survey's geometry: 11 shots, 351x701 padded, "
                        "nt 3001 + 119 levels, boundary velocity given",
            "forward_rbc": {"updates_per_s": ups / (mean("fwd_ms") * 1e-3), "ms": mean("fwd_ms")},
            "rtm_backward": {"updates_per_s": ups / (mean("rtm_bwd_ms") * 1e-3), "ms": mean("rtm_bwd_ms")},
            "gradient_backward": {"updates_per_s": ups / (mean("grad_bwd_ms") * 1e-3), "ms": mean("grad_bwd_ms")},
            "modeling_forward": {"updates_per_s": ups / (mean("fwd_abc_ms") * 1e-3), "ms": mean("fwd_abc_ms")},
            "reference_build": "oracle/_ref/ref_harness", "repetitions_timed": len(rows)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-survey companion measurement")
    ap.add_argument("--fwi-iterations", type=int, default=5,
                    help="FWI iterations of the 81-shot survey companion measurement (0: skip)")
    ap.add_argument("--fwi-batched-iterations", type=int, default=1,
                    help="FWI iterations of the 240-shot windowed survey companion measurement (0: skip)")
    ap.add_argument("--profile", nargs="?", const="large",
                    choices=["large", "small", "batched", "unet", "resident", "unet-time", "batch-sweep"],
                    help="for ncu: one forward survey (large: 81 shots on 501x1901, fields ~630 MB > L2, short "
                         "time axis; small: the benchmark survey); unet: the CNN's forward + backward; unet-time: "
                         "CUDA-event timing of the CNN's kernels; batch-sweep: RTM of the 240-shot survey in "
                         "batches of 240, 120 and 80 shots (both no ncu)")
    args = ap.parse_args()
    if args.profile:
        return profile_case(args.profile)
    rank, world, local = dist_env()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line:
            print(json.dumps(line))
        return

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from fwi2d_b200 import api
    case, vp = make_case()
    ctx = api.Context(case.params, api.MODE_MODELING)
    d = ctx.dims
    stream = torch.cuda.ExternalStream(ctx.stream)
    ups = updates_per_step(ctx)
    nseis = d.nsrc * d.nrec * d.nt
    d_seis = torch.empty(nseis, dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    # ---- device-resident timing
    for _ in range(args.warmup):
        ctx.model_survey_dev(d_seis.data_ptr())
    barrier()
    times = []
    launches0 = ctx.launches()
    ctx.fwd_timing(True)
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.model_survey_dev(d_seis.data_ptr())
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    launches = ctx.launches() - launches0
    k_ms, k_launches, k_updates = ctx.fwd_timing_read()
    ctx.fwd_timing(False)
    barrier()
    ms = float(np.mean(times))
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    value = world * ups / (ms * 1e-3)

    # ---- end to end through the C ABI with pinned host buffers
    h_model = torch.from_numpy(np.ascontiguousarray(vp.T).ravel()).pin_memory()
    h_seis = torch.empty(nseis, dtype=torch.float32).pin_memory()
    fptr = lambda t: api.C.cast(t.data_ptr(), api._F)
    e2e_times = []
    for k in range(args.warmup + args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx._check(ctx._lib.fwi_set_model(ctx._h, fptr(h_model)))
        ctx._check(ctx._lib.fwi_model_survey(ctx._h, fptr(h_seis)))
        e1.record(stream)
        e1.synchronize()
        if k >= args.warmup:
            e2e_times.append(e0.elapsed_time(e1))
    e2e_ms = float(np.mean(e2e_times))
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())

    peak, peak_kind = peaks()
    n_steps = d.nt + d.tlag
    plan = ctx.describe()
    # dominant kernel: the forward propagation kernel, timed by CUDA events on
    # the context stream around each of its launches inside the timed region
    bytes_per_launch = BYTES_PER_UPDATE * k_updates / k_launches
    avg_launch_ms = k_ms / k_launches
    achieved = bytes_per_launch / (avg_launch_ms * 1e-3) / 1e9
    traffic, traffic_src = traffic_from_profiles(plan)
    line = {
        "metric": "FD grid-pt updates/s", "value": value, "unit": "grid-pt updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded 4-layer + anomaly model, 151x501 at 10 m)",
        "config": {"workload": WORKLOAD, "shots_per_rank": d.nsrc, "grid": [d.nzz, d.nxx], "time_steps": n_steps,
                   "boundary": "100-cell absorbing boundary (ABC), as the reference's modeling.exe models",
                   "l2": "flushed (256 MiB write) between timed steps", "parallelism": f"shot replicas x{world}"},
        "e2e": {"value": world * ups / (e2e_ms * 1e-3), "unit": "grid-pt updates/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(h_model.numel() * 4), "d2h_bytes_per_step": int(nseis * 4)},
        "roofline": {"bound": "hbm", "kernel": "forward step (" + plan + ")", "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_source": traffic_src,
                     "algorithmic_bytes_per_launch": bytes_per_launch,
                     "avg_launch_us": 1e3 * avg_launch_ms, "launches_timed": k_launches,
                     "kernel_share_of_step": k_ms / (ms * args.steps),
                     "note": "achieved = 16 B per grid-point update x updates per launch / average launch time "
                             "(CUDA events around each forward-kernel launch on the context stream); one "
                             "multi-level launch covers all time levels of the batch; traffic = ncu DRAM "
                             "read+write bytes of that launch (profiles/); the 11-shot working set (~23 MB) fits "
                             "on chip: the 'resident' kernel keeps both time levels in the SMs' shared memory and "
                             "reads HBM once per launch, so frac is its speed against streaming the fields from "
                             "HBM at the measured peak, and its own limit is SM instruction issue"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(case, vp)
    if world == 1 and not args.no_batched:
        ctx.close()
        line["batched_survey"] = batched_survey(peak)
        line["rtm_benchmark_geometry"] = rtm_benchmark_geometry()
    if world == 1 and args.fwi_iterations > 0:
        ctx.close()
        line["fwi"] = fwi_surveys(args.fwi_iterations, args.fwi_batched_iterations)
    ctx.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
