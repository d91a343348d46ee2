"""Training data, training and FWI with the CNN preconditioner (fwi2d_b200.cnn).

  pairs:  for seeded random models (dipping layers + anomalies + water layer,
          the family of the FWI benchmark model) the FD engine models observed
          data in the true model and accumulates the raw gradient and source
          illumination in a 1-D depth-gradient starting model; the network
          input is (gradient, illumination, starting velocity) and the target
          the slowness^2 update direction (m_start - m_true), normalised by its
          max |.| (the engine normalises every direction the same way).
  train:  Adam on the mean-squared error, mini-batches of images.
  fwi:    the reference's iteration (inversion.cu:111-166, 286-358) with the
          network's direction in place of the illumination-normalised
          gradient; when the 3-point parabolic line search along it does not
          cut the misfit (no trial below f0, or a non-positive / non-finite
          step) the iteration falls back to the plain gradient.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import api, cnn, synth
from .sharded import DeviceFloats


def _torch():
    import torch
    return torch


@dataclass
class PairSetup:
    nz: int = 151
    nx: int = 501
    dh: float = 10.0
    nt: int = 2001
    dt: float = 1e-3
    fmax: float = 15.0
    nshots: int = 11
    nrec: int = 251
    boundary: float = 490.0  # abc / rbc length (50 cells at 10 m)


def write_setup(root, s: PairSetup, vp: np.ndarray) -> synth.Case:
    w = (s.nx - 1) * s.dh
    sx = np.linspace(0.0, w, s.nshots)
    rx = np.linspace(0.0, w, s.nrec)
    return synth.write_case(root, vp, s.dh, s.nt, s.dt, s.fmax, sx, np.full(s.nshots, 10.0), rx,
                            np.full(s.nrec, 10.0), abc_length=s.boundary, inv_rbc_length=s.boundary,
                            mig_rbc_length=s.boundary, inv_rbc_ratio=200, inv_rbc_varVp=500, depth_mask=0)


def true_model(s: PairSetup, seed: int) -> np.ndarray:
    return synth.dipping_model(s.nz, s.nx, s.dh, seed)


def start_model(v: np.ndarray, dh: float) -> np.ndarray:
    return synth.gradient_model(v, dh)


def _grid_dev(a: np.ndarray):
    """(nz, nx) host array -> device float32 in the engine's z-fastest order."""
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float32).T).ravel()).cuda()


_SCRATCH = {}


def features(ctx: api.Context, vp_dev, out) -> None:
    """Pack the context's raw accumulators and the velocity into NHWC bf16."""
    torch = _torch()
    a, b, n = ctx.accumulators()
    g = torch.as_tensor(DeviceFloats(a, n), device="cuda")
    il = torch.as_tensor(DeviceFloats(b, n), device="cuda")
    if "bits" not in _SCRATCH:
        _SCRATCH["bits"] = torch.zeros(2, dtype=torch.int32, device="cuda")
    d = ctx.dims
    cnn.pack(g, il, vp_dev, d.nz, d.nx, out, _SCRATCH["bits"])


VMIN, VMAX = 1400.0, 4800.0  # bounds of the safeguarded update (the model family spans 1500-4800 m/s)


STEP_CAP = 4.0  # largest step, in units of the second trial step a2


def line_search(ctx: api.Context, f0: float, cap: float | None = STEP_CAP) -> tuple[float, float, float]:
    """Trials at a1, a2 along the context's direction; returns (step, f1, f2).
    The step is the parabola's vertex (inversion.cu:286-308) when it is
    positive and finite, clipped to cap * a2 (the vertex of a parabola fitted
    on [0, a2] extrapolates badly far beyond it; None: no clip), else the
    better trial when it cut the misfit, else 0."""
    a1, a2 = ctx.trial_steps()
    f1 = float(np.sqrt(np.float32(ctx.linesearch_trial(a1))))
    f2 = float(np.sqrt(np.float32(ctx.linesearch_trial(a2))))
    step = ctx.parabola_step(f0, f1, f2)
    if np.isfinite(step) and step > 0.0:
        if cap is not None:
            step = min(step, cap * a2)
    else:
        fb, ab = min((f1, a1), (f2, a2))
        step = ab if fb < f0 else 0.0
    return step, f1, f2


TRAIN_SEED0 = 1000  # training models use seeds TRAIN_SEED0 ..; test models use seeds below it


def make_pairs(root, models: int, stages: int = 4, seed0: int = TRAIN_SEED0, setup: PairSetup = PairSetup(),
               log=print, net: cnn.UNet | None = None):
    """models x stages pairs -> (X: [n, P*16] bf16, T: [n, P] float32) on the device.
    Stage k of a model is its k-th FWI iterate from the 1-D start: plain FWI,
    or, given a network, the network-preconditioned iteration of fwi() (pairs
    along the trajectories the preconditioner itself takes, whose models are
    much closer to the truth than plain FWI's after the first step)."""
    torch = _torch()
    root = Path(root)
    s = setup
    case = write_setup(root, s, true_model(s, seed0))
    P = s.nz * s.nx
    n = models * stages
    X = torch.empty((n, P * 16), dtype=torch.bfloat16, device="cuda")
    T = torch.empty((n, P), dtype=torch.float32, device="cuda")
    t0 = time.perf_counter()
    with api.Context(case.params, api.MODE_INVERSION) as ctx:
        d = ctx.dims
        seis = torch.empty(d.nsrc * d.nrec * d.nt, dtype=torch.float32, device="cuda")
        k = 0
        for mi in range(models):
            vt = true_model(s, seed0 + mi)
            ctx.set_model(vt)
            ctx.model_survey_dev(seis.data_ptr())
            ctx.set_model(start_model(vt, s.dh))
            ctx.set_observed_dev(seis.data_ptr())
            ctx.set_seed(seed0 + mi)
            mt = 1.0 / vt.astype(np.float64) ** 2
            for st in range(stages):
                v = ctx.get_model()
                sum_res = ctx.gradient_accumulate(True)
                features(ctx, _grid_dev(v), X[k])
                dm = 1.0 / v.astype(np.float64) ** 2 - mt
                T[k].copy_(_grid_dev((dm / max(np.abs(dm).max(), 1e-30)).astype(np.float32)))
                k += 1
                if st + 1 < stages:
                    ctx.gradient_finish()
                    f0 = float(np.sqrt(np.float32(sum_res)))
                    if net is not None:
                        _network_direction(ctx, net, X[k - 1])
                        step, f1, f2 = line_search(ctx, f0)
                        if step <= 0.0 or min(f1, f2) >= f0:
                            ctx.gradient_finish()  # back to the illumination-normalised gradient
                            step, _, _ = line_search(ctx, f0)
                    else:
                        step, _, _ = line_search(ctx, f0)
                    ctx.update_model_bounded(step, VMIN, VMAX)
            if log and (mi + 1) % max(1, models // 8) == 0:
                log(f"pairs {k}/{n} ({time.perf_counter() - t0:.1f} s)")
    return X, T


def _network_direction(ctx: api.Context, net: cnn.UNet, x) -> None:
    """Set the context's search direction to the network's output for the
    packed input x (the context's current accumulators and model)."""
    torch = _torch()
    d = ctx.dims
    if "dir" not in _SCRATCH or _SCRATCH["dir"].numel() != d.nz * d.nx:
        _SCRATCH["dir"] = torch.empty(d.nz * d.nx, dtype=torch.float32, device="cuda")
    y = net.forward(x, 1, d.nx, d.nz)
    cnn.direction(net, y, d.nz, d.nx, _SCRATCH["dir"])
    torch.cuda.synchronize()
    ctx.set_direction_dev(_SCRATCH["dir"].data_ptr())


def train(net: cnn.UNet, X, T, setup: PairSetup = PairSetup(), epochs: int = 30, batch: int = 4, lr: float = 1e-3,
          val: int = 32, seed: int = 0, log=print) -> dict:
    """Adam on the first len(X) - val pairs; returns loss history (train / validation)."""
    torch = _torch()
    n = X.shape[0]
    ntr = n - val
    H, W = setup.nx, setup.nz
    P = H * W
    rng = np.random.default_rng(seed)
    hist = {"train": [], "val": []}
    xb = torch.empty((batch, P * 16), dtype=torch.bfloat16, device="cuda")
    tb = torch.empty((batch, P), dtype=torch.float32, device="cuda")
    t0 = time.perf_counter()
    for ep in range(epochs):
        order = rng.permutation(ntr)
        tot = 0.0
        for i in range(0, ntr - batch + 1, batch):
            idx = torch.from_numpy(order[i:i + batch]).cuda()
            torch.index_select(X, 0, idx, out=xb)
            torch.index_select(T, 0, idx, out=tb)
            net.forward(xb, batch, H, W)
            net.mse(tb)
            net.backward(xb, net.dout)
            net.adam(lr=lr)
            tot += float(net.loss.item()) / (batch * P)
        hist["train"].append(tot / max(1, ntr // batch))
        hist["val"].append(evaluate(net, X[ntr:], T[ntr:], setup, batch))
        if log:
            log(f"epoch {ep + 1}/{epochs}: train {hist['train'][-1]:.4g} val {hist['val'][-1]:.4g} "
                f"({time.perf_counter() - t0:.1f} s)")
    return hist


def evaluate(net: cnn.UNet, X, T, setup: PairSetup, batch: int) -> float:
    torch = _torch()
    H, W = setup.nx, setup.nz
    P = H * W
    tot, cnt = 0.0, 0
    for i in range(0, X.shape[0] - batch + 1, batch):
        net.forward(X[i:i + batch].contiguous(), batch, H, W)
        net.mse(T[i:i + batch].contiguous())
        tot += float(net.loss.item()) / (batch * P)
        cnt += 1
    return tot / max(1, cnt)


@dataclass
class FwiLog:
    residuo: list = field(default_factory=list)
    model_error: list = field(default_factory=list)
    seconds: list = field(default_factory=list)
    direction: list = field(default_factory=list)  # "cnn" / "gradient" / "fallback"


def model_error(v: np.ndarray, v_true: np.ndarray) -> float:
    v = v.astype(np.float64)
    t = v_true.astype(np.float64)
    return float(np.sqrt(np.mean((v - t) ** 2)) / np.sqrt(np.mean(t ** 2)))


def fwi(ctx: api.Context, v_true: np.ndarray, iterations: int, net: cnn.UNet | None = None, log=print,
        cap: float | None = STEP_CAP) -> FwiLog:
    """Plain (net None) or CNN-preconditioned FWI from the context's model;
    both take the safeguarded step of line_search and the bounded update."""
    torch = _torch()
    d = ctx.dims
    out = FwiLog()
    x = torch.empty(d.nz * d.nx * 16, dtype=torch.bfloat16, device="cuda") if net else None
    direction = torch.empty(d.nz * d.nx, dtype=torch.float32, device="cuda") if net else None
    out.model_error.append(model_error(ctx.get_model(), v_true))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for it in range(iterations):
        sum_res = ctx.gradient_accumulate(True)
        f0 = float(np.sqrt(np.float32(sum_res)))
        out.residuo.append(f0)
        ctx.gradient_finish()
        used = "gradient"
        if net is not None:
            vp = _grid_dev(ctx.get_model())
            features(ctx, vp, x)
            y = net.forward(x, 1, d.nx, d.nz)
            cnn.direction(net, y, d.nz, d.nx, direction)
            torch.cuda.synchronize()
            ctx.set_direction_dev(direction.data_ptr())
            used = "cnn"
        step, f1, f2 = line_search(ctx, f0, cap)
        if net is not None and (step <= 0.0 or min(f1, f2) >= f0):
            ctx.gradient_finish()  # back to the illumination-normalised gradient
            used = "fallback"
            step, f1, f2 = line_search(ctx, f0, cap)
        v = ctx.update_model_bounded(step, VMIN, VMAX)
        out.direction.append(used)
        out.model_error.append(model_error(v, v_true))
        out.seconds.append(time.perf_counter() - t0)
        if log:
            log(f"iteration {it + 1}: residuo {f0:.5g} step {step:.3g} ({used}) model error "
                f"{100 * out.model_error[-1]:.2f} % at {out.seconds[-1]:.1f} s")
    return out


THRESHOLDS = (0.12, 0.11, 0.10, 0.09, 0.08, 0.07, 0.06, 0.05, 0.04, 0.03)  # relative model RMS error


def time_to_error(log: FwiLog, target: float) -> float | None:
    """Seconds until the model error first reaches `target` (None if never)."""
    for e, t in zip(log.model_error[1:], log.seconds):
        if e <= target:
            return t
    return None


def main(argv=None) -> int:
    """Train the preconditioner and compare CNN-preconditioned with plain FWI.

    python -m fwi2d_b200.precond --models 512 --stages 4 --epochs 60 --iterations 10 --test small|aperture
        [--follow-stages 4 --follow-epochs 30]
    writes a JSON summary (--out) with the training history and both runs'
    misfit, model-error and wall-time trajectories."""
    import argparse
    import json
    import tempfile

    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--models", type=int, default=128)
    ap.add_argument("--stages", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--iterations", type=int, default=10)
    ap.add_argument("--test", choices=["small", "aperture"], default="small")
    ap.add_argument("--nt", type=int, default=None, help="time samples of the aperture-survey test (default 4001)")
    ap.add_argument("--target", type=float, default=0.03)
    ap.add_argument("--out", default=None)
    ap.add_argument("--weights", default=None, help="save / load the trained network here")
    ap.add_argument("--follow-stages", type=int, default=0,
                    help="after training, make this many more pairs per model along the network's own FWI "
                         "trajectories and continue training on all pairs (0: off)")
    ap.add_argument("--follow-epochs", type=int, default=30)
    a = ap.parse_args(argv)
    root = Path(tempfile.mkdtemp(prefix="fwi2d_precond_"))
    s = PairSetup()
    res = {"setup": vars(a)}
    net = cnn.UNet(seed=0)
    t0 = time.perf_counter()
    if a.weights and Path(a.weights).exists():
        net.load(a.weights)
        res["training"] = {"loaded": a.weights}
    else:
        X, T = make_pairs(root / "pairs", a.models, a.stages, setup=s)
        t1 = time.perf_counter()
        hist = train(net, X, T, s, epochs=a.epochs, batch=4, lr=1e-3, val=8 * a.stages)
        t2 = time.perf_counter()
        res["training"] = {"pairs": int(X.shape[0]), "pair_seconds": t1 - t0, "train_seconds": t2 - t1, **hist}
        if a.follow_stages > 0:
            X2, T2 = make_pairs(root / "pairs_follow", a.models, a.follow_stages, setup=s, net=net)
            X = torch.cat([X, X2])
            T = torch.cat([T, T2])
            del X2, T2
            t3 = time.perf_counter()
            hist2 = train(net, X, T, s, epochs=a.follow_epochs, batch=4, lr=5e-4, val=8 * a.stages, seed=1)
            t4 = time.perf_counter()
            res["training_follow"] = {"pairs": int(X.shape[0]), "pair_seconds": t3 - t2, "train_seconds": t4 - t3,
                                      **hist2}
        del X, T
        if a.weights:
            net.save(a.weights)
    if a.test == "small":
        vt = true_model(s, 7)
        case = write_setup(root / "test", s, vt)
        vs = start_model(vt, s.dh)
    else:
        kw = {"nt": a.nt} if a.nt else {}
        case, vt = synth.aperture_survey(root / "test", **kw)
        vs = synth.gradient_model(vt, case.dh)
    runs = {}
    for mode in ("plain", "cnn"):
        with api.Context(case.params, api.MODE_INVERSION) as ctx:
            d = ctx.dims
            seis = torch.empty(d.nsrc * d.nrec * d.nt, dtype=torch.float32, device="cuda")
            ctx.set_model(vt)
            ctx.model_survey_dev(seis.data_ptr())
            ctx.set_model(vs)
            ctx.set_observed_dev(seis.data_ptr())
            ctx.set_seed(7)
            lg = fwi(ctx, vt, a.iterations, net if mode == "cnn" else None)
            runs[mode] = {"residuo": lg.residuo, "model_error": lg.model_error, "seconds": lg.seconds,
                          "direction": lg.direction, "time_to_target": time_to_error(lg, a.target),
                          "time_to": {f"{t:.3f}": time_to_error(lg, t) for t in THRESHOLDS}}
    res["runs"] = runs
    txt = json.dumps(res)
    if a.out:
        Path(a.out).write_text(txt)
    print(txt)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
