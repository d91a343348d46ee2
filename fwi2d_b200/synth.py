"""Seeded synthetic inputs in the reference's file formats.

Writes what the reference's run/generate_setup.py and a model file would give
the executables: a velocity model (nz x nx float32, z fastest), SPS / RPS
geometry files ("x,z" per line, "%.2f") and a parameters.txt with the
reference's keys (run/parameters.txt).  The model families are the benchmark
workloads of this project:

* ``layered``  4 flat layers 1500/2000/2700/3500 m/s at random depths and one
  Gaussian anomaly of +-300 m/s, sigma 200 m (plain modeling / RTM survey);
* ``dipping``  a 300 m water layer at 1500 m/s over 8 dipping layers from 1500 to
  4500 m/s and 3 Gaussian anomalies (FWI surveys).

No public dataset is involved; every array comes from a numpy Generator seeded
by the caller.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np


def gaussian_bump(nz, nx, dh, zc, xc, sigma, amp):
    z = np.arange(nz)[:, None] * dh
    x = np.arange(nx)[None, :] * dh
    return amp * np.exp(-0.5 * ((z - zc) ** 2 + (x - xc) ** 2) / sigma**2)


def layered_model(nz: int, nx: int, dh: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    speeds = [1500.0, 2000.0, 2700.0, 3500.0]
    depth = (nz - 1) * dh
    tops = np.sort(rng.uniform(0.15, 0.85, 3)) * depth
    z = np.arange(nz)[:, None] * dh * np.ones((1, nx))
    v = np.full((nz, nx), speeds[0])
    for k, t in enumerate(tops):
        v[z >= t] = speeds[k + 1]
    amp = 300.0 * rng.choice([-1.0, 1.0])
    v += gaussian_bump(nz, nx, dh, rng.uniform(0.3, 0.7) * depth, rng.uniform(0.3, 0.7) * (nx - 1) * dh, 200.0, amp)
    return v.astype(np.float32)


def dipping_model(nz: int, nx: int, dh: float, seed: int, water: float = 300.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    depth, width = (nz - 1) * dh, (nx - 1) * dh
    speeds = np.linspace(1500.0, 4500.0, 8)
    z = np.arange(nz)[:, None] * dh
    x = np.arange(nx)[None, :] * dh
    tops = np.sort(rng.uniform(water, depth * 0.95, 7))
    dips = rng.uniform(-0.08, 0.08, 7)
    v = np.full((nz, nx), speeds[0])
    for k in range(7):
        surface = tops[k] + dips[k] * (x - width / 2)
        v = np.where(z >= surface, speeds[k + 1], v)
    for _ in range(3):
        v += gaussian_bump(nz, nx, dh, rng.uniform(water + 200, depth - 200), rng.uniform(0.1, 0.9) * width,
                           200.0, 300.0 * rng.choice([-1.0, 1.0]))
    v[z[:, 0] < water, :] = 1500.0
    return v.astype(np.float32)


def smooth_model(v: np.ndarray, dh: float, sigma_m: float, keep_top_m: float = 0.0) -> np.ndarray:
    """Gaussian smoothing of the slowness (as run/generate_setup.py:44-49 does), keeping the top rows."""
    from scipy.ndimage import gaussian_filter

    out = 1.0 / gaussian_filter(1.0 / v.astype(np.float64), sigma_m / dh)
    k = int(keep_top_m / dh)
    out[:k] = v[:k]
    return out.astype(np.float32)


def gradient_model(v: np.ndarray, dh: float, water: float = 300.0, vmax: float | None = None) -> np.ndarray:
    """1-D depth-gradient initial model: water velocity above `water`, then a linear ramp."""
    nz, nx = v.shape
    z = np.arange(nz) * dh
    top = 1500.0
    bottom = float(vmax if vmax is not None else np.percentile(v[-nz // 5:], 50))
    prof = np.where(z < water, top, top + (bottom - top) * (z - water) / max(z[-1] - water, 1.0))
    return np.repeat(prof[:, None], nx, axis=1).astype(np.float32)


def mute_direct(data: np.ndarray, sx: float, sz: float, rx: np.ndarray, rz: np.ndarray, dt: float,
                velocity: float, time_delay: float, gstd: float = 30.0) -> np.ndarray:
    """Direct-wave mute of run/generate_input_data.py:22-44: normalise by max |d|,
    then taper each trace before (distance/velocity + time_delay) with a Gaussian."""
    nt = data.shape[0]
    d = data / np.max(np.abs(data))
    dist = np.sqrt((rx - sx) ** 2 + (rz - sz) ** 2)
    tid = ((dist / velocity + time_delay) / dt).astype(int)
    t = np.arange(nt)
    for r in range(d.shape[1]):
        k = min(max(tid[r], 0), nt)
        d[:k, r] *= np.exp(-0.5 * ((t[:k] - tid[r]) / gstd) ** 2)
    return d.astype(np.float32)


@dataclass
class Case:
    """One survey on disk (paths relative to `root`)."""
    root: Path
    nz: int
    nx: int
    dh: float
    nt: int
    dt: float
    fmax: float
    sx: np.ndarray
    sz: np.ndarray
    rx: np.ndarray
    rz: np.ndarray
    keys: dict = field(default_factory=dict)

    @property
    def params(self) -> Path:
        return self.root / "parameters.txt"


def write_case(root: str | os.PathLike, vp: np.ndarray, dh: float, nt: int, dt: float, fmax: float, sx, sz, rx, rz,
               **keys) -> Case:
    """Write model.bin, SPS.txt, RPS.txt and parameters.txt under root."""
    root = Path(root)
    root.mkdir(parents=True, exist_ok=True)
    nz, nx = vp.shape
    (root / "data").mkdir(exist_ok=True)
    (root / "out").mkdir(exist_ok=True)
    np.ascontiguousarray(vp.T, dtype=np.float32).tofile(root / "model.bin")
    sx, sz, rx, rz = (np.asarray(a, dtype=np.float64) for a in (sx, sz, rx, rz))
    np.savetxt(root / "SPS.txt", np.stack([sx, sz], 1), fmt="%.2f", delimiter=",")
    np.savetxt(root / "RPS.txt", np.stack([rx, rz], 1), fmt="%.2f", delimiter=",")
    base = {
        "x_samples": nx, "z_samples": nz, "model_spacing": dh, "model_file": f"{root}/model.bin",
        "SPS": f"{root}/SPS.txt", "RPS": f"{root}/RPS.txt",
        "time_samples": nt, "time_spacing": dt, "max_frequency": fmax,
        "abc_length": 990, "abc_factor": 0.004, "mod_output_folder": f"{root}/data/",
        "max_iteration": 5, "depth_mask": 0, "inv_rbc_ratio": 200, "inv_rbc_varVp": 500, "inv_rbc_length": 990,
        "inv_input_folder": f"{root}/data/", "inv_input_prefix": f"seismogram_nt{nt}_nr{len(rx)}_{int(np.float32(1e6) * np.float32(dt))}us_shot_",
        "inv_output_folder": f"{root}/out/", "inv_residuo_folder": f"{root}/out/",
        "mig_rbc_ratio": 200, "mig_rbc_varVp": 500, "mig_rbc_length": 990,
        "mig_input_folder": f"{root}/data/", "mig_input_prefix": "input_RTM_", "mig_output_folder": f"{root}/out/",
    }
    base.update(keys)
    lines = ["# written by fwi2d_b200.synth"] + [f"{k} = {v}" for k, v in base.items()]
    (root / "parameters.txt").write_text("\n".join(lines) + "\n")
    return Case(root, nz, nx, dh, nt, dt, fmax, sx, sz, rx, rz, base)


# ---------------------------------------------------------------- workloads
def modeling_survey(root, seed: int = 0, **over) -> tuple[Case, np.ndarray]:
    """Plain forward modeling: 151 x 501 at 10 m, 11 shots every 500 m,
    251 receivers every 20 m at 10 m depth, 30 Hz, dt 1 ms, nt 3001, 100-cell boundary."""
    nz, nx, dh = 151, 501, 10.0
    vp = layered_model(nz, nx, dh, seed)
    sx = np.arange(11) * 500.0
    rx = np.arange(251) * 20.0
    kw = dict(nt=3001, dt=1e-3, fmax=30.0)
    kw.update({k: over.pop(k) for k in list(over) if k in kw})
    case = write_case(root, vp, dh, kw["nt"], kw["dt"], kw["fmax"], sx, np.full(11, 10.0), rx, np.full(251, 10.0),
                      **over)
    return case, vp


def fwi_survey(root, seed: int = 2, **over) -> tuple[Case, np.ndarray]:
    """Plain FWI: 301 x 1701 at 10 m, 81 shots every 200 m, 851 receivers every
    20 m, 15 Hz, dt 1 ms, nt 4001, 100-cell boundaries."""
    nz, nx, dh = 301, 1701, 10.0
    vp = dipping_model(nz, nx, dh, seed)
    sx = np.arange(81) * 200.0 + 500.0
    sx = sx[sx <= (nx - 1) * dh]
    rx = np.arange(851) * 20.0
    kw = dict(nt=4001, dt=1e-3, fmax=15.0)
    kw.update({k: over.pop(k) for k in list(over) if k in kw})
    case = write_case(root, vp, dh, kw["nt"], kw["dt"], kw["fmax"], sx, np.full(sx.size, 10.0), rx,
                      np.full(851, 10.0), **over)
    return case, vp


def aperture_survey(root, seed: int = 3, every: int = 1, **over) -> tuple[Case, np.ndarray]:
    """Batched uneven-aperture FWI: the FWI survey's model and receiver spread,
    240 shots every 70 m, each modeled on the columns within its own maximum
    offset (uniform 1.5-8 km from the seed; windows of about 300-1700 columns).
    every > 1 keeps every every-th shot (smaller profiling cases)."""
    nz, nx, dh = 301, 1701, 10.0
    vp = dipping_model(nz, nx, dh, 2)
    sx = np.arange(240) * 70.0 + 100.0
    rx = np.arange(851) * 20.0
    rng = np.random.default_rng(seed)
    offsets = rng.uniform(1500.0, 8000.0, sx.size).astype(np.float32)
    sx, offsets = sx[::every], offsets[::every]
    kw = dict(nt=4001, dt=1e-3, fmax=15.0)
    kw.update({k: over.pop(k) for k in list(over) if k in kw})
    root = Path(root)
    root.mkdir(parents=True, exist_ok=True)
    write_offsets(root / "offsets.txt", offsets)
    over.setdefault("aperture_file", f"{root}/offsets.txt")
    case = write_case(root, vp, dh, kw["nt"], kw["dt"], kw["fmax"], sx, np.full(sx.size, 10.0), rx,
                      np.full(851, 10.0), **over)
    return case, vp


def write_offsets(path, offsets) -> None:
    """One maximum offset (metres) per shot, as the key aperture_file reads them."""
    Path(path).write_text("".join(f"{float(np.float32(o)):.6g}\n" for o in offsets))


def small_case(root, seed: int = 5, nz: int = 48, nx: int = 96, dh: float = 10.0, nt: int = 500, fmax: float = 30.0,
               nshots: int = 3, nrec: int = 24, boundary: float = 190.0, **over) -> tuple[Case, np.ndarray]:
    """A few-second case for parity tests: layered model, `nshots` shots and
    `nrec` receivers spread over the surface, 20-cell boundaries."""
    vp = layered_model(nz, nx, dh, seed)
    w = (nx - 1) * dh
    sx = np.linspace(0.15 * w, 0.85 * w, nshots)
    rx = np.linspace(0.0, w, nrec)
    keys = dict(abc_length=boundary, inv_rbc_length=boundary, mig_rbc_length=boundary, inv_rbc_ratio=60,
                mig_rbc_ratio=60, max_iteration=2)
    offsets = keys.pop("max_offsets", None)
    keys.update(over)
    offsets = keys.pop("max_offsets", offsets)
    if offsets is not None:
        Path(root).mkdir(parents=True, exist_ok=True)
        write_offsets(Path(root) / "offsets.txt", offsets)
        keys["aperture_file"] = f"{root}/offsets.txt"
    case = write_case(root, vp, dh, nt, 1e-3, fmax, sx, np.full(nshots, 20.0), rx, np.full(nrec, 10.0), **keys)
    return case, vp
