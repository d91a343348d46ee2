"""CPU oracle of the FWI2D wave-propagation path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import
this module, and only as the checker.  The product (fwi2d_b200) never imports it.

Wraps oracle/fwi_oracle.c (liboracle64.so: FP64 fields and sums; liboracle32.so:
the reference's own float arithmetic) and restates in numpy the pieces that are
plain array arithmetic:
  wavelet()        set_wavelet's half-derivative filter (modeling.cu:32-90) with
                   numpy's FFT in place of FFTW (r2c, multiply, c2r, / nt)
  image_post()     Migration::export_seismic (migration.cu:90-115)
  gradient_post()  compute_gradient's post-processing (inversion.cu:136-165)
  parabola_step()  Inversion::optimization (inversion.cu:286-308)

Parity status: the modeling path (wavelet, indices, damping, stencil, receiver
sampling) and the migration / gradient back-propagation loops are pinned against
golden vectors produced by the reference's own CUDA code (tests/golden/,
generated by tests/golden/make_golden.py through oracle/_ref).  The random
boundary is this project's seeded restatement (the reference's is unseeded) and
is pinned by bit-exact agreement of two independent implementations.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, capture_output=True)


_libs: dict[int, C.CDLL] = {}


def _lib(bits: int = 64) -> C.CDLL:
    if bits not in _libs:
        path = HERE / f"liboracle{bits}.so"
        if not path.exists():
            build()
        lib = C.CDLL(str(path))
        R = C.POINTER(C.c_double if bits == 64 else C.c_float)
        lib.orc_ricker.argtypes = [C.c_int, C.c_float, C.c_float, _F, _I]
        lib.orc_b1d.argtypes = [C.c_int, C.c_float, _F]
        lib.orc_indices.argtypes = [C.c_int, _F, C.c_float, C.c_int, _I]
        lib.orc_expand.argtypes = [_F, C.c_int, C.c_int, C.c_int, _F]
        lib.orc_forward.argtypes = [_F, C.c_int, C.c_int, C.c_int, _F, _F, C.c_int, C.c_int, C.c_float, C.c_float,
                                    C.c_int, C.c_int, C.c_int, _I, _I, _F, R, R, C.c_int]
        lib.orc_forward.restype = C.c_int
        lib.orc_backward.argtypes = [_F, C.c_int, C.c_int, _F, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, _I, _I,
                                     R, R, C.c_int, R, R]
        lib.orc_backward.restype = C.c_int
        lib.orc_bumps.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_uint64, C.c_uint32,
                                  _F, C.c_int]
        lib.orc_bumps.restype = C.c_int
        lib.orc_pds.argtypes = [C.c_float, C.c_float, C.c_float, C.c_uint64, C.c_uint32, _F, C.c_int]
        lib.orc_pds.restype = C.c_int
        lib.orc_rbc.argtypes = [_F, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_uint64,
                                C.c_uint32, _F, C.c_int, _F]
        lib.orc_ppnd16.argtypes = [C.c_double]
        lib.orc_ppnd16.restype = C.c_double
        lib.orc_exp.argtypes = [C.c_double]
        lib.orc_exp.restype = C.c_double
        lib.orc_log.argtypes = [C.c_double]
        lib.orc_log.restype = C.c_double
        lib.orc_normal.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64]
        lib.orc_normal.restype = C.c_float
        _libs[bits] = lib
    return _libs[bits]


def _f(a):
    return a.ctypes.data_as(_F)


def _i(a):
    return a.ctypes.data_as(_I)


def _real(bits):
    return np.float64 if bits == 64 else np.float32


# ------------------------------------------------------------------- set-up
def ricker(nt: int, dt: float, fmax: float) -> tuple[np.ndarray, int]:
    out = np.empty(nt, np.float32)
    tl = C.c_int()
    _lib().orc_ricker(nt, dt, fmax, _f(out), C.byref(tl))
    return out, tl.value


def wavelet(nt: int, dt: float, fmax: float) -> tuple[np.ndarray, int]:
    """Ricker (float, as the reference) -> FFT (double) x (i 2 pi f)^0.5 -> inverse / nt."""
    r, tlag = ricker(nt, dt, fmax)
    X = np.fft.rfft(r.astype(np.float64))
    df = 1.0 / float(np.float32(nt) * np.float32(dt))
    f = np.arange(X.size) * df
    H = np.sqrt(1j * 2.0 * np.pi * f)
    w = np.fft.irfft(X * H, n=nt)
    return w.astype(np.float32), tlag


def b1d(nb: int, factor: float) -> np.ndarray:
    out = np.empty(nb, np.float32)
    _lib().orc_b1d(nb, factor, _f(out))
    return out


def indices(coord, dh: float, nb: int) -> np.ndarray:
    c = np.ascontiguousarray(coord, dtype=np.float32)
    out = np.empty(c.size, np.int32)
    _lib().orc_indices(c.size, _f(c), dh, nb, _i(out))
    return out


def expand(model: np.ndarray, nb: int) -> np.ndarray:
    """(nz, nx) -> (nzz, nxx) edge-replicated (expand_boundary)."""
    nz, nx = model.shape
    src = np.ascontiguousarray(model.T, dtype=np.float32)  # z fastest
    out = np.empty((nx + 2 * nb) * (nz + 2 * nb), np.float32)
    _lib().orc_expand(_f(src), nz, nx, nb, _f(out))
    return out.reshape(nx + 2 * nb, nz + 2 * nb).T


def crop(padded: np.ndarray, nb: int) -> np.ndarray:
    return padded[nb:padded.shape[0] - nb, nb:padded.shape[1] - nb]


# ------------------------------------------------- aperture windows (extension)
# Batched uneven-aperture surveys have no reference counterpart: the reference
# models every shot on the whole model.  These restate the engine's rule from
# its definition so the windowed paths have a CPU check.
def window(xs: float, max_offset: float, nx: int, dh: float) -> tuple[int, int]:
    """Model columns [c0, c0+w) within max_offset of a source at x = xs."""
    import math
    c0 = math.floor((float(xs) - float(max_offset)) / float(dh))
    c1 = math.ceil((float(xs) + float(max_offset)) / float(dh))
    c0 = min(max(c0, 0), nx - 1)
    c1 = min(max(c1, 0), nx - 1)
    while c1 - c0 + 1 < 9:
        if c0 > 0:
            c0 -= 1
        if c1 - c0 + 1 < 9 and c1 < nx - 1:
            c1 += 1
    return c0, c1 - c0 + 1


def window_velocity_abc(model: np.ndarray, nb: int, c0: int, w: int) -> np.ndarray:
    """ABC grid of a windowed shot: columns c0 .. c0+w+2nb-1 of the padded whole model."""
    return expand(model, nb)[:, c0:c0 + w + 2 * nb]


def window_velocity_rbc_base(model: np.ndarray, nb: int, c0: int, w: int) -> np.ndarray:
    """RBC base of a windowed shot: its window padded by edge replication."""
    return expand(np.ascontiguousarray(model[:, c0:c0 + w]), nb)


def scatter_windows(parts, windows, nz: int, nx: int, nb: int) -> np.ndarray:
    """Sum over shots of crop(part_s) placed at columns [c0_s, c0_s + w_s)."""
    out = np.zeros((nz, nx), np.float64)
    for p, (c0, w) in zip(parts, windows):
        out[:, c0:c0 + w] += crop(p, nb)
    return out


# --------------------------------------------------------------- propagation
def forward(vel: np.ndarray, nb: int, b1d_tab, wav: np.ndarray, nt: int, tlag: int, dt: float, dh: float,
            src: tuple[int, int], rx, rz, bits: int = 64, ordered: bool = False):
    """ABC (b1d_tab given) or plain forward run on the padded (nzz, nxx) velocity.

    Returns (seismogram (nt, nrec) float32, P final, Pold final) with the fields
    as (nzz, nxx) arrays of the oracle's precision."""
    nzz, nxx = vel.shape
    v = np.ascontiguousarray(vel.T, dtype=np.float32)
    rx = np.ascontiguousarray(rx, dtype=np.int32)
    rz = np.ascontiguousarray(rz, dtype=np.int32)
    seis = np.zeros(rx.size * nt, np.float32)
    R = _real(bits)
    P = np.zeros(nzz * nxx, R)
    Po = np.zeros(nzz * nxx, R)
    rp = (lambda a: a.ctypes.data_as(C.POINTER(C.c_double if bits == 64 else C.c_float)))
    tab = None if b1d_tab is None else np.ascontiguousarray(b1d_tab, dtype=np.float32)
    rc = _lib(bits).orc_forward(_f(v), nzz, nxx, nb, None if tab is None else _f(tab), _f(np.ascontiguousarray(wav, np.float32)),
                                nt, tlag, dt, dh, src[0], src[1], rx.size, _i(rx), _i(rz), _f(seis), rp(P), rp(Po),
                                int(ordered))
    assert rc == 0
    return seis.reshape(rx.size, nt).T, P.reshape(nxx, nzz).T, Po.reshape(nxx, nzz).T


def backward(vel: np.ndarray, data: np.ndarray, nt: int, tlag: int, dt: float, dh: float, rx, rz, p_final, pold_final,
             gradient: bool, bits: int = 64):
    """Migration (gradient=False) or adjoint (gradient=True) back-propagation of
    data (nt, nrec) on the padded velocity; returns (accumulator, illumination)
    as (nzz, nxx) arrays."""
    nzz, nxx = vel.shape
    R = _real(bits)
    v = np.ascontiguousarray(vel.T, dtype=np.float32)
    d = np.ascontiguousarray(np.asarray(data, np.float32).T)
    rx = np.ascontiguousarray(rx, dtype=np.int32)
    rz = np.ascontiguousarray(rz, dtype=np.int32)
    ps = np.ascontiguousarray(np.asarray(p_final).T, dtype=R).ravel().copy()
    pso = np.ascontiguousarray(np.asarray(pold_final).T, dtype=R).ravel().copy()
    acc = np.zeros(nzz * nxx, R)
    ill = np.zeros(nzz * nxx, R)
    rp = (lambda a: a.ctypes.data_as(C.POINTER(C.c_double if bits == 64 else C.c_float)))
    rc = _lib(bits).orc_backward(_f(v), nzz, nxx, _f(d), nt, tlag, dt, dh, rx.size, _i(rx), _i(rz), rp(ps), rp(pso),
                                 int(gradient), rp(acc), rp(ill))
    assert rc == 0
    return acc.reshape(nxx, nzz).T, ill.reshape(nxx, nzz).T


# ----------------------------------------------------------- random boundary
def normal(seed: int, shot: int, stream: int, ctr: int) -> float:
    return float(_lib().orc_normal(seed, shot, stream, ctr))


def pds(x_max: float, z_max: float, radius: float, seed: int, shot: int) -> np.ndarray:
    """The seeded Poisson-disk point set (n, 2) of (x, z) before the band filter."""
    cap = 1 << 20
    out = np.empty(2 * cap, np.float32)
    n = _lib().orc_pds(x_max, z_max, radius, seed, shot, _f(out), cap)
    assert n <= cap
    return out[: 2 * n].reshape(-1, 2)


def bumps(nxx, nzz, nb, dh, ratio, varVp, seed, shot) -> np.ndarray:
    cap = 1 << 16
    out = np.empty(5 * cap, np.float32)
    n = _lib().orc_bumps(nxx, nzz, nb, dh, ratio, varVp, seed, shot, _f(out), cap)
    assert n <= cap
    return out[: 5 * n].reshape(-1, 5)


def rbc(base: np.ndarray, nb: int, dh: float, varVp: float, vmin: float, vmax: float, seed: int, shot: int,
        bump_table: np.ndarray) -> np.ndarray:
    nzz, nxx = base.shape
    b = np.ascontiguousarray(base.T, dtype=np.float32)
    bt = np.ascontiguousarray(bump_table, dtype=np.float32).ravel()
    out = np.empty(nzz * nxx, np.float32)
    _lib().orc_rbc(_f(b), nzz, nxx, nb, dh, varVp, vmin, vmax, seed, shot, _f(bt), int(bump_table.shape[0]), _f(out))
    return out.reshape(nxx, nzz).T


# --------------------------------------------------------- data preparation
def mute_direct(data: np.ndarray, sps: np.ndarray, rps: np.ndarray, dt: float, velocity=3600, time_delay=0.18,
                gstd=30) -> np.ndarray:
    """run/generate_input_data.py:22-44 on (nsrc, nt, nrec) seismograms with the
    script's numpy dtypes: float32 data and geometry, Python scalars, the taper
    in float64 (numpy's in-place multiply rounds the product to float32)."""
    out = np.array(data, dtype=np.float32, copy=True)
    sps = np.asarray(sps, np.float32)
    rps = np.asarray(rps, np.float32)
    nt = out.shape[1]
    t = np.arange(nt)
    for s in range(out.shape[0]):
        d = out[s]
        d *= 1.0 / np.max(np.abs(d))
        dist = np.sqrt((rps[:, 0] - sps[s, 0]) ** 2 + (rps[:, 1] - sps[s, 1]) ** 2)
        tid = np.array((dist / velocity + time_delay) / dt, dtype=int)
        for r in range(out.shape[2]):
            k = tid[r]
            d[:k, r] *= np.exp(-0.5 * ((t - k) / gstd) ** 2)[:k]
    return out


def smooth_init(model: np.ndarray, sigma: float, depth_mask: float, dh: float) -> np.ndarray:
    """run/generate_setup.py:49-51: 1 / gaussian_filter(1 / model, sigma), the
    rows above int(depth_mask / dh) kept (scipy.ndimage, the script's own call)."""
    from scipy.ndimage import gaussian_filter
    m = np.asarray(model, np.float32)
    out = 1.0 / gaussian_filter(1.0 / m, sigma)
    z = int(depth_mask / dh)
    out[:z] = m[:z]
    return out.astype(np.float32)


# --------------------------------------------------------- post-processing
def image_post(img: np.ndarray, illum: np.ndarray, idh2: float) -> np.ndarray:
    q = (img.astype(np.float32) / illum.astype(np.float32)).astype(np.float32)
    out = np.zeros_like(q)
    out[1:-1] = -np.float32(1.0) * (q[:-2] - np.float32(2.0) * q[1:-1] + q[2:]) * np.float32(idh2)
    return out


def gradient_post(g: np.ndarray, illum: np.ndarray, idh2: float, zmask_i: int) -> np.ndarray:
    q = (g.astype(np.float32) / illum.astype(np.float32)).astype(np.float32)
    out = np.zeros_like(q)
    nz = q.shape[0]
    rows = np.arange(nz)
    sel = (rows > zmask_i) & (rows < nz - 1)
    lap = np.zeros_like(q)
    lap[1:-1] = -np.float32(1.0) * (q[:-2] - np.float32(2.0) * q[1:-1] + q[2:]) * np.float32(idh2)
    out[sel] = lap[sel]
    gmax = np.abs(out).max()
    return out * (np.float32(1.0) / np.float32(gmax))


def parabola_step(f0, f1, f2, vmin, vmax):
    f32 = np.float32
    dm = f32(1.0) / (f32(vmin) * f32(vmin)) - f32(1.0) / (f32(vmax) * f32(vmax))
    a0, a1, a2 = f32(0.0) * dm, f32(0.02) * dm, f32(0.05) * dm
    f0, f1, f2 = f32(f0), f32(f1), f32(f2)
    num = (a1 * a1 - a2 * a2) * f0 + (a2 * a2 - a0 * a0) * f1 + (a0 * a0 - a1 * a1) * f2
    den = (a1 - a2) * f0 + (a2 - a0) * f1 + (a0 - a1) * f2
    return float(f32(0.5) * (num / den)), (float(a1), float(a2))
