"""Properties of the CPU oracle itself (CPU only, small grids)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import rel_l2

NT, DT, DH, FMAX = 400, 1e-3, 10.0, 30.0


def _setup(nz=40, nx=80, nb=20, v=2000.0):
    vp = np.full((nz, nx), v, np.float32)
    wav, tlag = O.wavelet(NT, DT, FMAX)
    return vp, O.expand(vp, nb), wav, tlag


def test_float_arithmetic_vs_fp64():
    """The reference's float arithmetic (liboracle32) against FP64: the size of FP32 rounding."""
    rng = np.random.default_rng(0)
    nb = 20
    vp = rng.uniform(1500, 3000, (40, 80)).astype(np.float32)
    vel = O.expand(vp, nb)
    wav, tlag = O.wavelet(NT, DT, FMAX)
    rx = np.arange(nb, nb + 80, 4, dtype=np.int32)
    rz = np.full_like(rx, nb + 1)
    s64, _, _ = O.forward(vel, nb, O.b1d(nb, 0.004), wav, NT, tlag, DT, DH, (nb + 40, nb + 2), rx, rz, bits=64)
    s32, _, _ = O.forward(vel, nb, O.b1d(nb, 0.004), wav, NT, tlag, DT, DH, (nb + 40, nb + 2), rx, rz, bits=32)
    err = rel_l2(s32, s64)
    assert 0 < err < 1e-5, err


def test_reciprocity_homogeneous():
    nb = 20
    vp, vel, wav, tlag = _setup(nb=nb)
    a, b = (nb + 10, nb + 5), (nb + 60, nb + 25)
    s_ab, _, _ = O.forward(vel, nb, None, wav, NT, tlag, DT, DH, a, [b[0]], [b[1]], bits=64)
    s_ba, _, _ = O.forward(vel, nb, None, wav, NT, tlag, DT, DH, b, [a[0]], [a[1]], bits=64)
    assert rel_l2(s_ab, s_ba) < 1e-10


def test_direct_arrival_moveout():
    """Two receivers on a line through the source: arrival lag = extra distance / v."""
    nb, v = 20, 2000.0
    vp, vel, wav, tlag = _setup(nz=40, nx=140, nb=nb, v=v)
    src = (nb + 20, nb + 20)
    rx = np.array([nb + 40, nb + 70], np.int32)
    rz = np.array([nb + 20, nb + 20], np.int32)
    s, _, _ = O.forward(vel, nb, O.b1d(nb, 0.004), wav, NT, tlag, DT, DH, src, rx, rz, bits=64)
    lag = np.argmax(np.correlate(s[:, 1], s[:, 0], "full")) - (NT - 1)
    expect = (30 * DH / v) / DT
    assert abs(lag - expect) <= 1.5, (lag, expect)


def test_damping_race_bound():
    """The reference damps P in place while neighbours read it (modeling.cu:337-343).
    Without damping the update order is irrelevant; with it, a fully serialised
    order (earlier neighbours already damped) differs from the Jacobi order by
    ~12% rel L2 on this case, all from the boundary band's reflection.  The GPU
    reference runs every block of a step concurrently, which is close to the
    Jacobi order; tests/test_golden.py measures how close."""
    rng = np.random.default_rng(1)
    nb = 20
    vp = rng.uniform(1500, 3000, (40, 80)).astype(np.float32)
    vel = O.expand(vp, nb)
    wav, tlag = O.wavelet(NT, DT, FMAX)
    rx = np.arange(nb, nb + 80, 4, dtype=np.int32)
    rz = np.full_like(rx, nb + 1)
    tab = O.b1d(nb, 0.004)
    j, _, _ = O.forward(vel, nb, tab, wav, NT, tlag, DT, DH, (nb + 40, nb + 2), rx, rz, bits=64)
    o, _, _ = O.forward(vel, nb, tab, wav, NT, tlag, DT, DH, (nb + 40, nb + 2), rx, rz, bits=64, ordered=True)
    assert 0.01 < rel_l2(o, j) < 0.5
    jn, _, _ = O.forward(vel, nb, None, wav, NT, tlag, DT, DH, (nb + 40, nb + 2), rx, rz, bits=64)
    on, _, _ = O.forward(vel, nb, None, wav, NT, tlag, DT, DH, (nb + 40, nb + 2), rx, rz, bits=64, ordered=True)
    assert np.array_equal(jn, on)


def test_backward_zero_data_is_pure_reconstruction():
    """With zero input traces the receiver field stays 0: no image, only illumination."""
    nb = 20
    vp, vel, wav, tlag = _setup(nb=nb)
    rx = np.arange(nb, nb + 80, 8, dtype=np.int32)
    rz = np.full_like(rx, nb + 1)
    _, P, Po = O.forward(vel, nb, None, wav, NT, tlag, DT, DH, (nb + 40, nb + 2), rx, rz, bits=64)
    img, ill = O.backward(vel, np.zeros((NT, rx.size), np.float32), NT, tlag, DT, DH, rx, rz, P, Po, False)
    assert np.all(img == 0) and ill.sum() > 0


def test_parabola_vertex():
    # f(a) = (a - c)^2 + 1 sampled at 0, a1, a2 -> vertex c
    vmin, vmax = 1500.0, 3500.0
    dm = 1 / vmin**2 - 1 / vmax**2
    c = 0.03 * dm
    f = lambda a: (a - c) ** 2 / dm**2 + 1.0
    step, (a1, a2) = O.parabola_step(f(0.0), f(0.02 * dm), f(0.05 * dm), vmin, vmax)
    assert abs(step - c) / c < 1e-3


def test_image_post_matches_definition():
    rng = np.random.default_rng(3)
    img = rng.normal(size=(20, 30)).astype(np.float32)
    ill = rng.uniform(1, 2, size=(20, 30)).astype(np.float32)
    out = O.image_post(img, ill, 0.01)
    q = img / ill
    assert np.allclose(out[5, 7], -(q[4, 7] - 2 * q[5, 7] + q[6, 7]) * 0.01, rtol=1e-6)
    assert np.all(out[0] == 0) and np.all(out[-1] == 0)
