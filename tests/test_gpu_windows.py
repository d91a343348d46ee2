"""Batched uneven-aperture surveys on the GPU vs the CPU oracle (-m gpu).

Every shot runs on its own aperture window (model columns [c0, c0+w)) and all
shots of different widths share one batch.  The oracle runs each shot on its
own window grid (oracle.window_velocity_abc / window_velocity_rbc_base) and
scatters windowed images and gradients back (oracle.scatter_windows).  Same
bar as the whole-model path: relative L2 below 1e-4 against the FP64 oracle,
the random boundary bit-exact."""
import numpy as np
import pytest

from fwi2d_b200 import api, synth
from oracle import oracle as O
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu
RTOL = 1e-4
NB = 20
OFFSETS = [250.0, 420.0, 610.0, 1e5]  # the last shot spans the whole model


def _case(root, **kw):
    return synth.small_case(root, nx=160, nshots=4, nrec=40, max_offsets=OFFSETS, **kw)


def _geometry(c, nb):
    wav, tlag = O.wavelet(c.nt, c.dt, c.fmax)
    sx = O.indices(c.sx, c.dh, nb)
    sz = O.indices(c.sz, c.dh, nb)
    rx = O.indices(c.rx, c.dh, nb)
    rz = O.indices(c.rz, c.dh, nb)
    return wav, tlag, sx, sz, rx, rz


def _windows(c):
    return [O.window(float(np.float32(c.sx[s])), float(np.float32(OFFSETS[s])), c.nx, float(np.float32(c.dh)))
            for s in range(len(c.sx))]


def _inside(rx, nb, c0, w):
    m = rx - nb
    return (m >= c0) & (m < c0 + w)


def _oracle_windowed_modeling(c, vp, wins):
    wav, tlag, sx, sz, rx, rz = _geometry(c, NB)
    tab = O.b1d(NB, 0.004)
    out = []
    for s, (c0, w) in enumerate(wins):
        sel = _inside(rx, NB, c0, w)
        vel = O.window_velocity_abc(vp, NB, c0, w)
        seis = np.zeros((c.nt, len(rx)), np.float64)
        seis[:, sel] = O.forward(vel, NB, tab, wav, c.nt, tlag, c.dt, c.dh, (sx[s] - c0, sz[s]), rx[sel] - c0,
                                 rz[sel], bits=64)[0]
        out.append(seis)
    return out


def test_windows_reported(tmp_path):
    c, _ = _case(tmp_path)
    with api.Context(c.params, api.MODE_MODELING) as ctx:
        got = [ctx.window(s) for s in range(len(c.sx))]
        assert ctx.dims.nxx == max(w for _, w in got) + 2 * NB
    assert got == _windows(c)
    assert got[-1] == (0, c.nx) and all(w < c.nx for _, w in got[:-1])


@pytest.mark.parametrize("variant", ["auto", "simple", "tma:1,32,2", "tma:2,16,2", "loop:32,2", "loop:16,3", "resident"])
def test_windowed_modeling_vs_oracle(tmp_path, variant):
    c, vp = _case(tmp_path, fwd_kernel=variant)
    with api.Context(c.params, api.MODE_MODELING) as ctx:
        seis = ctx.model_survey()
    wins = _windows(c)
    ref = _oracle_windowed_modeling(c, vp, wins)
    rx = O.indices(c.rx, c.dh, NB)
    for s, (c0, w) in enumerate(wins):
        sel = _inside(rx, NB, c0, w)
        assert sel.any()
        assert rel_l2(seis[s][:, sel], ref[s][:, sel]) < RTOL, (variant, s)
        assert np.all(seis[s][:, ~sel] == 0.0)


def test_whole_model_windows_equal_plain_path(tmp_path):
    a, _ = synth.small_case(tmp_path / "plain", nx=160, nshots=4, nrec=40)
    b, _ = synth.small_case(tmp_path / "win", nx=160, nshots=4, nrec=40, max_offsets=[1e6] * 4)
    with api.Context(a.params, api.MODE_MODELING) as ctx:
        plain = ctx.model_survey()
    with api.Context(b.params, api.MODE_MODELING) as ctx:
        assert all(ctx.window(s) == (0, b.nx) for s in range(4))
        win = ctx.model_survey()
    assert np.array_equal(plain, win)


def test_windowed_random_boundary_bit_exact(tmp_path):
    c, vp = _case(tmp_path)
    with api.Context(c.params, api.MODE_MIGRATION) as ctx:
        nb = ctx.dims.rbc_nb
        for s, (c0, w) in enumerate(_windows(c)):
            gpu = ctx.random_boundary(s)
            base = O.window_velocity_rbc_base(vp, nb, c0, w)
            bt = O.bumps(w + 2 * nb, base.shape[0], nb, c.dh, 60.0, 500.0, 0, s)
            ref = O.rbc(base, nb, c.dh, 500.0, float(vp.min()), float(vp.max()), 0, s, bt)
            assert gpu.shape == ref.shape
            assert np.array_equal(gpu, ref), (s, np.abs(gpu - ref).max())


def _oracle_backward_windows(c, vels, series, wins, nb, gradient):
    wav, tlag, sx, sz, rx, rz = _geometry(c, nb)
    accs, ills = [], []
    for s, (c0, w) in enumerate(wins):
        sel = _inside(rx, nb, c0, w)
        _, P, Po = O.forward(vels[s], nb, None, wav, c.nt, tlag, c.dt, c.dh, (sx[s] - c0, sz[s]), rx[sel] - c0,
                             rz[sel], bits=64)
        a, b = O.backward(vels[s], np.ascontiguousarray(series[s][:, sel], np.float32), c.nt, tlag, c.dt, c.dh,
                          rx[sel] - c0, rz[sel], P, Po, gradient=gradient, bits=64)
        accs.append(a)
        ills.append(b)
    return (O.scatter_windows(accs, wins, c.nz, c.nx, nb), O.scatter_windows(ills, wins, c.nz, c.nx, nb))


def test_windowed_rtm_vs_oracle(tmp_path):
    c, vp = _case(tmp_path)
    wins = _windows(c)
    smooth = synth.smooth_model(vp, c.dh, 40.0)
    full, _ = synth.small_case(tmp_path / "full", nx=160, nshots=4, nrec=40)
    tab = O.b1d(NB, 0.004)
    wav, tlag, sx, sz, rx, rz = _geometry(full, NB)
    data = np.stack([O.forward(O.expand(vp, NB), NB, tab, wav, c.nt, tlag, c.dt, c.dh, (sx[s], sz[s]), rx, rz,
                               bits=64)[0] for s in range(4)]).astype(np.float32)
    with api.Context(c.params, api.MODE_MIGRATION) as ctx:
        ctx.set_model(smooth)
        nb = ctx.dims.rbc_nb
        vels = [ctx.random_boundary(s) for s in range(4)]
        ctx.rtm_reset()
        ctx.rtm_survey(data)
        img, ill = ctx.rtm_raw()
    ref_img, ref_ill = _oracle_backward_windows(c, vels, data, wins, nb, gradient=False)
    assert rel_l2(img, ref_img) < RTOL
    assert rel_l2(ill, ref_ill) < RTOL


def test_windowed_misfit_and_gradient_vs_oracle(tmp_path):
    c, vp = _case(tmp_path)
    wins = _windows(c)
    init = synth.smooth_model(vp, c.dh, 40.0)
    wav, tlag, sx, sz, rx, rz = _geometry(c, NB)
    tab = O.b1d(NB, 0.004)
    # observed data on the whole model for every receiver: the engine drops the
    # traces outside each shot's window from the misfit
    obs = np.stack([O.forward(O.expand(vp, NB), NB, tab, wav, c.nt, tlag, c.dt, c.dh, (sx[s], sz[s]), rx, rz,
                              bits=64)[0] for s in range(4)]).astype(np.float32)
    with api.Context(c.params, api.MODE_INVERSION) as ctx:
        ctx.set_model(init)
        ctx.set_observed(obs)
        nb = ctx.dims.rbc_nb
        vels = [ctx.random_boundary(s) for s in range(4)]
        sum_res = ctx.compute_gradient(True)
        graw, gill = ctx.gradient_raw()
    cal = _oracle_windowed_modeling(c, init, wins)
    res = []
    for s, (c0, w) in enumerate(wins):
        sel = _inside(rx, NB, c0, w)
        r = np.zeros_like(cal[s])
        r[:, sel] = obs[s][:, sel].astype(np.float64) - cal[s][:, sel]
        res.append(r)
    ref_sum = sum(float((r * r).sum()) for r in res)
    assert abs(sum_res - ref_sum) / ref_sum < RTOL
    ref_g, ref_ill = _oracle_backward_windows(c, vels, [r.astype(np.float32) for r in res], wins, nb, gradient=True)
    assert rel_l2(graw, ref_g) < RTOL
    assert rel_l2(gill, ref_ill) < RTOL
