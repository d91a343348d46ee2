"""The benchmark survey at full length against the CPU oracle (run on a B200: -m gpu).

The modeling benchmark times the 11-shot survey on the 151 x 501 layered model
(351 x 701 padded by a 100-cell ABC, 251 receivers, 30 Hz, dt 1 ms, nt 3001 +
119 delay levels = 3120 levels per shot).  On that geometry the resident kernel
splits each shot into 13 slabs that exchange halo columns every level through
parity-slot exchange buffers, so only a run of the full 3120 levels exercises
the exchange as the benchmark does.  These tests run the survey exactly as the
benchmark does and compare every shot with the oracle:

* seismograms of the resident kernel, the autotuned plan and a streaming kernel
  against liboracle64 (FP64 fields) and liboracle32 (the reference's float
  arithmetic, modeling.cu:301-353), relative L2 below 1e-4;
* RTM on the same geometry (migration.cu:49-115): random-boundary forward with
  one velocity per shot, receiver back-propagation and the imaging condition,
  raw image and illumination against the FP64 oracle at 1e-4, the
  post-processed section against the FP64 post-processing of the oracle's raw
  image at 1e-4, and against the FP32 post-processing of the engine's own raw
  image at 1e-6 (which isolates the post-processing kernel).

The measured errors are printed (pytest -s) so they can be quoted.
"""
import numpy as np
import pytest

from fwi2d_b200 import api, synth
from oracle import oracle as O
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu
RTOL = 1e-4
NB = 100


@pytest.fixture(scope="module")
def survey(tmp_path_factory):
    """The benchmark survey on disk and the oracle's seismograms of every shot."""
    root = tmp_path_factory.mktemp("modeling_survey")
    c, vp = synth.modeling_survey(root, seed=0)
    wav, tlag = O.wavelet(c.nt, c.dt, c.fmax)
    rx, rz = O.indices(c.rx, c.dh, NB), O.indices(c.rz, c.dh, NB)
    sx, sz = O.indices(c.sx, c.dh, NB), O.indices(c.sz, c.dh, NB)
    vel, tab = O.expand(vp, NB), O.b1d(NB, 0.004)
    refs = {}
    for bits in (64, 32):
        refs[bits] = np.stack([O.forward(vel, NB, tab, wav, c.nt, tlag, c.dt, c.dh, (sx[s], sz[s]), rx, rz,
                                         bits=bits)[0] for s in range(len(c.sx))])
    return dict(c=c, vp=vp, root=root, refs=refs, wav=wav, tlag=tlag, rx=rx, rz=rz, sx=sx, sz=sz)


@pytest.mark.parametrize("variant", ["auto", "resident", "loop:16,3"])
def test_benchmark_survey_full_length_vs_oracle(survey, tmp_path, variant):
    c0 = survey["c"]
    c, _ = synth.modeling_survey(tmp_path, seed=0, fwd_kernel=variant)
    assert c.nt == 3001 and len(c.sx) == 11 and len(c.rx) == 251
    with api.Context(c.params, api.MODE_MODELING) as ctx:
        d = ctx.dims
        assert (d.nzz, d.nxx, d.nb) == (351, 701, NB)
        seis = ctx.model_survey()
        plan = ctx.describe()
    if variant == "auto":
        assert plan.startswith("resident"), plan  # the benchmark's plan
    worst = {64: 0.0, 32: 0.0}
    for s in range(len(c0.sx)):
        for bits in (64, 32):
            e = rel_l2(seis[s], survey["refs"][bits][s])
            worst[bits] = max(worst[bits], e)
            assert e < RTOL, (variant, bits, s, e)
        assert np.all(seis[s][0] == 0.0)
    print(f"\n[full-length modeling] {variant}: worst shot rel L2 vs FP64 oracle {worst[64]:.3e}, "
          f"vs float oracle {worst[32]:.3e} ({plan.split('|')[0].strip()})")


@pytest.fixture(scope="module")
def rtm(survey, tmp_path_factory):
    """RTM of the benchmark geometry with the resident forward kernel: the
    engine's outputs plus the FP64 oracle's raw image and illumination computed
    on the engine's own random-boundary velocities."""
    root = tmp_path_factory.mktemp("rtm_survey")
    c, vp = synth.modeling_survey(root, seed=0, fwd_kernel="resident")
    sps = np.stack([c.sx, c.sz], 1)
    rps = np.stack([c.rx, c.rz], 1)
    data = O.mute_direct(survey["refs"][64].astype(np.float32), sps, rps, c.dt)  # generate_input_data.py:22-44
    smooth = synth.smooth_model(vp, c.dh, 150.0)
    with api.Context(c.params, api.MODE_MIGRATION) as ctx:
        ctx.set_model(smooth)
        assert ctx.dims.rbc_nb == NB
        vels = [ctx.random_boundary(s) for s in range(len(c.sx))]
        ctx.rtm_reset()
        ctx.rtm_survey(data)
        img, ill = ctx.rtm_raw()
        image = ctx.rtm_image()
        plan = ctx.describe()
    acc = np.zeros(vels[0].shape, np.float64)
    illum = np.zeros_like(acc)
    for s in range(len(c.sx)):
        _, P, Po = O.forward(vels[s], NB, None, survey["wav"], c.nt, survey["tlag"], c.dt, c.dh,
                             (survey["sx"][s], survey["sz"][s]), survey["rx"], survey["rz"], bits=64)
        a, b = O.backward(vels[s], data[s], c.nt, survey["tlag"], c.dt, c.dh, survey["rx"], survey["rz"], P, Po,
                          gradient=False, bits=64)
        acc += a
        illum += b
    return dict(c=c, img=img, ill=ill, image=image, plan=plan, ref_img=O.crop(acc, NB), ref_ill=O.crop(illum, NB))


def _image_post64(img, ill, idh2):
    """Migration::export_seismic (migration.cu:90-115) in FP64."""
    q = np.asarray(img, np.float64) / np.asarray(ill, np.float64)
    out = np.zeros_like(q)
    out[1:-1] = -(q[:-2] - 2.0 * q[1:-1] + q[2:]) * idh2
    return out


def test_benchmark_geometry_rtm_raw_vs_oracle(rtm):
    assert rtm["plan"].startswith("resident"), rtm["plan"]
    e_img = rel_l2(rtm["img"], rtm["ref_img"])
    e_ill = rel_l2(rtm["ill"], rtm["ref_ill"])
    print(f"\n[full-length RTM] raw image rel L2 {e_img:.3e}, illumination {e_ill:.3e} vs FP64 oracle")
    assert e_img < RTOL and e_ill < RTOL


def test_benchmark_geometry_rtm_section_vs_oracle(rtm):
    c = rtm["c"]
    idh2 = 1.0 / c.dh**2
    own = O.image_post(rtm["img"], rtm["ill"], idh2)
    e_own = rel_l2(rtm["image"], own)
    e_ref = rel_l2(rtm["image"], _image_post64(rtm["ref_img"], rtm["ref_ill"], idh2))
    print(f"\n[full-length RTM] section rel L2 vs FP64 oracle {e_ref:.3e}; vs FP32 post-processing of the "
          f"engine's raw image {e_own:.3e}")
    assert e_own < 1e-6
    assert e_ref < RTOL


def test_benchmark_geometry_gradient_vs_oracle(survey, tmp_path):
    """FWI gradient of the benchmark geometry (inversion.cu:111-166, 213-248,
    381-444): misfit of the smoothed model against the survey's data, raw
    gradient and illumination through the random boundary of every shot,
    against the FP64 oracle run on the engine's own boundary velocities."""
    c, vp = synth.modeling_survey(tmp_path, seed=0)
    smooth = synth.smooth_model(vp, c.dh, 150.0)
    obs = survey["refs"][64].astype(np.float32)
    with api.Context(c.params, api.MODE_INVERSION) as ctx:
        ctx.set_model(smooth)
        ctx.set_observed(obs)
        vels = [ctx.random_boundary(s) for s in range(len(c.sx))]
        sum_res = ctx.compute_gradient(True)
        graw, gill = ctx.gradient_raw()
        plan = ctx.describe()
    wav, tlag = survey["wav"], survey["tlag"]
    vel_abc, tab = O.expand(smooth, NB), O.b1d(NB, 0.004)
    ref_sum = 0.0
    acc = np.zeros(vels[0].shape, np.float64)
    ill = np.zeros_like(acc)
    for s in range(len(c.sx)):
        src = (survey["sx"][s], survey["sz"][s])
        cal = O.forward(vel_abc, NB, tab, wav, c.nt, tlag, c.dt, c.dh, src, survey["rx"], survey["rz"], bits=64)[0]
        res = obs[s].astype(np.float64) - cal
        ref_sum += float((res * res).sum())
        _, P, Po = O.forward(vels[s], NB, None, wav, c.nt, tlag, c.dt, c.dh, src, survey["rx"], survey["rz"], bits=64)
        a, b = O.backward(vels[s], res.astype(np.float32), c.nt, tlag, c.dt, c.dh, survey["rx"], survey["rz"], P, Po,
                          gradient=True, bits=64)
        acc += a
        ill += b
    e_sum = abs(sum_res - ref_sum) / ref_sum
    e_g = rel_l2(graw, O.crop(acc, NB))
    e_i = rel_l2(gill, O.crop(ill, NB))
    print(f"\n[full-length gradient] misfit {e_sum:.3e}, raw gradient {e_g:.3e}, illumination {e_i:.3e} "
          f"vs FP64 oracle ({plan.split('|')[0].strip()})")
    assert e_sum < RTOL and e_g < RTOL and e_i < RTOL
