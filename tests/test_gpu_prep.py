"""GPU data preparation vs the oracle restatement of the reference's scripts
(run/generate_input_data.py:22-44, run/generate_setup.py:49-51).

Float32 operations are rounded as numpy rounds them; the float64 parts (the
taper, the filter sums) may differ from numpy's libm / summation in the last
double bit, so the bar is at most 1 float32 ulp per sample, and nearly all
samples exact."""
import numpy as np
import pytest

from fwi2d_b200 import api, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _ulps(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    return synth.small_case(tmp_path_factory.mktemp("prep"), nshots=3, nrec=24, nt=400)


def test_mute_direct_matches_script(case):
    c, vp = case
    rng = np.random.default_rng(7)
    data = rng.standard_normal((len(c.sx), c.nt, len(c.rx))).astype(np.float32)
    sps = np.stack([c.sx, c.sz], 1).astype(np.float32)
    rps = np.stack([c.rx, c.rz], 1).astype(np.float32)
    with api.Context(c.params, api.MODE_MIGRATION) as ctx:
        got = ctx.mute_direct(data)
    # the script's dt is a Python float read from parameters.txt
    ref = O.mute_direct(data, sps, rps, float(c.keys["time_spacing"]))
    u = _ulps(got, ref)
    assert u.max() <= 1
    assert (u == 0).mean() > 0.999
    # the taper really ran: early samples near the source are attenuated
    assert np.abs(got[:, :50]).mean() < 0.5 * np.abs(got[:, -50:]).mean()


@pytest.mark.parametrize("sigma,zmask", [(3.0, 0.0), (3.0, 100.0), (7.5, 30.0)])
def test_smooth_model_matches_scipy(case, sigma, zmask):
    c, vp = case
    with api.Context(c.params, api.MODE_MODELING) as ctx:
        got = ctx.smooth_model(vp, sigma, zmask)
    ref = O.smooth_init(vp, sigma, zmask, c.dh)
    u = _ulps(got, ref)
    assert u.max() <= 2, u.max()
    z = int(zmask / c.dh)
    assert np.array_equal(got[:z], vp[:z].astype(np.float32))
