"""Failure detection of the bounded device waits (run on a B200: -m gpu).

Every device wait of the propagation kernels gives up after a bounded number
of polls, raises the context's error flag and returns; the host turns the flag
into FWI_ERR_TIMEOUT.  These tests make the waits run out on purpose, with no
fault: two test-only parameters.txt keys shorten the limit (test_wait_limit)
and make one CTA withhold its work (test_stall_fwd / test_stall_bwd):

* the resident forward kernel: one slab publishes no halo words, so its
  neighbours' halo polls give up (and every other slab leaves at its next
  missing word once the flag is up);
* the multi-level forward and backward kernels: one CTA issues no loads for
  its first tile, so its consumers' mbarrier waits give up, it never reaches
  the grid barrier and every other CTA's barrier poll gives up.

Each drill must end with FWI_ERR_TIMEOUT well within a second per wait, and a
fresh context in the same process must then reproduce, bit for bit, the
result computed before the drill: the failed launch left no tensor memory
allocated, no copy in flight and nothing waiting.
"""
import time

import numpy as np
import pytest

from fwi2d_b200 import api, synth

pytestmark = pytest.mark.gpu
FWI_ERR_TIMEOUT = -6
LIMIT = 4096  # polls per wait in the drills (the default is 2^22)


def _expect_timeout(fn):
    t0 = time.perf_counter()
    with pytest.raises(api.FwiError) as e:
        fn()
    elapsed = time.perf_counter() - t0
    assert e.value.code == FWI_ERR_TIMEOUT, str(e.value)
    assert "bounded wait" in str(e.value)
    assert elapsed < 60.0, elapsed
    return elapsed


def test_resident_halo_wait_runs_out_and_context_recovers(tmp_path):
    """The benchmark geometry (13 slabs per shot) for 179 levels."""
    clean, _ = synth.modeling_survey(tmp_path / "clean", seed=0, nt=60, fwd_kernel="resident")
    with api.Context(clean.params, api.MODE_MODELING) as ctx:
        ref = ctx.model_survey()
        assert ctx.describe().startswith("resident"), ctx.describe()
    drill, _ = synth.modeling_survey(tmp_path / "drill", seed=0, nt=60, fwd_kernel="resident",
                                     test_wait_limit=LIMIT, test_stall_fwd=5)
    with api.Context(drill.params, api.MODE_MODELING) as ctx:
        _expect_timeout(ctx.model_survey)
    with api.Context(clean.params, api.MODE_MODELING) as ctx:
        again = ctx.model_survey()
    assert np.array_equal(again, ref)


def test_forward_grid_barrier_runs_out_and_context_recovers(tmp_path):
    clean, _ = synth.small_case(tmp_path / "clean", nt=200, fwd_kernel="loop:16,3")
    with api.Context(clean.params, api.MODE_MODELING) as ctx:
        ref = ctx.model_survey()
    drill, _ = synth.small_case(tmp_path / "drill", nt=200, fwd_kernel="loop:16,3", test_wait_limit=LIMIT,
                                test_stall_fwd=0)
    with api.Context(drill.params, api.MODE_MODELING) as ctx:
        _expect_timeout(ctx.model_survey)
    with api.Context(clean.params, api.MODE_MODELING) as ctx:
        again = ctx.model_survey()
    assert np.array_equal(again, ref)


def test_backward_grid_barrier_runs_out_and_context_recovers(tmp_path):
    clean, vp = synth.small_case(tmp_path / "clean", nt=200, fwd_kernel="loop:16,3", bwd_kernel="loop:8,3")
    with api.Context(clean.params, api.MODE_MODELING) as ctx:
        data = ctx.model_survey()
    smooth = synth.smooth_model(vp, clean.dh, 40.0)

    def rtm(params):
        with api.Context(params, api.MODE_MIGRATION) as ctx:
            ctx.set_model(smooth)
            ctx.rtm_reset()
            ctx.rtm_survey(data)
            return ctx.rtm_raw()

    ref_img, ref_ill = rtm(clean.params)
    drill, _ = synth.small_case(tmp_path / "drill", nt=200, fwd_kernel="loop:16,3", bwd_kernel="loop:8,3",
                                test_wait_limit=LIMIT, test_stall_bwd=0)
    _expect_timeout(lambda: rtm(drill.params))
    img, ill = rtm(clean.params)
    assert np.array_equal(img, ref_img) and np.array_equal(ill, ref_ill)


def test_wait_limit_key_is_checked(tmp_path):
    c, _ = synth.small_case(tmp_path, nt=50, test_wait_limit=8)
    with pytest.raises(api.FwiError) as e:
        api.Context(c.params, api.MODE_MODELING)
    assert e.value.code == -1
