"""fwi_residual_noalloc: residual and FP64 misfit without any device allocation.

The entry point exists for callers that cannot call cudaMalloc - an
application whose own memory pool owns the whole device, code running inside a
CUDA stream capture, loops that cannot take cudaMalloc's implicit device
synchronisation.  Its scratch (per-chunk partial sums) lives in a file-scope
device array shared by all calls.  This test calls it through the C ABI on
device buffers and compares it with the existing entry point,
fwi_compute_gradient, whose misfit reduction uses context-allocated scratch:
two calls in a row on different data, each within the tolerance of the other
GPU tests (relative 1e-4), and the residual bit for bit.  The chunk edges of
the scratch (8192 samples a partial sum) are checked against numpy's FP64 sum
of squares: no sample, exactly one chunk, and a partial last chunk.  The file
sorts last so a run stopped at the first failure has run every other test
already.
"""
import ctypes as C

import numpy as np
import pytest

from fwi2d_b200 import api, synth

pytestmark = pytest.mark.gpu
RTOL = 1e-4


def _noalloc(d_obs, d_cal, d_res, n, d_sum):
    return api.lib().fwi_residual_noalloc(C.c_void_p(d_obs.data_ptr()), C.c_void_p(d_cal.data_ptr()),
                                          C.c_void_p(d_res.data_ptr()), n, C.c_void_p(d_sum.data_ptr()), None)


def test_noalloc_residual_matches_existing_entry_point(tmp_path):
    import torch

    case, vp = synth.small_case(tmp_path, nshots=3)
    init = synth.smooth_model(vp, case.dh, 40.0)
    with api.Context(case.params, api.MODE_MODELING) as mod:
        obs = mod.model_survey_raw().copy()
        mod.set_model(init)
        cal = mod.model_survey_raw().copy()
    n = obs.size
    dev = torch.device("cuda", 0)
    d_cal = torch.from_numpy(cal).to(dev)
    d_res = torch.empty(n, dtype=torch.float32, device=dev)
    d_sum = torch.zeros(1, dtype=torch.float64, device=dev)
    with api.Context(case.params, api.MODE_INVERSION) as inv:
        inv.set_model(init)
        for scale in (1.0, 0.5):  # two calls in a row on different observed data
            o = (obs * np.float32(scale)).astype(np.float32)
            inv.set_observed_raw(o)
            expected = inv.compute_gradient(False)
            d_obs = torch.from_numpy(o).to(dev)
            d_res.fill_(np.nan)
            d_sum.fill_(np.nan)
            torch.cuda.synchronize()
            assert _noalloc(d_obs, d_cal, d_res, n, d_sum) == 0, api.lib().fwi_last_error(None)
            torch.cuda.synchronize()
            got = float(d_sum.item())
            assert abs(got - expected) <= RTOL * abs(expected), (got, expected)
            assert torch.equal(d_res, d_obs - d_cal)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    dev = torch.device("cuda", 0)
    t = torch.zeros(4, dtype=torch.float32, device=dev)
    s = torch.zeros(1, dtype=torch.float64, device=dev)
    rc = api.lib().fwi_residual_noalloc(C.c_void_p(t.data_ptr()), C.c_void_p(t.data_ptr()),
                                        C.c_void_p(t.data_ptr()), 8192 * 8192 + 1, C.c_void_p(s.data_ptr()), None)
    assert rc == -8
    assert b"exceeds the maximum" in api.lib().fwi_last_error(None)


@pytest.mark.parametrize("n", [0, 8192, 3 * 8192 + 5])
def test_noalloc_chunk_edges_vs_numpy(n):
    import torch

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(n)
    obs = rng.standard_normal(max(n, 1)).astype(np.float32)
    cal = rng.standard_normal(max(n, 1)).astype(np.float32)
    d_obs, d_cal = torch.from_numpy(obs).to(dev), torch.from_numpy(cal).to(dev)
    d_res = torch.full((max(n, 1),), np.nan, dtype=torch.float32, device=dev)
    d_sum = torch.full((1,), np.nan, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    assert _noalloc(d_obs, d_cal, d_res, n, d_sum) == 0, api.lib().fwi_last_error(None)
    assert api.lib().fwi_last_error(None) == b""
    torch.cuda.synchronize()
    res = (obs[:n] - cal[:n]).astype(np.float32)
    ref = float(np.sum(res.astype(np.float64) ** 2))
    got = float(d_sum.item())
    if n == 0:
        assert got == 0.0
    else:
        assert abs(got - ref) <= 1e-12 * ref, (n, got, ref)
        assert np.array_equal(d_res[:n].cpu().numpy(), res)
