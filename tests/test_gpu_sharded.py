"""Sharded inversion on the GPU: one NCCL rank over the context's own device
accumulators (wrapped through __cuda_array_interface__) must reproduce the
one-call fwi_compute_gradient / fwi_optimization path bit for bit, and a
context whose shot range is split in two must sum to the whole survey."""
import numpy as np
import pytest

from fwi2d_b200 import api, synth
from fwi2d_b200.sharded import ShardedInversion, cuda_wrap
from tests.conftest import rel_l2
from tests.test_gpu_parity import _rtm_data

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def inv_case(tmp_path_factory):
    c, vp = synth.small_case(tmp_path_factory.mktemp("sh"), nshots=4)
    return c, vp, synth.smooth_model(vp, c.dh, 40.0), _rtm_data(c, vp)


def test_split_ranges_sum_to_survey(inv_case):
    c, vp, init, obs = inv_case
    with api.Context(c.params, api.MODE_INVERSION) as ctx:
        ctx.set_model(init)
        ctx.set_observed(obs)
        ctx.set_seed(0)
        whole = ctx.gradient_accumulate(True)
        g_all, i_all = ctx.gradient_raw()
        parts, gs, ils = [], [], []
        for s0, ns in ((0, 1), (1, 3)):
            ctx.set_seed(0)
            ctx.set_shot_range(s0, ns)
            parts.append(ctx.gradient_accumulate(True))
            g, i = ctx.gradient_raw()
            gs.append(g)
            ils.append(i)
    assert abs(sum(parts) - whole) / whole < 1e-12
    # same random boundaries (seed reset), other float summation order
    assert rel_l2(gs[0] + gs[1], g_all) < 1e-6
    assert rel_l2(ils[0] + ils[1], i_all) < 1e-6


def test_one_rank_nccl_equals_plain_path(inv_case, tmp_path):
    import torch
    import torch.distributed as dist
    c, vp, init, obs = inv_case
    with api.Context(c.params, api.MODE_INVERSION) as ctx:
        ctx.set_model(init)
        ctx.set_observed(obs)
        s = ctx.compute_gradient(True)
        f0 = float(np.sqrt(np.float32(s)))
        step = ctx.optimization(f0)
        plain = ctx.update_model(step)
    dist.init_process_group("nccl", init_method=f"file://{tmp_path}/store", rank=0, world_size=1)
    try:
        with api.Context(c.params, api.MODE_INVERSION) as ctx:
            ctx.set_model(init)
            ctx.set_observed(obs)
            run = ShardedInversion(ctx, wrap=cuda_wrap)
            st = run.iterate(update=True)
            assert run.residuo[0] == f0
            assert st == step
            assert np.array_equal(ctx.get_model(), plain)
    finally:
        dist.destroy_process_group()
