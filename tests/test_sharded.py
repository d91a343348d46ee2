"""Shot-sharded inversion / migration driver (fwi2d_b200.sharded) on CPU.

Two gloo ranks run the driver over a host-side stand-in of the context that
keeps the engine's contract (per-shot partial misfits and accumulators over
the context's shot range, post-processing of the summed accumulators, the
parabola step of inversion.cu:286-308).  The sharded run must equal the
one-process run: same misfits, steps and models on every rank."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fwi2d_b200.sharded import ShardedInversion, ShardedMigration, shard


class FakeDims:
    def __init__(self, nsrc, nz, nx):
        self.nsrc, self.nz, self.nx = nsrc, nz, nx


class FakeContext:
    """Per-shot 'physics': shot s sees target t_s; its residual is m - t_s on
    its own columns, its raw gradient that residual times an illumination."""

    def __init__(self, nsrc=7, nz=5, nx=11, seed=0):
        rng = np.random.default_rng(seed)
        self.dims = FakeDims(nsrc, nz, nx)
        self.targets = rng.uniform(0.5, 1.5, (nsrc, nz, nx)).astype(np.float32)
        self.illum_s = rng.uniform(1.0, 2.0, (nsrc, nz, nx)).astype(np.float32)
        self.m = np.ones((nz, nx), np.float32)
        self.img = np.zeros(nz * nx, np.float32)
        self.ill = np.zeros(nz * nx, np.float32)
        self.g = None
        self.s0, self.ns = 0, nsrc
        self.calls = []

    def set_shot_range(self, s0, ns):
        assert 0 <= s0 and 0 <= ns and s0 + ns <= self.dims.nsrc
        self.s0, self.ns = s0, ns

    def _misfit(self, m):
        return sum(float(((m - self.targets[s]).astype(np.float64) ** 2).sum()) for s in range(self.s0, self.s0 + self.ns))

    def gradient_accumulate(self, with_gradient=True):
        self.calls.append(("accumulate", self.s0, self.ns))
        if with_gradient:
            self.img[:] = 0
            self.ill[:] = 0
            for s in range(self.s0, self.s0 + self.ns):
                self.img += ((self.m - self.targets[s]) * self.illum_s[s]).ravel()
                self.ill += self.illum_s[s].ravel()
        return self._misfit(self.m)

    def accumulators(self):
        return self.img.ctypes.data, self.ill.ctypes.data, self.img.size

    def gradient_finish(self):
        q = (self.img / self.ill).reshape(self.m.shape)
        self.g = (q / np.abs(q).max()).astype(np.float32)

    def trial_steps(self):
        return 0.02, 0.05

    def linesearch_trial(self, alpha):
        return self._misfit(self.m - np.float32(alpha) * self.g)

    def parabola_step(self, f0, f1, f2):
        f32 = np.float32
        a0, a1, a2 = f32(0.0), f32(0.02), f32(0.05)
        f0, f1, f2 = f32(f0), f32(f1), f32(f2)
        num = (a1 * a1 - a2 * a2) * f0 + (a2 * a2 - a0 * a0) * f1 + (a0 * a0 - a1 * a1) * f2
        den = (a1 - a2) * f0 + (a2 - a0) * f1 + (a0 - a1) * f2
        return float(f32(0.5) * (num / den))

    def update_model(self, step):
        self.m = (self.m - np.float32(step) * self.g).astype(np.float32)
        return self.m

    # migration
    def rtm_reset(self):
        self.img[:] = 0
        self.ill[:] = 0

    def rtm_survey(self, data):
        for s in range(self.s0, self.s0 + self.ns):
            self.img += data[s].ravel()
            self.ill += 1.0

    def rtm_image(self):
        return (self.img / self.ill).reshape(self.m.shape)


def test_shard_partitions_every_shot_once():
    for nsrc in (0, 1, 5, 7, 81, 240):
        for world in (1, 2, 3, 4, 8):
            parts = [shard(nsrc, r, world) for r in range(world)]
            assert parts[0][0] == 0 and sum(n for _, n in parts) == nsrc
            for (a, n), (b, _) in zip(parts, parts[1:]):
                assert a + n == b
            assert max(n for _, n in parts) - min(n for _, n in parts) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, nsrc, iters, out):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        ctx = FakeContext(nsrc=nsrc)
        run = ShardedInversion(ctx)
        steps = [run.iterate(update=it < iters) for it in range(iters + 1)]
        data = np.random.default_rng(3).standard_normal((nsrc, 5, 11)).astype(np.float32)
        img = ShardedMigration(ctx).migrate(data)
        np.savez(os.path.join(out, f"rank{rank}.npz"), m=ctx.m, residuo=np.array(run.residuo),
                 steps=np.array(steps), img=img, s0=run.s0, ns=run.ns)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nsrc", [(2, 7), (2, 1)])
def test_sharded_run_equals_single_process(tmp_path, world, nsrc):
    iters = 3
    mp.start_processes(_rank_main, args=(world, _free_port(), nsrc, iters, str(tmp_path)), nprocs=world,
                       start_method="spawn")
    ranks = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    # one process, same driver logic without collectives
    ctx = FakeContext(nsrc=nsrc)
    residuo, steps = [], []
    for it in range(iters + 1):
        s = ctx.gradient_accumulate(it < iters)
        residuo.append(float(np.sqrt(np.float32(s))))
        if it == iters:
            steps.append(0.0)
            break
        ctx.gradient_finish()
        f1 = float(np.sqrt(np.float32(ctx.linesearch_trial(0.02))))
        f2 = float(np.sqrt(np.float32(ctx.linesearch_trial(0.05))))
        st = ctx.parabola_step(residuo[-1], f1, f2)
        assert np.isfinite(st)
        steps.append(st)
        ctx.update_model(st)
    data = np.random.default_rng(3).standard_normal((nsrc, 5, 11)).astype(np.float32)
    ctx.rtm_reset()
    ctx.rtm_survey(data)
    img = ctx.rtm_image()
    assert sum(int(r["ns"]) for r in ranks) == nsrc
    for r in ranks:
        np.testing.assert_allclose(r["residuo"], residuo, rtol=1e-6)
        np.testing.assert_allclose(r["steps"], steps, rtol=1e-5)
        np.testing.assert_allclose(r["m"], ctx.m, rtol=1e-5)
        np.testing.assert_allclose(r["img"], img, rtol=1e-5, atol=1e-7)  # float32 sums, other order
    # every rank ends with the identical model
    for r in ranks[1:]:
        assert np.array_equal(r["m"], ranks[0]["m"])
