"""Shot-sharded migration and inversion over torch.distributed (one process per GPU).

Shots are independent, so rank r of N owns a contiguous block of them
(shard()) and the only exchange is a sum per gradient (or image):

  inversion iteration (inversion.cu:111-166, 286-358 with the shots split)
    1. fwi_gradient_accumulate over the rank's shots: raw gradient,
       source illumination (nz x nx each, on the device) and the FP64 misfit
    2. all_reduce(SUM) of the two accumulators in place and of the misfit
    3. fwi_gradient_finish: post-processing, identical on every rank
    4. the two line-search trials: partial misfits, all_reduce(SUM) each
    5. fwi_parabola_step + fwi_update_model: identical on every rank

  migration: fwi_rtm_survey over the rank's shots, all_reduce(SUM) of image
  and illumination, fwi_rtm_image.

The accumulators are the context's own device buffers, wrapped for torch
through __cuda_array_interface__ (no copy); with the gloo backend on CPU the
caller passes its own `wrap` (tests use host arrays).  Every rank takes the
same collective steps in the same order, an empty shard included.

Run:  torchrun --nproc-per-node N -m fwi2d_b200.sharded parameters.txt [inversion|migration]
"""
from __future__ import annotations

import ctypes as C
import sys
from typing import Callable

import numpy as np


def shard(nsrc: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous block of shots of `rank`: sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    base, extra = divmod(nsrc, world)
    s0 = rank * base + min(rank, extra)
    return s0, base + (1 if rank < extra else 0)


class DeviceFloats:
    """A float32 device buffer owned elsewhere, importable by torch.as_tensor."""

    def __init__(self, address: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (address, False), "version": 3}


def cuda_wrap(address: int, n: int):
    import torch
    return torch.as_tensor(DeviceFloats(address, n), device="cuda")


def host_wrap(address: int, n: int):
    """Host float32 buffer at `address` as a CPU tensor (no copy)."""
    import torch
    return torch.from_numpy(np.ctypeslib.as_array((C.c_float * n).from_address(address)))


class _Sharded:
    def __init__(self, ctx, group=None, wrap: Callable | None = None):
        import torch
        import torch.distributed as dist
        self.ctx, self.group, self.dist, self.torch = ctx, group, dist, torch
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.s0, self.ns = shard(ctx.dims.nsrc, self.rank, self.world)
        ctx.set_shot_range(self.s0, self.ns)
        cpu = dist.get_backend(group) == "gloo"
        self.wrap = wrap or (host_wrap if cpu else cuda_wrap)
        self.device = "cpu" if cpu else "cuda"

    def _sum_scalar(self, x: float) -> float:
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return float(t.item())

    def _sum_accumulators(self) -> None:
        a, b, n = self.ctx.accumulators()  # the context's stream is idle here
        for addr in (a, b):
            self.dist.all_reduce(self.wrap(addr, n), op=self.dist.ReduceOp.SUM, group=self.group)
        if self.device == "cuda":
            self.torch.cuda.synchronize()  # the context's stream reads them next


class ShardedInversion(_Sharded):
    """One FWI iteration per call of iterate(); misfits as the reference reports them."""

    def __init__(self, ctx, group=None, wrap: Callable | None = None):
        super().__init__(ctx, group, wrap)
        self.residuo: list[float] = []

    def misfit(self) -> float:
        """Sum of squared residuals over all shots (no gradient)."""
        return self._sum_scalar(self.ctx.gradient_accumulate(False))

    def iterate(self, update: bool = True) -> float:
        """compute_gradient + check_convergence (+ optimization + update_model);
        returns the step (0 without update)."""
        ctx = self.ctx
        sum_res = self._sum_scalar(ctx.gradient_accumulate(update))
        self.residuo.append(float(np.sqrt(np.float32(sum_res))))
        if not update:
            return 0.0
        self._sum_accumulators()
        ctx.gradient_finish()
        a1, a2 = ctx.trial_steps()
        f1 = float(np.sqrt(np.float32(self._sum_scalar(ctx.linesearch_trial(a1)))))
        f2 = float(np.sqrt(np.float32(self._sum_scalar(ctx.linesearch_trial(a2)))))
        step = ctx.parabola_step(self.residuo[-1], f1, f2)
        ctx.update_model(step)
        return step


class ShardedMigration(_Sharded):
    def migrate(self, data_all: np.ndarray) -> np.ndarray:
        """RTM of the rank's shots of data_all (nsrc, nt, nrec), summed over ranks."""
        self.ctx.rtm_reset()
        if self.ns:
            self.ctx.rtm_survey(data_all)
        self._sum_accumulators()
        return self.ctx.rtm_image()


def main(argv: list[str]) -> int:
    import datetime
    import os

    import torch
    import torch.distributed as dist

    from . import api
    params = argv[1]
    what = argv[2] if len(argv) > 2 else "inversion"
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if what == "migration":
            mig = api.Migration(params)
            mig.set_parameters()
            d = mig.ctx.dims
            folder, prefix = mig.ctx.param("mig_input_folder"), mig.ctx.param("mig_input_prefix")
            data = np.stack([np.fromfile(f"{folder}{prefix}{s + 1}.bin", np.float32, d.nt * d.nrec)
                             .reshape(d.nrec, d.nt).T for s in range(d.nsrc)])
            ShardedMigration(mig.ctx).migrate(data)
            if dist.get_rank() == 0:
                print(mig.export_seismic())
            mig.ctx.close()
        else:
            inv = api.Inversion(params)
            inv.set_parameters()
            run = ShardedInversion(inv.ctx)
            for it in range(inv.max_iteration + 1):
                run.iterate(update=it < inv.max_iteration)
                if dist.get_rank() == 0:
                    print(f"iteration {it}: residuo {run.residuo[-1]:.6g}", flush=True)
            inv.ctx.close()
    finally:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
