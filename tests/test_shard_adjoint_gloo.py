"""The wavelength-sharded gradient (fastspec_b200.shard.adjoint) on two and three CPU ranks over gloo.
The backend is a stand-in with the structure of the library's range adjoint: each line's gradient is a
linear functional of dL/dflux over the part of its window inside the rank's range, plus an edge term
where the window's own edge lies in the range.  Summed over the ranks by the one all-reduce, the
result must equal the same functional over the whole grid in one process."""
import os

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from test_shard_gloo import free_port


def windows(n=400, nwl=900, seed=4):
    rng = np.random.default_rng(seed)
    il = rng.integers(1, nwl, n)
    ir = np.minimum(il + rng.integers(0, 200, n), nwl)
    fl = np.where(rng.uniform(0, 1, n) < 0.1, 1, 0)
    return torch.from_numpy(np.stack([fl, il, ir]).astype(np.int32)), nwl


class LinearAdjointBackend:
    """glin_l = sum over p in window_l and [i0, i1] of g[p] * w_l(p) + edge terms inside the range."""

    def __init__(self, win, nwl, seed=5):
        self.n, self.nwl, self.win = win.shape[1], nwl, win
        rng = np.random.default_rng(seed)
        self.scale = torch.from_numpy(rng.uniform(0.5, 2.0, self.n))

    def adjoint(self, win, i0, i1, gflux):
        glin = torch.zeros(self.n, dtype=torch.float64)
        gvm = torch.zeros(self.n, dtype=torch.float64)
        p = torch.arange(1, self.nwl + 1, dtype=torch.float64)
        for l in range(self.n):
            f, il, ir = (int(x) for x in win[:, l])
            if f & 1:
                continue
            a, b = max(il, i0), min(ir, i1)
            if a <= b:
                glin[l] = (gflux[a - 1:b] * torch.sqrt(p[a - 1:b]) * self.scale[l]).sum()
                gvm[l] = (gflux[a - 1:b] * self.scale[l] / p[a - 1:b]).sum()
            if i0 <= il <= i1:
                glin[l] += 3.0 * gflux[il - 1]
            if i0 <= ir <= i1:
                gvm[l] += 2.0 * gflux[ir - 1]
        return glin, gvm


def grad_worker(rank, world, port, out):
    import torch.distributed as dist
    from fastspec_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    win, nwl = windows()
    be = LinearAdjointBackend(win, nwl)
    ranges = shard.balanced_ranges(shard.pixel_cost(win, nwl), world)
    g = torch.from_numpy(np.random.default_rng(6).normal(0, 1, nwl))
    res = dict(windows=win, range=ranges[rank], ranges=ranges)
    glin, gvm = shard.adjoint(be, res, g)
    np.savez(out + ".rank%d.npz" % rank, glin=glin.numpy(), gvm=gvm.numpy(), ranges=np.array(ranges))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_gradient_sums_to_whole_grid(tmp_path, world):
    out = str(tmp_path / "grad")
    mp.start_processes(grad_worker, args=(world, free_port(), out), nprocs=world, join=True, start_method="spawn")
    win, nwl = windows()
    be = LinearAdjointBackend(win, nwl)
    g = torch.from_numpy(np.random.default_rng(6).normal(0, 1, nwl))
    ref_lin, ref_vm = be.adjoint(win, 1, nwl, g)
    for r in range(world):
        d = np.load(out + ".rank%d.npz" % r)
        # every rank holds the whole gradient; ranks' sums are in a different order: rounding only
        np.testing.assert_allclose(d["glin"], ref_lin.numpy(), rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(d["gvm"], ref_vm.numpy(), rtol=1e-12, atol=1e-12)
        assert len(d["ranges"]) == world
