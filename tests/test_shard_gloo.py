"""Sharding (fastspec_b200.shard) on two and three CPU ranks over gloo, with the oracle as the
backend.  Wavelength axis: the orchestration (line slices, the window all-gather, the balanced
wavelength ranges, the flux gather) must reproduce the single-process oracle synthesis.  Batch axis:
the cost partition and the gather to rank 0 must return every synthesis of the batch unchanged."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import helpers as H


class OracleBackend:
    """The oracle standing in for the CUDA library behind fastspec_b200.shard.run."""

    def __init__(self, oracle, grid, st, co, arrays, nmu=7):
        self.o, self.a = oracle, arrays
        self.S = oracle.State(grid, st, contopac=co, vmicro=1.0)
        self.n, self.nwl = len(arrays["wl"]), self.S.nwl
        self.x, self.w, _ = oracle.mu_quadrature(1, nmu)

    def _lines(self, sel):
        return self.o.Lines(**{k: np.ascontiguousarray(v[sel]) for k, v in self.a.items()}, kind=2)

    def central(self, a, b, m):
        win = torch.zeros((3, m), dtype=torch.int32)
        win[0, b - a:] = 1
        if b > a:
            r = self.o.lineop_calc(self.S, self._lines(slice(a, b)), list_type=2)
            win[0, :b - a] = torch.from_numpy(r["flags"])
            win[1, :b - a] = torch.from_numpy(r["ileft"])
            win[2, :b - a] = torch.from_numpy(r["iright"])
        return win

    def accumulate(self, win, i0, i1):
        w = win.numpy()
        sel = ((w[0] & 1) == 0) & (w[1] <= i1) & (w[2] >= i0)
        r = self.o.lineop_calc(self.S, self._lines(sel), list_type=2)
        spl, spc = self.o.radtran(self.S, self.x, r["lineopac"])
        self.sfl, self.sfc = self.o.disk_integ(self.w, spl, spc)
        return {"lines": int(sel.sum())}

    def flux(self, i0, i1):
        return torch.from_numpy(np.stack([self.sfl[i0 - 1:i1], self.sfc[i0 - 1:i1]]))


def case():
    from fastspec_b200 import workloads as W
    import fastspec_b200 as F
    st, meta = H.load_atm("solar")
    w0, span = 5000.0, 3.0
    grid = dict(wmode=0, wstart=w0, wend=w0 + span, dstep=0.005)
    co = H.contopac_on(meta, F.make_grid(0, w0, w0 + span, 0.005) + w0)
    return grid, st, co, W.atomic_lines(301, w0 - 0.5, w0 + span + 0.5, 17).arrays()


def worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import oracle
    from fastspec_b200 import shard
    grid, st, co, arr = case()
    res = shard.run(OracleBackend(oracle, grid, st, co, arr))
    if rank == 0:
        np.savez(out, flux=res["flux"].numpy(), ranges=np.array(res["ranges"]), windows=res["windows"].numpy())
    dist.barrier()
    dist.destroy_process_group()


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_synthesis_matches_single_process(tmp_path, oracle_mod, world):
    out = str(tmp_path / "res.npz")
    mp.start_processes(worker, args=(world, free_port(), out), nprocs=world, join=True, start_method="spawn")
    r = np.load(out)
    grid, st, co, arr = case()
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0)
    full = oracle_mod.lineop_calc(S, oracle_mod.Lines(**arr, kind=2), list_type=2)
    x, w, _ = oracle_mod.mu_quadrature(1, 7)
    sfl, sfc = oracle_mod.disk_integ(w, *oracle_mod.radtran(S, x, full["lineopac"]))
    # the gathered windows are the whole-list central pass
    assert np.array_equal(r["windows"][0] & 1, full["flags"] & 1)
    assert np.array_equal(r["windows"][1:], np.stack([full["ileft"], full["iright"]]))
    # ranges: contiguous, in order, covering the grid
    rg = r["ranges"]
    assert rg[0][0] == 1 and rg[-1][1] == S.nwl and all(rg[k + 1][0] == rg[k][1] + 1 for k in range(world - 1))
    # a rank's list holds only the lines meeting its range, so MarkWideLines (which counts the lines
    # inside a window, synth.f90:709-744) can class a line differently and the FP64 sums of a
    # wavelength change order: 1e-16 in LineOpac, ~1e-12 in the flux after the DELO sweep
    assert np.max(np.abs(r["flux"][0] / sfl - 1)) < 1e-10
    assert np.max(np.abs(r["flux"][1] / sfc - 1)) < 1e-12


def test_balanced_ranges_and_slices():
    from fastspec_b200 import shard
    cost = torch.tensor([0, 0, 10, 10, 10, 10, 0, 0, 40, 0], dtype=torch.int64)
    rg = shard.balanced_ranges(cost, 2)
    assert rg[0][0] == 1 and rg[1][1] == 10 and rg[1][0] == rg[0][1] + 1
    w = (cost.double() + 1).numpy()
    s0, s1 = w[rg[0][0] - 1:rg[0][1]].sum(), w[rg[1][0] - 1:rg[1][1]].sum()
    assert abs(s0 - s1) <= 41
    assert shard.balanced_ranges(torch.zeros(1, dtype=torch.int64), 3)[1][0] > shard.balanced_ranges(
        torch.zeros(1, dtype=torch.int64), 3)[1][1]                       # more ranks than wavelengths: empty ranges
    assert [shard.line_slice(10, 3, r) for r in range(3)] == [(0, 4, 4), (4, 8, 4), (8, 10, 4)]
    win = torch.tensor([[0, 1, 0], [2, 1, 5], [4, 9, 5]], dtype=torch.int32)
    c = shard.pixel_cost(win, 6)
    assert c.tolist() == [0, 1, 1, 1, 1, 0]


# ---- batch axis ------------------------------------------------------------------------------

def batch_cases():
    """Six small independent syntheses of the solar state: different spans, steps, angle sets and
    microturbulence, one line list covering all of them."""
    from fastspec_b200 import workloads as W
    import fastspec_b200 as F
    st, meta = H.load_atm("solar")
    specs = [(5000.0, 1.0, 0.005, 7, 1.0), (5001.0, 2.5, 0.01, 5, 0.5), (5002.0, 0.5, 0.005, 3, 2.0),
             (5000.5, 3.0, 0.02, 7, 1.5), (5003.0, 1.0, 0.0025, 9, 1.0), (5001.5, 0.2, 0.005, 7, 0.0)]
    cases = []
    for w0, span, dstep, nmu, vmic in specs:
        grid = dict(wmode=0, wstart=w0, wend=w0 + span, dstep=dstep)
        co = H.contopac_on(meta, F.make_grid(0, w0, w0 + span, dstep) + w0)
        cases.append((grid, co, nmu, vmic))
    return st, cases, W.atomic_lines(200, 4999.0, 5005.0, 23).arrays()


class OracleBatchBackend:
    def __init__(self, oracle, st, cases, arrays):
        self.o, self.st, self.cases, self.a = oracle, st, cases, arrays

    def one(self, i):
        grid, co, nmu, vmic = self.cases[i]
        S = self.o.State(grid, self.st, contopac=co, vmicro=vmic)
        r = self.o.lineop_calc(S, self.o.Lines(**self.a, kind=2), list_type=2)
        x, w, _ = self.o.mu_quadrature(1, nmu)
        return np.stack(self.o.disk_integ(w, *self.o.radtran(S, x, r["lineopac"])))

    def synthesize(self, idx):
        return [torch.from_numpy(self.one(i)) for i in idx]


def batch_inputs(oracle):
    from fastspec_b200 import shard
    st, cases, arr = batch_cases()
    sizes = [oracle.State(g, st).nwl for g, _, _, _ in cases]
    costs = [shard.batch_cost(n, len(st["T"]), len(arr["wl"])) for n in sizes]
    return st, cases, arr, sizes, costs


def batch_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import oracle
    from fastspec_b200 import shard
    st, cases, arr, sizes, costs = batch_inputs(oracle)
    res, mine = shard.run_batch(OracleBatchBackend(oracle, st, cases, arr), costs, sizes)
    np.save(out + ".mine%d.npy" % rank, np.array(mine, np.int64))
    if rank == 0:
        np.savez(out, *[r.numpy() for r in res])
    else:
        assert res is None
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_batch_axis_returns_every_synthesis(tmp_path, oracle_mod, world):
    out = str(tmp_path / "batch.npz")
    mp.start_processes(batch_worker, args=(world, free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    r = np.load(out)
    st, cases, arr, sizes, costs = batch_inputs(oracle_mod)
    be = OracleBatchBackend(oracle_mod, st, cases, arr)
    assert len(r.files) == len(cases)
    for i in range(len(cases)):
        # each synthesis ran whole on one rank: the same arithmetic, bit for bit
        assert np.array_equal(r["arr_%d" % i], be.one(i))
    mine = [np.load(out + ".mine%d.npy" % k).tolist() for k in range(world)]
    assert sorted(sum(mine, [])) == list(range(len(cases)))
    assert all(len(m) > 0 for m in mine)


def test_batch_partition():
    from fastspec_b200 import shard
    costs = [5.0, 1.0, 9.0, 3.0, 3.0, 7.0, 2.0]
    parts = shard.batch_partition(costs, 3)
    assert sorted(sum(parts, [])) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - sum(costs) / 3 <= max(costs)
    assert parts == shard.batch_partition(list(costs), 3)              # deterministic
    assert 2 in parts[0] and sorted(loads) == [10.0, 10.0, 10.0]        # the largest to rank 0; even here
    assert shard.batch_partition(costs, 1) == [list(range(len(costs)))]
    assert shard.batch_partition([1.0], 3) == [[0], [], []]              # more ranks than syntheses
    assert shard.batch_cost(100, 50, 0) == 5000.0

