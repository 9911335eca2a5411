"""Sharding over the ranks of a torch.distributed process group: the wavelength axis of one
synthesis (`run`) and the batch axis of many independent syntheses (`run_batch`).

One synthesis (one atmosphere, one line list, one grid) splits along the wavelength axis, the
sharding the reference's own loop structure allows (LineopCalc's accumulation, synth.f90:1075-1080,
and RadTranCalc, synth.f90:1825-1866, are independent per wavelength once the windows are known):

1. rank r runs the central pass (XlineSetup/XlineDepth, rejection, AnalyticWindow + WaveIdx) on the
   r-th slice of the line list, which every rank holds;
2. one all-gather exchanges LinFlag, Ileft and Iright of every line (12 bytes per line);
3. every rank derives the same contiguous wavelength ranges of about equal evaluation count from
   the gathered windows (a difference array of the windows, its prefix sum and a search);
4. rank r accumulates the lines whose windows meet its range, over that range only, and runs the
   formal solver and the flux quadrature there;
5. the flux slices are gathered to every rank.

The gradient of a loss of the flux splits the same way (`adjoint`): rank r runs the adjoint over its
range with the gathered windows (fsg_adjoint_range_dev: each line's sums over the part of its window
inside the range), and one all-reduce sums the per-line dL/d ln gf and vmicro shares over the ranks.
The adjoint is linear in dL/dflux and the ranges cover each window point once, so the sum is the
whole-grid gradient.

Between steps, `check_peers` is a heartbeat through the process group's store: every rank posts the
step number and waits, with a bound, for the others'; a rank that has left is reported (PeerLost)
before any collective of the next step is started, so no collective waits on it.

The arithmetic of each wavelength is the one of a single-GPU run; only which GPU does it changes.
The work is done by a backend: `GpuBackend` drives the CUDA library through its device entry
points (fsg_central_dev, fsg_accumulate_dev, fsg_radtran_dev).

Batch axis: atmospheres, abundance sets and angle sets of a grid are independent syntheses.  They
are split over the ranks by a static partition on estimated cost (wavelengths x depths x candidate
lines, longest first to the least loaded rank), each rank runs its share (`BatchGpuBackend`: one
batched CUDA graph over its atmospheres), and the fluxes are gathered to rank 0 in the grid's order.
No opacity crosses between GPUs.
"""
import ctypes as C

import numpy as np
import torch
import torch.distributed as dist


class PeerLost(RuntimeError):
    """Ranks of the group that did not reach a step (they left or hang)."""

    def __init__(self, step, ranks):
        super().__init__("ranks %s did not reach step %d" % (list(ranks), step))
        self.step, self.ranks = step, list(ranks)


def check_peers(step, timeout_s=10.0, group=None):
    """Heartbeat before `step`: post this rank's arrival in the process group's store and wait at most
    timeout_s for every other rank's; raises PeerLost naming the ranks that did not arrive."""
    import datetime
    store = dist.distributed_c10d._get_default_store()
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    store.set("fsg_step%d_rank%d" % (step, rank), "1")
    missing = []
    deadline = datetime.timedelta(seconds=float(timeout_s))
    for r in range(world):
        if r == rank:
            continue
        try:
            store.wait(["fsg_step%d_rank%d" % (step, r)], deadline)
        except Exception:
            missing.append(r)
            deadline = datetime.timedelta(seconds=0.1)    # the bound is spent: poll the rest
    if missing:
        raise PeerLost(step, missing)


def line_slice(n, world, rank):
    """Contiguous slice [a, b) of n lines for rank, and the padded slice length m (same on all ranks)."""
    m = (n + world - 1) // world if n > 0 else 0
    a = min(n, rank * m)
    b = min(n, a + m)
    return a, b, m


def pixel_cost(win, nwl):
    """Retained windows covering each wavelength (the accumulation's work per wavelength), int64 [nwl].
    win: int32 [3, n] = LinFlag, Ileft, Iright (1-based, inclusive)."""
    keep = (win[0] & 1) == 0
    il = win[1][keep].long() - 1
    ir = win[2][keep].long()
    d = torch.zeros(nwl + 1, dtype=torch.int64, device=win.device)
    d.index_add_(0, il, torch.ones_like(il))
    d.index_add_(0, ir, -torch.ones_like(ir))
    return torch.cumsum(d[:-1], 0)


def balanced_ranges(cost, world):
    """Contiguous 1-based inclusive ranges (i0, i1), one per rank, covering 1..nwl in order with about
    equal summed cost; every wavelength also carries one unit for the solver.  A rank may get an
    empty range (i0 > i1) when there are fewer wavelengths than ranks."""
    nwl = int(cost.numel())
    w = cost.double() + 1.0
    cum = torch.cumsum(w, 0)
    total = float(cum[-1]) if nwl else 0.0
    bounds = [0]
    for k in range(1, world):
        b = int(torch.searchsorted(cum, torch.tensor([total * k / world], dtype=torch.float64,
                                                     device=cum.device)).item()) + 1
        bounds.append(min(max(b, bounds[-1]), nwl))
    bounds.append(nwl)
    return [(bounds[r] + 1, bounds[r + 1]) for r in range(world)]


def all_gather_rows(t, group=None):
    """all_gather of an equally shaped tensor from every rank, concatenated along the last axis."""
    world = dist.get_world_size(group)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t.contiguous(), group=group)
    return torch.cat(parts, dim=-1)


def run(backend, group=None):
    """One sharded synthesis.  Returns dict(flux: float64 [2, nwl] (line+continuum, continuum) on
    every rank, ranges, range of this rank, stats of this rank's accumulation, windows [3, n])."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n, nwl = backend.n, backend.nwl
    a, b, m = line_slice(n, world, rank)
    win_local = backend.central(a, b, m)                  # int32 [3, m], padding rows marked weak
    win = all_gather_rows(win_local, group)[:, :n]
    ranges = balanced_ranges(pixel_cost(win, nwl), world)
    i0, i1 = ranges[rank]
    stats = backend.accumulate(win, i0, i1) if i0 <= i1 else None
    lmax = max(max(r1 - r0 + 1, 0) for r0, r1 in ranges)
    part = torch.zeros((2, lmax), dtype=torch.float64, device=win.device)
    if i0 <= i1:
        part[:, :i1 - i0 + 1] = backend.flux(i0, i1)
    parts = [torch.empty_like(part) for _ in range(world)]
    dist.all_gather(parts, part, group=group)
    flux = torch.cat([p[:, :max(r1 - r0 + 1, 0)] for p, (r0, r1) in zip(parts, ranges)], dim=1)
    return dict(flux=flux, ranges=ranges, range=(i0, i1), stats=stats, windows=win)


def adjoint(backend, res, gflux, group=None):
    """The wavelength-sharded gradient after `run`: gflux = dL/d(line flux) on the whole grid (each rank
    needs only its range's entries).  Returns (dL/d ln gf per line [n], dL/dvmicro per line [n]) summed
    over the ranks, on every rank."""
    i0, i1 = res["range"]
    n = backend.n
    if i0 <= i1:
        glin, gvm = backend.adjoint(res["windows"], i0, i1, gflux)
    else:
        glin = torch.zeros(n, dtype=torch.float64, device=res["windows"].device)
        gvm = torch.zeros_like(glin)
    buf = torch.cat([glin, gvm])
    dist.all_reduce(buf, group=group)
    return buf[:n], buf[n:]


class GpuBackend:
    """The CUDA library as the backend of `run`: a Context with grid, atmosphere, continuum and mu
    set, and the device copy of the whole line list (dict of torch tensors wl, elo, gf, grad, gqst,
    gvdw, spc, ismol; molecular/mixed kind 2 SoA).  The library works on its own stream and returns
    after its work there is done; torch's pending work is finished before each library call."""

    def __init__(self, F, ctx, dt, kind=2):
        self.F, self.C, self.dt, self.kind = F, ctx, dt, kind
        self.n = int(dt["wl"].numel())
        self.nwl = ctx.nwl
        self.dev = dt["wl"].device
        self.full = self._view(0, self.n)
        self.sfl = torch.empty(self.nwl, dtype=torch.float64, device=self.dev)
        self.sfc = torch.empty_like(self.sfl)

    def _view(self, a, b):
        F, dt = self.F, self.dt
        v = F.CLines()
        v.n = b - a
        v.kind = self.kind
        ptr = lambda t, ct: C.cast(t.data_ptr() + a * t.element_size(), C.POINTER(ct))
        v.wl = ptr(dt["wl"], C.c_double)
        for k in ("elo", "gf", "grad", "gqst", "gvdw"):
            setattr(v, k, ptr(dt[k], C.c_float))
        v.spc = ptr(dt["spc"], C.c_int32)
        if "ismol" in dt:
            v.ismol = ptr(dt["ismol"], C.c_int32)
        return v

    def central(self, a, b, m):
        win = torch.zeros((3, m), dtype=torch.int32, device=self.dev)
        win[0, b - a:] = 1                                 # padding rows: rejected
        torch.cuda.current_stream(self.dev).synchronize()
        if b > a:
            self.C.central_dev(self._view(a, b), win[0].data_ptr(), win[1].data_ptr(), win[2].data_ptr())
        return win

    def accumulate(self, win, i0, i1):
        win = win.contiguous()
        torch.cuda.current_stream(self.dev).synchronize()
        self.C.lineop_reset()
        return self.C.accumulate_dev(self.full, win[0].data_ptr(), win[1].data_ptr(), win[2].data_ptr(), i0, i1)

    def flux(self, i0, i1):
        self.C.radtran_range_dev(i0, i1, None, None, self.sfl.data_ptr(), self.sfc.data_ptr())
        return torch.stack([self.sfl[i0 - 1:i1], self.sfc[i0 - 1:i1]])

    def adjoint(self, win, i0, i1, gflux):
        """This rank's share of the gradient: fsg_adjoint_range_dev over [i0, i1] with the whole list's
        windows; gflux: dL/d(line flux) [nwl] (float64, this device)."""
        win = win.contiguous()
        g = gflux.to(self.dev, torch.float64).contiguous()
        glin = torch.empty(self.n, dtype=torch.float64, device=self.dev)
        gvm = torch.empty_like(glin)
        torch.cuda.current_stream(self.dev).synchronize()
        self.C.adjoint_range_dev(self.full, win[0].data_ptr(), win[1].data_ptr(), win[2].data_ptr(), i0, i1,
                                 g.data_ptr(), glin.data_ptr(), gvm.data_ptr())
        return glin, gvm


# ---- batch axis ------------------------------------------------------------------------------

def batch_cost(nwl, ntau, nlines):
    """Work estimate of one synthesis of a batch: wavelengths x depths x candidate lines."""
    return float(nwl) * float(ntau) * float(max(int(nlines), 1))


def batch_partition(costs, world):
    """Static partition of independent syntheses over `world` ranks: in order of decreasing cost (ties:
    lower index first) each goes to the rank with the least summed cost so far (ties: lower rank).
    Returns one ascending index list per rank; every rank derives the same lists from the same costs.
    The largest load exceeds the best possible by at most the largest single cost."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def run_batch(backend, costs, sizes, group=None, device=None):
    """Batch-axis sharding.  costs[i] and sizes[i] (wavelength count) of every synthesis are known on
    every rank; rank r runs batch_partition's share r through backend.synthesize(indices), which returns
    one float64 [2, sizes[i]] tensor (line+continuum flux, continuum flux) per index, on `device`.  The
    shares are packed, padded to the longest, and gathered to rank 0 (one collective) in a buffer on
    `device` (a CUDA device under NCCL; the host under gloo).  Returns (list of [2, sizes[i]] tensors in
    the original order on rank 0, None on the other ranks; this rank's indices)."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts = batch_partition(costs, world)
    mine = parts[rank]
    out = backend.synthesize(mine) if mine else []
    lens = [sum(2 * int(sizes[i]) for i in p) for p in parts]
    buf = torch.zeros(max(max(lens), 1), dtype=torch.float64, device=device)
    if mine:
        flat = torch.cat([f.reshape(-1).to(torch.float64) for f in out])
        assert flat.numel() == lens[rank], "backend returned fluxes of the wrong size"
        buf[:flat.numel()] = flat
    bufs = [torch.empty_like(buf) for _ in range(world)] if rank == 0 else None
    dist.gather(buf, bufs, dst=0, group=group)
    if rank != 0:
        return None, mine
    res = [None] * len(costs)
    for p, b in zip(parts, bufs):
        off = 0
        for i in p:
            n = int(sizes[i])
            res[i] = b[off:off + 2 * n].reshape(2, n)
            off += 2 * n
    return res, mine


class BatchGpuBackend:
    """The batched CUDA path as the backend of `run_batch`: make_context(i) returns synthesis i's mixed-
    precision Context (grid, atmosphere, continuum, mu set); one fastspec_b200.Batch over this rank's
    contexts and the shared line list runs them in one graph replay; the fluxes come back as float64
    tensors on `device`."""

    def __init__(self, F, make_context, lines, device, margin=0.0):
        self.F, self.make_context, self.lines, self.device, self.margin = F, make_context, lines, device, margin
        self.batch = None

    def synthesize(self, idx):
        self.contexts = [self.make_context(i) for i in idx]
        self.batch = self.F.Batch(self.contexts, self.lines, self.margin)
        self.stats = self.batch.run()
        out = []
        for k in range(len(idx)):
            sfl, sfc = self.batch.flux(k)
            out.append(torch.from_numpy(np.stack([sfl, sfc])).to(self.device))
        return out

