"""Wavelength sharding of one synthesis over the ranks of a torch.distributed process group.

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

The arithmetic of each wavelength is the one of a single-GPU run; only which GPU does it changes.
The work is done by a backend: `GpuBackend` drives the CUDA library through its device entry
points (fsg_central_dev, fsg_accumulate_dev, fsg_radtran_dev).
"""
import ctypes as C

import numpy as np
import torch
import torch.distributed as dist


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
        self.C.radtran_dev(None, None, self.sfl.data_ptr(), self.sfc.data_ptr())
        return torch.stack([self.sfl[i0 - 1:i1], self.sfc[i0 - 1:i1]])
