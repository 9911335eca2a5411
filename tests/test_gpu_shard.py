"""The device side of wavelength sharding on one GPU: fsg_central_dev over slices of a list gives the
whole-list windows, and fsg_accumulate_dev over adjacent wavelength ranges rebuilds the whole-grid
LineOpac (mixed-precision tolerance: the Kahan groups of the tiles cut by a range end differ)."""
import numpy as np
import pytest
import torch

import helpers as H

pytestmark = pytest.mark.gpu


def cooldwarf_case(n=4000, w0=9000.0, span=10.0, seed=23):
    from fastspec_b200 import workloads as W
    import fastspec_b200 as F
    st, meta = H.load_atm("cooldwarf")
    grid = dict(wmode=1, wstart=w0, wend=w0 + span, dstep=1.0)
    co = H.contopac_on(meta, F.make_grid(1, w0, w0 + span, 1.0) + w0)
    return grid, st, co, W.molecular_lines(n, w0 - 3, w0 + span + 3, seed).arrays()


def make(fsg, grid, st, co, prec=None):
    C = fsg.Context(precision=fsg.PREC_MIXED if prec is None else prec, vmicro=1.0, molbrd=1)
    C.set_grid(grid["wmode"], grid["wstart"], grid["wend"], grid["dstep"])
    C.set_atmosphere(st)
    C.set_contopac(co)
    x, w, _ = fsg.mu_quadrature(1, 7)
    C.set_mu(x, w)
    return C


def test_central_slices_and_range_accumulation(fsg):
    from fastspec_b200 import shard
    grid, st, co, arr = cooldwarf_case()
    C = make(fsg, grid, st, co)
    full = C.lineop_calc(fsg.LineList.from_arrays(arr))
    _, _, sfl, sfc = C.radtran()
    dt = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in arr.items()}
    B = shard.GpuBackend(fsg, C, dt)
    n = B.n
    parts = [B.central(*shard.line_slice(n, 3, r)) for r in range(3)]
    win = torch.cat(parts, dim=1)[:, :n].cpu().numpy()
    assert np.array_equal(win[0], full["flags"])
    assert np.array_equal(win[1], full["ileft"]) and np.array_equal(win[2], full["iright"])
    wt = torch.from_numpy(win).cuda()
    ranges = shard.balanced_ranges(shard.pixel_cost(wt, C.nwl), 3)
    assert ranges[0][0] == 1 and ranges[-1][1] == C.nwl
    C.lineop_reset()
    flux = []
    for i0, i1 in ranges:
        st_ = C.accumulate_dev(B.full, wt[0].data_ptr(), wt[1].data_ptr(), wt[2].data_ptr(), i0, i1)
        assert st_["line_evals"] > 0
    lo = C.lineop_get()
    ref = full["lineopac"]
    assert np.max(np.abs(lo - ref) / (ref + co)) < 2e-7
    # one range alone leaves the rest of LineOpac untouched, and its flux matches the whole-grid flux
    i0, i1 = ranges[1]
    C.lineop_reset()
    C.accumulate_dev(B.full, wt[0].data_ptr(), wt[1].data_ptr(), wt[2].data_ptr(), i0, i1)
    lo1 = C.lineop_get()
    assert np.all(lo1[:i0 - 1] == 0) and np.all(lo1[i1:] == 0)
    f = B.flux(i0, i1).cpu().numpy()
    assert np.max(np.abs(f[0] / sfl[i0 - 1:i1] - 1)) < 1e-6
    assert np.max(np.abs(f[1] / sfc[i0 - 1:i1] - 1)) < 1e-12


def test_range_accumulation_fp64_and_bad_ranges(fsg):
    """FP64: adjacent ranges rebuild the whole-grid LineOpac bit for bit (same segments, same order
    per wavelength); ranges outside 1..nwl or empty are refused."""
    from fastspec_b200 import shard
    grid, st, co, arr = cooldwarf_case(n=3000, seed=24)
    C = make(fsg, grid, st, co, prec=fsg.PREC_FP64)
    full = C.lineop_calc(fsg.LineList.from_arrays(arr))
    dt = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in arr.items()}
    B = shard.GpuBackend(fsg, C, dt)
    win = B.central(0, B.n, B.n)
    assert np.array_equal(win[1].cpu().numpy(), full["ileft"])
    C.lineop_reset()
    nwl = C.nwl
    for i0, i1 in ((1, nwl // 3), (nwl // 3 + 1, nwl // 2), (nwl // 2 + 1, nwl)):
        C.accumulate_dev(B.full, win[0].data_ptr(), win[1].data_ptr(), win[2].data_ptr(), i0, i1)
    assert np.array_equal(C.lineop_get(), full["lineopac"])
    with pytest.raises(fsg.FsgError):
        C.accumulate_dev(B.full, win[0].data_ptr(), win[1].data_ptr(), win[2].data_ptr(), 0, nwl)
    with pytest.raises(fsg.FsgError):
        C.accumulate_dev(B.full, win[0].data_ptr(), win[1].data_ptr(), win[2].data_ptr(), 5, 4)


def test_radtran_range_solves_only_its_rows(fsg):
    """fsg_radtran_range_dev writes rows i0..i1 of whole-grid outputs, equal to the whole-grid solve,
    and leaves the other rows as they were."""
    grid, st, co, arr = cooldwarf_case(n=800, seed=25)
    C = make(fsg, grid, st, co)
    C.lineop_calc(fsg.LineList.from_arrays(arr), want_lineopac=False, want_lines=False)
    spl, spc, sfl, sfc = C.radtran()
    nwl, nmu = C.nwl, C.nmu
    i0, i1 = nwl // 4, nwl // 2
    out = [torch.full((nwl, nmu), -7.0, dtype=torch.float64, device="cuda"),
           torch.full((nwl, nmu), -7.0, dtype=torch.float64, device="cuda"),
           torch.full((nwl,), -7.0, dtype=torch.float64, device="cuda"),
           torch.full((nwl,), -7.0, dtype=torch.float64, device="cuda")]
    torch.cuda.synchronize()
    C.radtran_range_dev(i0, i1, *[t.data_ptr() for t in out])
    got = [t.cpu().numpy() for t in out]
    for g, ref in zip(got, (spl, spc, sfl, sfc)):
        assert np.array_equal(g[i0 - 1:i1], ref[i0 - 1:i1])
        assert np.all(g[:i0 - 1] == -7.0) and np.all(g[i1:] == -7.0)
    with pytest.raises(fsg.FsgError):
        C.radtran_range_dev(0, 5, None, None, out[2].data_ptr(), None)
    with pytest.raises(fsg.FsgError):
        C.radtran_range_dev(10, nwl + 1, None, None, out[2].data_ptr(), None)


def test_range_adjoints_sum_to_the_whole_gradient(fsg):
    """fsg_adjoint_range_dev over a partition of the grid into three ranges, summed, equals the
    whole-grid fsg_adjoint_dev (dL/d ln gf and the vmicro shares of every line); the ranges' own
    LineOpac is the only opacity the sharded forward gives each rank."""
    from fastspec_b200 import shard
    grid, st, co, arr = cooldwarf_case(n=1500, seed=26)
    C = make(fsg, grid, st, co)
    dt = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in arr.items()}
    B = shard.GpuBackend(fsg, C, dt)
    n, nwl = B.n, C.nwl
    win = B.central(0, n, n)
    g = torch.from_numpy(np.random.default_rng(8).normal(0, 1, nwl)).cuda()
    glin = torch.empty(n, dtype=torch.float64, device="cuda")
    gvm = torch.empty_like(glin)
    torch.cuda.synchronize()
    C.lineop_reset()
    C.lineop_calc_dev(B.full)                      # the whole-grid adjoint reads the context's own windows
    C.radtran_dev(None, None, B.sfl.data_ptr(), B.sfc.data_ptr())
    C.adjoint_dev(B.full, g.data_ptr(), glin.data_ptr(), gvm.data_ptr())
    ref_lin, ref_vm = glin.cpu().numpy(), gvm.cpu().numpy()
    sum_lin, sum_vm = np.zeros(n), np.zeros(n)
    ranges = shard.balanced_ranges(shard.pixel_cost(win, nwl), 3)
    for i0, i1 in ranges:
        C.lineop_reset()
        C.accumulate_dev(B.full, win[0].data_ptr(), win[1].data_ptr(), win[2].data_ptr(), i0, i1)
        gl, gv = B.adjoint(win, i0, i1, g)
        sum_lin += gl.cpu().numpy()
        sum_vm += gv.cpu().numpy()
    scale = np.max(np.abs(ref_lin))
    assert np.max(np.abs(sum_lin - ref_lin)) <= 1e-6 * scale
    assert np.max(np.abs(sum_vm - ref_vm)) <= 1e-6 * np.max(np.abs(ref_vm))
    assert np.count_nonzero(ref_lin) > n // 2
