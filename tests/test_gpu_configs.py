"""Parity of the GPU path with the FP64 oracle at the sizes of the benchmark configurations.

C0  plain scalar synthesis: the solar-like atmosphere (56 depths), 20,000 atomic lines over
    5000-5200 A at 0.005 A (40,001 wavelengths), 7 angles.
C2  Stokes IQUV synthesis: the Teff 5000 K atmosphere, 5,000 Zeeman lines over 6000-6100 A at
    0.002 A (50,001 wavelengths), BFRAME 1 with |B| = 2 kG at inclination 60 and azimuth 30 deg,
    9 angles.
C4  forward synthesis of the differentiable fit: the solar-like atmosphere, 1e5 atomic lines over
    4800-5300 A at 0.005 A (100,001 wavelengths), 7 angles.
C1  slices of the full cool-dwarf synthesis: the whole list of 1e8 molecular lines over
    5000-25000 A at R = 3e5 (482,832 wavelengths, 71 depths); the windows of every line on the
    whole grid, then the accumulation, intensities and flux over 5 A slices at 6000, 10000 and
    20000 A, against the oracle run on every line whose window reaches the slice.  Strong-line
    windows at this density span thousands of angstroms (up to the whole grid), so no fixed margin
    around a slice would find its lines; the windows decide.  The GPU windows of a random sample of
    one million of the other lines are checked against the oracle too, which is what makes the
    selection trustworthy.  The oracle's accumulation over the slice alone is its whole-grid
    accumulation restricted to those wavelengths (independent per wavelength, synth.f90:1075-1080).

Every list follows the reference's reader rule: a synthesis over [Wstart, Wend] reads the lines
whose centres lie in that range (ioutils.f90:752-753, 1496-1497).

Bars, as in test_gpu_accuracy.py: windows identical; FP64 path LineOpac 1e-11 of the total
opacity, intensities and flux 1e-9 relative; mixed path LineOpac 2e-6 of the total opacity,
intensities and flux 1e-5 relative; Zeeman profiles on the scale of the depth's peak absorption
profile; Stokes Q, U, V on the scale of the continuum intensity.  With FSG_CONFIGS_JSON set, the
measured maxima are written to that file.
"""
import json
import os

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

BARS = {"fp64": dict(lineopac=1e-11, intensity=1e-9, flux=1e-9),
        "mixed": dict(lineopac=2e-6, intensity=1e-5, flux=1e-5)}
RESULTS = {}
_ORACLE = {}


def record(case, prec, **errs):
    RESULTS.setdefault(case, {})[prec] = {k: float(v) for k, v in errs.items()}
    path = os.environ.get("FSG_CONFIGS_JSON")
    if path:
        with open(path, "w") as f:
            json.dump(RESULTS, f, indent=1, sort_keys=True)


def once(key, fn):
    """The oracle's result for a case, computed by the first precision that needs it."""
    if key not in _ORACLE:
        _ORACLE[key] = fn()
    return _ORACLE[key]


def context(fsg, prec, grid, st, co, nmu, **kw):
    C = fsg.Context(precision=fsg.PREC_FP64 if prec == "fp64" else fsg.PREC_MIXED, **kw)
    C.set_grid(grid["wmode"], grid["wstart"], grid["wend"], grid["dstep"])
    C.set_atmosphere(st)
    C.set_contopac(co)
    x, w, _ = fsg.mu_quadrature(1, nmu)
    C.set_mu(x, w)
    return C, x, w


def scalar_config(fsg, oracle_mod, prec, key, atm, grid, lines):
    """LineopCalc + RadTranCalc + flux through the C-ABI against the oracle on the same inputs."""
    st, meta = H.load_atm(atm)
    wave = fsg.make_grid(grid["wmode"], grid["wstart"], grid["wend"], grid["dstep"]) + grid["wstart"]
    co = H.contopac_on(meta, wave)
    a = lines.arrays()
    C, x, w = context(fsg, prec, grid, st, co, 7, vmicro=meta["vmicro"], molbrd=meta["molbrd"])
    g = C.lineop_calc(fsg.LineList.from_arrays(a))
    spl, spc, sfl, sfc = C.radtran()
    C.close()

    def run():
        S = oracle_mod.State(grid, st, contopac=co, vmicro=meta["vmicro"], molbrd=meta["molbrd"])
        r = oracle_mod.lineop_calc(S, oracle_mod.Lines(**a, kind=2), list_type=2)
        ospl, ospc = oracle_mod.radtran(S, x, r["lineopac"])
        osfl, osfc = oracle_mod.disk_integ(w, ospl, ospc)
        return r, ospl, ospc, osfl, osfc
    r, ospl, ospc, osfl, osfc = once(key, run)
    keep = (r["flags"] & 1) == 0
    e = dict(lines=len(a["wl"]), retained=int(keep.sum()), wavelengths=len(wave),
             windows_differing=int(np.sum(g["ileft"][keep] != r["ileft"][keep]) +
                                   np.sum(g["iright"][keep] != r["iright"][keep])),
             retained_differing=int(np.sum(((g["flags"] & 1) == 0) != keep)),
             lineopac=np.max(np.abs(g["lineopac"] - r["lineopac"]) / (r["lineopac"] + co)),
             intensity=np.max(np.abs(spl / ospl - 1)), cont_intensity=np.max(np.abs(spc / ospc - 1)),
             flux=np.max(np.abs(sfl / osfl - 1)), cont_flux=np.max(np.abs(sfc / osfc - 1)),
             line_evals_gpu=g["stats"]["line_evals"],
             line_evals_oracle=r["stats"]["line_evals"] + r["stats"]["wide_evals"],
             line_depth_max=np.max(1.0 - osfl / osfc))
    record(key, prec, **e)
    b = BARS[prec]
    assert e["retained_differing"] == 0 and e["windows_differing"] == 0
    assert e["lineopac"] < b["lineopac"], e
    assert e["intensity"] < b["intensity"] and e["flux"] < b["flux"], e
    assert e["cont_intensity"] < 1e-9 and e["cont_flux"] < 1e-9, e


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_c0_plain_scalar_synthesis(fsg, oracle_mod, prec):
    from fastspec_b200 import workloads as W
    w0, w1 = 5000.0, 5200.0
    grid = dict(wmode=0, wstart=w0, wend=w1, dstep=0.005)
    lines = W.atomic_lines(20000, w0, w1, W.SEED0 + 0, exact=False)
    scalar_config(fsg, oracle_mod, prec, "c0", "solar", grid, lines)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_c4_fit_forward_synthesis(fsg, oracle_mod, prec):
    from fastspec_b200 import workloads as W
    w0, w1 = 4800.0, 5300.0
    grid = dict(wmode=0, wstart=w0, wend=w1, dstep=0.005)
    lines = W.atomic_lines(100_000, w0, w1, W.SEED0 + 4, exact=False)
    scalar_config(fsg, oracle_mod, prec, "c4", "solar", grid, lines)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_c2_stokes_synthesis(fsg, oracle_mod, prec):
    from fastspec_b200 import workloads as W
    st, meta = H.load_atm("magnetic")
    w0, w1, step = 6000.0, 6100.0, 0.002
    grid = dict(wmode=0, wstart=w0, wend=w1, dstep=step)
    co = H.contopac_on(meta, fsg.make_grid(0, w0, w1, step) + w0)
    L = W.zeeman_lines(5000, w0, w1, W.SEED0 + 2)
    z = W.zeeman_components(L, oracle_mod.zeeman_pattern)
    a = L.arrays()
    bframe, bfield = 1, np.array([2000.0, 60.0, 30.0])
    C, x, w = context(fsg, prec, grid, st, co, 9, vmicro=meta["vmicro"])
    g = C.mag_lineop_calc(fsg.LineList.from_arrays(a, zeeman=z), bframe, bfield)
    spz, spc, sfl, sfc = C.mag_radtran(bframe, bfield)
    C.close()

    def run():
        S = oracle_mod.State(grid, st, contopac=co, vmicro=meta["vmicro"])
        r = oracle_mod.mag_lineop_calc(S, oracle_mod.Lines(**a, kind=2, zeeman=z), bframe, bfield)
        ospz, ospc = oracle_mod.mag_radtran(S, x, bframe, bfield, np.zeros((S.nwl, S.ntau)), r["maglineopac"])
        osfl, _ = oracle_mod.disk_integ(w, ospz[:, 0], ospc)
        return r, ospz, ospc, osfl
    r, ospz, ospc, osfl = once("c2", run)
    keep = (r["flags"] & 1) == 0
    m, om = g["maglineopac"], r["maglineopac"]
    scale = np.maximum(om[..., :3].max(axis=(0, 2)), 1e-300)[None, :, None]   # the depth's peak absorption
    e = dict(lines=L.n, retained=int(keep.sum()), wavelengths=len(co),
             windows_differing=int(np.sum(g["ileft"][keep] != r["ileft"][keep]) +
                                   np.sum(g["iright"][keep] != r["iright"][keep])),
             retained_differing=int(np.sum(((g["flags"] & 1) == 0) != keep)),
             maglineopac=np.max(np.abs(m - om) / scale), stokes_i=np.max(np.abs(spz[:, 0] / ospz[:, 0] - 1)),
             stokes_quv=max(np.max(np.abs(spz[:, q] - ospz[:, q]) / ospc) for q in (1, 2, 3)),
             cont_intensity=np.max(np.abs(spc / ospc - 1)), flux=np.max(np.abs(sfl / osfl - 1)))
    record("c2", prec, **e)
    b = BARS[prec]
    assert e["retained_differing"] == 0 and e["windows_differing"] == 0
    assert e["maglineopac"] < b["lineopac"] and e["stokes_i"] < b["intensity"] and e["flux"] < b["flux"], e
    assert e["stokes_quv"] < b["intensity"] and e["cont_intensity"] < 1e-9, e


# ---- C1: slices of the full 1e8-line cool-dwarf synthesis -------------------------------------------
C1_W0, C1_W1, C1_DSTEP = 5000.0, 25000.0, 2.99792458e5 / 3e5
C1_SLICES = (6000.0, 10000.0, 20000.0)
C1_SLICE_A = 5.0
C1_SAMPLE = 1_000_000


@pytest.fixture(scope="module")
def c1_full(fsg):
    """The whole C1 list on the device, its windows on the whole grid (central pass), the state and
    continuum; shared by every slice and precision."""
    import torch
    dev = torch.device("cuda:0")
    st, meta = H.load_atm("cooldwarf")
    grid = dict(wmode=1, wstart=C1_W0, wend=C1_W1, dstep=C1_DSTEP)
    wave = fsg.make_grid(1, C1_W0, C1_W1, C1_DSTEP) + C1_W0
    co = H.contopac_on(meta, wave)
    dt = H.device_molecular_lines(100_000_000, C1_W0, C1_W1, 20261203 + 1, dev)
    C, _, _ = context(fsg, "mixed", grid, st, co, 7, vmicro=meta["vmicro"], molbrd=meta["molbrd"])
    n = int(dt["wl"].numel())
    win = torch.zeros((3, n), dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    C.central_dev(H.device_view(fsg, dt), win[0].data_ptr(), win[1].data_ptr(), win[2].data_ptr())
    C.close()
    yield dict(dt=dt, win=win, st=st, meta=meta, grid=grid, wave=wave, co=co, n=n)
    del dt, win
    torch.cuda.empty_cache()


def host_lines(dt, idx):
    return {k: v[idx].cpu().numpy() for k, v in dt.items()}


def c1_slice_oracle(oracle_mod, full, center):
    import torch
    wave, win, dt = full["wave"], full["win"], full["dt"]
    i0 = int(np.searchsorted(wave, center)) + 1
    i1 = int(np.searchsorted(wave, center + C1_SLICE_A, side="right"))
    keep = (win[0] & 1) == 0
    sel = keep & (win[1] <= i1) & (win[2] >= i0)
    sidx = torch.nonzero(sel).squeeze(1)
    # a random sample of the lines whose windows miss the slice (rejected lines included)
    g = torch.Generator(device=win.device)
    g.manual_seed(int(center))
    cand = torch.randint(0, full["n"], (C1_SAMPLE,), generator=g, device=win.device)
    oidx = torch.unique(cand[~sel[cand]])
    S = oracle_mod.State(full["grid"], full["st"], contopac=full["co"], vmicro=full["meta"]["vmicro"],
                         molbrd=full["meta"]["molbrd"])
    a = host_lines(dt, sidx)
    r = oracle_mod.lineop_calc(S, oracle_mod.Lines(**a, kind=2), list_type=2, wrange=(i0, i1))
    o = oracle_mod.lineop_calc(S, oracle_mod.Lines(**host_lines(dt, oidx), kind=2), list_type=2, wrange=(1, 0))
    x, w, _ = oracle_mod.mu_quadrature(1, 7)
    ospl, ospc = oracle_mod.radtran(S, x, r["lineopac"])
    osfl, osfc = oracle_mod.disk_integ(w, ospl, ospc)
    ospl, ospc, osfl, osfc = (q[i0 - 1:i1].copy() for q in (ospl, ospc, osfl, osfc))
    gw = win[:, sidx].cpu().numpy()
    ow = win[:, oidx].cpu().numpy()
    lo = r.pop("lineopac")[i0 - 1:i1].copy()          # keep the slice only: the whole grid is 274 MB
    o.pop("lineopac")
    return dict(i0=i0, i1=i1, nsel=len(a["wl"]), r=r, o=o, gw=gw, ow=ow, rows=slice(i0 - 1, i1),
                lineopac=lo, spl=ospl, spc=ospc, sfl=osfl, sfc=osfc)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("center", C1_SLICES)
def test_c1_slice_of_full_synthesis(fsg, oracle_mod, c1_full, center, prec):
    import torch
    full = c1_full
    ref = once(("c1", center), lambda: c1_slice_oracle(oracle_mod, full, center))
    r, o = ref["r"], ref["o"]
    # windows: every selected line retained by the oracle with the same window; the sampled others
    # rejected or with windows that miss the slice, identical to the GPU's
    okeep = (o["flags"] & 1) == 0
    gkeep = (ref["ow"][0] & 1) == 0
    win_ok = dict(
        selected_rejected_by_oracle=int(np.sum(r["flags"] & 1)),
        selected_windows_differing=int(np.sum(r["ileft"] != ref["gw"][1]) + np.sum(r["iright"] != ref["gw"][2])),
        sample_retained_differing=int(np.sum(okeep != gkeep)),
        sample_windows_differing=int(np.sum(o["ileft"][okeep] != ref["ow"][1][okeep]) +
                                     np.sum(o["iright"][okeep] != ref["ow"][2][okeep])))
    # the GPU synthesis over the slice: windows of the whole list, accumulation over [i0, i1]
    C, x, w = context(fsg, prec, full["grid"], full["st"], full["co"], 7, vmicro=full["meta"]["vmicro"],
                      molbrd=full["meta"]["molbrd"])
    win = full["win"]
    torch.cuda.synchronize()
    C.lineop_reset()
    C.accumulate_dev(H.device_view(fsg, full["dt"]), win[0].data_ptr(), win[1].data_ptr(), win[2].data_ptr(),
                     ref["i0"], ref["i1"])
    lo = C.lineop_get()
    spl, spc, sfl, sfc = C.radtran()
    C.close()
    rows = ref["rows"]
    co = full["co"][rows]
    e = dict(win_ok, lines_reaching_slice=ref["nsel"], sampled_other_lines=len(o["flags"]),
             lineopac=np.max(np.abs(lo[rows] - ref["lineopac"]) / (ref["lineopac"] + co)),
             intensity=np.max(np.abs(spl[rows] / ref["spl"] - 1)),
             cont_intensity=np.max(np.abs(spc[rows] / ref["spc"] - 1)),
             flux=np.max(np.abs(sfl[rows] / ref["sfl"] - 1)),
             line_evals_oracle=r["stats"]["line_evals"] + r["stats"]["wide_evals"],
             lineopac_over_cont_max=np.max(ref["lineopac"] / co),
             lineopac_over_cont_median=np.median(ref["lineopac"] / co),
             line_depth_max=np.max(1.0 - ref["sfl"] / ref["sfc"]),
             line_depth_median=np.median(1.0 - ref["sfl"] / ref["sfc"]))
    record("c1_slice_%d" % int(center), prec, **e)
    assert not any(win_ok.values()), win_ok
    b = BARS[prec]
    assert e["lineopac"] < b["lineopac"], e
    assert e["intensity"] < b["intensity"] and e["flux"] < b["flux"], e
    assert e["cont_intensity"] < 1e-9, e
