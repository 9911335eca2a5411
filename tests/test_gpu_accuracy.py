"""Maximum error of every output of the GPU path against the FP64 oracle, per configuration type and
precision, on seeded cases with the benchmark configurations' distributions (atomic lines on a solar
atmosphere, molecular lines on the cool dwarf at R = 3e5, Zeeman lines in a 2 kG field, a spherical
model).  Each case asserts the bars below; with FSG_ACCURACY_JSON set, the measured maxima are written
to that file as the error table of the library.

Bars: window indices identical; FP64 path: LineOpac 1e-11 of the total opacity, intensities and flux
1e-9 relative; mixed path: LineOpac 2e-6 of the total opacity, intensities and flux 1e-5 relative;
the six Zeeman profiles on the scale of the depth's peak absorption profile (the dispersion profiles
change sign and outlast the absorption ones in the far wings); Stokes Q, U, V on the scale of the
continuum intensity.
"""
import json
import os

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

RESULTS = {}
BARS = {"fp64": dict(lineopac=1e-11, intensity=1e-9, flux=1e-9),
        "mixed": dict(lineopac=2e-6, intensity=1e-5, flux=1e-5)}


def record(case, prec, **errs):
    RESULTS.setdefault(case, {})[prec] = {k: float(v) for k, v in errs.items()}
    path = os.environ.get("FSG_ACCURACY_JSON")
    if path:
        with open(path, "w") as f:
            json.dump(RESULTS, f, indent=1, sort_keys=True)


def scalar_case(name):
    import fastspec_b200 as F
    from fastspec_b200 import workloads as W
    if name == "atomic":
        st, meta = H.load_atm("solar")
        w0, w1 = 5000.0, 5010.0
        grid = dict(wmode=0, wstart=w0, wend=w1, dstep=0.005)
        L, kind, molbrd = W.atomic_lines(2000, w0 - 1.0, w1 + 1.0, W.SEED0 + 40), 2, 0
    else:
        st, meta = H.load_atm("cooldwarf")
        w0, w1 = 10000.0, 10010.0
        grid = dict(wmode=1, wstart=w0, wend=w1, dstep=2.99792458e5 / 3e5)
        L, kind, molbrd = W.molecular_lines(20000, w0 - 1.0, w1 + 1.0, W.SEED0 + 41), 2, 1
    wave = F.make_grid(grid["wmode"], w0, w1, grid["dstep"]) + w0
    return grid, st, H.contopac_on(meta, wave), L, kind, molbrd


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["atomic", "molecular"])
def test_scalar_errors(fsg, oracle_mod, name, prec):
    grid, st, co, L, kind, molbrd = scalar_case(name)
    C = fsg.Context(precision=fsg.PREC_FP64 if prec == "fp64" else fsg.PREC_MIXED, vmicro=1.0, molbrd=molbrd)
    C.set_grid(grid["wmode"], grid["wstart"], grid["wend"], grid["dstep"])
    C.set_atmosphere(st)
    C.set_contopac(co)
    x, w, _ = fsg.mu_quadrature(1, 7)
    C.set_mu(x, w)
    a = L.arrays()
    g = C.lineop_calc(fsg.LineList.from_arrays(a, kind=kind), want_linstr=True)
    spl, spc, sfl, sfc = C.radtran()
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0, molbrd=molbrd)
    OL = oracle_mod.Lines(wl=a["wl"], elo=a["elo"], gf=a["gf"], grad=a["grad"], gqst=a["gqst"], gvdw=a["gvdw"],
                          spc=a["spc"], ismol=a["ismol"], kind=kind)
    r = oracle_mod.lineop_calc(S, OL, list_type=kind, nmu=7, xmu=x, wmu=w, want_linstr=True)
    ospl, ospc = oracle_mod.radtran(S, x, r["lineopac"])
    osfl, osfc = oracle_mod.disk_integ(w, ospl, ospc)
    win = int(np.sum(g["ileft"] != r["ileft"]) + np.sum(g["iright"] != r["iright"]))
    keep = (r["flags"] & 1) == 0
    e = dict(windows_differing=win,
             lineopac=np.max(np.abs(g["lineopac"] - r["lineopac"]) / (r["lineopac"] + co)),
             intensity=np.max(np.abs(spl / ospl - 1)), cont_intensity=np.max(np.abs(spc / ospc - 1)),
             flux=np.max(np.abs(sfl / osfl - 1)), cont_flux=np.max(np.abs(sfc / osfc - 1)),
             line_strength=np.max(np.abs(g["linstr"][keep] - r["linstr"][keep])),
             retained_lines=int(keep.sum()), wavelengths=len(co))
    record(name, prec, **e)
    b = BARS[prec]
    assert win == 0
    assert e["lineopac"] < b["lineopac"] and e["intensity"] < b["intensity"] and e["flux"] < b["flux"]
    assert e["cont_intensity"] < 1e-9 and e["line_strength"] < 1e-6


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_stokes_errors(fsg, oracle_mod, prec):
    import fastspec_b200 as F
    from fastspec_b200 import workloads as W
    import sys
    sys.path.insert(0, H.GOLD)
    from make_atmospheres import mirrored_components
    st, meta = H.load_atm("magnetic")
    w0, w1 = 6000.0, 6006.0
    grid = dict(wmode=0, wstart=w0, wend=w1, dstep=0.002)
    co = H.contopac_on(meta, F.make_grid(0, w0, w1, 0.002) + w0)
    L = W.zeeman_lines(300, w0 + 0.3, w1 - 0.3, W.SEED0 + 42)
    jlo, jup, glo, gup = L.zeeman
    pats = []
    for i in range(L.n):
        p = oracle_mod.zeeman_pattern(jlo[i], jup[i], glo[i], gup[i])
        pats.append(p if len(p[0]) and len(p[2]) else oracle_mod.zeeman_pattern(1.0, 0.0, 1.0, 1.0))
    z = mirrored_components(pats)
    a = L.arrays()
    bframe, bfield = 1, np.array([2000.0, 60.0, 30.0])
    C = fsg.Context(precision=fsg.PREC_FP64 if prec == "fp64" else fsg.PREC_MIXED, vmicro=1.0)
    C.set_grid(0, w0, w1, 0.002)
    C.set_atmosphere(st)
    C.set_contopac(co)
    x, w, _ = fsg.mu_quadrature(1, 9)
    C.set_mu(x, w)
    g = C.mag_lineop_calc(fsg.LineList.from_arrays(a, zeeman=z), bframe, bfield)
    spz, spc, sfl, sfc = C.mag_radtran(bframe, bfield)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0)
    r = oracle_mod.mag_lineop_calc(S, oracle_mod.Lines(**{k: a[k] for k in ("wl", "elo", "gf", "grad", "gqst",
                                                                             "gvdw", "spc", "ismol")},
                                                      kind=2, zeeman=z), bframe, bfield)
    ospz, ospc = oracle_mod.mag_radtran(S, x, bframe, bfield, np.zeros((S.nwl, S.ntau)), r["maglineopac"])
    osfl, _ = oracle_mod.disk_integ(w, ospz[:, 0], ospc)
    m, om = g["maglineopac"], r["maglineopac"]
    scale = np.maximum(om[..., :3].max(axis=(0, 2)), 1e-300)[None, :, None]   # the depth's peak absorption
    e = dict(windows_differing=int(np.sum(g["ileft"] != r["ileft"]) + np.sum(g["iright"] != r["iright"])),
             maglineopac=np.max(np.abs(m - om) / scale), stokes_i=np.max(np.abs(spz[:, 0] / ospz[:, 0] - 1)),
             stokes_quv=max(np.max(np.abs(spz[:, q] - ospz[:, q]) / ospc) for q in (1, 2, 3)),
             cont_intensity=np.max(np.abs(spc / ospc - 1)), flux=np.max(np.abs(sfl / osfl - 1)),
             wavelengths=len(co))
    record("stokes", prec, **e)
    b = BARS[prec]
    assert e["windows_differing"] == 0
    assert e["maglineopac"] < b["lineopac"] and e["stokes_i"] < b["intensity"] and e["flux"] < b["flux"]
    assert e["stokes_quv"] < b["intensity"]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_spherical_errors(fsg, oracle_mod, prec):
    d = H.sphere_pin("s")
    grid, st, meta, co = H.pin_setup(d)
    C = fsg.Context(precision=fsg.PREC_FP64 if prec == "fp64" else fsg.PREC_MIXED, vmicro=1.0)
    C.set_grid(grid["wmode"], grid["wstart"], grid["wend"], grid["dstep"])
    C.set_atmosphere(st)
    C.set_geometry(float(d["radius"]), d["height"])
    C.set_contopac(co)
    x, w, _ = fsg.mu_quadrature(1, 7)
    C.set_mu(x, w)
    C.lineop_calc(fsg.LineList.from_arrays(H.pin_lines(d)))
    spl, spc, sfl, sfc = C.radtran()
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0)
    geo = S.set_sphere(float(d["radius"]), d["height"], x)
    r = oracle_mod.lineop_calc(S, oracle_mod.Lines(**H.pin_lines(d), kind=2), list_type=2)
    ospl, ospc = oracle_mod.radtran(S, x, r["lineopac"])
    osfl, _ = oracle_mod.disk_integ(w, ospl, ospc)
    normal = geo["graz"] == 0
    e = dict(intensity=np.max(np.abs(spl[:, normal] / ospl[:, normal] - 1)),
             grazing_intensity_over_ic=np.max(np.abs(spl[:, ~normal] - ospl[:, ~normal]) / ospc[:, :1]),
             flux=np.max(np.abs(sfl / osfl - 1)), wavelengths=len(co))
    record("spherical", prec, **e)
    b = BARS[prec]
    assert e["intensity"] < b["intensity"] and e["flux"] < b["flux"]
