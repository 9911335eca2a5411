"""GPU parity of the magnetic path (MagLineopCalc + MagRadTranCalc) against the oracle and the
reference.  Both run in FP64 in the reference's operation order, so:
  * window indices and flags: identical;
  * the six Zeeman profiles MagLineOpac: 1e-11 of the local absorption scale (dispersion
    profiles change sign, so the scale is the max of the absorption profiles at that depth);
  * Stokes I and Ic: 1e-9 relative; Q, U, V: 1e-9 of Ic (libm ulps amplified by the DELO
    coefficients just above their Taylor branch, solver.f90:357-370);
  * against the reference's own Stokes spectra: 1e-8.
"""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def mag_ctx(fsg, grid, st, co, nmu=9, vmicro=1.0, molbrd=0, prec=None):
    C = fsg.Context(precision=fsg.PREC_FP64 if prec is None else prec, vmicro=vmicro, molbrd=molbrd)
    C.set_grid(grid["wmode"], grid["wstart"], grid["wend"], grid["dstep"])
    C.set_atmosphere(st)
    C.set_contopac(co)
    x, w, _ = fsg.mu_quadrature(1, nmu)
    C.set_mu(x, w)
    return C, x, w


def zeeman_case(n=60, w0=6040.0, span=3.0, seed=31, nmu=9):
    st, meta = H.load_atm("magnetic")
    from fastspec_b200 import workloads as W
    import fastspec_b200 as F
    import oracle
    grid = dict(wmode=0, wstart=w0, wend=w0 + span, dstep=0.002)
    wave = F.make_grid(0, w0, w0 + span, 0.002) + w0
    co = H.contopac_on(meta, wave)
    L = W.zeeman_lines(n, w0 + 0.2, w0 + span - 0.2, seed)
    jlo, jup, glo, gup = L.zeeman
    pats = []
    for i in range(L.n):
        p = oracle.zeeman_pattern(jlo[i], jup[i], glo[i], gup[i])
        if len(p[0]) == 0 or len(p[2]) == 0:
            p = oracle.zeeman_pattern(1.0, 0.0, 1.0, 1.0)
        pats.append(p)
    import sys, os
    sys.path.insert(0, H.GOLD)
    from make_atmospheres import mirrored_components
    return grid, st, co, L.arrays(), mirrored_components(pats)


def run_both(fsg, oracle_mod, grid, st, co, lines, z, bframe, bfield, nmu=9):
    C, x, w = mag_ctx(fsg, grid, st, co, nmu=nmu)
    g = C.mag_lineop_calc(fsg.LineList.from_arrays(lines, zeeman=z), bframe, bfield)
    spz, spc, sfl, sfc = C.mag_radtran(bframe, bfield)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0)
    r = oracle_mod.mag_lineop_calc(S, oracle_mod.Lines(**lines, kind=2, zeeman=z), bframe, np.asarray(bfield, float))
    ospz, ospc = oracle_mod.mag_radtran(S, x, bframe, np.asarray(bfield, float), np.zeros((S.nwl, S.ntau)),
                                        r["maglineopac"])
    return g, r, (spz, spc, sfl, sfc), (ospz, ospc), w


@pytest.mark.parametrize("bframe,bfield", [(1, [2000.0, 60.0, 30.0]), (0, [1500.0, 800.0, -400.0])])
def test_mag_lineop_and_stokes_vs_oracle(fsg, oracle_mod, bframe, bfield):
    grid, st, co, lines, z = zeeman_case()
    g, r, G, O, w = run_both(fsg, oracle_mod, grid, st, co, lines, z, bframe, bfield)
    assert np.array_equal(g["flags"], r["flags"])
    assert np.array_equal(g["ileft"], r["ileft"]) and np.array_equal(g["iright"], r["iright"])
    m, om = g["maglineopac"], r["maglineopac"]
    scale = np.maximum(om[..., :3].max(axis=(0, 2)), 1e-300)[None, :, None]
    assert np.max(np.abs(m - om) / scale) < 1e-11
    spz, spc, sfl, sfc = G
    ospz, ospc = O
    assert np.max(np.abs(spz[:, 0] / ospz[:, 0] - 1)) < 1e-9
    assert np.max(np.abs(spc / ospc - 1)) < 1e-9
    for q in (1, 2, 3):
        assert np.max(np.abs(spz[:, q] - ospz[:, q]) / ospc) < 1e-9
    osfl, osfc = oracle_mod.disk_integ(w, ospz[:, 0], ospc)
    assert np.max(np.abs(sfl / osfl - 1)) < 1e-9
    assert np.max(np.abs(sfc / osfc - 1)) < 1e-9


def test_mag_frame2_per_angle_geometry(fsg, oracle_mod):
    grid, st, co, lines, z = zeeman_case(n=30, seed=33, nmu=5)
    bfield = [2500.0] + sum([[20.0 * k, 15.0 * k] for k in range(1, 6)], [])
    g, r, G, O, w = run_both(fsg, oracle_mod, grid, st, co, lines, z, 2, bfield, nmu=5)
    spz, spc, _, _ = G
    ospz, ospc = O
    for q in range(4):
        assert np.max(np.abs(spz[:, q] - ospz[:, q]) / ospc) < 1e-9


def test_mag_against_reference_pin(fsg):
    d = H.load_pin("pin_magnetic")
    grid, st, co, lines, z = H.mag_pin_setup(d)
    C, x, w = mag_ctx(fsg, grid, st, co, nmu=len(d["xmu"]), vmicro=float(d["vmicro"]))
    assert np.array_equal(x, d["xmu"])
    bframe, bfield = int(d["bframe"]), d["bfield"]
    C.mag_lineop_calc(fsg.LineList.from_arrays(lines, zeeman=z), bframe, bfield, want=False)
    spz, spc, sfl, sfc = C.mag_radtran(bframe, bfield)
    i0, i1 = int(d["i0"]), int(d["i1"])
    ref, ic = d["spz"], d["spc"]
    assert np.max(np.abs(spz[i0:i1 + 1, 0] / ref[:, 0] - 1)) < 1e-8
    assert np.max(np.abs(spc[i0:i1 + 1] / ic - 1)) < 1e-8
    for q in (1, 2, 3):
        assert np.max(np.abs(spz[i0:i1 + 1, q] - ref[:, q]) / ic) < 1e-8
    assert np.max(np.abs(sfl[i0:i1 + 1] / d["sfl"] - 1)) < 1e-8
    assert np.max(np.abs(sfc[i0:i1 + 1] / d["sfc"] - 1)) < 1e-8


@pytest.mark.parametrize("frame", [0, 2])
def test_mag_frames_against_reference_pin(fsg, frame):
    """The stellar-frame (BFRAME 0) and per-angle (BFRAME 2) field geometries on the GPU FP64 path against
    the reference's Stokes IQUV (tests/golden/pin_magnetic_frames.npz); 1e-8 of Ic as for BFRAME 1."""
    d = H.load_pin("pin_magnetic")
    f = H.load_pin("pin_magnetic_frames")
    grid, st, co, lines, z = H.mag_pin_setup(d)
    C, x, w = mag_ctx(fsg, grid, st, co, nmu=len(f["xmu"]), vmicro=float(d["vmicro"]))
    assert np.array_equal(x, f["xmu"])
    bfield = f["f%d_bfield" % frame]
    C.mag_lineop_calc(fsg.LineList.from_arrays(lines, zeeman=z), frame, bfield, want=False)
    spz, spc, sfl, sfc = C.mag_radtran(frame, bfield)
    i0, i1 = int(f["i0"]), int(f["i1"])
    ref, ic = f["f%d_spz" % frame], f["f%d_spc" % frame]
    assert np.max(np.abs(spz[i0:i1 + 1, 0] / ref[:, 0] - 1)) < 1e-8
    for q in (1, 2, 3):
        assert np.max(np.abs(spz[i0:i1 + 1, q] - ref[:, q]) / ic) < 1e-8
    assert np.max(np.abs(sfl[i0:i1 + 1] / f["f%d_sfl" % frame] - 1)) < 1e-8


def test_mag_linstr_against_reference_pin(fsg):
    """Line strengths of the magnetic driver on the GPU against the reference's fs_linst.bin for the
    pin_magnetic deck (tests/golden/pin_magnetic_linst.npz)."""
    d = H.load_pin("pin_magnetic")
    ref = H.load_pin("pin_magnetic_linst")
    grid, st, co, lines, z = H.mag_pin_setup(d)
    C, x, w = mag_ctx(fsg, grid, st, co, nmu=len(d["xmu"]), vmicro=float(d["vmicro"]))
    g = C.mag_lineop_calc(fsg.LineList.from_arrays(lines, zeeman=z), int(d["bframe"]), d["bfield"], want=False,
                          want_linstr=True)
    keep = (g["flags"] & 1) == 0
    assert keep.sum() == len(ref["wave"])
    assert np.max(np.abs(g["linstr"][keep] - ref["strength"])) < 1e-7


def test_mag_rejects_bad_field(fsg):
    grid, st, co, lines, z = zeeman_case(n=5)
    C, x, w = mag_ctx(fsg, grid, st, co)
    with pytest.raises(fsg.FsgError):
        C.mag_lineop_calc(fsg.LineList.from_arrays(lines, zeeman=z), 2, [1000.0, 1.0, 2.0])
    with pytest.raises(fsg.FsgError):
        C.mag_lineop_calc(fsg.LineList.from_arrays(lines), 1, [1000.0, 1.0, 2.0])


def test_mag_linstr_vs_oracle(fsg, oracle_mod):
    """Central depths from the magnetic driver: the non-magnetic LinStrCalc of each retained line."""
    grid, st, co, lines, z = zeeman_case(n=40, seed=35)
    C, x, w = mag_ctx(fsg, grid, st, co)
    g = C.mag_lineop_calc(fsg.LineList.from_arrays(lines, zeeman=z), 1, [2000.0, 60.0, 30.0], want=False,
                          want_linstr=True)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0)
    r = oracle_mod.mag_lineop_calc(S, oracle_mod.Lines(**lines, kind=2, zeeman=z), 1, np.array([2000.0, 60.0, 30.0]),
                                   nmu=len(x), xmu=x, wmu=w, want_linstr=True)
    assert np.array_equal(g["flags"] & 1, r["flags"] & 1)
    assert np.max(np.abs(g["linstr"] - r["linstr"])) < 1e-7
    assert np.any(g["linstr"] > 0)


@pytest.mark.parametrize("bframe,bfield", [(1, [2000.0, 60.0, 30.0]), (0, [1500.0, 800.0, -400.0])])
def test_mixed_mag_vs_oracle(fsg, oracle_mod, bframe, bfield):
    """Mixed precision (FP32 Faraday-Voigt on tiles, FP64 sums per line): the six planes within 2e-6
    of the local absorption scale, Stokes I and Q/U/V within 1e-5 (of Ic)."""
    grid, st, co, lines, z = zeeman_case()
    C, x, w = mag_ctx(fsg, grid, st, co, prec=fsg.PREC_MIXED)
    g = C.mag_lineop_calc(fsg.LineList.from_arrays(lines, zeeman=z), bframe, bfield)
    spz, spc, sfl, sfc = C.mag_radtran(bframe, bfield)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0)
    r = oracle_mod.mag_lineop_calc(S, oracle_mod.Lines(**lines, kind=2, zeeman=z), bframe, np.asarray(bfield, float))
    ospz, ospc = oracle_mod.mag_radtran(S, x, bframe, np.asarray(bfield, float), np.zeros((S.nwl, S.ntau)),
                                        r["maglineopac"])
    assert np.array_equal(g["flags"] & 1, r["flags"] & 1)
    assert np.array_equal(g["ileft"], r["ileft"]) and np.array_equal(g["iright"], r["iright"])
    m, om = g["maglineopac"], r["maglineopac"]
    scale = np.maximum(om[..., :3].max(axis=(0, 2)), 1e-300)[None, :, None]
    assert np.max(np.abs(m - om) / scale) < 2e-6
    assert np.max(np.abs(spz[:, 0] / ospz[:, 0] - 1)) < 1e-5
    for q in (1, 2, 3):
        assert np.max(np.abs(spz[:, q] - ospz[:, q]) / ospc) < 1e-5


def test_mixed_mag_against_reference_pin(fsg):
    d = H.load_pin("pin_magnetic")
    grid, st, co, lines, z = H.mag_pin_setup(d)
    C, x, w = mag_ctx(fsg, grid, st, co, nmu=len(d["xmu"]), vmicro=float(d["vmicro"]), prec=fsg.PREC_MIXED)
    bframe, bfield = int(d["bframe"]), d["bfield"]
    C.mag_lineop_calc(fsg.LineList.from_arrays(lines, zeeman=z), bframe, bfield, want=False)
    spz, spc, sfl, sfc = C.mag_radtran(bframe, bfield)
    i0, i1 = int(d["i0"]), int(d["i1"])
    ref, ic = d["spz"], d["spc"]
    assert np.max(np.abs(spz[i0:i1 + 1, 0] / ref[:, 0] - 1)) < 1e-5
    for q in (1, 2, 3):
        assert np.max(np.abs(spz[i0:i1 + 1, q] - ref[:, q]) / ic) < 1e-5
    assert np.max(np.abs(sfl[i0:i1 + 1] / d["sfl"] - 1)) < 1e-5


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_hot_he_zeeman_lines_against_reference_pin(fsg, prec):
    """Tabulated He I Stark lines as Zeeman lines in a Teff 15000 K atmosphere, 3 kG, BFRAME 1
    (hestark.f90 + MagLineOpacity1/2): Context.hestark_init builds the widths and shifts and matches the
    list to the table; the reference's Stokes IQUV (tests/golden/pin_hot_he_mag.npz).  FP64 1e-8 and
    mixed 1e-5 (I relative; Q, U, V relative to Ic), as for the other magnetic pins."""
    from test_hestark import hot_state
    d = H.load_pin("pin_hot_he_mag")
    grid, st, co, lines, z = H.mag_pin_setup(d)
    _, _, hii, heii = hot_state()
    C, x, w = mag_ctx(fsg, grid, st, co, nmu=len(d["xmu"]), vmicro=float(d["vmicro"]),
                      prec=fsg.PREC_FP64 if prec == "fp64" else fsg.PREC_MIXED)
    C.hestark_init(hii, heii, 0)
    bframe, bfield = int(d["bframe"]), d["bfield"]
    g = C.mag_lineop_calc(fsg.LineList.from_arrays(lines, zeeman=z), bframe, bfield, want=False)
    assert int((((g["flags"] >> 8) & 255) > 0).sum()) == 7
    spz, spc, sfl, sfc = C.mag_radtran(bframe, bfield)
    ref, ic = d["spz"], d["spc"]
    tol = 1e-8 if prec == "fp64" else 1e-5
    assert np.max(np.abs(spz[:, 0] / ref[:, 0] - 1)) < tol
    assert np.max(np.abs(spc / ic - 1)) < 1e-8
    for q in (1, 2, 3):
        assert np.max(np.abs(spz[:, q] - ref[:, q]) / ic) < tol
    assert np.max(np.abs(sfl / d["sfl"] - 1)) < tol


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_zh5_list_against_reference_pin(fsg, tmp_path, prec):
    """A Zeeman HDF5 list read by fsio.read_hdf5_lines, its splitting built from J and the Lande
    factors with the library's fsg_zeeman_pattern, through the GPU magnetic path: the reference's
    Stokes IQUV for the same file (tests/golden/pin_magnetic_zh5.npz)."""
    from test_hdf5 import zh5_pin_lines
    d, r, z = zh5_pin_lines(tmp_path, fsg.zeeman_pattern)
    grid, st, meta, co = H.pin_setup(d)
    C, x, w = mag_ctx(fsg, grid, st, co, nmu=len(d["xmu"]), prec=fsg.PREC_FP64 if prec == "fp64" else fsg.PREC_MIXED)
    a = {k: r[k] for k in ("wl", "elo", "gf", "grad", "gqst", "gvdw", "spc", "ismol")}
    C.mag_lineop_calc(fsg.LineList.from_arrays(a, kind=r["kind"], zeeman=z), int(d["bframe"]), d["bfield"])
    spz, spc, sfl, sfc = C.mag_radtran(int(d["bframe"]), d["bfield"])
    i0, i1 = int(d["i0"]), int(d["i1"])
    tol = 1e-8 if prec == "fp64" else 1e-5
    for q in range(4):
        assert np.max(np.abs(spz[i0:i1 + 1, q] - d["spz"][:, q]) / d["spc"]) < tol
    assert np.max(np.abs(sfl[i0:i1 + 1] / d["sfl"] - 1)) < tol


def _state_on_depths(name, nt_new):
    """The atmosphere state interpolated to nt_new depths (log Rhox uniform between its ends; every
    quantity log-linear in Rhox), with its continuum knots likewise: a synthetic state at the library's
    depth limit for the maximum-size tests."""
    st, meta = H.load_atm(name)
    x = np.log(st["rhox"])
    xn = np.linspace(x[0], x[-1], nt_new)
    out = {"rhox": np.exp(xn)}
    for k in ("T", "xne", "xna", "rho"):
        out[k] = np.exp(np.interp(xn, x, np.log(st[k])))
    for k in ("frac_h1", "frac_he1"):
        out[k] = np.exp(np.interp(xn, x, np.log(np.maximum(st[k].astype(np.float64), 1e-300)))).astype(np.float32)
    out["frac_h2"] = np.zeros(nt_new, np.float32)
    f = st["fractionpf"].astype(np.float64)
    out["fractionpf"] = np.stack([np.exp(np.interp(xn, x, np.log(f[:, s]))) for s in range(f.shape[1])],
                                 axis=1).astype(np.float32)
    for k in ("xamass", "potion", "ion"):
        out[k] = st[k]
    lk = np.log(meta["cont_opac"])
    meta = dict(meta)
    meta["cont_opac"] = np.exp(np.stack([np.interp(xn, x, lk[j]) for j in range(lk.shape[0])], axis=0))
    return out, meta


def test_max_sizes_stokes_vs_oracle(fsg, oracle_mod):
    """At the library's limits (128 depths, 16 angles): MagLineopCalc + the Stokes solver (frame 0) and
    the scalar RadTranCalc against the oracle, FP64."""
    import fastspec_b200 as F
    from fastspec_b200 import workloads as W
    st, meta = _state_on_depths("magnetic", 128)
    w0, span = 6040.0, 1.5
    grid = dict(wmode=0, wstart=w0, wend=w0 + span, dstep=0.002)
    co = H.contopac_on(meta, F.make_grid(0, w0, w0 + span, 0.002) + w0)
    L = W.zeeman_lines(25, w0 + 0.2, w0 + span - 0.2, W.SEED0 + 77)
    import sys, os
    sys.path.insert(0, H.GOLD)
    from make_atmospheres import mirrored_components
    jlo, jup, glo, gup = L.zeeman
    pats = []
    for i in range(L.n):
        p = oracle_mod.zeeman_pattern(jlo[i], jup[i], glo[i], gup[i])
        pats.append(p if len(p[0]) and len(p[2]) else oracle_mod.zeeman_pattern(1.0, 0.0, 1.0, 1.0))
    z = mirrored_components(pats)
    lines = L.arrays()
    bframe, bfield = 0, np.array([1200.0, -700.0, 500.0])
    C, x, w = mag_ctx(fsg, grid, st, co, nmu=16)
    g = C.mag_lineop_calc(fsg.LineList.from_arrays(lines, zeeman=z), bframe, bfield)
    spz, spc, sfl, sfc = C.mag_radtran(bframe, bfield)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0)
    r = oracle_mod.mag_lineop_calc(S, oracle_mod.Lines(**lines, kind=2, zeeman=z), bframe, bfield)
    assert np.array_equal(g["ileft"], r["ileft"]) and np.array_equal(g["iright"], r["iright"])
    ospz, ospc = oracle_mod.mag_radtran(S, x, bframe, bfield, np.zeros((S.nwl, S.ntau)), r["maglineopac"])
    assert spz.shape == (S.nwl, 4, 16)
    assert np.max(np.abs(spz[:, 0] / ospz[:, 0] - 1)) < 1e-9
    for q in (1, 2, 3):
        assert np.max(np.abs(spz[:, q] - ospz[:, q]) / ospc) < 1e-9
    # the scalar solver on the same state with a non-magnetic list
    C.lineop_calc(fsg.LineList.from_arrays(lines))
    spl, spc2, sfl2, sfc2 = C.radtran()
    r2 = oracle_mod.lineop_calc(S, oracle_mod.Lines(**lines, kind=2), list_type=2)
    ospl, ospc2 = oracle_mod.radtran(S, x, r2["lineopac"])
    assert np.max(np.abs(spl / ospl - 1)) < 1e-9 and np.max(np.abs(spc2 / ospc2 - 1)) < 1e-9
