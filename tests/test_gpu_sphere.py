"""GPU solvers for spherical models (LocPrfSph / DeloScalar, StokesPrfSph, LinStrCalc's spherical
branch, SphereInit on the host) against the oracle and the reference's own spherical runs
(tests/golden/pin_sphere.npz: solar-type and magnetic atmospheres written as spherical models whose
outermost Gauss-Legendre angle is a grazing ray).

Tolerances, per output:
  * FP64 solvers on the same opacities as the oracle: intensities 1e-9 relative on rays that reach the
    bottom layer; the grazing ray (an optically thin chord, I ~ 1e-3 of the disk-centre continuum Ic)
    1e-10 of Ic; Q, U, V 1e-9 of Ic;
  * against the reference's spectra: 1e-8 relative (grazing ray: 1e-9 of Ic), as the oracle's pins;
  * line strengths (REAL(4)) 1e-7; mixed-precision opacity: flux and Stokes I within 1e-5 relative,
    Q, U, V within 1e-5 of Ic.
"""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def sph_ctx(fsg, d, prec, nmu):
    grid, st, meta, co = H.pin_setup(d)
    C = fsg.Context(precision=prec, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    C.set_grid(grid["wmode"], grid["wstart"], grid["wend"], grid["dstep"])
    C.set_atmosphere(st)
    C.set_geometry(float(d["radius"]), d["height"])
    C.set_contopac(co)
    x, w, _ = fsg.mu_quadrature(1, nmu)
    C.set_mu(x, w)
    return C, grid, st, co, x, w


def oracle_sph(oracle_mod, d, grid, st, co, x):
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    geo = S.set_sphere(float(d["radius"]), d["height"], x)
    return S, geo["graz"] == 0


def check_intensity(sp, ref, normal, ic0, rel, graz_abs):
    assert np.max(np.abs(sp[:, normal] / ref[:, normal] - 1)) < rel
    assert np.max(np.abs(sp[:, ~normal] - ref[:, ~normal]) / ic0) < graz_abs


def test_sphere_radtran_on_reference_opacity(fsg, oracle_mod):
    """RadTranCalc's spherical branch given the reference's own LineOpac / ContOpac."""
    d = H.sphere_pin("s")
    C, grid, st, co, x, w = sph_ctx(fsg, d, fsg.PREC_FP64, len(d["xmu"]))
    assert np.array_equal(x, d["xmu"])
    i0, i1 = int(d["i0"]), int(d["i1"])
    lo = np.zeros((len(co), len(st["T"])))
    lo[i0:i1 + 1] = d["lineopac"]
    C.lineop_set(lo)
    spl, spc, sfl, sfc = C.radtran()
    S, normal = oracle_sph(oracle_mod, d, grid, st, co, x)
    ospl, ospc = oracle_mod.radtran(S, x, lo)
    ic0 = ospc[:, :1]
    check_intensity(spl, ospl, normal, ic0, 1e-9, 1e-10)
    check_intensity(spc, ospc, normal, ic0, 1e-9, 1e-10)
    r = slice(i0, i1 + 1)
    check_intensity(spl[r], d["spl"], normal, d["spc"][:, :1], 1e-8, 1e-9)
    check_intensity(spc[r], d["spc"], normal, d["spc"][:, :1], 1e-8, 1e-9)
    assert np.max(np.abs(sfl[r] / d["sfl"] - 1)) < 1e-8 and np.max(np.abs(sfc[r] / d["sfc"] - 1)) < 1e-8
    # the geometry matters: a plane-parallel solve of the same opacities differs
    C.set_geometry(-1.0)
    ppl = C.radtran()[0]
    assert np.max(np.abs(ppl[r, -1] / d["spl"][:, -1] - 1)) > 1e-2


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_sphere_synthesis_against_reference(fsg, prec):
    """LineopCalc + spherical RadTranCalc + LinStrCalc of the seeded list against the reference run."""
    d = H.sphere_pin("s")
    C, grid, st, co, x, w = sph_ctx(fsg, d, fsg.PREC_MIXED if prec == "mixed" else fsg.PREC_FP64, len(d["xmu"]))
    g = C.lineop_calc(fsg.LineList.from_arrays(H.pin_lines(d)), want_linstr=True)
    i0, i1 = int(d["i0"]), int(d["i1"])
    r = slice(i0, i1 + 1)
    keep = (g["flags"] & 1) == 0
    assert keep.sum() == len(d["linst_wave"])
    assert np.max(np.abs(g["linstr"][keep] - d["linst"])) < 1e-7
    spl, spc, sfl, sfc = C.radtran()
    tol = 1e-8 if prec == "fp64" else 1e-5
    assert np.max(np.abs(sfl[r] / d["sfl"] - 1)) < tol
    assert np.max(np.abs(sfc[r] / d["sfc"] - 1)) < 1e-8
    normal = np.ones(len(x), bool); normal[-1] = False
    check_intensity(spl[r], d["spl"], normal, d["spc"][:, :1], tol, tol / 10)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_sphere_stokes_against_reference(fsg, oracle_mod, prec):
    """StokesPrfSph with the stellar-frame field (BFRAME 0) against the reference's IQUV and the oracle."""
    d = H.sphere_pin("m")
    C, grid, st, co, x, w = sph_ctx(fsg, d, fsg.PREC_MIXED if prec == "mixed" else fsg.PREC_FP64, len(d["xmu"]))
    lines, z = H.pin_lines(d), (d["z_npi"], d["z_nsi"], d["z_spl_pi"], d["z_str_pi"], d["z_spl_si"], d["z_str_si"])
    bframe, bfield = int(d["bframe"]), d["bfield"]
    C.mag_lineop_calc(fsg.LineList.from_arrays(lines, zeeman=z), bframe, bfield)
    spz, spc, sfl, sfc = C.mag_radtran(bframe, bfield)
    i0, i1 = int(d["i0"]), int(d["i1"])
    r = slice(i0, i1 + 1)
    ref, ic = d["spz"], d["spc"]
    ic0 = ic[:, :1]
    tol = 1e-8 if prec == "fp64" else 1e-5
    for q in range(4):
        assert np.max(np.abs(spz[r, q] - ref[:, q]) / ic0) < tol
    assert np.max(np.abs(spc[r] / ic - 1)) < 1e-8
    assert np.max(np.abs(sfl[r] / d["sfl"] - 1)) < tol
    assert np.max(np.abs(sfc[r] / d["sfc"] - 1)) < 1e-8
    if prec == "fp64":
        S, normal = oracle_sph(oracle_mod, d, grid, st, co, x)
        o = oracle_mod.mag_lineop_calc(S, oracle_mod.Lines(**lines, kind=2, zeeman=z), bframe, bfield)
        ospz, ospc = oracle_mod.mag_radtran(S, x, bframe, bfield, np.zeros((S.nwl, S.ntau)), o["maglineopac"])
        oc0 = ospc[:, :1]
        check_intensity(spz[:, 0], ospz[:, 0], normal, oc0, 1e-9, 1e-10)
        for q in (1, 2, 3):
            assert np.max(np.abs(spz[:, q] - ospz[:, q]) / oc0) < 1e-9


@pytest.mark.parametrize("bframe", [1, 2])
def test_sphere_stokes_observer_frames_vs_oracle(fsg, oracle_mod, bframe):
    """Frames 1 and 2 (projection fixed along each ray) on the spherical magnetic model, FP64."""
    d = H.sphere_pin("m")
    nmu = len(d["xmu"])
    C, grid, st, co, x, w = sph_ctx(fsg, d, fsg.PREC_FP64, nmu)
    bfield = np.array([2000.0, 60.0, 30.0]) if bframe == 1 else \
        np.concatenate([[2500.0], np.ravel([(20.0 + 15.0 * k, 10.0 * k - 40.0) for k in range(nmu)])])
    lines, z = H.pin_lines(d), (d["z_npi"], d["z_nsi"], d["z_spl_pi"], d["z_str_pi"], d["z_spl_si"], d["z_str_si"])
    C.mag_lineop_calc(fsg.LineList.from_arrays(lines, zeeman=z), bframe, bfield)
    spz, spc, sfl, sfc = C.mag_radtran(bframe, bfield)
    S, normal = oracle_sph(oracle_mod, d, grid, st, co, x)
    o = oracle_mod.mag_lineop_calc(S, oracle_mod.Lines(**lines, kind=2, zeeman=z), bframe, bfield)
    ospz, ospc = oracle_mod.mag_radtran(S, x, bframe, bfield, np.zeros((S.nwl, S.ntau)), o["maglineopac"])
    oc0 = ospc[:, :1]
    check_intensity(spz[:, 0], ospz[:, 0], normal, oc0, 1e-9, 1e-10)
    for q in (1, 2, 3):
        assert np.max(np.abs(spz[:, q] - ospz[:, q]) / oc0) < 1e-9
    osfl, _ = oracle_mod.disk_integ(w, ospz[:, 0], ospc)
    assert np.max(np.abs(sfl / osfl - 1)) < 1e-9


def test_sphere_geometry_errors_and_reset(fsg, oracle_mod):
    """fsg_set_geometry checks the model as ReadModel does; SphereInit's errors surface at the solve;
    a new atmosphere is plane-parallel again."""
    d = H.sphere_pin("s")
    C, grid, st, co, x, w = sph_ctx(fsg, d, fsg.PREC_FP64, 7)
    h = d["height"]
    with pytest.raises(fsg.FsgError):
        C.set_geometry(float(d["radius"]), h[::-1].copy())           # heights must decrease inward
    with pytest.raises(fsg.FsgError):
        C.set_geometry(1e5, h)                                        # implausible radius
    with pytest.raises(fsg.FsgError):
        C.set_geometry(float(d["radius"]), None)
    C.set_geometry(2.0e9, h)                                          # outermost ray turns in the top layer
    C.set_mu(np.array([0.5, 0.01]), np.array([0.5, 0.5]))
    with pytest.raises(fsg.FsgError):
        C.radtran()
    C.set_mu(x, w)
    C.set_geometry(float(d["radius"]), h)
    sph = C.radtran()[2]
    C.set_atmosphere(st)                                              # back to plane-parallel
    C.set_contopac(co)
    pp = C.radtran()[2]
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0)
    ospl, ospc = oracle_mod.radtran(S, x, np.zeros((S.nwl, S.ntau)))
    osfl, _ = oracle_mod.disk_integ(w, ospl, ospc)
    assert np.max(np.abs(pp / osfl - 1)) < 1e-9
    assert np.max(np.abs(sph / pp - 1)) > 1e-4
