"""The CPU oracle against the reference program's own outputs (fixtures in tests/golden and
fastspec_b200/data, generated by tests/golden/make_atmospheres.py).

Tolerances: window indices are integers and must be identical; FP64 values differ only through
libm ulps (the reference's gfortran build uses glibc's vectorised exp/log in some loops), which
the DELO coefficients amplify near their Taylor branch (solver.f90:155-169), hence 1e-8."""
import numpy as np
import pytest

import helpers as H


def test_voigt_exact_vs_faddeeva(oracle_mod):
    scipy = pytest.importorskip("scipy.special")
    for a in (1e-5, 1e-3, 0.05, 0.5, 2.0, 5.9, 7.5):
        for v in (0.0, 0.2, 1.0, 2.7, 5.0, 7.9):
            z = scipy.wofz(v + 1j * a)
            assert abs(oracle_mod.hvoigt_exact(a, v) - z.real) <= 1e-9 * abs(z.real)
            w = oracle_mod.wvoigt_exact(a, v)
            assert abs(w.imag - z.imag) <= 1e-8 * abs(z.imag) + 1e-15   # method accuracy (h = 0.5, N = 16)


def test_voigt_table_lerp_accuracy(oracle_mod):
    scipy = pytest.importorskip("scipy.special")
    rng = np.random.default_rng(5)
    a = rng.uniform(0, 7.9, 2000); v = rng.uniform(-7.9, 7.9, 2000)
    h = np.array([oracle_mod.hvoigt(x, y) for x, y in zip(a, v)])
    ref = scipy.wofz(np.abs(v) + 1j * a).real
    # the table's own interpolation error (the reference's, by design) is below 1e-4 of H(a, 0)
    assert np.max(np.abs(h - ref)) < 2e-4


@pytest.mark.parametrize("name", ["pin_solar", "pin_cooldwarf"])
def test_oracle_lineop_pins_reference(oracle_mod, name):
    d = H.load_pin(name)
    grid, st, meta, co = H.pin_setup(d)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    i0, i1 = int(d["i0"]), int(d["i1"])
    assert np.abs(S.wave[i0:i1 + 1] + S.wfirst - d["wave"]).max() < 1e-9
    L = oracle_mod.Lines(**H.pin_lines(d), kind=2)
    r = oracle_mod.lineop_calc(S, L, list_type=2)
    lo, ref = r["lineopac"][i0:i1 + 1], d["lineopac"]
    # window pin: identical nonzero pattern (LineOpac is exactly 0 outside every window)
    assert np.array_equal(lo > 0, ref > 0)
    m = ref > 0
    assert np.max(np.abs(lo[m] / ref[m] - 1)) < 1e-8
    spl, spc = oracle_mod.radtran(S, d["xmu"], r["lineopac"])
    assert np.max(np.abs(spl[i0:i1 + 1] / d["spl"] - 1)) < 1e-8
    assert np.max(np.abs(spc[i0:i1 + 1] / d["spc"] - 1)) < 1e-8
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    assert np.max(np.abs(x - d["xmu"])) == 0.0
    sfl, sfc = oracle_mod.disk_integ(w, spl[i0:i1 + 1], spc[i0:i1 + 1])
    assert np.max(np.abs(sfl / d["sfl"] - 1)) < 1e-8
    assert np.max(np.abs(sfc / d["sfc"] - 1)) < 1e-8


def test_oracle_broadening_modes_pin_reference(oracle_mod):
    """Classical Stark (zero Stark input), Unsold (zero van der Waals input) and ABO (sigma.alpha) lines
    with EPSOPAC 3e-3 and VWFUDGE 1.8 (opacity.f90:185-227, 239-293) against the reference's run
    (tests/golden/pin_solar_modes.npz), on the solar state with the EOS's own ionisation potentials."""
    d = H.load_pin("pin_solar_modes")
    grid, st, meta, co = H.pin_setup(d)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]),
                         epsopac=float(d["epsopac"]), vwfudge=float(d["vwfudge"]))
    i0, i1 = int(d["i0"]), int(d["i1"])
    lines = H.pin_lines(d)
    assert np.sum(lines["gqst"] == 0) > 20 and np.sum(lines["gvdw"] == 0) > 20 and np.sum(lines["gvdw"] > 10) > 10
    r = oracle_mod.lineop_calc(S, oracle_mod.Lines(**lines, kind=2), list_type=2)
    assert np.sum((r["flags"] >> 2) & 1) == np.sum(lines["gvdw"] > 10)
    lo, ref = r["lineopac"][i0:i1 + 1], d["lineopac"]
    assert np.array_equal(lo > 0, ref > 0)
    m = ref > 0
    assert np.max(np.abs(lo[m] / ref[m] - 1)) < 1e-8
    spl, spc = oracle_mod.radtran(S, d["xmu"], r["lineopac"])
    assert np.max(np.abs(spl[i0:i1 + 1] / d["spl"] - 1)) < 1e-8
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    sfl, sfc = oracle_mod.disk_integ(w, spl[i0:i1 + 1], spc[i0:i1 + 1])
    assert np.max(np.abs(sfl / d["sfl"] - 1)) < 1e-8


def test_oracle_molecular_options_pin_reference(oracle_mod):
    """H2BRD 1.5 (H2 molecules among the van der Waals perturbers, opacity.f90:82, with the H2 density
    recovered from the reference) and VWMOL 4e-8 (opacity.f90:229-234) on the cool-dwarf list against
    the reference's run (tests/golden/pin_cooldwarf_opts.npz)."""
    d = H.load_pin("pin_cooldwarf_opts")
    grid, st, meta, co = H.pin_setup(d)
    assert np.all(st["frac_h2"] > 0)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]),
                         h2brd=float(d["h2brd"]), vwmol=float(d["vwmol"]))
    i0, i1 = int(d["i0"]), int(d["i1"])
    r = oracle_mod.lineop_calc(S, oracle_mod.Lines(**H.pin_lines(d), kind=2), list_type=2)
    lo, ref = r["lineopac"][i0:i1 + 1], d["lineopac"]
    assert np.array_equal(lo > 0, ref > 0)
    m = ref > 0
    assert np.max(np.abs(lo[m] / ref[m] - 1)) < 1e-8
    spl, spc = oracle_mod.radtran(S, d["xmu"], r["lineopac"])
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    sfl, sfc = oracle_mod.disk_integ(w, spl[i0:i1 + 1], spc[i0:i1 + 1])
    assert np.max(np.abs(sfl / d["sfl"] - 1)) < 1e-8
    # both options change the result: without them the same list differs
    S0 = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    r0 = oracle_mod.lineop_calc(S0, oracle_mod.Lines(**H.pin_lines(d), kind=2), list_type=2)
    assert np.max(np.abs(r0["lineopac"][i0:i1 + 1][m] / ref[m] - 1)) > 1e-3


@pytest.mark.parametrize("name", ["pin_solar", "pin_cooldwarf"])
def test_oracle_linstr_pins_reference(oracle_mod, name):
    """LinStrCalc (synth.f90:1774-1822): central depths of the retained lines against the reference's
    fs_linst.bin for the same deck (REAL(4) output; intensities agree to ~1e-9)."""
    d = H.load_pin(name)
    ref = H.load_pin(name + "_linst")
    grid, st, meta, co = H.pin_setup(d)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    r = oracle_mod.lineop_calc(S, oracle_mod.Lines(**H.pin_lines(d), kind=2), list_type=2, nmu=len(x), xmu=x,
                               wmu=w, want_linstr=True)
    keep = (r["flags"] & 1) == 0
    # the same lines are retained, in list order (the reference writes Wlcent + Wfirst: ~1e-11 off)
    assert keep.sum() == len(ref["wave"])
    assert np.max(np.abs(d["line_wl"][keep] - ref["wave"])) < 1e-9
    assert np.max(np.abs(r["linstr"][keep] - ref["strength"])) < 1e-7
    assert np.all(ref["strength"] > 0)


@pytest.mark.parametrize("frame", [0, 2])
def test_oracle_magnetic_frames_pin_reference(oracle_mod, frame):
    """MagRadTranCalc's other field frames (synth.f90:1948-1980): the stellar-frame field projected at
    each disk position (BFRAME 0) and per-angle observer-frame angles (BFRAME 2), on the pin_magnetic
    list, against the reference's Stokes IQUV (tests/golden/pin_magnetic_frames.npz)."""
    d = H.load_pin("pin_magnetic")
    f = H.load_pin("pin_magnetic_frames")
    grid, st, co, lines, z = H.mag_pin_setup(d)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    bfield = f["f%d_bfield" % frame]
    r = oracle_mod.mag_lineop_calc(S, oracle_mod.Lines(**lines, kind=2, zeeman=z), frame, bfield)
    spz, spc = oracle_mod.mag_radtran(S, f["xmu"], frame, bfield, np.zeros((S.nwl, S.ntau)), r["maglineopac"])
    i0, i1 = int(f["i0"]), int(f["i1"])
    ref, ic = f["f%d_spz" % frame], f["f%d_spc" % frame]
    assert np.max(np.abs(spz[i0:i1 + 1, 0] / ref[:, 0] - 1)) < 1e-8
    for q in (1, 2, 3):
        assert np.max(np.abs(spz[i0:i1 + 1, q] - ref[:, q]) / ic) < 1e-8
        assert np.max(np.abs(ref[:, q]) / ic) > 1e-5                 # the field polarises every parameter
    x, w, _ = oracle_mod.mu_quadrature(1, len(f["xmu"]))
    sfl, _ = oracle_mod.disk_integ(w, spz[i0:i1 + 1, 0], spc[i0:i1 + 1])
    assert np.max(np.abs(sfl / f["f%d_sfl" % frame] - 1)) < 1e-8


def test_oracle_magnetic_linstr_pin_reference(oracle_mod):
    """Line strengths from the magnetic driver (MagLineopCalc, SAVE flag 1) against the reference's
    fs_linst.bin for the pin_magnetic deck (9 angles, BFRAME 1)."""
    d = H.load_pin("pin_magnetic")
    ref = H.load_pin("pin_magnetic_linst")
    grid, st, co, lines, z = H.mag_pin_setup(d)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    r = oracle_mod.mag_lineop_calc(S, oracle_mod.Lines(**lines, kind=2, zeeman=z), int(d["bframe"]), d["bfield"],
                                   nmu=len(x), xmu=x, wmu=w, want_linstr=True)
    keep = (r["flags"] & 1) == 0
    assert keep.sum() == len(ref["wave"])
    assert np.max(np.abs(d["line_wl"][keep] - ref["wave"])) < 1e-9
    assert np.max(np.abs(r["linstr"][keep] - ref["strength"])) < 1e-7


def test_oracle_blocks_equal_single_block(oracle_mod):
    """Segmented blocks (NlinesStep < Nlines) give the single-block result (synth.f90:1012-1088)."""
    d = H.load_pin("pin_solar")
    grid, st, meta, co = H.pin_setup(d)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0)
    L = oracle_mod.Lines(**H.pin_lines(d), kind=2)
    r1 = oracle_mod.lineop_calc(S, L, list_type=2)
    r2 = oracle_mod.lineop_calc(S, L, list_type=2, nlines_lim=40)
    assert r2["stats"]["nsegments"] > 1
    np.testing.assert_allclose(r2["lineopac"], r1["lineopac"], rtol=1e-13, atol=0)
    assert np.array_equal(r1["ileft"], r2["ileft"]) and np.array_equal(r1["iright"], r2["iright"])


def test_mu_quadratures(oracle_mod):
    for q in (0, 1, 2):
        for n in (1, 2, 7, 9):
            x, w, r = oracle_mod.mu_quadrature(q, n)
            assert abs(w.sum() - 1.0) < 1e-12
            assert np.all(np.diff(x) <= 0)


def test_zeeman_pattern_normal_triplet(oracle_mod):
    spi, rpi, ssi, rsi = oracle_mod.zeeman_pattern(1.0, 0.0, 1.5, 1.5)
    assert len(spi) == 1 and spi[0] == 0 and rpi[0] == 1
    assert len(ssi) == 1 and abs(abs(ssi[0]) - 1.5) < 1e-6


def test_oracle_magnetic_pins_reference(oracle_mod):
    """MagLineopCalc + MagRadTranCalc (Stokes IQUV, BFRAME 1) against the reference's spectra."""
    d = H.load_pin("pin_magnetic")
    grid, st, co, lines, z = H.mag_pin_setup(d)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    i0, i1 = int(d["i0"]), int(d["i1"])
    L = oracle_mod.Lines(**lines, kind=2, zeeman=z)
    r = oracle_mod.mag_lineop_calc(S, L, int(d["bframe"]), d["bfield"])
    lo = np.zeros((S.nwl, S.ntau))
    spz, spc = oracle_mod.mag_radtran(S, d["xmu"], int(d["bframe"]), d["bfield"], lo, r["maglineopac"])
    ref = d["spz"]
    ic = d["spc"]
    # I and Ic relative; Q, U, V relative to the continuum intensity
    assert np.max(np.abs(spz[i0:i1 + 1, 0] / ref[:, 0] - 1)) < 1e-8
    assert np.max(np.abs(spc[i0:i1 + 1] / ic - 1)) < 1e-8
    for q in (1, 2, 3):
        assert np.max(np.abs(spz[i0:i1 + 1, q] - ref[:, q]) / ic) < 1e-8
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    sfl, sfc = oracle_mod.disk_integ(w, spz[i0:i1 + 1, 0], spc[i0:i1 + 1])
    assert np.max(np.abs(sfl / d["sfl"] - 1)) < 1e-8


def convol_cases():
    d = H.load_pin("pin_convol")
    return d, sorted(set(k.rsplit("_", 1)[0] for k in d))


@pytest.mark.parametrize("case", ["solar_0", "solar_1", "solar_2", "solar_3", "cooldwarf_0", "cooldwarf_1"])
def test_oracle_disk_integ_convol_pins_reference(oracle_mod, case):
    """DiskInteg with rotation, radial-tangential macroturbulence and Gaussian broadening
    (convol.f90:67-300) of the reference's own intensities against its broadened flux."""
    d = H.load_pin("pin_convol")
    g = d[case + "_grid"]
    grid = dict(wmode=int(g[3]), wstart=g[0], wend=g[1], dstep=g[2])
    vs, vm, vg = d[case + "_convol"]
    x, w, r = oracle_mod.mu_quadrature(1, 7)
    assert np.max(np.abs(x - d[case + "_xmu"])) == 0.0
    wave = d[case + "_wave"]
    dv = oracle_mod.grid_dv(grid, wave)
    gsig = oracle_mod.gauss_sigma_pix(grid, wave, vg) if vg > 0 else 0.0
    sfl, sfc = oracle_mod.disk_integ_conv(x, w, r, d[case + "_spl"], d[case + "_spc"], dv, vs, vm, gsig)
    assert np.max(np.abs(sfl / d[case + "_sfl"] - 1)) < 1e-12
    assert np.max(np.abs(sfc / d[case + "_sfc"] - 1)) < 1e-12
