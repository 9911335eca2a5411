"""Spherical geometry of the CPU oracle (SphereInit, LocPrfSph / DeloScalar, StokesPrfSph) against the
reference program's own spherical runs (tests/golden/pin_sphere.npz, made by
tests/golden/make_atmospheres.py sphere).

The fixture models are the solar-type and magnetic atmospheres written as spherical models whose
radius makes the outermost Gauss-Legendre angle a grazing ray (6 and 2n points along it) while the
other rays reach the bottom layer.  Tolerances as for the plane-parallel pins: libm ulps amplified by
the DELO coefficients, 1e-8 relative; the grazing ray's intensity is ~1e-3 of the disk-centre
continuum (an optically thin chord), so it is compared on that scale (|dI| / Ic(mu = 1) < 1e-9)."""
import numpy as np
import pytest

import helpers as H


def _state(oracle_mod, d, contopac=True):
    grid, st, meta, co = H.pin_setup(d)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    geo = S.set_sphere(float(d["radius"]), d["height"], d["xmu"])
    return S, geo, st


def test_sphere_rays_geometry(oracle_mod):
    """SphereInit invariants: normal rays cover every layer once with local cosines falling inward (z / r) and column mass = the radial one /
    mu at the top; a grazing ray of 2n points revisits layers n..1 with mirrored column-mass steps and
    flipped local cosines; an angle mu <= 0 and a ray tangent in the top layer are errors."""
    d = H.sphere_pin("s")
    st, _ = H.load_atm("solar")
    g = oracle_mod.sphere_init(st["rhox"], d["height"], float(d["radius"]), d["xmu"])
    nt = len(st["T"])
    for im, mu in enumerate(d["xmu"]):
        N = g["ntau_mu"][im]
        m, mp, ml = g["rhox_mu"][im][:N], g["map"][im][:N], g["mu_loc"][im][:N]
        assert m[0] == st["rhox"][0] / mu and np.all(np.diff(m) > 0)
        if not g["graz"][im]:
            assert N == nt and np.array_equal(mp, np.arange(1, nt + 1))
            assert np.all((ml > 0) & (ml <= 1)) and np.all(np.diff(ml) <= 0)   # more inclined deeper down
        else:
            n = N // 2
            assert N == 2 * n and np.array_equal(mp, np.concatenate([np.arange(1, n + 1), np.arange(n, 0, -1)]))
            assert np.array_equal(ml[n:], -ml[:n][::-1])
            dm = np.diff(m)
            assert np.allclose(dm[n:], dm[:n - 1][::-1], rtol=1e-12)
    assert g["graz"].sum() == 1 and g["graz"][-1] == 1
    with pytest.raises(ValueError):
        oracle_mod.sphere_init(st["rhox"], d["height"], float(d["radius"]), np.array([0.5, 0.0]))
    with pytest.raises(ValueError):   # a radius so small that the outermost ray turns inside the top layer
        oracle_mod.sphere_init(st["rhox"], d["height"], 2.0e9, np.array([0.5, 0.01]))


def test_oracle_sphere_radtran_reference(oracle_mod):
    """LocPrfSph on the reference's own LineOpac / ContOpac (exact RT inputs) against its intensities
    and flux, and the oracle's LineopCalc of the same list against its LineOpac (windows identical)."""
    d = H.sphere_pin("s")
    S, geo, st = _state(oracle_mod, d)
    i0, i1 = int(d["i0"]), int(d["i1"])
    nt = len(st["T"])
    lo = np.zeros((S.nwl, nt)); lo[i0:i1 + 1] = d["lineopac"]
    spl, spc = oracle_mod.radtran(S, d["xmu"], lo)
    spl, spc = spl[i0:i1 + 1], spc[i0:i1 + 1]
    normal = geo["graz"] == 0
    ic0 = d["spc"][:, :1]
    assert np.max(np.abs(spl[:, normal] / d["spl"][:, normal] - 1)) < 1e-8
    assert np.max(np.abs(spc[:, normal] / d["spc"][:, normal] - 1)) < 1e-8
    assert np.max(np.abs(spl[:, ~normal] - d["spl"][:, ~normal]) / ic0) < 1e-9
    assert np.max(np.abs(spc[:, ~normal] - d["spc"][:, ~normal]) / ic0) < 1e-9
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    sfl, sfc = oracle_mod.disk_integ(w, spl, spc)
    assert np.max(np.abs(sfl / d["sfl"] - 1)) < 1e-8 and np.max(np.abs(sfc / d["sfc"] - 1)) < 1e-8
    # the line opacity of the seeded list (geometry does not enter LineopCalc)
    r = oracle_mod.lineop_calc(S, oracle_mod.Lines(**H.pin_lines(d), kind=2), list_type=2)
    lo2, ref = r["lineopac"][i0:i1 + 1], d["lineopac"]
    assert np.array_equal(lo2 > 0, ref > 0)
    assert np.max(np.abs(lo2[ref > 0] / ref[ref > 0] - 1)) < 1e-8


def test_oracle_sphere_linstr_reference(oracle_mod):
    """LinStrCalc's spherical branch (LocPrfSph at the line centre, synth.f90:1801-1803)."""
    d = H.sphere_pin("s")
    S, geo, st = _state(oracle_mod, d)
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    r = oracle_mod.lineop_calc(S, oracle_mod.Lines(**H.pin_lines(d), kind=2), list_type=2, nmu=len(x), xmu=x,
                               wmu=w, want_linstr=True)
    keep = (r["flags"] & 1) == 0
    assert keep.sum() == len(d["linst_wave"])
    assert np.max(np.abs(d["line_wl"][keep] - d["linst_wave"])) < 1e-9
    assert np.max(np.abs(r["linstr"][keep] - d["linst"])) < 1e-7
    # and the spherical depths differ from the plane-parallel ones of the same lines
    ref_pp = H.load_pin("pin_solar_linst")["strength"]
    assert np.max(np.abs(d["linst"] - ref_pp)) > 1e-4


def test_oracle_sphere_stokes_reference(oracle_mod):
    """StokesPrfSph with the stellar-frame field projected at every ray point (BFRAME 0, the local
    cosine changes sign past the tangent point of the grazing ray) against the reference's IQUV."""
    d = H.sphere_pin("m")
    grid, st, co, lines, z = H.mag_pin_setup(d)
    S, geo, _ = _state(oracle_mod, d)
    i0, i1 = int(d["i0"]), int(d["i1"])
    r = oracle_mod.mag_lineop_calc(S, oracle_mod.Lines(**lines, kind=2, zeeman=z), int(d["bframe"]), d["bfield"])
    lo = np.zeros((S.nwl, S.ntau))
    spz, spc = oracle_mod.mag_radtran(S, d["xmu"], int(d["bframe"]), d["bfield"], lo, r["maglineopac"])
    spz, spc = spz[i0:i1 + 1], spc[i0:i1 + 1]
    ref, ic = d["spz"], d["spc"]
    ic0 = ic[:, :1]
    normal = geo["graz"] == 0
    assert np.max(np.abs(spz[:, 0][:, normal] / ref[:, 0][:, normal] - 1)) < 1e-8
    assert np.max(np.abs(spc[:, normal] / ic[:, normal] - 1)) < 1e-8
    for q in range(4):
        assert np.max(np.abs(spz[:, q] - ref[:, q]) / ic0) < 1e-8
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    sfl, _ = oracle_mod.disk_integ(w, spz[:, 0], spc)
    assert np.max(np.abs(sfl / d["sfl"] - 1)) < 1e-8
    # the polarisation is not trivially zero on the grazing ray
    assert np.max(np.abs(ref[:, 3][:, ~normal])) > 0
