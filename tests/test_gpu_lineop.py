"""GPU parity of the line-opacity / formal-solver path against the CPU oracle and the reference.

Tolerances, stated per output:
  * window indices (Ileft, Iright) and line flags: identical (integer work);
  * FP64-faithful path (PREC_FP64) LineOpac vs the oracle: 1e-11 relative (libm ulps only);
  * formal solver SpL/SpC/flux from the same LineOpac: 1e-10 relative (DELO cancellation
    above the Taylor branch amplifies exp/log ulps, solver.f90:155-169);
  * mixed-precision path (FP32 Voigt, compensated sums): LineOpac within 2e-6 of the total
    opacity LineOpac + ContOpac, intensities and flux within 1e-5 relative (the bar).
"""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def ctx_for(fsg, grid, st, co, precision, vmicro=1.0, molbrd=0, limitram_gb=16.0, nmu=7, motype=0, cstd=None):
    C = fsg.Context(precision=precision, vmicro=vmicro, molbrd=molbrd, limitram_gb=limitram_gb)
    C.set_grid(grid["wmode"], grid["wstart"], grid["wend"], grid["dstep"])
    C.set_atmosphere(st)
    C.set_contopac(co, cstd, motype)
    x, w, _ = fsg.mu_quadrature(1, nmu)
    C.set_mu(x, w)
    return C


def oracle_state(oracle_mod, grid, st, co, vmicro=1.0, molbrd=0, motype=0, cstd=None):
    return oracle_mod.State(grid, st, contopac=co, vmicro=vmicro, molbrd=molbrd, motype=motype, contopac_std=cstd)


def solar_case(n=400, w0=5000.0, span=4.0, seed=11, dstep=0.005):
    st, meta = H.load_atm("solar")
    from fastspec_b200 import workloads as W
    grid = dict(wmode=0, wstart=w0, wend=w0 + span, dstep=dstep)
    import fastspec_b200 as F
    wave = F.make_grid(0, w0, w0 + span, dstep) + w0
    co = H.contopac_on(meta, wave)
    L = W.atomic_lines(n, w0 - 0.5, w0 + span + 0.5, seed)
    return grid, st, co, L


def fsg_lines(fsg, L, kind=2):
    return fsg.LineList.from_arrays(L.arrays() if hasattr(L, "arrays") else L, kind=kind)


def ora_lines(oracle_mod, L, kind=2):
    a = L.arrays() if hasattr(L, "arrays") else L
    return oracle_mod.Lines(wl=a["wl"], elo=a["elo"], gf=a["gf"], grad=a["grad"], gqst=a["gqst"],
                            gvdw=a["gvdw"], spc=a["spc"], ismol=a["ismol"], kind=kind)


# ---- Voigt tables and elemental functions --------------------------------------------------------

def test_tables_match_oracle(fsg, oracle_mod):
    C = fsg.Context()
    v, f = C.voigt_tables()
    ov = oracle_mod.voigt_table()
    of = oracle_mod.fvoigt_table()
    # FP32 entries of FP64 sums: device and glibc libm differ by ulps, so a rounding flip
    # changes at most a few entries by one FP32 ulp
    dv = np.abs(v.view(np.int32).astype(np.int64) - ov.view(np.int32).astype(np.int64))
    assert dv.max() <= 1 and (dv > 0).sum() < 50
    df = np.abs(f.view(np.int32).astype(np.int64) - of.view(np.int32).astype(np.int64))
    assert df[..., 0].max() <= 1
    # L(a, 0) is zero analytically; the sums leave ~1e-17 noise there
    np.testing.assert_allclose(f[..., 1], of[..., 1], rtol=1e-6, atol=1e-12)


def test_hvoigt_fvoigt_elemental(fsg, oracle_mod):
    rng = np.random.default_rng(1)
    a = np.concatenate([rng.uniform(0, 9, 3000), 10 ** rng.uniform(-6, 1.5, 3000)])
    v = np.concatenate([rng.uniform(-20, 20, 3000), rng.uniform(-9, 9, 3000)])
    C = fsg.Context()
    h = C.hvoigt(a, v)
    ref = np.array([oracle_mod.hvoigt(x, y) for x, y in zip(a, v)])
    np.testing.assert_allclose(h, ref, rtol=1e-13, atol=0)
    hh, ll = C.fvoigt(a, v)
    refp = [oracle_mod.fvoigt(x, y) for x, y in zip(a, v)]
    np.testing.assert_allclose(hh, [r[0] for r in refp], rtol=1e-6, atol=1e-30)
    np.testing.assert_allclose(ll, [r[1] for r in refp], rtol=1e-6, atol=1e-12)


# ---- central pass, FP64 path, solver ---------------------------------------------------------------

@pytest.mark.parametrize("prec", [0, 1])
def test_windows_bit_exact(fsg, oracle_mod, prec):
    grid, st, co, L = solar_case()
    C = ctx_for(fsg, grid, st, co, prec)
    g = C.lineop_calc(fsg_lines(fsg, L))
    S = oracle_state(oracle_mod, grid, st, co)
    r = oracle_mod.lineop_calc(S, ora_lines(oracle_mod, L), list_type=2)
    assert np.array_equal(g["flags"] & 1, r["flags"] & 1)
    keep = (r["flags"] & 1) == 0
    assert keep.sum() > 50
    assert np.array_equal(g["ileft"][keep], r["ileft"][keep])
    assert np.array_equal(g["iright"][keep], r["iright"][keep])


def test_fp64_path_matches_oracle(fsg, oracle_mod):
    grid, st, co, L = solar_case()
    C = ctx_for(fsg, grid, st, co, fsg.PREC_FP64)
    g = C.lineop_calc(fsg_lines(fsg, L))
    S = oracle_state(oracle_mod, grid, st, co)
    r = oracle_mod.lineop_calc(S, ora_lines(oracle_mod, L), list_type=2)
    # same wide-line marking as the reference (bit 3)
    assert np.array_equal(g["flags"], r["flags"])
    m = r["lineopac"] > 0
    assert np.array_equal(g["lineopac"] > 0, m)
    assert np.max(np.abs(g["lineopac"][m] / r["lineopac"][m] - 1)) < 1e-11
    spl, spc, sfl, sfc = C.radtran()
    ospl, ospc = oracle_mod.radtran(S, C_mu(fsg), r["lineopac"])
    assert np.max(np.abs(spl / ospl - 1)) < 1e-10
    assert np.max(np.abs(spc / ospc - 1)) < 1e-10


def C_mu(fsg, n=7):
    return fsg.mu_quadrature(1, n)[0]


def test_radtran_matches_oracle_given_opacity(fsg, oracle_mod):
    grid, st, co, L = solar_case(n=10)
    rng = np.random.default_rng(2)
    lo = np.abs(co) * 10 ** rng.uniform(-6, 3, co.shape)
    C = ctx_for(fsg, grid, st, co, 0)
    C.lineop_set(lo)
    spl, spc, sfl, sfc = C.radtran()
    S = oracle_state(oracle_mod, grid, st, co)
    x, w, _ = oracle_mod.mu_quadrature(1, 7)
    ospl, ospc = oracle_mod.radtran(S, x, lo)
    osfl, osfc = oracle_mod.disk_integ(w, ospl, ospc)
    assert np.max(np.abs(spl / ospl - 1)) < 1e-10
    assert np.max(np.abs(spc / ospc - 1)) < 1e-10
    assert np.max(np.abs(sfl / osfl - 1)) < 1e-10
    assert np.max(np.abs(sfc / osfc - 1)) < 1e-10


def test_locprf_pp_matches_oracle(fsg, oracle_mod):
    st, _ = H.load_atm("solar")
    rng = np.random.default_rng(4)
    nt = len(st["T"])
    xki = 10 ** rng.uniform(-3, 2, (64, nt)) * np.linspace(1, 50, nt)
    src = 1e14 * (1 + rng.uniform(0, 1, (64, nt))) * np.linspace(1, 3, nt)
    x = np.array([1.0, 0.7, 0.3, 0.05])
    C = fsg.Context()
    g = C.locprf_pp(x, xki, src, st["rhox"])
    ref = np.array([oracle_mod.locprf_pp(x, xki[i], src[i], st["rhox"]) for i in range(64)])
    assert np.max(np.abs(g / ref - 1)) < 1e-10


# ---- mixed-precision path ------------------------------------------------------------------------------

def mixed_vs_oracle(fsg, oracle_mod, grid, st, co, L, vmicro=1.0, molbrd=0, limitram_gb=16.0, kind=2):
    C = ctx_for(fsg, grid, st, co, fsg.PREC_MIXED, vmicro=vmicro, molbrd=molbrd, limitram_gb=limitram_gb)
    g = C.lineop_calc(fsg_lines(fsg, L, kind), want_lines=True)
    spl, spc, sfl, sfc = C.radtran()
    S = oracle_state(oracle_mod, grid, st, co, vmicro=vmicro, molbrd=molbrd)
    r = oracle_mod.lineop_calc(S, ora_lines(oracle_mod, L, kind), list_type=kind)
    x, w, _ = oracle_mod.mu_quadrature(1, 7)
    ospl, ospc = oracle_mod.radtran(S, x, r["lineopac"])
    osfl, osfc = oracle_mod.disk_integ(w, ospl, ospc)
    return dict(g=g, r=r, spl=spl, ospl=ospl, spc=spc, ospc=ospc, sfl=sfl, osfl=osfl, co=co, C=C)


def check_mixed(R, lo_tol=2e-6, sp_tol=1e-5):
    g, r, co = R["g"], R["r"], R["co"]
    assert np.array_equal(g["lineopac"] > 0, r["lineopac"] > 0)
    err = np.abs(g["lineopac"] - r["lineopac"]) / (r["lineopac"] + co)
    assert err.max() < lo_tol, err.max()
    assert np.max(np.abs(R["spl"] / R["ospl"] - 1)) < sp_tol
    assert np.max(np.abs(R["sfl"] / R["osfl"] - 1)) < sp_tol
    return err.max()


def test_mixed_path_solar(fsg, oracle_mod):
    grid, st, co, L = solar_case(n=600, span=6.0)
    check_mixed(mixed_vs_oracle(fsg, oracle_mod, grid, st, co, L))


def test_mixed_path_cooldwarf_molecular_log_grid(fsg, oracle_mod):
    st, meta = H.load_atm("cooldwarf")
    from fastspec_b200 import workloads as W
    import fastspec_b200 as F
    w0, span = 9000.0, 12.0
    grid = dict(wmode=1, wstart=w0, wend=w0 + span, dstep=1.0)
    wave = F.make_grid(1, w0, w0 + span, 1.0) + w0
    co = H.contopac_on(meta, wave)
    L = W.molecular_lines(3000, w0 - 2, w0 + span + 2, 21)
    check_mixed(mixed_vs_oracle(fsg, oracle_mod, grid, st, co, L, molbrd=1))


@pytest.mark.parametrize("name", ["pin_solar", "pin_cooldwarf"])
def test_mixed_path_against_reference_pins(fsg, oracle_mod, name):
    d = H.load_pin(name)
    grid, st, meta, co = H.pin_setup(d)
    C = ctx_for(fsg, grid, st, co, fsg.PREC_MIXED, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    g = C.lineop_calc(fsg.LineList.from_arrays(H.pin_lines(d)))
    i0, i1 = int(d["i0"]), int(d["i1"])
    lo = g["lineopac"][i0:i1 + 1]
    assert np.array_equal(lo > 0, d["lineopac"] > 0)          # windows: bit-exact with the reference
    err = np.abs(lo - d["lineopac"]) / (d["lineopac"] + d["contopac"])
    assert err.max() < 2e-6
    spl, spc, sfl, sfc = C.radtran()
    assert np.max(np.abs(spl[i0:i1 + 1] / d["spl"] - 1)) < 1e-5
    assert np.max(np.abs(sfl[i0:i1 + 1] / d["sfl"] - 1)) < 1e-5
    assert np.max(np.abs(spc[i0:i1 + 1] / d["spc"] - 1)) < 1e-8


@pytest.mark.parametrize("name", ["pin_solar", "pin_cooldwarf"])
@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_linstr_against_reference_pins(fsg, name, prec):
    """LinStrCalc on the GPU (FP64 in both precisions) against the reference's fs_linst.bin:
    REAL(4) central depths of the retained lines, within 1e-7."""
    d = H.load_pin(name)
    ref = H.load_pin(name + "_linst")
    grid, st, meta, co = H.pin_setup(d)
    C = ctx_for(fsg, grid, st, co, fsg.PREC_MIXED if prec == "mixed" else fsg.PREC_FP64,
                vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]), nmu=len(d["xmu"]))
    g = C.lineop_calc(fsg.LineList.from_arrays(H.pin_lines(d)), want_linstr=True)
    keep = (g["flags"] & 1) == 0
    assert keep.sum() == len(ref["wave"])
    assert np.max(np.abs(d["line_wl"][keep] - ref["wave"])) < 1e-9
    assert np.max(np.abs(g["linstr"][keep] - ref["strength"])) < 1e-7
    assert np.all(g["linstr"][~keep] == 0.0)


@pytest.mark.parametrize("nmu", [1, 5])
def test_linstr_vs_oracle(fsg, oracle_mod, nmu):
    """Single-angle depth (nmu = 1) and disk-integrated depth against the oracle."""
    grid, st, co, L = solar_case(n=300, seed=41)
    C = ctx_for(fsg, grid, st, co, fsg.PREC_MIXED, nmu=nmu)
    g = C.lineop_calc(fsg_lines(fsg, L), want_linstr=True)
    S = oracle_state(oracle_mod, grid, st, co)
    x, w, _ = oracle_mod.mu_quadrature(1, nmu)
    r = oracle_mod.lineop_calc(S, ora_lines(oracle_mod, L), list_type=2, nmu=nmu, xmu=x, wmu=w, want_linstr=True)
    assert np.array_equal(g["flags"] & 1, r["flags"] & 1)        # the mixed path marks no wide lines
    assert np.max(np.abs(g["linstr"] - r["linstr"])) < 1e-7


def test_linstr_needs_mu(fsg):
    grid, st, co, L = solar_case(n=20, seed=42)
    C = fsg.Context()
    C.set_grid(grid["wmode"], grid["wstart"], grid["wend"], grid["dstep"])
    C.set_atmosphere(st)
    C.set_contopac(co)
    with pytest.raises(fsg.FsgError):
        C.lineop_calc(fsg_lines(fsg, L), want_linstr=True)


@pytest.mark.parametrize("name", ["pin_solar", "pin_cooldwarf"])
def test_fp64_path_against_reference_pins(fsg, name):
    d = H.load_pin(name)
    grid, st, meta, co = H.pin_setup(d)
    C = ctx_for(fsg, grid, st, co, fsg.PREC_FP64, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    g = C.lineop_calc(fsg.LineList.from_arrays(H.pin_lines(d)))
    i0, i1 = int(d["i0"]), int(d["i1"])
    lo, ref = g["lineopac"][i0:i1 + 1], d["lineopac"]
    m = ref > 0
    assert np.array_equal(lo > 0, m)
    assert np.max(np.abs(lo[m] / ref[m] - 1)) < 1e-8
    spl, spc, sfl, sfc = C.radtran()
    assert np.max(np.abs(spl[i0:i1 + 1] / d["spl"] - 1)) < 1e-8
    assert np.max(np.abs(sfl[i0:i1 + 1] / d["sfl"] - 1)) < 1e-8


def test_blocks_equal_single_block(fsg, oracle_mod):
    """A tiny LIMITRAM forces many blocks / segments; results must not change."""
    grid, st, co, L = solar_case(n=800, span=6.0, seed=5)
    # FP64 blocks hold limitram / (24 B x Ntau) lines: 1e-3 GB -> ~740 of 800 lines, two segments
    # (much smaller blocks trip the reference's own segmentation error, synth.f90:1035-1040)
    for prec, tol, ram in ((fsg.PREC_MIXED, 1e-6, 3e-5), (fsg.PREC_FP64, 1e-13, 1e-3)):
        a = ctx_for(fsg, grid, st, co, prec).lineop_calc(fsg_lines(fsg, L))
        b = ctx_for(fsg, grid, st, co, prec, limitram_gb=ram).lineop_calc(fsg_lines(fsg, L))
        assert b["stats"]["nblocks"] > a["stats"]["nblocks"]
        m = a["lineopac"] > 0
        assert np.array_equal(m, b["lineopac"] > 0)
        assert np.max(np.abs(a["lineopac"][m] / b["lineopac"][m] - 1)) < tol


def test_deterministic(fsg):
    grid, st, co, L = solar_case(n=500)
    C = ctx_for(fsg, grid, st, co, fsg.PREC_MIXED)
    a = C.lineop_calc(fsg_lines(fsg, L))["lineopac"]
    C.lineop_reset()
    b = C.lineop_calc(fsg_lines(fsg, L))["lineopac"]
    assert np.array_equal(a, b)


def test_accumulates_across_lists(fsg):
    grid, st, co, L = solar_case(n=300)
    C = ctx_for(fsg, grid, st, co, fsg.PREC_FP64)
    a = C.lineop_calc(fsg_lines(fsg, L))["lineopac"].copy()
    b = C.lineop_calc(fsg_lines(fsg, L))["lineopac"]
    np.testing.assert_allclose(b, 2 * a, rtol=1e-14, atol=0)   # wide-line and block sums add in a different order


# ---- edge cases ------------------------------------------------------------------------------------------

def test_empty_and_all_weak_lists(fsg, oracle_mod):
    grid, st, co, L = solar_case(n=50)
    C = ctx_for(fsg, grid, st, co, 0)
    a = L.arrays()
    empty = {k: v[:0] for k, v in a.items()}
    g = C.lineop_calc(fsg.LineList.from_arrays(empty))
    assert np.all(g["lineopac"] == 0)
    weak = dict(a)
    weak["gf"] = np.full_like(a["gf"], 1e-30)
    g = C.lineop_calc(fsg.LineList.from_arrays(weak))
    assert np.all(g["flags"] & 1) and np.all(g["lineopac"] == 0)
    spl, spc, sfl, sfc = C.radtran()
    np.testing.assert_allclose(spl, spc, rtol=0, atol=0)


def test_lines_outside_grid_and_single_line(fsg, oracle_mod):
    grid, st, co, L = solar_case(n=40, span=2.0)
    a = L.arrays()
    sel = dict((k, v.copy()) for k, v in a.items())
    sel["wl"] = np.sort(np.concatenate([[grid["wstart"] - 3.0], a["wl"][1:-1], [grid["wend"] + 3.0]]))
    for lst in (sel, {k: v[5:6] for k, v in a.items()}):
        for prec in (0, 1):
            C = ctx_for(fsg, grid, st, co, prec)
            g = C.lineop_calc(fsg.LineList.from_arrays(lst))
            S = oracle_state(oracle_mod, grid, st, co)
            r = oracle_mod.lineop_calc(S, ora_lines(oracle_mod, lst), list_type=2)
            assert np.array_equal(g["ileft"], r["ileft"]) and np.array_equal(g["iright"], r["iright"])
            err = np.abs(g["lineopac"] - r["lineopac"]) / (r["lineopac"] + co)
            assert err.max() < 2e-6


def test_motype1_abo_and_molecular_modes(fsg, oracle_mod):
    """ContOpacStd division (Motype 1), ABO van der Waals (Gvdw > 10), classical Stark/Unsold
    modes (non-positive inputs), molecules with MolBrd 0/1 and VWmol."""
    grid, st, co, L = solar_case(n=300, span=3.0, seed=8)
    a = {k: v.copy() for k, v in L.arrays().items()}
    n = len(a["wl"])
    a["gvdw"][::5] = np.float32(240.25)        # ABO sigma.alpha
    a["gqst"][1::7] = 0.0                       # classical Stark
    a["gvdw"][2::7] = 0.0                       # Unsold
    a["ismol"][3::9] = 1                        # molecule flag
    cstd = np.linspace(0.5, 2.0, len(st["T"]))
    for molbrd in (0, 1):
        for prec in (0, 1):
            C = fsg.Context(precision=prec, vmicro=1.0, molbrd=molbrd, vwmol=0.0)
            C.set_grid(0, grid["wstart"], grid["wend"], grid["dstep"]); C.set_atmosphere(st)
            C.set_contopac(co, cstd, 1)
            x, w, _ = fsg.mu_quadrature(1, 7); C.set_mu(x, w)
            g = C.lineop_calc(fsg.LineList.from_arrays(a))
            S = oracle_mod.State(grid, st, contopac=co, contopac_std=cstd, motype=1, vmicro=1.0, molbrd=molbrd)
            r = oracle_mod.lineop_calc(S, ora_lines(oracle_mod, a), list_type=2)
            assert np.array_equal(g["flags"] & 7, r["flags"] & 7)
            assert np.array_equal(g["ileft"], r["ileft"]) and np.array_equal(g["iright"], r["iright"])
            tol = 1e-11 if prec == 1 else 2e-6
            err = np.abs(g["lineopac"] - r["lineopac"]) / (r["lineopac"] + co / cstd)
            assert err.max() < tol


def test_call_order_errors(fsg):
    C = fsg.Context()
    grid, st, co, L = solar_case(n=5)
    with pytest.raises(fsg.FsgError):
        C.lineop_calc(fsg_lines(fsg, L))
    C.set_grid(0, grid["wstart"], grid["wend"], grid["dstep"])
    C.set_atmosphere(st)
    with pytest.raises(fsg.FsgError):
        C.lineop_calc(fsg_lines(fsg, L))
    with pytest.raises(fsg.FsgError):
        C.set_contopac(co[:-1])


def test_segmentation_overflow_is_reported(fsg):
    """A block too small for the lines at one wavelength stops with the reference's message."""
    grid, st, co, L = solar_case(n=800, span=6.0, seed=5)
    C = ctx_for(fsg, grid, st, co, fsg.PREC_FP64, limitram_gb=3e-5)
    with pytest.raises(fsg.FsgError, match="segmentation"):
        C.lineop_calc(fsg_lines(fsg, L))


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_he_stark_shifted_lines(fsg, oracle_mod, prec):
    """He I lines with per-depth Stark widths and shifts (hestark.f90 tables, opacity.f90:297-346):
    species 0 stands in for He I, a third of its lines carry table indices 1..3."""
    grid, st, co, L = solar_case(n=300, seed=61)
    a = dict(L.arrays())
    rng = np.random.default_rng(61)
    ihe = np.zeros(len(a["wl"]), np.int32)
    sel = np.nonzero(a["spc"] == 0)[0][::3]
    ihe[sel] = rng.integers(1, 4, len(sel))
    a["ihe"] = ihe
    nt = len(st["T"])
    depth = np.linspace(0.0, 1.0, nt)
    hegam = np.stack([1e9 * (1 + k) * (1 + 3 * depth) for k in range(3)])
    heshf = np.stack([(0.02 + 0.03 * k) * (0.2 + depth) for k in range(3)])
    C = ctx_for(fsg, grid, st, co, fsg.PREC_MIXED if prec == "mixed" else fsg.PREC_FP64)
    C.set_hestark(hegam, heshf, 0)
    g = C.lineop_calc(fsg.LineList.from_arrays(a))
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0, hegam=hegam, heshf=heshf, spc_he1=0)
    r = oracle_mod.lineop_calc(S, oracle_mod.Lines(**a, kind=2), list_type=2)
    assert np.any((r["flags"] >> 8) & 255)
    assert np.array_equal(g["flags"] & ~8, r["flags"] & ~8)
    assert np.array_equal(g["ileft"], r["ileft"]) and np.array_equal(g["iright"], r["iright"])
    tol = 2e-6 if prec == "mixed" else 1e-11
    assert np.max(np.abs(g["lineopac"] - r["lineopac"]) / (r["lineopac"] + co)) < tol


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_broadening_modes_against_reference_pin(fsg, prec):
    """Classical Stark, Unsold and ABO lines with EPSOPAC 3e-3 and VWFUDGE 1.8 through the GPU path: the
    reference's line opacity, windows and flux (tests/golden/pin_solar_modes.npz); FP64 1e-8, mixed
    within the mixed bars."""
    d = H.load_pin("pin_solar_modes")
    grid, st, meta, co = H.pin_setup(d)
    C = fsg.Context(precision=fsg.PREC_MIXED if prec == "mixed" else fsg.PREC_FP64, vmicro=float(d["vmicro"]),
                    molbrd=int(d["molbrd"]), epsopac=float(d["epsopac"]), vwfudge=float(d["vwfudge"]))
    C.set_grid(grid["wmode"], grid["wstart"], grid["wend"], grid["dstep"])
    C.set_atmosphere(st)
    C.set_contopac(co)
    x, w, _ = fsg.mu_quadrature(1, len(d["xmu"]))
    C.set_mu(x, w)
    g = C.lineop_calc(fsg.LineList.from_arrays(H.pin_lines(d)))
    i0, i1 = int(d["i0"]), int(d["i1"])
    lo, ref = g["lineopac"][i0:i1 + 1], d["lineopac"]
    assert np.array_equal(lo > 0, ref > 0)
    if prec == "fp64":
        assert np.max(np.abs(lo[ref > 0] / ref[ref > 0] - 1)) < 1e-8
    else:
        assert np.max(np.abs(lo - ref) / (ref + d["contopac"])) < 2e-6
    spl, spc, sfl, sfc = C.radtran()
    assert np.max(np.abs(sfl[i0:i1 + 1] / d["sfl"] - 1)) < (1e-8 if prec == "fp64" else 1e-5)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_molecular_options_against_reference_pin(fsg, prec):
    """H2BRD 1.5 (H2 among the van der Waals perturbers of XlineInit) and VWMOL 4e-8 on the cool-dwarf
    list through the GPU path: the reference's line opacity, windows and flux
    (tests/golden/pin_cooldwarf_opts.npz); FP64 1e-8, mixed within the mixed bars."""
    d = H.load_pin("pin_cooldwarf_opts")
    grid, st, meta, co = H.pin_setup(d)
    C = fsg.Context(precision=fsg.PREC_MIXED if prec == "mixed" else fsg.PREC_FP64, vmicro=float(d["vmicro"]),
                    molbrd=int(d["molbrd"]), h2brd=float(d["h2brd"]), vwmol=float(d["vwmol"]))
    C.set_grid(grid["wmode"], grid["wstart"], grid["wend"], grid["dstep"])
    C.set_atmosphere(st)
    C.set_contopac(co)
    x, w, _ = fsg.mu_quadrature(1, len(d["xmu"]))
    C.set_mu(x, w)
    g = C.lineop_calc(fsg.LineList.from_arrays(H.pin_lines(d)))
    i0, i1 = int(d["i0"]), int(d["i1"])
    lo, ref = g["lineopac"][i0:i1 + 1], d["lineopac"]
    assert np.array_equal(lo > 0, ref > 0)
    if prec == "fp64":
        assert np.max(np.abs(lo[ref > 0] / ref[ref > 0] - 1)) < 1e-8
    else:
        assert np.max(np.abs(lo - ref) / (ref + d["contopac"])) < 2e-6
    spl, spc, sfl, sfc = C.radtran()
    assert np.max(np.abs(sfl[i0:i1 + 1] / d["sfl"] - 1)) < (1e-8 if prec == "fp64" else 1e-5)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_opacity_reentry_against_reference_pin(fsg, tmp_path, prec):
    """OPACITY= re-entry through the library: list A's device line opacity (fsg_lineop_get) written by
    fsio.write_opac and read back, loaded into a fresh context (fsg_lineop_set), list B accumulated onto
    it; the reference program did the same with the file of the oracle's A
    (tests/golden/pin_solar_reentry.npz).  FP64 1e-8; mixed 4e-6 (two lists, each within the 2e-6 bar)."""
    from fastspec_b200 import fsio
    d = H.load_pin("pin_solar_reentry")
    grid, st, meta, co = H.pin_setup(d)
    prc = fsg.PREC_MIXED if prec == "mixed" else fsg.PREC_FP64
    C = ctx_for(fsg, grid, st, co, prc, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    A = {k[2:]: d[k] for k in d if k.startswith("a_")}
    C.lineop_calc(fsg.LineList.from_arrays(A), want_lines=False)
    p = str(tmp_path / "opac_a.bin")
    fsio.write_opac(p, C.wave + C.wfirst, C.lineop_get(), st["rhox"], st["T"], st["xne"], st["xna"], st["rho"])
    C2 = ctx_for(fsg, grid, st, co, prc, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    C2.lineop_set(fsio.read_opac(p)["opac"])
    g = C2.lineop_calc(fsg.LineList.from_arrays(H.pin_lines(d)))
    i0, i1 = int(d["i0"]), int(d["i1"])
    lo, ref = g["lineopac"][i0:i1 + 1], d["lineopac"]
    assert np.array_equal(lo > 0, ref > 0)
    if prec == "fp64":
        assert np.max(np.abs(lo[ref > 0] / ref[ref > 0] - 1)) < 1e-8
    else:
        assert np.max(np.abs(lo - ref) / (ref + d["contopac"])) < 4e-6
    spl, spc, sfl, sfc = C2.radtran()
    assert np.max(np.abs(sfl[i0:i1 + 1] / d["sfl"] - 1)) < (1e-8 if prec == "fp64" else 1e-5)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_hot_he_lines_against_reference_pin(fsg, prec):
    """Tabulated He I Stark lines in a Teff 15000 K atmosphere (hestark.f90): Context.hestark_init builds
    the 37 lines' widths and shifts on the host (fsg_hestark_tables) and the lists' table entries come
    from fsg_he_match_idx; line opacity, windows and flux against the reference program's run
    (tests/golden/pin_hot_he.npz).  FP64 1e-8; mixed within the mixed bars (the tabulated lines take
    the FP64 per-depth-shift kernel, the others the FP32 passes)."""
    from test_hestark import hot_state
    d = H.load_pin("pin_hot_he")
    grid, st, meta, co = H.pin_setup(d)
    _, _, hii, heii = hot_state()
    C = ctx_for(fsg, grid, st, co, fsg.PREC_MIXED if prec == "mixed" else fsg.PREC_FP64,
                vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    C.hestark_init(hii, heii, 0)
    g = C.lineop_calc(fsg.LineList.from_arrays(H.pin_lines(d)))
    assert np.array_equal((g["flags"] >> 8) & 255, d["ihe_expected"])
    lo, ref = g["lineopac"], d["lineopac"]
    assert np.array_equal(lo > 0, ref > 0)
    if prec == "fp64":
        assert np.max(np.abs(lo[ref > 0] / ref[ref > 0] - 1)) < 1e-8
    else:
        assert np.max(np.abs(lo - ref) / (ref + d["contopac"])) < 2e-6
    spl, spc, sfl, sfc = C.radtran()
    assert np.max(np.abs(sfl / d["sfl"] - 1)) < (1e-8 if prec == "fp64" else 1e-5)
    C.close()


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_hdf5_list_against_reference_pin(fsg, tmp_path, prec):
    """A line list in the reference's HDF5 layout, read by fsio.read_hdf5_lines as an atomic list
    (kind 0), through the GPU path: the reference program's line opacity and flux for the same file
    (tests/golden/pin_solar_h5.npz); windows identical, FP64 1e-8, mixed within the mixed bars."""
    from test_hdf5 import hdf5_pin_lines
    d, r = hdf5_pin_lines(tmp_path)
    grid, st, meta, co = H.pin_setup(d)
    C = ctx_for(fsg, grid, st, co, fsg.PREC_MIXED if prec == "mixed" else fsg.PREC_FP64,
                vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    a = {k: r[k] for k in ("wl", "elo", "gf", "grad", "gqst", "gvdw", "spc", "ismol")}
    g = C.lineop_calc(fsg.LineList.from_arrays(a, kind=r["kind"]))
    i0, i1 = int(d["i0"]), int(d["i1"])
    lo, ref = g["lineopac"][i0:i1 + 1], d["lineopac"]
    assert np.array_equal(lo > 0, ref > 0)
    if prec == "fp64":
        assert np.max(np.abs(lo[ref > 0] / ref[ref > 0] - 1)) < 1e-8
    else:
        assert np.max(np.abs(lo - ref) / (ref + d["contopac"])) < 2e-6
    spl, spc, sfl, sfc = C.radtran()
    assert np.max(np.abs(sfl[i0:i1 + 1] / d["sfl"] - 1)) < (1e-8 if prec == "fp64" else 1e-5)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_molecular_h5_lists_against_reference_pin(fsg, tmp_path, prec):
    """Four single-species molecular HDF5 lists (kind 1) through fsg_lineop_calc one after the other
    (the device LineOpac accumulates): the reference's line opacity and flux for the same files (FP64
    path within 2e-7: one-ulp differences of some lines' FP32 gf, as for the oracle)."""
    from test_hdf5 import mol_h5_pin_lists
    d, lists = mol_h5_pin_lists(tmp_path)
    grid, st, meta, co = H.pin_setup(d)
    C = ctx_for(fsg, grid, st, co, fsg.PREC_MIXED if prec == "mixed" else fsg.PREC_FP64,
                vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    for r in lists:
        a = {k: r[k] for k in ("wl", "elo", "gf", "grad", "gqst", "gvdw", "spc", "ismol")}
        g = C.lineop_calc(fsg.LineList.from_arrays(a, kind=r["kind"]))
    i0, i1 = int(d["i0"]), int(d["i1"])
    lo, ref = g["lineopac"][i0:i1 + 1], d["lineopac"]
    assert np.array_equal(lo > 0, ref > 0)
    if prec == "fp64":
        assert np.max(np.abs(lo[ref > 0] / ref[ref > 0] - 1)) < 2e-7
    else:
        assert np.max(np.abs(lo - ref) / (ref + d["contopac"])) < 2e-6
    spl, spc, sfl, sfc = C.radtran()
    assert np.max(np.abs(sfl[i0:i1 + 1] / d["sfl"] - 1)) < (2e-7 if prec == "fp64" else 1e-5)
