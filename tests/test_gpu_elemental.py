"""The kernel-level entry points of the C-ABI (the reference's elemental routines, batched on the GPU)
against the oracle's restatement of the same routine on the same inputs: XlineSetup / XlineDepth
(opacity.f90:96-293), LineOpacity1 / LineOpacity2 (opacity.f90:297-386), MagLineOpacity1
(opacity.f90:391-464), AnalyticWindow (opacity.f90:678-710) and StokesPrfPP (solver.f90:265-394).

Bars: integer fields identical; FP64 values within 1e-12 relative (the same operations in the same
order; CUDA's and glibc's exp/log/pow may differ in the last bit)."""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

REL = 1e-12


def rel_err(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    scale = np.maximum(np.abs(b), 1e-300)
    return float(np.max(np.abs(a - b) / scale)) if a.size else 0.0


def solar_setup(fsg, oracle_mod, w0=5000.0, w1=5006.0, dstep=0.005, lines=None, molbrd=0):
    st, meta = H.load_atm("solar")
    grid = dict(wmode=0, wstart=w0, wend=w1, dstep=dstep)
    co = H.contopac_on(meta, fsg.make_grid(0, w0, w1, dstep) + w0)
    C = fsg.Context(precision=fsg.PREC_FP64, vmicro=1.0, molbrd=molbrd)
    C.set_grid(0, w0, w1, dstep)
    C.set_atmosphere(st)
    C.set_contopac(co)
    x, w, _ = fsg.mu_quadrature(1, 7)
    C.set_mu(x, w)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0, molbrd=molbrd)
    return C, S, co


def block_of(oracle_mod, S, arrays):
    """The reference's block arrays for a list (one block, Loff = 0): windows from the oracle's
    LineopCalc central pass, parameters from its XlineSetup / XlineDepth."""
    OL = oracle_mod.Lines(**arrays, kind=2)
    r = oracle_mod.lineop_calc(S, OL, list_type=2, wrange=(1, 0))
    n = len(arrays["wl"])
    cop, vv, av = (np.zeros((n, S.ntau)) for _ in range(3))
    for i in range(n):
        xc = oracle_mod.xline_setup(S, OL, i)
        cop[i], vv[i], av[i] = oracle_mod.xline_depth(S, xc)
    return dict(wlcent=arrays["wl"] - S.wfirst, flags=r["flags"], ileft=r["ileft"], iright=r["iright"],
                lincop=cop, linvvgt=vv, linavgt=av)


def test_xline_setup_and_depth(fsg, oracle_mod):
    """Every Stark / van der Waals mode: the pin list of classical Stark, Unsold and ABO lines, seeded
    atomic lines, and molecular lines with molecular broadening on."""
    from fastspec_b200 import workloads as W
    cases = [(H.pin_lines(H.load_pin("pin_solar_modes")), 0),
             (W.atomic_lines(300, 5000.0, 5006.0, W.SEED0 + 70).arrays(), 0)]
    for arrays, molbrd in cases:
        C, S, _ = solar_setup(fsg, oracle_mod, molbrd=molbrd)
        xc = C.xline_setup(fsg.LineList.from_arrays(arrays))
        OL = oracle_mod.Lines(**arrays, kind=2)
        cop, vv, av = C.xline_depth(xc)
        for i in range(len(arrays["wl"])):
            o = oracle_mod.xline_setup(S, OL, i)
            for f in ("IxPF", "MdQst", "MdVdw", "IxHe"):
                assert int(xc[f][i]) == getattr(o, f), (i, f)
            for f in ("WaveL", "Hnux", "Elo", "Gf", "Grad", "Xmass", "Cqst", "Qdiv", "Cvdw", "AboPre", "AboVbc",
                      "AboExp"):
                assert rel_err(xc[f][i], getattr(o, f)) <= REL, (i, f, xc[f][i], getattr(o, f))
            oc, ov, oa = oracle_mod.xline_depth(S, o)
            assert rel_err(cop[i], oc) <= REL and rel_err(vv[i], ov) <= REL and rel_err(av[i], oa) <= REL
        C.close()


def test_xline_molecular(fsg, oracle_mod):
    from fastspec_b200 import workloads as W
    st, meta = H.load_atm("cooldwarf")
    grid = dict(wmode=1, wstart=10000.0, wend=10002.0, dstep=1.0)
    C = fsg.Context(precision=fsg.PREC_FP64, vmicro=meta["vmicro"], molbrd=meta["molbrd"])
    C.set_grid(1, 10000.0, 10002.0, 1.0)
    C.set_atmosphere(st)
    S = oracle_mod.State(grid, st, vmicro=meta["vmicro"], molbrd=meta["molbrd"])
    arrays = W.molecular_lines(200, 10000.0, 10002.0, W.SEED0 + 71).arrays()
    xc = C.xline_setup(fsg.LineList.from_arrays(arrays))
    cop, vv, av = C.xline_depth(xc)
    OL = oracle_mod.Lines(**arrays, kind=2)
    for i in range(len(arrays["wl"])):
        o = oracle_mod.xline_setup(S, OL, i)
        assert (int(xc["MdQst"][i]), int(xc["MdVdw"][i])) == (o.MdQst, o.MdVdw)
        oc, ov, oa = oracle_mod.xline_depth(S, o)
        assert rel_err(cop[i], oc) <= REL and rel_err(vv[i], ov) <= REL and rel_err(av[i], oa) <= REL
    C.close()


def test_lineopacity1_and_2(fsg, oracle_mod):
    from fastspec_b200 import workloads as W
    C, S, co = solar_setup(fsg, oracle_mod)
    arrays = W.atomic_lines(300, 4999.5, 5006.5, W.SEED0 + 72).arrays()
    b = block_of(oracle_mod, S, arrays)
    n = len(arrays["wl"])
    rng = np.random.default_rng(7)
    npts = 150
    iwl = rng.integers(1, S.nwl + 1, npts).astype(np.int32)
    wl = S.wave[iwl - 1]
    # LineOpacity1 over all lines (Loff = 0) and over a sub-block of lines 101..n (Loff = 100)
    l1 = np.ones(npts, np.int32)
    l2 = np.full(npts, n, np.int32)
    B = fsg.LineBlock(**b)
    got = C.lineopacity1(B, wl, l1, l2, iwl, 0)
    for k in range(npts):
        ref = oracle_mod.lineopacity1(S, b, wl[k], 1, n, iwl[k], 0)
        assert rel_err(got[k], ref) <= REL, k
    sub = dict(b, lincop=b["lincop"][100:], linvvgt=b["linvvgt"][100:], linavgt=b["linavgt"][100:])
    Bs = fsg.LineBlock(**sub)
    l1s = np.full(npts, 101, np.int32)
    got = C.lineopacity1(Bs, wl, l1s, l2, iwl, 100)
    for k in range(npts):
        ref = oracle_mod.lineopacity1(S, sub, wl[k], 101, n, iwl[k], 100)
        assert rel_err(got[k], ref) <= REL, k
    # LineOpacity2: point k = line q at wavelength iwl[k] (in or out of its window) with its own rows
    q = rng.integers(0, n, npts)
    got = C.lineopacity2(B, wl, (q + 1).astype(np.int32), iwl, b["lincop"][q], b["linvvgt"][q], b["linavgt"][q])
    nz = 0
    for k in range(npts):
        i = q[k]
        ref = oracle_mod.lineopacity2(S, wl[k], b["wlcent"][i], b["flags"][i], b["ileft"][i], b["iright"][i], iwl[k],
                                      b["lincop"][i], b["linvvgt"][i], b["linavgt"][i])
        assert rel_err(got[k], ref) <= REL, k
        nz += int(np.any(ref != 0))
    assert nz > 10
    # bad points are refused
    with pytest.raises(fsg.FsgError):
        C.lineopacity1(B, wl[:1], l1[:1], np.array([n + 1], np.int32), iwl[:1], 0)
    with pytest.raises(fsg.FsgError):
        C.lineopacity1(B, wl[:1], l1[:1], l2[:1], np.array([S.nwl + 1], np.int32), 0)
    C.close()


def test_analytic_window(fsg, oracle_mod):
    from fastspec_b200 import workloads as W
    C, S, co = solar_setup(fsg, oracle_mod)
    arrays = W.atomic_lines(400, 5000.0, 5006.0, W.SEED0 + 73).arrays()
    b = block_of(oracle_mod, S, arrays)
    n = len(arrays["wl"])
    # the continuum at each line's centre wavelength, as the central pass takes it
    idx = np.clip(np.searchsorted(S.wave, b["wlcent"]), 0, S.nwl - 1)
    cont = co[idx]
    dw = C.analytic_window(b["flags"], b["lincop"], b["linvvgt"], b["linavgt"], cont)
    ref = np.array([oracle_mod.analytic_window(S, b["flags"][i], b["lincop"][i], b["linvvgt"][i], b["linavgt"][i],
                                               cont[i]) for i in range(n)])
    assert rel_err(dw, ref) <= REL
    assert np.sum(ref > 0) > n // 2
    C.close()


def zeeman_case(fsg, oracle_mod, nlines=60):
    from fastspec_b200 import workloads as W
    st, meta = H.load_atm("magnetic")
    w0, w1, step = 6000.0, 6002.0, 0.002
    grid = dict(wmode=0, wstart=w0, wend=w1, dstep=step)
    co = H.contopac_on(meta, fsg.make_grid(0, w0, w1, step) + w0)
    L = W.zeeman_lines(nlines, w0 + 0.1, w1 - 0.1, W.SEED0 + 74)
    z = W.zeeman_components(L, oracle_mod.zeeman_pattern)
    return st, grid, co, L, z


def test_mag_lineopacity1(fsg, oracle_mod):
    st, grid, co, L, z = zeeman_case(fsg, oracle_mod)
    C = fsg.Context(precision=fsg.PREC_FP64, vmicro=1.0)
    C.set_grid(0, grid["wstart"], grid["wend"], grid["dstep"])
    C.set_atmosphere(st)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0)
    arrays = L.arrays()
    b = block_of(oracle_mod, S, arrays)
    n = L.n
    # component shifts in A, scaled as MagLineopCalc scales them for a 2 kG field (Kz |B| lambda^2)
    npi, nsi, spi, rpi, ssi, rsi = z
    lam_pi = np.repeat(arrays["wl"], npi)
    lam_si = np.repeat(arrays["wl"], nsi)
    kz = 4.668644778e-13 * 2000.0
    zs = (npi, nsi, (spi * kz * lam_pi ** 2).astype(np.float32), rpi, (ssi * kz * lam_si ** 2).astype(np.float32), rsi)
    B = fsg.LineBlock(**b, zeeman=zs)
    rng = np.random.default_rng(9)
    npts = 80
    iwl = rng.integers(1, S.nwl + 1, npts).astype(np.int32)
    wl = S.wave[iwl - 1]
    got = C.mag_lineopacity1(B, wl, np.ones(npts, np.int32), np.full(npts, n, np.int32), iwl, 0)
    for k in range(npts):
        ref = oracle_mod.mag_lineopacity1(S, b, zs, wl[k], 1, n, iwl[k], 0)
        scale = np.maximum(np.abs(ref[:, :3]).max(), 1e-300)
        assert float(np.max(np.abs(got[k] - ref))) <= REL * scale, k
        assert rel_err(got[k][:, :3], ref[:, :3]) <= 1e-11
    C.close()


def test_stokes_prf_pp(fsg, oracle_mod):
    """StokesPrfPP at given wavelengths with the context's MagLineOpac (from MagLineopCalc), LineOpac
    and ContOpac, an arbitrary source function and per-angle field projections."""
    st, grid, co, L, z = zeeman_case(fsg, oracle_mod, nlines=40)
    C = fsg.Context(precision=fsg.PREC_FP64, vmicro=1.0)
    C.set_grid(0, grid["wstart"], grid["wend"], grid["dstep"])
    C.set_atmosphere(st)
    C.set_contopac(co)
    x, w, _ = fsg.mu_quadrature(1, 5)
    C.set_mu(x, w)
    g = C.mag_lineop_calc(fsg.LineList.from_arrays(L.arrays(), zeeman=z), 1, np.array([2000.0, 60.0, 30.0]))
    mlo = g["maglineopac"]
    rng = np.random.default_rng(11)
    # a LineOpac of the non-Zeeman lines (StokesPrfPP adds it to the pi and sigma absorption)
    lo = co * rng.uniform(0.0, 3.0, co.shape)
    C.lineop_set(lo)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=1.0)
    npts = 64
    iwl = rng.integers(1, S.nwl + 1, npts).astype(np.int32)
    src = 1e14 * (1.0 + rng.uniform(0, 1, (npts, S.ntau))) * np.linspace(1, 4, S.ntau)
    gam = rng.uniform(0, np.pi, 5)
    chi = rng.uniform(0, np.pi, 5)
    geo = (np.sin(gam) ** 2, np.cos(gam) ** 2, np.cos(gam), np.sin(2 * chi), np.cos(2 * chi))
    got = C.stokes_prf_pp(iwl, src, *geo)
    for k in range(npts):
        i = iwl[k] - 1
        ref = oracle_mod.stokes_prf_pp(S, mlo[i], lo[i], co[i], src[k], x, *geo)
        assert rel_err(got[k][0], ref[0]) <= 1e-10, k
        assert float(np.max(np.abs(got[k][1:] - ref[1:]) / ref[0])) <= 1e-10, k
    with pytest.raises(fsg.FsgError):
        C.stokes_prf_pp(np.array([0], np.int32), src[:1], *geo)
    C.close()
