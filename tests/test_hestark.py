"""Tabulated He I Stark broadening (hestark.f90): the host routines of the library
(fsg_hestark_tables = HeStarkInit, fsg_he_match_idx = HeMatchIdx) against the oracle's
restatement, and the oracle against the reference program's run of a hot atmosphere with
tabulated He I lines (tests/golden/pin_hot_he.npz).  No device calls."""
import os

import numpy as np

import helpers as H


def he_entries():
    """(centre, lower level energy) of the 37 tabulated lines, parsed from the library's data header."""
    import re
    src = open(os.path.join(H.REPO, "fastspec_b200", "csrc", "fsg_hestark_tables.h")).read()
    return [(float(a), float(b)) for a, b in re.findall(r"^\s*\{([0-9.]+), ([0-9.]+), [46],$", src, re.M)]


def hot_state():
    d = np.load(os.path.join(H.DATA, "atm_hot.npz"))
    st, meta = H.load_atm("hot")
    return st, meta, d["frac_hii"], d["frac_heii"]


def test_tables_equal_oracle(fsg, oracle_mod):
    """HeStarkInit bit for bit: temperatures inside the knots, on them and beyond both ends of both
    tables (extrapolation), random densities; the hot atmosphere's own state."""
    rng = np.random.default_rng(7)
    nt = 64
    T = np.concatenate([10.0 ** np.array([3.699, 4.0, 4.301, 4.477, 4.602, 4.903]),
                        [3000.0, 4000.0, 90000.0, 120000.0], rng.uniform(5000.0, 80000.0, nt - 10)])
    xne = 10.0 ** rng.uniform(10.0, 17.0, nt)
    hii = (xne * rng.uniform(0.0, 1.0, nt)).astype(np.float32)
    heii = (xne * rng.uniform(0.0, 0.2, nt)).astype(np.float32)
    hii[3] = 0.0
    st, _, hot_hii, hot_heii = hot_state()
    for args in ((T, xne, hii, heii), (st["T"], st["xne"], hot_hii, hot_heii)):
        g, h = fsg.hestark_tables(*args)
        og, oh = oracle_mod.hestark_init(*args)
        assert g.shape == (37, len(args[0]))
        assert np.array_equal(g, og) and np.array_equal(h, oh)
        assert np.all(g >= 0.0)


def test_tables_reject_bad_input(fsg):
    import pytest
    with pytest.raises(fsg.FsgError):
        fsg.hestark_tables([5000.0, -1.0], [1e12, 1e12], [1e11, 1e11], [0.0, 0.0])
    with pytest.raises(fsg.FsgError):
        fsg.hestark_tables([5000.0, 6000.0], [1e12], [1e11, 1e11], [0.0, 0.0])


def test_match_idx_edges(fsg, oracle_mod):
    """HeMatchIdx: the 1 A and 0.01 eV windows (inclusive), the first entry wins, other species and a
    context without He I give 0, WaveL rebuilt from the grid's first wavelength as XlineSetup does."""
    wl = np.array([4471.5, 4472.5, 4472.5 + 1e-9, 4470.5, 4471.5, 4471.5, 3926.53, 3926.0, 10830.0,
                   3888.7, 3888.7, 5875.7, 2829.1, 4143.76])
    elo = np.array([20.96409, 20.96409, 20.96409, 20.96409, 20.975, 20.95, 21.21802, 21.216, 19.81961,
                    19.81961, 20.96409, 20.96409, 19.81961, 21.21802], np.float32)
    spc = np.array([0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1], np.int32)
    for wfirst in (0.0, 3800.0, 4471.5):
        ihe = fsg.he_match_idx(wl, elo, spc, 0, wfirst)
        want = [oracle_mod.he_match_idx((w - wfirst) + wfirst, float(e)) if s == 0 else 0
                for w, e, s in zip(wl, elo, spc)]
        assert ihe.tolist() == want
    assert ihe.tolist() == [19, 19, 0, 19, 0, 0, 35, 35, 32, 10, 0, 24, 1, 0]
    assert not np.any(fsg.he_match_idx(wl, elo, spc, -1))
    assert len(fsg.he_match_idx(np.zeros(0), np.zeros(0, np.float32), np.zeros(0, np.int32), 0)) == 0


def test_oracle_hot_he_pin_reference(fsg, oracle_mod):
    """The reference program's line opacity, windows and spectra for tabulated He I lines of both
    tables (with near misses in wavelength and energy) in a Teff 15000 K atmosphere: the oracle with
    HeStarkInit from the recovered H II / He II densities and the table match of XlineSetup."""
    d = H.load_pin("pin_hot_he")
    grid, st, meta, co = H.pin_setup(d)
    _, _, hii, heii = hot_state()
    g, h = fsg.hestark_tables(st["T"], st["xne"], hii, heii)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]),
                         hegam=g, heshf=h, spc_he1=0)
    lines = H.pin_lines(d)
    assert np.array_equal(fsg.he_match_idx(lines["wl"], lines["elo"], lines["spc"], 0, grid["wstart"]),
                          d["ihe_expected"])
    assert int((d["ihe_expected"] > 0).sum()) == 7
    r = oracle_mod.lineop_calc(S, oracle_mod.Lines(**lines, kind=2), list_type=2)
    assert np.array_equal((r["flags"] >> 8) & 255, d["ihe_expected"])
    lo, ref = r["lineopac"], d["lineopac"]
    assert np.array_equal(lo > 0, ref > 0)
    m = ref > 0
    assert np.max(np.abs(lo[m] / ref[m] - 1)) < 1e-10
    spl, spc = oracle_mod.radtran(S, d["xmu"], lo)
    # intensities as in the other reference pins (1e-9 level: the hot model's Planck terms and exp)
    assert np.max(np.abs(spl / d["spl"] - 1)) < 1e-8
    assert np.max(np.abs(spc / d["spc"] - 1)) < 1e-8
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    sfl, sfc = oracle_mod.disk_integ(w, spl, spc)
    assert np.max(np.abs(sfl / d["sfl"] - 1)) < 1e-8
    # the tabulated widths matter: without the table the same lines differ at the percent level
    S0 = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    r0 = oracle_mod.lineop_calc(S0, oracle_mod.Lines(**lines, kind=2), list_type=2)
    assert np.max(np.abs(r0["lineopac"] - ref)) > 1e-2 * np.max(ref)


def test_oracle_hot_he_magnetic_pin_reference(fsg, oracle_mod):
    """The same He I list as Zeeman lines (explicit patterns) in a 3 kG field, BFRAME 1, 9 angles: the
    oracle's MagLineopCalc + MagRadTranCalc with the tabulated widths and shifts against the reference's
    Stokes IQUV (tests/golden/pin_hot_he_mag.npz); I and Ic relative, Q, U, V relative to Ic."""
    d = H.load_pin("pin_hot_he_mag")
    grid, st, co, lines, z = H.mag_pin_setup(d)
    _, _, hii, heii = hot_state()
    g, h = fsg.hestark_tables(st["T"], st["xne"], hii, heii)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]),
                         hegam=g, heshf=h, spc_he1=0)
    bframe, bfield = int(d["bframe"]), d["bfield"]
    r = oracle_mod.mag_lineop_calc(S, oracle_mod.Lines(**lines, kind=2, zeeman=z), bframe, bfield)
    assert int((((r["flags"] >> 8) & 255) > 0).sum()) == 7
    spz, spc = oracle_mod.mag_radtran(S, d["xmu"], bframe, bfield, np.zeros((S.nwl, S.ntau)), r["maglineopac"])
    ref, ic = d["spz"], d["spc"]
    assert np.max(np.abs(spz[:, 0] / ref[:, 0] - 1)) < 1e-8
    assert np.max(np.abs(spc / ic - 1)) < 1e-8
    for q in (1, 2, 3):
        assert np.max(np.abs(spz[:, q] - ref[:, q]) / ic) < 1e-8
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    sfl, _ = oracle_mod.disk_integ(w, spz[:, 0], spc)
    assert np.max(np.abs(sfl / d["sfl"] - 1)) < 1e-8


def test_line_list_table_match_column(fsg):
    """Context.lineop_calc after hestark_init passes a copy of the list with the ihe column of
    fsg_he_match_idx (host logic; the caller's list keeps no column, an explicit column wins)."""
    d = H.load_pin("pin_hot_he")
    a = H.pin_lines(d)
    L = fsg.LineList.from_arrays(a)
    M = L._with_he_match(0, 3855.0)
    assert not L.c.ihe and M.c.ihe and M.n == L.n
    got = np.ctypeslib.as_array(M.c.ihe, shape=(M.n,))
    assert np.array_equal(got, d["ihe_expected"])
    assert M._keep["wl"] is L._keep["wl"]                       # the other columns are shared, not copied
    E = fsg.LineList.from_arrays(dict(a, ihe=np.zeros(len(a["wl"]), np.int32)))
    assert E._with_he_match(0, 3855.0) is E


def test_match_idx_random_lines_equal_oracle(fsg, oracle_mod):
    """HeMatchIdx over 50,000 seeded He I lines scattered around every table entry (within +-1.5 A and
    +-0.02 eV, so both edges of both windows are crossed): the library equals the oracle line by line."""
    HE_ENTRIES = he_entries()
    rng = np.random.default_rng(17)
    n = 50_000
    k = rng.integers(0, len(HE_ENTRIES), n)
    wl = np.array([HE_ENTRIES[i][0] for i in k]) + rng.uniform(-1.5, 1.5, n)
    elo = (np.array([HE_ENTRIES[i][1] for i in k]) + rng.uniform(-0.02, 0.02, n)).astype(np.float32)
    spc = np.zeros(n, np.int32)
    wfirst = 2000.0
    got = fsg.he_match_idx(wl, elo, spc, 0, wfirst)
    want = np.array([oracle_mod.he_match_idx((w - wfirst) + wfirst, float(e)) for w, e in zip(wl, elo)])
    assert np.array_equal(got, want)
    assert 0.2 < np.mean(got > 0) < 0.8
