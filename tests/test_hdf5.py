"""Line lists in the reference's HDF5 layout (fastspec_b200/hdf5.py, fsio.read_hdf5_lines /
write_hdf5_lines), on the CPU.

* The reader against the reference's own example lists (examples/lines/*.h5, written by its h5py
  converters: chunked, shuffled, gzip-compressed columns): the first 300 records equal the values
  parsed from the text sources the reference converted (tests/golden/hdf5_examples.npz, made by
  tests/golden/make_hdf5_golden.py).  Skipped where the reference tree is absent.
* The writer: round trip, and the pin of the reference program reading a written file
  (tests/golden/pin_solar_h5.npz, tests/golden/make_atmospheres.py h5): the oracle's atomic-list
  path on the list read back gives the reference's line opacity and spectra.
"""
import os

import numpy as np
import pytest

import helpers as H

EXAMPLES = os.path.join(H.REFERENCE, "examples", "lines")


def _golden():
    return np.load(os.path.join(H.GOLD, "hdf5_examples.npz"))


@pytest.mark.skipif(not os.path.isdir(EXAMPLES), reason="reference example line lists not present")
@pytest.mark.parametrize("name", ["VALD_all_500-600.h5", "VALD_all_500-600.zh5"])
def test_reader_atomic_lists_match_text_source(name):
    from fastspec_b200 import hdf5
    g = _golden()
    cols, attrs, units = hdf5.read_lines(os.path.join(EXAMPLES, name))
    n = len(g["vald_w"])
    assert attrs["NL"] == len(cols["W"]) == 136370 and attrs["NAME"].startswith("atom")
    assert attrs["WMIN"] == cols["W"][0] and attrs["WMAX"] == cols["W"][-1]
    assert np.all(np.diff(cols["W"]) >= 0)
    assert np.array_equal(cols["EL"][:n], g["vald_el"]) and np.array_equal(cols["ION"][:n], g["vald_ion"])
    assert np.array_equal(cols["W"][:n], g["vald_w"])
    for k in ("LGGF", "E", "GRAD", "GQST", "GVDW"):
        assert np.array_equal(cols[k][:n], g["vald_" + k.lower()]), k
    if name.endswith(".zh5"):
        assert np.array_equal(cols["JLO"][:n], g["vald_jlo"]) and np.array_equal(cols["JUP"][:n], g["vald_jup"])
        for k in ("GLO", "GUP"):          # the converter fills unknown factors and flags forbidden lines
            t, h = g["vald_" + k.lower()], cols[k][:n]
            known = (t != 99.0) & (h != 99.0)
            assert known.sum() > 250 and np.array_equal(t[known], h[known])
    assert units["W"].startswith("Angstrom")


@pytest.mark.skipif(not os.path.isdir(EXAMPLES), reason="reference example line lists not present")
def test_reader_molecular_list_matches_text_source():
    from fastspec_b200 import hdf5, fsio
    g = _golden()
    cols, attrs, units = hdf5.read_lines(os.path.join(EXAMPLES, "56Fe1H_Exomol_Irw.h5"))
    n = len(g["feh_w"])
    assert attrs["NAME"] == "FeH" and attrs["ION"] == 1 and attrs["WL_VAC"] == 1
    assert np.max(np.abs(cols["W"][:n] - g["feh_w"])) < 1e-9
    for k in ("E", "LGGF", "GU", "GRAD"):
        assert np.array_equal(cols[k][:n], g["feh_" + k.lower()]), k
    r = fsio.read_hdf5_lines(os.path.join(EXAMPLES, "56Fe1H_Exomol_Irw.h5"), [("FeH", 1)], exact=False)
    assert r["kind"] == 1 and np.all(r["spc"] == 0) and np.all(r["ismol"] == 1)
    assert np.array_equal(r["wl"], fsio.vac2air(cols["W"]))        # WL_VAC = 1: air wavelengths, as ReadHDF
    assert np.all(r["wl"] < cols["W"])
    assert np.array_equal(r["grad"], cols["GRAD"])               # molecular GRAD is taken as stored
    assert np.allclose(r["gf"], 10.0 ** cols["LGGF"].astype(np.float64), rtol=1e-6)


def test_writer_round_trip(tmp_path):
    from fastspec_b200 import fsio, hdf5, workloads as W
    L = W.zeeman_lines(50, 6000.0, 6005.0, W.SEED0 + 7)
    t = L._txt
    p = str(tmp_path / "z.zh5")
    f = lambda k, fmt: W.f32_of_text(t[k], fmt)
    fsio.write_hdf5_lines(p, L.species, L.spc, L.wl, f("elo", "%.4f"), f("loggf", "%.3f"), f("lgrad", "%.3f"),
                          f("lgqst", "%.3f"), f("lgvdw", "%.3f"), zeeman=L.zeeman, provenance="round trip")
    cols, attrs, units = hdf5.read_lines(p)
    assert attrs["NL"] == L.n and attrs["NAME"] == "atom Zeeman" and attrs["FORMAT_VERSION"] == "z-1.0"
    assert attrs["PROVENANCE"] == "round trip" and attrs["WMIN"] == L.wl[0] and attrs["WMAX"] == L.wl[-1]
    assert np.array_equal(cols["W"], L.wl)
    r = fsio.read_hdf5_lines(p, L.species)
    for k in ("wl", "elo", "gf", "grad", "gqst", "gvdw", "spc"):
        assert np.array_equal(r[k], getattr(L, k)), k
    for q, k in enumerate(("jlo", "jup", "glo", "gup")):
        assert np.array_equal(r[k], np.asarray(L.zeeman[q], np.float32)), k
    # a species missing from the caller's table is marked -1; an empty list round-trips
    r2 = fsio.read_hdf5_lines(p, L.species[:1])
    assert np.all((r2["spc"] == 0) | (r2["spc"] == -1)) and np.any(r2["spc"] == -1)
    e = str(tmp_path / "e.h5")
    fsio.write_hdf5_lines(e, L.species, [], [], [], [], [], [], [])
    ce, ae, _ = hdf5.read_lines(e)
    assert ae["NL"] == 0 and len(ce["W"]) == 0
    with pytest.raises(hdf5.HDF5Error):
        bad = tmp_path / "bad.h5"
        bad.write_bytes(b"not an hdf5 file at all")
        hdf5.read_lines(str(bad))
    with pytest.raises(ValueError):
        fsio.write_hdf5_lines(e, L.species, L.spc[::-1], L.wl[::-1], *(np.zeros(L.n),) * 5)


def hdf5_pin_lines(tmp_path):
    """The pin_solar_h5 list written to an HDF5 file and read back as SoA records (atomic list)."""
    from fastspec_b200 import fsio, workloads as W
    d = H.load_pin("pin_solar_h5")
    st, meta = H.load_atm("solar")
    species = [(s.split()[0], int(s.split()[1])) for s in meta["species"]]
    p = str(tmp_path / "lines.h5")
    f = lambda k, fmt: W.f32_of_text(d["txt_" + k], fmt)
    fsio.write_hdf5_lines(p, species, d["line_spc"], d["line_wl"], f("elo", "%.4f"), f("loggf", "%.3f"),
                          f("lgrad", "%.3f"), f("lgqst", "%.3f"), f("lgvdw", "%.3f"))
    return d, fsio.read_hdf5_lines(p, species)


def test_oracle_hdf5_list_against_reference_pin(oracle_mod, tmp_path):
    """The reference read the same written file as an atomic HDF5 list (LineTypeAtm records, wide lines
    taken out of blocking): the oracle's atomic-list path on the records read back reproduces its line
    opacity (windows identical) and spectra."""
    d, r = hdf5_pin_lines(tmp_path)
    grid, st, meta, co = H.pin_setup(d)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    L = oracle_mod.Lines(**{k: r[k] for k in ("wl", "elo", "gf", "grad", "gqst", "gvdw", "spc", "ismol")}, kind=0)
    o = oracle_mod.lineop_calc(S, L, list_type=0)
    i0, i1 = int(d["i0"]), int(d["i1"])
    lo, ref = o["lineopac"][i0:i1 + 1], d["lineopac"]
    assert np.array_equal(lo > 0, ref > 0)
    assert np.max(np.abs(lo[ref > 0] / ref[ref > 0] - 1)) < 1e-8
    assert o["stats"]["nwide"] > 0                              # the atomic path's wide lines were exercised
    spl, spc = oracle_mod.radtran(S, d["xmu"], o["lineopac"])
    assert np.max(np.abs(spl[i0:i1 + 1] / d["spl"] - 1)) < 1e-8
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    sfl, _ = oracle_mod.disk_integ(w, spl[i0:i1 + 1], spc[i0:i1 + 1])
    assert np.max(np.abs(sfl / d["sfl"] - 1)) < 1e-8


def test_oracle_vacuum_list_and_range_selection_against_reference_pin(oracle_mod, tmp_path):
    """A list written in vacuum wavelengths (WL_VAC = 1) with lines beyond both ends of WAVE=: read as
    ReadHDF reads it (Vac2Air, then only wstart <= W <= wend), the records give the reference's line
    opacity for the same file (tests/golden/pin_solar_h5vac.npz); the lines above the range would
    change the region if they were kept."""
    from fastspec_b200 import fsio, workloads as W
    d = H.load_pin("pin_solar_h5vac")
    st, meta = H.load_atm("solar")
    species = [(s.split()[0], int(s.split()[1])) for s in meta["species"]]
    p = str(tmp_path / "lines.h5")
    f = lambda k, fmt: W.f32_of_text(d["txt_" + k], fmt)
    fsio.write_hdf5_lines(p, species, d["line_spc"], d["line_wvac"], f("elo", "%.4f"), f("loggf", "%.3f"),
                          f("lgrad", "%.3f"), f("lgqst", "%.3f"), f("lgvdw", "%.3f"), wl_vac=1)
    grid, st, meta, co = H.pin_setup(d)
    r = fsio.read_hdf5_lines(p, species, wstart=grid["wstart"], wend=grid["wend"])
    assert len(r["wl"]) == int(d["nread"]) < len(d["line_wvac"])
    assert np.all((r["wl"] >= grid["wstart"]) & (r["wl"] <= grid["wend"]))
    wa = fsio.vac2air(d["line_wvac"])
    assert np.array_equal(r["wl"], wa[(wa >= grid["wstart"]) & (wa <= grid["wend"])])
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    keys = ("wl", "elo", "gf", "grad", "gqst", "gvdw", "spc", "ismol")
    o = oracle_mod.lineop_calc(S, oracle_mod.Lines(**{k: r[k] for k in keys}, kind=0), list_type=0)
    i0, i1 = int(d["i0"]), int(d["i1"])
    lo, ref = o["lineopac"][i0:i1 + 1], d["lineopac"]
    assert np.array_equal(lo > 0, ref > 0)
    assert np.max(np.abs(lo[ref > 0] / ref[ref > 0] - 1)) < 1e-8
    spl, spc = oracle_mod.radtran(S, d["xmu"], o["lineopac"])
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    sfl, _ = oracle_mod.disk_integ(w, spl[i0:i1 + 1], spc[i0:i1 + 1])
    assert np.max(np.abs(sfl / d["sfl"] - 1)) < 1e-8
    full = fsio.read_hdf5_lines(p, species)                       # no range: the outside lines stay
    o2 = oracle_mod.lineop_calc(S, oracle_mod.Lines(**{k: full[k] for k in keys}, kind=0), list_type=0)
    m = ref > 0
    assert np.max(np.abs(o2["lineopac"][i0:i1 + 1][m] / ref[m] - 1)) > 1e-4


def test_reader_rejects_unsorted_and_hydrogen_lists(tmp_path):
    """ReadHDF stops on an unsorted wavelength column; a dedicated hydrogen list (HFLAG = 1) belongs to
    the hydrogen line opacity, which is not part of this library."""
    from fastspec_b200 import fsio, hdf5
    import pytest
    p = str(tmp_path / "u.h5")
    fsio.write_hdf5_lines(p, [("Fe", 1)], [0, 0], [5000.0, 5001.0], [1.0, 1.0], [-1.0, -1.0], [8.0, 8.0],
                          [-5.0, -5.0], [-7.5, -7.5])
    cols, attrs, units = hdf5.read_lines(p)
    cols["W"] = cols["W"][::-1].copy()
    hdf5.write_lines(p, cols, attrs, units)
    with pytest.raises(ValueError, match="not sorted"):
        fsio.read_hdf5_lines(p, [("Fe", 1)])
    cols["W"] = cols["W"][::-1].copy()
    attrs["HFLAG"] = np.int16(1)
    hdf5.write_lines(p, cols, attrs, units)
    with pytest.raises(ValueError, match="hydrogen line list"):
        fsio.read_hdf5_lines(p, [("Fe", 1)])


def zh5_pin_lines(tmp_path, pattern):
    """pin_magnetic_zh5's seeded lines written as a Zeeman HDF5 list and read back: records and the
    CSR Zeeman components built from the J and Lande factor columns with `pattern`."""
    from fastspec_b200 import fsio, workloads as W
    d = H.load_pin("pin_magnetic_zh5")
    st, meta = H.load_atm("magnetic")
    species = [(s.split()[0], int(s.split()[1])) for s in meta["species"]]
    p = str(tmp_path / "lines.zh5")
    f = lambda k, fmt: W.f32_of_text(d["txt_" + k], fmt)
    fsio.write_hdf5_lines(p, species, d["line_spc"], d["line_wl"], f("elo", "%.4f"), f("loggf", "%.3f"),
                          f("lgrad", "%.3f"), f("lgqst", "%.3f"), f("lgvdw", "%.3f"),
                          zeeman=(d["jlo"], d["jup"], d["glo"], d["gup"]))
    r = fsio.read_hdf5_lines(p, species)
    return d, r, fsio.hdf5_zeeman_components(r, pattern)


def test_oracle_zh5_list_against_reference_pin(oracle_mod, tmp_path):
    """A Zeeman HDF5 list (the reference derives each line's splitting from J and the Lande factors; a
    factor of 99 marks an unsplit line): the oracle's magnetic path on the records and components read
    back reproduces the reference's Stokes IQUV for the same file (1e-8 of Ic)."""
    d, r, z = zh5_pin_lines(tmp_path, oracle_mod.zeeman_pattern)
    assert r["kind"] == 2 and np.sum(z[0] == 1) >= 3
    grid, st, meta, co = H.pin_setup(d)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    L = oracle_mod.Lines(**{k: r[k] for k in ("wl", "elo", "gf", "grad", "gqst", "gvdw", "spc", "ismol")},
                         kind=2, zeeman=z)
    o = oracle_mod.mag_lineop_calc(S, L, int(d["bframe"]), d["bfield"])
    spz, spc = oracle_mod.mag_radtran(S, d["xmu"], int(d["bframe"]), d["bfield"], np.zeros((S.nwl, S.ntau)),
                                      o["maglineopac"])
    i0, i1 = int(d["i0"]), int(d["i1"])
    ref, ic = d["spz"], d["spc"]
    for q in range(4):
        assert np.max(np.abs(spz[i0:i1 + 1, q] - ref[:, q]) / ic) < 1e-8
    x, w, _ = oracle_mod.mu_quadrature(1, len(d["xmu"]))
    sfl, _ = oracle_mod.disk_integ(w, spz[i0:i1 + 1, 0], spc[i0:i1 + 1])
    assert np.max(np.abs(sfl / d["sfl"] - 1)) < 1e-8


def mol_h5_pin_lists(tmp_path):
    """pin_cooldwarf_h5's seeded lines written as four single-species molecular HDF5 lists and read
    back, in the deck's order (one record dict per list)."""
    from fastspec_b200 import fsio, workloads as W
    d = H.load_pin("pin_cooldwarf_h5")
    st, meta = H.load_atm("cooldwarf")
    species = [(s.split()[0], int(s.split()[1])) for s in meta["species"]]
    f = lambda k, fmt, sel: W.f32_of_text(d["txt_" + k][sel], fmt)
    lists = []
    for k, (nm, ion) in enumerate(species):
        sel = d["line_spc"] == k
        p = str(tmp_path / ("%s.h5" % nm.lower()))
        fsio.write_hdf5_molecular(p, nm, ion, "0000.000000", d["line_wl"][sel], f("elo", "%.4f", sel),
                                  f("loggf", "%.3f", sel), np.zeros(int(sel.sum()), np.float32))
        lists.append(fsio.read_hdf5_lines(p, species))
    return d, lists


def test_oracle_molecular_h5_lists_against_reference_pin(oracle_mod, tmp_path):
    """Four single-species molecular HDF5 lists (LineTypeMol records: no Stark or van der Waals
    parameters, classical radiative damping) read by the reference program one after the other: the
    oracle's molecular-list path on the records read back reproduces its line opacity and spectra.
    Windows and line counts are identical; the values agree to 2e-7 (median 1e-9): the few larger
    differences are those of a one-ulp change of a line's FP32 gf (the reference's molecular reader
    takes 10.0**LGGF as a whole-array power, ioutils.f90:813, the other readers line by line)."""
    d, lists = mol_h5_pin_lists(tmp_path)
    grid, st, meta, co = H.pin_setup(d)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    lo = np.zeros((S.nwl, S.ntau))
    for r in lists:
        assert r["kind"] == 1 and np.all(r["ismol"] == 1) and np.all(r["spc"] >= 0)
        L = oracle_mod.Lines(**{k: r[k] for k in ("wl", "elo", "gf", "grad", "gqst", "gvdw", "spc", "ismol")},
                             kind=1)
        oracle_mod.lineop_calc(S, L, list_type=1, lineopac=lo)
    i0, i1 = int(d["i0"]), int(d["i1"])
    ref = d["lineopac"]
    assert np.array_equal(lo[i0:i1 + 1] > 0, ref > 0)
    rel = np.abs(lo[i0:i1 + 1][ref > 0] / ref[ref > 0] - 1)
    assert rel.max() < 2e-7 and np.median(rel) < 1e-8
    spl, spc = oracle_mod.radtran(S, d["xmu"], lo)
    assert np.max(np.abs(spl[i0:i1 + 1] / d["spl"] - 1)) < 2e-7


@pytest.mark.skipif(not os.path.isdir(EXAMPLES), reason="reference example line lists not present")
def test_reader_refuses_the_shipped_hydrogen_list():
    """VALD_H1_10-10000.h5 is the reference's dedicated hydrogen list (HFLAG = 1): it feeds the
    hydrogen line opacity, not this library."""
    from fastspec_b200 import fsio, hdf5
    cols, attrs, units = hdf5.read_lines(os.path.join(EXAMPLES, "VALD_H1_10-10000.h5"))
    assert int(attrs["HFLAG"]) == 1 and np.all(np.char.strip(np.asarray(cols["EL"]).astype("U8")) == "H")
    with pytest.raises(ValueError, match="hydrogen line list"):
        fsio.read_hdf5_lines(os.path.join(EXAMPLES, "VALD_H1_10-10000.h5"), [("Fe", 1)])
