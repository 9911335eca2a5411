"""The fs_*.bin readers and writers (fastspec_b200/fsio.py; the reference's WriteOut / WriteLinStr,
ioutils.f90:1751-1875): files the reference program wrote (tests/golden/fs_outputs.npz, made by
tests/golden/make_bin_golden.py) are read and written back byte for byte."""
import os

import numpy as np

import helpers as H


def golden():
    d = np.load(os.path.join(H.GOLD, "fs_outputs.npz"))
    return {k: d[k].tobytes() for k in d.files}


def put(tmp_path, name, data):
    p = str(tmp_path / name)
    with open(p, "wb") as f:
        f.write(data)
    return p


def test_opacity_files_round_trip(tmp_path):
    from fastspec_b200 import fsio
    g = golden()
    for key in ("lineop", "contop"):
        r = fsio.read_opac(put(tmp_path, key + ".bin", g[key]))
        assert r["opac"].shape == (51, 56) and np.all(r["opac"] >= 0)
        assert abs(r["wave"][0] - 5000.0) < 1e-9 and abs(r["wave"][-1] - 5001.0) < 1e-9
        out = str(tmp_path / (key + "_w.bin"))
        fsio.write_opac(out, r["wave"], r["opac"], r["rhox"], r["T"], r["xne"], r["xna"], r["rho"])
        assert open(out, "rb").read() == g[key]
    assert np.any(fsio.read_opac(put(tmp_path, "l.bin", g["lineop"]))["opac"] > 0)


def test_spectrum_and_flux_files_round_trip(tmp_path):
    from fastspec_b200 import fsio
    g = golden()
    for spec, flux, magnetic in (("spec", "flux", False), ("spec_mag", "flux_mag", True)):
        r = fsio.read_spec(put(tmp_path, spec + ".bin", g[spec]))
        assert r["magnetic"] == magnetic and r["spl"].shape == (51, 3) and len(r["xmu"]) == 3
        out = str(tmp_path / (spec + "_w.bin"))
        fsio.write_spec(out, r["wave"], r["xmu"], r["spl"], r["spc"], r.get("spz"))
        assert open(out, "rb").read() == g[spec]
        if magnetic:
            assert np.max(np.abs(r["spz"][:, 3])) > 0          # Stokes V of the Zeeman lines
        f = fsio.read_flux(put(tmp_path, flux + ".bin", g[flux]))
        assert np.array_equal(f["wave"], r["wave"]) and np.all(f["sfl"] <= f["sfc"] * (1 + 1e-12))
        out = str(tmp_path / (flux + "_w.bin"))
        fsio.write_flux(out, f["wave"], f["sfl"], f["sfc"])
        assert open(out, "rb").read() == g[flux]


def test_line_strength_file_round_trip(tmp_path):
    from fastspec_b200 import fsio
    g = golden()
    r = fsio.read_linst(put(tmp_path, "linst.bin", g["linst"]))
    assert r["nrec"].tolist() == [12, 7]                            # one record block per line list
    assert np.all((r["strength"] >= 0) & (r["strength"] <= 1))
    out = str(tmp_path / "linst_w.bin")
    a = 0
    for k, n in enumerate(r["nrec"]):
        sl = slice(a, a + n)
        fsio.write_linst(out, r["species"][sl], r["ion"][sl], r["wave"][sl], r["strength"][sl], append=k > 0)
        a += n
    assert open(out, "rb").read() == g["linst"]
