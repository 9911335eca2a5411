"""The fs_*.bin readers and writers (fastspec_b200/fsio.py; the reference's WriteOut / WriteLinStr,
ioutils.f90:1751-1875): files the reference program wrote (tests/golden/fs_outputs.npz, made by
tests/golden/make_bin_golden.py) are read and written back byte for byte."""
import os

import numpy as np
import pytest

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


def test_opacity_reentry_pin_reference(oracle_mod, tmp_path):
    """OPACITY= re-entry: the reference program read a file that fsio.write_opac wrote (the oracle's line
    opacity of list A on the pin_solar grid) and added list B (tests/golden/pin_solar_reentry.npz).  The
    same steps here: the oracle's A, written and read back through fsio, then B accumulated onto it."""
    from fastspec_b200 import fsio
    d = H.load_pin("pin_solar_reentry")
    grid, st, meta, co = H.pin_setup(d)
    S = oracle_mod.State(grid, st, contopac=co, vmicro=float(d["vmicro"]), molbrd=int(d["molbrd"]))
    A = {k[2:]: d[k] for k in d if k.startswith("a_")}
    ra = oracle_mod.lineop_calc(S, oracle_mod.Lines(**A, kind=2), list_type=2)
    p = str(tmp_path / "opac_a.bin")
    wave = S.wave + S.wfirst
    fsio.write_opac(p, wave, ra["lineopac"], st["rhox"], st["T"], st["xne"], st["xna"], st["rho"])
    back = fsio.read_opac(p)
    assert np.array_equal(back["opac"], ra["lineopac"]) and np.array_equal(back["wave"], wave)
    rb = oracle_mod.lineop_calc(S, oracle_mod.Lines(**H.pin_lines(d), kind=2), list_type=2,
                                lineopac=back["opac"].copy())
    i0, i1 = int(d["i0"]), int(d["i1"])
    lo, ref = rb["lineopac"][i0:i1 + 1], d["lineopac"]
    assert np.array_equal(lo > 0, ref > 0)
    m = ref > 0
    assert np.max(np.abs(lo[m] / ref[m] - 1)) < 1e-8


CONV = {"conv_a": ("spec", 15.0, 3.0, 60000.0), "conv_b": ("spec_mag", 5.0, 0.0, 2.5)}


def test_post_processing_mode_oracle(fsg, oracle_mod, tmp_path):
    """The reference's post-processing mode (fastspec <fs_spec.bin> Vsini Vmacro Vgau,
    fastspec.f90:75-134) on two of its intensity files: ReadSpec's grid and angle order (fsio.spec_grid),
    the quadrature from the angles (mu_quad_type) and the oracle's broadened disk integration give the
    reference's fs_flux.bin."""
    from fastspec_b200 import fsio
    g = golden()
    for key, (spec, vs, vm, vg) in CONV.items():
        s = fsio.spec_grid(fsio.read_spec(put(tmp_path, spec + ".bin", g[spec])))
        assert s["wmode"] == 0 and list(s["xmu"]) == sorted(s["xmu"], reverse=True)
        assert fsg.mu_quad_type(s["xmu"]) == 1
        x, w, r = fsg.mu_quadrature(1, len(s["xmu"]), x=s["xmu"])
        grid = dict(wmode=s["wmode"], wstart=s["wstart"], wend=s["wend"], dstep=s["dstep"])
        wave = s["wave"] + s["wstart"]
        sfl, sfc = oracle_mod.disk_integ_conv(x, w, r, s["spl"], s["spc"], oracle_mod.grid_dv(grid, wave), vs, vm,
                                              oracle_mod.gauss_sigma_pix(grid, wave, vg))
        ref = fsio.read_flux(put(tmp_path, key + ".bin", g[key]))
        assert np.array_equal(ref["wave"], wave)
        assert np.max(np.abs(sfl / ref["sfl"] - 1)) < 1e-12
        assert np.max(np.abs(sfc / ref["sfc"] - 1)) < 1e-12


def test_spec_grid_orders_angles_and_detects_log_grids():
    from fastspec_b200 import fsio
    wave = 5000.0 * np.exp(np.arange(6) * 1e-5)
    spl = np.arange(18, dtype=float).reshape(6, 3)
    s = fsio.spec_grid(dict(xmu=np.array([0.2, 0.9, 0.5]), wave=wave, spl=spl, spc=spl + 100))
    assert s["wmode"] == 1 and abs(s["dstep"] - 1e-5 * 299792.458) < 1e-6
    assert list(s["xmu"]) == [0.9, 0.5, 0.2] and list(s["spl"][0]) == [1.0, 2.0, 0.0]
    u = fsio.spec_grid(dict(xmu=np.array([1.0]), wave=5000.0 + 0.01 * np.arange(4), spl=np.zeros((4, 1)),
                            spc=np.ones((4, 1))))
    assert u["wmode"] == 0 and abs(u["dstep"] - 0.01) < 1e-12


REF_BIN = os.path.join(H.REFERENCE, "src", "fastspec_Linux_x86_64")
MAG_EXAMPLE = os.path.join(H.REFERENCE, "examples", "magnetic-synthesis", "fs_spec.bin")


@pytest.mark.skipif(not (os.path.exists(REF_BIN) and os.path.exists(MAG_EXAMPLE)),
                    reason="the reference program and its examples are not present")
def test_post_processing_of_the_shipped_magnetic_example(fsg, oracle_mod, tmp_path):
    """The post-processing mode on the reference's own shipped Stokes intensities (examples/
    magnetic-synthesis/fs_spec.bin: 7 angles, 39,194 wavelengths): the reference program run here on
    that file against fsio.spec_grid + mu_quad_type + the oracle's broadened disk integration."""
    import shutil
    import subprocess
    from fastspec_b200 import fsio
    shutil.copy(MAG_EXAMPLE, str(tmp_path / "fs_spec.bin"))
    vs, vm, vg = 12.0, 4.0, 80000.0
    r = subprocess.run([REF_BIN, "fs_spec.bin", "%g" % vs, "%g" % vm, "%g" % vg], cwd=str(tmp_path),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    ref = fsio.read_flux(str(tmp_path / "fs_flux.bin"))
    s = fsio.spec_grid(fsio.read_spec(MAG_EXAMPLE))
    q = fsg.mu_quad_type(s["xmu"])
    x, w, rr = fsg.mu_quadrature(q, len(s["xmu"]), x=s["xmu"])
    grid = dict(wmode=s["wmode"], wstart=s["wstart"], wend=s["wend"], dstep=s["dstep"])
    wave = s["wave"] + s["wstart"]
    sfl, sfc = oracle_mod.disk_integ_conv(x, w, rr, s["spl"], s["spc"], oracle_mod.grid_dv(grid, wave), vs, vm,
                                          oracle_mod.gauss_sigma_pix(grid, wave, vg))
    assert np.array_equal(ref["wave"], wave) and len(wave) > 30000
    assert np.max(np.abs(sfl / ref["sfl"] - 1)) < 1e-12
    assert np.max(np.abs(sfc / ref["sfc"] - 1)) < 1e-12


EXAMPLES = os.path.join(H.REFERENCE, "examples")


@pytest.mark.skipif(not os.path.isdir(EXAMPLES), reason="the reference's examples are not present")
def test_shipped_example_outputs_round_trip(tmp_path):
    """The reference's shipped outputs (examples/*-synthesis: the atomic flux and line strengths of
    44,380 lines, the molecular flux, the magnetic Stokes intensities) read and written back byte for
    byte."""
    from fastspec_b200 import fsio
    for sub, name in (("atomic-synthesis", "fs_flux.bin"), ("molecular-synthesis", "fs_flux.bin"),
                      ("atomic-synthesis", "fs_linst.bin"), ("magnetic-synthesis", "fs_spec.bin")):
        src = os.path.join(EXAMPLES, sub, name)
        raw = open(src, "rb").read()
        out = str(tmp_path / (sub + "_" + name))
        if name == "fs_flux.bin":
            f = fsio.read_flux(src)
            fsio.write_flux(out, f["wave"], f["sfl"], f["sfc"])
        elif name == "fs_spec.bin":
            r = fsio.read_spec(src)
            assert r["magnetic"] and len(r["xmu"]) == 7
            fsio.write_spec(out, r["wave"], r["xmu"], r["spl"], r["spc"], r["spz"])
        else:
            r = fsio.read_linst(src)
            assert len(r["wave"]) > 40000
            a = 0
            for k, n in enumerate(r["nrec"]):
                sl = slice(a, a + n)
                fsio.write_linst(out, r["species"][sl], r["ion"][sl], r["wave"][sl], r["strength"][sl], append=k > 0)
                a += n
        assert open(out, "rb").read() == raw, src
