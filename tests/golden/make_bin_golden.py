#!/usr/bin/env python3
"""Raw output files of the reference program for the fs_*.bin reader/writer round trips.

Runs the reference's shipped executable (this container only) on two tiny decks with the solar
model: (1) two ASCII line lists, SAVE=1,1,1,1,1 (line and continuum opacity, intensities, flux and
the line strengths of both lists); (2) a Zeeman list in a 2 kG field, SAVE=0,0,1,1,1 (Stokes
intensities and flux); and the post-processing mode (fastspec <fs_spec.bin> Vsini Vmacro Vgau) on
each intensity file (broadened flux).  The files' bytes go to tests/golden/fs_outputs.npz, which is committed.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
from fastspec_b200 import workloads as W  # noqa: E402

BIN = os.path.join(os.environ.get("FASTSPEC_REFERENCE", ""), "src", "fastspec_Linux_x86_64")
OUT = os.path.join(HERE, "fs_outputs.npz")
# post-processing runs (Vsini, Vmacro, Vgau) on the two intensity files: a resolving power, a FWHM
CONV = {"conv_a": (15.0, 3.0, 60000.0), "conv_b": (5.0, 0.0, 2.5)}


def run(wd, deck):
    with open(os.path.join(wd, "in.dat"), "w") as f:
        f.write(deck)
    r = subprocess.run([BIN, "in.dat"], cwd=wd, capture_output=True, text=True)
    if r.returncode != 0 or "Total time" not in r.stdout:
        raise RuntimeError(r.stdout + r.stderr)


def convolve(wd, spec, vsini, vmacro, vgau):
    """The post-processing mode: fastspec <intensity file> Vsini Vmacro Vgau -> fs_flux.bin."""
    r = subprocess.run([BIN, spec, "%g" % vsini, "%g" % vmacro, "%g" % vgau], cwd=wd, capture_output=True, text=True)
    if r.returncode != 0 or "Convolution and disk-integration" not in r.stdout:
        raise RuntimeError(r.stdout + r.stderr)
    return raw(wd, "fs_flux.bin")


def raw(wd, name):
    with open(os.path.join(wd, name), "rb") as f:
        return np.frombuffer(f.read(), np.uint8)


def main():
    model = W.eddington_model(5777.0, 4.44, 56)
    out = {}
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        a = W.atomic_lines(12, 5000.1, 5000.9, W.SEED0 + 70)
        b = W.atomic_lines(7, 5000.2, 5000.8, W.SEED0 + 71)
        a.write_z(os.path.join(wd, "a.z"), 5000.0, 5001.0)
        b.write_z(os.path.join(wd, "b.z"), 5000.0, 5001.0)
        run(wd, "wave=5000.0, 5001.0, 0.02, 0\nsave=1, 1, 1, 1, 1\nvmic=1.0\n"
                "lines=\n-1  a.z\n-1  b.z\n\nmodel=model.krz\nmus=3\n")
        for k, f in (("lineop", "fs_lineop.bin"), ("contop", "fs_contop.bin"), ("spec", "fs_spec.bin"),
                     ("flux", "fs_flux.bin"), ("linst", "fs_linst.bin")):
            out[k] = raw(wd, f)
        out["conv_a"] = convolve(wd, "fs_spec.bin", *CONV["conv_a"])
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        z = W.zeeman_lines(6, 6000.1, 6000.9, W.SEED0 + 72)
        jlo, jup, glo, gup = z.zeeman
        import oracle
        pats = [oracle.zeeman_pattern(jlo[i], jup[i], glo[i], gup[i]) for i in range(z.n)]
        z.write_z(os.path.join(wd, "z.z"), 6000.0, 6001.0, patterns=pats)
        run(wd, "wave=6000.0, 6001.0, 0.02, 0\nsave=0, 0, 1, 1, 1\nvmic=1.0\n"
                "lines=\n-1  z.z\n\nmodel=model.krz\nmus=3\nbframe=1\nbfield=2000, 60, 30\n")
        out["spec_mag"] = raw(wd, "fs_spec.bin")
        out["flux_mag"] = raw(wd, "fs_flux.bin")
        out["conv_b"] = convolve(wd, "fs_spec.bin", *CONV["conv_b"])
    np.savez_compressed(OUT, **out)
    print(OUT, {k: v.size for k, v in out.items()})


if __name__ == "__main__":
    main()
