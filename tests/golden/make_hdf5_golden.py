#!/usr/bin/env python3
"""Golden values for the HDF5 line-list reader: the first records of two of the reference's example
line lists, parsed from their TEXT sources (the VALD long-format extraction VALD_all_500-600.dat.gz and
the ExoMol FeH list 56Fe1H_Exomol_Irw.vac.gz in the reference's examples/lines), independently of any
HDF5 code.  The reference converted the same text files into VALD_all_500-600.h5 / .zh5 and
56Fe1H_Exomol_Irw.h5 (python/vald2hdf.py, python/mol2hdf.py), so the reader must return exactly these
values (as FP32 of the printed decimals) from the binary files.

Reads the reference tree (this container only); the output tests/golden/hdf5_examples.npz is committed.
"""
import gzip
import os

import numpy as np

LINES = os.path.join(os.environ.get("FASTSPEC_REFERENCE", ""), "examples", "lines")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hdf5_examples.npz")
N = 300


def vald_records(path, n):
    """First n records of a VALD long-format extraction: (El, Ion, wl, loggf, Elow, Jlo, Jup, Llo, Lup,
    Rad, Stark, Waals).  A record is one data line followed by three lines of level and reference text."""
    out = []
    with gzip.open(path, "rt") as f:
        f.readline(); f.readline()
        while len(out) < n:
            line = f.readline()
            if not line.startswith("'"):
                break
            q = line.index("'", 1)
            el, ion = line[1:q].split()
            v = [x.strip() for x in line[q + 2:].split(",")]
            out.append((el, int(ion), float(v[0]), v[1], v[2], v[3], v[5], v[6], v[7], v[9], v[10], v[11]))
            for _ in range(3):
                f.readline()
    return out


def exomol_records(path, wmin, n):
    """First n records with wavelength >= wmin of a Turbospectrum-format molecular list:
    (wl, Elow, loggf, g_up, gamma_rad)."""
    out = []
    with gzip.open(path, "rt") as f:
        f.readline(); f.readline()
        for line in f:
            v = line.split()
            if float(v[0]) < wmin:
                continue
            out.append((float(v[0]), v[1], v[2], v[4], v[5]))
            if len(out) == n:
                break
    return out


def main():
    f32 = lambda s: np.float32(float(s))
    r = vald_records(os.path.join(LINES, "VALD_all_500-600.dat.gz"), N)
    m = exomol_records(os.path.join(LINES, "56Fe1H_Exomol_Irw.vac.gz"), 9000.0, N)
    np.savez_compressed(
        OUT,
        vald_el=np.array([x[0] for x in r]), vald_ion=np.array([x[1] for x in r], np.int16),
        vald_w=np.array([x[2] for x in r]), vald_lggf=np.array([f32(x[3]) for x in r]),
        vald_e=np.array([f32(x[4]) for x in r]), vald_jlo=np.array([f32(x[5]) for x in r]),
        vald_jup=np.array([f32(x[6]) for x in r]), vald_glo=np.array([f32(x[7]) for x in r]),
        vald_gup=np.array([f32(x[8]) for x in r]), vald_grad=np.array([f32(x[9]) for x in r]),
        vald_gqst=np.array([f32(x[10]) for x in r]), vald_gvdw=np.array([f32(x[11]) for x in r]),
        feh_w=np.array([x[0] for x in m]), feh_e=np.array([f32(x[1]) for x in m]),
        feh_lggf=np.array([f32(x[2]) for x in m]), feh_gu=np.array([f32(x[3]) for x in m]),
        feh_grad=np.array([f32(x[4]) for x in m]))
    print(OUT, len(r), len(m))


if __name__ == "__main__":
    main()
