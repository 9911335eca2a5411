"""Readers and writers of FastSpec's unformatted-stream output files.

Byte layouts follow the reference writers (ioutils.f90:1751-1875, WriteOut / WriteLinStr) and
its readers (ioutils.f90:1878-1984, ReadOpac / ReadSpec); all are native little-endian,
Fortran column-major arrays with no record markers:

  fs_lineop.bin / fs_contop.bin : Nwl, Ntau (i4); Wave+Wfirst (f8[Nwl]); Opac(Ntau,Nwl) (f8);
                                  Rhox, T, Xne, Xna, Rho (f8[Ntau] each)
  fs_spec.bin                   : Nwl, Nmu (i4); Xmu (f8[Nmu]); Wave (f8[Nwl]);
                                  SpL, SpC (f8[Nmu,Nwl]) or, magnetic, I, Ic, Q, U, V
  fs_flux.bin                   : Nwl (i4); Wave (f8[Nwl]); SfL, SfC (f8[Nwl])
  fs_linst.bin                  : per line list: Nrec (i4); species (S8[Nrec]); ion (i4[Nrec]);
                                  wave (f8[Nrec]); strength (f4[Nrec])

Arrays are returned C-ordered with the fast Fortran index last, e.g. LineOpac -> [nwl][ntau],
SpL -> [nwl][nmu], SpZ -> [nwl][4][nmu].
"""
import numpy as np


def read_opac(path):
    """fs_lineop.bin / fs_contop.bin -> dict(wave, opac [nwl][ntau], rhox, T, xne, xna, rho)."""
    with open(path, "rb") as f:
        nwl, ntau = (int(x) for x in np.fromfile(f, "<i4", 2))
        wave = np.fromfile(f, "<f8", nwl)
        opac = np.fromfile(f, "<f8", nwl * ntau).reshape(nwl, ntau)
        atm = np.fromfile(f, "<f8", 5 * ntau).reshape(5, ntau)
    return dict(wave=wave, opac=opac, rhox=atm[0], T=atm[1], xne=atm[2], xna=atm[3], rho=atm[4])


def write_opac(path, wave, opac, rhox, T, xne, xna, rho):
    opac = np.ascontiguousarray(opac, dtype="<f8")
    nwl, ntau = opac.shape
    with open(path, "wb") as f:
        np.array([nwl, ntau], "<i4").tofile(f)
        np.asarray(wave, "<f8").tofile(f)
        opac.tofile(f)
        for a in (rhox, T, xne, xna, rho):
            np.asarray(a, "<f8").tofile(f)


def read_spec(path):
    """fs_spec.bin -> dict(wave, xmu, spl [nwl][nmu], spc [nwl][nmu], magnetic, spz [nwl][4][nmu])."""
    with open(path, "rb") as f:
        nwl, nmu = (int(x) for x in np.fromfile(f, "<i4", 2))
        xmu = np.fromfile(f, "<f8", nmu)
        wave = np.fromfile(f, "<f8", nwl)
        rest = np.fromfile(f, "<f8")
    narr = rest.size // (nwl * nmu)
    sp = rest.reshape(narr, nwl, nmu)
    out = dict(wave=wave, xmu=xmu, spl=sp[0], spc=sp[1], magnetic=(narr == 5))
    if narr == 5:
        out["spz"] = np.stack([sp[0], sp[2], sp[3], sp[4]], axis=1)
    return out


def write_spec(path, wave, xmu, spl, spc, spz=None):
    nwl = len(wave); nmu = len(xmu)
    with open(path, "wb") as f:
        np.array([nwl, nmu], "<i4").tofile(f)
        np.asarray(xmu, "<f8").tofile(f)
        np.asarray(wave, "<f8").tofile(f)
        if spz is None:
            np.asarray(spl, "<f8").tofile(f)
            np.asarray(spc, "<f8").tofile(f)
        else:
            spz = np.asarray(spz, "<f8")
            spz[:, 0, :].tofile(f)
            np.asarray(spc, "<f8").tofile(f)
            for q in (1, 2, 3):
                np.ascontiguousarray(spz[:, q, :]).tofile(f)


def read_flux(path):
    with open(path, "rb") as f:
        nwl = int(np.fromfile(f, "<i4", 1)[0])
        wave = np.fromfile(f, "<f8", nwl)
        sfl = np.fromfile(f, "<f8", nwl)
        sfc = np.fromfile(f, "<f8", nwl)
    return dict(wave=wave, sfl=sfl, sfc=sfc)


def write_flux(path, wave, sfl, sfc):
    with open(path, "wb") as f:
        np.array([len(wave)], "<i4").tofile(f)
        for a in (wave, sfl, sfc):
            np.asarray(a, "<f8").tofile(f)


def read_linst(path):
    species, ion, wave, strength = [], [], [], []
    with open(path, "rb") as f:
        while True:
            n = np.fromfile(f, "<i4", 1)
            if n.size == 0:
                break
            n = int(n[0])
            species.append(np.char.strip(np.fromfile(f, "S8", n).astype("U8")))
            ion.append(np.fromfile(f, "<i4", n))
            wave.append(np.fromfile(f, "<f8", n))
            strength.append(np.fromfile(f, "<f4", n))
    cat = lambda x, d: np.concatenate(x) if x else np.zeros(0, d)
    return dict(species=cat(species, "U8"), ion=cat(ion, "<i4"), wave=cat(wave, "<f8"),
                strength=cat(strength, "<f4"))


def write_linst(path, species, ion, wave, strength, append=False):
    n = len(wave)
    with open(path, "ab" if append else "wb") as f:
        np.array([n], "<i4").tofile(f)
        np.array([s.encode().ljust(8)[:8] for s in species], "S8").tofile(f)
        np.asarray(ion, "<i4").tofile(f)
        np.asarray(wave, "<f8").tofile(f)
        np.asarray(strength, "<f4").tofile(f)
