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


class FsioError(ValueError):
    """A file that is truncated or does not have the layout of the output it should hold."""


def _take(f, path, dtype, count, what):
    """Exactly count values of dtype from f, or FsioError naming the file and the field."""
    if count < 0:
        raise FsioError("%s: negative %s count %d (not a FastSpec output file?)" % (path, what, count))
    a = np.fromfile(f, dtype, count)
    if a.size != count:
        raise FsioError("%s: truncated: %s needs %d values, the file holds %d" % (path, what, count, a.size))
    return a


def read_opac(path):
    """fs_lineop.bin / fs_contop.bin -> dict(wave, opac [nwl][ntau], rhox, T, xne, xna, rho)."""
    with open(path, "rb") as f:
        nwl, ntau = (int(x) for x in _take(f, path, "<i4", 2, "header"))
        wave = _take(f, path, "<f8", nwl, "wavelengths")
        opac = _take(f, path, "<f8", nwl * ntau, "opacities").reshape(nwl, ntau)
        atm = _take(f, path, "<f8", 5 * ntau, "atmosphere").reshape(5, ntau)
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
        nwl, nmu = (int(x) for x in _take(f, path, "<i4", 2, "header"))
        xmu = _take(f, path, "<f8", nmu, "angles")
        wave = _take(f, path, "<f8", nwl, "wavelengths")
        rest = np.fromfile(f, "<f8")
    narr = rest.size // max(nwl * nmu, 1)
    if narr not in (2, 5) or rest.size != narr * nwl * nmu:
        raise FsioError("%s: truncated: %d intensity values, not 2 or 5 arrays of %d x %d" % (path, rest.size, nwl, nmu))
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


def spec_grid(spec):
    """The grid and angles ReadSpec (ioutils.f90:1930-1984) derives from an intensity file read by
    read_spec: the angles in descending order (its exchange sort, the spectra permuted alike), Wfirst =
    the first wavelength, offsets from it, and the step and mode (Wmode 1 with a velocity step when the
    first and last steps differ by more than 1e-6 A, else Wmode 0 with the first step).  Returns
    dict(wmode, wstart, wend, dstep, wave (offsets), xmu, spl, spc)."""
    xmu = np.asarray(spec["xmu"], np.float64)
    n = len(xmu)
    perm = list(range(n))
    for i in range(n - 1):
        for j in range(i + 1, n):
            if xmu[perm[j]] > xmu[perm[i]]:
                perm[i], perm[j] = perm[j], perm[i]
    wave_abs = np.asarray(spec["wave"], np.float64)
    if len(wave_abs) < 2 or n < 1:
        raise ValueError("intensity file needs two wavelengths and one angle")
    wfirst = float(wave_abs[0])
    wave = wave_abs - wfirst
    if abs((wave[1] - wave[0]) - (wave[-1] - wave[-2])) > 1e-6:
        dstep = 2.0 * (wave[1] - wave[0]) / (wave[0] + wave[1] + 2.0 * wfirst) * 299792.458
        wmode = 1
    else:
        dstep = wave[1] - wave[0]
        wmode = 0
    return dict(wmode=wmode, wstart=wfirst, wend=float(wave_abs[-1]), dstep=float(dstep), wave=wave,
                xmu=xmu[perm], spl=np.ascontiguousarray(spec["spl"][:, perm]),
                spc=np.ascontiguousarray(spec["spc"][:, perm]))


def read_flux(path):
    with open(path, "rb") as f:
        nwl = int(_take(f, path, "<i4", 1, "header")[0])
        wave = _take(f, path, "<f8", nwl, "wavelengths")
        sfl = _take(f, path, "<f8", nwl, "line flux")
        sfc = _take(f, path, "<f8", nwl, "continuum flux")
    return dict(wave=wave, sfl=sfl, sfc=sfc)


def write_flux(path, wave, sfl, sfc):
    with open(path, "wb") as f:
        np.array([len(wave)], "<i4").tofile(f)
        for a in (wave, sfl, sfc):
            np.asarray(a, "<f8").tofile(f)


def read_linst(path):
    """fs_linst.bin -> dict(species, ion, wave, strength) over all line lists, and nrec: the record
    count of each list in file order (write_linst with append=True rebuilds the file list by list)."""
    species, ion, wave, strength, nrec = [], [], [], [], []
    with open(path, "rb") as f:
        while True:
            n = np.fromfile(f, "<i4", 1)
            if n.size == 0:
                break
            n = int(n[0])
            nrec.append(n)
            species.append(np.char.strip(_take(f, path, "S8", n, "species").astype("U8")))
            ion.append(_take(f, path, "<i4", n, "ions"))
            wave.append(_take(f, path, "<f8", n, "wavelengths"))
            strength.append(_take(f, path, "<f4", n, "line strengths"))
    cat = lambda x, d: np.concatenate(x) if x else np.zeros(0, d)
    return dict(species=cat(species, "U8"), ion=cat(ion, "<i4"), wave=cat(wave, "<f8"),
                strength=cat(strength, "<f4"), nrec=np.array(nrec, np.int64))


def write_linst(path, species, ion, wave, strength, append=False):
    n = len(wave)
    with open(path, "ab" if append else "wb") as f:
        np.array([n], "<i4").tofile(f)
        np.array([s.encode().ljust(8)[:8] for s in species], "S8").tofile(f)
        np.asarray(ion, "<i4").tofile(f)
        np.asarray(wave, "<f8").tofile(f)
        np.asarray(strength, "<f4").tofile(f)


# ---- line lists in the reference's HDF5 layout (group /Lines, one dataset per column) ----------

MAXION = 5      # highest ionisation stage the reference's EOS supports (lines above it are dropped)


def vac2air(lam):
    """Vac2Air (utils.f90:1007-1017): vacuum to air wavelength [A] above 2000 A, unchanged below."""
    lam = np.asarray(lam, np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        s = 1e4 / lam
        s2 = s * s
        n = 1.0 + 8.34254e-5 + 2.406147e-2 / (130.0 - s2) + 1.5998e-4 / (38.9 - s2)
        return np.where(lam > 2000.0, lam / n, lam)


def _lower_bound(a, x):
    """LowerBoundReal8 (utils.f90:702-718): first 1-based i with a(i) >= x (n + 1 if none)."""
    return int(np.searchsorted(a, x, side="left")) + 1


def _upper_bound(a, x):
    """UpperBoundReal8 (utils.f90:721-737): last 1-based i with a(i) <= x (0 if none)."""
    return int(np.searchsorted(a, x, side="right"))


def read_hdf5_lines(path, species, exact=True, wstart=None, wend=None):
    """A FastSpec HDF5 line list as the library's SoA records, selected and converted as ReadHDF does
    (ioutils.f90:686-790): wavelengths of a list with WL_VAC = 1 turned to air (Vac2Air); the column
    must be sorted (ValueError otherwise, where ReadHDF stops); with wstart / wend (the synthesis range,
    WAVE=) only the lines with wstart <= W <= wend are kept, as the reader's bound search does.  Then
    the record conversions (ioutils.f90:889-1000 atomic / Zeeman, 790-812 molecular): gf = 10.0**LGGF; atomic Grad =
    10.0**GRAD for 0 < GRAD < 20, Gqst / Gvdw = 10.0**x for x < 0 (a positive GVDW is the packed ABO
    parameter), all in single precision (libm powf when exact, numpy's power otherwise); atomic lines
    above ionisation stage 5 are dropped.  Molecular single-species lists take GRAD as stored and no
    Stark / van der Waals parameters.

    species: the caller's species table, a list of (name, ion) in the order of the FractionPF columns
    of its atmosphere state; each line's index into it (spc) is -1 for a species the table lacks.
    Returns dict(wl, elo, gf, grad, gqst, gvdw, spc, ismol, kind, attrs[, jlo, jup, glo, gup]) with
    kind 0 (atomic list), 1 (molecular list) or 2 (Zeeman list, whose components hdf5_zeeman_components
    builds), the fsg_lines kinds."""
    from . import hdf5
    from .workloads import pow10f
    cols, attrs, _ = hdf5.read_lines(path)
    if int(attrs.get("HFLAG", 0)) == 1:
        # a dedicated hydrogen list goes to the reference's hydrogen line opacity (synth.f90:136-146),
        # which stays with the caller
        raise ValueError("read_hdf5_lines: %s is a hydrogen line list (HFLAG = 1)" % path)
    w = np.asarray(cols["W"], np.float64)
    if int(attrs.get("WL_VAC", 0)) == 1:
        w = vac2air(w)
    if not np.all(w[:-1] <= w[1:]):
        raise ValueError("read_hdf5_lines: wavelength array is not sorted in " + str(path))
    i1 = 1 if wstart is None else _lower_bound(w, wstart)
    i2 = len(w) if wend is None else _upper_bound(w, wend)
    sel = slice(i1 - 1, max(i2, i1 - 1))
    cols = {k: np.asarray(v)[sel] for k, v in cols.items()}
    cols["W"] = w[sel]
    p10 = pow10f if exact else (lambda v: np.power(np.float32(10.0), np.asarray(v, np.float32)).astype(np.float32))
    f32 = lambda a: np.asarray(a, np.float32)
    table = {(str(n), int(i)): k for k, (n, i) in enumerate(species)}
    if "EL" not in cols:                                 # single-species molecular list
        n = len(cols["W"])
        k = table.get((str(attrs.get("NAME", "")).strip(), int(attrs.get("ION", 1))), -1)
        z = np.zeros(n, np.float32)
        return dict(wl=np.asarray(cols["W"], np.float64), elo=f32(cols["E"]), gf=p10(f32(cols["LGGF"])),
                    grad=f32(cols["GRAD"]), gqst=z, gvdw=z.copy(), spc=np.full(n, k, np.int32),
                    ismol=np.ones(n, np.int32), kind=1, attrs=attrs)
    keep = np.asarray(cols["ION"]) <= MAXION
    el = np.asarray(cols["EL"])[keep]
    ion = np.asarray(cols["ION"], np.int32)[keep]
    lg, lq, lv = f32(cols["GRAD"])[keep], f32(cols["GQST"])[keep], f32(cols["GVDW"])[keep]
    out = dict(wl=np.asarray(cols["W"], np.float64)[keep], elo=f32(cols["E"])[keep],
               gf=p10(f32(cols["LGGF"])[keep]),
               grad=np.where((lg < 20.0) & (lg > 0.0), p10(lg), lg).astype(np.float32),
               gqst=np.where(lq < 0.0, p10(lq), lq).astype(np.float32),
               gvdw=np.where(lv < 0.0, p10(lv), lv).astype(np.float32),
               spc=np.array([table.get((str(e).strip(), int(i)), -1) for e, i in zip(el, ion)], np.int32),
               ismol=np.zeros(int(keep.sum()), np.int32), kind=0, attrs=attrs)
    for c in ("JLO", "JUP", "GLO", "GUP"):
        if c in cols:
            out[c.lower()] = f32(cols[c])[keep]
    if "jlo" in out:
        out["kind"] = 2                                  # Zeeman list: the magnetic records (LineTypeMag)
    return out


def write_hdf5_lines(path, species, spc, wl, elo, loggf, lgrad, lgqst, lgvdw, wl_vac=0, provenance="",
                     zeeman=None):
    """Write an atomic line list in the reference's HDF5 layout (the columns and group attributes of
    vald2hdf.py: EL, ION, W, E, LGGF, GRAD, GQST, GVDW, plus JLO, JUP, GLO, GUP when zeeman =
    (jlo, jup, glo, gup) is given), contiguous and unfiltered; the damping columns hold the logarithms
    (or the packed ABO parameter) as VALD gives them.  Lines must be sorted by wavelength."""
    import datetime
    from . import hdf5
    wl = np.asarray(wl, np.float64)
    if len(wl) > 1 and np.any(np.diff(wl) < 0):
        raise ValueError("write_hdf5_lines: lines must be sorted by wavelength")
    spc = np.asarray(spc)
    width = max(len(n) for n, _ in species) + 1
    cols = dict(EL=np.array([species[k][0] for k in spc], "S%d" % width),
                ION=np.array([species[k][1] for k in spc], np.int16), W=wl,
                E=np.asarray(elo, np.float32), LGGF=np.asarray(loggf, np.float32),
                GRAD=np.asarray(lgrad, np.float32), GQST=np.asarray(lgqst, np.float32),
                GVDW=np.asarray(lgvdw, np.float32))
    units = dict(EL="element symbol", ION="ionization stage (1 = neutral)",
                 W="Angstrom (air or vacuum per the WL_VAC attribute)", E="eV (lower-level excitation energy)",
                 LGGF="log10(gf) (dimensionless)", GRAD="log10(radiative damping /s) (VALD Rad.)",
                 GQST="log10(Stark damping /s per electron at 1e4 K) (VALD Stark)",
                 GVDW="VALD Waals: packed ABO sigma.alpha if >0, else log10(vdW damping /s per H atom at 1e4 K)")
    if zeeman is not None:
        for c, a in zip(("JLO", "JUP", "GLO", "GUP"), zeeman):
            cols[c] = np.asarray(a, np.float32)
            units[c] = "dimensionless"
    n = len(wl)
    attrs = dict(NL=np.int32(n), NAME="atom Zeeman" if zeeman is not None else "atom", WL_VAC=np.int16(wl_vac),
                 HFLAG=np.int16(0), FILE=str(path).rsplit("/", 1)[-1].rsplit(".", 1)[0],
                 DATE=datetime.date.today().isoformat(), PROVENANCE=provenance,
                 FORMAT_VERSION="z-1.0" if zeeman is not None else "a-1.0",
                 WMIN=np.float64(wl[0] if n else 0.0), WMAX=np.float64(wl[-1] if n else 0.0))
    hdf5.write_lines(path, cols, attrs, units)


def hdf5_zeeman_components(records, pattern):
    """Zeeman components of a Zeeman HDF5 list (records of read_hdf5_lines with jlo, jup, glo, gup) in
    the CSR form of fsg_lines, built as ReadHDF builds them (ioutils.f90:997-1031): a line with a Lande
    factor above 90 (the converters' 99 for unknown or forbidden) is one unshifted pi component of
    strength 1 and an unshifted sigma pair; otherwise the pattern's pi components as computed and its
    sigma branch mirrored, blue (negative shifts) first.  pattern(jlo, jup, glo, gup) -> (pi shifts,
    pi strengths, sigma shifts, sigma strengths), e.g. fastspec_b200.zeeman_pattern."""
    jlo, jup, glo, gup = (records[k] for k in ("jlo", "jup", "glo", "gup"))
    npi, nsi, spl_pi, str_pi, spl_si, str_si = [], [], [], [], [], []
    for i in range(len(jlo)):
        if glo[i] > 90.0 or gup[i] > 90.0:
            spi, rpi, ss, rs = [0.0], [1.0], [0.0], [1.0]
        else:
            spi, rpi, ss, rs = pattern(float(jlo[i]), float(jup[i]), float(glo[i]), float(gup[i]))
        npi.append(len(spi)); nsi.append(2 * len(ss))
        spl_pi += list(spi); str_pi += list(rpi)
        spl_si += list(-np.asarray(ss, np.float32)) + list(ss); str_si += list(rs) + list(rs)
    f = lambda a: np.asarray(a, np.float32)
    return (np.asarray(npi, np.int32), np.asarray(nsi, np.int32), f(spl_pi), f(str_pi), f(spl_si), f(str_si))


def write_hdf5_molecular(path, name, ion, code, wl, elo, loggf, grad, wl_vac=0, provenance=""):
    """Write a single-species molecular line list in the reference's HDF5 layout (the columns and
    group attributes of mol2hdf.py: W, E, LGGF, GRAD (linear radiative damping, 0 for the classical
    value); NL, ID (species code), NAME (the molecule as the EOS names it), ION, WL_VAC, FILE, DATE,
    PROVENANCE, FORMAT_VERSION, WMIN, WMAX), contiguous and unfiltered.  Lines sorted by wavelength."""
    import datetime
    from . import hdf5
    wl = np.asarray(wl, np.float64)
    if len(wl) > 1 and np.any(np.diff(wl) < 0):
        raise ValueError("write_hdf5_molecular: lines must be sorted by wavelength")
    cols = dict(W=wl, E=np.asarray(elo, np.float32), LGGF=np.asarray(loggf, np.float32),
                GRAD=np.asarray(grad, np.float32))
    units = dict(W="Angstrom (air or vacuum per the WL_VAC attribute)", E="eV (lower-level excitation energy)",
                 LGGF="log10(gf) (dimensionless)", GRAD="1/s (radiative damping constant, linear)")
    n = len(wl)
    attrs = dict(NL=np.int32(n), ID=str(code), NAME=str(name), ION=np.int32(ion), WL_VAC=np.int16(wl_vac),
                 FILE=str(path).rsplit("/", 1)[-1].rsplit(".", 1)[0], DATE=datetime.date.today().isoformat(),
                 PROVENANCE=provenance, FORMAT_VERSION="m-1.1",
                 WMIN=np.float64(wl[0] if n else 0.0), WMAX=np.float64(wl[-1] if n else 0.0))
    hdf5.write_lines(path, cols, attrs, units)
