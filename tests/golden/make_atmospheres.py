#!/usr/bin/env python3
"""Derive the host-side atmosphere states of the benchmark configurations from the reference.

The hot path consumes, per atmosphere, what the reference's host code (EOS, continuum) hands
it: T, Rhox, Xne, Rho, the species populations FractionPF (FP32), species masses, the
perturber density of van der Waals broadening, and the continuum opacity.  The EOS and the
continuum stay on the host and out of scope, and the reference is Fortran with no compiler on
either machine, so this script runs the reference's shipped program as a black box, here,
once, and stores what it computed:

  * model atmospheres: synthetic Eddington-grey hydrostatic models (workloads.eddington_model)
    for the solar-type (Teff 5777, log g 4.44, 56 depths), cool-dwarf (3500, 5.0, 72) and
    magnetic (5000, 4.5, 56) configurations;
  * T, Rhox, Xne, Xna, Rho after the EOS: read from fs_lineop.bin;
  * FractionPF per species: one probe line per species placed on a grid point, with only
    radiative damping, E_low = 0: LineOpac at the centre is H(a, 0) * LinCop, every factor of
    LinCop except FractionPF is known (opacity.f90:239-293), so FractionPF is the ratio.
    The recovered value must sit on an FP32 number (FractionPF is REAL(4)); that check
    confirms the species mass used for the Doppler width too;
  * the van der Waals perturber density Nprtb: one probe with a large G6: H(a, 0) is
    inverted on the table's bilinear lerp for a, a -> Gamma_6 -> Nprtb;
  * the continuum opacity on coarse knots spanning each configuration's range.

The states go to fastspec_b200/data/atm_*.npz (the benchmark workloads and the tests use them).
Also writes parity fixtures (tests/golden/pin_*.npz): line lists run through the reference
with the reference's line opacity, windows and spectra, for the oracle/GPU parity tests.
Test infrastructure: the oracle serves as the inversion model here.

Needs the reference tree named by $FASTSPEC_REFERENCE (its prebuilt executable is run); the outputs are
committed.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
DATA = os.path.join(REPO, "fastspec_b200", "data")
sys.path.insert(0, REPO)

import oracle  # noqa: E402  (fixture generation: the oracle is the inversion model)
from fastspec_b200 import fsio, workloads as W  # noqa: E402

BIN = os.path.join(os.environ.get("FASTSPEC_REFERENCE", ""), "src", "fastspec_Linux_x86_64")

AMASS = {"H": 1.00794, "He": 4.002602, "C": 12.0107, "N": 14.0067, "O": 15.9994,
         "Ca": 40.078, "Ti": 47.867, "Cr": 51.9961, "Fe": 55.845, "Ni": 58.6934}
# Ionisation potentials [eV]: the atomic ones are the reference EOS's own values as recover_potion
# finds them (they enter only the classical Stark and Unsold constants; molecules have neither).
POTION = {("Fe", 1): 7.902, ("Fe", 2): 16.199, ("Ti", 1): 6.819, ("Cr", 1): 6.764,
          ("Ni", 1): 7.64, ("Ca", 1): 6.11, ("TiO", 1): 6.4, ("H2O", 1): 12.621,
          ("CO", 1): 14.014, ("OH", 1): 13.017}
COMPOSITION = {"TiO": [("Ti", 1), ("O", 1)], "H2O": [("H", 2), ("O", 1)],
               "CO": [("C", 1), ("O", 1)], "OH": [("O", 1), ("H", 1)]}


def mass_candidates(name):
    """FP32 species mass as the EOS forms it: atoms REAL(4) Amass, molecules the REAL(4) sum of
    constituent masses (eos.f:1817, 1865); both summation orders are tried."""
    if name not in COMPOSITION:
        return [np.float32(AMASS[name])]
    comp = COMPOSITION[name]
    out = []
    for order in (comp, comp[::-1]):
        s = np.float32(0.0)
        for el, k in order:
            s = np.float32(s + np.float32(k) * np.float32(AMASS[el]))
        out.append(s)
    return out


def run_ref(workdir, deck):
    with open(os.path.join(workdir, "in.dat"), "w") as f:
        f.write(deck)
    r = subprocess.run([BIN, "in.dat"], cwd=workdir, capture_output=True, text=True)
    if r.returncode != 0 or "Total time" not in r.stdout:
        raise RuntimeError("reference run failed:\n" + r.stdout + r.stderr)
    return r.stdout


def probe_list(species, wl0, spacing, vdw_species=0, ismol=False, loggf=None):
    """One probe per species (G_rad only, E_low = 0) plus one van der Waals probe."""
    n = len(species)
    wl = wl0 + spacing * (1 + np.arange(n + 1))
    spc = np.concatenate([np.arange(n), [vdw_species]])
    loggf = np.full(n + 1, -1.0) if loggf is None else np.asarray(loggf, np.float64)
    elo = np.zeros(n + 1)
    lgrad = np.concatenate([np.full(n, 8.0), [5.0]])
    lgqst = np.full(n + 1, -30.0)
    lgvdw = np.concatenate([np.full(n, -30.0), [-6.5]])
    return W.LineList(species, wl, loggf, elo, lgrad, lgqst, lgvdw, spc,
                      np.full(n + 1, int(ismol), np.int32))


def calibrate_probes(species, ismol, wl0, dstep, vmic, molbrd, workdir, target=(0.3, 0.1)):
    """log gf of each probe so that its peak line/continuum ratio is about `target`
    (species probes, vdW probe): weak enough that the windows stay isolated."""
    nsp = len(species)
    probes = probe_list(species, wl0, 2.0, ismol=ismol)
    wend = wl0 + 2.0 * (nsp + 2)
    probes.write_z(os.path.join(workdir, "lines.z"), wl0, wend)
    deck = ("wave=%.4f, %.4f, %.6f, 0\nsave=0, 1, 1, 0, 0\nvmic=%.3f\nmolbrd=%d\n"
            "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=0\n" % (wl0, wend, dstep, vmic, molbrd))
    run_ref(workdir, deck)
    lo = fsio.read_opac(os.path.join(workdir, "fs_lineop.bin"))
    co = fsio.read_opac(os.path.join(workdir, "fs_contop.bin"))
    out = []
    for k in range(nsp + 1):
        ic = int(np.argmin(np.abs(lo["wave"] - probes.wl[k])))
        ratio = np.max(lo["opac"][ic] / co["opac"][ic])
        tgt = target[0] if k < nsp else target[1]
        out.append(round(-1.0 + np.log10(tgt / ratio), 3))
    return np.array(out)


def make_state(atm, species, masses, fpf, nprtb=None, contopac=None):
    nt = len(atm["T"])
    if nprtb is None:
        h1 = np.zeros(nt, np.float32); he1 = np.zeros(nt, np.float32)
    else:
        h1, he1 = encode_nprtb(nprtb)
    st = dict(rhox=atm["rhox"], T=atm["T"], xne=atm["xne"], xna=atm["xna"], rho=atm["rho"],
              fractionpf=fpf, xamass=np.asarray(masses, np.float32),
              potion=np.array([POTION.get(s, 7.0) for s in species], np.float32),
              ion=np.array([s[1] for s in species], np.int32), frac_h1=h1, frac_he1=he1,
              frac_h2=np.zeros(nt, np.float32))
    return st


def encode_nprtb(nprtb):
    """FP32 (H I, He I) pair with Fraction(H1) + 0.412265 Fraction(He1) == nprtb to ~1e-15."""
    h1 = nprtb.astype(np.float32)
    he1 = ((nprtb - h1.astype(np.float64)) / 0.412265).astype(np.float32)
    return h1, he1


def invert_h0(h, a_guess):
    """a with HVoigt(a, 0) == h (voigt.f90:76-110), by bisection on the oracle's HVoigt,
    which decreases monotonically in a at v = 0 (table lerp and asymptotic branches)."""
    out = np.empty_like(h)
    for i, hv in enumerate(h):
        lo, hi = 0.0, max(16.0, 4.0 * a_guess[i])
        while oracle.hvoigt(hi, 0.0) > hv:
            hi *= 2.0
        for _ in range(200):
            mid = 0.5 * (lo + hi)
            if mid == lo or mid == hi:
                break
            if oracle.hvoigt(mid, 0.0) > hv:
                lo = mid
            else:
                hi = mid
        out[i] = 0.5 * (lo + hi)
    return out


def recover(model, species, ismol, wl0, dstep, vmic, molbrd, workdir, extra_lines=None,
            extra_region=None, mus=0, save_spec=False, bfield=None):
    """Run the probes (+ optional extra lines in a separate region); recover the state."""
    nsp = len(species)
    W.write_krz(os.path.join(workdir, "model.krz"), model)
    pgf = calibrate_probes(species, ismol, wl0, dstep, vmic, molbrd, workdir)
    probes = probe_list(species, wl0, 2.0, vdw_species=0, ismol=ismol, loggf=pgf)
    wend = wl0 + 2.0 * (nsp + 2)
    if extra_region is not None:
        wend = extra_region[1]
    allw = [probes]
    if extra_lines is not None:
        allw.append(extra_lines)
    merged = merge(allw)
    W.write_krz(os.path.join(workdir, "model.krz"), model)
    pats = None
    if bfield is not None:
        pats = zeeman_blocks(merged)
    merged.write_z(os.path.join(workdir, "lines.z"), wl0, wend, patterns=pats)
    deck = ("wave=%.4f, %.4f, %.6f, 0\nsave=0, %d, 1, %d, %d\nvmic=%.3f\nmolbrd=%d\n"
            "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=%d\n"
            % (wl0, wend, dstep, 0 if bfield is not None else 1, int(save_spec), int(save_spec and mus > 1),
               vmic, molbrd, mus))
    if bfield is not None:
        deck += "bframe=1\nbfield=%g, %g, %g\n" % tuple(bfield)
    log = run_ref(workdir, deck)
    co = fsio.read_opac(os.path.join(workdir, "fs_contop.bin"))
    if bfield is None:
        lo = fsio.read_opac(os.path.join(workdir, "fs_lineop.bin"))
        atm = lo
    else:
        # the magnetic run saves no line opacity: recover from a companion field-free run
        raise RuntimeError("use recover() without bfield for the state")
    grid = dict(wmode=0, wstart=wl0, wend=wend, dstep=dstep)
    nt = len(atm["T"])
    # FractionPF per species, with the FP32 species mass that makes it land on FP32 values
    fpf = np.zeros((nt, nsp), np.float32)
    masses = []
    one = np.ones((nt, nsp), np.float32)
    wave = None
    for k, sp in enumerate(species):
        best = None
        for m in mass_candidates(sp[0]):
            ms = [np.float32(1.0)] * nsp
            ms[k] = m
            st = oracle.State(grid, make_state(atm, species, ms, one), contopac=co["opac"],
                              vmicro=vmic, molbrd=molbrd)
            if wave is None:
                wave = st.wave + st.wfirst
            L = oracle.Lines(**lines_args(probes), kind=2)
            cop, vv, av = oracle.xline(st, L, k)
            ic = int(np.argmin(np.abs(wave - probes.wl[k])))
            assert abs(wave[ic] - probes.wl[k]) < 1e-9, "probe not on a grid point"
            h0 = np.array([oracle.hvoigt(a, 0.0) for a in av])
            rec = atm["opac"][ic] / (h0 * cop)
            f32 = rec.astype(np.float32)
            dev = np.max(np.abs(rec / f32.astype(np.float64) - 1.0))
            if best is None or dev < best[0]:
                best = (dev, m, f32)
        if best[0] > 1e-10:
            print("  warning: %s %d FractionPF off FP32 by %.2e" % (sp[0], sp[1], best[0]))
        fpf[:, k] = best[2]
        masses.append(best[1])
        print("  %-4s %d  mass %.6f  FractionPF fp32 dev %.1e" % (sp[0], sp[1], best[1], best[0]))
    # Nprtb from the vdW probe (species 0)
    st = oracle.State(grid, make_state(atm, species, masses, fpf), contopac=co["opac"],
                      vmicro=vmic, molbrd=molbrd)
    L = oracle.Lines(**lines_args(probes), kind=2)
    kv = nsp
    cop, vv, av0 = oracle.xline(st, L, kv)
    ic = int(np.argmin(np.abs(wave - probes.wl[kv])))
    h = atm["opac"][ic] / cop
    a = invert_h0(h, av0)
    WaveL = probes.wl[kv]
    dopl = 1.0 / (vv * WaveL)
    dndopl = dopl / WaveL
    c4pi = 4.0 * 299792.458e13 * np.pi
    gam = a * (dndopl * c4pi)
    g6 = gam - float(probes.grad[kv])
    temp3 = (atm["T"] / 1e4) ** 0.3
    nprtb = g6 / (float(probes.gvdw[kv]) * temp3)
    state = make_state(atm, species, masses, fpf, nprtb=nprtb)
    # verify: the oracle reproduces the whole probe run
    st = oracle.State(grid, state, contopac=co["opac"], vmicro=vmic, molbrd=molbrd)
    Lall = oracle.Lines(**lines_args(merged), kind=2)
    res = oracle.lineop_calc(st, Lall, list_type=2)
    ref = atm["opac"]
    m = ref > 1e-30 * ref.max()
    rel = np.max(np.abs(res["lineopac"][m] / ref[m] - 1.0)) if m.any() else 0.0
    zero_match = np.array_equal(res["lineopac"] > 0, ref > 0)
    print("  probe run reproduced: max rel %.2e, nonzero pattern equal %s" % (rel, zero_match))
    return dict(state=state, nprtb=nprtb, masses=masses, atm=atm, contopac=co["opac"], probe_loggf=pgf,
                wave=wave, grid=grid, merged=merged, oracle_lineopac=res["lineopac"],
                ref_lineopac=ref, log=log, rel=rel, zero_match=zero_match, res=res)


def lines_args(L):
    a = L.arrays()
    return dict(wl=a["wl"], elo=a["elo"], gf=a["gf"], grad=a["grad"], gqst=a["gqst"],
                gvdw=a["gvdw"], spc=a["spc"], ismol=a["ismol"])


def merge(lists):
    sp = lists[0].species
    cat = lambda f: np.concatenate([getattr(l, f) for l in lists])
    txt = lambda f: np.concatenate([l._txt[f] for l in lists])
    out = W.LineList(sp, cat("wl"), txt("loggf"), txt("elo"), txt("lgrad"), txt("lgqst"),
                     txt("lgvdw"), cat("spc"), cat("ismol"))
    if any(l.zeeman is not None for l in lists):
        zz = []
        for l in lists:
            if l.zeeman is None:
                z = (np.full(l.n, 1.0, np.float32), np.full(l.n, 1.0, np.float32),
                     np.full(l.n, 1.0, np.float32), np.full(l.n, 1.0, np.float32))
            else:
                z = l.zeeman
            zz.append(z)
        z4 = [np.concatenate([z[q] for z in zz]) for q in range(4)]
        order = np.argsort(cat("wl"), kind="stable")
        out.zeeman = tuple(a[order] for a in z4)
    return out


def zeeman_blocks(L):
    pats = []
    jlo, jup, glo, gup = L.zeeman
    for i in range(L.n):
        spi, rpi, ss, rs = oracle.zeeman_pattern(jlo[i], jup[i], glo[i], gup[i])
        pats.append((spi, rpi, ss, rs))
    return pats


def coarse_contopac(model, wmin, wmax, step, species, vmic, molbrd, workdir, nknots):
    """Continuum opacity of the model on `nknots` knots spanning [wmin, wmax]."""
    probes = probe_list(species, wmin, 1.0)
    W.write_krz(os.path.join(workdir, "model.krz"), model)
    probes.write_z(os.path.join(workdir, "lines.z"), wmin, wmax)
    deck = ("wave=%.4f, %.4f, %.6f, 0\nsave=0, 0, 1, 0, 0\nvmic=%.3f\nmolbrd=%d\n"
            "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=0\n" % (wmin, wmax, step, vmic, molbrd))
    run_ref(workdir, deck)
    co = fsio.read_opac(os.path.join(workdir, "fs_contop.bin"))
    idx = np.unique(np.linspace(0, len(co["wave"]) - 1, nknots).round().astype(int))
    return co["wave"][idx], co["opac"][idx]


CONFIGS = {
    # name: (teff, logg, ntau, species, ismol, probe wl0, dstep, vmic, molbrd, range, nknots)
    "solar": (5777.0, 4.44, 56, W.ATOMIC_C0, 0, 5000.0, 0.005, 1.0, 0, (3000.0, 9000.0), 1201),
    "cooldwarf": (3500.0, 5.0, 72, W.MOLECULES_C1, 1, 9000.0, 0.01, 1.0, 1, (5000.0, 25000.0), 2001),
    "magnetic": (5000.0, 4.5, 56, W.ATOMIC_C0, 0, 6000.0, 0.002, 1.0, 0, (5900.0, 6200.0), 301),
}


def main():
    outdir = DATA
    gold = os.path.join(REPO, "tests", "golden")
    os.makedirs(gold, exist_ok=True)
    oracle.build()
    for name, (teff, logg, ntau, species, ismol, wl0, dstep, vmic, molbrd, rng_, nk) in CONFIGS.items():
        print(name)
        model = W.eddington_model(teff, logg, ntau)
        with tempfile.TemporaryDirectory() as wd:
            r = recover(model, species, ismol, wl0, dstep, vmic, molbrd, wd)
            kw, kc = coarse_contopac(model, rng_[0], rng_[1], 0.5 if name != "cooldwarf" else 1.0,
                                     species, vmic, molbrd, wd, nk)
        st = r["state"]
        np.savez_compressed(
            os.path.join(outdir, "atm_%s.npz" % name), teff=teff, logg=logg,
            species=np.array(["%s %d" % s for s in species]), ismol=ismol, vmicro=vmic,
            molbrd=molbrd, rhox=st["rhox"], T=st["T"], xne=st["xne"], xna=st["xna"],
            rho=st["rho"], fractionpf=st["fractionpf"], xamass=st["xamass"],
            potion=st["potion"], ion=st["ion"], frac_h1=st["frac_h1"], frac_he1=st["frac_he1"],
            nprtb=r["nprtb"], cont_wave=kw, cont_opac=kc.astype(np.float64),
            probe_rel=r["rel"], probe_loggf=r["probe_loggf"], model_rhox=model["rhox"],
            model_T=model["T"])
    make_pins(gold)


def load_state(name):
    d = np.load(os.path.join(DATA, "atm_%s.npz" % name))
    keys = ("rhox", "T", "xne", "xna", "rho", "fractionpf", "xamass", "potion", "ion",
            "frac_h1", "frac_he1")
    st = {k: d[k] for k in keys}
    st["frac_h2"] = d["frac_h2"] if "frac_h2" in d.files else np.zeros(len(d["T"]), np.float32)
    return st


def pin_specs():
    return [
        # name, atmosphere, list maker, (wstart, wend, step, wmode), pin region
        ("pin_solar", "solar", lambda: W.atomic_lines(160, 5040.5, 5044.5, W.SEED0 + 0),
         (5000.0, 5045.0, 0.005, 0), (5040.0, 5045.0)),
        ("pin_cooldwarf", "cooldwarf", lambda: W.molecular_lines(400, 9040.5, 9046.5, W.SEED0 + 1),
         (9000.0, 9047.0, 0.3, 1), (9040.0, 9047.0)),
    ]


def make_pins(gold):
    """Parity fixtures: reference line opacity and spectra of seeded lists on small grids.

    Each run holds the probe lines first (they fix the species inventory order of the EOS,
    hence the identical state) and the seeded list in a separate region; the region's line
    opacity, continuum opacity and spectra are stored with the list."""
    for name, atmname, mk, grid, region in pin_specs():
        teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS[atmname]
        model = W.eddington_model(teff, logg, ntau)
        state = load_state(atmname)
        extra = mk()
        pgf = np.load(os.path.join(DATA, "atm_%s.npz" % atmname))["probe_loggf"]
        probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
        merged = merge([probes, extra])
        with tempfile.TemporaryDirectory() as wd:
            W.write_krz(os.path.join(wd, "model.krz"), model)
            merged.write_z(os.path.join(wd, "lines.z"), grid[0], grid[1])
            deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=0, 1, 1, 1, 1\nvmic=%.3f\nmolbrd=%d\n"
                    "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=7\n"
                    % (grid[0], grid[1], grid[2], grid[3], vmic, molbrd))
            run_ref(wd, deck)
            lo = fsio.read_opac(os.path.join(wd, "fs_lineop.bin"))
            co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
            sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
            fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
        for k in ("rhox", "T", "xne", "xna", "rho"):
            assert np.array_equal(lo[k], state[k]), "EOS state differs from the recovered one: " + k
        wave = lo["wave"]
        sel = (wave >= region[0] - 1e-9) & (wave <= region[1] + 1e-9)
        i0, i1 = (int(x) for x in np.nonzero(sel)[0][[0, -1]])
        # the probes' windows must end before the region: check with the oracle
        g = dict(wmode=grid[3], wstart=grid[0], wend=grid[1], dstep=grid[2])
        st = oracle.State(g, state, contopac=co["opac"], vmicro=vmic, molbrd=molbrd)
        rp = oracle.lineop_calc(st, oracle.Lines(**lines_args(probes), kind=2), list_type=2)
        assert rp["iright"].max() < i0 + 1, "probe windows reach the pin region"
        a = extra.arrays()
        np.savez_compressed(
            os.path.join(gold, name + ".npz"),
            grid=np.array(grid, np.float64), i0=i0, i1=i1, atm=atmname,
            species=np.array(["%s %d" % s for s in species]), vmicro=vmic, molbrd=molbrd,
            contopac=co["opac"][i0:i1 + 1], lineopac=lo["opac"][i0:i1 + 1],
            wave=wave[i0:i1 + 1], xmu=sp["xmu"], spl=sp["spl"][i0:i1 + 1],
            spc=sp["spc"][i0:i1 + 1], sfl=fl["sfl"][i0:i1 + 1], sfc=fl["sfc"][i0:i1 + 1],
            **{"line_" + k: v for k, v in a.items()})
        print(name, "lines", extra.n, "region pixels", i1 - i0 + 1)


def make_linst_pins(gold):
    """Line-strength fixtures: the reference's fs_linst.bin (LinStrCalc, SAVE flag 1) for the decks
    of make_pins, restricted to the seeded lines (the probes come first in the list)."""
    for name, atmname, mk, grid, region in pin_specs():
        teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS[atmname]
        model = W.eddington_model(teff, logg, ntau)
        extra = mk()
        pgf = np.load(os.path.join(DATA, "atm_%s.npz" % atmname))["probe_loggf"]
        probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
        merged = merge([probes, extra])
        with tempfile.TemporaryDirectory() as wd:
            W.write_krz(os.path.join(wd, "model.krz"), model)
            merged.write_z(os.path.join(wd, "lines.z"), grid[0], grid[1])
            deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=1, 0, 0, 0, 0\nvmic=%.3f\nmolbrd=%d\n"
                    "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=7\n"
                    % (grid[0], grid[1], grid[2], grid[3], vmic, molbrd))
            run_ref(wd, deck)
            ls = fsio.read_linst(os.path.join(wd, "fs_linst.bin"))
        sel = ls["wave"] >= extra.arrays()["wl"].min() - 1e-9
        np.savez_compressed(os.path.join(gold, name + "_linst.npz"), wave=ls["wave"][sel],
                            strength=ls["strength"][sel], ion=ls["ion"][sel], nprobe_rows=int((~sel).sum()))
        print(name, "line strengths", int(sel.sum()), "of", extra.n, "seeded lines")


MAG_FRAMES = {
    # stellar frame: (Br, Bm, Bp) projected at each disk position (synth.f90:1960-1980)
    0: (1500.0, 800.0, -600.0),
    # observer frame per angle: |B| then (gamma, psi) for each of the 9 angles (synth.f90:1948-1959)
    2: (2500.0,) + tuple(v for k in range(9) for v in (10.0 + 17.0 * k, -40.0 + 11.0 * k)),
}


def make_mag_frames_pin(gold):
    """Stokes IQUV of the pin_magnetic list with the field in the stellar frame (BFRAME 0) and given per
    angle in the observer frame (BFRAME 2), 9 angles, plane-parallel (pin_magnetic_frames.npz; the
    BFRAME 1 run is pin_magnetic.npz)."""
    teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS["magnetic"]
    model = W.eddington_model(teff, logg, ntau)
    state = load_state("magnetic")
    grid = (6000.0, 6043.0, 0.002, 0)
    region = (6040.0, 6043.0)
    extra = W.zeeman_lines(60, 6040.3, 6042.7, W.SEED0 + 2)
    pgf = np.load(os.path.join(DATA, "atm_magnetic.npz"))["probe_loggf"]
    probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
    merged = merge([probes, extra])
    pats = zeeman_blocks(merged)
    out = {}
    for frame, bfield in MAG_FRAMES.items():
        with tempfile.TemporaryDirectory() as wd:
            W.write_krz(os.path.join(wd, "model.krz"), model)
            merged.write_z(os.path.join(wd, "lines.z"), grid[0], grid[1], patterns=pats)
            deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=0, 0, 1, 1, 1\nvmic=%.3f\nmolbrd=%d\n"
                    "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=9\nbframe=%d\nbfield=%s\n"
                    % (grid + (vmic, molbrd, frame, ", ".join("%g" % v for v in bfield))))
            log = run_ref(wd, deck)
            assert "polarised" in log, log
            co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
            sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
            fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
        for k in ("rhox", "T", "xne", "xna", "rho"):
            assert np.array_equal(co[k], state[k]), "EOS state differs from the recovered one: " + k
        wave = co["wave"]
        sel = (wave >= region[0] - 1e-9) & (wave <= region[1] + 1e-9)
        i0, i1 = (int(x) for x in np.nonzero(sel)[0][[0, -1]])
        out.update({"f%d_bfield" % frame: np.array(bfield), "f%d_spz" % frame: sp["spz"][i0:i1 + 1],
                    "f%d_spc" % frame: sp["spc"][i0:i1 + 1], "f%d_sfl" % frame: fl["sfl"][i0:i1 + 1]})
    np.savez_compressed(os.path.join(gold, "pin_magnetic_frames.npz"), i0=i0, i1=i1, xmu=sp["xmu"], **out)
    print("pin_magnetic_frames: frames", list(MAG_FRAMES), "region pixels", i1 - i0 + 1)


def make_mag_linst_pin(gold):
    """Line strengths of the magnetic driver (MagLineopCalc with SAVE flag 1, synth.f90:1098-1455): the
    pin_magnetic deck with BFRAME 1 and the explicit Zeeman patterns, its fs_linst.bin restricted to the
    seeded lines (pin_magnetic_linst.npz)."""
    teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS["magnetic"]
    model = W.eddington_model(teff, logg, ntau)
    grid = (6000.0, 6043.0, 0.002, 0)
    bfield = (2000.0, 60.0, 30.0)
    extra = W.zeeman_lines(60, 6040.3, 6042.7, W.SEED0 + 2)
    pgf = np.load(os.path.join(DATA, "atm_magnetic.npz"))["probe_loggf"]
    probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
    merged = merge([probes, extra])
    pats = zeeman_blocks(merged)
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        merged.write_z(os.path.join(wd, "lines.z"), grid[0], grid[1], patterns=pats)
        deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=1, 0, 0, 0, 0\nvmic=%.3f\nmolbrd=%d\n"
                "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=9\nbframe=1\nbfield=%g, %g, %g\n"
                % (grid + (vmic, molbrd) + bfield))
        log = run_ref(wd, deck)
        assert "polarised" in log, log
        ls = fsio.read_linst(os.path.join(wd, "fs_linst.bin"))
    sel = ls["wave"] >= extra.arrays()["wl"].min() - 1e-9
    np.savez_compressed(os.path.join(gold, "pin_magnetic_linst.npz"), wave=ls["wave"][sel],
                        strength=ls["strength"][sel], ion=ls["ion"][sel], nprobe_rows=int((~sel).sum()))
    print("pin_magnetic line strengths", int(sel.sum()), "of", extra.n, "seeded lines")


def make_reentry_pin(gold):
    """OPACITY= re-entry (ReadOpac, ioutils.f90:1878-1927; fastspec.f90:215): a line opacity file
    written by fsio.write_opac, holding the ORACLE's line opacity of list A on the pin_solar grid, is
    given to the reference program with list B; its output line opacity is the file plus B's opacity
    (LineopCalc adds to the array ReadOpac filled).  Pins the file writer (the reference accepts the
    grid and reads the array) and the accumulate-onto-loaded-opacity semantics
    (pin_solar_reentry.npz: the region's output line opacity, continuum and flux, lists A and B)."""
    name, atmname, mk, grid, region = pin_specs()[0]
    teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS[atmname]
    model = W.eddington_model(teff, logg, ntau)
    state = load_state(atmname)
    la = W.atomic_lines(90, 5040.5, 5044.5, W.SEED0 + 43)
    lb = W.atomic_lines(70, 5040.5, 5044.5, W.SEED0 + 44)
    pgf = np.load(os.path.join(DATA, "atm_%s.npz" % atmname))["probe_loggf"]
    probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
    g = dict(wmode=grid[3], wstart=grid[0], wend=grid[1], dstep=grid[2])
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        # continuum of the grid (probes only)
        probes.write_z(os.path.join(wd, "p.z"), grid[0], grid[1])
        run_ref(wd, "wave=%.4f, %.4f, %.6f, %d\nsave=0, 1, 1, 0, 0\nvmic=%.3f\nmolbrd=%d\n"
                    "lines=\n-1  p.z\n\nmodel=model.krz\nmus=0\n" % (grid + (vmic, molbrd)))
        lo0 = fsio.read_opac(os.path.join(wd, "fs_lineop.bin"))
        co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
        S = oracle.State(g, state, contopac=co["opac"], vmicro=vmic, molbrd=molbrd)
        ra = oracle.lineop_calc(S, oracle.Lines(**lines_args(la), kind=2), list_type=2)
        fsio.write_opac(os.path.join(wd, "opac_a.bin"), lo0["wave"], ra["lineopac"], lo0["rhox"], lo0["T"],
                        lo0["xne"], lo0["xna"], lo0["rho"])
        merged = merge([probes, lb])
        merged.write_z(os.path.join(wd, "lines.z"), grid[0], grid[1])
        log = run_ref(wd, "wave=%.4f, %.4f, %.6f, %d\nsave=0, 1, 1, 1, 1\nvmic=%.3f\nmolbrd=%d\n"
                          "opacity=opac_a.bin\nlines=\n-1  lines.z\n\nmodel=model.krz\nmus=7\n"
                          % (grid + (vmic, molbrd)))
        assert "Added line opacity from" in log, log
        lo = fsio.read_opac(os.path.join(wd, "fs_lineop.bin"))
        sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
        fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(lo[k], state[k]), "EOS state differs from the recovered one: " + k
    wave = lo["wave"]
    sel = (wave >= region[0] - 1e-9) & (wave <= region[1] + 1e-9)
    i0, i1 = (int(x) for x in np.nonzero(sel)[0][[0, -1]])
    rb = oracle.lineop_calc(S, oracle.Lines(**lines_args(lb), kind=2), list_type=2, lineopac=ra["lineopac"].copy())
    ref = lo["opac"][i0:i1 + 1]
    m = ref > 0
    mine = rb["lineopac"][i0:i1 + 1]
    print("  re-entry pin: pattern equal %s, line opacity max rel %.2e"
          % (np.array_equal(mine > 0, m), np.max(np.abs(mine[m] / ref[m] - 1))))
    A, B = la.arrays(), lb.arrays()
    np.savez_compressed(
        os.path.join(gold, "pin_solar_reentry.npz"), grid=np.array(grid, np.float64), i0=i0, i1=i1,
        atm=atmname, vmicro=vmic, molbrd=molbrd, contopac=co["opac"][i0:i1 + 1], lineopac=ref,
        wave=wave[i0:i1 + 1], xmu=sp["xmu"], sfl=fl["sfl"][i0:i1 + 1], sfc=fl["sfc"][i0:i1 + 1],
        **{"a_" + k: v for k, v in A.items()}, **{"line_" + k: v for k, v in B.items()})


def make_convol_pin(gold):
    """Broadening fixtures: the reference's intensities (fs_spec.bin) and its broadened flux
    (fs_flux.bin, IntegConvol / DiskInteg with CONVOL = Vsini, Vmacro, Vgau) of the same run, for
    a Wmode 0 and a Wmode 1 grid and several broadening settings."""
    cases = [
        # name, atmosphere, lines, (wstart, wend, step, wmode), convol settings
        ("solar", "solar", lambda: W.atomic_lines(160, 5040.5, 5044.5, W.SEED0 + 0), (5040.0, 5045.0, 0.005, 0),
         [(30.0, 4.0, 60000.0), (0.0, 3.0, 0.0), (12.0, 0.0, 0.0), (0.0, 0.0, 0.15)]),
        ("cooldwarf", "cooldwarf", lambda: W.molecular_lines(400, 9040.5, 9046.5, W.SEED0 + 1),
         (9040.0, 9047.0, 0.3, 1), [(8.0, 2.0, 3.0), (25.0, 0.0, 100000.0)]),
    ]
    out = {}
    for name, atmname, mk, grid, settings in cases:
        teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS[atmname]
        model = W.eddington_model(teff, logg, ntau)
        lines = mk()
        for k, (vs, vm, vg) in enumerate(settings):
            with tempfile.TemporaryDirectory() as wd:
                W.write_krz(os.path.join(wd, "model.krz"), model)
                lines.write_z(os.path.join(wd, "lines.z"), grid[0], grid[1])
                deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=0, 0, 0, 1, 1\nvmic=%.3f\nmolbrd=%d\n"
                        "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=7\nconvol=%g, %g, %g\n"
                        % (grid[0], grid[1], grid[2], grid[3], vmic, molbrd, vs, vm, vg))
                run_ref(wd, deck)
                sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
                fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
            key = "%s_%d" % (name, k)
            out[key + "_spl"] = sp["spl"]; out[key + "_spc"] = sp["spc"]
            out[key + "_sfl"] = fl["sfl"]; out[key + "_sfc"] = fl["sfc"]
            out[key + "_wave"] = fl["wave"] if "wave" in fl else sp["wave"]
            out[key + "_xmu"] = sp["xmu"]
            out[key + "_grid"] = np.array(grid, np.float64)
            out[key + "_convol"] = np.array([vs, vm, vg], np.float64)
    np.savez_compressed(os.path.join(gold, "pin_convol.npz"), **out)
    print("pin_convol", sorted(set(k.rsplit("_", 1)[0] for k in out)))


def mirrored_components(patterns):
    """Zeeman components as ReadAscMag stores an explicit block with a positive sigma count:
    pi as read, sigma mirrored (blue = -shift first, then red), ioutils.f90:1393-1410."""
    npi, nsi, spl_pi, str_pi, spl_si, str_si = [], [], [], [], [], []
    for spi, rpi, ss, rs in patterns:
        npi.append(len(spi)); nsi.append(2 * len(ss))
        spl_pi += list(spi); str_pi += list(rpi)
        spl_si += list(-np.asarray(ss)) + list(ss); str_si += list(rs) + list(rs)
    f = lambda a: np.asarray(a, np.float32)
    return (np.asarray(npi, np.int32), np.asarray(nsi, np.int32), f(spl_pi), f(str_pi), f(spl_si), f(str_si))


def make_mag_pin(gold):
    """Stokes IQUV of seeded Zeeman lines (explicit patterns), BFRAME 1, |B| = 2 kG at
    inclination 60 deg and azimuth 30 deg, 9 angles, on 6040-6046 A at 0.002 A."""
    teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS["magnetic"]
    model = W.eddington_model(teff, logg, ntau)
    state = load_state("magnetic")
    grid = (6000.0, 6043.0, 0.002, 0)
    region = (6040.0, 6043.0)
    bfield = (2000.0, 60.0, 30.0)
    extra = W.zeeman_lines(60, 6040.3, 6042.7, W.SEED0 + 2)
    pgf = np.load(os.path.join(DATA, "atm_magnetic.npz"))["probe_loggf"]
    probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
    merged = merge([probes, extra])
    pats = zeeman_blocks(merged)
    for q, (spi, rpi, ss, rs) in enumerate(pats):
        assert len(spi) >= 1 and len(ss) >= 1, "empty Zeeman branch"
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        merged.write_z(os.path.join(wd, "lines.z"), grid[0], grid[1], patterns=pats)
        deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=0, 0, 1, 1, 1\nvmic=%.3f\nmolbrd=%d\n"
                "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=9\nbframe=1\nbfield=%g, %g, %g\n"
                % (grid + (vmic, molbrd) + bfield))
        log = run_ref(wd, deck)
        assert "polarised" in log, log
        co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
        sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
        fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(co[k], state[k]), "EOS state differs from the recovered one: " + k
    assert sp["magnetic"]
    wave = co["wave"]
    sel = (wave >= region[0] - 1e-9) & (wave <= region[1] + 1e-9)
    i0, i1 = (int(x) for x in np.nonzero(sel)[0][[0, -1]])
    comp = mirrored_components(pats)
    # the probes' windows must end before the region (oracle, full continuum of this run)
    g = dict(wmode=grid[3], wstart=grid[0], wend=grid[1], dstep=grid[2])
    S = oracle.State(g, state, contopac=co["opac"], vmicro=vmic, molbrd=molbrd)
    npr = probes.n
    pa = probes.arrays()
    pc = mirrored_components(pats[:npr])
    rp = oracle.mag_lineop_calc(S, oracle.Lines(**lines_args(probes), kind=2, zeeman=pc), 1, np.array(bfield))
    assert rp["iright"].max() < i0 + 1, "probe windows reach the pin region"
    # keep only the seeded lines (the region's opacity comes from them alone)
    a = {k: v[npr:] for k, v in merged.arrays().items()}
    comp = mirrored_components(pats[npr:])
    np.savez_compressed(
        os.path.join(gold, "pin_magnetic.npz"),
        grid=np.array(grid, np.float64), i0=i0, i1=i1, atm="magnetic", bframe=1, bfield=np.array(bfield),
        species=np.array(["%s %d" % s for s in species]), vmicro=vmic, molbrd=molbrd,
        contopac=co["opac"][i0:i1 + 1], wave=wave[i0:i1 + 1], xmu=sp["xmu"],
        spz=sp["spz"][i0:i1 + 1], spc=sp["spc"][i0:i1 + 1], sfl=fl["sfl"][i0:i1 + 1], sfc=fl["sfc"][i0:i1 + 1],
        z_npi=comp[0], z_nsi=comp[1], z_spl_pi=comp[2], z_str_pi=comp[3], z_spl_si=comp[4], z_str_si=comp[5],
        **{"line_" + k: v for k, v in a.items()})
    print("pin_magnetic lines", merged.n, "region pixels", i1 - i0 + 1)


SPHERE_RADIUS = {"solar": 3.0e10, "magnetic": 5.0e10}


def sphere_model(atmname):
    """The configuration's model atmosphere as a spherical model: layer heights from hydrostatics
    (workloads.model_heights) and a radius small enough that the outermost angle of the default
    Gauss-Legendre set is a grazing ray while every other ray reaches the bottom layer."""
    teff, logg, ntau = CONFIGS[atmname][:3]
    model = W.eddington_model(teff, logg, ntau)
    return model, SPHERE_RADIUS[atmname], W.model_heights(model["rhox"], model["rho"])


def make_sphere_pins(gold):
    """Spherical fixtures (pin_sphere.npz): the decks of pin_solar and pin_magnetic with the model
    written as a spherical one.  Scalar: line opacity, continuum, intensities, flux and line strengths
    of one run (SAVE 1,1,1,1,1).  Polarised: Stokes IQUV with the field in the stellar frame
    (BFRAME 0), whose projection changes along the curved rays."""
    out = {}
    # scalar
    name, atmname, mk, grid, region = pin_specs()[0]
    teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS[atmname]
    model, radius, height = sphere_model(atmname)
    state = load_state(atmname)
    extra = mk()
    pgf = np.load(os.path.join(DATA, "atm_%s.npz" % atmname))["probe_loggf"]
    probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
    merged = merge([probes, extra])
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model, radius=radius, height=height)
        merged.write_z(os.path.join(wd, "lines.z"), grid[0], grid[1])
        deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=1, 1, 1, 1, 1\nvmic=%.3f\nmolbrd=%d\n"
                "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=7\n" % (grid + (vmic, molbrd)))
        log = run_ref(wd, deck)
        assert "Spherical" in log, log
        lo = fsio.read_opac(os.path.join(wd, "fs_lineop.bin"))
        co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
        sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
        fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
        ls = fsio.read_linst(os.path.join(wd, "fs_linst.bin"))
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(lo[k], state[k]), "EOS state differs from the recovered one: " + k
    g = oracle.sphere_init(state["rhox"], height, radius, sp["xmu"])
    assert 0 < g["graz"].sum() < len(g["graz"]), "want grazing and normal rays"
    wave = lo["wave"]
    sel = (wave >= region[0] - 1e-9) & (wave <= region[1] + 1e-9)
    i0, i1 = (int(x) for x in np.nonzero(sel)[0][[0, -1]])
    lsel = ls["wave"] >= extra.arrays()["wl"].min() - 1e-9
    out.update(s_grid=np.array(grid, np.float64), s_i0=i0, s_i1=i1, s_radius=radius, s_height=height,
               s_contopac=co["opac"][i0:i1 + 1], s_lineopac=lo["opac"][i0:i1 + 1], s_wave=wave[i0:i1 + 1],
               s_xmu=sp["xmu"], s_spl=sp["spl"][i0:i1 + 1], s_spc=sp["spc"][i0:i1 + 1],
               s_sfl=fl["sfl"][i0:i1 + 1], s_sfc=fl["sfc"][i0:i1 + 1], s_linst_wave=ls["wave"][lsel],
               s_linst=ls["strength"][lsel])
    print("sphere scalar: region pixels", i1 - i0 + 1, "grazing rays", int(g["graz"].sum()),
          "line strengths", int(lsel.sum()))
    # polarised, stellar-frame field
    teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS["magnetic"]
    model, radius, height = sphere_model("magnetic")
    state = load_state("magnetic")
    grid = (6000.0, 6043.0, 0.002, 0)
    region = (6040.0, 6043.0)
    bfield = (1500.0, 800.0, -600.0)
    extra = W.zeeman_lines(60, 6040.3, 6042.7, W.SEED0 + 2)
    pgf = np.load(os.path.join(DATA, "atm_magnetic.npz"))["probe_loggf"]
    probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
    merged = merge([probes, extra])
    pats = zeeman_blocks(merged)
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model, radius=radius, height=height)
        merged.write_z(os.path.join(wd, "lines.z"), grid[0], grid[1], patterns=pats)
        deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=0, 0, 1, 1, 1\nvmic=%.3f\nmolbrd=%d\n"
                "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=9\nbframe=0\nbfield=%g, %g, %g\n"
                % (grid + (vmic, molbrd) + bfield))
        log = run_ref(wd, deck)
        assert "Spherical polarised" in log, log
        co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
        sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
        fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(co[k], state[k]), "EOS state differs from the recovered one: " + k
    g = oracle.sphere_init(state["rhox"], height, radius, sp["xmu"])
    assert 0 < g["graz"].sum() < len(g["graz"]), "want grazing and normal rays"
    wave = co["wave"]
    sel = (wave >= region[0] - 1e-9) & (wave <= region[1] + 1e-9)
    i0, i1 = (int(x) for x in np.nonzero(sel)[0][[0, -1]])
    npr = probes.n
    a = {k: v[npr:] for k, v in merged.arrays().items()}
    comp = mirrored_components(pats[npr:])
    out.update(m_grid=np.array(grid, np.float64), m_i0=i0, m_i1=i1, m_radius=radius, m_height=height,
               m_bframe=0, m_bfield=np.array(bfield), m_contopac=co["opac"][i0:i1 + 1], m_wave=wave[i0:i1 + 1],
               m_xmu=sp["xmu"], m_spz=sp["spz"][i0:i1 + 1], m_spc=sp["spc"][i0:i1 + 1],
               m_sfl=fl["sfl"][i0:i1 + 1], m_sfc=fl["sfc"][i0:i1 + 1],
               z_npi=comp[0], z_nsi=comp[1], z_spl_pi=comp[2], z_str_pi=comp[3], z_spl_si=comp[4],
               z_str_si=comp[5], **{"mline_" + k: v for k, v in a.items()})
    np.savez_compressed(os.path.join(gold, "pin_sphere.npz"), **out)
    print("sphere polarised: region pixels", i1 - i0 + 1, "grazing rays", int(g["graz"].sum()))


def make_h5_pin(gold):
    """HDF5 fixture (pin_solar_h5.npz): the pin_solar list written by fsio.write_hdf5_lines (the
    reference's columnar /Lines layout) and read by the reference program as an atomic HDF5 list
    (ReadHDF, ioutils.f90:524-1159) after the probe list; the region's line opacity, continuum and
    spectra.  Pins the writer (the reference's HDF5 library accepts the file) and the atomic-list path
    (LineTypeAtm records, wide lines) of the oracle and the GPU."""
    name, atmname, mk, grid, region = pin_specs()[0]
    teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS[atmname]
    model = W.eddington_model(teff, logg, ntau)
    state = load_state(atmname)
    extra = mk()
    pgf = np.load(os.path.join(DATA, "atm_%s.npz" % atmname))["probe_loggf"]
    probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
    t = extra._txt
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        probes.write_z(os.path.join(wd, "probes.z"), grid[0], grid[1])
        fsio.write_hdf5_lines(os.path.join(wd, "lines.h5"), extra.species, extra.spc, extra.wl,
                              W.f32_of_text(t["elo"], "%.4f"), W.f32_of_text(t["loggf"], "%.3f"),
                              W.f32_of_text(t["lgrad"], "%.3f"), W.f32_of_text(t["lgqst"], "%.3f"),
                              W.f32_of_text(t["lgvdw"], "%.3f"), provenance="pin_solar seeded list")
        deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=0, 1, 1, 1, 1\nvmic=%.3f\nmolbrd=%d\n"
                "lines=\n-1  probes.z\n-1  lines.h5\n\nmodel=model.krz\nmus=7\n" % (grid + (vmic, molbrd)))
        log = run_ref(wd, deck)
        assert "File: lines.h5" in log and "Lines read: %d" % extra.n in log, log
        lo = fsio.read_opac(os.path.join(wd, "fs_lineop.bin"))
        co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
        sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
        fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(lo[k], state[k]), "EOS state differs from the recovered one: " + k
    wave = lo["wave"]
    sel = (wave >= region[0] - 1e-9) & (wave <= region[1] + 1e-9)
    i0, i1 = (int(x) for x in np.nonzero(sel)[0][[0, -1]])
    np.savez_compressed(
        os.path.join(gold, "pin_solar_h5.npz"), grid=np.array(grid, np.float64), i0=i0, i1=i1, atm=atmname,
        vmicro=vmic, molbrd=molbrd, contopac=co["opac"][i0:i1 + 1], lineopac=lo["opac"][i0:i1 + 1],
        wave=wave[i0:i1 + 1], xmu=sp["xmu"], spl=sp["spl"][i0:i1 + 1], spc=sp["spc"][i0:i1 + 1],
        sfl=fl["sfl"][i0:i1 + 1], sfc=fl["sfc"][i0:i1 + 1],
        **{"txt_" + k: np.asarray(v) for k, v in t.items()}, line_wl=extra.wl, line_spc=extra.spc)
    print("pin_solar_h5: region pixels", i1 - i0 + 1, "lines", extra.n)


def air2vac(lam):
    """Air2Vac (utils.f90:1020-1032) on an array."""
    return np.array([oracle.air2vac(float(x)) for x in np.asarray(lam, np.float64)])


def make_h5vac_pin(gold):
    """Vacuum wavelengths and range selection of HDF5 lists (ReadHDF, ioutils.f90:686-790;
    pin_solar_h5vac.npz): the pin_solar list plus 12 lines above the synthesis range (5045.2-5046.8 A,
    whose wings would reach the region) and 6 below it, all turned to vacuum (Air2Vac) and written with
    WL_VAC = 1; the reference converts back (Vac2Air) and keeps only the lines inside WAVE=."""
    name, atmname, mk, grid, region = pin_specs()[0]
    teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS[atmname]
    model = W.eddington_model(teff, logg, ntau)
    state = load_state(atmname)
    extra = merge([mk(), W.atomic_lines(12, 5045.2, 5046.8, W.SEED0 + 45), W.atomic_lines(6, 4998.0, 4999.8, W.SEED0 + 46)])
    pgf = np.load(os.path.join(DATA, "atm_%s.npz" % atmname))["probe_loggf"]
    probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
    t = extra._txt
    wvac = air2vac(extra.wl)
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        probes.write_z(os.path.join(wd, "probes.z"), grid[0], grid[1])
        path = os.path.join(wd, "lines.h5")
        fsio.write_hdf5_lines(path, extra.species, extra.spc, wvac,
                              W.f32_of_text(t["elo"], "%.4f"), W.f32_of_text(t["loggf"], "%.3f"),
                              W.f32_of_text(t["lgrad"], "%.3f"), W.f32_of_text(t["lgqst"], "%.3f"),
                              W.f32_of_text(t["lgvdw"], "%.3f"), wl_vac=1, provenance="pin_solar list in vacuum")
        deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=0, 1, 1, 1, 1\nvmic=%.3f\nmolbrd=%d\n"
                "lines=\n-1  probes.z\n-1  lines.h5\n\nmodel=model.krz\nmus=7\n" % (grid + (vmic, molbrd)))
        log = run_ref(wd, deck)
        r = fsio.read_hdf5_lines(path, species, wstart=grid[0], wend=grid[1])
        lo = fsio.read_opac(os.path.join(wd, "fs_lineop.bin"))
        co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
        sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
        fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
    assert "Lines read: %d" % len(r["wl"]) in log, log
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(lo[k], state[k]), "EOS state differs from the recovered one: " + k
    wave = lo["wave"]
    sel = (wave >= region[0] - 1e-9) & (wave <= region[1] + 1e-9)
    i0, i1 = (int(x) for x in np.nonzero(sel)[0][[0, -1]])
    g = dict(wmode=grid[3], wstart=grid[0], wend=grid[1], dstep=grid[2])
    S = oracle.State(g, state, contopac=co["opac"], vmicro=vmic, molbrd=molbrd)
    o = oracle.lineop_calc(S, oracle.Lines(**{k: r[k] for k in ("wl", "elo", "gf", "grad", "gqst", "gvdw", "spc",
                                                               "ismol")}, kind=0), list_type=0)
    ref = lo["opac"][i0:i1 + 1]
    m = ref > 0
    mine = o["lineopac"][i0:i1 + 1]
    print("  h5vac pin: %d of %d lines read, pattern equal %s, line opacity max rel %.2e"
          % (len(r["wl"]), extra.n, np.array_equal(mine > 0, m), np.max(np.abs(mine[m] / ref[m] - 1))))
    np.savez_compressed(
        os.path.join(gold, "pin_solar_h5vac.npz"), grid=np.array(grid, np.float64), i0=i0, i1=i1, atm=atmname,
        vmicro=vmic, molbrd=molbrd, contopac=co["opac"][i0:i1 + 1], lineopac=ref, wave=wave[i0:i1 + 1],
        xmu=sp["xmu"], sfl=fl["sfl"][i0:i1 + 1], sfc=fl["sfc"][i0:i1 + 1], nread=len(r["wl"]),
        **{"txt_" + k: np.asarray(v) for k, v in t.items()}, line_wvac=wvac, line_spc=extra.spc)


def zh5_seeded():
    """The Zeeman list of the .zh5 fixture: pin_magnetic's seeded lines with three Lande factors set to
    the converters' 99 (unknown), which the reader turns into unsplit lines."""
    extra = W.zeeman_lines(60, 6040.3, 6042.7, W.SEED0 + 2)
    jlo, jup, glo, gup = (np.asarray(a, np.float32).copy() for a in extra.zeeman)
    glo[[5, 23]] = 99.0
    gup[41] = 99.0
    return extra, (jlo, jup, glo, gup)


def make_zh5_pin(gold):
    """Zeeman HDF5 fixture (pin_magnetic_zh5.npz): the probes and pin_magnetic's seeded lines written by
    fsio.write_hdf5_lines as one .zh5 list (J and Lande factor columns; the reference builds the
    splitting patterns itself, ioutils.f90:997-1031), Stokes IQUV with BFRAME 1, |B| = 2 kG at 60/30 deg,
    9 angles, on 6040-6043 A at 0.002 A."""
    teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS["magnetic"]
    model = W.eddington_model(teff, logg, ntau)
    state = load_state("magnetic")
    grid = (6000.0, 6043.0, 0.002, 0)
    region = (6040.0, 6043.0)
    bfield = (2000.0, 60.0, 30.0)
    extra, z = zh5_seeded()
    pgf = np.load(os.path.join(DATA, "atm_magnetic.npz"))["probe_loggf"]
    probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
    merged = merge([probes, extra])
    npr = probes.n
    zz = [np.concatenate([np.full(npr, v, np.float32), a]) for v, a in zip((1.0, 1.0, 99.0, 99.0), z)]
    t = merged._txt
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        fsio.write_hdf5_lines(os.path.join(wd, "lines.zh5"), merged.species, merged.spc, merged.wl,
                              W.f32_of_text(t["elo"], "%.4f"), W.f32_of_text(t["loggf"], "%.3f"),
                              W.f32_of_text(t["lgrad"], "%.3f"), W.f32_of_text(t["lgqst"], "%.3f"),
                              W.f32_of_text(t["lgvdw"], "%.3f"), zeeman=zz, provenance="pin_magnetic seeded list")
        deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=0, 0, 1, 1, 1\nvmic=%.3f\nmolbrd=%d\n"
                "lines=\n-1  lines.zh5\n\nmodel=model.krz\nmus=9\nbframe=1\nbfield=%g, %g, %g\n"
                % (grid + (vmic, molbrd) + bfield))
        log = run_ref(wd, deck)
        assert "polarised" in log and "Lines read: %d" % merged.n in log, log
        co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
        sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
        fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(co[k], state[k]), "EOS state differs from the recovered one: " + k
    wave = co["wave"]
    sel = (wave >= region[0] - 1e-9) & (wave <= region[1] + 1e-9)
    i0, i1 = (int(x) for x in np.nonzero(sel)[0][[0, -1]])
    te = extra._txt
    np.savez_compressed(
        os.path.join(gold, "pin_magnetic_zh5.npz"), grid=np.array(grid, np.float64), i0=i0, i1=i1,
        atm="magnetic", bframe=1, bfield=np.array(bfield), vmicro=vmic, molbrd=molbrd,
        contopac=co["opac"][i0:i1 + 1], wave=wave[i0:i1 + 1], xmu=sp["xmu"], spz=sp["spz"][i0:i1 + 1],
        spc=sp["spc"][i0:i1 + 1], sfl=fl["sfl"][i0:i1 + 1], sfc=fl["sfc"][i0:i1 + 1],
        line_wl=extra.wl, line_spc=extra.spc, jlo=z[0], jup=z[1], glo=z[2], gup=z[3],
        **{"txt_" + k: np.asarray(v) for k, v in te.items()})
    print("pin_magnetic_zh5: region pixels", i1 - i0 + 1, "lines", merged.n)


MOL_CODES = {"TiO": "0822.000000", "H2O": "010108.000000", "CO": "0608.000000", "OH": "0108.000000"}


def make_mol_h5_pin(gold):
    """Molecular HDF5 fixture (pin_cooldwarf_h5.npz): pin_cooldwarf's seeded lines as four
    single-species molecular lists (fsio.write_hdf5_molecular, the mol2hdf.py layout: no Stark or van
    der Waals columns, GRAD linear with 0 for the classical value), read by the reference program with
    the isotopic factor 1 after the probe list; the region's line opacity, continuum and spectra."""
    name, atmname, mk, grid, region = pin_specs()[1]
    teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS[atmname]
    model = W.eddington_model(teff, logg, ntau)
    state = load_state(atmname)
    extra = mk()
    pgf = np.load(os.path.join(DATA, "atm_%s.npz" % atmname))["probe_loggf"]
    probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
    t = extra._txt
    entries = []
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        probes.write_z(os.path.join(wd, "probes.z"), grid[0], grid[1])
        for k, (nm, ion) in enumerate(species):
            sel = extra.spc == k
            fn = "%s.h5" % nm.lower()
            fsio.write_hdf5_molecular(os.path.join(wd, fn), nm, ion, MOL_CODES[nm], extra.wl[sel],
                                      W.f32_of_text(t["elo"][sel], "%.4f"), W.f32_of_text(t["loggf"][sel], "%.3f"),
                                      np.zeros(int(sel.sum()), np.float32), provenance="pin_cooldwarf seeded list")
            entries.append("1.0  %s" % fn)
        deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=0, 1, 1, 1, 1\nvmic=%.3f\nmolbrd=%d\n"
                "lines=\n-1  probes.z\n%s\n\nmodel=model.krz\nmus=7\n"
                % (grid + (vmic, molbrd) + ("\n".join(entries),)))
        log = run_ref(wd, deck)
        assert all(("File: %s" % e.split()[1]) in log for e in entries), log
        lo = fsio.read_opac(os.path.join(wd, "fs_lineop.bin"))
        co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
        sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
        fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(lo[k], state[k]), "EOS state differs from the recovered one: " + k
    wave = lo["wave"]
    sel = (wave >= region[0] - 1e-9) & (wave <= region[1] + 1e-9)
    i0, i1 = (int(x) for x in np.nonzero(sel)[0][[0, -1]])
    np.savez_compressed(
        os.path.join(gold, "pin_cooldwarf_h5.npz"), grid=np.array(grid, np.float64), i0=i0, i1=i1, atm=atmname,
        vmicro=vmic, molbrd=molbrd, contopac=co["opac"][i0:i1 + 1], lineopac=lo["opac"][i0:i1 + 1],
        wave=wave[i0:i1 + 1], xmu=sp["xmu"], spl=sp["spl"][i0:i1 + 1], spc=sp["spc"][i0:i1 + 1],
        sfl=fl["sfl"][i0:i1 + 1], sfc=fl["sfc"][i0:i1 + 1], line_wl=extra.wl, line_spc=extra.spc,
        **{"txt_" + k: np.asarray(v) for k, v in t.items()})
    print("pin_cooldwarf_h5: region pixels", i1 - i0 + 1, "lines", extra.n)
    print(log[-600:])


# ---- hot atmosphere with tabulated He I Stark lines (hestark.f90) -------------------------------
HOT = dict(teff=15000.0, logg=4.0, ntau=48, species=[("He", 1)], wl0=5000.0, dstep=0.01, vmic=1.0, molbrd=0)
HE_POTION = 24.581


def he_lines(wl, elo, loggf, lgrad=None, lgqst=None, lgvdw=None):
    n = len(wl)
    full = lambda v, d: np.full(n, d) if v is None else np.asarray(v, np.float64)
    return W.LineList(HOT["species"], np.asarray(wl, np.float64), np.asarray(loggf, np.float64),
                      np.asarray(elo, np.float64), full(lgrad, 5.0), full(lgqst, -30.0), full(lgvdw, -30.0),
                      np.zeros(n, np.int32), np.zeros(n, np.int32))


def he_run(model, probes, lines, grid, wd, save_spec=False):
    """Reference run of probes + lines on grid (w0, w1, dstep): (line opacity, continuum[, spec, flux])."""
    merged = merge([probes, lines])
    W.write_krz(os.path.join(wd, "model.krz"), model)
    merged.write_z(os.path.join(wd, "lines.z"), grid[0], grid[1])
    deck = ("wave=%.4f, %.4f, %.6f, 0\nsave=0, 1, 1, %d, %d\nvmic=%.3f\nmolbrd=%d\n"
            "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=%d\n"
            % (grid[0], grid[1], grid[2], int(save_spec), int(save_spec), HOT["vmic"], HOT["molbrd"],
               7 if save_spec else 0))
    log = run_ref(wd, deck)
    out = [fsio.read_opac(os.path.join(wd, "fs_lineop.bin")), fsio.read_opac(os.path.join(wd, "fs_contop.bin"))]
    if save_spec:
        out += [fsio.read_spec(os.path.join(wd, "fs_spec.bin")), fsio.read_flux(os.path.join(wd, "fs_flux.bin"))]
    return out + [log]


def f32_from_bits(b):
    return np.asarray(b, np.int32).view(np.float32)


def recover_he_density(state, co, grid, line, lo_ref, known, target, d_range=(5.0, 12.0)):
    """One FP32 density per depth (H II or He II: `target`) from a single tabulated He I line's reference
    line opacity.  The feature is the line opacity summed over the wing pixels 5-12 A either side of the
    centre, which grows monotonically with the damping parameter while it stays below the pixels' v
    (H ~ a / (sqrt(pi) (a^2 + v^2))), hence with the density between 0 and twice the electron density
    (each proton or He II ion has given an electron); bisection runs on the bit patterns of positive
    FP32 numbers, all depths at once, and ends on the FP32 value of least mismatch among the final
    neighbours."""
    g = dict(wmode=0, wstart=grid[0], wend=grid[1], dstep=grid[2])
    nt = len(state["T"])
    wave = lo_ref["wave"]
    dl = np.abs(wave - line.wl[0])
    px = np.nonzero((dl >= d_range[0]) & (dl <= d_range[1]))[0]
    assert np.all(lo_ref["opac"][px] > 0), "feature pixels outside the reference window"
    s_ref = lo_ref["opac"][px].sum(axis=0)
    L = oracle.Lines(**lines_args(line), kind=2)

    def feature(x32):
        dens = dict(known)
        dens[target] = x32
        hg, hs = oracle.hestark_init(state["T"], state["xne"], dens["hii"], dens["heii"])
        st = oracle.State(g, state, contopac=co, vmicro=HOT["vmic"], molbrd=HOT["molbrd"], hegam=hg,
                          heshf=hs, spc_he1=0)
        r = oracle.lineop_calc(st, L, list_type=2)
        return r["lineopac"][px].sum(axis=0)

    lo_b = np.zeros(nt, np.int64)
    hi_b = (2.0 * state["xne"]).astype(np.float32).view(np.int32).astype(np.int64)
    while np.any(hi_b - lo_b > 1):
        mid = (lo_b + hi_b) // 2
        up = feature(f32_from_bits(mid)) >= s_ref
        hi_b = np.where(up, mid, hi_b)
        lo_b = np.where(up, lo_b, mid)
    best = None
    for cand in (hi_b - 1, hi_b, hi_b + 1):
        dev = np.abs(feature(f32_from_bits(cand)) / s_ref - 1.0)
        if best is None:
            best = (dev, cand.copy())
        else:
            take = dev < best[0]
            best = (np.where(take, dev, best[0]), np.where(take, cand, best[1]))
    return f32_from_bits(best[1]), best[0]


def he_pin_list():
    """Tabulated lines of both tables (3867.5, 3871.79, 3888.7, 3926.53, 3935.9 A), near misses in
    wavelength (> 1 A) and lower level energy (> 0.01 eV), two lines on one entry, and 30 seeded
    He I lines (classical Stark and van der Waals constants given) on 3857-3943 A."""
    tab = [(3867.5, 20.96409), (3871.79, 21.21802), (3888.7, 19.81961), (3926.53, 21.21802), (3935.9, 21.21802)]
    near = [(3890.0, 19.81961),     # 1.3 A from 3888.7: no entry
            (3868.2, 19.81961),     # within 1 A of 3867.5, lower level 1.14 eV off: no entry
            (3926.0, 21.2160),      # second line on entry 35 (0.53 A, 0.002 eV off)
            (3889.65, 19.8196),     # 0.95 A from 3888.7: entry 10
            (3936.95, 21.2180)]     # 1.05 A from 3935.9: no entry
    rng = np.random.default_rng(W.SEED0 + 40)
    nr = 30
    wl = [w for w, _ in tab + near] + list(np.round(rng.uniform(3857.0, 3943.0, nr), 3))
    elo = [e for _, e in tab + near] + list(np.round(rng.uniform(19.5, 23.0, nr), 4))
    loggf = [-0.3, -0.8, 0.2, -1.0, -0.6, -0.5, -0.4, -0.9, -0.7, -0.5] + list(np.round(rng.normal(-1.5, 0.6, nr), 3))
    lgqst = [-30.0] * 10 + list(np.round(rng.uniform(-6.0, -4.5, nr), 3))
    lgvdw = [-30.0] * 10 + list(np.round(rng.uniform(-8.0, -7.0, nr), 3))
    lgrad = [8.5] * 10 + list(np.round(rng.uniform(7.0, 9.0, nr), 3))
    return he_lines(wl, elo, loggf, lgrad, lgqst, lgvdw)


def make_hot_he(gold):
    """Hot atmosphere (Teff 15000 K, log g 4.0, 48 depths, He I only) and the He I Stark pin.

    State: recover() with He I probes at 5000 A (FractionPF, masses, Nprtb).  The proton and He II
    densities that HeStarkInit (hestark.f90:332-370) reads are EOS outputs the program does not write;
    they are recovered from two single-line runs: the DS84 line at 3819.60 A (electrons + protons, no
    He II term) gives Fraction(H II), then the DS90 line at 4471.5 A gives Fraction(He II).
    Pin (pin_hot_he.npz): tabulated lines of both tables (3867.5, 3871.79, 3888.7, 3926.53, 3935.9 A),
    near misses in wavelength (> 1 A) and in lower level energy (> 0.01 eV), two lines matching one entry,
    and seeded non-tabulated He I lines, on 3855-3945 A; the whole grid's line and continuum opacity and
    the spectra."""
    model = W.eddington_model(HOT["teff"], HOT["logg"], HOT["ntau"])
    species = HOT["species"]
    POTION[("He", 1)] = HE_POTION
    with tempfile.TemporaryDirectory() as wd:
        r = recover(model, species, 0, HOT["wl0"], HOT["dstep"], HOT["vmic"], HOT["molbrd"], wd)
    state, atm = r["state"], r["atm"]
    pgf = r["probe_loggf"]
    probes = probe_list(species, HOT["wl0"], 2.0, ismol=0, loggf=pgf)
    nt = len(state["T"])
    known = dict(hii=np.zeros(nt, np.float32), heii=np.zeros(nt, np.float32))
    for target, wl, elo, grid in (("hii", 3819.60, 20.96409, (3805.0, 3835.0, 0.01)),
                                  ("heii", 4471.5, 20.96409, (4455.0, 4488.0, 0.01))):
        grid = (wl - 14.0, wl + 14.0, 0.01)
        line = he_lines([wl], [elo], [0.5])
        with tempfile.TemporaryDirectory() as wd:
            lo, co, _ = he_run(model, probes, line, grid, wd)
        for k in ("rhox", "T", "xne", "xna", "rho"):
            assert np.array_equal(lo[k], state[k]), "EOS state differs: " + k
        x, dev = recover_he_density(state, co["opac"], grid, line, lo, known, target)
        known[target] = x
        print("  %s: %s .. %s, feature mismatch max %.2e (median %.2e)"
              % (target, x[0], x[-1], dev.max(), np.median(dev)))
    # pin run
    pin = he_pin_list()
    grid = (3855.0, 3945.0, 0.05)
    with tempfile.TemporaryDirectory() as wd:
        lo, co, sp, fl, log = he_run(model, probes, pin, grid, wd, save_spec=True)
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(lo[k], state[k]), "EOS state differs: " + k
    g = dict(wmode=0, wstart=grid[0], wend=grid[1], dstep=grid[2])
    hg, hs = oracle.hestark_init(state["T"], state["xne"], known["hii"], known["heii"])
    st = oracle.State(g, state, contopac=co["opac"], vmicro=HOT["vmic"], molbrd=HOT["molbrd"], hegam=hg,
                      heshf=hs, spc_he1=0)
    res = oracle.lineop_calc(st, oracle.Lines(**lines_args(pin), kind=2), list_type=2)
    ref = lo["opac"]
    assert np.array_equal(res["lineopac"] > 0, ref > 0), "window pattern differs"
    m = ref > 0
    rel = np.max(np.abs(res["lineopac"][m] / ref[m] - 1.0))
    ihe = np.array([oracle.he_match_idx(w, e) for w, e in zip(pin.wl, pin.elo)], np.int32)
    print("  pin: %d lines (%d matched), line opacity max rel %.2e" % (pin.n, int((ihe > 0).sum()), rel))
    kidx = np.unique(np.linspace(0, len(co["wave"]) - 1, 61).round().astype(int))
    np.savez_compressed(
        os.path.join(DATA, "atm_hot.npz"), teff=HOT["teff"], logg=HOT["logg"],
        species=np.array(["%s %d" % s for s in species]), ismol=0, vmicro=HOT["vmic"], molbrd=HOT["molbrd"],
        rhox=state["rhox"], T=state["T"], xne=state["xne"], xna=state["xna"], rho=state["rho"],
        fractionpf=state["fractionpf"], xamass=state["xamass"], potion=state["potion"], ion=state["ion"],
        frac_h1=state["frac_h1"], frac_he1=state["frac_he1"], frac_hii=known["hii"], frac_heii=known["heii"],
        nprtb=r["nprtb"], cont_wave=co["wave"][kidx], cont_opac=co["opac"][kidx], probe_rel=r["rel"],
        probe_loggf=pgf, model_rhox=model["rhox"], model_T=model["T"])
    a = pin.arrays()
    np.savez_compressed(
        os.path.join(gold, "pin_hot_he.npz"), grid=np.array(grid + (0,), np.float64), i0=0, i1=len(lo["wave"]) - 1,
        atm="hot", vmicro=HOT["vmic"], molbrd=HOT["molbrd"], contopac=co["opac"], lineopac=ref,
        wave=lo["wave"], xmu=sp["xmu"], spl=sp["spl"], spc=sp["spc"], sfl=fl["sfl"], sfc=fl["sfc"],
        ihe_expected=ihe, **{"line_" + k: v for k, v in a.items()})
    print(log[-400:])


def make_hot_he_mag(gold):
    """Stokes IQUV of the pin_hot_he list as Zeeman lines (seeded J and Lande factors, explicit
    patterns) in the hot atmosphere, BFRAME 1 with |B| = 3 kG at inclination 45 deg and azimuth 20 deg,
    9 angles, on 3855-3945 A at 0.05 A (pin_hot_he_mag.npz).  Pins the tabulated He I widths and shifts
    in the magnetic driver (MagLineOpacity1/2 with the per-depth shift, opacity.f90:391-520)."""
    d = np.load(os.path.join(REPO, "tests", "golden", "pin_hot_he.npz"))
    a = np.load(os.path.join(DATA, "atm_hot.npz"))
    model = W.eddington_model(HOT["teff"], HOT["logg"], HOT["ntau"])
    state = load_state("hot")
    POTION[("He", 1)] = HE_POTION
    # the list alone (He I is the only species, so the EOS inventory is the probe runs')
    merged = he_pin_list()
    rng = np.random.default_rng(W.SEED0 + 41)
    n = merged.n
    jlo = rng.integers(0, 5, n).astype(np.float64)
    jup = np.clip(jlo + rng.integers(-1, 2, n), 0, 4)
    jup[(jlo == 0) & (jup == 0)] = 1.0
    glo, gup = rng.uniform(0.0, 2.5, n), rng.uniform(0.0, 2.5, n)
    merged.zeeman = (W.f32_of_text(jlo, "%.1f"), W.f32_of_text(jup, "%.1f"),
                     W.f32_of_text(glo, "%.3f"), W.f32_of_text(gup, "%.3f"))
    pats = zeeman_blocks(merged)
    grid = (3855.0, 3945.0, 0.05, 0)
    bfield = (3000.0, 45.0, 20.0)
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        merged.write_z(os.path.join(wd, "lines.z"), grid[0], grid[1], patterns=pats)
        deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=0, 0, 1, 1, 1\nvmic=%.3f\nmolbrd=%d\n"
                "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=9\nbframe=1\nbfield=%g, %g, %g\n"
                % (grid + (HOT["vmic"], HOT["molbrd"]) + bfield))
        log = run_ref(wd, deck)
        assert "polarised" in log, log
        co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
        sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
        fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(co[k], state[k]), "EOS state differs from the recovered one: " + k
    assert sp["magnetic"]
    la = merged.arrays()
    assert np.array_equal(la["wl"], d["line_wl"]) and np.array_equal(la["elo"], d["line_elo"])
    comp = mirrored_components(pats)
    g = dict(wmode=0, wstart=grid[0], wend=grid[1], dstep=grid[2])
    hg, hs = oracle.hestark_init(state["T"], state["xne"], a["frac_hii"], a["frac_heii"])
    S = oracle.State(g, state, contopac=co["opac"], vmicro=HOT["vmic"], molbrd=HOT["molbrd"], hegam=hg,
                     heshf=hs, spc_he1=0)
    r = oracle.mag_lineop_calc(S, oracle.Lines(**la, kind=2, zeeman=comp), 1, np.array(bfield))
    spz, spc = oracle.mag_radtran(S, sp["xmu"], 1, np.array(bfield), np.zeros((S.nwl, S.ntau)), r["maglineopac"])
    ic = sp["spc"]
    err = max(np.max(np.abs(spz[:, q] - sp["spz"][:, q]) / ic) for q in range(4))
    print("  magnetic He I pin: %d lines, Stokes max err %.2e of Ic" % (merged.n, err))
    np.savez_compressed(
        os.path.join(gold, "pin_hot_he_mag.npz"), grid=np.array(grid, np.float64), i0=0, i1=len(co["wave"]) - 1,
        atm="hot", bframe=1, bfield=np.array(bfield), vmicro=HOT["vmic"], molbrd=HOT["molbrd"],
        contopac=co["opac"], wave=co["wave"], xmu=sp["xmu"], spz=sp["spz"], spc=sp["spc"], sfl=fl["sfl"],
        sfc=fl["sfc"], z_npi=comp[0], z_nsi=comp[1], z_spl_pi=comp[2], z_str_pi=comp[3], z_spl_si=comp[4],
        z_str_si=comp[5], **{"line_" + k: v for k, v in la.items()})


def recover_potion(atmname, model, species, state, wl0, dstep, vmic, molbrd, probe_loggf):
    """The FP32 ionisation potential PotIon of every atomic species, as the reference's EOS holds it.

    One probe per species 8 A apart (E_low = 0, G_rad 1e5, log gf 2.5 dex above the FractionPF probe,
    a zero Stark constant so XlineSetup takes the classical treatment, opacity.f90:187-193, whose
    constant 2.26e-7 (5.42e-7 for ions) x (Ion^2 Hie / (PotIon - Eup))^2 falls with PotIon).  Per
    species, a bisection over the bit patterns of FP32 numbers in [3, 60] eV matches the probe's line
    opacity summed over its window pixels 0.1 A or more from the centre (the wing grows with the Stark
    width); the value of least profile mismatch among the final neighbours is kept.  Returns the potion
    array and the largest relative profile mismatch per species."""
    n = len(species)
    wl = wl0 + 8.0 * (1 + np.arange(n))
    wend = wl0 + 8.0 * (n + 1)
    L = W.LineList(species, wl, np.asarray(probe_loggf[:n]) + 2.5, np.zeros(n), np.full(n, 5.0), np.zeros(n),
                   np.full(n, -30.0), np.arange(n, dtype=np.int32), np.zeros(n, np.int32))
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        L.write_z(os.path.join(wd, "lines.z"), wl0, wend)
        deck = ("wave=%.4f, %.4f, %.6f, 0\nsave=0, 1, 1, 0, 0\nvmic=%.3f\nmolbrd=%d\n"
                "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=0\n" % (wl0, wend, dstep, vmic, molbrd))
        run_ref(wd, deck)
        lo = fsio.read_opac(os.path.join(wd, "fs_lineop.bin"))
        co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(lo[k], state[k]), "EOS state differs: " + k
    g = dict(wmode=0, wstart=wl0, wend=wend, dstep=dstep)
    wave, ref = lo["wave"], lo["opac"]
    nz = ref.max(axis=1) > 0
    pot = np.asarray(state["potion"], np.float32).copy()
    a = L.arrays()
    devs = []
    for k in range(n):
        Lk = oracle.Lines(**{q: np.ascontiguousarray(v[k:k + 1]) for q, v in a.items()}, kind=2)
        dl = np.abs(wave - wl[k])
        win = nz & (dl < 3.9)
        px = np.nonzero(win & (dl >= 0.1))[0]
        assert len(px) > 0, "probe window narrower than 0.1 A"
        sref = ref[px].sum()

        def profile(p):
            st = dict(state)
            pp = pot.copy()
            pp[k] = p
            st["potion"] = pp
            S = oracle.State(g, st, contopac=co["opac"], vmicro=vmic, molbrd=molbrd)
            return oracle.lineop_calc(S, Lk, list_type=2)["lineopac"]

        lob, hib = int(np.float32(3.0).view(np.int32)), int(np.float32(60.0).view(np.int32))
        while hib - lob > 1:
            mid = (lob + hib) // 2
            if profile(np.int32(mid).view(np.float32))[px].sum() > sref:
                lob = mid
            else:
                hib = mid
        best = None
        m = ref[win] > 0
        for c in (lob - 1, lob, hib, hib + 1):
            p = np.int32(c).view(np.float32)
            dev = np.max(np.abs(profile(p)[win][m] / ref[win][m] - 1))
            if best is None or dev < best[0]:
                best = (dev, p)
        pot[k] = best[1]
        devs.append(best[0])
        print("  %-4s %d  PotIon %.6g (guess %.6g), profile max rel %.1e"
              % (species[k][0], species[k][1], pot[k], state["potion"][k], best[0]))
    return pot, np.array(devs)


def make_modes_pin(gold):
    """Broadening modes and options (pin_solar_modes.npz): the pin_solar list with a quarter of its lines
    on the classical Stark constant (zero Stark input), a quarter on Unsold van der Waals (zero input),
    one in eight on ABO (sigma.alpha above 10), run with EPSOPAC 3e-3 and VWFUDGE 1.8 (opacity.f90:
    185-227, 239-293); needs the recovered ionisation potentials."""
    name, atmname, mk, grid, region = pin_specs()[0]
    teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS[atmname]
    model = W.eddington_model(teff, logg, ntau)
    state = load_state(atmname)
    base = mk()
    t = base._txt
    lgq = np.array(t["lgqst"], np.float64)
    lgv = np.array(t["lgvdw"], np.float64)
    lgq[1::4] = 0.0
    lgv[2::4] = 0.0
    rng = np.random.default_rng(W.SEED0 + 42)
    abo = np.arange(3, base.n, 8)
    lgv[abo] = np.round(rng.uniform(200.0, 400.0, len(abo))) + np.round(rng.uniform(0.2, 0.4, len(abo)), 3)
    extra = W.LineList(species, base.wl, t["loggf"], t["elo"], t["lgrad"], lgq, lgv, base.spc, base.ismol)
    pgf = np.load(os.path.join(DATA, "atm_%s.npz" % atmname))["probe_loggf"]
    probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
    merged = merge([probes, extra])
    eps, vwf = 3e-3, 1.8
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        merged.write_z(os.path.join(wd, "lines.z"), grid[0], grid[1])
        deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=0, 1, 1, 1, 1\nvmic=%.3f\nmolbrd=%d\nepsopac=%g\nvwfudge=%g\n"
                "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=7\n" % (grid + (vmic, molbrd, eps, vwf)))
        run_ref(wd, deck)
        lo = fsio.read_opac(os.path.join(wd, "fs_lineop.bin"))
        co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
        sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
        fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(lo[k], state[k]), "EOS state differs from the recovered one: " + k
    wave = lo["wave"]
    sel = (wave >= region[0] - 1e-9) & (wave <= region[1] + 1e-9)
    i0, i1 = (int(x) for x in np.nonzero(sel)[0][[0, -1]])
    g = dict(wmode=grid[3], wstart=grid[0], wend=grid[1], dstep=grid[2])
    S = oracle.State(g, state, contopac=co["opac"], vmicro=vmic, molbrd=molbrd, epsopac=eps, vwfudge=vwf)
    r = oracle.lineop_calc(S, oracle.Lines(**lines_args(merged), kind=2), list_type=2)
    ref = lo["opac"]
    m = ref > 0
    print("  modes pin: pattern equal %s, line opacity max rel %.2e"
          % (np.array_equal(r["lineopac"] > 0, m), np.max(np.abs(r["lineopac"][m] / ref[m] - 1))))
    a = extra.arrays()
    np.savez_compressed(
        os.path.join(gold, "pin_solar_modes.npz"),
        grid=np.array(grid, np.float64), i0=i0, i1=i1, atm=atmname, epsopac=eps, vwfudge=vwf,
        species=np.array(["%s %d" % s for s in species]), vmicro=vmic, molbrd=molbrd,
        contopac=co["opac"][i0:i1 + 1], lineopac=ref[i0:i1 + 1], wave=wave[i0:i1 + 1], xmu=sp["xmu"],
        spl=sp["spl"][i0:i1 + 1], spc=sp["spc"][i0:i1 + 1], sfl=fl["sfl"][i0:i1 + 1], sfc=fl["sfc"][i0:i1 + 1],
        **{"line_" + k: v for k, v in a.items()})


def update_h2(name="cooldwarf", h2brd=1.0):
    """The H2 molecule density Fraction(Hmol) of a state, which XlineInit adds to the van der Waals
    perturbers with weight H2Brd * 0.874307 (opacity.f90:82): the recover() probes run again with
    H2BRD set; the van der Waals probe's centre gives the perturber density as in recover(), and its
    excess over the H2-free one, / (H2Brd * 0.874307), is the FP32 density.  The oracle must then
    reproduce the whole probe run with H2BRD."""
    teff, logg, ntau, species, ismol, wl0, dstep, vmic, molbrd, _, _ = CONFIGS[name]
    path = os.path.join(DATA, "atm_%s.npz" % name)
    d = dict(np.load(path))
    model = W.eddington_model(teff, logg, ntau)
    state = load_state(name)
    nsp = len(species)
    probes = probe_list(species, wl0, 2.0, vdw_species=0, ismol=ismol, loggf=d["probe_loggf"])
    wend = wl0 + 2.0 * (nsp + 2)
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        probes.write_z(os.path.join(wd, "lines.z"), wl0, wend)
        deck = ("wave=%.4f, %.4f, %.6f, 0\nsave=0, 1, 1, 0, 0\nvmic=%.3f\nmolbrd=%d\nh2brd=%g\n"
                "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=0\n" % (wl0, wend, dstep, vmic, molbrd, h2brd))
        run_ref(wd, deck)
        lo = fsio.read_opac(os.path.join(wd, "fs_lineop.bin"))
        co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(lo[k], state[k]), "EOS state differs: " + k
    grid = dict(wmode=0, wstart=wl0, wend=wend, dstep=dstep)
    st = oracle.State(grid, state, contopac=co["opac"], vmicro=vmic, molbrd=molbrd)
    L = oracle.Lines(**lines_args(probes), kind=2)
    kv = nsp
    cop, vv, av0 = oracle.xline(st, L, kv)
    wave = st.wave + st.wfirst
    ic = int(np.argmin(np.abs(wave - probes.wl[kv])))
    a = invert_h0(lo["opac"][ic] / cop, av0)
    WaveL = probes.wl[kv]
    dopl = 1.0 / (vv * WaveL)
    gam = a * (dopl / WaveL * (4.0 * 299792.458e13 * np.pi))
    nprtb = (gam - float(probes.grad[kv])) / (float(probes.gvdw[kv]) * (lo["T"] / 1e4) ** 0.3)
    base = state["frac_h1"].astype(np.float64) + 0.412265 * state["frac_he1"].astype(np.float64)
    frac_h2 = ((nprtb - base) / (h2brd * 0.874307)).astype(np.float32)
    st2 = dict(state, frac_h2=frac_h2)
    S = oracle.State(grid, st2, contopac=co["opac"], vmicro=vmic, molbrd=molbrd, h2brd=h2brd)
    r = oracle.lineop_calc(S, L, list_type=2)
    m = lo["opac"] > 0
    rel = np.max(np.abs(r["lineopac"][m] / lo["opac"][m] - 1))
    print("  %s: n(H2) %.3e .. %.3e (%.0f%% .. %.0f%% of the perturbers), probe run reproduced to %.1e"
          % (name, frac_h2[0], frac_h2[-1], 100 * h2brd * 0.874307 * frac_h2[0] / nprtb[0],
             100 * h2brd * 0.874307 * frac_h2[-1] / nprtb[-1], rel))
    d["frac_h2"] = frac_h2
    d["h2_probe_rel"] = rel
    np.savez_compressed(path, **d)


def make_mol_opts_pin(gold):
    """Molecular broadening options (pin_cooldwarf_opts.npz): the pin_cooldwarf list with H2BRD 1.5 (H2 in
    the van der Waals perturbers, opacity.f90:82) and VWMOL 4e-8 (one van der Waals constant for every
    molecular line, opacity.f90:229-234), MolBrd on; needs the recovered H2 density."""
    name, atmname, mk, grid, region = pin_specs()[1]
    teff, logg, ntau, species, ismol, _, _, vmic, molbrd, _, _ = CONFIGS[atmname]
    model = W.eddington_model(teff, logg, ntau)
    state = load_state(atmname)
    extra = mk()
    pgf = np.load(os.path.join(DATA, "atm_%s.npz" % atmname))["probe_loggf"]
    probes = probe_list(species, grid[0], 2.0, ismol=ismol, loggf=pgf)
    merged = merge([probes, extra])
    h2brd, vwmol = 1.5, 4e-8
    with tempfile.TemporaryDirectory() as wd:
        W.write_krz(os.path.join(wd, "model.krz"), model)
        merged.write_z(os.path.join(wd, "lines.z"), grid[0], grid[1])
        deck = ("wave=%.4f, %.4f, %.6f, %d\nsave=0, 1, 1, 1, 1\nvmic=%.3f\nmolbrd=%d\nh2brd=%g\nvwmol=%g\n"
                "lines=\n-1  lines.z\n\nmodel=model.krz\nmus=7\n" % (grid + (vmic, molbrd, h2brd, vwmol)))
        run_ref(wd, deck)
        lo = fsio.read_opac(os.path.join(wd, "fs_lineop.bin"))
        co = fsio.read_opac(os.path.join(wd, "fs_contop.bin"))
        sp = fsio.read_spec(os.path.join(wd, "fs_spec.bin"))
        fl = fsio.read_flux(os.path.join(wd, "fs_flux.bin"))
    for k in ("rhox", "T", "xne", "xna", "rho"):
        assert np.array_equal(lo[k], state[k]), "EOS state differs from the recovered one: " + k
    wave = lo["wave"]
    sel = (wave >= region[0] - 1e-9) & (wave <= region[1] + 1e-9)
    i0, i1 = (int(x) for x in np.nonzero(sel)[0][[0, -1]])
    g = dict(wmode=grid[3], wstart=grid[0], wend=grid[1], dstep=grid[2])
    S = oracle.State(g, state, contopac=co["opac"], vmicro=vmic, molbrd=molbrd, h2brd=h2brd, vwmol=vwmol)
    r = oracle.lineop_calc(S, oracle.Lines(**lines_args(merged), kind=2), list_type=2)
    ref = lo["opac"][i0:i1 + 1]
    m = ref > 0
    lor = r["lineopac"][i0:i1 + 1]
    print("  molecular options pin: pattern equal %s, line opacity max rel %.2e"
          % (np.array_equal(lor > 0, m), np.max(np.abs(lor[m] / ref[m] - 1))))
    a = extra.arrays()
    np.savez_compressed(
        os.path.join(gold, "pin_cooldwarf_opts.npz"),
        grid=np.array(grid, np.float64), i0=i0, i1=i1, atm=atmname, h2brd=h2brd, vwmol=vwmol,
        species=np.array(["%s %d" % s for s in species]), vmicro=vmic, molbrd=molbrd,
        contopac=co["opac"][i0:i1 + 1], lineopac=ref, wave=wave[i0:i1 + 1], xmu=sp["xmu"],
        spl=sp["spl"][i0:i1 + 1], spc=sp["spc"][i0:i1 + 1], sfl=fl["sfl"][i0:i1 + 1], sfc=fl["sfc"][i0:i1 + 1],
        **{"line_" + k: v for k, v in a.items()})


def update_potion():
    """Replace the guessed ionisation potentials of the atomic atmospheres' states with the recovered
    ones (atm_solar, atm_magnetic, atm_hot)."""
    for name in ("solar", "magnetic", "hot"):
        path = os.path.join(DATA, "atm_%s.npz" % name)
        d = dict(np.load(path))
        if name == "hot":
            teff, logg, ntau, species, wl0, dstep, vmic, molbrd = (HOT["teff"], HOT["logg"], HOT["ntau"],
                                                                   HOT["species"], HOT["wl0"], HOT["dstep"],
                                                                   HOT["vmic"], HOT["molbrd"])
        else:
            teff, logg, ntau, species, _, wl0, dstep, vmic, molbrd, _, _ = CONFIGS[name]
        print(name)
        model = W.eddington_model(teff, logg, ntau)
        pot, dev = recover_potion(name, model, species, load_state(name), wl0, dstep, vmic, molbrd,
                                  d["probe_loggf"])
        assert dev.max() < 1e-12, "ionisation potential not recovered"
        d["potion"] = pot
        d["potion_profile_dev"] = dev
        np.savez_compressed(path, **d)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "potion":
        update_potion()
    elif len(sys.argv) > 1 and sys.argv[1] == "h2":
        update_h2()
    elif len(sys.argv) > 1 and sys.argv[1] == "molopts":
        make_mol_opts_pin(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "modes":
        make_modes_pin(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "hot":
        make_hot_he(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "hotmag":
        make_hot_he_mag(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "molh5":
        make_mol_h5_pin(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "zh5":
        make_zh5_pin(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "h5":
        make_h5_pin(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "sphere":
        make_sphere_pins(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "magpin":
        make_mag_pin(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "convol":
        make_convol_pin(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "reentry":
        make_reentry_pin(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "h5vac":
        make_h5vac_pin(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "magframes":
        make_mag_frames_pin(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "maglinst":
        make_mag_linst_pin(os.path.join(REPO, "tests", "golden"))
    elif len(sys.argv) > 1 and sys.argv[1] == "linst":
        make_linst_pins(os.path.join(REPO, "tests", "golden"))
    else:
        main()
        make_mag_pin(os.path.join(REPO, "tests", "golden"))
