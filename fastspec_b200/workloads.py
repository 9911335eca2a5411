"""Seeded synthetic workloads: model atmospheres and line lists.

No public benchmark is involved: every line below is generated from numpy's PCG64 with seed
20261203 + config, using the distributions of the five benchmark configurations (solar-type
atomic synthesis, cool-dwarf molecular synthesis, polarised Zeeman synthesis, a batched grid
and a differentiable fit).

Line records carry exactly the FP32 values the reference's ASCII reader stores
(ioutils.f90:1436-1466): gf = 10.0**loggf, Grad = 10.0**x for 0 < x < 20, Gqst/Gvdw =
10.0**x for x < 0, all in single precision through the C library's powf, applied to the FP32
parse of the printed decimal.  The same records can therefore be written as a `.z` file for
the reference program and uploaded to the GPU path bit-identically.
"""
import ctypes
import ctypes.util
import math
import os

import numpy as np

KBOLT = 1.380649e-16
AMU = 1.66053906660e-24
SEED0 = 20261203

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.powf.restype = ctypes.c_float
_libm.powf.argtypes = [ctypes.c_float, ctypes.c_float]


def pow10f(x):
    """Single-precision 10.0**x as the reference's REAL(4) exponentiation (libm powf)."""
    x = np.asarray(x, dtype=np.float32)
    out = np.empty(x.shape, np.float32)
    flat = x.ravel(); o = out.ravel()
    pw = _libm.powf
    for i in range(flat.size):
        o[i] = pw(10.0, float(flat[i]))
    return out


def f32_of_text(values, fmt):
    """FP32 value the reference parses from each number printed with `fmt`."""
    return np.array([np.float32(fmt % v) for v in np.asarray(values, dtype=np.float64)], np.float32)


# ---- model atmospheres ------------------------------------------------------------------------

# Asplund et al. (2021) log(N_el/N_tot) pattern of the reference (shared.f90:72-90), first 30
SOLAR30 = [0.923, -1.121, -11.07, -10.65, -9.33, -3.57, -4.20, -3.34, -7.63, -3.97, -5.81,
           -4.48, -5.60, -4.52, -6.62, -4.91, -6.72, -5.65, -6.96, -5.73, -8.89, -7.06, -8.13,
           -6.41, -6.61, -4.57, -7.09, -5.83, -7.85, -7.47]


def eddington_model(teff, logg, ntau, logtau_min=-5.0, logtau_max=2.0, metal=1e-4):
    """Eddington-grey plane-parallel model in hydrostatic equilibrium.

    T^4 = 3/4 Teff^4 (tau + 2/3) on a log tau grid.  dP/dtau = g / kappa with an H-minus
    bound-free opacity fit, kappa = 2.5e-31 (rho^0.5) T^9 cm^2/g for T <= 6000 K continued
    as T^3 above it, plus electron scattering; the fit only shapes P(tau) for this synthetic
    model (the reference re-solves the equation of state from Pgas = (Xna + Xne) k T).
    The electron density is a Saha estimate for hydrogen plus a metal donor of ionisation
    potential 7.9 eV at relative abundance `metal`.
    """
    g = 10.0 ** logg
    lt = np.linspace(logtau_min, logtau_max, ntau)
    tau = 10.0 ** lt
    T = (0.75 * teff ** 4 * (tau + 2.0 / 3.0)) ** 0.25
    mu = 1.3

    def kappa(P, T):
        rho = P * mu * AMU / (KBOLT * T)
        Tt = min(T, 6000.0)
        k = 2.5e-31 * math.sqrt(max(rho, 1e-30)) * Tt ** 9
        if T > 6000.0:
            k *= (T / 6000.0) ** 3
        return k + 0.03 + 1e-4

    # integrate d ln P / d ln tau = g tau / (kappa P) from a self-consistent top boundary
    P = g * tau[0] / 1.0
    for _ in range(50):
        P = g * tau[0] / kappa(P, T[0])
    Ps = [P]
    for i in range(1, ntau):
        x0, x1 = math.log(tau[i - 1]), math.log(tau[i])
        h = (x1 - x0) / 8.0
        y = math.log(Ps[-1])
        Tl = lambda x: (0.75 * teff ** 4 * (math.exp(x) + 2.0 / 3.0)) ** 0.25
        f = lambda x, y: g * math.exp(x) / (kappa(math.exp(y), Tl(x)) * math.exp(y))
        x = x0
        for _ in range(8):
            k1 = f(x, y); k2 = f(x + h / 2, y + h * k1 / 2); k3 = f(x + h / 2, y + h * k2 / 2)
            k4 = f(x + h, y + h * k3)
            y += h * (k1 + 2 * k2 + 2 * k3 + k4) / 6.0
            x += h
        Ps.append(math.exp(y))
    Pg = np.array(Ps)
    ntot = Pg / (KBOLT * T)
    # Saha electron density: hydrogen (13.6 eV) + metal donor (7.9 eV)
    xne = np.empty(ntau)
    for i in range(ntau):
        ne = 1e10
        for _ in range(200):
            def phi(chi, u):
                return 2.4148e15 * T[i] ** 1.5 * math.exp(-chi * 11604.518 / T[i]) * u
            fH = phi(13.598, 1.0) / (phi(13.598, 1.0) + ne)
            fM = phi(7.9, 1.0) / (phi(7.9, 1.0) + ne)
            nh = 0.92 * ntot[i]
            new = nh * fH + metal * ntot[i] * fM
            if abs(new - ne) <= 1e-10 * ne:
                ne = new
                break
            ne = math.sqrt(ne * max(new, 1.0))
        xne[i] = ne
    xna = ntot - xne
    rho = xna * mu * AMU
    rhox = Pg / g
    return dict(teff=float(teff), logg=float(logg), ntau=ntau, logtau=lt, rhox=rhox, T=T,
                xne=xne, xna=xna, rho=rho)


def write_krz(path, model, abund=None, title="synthetic Eddington-grey model", radius=None, height=None):
    """Write a `.krz` model (the format ReadModel parses, ioutils.f90:1614-1748): plane-parallel, or
    spherical with `radius` [cm] in the header and the layer heights [cm] as a sixth column."""
    ab = list(abund if abund is not None else SOLAR30) + [-20.0] * (99 - len(SOLAR30))
    sph = radius is not None and radius > 0
    with open(path, "w") as f:
        f.write("TITLE %s\n" % title)
        geo = ("SPHERICAL RADIUS= %.9E" % radius) if sph else "PLANE-PARALLEL."
        f.write("T EFF= %.0f. GRAV= %.2f  MODEL TYPE= 0 WLSTD= 5000 %s\n" % (model["teff"], model["logg"], geo))
        f.write(" 1 1 1 1 1 1 1 1 1 1 1 1 1 0 1 0 0 0 0 0 - OPACITY SWITCHES\n")
        for i in range(0, 99, 10):
            f.write(" ".join("%7.3f" % a for a in ab[i:i + 10]))
            f.write(" %d\n" % model["ntau"] if i + 10 >= 99 else "\n")
        for i in range(model["ntau"]):
            f.write(" %.9E, %8.1f, %.6E, %.6E, %.6E," % (
                model["rhox"][i], model["T"][i], model["xne"][i], model["xna"][i], model["rho"][i]))
            f.write(" %.9E,\n" % height[i] if sph else "\n")


def model_heights(rhox, rho):
    """Layer heights [cm] of a hydrostatic model, 0 at the top and decreasing inward:
    dh = -d(rhox) / rho by the trapezoid rule in 1/rho."""
    rhox = np.asarray(rhox, np.float64); rho = np.asarray(rho, np.float64)
    dh = np.diff(rhox) * 0.5 * (1.0 / rho[1:] + 1.0 / rho[:-1])
    return -np.concatenate([[0.0], np.cumsum(dh)])


# ---- line lists ------------------------------------------------------------------------------

# species tables: (name, ion, atomic/molecular mass) in the order their indices are used
ATOMIC_C0 = [("Fe", 1), ("Fe", 2), ("Ti", 1), ("Cr", 1), ("Ni", 1), ("Ca", 1)]
ATOMIC_C0_P = [0.5, 0.1, 0.1, 0.1, 0.1, 0.1]
MOLECULES_C1 = [("TiO", 1), ("H2O", 1), ("CO", 1), ("OH", 1)]


class LineList:
    """SoA line list with the reference's stored FP32 fields.

    wl (f8), elo/gf/grad/gqst/gvdw (f4, linear as stored), spc (species index into
    `species`), ismol, and the printed log values used to write the ASCII file.
    Zeeman components (optional): npi, nsi (int), comp arrays CSR by line.
    """

    def __init__(self, species, wl, loggf, elo, lgrad, lgqst, lgvdw, spc, ismol, zeeman=None, exact=True):
        """exact=True: values as the reference parses the printed decimals (libm powf, for
        lists that are also run through the reference); exact=False: FP32 rounding and numpy's
        vectorised power (large benchmark lists that only the GPU path and the oracle read)."""
        self.species = species
        order = np.argsort(wl, kind="stable")
        self.wl = np.asarray(wl, np.float64)[order]
        self._txt = dict(loggf=np.asarray(loggf)[order], elo=np.asarray(elo)[order],
                         lgrad=np.asarray(lgrad)[order], lgqst=np.asarray(lgqst)[order],
                         lgvdw=np.asarray(lgvdw)[order])
        self.spc = np.asarray(spc, np.int32)[order]
        self.ismol = np.asarray(ismol, np.int32)[order]
        t = self._txt
        if exact:
            conv, p10 = f32_of_text, pow10f
        else:
            conv = lambda v, fmt: np.asarray(v, np.float32)
            p10 = lambda v: np.power(np.float32(10.0), np.asarray(v, np.float32)).astype(np.float32)
        self.elo = conv(t["elo"], "%.4f")
        self.gf = p10(conv(t["loggf"], "%.3f"))
        lg = conv(t["lgrad"], "%.3f")
        self.grad = np.where((lg < 20.0) & (lg > 0.0), p10(lg), lg).astype(np.float32)
        lq = conv(t["lgqst"], "%.3f")
        self.gqst = np.where(lq < 0.0, p10(lq), lq).astype(np.float32)
        lv = conv(t["lgvdw"], "%.3f")
        self.gvdw = np.where(lv < 0.0, p10(lv), lv).astype(np.float32)
        if not exact:
            self._txt = None
        self.zeeman = None
        if zeeman is not None:
            jlo, jup, glo, gup = (np.asarray(a)[order] for a in zeeman)
            self.zeeman = (jlo, jup, glo, gup)
        self.n = len(self.wl)

    def write_z(self, path, wstart, wend, patterns=None):
        """ASCII list in the VALD-short / .z layout parsed by ReadAscMag (ioutils.f90:1194-1571).

        patterns: per-line (spi, rpi, ssig_half, rsig_half) Zeeman blocks written after a
        Lande factor below -10, with the sigma block holding the red half (ioutils.f90:1324-1410).
        """
        t = self._txt
        with open(path, "w") as f:
            f.write(" %.5f, %.5f, %d, %d, 1.0, Wavelength region, lines selected, lines processed, Vmicro\n"
                    % (wstart, wend, self.n, self.n))
            f.write("                                                   Damping parameters    Lande  Central\n")
            f.write(" Spec Ion       WL(A)   Excit(eV) Vmic  log gf*   Rad.   Stark  Waals  factor  depth  Reference\n")
            for i in range(self.n):
                nm, ion = self.species[self.spc[i]]
                lande = -99.0 if patterns is not None else 99.0
                f.write("'%s %d',%18.10f,%9.4f, 1.0,%8.3f,%8.3f,%8.3f,%8.3f,%8.3f, 0.500, 'syn'\n"
                        % (nm, ion, self.wl[i], t["elo"][i], t["loggf"][i], t["lgrad"][i],
                           t["lgqst"][i], t["lgvdw"][i], lande))
                if patterns is not None:
                    spi, rpi, ssh, rsh = patterns[i]
                    f.write("%d %s\n" % (len(spi), " ".join("%.9g" % x for x in spi)))
                    f.write("%s\n" % " ".join("%.9g" % x for x in rpi))
                    f.write("%d %s\n" % (len(ssh), " ".join("%.9g" % x for x in ssh)))
                    f.write("%s\n" % " ".join("%.9g" % x for x in rsh))
            f.write("'References:'\n")

    def arrays(self):
        return dict(wl=self.wl, elo=self.elo, gf=self.gf, grad=self.grad, gqst=self.gqst,
                    gvdw=self.gvdw, spc=self.spc, ismol=self.ismol)


def atomic_lines(n, wmin, wmax, seed, species=ATOMIC_C0, probs=ATOMIC_C0_P, exact=True):
    """Config-0 distributions: lambda0 ~ U, species mix, log gf ~ N(-2, 1.2) clipped [-6, 1],
    E_low ~ U(0, 6) eV, log Grad ~ U(7, 9), log G4/Ne ~ U(-7, -4), log G6/NH ~ U(-8, -7)."""
    rng = np.random.default_rng(seed)
    wl = rng.uniform(wmin, wmax, n)
    spc = rng.choice(len(species), size=n, p=probs)
    loggf = np.clip(rng.normal(-2.0, 1.2, n), -6.0, 1.0)
    elo = rng.uniform(0.0, 6.0, n)
    lgrad = rng.uniform(7.0, 9.0, n)
    lgqst = rng.uniform(-7.0, -4.0, n)
    lgvdw = rng.uniform(-8.0, -7.0, n)
    return LineList(species, wl, loggf, elo, lgrad, lgqst, lgvdw, spc, np.zeros(n, np.int32), exact=exact)


def molecular_lines(n, wmin, wmax, seed, species=MOLECULES_C1, exact=True):
    """Config-1 distributions: wavenumber uniform over [1e8/wmax, 1e8/wmin] cm^-1 (lambda in A),
    four species at 25 % each, log gf ~ N(-5, 1.5), E_low ~ Exp(1 eV) capped at 5 eV,
    log G6/NH ~ U(-8, -7), radiative damping from the classical fallback (Grad = 0)."""
    rng = np.random.default_rng(seed)
    sigma = rng.uniform(1e8 / wmax, 1e8 / wmin, n)
    wl = 1e8 / sigma
    spc = rng.integers(0, len(species), n)
    loggf = rng.normal(-5.0, 1.5, n)
    elo = np.minimum(rng.exponential(1.0, n), 5.0)
    lgvdw = rng.uniform(-8.0, -7.0, n)
    z = np.zeros(n, np.float32)
    return LineList(species, wl, loggf, elo, z, z, lgvdw, spc, np.ones(n, np.int32), exact=exact)


def zeeman_lines(n, wmin, wmax, seed):
    """Config-2: config-0 parameters plus Lande g_up, g_lo ~ U(0, 2.5) and J in {0..4} with
    Delta J in {-1, 0, 1}, excluding 0 -> 0."""
    L = atomic_lines(n, wmin, wmax, seed)
    rng = np.random.default_rng(seed + 1000)
    jlo = rng.integers(0, 5, n).astype(np.float64)
    dj = rng.integers(-1, 2, n)
    jup = np.clip(jlo + dj, 0, 4)
    bad = (jlo == 0) & (jup == 0)
    jup[bad] = 1.0
    glo = rng.uniform(0.0, 2.5, n)
    gup = rng.uniform(0.0, 2.5, n)
    L.zeeman = (f32_of_text(jlo, "%.1f"), f32_of_text(jup, "%.1f"),
                f32_of_text(glo, "%.3f"), f32_of_text(gup, "%.3f"))
    return L


def zeeman_components(L, pattern):
    """Zeeman components of a zeeman_lines list in the CSR form of fsg_lines: pi as the pattern gives
    them, sigma mirrored (blue = -shift first, then red) as the reader stores an explicit block
    (ioutils.f90:1393-1410).  pattern(jlo, jup, glo, gup) -> (pi shifts, pi strengths, sigma shifts,
    sigma strengths), e.g. fastspec_b200.zeeman_pattern; a line without pi or sigma components
    takes the normal triplet of J 1 -> 0, g = 1."""
    jlo, jup, glo, gup = L.zeeman
    npi, nsi, spl_pi, str_pi, spl_si, str_si = [], [], [], [], [], []
    for i in range(L.n):
        spi, rpi, ss, rs = pattern(float(jlo[i]), float(jup[i]), float(glo[i]), float(gup[i]))
        if len(spi) == 0 or len(ss) == 0:
            spi, rpi, ss, rs = pattern(1.0, 0.0, 1.0, 1.0)
        npi.append(len(spi)); nsi.append(2 * len(ss))
        spl_pi += list(spi); str_pi += list(rpi)
        spl_si += list(-np.asarray(ss)) + list(ss); str_si += list(rs) + list(rs)
    f = lambda a: np.asarray(a, np.float32)
    return (np.asarray(npi, np.int32), np.asarray(nsi, np.int32), f(spl_pi), f(str_pi), f(spl_si), f(str_si))


# ---- batched grid: many atmospheres sharing one atomic line list -------------------------------
# Element of each config-0 species and the solar-state file the batch states are derived from.
_BATCH_ELEMENTS = ["Fe", "Ti", "Cr", "Ni", "Ca"]
_R_BATCH = 5.0e5


def _solar_state():
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "atm_solar.npz"))
    return {k: d[k] for k in d.files}


def batch_atmosphere(teff, logg, ntau, abund, base=None):
    """Atmospheric state of one member of the batched grid, derived from the solar state (EOS of the
    reference, 56 depths) by a documented stand-in for the host EOS: quantities interpolated to
    ntau depths over the same log tau range; T scaled by Teff / 5777; densities by (g / g_sun)^0.6;
    electron density additionally by (Teff / 5777)^6; FractionPF of neutral species by the Saha
    factor Ne (T_sun / T)^1.5 exp(5040 chi (1/T - 1/T_sun)) relative to the solar state, of ions
    unchanged, both times the element's abundance factor 10^abund[element]; the continuum opacity
    knots scale with the electron density (H-minus).  abund: dict element -> dex offset.
    Returns (state dict for Context.set_atmosphere, continuum dict(cont_wave, cont_opac))."""
    s = _solar_state() if base is None else base
    n0 = len(s["T"])
    x0 = np.linspace(0.0, 1.0, n0)
    x = np.linspace(0.0, 1.0, ntau)
    li = lambda v: np.exp(np.interp(x, x0, np.log(np.abs(v) + 1e-300)))
    ft = teff / 5777.0
    fg = 10.0 ** (0.6 * (logg - 4.44))
    T = np.interp(x, x0, s["T"]) * ft
    Tsun = np.interp(x, x0, s["T"])
    xne = li(s["xne"]) * fg * ft ** 6
    xne_sun = li(s["xne"])
    st = dict(rhox=li(s["rhox"]) * fg, T=T, xne=xne, xna=li(s["xna"]) * fg, rho=li(s["rho"]) * fg,
              xamass=s["xamass"].astype(np.float32), potion=s["potion"].astype(np.float32),
              ion=s["ion"].astype(np.int32),
              frac_h1=(li(s["frac_h1"]) * fg).astype(np.float32),
              frac_he1=(np.interp(x, x0, s["frac_he1"]) * fg).astype(np.float32),
              frac_h2=np.zeros(ntau, np.float32))
    fpf = np.empty((ntau, len(s["species"])), np.float32)
    for k, name in enumerate(s["species"]):
        el, ion = str(name).split()
        base_f = li(s["fractionpf"][:, k])
        f = base_f * 10.0 ** abund.get(el, 0.0)
        if int(ion) == 1:
            chi = float(s["potion"][k])
            f = f * (xne / xne_sun) * (Tsun / T) ** 1.5 * np.exp(5040.0 * chi * (1.0 / T - 1.0 / Tsun))
        fpf[:, k] = f
    st["fractionpf"] = fpf
    ko = np.empty((len(s["cont_wave"]), ntau))
    lk = np.log(s["cont_opac"])
    for w in range(lk.shape[0]):
        ko[w] = np.exp(np.interp(x, x0, lk[w])) * (xne / xne_sun)
    return st, dict(cont_wave=s["cont_wave"], cont_opac=ko)


def batch_grid(n=256, seed=SEED0 + 3):
    """The batched configuration: n atmospheres with depth counts U{48..80}, Teff U(3800, 7500) K,
    log g U(3.5, 5.0), abundance offsets N(0, 0.2) dex per element, and wavelength spans U(20, 200) A
    at R = 5e5 (Wmode 1, dstep = c / R) starting U(3000, 9000 - span).  Returns a list of dicts
    (teff, logg, ntau, abund, grid dict, state, cont)."""
    rng = np.random.default_rng(seed)
    base = _solar_state()
    out = []
    for i in range(n):
        ntau = int(rng.integers(48, 81))
        teff = float(rng.uniform(3800.0, 7500.0))
        logg = float(rng.uniform(3.5, 5.0))
        abund = {el: float(v) for el, v in zip(_BATCH_ELEMENTS, rng.normal(0.0, 0.2, len(_BATCH_ELEMENTS)))}
        span = float(rng.uniform(20.0, 200.0))
        w0 = float(rng.uniform(3000.0, 9000.0 - span))
        st, cont = batch_atmosphere(teff, logg, ntau, abund, base)
        grid = dict(wmode=1, wstart=w0, wend=w0 + span, dstep=2.99792458e5 / _R_BATCH)
        out.append(dict(teff=teff, logg=logg, ntau=ntau, abund=abund, grid=grid, state=st, cont=cont))
    return out
