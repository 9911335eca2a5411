"""ctypes binding of the CPU FP64 oracle (oracle/fs_oracle.c).

TEST INFRASTRUCTURE ONLY.  The oracle restates the reference's Fortran algorithms
(voigt.f90, opacity.f90, solver.f90, synth.f90 drivers, convol.f90, utils.f90 quadrature)
operation by operation.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
reference arm may import this module, and only to check or to time a CPU baseline -- the
product (fastspec_b200) never calls it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libfsoracle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_long)


class _State(C.Structure):
    _fields_ = [
        ("wmode", C.c_int), ("wstart", C.c_double), ("wend", C.c_double), ("dstep", C.c_double),
        ("nwl", C.c_int), ("wave", _dp), ("wfirst", C.c_double), ("wlast", C.c_double),
        ("rstep", C.c_double),
        ("ntau", C.c_int), ("rhox", _dp), ("T", _dp), ("xne", _dp), ("xna", _dp), ("rho", _dp),
        ("height", _dp),
        ("nspc", C.c_int), ("fractionpf", _fp), ("xamass", _fp), ("potion", _fp), ("ion", _ip),
        ("frac_h1", _fp), ("frac_he1", _fp), ("frac_h2", _fp), ("spc_he1", C.c_int),
        ("contopac", _dp), ("contopac_std", _dp), ("motype", C.c_int),
        ("nhe", C.c_int), ("hegam", _dp), ("heshf", _dp),
        ("vmicro", C.c_double), ("epsopac", C.c_double), ("vwfudge", C.c_double),
        ("h2brd", C.c_double), ("vwmol", C.c_double), ("molbrd", C.c_int),
        ("x_nprtb", _dp), ("x_gvwprt", _dp), ("x_temp6", _dp), ("x_temp3", _dp), ("x_kbt", _dp),
        ("x_kbet", _dp), ("x_vturb2", C.c_double),
        ("radius", C.c_double), ("sph_nmu", C.c_int), ("sph_ntau", _ip), ("sph_graz", _ip),
        ("sph_map", _ip), ("sph_rhox", _dp), ("sph_muloc", _dp),
    ]


class _Lines(C.Structure):
    _fields_ = [
        ("n", C.c_long), ("wl", _dp), ("elo", _fp), ("gf", _fp), ("grad", _fp), ("gqst", _fp),
        ("gvdw", _fp), ("spc", _ip), ("kind", _ip), ("ismol", _ip), ("ihe", _ip),
        ("npi", _ip), ("nsi", _ip), ("pi_off", _lp), ("si_off", _lp),
        ("spl_pi", _fp), ("str_pi", _fp), ("spl_si", _fp), ("str_si", _fp),
    ]


class XCoef(C.Structure):
    """or_xcoef: XlineCoef (opacity.f90:43-58)."""
    _fields_ = [(n, C.c_double) for n in ("WaveL", "Hnux", "Elo", "Gf", "Grad", "Xmass", "Cqst", "Qdiv", "Cvdw",
                                          "AboPre", "AboVbc", "AboExp")] + \
               [(n, C.c_int) for n in ("IxPF", "MdQst", "MdVdw", "IxHe")]


class _Stats(C.Structure):
    _fields_ = [("nlines_in", C.c_long), ("nlines_used", C.c_long), ("nwide", C.c_long),
                ("nweak", C.c_long), ("nsegments", C.c_long), ("nrefills", C.c_long),
                ("line_evals", C.c_double), ("wide_evals", C.c_double)]


def build():
    """Compile oracle/libfsoracle.so with its Makefile (gcc, OpenMP, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.or_hvoigt_exact.restype = C.c_double
        L.or_hvoigt_exact.argtypes = [C.c_double, C.c_double]
        L.or_wvoigt_exact.argtypes = [C.c_double, C.c_double, _dp, _dp]
        L.or_hvoigt.restype = C.c_double
        L.or_hvoigt.argtypes = [C.c_double, C.c_double]
        L.or_fvoigt.argtypes = [C.c_double, C.c_double, _dp, _dp]
        L.or_voigt_table.restype = _fp
        L.or_fvoigt_table.restype = _fp
        L.or_grid_init.argtypes = [C.POINTER(_State)]
        L.or_xline_init.argtypes = [C.POINTER(_State)]
        L.or_state_free.argtypes = [C.POINTER(_State)]
        L.or_waveidx.argtypes = [C.POINTER(_State), C.c_double]
        L.or_air2vac.restype = C.c_double
        L.or_air2vac.argtypes = [C.c_double]
        L.or_xline.argtypes = [C.POINTER(_State), C.POINTER(_Lines), C.c_long, _dp, _dp, _dp]
        L.or_lineop_calc.argtypes = [C.POINTER(_State), C.POINTER(_Lines), C.c_int, C.c_long, _dp,
                                     _ip, _ip, _ip, _fp, C.c_int, _dp, _dp, C.POINTER(_Stats)]
        L.or_lineop_calc_range.argtypes = [C.POINTER(_State), C.POINTER(_Lines), C.c_int, C.c_long, _dp,
                                           _ip, _ip, _ip, _fp, C.c_int, _dp, _dp, C.POINTER(_Stats),
                                           C.c_int, C.c_int]
        L.or_mag_lineop_calc.argtypes = [C.POINTER(_State), C.POINTER(_Lines), C.c_int, _dp,
                                         C.c_long, _dp, _ip, _ip, _ip, _fp, C.c_int, _dp, _dp,
                                         C.POINTER(_Stats)]
        L.or_locprf_pp.argtypes = [_dp, _dp, C.c_int, _dp, _dp, _dp, C.c_int]
        L.or_xline_setup.argtypes = [C.POINTER(_State), C.POINTER(_Lines), C.c_long, C.c_int, C.POINTER(XCoef)]
        L.or_xline_depth.argtypes = [C.POINTER(_State), C.c_int, C.POINTER(XCoef), _dp, _dp, _dp]
        L.or_lineopacity1.argtypes = [C.POINTER(_State), _dp, _ip, _ip, _ip, _dp, _dp, _dp, C.c_double, C.c_int,
                                      C.c_int, C.c_int, C.c_long, _dp]
        L.or_lineopacity2.argtypes = [C.POINTER(_State), C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                      _dp, _dp, _dp, _dp]
        L.or_mag_lineopacity1.argtypes = [C.POINTER(_State), _dp, _ip, _ip, _ip, _dp, _dp, _dp, _ip, _ip, _lp, _lp,
                                          _fp, _fp, _fp, _fp, C.c_double, C.c_int, C.c_int, C.c_int, C.c_long, _dp]
        L.or_analytic_window.restype = C.c_double
        L.or_analytic_window.argtypes = [C.POINTER(_State), C.c_int, _dp, _dp, _dp, _dp]
        L.or_stokes_prf_pp.argtypes = [C.POINTER(_State), _dp, _dp, _dp, _dp, C.c_int, _dp, _dp, _dp, _dp, _dp,
                                       _dp, _dp]
        L.or_solve4x4.argtypes = [_dp, _dp, _dp]
        L.or_radtran.argtypes = [C.POINTER(_State), C.c_int, _dp, _dp, _dp, _dp]
        L.or_mag_radtran.argtypes = [C.POINTER(_State), C.c_int, _dp, C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.or_mu_quadrature.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, C.c_int]
        L.or_gauss_mu.argtypes = [C.c_int, C.c_int, _dp, _dp]
        L.or_disk_integ.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.or_zeeman_pattern.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float, _ip, _fp, _fp,
                                        _ip, _fp, _fp]
        L.or_hestark_init.argtypes = [C.c_int, _dp, _dp, _fp, _fp, _dp, _dp]
        L.or_he_match_idx.argtypes = [C.c_double, C.c_double]
        _lib = L
    return _lib


def _p(a, ct):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ct))


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


# ---- Voigt ------------------------------------------------------------------------------

def hvoigt_exact(a, v):
    return lib().or_hvoigt_exact(float(a), float(v))


def wvoigt_exact(a, v):
    re, im = C.c_double(), C.c_double()
    lib().or_wvoigt_exact(float(a), float(v), C.byref(re), C.byref(im))
    return re.value + 1j * im.value


def hvoigt(a, v):
    return lib().or_hvoigt(float(a), float(v))


def fvoigt(a, v):
    h, l = C.c_double(), C.c_double()
    lib().or_fvoigt(float(a), float(v), C.byref(h), C.byref(l))
    return h.value, l.value


def voigt_table():
    """VgtTab as float32 [402][1002] (row = a node, column = v node)."""
    p = lib().or_voigt_table()
    return np.ctypeslib.as_array(p, shape=(402 * 1002,)).reshape(402, 1002).copy()


def fvoigt_table():
    """FvTab as float32 [402][1002][2] (H, L)."""
    p = lib().or_fvoigt_table()
    return np.ctypeslib.as_array(p, shape=(402 * 1002 * 2,)).reshape(402, 1002, 2).copy()


# ---- state --------------------------------------------------------------------------------

class State:
    """One atmosphere + grid + configuration, as consumed by the hot path.

    atm: dict with rhox, T, xne, xna, rho (FP64 [ntau]); species: fractionpf (FP32 [ntau][nspc]),
    xamass, potion (FP32 [nspc]), ion (int [nspc]); frac_h1/frac_he1/frac_h2 (FP32 [ntau]);
    contopac (FP64 [nwl][ntau]); grid: wmode, wstart, wend, dstep.
    """

    def __init__(self, grid, atm, contopac=None, contopac_std=None, motype=0, vmicro=0.0,
                 epsopac=1e-4, vwfudge=1.0, h2brd=0.0, vwmol=0.0, molbrd=0, hegam=None,
                 heshf=None, spc_he1=-1):
        L = lib()
        s = _State()
        s.wmode = int(grid["wmode"]); s.wstart = float(grid["wstart"])
        s.wend = float(grid["wend"]); s.dstep = float(grid["dstep"])
        nwl = L.or_grid_init(C.byref(s))
        if nwl < 2:
            raise ValueError("grid has fewer than two points")
        self._keep = {}
        k = self._keep
        for name in ("rhox", "T", "xne", "xna", "rho"):
            k[name] = _f64(atm[name])
            setattr(s, name, _p(k[name], C.c_double))
        s.ntau = len(k["T"])
        k["fractionpf"] = _f32(atm["fractionpf"])
        s.nspc = k["fractionpf"].shape[1]
        s.fractionpf = _p(k["fractionpf"], C.c_float)
        for name in ("xamass", "potion", "frac_h1", "frac_he1", "frac_h2"):
            k[name] = _f32(atm[name])
            setattr(s, name, _p(k[name], C.c_float))
        k["ion"] = _i32(atm["ion"]); s.ion = _p(k["ion"], C.c_int)
        s.spc_he1 = int(spc_he1)
        if contopac is not None:
            k["contopac"] = _f64(contopac)
            if k["contopac"].shape != (nwl, s.ntau):
                raise ValueError("contopac shape %s != (%d, %d)" % (k["contopac"].shape, nwl, s.ntau))
            s.contopac = _p(k["contopac"], C.c_double)
        if contopac_std is not None:
            k["contopac_std"] = _f64(contopac_std); s.contopac_std = _p(k["contopac_std"], C.c_double)
        s.motype = int(motype)
        if hegam is not None:
            k["hegam"] = _f64(hegam); k["heshf"] = _f64(heshf)
            s.nhe = k["hegam"].shape[0]
            s.hegam = _p(k["hegam"], C.c_double); s.heshf = _p(k["heshf"], C.c_double)
        s.vmicro = vmicro; s.epsopac = epsopac; s.vwfudge = vwfudge; s.h2brd = h2brd
        s.vwmol = vwmol; s.molbrd = int(molbrd)
        L.or_xline_init(C.byref(s))
        self.s = s
        self.nwl = nwl
        self.ntau = s.ntau

    @property
    def wave(self):
        return np.ctypeslib.as_array(self.s.wave, shape=(self.nwl,)).copy()

    @property
    def wfirst(self):
        return self.s.wfirst

    def waveidx(self, w):
        return lib().or_waveidx(C.byref(self.s), float(w))

    def xline_init_arrays(self):
        n = self.ntau
        g = lambda p: np.ctypeslib.as_array(p, shape=(n,)).copy()
        return dict(nprtb=g(self.s.x_nprtb), gvwprt=g(self.s.x_gvwprt), temp6=g(self.s.x_temp6),
                    temp3=g(self.s.x_temp3), kbt=g(self.s.x_kbt), kbet=g(self.s.x_kbet),
                    vturb2=self.s.x_vturb2)

    def set_sphere(self, radius, height, xmu):
        """Spherical geometry (ReadModel's RADIUS and layer heights, ioutils.f90:1630-1700) with the
        rays of SphereInit for the angles xmu; radius <= 0 returns to plane-parallel."""
        k = self._keep
        if radius <= 0:
            self.s.radius = -1.0; self.s.sph_nmu = 0
            return None
        g = sphere_init(self._keep["rhox"], height, radius, xmu)
        for name in ("ntau_mu", "graz", "map"):
            k["sph_" + name] = g[name]
        k["sph_rhox"] = g["rhox_mu"]; k["sph_muloc"] = g["mu_loc"]; k["height"] = _f64(height)
        self.s.sph_ntau = _p(k["sph_ntau_mu"], C.c_int); self.s.sph_graz = _p(k["sph_graz"], C.c_int)
        self.s.sph_map = _p(k["sph_map"], C.c_int); self.s.sph_rhox = _p(k["sph_rhox"], C.c_double)
        self.s.sph_muloc = _p(k["sph_muloc"], C.c_double); self.s.height = _p(k["height"], C.c_double)
        self.s.sph_nmu = len(xmu); self.s.radius = float(radius)
        return g

    def __del__(self):
        try:
            lib().or_state_free(C.byref(self.s))
        except Exception:
            pass


class Lines:
    """SoA line list.  kind: 0 atomic, 1 molecular, 2 magnetic/ASCII record."""

    def __init__(self, wl, elo, gf, grad, gqst, gvdw, spc, kind=2, ismol=None, ihe=None,
                 zeeman=None):
        n = len(wl)
        k = self._keep = {}
        L = _Lines()
        L.n = n
        k["wl"] = _f64(wl); L.wl = _p(k["wl"], C.c_double)
        for name, arr in (("elo", elo), ("gf", gf), ("grad", grad), ("gqst", gqst), ("gvdw", gvdw)):
            k[name] = _f32(arr); setattr(L, name, _p(k[name], C.c_float))
        k["spc"] = _i32(spc); L.spc = _p(k["spc"], C.c_int)
        k["kind"] = _i32(np.broadcast_to(np.asarray(kind, dtype=np.int32), (n,)))
        L.kind = _p(k["kind"], C.c_int)
        if ismol is not None:
            k["ismol"] = _i32(ismol); L.ismol = _p(k["ismol"], C.c_int)
        if ihe is not None:
            k["ihe"] = _i32(ihe); L.ihe = _p(k["ihe"], C.c_int)
        if zeeman is not None:
            npi, nsi, spl_pi, str_pi, spl_si, str_si = zeeman
            k["npi"] = _i32(npi); k["nsi"] = _i32(nsi)
            k["pi_off"] = np.ascontiguousarray(np.concatenate([[0], np.cumsum(k["npi"])[:-1]]), dtype=np.int64)
            k["si_off"] = np.ascontiguousarray(np.concatenate([[0], np.cumsum(k["nsi"])[:-1]]), dtype=np.int64)
            for name, arr in (("spl_pi", spl_pi), ("str_pi", str_pi), ("spl_si", spl_si), ("str_si", str_si)):
                k[name] = _f32(arr if len(arr) else np.zeros(1, np.float32))
                setattr(L, name, _p(k[name], C.c_float))
            L.npi = _p(k["npi"], C.c_int); L.nsi = _p(k["nsi"], C.c_int)
            L.pi_off = _p(k["pi_off"], C.c_long); L.si_off = _p(k["si_off"], C.c_long)
        self.L = L
        self.n = n


# ---- the elemental routines on their own (checks of the library's kernel-level entry points) --------
def xline_setup(state, lines, i, list_type=2):
    """XlineSetup of line i (0-based): an XCoef structure."""
    xc = XCoef()
    lib().or_xline_setup(C.byref(state.s), C.byref(lines.L), int(i), int(list_type), C.byref(xc))
    return xc


def xline_depth(state, xc):
    """XlineDepth of one XCoef at every depth: (lincop, linvvgt, linavgt) [ntau]."""
    n = state.ntau
    out = [np.zeros(n) for _ in range(3)]
    for t in range(n):
        c, v, a = C.c_double(), C.c_double(), C.c_double()
        lib().or_xline_depth(C.byref(state.s), t, C.byref(xc), C.byref(c), C.byref(v), C.byref(a))
        out[0][t], out[1][t], out[2][t] = c.value, v.value, a.value
    return tuple(out)


def lineopacity1(state, blk, Wl, l1, l2, iwl, loff=0):
    """LineOpacity1 over the block dict (wlcent, flags, ileft, iright, lincop, linvvgt, linavgt): [ntau]."""
    out = np.zeros(state.ntau)
    b = {k: (_f64(v) if k in ("wlcent", "lincop", "linvvgt", "linavgt") else _i32(v)) for k, v in blk.items()
         if k in ("wlcent", "flags", "ileft", "iright", "lincop", "linvvgt", "linavgt")}
    lib().or_lineopacity1(C.byref(state.s), _p(b["wlcent"], C.c_double), _p(b["flags"], C.c_int),
                          _p(b["ileft"], C.c_int), _p(b["iright"], C.c_int), _p(b["lincop"], C.c_double),
                          _p(b["linvvgt"], C.c_double), _p(b["linavgt"], C.c_double), float(Wl), int(l1), int(l2),
                          int(iwl), int(loff), _p(out, C.c_double))
    return out


def lineopacity2(state, Wl, wlcent, flag, ileft, iright, iwl, lincop, linvvgt, linavgt):
    out = np.zeros(state.ntau)
    c, v, a = _f64(lincop), _f64(linvvgt), _f64(linavgt)
    lib().or_lineopacity2(C.byref(state.s), float(Wl), float(wlcent), int(flag), int(ileft), int(iright), int(iwl),
                          _p(c, C.c_double), _p(v, C.c_double), _p(a, C.c_double), _p(out, C.c_double))
    return out


def mag_lineopacity1(state, blk, zeeman, Wl, l1, l2, iwl, loff=0):
    """MagLineOpacity1 over the block dict and Zeeman components (npi, nsi, spl_pi, str_pi, spl_si,
    str_si; shifts in A): [ntau][6]."""
    out = np.zeros((state.ntau, 6))
    b = {k: (_f64(v) if k in ("wlcent", "lincop", "linvvgt", "linavgt") else _i32(v)) for k, v in blk.items()
         if k in ("wlcent", "flags", "ileft", "iright", "lincop", "linvvgt", "linavgt")}
    npi, nsi = _i32(zeeman[0]), _i32(zeeman[1])
    poff = np.ascontiguousarray(np.concatenate([[0], np.cumsum(npi)[:-1]]), np.int64)
    soff = np.ascontiguousarray(np.concatenate([[0], np.cumsum(nsi)[:-1]]), np.int64)
    z = [_f32(x) if len(x) else np.zeros(1, np.float32) for x in zeeman[2:]]
    lib().or_mag_lineopacity1(C.byref(state.s), _p(b["wlcent"], C.c_double), _p(b["flags"], C.c_int),
                              _p(b["ileft"], C.c_int), _p(b["iright"], C.c_int), _p(b["lincop"], C.c_double),
                              _p(b["linvvgt"], C.c_double), _p(b["linavgt"], C.c_double), _p(npi, C.c_int),
                              _p(nsi, C.c_int), _p(poff, C.c_long), _p(soff, C.c_long), _p(z[0], C.c_float),
                              _p(z[1], C.c_float), _p(z[2], C.c_float), _p(z[3], C.c_float), float(Wl), int(l1),
                              int(l2), int(iwl), int(loff), _p(out, C.c_double))
    return out


def analytic_window(state, flag, lincop, linvvgt, linavgt, contopac):
    c, v, a, co = _f64(lincop), _f64(linvvgt), _f64(linavgt), _f64(contopac)
    return lib().or_analytic_window(C.byref(state.s), int(flag), _p(c, C.c_double), _p(v, C.c_double),
                                    _p(a, C.c_double), _p(co, C.c_double))


def stokes_prf_pp(state, m6, lop, cop, src, xmu, sphi2, cphi2, cphi, s2psi, c2psi):
    """StokesPrfPP: m6 [ntau][6], lop/cop/src [ntau], field per angle: [4][nmu]."""
    xmu = _f64(xmu)
    out = np.zeros((4, len(xmu)))
    arr = [_f64(x) for x in (m6, lop, cop, src)]
    g = [_f64(x) for x in (sphi2, cphi2, cphi, s2psi, c2psi)]
    lib().or_stokes_prf_pp(C.byref(state.s), *[_p(x, C.c_double) for x in arr], len(xmu), _p(xmu, C.c_double),
                           *[_p(x, C.c_double) for x in g], _p(out, C.c_double))
    return out


def reader_select(arrays, wstart, wend):
    """The lines a synthesis over [wstart, wend] reads from a list sorted by wavelength: those with
    wstart <= wl <= wend, as ReadHDF locates them (LowerBoundReal8 / UpperBoundReal8 on the sorted
    wavelength column, ioutils.f90:752-753) and ReadAscMag packs them (ioutils.f90:1496-1497).
    arrays: dict of per-line numpy arrays with "wl"; returns the same dict restricted."""
    wl = arrays["wl"]
    i1 = int(np.searchsorted(wl, wstart, side="left"))
    i2 = int(np.searchsorted(wl, wend, side="right"))
    return {k: np.ascontiguousarray(v[i1:i2]) for k, v in arrays.items()}


def xline(state, lines, i):
    n = state.ntau
    cop, vv, av = (np.zeros(n) for _ in range(3))
    lib().or_xline(C.byref(state.s), C.byref(lines.L), int(i), _p(cop, C.c_double),
                   _p(vv, C.c_double), _p(av, C.c_double))
    return cop, vv, av


def lineop_calc(state, lines, list_type=2, nlines_lim=0, lineopac=None, nmu=0, xmu=None, wmu=None,
                want_linstr=False, wrange=None):
    """LineopCalc.  Returns dict(lineopac [nwl][ntau], flags, ileft, iright, stats, linstr).
    wrange = (i0, i1), 1-based inclusive: windows on the whole grid, accumulation only over those
    wavelengths (the rows of a whole-grid run; other rows stay zero)."""
    n = lines.n
    lo = np.zeros((state.nwl, state.ntau)) if lineopac is None else lineopac
    flags = np.zeros(max(n, 1), np.int32); il = np.zeros(max(n, 1), np.int32)
    ir = np.zeros(max(n, 1), np.int32)
    ls = np.zeros(max(n, 1), np.float32) if want_linstr else None
    st = _Stats()
    xmu = _f64(xmu); wmu = _f64(wmu)
    i0, i1 = (1, state.nwl) if wrange is None else (int(wrange[0]), int(wrange[1]))
    rc = lib().or_lineop_calc_range(C.byref(state.s), C.byref(lines.L), int(list_type), int(nlines_lim),
                                    _p(lo, C.c_double), _p(flags, C.c_int), _p(il, C.c_int), _p(ir, C.c_int),
                                    _p(ls, C.c_float), int(nmu), _p(xmu, C.c_double), _p(wmu, C.c_double),
                                    C.byref(st), i0, i1)
    if rc != 0:
        raise RuntimeError("or_lineop_calc failed: %d" % rc)
    return dict(lineopac=lo, flags=flags[:n], ileft=il[:n], iright=ir[:n], linstr=None if ls is None else ls[:n],
                stats={f: getattr(st, f) for f, _ in _Stats._fields_})


def mag_lineop_calc(state, lines, bframe, bfield, nlines_lim=0, nmu=0, xmu=None, wmu=None,
                    want_linstr=False):
    n = lines.n
    mlo = np.zeros((state.nwl, state.ntau, 6))
    flags = np.zeros(max(n, 1), np.int32); il = np.zeros(max(n, 1), np.int32)
    ir = np.zeros(max(n, 1), np.int32)
    ls = np.zeros(max(n, 1), np.float32) if want_linstr else None
    st = _Stats()
    bf = _f64(bfield); xmu = _f64(xmu); wmu = _f64(wmu)
    rc = lib().or_mag_lineop_calc(C.byref(state.s), C.byref(lines.L), int(bframe), _p(bf, C.c_double),
                                  int(nlines_lim), _p(mlo, C.c_double), _p(flags, C.c_int),
                                  _p(il, C.c_int), _p(ir, C.c_int), _p(ls, C.c_float), int(nmu),
                                  _p(xmu, C.c_double), _p(wmu, C.c_double), C.byref(st))
    if rc != 0:
        raise RuntimeError("or_mag_lineop_calc failed: %d" % rc)
    return dict(maglineopac=mlo, flags=flags[:n], ileft=il[:n], iright=ir[:n],
                linstr=None if ls is None else ls[:n],
                stats={f: getattr(st, f) for f, _ in _Stats._fields_})


def _check_rays(state, nmu):
    if state.s.radius > 0 and state.s.sph_nmu != nmu:
        raise ValueError("spherical state: the rays were set for %d angles, not %d" % (state.s.sph_nmu, nmu))


def radtran(state, xmu, lineopac, want_spc=True):
    xmu = _f64(xmu); nmu = len(xmu)
    _check_rays(state, nmu)
    lo = _f64(lineopac)
    spl = np.zeros((state.nwl, nmu)); spc = np.zeros((state.nwl, nmu)) if want_spc else None
    lib().or_radtran(C.byref(state.s), nmu, _p(xmu, C.c_double), _p(lo, C.c_double),
                     _p(spl, C.c_double), _p(spc, C.c_double))
    return spl, spc


def mag_radtran(state, xmu, bframe, bfield, lineopac, maglineopac):
    xmu = _f64(xmu); nmu = len(xmu)
    _check_rays(state, nmu)
    bf = _f64(bfield); lo = _f64(lineopac); mlo = _f64(maglineopac)
    spz = np.zeros((state.nwl, 4, nmu)); spc = np.zeros((state.nwl, nmu))
    lib().or_mag_radtran(C.byref(state.s), nmu, _p(xmu, C.c_double), int(bframe), _p(bf, C.c_double),
                         _p(lo, C.c_double), _p(mlo, C.c_double), _p(spz, C.c_double), _p(spc, C.c_double))
    return spz, spc


def sphere_init(rhox, height, radius, xmu):
    """SphereInit (solver.f90:45-120): ray geometry per angle; map is 1-based as MapMu."""
    rhox = _f64(rhox); height = _f64(height); xmu = _f64(xmu)
    nt, nmu = len(rhox), len(xmu)
    out = dict(ntau_mu=np.zeros(nmu, np.int32), graz=np.zeros(nmu, np.int32),
               map=np.zeros((nmu, 2 * nt), np.int32), rhox_mu=np.zeros((nmu, 2 * nt)),
               mu_loc=np.zeros((nmu, 2 * nt)))
    rc = lib().or_sphere_init(nt, _p(rhox, C.c_double), _p(height, C.c_double), C.c_double(radius), nmu,
                              _p(xmu, C.c_double), _p(out["ntau_mu"], C.c_int), _p(out["graz"], C.c_int),
                              _p(out["map"], C.c_int), _p(out["rhox_mu"], C.c_double),
                              _p(out["mu_loc"], C.c_double))
    if rc == -1:
        raise ValueError("SphereInit: mu = 0 rays are unsupported for spherical models")
    if rc == -2:
        raise ValueError("SphereInit: grazing ray tangent in the top model layer")
    return out


def air2vac(lam):
    """Air2Vac (utils.f90:1020-1032) of one wavelength [A]."""
    return float(lib().or_air2vac(float(lam)))


HE_NTAB = 37


def hestark_init(T, xne, frac_hii, frac_heii):
    """HeStarkInit (hestark.f90:332-370): (HeGam [rad/s], HeShf [A]) of the 37 tabulated He I lines,
    each [37][ntau], from T, Xne and the FP32 H II and He II densities (Fraction)."""
    T = _f64(T); xne = _f64(xne); hii = _f32(frac_hii); heii = _f32(frac_heii)
    nt = len(T)
    g = np.zeros((HE_NTAB, nt)); h = np.zeros((HE_NTAB, nt))
    lib().or_hestark_init(nt, _p(T, C.c_double), _p(xne, C.c_double), _p(hii, C.c_float), _p(heii, C.c_float),
                          _p(g, C.c_double), _p(h, C.c_double))
    return g, h


def he_match_idx(wave_air, elo):
    """HeMatchIdx (hestark.f90:376-389): table entry 1..37, or 0."""
    return int(lib().or_he_match_idx(float(wave_air), float(elo)))


def locprf_pp(xmu, xki, src, rhox):
    xmu = _f64(xmu); xki = _f64(xki); src = _f64(src); rhox = _f64(rhox)
    out = np.zeros(len(xmu))
    lib().or_locprf_pp(_p(out, C.c_double), _p(xmu, C.c_double), len(xmu), _p(xki, C.c_double),
                       _p(src, C.c_double), _p(rhox, C.c_double), len(xki))
    return out


def mu_quadrature(quad, n, x=None):
    setnodes = x is None
    x = np.zeros(n) if x is None else _f64(x).copy()
    w = np.zeros(n); r = np.zeros(n + 1)
    rc = lib().or_mu_quadrature(int(quad), int(n), _p(x, C.c_double), _p(w, C.c_double),
                                _p(r, C.c_double), int(setnodes))
    if rc != 0:
        raise ValueError("unknown quadrature %d" % quad)
    return x, w, r


def disk_integ(wmu, spl, spc):
    wmu = _f64(wmu); spl = _f64(spl); spc = _f64(spc)
    nwl, nmu = spl.shape
    sfl = np.zeros(nwl); sfc = np.zeros(nwl)
    lib().or_disk_integ(nmu, nwl, _p(wmu, C.c_double), _p(spl, C.c_double), _p(spc, C.c_double),
                        _p(sfl, C.c_double), _p(sfc, C.c_double))
    return sfl, sfc


def grid_dv(grid, wave_abs):
    """Velocity step of the grid as DiskInteg takes it (convol.f90:86-91)."""
    if grid["wmode"] == 0:
        return 2.0 * grid["dstep"] / (wave_abs[0] + wave_abs[-1]) * 299792.458
    return grid["dstep"]


def gauss_sigma_pix(grid, wave_abs, vgau):
    """ConvolGau's Fwhm / step in pixels (convol.f90:259-264); vgau > 1000 is a resolving power."""
    if vgau > 1000:
        vgau = 299792.458 / vgau
    if grid["wmode"] == 0:
        return vgau * (wave_abs[0] + wave_abs[-1]) / 299792.458 / 2.0 / grid["dstep"]
    return vgau / grid["dstep"]


def disk_integ_conv(xmu, wmu, radii, spl, spc, dv, vsini, vmacro, gsig):
    """DiskInteg with rotation, radial-tangential macroturbulence and Gaussian broadening."""
    xmu = _f64(xmu); wmu = _f64(wmu); radii = _f64(radii); spl = _f64(spl); spc = _f64(spc)
    nwl, nmu = spl.shape
    sfl = np.zeros(nwl); sfc = np.zeros(nwl)
    lib().or_disk_integ_conv(nmu, nwl, _p(xmu, C.c_double), _p(wmu, C.c_double), _p(radii, C.c_double),
                             C.c_double(dv), C.c_double(vsini), C.c_double(vmacro), C.c_double(gsig),
                             _p(spl, C.c_double), _p(spc, C.c_double), _p(sfl, C.c_double), _p(sfc, C.c_double))
    return sfl, sfc


def zeeman_pattern(jlo, jup, glo, gup):
    m = int(round(2 * jup)) + 1
    npi, nsi = C.c_int(), C.c_int()
    spi, rpi, ssi, rsi = (np.zeros(max(m, 1), np.float32) for _ in range(4))
    lib().or_zeeman_pattern(jlo, jup, glo, gup, C.byref(npi), _p(spi, C.c_float), _p(rpi, C.c_float),
                            C.byref(nsi), _p(ssi, C.c_float), _p(rsi, C.c_float))
    return spi[:npi.value], rpi[:npi.value], ssi[:nsi.value], rsi[:nsi.value]
