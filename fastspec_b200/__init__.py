"""fastspec_b200 -- B200-native line-opacity -> formal-solver path of FastSpec.

The product is the sm_100a CUDA library libfastspec_b200.so behind the C-ABI in
include/fastspec_gpu.h.  This module binds that ABI with ctypes and mirrors the reference's
driver sequence (Init grid -> EOS state -> ContopCalc -> LineopCalc per list -> RadTranCalc ->
DiskInteg, fastspec.f90:192-461).  There is no CPU fallback: every call fails loudly when the
library is missing or no CUDA device is present.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfastspec_b200.so")

PREC_MIXED = 0
PREC_FP64 = 1
FAULT_NONE, FAULT_ALLOC_LIMIT, FAULT_COPY_TIMEOUT = 0, 1, 2
F_WEAK, F_MOL, F_ABO, F_WIDE = 1, 2, 4, 8

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


class FsgError(RuntimeError):
    pass


class Config(C.Structure):
    _fields_ = [("device", C.c_int), ("precision", C.c_int), ("vmicro", C.c_double),
                ("epsopac", C.c_double), ("vwfudge", C.c_double), ("h2brd", C.c_double),
                ("vwmol", C.c_double), ("molbrd", C.c_int), ("limitram_gb", C.c_double)]


class CLines(C.Structure):
    _fields_ = [("n", C.c_int64), ("wl", _dp), ("elo", _fp), ("gf", _fp), ("grad", _fp),
                ("gqst", _fp), ("gvdw", _fp), ("spc", _ip), ("kind", C.c_int32), ("ismol", _ip),
                ("ihe", _ip), ("npi", _ip), ("nsi", _ip), ("pi_off", _lp), ("si_off", _lp),
                ("spl_pi", _fp), ("str_pi", _fp), ("spl_si", _fp), ("str_si", _fp)]


class Stats(C.Structure):
    _fields_ = [("nlines_in", C.c_int64), ("nlines_used", C.c_int64), ("nwide", C.c_int64),
                ("nweak", C.c_int64), ("nblocks", C.c_int64), ("line_evals", C.c_double),
                ("ms_center", C.c_double), ("ms_params", C.c_double), ("ms_accum", C.c_double),
                ("ms_total", C.c_double), ("accum_launches", C.c_int64), ("ms_accum_kernels", C.c_double),
                ("ms_wing_kernels", C.c_double), ("ms_core_kernels", C.c_double), ("core_evals", C.c_double)]

    def asdict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class BatchTuning(C.Structure):
    _fields_ = [("tile_pix", C.c_int32), ("wing_ctas", C.c_int32), ("core_ctas", C.c_int32),
                ("ms_wing", C.c_double), ("ms_core", C.c_double)]

    def asdict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class BatchStats(C.Structure):
    _fields_ = [("natm", C.c_int32), ("nlines_candidate", C.c_int64), ("line_evals", C.c_double),
                ("ms_total", C.c_double), ("tuning", BatchTuning), ("ms_prepare", C.c_double),
                ("ms_wing", C.c_double), ("ms_core", C.c_double), ("ms_solve", C.c_double),
                ("core_evals", C.c_double)]

    def asdict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if f != "tuning"}
        d["tuning"] = self.tuning.asdict()
        return d


# every symbol the header declares (checked by the CPU test suite)
EXPORTS = [
    "fsg_create", "fsg_destroy", "fsg_last_error", "fsg_version", "fsg_kernel_launches", "fsg_cuda_stream", "fsg_make_grid", "fsg_set_grid",
    "fsg_set_atmosphere", "fsg_set_contopac", "fsg_set_contopac_dev", "fsg_set_hestark", "fsg_hestark_tables",
    "fsg_he_match_idx",
    "fsg_lineop_calc", "fsg_lineop_calc_dev", "fsg_lineop_reset", "fsg_lineop_get", "fsg_lineop_set",
    "fsg_lineop_device_ptr", "fsg_set_mu", "fsg_radtran", "fsg_radtran_dev", "fsg_radtran_range_dev",
    "fsg_mag_lineop_calc",
    "fsg_mag_lineop_reset", "fsg_mag_radtran", "fsg_hvoigt", "fsg_fvoigt", "fsg_voigt_tables",
    "fsg_locprf_pp", "fsg_locprf_pp_noalloc", "fsg_mu_quadrature", "fsg_zeeman_pattern",
    "fsg_central_dev", "fsg_accumulate_dev", "fsg_batch_create", "fsg_batch_tune", "fsg_batch_set_tuning",
    "fsg_batch_run", "fsg_batch_flux", "fsg_batch_stream", "fsg_batch_last_error", "fsg_batch_destroy",
    "fsg_set_vmicro", "fsg_set_fractionpf", "fsg_adjoint_dev", "fsg_disk_integ_conv", "fsg_disk_integ_conv_dev",
    "fsg_xline_setup", "fsg_xline_depth", "fsg_lineopacity1", "fsg_lineopacity2", "fsg_mag_lineopacity1",
    "fsg_analytic_window", "fsg_stokes_prf_pp", "fsg_adjoint_range_dev", "fsg_set_fault",
]

_lib = None


def build_library(force=False):
    """Compile libfastspec_b200.so for sm_100a (nvcc; see fastspec_b200/build.py)."""
    import importlib
    return importlib.import_module(__name__ + ".build").build(force=force)


def lib():
    """Load libfastspec_b200.so (raises FsgError when it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FsgError("libfastspec_b200.so not built: run python -m fastspec_b200.build")
    L = C.CDLL(LIB_PATH)
    L.fsg_create.argtypes = [C.POINTER(Config), C.POINTER(C.c_void_p)]
    L.fsg_destroy.argtypes = [C.c_void_p]
    L.fsg_destroy.restype = None
    L.fsg_last_error.argtypes = [C.c_void_p]
    L.fsg_last_error.restype = C.c_char_p
    L.fsg_kernel_launches.argtypes = [C.c_void_p]
    L.fsg_kernel_launches.restype = C.c_int64
    L.fsg_cuda_stream.argtypes = [C.c_void_p]
    L.fsg_cuda_stream.restype = C.c_void_p
    L.fsg_make_grid.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, _dp, C.POINTER(C.c_int)]
    L.fsg_set_grid.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, _dp]
    L.fsg_set_atmosphere.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_int, _fp, _fp, _fp,
                                     _ip, _fp, _fp, _fp]
    L.fsg_set_contopac.argtypes = [C.c_void_p, _dp, _dp, C.c_int]
    L.fsg_set_contopac_dev.argtypes = [C.c_void_p, C.c_void_p]
    L.fsg_set_hestark.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_int]
    L.fsg_hestark_tables.argtypes = [C.c_int, _dp, _dp, _fp, _fp, _dp, _dp]
    L.fsg_he_match_idx.argtypes = [C.c_long, _dp, _fp, _ip, C.c_int, C.c_double, _ip]
    L.fsg_lineop_calc.argtypes = [C.c_void_p, C.POINTER(CLines), _dp, _ip, _ip, _ip, _fp, C.POINTER(Stats)]
    L.fsg_lineop_calc_dev.argtypes = [C.c_void_p, C.POINTER(CLines), C.POINTER(Stats)]
    L.fsg_lineop_reset.argtypes = [C.c_void_p]
    L.fsg_lineop_get.argtypes = [C.c_void_p, _dp]
    L.fsg_lineop_set.argtypes = [C.c_void_p, _dp]
    L.fsg_lineop_device_ptr.argtypes = [C.c_void_p]
    L.fsg_lineop_device_ptr.restype = C.c_void_p
    L.fsg_set_mu.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
    L.fsg_set_geometry.argtypes = [C.c_void_p, C.c_double, _dp]
    L.fsg_radtran.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
    L.fsg_radtran_dev.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.fsg_radtran_range_dev.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]
    L.fsg_mag_lineop_calc.argtypes = [C.c_void_p, C.POINTER(CLines), C.c_int, _dp, C.c_int, _dp, _ip, _ip,
                                      _ip, _fp, C.POINTER(Stats)]
    L.fsg_mag_lineop_reset.argtypes = [C.c_void_p]
    L.fsg_mag_radtran.argtypes = [C.c_void_p, C.c_int, _dp, C.c_int, _dp, _dp, _dp, _dp]
    L.fsg_hvoigt.argtypes = [C.c_void_p, C.c_int64, _dp, _dp, _dp]
    L.fsg_fvoigt.argtypes = [C.c_void_p, C.c_int64, _dp, _dp, _dp, _dp]
    L.fsg_voigt_tables.argtypes = [C.c_void_p, _fp, _fp]
    L.fsg_locprf_pp.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int, _dp, _dp, _dp, _dp]
    L.fsg_locprf_pp_noalloc.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p]
    L.fsg_mu_quadrature.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, C.c_int]
    L.fsg_zeeman_pattern.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float, _ip, _fp, _fp, _ip, _fp, _fp]
    L.fsg_batch_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(CLines), C.c_double,
                                   C.POINTER(C.c_void_p)]
    L.fsg_batch_tune.argtypes = [C.c_void_p, C.POINTER(BatchTuning)]
    L.fsg_batch_set_tuning.argtypes = [C.c_void_p, C.POINTER(BatchTuning)]
    L.fsg_batch_run.argtypes = [C.c_void_p, C.POINTER(BatchStats)]
    L.fsg_batch_flux.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
    L.fsg_batch_stream.argtypes = [C.c_void_p]
    L.fsg_batch_stream.restype = C.c_void_p
    L.fsg_batch_last_error.argtypes = [C.c_void_p]
    L.fsg_batch_last_error.restype = C.c_char_p
    L.fsg_batch_destroy.argtypes = [C.c_void_p]
    L.fsg_batch_destroy.restype = None
    vp = C.c_void_p
    L.fsg_xline_setup.argtypes = [vp, C.POINTER(CLines), vp]
    L.fsg_xline_depth.argtypes = [vp, C.c_int64, vp, vp, vp, vp]
    L.fsg_lineopacity1.argtypes = [vp, C.POINTER(CLineBlock), C.c_int64, vp, vp, vp, vp, C.c_int64, vp]
    L.fsg_mag_lineopacity1.argtypes = [vp, C.POINTER(CLineBlock), C.c_int64, vp, vp, vp, vp, C.c_int64, vp]
    L.fsg_lineopacity2.argtypes = [vp, C.POINTER(CLineBlock), C.c_int64, vp, vp, vp, vp, vp, vp, vp]
    L.fsg_analytic_window.argtypes = [vp, C.c_int64, vp, vp, vp, vp, vp, vp]
    L.fsg_stokes_prf_pp.argtypes = [vp, C.c_int64, vp, vp, vp, vp, vp, vp, vp, vp]
    L.fsg_adjoint_range_dev.argtypes = [vp, C.POINTER(CLines), vp, vp, vp, C.c_int, C.c_int, vp, vp, vp, vp]
    L.fsg_set_fault.argtypes = [vp, C.c_int, C.c_double]
    _lib = L
    return L


def _p(a, ct):
    return None if a is None else a.ctypes.data_as(C.POINTER(ct))


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


# ---- host set-up routines ------------------------------------------------------------------

def make_grid(wmode, wstart, wend, dstep):
    """Wavelength grid of Init (synth.f90:56-74): offsets from wstart."""
    n = C.c_int()
    rc = lib().fsg_make_grid(int(wmode), float(wstart), float(wend), float(dstep), None, C.byref(n))
    if rc != 0:
        raise FsgError("fsg_make_grid: bad grid (%d)" % rc)
    w = np.zeros(n.value)
    lib().fsg_make_grid(int(wmode), float(wstart), float(wend), float(dstep), _p(w, C.c_double), C.byref(n))
    return w


def mu_quadrature(quad, n, x=None):
    setnodes = x is None
    x = np.zeros(n) if x is None else _f64(x).copy()
    w = np.zeros(n); r = np.zeros(n + 1)
    rc = lib().fsg_mu_quadrature(int(quad), int(n), _p(x, C.c_double), _p(w, C.c_double), _p(r, C.c_double),
                                 int(setnodes))
    if rc != 0:
        raise FsgError("fsg_mu_quadrature failed (%d)" % rc)
    return x, w, r


def mu_quad_type(xmu):
    """MuQuadType (utils.f90:1337-1354): the quadrature (1 Gauss-Legendre, 2 Gauss-Radau) whose nodes
    are the given angles to 1e-6, else 0 (also for fewer than two angles)."""
    xmu = _f64(xmu)
    n = len(xmu)
    if n < 2:
        return 0
    for q in (1, 2):
        xg, _, _ = mu_quadrature(q, n)
        if np.max(np.abs(xmu - xg)) < 1e-6:
            return q
    return 0


def convolve_spec_file(spec_path, vsini, vmacro, vgau, flux_path=None, device=0):
    """The reference's post-processing mode (`fastspec <fs_spec.bin> Vsini Vmacro Vgau`,
    fastspec.f90:75-134): read the intensities (ReadSpec's grid and angle order, fsio.spec_grid), take
    the quadrature from the angles (MuQuadType), disk-integrate with rotation, radial-tangential
    macroturbulence and Gaussian broadening on the device (fsg_disk_integ_conv_dev; Vgau above 1000 is
    a resolving power) and return (wave, sfl, sfc); with flux_path, also write fs_flux.bin there."""
    import torch
    from . import fsio
    if vsini < 0 or vmacro < 0 or vgau < 0:
        raise FsgError("convolve_spec_file: invalid convolution parameters")
    g = fsio.spec_grid(fsio.read_spec(spec_path))
    nmu = len(g["xmu"])
    x, w, r = mu_quadrature(mu_quad_type(g["xmu"]), nmu, x=g["xmu"])
    C = Context(device=device)
    try:
        C.set_grid(g["wmode"], g["wstart"], g["wend"], g["dstep"], wave=g["wave"])
        C.set_mu(x, w)
        dev = torch.device("cuda", device)
        spl = torch.from_numpy(g["spl"]).to(dev)
        spc = torch.from_numpy(g["spc"]).to(dev)
        sfl = torch.empty(len(g["wave"]), dtype=torch.float64, device=dev)
        sfc = torch.empty_like(sfl)
        torch.cuda.synchronize(dev)
        C.disk_integ_conv_dev(r, float(vsini), float(vmacro), float(vgau), spl.data_ptr(), spc.data_ptr(),
                              sfl.data_ptr(), sfc.data_ptr())
        sfl, sfc = sfl.cpu().numpy(), sfc.cpu().numpy()
    finally:
        C.close()
    wave = g["wave"] + g["wstart"]
    if flux_path is not None:
        fsio.write_flux(flux_path, wave, sfl, sfc)
    return wave, sfl, sfc


def zeeman_pattern(jlo, jup, glo, gup):
    m = int(round(2 * jup)) + 1
    npi, nsi = C.c_int32(), C.c_int32()
    spi, rpi, ssi, rsi = (np.zeros(max(m, 1), np.float32) for _ in range(4))
    rc = lib().fsg_zeeman_pattern(jlo, jup, glo, gup, C.byref(npi), _p(spi, C.c_float), _p(rpi, C.c_float),
                                  C.byref(nsi), _p(ssi, C.c_float), _p(rsi, C.c_float))
    if rc != 0:
        raise FsgError("fsg_zeeman_pattern failed (%d)" % rc)
    return spi[:npi.value], rpi[:npi.value], ssi[:nsi.value], rsi[:nsi.value]


HE_NTAB = 37


def hestark_tables(T, xne, frac_hii, frac_heii):
    """HeStarkInit (hestark.f90:332-370) through fsg_hestark_tables: (HeGam [rad/s], HeShf [A]) of the
    37 tabulated He I lines, each [37][ntau], from T, Xne and the FP32 H II and He II densities."""
    T = _f64(T); xne = _f64(xne); hii = _f32(frac_hii); heii = _f32(frac_heii)
    nt = len(T)
    if not (len(xne) == len(hii) == len(heii) == nt):
        raise FsgError("hestark_tables: T, xne, frac_hii and frac_heii differ in length")
    g = np.zeros((HE_NTAB, nt)); h = np.zeros((HE_NTAB, nt))
    rc = lib().fsg_hestark_tables(nt, _p(T, C.c_double), _p(xne, C.c_double), _p(hii, C.c_float),
                                  _p(heii, C.c_float), _p(g, C.c_double), _p(h, C.c_double))
    if rc != 0:
        raise FsgError("fsg_hestark_tables failed (%d): empty atmosphere or T <= 0" % rc)
    return g, h


def he_match_idx(wl, elo, spc, spc_he1, wfirst=0.0):
    """HeMatchIdx (hestark.f90:376-389) at XlineSetup (opacity.f90:176) through fsg_he_match_idx: the
    table entry 1..37 of each line of species spc_he1 (0: none), the ihe column of a LineList."""
    wl = _f64(wl); elo = _f32(elo); spc = _i32(spc)
    out = np.zeros(max(len(wl), 1), np.int32)
    rc = lib().fsg_he_match_idx(len(wl), _p(wl, C.c_double), _p(elo, C.c_float), _p(spc, C.c_int32),
                                int(spc_he1), float(wfirst), _p(out, C.c_int32))
    if rc != 0:
        raise FsgError("fsg_he_match_idx failed (%d)" % rc)
    return out[:len(wl)]


class LineList:
    """Host SoA line list in the reference's stored precision (wl FP64, the rest FP32).

    kind: 0 atomic HDF records, 1 single-species molecular, 2 ASCII / magnetic records.
    zeeman: (npi, nsi, spl_pi, str_pi, spl_si, str_si) with the sigma components mirrored as
    the .z reader stores them (blue half first)."""

    def __init__(self, wl, elo, gf, grad, gqst, gvdw, spc, kind=2, ismol=None, ihe=None, zeeman=None):
        k = self._keep = {}
        s = CLines()
        n = len(wl)
        s.n = n
        k["wl"] = _f64(wl); s.wl = _p(k["wl"], C.c_double)
        for name, arr in (("elo", elo), ("gf", gf), ("grad", grad), ("gqst", gqst), ("gvdw", gvdw)):
            k[name] = _f32(arr); setattr(s, name, _p(k[name], C.c_float))
        k["spc"] = _i32(spc); s.spc = _p(k["spc"], C.c_int32)
        s.kind = int(kind)
        if ismol is not None:
            k["ismol"] = _i32(ismol); s.ismol = _p(k["ismol"], C.c_int32)
        if ihe is not None:
            k["ihe"] = _i32(ihe); s.ihe = _p(k["ihe"], C.c_int32)
        if zeeman is not None:
            npi, nsi, spl_pi, str_pi, spl_si, str_si = zeeman
            k["npi"] = _i32(npi); k["nsi"] = _i32(nsi)
            k["pi_off"] = np.ascontiguousarray(np.concatenate([[0], np.cumsum(k["npi"])[:-1]]), np.int64)
            k["si_off"] = np.ascontiguousarray(np.concatenate([[0], np.cumsum(k["nsi"])[:-1]]), np.int64)
            for name, arr in (("spl_pi", spl_pi), ("str_pi", str_pi), ("spl_si", spl_si), ("str_si", str_si)):
                k[name] = _f32(arr if len(arr) else np.zeros(1, np.float32))
                setattr(s, name, _p(k[name], C.c_float))
            s.npi = _p(k["npi"], C.c_int32); s.nsi = _p(k["nsi"], C.c_int32)
            s.pi_off = _p(k["pi_off"], C.c_int64); s.si_off = _p(k["si_off"], C.c_int64)
        self.c = s
        self.n = n

    def _with_he_match(self, spc_he1, wfirst):
        """The list with its ihe column from he_match_idx when it has none (XlineSetup's table match)."""
        if self.c.ihe:
            return self
        k = self._keep
        ihe = he_match_idx(k["wl"], k["elo"], k["spc"], spc_he1, wfirst)
        out = LineList.__new__(LineList)
        out._keep = dict(k, ihe=ihe)
        out.c = CLines.from_buffer_copy(self.c)
        out.c.ihe = _p(ihe, C.c_int32)
        out.n = self.n
        return out

    @classmethod
    def from_arrays(cls, a, kind=2, zeeman=None):
        return cls(a["wl"], a["elo"], a["gf"], a["grad"], a["gqst"], a["gvdw"], a["spc"], kind=kind,
                   ismol=a.get("ismol"), ihe=a.get("ihe"), zeeman=zeeman)


# XlineCoef (opacity.f90:43-58) as fsg_xcoef lays it out
XCOEF_DTYPE = np.dtype([(n, np.float64) for n in ("WaveL", "Hnux", "Elo", "Gf", "Grad", "Xmass", "Cqst", "Qdiv",
                                                  "Cvdw", "AboPre", "AboVbc", "AboExp")] +
                       [(n, np.int32) for n in ("IxPF", "MdQst", "MdVdw", "IxHe")])


class CLineBlock(C.Structure):
    _fields_ = [("nlines", C.c_int64), ("nblock", C.c_int64), ("wlcent", _dp), ("flags", _ip), ("ileft", _ip),
                ("iright", _ip), ("lincop", _dp), ("linvvgt", _dp), ("linavgt", _dp), ("npi", _ip), ("nsi", _ip),
                ("pi_off", C.POINTER(C.c_int64)), ("si_off", C.POINTER(C.c_int64)), ("splpi", _fp), ("strpi", _fp),
                ("splsi", _fp), ("strsi", _fp)]


class LineBlock:
    """The reference's line arrays for the kernel-level routines (fsg_lineblock): per line wlcent (centre
    less Wfirst), flags, ileft, iright; per block line lincop / linvvgt / linavgt [nblock][ntau]; optional
    Zeeman components (npi, nsi, spl_pi, str_pi, spl_si, str_si) with shifts in [A]."""

    def __init__(self, wlcent, flags, ileft, iright, lincop=None, linvvgt=None, linavgt=None, zeeman=None):
        k = self._keep = {}
        b = CLineBlock()
        k["wlcent"] = _f64(wlcent); b.wlcent = _p(k["wlcent"], C.c_double)
        for name, arr in (("flags", flags), ("ileft", ileft), ("iright", iright)):
            k[name] = _i32(arr); setattr(b, name, _p(k[name], C.c_int32))
        b.nlines = len(k["wlcent"])
        if lincop is not None:
            for name, arr in (("lincop", lincop), ("linvvgt", linvvgt), ("linavgt", linavgt)):
                k[name] = _f64(arr); setattr(b, name, _p(k[name], C.c_double))
            b.nblock = k["lincop"].shape[0]
        if zeeman is not None:
            npi, nsi, spl_pi, str_pi, spl_si, str_si = zeeman
            k["npi"] = _i32(npi); k["nsi"] = _i32(nsi)
            k["pi_off"] = np.ascontiguousarray(np.concatenate([[0], np.cumsum(k["npi"])[:-1]]), np.int64)
            k["si_off"] = np.ascontiguousarray(np.concatenate([[0], np.cumsum(k["nsi"])[:-1]]), np.int64)
            for name, arr in (("splpi", spl_pi), ("strpi", str_pi), ("splsi", spl_si), ("strsi", str_si)):
                k[name] = _f32(arr if len(arr) else np.zeros(1, np.float32)); setattr(b, name, _p(k[name], C.c_float))
            b.npi = _p(k["npi"], C.c_int32); b.nsi = _p(k["nsi"], C.c_int32)
            b.pi_off = _p(k["pi_off"], C.c_int64); b.si_off = _p(k["si_off"], C.c_int64)
        self.c = b


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class Context:
    """One device context: grid + atmosphere + continuum + accumulators (fsg_ctx)."""

    def __init__(self, device=0, precision=PREC_MIXED, vmicro=0.0, epsopac=1e-4, vwfudge=1.0, h2brd=0.0,
                 vwmol=0.0, molbrd=0, limitram_gb=16.0):
        self._lib = lib()
        cfg = Config(device, precision, vmicro, epsopac, vwfudge, h2brd, vwmol, int(molbrd), limitram_gb)
        h = C.c_void_p()
        rc = self._lib.fsg_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise FsgError("fsg_create failed (%d): no usable CUDA device or bad configuration" % rc)
        self.h = h
        self.nwl = self.ntau = self.nmu = 0
        self._keep = {}

    def close(self):
        if getattr(self, "h", None):
            self._lib.fsg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stream_ptr(self):
        """The context's cudaStream_t as an integer (torch.cuda.ExternalStream can wrap it)."""
        return int(self._lib.fsg_cuda_stream(self.h))

    def launches(self):
        """Kernels launched by this context so far."""
        return int(self._lib.fsg_kernel_launches(self.h))

    def _ck(self, rc, what):
        if rc != 0:
            msg = self._lib.fsg_last_error(self.h)
            raise FsgError("%s failed (%d): %s" % (what, rc, msg.decode() if msg else ""))

    def set_grid(self, wmode, wstart, wend, dstep, wave=None):
        w = make_grid(wmode, wstart, wend, dstep) if wave is None else _f64(wave)
        self._ck(self._lib.fsg_set_grid(self.h, int(wmode), float(wstart), float(wend), float(dstep), len(w),
                                        _p(w, C.c_double)), "fsg_set_grid")
        self.nwl = len(w)
        self.wave = w
        self.wfirst = float(wstart)
        return w

    def set_atmosphere(self, st):
        """st: dict rhox, T, xne, xna, rho (FP64 [ntau]); fractionpf (FP32 [ntau][nspc]); xamass,
        potion (FP32 [nspc]); ion (int [nspc]); frac_h1, frac_he1[, frac_h2] (FP32 [ntau])."""
        a = {k: _f64(st[k]) for k in ("rhox", "T", "xne", "xna", "rho")}
        fpf = _f32(st["fractionpf"])
        ntau, nspc = fpf.shape
        x = dict(xamass=_f32(st["xamass"]), potion=_f32(st["potion"]), ion=_i32(st["ion"]),
                 h1=_f32(st["frac_h1"]), he1=_f32(st["frac_he1"]),
                 h2=_f32(st.get("frac_h2", np.zeros(ntau, np.float32))))
        self._ck(self._lib.fsg_set_atmosphere(
            self.h, ntau, _p(a["rhox"], C.c_double), _p(a["T"], C.c_double), _p(a["xne"], C.c_double),
            _p(a["xna"], C.c_double), _p(a["rho"], C.c_double), nspc, _p(fpf, C.c_float),
            _p(x["xamass"], C.c_float), _p(x["potion"], C.c_float), _p(x["ion"], C.c_int32),
            _p(x["h1"], C.c_float), _p(x["he1"], C.c_float), _p(x["h2"], C.c_float)), "fsg_set_atmosphere")
        self.ntau = ntau
        self.rhox = a["rhox"]; self.T = a["T"]; self.xne = a["xne"]

    def set_contopac(self, contopac, contopac_std=None, motype=0):
        co = _f64(contopac)
        if co.shape != (self.nwl, self.ntau):
            raise FsgError("contopac shape %s != (%d, %d)" % (co.shape, self.nwl, self.ntau))
        cs = _f64(contopac_std)
        self._ck(self._lib.fsg_set_contopac(self.h, _p(co, C.c_double), _p(cs, C.c_double), int(motype)),
                 "fsg_set_contopac")

    def set_contopac_dev(self, ptr):
        self._ck(self._lib.fsg_set_contopac_dev(self.h, C.c_void_p(ptr)), "fsg_set_contopac_dev")

    def set_geometry(self, radius, height=None):
        """fsg_set_geometry: spherical model of the given radius [cm] and layer heights [cm]
        (after set_atmosphere, which resets the model to plane-parallel); radius <= 0: plane-parallel."""
        h = None if height is None else _f64(height)
        self._keep["height"] = h
        self._ck(self._lib.fsg_set_geometry(self.h, float(radius), _p(h, C.c_double)), "fsg_set_geometry")

    def set_mu(self, xmu, wmu):
        xmu = _f64(xmu); wmu = _f64(wmu)
        self._ck(self._lib.fsg_set_mu(self.h, len(xmu), _p(xmu, C.c_double), _p(wmu, C.c_double)), "fsg_set_mu")
        self.nmu = len(xmu)

    def lineop_reset(self):
        self._ck(self._lib.fsg_lineop_reset(self.h), "fsg_lineop_reset")

    def lineop_calc(self, lines, want_lineopac=True, want_lines=True, want_linstr=False):
        """LineopCalc for one list; returns dict(lineopac, flags, ileft, iright, stats[, linstr]).
        want_linstr: central line depths of the retained lines (LinStrCalc; needs set_mu)."""
        n = lines.n
        lo = np.zeros((self.nwl, self.ntau)) if want_lineopac else None
        fl = np.zeros(max(n, 1), np.int32) if want_lines else None
        il = np.zeros(max(n, 1), np.int32) if want_lines else None
        ir = np.zeros(max(n, 1), np.int32) if want_lines else None
        ls = np.zeros(max(n, 1), np.float32) if want_linstr else None
        st = Stats()
        lines = self._he(lines)
        self._ck(self._lib.fsg_lineop_calc(self.h, C.byref(lines.c), _p(lo, C.c_double), _p(fl, C.c_int32),
                                           _p(il, C.c_int32), _p(ir, C.c_int32), _p(ls, C.c_float), C.byref(st)),
                 "fsg_lineop_calc")
        out = dict(lineopac=lo, stats=st.asdict())
        if want_lines:
            out.update(flags=fl[:n], ileft=il[:n], iright=ir[:n])
        if want_linstr:
            out["linstr"] = ls[:n]
        return out

    def lineop_calc_dev(self, dlines):
        st = Stats()
        self._ck(self._lib.fsg_lineop_calc_dev(self.h, C.byref(dlines), C.byref(st)), "fsg_lineop_calc_dev")
        return st.asdict()

    def central_dev(self, dlines, d_flags, d_ileft, d_iright):
        """Central pass of a device list into device int32 arrays (pointers); returns the retained count."""
        nk = C.c_int64(0)
        v = lambda p: C.cast(C.c_void_p(p), C.POINTER(C.c_int32)) if p else None
        self._ck(self._lib.fsg_central_dev(self.h, C.byref(dlines), v(d_flags), v(d_ileft), v(d_iright),
                                           C.byref(nk)), "fsg_central_dev")
        return nk.value

    def accumulate_dev(self, dlines, d_flags, d_ileft, d_iright, i0, i1):
        """Accumulate a device list with given windows over wavelengths i0..i1 (1-based, inclusive)."""
        st = Stats()
        v = lambda p: C.cast(C.c_void_p(p), C.POINTER(C.c_int32)) if p else None
        self._ck(self._lib.fsg_accumulate_dev(self.h, C.byref(dlines), v(d_flags), v(d_ileft), v(d_iright), int(i0),
                                              int(i1), C.byref(st)), "fsg_accumulate_dev")
        return st.asdict()

    def disk_integ_conv(self, radii, vsini=0.0, vmacro=0.0, vgau=0.0):
        """RadTranCalc + DiskInteg with broadening: (sfl, sfc) [nwl]."""
        r = _f64(radii)
        sfl = np.zeros(self.nwl); sfc = np.zeros(self.nwl)
        self._ck(self._lib.fsg_disk_integ_conv(self.h, _p(r, C.c_double), C.c_double(vsini), C.c_double(vmacro),
                                               C.c_double(vgau), _p(sfl, C.c_double), _p(sfc, C.c_double)),
                 "fsg_disk_integ_conv")
        return sfl, sfc

    def disk_integ_conv_dev(self, radii, vsini, vmacro, vgau, d_spl, d_spc, d_sfl, d_sfc):
        r = _f64(radii)
        v = C.c_void_p
        self._ck(self._lib.fsg_disk_integ_conv_dev(self.h, _p(r, C.c_double), C.c_double(vsini), C.c_double(vmacro),
                                                   C.c_double(vgau), v(d_spl), v(d_spc), v(d_sfl), v(d_sfc)),
                 "fsg_disk_integ_conv_dev")

    def set_fractionpf(self, fractionpf):
        fpf = _f32(fractionpf)
        self._ck(self._lib.fsg_set_fractionpf(self.h, _p(fpf, C.c_float)), "fsg_set_fractionpf")

    def set_hestark(self, hegam, heshf, spc_he1):
        """He I Stark broadening and shift tables [nhe][ntau] (hestark.f90) and the He I species index;
        the lists' ihe columns pick the entries."""
        g = _f64(hegam); h = _f64(heshf)
        self._ck(self._lib.fsg_set_hestark(self.h, g.shape[0], _p(g, C.c_double), _p(h, C.c_double), int(spc_he1)),
                 "fsg_set_hestark")
        self._he_spc = None

    def hestark_init(self, frac_hii, frac_heii, spc_he1):
        """HeStarkInit for the current atmosphere (as XlineInit runs it, opacity.f90:91): the 37 tabulated
        He I lines' widths and shifts from its T, Xne and the FP32 H II and He II densities, uploaded with
        fsg_set_hestark; from then on lists without an ihe column are matched to the table as XlineSetup
        does (opacity.f90:176).  Call again after set_atmosphere."""
        g, h = hestark_tables(self.T, self.xne, frac_hii, frac_heii)
        self.set_hestark(g, h, spc_he1)
        self._he_spc = int(spc_he1)

    def _he(self, lines):
        spc = getattr(self, "_he_spc", None)
        return lines if spc is None else lines._with_he_match(spc, self.wfirst)

    def set_fault(self, kind, value=0.0):
        """Failure injection for tests of the error paths: FAULT_ALLOC_LIMIT (bytes), FAULT_COPY_TIMEOUT
        (wait bound in ms), FAULT_NONE."""
        self._ck(self._lib.fsg_set_fault(self.h, int(kind), float(value)), "fsg_set_fault")

    def set_vmicro(self, vmicro):
        self._ck(self._lib.fsg_set_vmicro(self.h, C.c_double(float(vmicro))), "fsg_set_vmicro")

    def adjoint_dev(self, dlines, d_gflux, d_glin, d_gvmic, d_gkappa=None):
        """dL/dSfL (device pointer, [nwl]) -> per-line dL/d ln gf and vmicro shares (device pointers)."""
        v = lambda p: C.c_void_p(p) if p else None
        self._ck(self._lib.fsg_adjoint_dev(self.h, C.byref(dlines), v(d_gflux), v(d_gkappa), v(d_glin), v(d_gvmic)),
                 "fsg_adjoint_dev")

    def adjoint_range_dev(self, dlines, d_flags, d_ileft, d_iright, i0, i1, d_gflux, d_glin, d_gvmic, d_gkappa=None):
        """The adjoint of one wavelength shard [i0, i1] with the whole list's windows (device pointers)."""
        v = lambda p: C.c_void_p(p) if p else None
        self._ck(self._lib.fsg_adjoint_range_dev(self.h, C.byref(dlines), v(d_flags), v(d_ileft), v(d_iright), int(i0),
                                                 int(i1), v(d_gflux), v(d_gkappa), v(d_glin), v(d_gvmic)),
                 "fsg_adjoint_range_dev")

    def lineop_get(self):
        lo = np.zeros((self.nwl, self.ntau))
        self._ck(self._lib.fsg_lineop_get(self.h, _p(lo, C.c_double)), "fsg_lineop_get")
        return lo

    def lineop_set(self, lineopac):
        lo = _f64(lineopac)
        self._ck(self._lib.fsg_lineop_set(self.h, _p(lo, C.c_double)), "fsg_lineop_set")

    def radtran(self):
        """RadTranCalc + disk integration: (spl [nwl][nmu], spc, sfl [nwl], sfc)."""
        spl = np.zeros((self.nwl, self.nmu)); spc = np.zeros((self.nwl, self.nmu))
        sfl = np.zeros(self.nwl); sfc = np.zeros(self.nwl)
        self._ck(self._lib.fsg_radtran(self.h, _p(spl, C.c_double), _p(spc, C.c_double), _p(sfl, C.c_double),
                                       _p(sfc, C.c_double)), "fsg_radtran")
        return spl, spc, sfl, sfc

    def radtran_dev(self, d_spl, d_spc, d_sfl, d_sfc):
        v = lambda p: C.c_void_p(p) if p else None
        self._ck(self._lib.fsg_radtran_dev(self.h, v(d_spl), v(d_spc), v(d_sfl), v(d_sfc)), "fsg_radtran_dev")

    def radtran_range_dev(self, i0, i1, d_spl, d_spc, d_sfl, d_sfc):
        """RadTranCalc + flux over wavelengths i0..i1 (1-based, inclusive) into whole-grid device arrays."""
        v = lambda p: C.c_void_p(p) if p else None
        self._ck(self._lib.fsg_radtran_range_dev(self.h, int(i0), int(i1), v(d_spl), v(d_spc), v(d_sfl), v(d_sfc)),
                 "fsg_radtran_range_dev")

    def mag_lineop_calc(self, lines, bframe, bfield, want=True, want_linstr=False):
        n = lines.n
        bf = _f64(bfield)
        mlo = np.zeros((self.nwl, self.ntau, 6)) if want else None
        fl = np.zeros(max(n, 1), np.int32); il = np.zeros(max(n, 1), np.int32); ir = np.zeros(max(n, 1), np.int32)
        ls = np.zeros(max(n, 1), np.float32) if want_linstr else None
        st = Stats()
        lines = self._he(lines)
        self._ck(self._lib.fsg_mag_lineop_calc(self.h, C.byref(lines.c), int(bframe), _p(bf, C.c_double), len(bf),
                                               _p(mlo, C.c_double), _p(fl, C.c_int32), _p(il, C.c_int32),
                                               _p(ir, C.c_int32), _p(ls, C.c_float), C.byref(st)),
                 "fsg_mag_lineop_calc")
        out = dict(maglineopac=mlo, flags=fl[:n], ileft=il[:n], iright=ir[:n], stats=st.asdict())
        if want_linstr:
            out["linstr"] = ls[:n]
        return out

    def mag_radtran(self, bframe, bfield):
        bf = _f64(bfield)
        spz = np.zeros((self.nwl, 4, self.nmu)); spc = np.zeros((self.nwl, self.nmu))
        sfl = np.zeros(self.nwl); sfc = np.zeros(self.nwl)
        self._ck(self._lib.fsg_mag_radtran(self.h, int(bframe), _p(bf, C.c_double), len(bf), _p(spz, C.c_double),
                                           _p(spc, C.c_double), _p(sfl, C.c_double), _p(sfc, C.c_double)),
                 "fsg_mag_radtran")
        return spz, spc, sfl, sfc

    # ---- kernel-level routines (the reference's elemental functions, batched on the GPU) -----------
    def xline_setup(self, lines):
        """XlineSetup of every line of a LineList: structured array of XCOEF_DTYPE."""
        xc = np.zeros(max(lines.n, 1), XCOEF_DTYPE)
        self._ck(self._lib.fsg_xline_setup(self.h, C.byref(lines.c), _ptr(xc)), "fsg_xline_setup")
        return xc[:lines.n]

    def xline_depth(self, xc):
        """XlineDepth at every depth: (lincop, linvvgt, linavgt) [n][ntau]."""
        xc = np.ascontiguousarray(xc, XCOEF_DTYPE)
        n = len(xc)
        out = [np.zeros((max(n, 1), self.ntau)) for _ in range(3)]
        self._ck(self._lib.fsg_xline_depth(self.h, n, _ptr(xc), *[_ptr(o) for o in out]), "fsg_xline_depth")
        return tuple(o[:n] for o in out)

    def lineopacity1(self, block, wl, l1, l2, iwl, loff=0):
        """LineOpacity1 at points (wl, l1, l2, iwl arrays; 1-based): [npts][ntau]."""
        wl = _f64(wl); l1 = _i32(l1); l2 = _i32(l2); iwl = _i32(iwl)
        out = np.zeros((max(len(wl), 1), self.ntau))
        self._ck(self._lib.fsg_lineopacity1(self.h, C.byref(block.c), len(wl), _ptr(wl), _ptr(l1), _ptr(l2), _ptr(iwl),
                                            int(loff), _ptr(out)), "fsg_lineopacity1")
        return out[:len(wl)]

    def mag_lineopacity1(self, block, wl, l1, l2, iwl, loff=0):
        """MagLineOpacity1 at points: [npts][ntau][6]."""
        wl = _f64(wl); l1 = _i32(l1); l2 = _i32(l2); iwl = _i32(iwl)
        out = np.zeros((max(len(wl), 1), self.ntau, 6))
        self._ck(self._lib.fsg_mag_lineopacity1(self.h, C.byref(block.c), len(wl), _ptr(wl), _ptr(l1), _ptr(l2),
                                                _ptr(iwl), int(loff), _ptr(out)), "fsg_mag_lineopacity1")
        return out[:len(wl)]

    def lineopacity2(self, block, wl, iline, iwl, lincop, linvvgt, linavgt):
        """LineOpacity2 at points, each with its own parameter rows [npts][ntau]: [npts][ntau]."""
        wl = _f64(wl); iline = _i32(iline); iwl = _i32(iwl)
        c, v, a = _f64(lincop), _f64(linvvgt), _f64(linavgt)
        out = np.zeros((max(len(wl), 1), self.ntau))
        self._ck(self._lib.fsg_lineopacity2(self.h, C.byref(block.c), len(wl), _ptr(wl), _ptr(iline), _ptr(iwl),
                                            _ptr(c), _ptr(v), _ptr(a), _ptr(out)), "fsg_lineopacity2")
        return out[:len(wl)]

    def analytic_window(self, flags, lincop, linvvgt, linavgt, contopac):
        """AnalyticWindow of n lines (rows [n][ntau]): half-widths [n] in A."""
        f = _i32(flags); c, v, a, co = _f64(lincop), _f64(linvvgt), _f64(linavgt), _f64(contopac)
        out = np.zeros(max(len(f), 1))
        self._ck(self._lib.fsg_analytic_window(self.h, len(f), _ptr(f), _ptr(c), _ptr(v), _ptr(a), _ptr(co),
                                               _ptr(out)), "fsg_analytic_window")
        return out[:len(f)]

    def stokes_prf_pp(self, iwl, src, sphi2, cphi2, cphi, s2psi, c2psi):
        """StokesPrfPP at grid wavelengths iwl (1-based) with sources src [npts][ntau]: [npts][4][nmu]."""
        iwl = _i32(iwl); src = _f64(src)
        g = [_f64(x) for x in (sphi2, cphi2, cphi, s2psi, c2psi)]
        out = np.zeros((max(len(iwl), 1), 4, self.nmu))
        self._ck(self._lib.fsg_stokes_prf_pp(self.h, len(iwl), _ptr(iwl), _ptr(src), *[_ptr(x) for x in g], _ptr(out)),
                 "fsg_stokes_prf_pp")
        return out[:len(iwl)]

    def hvoigt(self, a, v):
        a = _f64(a); v = _f64(v); h = np.zeros_like(a)
        self._ck(self._lib.fsg_hvoigt(self.h, len(a), _p(a, C.c_double), _p(v, C.c_double), _p(h, C.c_double)),
                 "fsg_hvoigt")
        return h

    def fvoigt(self, a, v):
        a = _f64(a); v = _f64(v); h = np.zeros_like(a); l = np.zeros_like(a)
        self._ck(self._lib.fsg_fvoigt(self.h, len(a), _p(a, C.c_double), _p(v, C.c_double), _p(h, C.c_double),
                                      _p(l, C.c_double)), "fsg_fvoigt")
        return h, l

    def voigt_tables(self):
        v = np.zeros((402, 1002), np.float32); f = np.zeros((402, 1002, 2), np.float32)
        self._ck(self._lib.fsg_voigt_tables(self.h, _p(v, C.c_float), _p(f, C.c_float)), "fsg_voigt_tables")
        return v, f

    def locprf_pp(self, xmu, xki, src, rhox):
        xmu = _f64(xmu); xki = np.atleast_2d(_f64(xki)); src = np.atleast_2d(_f64(src)); rhox = _f64(rhox)
        nprof, ntau = xki.shape
        out = np.zeros((nprof, len(xmu)))
        self._ck(self._lib.fsg_locprf_pp(self.h, nprof, len(xmu), _p(xmu, C.c_double), ntau, _p(xki, C.c_double),
                                         _p(src, C.c_double), _p(rhox, C.c_double), _p(out, C.c_double)),
                 "fsg_locprf_pp")
        return out


class Batch:
    """Batched synthesis (fsg_batch_*): many contexts (grid, atmosphere, continuum and mu set, mixed
    precision) and one line list sorted by wavelength.  run() replays one CUDA graph of the whole
    batch (tuned and captured on the first call); flux(i) reads atmosphere i's flux.  Each atmosphere
    takes the lines with centres in [wstart - margin, wend + margin]; margin = 0 (the default) is the
    reference's reader rule (ioutils.f90:752-753, 1496-1497)."""

    def __init__(self, contexts, lines, margin=0.0):
        self._lib = lib()
        self.contexts = list(contexts)
        self.lines = lines
        hs = (C.c_void_p * len(self.contexts))(*[c.h.value for c in self.contexts])
        h = C.c_void_p()
        rc = self._lib.fsg_batch_create(hs, len(self.contexts), C.byref(lines.c), float(margin), C.byref(h))
        if rc != 0:
            raise FsgError("fsg_batch_create (%d): %s" % (rc, self._lib.fsg_batch_last_error(None).decode()))
        self.h = h

    def _ck(self, rc, what):
        if rc != 0:
            raise FsgError("%s (%d): %s" % (what, rc, self._lib.fsg_batch_last_error(self.h).decode()))

    def tune(self):
        t = BatchTuning()
        self._ck(self._lib.fsg_batch_tune(self.h, C.byref(t)), "fsg_batch_tune")
        return t.asdict()

    def set_tuning(self, tuning):
        t = BatchTuning(int(tuning["tile_pix"]), int(tuning["wing_ctas"]), int(tuning["core_ctas"]),
                        float(tuning.get("ms_wing", 0.0)), float(tuning.get("ms_core", 0.0)))
        self._ck(self._lib.fsg_batch_set_tuning(self.h, C.byref(t)), "fsg_batch_set_tuning")

    def run(self):
        st = BatchStats()
        self._ck(self._lib.fsg_batch_run(self.h, C.byref(st)), "fsg_batch_run")
        return st.asdict()

    def flux(self, i):
        n = self.contexts[i].nwl
        sfl = np.zeros(n); sfc = np.zeros(n)
        self._ck(self._lib.fsg_batch_flux(self.h, int(i), _p(sfl, C.c_double), _p(sfc, C.c_double)), "fsg_batch_flux")
        return sfl, sfc

    def stream_ptr(self):
        return self._lib.fsg_batch_stream(self.h)

    def close(self):
        if getattr(self, "h", None):
            self._lib.fsg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
