/*
 * fastspec_gpu.h -- C-ABI of the B200 line-opacity -> formal-solver path of FastSpec.
 *
 * The reference is a Fortran 90 program whose drivers exchange data through module globals
 * (shared.f90:447-548).  This ABI is what its ISO_C_BINDING shim would bind in their place:
 * plain pointers and sizes, no CUDA or torch types.  Every entry point returns 0 on success
 * or a negative FSG_E* code; fsg_last_error() gives the message.  The Fortran shim maps a
 * nonzero status to ErrStop (utils.f90:201), the reference's fatal-error path.
 *
 * Conventions (the reference's, seen from C):
 *   - arrays are Fortran column-major: LineOpac(Ntau,Nwl) -> double[nwl][ntau],
 *     MagLineOpac(6,Ntau,Nwl) -> double[nwl][ntau][6], SpL/SpC(Nmu,Nwl) -> double[nwl][nmu],
 *     SpZ(Nmu,4,Nwl) -> double[nwl][4][nmu], FractionPF(Maxspl,Ntau) -> float[ntau][nspc];
 *   - line and wavelength indices on output are 1-based (Ileft, Iright as the reference);
 *   - the caller owns every host array; the context owns device buffers;
 *   - a context is not thread-safe; use one per host thread (each has its own stream).
 * Functions with a _dev suffix take DEVICE pointers (inputs already resident in HBM).
 */
#ifndef FASTSPEC_GPU_H
#define FASTSPEC_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FSG_OK            0
#define FSG_E_ARG        -1   /* invalid argument (sizes, null pointers, ranges) */
#define FSG_E_CUDA       -2   /* CUDA runtime error */
#define FSG_E_NOMEM      -3   /* device or host allocation failed */
#define FSG_E_STATE      -4   /* call order: grid / atmosphere / continuum not set */
#define FSG_E_SEGMENT    -5   /* lines at one wavelength exceed the block capacity */
#define FSG_E_TIMEOUT    -6   /* a bounded device wait gave up (error word set) */

#define FSG_PREC_MIXED    0   /* FP32 Voigt + compensated on-chip sums, FP64 prefactors */
#define FSG_PREC_FP64     1   /* plain FP64-faithful path: per-wavelength gather as LineOpacity1 */

typedef struct fsg_ctx fsg_ctx;

/* Configuration: the Config-module fields the hot path reads (shared.f90:416-443). */
typedef struct {
    int    device;        /* CUDA device ordinal */
    int    precision;     /* FSG_PREC_MIXED or FSG_PREC_FP64 */
    double vmicro;        /* VMIC [km/s] */
    double epsopac;       /* EPSOPAC, line inclusion threshold (default 1e-4) */
    double vwfudge;       /* VWFUDGE (default 1) */
    double h2brd;         /* H2BRD (default 0) */
    double vwmol;         /* VWMOL (default 0) */
    int    molbrd;        /* MOLBRD 0/1 */
    double limitram_gb;   /* LIMITRAM: cap of the per-block line parameter buffers [GB] */
} fsg_config;

/* Line list, structure of arrays (LineData records, shared.f90:451-482).
 * kind: 0 LineTypeAtm (HDF atomic), 1 LineTypeMol (single-species molecular), 2 LineTypeMag
 * (ASCII .z / magnetic).  ismol: molecule flag of LineTypeMag records (IsMolecule).
 * ihe: He I Stark table entry (HeMatchIdx, 1-based; fsg_he_match_idx fills it) or 0; may be NULL.
 * Zeeman components (magnetic lists only; NULL otherwise): line i owns npi[i] pi components at
 * spl_pi[pi_off[i] ...] / str_pi[...] and nsi[i] sigma components (blue half first, then red,
 * as ReadAscMag stores them, ioutils.f90:1393-1410).  Shifts are in the reader's units
 * (Lande-type factors), scaled by Kz |B| lambda^2 inside fsg_mag_lineop_calc. */
typedef struct {
    int64_t       n;
    const double *wl;                 /* air wavelength [A], sorted ascending */
    const float  *elo, *gf, *grad, *gqst, *gvdw;
    const int32_t *spc;               /* species index 0..nspc-1 */
    int32_t       kind;               /* one kind for the whole list */
    const int32_t *ismol;             /* may be NULL (all 0) */
    const int32_t *ihe;               /* may be NULL */
    const int32_t *npi, *nsi;
    const int64_t *pi_off, *si_off;
    const float   *spl_pi, *str_pi, *spl_si, *str_si;
} fsg_lines;

typedef struct {
    int64_t nlines_in, nlines_used, nwide, nweak, nblocks;
    double  line_evals;     /* profile evaluations inside windows: Ntau x the retained lines' window
                               wavelengths (x each line's Zeeman components if magnetic), in both
                               precisions */
    double  ms_center, ms_params, ms_accum, ms_total;   /* device time per stage [ms] */
    int64_t accum_launches; /* launches of the accumulation kernel */
    double  ms_accum_kernels;   /* summed device time of those launches [ms] */
    double  ms_wing_kernels, ms_core_kernels;   /* mixed path: the wing and core passes of it [ms] */
    double  core_evals;     /* mixed path: the core pass's evaluations (table and continued fraction, s < 196) */
} fsg_stats;

/* Tracing and metrics.  Every driver call (fsg_lineop_calc(_dev), fsg_mag_lineop_calc, fsg_radtran(_dev),
 * fsg_radtran_range_dev, fsg_mag_radtran, fsg_batch_run) is an NVTX range named after the entry point.
 * When the environment variable FSG_METRICS_JSONL names a file, each such call appends one JSON line to
 * it: the call, its status, its host wall time [ms] and the stage figures it produced (fsg_stats /
 * fsg_batch_stats fields, or the grid sizes for the solvers) -- the counterpart of the reference's
 * per-stage reports (lines read and used, time of the line opacity and of the radiative transfer,
 * fastspec.f90:393-425). */

/* ---- context ------------------------------------------------------------------------- */
int         fsg_create(const fsg_config *cfg, fsg_ctx **out);
void        fsg_destroy(fsg_ctx *ctx);
const char *fsg_last_error(const fsg_ctx *ctx);
int         fsg_version(void);
/* Number of kernels this context has launched since it was created (monotonic). */
int64_t     fsg_kernel_launches(const fsg_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t, as void*), for callers that time or order work
 * on it.  Every entry point returns after its work on this stream has completed. */
void       *fsg_cuda_stream(fsg_ctx *ctx);

/* ---- set-up (the reference's Init, synth.f90:22-331) ------------------------------------ */
/* Wavelength grid of Init (synth.f90:56-74): wave[] = offsets from wstart.  Returns Nwl in
 * *nwl; wave may be NULL to query the size.  Host computation: set-up, not hot path. */
int fsg_make_grid(int wmode, double wstart, double wend, double dstep, double *wave, int *nwl);
/* Upload the grid (wave = offsets from wfirst = wstart, as Wave in SpecData). */
int fsg_set_grid(fsg_ctx *ctx, int wmode, double wstart, double wend, double dstep, int nwl,
                 const double *wave);
/* Model atmosphere after the EOS (AtmosData) and the species data the opacity kernel reads:
 * FractionPF [ntau][nspc] (FP32), Xamass, PotIon (FP32), ion stage per species, and the
 * H I / He I / H2 number densities of the perturber sum (Fraction, FP32).  Runs XlineInit
 * (opacity.f90:65-93) on the device.  Replaces (opacity.f90:65-93) + module state. */
int fsg_set_atmosphere(fsg_ctx *ctx, int ntau, const double *rhox, const double *T,
                       const double *xne, const double *xna, const double *rho, int nspc,
                       const float *fractionpf, const float *xamass, const float *potion,
                       const int32_t *ion, const float *frac_h1, const float *frac_he1,
                       const float *frac_h2);
/* Model geometry (ReadModel, ioutils.f90:1630-1700; SphereInit, solver.f90:45-120): radius [cm] > 0
 * makes the model spherical with layer heights height [ntau] [cm] above the radius (decreasing inward,
 * radius + height > 0, 1e9 <= radius <= 1e15, as ReadModel checks); radius <= 0 returns to plane-parallel
 * (height may then be NULL).  fsg_set_atmosphere resets the model to plane-parallel, as reading a new
 * model does, so call this after it.  The rays (one per angle of fsg_set_mu) are built on the host at
 * the next RadTranCalc / LinStrCalc / MagRadTranCalc call, which then solve along them (LocPrfSph,
 * StokesPrfSph; errors: an angle mu <= 0, a ray tangent in the top layer); the batched path and the
 * adjoint solve along them too.  Replaces Radius/Atmos%Height (shared.f90:520-527). */
int fsg_set_geometry(fsg_ctx *ctx, double radius, const double *height);
/* Continuum opacity ContOpac [nwl][ntau] (ContopCalc output, synth.f90:642-674), ContOpacStd
 * [ntau] (may be NULL when motype == 0) and the model type (Motype). */
int fsg_set_contopac(fsg_ctx *ctx, const double *contopac, const double *contopac_std, int motype);
int fsg_set_contopac_dev(fsg_ctx *ctx, const double *d_contopac);
/* He I Stark widths/shifts HeGam/HeShf [nhe][ntau] (hestark.f90:332-370), optional; spc_he1 is the
 * 0-based index of He I among the species (IdxSpc(Ix%He1)).  Lines of that species take the Stark
 * width and shift of table entry ihe (fsg_lines.ihe, 1..nhe; 0 or ihe == NULL: none). */
int fsg_set_hestark(fsg_ctx *ctx, int nhe, const double *hegam, const double *heshf, int spc_he1);

/* HeStarkInit (hestark.f90:332-370), on the host, no context: HeGam [rad/s] and HeShf [A] of the
 * FSG_HE_NTAB tabulated He I lines (Dimitrijevic & Sahal-Brechot 1990 entries 1-32, 1984 entries
 * 33-37), [FSG_HE_NTAB][ntau], from T [K], Xne and the FP32 number densities of protons (Fraction
 * of H II) and He II ions, by three-point Lagrange interpolation in log10 T.  The tables go to
 * fsg_set_hestark with nhe = FSG_HE_NTAB.  FSG_E_ARG for null pointers, ntau < 1 or T <= 0. */
#define FSG_HE_NTAB 37
int fsg_hestark_tables(int ntau, const double *T, const double *xne, const float *frac_hii,
                       const float *frac_heii, double *hegam, double *heshf);
/* HeMatchIdx (hestark.f90:376-389) at its XlineSetup call site (opacity.f90:176), on the host, no
 * context: ihe[i] = the first table entry 1..FSG_HE_NTAB whose centre lies within 1 A of the line's
 * WaveL = (wl[i] - wfirst) + wfirst and whose lower level energy lies within 0.01 eV of elo[i], for
 * lines of species spc_he1; 0 otherwise.  wfirst is the grid's first wavelength (fsg_set_grid's
 * wstart).  The result is the ihe column of fsg_lines. */
int fsg_he_match_idx(long n, const double *wl, const float *elo, const int32_t *spc, int spc_he1,
                     double wfirst, int32_t *ihe);

/* ---- hot path ------------------------------------------------------------------------- */
/* LineopCalc (synth.f90:747-1095): central pass (XlineSetup/XlineDepth, weak-line rejection,
 * AnalyticWindow + WaveIdx), then the line opacity accumulated onto the device LineOpac.
 * lineopac (host, [nwl][ntau], may be NULL) receives the accumulated total when non-NULL.
 * Per-line outputs (host, length n, may be NULL): LinFlag bits, Ileft, Iright, LinStr
 * (LinStrCalc, synth.f90:1774-1822: REAL(4) central depth of each retained line from the
 * continuum and line + continuum intensities at its centre, disk-integrated with the fsg_set_mu
 * weights when nmu > 1; 0 for rejected lines; FSG_E_STATE without fsg_set_mu). */
int fsg_lineop_calc(fsg_ctx *ctx, const fsg_lines *lines, double *lineopac, int32_t *flags,
                    int32_t *ileft, int32_t *iright, float *linstr, fsg_stats *stats);
int fsg_lineop_calc_dev(fsg_ctx *ctx, const fsg_lines *d_lines, fsg_stats *stats);
/* LineopCalc split for wavelength sharding (no counterpart call in the reference, whose driver does
 * both steps in one routine, synth.f90:833-907 and 1000-1090):
 * fsg_central_dev runs the central pass (weak-line tests, AnalyticWindow, WaveIdx) of a device
 * list into caller-owned device arrays LinFlag / Ileft / Iright (n each) and returns the retained
 * count; fsg_accumulate_dev accumulates a device list whose windows are given onto the device
 * LineOpac, over wavelength indices i0..i1 (1-based, inclusive) only.  Each wavelength of the range
 * sums the same lines in the same order as a whole-grid fsg_lineop_calc_dev (mixed precision: equal
 * to rounding, as the Kahan groups of a tile cut by the range ends, and the blocks of a class, may
 * differ; FP64: the same segments and order, so equal bit for bit); other wavelengths are left as
 * they are. */
int fsg_central_dev(fsg_ctx *ctx, const fsg_lines *d_lines, int32_t *d_flags, int32_t *d_ileft,
                    int32_t *d_iright, int64_t *nkeep);
int fsg_accumulate_dev(fsg_ctx *ctx, const fsg_lines *d_lines, const int32_t *d_flags,
                       const int32_t *d_ileft, const int32_t *d_iright, int i0, int i1, fsg_stats *stats);
/* Zero / read / write the device LineOpac accumulator ([nwl][ntau]; OPACITY= re-entry). */
int fsg_lineop_reset(fsg_ctx *ctx);
int fsg_lineop_get(fsg_ctx *ctx, double *lineopac);
int fsg_lineop_set(fsg_ctx *ctx, const double *lineopac);
const double *fsg_lineop_device_ptr(fsg_ctx *ctx);

/* Limb angles and flux weights used by RadTranCalc, LinStrCalc and the disk integration. */
int fsg_set_mu(fsg_ctx *ctx, int nmu, const double *xmu, const double *wmu);
/* RadTranCalc (synth.f90:1825-1901; plane-parallel or spherical, fsg_set_geometry) + DiskInteg without
 * broadening (convol.f90:111-235):
 * spl/spc [nwl][nmu], sfl/sfc [nwl]; any output may be NULL.  Uses the device LineOpac. */
int fsg_radtran(fsg_ctx *ctx, double *spl, double *spc, double *sfl, double *sfc);
int fsg_radtran_dev(fsg_ctx *ctx, double *d_spl, double *d_spc, double *d_sfl, double *d_sfc);
/* The same over the wavelength indices i0..i1 only (1-based, inclusive): the formal solver and flux
 * of one wavelength shard.  The device outputs keep the whole grid's layout; rows i0..i1 are
 * written, the others are left as they are.  RadTranCalc's loop over wavelengths is independent per
 * wavelength (synth.f90:1825-1866), so each row equals the whole-grid call's. */
int fsg_radtran_range_dev(fsg_ctx *ctx, int i0, int i1, double *d_spl, double *d_spc, double *d_sfl,
                          double *d_sfc);

/* DiskInteg with broadening (convol.f90:67-300): rotation (vsini [km/s], annulus kernels from the
 * nmu + 1 projected radii of fsg_mu_quadrature), radial-tangential macroturbulence (vmacro
 * [km/s]), then Gaussian broadening of the flux (vgau: FWHM [km/s], or a resolving power when
 * > 1000).  _dev: spl/spc [nwl][nmu] and sfl/sfc [nwl] on the device; the host form runs
 * RadTranCalc on the device LineOpac first and returns the broadened flux. */
int fsg_disk_integ_conv_dev(fsg_ctx *ctx, const double *radii, double vsini, double vmacro, double vgau,
                            const double *d_spl, const double *d_spc, double *d_sfl, double *d_sfc);
int fsg_disk_integ_conv(fsg_ctx *ctx, const double *radii, double vsini, double vmacro, double vgau,
                        double *sfl, double *sfc);

/* ---- magnetic path ---------------------------------------------------------------------- */
/* MagLineopCalc (synth.f90:1098-1455): bframe/bfield as BFRAME/BFIELD (3 values for frames
 * 0/1, 2*nmu+1 for frame 2).  Accumulates the device MagLineOpac [nwl][ntau][6].  linstr as for
 * fsg_lineop_calc (the magnetic driver uses the same non-magnetic central depths). */
int fsg_mag_lineop_calc(fsg_ctx *ctx, const fsg_lines *lines, int bframe, const double *bfield,
                        int nbfield, double *maglineopac, int32_t *flags, int32_t *ileft,
                        int32_t *iright, float *linstr, fsg_stats *stats);
int fsg_mag_lineop_reset(fsg_ctx *ctx);
/* MagRadTranCalc (synth.f90:1904-2111; plane-parallel or spherical): spz [nwl][4][nmu], spc [nwl][nmu],
 * and the Stokes-I flux sfl / continuum flux sfc [nwl] (may be NULL). */
int fsg_mag_radtran(fsg_ctx *ctx, int bframe, const double *bfield, int nbfield, double *spz,
                    double *spc, double *sfl, double *sfc);

/* ---- kernel-level entry points (elemental reference functions, batched on the GPU) -------
 * Each evaluates many lines or wavelengths in one call with the drivers' own device code (FP64, the
 * reference's operand order).  Host arrays in the reference's argument meaning; line and wavelength
 * indices 1-based.  The atmosphere (and, for StokesPrfPP, the continuum, LineOpac, MagLineOpac and
 * angles) come from the context, as the reference's routines read them from module globals. */
typedef struct {            /* XlineCoef (opacity.f90:43-58); IxPF: 0-based species column */
    double  WaveL, Hnux, Elo, Gf, Grad, Xmass, Cqst, Qdiv, Cvdw, AboPre, AboVbc, AboExp;
    int32_t IxPF, MdQst, MdVdw, IxHe;
} fsg_xcoef;
/* The reference's line arrays as LineopCalc / MagLineopCalc hold them: per line (nlines) Wlcent (the
 * centre less Wfirst [A]), LinFlag, Ileft, Iright; per block line (nblock) LinCop, LinVvgt, LinAvgt
 * [nblock][ntau] (the reference's (Ntau, NlinesStep) arrays); for the magnetic routine the Zeeman
 * components by line (npi / nsi counts, pi_off / si_off offsets, shifts scaled to [A] as MagLineopCalc
 * scales them, synth.f90:1150-1154, and strengths; each sigma list holds its blue half first). */
typedef struct {
    int64_t nlines, nblock;
    const double *wlcent;
    const int32_t *flags, *ileft, *iright;
    const double *lincop, *linvvgt, *linavgt;
    const int32_t *npi, *nsi;
    const int64_t *pi_off, *si_off;
    const float *splpi, *strpi, *splsi, *strsi;
} fsg_lineblock;
/* XlineSetup (opacity.f90:96-235) of every line of a host list, with the flags the drivers set
 * before it (molecule and ABO bits from the list, synth.f90:837-845): xc[n]. Needs the grid and the
 * atmosphere, not the continuum. */
int fsg_xline_setup(fsg_ctx *ctx, const fsg_lines *lines, fsg_xcoef *xc);
/* XlineDepth (opacity.f90:239-293) of n lines at every depth: lincop/linvvgt/linavgt [n][ntau]. */
int fsg_xline_depth(fsg_ctx *ctx, int64_t n, const fsg_xcoef *xc, double *lincop, double *linvvgt,
                    double *linavgt);
/* LineOpacity1 (opacity.f90:297-346) at npts points: point k sums lines l1[k]..l2[k] of the block
 * (weak and wide lines, and lines whose window misses iwl[k], skipped) at Wl = wl[k] (the grid offset
 * Wave(iwl[k])), block line = line - loff: linop [npts][ntau] (divided by ContOpacStd under Motype 1). */
int fsg_lineopacity1(fsg_ctx *ctx, const fsg_lineblock *blk, int64_t npts, const double *wl,
                     const int32_t *l1, const int32_t *l2, const int32_t *iwl, int64_t loff, double *linop);
/* LineOpacity2 (opacity.f90:350-386): point k is line iline[k] of the block at Wl = wl[k], grid index
 * iwl[k], with its own rows lincop/linvvgt/linavgt [npts][ntau]: linop [npts][ntau]. */
int fsg_lineopacity2(fsg_ctx *ctx, const fsg_lineblock *blk, int64_t npts, const double *wl,
                     const int32_t *iline, const int32_t *iwl, const double *lincop, const double *linvvgt,
                     const double *linavgt, double *linop);
/* MagLineOpacity1 (opacity.f90:391-464) as LineOpacity1 over the block's Zeeman components:
 * maglinop [npts][ntau][6] (pi, blue and red sigma absorption; pi, blue and red dispersion). */
int fsg_mag_lineopacity1(fsg_ctx *ctx, const fsg_lineblock *blk, int64_t npts, const double *wl,
                         const int32_t *l1, const int32_t *l2, const int32_t *iwl, int64_t loff,
                         double *maglinop);
/* AnalyticWindow (opacity.f90:678-710) of n lines: line k with LinFlag flags[k] (He I entry in bits
 * 8-15) and rows lincop/linvvgt/linavgt/contopac [n][ntau] (ContOpacL: the continuum at its centre):
 * the window half-widths dw[n] [A]. */
int fsg_analytic_window(fsg_ctx *ctx, int64_t n, const int32_t *flags, const double *lincop,
                        const double *linvvgt, const double *linavgt, const double *contopac, double *dw);
/* StokesPrfPP (solver.f90:265-394) at npts grid wavelengths iwl[k]: the context's MagLineOpac (after
 * fsg_mag_lineop_calc), LineOpac, ContOpac, Rhox and angles, the source function src [npts][ntau] and
 * the field projection per angle sphi2, cphi2, cphi, s2psi, c2psi [nmu]: stokes [npts][4][nmu]
 * (I, Q, U, V). */
int fsg_stokes_prf_pp(fsg_ctx *ctx, int64_t npts, const int32_t *iwl, const double *src, const double *sphi2,
                      const double *cphi2, const double *cphi, const double *s2psi, const double *c2psi,
                      double *stokes);
/* HVoigt (voigt.f90:76-110) and FVoigt (voigt.f90:256-299) over host arrays of length n. */
int fsg_hvoigt(fsg_ctx *ctx, int64_t n, const double *a, const double *v, double *h);
int fsg_fvoigt(fsg_ctx *ctx, int64_t n, const double *a, const double *v, double *h, double *l);
/* The device-built FP32 tables VgtTab [402][1002] and FvTab [402][1002][2]. */
int fsg_voigt_tables(fsg_ctx *ctx, float *vgt, float *fvt);
/* LocPrfPP (solver.f90:123-179) for nprof independent profiles: xki/src [nprof][ntau],
 * ploc [nprof][nmu]. */
int fsg_locprf_pp(fsg_ctx *ctx, int nprof, int nmu, const double *xmu, int ntau,
                  const double *xki, const double *src, const double *rhox, double *ploc);
/* LocPrfPP for callers that cannot allocate device memory (no counterpart in the reference,
 * which allocates nothing on a device).  Hosts whose device memory belongs to their own pool
 * allocator (a framework's caching allocator, a Fortran driver that reserves its arrays at
 * start-up) cannot let a library call cudaMalloc/cudaFree per call: those calls synchronise the
 * device and fail when the pool holds the memory.  Every pointer is DEVICE memory owned by the
 * caller (xmu [nmu], xki/src [nprof][ntau], rhox [ntau], ploc [nprof][nmu]); the kernel's work
 * arrays sit in a fixed 8 MiB device array of the library, so nprof * ntau * 3 may not exceed
 * 1,048,576 (larger sizes return FSG_E_ARG).  stream is a cudaStream_t (NULL: the default
 * stream); the call waits for the kernel with cudaStreamSynchronize on that stream and returns
 * after it has finished.  The first call on a device looks up the array's device address with
 * that device current.  All calls share the array, so calls that overlap on the GPU race. */
int fsg_locprf_pp_noalloc(int nprof, int nmu, const double *d_xmu, int ntau, const double *d_xki,
                          const double *d_src, const double *d_rhox, double *d_ploc, void *stream);
/* MuQuadrature (utils.f90:1273-1330): x (in/out when setnodes == 0), w, r [n+1]. */
int fsg_mu_quadrature(int quad, int n, double *x, double *w, double *r, int setnodes);
/* ZeemanPattern (utils.f90:901-1004): outputs hold up to 2*jup+1 entries each. */
int fsg_zeeman_pattern(float jlo, float jup, float glo, float gup, int32_t *npi, float *spi,
                       float *rpi, int32_t *nsig, float *ssig, float *rsig);


/* ---- derivatives (no counterpart in the reference) ---------------------------------------------
 * fsg_set_vmicro changes the microturbulence of later calls [km/s]; fsg_set_fractionpf replaces the
 * FractionPF of fsg_set_atmosphere ([ntau][nspc]) and keeps the rest of the atmosphere.
 * fsg_adjoint_dev: given d_gflux = dL/dSfL [nwl] (device) for the flux of the last fsg_radtran(_dev)
 * of this context, computes with one backward sweep of the DELO-Bezier solver per wavelength (per ray
 * of a spherical model, each ray point's derivative returned to the layer it samples)
 * d_gkappa = dL/dLineOpac [nwl][ntau] (may be NULL: kept inside the context), and per line of the
 * device list d_lines -- which must be the list of the last fsg_lineop_calc(_dev), whose windows it
 * uses -- d_glin[l] = sum dL/dLineOpac * H * LinCop (= dL/d ln gf_l and, summed over an element's
 * lines, dL/d ln abundance with the continuum and the EOS held fixed) and d_gvmic[l] = the line's
 * share of dL/dvmicro.  Profiles are recomputed (FP64, the reference's tables), their v and a
 * derivatives from the Faddeeva relation dw/dz = -2 z w + 2i/sqrt(pi). */
int fsg_set_vmicro(fsg_ctx *ctx, double vmicro);
int fsg_set_fractionpf(fsg_ctx *ctx, const float *fractionpf);
int fsg_adjoint_dev(fsg_ctx *ctx, const fsg_lines *d_lines, const double *d_gflux, double *d_gkappa,
                    double *d_glin, double *d_gvmic);
/* The same for one wavelength shard: the windows of the whole list are given (the sharded forward's
 * gathered LinFlag / Ileft / Iright), and each line's sums run over the part of its window inside
 * wavelengths i0..i1 (1-based, inclusive), window-edge terms only where the window's own edge lies
 * in the range.  The adjoint is linear in dL/dSfL and the ranges of a partition cover each window
 * point once, so the sum over ranks of glin and gvmic is the whole-grid gradient (one all-reduce);
 * LineOpac outside the range is not read. */
int fsg_adjoint_range_dev(fsg_ctx *ctx, const fsg_lines *d_lines, const int32_t *d_flags,
                          const int32_t *d_ileft, const int32_t *d_iright, int i0, int i1,
                          const double *d_gflux, double *d_gkappa, double *d_glin, double *d_gvmic);

/* ---- failure injection, for tests of the error paths (no counterpart in the reference) -------
 * FSG_FAULT_ALLOC_LIMIT: the context's device allocations larger than value bytes fail as on an
 * exhausted device (FSG_E_NOMEM with the buffer's name; the context stays usable).
 * FSG_FAULT_COPY_TIMEOUT: every chunk of line records the accumulation kernels stage expects 16 bytes
 * more than its bulk copies deliver, so its mbarrier phase never completes and the bounded wait gives
 * up after value milliseconds (0.01-1000); the copies themselves complete, the kernel drains and
 * returns, and the call reports FSG_E_TIMEOUT.  FSG_FAULT_NONE restores normal operation. */
enum { FSG_FAULT_NONE = 0, FSG_FAULT_ALLOC_LIMIT = 1, FSG_FAULT_COPY_TIMEOUT = 2 };
int fsg_set_fault(fsg_ctx *ctx, int kind, double value);

/* ---- batched synthesis ---------------------------------------------------------------------
 * Many atmospheres (each a context with grid, atmosphere, continuum and mu set; mixed precision)
 * and one line list sorted by wavelength: per atmosphere the lines with centres in
 * [wstart - margin, wend + margin] [A] take the central pass and block refill.  margin = 0 is the
 * reference's own rule: a synthesis over [Wstart, Wend] reads the lines whose centres lie in that
 * range (ReadHDF, ioutils.f90:752-753; ReadAscMag, ioutils.f90:1496-1497), so each atmosphere's
 * result is the reference's run of its deck on the shared list; margin > 0 adds the lines just
 * outside, whose windows the reference's WaveIdx clamps to the grid's ends (opacity.f90:594-608).
 * Each atmosphere's records are grouped by window-width class; atmospheres are grouped by depth
 * count (buckets of 8).  Per group, persistent launches (wing pass over the narrow classes, wing pass
 * over the wide ones, core pass) take (atmosphere, tile) items from device work queues, each tile
 * adding its classes in turn; then the formal solver and flux run per atmosphere, plane-parallel or
 * spherical as each context's geometry says (the rays of a spherical one are built by
 * fsg_batch_create, so the contexts' geometry and angles must not change after it).  The sequence
 * has no host synchronisation; the
 * first fsg_batch_run tunes it (unless fsg_batch_set_tuning gave a choice), captures it as a CUDA
 * graph and replays it; later runs replay.  No counterpart in the reference, which synthesises
 * one atmosphere per run (fastspec.f90:192-449). */
typedef struct fsg_batch fsg_batch;
typedef struct {
    int32_t tile_pix;       /* wing-pass tile width of the wide classes (windows over 512
                             * wavelengths): 64 or 128; the narrower ones take 64 */
    int32_t wing_ctas, core_ctas;   /* CTAs of the persistent wing / core launches */
    double  ms_wing, ms_core;       /* their times in the tuning run [ms] */
} fsg_batch_tuning;
typedef struct {
    int32_t natm;
    int64_t nlines_candidate;       /* lines taken by the atmospheres (sum) */
    double  line_evals;             /* profile evaluations inside windows (sum) */
    double  ms_total;               /* device time of one graph replay [ms] */
    fsg_batch_tuning tuning;
    double  ms_prepare, ms_wing, ms_core, ms_solve;   /* its stages: central pass, class order, records
                                                       * and tile ranges; wing launches; core launches;
                                                       * formal solver and flux [ms] */
    double  core_evals;     /* the core pass's evaluations (table and continued fraction, s < 196) */
} fsg_batch_stats;
/* On failure *out stays NULL and fsg_batch_last_error(NULL) gives the reason. */
int  fsg_batch_create(fsg_ctx *const *atms, int natm, const fsg_lines *lines, double margin, fsg_batch **out);
int  fsg_batch_tune(fsg_batch *b, fsg_batch_tuning *result);
int  fsg_batch_set_tuning(fsg_batch *b, const fsg_batch_tuning *t);
int  fsg_batch_run(fsg_batch *b, fsg_batch_stats *stats);
/* Flux (line + continuum, continuum; [nwl] each) of atmosphere iatm after a run. */
int  fsg_batch_flux(fsg_batch *b, int iatm, double *sfl, double *sfc);
void *fsg_batch_stream(fsg_batch *b);
const char *fsg_batch_last_error(const fsg_batch *b);
void fsg_batch_destroy(fsg_batch *b);

#ifdef __cplusplus
}
#endif
#endif
