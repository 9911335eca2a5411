/*
 * fs_oracle.h -- CPU FP64 restatement of FastSpec's line-opacity -> formal-solver path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA product in
 * fastspec_b200/.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference arm may load it, and only as the checker or as the timed CPU baseline, never
 * as a code path of the product.
 *
 * Every routine restates the reference algorithm operation by operation (same operand order,
 * FP64, no FMA contraction: build with -ffp-contract=off) and cites the reference file:line
 * it follows.  Arrays use the reference's Fortran column-major layouts seen from C:
 *   LineOpac(Ntau,Nwl)        -> double[nwl][ntau]
 *   MagLineOpac(6,Ntau,Nwl)   -> double[nwl][ntau][6]
 *   SpL/SpC(Nmu,Nwl)          -> double[nwl][nmu]
 *   SpZ(Nmu,4,Nwl)            -> double[nwl][4][nmu]
 *   FractionPF(Maxspl,Ntau)   -> float[ntau][nspc]     (species fastest, FP32 as the EOS)
 * Line and wavelength indices on this interface are 1-based, as in the reference.
 */
#ifndef FS_ORACLE_H
#define FS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Voigt / Faraday-Voigt (voigt.f90) ------------------------------------------------ */
void   or_voigt_init(void);                                   /* VoigtInit  voigt.f90:42-72   */
void   or_fvoigt_init(void);                                  /* FVoigtInit voigt.f90:219-251 */
double or_hvoigt_exact(double a, double v);                   /* voigt.f90:158-187 */
void   or_wvoigt_exact(double a, double v, double *re, double *im); /* voigt.f90:356-393 */
double or_hvoigt(double a, double v);                         /* voigt.f90:76-110 */
void   or_fvoigt(double a, double v, double *vgt, double *fvgt);    /* voigt.f90:256-299 */
const float *or_voigt_table(void);    /* VgtTab(NVv+1,NVa+1), v fastest: 1002 x 402 */
const float *or_fvoigt_table(void);   /* FvTab(2,NVv+1,NVa+1): 2 x 1002 x 402 */

/* ---- Physical state of one atmosphere (host inputs of the hot path) ------------------- */
typedef struct {
    /* wavelength grid (synth.f90:56-74) */
    int     wmode;          /* 0: uniform in lambda, 1: uniform in ln lambda */
    double  wstart, wend, dstep;
    int     nwl;
    double *wave;           /* [nwl] offsets from wfirst (filled by or_grid_init) */
    double  wfirst, wlast, rstep;

    /* model atmosphere after the EOS (shared.f90:514-534) */
    int     ntau;
    const double *rhox, *T, *xne, *xna, *rho, *height;
    int     nspc;
    const float *fractionpf;   /* [ntau][nspc] */
    const float *xamass;       /* [nspc] */
    const float *potion;       /* [nspc] */
    const int   *ion;          /* [nspc] ionization stage (1 = neutral) */
    const float *frac_h1, *frac_he1, *frac_h2;   /* [ntau] number densities (Fraction) */
    int     spc_he1;           /* species index (0-based) of He I for Stark tables, -1 none */

    /* continuum opacity (ContopCalc output) */
    const double *contopac;    /* [nwl][ntau] */
    const double *contopac_std;/* [ntau] (Motype 1 only) */
    int     motype;

    /* He I Stark tables (hestark.f90), optional */
    int     nhe;
    const double *hegam, *heshf;   /* [nhe][ntau] */

    /* configuration (shared.f90:416-443) */
    double  vmicro, epsopac, vwfudge, h2brd, vwmol;
    int     molbrd;

    /* XlineInit state (opacity.f90:65-93) */
    double *x_nprtb, *x_gvwprt, *x_temp6, *x_temp3, *x_kbt, *x_kbet;
    double  x_vturb2;

    /* geometry (shared.f90:527, solver.f90:27-33): radius <= 0 is plane-parallel; otherwise
     * the rays of or_sphere_init for sph_nmu angles, arrays [nmu][2*ntau] (NtauMu, GrazMu,
     * MapMu 1-based, RhoxMu, MuLoc) */
    double  radius;
    int     sph_nmu;
    const int    *sph_ntau, *sph_graz, *sph_map;
    const double *sph_rhox, *sph_muloc;
} or_state;

/* SphereInit (solver.f90:45-120): rays of a spherical model for the nmu angles xmu; layer radii
 * radius + height[k].  Outputs [nmu] (ntau_mu, graz) and [nmu][2*ntau] (map 1-based, rhox_mu,
 * mu_loc).  Returns 0; -1 for an angle mu <= 0; -2 for a grazing ray tangent in the top layer. */
int or_sphere_init(int ntau, const double *rhox, const double *height, double radius, int nmu,
                   const double *xmu, int *ntau_mu, int *graz, int *map, double *rhox_mu, double *mu_loc);
/* LocPrfSph (solver.f90:182-216) + DeloScalar (solver.f90:220-261) over the rays of s */
void or_locprf_sph(const or_state *s, double *Ploc, const double *Xki, const double *Src);

/* ---- Line list (SoA; LineData records shared.f90:451-482) ----------------------------- */
typedef struct {
    long    n;
    const double *wl;                     /* air wavelength [A], FP64 */
    const float  *elo, *gf, *grad, *gqst, *gvdw;   /* FP32 as stored by the readers */
    const int    *spc;                    /* species index 0-based */
    const int    *kind;                   /* 0 LineTypeAtm, 1 LineTypeMol, 2 LineTypeMag */
    const int    *ismol;                  /* molecule flag (LineTypeMag: bit 1) */
    const int    *ihe;                    /* He I Stark table entry 1..nhe, 0 none */
    /* Zeeman components (LineTypeMag), CSR: line i has npi[i] pi and nsi[i] sigma comps */
    const int    *npi, *nsi;
    const long   *pi_off, *si_off;
    const float  *spl_pi, *str_pi, *spl_si, *str_si;
} or_lines;

typedef struct {
    long nlines_in, nlines_used, nwide, nweak, nsegments, nrefills;
    double line_evals;          /* Ntau * sum over retained non-wide lines of window length */
    double wide_evals;
} or_stats;

/* HeStarkInit (hestark.f90:332-370): per-depth Stark widths [rad/s] and shifts [A] of the 37
 * tabulated He I lines, [37][ntau], from T, Xne and the FP32 proton (H II) and He II densities. */
void or_hestark_init(int ntau, const double *T, const double *xne, const float *frac_hii,
                     const float *frac_heii, double *hegam, double *heshf);
/* HeMatchIdx (hestark.f90:376-389): table entry 1..37 within 1 A and 0.01 eV, else 0 */
int  or_he_match_idx(double wave_air, double elo);

int  or_grid_init(or_state *s);          /* allocates s->wave; returns nwl or <0 */
void or_xline_init(or_state *s);         /* allocates x_* */
void or_state_free(or_state *s);
int  or_waveidx(const or_state *s, double wavein);   /* opacity.f90:594-608 */
double or_air2vac(double lambda_air);                /* utils.f90:1020-1032 */

/* per-line prefactors, all depths: XlineSetup + XlineDepth (opacity.f90:96-293) */
void or_xline(const or_state *s, const or_lines *L, long iline0, double *lincop,
              double *linvvgt, double *linavgt);

/* LineopCalc (synth.f90:747-1095).  lineopac [nwl][ntau] is ACCUMULATED into.
 * list_type 0 atomic HDF, 1 molecular HDF, 2 ASCII/.z (LineTypeMag).
 * Per-line outputs (original order, may be NULL): flags, ileft, iright (1-based).
 * linstr (may be NULL): central depths of retained lines (LinStrCalc), needs nmu/xmu/wmu. */
int or_lineop_calc(const or_state *s, const or_lines *L, int list_type, long nlines_lim,
                   double *lineopac, int *flags_out, int *ileft_out, int *iright_out,
                   float *linstr_out, int nmu, const double *xmu, const double *wmu,
                   or_stats *st);
/* The same with the accumulation (wide lines and LineOpacity1) restricted to the wavelengths
 * [i0, i1] (1-based, inclusive) of the grid; windows, rejection and segments are those of the whole
 * grid.  The reference's accumulation is independent per wavelength (synth.f90:1075-1080), so the
 * rows [i0, i1] equal the whole-grid call's; the other rows are left untouched. */
int or_lineop_calc_range(const or_state *s, const or_lines *L, int list_type, long nlines_lim,
                         double *lineopac, int *flags_out, int *ileft_out, int *iright_out,
                         float *linstr_out, int nmu, const double *xmu, const double *wmu,
                         or_stats *st, int i0, int i1);

/* ---- the elemental routines on their own (checks of the library's kernel-level entry points) ---- */
typedef struct {           /* XlineCoef (opacity.f90:43-58); IxPF the 0-based species column */
    double WaveL, Hnux, Elo, Gf, Grad, Xmass, Cqst, Qdiv, Cvdw, AboPre, AboVbc, AboExp;
    int IxPF, MdQst, MdVdw, IxHe;
} or_xcoef;
/* XlineSetup (opacity.f90:96-235) of line i with the drivers' input flags (synth.f90:837-845) */
void or_xline_setup(const or_state *s, const or_lines *L, long i, int list_type, or_xcoef *xc);
/* XlineDepth (opacity.f90:239-293) at depth t (0-based) */
void or_xline_depth(const or_state *s, int t, const or_xcoef *xc, double *lincop, double *linvvgt,
                    double *linavgt);
/* LineOpacity1 (opacity.f90:297-346) over explicit block arrays: per line wlcent, flags, ileft,
 * iright; per block line lincop/linvvgt/linavgt [nblock][ntau]; lines l1..l2 (1-based), offset loff */
void or_lineopacity1(const or_state *s, const double *wlcent, const int *flags, const int *ileft,
                     const int *iright, const double *lincop, const double *linvvgt, const double *linavgt,
                     double Wl, int l1, int l2, int iwl, long loff, double *linop);
/* LineOpacity2 (opacity.f90:350-386) of one line (its wlcent, flag, ileft, iright) */
void or_lineopacity2(const or_state *s, double Wl, double wlcent, int flag, int ileft, int iright, int iwl,
                     const double *lincop, const double *linvvgt, const double *linavgt, double *linop);
/* MagLineOpacity1 (opacity.f90:391-464) over explicit block arrays and Zeeman components (CSR by
 * line, shifts in A): maglinop [ntau][6] */
void or_mag_lineopacity1(const or_state *s, const double *wlcent, const int *flags, const int *ileft,
                         const int *iright, const double *lincop, const double *linvvgt, const double *linavgt,
                         const int *npi, const int *nsi, const long *pi_off, const long *si_off,
                         const float *splpi, const float *strpi, const float *splsi, const float *strsi,
                         double Wl, int l1, int l2, int iwl, long loff, double *maglinop);
/* AnalyticWindow (opacity.f90:678-710) */
double or_analytic_window(const or_state *s, int flag, const double *lincop, const double *linvvgt,
                          const double *linavgt, const double *contopac);
/* StokesPrfPP (solver.f90:265-394): m6 [ntau][6], lop/cop/src [ntau], field per angle; stokes [4][nmu] */
void or_stokes_prf_pp(const or_state *s, const double *m6, const double *lop, const double *cop,
                      const double *src, int nmu, const double *xmu, const double *sphi2, const double *cphi2,
                      const double *cphi, const double *s2psi, const double *c2psi, double *stokes);

/* MagLineopCalc (synth.f90:1098-1455); maglineopac [nwl][ntau][6] accumulated. */
int or_mag_lineop_calc(const or_state *s, const or_lines *L, int bframe, const double *bfield,
                       long nlines_lim, double *maglineopac, int *flags_out, int *ileft_out,
                       int *iright_out, float *linstr_out, int nmu, const double *xmu,
                       const double *wmu, or_stats *st);

/* Solver (solver.f90) */
void or_taustep(const double *rhox, const double *xki, double xmu, int n, double *dtau);
void or_centder(const double *dxx, const double *y, int m, int n, double *yp);
void or_locprf_pp(double *ploc, const double *xmu, int nmu, const double *xki,
                  const double *src, const double *rhox, int ntau);
void or_solve4x4(const double *a /*[4][4] col-major*/, const double *b, double *x);

/* RadTranCalc (synth.f90:1825-1901): spl/spc [nwl][nmu]; spherical (s->radius > 0) along the rays
 * of s, whose angles must be xmu */
void or_radtran(const or_state *s, int nmu, const double *xmu, const double *lineopac,
                double *spl, double *spc);
/* MagRadTranCalc (synth.f90:1904-2111): spz [nwl][4][nmu], spc [nwl][nmu]; spherical when
 * s->radius > 0 (StokesPrfSph along the rays of s) */
void or_mag_radtran(const or_state *s, int nmu, const double *xmu, int bframe,
                    const double *bfield, const double *lineopac, const double *maglineopac,
                    double *spz, double *spc);

/* Quadrature (utils.f90:1273-1431) and disk integration (convol.f90:67-246, no broadening) */
int  or_mu_quadrature(int quad, int n, double *x, double *w, double *r, int setnodes);
void or_gauss_mu(int quad, int n, double *x, double *w);
/* DiskInteg with broadening (convol.f90:67-246) and ConvolGau (convol.f90:249-300).  dv: velocity
 * step of the grid [km/s] (2 Dstep / (Wfirst + Wlast) c for Wmode 0, Dstep for Wmode 1); gsig: the
 * Gaussian sigma in pixels of ConvolGau before the FWHM->sigma factor (Fwhm / step).  radii: the
 * nmu + 1 projected annulus radii of MuQuadrature.  spl/spc [nwl][nmu] in, sfl/sfc [nwl] out. */
void or_disk_integ_conv(int nmu, int nwl, const double *xmu, const double *wmu, const double *radii, double dv,
                        double vsini, double vmacro, double gsig, const double *spl, const double *spc,
                        double *sfl, double *sfc);
/* ConvolGau of one spectrum in place (convol.f90:249-300); sigma_pix = Fwhm / step. */
void or_convol_gau(int nw, double *S, double sigma_pix);
void or_disk_integ(int nmu, int nwl, const double *wmu, const double *spl, const double *spc,
                   double *sfl, double *sfc);

/* ZeemanPattern (utils.f90:901-1004).  Outputs must hold 2*Jup+1 entries each. */
void or_zeeman_pattern(float jlo, float jup, float glo, float gup, int *npi, float *spi,
                       float *rpi, int *nsig, float *ssig, float *rsig);

/* ZeemanPattern sigma mirroring of the .z reader (ioutils.f90:1393-1410) is done by callers. */

#ifdef __cplusplus
}
#endif
#endif
