/*
 * fs_oracle.c -- CPU FP64 restatement of FastSpec's line-opacity -> formal-solver path.
 *
 * TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline); see fs_oracle.h.
 *
 * Build: gcc -O2 -fopenmp -ffp-contract=off -fPIC -shared (the reference is gfortran -O3 on
 * x86-64 without -march, i.e. SSE2 scalar arithmetic with no fused multiply-add; every
 * expression below keeps the reference's left-to-right operand order so the FP64 results
 * match it to the last bit wherever the same libm is used).
 *
 * Complex arithmetic follows gfortran's -fcx-fortran-rules expansion: naive multiplication
 * and Smith's range-reduced division (GCC expand_complex_div_wide), complex EXP via cexp.
 */
#include "fs_oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- constants (shared.f90:20-33) ------------------------------------------------------ */
#define C_PI      3.141592653589793115997963468544185161590576171875
static const double Vc = 299792.458;
static const double Hc = 6.62607015e-27;
static const double Kbolt = 1.380649e-16;
static const double ev2Ang = 8065.544005e-8;
static const double A0 = 5.29177210903e-11;
static const double M0 = 1.66053906660e-27;
static const double Ce = 4.803204712e-10;
static const double Me = 9.1093837139e-28;
static const double Mh = 1.673532499e-24;
static const double Hie = 13.598434005;
static const double Kz = 4.668644778e-13;

static double erg2ev(void) { return 1e-7 / 1.602176634e-19; }

/* opacity.f90:35-39 */
static double XlnC(void)    { return Vc * 1e13; }
static double XlnC4Pi(void) { return 4.0 * XlnC() * C_PI; }
static double XlnZ(void)    { return sqrt(C_PI) * (Ce * Ce) / (Me * (Vc * Vc)) * 1e-18; }
static double XlnKM0(void)  { return Kbolt * 1e-7 / M0; }
static double XlnDop(void)  { return 2.0 * Kbolt / (M0 * 1e3) * 1e16; }

/* ---- Voigt table (voigt.f90:15-189) ---------------------------------------------------- */
#define NVV 1001
#define NVA 401
#define NV1 (NVV + 1)
#define NA1 (NVA + 1)
static const double VgtVmax = 8.0, VgtAmax = 8.0;
static const double SqrtPiInv = 0.56418958354775628695;

static float  VgtTab[NA1 * NV1];          /* VgtTab(iv,ia) -> [ia-1][iv-1] */
static double VgtANode[NA1], VgtAIDa[NA1];
static double VgtIDv, VgtIDt, VgtA1, VgtIA1;
static int    VgtReady = 0;
static float  FvTab[NA1 * NV1 * 2];       /* FvTab(c,iv,ia) -> [ia-1][iv-1][c-1] */
static double FvANode[NA1], FvAIDa[NA1];
static double FvIDv, FvIDt, FvA1, FvIA1;
static int    FvReady = 0;

/* complex helpers with gfortran's expansion */
typedef struct { double re, im; } cplx;
static inline cplx cmul(cplx a, cplx b) {
    cplx r; double t1 = a.re * b.re, t2 = a.im * b.im, t3 = a.re * b.im, t4 = a.im * b.re;
    r.re = t1 - t2; r.im = t3 + t4; return r;
}
static inline cplx cdiv(cplx a, cplx b) {     /* GCC expand_complex_div_wide */
    cplx r; double ratio, div, tr, ti;
    if (fabs(b.re) < fabs(b.im)) {
        ratio = b.re / b.im; div = (b.re * ratio) + b.im;
        tr = (a.re * ratio) + a.im; ti = (a.im * ratio) - a.re;
    } else {
        ratio = b.im / b.re; div = (b.im * ratio) + b.re;
        tr = (a.im * ratio) + a.re; ti = a.im - (a.re * ratio);
    }
    r.re = tr / div; r.im = ti / div; return r;
}
static inline cplx cexp_(cplx z) {
    double complex w = cexp(z.re + I * z.im); cplx r = { creal(w), cimag(w) }; return r;
}

/* Chiarella-Reichel sum shared by HVoigtExact/WVoigtExact (voigt.f90:171-185, 376-390) */
static cplx cr_sum(double a, double av, double pi_) {
    const double HH = 0.5; const int NN = 16;
    cplx z = { av, a }, z2 = cmul(z, z), s, one = { 1.0, 0.0 };
    s = cdiv(one, z);
    for (int n = 1; n <= NN; n++) {
        double nh = (double)n * HH;
        double e = exp(-nh * nh);
        cplx num = { (2.0 * z.re) * e, (2.0 * z.im) * e };
        cplx den = { z2.re - nh * nh, z2.im };
        cplx q = cdiv(num, den);
        s.re = s.re + q.re; s.im = s.im + q.im;
    }
    {   /* CMPLX(0, HH/pi) * s : ONLY_IMAG x VARYING expansion */
        double c = HH / pi_; cplx t; t.re = -(c * s.im); t.im = c * s.re; s = t;
    }
    if (a < 6.0) {
        double p = 2.0 * pi_ * a / HH;
        double th = 2.0 * pi_ * (2.0 * av - round(2.0 * av));
        double sn = sin(0.5 * th);
        double redd = -(2.0 * exp(0.5 * p) * sinh(0.5 * p)) + exp(p) * 2.0 * (sn * sn);
        double imdd = exp(p) * sin(th);
        cplx ex = cexp_((cplx){ a * a - av * av, -2.0 * a * av });
        cplx num = { 2.0 * ex.re, 2.0 * ex.im };
        cplx q = cdiv(num, (cplx){ redd, imdd });
        s.re = s.re + q.re; s.im = s.im + q.im;
    }
    return s;
}

/* voigt.f90:158-187 */
double or_hvoigt_exact(double a, double v) {
    double av = fabs(v);
    if (a <= 0.0) return exp(-fmin(av * av, 700.0));
    return cr_sum(a, av, C_PI).re;
}

/* voigt.f90:356-393 */
void or_wvoigt_exact(double a, double v, double *re, double *im) {
    double av = fabs(v);
    if (a <= 0.0) {
        int m = 2 * (int)lround(2.0 * av);
        double x0 = av - 0.25 * (double)m, p = 0.0;
        for (int n = -31; n <= 31; n += 2) {
            double t = x0 - 0.25 * (double)n;
            p = p + exp(-(t * t)) / (double)(m + n);
        }
        *re = exp(-fmin(av * av, 700.0)); *im = (2.0 / C_PI) * p;
        if (v < 0.0) *im = -*im;
        return;
    }
    cplx s = cr_sum(a, av, C_PI);
    if (v < 0.0) s.im = -s.im;
    *re = s.re; *im = s.im;
}

/* voigt.f90:42-72 */
void or_voigt_init(void) {
    if (VgtReady) return;
    double dv = VgtVmax / (double)(NVV - 1);
    double dt = sqrt(VgtAmax) / (double)(NVA - 1);
    VgtIDv = 1.0 / dv; VgtIDt = 1.0 / dt;
    for (int ia = 1; ia <= NVA + 1; ia++) { double t = (double)(ia - 1) * dt; VgtANode[ia - 1] = t * t; }
    for (int ia = 1; ia <= NVA; ia++) VgtAIDa[ia - 1] = 1.0 / (VgtANode[ia] - VgtANode[ia - 1]);
    VgtAIDa[NVA] = 0.0;
    VgtA1 = VgtANode[1]; VgtIA1 = VgtAIDa[0];
    #pragma omp parallel for schedule(static)
    for (int ia = 1; ia <= NVA + 1; ia++) {
        double aa = VgtANode[ia - 1];
        for (int iv = 1; iv <= NVV + 1; iv++) {
            double vv = (double)(iv - 1) * dv;
            VgtTab[(ia - 1) * NV1 + (iv - 1)] = (float)or_hvoigt_exact(aa, vv);
        }
    }
    VgtReady = 1;
}

/* voigt.f90:219-251 */
void or_fvoigt_init(void) {
    if (FvReady) return;
    double dv = 8.0 / (double)(NVV - 1);
    double dt = sqrt(8.0) / (double)(NVA - 1);
    FvIDv = 1.0 / dv; FvIDt = 1.0 / dt;
    for (int ia = 1; ia <= NVA + 1; ia++) { double t = (double)(ia - 1) * dt; FvANode[ia - 1] = t * t; }
    for (int ia = 1; ia <= NVA; ia++) FvAIDa[ia - 1] = 1.0 / (FvANode[ia] - FvANode[ia - 1]);
    FvAIDa[NVA] = 0.0;
    FvA1 = FvANode[1]; FvIA1 = FvAIDa[0];
    #pragma omp parallel for schedule(static)
    for (int ia = 1; ia <= NVA + 1; ia++) {
        for (int iv = 1; iv <= NVV + 1; iv++) {
            double vv = (double)(iv - 1) * dv, re, im;
            or_wvoigt_exact(FvANode[ia - 1], vv, &re, &im);
            FvTab[((ia - 1) * NV1 + (iv - 1)) * 2 + 0] = (float)re;
            FvTab[((ia - 1) * NV1 + (iv - 1)) * 2 + 1] = (float)im;
        }
    }
    FvReady = 1;
}

const float *or_voigt_table(void)  { or_voigt_init(); return VgtTab; }
const float *or_fvoigt_table(void) { or_fvoigt_init(); return FvTab; }

#define VT(iv1, ia1) VgtTab[((ia1) - 1) * NV1 + ((iv1) - 1)]      /* 1-based like Fortran */
#define FT(c, iv1, ia1) FvTab[(((ia1) - 1) * NV1 + ((iv1) - 1)) * 2 + ((c) - 1)]

/* asymptotic branch of HVoigt / HVoigtLine (voigt.f90:97-108) */
static inline double hv_asym(double A, double av) {
    double a2 = A * A, v2 = av * av, s = v2 + a2;
    if (s >= 196.0) return SqrtPiInv * A * (s + 0.5) / (s * s - v2 + a2 + 0.25);
    double p = v2 - a2 - 1.5, q = 2.0 * av * A;
    double dr = av * p - A * q, di = av * q + A * p;
    return SqrtPiInv * ((p + 0.5) * di - q * dr) / (dr * dr + di * di);
}

/* voigt.f90:76-110 */
double or_hvoigt(double A, double V) {
    if (!VgtReady) or_voigt_init();
    double av = fabs(V);
    if (A < VgtAmax && av < VgtVmax) {
        double fv = av * VgtIDv; int iv = (int)fv; double tv = fv - (double)iv, ua; int ia;
        if (A < VgtA1) { ia = 1; ua = A * VgtIA1; }
        else { ia = (int)(sqrt(A) * VgtIDt) + 1; ua = (A - VgtANode[ia - 1]) * VgtAIDa[ia - 1]; }
        double c0 = (double)VT(iv + 1, ia) + tv * (double)(VT(iv + 2, ia) - VT(iv + 1, ia));
        double c1 = (double)VT(iv + 1, ia + 1) + tv * (double)(VT(iv + 2, ia + 1) - VT(iv + 1, ia + 1));
        return c0 + ua * (c1 - c0);
    }
    return hv_asym(A, av);
}

/* VoigtLineInit / HVoigtLine (voigt.f90:113-154) */
typedef struct { double A, UA; int IA; } vline;
static inline vline vline_init(double A) {
    vline L; L.A = A;
    if (A < VgtAmax) { L.IA = (int)(sqrt(A) * VgtIDt) + 1; L.UA = (A - VgtANode[L.IA - 1]) * VgtAIDa[L.IA - 1]; }
    else { L.IA = 0; L.UA = 0.0; }
    return L;
}
static inline double hvoigt_line(vline L, double V) {
    double av = fabs(V);
    if (L.IA > 0 && av < VgtVmax) {
        double fv = av * VgtIDv; int iv = (int)fv; double tv = fv - (double)iv;
        double c0 = (double)VT(iv + 1, L.IA) + tv * (double)(VT(iv + 2, L.IA) - VT(iv + 1, L.IA));
        double c1 = (double)VT(iv + 1, L.IA + 1) + tv * (double)(VT(iv + 2, L.IA + 1) - VT(iv + 1, L.IA + 1));
        return c0 + L.UA * (c1 - c0);
    }
    return hv_asym(L.A, av);
}

/* FVoigt asymptotic (voigt.f90:280-297) */
static inline void fv_asym(double A, double av, double *vgt, double *fvgt) {
    double a2 = A * A, v2 = av * av, s = v2 + a2, w;
    if (s >= 196.0) {
        w = SqrtPiInv / (s * s - v2 + a2 + 0.25);
        *vgt = w * A * (s + 0.5); *fvgt = w * av * (s - 0.5);
    } else {
        double p = v2 - a2 - 1.5, q = 2.0 * av * A;
        double dr = av * p - A * q, di = av * q + A * p;
        w = SqrtPiInv / (dr * dr + di * di);
        *vgt = w * ((p + 0.5) * di - q * dr); *fvgt = w * ((p + 0.5) * dr + q * di);
    }
}

/* voigt.f90:256-299 */
void or_fvoigt(double A, double V, double *vgt, double *fvgt) {
    if (!FvReady) or_fvoigt_init();
    double av = fabs(V);
    if (A < 8.0 && av < 8.0) {
        double fv = av * FvIDv; int iv = (int)fv; double tv = fv - (double)iv, ua; int ia;
        if (A < FvA1) { ia = 1; ua = A * FvIA1; }
        else { ia = (int)(sqrt(A) * FvIDt) + 1; ua = (A - FvANode[ia - 1]) * FvAIDa[ia - 1]; }
        double h0 = (double)FT(1, iv + 1, ia) + tv * (double)(FT(1, iv + 2, ia) - FT(1, iv + 1, ia));
        double h1 = (double)FT(1, iv + 1, ia + 1) + tv * (double)(FT(1, iv + 2, ia + 1) - FT(1, iv + 1, ia + 1));
        double l0 = (double)FT(2, iv + 1, ia) + tv * (double)(FT(2, iv + 2, ia) - FT(2, iv + 1, ia));
        double l1 = (double)FT(2, iv + 1, ia + 1) + tv * (double)(FT(2, iv + 2, ia + 1) - FT(2, iv + 1, ia + 1));
        *vgt = h0 + ua * (h1 - h0); *fvgt = l0 + ua * (l1 - l0);
    } else fv_asym(A, av, vgt, fvgt);
    *fvgt = copysign(fabs(*fvgt), V);
}

/* FvLineInit / FVoigtLine (voigt.f90:302-352) */
static inline vline fvline_init(double A) {
    vline L; L.A = A;
    if (A < 8.0) { L.IA = (int)(sqrt(A) * FvIDt) + 1; L.UA = (A - FvANode[L.IA - 1]) * FvAIDa[L.IA - 1]; }
    else { L.IA = 0; L.UA = 0.0; }
    return L;
}
static inline void fvoigt_line(vline L, double V, double *vgt, double *fvgt) {
    double av = fabs(V);
    if (L.IA > 0 && av < 8.0) {
        double fv = av * FvIDv; int iv = (int)fv; double tv = fv - (double)iv;
        double h0 = (double)FT(1, iv + 1, L.IA) + tv * (double)(FT(1, iv + 2, L.IA) - FT(1, iv + 1, L.IA));
        double h1 = (double)FT(1, iv + 1, L.IA + 1) + tv * (double)(FT(1, iv + 2, L.IA + 1) - FT(1, iv + 1, L.IA + 1));
        double l0 = (double)FT(2, iv + 1, L.IA) + tv * (double)(FT(2, iv + 2, L.IA) - FT(2, iv + 1, L.IA));
        double l1 = (double)FT(2, iv + 1, L.IA + 1) + tv * (double)(FT(2, iv + 2, L.IA + 1) - FT(2, iv + 1, L.IA + 1));
        *vgt = h0 + L.UA * (h1 - h0); *fvgt = l0 + L.UA * (l1 - l0);
    } else fv_asym(L.A, av, vgt, fvgt);
    *fvgt = copysign(fabs(*fvgt), V);
}

/* ---- grid, indices, utilities ---------------------------------------------------------- */

/* Init wavelength grid (synth.f90:56-74) */
int or_grid_init(or_state *s) {
    const double EpsWl = 1e-12;
    if (s->wmode == 0) {
        s->nwl = (int)floor((s->wend - s->wstart) / s->dstep + EpsWl) + 1;
        if (s->nwl < 2) return -1;
        s->wave = (double *)malloc(sizeof(double) * s->nwl);
        for (int i = 1; i <= s->nwl; i++) s->wave[i - 1] = (double)(i - 1) * s->dstep;
        s->wfirst = s->wstart; s->wlast = s->wave[s->nwl - 1] + s->wfirst;
    } else {
        s->rstep = s->dstep / Vc;
        s->nwl = (int)floor(log(s->wend / s->wstart) / s->rstep + EpsWl) + 1;
        if (s->nwl < 2) return -1;
        s->wave = (double *)malloc(sizeof(double) * s->nwl);
        for (int i = 1; i <= s->nwl; i++) s->wave[i - 1] = s->wstart * exp((double)(i - 1) * s->rstep);
        s->wfirst = s->wstart; s->wlast = s->wave[s->nwl - 1];
        for (int i = 0; i < s->nwl; i++) s->wave[i] = s->wave[i] - s->wstart;
    }
    return s->nwl;
}

/* WaveIdx (opacity.f90:594-608) */
int or_waveidx(const or_state *s, double wavein) {
    if (s->wmode == 0) {
        double X = fmin(fmax(wavein / s->dstep, 0.0), (double)(s->nwl - 2));
        return (int)X + 1;
    }
    double X = 1.0 + log(fmax((wavein / s->wstart) + 1.0, DBL_MIN)) / s->rstep;
    return (int)fmin(fmax(X, 1.0), (double)(s->nwl - 1));
}

/* Air2Vac (utils.f90:1020-1032) */
double or_air2vac(double la) {
    double S = 1e4 / la, S2 = S * S;
    double N = 1.0 + 8.336624212083e-5 + 2.408926869968e-2 / (1.301065924522e2 - S2) +
               1.599740894897e-4 / (3.892568793293e1 - S2);
    return (la > 1999.352) ? la * N : la;
}

/* ---- tabulated He I Stark broadening (hestark.f90) --------------------------------------
 * The published width/shift tables are data shared with the library (one header); the
 * interpolation and assembly below are this file's own restatement. */
#include "../fastspec_b200/csrc/fsg_hestark_tables.h"

/* LagWt3 (hestark.f90:394-415): three-point Lagrange weights on knots t[0..n-1] at x; the
 * returned j is the reference's 1-based knot index (value = w0 F(j) + w1 F(j-1) + w2 F(j-2)) */
static int he_lagwt3(const double *t, int n, double x, double *w0, double *w1, double *w2) {
    int j = n;
    for (int it = 3; it <= n; it++)
        if (t[it - 1] > x) { j = it; break; }
    double tj = t[j - 1], tj1 = t[j - 2], tj2 = t[j - 3];
    double Tj = (tj - tj1) * (tj - tj2) * (tj1 - tj2);
    *w0 = (x - tj2) * (x - tj1) * (tj1 - tj2) / Tj;
    *w1 = (x - tj2) * (tj - x) * (tj - tj2) / Tj;
    *w2 = (x - tj1) * (x - tj) * (tj - tj1) / Tj;
    return j;
}

/* HeStarkInit (hestark.f90:332-370); HeGamCnv = 1.884e3 (hestark.f90:39) */
void or_hestark_init(int ntau, const double *T, const double *xne, const float *frac_hii,
                     const float *frac_heii, double *hegam, double *heshf) {
    for (int t = 0; t < ntau; t++) {
        double Tlg = log10(T[t]), Xne = xne[t], Xnp = (double)frac_hii[t], Xnhe2 = (double)frac_heii[t];
        for (int k = 0; k < FSG_HE_NTAB; k++) {
            const fsg_he_line *e = &FSG_HE_TAB[k];
            int ds90 = k < FSG_HE_NDS90;
            double w0, w1, w2;
            int j = he_lagwt3(ds90 ? FSG_HE_LOGT90 : FSG_HE_LOGT84, e->nknot, Tlg, &w0, &w1, &w2) - 1;
#define LAG(a) (w0 * (a)[j] + w1 * (a)[j - 1] + w2 * (a)[j - 2])
            double g, sh;
            if (ds90) {
                g = (LAG(e->w[0]) * Xne + LAG(e->w[1]) * Xnp + LAG(e->w[2]) * Xnhe2) * 1.884e3 / (e->wlc * e->wlc);
                sh = (LAG(e->s[0]) * Xne + LAG(e->s[1]) * Xnp + LAG(e->s[2]) * Xnhe2) * 1e-16;
            } else {
                g = (LAG(e->w[0]) * Xne + LAG(e->w[1]) * Xnp) * 1.884e3 / (e->wlc * e->wlc);
                sh = (LAG(e->s[0]) * Xne + LAG(e->s[1]) * Xnp) * 1e-16;
            }
#undef LAG
            hegam[(size_t)k * ntau + t] = g > 0.0 ? g : 0.0;   /* MAX(Gam, 0d0) */
            heshf[(size_t)k * ntau + t] = sh;
        }
    }
}

/* HeMatchIdx (hestark.f90:376-389): HeMatchTol 1 A, HeEloTol 0.01 eV (hestark.f90:31, 36) */
int or_he_match_idx(double wave_air, double elo) {
    for (int k = 0; k < FSG_HE_NTAB; k++)
        if (fabs(wave_air - FSG_HE_TAB[k].wlc) <= 1.0 && fabs(elo - FSG_HE_TAB[k].elo) <= 0.01) return k + 1;
    return 0;
}

/* XlineInit (opacity.f90:65-93) */
void or_xline_init(or_state *s) {
    int nt = s->ntau;
    s->x_nprtb = (double *)malloc(sizeof(double) * nt);  s->x_gvwprt = (double *)malloc(sizeof(double) * nt);
    s->x_temp6 = (double *)malloc(sizeof(double) * nt);  s->x_temp3 = (double *)malloc(sizeof(double) * nt);
    s->x_kbt = (double *)malloc(sizeof(double) * nt);    s->x_kbet = (double *)malloc(sizeof(double) * nt);
    double c = XlnC();
    s->x_vturb2 = 1e26 / c / c * (s->vmicro * s->vmicro);
    for (int t = 0; t < nt; t++) {
        double Temp = s->T[t], Xne = s->xne[t];
        double Vh = sqrt(2.0 * Kbolt * Temp / Mh);
        s->x_nprtb[t] = (double)s->frac_h1[t] + 0.412265 * (double)s->frac_he1[t];
        if (s->h2brd > 0.0) s->x_nprtb[t] = s->x_nprtb[t] + s->h2brd * 0.874307 * (double)s->frac_h2[t];
        s->x_gvwprt[t] = 17.0 * pow(Vh, 0.6) * s->x_nprtb[t];
        s->x_temp6[t] = pow(Temp / 1e4, 1.0 / 6.0) * Xne;
        s->x_temp3[t] = pow(Temp / 1e4, 0.3) * s->x_nprtb[t];
        s->x_kbt[t] = Kbolt * Temp;
        s->x_kbet[t] = Kbolt * erg2ev() * Temp;
    }
}

void or_state_free(or_state *s) {
    free(s->wave); free(s->x_nprtb); free(s->x_gvwprt); free(s->x_temp6); free(s->x_temp3);
    free(s->x_kbt); free(s->x_kbet);
    s->wave = s->x_nprtb = s->x_gvwprt = s->x_temp6 = s->x_temp3 = s->x_kbt = s->x_kbet = NULL;
}

/* XlineCoef (opacity.f90:43-58) */
typedef struct {
    double WaveL, Hnux, Elo, Gf, Grad, Xmass, Cqst, Qdiv, Cvdw, AboPre, AboVbc, AboExp;
    int IxPF, MdQst, MdVdw, IxHe;
} xcoef;

/* XlineSetup (opacity.f90:96-235).  flag: the line's joint flag (bit 1 molecule, bit 2 ABO). */
static void xline_setup(const or_state *s, const or_lines *L, long i, double wlc, int flag,
                        xcoef *XC) {
    double WaveL = wlc + s->wfirst;
    double Elo = (double)L->elo[i];
    XC->WaveL = WaveL; XC->Elo = Elo; XC->Gf = (double)L->gf[i];
    double GradL = (double)L->grad[i], GqstL, GvdwL; int IsMol;
    int ispc = L->spc[i]; int IonL = s->ion[ispc]; XC->IxPF = ispc;
    switch (L->kind[i]) {
        case 0: GqstL = (double)L->gqst[i]; GvdwL = (double)L->gvdw[i]; IsMol = 0; break;
        case 1: GqstL = 0.0; GvdwL = 0.0; IsMol = 1; break;
        default: GqstL = (double)L->gqst[i]; GvdwL = (double)L->gvdw[i]; IsMol = (flag >> 1) & 1; break;
    }
    double c = XlnC();
    XC->Hnux = c * Hc / WaveL;
    XC->Xmass = XlnDop() / c / c / (double)s->xamass[ispc];
    XC->Grad = (GradL > 0.0) ? GradL : 0.22233e16 / (WaveL * WaveL);
    XC->Cqst = 0.0; XC->Qdiv = 1.0; XC->Cvdw = 0.0; XC->AboPre = 0.0; XC->AboVbc = 0.0; XC->AboExp = 0.0;
    XC->IxHe = 0;
    if (IsMol && !s->molbrd) { XC->MdQst = 9; XC->MdVdw = 9; }
    else {
        double Wavevac = or_air2vac(WaveL);
        double Eup = Elo + 1.0 / (Wavevac * ev2Ang);
        double pot = (double)s->potion[ispc];
        double t1 = (double)(IonL * IonL) * Hie / (pot - Eup);
        double t2 = (double)(IonL * IonL) * Hie / (pot - Elo);
        double Enu4 = t1 * t1, Enl4 = t2 * t2;
        /* opacity.f90:176: a He I line matching a table entry (HeMatchIdx); an explicit entry
         * list L->ihe overrides the match */
        if (ispc == s->spc_he1)
            XC->IxHe = L->ihe ? L->ihe[i] : (s->nhe == FSG_HE_NTAB ? or_he_match_idx(WaveL, Elo) : 0);
        if (XC->IxHe > 0) XC->MdQst = 3;
        else if (GqstL > 0.0) { XC->MdQst = 0; XC->Cqst = GqstL; }
        else if (IsMol) XC->MdQst = 9;
        else if (IonL == 1) { XC->MdQst = 1; XC->Cqst = 2.26e-07 * Enu4; }
        else { XC->MdQst = 2; XC->Cqst = 5.42e-07 * Enu4; XC->Qdiv = ((double)IonL + 1.0) * ((double)IonL + 1.0); }
        if ((flag >> 2) & 1) {
            XC->MdVdw = 2;
            double Sigma = A0 * A0 * (double)(int)GvdwL;
            double Alpha = GvdwL - (double)(int)GvdwL;
            double X = 2.0 - Alpha * 0.5, Gx = X - 1.0;
            double GammaF = 1.0 + (-0.5748646 + (0.9512363 + (-0.6998588 +
                            (0.4245549 - 0.1010678 * Gx) * Gx) * Gx) * Gx) * Gx;
            XC->AboPre = 2e6 * (pow(4.0 / C_PI, Alpha * 0.5) * GammaF * 1e4 * Sigma);
            XC->AboVbc = 1.0 / 1.00794 + 1.0 / (double)s->xamass[ispc];
            XC->AboExp = 1.0 - Alpha;
        } else if (GvdwL > 0.0) { XC->MdVdw = 0; XC->Cvdw = GvdwL; }
        else if (IsMol) XC->MdVdw = 9;
        else {
            XC->MdVdw = 1;
            double Cw = 1.61e-33 * fabs(Enu4 - Enl4) / (double)(IonL * IonL);
            XC->Cvdw = pow(Cw, 0.4);
        }
    }
    if (IsMol && s->vwmol > 0.0) { XC->MdVdw = 0; XC->Cvdw = s->vwmol; }
}

/* XlineDepth (opacity.f90:239-293); itau 0-based */
static inline void xline_depth(const or_state *s, int t, const xcoef *XC, double *cop,
                               double *vv, double *av) {
    double Xstim = 1.0 - exp(-XC->Hnux / s->x_kbt[t]);
    double Efract = exp(-XC->Elo / s->x_kbet[t]);
    double Dopl = sqrt(s->T[t] * XC->Xmass + s->x_vturb2);
    double Dldopl = XC->WaveL * Dopl, Dndopl = Dopl / XC->WaveL;
    double Gqst, Gvdw;
    switch (XC->MdQst) {
        case 0: Gqst = XC->Cqst * s->x_temp6[t]; break;
        case 1: Gqst = XC->Cqst * s->xne[t]; break;
        case 2: Gqst = XC->Cqst * s->xne[t] / XC->Qdiv; break;
        case 3: Gqst = s->hegam[(XC->IxHe - 1) * s->ntau + t]; break;
        default: Gqst = 0.0;
    }
    switch (XC->MdVdw) {
        case 0: Gvdw = XC->Cvdw * s->x_temp3[t]; break;
        case 1: Gvdw = s->vwfudge * s->x_gvwprt[t] * XC->Cvdw; break;
        case 2: {
            double Vbar = sqrt(8.0 * XlnKM0() * s->T[t] / C_PI * XC->AboVbc);
            Gvdw = XC->AboPre * pow(Vbar / 1e4, XC->AboExp) * s->x_nprtb[t];
        } break;
        default: Gvdw = 0.0;
    }
    double Gamtot = XC->Grad + Gqst + Gvdw;
    *av = Gamtot / (Dndopl * XlnC4Pi());
    *vv = 1.0 / Dldopl;
    double c = XlnZ() * Efract * XC->Gf * Xstim / (s->rho[t] * Dndopl);
    *cop = c * (double)s->fractionpf[(size_t)t * s->nspc + XC->IxPF];
}

/* joint flag bits set by the drivers before XlineSetup (synth.f90:837-845, 1185-1188) */
static int input_flags(const or_lines *L, long i, int list_type) {
    int f = 0;
    if (list_type == 0) { if (L->gvdw[i] > 10.0f) f |= 4; }
    else if (list_type == 2) { if (L->ismol && L->ismol[i]) f |= 2; if (L->gvdw[i] > 10.0f) f |= 4; }
    return f;
}

void or_xline(const or_state *s, const or_lines *L, long i0, double *lincop, double *linvvgt,
              double *linavgt) {
    double wlc = L->wl[i0] - s->wfirst;
    xcoef XC;
    int kind = L->kind[i0];
    int lt = (kind == 0) ? 0 : (kind == 1 ? 1 : 2);
    xline_setup(s, L, i0, wlc, input_flags(L, i0, lt), &XC);
    for (int t = 0; t < s->ntau; t++) xline_depth(s, t, &XC, &lincop[t], &linvvgt[t], &linavgt[t]);
}

/* ---- solver (solver.f90) ---------------------------------------------------------------- */

/* TauStep (solver.f90:591-615); dtau[n-1] untouched */
void or_taustep(const double *Rhox, const double *Xki, double Xmu, int N, double *Dtau) {
    double Dx1 = (Rhox[1] - Rhox[0]) / Xmu;
    double Yp = (Xki[1] - Xki[0]) / Dx1;
    Dtau[0] = Dx1 * (Xki[1] + 2.0 * Xki[0] + Dx1 / 2.0 * Yp) / 3.0;
    for (int k = 2; k <= N - 1; k++) {
        double Dx = (Rhox[k - 1] - Rhox[k - 2]) / Xmu;
        Dx1 = (Rhox[k] - Rhox[k - 1]) / Xmu;
        double Der = (Xki[k - 1] - Xki[k - 2]) / Dx;
        double Der1 = (Xki[k] - Xki[k - 1]) / Dx1;
        if (Der * Der1 > 0.0) {
            double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0;
            Yp = (Der / (Lambda * Der1 + (1.0 - Lambda) * Der)) * Der1;
        } else Yp = 0.0;
        Dtau[k - 1] = Dx1 * (Xki[k] + 2.0 * Xki[k - 1] + Dx1 / 2.0 * Yp) / 3.0;
    }
}

/* CentDer (solver.f90:618-647): Y(M,N) column-major -> y[k*m + j] */
void or_centder(const double *Dxx, const double *Y, int M, int N, double *Yp) {
    for (int k = 2; k <= N - 1; k++) {
        double Dx = Dxx[k - 2], Dx1 = Dxx[k - 1];
        double InvDx = 1.0 / Dx, InvDx1 = 1.0 / Dx1;
        double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0, Lambda1 = 1.0 - Lambda;
        for (int j = 0; j < M; j++) {
            double Der = (Y[(k - 1) * M + j] - Y[(k - 2) * M + j]) * InvDx;
            double Der1 = (Y[k * M + j] - Y[(k - 1) * M + j]) * InvDx1;
            Yp[(k - 1) * M + j] = (Der * Der1 > 0.0) ? (Der / (Lambda * Der1 + Lambda1 * Der)) * Der1 : 0.0;
        }
    }
    for (int j = 0; j < M; j++) {
        Yp[j] = (Y[M + j] - Y[j]) / Dxx[0];
        Yp[(N - 1) * M + j] = (Y[(N - 1) * M + j] - Y[(N - 2) * M + j]) / Dxx[N - 2];
    }
}

/* Bezier coefficients of the DELO step (solver.f90:155-169) */
static inline void delo_coef(double Dtau, double *Eps, double *Alpha, double *Beta, double *Gamma) {
    double Dtau2 = Dtau * Dtau, Idtau2 = 1.0 / Dtau2;
    if (Dtau < 5e-3) {
        *Eps = 1.0 - Dtau + 0.5 * Dtau2 - Dtau2 * Dtau / 6.0 + Dtau2 * Dtau2 / 24.0;
        *Alpha = Dtau / 3.0 - Dtau2 / 12.0 + Dtau2 * Dtau / 60.0;
        *Beta = Dtau / 3.0 - Dtau2 * 0.25 + Dtau2 * Dtau * 0.1;
        *Gamma = Dtau / 3.0 - Dtau2 / 6.0 + Dtau2 * Dtau * 0.05;
    } else {
        *Eps = (Dtau < 100.0) ? exp(-Dtau) : 0.0;
        *Alpha = (Dtau2 - 2.0 * Dtau + 2.0 - 2.0 * *Eps) * Idtau2;
        *Beta = (2.0 - (2.0 + 2.0 * Dtau + Dtau2) * *Eps) * Idtau2;
        *Gamma = (2.0 * Dtau - 4.0 + (2.0 * Dtau + 4.0) * *Eps) * Idtau2;
    }
}

/* LocPrfPP (solver.f90:123-179) */
void or_locprf_pp(double *Ploc, const double *Xmu, int Nmu, const double *Xki, const double *Src,
                  const double *Rhox, int Ntau) {
    double *Srd = (double *)malloc(sizeof(double) * 3 * Ntau), *Deltau = Srd + Ntau, *U = Srd + 2 * Ntau;
    or_taustep(Rhox, Xki, 1.0, Ntau, Deltau);
    or_centder(Deltau, Src, 1, Ntau, Srd);
    for (int k = 0; k < Ntau - 1; k++)
        U[k] = 0.5 * (Src[k] + 0.5 * Deltau[k] * Srd[k] + Src[k + 1] - 0.5 * Deltau[k] * Srd[k + 1]);
    for (int im = 0; im < Nmu; im++) {
        double Imu = 1.0 / Xmu[im], Y = Src[Ntau - 1];
        for (int k = Ntau - 2; k >= 0; k--) {
            double Eps, Alpha, Beta, Gamma;
            delo_coef(Deltau[k] * Imu, &Eps, &Alpha, &Beta, &Gamma);
            Y = Y * Eps + Alpha * Src[k] + Beta * Src[k + 1] + Gamma * U[k];
        }
        Ploc[im] = Y;
    }
    free(Srd);
}

/* SphereInit (solver.f90:45-120).  Ray im (impact parameter p = R_top sqrt(1 - mu^2)) crosses the
 * layers 1..n on its near half; a grazing ray (p > R_bottom) turns at the shell below layer n and
 * comes back through layers n..1, so its points n+1..2n mirror 1..n.  Column mass along the ray
 * grows by the radial step times (r_k + r_k-1) / (z_k + z_k-1), z = sqrt(r^2 - p^2) in the factored
 * form, and by chord x dm/dr across the tangent shell. */
int or_sphere_init(int ntau, const double *rhox, const double *height, double radius, int nmu,
                   const double *xmu, int *ntau_mu, int *graz, int *map, double *rhox_mu, double *mu_loc) {
    const int M = 2 * ntau;
    double *Rk = (double *)malloc(sizeof(double) * ntau);
    for (int k = 0; k < ntau; k++) Rk[k] = radius + height[k];
    int rc = 0;
    for (int im = 0; im < nmu && rc == 0; im++) {
        int *mp = map + (size_t)im * M;
        double *rm = rhox_mu + (size_t)im * M, *ml = mu_loc + (size_t)im * M;
        for (int k = 0; k < M; k++) { mp[k] = 0; rm[k] = 0.0; ml[k] = 0.0; }
        if (xmu[im] <= 0.0) { rc = -1; break; }
        double P = Rk[0] * sqrt((1.0 - xmu[im]) * (1.0 + xmu[im]));
        int g = P > Rk[ntau - 1], n = ntau;
        if (g) {
            int kt = 2;
            while (kt <= ntau && !(P >= Rk[kt - 1])) kt++;
            n = kt - 1;
            if (n < 2) { rc = -2; break; }
        }
        rm[0] = rhox[0] / xmu[im];
        double Zk1 = sqrt((Rk[0] - P) * (Rk[0] + P));
        ml[0] = Zk1 / Rk[0];
        mp[0] = 1;
        for (int k = 2; k <= n; k++) {
            double Zk = sqrt((Rk[k - 1] - P) * (Rk[k - 1] + P));
            rm[k - 1] = rm[k - 2] + (rhox[k - 1] - rhox[k - 2]) * (Rk[k - 1] + Rk[k - 2]) / (Zk + Zk1);
            ml[k - 1] = Zk / Rk[k - 1];
            mp[k - 1] = k;
            Zk1 = Zk;
        }
        graz[im] = g;
        if (!g) { ntau_mu[im] = ntau; continue; }
        double Chord = 2.0 * sqrt((Rk[n - 1] - P) * (Rk[n - 1] + P));
        rm[n] = rm[n - 1] + Chord * (rhox[n] - rhox[n - 1]) / (Rk[n - 1] - Rk[n]);
        mp[n] = n;
        ml[n] = -ml[n - 1];
        for (int k = n + 2; k <= 2 * n; k++) {
            rm[k - 1] = rm[k - 2] + (rm[2 * n - k + 1] - rm[2 * n - k]);
            mp[k - 1] = 2 * n + 1 - k;
            ml[k - 1] = -ml[2 * n - k];
        }
        ntau_mu[im] = 2 * n;
    }
    free(Rk);
    return rc;
}

/* DeloScalar (solver.f90:220-261): emergent intensity along one ray from its optical-depth steps,
 * source function and boundary intensity Y0 */
static double delo_scalar(const double *Deltau, const double *Src, int N, double Y0) {
    double *Srd = (double *)malloc(sizeof(double) * N);
    or_centder(Deltau, Src, 1, N, Srd);
    double Y = Y0;
    for (int k = N - 2; k >= 0; k--) {
        double Dtau = Deltau[k], Eps, Alpha, Beta, Gamma;
        delo_coef(Dtau, &Eps, &Alpha, &Beta, &Gamma);
        double U = 0.5 * (Src[k] + 0.5 * Dtau * Srd[k] + Src[k + 1] - 0.5 * Dtau * Srd[k + 1]);
        Y = Y * Eps + Alpha * Src[k] + Beta * Src[k + 1] + Gamma * U;
    }
    free(Srd);
    return Y;
}

/* LocPrfSph (solver.f90:182-216): opacity and source gathered along each ray (MapMu), TauStep on the
 * ray's column mass with mu = 1, zero incoming intensity for grazing rays, Src(N) otherwise */
void or_locprf_sph(const or_state *s, double *Ploc, const double *Xki, const double *Src) {
    const int M = 2 * s->ntau;
    double *XkiR = (double *)malloc(sizeof(double) * 3 * M), *SrcR = XkiR + M, *Deltau = SrcR + M;
    for (int im = 0; im < s->sph_nmu; im++) {
        const int N = s->sph_ntau[im];
        const int *mp = s->sph_map + (size_t)im * M;
        for (int k = 0; k < N; k++) { XkiR[k] = Xki[mp[k] - 1]; SrcR[k] = Src[mp[k] - 1]; }
        or_taustep(s->sph_rhox + (size_t)im * M, XkiR, 1.0, N, Deltau);
        double Y = s->sph_graz[im] ? 0.0 : SrcR[N - 1];
        Ploc[im] = delo_scalar(Deltau, SrcR, N, Y);
    }
    free(XkiR);
}

/* Solve4x4 (solver.f90:541-588): A column-major A[i + 4*j] */
void or_solve4x4(const double *A, const double *B, double *X) {
    double M[16], R[4];
    memcpy(M, A, sizeof M); memcpy(R, B, sizeof R);
#define MM(i, j) M[((i) - 1) + 4 * ((j) - 1)]
    for (int k = 1; k <= 3; k++) {
        int ip = k; double p = fabs(MM(k, k));
        for (int i = k + 1; i <= 4; i++) if (fabs(MM(i, k)) > p) { p = fabs(MM(i, k)); ip = i; }
        if (ip != k) {
            for (int j = k; j <= 4; j++) { double sw = MM(k, j); MM(k, j) = MM(ip, j); MM(ip, j) = sw; }
            double sw = R[k - 1]; R[k - 1] = R[ip - 1]; R[ip - 1] = sw;
        }
        p = 1.0 / MM(k, k);
        for (int i = k + 1; i <= 4; i++) {
            double f = MM(i, k) * p;
            for (int j = k + 1; j <= 4; j++) MM(i, j) = MM(i, j) - f * MM(k, j);
            R[i - 1] = R[i - 1] - f * R[k - 1];
        }
    }
    X[3] = R[3] / MM(4, 4);
    X[2] = (R[2] - MM(3, 4) * X[3]) / MM(3, 3);
    X[1] = (R[1] - MM(2, 3) * X[2] - MM(2, 4) * X[3]) / MM(2, 2);
    X[0] = (R[0] - MM(1, 2) * X[1] - MM(1, 3) * X[2] - MM(1, 4) * X[3]) / MM(1, 1);
#undef MM
}

/* Planck source (synth.f90:1841-1843) */
static void planck(const or_state *s, double wl, double *Src) {
    const double PlkC1 = Hc * Vc * 1e13 / Kbolt;
    double C1 = PlkC1 / wl, C2 = exp(50.7649141 - 5.0 * log(wl));
    for (int t = 0; t < s->ntau; t++) Src[t] = C2 / (exp(C1 / s->T[t]) - 1.0);
}

/* RadTranCalc (synth.f90:1825-1901): LocPrfPP for plane-parallel models, LocPrfSph along the rays
 * of s for spherical ones (radius > 0) */
void or_radtran(const or_state *s, int nmu, const double *xmu, const double *lineopac,
                double *spl, double *spc) {
    int nt = s->ntau;
    const int sph = s->radius > 0.0;
    #pragma omp parallel
    {
        double *Src = (double *)malloc(sizeof(double) * 2 * nt), *Xki = Src + nt;
        #pragma omp for schedule(static)
        for (int iwl = 0; iwl < s->nwl; iwl++) {
            planck(s, s->wave[iwl] + s->wfirst, Src);
            const double *co = s->contopac + (size_t)iwl * nt;
            if (spc) {
                for (int t = 0; t < nt; t++) Xki[t] = co[t];
                if (sph) or_locprf_sph(s, spc + (size_t)iwl * nmu, Xki, Src);
                else or_locprf_pp(spc + (size_t)iwl * nmu, xmu, nmu, Xki, Src, s->rhox, nt);
            }
            for (int t = 0; t < nt; t++) Xki[t] = co[t] + lineopac[(size_t)iwl * nt + t];
            if (sph) or_locprf_sph(s, spl + (size_t)iwl * nmu, Xki, Src);
            else or_locprf_pp(spl + (size_t)iwl * nmu, xmu, nmu, Xki, Src, s->rhox, nt);
        }
        free(Src);
    }
}

/* LinStrCalc (synth.f90:1774-1822) */
static float linstr_calc(const or_state *s, double Wl, const double *LineOpacL,
                         const double *ContOpacL, int nmu, const double *xmu, const double *wmu) {
    int nt = s->ntau;
    double Src[nt], Xki[nt], IntL[nmu > 0 ? nmu : 1], IntC[nmu > 0 ? nmu : 1];
    planck(s, Wl, Src);
    for (int t = 0; t < nt; t++) Xki[t] = ContOpacL[t] + LineOpacL[t];
    if (s->radius > 0.0) {
        or_locprf_sph(s, IntC, ContOpacL, Src);
        or_locprf_sph(s, IntL, Xki, Src);
    } else {
        or_locprf_pp(IntC, xmu, nmu, ContOpacL, Src, s->rhox, nt);
        or_locprf_pp(IntL, xmu, nmu, Xki, Src, s->rhox, nt);
    }
    if (nmu == 1) return (float)(1.0 - IntL[0] / IntC[0]);
    double FlxL = 0.0, FlxC = 0.0;
    for (int i = 0; i < nmu; i++) { FlxL = FlxL + wmu[i] * IntL[i]; FlxC = FlxC + wmu[i] * IntC[i]; }
    return (float)(1.0 - FlxL / FlxC);
}

/* ---- non-magnetic opacity (opacity.f90:297-386, 678-710) -------------------------------- */

typedef struct {           /* working view of the driver's module arrays after PACK */
    long n;
    double *wlcent; int *flag, *ileft, *iright; long *orig;
} linework;

/* LineOpacity2 (opacity.f90:350-386) */
static void lineopacity2(const or_state *s, double Wl, const linework *W, long il, int iwl,
                         const double *cop, const double *vv, const double *av, double *Linop) {
    int nt = s->ntau;
    for (int t = 0; t < nt; t++) Linop[t] = 0.0;
    if (!(W->flag[il] & 1) && iwl >= W->ileft[il] && iwl <= W->iright[il]) {
        int ihe = (W->flag[il] >> 8) & 255;
        double dWl0 = Wl - W->wlcent[il];
        for (int t = 0; t < nt; t++) {
            double dWl = dWl0;
            if (ihe > 0) dWl = dWl0 - s->heshf[(ihe - 1) * nt + t];
            double V = dWl * vv[t];
            Linop[t] = or_hvoigt(av[t], V) * cop[t];
        }
    }
    if (s->motype == 1) for (int t = 0; t < nt; t++) Linop[t] = Linop[t] / s->contopac_std[t];
}

/* AnalyticWindow (opacity.f90:678-710) */
static double analytic_window(const or_state *s, int flag, const double *cop, const double *vv,
                              const double *av, const double *ContOpacL) {
    const double iSqrtPi = 0.5641895835477563;
    int ihe = (flag >> 8) & 255;
    double dWwin = 0.0;
    for (int t = 0; t < s->ntau; t++) {
        double r = cop[t] / (s->epsopac * ContOpacL[t]);
        if (s->motype == 1) r = r / s->contopac_std[t];
        if (r <= 1.0) continue;
        double w = sqrt(log(r) + fmax(0.0, av[t] * (r * iSqrtPi - av[t]))) / vv[t];
        if (ihe > 0) w = w + fabs(s->heshf[(ihe - 1) * s->ntau + t]);
        dWwin = fmax(dWwin, w);
    }
    return dWwin;
}

/* WlcIdx (synth.f90:677-706) over the packed centres */
static long wlc_idx(const linework *W, double w) {
    if (W->n == 0 || w < W->wlcent[0]) return 0;
    long ia = 1, ib = W->n;
    while (ib - ia > 1) { long im = (ia + ib) / 2; if (W->wlcent[im - 1] <= w) ia = im; else ib = im; }
    return (W->wlcent[ib - 1] <= w) ? ib : ia;
}

/* MarkWideLines (synth.f90:709-744) */
static long mark_wide(const or_state *s, linework *W, long nlines_step) {
    long nwide = 0;
    #pragma omp parallel for schedule(static) reduction(+:nwide)
    for (long i = 0; i < W->n; i++) {
        if (W->flag[i] & 1) continue;
        long nrec = wlc_idx(W, s->wave[W->iright[i] - 1]) - wlc_idx(W, s->wave[W->ileft[i] - 1]) + 1;
        double dv = Vc * (s->wave[W->iright[i] - 1] - s->wave[W->ileft[i] - 1]) / (W->wlcent[i] + s->wfirst);
        if (nrec > nlines_step / 2 || dv > 5e3) { W->flag[i] |= 8; nwide++; }
    }
    return nwide;
}

/* central continuum at the line centre (synth.f90:870-874) */
static int cont_at_center(const or_state *s, double wlc, double *ContOpacL) {
    int iwl = or_waveidx(s, wlc), nt = s->ntau;
    double dW = (wlc - s->wave[iwl - 1]) / (s->wave[iwl] - s->wave[iwl - 1]);
    const double *c0 = s->contopac + (size_t)(iwl - 1) * nt, *c1 = c0 + nt;
    for (int t = 0; t < nt; t++) ContOpacL[t] = c0[t] * (1.0 - dW) + c1[t] * dW;
    return iwl;
}

/* Lstart/Lstop (synth.f90:955-978 / 1314-1338) */
static long line_pointers(const or_state *s, const linework *W, int *Lstart, int *Lstop) {
    long nuse = W->n;
    for (int i = 0; i < s->nwl; i++) { Lstart[i] = (int)W->n; Lstop[i] = 1; }
    for (long il = 0; il < W->n; il++) {
        if (W->flag[il] & 1) { nuse--; continue; }
        if (W->flag[il] & 8) continue;
        for (int iwl = W->ileft[il]; iwl <= W->iright[il]; iwl++) {
            if ((long)Lstart[iwl - 1] > il + 1) Lstart[iwl - 1] = (int)(il + 1);
            if ((long)Lstop[iwl - 1] < il + 1) Lstop[iwl - 1] = (int)(il + 1);
        }
    }
    return nuse;
}

/* segment selection (synth.f90:1014-1044); returns iwl2 or -1 on overflow */
static int next_segment(const or_state *s, const int *Lstart, const int *Lstop, long nlines,
                        long nlines_step, int iwl1, long *iline1) {
    if (nlines_step >= nlines) return s->nwl;
    long ilo = nlines + 1, ihi = 0; int iwl2 = iwl1 - 1;
    for (int iwl = iwl1; iwl <= s->nwl; iwl++) {
        long ilot = ilo < Lstart[iwl - 1] ? ilo : Lstart[iwl - 1];
        long ihit = ihi > Lstop[iwl - 1] ? ihi : Lstop[iwl - 1];
        if (ihit - ilot + 1 > nlines_step) break;
        ilo = ilot; ihi = ihit; iwl2 = iwl;
    }
    if (iwl2 < iwl1) return -1;
    long t = ilo > 1 ? ilo : 1; *iline1 = t < nlines ? t : nlines;
    return iwl2;
}

static void pack_lines(const or_state *s, linework *W, double *bc, double *bv, double *ba) {
    long m = 0; int nt = s->ntau;
    for (long i = 0; i < W->n; i++) {
        if (W->flag[i] & 1) continue;
        W->wlcent[m] = W->wlcent[i]; W->flag[m] = W->flag[i]; W->ileft[m] = W->ileft[i];
        W->iright[m] = W->iright[i]; W->orig[m] = W->orig[i];
        memmove(bc + m * nt, bc + i * nt, sizeof(double) * nt);
        memmove(bv + m * nt, bv + i * nt, sizeof(double) * nt);
        memmove(ba + m * nt, ba + i * nt, sizeof(double) * nt);
        m++;
    }
    W->n = m;
}

/* LineopCalc (synth.f90:747-1095) */
int or_lineop_calc(const or_state *s, const or_lines *L, int list_type, long nlines_lim,
                   double *lineopac, int *flags_out, int *ileft_out, int *iright_out,
                   float *linstr_out, int nmu, const double *xmu, const double *wmu,
                   or_stats *st) {
    return or_lineop_calc_range(s, L, list_type, nlines_lim, lineopac, flags_out, ileft_out, iright_out,
                                linstr_out, nmu, xmu, wmu, st, 1, s->nwl);
}

/* LineopCalc with the accumulation restricted to the wavelengths [r0, r1] */
int or_lineop_calc_range(const or_state *s, const or_lines *L, int list_type, long nlines_lim,
                         double *lineopac, int *flags_out, int *ileft_out, int *iright_out,
                         float *linstr_out, int nmu, const double *xmu, const double *wmu,
                         or_stats *st, int r0, int r1) {
    or_voigt_init();
    int nt = s->ntau, nwl = s->nwl;
    if (r0 < 1) r0 = 1;
    if (r1 > nwl) r1 = nwl;
    long N = L->n;
    long nstep = (nlines_lim > 0 && nlines_lim < N) ? nlines_lim : N;
    linework W; W.n = N;
    W.wlcent = (double *)malloc(sizeof(double) * (N ? N : 1));
    W.flag = (int *)calloc(N ? N : 1, sizeof(int));
    W.ileft = (int *)malloc(sizeof(int) * (N ? N : 1));
    W.iright = (int *)malloc(sizeof(int) * (N ? N : 1));
    W.orig = (long *)malloc(sizeof(long) * (N ? N : 1));
    double *bc = (double *)malloc(sizeof(double) * nt * (nstep ? nstep : 1));
    double *bv = (double *)malloc(sizeof(double) * nt * (nstep ? nstep : 1));
    double *ba = (double *)malloc(sizeof(double) * nt * (nstep ? nstep : 1));
    if (!W.wlcent || !W.flag || !W.ileft || !W.iright || !W.orig || !bc || !bv || !ba) return -1;
    for (long i = 0; i < N; i++) {
        W.wlcent[i] = L->wl[i] - s->wfirst; W.ileft[i] = 1; W.iright[i] = nwl; W.orig[i] = i;
    }
    int dolinstr = (linstr_out != NULL) && nmu >= 1;

    /* central pass (synth.f90:833-907) */
    #pragma omp parallel
    {
        double *cop = (double *)malloc(sizeof(double) * 5 * nt), *vv = cop + nt, *av = cop + 2 * nt;
        double *lo = cop + 3 * nt, *co = cop + 4 * nt;
        #pragma omp for schedule(guided, 1000)
        for (long i = 0; i < N; i++) {
            xcoef XC; int f = input_flags(L, i, list_type);
            xline_setup(s, L, i, W.wlcent[i], f, &XC);
            if (XC.IxHe > 0) f |= (XC.IxHe << 8);
            for (int t = 0; t < nt; t++) xline_depth(s, t, &XC, &cop[t], &vv[t], &av[t]);
            if (i < nstep) { memcpy(bc + i * nt, cop, sizeof(double) * nt);
                             memcpy(bv + i * nt, vv, sizeof(double) * nt);
                             memcpy(ba + i * nt, av, sizeof(double) * nt); }
            int iwl = cont_at_center(s, W.wlcent[i], co);
            double mx = -DBL_MAX;
            for (int t = 0; t < nt; t++) {
                double r = (s->motype == 1) ? cop[t] / (co[t] * s->contopac_std[t]) : cop[t] / co[t];
                mx = fmax(mx, r);
            }
            if (mx < s->epsopac) { W.flag[i] = f | 1; continue; }
            W.flag[i] = f;
            lineopacity2(s, W.wlcent[i], &W, i, iwl, cop, vv, av, lo);
            mx = -DBL_MAX;
            for (int t = 0; t < nt; t++) mx = fmax(mx, lo[t] / co[t]);
            if (mx < s->epsopac) { W.flag[i] = f | 1; continue; }
            else if (dolinstr) linstr_out[i] = linstr_calc(s, W.wlcent[i] + s->wfirst, lo, co, nmu, xmu, wmu);
            double dW = analytic_window(s, f, cop, vv, av, co);
            W.ileft[i] = or_waveidx(s, W.wlcent[i] - dW);
            int ir = or_waveidx(s, W.wlcent[i] + dW) + 1;
            W.iright[i] = ir < nwl ? ir : nwl;
        }
        free(cop);
    }
    if (flags_out || ileft_out || iright_out)
        for (long i = 0; i < N; i++) {
            if (flags_out) flags_out[i] = W.flag[i];
            if (ileft_out) ileft_out[i] = W.ileft[i];
            if (iright_out) iright_out[i] = W.iright[i];
        }

    /* PACK (synth.f90:915-933) */
    if ((list_type == 0 || list_type == 2) && nstep == N) pack_lines(s, &W, bc, bv, ba);
    if (st) { memset(st, 0, sizeof *st); st->nlines_in = N; }
    if (W.n == 0) { if (st) st->nweak = N; goto done; }

    long nwide = mark_wide(s, &W, nstep);
    if (flags_out) for (long i = 0; i < W.n; i++) flags_out[W.orig[i]] = W.flag[i];
    int *Lstart = (int *)malloc(sizeof(int) * nwl), *Lstop = (int *)malloc(sizeof(int) * nwl);
    long nuse = line_pointers(s, &W, Lstart, Lstop);

    /* wide lines (synth.f90:981-1001) */
    double wide_evals = 0.0;
    if (nwide > 0) {
        double *cop = (double *)malloc(sizeof(double) * 3 * nt), *vv = cop + nt, *av = cop + 2 * nt;
        for (long il = 0; il < W.n; il++) {
            if (!(W.flag[il] & 8)) continue;
            xcoef XC; long i0 = W.orig[il];
            xline_setup(s, L, i0, W.wlcent[il], W.flag[il], &XC);
            for (int t = 0; t < nt; t++) xline_depth(s, t, &XC, &cop[t], &vv[t], &av[t]);
            const int wa = W.ileft[il] > r0 ? W.ileft[il] : r0, wb = W.iright[il] < r1 ? W.iright[il] : r1;
            if (wa <= wb) wide_evals += (double)nt * (wb - wa + 1);
            #pragma omp parallel
            {
                double *lo = (double *)malloc(sizeof(double) * nt);
                #pragma omp for schedule(dynamic, 1000)
                for (int iwl = wa; iwl <= wb; iwl++) {
                    lineopacity2(s, s->wave[iwl - 1], &W, il, iwl, cop, vv, av, lo);
                    double *dst = lineopac + (size_t)(iwl - 1) * nt;
                    for (int t = 0; t < nt; t++) dst[t] = dst[t] + lo[t];
                }
                free(lo);
            }
        }
        free(cop);
    }

    /* segment loop (synth.f90:1006-1088) */
    long iline1 = 1, ilineb = 1, nseg = 0, nrefill = 0; int iwl1 = 1;
    double evals = 0.0;
    for (;;) {
        int iwl2 = next_segment(s, Lstart, Lstop, W.n, nstep, iwl1, &iline1);
        if (iwl2 < 0) { free(Lstart); free(Lstop); return -2; }
        nseg++;
        long iline2 = iline1 + nstep - 1 < W.n ? iline1 + nstep - 1 : W.n;
        long Loff = iline1 - 1;
        if (iline1 != ilineb) {
            ilineb = iline1; nrefill++;
            #pragma omp parallel for
            for (long il = iline1; il <= iline2; il++) {
                if (W.flag[il - 1] & 1) continue;
                long j = il - iline1; xcoef XC; long i0 = W.orig[il - 1];
                xline_setup(s, L, i0, W.wlcent[il - 1], W.flag[il - 1], &XC);
                for (int t = 0; t < nt; t++)
                    xline_depth(s, t, &XC, &bc[j * nt + t], &bv[j * nt + t], &ba[j * nt + t]);
            }
        }
        /* LineOpacity1 (opacity.f90:297-346) */
        #pragma omp parallel reduction(+:evals)
        {
            double *lo = (double *)malloc(sizeof(double) * nt);
            const int pa = iwl1 > r0 ? iwl1 : r0, pb = iwl2 < r1 ? iwl2 : r1;
            #pragma omp for schedule(dynamic)
            for (int iwl = pa; iwl <= pb; iwl++) {
                double Wl = s->wave[iwl - 1];
                for (int t = 0; t < nt; t++) lo[t] = 0.0;
                for (long il = Lstart[iwl - 1]; il <= Lstop[iwl - 1]; il++) {
                    int f = W.flag[il - 1];
                    if ((f & 1) || (f & 8) || iwl < W.ileft[il - 1] || iwl > W.iright[il - 1]) continue;
                    int ihe = (f >> 8) & 255;
                    double dWl0 = Wl - W.wlcent[il - 1];
                    const double *c = bc + (il - Loff - 1) * nt, *v = bv + (il - Loff - 1) * nt,
                                 *a = ba + (il - Loff - 1) * nt;
                    for (int t = 0; t < nt; t++) {
                        double dWl = dWl0;
                        if (ihe > 0) dWl = dWl0 - s->heshf[(ihe - 1) * nt + t];
                        double V = dWl * v[t];
                        lo[t] = lo[t] + or_hvoigt(a[t], V) * c[t];
                    }
                    evals += (double)nt;
                }
                if (s->motype == 1) for (int t = 0; t < nt; t++) lo[t] = lo[t] / s->contopac_std[t];
                double *dst = lineopac + (size_t)(iwl - 1) * nt;
                for (int t = 0; t < nt; t++) dst[t] = dst[t] + lo[t];
            }
            free(lo);
        }
        if (iwl2 == nwl) break;
        iwl1 = iwl2 + 1;
    }
    if (st) { st->nlines_used = nuse; st->nwide = nwide; st->nweak = N - nuse;
              st->nsegments = nseg; st->nrefills = nrefill; st->line_evals = evals;
              st->wide_evals = wide_evals; }
    free(Lstart); free(Lstop);
done:
    free(W.wlcent); free(W.flag); free(W.ileft); free(W.iright); free(W.orig);
    free(bc); free(bv); free(ba);
    return 0;
}

/* ---- magnetic opacity (opacity.f90:391-591, 611-675; synth.f90:1098-1455) ---------------- */

typedef struct {           /* per-line scaled Zeeman components (FP32, synth.f90:1193-1194) */
    int npi, nsi; const float *strpi, *strsi; float *splpi, *splsi;
} zlines;

/* MagLineOpacity2 (opacity.f90:468-520) */
static void maglineopacity2(const or_state *s, double Wl, const linework *W, long il, int iwl,
                            const zlines *Z, const double *cop, const double *vv, const double *av,
                            double *Linop) {
    int nt = s->ntau;
    for (int t = 0; t < nt; t++) Linop[t] = 0.0;
    if (!(W->flag[il] & 1) && iwl >= W->ileft[il] && iwl <= W->iright[il]) {
        int ihe = (W->flag[il] >> 8) & 255;
        double dWl0 = Wl - W->wlcent[il];
        for (int t = 0; t < nt; t++) {
            double dWl = dWl0;
            if (ihe > 0) dWl = dWl0 - s->heshf[(ihe - 1) * nt + t];
            vline VL = vline_init(av[t]);
            double Pp = 0.0, Ps = 0.0;
            for (int k = 0; k < Z->npi; k++)
                Pp = Pp + (double)Z->strpi[k] * hvoigt_line(VL, (dWl - (double)Z->splpi[k]) * vv[t]);
            for (int k = 0; k < Z->nsi; k++)
                Ps = Ps + (double)Z->strsi[k] * hvoigt_line(VL, (dWl - (double)Z->splsi[k]) * vv[t]);
            Linop[t] = fmax(0.5 * Ps, 0.5 * Pp + 0.25 * Ps) * cop[t];
        }
    }
    if (s->motype == 1) for (int t = 0; t < nt; t++) Linop[t] = Linop[t] / s->contopac_std[t];
}

/* six Zeeman profiles of one line at one wavelength (MagLineOpacity1/3 inner loops) */
static void mag_profiles(const or_state *s, double Wl, double wlc, int ihe, const zlines *Z,
                         const double *cop, const double *vv, const double *av, double *M) {
    int nt = s->ntau;
    for (int t = 0; t < nt; t++) {
        vline FL = fvline_init(av[t]);
        double Xn = cop[t], sc = vv[t], Vbase = (Wl - wlc) * sc;
        if (ihe > 0) Vbase = Vbase - s->heshf[(ihe - 1) * nt + t] * sc;
        double *m = M + 6 * t;
        for (int k = 0; k < Z->npi; k++) {
            double V = Vbase - (double)Z->splpi[k] * sc, Vg, Fv; fvoigt_line(FL, V, &Vg, &Fv);
            double Str = Xn * (double)Z->strpi[k];
            m[0] = m[0] + Str * Vg; m[3] = m[3] + Str * Fv;
        }
        int Nsh = Z->nsi / 2;
        for (int k = 0; k < Nsh; k++) {
            double V = Vbase - (double)Z->splsi[k] * sc, Vg, Fv; fvoigt_line(FL, V, &Vg, &Fv);
            double Str = Xn * (double)Z->strsi[k];
            m[1] = m[1] + Str * Vg; m[4] = m[4] + Str * Fv;
        }
        for (int k = Nsh; k < Z->nsi; k++) {
            double V = Vbase - (double)Z->splsi[k] * sc, Vg, Fv; fvoigt_line(FL, V, &Vg, &Fv);
            double Str = Xn * (double)Z->strsi[k];
            m[2] = m[2] + Str * Vg; m[5] = m[5] + Str * Fv;
        }
    }
}

/* RefineIdx (opacity.f90:611-675), magnetic branch */
static void refine_idx(const or_state *s, linework *W, long il, int iwl, int idw, const zlines *Z,
                       const double *cop, const double *vv, const double *av, const double *co,
                       double SplMax, double *lo) {
    int nt = s->ntau, isw, ikw;
    if (W->wlcent[il] > 0.5 * (s->wave[0] + s->wave[s->nwl - 1])) { isw = -1; ikw = 0; }
    else { isw = 1; ikw = 1; }
    double Wl = W->wlcent[il], dW; int ia, ib;
    if (idw == 0) ia = or_waveidx(s, Wl + (double)isw * SplMax) + ikw;
    else {
        dW = (0.2 * pow(2.0, idw - 1)) * (W->wlcent[il] + s->wfirst) / 5e3;
        ia = or_waveidx(s, Wl + (double)isw * (SplMax + dW)) + ikw;
    }
    dW = (0.2 * pow(2.0, idw)) * (W->wlcent[il] + s->wfirst) / 5e3;
    ib = or_waveidx(s, Wl + (double)isw * (SplMax + dW)) + ikw;
    while (abs(ia - ib) > 1) {
        int im = (ia + ib) / 2;
        maglineopacity2(s, s->wave[im - 1], W, il, iwl, Z, cop, vv, av, lo);
        double mx = -DBL_MAX; for (int t = 0; t < nt; t++) mx = fmax(mx, lo[t] / co[t]);
        if (mx < s->epsopac) ib = im; else ia = im;
    }
    if (isw == 1) { W->iright[il] = ia; W->ileft[il] = or_waveidx(s, 2.0 * Wl - s->wave[ia - 1]); }
    else { W->ileft[il] = ia; W->iright[il] = or_waveidx(s, 2.0 * Wl - s->wave[ia - 1]) + 1; }
}

int or_mag_lineop_calc(const or_state *s, const or_lines *L, int bframe, const double *bfield,
                       long nlines_lim, double *maglineopac, int *flags_out, int *ileft_out,
                       int *iright_out, float *linstr_out, int nmu, const double *xmu,
                       const double *wmu, or_stats *st) {
    or_voigt_init(); or_fvoigt_init();
    int nt = s->ntau, nwl = s->nwl;
    long N = L->n;
    long nstep = (nlines_lim > 0 && nlines_lim < N) ? nlines_lim : N;
    linework W; W.n = N;
    W.wlcent = (double *)malloc(sizeof(double) * (N ? N : 1));
    W.flag = (int *)calloc(N ? N : 1, sizeof(int));
    W.ileft = (int *)malloc(sizeof(int) * (N ? N : 1));
    W.iright = (int *)malloc(sizeof(int) * (N ? N : 1));
    W.orig = (long *)malloc(sizeof(long) * (N ? N : 1));
    zlines *Z = (zlines *)malloc(sizeof(zlines) * (N ? N : 1));
    long ntot_pi = N ? L->pi_off[N - 1] + L->npi[N - 1] : 0, ntot_si = N ? L->si_off[N - 1] + L->nsi[N - 1] : 0;
    float *spl_pi = (float *)malloc(sizeof(float) * (ntot_pi + 1)), *spl_si = (float *)malloc(sizeof(float) * (ntot_si + 1));
    double *bc = (double *)malloc(sizeof(double) * nt * (nstep ? nstep : 1));
    double *bv = (double *)malloc(sizeof(double) * nt * (nstep ? nstep : 1));
    double *ba = (double *)malloc(sizeof(double) * nt * (nstep ? nstep : 1));
    for (long i = 0; i < N; i++) {
        W.wlcent[i] = L->wl[i] - s->wfirst; W.ileft[i] = 1; W.iright[i] = nwl; W.orig[i] = i;
        Z[i].npi = L->npi[i]; Z[i].nsi = L->nsi[i];
        Z[i].strpi = L->str_pi + L->pi_off[i]; Z[i].strsi = L->str_si + L->si_off[i];
        Z[i].splpi = spl_pi + L->pi_off[i]; Z[i].splsi = spl_si + L->si_off[i];
    }
    double Bsplit = (bframe == 0)
        ? Kz * sqrt(bfield[0] * bfield[0] + bfield[1] * bfield[1] + bfield[2] * bfield[2])
        : Kz * fabs(bfield[0]);
    int dolinstr = (linstr_out != NULL) && nmu >= 1;

    #pragma omp parallel
    {
        double *cop = (double *)malloc(sizeof(double) * 5 * nt), *vv = cop + nt, *av = cop + 2 * nt;
        double *lo = cop + 3 * nt, *co = cop + 4 * nt;
        #pragma omp for schedule(guided, 1000)
        for (long i = 0; i < N; i++) {
            int f = 0;
            if (L->ismol && L->ismol[i]) f |= 2;
            if (L->gvdw[i] > 10.0f) f |= 4;
            double w = W.wlcent[i] + s->wfirst;
            double SplMax = -(double)FLT_MAX, mpi = -(double)FLT_MAX;
            for (int k = 0; k < Z[i].npi; k++) {
                Z[i].splpi[k] = (float)((double)L->spl_pi[L->pi_off[i] + k] * Bsplit * (w * w));
                mpi = fmax(mpi, fabs((double)Z[i].splpi[k]));
            }
            for (int k = 0; k < Z[i].nsi; k++) {
                Z[i].splsi[k] = (float)((double)L->spl_si[L->si_off[i] + k] * Bsplit * (w * w));
                SplMax = fmax(SplMax, fabs((double)Z[i].splsi[k]));
            }
            SplMax = fmax(SplMax, mpi);
            xcoef XC; xline_setup(s, L, i, W.wlcent[i], f, &XC);
            if (XC.IxHe > 0) f |= (XC.IxHe << 8);
            for (int t = 0; t < nt; t++) xline_depth(s, t, &XC, &cop[t], &vv[t], &av[t]);
            if (i < nstep) { memcpy(bc + i * nt, cop, sizeof(double) * nt);
                             memcpy(bv + i * nt, vv, sizeof(double) * nt);
                             memcpy(ba + i * nt, av, sizeof(double) * nt); }
            int iwl = cont_at_center(s, W.wlcent[i], co);
            W.flag[i] = f;
            lineopacity2(s, W.wlcent[i], &W, i, iwl, cop, vv, av, lo);
            double mx = -DBL_MAX; for (int t = 0; t < nt; t++) mx = fmax(mx, lo[t] / co[t]);
            if (mx < s->epsopac) { W.flag[i] = f | 1; continue; }
            else if (dolinstr) linstr_out[i] = linstr_calc(s, W.wlcent[i] + s->wfirst, lo, co, nmu, xmu, wmu);
            for (int idw = 0;; idw++) {
                double dW = (0.2 * pow(2.0, idw)) * (W.wlcent[i] + s->wfirst) / 5e3;
                double Wl = W.wlcent[i] + SplMax + dW;
                maglineopacity2(s, Wl, &W, i, iwl, &Z[i], cop, vv, av, lo);
                mx = -DBL_MAX; for (int t = 0; t < nt; t++) mx = fmax(mx, lo[t] / co[t]);
                if (mx < s->epsopac) { refine_idx(s, &W, i, iwl, idw, &Z[i], cop, vv, av, co, SplMax, lo); break; }
                else if (W.wlcent[i] - SplMax - dW < s->wave[0] && W.wlcent[i] + SplMax + dW > s->wave[nwl - 1]) break;
            }
        }
        free(cop);
    }
    if (flags_out || ileft_out || iright_out)
        for (long i = 0; i < N; i++) {
            if (flags_out) flags_out[i] = W.flag[i];
            if (ileft_out) ileft_out[i] = W.ileft[i];
            if (iright_out) iright_out[i] = W.iright[i];
        }
    /* PACK (synth.f90:1283-1297): compact Z alongside */
    if (nstep == N) {
        long m = 0;
        for (long i = 0; i < W.n; i++) if (!(W.flag[i] & 1)) Z[m++] = Z[i];
        pack_lines(s, &W, bc, bv, ba);
    }
    if (st) { memset(st, 0, sizeof *st); st->nlines_in = N; }
    if (W.n == 0) goto done;
    long nwide = mark_wide(s, &W, nstep);
    if (flags_out) for (long i = 0; i < W.n; i++) flags_out[W.orig[i]] = W.flag[i];
    int *Lstart = (int *)malloc(sizeof(int) * nwl), *Lstop = (int *)malloc(sizeof(int) * nwl);
    long nuse = line_pointers(s, &W, Lstart, Lstop);
    double wide_evals = 0.0;
    if (nwide > 0) {
        double *cop = (double *)malloc(sizeof(double) * 3 * nt), *vv = cop + nt, *av = cop + 2 * nt;
        for (long il = 0; il < W.n; il++) {
            if (!(W.flag[il] & 8)) continue;
            xcoef XC; long i0 = W.orig[il];
            xline_setup(s, L, i0, W.wlcent[il], W.flag[il], &XC);
            for (int t = 0; t < nt; t++) xline_depth(s, t, &XC, &cop[t], &vv[t], &av[t]);
            wide_evals += (double)nt * (W.iright[il] - W.ileft[il] + 1);
            int ihe = (W.flag[il] >> 8) & 255;
            #pragma omp parallel
            {
                double *M = (double *)malloc(sizeof(double) * 6 * nt);
                #pragma omp for schedule(dynamic, 1000)
                for (int iwl = W.ileft[il]; iwl <= W.iright[il]; iwl++) {
                    for (int q = 0; q < 6 * nt; q++) M[q] = 0.0;
                    mag_profiles(s, s->wave[iwl - 1], W.wlcent[il], ihe, &Z[il], cop, vv, av, M);
                    double *dst = maglineopac + (size_t)(iwl - 1) * nt * 6;
                    for (int t = 0; t < nt; t++)
                        for (int q = 0; q < 6; q++) {
                            double v = M[6 * t + q];
                            if (s->motype == 1) v = v / s->contopac_std[t];
                            dst[6 * t + q] = dst[6 * t + q] + v;
                        }
                }
                free(M);
            }
        }
        free(cop);
    }
    long iline1 = 1, ilineb = 1, nseg = 0, nrefill = 0; int iwl1 = 1;
    double evals = 0.0;
    for (;;) {
        int iwl2 = next_segment(s, Lstart, Lstop, W.n, nstep, iwl1, &iline1);
        if (iwl2 < 0) { free(Lstart); free(Lstop); return -2; }
        nseg++;
        long iline2 = iline1 + nstep - 1 < W.n ? iline1 + nstep - 1 : W.n;
        long Loff = iline1 - 1;
        if (iline1 != ilineb) {
            ilineb = iline1; nrefill++;
            #pragma omp parallel for
            for (long il = iline1; il <= iline2; il++) {
                if (W.flag[il - 1] & 1) continue;
                long j = il - iline1; xcoef XC; long i0 = W.orig[il - 1];
                xline_setup(s, L, i0, W.wlcent[il - 1], W.flag[il - 1], &XC);
                for (int t = 0; t < nt; t++)
                    xline_depth(s, t, &XC, &bc[j * nt + t], &bv[j * nt + t], &ba[j * nt + t]);
            }
        }
        /* MagLineOpacity1 (opacity.f90:391-464) */
        #pragma omp parallel reduction(+:evals)
        {
            double *M = (double *)malloc(sizeof(double) * 6 * nt);
            #pragma omp for schedule(dynamic)
            for (int iwl = iwl1; iwl <= iwl2; iwl++) {
                double Wl = s->wave[iwl - 1];
                for (int q = 0; q < 6 * nt; q++) M[q] = 0.0;
                for (long il = Lstart[iwl - 1]; il <= Lstop[iwl - 1]; il++) {
                    int f = W.flag[il - 1];
                    if ((f & 1) || (f & 8) || iwl < W.ileft[il - 1] || iwl > W.iright[il - 1]) continue;
                    long j = il - Loff - 1;
                    mag_profiles(s, Wl, W.wlcent[il - 1], (f >> 8) & 255, &Z[il - 1], bc + j * nt,
                                 bv + j * nt, ba + j * nt, M);
                    evals += (double)nt * (Z[il - 1].npi + Z[il - 1].nsi);
                }
                double *dst = maglineopac + (size_t)(iwl - 1) * nt * 6;
                for (int t = 0; t < nt; t++)
                    for (int q = 0; q < 6; q++) {
                        double v = M[6 * t + q];
                        if (s->motype == 1) v = v / s->contopac_std[t];
                        dst[6 * t + q] = dst[6 * t + q] + v;
                    }
            }
            free(M);
        }
        if (iwl2 == nwl) break;
        iwl1 = iwl2 + 1;
    }
    if (st) { st->nlines_used = nuse; st->nwide = nwide; st->nweak = N - W.n;
              st->nsegments = nseg; st->nrefills = nrefill; st->line_evals = evals;
              st->wide_evals = wide_evals; }
    free(Lstart); free(Lstop);
done:
    free(W.wlcent); free(W.flag); free(W.ileft); free(W.iright); free(W.orig);
    free(Z); free(spl_pi); free(spl_si); free(bc); free(bv); free(ba);
    return 0;
}

/* The DELO-Bezier sweep of StokesPrfPP / StokesPrfSph (solver.f90:341-390, 486-534) along one ray of N
 * points: XK/XKD [N][16] column-major 4x4 per point, SRC4/SRD [N][4], Deltau [N-1]; XINT2 holds the
 * boundary Stokes vector on entry and the emergent one on return */
static void stokes_sweep(int N, const double *XK, const double *XKD, const double *SRC4, const double *SRD,
                         const double *Deltau, double *XINT2) {
#define K(i, j, t) XK[(t) * 16 + ((i) - 1) + 4 * ((j) - 1)]
#define KD(i, j, t) XKD[(t) * 16 + ((i) - 1) + 4 * ((j) - 1)]
    double XINT1[4], XKA[16], XKB[16], QA[16], QB[16], AA[16];
    for (int j = 1; j <= 4; j++) for (int i = 1; i <= 4; i++) {
        double acc = 0.0;
        for (int k = 1; k <= 4; k++) acc = acc + K(i, k, N - 1) * K(k, j, N - 1);
        XKB[(i - 1) + 4 * (j - 1)] = acc + KD(i, j, N - 1);
    }
    for (int k = N - 2; k >= 0; k--) {
        int k1 = k + 1;
        double Dtau = Deltau[k], Dtau05 = 0.5 * Dtau, Eps, Alpha, Beta, Gamma;
        delo_coef(Dtau, &Eps, &Alpha, &Beta, &Gamma);
        Gamma = Gamma * 0.5;
        memcpy(XKA, XKB, sizeof XKA);
        for (int j = 1; j <= 4; j++) for (int i = 1; i <= 4; i++) {
            double acc = 0.0;
            for (int q = 1; q <= 4; q++) acc = acc + K(i, q, k) * K(q, j, k);
            XKB[(i - 1) + 4 * (j - 1)] = acc + KD(i, j, k);
        }
        for (int j = 1; j <= 4; j++) for (int i = 1; i <= 4; i++) {
            int e = (i - 1) + 4 * (j - 1);
            QA[e] = Dtau05 * XKA[e] + (Dtau05 - 1.0) * K(i, j, k1);
            QB[e] = -(Dtau05 * XKB[e]) - (Dtau05 + 1.0) * K(i, j, k);
            AA[e] = ((i == j) ? 1.0 : 0.0) + Alpha * K(i, j, k) - Gamma * QB[e];
        }
        double GD = Gamma * Dtau05;
        for (int i = 1; i <= 4; i++) {
            double m1 = 0.0, m2 = 0.0, m3 = 0.0, m4 = 0.0;
            for (int q = 1; q <= 4; q++) {
                m1 = m1 + K(i, q, k1) * XINT2[q - 1];
                m2 = m2 + QA[(i - 1) + 4 * (q - 1)] * XINT2[q - 1];
                m3 = m3 + K(i, q, k1) * SRC4[4 * k1 + q - 1];
                m4 = m4 + K(i, q, k) * SRC4[4 * k + q - 1];
            }
            XINT1[i - 1] = Eps * XINT2[i - 1] - Beta * m1 + Gamma * m2 + (Beta + Gamma) * SRC4[4 * k1 + i - 1]
                         - GD * m3 + (Alpha + Gamma) * SRC4[4 * k + i - 1] + GD * m4
                         + GD * (SRD[4 * k + i - 1] - SRD[4 * k1 + i - 1]);
        }
        or_solve4x4(AA, XINT1, XINT2);
    }
#undef K
#undef KD
}

/* Propagation matrix normalised by PhiI and source vector at one point (solver.f90:296-330, 431-465):
 * m = MagLineOpac(:, ia), lop/cop the line and continuum opacity there, geometry g = (SPhi2, CPhi2,
 * CPhi, S2Psi, C2Psi) of this point; writes the 4x4 K (column-major) and SRC4, returns PhiI */
static double stokes_point(const double *m, double lop, double cop, double Src, const double *g,
                           double *K16, double *S4) {
    double Php = m[0], Phb = m[1], Phr = m[2], Psp = m[3], Psb = m[4], Psr = m[5];
    double SPhi2 = g[0], CPhi2 = g[1], CPhi = g[2], S2Psi = g[3], C2Psi = g[4];
    double PhiI = 0.5 * (Php * SPhi2 + 0.5 * (Phr + Phb) * (1.0 + CPhi2)) + lop + cop;
    double InvPhiI = 1.0 / PhiI;
    double Sabs = 0.5 * (Php - 0.5 * (Phr + Phb)) * SPhi2;
    double PhiQ = Sabs * C2Psi * InvPhiI, PhiU = Sabs * S2Psi * InvPhiI;
    double PhiV = 0.5 * (Phr - Phb) * CPhi * InvPhiI;
    double Sdis = 0.5 * (Psp - 0.5 * (Psr + Psb)) * SPhi2;
    double PsiQ = Sdis * C2Psi * InvPhiI, PsiU = Sdis * S2Psi * InvPhiI;
    double PsiV = 0.5 * (Psr - Psb) * CPhi * InvPhiI;
#define K(i, j) K16[((i) - 1) + 4 * ((j) - 1)]
    K(1,1) = 0.0;   K(1,2) = PhiQ;  K(1,3) = PhiU;  K(1,4) = PhiV;
    K(2,1) = PhiQ;  K(2,2) = 0.0;   K(2,3) = PsiV;  K(2,4) = -PsiU;
    K(3,1) = PhiU;  K(3,2) = -PsiV; K(3,3) = 0.0;   K(3,4) = PsiQ;
    K(4,1) = PhiV;  K(4,2) = PsiU;  K(4,3) = -PsiQ; K(4,4) = 0.0;
#undef K
    S4[0] = Src; S4[1] = Src * PhiQ; S4[2] = Src * PhiU; S4[3] = Src * PhiV;
    return PhiI;
}

/* StokesPrfPP (solver.f90:265-394); M6 = MagLineOpac(:, :, iwl) as [ntau][6] */
static void stokes_prf_pp(const or_state *s, const double *M6, const double *lop, const double *cop,
                          const double *Src, int nmu, const double *xmu, const double *SPhi2,
                          const double *CPhi2, const double *CPhi, const double *S2Psi,
                          const double *C2Psi, double *Stokes /*[4][nmu]*/) {
    int N = s->ntau;
    double *XK = (double *)malloc(sizeof(double) * (16 * N * 2 + N * 10));
    double *XKD = XK + 16 * N, *XKI = XKD + 16 * N, *Deltau = XKI + N, *SRC4 = Deltau + N, *SRD = SRC4 + 4 * N;
    for (int im = 0; im < nmu; im++) {
        double g[5] = { SPhi2[im], CPhi2[im], CPhi[im], S2Psi[im], C2Psi[im] };
        for (int t = 0; t < N; t++) XKI[t] = stokes_point(M6 + 6 * t, lop[t], cop[t], Src[t], g, XK + 16 * t, SRC4 + 4 * t);
        or_taustep(s->rhox, XKI, xmu[im], N, Deltau);
        or_centder(Deltau, SRC4, 4, N, SRD);
        or_centder(Deltau, XK, 16, N, XKD);
        double XINT2[4] = { SRC4[4 * (N - 1)], 0.0, 0.0, 0.0 };
        stokes_sweep(N, XK, XKD, SRC4, SRD, Deltau, XINT2);
        for (int q = 0; q < 4; q++) Stokes[q * nmu + im] = XINT2[q];
    }
    free(XK);
}

/* StokesPrfSph (solver.f90:402-538): the same along the rays of s; geometry G [5][nmu][2 ntau] per ray
 * point (SPhi2S, CPhi2S, CPhiS, S2PsiS, C2PsiS); zero incoming Stokes vector for grazing rays */
static void stokes_prf_sph(const or_state *s, const double *M6, const double *lop, const double *cop,
                           const double *Src, const double *G, double *Stokes /*[4][nmu]*/) {
    const int M = 2 * s->ntau, nmu = s->sph_nmu;
    double *XK = (double *)malloc(sizeof(double) * (16 * M * 2 + M * 10));
    double *XKD = XK + 16 * M, *XKI = XKD + 16 * M, *Deltau = XKI + M, *SRC4 = Deltau + M, *SRD = SRC4 + 4 * M;
    for (int im = 0; im < nmu; im++) {
        const int N = s->sph_ntau[im];
        const int *mp = s->sph_map + (size_t)im * M;
        for (int k = 0; k < N; k++) {
            int ia = mp[k] - 1;
            size_t o = (size_t)im * M + k, st = (size_t)nmu * M;
            double g[5] = { G[o], G[st + o], G[2 * st + o], G[3 * st + o], G[4 * st + o] };
            XKI[k] = stokes_point(M6 + 6 * ia, lop[ia], cop[ia], Src[ia], g, XK + 16 * k, SRC4 + 4 * k);
        }
        or_taustep(s->sph_rhox + (size_t)im * M, XKI, 1.0, N, Deltau);
        or_centder(Deltau, SRC4, 4, N, SRD);
        or_centder(Deltau, XK, 16, N, XKD);
        double XINT2[4] = { s->sph_graz[im] ? 0.0 : SRC4[4 * (N - 1)], 0.0, 0.0, 0.0 };
        stokes_sweep(N, XK, XKD, SRC4, SRD, Deltau, XINT2);
        for (int q = 0; q < 4; q++) Stokes[q * nmu + im] = XINT2[q];
    }
    free(XK);
}

/* Field projection of MagRadTranCalc (synth.f90:1931-1993, 2022-2087) for one disk position or ray
 * point: frame 1 and 2 give (gamma, psi) directly (j = the angle index for frame 2), frame 0 projects
 * the stellar-frame field with the local cosine Coslon */
static void field_geometry(int bframe, const double *bfield, int j, double Coslon, double *g) {
    const double d2r = C_PI / 180.0;
    double Sphi, Spsi, Cpsi, Cg;
    if (bframe == 1) {
        Sphi = sin(bfield[1] * d2r); Spsi = sin(bfield[2] * d2r); Cpsi = cos(bfield[2] * d2r); Cg = cos(bfield[1] * d2r);
    } else if (bframe == 2) {
        Sphi = sin(bfield[2 * j + 1] * d2r); Spsi = sin(bfield[2 * j + 2] * d2r);
        Cpsi = cos(bfield[2 * j + 2] * d2r); Cg = cos(bfield[2 * j + 1] * d2r);
    } else {
        double Fldmod = sqrt(bfield[0] * bfield[0] + bfield[1] * bfield[1] + bfield[2] * bfield[2]);
        if (Fldmod > 0.0) {
            double Sinlon = sqrt(1.0 - Coslon * Coslon);
            double Bx = bfield[0] * Sinlon + bfield[2] * Coslon, By = bfield[1];
            double Bz = bfield[0] * Coslon - bfield[2] * Sinlon, Bt = sqrt(Bx * Bx + By * By);
            Sphi = Bt / Fldmod; Cg = Bz / Fldmod;
            if (Bt > 0.0) { Spsi = By / Bt; Cpsi = Bx / Bt; } else { Spsi = 0.0; Cpsi = 1.0; }
        } else { Sphi = 0.0; Cg = 1.0; Spsi = 0.0; Cpsi = 1.0; }
    }
    g[0] = Sphi * Sphi; g[1] = Cg * Cg; g[2] = Cg; g[3] = 2.0 * Spsi * Cpsi; g[4] = Cpsi * Cpsi - Spsi * Spsi;
}

/* MagRadTranCalc (synth.f90:1904-2111): StokesPrfPP with one projection per angle for plane-parallel
 * models; StokesPrfSph with the projection at every ray point for spherical ones */
void or_mag_radtran(const or_state *s, int nmu, const double *xmu, int bframe,
                    const double *bfield, const double *lineopac, const double *maglineopac,
                    double *spz, double *spc) {
    const int sph = s->radius > 0.0, nt = s->ntau, M = 2 * nt;
    double SPhi2[nmu], CPhi2[nmu], CPhi[nmu], S2Psi[nmu], C2Psi[nmu];
    double *G = NULL;
    if (!sph) {
        for (int im = 0; im < nmu; im++) {
            double g[5];
            field_geometry(bframe, bfield, im, xmu[im], g);
            SPhi2[im] = g[0]; CPhi2[im] = g[1]; CPhi[im] = g[2]; S2Psi[im] = g[3]; C2Psi[im] = g[4];
        }
    } else {
        /* frame 1 fills every point of every ray, frames 2 and 0 the points each ray has */
        size_t st = (size_t)nmu * M;
        G = (double *)calloc(5 * st, sizeof(double));
        for (int im = 0; im < nmu; im++) {
            int np = (bframe == 1) ? M : s->sph_ntau[im];
            for (int k = 0; k < np; k++) {
                double g[5];
                field_geometry(bframe, bfield, im, s->sph_muloc[(size_t)im * M + k], g);
                for (int q = 0; q < 5; q++) G[q * st + (size_t)im * M + k] = g[q];
            }
        }
    }
    #pragma omp parallel
    {
        double *Src = (double *)malloc(sizeof(double) * nt);
        #pragma omp for schedule(static)
        for (int iwl = 0; iwl < s->nwl; iwl++) {
            planck(s, s->wave[iwl] + s->wfirst, Src);
            const double *co = s->contopac + (size_t)iwl * nt;
            if (sph) {
                if (spc) or_locprf_sph(s, spc + (size_t)iwl * nmu, co, Src);
                stokes_prf_sph(s, maglineopac + (size_t)iwl * nt * 6, lineopac + (size_t)iwl * nt, co, Src, G,
                               spz + (size_t)iwl * 4 * nmu);
            } else {
                if (spc) or_locprf_pp(spc + (size_t)iwl * nmu, xmu, nmu, co, Src, s->rhox, nt);
                stokes_prf_pp(s, maglineopac + (size_t)iwl * nt * 6, lineopac + (size_t)iwl * nt, co, Src,
                              nmu, xmu, SPhi2, CPhi2, CPhi, S2Psi, C2Psi, spz + (size_t)iwl * 4 * nmu);
            }
        }
        free(Src);
    }
    free(G);
}

/* ---- quadrature and disk integration ---------------------------------------------------- */

static void legendre_p(int N, double Z, double *Pn, double *Pn1, double *Pn2) {
    *Pn1 = 0.0; *Pn = 1.0; *Pn2 = 0.0;
    for (int j = 1; j <= N; j++) {
        *Pn2 = *Pn1; *Pn1 = *Pn;
        *Pn = ((2.0 * j - 1.0) * Z * *Pn1 - (j - 1.0) * *Pn2) / j;
    }
}

/* GaussMu (utils.f90:1367-1417) */
void or_gauss_mu(int quad, int N, double *X, double *W) {
    double Z, Dz, Pn, Pn1, Pn2, F, Df;
    if (quad == 1) {
        for (int i = 1; i <= (N + 1) / 2; i++) {
            Z = cos(C_PI * (i - 0.25) / (N + 0.5));
            for (int it = 1; it <= 100; it++) {
                legendre_p(N, Z, &Pn, &Pn1, &Pn2);
                Df = N * (Z * Pn - Pn1) / (Z * Z - 1.0);
                Dz = Pn / Df; Z = Z - Dz;
                if (fabs(Dz) < 1e-15) break;
            }
            legendre_p(N, Z, &Pn, &Pn1, &Pn2);
            Df = N * (Z * Pn - Pn1) / (Z * Z - 1.0);
            X[i - 1] = 0.5 * (1.0 + Z); X[N - i] = 0.5 * (1.0 - Z);
            W[i - 1] = 1.0 / ((1.0 - Z * Z) * Df * Df); W[N - i] = W[i - 1];
        }
    } else {
        X[0] = 1.0; W[0] = 1.0 / (double)(N * N);
        for (int i = 1; i <= N - 1; i++) {
            Z = cos(2.0 * C_PI * i / (2.0 * N - 1.0));
            for (int it = 1; it <= 100; it++) {
                legendre_p(N, Z, &Pn, &Pn1, &Pn2);
                F = Pn1 - Pn;
                Df = ((N - 1) * (Z * Pn1 - Pn2) - N * (Z * Pn - Pn1)) / (Z * Z - 1.0);
                Dz = F / Df; Z = Z - Dz;
                if (fabs(Dz) < 1e-15) break;
            }
            legendre_p(N, Z, &Pn, &Pn1, &Pn2);
            X[i] = 0.5 * (1.0 + Z);
            W[i] = 0.5 * (1.0 + Z) / ((double)(N * N) * Pn1 * Pn1);
        }
    }
}

/* MuQuadrature (utils.f90:1273-1330) */
int or_mu_quadrature(int quad, int N, double *X, double *W, double *R, int setnodes) {
    if (N == 1) { if (setnodes) X[0] = 1.0; W[0] = 1.0; R[0] = 0.0; R[1] = 1.0; return 0; }
    if (quad == 0) {
        double Rmu[N];
        if (setnodes) for (int i = 1; i <= N; i++) X[i - 1] = sqrt(fmax(0.0, 1.0 - ((double)i - 0.5) / (double)N));
        for (int i = 0; i < N; i++) Rmu[i] = sqrt(1.0 - X[i] * X[i]);
        R[0] = 0.0;
        for (int i = 2; i <= N; i++) R[i - 1] = sqrt(0.5 * (Rmu[i - 2] * Rmu[i - 2] + Rmu[i - 1] * Rmu[i - 1]));
        R[N] = 1.0;
        for (int i = 1; i <= N; i++) W[i - 1] = R[i] * R[i] - R[i - 1] * R[i - 1];
        return 0;
    }
    if (quad == 1 || quad == 2) {
        double Xg[N], Wg[N];
        or_gauss_mu(quad, N, Xg, Wg);
        if (setnodes) for (int i = 0; i < N; i++) X[i] = Xg[i];
        for (int i = 0; i < N; i++) W[i] = 2.0 * Wg[i] * Xg[i];
        R[0] = 0.0;
        for (int i = 1; i <= N - 1; i++) R[i] = sqrt(R[i - 1] * R[i - 1] + W[i - 1]);
        R[N] = 1.0;
        return 0;
    }
    return -1;
}

/* DiskInteg without broadening (convol.f90:111-235) */
void or_disk_integ(int nmu, int nwl, const double *wmu, const double *spl, const double *spc,
                   double *sfl, double *sfc) {
    for (int i = 0; i < nwl; i++) {
        double a = 0.0, c = 0.0;
        for (int im = 0; im < nmu; im++) {
            a = a + spl[(size_t)i * nmu + im] * wmu[im];
            c = c + spc[(size_t)i * nmu + im] * wmu[im];
        }
        sfl[i] = a; sfc[i] = c;
    }
}

/* ---- ZeemanPattern (utils.f90:901-1004) -------------------------------------------------- */
static void merge_shifts(double *G, double *R, int *N, double Tol) {
    double Gm[64], Rm[64]; int Nm = 0;
    for (int i = 0; i < *N; i++) {
        int found = 0;
        for (int k = 0; k < Nm; k++) if (fabs(G[i] - Gm[k]) < Tol) { Rm[k] = Rm[k] + R[i]; found = 1; break; }
        if (!found) { Gm[Nm] = G[i]; Rm[Nm] = R[i]; Nm++; }
    }
    for (int i = 0; i < Nm; i++) { G[i] = Gm[i]; R[i] = Rm[i]; }
    *N = Nm;
}

void or_zeeman_pattern(float jlo, float jup, float glo, float gup, int *npi, float *spi,
                       float *rpi, int *nsig, float *ssig, float *rsig) {
    const double TolZ = 1e-5;
    double Jl = jlo, Ju = jup, Gl = glo, Gu = gup;
    int Nm = (int)lround(2.0 * Ju) + 1;
    double gp[64], rp[64], gs[64], rs[64];
    for (int i = 1; i <= Nm; i++) {
        double m = Ju - (double)(i - 1);
        gp[i - 1] = m * (Gu - Gl);
        gs[i - 1] = m * Gu - (m + 1.0) * Gl;
        if (Jl == Ju) { rp[i - 1] = m * m; rs[i - 1] = 0.25 * (Ju - m) * (Ju + m + 1.0); }
        else if (Jl > Ju) { rp[i - 1] = (Ju + 1.0) * (Ju + 1.0) - m * m; rs[i - 1] = 0.25 * (Ju + m + 1.0) * (Ju + m + 2.0); }
        else { rp[i - 1] = Ju * Ju - m * m; rs[i - 1] = 0.25 * (Ju - m) * (Ju - m - 1.0); }
    }
    for (int i = 0; i < Nm; i++) { if (fabs(gp[i]) < TolZ) gp[i] = 0.0; if (fabs(gs[i]) < TolZ) gs[i] = 0.0; }
    int Np = 0, Ns = 0;
    for (int i = 0; i < Nm; i++) if (fabs(rp[i]) > TolZ) { gp[Np] = gp[i]; rp[Np] = rp[i]; Np++; }
    for (int i = 0; i < Nm; i++) if (fabs(rs[i]) > TolZ) { gs[Ns] = -gs[i]; rs[Ns] = rs[i]; Ns++; }
    merge_shifts(gp, rp, &Np, TolZ);
    merge_shifts(gs, rs, &Ns, TolZ);
    double sm = 0.0; for (int i = 0; i < Np; i++) sm = sm + rp[i];
    if (sm > 0.0) for (int i = 0; i < Np; i++) rp[i] = rp[i] / sm;
    sm = 0.0; for (int i = 0; i < Ns; i++) sm = sm + rs[i];
    if (sm > 0.0) for (int i = 0; i < Ns; i++) rs[i] = rs[i] / sm;
    *npi = Np; *nsig = Ns;
    for (int i = 0; i < Np; i++) { spi[i] = (float)gp[i]; rpi[i] = (float)rp[i]; }
    for (int i = 0; i < Ns; i++) { ssig[i] = (float)gs[i]; rsig[i] = (float)rs[i]; }
}


/* ---- disk integration with broadening (convol.f90:67-300) ------------------------------------ */

/* SemiArea (utils.f90:1435-1445): area under a semicircle of radius R from -R to V */
static double semi_area(double R, double V) {
    if (R <= 0.0) return 0.0;
    double X = fmax(-R, fmin(R, V));
    return 0.5 * (X * sqrt(fmax(0.0, (R - X) * (R + X))) + R * R * asin(X / R));
}

/* out(i) = sum_j T(i + j - 1 - h) kern(j), T the spectrum padded with its end values, h = (n - 1) / 2;
 * in/out with stride st between wavelengths */
static void conv_padded(int nwl, const double *in, int st_in, const double *kern, int n, double *out) {
    int h = (int)((n - 1.0) / 2.0);
    for (int i = 0; i < nwl; i++) {
        double sm = 0.0;
        for (int j = 0; j < n; j++) {
            int m = i + j - h;
            m = m < 0 ? 0 : (m >= nwl ? nwl - 1 : m);
            sm = sm + in[(size_t)m * st_in] * kern[j];
        }
        out[i] = sm;
    }
}

static int gauss_kernel(double sig, int nmax, double *k) {   /* returns Ng = 2 j + 1 */
    int j = (int)(10.0 * sig);
    int lim = (int)((nmax - 3.0) / 2.0);
    if (j > lim) j = lim;
    if (j < 3) j = 3;
    int ng = 2 * j + 1;
    double norm = 0.0;
    for (int i = 1; i <= ng; i++) {
        double arg = fmax(-20.0, -0.5 * ((i - j - 1) / sig) * ((i - j - 1) / sig));
        k[i - 1] = exp(arg);
        norm = norm + k[i - 1];
    }
    for (int i = 0; i < ng; i++) k[i] = k[i] / norm;
    return ng;
}

void or_convol_gau(int nw, double *S, double sigma_pix) {
    double sig = sigma_pix / (2.0 * sqrt(2.0 * log(2.0)));
    int j = (int)(10.0 * sig), lim = (int)((nw - 3.0) / 2.0);
    if (j > lim) j = lim;
    if (j < 3) j = 3;
    double *k = (double *)malloc(sizeof(double) * (2 * j + 1));
    double *T = (double *)malloc(sizeof(double) * nw);
    int ng = 2 * j + 1;
    double norm = 0.0;
    for (int i = 1; i <= ng; i++) {
        double arg = fmax(-20.0, -0.5 * ((i - j - 1) / sig) * ((i - j - 1) / sig));
        k[i - 1] = exp(arg);
        norm = norm + k[i - 1];
    }
    for (int i = 0; i < ng; i++) k[i] = k[i] / norm;
    memcpy(T, S, sizeof(double) * nw);
    conv_padded(nw, T, 1, k, ng, S);
    free(k); free(T);
}

void or_disk_integ_conv(int nmu, int nwl, const double *xmu, const double *wmu, const double *radii, double dv,
                        double vsini, double vmacro, double gsig, const double *spl, const double *spc,
                        double *sfl, double *sfc) {
    double sigma = vmacro / dv / sqrt(2.0);
    int nmk = (int)(10.0 * sigma), lim = (int)((nwl - 3) / 2);
    if (nmk > lim) nmk = lim;
    if (nmk < 3) nmk = 3;
    int nm = 2 * nmk + 1;
    int nrk_max = 2 * (int)(vsini / dv) + 3;
    double *rk = (double *)malloc(sizeof(double) * (nrk_max + 2));
    double *mk = (double *)malloc(sizeof(double) * nm), *mr = (double *)malloc(sizeof(double) * nm);
    double *mt = (double *)malloc(sizeof(double) * nm);
    double *siL = (double *)malloc(sizeof(double) * nwl), *siC = (double *)malloc(sizeof(double) * nwl);
    double *tL = (double *)malloc(sizeof(double) * nwl), *tC = (double *)malloc(sizeof(double) * nwl);
    for (int i = 0; i < nwl; i++) { sfl[i] = 0.0; sfc[i] = 0.0; }
    for (int im = 0; im < nmu; im++) {
        for (int i = 0; i < nwl; i++) { siL[i] = spl[(size_t)i * nmu + im]; siC[i] = spc[(size_t)i * nmu + im]; }
        if (vsini > 0.0) {
            double R1 = vsini * radii[im], R2 = vsini * radii[im + 1];
            int nrk = 2 * (int)(R2 / dv) + 3;
            double norm = 0.0;
            for (int i = 1; i <= nrk; i++) {
                double V = fabs(dv * (i - 1 - (nrk - 1) / 2));
                rk[i - 1] = semi_area(R2, V + 0.5 * dv) - semi_area(R2, V - 0.5 * dv) -
                            semi_area(R1, V + 0.5 * dv) + semi_area(R1, V - 0.5 * dv);
                norm = norm + rk[i - 1];
            }
            for (int i = 0; i < nrk; i++) rk[i] = rk[i] / norm;
            if (R2 > 0.5 * dv) {
                memcpy(tL, siL, sizeof(double) * nwl); memcpy(tC, siC, sizeof(double) * nwl);
                conv_padded(nwl, tL, 1, rk, nrk, siL);
                conv_padded(nwl, tC, 1, rk, nrk, siC);
            }
        }
        if (vmacro > 0.0) {
            double sigr = sigma * xmu[im], sigt = sigma * sqrt(1.0 - xmu[im] * xmu[im]);
            double nr = 0.0, nt = 0.0;
            for (int i = 1; i <= nm; i++) {
                if (sigr > 0.0) {
                    double a = fmax(-20.0, -0.5 * ((i - nmk - 1) / sigr) * ((i - nmk - 1) / sigr));
                    mr[i - 1] = exp(a); nr = nr + mr[i - 1];
                }
                if (sigt > 0.0) {
                    double a = fmax(-20.0, -0.5 * ((i - nmk - 1) / sigt) * ((i - nmk - 1) / sigt));
                    mt[i - 1] = exp(a); nt = nt + mt[i - 1];
                }
            }
            for (int i = 0; i < nm; i++) {
                mr[i] = sigr > 0.0 ? mr[i] / nr : (i == nmk ? 1.0 : 0.0);
                mt[i] = sigt > 0.0 ? mt[i] / nt : (i == nmk ? 1.0 : 0.0);
                mk[i] = 0.5 * mr[i] + 0.5 * mt[i];
            }
            memcpy(tL, siL, sizeof(double) * nwl); memcpy(tC, siC, sizeof(double) * nwl);
            conv_padded(nwl, tL, 1, mk, nm, siL);
            conv_padded(nwl, tC, 1, mk, nm, siC);
        }
        for (int i = 0; i < nwl; i++) { sfl[i] = sfl[i] + siL[i] * wmu[im]; sfc[i] = sfc[i] + siC[i] * wmu[im]; }
    }
    if (gsig > 0.0) { or_convol_gau(nwl, sfl, gsig); or_convol_gau(nwl, sfc, gsig); }
    free(rk); free(mk); free(mr); free(mt); free(siL); free(siC); free(tL); free(tC);
}


/* ---- the elemental routines on their own ------------------------------------------------------- */
void or_xline_setup(const or_state *s, const or_lines *L, long i, int list_type, or_xcoef *xc) {
    xcoef XC;
    xline_setup(s, L, i, L->wl[i] - s->wfirst, input_flags(L, i, list_type), &XC);
    xc->WaveL = XC.WaveL; xc->Hnux = XC.Hnux; xc->Elo = XC.Elo; xc->Gf = XC.Gf; xc->Grad = XC.Grad;
    xc->Xmass = XC.Xmass; xc->Cqst = XC.Cqst; xc->Qdiv = XC.Qdiv; xc->Cvdw = XC.Cvdw;
    xc->AboPre = XC.AboPre; xc->AboVbc = XC.AboVbc; xc->AboExp = XC.AboExp;
    xc->IxPF = XC.IxPF; xc->MdQst = XC.MdQst; xc->MdVdw = XC.MdVdw; xc->IxHe = XC.IxHe;
}

void or_xline_depth(const or_state *s, int t, const or_xcoef *xc, double *lincop, double *linvvgt,
                    double *linavgt) {
    xcoef XC;
    XC.WaveL = xc->WaveL; XC.Hnux = xc->Hnux; XC.Elo = xc->Elo; XC.Gf = xc->Gf; XC.Grad = xc->Grad;
    XC.Xmass = xc->Xmass; XC.Cqst = xc->Cqst; XC.Qdiv = xc->Qdiv; XC.Cvdw = xc->Cvdw;
    XC.AboPre = xc->AboPre; XC.AboVbc = xc->AboVbc; XC.AboExp = xc->AboExp;
    XC.IxPF = xc->IxPF; XC.MdQst = xc->MdQst; XC.MdVdw = xc->MdVdw; XC.IxHe = xc->IxHe;
    xline_depth(s, t, &XC, lincop, linvvgt, linavgt);
}

void or_lineopacity1(const or_state *s, const double *wlcent, const int *flags, const int *ileft,
                     const int *iright, const double *lincop, const double *linvvgt, const double *linavgt,
                     double Wl, int l1, int l2, int iwl, long loff, double *linop) {
    or_voigt_init();                       /* VgtTab and its damping nodes, built once */
    int nt = s->ntau;
    for (int t = 0; t < nt; t++) linop[t] = 0.0;
    for (long il = l1; il <= l2; il++) {
        int f = flags[il - 1];
        if ((f & 1) || (f & 8) || iwl < ileft[il - 1] || iwl > iright[il - 1]) continue;
        int ihe = (f >> 8) & 255;
        double dWl0 = Wl - wlcent[il - 1];
        const double *c = lincop + (il - loff - 1) * nt, *v = linvvgt + (il - loff - 1) * nt,
                     *a = linavgt + (il - loff - 1) * nt;
        for (int t = 0; t < nt; t++) {
            double dWl = dWl0;
            if (ihe > 0) dWl = dWl0 - s->heshf[(ihe - 1) * nt + t];
            double V = dWl * v[t];
            linop[t] = linop[t] + or_hvoigt(a[t], V) * c[t];
        }
    }
    if (s->motype == 1) for (int t = 0; t < nt; t++) linop[t] = linop[t] / s->contopac_std[t];
}

void or_lineopacity2(const or_state *s, double Wl, double wlcent, int flag, int ileft, int iright, int iwl,
                     const double *lincop, const double *linvvgt, const double *linavgt, double *linop) {
    or_voigt_init();
    linework W;
    long orig = 0;
    W.n = 1; W.wlcent = &wlcent; W.flag = &flag; W.ileft = &ileft; W.iright = &iright; W.orig = &orig;
    lineopacity2(s, Wl, &W, 0, iwl, lincop, linvvgt, linavgt, linop);
}

void or_mag_lineopacity1(const or_state *s, const double *wlcent, const int *flags, const int *ileft,
                         const int *iright, const double *lincop, const double *linvvgt, const double *linavgt,
                         const int *npi, const int *nsi, const long *pi_off, const long *si_off,
                         const float *splpi, const float *strpi, const float *splsi, const float *strsi,
                         double Wl, int l1, int l2, int iwl, long loff, double *M) {
    or_fvoigt_init();                      /* FvTab and its damping nodes, built once */
    int nt = s->ntau;
    for (int q = 0; q < 6 * nt; q++) M[q] = 0.0;
    for (long iline = l1; iline <= l2; iline++) {
        int f = flags[iline - 1];
        if ((f & 1) || (f & 8) || iwl < ileft[iline - 1] || iwl > iright[iline - 1]) continue;
        long il = iline - loff - 1;
        int ihe = (f >> 8) & 255;
        const long i = iline - 1;
        for (int t = 0; t < nt; t++) {
            vline FL = fvline_init(linavgt[il * nt + t]);
            double Xn = lincop[il * nt + t], sc = linvvgt[il * nt + t];
            double Vbase = (Wl - wlcent[i]) * sc;
            if (ihe > 0) Vbase = Vbase - s->heshf[(ihe - 1) * nt + t] * sc;
            double *m = M + 6 * t, V, Vg, Fv, Str;
            for (int k = 0; k < npi[i]; k++) {
                V = Vbase - (double)splpi[pi_off[i] + k] * sc;
                fvoigt_line(FL, V, &Vg, &Fv);
                Str = Xn * (double)strpi[pi_off[i] + k];
                m[0] = m[0] + Str * Vg; m[3] = m[3] + Str * Fv;
            }
            int Nsh = nsi[i] / 2;
            for (int k = 0; k < Nsh; k++) {
                V = Vbase - (double)splsi[si_off[i] + k] * sc;
                fvoigt_line(FL, V, &Vg, &Fv);
                Str = Xn * (double)strsi[si_off[i] + k];
                m[1] = m[1] + Str * Vg; m[4] = m[4] + Str * Fv;
            }
            for (int k = Nsh; k < nsi[i]; k++) {
                V = Vbase - (double)splsi[si_off[i] + k] * sc;
                fvoigt_line(FL, V, &Vg, &Fv);
                Str = Xn * (double)strsi[si_off[i] + k];
                m[2] = m[2] + Str * Vg; m[5] = m[5] + Str * Fv;
            }
        }
    }
    if (s->motype == 1)
        for (int t = 0; t < nt; t++)
            for (int q = 0; q < 6; q++) M[6 * t + q] = M[6 * t + q] / s->contopac_std[t];
}

double or_analytic_window(const or_state *s, int flag, const double *lincop, const double *linvvgt,
                          const double *linavgt, const double *contopac) {
    or_voigt_init();
    return analytic_window(s, flag, lincop, linvvgt, linavgt, contopac);
}

void or_stokes_prf_pp(const or_state *s, const double *m6, const double *lop, const double *cop,
                      const double *src, int nmu, const double *xmu, const double *sphi2, const double *cphi2,
                      const double *cphi, const double *s2psi, const double *c2psi, double *stokes) {
    stokes_prf_pp(s, m6, lop, cop, src, nmu, xmu, sphi2, cphi2, cphi, s2psi, c2psi, stokes);
}
