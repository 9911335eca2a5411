// fsg_mag.cu -- magnetic path: MagLineopCalc (Zeeman-split Faraday-Voigt opacity into the six
// profiles) and MagRadTranCalc (Stokes DELO-Bezier solver, plane-parallel and spherical).  Built -fmad=false:
// FP64 throughout, in the reference's operation order.
//
//   k_mag_center    MagLineopCalc central pass (synth.f90:1182-1275), one warp per line: Zeeman shifts scaled to
//                   FP32 (Kz |B| lambda^2, synth.f90:1193-1194), centre test (LineOpacity2),
//                   doubling search with MagLineOpacity2 and RefineIdx bisection
//                   (opacity.f90:468-520, 611-675)
//   k_mag_accum     MagLineOpacity1 per wavelength (opacity.f90:391-464)
//   k_mag_wide      MagLineOpacity3 for the wide lines, in line order (synth.f90:1341-1361)
//   k_stokes_thr    StokesPrfPP (solver.f90:265-394) + Solve4x4 (solver.f90:541-588), one thread per
//                   (wavelength, angle); k_stokes_flux the Stokes-I flux quadrature
//   k_stokes_sph    StokesPrfSph (solver.f90:402-538) along the rays of a spherical model, one thread per
//                   (wavelength, ray)
#include "fsg_fp64.cuh"

#include <algorithm>
#include <math.h>
#include <string.h>
#include <vector>

// MagLineOpacity2 at one wavelength, max over depths of LineOpac/ContOpacL (opacity.f90:468-520)
// over the depths t0, t0 + tstep, ... (a lane's share when a warp takes the line)
__device__ double mag_lineop2_max(const AtmView &A, const XCoef &XC, double Wl, double wlc, int ihe,
                                  const ZView &Z, int64_t i, int iwl, double dW, const float *vtab,
                                  const double *anode, const double *aida, int t0 = 0, int tstep = 1) {
    const int nt = A.ntau;
    double mx = -1.0e308;
    const int np = Z.npi[i], ns = Z.nsi[i];
    const float *spi = Z.splpi + Z.pi_off[i], *ssi = Z.splsi + Z.si_off[i];
    const float *rpi = Z.strpi + Z.pi_off[i], *rsi = Z.strsi + Z.si_off[i];
    double dWl0 = Wl - wlc;
    for (int t = t0; t < nt; t += tstep) {
        double cop, vv, av;
        xline_depth(A, t, XC, &cop, &vv, &av);
        double dWl = dWl0;
        if (ihe > 0) dWl = dWl0 - A.heshf[(ihe - 1) * nt + t];
        VLine64 VL = vline64(anode, aida, av);
        double Pp = 0.0, Ps = 0.0;
        for (int k = 0; k < np; k++) Pp = Pp + (double)rpi[k] * hvoigt_line64(vtab, VL, (dWl - (double)spi[k]) * vv);
        for (int k = 0; k < ns; k++) Ps = Ps + (double)rsi[k] * hvoigt_line64(vtab, VL, (dWl - (double)ssi[k]) * vv);
        double lo = fmax(0.5 * Ps, 0.5 * Pp + 0.25 * Ps) * cop;
        if (A.motype == 1) lo = lo / A.contstd[t];
        mx = fmax(mx, lo / cont_center(A, iwl, dW, t));
    }
    return mx;
}

__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// MagLineOpacity2's maximum over depths (opacity.f90:468-520), the lanes of a warp over the depths
__device__ __forceinline__ double mag_lineop2_max_warp(const AtmView &A, const XCoef &XC, double Wl, double wlc,
                                                       int ihe, const ZView &Z, int64_t i, int iwl, double dW,
                                                       const float *vtab, const double *anode, const double *aida,
                                                       int lane) {
    return warp_max(mag_lineop2_max(A, XC, Wl, wlc, ihe, Z, i, iwl, dW, vtab, anode, aida, lane, 32));
}

// Magnetic central pass, one warp per line: the lanes share the depth loops of the centre test and of
// every MagLineOpacity2 evaluation of the window search (maxima over depths, so the lanes' partial
// maxima combine exactly), the search itself is warp-uniform.
__global__ void k_mag_center(AtmView A, LineView L, ZView Z, double Bsplit, const float *__restrict__ vtab,
                             const double *__restrict__ anode, const double *__restrict__ aida,
                             int32_t *flags, int32_t *ileft, int32_t *iright, unsigned long long *nkeep) {
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= L.n) return;                                // whole warps leave together
    const int nt = A.ntau;
    int f = 0;
    if (L.ismol && L.ismol[i]) f |= FSG_F_MOL;
    if (L.gvdw[i] > 10.0f) f |= FSG_F_ABO;
    double wlc = L.wl[i] - A.wfirst;
    double w = wlc + A.wfirst;
    // scale the pattern by Kz |B| lambda^2, rounded to FP32 (synth.f90:1193-1194)
    const int np = Z.npi[i], ns = Z.nsi[i];
    double smx_pi = -3.4028234663852886e38, smx_si = -3.4028234663852886e38;
    for (int k = lane; k < np; k += 32) {
        float v = (float)((double)Z.rawpi[Z.pi_off[i] + k] * Bsplit * (w * w));
        Z.splpi[Z.pi_off[i] + k] = v;
        smx_pi = fmax(smx_pi, fabs((double)v));
    }
    for (int k = lane; k < ns; k += 32) {
        float v = (float)((double)Z.rawsi[Z.si_off[i] + k] * Bsplit * (w * w));
        Z.splsi[Z.si_off[i] + k] = v;
        smx_si = fmax(smx_si, fabs((double)v));
    }
    const double SplMax = fmax(warp_max(smx_si), warp_max(smx_pi));
    __syncwarp();                                        // every lane's scaled shifts are visible below
    XCoef XC;
    xline_setup(A, L, i, wlc, f, &XC);
    if (XC.IxHe > 0) f |= (XC.IxHe << 8);
    int ihe = XC.IxHe;
    int iwl = waveidx(A, wlc);
    double dW = (wlc - A.wave[iwl - 1]) / (A.wave[iwl] - A.wave[iwl - 1]);
    // non-magnetic centre opacity (synth.f90:1215-1224)
    double mx = -1.0e308;
    for (int t = lane; t < nt; t += 32) {
        double cop, vv, av;
        xline_depth(A, t, XC, &cop, &vv, &av);
        double dWl = 0.0;
        if (ihe > 0) dWl = 0.0 - A.heshf[(ihe - 1) * nt + t];
        double lo = hvoigt64(vtab, anode, aida, av, dWl * vv) * cop;
        if (A.motype == 1) lo = lo / A.contstd[t];
        mx = fmax(mx, lo / cont_center(A, iwl, dW, t));
    }
    mx = warp_max(mx);
    int il = 1, ir = A.nwl;
    if (mx < A.epsopac) f |= FSG_F_WEAK;
    else {
        // doubling search (synth.f90:1233-1272)
        for (int idw = 0; idw < 64; idw++) {
            double dWo = (0.2 * ldexp(1.0, idw)) * (wlc + A.wfirst) / 5e3;
            double Wl = wlc + SplMax + dWo;
            double m2 = mag_lineop2_max_warp(A, XC, Wl, wlc, ihe, Z, i, iwl, dW, vtab, anode, aida, lane);
            if (m2 < A.epsopac) {
                // RefineIdx (opacity.f90:611-675), magnetic branch
                int isw, ikw;
                if (wlc > 0.5 * (A.wave[0] + A.wave[A.nwl - 1])) { isw = -1; ikw = 0; }
                else { isw = 1; ikw = 1; }
                int ia, ib;
                if (idw == 0) ia = waveidx(A, wlc + (double)isw * SplMax) + ikw;
                else {
                    double d1 = (0.2 * ldexp(1.0, idw - 1)) * (wlc + A.wfirst) / 5e3;
                    ia = waveidx(A, wlc + (double)isw * (SplMax + d1)) + ikw;
                }
                ib = waveidx(A, wlc + (double)isw * (SplMax + dWo)) + ikw;
                for (int it = 0; it < 64 && abs(ia - ib) > 1; it++) {
                    int im = (ia + ib) / 2;
                    double m3 = mag_lineop2_max_warp(A, XC, A.wave[im - 1], wlc, ihe, Z, i, iwl, dW, vtab, anode,
                                                     aida, lane);
                    if (m3 < A.epsopac) ib = im; else ia = im;
                }
                if (isw == 1) { ir = ia; il = waveidx(A, 2.0 * wlc - A.wave[ia - 1]); }
                else { il = ia; ir = waveidx(A, 2.0 * wlc - A.wave[ia - 1]) + 1; }
                break;
            } else if (wlc - SplMax - dWo < A.wave[0] && wlc + SplMax + dWo > A.wave[A.nwl - 1]) break;
        }
    }
    if (lane == 0) {
        flags[i] = f; ileft[i] = il; iright[i] = ir;
        if (!(f & FSG_F_WEAK)) atomicAdd(nkeep, 1ull);
    }
}

// six profiles of one line at one wavelength for depth t (MagLineOpacity1/3 inner loops)
__device__ __forceinline__ void mag_profiles_t(const AtmView &A, int t, double Wl, double wlc, int ihe,
                                               const ZView &Z, int64_t i, double cop, double vv, double av,
                                               const float2 *fvtab, const double *anode, const double *aida,
                                               double *m) {
    VLine64 FL = vline64(anode, aida, av);
    double Xn = cop, sc = vv, Vbase = (Wl - wlc) * sc;
    if (ihe > 0) Vbase = Vbase - A.heshf[(ihe - 1) * A.ntau + t] * sc;
    const int np = Z.npi[i], ns = Z.nsi[i];
    const float *spi = Z.splpi + Z.pi_off[i], *ssi = Z.splsi + Z.si_off[i];
    const float *rpi = Z.strpi + Z.pi_off[i], *rsi = Z.strsi + Z.si_off[i];
    for (int k = 0; k < np; k++) {
        double V = Vbase - (double)spi[k] * sc, Vg, Fv;
        fvoigt_line64(fvtab, FL, V, &Vg, &Fv);
        double Str = Xn * (double)rpi[k];
        m[0] = m[0] + Str * Vg; m[3] = m[3] + Str * Fv;
    }
    int Nsh = ns / 2;
    for (int k = 0; k < Nsh; k++) {
        double V = Vbase - (double)ssi[k] * sc, Vg, Fv;
        fvoigt_line64(fvtab, FL, V, &Vg, &Fv);
        double Str = Xn * (double)rsi[k];
        m[1] = m[1] + Str * Vg; m[4] = m[4] + Str * Fv;
    }
    for (int k = Nsh; k < ns; k++) {
        double V = Vbase - (double)ssi[k] * sc, Vg, Fv;
        fvoigt_line64(fvtab, FL, V, &Vg, &Fv);
        double Str = Xn * (double)rsi[k];
        m[2] = m[2] + Str * Vg; m[5] = m[5] + Str * Fv;
    }
}

// MagLineOpacity1 (opacity.f90:391-464): one warp per wavelength, lanes stride the depths.
__global__ void k_mag_accum(AtmView A, const double *__restrict__ wl, ZView Z, const int64_t *__restrict__ zmap,
                            int iwl1, int iwl2, const int *__restrict__ lstart, const int *__restrict__ lstop,
                            const int32_t *__restrict__ flags, const int32_t *__restrict__ ileft,
                            const int32_t *__restrict__ iright, int64_t loff, const double3 *__restrict__ p64,
                            const float2 *__restrict__ fvtab, const double *__restrict__ anode,
                            const double *__restrict__ aida, double *mlo, double *evals) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    int iwl = iwl1 + warp;
    if (iwl > iwl2) return;
    const int nt = A.ntau;
    double Wl = A.wave[iwl - 1];
    double cnt = 0.0;
    for (int t0 = 0; t0 < nt; t0 += 32) {
        int t = t0 + lane;
        double m[6] = { 0, 0, 0, 0, 0, 0 };
        for (int il = lstart[iwl - 1]; il <= lstop[iwl - 1]; il++) {
            int f = flags[il - 1];
            if ((f & FSG_F_WEAK) || (f & FSG_F_WIDE) || iwl < ileft[il - 1] || iwl > iright[il - 1]) continue;
            if (t < nt) {
                double3 p = p64[(size_t)(il - 1 - loff) * nt + t];
                mag_profiles_t(A, t, Wl, wl[il - 1] - A.wfirst, (f >> 8) & 255, Z, zmap[il - 1], p.x, p.y, p.z,
                               fvtab, anode, aida, m);
            }
            if (t0 == 0) cnt += 1.0;
        }
        if (t < nt) {
            double *dst = mlo + ((size_t)(iwl - 1) * nt + t) * 6;
            for (int q = 0; q < 6; q++) {
                double v = m[q];
                if (A.motype == 1) v = v / A.contstd[t];
                dst[q] = dst[q] + v;
            }
        }
    }
    if (lane == 0 && cnt > 0.0) atomicAdd(evals, cnt * nt);
}

// MagLineOpacity3 over the wide lines, in line order, one warp per wavelength
__global__ void k_mag_wide(AtmView A, const double *__restrict__ wl, ZView Z, const int64_t *__restrict__ zmap,
                           int nwide, const int64_t *__restrict__ widx, const int32_t *__restrict__ flags,
                           const int32_t *__restrict__ ileft, const int32_t *__restrict__ iright,
                           const double3 *__restrict__ pw, const float2 *__restrict__ fvtab,
                           const double *__restrict__ anode, const double *__restrict__ aida, double *mlo) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    int iwl = 1 + warp;
    if (iwl > A.nwl) return;
    const int nt = A.ntau;
    double Wl = A.wave[iwl - 1];
    for (int q = 0; q < nwide; q++) {
        int64_t il = widx[q];
        if (iwl < ileft[il] || iwl > iright[il]) continue;
        int ihe = (flags[il] >> 8) & 255;
        for (int t = lane; t < nt; t += 32) {
            double m[6] = { 0, 0, 0, 0, 0, 0 };
            double3 p = pw[(size_t)q * nt + t];
            mag_profiles_t(A, t, Wl, wl[il] - A.wfirst, ihe, Z, zmap[il], p.x, p.y, p.z, fvtab, anode, aida, m);
            double *dst = mlo + ((size_t)(iwl - 1) * nt + t) * 6;
            for (int r = 0; r < 6; r++) {
                double v = m[r];
                if (A.motype == 1) v = v / A.contstd[t];
                dst[r] = dst[r] + v;
            }
        }
    }
}

__global__ void k_mag_params(AtmView A, LineView L, int64_t n, const int64_t *__restrict__ list, int64_t off,
                             const int32_t *__restrict__ flags, double3 *p) {
    int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int64_t i = list ? list[q] : off + q;
    int f = flags[i];
    if (f & FSG_F_WEAK) return;
    XCoef XC;
    xline_setup(A, L, i, L.wl[i] - A.wfirst, f, &XC);
    for (int t = 0; t < A.ntau; t++) {
        double cop, vv, av;
        xline_depth(A, t, XC, &cop, &vv, &av);
        p[(size_t)q * A.ntau + t] = make_double3(cop, vv, av);
    }
}

// ================================================================================================
// Stokes solvers (solver.f90:265-538).  The per-depth propagation data are the 6 distinct elements of
// the normalised 4x4 matrix, the source vector, their CentDer derivatives and the TauStep steps;
// CentDer of the full matrix is taken through its 6 distinct elements (CentDer commutes with negation
// exactly and maps the zero diagonal to zero).  k_stokes_thr (plane-parallel) and k_stokes_sph (spherical
// rays of up to 2 ntau points) give every thread one (wavelength, angle) sweep over per-thread work
// arrays in global memory.
// ================================================================================================
#define STK_FIELDS 22   // per depth: PhiI, 6 K, 6 KD, 4 SRC4, 4 SRD, Deltau

__device__ __forceinline__ void centder_pt(const double *D, const double *Y, int stride, int N, int k, double *out) {
    // Yp at 0-based depth k for one component with values Y[t * stride]
    if (k == 0) { *out = (Y[stride] - Y[0]) / D[0]; return; }
    if (k == N - 1) { *out = (Y[(N - 1) * stride] - Y[(N - 2) * stride]) / D[N - 2]; return; }
    double Dx = D[k - 1], Dx1 = D[k];
    double InvDx = 1.0 / Dx, InvDx1 = 1.0 / Dx1;
    double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0, Lambda1 = 1.0 - Lambda;
    double Der = (Y[k * stride] - Y[(k - 1) * stride]) * InvDx, Der1 = (Y[(k + 1) * stride] - Y[k * stride]) * InvDx1;
    *out = (Der * Der1 > 0.0) ? (Der / (Lambda * Der1 + Lambda1 * Der)) * Der1 : 0.0;
}

// full 4x4 propagation matrix from its 6 distinct elements (solver.f90:311-326), column-major
__device__ __forceinline__ void build_k(const double *e, double *K) {
    double PhiQ = e[0], PhiU = e[1], PhiV = e[2], PsiQ = e[3], PsiU = e[4], PsiV = e[5];
    K[0] = 0.0;   K[4] = PhiQ;  K[8] = PhiU;   K[12] = PhiV;
    K[1] = PhiQ;  K[5] = 0.0;   K[9] = PsiV;   K[13] = -PsiU;
    K[2] = PhiU;  K[6] = -PsiV; K[10] = 0.0;   K[14] = PsiQ;
    K[3] = PhiV;  K[7] = PsiU;  K[11] = -PsiQ; K[15] = 0.0;
}

__device__ void solve4x4(const double *A, const double *B, double *X) {
    double M[16], R[4];
    for (int q = 0; q < 16; q++) M[q] = A[q];
    for (int q = 0; q < 4; q++) R[q] = B[q];
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

// The DELO-Bezier sweep of StokesPrfPP / StokesPrfSph (solver.f90:341-390, 486-534) over the N points of
// one ray, run by one thread from the per-point fields in shared memory (field-major, leading dimension
// ld): Kv / KD the 6 distinct propagation elements and their derivatives, SRC4 / SRD the source vector
// and its derivative, Dt the optical-depth steps.  XINT2 holds the boundary Stokes vector on entry and
// the emergent one on return.
__device__ void stokes_sweep(int N, int ld, const double *Kv, const double *KD, const double *SRC4,
                             const double *SRD, const double *Dt, double *XINT2, size_t es = 1) {
    double K1[16], K0[16], KD0[16], XKA[16], XKB[16], QA[16], QB[16], AA[16], e6[6], d6[6], XINT1[4];
    for (int q = 0; q < 6; q++) { e6[q] = Kv[(q * ld + N - 1) * es]; d6[q] = KD[(q * ld + N - 1) * es]; }
    build_k(e6, K0); build_k(d6, KD0);
    for (int j = 0; j < 4; j++) for (int i = 0; i < 4; i++) {
        double acc = 0.0;
        for (int q = 0; q < 4; q++) acc = acc + K0[i + 4 * q] * K0[q + 4 * j];
        XKB[i + 4 * j] = acc + KD0[i + 4 * j];
    }
    for (int q = 0; q < 16; q++) K1[q] = K0[q];         // XK at k1
    for (int k = N - 2; k >= 0; k--) {
        int k1 = k + 1;
        double Dtau = Dt[k * es], Dtau05 = 0.5 * Dtau, Eps, Alpha, Beta, Gamma;
        delo_coef(Dtau, Eps, Alpha, Beta, Gamma);
        Gamma = Gamma * 0.5;
        for (int q = 0; q < 6; q++) { e6[q] = Kv[(q * ld + k) * es]; d6[q] = KD[(q * ld + k) * es]; }
        build_k(e6, K0); build_k(d6, KD0);
        for (int q = 0; q < 16; q++) XKA[q] = XKB[q];
        for (int j = 0; j < 4; j++) for (int i = 0; i < 4; i++) {
            double acc = 0.0;
            for (int q = 0; q < 4; q++) acc = acc + K0[i + 4 * q] * K0[q + 4 * j];
            XKB[i + 4 * j] = acc + KD0[i + 4 * j];
        }
        for (int j = 0; j < 4; j++) for (int i = 0; i < 4; i++) {
            int e = i + 4 * j;
            QA[e] = Dtau05 * XKA[e] + (Dtau05 - 1.0) * K1[e];
            QB[e] = -(Dtau05 * XKB[e]) - (Dtau05 + 1.0) * K0[e];
            AA[e] = ((i == j) ? 1.0 : 0.0) + Alpha * K0[e] - Gamma * QB[e];
        }
        double GD = Gamma * Dtau05;
        for (int i = 0; i < 4; i++) {
            double m1 = 0.0, m2 = 0.0, m3 = 0.0, m4 = 0.0;
            for (int q = 0; q < 4; q++) {
                m1 = m1 + K1[i + 4 * q] * XINT2[q];
                m2 = m2 + QA[i + 4 * q] * XINT2[q];
                m3 = m3 + K1[i + 4 * q] * SRC4[(q * ld + k1) * es];
                m4 = m4 + K0[i + 4 * q] * SRC4[(q * ld + k) * es];
            }
            XINT1[i] = Eps * XINT2[i] - Beta * m1 + Gamma * m2 + (Beta + Gamma) * SRC4[(i * ld + k1) * es]
                     - GD * m3 + (Alpha + Gamma) * SRC4[(i * ld + k) * es] + GD * m4
                     + GD * (SRD[(i * ld + k) * es] - SRD[(i * ld + k1) * es]);
        }
        solve4x4(AA, XINT1, XINT2);
        for (int q = 0; q < 16; q++) K1[q] = K0[q];
    }
}

// propagation matrix elements normalised by PhiI and the source vector at one point (solver.f90:296-330,
// 431-465): m = MagLineOpac(:, ia), g = (SPhi2, CPhi2, CPhi, S2Psi, C2Psi); returns PhiI
__device__ __forceinline__ double stokes_point(const double *m, double lop, double cop, double sr, const double *g,
                                               double *e6, double *s4) {
    double Php = m[0], Phb = m[1], Phr = m[2], Psp = m[3], Psb = m[4], Psr = m[5];
    double SPhi2 = g[0], CPhi2 = g[1], CPhi = g[2], S2Psi = g[3], C2Psi = g[4];
    double PI = 0.5 * (Php * SPhi2 + 0.5 * (Phr + Phb) * (1.0 + CPhi2)) + lop + cop;
    double InvPhiI = 1.0 / PI;
    double Sabs = 0.5 * (Php - 0.5 * (Phr + Phb)) * SPhi2;
    double PhiQ = Sabs * C2Psi * InvPhiI, PhiU = Sabs * S2Psi * InvPhiI;
    double PhiV = 0.5 * (Phr - Phb) * CPhi * InvPhiI;
    double Sdis = 0.5 * (Psp - 0.5 * (Psr + Psb)) * SPhi2;
    double PsiQ = Sdis * C2Psi * InvPhiI, PsiU = Sdis * S2Psi * InvPhiI;
    double PsiV = 0.5 * (Psr - Psb) * CPhi * InvPhiI;
    e6[0] = PhiQ; e6[1] = PhiU; e6[2] = PhiV; e6[3] = PsiQ; e6[4] = PsiU; e6[5] = PsiV;
    s4[0] = sr; s4[1] = sr * PhiQ; s4[2] = sr * PhiU; s4[3] = sr * PhiV;
    return PI;
}

// StokesPrfPP, one thread per (wavelength, angle) from the first wavelength iwl0 on, in two launches
// over per-thread global work arrays (STK_FIELDS x ntau doubles, element stride = the launch's thread
// count T, so that the threads of a warp touch consecutive addresses).  k_stokes_prep builds the
// propagation data, TauStep and CentDer over depth; it needs few registers, so many warps hide the
// latency of its array traffic.  k_stokes_thr runs the sequential 4x4 sweep (about 200 registers);
// every lane of every warp sweeps.  The reference's operations, in its order.
__global__ void __launch_bounds__(128)
k_stokes_prep(AtmView A, const double *__restrict__ lineopac, const double *__restrict__ mlo,
              const double *__restrict__ rhox, int nmu, const double *__restrict__ xmu,
              const double *__restrict__ geo, int iwl0, int nwl_chunk, double *work) {
    const size_t T = (size_t)gridDim.x * blockDim.x;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nwl_chunk * nmu) return;
    const int iwl = iwl0 + g / nmu, im = g - (g / nmu) * nmu;
    const int N = A.ntau;
    double *W = work + g;
#define F(f, t) W[((size_t)(f) * N + (t)) * T]
    const double PlkC1 = FSG_HC * FSG_VC * 1e13 / FSG_KBOLT;
    const double wl = A.wave[iwl] + A.wfirst;
    const double C1 = PlkC1 / wl, C2 = exp(50.7649141 - 5.0 * log(wl));
    const double gm[5] = { geo[0 * nmu + im], geo[1 * nmu + im], geo[2 * nmu + im], geo[3 * nmu + im],
                           geo[4 * nmu + im] };
    for (int t = 0; t < N; t++) {
        const size_t o = (size_t)iwl * N + t;
        const double sr = C2 / (exp(C1 / A.xi[XI_T * N + t]) - 1.0);
        double e6[6], s4[4];
        F(0, t) = stokes_point(mlo + o * 6, lineopac[o], A.contopac[o], sr, gm, e6, s4);
        for (int q = 0; q < 6; q++) F(1 + q, t) = e6[q];
        for (int q = 0; q < 4; q++) F(13 + q, t) = s4[q];
    }
    // TauStep (solver.f90:591-615) with Xmu(im)
    const double Xmu = xmu[im];
    for (int t = 0; t < N - 1; t++) {
        if (t == 0) {
            double Dx1 = (rhox[1] - rhox[0]) / Xmu;
            double Yp = (F(0, 1) - F(0, 0)) / Dx1;
            F(21, 0) = Dx1 * (F(0, 1) + 2.0 * F(0, 0) + Dx1 / 2.0 * Yp) / 3.0;
        } else {
            const int k = t + 1;
            double Dx = (rhox[k - 1] - rhox[k - 2]) / Xmu, Dx1 = (rhox[k] - rhox[k - 1]) / Xmu;
            double Der = (F(0, k - 1) - F(0, k - 2)) / Dx, Der1 = (F(0, k) - F(0, k - 1)) / Dx1, Yp;
            if (Der * Der1 > 0.0) {
                double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0;
                Yp = (Der / (Lambda * Der1 + (1.0 - Lambda) * Der)) * Der1;
            } else Yp = 0.0;
            F(21, k - 1) = Dx1 * (F(0, k) + 2.0 * F(0, k - 1) + Dx1 / 2.0 * Yp) / 3.0;
        }
    }
    // CentDer (solver.f90:618-647) of SRC4 (fields 13-16 -> 17-20) and of the 6 elements (1-6 -> 7-12)
    for (int row = 0; row < 10; row++) {
        const int fi = row < 4 ? 13 + row : 1 + (row - 4), fo = row < 4 ? 17 + row : 7 + (row - 4);
        for (int k = 0; k < N; k++) {
            double out;
            if (k == 0) out = (F(fi, 1) - F(fi, 0)) / F(21, 0);
            else if (k == N - 1) out = (F(fi, N - 1) - F(fi, N - 2)) / F(21, N - 2);
            else {
                double Dx = F(21, k - 1), Dx1 = F(21, k);
                double InvDx = 1.0 / Dx, InvDx1 = 1.0 / Dx1;
                double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0, Lambda1 = 1.0 - Lambda;
                double Der = (F(fi, k) - F(fi, k - 1)) * InvDx, Der1 = (F(fi, k + 1) - F(fi, k)) * InvDx1;
                out = (Der * Der1 > 0.0) ? (Der / (Lambda * Der1 + Lambda1 * Der)) * Der1 : 0.0;
            }
            F(fo, k) = out;
        }
    }
#undef F
}

__global__ void __launch_bounds__(128)
k_stokes_thr(AtmView A, int nmu, int iwl0, int nwl_chunk, const double *work, double *spz) {
    const size_t T = (size_t)gridDim.x * blockDim.x;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nwl_chunk * nmu) return;
    const int iwl = iwl0 + g / nmu, im = g - (g / nmu) * nmu;
    const int N = A.ntau;
    const double *W = work + g;
#define F(f, t) W[((size_t)(f) * N + (t)) * T]
    double XINT2[4] = { F(13, N - 1), 0.0, 0.0, 0.0 };
    stokes_sweep(N, N, &F(1, 0), &F(7, 0), &F(13, 0), &F(17, 0), &F(21, 0), XINT2, T);
    for (int q = 0; q < 4; q++) spz[((size_t)iwl * 4 + q) * nmu + im] = XINT2[q];
#undef F
}

// StokesPrfSph (solver.f90:402-538), one thread per (wavelength, ray) from the first wavelength iwl0
// on, with per-thread work arrays as k_stokes_thr (up to 2 ntau points per ray).  Each point gathers the
// six profiles, line and continuum opacity and source of the layer it samples, with the field
// projection of that point (geo [5][nmu][stride]); TauStep runs on the ray's column mass (mu = 1); the
// sweep starts from zero incoming light for grazing rays, Src(N) otherwise.
__global__ void __launch_bounds__(128)
k_stokes_sph(AtmView A, const double *__restrict__ lineopac, const double *__restrict__ mlo, RayView R,
             const double *__restrict__ geo, int iwl0, int nwl_chunk, double *work, double *spz) {
    const size_t T = (size_t)gridDim.x * blockDim.x;
    const int nmu = R.nmu, M = R.stride, nt = A.ntau;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nwl_chunk * nmu) return;
    const int iwl = iwl0 + g / nmu, im = g - (g / nmu) * nmu;
    const int N = R.n[im];
    const int *mp = R.map + (size_t)im * M;
    const double *m = R.m + (size_t)im * M;
    double *W = work + g;
#define F(f, t) W[((size_t)(f) * M + (t)) * T]
    const double PlkC1 = FSG_HC * FSG_VC * 1e13 / FSG_KBOLT;
    const double wl = A.wave[iwl] + A.wfirst;
    const double C1 = PlkC1 / wl, C2 = exp(50.7649141 - 5.0 * log(wl));
    const size_t gs = (size_t)nmu * M, go = (size_t)im * M;
    for (int t = 0; t < N; t++) {
        const int ia = mp[t];
        const size_t o = (size_t)iwl * nt + ia;
        const double sr = C2 / (exp(C1 / A.xi[XI_T * nt + ia]) - 1.0);
        const double gm[5] = { geo[go + t], geo[gs + go + t], geo[2 * gs + go + t], geo[3 * gs + go + t],
                               geo[4 * gs + go + t] };
        double e6[6], s4[4];
        F(0, t) = stokes_point(mlo + o * 6, lineopac[o], A.contopac[o], sr, gm, e6, s4);
        for (int q = 0; q < 6; q++) F(1 + q, t) = e6[q];
        for (int q = 0; q < 4; q++) F(13 + q, t) = s4[q];
    }
    // TauStep (solver.f90:591-615) on the ray's column mass
    for (int t = 0; t < N - 1; t++) {
        if (t == 0) {
            double Dx1 = m[1] - m[0], Yp = (F(0, 1) - F(0, 0)) / Dx1;
            F(21, 0) = Dx1 * (F(0, 1) + 2.0 * F(0, 0) + Dx1 / 2.0 * Yp) / 3.0;
        } else {
            double Dx = m[t] - m[t - 1], Dx1 = m[t + 1] - m[t];
            double Der = (F(0, t) - F(0, t - 1)) / Dx, Der1 = (F(0, t + 1) - F(0, t)) / Dx1, Yp;
            if (Der * Der1 > 0.0) {
                double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0;
                Yp = (Der / (Lambda * Der1 + (1.0 - Lambda) * Der)) * Der1;
            } else Yp = 0.0;
            F(21, t) = Dx1 * (F(0, t + 1) + 2.0 * F(0, t) + Dx1 / 2.0 * Yp) / 3.0;
        }
    }
    // CentDer (solver.f90:618-647) of SRC4 (fields 13-16 -> 17-20) and of the 6 elements (1-6 -> 7-12)
    for (int row = 0; row < 10; row++) {
        const int fi = row < 4 ? 13 + row : 1 + (row - 4), fo = row < 4 ? 17 + row : 7 + (row - 4);
        for (int k = 0; k < N; k++) {
            double out;
            if (k == 0) out = (F(fi, 1) - F(fi, 0)) / F(21, 0);
            else if (k == N - 1) out = (F(fi, N - 1) - F(fi, N - 2)) / F(21, N - 2);
            else {
                double Dx = F(21, k - 1), Dx1 = F(21, k);
                double InvDx = 1.0 / Dx, InvDx1 = 1.0 / Dx1;
                double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0, Lambda1 = 1.0 - Lambda;
                double Der = (F(fi, k) - F(fi, k - 1)) * InvDx, Der1 = (F(fi, k + 1) - F(fi, k)) * InvDx1;
                out = (Der * Der1 > 0.0) ? (Der / (Lambda * Der1 + Lambda1 * Der)) * Der1 : 0.0;
            }
            F(fo, k) = out;
        }
    }
    double XINT2[4] = { R.graz[im] ? 0.0 : F(13, N - 1), 0.0, 0.0, 0.0 };
    stokes_sweep(N, M, &F(1, 0), &F(7, 0), &F(13, 0), &F(17, 0), &F(21, 0), XINT2, T);
    for (int q = 0; q < 4; q++) spz[((size_t)iwl * 4 + q) * nmu + im] = XINT2[q];
#undef F
}

// Stokes-I flux of the spherical path: Sf = sum over mu of SpZ(mu, 1) Wmu (convol.f90:233-234)
__global__ void k_stokes_flux(int nwl, int nmu, const double *__restrict__ spz, const double *__restrict__ wmu,
                              double *sfl) {
    int iwl = blockIdx.x * blockDim.x + threadIdx.x;
    if (iwl >= nwl) return;
    double a = 0.0;
    for (int q = 0; q < nmu; q++) a = a + spz[(size_t)iwl * 4 * nmu + q] * wmu[q];
    sfl[iwl] = a;
}

// ================================================================================================
// host drivers
// ================================================================================================
struct fsg_ctx;
AtmView fsg_view(const fsg_ctx *ctx);

// per-thread work arrays of k_stokes_thr for one chunk of nwl_chunk wavelengths
size_t fsg_stokes_work(int nt, int nmu, int nwl_chunk) {
    const size_t nthr = ((size_t)nwl_chunk * nmu + 127) / 128 * 128;
    return sizeof(double) * STK_FIELDS * (size_t)nt * nthr;
}

// the most wavelengths (at least 1, at most nwl) whose work arrays fit in max_bytes
int fsg_stokes_chunk(int nt, int nmu, int nwl, size_t max_bytes) {
    const size_t per_wl = sizeof(double) * STK_FIELDS * (size_t)nt * nmu;
    size_t c = max_bytes / per_wl;
    if (c > (size_t)nwl) c = (size_t)nwl;
    return c < 1 ? 1 : (int)c;
}

// StokesPrfPP over the grid: k_stokes_thr in chunks of nwl_chunk wavelengths whose work arrays fit `work`
// (fsg_stokes_work bytes), then the Stokes-I flux.
int fsg_launch_stokes(cudaStream_t s, const AtmView &A, const double *lineopac, const double *mlo, const double *rhox,
                      int nmu, const double *xmu, const double *wmu, const double *geo, double *spz, double *sfl,
                      double *work, int nwl_chunk) {
    if (nwl_chunk < 1) return FSG_E_ARG;
    for (int w0 = 0; w0 < A.nwl; w0 += nwl_chunk) {
        const int nw = std::min(nwl_chunk, A.nwl - w0);
        const int nb = (nwl_chunk * nmu + 127) / 128;      // the grid of a full chunk: fixed element stride
        k_stokes_prep<<<nb, 128, 0, s>>>(A, lineopac, mlo, rhox, nmu, xmu, geo, w0, nw, work);
        k_stokes_thr<<<nb, 128, 0, s>>>(A, nmu, w0, nw, work, spz);
    }
    if (sfl) k_stokes_flux<<<(A.nwl + 127) / 128, 128, 0, s>>>(A.nwl, nmu, spz, wmu, sfl);
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}

int fsg_launch_stokes_sph(cudaStream_t s, const AtmView &A, const double *lineopac, const double *mlo,
                          const RayView &R, const double *wmu, const double *geo, double *spz, double *sfl,
                          double *work, int nwl_chunk) {
    if (nwl_chunk < 1) return FSG_E_ARG;
    for (int w0 = 0; w0 < A.nwl; w0 += nwl_chunk) {
        const int nw = std::min(nwl_chunk, A.nwl - w0);
        const int nb = (nwl_chunk * R.nmu + 127) / 128;     // the grid of a full chunk: fixed element stride
        k_stokes_sph<<<nb, 128, 0, s>>>(A, lineopac, mlo, R, geo, w0, nw, work, spz);
    }
    if (sfl) k_stokes_flux<<<(A.nwl + 127) / 128, 128, 0, s>>>(A.nwl, R.nmu, spz, wmu, sfl);
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}

void fsg_launch_mag_center(cudaStream_t s, const AtmView &A, const LineView &L, const ZView &Z, double Bsplit,
                           const VoigtTables &T, int32_t *flags, int32_t *ileft, int32_t *iright,
                           unsigned long long *nkeep) {
    if (L.n > 0)
        k_mag_center<<<(unsigned)((L.n + 3) / 4), 128, 0, s>>>(A, L, Z, Bsplit, T.vtab, T.anode, T.aida, flags, ileft,
                                                                iright, nkeep);
}

void fsg_launch_mag_params(cudaStream_t s, const AtmView &A, const LineView &L, int64_t n, const int64_t *list,
                           int64_t off, const int32_t *flags, double3 *p) {
    if (n > 0) k_mag_params<<<(unsigned)((n + 63) / 64), 64, 0, s>>>(A, L, n, list, off, flags, p);
}

void fsg_launch_mag_accum(cudaStream_t s, const AtmView &A, const double *wl, const ZView &Z, const int64_t *zmap,
                          int iwl1, int iwl2, const int *lstart, const int *lstop, const int32_t *flags,
                          const int32_t *ileft, const int32_t *iright, int64_t loff, const double3 *p64,
                          const VoigtTables &T, double *mlo, double *evals) {
    int nw = iwl2 - iwl1 + 1;
    if (nw > 0)
        k_mag_accum<<<(nw + 7) / 8, 256, 0, s>>>(A, wl, Z, zmap, iwl1, iwl2, lstart, lstop, flags, ileft, iright, loff,
                                                 p64, T.fvtab, T.anode, T.aida, mlo, evals);
}

void fsg_launch_mag_wide(cudaStream_t s, const AtmView &A, const double *wl, const ZView &Z, const int64_t *zmap,
                         int nwide, const int64_t *widx, const int32_t *flags, const int32_t *ileft,
                         const int32_t *iright, const double3 *pw, const VoigtTables &T, double *mlo) {
    if (nwide > 0)
        k_mag_wide<<<(A.nwl + 7) / 8, 256, 0, s>>>(A, wl, Z, zmap, nwide, widx, flags, ileft, iright, pw, T.fvtab,
                                                   T.anode, T.aida, mlo);
}


// ================================================================================================
// MagLineOpacity1 and StokesPrfPP on their own, batched (kernel-level entry points)
// ================================================================================================
// MagLineOpacity1 (opacity.f90:391-464) at npts points; the block's Zeeman components are indexed by
// line (Z's CSR arrays); one warp per point, lanes over depths; out [npts][ntau][6]
__global__ void k_mag_lineopacity1_pts(AtmView A, BlockView B, ZView Z, int64_t npts, const double *__restrict__ wl,
                                       const int32_t *__restrict__ l1, const int32_t *__restrict__ l2,
                                       const int32_t *__restrict__ iwl, int64_t loff, const float2 *__restrict__ fvtab,
                                       const double *__restrict__ anode, const double *__restrict__ aida, double *out) {
    const int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (k >= npts) return;
    const int nt = A.ntau;
    for (int t = lane; t < nt; t += 32) {
        double m[6] = { 0, 0, 0, 0, 0, 0 };
        for (int64_t il = l1[k]; il <= l2[k]; il++) {
            const int f = B.flags[il - 1];
            if ((f & FSG_F_WEAK) || (f & FSG_F_WIDE) || iwl[k] < B.ileft[il - 1] || iwl[k] > B.iright[il - 1]) continue;
            const size_t o = (size_t)(il - loff - 1) * nt + t;
            mag_profiles_t(A, t, wl[k], B.wlcent[il - 1], (f >> 8) & 255, Z, il - 1, B.cop[o], B.vv[o], B.av[o],
                           fvtab, anode, aida, m);
        }
        double *dst = out + ((size_t)k * nt + t) * 6;
        for (int q = 0; q < 6; q++) dst[q] = (A.motype == 1) ? m[q] / A.contstd[t] : m[q];
    }
}

// StokesPrfPP (solver.f90:265-394) at the grid wavelengths iwl[k] (1-based) with given source functions
// src [npts][ntau]: one thread per (point, angle) over per-thread work arrays, as k_stokes_thr;
// geo [5][nmu] (SPhi2, CPhi2, CPhi, S2Psi, C2Psi); out [npts][4][nmu]
__global__ void __launch_bounds__(128)
k_stokes_prf_pts(AtmView A, const double *__restrict__ lineopac, const double *__restrict__ mlo,
                 const double *__restrict__ rhox, int nmu, const double *__restrict__ xmu,
                 const double *__restrict__ geo, int64_t npts, const int32_t *__restrict__ iwls,
                 const double *__restrict__ src, double *work, double *out) {
    const size_t T = (size_t)gridDim.x * blockDim.x;
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= npts * nmu) return;
    const int64_t k = g / nmu;
    const int im = (int)(g - k * nmu);
    const int iwl = iwls[k] - 1;
    const int N = A.ntau;
    double *W = work + g;
#define F(f, t) W[((size_t)(f) * N + (t)) * T]
    const double gm[5] = { geo[0 * nmu + im], geo[1 * nmu + im], geo[2 * nmu + im], geo[3 * nmu + im],
                           geo[4 * nmu + im] };
    for (int t = 0; t < N; t++) {
        const size_t o = (size_t)iwl * N + t;
        double e6[6], s4[4];
        F(0, t) = stokes_point(mlo + o * 6, lineopac[o], A.contopac[o], src[(size_t)k * N + t], gm, e6, s4);
        for (int q = 0; q < 6; q++) F(1 + q, t) = e6[q];
        for (int q = 0; q < 4; q++) F(13 + q, t) = s4[q];
    }
    const double Xmu = xmu[im];
    for (int t = 0; t < N - 1; t++) {
        if (t == 0) {
            double Dx1 = (rhox[1] - rhox[0]) / Xmu;
            double Yp = (F(0, 1) - F(0, 0)) / Dx1;
            F(21, 0) = Dx1 * (F(0, 1) + 2.0 * F(0, 0) + Dx1 / 2.0 * Yp) / 3.0;
        } else {
            const int kk = t + 1;
            double Dx = (rhox[kk - 1] - rhox[kk - 2]) / Xmu, Dx1 = (rhox[kk] - rhox[kk - 1]) / Xmu;
            double Der = (F(0, kk - 1) - F(0, kk - 2)) / Dx, Der1 = (F(0, kk) - F(0, kk - 1)) / Dx1, Yp;
            if (Der * Der1 > 0.0) {
                double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0;
                Yp = (Der / (Lambda * Der1 + (1.0 - Lambda) * Der)) * Der1;
            } else Yp = 0.0;
            F(21, kk - 1) = Dx1 * (F(0, kk) + 2.0 * F(0, kk - 1) + Dx1 / 2.0 * Yp) / 3.0;
        }
    }
    for (int row = 0; row < 10; row++) {
        const int fi = row < 4 ? 13 + row : 1 + (row - 4), fo = row < 4 ? 17 + row : 7 + (row - 4);
        for (int kk = 0; kk < N; kk++) {
            double o;
            if (kk == 0) o = (F(fi, 1) - F(fi, 0)) / F(21, 0);
            else if (kk == N - 1) o = (F(fi, N - 1) - F(fi, N - 2)) / F(21, N - 2);
            else {
                double Dx = F(21, kk - 1), Dx1 = F(21, kk);
                double InvDx = 1.0 / Dx, InvDx1 = 1.0 / Dx1;
                double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0, Lambda1 = 1.0 - Lambda;
                double Der = (F(fi, kk) - F(fi, kk - 1)) * InvDx, Der1 = (F(fi, kk + 1) - F(fi, kk)) * InvDx1;
                o = (Der * Der1 > 0.0) ? (Der / (Lambda * Der1 + Lambda1 * Der)) * Der1 : 0.0;
            }
            F(fo, kk) = o;
        }
    }
    double XINT2[4] = { F(13, N - 1), 0.0, 0.0, 0.0 };
    stokes_sweep(N, N, &F(1, 0), &F(7, 0), &F(13, 0), &F(17, 0), &F(21, 0), XINT2, T);
    for (int q = 0; q < 4; q++) out[((size_t)k * 4 + q) * nmu + im] = XINT2[q];
#undef F
}

void fsg_launch_mag_lineopacity1_pts(cudaStream_t s, const AtmView &A, const BlockView &B, const ZView &Z,
                                     int64_t npts, const double *wl, const int32_t *l1, const int32_t *l2,
                                     const int32_t *iwl, int64_t loff, const VoigtTables &T, double *out) {
    if (npts > 0)
        k_mag_lineopacity1_pts<<<(unsigned)((npts + 7) / 8), 256, 0, s>>>(A, B, Z, npts, wl, l1, l2, iwl, loff,
                                                                          T.fvtab, T.anode, T.aida, out);
}

size_t fsg_stokes_pts_work(int64_t npts, int nmu, int ntau) {
    const int64_t thr = ((npts * nmu + 127) / 128) * 128;
    return sizeof(double) * (size_t)STK_FIELDS * (size_t)ntau * (size_t)thr;
}

void fsg_launch_stokes_prf_pts(cudaStream_t s, const AtmView &A, const double *lineopac, const double *mlo,
                               const double *rhox, int nmu, const double *xmu, const double *geo, int64_t npts,
                               const int32_t *iwl, const double *src, double *work, double *out) {
    const int64_t m = npts * nmu;
    if (m > 0)
        k_stokes_prf_pts<<<(unsigned)((m + 127) / 128), 128, 0, s>>>(A, lineopac, mlo, rhox, nmu, xmu, geo, npts, iwl,
                                                                     src, work, out);
}
