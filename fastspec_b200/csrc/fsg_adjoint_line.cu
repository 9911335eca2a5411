// fsg_adjoint_line.cu -- the line part of the adjoint: the transpose of the line accumulation.
//   glin_l  = sum_{t, lambda in window} dL/dkappa(t, lambda) LinCop_t H(a_t, v)              (d / d ln gf)
//   gvmic_l = sum dL/dkappa LinCop_t q_t Hd,  Hd = -H - v dH/dv - a dH/da                      (d / d vmic)
// (LinCop, v and a all scale as 1/Dopl; q = d ln Dopl / d vmic = vturb2 / (vmic Dopl^2).)
//
// Pass 1, k_adj_setup: one warp per line computes the per-depth LinCop, LinVvgt, LinAvgt and q with
// the forward's FP64 arithmetic (XlineSetup / XlineDepth), writes the line's records for pass 2, its
// core range (the wavelengths where some depth has s = v^2 + a^2 < 196, widened by one) and the
// window-edge term (below).  Helium lines with a per-depth Stark shift (few) are reduced there
// over their whole window in FP64 and left out of pass 2.
//
// Pass 2, k_adj_tiles: the accumulation's tiling turned around.  A CTA owns a tile of 64
// wavelengths x all depths: consumer warp w keeps dL/dkappa of depths [w KD, w KD + KD) at the
// lane's two wavelengths in registers; one producer warp picks the lines whose windows meet the
// tile, 16 at a time, and brings their records into a double-buffered shared-memory stage by bulk
// copies (mbarrier-tracked, released by the consumers through a second mbarrier pair).  Outside a
// line's core range the wing form is two polynomials in X = dl^2 and one reciprocal per point,
// with depth pairs in packed FP32 (FFMA2):
//   D = y^2 + B1 y + B0,  y = vv^2 X,  B1 = 2a^2 - 1,  B0 = a^4 + a^2 + 1/4
//   LinCop H  = K1 (y + a^2 + 1/2) / D                                    K1 = LinCop a / sqrt(pi)
//   LinCop q Hd = K2 (1 + 2 (y^2 - B0) / D) / D                           K2 = LinCop q a / sqrt(pi)
// i.e. per point D = (c4 X + c2) X + B0, h = e1 X + e0, p = f2 X^2 + f0, and the sums take
// g/D * h and g/D * (p/D + K2).  Lines whose core range meets the tile take the point-by-point
// path (FvTab or the complex rational inside, the same wing form outside).  Partial sums are
// reduced over lanes by shuffles, over warps by the producer (FP64, fixed order), and each
// tile's part is added to the line's FP64 sums with one atomic.
//
// Profile and derivative forms (FVoigt / FVoigtLine, voigt.f90:256-352):
//  * wing, s >= 196: the rational H = a (s + 1/2) / (sqrt(pi) D), D = s^2 - (v^2 - a^2) + 1/4, the
//    form the forward evaluates there.  Hd is its exact scaling derivative, which with y = v^2 is
//    a (3y^2 + B1 y - B0) / (sqrt(pi) D^2) = a (D + 2 (y^2 - B0)) / (sqrt(pi) D^2): no cancellation
//    of the leading terms of -H - v dH/dv - a dH/da (which cancel as 1/v^2).
//  * core: H and L from FvTab (|v| < 8, a < 8) or the complex rational, and the Faddeeva derivative
//    dw/dz = -2 z w + 2i/sqrt(pi), w = H + iL, z = v + ia:  dH/dv = -2 (v H - a L),
//    dH/da = 2 (v L + a H) - 2/sqrt(pi), so Hd = H (2 (v^2 - a^2) - 1) - 4 a v L + 2 a / sqrt(pi).
//
// Window edges (AnalyticWindow, opacity.f90:678-710): W = max_t sqrt(S_t) / LinVvgt_t with
// S = ln r + max(0, a (r / sqrt(pi) - a)), r = LinCop / (EpsOpac ContOpac), grows with gf and vmic;
// its free edges move by dW, adding the edge profile over dW / (wavelength step) at each edge
// (d ln W from the depth giving the maximum).
#include "fsg_fp64.cuh"
#include "fsg_mbar.cuh"

size_t fsg_tile_span_scratch(int64_t);
int fsg_launch_tile_span_tw(cudaStream_t, int, int, int, int64_t, const LineHdr *, int *, int *, void *, size_t);

#define ADJ_SETUP_WARPS 8
#define ADJ_P 2                        // wavelengths per lane
#define ADJ_TW (32 * ADJ_P)            // wavelengths per tile
#define ADJ_CL 16                      // lines per stage

// depths per consumer warp, and the depth count padded to a multiple of it
static int adj_kd(int nt) { return nt >= 32 ? 8 : (nt >= 8 ? 4 : 2); }
static int adj_ntp(int nt) { const int k = adj_kd(nt); return (nt + k - 1) / k * k; }

// Pass-2 records of line i: ntp/2 depth pairs x 4 float4, pair (t, t+1) as
//   {c4, c4', c2, c2'} {B0, B0', e1, e1'} {e0, e0', f2, f2'} {f0, f0', K2, K2'}
// with c4 = vv^4, c2 = B1 vv^2, e1 = K1 vv^2, e0 = K1 (a^2 + 1/2), f2 = 2 K2 vv^4, f0 = -2 K2 B0.
// Padding depths (t >= nt) hold D = 1 and zero weights.
__device__ __forceinline__ void put_pair_rec(float *r, int t, double vv, double a, double c, double cq) {
    const int e = t & 1;
    float *q = r + (size_t)(t >> 1) * 16;
    const double a2 = a * a, B1 = 2.0 * a2 - 1.0, B0 = a2 * a2 + a2 + 0.25;
    const double K1 = c * a * FSG_SQRTPIINV, K2 = cq * a * FSG_SQRTPIINV;
    const double vv2 = vv * vv, vv4 = vv2 * vv2;
    q[0 + e] = (float)vv4;
    q[2 + e] = (float)(B1 * vv2);
    q[4 + e] = (float)B0;
    q[6 + e] = (float)(K1 * vv2);
    q[8 + e] = (float)(K1 * (a2 + 0.5));
    q[10 + e] = (float)(2.0 * K2 * vv4);
    q[12 + e] = (float)(-2.0 * K2 * B0);
    q[14 + e] = (float)K2;
}
__device__ __forceinline__ void put_pad_rec(float *r, int t) {
    const int e = t & 1;
    float *q = r + (size_t)(t >> 1) * 16;
    q[0 + e] = 0.0f; q[2 + e] = 0.0f; q[4 + e] = 1.0f; q[6 + e] = 0.0f;
    q[8 + e] = 0.0f; q[10 + e] = 0.0f; q[12 + e] = 0.0f; q[14 + e] = 0.0f;
}

// crec[i][t] = (LinVvgt, LinAvgt, LinCop, LinCop q); tabi[i][t] = (UA, IA) of FVoigtLine (IA = 0: a >= 8)
__global__ void __launch_bounds__(32 * ADJ_SETUP_WARPS)
k_adj_setup(AtmView A, LineView L, const float *__restrict__ vtab, const float2 *__restrict__ fvtab,
            const double *__restrict__ anode, const double *__restrict__ aida, const int32_t *__restrict__ flags,
            const int32_t *__restrict__ ileft, const int32_t *__restrict__ iright,
            const double *__restrict__ gkappa, double vmic, int ntp, float *__restrict__ prec,
            float4 *__restrict__ crec, float2 *__restrict__ tabi, LineHdr *__restrict__ hdr, double *glin,
            double *gvmic, int i0, int i1) {
    extern __shared__ double sh[];
    const int nt = A.ntau;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *cop = sh + (size_t)warp * 6 * nt, *vv = cop + nt, *av = vv + nt, *q = av + nt, *shf = q + nt;
    double *rr = shf + nt;
    const int64_t i = (int64_t)blockIdx.x * ADJ_SETUP_WARPS + warp;
    if (i >= L.n) return;
    const int f = flags[i];
    if (f & FSG_F_WEAK) {
        if (lane == 0) {
            glin[i] = 0.0; gvmic[i] = 0.0;
            LineHdr h = {}; h.ileft = 1; h.iright = 0; h.cl = 1; h.cr = 0;
            hdr[i] = h;
        }
        return;
    }
    const double wlc = L.wl[i] - A.wfirst;
    XCoef XC;
    xline_setup(A, L, i, wlc, line_input_flags(L, i, 0), &XC);
    const int iwc = waveidx(A, wlc);
    const double dWc = (wlc - A.wave[iwc - 1]) / (A.wave[iwc] - A.wave[iwc - 1]);
    const bool he = XC.IxHe > 0;
    float *pr = prec + (size_t)i * ntp * 8;
    double hcore = -1.0;                                  // largest |dl| of any depth's s < 196
    for (int t = lane; t < nt; t += 32) {
        double Dopl;
        double c = xline_cop(A, t, XC, &Dopl);
        double v_, a_;
        xline_av(A, t, XC, Dopl, &v_, &a_);
        double r = c / (A.epsopac * cont_center(A, iwc, dWc, t));
        if (A.motype == 1) { c = c / A.contstd[t]; r = r / A.contstd[t]; }
        rr[t] = r;
        cop[t] = c; vv[t] = v_; av[t] = a_;
        q[t] = (vmic > 0.0) ? A.vturb2 / (vmic * Dopl * Dopl) : 0.0;
        shf[t] = he ? A.heshf[(XC.IxHe - 1) * nt + t] : 0.0;
        const VLine64 VL = vline64(anode, aida, a_);
        crec[i * nt + t] = make_float4((float)v_, (float)a_, (float)c, (float)(c * q[t]));
        tabi[i * nt + t] = make_float2((float)VL.UA, (float)VL.IA);
        put_pair_rec(pr, t, v_, a_, c, c * q[t]);
        if (a_ * a_ < 196.0) hcore = fmax(hcore, sqrt(196.0 - a_ * a_) / v_);
    }
    for (int t = nt + lane; t < ntp; t += 32) put_pad_rec(pr, t);
    __syncwarp();
    // the line's window and its part inside the wavelength range [i0, i1] this call reduces over
    const int il = ileft[i], ir = iright[i];
    const int rl = max(il, i0), rr_ = min(ir, i1);
    double sl = 0.0, sv = 0.0;
    const double isp2 = 2.0 * FSG_SQRTPIINV;
    if (he) {
        // lanes over depths, a loop over the window's wavelengths, all in FP64
        for (int t = lane; t < nt; t += 32) {
            const double c = cop[t], vvt = vv[t], a = av[t], qt = q[t], off = wlc + shf[t];
            const VLine64 VL = vline64(anode, aida, a);
            double s1 = 0.0, s2 = 0.0;
            for (int iw = rl - 1; iw < rr_; iw++) {
                const double g = gkappa[(size_t)iw * nt + t];
                const double v = (A.wave[iw] - off) * vvt;
                double Hf, Lf;
                fvoigt_line64(fvtab, VL, v, &Hf, &Lf);
                const double Hv = -2.0 * (v * Hf - a * Lf), Ha = 2.0 * (v * Lf + a * Hf) - isp2;
                s1 += g * Hf;
                s2 += g * (-v * Hv - a * Ha - Hf);
            }
            sl += s1 * c;
            sv += s2 * c * qt;
        }
    }
    // window edges: the depth giving W, and the edge profiles weighted by dL/dkappa
    const double iSqrtPi = FSG_SQRTPIINV;
    double wbest = -1.0, dgf = 0.0, dvm = 0.0;
    for (int t = lane; t < nt; t += 32) {
        const double r = rr[t];
        if (!(r > 1.0)) continue;
        const double X = av[t] * (r * iSqrtPi - av[t]), S = log(r) + fmax(0.0, X);
        const double w = sqrt(S) / vv[t];
        if (w > wbest) {
            wbest = w;
            dgf = w * (1.0 + (X > 0.0 ? av[t] * r * iSqrtPi : 0.0)) / (2.0 * S);          // dW / d ln gf
            dvm = q[t] * w * (1.0 + (-1.0 - (X > 0.0 ? 2.0 * X : 0.0)) / (2.0 * S));     // dW / d vmic
        }
    }
    double eb = 0.0;                                      // sum over free edges of dL/dkappa * profile / step
    for (int t = lane; t < nt; t += 32) {
        const VLine64 VL = vline64(anode, aida, av[t]);
        if (il > 1 && il >= i0 && il <= i1) {            // a free edge inside the range
            const int iw = il - 1;
            const double v = (A.wave[iw] - wlc - shf[t]) * vv[t];
            eb += gkappa[(size_t)iw * nt + t] * hvoigt_line64(vtab, VL, v) * cop[t] / (A.wave[iw] - A.wave[iw - 1]);
        }
        if (ir < A.nwl && ir >= i0 && ir <= i1) {
            const int iw = ir - 1;
            const double v = (A.wave[iw] - wlc - shf[t]) * vv[t];
            eb += gkappa[(size_t)iw * nt + t] * hvoigt_line64(vtab, VL, v) * cop[t] / (A.wave[iw + 1] - A.wave[iw]);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        sl += __shfl_xor_sync(0xffffffffu, sl, o);
        sv += __shfl_xor_sync(0xffffffffu, sv, o);
        eb += __shfl_xor_sync(0xffffffffu, eb, o);
        hcore = fmax(hcore, __shfl_xor_sync(0xffffffffu, hcore, o));
        const double wo = __shfl_xor_sync(0xffffffffu, wbest, o), go = __shfl_xor_sync(0xffffffffu, dgf, o);
        const double vo = __shfl_xor_sync(0xffffffffu, dvm, o);
        if (wo > wbest || (wo == wbest && go > dgf)) { wbest = wo; dgf = go; dvm = vo; }
    }
    if (lane == 0) {
        if (wbest < 0.0) { dgf = 0.0; dvm = 0.0; }
        glin[i] = sl + eb * dgf;
        gvmic[i] = sv + eb * dvm;
        LineHdr h = {};
        h.wlh = (float)wlc;
        h.wll = (float)(wlc - (double)h.wlh);
        h.ileft = he ? 1 : rl;                            // helium lines: done above
        h.iright = he ? 0 : rr_;
        h.cl = 1; h.cr = 0;
        if (hcore >= 0.0 && !he) {
            // 1-based indices of the first wavelength >= wlc - hcore and the last <= wlc + hcore,
            // widened by one wavelength and clipped to the window
            const int a = lower_index(A.wave, A.nwl, wlc - hcore) + 1;
            int b = lower_index(A.wave, A.nwl, wlc + hcore);
            if (b < A.nwl && A.wave[b] == wlc + hcore) b++;
            const int cl = max(a - 1, rl), cr = min(b + 1, rr_);
            if (cl <= cr) { h.cl = cl; h.cr = cr; }
        }
        hdr[i] = h;
    }
}

struct AdjTileJob {
    int nwl, nt, ntp, nw;              // wavelengths, depths, padded depths, consumer warps
    const float *gk32;                 // dL/dkappa, FP32, [nt][nwl]
    const float *wvh, *wvl;            // wavelength offsets as FP32 hi + lo, [nwl]
    const float4 *prec;                // [n][ntp / 2][4]
    const float4 *crec;                // [n][nt]
    const float2 *tabi;                // [n][nt]
    const LineHdr *hdr;                // [n]
    const int *tlo, *thi;              // line range of each tile (inclusive)
    const float2 *fvtab;
    double *glin, *gvmic;
    int *err;
};

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// H and Hd at (v, a) for s = v^2 + a^2 < 196: FvTab interpolation or the complex rational
__device__ __forceinline__ void core_h_hd(const float2 *__restrict__ ftab, float2 ti, float v, float a,
                                          float *H, float *Hd) {
    const float av = fabsf(v);
    const int ia = (int)ti.y;
    float h, l;
    if (ia > 0 && av < 8.0f) {
        const float fv = av * 125.0f;                     // 1 / (8 / 1000)
        const int iv = (int)fv;
        const float tv = fv - (float)iv;
        const float2 *c0p = ftab + (ia - 1) * FSG_NV1 + iv, *c1p = c0p + FSG_NV1;
        const float2 t00 = __ldg(c0p), t01 = __ldg(c0p + 1), t10 = __ldg(c1p), t11 = __ldg(c1p + 1);
        const float h0 = fmaf(tv, t01.x - t00.x, t00.x), h1 = fmaf(tv, t11.x - t10.x, t10.x);
        const float l0 = fmaf(tv, t01.y - t00.y, t00.y), l1 = fmaf(tv, t11.y - t10.y, t10.y);
        h = fmaf(ti.x, h1 - h0, h0);
        l = fmaf(ti.x, l1 - l0, l0);
    } else {
        const float p = av * av - a * a - 1.5f, q = 2.0f * av * a;
        const float dr = av * p - a * q, di = av * q + a * p;
        const float w = 0.56418958f / (dr * dr + di * di);
        h = w * ((p + 0.5f) * di - q * dr);
        l = w * ((p + 0.5f) * dr + q * di);
    }
    l = copysignf(fabsf(l), v);
    *H = h;
    *Hd = fmaf(h, 2.0f * (v * v - a * a) - 1.0f, fmaf(-4.0f * a * v, l, 1.1283792f * a));
}

// wing form over the warp's depth pairs and the lane's wavelengths (MASK: some lanes outside the window)
template <int KD, bool MASK>
__device__ __forceinline__ void wing_line(const float4 *__restrict__ rp, const float2 (&g)[ADJ_P][KD / 2],
                                          const float (&X)[ADJ_P], const float (&XX)[ADJ_P],
                                          const bool (&in)[ADJ_P], float2 &s1, float2 &s2) {
#pragma unroll
    for (int j = 0; j < KD / 2; j++) {
        const float4 r0 = rp[4 * j], r1 = rp[4 * j + 1], r2 = rp[4 * j + 2], r3 = rp[4 * j + 3];
        const float2 c4 = make_float2(r0.x, r0.y), c2 = make_float2(r0.z, r0.w);
        const float2 B0 = make_float2(r1.x, r1.y), e1 = make_float2(r1.z, r1.w);
        const float2 e0 = make_float2(r2.x, r2.y), f2 = make_float2(r2.z, r2.w);
        const float2 f0 = make_float2(r3.x, r3.y), K2 = make_float2(r3.z, r3.w);
#pragma unroll
        for (int k = 0; k < ADJ_P; k++) {
            const float2 x2 = make_float2(X[k], X[k]), xx2 = make_float2(XX[k], XX[k]);
            const float2 D = __ffma2_rn(__ffma2_rn(c4, x2, c2), x2, B0);
            const float2 rD = make_float2(rcp_approx(D.x), rcp_approx(D.y));
            const float2 h = __ffma2_rn(x2, e1, e0);
            const float2 p = __ffma2_rn(xx2, f2, f0);
            const float2 inner = __ffma2_rn(p, rD, K2);
            float2 gg = g[k][j];
            if (MASK && !in[k]) gg = make_float2(0.0f, 0.0f);
            const float2 gr = __fmul2_rn(gg, rD);
            s1 = __ffma2_rn(gr, h, s1);
            s2 = __ffma2_rn(gr, inner, s2);
        }
    }
}

// point by point: lines whose core range meets the tile
template <int KD>
__device__ __forceinline__ void core_line(const AdjTileJob &J, int line, int t0, const float2 (&g)[ADJ_P][KD / 2],
                                          const float (&dl)[ADJ_P], const bool (&in)[ADJ_P], float2 &s1,
                                          float2 &s2) {
    const int nt = J.nt;
#pragma unroll
    for (int k = 0; k < ADJ_P; k++) {
        if (!in[k]) continue;
#pragma unroll
        for (int d = 0; d < KD; d++) {
            const int t = t0 + d;
            if (t >= nt) break;
            const float4 cr = __ldg(&J.crec[(size_t)line * nt + t]);
            const float v = dl[k] * cr.x, a = cr.y, a2 = a * a;
            const float s = fmaf(v, v, a2);
            float H, Hd;
            if (s >= 196.0f) {
                const float u = s - 2.0f * a2;
                const float rD = rcp_approx(fmaf(s, s, 0.25f - u));
                const float aw = 0.56418958f * a * rD;
                H = aw * (s + 0.5f);
                Hd = aw * rD * (fmaf(s, s + 2.0f * u, -s) - 0.25f);
            } else {
                core_h_hd(J.fvtab, __ldg(&J.tabi[(size_t)line * nt + t]), v, a, &H, &Hd);
            }
            const float gv = (d & 1) ? g[k][d >> 1].y : g[k][d >> 1].x;
            s1.x = fmaf(gv * cr.z, H, s1.x);
            s2.x = fmaf(gv * cr.w, Hd, s2.x);
        }
    }
}

// shared memory: mbarriers full[2], empty[2] | nsel[2] (+pad) | records [2][CL][2 ntp] float4 |
// headers [2][CL] | partials [2][CL][nw][8] float2 | line indices [2][CL]
static size_t adj_tile_smem(int nt) {
    const int ntp = adj_ntp(nt), nw = ntp / adj_kd(nt);
    return 4 * sizeof(uint64_t) + 4 * sizeof(int) + sizeof(float4) * 2 * ADJ_CL * 2 * (size_t)ntp +
           sizeof(LineHdr) * 2 * ADJ_CL + sizeof(float2) * 2 * ADJ_CL * (size_t)nw * 8 + sizeof(int) * 2 * ADJ_CL;
}

// grid: one CTA per tile; block: nw consumer warps + 1 producer warp
template <int KD>
__global__ void __launch_bounds__(32 * 17) k_adj_tiles(AdjTileJob J) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int nt = J.nt, ntp = J.ntp, nw = J.nw, nwl = J.nwl;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint64_t *full = (uint64_t *)smem_raw, *empty = full + 2;
    int *snsel = (int *)(empty + 2);
    float4 *srec = (float4 *)(snsel + 4);
    LineHdr *shdr = (LineHdr *)(srec + 2 * ADJ_CL * 2 * ntp);
    float2 *spart = (float2 *)(shdr + 2 * ADJ_CL);
    int *sidx = (int *)(spart + 2 * ADJ_CL * nw * 8);
    const int tile = blockIdx.x;
    const int lo = J.tlo[tile], hi = J.thi[tile];
    if (lo > hi) return;
    if (threadIdx.x == 0) {
        mbar_init(&full[0], 1); mbar_init(&full[1], 1);
        mbar_init(&empty[0], nw); mbar_init(&empty[1], nw);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int f1 = tile * ADJ_TW + 1, l1 = min(tile * ADJ_TW + ADJ_TW, nwl);     // 1-based wavelengths
    if (warp == nw) {
        // producer: select, stage, and reduce what the consumers leave in the partials
        const unsigned recb = (unsigned)(ntp * 32);
        auto reduce = [&](int b) {
            const int n = snsel[b];
            if (lane < n) {
                const float2 *pp = spart + (size_t)(b * ADJ_CL + lane) * nw * 8;
                double a1 = 0.0, a2 = 0.0;
                for (int w = 0; w < nw * 8; w++) { const float2 v = pp[w]; a1 += (double)v.x; a2 += (double)v.y; }
                const int j = sidx[b * ADJ_CL + lane];
                atomicAdd(&J.glin[j], a1);
                atomicAdd(&J.gvmic[j], a2);
            }
            __syncwarp();
        };
        int c = 0, cand = lo;
        bool ok = true;
        for (;;) {
            unsigned m = 0;
            bool sel = false;
            int j = 0;
            LineHdr h = {};
            while (cand <= hi && m == 0) {
                j = cand + lane;
                sel = false;
                if (lane < ADJ_CL && j <= hi) {
                    h = J.hdr[j];
                    sel = h.ileft <= h.iright && h.iright >= f1 && h.ileft <= l1;
                }
                m = __ballot_sync(0xffffffffu, sel);
                cand += ADJ_CL;
            }
            const int b = c & 1, u = c >> 1;
            if (c >= 2) {
                if (!mbar_wait(&empty[b], (u - 1) & 1)) { ok = false; break; }
                reduce(b);
            }
            if (m == 0) {                                 // no more lines: tell the consumers
                if (lane == 0) { snsel[b] = 0; mbar_arrive(&full[b]); }
                break;
            }
            const int pos = __popc(m & ((1u << lane) - 1u));
            if (sel) { sidx[b * ADJ_CL + pos] = j; shdr[b * ADJ_CL + pos] = h; }
            if (lane == 0) snsel[b] = __popc(m);
            __syncwarp();
            if (lane == 0) mbar_expect_tx(&full[b], (unsigned)__popc(m) * recb);
            __syncwarp();
            if (sel)
                tma_bulk_g2s(srec + (size_t)(b * ADJ_CL + pos) * 2 * ntp, J.prec + (size_t)j * 2 * ntp, recb, &full[b]);
            c++;
        }
        if (ok && c >= 1) {                               // the last stage
            const int b = (c - 1) & 1, u = (c - 1) >> 1;
            if (mbar_wait(&empty[b], u & 1)) reduce(b);
            else ok = false;
        }
        if (!ok && lane == 0) atomicExch(J.err, 1);
        return;
    }
    // consumers
    const int t0 = warp * KD;
    float2 g[ADJ_P][KD / 2];
    float wh[ADJ_P], wl[ADJ_P];
    int pix[ADJ_P];
#pragma unroll
    for (int k = 0; k < ADJ_P; k++) {
        pix[k] = tile * ADJ_TW + lane + 32 * k;
        const bool pin = pix[k] < nwl;
        // past the grid: the last wavelength's offsets (zero weights, finite wing values)
        wh[k] = J.wvh[min(pix[k], nwl - 1)];
        wl[k] = J.wvl[min(pix[k], nwl - 1)];
#pragma unroll
        for (int j = 0; j < KD / 2; j++) {
            const int t = t0 + 2 * j;
            g[k][j].x = (pin && t < nt) ? J.gk32[(size_t)t * nwl + pix[k]] : 0.0f;
            g[k][j].y = (pin && t + 1 < nt) ? J.gk32[(size_t)(t + 1) * nwl + pix[k]] : 0.0f;
        }
    }
    for (int c = 0;; c++) {
        const int b = c & 1, u = c >> 1;
        if (!mbar_wait(&full[b], u & 1)) { if (lane == 0) atomicExch(J.err, 1); break; }
        const int n = snsel[b];
        if (n == 0) break;
        for (int m = 0; m < n; m++) {
            const LineHdr h = shdr[b * ADJ_CL + m];
            float dl[ADJ_P], X[ADJ_P], XX[ADJ_P];
            bool in[ADJ_P];
#pragma unroll
            for (int k = 0; k < ADJ_P; k++) {
                dl[k] = (wh[k] - h.wlh) + (wl[k] - h.wll);
                X[k] = dl[k] * dl[k];
                XX[k] = X[k] * X[k];
                in[k] = pix[k] + 1 >= h.ileft && pix[k] + 1 <= h.iright;
            }
            float2 s1 = make_float2(0.0f, 0.0f), s2 = make_float2(0.0f, 0.0f);
            const float4 *rp = srec + (size_t)(b * ADJ_CL + m) * 2 * ntp + (t0 >> 1) * 4;
            if (!(h.cr < f1 || h.cl > l1)) core_line<KD>(J, sidx[b * ADJ_CL + m], t0, g, dl, in, s1, s2);
            else if (h.ileft <= f1 && h.iright >= l1) wing_line<KD, false>(rp, g, X, XX, in, s1, s2);
            else wing_line<KD, true>(rp, g, X, XX, in, s1, s2);
            float v1 = s1.x + s1.y, v2 = s2.x + s2.y;
            v1 += __shfl_xor_sync(0xffffffffu, v1, 16);
            v2 += __shfl_xor_sync(0xffffffffu, v2, 16);
            v1 += __shfl_xor_sync(0xffffffffu, v1, 8);
            v2 += __shfl_xor_sync(0xffffffffu, v2, 8);
            if (lane < 8) spart[((size_t)(b * ADJ_CL + m) * nw + warp) * 8 + lane] = make_float2(v1, v2);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[b]);
    }
}

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// workspace of the line pass for n lines
size_t fsg_line_adjoint_work(int nwl, int nt, int64_t n) {
    const int ntiles = (nwl + ADJ_TW - 1) / ADJ_TW;
    return al256(sizeof(float) * 8 * (size_t)n * adj_ntp(nt)) + al256(sizeof(float4) * (size_t)n * nt) +
           al256(sizeof(float2) * (size_t)n * nt) + al256(sizeof(LineHdr) * (size_t)n) +
           2 * al256(sizeof(int) * (size_t)ntiles) + al256(sizeof(int)) + al256(fsg_tile_span_scratch(n)) + 256;
}

int fsg_launch_line_adjoint(cudaStream_t s, const AtmView &A, const LineView &L, const VoigtTables &T,
                            const int32_t *flags, const int32_t *ileft, const int32_t *iright, const double *gkappa,
                            const float *gk32, const float *wvh, const float *wvl, double vmic, double *glin,
                            double *gvmic, void *work, int i0, int i1) {
    const int nt = A.ntau, nwl = A.nwl, ntp = adj_ntp(nt), kd = adj_kd(nt), nw = ntp / kd;
    const int64_t n = L.n;
    const int ntiles = (nwl + ADJ_TW - 1) / ADJ_TW;
    char *w = (char *)(((uintptr_t)work + 255) & ~(uintptr_t)255);
    float *prec = (float *)w; w += al256(sizeof(float) * 8 * (size_t)n * ntp);
    float4 *crec = (float4 *)w; w += al256(sizeof(float4) * (size_t)n * nt);
    float2 *tabi = (float2 *)w; w += al256(sizeof(float2) * (size_t)n * nt);
    LineHdr *hdr = (LineHdr *)w; w += al256(sizeof(LineHdr) * (size_t)n);
    int *tlo = (int *)w; w += al256(sizeof(int) * (size_t)ntiles);
    int *thi = (int *)w; w += al256(sizeof(int) * (size_t)ntiles);
    int *err = (int *)w; w += al256(sizeof(int));
    const size_t span_bytes = fsg_tile_span_scratch(n);
    void *span = (void *)w;
    if (cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess) return FSG_E_CUDA;
    size_t smem = sizeof(double) * 6 * nt * ADJ_SETUP_WARPS;
    k_adj_setup<<<(unsigned)((n + ADJ_SETUP_WARPS - 1) / ADJ_SETUP_WARPS), 32 * ADJ_SETUP_WARPS, smem, s>>>(
        A, L, T.vtab, T.fvtab, T.anode, T.aida, flags, ileft, iright, gkappa, vmic, ntp, prec, crec, tabi, hdr, glin,
        gvmic, i0, i1);
    int rc = fsg_launch_tile_span_tw(s, ADJ_TW, 0, nwl, n, hdr, tlo, thi, span, span_bytes);
    if (rc) return rc;
    AdjTileJob J;
    J.nwl = nwl; J.nt = nt; J.ntp = ntp; J.nw = nw; J.gk32 = gk32; J.wvh = wvh; J.wvl = wvl;
    J.prec = (const float4 *)prec; J.crec = crec; J.tabi = tabi; J.hdr = hdr; J.tlo = tlo; J.thi = thi;
    J.fvtab = T.fvtab; J.glin = glin; J.gvmic = gvmic; J.err = err;
    const size_t tsm = adj_tile_smem(nt);
#define ADJ_LAUNCH(K)                                                                                     \
    do {                                                                                                  \
        if (cudaFuncSetAttribute(k_adj_tiles<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm) != \
            cudaSuccess)                                                                                  \
            return FSG_E_CUDA;                                                                            \
        k_adj_tiles<K><<<ntiles, 32 * (nw + 1), tsm, s>>>(J);                                             \
    } while (0)
    if (kd == 8) ADJ_LAUNCH(8);
    else if (kd == 4) ADJ_LAUNCH(4);
    else ADJ_LAUNCH(2);
#undef ADJ_LAUNCH
    if (cudaGetLastError() != cudaSuccess) return FSG_E_CUDA;
    int herr = 0;
    if (cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return FSG_E_CUDA;
    return herr ? FSG_E_CUDA : FSG_OK;
}
