// fsg_kernels64.cu -- FP64 kernels of the line-opacity / formal-solver path (built -fmad=false).
//
//   k_tables        VoigtInit / FVoigtInit (voigt.f90:42-72, 219-251) on the device
//   k_xline_init    XlineInit (opacity.f90:65-93)
//   k_center        LineopCalc central pass (synth.f90:833-907): XlineSetup + XlineDepth,
//                   weak-line bound and centre tests, AnalyticWindow + WaveIdx windows
//   k_params_fast   block refill (synth.f90:1049-1070) into FP32 wing/core records
//   k_params_fp64   block refill into FP64 (LinCop, LinVvgt, LinAvgt) for the plain path
//   k_span, k_accum_fp64, k_wide_fp64   plain FP64 LineOpacity1 gather (opacity.f90:297-346)
//                   and the wide-line accumulation (synth.f90:981-1001)
//   k_radtran       RadTranCalc (synth.f90:1825-1866) + DiskInteg quadrature (convol.f90:233-234)
//   k_radtran_sph   RadTranCalc for spherical models (synth.f90:1868-1898): LocPrfSph along each ray
//   k_linstr        LinStrCalc (synth.f90:1774-1822), both geometries
#include "fsg_fp64.cuh"

#include <stdio.h>

// ================================================================================================
// Voigt tables: Chiarella-Reichel (1968) trapezoid sum with pole correction (voigt.f90:158-187,
// 356-393).  Complex arithmetic as gfortran expands it: naive products, Smith's division.
// ================================================================================================
struct cd { double re, im; };
__device__ __forceinline__ cd c_mul(cd a, cd b) {
    double t1 = a.re * b.re, t2 = a.im * b.im, t3 = a.re * b.im, t4 = a.im * b.re;
    return cd{ t1 - t2, t3 + t4 };
}
__device__ __forceinline__ cd c_div(cd a, cd b) {
    double ratio, div, tr, ti;
    if (fabs(b.re) < fabs(b.im)) {
        ratio = b.re / b.im; div = (b.re * ratio) + b.im;
        tr = (a.re * ratio) + a.im; ti = (a.im * ratio) - a.re;
    } else {
        ratio = b.im / b.re; div = (b.im * ratio) + b.re;
        tr = (a.im * ratio) + a.re; ti = a.im - (a.re * ratio);
    }
    return cd{ tr / div, ti / div };
}

__device__ cd cr_sum(double a, double av) {
    const double HH = 0.5;
    cd z{ av, a }, z2 = c_mul(z, z);
    cd s = c_div(cd{ 1.0, 0.0 }, z);
    for (int n = 1; n <= 16; n++) {
        double nh = (double)n * HH;
        double e = exp(-nh * nh);
        cd num{ (2.0 * z.re) * e, (2.0 * z.im) * e };
        cd q = c_div(num, cd{ z2.re - nh * nh, z2.im });
        s.re = s.re + q.re; s.im = s.im + q.im;
    }
    double c = HH / FSG_PI;
    s = cd{ -(c * s.im), c * s.re };
    if (a < 6.0) {
        double p = 2.0 * FSG_PI * a / HH;
        double th = 2.0 * FSG_PI * (2.0 * av - round(2.0 * av));
        double sn = sin(0.5 * th);
        double redd = -(2.0 * exp(0.5 * p) * sinh(0.5 * p)) + exp(p) * 2.0 * (sn * sn);
        double imdd = exp(p) * sin(th);
        double ex = exp(a * a - av * av), ang = -2.0 * a * av;
        cd num{ 2.0 * (ex * cos(ang)), 2.0 * (ex * sin(ang)) };
        cd q = c_div(num, cd{ redd, imdd });
        s.re = s.re + q.re; s.im = s.im + q.im;
    }
    return s;
}

__global__ void k_tables(float *vtab, float2 *fvtab, double *anode, double *aida) {
    const double dv = 8.0 / 1000.0, dt = 2.8284271247461903 / 400.0;
    int iv = blockIdx.x * blockDim.x + threadIdx.x;   // 0..1001
    int ia = blockIdx.y;                              // 0..401
    double aa = ((double)ia * dt) * ((double)ia * dt);
    if (iv == 0) {
        anode[ia] = aa;
        if (ia < FSG_NVA) {
            double an1 = ((double)(ia + 1) * dt) * ((double)(ia + 1) * dt);
            aida[ia] = 1.0 / (an1 - aa);
        } else aida[ia] = 0.0;
    }
    if (iv >= FSG_NV1) return;
    double vv = (double)iv * dv;
    double h, l;
    if (aa <= 0.0) {
        h = exp(-fmin(vv * vv, 700.0));
        int m = 2 * (int)llround(2.0 * vv);
        double x0 = vv - 0.25 * (double)m, p = 0.0;
        for (int n = -31; n <= 31; n += 2) {
            double t = x0 - 0.25 * (double)n;
            p = p + exp(-(t * t)) / (double)(m + n);
        }
        l = (2.0 / FSG_PI) * p;
    } else {
        cd s = cr_sum(aa, vv);
        h = s.re; l = s.im;
    }
    vtab[ia * FSG_NV1 + iv] = (float)h;
    fvtab[ia * FSG_NV1 + iv] = make_float2((float)h, (float)l);
}

// the four VgtTab entries of one bilinear cell side by side
__global__ void k_vtab4(const float *vtab, float4 *vtab4) {
    int iv = blockIdx.x * blockDim.x + threadIdx.x;   // 0..NVV-1
    int r = blockIdx.y;                               // 0..NVA-1
    if (iv >= FSG_NVV) return;
    const float *p0 = vtab + r * FSG_NV1 + iv, *p1 = p0 + FSG_NV1;
    vtab4[r * FSG_NV1 + iv] = make_float4(p0[0], p0[1], p1[0], p1[1]);
}

// (H, L) at two neighbouring v nodes side by side (the last node repeated at the row end)
__global__ void k_fvtab2(const float2 *fvtab, float4 *fvtab2) {
    int iv = blockIdx.x * blockDim.x + threadIdx.x;   // 0..NV1-1
    int r = blockIdx.y;                               // 0..NA1-1
    if (iv >= FSG_NV1) return;
    const float2 a = fvtab[r * FSG_NV1 + iv], b = fvtab[r * FSG_NV1 + min(iv + 1, FSG_NV1 - 1)];
    fvtab2[r * FSG_NV1 + iv] = make_float4(a.x, a.y, b.x, b.y);
}

int fsg_build_tables(VoigtTables *t, cudaStream_t s, std::string *err) {
    cudaError_t e;
    if ((e = cudaMalloc(&t->vtab4, sizeof(float4) * FSG_NVA * FSG_NV1)) != cudaSuccess ||
        (e = cudaMalloc(&t->vtab, sizeof(float) * FSG_NA1 * FSG_NV1)) != cudaSuccess ||
        (e = cudaMalloc(&t->fvtab, sizeof(float2) * FSG_NA1 * FSG_NV1)) != cudaSuccess ||
        (e = cudaMalloc(&t->fvtab2, sizeof(float4) * FSG_NA1 * FSG_NV1)) != cudaSuccess ||
        (e = cudaMalloc(&t->anode, sizeof(double) * FSG_NA1)) != cudaSuccess ||
        (e = cudaMalloc(&t->aida, sizeof(double) * FSG_NA1)) != cudaSuccess) {
        *err = fsg_cuda_msg(e, "table allocation");
        return FSG_E_NOMEM;
    }
    dim3 grid((FSG_NV1 + 127) / 128, FSG_NA1);
    k_tables<<<grid, 128, 0, s>>>(t->vtab, t->fvtab, t->anode, t->aida);
    if ((e = cudaGetLastError()) != cudaSuccess) { *err = fsg_cuda_msg(e, "k_tables"); return FSG_E_CUDA; }
    k_vtab4<<<dim3((FSG_NVV + 127) / 128, FSG_NVA), 128, 0, s>>>(t->vtab, t->vtab4);
    if ((e = cudaGetLastError()) != cudaSuccess) { *err = fsg_cuda_msg(e, "k_vtab4"); return FSG_E_CUDA; }
    k_fvtab2<<<dim3((FSG_NV1 + 127) / 128, FSG_NA1), 128, 0, s>>>(t->fvtab, t->fvtab2);
    if ((e = cudaGetLastError()) != cudaSuccess) { *err = fsg_cuda_msg(e, "k_fvtab2"); return FSG_E_CUDA; }
    return FSG_OK;
}

void fsg_free_tables(VoigtTables *t) {
    cudaFree(t->vtab); cudaFree(t->vtab4); cudaFree(t->fvtab); cudaFree(t->fvtab2); cudaFree(t->anode); cudaFree(t->aida);
    t->vtab = nullptr; t->vtab4 = nullptr; t->fvtab = nullptr; t->fvtab2 = nullptr; t->anode = nullptr; t->aida = nullptr;
}

// ================================================================================================
// XlineInit (opacity.f90:65-93): rows of A.xi
// ================================================================================================
__global__ void k_xline_init(int nt, const double *T, const double *xne, const double *rho,
                             const float *h1, const float *he1, const float *h2, double h2brd,
                             double *xi) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    double Temp = T[t], Xne = xne[t];
    double Vh = sqrt(2.0 * FSG_KBOLT * Temp / FSG_MH);
    double np = (double)h1[t] + 0.412265 * (double)he1[t];
    if (h2brd > 0.0) np = np + h2brd * 0.874307 * (double)h2[t];
    const double erg2ev = 1e-7 / 1.602176634e-19;
    xi[XI_NPRTB * nt + t] = np;
    xi[XI_GVWPRT * nt + t] = 17.0 * pow(Vh, 0.6) * np;
    xi[XI_TEMP6 * nt + t] = pow(Temp / 1e4, 1.0 / 6.0) * Xne;
    xi[XI_TEMP3 * nt + t] = pow(Temp / 1e4, 0.3) * np;
    xi[XI_KBT * nt + t] = FSG_KBOLT * Temp;
    xi[XI_KBET * nt + t] = FSG_KBOLT * erg2ev * Temp;
    xi[XI_T * nt + t] = Temp;
    xi[XI_XNE * nt + t] = Xne;
    xi[XI_RHO * nt + t] = rho[t];
}

void fsg_launch_xline_init(cudaStream_t s, int nt, const double *T, const double *xne, const double *rho,
                           const float *h1, const float *he1, const float *h2, double h2brd, double *xi) {
    k_xline_init<<<(nt + 127) / 128, 128, 0, s>>>(nt, T, xne, rho, h1, he1, h2, h2brd, xi);
}

// ================================================================================================
// Central pass (synth.f90:833-907).  One thread per line and one sweep over depth: XlineDepth once per
// depth feeds the LinCop bound test against the continuum, the single-line opacity at the line centre
// (LineOpacity2) and AnalyticWindow; no Ntau-long arrays are held.
// ================================================================================================
__device__ __forceinline__ double center_shift(const AtmView &A, int ihe, int t) {
    return (ihe > 0) ? A.heshf[(ihe - 1) * A.ntau + t] : 0.0;
}

// Eight 128-thread CTAs per SM (64 registers, a few spilled): the sweep is bound by the FP64 pipe,
// and the extra resident warps hide more of its latency (177 -> 150 ms on the 1e8-line list).
__global__ void __launch_bounds__(128, 8) k_center(AtmView A, LineView L, const float *__restrict__ vtab,
                         const double *__restrict__ anode, const double *__restrict__ aida,
                         int32_t *flags, int32_t *ileft, int32_t *iright, unsigned long long *nkeep) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n) return;
    const int nt = A.ntau;
    int f = line_input_flags(L, i, 0);
    double wlc = L.wl[i] - A.wfirst;
    XCoef XC;
    xline_setup(A, L, i, wlc, f, &XC);
    if (XC.IxHe > 0) f |= (XC.IxHe << 8);
    int ihe = XC.IxHe;
    int iwl = waveidx(A, wlc);
    double dW = (wlc - A.wave[iwl - 1]) / (A.wave[iwl] - A.wave[iwl - 1]);
    // One sweep over depth gives the three maxima the reference takes in turn (synth.f90:876-907):
    // (1) the upper bound LinCop / ContOpac (H(a, v) <= 1), (2) the single-line opacity at the line
    // centre (LineOpacity2 at Wl = Wlcent) and (3) the AnalyticWindow half-width (opacity.f90:678-710).
    // Each is a maximum over depths of per-depth values that do not depend on the others, so computing
    // XlineDepth once per depth for all three gives the reference's tests and windows exactly; the
    // later maxima are used only when the earlier tests keep the line.
    const double iSqrtPi = 0.5641895835477563;
    double mx1 = -1.0e308, mx2 = -1.0e308, dWwin = 0.0;
    for (int t = 0; t < nt; t++) {
        double cop, vv, av;
        xline_depth(A, t, XC, &cop, &vv, &av);
        const double co = cont_center(A, iwl, dW, t);
        mx1 = fmax(mx1, (A.motype == 1) ? cop / (co * A.contstd[t]) : cop / co);
        double dWl = 0.0;
        if (ihe > 0) dWl = 0.0 - center_shift(A, ihe, t);
        double lo = hvoigt64(vtab, anode, aida, av, dWl * vv) * cop;
        if (A.motype == 1) lo = lo / A.contstd[t];
        mx2 = fmax(mx2, lo / co);
        double r = cop / (A.epsopac * co);
        if (A.motype == 1) r = r / A.contstd[t];
        if (r <= 1.0) continue;
        double w = sqrt(log(r) + fmax(0.0, av * (r * iSqrtPi - av))) / vv;
        if (ihe > 0) w = w + fabs(center_shift(A, ihe, t));
        dWwin = fmax(dWwin, w);
    }
    int il = 1, ir = A.nwl;
    if (mx1 < A.epsopac || mx2 < A.epsopac) {
        f |= FSG_F_WEAK;
    } else {
        il = waveidx(A, wlc - dWwin);                      // WaveIdx (synth.f90:904-906)
        ir = waveidx(A, wlc + dWwin) + 1;
        if (ir > A.nwl) ir = A.nwl;
    }
    flags[i] = f; ileft[i] = il; iright[i] = ir;
    // warp-aggregated count of retained lines
    unsigned m = __ballot_sync(__activemask(), !(f & FSG_F_WEAK));
    if ((threadIdx.x & 31) == (__ffs(__activemask()) - 1) && m) atomicAdd(nkeep, (unsigned long long)__popc(m));
}

void fsg_launch_center(cudaStream_t s, const AtmView &A, const LineView &L, const VoigtTables &T,
                       int32_t *flags, int32_t *ileft, int32_t *iright, unsigned long long *nkeep) {
    if (L.n <= 0) return;
    unsigned nb = (unsigned)((L.n + 127) / 128);
    k_center<<<nb, 128, 0, s>>>(A, L, T.vtab, T.anode, T.aida, flags, ileft, iright, nkeep);
}

// ================================================================================================
// Block refill: per retained line of the block, XlineSetup once then XlineDepth over depths.
// ================================================================================================

// Line j of the block is list line idx[j0 + j * stride].  One warp per group of 32 lines: lane k
// runs XlineSetup for line k of the group into shared memory, then the warp walks the group's
// (line, depth) pairs in record order, one pair per lane, so that each store of wing and core
// records covers consecutive records of the arrays.  The per-line maximum core half-width and the
// minimum vv2 are reduced over each line's run of lanes with shuffles (a run is a line's depths in
// one step) and merged into shared memory by the run's first lane; lane k then writes the header of
// line k.  Both reductions are exact (max / min), so the records and headers do not depend on the
// order in which depths are taken.
#define PF_WARPS 4
__global__ void __launch_bounds__(PF_WARPS * 32)
k_params_fast(AtmView A, LineView L, const int64_t *__restrict__ idx, int64_t j0, int64_t stride,
              int64_t nb, const int32_t *__restrict__ flags,
              const int32_t *__restrict__ ileft, const int32_t *__restrict__ iright,
              const double *__restrict__ anode, const double *__restrict__ aida,
              WingRec *wing, CoreRec *core, LineHdr *hdr) {
    __shared__ XCoef xs[PF_WARPS][32];
    __shared__ unsigned long long hcs[PF_WARPS][32];   // bits of hcore + 1 (0: no depth has a core)
    __shared__ unsigned vms[PF_WARPS][32];             // bits of the smallest vv2 (non-negative floats)
    const int wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t jb = ((int64_t)blockIdx.x * PF_WARPS + wp) * 32;
    if (jb >= nb) return;                               // whole warps only: no block barrier below
    const int ng = (nb - jb < 32) ? (int)(nb - jb) : 32;
    const int nt = A.ntau;
    int64_t i = 0; int f = 0; double wlc = 0.0;
    if (lane < ng) {
        i = idx[j0 + (jb + lane) * stride];
        f = flags[i];
        wlc = L.wl[i] - A.wfirst;
        xline_setup(A, L, i, wlc, f, &xs[wp][lane]);
    }
    hcs[wp][lane] = 0ull;
    vms[wp][lane] = __float_as_uint(3.0e38f);
    __syncwarp();
    const int tot = ng * nt;
    WingRec *wg = wing + (size_t)jb * nt;
    CoreRec *cg = core + (size_t)jb * nt;
    // pair p = lane + step: line ln = p / nt, depth t = p % nt, advanced by 32 per step
    int ln = lane / nt, t = lane - (lane / nt) * nt;
    for (int p0 = 0; p0 < tot; p0 += 32) {
        const int p = p0 + lane;
        const bool on = p < tot;
        double hc = -1.0;          // this pair's core half-width (s < 196), -1 when none
        float vv2 = 3.0e38f;
        if (on) {
            const XCoef &XC = xs[wp][ln];
            double cop, vv, av;
            xline_depth(A, t, XC, &cop, &vv, &av);
            if (A.motype == 1) cop = cop / A.contstd[t];     // LineOpacity1 divides the sum by ContOpacStd
            double a2 = av * av;
            WingRec w;
            w.vv2 = (float)(vv * vv);
            w.c2m1 = (float)(a2 - 0.5);
            w.twoA = (float)(2.0 * a2);
            w.c1 = (float)(cop * av * FSG_SQRTPIINV);
            vv2 = w.vv2;
            CoreRec c;
            c.vv = vv; c.cop = (float)cop; c.a = (float)av; c.pad0 = c.pad1 = 0;
            // table row and weight of a in FP64 (sqrt(a) nodes, voigt.f90:84-92); ia = 0: a >= 8
            if (!(av < 8.0)) { c.ia = 0; c.ua = 0.0f; }
            else if (av < anode[1]) { c.ia = 1; c.ua = (float)(av * aida[0]); }
            else {
                const int ia = min((int)(sqrt(av) * (1.0 / (2.8284271247461903 / 400.0))) + 1, FSG_NVA);
                c.ia = ia;
                c.ua = (float)((av - anode[ia - 1]) * aida[ia - 1]);
            }
            wg[p] = w;
            cg[p] = c;
            // the accumulation evaluates the core form where fl32(dl^2 vv2 + c2m1) < 195.5; a margin
            // of 0.05 in s and 1e-5 in dl covers the FP32 rounding of the records and of dl^2
            double q = 196.05 - a2;
            if (q > 0.0) hc = sqrt(q) / vv * (1.0 + 1e-5);
        }
        // segmented reduction over the run of lanes that share this lane's line (lanes past the
        // last pair form their own run at the end); the run's first lane ends with the run's value
        #pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            double oh = __shfl_down_sync(0xffffffffu, hc, off);
            float ov = __shfl_down_sync(0xffffffffu, vv2, off);
            if (lane + off < 32 && t + off < nt) { hc = fmax(hc, oh); vv2 = fminf(vv2, ov); }
        }
        if (on && (lane == 0 || t == 0)) {
            if (hc >= 0.0) atomicMax(&hcs[wp][ln], (unsigned long long)__double_as_longlong(hc) + 1ull);
            atomicMin(&vms[wp][ln], __float_as_uint(vv2));
        }
        t += 32;
        while (t >= nt) { t -= nt; ln++; }
    }
    __syncwarp();
    if (lane >= ng) return;
    const unsigned long long hb = hcs[wp][lane];
    const double hcore = hb ? __longlong_as_double((long long)(hb - 1ull)) : -1.0;
    const float vv2min = __uint_as_float(vms[wp][lane]);
    LineHdr h;
    h.wlh = (float)wlc;
    h.wll = (float)(wlc - (double)h.wlh);
    h.ileft = ileft[i]; h.iright = iright[i];
    h.cl = 1; h.cr = 0;
    if (f & FSG_F_WEAK) { h.ileft = 1; h.iright = 0; }    // rejected line (batched lists): empty window
    else if (hcore >= 0.0) {
        // 1-based indices of the first wavelength >= wlc - hcore and the last <= wlc + hcore,
        // widened by one wavelength and clipped to the window
        int a = lower_index(A.wave, A.nwl, wlc - hcore) + 1;
        int b = lower_index(A.wave, A.nwl, wlc + hcore);
        if (b < A.nwl && A.wave[b] == wlc + hcore) b++;
        int cl = max(a - 1, h.ileft), cr = min(b + 1, h.iright);
        if (cl <= cr) { h.cl = cl; h.cr = cr; }
    }
    // x offset that silences a point in the wing pass: with dl^2 replaced by 1e19 / min vv2, every
    // depth has t >= 1e19, so t^2 >= 1e38 and the FP32 reciprocal (flush-to-zero) is exactly 0 while
    // c1 (t + 1) stays finite; the point then adds exactly 0
    h.pad0 = __float_as_int(1.0e19f / vv2min);
    h.pad1 = 0;
    hdr[jb + lane] = h;
}

void fsg_launch_params_fast(cudaStream_t s, const AtmView &A, const LineView &L, const int64_t *idx,
                            int64_t j0, int64_t stride, int64_t nb, const int32_t *flags, const int32_t *ileft,
                            const int32_t *iright, const VoigtTables &T, WingRec *wing, CoreRec *core,
                            LineHdr *hdr) {
    if (nb <= 0) return;
    const int64_t per = PF_WARPS * 32;
    k_params_fast<<<(unsigned)((nb + per - 1) / per), PF_WARPS * 32, 0, s>>>(A, L, idx, j0, stride, nb, flags, ileft,
                                                                            iright, T.anode, T.aida, wing, core, hdr);
}

// FP64 parameters for the plain path: p64[j][t] = (LinCop, LinVvgt, LinAvgt)
__global__ void k_params_fp64(AtmView A, LineView L, int64_t i0, int64_t nb,
                              const int32_t *__restrict__ flags, double3 *p64) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nb) return;
    int64_t i = i0 + j;
    int f = flags[i];
    if (f & FSG_F_WEAK) return;
    double wlc = L.wl[i] - A.wfirst;
    XCoef XC;
    xline_setup(A, L, i, wlc, f, &XC);
    for (int t = 0; t < A.ntau; t++) {
        double cop, vv, av;
        xline_depth(A, t, XC, &cop, &vv, &av);
        p64[(size_t)j * A.ntau + t] = make_double3(cop, vv, av);
    }
}

void fsg_launch_params_fp64(cudaStream_t s, const AtmView &A, const LineView &L, int64_t i0, int64_t nb,
                            const int32_t *flags, double3 *p64) {
    if (nb <= 0) return;
    k_params_fp64<<<(unsigned)((nb + 127) / 128), 128, 0, s>>>(A, L, i0, nb, flags, p64);
}

// ================================================================================================
// Plain FP64 path: Lstart/Lstop pointers (synth.f90:955-978), wide lines (synth.f90:981-1001)
// and the per-wavelength gather LineOpacity1 (opacity.f90:297-346).
// ================================================================================================
__global__ void k_span(int64_t n, const int32_t *flags, const int32_t *ileft, const int32_t *iright,
                       int *lstart, int *lstop) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int f = flags[i];
    if ((f & FSG_F_WEAK) || (f & FSG_F_WIDE)) return;
    for (int w = ileft[i]; w <= iright[i]; w++) {
        atomicMin(&lstart[w - 1], (int)(i + 1));
        atomicMax(&lstop[w - 1], (int)(i + 1));
    }
}

void fsg_launch_span(cudaStream_t s, int64_t n, const int32_t *flags, const int32_t *ileft,
                     const int32_t *iright, int *lstart, int *lstop) {
    if (n <= 0) return;
    k_span<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(n, flags, ileft, iright, lstart, lstop);
}

// One warp per wavelength; lanes stride the depths.  Lines l1..l2 (1-based), block offset loff.
#define FP64_MAXD 4   // up to 128 depths
__global__ void k_accum_fp64(AtmView A, const double *__restrict__ wl, int iwl1, int iwl2,
                             const int *__restrict__ lstart, const int *__restrict__ lstop,
                             const int32_t *__restrict__ flags, const int32_t *__restrict__ ileft,
                             const int32_t *__restrict__ iright, int64_t loff, const double3 *__restrict__ p64,
                             const float *__restrict__ vtab, const double *__restrict__ anode,
                             const double *__restrict__ aida, double *lineopac, double *evals) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    int iwl = iwl1 + warp;
    if (iwl > iwl2) return;
    const int nt = A.ntau;
    double acc[FP64_MAXD];
#pragma unroll
    for (int k = 0; k < FP64_MAXD; k++) acc[k] = 0.0;
    double Wl = A.wave[iwl - 1];
    int l1 = lstart[iwl - 1], l2 = lstop[iwl - 1];
    double cnt = 0.0;
    for (int il = l1; il <= l2; il++) {
        int f = flags[il - 1];
        if ((f & FSG_F_WEAK) || (f & FSG_F_WIDE) || iwl < ileft[il - 1] || iwl > iright[il - 1]) continue;
        int ihe = (f >> 8) & 255;
        double dWl0 = Wl - (wl[il - 1] - A.wfirst);
        const double3 *p = p64 + (size_t)(il - 1 - loff) * nt;
#pragma unroll
        for (int k = 0; k < FP64_MAXD; k++) {
            int t = lane + 32 * k;
            if (t < nt) {
                double dWl = dWl0;
                if (ihe > 0) dWl = dWl0 - A.heshf[(ihe - 1) * nt + t];
                double3 q = p[t];
                double V = dWl * q.y;
                acc[k] = acc[k] + hvoigt64(vtab, anode, aida, q.z, V) * q.x;
            }
        }
        cnt += 1.0;
    }
    double *dst = lineopac + (size_t)(iwl - 1) * nt;
#pragma unroll
    for (int k = 0; k < FP64_MAXD; k++) {
        int t = lane + 32 * k;
        if (t < nt) {
            double v = acc[k];
            if (A.motype == 1) v = v / A.contstd[t];
            dst[t] = dst[t] + v;
        }
    }
    if (lane == 0 && cnt > 0.0) atomicAdd(evals, cnt * nt);
}

void fsg_launch_accum_fp64(cudaStream_t s, const AtmView &A, const double *wl, int iwl1, int iwl2,
                           const int *lstart, const int *lstop, const int32_t *flags, const int32_t *ileft,
                           const int32_t *iright, int64_t loff, const double3 *p64, const VoigtTables &T,
                           double *lineopac, double *evals) {
    int nw = iwl2 - iwl1 + 1;
    if (nw <= 0) return;
    k_accum_fp64<<<(nw + 7) / 8, 256, 0, s>>>(A, wl, iwl1, iwl2, lstart, lstop, flags, ileft, iright, loff,
                                              p64, T.vtab, T.anode, T.aida, lineopac, evals);
}

// Wide lines, in line order, each over its own window (LineOpacity2): one warp per wavelength,
// looping over the wide-line list so the per-wavelength additions keep the reference's order.
__global__ void k_wide_fp64(AtmView A, LineView L, int nwide, const int64_t *__restrict__ widx,
                            const int32_t *__restrict__ flags, const int32_t *__restrict__ ileft,
                            const int32_t *__restrict__ iright, const double3 *__restrict__ pw,
                            const float *__restrict__ vtab, const double *__restrict__ anode,
                            const double *__restrict__ aida, int wlo, int whi, double *lineopac,
                            double *evals) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    int iwl = wlo + warp;
    if (iwl > whi) return;
    const int nt = A.ntau;
    double Wl = A.wave[iwl - 1];
    double *dst = lineopac + (size_t)(iwl - 1) * nt;
    double cnt = 0.0;
    for (int q = 0; q < nwide; q++) {
        int64_t i = widx[q];
        if (iwl < ileft[i] || iwl > iright[i]) continue;
        int f = flags[i], ihe = (f >> 8) & 255;
        double dWl0 = Wl - (L.wl[i] - A.wfirst);
        for (int t = lane; t < nt; t += 32) {
            double dWl = dWl0;
            if (ihe > 0) dWl = dWl0 - A.heshf[(ihe - 1) * nt + t];
            double3 p = pw[(size_t)q * nt + t];
            double v = hvoigt64(vtab, anode, aida, p.z, dWl * p.y) * p.x;
            if (A.motype == 1) v = v / A.contstd[t];
            dst[t] = dst[t] + v;
        }
        cnt += 1.0;
    }
    if (lane == 0 && cnt > 0.0) atomicAdd(evals, cnt * nt);
}

__global__ void k_params_wide(AtmView A, LineView L, int nwide, const int64_t *widx,
                              const int32_t *flags, double3 *pw) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nwide) return;
    int64_t i = widx[q];
    double wlc = L.wl[i] - A.wfirst;
    XCoef XC;
    xline_setup(A, L, i, wlc, flags[i], &XC);
    for (int t = 0; t < A.ntau; t++) {
        double cop, vv, av;
        xline_depth(A, t, XC, &cop, &vv, &av);
        pw[(size_t)q * A.ntau + t] = make_double3(cop, vv, av);
    }
}

void fsg_launch_wide_fp64(cudaStream_t s, const AtmView &A, const LineView &L, int nwide, const int64_t *widx,
                          const int32_t *flags, const int32_t *ileft, const int32_t *iright, double3 *pw,
                          const VoigtTables &T, int wlo, int whi, double *lineopac, double *evals) {
    if (nwide <= 0 || whi < wlo) return;
    k_params_wide<<<(nwide + 63) / 64, 64, 0, s>>>(A, L, nwide, widx, flags, pw);
    int nw = whi - wlo + 1;
    k_wide_fp64<<<(nw + 7) / 8, 256, 0, s>>>(A, L, nwide, widx, flags, ileft, iright, pw, T.vtab, T.anode,
                                             T.aida, wlo, whi, lineopac, evals);
}

// ================================================================================================
// RadTranCalc + disk integration.  A CTA takes RT_LW wavelengths; the two opacity columns
// (continuum, continuum + line) of each wavelength are staged in shared memory with coalesced
// loads, TauStep / CentDer / U run over depths in parallel, then one thread per
// (wavelength, kind, mu) sweeps the depths (LocPrfPP, solver.f90:123-179).
// ================================================================================================
#define RT_LW 8
#define RT_MAXT 128
#define RT_MAXMU 16

__global__ void k_radtran(AtmView A, const double *__restrict__ lineopac, const double *__restrict__ rhox,
                          int nmu, const double *__restrict__ xmu, const double *__restrict__ wmu,
                          double *spl, double *spc, double *sfl, double *sfc) {
    extern __shared__ double sm[];
    const int nt = A.ntau;
    const int w0 = blockIdx.x * RT_LW;
    const int nw = min(RT_LW, A.nwl - w0);
    // layout: X[kind][w][t], S[w][t], D[kind][w][t], R[kind][w][t] (derivative), U[kind][w][t]
    double *X = sm, *S = X + 2 * RT_LW * nt, *D = S + RT_LW * nt, *R = D + 2 * RT_LW * nt,
           *U = R + 2 * RT_LW * nt, *I = U + 2 * RT_LW * nt;      // I[kind][w][mu]
    const double PlkC1 = FSG_HC * FSG_VC * 1e13 / FSG_KBOLT;
    for (int e = threadIdx.x; e < nw * nt; e += blockDim.x) {
        int w = e / nt, t = e - w * nt;
        size_t g = (size_t)(w0 + w) * nt + t;
        double c = A.contopac[g];
        X[(0 * RT_LW + w) * nt + t] = c;
        X[(1 * RT_LW + w) * nt + t] = c + lineopac[g];
        double wl = A.wave[w0 + w] + A.wfirst;
        double C1 = PlkC1 / wl, C2 = exp(50.7649141 - 5.0 * log(wl));
        S[w * nt + t] = C2 / (exp(C1 / A.xi[XI_T * nt + t]) - 1.0);
    }
    __syncthreads();
    // TauStep at mu = 1 (solver.f90:591-615)
    for (int e = threadIdx.x; e < 2 * nw * nt; e += blockDim.x) {
        int kw = e / nt, t = e - kw * nt;            // kw = kind * nw + w
        int kind = kw / nw, w = kw - kind * nw;
        const double *x = X + (kind * RT_LW + w) * nt;
        double *d = D + (kind * RT_LW + w) * nt;
        if (t == 0) {
            double Dx1 = (rhox[1] - rhox[0]) / 1.0;
            double Yp = (x[1] - x[0]) / Dx1;
            d[0] = Dx1 * (x[1] + 2.0 * x[0] + Dx1 / 2.0 * Yp) / 3.0;
        } else if (t < nt - 1) {
            int k = t + 1;
            double Dx = (rhox[k - 1] - rhox[k - 2]) / 1.0, Dx1 = (rhox[k] - rhox[k - 1]) / 1.0;
            double Der = (x[k - 1] - x[k - 2]) / Dx, Der1 = (x[k] - x[k - 1]) / Dx1, Yp;
            if (Der * Der1 > 0.0) {
                double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0;
                Yp = (Der / (Lambda * Der1 + (1.0 - Lambda) * Der)) * Der1;
            } else Yp = 0.0;
            d[k - 1] = Dx1 * (x[k] + 2.0 * x[k - 1] + Dx1 / 2.0 * Yp) / 3.0;
        } else d[nt - 1] = 0.0;
    }
    __syncthreads();
    // CentDer of the source function on each Deltau scale (solver.f90:618-647)
    for (int e = threadIdx.x; e < 2 * nw * nt; e += blockDim.x) {
        int kw = e / nt, t = e - kw * nt;
        int kind = kw / nw, w = kw - kind * nw;
        const double *d = D + (kind * RT_LW + w) * nt, *y = S + w * nt;
        double *r = R + (kind * RT_LW + w) * nt;
        if (t == 0) r[0] = (y[1] - y[0]) / d[0];
        else if (t == nt - 1) r[nt - 1] = (y[nt - 1] - y[nt - 2]) / d[nt - 2];
        else {
            int k = t + 1;
            double Dx = d[k - 2], Dx1 = d[k - 1];
            double InvDx = 1.0 / Dx, InvDx1 = 1.0 / Dx1;
            double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0, Lambda1 = 1.0 - Lambda;
            double Der = (y[k - 1] - y[k - 2]) * InvDx, Der1 = (y[k] - y[k - 1]) * InvDx1;
            r[k - 1] = (Der * Der1 > 0.0) ? (Der / (Lambda * Der1 + Lambda1 * Der)) * Der1 : 0.0;
        }
    }
    __syncthreads();
    // Bezier control term U (solver.f90:136-138)
    for (int e = threadIdx.x; e < 2 * nw * nt; e += blockDim.x) {
        int kw = e / nt, t = e - kw * nt;
        int kind = kw / nw, w = kw - kind * nw;
        if (t >= nt - 1) continue;
        const double *d = D + (kind * RT_LW + w) * nt, *r = R + (kind * RT_LW + w) * nt, *y = S + w * nt;
        U[(kind * RT_LW + w) * nt + t] = 0.5 * (y[t] + 0.5 * d[t] * r[t] + y[t + 1] - 0.5 * d[t] * r[t + 1]);
    }
    __syncthreads();
    // sweeps: one thread per (kind, w, mu)
    for (int e = threadIdx.x; e < 2 * nw * nmu; e += blockDim.x) {
        int kw = e / nmu, im = e - kw * nmu;
        int kind = kw / nw, w = kw - kind * nw;
        const double *d = D + (kind * RT_LW + w) * nt, *u = U + (kind * RT_LW + w) * nt, *y = S + w * nt;
        double Imu = 1.0 / xmu[im], Y = y[nt - 1];
        for (int k = nt - 2; k >= 0; k--) {
            double Eps, Alpha, Beta, Gamma;
            delo_coef(d[k] * Imu, Eps, Alpha, Beta, Gamma);
            Y = Y * Eps + Alpha * y[k] + Beta * y[k + 1] + Gamma * u[k];
        }
        I[(kind * RT_LW + w) * nmu + im] = Y;
        double *out = (kind == 0) ? spc : spl;
        if (out) out[(size_t)(w0 + w) * nmu + im] = Y;
    }
    __syncthreads();
    // disk integration without broadening: Sf = sum over mu of Sp * Wmu (convol.f90:233-234)
    for (int e = threadIdx.x; e < 2 * nw; e += blockDim.x) {
        int kind = e / nw, w = e - kind * nw;
        double a = 0.0;
        for (int im = 0; im < nmu; im++) a = a + I[(kind * RT_LW + w) * nmu + im] * wmu[im];
        double *out = (kind == 0) ? sfc : sfl;
        if (out) out[w0 + w] = a;
    }
}

size_t fsg_radtran_smem(int nt, int nmu) {
    return sizeof(double) * ((size_t)(2 + 1 + 2 + 2 + 2) * RT_LW * nt + 2 * RT_LW * nmu);
}

int fsg_launch_radtran(cudaStream_t s, const AtmView &A, const double *lineopac, const double *rhox,
                       int nmu, const double *xmu, const double *wmu, double *spl, double *spc,
                       double *sfl, double *sfc) {
    size_t sm = fsg_radtran_smem(A.ntau, nmu);
    static int attr_set = 0;
    if (!attr_set) {
        cudaFuncSetAttribute(k_radtran, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr_set = 1;
    }
    int nb = (A.nwl + RT_LW - 1) / RT_LW;
    k_radtran<<<nb, 128, sm, s>>>(A, lineopac, rhox, nmu, xmu, wmu, spl, spc, sfl, sfc);
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}

// RadTranCalc for spherical models (synth.f90:1868-1898): LocPrfSph along each ray.  A CTA stages
// RT_LW wavelengths' opacity columns and Planck source as k_radtran does; then one thread per
// (wavelength, kind, ray) runs delo_ray, whose steps come from that ray's own column-mass scale.
// With spl and sfl null only the continuum is solved (as MagRadTranCalc needs).
__global__ void k_radtran_sph(AtmView A, const double *__restrict__ lineopac, RayView R,
                              const double *__restrict__ wmu, double *spl, double *spc, double *sfl, double *sfc) {
    extern __shared__ double sm[];
    const int nt = A.ntau, nmu = R.nmu;
    const int w0 = blockIdx.x * RT_LW;
    const int nw = min(RT_LW, A.nwl - w0);
    const int nk = (spl || sfl) ? 2 : 1;                    // kinds computed: 0 continuum, 1 line
    double *X = sm, *S = X + 2 * RT_LW * nt, *I = S + RT_LW * nt;   // X[kind][w][t], S[w][t], I[kind][w][mu]
    const double PlkC1 = FSG_HC * FSG_VC * 1e13 / FSG_KBOLT;
    for (int e = threadIdx.x; e < nw * nt; e += blockDim.x) {
        int w = e / nt, t = e - w * nt;
        size_t g = (size_t)(w0 + w) * nt + t;
        double c = A.contopac[g];
        X[(0 * RT_LW + w) * nt + t] = c;
        if (nk == 2) X[(1 * RT_LW + w) * nt + t] = c + lineopac[g];
        double wl = A.wave[w0 + w] + A.wfirst;
        double C1 = PlkC1 / wl, C2 = exp(50.7649141 - 5.0 * log(wl));
        S[w * nt + t] = C2 / (exp(C1 / A.xi[XI_T * nt + t]) - 1.0);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nk * nw * nmu; e += blockDim.x) {
        int kw = e / nmu, im = e - kw * nmu;
        int kind = kw / nw, w = kw % nw;
        double Y = delo_ray(R, im, X + (kind * RT_LW + w) * nt, S + w * nt);
        I[(kind * RT_LW + w) * nmu + im] = Y;
        double *out = (kind == 0) ? spc : spl;
        if (out) out[(size_t)(w0 + w) * nmu + im] = Y;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nk * nw; e += blockDim.x) {
        int kind = e / nw, w = e % nw;
        double a = 0.0;
        for (int im = 0; im < nmu; im++) a = a + I[(kind * RT_LW + w) * nmu + im] * wmu[im];
        double *out = (kind == 0) ? sfc : sfl;
        if (out) out[w0 + w] = a;
    }
}

int fsg_launch_radtran_sph(cudaStream_t s, const AtmView &A, const double *lineopac, const RayView &R,
                           const double *wmu, double *spl, double *spc, double *sfl, double *sfc) {
    size_t sm = sizeof(double) * ((size_t)3 * RT_LW * A.ntau + 2 * RT_LW * R.nmu);
    int nb = (A.nwl + RT_LW - 1) / RT_LW;
    k_radtran_sph<<<nb, 128, sm, s>>>(A, lineopac, R, wmu, spl, spc, sfl, sfc);
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}

// ================================================================================================
// Elemental HVoigt / FVoigt over arrays (kernel-level entry points)
// ================================================================================================
__global__ void k_hvoigt(int64_t n, const double *a, const double *v, double *h, const float *vtab,
                         const double *anode, const double *aida) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) h[i] = hvoigt64(vtab, anode, aida, a[i], v[i]);
}

__global__ void k_fvoigt(int64_t n, const double *a, const double *v, double *h, double *l,
                         const float2 *fvtab, const double *anode, const double *aida) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // FVoigt (voigt.f90:256-299): same a-state rule as HVoigt
    double A = a[i], V = v[i], av = fabs(V), vg, fv;
    if (A < 8.0 && av < 8.0) {
        VLine64 L;
        L.A = A;
        if (A < anode[1]) { L.IA = 1; L.UA = A * aida[0]; }
        else { L = vline64(anode, aida, A); }
        fvoigt_line64(fvtab, L, V, &vg, &fv);
    } else { fv_asym64(A, av, &vg, &fv); fv = copysign(fabs(fv), V); }
    h[i] = vg; l[i] = fv;
}

void fsg_launch_hvoigt(cudaStream_t s, int64_t n, const double *a, const double *v, double *h,
                       const VoigtTables &T) {
    if (n > 0) k_hvoigt<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, a, v, h, T.vtab, T.anode, T.aida);
}
void fsg_launch_fvoigt(cudaStream_t s, int64_t n, const double *a, const double *v, double *h, double *l,
                       const VoigtTables &T) {
    if (n > 0) k_fvoigt<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, a, v, h, l, T.fvtab, T.anode, T.aida);
}

// LocPrfPP over independent profiles: one thread per profile (kernel-level entry point)
// LocPrfPP (solver.f90:123-179) of one profile: x = Xki, y = Src over nt depths, d/r/u work arrays
// of nt doubles each; the nmu emergent intensities go to out[0 .. nmu-1]
__device__ void locprf_one(int nmu, const double *xmu, int nt, const double *x, const double *y,
                           const double *rhox, double *d, double *r, double *u, double *out) {
    // TauStep
    {
        double Dx1 = (rhox[1] - rhox[0]) / 1.0, Yp = (x[1] - x[0]) / Dx1;
        d[0] = Dx1 * (x[1] + 2.0 * x[0] + Dx1 / 2.0 * Yp) / 3.0;
        for (int k = 2; k <= nt - 1; k++) {
            double Dx = (rhox[k - 1] - rhox[k - 2]) / 1.0; Dx1 = (rhox[k] - rhox[k - 1]) / 1.0;
            double Der = (x[k - 1] - x[k - 2]) / Dx, Der1 = (x[k] - x[k - 1]) / Dx1;
            if (Der * Der1 > 0.0) {
                double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0;
                Yp = (Der / (Lambda * Der1 + (1.0 - Lambda) * Der)) * Der1;
            } else Yp = 0.0;
            d[k - 1] = Dx1 * (x[k] + 2.0 * x[k - 1] + Dx1 / 2.0 * Yp) / 3.0;
        }
    }
    for (int k = 2; k <= nt - 1; k++) {
        double Dx = d[k - 2], Dx1 = d[k - 1];
        double InvDx = 1.0 / Dx, InvDx1 = 1.0 / Dx1;
        double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0, Lambda1 = 1.0 - Lambda;
        double Der = (y[k - 1] - y[k - 2]) * InvDx, Der1 = (y[k] - y[k - 1]) * InvDx1;
        r[k - 1] = (Der * Der1 > 0.0) ? (Der / (Lambda * Der1 + Lambda1 * Der)) * Der1 : 0.0;
    }
    r[0] = (y[1] - y[0]) / d[0];
    r[nt - 1] = (y[nt - 1] - y[nt - 2]) / d[nt - 2];
    for (int k = 0; k < nt - 1; k++) u[k] = 0.5 * (y[k] + 0.5 * d[k] * r[k] + y[k + 1] - 0.5 * d[k] * r[k + 1]);
    for (int im = 0; im < nmu; im++) {
        double Imu = 1.0 / xmu[im], Y = y[nt - 1];
        for (int k = nt - 2; k >= 0; k--) {
            double Eps, Alpha, Beta, Gamma;
            delo_coef(d[k] * Imu, Eps, Alpha, Beta, Gamma);
            Y = Y * Eps + Alpha * y[k] + Beta * y[k + 1] + Gamma * u[k];
        }
        out[im] = Y;
    }
}

__global__ void k_locprf(int nprof, int nmu, const double *xmu, int nt, const double *xki,
                         const double *src, const double *rhox, double *ploc, double *work) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nprof) return;
    double *d = work + (size_t)p * 3 * nt;
    locprf_one(nmu, xmu, nt, xki + (size_t)p * nt, src + (size_t)p * nt, rhox, d, d + nt, d + 2 * nt,
               ploc + (size_t)p * nmu);
}

// LinStrCalc (synth.f90:1774-1822): central depth of each retained line from the
// continuum and continuum + line intensities at its centre (the centre opacities of the central
// pass: ContOpac at Wlcent, LineOpacity2 at Wlcent), disk-integrated with Wmu when nmu > 1.
// One thread per line of [i0, i0 + nl); work holds 6 nt + 2 nmu doubles per thread.
__global__ void k_linstr(AtmView A, LineView L, const float *__restrict__ vtab, const double *__restrict__ anode,
                         const double *__restrict__ aida, const int32_t *__restrict__ flags, int64_t i0, int64_t nl,
                         int nmu, const double *__restrict__ xmu, const double *__restrict__ wmu,
                         const double *__restrict__ rhox, RayView R, double *work, float *linstr) {
    const double PlkC1 = FSG_HC * FSG_VC * 1e13 / FSG_KBOLT;
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nl) return;
    const int64_t i = i0 + k;
    const int f = flags[i];
    if (f & FSG_F_WEAK) { linstr[i] = 0.0f; return; }
    const int nt = A.ntau;
    double *xc = work + (size_t)k * (6 * nt + 2 * nmu), *xl = xc + nt, *y = xl + nt, *d = y + nt;
    double *ic = d + 3 * nt, *il = ic + nmu;
    double wlc = L.wl[i] - A.wfirst;
    XCoef XC;
    xline_setup(A, L, i, wlc, line_input_flags(L, i, 0), &XC);
    const int ihe = XC.IxHe;
    int iwl = waveidx(A, wlc);
    double dW = (wlc - A.wave[iwl - 1]) / (A.wave[iwl] - A.wave[iwl - 1]);
    const double wl = wlc + A.wfirst;
    const double C1 = PlkC1 / wl, C2 = exp(50.7649141 - 5.0 * log(wl));
    for (int t = 0; t < nt; t++) {
        double cop, vv, av;
        xline_depth(A, t, XC, &cop, &vv, &av);
        double dWl = 0.0;
        if (ihe > 0) dWl = 0.0 - center_shift(A, ihe, t);
        double lo = hvoigt64(vtab, anode, aida, av, dWl * vv) * cop;
        if (A.motype == 1) lo = lo / A.contstd[t];
        double co = cont_center(A, iwl, dW, t);
        xc[t] = co;
        xl[t] = co + lo;
        y[t] = C2 / (exp(C1 / A.xi[XI_T * nt + t]) - 1.0);
    }
    if (R.nmu > 0) {                       // spherical: LocPrfSph (synth.f90:1801-1803)
        for (int m = 0; m < nmu; m++) { ic[m] = delo_ray(R, m, xc, y); il[m] = delo_ray(R, m, xl, y); }
    } else {
        locprf_one(nmu, xmu, nt, xc, y, rhox, d, d + nt, d + 2 * nt, ic);
        locprf_one(nmu, xmu, nt, xl, y, rhox, d, d + nt, d + 2 * nt, il);
    }
    if (nmu == 1) { linstr[i] = (float)(1.0 - il[0] / ic[0]); return; }
    double FlxL = 0.0, FlxC = 0.0;
    for (int m = 0; m < nmu; m++) { FlxL = FlxL + wmu[m] * il[m]; FlxC = FlxC + wmu[m] * ic[m]; }
    linstr[i] = (float)(1.0 - FlxL / FlxC);
}

size_t fsg_linstr_work(int64_t nl, int nt, int nmu) { return sizeof(double) * (size_t)nl * (6 * nt + 2 * nmu); }

void fsg_launch_linstr(cudaStream_t s, const AtmView &A, const LineView &L, const VoigtTables &T,
                       const int32_t *flags, int64_t i0, int64_t nl, int nmu, const double *xmu, const double *wmu,
                       const double *rhox, const RayView &R, double *work, float *linstr) {
    if (nl > 0)
        k_linstr<<<(unsigned)((nl + 127) / 128), 128, 0, s>>>(A, L, T.vtab, T.anode, T.aida, flags, i0, nl, nmu,
                                                              xmu, wmu, rhox, R, work, linstr);
}

void fsg_launch_locprf(cudaStream_t s, int nprof, int nmu, const double *xmu, int nt, const double *xki,
                       const double *src, const double *rhox, double *ploc, double *work) {
    if (nprof > 0) k_locprf<<<(nprof + 127) / 128, 128, 0, s>>>(nprof, nmu, xmu, nt, xki, src, rhox, ploc, work);
}

// ================================================================================================
// MarkWideLines (synth.f90:709-744) over the (packed) line arrays; WlcIdx (synth.f90:677-706)
// ================================================================================================
__device__ __forceinline__ int64_t wlc_idx(const double *wl, double wfirst, int64_t n, double w) {
    if (n == 0 || w < wl[0] - wfirst) return 0;
    int64_t ia = 1, ib = n;
    while (ib - ia > 1) {
        int64_t im = (ia + ib) / 2;
        if (wl[im - 1] - wfirst <= w) ia = im; else ib = im;
    }
    return (wl[ib - 1] - wfirst <= w) ? ib : ia;
}

__global__ void k_mark_wide(AtmView A, int64_t n, const double *wl, int64_t nstep, int32_t *flags,
                            const int32_t *ileft, const int32_t *iright, unsigned long long *nwide) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int f = flags[i];
    if (f & FSG_F_WEAK) return;
    double wr = A.wave[iright[i] - 1], wlft = A.wave[ileft[i] - 1];
    int64_t nrec = wlc_idx(wl, A.wfirst, n, wr) - wlc_idx(wl, A.wfirst, n, wlft) + 1;
    double dv = FSG_VC * (wr - wlft) / ((wl[i] - A.wfirst) + A.wfirst);
    if (nrec > nstep / 2 || dv > 5e3) { flags[i] = f | FSG_F_WIDE; atomicAdd(nwide, 1ull); }
}

void fsg_launch_mark_wide(cudaStream_t s, const AtmView &A, int64_t n, const double *wl, int64_t nstep,
                          int32_t *flags, const int32_t *ileft, const int32_t *iright, unsigned long long *nwide) {
    if (n > 0) k_mark_wide<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(A, n, wl, nstep, flags, ileft, iright, nwide);
}

// ================================================================================================
// Convolution with a short kernel over a spectrum padded with its end values (convol.f90:143-165,
// 206-227, 277-294): out(i) = sum_j in(clamp(i + j - h)) kern(j), h = (n - 1) / 2, in order of j;
// with acc: out(i) = acc(i) + sum * w (the flux sum of the annuli).  One thread per wavelength.
// ================================================================================================
__global__ void k_conv(int nwl, const double *__restrict__ in, int st, const double *__restrict__ kern, int n,
                       double *out, const double *acc, double w) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nwl) return;
    const int h = (int)((n - 1.0) / 2.0);
    double sm = 0.0;
    for (int j = 0; j < n; j++) {
        int m = min(max(i + j - h, 0), nwl - 1);
        sm = sm + in[(size_t)m * st] * kern[j];
    }
    out[i] = acc ? acc[i] + sm * w : sm;
}

void fsg_launch_conv(cudaStream_t s, int nwl, const double *in, int st, const double *kern, int n, double *out,
                     const double *acc, double w) {
    if (nwl > 0) k_conv<<<(nwl + 255) / 256, 256, 0, s>>>(nwl, in, st, kern, n, out, acc, w);
}


// ================================================================================================
// The reference's elemental line-opacity routines on their own, batched (kernel-level entry points):
// XlineSetup / XlineDepth, LineOpacity1 and LineOpacity2 at given points, AnalyticWindow.  The same
// device functions as the drivers, in the reference's operand order.
// ================================================================================================
// XlineSetup of every line with the drivers' input flags (synth.f90:837-845)
__global__ void k_xline_setup(AtmView A, LineView L, XCoef *xc) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n) return;
    XCoef XC;
    xline_setup(A, L, i, L.wl[i] - A.wfirst, line_input_flags(L, i, 0), &XC);
    xc[i] = XC;
}

// XlineDepth of n lines at every depth: out [n][ntau]
__global__ void k_xline_depth(AtmView A, int64_t n, const XCoef *__restrict__ xc, double *cop, double *vv,
                              double *av) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n * A.ntau) return;
    const int64_t i = g / A.ntau;
    const int t = (int)(g - i * A.ntau);
    xline_depth(A, t, xc[i], &cop[g], &vv[g], &av[g]);
}

// LineOpacity1 (opacity.f90:297-346) at npts points, one warp per point, lanes over depths
__global__ void k_lineopacity1_pts(AtmView A, BlockView B, int64_t npts, const double *__restrict__ wl,
                                   const int32_t *__restrict__ l1, const int32_t *__restrict__ l2,
                                   const int32_t *__restrict__ iwl, int64_t loff, const float *__restrict__ vtab,
                                   const double *__restrict__ anode, const double *__restrict__ aida, double *out) {
    const int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (k >= npts) return;
    const int nt = A.ntau;
    for (int t = lane; t < nt; t += 32) {
        double acc = 0.0;
        for (int64_t il = l1[k]; il <= l2[k]; il++) {
            const int f = B.flags[il - 1];
            if ((f & FSG_F_WEAK) || (f & FSG_F_WIDE) || iwl[k] < B.ileft[il - 1] || iwl[k] > B.iright[il - 1]) continue;
            const int ihe = (f >> 8) & 255;
            const double dWl0 = wl[k] - B.wlcent[il - 1];
            double dWl = dWl0;
            if (ihe > 0) dWl = dWl0 - A.heshf[(ihe - 1) * nt + t];
            const size_t o = (size_t)(il - loff - 1) * nt + t;
            const double V = dWl * B.vv[o];
            const double Vgt = hvoigt64(vtab, anode, aida, B.av[o], V) * B.cop[o];
            acc = acc + Vgt;
        }
        if (A.motype == 1) acc = acc / A.contstd[t];
        out[(size_t)k * nt + t] = acc;
    }
}

// LineOpacity2 (opacity.f90:350-386): point k is line iline[k] at wl[k], grid index iwl[k], with its
// own parameter rows; one thread per (point, depth)
__global__ void k_lineopacity2_pts(AtmView A, BlockView B, int64_t npts, const double *__restrict__ wl,
                                   const int32_t *__restrict__ iline, const int32_t *__restrict__ iwl,
                                   const double *__restrict__ cop, const double *__restrict__ vv,
                                   const double *__restrict__ av, const float *__restrict__ vtab,
                                   const double *__restrict__ anode, const double *__restrict__ aida, double *out) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int nt = A.ntau;
    if (g >= npts * nt) return;
    const int64_t k = g / nt;
    const int t = (int)(g - k * nt);
    const int64_t il = iline[k] - 1;
    const int f = B.flags[il];
    double v = 0.0;
    if (!(f & FSG_F_WEAK) && iwl[k] >= B.ileft[il] && iwl[k] <= B.iright[il]) {
        const int ihe = (f >> 8) & 255;
        const double dWl0 = wl[k] - B.wlcent[il];
        double dWl = dWl0;
        if (ihe > 0) dWl = dWl0 - A.heshf[(ihe - 1) * nt + t];
        const double V = dWl * vv[g];
        v = hvoigt64(vtab, anode, aida, av[g], V) * cop[g];
    }
    if (A.motype == 1) v = v / A.contstd[t];
    out[g] = v;
}

// AnalyticWindow (opacity.f90:678-710) of n lines, one thread per line
__global__ void k_analytic_window(AtmView A, int64_t n, const int32_t *__restrict__ flags,
                                  const double *__restrict__ cop, const double *__restrict__ vv,
                                  const double *__restrict__ av, const double *__restrict__ co, double *dw) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nt = A.ntau;
    const double iSqrtPi = 0.5641895835477563;
    const int ihe = (flags[i] >> 8) & 255;
    double dWwin = 0.0;
    for (int t = 0; t < nt; t++) {
        const size_t o = (size_t)i * nt + t;
        double r = cop[o] / (A.epsopac * co[o]);
        if (A.motype == 1) r = r / A.contstd[t];
        if (r <= 1.0) continue;
        double w = sqrt(log(r) + fmax(0.0, av[o] * (r * iSqrtPi - av[o]))) / vv[o];
        if (ihe > 0) w = w + fabs(A.heshf[(ihe - 1) * nt + t]);
        dWwin = fmax(dWwin, w);
    }
    dw[i] = dWwin;
}

void fsg_launch_xline_setup(cudaStream_t s, const AtmView &A, const LineView &L, XCoef *xc) {
    if (L.n > 0) k_xline_setup<<<(unsigned)((L.n + 127) / 128), 128, 0, s>>>(A, L, xc);
}
void fsg_launch_xline_depth(cudaStream_t s, const AtmView &A, int64_t n, const XCoef *xc, double *cop, double *vv,
                            double *av) {
    const int64_t m = n * A.ntau;
    if (m > 0) k_xline_depth<<<(unsigned)((m + 127) / 128), 128, 0, s>>>(A, n, xc, cop, vv, av);
}
void fsg_launch_lineopacity1_pts(cudaStream_t s, const AtmView &A, const BlockView &B, int64_t npts, const double *wl,
                                 const int32_t *l1, const int32_t *l2, const int32_t *iwl, int64_t loff,
                                 const VoigtTables &T, double *out) {
    if (npts > 0)
        k_lineopacity1_pts<<<(unsigned)((npts + 7) / 8), 256, 0, s>>>(A, B, npts, wl, l1, l2, iwl, loff, T.vtab,
                                                                      T.anode, T.aida, out);
}
void fsg_launch_lineopacity2_pts(cudaStream_t s, const AtmView &A, const BlockView &B, int64_t npts, const double *wl,
                                 const int32_t *iline, const int32_t *iwl, const double *cop, const double *vv,
                                 const double *av, const VoigtTables &T, double *out) {
    const int64_t m = npts * A.ntau;
    if (m > 0)
        k_lineopacity2_pts<<<(unsigned)((m + 127) / 128), 128, 0, s>>>(A, B, npts, wl, iline, iwl, cop, vv, av,
                                                                       T.vtab, T.anode, T.aida, out);
}
void fsg_launch_analytic_window(cudaStream_t s, const AtmView &A, int64_t n, const int32_t *flags, const double *cop,
                                const double *vv, const double *av, const double *co, double *dw) {
    if (n > 0) k_analytic_window<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(A, n, flags, cop, vv, av, co, dw);
}
