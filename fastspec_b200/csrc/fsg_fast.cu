// fsg_fast.cu -- mixed-precision line-opacity accumulation (FP32 Voigt, compensated sums).
//
// The work of LineopCalc's accumulation (LineOpacity1, opacity.f90:297-346) is
//   LineOpac(t, p) = sum over retained lines l with Ileft(l) <= p <= Iright(l) of
//                    HVoigt(a(l,t), (lambda_p - lambda_l) / dlD(l,t)) * LinCop(l,t).
// Here a CTA owns a tile of TW = 32 P wavelengths x all depths.  Warp w owns depths
// [w*D, w*D + D); lane l owns the wavelengths tile0 + l + 32k (k < P).  Each thread keeps its
// P x D sums in registers with Kahan compensation: no shared-memory or global atomics, one
// read-modify-write of the FP64 LineOpac per tile and launch, deterministic order.
//
// Lines are binned by window width (class c holds windows of up to 256 * 2^c wavelengths) and
// processed class by class, so the candidate line range of a tile [lo, hi] -- the lines of the
// class whose windows touch it -- stays within a small factor of the lines that do.  Narrow
// classes use narrow tiles (P = 1 for class 0, 2 for class 1, 4 above) so fewer lanes idle at
// the window edges.
//
// The profile is evaluated in FP32 from the per-(line, depth) FP32 records that k_params_fast
// derives from the FP64 XlineDepth values: for s = v^2 + a^2 >= 196 (almost every wing point)
// the reference's rational form (voigt.f90:100-101) as c1 (x + c2) / (x^2 + d1 x + d0), x = v^2;
// below that the table lerp (|v| < 8, a < 8) or the two-term continued fraction (voigt.f90:103-107),
// exactly as HVoigt branches.
#include "fsg_internal.cuh"

#define CLASS_W0 128      // class c: windows of at most CLASS_W0 * 2^(c+1) wavelengths

__constant__ float c_anode[FSG_NA1];
__constant__ float c_aida[FSG_NA1];

int fsg_fast_set_constants(const double *anode_h, const double *aida_h) {
    float a[FSG_NA1], b[FSG_NA1];
    for (int i = 0; i < FSG_NA1; i++) { a[i] = (float)anode_h[i]; b[i] = (float)aida_h[i]; }
    if (cudaMemcpyToSymbol(c_anode, a, sizeof a) != cudaSuccess) return FSG_E_CUDA;
    if (cudaMemcpyToSymbol(c_aida, b, sizeof b) != cudaSuccess) return FSG_E_CUDA;
    return FSG_OK;
}

// HVoigt * LinCop in FP32 for the table / continued-fraction region (voigt.f90:81-108)
__device__ __noinline__ float hv_core32(const float *__restrict__ vtab, float v, float a, float cop) {
    float av = fabsf(v);
    if (a < 8.0f && av < 8.0f) {
        float fv = av * 125.0f;
        int iv = min((int)fv, FSG_NVV - 1);
        float tv = fv - (float)iv, ua;
        int ia;
        if (a < c_anode[1]) { ia = 1; ua = a * c_aida[0]; }
        else {
            ia = (int)(sqrtf(a) * 141.42135623730951f) + 1;
            ia = min(ia, FSG_NVA);
            ua = (a - c_anode[ia - 1]) * c_aida[ia - 1];
        }
        const float *p0 = vtab + (ia - 1) * FSG_NV1 + iv, *p1 = p0 + FSG_NV1;
        float t00 = __ldg(p0), t01 = __ldg(p0 + 1), t10 = __ldg(p1), t11 = __ldg(p1 + 1);
        float c0 = t00 + tv * (t01 - t00), c1 = t10 + tv * (t11 - t10);
        return (c0 + ua * (c1 - c0)) * cop;
    }
    float a2 = a * a, v2 = av * av;
    float p = v2 - a2 - 1.5f, q = 2.0f * av * a;
    float dr = av * p - a * q, di = av * q + a * p;
    return 0.56418958354775628f * ((p + 0.5f) * di - q * dr) / (dr * dr + di * di) * cop;
}

// Kahan-compensated accumulation of one value
#define KAHAN(S, CC, V) do { float _y = (V) - (CC); float _t = (S) + _y; (CC) = (_t - (S)) - _y; (S) = _t; } while (0)

template <int D, int P>
__global__ void __launch_bounds__(32 * 18)
k_accum_fast(int ntau, int nwl, const double *__restrict__ wave, const LineHdr *__restrict__ hdr,
             const WingRec *__restrict__ wing, const CoreRec *__restrict__ core,
             const int *__restrict__ tile_lo, const int *__restrict__ tile_hi,
             const float *__restrict__ vtab, double *__restrict__ lineopac) {
    constexpr int TW = 32 * P;
    const int tile = blockIdx.x;
    const int lo = tile_lo[tile], hi = tile_hi[tile];
    if (lo > hi) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t0 = warp * D;
    if (t0 >= ntau) return;
    const int nd = min(D, ntau - t0);
    const int p0 = tile * TW;                 // 0-based wavelength index of the tile start
    double wv[P];
    int pix[P];
#pragma unroll
    for (int k = 0; k < P; k++) {
        pix[k] = p0 + lane + 32 * k;          // 0-based
        wv[k] = wave[min(pix[k], nwl - 1)];
    }
    float s[D][P], c[D][P];
#pragma unroll
    for (int d = 0; d < D; d++)
#pragma unroll
        for (int k = 0; k < P; k++) { s[d][k] = 0.0f; c[d][k] = 0.0f; }

    const int tile_first = p0 + 1, tile_last = min(p0 + TW, nwl);   // 1-based bounds
    for (int j = lo; j <= hi; j++) {
        const LineHdr h = hdr[j];
        if (h.iright < tile_first || h.ileft > tile_last) continue;  // window misses the tile
        float dl2[P];
        bool in[P];
#pragma unroll
        for (int k = 0; k < P; k++) {
            int p1 = pix[k] + 1;
            in[k] = (p1 >= h.ileft) && (p1 <= h.iright);
            float dl = (float)(wv[k] - h.wlc);
            dl2[k] = dl * dl;
        }
        const WingRec *wr = wing + (size_t)j * ntau + t0;
        WingRec w[D];
#pragma unroll
        for (int d = 0; d < D; d++) w[d] = wr[min(d, nd - 1)];
        // wing form for every point, branch-free: one basic block, P x D independent chains
        float val[D][P];
        bool core_any = false;
#pragma unroll
        for (int d = 0; d < D; d++)
#pragma unroll
            for (int k = 0; k < P; k++) {
                float y = fmaf(dl2[k], w[d].vv2, w[d].c2);
                float t = y - 1.0f;
                float den = fmaf(t, t, w[d].twoA);
                val[d][k] = __fdividef(w[d].c1 * y, den);
                core_any |= (y < 196.5f);
            }
        // rare: points with s < 196 take the reference's table / continued fraction
        if (core_any) {
            const CoreRec *cr = core + (size_t)j * ntau + t0;
#pragma unroll
            for (int d = 0; d < D; d++)
#pragma unroll
                for (int k = 0; k < P; k++) {
                    float y = fmaf(dl2[k], w[d].vv2, w[d].c2);
                    if (d < nd && y < 196.5f) {
                        const CoreRec cc = cr[d];
                        val[d][k] = hv_core32(vtab, sqrtf(dl2[k]) * cc.vv, cc.a, cc.cop);
                    }
                }
        }
#pragma unroll
        for (int d = 0; d < D; d++)
#pragma unroll
            for (int k = 0; k < P; k++) {
                float v = in[k] ? val[d][k] : 0.0f;
                KAHAN(s[d][k], c[d][k], v);
            }
    }
#pragma unroll
    for (int k = 0; k < P; k++) {
        if (pix[k] >= nwl) continue;
        double *dst = lineopac + (size_t)pix[k] * ntau + t0;
#pragma unroll
        for (int d = 0; d < D; d++)
            if (d < nd) dst[d] = dst[d] + ((double)s[d][k] - (double)c[d][k]);
    }
}

// Tile width per window-width class: narrow windows get narrower tiles so fewer lanes idle.
int fsg_class_pix(int cls) { return cls <= 1 ? 2 : 4; }

int fsg_launch_accum_fast(cudaStream_t st, int cls, int ntau, int nwl, const double *wave, const LineHdr *hdr,
                          const WingRec *wing, const CoreRec *core, const int *tile_lo, const int *tile_hi,
                          const float *vtab, double *lineopac) {
    const int P = fsg_class_pix(cls);
    const int TW = 32 * P;
    const int ntiles = (nwl + TW - 1) / TW;
    // depths per warp: P x D = 16 evaluations per thread and line, at most 18 warps per CTA
    int D = 16 / P;
    if ((ntau + D - 1) / D > 18) D = (ntau + 17) / 18;
    int nwarps = (ntau + D - 1) / D;
#define LAUNCH(DD, PP) k_accum_fast<DD, PP><<<ntiles, 32 * nwarps, 0, st>>>(ntau, nwl, wave, hdr, wing, core, \
                                                                             tile_lo, tile_hi, vtab, lineopac)
    if (P == 1) {
        if (D == 16) LAUNCH(16, 1); else return FSG_E_ARG;
    } else if (P == 2) {
        if (D == 8) LAUNCH(8, 2); else return FSG_E_ARG;
    } else {
        switch (D) {
            case 4: LAUNCH(4, 4); break;
            case 5: LAUNCH(5, 4); break;
            case 6: LAUNCH(6, 4); break;
            case 7: LAUNCH(7, 4); break;
            case 8: LAUNCH(8, 4); break;
            default: return FSG_E_ARG;
        }
    }
#undef LAUNCH
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}

// ---- tile candidate ranges of one block: lo/hi of the block-local line index -------------------
__global__ void k_tile_reset(int ntiles, int *lo, int *hi) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ntiles) { lo[i] = 0x7fffffff; hi[i] = -1; }
}

__global__ void k_tile_span(int64_t nb, int tw, const LineHdr *hdr, int *lo, int *hi) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nb) return;
    LineHdr h = hdr[j];
    int a = (h.ileft - 1) / tw, b = (h.iright - 1) / tw;
    for (int t = a; t <= b; t++) { atomicMin(&lo[t], (int)j); atomicMax(&hi[t], (int)j); }
}

// tile count of the narrowest tiles (sizes the lo/hi arrays)
int fsg_fast_tiles(int nwl) { return (nwl + 31) / 32; }

void fsg_launch_tile_span(cudaStream_t s, int cls, int nwl, int64_t nb, const LineHdr *hdr, int *lo, int *hi) {
    int tw = 32 * fsg_class_pix(cls);
    int ntiles = (nwl + tw - 1) / tw;
    k_tile_reset<<<(ntiles + 255) / 256, 256, 0, s>>>(ntiles, lo, hi);
    if (nb > 0) k_tile_span<<<(unsigned)((nb + 127) / 128), 128, 0, s>>>(nb, tw, hdr, lo, hi);
}

// ---- window-width classes and order-preserving compaction -----------------------------------
// class 0: windows up to 256 wavelengths; class c: up to 256 * 2^c.
__device__ __forceinline__ int width_class(int il, int ir) {
    int w = ir - il + 1;
    int c = 0;
    while ((CLASS_W0 << (c + 1)) < w && c < 30) c++;
    return c;
}

#define SCAN_BS 1024
// selection predicate: cls >= 0 retained lines of that width class, -1 every retained line,
// -2 retained wide lines (flag bit 3)
__device__ __forceinline__ int sel_pred(int f, int il, int ir, int cls) {
    if (f & FSG_F_WEAK) return 0;
    if (cls == -1) return 1;
    if (cls == -2) return (f & FSG_F_WIDE) != 0;
    return width_class(il, ir) == cls;
}
// Count retained lines of class `cls` (cls < 0: every retained line) per CTA of SCAN_BS lines.
__global__ void k_sel_count(int64_t n, const int32_t *flags, const int32_t *il, const int32_t *ir, int cls,
                            int *counts) {
    __shared__ int warp_sums[SCAN_BS / 32];
    int64_t i = (int64_t)blockIdx.x * SCAN_BS + threadIdx.x;
    int pred = 0;
    if (i < n) pred = sel_pred(flags[i], il[i], ir[i], cls);
    unsigned m = __ballot_sync(0xffffffffu, pred);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < SCAN_BS / 32; w++) s += warp_sums[w];
        counts[blockIdx.x] = s;
    }
}

// Exclusive scan of the per-CTA counts (single CTA, serial over chunks of 1024).
__global__ void k_scan_counts(int nblk, const int *counts, int64_t *offs, int64_t *total) {
    __shared__ int64_t buf[1024];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nblk; base += 1024) {
        int i = base + threadIdx.x;
        int64_t v = (i < nblk) ? counts[i] : 0;
        buf[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            int64_t t = (threadIdx.x >= off) ? buf[threadIdx.x - off] : 0;
            __syncthreads();
            buf[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < nblk) offs[i] = carry + buf[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += buf[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_sel_scatter(int64_t n, const int32_t *flags, const int32_t *il, const int32_t *ir, int cls,
                              const int64_t *offs, int64_t *out) {
    __shared__ int warp_offs[SCAN_BS / 32];
    int64_t i = (int64_t)blockIdx.x * SCAN_BS + threadIdx.x;
    int pred = 0;
    if (i < n) pred = sel_pred(flags[i], il[i], ir[i], cls);
    unsigned m = __ballot_sync(0xffffffffu, pred);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_offs[w] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int q = 0; q < SCAN_BS / 32; q++) { int t = warp_offs[q]; warp_offs[q] = s; s += t; }
    }
    __syncthreads();
    if (pred) {
        int r = warp_offs[w] + __popc(m & ((1u << lane) - 1u));
        out[offs[blockIdx.x] + r] = i;
    }
}

// Select (in order) the retained lines of class cls into out[]; *count receives the number (device).
int fsg_select(cudaStream_t s, int64_t n, const int32_t *flags, const int32_t *il, const int32_t *ir, int cls,
               int *counts, int64_t *offs, int64_t *out, int64_t *d_total) {
    if (n <= 0) { cudaMemsetAsync(d_total, 0, sizeof(int64_t), s); return FSG_OK; }
    int nblk = (int)((n + SCAN_BS - 1) / SCAN_BS);
    k_sel_count<<<nblk, SCAN_BS, 0, s>>>(n, flags, il, ir, cls, counts);
    k_scan_counts<<<1, 1024, 0, s>>>(nblk, counts, offs, d_total);
    k_sel_scatter<<<nblk, SCAN_BS, 0, s>>>(n, flags, il, ir, cls, offs, out);
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}

// Histogram of window classes of the retained lines (for the host loop over classes).
__global__ void k_class_hist(int64_t n, const int32_t *flags, const int32_t *il, const int32_t *ir,
                             unsigned long long *hist) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (flags[i] & FSG_F_WEAK)) return;
    atomicAdd(&hist[width_class(il[i], ir[i])], 1ull);
}

void fsg_launch_class_hist(cudaStream_t s, int64_t n, const int32_t *flags, const int32_t *il,
                           const int32_t *ir, unsigned long long *hist) {
    if (n > 0) k_class_hist<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, flags, il, ir, hist);
}

// Motype 1 is folded into the records; nothing else to finish.

int fsg_select_wide(cudaStream_t s, int64_t n, const int32_t *flags, int *counts, int64_t *offs, int64_t *out,
                    int64_t *d_total) {
    return fsg_select(s, n, flags, flags, flags, -2, counts, offs, out, d_total);
}

// Gather the retained lines' SoA fields and per-line outputs into packed arrays (PACK,
// synth.f90:915-933).  buf must hold 64 bytes per packed line.
__global__ void k_gather_lines(LineView L, const int64_t *idx, int64_t nw, double *wl, float *elo, float *gf,
                               float *grad, float *gqst, float *gvdw, int32_t *spc, int32_t *ismol, int32_t *ihe,
                               const int32_t *f0, const int32_t *l0, const int32_t *r0, int32_t *f1, int32_t *l1,
                               int32_t *r1) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nw) return;
    int64_t i = idx[j];
    wl[j] = L.wl[i]; elo[j] = L.elo[i]; gf[j] = L.gf[i]; grad[j] = L.grad[i]; gqst[j] = L.gqst[i];
    gvdw[j] = L.gvdw[i]; spc[j] = L.spc[i];
    if (L.ismol) ismol[j] = L.ismol[i];
    if (L.ihe) ihe[j] = L.ihe[i];
    f1[j] = f0[i]; l1[j] = l0[i]; r1[j] = r0[i];
}

void fsg_launch_gather_lines(cudaStream_t s, const LineView &L, const int64_t *idx, int64_t nw, char *buf,
                             const int32_t *f0, const int32_t *l0, const int32_t *r0, LineView *W, int32_t **f1,
                             int32_t **l1, int32_t **r1) {
    size_t n = (size_t)(nw > 0 ? nw : 1);
    double *wl = (double *)buf;
    float *elo = (float *)(wl + n), *gf = elo + n, *grad = gf + n, *gqst = grad + n, *gvdw = gqst + n;
    int32_t *spc = (int32_t *)(gvdw + n), *ismol = spc + n, *ihe = ismol + n, *ff = ihe + n, *ll = ff + n, *rr = ll + n;
    if (nw > 0)
        k_gather_lines<<<(unsigned)((nw + 255) / 256), 256, 0, s>>>(L, idx, nw, wl, elo, gf, grad, gqst, gvdw, spc,
                                                                    ismol, ihe, f0, l0, r0, ff, ll, rr);
    *W = L;
    W->n = nw; W->wl = wl; W->elo = elo; W->gf = gf; W->grad = grad; W->gqst = gqst; W->gvdw = gvdw; W->spc = spc;
    W->ismol = L.ismol ? ismol : nullptr; W->ihe = L.ihe ? ihe : nullptr;
    *f1 = ff; *l1 = ll; *r1 = rr;
}

__global__ void k_scatter_flags(int64_t nw, const int64_t *idx, const int32_t *pf, int32_t *flags) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < nw) flags[idx[j]] = pf[j];
}

void fsg_launch_scatter_flags(cudaStream_t s, int64_t nw, const int64_t *idx, const int32_t *pf, int32_t *flags) {
    if (nw > 0) k_scatter_flags<<<(unsigned)((nw + 255) / 256), 256, 0, s>>>(nw, idx, pf, flags);
}
