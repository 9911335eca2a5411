// fsg_fast.cu -- mixed-precision line-opacity accumulation (FP32 Voigt, compensated sums).
//
// The work of LineopCalc's accumulation (LineOpacity1, opacity.f90:297-346) is
//   LineOpac(t, p) = sum over retained lines l with Ileft(l) <= p <= Iright(l) of
//                    HVoigt(a(l,t), (lambda_p - lambda_l) / dlD(l,t)) * LinCop(l,t).
// It is split by the branch HVoigt takes.  Each line has a core range (every wavelength of its
// window where some depth may have s = v^2 + a^2 < 196); outside it every depth takes the
// reference's rational wing form (voigt.f90:100-101).
//
// Wing pass (k_accum_fast): a CTA owns a tile of TW = 32 P wavelengths x all depths; warp w owns
// depths [w*D, w*D + D), lane l the wavelengths tile0 + l + 32k (k < P).  Line headers and wing
// records arrive in shared memory by bulk copies; each thread keeps P x D FP32 partials over FOLD
// lines, folded into Kahan (sum, compensation) pairs in shared memory.  Lines are binned by window
// width (class c holds windows of up to 256 * 2^c wavelengths) and processed class by class, so a
// tile's candidate range stays close to the lines that touch it; narrow classes use 64-wavelength
// tiles, wide ones 128.
//
// Core pass (k_core_fast): over the core ranges, 32-wavelength tiles, the points where s < 196: the
// table lerp (|v| < 8, a < 8) or the two-term continued fraction (voigt.f90:103-107), exactly as
// HVoigt branches.  No atomics; one read-modify-write of the FP64 LineOpac per tile and launch;
// deterministic order.
#include "fsg_internal.cuh"
#include "fsg_mbar.cuh"

#include <cub/device/device_scan.cuh>
#include <cuda/functional>
#include <algorithm>

#define CLASS_W0 128      // class c: windows of at most CLASS_W0 * 2^(c+1) wavelengths

// HVoigt * LinCop in FP32 outside the table (a >= 8 or |v| >= 8, s < 196): the two-term continued
// fraction of voigt.f90:103-107 at |v| = av
__device__ __forceinline__ float hv_cf32(float av, float a, float cop) {
    float a2 = a * a, v2 = av * av;
    float p = v2 - a2 - 1.5f, q = 2.0f * av * a;
    float dr = av * p - a * q, di = av * q + a * p;
    return 0.56418958354775628f * __fdividef((p + 0.5f) * di - q * dr, dr * dr + di * di) * cop;
}

// Kahan-compensated accumulation of one value
#define KAHAN(S, CC, V) do { float _y = (V) - (CC); float _t = (S) + _y; (CC) = (_t - (S)) - _y; (S) = _t; } while (0)

// Lines folded into the compensated sums at a time: each thread adds up to FOLD lines into FP32
// register partials, then Kahan-adds every partial into its (sum, compensation) pair in shared
// memory.  The partials carry at most FOLD terms, so their rounding stays at the FP32 unit
// roundoff of a few terms; the Kahan pairs carry the long sums.
#define FOLD 32
// Candidate lines staged per TMA bulk copy, and the wing pass's staging buffers (copies in flight)
#define CH 32
#define WNB 2
// cp.async.bulk moves multiples of 16 bytes between 16-byte aligned addresses
static_assert(sizeof(WingRec) % 16 == 0 && sizeof(LineHdr) % 16 == 0 && sizeof(CoreRec) % 16 == 0, "bulk-copied records: multiples of 16 bytes");

// Issue the bulk copies of chunk c (lines lo + c*CH ...) into buffer b; one thread calls this.
__device__ __forceinline__ void stage_chunk(int c, int lo, int hi, int ntau, const LineHdr *hdr, const WingRec *wing,
                                            LineHdr *shdr, WingRec *swing, uint64_t *bar, unsigned extra_tx) {
    int j0 = lo + c * CH;
    int n = min(CH, hi - j0 + 1);
    unsigned brec = (unsigned)(n * ntau * (int)sizeof(WingRec)), bhdr = (unsigned)(n * (int)sizeof(LineHdr));
    mbar_expect_tx(bar, brec + bhdr + extra_tx);
    tma_bulk_g2s(swing, wing + (size_t)j0 * ntau, brec, bar);
    tma_bulk_g2s(shdr, hdr + j0, bhdr, bar);
}

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Wing pass.  Every window point where fl32(t) >= 195.5 (s >= 196) takes HVoigt's rational wing
// form:
//   val = c1 (t + 1) / (t^2 + twoA),  t = dl^2 vv2 + c2m1
// (three FMAs, one reciprocal, one FMA into the partial sum).  Outside the line's core range [cl, cr]
// that is every depth.  Lines whose window covers the whole tile outside their core range (the common
// case for wide windows) skip the mask; for the others the points outside the window get an x for
// which the term is exactly 0.  On tiles that meet the core range, each point whose t is below 195.5
// (table or continued fraction, the core pass's share) has its t replaced by 1e19, whose term is
// exactly 0 too: the two passes split the points by the same FP32 test, so each point is evaluated
// once.

// shared memory of the wing pass for at most ntau_max depths:
// wing records [WNB][CH][ntau_max] | headers [WNB][CH] | mbarriers [WNB] | Kahan pairs [D * P][blockDim.x]
// (a warp reads up to D - 1 <= 7 records past its line's last depth: at most 112 bytes past the
// last record buffer, inside the headers that follow it)
__host__ __device__ inline size_t wing_smem_recs(int ntau_max) {
    return sizeof(WingRec) * WNB * CH * (size_t)ntau_max + sizeof(LineHdr) * WNB * CH;
}

// One tile of one job.  Called by every thread of the CTA with the mbarriers initialised; kk counts
// the chunks the CTA has consumed so far (their buffer and phase parity), across tiles.  Returns
// false after a copy did not complete within its bound (error reported in *err).
template <int D, int P>
__device__ __forceinline__ bool wing_tile(const WingJob &J, int tile, unsigned char *smem_raw, int ntau_max,
                                          unsigned &kk, int *err) {
    const int ntau = J.ntau, nwl = J.nwl;
    const double *__restrict__ wave = J.wave;
    const LineHdr *__restrict__ hdr = J.hdr;
    const WingRec *__restrict__ wing = J.wing;
    WingRec *swing = (WingRec *)smem_raw;
    LineHdr *shdr = (LineHdr *)(swing + WNB * CH * ntau_max);
    uint64_t *bars = (uint64_t *)(shdr + WNB * CH);
    float2 *ksum = (float2 *)(bars + WNB);               // [D * P][blockDim.x]
    constexpr int TW = 32 * P;
    bool any = false;                                   // some segment has lines touching the tile
    for (int sg = 0; sg < J.nseg; sg++)
        any = any || J.tile_lo[sg * J.seg_stride + tile] <= J.tile_hi[sg * J.seg_stride + tile];
    if (!any) return true;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t0 = warp * D;
    const int nd = max(0, min(D, ntau - t0));            // warps past the last depth only help staging
    const int p0 = tile * TW;
    const int nth = blockDim.x;
    // wavelength offsets as FP32 hi + lo: dl = (wvh - wlh) + (wvl - wll) keeps dl to FP32 relative
    // accuracy next to the line centre
    float wvh[P], wvl[P];
    int pix[P];
#pragma unroll
    for (int k = 0; k < P; k++) {
        pix[k] = p0 + lane + 32 * k;
        double w = wave[min(pix[k], nwl - 1)];
        wvh[k] = (float)w;
        wvl[k] = (float)(w - (double)wvh[k]);
    }
    float part[D][P];
#pragma unroll
    for (int d = 0; d < D; d++)
#pragma unroll
        for (int k = 0; k < P; k++) {
            part[d][k] = 0.0f;
            ksum[(d * P + k) * nth + threadIdx.x] = make_float2(0.0f, 0.0f);
        }
    int nfold = 0;
    const int tile_first = p0 + 1, tile_last = min(p0 + TW, nwl);
    for (int sg = 0; sg < J.nseg; sg++) {               // the job's segments of lines, in turn
        const int lo = J.tile_lo[sg * J.seg_stride + tile], hi = J.tile_hi[sg * J.seg_stride + tile];
        if (lo > hi) continue;
        const int nchunks = (hi - lo + CH) / CH;
        // chunk c of this tile is the CTA's chunk g = kk + c: buffer g % WNB, phase parity (g / WNB) & 1
        if (threadIdx.x == 0) {
            for (int c = 0; c < WNB && c < nchunks; c++) {
                const int b = (kk + c) % WNB;
                stage_chunk(c, lo, hi, ntau, hdr, wing, shdr + b * CH, swing + b * CH * ntau_max, &bars[b],
                            J.extra_tx);
            }
        }
        int failed = -1;                                     // chunk whose copy did not complete
        for (int c = 0; c < nchunks; c++) {
            const unsigned g = kk + c;
            const int b = g % WNB;
            const bool ok = mbar_wait(&bars[b], (g / WNB) & 1, J.wait_ns);
            if (__syncthreads_or(!ok)) { failed = c; break; }
            const LineHdr *ch = shdr + b * CH;
            const WingRec *cw = swing + b * CH * ntau_max;
            const int n = min(CH, hi - (lo + c * CH) + 1);
            if (nd > 0) {
                for (int q = 0; q < n; q++) {
                    const LineHdr h = ch[q];
                    if (h.iright < tile_first || h.ileft > tile_last) continue;   // window misses the tile
                    float x[P];
#pragma unroll
                    for (int k = 0; k < P; k++) {
                        float dl = (wvh[k] - h.wlh) + (wvl[k] - h.wll);
                        x[k] = dl * dl;
                    }
                    // depths past the job's last (last warp only) read the next records of the buffer, or
                    // the headers after it: their partials are never stored
                    const WingRec *wq = cw + q * ntau + t0;
                    WingRec w[D];
#pragma unroll
                    for (int d = 0; d < D; d++) w[d] = wq[d];
                    const bool core_hit = h.cl <= h.cr && h.cr >= tile_first && h.cl <= tile_last;
                    const bool full = h.ileft <= tile_first && h.iright >= tile_last && !core_hit;
                    if (!full) {
                        // points outside the window take the header's offset x, for which the wing term is
                        // exactly 0
                        const float xm = __int_as_float(h.pad0);
#pragma unroll
                        for (int k = 0; k < P; k++) {
                            const int p1 = pix[k] + 1;
                            const bool in = p1 >= h.ileft && p1 <= h.iright;
                            x[k] = in ? x[k] : xm;
                        }
                    }
                    if (!core_hit) {
#pragma unroll
                        for (int d = 0; d < D; d++)
#pragma unroll
                            for (int k = 0; k < P; k++) {
                                float t = fmaf(x[k], w[d].vv2, w[d].c2m1);
                                float den = fmaf(t, t, w[d].twoA);
                                float num = fmaf(w[d].c1, t, w[d].c1);
                                part[d][k] = fmaf(num, rcp_approx(den), part[d][k]);
                            }
                    } else {
#pragma unroll
                        for (int d = 0; d < D; d++)
#pragma unroll
                            for (int k = 0; k < P; k++) {
                                float t = fmaf(x[k], w[d].vv2, w[d].c2m1);
                                t = t < 195.5f ? 1.0e19f : t;        // the core pass's point
                                float den = fmaf(t, t, w[d].twoA);
                                float num = fmaf(w[d].c1, t, w[d].c1);
                                part[d][k] = fmaf(num, rcp_approx(den), part[d][k]);
                            }
                    }
                    if (++nfold == FOLD) {
                        nfold = 0;
#pragma unroll
                        for (int d = 0; d < D; d++)
#pragma unroll
                            for (int k = 0; k < P; k++) {
                                float2 &qq = ksum[(d * P + k) * nth + threadIdx.x];
                                float2 sc = qq;
                                KAHAN(sc.x, sc.y, part[d][k]);
                                qq = sc;
                                part[d][k] = 0.0f;
                            }
                    }
                }
            }
            __syncthreads();                                   // every warp is done with buffer b
            if (threadIdx.x == 0 && c + WNB < nchunks)
                stage_chunk(c + WNB, lo, hi, ntau, hdr, wing, shdr + b * CH, swing + b * CH * ntau_max, &bars[b],
                            J.extra_tx);
        }
        if (failed >= 0) {
            // a copy never completed: report, then wait (bounded) for the copies still in flight,
            // chunks failed .. failed + WNB - 1, before the CTA's shared memory is released
            if (threadIdx.x == 0) {
                atomicExch(err, FSG_E_TIMEOUT);
                for (int c = failed; c < nchunks && c < failed + WNB; c++) {
                    const unsigned g = kk + c;
                    mbar_wait(&bars[g % WNB], (g / WNB) & 1, J.wait_ns);
                }
            }
            __syncthreads();
            return false;
        }
        kk += nchunks;
    }
    if (nd <= 0) return true;
#pragma unroll
    for (int k = 0; k < P; k++) {
        if (pix[k] >= nwl) continue;
        double *dst = J.lineopac + (size_t)pix[k] * ntau + t0;
#pragma unroll
        for (int d = 0; d < D; d++) {
            float2 sc = ksum[(d * P + k) * nth + threadIdx.x];
            KAHAN(sc.x, sc.y, part[d][k]);
            if (d < nd) dst[d] = dst[d] + ((double)sc.x - (double)sc.y);
        }
    }
    return true;
}

__device__ __forceinline__ void wing_bars_init(unsigned char *smem_raw, int ntau_max) {
    uint64_t *bars = (uint64_t *)(smem_raw + wing_smem_recs(ntau_max));
    if (threadIdx.x == 0) {
        for (int b = 0; b < WNB; b++) mbar_init(&bars[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
}

// one tile per CTA (blockIdx.x)
template <int D, int P>
__global__ void __launch_bounds__(32 * 18, 1)
k_accum_fast(WingJob J, int *__restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    if (J.tile_lo[blockIdx.x] > J.tile_hi[blockIdx.x]) return;
    wing_bars_init(smem_raw, J.ntau);
    unsigned kk = 0;
    wing_tile<D, P>(J, blockIdx.x, smem_raw, J.ntau, kk, err);
}

// Persistent form for many jobs (batched atmospheres): CTAs take (job, tile) items from a device
// work queue (*queue, zero at launch) until jobs[njobs - 1] is done; tile0[j] is the first item of
// job j (prefix sums of the jobs' tile counts, tile0[njobs] = total).
template <int D, int P>
__global__ void __launch_bounds__(32 * 18, 1)
k_accum_batch(const WingJob *__restrict__ jobs, const int *__restrict__ tile0, int njobs, int ntau_max,
              unsigned *queue, int *__restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ int s_item;
    wing_bars_init(smem_raw, ntau_max);
    unsigned kk = 0;
    const int total = tile0[njobs];
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= total) break;
        int a = 0, b = njobs - 1;                          // job with tile0[a] <= item < tile0[a + 1]
        while (a < b) { int m = (a + b + 1) >> 1; if (tile0[m] <= item) a = m; else b = m - 1; }
        const WingJob J = jobs[a];
        if (!wing_tile<D, P>(J, item - tile0[a], smem_raw, ntau_max, kk, err)) break;
    }
}

// Tile width per window-width class: narrow windows get narrower tiles so fewer lanes idle.
int fsg_class_pix(int cls) { return cls <= 1 ? 2 : 4; }

// depths per warp for P wavelengths per lane: P x D = 16 evaluations per thread and line, at most
// 18 warps per CTA
static int wing_depths(int P, int ntau) {
    int D = 16 / P;
    if ((ntau + D - 1) / D > 18) D = (ntau + 17) / 18;
    return D;
}

size_t fsg_wing_smem(int P, int ntau_max) {
    const int D = wing_depths(P, ntau_max), nwarps = (ntau_max + D - 1) / D;
    return wing_smem_recs(ntau_max) + WNB * sizeof(uint64_t) + sizeof(float2) * (size_t)D * P * 32 * nwarps;
}

#define WING_DISPATCH(P, D, LAUNCH) do { \
        if (P == 2) { if (D == 8) LAUNCH(8, 2); else return FSG_E_ARG; } \
        else switch (D) { case 4: LAUNCH(4, 4); break; case 5: LAUNCH(5, 4); break; case 6: LAUNCH(6, 4); break; \
                          case 7: LAUNCH(7, 4); break; case 8: LAUNCH(8, 4); break; default: return FSG_E_ARG; } \
    } while (0)

int fsg_launch_accum_fast(cudaStream_t st, int cls, int ntau, int nwl, const double *wave, const LineHdr *hdr,
                          const WingRec *wing, const int *tile_lo, const int *tile_hi, double *lineopac, int *err,
                          unsigned extra_tx, unsigned long long wait_ns) {
    const int P = fsg_class_pix(cls);
    const int TW = 32 * P;
    const int ntiles = (nwl + TW - 1) / TW;
    const int D = wing_depths(P, ntau);
    const int nwarps = (ntau + D - 1) / D;
    const size_t smem = fsg_wing_smem(P, ntau);
    if (smem > 200 * 1024) return FSG_E_ARG;
    WingJob J{ ntau, nwl, wave, hdr, wing, tile_lo, tile_hi, lineopac, extra_tx, wait_ns, 1, 0 };
#define LAUNCH(DD, PP) do { \
        cudaFuncSetAttribute(k_accum_fast<DD, PP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        k_accum_fast<DD, PP><<<ntiles, 32 * nwarps, smem, st>>>(J, err); } while (0)
    WING_DISPATCH(P, D, LAUNCH);
#undef LAUNCH
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}

// the persistent wing pass over njobs jobs (device array), P wavelengths per lane, ctas CTAs
int fsg_launch_accum_batch(cudaStream_t st, int P, int ntau_max, const WingJob *jobs, const int *tile0, int njobs,
                           int ctas, unsigned *queue, int *err) {
    const int D = wing_depths(P, ntau_max);
    const int nwarps = (ntau_max + D - 1) / D;
    const size_t smem = fsg_wing_smem(P, ntau_max);
    if (smem > 200 * 1024) return FSG_E_ARG;
#define LAUNCH(DD, PP) do { \
        cudaFuncSetAttribute(k_accum_batch<DD, PP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        k_accum_batch<DD, PP><<<ctas, 32 * nwarps, smem, st>>>(jobs, tile0, njobs, ntau_max, queue, err); } while (0)
    WING_DISPATCH(P, D, LAUNCH);
#undef LAUNCH
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}

// Core pass.  Over each line's core range [cl, cr], the points where fl32(t) < 195.5 (s < 196): the
// table lerp or the continued fraction, as HVoigt branches (voigt.f90:81-107); the wing pass takes the
// others (the same FP32 test splits the points, so each is evaluated once).  A CTA owns 32 wavelengths
// x all depths: warp w depths [w*D, w*D + D), lane l wavelength tile0 + l, Kahan sums in
// registers.  Headers, wing records and core records of the tile's candidate lines arrive in shared
// memory CHC lines at a time by double-buffered bulk copies completing on mbarriers (waits bounded;
// on expiry the kernel reports FSG_E_TIMEOUT and drains its copies), so the loop over lines reads
// shared memory; per line a thread forms its depths' branch predicates first and issues their table
// gathers (one 16-byte load of the cell-major VgtTab copy each) together.  D = 4 depths per warp up to
// 72 depths, 8 beyond (18 warps at most).


// shared memory of the core pass for at most ntau_max depths and chc lines per chunk:
// wing records [2][chc][ntau_max] | core records [2][chc][ntau_max] | headers [2][chc] | mbarriers [2]
__host__ __device__ inline size_t core_smem(int ntau_max, int chc) {
    return (sizeof(WingRec) + sizeof(CoreRec)) * 2 * (size_t)chc * ntau_max + sizeof(LineHdr) * 2 * (size_t)chc +
           2 * sizeof(uint64_t);
}

__device__ __forceinline__ void core_stage(int c, int lo, int hi, int ntau, int chc, const CoreJob &J,
                                           WingRec *sw, CoreRec *sc, LineHdr *sh, uint64_t *bar) {
    const int j0 = lo + c * chc;
    const int n = min(chc, hi - j0 + 1);
    const unsigned bw = (unsigned)(n * ntau * (int)sizeof(WingRec)), bc = (unsigned)(n * ntau * (int)sizeof(CoreRec));
    const unsigned bh = (unsigned)(n * (int)sizeof(LineHdr));
    mbar_expect_tx(bar, bw + bc + bh + J.extra_tx);
    tma_bulk_g2s(sw, J.wing + (size_t)j0 * ntau, bw, bar);
    tma_bulk_g2s(sc, J.core + (size_t)j0 * ntau, bc, bar);
    tma_bulk_g2s(sh, J.hdr + j0, bh, bar);
}

// One tile of one job, called by every thread of the CTA with the mbarriers initialised; kk counts
// the chunks the CTA has consumed (their buffer and phase parity) across tiles.  Returns false after a
// copy did not complete within its bound (error in *err).
template <int D>
__device__ bool core_tile(const CoreJob &J, int tile, const float4 *__restrict__ vtab4, unsigned char *smem_raw,
                          int ntau_max, int chc, unsigned &kk, int *err) {
    const int ntau = J.ntau, nwl = J.nwl;
    bool any = false;                              // some segment has core ranges touching the tile
    for (int sg = 0; sg < J.nseg; sg++)
        any = any || J.tile_lo[sg * J.seg_stride + tile] <= J.tile_hi[sg * J.seg_stride + tile];
    if (!any) return true;
    WingRec *sw = (WingRec *)smem_raw;
    CoreRec *sc = (CoreRec *)(sw + 2 * (size_t)chc * ntau_max);
    LineHdr *sh = (LineHdr *)(sc + 2 * (size_t)chc * ntau_max);
    uint64_t *bars = (uint64_t *)(sh + 2 * chc);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t0 = warp * D;
    const int nd = max(0, min(D, ntau - t0));      // warps past the last depth only wait with the others
    const int p = tile * 32 + lane, p1 = p + 1;
    const int tile_first = tile * 32 + 1, tile_last = min(tile * 32 + 32, nwl);
    const double wd = J.wave[min(p, nwl - 1)];
    const float wvh = (float)wd, wvl = (float)(wd - (double)wvh);
    float sum[D], cmp[D];
#pragma unroll
    for (int d = 0; d < D; d++) { sum[d] = 0.0f; cmp[d] = 0.0f; }
    unsigned cnt = 0;
    for (int sg = 0; sg < J.nseg; sg++) {         // the job's segments of lines, in turn
        const int lo = J.tile_lo[sg * J.seg_stride + tile], hi = J.tile_hi[sg * J.seg_stride + tile];
        if (lo > hi) continue;
        const int nchunks = (hi - lo + chc) / chc;
        if (threadIdx.x == 0)
            for (int c = 0; c < 2 && c < nchunks; c++) {
                const int b = (kk + c) & 1;
                core_stage(c, lo, hi, ntau, chc, J, sw + (size_t)b * chc * ntau_max, sc + (size_t)b * chc * ntau_max,
                           sh + b * chc, &bars[b]);
            }
        int failed = -1;
        for (int c = 0; c < nchunks; c++) {
            const unsigned g = kk + c;
            const int b = g & 1;
            const bool ok = mbar_wait(&bars[b], (g >> 1) & 1, J.wait_ns);
            if (__syncthreads_or(!ok)) { failed = c; break; }
            const LineHdr *ch = sh + b * chc;
            const WingRec *cw = sw + (size_t)b * chc * ntau_max;
            const CoreRec *cc = sc + (size_t)b * chc * ntau_max;
            const int n = min(chc, hi - (lo + c * chc) + 1);
            if (nd > 0) {
                for (int q = 0; q < n; q++) {
                    const LineHdr h = ch[q];
                    if (h.cr < tile_first || h.cl > tile_last) continue;          // core range misses the tile
                    const bool in = p1 >= h.cl && p1 <= h.cr;
                    if (!__any_sync(0xffffffffu, in)) continue;
                    const float dl = (wvh - h.wlh) + (wvl - h.wll);
                    const float x = dl * dl;                  // the wing pass's x: the same branch split
                    const double adl = fabs(wd - ((double)h.wlh + (double)h.wll));
#pragma unroll
                    for (int g0 = 0; g0 < D; g0 += 4) {               // depths in groups of four
                        bool core[4], tab[4];
                        float tv[4];
                        int cell[4];
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            const int d = g0 + e;
                            const int td = t0 + min(d, nd - 1);
                            const WingRec w = cw[q * ntau + td];
                            const CoreRec cr = cc[q * ntau + td];
                            const float t = fmaf(x, w.vv2, w.c2m1);
                            core[e] = in && d < nd && t < 195.5f;
                            const double av = adl * cr.vv;
                            tab[e] = core[e] && cr.ia > 0 && av < 8.0;
                            const double fv = av * 125.0;
                            const int iv = tab[e] ? min((int)fv, FSG_NVV - 1) : 0;
                            tv[e] = tab[e] ? (float)(fv - (double)iv) : (float)av;   // CF: |v| in FP32
                            cell[e] = tab[e] ? (cr.ia - 1) * FSG_NV1 + iv : 0;
                        }
                        float4 gv[4];
#pragma unroll
                        for (int e = 0; e < 4; e++)
                            if (tab[e]) gv[e] = __ldg(vtab4 + cell[e]);
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            if (!core[e]) continue;
                            const int d = g0 + e;
                            const CoreRec &cr = cc[q * ntau + t0 + d];
                            float v;
                            if (tab[e]) {
                                const float4 gg = gv[e];
                                const float c0 = gg.x + tv[e] * (gg.y - gg.x), c1 = gg.z + tv[e] * (gg.w - gg.z);
                                v = (c0 + cr.ua * (c1 - c0)) * cr.cop;
                            } else {
                                v = hv_cf32(tv[e], cr.a, cr.cop);
                            }
                            KAHAN(sum[d], cmp[d], v);
                            cnt++;
                        }
                    }
                }
            }
            __syncthreads();                                   // every warp is done with buffer b
            if (threadIdx.x == 0 && c + 2 < nchunks)
                core_stage(c + 2, lo, hi, ntau, chc, J, sw + (size_t)b * chc * ntau_max,
                           sc + (size_t)b * chc * ntau_max, sh + b * chc, &bars[b]);
        }
        if (failed >= 0) {
            if (threadIdx.x == 0) {
                atomicExch(err, FSG_E_TIMEOUT);
                for (int c = failed; c < nchunks && c < failed + 2; c++) {
                    const unsigned g = kk + c;
                    mbar_wait(&bars[g & 1], (g >> 1) & 1, J.wait_ns);
                }
            }
            __syncthreads();
            return false;
        }
        kk += nchunks;
    }
    if (J.nevals) {
        unsigned long long v = cnt;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0 && v) atomicAdd(J.nevals, v);
    }
    if (nd <= 0 || p >= nwl) return true;
    double *dst = J.lineopac + (size_t)p * ntau + t0;
#pragma unroll
    for (int d = 0; d < D; d++)
        if (d < nd) dst[d] = dst[d] + ((double)sum[d] - (double)cmp[d]);
    return true;
}

__device__ __forceinline__ void core_bars_init(unsigned char *smem_raw, int ntau_max, int chc) {
    uint64_t *bars = (uint64_t *)(smem_raw + core_smem(ntau_max, chc) - 2 * sizeof(uint64_t));
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
}

template <int D>
__global__ void __launch_bounds__(32 * 18, D == 4 ? 2 : 1)
k_core_fast(CoreJob J, const float4 *__restrict__ vtab4, int chc, int *__restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    if (J.tile_lo[blockIdx.x] > J.tile_hi[blockIdx.x]) return;
    core_bars_init(smem_raw, J.ntau, chc);
    unsigned kk = 0;
    core_tile<D>(J, blockIdx.x, vtab4, smem_raw, J.ntau, chc, kk, err);
}

// persistent form: CTAs take (job, tile) items from the queue; a CTA of nwarps warps covers
// nwarps * D depths, so every item is taken by whole CTAs
template <int D>
__global__ void __launch_bounds__(32 * 18, D == 4 ? 2 : 1)
k_core_batch(const CoreJob *__restrict__ jobs, const int *__restrict__ tile0, int njobs, int ntau_max, int chc,
             const float4 *__restrict__ vtab4, unsigned *queue, int *__restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ int s_item;
    core_bars_init(smem_raw, ntau_max, chc);
    unsigned kk = 0;
    const int total = tile0[njobs];
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= total) break;
        int a = 0, b = njobs - 1;
        while (a < b) { int m = (a + b + 1) >> 1; if (tile0[m] <= item) a = m; else b = m - 1; }
        if (!core_tile<D>(jobs[a], item - tile0[a], vtab4, smem_raw, ntau_max, chc, kk, err)) break;
    }
}

// lines per staged chunk: about 32 KB of records per buffer, 4 to 16 lines.  The buffers share the
// SM's L1 with the table gathers: per 1e8-line step the core pass took 1.82 / 1.71 / 1.75 / 1.85 s
// with 48 / 32 / 24 / 16 KB.
static int core_chunk(int ntau_max) {
    const int per_line = ntau_max * (int)(sizeof(WingRec) + sizeof(CoreRec)) + (int)sizeof(LineHdr);
    return std::max(4, std::min(16, (32 * 1024) / per_line));
}

// depths per warp: 8 (two groups of four gathers; 4 depths per warp, for up to 72 depths, took 3 %
// longer on the 1e8-line step)
static int core_depths(int) { return 8; }

int fsg_launch_core_fast(cudaStream_t st, int ntau, int nwl, const double *wave, const LineHdr *hdr,
                         const WingRec *wing, const CoreRec *core, const int *tile_lo, const int *tile_hi,
                         const float4 *vtab4, double *lineopac, unsigned long long *nevals, int *err,
                         unsigned extra_tx, unsigned long long wait_ns) {
    const int ntiles = (nwl + 31) / 32;
    const int D = core_depths(ntau), nwarps = (ntau + D - 1) / D;
    if (nwarps > 18) return FSG_E_ARG;
    const int chc = core_chunk(ntau);
    const size_t smem = core_smem(ntau, chc);
    CoreJob J{ ntau, nwl, wave, hdr, wing, core, tile_lo, tile_hi, lineopac, nevals, extra_tx, wait_ns, 1, 0 };
    if (D == 4) {
        cudaFuncSetAttribute(k_core_fast<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_core_fast<4><<<ntiles, 32 * nwarps, smem, st>>>(J, vtab4, chc, err);
    } else {
        cudaFuncSetAttribute(k_core_fast<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_core_fast<8><<<ntiles, 32 * nwarps, smem, st>>>(J, vtab4, chc, err);
    }
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}

int fsg_launch_core_batch(cudaStream_t st, int ntau_max, const CoreJob *jobs, const int *tile0, int njobs,
                          int ctas, const float4 *vtab4, unsigned *queue, int *err) {
    const int D = core_depths(ntau_max), nwarps = (ntau_max + D - 1) / D;
    if (nwarps > 18) return FSG_E_ARG;
    const int chc = core_chunk(ntau_max);
    const size_t smem = core_smem(ntau_max, chc);
    if (D == 4) {
        cudaFuncSetAttribute(k_core_batch<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_core_batch<4><<<ctas, 32 * nwarps, smem, st>>>(jobs, tile0, njobs, ntau_max, chc, vtab4, queue, err);
    } else {
        cudaFuncSetAttribute(k_core_batch<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_core_batch<8><<<ctas, 32 * nwarps, smem, st>>>(jobs, tile0, njobs, ntau_max, chc, vtab4, queue, err);
    }
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}

__global__ void k_tile_reset(int ntiles, int *lo, int *hi) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ntiles) { lo[i] = 0x7fffffff; hi[i] = -1; }
}

// ---- tile candidate ranges of one block: lo/hi of the block-local line index -------------------
// The block's lines are in wavelength order.  With R_j = max_{i<=j} right_i (prefix max) and
// S_j = min_{i>=j} left_i (suffix min), both non-decreasing in j, the lines whose span [left,
// right] meets tile [f, l] all lie in [lo, hi] with lo = first j with R_j >= f and hi = last j
// with S_j <= l; both come from one binary search per tile.  Spans are the windows (use_core = 0)
// or the core ranges (use_core = 1; lines without one are left out).
__device__ __forceinline__ void span_of(const LineHdr &h, int use_core, int *l, int *r) {
    int a = use_core ? h.cl : h.ileft, b = use_core ? h.cr : h.iright;
    if (a > b) { a = 0x7fffffff; b = -1; }
    *l = a; *r = b;
}

// right_j in order, left_j in reverse order (rev[k] = left_{nb-1-k})
__global__ void k_span_extract(int nb, int use_core, const LineHdr *__restrict__ hdr, int *right, int *rev_left) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nb) return;
    int l, r;
    span_of(hdr[j], use_core, &l, &r);
    right[j] = r;
    rev_left[nb - 1 - j] = l;
}

// R: prefix max of right (non-decreasing); V: prefix min of reversed left, S_j = V[nb-1-j]
__global__ void k_tile_search(int nb, int ntiles, int tw, int nwl, const int *__restrict__ R,
                              const int *__restrict__ V, int *lo, int *hi) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    const int f = t * tw + 1, l = min(t * tw + tw, nwl);
    int a = 0, b = nb;                                   // first j with R_j >= f
    while (a < b) { int m = (a + b) >> 1; if (R[m] >= f) b = m; else a = m + 1; }
    const int jlo = a;
    a = 0; b = nb;                                       // first j with S_j > l
    while (a < b) { int m = (a + b) >> 1; if (V[nb - 1 - m] > l) b = m; else a = m + 1; }
    lo[t] = jlo;
    hi[t] = a - 1;
}

// tile count of the narrowest tiles (sizes the lo/hi arrays)
int fsg_fast_tiles(int nwl) { return (nwl + 31) / 32; }

// scratch bytes of fsg_launch_tile_span for nb lines
size_t fsg_tile_span_scratch(int64_t nb) {
    size_t t1 = 0, t2 = 0;
    cub::DeviceScan::InclusiveScan(nullptr, t1, (const int *)nullptr, (int *)nullptr, cuda::maximum<>{}, (int)nb);
    cub::DeviceScan::InclusiveScan(nullptr, t2, (const int *)nullptr, (int *)nullptr, cuda::minimum<>{}, (int)nb);
    return 4 * sizeof(int) * (size_t)nb + std::max(t1, t2) + 256;
}

int fsg_launch_tile_span_tw(cudaStream_t s, int tw, int use_core, int nwl, int64_t nb, const LineHdr *hdr, int *lo,
                            int *hi, void *scratch, size_t scratch_bytes);

int fsg_launch_tile_span(cudaStream_t s, int cls, int nwl, int64_t nb, const LineHdr *hdr, int *lo, int *hi,
                         void *scratch, size_t scratch_bytes) {
    return fsg_launch_tile_span_tw(s, cls < 0 ? 32 : 32 * fsg_class_pix(cls), cls < 0 ? 1 : 0, nwl, nb, hdr, lo, hi,
                                   scratch, scratch_bytes);
}

// tile ranges for tiles of tw wavelengths over the windows (use_core = 0) or the core ranges
int fsg_launch_tile_span_tw(cudaStream_t s, int tw, int use_core, int nwl, int64_t nb, const LineHdr *hdr, int *lo,
                            int *hi, void *scratch, size_t scratch_bytes) {
    const int ntiles = (nwl + tw - 1) / tw;
    if (nb <= 0) {
        k_tile_reset<<<(ntiles + 255) / 256, 256, 0, s>>>(ntiles, lo, hi);
        return FSG_OK;
    }
    int *right = (int *)scratch, *revl = right + nb, *R = revl + nb, *V = R + nb;
    void *tmp = (void *)(((uintptr_t)(V + nb) + 255) & ~(uintptr_t)255);
    size_t tb = scratch_bytes - ((char *)tmp - (char *)scratch);
    k_span_extract<<<(unsigned)((nb + 255) / 256), 256, 0, s>>>((int)nb, use_core, hdr, right, revl);
    if (cub::DeviceScan::InclusiveScan(tmp, tb, right, R, cuda::maximum<>{}, (int)nb, s) != cudaSuccess) return FSG_E_CUDA;
    if (cub::DeviceScan::InclusiveScan(tmp, tb, revl, V, cuda::minimum<>{}, (int)nb, s) != cudaSuccess) return FSG_E_CUDA;
    k_tile_search<<<(ntiles + 255) / 256, 256, 0, s>>>((int)nb, ntiles, tw, nwl, R, V, lo, hi);
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}

// Restriction to the wavelength range [i0, i1]: lines whose window misses it are marked weak for the
// selection, the others keep their flags and get the window clipped to the range.
__global__ void k_range_clip(int64_t n, const int32_t *fl, const int32_t *il, const int32_t *ir, int i0, int i1,
                             int32_t *rf, int32_t *rl, int32_t *rr) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int f = fl[i], a = max(il[i], i0), b = min(ir[i], i1);
    if (a > b) f |= FSG_F_WEAK;
    rf[i] = f; rl[i] = a; rr[i] = b;
}

void fsg_launch_range_clip(cudaStream_t s, int64_t n, const int32_t *fl, const int32_t *il, const int32_t *ir, int i0,
                           int i1, int32_t *rf, int32_t *rl, int32_t *rr) {
    if (n > 0) k_range_clip<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, fl, il, ir, i0, i1, rf, rl, rr);
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
// selection predicate: cls >= 0 retained lines of that width class (He I shifted lines excluded),
// -1 every retained line, -2 retained wide lines (flag bit 3), -3 retained He I shifted lines
__device__ __forceinline__ int sel_pred(int f, int il, int ir, int cls) {
    if (f & FSG_F_WEAK) return 0;
    if (cls == -1) return 1;
    if (cls == -2) return (f & FSG_F_WIDE) != 0;
    if (cls == -3) return ((f >> 8) & 255) != 0;         // He I lines with Stark-shifted profiles
    if ((f >> 8) & 255) return 0;                        // ... which the FP32 classes leave out
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
    if (i >= n || (flags[i] & FSG_F_WEAK) || ((flags[i] >> 8) & 255)) return;
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

// ---- batched lists: records in window-width-class order --------------------------------------
// An atmosphere of a batch keeps its candidate lines in one record array, grouped by window-width
// class (retained lines of class 0, 1, ..., ncls - 1, then the rejected ones), in list (wavelength)
// order inside each class.  A tile's candidate range is then searched inside one class, so it spans
// lines of like width only: the prefix-max / suffix-min spans of a single list with a few very wide
// windows would stage every line between such a window's centre and the tile.
#define BCLS_MAX 24

// class of a line for the record order: ncls for rejected lines (and empty windows)
__device__ __forceinline__ int bclass_of(int f, int il, int ir, int ncls) {
    if ((f & FSG_F_WEAK) || il > ir) return ncls;
    return min(width_class(il, ir), ncls - 1);
}

// lines per class and CTA of SCAN_BS lines: counts[c * nblk + blk], c = 0 .. ncls
__global__ void k_bclass_count(int64_t n, const int32_t *__restrict__ flags, const int32_t *__restrict__ il,
                               const int32_t *__restrict__ ir, int ncls, int *counts) {
    __shared__ int h[BCLS_MAX + 1];
    for (int c = threadIdx.x; c <= ncls; c += blockDim.x) h[c] = 0;
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * SCAN_BS + threadIdx.x;
    if (i < n) atomicAdd(&h[bclass_of(flags[i], il[i], ir[i], ncls)], 1);
    __syncthreads();
    for (int c = threadIdx.x; c <= ncls; c += blockDim.x) counts[c * gridDim.x + blockIdx.x] = h[c];
}

// order[offs[c * nblk + blk] + rank of line i among the CTA's class-c lines] = i (stable)
__global__ void k_bclass_scatter(int64_t n, const int32_t *__restrict__ flags, const int32_t *__restrict__ il,
                                 const int32_t *__restrict__ ir, int ncls, const int64_t *__restrict__ offs,
                                 int64_t *order) {
    __shared__ int wc[SCAN_BS / 32][BCLS_MAX + 1];       // per warp and class: count, then prefix over warps
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < (SCAN_BS / 32) * (BCLS_MAX + 1); k += blockDim.x) (&wc[0][0])[k] = 0;
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * SCAN_BS + threadIdx.x;
    const int c = i < n ? bclass_of(flags[i], il[i], ir[i], ncls) : -1;
    const unsigned same = __match_any_sync(0xffffffffu, c);
    const int rank = __popc(same & ((1u << lane) - 1u));
    if (c >= 0 && rank == 0) wc[w][c] = __popc(same);  // the class's lowest lane in the warp
    __syncthreads();
    if (threadIdx.x <= ncls) {
        int acc = 0;
        for (int q = 0; q < SCAN_BS / 32; q++) { const int t = wc[q][threadIdx.x]; wc[q][threadIdx.x] = acc; acc += t; }
    }
    __syncthreads();
    if (c >= 0) order[offs[c * gridDim.x + blockIdx.x] + wc[w][c] + rank] = i;
}

// Class order of n lines (ncls <= BCLS_MAX classes + the rejected): order[n] and the class offsets,
// class c starting at record offs[c * nblk] (nblk = ceil(n / SCAN_BS)); counts and offs hold
// (ncls + 1) * nblk entries.
int fsg_launch_bclass_order(cudaStream_t s, int64_t n, const int32_t *flags, const int32_t *il, const int32_t *ir,
                            int ncls, int *counts, int64_t *offs, int64_t *total, int64_t *order) {
    if (n <= 0 || ncls < 1 || ncls > BCLS_MAX) return n <= 0 ? FSG_OK : FSG_E_ARG;
    const int nblk = (int)((n + SCAN_BS - 1) / SCAN_BS);
    k_bclass_count<<<nblk, SCAN_BS, 0, s>>>(n, flags, il, ir, ncls, counts);
    k_scan_counts<<<1, 1024, 0, s>>>((ncls + 1) * nblk, counts, offs, total);
    k_bclass_scatter<<<nblk, SCAN_BS, 0, s>>>(n, flags, il, ir, ncls, offs, order);
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}

// classes of an atmosphere's order: every window fits the grid, so the widest class is that of nwl
int fsg_bclass_count(int nwl) {
    int c = 0;
    while ((CLASS_W0 << (c + 1)) < nwl && c < 30) c++;
    return std::min(c + 1, BCLS_MAX);
}

// Segmented spans: key = class << 32 | value, so one prefix max (of right + 1) and one suffix min
// (of left) over the whole record array stay inside each class, and both key arrays are sorted.
__global__ void k_bspan_extract(int nb, int use_core, const LineHdr *__restrict__ hdr,
                                const int64_t *__restrict__ offs, int nblk, int ncls, unsigned long long *right,
                                unsigned long long *rev_left) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nb) return;
    int seg = 0;
    while (seg < ncls && offs[(seg + 1) * nblk] <= j) seg++;
    int l, r;
    span_of(hdr[j], use_core, &l, &r);
    if (seg == ncls) { l = 0x7fffffff; r = -1; }
    right[j] = ((unsigned long long)seg << 32) | (unsigned)(r + 1);
    rev_left[nb - 1 - j] = ((unsigned long long)seg << 32) | (unsigned)l;
}

// Tile t of class c (blockIdx.y): tiles of tw_n wavelengths for classes <= cnarrow, tw_w for the
// others; lo/hi at c * tstride + t are record indices of class c (lo > hi: no line touches it).
__global__ void k_btile_search(int nb, int cnarrow, int tw_n, int tw_w, int nwl, int tstride,
                               const unsigned long long *__restrict__ R, const unsigned long long *__restrict__ V,
                               int *lo, int *hi) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
    const int tw = c <= cnarrow ? tw_n : tw_w;
    if (t >= (nwl + tw - 1) / tw) return;
    const int f = t * tw + 1, l = min(t * tw + tw, nwl);
    const unsigned long long kf = ((unsigned long long)c << 32) | (unsigned)(f + 1);
    const unsigned long long kl = ((unsigned long long)c << 32) | (unsigned)l;
    int a = 0, b = nb;                                   // first j with R_j >= kf
    while (a < b) { const int m = (a + b) >> 1; if (R[m] >= kf) b = m; else a = m + 1; }
    const int jlo = a;
    a = 0; b = nb;                                       // first j with S_j > kl, S_j = V[nb - 1 - j]
    while (a < b) { const int m = (a + b) >> 1; if (V[nb - 1 - m] > kl) b = m; else a = m + 1; }
    lo[c * tstride + t] = jlo;
    hi[c * tstride + t] = a - 1;
}

size_t fsg_bspan_scratch(int64_t nb) {
    size_t t1 = 0, t2 = 0;
    typedef unsigned long long u64;
    cub::DeviceScan::InclusiveScan(nullptr, t1, (const u64 *)nullptr, (u64 *)nullptr, cuda::maximum<>{}, (int)nb);
    cub::DeviceScan::InclusiveScan(nullptr, t2, (const u64 *)nullptr, (u64 *)nullptr, cuda::minimum<>{}, (int)nb);
    return 4 * sizeof(u64) * (size_t)nb + std::max(t1, t2) + 256;
}

// tile ranges of every class of a class-ordered record array (offs from fsg_launch_bclass_order)
int fsg_launch_btile_span(cudaStream_t s, int use_core, int64_t nb, const LineHdr *hdr, const int64_t *offs,
                          int ncls, int cnarrow, int tw_n, int tw_w, int nwl, int tstride, int *lo, int *hi,
                          void *scratch, size_t scratch_bytes) {
    typedef unsigned long long u64;
    if (nb <= 0) {
        for (int c = 0; c < ncls; c++) k_tile_reset<<<(tstride + 255) / 256, 256, 0, s>>>(tstride, lo + c * tstride,
                                                                                          hi + c * tstride);
        return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
    }
    const int nblk = (int)((nb + SCAN_BS - 1) / SCAN_BS);
    u64 *right = (u64 *)scratch, *revl = right + nb, *R = revl + nb, *V = R + nb;
    void *tmp = (void *)(((uintptr_t)(V + nb) + 255) & ~(uintptr_t)255);
    size_t tb = scratch_bytes - ((char *)tmp - (char *)scratch);
    k_bspan_extract<<<(unsigned)((nb + 255) / 256), 256, 0, s>>>((int)nb, use_core, hdr, offs, nblk, ncls, right, revl);
    if (cub::DeviceScan::InclusiveScan(tmp, tb, right, R, cuda::maximum<>{}, (int)nb, s) != cudaSuccess) return FSG_E_CUDA;
    if (cub::DeviceScan::InclusiveScan(tmp, tb, revl, V, cuda::minimum<>{}, (int)nb, s) != cudaSuccess) return FSG_E_CUDA;
    const int tmax = (nwl + std::min(tw_n, tw_w) - 1) / std::min(tw_n, tw_w);
    k_btile_search<<<dim3((tmax + 255) / 256, ncls), 256, 0, s>>>((int)nb, cnarrow, tw_n, tw_w, nwl, tstride, R, V,
                                                                  lo, hi);
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
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
