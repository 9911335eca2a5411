// fsg_magfast.cu -- mixed-precision magnetic line opacity (MagLineOpacity1/3, opacity.f90:391-464,
// 526-591) on wavelength tiles.
//
// MagLineOpac(6, t, lambda) = sum over lines and Zeeman components of (H, L)(a, v_k) LinCop Str_k,
// v_k = (lambda - lambda_c - shift_k) LinVvgt, into the pi / sigma-blue / sigma-red absorption
// (H) and dispersion (L) planes.  A CTA owns 32 wavelengths (lanes) x a slab of MAG_W * MAG_D
// depths (blockIdx.y; warps of MAG_D depths); per line the components are evaluated in FP32 -- FVoigt's table lerp of FvTab
// for a < 8, |v| < 8, its rational wing pair for s = v^2 + a^2 >= 196, the two-term continued
// fraction between (voigt.f90:256-352) -- summed per line in FP32 and added to FP64 accumulators.
// The per-(line, depth) records come from the FP64 XlineDepth values (k_mag_params_fast).
#include "fsg_fp64.cuh"

#define MAG_D 4
#define MAG_W 8

struct __align__(16) MagRec { float vv, cop, a, ua; int ia, pad0, pad1, pad2; };

// Records of a block's lines, and per line its header with the core range [cl, cr]: every wavelength
// of the window where some depth and Zeeman component may have s = v^2 + a^2 < 196 (half-width
// max_t sqrt(196.05 - a^2) / LinVvgt, + the largest |component shift| and |He I shift|, + one
// wavelength); outside it every point takes FVoigt's rational wing pair.
__global__ void k_mag_params_fast(AtmView A, LineView L, ZView Z, const int64_t *__restrict__ idx, int64_t j0,
                                  int64_t nb, const int32_t *__restrict__ flags, const int32_t *__restrict__ ileft,
                                  const int32_t *__restrict__ iright, const double *__restrict__ anode,
                                  const double *__restrict__ aida, MagRec *rec, LineHdr *hdr, int64_t *zidx) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nb) return;
    const int64_t i = idx[j0 + j];
    const int nt = A.ntau;
    const int f = flags[i];
    const double wlc = L.wl[i] - A.wfirst;
    XCoef XC;
    xline_setup(A, L, i, wlc, f, &XC);
    const float an1 = (float)anode[1], ai0 = (float)aida[0];
    const int ihe = (f >> 8) & 255;
    double hcore = -1.0, shmax = 0.0;
    for (int t = 0; t < nt; t++) {
        double cop, vv, av;
        xline_depth(A, t, XC, &cop, &vv, &av);
        const double q = 196.05 - av * av;
        if (q > 0.0) hcore = fmax(hcore, sqrt(q) / vv * (1.0 + 1e-5));
        if (ihe > 0) shmax = fmax(shmax, fabs(A.heshf[(size_t)(ihe - 1) * nt + t]));
        if (A.motype == 1) cop = cop / A.contstd[t];
        MagRec r;
        r.vv = (float)vv; r.cop = (float)cop; r.a = (float)av;
        if (!(r.a < 8.0f)) { r.ia = 0; r.ua = 0.0f; }
        else if (r.a < an1) { r.ia = 1; r.ua = r.a * ai0; }
        else {
            int ia = min((int)(sqrtf(r.a) * 141.42135623730951f) + 1, FSG_NVA);
            r.ia = ia;
            r.ua = (r.a - (float)anode[ia - 1]) * (float)aida[ia - 1];
        }
        r.pad0 = r.pad1 = r.pad2 = 0;
        rec[(size_t)j * nt + t] = r;
    }
    LineHdr h;
    h.wlh = (float)wlc;
    h.wll = (float)(wlc - (double)h.wlh);
    h.ileft = ileft[i]; h.iright = iright[i];
    h.cl = 1; h.cr = 0;
    if (hcore >= 0.0) {
        double zmax = 0.0;
        for (int k = 0; k < Z.npi[i]; k++) zmax = fmax(zmax, fabs((double)Z.splpi[Z.pi_off[i] + k]));
        for (int k = 0; k < Z.nsi[i]; k++) zmax = fmax(zmax, fabs((double)Z.splsi[Z.si_off[i] + k]));
        const double half = hcore + zmax + shmax;
        int a = lower_index(A.wave, A.nwl, wlc - half) + 1;
        int b = lower_index(A.wave, A.nwl, wlc + half);
        if (b < A.nwl && A.wave[b] == wlc + half) b++;
        const int cl = max(a - 1, h.ileft), cr = min(b + 1, h.iright);
        if (cl <= cr) { h.cl = cl; h.cr = cr; }
    }
    h.pad0 = ihe;                                     // He I table index (0: none)
    h.pad1 = 0;
    hdr[j] = h;
    zidx[j] = i;
}

__device__ __forceinline__ float rcp_approx_m(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// FVoigt (H, L) in FP32 at v (signed), L odd in v.  The table lerp takes each row's two v nodes in one
// 16-byte load (fvtab2); the wing and continued-fraction forms take one approximate reciprocal.
__device__ __forceinline__ void fv32(const float4 *__restrict__ fvtab2, const MagRec &r, float v, float &H, float &L) {
    const float av = fabsf(v), a = r.a, a2 = a * a, v2 = av * av, s = v2 + a2;
    if (r.ia > 0 && av < 8.0f) {
        const float fv = av * 125.0f;
        const int iv = min((int)fv, FSG_NVV - 1);
        const float tv = fv - (float)iv;
        const float4 *p0 = fvtab2 + (r.ia - 1) * FSG_NV1 + iv;
        const float4 g0 = __ldg(p0), g1 = __ldg(p0 + FSG_NV1);      // (H_i, L_i, H_i+1, L_i+1) of rows ia, ia+1
        const float h0 = g0.x + tv * (g0.z - g0.x), h1 = g1.x + tv * (g1.z - g1.x);
        const float l0 = g0.y + tv * (g0.w - g0.y), l1 = g1.y + tv * (g1.w - g1.y);
        H = h0 + r.ua * (h1 - h0);
        L = l0 + r.ua * (l1 - l0);
    } else if (s >= 196.0f) {
        const float w = 0.56418958354775628f * rcp_approx_m(s * s - v2 + a2 + 0.25f);
        H = w * a * (s + 0.5f);
        L = w * av * (s - 0.5f);
    } else {
        const float p = v2 - a2 - 1.5f, q = 2.0f * av * a;
        const float dr = av * p - a * q, di = av * q + a * p;
        const float w = 0.56418958354775628f * rcp_approx_m(dr * dr + di * di);
        H = w * ((p + 0.5f) * di - q * dr);
        L = w * ((p + 0.5f) * dr + q * di);
    }
    L = copysignf(fabsf(L), v);
}

__global__ void __launch_bounds__(32 * MAG_W)
k_mag_fast(int ntau, int nwl, const double *__restrict__ wave, const LineHdr *__restrict__ hdr,
           const MagRec *__restrict__ rec, const int64_t *__restrict__ zidx, ZView Z, const double *__restrict__ heshf,
           const int *__restrict__ tile_lo, const int *__restrict__ tile_hi, const float4 *__restrict__ fvtab2,
           double *__restrict__ mlo) {
    const int tile = blockIdx.x;
    const int lo = tile_lo[tile], hi = tile_hi[tile];
    if (lo > hi) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t0 = (blockIdx.y * MAG_W + warp) * MAG_D;
    const int nd = min(MAG_D, ntau - t0);
    if (nd <= 0) return;
    const int p = tile * 32 + lane, p1 = p + 1;
    const int tile_first = tile * 32 + 1, tile_last = min(tile * 32 + 32, nwl);
    const double wd = wave[min(p, nwl - 1)];
    const float wvh = (float)wd, wvl = (float)(wd - (double)wvh);
    double acc[MAG_D][6];
#pragma unroll
    for (int d = 0; d < MAG_D; d++)
#pragma unroll
        for (int q = 0; q < 6; q++) acc[d][q] = 0.0;
    for (int j = lo; j <= hi; j++) {
        const LineHdr h = hdr[j];
        if (h.iright < tile_first || h.ileft > tile_last) continue;      // window misses the tile
        if (p1 < h.ileft || p1 > h.iright) continue;
        const float dl = (wvh - h.wlh) + (wvl - h.wll);
        MagRec r[MAG_D];
        float vb[MAG_D];
#pragma unroll
        for (int d = 0; d < MAG_D; d++) {
            const int t = t0 + min(d, nd - 1);
            r[d] = rec[(size_t)j * ntau + t];
            const float sh = h.pad0 > 0 ? (float)heshf[(size_t)(h.pad0 - 1) * ntau + t] : 0.0f;
            vb[d] = (dl - sh) * r[d].vv;
        }
        const int64_t zi = zidx[j];
        const int np = Z.npi[zi], ns = Z.nsi[zi], nsh = ns / 2;
        const float *spi = Z.splpi + Z.pi_off[zi], *ssi = Z.splsi + Z.si_off[zi];
        const float *rpi = Z.strpi + Z.pi_off[zi], *rsi = Z.strsi + Z.si_off[zi];
        float s[MAG_D][6];
#pragma unroll
        for (int d = 0; d < MAG_D; d++)
#pragma unroll
            for (int q = 0; q < 6; q++) s[d][q] = 0.0f;
        if (h.cl > h.cr || h.cr < tile_first || h.cl > tile_last) {
            // the tile lies outside the line's core range: every point takes the wing pair, here as
            // H = a/sqrt(pi) (u + a^2 + 1/2) / D and L = v/sqrt(pi) (u + a^2 - 1/2) / D with u = v^2 and
            // D = s^2 - v^2 + a^2 + 1/4 = u (u + 2a^2 - 1) + (a^2 + 1/2)^2 (voigt.f90:280-289)
            float b1[MAG_D], b0[MAG_D], ah[MAG_D], am[MAG_D];
#pragma unroll
            for (int d = 0; d < MAG_D; d++) {
                const float a2 = r[d].a * r[d].a;
                b1[d] = 2.0f * a2 - 1.0f; ah[d] = a2 + 0.5f; am[d] = a2 - 0.5f; b0[d] = ah[d] * ah[d];
            }
            auto comps = [&](const float *sp_, const float *st_, int k0, int k1, int qh) {
                for (int k = k0; k < k1; k++) {
                    const float sp = sp_[k], st = st_[k];
#pragma unroll
                    for (int d = 0; d < MAG_D; d++) {
                        const float v = fmaf(-sp, r[d].vv, vb[d]);
                        const float u = v * v;
                        const float rr = rcp_approx_m(fmaf(u, u + b1[d], b0[d]));
                        s[d][qh] = fmaf(st, (u + ah[d]) * rr, s[d][qh]);
                        s[d][qh + 3] = fmaf(st, (u + am[d]) * rr * v, s[d][qh + 3]);
                    }
                }
            };
            comps(spi, rpi, 0, np, 0);
            comps(ssi, rsi, 0, nsh, 1);
            comps(ssi, rsi, nsh, ns, 2);
#pragma unroll
            for (int d = 0; d < MAG_D; d++) {
                const float ch = 0.56418958354775628f * r[d].a * r[d].cop, cv = 0.56418958354775628f * r[d].cop;
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    acc[d][q] += (double)(s[d][q] * ch);
                    acc[d][q + 3] += (double)(s[d][q + 3] * cv);
                }
            }
            continue;
        }
        for (int k = 0; k < np; k++) {
            const float sp = spi[k], st = rpi[k];
#pragma unroll
            for (int d = 0; d < MAG_D; d++) {
                float H, L;
                fv32(fvtab2, r[d], vb[d] - sp * r[d].vv, H, L);
                s[d][0] += st * H; s[d][3] += st * L;
            }
        }
        for (int k = 0; k < ns; k++) {
            const float sp = ssi[k], st = rsi[k];
            const int qa = k < nsh ? 1 : 2;
#pragma unroll
            for (int d = 0; d < MAG_D; d++) {
                float H, L;
                fv32(fvtab2, r[d], vb[d] - sp * r[d].vv, H, L);
                if (qa == 1) { s[d][1] += st * H; s[d][4] += st * L; }
                else { s[d][2] += st * H; s[d][5] += st * L; }
            }
        }
#pragma unroll
        for (int d = 0; d < MAG_D; d++)
#pragma unroll
            for (int q = 0; q < 6; q++) acc[d][q] += (double)(s[d][q] * r[d].cop);
    }
    if (p >= nwl) return;
#pragma unroll
    for (int d = 0; d < MAG_D; d++) {
        if (d >= nd) break;
        double *dst = mlo + ((size_t)p * ntau + t0 + d) * 6;
#pragma unroll
        for (int q = 0; q < 6; q++) dst[q] = dst[q] + acc[d][q];
    }
}

void fsg_launch_mag_params_fast(cudaStream_t s, const AtmView &A, const LineView &L, const ZView &Z, const int64_t *idx,
                                int64_t j0, int64_t nb, const int32_t *flags, const int32_t *il, const int32_t *ir,
                                const VoigtTables &T, void *rec, LineHdr *hdr, int64_t *zidx) {
    if (nb > 0)
        k_mag_params_fast<<<(unsigned)((nb + 127) / 128), 128, 0, s>>>(A, L, Z, idx, j0, nb, flags, il, ir, T.anode,
                                                                       T.aida, (MagRec *)rec, hdr, zidx);
}

size_t fsg_mag_rec_bytes() { return sizeof(MagRec); }

int fsg_launch_mag_fast(cudaStream_t s, const AtmView &A, const LineHdr *hdr, const void *rec, const int64_t *zidx,
                        const ZView &Z, const int *tlo, const int *thi, const VoigtTables &T, double *mlo) {
    const dim3 grid((A.nwl + 31) / 32, (A.ntau + MAG_W * MAG_D - 1) / (MAG_W * MAG_D));
    k_mag_fast<<<grid, 32 * MAG_W, 0, s>>>(A.ntau, A.nwl, A.wave, hdr, (const MagRec *)rec, zidx, Z, A.heshf, tlo,
                                              thi, T.fvtab2, mlo);
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}
