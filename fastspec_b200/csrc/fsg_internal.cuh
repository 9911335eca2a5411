// fsg_internal.cuh -- shared definitions of the B200 line-opacity / formal-solver library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/fastspec_gpu.h"

// ---- physical constants (shared.f90:20-33) --------------------------------------------------
#define FSG_PI        3.141592653589793115997963468544185161590576171875
#define FSG_VC        299792.458
#define FSG_HC        6.62607015e-27
#define FSG_KBOLT     1.380649e-16
#define FSG_EV2ANG    8065.544005e-8
#define FSG_A0        5.29177210903e-11
#define FSG_M0        1.66053906660e-27
#define FSG_CE        4.803204712e-10
#define FSG_ME        9.1093837139e-28
#define FSG_MH        1.673532499e-24
#define FSG_HIE       13.598434005
#define FSG_KZ        4.668644778e-13
#define FSG_SQRTPIINV 0.56418958354775628695

// ---- Voigt table geometry (voigt.f90:19-26) ------------------------------------------------
#define FSG_NVV 1001
#define FSG_NVA 401
#define FSG_NV1 (FSG_NVV + 1)    // 1002 v nodes, v in [0, 8], dv = 0.008
#define FSG_NA1 (FSG_NVA + 1)    // 402 a nodes, sqrt(a) uniform in [0, sqrt(8)]

// Per-line flag bits (synth.f90:850 and opacity.f90:314): 0 weak, 1 molecule, 2 ABO,
// 3 wide, 8..15 He I Stark table entry.
#define FSG_F_WEAK 1
#define FSG_F_MOL  2
#define FSG_F_ABO  4
#define FSG_F_WIDE 8

// Per-depth precomputation of XlineInit (opacity.f90:65-93), FP64, one row each.
enum { XI_NPRTB = 0, XI_GVWPRT, XI_TEMP6, XI_TEMP3, XI_KBT, XI_KBET, XI_T, XI_XNE, XI_RHO, XI_NROWS };

// Device view of one atmosphere + grid + configuration (passed by value to kernels).
struct AtmView {
    int     ntau, nspc, nwl, wmode, motype, nhe, spc_he1, molbrd;
    double  wfirst, wstart, dstep, rstep;
    double  vturb2, epsopac, vwfudge, vwmol;
    const double *xi;          // [XI_NROWS][ntau]
    const float  *fpf;         // [nspc][ntau]   species-major (transposed on upload)
    const float  *xamass, *potion;
    const int    *ion;
    const double *wave;        // [nwl] offsets from wfirst
    const double *contopac;    // [nwl][ntau]
    const double *contstd;     // [ntau] or null
    const double *hegam, *heshf;   // [nhe][ntau] or null
};

// Device view of a line list (SoA, device pointers).
struct LineView {
    int64_t n;
    int     kind;
    const double  *wl;
    const float   *elo, *gf, *grad, *gqst, *gvdw;
    const int32_t *spc, *ismol, *ihe;
};

// XlineCoef (opacity.f90:43-58)
struct XCoef {
    double WaveL, Hnux, Elo, Gf, Grad, Xmass, Cqst, Qdiv, Cvdw, AboPre, AboVbc, AboExp;
    int    IxPF, MdQst, MdVdw, IxHe;
};

// Fast-path record of one (line, depth): FP32 wing coefficients of HVoigt * LinCop.
// For s = v^2 + a^2 >= 196 the reference evaluates (voigt.f90:100-101)
//   H = a (s + 1/2) / (sqrt(pi) (s^2 - v^2 + a^2 + 1/4)).
// With y = s + 1/2 the denominator is exactly (y - 1)^2 + 2 a^2, so with t = y - 1
//   H * LinCop = c1 (t + 1) / (t^2 + twoA),  t = dl^2 vv2 + c2m1,
// with vv2 = LinVvgt^2, c2m1 = a^2 - 1/2, twoA = 2 a^2, c1 = LinCop a / sqrt(pi).
struct __align__(16) WingRec { float vv2, c2m1, twoA, c1; };
// Table / continued-fraction region (s < 196): LinVvgt in FP64, LinCop, a, and the table row ia
// (1-based) with its interpolation weight ua as HVoigt derives them from a in FP64
// (voigt.f90:84-92); ia = 0 when a >= 8 (no table).  v = |dl| LinVvgt and the table column and
// fraction are formed in FP64 as the reference forms them: on the Gaussian flanks of a line core
// H falls as exp(-v^2), so an FP32 v (relative error ~1e-7) would move H by 2 v^2 * 1e-7.
struct __align__(16) CoreRec { double vv; float cop, ua, a; int ia; int pad0, pad1; };
static_assert(sizeof(CoreRec) == 32, "core record: 32 bytes");

// Line header of a retained line inside a block (fast path).  The centre offset Wlcent is split
// into FP32 wlh + wll (wlh = fl32(Wlcent), wll = fl32(Wlcent - wlh)).  [cl, cr] is the core range:
// every wavelength index of the window where some depth may have s < 196 lies inside it
// (cl > cr when no depth has a core).  pad0 holds, in the wing pass's headers, the FP32 bits of the
// x = dl^2 that makes every depth's wing term exactly 0 (points outside the window or inside the core
// range of a partly covered tile); the magnetic pass keeps its He I table index there.
struct __align__(16) LineHdr { float wlh, wll; int ileft, iright; int cl, cr, pad0, pad1; };

// Zeeman components of a device line list (CSR by line)
struct ZView {
    const int32_t *npi, *nsi;
    const int64_t *pi_off, *si_off;
    const float *strpi, *strsi;
    float *splpi, *splsi;             // shifts scaled to [A] (written by the magnetic central pass)
    const float *rawpi, *rawsi;       // shifts as read (Lande-type units)
};

// The reference's per-line and block arrays as the elemental routines read them (device pointers):
// Wlcent, LinFlag, Ileft, Iright per line; LinCop, LinVvgt, LinAvgt [nblock][ntau] per block line.
struct BlockView {
    const double *wlcent;
    const int32_t *flags, *ileft, *iright;
    const double *cop, *vv, *av;
};
static_assert(sizeof(XCoef) == sizeof(fsg_xcoef), "fsg_xcoef mirrors XCoef");

// One wing-pass job: the line records and tiles of one LineOpac (one atmosphere and grid).  Its
// tile ranges come in nseg segments (window-width classes of one record array), segment s at
// tile_lo / tile_hi + s * seg_stride; a tile takes the segments' lines in turn into one sum.
// extra_tx / wait_ns: 0 and WAIT_NS in use; a test of the error path (fsg_set_fault) makes every
// chunk expect extra_tx bytes more than its copies deliver and bounds the waits by wait_ns.
struct WingJob {
    int ntau, nwl;
    const double *wave;
    const LineHdr *hdr;
    const WingRec *wing;
    const int *tile_lo, *tile_hi;
    double *lineopac;
    unsigned extra_tx;
    unsigned long long wait_ns;
    int nseg, seg_stride;
};

// One core-pass job: as WingJob plus the core records; tiles of 32 wavelengths.  nevals (may be
// null) counts the evaluations.
struct CoreJob {
    int ntau, nwl;
    const double *wave;
    const LineHdr *hdr;
    const WingRec *wing;
    const CoreRec *core;
    const int *tile_lo, *tile_hi;
    double *lineopac;
    unsigned long long *nevals;
    unsigned extra_tx;
    unsigned long long wait_ns;
    int nseg, seg_stride;
};

// Rays of a spherical model (SphereInit, solver.f90:45-120), device arrays [nmu][stride], stride =
// 2 ntau.  Ray im has n[im] points (ntau, or 2 n for a grazing ray that turns below layer n); point k
// samples layer map[im][k] (0-based) at column mass m[im][k] along the ray.  nmu = 0: plane-parallel.
struct RayView {
    int nmu, stride;
    const int *n, *graz, *map;
    const double *m;
};

// Error reporting
std::string fsg_cuda_msg(cudaError_t e, const char *what);

// Tables in device memory (built by fsg_tables.cu).
struct VoigtTables {
    float  *vtab;      // [402][1002]
    float4 *vtab4;     // [401][1002]: (T[r][i], T[r][i+1], T[r+1][i], T[r+1][i+1]) -- one load per lerp
    float2 *fvtab;     // [402][1002] (H, L)
    float4 *fvtab2;    // [402][1002]: (H, L) at v nodes i and i + 1 of a row -- one 16-byte load per row of a lerp
    double *anode, *aida;   // [402] each
};
int fsg_build_tables(VoigtTables *t, cudaStream_t s, std::string *err);
void fsg_free_tables(VoigtTables *t);
