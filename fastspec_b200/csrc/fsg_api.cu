// fsg_api.cu -- C-ABI entry points: context, uploads, and the LineopCalc / RadTranCalc drivers.
#include "fsg_internal.cuh"
#include "fsg_mbar.cuh"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <mutex>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

// ---- tracing and metrics of the C-ABI drivers -----------------------------------------------------
// The reference reports each stage of a synthesis (lines read and used, time of the line opacity, then
// of the radiative transfer: fastspec.f90:393-425, timed by MDtime, utils.f90:63-91).  Here every driver
// call is an NVTX range (visible to Nsight Systems and to ncu's NVTX filters), and when the environment
// names a file in FSG_METRICS_JSONL each call appends one JSON line to it: the call, its status, its host
// wall time and the stage figures it produced.
namespace {
struct CallTrace {
    std::chrono::steady_clock::time_point t0;
    explicit CallTrace(const char *name) : t0(std::chrono::steady_clock::now()) { nvtxRangePushA(name); }
    ~CallTrace() { nvtxRangePop(); }
    double ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};
std::mutex g_metrics_mu;
bool metrics_on() {
    const char *p = getenv("FSG_METRICS_JSONL");
    return p && *p;
}
void metrics_emit(const char *call, int rc, double wall_ms, const std::string &fields) {
    const char *path = getenv("FSG_METRICS_JSONL");
    if (!path || !*path) return;
    std::lock_guard<std::mutex> lock(g_metrics_mu);
    FILE *f = fopen(path, "a");
    if (!f) return;
    fprintf(f, "{\"call\": \"%s\", \"rc\": %d, \"wall_ms\": %.6f%s%s}\n", call, rc, wall_ms,
            fields.empty() ? "" : ", ", fields.c_str());
    fclose(f);
}
std::string stats_fields(const fsg_stats &t) {
    char b[640];
    snprintf(b, sizeof b,
             "\"nlines_in\": %lld, \"nlines_used\": %lld, \"nwide\": %lld, \"nweak\": %lld, \"nblocks\": %lld, "
             "\"line_evals\": %.17g, \"ms_center\": %.6f, \"ms_params\": %.6f, \"ms_accum\": %.6f, "
             "\"ms_total\": %.6f, \"ms_wing_kernels\": %.6f, \"ms_core_kernels\": %.6f, \"core_evals\": %.17g",
             (long long)t.nlines_in, (long long)t.nlines_used, (long long)t.nwide, (long long)t.nweak,
             (long long)t.nblocks, t.line_evals, t.ms_center, t.ms_params, t.ms_accum, t.ms_total,
             t.ms_wing_kernels, t.ms_core_kernels, t.core_evals);
    return b;
}
}  // namespace

// ---- kernels defined in fsg_kernels64.cu / fsg_fast.cu / fsg_mag.cu ------------------------------
void fsg_launch_xline_setup(cudaStream_t, const AtmView &, const LineView &, XCoef *);
void fsg_launch_xline_depth(cudaStream_t, const AtmView &, int64_t, const XCoef *, double *, double *, double *);
void fsg_launch_lineopacity1_pts(cudaStream_t, const AtmView &, const BlockView &, int64_t, const double *,
                                 const int32_t *, const int32_t *, const int32_t *, int64_t, const VoigtTables &,
                                 double *);
void fsg_launch_lineopacity2_pts(cudaStream_t, const AtmView &, const BlockView &, int64_t, const double *,
                                 const int32_t *, const int32_t *, const double *, const double *, const double *,
                                 const VoigtTables &, double *);
void fsg_launch_analytic_window(cudaStream_t, const AtmView &, int64_t, const int32_t *, const double *,
                                const double *, const double *, const double *, double *);
void fsg_launch_mag_lineopacity1_pts(cudaStream_t, const AtmView &, const BlockView &, const ZView &, int64_t,
                                     const double *, const int32_t *, const int32_t *, const int32_t *, int64_t,
                                     const VoigtTables &, double *);
size_t fsg_stokes_pts_work(int64_t, int, int);
void fsg_launch_stokes_prf_pts(cudaStream_t, const AtmView &, const double *, const double *, const double *, int,
                               const double *, const double *, int64_t, const int32_t *, const double *, double *,
                               double *);
void fsg_launch_xline_init(cudaStream_t, int, const double *, const double *, const double *, const float *,
                           const float *, const float *, double, double *);
void fsg_launch_center(cudaStream_t, const AtmView &, const LineView &, const VoigtTables &, int32_t *,
                       int32_t *, int32_t *, unsigned long long *);
void fsg_launch_params_fast(cudaStream_t, const AtmView &, const LineView &, const int64_t *, int64_t, int64_t,
                            int64_t, const int32_t *, const int32_t *, const int32_t *, const VoigtTables &,
                            WingRec *, CoreRec *, LineHdr *);
void fsg_launch_params_fp64(cudaStream_t, const AtmView &, const LineView &, int64_t, int64_t, const int32_t *,
                            double3 *);
void fsg_launch_span(cudaStream_t, int64_t, const int32_t *, const int32_t *, const int32_t *, int *, int *);
void fsg_launch_accum_fp64(cudaStream_t, const AtmView &, const double *, int, int, const int *, const int *,
                           const int32_t *, const int32_t *, const int32_t *, int64_t, const double3 *,
                           const VoigtTables &, double *, double *);
void fsg_launch_wide_fp64(cudaStream_t, const AtmView &, const LineView &, int, const int64_t *, const int32_t *,
                          const int32_t *, const int32_t *, double3 *, const VoigtTables &, int, int, double *,
                          double *);
int fsg_launch_radtran(cudaStream_t, const AtmView &, const double *, const double *, int, const double *,
                       const double *, double *, double *, double *, double *);
void fsg_launch_hvoigt(cudaStream_t, int64_t, const double *, const double *, double *, const VoigtTables &);
void fsg_launch_fvoigt(cudaStream_t, int64_t, const double *, const double *, double *, double *,
                       const VoigtTables &);
void fsg_launch_locprf(cudaStream_t, int, int, const double *, int, const double *, const double *, const double *,
                       double *, double *);
int fsg_launch_accum_fast(cudaStream_t, int, int, int, const double *, const LineHdr *, const WingRec *,
                          const int *, const int *, double *, int *, unsigned, unsigned long long);
int fsg_launch_core_fast(cudaStream_t, int, int, const double *, const LineHdr *, const WingRec *, const CoreRec *,
                         const int *, const int *, const float4 *, double *, unsigned long long *, int *, unsigned,
                         unsigned long long);
int fsg_launch_accum_batch(cudaStream_t, int, int, const WingJob *, const int *, int, int, unsigned *, int *);
int fsg_launch_core_batch(cudaStream_t, int, const CoreJob *, const int *, int, int, const float4 *, unsigned *,
                          int *);
int fsg_class_pix(int);
int fsg_fast_tiles(int);
int fsg_bclass_count(int);
int fsg_launch_bclass_order(cudaStream_t, int64_t, const int32_t *, const int32_t *, const int32_t *, int, int *,
                            int64_t *, int64_t *, int64_t *);
size_t fsg_bspan_scratch(int64_t);
int fsg_launch_btile_span(cudaStream_t, int, int64_t, const LineHdr *, const int64_t *, int, int, int, int, int, int,
                          int *, int *, void *, size_t);
size_t fsg_tile_span_scratch(int64_t);
int fsg_launch_tile_span_tw(cudaStream_t, int, int, int, int64_t, const LineHdr *, int *, int *, void *, size_t);
void fsg_launch_mag_params_fast(cudaStream_t, const AtmView &, const LineView &, const ZView &, const int64_t *, int64_t,
                                int64_t, const int32_t *, const int32_t *, const int32_t *, const VoigtTables &, void *,
                                LineHdr *, int64_t *);
size_t fsg_mag_rec_bytes();
int fsg_launch_mag_fast(cudaStream_t, const AtmView &, const LineHdr *, const void *, const int64_t *, const ZView &,
                        const int *, const int *, const VoigtTables &, double *);
void fsg_launch_conv(cudaStream_t, int, const double *, int, const double *, int, double *, const double *, double);
size_t fsg_adjoint_work(int, int, int64_t, int);
int fsg_launch_adjoint(cudaStream_t, const AtmView &, const LineView &, const VoigtTables &, const double *,
                       const double *, int, const double *, const double *, const RayView &, const int32_t *,
                       const int32_t *, const int32_t *, const double *, double *, double *, double, double *,
                       double *, int, int);
size_t fsg_linstr_work(int64_t, int, int);
void fsg_launch_linstr(cudaStream_t, const AtmView &, const LineView &, const VoigtTables &, const int32_t *, int64_t,
                       int64_t, int, const double *, const double *, const double *, const RayView &, double *, float *);
int fsg_launch_radtran_sph(cudaStream_t, const AtmView &, const double *, const RayView &, const double *, double *,
                           double *, double *, double *);
int fsg_launch_stokes_sph(cudaStream_t, const AtmView &, const double *, const double *, const RayView &,
                          const double *, const double *, double *, double *, double *, int);
int fsg_launch_tile_span(cudaStream_t, int, int, int64_t, const LineHdr *, int *, int *, void *, size_t);
int fsg_select(cudaStream_t, int64_t, const int32_t *, const int32_t *, const int32_t *, int, int *, int64_t *,
               int64_t *, int64_t *);
void fsg_launch_class_hist(cudaStream_t, int64_t, const int32_t *, const int32_t *, const int32_t *,
                           unsigned long long *);
void fsg_launch_mark_wide(cudaStream_t, const AtmView &, int64_t, const double *, int64_t, int32_t *,
                          const int32_t *, const int32_t *, unsigned long long *);

void fsg_launch_gather_lines(cudaStream_t, const LineView &, const int64_t *, int64_t, char *, const int32_t *,
                             const int32_t *, const int32_t *, LineView *, int32_t **, int32_t **, int32_t **);
int fsg_select_wide(cudaStream_t, int64_t, const int32_t *, int *, int64_t *, int64_t *, int64_t *);
void fsg_launch_scatter_flags(cudaStream_t, int64_t, const int64_t *, const int32_t *, int32_t *);
double fsg_count_evals(fsg_ctx *, int64_t, const int32_t *, const int32_t *, const int32_t *, int, int);
static double count_windows(fsg_ctx *, int64_t, const int32_t *, const int32_t *, const int32_t *, int, int,
                            const int32_t *npi = nullptr, const int32_t *nsi = nullptr);
void fsg_launch_range_clip(cudaStream_t, int64_t, const int32_t *, const int32_t *, const int32_t *, int, int,
                           int32_t *, int32_t *, int32_t *);
int fsg_launch_stokes(cudaStream_t, const AtmView &, const double *, const double *, const double *, int,
                      const double *, const double *, const double *, double *, double *, double *, int);
size_t fsg_stokes_work(int, int, int);
int fsg_stokes_chunk(int, int, int, size_t);
void fsg_launch_mag_center(cudaStream_t, const AtmView &, const LineView &, const ZView &, double, const VoigtTables &,
                           int32_t *, int32_t *, int32_t *, unsigned long long *);
void fsg_launch_mag_params(cudaStream_t, const AtmView &, const LineView &, int64_t, const int64_t *, int64_t,
                           const int32_t *, double3 *);
void fsg_launch_mag_accum(cudaStream_t, const AtmView &, const double *, const ZView &, const int64_t *, int, int,
                          const int *, const int *, const int32_t *, const int32_t *, const int32_t *, int64_t,
                          const double3 *, const VoigtTables &, double *, double *);
void fsg_launch_mag_wide(cudaStream_t, const AtmView &, const double *, const ZView &, const int64_t *, int,
                         const int64_t *, const int32_t *, const int32_t *, const int32_t *, const double3 *,
                         const VoigtTables &, double *);

std::string fsg_cuda_msg(cudaError_t e, const char *what) {
    char b[512];
    snprintf(b, sizeof b, "%s: CUDA error %d (%s)", what, (int)e, cudaGetErrorString(e));
    return b;
}

// ---- device buffer that only grows ---------------------------------------------------------------
struct DBuf {
    void *p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes) {
        if (bytes <= cap) return FSG_OK;
        if (p) cudaFree(p);
        p = nullptr; cap = 0;
        if (bytes == 0) return FSG_OK;
        if (cudaMalloc(&p, bytes) != cudaSuccess) { cudaGetLastError(); return FSG_E_NOMEM; }
        cap = bytes;
        return FSG_OK;
    }
    void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
    template <class T> T *as() const { return (T *)p; }
};

struct fsg_ctx {
    fsg_config cfg;
    int device = 0;
    // failure injection (fsg_set_fault): allocation cap [bytes, 0 = none]; extra bytes every staged chunk
    // expects and the bound of the staging waits
    size_t fault_alloc = 0;
    unsigned fault_extra_tx = 0;
    unsigned long long fault_wait_ns = WAIT_NS;
    cudaStream_t stream = nullptr;
    std::string err;
    VoigtTables tab{};
    double h_anode[FSG_NA1], h_aida[FSG_NA1];
    // grid
    int have_grid = 0, wmode = 0, nwl = 0;
    double wstart = 0, wend = 0, dstep = 0, rstep = 0, wfirst = 0, wlast = 0;
    DBuf d_wave;
    // atmosphere
    int have_atm = 0, ntau = 0, nspc = 0;
    DBuf d_xi, d_fpf, d_xamass, d_potion, d_ion, d_rhox, d_tmp;
    int have_cont = 0, motype = 0;
    DBuf d_cont, d_contstd;
    int nhe = 0, spc_he1 = -1;
    DBuf d_hegam, d_heshf;
    // mu
    int nmu = 0;
    DBuf d_xmu, d_wmu;
    std::vector<double> h_xmu;
    // geometry: radius <= 0 plane-parallel; spherical rays (SphereInit) rebuilt when mu, the
    // atmosphere or the geometry change
    double radius = -1.0;
    std::vector<double> h_rhox, h_height, h_muloc;
    std::vector<int> h_ray_n;
    int rays_ok = 0;
    DBuf d_ray_n, d_ray_graz, d_ray_map, d_ray_m, d_ray_geo;
    // accumulators
    DBuf d_lineopac, d_maglineopac;
    // line list staging + per-line outputs
    DBuf l_wl, l_elo, l_gf, l_grad, l_gqst, l_gvdw, l_spc, l_ismol, l_ihe;
    DBuf d_flags, d_ileft, d_iright, d_idx, d_counts, d_offs, d_total, d_hist, d_nkeep;
    // block buffers
    DBuf d_wing, d_core, d_hdr, d_tlo, d_thi, d_p64, d_lstart, d_lstop, d_widx, d_pw, d_evals, d_err, d_ncore, d_span, d_lswork, d_linstr, d_rflags, d_rleft, d_rright, d_gkappa, d_adjwork, d_cbuf, d_ctaps;
    // spectra
    DBuf d_spl, d_spc, d_sfl, d_sfc, d_work, d_a, d_v, d_h, d_l;
    // magnetic
    DBuf z_npi, z_nsi, z_pioff, z_sioff, z_splpi, z_strpi, z_splsi, z_strsi, d_zsc, z_rawpi, z_rawsi, d_zmap, d_geo;
    DBuf d_stkwork;                            // per-thread work arrays of the Stokes solver
    cudaEvent_t ev[8];
    cudaStream_t cstream = nullptr;            // host->device line uploads, overlapped with the central pass
    std::vector<cudaEvent_t> cev;
    int64_t launches = 0;
    std::vector<cudaEvent_t> kev;
};

static int fail(fsg_ctx *c, int code, const char *msg) { if (c) c->err = msg; return code; }
static int cuda_fail(fsg_ctx *c, cudaError_t e, const char *what) {
    if (c) c->err = fsg_cuda_msg(e, what);
    return FSG_E_CUDA;
}
#define CK(call, what) do { cudaError_t _e = (call); if (_e != cudaSuccess) return cuda_fail(ctx, _e, what); } while (0)
#define ALLOC(buf, bytes) do { \
        if (ctx->fault_alloc && (size_t)(bytes) > ctx->fault_alloc && (buf).cap < (size_t)(bytes)) \
            return fail(ctx, FSG_E_NOMEM, "device allocation refused (fault injection): " #buf); \
        if ((buf).ensure(bytes) != FSG_OK) return fail(ctx, FSG_E_NOMEM, "device allocation failed: " #buf); } while (0)

AtmView fsg_view(const fsg_ctx *ctx) {
    AtmView A;
    memset(&A, 0, sizeof A);
    A.ntau = ctx->ntau; A.nspc = ctx->nspc; A.nwl = ctx->nwl; A.wmode = ctx->wmode; A.motype = ctx->motype;
    A.nhe = ctx->nhe; A.spc_he1 = ctx->spc_he1; A.molbrd = ctx->cfg.molbrd;
    A.wfirst = ctx->wfirst; A.wstart = ctx->wstart; A.dstep = ctx->dstep; A.rstep = ctx->rstep;
    double c = FSG_VC * 1e13;
    A.vturb2 = 1e26 / c / c * (ctx->cfg.vmicro * ctx->cfg.vmicro);
    A.epsopac = ctx->cfg.epsopac; A.vwfudge = ctx->cfg.vwfudge; A.vwmol = ctx->cfg.vwmol;
    A.xi = ctx->d_xi.as<double>(); A.fpf = ctx->d_fpf.as<float>(); A.xamass = ctx->d_xamass.as<float>();
    A.potion = ctx->d_potion.as<float>(); A.ion = ctx->d_ion.as<int>(); A.wave = ctx->d_wave.as<double>();
    A.contopac = ctx->d_cont.as<double>(); A.contstd = ctx->d_contstd.as<double>();
    A.hegam = ctx->d_hegam.as<double>(); A.heshf = ctx->d_heshf.as<double>();
    return A;
}

extern "C" {

int fsg_version(void) { return 10000; }

int64_t fsg_kernel_launches(const fsg_ctx *ctx) { return ctx ? ctx->launches : -1; }

void *fsg_cuda_stream(fsg_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

const char *fsg_last_error(const fsg_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int fsg_create(const fsg_config *cfg, fsg_ctx **out) {
    if (!cfg || !out) return FSG_E_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) { cudaGetLastError(); return FSG_E_CUDA; }
    if (cfg->device < 0 || cfg->device >= ndev) return FSG_E_ARG;
    if (cfg->precision != FSG_PREC_MIXED && cfg->precision != FSG_PREC_FP64) return FSG_E_ARG;
    cudaGetLastError();                                 // an earlier caller's error is not this context's
    fsg_ctx *ctx = new fsg_ctx();
    ctx->cfg = *cfg;
    if (ctx->cfg.epsopac <= 0) ctx->cfg.epsopac = 1e-4;
    if (ctx->cfg.limitram_gb <= 0) ctx->cfg.limitram_gb = 16.0;
    ctx->device = cfg->device;
    if (cudaSetDevice(ctx->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError(); delete ctx; return FSG_E_CUDA;
    }
    for (int i = 0; i < 8; i++) cudaEventCreate(&ctx->ev[i]);
    cudaStreamCreateWithFlags(&ctx->cstream, cudaStreamNonBlocking);
    std::string e;
    int rc = fsg_build_tables(&ctx->tab, ctx->stream, &e);
    if (rc == FSG_OK) {
        if (cudaMemcpyAsync(ctx->h_anode, ctx->tab.anode, sizeof ctx->h_anode, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
            cudaMemcpyAsync(ctx->h_aida, ctx->tab.aida, sizeof ctx->h_aida, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = FSG_E_CUDA;
    }
    if (rc != FSG_OK) { fsg_destroy(ctx); return rc; }
    *out = ctx;
    return FSG_OK;
}

void fsg_destroy(fsg_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    fsg_free_tables(&ctx->tab);
    DBuf *bufs[] = { &ctx->d_wave, &ctx->d_xi, &ctx->d_fpf, &ctx->d_xamass, &ctx->d_potion, &ctx->d_ion, &ctx->d_rhox,
                     &ctx->d_tmp, &ctx->d_cont, &ctx->d_contstd, &ctx->d_hegam, &ctx->d_heshf, &ctx->d_xmu,
                     &ctx->d_wmu, &ctx->d_lineopac, &ctx->d_maglineopac, &ctx->l_wl, &ctx->l_elo, &ctx->l_gf,
                     &ctx->l_grad, &ctx->l_gqst, &ctx->l_gvdw, &ctx->l_spc, &ctx->l_ismol, &ctx->l_ihe,
                     &ctx->d_flags, &ctx->d_ileft, &ctx->d_iright, &ctx->d_idx, &ctx->d_counts, &ctx->d_offs,
                     &ctx->d_total, &ctx->d_hist, &ctx->d_nkeep, &ctx->d_wing, &ctx->d_core, &ctx->d_hdr,
                     &ctx->d_tlo, &ctx->d_thi, &ctx->d_err, &ctx->d_ncore, &ctx->d_span, &ctx->d_lswork, &ctx->d_linstr, &ctx->d_rflags, &ctx->d_rleft, &ctx->d_rright, &ctx->d_gkappa, &ctx->d_adjwork, &ctx->d_cbuf, &ctx->d_ctaps, &ctx->d_p64, &ctx->d_lstart, &ctx->d_lstop, &ctx->d_widx,
                     &ctx->d_pw, &ctx->d_evals, &ctx->d_spl, &ctx->d_spc, &ctx->d_sfl, &ctx->d_sfc,
                     &ctx->d_work, &ctx->d_a, &ctx->d_v, &ctx->d_h, &ctx->d_l, &ctx->z_npi, &ctx->z_nsi,
                     &ctx->z_pioff, &ctx->z_sioff, &ctx->z_splpi, &ctx->z_strpi, &ctx->z_splsi, &ctx->z_strsi,
                     &ctx->d_zsc, &ctx->z_rawpi, &ctx->z_rawsi, &ctx->d_zmap, &ctx->d_geo,
                     &ctx->d_ray_n, &ctx->d_ray_graz, &ctx->d_ray_map, &ctx->d_ray_m, &ctx->d_ray_geo,
                     &ctx->d_stkwork };
    for (DBuf *b : bufs) b->release();
    for (int i = 0; i < 8; i++) if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
    for (cudaEvent_t e : ctx->cev) cudaEventDestroy(e);
    if (ctx->cstream) { cudaStreamSynchronize(ctx->cstream); cudaStreamDestroy(ctx->cstream); }
    for (cudaEvent_t e : ctx->kev) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

// ---- grid (synth.f90:56-74) ---------------------------------------------------------------------
int fsg_make_grid(int wmode, double wstart, double wend, double dstep, double *wave, int *nwl) {
    if (!nwl || dstep <= 0 || wend <= wstart || (wmode != 0 && wmode != 1)) return FSG_E_ARG;
    const double EpsWl = 1e-12;
    int n;
    if (wmode == 0) {
        n = (int)floor((wend - wstart) / dstep + EpsWl) + 1;
        if (n < 2) return FSG_E_ARG;
        if (wave) for (int i = 1; i <= n; i++) wave[i - 1] = (double)(i - 1) * dstep;
    } else {
        double rstep = dstep / FSG_VC;
        n = (int)floor(log(wend / wstart) / rstep + EpsWl) + 1;
        if (n < 2) return FSG_E_ARG;
        if (wave) for (int i = 1; i <= n; i++) wave[i - 1] = wstart * exp((double)(i - 1) * rstep) - wstart;
    }
    *nwl = n;
    return FSG_OK;
}

int fsg_set_grid(fsg_ctx *ctx, int wmode, double wstart, double wend, double dstep, int nwl, const double *wave) {
    if (!ctx || !wave || nwl < 2 || (wmode != 0 && wmode != 1) || dstep <= 0) return fail(ctx, FSG_E_ARG, "fsg_set_grid: bad arguments");
    cudaSetDevice(ctx->device);
    ctx->wmode = wmode; ctx->wstart = wstart; ctx->wend = wend; ctx->dstep = dstep; ctx->nwl = nwl;
    ctx->rstep = dstep / FSG_VC; ctx->wfirst = wstart; ctx->wlast = wstart + wave[nwl - 1];
    ALLOC(ctx->d_wave, sizeof(double) * nwl);
    CK(cudaMemcpyAsync(ctx->d_wave.p, wave, sizeof(double) * nwl, cudaMemcpyHostToDevice, ctx->stream), "grid upload");
    CK(cudaStreamSynchronize(ctx->stream), "grid upload");
    ctx->have_grid = 1; ctx->have_cont = 0;
    return FSG_OK;
}

int fsg_set_atmosphere(fsg_ctx *ctx, int ntau, const double *rhox, const double *T, const double *xne,
                       const double *xna, const double *rho, int nspc, const float *fractionpf, const float *xamass,
                       const float *potion, const int32_t *ion, const float *frac_h1, const float *frac_he1,
                       const float *frac_h2) {
    (void)xna;
    if (!ctx || ntau < 3 || ntau > 128 || nspc < 1 || !rhox || !T || !xne || !rho || !fractionpf || !xamass ||
        !potion || !ion || !frac_h1 || !frac_he1)
        return fail(ctx, FSG_E_ARG, "fsg_set_atmosphere: bad arguments (3 <= ntau <= 128, nspc >= 1)");
    cudaSetDevice(ctx->device);
    ctx->ntau = ntau; ctx->nspc = nspc;
    ALLOC(ctx->d_xi, sizeof(double) * XI_NROWS * ntau);
    ALLOC(ctx->d_fpf, sizeof(float) * (size_t)nspc * ntau);
    ALLOC(ctx->d_xamass, sizeof(float) * nspc);
    ALLOC(ctx->d_potion, sizeof(float) * nspc);
    ALLOC(ctx->d_ion, sizeof(int) * nspc);
    ALLOC(ctx->d_rhox, sizeof(double) * ntau);
    ALLOC(ctx->d_tmp, sizeof(double) * 3 * ntau + sizeof(float) * 3 * ntau);
    // FractionPF arrives as [ntau][nspc] (species fastest); stored species-major [nspc][ntau]
    std::vector<float> fpf((size_t)nspc * ntau);
    for (int t = 0; t < ntau; t++) for (int s = 0; s < nspc; s++) fpf[(size_t)s * ntau + t] = fractionpf[(size_t)t * nspc + s];
    std::vector<float> h2(ntau, 0.0f);
    if (frac_h2) for (int t = 0; t < ntau; t++) h2[t] = frac_h2[t];
    double *dT = ctx->d_tmp.as<double>(), *dxne = dT + ntau, *drho = dxne + ntau;
    float *dh1 = (float *)(drho + ntau), *dhe1 = dh1 + ntau, *dh2 = dhe1 + ntau;
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(ctx->d_fpf.p, fpf.data(), sizeof(float) * fpf.size(), cudaMemcpyHostToDevice, s), "atm upload");
    CK(cudaMemcpyAsync(ctx->d_xamass.p, xamass, sizeof(float) * nspc, cudaMemcpyHostToDevice, s), "atm upload");
    CK(cudaMemcpyAsync(ctx->d_potion.p, potion, sizeof(float) * nspc, cudaMemcpyHostToDevice, s), "atm upload");
    CK(cudaMemcpyAsync(ctx->d_ion.p, ion, sizeof(int) * nspc, cudaMemcpyHostToDevice, s), "atm upload");
    CK(cudaMemcpyAsync(ctx->d_rhox.p, rhox, sizeof(double) * ntau, cudaMemcpyHostToDevice, s), "atm upload");
    CK(cudaMemcpyAsync(dT, T, sizeof(double) * ntau, cudaMemcpyHostToDevice, s), "atm upload");
    CK(cudaMemcpyAsync(dxne, xne, sizeof(double) * ntau, cudaMemcpyHostToDevice, s), "atm upload");
    CK(cudaMemcpyAsync(drho, rho, sizeof(double) * ntau, cudaMemcpyHostToDevice, s), "atm upload");
    CK(cudaMemcpyAsync(dh1, frac_h1, sizeof(float) * ntau, cudaMemcpyHostToDevice, s), "atm upload");
    CK(cudaMemcpyAsync(dhe1, frac_he1, sizeof(float) * ntau, cudaMemcpyHostToDevice, s), "atm upload");
    CK(cudaMemcpyAsync(dh2, h2.data(), sizeof(float) * ntau, cudaMemcpyHostToDevice, s), "atm upload");
    fsg_launch_xline_init(s, ntau, dT, dxne, drho, dh1, dhe1, dh2, ctx->cfg.h2brd, ctx->d_xi.as<double>());
    CK(cudaGetLastError(), "k_xline_init");
    CK(cudaStreamSynchronize(s), "atm upload");
    ctx->have_atm = 1; ctx->have_cont = 0;
    // a new model is plane-parallel until fsg_set_geometry says otherwise (ReadModel, ioutils.f90:1622)
    ctx->h_rhox.assign(rhox, rhox + ntau);
    ctx->radius = -1.0; ctx->h_height.clear(); ctx->rays_ok = 0;
    return FSG_OK;
}

int fsg_set_geometry(fsg_ctx *ctx, double radius, const double *height) {
    if (!ctx) return FSG_E_ARG;
    if (!ctx->have_atm) return fail(ctx, FSG_E_STATE, "fsg_set_geometry: set the atmosphere first");
    ctx->rays_ok = 0;
    if (radius <= 0.0) { ctx->radius = -1.0; ctx->h_height.clear(); return FSG_OK; }
    const int nt = ctx->ntau;
    if (!height) return fail(ctx, FSG_E_ARG, "fsg_set_geometry: a spherical model needs the layer heights");
    if (radius < 1e9 || radius > 1e15) return fail(ctx, FSG_E_ARG, "fsg_set_geometry: implausible model radius");
    for (int t = 1; t < nt; t++)
        if (!(height[t] < height[t - 1]))
            return fail(ctx, FSG_E_ARG, "fsg_set_geometry: heights of a spherical model do not decrease inward");
    if (!(radius + height[nt - 1] > 0.0)) return fail(ctx, FSG_E_ARG, "fsg_set_geometry: negative layer radius");
    ctx->radius = radius;
    ctx->h_height.assign(height, height + nt);
    return FSG_OK;
}

int fsg_set_contopac(fsg_ctx *ctx, const double *contopac, const double *contopac_std, int motype) {
    if (!ctx) return FSG_E_ARG;
    if (!ctx->have_grid || !ctx->have_atm) return fail(ctx, FSG_E_STATE, "fsg_set_contopac: set grid and atmosphere first");
    if (!contopac || (motype == 1 && !contopac_std) || (motype != 0 && motype != 1))
        return fail(ctx, FSG_E_ARG, "fsg_set_contopac: bad arguments");
    cudaSetDevice(ctx->device);
    size_t nb = sizeof(double) * (size_t)ctx->nwl * ctx->ntau;
    ALLOC(ctx->d_cont, nb);
    CK(cudaMemcpyAsync(ctx->d_cont.p, contopac, nb, cudaMemcpyHostToDevice, ctx->stream), "contopac upload");
    ctx->motype = motype;
    if (motype == 1) {
        ALLOC(ctx->d_contstd, sizeof(double) * ctx->ntau);
        CK(cudaMemcpyAsync(ctx->d_contstd.p, contopac_std, sizeof(double) * ctx->ntau, cudaMemcpyHostToDevice, ctx->stream), "contstd upload");
    }
    CK(cudaStreamSynchronize(ctx->stream), "contopac upload");
    ctx->have_cont = 1;
    return FSG_OK;
}

int fsg_set_contopac_dev(fsg_ctx *ctx, const double *d_contopac) {
    if (!ctx || !d_contopac) return FSG_E_ARG;
    if (!ctx->have_grid || !ctx->have_atm) return fail(ctx, FSG_E_STATE, "fsg_set_contopac_dev: set grid and atmosphere first");
    cudaSetDevice(ctx->device);
    size_t nb = sizeof(double) * (size_t)ctx->nwl * ctx->ntau;
    ALLOC(ctx->d_cont, nb);
    CK(cudaMemcpyAsync(ctx->d_cont.p, d_contopac, nb, cudaMemcpyDeviceToDevice, ctx->stream), "contopac copy");
    CK(cudaStreamSynchronize(ctx->stream), "contopac copy");
    ctx->motype = 0; ctx->have_cont = 1;
    return FSG_OK;
}

int fsg_set_hestark(fsg_ctx *ctx, int nhe, const double *hegam, const double *heshf, int spc_he1) {
    if (!ctx || nhe < 0 || nhe > 255 || (nhe > 0 && (!hegam || !heshf)) || !ctx->have_atm)
        return fail(ctx, FSG_E_ARG, "fsg_set_hestark: bad arguments");
    cudaSetDevice(ctx->device);
    ctx->nhe = nhe; ctx->spc_he1 = spc_he1;
    if (nhe > 0) {
        size_t nb = sizeof(double) * (size_t)nhe * ctx->ntau;
        ALLOC(ctx->d_hegam, nb); ALLOC(ctx->d_heshf, nb);
        CK(cudaMemcpyAsync(ctx->d_hegam.p, hegam, nb, cudaMemcpyHostToDevice, ctx->stream), "hestark upload");
        CK(cudaMemcpyAsync(ctx->d_heshf.p, heshf, nb, cudaMemcpyHostToDevice, ctx->stream), "hestark upload");
        CK(cudaStreamSynchronize(ctx->stream), "hestark upload");
    }
    return FSG_OK;
}

int fsg_set_mu(fsg_ctx *ctx, int nmu, const double *xmu, const double *wmu) {
    if (!ctx || nmu < 1 || nmu > 16 || !xmu || !wmu) return fail(ctx, FSG_E_ARG, "fsg_set_mu: 1 <= nmu <= 16");
    for (int i = 0; i < nmu; i++) if (!(xmu[i] > 0.0 && xmu[i] <= 1.0)) return fail(ctx, FSG_E_ARG, "fsg_set_mu: mu outside (0, 1]");
    cudaSetDevice(ctx->device);
    ALLOC(ctx->d_xmu, sizeof(double) * nmu); ALLOC(ctx->d_wmu, sizeof(double) * nmu);
    CK(cudaMemcpyAsync(ctx->d_xmu.p, xmu, sizeof(double) * nmu, cudaMemcpyHostToDevice, ctx->stream), "mu upload");
    CK(cudaMemcpyAsync(ctx->d_wmu.p, wmu, sizeof(double) * nmu, cudaMemcpyHostToDevice, ctx->stream), "mu upload");
    CK(cudaStreamSynchronize(ctx->stream), "mu upload");
    ctx->nmu = nmu;
    ctx->h_xmu.assign(xmu, xmu + nmu);
    ctx->rays_ok = 0;
    return FSG_OK;
}

// SphereInit (solver.f90:45-120) on the host, once per model and angle set (set-up, as in the
// reference's Init, synth.f90:306): for ray im with impact parameter p = r_top sqrt(1 - mu^2), the
// column mass along the ray grows by the radial step times (r_k + r_k-1) / (z_k + z_k-1), z the
// distance sqrt(r^2 - p^2) in the factored form; a ray with p above the bottom radius turns inside the
// shell below its deepest layer n (the chord times dm/dr crosses it) and comes back through n..1 with
// mirrored steps and the local cosine negated.  Uploads RayView arrays [nmu][2 ntau]; R->nmu = 0 for a
// plane-parallel model.
static int rays_prepare(fsg_ctx *ctx, RayView *R) {
    memset(R, 0, sizeof *R);
    if (ctx->radius <= 0.0) return FSG_OK;
    const int nt = ctx->ntau, nmu = ctx->nmu, M = 2 * nt;
    R->nmu = nmu; R->stride = M;
    if (!ctx->rays_ok) {
        std::vector<double> rk(nt), rm((size_t)nmu * M, 0.0), ml((size_t)nmu * M, 0.0);
        std::vector<int> n(nmu), gz(nmu), mp((size_t)nmu * M, 0);
        for (int k = 0; k < nt; k++) rk[k] = ctx->radius + ctx->h_height[k];
        const double *rhox = ctx->h_rhox.data();
        for (int im = 0; im < nmu; im++) {
            const double mu = ctx->h_xmu[im];
            double *m = &rm[(size_t)im * M], *c = &ml[(size_t)im * M];
            int *q = &mp[(size_t)im * M];
            if (!(mu > 0.0)) return fail(ctx, FSG_E_ARG, "SphereInit: mu = 0 rays are unsupported for spherical models");
            const double P = rk[0] * sqrt((1.0 - mu) * (1.0 + mu));
            const int g = P > rk[nt - 1];
            int deep = nt;
            if (g) {
                int kt = 2;
                while (kt <= nt && !(P >= rk[kt - 1])) kt++;
                deep = kt - 1;
                if (deep < 2) return fail(ctx, FSG_E_ARG, "SphereInit: grazing ray tangent in the top model layer");
            }
            m[0] = rhox[0] / mu;
            double z1 = sqrt((rk[0] - P) * (rk[0] + P));
            c[0] = z1 / rk[0];
            for (int k = 1; k < deep; k++) {
                double z = sqrt((rk[k] - P) * (rk[k] + P));
                m[k] = m[k - 1] + (rhox[k] - rhox[k - 1]) * (rk[k] + rk[k - 1]) / (z + z1);
                c[k] = z / rk[k];
                q[k] = k;
                z1 = z;
            }
            gz[im] = g;
            n[im] = nt;
            if (!g) continue;
            double chord = 2.0 * sqrt((rk[deep - 1] - P) * (rk[deep - 1] + P));
            m[deep] = m[deep - 1] + chord * (rhox[deep] - rhox[deep - 1]) / (rk[deep - 1] - rk[deep]);
            q[deep] = deep - 1;
            c[deep] = -c[deep - 1];
            for (int k = deep + 1; k < 2 * deep; k++) {          // the far half mirrors the near one
                m[k] = m[k - 1] + (m[2 * deep - k] - m[2 * deep - k - 1]);
                q[k] = 2 * deep - 1 - k;
                c[k] = -c[2 * deep - 1 - k];
            }
            n[im] = 2 * deep;
        }
        ALLOC(ctx->d_ray_n, sizeof(int) * nmu); ALLOC(ctx->d_ray_graz, sizeof(int) * nmu);
        ALLOC(ctx->d_ray_map, sizeof(int) * mp.size()); ALLOC(ctx->d_ray_m, sizeof(double) * rm.size());
        cudaStream_t s = ctx->stream;
        CK(cudaMemcpyAsync(ctx->d_ray_n.p, n.data(), sizeof(int) * nmu, cudaMemcpyHostToDevice, s), "rays");
        CK(cudaMemcpyAsync(ctx->d_ray_graz.p, gz.data(), sizeof(int) * nmu, cudaMemcpyHostToDevice, s), "rays");
        CK(cudaMemcpyAsync(ctx->d_ray_map.p, mp.data(), sizeof(int) * mp.size(), cudaMemcpyHostToDevice, s), "rays");
        CK(cudaMemcpyAsync(ctx->d_ray_m.p, rm.data(), sizeof(double) * rm.size(), cudaMemcpyHostToDevice, s), "rays");
        CK(cudaStreamSynchronize(s), "rays");
        ctx->h_muloc.swap(ml); ctx->h_ray_n.swap(n);
        ctx->rays_ok = 1;
    }
    R->n = ctx->d_ray_n.as<int>(); R->graz = ctx->d_ray_graz.as<int>();
    R->map = ctx->d_ray_map.as<int>(); R->m = ctx->d_ray_m.as<double>();
    return FSG_OK;
}

// ---- line opacity accumulator -----------------------------------------------------------------------
static int ensure_lineopac(fsg_ctx *ctx) {
    size_t nb = sizeof(double) * (size_t)ctx->nwl * ctx->ntau;
    if (ctx->d_lineopac.cap < nb) {
        ALLOC(ctx->d_lineopac, nb);
        CK(cudaMemsetAsync(ctx->d_lineopac.p, 0, nb, ctx->stream), "lineopac reset");
    }
    return FSG_OK;
}

int fsg_lineop_reset(fsg_ctx *ctx) {
    if (!ctx) return FSG_E_ARG;
    if (!ctx->have_grid || !ctx->have_atm) return fail(ctx, FSG_E_STATE, "fsg_lineop_reset: set grid and atmosphere first");
    cudaSetDevice(ctx->device);
    int rc = ensure_lineopac(ctx); if (rc) return rc;
    CK(cudaMemsetAsync(ctx->d_lineopac.p, 0, sizeof(double) * (size_t)ctx->nwl * ctx->ntau, ctx->stream), "lineopac reset");
    CK(cudaStreamSynchronize(ctx->stream), "lineopac reset");
    return FSG_OK;
}

int fsg_lineop_get(fsg_ctx *ctx, double *lineopac) {
    if (!ctx || !lineopac) return FSG_E_ARG;
    if (!ctx->d_lineopac.p) return fail(ctx, FSG_E_STATE, "fsg_lineop_get: no line opacity");
    cudaSetDevice(ctx->device);
    CK(cudaMemcpyAsync(lineopac, ctx->d_lineopac.p, sizeof(double) * (size_t)ctx->nwl * ctx->ntau, cudaMemcpyDeviceToHost, ctx->stream), "lineopac get");
    CK(cudaStreamSynchronize(ctx->stream), "lineopac get");
    return FSG_OK;
}

int fsg_lineop_set(fsg_ctx *ctx, const double *lineopac) {
    if (!ctx || !lineopac) return FSG_E_ARG;
    if (!ctx->have_grid || !ctx->have_atm) return fail(ctx, FSG_E_STATE, "fsg_lineop_set: set grid and atmosphere first");
    cudaSetDevice(ctx->device);
    int rc = ensure_lineopac(ctx); if (rc) return rc;
    CK(cudaMemcpyAsync(ctx->d_lineopac.p, lineopac, sizeof(double) * (size_t)ctx->nwl * ctx->ntau, cudaMemcpyHostToDevice, ctx->stream), "lineopac set");
    CK(cudaStreamSynchronize(ctx->stream), "lineopac set");
    return FSG_OK;
}

const double *fsg_lineop_device_ptr(fsg_ctx *ctx) { return ctx ? ctx->d_lineopac.as<double>() : nullptr; }

// ---- LineopCalc -----------------------------------------------------------------------------------
static LineView make_view(const fsg_lines *L) {
    LineView v;
    v.n = L->n; v.kind = L->kind; v.wl = L->wl; v.elo = L->elo; v.gf = L->gf; v.grad = L->grad;
    v.gqst = L->gqst; v.gvdw = L->gvdw; v.spc = L->spc; v.ismol = L->ismol; v.ihe = L->ihe;
    return v;
}

// device buffers for a host list (no copy: central_pass_streamed uploads)
static int device_lines(fsg_ctx *ctx, const fsg_lines *L, fsg_lines *D) {
    int64_t n = L->n;
    size_t n8 = sizeof(double) * n, n4 = sizeof(float) * n;
    ALLOC(ctx->l_wl, n8); ALLOC(ctx->l_elo, n4); ALLOC(ctx->l_gf, n4); ALLOC(ctx->l_grad, n4);
    ALLOC(ctx->l_gqst, n4); ALLOC(ctx->l_gvdw, n4); ALLOC(ctx->l_spc, n4);
    *D = *L;
    D->wl = ctx->l_wl.as<double>(); D->elo = ctx->l_elo.as<float>(); D->gf = ctx->l_gf.as<float>();
    D->grad = ctx->l_grad.as<float>(); D->gqst = ctx->l_gqst.as<float>(); D->gvdw = ctx->l_gvdw.as<float>();
    D->spc = ctx->l_spc.as<int32_t>();
    D->ismol = nullptr; D->ihe = nullptr;
    if (L->ismol) { ALLOC(ctx->l_ismol, n4); D->ismol = ctx->l_ismol.as<int32_t>(); }
    if (L->ihe) { ALLOC(ctx->l_ihe, n4); D->ihe = ctx->l_ihe.as<int32_t>(); }
    return FSG_OK;
}

static int upload_lines(fsg_ctx *ctx, const fsg_lines *L, fsg_lines *D) {
    int64_t n = L->n;
    size_t n8 = sizeof(double) * n, n4 = sizeof(float) * n;
    ALLOC(ctx->l_wl, n8); ALLOC(ctx->l_elo, n4); ALLOC(ctx->l_gf, n4); ALLOC(ctx->l_grad, n4);
    ALLOC(ctx->l_gqst, n4); ALLOC(ctx->l_gvdw, n4); ALLOC(ctx->l_spc, n4);
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(ctx->l_wl.p, L->wl, n8, cudaMemcpyHostToDevice, s), "line upload");
    CK(cudaMemcpyAsync(ctx->l_elo.p, L->elo, n4, cudaMemcpyHostToDevice, s), "line upload");
    CK(cudaMemcpyAsync(ctx->l_gf.p, L->gf, n4, cudaMemcpyHostToDevice, s), "line upload");
    CK(cudaMemcpyAsync(ctx->l_grad.p, L->grad, n4, cudaMemcpyHostToDevice, s), "line upload");
    CK(cudaMemcpyAsync(ctx->l_gqst.p, L->gqst, n4, cudaMemcpyHostToDevice, s), "line upload");
    CK(cudaMemcpyAsync(ctx->l_gvdw.p, L->gvdw, n4, cudaMemcpyHostToDevice, s), "line upload");
    CK(cudaMemcpyAsync(ctx->l_spc.p, L->spc, n4, cudaMemcpyHostToDevice, s), "line upload");
    *D = *L;
    D->wl = ctx->l_wl.as<double>(); D->elo = ctx->l_elo.as<float>(); D->gf = ctx->l_gf.as<float>();
    D->grad = ctx->l_grad.as<float>(); D->gqst = ctx->l_gqst.as<float>(); D->gvdw = ctx->l_gvdw.as<float>();
    D->spc = ctx->l_spc.as<int32_t>();
    D->ismol = nullptr; D->ihe = nullptr;
    if (L->ismol) {
        ALLOC(ctx->l_ismol, n4);
        CK(cudaMemcpyAsync(ctx->l_ismol.p, L->ismol, n4, cudaMemcpyHostToDevice, s), "line upload");
        D->ismol = ctx->l_ismol.as<int32_t>();
    }
    if (L->ihe) {
        ALLOC(ctx->l_ihe, n4);
        CK(cudaMemcpyAsync(ctx->l_ihe.p, L->ihe, n4, cudaMemcpyHostToDevice, s), "line upload");
        D->ihe = ctx->l_ihe.as<int32_t>();
    }
    return FSG_OK;
}

static int check_lines(fsg_ctx *ctx, const fsg_lines *L, bool need_cont = true) {
    if (!ctx) return FSG_E_ARG;
    if (!ctx->have_grid || !ctx->have_atm) return fail(ctx, FSG_E_STATE, "lineop: set grid and atmosphere first");
    if (need_cont && !ctx->have_cont) return fail(ctx, FSG_E_STATE, "lineop: set continuum opacity first");
    if (!L || L->n < 0 || (L->n > 0 && (!L->wl || !L->elo || !L->gf || !L->grad || !L->gqst || !L->gvdw || !L->spc)))
        return fail(ctx, FSG_E_ARG, "lineop: bad line list");
    if (L->kind < 0 || L->kind > 2) return fail(ctx, FSG_E_ARG, "lineop: kind must be 0, 1 or 2");
    if (L->n > 2000000000LL) return fail(ctx, FSG_E_ARG, "lineop: more than 2e9 lines");
    return FSG_OK;
}

static int64_t block_capacity(const fsg_ctx *ctx, size_t per_line) {
    double cap = ctx->cfg.limitram_gb * 1e9 / (double)per_line;
    int64_t c = (int64_t)cap;
    if (c < 8) c = 8;
    return c;
}

// central pass common to both precisions; leaves flags/ileft/iright on the device
static int central_pass(fsg_ctx *ctx, const LineView &LV, int64_t *nkeep) {
    int64_t n = LV.n;
    ALLOC(ctx->d_flags, sizeof(int32_t) * std::max<int64_t>(n, 1));
    ALLOC(ctx->d_ileft, sizeof(int32_t) * std::max<int64_t>(n, 1));
    ALLOC(ctx->d_iright, sizeof(int32_t) * std::max<int64_t>(n, 1));
    ALLOC(ctx->d_nkeep, sizeof(unsigned long long));
    CK(cudaMemsetAsync(ctx->d_nkeep.p, 0, sizeof(unsigned long long), ctx->stream), "center");
    AtmView A = fsg_view(ctx);
    fsg_launch_center(ctx->stream, A, LV, ctx->tab, ctx->d_flags.as<int32_t>(), ctx->d_ileft.as<int32_t>(),
                      ctx->d_iright.as<int32_t>(), ctx->d_nkeep.as<unsigned long long>());
    ctx->launches += 1;
    CK(cudaGetLastError(), "k_center");
    unsigned long long nk = 0;
    CK(cudaMemcpyAsync(&nk, ctx->d_nkeep.p, sizeof nk, cudaMemcpyDeviceToHost, ctx->stream), "center");
    CK(cudaStreamSynchronize(ctx->stream), "center");
    *nkeep = (int64_t)nk;
    return FSG_OK;
}

// mixed-precision accumulation: classes by window width, blocks within a class
// fl/il/ir: LinFlag, Ileft, Iright of the list (device); [i0, i1]: 1-based wavelength range to fill
// (1..nwl for the whole grid).  Lines are classed by their full windows and evaluated over the part
// of the window inside the range, so each wavelength of the range sums the same lines in the same
// order as in a whole-grid run.
static int accumulate_fast(fsg_ctx *ctx, const LineView &LV, fsg_stats *st, const int32_t *fl, const int32_t *il,
                           const int32_t *ir, int i0, int i1) {
    int64_t n = LV.n;
    const int nt = ctx->ntau;
    AtmView A = fsg_view(ctx);
    cudaStream_t s = ctx->stream;
    const int32_t *sf = fl, *wl_ = il, *wr_ = ir;       // selection flags, evaluated window bounds
    if (i0 > 1 || i1 < ctx->nwl) {
        ALLOC(ctx->d_rflags, sizeof(int32_t) * std::max<int64_t>(n, 1));
        ALLOC(ctx->d_rleft, sizeof(int32_t) * std::max<int64_t>(n, 1));
        ALLOC(ctx->d_rright, sizeof(int32_t) * std::max<int64_t>(n, 1));
        fsg_launch_range_clip(s, n, fl, il, ir, i0, i1, ctx->d_rflags.as<int32_t>(), ctx->d_rleft.as<int32_t>(),
                              ctx->d_rright.as<int32_t>());
        ctx->launches += 1;
        sf = ctx->d_rflags.as<int32_t>(); wl_ = ctx->d_rleft.as<int32_t>(); wr_ = ctx->d_rright.as<int32_t>();
    }
    ALLOC(ctx->d_hist, sizeof(unsigned long long) * 32);
    CK(cudaMemsetAsync(ctx->d_hist.p, 0, sizeof(unsigned long long) * 32, s), "hist");
    fsg_launch_class_hist(s, n, sf, il, ir, ctx->d_hist.as<unsigned long long>());
    ctx->launches += 1;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> kt, kc;   // wing pass, core pass
    size_t kev_used = 0;
    auto kevent = [&]() -> cudaEvent_t {
        if (kev_used == ctx->kev.size()) { cudaEvent_t e; cudaEventCreate(&e); ctx->kev.push_back(e); }
        return ctx->kev[kev_used++];
    };
    unsigned long long hist[32];
    CK(cudaMemcpyAsync(hist, ctx->d_hist.p, sizeof hist, cudaMemcpyDeviceToHost, s), "hist");
    CK(cudaStreamSynchronize(s), "hist");
    if (st) {                                          // lines evaluated (those meeting the range)
        int64_t nsel = 0;
        for (int c = 0; c < 32; c++) nsel += (int64_t)hist[c];
        st->nlines_used = nsel;
    }
    int64_t nblkscan = (n + 1023) / 1024;
    ALLOC(ctx->d_counts, sizeof(int) * std::max<int64_t>(nblkscan, 1));
    ALLOC(ctx->d_offs, sizeof(int64_t) * std::max<int64_t>(nblkscan, 1));
    ALLOC(ctx->d_total, sizeof(int64_t));
    ALLOC(ctx->d_idx, sizeof(int64_t) * std::max<int64_t>(n, 1));
    int ntiles = fsg_fast_tiles(ctx->nwl);
    ALLOC(ctx->d_tlo, sizeof(int) * ntiles); ALLOC(ctx->d_thi, sizeof(int) * ntiles);
    ALLOC(ctx->d_err, sizeof(int));
    CK(cudaMemsetAsync(ctx->d_err.p, 0, sizeof(int), s), "err reset");
    ALLOC(ctx->d_ncore, sizeof(unsigned long long));
    CK(cudaMemsetAsync(ctx->d_ncore.p, 0, sizeof(unsigned long long), s), "core count reset");
    size_t per_line = (size_t)nt * (sizeof(WingRec) + sizeof(CoreRec)) + sizeof(LineHdr);
    int64_t cap = block_capacity(ctx, per_line);
    int64_t nblocks = 0;
    for (int c = 0; c < 32; c++) {
        if (!hist[c]) continue;
        int rc = fsg_select(s, n, sf, il, ir, c,
                            ctx->d_counts.as<int>(), ctx->d_offs.as<int64_t>(), ctx->d_idx.as<int64_t>(),
                            ctx->d_total.as<int64_t>());
        if (rc) return cuda_fail(ctx, cudaGetLastError(), "select");
        ctx->launches += 3;
        int64_t nc = (int64_t)hist[c];
        // blocks of at most cap lines (LIMITRAM); block b takes every nblk-th line of the class from
        // its b-th, so each block is sorted by wavelength and spans the whole grid: every tile of a
        // launch has work, however small the blocks
        const int64_t nblk = (nc + cap - 1) / cap;
        const int64_t bcap = (nc + nblk - 1) / nblk;
        ALLOC(ctx->d_wing, sizeof(WingRec) * (size_t)bcap * nt);
        ALLOC(ctx->d_core, sizeof(CoreRec) * (size_t)bcap * nt);
        ALLOC(ctx->d_hdr, sizeof(LineHdr) * (size_t)bcap);
        ALLOC(ctx->d_span, fsg_tile_span_scratch(bcap));
        for (int64_t b = 0; b < nblk; b++) {
            const int64_t nb = (nc - b + nblk - 1) / nblk;
            fsg_launch_params_fast(s, A, LV, ctx->d_idx.as<int64_t>(), b, nblk, nb, fl, wl_, wr_, ctx->tab,
                                   ctx->d_wing.as<WingRec>(), ctx->d_core.as<CoreRec>(), ctx->d_hdr.as<LineHdr>());
            if (fsg_launch_tile_span(s, c, ctx->nwl, nb, ctx->d_hdr.as<LineHdr>(), ctx->d_tlo.as<int>(),
                                     ctx->d_thi.as<int>(), ctx->d_span.p, ctx->d_span.cap))
                return cuda_fail(ctx, cudaGetLastError(), "tile span");
            cudaEvent_t ea = kevent(), em = kevent(), eb = kevent();
            cudaEventRecord(ea, s);
            int rc2 = fsg_launch_accum_fast(s, c, nt, ctx->nwl, ctx->d_wave.as<double>(), ctx->d_hdr.as<LineHdr>(),
                                            ctx->d_wing.as<WingRec>(), ctx->d_tlo.as<int>(), ctx->d_thi.as<int>(),
                                            ctx->d_lineopac.as<double>(), ctx->d_err.as<int>(), ctx->fault_extra_tx,
                                            ctx->fault_wait_ns);
            if (rc2) return cuda_fail(ctx, cudaGetLastError(), "k_accum_fast");
            cudaEventRecord(em, s);
            // core ranges of the same lines, 32-wavelength tiles
            if (fsg_launch_tile_span(s, -1, ctx->nwl, nb, ctx->d_hdr.as<LineHdr>(), ctx->d_tlo.as<int>(),
                                     ctx->d_thi.as<int>(), ctx->d_span.p, ctx->d_span.cap))
                return cuda_fail(ctx, cudaGetLastError(), "core tile span");
            rc2 = fsg_launch_core_fast(s, nt, ctx->nwl, ctx->d_wave.as<double>(), ctx->d_hdr.as<LineHdr>(),
                                       ctx->d_wing.as<WingRec>(), ctx->d_core.as<CoreRec>(), ctx->d_tlo.as<int>(),
                                       ctx->d_thi.as<int>(), ctx->tab.vtab4, ctx->d_lineopac.as<double>(),
                                       ctx->d_ncore.as<unsigned long long>(), ctx->d_err.as<int>(),
                                       ctx->fault_extra_tx, ctx->fault_wait_ns);
            if (rc2) return cuda_fail(ctx, cudaGetLastError(), "k_core_fast");
            cudaEventRecord(eb, s);
            kt.push_back({ ea, em });
            kc.push_back({ em, eb });
            ctx->launches += 16;   // params, 2 x (extract, 2 scans of 2 kernels, search), count, wing, core
            nblocks++;
        }
    }
    // He I lines with Stark-shifted profiles (hestark.f90): the FP64 per-wavelength kernel of the
    // wide lines, which applies the per-depth shift (opacity.f90:297-346)
    if (ctx->nhe > 0) {
        int rc3 = fsg_select(s, n, sf, il, ir, -3, ctx->d_counts.as<int>(), ctx->d_offs.as<int64_t>(),
                             ctx->d_idx.as<int64_t>(), ctx->d_total.as<int64_t>());
        if (rc3) return cuda_fail(ctx, cudaGetLastError(), "select He I lines");
        int64_t nhl = 0;
        CK(cudaMemcpyAsync(&nhl, ctx->d_total.p, sizeof nhl, cudaMemcpyDeviceToHost, s), "He I lines");
        CK(cudaStreamSynchronize(s), "He I lines");
        ctx->launches += 3;
        if (nhl > 0) {
            ALLOC(ctx->d_pw, sizeof(double3) * nhl * nt);
            ALLOC(ctx->d_evals, sizeof(double));
            fsg_launch_wide_fp64(s, A, LV, (int)nhl, ctx->d_idx.as<int64_t>(), sf, wl_, wr_, ctx->d_pw.as<double3>(),
                                 ctx->tab, i0, i1, ctx->d_lineopac.as<double>(), ctx->d_evals.as<double>());
            ctx->launches += 2;
        }
    }
    CK(cudaGetLastError(), "fast accumulation");
    CK(cudaStreamSynchronize(s), "fast accumulation");
    int kerr = 0;
    CK(cudaMemcpy(&kerr, ctx->d_err.p, sizeof(int), cudaMemcpyDeviceToHost), "err read");
    if (kerr) return fail(ctx, FSG_E_TIMEOUT, "k_accum_fast: a line-record copy did not complete within its bound");
    unsigned long long ncore = 0;
    CK(cudaMemcpy(&ncore, ctx->d_ncore.p, sizeof ncore, cudaMemcpyDeviceToHost), "core count read");
    double msw = 0.0, msc = 0.0;
    for (auto &p : kt) { float x = 0; cudaEventElapsedTime(&x, p.first, p.second); msw += x; }
    for (auto &p : kc) { float x = 0; cudaEventElapsedTime(&x, p.first, p.second); msc += x; }
    if (st) {
        st->nblocks = nblocks; st->accum_launches = (int64_t)kt.size(); st->ms_accum_kernels = msw + msc;
        st->ms_wing_kernels = msw; st->ms_core_kernels = msc;
        st->core_evals = (double)ncore;
    }
    return FSG_OK;
}

// plain FP64 path mirroring LineopCalc's PACK / MarkWideLines / Lstart-Lstop / segment loop, over the
// windows in ctx->d_flags / d_ileft / d_iright.  [i0, i1]: 1-based wavelength range to fill (1..nwl for
// the whole grid); PACK, the wide-line marking and the segments are those of the whole grid, so every
// wavelength of the range sums the same lines in the same order as a whole-grid run.  nkeep < 0: count
// the retained lines here.
static int accumulate_fp64(fsg_ctx *ctx, const LineView &LV, int64_t nkeep, fsg_stats *st, int i0, int i1) {
    int64_t n = LV.n;
    const int nt = ctx->ntau, nwl = ctx->nwl;
    cudaStream_t s = ctx->stream;
    AtmView A = fsg_view(ctx);
    // NlinesStep (synth.f90:767): lines per FP64 block within LIMITRAM
    int64_t cap = block_capacity(ctx, sizeof(double3) * nt);
    int64_t nstep = std::min<int64_t>(n, cap);
    // PACK for atomic and .z lists in a single block (synth.f90:915-933)
    bool pack = (LV.kind == 0 || LV.kind == 2) && nstep == n;
    int64_t nblkscan = (n + 1023) / 1024;
    ALLOC(ctx->d_counts, sizeof(int) * std::max<int64_t>(nblkscan, 1));
    ALLOC(ctx->d_offs, sizeof(int64_t) * std::max<int64_t>(nblkscan, 1));
    ALLOC(ctx->d_total, sizeof(int64_t));
    ALLOC(ctx->d_idx, sizeof(int64_t) * std::max<int64_t>(n, 1));
    // working arrays in packed order: wl, flags, ileft, iright (gathered)
    LineView W = LV;
    int32_t *pf = ctx->d_flags.as<int32_t>(), *pl = ctx->d_ileft.as<int32_t>(), *pr = ctx->d_iright.as<int32_t>();
    int64_t nw = n;
    DBuf &gbuf = ctx->d_work;
    if (pack) {
        fsg_select(s, n, pf, pl, pr, -1, ctx->d_counts.as<int>(), ctx->d_offs.as<int64_t>(), ctx->d_idx.as<int64_t>(),
                   ctx->d_total.as<int64_t>());
        if (nkeep < 0) {
            CK(cudaMemcpyAsync(&nkeep, ctx->d_total.p, sizeof nkeep, cudaMemcpyDeviceToHost, s), "retained lines");
            CK(cudaStreamSynchronize(s), "retained lines");
        }
        nw = nkeep;
        // gather the per-line arrays of the retained lines (host-side gather is avoided: device gather)
        size_t need = 64 * (size_t)std::max<int64_t>(nw, 1);
        ALLOC(gbuf, need);
        int32_t *gf, *gl, *gr;
        fsg_launch_gather_lines(s, LV, ctx->d_idx.as<int64_t>(), nw, gbuf.as<char>(), pf, pl, pr, &W, &gf, &gl, &gr);
        pf = gf; pl = gl; pr = gr;
        W.n = nw;
    }
    if (nw == 0) { if (st) st->nlines_used = 0; return FSG_OK; }
    // MarkWideLines (synth.f90:709-744)
    ALLOC(ctx->d_nkeep, sizeof(unsigned long long));
    unsigned long long *d_nw = ctx->d_nkeep.as<unsigned long long>();
    CK(cudaMemsetAsync(d_nw, 0, sizeof(unsigned long long), s), "wide");
    fsg_launch_mark_wide(s, A, nw, W.wl, nstep, pf, pl, pr, d_nw);
    ctx->launches += pack ? 5 : 1;
    unsigned long long nwide = 0;
    CK(cudaMemcpyAsync(&nwide, d_nw, sizeof nwide, cudaMemcpyDeviceToHost, s), "wide");
    // Lstart/Lstop (synth.f90:955-978)
    ALLOC(ctx->d_lstart, sizeof(int) * nwl); ALLOC(ctx->d_lstop, sizeof(int) * nwl);
    {
        std::vector<int> ls(nwl, (int)nw), le(nwl, 1);
        CK(cudaMemcpyAsync(ctx->d_lstart.p, ls.data(), sizeof(int) * nwl, cudaMemcpyHostToDevice, s), "lstart");
        CK(cudaMemcpyAsync(ctx->d_lstop.p, le.data(), sizeof(int) * nwl, cudaMemcpyHostToDevice, s), "lstop");
        CK(cudaStreamSynchronize(s), "lstart");
    }
    fsg_launch_span(s, nw, pf, pl, pr, ctx->d_lstart.as<int>(), ctx->d_lstop.as<int>());
    ctx->launches += 1;
    ALLOC(ctx->d_evals, sizeof(double));
    CK(cudaMemsetAsync(ctx->d_evals.p, 0, sizeof(double), s), "evals");
    // wide lines: list, parameters, per-wavelength ordered accumulation
    if (nwide > 0) {
        ALLOC(ctx->d_widx, sizeof(int64_t) * nwide);
        fsg_select_wide(s, nw, pf, ctx->d_counts.as<int>(), ctx->d_offs.as<int64_t>(), ctx->d_widx.as<int64_t>(),
                        ctx->d_total.as<int64_t>());
        ALLOC(ctx->d_pw, sizeof(double3) * nwide * nt);
        fsg_launch_wide_fp64(s, A, W, (int)nwide, ctx->d_widx.as<int64_t>(), pf, pl, pr, ctx->d_pw.as<double3>(),
                             ctx->tab, i0, i1, ctx->d_lineopac.as<double>(), ctx->d_evals.as<double>());
        ctx->launches += 5;
    }
    // segment loop (synth.f90:1006-1088): choose segments on the host from Lstart/Lstop
    std::vector<int> ls(nwl), le(nwl);
    CK(cudaMemcpyAsync(ls.data(), ctx->d_lstart.p, sizeof(int) * nwl, cudaMemcpyDeviceToHost, s), "lstart");
    CK(cudaMemcpyAsync(le.data(), ctx->d_lstop.p, sizeof(int) * nwl, cudaMemcpyDeviceToHost, s), "lstop");
    CK(cudaStreamSynchronize(s), "lstart");
    ALLOC(ctx->d_p64, sizeof(double3) * (size_t)std::min<int64_t>(nstep, nw) * nt);
    int64_t iline1 = 1, ilineb = 0;
    int iwl1 = 1;
    int64_t nblocks = 0;
    for (;;) {
        int iwl2;
        if (nstep >= nw) iwl2 = nwl;
        else {
            int64_t ilo = nw + 1, ihi = 0;
            iwl2 = iwl1 - 1;
            for (int iwl = iwl1; iwl <= nwl; iwl++) {
                int64_t ilot = std::min<int64_t>(ilo, ls[iwl - 1]), ihit = std::max<int64_t>(ihi, le[iwl - 1]);
                if (ihit - ilot + 1 > nstep) break;
                ilo = ilot; ihi = ihit; iwl2 = iwl;
            }
            if (iwl2 < iwl1) {
                char m[256];
                snprintf(m, sizeof m, "line opacity segmentation: lines contributing to wavelength point #%d span more "
                         "than %lld line records; increase limitram", iwl1, (long long)nstep);
                return fail(ctx, FSG_E_SEGMENT, m);
            }
            iline1 = std::min<int64_t>(std::max<int64_t>(ilo, 1), nw);
        }
        int64_t iline2 = std::min<int64_t>(iline1 + nstep - 1, nw);
        int64_t loff = iline1 - 1;
        const int ra = std::max(iwl1, i0), rb = std::min(iwl2, i1);    // the segment's part of the range
        if (ra <= rb) {
            if (iline1 != ilineb) {
                ilineb = iline1;
                fsg_launch_params_fp64(s, A, W, loff, iline2 - loff, pf, ctx->d_p64.as<double3>());
                ctx->launches += 1;
                nblocks++;
            }
            cudaEvent_t ea = ctx->ev[4], eb = ctx->ev[5];
            cudaEventRecord(ea, s);
            fsg_launch_accum_fp64(s, A, W.wl, ra, rb, ctx->d_lstart.as<int>(), ctx->d_lstop.as<int>(), pf, pl, pr,
                                  loff, ctx->d_p64.as<double3>(), ctx->tab, ctx->d_lineopac.as<double>(),
                                  ctx->d_evals.as<double>());
            CK(cudaGetLastError(), "fp64 accumulation");
            cudaEventRecord(eb, s);
            CK(cudaEventSynchronize(eb), "fp64 accumulation");
            { float x = 0; cudaEventElapsedTime(&x, ea, eb); if (st) { st->ms_accum_kernels += x; st->accum_launches++; } }
            ctx->launches += 1;
        }
        if (iwl2 == nwl) break;
        iwl1 = iwl2 + 1;
    }
    double ev = 0;
    CK(cudaMemcpyAsync(&ev, ctx->d_evals.p, sizeof ev, cudaMemcpyDeviceToHost, s), "evals");
    CK(cudaStreamSynchronize(s), "fp64 accumulation");
    if (st) { st->nwide = (int64_t)nwide; st->nblocks = nblocks; st->line_evals = ev; }
    // per-line outputs in original order: scatter the packed wide flags back
    if (pack) {
        fsg_launch_scatter_flags(s, nw, ctx->d_idx.as<int64_t>(), pf, ctx->d_flags.as<int32_t>());
        ctx->launches += 1;
    }
    return FSG_OK;
}

// The host list streams to the device in chunks on the copy stream; the central pass of each chunk
// starts on the compute stream as soon as its copy has landed (pinned host memory overlaps both).
#define UPLOAD_CHUNK ((int64_t)1 << 23)
static int central_pass_streamed(fsg_ctx *ctx, const fsg_lines *H, const fsg_lines *D, int64_t *nkeep) {
    const int64_t n = D->n;
    ALLOC(ctx->d_flags, sizeof(int32_t) * std::max<int64_t>(n, 1));
    ALLOC(ctx->d_ileft, sizeof(int32_t) * std::max<int64_t>(n, 1));
    ALLOC(ctx->d_iright, sizeof(int32_t) * std::max<int64_t>(n, 1));
    ALLOC(ctx->d_nkeep, sizeof(unsigned long long));
    cudaStream_t s = ctx->stream, c = ctx->cstream;
    CK(cudaMemsetAsync(ctx->d_nkeep.p, 0, sizeof(unsigned long long), s), "center");
    const int64_t nch = (n + UPLOAD_CHUNK - 1) / UPLOAD_CHUNK;
    while ((int64_t)ctx->cev.size() < nch) { cudaEvent_t e; cudaEventCreateWithFlags(&e, cudaEventDisableTiming); ctx->cev.push_back(e); }
    // the copy stream must not overwrite buffers the compute stream still reads from a previous call
    CK(cudaEventRecord(ctx->ev[7], s), "event");
    CK(cudaStreamWaitEvent(c, ctx->ev[7], 0), "event");
    AtmView A = fsg_view(ctx);
    for (int64_t k = 0; k < nch; k++) {
        const int64_t a = k * UPLOAD_CHUNK, m = std::min(UPLOAD_CHUNK, n - a);
        auto cp = [&](void *dst, const void *src, size_t esz) {
            return cudaMemcpyAsync((char *)dst + a * esz, (const char *)src + a * esz, m * esz, cudaMemcpyHostToDevice, c);
        };
        CK(cp((void *)D->wl, H->wl, 8), "line upload");
        CK(cp((void *)D->elo, H->elo, 4), "line upload");
        CK(cp((void *)D->gf, H->gf, 4), "line upload");
        CK(cp((void *)D->grad, H->grad, 4), "line upload");
        CK(cp((void *)D->gqst, H->gqst, 4), "line upload");
        CK(cp((void *)D->gvdw, H->gvdw, 4), "line upload");
        CK(cp((void *)D->spc, H->spc, 4), "line upload");
        if (H->ismol) CK(cp((void *)D->ismol, H->ismol, 4), "line upload");
        if (H->ihe) CK(cp((void *)D->ihe, H->ihe, 4), "line upload");
        CK(cudaEventRecord(ctx->cev[k], c), "event");
        CK(cudaStreamWaitEvent(s, ctx->cev[k], 0), "event");
        fsg_lines Dk = *D;
        Dk.n = m;
        Dk.wl += a; Dk.elo += a; Dk.gf += a; Dk.grad += a; Dk.gqst += a; Dk.gvdw += a; Dk.spc += a;
        if (Dk.ismol) Dk.ismol += a;
        if (Dk.ihe) Dk.ihe += a;
        fsg_launch_center(s, A, make_view(&Dk), ctx->tab, ctx->d_flags.as<int32_t>() + a, ctx->d_ileft.as<int32_t>() + a,
                          ctx->d_iright.as<int32_t>() + a, ctx->d_nkeep.as<unsigned long long>());
        ctx->launches += 1;
    }
    CK(cudaGetLastError(), "k_center");
    unsigned long long nk = 0;
    CK(cudaMemcpyAsync(&nk, ctx->d_nkeep.p, sizeof nk, cudaMemcpyDeviceToHost, s), "center");
    CK(cudaStreamSynchronize(s), "center");
    *nkeep = (int64_t)nk;
    return FSG_OK;
}

// D: device list; H: the host list it is uploaded from during the central pass (NULL: D is resident)
static int lineop_dev(fsg_ctx *ctx, const fsg_lines *D, fsg_stats *st, const fsg_lines *H = nullptr) {
    LineView LV = make_view(D);
    int rc = ensure_lineopac(ctx); if (rc) return rc;
    if (st) { memset(st, 0, sizeof *st); st->nlines_in = D->n; }
    if (D->n == 0) return FSG_OK;
    cudaStream_t s = ctx->stream;
    CK(cudaEventRecord(ctx->ev[0], s), "event");
    int64_t nkeep = 0;
    rc = H ? central_pass_streamed(ctx, H, D, &nkeep) : central_pass(ctx, LV, &nkeep);
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev[1], s), "event");
    if (st) { st->nlines_used = nkeep; st->nweak = D->n - nkeep; }
    if (ctx->cfg.precision == FSG_PREC_FP64) rc = accumulate_fp64(ctx, LV, nkeep, st, 1, ctx->nwl);
    else rc = accumulate_fast(ctx, LV, st, ctx->d_flags.as<int32_t>(), ctx->d_ileft.as<int32_t>(),
                              ctx->d_iright.as<int32_t>(), 1, ctx->nwl);
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev[2], s), "event");
    CK(cudaStreamSynchronize(s), "lineop");
    if (st) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]);
        cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]);
        st->ms_center = a; st->ms_accum = b; st->ms_total = a + b;
        if (ctx->cfg.precision != FSG_PREC_FP64)
            st->line_evals = fsg_count_evals(ctx, D->n, ctx->d_flags.as<int32_t>(), ctx->d_ileft.as<int32_t>(),
                                             ctx->d_iright.as<int32_t>(), 1, ctx->nwl);
    }
    return FSG_OK;
}

// ---- split driver for wavelength sharding: central pass of a subset, accumulation of a range ----
int fsg_central_dev(fsg_ctx *ctx, const fsg_lines *d_lines, int32_t *d_flags, int32_t *d_ileft, int32_t *d_iright,
                    int64_t *nkeep) {
    int rc = check_lines(ctx, d_lines); if (rc) return rc;
    if (d_lines->n > 0 && (!d_flags || !d_ileft || !d_iright))
        return fail(ctx, FSG_E_ARG, "fsg_central_dev: output arrays missing");
    cudaSetDevice(ctx->device);
    LineView LV = make_view(d_lines);
    ALLOC(ctx->d_nkeep, sizeof(unsigned long long));
    CK(cudaMemsetAsync(ctx->d_nkeep.p, 0, sizeof(unsigned long long), ctx->stream), "center");
    if (d_lines->n > 0) {
        fsg_launch_center(ctx->stream, fsg_view(ctx), LV, ctx->tab, d_flags, d_ileft, d_iright,
                          ctx->d_nkeep.as<unsigned long long>());
        ctx->launches += 1;
        CK(cudaGetLastError(), "k_center");
    }
    unsigned long long nk = 0;
    CK(cudaMemcpyAsync(&nk, ctx->d_nkeep.p, sizeof nk, cudaMemcpyDeviceToHost, ctx->stream), "center");
    CK(cudaStreamSynchronize(ctx->stream), "center");
    if (nkeep) *nkeep = (int64_t)nk;
    return FSG_OK;
}

int fsg_accumulate_dev(fsg_ctx *ctx, const fsg_lines *d_lines, const int32_t *d_flags, const int32_t *d_ileft,
                       const int32_t *d_iright, int i0, int i1, fsg_stats *st) {
    int rc = check_lines(ctx, d_lines); if (rc) return rc;
    if (i0 < 1 || i1 > ctx->nwl || i0 > i1) return fail(ctx, FSG_E_ARG, "fsg_accumulate_dev: need 1 <= i0 <= i1 <= nwl");
    if (d_lines->n > 0 && (!d_flags || !d_ileft || !d_iright))
        return fail(ctx, FSG_E_ARG, "fsg_accumulate_dev: window arrays missing");
    cudaSetDevice(ctx->device);
    rc = ensure_lineopac(ctx); if (rc) return rc;
    if (st) { memset(st, 0, sizeof *st); st->nlines_in = d_lines->n; }
    if (d_lines->n == 0) return FSG_OK;
    cudaStream_t s = ctx->stream;
    CK(cudaEventRecord(ctx->ev[1], s), "event");
    if (ctx->cfg.precision == FSG_PREC_FP64) {
        // the FP64 path marks wide lines in its own copy of the windows
        const size_t nb = sizeof(int32_t) * (size_t)d_lines->n;
        ALLOC(ctx->d_flags, nb); ALLOC(ctx->d_ileft, nb); ALLOC(ctx->d_iright, nb);
        CK(cudaMemcpyAsync(ctx->d_flags.p, d_flags, nb, cudaMemcpyDeviceToDevice, s), "windows");
        CK(cudaMemcpyAsync(ctx->d_ileft.p, d_ileft, nb, cudaMemcpyDeviceToDevice, s), "windows");
        CK(cudaMemcpyAsync(ctx->d_iright.p, d_iright, nb, cudaMemcpyDeviceToDevice, s), "windows");
        rc = accumulate_fp64(ctx, make_view(d_lines), -1, st, i0, i1);
    } else {
        rc = accumulate_fast(ctx, make_view(d_lines), st, d_flags, d_ileft, d_iright, i0, i1);
    }
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev[2], s), "event");
    CK(cudaStreamSynchronize(s), "accumulate");
    if (st) {
        float b = 0;
        cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]);
        st->ms_accum = b; st->ms_total = b;
        if (ctx->cfg.precision != FSG_PREC_FP64)
            st->line_evals = fsg_count_evals(ctx, d_lines->n, d_flags, d_ileft, d_iright, i0, i1);
    }
    return FSG_OK;
}

static int lineop_calc_dev_body(fsg_ctx *ctx, const fsg_lines *d_lines, fsg_stats *st) {
    int rc = check_lines(ctx, d_lines); if (rc) return rc;
    cudaSetDevice(ctx->device);
    return lineop_dev(ctx, d_lines, st);
}

// LinStrCalc (synth.f90:1774-1822) for the retained lines of the list whose central pass set
// ctx->d_flags (original order); host output, 0 for rejected lines.  Chunks of at most 2^18 lines.
static int linstr_calc(fsg_ctx *ctx, const fsg_lines *D, float *linstr) {
    cudaStream_t s = ctx->stream;
    const int64_t n = D->n;
    const int64_t chunk = std::min<int64_t>(n, 1 << 18);
    ALLOC(ctx->d_lswork, fsg_linstr_work(chunk, ctx->ntau, ctx->nmu));
    ALLOC(ctx->d_linstr, sizeof(float) * (size_t)n);
    LineView LV = make_view(D);
    AtmView A = fsg_view(ctx);
    RayView R;
    int rc = rays_prepare(ctx, &R); if (rc) return rc;
    for (int64_t i0 = 0; i0 < n; i0 += chunk) {
        fsg_launch_linstr(s, A, LV, ctx->tab, ctx->d_flags.as<int32_t>(), i0, std::min(chunk, n - i0), ctx->nmu,
                          ctx->d_xmu.as<double>(), ctx->d_wmu.as<double>(), ctx->d_rhox.as<double>(), R,
                          ctx->d_lswork.as<double>(), ctx->d_linstr.as<float>());
        ctx->launches += 1;
    }
    CK(cudaGetLastError(), "k_linstr");
    CK(cudaMemcpyAsync(linstr, ctx->d_linstr.p, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, s), "linstr");
    CK(cudaStreamSynchronize(s), "linstr");
    return FSG_OK;
}

static int lineop_calc_body(fsg_ctx *ctx, const fsg_lines *lines, double *lineopac, int32_t *flags,
                            int32_t *ileft, int32_t *iright, float *linstr, fsg_stats *st) {
    int rc = check_lines(ctx, lines); if (rc) return rc;
    if (linstr && ctx->nmu < 1) return fail(ctx, FSG_E_STATE, "fsg_lineop_calc: line strengths need fsg_set_mu first");
    cudaSetDevice(ctx->device);
    fsg_lines D;
    if (lines->n > 0) { rc = device_lines(ctx, lines, &D); if (rc) return rc; }
    else D = *lines;
    rc = lineop_dev(ctx, &D, st, lines->n > 0 ? lines : nullptr); if (rc) return rc;
    cudaStream_t s = ctx->stream;
    if (linstr && lines->n > 0) { rc = linstr_calc(ctx, &D, linstr); if (rc) return rc; }
    size_t n4 = sizeof(int32_t) * lines->n;
    if (lines->n > 0) {
        if (flags) CK(cudaMemcpyAsync(flags, ctx->d_flags.p, n4, cudaMemcpyDeviceToHost, s), "flags");
        if (ileft) CK(cudaMemcpyAsync(ileft, ctx->d_ileft.p, n4, cudaMemcpyDeviceToHost, s), "ileft");
        if (iright) CK(cudaMemcpyAsync(iright, ctx->d_iright.p, n4, cudaMemcpyDeviceToHost, s), "iright");
    }
    if (lineopac) CK(cudaMemcpyAsync(lineopac, ctx->d_lineopac.p, sizeof(double) * (size_t)ctx->nwl * ctx->ntau, cudaMemcpyDeviceToHost, s), "lineopac");
    CK(cudaStreamSynchronize(s), "lineop outputs");
    return FSG_OK;
}

// ---- RadTranCalc ------------------------------------------------------------------------------------
// RadTranCalc + flux over the wavelengths i0..i1 (1-based, inclusive) into arrays laid out over the
// whole grid.  The solver kernels index wavelengths from the view's base pointers, so the range is a
// view whose wave / continuum / line-opacity / output bases start at wavelength i0.
static int radtran_dev(fsg_ctx *ctx, double *spl, double *spc, double *sfl, double *sfc, int i0 = 1,
                       int i1 = -1) {
    if (!ctx->have_grid || !ctx->have_atm || !ctx->have_cont || ctx->nmu < 1)
        return fail(ctx, FSG_E_STATE, "radtran: set grid, atmosphere, continuum and mu first");
    if (i1 < 0) i1 = ctx->nwl;
    if (i0 < 1 || i1 > ctx->nwl || i0 > i1) return fail(ctx, FSG_E_ARG, "radtran: need 1 <= i0 <= i1 <= nwl");
    int rc = ensure_lineopac(ctx); if (rc) return rc;
    AtmView A = fsg_view(ctx);
    const size_t o = (size_t)(i0 - 1), nt = (size_t)ctx->ntau, nmu = (size_t)ctx->nmu;
    A.nwl = i1 - i0 + 1;
    A.wave += o;
    A.contopac += o * nt;
    const double *lop = ctx->d_lineopac.as<double>() + o * nt;
    if (spl) spl += o * nmu;
    if (spc) spc += o * nmu;
    if (sfl) sfl += o;
    if (sfc) sfc += o;
    RayView R;
    rc = rays_prepare(ctx, &R); if (rc) return rc;
    if (R.nmu > 0)
        rc = fsg_launch_radtran_sph(ctx->stream, A, lop, R, ctx->d_wmu.as<double>(), spl, spc, sfl, sfc);
    else
        rc = fsg_launch_radtran(ctx->stream, A, lop, ctx->d_rhox.as<double>(), ctx->nmu, ctx->d_xmu.as<double>(),
                                ctx->d_wmu.as<double>(), spl, spc, sfl, sfc);
    ctx->launches += 1;
    if (rc) return cuda_fail(ctx, cudaGetLastError(), "k_radtran");
    return FSG_OK;
}

static int radtran_dev_body(fsg_ctx *ctx, double *d_spl, double *d_spc, double *d_sfl, double *d_sfc) {
    if (!ctx) return FSG_E_ARG;
    cudaSetDevice(ctx->device);
    int rc = radtran_dev(ctx, d_spl, d_spc, d_sfl, d_sfc); if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream), "radtran");
    return FSG_OK;
}

static int radtran_range_dev_body(fsg_ctx *ctx, int i0, int i1, double *d_spl, double *d_spc, double *d_sfl,
                                  double *d_sfc) {
    if (!ctx) return FSG_E_ARG;
    cudaSetDevice(ctx->device);
    int rc = radtran_dev(ctx, d_spl, d_spc, d_sfl, d_sfc, i0, i1); if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream), "radtran");
    return FSG_OK;
}

static int radtran_body(fsg_ctx *ctx, double *spl, double *spc, double *sfl, double *sfc) {
    if (!ctx) return FSG_E_ARG;
    cudaSetDevice(ctx->device);
    size_t nsp = sizeof(double) * (size_t)ctx->nwl * ctx->nmu, nf = sizeof(double) * ctx->nwl;
    ALLOC(ctx->d_spl, nsp); ALLOC(ctx->d_spc, nsp); ALLOC(ctx->d_sfl, nf); ALLOC(ctx->d_sfc, nf);
    int rc = radtran_dev(ctx, ctx->d_spl.as<double>(), ctx->d_spc.as<double>(), ctx->d_sfl.as<double>(),
                         ctx->d_sfc.as<double>());
    if (rc) return rc;
    cudaStream_t s = ctx->stream;
    if (spl) CK(cudaMemcpyAsync(spl, ctx->d_spl.p, nsp, cudaMemcpyDeviceToHost, s), "spl");
    if (spc) CK(cudaMemcpyAsync(spc, ctx->d_spc.p, nsp, cudaMemcpyDeviceToHost, s), "spc");
    if (sfl) CK(cudaMemcpyAsync(sfl, ctx->d_sfl.p, nf, cudaMemcpyDeviceToHost, s), "sfl");
    if (sfc) CK(cudaMemcpyAsync(sfc, ctx->d_sfc.p, nf, cudaMemcpyDeviceToHost, s), "sfc");
    CK(cudaStreamSynchronize(s), "radtran");
    return FSG_OK;
}


// ---- MagLineopCalc (synth.f90:1098-1455) ---------------------------------------------------------
static int ensure_maglineopac(fsg_ctx *ctx) {
    size_t nb = sizeof(double) * 6 * (size_t)ctx->nwl * ctx->ntau;
    if (ctx->d_maglineopac.cap < nb) {
        ALLOC(ctx->d_maglineopac, nb);
        CK(cudaMemsetAsync(ctx->d_maglineopac.p, 0, nb, ctx->stream), "maglineopac reset");
    }
    return FSG_OK;
}

int fsg_mag_lineop_reset(fsg_ctx *ctx) {
    if (!ctx) return FSG_E_ARG;
    if (!ctx->have_grid || !ctx->have_atm) return fail(ctx, FSG_E_STATE, "fsg_mag_lineop_reset: set grid and atmosphere first");
    cudaSetDevice(ctx->device);
    int rc = ensure_maglineopac(ctx); if (rc) return rc;
    CK(cudaMemsetAsync(ctx->d_maglineopac.p, 0, sizeof(double) * 6 * (size_t)ctx->nwl * ctx->ntau, ctx->stream), "reset");
    CK(cudaStreamSynchronize(ctx->stream), "reset");
    return FSG_OK;
}

static int mag_lineop_calc_body(fsg_ctx *ctx, const fsg_lines *lines, int bframe, const double *bfield,
                                int nbfield, double *maglineopac, int32_t *flags, int32_t *ileft, int32_t *iright,
                                float *linstr, fsg_stats *st) {
    int rc = check_lines(ctx, lines); if (rc) return rc;
    if (linstr && ctx->nmu < 1) return fail(ctx, FSG_E_STATE, "fsg_mag_lineop_calc: line strengths need fsg_set_mu first");
    if (lines->kind != 2) return fail(ctx, FSG_E_ARG, "fsg_mag_lineop_calc: magnetic lists have kind 2");
    if (!bfield || (bframe < 0 || bframe > 2) || nbfield < 3 || (bframe == 2 && nbfield != 2 * ctx->nmu + 1))
        return fail(ctx, FSG_E_ARG, "fsg_mag_lineop_calc: BFIELD needs 3 values (frames 0, 1) or 2*nmu+1 (frame 2)");
    int64_t n = lines->n;
    if (n > 0 && (!lines->npi || !lines->nsi || !lines->pi_off || !lines->si_off || !lines->spl_pi || !lines->str_pi ||
                  !lines->spl_si || !lines->str_si))
        return fail(ctx, FSG_E_ARG, "fsg_mag_lineop_calc: Zeeman component arrays missing");
    cudaSetDevice(ctx->device);
    rc = ensure_maglineopac(ctx); if (rc) return rc;
    if (st) { memset(st, 0, sizeof *st); st->nlines_in = n; }
    if (n == 0) return FSG_OK;
    cudaStream_t s = ctx->stream;
    const int nt = ctx->ntau, nwl = ctx->nwl;
    CK(cudaEventRecord(ctx->ev[0], s), "event");
    fsg_lines D;
    rc = upload_lines(ctx, lines, &D); if (rc) return rc;
    int64_t npi_tot = lines->pi_off[n - 1] + lines->npi[n - 1], nsi_tot = lines->si_off[n - 1] + lines->nsi[n - 1];
    ALLOC(ctx->z_npi, sizeof(int32_t) * n); ALLOC(ctx->z_nsi, sizeof(int32_t) * n);
    ALLOC(ctx->z_pioff, sizeof(int64_t) * n); ALLOC(ctx->z_sioff, sizeof(int64_t) * n);
    ALLOC(ctx->z_rawpi, sizeof(float) * (npi_tot + 1)); ALLOC(ctx->z_strpi, sizeof(float) * (npi_tot + 1));
    ALLOC(ctx->z_rawsi, sizeof(float) * (nsi_tot + 1)); ALLOC(ctx->z_strsi, sizeof(float) * (nsi_tot + 1));
    ALLOC(ctx->z_splpi, sizeof(float) * (npi_tot + 1)); ALLOC(ctx->z_splsi, sizeof(float) * (nsi_tot + 1));
    CK(cudaMemcpyAsync(ctx->z_npi.p, lines->npi, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s), "zeeman upload");
    CK(cudaMemcpyAsync(ctx->z_nsi.p, lines->nsi, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s), "zeeman upload");
    CK(cudaMemcpyAsync(ctx->z_pioff.p, lines->pi_off, sizeof(int64_t) * n, cudaMemcpyHostToDevice, s), "zeeman upload");
    CK(cudaMemcpyAsync(ctx->z_sioff.p, lines->si_off, sizeof(int64_t) * n, cudaMemcpyHostToDevice, s), "zeeman upload");
    if (npi_tot > 0) {
        CK(cudaMemcpyAsync(ctx->z_rawpi.p, lines->spl_pi, sizeof(float) * npi_tot, cudaMemcpyHostToDevice, s), "zeeman upload");
        CK(cudaMemcpyAsync(ctx->z_strpi.p, lines->str_pi, sizeof(float) * npi_tot, cudaMemcpyHostToDevice, s), "zeeman upload");
    }
    if (nsi_tot > 0) {
        CK(cudaMemcpyAsync(ctx->z_rawsi.p, lines->spl_si, sizeof(float) * nsi_tot, cudaMemcpyHostToDevice, s), "zeeman upload");
        CK(cudaMemcpyAsync(ctx->z_strsi.p, lines->str_si, sizeof(float) * nsi_tot, cudaMemcpyHostToDevice, s), "zeeman upload");
    }
    ZView Z;
    Z.npi = ctx->z_npi.as<int32_t>(); Z.nsi = ctx->z_nsi.as<int32_t>();
    Z.pi_off = ctx->z_pioff.as<int64_t>(); Z.si_off = ctx->z_sioff.as<int64_t>();
    Z.strpi = ctx->z_strpi.as<float>(); Z.strsi = ctx->z_strsi.as<float>();
    Z.splpi = ctx->z_splpi.as<float>(); Z.splsi = ctx->z_splsi.as<float>();
    Z.rawpi = ctx->z_rawpi.as<float>(); Z.rawsi = ctx->z_rawsi.as<float>();
    double Bsplit = (bframe == 0) ? FSG_KZ * sqrt(bfield[0] * bfield[0] + bfield[1] * bfield[1] + bfield[2] * bfield[2])
                                  : FSG_KZ * fabs(bfield[0]);
    LineView LV = make_view(&D);
    AtmView A = fsg_view(ctx);
    ALLOC(ctx->d_flags, sizeof(int32_t) * n); ALLOC(ctx->d_ileft, sizeof(int32_t) * n);
    ALLOC(ctx->d_iright, sizeof(int32_t) * n); ALLOC(ctx->d_nkeep, sizeof(unsigned long long));
    CK(cudaMemsetAsync(ctx->d_nkeep.p, 0, sizeof(unsigned long long), s), "mag center");
    int32_t *pf = ctx->d_flags.as<int32_t>(), *pl = ctx->d_ileft.as<int32_t>(), *pr = ctx->d_iright.as<int32_t>();
    fsg_launch_mag_center(s, A, LV, Z, Bsplit, ctx->tab, pf, pl, pr, ctx->d_nkeep.as<unsigned long long>());
    ctx->launches += 1;
    CK(cudaGetLastError(), "k_mag_center");
    unsigned long long nk = 0;
    CK(cudaMemcpyAsync(&nk, ctx->d_nkeep.p, sizeof nk, cudaMemcpyDeviceToHost, s), "mag center");
    CK(cudaStreamSynchronize(s), "mag center");
    // the magnetic driver takes the same non-magnetic central depths (synth.f90:1236-1239)
    if (linstr) { rc = linstr_calc(ctx, &D, linstr); if (rc) return rc; }
    CK(cudaEventRecord(ctx->ev[1], s), "event");
    int64_t nkeep = (int64_t)nk;
    if (st) { st->nlines_used = nkeep; st->nweak = n - nkeep; }
    if (ctx->cfg.precision == FSG_PREC_MIXED) {
        // mixed precision: retained lines in blocks, FP32 Faraday-Voigt on 32-wavelength tiles
        int64_t nblkscan = (n + 1023) / 1024;
        ALLOC(ctx->d_counts, sizeof(int) * std::max<int64_t>(nblkscan, 1));
        ALLOC(ctx->d_offs, sizeof(int64_t) * std::max<int64_t>(nblkscan, 1));
        ALLOC(ctx->d_total, sizeof(int64_t));
        ALLOC(ctx->d_idx, sizeof(int64_t) * n);
        if (fsg_select(s, n, pf, pl, pr, -1, ctx->d_counts.as<int>(), ctx->d_offs.as<int64_t>(),
                       ctx->d_idx.as<int64_t>(), ctx->d_total.as<int64_t>()))
            return cuda_fail(ctx, cudaGetLastError(), "select");
        ctx->launches += 3;
        const size_t per_line = fsg_mag_rec_bytes() * nt + sizeof(LineHdr) + sizeof(int64_t);
        const int64_t bcap = std::min<int64_t>(std::max<int64_t>(nkeep, 1), block_capacity(ctx, per_line));
        ALLOC(ctx->d_wing, fsg_mag_rec_bytes() * (size_t)bcap * nt);
        ALLOC(ctx->d_hdr, sizeof(LineHdr) * (size_t)bcap);
        ALLOC(ctx->d_zmap, sizeof(int64_t) * (size_t)bcap);
        ALLOC(ctx->d_span, fsg_tile_span_scratch(bcap));
        ALLOC(ctx->d_tlo, sizeof(int) * (size_t)fsg_fast_tiles(nwl)); ALLOC(ctx->d_thi, sizeof(int) * (size_t)fsg_fast_tiles(nwl));
        double *mlo = ctx->d_maglineopac.as<double>();
        int64_t nblocks = 0;
        for (int64_t j0 = 0; j0 < nkeep; j0 += bcap) {
            const int64_t nb = std::min(bcap, nkeep - j0);
            fsg_launch_mag_params_fast(s, A, LV, Z, ctx->d_idx.as<int64_t>(), j0, nb, pf, pl, pr, ctx->tab, ctx->d_wing.p,
                                       ctx->d_hdr.as<LineHdr>(), ctx->d_zmap.as<int64_t>());
            if (fsg_launch_tile_span_tw(s, 32, 0, nwl, nb, ctx->d_hdr.as<LineHdr>(), ctx->d_tlo.as<int>(),
                                        ctx->d_thi.as<int>(), ctx->d_span.p, ctx->d_span.cap) ||
                fsg_launch_mag_fast(s, A, ctx->d_hdr.as<LineHdr>(), ctx->d_wing.p, ctx->d_zmap.as<int64_t>(), Z,
                                    ctx->d_tlo.as<int>(), ctx->d_thi.as<int>(), ctx->tab, mlo))
                return cuda_fail(ctx, cudaGetLastError(), "k_mag_fast");
            ctx->launches += 8;
            nblocks++;
        }
        CK(cudaEventRecord(ctx->ev[2], s), "event");
        size_t n4 = sizeof(int32_t) * n;
        if (flags) CK(cudaMemcpyAsync(flags, ctx->d_flags.p, n4, cudaMemcpyDeviceToHost, s), "flags");
        if (ileft) CK(cudaMemcpyAsync(ileft, ctx->d_ileft.p, n4, cudaMemcpyDeviceToHost, s), "ileft");
        if (iright) CK(cudaMemcpyAsync(iright, ctx->d_iright.p, n4, cudaMemcpyDeviceToHost, s), "iright");
        if (maglineopac)
            CK(cudaMemcpyAsync(maglineopac, mlo, sizeof(double) * 6 * (size_t)nwl * nt, cudaMemcpyDeviceToHost, s), "mlo");
        CK(cudaStreamSynchronize(s), "mag lineop");
        if (st) {
            float a = 0, b = 0;
            cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]);
            cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]);
            st->ms_center = a; st->ms_accum = b; st->ms_total = a + b;
            st->nblocks = nblocks;
            st->line_evals = count_windows(ctx, n, ctx->d_flags.as<int32_t>(), ctx->d_ileft.as<int32_t>(),
                                           ctx->d_iright.as<int32_t>(), 1, nwl, Z.npi, Z.nsi) * nt;
        }
        return FSG_OK;
    }
    // NlinesStep and PACK (synth.f90:1131, 1283-1297)
    int64_t cap = block_capacity(ctx, sizeof(double3) * nt);
    int64_t nstep = std::min<int64_t>(n, cap);
    bool pack = (nstep == n);
    int64_t nblkscan = (n + 1023) / 1024;
    ALLOC(ctx->d_counts, sizeof(int) * std::max<int64_t>(nblkscan, 1));
    ALLOC(ctx->d_offs, sizeof(int64_t) * std::max<int64_t>(nblkscan, 1));
    ALLOC(ctx->d_total, sizeof(int64_t));
    ALLOC(ctx->d_idx, sizeof(int64_t) * n);
    LineView W = LV;
    int64_t nw = n;
    const int64_t *zmap = nullptr;
    if (pack) {
        fsg_select(s, n, pf, pl, pr, -1, ctx->d_counts.as<int>(), ctx->d_offs.as<int64_t>(), ctx->d_idx.as<int64_t>(),
                   ctx->d_total.as<int64_t>());
        nw = nkeep;
        ALLOC(ctx->d_work, 64 * (size_t)std::max<int64_t>(nw, 1));
        int32_t *gf, *gl, *gr;
        fsg_launch_gather_lines(s, LV, ctx->d_idx.as<int64_t>(), nw, ctx->d_work.as<char>(), pf, pl, pr, &W, &gf, &gl, &gr);
        ctx->launches += 4;
        pf = gf; pl = gl; pr = gr;
        W.n = nw;
        zmap = ctx->d_idx.as<int64_t>();
    } else {
        std::vector<int64_t> iota(n);
        for (int64_t i = 0; i < n; i++) iota[i] = i;
        ALLOC(ctx->d_zmap, sizeof(int64_t) * n);
        CK(cudaMemcpyAsync(ctx->d_zmap.p, iota.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, s), "zmap");
        zmap = ctx->d_zmap.as<int64_t>();
    }
    if (nw == 0) {                                   // every line rejected: per-line outputs only
        size_t n4 = sizeof(int32_t) * n;
        if (flags) CK(cudaMemcpyAsync(flags, ctx->d_flags.p, n4, cudaMemcpyDeviceToHost, s), "flags");
        if (ileft) CK(cudaMemcpyAsync(ileft, ctx->d_ileft.p, n4, cudaMemcpyDeviceToHost, s), "ileft");
        if (iright) CK(cudaMemcpyAsync(iright, ctx->d_iright.p, n4, cudaMemcpyDeviceToHost, s), "iright");
        CK(cudaStreamSynchronize(s), "mag lineop");
        return FSG_OK;
    }
    unsigned long long *d_nw = ctx->d_nkeep.as<unsigned long long>();
    CK(cudaMemsetAsync(d_nw, 0, sizeof(unsigned long long), s), "wide");
    fsg_launch_mark_wide(s, A, nw, W.wl, nstep, pf, pl, pr, d_nw);
    unsigned long long nwide = 0;
    CK(cudaMemcpyAsync(&nwide, d_nw, sizeof nwide, cudaMemcpyDeviceToHost, s), "wide");
    ALLOC(ctx->d_lstart, sizeof(int) * nwl); ALLOC(ctx->d_lstop, sizeof(int) * nwl);
    {
        std::vector<int> ls(nwl, (int)nw), le(nwl, 1);
        CK(cudaMemcpyAsync(ctx->d_lstart.p, ls.data(), sizeof(int) * nwl, cudaMemcpyHostToDevice, s), "lstart");
        CK(cudaMemcpyAsync(ctx->d_lstop.p, le.data(), sizeof(int) * nwl, cudaMemcpyHostToDevice, s), "lstop");
        CK(cudaStreamSynchronize(s), "lstart");
    }
    fsg_launch_span(s, nw, pf, pl, pr, ctx->d_lstart.as<int>(), ctx->d_lstop.as<int>());
    ctx->launches += 2;
    ALLOC(ctx->d_evals, sizeof(double));
    CK(cudaMemsetAsync(ctx->d_evals.p, 0, sizeof(double), s), "evals");
    double *mlo = ctx->d_maglineopac.as<double>();
    if (nwide > 0) {
        ALLOC(ctx->d_widx, sizeof(int64_t) * nwide);
        fsg_select_wide(s, nw, pf, ctx->d_counts.as<int>(), ctx->d_offs.as<int64_t>(), ctx->d_widx.as<int64_t>(),
                        ctx->d_total.as<int64_t>());
        ALLOC(ctx->d_pw, sizeof(double3) * nwide * nt);
        fsg_launch_mag_params(s, A, W, (int64_t)nwide, ctx->d_widx.as<int64_t>(), 0, pf, ctx->d_pw.as<double3>());
        fsg_launch_mag_wide(s, A, W.wl, Z, zmap, (int)nwide, ctx->d_widx.as<int64_t>(), pf, pl, pr,
                            ctx->d_pw.as<double3>(), ctx->tab, mlo);
        ctx->launches += 5;
    }
    std::vector<int> ls(nwl), le(nwl);
    CK(cudaMemcpyAsync(ls.data(), ctx->d_lstart.p, sizeof(int) * nwl, cudaMemcpyDeviceToHost, s), "lstart");
    CK(cudaMemcpyAsync(le.data(), ctx->d_lstop.p, sizeof(int) * nwl, cudaMemcpyDeviceToHost, s), "lstop");
    CK(cudaStreamSynchronize(s), "lstart");
    ALLOC(ctx->d_p64, sizeof(double3) * (size_t)std::min<int64_t>(nstep, nw) * nt);
    int64_t iline1 = 1, ilineb = 0, nblocks = 0;
    int iwl1 = 1;
    for (;;) {
        int iwl2;
        if (nstep >= nw) iwl2 = nwl;
        else {
            int64_t ilo = nw + 1, ihi = 0;
            iwl2 = iwl1 - 1;
            for (int iwl = iwl1; iwl <= nwl; iwl++) {
                int64_t ilot = std::min<int64_t>(ilo, ls[iwl - 1]), ihit = std::max<int64_t>(ihi, le[iwl - 1]);
                if (ihit - ilot + 1 > nstep) break;
                ilo = ilot; ihi = ihit; iwl2 = iwl;
            }
            if (iwl2 < iwl1) {
                char m[256];
                snprintf(m, sizeof m, "line opacity segmentation: lines contributing to wavelength point #%d span more "
                         "than %lld line records; increase limitram", iwl1, (long long)nstep);
                return fail(ctx, FSG_E_SEGMENT, m);
            }
            iline1 = std::min<int64_t>(std::max<int64_t>(ilo, 1), nw);
        }
        int64_t iline2 = std::min<int64_t>(iline1 + nstep - 1, nw);
        int64_t loff = iline1 - 1;
        if (iline1 != ilineb) {
            ilineb = iline1;
            fsg_launch_mag_params(s, A, W, iline2 - loff, nullptr, loff, pf, ctx->d_p64.as<double3>());
            ctx->launches += 1;
            nblocks++;
        }
        fsg_launch_mag_accum(s, A, W.wl, Z, zmap, iwl1, iwl2, ctx->d_lstart.as<int>(), ctx->d_lstop.as<int>(), pf, pl,
                             pr, loff, ctx->d_p64.as<double3>(), ctx->tab, mlo, ctx->d_evals.as<double>());
        ctx->launches += 1;
        CK(cudaGetLastError(), "mag accumulation");
        if (iwl2 == nwl) break;
        iwl1 = iwl2 + 1;
    }
    if (pack) {
        fsg_launch_scatter_flags(s, nw, ctx->d_idx.as<int64_t>(), pf, ctx->d_flags.as<int32_t>());
        ctx->launches += 1;
    }
    double ev = 0;
    CK(cudaMemcpyAsync(&ev, ctx->d_evals.p, sizeof ev, cudaMemcpyDeviceToHost, s), "evals");
    CK(cudaEventRecord(ctx->ev[2], s), "event");
    size_t n4 = sizeof(int32_t) * n;
    if (flags) CK(cudaMemcpyAsync(flags, ctx->d_flags.p, n4, cudaMemcpyDeviceToHost, s), "flags");
    if (ileft) CK(cudaMemcpyAsync(ileft, ctx->d_ileft.p, n4, cudaMemcpyDeviceToHost, s), "ileft");
    if (iright) CK(cudaMemcpyAsync(iright, ctx->d_iright.p, n4, cudaMemcpyDeviceToHost, s), "iright");
    if (maglineopac)
        CK(cudaMemcpyAsync(maglineopac, mlo, sizeof(double) * 6 * (size_t)nwl * nt, cudaMemcpyDeviceToHost, s), "mlo");
    CK(cudaStreamSynchronize(s), "mag lineop");
    if (st) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]);
        cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]);
        st->ms_center = a; st->ms_accum = b; st->ms_total = a + b;
        st->nwide = (int64_t)nwide; st->nblocks = nblocks;
        (void)ev;                                          // the kernels' own count leaves components out
        st->line_evals = count_windows(ctx, n, ctx->d_flags.as<int32_t>(), ctx->d_ileft.as<int32_t>(),
                                       ctx->d_iright.as<int32_t>(), 1, nwl, Z.npi, Z.nsi) * nt;
    }
    return FSG_OK;
}

// ---- MagRadTranCalc (synth.f90:1904-2111) --------------------------------------------------------------
// Field projection for one disk position or ray point (synth.f90:1931-1993, 2022-2087): frames 1 and 2
// give (gamma, psi) directly (j = the angle's pair for frame 2), frame 0 projects the stellar-frame
// field with the local cosine Coslon.  g = (SPhi2, CPhi2, CPhi, S2Psi, C2Psi).
static void field_geometry(int bframe, const double *bfield, int j, double Coslon, double *g) {
    const double d2r = FSG_PI / 180.0;
    double Sphi, Spsi, Cpsi, CPhi;
    if (bframe == 1) {
        Sphi = sin(bfield[1] * d2r); Spsi = sin(bfield[2] * d2r); Cpsi = cos(bfield[2] * d2r); CPhi = cos(bfield[1] * d2r);
    } else if (bframe == 2) {
        Sphi = sin(bfield[2 * j + 1] * d2r); Spsi = sin(bfield[2 * j + 2] * d2r);
        Cpsi = cos(bfield[2 * j + 2] * d2r); CPhi = cos(bfield[2 * j + 1] * d2r);
    } else {
        double Fldmod = sqrt(bfield[0] * bfield[0] + bfield[1] * bfield[1] + bfield[2] * bfield[2]);
        if (Fldmod > 0.0) {
            double Sinlon = sqrt(1.0 - Coslon * Coslon);
            double Bx = bfield[0] * Sinlon + bfield[2] * Coslon, By = bfield[1];
            double Bz = bfield[0] * Coslon - bfield[2] * Sinlon, Bt = sqrt(Bx * Bx + By * By);
            Sphi = Bt / Fldmod; CPhi = Bz / Fldmod;
            if (Bt > 0.0) { Spsi = By / Bt; Cpsi = Bx / Bt; } else { Spsi = 0.0; Cpsi = 1.0; }
        } else { Sphi = 0.0; CPhi = 1.0; Spsi = 0.0; Cpsi = 1.0; }
    }
    g[0] = Sphi * Sphi; g[1] = CPhi * CPhi; g[2] = CPhi; g[3] = 2.0 * Spsi * Cpsi; g[4] = Cpsi * Cpsi - Spsi * Spsi;
}

// MagRadTranCalc for spherical models (synth.f90:2013-2108): continuum by LocPrfSph, Stokes vector by
// StokesPrfSph with the projection at every ray point (frame 0 follows the local radial direction).
static int mag_radtran_sph(fsg_ctx *ctx, const RayView &R, int bframe, const double *bfield, double *spz,
                           double *spc, double *sfl, double *sfc) {
    const int nmu = ctx->nmu, M = R.stride;
    const size_t gs = (size_t)nmu * M;
    std::vector<double> geo(5 * gs, 0.0);
    for (int im = 0; im < nmu; im++)
        for (int k = 0; k < ctx->h_ray_n[im]; k++) {
            double g[5];
            field_geometry(bframe, bfield, im, ctx->h_muloc[(size_t)im * M + k], g);
            for (int q = 0; q < 5; q++) geo[q * gs + (size_t)im * M + k] = g[q];
        }
    cudaStream_t s = ctx->stream;
    ALLOC(ctx->d_ray_geo, sizeof(double) * geo.size());
    CK(cudaMemcpyAsync(ctx->d_ray_geo.p, geo.data(), sizeof(double) * geo.size(), cudaMemcpyHostToDevice, s), "geo");
    AtmView A = fsg_view(ctx);
    int rc = fsg_launch_radtran_sph(s, A, ctx->d_lineopac.as<double>(), R, ctx->d_wmu.as<double>(), nullptr, spc,
                                    nullptr, sfc);
    if (rc) return cuda_fail(ctx, cudaGetLastError(), "k_radtran_sph");
    // chunks of wavelengths whose per-thread work arrays (rays of up to 2 ntau points) take at most 2 GiB
    const int chunk = fsg_stokes_chunk(M, nmu, ctx->nwl, (size_t)2 << 30);
    ALLOC(ctx->d_stkwork, fsg_stokes_work(M, nmu, chunk));
    rc = fsg_launch_stokes_sph(s, A, ctx->d_lineopac.as<double>(), ctx->d_maglineopac.as<double>(), R,
                               ctx->d_wmu.as<double>(), ctx->d_ray_geo.as<double>(), spz, sfl,
                               ctx->d_stkwork.as<double>(), chunk);
    if (rc) return cuda_fail(ctx, cudaGetLastError(), "k_stokes_sph");
    ctx->launches += sfl ? 3 : 2;
    return FSG_OK;
}


static int mag_radtran_body(fsg_ctx *ctx, int bframe, const double *bfield, int nbfield, double *spz,
                            double *spc, double *sfl, double *sfc) {
    if (!ctx) return FSG_E_ARG;
    if (!ctx->have_grid || !ctx->have_atm || !ctx->have_cont || ctx->nmu < 1)
        return fail(ctx, FSG_E_STATE, "mag_radtran: set grid, atmosphere, continuum and mu first");
    const int nmu = ctx->nmu;
    if (!bfield || bframe < 0 || bframe > 2 || (bframe == 2 ? nbfield != 2 * nmu + 1 : nbfield != 3))
        return fail(ctx, FSG_E_ARG, "mag_radtran: BFIELD needs 3 values (frames 0, 1) or 2*nmu+1 (frame 2)");
    cudaSetDevice(ctx->device);
    int rc = ensure_lineopac(ctx); if (rc) return rc;
    rc = ensure_maglineopac(ctx); if (rc) return rc;
    RayView R;
    rc = rays_prepare(ctx, &R); if (rc) return rc;
    if (R.nmu > 0) {
        size_t nsp = sizeof(double) * (size_t)ctx->nwl * nmu, nf = sizeof(double) * ctx->nwl;
        ALLOC(ctx->d_spl, 4 * nsp); ALLOC(ctx->d_spc, nsp); ALLOC(ctx->d_sfl, nf); ALLOC(ctx->d_sfc, nf);
        rc = mag_radtran_sph(ctx, R, bframe, bfield, ctx->d_spl.as<double>(), ctx->d_spc.as<double>(),
                             ctx->d_sfl.as<double>(), ctx->d_sfc.as<double>());
        if (rc) return rc;
        cudaStream_t s = ctx->stream;
        if (spz) CK(cudaMemcpyAsync(spz, ctx->d_spl.p, 4 * nsp, cudaMemcpyDeviceToHost, s), "spz");
        if (spc) CK(cudaMemcpyAsync(spc, ctx->d_spc.p, nsp, cudaMemcpyDeviceToHost, s), "spc");
        if (sfl) CK(cudaMemcpyAsync(sfl, ctx->d_sfl.p, nf, cudaMemcpyDeviceToHost, s), "sfl");
        if (sfc) CK(cudaMemcpyAsync(sfc, ctx->d_sfc.p, nf, cudaMemcpyDeviceToHost, s), "sfc");
        CK(cudaStreamSynchronize(s), "mag radtran");
        return FSG_OK;
    }
    std::vector<double> xmu(nmu), geo(5 * nmu);
    CK(cudaMemcpy(xmu.data(), ctx->d_xmu.p, sizeof(double) * nmu, cudaMemcpyDeviceToHost), "mu");
    const double d2r = FSG_PI / 180.0;
    for (int im = 0; im < nmu; im++) {
        double Sphi, Spsi, Cpsi, CPhi;
        if (bframe == 1) {
            Sphi = sin(bfield[1] * d2r); Spsi = sin(bfield[2] * d2r); Cpsi = cos(bfield[2] * d2r); CPhi = cos(bfield[1] * d2r);
        } else if (bframe == 2) {
            Sphi = sin(bfield[2 * im + 1] * d2r); Spsi = sin(bfield[2 * im + 2] * d2r);
            Cpsi = cos(bfield[2 * im + 2] * d2r); CPhi = cos(bfield[2 * im + 1] * d2r);
        } else {
            double Fldmod = sqrt(bfield[0] * bfield[0] + bfield[1] * bfield[1] + bfield[2] * bfield[2]);
            if (Fldmod > 0.0) {
                double Coslon = xmu[im], Sinlon = sqrt(1.0 - Coslon * Coslon);
                double Bx = bfield[0] * Sinlon + bfield[2] * Coslon, By = bfield[1];
                double Bz = bfield[0] * Coslon - bfield[2] * Sinlon, Bt = sqrt(Bx * Bx + By * By);
                Sphi = Bt / Fldmod; CPhi = Bz / Fldmod;
                if (Bt > 0.0) { Spsi = By / Bt; Cpsi = Bx / Bt; } else { Spsi = 0.0; Cpsi = 1.0; }
            } else { Sphi = 0.0; CPhi = 1.0; Spsi = 0.0; Cpsi = 1.0; }
        }
        geo[0 * nmu + im] = Sphi * Sphi; geo[1 * nmu + im] = CPhi * CPhi; geo[2 * nmu + im] = CPhi;
        geo[3 * nmu + im] = 2.0 * Spsi * Cpsi; geo[4 * nmu + im] = Cpsi * Cpsi - Spsi * Spsi;
    }
    cudaStream_t s = ctx->stream;
    ALLOC(ctx->d_geo, sizeof(double) * 5 * nmu);
    CK(cudaMemcpyAsync(ctx->d_geo.p, geo.data(), sizeof(double) * 5 * nmu, cudaMemcpyHostToDevice, s), "geo");
    size_t nsp = sizeof(double) * (size_t)ctx->nwl * nmu, nf = sizeof(double) * ctx->nwl;
    ALLOC(ctx->d_spl, 4 * nsp); ALLOC(ctx->d_spc, nsp); ALLOC(ctx->d_sfl, nf); ALLOC(ctx->d_sfc, nf);
    AtmView A = fsg_view(ctx);
    // continuum intensity and flux (LocPrfPP with ContOpac)
    rc = fsg_launch_radtran(s, A, ctx->d_lineopac.as<double>(), ctx->d_rhox.as<double>(), nmu, ctx->d_xmu.as<double>(),
                            ctx->d_wmu.as<double>(), nullptr, ctx->d_spc.as<double>(), nullptr, ctx->d_sfc.as<double>());
    if (rc) return cuda_fail(ctx, cudaGetLastError(), "k_radtran");
    // chunks of wavelengths whose per-thread work arrays take at most 2 GiB
    const int chunk = fsg_stokes_chunk(ctx->ntau, nmu, ctx->nwl, (size_t)2 << 30);
    ALLOC(ctx->d_stkwork, fsg_stokes_work(ctx->ntau, nmu, chunk));
    rc = fsg_launch_stokes(s, A, ctx->d_lineopac.as<double>(), ctx->d_maglineopac.as<double>(), ctx->d_rhox.as<double>(),
                           nmu, ctx->d_xmu.as<double>(), ctx->d_wmu.as<double>(), ctx->d_geo.as<double>(),
                           ctx->d_spl.as<double>(), ctx->d_sfl.as<double>(), ctx->d_stkwork.as<double>(), chunk);
    if (rc) return cuda_fail(ctx, cudaGetLastError(), "k_stokes_thr");
    ctx->launches += 2;
    if (spz) CK(cudaMemcpyAsync(spz, ctx->d_spl.p, 4 * nsp, cudaMemcpyDeviceToHost, s), "spz");
    if (spc) CK(cudaMemcpyAsync(spc, ctx->d_spc.p, nsp, cudaMemcpyDeviceToHost, s), "spc");
    if (sfl) CK(cudaMemcpyAsync(sfl, ctx->d_sfl.p, nf, cudaMemcpyDeviceToHost, s), "sfl");
    if (sfc) CK(cudaMemcpyAsync(sfc, ctx->d_sfc.p, nf, cudaMemcpyDeviceToHost, s), "sfc");
    CK(cudaStreamSynchronize(s), "mag radtran");
    return FSG_OK;
}

// ---- elemental entry points --------------------------------------------------------------------------
// ---- kernel-level entry points (XlineSetup / XlineDepth, LineOpacity1/2, MagLineOpacity1,
// AnalyticWindow, StokesPrfPP): host arrays staged in per-call device buffers ---------------------
}  // extern "C"
namespace {
struct Stage {                                      // device copies freed when the call returns
    std::vector<DBuf *> bufs;
    ~Stage() { for (DBuf *b : bufs) { b->release(); delete b; } }
    template <class T> T *put(const T *h, size_t n, cudaStream_t s, int *rc) {
        DBuf *b = new DBuf();
        bufs.push_back(b);
        if (b->ensure(sizeof(T) * std::max<size_t>(n, 1)) != FSG_OK) { *rc = FSG_E_NOMEM; return nullptr; }
        if (h && n && cudaMemcpyAsync(b->p, h, sizeof(T) * n, cudaMemcpyHostToDevice, s) != cudaSuccess)
            *rc = FSG_E_CUDA;
        return (T *)b->p;
    }
    template <class T> T *out(size_t n, int *rc) { return put<T>(nullptr, n, nullptr, rc); }
};
}  // namespace
extern "C" {

static int block_stage(fsg_ctx *ctx, Stage &S, const fsg_lineblock *b, int mag, BlockView *B, ZView *Z) {
    int rc = FSG_OK;
    cudaStream_t s = ctx->stream;
    const size_t nl = (size_t)b->nlines, nb = (size_t)b->nblock * ctx->ntau;
    B->wlcent = S.put(b->wlcent, nl, s, &rc);
    B->flags = S.put(b->flags, nl, s, &rc); B->ileft = S.put(b->ileft, nl, s, &rc);
    B->iright = S.put(b->iright, nl, s, &rc);
    B->cop = S.put(b->lincop, nb, s, &rc); B->vv = S.put(b->linvvgt, nb, s, &rc); B->av = S.put(b->linavgt, nb, s, &rc);
    if (mag) {
        int64_t np = 0, ns = 0;
        for (size_t i = 0; i < nl; i++) {
            np = std::max<int64_t>(np, b->pi_off[i] + b->npi[i]);
            ns = std::max<int64_t>(ns, b->si_off[i] + b->nsi[i]);
        }
        memset(Z, 0, sizeof *Z);
        Z->npi = S.put(b->npi, nl, s, &rc); Z->nsi = S.put(b->nsi, nl, s, &rc);
        Z->pi_off = S.put(b->pi_off, nl, s, &rc); Z->si_off = S.put(b->si_off, nl, s, &rc);
        Z->splpi = S.put(b->splpi, (size_t)np, s, &rc); Z->strpi = S.put(b->strpi, (size_t)np, s, &rc);
        Z->splsi = S.put(b->splsi, (size_t)ns, s, &rc); Z->strsi = S.put(b->strsi, (size_t)ns, s, &rc);
    }
    return rc;
}

static int check_block(fsg_ctx *ctx, const fsg_lineblock *b, int mag, const char *who) {
    if (!b || b->nlines < 0 || b->nblock < 0 || (b->nlines > 0 && (!b->wlcent || !b->flags || !b->ileft || !b->iright)) ||
        (b->nblock > 0 && (!b->lincop || !b->linvvgt || !b->linavgt)))
        return fail(ctx, FSG_E_ARG, who);
    if (mag && b->nlines > 0 && (!b->npi || !b->nsi || !b->pi_off || !b->si_off || !b->splpi || !b->strpi ||
                                 !b->splsi || !b->strsi))
        return fail(ctx, FSG_E_ARG, who);
    return FSG_OK;
}

// line ranges of the points inside the list and the block (LineOpacity1's L1..L2 - Loff)
static int check_points(fsg_ctx *ctx, const fsg_lineblock *b, int64_t npts, const int32_t *l1, const int32_t *l2,
                        const int32_t *iwl, int64_t loff, const char *who) {
    for (int64_t k = 0; k < npts; k++) {
        if (iwl[k] < 1 || iwl[k] > ctx->nwl) return fail(ctx, FSG_E_ARG, who);
        if (l1[k] > l2[k]) continue;
        if (l1[k] < 1 || l2[k] > b->nlines || l1[k] - loff < 1 || l2[k] - loff > b->nblock) return fail(ctx, FSG_E_ARG, who);
    }
    return FSG_OK;
}

int fsg_xline_setup(fsg_ctx *ctx, const fsg_lines *lines, fsg_xcoef *xc) {
    int rc = check_lines(ctx, lines, false); if (rc) return rc;      // XlineSetup reads no continuum
    if (lines->n > 0 && !xc) return fail(ctx, FSG_E_ARG, "fsg_xline_setup: output missing");
    if (lines->n == 0) return FSG_OK;
    cudaSetDevice(ctx->device);
    fsg_lines D{};
    rc = upload_lines(ctx, lines, &D); if (rc) return rc;
    Stage S;
    XCoef *dx = S.out<XCoef>((size_t)lines->n, &rc);
    if (rc) return fail(ctx, rc, "fsg_xline_setup: device buffers");
    fsg_launch_xline_setup(ctx->stream, fsg_view(ctx), make_view(&D), dx);
    ctx->launches += 1;
    CK(cudaGetLastError(), "k_xline_setup");
    CK(cudaMemcpyAsync(xc, dx, sizeof(XCoef) * (size_t)lines->n, cudaMemcpyDeviceToHost, ctx->stream), "xline setup");
    CK(cudaStreamSynchronize(ctx->stream), "xline setup");
    return FSG_OK;
}

int fsg_xline_depth(fsg_ctx *ctx, int64_t n, const fsg_xcoef *xc, double *lincop, double *linvvgt, double *linavgt) {
    if (!ctx || n < 0 || (n > 0 && (!xc || !lincop || !linvvgt || !linavgt)))
        return fail(ctx, FSG_E_ARG, "fsg_xline_depth: bad arguments");
    if (!ctx->have_atm) return fail(ctx, FSG_E_STATE, "fsg_xline_depth: set the atmosphere first");
    if (n == 0) return FSG_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    Stage S;
    int rc = FSG_OK;
    const size_t m = (size_t)n * ctx->ntau;
    const XCoef *dx = S.put((const XCoef *)xc, (size_t)n, s, &rc);
    double *c = S.out<double>(m, &rc), *v = S.out<double>(m, &rc), *a = S.out<double>(m, &rc);
    if (rc) return fail(ctx, rc, "fsg_xline_depth: device buffers");
    fsg_launch_xline_depth(s, fsg_view(ctx), n, dx, c, v, a);
    ctx->launches += 1;
    CK(cudaGetLastError(), "k_xline_depth");
    CK(cudaMemcpyAsync(lincop, c, sizeof(double) * m, cudaMemcpyDeviceToHost, s), "xline depth");
    CK(cudaMemcpyAsync(linvvgt, v, sizeof(double) * m, cudaMemcpyDeviceToHost, s), "xline depth");
    CK(cudaMemcpyAsync(linavgt, a, sizeof(double) * m, cudaMemcpyDeviceToHost, s), "xline depth");
    CK(cudaStreamSynchronize(s), "xline depth");
    return FSG_OK;
}

static int lineop1_common(fsg_ctx *ctx, const fsg_lineblock *blk, int64_t npts, const double *wl, const int32_t *l1,
                          const int32_t *l2, const int32_t *iwl, int64_t loff, double *out, int mag) {
    const char *who = mag ? "fsg_mag_lineopacity1: bad arguments" : "fsg_lineopacity1: bad arguments";
    if (!ctx) return FSG_E_ARG;
    if (npts < 0 || (npts > 0 && (!wl || !l1 || !l2 || !iwl || !out))) return fail(ctx, FSG_E_ARG, who);
    if (!ctx->have_grid || !ctx->have_atm) return fail(ctx, FSG_E_STATE, "set grid and atmosphere first");
    int rc = check_block(ctx, blk, mag, who); if (rc) return rc;
    rc = check_points(ctx, blk, npts, l1, l2, iwl, loff, who); if (rc) return rc;
    if (npts == 0) return FSG_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    Stage S;
    BlockView B; ZView Z;
    rc = block_stage(ctx, S, blk, mag, &B, &Z);
    const double *dwl = S.put(wl, (size_t)npts, s, &rc);
    const int32_t *d1 = S.put(l1, (size_t)npts, s, &rc), *d2 = S.put(l2, (size_t)npts, s, &rc);
    const int32_t *di = S.put(iwl, (size_t)npts, s, &rc);
    const size_t m = (size_t)npts * ctx->ntau * (mag ? 6 : 1);
    double *dout = S.out<double>(m, &rc);
    if (rc) return fail(ctx, rc, "lineopacity1: device buffers");
    if (mag) fsg_launch_mag_lineopacity1_pts(s, fsg_view(ctx), B, Z, npts, dwl, d1, d2, di, loff, ctx->tab, dout);
    else fsg_launch_lineopacity1_pts(s, fsg_view(ctx), B, npts, dwl, d1, d2, di, loff, ctx->tab, dout);
    ctx->launches += 1;
    CK(cudaGetLastError(), "lineopacity1");
    CK(cudaMemcpyAsync(out, dout, sizeof(double) * m, cudaMemcpyDeviceToHost, s), "lineopacity1");
    CK(cudaStreamSynchronize(s), "lineopacity1");
    return FSG_OK;
}

int fsg_lineopacity1(fsg_ctx *ctx, const fsg_lineblock *blk, int64_t npts, const double *wl, const int32_t *l1,
                     const int32_t *l2, const int32_t *iwl, int64_t loff, double *linop) {
    return lineop1_common(ctx, blk, npts, wl, l1, l2, iwl, loff, linop, 0);
}

int fsg_mag_lineopacity1(fsg_ctx *ctx, const fsg_lineblock *blk, int64_t npts, const double *wl, const int32_t *l1,
                         const int32_t *l2, const int32_t *iwl, int64_t loff, double *maglinop) {
    return lineop1_common(ctx, blk, npts, wl, l1, l2, iwl, loff, maglinop, 1);
}

int fsg_lineopacity2(fsg_ctx *ctx, const fsg_lineblock *blk, int64_t npts, const double *wl, const int32_t *iline,
                     const int32_t *iwl, const double *lincop, const double *linvvgt, const double *linavgt,
                     double *linop) {
    if (!ctx) return FSG_E_ARG;
    const char *who = "fsg_lineopacity2: bad arguments";
    if (npts < 0 || (npts > 0 && (!wl || !iline || !iwl || !lincop || !linvvgt || !linavgt || !linop)))
        return fail(ctx, FSG_E_ARG, who);
    if (!ctx->have_grid || !ctx->have_atm) return fail(ctx, FSG_E_STATE, "set grid and atmosphere first");
    int rc = check_block(ctx, blk, 0, who); if (rc) return rc;
    for (int64_t k = 0; k < npts; k++)
        if (iline[k] < 1 || iline[k] > blk->nlines || iwl[k] < 1 || iwl[k] > ctx->nwl) return fail(ctx, FSG_E_ARG, who);
    if (npts == 0) return FSG_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    Stage S;
    fsg_lineblock lb = *blk;
    lb.nblock = 0;                                  // the points carry their own parameter rows
    BlockView B; ZView Z;
    rc = block_stage(ctx, S, &lb, 0, &B, &Z);
    const size_t m = (size_t)npts * ctx->ntau;
    const double *dwl = S.put(wl, (size_t)npts, s, &rc);
    const int32_t *dl = S.put(iline, (size_t)npts, s, &rc), *di = S.put(iwl, (size_t)npts, s, &rc);
    const double *c = S.put(lincop, m, s, &rc), *v = S.put(linvvgt, m, s, &rc), *a = S.put(linavgt, m, s, &rc);
    double *dout = S.out<double>(m, &rc);
    if (rc) return fail(ctx, rc, "fsg_lineopacity2: device buffers");
    fsg_launch_lineopacity2_pts(s, fsg_view(ctx), B, npts, dwl, dl, di, c, v, a, ctx->tab, dout);
    ctx->launches += 1;
    CK(cudaGetLastError(), "k_lineopacity2_pts");
    CK(cudaMemcpyAsync(linop, dout, sizeof(double) * m, cudaMemcpyDeviceToHost, s), "lineopacity2");
    CK(cudaStreamSynchronize(s), "lineopacity2");
    return FSG_OK;
}

int fsg_analytic_window(fsg_ctx *ctx, int64_t n, const int32_t *flags, const double *lincop, const double *linvvgt,
                        const double *linavgt, const double *contopac, double *dw) {
    if (!ctx) return FSG_E_ARG;
    if (n < 0 || (n > 0 && (!flags || !lincop || !linvvgt || !linavgt || !contopac || !dw)))
        return fail(ctx, FSG_E_ARG, "fsg_analytic_window: bad arguments");
    if (!ctx->have_atm) return fail(ctx, FSG_E_STATE, "fsg_analytic_window: set the atmosphere first");
    if (n == 0) return FSG_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    Stage S;
    int rc = FSG_OK;
    const size_t m = (size_t)n * ctx->ntau;
    const int32_t *df = S.put(flags, (size_t)n, s, &rc);
    const double *c = S.put(lincop, m, s, &rc), *v = S.put(linvvgt, m, s, &rc), *a = S.put(linavgt, m, s, &rc);
    const double *co = S.put(contopac, m, s, &rc);
    double *dout = S.out<double>((size_t)n, &rc);
    if (rc) return fail(ctx, rc, "fsg_analytic_window: device buffers");
    fsg_launch_analytic_window(s, fsg_view(ctx), n, df, c, v, a, co, dout);
    ctx->launches += 1;
    CK(cudaGetLastError(), "k_analytic_window");
    CK(cudaMemcpyAsync(dw, dout, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, s), "analytic window");
    CK(cudaStreamSynchronize(s), "analytic window");
    return FSG_OK;
}

int fsg_stokes_prf_pp(fsg_ctx *ctx, int64_t npts, const int32_t *iwl, const double *src, const double *sphi2,
                      const double *cphi2, const double *cphi, const double *s2psi, const double *c2psi, double *stokes) {
    if (!ctx) return FSG_E_ARG;
    if (npts < 0 || (npts > 0 && (!iwl || !src || !sphi2 || !cphi2 || !cphi || !s2psi || !c2psi || !stokes)))
        return fail(ctx, FSG_E_ARG, "fsg_stokes_prf_pp: bad arguments");
    if (!ctx->have_grid || !ctx->have_atm || !ctx->have_cont || ctx->nmu < 1)
        return fail(ctx, FSG_E_STATE, "fsg_stokes_prf_pp: set grid, atmosphere, continuum and mu first");
    if (ctx->d_maglineopac.cap < sizeof(double) * 6 * (size_t)ctx->nwl * ctx->ntau)
        return fail(ctx, FSG_E_STATE, "fsg_stokes_prf_pp: run fsg_mag_lineop_calc first");
    for (int64_t k = 0; k < npts; k++)
        if (iwl[k] < 1 || iwl[k] > ctx->nwl) return fail(ctx, FSG_E_ARG, "fsg_stokes_prf_pp: wavelength index");
    if (npts == 0) return FSG_OK;
    cudaSetDevice(ctx->device);
    int rc = ensure_lineopac(ctx); if (rc) return rc;
    cudaStream_t s = ctx->stream;
    Stage S;
    const int nmu = ctx->nmu;
    std::vector<double> geo(5 * (size_t)nmu);
    for (int im = 0; im < nmu; im++) {
        geo[0 * nmu + im] = sphi2[im]; geo[1 * nmu + im] = cphi2[im]; geo[2 * nmu + im] = cphi[im];
        geo[3 * nmu + im] = s2psi[im]; geo[4 * nmu + im] = c2psi[im];
    }
    const double *dg = S.put(geo.data(), geo.size(), s, &rc);
    const int32_t *di = S.put(iwl, (size_t)npts, s, &rc);
    const double *dsrc = S.put(src, (size_t)npts * ctx->ntau, s, &rc);
    double *work = S.out<double>(fsg_stokes_pts_work(npts, nmu, ctx->ntau) / sizeof(double), &rc);
    double *dout = S.out<double>((size_t)npts * 4 * nmu, &rc);
    if (rc) return fail(ctx, rc, "fsg_stokes_prf_pp: device buffers");
    fsg_launch_stokes_prf_pts(s, fsg_view(ctx), ctx->d_lineopac.as<double>(), ctx->d_maglineopac.as<double>(),
                              ctx->d_rhox.as<double>(), nmu, ctx->d_xmu.as<double>(), dg, npts, di, dsrc, work, dout);
    ctx->launches += 1;
    CK(cudaGetLastError(), "k_stokes_prf_pts");
    CK(cudaMemcpyAsync(stokes, dout, sizeof(double) * (size_t)npts * 4 * nmu, cudaMemcpyDeviceToHost, s), "stokes");
    CK(cudaStreamSynchronize(s), "stokes");
    return FSG_OK;
}

int fsg_hvoigt(fsg_ctx *ctx, int64_t n, const double *a, const double *v, double *h) {
    if (!ctx || n < 0 || (n > 0 && (!a || !v || !h))) return fail(ctx, FSG_E_ARG, "fsg_hvoigt: bad arguments");
    if (n == 0) return FSG_OK;
    cudaSetDevice(ctx->device);
    size_t nb = sizeof(double) * n;
    ALLOC(ctx->d_a, nb); ALLOC(ctx->d_v, nb); ALLOC(ctx->d_h, nb);
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(ctx->d_a.p, a, nb, cudaMemcpyHostToDevice, s), "hvoigt");
    CK(cudaMemcpyAsync(ctx->d_v.p, v, nb, cudaMemcpyHostToDevice, s), "hvoigt");
    fsg_launch_hvoigt(s, n, ctx->d_a.as<double>(), ctx->d_v.as<double>(), ctx->d_h.as<double>(), ctx->tab);
    CK(cudaGetLastError(), "k_hvoigt");
    CK(cudaMemcpyAsync(h, ctx->d_h.p, nb, cudaMemcpyDeviceToHost, s), "hvoigt");
    CK(cudaStreamSynchronize(s), "hvoigt");
    return FSG_OK;
}

int fsg_fvoigt(fsg_ctx *ctx, int64_t n, const double *a, const double *v, double *h, double *l) {
    if (!ctx || n < 0 || (n > 0 && (!a || !v || !h || !l))) return fail(ctx, FSG_E_ARG, "fsg_fvoigt: bad arguments");
    if (n == 0) return FSG_OK;
    cudaSetDevice(ctx->device);
    size_t nb = sizeof(double) * n;
    ALLOC(ctx->d_a, nb); ALLOC(ctx->d_v, nb); ALLOC(ctx->d_h, nb); ALLOC(ctx->d_l, nb);
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(ctx->d_a.p, a, nb, cudaMemcpyHostToDevice, s), "fvoigt");
    CK(cudaMemcpyAsync(ctx->d_v.p, v, nb, cudaMemcpyHostToDevice, s), "fvoigt");
    fsg_launch_fvoigt(s, n, ctx->d_a.as<double>(), ctx->d_v.as<double>(), ctx->d_h.as<double>(), ctx->d_l.as<double>(), ctx->tab);
    CK(cudaGetLastError(), "k_fvoigt");
    CK(cudaMemcpyAsync(h, ctx->d_h.p, nb, cudaMemcpyDeviceToHost, s), "fvoigt");
    CK(cudaMemcpyAsync(l, ctx->d_l.p, nb, cudaMemcpyDeviceToHost, s), "fvoigt");
    CK(cudaStreamSynchronize(s), "fvoigt");
    return FSG_OK;
}

int fsg_voigt_tables(fsg_ctx *ctx, float *vgt, float *fvt) {
    if (!ctx) return FSG_E_ARG;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    if (vgt) CK(cudaMemcpyAsync(vgt, ctx->tab.vtab, sizeof(float) * FSG_NA1 * FSG_NV1, cudaMemcpyDeviceToHost, s), "tables");
    if (fvt) CK(cudaMemcpyAsync(fvt, ctx->tab.fvtab, sizeof(float2) * FSG_NA1 * FSG_NV1, cudaMemcpyDeviceToHost, s), "tables");
    CK(cudaStreamSynchronize(s), "tables");
    return FSG_OK;
}

int fsg_locprf_pp(fsg_ctx *ctx, int nprof, int nmu, const double *xmu, int ntau, const double *xki,
                  const double *src, const double *rhox, double *ploc) {
    if (!ctx || nprof < 0 || nmu < 1 || ntau < 3 || !xmu || !xki || !src || !rhox || !ploc)
        return fail(ctx, FSG_E_ARG, "fsg_locprf_pp: bad arguments");
    if (nprof == 0) return FSG_OK;
    cudaSetDevice(ctx->device);
    size_t np = (size_t)nprof * ntau * sizeof(double);
    DBuf bx, bs, br, bm, bp, bw;
    int ok = bx.ensure(np) | bs.ensure(np) | br.ensure(sizeof(double) * ntau) | bm.ensure(sizeof(double) * nmu) |
             bp.ensure(sizeof(double) * (size_t)nprof * nmu) | bw.ensure(3 * np);
    int rc = FSG_OK;
    cudaStream_t s = ctx->stream;
    if (ok != FSG_OK) rc = fail(ctx, FSG_E_NOMEM, "fsg_locprf_pp: allocation failed");
    else if (cudaMemcpyAsync(bx.p, xki, np, cudaMemcpyHostToDevice, s) != cudaSuccess ||
             cudaMemcpyAsync(bs.p, src, np, cudaMemcpyHostToDevice, s) != cudaSuccess ||
             cudaMemcpyAsync(br.p, rhox, sizeof(double) * ntau, cudaMemcpyHostToDevice, s) != cudaSuccess ||
             cudaMemcpyAsync(bm.p, xmu, sizeof(double) * nmu, cudaMemcpyHostToDevice, s) != cudaSuccess) rc = FSG_E_CUDA;
    if (rc == FSG_OK) {
        fsg_launch_locprf(s, nprof, nmu, bm.as<double>(), ntau, bx.as<double>(), bs.as<double>(), br.as<double>(),
                          bp.as<double>(), bw.as<double>());
        if (cudaMemcpyAsync(ploc, bp.p, sizeof(double) * (size_t)nprof * nmu, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) rc = cuda_fail(ctx, cudaGetLastError(), "locprf");
    }
    bx.release(); bs.release(); br.release(); bm.release(); bp.release(); bw.release();
    return rc;
}

// ---- quadrature and Zeeman patterns (host set-up routines) -------------------------------------------
static void legendre_p(int N, double Z, double *Pn, double *Pn1, double *Pn2) {
    *Pn1 = 0.0; *Pn = 1.0; *Pn2 = 0.0;
    for (int j = 1; j <= N; j++) { *Pn2 = *Pn1; *Pn1 = *Pn; *Pn = ((2.0 * j - 1.0) * Z * *Pn1 - (j - 1.0) * *Pn2) / j; }
}

static void gauss_mu(int quad, int N, double *X, double *W) {
    double Z, Dz, Pn, Pn1, Pn2, F, Df;
    if (quad == 1) {
        for (int i = 1; i <= (N + 1) / 2; i++) {
            Z = cos(FSG_PI * (i - 0.25) / (N + 0.5));
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
            Z = cos(2.0 * FSG_PI * i / (2.0 * N - 1.0));
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

int fsg_mu_quadrature(int quad, int N, double *X, double *W, double *R, int setnodes) {
    if (N < 1 || N > 64 || !X || !W || !R) return FSG_E_ARG;
    if (N == 1) { if (setnodes) X[0] = 1.0; W[0] = 1.0; R[0] = 0.0; R[1] = 1.0; return FSG_OK; }
    if (quad == 0) {
        double Rmu[64];
        if (setnodes) for (int i = 1; i <= N; i++) X[i - 1] = sqrt(fmax(0.0, 1.0 - ((double)i - 0.5) / (double)N));
        for (int i = 0; i < N; i++) Rmu[i] = sqrt(1.0 - X[i] * X[i]);
        R[0] = 0.0;
        for (int i = 2; i <= N; i++) R[i - 1] = sqrt(0.5 * (Rmu[i - 2] * Rmu[i - 2] + Rmu[i - 1] * Rmu[i - 1]));
        R[N] = 1.0;
        for (int i = 1; i <= N; i++) W[i - 1] = R[i] * R[i] - R[i - 1] * R[i - 1];
        return FSG_OK;
    }
    if (quad != 1 && quad != 2) return FSG_E_ARG;
    double Xg[64], Wg[64];
    gauss_mu(quad, N, Xg, Wg);
    if (setnodes) for (int i = 0; i < N; i++) X[i] = Xg[i];
    for (int i = 0; i < N; i++) W[i] = 2.0 * Wg[i] * Xg[i];
    R[0] = 0.0;
    for (int i = 1; i <= N - 1; i++) R[i] = sqrt(R[i - 1] * R[i - 1] + W[i - 1]);
    R[N] = 1.0;
    return FSG_OK;
}

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

int fsg_zeeman_pattern(float jlo, float jup, float glo, float gup, int32_t *npi, float *spi, float *rpi,
                       int32_t *nsig, float *ssig, float *rsig) {
    if (!npi || !spi || !rpi || !nsig || !ssig || !rsig || jup < 0 || jlo < 0 || jup > 30 || fabsf(jup - jlo) > 1.0f)
        return FSG_E_ARG;
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
    return FSG_OK;
}


// ---- disk integration with broadening (convol.f90:67-300) ------------------------------------------
// SemiArea (utils.f90:1435-1445): area under the semicircle of radius R from -R to V
static double semi_area(double R, double V) {
    if (R <= 0.0) return 0.0;
    double X = std::max(-R, std::min(R, V));
    return 0.5 * (X * std::sqrt(std::max(0.0, (R - X) * (R + X))) + R * R * std::asin(X / R));
}

// Gaussian taps exp(max(-20, -(i - j - 1)^2 / (2 sig^2))), i = 1..2j+1, normalised (convol.f90:186-196, 266-275)
static std::vector<double> gauss_taps(double sig, int j) {
    std::vector<double> k(2 * j + 1);
    double norm = 0.0;
    for (int i = 1; i <= 2 * j + 1; i++) {
        double arg = std::max(-20.0, -0.5 * ((i - j - 1) / sig) * ((i - j - 1) / sig));
        k[i - 1] = std::exp(arg);
        norm = norm + k[i - 1];
    }
    for (auto &v : k) v = v / norm;
    return k;
}

int fsg_disk_integ_conv_dev(fsg_ctx *ctx, const double *radii, double vsini, double vmacro, double vgau,
                            const double *d_spl, const double *d_spc, double *d_sfl, double *d_sfc) {
    if (!ctx || !radii || !d_spl || !d_spc || !d_sfl || !d_sfc || vsini < 0 || vmacro < 0 || vgau < 0)
        return fail(ctx, FSG_E_ARG, "fsg_disk_integ_conv_dev: bad arguments");
    if (!ctx->have_grid || ctx->nmu < 1) return fail(ctx, FSG_E_STATE, "fsg_disk_integ_conv_dev: set grid and mu first");
    cudaSetDevice(ctx->device);
    const int nwl = ctx->nwl, nmu = ctx->nmu;
    std::vector<double> xmu(nmu), wmu(nmu);
    CK(cudaMemcpy(xmu.data(), ctx->d_xmu.p, sizeof(double) * nmu, cudaMemcpyDeviceToHost), "mu");
    CK(cudaMemcpy(wmu.data(), ctx->d_wmu.p, sizeof(double) * nmu, cudaMemcpyDeviceToHost), "mu");
    const double dv = ctx->wmode == 0 ? 2.0 * ctx->dstep / (ctx->wfirst + ctx->wlast) * FSG_VC : ctx->dstep;
    const double sigma = vmacro / dv / std::sqrt(2.0);
    const int nmk = std::max(3, std::min((int)(10.0 * sigma), (int)((nwl - 3) / 2)));
    const int nm = 2 * nmk + 1, nrk_max = 2 * (int)(vsini * std::max(1.0, radii[nmu]) / dv) + 3;
    ALLOC(ctx->d_cbuf, sizeof(double) * 4 * (size_t)nwl);
    ALLOC(ctx->d_ctaps, sizeof(double) * (size_t)(nmu * (nrk_max + nm) + 2 * nm + 8));
    double *tL = ctx->d_cbuf.as<double>(), *tC = tL + nwl, *uL = tC + nwl, *uC = uL + nwl;
    cudaStream_t s = ctx->stream;
    CK(cudaMemsetAsync(d_sfl, 0, sizeof(double) * nwl, s), "flux reset");
    CK(cudaMemsetAsync(d_sfc, 0, sizeof(double) * nwl, s), "flux reset");
    // all taps of all annuli in one upload: [rotation | macroturbulence] per annulus
    std::vector<double> taps;
    std::vector<int> roff(nmu), rn(nmu, 0), moff(nmu), mn(nmu, 0);
    for (int im = 0; im < nmu; im++) {
        if (vsini > 0.0) {
            const double R1 = vsini * radii[im], R2 = vsini * radii[im + 1];
            const int nrk = 2 * (int)(R2 / dv) + 3;
            std::vector<double> rk(nrk);
            double norm = 0.0;
            for (int i = 1; i <= nrk; i++) {
                const double V = std::fabs(dv * (i - 1 - (nrk - 1) / 2));
                rk[i - 1] = semi_area(R2, V + 0.5 * dv) - semi_area(R2, V - 0.5 * dv) - semi_area(R1, V + 0.5 * dv) +
                            semi_area(R1, V - 0.5 * dv);
                norm = norm + rk[i - 1];
            }
            if (R2 > 0.5 * dv) {                      // otherwise every velocity falls in the central pixel
                roff[im] = (int)taps.size(); rn[im] = nrk;
                for (double v : rk) taps.push_back(v / norm);
            }
        }
        if (vmacro > 0.0) {
            const double sigr = sigma * xmu[im], sigt = sigma * std::sqrt(1.0 - xmu[im] * xmu[im]);
            std::vector<double> mr(nm, 0.0), mt(nm, 0.0);
            if (sigr > 0.0) mr = gauss_taps(sigr, nmk); else mr[nmk] = 1.0;
            if (sigt > 0.0) mt = gauss_taps(sigt, nmk); else mt[nmk] = 1.0;
            moff[im] = (int)taps.size(); mn[im] = nm;
            for (int i = 0; i < nm; i++) taps.push_back(0.5 * mr[i] + 0.5 * mt[i]);
        }
    }
    const int unit = (int)taps.size();
    taps.push_back(1.0);
    int goff = 0, gn = 0;
    if (vgau > 0.0) {
        double fwhm = vgau > 1000.0 ? FSG_VC / vgau : vgau;
        double sp = ctx->wmode == 0 ? fwhm * (ctx->wfirst + ctx->wlast) / FSG_VC / 2.0 / ctx->dstep : fwhm / ctx->dstep;
        double sig = sp / (2.0 * std::sqrt(2.0 * std::log(2.0)));
        int j = std::max(3, std::min((int)(10.0 * sig), (int)((nwl - 3.0) / 2.0)));
        std::vector<double> gk = gauss_taps(sig, j);
        goff = (int)taps.size(); gn = 2 * j + 1;
        for (double v : gk) taps.push_back(v);
    }
    ALLOC(ctx->d_ctaps, sizeof(double) * taps.size());
    CK(cudaMemcpyAsync(ctx->d_ctaps.p, taps.data(), sizeof(double) * taps.size(), cudaMemcpyHostToDevice, s), "taps");
    const double *dk = ctx->d_ctaps.as<double>();
    for (int im = 0; im < nmu; im++) {
        // SiL, SiC: the annulus intensities (stride nmu), rotation, macroturbulence, then the flux sum
        const double *iL = d_spl + im, *iC = d_spc + im;
        int st = nmu;
        if (rn[im]) {
            fsg_launch_conv(s, nwl, iL, st, dk + roff[im], rn[im], tL, nullptr, 0.0);
            fsg_launch_conv(s, nwl, iC, st, dk + roff[im], rn[im], tC, nullptr, 0.0);
            iL = tL; iC = tC; st = 1;
        }
        if (mn[im]) {
            double *oL = (iL == tL) ? uL : tL, *oC = (iC == tC) ? uC : tC;
            fsg_launch_conv(s, nwl, iL, st, dk + moff[im], mn[im], oL, nullptr, 0.0);
            fsg_launch_conv(s, nwl, iC, st, dk + moff[im], mn[im], oC, nullptr, 0.0);
            iL = oL; iC = oC; st = 1;
        }
        // SfL = SfL + SiL Wmu (convol.f90:230-231)
        fsg_launch_conv(s, nwl, iL, st, dk + unit, 1, d_sfl, d_sfl, wmu[im]);
        fsg_launch_conv(s, nwl, iC, st, dk + unit, 1, d_sfc, d_sfc, wmu[im]);
        ctx->launches += 2 + (rn[im] ? 2 : 0) + (mn[im] ? 2 : 0);
    }
    if (gn) {                                           // ConvolGau of the flux (convol.f90:236-240)
        CK(cudaMemcpyAsync(tL, d_sfl, sizeof(double) * nwl, cudaMemcpyDeviceToDevice, s), "gau");
        CK(cudaMemcpyAsync(tC, d_sfc, sizeof(double) * nwl, cudaMemcpyDeviceToDevice, s), "gau");
        fsg_launch_conv(s, nwl, tL, 1, dk + goff, gn, d_sfl, nullptr, 0.0);
        fsg_launch_conv(s, nwl, tC, 1, dk + goff, gn, d_sfc, nullptr, 0.0);
        ctx->launches += 2;
    }
    CK(cudaGetLastError(), "disk integration");
    CK(cudaStreamSynchronize(s), "disk integration");
    return FSG_OK;
}

int fsg_disk_integ_conv(fsg_ctx *ctx, const double *radii, double vsini, double vmacro, double vgau, double *sfl,
                        double *sfc) {
    if (!ctx || !sfl || !sfc) return fail(ctx, FSG_E_ARG, "fsg_disk_integ_conv: null output");
    cudaSetDevice(ctx->device);
    size_t nsp = sizeof(double) * (size_t)ctx->nwl * std::max(ctx->nmu, 1), nf = sizeof(double) * ctx->nwl;
    ALLOC(ctx->d_spl, nsp); ALLOC(ctx->d_spc, nsp); ALLOC(ctx->d_sfl, nf); ALLOC(ctx->d_sfc, nf);
    int rc = radtran_dev(ctx, ctx->d_spl.as<double>(), ctx->d_spc.as<double>(), nullptr, nullptr);
    if (rc) return rc;
    rc = fsg_disk_integ_conv_dev(ctx, radii, vsini, vmacro, vgau, ctx->d_spl.as<double>(), ctx->d_spc.as<double>(),
                                 ctx->d_sfl.as<double>(), ctx->d_sfc.as<double>());
    if (rc) return rc;
    CK(cudaMemcpy(sfl, ctx->d_sfl.p, nf, cudaMemcpyDeviceToHost), "flux");
    CK(cudaMemcpy(sfc, ctx->d_sfc.p, nf, cudaMemcpyDeviceToHost), "flux");
    return FSG_OK;
}

// ---- derivatives of the flux (adjoint of RadTranCalc + DiskInteg and of the line opacity) --------
int fsg_set_fractionpf(fsg_ctx *ctx, const float *fractionpf) {
    if (!ctx || !fractionpf) return FSG_E_ARG;
    if (!ctx->have_atm) return fail(ctx, FSG_E_STATE, "fsg_set_fractionpf: set the atmosphere first");
    const int nt = ctx->ntau, ns = ctx->nspc;
    std::vector<float> fpf((size_t)ns * nt);
    for (int t = 0; t < nt; t++) for (int k = 0; k < ns; k++) fpf[(size_t)k * nt + t] = fractionpf[(size_t)t * ns + k];
    cudaSetDevice(ctx->device);
    CK(cudaMemcpyAsync(ctx->d_fpf.p, fpf.data(), sizeof(float) * fpf.size(), cudaMemcpyHostToDevice, ctx->stream),
       "fractionpf upload");
    CK(cudaStreamSynchronize(ctx->stream), "fractionpf upload");
    return FSG_OK;
}

int fsg_set_fault(fsg_ctx *ctx, int kind, double value) {
    if (!ctx) return FSG_E_ARG;
    switch (kind) {
        case FSG_FAULT_NONE:
            ctx->fault_alloc = 0; ctx->fault_extra_tx = 0; ctx->fault_wait_ns = WAIT_NS;
            return FSG_OK;
        case FSG_FAULT_ALLOC_LIMIT:
            if (!(value >= 1.0)) return fail(ctx, FSG_E_ARG, "fsg_set_fault: allocation cap >= 1 byte");
            ctx->fault_alloc = (size_t)value;
            return FSG_OK;
        case FSG_FAULT_COPY_TIMEOUT:
            if (!(value >= 0.01 && value <= 1000.0)) return fail(ctx, FSG_E_ARG, "fsg_set_fault: wait bound 0.01-1000 ms");
            ctx->fault_extra_tx = 16;
            ctx->fault_wait_ns = (unsigned long long)(value * 1e6);
            return FSG_OK;
        default:
            return fail(ctx, FSG_E_ARG, "fsg_set_fault: unknown kind");
    }
}

int fsg_set_vmicro(fsg_ctx *ctx, double vmicro) {
    if (!ctx || !(vmicro >= 0.0)) return fail(ctx, FSG_E_ARG, "fsg_set_vmicro: vmicro >= 0");
    ctx->cfg.vmicro = vmicro;
    return FSG_OK;
}

static int adjoint_common(fsg_ctx *ctx, const fsg_lines *d_lines, const int32_t *fl, const int32_t *il,
                          const int32_t *ir, int i0, int i1, const double *d_gflux, double *d_gkappa, double *d_glin,
                          double *d_gvmic);

int fsg_adjoint_dev(fsg_ctx *ctx, const fsg_lines *d_lines, const double *d_gflux, double *d_gkappa, double *d_glin,
                    double *d_gvmic) {
    int rc = check_lines(ctx, d_lines); if (rc) return rc;
    if (ctx->d_flags.cap < sizeof(int32_t) * (size_t)d_lines->n)
        return fail(ctx, FSG_E_STATE, "fsg_adjoint_dev: run fsg_lineop_calc(_dev) on this list first");
    return adjoint_common(ctx, d_lines, ctx->d_flags.as<int32_t>(), ctx->d_ileft.as<int32_t>(),
                          ctx->d_iright.as<int32_t>(), 1, ctx->nwl, d_gflux, d_gkappa, d_glin, d_gvmic);
}

int fsg_adjoint_range_dev(fsg_ctx *ctx, const fsg_lines *d_lines, const int32_t *d_flags, const int32_t *d_ileft,
                          const int32_t *d_iright, int i0, int i1, const double *d_gflux, double *d_gkappa,
                          double *d_glin, double *d_gvmic) {
    int rc = check_lines(ctx, d_lines); if (rc) return rc;
    if (i0 < 1 || i1 > ctx->nwl || i0 > i1) return fail(ctx, FSG_E_ARG, "fsg_adjoint_range_dev: need 1 <= i0 <= i1 <= nwl");
    if (d_lines->n > 0 && (!d_flags || !d_ileft || !d_iright))
        return fail(ctx, FSG_E_ARG, "fsg_adjoint_range_dev: window arrays missing");
    return adjoint_common(ctx, d_lines, d_flags, d_ileft, d_iright, i0, i1, d_gflux, d_gkappa, d_glin, d_gvmic);
}

static int adjoint_common(fsg_ctx *ctx, const fsg_lines *d_lines, const int32_t *fl, const int32_t *il,
                          const int32_t *ir, int i0, int i1, const double *d_gflux, double *d_gkappa, double *d_glin,
                          double *d_gvmic) {
    int rc;
    if (ctx->nmu < 1) return fail(ctx, FSG_E_STATE, "fsg_adjoint_dev: set mu first");
    if (!d_gflux || !d_glin || !d_gvmic) return fail(ctx, FSG_E_ARG, "fsg_adjoint_dev: null argument");
    cudaSetDevice(ctx->device);
    rc = ensure_lineopac(ctx); if (rc) return rc;
    const size_t ng = sizeof(double) * (size_t)ctx->nwl * ctx->ntau;
    if (!d_gkappa) { ALLOC(ctx->d_gkappa, ng); d_gkappa = ctx->d_gkappa.as<double>(); }
    RayView rays;                                      // spherical models: the rays of LocPrfSph
    rc = rays_prepare(ctx, &rays); if (rc) return rc;
    ALLOC(ctx->d_adjwork, fsg_adjoint_work(ctx->nwl, ctx->ntau, d_lines->n, rays.nmu > 0));
    rc = fsg_launch_adjoint(ctx->stream, fsg_view(ctx), make_view(d_lines), ctx->tab, ctx->d_lineopac.as<double>(),
                            ctx->d_rhox.as<double>(), ctx->nmu, ctx->d_xmu.as<double>(), ctx->d_wmu.as<double>(),
                            rays, fl, il, ir, d_gflux, d_gkappa, ctx->d_adjwork.as<double>(), ctx->cfg.vmicro, d_glin,
                            d_gvmic, i0, i1);
    ctx->launches += 2;
    if (rc) return cuda_fail(ctx, cudaGetLastError(), "adjoint");
    CK(cudaStreamSynchronize(ctx->stream), "adjoint");
    return FSG_OK;
}

// ================================================================================================
// Batched synthesis: many atmospheres (each an fsg_ctx with grid, atmosphere, continuum and mu
// set), one shared line list.  Per atmosphere: central pass of the lines in its span (plus a
// margin), their records in window-width-class order (block refill), tile ranges per class; then
// per group of atmospheres of like depth count and per class, a persistent wing-pass launch and a
// persistent core-pass launch take (atmosphere, tile) items from device work queues; then the formal
// solver and flux of each atmosphere.  The whole sequence has no host synchronisation and is captured
// once as a CUDA graph; later runs replay it.  The wide classes' tile width and the CTA counts of
// the persistent launches are chosen by timing the candidates on the first run (fsg_batch_tune).
// ================================================================================================
static thread_local std::string g_batch_err;        // failure of the last fsg_batch_create on this thread

struct BAtm {
    fsg_ctx *ctx = nullptr;
    int64_t c0 = 0, cn = 0;                    // candidate lines [c0, c0 + cn) of the shared list
    int ncls = 1;                              // window-width classes of its record order
    DBuf flags, il, ir, wing, core, hdr, wtlo, wthi, ctlo, cthi, span, sfl, sfc, order, ccnt, coff, ctot;
};

struct fsg_batch {
    fsg_ctx *own = nullptr;                    // stream, shared list, error text
    std::vector<BAtm> atm;
    fsg_lines dlines{};
    int ntau_max = 0;
    // persistent launches (wing: lw, core: lc): a launch's jobs (one per atmosphere, so no two CTAs of
    // it update the same LineOpac tile) at j0 in its pass's job array, its queue prefix sums (starting
    // at 0) at t0 in the pass's tile0 array; P wavelengths per lane (wing)
    struct Launch { int ntau_max, P, j0, nj, t0; };
    std::vector<Launch> lw, lc;
    DBuf jobs_w, jobs_c, tile0_w, tile0_c, queue, err, nk, evals;
    fsg_batch_tuning tune{};
    int tuned = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double line_evals = 0.0;
    // ev[0..2]: around the wing and core launches; ev[3], ev[4]: around a replay; ev[5..7]: the
    // replay's stage boundaries (before the central pass, after the core launches, after the solver)
    cudaEvent_t ev[8] = {};
    // per-atmosphere stages run round-robin on these streams, forked from and joined to the batch's
    // stream (inside a capture they become parallel branches of the graph)
    static const int NAUX = 8;
    cudaStream_t aux[NAUX] = {};
    cudaEvent_t fork = nullptr, join[NAUX] = {};
};

static LineView batch_view(const fsg_batch *b, const BAtm &a) {
    fsg_lines D = b->dlines;
    D.n = a.cn;
    D.wl += a.c0; D.elo += a.c0; D.gf += a.c0; D.grad += a.c0; D.gqst += a.c0; D.gvdw += a.c0; D.spc += a.c0;
    if (D.ismol) D.ismol += a.c0;
    if (D.ihe) D.ihe += a.c0;
    return make_view(&D);
}

// Wing tiles: 64 wavelengths for the two narrowest window classes (windows up to 512), 32 * P for
// the others; core tiles: 32 wavelengths.  Tile arrays hold ncls rows of tstride entries.
static const int BATCH_NARROW = 1;             // classes 0 .. BATCH_NARROW take the narrow tiles
static int batch_wing_stride(const fsg_ctx *c) { return (c->nwl + 63) / 64; }
static int batch_core_stride(const fsg_ctx *c) { return (c->nwl + 31) / 32; }

static void batch_fork(fsg_batch *b, cudaStream_t s) {
    cudaEventRecord(b->fork, s);
    for (int k = 0; k < fsg_batch::NAUX; k++) cudaStreamWaitEvent(b->aux[k], b->fork, 0);
}
static void batch_join(fsg_batch *b, cudaStream_t s) {
    for (int k = 0; k < fsg_batch::NAUX; k++) {
        cudaEventRecord(b->join[k], b->aux[k]);
        cudaStreamWaitEvent(s, b->join[k], 0);
    }
}

// the per-atmosphere stages up to the tile ranges: central pass, class order, records in that order,
// tile ranges per class (wide-class wing tiles of P wavelengths per lane); atmospheres in parallel on
// the auxiliary streams
static int batch_prepare(fsg_batch *b, int P) {
    fsg_ctx *ctx = b->own;
    batch_fork(b, ctx->stream);
    int k = 0;
    for (auto &a : b->atm) {
        if (a.cn == 0) continue;
        const cudaStream_t s = b->aux[k++ % fsg_batch::NAUX];
        fsg_ctx *c = a.ctx;
        AtmView A = fsg_view(c);
        LineView LV = batch_view(b, a);
        fsg_launch_center(s, A, LV, c->tab, a.flags.as<int32_t>(), a.il.as<int32_t>(), a.ir.as<int32_t>(),
                          b->nk.as<unsigned long long>());
        if (fsg_launch_bclass_order(s, a.cn, a.flags.as<int32_t>(), a.il.as<int32_t>(), a.ir.as<int32_t>(), a.ncls,
                                    a.ccnt.as<int>(), a.coff.as<int64_t>(), a.ctot.as<int64_t>(), a.order.as<int64_t>()))
        {
            const cudaError_t e = cudaGetLastError();
            batch_join(b, ctx->stream);                // the forked streams rejoin on every path
            return cuda_fail(ctx, e, "batch class order");
        }
        fsg_launch_params_fast(s, A, LV, a.order.as<int64_t>(), 0, 1, a.cn, a.flags.as<int32_t>(), a.il.as<int32_t>(),
                               a.ir.as<int32_t>(), c->tab, a.wing.as<WingRec>(), a.core.as<CoreRec>(),
                               a.hdr.as<LineHdr>());
        if (fsg_launch_btile_span(s, 0, a.cn, a.hdr.as<LineHdr>(), a.coff.as<int64_t>(), a.ncls, BATCH_NARROW, 64,
                                  32 * P, c->nwl, batch_wing_stride(c), a.wtlo.as<int>(), a.wthi.as<int>(), a.span.p,
                                  a.span.cap) ||
            fsg_launch_btile_span(s, 1, a.cn, a.hdr.as<LineHdr>(), a.coff.as<int64_t>(), a.ncls, a.ncls, 32, 32,
                                  c->nwl, batch_core_stride(c), a.ctlo.as<int>(), a.cthi.as<int>(), a.span.p,
                                  a.span.cap))
        {
            const cudaError_t e = cudaGetLastError();
            batch_join(b, ctx->stream);
            return cuda_fail(ctx, e, "batch tile ranges");
        }
    }
    batch_join(b, ctx->stream);
    CK(cudaGetLastError(), "batch prepare");
    return FSG_OK;
}

// Job tables and queue prefix sums (host, then uploaded).  Atmospheres are grouped by depth count
// (buckets of 8 depths), so a persistent launch is shaped for its own group's deepest member and few
// warps idle.  Per group three launches, each with one job per atmosphere (so no two CTAs of a launch
// update the same LineOpac tile): the wing pass over the narrow classes (64-wavelength tiles), the
// wing pass over the wide ones (32 P), the core pass over all; a job's tile takes its classes' lines
// in turn into one sum.
static int batch_jobs(fsg_batch *b, int P) {
    fsg_ctx *ctx = b->own;
    std::vector<WingJob> jw; std::vector<CoreJob> jc;
    std::vector<int> tw, tc;
    b->lw.clear(); b->lc.clear();
    for (int bucket = 0; bucket * 8 < 128; bucket++) {
        int ntmax = 0;
        for (auto &a : b->atm)
            if (a.cn && (a.ctx->ntau - 1) / 8 == bucket) ntmax = std::max(ntmax, a.ctx->ntau);
        if (!ntmax) continue;
        for (int kind = 0; kind < 3; kind++) {             // narrow wing, wide wing, core
            const int Pk = kind == 0 ? 2 : P;
            std::vector<int> &t0 = kind < 2 ? tw : tc;
            fsg_batch::Launch L{ ntmax, Pk, (int)(kind < 2 ? jw.size() : jc.size()), 0, (int)t0.size() };
            t0.push_back(0);
            for (auto &a : b->atm) {
                fsg_ctx *c = a.ctx;
                if (a.cn == 0 || (c->ntau - 1) / 8 != bucket) continue;
                const int c0 = kind == 1 ? BATCH_NARROW + 1 : 0;
                const int nseg = kind == 0 ? std::min(a.ncls, BATCH_NARROW + 1) : kind == 1 ? a.ncls - c0 : a.ncls;
                if (nseg <= 0) continue;
                const int ws = batch_wing_stride(c), cs = batch_core_stride(c);
                if (kind < 2) {
                    jw.push_back(WingJob{ c->ntau, c->nwl, c->d_wave.as<double>(), a.hdr.as<LineHdr>(),
                                          a.wing.as<WingRec>(), a.wtlo.as<int>() + (size_t)c0 * ws,
                                          a.wthi.as<int>() + (size_t)c0 * ws, c->d_lineopac.as<double>(), 0u, WAIT_NS,
                                          nseg, ws });
                    t0.push_back(t0.back() + (c->nwl + 32 * Pk - 1) / (32 * Pk));
                } else {
                    jc.push_back(CoreJob{ c->ntau, c->nwl, c->d_wave.as<double>(), a.hdr.as<LineHdr>(),
                                          a.wing.as<WingRec>(), a.core.as<CoreRec>(), a.ctlo.as<int>(), a.cthi.as<int>(),
                                          c->d_lineopac.as<double>(), b->evals.as<unsigned long long>(), 0u, WAIT_NS,
                                          nseg, cs });
                    t0.push_back(t0.back() + (c->nwl + 31) / 32);
                }
                L.nj++;
            }
            if (L.nj) (kind < 2 ? b->lw : b->lc).push_back(L);
        }
    }
    ALLOC(b->jobs_w, sizeof(WingJob) * std::max<size_t>(jw.size(), 1));
    ALLOC(b->jobs_c, sizeof(CoreJob) * std::max<size_t>(jc.size(), 1));
    ALLOC(b->tile0_w, sizeof(int) * std::max<size_t>(tw.size(), 1));
    ALLOC(b->tile0_c, sizeof(int) * std::max<size_t>(tc.size(), 1));
    ALLOC(b->queue, sizeof(unsigned) * std::max<size_t>(b->lw.size() + b->lc.size(), 1));
    cudaStream_t s = ctx->stream;
    auto up = [&](DBuf &d, const void *h, size_t nb) {
        return nb ? cudaMemcpyAsync(d.p, h, nb, cudaMemcpyHostToDevice, s) : cudaSuccess;
    };
    CK(up(b->jobs_w, jw.data(), sizeof(WingJob) * jw.size()), "jobs");
    CK(up(b->jobs_c, jc.data(), sizeof(CoreJob) * jc.size()), "jobs");
    CK(up(b->tile0_w, tw.data(), sizeof(int) * tw.size()), "jobs");
    CK(up(b->tile0_c, tc.data(), sizeof(int) * tc.size()), "jobs");
    CK(cudaStreamSynchronize(s), "jobs");
    return FSG_OK;
}

// an event record; inside a stream capture it becomes an event-record node of the graph (timed
// replays), which only the external flag gives, and that flag is refused outside a capture
static void batch_mark(cudaEvent_t e, cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cs);
    if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
    else cudaEventRecord(e, s);
}

// accumulation (zeroed LineOpac, the persistent launches), then solver and flux per atmosphere;
// ev: optional events around the wing and core launches (ev[0..2]) and after the solver (ev[7])
static int batch_accumulate_solve(fsg_batch *b, const fsg_batch_tuning &t, cudaEvent_t *ev) {
    fsg_ctx *ctx = b->own;
    cudaStream_t s = ctx->stream;
    for (auto &a : b->atm) {
        fsg_ctx *c = a.ctx;
        CK(cudaMemsetAsync(c->d_lineopac.p, 0, sizeof(double) * (size_t)c->nwl * c->ntau, s), "batch reset");
    }
    const size_t nw = b->lw.size(), nc = b->lc.size();
    CK(cudaMemsetAsync(b->queue.p, 0, sizeof(unsigned) * std::max<size_t>(nw + nc, 1), s), "queue reset");
    CK(cudaMemsetAsync(b->evals.p, 0, sizeof(unsigned long long), s), "count reset");
    unsigned *q = b->queue.as<unsigned>();
    // the wing launches (each read-modify-writes its atmospheres' LineOpac tiles), then the core ones
    if (ev) batch_mark(ev[0], s);
    for (size_t i = 0; i < nw; i++) {
        const fsg_batch::Launch &L = b->lw[i];
        if (fsg_launch_accum_batch(s, L.P, L.ntau_max, b->jobs_w.as<WingJob>() + L.j0, b->tile0_w.as<int>() + L.t0,
                                   L.nj, t.wing_ctas, q + i, b->err.as<int>()))
            return cuda_fail(ctx, cudaGetLastError(), "k_accum_batch");
    }
    if (ev) batch_mark(ev[1], s);
    for (size_t i = 0; i < nc; i++) {
        const fsg_batch::Launch &L = b->lc[i];
        if (fsg_launch_core_batch(s, L.ntau_max, b->jobs_c.as<CoreJob>() + L.j0, b->tile0_c.as<int>() + L.t0, L.nj,
                                  t.core_ctas, b->atm[0].ctx->tab.vtab4, q + nw + i, b->err.as<int>()))
            return cuda_fail(ctx, cudaGetLastError(), "k_core_batch");
    }
    if (ev) batch_mark(ev[2], s);
    batch_fork(b, s);
    int k = 0;
    for (auto &a : b->atm) {
        fsg_ctx *c = a.ctx;
        const cudaStream_t as = b->aux[k++ % fsg_batch::NAUX];
        RayView R;
        if (rays_prepare(c, &R)) {                     // built at create: no host work here
            batch_join(b, s);
            return fail(ctx, FSG_E_STATE, c->err.c_str());
        }
        const int rr = R.nmu > 0
            ? fsg_launch_radtran_sph(as, fsg_view(c), c->d_lineopac.as<double>(), R, c->d_wmu.as<double>(), nullptr,
                                     nullptr, a.sfl.as<double>(), a.sfc.as<double>())
            : fsg_launch_radtran(as, fsg_view(c), c->d_lineopac.as<double>(), c->d_rhox.as<double>(), c->nmu,
                                 c->d_xmu.as<double>(), c->d_wmu.as<double>(), nullptr, nullptr, a.sfl.as<double>(),
                                 a.sfc.as<double>());
        if (rr) {
            const cudaError_t e = cudaGetLastError();
            batch_join(b, s);
            return cuda_fail(ctx, e, "k_radtran (batch)");
        }
    }
    batch_join(b, s);
    if (ev && ev[7]) batch_mark(ev[7], s);
    CK(cudaGetLastError(), "batch");
    return FSG_OK;
}

int fsg_batch_create(fsg_ctx *const *atms, int natm, const fsg_lines *lines, double margin, fsg_batch **out) {
    if (!atms || natm < 1 || !lines || !out || margin < 0) return FSG_E_ARG;
    *out = nullptr;
    fsg_config cfg = atms[0]->cfg;
    fsg_batch *b = new fsg_batch();
    int rc = fsg_create(&cfg, &b->own);
    if (rc) { delete b; g_batch_err = "fsg_batch_create: context creation failed"; return rc; }
    fsg_ctx *ctx = b->own;
    auto bail = [&](int code, const char *m) {
        g_batch_err = m ? m : ctx->err;
        fsg_batch_destroy(b);
        return code;
    };
    for (int i = 0; i < natm; i++) {
        fsg_ctx *c = atms[i];
        if (!c || c->device != ctx->device) return bail(FSG_E_ARG, "fsg_batch_create: contexts must share one device");
        if (c->cfg.precision != FSG_PREC_MIXED) return bail(FSG_E_STATE, "fsg_batch_create: mixed precision only");
        if (!c->have_grid || !c->have_atm || !c->have_cont || c->nmu < 1)
            return bail(FSG_E_STATE, "fsg_batch_create: set grid, atmosphere, continuum and mu of every context");
        if (c->ntau > 128) return bail(FSG_E_ARG, "fsg_batch_create: ntau <= 128");
        if (c->radius > 0.0) {                         // spherical: the rays (SphereInit) built now, once
            RayView R;
            if (rays_prepare(c, &R)) return bail(FSG_E_ARG, c->err.c_str());
        }
    }
    rc = check_lines(atms[0], lines); if (rc) return bail(rc, atms[0]->err.c_str());
    bool has_he = false;
    for (int i = 0; i < natm; i++) has_he = has_he || atms[i]->nhe > 0;
    if (has_he && lines->ihe)
        for (int64_t i = 0; i < lines->n; i++)
            if (lines->ihe[i] > 0)
                return bail(FSG_E_ARG, "fsg_batch_create: He I Stark-shifted lines are not batched");
    int nspc_min = atms[0]->nspc;
    for (int i = 1; i < natm; i++) nspc_min = std::min(nspc_min, atms[i]->nspc);
    for (int64_t i = 0; i < lines->n; i++) {
        if (i > 0 && lines->wl[i] < lines->wl[i - 1])
            return bail(FSG_E_ARG, "fsg_batch_create: the line list must be sorted by wavelength");
        if (lines->spc[i] < 0 || lines->spc[i] >= nspc_min)
            return bail(FSG_E_ARG, "fsg_batch_create: a species index is outside some atmosphere's species");
    }
    cudaSetDevice(ctx->device);
    if (lines->n > 0) { rc = upload_lines(ctx, lines, &b->dlines); if (rc) return bail(rc, nullptr); }
    b->atm.resize(natm);
    for (int i = 0; i < natm; i++) {
        BAtm &a = b->atm[i];
        fsg_ctx *c = atms[i];
        a.ctx = c;
        b->ntau_max = std::max(b->ntau_max, c->ntau);
        // candidates: lines with centres in [wstart - margin, wend + margin]; margin 0 is the reference
        // readers' WAVE= selection (ioutils.f90:752-753, 1496-1497)
        double w0 = c->wstart - margin, w1 = c->wend + margin;
        const double *wl = lines->wl;
        a.c0 = std::lower_bound(wl, wl + lines->n, w0) - wl;
        a.cn = (std::upper_bound(wl, wl + lines->n, w1) - wl) - a.c0;
        int rca = ensure_lineopac(c); if (rca) return bail(rca, c->err.c_str());
        if (a.cn > 2000000000LL) return bail(FSG_E_ARG, "fsg_batch_create: more than 2e9 lines in one span");
        a.ncls = fsg_bclass_count(c->nwl);
        const size_t nt = c->ntau, cn = std::max<int64_t>(a.cn, 1), ncl = a.ncls;
        const size_t nsb = (cn + 1023) / 1024 * (ncl + 1);          // class counts per CTA of the order
        const size_t ws = batch_wing_stride(c) * ncl, cs = batch_core_stride(c) * ncl;
        if (a.flags.ensure(4 * cn) || a.il.ensure(4 * cn) || a.ir.ensure(4 * cn) ||
            a.wing.ensure(sizeof(WingRec) * cn * nt) || a.core.ensure(sizeof(CoreRec) * cn * nt) ||
            a.hdr.ensure(sizeof(LineHdr) * cn) || a.wtlo.ensure(4 * ws) || a.wthi.ensure(4 * ws) ||
            a.ctlo.ensure(4 * cs) || a.cthi.ensure(4 * cs) || a.span.ensure(fsg_bspan_scratch(cn)) ||
            a.order.ensure(8 * cn) || a.ccnt.ensure(4 * nsb) || a.coff.ensure(8 * nsb) || a.ctot.ensure(8) ||
            a.sfl.ensure(8 * (size_t)c->nwl) || a.sfc.ensure(8 * (size_t)c->nwl))
            return bail(FSG_E_NOMEM, "fsg_batch_create: device allocation failed");
    }
    if (b->err.ensure(sizeof(int)) || b->nk.ensure(sizeof(unsigned long long)) ||
        b->evals.ensure(sizeof(unsigned long long)))
        return bail(FSG_E_NOMEM, "fsg_batch_create: device allocation failed");
    if (cudaMemset(b->err.p, 0, sizeof(int)) != cudaSuccess) return bail(FSG_E_CUDA, "fsg_batch_create: upload failed");
    for (int i = 0; i < 8; i++) cudaEventCreate(&b->ev[i]);
    if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
        return bail(FSG_E_CUDA, "fsg_batch_create: event creation failed");
    for (int k = 0; k < fsg_batch::NAUX; k++)
        if (cudaStreamCreateWithFlags(&b->aux[k], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming) != cudaSuccess)
            return bail(FSG_E_CUDA, "fsg_batch_create: stream creation failed");
    b->tune.tile_pix = 128;
    b->tune.wing_ctas = 148;
    b->tune.core_ctas = 4 * 148;
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device) == cudaSuccess && nsm > 0) {
        b->tune.wing_ctas = nsm;
        b->tune.core_ctas = 4 * nsm;
    }
    *out = b;
    return FSG_OK;
}

const char *fsg_batch_last_error(const fsg_batch *b) { return b ? b->own->err.c_str() : g_batch_err.c_str(); }

// windows and line evaluations of the batch (after a prepare): counted once, outside the graph
static int batch_count(fsg_batch *b) {
    fsg_ctx *ctx = b->own;
    double ev = 0;
    for (auto &a : b->atm) {
        if (!a.cn) continue;
        ev += count_windows(ctx, a.cn, a.flags.as<int32_t>(), a.il.as<int32_t>(), a.ir.as<int32_t>(), 1, a.ctx->nwl) *
              a.ctx->ntau;
    }
    b->line_evals = ev;
    return FSG_OK;
}

int fsg_batch_tune(fsg_batch *b, fsg_batch_tuning *result) {
    if (!b) return FSG_E_ARG;
    fsg_ctx *ctx = b->own;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
    // (1) wing pass: tile width x CTAs per SM, core pass at 4 CTAs per SM; (2) core pass CTAs
    fsg_batch_tuning best{ 128, nsm, 4 * nsm, 1e300, 1e300 };
    const int pix[2] = { 64, 128 };
    auto trial = [&](const fsg_batch_tuning &t, float *mw, float *mc) -> int {
        int rc2 = batch_accumulate_solve(b, t, b->ev); if (rc2) return rc2;
        CK(cudaStreamSynchronize(s), "batch tune");
        cudaEventElapsedTime(mw, b->ev[0], b->ev[1]);
        cudaEventElapsedTime(mc, b->ev[1], b->ev[2]);
        return FSG_OK;
    };
    for (int ip = 0; ip < 2; ip++) {
        int rc = batch_prepare(b, pix[ip] / 32); if (rc) return rc;
        rc = batch_jobs(b, pix[ip] / 32); if (rc) return rc;
        for (int wm = 1; wm <= 2; wm++) {
            fsg_batch_tuning t{ pix[ip], wm * nsm, 4 * nsm, 0.0, 0.0 };
            float mw = 0, mc = 0;
            rc = trial(t, &mw, &mc); if (rc) return rc;
            if (mw < best.ms_wing) { best.tile_pix = t.tile_pix; best.wing_ctas = t.wing_ctas; best.ms_wing = mw; }
        }
    }
    int rc = batch_prepare(b, best.tile_pix / 32); if (rc) return rc;
    rc = batch_jobs(b, best.tile_pix / 32); if (rc) return rc;
    for (int cm = 2; cm <= 8; cm *= 2) {
        fsg_batch_tuning t = best;
        t.core_ctas = cm * nsm;
        float mw = 0, mc = 0;
        rc = trial(t, &mw, &mc); if (rc) return rc;
        if (mc < best.ms_core) { best.core_ctas = t.core_ctas; best.ms_core = mc; }
    }
    int kerr = 0;
    CK(cudaMemcpy(&kerr, b->err.p, sizeof(int), cudaMemcpyDeviceToHost), "batch err");
    if (kerr) return fail(ctx, FSG_E_TIMEOUT, "k_accum_batch: a line-record copy did not complete within its bound");
    b->tune = best;
    b->tuned = 1;
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    if (result) *result = best;
    return FSG_OK;
}

int fsg_batch_set_tuning(fsg_batch *b, const fsg_batch_tuning *t) {
    if (!b || !t || (t->tile_pix != 64 && t->tile_pix != 128) || t->wing_ctas < 1 || t->core_ctas < 1)
        return FSG_E_ARG;
    b->tune = *t;
    b->tuned = 1;
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    return FSG_OK;
}

static int batch_run_body(fsg_batch *b, fsg_batch_stats *st) {
    if (!b) return FSG_E_ARG;
    fsg_ctx *ctx = b->own;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    int rc;
    if (!b->tuned) { rc = fsg_batch_tune(b, nullptr); if (rc) return rc; }
    if (!b->exec) {
        const int P = b->tune.tile_pix / 32;
        rc = batch_jobs(b, P); if (rc) return rc;
        rc = batch_prepare(b, P); if (rc) return rc;   // outside the graph once: counts and attributes
        CK(cudaStreamSynchronize(s), "batch");
        batch_count(b);
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "graph capture");
        batch_mark(b->ev[5], s);                        // event-record nodes: the replay's stage times
        rc = batch_prepare(b, P);
        if (!rc) rc = batch_accumulate_solve(b, b->tune, b->ev);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(s, &g);
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return cuda_fail(ctx, e, "graph capture");
        b->graph = g;
        CK(cudaGraphInstantiate(&b->exec, g, 0), "graph instantiate");
    }
    CK(cudaEventRecord(b->ev[3], s), "event");
    CK(cudaGraphLaunch(b->exec, s), "graph launch");
    CK(cudaEventRecord(b->ev[4], s), "event");
    CK(cudaStreamSynchronize(s), "batch run");
    int kerr = 0;
    CK(cudaMemcpy(&kerr, b->err.p, sizeof(int), cudaMemcpyDeviceToHost), "batch err");
    if (kerr) return fail(ctx, FSG_E_TIMEOUT, "k_accum_batch: a line-record copy did not complete within its bound");
    if (st) {
        memset(st, 0, sizeof *st);
        float ms = 0;
        cudaEventElapsedTime(&ms, b->ev[3], b->ev[4]);
        st->ms_total = ms;
        float m0 = 0, m1 = 0, m2 = 0, m3 = 0;
        cudaEventElapsedTime(&m0, b->ev[5], b->ev[0]);
        cudaEventElapsedTime(&m1, b->ev[0], b->ev[1]);
        cudaEventElapsedTime(&m2, b->ev[1], b->ev[2]);
        cudaEventElapsedTime(&m3, b->ev[2], b->ev[7]);
        st->ms_prepare = m0; st->ms_wing = m1; st->ms_core = m2; st->ms_solve = m3;
        unsigned long long nc = 0;
        CK(cudaMemcpy(&nc, b->evals.p, sizeof nc, cudaMemcpyDeviceToHost), "core count read");
        st->core_evals = (double)nc;
        st->line_evals = b->line_evals;
        for (auto &a : b->atm) st->nlines_candidate += a.cn;
        st->natm = (int)b->atm.size();
        st->tuning = b->tune;
    }
    return FSG_OK;
}

int fsg_batch_flux(fsg_batch *b, int iatm, double *sfl, double *sfc) {
    if (!b || iatm < 0 || iatm >= (int)b->atm.size()) return FSG_E_ARG;
    fsg_ctx *ctx = b->own;
    cudaSetDevice(ctx->device);
    BAtm &a = b->atm[iatm];
    size_t nb = sizeof(double) * (size_t)a.ctx->nwl;
    if (sfl) CK(cudaMemcpyAsync(sfl, a.sfl.p, nb, cudaMemcpyDeviceToHost, ctx->stream), "batch flux");
    if (sfc) CK(cudaMemcpyAsync(sfc, a.sfc.p, nb, cudaMemcpyDeviceToHost, ctx->stream), "batch flux");
    CK(cudaStreamSynchronize(ctx->stream), "batch flux");
    return FSG_OK;
}

void *fsg_batch_stream(fsg_batch *b) { return b ? (void *)b->own->stream : nullptr; }

void fsg_batch_destroy(fsg_batch *b) {
    if (!b) return;
    cudaSetDevice(b->own->device);
    cudaStreamSynchronize(b->own->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto &a : b->atm) {
        DBuf *bufs[] = { &a.flags, &a.il, &a.ir, &a.wing, &a.core, &a.hdr, &a.wtlo, &a.wthi, &a.ctlo, &a.cthi,
                         &a.span, &a.sfl, &a.sfc, &a.order, &a.ccnt, &a.coff, &a.ctot };
        for (DBuf *d : bufs) d->release();
    }
    DBuf *bufs[] = { &b->jobs_w, &b->jobs_c, &b->tile0_w, &b->tile0_c, &b->queue, &b->err, &b->nk,
                     &b->evals };
    for (DBuf *d : bufs) d->release();
    for (int i = 0; i < 8; i++) if (b->ev[i]) cudaEventDestroy(b->ev[i]);
    for (int k = 0; k < fsg_batch::NAUX; k++) {
        if (b->aux[k]) { cudaStreamSynchronize(b->aux[k]); cudaStreamDestroy(b->aux[k]); }
        if (b->join[k]) cudaEventDestroy(b->join[k]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    fsg_destroy(b->own);
    cudaGetLastError();
    delete b;
}

// ---- the drivers' public entries: an NVTX range each, and a metrics line when FSG_METRICS_JSONL is set ----
static std::string grid_fields(const fsg_ctx *ctx) {
    char b[160];
    snprintf(b, sizeof b, "\"nwl\": %d, \"ntau\": %d, \"nmu\": %d", ctx ? ctx->nwl : 0, ctx ? ctx->ntau : 0,
             ctx ? ctx->nmu : 0);
    return b;
}

int fsg_lineop_calc(fsg_ctx *ctx, const fsg_lines *lines, double *lineopac, int32_t *flags, int32_t *ileft,
                    int32_t *iright, float *linstr, fsg_stats *st) {
    CallTrace tr("fsg_lineop_calc");
    fsg_stats local{};
    fsg_stats *s = st ? st : (metrics_on() ? &local : nullptr);
    const int rc = lineop_calc_body(ctx, lines, lineopac, flags, ileft, iright, linstr, s);
    if (metrics_on()) metrics_emit("fsg_lineop_calc", rc, tr.ms(), rc || !s ? std::string() : stats_fields(*s));
    return rc;
}

int fsg_lineop_calc_dev(fsg_ctx *ctx, const fsg_lines *d_lines, fsg_stats *st) {
    CallTrace tr("fsg_lineop_calc_dev");
    fsg_stats local{};
    fsg_stats *s = st ? st : (metrics_on() ? &local : nullptr);
    const int rc = lineop_calc_dev_body(ctx, d_lines, s);
    if (metrics_on()) metrics_emit("fsg_lineop_calc_dev", rc, tr.ms(), rc || !s ? std::string() : stats_fields(*s));
    return rc;
}

int fsg_mag_lineop_calc(fsg_ctx *ctx, const fsg_lines *lines, int bframe, const double *bfield, int nbfield,
                        double *maglineopac, int32_t *flags, int32_t *ileft, int32_t *iright, float *linstr,
                        fsg_stats *st) {
    CallTrace tr("fsg_mag_lineop_calc");
    fsg_stats local{};
    fsg_stats *s = st ? st : (metrics_on() ? &local : nullptr);
    const int rc = mag_lineop_calc_body(ctx, lines, bframe, bfield, nbfield, maglineopac, flags, ileft, iright,
                                        linstr, s);
    if (metrics_on()) metrics_emit("fsg_mag_lineop_calc", rc, tr.ms(), rc || !s ? std::string() : stats_fields(*s));
    return rc;
}

int fsg_radtran(fsg_ctx *ctx, double *spl, double *spc, double *sfl, double *sfc) {
    CallTrace tr("fsg_radtran");
    const int rc = radtran_body(ctx, spl, spc, sfl, sfc);
    if (metrics_on()) metrics_emit("fsg_radtran", rc, tr.ms(), grid_fields(ctx));
    return rc;
}

int fsg_radtran_dev(fsg_ctx *ctx, double *d_spl, double *d_spc, double *d_sfl, double *d_sfc) {
    CallTrace tr("fsg_radtran_dev");
    const int rc = radtran_dev_body(ctx, d_spl, d_spc, d_sfl, d_sfc);
    if (metrics_on()) metrics_emit("fsg_radtran_dev", rc, tr.ms(), grid_fields(ctx));
    return rc;
}

int fsg_radtran_range_dev(fsg_ctx *ctx, int i0, int i1, double *d_spl, double *d_spc, double *d_sfl, double *d_sfc) {
    CallTrace tr("fsg_radtran_range_dev");
    const int rc = radtran_range_dev_body(ctx, i0, i1, d_spl, d_spc, d_sfl, d_sfc);
    if (metrics_on()) {
        char b[64];
        snprintf(b, sizeof b, ", \"i0\": %d, \"i1\": %d", i0, i1);
        metrics_emit("fsg_radtran_range_dev", rc, tr.ms(), grid_fields(ctx) + b);
    }
    return rc;
}

int fsg_mag_radtran(fsg_ctx *ctx, int bframe, const double *bfield, int nbfield, double *spz, double *spc,
                    double *sfl, double *sfc) {
    CallTrace tr("fsg_mag_radtran");
    const int rc = mag_radtran_body(ctx, bframe, bfield, nbfield, spz, spc, sfl, sfc);
    if (metrics_on()) metrics_emit("fsg_mag_radtran", rc, tr.ms(), grid_fields(ctx));
    return rc;
}

int fsg_batch_run(fsg_batch *b, fsg_batch_stats *st) {
    CallTrace tr("fsg_batch_run");
    fsg_batch_stats local{};
    fsg_batch_stats *s = st ? st : (metrics_on() ? &local : nullptr);
    const int rc = batch_run_body(b, s);
    if (metrics_on()) {
        char f[512] = "";
        if (!rc && s)
            snprintf(f, sizeof f,
                     "\"natm\": %d, \"nlines_candidate\": %lld, \"line_evals\": %.17g, \"ms_total\": %.6f, "
                     "\"ms_prepare\": %.6f, \"ms_wing\": %.6f, \"ms_core\": %.6f, \"ms_solve\": %.6f, \"core_evals\": %.17g",
                     s->natm, (long long)s->nlines_candidate, s->line_evals, s->ms_total, s->ms_prepare, s->ms_wing,
                     s->ms_core, s->ms_solve, s->core_evals);
        metrics_emit("fsg_batch_run", rc, tr.ms(), f);
    }
    return rc;
}

}  // extern "C"

// ---- eval counting for the stats (sum over retained lines of Ntau x window) -------------------------
// npi / nsi (may be null): Zeeman component counts; each window wavelength then counts once per component
__global__ void k_count_evals(int64_t n, const int32_t *flags, const int32_t *il, const int32_t *ir, int i0, int i1,
                              const int32_t *npi, const int32_t *nsi, unsigned long long *acc) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long v = 0;
    if (i < n && !(flags[i] & FSG_F_WEAK)) {
        int a = max(il[i], i0), b = min(ir[i], i1);
        if (a <= b) v = (unsigned long long)(b - a + 1) * (npi ? (unsigned long long)(npi[i] + nsi[i]) : 1ull);
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(acc, v);
}

double fsg_count_evals(fsg_ctx *ctx, int64_t n, const int32_t *fl, const int32_t *il, const int32_t *ir, int i0,
                       int i1) {
    return count_windows(ctx, n, fl, il, ir, i0, i1) * ctx->ntau;
}

// retained-window wavelengths (inside [i0, i1]) of n lines, times their Zeeman components when given
static double count_windows(fsg_ctx *ctx, int64_t n, const int32_t *fl, const int32_t *il, const int32_t *ir, int i0,
                            int i1, const int32_t *npi, const int32_t *nsi) {
    if (ctx->d_nkeep.ensure(sizeof(unsigned long long)) != FSG_OK) return 0.0;
    ctx->launches += 1;
    unsigned long long *d = ctx->d_nkeep.as<unsigned long long>();
    cudaMemsetAsync(d, 0, sizeof(unsigned long long), ctx->stream);
    k_count_evals<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(n, fl, il, ir, i0, i1, npi, nsi, d);
    unsigned long long h = 0;
    cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    return (double)h;
}
