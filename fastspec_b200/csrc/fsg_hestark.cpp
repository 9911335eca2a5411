// Tabulated He I Stark broadening on the host: the per-atmosphere width/shift tables (HeStarkInit,
// hestark.f90:332-370) and the per-line table match (HeMatchIdx, hestark.f90:376-389, called from
// XlineSetup at opacity.f90:176).  Both are O(37 x Ntau) and O(lines) integer/FP64 bookkeeping done
// once per atmosphere and once per list; the device path consumes their results through
// fsg_set_hestark and the ihe column of fsg_lines.  FP64 in the reference's operand order (this
// unit is built without floating-point contraction).
#include <cmath>
#include <cstdint>

#include "../../include/fastspec_gpu.h"
#include "fsg_hestark_tables.h"

namespace {

// LagWt3 (hestark.f90:394-415): three-point Lagrange weights on the knots t[0..n-1] at x; j is the
// 0-based index of the upper knot (value = w0 F[j] + w1 F[j-1] + w2 F[j-2]); the first knot above x
// from the third on, else the last (extrapolation at both ends).
int lagwt3(const double *t, int n, double x, double &w0, double &w1, double &w2) {
    int j = n - 1;
    for (int k = 2; k < n; k++)
        if (t[k] > x) { j = k; break; }
    const double a = t[j], b = t[j - 1], c = t[j - 2];
    const double den = (a - b) * (a - c) * (b - c);
    w0 = (x - c) * (x - b) * (b - c) / den;
    w1 = (x - c) * (a - x) * (a - c) / den;
    w2 = (x - b) * (x - a) * (a - b) / den;
    return j;
}

inline double lag(const double *f, int j, double w0, double w1, double w2) {
    return w0 * f[j] + w1 * f[j - 1] + w2 * f[j - 2];
}

constexpr double kHeGamCnv = 1.884e3;   // 2 pi c / 1e16 [A/s] (hestark.f90:39)
constexpr double kHeMatchTol = 1.0;     // A (hestark.f90:31)
constexpr double kHeEloTol = 0.01;      // eV (hestark.f90:36)

}  // namespace

extern "C" int fsg_hestark_tables(int ntau, const double *T, const double *xne, const float *frac_hii,
                                  const float *frac_heii, double *hegam, double *heshf) {
    if (ntau < 1 || !T || !xne || !frac_hii || !frac_heii || !hegam || !heshf) return FSG_E_ARG;
    for (int t = 0; t < ntau; t++)
        if (!(T[t] > 0.0)) return FSG_E_ARG;
    for (int t = 0; t < ntau; t++) {
        const double lt = std::log10(T[t]);
        const double ne = xne[t], np = (double)frac_hii[t], nhe2 = (double)frac_heii[t];
        double w90[3], w84[3];
        const int j90 = lagwt3(FSG_HE_LOGT90, 6, lt, w90[0], w90[1], w90[2]);
        const int j84 = lagwt3(FSG_HE_LOGT84, 4, lt, w84[0], w84[1], w84[2]);
        for (int k = 0; k < FSG_HE_NTAB; k++) {
            const fsg_he_line &e = FSG_HE_TAB[k];
            double g, sh;
            if (k < FSG_HE_NDS90) {
                // electrons, protons and He II ions (DS90)
                const double *w = w90; const int j = j90;
                g = (lag(e.w[0], j, w[0], w[1], w[2]) * ne + lag(e.w[1], j, w[0], w[1], w[2]) * np +
                     lag(e.w[2], j, w[0], w[1], w[2]) * nhe2) * kHeGamCnv / (e.wlc * e.wlc);
                sh = (lag(e.s[0], j, w[0], w[1], w[2]) * ne + lag(e.s[1], j, w[0], w[1], w[2]) * np +
                      lag(e.s[2], j, w[0], w[1], w[2]) * nhe2) * 1e-16;
            } else {
                // electrons and protons (DS84)
                const double *w = w84; const int j = j84;
                g = (lag(e.w[0], j, w[0], w[1], w[2]) * ne + lag(e.w[1], j, w[0], w[1], w[2]) * np) *
                    kHeGamCnv / (e.wlc * e.wlc);
                sh = (lag(e.s[0], j, w[0], w[1], w[2]) * ne + lag(e.s[1], j, w[0], w[1], w[2]) * np) * 1e-16;
            }
            hegam[(size_t)k * ntau + t] = g > 0.0 ? g : 0.0;
            heshf[(size_t)k * ntau + t] = sh;
        }
    }
    return FSG_OK;
}

extern "C" int fsg_he_match_idx(long n, const double *wl, const float *elo, const int32_t *spc, int spc_he1,
                                double wfirst, int32_t *ihe) {
    if (n < 0 || (n > 0 && (!wl || !elo || !spc || !ihe))) return FSG_E_ARG;
    for (long i = 0; i < n; i++) {
        int32_t m = 0;
        if (spc[i] == spc_he1) {
            // XlineSetup's WaveL = Wlcent + Wfirst with Wlcent = Wl - Wfirst; Elo widened from FP32
            const double wave = (wl[i] - wfirst) + wfirst, e = (double)elo[i];
            for (int k = 0; k < FSG_HE_NTAB; k++)
                if (std::fabs(wave - FSG_HE_TAB[k].wlc) <= kHeMatchTol && std::fabs(e - FSG_HE_TAB[k].elo) <= kHeEloTol) {
                    m = k + 1;
                    break;
                }
        }
        ihe[i] = m;
    }
    return FSG_OK;
}
