// fsg_mag.cu -- magnetic (Zeeman / Faraday-Voigt) path: MagLineopCalc and MagRadTranCalc.
#include "fsg_internal.cuh"

extern "C" {
int fsg_mag_lineop_calc(fsg_ctx *ctx, const fsg_lines *lines, int bframe, const double *bfield, int nbfield,
                        double *maglineopac, int32_t *flags, int32_t *ileft, int32_t *iright, float *linstr,
                        fsg_stats *stats) {
    (void)ctx; (void)lines; (void)bframe; (void)bfield; (void)nbfield; (void)maglineopac; (void)flags;
    (void)ileft; (void)iright; (void)linstr; (void)stats;
    return FSG_E_STATE;
}
int fsg_mag_lineop_reset(fsg_ctx *ctx) { (void)ctx; return FSG_E_STATE; }
int fsg_mag_radtran(fsg_ctx *ctx, int bframe, const double *bfield, int nbfield, double *spz, double *spc,
                    double *sfl, double *sfc) {
    (void)ctx; (void)bframe; (void)bfield; (void)nbfield; (void)spz; (void)spc; (void)sfl; (void)sfc;
    return FSG_E_STATE;
}
}
