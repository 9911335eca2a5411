// fsg_adjoint.cu -- reverse-mode derivatives of the disk-integrated flux (FP64).
//
// The forward chain is LineopCalc -> RadTranCalc -> DiskInteg:
//   kappa(t, lambda) = ContOpac + sum_lines H(a, v) LinCop        (opacity.f90:297-346)
//   I_mu(lambda)     = DELO-Bezier sweep of kappa and the Planck source (solver.f90:123-179)
//   SfL(lambda)      = sum_mu Wmu I_mu                              (convol.f90:233-234)
// Given dL/dSfL, k_solver_adjoint runs the sweep backwards (TauStep, CentDer, the Bezier control
// terms and the DELO coefficients differentiated in the order the forward evaluates them) and
// gives dL/dkappa for every depth and wavelength.  k_line_adjoint then recomputes every retained
// line's profile over its window (nothing is stored from the forward) and reduces
//   glin_l  = sum_{t, lambda} dL/dkappa * H * LinCop          (= dL/dln(gf), = dL/dln(abundance))
// (H and L from FvTab, the FP32 table of the Faraday-Voigt pair: H agrees with VgtTab's to ~1e-7)
//   gvmic_l = sum_{t, lambda} dL/dkappa * dLinCop H / dvmic
// with H, L from the reference's tables and asymptotics and the Faddeeva derivative
// dw/dz = -2 z w + 2i/sqrt(pi), w = H + iL, z = v + ia:
//   dH/dv = -2 (v H - a L),   dH/da = 2 (v L + a H) - 2/sqrt(pi);
// LinCop, v and a all scale as 1/Dopl, and d ln Dopl / d vmic = vturb2 / (vmic Dopl^2).
// The window half-width of AnalyticWindow (opacity.f90:678-710), W = max_t sqrt(S_t) / LinVvgt_t with
// S = ln r + max(0, a (r / sqrt(pi) - a)), r = LinCop / (EpsOpac ContOpac), also grows with gf and
// vmic; its edges move by dW, adding the edge profile over dW / (wavelength step) at each free
// edge.  That boundary term is added to both sums (d ln W from the depth giving the maximum).
#include "fsg_fp64.cuh"

// DELO coefficients (solver.f90:357-370) and their derivatives with respect to Dtau
__device__ __forceinline__ void delo_coef_d(double D, double &E, double &A, double &B, double &G, double &dE,
                                            double &dA, double &dB, double &dG) {
    delo_coef(D, E, A, B, G);
    if (D < 5e-3) {
        const double D2 = D * D;
        dE = -1.0 + D - 0.5 * D2 + D2 * D / 6.0;
        dA = 1.0 / 3.0 - D / 6.0 + D2 / 20.0;
        dB = 1.0 / 3.0 - 0.5 * D + 0.3 * D2;
        dG = 1.0 / 3.0 - D / 3.0 + 0.15 * D2;
    } else {
        const double iD = 1.0 / D, iD2 = iD * iD;
        dE = -E;
        dA = (2.0 * D - 2.0 + 2.0 * E) * iD2 - 2.0 * A * iD;
        dB = E - 2.0 * B * iD;
        dG = (2.0 - 2.0 * E - 2.0 * D * E) * iD2 - 2.0 * G * iD;
    }
}

// monotone harmonic-mean derivative Yp = Der Der1 / (Lambda Der1 + (1 - Lambda) Der) and its
// partial derivatives (Der Der1 > 0)
__device__ __forceinline__ void hmean_d(double Der, double Der1, double Lambda, double &Y, double &dDer,
                                       double &dDer1, double &dLambda) {
    const double N = Der * Der1, Q = Lambda * Der1 + (1.0 - Lambda) * Der, iQ2 = 1.0 / (Q * Q);
    Y = N / Q;
    dDer = (Der1 * Q - N * (1.0 - Lambda)) * iQ2;
    dDer1 = (Der * Q - N * Lambda) * iQ2;
    dLambda = -N * (Der1 - Der) * iQ2;
}

// one thread per wavelength; work: 10 arrays of nt x nwl doubles (wavelength fastest)
__global__ void k_solver_adjoint(AtmView A, const double *__restrict__ lineopac, const double *__restrict__ rhox,
                                 int nmu, const double *__restrict__ xmu, const double *__restrict__ wmu,
                                 const double *__restrict__ gflux, double *__restrict__ gkappa, double *work) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    const int nwl = A.nwl, nt = A.ntau;
    if (w >= nwl) return;
    const double PlkC1 = FSG_HC * FSG_VC * 1e13 / FSG_KBOLT;
    auto W = [&](int k, int t) -> double & { return work[((size_t)k * nt + t) * nwl + w]; };
    enum { X, Y, D, R, U, GD, GR, GU, GX, YS };
    const double wl = A.wave[w] + A.wfirst;
    const double C1 = PlkC1 / wl, C2 = exp(50.7649141 - 5.0 * log(wl));
    for (int t = 0; t < nt; t++) {
        size_t g = (size_t)w * nt + t;
        W(X, t) = A.contopac[g] + lineopac[g];
        W(Y, t) = C2 / (exp(C1 / A.xi[XI_T * nt + t]) - 1.0);
        W(GD, t) = 0.0; W(GR, t) = 0.0; W(GU, t) = 0.0; W(GX, t) = 0.0;
    }
    // forward: TauStep (solver.f90:591-615)
    {
        double Dx1 = rhox[1] - rhox[0], Yp = (W(X, 1) - W(X, 0)) / Dx1;
        W(D, 0) = Dx1 * (W(X, 1) + 2.0 * W(X, 0) + Dx1 / 2.0 * Yp) / 3.0;
        for (int k = 2; k <= nt - 1; k++) {
            double Dx = rhox[k - 1] - rhox[k - 2]; Dx1 = rhox[k] - rhox[k - 1];
            double Der = (W(X, k - 1) - W(X, k - 2)) / Dx, Der1 = (W(X, k) - W(X, k - 1)) / Dx1;
            if (Der * Der1 > 0.0) {
                double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0;
                Yp = (Der / (Lambda * Der1 + (1.0 - Lambda) * Der)) * Der1;
            } else Yp = 0.0;
            W(D, k - 1) = Dx1 * (W(X, k) + 2.0 * W(X, k - 1) + Dx1 / 2.0 * Yp) / 3.0;
        }
    }
    // CentDer of the source (solver.f90:618-647) and the Bezier control terms
    for (int k = 2; k <= nt - 1; k++) {
        double Dx = W(D, k - 2), Dx1 = W(D, k - 1);
        double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0;
        double Der = (W(Y, k - 1) - W(Y, k - 2)) / Dx, Der1 = (W(Y, k) - W(Y, k - 1)) / Dx1;
        W(R, k - 1) = (Der * Der1 > 0.0) ? (Der / (Lambda * Der1 + (1.0 - Lambda) * Der)) * Der1 : 0.0;
    }
    W(R, 0) = (W(Y, 1) - W(Y, 0)) / W(D, 0);
    W(R, nt - 1) = (W(Y, nt - 1) - W(Y, nt - 2)) / W(D, nt - 2);
    for (int k = 0; k < nt - 1; k++)
        W(U, k) = 0.5 * (W(Y, k) + 0.5 * W(D, k) * W(R, k) + W(Y, k + 1) - 0.5 * W(D, k) * W(R, k + 1));
    // sweeps: forward (storing Y_k), then backwards from dL/dI_mu = Wmu dL/dSfL
    const double gF = gflux[w];
    for (int im = 0; im < nmu; im++) {
        const double Imu = 1.0 / xmu[im];
        double Yv = W(Y, nt - 1);
        W(YS, nt - 1) = Yv;
        for (int k = nt - 2; k >= 0; k--) {
            double E, Al, Be, Ga;
            delo_coef(W(D, k) * Imu, E, Al, Be, Ga);
            Yv = Yv * E + Al * W(Y, k) + Be * W(Y, k + 1) + Ga * W(U, k);
            W(YS, k) = Yv;
        }
        double gY = wmu[im] * gF;
        for (int k = 0; k <= nt - 2; k++) {
            double E, Al, Be, Ga, dE, dAl, dBe, dGa;
            delo_coef_d(W(D, k) * Imu, E, Al, Be, Ga, dE, dAl, dBe, dGa);
            double gDt = gY * (W(YS, k + 1) * dE + W(Y, k) * dAl + W(Y, k + 1) * dBe + W(U, k) * dGa);
            W(GD, k) += gDt * Imu;
            W(GU, k) += gY * Ga;
            gY = gY * E;
        }
    }
    // u_k -> d_k, r_k, r_{k+1}
    for (int k = 0; k < nt - 1; k++) {
        double gu = W(GU, k);
        W(GD, k) += gu * 0.25 * (W(R, k) - W(R, k + 1));
        W(GR, k) += gu * 0.25 * W(D, k);
        W(GR, k + 1) -= gu * 0.25 * W(D, k);
    }
    // CentDer -> d
    W(GD, 0) -= W(GR, 0) * W(R, 0) / W(D, 0);
    W(GD, nt - 2) -= W(GR, nt - 1) * W(R, nt - 1) / W(D, nt - 2);
    for (int k = 2; k <= nt - 1; k++) {
        double Dx = W(D, k - 2), Dx1 = W(D, k - 1);
        double Der = (W(Y, k - 1) - W(Y, k - 2)) / Dx, Der1 = (W(Y, k) - W(Y, k - 1)) / Dx1;
        if (!(Der * Der1 > 0.0)) continue;
        double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0, Yp, dDer, dDer1, dLam;
        hmean_d(Der, Der1, Lambda, Yp, dDer, dDer1, dLam);
        double s = Dx + Dx1, g = W(GR, k - 1);
        W(GD, k - 2) += g * (dDer * (-Der / Dx) + dLam * (-Dx1 / (3.0 * s * s)));
        W(GD, k - 1) += g * (dDer1 * (-Der1 / Dx1) + dLam * (Dx / (3.0 * s * s)));
    }
    // TauStep -> kappa
    {
        double Dx1 = rhox[1] - rhox[0];
        W(GX, 0) += W(GD, 0) * 0.5 * Dx1;
        W(GX, 1) += W(GD, 0) * 0.5 * Dx1;
        for (int k = 2; k <= nt - 1; k++) {
            double Dx = rhox[k - 1] - rhox[k - 2]; Dx1 = rhox[k] - rhox[k - 1];
            double Der = (W(X, k - 1) - W(X, k - 2)) / Dx, Der1 = (W(X, k) - W(X, k - 1)) / Dx1;
            double g = W(GD, k - 1);
            W(GX, k) += g * Dx1 / 3.0;
            W(GX, k - 1) += g * 2.0 * Dx1 / 3.0;
            if (Der * Der1 > 0.0) {
                double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0, Yp, dDer, dDer1, dLam;
                hmean_d(Der, Der1, Lambda, Yp, dDer, dDer1, dLam);
                double c = g * Dx1 * Dx1 / 6.0;
                W(GX, k) += c * dDer1 / Dx1;
                W(GX, k - 1) += c * (dDer / Dx - dDer1 / Dx1);
                W(GX, k - 2) += c * (-dDer / Dx);
            }
        }
    }
    for (int t = 0; t < nt; t++) gkappa[(size_t)w * nt + t] = W(GX, t);
}

// one warp per line; per-depth LinCop, LinVvgt, LinAvgt and d ln Dopl / d vmic in shared memory
#define LADJ_WARPS 8
__global__ void __launch_bounds__(32 * LADJ_WARPS)
k_line_adjoint(AtmView A, LineView L, const float *__restrict__ vtab, const float2 *__restrict__ fvtab,
               const double *__restrict__ anode, const double *__restrict__ aida, const int32_t *__restrict__ flags,
               const int32_t *__restrict__ ileft, const int32_t *__restrict__ iright,
               const double *__restrict__ gkappa, double vmic, double *glin, double *gvmic) {
    extern __shared__ double sh[];
    const int nt = A.ntau;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *cop = sh + (size_t)warp * 6 * nt, *vv = cop + nt, *av = vv + nt, *q = av + nt, *shf = q + nt;
    double *rr = shf + nt;
    const int64_t i = (int64_t)blockIdx.x * LADJ_WARPS + warp;
    if (i >= L.n) return;
    const int f = flags[i];
    if (f & FSG_F_WEAK) {
        if (lane == 0) { glin[i] = 0.0; gvmic[i] = 0.0; }
        return;
    }
    const double wlc = L.wl[i] - A.wfirst;
    XCoef XC;
    xline_setup(A, L, i, wlc, line_input_flags(L, i, 0), &XC);
    const int iwc = waveidx(A, wlc);
    const double dWc = (wlc - A.wave[iwc - 1]) / (A.wave[iwc] - A.wave[iwc - 1]);
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
        shf[t] = (XC.IxHe > 0) ? A.heshf[(XC.IxHe - 1) * nt + t] : 0.0;
    }
    __syncwarp();
    const int il = ileft[i], ir = iright[i];
    double sl = 0.0, sv = 0.0;
    const double isp2 = 2.0 * FSG_SQRTPIINV;
    // lanes over depths (t = lane, lane + 32, ...), a loop over the window's wavelengths: the
    // dL/dkappa reads of a wavelength are contiguous across the lanes
    for (int t = lane; t < nt; t += 32) {
        const double c = cop[t], vvt = vv[t], a = av[t], qt = q[t], off = wlc + shf[t];
        const VLine64 VL = vline64(anode, aida, a);
        double s1 = 0.0, s2 = 0.0;
        const float af = (float)a, a2f = af * af;
        for (int iw = il - 1; iw < ir; iw++) {
            const double g = gkappa[(size_t)iw * nt + t];
            const double v = (A.wave[iw] - off) * vvt;
            const float vf = (float)v, sf = vf * vf + a2f;
            if (sf >= 196.0f) {
                // wing: the rational (H, L) pair of FVoigt (voigt.f90:256-352) in FP32 (the gradient needs no more)
                const float w = 0.56418958f / (sf * sf - vf * vf + a2f + 0.25f);
                const float Hf = af * (sf + 0.5f) * w, Lf = vf * (sf - 0.5f) * w;
                const float Hv = -2.0f * (vf * Hf - af * Lf), Ha = 2.0f * (vf * Lf + af * Hf) - (float)isp2;
                s1 += g * (double)Hf;
                s2 += g * (double)(-vf * Hv - af * Ha - Hf);
            } else {
                double Hf, Lf;
                fvoigt_line64(fvtab, VL, v, &Hf, &Lf);
                const double Hv = -2.0 * (v * Hf - a * Lf), Ha = 2.0 * (v * Lf + a * Hf) - isp2;
                s1 += g * Hf;
                s2 += g * (-v * Hv - a * Ha - Hf);
            }
        }
        sl += s1 * c;
        sv += s2 * c * qt;
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
        if (il > 1) {
            const int iw = il - 1;
            const double v = (A.wave[iw] - wlc - shf[t]) * vv[t];
            eb += gkappa[(size_t)iw * nt + t] * hvoigt_line64(vtab, VL, v) * cop[t] / (A.wave[iw] - A.wave[iw - 1]);
        }
        if (ir < A.nwl) {
            const int iw = ir - 1;
            const double v = (A.wave[iw] - wlc - shf[t]) * vv[t];
            eb += gkappa[(size_t)iw * nt + t] * hvoigt_line64(vtab, VL, v) * cop[t] / (A.wave[iw + 1] - A.wave[iw]);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        sl += __shfl_xor_sync(0xffffffffu, sl, o);
        sv += __shfl_xor_sync(0xffffffffu, sv, o);
        eb += __shfl_xor_sync(0xffffffffu, eb, o);
        const double wo = __shfl_xor_sync(0xffffffffu, wbest, o), go = __shfl_xor_sync(0xffffffffu, dgf, o);
        const double vo = __shfl_xor_sync(0xffffffffu, dvm, o);
        if (wo > wbest || (wo == wbest && go > dgf)) { wbest = wo; dgf = go; dvm = vo; }
    }
    if (lane == 0) {
        if (wbest < 0.0) { dgf = 0.0; dvm = 0.0; }
        glin[i] = sl + eb * dgf;
        gvmic[i] = sv + eb * dvm;
    }
}

size_t fsg_adjoint_work(int nwl, int nt) { return sizeof(double) * 10 * (size_t)nt * nwl; }

int fsg_launch_adjoint(cudaStream_t s, const AtmView &A, const LineView &L, const VoigtTables &T,
                       const double *lineopac, const double *rhox, int nmu, const double *xmu, const double *wmu,
                       const int32_t *flags, const int32_t *ileft, const int32_t *iright, const double *gflux,
                       double *gkappa, double *work, double vmic, double *glin, double *gvmic) {
    k_solver_adjoint<<<(A.nwl + 127) / 128, 128, 0, s>>>(A, lineopac, rhox, nmu, xmu, wmu, gflux, gkappa, work);
    if (L.n > 0) {
        size_t smem = sizeof(double) * 6 * A.ntau * LADJ_WARPS;
        k_line_adjoint<<<(unsigned)((L.n + LADJ_WARPS - 1) / LADJ_WARPS), 32 * LADJ_WARPS, smem, s>>>(
            A, L, T.vtab, T.fvtab, T.anode, T.aida, flags, ileft, iright, gkappa, vmic, glin, gvmic);
    }
    return cudaGetLastError() == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}
