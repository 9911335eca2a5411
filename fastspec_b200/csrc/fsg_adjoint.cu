// fsg_adjoint.cu -- reverse-mode derivatives of the disk-integrated flux (FP64).
//
// The forward chain is LineopCalc -> RadTranCalc -> DiskInteg:
//   kappa(t, lambda) = ContOpac + sum_lines H(a, v) LinCop        (opacity.f90:297-346)
//   I_mu(lambda)     = DELO-Bezier sweep of kappa and the Planck source (solver.f90:123-179)
//   SfL(lambda)      = sum_mu Wmu I_mu                              (convol.f90:233-234)
// Given dL/dSfL, k_solver_adjoint runs the sweep backwards (TauStep, CentDer, the Bezier control
// terms and the DELO coefficients differentiated in the order the forward evaluates them) and
// gives dL/dkappa for every depth and wavelength, in FP64 and as an FP32 copy (wavelength fastest)
// for the line pass of fsg_adjoint_line.cu, which recomputes every retained line's profile over its
// window (nothing is stored from the forward) and reduces it against dL/dkappa.
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
                                 const double *__restrict__ gflux, double *__restrict__ gkappa, double *work,
                                 float *__restrict__ gk32, float *__restrict__ wvh, float *__restrict__ wvl) {
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
    for (int t = 0; t < nt; t++) {
        gkappa[(size_t)w * nt + t] = W(GX, t);
        gk32[(size_t)t * nwl + w] = (float)W(GX, t);          // FP32 copy, wavelength fastest
    }
    // the wavelength offset as FP32 hi + lo for the line pass
    const double wv = A.wave[w];
    wvh[w] = (float)wv;
    wvl[w] = (float)(wv - (double)wvh[w]);
}

// Spherical models: the same chain along each ray of LocPrfSph (solver.f90:182-261, the forward is
// delo_ray): per ray the TauStep steps on the ray's column mass, CentDer of the source, the Bezier
// terms and the sweep (grazing rays start from zero at the far side), run backwards from dL/dI_ray =
// Wmu dL/dSfL; a ray point's derivative goes to the layer it samples.  One thread per wavelength; work:
// per wavelength X, Y, GX by layer (3 nt) and D, R, U, YS, GD, GR, GU by ray point (7 x 2 nt).
#define SPH_WORK 17
__global__ void k_solver_adjoint_sph(AtmView A, const double *__restrict__ lineopac, RayView RV,
                                     const double *__restrict__ wmu, const double *__restrict__ gflux,
                                     double *__restrict__ gkappa, double *work, float *__restrict__ gk32,
                                     float *__restrict__ wvh, float *__restrict__ wvl) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    const int nwl = A.nwl, nt = A.ntau, M = 2 * nt;
    if (w >= nwl) return;
    const double PlkC1 = FSG_HC * FSG_VC * 1e13 / FSG_KBOLT;
    // layer arrays at 0, nt, 2 nt; ray-point arrays at 3 nt + k M
    auto L = [&](int k, int t) -> double & { return work[((size_t)k * nt + t) * nwl + w]; };
    auto P = [&](int k, int j) -> double & { return work[((size_t)3 * nt + (size_t)k * M + j) * nwl + w]; };
    enum { X, Y, GX };
    enum { D, R, U, YS, GD, GR, GU };
    const double wl = A.wave[w] + A.wfirst;
    const double C1 = PlkC1 / wl, C2 = exp(50.7649141 - 5.0 * log(wl));
    for (int t = 0; t < nt; t++) {
        size_t g = (size_t)w * nt + t;
        L(X, t) = A.contopac[g] + lineopac[g];
        L(Y, t) = C2 / (exp(C1 / A.xi[XI_T * nt + t]) - 1.0);
        L(GX, t) = 0.0;
    }
    const double gF = gflux[w];
    for (int im = 0; im < RV.nmu; im++) {
        const int N = RV.n[im];
        const int *mp = RV.map + (size_t)im * RV.stride;
        const double *m = RV.m + (size_t)im * RV.stride;
        auto x = [&](int j) { return L(X, mp[j]); };
        auto y = [&](int j) { return L(Y, mp[j]); };
        // forward: TauStep on the ray, CentDer of the source, Bezier terms, the sweep (storing Y_j)
        for (int j = 0; j <= N - 2; j++) {
            double d;
            if (j == 0) {
                const double Dx1 = m[1] - m[0], Yp = (x(1) - x(0)) / Dx1;
                d = Dx1 * (x(1) + 2.0 * x(0) + Dx1 / 2.0 * Yp) / 3.0;
            } else {
                const double Dx = m[j] - m[j - 1], Dx1 = m[j + 1] - m[j];
                const double Der = (x(j) - x(j - 1)) / Dx, Der1 = (x(j + 1) - x(j)) / Dx1;
                double Yp = 0.0;
                if (Der * Der1 > 0.0) {
                    const double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0;
                    Yp = (Der / (Lambda * Der1 + (1.0 - Lambda) * Der)) * Der1;
                }
                d = Dx1 * (x(j + 1) + 2.0 * x(j) + Dx1 / 2.0 * Yp) / 3.0;
            }
            P(D, j) = d;
            P(GD, j) = 0.0; P(GU, j) = 0.0;
        }
        for (int j = 0; j < N; j++) P(GR, j) = 0.0;
        P(R, 0) = (y(1) - y(0)) / P(D, 0);
        P(R, N - 1) = (y(N - 1) - y(N - 2)) / P(D, N - 2);
        for (int j = 1; j <= N - 2; j++) P(R, j) = centder3(P(D, j - 1), P(D, j), y(j - 1), y(j), y(j + 1));
        for (int j = 0; j <= N - 2; j++)
            P(U, j) = 0.5 * (y(j) + 0.5 * P(D, j) * P(R, j) + y(j + 1) - 0.5 * P(D, j) * P(R, j + 1));
        double Yv = RV.graz[im] ? 0.0 : y(N - 1);
        P(YS, N - 1) = Yv;
        for (int j = N - 2; j >= 0; j--) {
            double E, Al, Be, Ga;
            delo_coef(P(D, j), E, Al, Be, Ga);
            Yv = Yv * E + Al * y(j) + Be * y(j + 1) + Ga * P(U, j);
            P(YS, j) = Yv;
        }
        // backward from dL/dI = Wmu dL/dSfL
        double gY = wmu[im] * gF;
        for (int j = 0; j <= N - 2; j++) {
            double E, Al, Be, Ga, dE, dAl, dBe, dGa;
            delo_coef_d(P(D, j), E, Al, Be, Ga, dE, dAl, dBe, dGa);
            P(GD, j) += gY * (P(YS, j + 1) * dE + y(j) * dAl + y(j + 1) * dBe + P(U, j) * dGa);
            P(GU, j) += gY * Ga;
            gY = gY * E;
        }
        for (int j = 0; j <= N - 2; j++) {                 // U_j -> D_j, R_j, R_j+1
            const double gu = P(GU, j);
            P(GD, j) += gu * 0.25 * (P(R, j) - P(R, j + 1));
            P(GR, j) += gu * 0.25 * P(D, j);
            P(GR, j + 1) -= gu * 0.25 * P(D, j);
        }
        P(GD, 0) -= P(GR, 0) * P(R, 0) / P(D, 0);          // CentDer -> D
        P(GD, N - 2) -= P(GR, N - 1) * P(R, N - 1) / P(D, N - 2);
        for (int j = 1; j <= N - 2; j++) {
            const double Dx = P(D, j - 1), Dx1 = P(D, j);
            const double Der = (y(j) - y(j - 1)) / Dx, Der1 = (y(j + 1) - y(j)) / Dx1;
            if (!(Der * Der1 > 0.0)) continue;
            double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0, Yp, dDer, dDer1, dLam;
            hmean_d(Der, Der1, Lambda, Yp, dDer, dDer1, dLam);
            const double sm = Dx + Dx1, g = P(GR, j);
            P(GD, j - 1) += g * (dDer * (-Der / Dx) + dLam * (-Dx1 / (3.0 * sm * sm)));
            P(GD, j) += g * (dDer1 * (-Der1 / Dx1) + dLam * (Dx / (3.0 * sm * sm)));
        }
        {                                                  // TauStep -> the opacity of each ray point's layer
            const double Dx1 = m[1] - m[0];
            L(GX, mp[0]) += P(GD, 0) * 0.5 * Dx1;
            L(GX, mp[1]) += P(GD, 0) * 0.5 * Dx1;
        }
        for (int j = 1; j <= N - 2; j++) {
            const double Dx = m[j] - m[j - 1], Dx1 = m[j + 1] - m[j];
            const double Der = (x(j) - x(j - 1)) / Dx, Der1 = (x(j + 1) - x(j)) / Dx1;
            const double g = P(GD, j);
            L(GX, mp[j + 1]) += g * Dx1 / 3.0;
            L(GX, mp[j]) += g * 2.0 * Dx1 / 3.0;
            if (Der * Der1 > 0.0) {
                double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0, Yp, dDer, dDer1, dLam;
                hmean_d(Der, Der1, Lambda, Yp, dDer, dDer1, dLam);
                const double c = g * Dx1 * Dx1 / 6.0;
                L(GX, mp[j + 1]) += c * dDer1 / Dx1;
                L(GX, mp[j]) += c * (dDer / Dx - dDer1 / Dx1);
                L(GX, mp[j - 1]) += c * (-dDer / Dx);
            }
        }
    }
    for (int t = 0; t < nt; t++) {
        gkappa[(size_t)w * nt + t] = L(GX, t);
        gk32[(size_t)t * nwl + w] = (float)L(GX, t);
    }
    const double wv = A.wave[w];
    wvh[w] = (float)wv;
    wvl[w] = (float)(wv - (double)wvh[w]);
}

size_t fsg_line_adjoint_work(int, int, int64_t);
int fsg_launch_line_adjoint(cudaStream_t, const AtmView &, const LineView &, const VoigtTables &, const int32_t *,
                            const int32_t *, const int32_t *, const double *, const float *, const float *,
                            const float *, double, double *, double *, void *, int, int);

// solver work (10 x nt x nwl doubles; SPH_WORK x nt x nwl for spherical models), dL/dkappa in FP32,
// the wavelength offsets as FP32 hi + lo, then the line pass's workspace
static size_t solver_doubles(int nwl, int nt, int sph) { return (size_t)(sph ? SPH_WORK : 10) * nt * nwl; }
static size_t solver_part(int nwl, int nt, int sph) {
    return (sizeof(double) * solver_doubles(nwl, nt, sph) + sizeof(float) * ((size_t)nt * nwl + 2 * (size_t)nwl) +
            255) & ~(size_t)255;
}

size_t fsg_adjoint_work(int nwl, int nt, int64_t n, int sph) {
    return solver_part(nwl, nt, sph) + fsg_line_adjoint_work(nwl, nt, n) + 256;
}

// rays: the spherical model's rays (nmu = 0: plane-parallel)
int fsg_launch_adjoint(cudaStream_t s, const AtmView &A, const LineView &L, const VoigtTables &T,
                       const double *lineopac, const double *rhox, int nmu, const double *xmu, const double *wmu,
                       const RayView &rays, const int32_t *flags, const int32_t *ileft, const int32_t *iright,
                       const double *gflux, double *gkappa, double *work, double vmic, double *glin, double *gvmic,
                       int i0, int i1) {
    const int sph = rays.nmu > 0;
    float *gk32 = (float *)(work + solver_doubles(A.nwl, A.ntau, sph)), *wvh = gk32 + (size_t)A.ntau * A.nwl;
    float *wvl = wvh + A.nwl;
    if (sph)
        k_solver_adjoint_sph<<<(A.nwl + 127) / 128, 128, 0, s>>>(A, lineopac, rays, wmu, gflux, gkappa, work, gk32,
                                                                  wvh, wvl);
    else
        k_solver_adjoint<<<(A.nwl + 127) / 128, 128, 0, s>>>(A, lineopac, rhox, nmu, xmu, wmu, gflux, gkappa, work,
                                                              gk32, wvh, wvl);
    if (cudaGetLastError() != cudaSuccess) return FSG_E_CUDA;
    if (L.n > 0)
        return fsg_launch_line_adjoint(s, A, L, T, flags, ileft, iright, gkappa, gk32, wvh, wvl, vmic, glin, gvmic,
                                       (char *)work + solver_part(A.nwl, A.ntau, sph), i0, i1);
    return FSG_OK;
}
