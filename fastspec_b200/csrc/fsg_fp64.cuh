// fsg_fp64.cuh -- FP64 device functions restating voigt.f90 / opacity.f90 / solver.f90.
// Included only by translation units built with -fmad=false: every a*b+c below must stay an
// unfused multiply and add, as the reference's SSE2 build evaluates it.
#pragma once
#include "fsg_internal.cuh"

// ---- Voigt table lerp, FP64 (voigt.f90:76-110, 113-154) -------------------------------------
// The v-difference of two FP32 table entries is taken in FP32, as the REAL(4) operands of the
// reference's expression VgtTab(iv+2,ia) - VgtTab(iv+1,ia).
__device__ __forceinline__ double hv_asym64(double A, double av) {
    double a2 = A * A, v2 = av * av, s = v2 + a2;
    if (s >= 196.0) return FSG_SQRTPIINV * A * (s + 0.5) / (s * s - v2 + a2 + 0.25);
    double p = v2 - a2 - 1.5, q = 2.0 * av * A;
    double dr = av * p - A * q, di = av * q + A * p;
    return FSG_SQRTPIINV * ((p + 0.5) * di - q * dr) / (dr * dr + di * di);
}

__device__ __forceinline__ double hvoigt64(const float *__restrict__ tab, const double *__restrict__ anode,
                                           const double *__restrict__ aida, double A, double V) {
    const double IDv = 1.0 / (8.0 / 1000.0);
    const double IDt = 1.0 / (2.8284271247461903 / 400.0);
    double av = fabs(V);
    if (A < 8.0 && av < 8.0) {
        double fv = av * IDv; int iv = (int)fv; double tv = fv - (double)iv, ua; int ia;
        if (A < anode[1]) { ia = 1; ua = A * aida[0]; }
        else { ia = (int)(sqrt(A) * IDt) + 1; ua = (A - anode[ia - 1]) * aida[ia - 1]; }
        const float *c0p = tab + (ia - 1) * FSG_NV1 + iv, *c1p = c0p + FSG_NV1;
        float t00 = __ldg(c0p), t01 = __ldg(c0p + 1), t10 = __ldg(c1p), t11 = __ldg(c1p + 1);
        double c0 = (double)t00 + tv * (double)(t01 - t00);
        double c1 = (double)t10 + tv * (double)(t11 - t10);
        return c0 + ua * (c1 - c0);
    }
    return hv_asym64(A, av);
}

// FVoigt / FVoigtLine (voigt.f90:256-352)
__device__ __forceinline__ void fv_asym64(double A, double av, double *vgt, double *fvgt) {
    double a2 = A * A, v2 = av * av, s = v2 + a2, w;
    if (s >= 196.0) {
        w = FSG_SQRTPIINV / (s * s - v2 + a2 + 0.25);
        *vgt = w * A * (s + 0.5); *fvgt = w * av * (s - 0.5);
    } else {
        double p = v2 - a2 - 1.5, q = 2.0 * av * A;
        double dr = av * p - A * q, di = av * q + A * p;
        w = FSG_SQRTPIINV / (dr * dr + di * di);
        *vgt = w * ((p + 0.5) * di - q * dr); *fvgt = w * ((p + 0.5) * dr + q * di);
    }
}

struct VLine64 { double A, UA; int IA; };
__device__ __forceinline__ VLine64 vline64(const double *anode, const double *aida, double A) {
    const double IDt = 1.0 / (2.8284271247461903 / 400.0);
    VLine64 L; L.A = A;
    if (A < 8.0) { L.IA = (int)(sqrt(A) * IDt) + 1; L.UA = (A - anode[L.IA - 1]) * aida[L.IA - 1]; }
    else { L.IA = 0; L.UA = 0.0; }
    return L;
}
__device__ __forceinline__ double hvoigt_line64(const float *__restrict__ tab, VLine64 L, double V) {
    const double IDv = 1.0 / (8.0 / 1000.0);
    double av = fabs(V);
    if (L.IA > 0 && av < 8.0) {
        double fv = av * IDv; int iv = (int)fv; double tv = fv - (double)iv;
        const float *c0p = tab + (L.IA - 1) * FSG_NV1 + iv, *c1p = c0p + FSG_NV1;
        float t00 = __ldg(c0p), t01 = __ldg(c0p + 1), t10 = __ldg(c1p), t11 = __ldg(c1p + 1);
        double c0 = (double)t00 + tv * (double)(t01 - t00);
        double c1 = (double)t10 + tv * (double)(t11 - t10);
        return c0 + L.UA * (c1 - c0);
    }
    return hv_asym64(L.A, av);
}
__device__ __forceinline__ void fvoigt_line64(const float2 *__restrict__ ftab, VLine64 L, double V,
                                              double *vgt, double *fvgt) {
    const double IDv = 1.0 / (8.0 / 1000.0);
    double av = fabs(V);
    if (L.IA > 0 && av < 8.0) {
        double fv = av * IDv; int iv = (int)fv; double tv = fv - (double)iv;
        const float2 *c0p = ftab + (L.IA - 1) * FSG_NV1 + iv, *c1p = c0p + FSG_NV1;
        float2 t00 = __ldg(c0p), t01 = __ldg(c0p + 1), t10 = __ldg(c1p), t11 = __ldg(c1p + 1);
        double h0 = (double)t00.x + tv * (double)(t01.x - t00.x);
        double h1 = (double)t10.x + tv * (double)(t11.x - t10.x);
        double l0 = (double)t00.y + tv * (double)(t01.y - t00.y);
        double l1 = (double)t10.y + tv * (double)(t11.y - t10.y);
        *vgt = h0 + L.UA * (h1 - h0); *fvgt = l0 + L.UA * (l1 - l0);
    } else fv_asym64(L.A, av, vgt, fvgt);
    *fvgt = copysign(fabs(*fvgt), V);
}

// ---- grid ---------------------------------------------------------------------------------
// first index i in [0, n) with w[i] >= x (n when none)
__device__ __forceinline__ int lower_index(const double *__restrict__ w, int n, double x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int m = (lo + hi) >> 1;
        if (w[m] < x) lo = m + 1; else hi = m;
    }
    return lo;
}

// WaveIdx (opacity.f90:594-608); 1-based
__device__ __forceinline__ int waveidx(const AtmView &A, double wavein) {
    if (A.wmode == 0) {
        double X = fmin(fmax(wavein / A.dstep, 0.0), (double)(A.nwl - 2));
        return (int)X + 1;
    }
    double X = 1.0 + log(fmax((wavein / A.wstart) + 1.0, 2.2250738585072014e-308)) / A.rstep;
    return (int)fmin(fmax(X, 1.0), (double)(A.nwl - 1));
}

// Air2Vac (utils.f90:1020-1032)
__device__ __forceinline__ double air2vac(double la) {
    double S = 1e4 / la, S2 = S * S;
    double N = 1.0 + 8.336624212083e-5 + 2.408926869968e-2 / (1.301065924522e2 - S2) +
               1.599740894897e-4 / (3.892568793293e1 - S2);
    return (la > 1999.352) ? la * N : la;
}

// ---- line opacity kernel (opacity.f90:96-293) -----------------------------------------------
__device__ __forceinline__ double xln_c() { return FSG_VC * 1e13; }

// joint flag bits set by the drivers before XlineSetup (synth.f90:837-845, 1185-1188)
__device__ __forceinline__ int line_input_flags(const LineView &L, int64_t i, int mag) {
    int f = 0;
    if (L.kind == 0) { if (L.gvdw[i] > 10.0f) f |= FSG_F_ABO; }
    else if (L.kind == 2) {
        if (L.ismol && L.ismol[i]) f |= FSG_F_MOL;
        if (L.gvdw[i] > 10.0f) f |= FSG_F_ABO;
    }
    (void)mag;
    return f;
}

// XlineSetup (opacity.f90:96-235)
__device__ __forceinline__ void xline_setup(const AtmView &A, const LineView &L, int64_t i,
                                            double wlc, int flag, XCoef *XC) {
    double WaveL = wlc + A.wfirst;
    double Elo = (double)L.elo[i];
    XC->WaveL = WaveL; XC->Elo = Elo; XC->Gf = (double)L.gf[i];
    double GradL = (double)L.grad[i], GqstL, GvdwL; int IsMol;
    int ispc = L.spc[i]; int IonL = A.ion[ispc]; XC->IxPF = ispc;
    if (L.kind == 0) { GqstL = (double)L.gqst[i]; GvdwL = (double)L.gvdw[i]; IsMol = 0; }
    else if (L.kind == 1) { GqstL = 0.0; GvdwL = 0.0; IsMol = 1; }
    else { GqstL = (double)L.gqst[i]; GvdwL = (double)L.gvdw[i]; IsMol = (flag >> 1) & 1; }
    const double c = xln_c();
    XC->Hnux = c * FSG_HC / WaveL;
    const double XlnDop = 2.0 * FSG_KBOLT / (FSG_M0 * 1e3) * 1e16;
    XC->Xmass = XlnDop / c / c / (double)A.xamass[ispc];
    XC->Grad = (GradL > 0.0) ? GradL : 0.22233e16 / (WaveL * WaveL);
    XC->Cqst = 0.0; XC->Qdiv = 1.0; XC->Cvdw = 0.0; XC->AboPre = 0.0; XC->AboVbc = 0.0;
    XC->AboExp = 0.0; XC->IxHe = 0;
    if (IsMol && !A.molbrd) { XC->MdQst = 9; XC->MdVdw = 9; }
    else {
        double Wavevac = air2vac(WaveL);
        double Eup = Elo + 1.0 / (Wavevac * FSG_EV2ANG);
        double pot = (double)A.potion[ispc];
        double t1 = (double)(IonL * IonL) * FSG_HIE / (pot - Eup);
        double t2 = (double)(IonL * IonL) * FSG_HIE / (pot - Elo);
        double Enu4 = t1 * t1, Enl4 = t2 * t2;
        if (L.ihe && ispc == A.spc_he1) XC->IxHe = L.ihe[i];
        if (XC->IxHe > 0) XC->MdQst = 3;
        else if (GqstL > 0.0) { XC->MdQst = 0; XC->Cqst = GqstL; }
        else if (IsMol) XC->MdQst = 9;
        else if (IonL == 1) { XC->MdQst = 1; XC->Cqst = 2.26e-07 * Enu4; }
        else { XC->MdQst = 2; XC->Cqst = 5.42e-07 * Enu4;
               XC->Qdiv = ((double)IonL + 1.0) * ((double)IonL + 1.0); }
        if ((flag >> 2) & 1) {
            XC->MdVdw = 2;
            double Sigma = FSG_A0 * FSG_A0 * (double)(int)GvdwL;
            double Alpha = GvdwL - (double)(int)GvdwL;
            double X = 2.0 - Alpha * 0.5, Gx = X - 1.0;
            double GammaF = 1.0 + (-0.5748646 + (0.9512363 + (-0.6998588 +
                            (0.4245549 - 0.1010678 * Gx) * Gx) * Gx) * Gx) * Gx;
            XC->AboPre = 2e6 * (pow(4.0 / FSG_PI, Alpha * 0.5) * GammaF * 1e4 * Sigma);
            XC->AboVbc = 1.0 / 1.00794 + 1.0 / (double)A.xamass[ispc];
            XC->AboExp = 1.0 - Alpha;
        } else if (GvdwL > 0.0) { XC->MdVdw = 0; XC->Cvdw = GvdwL; }
        else if (IsMol) XC->MdVdw = 9;
        else {
            XC->MdVdw = 1;
            double Cw = 1.61e-33 * fabs(Enu4 - Enl4) / (double)(IonL * IonL);
            XC->Cvdw = pow(Cw, 0.4);
        }
    }
    if (IsMol && A.vwmol > 0.0) { XC->MdVdw = 0; XC->Cvdw = A.vwmol; }
}

// LinCop alone (the first lines and the last two of XlineDepth, opacity.f90:247-253, 290-291)
__device__ __forceinline__ double xline_cop(const AtmView &A, int t, const XCoef &XC, double *dopl_out) {
    const double *xi = A.xi; int nt = A.ntau;
    double Xstim = 1.0 - exp(-XC.Hnux / xi[XI_KBT * nt + t]);
    double Efract = exp(-XC.Elo / xi[XI_KBET * nt + t]);
    double Dopl = sqrt(xi[XI_T * nt + t] * XC.Xmass + A.vturb2);
    double Dndopl = Dopl / XC.WaveL;
    *dopl_out = Dopl;
    const double XlnZ = sqrt(FSG_PI) * (FSG_CE * FSG_CE) / (FSG_ME * (FSG_VC * FSG_VC)) * 1e-18;
    double c = XlnZ * Efract * XC.Gf * Xstim / (xi[XI_RHO * nt + t] * Dndopl);
    return c * (double)__ldg(A.fpf + (size_t)XC.IxPF * nt + t);
}

// Voigt parameters of XlineDepth (opacity.f90:250-287) given Dopl
__device__ __forceinline__ void xline_av(const AtmView &A, int t, const XCoef &XC, double Dopl,
                                         double *vv, double *av) {
    const double *xi = A.xi; int nt = A.ntau;
    double Dldopl = XC.WaveL * Dopl, Dndopl = Dopl / XC.WaveL;
    double Gqst, Gvdw;
    switch (XC.MdQst) {
        case 0: Gqst = XC.Cqst * xi[XI_TEMP6 * nt + t]; break;
        case 1: Gqst = XC.Cqst * xi[XI_XNE * nt + t]; break;
        case 2: Gqst = XC.Cqst * xi[XI_XNE * nt + t] / XC.Qdiv; break;
        case 3: Gqst = A.hegam[(XC.IxHe - 1) * nt + t]; break;
        default: Gqst = 0.0;
    }
    switch (XC.MdVdw) {
        case 0: Gvdw = XC.Cvdw * xi[XI_TEMP3 * nt + t]; break;
        case 1: Gvdw = A.vwfudge * xi[XI_GVWPRT * nt + t] * XC.Cvdw; break;
        case 2: {
            const double XlnKM0 = FSG_KBOLT * 1e-7 / FSG_M0;
            double Vbar = sqrt(8.0 * XlnKM0 * xi[XI_T * nt + t] / FSG_PI * XC.AboVbc);
            Gvdw = XC.AboPre * pow(Vbar / 1e4, XC.AboExp) * xi[XI_NPRTB * nt + t];
        } break;
        default: Gvdw = 0.0;
    }
    double Gamtot = XC.Grad + Gqst + Gvdw;
    const double XlnC4Pi = 4.0 * xln_c() * FSG_PI;
    *av = Gamtot / (Dndopl * XlnC4Pi);
    *vv = 1.0 / Dldopl;
}

// Full XlineDepth (opacity.f90:239-293)
__device__ __forceinline__ void xline_depth(const AtmView &A, int t, const XCoef &XC, double *cop,
                                            double *vv, double *av) {
    double Dopl;
    *cop = xline_cop(A, t, XC, &Dopl);
    xline_av(A, t, XC, Dopl, vv, av);
}

// Continuum at the line centre (synth.f90:870-874)
__device__ __forceinline__ double cont_center(const AtmView &A, int iwl, double dW, int t) {
    const double *c0 = A.contopac + (size_t)(iwl - 1) * A.ntau;
    return c0[t] * (1.0 - dW) + c0[A.ntau + t] * dW;
}

// ---- DELO-Bezier (solver.f90) -----------------------------------------------------------------
__device__ __forceinline__ void delo_coef(double Dtau, double &Eps, double &Alpha, double &Beta, double &Gamma) {
    double Dtau2 = Dtau * Dtau, Idtau2 = 1.0 / Dtau2;
    if (Dtau < 5e-3) {
        Eps = 1.0 - Dtau + 0.5 * Dtau2 - Dtau2 * Dtau / 6.0 + Dtau2 * Dtau2 / 24.0;
        Alpha = Dtau / 3.0 - Dtau2 / 12.0 + Dtau2 * Dtau / 60.0;
        Beta = Dtau / 3.0 - Dtau2 * 0.25 + Dtau2 * Dtau * 0.1;
        Gamma = Dtau / 3.0 - Dtau2 / 6.0 + Dtau2 * Dtau * 0.05;
    } else {
        Eps = (Dtau < 100.0) ? exp(-Dtau) : 0.0;
        Alpha = (Dtau2 - 2.0 * Dtau + 2.0 - 2.0 * Eps) * Idtau2;
        Beta = (2.0 - (2.0 + 2.0 * Dtau + Dtau2) * Eps) * Idtau2;
        Gamma = (2.0 * Dtau - 4.0 + (2.0 * Dtau + 4.0) * Eps) * Idtau2;
    }
}

// ---- spherical rays ---------------------------------------------------------------------------
// TauStep (solver.f90:591-615) at point j of a ray (mu = 1 on the ray's column mass m, opacity x by
// layer read through the map): the step from point j to j + 1, 0 <= j <= N - 2.
__device__ __forceinline__ double ray_taustep(const int *mp, const double *m, const double *x, int j) {
    if (j == 0) {
        double x0 = x[mp[0]], x1 = x[mp[1]];
        double Dx1 = m[1] - m[0], Yp = (x1 - x0) / Dx1;
        return Dx1 * (x1 + 2.0 * x0 + Dx1 / 2.0 * Yp) / 3.0;
    }
    double xa = x[mp[j - 1]], xb = x[mp[j]], xc = x[mp[j + 1]];
    double Dx = m[j] - m[j - 1], Dx1 = m[j + 1] - m[j];
    double Der = (xb - xa) / Dx, Der1 = (xc - xb) / Dx1, Yp;
    if (Der * Der1 > 0.0) {
        double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0;
        Yp = (Der / (Lambda * Der1 + (1.0 - Lambda) * Der)) * Der1;
    } else Yp = 0.0;
    return Dx1 * (xc + 2.0 * xb + Dx1 / 2.0 * Yp) / 3.0;
}

// CentDer (solver.f90:618-647) at an interior point from the steps on either side and three values
__device__ __forceinline__ double centder3(double Dx, double Dx1, double ya, double yb, double yc) {
    double InvDx = 1.0 / Dx, InvDx1 = 1.0 / Dx1;
    double Lambda = (1.0 + Dx1 / (Dx + Dx1)) / 3.0, Lambda1 = 1.0 - Lambda;
    double Der = (yb - ya) * InvDx, Der1 = (yc - yb) * InvDx1;
    return (Der * Der1 > 0.0) ? (Der / (Lambda * Der1 + Lambda1 * Der)) * Der1 : 0.0;
}

// LocPrfSph + DeloScalar (solver.f90:182-261) along ray im: opacity x and source y by layer.  The
// reference builds Deltau and Srd as arrays and then sweeps; here one backward pass computes each step,
// derivative and Bezier term U where the sweep reaches it, from the same operands, so the values are
// the same and no per-ray arrays are needed.  Grazing rays start from zero intensity at the far side.
__device__ __forceinline__ double delo_ray(const RayView &R, int im, const double *x, const double *y) {
    const int N = R.n[im];
    const int *mp = R.map + (size_t)im * R.stride;
    const double *m = R.m + (size_t)im * R.stride;
    double dcur = ray_taustep(mp, m, x, N - 2);                  // Deltau(N-1)
    double yhi = y[mp[N - 1]], ylo = y[mp[N - 2]];
    double srd_hi = (yhi - ylo) / dcur;                         // Srd(N)
    double Y = R.graz[im] ? 0.0 : yhi;
    for (int j = N - 2; j >= 0; j--) {
        double yj = y[mp[j]], yj1 = y[mp[j + 1]], srd_j, dprev = 0.0;
        if (j > 0) {
            dprev = ray_taustep(mp, m, x, j - 1);
            srd_j = centder3(dprev, dcur, y[mp[j - 1]], yj, yj1);
        } else srd_j = (yj1 - yj) / dcur;
        double Eps, Alpha, Beta, Gamma;
        delo_coef(dcur, Eps, Alpha, Beta, Gamma);
        double U = 0.5 * (yj + 0.5 * dcur * srd_j + yj1 - 0.5 * dcur * srd_hi);
        Y = Y * Eps + Alpha * yj + Beta * yj1 + Gamma * U;
        srd_hi = srd_j; dcur = dprev;
    }
    return Y;
}
