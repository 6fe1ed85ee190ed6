// physics.cuh -- pointwise physics of the CSU residual path, as device functions.
//
// Every function mirrors one reference function (file:line given) with the same floating-point
// operations in the same order; the library is compiled with --fmad=false and IEEE division/sqrt,
// so for identical inputs these return the reference's doubles bit for bit (libm transcendental
// functions aside). Arrays P[] use the reference's primitive layout r, u, v, p, T, (nt | k, w).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace csu {

// Thermally perfect polynomial of gaspropInit (gasprop.c:28-35): e(T) = sum cc[i] T^i.
__device__ __constant__ static const double TP_CC[6] = {1.81716e3, 9.890504e2 - 287.0530, -9.595592e-3,
                                                         1.041469e-4, -4.433065e-8, 5.879263e-12};

struct Gas {
    double gamma, R, Cp, Cv;
    int tp;
};

// gasprop_T2e (gasprop.c:47-69)
__device__ __forceinline__ double T2e(const Gas& g, double T)
{
    if (g.tp) {
        double P = 1, aux = TP_CC[0];
#pragma unroll
        for (int ii = 1; ii < 6; ii++) {
            P *= T;
            aux += TP_CC[ii] * P;
        }
        return aux;
    }
    return g.Cv * T;
}

// gasprop_T2Cv (gasprop.c:71-94)
__device__ __forceinline__ double T2Cv(const Gas& g, double T)
{
    if (g.tp) {
        double P = 1, aux = TP_CC[1];
#pragma unroll
        for (int ii = 2; ii < 6; ii++) {
            P *= T;
            aux += ii * TP_CC[ii] * P;
        }
        return aux;
    }
    return g.Cv;
}

// gasprop_T2eCv (gasprop.c:96-112)
__device__ __forceinline__ void T2eCv(double T, double* e, double* Cv)
{
    double P = 1;
    *e = TP_CC[0];
    *Cv = TP_CC[1];
#pragma unroll
    for (int ii = 1; ii < 6; ii++) {
        P *= T;
        *e += TP_CC[ii] * P;
        if (ii + 1 < 6) *Cv += (ii + 1) * TP_CC[ii + 1] * P;
    }
}

// gasprop_e2T (gasprop.c:114-136): Newton on the polynomial, at most 8 steps
__device__ __forceinline__ double e2T(const Gas& g, double e)
{
    double T = e / g.Cv;
    if (g.tp) {
        double error = 1, e1, Cv;
        int ii = 0;
        while ((fabs(error) > 1e-14) & (ii < 8)) {
            T2eCv(T, &e1, &Cv);
            error = (e - e1) / Cv;
            T += error;
            ii++;
        }
    }
    return T;
}

// gasprop_T2gamma (gasprop.c:150-154) and gasprop_T2c (138-141)
__device__ __forceinline__ double T2gamma(const Gas& g, double T)
{
    double Cv = T2Cv(g, T);
    return (Cv + g.R) / Cv;
}

__device__ __forceinline__ double T2c(const Gas& g, double T)
{
    return sqrt(T2gamma(g, T) * g.R * T);
}

// gasprop_e2Taprox (gasprop.c:156-159)
__device__ __forceinline__ double e2Taprox(const Gas& g, double e0, double T0, double e1)
{
    return T0 + (e1 - e0) / T2Cv(g, T0);
}

// gasprop_critic_H2c (gasprop.c:212-244) with gasprop_critic_T2entalpyDer (200-209)
__device__ __forceinline__ double critic_H2c(const Gas& g, double H)
{
    double c2 = 2 * (g.gamma - 1) * H / (g.gamma + 1);
    if (g.tp) {
        double T = c2 / (g.gamma * g.R), e, Cv, H0, dHdT, error;
        int ii = 0;
        T2eCv(T, &e, &Cv);
        {
            double RT = g.R * T, gam = (Cv + g.R) / Cv;
            H0 = e + RT + gam * RT * 0.5;
            dHdT = Cv + g.R + gam * g.R * 0.5;
        }
        error = (H - H0) / dHdT;
        T += error;
        while ((fabs(error) > 1.0e-12) & (ii < 3)) {
            T2eCv(T, &e, &Cv);
            double RT = g.R * T, gam = (Cv + g.R) / Cv;
            H0 = e + RT + gam * RT * 0.5;
            dHdT = Cv + g.R + gam * g.R * 0.5;
            error = (H - H0) / dHdT;
            T += error;
            ii++;
        }
        return T2c(g, T);
    }
    return sqrt(c2);
}

// sutherland (solver.c:1222-1225)
__device__ __forceinline__ double sutherland(double T)
{
    return 1.458e-6 * T * sqrt(T) / (T + 110.4);
}

// rotation (solver.c:441-448): velocity into the face frame (dSy negated rotates back)
__device__ __forceinline__ void rotation(double* U, double dSx, double dSy, double dS)
{
    double aux = (U[1] * dSx + U[2] * dSy) / dS;
    U[2] = (-U[1] * dSy + U[2] * dSx) / dS;
    U[1] = aux;
}

// limiterV2 (limiter.c:121-147): Venkatakrishnan-type limiter of one cell edge
__device__ __forceinline__ double limiterV2(double Ui, double Umin, double Umax, double d2, double ee)
{
    double ans;
    double d1max = Umax - Ui;
    double d1min = Umin - Ui;
    if (d2 == 0) {
        ans = 1;
    } else if (d2 > 0) {
        ans = (d1max * d1max + ee) * d2 + 2 * d2 * d2 * d1max;
        ans /= d1max * d1max + 2 * d2 * d2 + d1max * d2 + ee;
        ans /= d2;
    } else {
        ans = (d1min * d1min + ee) * d2 + 2 * d2 * d2 * d1min;
        ans /= d1min * d1min + 2 * d2 * d2 + d1min * d2 + ee;
        ans /= d2;
    }
    return ans;
}

// ---------------------------------------------------------------------------------------------
// Riemann fluxes in the face frame (flux.c). MODEL: 0 Euler (4 vars), 1 SA (5), 2 SST (6).
// L/R arrays hold r, u, v, p, then the transported scalars (nt | k, w).
// ---------------------------------------------------------------------------------------------

// entropyFix (flux.c:48-57)
__device__ __forceinline__ void entropyFix(double eFix, double* l)
{
    if ((*l < eFix) & (*l > -eFix)) *l = 0.5 * (*l * *l / eFix + eFix);
}

// fluxRoe (flux.c:59-129); 4 variables only (flux_sa/flux_sst have no Roe branch)
__device__ __forceinline__ void fluxRoe(const Gas& g, double eFix, const double* L, const double* Rr, double* f)
{
    double rL = L[0], uL = L[1], vL = L[2], pL = L[3];
    double rR = Rr[0], uR = Rr[1], vR = Rr[2], pR = Rr[3];
    double U0L = rL;
    double U1L = rL * uL;
    double U2L = rL * vL;
    double U3L = pL / (g.gamma - 1) + (uL * uL + vL * vL) * rL / 2;
    double HL = (U3L + pL) / rL;
    double U0R = rR;
    double U1R = rR * uR;
    double U2R = rR * vR;
    double U3R = pR / (g.gamma - 1) + (uR * uR + vR * vR) * rR / 2;
    double HR = (U3R + pR) / rR;
    double rqL = sqrt(rL);
    double rqR = sqrt(rR);
    double ub = (rqL * uL + rqR * uR) / (rqL + rqR);
    double vb = (rqL * vL + rqR * vR) / (rqL + rqR);
    double Hb = (rqL * HL + rqR * HR) / (rqL + rqR);
    double ab = sqrt((g.gamma - 1) * (Hb - (ub * ub + vb * vb) / 2));
    double l1 = ub - ab;
    double l2 = ub;
    double l4 = ub;
    double l5 = ub + ab;
    double e1[4] = {1.0, ub - ab, vb, Hb - ub * ab};
    double e2v[4] = {0.0, 0.0, 1.0, vb};
    double e4[4] = {1.0, ub, vb, 0.5 * (ub * ub + vb * vb)};
    double e5[4] = {1.0, ub + ab, vb, Hb + ub * ab};
    double d1 = U0R - U0L;
    double d2 = U1R - U1L;
    double d3 = U2R - U2L;
    double d5 = U3R - U3L;
    double a4 = (Hb - (ub * ub + vb * vb)) * d1 + ub * d2 + vb * d3 - d5;
    a4 /= (ab * ab) / (g.gamma - 1);
    double a2v = d3 - d1 * vb;
    double a5 = ((d1 - a4) + (d2 - ub * d1) / ab) * 0.5;
    double a1 = ((d1 - a4) - (d2 - ub * d1) / ab) * 0.5;
    double fL[4] = {U1L, U1L * uL + pL, U1L * vL, uL * (U3L + pL)};
    double fR[4] = {U1R, U1R * uR + pR, U1R * vR, uR * (U3R + pR)};
    entropyFix(eFix, &l1);
    entropyFix(eFix, &l2);
    entropyFix(eFix, &l4);
    entropyFix(eFix, &l5);
#pragma unroll
    for (int ii = 0; ii < 4; ++ii)
        f[ii] = 0.5 * (fR[ii] + fL[ii] - a1 * fabs(l1) * e1[ii] - a2v * fabs(l2) * e2v[ii] - a4 * fabs(l4) * e4[ii] -
                       a5 * fabs(l5) * e5[ii]);
}

// Total energy per volume and enthalpy of a face state. SST adds k*r (AUSM, AUSM+up(2): flux.c:908,1073,
// 1191) except AUSMDV_sst, which adds k alone (flux.c:992) -- both kept as the reference has them.
template <int MODEL, bool KPLAIN>
__device__ __forceinline__ void energy(const Gas& g, const double* Q, double* T, double* H)
{
    double r = Q[0], u = Q[1], v = Q[2], p = Q[3];
    *T = p / (g.R * r);
    double U3 = T2e(g, *T) * r + (u * u + v * v) * r / 2;
    if constexpr (MODEL == 2) {
        if constexpr (KPLAIN) U3 = U3 + Q[4];
        else U3 = U3 + Q[4] * r;
    }
    *H = (U3 + p) / r;
}

// fluxAUSM (flux.c:132-203), fluxAUSM_sa (512-585), fluxAUSM_sst (901-976)
template <int MODEL>
__device__ __forceinline__ void fluxAUSM(const Gas& g, const double* L, const double* Rr, double* f)
{
    double TL, HL, TR, HR;
    energy<MODEL, false>(g, L, &TL, &HL);
    energy<MODEL, false>(g, Rr, &TR, &HR);
    double rL = L[0], uL = L[1], vL = L[2], pL = L[3];
    double rR = Rr[0], uR = Rr[1], vR = Rr[2], pR = Rr[3];
    double cL = T2c(g, TL);
    double cR = T2c(g, TR);
    double ML = uL / cL;
    double MR = uR / cR;
    double Mplus, Mminus, Pplus, Pminus, M2p, M2m;
    if (fabs(ML) >= 1) {
        Mplus = 0.5 * (ML + fabs(ML));
        Pplus = Mplus / ML;
    } else {
        M2p = 0.25 * (ML + 1) * (ML + 1);
        Mplus = M2p;
        Pplus = M2p * (2 - ML);
    }
    if (fabs(MR) >= 1) {
        Mminus = 0.5 * (MR - fabs(MR));
        Pminus = Mminus / MR;
    } else {
        M2m = -0.25 * (MR - 1) * (MR - 1);
        Mminus = M2m;
        Pminus = -M2m * (2 + MR);
    }
    double Mm = Mplus + Mminus;
    double pm = Pplus * pL + Pminus * pR;
    const double* S;
    if (Mm > 0) {
        f[0] = rL * cL * Mm;
        f[1] = f[0] * uL + pm;
        f[2] = f[0] * vL;
        f[3] = f[0] * HL;
        S = L;
    } else {
        f[0] = rR * cR * Mm;
        f[1] = f[0] * uR + pm;
        f[2] = f[0] * vR;
        f[3] = f[0] * HR;
        S = Rr;
    }
    if constexpr (MODEL >= 1) f[4] = f[0] * S[4];
    if constexpr (MODEL == 2) f[5] = f[0] * S[5];
}

// fluxAUSMDV (flux.c:206-287), fluxAUSMDV_sa (588-670), fluxAUSMDV_sst (979-1062)
template <int MODEL>
__device__ __forceinline__ void fluxAUSMDV(const Gas& g, const double* L, const double* Rr, double* f)
{
    constexpr int NV = MODEL == 0 ? 4 : (MODEL == 1 ? 5 : 6);
    double aux, TL, HL, TR, HR;
    energy<MODEL, true>(g, L, &TL, &HL);
    energy<MODEL, true>(g, Rr, &TR, &HR);
    double rL = L[0], uL = L[1], vL = L[2], pL = L[3];
    double rR = Rr[0], uR = Rr[1], vR = Rr[2], pR = Rr[3];
    double cL = T2c(g, TL);
    double cR = T2c(g, TR);
    double cm = fmax(cL, cR);
    double alphaL = (2.0 * pL / rL) / (pL / rL + pR / rR);
    double alphaR = (2.0 * pR / rR) / (pL / rL + pR / rR);
    double uLPlus, pLPlus;
    aux = 0.5 * (uL + fabs(uL));
    if (fabs(uL) < cm) {
        uLPlus = alphaL * (0.25 * (uL + cm) * (uL + cm) / cm - aux) + aux;
        pLPlus = 0.25 * pL * (uL + cm) * (uL + cm) * (2.0 - uL / cm) / (cm * cm);
    } else {
        uLPlus = aux;
        pLPlus = pL * aux / uL;
    }
    double uRMinus, pRMinus;
    aux = 0.5 * (uR - fabs(uR));
    if (fabs(uR) < cm) {
        uRMinus = alphaR * (-0.25 * (uR - cm) * (uR - cm) / cm - aux) + aux;
        pRMinus = 0.25 * pR * (uR - cm) * (uR - cm) * (2.0 + uR / cm) / (cm * cm);
    } else {
        uRMinus = aux;
        pRMinus = pR * aux / uR;
    }
    double rU = uLPlus * rL + uRMinus * rR;
    f[0] = rU;
    f[1] = (pLPlus + pRMinus);
    f[2] = 0.5 * (rU * (vR + vL) - fabs(rU) * (vR - vL));
    f[3] = 0.5 * (rU * (HR + HL) - fabs(rU) * (HR - HL));
#pragma unroll
    for (int kk = 4; kk < NV; kk++) f[kk] = 0.5 * (rU * (Rr[kk] + L[kk]) - fabs(rU) * (Rr[kk] - L[kk]));
    double f1AUSMD = 0.5 * (rU * (uR + uL) - fabs(rU) * (uR - uL));
    double f1AUSMV = uLPlus * rL * uL + uRMinus * rR * uR;
    double s = 0.5 * fmin(1, 10 * fabs(pR - pL) / fmin(pL, pR));
    f[1] += (0.5 + s) * f1AUSMV + (0.5 - s) * f1AUSMD;
    // entropy fix; caseA & ~caseB on 0/1 ints equals caseA && !caseB
    int caseA = (uL - cL < 0.0) & (uR - cR > 0.0);
    int caseB = (uL + cL < 0.0) & (uR + cR > 0.0);
    double psiL[NV], psiR[NV];
    psiL[0] = 1.0; psiL[1] = uL; psiL[2] = vL; psiL[3] = HL;
    psiR[0] = 1.0; psiR[1] = uR; psiR[2] = vR; psiR[3] = HR;
#pragma unroll
    for (int kk = 4; kk < NV; kk++) {
        psiL[kk] = L[kk];
        psiR[kk] = Rr[kk];
    }
    if (caseA & ~caseB) {
        aux = 0.125 * ((uR - cR) - (uL - cL));
#pragma unroll
        for (int kk = 0; kk < NV; kk++) f[kk] -= aux * (rR * psiR[kk] - rL * psiL[kk]);
    } else if (~caseA & caseB) {
        aux = 0.125 * ((uR + cR) - (uL + cL));
#pragma unroll
        for (int kk = 0; kk < NV; kk++) f[kk] -= aux * (rR * psiR[kk] - rL * psiL[kk]);
    }
}

// fluxAUSMpup (flux.c:290-398) / fluxAUSMpup2 (401-508) and their _sa (673-899) / _sst (1066-1297) forms.
// SECOND selects the AUSM+up2 pressure flux. SST takes a* from H - k (flux.c:1082,1201).
template <int MODEL, bool SECOND>
__device__ __forceinline__ void fluxAUSMpup(const Gas& g, double Minf, const double* L, const double* Rr, double* f)
{
    double TL, HL, TR, HR;
    energy<MODEL, false>(g, L, &TL, &HL);
    energy<MODEL, false>(g, Rr, &TR, &HR);
    double rL = L[0], uL = L[1], vL = L[2], pL = L[3];
    double rR = Rr[0], uR = Rr[1], vR = Rr[2], pR = Rr[3];
    double astar;
    if constexpr (MODEL == 2) astar = critic_H2c(g, HL - L[4]);
    else astar = critic_H2c(g, HL);
    double ahL = astar * astar / fmax(astar, fabs(uL));
    if constexpr (MODEL == 2) astar = critic_H2c(g, HR - Rr[4]);
    else astar = critic_H2c(g, HR);
    double ahR = astar * astar / fmax(astar, fabs(uR));
    double am = fmin(ahL, ahR);
    double Kp = 0.25;
    double Ku = 0.75;
    double sig = 1.0;
    double beta = 1.0 / 8.0;
    double ML = uL / am;
    double MR = uR / am;
    double Mbar = sqrt((uL * uL + uR * uR) / (2 * am * am));
    double M0 = sqrt(fmin(1, fmax(Mbar * Mbar, Minf * Minf)));
    double fa = M0 * (2 - M0);
    if (fa < 1e-3) fa = 1e-3;
    double alpha = (3.0 / 16.0) * (-4 + 5 * fa * fa);
    double rhom = 0.5 * (rL + rR);
    double Mplus, Mminus, Pplus, Pminus, M2p, M2m;
    if (fabs(ML) >= 1) {
        Mplus = 0.5 * (ML + fabs(ML));
        Pplus = Mplus / ML;
    } else {
        M2p = 0.25 * (ML + 1) * (ML + 1);
        M2m = -0.25 * (ML - 1) * (ML - 1);
        Mplus = M2p * (1 - 16 * beta * M2m);
        Pplus = M2p * ((2 - ML) - 16 * alpha * ML * M2m);
    }
    if (fabs(MR) >= 1) {
        Mminus = 0.5 * (MR - fabs(MR));
        Pminus = Mminus / MR;
    } else {
        M2p = 0.25 * (MR + 1) * (MR + 1);
        M2m = -0.25 * (MR - 1) * (MR - 1);
        Mminus = M2m * (1 + 16 * beta * M2p);
        Pminus = M2m * ((-2 - MR) + 16 * alpha * MR * M2p);
    }
    double Mm = Mplus + Mminus - (Kp / fa) * fmax(1 - sig * Mbar * Mbar, 0) * (pR - pL) / (rhom * am * am);
    double pm;
    if constexpr (SECOND) {
        pm = 0.5 * (pL + pR) + 0.5 * (Pplus - Pminus) * (pL - pR) +
             sqrt(0.5 * (uL * uL + vL * vL + uR * uR + vR * vR)) * (Pplus + Pminus - 1) * 0.5 * (pL + pR) / am;
    } else if constexpr (MODEL == 0) {
        pm = Pplus * pL + Pminus * pR - Ku * Pplus * Pminus * (rL + rR) * (fa * am) * (uR - uL);
    } else {
        pm = Pplus * pL + Pminus * pR - Ku * Pplus * Pminus * (rL + rR) * (am * fa) * (uR - uL);
    }
    double mm;
    if (Mm > 0) mm = am * Mm * rL;
    else mm = am * Mm * rR;
    const double* S;
    if (mm > 0) {
        f[0] = mm;
        f[1] = mm * uL + pm;
        f[2] = mm * vL;
        f[3] = mm * HL;
        S = L;
    } else {
        f[0] = mm;
        f[1] = mm * uR + pm;
        f[2] = mm * vR;
        f[3] = mm * HR;
        S = Rr;
    }
    if constexpr (MODEL >= 1) f[4] = mm * S[4];
    if constexpr (MODEL == 2) f[5] = mm * S[5];
}

// flux / flux_sa / flux_sst dispatch (flux.c:1300-1366)
template <int MODEL>
__device__ __forceinline__ void riemann(int scheme, const Gas& g, double eFix, double Minf, const double* L,
                                        const double* Rr, double* f)
{
    switch (scheme) {
    case 0:
        if constexpr (MODEL == 0) fluxRoe(g, eFix, L, Rr, f);
        if constexpr (MODEL == 1) {
            // extension: the reference's flux_sa has no Roe branch (flux.c:1325-1345); Roe for the mean flow,
            // the SA working variable carried by the Roe mass flux from the upwind side
            fluxRoe(g, eFix, L, Rr, f);
            f[4] = f[0] * (f[0] > 0.0 ? L[4] : Rr[4]);
        }
        break;
    case 1: fluxAUSM<MODEL>(g, L, Rr, f); break;
    case 2: fluxAUSMDV<MODEL>(g, L, Rr, f); break;
    case 3: fluxAUSMpup<MODEL, false>(g, Minf, L, Rr, f); break;
    default: fluxAUSMpup<MODEL, true>(g, Minf, L, Rr, f); break;
    }
}

// fluxFree (flux.c:1369-1380): pressure-dominated flux of a wall state
__device__ __forceinline__ void fluxFree(const Gas& g, const double* Q, double* f)
{
    double rL = Q[0], uL = Q[1], vL = Q[2], pL = Q[3];
    double TL = pL / (g.R * rL);
    double U3L = T2e(g, TL) * rL + (uL * uL + vL * vL) * rL / 2;
    double HL = (U3L + pL) / rL;
    f[0] = rL * uL;
    f[1] = rL * uL * uL + pL;
    f[2] = rL * uL * vL;
    f[3] = rL * uL * HL;
}

// ---------------------------------------------------------------- boundary states (boundary.c)

// boundaryInlet (boundary.c:17-51): Pa free stream, Pd domain
__device__ __forceinline__ void bcInlet(const Gas& g, const double* Pa, const double* Pd, double* Pb, double nx,
                                        double ny)
{
    double rd = Pd[0], ud = Pd[1], vd = Pd[2], pd = Pd[3];
    double T = pd / rd / g.R;
    double c0 = T2c(g, T);
    double m = sqrt(ud * ud + vd * vd) / c0;
    if (m < 1.) {
        double ra = Pa[0], ua = Pa[1], va = Pa[2], pa = Pa[3];
        double pb = 0.5 * (pa + pd - rd * c0 * (nx * (ua - ud) + ny * (va - vd)));
        double rb = ra + (pb - pa) / (c0 * c0);
        double ub = ua - nx * (pa - pb) / (rd * c0);
        double vb = va - ny * (pa - pb) / (rd * c0);
        Pb[0] = rb; Pb[1] = ub; Pb[2] = vb; Pb[3] = pb;
    } else {
        for (int ii = 0; ii < 4; ii++) Pb[ii] = Pa[ii];
    }
}

// limiterBJ (solver.c:1132-1150): Barth-Jespersen, min(1, (Umax - Ui) / d2) -- the minmod limiter function
// min(1, r) of the ratio of the largest admissible change to the reconstructed one. The reference defines
// it but never calls it; here it is selected by the limiterFunc extension.
__host__ __device__ __forceinline__ double limiterBJ(double Ui, double Umin, double Umax, double d2)
{
    if (d2 == 0) return 1.0;
    if (d2 > 0) return fmin(1.0, (Umax - Ui) / d2);
    return fmin(1.0, (Umin - Ui) / d2);
}

// boundaryOutlet (boundary.c:53-83)
__device__ __forceinline__ void bcOutlet(const Gas& g, double pout, const double* Pd, double* Pb, double nx,
                                         double ny)
{
    double rd = Pd[0], ud = Pd[1], vd = Pd[2], pd = Pd[3];
    double T = pd / rd / g.R;
    double c0 = T2c(g, T);
    double m = sqrt(ud * ud + vd * vd) / c0;
    if (m < 1.) {
        double pb = pout;
        double rb = rd + (pb - pd) / (c0 * c0);
        double ub = ud + nx * (pd - pb) / (rd * c0);
        double vb = vd + ny * (pd - pb) / (rd * c0);
        Pb[0] = rb; Pb[1] = ub; Pb[2] = vb; Pb[3] = pb;
    } else {
        for (int ii = 0; ii < 4; ii++) Pb[ii] = Pd[ii];
    }
}

// boundaryWall (boundary.c:121-141): slip-wall characteristic state
__device__ __forceinline__ void bcWall(const Gas& g, const double* Pd, double* Pb, double nx, double ny)
{
    double rd = Pd[0], ud = Pd[1], vd = Pd[2], pd = Pd[3];
    double T = pd / rd / g.R;
    double c0 = T2c(g, T);
    double pb = pd + rd * c0 * (nx * ud + ny * vd);
    double rb = rd + (pb - pd) / (c0 * c0);
    double ub = ud - nx * (nx * ud + ny * vd);
    double vb = vd - ny * (nx * ud + ny * vd);
    Pb[0] = rb; Pb[1] = ub; Pb[2] = vb; Pb[3] = pb;
}

} // namespace csu
