// sst.cuh -- Menter SST k-omega terms (sst.c) as device functions, in the reference's operation order:
// face diffusion (sstInterFace, sst.c:56-193, sstFlux 749-786), cell sources (sstInterSource 595-691,
// sstSources 698-747), blending functions (sstF1/sstF2 788-818) and boundary viscous fluxes
// (sstBoundaryFaceViscFlux 202-547).
#pragma once
#include "viscous.cuh"

namespace csu {

// constants of sstInit (sst.c:18-39); g1, g2 evaluated on the host with the reference's expressions
struct SstK {
    double sk1, so1, b1, sk2, so2, b2, bs, a1, g1, g2, o_wall_factor;
    int trans; // sstTrans 1: the low-Reynolds variant of sstTrans.c (sstTransFlux, sstTransSources)
};

struct SstVar {
    double dux, duy, dvx, dvy, dkx, dky, dox, doy;
    double r, T, k, om, d, mi_L, mi_t;
    double tkx, tky, tox, toy;
    double F1, F2, Qtk, Qto;
};

__device__ __forceinline__ double sst_blend(double x1, double x2, double F1)
{
    return x1 * F1 + x2 * (1 - F1);
}

// sstF1 (sst.c:788-809); its long double temporaries only ever hold double values
__device__ __forceinline__ double sst_F1(const SstK& c, const SstVar& v, double n_L_term, double sqrtk_term)
{
    double aux1, aux2;
    aux1 = 2 * v.r * c.so2 * (v.dkx * v.dox + v.dky * v.doy) / v.om;
    if (v.om == 0) aux1 = 0;
    double CD = fmax(aux1, 1.0e-20);
    aux1 = sqrtk_term;
    aux2 = n_L_term;
    aux1 = fmax(aux1, aux2);
    aux2 = 4 * v.r * c.so2 * v.k / (CD * v.d * v.d);
    double arg1 = fmin(aux1, aux2);
    return tanh(arg1 * arg1 * arg1 * arg1);
}

// sstF2 (sst.c:811-818)
__device__ __forceinline__ double sst_F2(double n_L_term, double sqrtk_term)
{
    double arg2 = fmax(2 * sqrtk_term, n_L_term);
    return tanh(arg2 * arg2);
}

// The sstTrans variant (sstTrans.c; constants of sstTransInit, lines 18-35, equal to sstInit's where the
// names agree: sk1 so1 b1 sk2 so2 b2, bs2 = bs, a1). Its Reynolds numbers are fixed at Ry = Rt = 1e6.
// sstTransF1 (sstTrans.c:120-139) is sstF1 without the omega = 0 guard.
__device__ __forceinline__ double sst_trans_F1(const SstK& c, const SstVar& v, double n_L_term, double sqrtk_term)
{
    double aux1, aux2;
    aux1 = 2 * v.r * c.so2 * (v.dkx * v.dox + v.dky * v.doy) / v.om;
    double CD = fmax(aux1, 1.0e-20);
    aux1 = sqrtk_term;
    aux2 = n_L_term;
    aux1 = fmax(aux1, aux2);
    aux2 = 4 * v.r * c.so2 * v.k / (CD * v.d * v.d);
    double arg1 = fmin(aux1, aux2);
    return tanh(arg1 * arg1 * arg1 * arg1);
}

// the blend factor F1 of the variant: max(F1s, exp(-(Ry / 120)^8)) (sstTrans.c:57-64, 146-153)
__device__ __forceinline__ double sst_trans_blend_F1(const SstK& c, const SstVar& v, double n_L_term,
                                                     double sqrtk_term)
{
    double Fs1 = sst_trans_F1(c, v, n_L_term, sqrtk_term);
    double Ry = 1e6;
    double aux = Ry / 120;
    aux = aux * aux;
    aux = aux * aux;
    aux = aux * aux;
    return fmax(Fs1, exp(-aux));
}

// sstTransFlux (sstTrans.c:42-81)
__device__ __forceinline__ void sst_trans_flux(const SstK& c, SstVar& v)
{
    double n_L = v.mi_L / v.r;
    double omega = fabs(v.duy - v.dvx);
    double sqrtk = sqrt(v.k);
    double sqrtk_term = sqrtk / (c.bs * v.om * v.d);
    double n_L_term = 500 * n_L / (v.d * v.d * v.om);
    double F1 = sst_trans_blend_F1(c, v, n_L_term, sqrtk_term);
    double F2 = sst_F2(n_L_term, sqrtk_term);
    double Rt = 1e6;
    double alphas1 = (.025 + Rt / 6) / (1 + Rt / 6);
    double alphas = sst_blend(alphas1, 1.0, F1);
    double sk = sst_blend(c.sk1, c.sk2, F1);
    double so = sst_blend(c.so1, c.so2, F1);
    v.mi_t = fmin(alphas * v.r * v.k / v.om, c.a1 * v.r * v.k / (omega * F2));
    double aux = (v.mi_L + sk * v.mi_t);
    v.tkx = aux * v.dkx;
    v.tky = aux * v.dky;
    aux = (v.mi_L + so * v.mi_t);
    v.tox = aux * v.dox;
    v.toy = aux * v.doy;
}

// sstTransSources (sstTrans.c:141-174, with sstTransAlpha1 / Alphas1 / Bs1)
__device__ __forceinline__ void sst_trans_sources(const SstK& c, SstVar& v)
{
    double n_L = v.mi_L / v.r;
    double omega = fabs(v.duy - v.dvx);
    double sqrtk = sqrt(v.k);
    double sqrtk_term = sqrtk / (c.bs * v.om * v.d);
    double n_L_term = 500 * n_L / (v.d * v.d * v.om);
    double F1 = sst_trans_blend_F1(c, v, n_L_term, sqrtk_term);
    double F2 = sst_F2(n_L_term, sqrtk_term);
    double Rt = 1e6;
    double alpha1 = (5. / 9.) * (0.1 + Rt / 2.7) / (1 + Rt / 2.7);
    double alphas1 = (.025 + Rt / 6) / (1 + Rt / 6);
    double a8 = Rt / 8;
    a8 = a8 * a8;
    a8 = a8 * a8;
    double bs1 = 0.09 * (5. / 18. + a8) / (1 + a8);
    double alpha = sst_blend(alpha1, 0.4403, F1);
    double alphas = sst_blend(alphas1, 1.0, F1);
    double b = sst_blend(c.b1, c.b2, F1);
    double bs = sst_blend(bs1, c.bs, F1);
    v.mi_t = fmin(alphas * v.r * v.k / v.om, c.a1 * v.r * v.k / (omega * F2));
    double n_t = v.mi_t / v.r;
    double P = v.mi_t * omega * omega;
    v.F1 = F1;
    v.F2 = F2;
    v.Qtk = P - bs * v.r * v.om * v.k;
    v.Qto = alpha * P / n_t - b * v.r * v.om * v.om + 2 * (1 - F1) * v.r * c.so2 * (v.dkx * v.dox + v.dky * v.doy) / v.om;
}

// sstFlux (sst.c:749-786): eddy viscosity and the k, omega diffusion fluxes
__device__ __forceinline__ void sst_flux(const SstK& c, SstVar& v)
{
    if (c.trans) {
        sst_trans_flux(c, v);
        return;
    }
    double n_L = v.mi_L / v.r;
    double omega = fabs(v.duy - v.dvx);
    double sqrtk_term = sqrt(v.k) / (c.bs * v.om * v.d);
    double n_L_term = 500 * n_L / (v.d * v.d * v.om);
    double F1 = sst_F1(c, v, n_L_term, sqrtk_term);
    double F2 = sst_F2(n_L_term, sqrtk_term);
    v.mi_t = v.r * c.a1 * v.k / fmax(c.a1 * v.om, omega * F2);
    double sk = sst_blend(c.sk1, c.sk2, F1);
    double so = sst_blend(c.so1, c.so2, F1);
    double aux;
    aux = (v.mi_L + sk * v.mi_t);
    v.tkx = aux * v.dkx;
    v.tky = aux * v.dky;
    aux = (v.mi_L + so * v.mi_t);
    v.tox = aux * v.dox;
    v.toy = aux * v.doy;
}

// sstSources (sst.c:698-747): Qtk, Qto per unit volume
__device__ __forceinline__ void sst_sources(const SstK& c, SstVar& v)
{
    if (c.trans) {
        sst_trans_sources(c, v);
        return;
    }
    double n_L = v.mi_L / v.r;
    double omega = fabs(v.duy - v.dvx);
    double sqrtk_term = sqrt(v.k) / (c.bs * v.om * v.d);
    double n_L_term = 500 * n_L / (v.d * v.d * v.om);
    double F1 = sst_F1(c, v, n_L_term, sqrtk_term);
    double F2 = sst_F2(n_L_term, sqrtk_term);
    v.mi_t = v.r * c.a1 * v.k / fmax(c.a1 * v.om, omega * F2);
    double n_t = v.mi_t / v.r;
    double g = sst_blend(c.g1, c.g2, F1);
    double b = sst_blend(c.b1, c.b2, F1);
    double txx = 2 * v.mi_t * (v.dux - (v.dux + v.dvy) / 3) - 2. * v.r * v.k / 3;
    double tyy = 2 * v.mi_t * (v.dvy - (v.dux + v.dvy) / 3) - 2. * v.r * v.k / 3;
    double txy = v.mi_t * (v.duy + v.dvx);
    double P = v.dux * txx + v.dvy * tyy + (v.duy + v.dvx) * txy;
    P = fmin(P, 10 * c.bs * v.r * v.om * v.k);
    v.F1 = F1;
    v.F2 = F2;
    double cd = 2 * (1 - F1) * v.r * c.so2 * (v.dkx * v.dox + v.dky * v.doy) / v.om;
    v.Qtk = P - c.bs * v.r * v.om * v.k;
    v.Qto = g * P / n_t - b * v.r * v.om * v.om + cd;
}

// stress and energy/turbulence fluxes shared by the face and boundary forms
__device__ __forceinline__ void sst_stress(const SstVar& v, double mi, double* txx, double* tyy, double* txy)
{
    *txx = 2 * mi * (v.dux - (v.dux + v.dvy) / 3) - 2. * v.r * v.k / 3.;
    *tyy = 2 * mi * (v.dvy - (v.dux + v.dvy) / 3) - 2. * v.r * v.k / 3.;
    *txy = mi * (v.duy + v.dvx);
}

// One interior face of sstInterFace: components 1..5 and the face eddy viscosity.
// g0/g1: gradients of u, v, T, k, w of e0/e1; P0/P1 primitives r u v p T k w; d0/d1 wall distances.
__device__ __forceinline__ void sst_face_flux(const Gas& g, const SstK& c, double Pr, double Prt, const double* g0x,
                                              const double* g0y, const double* g1x, const double* g1y,
                                              const double* P0, const double* P1, double d0, double d1, double dx,
                                              double dy, double L, double dSx, double dSy, double* fv, double* miT)
{
    SstVar v;
    double nx = dx / L;
    double ny = dy / L;
    double dul = (P1[1] - P0[1]) / L;
    double dvl = (P1[2] - P0[2]) / L;
    double dTl = (P1[4] - P0[4]) / L;
    double dkl = (P1[5] - P0[5]) / L;
    double dol = (P1[6] - P0[6]) / L;
    double duxm = 0.5 * (g0x[0] + g1x[0]);
    double dvxm = 0.5 * (g0x[1] + g1x[1]);
    double dTxm = 0.5 * (g0x[2] + g1x[2]);
    double dkxm = 0.5 * (g0x[3] + g1x[3]);
    double doxm = 0.5 * (g0x[4] + g1x[4]);
    double duym = 0.5 * (g0y[0] + g1y[0]);
    double dvym = 0.5 * (g0y[1] + g1y[1]);
    double dTym = 0.5 * (g0y[2] + g1y[2]);
    double dkym = 0.5 * (g0y[3] + g1y[3]);
    double doym = 0.5 * (g0y[4] + g1y[4]);
    double aux;
    aux = duxm * nx + duym * ny;
    v.dux = duxm + (dul - aux) * nx;
    v.duy = duym + (dul - aux) * ny;
    aux = dvxm * nx + dvym * ny;
    v.dvx = dvxm + (dvl - aux) * nx;
    v.dvy = dvym + (dvl - aux) * ny;
    aux = dTxm * nx + dTym * ny;
    double dTx = dTxm + (dTl - aux) * nx;
    double dTy = dTym + (dTl - aux) * ny;
    aux = dkxm * nx + dkym * ny;
    v.dkx = dkxm + (dkl - aux) * nx;
    v.dky = dkym + (dkl - aux) * ny;
    aux = doxm * nx + doym * ny;
    v.dox = doxm + (dol - aux) * nx;
    v.doy = doym + (dol - aux) * ny;
    v.r = (P1[0] + P0[0]) * 0.5;
    double u = (P1[1] + P0[1]) * 0.5;
    double w = (P1[2] + P0[2]) * 0.5;
    v.T = (P1[4] + P0[4]) * 0.5;
    v.k = (P1[5] + P0[5]) * 0.5;
    v.om = (P1[6] + P0[6]) * 0.5;
    v.d = (d1 + d0) * 0.5;
    v.mi_L = sutherland(v.T);
    sst_flux(c, v);
    double mi = v.mi_L + v.mi_t;
    double kk = T2Cp(g, v.T) * (v.mi_L / Pr + v.mi_t / Prt);
    *miT = v.mi_t;
    double txx, tyy, txy;
    sst_stress(v, mi, &txx, &tyy, &txy);
    fv[0] = txx * dSx + txy * dSy;
    fv[1] = txy * dSx + tyy * dSy;
    fv[2] = (txx * dSx + txy * dSy) * u + (txy * dSx + tyy * dSy) * w + kk * (dTx * dSx + dTy * dSy);
    fv[3] = v.tkx * dSx + v.tky * dSy;
    fv[4] = v.tox * dSx + v.toy * dSy;
}

// sstBoundaryFaceViscFlux (sst.c:202-547): components 1..5 of one boundary face, subtracted from the owner
__device__ __forceinline__ void sst_boundary_flux(const Gas& g, const SstK& c, double Pr, double Prt, double Twall,
                                                  const double* pin, int flag, const double* gx, const double* gy,
                                                  const double* P, double dwall, double dSx, double dSy, double dx,
                                                  double dy, double L, double nx, double ny, double dS2, double* f)
{
    SstVar v;
    double dTx = 0.0, dTy = 0.0, u = 0.0, w = 0.0;
    if (flag == 0) {
        double duxm = gx[0], dvxm = gx[1], dTxm = gx[2], dkxm = gx[3], doxm = gx[4];
        double duym = gy[0], dvym = gy[1], dTym = gy[2], dkym = gy[3], doym = gy[4];
        v.dux = duxm - (duxm * nx + duym * ny) * nx;
        v.duy = duym - (duxm * nx + duym * ny) * ny;
        v.dvx = dvxm - (dvxm * nx + dvym * ny) * nx;
        v.dvy = dvym - (dvxm * nx + dvym * ny) * ny;
        dTx = dTxm - (dTxm * nx + dTym * ny) * nx;
        dTy = dTym - (dTxm * nx + dTym * ny) * ny;
        v.dkx = dkxm - (dkxm * nx + dkym * ny) * nx;
        v.dky = dkym - (dkxm * nx + dkym * ny) * ny;
        v.dox = doxm - (doxm * nx + doym * ny) * nx;
        v.doy = doym - (doxm * nx + doym * ny) * ny;
        v.r = P[0];
        u = P[1];
        w = P[2];
        v.T = P[4];
        v.k = P[5];
        v.om = P[6];
        v.d = dwall;
        v.mi_L = sutherland(v.T);
        sst_flux(c, v);
        double mi = v.mi_L + v.mi_t;
        double txx, tyy, txy;
        sst_stress(v, mi, &txx, &tyy, &txy);
        f[0] = (txx * nx + txy * ny) * dS2;
        f[1] = (txy * nx + tyy * ny) * dS2;
        f[2] = (u * (txx * nx + txy * ny) + w * (txy * nx + tyy * ny)) * dS2;
        f[3] = 0.0;
        f[4] = 0.0;
        return;
    }
    if (flag == 2) {
        v.dux = gx[0]; v.dvx = gx[1]; dTx = gx[2]; v.dkx = gx[3]; v.dox = gx[4];
        v.duy = gy[0]; v.dvy = gy[1]; dTy = gy[2]; v.dky = gy[3]; v.doy = gy[4];
        v.r = P[0];
        u = P[1];
        w = P[2];
        v.T = P[4];
        v.k = P[5];
        v.om = P[6];
        v.d = dwall;
    } else {
        double ub, vb, Tb, kb, ob;
        if (flag == 1) {
            ub = pin[1]; vb = pin[2]; Tb = pin[4]; kb = pin[5]; ob = pin[6];
            v.r = pin[0]; u = pin[1]; w = pin[2]; v.T = pin[4]; v.k = pin[5]; v.om = pin[6];
            v.d = dwall;
        } else {
            v.r = P[0]; v.T = P[4]; v.k = P[5]; v.om = P[6];
            v.d = dwall;
            v.mi_L = sutherland(v.T);
            double n_L = v.mi_L / v.r;
            ub = 0.0; vb = 0.0; kb = 0.0; Tb = Twall;
            ob = c.o_wall_factor * 6 * n_L / (c.b1 * v.d * v.d);
        }
        double dul = (ub - P[1]) / L;
        double dvl = (vb - P[2]) / L;
        double dkl = (kb - P[5]) / L;
        double dol = (ob - P[6]) / L;
        double duxm = gx[0], dvxm = gx[1], dkxm = gx[3], doxm = gx[4];
        double duym = gy[0], dvym = gy[1], dkym = gy[3], doym = gy[4];
        v.dux = duxm + (dul - (duxm * dx + duym * dy) / L) * dx / L;
        v.duy = duym + (dul - (duxm * dx + duym * dy) / L) * dy / L;
        v.dvx = dvxm + (dvl - (dvxm * dx + dvym * dy) / L) * dx / L;
        v.dvy = dvym + (dvl - (dvxm * dx + dvym * dy) / L) * dy / L;
        if (flag != 3) {
            double dTl = (Tb - P[4]) / L;
            double dTxm = gx[2], dTym = gy[2];
            dTx = dTxm + (dTl - (dTxm * dx + dTym * dy) / L) * dx / L;
            dTy = dTym + (dTl - (dTxm * dx + dTym * dy) / L) * dy / L;
        }
        v.dkx = dkxm + (dkl - (dkxm * dx + dkym * dy) / L) * dx / L;
        v.dky = dkym + (dkl - (dkxm * dx + dkym * dy) / L) * dy / L;
        v.dox = doxm + (dol - (doxm * dx + doym * dy) / L) * dx / L;
        v.doy = doym + (dol - (doxm * dx + doym * dy) / L) * dy / L;
    }
    v.mi_L = sutherland(v.T);
    sst_flux(c, v);
    double mi = v.mi_L + v.mi_t;
    double txx, tyy, txy;
    sst_stress(v, mi, &txx, &tyy, &txy);
    f[0] = txx * dSx + txy * dSy;
    f[1] = txy * dSx + tyy * dSy;
    if (flag == 3) {
        f[2] = 0.0;
    } else {
        double kk = T2Cp(g, v.T) * (v.mi_L / Pr + v.mi_t / Prt);
        if (flag == 4) f[2] = kk * (dTx * dSx + dTy * dSy);
        else f[2] = u * (txx * dSx + txy * dSy) + w * (txy * dSx + tyy * dSy) + kk * (dTx * dSx + dTy * dSy);
    }
    f[3] = v.tkx * dSx + v.tky * dSy;
    f[4] = v.tox * dSx + v.toy * dSy;
}

// sstInterSource for one cell (sst.c:600-641): the sources subtracted from R[4], R[5] (zero when omega
// sits at its lower limit 0). g: cell gradients of u, v, k, w (x, y).
__device__ __forceinline__ void sst_cell_source(const SstK& c, const double* gx, const double* gy, const double* P,
                                                double d, double* Qtk, double* Qto)
{
    SstVar v;
    v.dux = gx[0]; v.dvx = gx[1]; v.dkx = gx[2]; v.dox = gx[3];
    v.duy = gy[0]; v.dvy = gy[1]; v.dky = gy[2]; v.doy = gy[3];
    v.r = P[0];
    v.T = P[4];
    v.k = P[5];
    v.om = P[6];
    v.d = d;
    v.mi_L = sutherland(v.T);
    if (v.om == 0.0) {
        *Qtk = 0.0;
        *Qto = 0.0;
        return;
    }
    sst_sources(c, v);
    *Qtk = v.Qtk;
    *Qto = v.Qto;
}

// sstInterSource's source Jacobians for LU-SGS (sst.c:643-680): forward differences of Qtk, Qto in omega,
// k and rho (step max(|x| 1e-6, 1e-6), the variable record reused between evaluations as there), combined
// into derivatives with respect to rho, rho k and rho omega and multiplied by the cell area. J: dQk/dr,
// dQk/d(rk), dQk/d(ro), dQo/dr, dQo/d(rk), dQo/d(ro); all zero when omega sits at its lower limit 0.
__device__ __forceinline__ void sst_source_jacobians(const SstK& c, const double* gx, const double* gy,
                                                     const double* P, double d, double area, double* J)
{
    SstVar v;
    v.dux = gx[0]; v.dvx = gx[1]; v.dkx = gx[2]; v.dox = gx[3];
    v.duy = gy[0]; v.dvy = gy[1]; v.dky = gy[2]; v.doy = gy[3];
    v.r = P[0];
    v.T = P[4];
    v.k = P[5];
    v.om = P[6];
    v.d = d;
    v.mi_L = sutherland(v.T);
    if (v.om == 0.0) {
        for (int q = 0; q < 6; q++) J[q] = 0.0;
        return;
    }
    sst_sources(c, v);
    const double Qk0 = v.Qtk, Qo0 = v.Qto;
    const double h = 1e-6, dh = 1e-6;
    double hh = fmax(fabs(v.om * h), dh);
    v.om += hh;
    sst_sources(c, v);
    const double dQkdo = (v.Qtk - Qk0) / hh, dQodo = (v.Qto - Qo0) / hh;
    v.om = P[6];
    hh = fmax(fabs(v.k * h), dh);
    v.k += hh;
    sst_sources(c, v);
    const double dQkdk = (v.Qtk - Qk0) / hh, dQodk = (v.Qto - Qo0) / hh;
    v.k = P[5];
    hh = fmax(fabs(v.r * h), dh);
    v.r += hh;
    sst_sources(c, v);
    const double dQkdr = (v.Qtk - Qk0) / hh, dQodr = (v.Qto - Qo0) / hh;
    v.r = P[0];
    J[0] = (dQkdr - dQkdk * v.k / v.r - dQkdo * v.om / v.r) * area;
    J[1] = dQkdk * area / v.r;
    J[2] = dQkdo * area / v.r;
    J[3] = (dQodr - dQodk * v.k / v.r - dQodo * v.om / v.r) * area;
    J[4] = dQodk * area / v.r;
    J[5] = dQodo * area / v.r;
}

} // namespace csu
