// sacc.cuh -- the saCC variant of Spalart-Allmaras (saCC.c, `saCC 1` with `sa 1`): the SA diffusion and
// source with the density-gradient terms of the conservative form, in the reference's operation order.
// Face diffusion (saCC_InterFace, saCC.c:18-99: always the averaged face gradients), cell source
// (saCC_InterSource 102-137 with saCC_CalcSource 167-237) and boundary viscous fluxes
// (saCC_BoundaryFaceViscFlux 257-588).
#pragma once
#include "sa.cuh"

namespace csu {

// saCC_CalcFace (saCC.c:146-165)
__device__ __forceinline__ void sacc_face(double ni, double ni_L, double r, double dnix, double dniy, double drx,
                                          double dry, double* fv1, double* tx, double* ty)
{
    double aux;
    double Cv1 = 7.1;
    double X = ni / ni_L;
    aux = X * X * X;
    *fv1 = aux / (aux + Cv1 * Cv1 * Cv1);
    double sig = 2. / 3.;
    *tx = (r * (ni_L + ni) * dnix + 0.5 * ni * ni * drx) / sig;
    *ty = (r * (ni_L + ni) * dniy + 0.5 * ni * ni * dry) / sig;
}

// saCC_CalcSource (saCC.c:167-237); its diagnostic print of a negative modified vorticity is not reproduced
__device__ __forceinline__ double sacc_source(double ni, double ni_L, double S, double d, double rho, double drx,
                                              double dry, double dnix, double dniy)
{
    double aux;
    double Cv1 = 7.1;
    double X = ni / ni_L;
    aux = X * X * X;
    double fv1 = aux / (aux + Cv1 * Cv1 * Cv1);
    double k = 0.41;
    double fv2 = 1. - X / (1. + X * fv1);
    double Sbar = ni * fv2 / (k * k * d * d);
    double Stil;
    double cv2 = 0.7;
    double cv3 = 0.9;
    if (Sbar >= -cv2 * S) {
        Stil = S + Sbar;
    } else {
        double aux2 = ((cv3 - 2 * cv2) * S - Sbar);
        if (aux2 == 0) Stil = S;
        else Stil = S + S * (cv2 * cv2 * S + cv3 * Sbar) / aux2;
    }
    // as in sa_source: a negative value, reachable only by rounding a denormal S, is taken as +0
    if (Stil < 0.0) Stil = 0.0;
    double sig = 2. / 3.;
    double Cb1 = 0.1355;
    double Cb2 = 0.622;
    double Cw1 = Cb1 / (k * k) + (1. + Cb2) / sig;
    double Cw2 = 0.3;
    double r = ni / (Stil * k * k * d * d);
    r = fmin(r, 10);
    aux = r * r;
    aux = aux * aux * aux;
    double g = r + Cw2 * (aux - r);
    double Cw3 = 2.;
    aux = Cw3 * Cw3;
    aux = aux * aux * aux;
    double fw = g * pow((1. + aux) / (g * g * g * g * g * g + aux), 1. / 6.);
    double Qt = rho * (Cb1 * Stil * ni + Cb2 * (dnix * dnix + dniy * dniy) / sig - Cw1 * fw * (ni * ni / (d * d)));
    Qt += (Cb2 / sig) * (ni * (dnix * drx + dniy * dry) + 0.25 * ni * ni * (drx * drx + dry * dry) / rho);
    return Qt;
}

// One interior face of saCC_InterFace: viscous flux components 1..4 and the face eddy viscosity.
// g0/g1: gradients of u, v, T, nt, rho of e0/e1 (x then y); P0/P1 primitives r u v p T nt.
__device__ __forceinline__ void sacc_face_flux(const Gas& g, double Pr, double Prt, const double* g0x,
                                               const double* g0y, const double* g1x, const double* g1y,
                                               const double* P0, const double* P1, double dSx, double dSy,
                                               double* fv, double* miT)
{
    double drx = (g0x[4] + g1x[4]) * 0.5;
    double dux = (g0x[0] + g1x[0]) * 0.5;
    double dvx = (g0x[1] + g1x[1]) * 0.5;
    double dTx = (g0x[2] + g1x[2]) * 0.5;
    double dnx = (g0x[3] + g1x[3]) * 0.5;
    double dry = (g0y[4] + g1y[4]) * 0.5;
    double duy = (g0y[0] + g1y[0]) * 0.5;
    double dvy = (g0y[1] + g1y[1]) * 0.5;
    double dTy = (g0y[2] + g1y[2]) * 0.5;
    double dny = (g0y[3] + g1y[3]) * 0.5;
    double r = (P1[0] + P0[0]) * 0.5;
    double u = (P1[1] + P0[1]) * 0.5;
    double v = (P1[2] + P0[2]) * 0.5;
    double T = (P1[4] + P0[4]) * 0.5;
    double n = (P1[5] + P0[5]) * 0.5;
    double mi_L = sutherland(T);
    double n_L = mi_L / r;
    double fv1, tx, ty;
    sacc_face(n, n_L, r, dnx, dny, drx, dry, &fv1, &tx, &ty);
    double mi_t = fv1 * r * n;
    double mi = mi_L + mi_t;
    double k = T2Cp(g, T) * (mi_L / Pr + mi_t / Prt);
    *miT = mi_t;
    double txx = 2 * mi * (dux - (dux + dvy) / 3);
    double tyy = 2 * mi * (dvy - (dux + dvy) / 3);
    double txy = mi * (duy + dvx);
    fv[0] = txx * dSx + txy * dSy;
    fv[1] = txy * dSx + tyy * dSy;
    fv[2] = (txx * dSx + txy * dSy) * u + (txy * dSx + tyy * dSy) * v + k * (dTx * dSx + dTy * dSy);
    fv[3] = tx * dSx + ty * dSy;
}

// saCC_BoundaryFaceViscFlux (saCC.c:257-588): components 1..4 of one boundary face, subtracted from the
// owner. gx/gy: owner gradients of u, v, T, nt, rho. P: owner primitives. pin: inlet primitives.
__device__ __forceinline__ void sacc_boundary_flux(const Gas& g, double Pr, double Prt, double Twall,
                                                   const double* pin, int flag, const double* gx, const double* gy,
                                                   const double* P, double dSx, double dSy, double dx, double dy,
                                                   double L, double nx, double ny, double dS2, double* f)
{
    double dux, duy, dvx, dvy, dTx, dTy, dnx, dny, drx, dry;
    if (flag == 0) {
        // symmetry: the nt and rho gradients only reach tx, ty, which this branch does not use
        double duxm = gx[0], dvxm = gx[1], dTxm = gx[2];
        double duym = gy[0], dvym = gy[1], dTym = gy[2];
        dux = duxm - (duxm * nx + duym * ny) * nx;
        duy = duym - (duxm * nx + duym * ny) * ny;
        dvx = dvxm - (dvxm * nx + dvym * ny) * nx;
        dvy = dvym - (dvxm * nx + dvym * ny) * ny;
        dTx = dTxm - (dTxm * nx + dTym * ny) * nx;
        dTy = dTym - (dTxm * nx + dTym * ny) * ny;
        double rho = P[0], u = P[1], v = P[2], T = P[4], n = P[5];
        double mi_L = sutherland(T);
        double n_L = mi_L / rho;
        double fv1, tx, ty;
        sacc_face(n, n_L, rho, 0.0, 0.0, 0.0, 0.0, &fv1, &tx, &ty);
        double mi_t = fv1 * rho * n;
        double mi = mi_L + mi_t;
        double k = T2Cp(g, T) * (mi_L / Pr + mi_t / Prt);
        double txx = 2 * mi * (dux - (dux + dvy) / 3);
        double tyy = 2 * mi * (dvy - (dux + dvy) / 3);
        double txy = mi * (duy + dvx);
        f[0] = (txx * nx + txy * ny) * dS2;
        f[1] = (txy * nx + tyy * ny) * dS2;
        f[2] = (u * (txx * nx + txy * ny) + v * (txy * nx + tyy * ny) + k * (dTx * nx + dTy * ny)) * dS2;
        f[3] = 0.0;
        return;
    }
    if (flag == 1 || flag == 3 || flag == 4) {
        double ub = flag == 1 ? pin[1] : 0.0, vb = flag == 1 ? pin[2] : 0.0, nb = flag == 1 ? pin[5] : 0.0;
        double dul = (ub - P[1]) / L;
        double dvl = (vb - P[2]) / L;
        double dnl = (nb - P[5]) / L;
        double duxm = gx[0], dvxm = gx[1], dnxm = gx[3];
        double duym = gy[0], dvym = gy[1], dnym = gy[3];
        if (flag == 1) {
            double drl = (pin[0] - P[0]) / L;
            double drxm = gx[4], drym = gy[4];
            drx = drxm + (drl - (drxm * dx + drym * dy) / L) * dx / L;
            dry = drym + (drl - (drxm * dx + drym * dy) / L) * dy / L;
        } else {
            // the wall branch takes dry from the x gradient (saCC.c:423-424), the isothermal one from y
            drx = gx[4];
            dry = flag == 3 ? gx[4] : gy[4];
        }
        dux = duxm + (dul - (duxm * dx + duym * dy) / L) * dx / L;
        duy = duym + (dul - (duxm * dx + duym * dy) / L) * dy / L;
        dvx = dvxm + (dvl - (dvxm * dx + dvym * dy) / L) * dx / L;
        dvy = dvym + (dvl - (dvxm * dx + dvym * dy) / L) * dy / L;
        if (flag != 3) {
            double Tb = flag == 1 ? pin[4] : Twall;
            double dTl = (Tb - P[4]) / L;
            double dTxm = gx[2], dTym = gy[2];
            dTx = dTxm + (dTl - (dTxm * dx + dTym * dy) / L) * dx / L;
            dTy = dTym + (dTl - (dTxm * dx + dTym * dy) / L) * dy / L;
        }
        dnx = dnxm + (dnl - (dnxm * dx + dnym * dy) / L) * dx / L;
        dny = dnym + (dnl - (dnxm * dx + dnym * dy) / L) * dy / L;
        double rho = flag == 1 ? pin[0] : P[0];
        double T = flag == 1 ? pin[4] : (flag == 4 ? Twall : P[4]);
        double n = flag == 1 ? pin[5] : 0.0;
        double mi_L = sutherland(T);
        double n_L = mi_L / rho;
        double fv1, tx, ty;
        sacc_face(n, n_L, rho, dnx, dny, drx, dry, &fv1, &tx, &ty);
        double mi, k = 0.0;
        if (flag == 3) {
            mi = mi_L;
        } else {
            double mi_t = fv1 * rho * n;
            mi = mi_L + mi_t;
            k = T2Cp(g, T) * (mi_L / Pr + mi_t / Prt);
        }
        double txx = 2 * mi * (dux - (dux + dvy) / 3);
        double tyy = 2 * mi * (dvy - (dux + dvy) / 3);
        double txy = mi * (duy + dvx);
        f[0] = txx * dSx + txy * dSy;
        f[1] = txy * dSx + tyy * dSy;
        if (flag == 1) {
            double u = pin[1], v = pin[2];
            f[2] = u * (txx * dSx + txy * dSy) + v * (txy * dSx + tyy * dSy) + k * (dTx * dSx + dTy * dSy);
        } else if (flag == 4) {
            f[2] = k * (dTx * dSx + dTy * dSy);
        } else {
            f[2] = 0.0;
        }
        f[3] = tx * dSx + ty * dSy;
        return;
    }
    dux = gx[0]; dvx = gx[1]; dTx = gx[2]; dnx = gx[3]; drx = gx[4];
    duy = gy[0]; dvy = gy[1]; dTy = gy[2]; dny = gy[3]; dry = gy[4];
    double rho = P[0], u = P[1], v = P[2], T = P[4], n = P[5];
    double mi_L = sutherland(T);
    double n_L = mi_L / rho;
    double fv1, tx, ty;
    sacc_face(n, n_L, rho, dnx, dny, drx, dry, &fv1, &tx, &ty);
    double mi_t = fv1 * rho * n;
    double mi = mi_L + mi_t;
    double k = T2Cp(g, T) * (mi_L / Pr + mi_t / Prt);
    double txx = 2 * mi * (dux - (dux + dvy) / 3);
    double tyy = 2 * mi * (dvy - (dux + dvy) / 3);
    double txy = mi * (duy + dvx);
    f[0] = txx * dSx + txy * dSy;
    f[1] = txy * dSx + tyy * dSy;
    f[2] = u * (txx * dSx + txy * dSy) + v * (txy * dSx + tyy * dSy) + k * (dTx * dSx + dTy * dSy);
    f[3] = tx * dSx + ty * dSy;
}

} // namespace csu
