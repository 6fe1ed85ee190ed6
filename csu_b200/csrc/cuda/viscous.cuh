// viscous.cuh -- laminar Navier-Stokes terms (laminar.c) and wall friction (boundary.c:695-742), as device
// functions with the reference's operation order. Face gradients are the average of the two cell
// gradients corrected along the centroid-to-centroid direction (laminar.c:33-59); the stress tensor uses
// Sutherland's law at the face temperature and the heat flux k = Cp mu / Pr.
#pragma once
#include "physics.cuh"

namespace csu {

// gasprop_T2Cp (gasprop.c:144-147)
__device__ __forceinline__ double T2Cp(const Gas& g, double T)
{
    return T2Cv(g, T) + g.R;
}

// laminarInter face part (laminar.c:20-74): viscous flux of one interior face, components 1..3 (x, y
// momentum, energy), to be subtracted from e0 and added to e1.
//   g0/g1: gradients of u, v, T of e0/e1 (x then y); P0/P1: primitives; d = x_e1 - x_e0, L = |d|
__device__ __forceinline__ void laminar_face(const Gas& g, double Pr, const double* g0x, const double* g0y,
                                             const double* g1x, const double* g1y, const double* P0,
                                             const double* P1, double dx, double dy, double L, double dSx,
                                             double dSy, double* fv)
{
    double duxm = (g0x[0] + g1x[0]) * 0.5;
    double dvxm = (g0x[1] + g1x[1]) * 0.5;
    double dTxm = (g0x[2] + g1x[2]) * 0.5;
    double duym = (g0y[0] + g1y[0]) * 0.5;
    double dvym = (g0y[1] + g1y[1]) * 0.5;
    double dTym = (g0y[2] + g1y[2]) * 0.5;
    double dul = (P1[1] - P0[1]) / L;
    double dvl = (P1[2] - P0[2]) / L;
    double dTl = (P1[4] - P0[4]) / L;
    double dux = duxm + (dul - (duxm * dx + duym * dy) / L) * dx / L;
    double duy = duym + (dul - (duxm * dx + duym * dy) / L) * dy / L;
    double dvx = dvxm + (dvl - (dvxm * dx + dvym * dy) / L) * dx / L;
    double dvy = dvym + (dvl - (dvxm * dx + dvym * dy) / L) * dy / L;
    double dTx = dTxm + (dTl - (dTxm * dx + dTym * dy) / L) * dx / L;
    double dTy = dTym + (dTl - (dTxm * dx + dTym * dy) / L) * dy / L;
    double T = (P1[4] + P0[4]) * 0.5;
    double mi = sutherland(T);
    double k = T2Cp(g, T) * mi / Pr;
    double txx = 2 * mi * (dux - (dux + dvy) / 3);
    double tyy = 2 * mi * (dvy - (dux + dvy) / 3);
    double txy = mi * (duy + dvx);
    double u = (P1[1] + P0[1]) * 0.5;
    double v = (P1[2] + P0[2]) * 0.5;
    fv[0] = txx * dSx + txy * dSy;
    fv[1] = txy * dSx + tyy * dSy;
    fv[2] = (txx * dSx + txy * dSy) * u + (txy * dSx + tyy * dSy) * v + k * (dTx * dSx + dTy * dSy);
}

// boundaryFaceViscFlux (laminar.c:128-346): viscous flux of one boundary face (components 1..3), to be
// subtracted from the owner. gx/gy: owner gradients of u, v, T. dx, dy, L: face midpoint minus owner
// centroid. nx, ny, dS2: unit normal and length of meshCalcDS2 (mesh.c:742-764, used by symmetry faces).
// For adiabatic walls (flag 3) the reference leaves the energy component unset (an uninitialised local,
// laminar.c:104-115 with 230-268); it is zero here: no heat flux and no wall velocity.
__device__ __forceinline__ void laminar_boundary(const Gas& g, double Pr, double Twall, const double* pin,
                                                 int flag, const double* gx, const double* gy, const double* P,
                                                 double dSx, double dSy, double dx, double dy, double L,
                                                 double nx, double ny, double dS2, double* f)
{
    double dux, duy, dvx, dvy, dTx, dTy;
    if (flag == 0) {
        double duxm = gx[0], dvxm = gx[1], dTxm = gx[2];
        double duym = gy[0], dvym = gy[1], dTym = gy[2];
        dux = duxm - (duxm * nx + duym * ny) * nx;
        duy = duym - (duxm * nx + duym * ny) * ny;
        dvx = dvxm - (dvxm * nx + dvym * ny) * nx;
        dvy = dvym - (dvxm * nx + dvym * ny) * ny;
        dTx = dTxm - (dTxm * nx + dTym * ny) * nx;
        dTy = dTym - (dTxm * nx + dTym * ny) * ny;
        double T = P[4];
        double mi = sutherland(T);
        double k = T2Cp(g, T) * mi / Pr;
        double txx = 2 * mi * (dux - (dux + dvy) / 3);
        double tyy = 2 * mi * (dvy - (dux + dvy) / 3);
        double txy = mi * (duy + dvx);
        double u = P[1], v = P[2];
        f[0] = (txx * nx + txy * ny) * dS2;
        f[1] = (txy * nx + tyy * ny) * dS2;
        f[2] = (u * (txx * nx + txy * ny) + v * (txy * nx + tyy * ny) + k * (dTx * nx + dTy * ny)) * dS2;
    } else if (flag == 1 || flag == 3 || flag == 4) {
        double ub = flag == 1 ? pin[1] : 0.0, vb = flag == 1 ? pin[2] : 0.0;
        double dul = (ub - P[1]) / L;
        double dvl = (vb - P[2]) / L;
        double duxm = gx[0], dvxm = gx[1], duym = gy[0], dvym = gy[1];
        dux = duxm + (dul - (duxm * dx + duym * dy) / L) * dx / L;
        duy = duym + (dul - (duxm * dx + duym * dy) / L) * dy / L;
        dvx = dvxm + (dvl - (dvxm * dx + dvym * dy) / L) * dx / L;
        dvy = dvym + (dvl - (dvxm * dx + dvym * dy) / L) * dy / L;
        double T = flag == 4 ? Twall : P[4];
        double mi = sutherland(T);
        double txx = 2 * mi * (dux - (dux + dvy) / 3);
        double tyy = 2 * mi * (dvy - (dux + dvy) / 3);
        double txy = mi * (duy + dvx);
        f[0] = txx * dSx + txy * dSy;
        f[1] = txy * dSx + tyy * dSy;
        if (flag == 3) {
            f[2] = 0.0;
        } else {
            double Tb = flag == 1 ? pin[4] : Twall;
            double dTl = (Tb - P[4]) / L;
            double dTxm = gx[2], dTym = gy[2];
            dTx = dTxm + (dTl - (dTxm * dx + dTym * dy) / L) * dx / L;
            dTy = dTym + (dTl - (dTxm * dx + dTym * dy) / L) * dy / L;
            double k = T2Cp(g, T) * mi / Pr;
            if (flag == 1) {
                double u = P[1], v = P[2];
                f[2] = u * (txx * dSx + txy * dSy) + v * (txy * dSx + tyy * dSy) + k * (dTx * dSx + dTy * dSy);
            } else {
                f[2] = k * (dTx * dSx + dTy * dSy);
            }
        }
    } else {
        dux = gx[0]; dvx = gx[1]; dTx = gx[2];
        duy = gy[0]; dvy = gy[1]; dTy = gy[2];
        double T = P[4];
        double mi = sutherland(T);
        double k = T2Cp(g, T) * mi / Pr;
        double txx = 2 * mi * (dux - (dux + dvy) / 3);
        double tyy = 2 * mi * (dvy - (dux + dvy) / 3);
        double txy = mi * (duy + dvx);
        double u = P[1], v = P[2];
        f[0] = txx * dSx + txy * dSy;
        f[1] = txy * dSx + tyy * dSy;
        f[2] = u * (txx * dSx + txy * dSy) + v * (txy * dSx + tyy * dSy) + k * (dTx * dSx + dTy * dSy);
    }
}

// boundaryCalcFrictionWall (boundary.c:695-742): wall shear force of one wall face
__device__ __forceinline__ void friction_wall(const double* gx, const double* gy, const double* P, double dSx,
                                              double dSy, double dx, double dy, double L, double* fx, double* fy)
{
    double dul = (0 - P[1]) / L;
    double dvl = (0 - P[2]) / L;
    double duxm = gx[0], dvxm = gx[1], duym = gy[0], dvym = gy[1];
    double dux = duxm + (dul - (duxm * dx + duym * dy) / L) * dx / L;
    double duy = duym + (dul - (duxm * dx + duym * dy) / L) * dy / L;
    double dvx = dvxm + (dvl - (dvxm * dx + dvym * dy) / L) * dx / L;
    double dvy = dvym + (dvl - (dvxm * dx + dvym * dy) / L) * dy / L;
    double T = P[4];
    double mi = sutherland(T);
    double txx = 2 * mi * (dux - (dux + dvy) / 3);
    double tyy = 2 * mi * (dvy - (dux + dvy) / 3);
    double txy = mi * (duy + dvx);
    *fx = txx * dSx + txy * dSy;
    *fy = txy * dSx + tyy * dSy;
}

// viscous spectral radius factor fmax(4/(3 r), gamma(T)/r) (mi/Pr) of implicit.c:76, 143, 265, 804
__device__ __forceinline__ double visc_radius(const Gas& g, double Pr, double r, double T)
{
    double mi = sutherland(T);
    return fmax(4 / (3 * r), T2gamma(g, T) / r) * (mi / Pr);
}

} // namespace csu
