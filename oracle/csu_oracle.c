/*
 * csu_oracle.c -- TEST INFRASTRUCTURE ONLY: the checker of the CUDA engine, never part of the product.
 *
 * A sequential plain-C restatement of the reference's residual-and-update path for the inviscid
 * (Euler) model: one loop per reference loop, in the reference's cell/face order, on flat arrays
 * instead of ELEMENT pointer lists. Each function names the reference function (file:line) it
 * restates. Pinned against the reference itself (oracle/_ref, built from its sources) by
 * tests/test_oracle_pin.py.
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "csu_oracle.h"

struct orc {
    csu_config c;
    int nc, nf, nb, nv, nm;
    double* xy;
    int *npts, *nodes, *con, *nint, *f, *nei, *bface, *bflag;
    double *omega, *wall;
    double *U, *Uaux, *R, *P, *G, *dPx, *dPy, *phi, *ff, *dtL, *D, *dW0, *dW1, *A;
    double gam, Rg, Cp, Cv;
    double dt, volMax, Pref20[6];
    int dtLocal;
    double res[6];
};

/* ------------------------------------------------------------------ gas (gasprop.c) */
static double T2e(const orc* o, double T) { return o->Cv * T; }            /* gasprop.c:47-69 */
static double T2gamma(const orc* o, double T) { (void)T; return (o->Cv + o->Rg) / o->Cv; } /* 150-154 */
static double T2c(const orc* o, double T) { return sqrt(T2gamma(o, T) * o->Rg * T); }   /* 138-141 */
static double e2T(const orc* o, double e) { return e / o->Cv; }            /* 114-136 */
static double e2Taprox(const orc* o, double e0, double T0, double e1) { return T0 + (e1 - e0) / o->Cv; }
static double critic_H2c(const orc* o, double H)                           /* 212-244 */
{
    return sqrt(2 * (o->gam - 1) * H / (o->gam + 1));
}

static void rot(double* U, double sx, double sy, double s)                 /* solver.c:441-448 */
{
    double a = (U[1] * sx + U[2] * sy) / s;
    U[2] = (-U[1] * sy + U[2] * sx) / s;
    U[1] = a;
}

static void calc_ds(const orc* o, int p0, int p1, double* sx, double* sy)  /* mesh.c:720-740 */
{
    double x0 = o->xy[2 * p0], y0 = o->xy[2 * p0 + 1], x1 = o->xy[2 * p1], y1 = o->xy[2 * p1 + 1];
    *sx = y1 - y0;
    *sy = -(x1 - x0);
    if (o->c.axisymmetric == 1) {
        double y = (y0 + y1) / 2;
        *sx = (*sx) * y;
        *sy = (*sy) * y;
    }
}

static void center(const orc* o, int c, double* x, double* y)              /* mesh.c:371-386 */
{
    double sx = 0, sy = 0;
    for (int j = 0; j < o->npts[c]; j++) {
        sx += o->xy[2 * o->nodes[4 * c + j]];
        sy += o->xy[2 * o->nodes[4 * c + j] + 1];
    }
    *x = sx / o->npts[c];
    *y = sy / o->npts[c];
}

/* ------------------------------------------------------------------ fluxes (flux.c) */
static void efix(double e, double* l)                                      /* flux.c:48-57 */
{
    if ((*l < e) & (*l > -e)) *l = 0.5 * (*l * *l / e + e);
}

static void roe(const orc* o, const double* L, const double* R, double* f) /* flux.c:59-129 */
{
    double g1 = o->gam - 1;
    double rL = L[0], uL = L[1], vL = L[2], pL = L[3], rR = R[0], uR = R[1], vR = R[2], pR = R[3];
    double U1L = rL * uL, U2L = rL * vL, U3L = pL / g1 + (uL * uL + vL * vL) * rL / 2, HL = (U3L + pL) / rL;
    double U1R = rR * uR, U2R = rR * vR, U3R = pR / g1 + (uR * uR + vR * vR) * rR / 2, HR = (U3R + pR) / rR;
    double qL = sqrt(rL), qR = sqrt(rR);
    double ub = (qL * uL + qR * uR) / (qL + qR), vb = (qL * vL + qR * vR) / (qL + qR);
    double Hb = (qL * HL + qR * HR) / (qL + qR);
    double ab = sqrt(g1 * (Hb - (ub * ub + vb * vb) / 2));
    double l1 = ub - ab, l2 = ub, l4 = ub, l5 = ub + ab;
    double e1[4] = {1.0, ub - ab, vb, Hb - ub * ab}, e2[4] = {0.0, 0.0, 1.0, vb};
    double e4[4] = {1.0, ub, vb, 0.5 * (ub * ub + vb * vb)}, e5[4] = {1.0, ub + ab, vb, Hb + ub * ab};
    double d1 = rR - rL, d2 = U1R - U1L, d3 = U2R - U2L, d5 = U3R - U3L;
    double a4 = (Hb - (ub * ub + vb * vb)) * d1 + ub * d2 + vb * d3 - d5;
    a4 /= (ab * ab) / g1;
    double a2 = d3 - d1 * vb;
    double a5 = ((d1 - a4) + (d2 - ub * d1) / ab) * 0.5;
    double a1 = ((d1 - a4) - (d2 - ub * d1) / ab) * 0.5;
    double fL[4] = {U1L, U1L * uL + pL, U1L * vL, uL * (U3L + pL)};
    double fR[4] = {U1R, U1R * uR + pR, U1R * vR, uR * (U3R + pR)};
    efix(o->c.e_fix, &l1); efix(o->c.e_fix, &l2); efix(o->c.e_fix, &l4); efix(o->c.e_fix, &l5);
    for (int i = 0; i < 4; i++)
        f[i] = 0.5 * (fR[i] + fL[i] - a1 * fabs(l1) * e1[i] - a2 * fabs(l2) * e2[i] - a4 * fabs(l4) * e4[i] -
                      a5 * fabs(l5) * e5[i]);
}

static void state_TH(const orc* o, const double* Q, double* T, double* H)
{
    *T = Q[3] / (o->Rg * Q[0]);
    double U3 = T2e(o, *T) * Q[0] + (Q[1] * Q[1] + Q[2] * Q[2]) * Q[0] / 2;
    *H = (U3 + Q[3]) / Q[0];
}

static void ausm(const orc* o, const double* L, const double* R, double* f) /* flux.c:132-203 */
{
    double TL, HL, TR, HR;
    state_TH(o, L, &TL, &HL);
    state_TH(o, R, &TR, &HR);
    double cL = T2c(o, TL), cR = T2c(o, TR), ML = L[1] / cL, MR = R[1] / cR, Mp, Mm, Pp, Pm;
    if (fabs(ML) >= 1) { Mp = 0.5 * (ML + fabs(ML)); Pp = Mp / ML; }
    else { Mp = 0.25 * (ML + 1) * (ML + 1); Pp = Mp * (2 - ML); }
    if (fabs(MR) >= 1) { Mm = 0.5 * (MR - fabs(MR)); Pm = Mm / MR; }
    else { Mm = -0.25 * (MR - 1) * (MR - 1); Pm = -Mm * (2 + MR); }
    double M = Mp + Mm, pm = Pp * L[3] + Pm * R[3];
    if (M > 0) { f[0] = L[0] * cL * M; f[1] = f[0] * L[1] + pm; f[2] = f[0] * L[2]; f[3] = f[0] * HL; }
    else { f[0] = R[0] * cR * M; f[1] = f[0] * R[1] + pm; f[2] = f[0] * R[2]; f[3] = f[0] * HR; }
}

static void ausmdv(const orc* o, const double* L, const double* R, double* f) /* flux.c:206-287 */
{
    double TL, HL, TR, HR;
    state_TH(o, L, &TL, &HL);
    state_TH(o, R, &TR, &HR);
    double rL = L[0], uL = L[1], vL = L[2], pL = L[3], rR = R[0], uR = R[1], vR = R[2], pR = R[3];
    double cL = T2c(o, TL), cR = T2c(o, TR), cm = fmax(cL, cR);
    double aL = (2.0 * pL / rL) / (pL / rL + pR / rR), aR = (2.0 * pR / rR) / (pL / rL + pR / rR);
    double up, pp, um, pmn, x = 0.5 * (uL + fabs(uL));
    if (fabs(uL) < cm) {
        up = aL * (0.25 * (uL + cm) * (uL + cm) / cm - x) + x;
        pp = 0.25 * pL * (uL + cm) * (uL + cm) * (2.0 - uL / cm) / (cm * cm);
    } else { up = x; pp = pL * x / uL; }
    x = 0.5 * (uR - fabs(uR));
    if (fabs(uR) < cm) {
        um = aR * (-0.25 * (uR - cm) * (uR - cm) / cm - x) + x;
        pmn = 0.25 * pR * (uR - cm) * (uR - cm) * (2.0 + uR / cm) / (cm * cm);
    } else { um = x; pmn = pR * x / uR; }
    double rU = up * rL + um * rR;
    f[0] = rU;
    f[1] = (pp + pmn);
    f[2] = 0.5 * (rU * (vR + vL) - fabs(rU) * (vR - vL));
    f[3] = 0.5 * (rU * (HR + HL) - fabs(rU) * (HR - HL));
    double fD = 0.5 * (rU * (uR + uL) - fabs(rU) * (uR - uL)), fV = up * rL * uL + um * rR * uR;
    double s = 0.5 * fmin(1, 10 * fabs(pR - pL) / fmin(pL, pR));
    f[1] += (0.5 + s) * fV + (0.5 - s) * fD;
    int A = (uL - cL < 0.0) && (uR - cR > 0.0), B = (uL + cL < 0.0) && (uR + cR > 0.0);
    double psL[4] = {1.0, uL, vL, HL}, psR[4] = {1.0, uR, vR, HR};
    if (A && !B) {
        x = 0.125 * ((uR - cR) - (uL - cL));
        for (int k = 0; k < 4; k++) f[k] -= x * (rR * psR[k] - rL * psL[k]);
    } else if (!A && B) {
        x = 0.125 * ((uR + cR) - (uL + cL));
        for (int k = 0; k < 4; k++) f[k] -= x * (rR * psR[k] - rL * psL[k]);
    }
}

/* flux.c:290-508: AUSM+up (second == 0) and AUSM+up2 (second == 1) */
static void ausmpup(const orc* o, int second, const double* L, const double* R, double* f)
{
    double TL, HL, TR, HR;
    state_TH(o, L, &TL, &HL);
    state_TH(o, R, &TR, &HR);
    double rL = L[0], uL = L[1], vL = L[2], pL = L[3], rR = R[0], uR = R[1], vR = R[2], pR = R[3];
    double as = critic_H2c(o, HL), ahL = as * as / fmax(as, fabs(uL));
    as = critic_H2c(o, HR);
    double ahR = as * as / fmax(as, fabs(uR)), am = fmin(ahL, ahR);
    double Kp = 0.25, Ku = 0.75, sig = 1.0, beta = 1.0 / 8.0;
    double ML = uL / am, MR = uR / am, Mbar = sqrt((uL * uL + uR * uR) / (2 * am * am)), Mi = o->c.mach_inf;
    double M0 = sqrt(fmin(1, fmax(Mbar * Mbar, Mi * Mi)));
    double fa = M0 * (2 - M0);
    if (fa < 1e-3) fa = 1e-3;
    double alpha = (3.0 / 16.0) * (-4 + 5 * fa * fa), rhom = 0.5 * (rL + rR), Mp, Mm, Pp, Pm, a, b;
    if (fabs(ML) >= 1) { Mp = 0.5 * (ML + fabs(ML)); Pp = Mp / ML; }
    else {
        a = 0.25 * (ML + 1) * (ML + 1); b = -0.25 * (ML - 1) * (ML - 1);
        Mp = a * (1 - 16 * beta * b); Pp = a * ((2 - ML) - 16 * alpha * ML * b);
    }
    if (fabs(MR) >= 1) { Mm = 0.5 * (MR - fabs(MR)); Pm = Mm / MR; }
    else {
        a = 0.25 * (MR + 1) * (MR + 1); b = -0.25 * (MR - 1) * (MR - 1);
        Mm = b * (1 + 16 * beta * a); Pm = b * ((-2 - MR) + 16 * alpha * MR * a);
    }
    double M = Mp + Mm - (Kp / fa) * fmax(1 - sig * Mbar * Mbar, 0) * (pR - pL) / (rhom * am * am), pm;
    if (second)
        pm = 0.5 * (pL + pR) + 0.5 * (Pp - Pm) * (pL - pR) +
             sqrt(0.5 * (uL * uL + vL * vL + uR * uR + vR * vR)) * (Pp + Pm - 1) * 0.5 * (pL + pR) / am;
    else pm = Pp * pL + Pm * pR - Ku * Pp * Pm * (rL + rR) * (fa * am) * (uR - uL);
    double mm = M > 0 ? am * M * rL : am * M * rR;
    if (mm > 0) { f[0] = mm; f[1] = mm * uL + pm; f[2] = mm * vL; f[3] = mm * HL; }
    else { f[0] = mm; f[1] = mm * uR + pm; f[2] = mm * vR; f[3] = mm * HR; }
}

static void riemann(const orc* o, const double* L, const double* R, double* f) /* flux.c:1300-1323 */
{
    switch (o->c.flux) {
    case 0: roe(o, L, R, f); break;
    case 1: ausm(o, L, R, f); break;
    case 2: ausmdv(o, L, R, f); break;
    case 3: ausmpup(o, 0, L, R, f); break;
    default: ausmpup(o, 1, L, R, f); break;
    }
}

/* ------------------------------------------------------------------ boundaries (boundary.c) */
static void bc_inlet(const orc* o, const double* Pa, const double* Pd, double* Pb, double nx, double ny)
{   /* boundary.c:17-51 */
    double rd = Pd[0], ud = Pd[1], vd = Pd[2], pd = Pd[3];
    double c0 = T2c(o, pd / rd / o->Rg);
    if (sqrt(ud * ud + vd * vd) / c0 < 1.) {
        double pb = 0.5 * (Pa[3] + pd - rd * c0 * (nx * (Pa[1] - ud) + ny * (Pa[2] - vd)));
        Pb[0] = Pa[0] + (pb - Pa[3]) / (c0 * c0);
        Pb[1] = Pa[1] - nx * (Pa[3] - pb) / (rd * c0);
        Pb[2] = Pa[2] - ny * (Pa[3] - pb) / (rd * c0);
        Pb[3] = pb;
    } else memcpy(Pb, Pa, 4 * sizeof(double));
}

static void bc_outlet(const orc* o, const double* Pd, double* Pb, double nx, double ny)
{   /* boundary.c:53-83 */
    double rd = Pd[0], ud = Pd[1], vd = Pd[2], pd = Pd[3];
    double c0 = T2c(o, pd / rd / o->Rg);
    if (sqrt(ud * ud + vd * vd) / c0 < 1.) {
        double pb = o->c.p_out;
        Pb[0] = rd + (pb - pd) / (c0 * c0);
        Pb[1] = ud + nx * (pd - pb) / (rd * c0);
        Pb[2] = vd + ny * (pd - pb) / (rd * c0);
        Pb[3] = pb;
    } else memcpy(Pb, Pd, 4 * sizeof(double));
}

static void bc_wall(const orc* o, const double* Pd, double* Pb, double nx, double ny)
{   /* boundary.c:121-141 */
    double rd = Pd[0], ud = Pd[1], vd = Pd[2], pd = Pd[3];
    double c0 = T2c(o, pd / rd / o->Rg);
    double pb = pd + rd * c0 * (nx * ud + ny * vd);
    Pb[0] = rd + (pb - pd) / (c0 * c0);
    Pb[1] = ud - nx * (nx * ud + ny * vd);
    Pb[2] = vd - ny * (nx * ud + ny * vd);
    Pb[3] = pb;
}

/* boundaryCalcPrimitive (boundary.c:514-693), inviscid/laminar part */
static void ghosts(orc* o)
{
    int NP = o->nv + 1;
    for (int b = 0; b < o->nb; b++) {
        const double* E = o->P + (size_t)o->bface[3 * b + 2] * NP;
        double* Gb = o->G + (size_t)b * NP;
        double sx, sy, PL[4] = {E[0], E[1], E[2], E[3]}, Pb[4];
        calc_ds(o, o->bface[3 * b], o->bface[3 * b + 1], &sx, &sy);
        double s = sqrt(sx * sx + sy * sy);
        int fl = o->bflag[b];
        if (fl == 0) {
            if (s > 0) { rot(PL, sx, sy, s); PL[1] = 0.0; rot(PL, sx, -sy, s); }
            else PL[2] = 0.0;
            memcpy(Gb, PL, 4 * sizeof(double));
        } else if (fl == 1) {
            bc_inlet(o, o->c.pin, PL, Pb, sx / s, sy / s);
            memcpy(Gb, Pb, 4 * sizeof(double));
        } else if (fl == 2) {
            bc_outlet(o, PL, Pb, sx / s, sy / s);
            memcpy(Gb, Pb, 4 * sizeof(double));
        } else if (o->c.laminar == 1) {
            if (fl == 4) {
                Gb[0] = PL[3] / (o->Rg * o->c.t_wall); Gb[1] = 0.0; Gb[2] = 0.0; Gb[3] = PL[3]; Gb[4] = o->c.t_wall;
                continue;
            }
            Gb[0] = PL[0]; Gb[1] = 0.0; Gb[2] = 0.0; Gb[3] = PL[3];
        } else if (s > 0) {
            bc_wall(o, PL, Pb, sx / s, sy / s);
            memcpy(Gb, Pb, 4 * sizeof(double));
        } else {
            PL[2] = 0.0;
            memcpy(Gb, PL, 4 * sizeof(double));
        }
        Gb[4] = Gb[3] / (Gb[0] * o->Rg);
    }
}

/* ------------------------------------------------------------------ residual */
static void primitives(orc* o, double* U)                                   /* solver.c:1153-1220 */
{
    int nc = o->nc, NP = o->nv + 1;
    for (int i = 0; i < nc; i++) {
        double* P = o->P + (size_t)i * NP;
        P[0] = fmax(U[i], o->c.r_lim);
        U[i] = P[0];
        double u = U[nc + i] / P[0], v = U[2 * nc + i] / P[0];
        P[1] = u;
        P[2] = v;
        double e = fmax(U[3 * nc + i] / P[0] - 0.5 * (u * u + v * v) - 0, 7.176325e+02);
        double T = e2T(o, e);
        if (T < 1) {
            T = 1;
            e = T2e(o, T);
            U[3 * nc + i] = (e + 0.5 * (u * u + v * v) + 0) * P[0];
        }
        P[4] = T;
        P[3] = o->Rg * P[4] * P[0];
    }
    ghosts(o);
}

static const double* nei_P(const orc* o, int i, int j)
{
    int n = o->nei[4 * i + j];
    return n >= 0 ? o->P + (size_t)n * (o->nv + 1) : o->G + (size_t)(-n - 1) * (o->nv + 1);
}

static void nei_center(const orc* o, int i, int j, double* x, double* y)
{
    int n = o->nei[4 * i + j];
    if (n >= 0) center(o, n, x, y);
    else {
        int b = -n - 1, p0 = o->bface[3 * b], p1 = o->bface[3 * b + 1];
        *x = (o->xy[2 * p0] + o->xy[2 * p1]) / 2;
        *y = (o->xy[2 * p0 + 1] + o->xy[2 * p1 + 1]) / 2;
    }
}

static void gradients(orc* o)                                               /* solver.c:451-474, 1031-1074 */
{
    int nc = o->nc, NP = o->nv + 1;
    for (int i = 0; i < nc; i++) {
        double x0, y0, xs[4], ys[4];
        center(o, i, &x0, &y0);
        for (int j = 0; j < o->npts[i]; j++) nei_center(o, i, j, &xs[j], &ys[j]);
        for (int kk = 0; kk < o->nv; kk++) {
            int m = kk > 3 ? kk + 1 : kk;
            long double a = 0, b = 0, c = 0, A = 0, B = 0;
            double u0 = o->P[(size_t)i * NP + m];
            for (int j = 0; j < o->npts[i]; j++) {
                double dx = xs[j] - x0, dy = ys[j] - y0, du = nei_P(o, i, j)[m] - u0;
                a += dx * dx; b += dx * dy; c += dy * dy; A += dx * du; B += dy * du;
            }
            o->dPx[(size_t)kk * nc + i] = (c * A - b * B) / (a * c - b * b);
            o->dPy[(size_t)kk * nc + i] = (-b * A + a * B) / (a * c - b * b);
        }
    }
}

static double lim_v2(double Ui, double mn, double mx, double d2, double ee) /* limiter.c:121-147 */
{
    if (d2 == 0) return 1;
    double d1 = d2 > 0 ? mx - Ui : mn - Ui;
    double a = (d1 * d1 + ee) * d2 + 2 * d2 * d2 * d1;
    a /= d1 * d1 + 2 * d2 * d2 + d1 * d2 + ee;
    return a / d2;
}

static void inter(orc* o)                                                   /* solver.c:493-668 */
{
    int nc = o->nc, nv = o->nv, NP = nv + 1;
    if (o->c.order == 2) {
        double ee1[6] = {0, 0, 0, 0, 0, 0};
        if (o->c.limiter_type == 1) {                                        /* limiter.c:61-94 */
            double mn[6], mx[6];
            for (int kk = 0; kk < nv; kk++) mn[kk] = mx[kk] = o->P[kk == 4 ? 5 : kk];
            for (int i = 1; i < nc; i++)
                for (int kk = 0; kk < nv; kk++) {
                    mn[kk] = fmin(mn[kk], o->P[(size_t)i * NP + (kk == 4 ? 5 : kk)]);
                    mx[kk] = fmax(mx[kk], o->P[(size_t)i * NP + (kk == 4 ? 5 : kk)]);
                }
            for (int kk = 0; kk < nv; kk++) {
                double a = (mx[kk] - mn[kk]) * o->c.limiter_k;
                ee1[kk] = a * a;
            }
        }
        for (int i = 0; i < nc; i++) {
            double x0, y0, aux = o->c.limiter_k * sqrt(o->omega[i] / o->volMax);
            aux = aux * aux * aux;
            center(o, i, &x0, &y0);
            for (int kk = 0; kk < nv; kk++) {
                int m = kk > 3 ? kk + 1 : kk;
                double Pi = o->P[(size_t)i * NP + m], mn = Pi, mx = Pi, phi = 1;
                for (int j = 0; j < o->npts[i]; j++) {
                    double q = nei_P(o, i, j)[m];
                    mx = fmax(mx, q);
                    mn = fmin(mn, q);
                }
                for (int j = 0; j < o->npts[i]; j++) {
                    int p0 = o->nodes[4 * i + j], p1 = o->nodes[4 * i + (j + 1) % o->npts[i]];
                    double xm = (o->xy[2 * p0] + o->xy[2 * p1]) * 0.5, ym = (o->xy[2 * p0 + 1] + o->xy[2 * p1 + 1]) * 0.5;
                    double d2 = (o->dPx[(size_t)kk * nc + i] * (xm - x0) + o->dPy[(size_t)kk * nc + i] * (ym - y0));
                    double p = lim_v2(Pi, mn, mx, d2, o->c.limiter_type == 1 ? ee1[kk] : o->Pref20[kk] * aux);
                    phi = j == 0 ? p : fmin(phi, p);
                }
                o->phi[(size_t)kk * nc + i] = phi;
            }
        }
    }
    for (int f = 0; f < o->nf; f++) {
        int e0 = o->con[4 * f], e1 = o->con[4 * f + 1], p0 = o->con[4 * f + 2], p1 = o->con[4 * f + 3];
        double sx, sy, PL[6] = {0}, PR[6] = {0}, fl[6];
        calc_ds(o, p0, p1, &sx, &sy);
        double s = sqrt(sx * sx + sy * sy);
        const double* A = o->P + (size_t)e0 * NP;
        const double* B = o->P + (size_t)e1 * NP;
        if (o->c.order == 2) {
            double xm = (o->xy[2 * p0] + o->xy[2 * p1]) * 0.5, ym = (o->xy[2 * p0 + 1] + o->xy[2 * p1 + 1]) * 0.5;
            double x0, y0, x1, y1;
            center(o, e0, &x0, &y0);
            center(o, e1, &x1, &y1);
            for (int kk = 0; kk < nv; kk++) {
                int m = kk > 3 ? kk + 1 : kk;
                PL[kk] = A[m] + (o->dPx[(size_t)kk * nc + e0] * (xm - x0) + o->dPy[(size_t)kk * nc + e0] * (ym - y0)) *
                                    o->phi[(size_t)kk * nc + e0];
                PR[kk] = B[m] + (o->dPx[(size_t)kk * nc + e1] * (xm - x1) + o->dPy[(size_t)kk * nc + e1] * (ym - y1)) *
                                    o->phi[(size_t)kk * nc + e1];
            }
        } else {
            for (int kk = 0; kk < nv; kk++) {
                PL[kk] = A[kk > 3 ? kk + 1 : kk];
                PR[kk] = B[kk > 3 ? kk + 1 : kk];
            }
        }
        rot(PL, sx, sy, s);
        rot(PR, sx, sy, s);
        riemann(o, PL, PR, fl);
        rot(fl, sx, -sy, s);
        for (int kk = 0; kk < nv; kk++) o->ff[(size_t)kk * o->nf + f] = fl[kk] * s;
    }
    for (int i = 0; i < nc; i++)
        for (int j = 0; j < o->nint[i]; j++) {
            int face = o->f[4 * i + j];
            for (int kk = 0; kk < nv; kk++) {
                if (face > 0) o->R[(size_t)kk * nc + i] += o->ff[(size_t)kk * o->nf + face - 1];
                else o->R[(size_t)kk * nc + i] -= o->ff[(size_t)kk * o->nf - face - 1];
            }
        }
}

static void boundary(orc* o)                                                /* boundary.c:143-253, 447-464 */
{
    int nc = o->nc, NP = o->nv + 1;
    for (int b = 0; b < o->nb; b++) {
        int e0 = o->bface[3 * b + 2], fl = o->bflag[b];
        double sx, sy, PL[4], Pb[4], Q[4], f[4];
        calc_ds(o, o->bface[3 * b], o->bface[3 * b + 1], &sx, &sy);
        double s = sqrt(sx * sx + sy * sy);
        memcpy(PL, o->P + (size_t)e0 * NP, 4 * sizeof(double));
        if (fl == 0) {
            rot(PL, sx, sy, s);
            Q[0] = PL[0]; Q[1] = -PL[1]; Q[2] = PL[2]; Q[3] = PL[3];
            riemann(o, PL, Q, f);
        } else if (fl == 1 || fl == 2) {
            if (fl == 1) bc_inlet(o, o->c.pin, PL, Pb, sx / s, sy / s);
            else bc_outlet(o, PL, Pb, sx / s, sy / s);
            rot(PL, sx, sy, s);
            rot(Pb, sx, sy, s);
            riemann(o, PL, Pb, f);
        } else if (o->c.laminar == 1) {
            rot(PL, sx, sy, s);
            Q[0] = PL[0]; Q[1] = -PL[1]; Q[2] = -PL[2]; Q[3] = PL[3];
            riemann(o, PL, Q, f);
        } else {
            bc_wall(o, PL, Pb, sx / s, sy / s);
            rot(Pb, sx, sy, s);
            double T = Pb[3] / (o->Rg * Pb[0]);                              /* fluxFree, flux.c:1369-1380 */
            double H = (T2e(o, T) * Pb[0] + (Pb[1] * Pb[1] + Pb[2] * Pb[2]) * Pb[0] / 2 + Pb[3]) / Pb[0];
            f[0] = Pb[0] * Pb[1]; f[1] = Pb[0] * Pb[1] * Pb[1] + Pb[3]; f[2] = Pb[0] * Pb[1] * Pb[2];
            f[3] = Pb[0] * Pb[1] * H;
        }
        rot(f, sx, -sy, s);
        if (s > 0)
            for (int k = 0; k < 4; k++) o->R[(size_t)k * nc + e0] += f[k] * s;
    }
}

void orc_residual(orc* o)                                                   /* solverCalcR, solver.c:685-739 */
{
    memset(o->R, 0, sizeof(double) * o->nv * o->nc);
    primitives(o, o->U);
    gradients(o);
    inter(o);
    boundary(o);
    if (o->c.axisymmetric == 1)                                             /* solver.c:670-683 */
        for (int i = 0; i < o->nc; i++) {
            const int* p = o->nodes + 4 * i;
            double x1 = o->xy[2 * p[0]], x2 = o->xy[2 * p[1]], x3 = o->xy[2 * p[2]];
            double y1 = o->xy[2 * p[0] + 1], y2 = o->xy[2 * p[1] + 1], y3 = o->xy[2 * p[2] + 1];
            double s = 0.5 * ((x1 - x2) * (y1 + y2) + (x2 - x3) * (y2 + y3) + (x3 - x1) * (y3 + y1));
            if (o->npts[i] == 4) {
                double x4 = o->xy[2 * p[3]], y4 = o->xy[2 * p[3] + 1];
                s += 0.5 * ((x3 - x4) * (y3 + y4) + (x4 - x1) * (y4 + y1) + (x1 - x3) * (y1 + y3));
            }
            o->R[2 * o->nc + i] -= o->P[(size_t)i * (o->nv + 1) + 3] * s;
        }
}

/* ------------------------------------------------------------------ time integration */
static double local_step(const orc* o, int i)                              /* solver.c:895-923 */
{
    int nc = o->nc;
    double sxm = 0., sym = 0.;
    for (int j = 0; j < o->npts[i]; j++) {
        double sx, sy;
        calc_ds(o, o->nodes[4 * i + j], o->nodes[4 * i + (j + 1) % o->npts[i]], &sx, &sy);
        sxm += fabs(sx);
        sym += fabs(sy);
    }
    sxm *= 0.5;
    sym *= 0.5;
    double r = o->U[i], u = o->U[nc + i] / r, v = o->U[2 * nc + i] / r, E = o->U[3 * nc + i] / r;
    double c = T2c(o, e2T(o, (E - (u * u + v * v) / 2 - 0)));
    return o->omega[i] / ((fabs(u) + c) * sxm + (fabs(v) + c) * sym);
}

static void calc_dt(orc* o)                                                 /* solver.c:925-950 */
{
    if (o->dtLocal == 1) {
        for (int i = 0; i < o->nc; i++) o->dtL[i] = o->c.cfl * local_step(o, i);
    } else {
        double dt = local_step(o, 0);
        for (int i = 1; i < o->nc; i++) {
            double d = local_step(o, i);
            if (d < dt) dt = d;
        }
        o->dt = dt * o->c.cfl;
    }
}

static void rk_stage(orc* o, double a)                                      /* solver.c:741-766 */
{
    double sigma = 0.5 * o->c.stages;
    for (int i = 0; i < o->nc; i++)
        for (int k = 0; k < o->nv; k++) {
            size_t q = (size_t)k * o->nc + i;
            double dt = o->dtLocal == 1 ? o->dtL[i] : o->dt;
            o->Uaux[q] = o->U[q] - dt * sigma * a * o->R[q] / o->omega[i];
        }
}

static void residual_of(orc* o, double* U)
{
    double* keep = o->U;
    o->U = U;
    orc_residual(o);
    o->U = keep;
}

static void step_rk(orc* o)                                                 /* solver.c:788-840 */
{
    /* two stages {1/2, 1} (midpoint rule) is an extension restated here for the engine's 2-stage RK; the
       reference implements 1, 3, 4 and 5 stages */
    static const double a1[1] = {1.0}, a2[2] = {0.5, 1.0}, a3[3] = {0.1481, 0.4, 1.0},
                        a4[4] = {0.0833, 0.2069, 0.4265, 1.0}, a5[5] = {0.0533, 0.1263, 0.2375, 0.4414, 1.0};
    const double* a = o->c.stages == 1 ? a1 : o->c.stages == 2 ? a2 : o->c.stages == 3 ? a3
                      : o->c.stages == 4 ? a4 : a5;
    for (int s = 0; s < o->c.stages; s++) {
        residual_of(o, s == 0 ? o->U : o->Uaux);
        rk_stage(o, a[s]);
    }
    double* t = o->U;
    o->U = o->Uaux;
    o->Uaux = t;
}

static void implicit_D(orc* o)                                              /* implicit.c:19-181 */
{
    int nc = o->nc, NP = o->nv + 1;
    for (int i = 0; i < nc; i++) {
        double Lc = 0;
        for (int j = 0; j < o->nint[i]; j++) {
            int fa = abs(o->f[4 * i + j]) - 1;
            const double* A = o->P + (size_t)o->con[4 * fa] * NP;
            const double* B = o->P + (size_t)o->con[4 * fa + 1] * NP;
            double sx, sy;
            calc_ds(o, o->con[4 * fa + 2], o->con[4 * fa + 3], &sx, &sy);
            double s = sqrt(sx * sx + sy * sy);
            double u = (A[1] + B[1]) * 0.5, v = (A[2] + B[2]) * 0.5, T = (A[4] + B[4]) * 0.5;
            Lc += (fabs(sx / s * u + sy / s * v) + T2c(o, T)) * s;
        }
        o->dtL[i] = Lc;
        o->D[i] = 0.5 * o->c.w_imp * Lc;
    }
    for (int b = 0; b < o->nb; b++) {
        int e = o->bface[3 * b + 2];
        const double* E = o->P + (size_t)e * NP;
        double sx, sy, nx, ny;
        calc_ds(o, o->bface[3 * b], o->bface[3 * b + 1], &sx, &sy);
        double s = sqrt(sx * sx + sy * sy);
        if (s > 0) { nx = sx / s; ny = sy / s; }
        else { nx = 0.0; ny = 1.0; }
        double Lc = (fabs(nx * E[1] + ny * E[2]) + T2c(o, E[4])) * s;
        o->dtL[e] += Lc;
        o->D[e] += 0.5 * o->c.w_imp * Lc;
    }
    for (int i = 0; i < nc; i++) o->dtL[i] = o->omega[i] / o->dtL[i];
    double dt = o->dtL[0];
    for (int i = 1; i < nc; i++) dt = fmin(dt, o->dtL[i]);
    dt *= o->c.cfl;
    for (int i = 0; i < nc; i++) o->D[i] += o->omega[i] / dt;
}

static void aux_flux(const double* U, double p, double nx, double ny, double* F) /* implicit.c:183-191 */
{
    double V = (nx * U[1] + ny * U[2]) / U[0];
    F[0] = U[0] * V; F[1] = U[1] * V + nx * p; F[2] = U[2] * V + ny * p; F[3] = (U[3] + p) * V;
}

static void implicit_A(orc* o)                                              /* implicit.c:689-813 */
{
    int nc = o->nc, NP = o->nv + 1;
    const double h = 1.0e-6;
    for (int i = 0; i < nc; i++)
        for (int j = 0; j < o->nint[i]; j++) {
            int face = o->f[4 * i + j], fa = abs(face) - 1, e1, p0, p1;
            if (face > 0) { e1 = o->con[4 * fa + 1]; p0 = o->con[4 * fa + 2]; p1 = o->con[4 * fa + 3]; }
            else { e1 = o->con[4 * fa]; p1 = o->con[4 * fa + 2]; p0 = o->con[4 * fa + 3]; }
            double sx, sy;
            calc_ds(o, p0, p1, &sx, &sy);
            double s = sqrt(sx * sx + sy * sy), nx = sx / s, ny = sy / s;
            const double* E1 = o->P + (size_t)e1 * NP;
            double Un[4] = {o->U[e1], o->U[nc + e1], o->U[2 * nc + e1], o->U[3 * nc + e1]}, F0[4], F[4], Uq[4];
            double u = Un[1] / Un[0], v = Un[2] / Un[0], E = Un[3] / Un[0];
            aux_flux(Un, E1[3], nx, ny, F0);
            double ee0 = E - 0.5 * (u * u + v * v);
            double* A = o->A + ((size_t)i * 4 + j) * 16;
            for (int m = 0; m < 4; m++) {
                for (int n = 0; n < 4; n++) Uq[n] = m == n ? Un[n] + h : Un[n];
                double r = Uq[0], u2 = Uq[1] / r, v2 = Uq[2] / r, E2 = Uq[3] / r;
                double T = e2Taprox(o, ee0, E1[4], E2 - 0.5 * (u2 * u2 + v2 * v2));
                aux_flux(Uq, o->Rg * r * T, nx, ny, F);
                for (int n = 0; n < 4; n++) A[n * 4 + m] = 0.5 * (F[n] - F0[n]) * s / h;
            }
            double ra = o->c.w_imp * (fabs(nx * E1[1] + ny * E1[2]) + T2c(o, E1[4])) * s;
            for (int n = 0; n < 4; n++) A[n * 4 + n] -= 0.5 * ra;
        }
}

static void dplur(orc* o)                                                   /* implicit.c:990-1034 */
{
    int nc = o->nc, nv = o->nv;
    implicit_D(o);
    implicit_A(o);
    double w = 2. / 3.;
    for (int m = 0; m < o->c.n_linear; m++) {
        double* t = o->dW1;
        o->dW1 = o->dW0;
        o->dW0 = t;
        for (int i = 0; i < nc; i++) {                                       /* implicitMultA 938-972 */
            double y[6];
            for (int k = 0; k < nv; k++) y[k] = o->D[i] * o->dW0[(size_t)k * nc + i];
            for (int j = 0; j < o->nint[i]; j++) {
                int face = o->f[4 * i + j], fa = abs(face) - 1;
                int nb = face > 0 ? o->con[4 * fa + 1] : o->con[4 * fa];
                const double* A = o->A + ((size_t)i * 4 + j) * 16;
                for (int k = 0; k < nv; k++)
                    for (int n = 0; n < nv; n++) y[k] += A[k * 4 + n] * o->dW0[(size_t)n * nc + nb];
            }
            for (int k = 0; k < nv; k++)
                o->dW1[(size_t)k * nc + i] = w * (-o->R[(size_t)k * nc + i] - y[k]) / o->D[i] + o->dW0[(size_t)k * nc + i];
        }
        double ans = fabs(o->dW1[0] - o->dW0[0]);
        for (int i = 1; i < nc; i++) ans = fmax(ans, fabs(o->dW1[i] - o->dW0[i]));
        if (ans < 1e-14) break;
    }
}

static void coeff(const orc* o, double* out)                                /* solver.c:1342-1401 */
{
    double r = o->c.pin[0], u = o->c.pin[1], v = o->c.pin[2], P = o->c.pin[3], q = 0.5 * r * (u * u + v * v);
    double cx = 0, cy = 0;
    for (int b = 0; b < o->nb; b++)
        if (o->bflag[b] == 3 || o->bflag[b] == 4) {
            double sx, sy, cp = (o->G[(size_t)b * (o->nv + 1) + 3] - P) / q;
            calc_ds(o, o->bface[3 * b], o->bface[3 * b + 1], &sx, &sy);
            cx += cp * sx;
            cy += cp * sy;
        }
    cx /= o->c.sref;
    cy /= o->c.sref;
    if (o->c.axisymmetric) cx *= 2 * M_PI;
    out[0] = cx; out[1] = 0.0; out[2] = cy; out[3] = 0.0;
}

void orc_iterate(orc* o, int n, int it0, double* hist)                     /* solver.c:1864-1906 */
{
    int nc = o->nc, nv = o->nv;
    for (int it = 0; it < n; it++) {
        if (o->c.time_scheme == CSU_TS_RK) {
            calc_dt(o);
            step_rk(o);
        } else {
            orc_residual(o);
            dplur(o);
            for (size_t q = 0; q < (size_t)nv * nc; q++) o->U[q] += o->dW1[q];
        }
        if (it0 + it == o->c.dt_local_n) o->dtLocal = 0;
        for (int k = 0; k < nv; k++) {                                       /* solverCalcRes 867-892 */
            double s = 0.0;
            for (int i = 0; i < nc; i++) s += o->R[(size_t)k * nc + i] * o->R[(size_t)k * nc + i];
            o->res[k] = sqrt(s / nc);
        }
        if (hist) {
            double* row = hist + (size_t)it * (nv + 4);
            memcpy(row, o->res, sizeof(double) * nv);
            coeff(o, row + nv);
        }
    }
}

int orc_tube(orc* o, double tmax, double* t_out)                           /* solver.c:1912-1942 */
{
    double t = 0.0;
    int stop = 0, ii = 0;
    while (!stop) {
        calc_dt(o);
        if (t + o->dt > tmax) {
            o->dt = tmax - t;
            stop = 1;
        }
        step_rk(o);
        t += o->dt * o->c.stages / 2.0;
        ii++;
    }
    *t_out = t;
    return ii;
}

/* ------------------------------------------------------------------ setup and views */
orc* orc_create(const csu_mesh_desc* m, const csu_config* c)
{
    orc* o = calloc(1, sizeof(orc));
    o->c = *c;
    o->nc = m->n_cells; o->nf = m->n_faces; o->nb = m->n_bfaces; o->nv = c->nvar; o->nm = m->n_markers;
    int nc = o->nc, nv = o->nv;
#define DUP(dst, src, n) do { dst = malloc(sizeof(*(dst)) * ((n) > 0 ? (n) : 1)); memcpy(dst, src, sizeof(*(dst)) * (n)); } while (0)
    DUP(o->xy, m->xy, 2 * m->n_points);
    DUP(o->npts, m->cell_npts, nc);
    DUP(o->nodes, m->cell_nodes, 4 * nc);
    DUP(o->con, m->con, 4 * o->nf);
    DUP(o->nint, m->cell_nint, nc);
    DUP(o->f, m->cell_faces, 4 * nc);
    DUP(o->nei, m->cell_nei, 4 * nc);
    DUP(o->bface, m->bface, 3 * o->nb);
#undef DUP
    o->bflag = malloc(sizeof(int) * (o->nb > 0 ? o->nb : 1));
    for (int k = 0, b = 0; k < o->nm; k++)
        for (int j = 0; j < m->marker_nbf[k]; j++) o->bflag[b++] = m->marker_flag[k];
    o->gam = c->gamma;
    o->Rg = c->gas_r;
    o->Cp = o->gam * o->Rg / (o->gam - 1);
    o->Cv = o->Cp - o->Rg;
    o->omega = malloc(sizeof(double) * nc);
    o->volMax = 0.0;
    for (int i = 0; i < nc; i++) {                                           /* mesh.c:420-449 */
        const int* p = o->nodes + 4 * i;
        double x1 = o->xy[2 * p[0]], x2 = o->xy[2 * p[1]], x3 = o->xy[2 * p[2]];
        double y1 = o->xy[2 * p[0] + 1], y2 = o->xy[2 * p[1] + 1], y3 = o->xy[2 * p[2] + 1];
        double a = 0.5 * ((x1 - x2) * (y1 + y2) + (x2 - x3) * (y2 + y3) + (x3 - x1) * (y3 + y1));
        if (o->npts[i] == 4) {
            double x4 = o->xy[2 * p[3]], y4 = o->xy[2 * p[3] + 1];
            a += 0.5 * ((x3 - x4) * (y3 + y4) + (x4 - x1) * (y4 + y1) + (x1 - x3) * (y1 + y3));
        }
        if (c->axisymmetric == 1) {
            double xc, yc;
            center(o, i, &xc, &yc);
            a *= yc;
        }
        o->omega[i] = a;
        o->volMax = fmax(a, o->volMax);
    }
    o->Pref20[0] = c->pin[0] * c->pin[0];                                    /* limiter.c:49-59 */
    o->Pref20[1] = c->pin[1] * c->pin[1] + c->pin[2] * c->pin[2];
    o->Pref20[2] = o->Pref20[1];
    o->Pref20[3] = c->pin[3] * c->pin[3];
    size_t s = (size_t)nv * nc;
    o->U = calloc(s, 8); o->Uaux = calloc(s, 8); o->R = calloc(s, 8); o->dPx = calloc(s, 8);
    o->dPy = calloc(s, 8); o->phi = calloc(s, 8); o->dW0 = calloc(s, 8); o->dW1 = calloc(s, 8);
    o->P = calloc((size_t)nc * (nv + 1), 8);
    o->G = calloc((size_t)(o->nb > 0 ? o->nb : 1) * (nv + 1), 8);
    o->ff = calloc((size_t)nv * (o->nf > 0 ? o->nf : 1), 8);
    o->dtL = calloc(nc, 8); o->D = calloc(nc, 8);
    o->A = calloc((size_t)nc * 4 * 16, 8);
    o->dtLocal = c->dt_local;
    return o;
}

void orc_free(orc* o)
{
    if (!o) return;
    void* p[] = {o->xy, o->npts, o->nodes, o->con, o->nint, o->f, o->nei, o->bface, o->bflag, o->omega, o->U,
                 o->Uaux, o->R, o->P, o->G, o->dPx, o->dPy, o->phi, o->ff, o->dtL, o->D, o->dW0, o->dW1, o->A};
    for (size_t i = 0; i < sizeof(p) / sizeof(p[0]); i++) free(p[i]);
    free(o);
}

void orc_set_U(orc* o, const double* U) { memcpy(o->U, U, sizeof(double) * o->nv * o->nc); }
void orc_get_U(orc* o, double* U) { memcpy(U, o->U, sizeof(double) * o->nv * o->nc); }

void orc_get(orc* o, int what, double* out)
{
    size_t s = (size_t)o->nv * o->nc;
    switch (what) {
    case 1: memcpy(out, o->P, sizeof(double) * o->nc * (o->nv + 1)); break;
    case 2: memcpy(out, o->G, sizeof(double) * o->nb * (o->nv + 1)); break;
    case 3: memcpy(out, o->dPx, 8 * s); memcpy(out + s, o->dPy, 8 * s); break;
    case 4: memcpy(out, o->phi, 8 * s); break;
    case 5: memcpy(out, o->ff, sizeof(double) * o->nv * o->nf); break;
    case 6: memcpy(out, o->R, 8 * s); break;
    case 7: memcpy(out, o->D, 8 * o->nc); break;
    case 8: memcpy(out, o->dtL, 8 * o->nc); break;
    case 9: memcpy(out, o->dW1, 8 * s); break;
    case 10: memcpy(out, o->A, sizeof(double) * o->nc * 4 * 16); break;
    }
}
