/*
 * ref_harness.c -- test infrastructure only.
 *
 * A thin C layer linked against the reference CSU solver compiled from its own, unmodified sources
 * (see oracle/Makefile). It calls the reference's functions and copies the reference's internal
 * arrays out at full precision, so that tests can pin both the plain-C restatement (csu_oracle.c)
 * and the CUDA path against the reference itself. Nothing in the product links or loads this.
 *
 * Array layouts returned here follow the reference:
 *   U, R, dPx, dPy, phi, dW      [kk][ii]  (Nvar rows of Nelem)           solver.h:152-163
 *   faceFlux                     [kk][face] (Nvar rows of Ncon)
 *   P (cell primitives)          [ii][kk]  (Nelem rows of Nvar+1)          mesh.h:9 (ELEMENT.P)
 *   ghost P                      [gid][kk] (boundary elements, marker-major order)
 * Neighbour ids: >= 0 is a cell index, < 0 is -(1 + global boundary element id).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <unistd.h>
#include <fcntl.h>
#include "utils.h"
#include "input.h"
#include "mesh.h"
#include "solver.h"
#include "flux.h"
#include "boundary.h"
#include "implicit.h"
#include "limiter.h"
#include "gasprop.h"

static SOLVER* g = NULL;
static char* g_wd = NULL;
static int g_quiet = 1;
static int g_saved_fd = -1;

static void quiet_on(void)
{
    if (!g_quiet) return;
    fflush(stdout);
    g_saved_fd = dup(1);
    int fd = open("/dev/null", O_WRONLY);
    dup2(fd, 1);
    close(fd);
}

static void quiet_off(void)
{
    if (!g_quiet || g_saved_fd < 0) return;
    fflush(stdout);
    dup2(g_saved_fd, 1);
    close(g_saved_fd);
    g_saved_fd = -1;
}

static int total_bc(void)
{
    int n = 0;
    for (int m = 0; m < g->mesh->Nmark; m++) n += g->mesh->bc[m]->Nelem;
    return n;
}

/* global id of a boundary element pointer, or -1 */
static int bc_gid(const ELEMENT* e)
{
    int base = 0;
    for (int m = 0; m < g->mesh->Nmark; m++) {
        MESHBC* bc = g->mesh->bc[m];
        if (e->ii >= 0 && e->ii < bc->Nelem && bc->elemL[e->ii] == e) return base + e->ii;
        base += bc->Nelem;
    }
    return -1;
}

/* solverInit (solver.c:1728). wd must end with '/' and be short (the reference uses char[50]). */
int ref_open(const char* wd, int quiet)
{
    g_quiet = quiet;
    free(g_wd);
    g_wd = strdup(wd);
    quiet_on();
    g = solverInit(g_wd);
    quiet_off();
    return g ? 0 : 1;
}

void ref_sizes(int* out)
{
    out[0] = g->mesh->Nelem;
    out[1] = g->mesh->Np;
    out[2] = g->mesh->Ncon;
    out[3] = g->mesh->Nmark;
    out[4] = g->Nvar;
    out[5] = total_bc();
    out[6] = g->timeScheme;
    out[7] = g->stages;
    out[8] = g->order;
    out[9] = g->flux;
    out[10] = g->laminar;
    out[11] = g->sa;
    out[12] = g->sstFlag;
    out[13] = g->mesh->axi;
    out[14] = g->dtLocal;
    out[15] = g->Nlinear;
}

void ref_points(double* xy)
{
    for (int i = 0; i < g->mesh->Np; i++) {
        xy[2 * i] = g->mesh->p[i][0];
        xy[2 * i + 1] = g->mesh->p[i][1];
    }
}

void ref_cells(int* nodes, int* npts, int* f, int* neiN, int* nei, double* omega)
{
    for (int i = 0; i < g->mesh->Nelem; i++) {
        ELEMENT* E = g->mesh->elemL[i];
        npts[i] = E->Np;
        neiN[i] = E->neiN;
        omega[i] = E->omega;
        for (int j = 0; j < 4; j++) {
            nodes[4 * i + j] = j < E->Np ? E->p[j] : -1;
            f[4 * i + j] = j < E->neiN ? E->f[j] : 0;
            nei[4 * i + j] = 0x7fffffff;
        }
        for (int j = 0; j < E->Np; j++) {
            ELEMENT* n = E->neiL[j];
            if (n->Np == 2) nei[4 * i + j] = -(1 + bc_gid(n));
            else nei[4 * i + j] = n->ii;
        }
    }
}

void ref_wall_distance(double* d)
{
    for (int i = 0; i < g->mesh->Nelem; i++) d[i] = g->mesh->elemL[i]->d;
}

void ref_con(int* con)
{
    for (int i = 0; i < g->mesh->Ncon; i++)
        for (int k = 0; k < 4; k++) con[4 * i + k] = g->mesh->con[i][k];
}

void ref_bc(int* marker_nelem, int* flags, int* bcdata)
{
    int gid = 0;
    for (int m = 0; m < g->mesh->Nmark; m++) {
        MESHBC* bc = g->mesh->bc[m];
        marker_nelem[m] = bc->Nelem;
        flags[m] = bc->flagBC;
        for (int j = 0; j < bc->Nelem; j++, gid++) {
            bcdata[3 * gid] = bc->elemL[j]->p[0];
            bcdata[3 * gid + 1] = bc->elemL[j]->p[1];
            bcdata[3 * gid + 2] = bc->elemL[j]->neiL[0]->ii;
        }
    }
}

void ref_bc_name(int m, char* out, int cap)
{
    snprintf(out, cap, "%s", g->mesh->bc[m]->name);
}

void ref_inlet(double* Pin, double* Uin, double* mach)
{
    for (int k = 0; k < 7; k++) Pin[k] = g->inlet->Pin[k];
    for (int k = 0; k < 6; k++) Uin[k] = g->inlet->Uin[k];
    *mach = g->inlet->mach;
}

void ref_get_U(double* U)
{
    for (int k = 0; k < g->Nvar; k++)
        memcpy(U + (size_t)k * g->mesh->Nelem, g->U[k], sizeof(double) * g->mesh->Nelem);
}

void ref_set_U(const double* U)
{
    for (int k = 0; k < g->Nvar; k++)
        memcpy(g->U[k], U + (size_t)k * g->mesh->Nelem, sizeof(double) * g->mesh->Nelem);
}

/* one residual evaluation solverCalcR(solver, solver->U) (solver.c:685) */
void ref_calc_R(void)
{
    solverCalcR(g, g->U);
}

/* the SST source Jacobians of the last solverCalcR (sstInterSource): dQkdr, dQkdrk, dQkdro, dQodr, dQodrk,
   dQodro, [6][cell] */
void ref_sst_jac(double* J)
{
    const int n = g->mesh->Nelem;
    const double* a[6] = {g->dQkdr, g->dQkdrk, g->dQkdro, g->dQodr, g->dQodrk, g->dQodro};
    for (int q = 0; q < 6; q++) memcpy(J + (size_t)q * n, a[q], sizeof(double) * n);
}

/* the face eddy viscosity of the last solverCalcR (SA, SST): miT[face], mesh->con order */
void ref_get_miT(double* miT)
{
    memcpy(miT, g->miT, sizeof(double) * g->mesh->Ncon);
}

void ref_get_R(double* R)
{
    for (int k = 0; k < g->Nvar; k++)
        memcpy(R + (size_t)k * g->mesh->Nelem, g->R[k], sizeof(double) * g->mesh->Nelem);
}

void ref_get_P(double* P)
{
    int n = g->Nvar + 1;
    for (int i = 0; i < g->mesh->Nelem; i++)
        for (int k = 0; k < n; k++) P[(size_t)i * n + k] = g->mesh->elemL[i]->P[k];
}

void ref_get_ghostP(double* P)
{
    int n = g->Nvar + 1, gid = 0;
    for (int m = 0; m < g->mesh->Nmark; m++) {
        MESHBC* bc = g->mesh->bc[m];
        for (int j = 0; j < bc->Nelem; j++, gid++)
            for (int k = 0; k < n; k++) P[(size_t)gid * n + k] = bc->elemL[j]->P[k];
    }
}

void ref_get_grad(double* dPx, double* dPy)
{
    for (int k = 0; k < g->Nvar; k++) {
        memcpy(dPx + (size_t)k * g->mesh->Nelem, g->dPx[k], sizeof(double) * g->mesh->Nelem);
        memcpy(dPy + (size_t)k * g->mesh->Nelem, g->dPy[k], sizeof(double) * g->mesh->Nelem);
    }
}

void ref_get_phi(double* phi)
{
    for (int k = 0; k < g->Nvar; k++)
        memcpy(phi + (size_t)k * g->mesh->Nelem, g->phi[k], sizeof(double) * g->mesh->Nelem);
}

void ref_get_faceflux(double* ff)
{
    for (int k = 0; k < g->Nvar; k++)
        memcpy(ff + (size_t)k * g->mesh->Ncon, g->faceFlux[k], sizeof(double) * g->mesh->Ncon);
}

/* solverCalcDt (solver.c:925); returns the global dt, dtL is filled when dtLocal == 1 */
double ref_calc_dt(double* dtL)
{
    solverCalcDt(g);
    if (g->dtLocal == 1 && dtL) memcpy(dtL, g->dtL, sizeof(double) * g->mesh->Nelem);
    return g->dt;
}

/* implicitCalcD (implicit.c:19); after solverCalcR. */
void ref_implicit_D(double* D, double* dtL)
{
    implicitCalcD(g);
    memcpy(D, g->D, sizeof(double) * g->mesh->Nelem);
    memcpy(dtL, g->dtL, sizeof(double) * g->mesh->Nelem);
}

/* implicitUpdateA(_sa) (implicit.c:689,815): blocks as [cell][slot 0..3][N][N], slots in E->f order */
void ref_implicit_A(double* A)
{
    if (g->sa) implicitUpdateA_sa(g);
    else implicitUpdateA(g);
    int N = g->Nvar;
    size_t per = (size_t)4 * N * N;
    for (int i = 0; i < g->mesh->Nelem; i++) {
        BLOCK* B = NULL;
        for (int j = 0; j < g->mesh->elemL[i]->neiN; j++) {
            B = (j == 0) ? g->BB[i] : B->next;
            for (int r = 0; r < N; r++)
                for (int c = 0; c < N; c++) A[i * per + (size_t)j * N * N + r * N + c] = B->A[r][c];
        }
    }
}

/* implicitCalcDPLUR (implicit.c:990) and the increment it leaves in dW1 */
void ref_implicit_dplur(double* dW1)
{
    implicitCalcDPLUR(g);
    for (int k = 0; k < g->Nvar; k++)
        memcpy(dW1 + (size_t)k * g->mesh->Nelem, g->dW1[k], sizeof(double) * g->mesh->Nelem);
}

/* The coefficient sums of solverCalcCoeff3 (solver.c:1342-1401) at full precision. */
static void coeff3(double* out4)
{
    double r = g->inlet->Pin[0], u = g->inlet->Pin[1], v = g->inlet->Pin[2], P = g->inlet->Pin[3];
    double q = 0.5 * r * (u * u + v * v);
    double Cx_p = 0, Cx_v = 0, Cy_p = 0, Cy_v = 0;
    for (int jj = 0; jj < g->mesh->Nmark; jj++) {
        MESHBC* bc = g->mesh->bc[jj];
        if (bc->flagBC == 3 || bc->flagBC == 4) {
            for (int ii = 0; ii < bc->Nelem; ii++) {
                double dSx, dSy, fx, fy;
                double cp = (bc->elemL[ii]->P[3] - P) / q;
                meshCalcDS(g->mesh, bc->elemL[ii]->p[0], bc->elemL[ii]->p[1], &dSx, &dSy);
                Cx_p += cp * dSx;
                Cy_p += cp * dSy;
                if (g->laminar == 1 || g->sa == 1 || g->sstFlag == 1) {
                    boundaryCalcFrictionWall(g, bc->elemL[ii], &fx, &fy);
                    Cx_v -= fx / q;
                    Cy_v -= fy / q;
                }
            }
        }
    }
    Cx_p /= g->Sref; Cx_v /= g->Sref; Cy_p /= g->Sref; Cy_v /= g->Sref;
    if (g->mesh->axi) { Cx_p *= 2 * M_PI; Cx_v *= 2 * M_PI; }
    out4[0] = Cx_p; out4[1] = Cx_v; out4[2] = Cy_p; out4[3] = Cy_v;
}

/*
 * n iterations of the steady loop body of solverSolve (solver.c:1864-1906). Per iteration the row
 * hist[it*(Nvar+4) ...] holds res[0..Nvar-1] (solverCalcRes) then Cx_p, Cx_v, Cy_p, Cy_v.
 * it0 is the value of the loop counter for the first iteration (the dtLocalN switch uses it).
 */
void ref_iterate(int n, int it0, double* hist)
{
    int N = g->Nvar;
    quiet_on();
    for (int it = 0; it < n; it++) {
        int ii = it0 + it;
        if (g->timeScheme == 0) {
            solverCalcDt(g);
            solverStepRK(g);
        } else if (g->timeScheme == 1) {
            solverCalcR(g, g->U);
            implicitCalcD(g);
            implicitLUSGS_L(g);
            implicitLUSGS_U(g);
            solverUpdateUImplicit(g);
        } else if (g->timeScheme == 2) {
            solverCalcR(g, g->U);
            implicitCalcDPLUR(g);
            solverUpdateUImplicit(g);
        }
        if (ii == g->dtLocalN) g->dtLocal = 0;
        solverCalcRes(g);
        if (hist) {
            for (int k = 0; k < N; k++) hist[(size_t)it * (N + 4) + k] = g->res[k];
            coeff3(hist + (size_t)it * (N + 4) + N);
        }
    }
    quiet_off();
}

/* The unsteady (tube) loop of solverSolve (solver.c:1912-1942). Returns the number of steps. */
int ref_tube_run(double tmax, double* t_out)
{
    double t = 0.0;
    int stopLoop = 0, ii = 0;
    quiet_on();
    while (stopLoop == 0) {
        solverCalcDt(g);
        if (t + g->dt > tmax) {
            g->dt = (tmax - t);
            stopLoop = 1;
        }
        solverStepRK(g);
        t += g->dt * g->stages / 2.0;
        ii++;
    }
    quiet_off();
    *t_out = t;
    return ii;
}

/* The reference's own solve loop (solver.c:1836), untouched; writes convergence.csv in wd. */
void ref_solve(void)
{
    quiet_on();
    solverSolve(g);
    quiet_off();
}

/* The reference writers (main.c:29-35) */
void ref_write_outputs(void)
{
    quiet_on();
    solverWriteSolution(g);
    solverWriteSolution2(g);
    solverWriteReestart(g);
    solverWriteSurf(g);
    quiet_off();
}

/* the reference is abandoned rather than freed: solverFree frees LIMITER.Pref2, never allocated. */
void ref_close(void)
{
    g = NULL;
}
