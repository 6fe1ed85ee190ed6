/*
 * driver.c -- the reference's program flow (main.c:18-45, solverSolve solver.c:1836-1943) on the device
 * engine: read a case folder, iterate, write the same files.
 *
 *   convergence.csv  one row per iteration: "%i," then " %+.4e," per variable, then " %e, %e, %e, %e,"
 *                    (Cx_p, Cx_v, Cy_p, Cy_v) (solver.c:1899-1905, 1399); appended when restarting
 *   friction.csv     per wall face: x, txx, txy, tyy, y+ (solverCalcCoeff2, solver.c:1303-1340)
 *   solution.csv     node values of U by inverse-distance weighting of the cells (solver.c:222-325)
 *   solution2.csv    node values of primitives, Mach, H, entropy (solver.c:2009-2220)
 *   restart.csv      cell values of U (solver.c:327-355), after the primitive clamps of solution2
 *   surfData.csv     wall data along the `writeSurf` marker (laminar.c:350-492, sa.c:854-996,
 *                    saCC.c:599-745, sst.c:820-962; dispatched as solverWriteSurf, solver.c:1984-2007)
 *
 * The iteration history comes from the device (csu_iterate). Node interpolation and file writing stay on
 * the host: they run once per solve. The wall files follow the reference's order of events. friction.csv is
 * written inside solverSolve from what the last residual evaluation left: primitives and gradients of the
 * state the last iteration started from (implicit schemes) or of its last RK stage's input. The engine
 * therefore runs Nmax - 1 iterations, then the last one through csu_iterate_views, which returns exactly
 * those arrays, and writes friction.csv. surfData.csv comes after solverWriteSolution2, which recomputes
 * the cell and ghost primitives of the final state: csu_wall_data gives the ghost states and boundary
 * viscous fluxes of the final primitives with the last gradients.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <sys/time.h>
#include "case.h"

static double now(void)
{
    struct timeval t;
    gettimeofday(&t, NULL);
    return t.tv_sec + t.tv_usec * 1e-6;
}

static FILE* open_in(const char* wd, const char* name, const char* mode)
{
    char path[4096];
    snprintf(path, sizeof(path), "%s%s", wd, name);
    return fopen(path, mode);
}

/* inverse-distance node interpolation of per-cell rows (solver.c:245-285) */
static void to_nodes(const csu_mesh* m, const double* cellv, int nv, int stride_cell, double* nodev)
{
    double* den = calloc(m->n_points, sizeof(double));
    memset(nodev, 0, sizeof(double) * (size_t)nv * m->n_points);
    for (int i = 0; i < m->n_cells; i++) {
        double xc, yc;
        csu_mesh_center(m, i, &xc, &yc);
        for (int j = 0; j < m->cell_npts[i]; j++) {
            int p = m->cell_nodes[4 * i + j];
            double xp = m->xy[2 * p], yp = m->xy[2 * p + 1];
            double L = sqrt((xp - xc) * (xp - xc) + (yp - yc) * (yp - yc));
            for (int k = 0; k < nv; k++) nodev[(size_t)k * m->n_points + p] += cellv[stride_cell == 0 ? (size_t)k * m->n_cells + i : (size_t)i * stride_cell + k] / L;
            den[p] += 1 / L;
        }
    }
    for (int p = 0; p < m->n_points; p++)
        if (den[p] != 0)
            for (int k = 0; k < nv; k++) nodev[(size_t)k * m->n_points + p] /= den[p];
    free(den);
}

static void zero_wall_velocity(const csu_mesh* m, double* nodev, int np, int both_wall_kinds)
{
    int b = 0;
    for (int k = 0; k < m->n_markers; k++) {
        int fl = m->marker_flag[k];
        int hit = fl == CSU_BC_WALL || (both_wall_kinds && fl == CSU_BC_WALLT);
        for (int j = 0; j < m->marker_nbf[k]; j++, b++) {
            if (!hit) continue;
            for (int q = 0; q < 2; q++) {
                int p = m->bface[3 * b + q];
                nodev[(size_t)1 * np + p] = 0.0;
                nodev[(size_t)2 * np + p] = 0.0;
            }
        }
    }
}

static int write_solution(const char* wd, const csu_case* cs, const double* U)
{
    const csu_mesh* m = &cs->mesh;
    int nv = cs->cfg.nvar, np = m->n_points;
    double* Up = malloc(sizeof(double) * (size_t)nv * np);
    to_nodes(m, U, nv, 0, Up);
    if (cs->cfg.laminar || cs->cfg.sa || cs->cfg.sst) zero_wall_velocity(m, Up, np, 1);
    FILE* f = open_in(wd, "solution.csv", "w");
    if (!f) {
        free(Up);
        csu_set_error("cannot write %ssolution.csv", wd);
        return CSU_ERR_IO;
    }
    fprintf(f, "0, %i, %i,\n", np, nv);
    for (int p = 0; p < np; p++) {
        for (int k = 0; k < nv; k++) fprintf(f, "%.10e, ", Up[(size_t)k * np + p]);
        fprintf(f, "\n");
    }
    fclose(f);
    free(Up);
    return CSU_OK;
}

/* gasprop_T2fentro / gasprop_Tp2entropy (gasprop.c:309-335) for the calorically perfect gas */
static double entropy(const csu_config* c, double T, double p)
{
    double cp = c->gamma * c->gas_r / (c->gamma - 1);
    if (c->tp) {
        static const double cc1 = 9.890504e2 - 287.0530, cc[6] = {1.81716e3, 9.890504e2 - 287.0530, -9.595592e-3,
                                                                    1.041469e-4, -4.433065e-8, 5.879263e-12};
        double P = 1, aux = (cc1 + c->gas_r) * log(T);
        for (int i = 2; i < 6; i++) {
            P *= T;
            aux += i * cc[i] * P / (i - 1);
        }
        return aux - c->gas_r * log(p);
    }
    return cp * log(T) - c->gas_r * log(p);
}

static int write_solution2(const char* wd, const csu_case* cs, const double* P)
{
    const csu_mesh* m = &cs->mesh;
    const csu_config* c = &cs->cfg;
    int nv = c->nvar, np = m->n_points, npr = nv + 1;
    double* Pp = malloc(sizeof(double) * (size_t)npr * np);
    to_nodes(m, P, npr, npr, Pp);
    if (c->laminar || c->sa || c->sst) {
        int b = 0;
        for (int k = 0; k < m->n_markers; k++)
            for (int j = 0; j < m->marker_nbf[k]; j++, b++) {
                if (m->marker_flag[k] != CSU_BC_WALL) continue;
                for (int q = 0; q < 2; q++) {
                    int p = m->bface[3 * b + q];
                    Pp[(size_t)1 * np + p] = 0.0;
                    Pp[(size_t)2 * np + p] = 0.0;
                    if (c->sa || c->sst) {
                        Pp[(size_t)5 * np + p] = 0.0;
                        if (c->t_wall >= 0) Pp[(size_t)4 * np + p] = c->t_wall;
                    }
                }
            }
    }
    FILE* f = open_in(wd, "solution2.csv", "w");
    if (!f) {
        free(Pp);
        csu_set_error("cannot write %ssolution2.csv", wd);
        return CSU_ERR_IO;
    }
    if (c->sst) fprintf(f, "r,u,v,p,T,k,o,mach,H,s,\n");
    else if (c->sa) fprintf(f, "r,u,v,p,T,n,mach,H,s,\n");
    else fprintf(f, "r,u,v,p,T,mach,H,s,\n");
    double s0 = entropy(c, c->inlet_t, c->inlet_p);
    for (int p = 0; p < np; p++) {
        double u = Pp[(size_t)1 * np + p], v = Pp[(size_t)2 * np + p], T = Pp[(size_t)4 * np + p];
        double r = Pp[p], pr = Pp[(size_t)3 * np + p];
        double V2 = u * u + v * v;
        for (int k = 0; k < npr; k++) fprintf(f, "%.10e, ", Pp[(size_t)k * np + p]);
        fprintf(f, "%.10e, ", sqrt(V2) / csu_host_T2c(c, T));
        fprintf(f, "%.10e, ", csu_host_T2e(c, T) + pr / r + 0.5 * V2);
        fprintf(f, "%.10e, ", entropy(c, T, pr) - s0);
        fprintf(f, "\n");
    }
    fclose(f);
    free(Pp);
    return CSU_OK;
}

static int write_restart(const char* wd, const csu_case* cs, const double* U)
{
    FILE* f = open_in(wd, "restart.csv", "w");
    if (!f) {
        csu_set_error("cannot write %srestart.csv", wd);
        return CSU_ERR_IO;
    }
    int nc = cs->mesh.n_cells, nv = cs->cfg.nvar;
    fprintf(f, "1,\n");
    fprintf(f, "0, %i, %i,\n", nc, nv);
    for (int i = 0; i < nc; i++) {
        for (int k = 0; k < nv; k++) fprintf(f, "%.10e, ", U[(size_t)k * nc + i]);
        fprintf(f, "\n");
    }
    fclose(f);
    return CSU_OK;
}

/* meshCalcDS (mesh.c:720-740): face normal of the edge p0 -> p1, times the mean y when axisymmetric */
static void face_ds(const csu_mesh* m, int axi, int p0, int p1, double* dSx, double* dSy)
{
    double x0 = m->xy[2 * p0], y0 = m->xy[2 * p0 + 1], x1 = m->xy[2 * p1], y1 = m->xy[2 * p1 + 1];
    *dSx = y1 - y0;
    *dSy = -(x1 - x0);
    double y = (y0 + y1) / 2;
    if (axi == 1) {
        *dSx = (*dSx) * y;
        *dSy = (*dSy) * y;
    }
}

/* Eddy viscosity that saBoundaryFaceViscFlux (sa.c:370-692) reports for one boundary face: fv1 of
 * saCalcFace (sa.c:273-290) times rho nt, from the inlet state (flag 1), the owner with the wall
 * temperature and nt = 0 (flag 4), the owner (flags 0, 2); 0 on adiabatic walls (flag 3). */
static double sa_face_eddy(const csu_config* c, int flag, const double* E)
{
    if (flag == CSU_BC_WALL) return 0.0;
    double rho = E[0], T = E[4], n = E[5];
    if (flag == CSU_BC_INLET) {
        rho = c->pin[0];
        T = c->pin[4];
        n = c->pin[5];
    } else if (flag == CSU_BC_WALLT) {
        T = c->t_wall;
        n = 0.0;
    }
    double mi_L = csu_host_sutherland(T);
    double n_L = mi_L / rho;
    double Cv1 = 7.1;
    double X = n / n_L;
    double aux = X * X * X;
    double fv1 = aux / (aux + Cv1 * Cv1 * Cv1);
    return fv1 * rho * n;
}

/* The surface writers of the viscous models, along the marker named by writeSurf (default "wall"; solver.c:
 * 1585-1594). Per boundary face: the ghost primitives of the last residual evaluation (boundary element P),
 * pressure coefficient, skin friction and heat flux from the face's viscous flux (components 1..3 of
 * boundaryFaceViscFlux and its SA/SST variants), y+ from the owner's wall distance, Mach; then each node of
 * the marker gets the mean of its faces. Columns the reference leaves undefined are written as 0: the
 * 'n' column of the laminar model (it reads past the five primitives of a boundary element), y+ of the
 * laminar model (the wall distance is never computed), 'q' of adiabatic laminar walls (the energy
 * component of the flux is never set), miEddy of SST (never set). */
static int write_surf(const char* wd, const csu_case* cs, const double* ghost, const double* bvisc,
                      const double* P)
{
    const csu_mesh* m = &cs->mesh;
    const csu_config* c = &cs->cfg;
    const int npr = c->nvar + 1;
    const char* target = csu_keywords_get(&cs->kw, "writeSurf");
    if (!target) target = "wall";
    FILE* f = open_in(wd, "surfData.csv", "w");
    if (!f) {
        csu_set_error("cannot write %ssurfData.csv", wd);
        return CSU_ERR_IO;
    }
    const double rin = c->pin[0], uin = c->pin[1], vin = c->pin[2], pin = c->pin[3];
    const double qdin = 0.5 * rin * (uin * uin + vin * vin);
    const int turb = c->sa || c->sst;
    const int nq = turb ? 13 : 12;
    int b0 = 0;
    for (int k = 0; k < m->n_markers; b0 += m->marker_nbf[k], k++) {
        if (strcmp(m->marker_name[k], target) != 0) continue;
        if (turb) fprintf(f, "x,y,rho,u,v,p,T,n,Cp,Cfx,Cfy,q,yplus,mach,miEddy,\n");
        else fprintf(f, "x,y,rho,u,v,p,T,n,Cp,Cfx,Cfy,q,yplus,mach,\n");
        const int ne = m->marker_nbf[k], flag = m->marker_flag[k];
        if (ne == 0) continue;
        double* D = calloc((size_t)nq * ne, sizeof(double));
        double* Dp = calloc((size_t)nq * (ne + 1), sizeof(double));
        int* d = calloc(ne + 1, sizeof(int));
        int* pn = calloc(ne + 1, sizeof(int));
        int* pn2 = calloc(m->n_points, sizeof(int));
        for (int i = 0; i < ne; i++) pn[i] = m->bface[3 * (b0 + i)];
        pn[ne] = m->bface[3 * (b0 + ne - 1) + 1];
        for (int i = 0; i < ne + 1; i++) pn2[pn[i]] = i;
        for (int i = 0; i < ne; i++) {
            const int b = b0 + i, p0 = m->bface[3 * b], p1 = m->bface[3 * b + 1], own = m->bface[3 * b + 2];
            double dSx, dSy;
            face_ds(m, c->axisymmetric, p0, p1, &dSx, &dSy);
            double dS = sqrt(dSx * dSx + dSy * dSy);
            const double* G = ghost + (size_t)b * npr;
            const double* fv = bvisc + (size_t)b * 4;
            double r = G[0], u = G[1], v = G[2], p = G[3], T = G[4];
            double Cp = (p - pin) / qdin;
            double Cfx = fv[0] / (dS * qdin);
            double Cfy = fv[1] / (dS * qdin);
            double q = (fv[2] - u * fv[0] - v * fv[1]) / dS;
            double tau = sqrt(fv[0] * fv[0] + fv[1] * fv[1]) / dS;
            double uplus = sqrt(tau / r);
            double dwall = m->wall_dist ? m->wall_dist[own] : 0.0;
            double yplus = fabs(r * uplus * dwall) / csu_host_sutherland(T);
            double cc = csu_host_T2c(c, T);
            double mach = sqrt(u * u + v * v) / cc;
            if (!turb && flag == CSU_BC_WALL) q = 0.0;
            double* col = D + i;
            col[0 * ne] = r;
            col[1 * ne] = u;
            col[2 * ne] = v;
            col[3 * ne] = p;
            col[4 * ne] = T;
            col[5 * ne] = turb ? G[5] : 0.0;
            col[6 * ne] = Cp;
            col[7 * ne] = Cfx;
            col[8 * ne] = Cfy;
            col[9 * ne] = q;
            col[10 * ne] = yplus;
            col[11 * ne] = mach;
            if (turb) col[12 * ne] = c->sa ? sa_face_eddy(c, flag, P + (size_t)own * npr) : 0.0;
        }
        for (int i = 0; i < ne; i++) {
            const int b = b0 + i, p0 = m->bface[3 * b], p1 = m->bface[3 * b + 1];
            for (int q = 0; q < nq; q++) {
                Dp[(size_t)q * (ne + 1) + pn2[p0]] += D[(size_t)q * ne + i];
                Dp[(size_t)q * (ne + 1) + pn2[p1]] += D[(size_t)q * ne + i];
            }
            d[pn2[p0]] += 1;
            d[pn2[p1]] += 1;
        }
        for (int i = 0; i < ne + 1; i++)
            for (int q = 0; q < nq; q++) Dp[(size_t)q * (ne + 1) + i] /= d[i];
        for (int i = 0; i < ne + 1; i++) {
            fprintf(f, "% .10e,", m->xy[2 * pn[i]]);
            fprintf(f, "% .10e,", m->xy[2 * pn[i] + 1]);
            for (int q = 0; q < nq; q++) fprintf(f, "% .10e,", Dp[(size_t)q * (ne + 1) + i]);
            fprintf(f, "\n");
        }
        free(D);
        free(Dp);
        free(d);
        free(pn);
        free(pn2);
    }
    fclose(f);
    return CSU_OK;
}

/* solverCalcCoeff2 (solver.c:1303-1340) per wall face, from the owner's gradients and primitives:
 * boundaryCalcTensorWall (boundary.c:744-794) for the laminar model, saCalcTensorWall (sa.c:795-852: the
 * wall-tangent shear in the txy column, zeros beside it, y+ from the wall distance) for SA and SST. */
static int write_friction(const char* wd, const csu_case* cs, const double* P, const double* G)
{
    const csu_mesh* m = &cs->mesh;
    const csu_config* c = &cs->cfg;
    int nc = m->n_cells, nv = c->nvar, npr = nv + 1;
    FILE* f = open_in(wd, "friction.csv", "w");
    if (!f) {
        csu_set_error("cannot write %sfriction.csv", wd);
        return CSU_ERR_IO;
    }
    int b = 0;
    for (int k = 0; k < m->n_markers; k++)
        for (int j = 0; j < m->marker_nbf[k]; j++, b++) {
            int fl = m->marker_flag[k];
            if (!(fl == CSU_BC_WALL || fl == CSU_BC_WALLT) || !(c->laminar || c->sa || c->sst)) continue;
            int e0 = m->bface[3 * b + 2], p0 = m->bface[3 * b], p1 = m->bface[3 * b + 1];
            double x0, y0;
            csu_mesh_center(m, e0, &x0, &y0);
            double x1 = (m->xy[2 * p0] + m->xy[2 * p1]) / 2, y1 = (m->xy[2 * p0 + 1] + m->xy[2 * p1 + 1]) / 2;
            double dx = x1 - x0, dy = y1 - y0, L = sqrt(dx * dx + dy * dy);
            const double* E = P + (size_t)e0 * npr;
            double dul = (0 - E[1]) / L, dvl = (0 - E[2]) / L;
            double duxm = G[(size_t)1 * nc + e0], dvxm = G[(size_t)2 * nc + e0];
            double duym = G[(size_t)(nv + 1) * nc + e0], dvym = G[(size_t)(nv + 2) * nc + e0];
            double dux = duxm + (dul - (duxm * dx + duym * dy) / L) * dx / L;
            double duy = duym + (dul - (duxm * dx + duym * dy) / L) * dy / L;
            double dvx = dvxm + (dvl - (dvxm * dx + dvym * dy) / L) * dx / L;
            double dvy = dvym + (dvl - (dvxm * dx + dvym * dy) / L) * dy / L;
            double mi = csu_host_sutherland(E[4]);
            double txx = 2 * mi * (dux - (dux + dvy) / 3);
            double tyy = 2 * mi * (dvy - (dux + dvy) / 3);
            double txy = mi * (duy + dvx);
            if (c->sa || c->sst) {
                double dSx, dSy;
                face_ds(m, c->axisymmetric, p0, p1, &dSx, &dSy);
                double dS = sqrt(dSx * dSx + dSy * dSy);
                double fx = (txx * dSx + txy * dSy) / dS;
                double fy = (txy * dSx + tyy * dSy) / dS;
                double ft = (fx * dSy - fy * dSx) / dS;
                double ut = sqrt(fabs(ft) / E[0]);
                double dwall = m->wall_dist ? m->wall_dist[e0] : 0.0;
                fprintf(f, "%e, %e, %e, %e, %e,\n", x1, 0.0, ft, 0.0, E[0] * dwall * ut / mi);
                continue;
            }
            double aux = 5.29 * x1 / sqrt(E[0] * E[1] * x1 / mi);
            fprintf(f, "%e, %e, %e, %e, %e,\n", x1, txx, txy, tyy, L / aux);
        }
    fclose(f);
    return CSU_OK;
}

int csu_run_case(const char* wd, int verbose)
{
    double t0 = now();
    csu_case* cs = NULL;
    csu_ctx* ctx = NULL;
    int st = csu_case_load(wd, &cs);
    if (st) return st;
    csu_mesh_desc d;
    csu_case_mesh(cs, &d);
    const csu_config* c = &cs->cfg;
    int nc = d.n_cells, nv = c->nvar;
    double *U = NULL, *hist = NULL, *P = NULL, *G = NULL;
    int wrote_wall = 0;
    FILE* conv = NULL;
    if ((st = csu_create(&d, c, &ctx))) goto done;
    U = malloc(sizeof(double) * (size_t)nv * nc);
    P = malloc(sizeof(double) * (size_t)(nv + 1) * nc);
    G = malloc(sizeof(double) * (size_t)2 * nv * nc);
    csu_case_initial_state(cs, U);
    if ((st = csu_set_state(ctx, U))) goto done;
    if (!c->tube) {
        int nmax, restart = 0;
        if ((st = csu_case_get_int(cs, "Nmax", &nmax))) goto done;
        csu_case_get_int(cs, "restart", &restart);
        conv = open_in(wd, "convergence.csv", restart ? "a" : "w");
        if (!conv) {
            csu_set_error("cannot write %sconvergence.csv", wd);
            st = CSU_ERR_IO;
            goto done;
        }
        const int chunk = 1000;
        const int visc = c->laminar || c->sa || c->sst;
        hist = malloc(sizeof(double) * (size_t)chunk * (nv + 4));
        if (verbose) printf("\nmain: running solution:\n");
        for (int it = 0; it < nmax;) {
            int n = nmax - it < chunk ? nmax - it : chunk;
            if (visc && it + n == nmax) {
                if (n > 1) n--;
                else {
                    /* the last iteration, with the views of its last residual evaluation for friction.csv */
                    if ((st = csu_iterate_views(ctx, it, hist, P, G))) goto done;
                    if ((st = write_friction(wd, cs, P, G))) goto done;
                    wrote_wall = 1;
                }
            }
            if (!wrote_wall && (st = csu_iterate(ctx, n, it, hist))) goto done;
            for (int r = 0; r < n; r++) {
                const double* h = hist + (size_t)r * (nv + 4);
                if (verbose) {
                    printf("%i, ", it + r);
                    for (int k = 0; k < nv; k++) printf(" %+.4e,", h[k]);
                    printf("\n%f, %f\n", h[nv] + h[nv + 1], h[nv + 2] + h[nv + 3]);
                }
                fprintf(conv, "%i,", it + r);
                for (int k = 0; k < nv; k++) fprintf(conv, " %+.4e,", h[k]);
                fprintf(conv, " %e, %e, %e, %e,", h[nv], h[nv + 1], h[nv + 2], h[nv + 3]);
                fprintf(conv, "\n");
            }
            it += n;
        }
        fclose(conv);
        conv = NULL;
        if (!wrote_wall) {
            /* inviscid (friction.csv holds no rows) or Nmax = 0 */
            if ((st = csu_dump(ctx, CSU_DUMP_GRAD, G)) || (st = csu_dump(ctx, CSU_DUMP_P, P))) goto done;
            if ((st = write_friction(wd, cs, P, G))) goto done;
        }
    } else {
        double tmax, t = 0;
        int steps = 0;
        if ((st = csu_case_get_double(cs, "tmax", &tmax))) goto done;
        if (verbose) printf("\nmain: running solution:\n");
        if ((st = csu_tube_run(ctx, tmax, &steps, &t))) goto done;
        if (verbose) printf("time %f s\n", t);
    }
    if (wrote_wall) {
        /* surfData.csv: the final state's primitives and ghost states, the last gradients */
        double* GP = malloc(sizeof(double) * (size_t)(nv + 1) * (d.n_bfaces > 0 ? d.n_bfaces : 1));
        double* BV = malloc(sizeof(double) * (size_t)4 * (d.n_bfaces > 0 ? d.n_bfaces : 1));
        st = csu_wall_data(ctx);
        if (!st) st = csu_dump(ctx, CSU_DUMP_GHOST_P, GP);
        if (!st) st = csu_dump(ctx, CSU_DUMP_BVISC, BV);
        if (!st) st = csu_dump(ctx, CSU_DUMP_P, P);
        if (!st) st = write_surf(wd, cs, GP, BV, P);
        free(GP);
        free(BV);
        if (st) goto done;
    }
    if ((st = csu_get_state(ctx, U))) goto done;
    if ((st = write_solution(wd, cs, U))) goto done;
    if ((st = csu_dump(ctx, CSU_DUMP_P, P))) goto done;
    if ((st = write_solution2(wd, cs, P))) goto done;
    if ((st = write_restart(wd, cs, U))) goto done;
    if (verbose) printf("\nDuration %f s\n", now() - t0);
done:
    if (conv) fclose(conv);
    free(U);
    free(hist);
    free(P);
    free(G);
    csu_destroy(ctx);
    csu_case_free(cs);
    return st;
}
