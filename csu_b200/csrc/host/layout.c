/*
 * layout.c -- builds the device data layout from the reference-order mesh.
 *
 * Locality: the reference stores cells in file order (its face list has a bandwidth close to the cell
 * count), so every gather misses. Cells are renumbered along a Hilbert curve through the centroids; a
 * warp of consecutive cells then touches neighbours a few cache lines away. Interior faces are sorted
 * by their lower renumbered cell and boundary faces by owner, so the face kernels stream cells in the
 * same order.
 *
 * Geometry that the reference recomputes in every loop (elementCenter 28% of its run time, meshCalcDS,
 * midpoints) is evaluated once here with the same expressions, so the device reads bit-identical values.
 * The least-squares normal equations of solverCalcGrad3 (solver.c:1031-1074) depend only on geometry: their
 * long double coefficients a, b, c and determinant are evaluated here exactly as the reference does (this
 * host's long double is the same x87 format) and handed to the device's exact extended-precision model,
 * together with per-neighbour weights for the faster, non-exact gradient variant.
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "layout.h"

static void center(const csu_mesh_desc* m, int c, double* x, double* y)
{
    int np = m->cell_npts[c];
    double sx = 0.0, sy = 0.0;
    for (int j = 0; j < np; j++) {
        int p = m->cell_nodes[4 * c + j];
        sx += m->xy[2 * p];
        sy += m->xy[2 * p + 1];
    }
    *x = sx / np;
    *y = sy / np;
}

/* meshCalcDS (mesh.c:720-740) */
static void calc_ds(const csu_mesh_desc* m, int axi, int p0, int p1, double* dSx, double* dSy)
{
    double x0 = m->xy[2 * p0], y0 = m->xy[2 * p0 + 1];
    double x1 = m->xy[2 * p1], y1 = m->xy[2 * p1 + 1];
    *dSx = y1 - y0;
    *dSy = -(x1 - x0);
    double y = (y0 + y1) / 2;
    if (axi == 1) {
        *dSx = (*dSx) * y;
        *dSy = (*dSy) * y;
    }
}

static double tri_area(const double* xy, int p0, int p1, int p2)
{
    double x1 = xy[2 * p0], x2 = xy[2 * p1], x3 = xy[2 * p2];
    double y1 = xy[2 * p0 + 1], y2 = xy[2 * p1 + 1], y3 = xy[2 * p2 + 1];
    return 0.5 * ((x1 - x2) * (y1 + y2) + (x2 - x3) * (y2 + y3) + (x3 - x1) * (y3 + y1));
}

/* Hilbert index of (x, y) on a 2^16 grid */
static unsigned long long hilbert_key(unsigned x, unsigned y)
{
    unsigned long long d = 0;
    for (unsigned s = 1u << 15; s > 0; s >>= 1) {
        unsigned rx = (x & s) > 0, ry = (y & s) > 0;
        d += (unsigned long long)s * s * ((3 * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) {
                x = s - 1 - x;
                y = s - 1 - y;
            }
            unsigned t = x;
            x = y;
            y = t;
        }
    }
    return d;
}

/* x87 long double as significand (bit 63 set) and exponent<<1|sign, the device's ext80 format */
static void split_ld(long double v, unsigned long long* m, int* es)
{
    if (v == 0) {
        *m = 0;
        *es = signbit(v) ? 1 : 0;
        return;
    }
    int e;
    long double f = frexpl(fabsl(v), &e);
    *m = (unsigned long long)ldexpl(f, 64);
    *es = ((e - 64) * 2) | (v < 0 ? 1 : 0);
}

/* floor((2^128 - 1) / d) - 2^64 for a normalised d (invariant-divisor reciprocal) */
static unsigned long long recip64(unsigned long long d)
{
    if (d == 0) return 0;
    unsigned __int128 all = ~(unsigned __int128)0;
    return (unsigned long long)(all / d - ((unsigned __int128)1 << 64));
}

typedef struct {
    unsigned long long key;
    int id;
} keyed;

static int cmp_keyed(const void* a, const void* b)
{
    const keyed* x = a;
    const keyed* y = b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->id - y->id;
}

void csu_layout_free(csu_layout* L)
{
    void* ptrs[] = {L->cell_new2old, L->cell_old2new, L->face_new2old, L->face_old2new, L->bface_new2old,
                    L->bface_old2new, L->npts, L->nint, L->nslot, L->nei, L->wx, L->wy, L->ex, L->ey,
                    L->fslot, L->fnb, L->omega, L->sxh, L->syh, L->xc, L->yc, L->wall_d, L->dslat, L->fe0, L->fe1,
                    L->fdsx, L->fdsy, L->fds, L->r0x, L->r0y, L->r1x, L->r1y, L->fdist, L->bown, L->bflag,
                    L->bold, L->bdsx, L->bdsy, L->bds, L->bmx, L->bmy, L->ldx, L->ldy, L->lm, L->les, L->lrv, L->lq,
                    L->fdx, L->fdy, L->bdx, L->bdy, L->bL, L->bunx, L->buny, L->bds2, L->color,
                    L->color_start, L->color_cells};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
    memset(L, 0, sizeof(*L));
}

int csu_layout_sequential_colors(csu_layout* L)
{
    const int nc = L->nc;
    int* start = malloc(sizeof(int) * (nc + 1));
    int* cells = malloc(sizeof(int) * (nc > 0 ? nc : 1));
    if (!start || !cells) {
        free(start);
        free(cells);
        return CSU_ERR_OOM;
    }
    for (int c = 0; c < nc; c++) {
        L->color[c] = L->cell_new2old[c];
        cells[L->cell_new2old[c]] = c;
    }
    for (int k = 0; k <= nc; k++) start[k] = k;
    free(L->color_start);
    free(L->color_cells);
    L->color_start = start;
    L->color_cells = cells;
    L->ncolors = nc;
    return CSU_OK;
}

int csu_layout_build(const csu_mesh_desc* m, int axi, csu_layout* L)
{
    memset(L, 0, sizeof(*L));
    int nc = m->n_cells, nf = m->n_faces, nb = m->n_bfaces;
    L->nc = nc;
    L->nf = nf;
    L->nb = nb;
    size_t c4 = (size_t)4 * nc;
#define ALLOC(p, n) (p) = calloc((n) > 0 ? (n) : 1, sizeof(*(p)))
    ALLOC(L->cell_new2old, nc); ALLOC(L->cell_old2new, nc);
    ALLOC(L->face_new2old, nf); ALLOC(L->face_old2new, nf);
    ALLOC(L->bface_new2old, nb); ALLOC(L->bface_old2new, nb);
    ALLOC(L->npts, nc); ALLOC(L->nint, nc); ALLOC(L->nslot, nc); ALLOC(L->nei, c4);
    ALLOC(L->wx, c4); ALLOC(L->wy, c4); ALLOC(L->ex, c4); ALLOC(L->ey, c4); ALLOC(L->fslot, c4); ALLOC(L->fnb, c4);
    ALLOC(L->ldx, c4); ALLOC(L->ldy, c4); ALLOC(L->lm, c4); ALLOC(L->les, c4); ALLOC(L->lrv, nc); ALLOC(L->lq, 2 * c4);
    ALLOC(L->omega, nc); ALLOC(L->sxh, nc); ALLOC(L->syh, nc); ALLOC(L->xc, nc); ALLOC(L->yc, nc);
    ALLOC(L->dslat, nc);
    if (m->wall_dist) ALLOC(L->wall_d, nc);
    ALLOC(L->fe0, nf); ALLOC(L->fe1, nf); ALLOC(L->fdsx, nf); ALLOC(L->fdsy, nf); ALLOC(L->fds, nf);
    ALLOC(L->r0x, nf); ALLOC(L->r0y, nf); ALLOC(L->r1x, nf); ALLOC(L->r1y, nf); ALLOC(L->fdist, nf);
    ALLOC(L->bown, nb); ALLOC(L->bflag, nb); ALLOC(L->bold, nb); ALLOC(L->bdsx, nb); ALLOC(L->bdsy, nb);
    ALLOC(L->bds, nb); ALLOC(L->bmx, nb); ALLOC(L->bmy, nb);
    ALLOC(L->fdx, nf); ALLOC(L->fdy, nf); ALLOC(L->bdx, nb); ALLOC(L->bdy, nb); ALLOC(L->bL, nb);
    ALLOC(L->bunx, nb); ALLOC(L->buny, nb); ALLOC(L->bds2, nb);
#undef ALLOC
    if (!L->bmy || !L->fslot || !L->fdist) {
        csu_layout_free(L);
        return CSU_ERR_OOM;
    }

    /* centroids in reference order */
    double* cx = malloc(sizeof(double) * (nc > 0 ? nc : 1));
    double* cy = malloc(sizeof(double) * (nc > 0 ? nc : 1));
    double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
    for (int o = 0; o < nc; o++) {
        center(m, o, &cx[o], &cy[o]);
        if (cx[o] < xmin) xmin = cx[o];
        if (cx[o] > xmax) xmax = cx[o];
        if (cy[o] < ymin) ymin = cy[o];
        if (cy[o] > ymax) ymax = cy[o];
    }
    double span = fmax(xmax - xmin, ymax - ymin);
    if (!(span > 0)) span = 1.0;

    /* cell order along the Hilbert curve */
    keyed* k = malloc(sizeof(keyed) * (size_t)(nc > nf ? (nc > nb ? nc : nb) : (nf > nb ? nf : nb)) + 1);
    for (int o = 0; o < nc; o++) {
        unsigned qx = (unsigned)((cx[o] - xmin) / span * 65535.0);
        unsigned qy = (unsigned)((cy[o] - ymin) / span * 65535.0);
        k[o].key = hilbert_key(qx, qy);
        k[o].id = o;
    }
    qsort(k, nc, sizeof(keyed), cmp_keyed);
    for (int c = 0; c < nc; c++) {
        L->cell_new2old[c] = k[c].id;
        L->cell_old2new[k[c].id] = c;
    }
    /* faces by (lower, upper) renumbered cell */
    for (int f = 0; f < nf; f++) {
        unsigned a = L->cell_old2new[m->con[4 * f]], b = L->cell_old2new[m->con[4 * f + 1]];
        unsigned lo = a < b ? a : b, hi = a < b ? b : a;
        k[f].key = ((unsigned long long)lo << 32) | hi;
        k[f].id = f;
    }
    qsort(k, nf, sizeof(keyed), cmp_keyed);
    for (int f = 0; f < nf; f++) {
        L->face_new2old[f] = k[f].id;
        L->face_old2new[k[f].id] = f;
    }
    for (int b = 0; b < nb; b++) {
        k[b].key = ((unsigned long long)L->cell_old2new[m->bface[3 * b + 2]] << 32) | (unsigned)b;
        k[b].id = b;
    }
    qsort(k, nb, sizeof(keyed), cmp_keyed);
    for (int b = 0; b < nb; b++) {
        L->bface_new2old[b] = k[b].id;
        L->bface_old2new[k[b].id] = b;
    }
    free(k);

    /* boundary-face flags (marker-major reference numbering) */
    int* oflag = malloc(sizeof(int) * (nb > 0 ? nb : 1));
    for (int mk = 0, b = 0; mk < m->n_markers; mk++)
        for (int j = 0; j < m->marker_nbf[mk]; j++, b++) oflag[b] = m->marker_flag[mk];

    /* interior faces */
    for (int f = 0; f < nf; f++) {
        int o = L->face_new2old[f];
        int e0 = m->con[4 * o], e1 = m->con[4 * o + 1], p0 = m->con[4 * o + 2], p1 = m->con[4 * o + 3];
        double dSx, dSy;
        calc_ds(m, axi, p0, p1, &dSx, &dSy);
        L->fe0[f] = L->cell_old2new[e0];
        L->fe1[f] = L->cell_old2new[e1];
        L->fdsx[f] = dSx;
        L->fdsy[f] = dSy;
        L->fds[f] = sqrt(dSx * dSx + dSy * dSy);
        double xm = (m->xy[2 * p0] + m->xy[2 * p1]) * 0.5;
        double ym = (m->xy[2 * p0 + 1] + m->xy[2 * p1 + 1]) * 0.5;
        L->r0x[f] = xm - cx[e0];
        L->r0y[f] = ym - cy[e0];
        L->r1x[f] = xm - cx[e1];
        L->r1y[f] = ym - cy[e1];
        L->fdx[f] = cx[e1] - cx[e0];
        L->fdy[f] = cy[e1] - cy[e0];
        L->fdist[f] = sqrt(L->fdx[f] * L->fdx[f] + L->fdy[f] * L->fdy[f]);
    }
    /* boundary faces */
    for (int b = 0; b < nb; b++) {
        int o = L->bface_new2old[b];
        int p0 = m->bface[3 * o], p1 = m->bface[3 * o + 1];
        double dSx, dSy;
        calc_ds(m, axi, p0, p1, &dSx, &dSy);
        L->bown[b] = L->cell_old2new[m->bface[3 * o + 2]];
        L->bflag[b] = oflag[o];
        L->bold[b] = o;
        L->bdsx[b] = dSx;
        L->bdsy[b] = dSy;
        L->bds[b] = sqrt(dSx * dSx + dSy * dSy);
        /* elementCenter of the two-node boundary element */
        L->bmx[b] = (m->xy[2 * p0] + m->xy[2 * p1]) / 2;
        L->bmy[b] = (m->xy[2 * p0 + 1] + m->xy[2 * p1 + 1]) / 2;
        {
            int ow = m->bface[3 * o + 2];
            double ox = 0.0, oy = 0.0;
            center(m, ow, &ox, &oy);
            double x1 = (m->xy[2 * p0] + m->xy[2 * p1]) * 0.5, y1 = (m->xy[2 * p0 + 1] + m->xy[2 * p1 + 1]) * 0.5;
            L->bdx[b] = x1 - ox;
            L->bdy[b] = y1 - oy;
            L->bL[b] = sqrt(L->bdx[b] * L->bdx[b] + L->bdy[b] * L->bdy[b]);
            double ux = m->xy[2 * p1 + 1] - m->xy[2 * p0 + 1], uy = -(m->xy[2 * p1] - m->xy[2 * p0]);
            double s2 = sqrt(ux * ux + uy * uy);
            L->bunx[b] = ux / s2;
            L->buny[b] = uy / s2;
            L->bds2[b] = axi == 1 ? s2 * (m->xy[2 * p0 + 1] + m->xy[2 * p1 + 1]) * 0.5 : s2;
        }
    }
    free(oflag);

    /* cells */
    L->vol_max = 0.0;
    L->max_npts = 0;
    for (int c = 0; c < nc; c++) {
        int o = L->cell_new2old[c];
        int np = m->cell_npts[o];
        const int* nodes = m->cell_nodes + 4 * o;
        L->npts[c] = np;
        if (np > L->max_npts) L->max_npts = np;
        L->nint[c] = m->cell_nint[o];
        L->xc[c] = cx[o];
        L->yc[c] = cy[o];
        /* meshCalcOmega (mesh.c:420-441) */
        double om = tri_area(m->xy, nodes[0], nodes[1], nodes[2]);
        if (np == 4) om += tri_area(m->xy, nodes[2], nodes[3], nodes[0]);
        L->dslat[c] = om; /* meshCalcDSlateral (mesh.c:404-418) */
        if (axi == 1) om *= cy[o];
        L->omega[c] = om;
        L->vol_max = fmax(om, L->vol_max);
        if (L->wall_d) L->wall_d[c] = m->wall_dist[o];

        double sxm = 0., sym = 0.;
        for (int j = 0; j < 4; j++) {
            L->nei[(size_t)j * nc + c] = -1;
            L->fslot[(size_t)j * nc + c] = 0;
        }
        for (int j = 0; j < np; j++) {
            int p0 = nodes[j], p1 = nodes[(j + 1) % np];
            double dSx, dSy;
            calc_ds(m, axi, p0, p1, &dSx, &dSy);
            sxm += fabs(dSx);
            sym += fabs(dSy);
            double xm = (m->xy[2 * p0] + m->xy[2 * p1]) * 0.5;
            double ym = (m->xy[2 * p0 + 1] + m->xy[2 * p1 + 1]) * 0.5;
            L->ex[(size_t)j * nc + c] = xm - cx[o];
            L->ey[(size_t)j * nc + c] = ym - cy[o];
        }
        L->sxh[c] = sxm * 0.5;
        L->syh[c] = sym * 0.5;

        /* neighbours and least-squares weights (solverCalcGrad3) */
        double dx[4], dy[4];
        long double a = 0, bb = 0, cc = 0;
        for (int j = 0; j < np; j++) {
            int n = m->cell_nei[4 * o + j];
            double xn, yn;
            if (n >= 0) {
                L->nei[(size_t)j * nc + c] = L->cell_old2new[n];
                xn = cx[n];
                yn = cy[n];
            } else {
                int bo = -n - 1;
                int bn = L->bface_old2new[bo];
                L->nei[(size_t)j * nc + c] = nc + bn;
                xn = L->bmx[bn];
                yn = L->bmy[bn];
            }
            dx[j] = xn - cx[o];
            dy[j] = yn - cy[o];
            a += dx[j] * dx[j];
            bb += dx[j] * dy[j];
            cc += dy[j] * dy[j];
        }
        long double det = a * cc - bb * bb;
        long double k4[4] = {a, bb, cc, det};
        for (int q = 0; q < 4; q++) split_ld(k4[q], &L->lm[(size_t)q * nc + c], &L->les[(size_t)q * nc + c]);
        L->lrv[c] = recip64(L->lm[(size_t)3 * nc + c]);
        /* the same as exact double-doubles for the device's certified FP64 evaluation: a, b, c as
           (RN53, remainder) and 1/det to ~2^-103 (FP64 reciprocal + one Newton correction) */
        for (int q = 0; q < 3; q++) {
            double h = (double)k4[q];
            L->lq[2 * ((size_t)q * nc + c)] = h;
            L->lq[2 * ((size_t)q * nc + c) + 1] = (double)(k4[q] - (long double)h);
        }
        {
            double dh = (double)det, dl = (double)(det - (long double)dh);
            double r = 1.0 / dh;
            double e = fma(-dh, r, 1.0);
            e = e - dl * r;
            double re = e * r, rs = r + re;
            L->lq[2 * ((size_t)3 * nc + c)] = rs;
            L->lq[2 * ((size_t)3 * nc + c) + 1] = re - (rs - r);
        }
        for (int j = 0; j < np; j++) {
            L->ldx[(size_t)j * nc + c] = dx[j];
            L->ldy[(size_t)j * nc + c] = dy[j];
            L->wx[(size_t)j * nc + c] = (double)((cc * dx[j] - bb * dy[j]) / det);
            L->wy[(size_t)j * nc + c] = (double)((-bb * dx[j] + a * dy[j]) / det);
        }

        /* face slots: interior faces in ELEMENT.f order, then this cell's boundary faces in reference order */
        int ns = 0;
        for (int j = 0; j < m->cell_nint[o]; j++) {
            int sf = m->cell_faces[4 * o + j];
            int fo = sf > 0 ? sf - 1 : -sf - 1;
            int fnew = L->face_old2new[fo];
            L->fslot[(size_t)ns * nc + c] = sf > 0 ? fnew + 1 : -(fnew + 1);
            ns++;
        }
        L->nslot[c] = ns;
    }
    /* boundary face slots, ascending reference id per owner */
    for (int bo = 0; bo < nb; bo++) {
        int bn = L->bface_old2new[bo];
        int c = L->bown[bn];
        int ns = L->nslot[c];
        if (ns >= 4) {
            free(cx);
            free(cy);
            csu_layout_free(L);
            return CSU_ERR_INPUT;
        }
        L->fslot[(size_t)ns * nc + c] = nf + bn + 1;
        L->nslot[c] = ns + 1;
    }
    /* neighbour across each interior face slot (the sweeps gather through it in one step) */
    for (size_t q = 0; q < c4; q++) L->fnb[q] = -1;
    for (int c = 0; c < nc; c++)
        for (int j = 0; j < L->nint[c]; j++) {
            int sf = L->fslot[(size_t)j * nc + c];
            int f = (sf > 0 ? sf : -sf) - 1;
            L->fnb[(size_t)j * nc + c] = sf > 0 ? L->fe1[f] : L->fe0[f];
        }
    /* greedy colouring in the renumbered (Hilbert) order: the multicolour Gauss-Seidel of LU-SGS */
    L->color = malloc(sizeof(int) * (nc > 0 ? nc : 1));
    L->ncolors = 0;
    for (int c = 0; c < nc; c++) {
        unsigned used = 0;
        for (int j = 0; j < L->nint[c]; j++) {
            int sf = L->fslot[(size_t)j * nc + c];
            int f = sf > 0 ? sf - 1 : -sf - 1;
            int nb = sf > 0 ? L->fe1[f] : L->fe0[f];
            if (nb < c) used |= 1u << L->color[nb];
        }
        int k = 0;
        while (used & (1u << k)) k++;
        L->color[c] = k;
        if (k + 1 > L->ncolors) L->ncolors = k + 1;
    }
    L->color_start = calloc(L->ncolors + 1, sizeof(int));
    L->color_cells = malloc(sizeof(int) * (nc > 0 ? nc : 1));
    for (int c = 0; c < nc; c++) L->color_start[L->color[c] + 1]++;
    for (int k = 0; k < L->ncolors; k++) L->color_start[k + 1] += L->color_start[k];
    {
        int* fill = malloc(sizeof(int) * (L->ncolors + 1));
        memcpy(fill, L->color_start, sizeof(int) * (L->ncolors + 1));
        for (int c = 0; c < nc; c++) L->color_cells[fill[L->color[c]]++] = c;
        free(fill);
    }
    free(cx);
    free(cy);
    return CSU_OK;
}

/*
 * Green-Gauss gradient weights (an extension; the reference uses least squares, solver.c:1031-1074):
 * grad q_i = (1 / Omega_i) sum_j q_f S_j with the face value q_f = (q_i + q_j) / 2 and outward face vectors
 * S_j; since sum_j S_j = 0 on a closed planar cell, grad q_i = sum_j (q_j - q_i) S_j / (2 Omega_i), the
 * same linear form in the neighbour differences as the least-squares weights, which it replaces.
 */
int csu_layout_green_gauss(csu_layout* L)
{
    const int nc = L->nc, nf = L->nf;
    for (int c = 0; c < nc; c++) {
        const double w = 0.5 / L->omega[c];
        for (int j = 0; j < L->npts[c]; j++) {
            int n = L->nei[(size_t)j * nc + c];
            double sx = 0.0, sy = 0.0;
            int found = 0;
            if (n >= nc) {
                int b = n - nc;
                sx = L->bdsx[b];
                sy = L->bdsy[b];
                found = 1;
            } else {
                for (int s = 0; s < L->nint[c] && !found; s++) {
                    int sf = L->fslot[(size_t)s * nc + c];
                    int f = (sf > 0 ? sf : -sf) - 1;
                    if (f >= nf) continue;
                    int other = L->fe0[f] == c ? L->fe1[f] : L->fe0[f];
                    if (other != n) continue;
                    double sg = L->fe0[f] == c ? 1.0 : -1.0;
                    sx = sg * L->fdsx[f];
                    sy = sg * L->fdsy[f];
                    found = 1;
                }
            }
            if (!found) return CSU_ERR_INPUT;
            L->wx[(size_t)j * nc + c] = sx * w;
            L->wy[(size_t)j * nc + c] = sy * w;
        }
    }
    return CSU_OK;
}
