/*
 * su2.c -- SU2 mesh reader and face connectivity, integer-exact with the reference's meshInit.
 *
 * Everything downstream (face order of the flux loop, neighbour order of the gradients, signed face
 * lists, boundary orientation) depends on these integers, so this file reproduces the reference's
 * results exactly while using its own data structures:
 *
 *  tokenizer    a token is the run of characters before the next ' ', '\r' or '\n' (meshGetWord,
 *               mesh.c:10-42), so consecutive separators give empty tokens and marker lines need their
 *               trailing space (mesh.c:102-107 reads four tokens per boundary line). Unlike the reference,
 *               end of file ends a token instead of looping, and counts/types are validated.
 *  orientation  cells with negative area (meshCalcOmega, mesh.c:420-441, times the centroid y when
 *               axisymmetric) have their node order reversed (mesh.c:222-242).
 *  faces        half-edges (p[j], p[j+1]) are inserted cell by cell into a hash table of Nelem+Np
 *               buckets, bucket = floor(size * frac((p0+p1) * (sqrt(5)-1)/2)) (mesh.c:1083-1090); an
 *               edge pairs with the first not-yet-paired half-edge (q0,q1) of its bucket chain with
 *               q0 == p1 and q1 == p0, otherwise it is appended to the chain (mesh.c:1092-1142). Faces
 *               are the paired half-edges in bucket order, then chain order (mesh.c:1192-1216), keeping
 *               the first half-edge's cell as e0 and its nodes as p0, p1.
 *  neighbours   interior neighbours in face order (mesh.c:792-809), then per marker and boundary element
 *               the lowest-numbered cell containing both of its nodes (mesh.c:812-830; counted the way
 *               meshBCIsConnect, mesh.c:766-790, counts) -- found here through a point->cell index
 *               instead of the reference's O(Nbc*Ncell) scan.
 *  orientation  boundary edges are flipped unless (p0,p1) is a consecutive node pair of the owner
 *               (meshPOri/meshFixBorderOrientation, mesh.c:948-1009).
 *  face lists   f[j] = +(face+1) where the cell is e0, -(face+1) where it is e1, in face order
 *               (meshCalcFaces, mesh.c:1011-1037).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "case.h"

typedef struct {
    const char* s;
    size_t len, pos;
} tokstream;

/* next token into buf (cap bytes); returns 0 at end of input with an empty token */
static int next_token(tokstream* ts, char* buf, int cap)
{
    int n = 0;
    if (ts->pos >= ts->len) {
        buf[0] = '\0';
        return 0;
    }
    while (ts->pos < ts->len) {
        char c = ts->s[ts->pos++];
        if (c == ' ' || c == '\r' || c == '\n') break;
        if (n < cap - 1) buf[n++] = c;
    }
    buf[n] = '\0';
    return 1;
}

void csu_mesh_free(csu_mesh* m)
{
    free(m->xy); free(m->cell_npts); free(m->cell_nodes); free(m->con); free(m->cell_nint);
    free(m->cell_faces); free(m->cell_nei); free(m->marker_nbf); free(m->marker_flag);
    free(m->marker_name); free(m->bface); free(m->omega); free(m->wall_dist);
    memset(m, 0, sizeof(*m));
}

void csu_mesh_center(const csu_mesh* m, int cell, double* x, double* y)
{
    /* elementCenter, mesh.c:371-386: vertex average */
    int np = m->cell_npts[cell];
    double sx = 0.0, sy = 0.0;
    for (int j = 0; j < np; j++) {
        int p = m->cell_nodes[4 * cell + j];
        sx += m->xy[2 * p];
        sy += m->xy[2 * p + 1];
    }
    *x = sx / np;
    *y = sy / np;
}

static double tri_area(const double* xy, int p0, int p1, int p2)
{
    /* meshCalcOmegaTri, mesh.c:388-401 */
    double x1 = xy[2 * p0], x2 = xy[2 * p1], x3 = xy[2 * p2];
    double y1 = xy[2 * p0 + 1], y2 = xy[2 * p1 + 1], y3 = xy[2 * p2 + 1];
    return 0.5 * ((x1 - x2) * (y1 + y2) + (x2 - x3) * (y2 + y3) + (x3 - x1) * (y3 + y1));
}

double csu_mesh_cell_omega(const csu_mesh* m, int cell, int axi)
{
    const int* p = m->cell_nodes + 4 * cell;
    double a = tri_area(m->xy, p[0], p[1], p[2]);
    if (m->cell_npts[cell] == 4) a += tri_area(m->xy, p[2], p[3], p[0]);
    if (axi == 1) {
        double x, y;
        csu_mesh_center(m, cell, &x, &y);
        a *= y;
    }
    return a;
}

/* ---------------------------------------------------------------- face hashing (mesh.c:1039-1218) */
typedef struct {
    int p0, p1, e0, e1, full, next;
} halfedge;

static int hash_bucket(int size, int p0, int p1)
{
    const double c = (sqrt(5) - 1.0) / 2.0;
    double aux = (p0 + p1) * c;
    aux = aux - floor(aux);
    return (int)floor(size * aux);
}

static int build_faces(csu_mesh* m)
{
    int size = m->n_cells + m->n_points;
    int* head = malloc(sizeof(int) * size);
    int* tail = malloc(sizeof(int) * size);
    halfedge* he = malloc(sizeof(halfedge) * (size_t)4 * m->n_cells + 1);
    if (!head || !tail || !he) {
        free(head); free(tail); free(he);
        csu_set_error("out of host memory building faces");
        return CSU_ERR_OOM;
    }
    for (int b = 0; b < size; b++) head[b] = tail[b] = -1;
    int nhe = 0, nfaces = 0;
    for (int i = 0; i < m->n_cells; i++) {
        int np = m->cell_npts[i];
        for (int j = 0; j < np; j++) {
            int p0 = m->cell_nodes[4 * i + j], p1 = m->cell_nodes[4 * i + (j + 1) % np];
            int b = hash_bucket(size, p0, p1);
            int matched = 0;
            for (int h = head[b]; h >= 0; h = he[h].next) {
                if (!he[h].full && he[h].p0 == p1 && he[h].p1 == p0) {
                    he[h].e1 = i;
                    he[h].full = 1;
                    nfaces++;
                    matched = 1;
                    break;
                }
            }
            if (!matched) {
                halfedge* e = &he[nhe];
                e->p0 = p0; e->p1 = p1; e->e0 = i; e->e1 = -1; e->full = 0; e->next = -1;
                if (head[b] < 0) head[b] = nhe;
                else he[tail[b]].next = nhe;
                tail[b] = nhe;
                nhe++;
            }
        }
    }
    m->n_faces = nfaces;
    m->con = malloc(sizeof(int) * 4 * (size_t)(nfaces > 0 ? nfaces : 1));
    int f = 0;
    for (int b = 0; b < size; b++)
        for (int h = head[b]; h >= 0; h = he[h].next)
            if (he[h].full) {
                m->con[4 * f] = he[h].e0;
                m->con[4 * f + 1] = he[h].e1;
                m->con[4 * f + 2] = he[h].p0;
                m->con[4 * f + 3] = he[h].p1;
                f++;
            }
    free(head); free(tail); free(he);
    return CSU_OK;
}

/* ------------------------------------------------ boundary elements to cells (mesh.c:766-830) */
static int build_neighbours(csu_mesh* m)
{
    int nc = m->n_cells;
    int* cnt = calloc(nc, sizeof(int)); /* neighbours recorded per cell (ELEMENT.neiN) */
    /* point -> cells incidence, ascending cell ids */
    int* pstart = calloc((size_t)m->n_points + 1, sizeof(int));
    int total = 0;
    for (int i = 0; i < nc; i++) total += m->cell_npts[i];
    int* plist = malloc(sizeof(int) * (size_t)(total > 0 ? total : 1));
    if (!cnt || !pstart || !plist) {
        free(cnt); free(pstart); free(plist);
        csu_set_error("out of host memory building neighbours");
        return CSU_ERR_OOM;
    }
    for (int i = 0; i < nc; i++)
        for (int j = 0; j < m->cell_npts[i]; j++) pstart[m->cell_nodes[4 * i + j] + 1]++;
    for (int p = 0; p < m->n_points; p++) pstart[p + 1] += pstart[p];
    int* fill = malloc(sizeof(int) * (size_t)(m->n_points > 0 ? m->n_points : 1));
    memcpy(fill, pstart, sizeof(int) * m->n_points);
    for (int i = 0; i < nc; i++)
        for (int j = 0; j < m->cell_npts[i]; j++) {
            int p = m->cell_nodes[4 * i + j];
            /* a cell listing a point twice appears twice; harmless for the first-match search */
            plist[fill[p]++] = i;
        }
    free(fill);

    for (int i = 0; i < 4 * nc; i++) m->cell_nei[i] = 0x7fffffff;
    for (int f = 0; f < m->n_faces; f++) {
        int e0 = m->con[4 * f], e1 = m->con[4 * f + 1];
        if (cnt[e0] >= m->cell_npts[e0] || cnt[e1] >= m->cell_npts[e1]) {
            csu_set_error("mesh: cell %d or %d has more faces than nodes", e0, e1);
            goto fail;
        }
        m->cell_nei[4 * e0 + cnt[e0]++] = e1;
        m->cell_nei[4 * e1 + cnt[e1]++] = e0;
    }
    for (int b = 0; b < m->n_bfaces; b++) {
        int q0 = m->bface[3 * b], q1 = m->bface[3 * b + 1];
        int best = -1;
        /* candidates: cells holding q0 or q1; the answer is the lowest id with link == 2 */
        for (int pass = 0; pass < 2; pass++) {
            int q = pass == 0 ? q0 : q1;
            for (int k = pstart[q]; k < pstart[q + 1]; k++) {
                int c = plist[k];
                if (best >= 0 && c >= best) break;
                int link = 0;
                for (int jj = 0; jj < m->cell_npts[c]; jj++) {
                    int p = m->cell_nodes[4 * c + jj];
                    link += (q0 == p) + (q1 == p);
                }
                if (link == 2) {
                    best = c;
                    break;
                }
            }
        }
        if (best < 0) {
            csu_set_error("mesh: boundary element %d (%d, %d) touches no cell", b, q0, q1);
            goto fail;
        }
        if (cnt[best] >= m->cell_npts[best]) {
            csu_set_error("mesh: cell %d has more neighbours than nodes", best);
            goto fail;
        }
        m->bface[3 * b + 2] = best;
        m->cell_nei[4 * best + cnt[best]++] = -(1 + b);
    }
    /* every edge needs a neighbour: the reference would follow a dangling pointer (an edge with neither a
       second cell nor a boundary marker); refuse such meshes */
    for (int c = 0; c < nc; c++)
        if (cnt[c] != m->cell_npts[c]) {
            csu_set_error("mesh: cell %d has %d edges but %d neighbours (an edge with neither a second cell nor "
                          "a boundary marker)", c, m->cell_npts[c], cnt[c]);
            goto fail;
        }
    free(cnt); free(pstart); free(plist);
    return CSU_OK;
fail:
    free(cnt); free(pstart); free(plist);
    return CSU_ERR_INPUT;
}

static int pori(const csu_mesh* m, int cell, int p0, int p1)
{
    int ans = -1, np = m->cell_npts[cell];
    for (int i = 0; i < np; i++)
        if (m->cell_nodes[4 * cell + i] == p0 && m->cell_nodes[4 * cell + (i + 1) % np] == p1) ans = 1;
    return ans;
}

static int parse_int_token(tokstream* ts, const char* what, int* out)
{
    char s[128];
    if (!next_token(ts, s, sizeof(s))) {
        csu_set_error("mesh.su2: unexpected end of file reading %s", what);
        return CSU_ERR_INPUT;
    }
    *out = atoi(s);
    return CSU_OK;
}

int csu_mesh_read_su2(const char* text, size_t len, int axi, csu_mesh* m)
{
    tokstream ts = {text, len, 0};
    char s[128];
    int st;
    memset(m, 0, sizeof(*m));

    next_token(&ts, s, sizeof(s));
    if (strcmp(s, "NDIME=") == 0) {
        if ((st = parse_int_token(&ts, "NDIME", &m->ndim))) return st;
    }
    next_token(&ts, s, sizeof(s));
    if (strcmp(s, "NELEM=") != 0) {
        csu_set_error("mesh.su2: expected NELEM=, got '%s'", s);
        return CSU_ERR_INPUT;
    }
    if ((st = parse_int_token(&ts, "NELEM", &m->n_cells))) return st;
    if (m->n_cells <= 0) {
        csu_set_error("mesh.su2: NELEM must be positive");
        return CSU_ERR_INPUT;
    }
    int nc = m->n_cells;
    m->cell_npts = malloc(sizeof(int) * nc);
    m->cell_nodes = malloc(sizeof(int) * 4 * (size_t)nc);
    m->cell_nint = calloc(nc, sizeof(int));
    m->cell_faces = calloc(4 * (size_t)nc, sizeof(int));
    m->cell_nei = malloc(sizeof(int) * 4 * (size_t)nc);
    m->omega = malloc(sizeof(double) * nc);
    if (!m->cell_npts || !m->cell_nodes || !m->cell_nint || !m->cell_faces || !m->cell_nei || !m->omega) {
        csu_mesh_free(m);
        csu_set_error("out of host memory reading mesh");
        return CSU_ERR_OOM;
    }
    for (int i = 0; i < nc; i++) {
        int type, np;
        if ((st = parse_int_token(&ts, "element type", &type))) goto fail;
        if (type == 5) np = 3;
        else if (type == 9) np = 4;
        else {
            csu_set_error("mesh.su2: element %d has unsupported type %d (5 triangle, 9 quad)", i, type);
            st = CSU_ERR_INPUT;
            goto fail;
        }
        m->cell_npts[i] = np;
        for (int j = 0; j < 4; j++) m->cell_nodes[4 * i + j] = -1;
        for (int j = 0; j < np; j++)
            if ((st = parse_int_token(&ts, "element node", &m->cell_nodes[4 * i + j]))) goto fail;
        next_token(&ts, s, sizeof(s)); /* element index */
    }
    next_token(&ts, s, sizeof(s));
    if (strcmp(s, "NPOIN=") != 0) {
        csu_set_error("mesh.su2: expected NPOIN=, got '%s'", s);
        st = CSU_ERR_INPUT;
        goto fail;
    }
    if ((st = parse_int_token(&ts, "NPOIN", &m->n_points))) goto fail;
    if (m->n_points <= 0) {
        csu_set_error("mesh.su2: NPOIN must be positive");
        st = CSU_ERR_INPUT;
        goto fail;
    }
    m->xy = malloc(sizeof(double) * 2 * (size_t)m->n_points);
    for (int p = 0; p < m->n_points; p++) {
        for (int d = 0; d < 2; d++) {
            if (!next_token(&ts, s, sizeof(s))) {
                csu_set_error("mesh.su2: unexpected end of file in points");
                st = CSU_ERR_INPUT;
                goto fail;
            }
            m->xy[2 * p + d] = strtod(s, NULL);
        }
        next_token(&ts, s, sizeof(s)); /* point index */
    }
    for (int i = 0; i < nc; i++)
        for (int j = 0; j < m->cell_npts[i]; j++) {
            int p = m->cell_nodes[4 * i + j];
            if (p < 0 || p >= m->n_points) {
                csu_set_error("mesh.su2: element %d references point %d of %d", i, p, m->n_points);
                st = CSU_ERR_INPUT;
                goto fail;
            }
        }
    next_token(&ts, s, sizeof(s));
    if (strcmp(s, "NMARK=") != 0) {
        csu_set_error("mesh.su2: expected NMARK=, got '%s'", s);
        st = CSU_ERR_INPUT;
        goto fail;
    }
    if ((st = parse_int_token(&ts, "NMARK", &m->n_markers))) goto fail;
    if (m->n_markers < 0) {
        st = CSU_ERR_INPUT;
        csu_set_error("mesh.su2: negative NMARK");
        goto fail;
    }
    int nm = m->n_markers;
    m->marker_nbf = calloc(nm + 1, sizeof(int));
    m->marker_flag = calloc(nm + 1, sizeof(int));
    m->marker_name = calloc(nm + 1, sizeof(*m->marker_name));
    /* boundary elements are stored marker-major; grow as markers are read */
    size_t cap = 1024, nb = 0;
    m->bface = malloc(sizeof(int) * 3 * cap);
    for (int k = 0; k < nm; k++) {
        next_token(&ts, s, sizeof(s)); /* MARKER_TAG= */
        next_token(&ts, s, sizeof(s));
        snprintf(m->marker_name[k], CSU_KW_LEN, "%s", s);
        next_token(&ts, s, sizeof(s));
        if (strcmp(s, "MARKER_ELEMS=") != 0) {
            csu_set_error("mesh.su2: marker %d: expected MARKER_ELEMS=, got '%s'", k, s);
            st = CSU_ERR_INPUT;
            goto fail;
        }
        int ne;
        if ((st = parse_int_token(&ts, "MARKER_ELEMS", &ne))) goto fail;
        if (ne < 0) {
            csu_set_error("mesh.su2: marker %d has negative size", k);
            st = CSU_ERR_INPUT;
            goto fail;
        }
        m->marker_nbf[k] = ne;
        for (int j = 0; j < ne; j++) {
            int q0, q1;
            next_token(&ts, s, sizeof(s)); /* line type (3) */
            if ((st = parse_int_token(&ts, "boundary node", &q0))) goto fail;
            if ((st = parse_int_token(&ts, "boundary node", &q1))) goto fail;
            next_token(&ts, s, sizeof(s)); /* the token ended by the line's trailing space */
            if (q0 < 0 || q0 >= m->n_points || q1 < 0 || q1 >= m->n_points) {
                csu_set_error("mesh.su2: marker %d element %d references a missing point", k, j);
                st = CSU_ERR_INPUT;
                goto fail;
            }
            if (nb == cap) {
                cap *= 2;
                m->bface = realloc(m->bface, sizeof(int) * 3 * cap);
            }
            m->bface[3 * nb] = q0;
            m->bface[3 * nb + 1] = q1;
            m->bface[3 * nb + 2] = -1;
            nb++;
        }
    }
    m->n_bfaces = (int)nb;

    /* orientation fix, mesh.c:222-242 */
    for (int i = 0; i < nc; i++) {
        if (csu_mesh_cell_omega(m, i, axi) < 0) {
            int np = m->cell_npts[i], tmp[4];
            for (int j = 0; j < np; j++) tmp[j] = m->cell_nodes[4 * i + np - 1 - j];
            for (int j = 0; j < np; j++) m->cell_nodes[4 * i + j] = tmp[j];
        }
    }
    if ((st = build_faces(m))) goto fail;
    if ((st = build_neighbours(m))) goto fail;
    /* boundary orientation, mesh.c:987-1009 */
    for (int b = 0; b < m->n_bfaces; b++) {
        int q0 = m->bface[3 * b], q1 = m->bface[3 * b + 1], own = m->bface[3 * b + 2];
        if (pori(m, own, q0, q1) < 0) {
            m->bface[3 * b] = q1;
            m->bface[3 * b + 1] = q0;
        }
    }
    /* signed face lists, mesh.c:1011-1037 */
    for (int f = 0; f < m->n_faces; f++) {
        int e0 = m->con[4 * f], e1 = m->con[4 * f + 1];
        m->cell_faces[4 * e0 + m->cell_nint[e0]++] = f + 1;
        m->cell_faces[4 * e1 + m->cell_nint[e1]++] = -(f + 1);
    }
    for (int i = 0; i < nc; i++) m->omega[i] = csu_mesh_cell_omega(m, i, axi);
    return CSU_OK;
fail:
    csu_mesh_free(m);
    return st;
}

/* saCalcD (sa.c:703-793): brute-force distance from the cell centroid to every wall edge (flags 3, 4).
 * Kept O(Ncell * Nwall) so the minimum is taken over the same candidates in the same order. */
/* saCalcD (sa.c:703-793): each cell's distance d = min over the wall faces (flags 3, 4) of the reference's
 * point-to-segment expression from the cell's vertex-average centre, starting from 1e6. A minimum does not
 * depend on the order of its terms, so any search that evaluates that same expression on a set of faces
 * containing the nearest ones gives the reference's d bit for bit. The faces go into a uniform grid of
 * buckets over their bounding box (each face into every bucket its own bounding box touches); a cell looks
 * at the buckets ring by ring around the bucket nearest to it and stops once no face beyond the current ring
 * can be closer: every bucket of ring k (k >= 1) lies at least (k - 1) bucket widths from the cell, which
 * must exceed the best distance found, with a relative margin far above rounding. Cost: about the number of
 * faces in a few buckets per cell instead of all of them (O(N_cells * N_wall) in the reference). */
typedef struct {
    double p0x, p0y, p1x, p1y;
} wall_seg;

static double seg_distance(const wall_seg* w, double xv, double yv)
{
    double num = (w->p1x - w->p0x) * (xv - w->p0x) + (w->p1y - w->p0y) * (yv - w->p0y);
    double den = (w->p1x - w->p0x) * (w->p1x - w->p0x) + (w->p1y - w->p0y) * (w->p1y - w->p0y);
    double t = num / den;
    if (t > 1.) t = 1.;
    else if (t < 0.) t = 0.;
    double dx = (w->p1x - w->p0x) * t + w->p0x - xv;
    double dy = (w->p1y - w->p0y) * t + w->p0y - yv;
    return sqrt(dx * dx + dy * dy);
}

void csu_mesh_wall_distance(csu_mesh* m)
{
    if (!m->wall_dist) m->wall_dist = malloc(sizeof(double) * m->n_cells);
    for (int i = 0; i < m->n_cells; i++) m->wall_dist[i] = 1e6;
    int nw = 0, base = 0;
    for (int k = 0; k < m->n_markers; k++)
        if (m->marker_flag[k] == CSU_BC_WALL || m->marker_flag[k] == CSU_BC_WALLT) nw += m->marker_nbf[k];
    if (nw == 0) return;
    wall_seg* w = malloc(sizeof(wall_seg) * nw);
    double xlo = 1e300, xhi = -1e300, ylo = 1e300, yhi = -1e300;
    nw = 0;
    for (int k = 0; k < m->n_markers; k++) {
        int nb = m->marker_nbf[k];
        if (m->marker_flag[k] == CSU_BC_WALL || m->marker_flag[k] == CSU_BC_WALLT) {
            for (int j = 0; j < nb; j++) {
                const int* bf = m->bface + 3 * (base + j);
                wall_seg* g = &w[nw++];
                g->p0x = m->xy[2 * bf[0]];
                g->p0y = m->xy[2 * bf[0] + 1];
                g->p1x = m->xy[2 * bf[1]];
                g->p1y = m->xy[2 * bf[1] + 1];
                xlo = fmin(xlo, fmin(g->p0x, g->p1x));
                xhi = fmax(xhi, fmax(g->p0x, g->p1x));
                ylo = fmin(ylo, fmin(g->p0y, g->p1y));
                yhi = fmax(yhi, fmax(g->p0y, g->p1y));
            }
        }
        base += nb;
    }
    /* about two faces per bucket, buckets as square as the box allows */
    double wx = xhi - xlo, wy = yhi - ylo;
    double span = fmax(fmax(wx, wy), 1e-300);
    double h = fmax(sqrt(wx * wy / (0.5 * nw)), span / (2.0 * nw));
    if (!(h > 0) || !isfinite(h)) h = span;
    int gx = (int)fmin(fmax(ceil(wx / h), 1.0), 4096.0), gy = (int)fmin(fmax(ceil(wy / h), 1.0), 4096.0);
    double hx = fmax(wx / gx, 1e-300), hy = fmax(wy / gy, 1e-300);
    /* bucket lists: counts, prefix sums, fill */
    int nbk = gx * gy;
    int* cnt = calloc(nbk + 1, sizeof(int));
    for (int pass = 0; pass < 2; pass++) {
        int* fillp = NULL;
        int* items = NULL;
        if (pass == 1) {
            for (int b = 0; b < nbk; b++) cnt[b + 1] += cnt[b];
            fillp = malloc(sizeof(int) * nbk);
            memcpy(fillp, cnt, sizeof(int) * nbk);
            items = malloc(sizeof(int) * (cnt[nbk] > 0 ? cnt[nbk] : 1));
        }
        for (int s2 = 0; s2 < nw; s2++) {
            const wall_seg* g = &w[s2];
            int i0 = (int)floor((fmin(g->p0x, g->p1x) - xlo) / hx), i1 = (int)floor((fmax(g->p0x, g->p1x) - xlo) / hx);
            int j0 = (int)floor((fmin(g->p0y, g->p1y) - ylo) / hy), j1 = (int)floor((fmax(g->p0y, g->p1y) - ylo) / hy);
            i0 = i0 < 0 ? 0 : (i0 >= gx ? gx - 1 : i0);
            i1 = i1 < 0 ? 0 : (i1 >= gx ? gx - 1 : i1);
            j0 = j0 < 0 ? 0 : (j0 >= gy ? gy - 1 : j0);
            j1 = j1 < 0 ? 0 : (j1 >= gy ? gy - 1 : j1);
            for (int j = j0; j <= j1; j++)
                for (int i = i0; i <= i1; i++) {
                    if (pass == 0) cnt[j * gx + i + 1]++;
                    else items[fillp[j * gx + i]++] = s2;
                }
        }
        if (pass == 1) {
            free(fillp);
            /* search */
            int last = -1; /* the previous cell's nearest face: a first candidate for the next cell */
            for (int c = 0; c < m->n_cells; c++) {
                double xv, yv;
                csu_mesh_center(m, c, &xv, &yv);
                int ic = (int)floor((xv - xlo) / hx), jc = (int)floor((yv - ylo) / hy);
                ic = ic < 0 ? 0 : (ic >= gx ? gx - 1 : ic);
                jc = jc < 0 ? 0 : (jc >= gy ? gy - 1 : jc);
                /* the point's distance to the grid's x and y ranges (0 inside) */
                const double dxg = xv < xlo ? xlo - xv : (xv > xhi ? xv - xhi : 0.0);
                const double dyg = yv < ylo ? ylo - yv : (yv > yhi ? yv - yhi : 0.0);
                double best = m->wall_dist[c];
                int arg = -1;
                if (last >= 0) {
                    double d = seg_distance(&w[last], xv, yv);
                    if (best > d) {
                        best = d;
                        arg = last;
                    }
                }
                const int kmax = gx > gy ? gx : gy;
                for (int k = 0; k <= kmax; k++) {
                    const double lim = best * (1.0 + 1e-9) + 1e-300;
                    if (k >= 1) {
                        /* every bucket of ring k or beyond is k - 1 columns beyond the point's column (x
                         * distance >= (k-1) hx + dxg, y distance >= dyg) or k - 1 rows beyond its row */
                        double lb = 1e300;
                        if (ic - k >= 0 || ic + k < gx) {
                            double a = (k - 1) * hx + dxg;
                            lb = fmin(lb, sqrt(a * a + dyg * dyg));
                        }
                        if (jc - k >= 0 || jc + k < gy) {
                            double b = (k - 1) * hy + dyg;
                            lb = fmin(lb, sqrt(dxg * dxg + b * b));
                        }
                        if (lb > lim) break;
                    }
                    for (int j = jc - k; j <= jc + k; j++) {
                        if (j < 0 || j >= gy) continue;
                        const double by0 = ylo + j * hy;
                        const double ddy = yv < by0 ? by0 - yv : (yv > by0 + hy ? yv - by0 - hy : 0.0);
                        if (ddy > lim) continue;
                        int step = (j == jc - k || j == jc + k) ? 1 : 2 * k;
                        for (int i = ic - k; i <= ic + k; i += (step > 0 ? step : 1)) {
                            if (i < 0 || i >= gx) continue;
                            const int b = j * gx + i;
                            if (cnt[b] == cnt[b + 1]) continue;
                            const double bx0 = xlo + i * hx;
                            const double ddx = xv < bx0 ? bx0 - xv : (xv > bx0 + hx ? xv - bx0 - hx : 0.0);
                            if (ddx * ddx + ddy * ddy > lim * lim) continue;
                            for (int q = cnt[b]; q < cnt[b + 1]; q++) {
                                double d = seg_distance(&w[items[q]], xv, yv);
                                if (best > d) {
                                    best = d;
                                    arg = items[q];
                                }
                            }
                        }
                    }
                }
                if (arg >= 0) last = arg;
                m->wall_dist[c] = best;
            }
            free(items);
        }
    }
    free(cnt);
    free(w);
}
