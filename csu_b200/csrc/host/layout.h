/* layout.h -- device data layout built on the host from a csu_mesh_desc (internal). */
#ifndef CSU_LAYOUT_H
#define CSU_LAYOUT_H

#include "csu_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/*
 * Cells are renumbered along a Hilbert curve through their centroids; interior faces are sorted by their
 * lower renumbered cell, boundary faces by owner. All per-cell slot arrays are [slot][cell] (4 slots).
 * Geometry is computed with the reference's expressions so it is bit-identical to what the reference
 * recomputes on the fly (elementCenter, meshCalcDS, edge midpoints).
 */
typedef struct csu_layout {
    int nc, nf, nb, nv;
    int* cell_new2old;
    int* cell_old2new;
    int* face_new2old;
    int* face_old2new;
    int* bface_new2old;
    int* bface_old2new;

    /* per renumbered cell */
    int* npts;     /* nodes = edges = neighbour slots                                                 */
    int* nint;     /* interior faces                                                                  */
    int* nslot;    /* face slots = interior + boundary faces of the cell                              */
    int* nei;      /* [4][nc] neighbour (ELEMENT.neiL order): cell id, or nc + boundary face id       */
    double* wx;    /* [4][nc] least-squares weights: dUx = sum wx (u_nei - u_cell)                     */
    double* wy;
    double* ldx;   /* [4][nc] neighbour centre minus centroid, x and y (solverCalcGrad3 x[jj] - x[0])   */
    double* ldy;
    unsigned long long* lm;  /* [4][nc] x87 significands of a, b, c, a*c - b*b (long double, solver.c:1058-1073) */
    int* les;      /* [4][nc] exponent << 1 | sign of the same                                          */
    unsigned long long* lrv; /* [nc] invariant-divisor reciprocal of the determinant's significand       */
    double* lq;    /* [4][nc][2] a, b, c, 1/(a*c - b*b) as (high, low) double pairs                          */
    double* ex;    /* [4][nc] edge midpoint minus centroid, edges in node order (limiter, inter)        */
    double* ey;
    int* fslot;    /* [4][nc] +-(flux index + 1): interior faces (ELEMENT.f order) then boundary faces  */
    int* fnb;      /* [4][nc] the neighbour cell across interior face slot j (j < nint), else -1          */
    double* omega;
    double* sxh;   /* 0.5 * sum |dSx| over the cell edges (solverLocalTimeStep, solver.c:904-914)      */
    double* syh;
    double* xc;    /* centroid (elementCenter)                                                        */
    double* yc;
    double* wall_d;/* wall distance or NULL                                                           */
    double* dslat; /* meshCalcDSlateral (axisymmetric pressure source)                                */

    /* per renumbered interior face (orientation of mesh->con) */
    int* fe0;
    int* fe1;
    double* fdsx;  /* meshCalcDS (axisymmetric scaling included)                                      */
    double* fdsy;
    double* fds;   /* sqrt(dSx^2 + dSy^2)                                                             */
    double* r0x;   /* face midpoint minus centroid of e0 / e1                                         */
    double* r0y;
    double* r1x;
    double* r1y;
    double* fdist; /* centroid distance |x_e1 - x_e0| (viscous terms)                                 */
    double* fdx;   /* x_e1 - x_e0, y_e1 - y_e0 (laminar.c:44-45)                                        */
    double* fdy;

    /* per renumbered boundary face */
    int* bown;
    int* bflag;
    int* bold;     /* reference (marker-major) id                                                     */
    double* bdsx;
    double* bdsy;
    double* bds;
    double* bmx;   /* edge midpoint (ghost centre)                                                    */
    double* bmy;
    double* bdx;   /* edge midpoint minus owner centroid, and its length (laminar.c:184-191)            */
    double* bdy;
    double* bL;
    double* bunx;  /* meshCalcDS2 unit normal and length (mesh.c:742-764)                               */
    double* buny;
    double* bds2;

    int* color;    /* greedy colouring of the cell graph (no two face neighbours share a colour)         */
    int ncolors;
    int* color_start;/* [ncolors + 1] ranges into color_cells                                         */
    int* color_cells;/* cells grouped by colour, ascending within a colour                            */

    double vol_max;/* max omega (limiterUpdate type 0, limiter.c:44-48)                               */
    int max_npts;
} csu_layout;

int csu_layout_build(const csu_mesh_desc* m, int axi, csu_layout* L);
void csu_layout_free(csu_layout* L);
int csu_layout_green_gauss(csu_layout* L);
/* LU-SGS colouring with one cell per colour in the reference's cell order: the multicolour sweeps then
   visit cells exactly as implicitLUSGS_L / _U do (implicit.c:274-482), one launch per cell (for checks) */
int csu_layout_sequential_colors(csu_layout* L);

#ifdef __cplusplus
}
#endif
#endif
