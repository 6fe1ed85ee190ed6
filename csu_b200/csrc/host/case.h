/* case.h -- host-side case representation (internal to libcsu_b200). */
#ifndef CSU_CASE_H
#define CSU_CASE_H

#include <stddef.h>
#include "csu_gpu.h"

#define CSU_KW_MAX 100 /* entries in input.dat (input.c:17)        */
#define CSU_KW_LEN 50  /* name/value buffer length (solver.c:1740) */

typedef struct csu_keywords {
    int n;
    char name[CSU_KW_MAX][CSU_KW_LEN];
    char value[CSU_KW_MAX][CSU_KW_LEN];
} csu_keywords;

typedef struct csu_mesh {
    int ndim, n_points, n_cells, n_faces, n_markers, n_bfaces;
    double* xy;       /* 2 per point                                   */
    int* cell_npts;   /* per cell                                      */
    int* cell_nodes;  /* 4 per cell (-1 padded)                        */
    int* con;         /* 4 per interior face: e0 e1 p0 p1              */
    int* cell_nint;   /* interior faces per cell                       */
    int* cell_faces;  /* 4 per cell, signed                            */
    int* cell_nei;    /* 4 per cell, >=0 cell, <0 -(1+bface)           */
    int* marker_nbf;
    int* marker_flag;
    char (*marker_name)[CSU_KW_LEN];
    int* bface;       /* 3 per boundary face: p0 p1 owner              */
    double* omega;    /* per cell (meshUpdateOmega)                    */
    double* wall_dist;/* per cell or NULL                              */
} csu_mesh;

struct csu_case {
    csu_keywords kw;
    csu_mesh mesh;
    csu_config cfg;
    double* U0;       /* initial state [var][cell]                     */
};

/* thread-local error message shared by the whole library */
void csu_set_error(const char* fmt, ...);

/* input.c */
int csu_keywords_parse(const char* text, size_t len, csu_keywords* kw);
int csu_keywords_has(const csu_keywords* kw, const char* name);
const char* csu_keywords_get(const csu_keywords* kw, const char* name); /* NULL if missing */

/* su2.c */
int csu_mesh_read_su2(const char* text, size_t len, int axi, csu_mesh* m);
void csu_mesh_free(csu_mesh* m);
double csu_mesh_cell_omega(const csu_mesh* m, int cell, int axi);
void csu_mesh_center(const csu_mesh* m, int cell, double* x, double* y);
void csu_mesh_wall_distance(csu_mesh* m);

/* gas helpers shared by the host setup (gasprop.c) */
double csu_host_T2e(const csu_config* c, double T);
double csu_host_T2c(const csu_config* c, double T);
double csu_host_sutherland(double T);

#endif
