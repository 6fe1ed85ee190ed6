/*
 * csu_oracle.h -- TEST INFRASTRUCTURE. A plain-C restatement of CSU's residual-and-update path, used only
 * by tests/, bench.py's CPU arm and smoke() as the checker of the CUDA engine. Never linked into the
 * product. Arrays are in the reference's numbering and layouts ([var][cell] for U, R, gradients).
 */
#ifndef CSU_ORACLE_H
#define CSU_ORACLE_H

#include "../include/csu_gpu.h"

typedef struct orc orc;

orc* orc_create(const csu_mesh_desc* m, const csu_config* c);
void orc_free(orc* o);
void orc_set_U(orc* o, const double* U);
void orc_get_U(orc* o, double* U);
void orc_residual(orc* o);
/* what: 1 P, 2 ghost P, 3 grad, 4 phi, 5 faceflux, 6 R, 7 D, 8 dtL, 9 dW, 10 blocks (csu_gpu.h CSU_DUMP_*) */
void orc_get(orc* o, int what, double* out);
void orc_iterate(orc* o, int n, int it0, double* hist);
int orc_tube(orc* o, double tmax, double* t_out);

#endif
