/*
 * case.c -- a CSU case folder as the host side of the engine sees it.
 *
 * Follows solverInit (solver.c:1728-1834): keywords (input.c), model flags and Nvar (1748-1798),
 * mesh (mesh.c via su2.c), solverSetData keywords and defaults (1403-1658), wall distance for SA/SST
 * (1809-1814), and solverInitDomain (1660-1726): freestream state from conditionState (40-89), the
 * two-state shock tube (952-975) or restart.csv (358-373). The reference prints and calls exit(0) on a
 * missing keyword or a bad choice; here those return CSU_ERR_INPUT with a message.
 */
#include <stdio.h>
#include <stdlib.h>
#include <stdarg.h>
#include <string.h>
#include <math.h>
#include "case.h"

static __thread char g_err[512];

void csu_set_error(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

const char* csu_last_error(void)
{
    return g_err;
}

const char* csu_strerror(int st)
{
    switch (st) {
    case CSU_OK: return "ok";
    case CSU_ERR_INPUT: return "invalid input";
    case CSU_ERR_IO: return "i/o error";
    case CSU_ERR_OOM: return "out of memory or over budget";
    case CSU_ERR_NONFINITE: return "non-finite state";
    case CSU_ERR_DIVERGED: return "diverged";
    case CSU_ERR_CANCELLED: return "cancelled";
    case CSU_ERR_CUDA: return "cuda error";
    case CSU_ERR_UNSUPPORTED: return "unsupported setting";
    case CSU_ERR_STATE: return "invalid call order";
    case CSU_ERR_NO_DEVICE: return "no cuda device";
    default: return "unknown status";
    }
}

/* ---------------------------------------------------------------- gas (gasprop.c:14-154) */
static const double TP_CC[6] = {1.81716e3, 9.890504e2 - 287.0530, -9.595592e-3, 1.041469e-4, -4.433065e-8,
                                5.879263e-12};

static double cv_const(const csu_config* c)
{
    double cp = c->gamma * c->gas_r / (c->gamma - 1);
    return cp - c->gas_r;
}

double csu_host_T2e(const csu_config* c, double T)
{
    if (c->tp) {
        double P = 1, aux = TP_CC[0];
        for (int i = 1; i < 6; i++) {
            P *= T;
            aux += TP_CC[i] * P;
        }
        return aux;
    }
    return cv_const(c) * T;
}

static double host_T2Cv(const csu_config* c, double T)
{
    if (c->tp) {
        double P = 1, aux = TP_CC[1];
        for (int i = 2; i < 6; i++) {
            P *= T;
            aux += i * TP_CC[i] * P;
        }
        return aux;
    }
    return cv_const(c);
}

double csu_host_T2c(const csu_config* c, double T)
{
    double Cv = host_T2Cv(c, T);
    double gam = (Cv + c->gas_r) / Cv;
    return sqrt(gam * c->gas_r * T);
}

double csu_host_sutherland(double T)
{
    return 1.458e-6 * T * sqrt(T) / (T + 110.4);
}

/* ---------------------------------------------------------------- keyword helpers */
static int kw_required(const csu_keywords* kw, const char* name, const char** out)
{
    *out = csu_keywords_get(kw, name);
    if (!*out) {
        csu_set_error("Error: Value not found in the input file: %s.", name);
        return CSU_ERR_INPUT;
    }
    return CSU_OK;
}

static int kw_int(const csu_keywords* kw, const char* name, int def)
{
    const char* v = csu_keywords_get(kw, name);
    return v ? atoi(v) : def;
}

static double kw_dbl(const csu_keywords* kw, const char* name, double def)
{
    const char* v = csu_keywords_get(kw, name);
    return v ? strtod(v, NULL) : def;
}

static int flux_choice(const char* s, int* out)
{
    static const char* names[] = {"ROE", "AUSM", "AUSMDV", "AUSMpup", "AUSMpup2"};
    for (int i = 0; i < 5; i++)
        if (strcmp(s, names[i]) == 0) {
            *out = i;
            return CSU_OK;
        }
    csu_set_error("Error in flux choice: %s.", s);
    return CSU_ERR_INPUT;
}

static int bc_choice(const char* s, int* out)
{
    static const char* names[] = {"symmetry", "inlet", "outlet", "wall", "wallT"};
    for (int i = 0; i < 5; i++)
        if (strcmp(s, names[i]) == 0) {
            *out = i;
            return CSU_OK;
        }
    csu_set_error("Error: incorrent input of bc: %s", s);
    return CSU_ERR_INPUT;
}

static int ts_choice(const char* s, int* out)
{
    static const char* names[] = {"RK", "LUSGS", "DPLUR"};
    for (int i = 0; i < 3; i++)
        if (strcmp(s, names[i]) == 0) {
            *out = i;
            return CSU_OK;
        }
    csu_set_error("Error in time scheme choice: %s.", s);
    return CSU_ERR_INPUT;
}

/* conditionState (solver.c:40-89) */
static void condition_state(const csu_config* c, double p, double T, double mach, double nx, double ny,
                            double* Uin, double* Pin)
{
    double r, u, v, E, cc, k = 0.0;
    r = p / (c->gas_r * T);
    cc = csu_host_T2c(c, T);
    u = nx * mach * cc;
    v = ny * mach * cc;
    for (int i = 0; i < 6; i++) Uin[i] = 0.0;
    for (int i = 0; i < 7; i++) Pin[i] = 0.0;
    if (c->sst == 1) {
        double L = c->sst_l;
        double U = cc * mach;
        double ReL = (r * U * L) / csu_host_sutherland(T);
        k = c->k_factor * U * U / ReL;
        double om = c->o_factor * U / L;
        Uin[4] = r * k;
        Uin[5] = r * om;
        Pin[5] = k;
        Pin[6] = om;
    }
    E = csu_host_T2e(c, T) + (u * u + v * v) / 2 + k;
    Uin[0] = r;
    Uin[1] = r * u;
    Uin[2] = r * v;
    Uin[3] = r * E;
    Pin[0] = r;
    Pin[1] = u;
    Pin[2] = v;
    Pin[3] = c->gas_r * T * r;
    Pin[4] = T;
    if (c->sa == 1) {
        double n = c->turb_ratio * csu_host_sutherland(T) / r;
        Uin[4] = r * n;
        Pin[5] = n;
    }
}

/* fReadTables/tableRead (readTables.c:5-124): tokens end at ',' or '\n' */
static int restart_token(const char* s, size_t len, size_t* pos, char* out, int cap)
{
    int n = 0;
    if (*pos >= len) {
        out[0] = '\0';
        return 0;
    }
    while (*pos < len) {
        char c = s[(*pos)++];
        if (c == ',' || c == '\n') break;
        if (n < cap - 1) out[n++] = c;
    }
    out[n] = '\0';
    return 1;
}

static int load_restart(csu_case* cs, const char* text, size_t len)
{
    size_t pos = 0;
    char s[128];
    int nc = cs->mesh.n_cells, nv = cs->cfg.nvar;
    restart_token(text, len, &pos, s, sizeof(s)); /* number of tables */
    if (atoi(s) < 1) {
        csu_set_error("restart.csv: no table");
        return CSU_ERR_INPUT;
    }
    restart_token(text, len, &pos, s, sizeof(s));
    restart_token(text, len, &pos, s, sizeof(s)); /* table number */
    restart_token(text, len, &pos, s, sizeof(s));
    int nrow = atoi(s);
    restart_token(text, len, &pos, s, sizeof(s));
    int ncol = atoi(s);
    restart_token(text, len, &pos, s, sizeof(s));
    if (nrow < nc || ncol < nv) {
        csu_set_error("restart.csv: table is %d x %d, need %d x %d", nrow, ncol, nc, nv);
        return CSU_ERR_INPUT;
    }
    for (int i = 0; i < nc; i++) {
        for (int j = 0; j < ncol; j++) {
            if (!restart_token(text, len, &pos, s, sizeof(s))) {
                csu_set_error("restart.csv: truncated at row %d", i);
                return CSU_ERR_INPUT;
            }
            if (j < nv) cs->U0[(size_t)j * nc + i] = strtod(s, NULL);
        }
        restart_token(text, len, &pos, s, sizeof(s));
    }
    return CSU_OK;
}

static int read_file(const char* path, char** out, size_t* len)
{
    FILE* f = fopen(path, "rb");
    if (!f) {
        csu_set_error("cannot open %s", path);
        return CSU_ERR_IO;
    }
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    char* buf = malloc((size_t)n + 1);
    if (!buf) {
        fclose(f);
        csu_set_error("out of host memory reading %s", path);
        return CSU_ERR_OOM;
    }
    size_t got = fread(buf, 1, (size_t)n, f);
    fclose(f);
    buf[got] = '\0';
    *out = buf;
    *len = got;
    return CSU_OK;
}

static int setup(csu_case* cs, const char* mesh_text, size_t mesh_len, const char* restart_text,
                 size_t restart_len)
{
    const csu_keywords* kw = &cs->kw;
    csu_config* c = &cs->cfg;
    const char* v;
    int st;
    memset(c, 0, sizeof(*c));

    if ((st = kw_required(kw, "threads", &v))) return st; /* solver.c:1745 */
    c->sa = kw_int(kw, "sa", 0);
    c->sa_cc = kw_int(kw, "saCC", 0);
    c->sst = kw_int(kw, "sst", 0);
    c->sst_trans = c->sst ? kw_int(kw, "sstTrans", 0) : 0;
    c->nvar = 4;
    if (c->sa == 1) c->nvar = 5;
    if (c->sst == 1) c->nvar = 6;
    if ((st = kw_required(kw, "axisymmetric", &v))) return st;
    c->axisymmetric = atoi(v);

    if ((st = csu_mesh_read_su2(mesh_text, mesh_len, c->axisymmetric, &cs->mesh))) return st;

    /* solverSetData, solver.c:1403-1658 */
    if ((st = kw_required(kw, "order", &v))) return st;
    c->order = atoi(v);
    for (int k = 0; k < cs->mesh.n_markers; k++) {
        char key[2 * CSU_KW_LEN];
        snprintf(key, sizeof(key), "BC:%s", cs->mesh.marker_name[k]);
        if ((st = kw_required(kw, key, &v))) return st;
        if ((st = bc_choice(v, &cs->mesh.marker_flag[k]))) return st;
    }
    c->tp = kw_int(kw, "TP", 0);
    c->gamma = 1.4;
    c->gas_r = 287.0530;
    c->pr = 0.72;
    c->pr_t = 0.9;
    c->e_fix = 0.1;
    c->laminar = kw_int(kw, "laminar", 0);
    c->sref = kw_dbl(kw, "Sref", 1.0);
    c->turb_ratio = kw_dbl(kw, "turbRatio", 10.0);
    c->dt_local = kw_int(kw, "dtLocal", 0);
    c->dt_local_n = kw_int(kw, "dtLocalN", -1);
    c->w_imp = kw_dbl(kw, "wImp", 1.0);
    c->turb1order = kw_int(kw, "turb1order", 0);
    c->time_scheme = 0;
    if ((v = csu_keywords_get(kw, "timeScheme")) && (st = ts_choice(v, &c->time_scheme))) return st;
    c->n_linear = kw_int(kw, "Nlinear", 20);
    c->r_lim = kw_dbl(kw, "rLim", 1e-6);
    if ((st = kw_required(kw, "flux", &v))) return st;
    if ((st = flux_choice(v, &c->flux))) return st;
    if ((st = kw_required(kw, "stages", &v))) return st;
    c->stages = atoi(v);
    if ((st = kw_required(kw, "CFL", &v))) return st;
    c->cfl = strtod(v, NULL);
    c->p_out = kw_dbl(kw, "pout", 1.0e5);
    c->visc_blazek = kw_int(kw, "viscBlazek", 0);
    c->t_wall = kw_dbl(kw, "Twall", 300);
    c->limiter_type = kw_int(kw, "limiter", 0);
    c->limiter_k = kw_dbl(kw, "limK", 1.0);
    if (c->sst) {
        c->k_factor = kw_dbl(kw, "kFactor", 1.125);
        c->o_factor = kw_dbl(kw, "oFactor", 125.0);
        c->o_wall_factor = kw_dbl(kw, "oWallFactor", 10);
        c->sst_l = kw_dbl(kw, "Lsst", 1.0);
    }
    int restart = kw_int(kw, "restart", 0);
    /* extensions */
    c->implicit_fp32 = kw_int(kw, "implicitFP32", 0);
    c->implicit_local_dt = kw_int(kw, "implicitLocalDt", 0);
    c->cfl_ramp_iters = kw_int(kw, "CFLramp", 0);
    c->cfl_max = kw_dbl(kw, "CFLmax", c->cfl);
    c->conv_drop = kw_dbl(kw, "convDrop", 0.0);
    c->iter_cap = kw_int(kw, "iterCap", 0);
    c->limiter_func = kw_int(kw, "limiterFunc", 0);
    c->gradient = kw_int(kw, "gradient", 0);
    c->sa_implicit_source = kw_int(kw, "saImplicitSource", 0);

    if (c->sa == 1 || c->sst == 1) csu_mesh_wall_distance(&cs->mesh);

    /* solverInitDomain, solver.c:1660-1726 */
    int nc = cs->mesh.n_cells, nv = c->nvar;
    cs->U0 = calloc((size_t)nv * nc, sizeof(double));
    if (!cs->U0) {
        csu_set_error("out of host memory for the state");
        return CSU_ERR_OOM;
    }
    if ((st = kw_required(kw, "tube", &v))) return st;
    c->tube = atoi(v);
    if (c->tube == 0) {
        const char *sp, *sT, *sm, *snx, *sny;
        if ((st = kw_required(kw, "pressure", &sp)) || (st = kw_required(kw, "temperature", &sT)) ||
            (st = kw_required(kw, "mach", &sm)) || (st = kw_required(kw, "nx", &snx)) ||
            (st = kw_required(kw, "ny", &sny)))
            return st;
        c->inlet_p = strtod(sp, NULL);
        c->inlet_t = strtod(sT, NULL);
        c->mach_inf = strtod(sm, NULL);
        condition_state(c, c->inlet_p, c->inlet_t, c->mach_inf, strtod(snx, NULL), strtod(sny, NULL), c->uin,
                        c->pin);
        if (restart) {
            if (!restart_text) {
                csu_set_error("restart requested but no restart.csv");
                return CSU_ERR_IO;
            }
            if ((st = load_restart(cs, restart_text, restart_len))) return st;
        } else {
            for (int k = 0; k < 4; k++)
                for (int i = 0; i < nc; i++) cs->U0[(size_t)k * nc + i] = c->uin[k];
            if (c->sa == 1)
                for (int i = 0; i < nc; i++) cs->U0[(size_t)4 * nc + i] = c->uin[4];
            else if (c->sst == 1)
                for (int i = 0; i < nc; i++) {
                    cs->U0[(size_t)4 * nc + i] = c->uin[4];
                    cs->U0[(size_t)5 * nc + i] = c->uin[5];
                }
        }
    } else {
        if (restart) {
            if (!restart_text) {
                csu_set_error("restart requested but no restart.csv");
                return CSU_ERR_IO;
            }
            if ((st = load_restart(cs, restart_text, restart_len))) return st;
            /* the reference leaves solver->inlet unset here (solver.c:1700-1706) */
        } else {
            const char* names[2][5] = {{"pressure1", "temperature1", "mach1", "nx1", "ny1"},
                                       {"pressure2", "temperature2", "mach2", "nx2", "ny2"}};
            double val[2][5], Uin[2][6], Pin[2][7];
            for (int s = 0; s < 2; s++)
                for (int q = 0; q < 5; q++) {
                    if ((st = kw_required(kw, names[s][q], &v))) return st;
                    val[s][q] = strtod(v, NULL);
                }
            const char* sxm;
            if ((st = kw_required(kw, "xm", &sxm))) return st;
            double xm = strtod(sxm, NULL);
            for (int s = 0; s < 2; s++)
                condition_state(c, val[s][0], val[s][1], val[s][2], val[s][3], val[s][4], Uin[s], Pin[s]);
            for (int k = 0; k < 4; k++)
                for (int i = 0; i < nc; i++) {
                    double x, y;
                    csu_mesh_center(&cs->mesh, i, &x, &y);
                    cs->U0[(size_t)k * nc + i] = x < xm ? Uin[0][k] : Uin[1][k];
                }
            memcpy(c->uin, Uin[0], sizeof(c->uin));
            memcpy(c->pin, Pin[0], sizeof(c->pin));
            c->inlet_p = val[0][0];
            c->inlet_t = val[0][1];
            c->mach_inf = val[0][2];
        }
    }
    return CSU_OK;
}

static int case_new(csu_case** out)
{
    *out = calloc(1, sizeof(csu_case));
    if (!*out) {
        csu_set_error("out of host memory");
        return CSU_ERR_OOM;
    }
    return CSU_OK;
}

int csu_case_load_mem(const char* input_dat, const char* mesh_su2, const char* restart_csv, csu_case** out)
{
    int st;
    *out = NULL;
    if (!input_dat || !mesh_su2) {
        csu_set_error("csu_case_load_mem: input_dat and mesh_su2 are required");
        return CSU_ERR_INPUT;
    }
    csu_case* cs;
    if ((st = case_new(&cs))) return st;
    if ((st = csu_keywords_parse(input_dat, strlen(input_dat), &cs->kw)) ||
        (st = setup(cs, mesh_su2, strlen(mesh_su2), restart_csv, restart_csv ? strlen(restart_csv) : 0))) {
        csu_case_free(cs);
        return st;
    }
    *out = cs;
    return CSU_OK;
}

int csu_case_load(const char* wd, csu_case** out)
{
    char path[4096];
    char *inp = NULL, *msh = NULL, *rst = NULL;
    size_t li, lm, lr = 0;
    int st;
    *out = NULL;
    snprintf(path, sizeof(path), "%sinput.dat", wd);
    if ((st = read_file(path, &inp, &li))) return st;
    snprintf(path, sizeof(path), "%smesh.su2", wd);
    if ((st = read_file(path, &msh, &lm))) {
        free(inp);
        return st;
    }
    snprintf(path, sizeof(path), "%srestart.csv", wd);
    if (read_file(path, &rst, &lr) != CSU_OK) rst = NULL;
    csu_case* cs;
    if ((st = case_new(&cs))) goto done;
    if ((st = csu_keywords_parse(inp, li, &cs->kw)) || (st = setup(cs, msh, lm, rst, lr))) {
        csu_case_free(cs);
        goto done;
    }
    *out = cs;
done:
    free(inp);
    free(msh);
    free(rst);
    return st;
}

int csu_case_mesh(const csu_case* cs, csu_mesh_desc* d)
{
    const csu_mesh* m = &cs->mesh;
    d->n_points = m->n_points;
    d->xy = m->xy;
    d->n_cells = m->n_cells;
    d->cell_npts = m->cell_npts;
    d->cell_nodes = m->cell_nodes;
    d->n_faces = m->n_faces;
    d->con = m->con;
    d->cell_nint = m->cell_nint;
    d->cell_faces = m->cell_faces;
    d->cell_nei = m->cell_nei;
    d->n_markers = m->n_markers;
    d->marker_nbf = m->marker_nbf;
    d->marker_flag = m->marker_flag;
    d->n_bfaces = m->n_bfaces;
    d->bface = m->bface;
    d->wall_dist = m->wall_dist;
    return CSU_OK;
}

int csu_case_config(const csu_case* cs, csu_config* out)
{
    *out = cs->cfg;
    return CSU_OK;
}

int csu_case_initial_state(const csu_case* cs, double* U)
{
    memcpy(U, cs->U0, sizeof(double) * (size_t)cs->cfg.nvar * cs->mesh.n_cells);
    return CSU_OK;
}

int csu_case_get_int(const csu_case* cs, const char* keyword, int* out)
{
    const char* v = csu_keywords_get(&cs->kw, keyword);
    if (!v) {
        csu_set_error("Error: Value not found in the input file: %s.", keyword);
        return CSU_ERR_INPUT;
    }
    *out = atoi(v);
    return CSU_OK;
}

int csu_case_get_double(const csu_case* cs, const char* keyword, double* out)
{
    const char* v = csu_keywords_get(&cs->kw, keyword);
    if (!v) {
        csu_set_error("Error: Value not found in the input file: %s.", keyword);
        return CSU_ERR_INPUT;
    }
    *out = strtod(v, NULL);
    return CSU_OK;
}

int csu_case_marker_name(const csu_case* cs, int marker, char* out, int cap)
{
    if (marker < 0 || marker >= cs->mesh.n_markers) return CSU_ERR_INPUT;
    snprintf(out, cap, "%s", cs->mesh.marker_name[marker]);
    return CSU_OK;
}

void csu_case_free(csu_case* cs)
{
    if (!cs) return;
    csu_mesh_free(&cs->mesh);
    free(cs->U0);
    free(cs);
}
