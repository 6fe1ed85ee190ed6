/*
 * csu_gpu.h -- C ABI of the B200 residual-and-update engine for CSU cases.
 *
 * The reference solver has no plugin API: its seam is the C function interface of solver.h:172-260 and
 * implicit.h, every function taking a SOLVER* that owns all host arrays. This header replaces the
 * per-iteration body of solverSolve (solver.c:1864-1907 and the tube loop 1921-1940) -- solverCalcR
 * (solver.c:685), solverCalcDt (925), solverStepRK (788), implicitCalcD/LUSGS_L/LUSGS_U/CalcDPLUR
 * (implicit.c:19,274,365,990), solverUpdateUImplicit (solver.c:1945), solverCalcRes (867) and
 * solverCalcCoeff3 (1342) -- with calls that take plain pointers and sizes.
 *
 * Conventions
 *  - Every entry returns an int status (CSU_OK == 0). The library never calls exit() and never aborts;
 *    csu_last_error() gives a one-line message for the calling thread's last failure.
 *  - Host arrays are caller-owned; device arrays are library-owned (allocated in csu_create, freed in
 *    csu_destroy). All host-side state arrays are in the reference's numbering (cell ii of
 *    mesh->elemL, face of mesh->con, boundary elements marker-major), whatever order the device uses.
 *  - Conserved state U and residual R are "[var][cell]" flat arrays: U[k*ncells + i] == solver->U[k][i].
 *  - One context per host thread; calls on one context are not re-entrant.
 */
#ifndef CSU_GPU_H
#define CSU_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference prints and exit(0)s instead: input.c:136-140, flux.c:38-42) ---- */
#define CSU_OK 0
#define CSU_ERR_INPUT 1       /* missing/invalid keyword, malformed SU2 file, bad argument          */
#define CSU_ERR_IO 2          /* file cannot be opened/written                                        */
#define CSU_ERR_OOM 3         /* device allocation failed or the request exceeds the memory budget   */
#define CSU_ERR_NONFINITE 4   /* a residual or state value became NaN/Inf on the device              */
#define CSU_ERR_DIVERGED 5    /* residual grew past the divergence threshold                          */
#define CSU_ERR_CANCELLED 6   /* a serving request was cancelled                                      */
#define CSU_ERR_CUDA 7        /* a CUDA runtime call failed                                           */
#define CSU_ERR_UNSUPPORTED 8 /* setting the engine does not implement                               */
#define CSU_ERR_STATE 9       /* call made in the wrong state (e.g. before csu_set_state)            */
#define CSU_ERR_NO_DEVICE 10  /* no CUDA device / extension missing                                   */

/* flux schemes, fluxChoice (flux.c:14-46) */
#define CSU_FLUX_ROE 0
#define CSU_FLUX_AUSM 1
#define CSU_FLUX_AUSMDV 2
#define CSU_FLUX_AUSMPUP 3
#define CSU_FLUX_AUSMPUP2 4

/* boundary flags, boundaryChoice (boundary.c:479-511) */
#define CSU_BC_SYMMETRY 0
#define CSU_BC_INLET 1
#define CSU_BC_OUTLET 2
#define CSU_BC_WALL 3
#define CSU_BC_WALLT 4

/* time schemes, solverTimeSchemeChoice (solver.c:1957-1981) */
#define CSU_TS_RK 0
#define CSU_TS_LUSGS 1
#define CSU_TS_DPLUR 2

/* Scalar settings of one solve: the SOLVER fields of solver.h:86-170 that the hot path reads. */
typedef struct csu_config {
    int nvar;          /* 4 Euler/laminar, 5 SA, 6 SST (solver.c:1789-1798)                      */
    int order;         /* 1 or 2                                                                 */
    int flux;          /* CSU_FLUX_*                                                             */
    int stages;        /* RK stages 1, 3, 4, 5 (solver.c:788-840)                                */
    int time_scheme;   /* CSU_TS_*                                                               */
    int n_linear;      /* DPLUR sweeps (Nlinear, default 20)                                     */
    int dt_local;      /* local time step for RK (dtLocal)                                       */
    int dt_local_n;    /* iteration after which dtLocal switches off (dtLocalN, -1 = never)      */
    int laminar, sa, sa_cc, sst, sst_trans, axisymmetric, turb1order, visc_blazek, tp;
    int limiter_type;  /* 0: K^3 (omega/omega_max)^1.5 q_inf^2, 1: (K (max-min))^2 (limiter.c)  */
    int tube;          /* unsteady shock-tube mode (solver.c:1912)                               */
    double limiter_k;  /* limK                                                                   */
    double cfl, w_imp, r_lim, p_out, t_wall, sref, turb_ratio, e_fix, pr, pr_t;
    double gamma, gas_r;                  /* 1.4, 287.0530 (solver.c:1425)                       */
    double pin[7];                        /* inlet primitives r,u,v,p,T,(nt | k,w) CONDITION.Pin */
    double uin[6];                        /* inlet conserved state CONDITION.Uin                  */
    double mach_inf;                      /* CONDITION.mach (AUSM+up M_inf)                       */
    double inlet_p, inlet_t;              /* CONDITION.p, CONDITION.T                             */
    double sst_l, k_factor, o_factor, o_wall_factor;
    /* Extensions (no reference keyword semantics to follow; 0 keeps the reference behaviour). */
    int implicit_fp32;       /* DPLUR blocks stored and applied in FP32 (keyword implicitFP32)           */
    int implicit_local_dt;   /* implicit diagonal with each cell's own step, Omega/(CFL dtL_i)
                                (keyword implicitLocalDt) instead of the global minimum step            */
    int cfl_ramp_iters;      /* CFL grows geometrically from CFL to cfl_max over this many iterations
                                (keywords CFLramp, CFLmax)                                              */
    double cfl_max;
    double conv_drop;        /* stop once res[0] <= conv_drop * the largest res[0] so far (convDrop)     */
    int iter_cap;            /* packs: freeze a solve after this many iterations (iterCap; 0: none)     */
    int limiter_func;        /* limiterFunc: 0 Venkatakrishnan (reference), 1 Barth-Jespersen / minmod  */
    int gradient;            /* gradient: 0 least squares (reference), 1 Green-Gauss                    */
    int sa_implicit_source;  /* saImplicitSource: SA with DPLUR, the source's destruction-dominated part in
                                the diagonal of the nt row (-Omega min(dQ/d(rho nt), 0)); 0 explicit source
                                as the reference                                                          */
} csu_config;

/*
 * The mesh as meshInit (mesh.c:115-266) leaves it, as plain arrays. A caller holding the reference's
 * MESH* fills it directly (con from mesh->con, cell_faces from ELEMENT.f, cell_nei from ELEMENT.neiL, the
 * boundary faces from mesh->bc[m]->elem); csu_case_load builds the same arrays from a case folder.
 */
typedef struct csu_mesh_desc {
    int n_points;
    const double* xy;          /* 2 per point (mesh->p)                                           */
    int n_cells;
    const int* cell_npts;      /* 3 or 4 (ELEMENT.Np)                                             */
    const int* cell_nodes;     /* 4 per cell, counter-clockwise after mesh.c:222-242, -1 padded   */
    int n_faces;               /* interior faces (mesh->Ncon)                                     */
    const int* con;            /* 4 per face: e0, e1, p0, p1 (mesh->con, face order of mesh.c:1172) */
    const int* cell_nint;      /* interior faces of the cell (ELEMENT.neiN after meshCalcFaces)    */
    const int* cell_faces;     /* 4 per cell: +(f+1) owner / -(f+1) neighbour (ELEMENT.f)          */
    const int* cell_nei;       /* 4 per cell in ELEMENT.neiL order: >=0 cell, <0 -(1+boundary face) */
    int n_markers;
    const int* marker_nbf;     /* boundary faces per marker (MESHBC.Nelem)                        */
    const int* marker_flag;    /* CSU_BC_* per marker (MESHBC.flagBC)                             */
    int n_bfaces;              /* sum of marker_nbf                                               */
    const int* bface;          /* 3 per boundary face, marker-major: p0, p1 (mesh.c:987), owner   */
    const double* wall_dist;   /* per cell (ELEMENT.d, sa.c:703) or NULL                          */
} csu_mesh_desc;

/* Per-iteration record, the quantities solverSolve prints and writes to convergence.csv
 * (solver.c:1891-1906): hist[it*(nvar+4) + k] = res[k], then Cx_p, Cx_v, Cy_p, Cy_v. */
#define CSU_HIST_STRIDE(nvar) ((nvar) + 4)

typedef struct csu_ctx csu_ctx;
typedef struct csu_case csu_case;

/* ------------------------------------------------------------------------------------------------
 * Host front end (C): a case folder as the reference reads it.
 * ---------------------------------------------------------------------------------------------- */

/* Parse <wd>input.dat (input.c:7-95), read <wd>mesh.su2 and build the connectivity
 * (meshInit, mesh.c:115-266), apply solverSetData/solverInit (solver.c:1403-1834) and the initial
 * state of solverInitDomain (solver.c:1660-1726: freestream, tube or restart.csv). Replaces
 * solverInit (solver.c:1728) minus device work. Wall distance (sa.c:703-793) is computed when sa/sst. */
int csu_case_load(const char* wd, csu_case** out);
/* Same from in-memory file contents (no file system). */
int csu_case_load_mem(const char* input_dat, const char* mesh_su2, const char* restart_csv, csu_case** out);
int csu_case_mesh(const csu_case* c, csu_mesh_desc* out);         /* views into the case          */
int csu_case_config(const csu_case* c, csu_config* out);
int csu_case_initial_state(const csu_case* c, double* U);         /* nvar*ncells, [var][cell]     */
int csu_case_get_int(const csu_case* c, const char* keyword, int* out);        /* inputGetValue  */
int csu_case_get_double(const csu_case* c, const char* keyword, double* out);
int csu_case_marker_name(const csu_case* c, int marker, char* out, int cap);
void csu_case_free(csu_case* c);

/* The whole program flow of the reference executable (main.c:18-45 with solverSolve, solver.c:1836-1943)
 * on the engine: read <wd>, iterate Nmax times (or run the tube to tmax), and write convergence.csv,
 * friction.csv, solution.csv, solution2.csv and restart.csv into <wd>. verbose prints like the reference. */
int csu_run_case(const char* wd, int verbose);

/* ------------------------------------------------------------------------------------------------
 * Device engine.
 * ---------------------------------------------------------------------------------------------- */

/* Build the device layout (renumbered cells, face streams, geometry, least-squares weights) and
 * allocate all device state on the current CUDA device. The DPLUR increment starts at zero like
 * implicitInitDPLUR (implicit.c:649-656). */
int csu_create(const csu_mesh_desc* mesh, const csu_config* cfg, csu_ctx** out);
void csu_destroy(csu_ctx* ctx);

/* Upload/download the conserved state, [var][cell] in reference cell order (one copy of the caller's
 * array each way, a DMA when it is pinned; the renumbering runs on the device; both return once the copy
 * is done). A new state restarts the solve's scalars (history rows, residual-drop reference, halt flags)
 * for the next csu_iterate; a DPLUR context also computes the state's primitives (solverCalcPrimitive's
 * clamps written back, solver.c:1153-1220) during the upload. */
int csu_set_state(csu_ctx* ctx, const double* U);
int csu_get_state(csu_ctx* ctx, double* U);
/* Same with the reference's row pointers: U[k][i] (solver->U). */
int csu_set_state_rows(csu_ctx* ctx, const double* const* U);
int csu_get_state_rows(csu_ctx* ctx, double* const* U);

/* One residual evaluation solverCalcR(solver, solver->U) (solver.c:685) on the device, including its
 * write-back clamps into U (solver.c:1163-1211). R (nullable) receives [var][cell]. */
int csu_residual(csu_ctx* ctx, double* R);

/* n iterations of the steady loop of solverSolve (solver.c:1864-1906) on the device; it0 is the
 * iteration counter of the first one (dtLocalN uses it). hist (nullable) gets n rows of
 * CSU_HIST_STRIDE(nvar) doubles. Returns CSU_ERR_NONFINITE if the state became non-finite. */
int csu_iterate(csu_ctx* ctx, int n, int it0, double* hist);
/* Same, also reporting how many iterations ran before the convergence stop (conv_drop) triggered. */
int csu_iterate_ex(csu_ctx* ctx, int n, int it0, double* hist, int* n_done);

/* One iteration like csu_iterate(ctx, 1, it0, hist) that also returns what its last residual evaluation
 * worked on: the cell primitives P (ncells*(nvar+1), [cell][k], as CSU_DUMP_P) and the gradients G (dPx rows
 * then dPy rows, as CSU_DUMP_GRAD) -- the state the iteration started from for the implicit schemes, the last
 * stage's input for RK. These are the E->P and dPx the reference's friction output reads after its loop
 * (solverCalcCoeff2, solver.c:1303-1340, called at 1908). */
int csu_iterate_views(csu_ctx* ctx, int it0, double* hist, double* P, double* G);

/* The unsteady tube loop (solver.c:1912-1942) up to tmax; returns steps taken and final time. */
int csu_tube_run(csu_ctx* ctx, double tmax, int* steps, double* t_final);

/* Debug/parity views of the last residual evaluation, reference layouts:
 *  CSU_DUMP_P       ncells*(nvar+1) [cell][k]   cell primitives ELEMENT.P
 *  CSU_DUMP_GHOST_P nbfaces*(nvar+1)            ghost primitives of boundary elements
 *  CSU_DUMP_GRAD    2*nvar*ncells               dPx rows then dPy rows ([k][cell])
 *  CSU_DUMP_PHI     nvar*ncells                 limiter phi
 *  CSU_DUMP_FACEFLUX nvar*nfaces                faceFlux [k][face]
 *  CSU_DUMP_R       nvar*ncells                 residual
 *  CSU_DUMP_D       ncells                      implicit diagonal D (after an implicit iteration)
 *  CSU_DUMP_DTL     ncells                      dtL (local steps, or Omega/Lc for implicit)
 *  CSU_DUMP_DW      nvar*ncells                 last implicit increment dW1
 *  CSU_DUMP_BLOCKS  ncells*4*nvar*nvar          DPLUR blocks [cell][slot][row][col], slots in ELEMENT.f order
 *  CSU_DUMP_LSQ_X87 1                           gradient slots (cell, variable) so far that the FP64
 *                                               least squares could not decide and left to the integer x87
 *                                               model (no reference counterpart: a diagnostic of this engine)
 *  CSU_DUMP_SST_JAC 6*ncells                    SST source Jacobians dQkdr, dQkdrk, dQkdro, dQodr, dQodrk,
 *                                               dQodro [6][cell] of the last LU-SGS or DPLUR iteration
 *                                               (sst.c:643-680)
 *  CSU_DUMP_BVISC   nbfaces*4 [bface][k]        viscous flux of each boundary face: x and y momentum, energy,
 *                                               transported scalar (components 1..4 of boundaryFaceViscFlux,
 *                                               laminar.c:128-346; saBoundaryFaceViscFlux, sa.c:370-692;
 *                                               sstBoundaryFaceViscFlux, sst.c:202-547); viscous models only */
#define CSU_DUMP_P 1
#define CSU_DUMP_GHOST_P 2
#define CSU_DUMP_GRAD 3
#define CSU_DUMP_PHI 4
#define CSU_DUMP_FACEFLUX 5
#define CSU_DUMP_R 6
#define CSU_DUMP_D 7
#define CSU_DUMP_DTL 8
#define CSU_DUMP_DW 9
#define CSU_DUMP_BLOCKS 10
#define CSU_DUMP_LSQ_X87 11
#define CSU_DUMP_SST_JAC 12
#define CSU_DUMP_BVISC 13
int csu_dump(csu_ctx* ctx, int what, double* out);

/* Ghost primitives and boundary viscous fluxes of the current state, the inputs of the reference's surface
 * writers after its last iteration (laminar.c:350-492, sa.c:854-996, sst.c:820-962): solverWriteSolution2
 * recomputes the cell and ghost primitives of the final state (solver.c:2038) while the gradients stay those
 * of the last residual evaluation. Afterwards CSU_DUMP_GHOST_P and CSU_DUMP_BVISC return them. */
int csu_wall_data(csu_ctx* ctx);

/* Run the engine's work on a caller-provided cudaStream_t (NULL: the context's own stream). */
int csu_set_stream(csu_ctx* ctx, void* stream);

/* Kernel kinds of csu_time_kernels. */
#define CSU_K_PRIM 0     /* primitives + clamps (solverCalcPrimitive)                    */
#define CSU_K_GRAD 1     /* least-squares gradient + limiter (solverUpdateGrad, inter)    */
#define CSU_K_FLUX 2     /* interior and boundary face fluxes (inter, boundary)           */
#define CSU_K_RK 3       /* residual gather + RK stage (solverRK)                         */
#define CSU_K_IMPL 4     /* residual gather + implicit diagonal                           */
#define CSU_K_SWEEP 5    /* one DPLUR Jacobi sweep                                        */
#define CSU_K_FINALIZE 6 /* norms, force coefficients, step size                          */
#define CSU_K_RESID 7    /* residual gather only                                          */
#define CSU_K_BLOCKS 8   /* DPLUR off-diagonal blocks (finite-difference face Jacobians)  */
#define CSU_K_COUNT 9
/* Runs `iters` iterations with a CUDA event after every kernel and returns, per kind, the summed device
 * time in ms and the launch count (the iterations advance the state like csu_iterate). */
int csu_time_kernels(csu_ctx* ctx, int iters, double* ms, int* count);

/* Residual RMS norms res[k] = sqrt(sum_i R[k][i]^2 / ncells) -- the quantity of solverCalcRes -- from a
 * residual the caller holds in device memory ([var][cell], nvar <= 6), written to the caller's device array
 * res (nvar doubles), asynchronously on `stream` (a cudaStream_t, NULL for the default stream). No
 * counterpart in the reference: this entry allocates nothing, for callers that give the solver a fixed
 * device-memory budget under their own allocator or must not call cudaMalloc/cudaFree (which synchronize
 * the device). Its scratch is a fixed array inside the library, held by every GPU that loads it (192 KiB);
 * ncells is limited to 8,388,608 (CSU_ERR_INPUT beyond). The first call on a device looks the scratch
 * address up (cudaGetSymbolAddress) and should come before any stream capture on that device; the address
 * is kept for the process, so the entry must not be used across a cudaDeviceReset. Calls whose kernels
 * overlap on one GPU share the scratch and race. A CUDA error already pending from earlier work is returned
 * (CSU_ERR_CUDA) before anything is launched. */
int csu_residual_norms_noalloc(const double* R, int nvar, int ncells, double* res, void* stream);

/* Launch-shape autotuner (no counterpart in the reference): times the face-chunk size of the face-flux
 * kernel (32 or 64 faces per block reading their cells from global memory, or 128 faces per block staging
 * their cells through a shared-memory window) and the cell-block size of the DPLUR sweeps (64, 128 or 256) on this
 * context and keeps the fastest; neither choice changes a result bit. A context tunes itself on its first
 * csu_iterate (16,384 cells or more; a cache per device, model and size class spares packs of a class seen
 * before the timing); this call re-times now and reports the choice. CSU_AUTOTUNE=0 in the environment
 * keeps the default shapes (64 faces, 128 cells). */
int csu_autotune(csu_ctx* ctx, int* flux_faces_per_block, int* sweep_cells_per_block);

/* Counters of the engine: kernels launched since creation, device bytes held. */
int csu_stats(csu_ctx* ctx, long long* kernel_launches, long long* device_bytes);

/* ---- packs: several steady solves advanced by one launch of each kernel --------------------------------
 * No counterpart in the reference (it runs one case per process). A solve is first prepared on the host
 * (its device layout and byte count, no device memory); a pack concatenates prepared solves that share the
 * settings the launch sequence depends on (model, scheme, order, time stepping, Nlinear, limiter, gas
 * model); their flow conditions, CFL schedule, stopping drop and reference length may differ. Cells of a
 * solve are block aligned and every reduction (norms, time step, coefficients, DPLUR early exit,
 * convergence stop) is per solve, so a solve's iterations are bit-identical alone and in a pack.
 * csu_iterate advances every solve of a pack; a converged or failed solve is frozen while the others run.
 * On a pack, csu_iterate returns once the iterations are queued on the device (its n_done reports the
 * iterations queued); csu_pack_info / csu_pack_infos / csu_pack_get_state wait for them.
 */
typedef struct csu_prep csu_prep;
typedef struct csu_solve_info {
    int iter;        /* iterations done (the solve's own counter)                  */
    int status;      /* CSU_OK or CSU_ERR_NONFINITE                                 */
    int done;        /* 1: the residual-drop stop (convDrop) was reached; 2: iterCap; 3: stopped by
                        csu_pack_stop                                                */
    int hist_rows;   /* history rows recorded by the last csu_iterate call          */
    int have_res0;   /* res0 holds a residual                                       */
    double res0[6];  /* largest RMS residuals of the solve so far (per variable)    */
    double res[6];   /* RMS residuals of its last iteration                         */
    double coef[4];  /* Cx_p, Cx_v, Cy_p, Cy_v of its last iteration                */
} csu_solve_info;

int csu_prep_create(const csu_mesh_desc* mesh, const csu_config* cfg, csu_prep** out);
long long csu_prep_bytes(const csu_prep* p);   /* device bytes the solve needs in a pack   */
int csu_prep_cells(const csu_prep* p);
void csu_prep_destroy(csu_prep* p);
int csu_pack_create(const csu_prep* const* solves, int n, csu_ctx** out);
int csu_pack_size(csu_ctx* ctx);
int csu_pack_set_state(csu_ctx* ctx, int k, const double* U);   /* U[nvar][ncells_k], reference order */
int csu_pack_get_state(csu_ctx* ctx, int k, double* U);
int csu_pack_info(csu_ctx* ctx, int k, csu_solve_info* info);
int csu_pack_infos(csu_ctx* ctx, csu_solve_info* infos);        /* all solves, one device read */
int csu_pack_history(csu_ctx* ctx, int k, double* hist, int max_rows, int* rows);
int csu_pack_transfer(csu_ctx* from, int k_from, csu_ctx* to, int k_to);
/* Freezes solve k of a pack where it stands (done = 3): the pack's next iterations leave it unchanged while
 * the other solves go on as before. The serving layer's cancellation uses it. */
int csu_pack_stop(csu_ctx* ctx, int k);
/* A new pack of `solves` in which solve k, when keep[k] >= 0, is solve keep[k] of `old` (mesh rows and
 * iteration state copied on the device, nothing re-uploaded); the others come from their host layouts and
 * need csu_pack_set_state. `old` is left unchanged (destroy it afterwards). */
int csu_pack_rebuild(csu_ctx* old, const int* keep, const csu_prep* const* solves, int n, csu_ctx** out);

/* ---- serving: continuous batching of steady solves on one GPU ------------------------------------------
 * No counterpart in the reference. Requests queue on submission; every csu_srv_step retires converged /
 * failed / capped solves, admits queued requests (first fit, arrival order) while their device bytes
 * (csu_prep_bytes) fit the budget, rebuilds the packs whose membership changed (continuing solves move with
 * their iteration state, so each result is the same as the solve alone) and advances every pack by
 * iters_per_step iterations. Each request stops at its configuration's convDrop (csu_config.conv_drop) or
 * after max_iters iterations. Times are seconds since csu_srv_create (host clock).
 */
#define CSU_SRV_QUEUED 0
#define CSU_SRV_RUNNING 1
#define CSU_SRV_CONVERGED 2
#define CSU_SRV_FAILED 3
#define CSU_SRV_MAXITER 4
#define CSU_SRV_CANCELLED 5
typedef struct csu_srv csu_srv;
typedef struct csu_srv_config {
    long long budget_bytes;  /* device bytes the running solves may take                      */
    int iters_per_step;      /* iterations per csu_srv_step (a multiple of 8 replays graphs)   */
    int max_pack;            /* most solves per pack (0: no limit)                             */
    int rebuild_steps;       /* admit into a running pack at most every this many steps (a pack
                                rebuild re-uploads its meshes; finished solves stay frozen in the
                                pack until the next rebuild); 0 or 1: every step                  */
    int prep_threads;        /* host threads that build submitted meshes' device layouts while the
                                packs iterate (csu_srv_submit then copies the mesh and returns at
                                once; a request is admitted once prepared, and one whose layout
                                fails or exceeds the budget ends CSU_SRV_FAILED); 0: csu_srv_submit
                                prepares the mesh itself and reports those errors                  */
} csu_srv_config;
typedef struct csu_srv_request_info {
    int state;               /* CSU_SRV_*                                                      */
    int iters;               /* iterations done                                                */
    int n_cells;
    double drop;             /* RMS rho-residual / its first value                             */
    double t_submit, t_start, t_end;
    int status;              /* CSU_OK, or why it failed or stopped: CSU_ERR_OOM (over the budget),
                                CSU_ERR_INPUT (its layout failed), CSU_ERR_NONFINITE, CSU_ERR_CANCELLED */
    double coef[4];          /* Cx_p, Cx_v, Cy_p, Cy_v of its last iteration (solverCalcCoeff3)           */
} csu_srv_request_info;

int csu_srv_create(const csu_srv_config* cfg, csu_srv** out);
int csu_srv_submit(csu_srv* s, const csu_mesh_desc* mesh, const csu_config* cfg, const double* U0, int max_iters,
                   long long* id);
int csu_srv_step(csu_srv* s, int* n_running, int* n_queued);
int csu_srv_info(csu_srv* s, long long id, csu_srv_request_info* out);
int csu_srv_take(csu_srv* s, long long id, double* U);      /* final state (reference order); forgets it */
/* Cancels a queued or running request (CSU_ERR_STATE once it has finished). A queued one never starts; a
 * running one stops where it stands (csu_srv_take returns that state) and its pack is rebuilt without it at
 * the next csu_srv_step; the other solves' iterations are not affected. Its state becomes
 * CSU_SRV_CANCELLED and its status CSU_ERR_CANCELLED. */
int csu_srv_cancel(csu_srv* s, long long id);
/* The message of a failed or cancelled request (also for failures met on a preparation thread). */
int csu_srv_message(csu_srv* s, long long id, char* buf, int cap);
/* Requests that reached a final state (converged, failed, iteration cap, cancelled) since the last call, in
 * the order they got there: up to cap ids into ids, their number into *n (the rest wait for the next call). */
int csu_srv_poll(csu_srv* s, long long* ids, int cap, int* n);
int csu_srv_totals(csu_srv* s, long long* solve_iterations, long long* cell_updates, long long* used_bytes);
/* host seconds spent rebuilding packs, iterating and polling, and the number of rebuilds */
int csu_srv_times(csu_srv* s, double* rebuild_s, double* iterate_s, double* poll_s, int* rebuilds);
void csu_srv_destroy(csu_srv* s);

const char* csu_last_error(void);
const char* csu_strerror(int status);

#ifdef __cplusplus
}
#endif
#endif
