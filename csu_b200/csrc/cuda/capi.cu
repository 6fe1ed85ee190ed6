// capi.cu -- the extern "C" entry points of include/csu_gpu.h: device context, data upload, the per-iteration
// launch sequences and their CUDA-graph replay.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <vector>
#include <algorithm>
#include <mutex>
#include <map>
#include <tuple>
#include "csu_gpu.h"
#include "kernels.cuh"

extern "C" {
#include "../host/layout.h"
void csu_set_error(const char* fmt, ...);
}

using namespace csu;

namespace {

struct Arena {
    char* base = nullptr;
    size_t size = 0, used = 0;
};

// Device arenas of destroyed packs kept for the next pack: a rebuild makes the new pack before it frees the
// old one, so two arenas alternate and the serving loop stops allocating and freeing gigabytes per rebuild.
// An arena is reused when it holds the request and at most twice it; new pack arenas get 25 % headroom.
// Entries remember their device: a pack takes only arenas of the device current when it is made.
struct CachedArena {
    int dev;
    char* base;
    size_t size;
};
std::mutex g_arena_mu;
std::vector<CachedArena> g_arena_cache;

cudaError_t pack_arena_take(int dev, size_t need, char** base, size_t* size)
{
    {
        std::lock_guard<std::mutex> lk(g_arena_mu);
        size_t best = g_arena_cache.size();
        for (size_t k = 0; k < g_arena_cache.size(); k++) {
            if (g_arena_cache[k].dev != dev) continue;
            size_t sz = g_arena_cache[k].size;
            if (sz >= need && sz <= 2 * need && (best == g_arena_cache.size() || sz < g_arena_cache[best].size))
                best = k;
        }
        if (best < g_arena_cache.size()) {
            *base = g_arena_cache[best].base;
            *size = g_arena_cache[best].size;
            g_arena_cache.erase(g_arena_cache.begin() + best);
            return cudaSuccess;
        }
    }
    size_t want = (need + need / 4 + 255) & ~size_t(255);
    cudaError_t e = cudaMalloc((void**)base, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        want = need;
        e = cudaMalloc((void**)base, want);
    }
    *size = e == cudaSuccess ? want : 0;
    return e;
}

void pack_arena_give(int dev, char* base, size_t size)
{
    std::lock_guard<std::mutex> lk(g_arena_mu);
    int held = 0;
    for (const CachedArena& a : g_arena_cache) held += a.dev == dev;
    if (held < 2) {
        g_arena_cache.push_back({dev, base, size});
        return;
    }
    cudaFree(base);
}

// RK stage coefficients of solverStepRK (solver.c:788-840)
const double RK1[1] = {1.0};
const double RK2[2] = {0.5, 1.0}; // extension: midpoint rule (the reference has no 2-stage scheme)
const double RK3[3] = {0.1481, 0.4, 1.0};
const double RK4[4] = {0.0833, 0.2069, 0.4265, 1.0};
const double RK5[5] = {0.0533, 0.1263, 0.2375, 0.4414, 1.0};

} // namespace

// Launch shapes the autotuner chooses among (csu_autotune): faces per k_flux block (32 or 64 reading the
// cells from global memory; 128 staging each block's cells through shared memory, k_flux_st) and cells per
// DPLUR sweep block. None changes a result bit: fluxes are per face with the same arithmetic, sweeps per
// cell, and the first sweep's partial norms come one row per warp whatever the block size.
static const int FLUX_BLOCKS[3] = {32, 64, 128};
static const int SWEEP_BLOCKS[3] = {64, 128, 256};

struct csu_ctx {
    int model = 0, nv = 4;
    csu_config cfg;
    csu_layout L;
    Prm prm;                 // parameters of solve 0 (the only one outside packs)
    int nsolve = 1;
    bool is_pack = false;    // made by csu_pack_create (even with one solve): solves keep their own counters
    bool pack_wall_d = false;// packs: the solves carry wall distances (SA, SST)
    std::vector<Prm> prms;   // per solve, mirrored at d_prm
    Prm* d_prm = nullptr;
    double* hist = nullptr;  // nsolve blocks of hist_cap rows
    // packs: cell / interior-face / boundary-face offsets, cell counts and renumbering of each solve
    std::vector<int> cell0, face0, bface0, ncs;
    std::vector<std::vector<int>> n2o;
    Mesh mesh;
    State st;
    Arena arena;
    void* state_base = nullptr;
    size_t state_bytes = 0;
    int* d_wall_rank = nullptr;
    int nwall = 0;
    cudaStream_t stream = nullptr;
    int prepared = 0;
    int xcur = 0;
    long long launches = 0;
    int hist_cap = 0;
    int gb_c = 0;
    const double* rk = nullptr;
    // CUDA graphs of GRAPH_SIZES[g] iterations, one per DPLUR increment-buffer parity at their start (an odd
    // Nlinear flips it every iteration); captured on first use, kept until the launch sequence changes
    cudaGraphExec_t graphs[4][2] = {};
    long long graph_launches[4][2] = {};
    // L2 residency of the DPLUR blocks when they fit in the persisting part of L2 (plan_l2_window); the window
    // is set on the kernel nodes of the captured iteration graphs
    cudaAccessPolicyWindow l2win = {};
    Scalars* h_sc = nullptr;   // pinned: solve 0's scalars, read back once at the end of csu_iterate
    int* h_flags = nullptr;    // pinned: halt flags (status, done) of two chunks in flight
    bool snap = false;         // csu_iterate_views: copy the last residual evaluation's primitives/gradients
    double* h_snap = nullptr;  // pinned: those copies (W4, WT, Wx, G4x, G4y, Gxx, Gxy in device order)
    cudaEvent_t ev_poll[2] = {nullptr, nullptr};
    double* h_hist = nullptr;  // pinned: solve 0's history rows (hist_cap rows)
    int have_debug = 0;
    cudaStream_t own_stream = nullptr;
    // DPLUR blocks run on a side stream, forked from and joined back to the engine stream
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_grad = nullptr;
    // DPLUR graph capture: iterations in the graph being captured and the next one's index; an iteration's
    // k_finalize left to run on the side stream beside the next iteration's gradients and fluxes, with the
    // face-coefficient buffer it sums
    int defer_n = 0, defer_i = 0;
    bool fin_pending = false;
    int fin_bsel = 0;
    int max_ni = 4;          // most interior faces of a cell (k_blocks covers slots [0, max_ni))
    int flux_fb = 64;        // faces per k_flux block (one of FLUX_BLOCKS)
    int sweep_sb = 128;      // cells per DPLUR sweep block (one of SWEEP_BLOCKS)
    bool tuned = false;      // launch shapes chosen (csu_autotune, or its cache on the first iteration)
    int device = 0;          // the CUDA device current when the context was made (its memory lives there)
    int sm_count = 148;      // that device's multiprocessors
    // one-solve contexts: the renumbering on the device and a staging buffer for the state in reference order
    int* d_n2o = nullptr;
    double* d_stage = nullptr;
    // kernel timing (csu_time_kernels): an event after every launch, tagged with the kernel kind
    bool timing = false;
    std::vector<cudaEvent_t> ev;
    std::vector<int> ev_kind;
    size_t ev_used = 0;
};

// kinds of csu_time_kernels
enum { KPRIM = 0, KGRAD, KFLUX, KRK, KIMPL, KSWEEP, KFIN, KRESID, KBLK, KCOUNT };

static void tmark(csu_ctx* x, int kind)
{
    if (!x->timing) return;
    if (x->ev_used == x->ev.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        x->ev.push_back(e);
        x->ev_kind.push_back(kind);
    }
    x->ev_kind[x->ev_used] = kind;
    cudaEventRecord(x->ev[x->ev_used], x->stream);
    x->ev_used++;
}

// iterations per captured graph; a call of n iterations replays the largest first (n = 8a + 4b + 2c + d)
static const int GRAPH_SIZES[4] = {8, 4, 2, 1};
// one-solve calls longer than this are launched in chunks of it, checking between chunks whether the solve
// has halted
static const int STOP_CHUNK = 64;

static void drop_graphs(csu_ctx* x)
{
    for (int g = 0; g < 4; g++)
        for (int q = 0; q < 2; q++) {
            if (x->graphs[g][q]) cudaGraphExecDestroy(x->graphs[g][q]);
            x->graphs[g][q] = nullptr;
            x->graph_launches[g][q] = 0;
        }
}

static int cuda_fail(cudaError_t e, const char* what)
{
    csu_set_error("%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? CSU_ERR_OOM : CSU_ERR_CUDA;
}

#define CK(call)                                                                                                   \
    do {                                                                                                           \
        cudaError_t e_ = (call);                                                                                   \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);                                                        \
    } while (0)

template <typename T>
static T* carve(Arena& a, size_t count)
{
    size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    if (a.base == nullptr) {
        a.size += bytes; // sizing pass
        return nullptr;
    }
    T* p = reinterpret_cast<T*>(a.base + a.used);
    a.used += bytes;
    return p;
}

// Lays out every device array of a context in one allocation (first pass sizes, second pass carves).
static void plan(csu_ctx* x, Arena& a)
{
    const int nc = x->L.nc, nf = x->L.nf, nb = x->L.nb, nv = x->nv, nx = nv - 4;
    const size_t c4 = (size_t)4 * nc;
    Mesh& m = x->mesh;
    State& s = x->st;
    m.npts = carve<int>(a, nc);
    m.nint = carve<int>(a, nc);
    m.nslot = carve<int>(a, nc);
    m.nei = carve<int>(a, c4);
    m.wx = carve<double>(a, c4);
    m.wy = carve<double>(a, c4);
    m.ldx = carve<double>(a, c4);
    m.ldy = carve<double>(a, c4);
    m.lm = carve<unsigned long long>(a, c4);
    m.les = carve<int>(a, c4);
    m.lrv = carve<unsigned long long>(a, nc);
    m.lq = carve<double2>(a, c4);
    m.ex = carve<double>(a, c4);
    m.ey = carve<double>(a, c4);
    m.fslot = carve<int>(a, c4);
    m.fnb = carve<int>(a, c4);
    m.omega = carve<double>(a, nc);
    m.sxh = carve<double>(a, nc);
    m.syh = carve<double>(a, nc);
    m.wall_d = (x->is_pack ? x->pack_wall_d : x->L.wall_d != nullptr) ? carve<double>(a, nc) : nullptr;
    m.dslat = carve<double>(a, nc);
    m.fe = carve<int2>(a, nf);
    m.fn = carve<double2>(a, nf);
    m.fds = carve<double>(a, nf);
    m.r0 = carve<double2>(a, nf);
    m.r1 = carve<double2>(a, nf);
    m.fd = carve<double2>(a, nf);
    m.fL = carve<double>(a, nf);
    m.bown = carve<int>(a, nb);
    m.bflag = carve<int>(a, nb);
    m.bold = carve<int>(a, nb);
    m.bn = carve<double2>(a, nb);
    m.bds = carve<double>(a, nb);
    m.bd = carve<double2>(a, nb);
    m.bL = carve<double>(a, nb);
    m.bun = carve<double2>(a, nb);
    m.bds2 = carve<double>(a, nb);
    m.color = carve<int>(a, nc);
    m.color_cells = carve<int>(a, nc);
    x->d_wall_rank = carve<int>(a, nb);

    s.U4 = carve<double4>(a, nc);
    s.Ux = carve<double>(a, (size_t)nx * nc);
    s.W4 = carve<double4>(a, nc);
    s.WT = carve<double>(a, nc);
    s.Wx = carve<double>(a, (size_t)nx * nc);
    s.G4x = carve<double4>(a, nc);
    s.G4y = carve<double4>(a, nc);
    s.PH4 = carve<double4>(a, nc);
    int visc = x->cfg.laminar || x->cfg.sa || x->cfg.sst;
    s.GTx = carve<double>(a, visc ? nc : 0);
    s.GTy = carve<double>(a, visc ? nc : 0);
    s.FV = carve<double4>(a, visc ? (size_t)nf + nb : 0);
    s.MIT = carve<double>(a, (x->cfg.sa || x->cfg.sst) ? nf : 0);
    s.FV5 = carve<double>(a, x->cfg.sst ? (size_t)nf + nb : 0);
    s.Gxx = carve<double>(a, (size_t)nx * nc);
    s.Gxy = carve<double>(a, (size_t)nx * nc);
    s.PHx = carve<double>(a, (size_t)nx * nc);
    s.F4 = carve<double4>(a, (size_t)nf + nb);
    s.Fx = carve<double>(a, (size_t)nx * (nf + nb));
    s.R4 = carve<double4>(a, nc);
    s.Rx = carve<double>(a, (size_t)nx * nc);
    s.dtl = carve<double>(a, nc);
    s.dpart = carve<double>(a, nc);
    int implicit = x->cfg.time_scheme != CSU_TS_RK;
    for (int k = 0; k < 2; k++) {
        s.X4[k] = implicit ? carve<double4>(a, nc) : nullptr;
        s.Xx[k] = implicit ? carve<double>(a, (size_t)nx * nc) : nullptr;
    }
    bool dplur = x->cfg.time_scheme == CSU_TS_DPLUR;
    s.blocks = dplur && !x->cfg.implicit_fp32 ? carve<double>(a, c4 * nv * nv) : nullptr;
    s.blocks32 = dplur && x->cfg.implicit_fp32 ? carve<float>(a, c4 * nv * nv) : nullptr;
    // partial norms: one row per 256-cell block, or per 128-cell block from the DPLUR first sweep
    s.part = carve<double>(a, (size_t)((nc + BLOCK - 1) / BLOCK) * (BLOCK / 32) * nv);
    s.bcoef = carve<double>(a, (size_t)4 * (nb > 0 ? nb : 1));
    s.bcoef2 = dplur ? carve<double>(a, (size_t)4 * (nb > 0 ? nb : 1)) : nullptr;
    s.sc = carve<Scalars>(a, x->nsolve);
    s.bsolve = x->nsolve > 1 ? carve<int>(a, (nc + BLOCK - 1) / BLOCK) : nullptr;
    s.csolve = x->nsolve > 1 ? carve<int>(a, nc) : nullptr;
    x->d_prm = carve<Prm>(a, x->nsolve);
    s.dbg_ghost = carve<double>(a, (size_t)(nb > 0 ? nb : 1) * (nv + 1));
    s.lsq_x87 = carve<unsigned long long>(a, 1);
    s.dQ = x->cfg.sst && x->cfg.time_scheme != CSU_TS_RK ? carve<double>(a, (size_t)6 * nc)
           : (x->cfg.sa && x->cfg.time_scheme == CSU_TS_DPLUR && x->cfg.sa_implicit_source) ? carve<double>(a, nc)
                                                                                            : nullptr;
    s.gfix = carve<int2>(a, (size_t)nc * (nv + 1)); // at most one entry per cell and variable (and T)
    s.gfix_n = carve<unsigned>(a, 1);
    if (!x->is_pack) {
        x->d_n2o = carve<int>(a, nc);
        x->d_stage = carve<double>(a, (size_t)nv * nc);
    }
}

static int upload_mesh(csu_ctx* x)
{
    const csu_layout& L = x->L;
    const int nc = L.nc, nf = L.nf, nb = L.nb;
    const size_t c4 = (size_t)4 * nc;
    Mesh& m = x->mesh;
    auto up = [&](const void* dst, const void* src, size_t bytes) -> cudaError_t {
        if (bytes == 0) return cudaSuccess;
        return cudaMemcpy(const_cast<void*>(dst), src, bytes, cudaMemcpyHostToDevice);
    };
    std::vector<int2> fe(nf);
    std::vector<double2> fn(nf), r0(nf), r1(nf), bn(nb), fd(nf), bd(nb), bun(nb);
    for (int f = 0; f < nf; f++) {
        fe[f] = make_int2(L.fe0[f], L.fe1[f]);
        fd[f] = make_double2(L.fdx[f], L.fdy[f]);
        fn[f] = make_double2(L.fdsx[f], L.fdsy[f]);
        r0[f] = make_double2(L.r0x[f], L.r0y[f]);
        r1[f] = make_double2(L.r1x[f], L.r1y[f]);
    }
    for (int b = 0; b < nb; b++) {
        bn[b] = make_double2(L.bdsx[b], L.bdsy[b]);
        bd[b] = make_double2(L.bdx[b], L.bdy[b]);
        bun[b] = make_double2(L.bunx[b], L.buny[b]);
    }
    // walls in reference order (solverCalcCoeff3 sums over wall markers, marker-major), per solve
    std::vector<int> rank(nb > 0 ? nb : 1, -1);
    {
        int r = 0;
        for (int k = 0; k < x->nsolve; k++) {
            int b0 = x->bface0[k], nbk = (k + 1 < x->nsolve ? x->bface0[k + 1] : nb) - b0;
            std::vector<int> by_old(nbk, -1);
            for (int b = 0; b < nbk; b++) by_old[L.bold[b0 + b]] = b0 + b;
            x->prms[k].wall0 = r;
            for (int o = 0; o < nbk; o++) {
                int b = by_old[o];
                if (L.bflag[b] == CSU_BC_WALL || L.bflag[b] == CSU_BC_WALLT) rank[b] = r++;
            }
            x->prms[k].nwall = r - x->prms[k].wall0;
        }
        x->nwall = r;
    }
    if (x->nsolve > 1) {
        int nblk = (nc + BLOCK - 1) / BLOCK;
        std::vector<int> bs(nblk, 0), cs(nc, 0);
        for (int k = 0; k < x->nsolve; k++) {
            int c1 = k + 1 < x->nsolve ? x->cell0[k + 1] : nc;
            for (int c = x->cell0[k]; c < c1; c++) cs[c] = k;
            for (int b = x->cell0[k] / BLOCK; b < (c1 + BLOCK - 1) / BLOCK; b++) bs[b] = k;
        }
        CK(up(x->st.bsolve, bs.data(), sizeof(int) * nblk));
        CK(up(x->st.csolve, cs.data(), sizeof(int) * nc));
    }
    CK(up(m.npts, L.npts, sizeof(int) * nc));
    CK(up(m.nint, L.nint, sizeof(int) * nc));
    CK(up(m.nslot, L.nslot, sizeof(int) * nc));
    CK(up(m.nei, L.nei, sizeof(int) * c4));
    CK(up(m.wx, L.wx, sizeof(double) * c4));
    CK(up(m.wy, L.wy, sizeof(double) * c4));
    CK(up(m.ldx, L.ldx, sizeof(double) * c4));
    CK(up(m.ldy, L.ldy, sizeof(double) * c4));
    CK(up(m.lm, L.lm, sizeof(unsigned long long) * c4));
    CK(up(m.les, L.les, sizeof(int) * c4));
    CK(up(m.lrv, L.lrv, sizeof(unsigned long long) * nc));
    CK(up(m.lq, L.lq, sizeof(double2) * c4));
    CK(up(m.ex, L.ex, sizeof(double) * c4));
    CK(up(m.ey, L.ey, sizeof(double) * c4));
    CK(up(m.fslot, L.fslot, sizeof(int) * c4));
    CK(up(m.fnb, L.fnb, sizeof(int) * c4));
    CK(up(x->d_n2o, L.cell_new2old, sizeof(int) * nc));
    CK(up(m.omega, L.omega, sizeof(double) * nc));
    CK(up(m.sxh, L.sxh, sizeof(double) * nc));
    CK(up(m.syh, L.syh, sizeof(double) * nc));
    if (m.wall_d) CK(up(m.wall_d, L.wall_d, sizeof(double) * nc));
    CK(up(m.dslat, L.dslat, sizeof(double) * nc));
    CK(up(m.fe, fe.data(), sizeof(int2) * nf));
    CK(up(m.fn, fn.data(), sizeof(double2) * nf));
    CK(up(m.fds, L.fds, sizeof(double) * nf));
    CK(up(m.r0, r0.data(), sizeof(double2) * nf));
    CK(up(m.r1, r1.data(), sizeof(double2) * nf));
    CK(up(m.fd, fd.data(), sizeof(double2) * nf));
    CK(up(m.fL, L.fdist, sizeof(double) * nf));
    CK(up(m.bown, L.bown, sizeof(int) * nb));
    CK(up(m.bflag, L.bflag, sizeof(int) * nb));
    CK(up(m.bold, L.bold, sizeof(int) * nb));
    CK(up(m.bn, bn.data(), sizeof(double2) * nb));
    CK(up(m.bds, L.bds, sizeof(double) * nb));
    CK(up(m.bd, bd.data(), sizeof(double2) * nb));
    CK(up(m.bL, L.bL, sizeof(double) * nb));
    CK(up(m.bun, bun.data(), sizeof(double2) * nb));
    CK(up(m.bds2, L.bds2, sizeof(double) * nb));
    CK(up(m.color, L.color, sizeof(int) * nc));
    CK(up(m.color_cells, L.color_cells, sizeof(int) * nc));
    CK(up(x->d_wall_rank, rank.data(), sizeof(int) * nb));
    return CSU_OK;
}

static void fill_params_from(const csu_config& c, const csu_layout& L, Prm& p)
{
    memset(&p, 0, sizeof(p));
    p.gas.gamma = c.gamma;
    p.gas.R = c.gas_r;
    p.gas.Cp = c.gamma * c.gas_r / (c.gamma - 1); // gaspropInit (gasprop.c:14-37)
    p.gas.Cv = p.gas.Cp - c.gas_r;
    p.gas.tp = c.tp;
    p.nc = L.nc;
    p.nf = L.nf;
    p.nb = L.nb;
    p.order = c.order;
    p.scheme = c.flux;
    p.laminar = c.laminar;
    p.sa = c.sa;
    p.sst = c.sst;
    p.axi = c.axisymmetric;
    p.turb1order = c.turb1order;
    p.limiter_type = c.limiter_type;
    p.stages = c.stages;
    p.dt_local_n = c.dt_local_n;
    p.tube = c.tube;
    p.n_linear = c.n_linear;
    p.lim_k = c.limiter_k;
    p.vol_max = L.vol_max;
    p.e_fix = c.e_fix;
    p.r_lim = c.r_lim;
    p.p_out = c.p_out;
    p.t_wall = c.t_wall;
    p.pr = c.pr;
    p.pr_t = c.pr_t;
    p.w_imp = c.w_imp;
    p.cfl = c.cfl;
    p.sigma = 0.5 * c.stages;
    p.mach_inf = c.mach_inf;
    p.sref = c.sref;
    for (int k = 0; k < 7; k++) p.pin[k] = c.pin[k];
    // limiterUpdate type 0 (limiter.c:49-59)
    p.pref20[0] = c.pin[0] * c.pin[0];
    p.pref20[1] = c.pin[1] * c.pin[1] + c.pin[2] * c.pin[2];
    p.pref20[2] = p.pref20[1];
    p.pref20[3] = c.pin[3] * c.pin[3];
    for (int k = 4; k < c.nvar; k++) p.pref20[k] = c.pin[k + 1] * c.pin[k + 1];
    // solverCalcCoeff3 (solver.c:1348-1352)
    p.p_inf = c.pin[3];
    p.q_inf = 0.5 * c.pin[0] * (c.pin[1] * c.pin[1] + c.pin[2] * c.pin[2]);
    p.sst_b1 = 0.075;
    {
        // sstInit (sst.c:18-39)
        SstK& k = p.sst_k;
        k.sk1 = 0.85; k.so1 = 0.5; k.b1 = 0.075; k.sk2 = 1.0; k.so2 = 0.856; k.b2 = 0.0828; k.bs = 0.09; k.a1 = 0.31;
        double kap = 0.41;
        k.g1 = k.b1 / k.bs - k.so1 * kap * kap / sqrt(k.bs);
        k.g2 = k.b2 / k.bs - k.so2 * kap * kap / sqrt(k.bs);
        k.o_wall_factor = c.o_wall_factor;
        k.trans = c.sst_trans ? 1 : 0;
    }
    p.o_wall_factor = c.o_wall_factor;
    p.tmax = 0;
    // exact x87 gradients unless CSU_LSQ_FAST=1 (FP64 weights: faster, last-bit differences)
    // least squares: certified double-double with x87 fallback (default, bit-exact); CSU_LSQ=x87 runs the
    // x87 model on every component; CSU_LSQ=weights (or CSU_LSQ_FAST=1) precomputed FP64 weights
    const char* fast = getenv("CSU_LSQ_FAST");
    const char* lsq = getenv("CSU_LSQ");
    p.lsq_exact = 2;
    if (lsq && !strcmp(lsq, "x87")) p.lsq_exact = 1;
    if ((lsq && !strcmp(lsq, "weights")) || (fast && fast[0] == '1')) p.lsq_exact = 0;
    p.visc = (c.laminar || c.sa || c.sst) ? 1 : 0;
    p.visc_blazek = c.visc_blazek;
    p.sa_cc = c.sa_cc ? 1 : 0;
    p.conv_tol = c.conv_drop;
    p.iter_cap = c.iter_cap;
    p.lim_func = c.limiter_func;
    if (c.gradient == 1) p.lsq_exact = 0; // Green-Gauss weights replace the least-squares weights
    p.blk32 = c.implicit_fp32;
    p.sa_isrc = c.sa && c.time_scheme == CSU_TS_DPLUR && c.sa_implicit_source;
    p.defer_fin = c.time_scheme == CSU_TS_DPLUR;
    p.mit_early = c.sa && c.time_scheme == CSU_TS_DPLUR;
    p.implicit_local_dt = c.implicit_local_dt;
    p.cfl_ramp_iters = c.cfl_ramp_iters;
    p.cfl_max = c.cfl_ramp_iters > 0 ? c.cfl_max : c.cfl;
}

static double* hist_of(csu_ctx* x, int k)
{
    return x->hist ? x->hist + (size_t)k * x->hist_cap * (x->nv + 4) : nullptr;
}

static int reset_scalars(csu_ctx* x, int it0)
{
    std::vector<Scalars> hs(x->nsolve);
    for (int k = 0; k < x->nsolve; k++) {
        Scalars& h = hs[k];
        memset(&h, 0, sizeof(h));
        h.dtmin_bits = 0x7ff0000000000000ULL;
        h.dt_local = x->cfg.dt_local;
        h.iter = it0;
        h.fresh = 1;
        h.hist = hist_of(x, k);
        h.hist_cap = x->hist_cap;
    }
    CK(cudaStreamSynchronize(x->stream));
    CK(cudaMemcpy(x->st.sc, hs.data(), sizeof(Scalars) * hs.size(), cudaMemcpyHostToDevice));
    return CSU_OK;
}

// scalars of solves [0, n)
static int read_scalars_n(csu_ctx* x, Scalars* h, int n)
{
    CK(cudaStreamSynchronize(x->stream));
    CK(cudaMemcpy(h, x->st.sc, sizeof(Scalars) * n, cudaMemcpyDeviceToHost));
    return CSU_OK;
}

static int read_scalars(csu_ctx* x, Scalars* h)
{
    return read_scalars_n(x, h, 1);
}

static int write_scalars_n(csu_ctx* x, const Scalars* h, int n)
{
    CK(cudaStreamSynchronize(x->stream));
    CK(cudaMemcpy(x->st.sc, h, sizeof(Scalars) * n, cudaMemcpyHostToDevice));
    return CSU_OK;
}

// host parameters to the device copy (after any change of prms)
static int upload_prm(csu_ctx* x)
{
    CK(cudaStreamSynchronize(x->stream));
    CK(cudaMemcpy(x->d_prm, x->prms.data(), sizeof(Prm) * x->nsolve, cudaMemcpyHostToDevice));
    return CSU_OK;
}

// The settings this engine runs (csu_create's checks); sets the model (0 Euler/laminar, 1 SA, 2 SST).
static int validate_config(const char* who, const csu_config* cfg, int* model_out, int* nv_out)
{
    int model = cfg->sst ? 2 : (cfg->sa ? 1 : 0);
    int nv = model == 0 ? 4 : (model == 1 ? 5 : 6);
    if (cfg->nvar != nv) {
        csu_set_error("%s: nvar %d does not match the turbulence model", who, cfg->nvar);
        return CSU_ERR_INPUT;
    }
    if (model == 2 && cfg->flux == CSU_FLUX_ROE) {
        csu_set_error("%s: SST with the AUSM family only (the reference has no Roe branch for SST)", who);
        return CSU_ERR_UNSUPPORTED;
    }
    if (cfg->time_scheme == CSU_TS_RK && !(cfg->stages >= 1 && cfg->stages <= 5)) {
        csu_set_error("%s: RK with %d stages (1, 3, 4, 5 as the reference; 2 as an extension)", who, cfg->stages);
        return CSU_ERR_UNSUPPORTED;
    }
    if (cfg->limiter_func != 0 && cfg->limiter_func != 1) {
        csu_set_error("%s: limiterFunc %d (0 Venkatakrishnan, 1 Barth-Jespersen)", who, cfg->limiter_func);
        return CSU_ERR_INPUT;
    }
    if (cfg->gradient != 0 && (cfg->gradient != 1 || cfg->axisymmetric)) {
        csu_set_error("%s: gradient %d%s (0 least squares, 1 Green-Gauss, planar only)", who, cfg->gradient,
                      cfg->axisymmetric ? " with axisymmetry" : "");
        return CSU_ERR_INPUT;
    }
    if (cfg->time_scheme == CSU_TS_DPLUR && (cfg->n_linear < 1 || cfg->n_linear > MAX_SWEEPS)) {
        csu_set_error("%s: Nlinear must be in [1, %d]", who, MAX_SWEEPS);
        return CSU_ERR_UNSUPPORTED;
    }
    if (cfg->order != 1 && cfg->order != 2) {
        csu_set_error("%s: order must be 1 or 2", who);
        return CSU_ERR_INPUT;
    }
    if (cfg->limiter_type != 0 && cfg->limiter_type != 1) {
        csu_set_error("%s: limiter type %d (the reference has types 0 and 1)", who, cfg->limiter_type);
        return CSU_ERR_INPUT;
    }
    if (cfg->limiter_type == 1 && model == 2) {
        csu_set_error("%s: limiter type 1 with SST (the reference writes past its 5-entry Pmin/Pmax, "
                      "limiter.c:37-38)", who);
        return CSU_ERR_UNSUPPORTED;
    }
    *model_out = model;
    *nv_out = nv;
    return CSU_OK;
}

// Allocates and fills the device side of x (x->L, x->prms and the pack offsets set by the caller).
static int max_nint(const csu_layout& L)
{
    int m = 1;
    for (int c = 0; c < L.nc; c++) m = std::max(m, L.nint[c]);
    return m;
}

static void plan_l2_window(csu_ctx* x);

static int ctx_setup(csu_ctx* x)
{
    int st;
    x->mesh.nc = x->L.nc;
    x->mesh.nf = x->L.nf;
    x->mesh.nb = x->L.nb;
    // size, allocate once, carve
    Arena a;
    plan(x, a);
    size_t bytes = a.size;
    cudaError_t e;
    e = cudaGetDevice(&x->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&x->sm_count, cudaDevAttrMultiProcessorCount, x->device);
    if (e != cudaSuccess) return cuda_fail(e, "device query");
    if (x->is_pack) {
        size_t got = 0;
        e = pack_arena_take(x->device, bytes, &x->arena.base, &got);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(pack arena)");
        x->arena.size = got;
    } else {
        e = cudaMalloc((void**)&x->arena.base, bytes);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(context arena)");
        x->arena.size = bytes;
    }
    x->arena.used = 0;
    plan(x, x->arena);
    e = cudaMemset(x->arena.base, 0, bytes);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&x->own_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&x->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x->ev_grad, cudaEventDisableTiming);
    x->stream = x->own_stream;
    if (e != cudaSuccess) return cuda_fail(e, "context setup");
    x->gb_c = (x->L.nc + BLOCK - 1) / BLOCK;
    if (x->L.nint) x->max_ni = max_nint(x->L); // packs set it from their solves
    plan_l2_window(x);
    if (!x->is_pack && (st = upload_mesh(x))) return st; // packs: pack_build fills the mesh rows
    x->prm = x->prms[0];
    if ((st = upload_prm(x)) || (st = reset_scalars(x, 0))) return st;
    switch (x->cfg.stages) {
    case 1: x->rk = RK1; break;
    case 2: x->rk = RK2; break;
    case 3: x->rk = RK3; break;
    case 4: x->rk = RK4; break;
    default: x->rk = RK5; break;
    }
    return CSU_OK;
}

extern "C" int csu_create(const csu_mesh_desc* md, const csu_config* cfg, csu_ctx** out)
{
    *out = nullptr;
    if (!md || !cfg || md->n_cells <= 0) {
        csu_set_error("csu_create: empty mesh or missing config");
        return CSU_ERR_INPUT;
    }
    int model, nv;
    int st = validate_config("csu_create", cfg, &model, &nv);
    if (st) return st;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        csu_set_error("csu_create: no CUDA device");
        return CSU_ERR_NO_DEVICE;
    }
    csu_ctx* x = new csu_ctx();
    x->model = model;
    x->nv = nv;
    x->cfg = *cfg;
    st = csu_layout_build(md, cfg->axisymmetric, &x->L);
    if (!st && cfg->gradient == 1) st = csu_layout_green_gauss(&x->L);
    {
        // CSU_LUSGS_ORDER=sequential: LU-SGS in the reference's cell order (one cell per colour), for checks
        const char* ord = getenv("CSU_LUSGS_ORDER");
        if (!st && ord && strcmp(ord, "sequential") == 0) st = csu_layout_sequential_colors(&x->L);
    }
    if (st) {
        delete x;
        csu_set_error("csu_create: mesh layout failed (a cell with more than four faces?)");
        return st;
    }
    x->cell0 = {0};
    x->face0 = {0};
    x->bface0 = {0};
    x->ncs = {x->L.nc};
    x->prms.resize(1);
    fill_params_from(x->cfg, x->L, x->prms[0]);
    x->prms[0].cell0 = 0;
    x->prms[0].blk0 = 0;
    x->prms[0].nblk = (x->L.nc + BLOCK - 1) / BLOCK;
    if ((st = ctx_setup(x))) {
        csu_destroy(x);
        return st;
    }
    *out = x;
    return CSU_OK;
}

extern "C" void csu_destroy(csu_ctx* x)
{
    if (!x) return;
    if (x->is_pack && x->arena.base) {
        // the arena goes back for the next pack to reuse: this pack's work must be done first (while its
        // streams still exist)
        if (x->stream) cudaStreamSynchronize(x->stream);
        if (x->side) cudaStreamSynchronize(x->side);
    }
    drop_graphs(x);
    if (x->hist) cudaFree(x->hist);
    if (x->h_sc) cudaFreeHost(x->h_sc);
    if (x->h_hist) cudaFreeHost(x->h_hist);
    if (x->h_flags) cudaFreeHost(x->h_flags);
    if (x->h_snap) cudaFreeHost(x->h_snap);
    for (cudaEvent_t e : x->ev_poll)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : x->ev) cudaEventDestroy(e);
    if (x->own_stream) cudaStreamDestroy(x->own_stream);
    if (x->side) cudaStreamDestroy(x->side);
    if (x->ev_fork) cudaEventDestroy(x->ev_fork);
    if (x->ev_join) cudaEventDestroy(x->ev_join);
    if (x->ev_grad) cudaEventDestroy(x->ev_grad);
    if (x->arena.base) {
        if (x->is_pack) {
            pack_arena_give(x->device, x->arena.base, x->arena.size);
        } else {
            cudaFree(x->arena.base);
        }
    }
    csu_layout_free(&x->L);
    delete x;
}

static void release_copy_jobs();

// Frees the pack arenas kept for reuse (the serving layer calls it when it shuts down).
extern "C" void csu_pack_arena_release(void)
{
    {
        std::lock_guard<std::mutex> lk(g_arena_mu);
        for (const CachedArena& a : g_arena_cache) cudaFree(a.base);
        g_arena_cache.clear();
    }
    release_copy_jobs();
}

// State of solve k in its reference order ([var][cell], nvar x its cell count), to or from the device.
// The state of a one-solve context between reference order ([var][cell], in the staging buffer) and the
// renumbered device layout (U4 + SoA scalars); k_state_in also marks the state as set from outside.
__global__ void k_state_in(State s, const double* stage, const int* n2o, int nc, int nv)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) s.sc[0].fresh = 1;
    if (c >= nc) return;
    const int q = n2o[c];
    s.U4[c] = make_double4(stage[q], stage[(size_t)nc + q], stage[(size_t)2 * nc + q], stage[(size_t)3 * nc + q]);
    for (int r = 4; r < nv; r++) s.Ux[(size_t)(r - 4) * nc + c] = stage[(size_t)r * nc + q];
}

// DPLUR one-solve contexts: the state goes in with its primitives (U := clamp(U), W = primitives, as the
// prologue's k_prim computes them) ...
template <int MODEL>
__global__ void __launch_bounds__(BLOCK) k_state_in_prim(const Prm* __restrict__ P, State s, const double* stage,
                                                         const int* n2o, int nc)
{
    constexpr int NV = Model<MODEL>::NV, NP = Model<MODEL>::NP;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int q = n2o[c];
    double U[NV], W[NP];
#pragma unroll
    for (int k = 0; k < NV; k++) U[k] = stage[(size_t)k * nc + q];
    clamp_prim<MODEL>(P[0], U, W);
    storeU<MODEL>(s, nc, c, U);
    storeP<MODEL>(s, nc, c, W);
}

// ... and fresh scalars, as reset_scalars and the prologue's k_finalize leave them for DPLUR (the step
// size the prologue computes is an RK quantity), so that the next call goes straight to its iterations
__global__ void k_scalars_fresh(Scalars* sc, double* hist, int hist_cap, int dt_local)
{
    if (threadIdx.x != 0) return;
    Scalars h;
    memset(&h, 0, sizeof(h));
    h.dtmin_bits = 0x7ff0000000000000ULL;
    h.dt_local = dt_local;
    h.hist = hist;
    h.hist_cap = hist_cap;
    *sc = h;
}

__global__ void k_state_out(State s, double* stage, const int* n2o, int nc, int nv)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int q = n2o[c];
    const double4 u = s.U4[c];
    stage[q] = u.x;
    stage[(size_t)nc + q] = u.y;
    stage[(size_t)2 * nc + q] = u.z;
    stage[(size_t)3 * nc + q] = u.w;
    for (int r = 4; r < nv; r++) stage[(size_t)r * nc + q] = s.Ux[(size_t)(r - 4) * nc + c];
}

static int solve_state_io(csu_ctx* x, int k, double* U, bool put)
{
    if (!x->is_pack) {
        // one copy of the caller's array (a DMA when it is pinned) and the renumbering on the device
        const int nc = x->L.nc, nv = x->nv;
        const size_t bytes = sizeof(double) * (size_t)nv * nc;
        const int g = (nc + BLOCK - 1) / BLOCK;
        if (put) {
            CK(cudaMemcpyAsync(x->d_stage, U, bytes, cudaMemcpyHostToDevice, x->stream));
            const bool dplur = x->cfg.time_scheme == CSU_TS_DPLUR;
            if (dplur) {
                // primitives and fresh scalars on the device: the next csu_iterate needs no host round trip
                // for the scalars and no prologue kernels
                switch (x->model) {
                case 0: k_state_in_prim<0><<<g, BLOCK, 0, x->stream>>>(x->d_prm, x->st, x->d_stage, x->d_n2o, nc); break;
                case 1: k_state_in_prim<1><<<g, BLOCK, 0, x->stream>>>(x->d_prm, x->st, x->d_stage, x->d_n2o, nc); break;
                default: k_state_in_prim<2><<<g, BLOCK, 0, x->stream>>>(x->d_prm, x->st, x->d_stage, x->d_n2o, nc); break;
                }
                k_scalars_fresh<<<1, 32, 0, x->stream>>>(x->st.sc, hist_of(x, 0), x->hist_cap, x->cfg.dt_local);
            } else {
                k_state_in<<<g, BLOCK, 0, x->stream>>>(x->st, x->d_stage, x->d_n2o, nc, nv);
            }
            CK(cudaGetLastError());
            CK(cudaStreamSynchronize(x->stream)); // the caller may reuse U on return
            x->prepared = dplur ? 1 : 0;
            return CSU_OK;
        }
        k_state_out<<<g, BLOCK, 0, x->stream>>>(x->st, x->d_stage, x->d_n2o, nc, nv);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(U, x->d_stage, bytes, cudaMemcpyDeviceToHost, x->stream));
        CK(cudaStreamSynchronize(x->stream));
        return CSU_OK;
    }
    const int nck = x->ncs[k], o = x->cell0[k], NC = x->L.nc, nv = x->nv;
    // a pack keeps each solve's renumbering (its concatenated layout has none); a one-solve context its own
    const int* n2o = x->is_pack ? x->n2o[k].data() : x->L.cell_new2old;
    std::vector<double4> u4(nck);
    std::vector<double> ux((size_t)(nv - 4) * nck + 1);
    if (put) {
        for (int c = 0; c < nck; c++) {
            int q = n2o[c];
            u4[c] = make_double4(U[q], U[(size_t)nck + q], U[(size_t)2 * nck + q], U[(size_t)3 * nck + q]);
            for (int r = 4; r < nv; r++) ux[(size_t)(r - 4) * nck + c] = U[(size_t)r * nck + q];
        }
        CK(cudaStreamSynchronize(x->stream));
        CK(cudaMemcpy(x->st.U4 + o, u4.data(), sizeof(double4) * nck, cudaMemcpyHostToDevice));
        {
            Scalars h;
            CK(cudaMemcpy(&h, x->st.sc + k, sizeof(Scalars), cudaMemcpyDeviceToHost));
            h.fresh = 1;
            CK(cudaMemcpy(x->st.sc + k, &h, sizeof(Scalars), cudaMemcpyHostToDevice));
        }
        for (int r = 4; r < nv; r++)
            CK(cudaMemcpy(x->st.Ux + (size_t)(r - 4) * NC + o, ux.data() + (size_t)(r - 4) * nck,
                          sizeof(double) * nck, cudaMemcpyHostToDevice));
        x->prepared = 0;
        return CSU_OK;
    }
    CK(cudaStreamSynchronize(x->stream));
    CK(cudaMemcpy(u4.data(), x->st.U4 + o, sizeof(double4) * nck, cudaMemcpyDeviceToHost));
    for (int r = 4; r < nv; r++)
        CK(cudaMemcpy(ux.data() + (size_t)(r - 4) * nck, x->st.Ux + (size_t)(r - 4) * NC + o, sizeof(double) * nck,
                      cudaMemcpyDeviceToHost));
    for (int c = 0; c < nck; c++) {
        int q = n2o[c];
        U[q] = u4[c].x;
        U[(size_t)nck + q] = u4[c].y;
        U[(size_t)2 * nck + q] = u4[c].z;
        U[(size_t)3 * nck + q] = u4[c].w;
        for (int r = 4; r < nv; r++) U[(size_t)r * nck + q] = ux[(size_t)(r - 4) * nck + c];
    }
    return CSU_OK;
}

extern "C" int csu_set_state(csu_ctx* x, const double* U)
{
    if (!x || !U) return CSU_ERR_INPUT;
    if (x->is_pack) {
        csu_set_error("csu_set_state: a pack holds its solves separately (use csu_pack_set_state)");
        return CSU_ERR_STATE;
    }
    return solve_state_io(x, 0, const_cast<double*>(U), true);
}

extern "C" int csu_get_state(csu_ctx* x, double* U)
{
    if (!x || !U) return CSU_ERR_INPUT;
    if (x->is_pack) {
        csu_set_error("csu_get_state: a pack holds its solves separately (use csu_pack_get_state)");
        return CSU_ERR_STATE;
    }
    return solve_state_io(x, 0, U, false);
}

extern "C" int csu_set_state_rows(csu_ctx* x, const double* const* U)
{
    const int nc = x->L.nc, nv = x->nv;
    std::vector<double> flat((size_t)nv * nc);
    for (int k = 0; k < nv; k++) memcpy(flat.data() + (size_t)k * nc, U[k], sizeof(double) * nc);
    return csu_set_state(x, flat.data());
}

extern "C" int csu_get_state_rows(csu_ctx* x, double* const* U)
{
    const int nc = x->L.nc, nv = x->nv;
    std::vector<double> flat((size_t)nv * nc);
    int st = csu_get_state(x, flat.data());
    if (st) return st;
    for (int k = 0; k < nv; k++) memcpy(U[k], flat.data() + (size_t)k * nc, sizeof(double) * nc);
    return CSU_OK;
}

// ---------------------------------------------------------------------------------------------- launches

template <int MODEL, bool DBG>
static void launch_grad_lsq(csu_ctx* x)
{
    switch (x->prm.lsq_exact) {
    case 0: k_grad<MODEL, DBG, 0><<<x->gb_c, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st); break;
    case 1: k_grad<MODEL, DBG, 1><<<x->gb_c, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st); break;
    default:
        // the rare components left undecided by the FP64 paths are finished by k_grad_fix: grid-stride over a
        // list whose length only the device knows, two blocks per SM (strongly stretched cells, as beside a
        // wall at y+ < 1, leave thousands of entries; an empty list costs one short launch)
        k_grad<MODEL, DBG, 2><<<x->gb_c, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st);
        k_grad_fix<MODEL><<<2 * x->sm_count, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st);
        x->launches++;
        break;
    }
}

template <int MODEL>
static void launch_grad(csu_ctx* x, bool dbg)
{
    if (x->cfg.order == 2 && x->cfg.limiter_type == 1) {
        k_minmax_init<<<x->nsolve, 32, 0, x->stream>>>(x->st);
        k_minmax<MODEL><<<x->gb_c, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st);
        x->launches += 2;
    }
    if (dbg) launch_grad_lsq<MODEL, true>(x);
    else launch_grad_lsq<MODEL, false>(x);
    x->launches++;
    tmark(x, KGRAD);
}

// faces in blocks of FB threads
template <int MODEL, int FB>
static void launch_flux_fb(csu_ctx* x, int coef)
{
    const int gi = (x->L.nf + FB - 1) / FB, gb = (x->L.nb + FB - 1) / FB;
    k_flux<MODEL, FB><<<gi + gb, FB, 0, x->stream>>>(x->d_prm, x->mesh, x->st, gi, x->d_wall_rank, coef);
}

// blocks of 128 faces whose cells are staged through a 256-cell shared-memory window (k_flux_st)
template <int MODEL>
static void launch_flux_staged(csu_ctx* x, int coef)
{
    constexpr int FB = 128;
    const int gi = (x->L.nf + FB - 1) / FB, gb = (x->L.nb + FB - 1) / FB;
    k_flux_st<MODEL, FB, 256><<<gi + gb, FB, 0, x->stream>>>(x->d_prm, x->mesh, x->st, gi, x->d_wall_rank, coef);
}

template <int MODEL>
static void launch_flux(csu_ctx* x, int coef)
{
    switch (x->flux_fb) {
    case 32: launch_flux_fb<MODEL, 32>(x, coef); break;
    case 128: launch_flux_staged<MODEL>(x, coef); break;
    default: launch_flux_fb<MODEL, 64>(x, coef); break;
    }
    x->launches++;
    tmark(x, KFLUX);
}

template <int MODEL>
static void launch_finalize(csu_ctx* x, int mode, int bsel = 0, cudaStream_t stream = nullptr)
{
    // the first DPLUR sweep writes one partial row per warp; the other kernels one per cell block
    const int ppb = x->cfg.time_scheme == CSU_TS_DPLUR && mode == 1 ? BLOCK / 32 : 1;
    k_finalize<MODEL><<<x->nsolve, BLOCK, 0, stream ? stream : x->stream>>>(x->d_prm, x->mesh, x->st, mode, ppb,
                                                                            bsel);
    x->launches++;
    tmark(x, KFIN);
}

template <int MODEL>
static void launch_prologue(csu_ctx* x)
{
    int rk = x->cfg.time_scheme == CSU_TS_RK;
    k_prim<MODEL><<<x->gb_c, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st, rk, 1);
    x->launches++;
    tmark(x, KPRIM);
    launch_finalize<MODEL>(x, 2);
}

// DPLUR blocks of this iteration on the side stream, forked from the engine stream at ev_fork (recorded by
// the caller before the kernels they run beside, which are launched first so that their blocks are dispatched
// first and k_blocks fills the SMs their last wave leaves idle); the first sweep joins. Timed runs keep them
// on the engine stream, so each kernel kind's events bracket it alone.
// The implicit diagonal and step (k_impl without R) go on the same side stream. SA first computes the face
// eddy viscosity the blocks and the diagonal use (k_face_mit); with saImplicitSource its diagonal also needs
// the gradients, so k_impl waits for ev_grad (recorded after them).
template <int MODEL>
static void launch_blocks(csu_ctx* x)
{
    cudaStream_t s = x->stream;
    if (!x->timing) {
        cudaStreamWaitEvent(x->side, x->ev_fork, 0);
        s = x->side;
    }
    if (MODEL == 1 && x->prm.mit_early) {
        k_face_mit<<<(x->L.nf + BLOCK - 1) / BLOCK, BLOCK, 0, s>>>(x->d_prm, x->mesh, x->st);
        x->launches++;
    }
    k_blocks<MODEL><<<x->max_ni * x->gb_c, BLOCK, 0, s>>>(x->d_prm, x->mesh, x->st, x->gb_c);
    x->launches++;
    if (x->timing) tmark(x, KBLK);
    if (x->fin_pending) {
        // the previous iteration's k_finalize, after the blocks (which need no scalar it writes) and before
        // the diagonal (whose step minimum it resets)
        launch_finalize<MODEL>(x, 1, x->fin_bsel, s);
        x->fin_pending = false;
    }
    if (MODEL == 1 && x->prm.sa_isrc && !x->timing) cudaStreamWaitEvent(x->side, x->ev_grad, 0);
    k_impl<MODEL, false><<<x->gb_c, BLOCK, 0, s>>>(x->d_prm, x->mesh, x->st);
    x->launches++;
    if (x->timing) tmark(x, KIMPL);
    else cudaEventRecord(x->ev_join, x->side);
}

template <int MODEL, int SB>
static void launch_sweep_sb(csu_ctx* x, int m, int n)
{
    if (m == 0) {
        auto* k = x->cfg.implicit_fp32
                      ? (m == n - 1 ? k_sweep<MODEL, true, true, SB, true> : k_sweep<MODEL, false, true, SB, true>)
                      : (m == n - 1 ? k_sweep<MODEL, true, true, SB, false> : k_sweep<MODEL, false, true, SB, false>);
        k<<<x->gb_c * (BLOCK / SB), SB, 0, x->stream>>>(x->d_prm, x->mesh, x->st, m, x->xcur);
    } else {
        auto* k = x->cfg.implicit_fp32
                      ? (m == n - 1 ? k_sweep<MODEL, true, false, SB, true> : k_sweep<MODEL, false, false, SB, true>)
                      : (m == n - 1 ? k_sweep<MODEL, true, false, SB, false> : k_sweep<MODEL, false, false, SB, false>);
        k<<<x->gb_c * (BLOCK / SB), SB, 0, x->stream>>>(x->d_prm, x->mesh, x->st, m, x->xcur);
    }
}

template <int MODEL>
static void launch_sweep(csu_ctx* x, int m, int n)
{
    switch (x->sweep_sb) {
    case 64: launch_sweep_sb<MODEL, 64>(x, m, n); break;
    case 256: launch_sweep_sb<MODEL, 256>(x, m, n); break;
    default: launch_sweep_sb<MODEL, 128>(x, m, n); break;
    }
    x->launches++;
    tmark(x, KSWEEP);
    x->xcur ^= 1;
}

// csu_iterate_views: the primitives and gradients the residual evaluation just launched works on, copied in
// stream order to pinned host memory (device layout; unpacked after the iteration)
static void snapshot_views(csu_ctx* x)
{
    if (!x->snap || !x->h_snap) return;
    const size_t nc = x->L.nc, nx = x->nv - 4;
    double* h = x->h_snap;
    auto cp = [&](const void* src, size_t n) {
        if (n) cudaMemcpyAsync(h, src, sizeof(double) * n, cudaMemcpyDeviceToHost, x->stream);
        h += n;
    };
    cp(x->st.W4, 4 * nc);
    cp(x->st.WT, nc);
    cp(x->st.Wx, nx * nc);
    cp(x->st.G4x, 4 * nc);
    cp(x->st.G4y, 4 * nc);
    cp(x->st.Gxx, nx * nc);
    cp(x->st.Gxy, nx * nc);
}

// one iteration of the steady loop body (solver.c:1866-1906)
template <int MODEL>
static void launch_iteration(csu_ctx* x)
{
    const csu_config& c = x->cfg;
    if (c.time_scheme == CSU_TS_RK) {
        for (int sgi = 0; sgi < c.stages; sgi++) {
            bool last = sgi == c.stages - 1;
            if (c.order == 2 || x->prm.visc) launch_grad<MODEL>(x, false);
            if (last) snapshot_views(x);
            launch_flux<MODEL>(x, last ? 1 : 0);
            if (last) k_rk<MODEL, true><<<x->gb_c, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st, x->rk[sgi]);
            else k_rk<MODEL, false><<<x->gb_c, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st, x->rk[sgi]);
            x->launches++;
            tmark(x, KRK);
        }
        launch_finalize<MODEL>(x, 0);
    } else if (c.time_scheme == CSU_TS_LUSGS) {
        if (c.order == 2 || x->prm.visc) launch_grad<MODEL>(x, false);
        snapshot_views(x);
        launch_flux<MODEL>(x, 1);
        k_impl<MODEL, true><<<x->gb_c, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st);
        x->launches++;
        tmark(x, KIMPL);
        const int K = x->L.ncolors;
        for (int pass = 0; pass < 2; pass++)
            for (int q = 0; q < K; q++) {
                int col = pass == 0 ? q : K - 1 - q;
                int start = x->L.color_start[col], count = x->L.color_start[col + 1] - start;
                if (count == 0) continue;
                int g = (count + BLOCK - 1) / BLOCK;
                if (pass == 0)
                    k_lusgs<MODEL, true><<<g, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st, x->mesh.color,
                                                                     x->mesh.color_cells, col, start, count);
                else
                    k_lusgs<MODEL, false><<<g, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st, x->mesh.color,
                                                                      x->mesh.color_cells, col, start, count);
                x->launches++;
                tmark(x, KSWEEP);
            }
        k_update<MODEL><<<x->gb_c, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st);
        x->launches++;
        tmark(x, KPRIM);
        launch_finalize<MODEL>(x, 1);
    } else {
        // the SST blocks and diagonal need the face eddy viscosity of k_flux (and the gradients, for the
        // source Jacobians); the SA ones only k_face_mit's, the Euler/laminar ones the iteration's start state
        constexpr bool early = MODEL <= 1;
        const bool grad = c.order == 2 || x->prm.visc;
        // Inside a captured graph an iteration's k_finalize (norms, history row, halt flags, counters) runs on
        // the side stream beside the next iteration's gradients and face fluxes, which test halted_behind;
        // the graph's last iteration finalizes in line. The face coefficients alternate between two buffers,
        // so that the next k_flux does not overwrite the ones being summed.
        const bool defer = x->defer_n > 0 && !x->timing;
        const int bsel = defer ? (x->defer_i & 1) : 0;
        if (!x->timing) cudaEventRecord(x->ev_fork, x->stream);
        if (x->fin_pending && !early) {
            // the side stream waits for k_flux before the blocks: the pending k_finalize goes first
            cudaStreamWaitEvent(x->side, x->ev_fork, 0);
            launch_finalize<MODEL>(x, 1, x->fin_bsel, x->side);
            x->fin_pending = false;
        }
        if (grad) launch_grad<MODEL>(x, false);
        if (MODEL == 1 && x->prm.sa_isrc && !x->timing) cudaEventRecord(x->ev_grad, x->stream);
        snapshot_views(x);
        if (early) launch_blocks<MODEL>(x);
        launch_flux<MODEL>(x, 1 + bsel);
        if (!early) {
            if (!x->timing) cudaEventRecord(x->ev_fork, x->stream);
            launch_blocks<MODEL>(x);
        }
        if (!x->timing) cudaStreamWaitEvent(x->stream, x->ev_join, 0);
        // the first sweep gathers R (and its norms) from the face fluxes
        for (int m = 0; m < c.n_linear; m++) launch_sweep<MODEL>(x, m, c.n_linear);
        if (defer && x->defer_i + 1 < x->defer_n) {
            x->fin_pending = true;
            x->fin_bsel = bsel;
        } else {
            launch_finalize<MODEL>(x, 1, bsel);
        }
        if (defer) x->defer_i++;
    }
}

template <int MODEL>
static void launch_residual(csu_ctx* x, bool dbg)
{
    k_prim<MODEL><<<x->gb_c, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st, 0, 0);
    x->launches++;
    if (x->cfg.order == 2 || dbg) launch_grad<MODEL>(x, dbg);
    launch_flux<MODEL>(x, 1);
    k_resid<MODEL><<<x->gb_c, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st);
    x->launches++;
    launch_finalize<MODEL>(x, 3);
}

#define DISPATCH(fn, ...)                                                                                          \
    do {                                                                                                           \
        switch (x->model) {                                                                                        \
        case 0: fn<0>(__VA_ARGS__); break;                                                                         \
        case 1: fn<1>(__VA_ARGS__); break;                                                                         \
        default: fn<2>(__VA_ARGS__); break;                                                                        \
        }                                                                                                          \
    } while (0)

static int check_launch(const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, what);
    return CSU_OK;
}

static int ensure_hist(csu_ctx* x, int n)
{
    if (n <= x->hist_cap) return CSU_OK;
    int cap = n < 1024 ? 1024 : n;
    CK(cudaStreamSynchronize(x->stream));
    if (x->hist) CK(cudaFree(x->hist));
    x->hist = nullptr;
    CK(cudaMalloc((void**)&x->hist, sizeof(double) * (size_t)cap * (x->nv + 4) * x->nsolve));
    if (!x->is_pack) {
        if (x->h_hist) CK(cudaFreeHost(x->h_hist));
        x->h_hist = nullptr;
        CK(cudaMallocHost((void**)&x->h_hist, sizeof(double) * (size_t)cap * (x->nv + 4)));
    }
    x->hist_cap = cap;
    // point every solve's scalars at its new rows (the graphs read the pointer from the scalars at run time)
    std::vector<Scalars> hs(x->nsolve);
    int st;
    if ((st = read_scalars_n(x, hs.data(), x->nsolve))) return st;
    for (int k = 0; k < x->nsolve; k++) {
        hs[k].hist = hist_of(x, k);
        hs[k].hist_cap = cap;
    }
    return write_scalars_n(x, hs.data(), x->nsolve);
}

// The DPLUR blocks (written once per iteration, read by every sweep) as a persisting L2 window, when all of
// them fit in the part of L2 the device lets persist (cudaDevAttrMaxPersistingL2CacheSize): the bench's 61 MB
// of FP64 blocks, sweep 19.9 -> 18.9 us. Blocks larger than that are left alone: persisting a fraction of
// them kept that much L2 from the other kernels and cost more than it saved (a 400k-cell laminar FP64 solve
// with 205 MB of blocks: 1.16 ms per iteration without the window, 1.41 ms with 40 % of the blocks
// persisting). Only a cache policy: no result depends on it. CSU_L2_PERSIST=0 leaves the L2 alone.
static void plan_l2_window(csu_ctx* x)
{
    x->l2win = cudaAccessPolicyWindow{};
    const char* env = getenv("CSU_L2_PERSIST");
    if (env && strcmp(env, "0") == 0) return;
    void* base = x->st.blocks32 ? (void*)x->st.blocks32 : (void*)x->st.blocks;
    if (!base || x->cfg.time_scheme != CSU_TS_DPLUR) return;
    const size_t bytes = (size_t)x->max_ni * x->nv * x->nv * x->L.nc * (x->st.blocks32 ? sizeof(float) : sizeof(double));
    int max_persist = 0, max_window = 0;
    if (cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, x->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, x->device) != cudaSuccess ||
        max_persist <= 0 || max_window <= 0) {
        cudaGetLastError();
        return;
    }
    if (bytes > (size_t)max_persist || bytes > (size_t)max_window) return;
    size_t cur = 0;
    cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize);
    const size_t want = std::min(bytes, (size_t)max_persist);
    if (cur < want && cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize);
    const size_t win = std::min(bytes, (size_t)max_window);
    x->l2win.base_ptr = base;
    x->l2win.num_bytes = win;
    x->l2win.hitRatio = (float)std::min(1.0, (double)cur / (double)win);
    x->l2win.hitProp = cudaAccessPropertyPersisting;
    x->l2win.missProp = cudaAccessPropertyStreaming;
}

static void apply_l2_window(csu_ctx* x, cudaGraph_t g)
{
    if (!x->l2win.num_bytes) return;
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return;
    std::vector<cudaGraphNode_t> nodes(n);
    if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return;
    cudaKernelNodeAttrValue v = {};
    v.accessPolicyWindow = x->l2win;
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
            cudaGraphKernelNodeSetAttribute(nd, cudaKernelNodeAttributeAccessPolicyWindow, &v);
    }
    cudaGetLastError();
}

// Captures GRAPH_SIZES[gi] iterations into a graph starting at the current DPLUR buffer parity.
static int build_graph(csu_ctx* x, int gi)
{
    const int q = x->xcur;
    if (x->graphs[gi][q]) {
        cudaGraphExecDestroy(x->graphs[gi][q]);
        x->graphs[gi][q] = nullptr;
    }
    long long l0 = x->launches;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal));
    x->defer_n = GRAPH_SIZES[gi];
    x->defer_i = 0;
    x->fin_pending = false;
    for (int i = 0; i < GRAPH_SIZES[gi]; i++) DISPATCH(launch_iteration, x);
    x->defer_n = 0;
    cudaError_t e = cudaStreamEndCapture(x->stream, &g);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    apply_l2_window(x, g);
    e = cudaGraphInstantiate(&x->graphs[gi][q], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    x->graph_launches[gi][q] = x->launches - l0;
    x->xcur = q;
    x->launches = l0;
    return CSU_OK;
}

// ------------------------------------------------------------------------------------------------ autotuner
// Launch shapes of k_flux (faces per block) and of the DPLUR sweeps (cells per block) picked by timing each
// candidate on the context itself: `reps` launches after one warm-up, CUDA events on the context's stream.
// The timed launches leave no trace a later iteration could see: k_flux rewrites the face fluxes the next
// iteration computes again before reading them; the timed sweep is a middle sweep that writes the spare
// increment buffer (the next iteration's first sweep overwrites it) and uses the last early-exit slot pair,
// cleared afterwards. Choices are cached per device, model, order, viscosity, block precision and size class
// (half octaves of the cell count), so packs of a size class seen before take the cached shapes.
namespace {
struct TuneKey {
    int dev, model, order, visc, blk32, implicit, size_class;
    bool operator<(const TuneKey& o) const
    {
        return std::tie(dev, model, order, visc, blk32, implicit, size_class) <
               std::tie(o.dev, o.model, o.order, o.visc, o.blk32, o.implicit, o.size_class);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, std::pair<int, int>> g_tune_cache;
} // namespace

template <int MODEL>
static int time_flux_shape(csu_ctx* x, int fb, int reps, cudaEvent_t e0, cudaEvent_t e1, float* ms)
{
    const int save = x->flux_fb;
    x->flux_fb = fb;
    const long long l0 = x->launches;
    launch_flux<MODEL>(x, 1);
    CK(cudaEventRecord(e0, x->stream));
    for (int r = 0; r < reps; r++) launch_flux<MODEL>(x, 1);
    CK(cudaEventRecord(e1, x->stream));
    x->flux_fb = save;
    x->launches = l0;
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(ms, e0, e1));
    return CSU_OK;
}

template <int MODEL>
static int time_sweep_shape(csu_ctx* x, int sb, int reps, cudaEvent_t e0, cudaEvent_t e1, float* ms)
{
    // the slot before the timed one says "not converged" so the timed sweep does its full work
    const int slot = MAX_SWEEPS - 1;
    std::vector<unsigned long long> big(x->nsolve, 0x3ff0000000000000ULL); // 1.0 for every solve
    CK(cudaMemcpy2DAsync(&x->st.sc[0].sweep_max[slot - 1], sizeof(Scalars), big.data(), sizeof(unsigned long long),
                         sizeof(unsigned long long), x->nsolve, cudaMemcpyHostToDevice, x->stream));
    auto launch = [&]() {
        switch (sb) {
        case 64:
            (x->cfg.implicit_fp32 ? k_sweep<MODEL, false, false, 64, true> : k_sweep<MODEL, false, false, 64, false>)
                <<<x->gb_c * (BLOCK / 64), 64, 0, x->stream>>>(x->d_prm, x->mesh, x->st, slot, x->xcur);
            break;
        case 256:
            (x->cfg.implicit_fp32 ? k_sweep<MODEL, false, false, 256, true> : k_sweep<MODEL, false, false, 256, false>)
                <<<x->gb_c, 256, 0, x->stream>>>(x->d_prm, x->mesh, x->st, slot, x->xcur);
            break;
        default:
            (x->cfg.implicit_fp32 ? k_sweep<MODEL, false, false, 128, true> : k_sweep<MODEL, false, false, 128, false>)
                <<<x->gb_c * 2, 128, 0, x->stream>>>(x->d_prm, x->mesh, x->st, slot, x->xcur);
            break;
        }
    };
    launch();
    CK(cudaEventRecord(e0, x->stream));
    for (int r = 0; r < reps; r++) launch();
    CK(cudaEventRecord(e1, x->stream));
    CK(cudaGetLastError());
    CK(cudaMemset2DAsync(&x->st.sc[0].sweep_max[slot - 1], sizeof(Scalars), 0, 2 * sizeof(unsigned long long),
                         x->nsolve, x->stream));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(ms, e0, e1));
    return CSU_OK;
}

template <int MODEL>
static int tune_shapes(csu_ctx* x, int* fb_out, int* sb_out)
{
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    cudaError_t e = cudaEventCreate(&e1);
    if (e != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_fail(e, "cudaEventCreate");
    }
    const int reps = 5;
    int st = CSU_OK;
    float best = 1e30f;
    *fb_out = x->flux_fb;
    for (int fb : FLUX_BLOCKS) {
        float ms = 0;
        if ((st = time_flux_shape<MODEL>(x, fb, reps, e0, e1, &ms))) break;
        if (ms < best) {
            best = ms;
            *fb_out = fb;
        }
    }
    *sb_out = x->sweep_sb;
    if (!st && x->cfg.time_scheme == CSU_TS_DPLUR) {
        best = 1e30f;
        for (int sb : SWEEP_BLOCKS) {
            float ms = 0;
            if ((st = time_sweep_shape<MODEL>(x, sb, reps, e0, e1, &ms))) break;
            if (ms < best) {
                best = ms;
                *sb_out = sb;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}

// Picks the launch shapes of x (from the cache, or by timing when its class has not been seen); contexts
// under 16,384 cells keep the defaults (launch latency, not the shape, bounds them). CSU_AUTOTUNE=0 keeps
// the defaults everywhere.
static int autotune(csu_ctx* x, bool force)
{
    if (x->tuned && !force) return CSU_OK;
    x->tuned = true;
    const char* env = getenv("CSU_AUTOTUNE");
    if (env && strcmp(env, "0") == 0) return CSU_OK;
    if (x->L.nc < 16384 && !force) return CSU_OK;
    TuneKey key{x->device, x->model, x->cfg.order, x->prm.visc, x->cfg.implicit_fp32,
                x->cfg.time_scheme, (int)floor(2.0 * log2((double)x->L.nc))};
    int fb = x->flux_fb, sb = x->sweep_sb;
    bool hit = false;
    if (!force) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            fb = it->second.first;
            sb = it->second.second;
            hit = true;
        }
    }
    if (!hit) {
        int st;
        switch (x->model) {
        case 0: st = tune_shapes<0>(x, &fb, &sb); break;
        case 1: st = tune_shapes<1>(x, &fb, &sb); break;
        default: st = tune_shapes<2>(x, &fb, &sb); break;
        }
        if (st) return st;
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = {fb, sb};
    }
    if (fb != x->flux_fb || sb != x->sweep_sb) {
        x->flux_fb = fb;
        x->sweep_sb = sb;
        drop_graphs(x);
    }
    return CSU_OK;
}

extern "C" int csu_autotune(csu_ctx* x, int* flux_faces_per_block, int* sweep_cells_per_block)
{
    if (!x) return CSU_ERR_INPUT;
    int st = autotune(x, true);
    if (st) return st;
    if (flux_faces_per_block) *flux_faces_per_block = x->flux_fb;
    if (sweep_cells_per_block) *sweep_cells_per_block = x->sweep_sb;
    return CSU_OK;
}

// Start of a call on the device: history rows and the call's iteration count restart; a one-solve context
// also restarts its loop counter at it0 (the solves of a pack keep their own).
__global__ void k_call_begin(Scalars* sc, int n, int it0, int set_iter)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    sc[k].hist_row = 0;
    sc[k].steps = 0;
    if (set_iter) sc[k].iter = it0;
    // halt flags set or cleared between calls take effect for every kernel from the call's first launch
    sc[k].frozen = (sc[k].status | sc[k].done) != 0;
}

// The parity the DPLUR increment buffers have after `iters` iterations from parity q.
static int parity_after(const csu_ctx* x, int q, int iters)
{
    const int flips = x->cfg.time_scheme == CSU_TS_DPLUR ? x->cfg.n_linear * iters : 0;
    return q ^ (flips & 1);
}

// n iterations on the device: graphs of 8, 4, 2 and 1 iterations replayed largest first, nothing waited on
// before the launches; the scalars of solve 0 (and its history rows, when asked) come back at the end in
// one synchronization. One-solve contexts capture all four graphs the first time they need one (a later
// call of another length then replays without capturing); packs capture the ones their calls use.
static int run_iterations(csu_ctx* x, int n, int it0, Scalars* out, double* hist_rows)
{
    int st;
    if ((st = ensure_hist(x, n))) return st;
    if (!x->h_sc) CK(cudaMallocHost((void**)&x->h_sc, sizeof(Scalars)));
    if (!x->prepared && !x->is_pack) {
        if ((st = reset_scalars(x, it0))) return st;
    } else {
        k_call_begin<<<(x->nsolve + 31) / 32, 32, 0, x->stream>>>(x->st.sc, x->nsolve, it0, x->is_pack ? 0 : 1);
        x->launches++;
    }
    if (!x->prepared) {
        DISPATCH(launch_prologue, x);
        if ((st = check_launch("prologue"))) return st;
        x->prepared = 1;
    }
    if ((st = autotune(x, false))) return st;
    if (!x->is_pack) {
        // every size at the parities this context can start a graph with
        for (int gi = 0; gi < 4; gi++)
            if (!x->graphs[gi][x->xcur])
                if ((st = build_graph(x, gi))) return st;
    }
    auto launch_span = [&](int count) -> int {
        for (int gi = 0; gi < 4; gi++) {
            while (count >= GRAPH_SIZES[gi]) {
                const int q = x->xcur;
                int st2;
                if (!x->graphs[gi][q])
                    if ((st2 = build_graph(x, gi))) return st2;
                CK(cudaGraphLaunch(x->graphs[gi][q], x->stream));
                x->launches += x->graph_launches[gi][q];
                x->xcur = parity_after(x, q, GRAPH_SIZES[gi]);
                count -= GRAPH_SIZES[gi];
            }
        }
        return CSU_OK;
    };
    if (x->is_pack || n <= STOP_CHUNK) {
        if ((st = launch_span(n))) return st;
    } else {
        // A solve that halts (residual-drop stop, iteration cap, non-finite state) leaves the rest of the
        // call's kernels with nothing to do, but they would still be launched. Chunks of STOP_CHUNK
        // iterations instead, each followed by a copy of the halt flags; the host waits for the flags of the
        // chunk before the one just enqueued, so the device always has a chunk queued while it looks.
        if (!x->h_flags) CK(cudaMallocHost((void**)&x->h_flags, 4 * sizeof(int)));
        for (int q = 0; q < 2; q++)
            if (!x->ev_poll[q]) CK(cudaEventCreateWithFlags(&x->ev_poll[q], cudaEventDisableTiming));
        int left = n;
        for (int j = 0; left > 0; j++) {
            const int c = left < STOP_CHUNK ? left : STOP_CHUNK;
            if ((st = launch_span(c))) return st;
            left -= c;
            // status and done are adjacent in Scalars
            CK(cudaMemcpyAsync(x->h_flags + 2 * (j & 1), &x->st.sc[0].status, 2 * sizeof(int),
                               cudaMemcpyDeviceToHost, x->stream));
            CK(cudaEventRecord(x->ev_poll[j & 1], x->stream));
            if (j >= 1) {
                CK(cudaEventSynchronize(x->ev_poll[(j - 1) & 1]));
                const int* f = x->h_flags + 2 * ((j - 1) & 1);
                if (f[0] | f[1]) break;
            }
        }
    }
    if ((st = check_launch("iteration"))) return st;
    if (x->is_pack) {
        // a pack's results are read per solve (csu_pack_info / csu_pack_infos, which wait for this work), so
        // the call returns as soon as the iterations are queued and the caller's bookkeeping overlaps them
        memset(out, 0, sizeof(*out));
        out->steps = n;
        return CSU_OK;
    }
    CK(cudaMemcpyAsync(x->h_sc, x->st.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, x->stream));
    if (hist_rows && x->h_hist)
        CK(cudaMemcpyAsync(x->h_hist, x->hist, sizeof(double) * (size_t)n * (x->nv + 4), cudaMemcpyDeviceToHost,
                           x->stream));
    CK(cudaStreamSynchronize(x->stream));
    *out = *x->h_sc;
    if (hist_rows && x->h_hist) {
        const int rows = out->hist_row < n ? out->hist_row : n;
        memcpy(hist_rows, x->h_hist, sizeof(double) * (size_t)rows * (x->nv + 4));
    }
    return CSU_OK;
}

extern "C" int csu_iterate_ex(csu_ctx* x, int n, int it0, double* hist, int* n_done)
{
    if (!x || n < 0) return CSU_ERR_INPUT;
    if (n_done) *n_done = 0;
    if (n == 0) return CSU_OK;
    Scalars h;
    int st = run_iterations(x, n, it0, &h, x->is_pack ? nullptr : hist);
    if (!st && n_done) *n_done = h.steps;
    if (st) return st;
    if (x->is_pack) return CSU_OK; // per-solve results: csu_pack_info, csu_pack_history
    if (h.status) {
        csu_set_error("csu_iterate: state became non-finite at iteration %d", h.iter);
        return h.status;
    }
    return CSU_OK;
}

extern "C" int csu_iterate(csu_ctx* x, int n, int it0, double* hist)
{
    return csu_iterate_ex(x, n, it0, hist, nullptr);
}

extern "C" int csu_iterate_views(csu_ctx* x, int it0, double* hist, double* P, double* G)
{
    if (!x || !P || !G) return CSU_ERR_INPUT;
    if (x->is_pack) {
        csu_set_error("csu_iterate_views: views in reference order are per solve and not available for packs");
        return CSU_ERR_STATE;
    }
    const int nc = x->L.nc, nv = x->nv, nx = nv - 4;
    if (!x->h_snap) CK(cudaMallocHost((void**)&x->h_snap, sizeof(double) * (size_t)nc * (5 + nx + 8 + 2 * nx)));
    int st;
    if ((st = ensure_hist(x, 1))) return st;
    if (!x->h_sc) CK(cudaMallocHost((void**)&x->h_sc, sizeof(Scalars)));
    if (!x->prepared) {
        if ((st = reset_scalars(x, it0))) return st;
        DISPATCH(launch_prologue, x);
        x->prepared = 1;
    } else {
        k_call_begin<<<1, 32, 0, x->stream>>>(x->st.sc, 1, it0, 1);
        x->launches++;
    }
    if ((st = autotune(x, false))) return st;
    // one iteration launched directly (not from a graph), copying the views at its last residual evaluation
    x->snap = true;
    DISPATCH(launch_iteration, x);
    x->snap = false;
    if ((st = check_launch("csu_iterate_views"))) return st;
    CK(cudaMemcpyAsync(x->h_sc, x->st.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, x->stream));
    CK(cudaStreamSynchronize(x->stream));
    const Scalars h = *x->h_sc;
    if (hist && h.hist_row > 0) CK(cudaMemcpy(hist, x->hist, sizeof(double) * (nv + 4), cudaMemcpyDeviceToHost));
    const int* n2o = x->L.cell_new2old;
    const double *W4 = x->h_snap, *WT = W4 + 4 * (size_t)nc, *Wx = WT + nc, *G4x = Wx + (size_t)nx * nc,
                 *G4y = G4x + 4 * (size_t)nc, *Gxx = G4y + 4 * (size_t)nc, *Gxy = Gxx + (size_t)nx * nc;
    for (int c = 0; c < nc; c++) {
        const int o = n2o[c];
        double* row = P + (size_t)o * (nv + 1);
        for (int k = 0; k < 4; k++) row[k] = W4[(size_t)4 * c + k];
        row[4] = WT[c];
        for (int k = 5; k < nv + 1; k++) row[k] = Wx[(size_t)(k - 5) * nc + c];
        for (int k = 0; k < 4; k++) {
            G[(size_t)k * nc + o] = G4x[(size_t)4 * c + k];
            G[(size_t)(nv + k) * nc + o] = G4y[(size_t)4 * c + k];
        }
        for (int k = 4; k < nv; k++) {
            G[(size_t)k * nc + o] = Gxx[(size_t)(k - 4) * nc + c];
            G[(size_t)(nv + k) * nc + o] = Gxy[(size_t)(k - 4) * nc + c];
        }
    }
    if (h.status) {
        csu_set_error("csu_iterate_views: state became non-finite at iteration %d", h.iter);
        return h.status;
    }
    return CSU_OK;
}

extern "C" int csu_tube_run(csu_ctx* x, double tmax, int* steps, double* t_final)
{
    if (!x->cfg.tube || x->cfg.time_scheme != CSU_TS_RK) {
        csu_set_error("csu_tube_run: the case is not a tube case with RK time stepping");
        return CSU_ERR_STATE;
    }
    x->prm.tube = 1;
    x->prm.tmax = tmax;
    x->prms[0].tube = 1;
    x->prms[0].tmax = tmax;
    int st0 = upload_prm(x);
    if (st0) return st0;
    x->prepared = 0;
    drop_graphs(x);
    Scalars h;
    int st, total = 0;
    memset(&h, 0, sizeof(h));
    // the loop of solver.c:1921-1940 runs until the step that reaches tmax; checked every 64 steps
    for (int guard = 0; guard < 20000; guard++) {
        if ((st = run_iterations(x, 64, total, &h, nullptr))) return st;
        total = h.iter;
        if (h.done || h.status) break;
    }
    drop_graphs(x);
    *steps = total;
    *t_final = h.t;
    if (h.status) {
        csu_set_error("csu_tube_run: state became non-finite at step %d", total);
        return h.status;
    }
    return CSU_OK;
}

extern "C" int csu_wall_data(csu_ctx* x)
{
    if (!x) return CSU_ERR_INPUT;
    if (x->is_pack) {
        csu_set_error("csu_wall_data: views in reference order are per solve and not available for packs");
        return CSU_ERR_STATE;
    }
    if (x->L.nb == 0) return CSU_OK;
    const int g = (x->L.nb + BLOCK - 1) / BLOCK;
    switch (x->model) {
    case 0: k_wall_data<0><<<g, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st); break;
    case 1: k_wall_data<1><<<g, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st); break;
    default: k_wall_data<2><<<g, BLOCK, 0, x->stream>>>(x->d_prm, x->mesh, x->st); break;
    }
    x->launches++;
    int st = check_launch("csu_wall_data");
    if (st) return st;
    CK(cudaStreamSynchronize(x->stream));
    return CSU_OK;
}

extern "C" int csu_residual(csu_ctx* x, double* R)
{
    if (!x) return CSU_ERR_INPUT;
    int st;
    // a fresh evaluation: scalars keep the step state but not a halt flag
    Scalars h;
    if ((st = read_scalars(x, &h))) return st;
    h.done = 0;
    h.status = 0;
    h.frozen = 0;
    if ((st = write_scalars_n(x, &h, 1))) return st;
    DISPATCH(launch_residual, x, true);
    if ((st = check_launch("residual"))) return st;
    x->prepared = 0;
    CK(cudaStreamSynchronize(x->stream));
    if (R) return csu_dump(x, CSU_DUMP_R, R);
    return CSU_OK;
}

extern "C" int csu_dump(csu_ctx* x, int what, double* out)
{
    if (!x || !out) return CSU_ERR_INPUT;
    if (x->is_pack && what != CSU_DUMP_LSQ_X87) {
        csu_set_error("csu_dump: views in reference order are per solve and not available for packs");
        return CSU_ERR_STATE;
    }
    const int nc = x->L.nc, nf = x->L.nf, nb = x->L.nb, nv = x->nv, nx = nv - 4;
    CK(cudaStreamSynchronize(x->stream));
    auto d2h = [&](std::vector<double>& v, const void* src, size_t n) -> cudaError_t {
        v.resize(n > 0 ? n : 1);
        if (n == 0) return cudaSuccess;
        return cudaMemcpy(v.data(), src, sizeof(double) * n, cudaMemcpyDeviceToHost);
    };
    std::vector<double> a, b, c2;
    const int* n2o = x->L.cell_new2old;
    switch (what) {
    case CSU_DUMP_P: {
        CK(d2h(a, x->st.W4, (size_t)4 * nc));
        CK(d2h(b, x->st.WT, nc));
        CK(d2h(c2, x->st.Wx, (size_t)nx * nc));
        for (int c = 0; c < nc; c++) {
            double* row = out + (size_t)n2o[c] * (nv + 1);
            for (int k = 0; k < 4; k++) row[k] = a[(size_t)4 * c + k];
            row[4] = b[c];
            for (int k = 5; k < nv + 1; k++) row[k] = c2[(size_t)(k - 5) * nc + c];
        }
        return CSU_OK;
    }
    case CSU_DUMP_GHOST_P:
        CK(d2h(a, x->st.dbg_ghost, (size_t)nb * (nv + 1)));
        memcpy(out, a.data(), sizeof(double) * (size_t)nb * (nv + 1));
        return CSU_OK;
    case CSU_DUMP_GRAD:
    case CSU_DUMP_PHI: {
        const double4* s4[2] = {x->st.G4x, x->st.G4y};
        const double* sx[2] = {x->st.Gxx, x->st.Gxy};
        int nparts = what == CSU_DUMP_GRAD ? 2 : 1;
        if (what == CSU_DUMP_PHI) {
            s4[0] = x->st.PH4;
            sx[0] = x->st.PHx;
        }
        for (int part = 0; part < nparts; part++) {
            CK(d2h(a, s4[part], (size_t)4 * nc));
            CK(d2h(b, sx[part], (size_t)nx * nc));
            double* o = out + (size_t)part * nv * nc;
            for (int c = 0; c < nc; c++) {
                for (int k = 0; k < 4; k++) o[(size_t)k * nc + n2o[c]] = a[(size_t)4 * c + k];
                for (int k = 4; k < nv; k++) o[(size_t)k * nc + n2o[c]] = b[(size_t)(k - 4) * nc + c];
            }
        }
        return CSU_OK;
    }
    case CSU_DUMP_FACEFLUX: {
        CK(d2h(a, x->st.F4, (size_t)4 * (nf + nb)));
        CK(d2h(b, x->st.Fx, (size_t)nx * (nf + nb)));
        for (int f = 0; f < nf; f++) {
            int o = x->L.face_new2old[f];
            for (int k = 0; k < 4; k++) out[(size_t)k * nf + o] = a[(size_t)4 * f + k];
            for (int k = 4; k < nv; k++) out[(size_t)k * nf + o] = b[(size_t)(k - 4) * (nf + nb) + f];
        }
        return CSU_OK;
    }
    case CSU_DUMP_R:
    case CSU_DUMP_DW: {
        const double4* s4 = what == CSU_DUMP_R ? x->st.R4 : x->st.X4[x->xcur];
        const double* sx = what == CSU_DUMP_R ? x->st.Rx : x->st.Xx[x->xcur];
        if (!s4) {
            csu_set_error("csu_dump: no implicit increment in this context");
            return CSU_ERR_STATE;
        }
        CK(d2h(a, s4, (size_t)4 * nc));
        CK(d2h(b, sx, (size_t)nx * nc));
        for (int c = 0; c < nc; c++) {
            for (int k = 0; k < 4; k++) out[(size_t)k * nc + n2o[c]] = a[(size_t)4 * c + k];
            for (int k = 4; k < nv; k++) out[(size_t)k * nc + n2o[c]] = b[(size_t)(k - 4) * nc + c];
        }
        return CSU_OK;
    }
    case CSU_DUMP_D:
    case CSU_DUMP_DTL: {
        CK(d2h(a, what == CSU_DUMP_D ? x->st.dpart : x->st.dtl, nc));
        if (what == CSU_DUMP_D) {
            // D = dpart + Omega/dt with the step of the last implicit iteration (implicit.c:167-180)
            Scalars h;
            int st = read_scalars(x, &h);
            if (st) return st;
            (void)h;
            std::vector<double> dtl;
            CK(d2h(dtl, x->st.dtl, nc));
            double mn = dtl[0];
            for (int c = 1; c < nc; c++) mn = fmin(mn, dtl[c]);
            double dt = mn * x->cfg.cfl;
            for (int c = 0; c < nc; c++) out[n2o[c]] = a[c] + x->L.omega[c] / dt;
        } else {
            for (int c = 0; c < nc; c++) out[n2o[c]] = a[c];
        }
        return CSU_OK;
    }
    case CSU_DUMP_BLOCKS: {
        if (!x->st.blocks && !x->st.blocks32) {
            csu_set_error("csu_dump: no DPLUR blocks in this context");
            return CSU_ERR_STATE;
        }
        size_t per = (size_t)nv * nv;
        if (x->st.blocks) {
            CK(d2h(a, x->st.blocks, (size_t)4 * per * nc));
        } else {
            std::vector<float> f((size_t)4 * per * nc);
            CK(cudaMemcpy(f.data(), x->st.blocks32, sizeof(float) * f.size(), cudaMemcpyDeviceToHost));
            a.assign(f.begin(), f.end());
        }
        for (int c = 0; c < nc; c++) {
            double* o = out + (size_t)n2o[c] * 4 * per;
            for (int j = 0; j < 4; j++)
                for (size_t e = 0; e < per; e++) o[j * per + e] = a[((size_t)j * per + e) * nc + c];
        }
        return CSU_OK;
    }
    case CSU_DUMP_SST_JAC: {
        if (!x->st.dQ) {
            csu_set_error("csu_dump: no SST source Jacobians in this context (SST with LU-SGS or DPLUR only)");
            return CSU_ERR_STATE;
        }
        CK(d2h(a, x->st.dQ, (size_t)6 * nc));
        for (int q = 0; q < 6; q++)
            for (int c = 0; c < nc; c++) out[(size_t)q * nc + n2o[c]] = a[(size_t)q * nc + c];
        return CSU_OK;
    }
    case CSU_DUMP_BVISC: {
        if (!x->prm.visc) {
            csu_set_error("csu_dump: no viscous fluxes in this context (laminar, SA or SST only)");
            return CSU_ERR_STATE;
        }
        CK(d2h(a, x->st.FV + nf, (size_t)4 * nb));
        for (int b = 0; b < nb; b++) {
            double* o = out + (size_t)x->L.bold[b] * 4;
            for (int k = 0; k < 4; k++) o[k] = a[(size_t)4 * b + k];
        }
        return CSU_OK;
    }
    case CSU_DUMP_LSQ_X87: {
        unsigned long long q = 0;
        CK(cudaMemcpy(&q, x->st.lsq_x87, sizeof(q), cudaMemcpyDeviceToHost));
        out[0] = (double)q;
        return CSU_OK;
    }
    default:
        csu_set_error("csu_dump: unknown view %d", what);
        return CSU_ERR_INPUT;
    }
}

extern "C" int csu_stats(csu_ctx* x, long long* launches, long long* bytes)
{
    if (launches) *launches = x->launches;
    if (bytes) *bytes = (long long)x->arena.size + (long long)x->hist_cap * (x->nv + 4) * 8;
    return CSU_OK;
}

extern "C" int csu_set_stream(csu_ctx* x, void* stream)
{
    if (!x) return CSU_ERR_INPUT;
    CK(cudaStreamSynchronize(x->stream));
    x->stream = stream ? (cudaStream_t)stream : x->own_stream;
    return CSU_OK;
}

extern "C" int csu_time_kernels(csu_ctx* x, int iters, double* ms, int* count)
{
    if (!x || iters < 1) return CSU_ERR_INPUT;
    int st;
    for (int k = 0; k < CSU_K_COUNT; k++) {
        ms[k] = 0.0;
        count[k] = 0;
    }
    if (!x->prepared) {
        Scalars h;
        if ((st = run_iterations(x, 1, 0, &h, nullptr))) return st;
    }
    CK(cudaStreamSynchronize(x->stream));
    // the launches below are not graph nodes: give them the graphs' L2 window through the stream (the previous
    // attribute of the caller's stream is put back afterwards)
    cudaStreamAttrValue prev = {}, mine = {};
    const bool win = x->l2win.num_bytes > 0 &&
                     cudaStreamGetAttribute(x->stream, cudaStreamAttributeAccessPolicyWindow, &prev) == cudaSuccess;
    if (win) {
        mine.accessPolicyWindow = x->l2win;
        CK(cudaStreamSetAttribute(x->stream, cudaStreamAttributeAccessPolicyWindow, &mine));
    }
    x->timing = true;
    x->ev_used = 0;
    tmark(x, -1);
    for (int i = 0; i < iters; i++) DISPATCH(launch_iteration, x);
    x->timing = false;
    if ((st = check_launch("timed iterations"))) return st;
    if (win) CK(cudaStreamSetAttribute(x->stream, cudaStreamAttributeAccessPolicyWindow, &prev));
    if ((st = check_launch("timed iterations"))) return st;
    CK(cudaStreamSynchronize(x->stream));
    for (size_t i = 1; i < x->ev_used; i++) {
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, x->ev[i - 1], x->ev[i]));
        int k = x->ev_kind[i];
        if (k >= 0 && k < CSU_K_COUNT) {
            ms[k] += t;
            count[k]++;
        }
    }
    return CSU_OK;
}

// ------------------------------------------------------------------------------------------------ packs

struct csu_prep {
    csu_config cfg;
    csu_layout L;
    int model = 0, nv = 4;
    long long bytes = 0;
};

// Settings every solve of a pack shares (the launch sequence and the kernels' specialisation depend on
// them); flow conditions, walls' temperature, outlet pressure, CFL schedule, stopping drop and reference
// length may differ per solve.
static bool same_structure(const csu_config& a, const csu_config& b)
{
    if (a.sa_implicit_source != b.sa_implicit_source) return false;
    return a.nvar == b.nvar && a.order == b.order && a.flux == b.flux && a.stages == b.stages &&
           a.time_scheme == b.time_scheme && a.n_linear == b.n_linear && a.dt_local == b.dt_local &&
           a.dt_local_n == b.dt_local_n && a.laminar == b.laminar && a.sa == b.sa && a.sa_cc == b.sa_cc &&
           a.sst == b.sst && a.sst_trans == b.sst_trans && a.axisymmetric == b.axisymmetric &&
           a.turb1order == b.turb1order && a.visc_blazek == b.visc_blazek && a.tp == b.tp &&
           a.limiter_type == b.limiter_type && a.tube == b.tube && a.implicit_fp32 == b.implicit_fp32 &&
           a.implicit_local_dt == b.implicit_local_dt;
}

extern "C" int csu_prep_create(const csu_mesh_desc* md, const csu_config* cfg, csu_prep** out)
{
    if (!out) return CSU_ERR_INPUT;
    *out = nullptr;
    if (!md || !cfg || md->n_cells <= 0) {
        csu_set_error("csu_prep_create: empty mesh or missing config");
        return CSU_ERR_INPUT;
    }
    int model, nv;
    int st = validate_config("csu_prep_create", cfg, &model, &nv);
    if (st) return st;
    csu_prep* p = new csu_prep();
    p->cfg = *cfg;
    p->model = model;
    p->nv = nv;
    st = csu_layout_build(md, cfg->axisymmetric, &p->L);
    if (!st && cfg->gradient == 1) st = csu_layout_green_gauss(&p->L);
    if (st) {
        delete p;
        csu_set_error("csu_prep_create: mesh layout failed (a cell with more than four faces?)");
        return st;
    }
    // device bytes of the solve: the arena a one-solve context would carve, plus 1024 history rows
    csu_ctx t;
    t.model = model;
    t.nv = nv;
    t.cfg = *cfg;
    t.L = p->L;
    Arena a;
    plan(&t, a);
    memset(&t.L, 0, sizeof(t.L)); // owned by p
    p->bytes = (long long)a.size + 1024LL * (nv + 4) * 8;
    *out = p;
    return CSU_OK;
}

extern "C" long long csu_prep_bytes(const csu_prep* p)
{
    return p ? p->bytes : 0;
}

extern "C" int csu_prep_cells(const csu_prep* p)
{
    return p ? p->L.nc : 0;
}

extern "C" void csu_prep_destroy(csu_prep* p)
{
    if (!p) return;
    csu_layout_free(&p->L);
    delete p;
}

extern "C" int csu_pack_size(csu_ctx* x)
{
    return x ? x->nsolve : 0;
}

extern "C" int csu_pack_set_state(csu_ctx* x, int k, const double* U)
{
    if (!x || !U || k < 0 || k >= x->nsolve) return CSU_ERR_INPUT;
    return solve_state_io(x, k, const_cast<double*>(U), true);
}

extern "C" int csu_pack_get_state(csu_ctx* x, int k, double* U)
{
    if (!x || !U || k < 0 || k >= x->nsolve) return CSU_ERR_INPUT;
    return solve_state_io(x, k, U, false);
}

extern "C" int csu_pack_stop(csu_ctx* x, int k)
{
    if (!x || k < 0 || k >= x->nsolve) return CSU_ERR_INPUT;
    // done = 3: every kernel skips the solve from the next launch on, like a converged one
    static const int stopped = 3;
    CK(cudaMemcpyAsync(&x->st.sc[k].done, &stopped, sizeof(int), cudaMemcpyHostToDevice, x->stream));
    CK(cudaStreamSynchronize(x->stream));
    return CSU_OK;
}

static void solve_info_from(const csu_ctx* x, const Scalars& h, csu_solve_info* info)
{
    memset(info, 0, sizeof(*info));
    info->iter = h.iter;
    info->status = h.status;
    info->done = h.done;
    info->hist_rows = h.hist_row < h.hist_cap ? h.hist_row : h.hist_cap;
    info->have_res0 = h.have_res0;
    for (int v = 0; v < x->nv; v++) {
        info->res0[v] = h.res0[v];
        info->res[v] = h.res[v];
    }
    for (int v = 0; v < 4; v++) info->coef[v] = h.coef[v];
}

extern "C" int csu_pack_infos(csu_ctx* x, csu_solve_info* infos)
{
    if (!x || !infos) return CSU_ERR_INPUT;
    std::vector<Scalars> hs(x->nsolve);
    int st = read_scalars_n(x, hs.data(), x->nsolve);
    if (st) return st;
    for (int k = 0; k < x->nsolve; k++) solve_info_from(x, hs[k], infos + k);
    return CSU_OK;
}

extern "C" int csu_pack_info(csu_ctx* x, int k, csu_solve_info* info)
{
    if (!x || !info || k < 0 || k >= x->nsolve) return CSU_ERR_INPUT;
    std::vector<Scalars> hs(x->nsolve);
    int st = read_scalars_n(x, hs.data(), x->nsolve);
    if (st) return st;
    const Scalars& h = hs[k];
    memset(info, 0, sizeof(*info));
    info->iter = h.iter;
    info->status = h.status;
    info->done = h.done;
    info->hist_rows = h.hist_row < h.hist_cap ? h.hist_row : h.hist_cap;
    info->have_res0 = h.have_res0;
    for (int v = 0; v < x->nv; v++) {
        info->res0[v] = h.res0[v];
        info->res[v] = h.res[v];
    }
    for (int v = 0; v < 4; v++) info->coef[v] = h.coef[v];
    return CSU_OK;
}

extern "C" int csu_pack_history(csu_ctx* x, int k, double* hist, int max_rows, int* rows)
{
    if (!x || !hist || k < 0 || k >= x->nsolve) return CSU_ERR_INPUT;
    csu_solve_info info;
    int st = csu_pack_info(x, k, &info);
    if (st) return st;
    int n = info.hist_rows < max_rows ? info.hist_rows : max_rows;
    if (n > 0) CK(cudaMemcpy(hist, hist_of(x, k), sizeof(double) * (size_t)n * (x->nv + 4), cudaMemcpyDeviceToHost));
    if (rows) *rows = n;
    return CSU_OK;
}

// Device copy of solve kf of `from` into solve kt of `to` (same mesh and settings): conserved state,
// primitives, the implicit increments (DPLUR warm start) and the solve's counters, first residual and
// flags, so that `to` continues the solve where `from` left it.
static int transfer_state_copies(csu_ctx* from, int kf, csu_ctx* to, int kt);

extern "C" int csu_pack_transfer(csu_ctx* from, int kf, csu_ctx* to, int kt)
{
    if (!from || !to || kf < 0 || kf >= from->nsolve || kt < 0 || kt >= to->nsolve) return CSU_ERR_INPUT;
    if (from->model != to->model || from->ncs[kf] != to->ncs[kt] || !same_structure(from->cfg, to->cfg)) {
        csu_set_error("csu_pack_transfer: the two solves differ in size or settings");
        return CSU_ERR_INPUT;
    }
    CK(cudaStreamSynchronize(from->stream));
    CK(cudaStreamSynchronize(to->stream));
    int st = transfer_state_copies(from, kf, to, kt);
    if (st) return st;
    Scalars hf, ht;
    CK(cudaMemcpy(&hf, from->st.sc + kf, sizeof(Scalars), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&ht, to->st.sc + kt, sizeof(Scalars), cudaMemcpyDeviceToHost));
    double* hist = ht.hist;
    int cap = ht.hist_cap;
    ht = hf;
    ht.hist = hist;
    ht.hist_cap = cap;
    ht.hist_row = 0;
    ht.steps = 0;
    ht.fresh = 0;
    CK(cudaMemcpy(to->st.sc + kt, &ht, sizeof(Scalars), cudaMemcpyHostToDevice));
    to->prepared = 0;
    return CSU_OK;
}

// ------------------------------------------------------------------------------------------------ pack assembly
// A pack's mesh arrays are its solves' arrays side by side. Building a pack copies each solve's rows into
// place -- from the host layout of a new solve, or device to device from the pack that held it before --
// and then re-bases the index-valued entries (cells, ghost and face codes, wall ranks) on the new offsets.
// No concatenated host layout is built, and a rebuild uploads only the solves that are new.

namespace {

enum { SEG_CELL = 0, SEG_CELL4, SEG_FACE, SEG_BFACE };

struct SegArr {
    char* dev;
    size_t es;
    int kind;
};

// Where a solve's rows lie: cells [c0, c0 + nc), faces [f0, ...), boundary faces [b0, ...) of a pack with
// NC cells (stride of [slot][cell] arrays, ghost base) and NF interior faces (boundary flux base); w0 is the
// solve's first wall rank.
struct SegGeo {
    int c0, nc, f0, nf, b0, nb, NC, NF, w0;
};

} // namespace

static std::vector<SegArr> seg_arrays(csu_ctx* x)
{
    Mesh& m = x->mesh;
    auto P = [](const void* p) { return (char*)const_cast<void*>(p); };
    std::vector<SegArr> v = {
        {P(m.npts), 4, SEG_CELL}, {P(m.nint), 4, SEG_CELL}, {P(m.nslot), 4, SEG_CELL},
        {P(m.nei), 4, SEG_CELL4}, {P(m.wx), 8, SEG_CELL4}, {P(m.wy), 8, SEG_CELL4},
        {P(m.ldx), 8, SEG_CELL4}, {P(m.ldy), 8, SEG_CELL4}, {P(m.lm), 8, SEG_CELL4},
        {P(m.les), 4, SEG_CELL4}, {P(m.lrv), 8, SEG_CELL}, {P(m.lq), 16, SEG_CELL4},
        {P(m.ex), 8, SEG_CELL4}, {P(m.ey), 8, SEG_CELL4}, {P(m.fslot), 4, SEG_CELL4}, {P(m.fnb), 4, SEG_CELL4},
        {P(m.omega), 8, SEG_CELL}, {P(m.sxh), 8, SEG_CELL}, {P(m.syh), 8, SEG_CELL},
        {P(m.dslat), 8, SEG_CELL}, {P(m.color), 4, SEG_CELL},
        {P(m.fe), 8, SEG_FACE}, {P(m.fn), 16, SEG_FACE}, {P(m.fds), 8, SEG_FACE}, {P(m.r0), 16, SEG_FACE},
        {P(m.r1), 16, SEG_FACE}, {P(m.fd), 16, SEG_FACE}, {P(m.fL), 8, SEG_FACE},
        {P(m.bown), 4, SEG_BFACE}, {P(m.bflag), 4, SEG_BFACE}, {P(m.bold), 4, SEG_BFACE},
        {P(m.bn), 16, SEG_BFACE}, {P(m.bds), 8, SEG_BFACE}, {P(m.bd), 16, SEG_BFACE}, {P(m.bL), 8, SEG_BFACE},
        {P(m.bun), 16, SEG_BFACE}, {P(m.bds2), 8, SEG_BFACE}, {P(x->d_wall_rank), 4, SEG_BFACE}};
    if (m.wall_d) v.push_back({P(m.wall_d), 8, SEG_CELL});
    return v;
}

// Walls of one solve in reference (marker-major) order: rank per boundary face, -1 elsewhere.
static int local_wall_ranks(const csu_layout& L, int* rank)
{
    std::vector<int> by_old(L.nb, -1);
    for (int b = 0; b < L.nb; b++) by_old[L.bold[b]] = b;
    int r = 0;
    for (int b = 0; b < L.nb; b++) rank[b] = -1;
    for (int o = 0; o < L.nb; o++) {
        int b = by_old[o];
        if (L.bflag[b] == CSU_BC_WALL || L.bflag[b] == CSU_BC_WALLT) rank[b] = r++;
    }
    return r;
}

// The same arrays of one solve's host layout, in seg_arrays order (device formats built in `keep`).
static std::vector<const void*> seg_host(const csu_layout& L, std::vector<std::vector<char>>& keep)
{
    const int nf = L.nf, nb = L.nb;
    auto pairs = [&](const double* a, const double* b, int n) {
        keep.emplace_back((size_t)n * sizeof(double2) + 1);
        double2* d = (double2*)keep.back().data();
        for (int i = 0; i < n; i++) d[i] = make_double2(a[i], b[i]);
        return (const void*)d;
    };
    keep.emplace_back((size_t)nf * sizeof(int2) + 1);
    int2* fe = (int2*)keep.back().data();
    for (int f = 0; f < nf; f++) fe[f] = make_int2(L.fe0[f], L.fe1[f]);
    keep.emplace_back((size_t)nb * sizeof(int) + 1);
    int* rank = (int*)keep.back().data();
    local_wall_ranks(L, rank);
    std::vector<const void*> v = {
        L.npts, L.nint, L.nslot, L.nei, L.wx, L.wy, L.ldx, L.ldy, L.lm, L.les, L.lrv, L.lq, L.ex, L.ey, L.fslot, L.fnb,
        L.omega, L.sxh, L.syh, L.dslat, L.color,
        fe, pairs(L.fdsx, L.fdsy, nf), L.fds, pairs(L.r0x, L.r0y, nf), pairs(L.r1x, L.r1y, nf),
        pairs(L.fdx, L.fdy, nf), L.fdist,
        L.bown, L.bflag, L.bold, pairs(L.bdsx, L.bdsy, nb), L.bds, pairs(L.bdx, L.bdy, nb), L.bL,
        pairs(L.bunx, L.buny, nb), L.bds2, rank};
    if (L.wall_d) v.push_back(L.wall_d);
    return v;
}

// Re-bases the index-valued rows of one solve from geometry S (where they were written) to D.
__global__ void k_seg_fix(Mesh m, int* wall_rank, SegGeo S, SegGeo D)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int dc = D.c0 - S.c0;
    if (t < D.nc) {
        int c = D.c0 + t;
        int* nei = const_cast<int*>(m.nei);
        int* fs = const_cast<int*>(m.fslot);
        int* fnb = const_cast<int*>(m.fnb);
        for (int j = 0; j < 4; j++) {
            size_t o = (size_t)j * D.NC + c;
            if (fnb[o] >= 0) fnb[o] += dc;
            int v = nei[o];
            nei[o] = v < S.NC ? v + dc : v - S.NC - S.b0 + D.NC + D.b0;
            int f = fs[o];
            if (f != 0) {
                int a = (f < 0 ? -f : f) - 1;
                a = a < S.NF ? a - S.f0 + D.f0 : a - S.NF - S.b0 + D.NF + D.b0;
                fs[o] = f < 0 ? -(a + 1) : a + 1;
            }
        }
    }
    if (t < D.nf) {
        int2* fe = const_cast<int2*>(m.fe);
        int2 e = fe[D.f0 + t];
        fe[D.f0 + t] = make_int2(e.x + dc, e.y + dc);
    }
    if (t < D.nb) {
        int* bown = const_cast<int*>(m.bown);
        bown[D.b0 + t] += dc;
        int r = wall_rank[D.b0 + t];
        if (r >= 0) wall_rank[D.b0 + t] = r - S.w0 + D.w0;
    }
}

static SegGeo seg_geo(const csu_ctx* x, int k)
{
    SegGeo g;
    g.c0 = x->cell0[k];
    g.nc = x->ncs[k];
    g.f0 = x->face0[k];
    g.nf = x->prms[k].nf;
    g.b0 = x->bface0[k];
    g.nb = x->prms[k].nb;
    g.NC = x->L.nc;
    g.NF = x->L.nf;
    g.w0 = x->prms[k].wall0;
    return g;
}

// Device-to-device copies of a pack rebuild, gathered into one table and run by one kernel (a rebuild of a
// large pack would otherwise issue thousands of small copies). Jobs are split into pieces of at most 256 KiB
// so the blocks share the work; each piece moves 8-byte words when its addresses and length allow.
struct CopyJob {
    const char* src;
    char* dst;
    unsigned long long bytes;
};

struct CopyPlan {
    std::vector<CopyJob> jobs;
    void add(void* dst, const void* src, size_t bytes)
    {
        const size_t piece = 256 << 10;
        for (size_t o = 0; o < bytes; o += piece)
            jobs.push_back({(const char*)src + o, (char*)dst + o, (unsigned long long)std::min(piece, bytes - o)});
    }
};

__global__ void k_copy_jobs(const CopyJob* __restrict__ jobs, int n)
{
    for (int j = blockIdx.x; j < n; j += gridDim.x) {
        const CopyJob J = jobs[j];
        if ((((unsigned long long)J.src | (unsigned long long)J.dst | J.bytes) & 7) == 0) {
            const unsigned long long* s = reinterpret_cast<const unsigned long long*>(J.src);
            unsigned long long* d = reinterpret_cast<unsigned long long*>(J.dst);
            for (unsigned long long i = threadIdx.x; i < J.bytes / 8; i += blockDim.x) d[i] = s[i];
        } else {
            for (unsigned long long i = threadIdx.x; i < J.bytes; i += blockDim.x) J.dst[i] = J.src[i];
        }
    }
}

// the device copy of a plan's job table per device, kept and grown across rebuilds (freed with the pack
// arenas)
struct JobTable {
    CopyJob* p = nullptr;
    size_t cap = 0;
};
constexpr int MAX_JOB_DEVICES = 64;
std::mutex g_jobs_mu;
JobTable g_jobs[MAX_JOB_DEVICES];

static int run_copy_plan(csu_ctx* x, CopyPlan& plan)
{
    if (plan.jobs.empty()) return CSU_OK;
    if (x->device < 0 || x->device >= MAX_JOB_DEVICES) {
        csu_set_error("pack rebuild: device %d beyond the %d supported", x->device, MAX_JOB_DEVICES);
        return CSU_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lk(g_jobs_mu);
    JobTable& T = g_jobs[x->device];
    const size_t n = plan.jobs.size();
    if (n > T.cap) {
        if (T.p) cudaFree(T.p);
        T.p = nullptr;
        T.cap = 0;
        size_t cap = std::max(n, (size_t)4096);
        CK(cudaMalloc((void**)&T.p, sizeof(CopyJob) * cap));
        T.cap = cap;
    }
    CK(cudaMemcpyAsync(T.p, plan.jobs.data(), sizeof(CopyJob) * n, cudaMemcpyHostToDevice, x->stream));
    // enough blocks to fill the device (8 per multiprocessor), never more than there are jobs
    k_copy_jobs<<<(int)std::min(n, (size_t)x->sm_count * 8), 256, 0, x->stream>>>(T.p, (int)n);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(x->stream)); // the table is reused by the next plan
    plan.jobs.clear();
    return CSU_OK;
}

// The iteration state of solve kf of `from` (U, W, T, Omega/Lc or local steps, both DPLUR increments) queued
// as copies into solve kt of `to`; the scalars are the caller's (csu_pack_transfer moves the same arrays).
static void state_copy_plan(csu_ctx* from, int kf, csu_ctx* to, int kt, CopyPlan& plan)
{
    const int n = from->ncs[kf], of = from->cell0[kf], ot = to->cell0[kt], NF = from->L.nc, NT = to->L.nc;
    const int nx = from->nv - 4;
    plan.add(to->st.U4 + ot, from->st.U4 + of, sizeof(double4) * n);
    plan.add(to->st.W4 + ot, from->st.W4 + of, sizeof(double4) * n);
    plan.add(to->st.WT + ot, from->st.WT + of, sizeof(double) * n);
    plan.add(to->st.dtl + ot, from->st.dtl + of, sizeof(double) * n);
    for (int r = 0; r < nx; r++) {
        plan.add(to->st.Ux + (size_t)r * NT + ot, from->st.Ux + (size_t)r * NF + of, sizeof(double) * n);
        plan.add(to->st.Wx + (size_t)r * NT + ot, from->st.Wx + (size_t)r * NF + of, sizeof(double) * n);
    }
    if (from->st.X4[0] && to->st.X4[0]) {
        for (int q = 0; q < 2; q++) {
            int qf = from->xcur ^ q, qt = to->xcur ^ q;
            plan.add(to->st.X4[qt] + ot, from->st.X4[qf] + of, sizeof(double4) * n);
            for (int r = 0; r < nx; r++)
                plan.add(to->st.Xx[qt] + (size_t)r * NT + ot, from->st.Xx[qf] + (size_t)r * NF + of,
                         sizeof(double) * n);
        }
    }
}

static void release_copy_jobs()
{
    std::lock_guard<std::mutex> lk(g_jobs_mu);
    for (JobTable& T : g_jobs) {
        if (T.p) cudaFree(T.p);
        T.p = nullptr;
        T.cap = 0;
    }
}

// The state copies of csu_pack_transfer, run at once.
static int transfer_state_copies(csu_ctx* from, int kf, csu_ctx* to, int kt)
{
    CopyPlan plan;
    state_copy_plan(from, kf, to, kt, plan);
    return run_copy_plan(to, plan);
}

// Re-bases the index-valued rows of one solve whose rows are in place (k_seg_fix).
static int seg_fix(csu_ctx* x, SegGeo S, SegGeo D)
{
    int nt = std::max(D.nc, std::max(D.nf, D.nb));
    if (nt > 0) k_seg_fix<<<(nt + BLOCK - 1) / BLOCK, BLOCK, 0, x->stream>>>(x->mesh, x->d_wall_rank, S, D);
    CK(cudaGetLastError());
    return CSU_OK;
}

// Copies solve k's mesh rows into x: device to device from solve ks of `src` (queued on `plan`, and
// re-based by k_seg_fix once the plan has run: see seg_fix), or from `L` (src null).
static int seg_fill(csu_ctx* x, int k, const csu_layout* L, csu_ctx* src, int ks, CopyPlan* plan)
{
    SegGeo D = seg_geo(x, k), S;
    std::vector<SegArr> dst = seg_arrays(x);
    if (src) {
        S = seg_geo(src, ks);
        std::vector<SegArr> from = seg_arrays(src);
        if (from.size() != dst.size()) return CSU_ERR_INPUT;
        for (size_t a = 0; a < dst.size(); a++) {
            const size_t es = dst[a].es;
            auto cp = [&](size_t so, size_t dof, size_t n) {
                plan->add(dst[a].dev + dof * es, from[a].dev + so * es, n * es);
                return cudaSuccess;
            };
            switch (dst[a].kind) {
            case SEG_CELL: CK(cp(S.c0, D.c0, D.nc)); break;
            case SEG_CELL4:
                for (int j = 0; j < 4; j++) CK(cp((size_t)j * S.NC + S.c0, (size_t)j * D.NC + D.c0, D.nc));
                break;
            case SEG_FACE: if (D.nf) CK(cp(S.f0, D.f0, D.nf)); break;
            default: if (D.nb) CK(cp(S.b0, D.b0, D.nb)); break;
            }
        }
    } else {
        S = {0, L->nc, 0, L->nf, 0, L->nb, L->nc, L->nf, 0};
        std::vector<std::vector<char>> keep;
        std::vector<const void*> from = seg_host(*L, keep);
        if (from.size() != dst.size()) return CSU_ERR_INPUT;
        CK(cudaStreamSynchronize(x->stream));
        for (size_t a = 0; a < dst.size(); a++) {
            const size_t es = dst[a].es;
            const char* h = (const char*)from[a];
            auto up = [&](size_t so, size_t dof, size_t n) {
                return cudaMemcpy(dst[a].dev + dof * es, h + so * es, n * es, cudaMemcpyHostToDevice);
            };
            switch (dst[a].kind) {
            case SEG_CELL: CK(up(0, D.c0, D.nc)); break;
            case SEG_CELL4:
                for (int j = 0; j < 4; j++) CK(up((size_t)j * S.NC, (size_t)j * D.NC + D.c0, D.nc));
                break;
            case SEG_FACE: if (D.nf) CK(up(0, D.f0, D.nf)); break;
            default: if (D.nb) CK(up(0, D.b0, D.nb)); break;
            }
        }
    }
    if (!src) return seg_fix(x, S, D);
    return CSU_OK;
}

// A pack of `solves`; with `old`, solve k with keep[k] >= 0 comes from solve keep[k] of `old` (its mesh rows
// and iteration state copied on the device), the others from their host layouts (initial state to be set).
static int pack_build(const char* who, const csu_prep* const* solves, int n, csu_ctx* old, const int* keep,
                      csu_ctx** out)
{
    if (!out) return CSU_ERR_INPUT;
    *out = nullptr;
    if (!solves || n < 1) {
        csu_set_error("%s: no solves", who);
        return CSU_ERR_INPUT;
    }
    for (int k = 0; k < n; k++) {
        if (!solves[k]) return CSU_ERR_INPUT;
        if (!same_structure(solves[0]->cfg, solves[k]->cfg)) {
            csu_set_error("%s: solve %d differs from solve 0 in a setting a pack shares (model, scheme, order, "
                          "time stepping, ...)", who, k);
            return CSU_ERR_INPUT;
        }
        if (old && keep && keep[k] >= 0) {
            if (keep[k] >= old->nsolve || old->ncs[keep[k]] != solves[k]->L.nc ||
                !same_structure(old->cfg, solves[k]->cfg)) {
                csu_set_error("%s: solve %d does not match solve %d of the old pack", who, k, keep[k]);
                return CSU_ERR_INPUT;
            }
        }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        csu_set_error("%s: no CUDA device", who);
        return CSU_ERR_NO_DEVICE;
    }
    // a pack's iterations return without waiting: the old pack's work must be done before it is read
    if (old) CK(cudaStreamSynchronize(old->stream));
    csu_ctx* x = new csu_ctx();
    x->model = solves[0]->model;
    x->nv = solves[0]->nv;
    x->cfg = solves[0]->cfg;
    x->nsolve = n;
    x->is_pack = true;
    x->pack_wall_d = solves[0]->L.wall_d != nullptr;
    x->cell0.resize(n);
    x->face0.resize(n);
    x->bface0.resize(n);
    x->prms.resize(n);
    x->ncs.resize(n);
    x->n2o.resize(n);
    memset(&x->L, 0, sizeof(x->L));
    x->max_ni = 1;
    for (int k = 0; k < n; k++) x->max_ni = std::max(x->max_ni, max_nint(solves[k]->L));
    int NC = 0, NF = 0, NB = 0, K = 0, walls = 0;
    std::vector<int> rank;
    for (int k = 0; k < n; k++) {
        const csu_layout& L = solves[k]->L;
        x->cell0[k] = NC;
        x->face0[k] = NF;
        x->bface0[k] = NB;
        NC += (L.nc + BLOCK - 1) / BLOCK * BLOCK;
        NF += L.nf;
        NB += L.nb;
        if (L.ncolors > K) K = L.ncolors;
        Prm& p = x->prms[k];
        fill_params_from(solves[k]->cfg, L, p);
        p.cell0 = x->cell0[k];
        p.blk0 = x->cell0[k] / BLOCK;
        p.nblk = (L.nc + BLOCK - 1) / BLOCK;
        rank.resize(L.nb + 1);
        p.wall0 = walls;
        p.nwall = local_wall_ranks(L, rank.data());
        walls += p.nwall;
        x->ncs[k] = L.nc;
        x->n2o[k].assign(L.cell_new2old, L.cell_new2old + L.nc);
    }
    x->L.nc = NC;
    x->L.nf = NF;
    x->L.nb = NB;
    x->nwall = walls;
    // colour lists over the pack (LU-SGS): same-colour cells of all solves together, ascending
    x->L.ncolors = K;
    x->L.color_start = (int*)calloc(K + 1, sizeof(int));
    std::vector<int> color_cells(NC > 0 ? NC : 1);
    for (int k = 0; k < n; k++)
        for (int c = 0; c < solves[k]->L.nc; c++) x->L.color_start[solves[k]->L.color[c] + 1]++;
    for (int q = 0; q < K; q++) x->L.color_start[q + 1] += x->L.color_start[q];
    {
        std::vector<int> fill(x->L.color_start, x->L.color_start + K + 1);
        for (int k = 0; k < n; k++)
            for (int c = 0; c < solves[k]->L.nc; c++) color_cells[fill[solves[k]->L.color[c]]++] = x->cell0[k] + c;
    }
    int st = ctx_setup(x);
    // mesh rows (kept solves: one batched device copy, then their re-basing), solve maps and colour lists
    CopyPlan plan;
    if (!st && old) {
        // the old pack's last iterations must be done before its rows are read from another stream
        cudaError_t e = cudaStreamSynchronize(old->stream);
        if (e != cudaSuccess) st = cuda_fail(e, "pack rebuild");
    }
    for (int k = 0; k < n && !st; k++) {
        bool kept = old && keep && keep[k] >= 0;
        st = kept ? seg_fill(x, k, nullptr, old, keep[k], &plan) : seg_fill(x, k, &solves[k]->L, nullptr, 0, &plan);
    }
    if (!st) st = run_copy_plan(x, plan);
    for (int k = 0; k < n && !st; k++)
        if (old && keep && keep[k] >= 0) st = seg_fix(x, seg_geo(old, keep[k]), seg_geo(x, k));
    if (!st) {
        int nblk = (NC + BLOCK - 1) / BLOCK;
        std::vector<int> bs(nblk, 0), cs(NC, 0);
        for (int k = 0; k < n; k++) {
            int c1 = k + 1 < n ? x->cell0[k + 1] : NC;
            for (int c = x->cell0[k]; c < c1; c++) cs[c] = k;
            for (int b = x->cell0[k] / BLOCK; b < (c1 + BLOCK - 1) / BLOCK; b++) bs[b] = k;
        }
        cudaError_t e = cudaStreamSynchronize(x->stream);
        if (e == cudaSuccess && n > 1) e = cudaMemcpy(const_cast<int*>(x->st.bsolve), bs.data(), sizeof(int) * nblk, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && n > 1) e = cudaMemcpy(const_cast<int*>(x->st.csolve), cs.data(), sizeof(int) * NC, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(const_cast<int*>(x->mesh.color_cells), color_cells.data(), sizeof(int) * NC,
                           cudaMemcpyHostToDevice);
        if (e != cudaSuccess) st = cuda_fail(e, "pack maps");
    }
    // iteration state of the kept solves: one batched copy, their scalars in one read and one write
    if (!st && old && keep) {
        std::vector<Scalars> ho(old->nsolve), hn(n);
        st = read_scalars_n(old, ho.data(), old->nsolve);
        if (!st) st = read_scalars_n(x, hn.data(), n);
        for (int k = 0; k < n && !st; k++) {
            if (keep[k] < 0) continue;
            state_copy_plan(old, keep[k], x, k, plan);
            Scalars h = ho[keep[k]];
            h.hist = hn[k].hist;
            h.hist_cap = hn[k].hist_cap;
            h.hist_row = 0;
            h.steps = 0;
            h.fresh = 0;
            hn[k] = h;
        }
        if (!st) st = run_copy_plan(x, plan);
        if (!st) st = write_scalars_n(x, hn.data(), n);
        x->prepared = 0;
    }
    if (st) {
        csu_destroy(x);
        return st;
    }
    *out = x;
    return CSU_OK;
}

extern "C" int csu_pack_create(const csu_prep* const* solves, int n, csu_ctx** out)
{
    return pack_build("csu_pack_create", solves, n, nullptr, nullptr, out);
}

extern "C" int csu_pack_rebuild(csu_ctx* old, const int* keep, const csu_prep* const* solves, int n, csu_ctx** out)
{
    if (!old || !old->is_pack || !keep) {
        csu_set_error("csu_pack_rebuild: an old pack and the keep map are required");
        return CSU_ERR_INPUT;
    }
    return pack_build("csu_pack_rebuild", solves, n, old, keep, out);
}
