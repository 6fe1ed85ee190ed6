// serve.cu -- continuous batching of steady solves on one GPU (no counterpart in the reference, which runs
// one case per process).
//
// Requests (a mesh, a configuration with its stopping drop, an initial state) queue on arrival. Each call of
// csu_srv_step (the caller's persistent request loop):
//   1. retires the running solves that converged (residual drop), failed (non-finite) or reached their
//      iteration cap, and keeps their final states until taken;
//   2. admits queued requests, first fit in arrival order, while their device bytes fit the budget;
//   3. rebuilds the pack of every class whose membership changed: the continuing solves move with their
//      full iteration state (csu_pack_transfer), so a solve's iterations are the same whatever joins or
//      leaves; the new members start from their initial states;
//   4. advances every pack by `iters_per_step` iterations (CUDA graphs; one launch per kernel per
//      iteration for all members).
// A class is the set of settings a pack shares (model, scheme, order, time stepping, ...); requests of
// different classes run in separate packs, one after the other within a step.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <vector>

#include "csu_gpu.h"

extern "C" void csu_set_error(const char* fmt, ...);

namespace {

struct Req;

struct Group {
    csu_config key;
    csu_ctx* pack = nullptr;
    std::vector<Req*> members; // in pack order
    bool dirty = false;
};

struct Req {
    long long id = 0;
    csu_prep* prep = nullptr;
    csu_config cfg;
    std::vector<double> U;     // initial state, then the final one
    int nv = 0, nc = 0;
    int max_iters = 0;
    int state = CSU_SRV_QUEUED;
    double t_submit = 0, t_start = 0, t_end = 0;
    int iters = 0;
    double drop = 0;
    long long bytes = 0;
    Group* group = nullptr;
};

bool same_class(const csu_config& a, const csu_config& b)
{
    return a.nvar == b.nvar && a.order == b.order && a.flux == b.flux && a.stages == b.stages &&
           a.time_scheme == b.time_scheme && a.n_linear == b.n_linear && a.dt_local == b.dt_local &&
           a.dt_local_n == b.dt_local_n && a.laminar == b.laminar && a.sa == b.sa && a.sa_cc == b.sa_cc &&
           a.sst == b.sst && a.sst_trans == b.sst_trans && a.axisymmetric == b.axisymmetric &&
           a.turb1order == b.turb1order && a.visc_blazek == b.visc_blazek && a.tp == b.tp &&
           a.limiter_type == b.limiter_type && a.tube == b.tube && a.implicit_fp32 == b.implicit_fp32 &&
           a.implicit_local_dt == b.implicit_local_dt;
}

} // namespace

struct csu_srv {
    csu_srv_config cfg;
    std::map<long long, Req*> reqs;
    std::deque<Req*> queue;
    std::vector<Group*> groups;
    long long used = 0;
    long long next_id = 1;
    long long iterations = 0;      // solve-iterations run (sum over members)
    long long cell_updates = 0;    // cells x iterations run
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

    double now() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

extern "C" int csu_srv_create(const csu_srv_config* cfg, csu_srv** out)
{
    if (!cfg || !out || cfg->budget_bytes <= 0 || cfg->iters_per_step < 1) {
        csu_set_error("csu_srv_create: a positive budget and iterations per step are required");
        return CSU_ERR_INPUT;
    }
    csu_srv* s = new csu_srv();
    s->cfg = *cfg;
    if (s->cfg.max_pack < 1) s->cfg.max_pack = 1 << 20;
    *out = s;
    return CSU_OK;
}

extern "C" int csu_srv_submit(csu_srv* s, const csu_mesh_desc* mesh, const csu_config* cfg, const double* U0,
                              int max_iters, long long* id)
{
    if (!s || !mesh || !cfg || !U0 || max_iters < 1) return CSU_ERR_INPUT;
    csu_config c = *cfg;
    c.iter_cap = max_iters; // the pack freezes the solve at its cap, whatever the step length
    csu_prep* p = nullptr;
    int st = csu_prep_create(mesh, &c, &p);
    if (st) return st;
    long long need = csu_prep_bytes(p);
    if (need > s->cfg.budget_bytes) {
        csu_prep_destroy(p);
        csu_set_error("csu_srv_submit: the solve needs %lld bytes, more than the budget", need);
        return CSU_ERR_OOM;
    }
    Req* r = new Req();
    r->id = s->next_id++;
    r->prep = p;
    r->cfg = c;
    r->nv = cfg->nvar;
    r->nc = mesh->n_cells;
    r->U.assign(U0, U0 + (size_t)r->nv * r->nc);
    r->max_iters = max_iters;
    r->bytes = csu_prep_bytes(p);
    r->t_submit = s->now();
    s->reqs[r->id] = r;
    s->queue.push_back(r);
    if (id) *id = r->id;
    return CSU_OK;
}

static int retire(csu_srv* s, Group* g)
{
    if (!g->pack) return CSU_OK;
    std::vector<Req*> keep;
    for (size_t k = 0; k < g->members.size(); k++) {
        Req* r = g->members[k];
        csu_solve_info info;
        int st = csu_pack_info(g->pack, (int)k, &info);
        if (st) return st;
        r->iters = info.iter;
        r->drop = info.have_res0 && info.res0[0] > 0 ? info.res[0] / info.res0[0] : 1.0;
        int fin = info.status ? CSU_SRV_FAILED
                  : info.done == 1 ? CSU_SRV_CONVERGED
                  : (info.done == 2 || info.iter >= r->max_iters) ? CSU_SRV_MAXITER : 0;
        if (!fin) {
            keep.push_back(r);
            continue;
        }
        if ((st = csu_pack_get_state(g->pack, (int)k, r->U.data()))) return st;
        r->state = fin;
        r->t_end = s->now();
        r->group = nullptr;
        s->used -= r->bytes;
        csu_prep_destroy(r->prep);
        r->prep = nullptr;
        g->dirty = true;
    }
    // the retired solves' slots are released when the pack is rebuilt
    if (g->dirty) g->members = keep;
    return CSU_OK;
}

static Group* group_for(csu_srv* s, const csu_config& c)
{
    for (Group* g : s->groups)
        if (same_class(g->key, c)) return g;
    Group* g = new Group();
    g->key = c;
    s->groups.push_back(g);
    return g;
}

static int rebuild(csu_srv* s, Group* g, const std::vector<Req*>& old_members)
{
    csu_ctx* old = g->pack;
    g->pack = nullptr;
    int st = CSU_OK;
    if (!g->members.empty()) {
        std::vector<const csu_prep*> preps;
        for (Req* r : g->members) preps.push_back(r->prep);
        if ((st = csu_pack_create(preps.data(), (int)preps.size(), &g->pack))) {
            if (old) csu_destroy(old);
            return st;
        }
        for (size_t k = 0; k < g->members.size(); k++) {
            Req* r = g->members[k];
            auto it = std::find(old_members.begin(), old_members.end(), r);
            if (old && it != old_members.end()) {
                st = csu_pack_transfer(old, (int)(it - old_members.begin()), g->pack, (int)k);
            } else {
                st = csu_pack_set_state(g->pack, (int)k, r->U.data());
            }
            if (st) break;
        }
    }
    if (old) csu_destroy(old);
    g->dirty = false;
    (void)s;
    return st;
}

extern "C" int csu_srv_step(csu_srv* s, int* n_running, int* n_queued)
{
    if (!s) return CSU_ERR_INPUT;
    int st;
    // 1. retire (member lists of the old packs are kept for the transfers below)
    std::map<Group*, std::vector<Req*>> before;
    for (Group* g : s->groups) {
        before[g] = g->members;
        if ((st = retire(s, g))) return st;
    }
    // 2. admit, first fit in arrival order
    for (auto it = s->queue.begin(); it != s->queue.end();) {
        Req* r = *it;
        Group* g = group_for(s, r->cfg);
        if (s->used + r->bytes <= s->cfg.budget_bytes && (int)g->members.size() < s->cfg.max_pack) {
            s->used += r->bytes;
            r->state = CSU_SRV_RUNNING;
            r->t_start = s->now();
            r->group = g;
            g->members.push_back(r);
            g->dirty = true;
            it = s->queue.erase(it);
        } else {
            ++it;
        }
    }
    // 3. rebuild changed packs
    for (Group* g : s->groups)
        if (g->dirty && (st = rebuild(s, g, before[g]))) return st;
    // 4. advance
    int running = 0;
    for (Group* g : s->groups) {
        if (!g->pack) continue;
        if ((st = csu_iterate(g->pack, s->cfg.iters_per_step, 0, nullptr))) return st;
        running += (int)g->members.size();
        for (Req* r : g->members) s->cell_updates += (long long)r->nc * s->cfg.iters_per_step;
        s->iterations += (long long)g->members.size() * s->cfg.iters_per_step;
    }
    if (n_running) *n_running = running;
    if (n_queued) *n_queued = (int)s->queue.size();
    return CSU_OK;
}

extern "C" int csu_srv_info(csu_srv* s, long long id, csu_srv_request_info* out)
{
    if (!s || !out) return CSU_ERR_INPUT;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) {
        csu_set_error("csu_srv_info: no request %lld", id);
        return CSU_ERR_INPUT;
    }
    const Req* r = it->second;
    out->state = r->state;
    out->iters = r->iters;
    out->drop = r->drop;
    out->t_submit = r->t_submit;
    out->t_start = r->t_start;
    out->t_end = r->t_end;
    out->n_cells = r->nc;
    return CSU_OK;
}

extern "C" int csu_srv_take(csu_srv* s, long long id, double* U)
{
    if (!s) return CSU_ERR_INPUT;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return CSU_ERR_INPUT;
    Req* r = it->second;
    if (r->state == CSU_SRV_QUEUED || r->state == CSU_SRV_RUNNING) {
        csu_set_error("csu_srv_take: request %lld has not finished", id);
        return CSU_ERR_STATE;
    }
    if (U) memcpy(U, r->U.data(), sizeof(double) * r->U.size());
    delete r;
    s->reqs.erase(it);
    return CSU_OK;
}

extern "C" int csu_srv_totals(csu_srv* s, long long* solve_iterations, long long* cell_updates, long long* used_bytes)
{
    if (!s) return CSU_ERR_INPUT;
    if (solve_iterations) *solve_iterations = s->iterations;
    if (cell_updates) *cell_updates = s->cell_updates;
    if (used_bytes) *used_bytes = s->used;
    return CSU_OK;
}

extern "C" void csu_srv_destroy(csu_srv* s)
{
    if (!s) return;
    for (Group* g : s->groups) {
        if (g->pack) csu_destroy(g->pack);
        delete g;
    }
    for (auto& kv : s->reqs) {
        if (kv.second->prep) csu_prep_destroy(kv.second->prep);
        delete kv.second;
    }
    delete s;
}
