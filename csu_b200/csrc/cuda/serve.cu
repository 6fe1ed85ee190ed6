// serve.cu -- continuous batching of steady solves on one GPU (no counterpart in the reference, which runs
// one case per process).
//
// Requests (a mesh, a configuration with its stopping drop, an initial state) queue on arrival. Each call of
// csu_srv_step (the caller's persistent request loop):
//   1. reads back the solves that converged (residual drop), failed (non-finite) or reached their
//      iteration cap; they stay frozen in their pack until its next rebuild;
//   2. admits queued requests, first fit in arrival order, while their device bytes fit the budget, into a
//      class whose pack may be rebuilt now (at most every `rebuild_steps` steps, or when it is empty);
//   3. rebuilds the packs with admissions: running solves move with their full iteration state
//      (csu_pack_transfer), so a solve's iterations are the same whatever joins or leaves; finished ones are
//      dropped and their bytes released; the new members start from their initial states;
//   4. advances every pack by `iters_per_step` iterations (CUDA graphs; one launch per kernel per
//      iteration for all members).
// A class is the set of settings a pack shares (model, scheme, order, time stepping, ...); requests of
// different classes run in separate packs, one after the other within a step.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "csu_gpu.h"

extern "C" void csu_set_error(const char* fmt, ...);
extern "C" void csu_pack_arena_release(void);

namespace {

struct Req;

struct Group {
    csu_config key;
    csu_ctx* pack = nullptr;
    std::vector<Req*> members; // in pack order (finished ones stay frozen until the next rebuild)
    std::vector<Req*> pending; // admitted, joining at the next rebuild
    int steps_since = 0;       // steps since the pack was built
    bool drop_now = false;     // a member was cancelled: rebuild without it at the next step
};

// A submitted mesh, owned by the request while a preparation thread builds its layout.
struct MeshCopy {
    std::vector<double> xy, wall;
    std::vector<int> npts, nodes, con, nint, faces, nei, mnbf, mflag, bface;
    csu_mesh_desc d;

    explicit MeshCopy(const csu_mesh_desc& m) : d(m)
    {
        const size_t nc = (size_t)m.n_cells, nf = (size_t)m.n_faces, nb = (size_t)m.n_bfaces;
        xy.assign(m.xy, m.xy + 2 * (size_t)m.n_points);
        npts.assign(m.cell_npts, m.cell_npts + nc);
        nodes.assign(m.cell_nodes, m.cell_nodes + 4 * nc);
        con.assign(m.con, m.con + 4 * nf);
        nint.assign(m.cell_nint, m.cell_nint + nc);
        faces.assign(m.cell_faces, m.cell_faces + 4 * nc);
        nei.assign(m.cell_nei, m.cell_nei + 4 * nc);
        mnbf.assign(m.marker_nbf, m.marker_nbf + m.n_markers);
        mflag.assign(m.marker_flag, m.marker_flag + m.n_markers);
        bface.assign(m.bface, m.bface + 3 * nb);
        if (m.wall_dist) wall.assign(m.wall_dist, m.wall_dist + nc);
        d.xy = xy.data();
        d.cell_npts = npts.data();
        d.cell_nodes = nodes.data();
        d.con = con.data();
        d.cell_nint = nint.data();
        d.cell_faces = faces.data();
        d.cell_nei = nei.data();
        d.marker_nbf = mnbf.data();
        d.marker_flag = mflag.data();
        d.bface = bface.data();
        d.wall_dist = m.wall_dist ? wall.data() : nullptr;
    }
};

struct Req {
    long long id = 0;
    csu_prep* prep = nullptr;
    MeshCopy* mesh = nullptr;  // while a preparation thread has it
    std::atomic<int> ready{1}; // 0 being prepared, 1 prepared, 2 preparation failed
    csu_config cfg;
    std::vector<double> U;     // initial state, then the final one
    int nv = 0, nc = 0;
    int max_iters = 0;
    int state = CSU_SRV_QUEUED;
    double t_submit = 0, t_start = 0, t_end = 0;
    int iters = 0;
    double drop = 0;
    double coef[4] = {0, 0, 0, 0};  // force coefficients of its last iteration
    long long bytes = 0;
    Group* group = nullptr;   // the group whose pack holds it (frozen there once finished)
    bool taken = false;       // result taken while still frozen in a pack: freed at the rebuild
    int status = CSU_OK;      // why it failed or stopped (CSU_ERR_*)
    char message[192] = {0};  // the failure's message, kept with the request (errors of a preparation
                              // thread are that thread's own csu_last_error)
};

void fail_req(Req* r, int status, const char* msg)
{
    r->status = status;
    snprintf(r->message, sizeof(r->message), "%s", msg ? msg : "");
}

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
    std::deque<long long> finished;  // ids that reached a final state, not yet polled
    std::vector<Group*> groups;
    long long used = 0;
    long long next_id = 1;
    long long iterations = 0;      // solve-iterations run (sum over members)
    long long cell_updates = 0;    // cells x iterations run
    double t_rebuild = 0, t_iterate = 0, t_poll = 0; // host seconds in the phases of csu_srv_step
    int rebuilds = 0;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    // preparation threads (prep_threads > 0)
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Req*> todo;
    bool stop = false;

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

// Builds a request's layout on a preparation thread; the step loop admits it once `ready` says so.
static void prepare(csu_srv* s, Req* r)
{
    csu_prep* p = nullptr;
    int st = csu_prep_create(&r->mesh->d, &r->cfg, &p);
    if (st) {
        fail_req(r, st, csu_last_error());
    } else if (csu_prep_bytes(p) > s->cfg.budget_bytes) {
        char msg[160];
        snprintf(msg, sizeof(msg), "the solve needs %lld device bytes, more than the budget of %lld",
                 csu_prep_bytes(p), s->cfg.budget_bytes);
        fail_req(r, CSU_ERR_OOM, msg);
        csu_prep_destroy(p);
        p = nullptr;
        st = CSU_ERR_OOM;
    }
    delete r->mesh;
    r->mesh = nullptr;
    r->prep = p;
    r->bytes = p ? csu_prep_bytes(p) : 0;
    r->ready.store(st ? 2 : 1, std::memory_order_release);
}

static void prep_worker(csu_srv* s)
{
    for (;;) {
        Req* r;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait(lk, [s] { return s->stop || !s->todo.empty(); });
            if (s->stop) return;
            r = s->todo.front();
            s->todo.pop_front();
        }
        prepare(s, r);
    }
}

extern "C" int csu_srv_submit(csu_srv* s, const csu_mesh_desc* mesh, const csu_config* cfg, const double* U0,
                              int max_iters, long long* id)
{
    if (!s || !mesh || !cfg || !U0 || max_iters < 1) return CSU_ERR_INPUT;
    csu_config c = *cfg;
    c.iter_cap = max_iters; // the pack freezes the solve at its cap, whatever the step length
    if (s->cfg.prep_threads > 0) {
        if (mesh->n_cells <= 0) return CSU_ERR_INPUT;
        Req* r = new Req();
        r->id = s->next_id++;
        r->cfg = c;
        r->nv = cfg->nvar;
        r->nc = mesh->n_cells;
        r->U.assign(U0, U0 + (size_t)r->nv * r->nc);
        r->max_iters = max_iters;
        r->t_submit = s->now();
        r->mesh = new MeshCopy(*mesh);
        r->ready.store(0, std::memory_order_relaxed);
        s->reqs[r->id] = r;
        s->queue.push_back(r);
        if (s->workers.empty())
            for (int k = 0; k < s->cfg.prep_threads; k++) s->workers.emplace_back(prep_worker, s);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->todo.push_back(r);
        }
        s->cv.notify_one();
        if (id) *id = r->id;
        return CSU_OK;
    }
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

// Marks the pack's solves that finished (converged, failed, capped): their states are read back; they
// stay frozen in the pack (holding their bytes) until the next rebuild drops them.
static int retire(csu_srv* s, Group* g)
{
    if (!g->pack) return CSU_OK;
    std::vector<csu_solve_info> infos(g->members.size());
    int st = csu_pack_infos(g->pack, infos.data());
    if (st) return st;
    for (size_t k = 0; k < g->members.size(); k++) {
        Req* r = g->members[k];
        if (r->state != CSU_SRV_RUNNING) continue;
        const csu_solve_info& info = infos[k];
        r->iters = info.iter;
        r->drop = info.have_res0 && info.res0[0] > 0 ? info.res[0] / info.res0[0] : 1.0;
        for (int q = 0; q < 4; q++) r->coef[q] = info.coef[q];
        int fin = info.status ? CSU_SRV_FAILED
                  : info.done == 1 ? CSU_SRV_CONVERGED
                  : (info.done == 2 || info.iter >= r->max_iters) ? CSU_SRV_MAXITER : 0;
        if (!fin) continue;
        if ((st = csu_pack_get_state(g->pack, (int)k, r->U.data()))) return st;
        r->state = fin;
        r->t_end = s->now();
        s->finished.push_back(r->id);
        if (fin == CSU_SRV_FAILED) {
            char msg[96];
            snprintf(msg, sizeof(msg), "the state became non-finite by iteration %d", info.iter);
            fail_req(r, info.status, msg);
        }
    }
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

static int active(const Group* g)
{
    int n = 0;
    for (const Req* r : g->members) n += r->state == CSU_SRV_RUNNING;
    return n;
}

// New pack of the group's running solves (moved with their iteration state) and the admitted ones (from
// their initial states); finished solves are dropped and their bytes released.
static int rebuild(csu_srv* s, Group* g)
{
    csu_ctx* old = g->pack;
    std::vector<Req*> old_members = g->members;
    std::vector<Req*> next;
    for (Req* r : old_members) {
        if (r->state == CSU_SRV_RUNNING) next.push_back(r);
        else {
            s->used -= r->bytes;
            if (r->prep) csu_prep_destroy(r->prep);
            r->prep = nullptr;
            r->group = nullptr;
            if (r->taken) delete r;
        }
    }
    for (Req* r : g->pending) next.push_back(r);
    g->pending.clear();
    g->members = next;
    g->pack = nullptr;
    g->steps_since = 0;
    int st = CSU_OK;
    if (!next.empty()) {
        std::vector<const csu_prep*> preps;
        for (Req* r : next) preps.push_back(r->prep);
        // running solves move on the device (mesh rows and iteration state); new ones are uploaded
        std::vector<int> keep(next.size(), -1);
        for (size_t k = 0; k < next.size(); k++) {
            auto it = std::find(old_members.begin(), old_members.end(), next[k]);
            if (old && it != old_members.end()) keep[k] = (int)(it - old_members.begin());
        }
        st = old ? csu_pack_rebuild(old, keep.data(), preps.data(), (int)preps.size(), &g->pack)
                 : csu_pack_create(preps.data(), (int)preps.size(), &g->pack);
        if (st) {
            if (old) csu_destroy(old);
            return st;
        }
        for (size_t k = 0; k < next.size() && !st; k++)
            if (keep[k] < 0) st = csu_pack_set_state(g->pack, (int)k, next[k]->U.data());
    }
    if (old) csu_destroy(old);
    return st;
}

extern "C" int csu_srv_step(csu_srv* s, int* n_running, int* n_queued)
{
    if (!s) return CSU_ERR_INPUT;
    int st;
    // 1. finished solves
    double t = s->now();
    for (Group* g : s->groups)
        if ((st = retire(s, g))) return st;
    s->t_poll += s->now() - t;
    // 2. admit, first fit in arrival order, into groups whose pack may be rebuilt now
    const int every = s->cfg.rebuild_steps > 1 ? s->cfg.rebuild_steps : 1;
    for (auto it = s->queue.begin(); it != s->queue.end();) {
        Req* r = *it;
        const int rd = r->ready.load(std::memory_order_acquire);
        if (rd == 0) { // still being prepared
            ++it;
            continue;
        }
        if (r->state == CSU_SRV_CANCELLED) {
            it = s->queue.erase(it);
            continue;
        }
        if (rd == 2) { // its layout failed or it exceeds the budget (status and message set by prepare)
            r->state = CSU_SRV_FAILED;
            r->t_start = r->t_end = s->now();
            s->finished.push_back(r->id);
            it = s->queue.erase(it);
            continue;
        }
        Group* g = group_for(s, r->cfg);
        bool window = !g->pack || active(g) == 0 || g->steps_since >= every;
        int size = active(g) + (int)g->pending.size();
        if (window && s->used + r->bytes <= s->cfg.budget_bytes && size < s->cfg.max_pack) {
            s->used += r->bytes;
            r->state = CSU_SRV_RUNNING;
            r->t_start = s->now();
            r->group = g;
            g->pending.push_back(r);
            it = s->queue.erase(it);
        } else {
            ++it;
        }
    }
    // 3. rebuild packs with admissions, and packs whose solves all finished
    t = s->now();
    for (Group* g : s->groups) {
        bool idle = g->pack && active(g) == 0;
        if (!g->pending.empty() || idle || g->drop_now) {
            g->drop_now = false;
            if ((st = rebuild(s, g))) return st;
            s->rebuilds++;
        }
    }
    s->t_rebuild += s->now() - t;
    // 4. advance
    t = s->now();
    int running = 0;
    for (Group* g : s->groups) {
        if (!g->pack) continue;
        if ((st = csu_iterate(g->pack, s->cfg.iters_per_step, 0, nullptr))) return st;
        g->steps_since++;
        for (Req* r : g->members) {
            if (r->state != CSU_SRV_RUNNING) continue;
            running++;
            s->cell_updates += (long long)r->nc * s->cfg.iters_per_step;
            s->iterations += s->cfg.iters_per_step;
        }
    }
    s->t_iterate += s->now() - t;
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
    out->status = r->status;
    for (int q = 0; q < 4; q++) out->coef[q] = r->coef[q];
    return CSU_OK;
}

extern "C" int csu_srv_message(csu_srv* s, long long id, char* buf, int cap)
{
    if (!s || !buf || cap < 1) return CSU_ERR_INPUT;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) {
        csu_set_error("csu_srv_message: no request %lld", id);
        return CSU_ERR_INPUT;
    }
    snprintf(buf, (size_t)cap, "%s", it->second->message);
    return CSU_OK;
}

extern "C" int csu_srv_poll(csu_srv* s, long long* ids, int cap, int* n)
{
    if (!s || !n || cap < 0 || (cap > 0 && !ids)) return CSU_ERR_INPUT;
    int k = 0;
    while (k < cap && !s->finished.empty()) {
        ids[k++] = s->finished.front();
        s->finished.pop_front();
    }
    *n = k;
    return CSU_OK;
}

extern "C" int csu_srv_cancel(csu_srv* s, long long id)
{
    if (!s) return CSU_ERR_INPUT;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) {
        csu_set_error("csu_srv_cancel: no request %lld", id);
        return CSU_ERR_INPUT;
    }
    Req* r = it->second;
    if (r->state != CSU_SRV_QUEUED && r->state != CSU_SRV_RUNNING) {
        csu_set_error("csu_srv_cancel: request %lld has already finished", id);
        return CSU_ERR_STATE;
    }
    Group* g = r->group;
    if (r->state == CSU_SRV_RUNNING && g) {
        auto pit = std::find(g->pending.begin(), g->pending.end(), r);
        if (pit != g->pending.end()) {
            // admitted, not in a pack yet: its bytes go back now, its state is still the initial one
            g->pending.erase(pit);
            s->used -= r->bytes;
            r->group = nullptr;
        } else {
            // in the pack: its state as it stands, then frozen there until the rebuild at the next step
            auto mit = std::find(g->members.begin(), g->members.end(), r);
            if (mit != g->members.end() && g->pack) {
                const int k = (int)(mit - g->members.begin());
                int st = csu_pack_stop(g->pack, k);
                if (!st) st = csu_pack_get_state(g->pack, k, r->U.data());
                if (!st) {
                    csu_solve_info info;
                    if (!(st = csu_pack_info(g->pack, k, &info))) r->iters = info.iter;
                }
                if (st) return st;
            }
            g->drop_now = true;
        }
    }
    // a queued request leaves the queue at the next step (a preparation thread may still hold it)
    r->state = CSU_SRV_CANCELLED;
    r->t_end = s->now();
    s->finished.push_back(r->id);
    if (r->t_start == 0) r->t_start = r->t_end;
    fail_req(r, CSU_ERR_CANCELLED, "cancelled by the caller");
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
    // a request cancelled while a preparation thread builds its layout: wait for the thread to let go of it
    while (r->ready.load(std::memory_order_acquire) == 0) std::this_thread::sleep_for(std::chrono::microseconds(200));
    if (U) memcpy(U, r->U.data(), sizeof(double) * r->U.size());
    s->reqs.erase(it);
    s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), r), s->queue.end());
    if (r->group) {
        r->taken = true; // still frozen in a pack: released when the pack is rebuilt
    } else {
        if (r->prep) csu_prep_destroy(r->prep);
        delete r;
    }
    return CSU_OK;
}

extern "C" int csu_srv_times(csu_srv* s, double* rebuild_s, double* iterate_s, double* poll_s, int* rebuilds)
{
    if (!s) return CSU_ERR_INPUT;
    if (rebuild_s) *rebuild_s = s->t_rebuild;
    if (iterate_s) *iterate_s = s->t_iterate;
    if (poll_s) *poll_s = s->t_poll;
    if (rebuilds) *rebuilds = s->rebuilds;
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
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->todo.clear();
        s->stop = true;
    }
    s->cv.notify_all();
    for (std::thread& t : s->workers) t.join();
    for (Group* g : s->groups) {
        for (Req* r : g->members)
            if (r->taken) {
                if (r->prep) csu_prep_destroy(r->prep);
                delete r;
            }
        if (g->pack) csu_destroy(g->pack);
        delete g;
    }
    for (auto& kv : s->reqs) {
        if (kv.second->prep) csu_prep_destroy(kv.second->prep);
        delete kv.second->mesh;
        delete kv.second;
    }
    csu_pack_arena_release();
    delete s;
}
