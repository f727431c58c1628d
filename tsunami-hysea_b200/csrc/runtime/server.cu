// Multi-scenario runtime: many scenarios stepped together by one batch (one
// work list over all their tiles, one CUDA graph of step chunks), admitted
// from a queue under an HBM budget, retired as they finish (continuous
// batching).  Drives the same kernels and control blocks as thy_run; each
// scenario's arithmetic is independent of the others, so a result is the
// same alone and in any mix.
//
// The reference runs one scenario per process (src/ShallowWater.cxx:146-151
// calls shallowWater() once); this is the batched / serving layer above it.
#include "engine.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <memory>

namespace thy {

int handle_events_ex(DevScenario &s, const thy_outputs *o, cudaStream_t st, bool *changed);

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    long long id = 0;
    const thy_problem *p = nullptr;
    const thy_outputs *o = nullptr;
    thy_done_fn done = nullptr;
    void *user = nullptr;
    size_t bytes = 0;
    Clock::time_point submitted;
};

struct Active {
    Request r;
    std::unique_ptr<DevScenario> s;
    bool fresh = true;            // admitted, its first events not handled yet
    bool cancelled = false;
    bool deferred = false;        // resident but not stepped in the coming chunk
    Clock::time_point admitted;
};

}  // namespace
}  // namespace thy

struct thy_server {
    cudaStream_t st = nullptr;
    thy::Batch b;
    size_t budget = 0, in_use = 0;
    long long chunk_cells = 0;    // < 0: step every resident scenario
    long long next_id = 1;
    std::deque<thy::Request> queue;
    std::vector<thy::Active *> slots;     // by batch slot
    bool members_changed = false;
    bool alone = false;                   // the last chunk stepped one large request alone
    std::vector<char> selected;           // by batch slot: stepped in the last chunk (its work list)
    thy_server_stats stats{};
};

using namespace thy;

static size_t request_bytes(const thy_problem *p)
{
    return scenario_bytes(p->nx, p->ny, p->nfaults > 0) + sizeof(ScenarioCtl);
}

static void complete(thy_server *S, int slot, int status)
{
    Active *a = S->slots[slot];
    DevScenario &s = *a->s;
    thy_stats st{};
    st.steps = s.hctl.step;
    st.final_time_s = s.hctl.t * s.Ts;
    st.first_dt_s = s.first_dt_s;
    st.snapshots = s.snapshots;
    st.series_samples = s.series;
    st.tiles = s.hctl.step * s.units();
    st.deep_tiles = (long long)s.hctl.units_deep;
    st.dry_tiles = (long long)s.hctl.units_dry;
    st.tiling = thy_tiling{S->b.tiling.deep1, S->b.tiling.deep2, S->b.tiling.general};
    st.tune_samples = S->b.tune_samples;   // of the batch, so far
    if (status == THY_OK && a->r.o) {
        const auto t0 = Clock::now();
        status = s.finish(a->r.o, S->st);
        st.output_seconds = std::chrono::duration<double>(Clock::now() - t0).count();
    }
    st.loop_seconds = std::chrono::duration<double>(Clock::now() - a->admitted).count();
    st.total_seconds = std::chrono::duration<double>(Clock::now() - a->r.submitted).count();
    st.setup_seconds = std::chrono::duration<double>(a->admitted - a->r.submitted).count();   // queueing
    S->b.detach(&s);
    S->in_use -= a->r.bytes;
    if (status == THY_OK) S->stats.completed++;
    else if (status == THY_ERR_CANCELLED) S->stats.cancelled++;
    else S->stats.failed++;
    S->stats.cell_updates += (double)s.nx * s.ny * (double)s.hctl.step;
    const Request r = a->r;
    S->slots[slot] = nullptr;
    delete a;
    S->members_changed = true;
    if (r.done) r.done(r.user, r.id, status, &st);
}

// Admits queued requests in order while they fit the budget and a slot: all
// of them into an empty server, one a round otherwise (the set-up of each -
// uploads, table, initial dt - holds the stepping thread, so a queue that
// built up behind a large request joins one request a chunk, the first one
// stepping as soon as it is set up).
static int admit(thy_server *S)
{
    bool resident = false;
    for (auto *a : S->slots) resident |= a != nullptr;
    for (int n = 0; !S->queue.empty() && !(resident && n >= 1); n++) {
        Request &r = S->queue.front();
        if (S->in_use + r.bytes > S->budget && S->in_use > 0) break;   // wait for memory (an empty server admits anyway)
        int slot = -1;
        for (int i = 0; i < S->b.capacity; i++)
            if (!S->slots[i]) { slot = i; break; }
        if (slot < 0) break;
        Active *a = new Active();
        a->r = r;
        a->s.reset(new DevScenario());
        a->admitted = Clock::now();
        S->queue.pop_front();
        S->slots[slot] = a;
        S->in_use += a->r.bytes;
        S->stats.admitted++;
        int rc = S->b.attach(a->s.get());
        if (rc == THY_OK) rc = a->s->setup(a->r.p, S->st);
        a->s->desc.ctl = a->s->ctl;
        if (rc == THY_OK) rc = S->b.update();
        if (rc == THY_OK) rc = S->b.initial_dt_of(a->s.get());
        if (rc != THY_OK) {
            cudaGetLastError();
            complete(S, slot, rc);
            continue;
        }
        S->members_changed = true;
    }
    return THY_OK;
}

extern "C" int thy_server_open(const thy_server_opts *opts, thy_server **out)
{
    if (!out) return THY_ERR_INVALID;
    *out = nullptr;
    thy_server_opts o{};
    if (opts) o = *opts;
    if (o.device < 0) return THY_ERR_INVALID;
    if (opts) thy_set_device(o.device);
    int rc = ensure_device();
    if (rc) return rc;
    size_t free_b = 0, total_b = 0;
    THY_CK(cudaMemGetInfo(&free_b, &total_b));
    thy_server *S = new thy_server();
    S->budget = o.hbm_budget_bytes ? (size_t)o.hbm_budget_bytes : free_b / 10 * 9;
    // by default one 4096^2 grid's cells: enough work to fill the GPU, and a
    // large request runs alone at its own speed instead of sharing its steps
    S->chunk_cells = o.chunk_cells ? o.chunk_cells : 1ll << 24;
    const int cap = o.max_scenarios > 0 ? o.max_scenarios : 256;
    // work-list capacity: the tiles of the budget's worth of cells, at least one grid of 4096^2
    const size_t cells = S->budget / 40 + (size_t)4096 * 4096;
    const int items = (int)std::min<size_t>(cells / (kTileX * kTileY) + 1024, (size_t)1 << 26);
    if ((rc = cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking) == cudaSuccess ? THY_OK : THY_ERR_CUDA) ||
        (rc = S->b.init(cap, items, S->st)) || (rc = S->b.rebuild())) {
        cudaStream_t st = S->st;
        delete S;
        if (st) cudaStreamDestroy(st);
        return rc;
    }
    S->slots.assign(cap, nullptr);
    *out = S;
    return THY_OK;
}

extern "C" int thy_server_submit(thy_server *S, const thy_problem *p, const thy_outputs *o, thy_done_fn done,
                                 void *user, long long *request)
{
    if (!S || !p || p->nx < 2 || p->ny < 2 || !p->h || !p->Hs) return THY_ERR_INVALID;
    const size_t need = request_bytes(p);
    if (need > S->budget) {
        S->stats.rejected++;
        return THY_ERR_BUDGET;
    }
    Request r;
    r.id = S->next_id++;
    r.p = p;
    r.o = o;
    r.done = done;
    r.user = user;
    r.bytes = need;
    r.submitted = Clock::now();
    S->queue.push_back(r);
    S->stats.submitted++;
    if (request) *request = r.id;
    return THY_OK;
}

extern "C" int thy_server_cancel(thy_server *S, long long request)
{
    if (!S) return THY_ERR_INVALID;
    for (auto it = S->queue.begin(); it != S->queue.end(); ++it)
        if (it->id == request) {
            const Request r = *it;
            S->queue.erase(it);
            S->stats.cancelled++;
            if (r.done) r.done(r.user, r.id, THY_ERR_CANCELLED, nullptr);
            return THY_OK;
        }
    for (auto *a : S->slots)
        if (a && a->r.id == request) {
            a->cancelled = true;   // retired at the next progress, between chunks
            return THY_OK;
        }
    return THY_ERR_INVALID;
}

// One round: admit, perform due events, run one chunk of steps for the
// scenarios the chunk's work budget selects, retire the finished, cancelled
// and failed ones.
extern "C" int thy_server_progress(thy_server *S, int *active)
{
    if (!S) return THY_ERR_INVALID;
    int rc;
    // while a large request runs alone, new requests wait in the queue: their
    // set-up (uploads, Okada) would hold up its chunks, and none of them
    // could be stepped before it ends
    if (!S->alone && (rc = admit(S))) return rc;
    const int cap = S->b.capacity;
    bool state_changed = false, any_running = false;
    for (int i = 0; i < cap; i++) {
        Active *a = S->slots[i];
        if (!a) continue;
        DevScenario &s = *a->s;
        if (a->cancelled) {
            complete(S, i, THY_ERR_CANCELLED);
            continue;
        }
        if (s.hctl.status == kFailed) {
            complete(S, i, failure_code(s.hctl));
            continue;
        }
        const bool ended = !(s.hctl.t < s.t_end) || (s.max_steps >= 0 && s.hctl.step >= s.max_steps);
        if (ended) {
            complete(S, i, THY_OK);
            continue;
        }
        if (a->fresh || (s.hctl.status != kRunning && !a->deferred)) {
            bool changed = false;
            if ((rc = handle_events_ex(s, a->r.o, S->st, &changed))) {
                complete(S, i, rc);
                continue;
            }
            state_changed |= changed;
            a->fresh = false;
            s.hctl.status = kRunning;
            s.hctl.events = 0;
            a->deferred = false;
            if ((rc = s.upload_ctl(S->st))) return rc;
        }
        any_running = true;
    }
    // Work budget of the chunk: the resident scenario submitted first, then
    // those with the least remaining work (cells x remaining steps at the
    // current dt), are stepped until their cells reach chunk_cells; the
    // others wait (status idle on the device, and their tiles are not on the
    // chunk's work list).  Small requests are batched, a large one runs
    // alone, and no request's arithmetic changes.
    std::vector<char> sel(cap, 0);
    S->alone = false;
    if (any_running) {
        // the request submitted first is always stepped (so that no request
        // waits behind a stream of smaller ones: the tail of time-to-result),
        // the others by least remaining work
        std::vector<std::pair<double, int>> order;
        int first = -1;
        for (int i = 0; i < cap; i++) {
            Active *a = S->slots[i];
            if (!a) continue;
            if (first < 0 || a->r.submitted < S->slots[first]->r.submitted) first = i;
        }
        for (int i = 0; i < cap; i++) {
            Active *a = S->slots[i];
            if (!a) continue;
            const DevScenario &s = *a->s;
            const double cells = (double)s.nx * s.ny;
            const double steps = s.hctl.dt > 0.0 ? (s.t_end - s.hctl.t) / s.hctl.dt : 0.0;
            order.emplace_back(i == first ? -1.0 : cells * std::max(steps, 1.0), i);
        }
        std::sort(order.begin(), order.end());
        // a large request (at least half the chunk's cells) is stepped only
        // when it was submitted first, and then alone, so that it runs at its
        // own speed as in first-come-first-served; smaller ones are batched
        double taken = 0.0;
        const double big = S->chunk_cells < 0 ? 1e300 : 0.5 * (double)S->chunk_cells;
        bool alone = false;
        for (const auto &e : order) {
            Active *a = S->slots[e.second];
            DevScenario &s = *a->s;
            const double cells = (double)s.nx * s.ny;
            bool step = !alone && (S->chunk_cells < 0 || taken < (double)S->chunk_cells);
            if (step && cells >= big) {
                if (e.second == first) alone = S->alone = true;
                else step = false;
            }
            if (step) taken += cells;
            sel[e.second] = step ? 1 : 0;
            const int want = step ? kRunning : kIdle;
            if (s.hctl.status != want || a->deferred == step) {
                s.hctl.status = want;
                a->deferred = !step;
                if ((rc = s.upload_ctl(S->st))) return rc;
            }
        }
    }
    if (S->members_changed || sel != S->selected) {
        // table + the work list of the stepped scenarios, classified for their current states
        if ((rc = S->b.update(&sel))) return rc;
        if (!S->b.gexec && (rc = S->b.capture())) return rc;   // the list outgrew its capacity
        S->members_changed = false;
        S->selected = sel;
    } else if (state_changed) {
        if ((rc = S->b.reset_lists())) return rc;
    }
    if (any_running) {
        // no longer than the steps the first stepped scenario has left
        // before an event or its end, so that it is handled (and a finished
        // one retired, its slot and memory free) without idle launches
        long long horizon = S->b.chunk;
        for (int i = 0; i < cap; i++)
            if (S->slots[i] && sel[i]) horizon = std::min(horizon, Batch::steps_to_event(*S->slots[i]->s));
        if ((rc = S->b.run_chunk(true, S->b.chunk_for(horizon)))) return rc;
        S->stats.chunks++;
        // hand on the gauge samples the chunk took; retire what finished in
        // this chunk right away
        for (int i = 0; i < cap; i++) {
            Active *a = S->slots[i];
            if (!a) continue;
            DevScenario &s = *a->s;
            if ((rc = s.read_device_gauges(a->r.o, S->st))) {
                complete(S, i, rc);
                continue;
            }
            if (s.hctl.status == kFailed) complete(S, i, failure_code(s.hctl));
            else if (!(s.hctl.t < s.t_end) || (s.max_steps >= 0 && s.hctl.step >= s.max_steps))
                complete(S, i, THY_OK);
        }
    }
    S->stats.device_ms = S->b.device_ms;
    int n = (int)S->queue.size();
    for (auto *a : S->slots) n += a ? 1 : 0;
    if (active) *active = n;
    return THY_OK;
}

extern "C" int thy_server_drain(thy_server *S)
{
    int active = 1, rc;
    while (active > 0)
        if ((rc = thy_server_progress(S, &active))) return rc;
    return THY_OK;
}

extern "C" int thy_server_get_stats(const thy_server *S, thy_server_stats *out)
{
    if (!S || !out) return THY_ERR_INVALID;
    *out = S->stats;
    out->queued = (int)S->queue.size();
    int n = 0;
    for (auto *a : S->slots) n += a ? 1 : 0;
    out->running = n;
    out->hbm_in_use = (long long)S->in_use;
    out->hbm_budget = (long long)S->budget;
    return THY_OK;
}

extern "C" void thy_server_close(thy_server *S)
{
    if (!S) return;
    for (int i = 0; i < (int)S->slots.size(); i++)
        if (S->slots[i]) complete(S, i, THY_ERR_CANCELLED);
    while (!S->queue.empty()) {
        const Request r = S->queue.front();
        S->queue.pop_front();
        if (r.done) r.done(r.user, r.id, THY_ERR_CANCELLED, nullptr);
    }
    cudaStream_t st = S->st;
    delete S;
    if (st) cudaStreamDestroy(st);
}
