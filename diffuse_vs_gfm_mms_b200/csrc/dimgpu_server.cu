// dimgpu_server.cu — the continuous-batching serving loop behind the C-ABI
// (include/dimgpu.h: dimgpu_server_*).
//
// Requests (a grid, its initial state, a step budget) are submitted from any
// host thread and queue in arrival order.  A server thread drives two kinds
// of lanes, each on its own CUDA stream:
//
//   batch lanes  one per (material count, dimension) group: an arena-mode
//                dimgpu_batch whose device memory was reserved once, holding
//                the group's small solves;
//   solo lanes   `solo_slots` session shells for solves of at least
//                `solo_min_cells` cells, which fill the GPU on their own and
//                run fastest as one grid (the staged single-grid sweep); their
//                state and scratch are ranges of one solo arena, also
//                reserved once.
//
// The loop never waits for all lanes together: a lane whose quantum (a few
// steps, enqueued as one unit) has finished — found by an event query, no
// host synchronisation — retires its finished solves, takes in queued ones
// and gets its next quantum at once, while the other lanes keep running.
// Admission is first come first served per lane kind and group and neither
// allocates nor synchronises; a solve that does not fit waits for room
// (later solves of other lanes may go ahead).
//
// Every solve's arithmetic is the single-grid step's: a result does not
// depend on the lane or on what else was resident.  Latency is measured on
// the host from submission to the completion of the quantum in which the
// solve finished.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "dim_launch.h"
#include "dimgpu.h"
#include "dimgpu_session.h"
#include "range_alloc.h"

using namespace dimgpu;

namespace {

using Clock = std::chrono::steady_clock;

constexpr int kSoloHistCap = 4096;  // dt entries a session keeps between collections

// Device bytes per cell of a resident solve in a group's arena: two state
// copies and the staged-sweep scratch.
double bytes_per_cell(int nmat, int dim)
{
    return 8.0 * (2.0 * (2 * nmat + dim) + staged_scratch_doubles(nmat, dim));
}

struct Req {
    long long id = 0;
    dimgpu_desc desc{};
    std::vector<double> state;   // the initial state, then the result
    std::vector<double> dts;
    long long ncell = 0;
    int steps = 0;
    double cfl = 0.0, dt_max = 0.0;
    int status = DIMGPU_REQ_QUEUED;
    bool cancel = false;
    int group = -1;   // batch lane
    int inst = -1;    // instance in that lane's batch
    int solo = -1;    // solo lane
    Clock::time_point submitted, finished;
    std::string msg;
};

struct Group {
    int nmat = 0, dim = 0;
    dimgpu_batch* batch = nullptr;
    std::vector<long long> resident;  // request ids
    bool busy = false;                // a quantum is in flight
};

struct Solo {
    dimgpu_session* s = nullptr;
    cudaEvent_t done = nullptr;
    long long req = 0;                // resident request id, 0 when free
    long long off = 0, len = 0;       // its range of the solo arena (doubles)
    int steps_done = 0;               // steps enqueued so far
    bool busy = false;
};

}  // namespace

struct dimgpu_server {
    dimgpu_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv;
    std::thread worker;
    bool stop = false;
    long long next_id = 1;
    std::deque<long long> queue;                      // queued request ids, arrival order
    std::map<long long, std::unique_ptr<Req>> reqs;   // every request not yet collected
    std::vector<Group> groups;
    std::vector<Solo> solos;
    double* solo_arena = nullptr;
    RangeAlloc solo_cells;
    std::string solo_error;                           // why the solo lanes could not be set up
    long long submitted = 0, completed = 0, cancelled = 0, failed = 0, quanta = 0;
    int resident = 0, peak_resident = 0;
    double peak_bytes = 0.0, used_bytes = 0.0;
    std::string msg;
};

namespace {

int sfail(dimgpu_server* s, int code, const std::string& m)
{
    if (s) s->msg = m;
    set_sessionless_error(m);
    return code;
}

bool is_solo(const dimgpu_server* s, const dimgpu_desc& d, long long ncell)
{
    return s->cfg.solo_slots > 0 && s->cfg.solo_min_cells > 0 && ncell >= s->cfg.solo_min_cells &&
           d.model == DIMGPU_MODEL_DIM;
}

// The group of a request, created (and its arena reserved) on first use.
// Called by the server thread only.
int group_of(dimgpu_server* s, const dimgpu_desc& d, std::string* err)
{
    for (size_t g = 0; g < s->groups.size(); ++g)
        if (s->groups[g].nmat == d.nmat && s->groups[g].dim == d.dim) return (int)g;
    const double share = s->cfg.dim_share[d.dim - 1];
    const long long cells = (long long)(s->cfg.hbm_budget_bytes * share / bytes_per_cell(d.nmat, d.dim));
    if (share <= 0.0 || cells < 1) {
        *err = "no share of the budget for " + std::to_string(d.dim) + "D solves";
        return -1;
    }
    Group G;
    G.nmat = d.nmat;
    G.dim = d.dim;
    int rc = dimgpu_batch_create(d.nmat, d.dim, &G.batch);
    if (rc == DIMGPU_OK)
        rc = dimgpu_batch_reserve(G.batch, cells, s->cfg.max_slots,
                                  (long long)s->cfg.max_slots * std::max(1, s->cfg.max_steps_per_solve));
    if (rc != DIMGPU_OK) {
        *err = std::string("reserving the group's arena: ") + dimgpu_last_error(nullptr);
        if (G.batch) dimgpu_batch_destroy(G.batch);
        return -1;
    }
    s->groups.push_back(G);
    return (int)s->groups.size() - 1;
}

// The solo lanes and their arena, set up on first use.  Server thread only.
bool solo_ready(dimgpu_server* s)
{
    if (!s->solos.empty()) return true;
    if (!s->solo_error.empty()) return false;
    const long long cap = (long long)(s->cfg.hbm_budget_bytes * s->cfg.solo_share / 8.0);
    cudaError_t e = cap > 0 ? cudaMalloc(&s->solo_arena, sizeof(double) * (size_t)cap) : cudaErrorInvalidValue;
    if (e != cudaSuccess) {
        s->solo_error = std::string("reserving the solo arena: ") + cudaGetErrorString(e);
        s->solo_arena = nullptr;
        return false;
    }
    s->solo_cells.reset(cap);
    for (int k = 0; k < s->cfg.solo_slots; ++k) {
        Solo L;
        int rc = session_shell_create(&L.s);
        if (rc == DIMGPU_OK && cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming) != cudaSuccess)
            rc = DIMGPU_E_CUDA;
        if (rc != DIMGPU_OK) {
            s->solo_error = std::string("creating the solo lanes: ") + dimgpu_last_error(nullptr);
            if (L.s) dimgpu_destroy(L.s);
            for (auto& o : s->solos) {
                dimgpu_destroy(o.s);
                cudaEventDestroy(o.done);
            }
            s->solos.clear();
            cudaFree(s->solo_arena);
            s->solo_arena = nullptr;
            return false;
        }
        s->solos.push_back(L);
    }
    return true;
}

void finish(dimgpu_server* s, Req& r, int status, const std::string& msg = "")
{
    r.status = status;
    r.msg = msg;
    r.finished = Clock::now();
    if (status == DIMGPU_REQ_DONE) s->completed++;
    else if (status == DIMGPU_REQ_CANCELLED) s->cancelled++;
    else if (status == DIMGPU_REQ_FAILED) s->failed++;
}

void release_batch(dimgpu_server* s, Group& G, Req& r)
{
    dimgpu_batch_remove(G.batch, r.inst);
    G.resident.erase(std::find(G.resident.begin(), G.resident.end(), r.id));
    s->resident--;
    s->used_bytes -= bytes_per_cell(r.desc.nmat, r.desc.dim) * (double)r.ncell;
    r.inst = -1;
}

void release_solo(dimgpu_server* s, Solo& L, Req& r)
{
    s->solo_cells.release(L.off, L.len);
    s->resident--;
    s->used_bytes -= 8.0 * (double)L.len;
    L.req = 0;
    r.solo = -1;
}

void admitted(dimgpu_server* s, Req& r, double bytes)
{
    r.status = DIMGPU_REQ_RUNNING;
    s->resident++;
    s->peak_resident = std::max(s->peak_resident, s->resident);
    s->used_bytes += bytes;
    s->peak_bytes = std::max(s->peak_bytes, s->used_bytes);
}

}  // namespace

namespace {

std::string session_message(const dimgpu_session* sess)
{
    const std::string m = dimgpu_last_error(sess);
    return m.empty() ? std::string(dimgpu_last_error(nullptr)) : m;
}

// Admission (lock held): first come first served within the solo lanes and
// within each batch group; a lane kind or group whose head cannot be taken
// now (no free lane, no room, or its batch lane is mid-quantum) takes
// nothing more in this admission pass, so its later requests cannot
// overtake it.
void admit(dimgpu_server* s)
{
    std::vector<char> blocked(s->groups.size() + 16, 0);
    bool solo_blocked = false;
    for (auto it = s->queue.begin(); it != s->queue.end();) {
        Req& r = *s->reqs[*it];
        if (r.cancel) {
            finish(s, r, DIMGPU_REQ_CANCELLED);
            it = s->queue.erase(it);
            continue;
        }
        if (r.steps == 0) {
            r.dts.clear();
            finish(s, r, DIMGPU_REQ_DONE);
            it = s->queue.erase(it);
            continue;
        }
        if (s->resident >= s->cfg.max_slots) break;
        if (is_solo(s, r.desc, r.ncell)) {
            if (solo_blocked) {
                ++it;
                continue;
            }
            if (!solo_ready(s)) {
                finish(s, r, DIMGPU_REQ_FAILED, s->solo_error);
                it = s->queue.erase(it);
                continue;
            }
            int lane = -1;
            for (size_t k = 0; k < s->solos.size() && lane < 0; ++k)
                if (s->solos[k].req == 0 && !s->solos[k].busy) lane = (int)k;
            const long long need = session_grid_doubles(&r.desc);
            const long long off = lane < 0 ? -1 : s->solo_cells.alloc(need);
            if (off < 0) {
                solo_blocked = true;
                ++it;
                continue;
            }
            Solo& L = s->solos[(size_t)lane];
            int rc = session_shell_bind(L.s, &r.desc, s->solo_arena + off);
            if (rc == DIMGPU_OK) rc = dimgpu_upload(L.s, r.state.data(), r.state.size());
            if (rc != DIMGPU_OK) {
                s->solo_cells.release(off, need);
                finish(s, r, DIMGPU_REQ_FAILED, session_message(L.s));
                it = s->queue.erase(it);
                continue;
            }
            L.req = r.id;
            L.off = off;
            L.len = need;
            L.steps_done = 0;
            r.solo = lane;
            admitted(s, r, 8.0 * (double)need);
            it = s->queue.erase(it);
            continue;
        }
        std::string err;
        const int g = group_of(s, r.desc, &err);
        if (g < 0) {
            finish(s, r, DIMGPU_REQ_FAILED, err);
            it = s->queue.erase(it);
            continue;
        }
        if ((size_t)g >= blocked.size()) blocked.resize((size_t)g + 1, 0);
        Group& G = s->groups[(size_t)g];
        if (blocked[(size_t)g] || G.busy) {
            blocked[(size_t)g] = 1;
            ++it;
            continue;
        }
        int iid = -1;
        const int rc = dimgpu_batch_add(G.batch, &r.desc, r.state.data(), r.steps, r.cfl, r.dt_max, &iid);
        if (rc == DIMGPU_E_OOM) {
            blocked[(size_t)g] = 1;
            ++it;
            continue;
        }
        if (rc != DIMGPU_OK) {
            finish(s, r, DIMGPU_REQ_FAILED, dimgpu_batch_last_error(G.batch));
            it = s->queue.erase(it);
            continue;
        }
        r.group = g;
        r.inst = iid;
        G.resident.push_back(r.id);
        admitted(s, r, bytes_per_cell(r.desc.nmat, r.desc.dim) * (double)r.ncell);
        it = s->queue.erase(it);
    }
}

// A batch lane whose quantum has ended: copy out and retire its finished
// solves (all of them, failed, on an error).
void retire_batch(dimgpu_server* s, Group& G)
{
    G.busy = false;
    const int rc = dimgpu_batch_wait(G.batch);  // the quantum has ended: returns at once
    const std::string err = rc != DIMGPU_OK ? dimgpu_batch_last_error(G.batch) : "";
    for (size_t q = 0; q < G.resident.size();) {
        Req& r = *s->reqs[G.resident[q]];
        int done = 0, left = 0;
        dimgpu_batch_status(G.batch, r.inst, &done, &left);
        if (rc == DIMGPU_OK && left > 0) {
            ++q;
            continue;
        }
        int st = DIMGPU_REQ_FAILED;
        std::string m = err;
        if (rc == DIMGPU_OK) {
            r.dts.assign((size_t)std::max(done, 1), 0.0);
            const int rd = dimgpu_batch_download(G.batch, r.inst, r.state.data(), r.state.size(), r.dts.data());
            r.dts.resize((size_t)done);
            st = rd == DIMGPU_OK ? DIMGPU_REQ_DONE : DIMGPU_REQ_FAILED;
            if (rd != DIMGPU_OK) m = dimgpu_batch_last_error(G.batch);
        }
        release_batch(s, G, r);
        finish(s, r, st, m);
    }
}

// A solo lane whose quantum has ended: check its error flag; when every step
// has run, collect the dt log and the state.
void retire_solo(dimgpu_server* s, Solo& L)
{
    L.busy = false;
    Req& r = *s->reqs[L.req];
    int rc = session_check(L.s);
    if (rc == DIMGPU_OK && L.steps_done < r.steps) return;
    if (rc == DIMGPU_OK) {
        r.dts.assign((size_t)r.steps, 0.0);
        int count = 0;
        rc = dimgpu_collect(L.s, r.dts.data(), r.steps, &count);
        if (rc == DIMGPU_OK) rc = dimgpu_download(L.s, r.state.data(), r.state.size());
        r.dts.resize((size_t)count);
    }
    const std::string m = rc == DIMGPU_OK ? "" : session_message(L.s);
    release_solo(s, L, r);
    finish(s, r, rc == DIMGPU_OK ? DIMGPU_REQ_DONE : DIMGPU_REQ_FAILED, m);
}

// Cancellations of resident solves, on lanes between quanta.
void cancel_resident(dimgpu_server* s)
{
    for (auto& G : s->groups) {
        if (G.busy) continue;
        for (size_t k = 0; k < G.resident.size();) {
            Req& r = *s->reqs[G.resident[k]];
            if (!r.cancel) {
                ++k;
                continue;
            }
            release_batch(s, G, r);
            finish(s, r, DIMGPU_REQ_CANCELLED);
        }
    }
    for (auto& L : s->solos) {
        if (L.busy || L.req == 0) continue;
        Req& r = *s->reqs[L.req];
        if (!r.cancel) continue;
        release_solo(s, L, r);
        finish(s, r, DIMGPU_REQ_CANCELLED);
    }
}

// The next quantum on every idle lane that holds solves.
void enqueue_lanes(dimgpu_server* s)
{
    for (auto& G : s->groups) {
        if (G.busy || G.resident.empty()) continue;
        if (dimgpu_batch_enqueue(G.batch, s->cfg.quantum) == DIMGPU_OK) {
            G.busy = true;
            s->quanta++;
            continue;
        }
        const std::string err = dimgpu_batch_last_error(G.batch);
        while (!G.resident.empty()) {
            Req& r = *s->reqs[G.resident.back()];
            release_batch(s, G, r);
            finish(s, r, DIMGPU_REQ_FAILED, err);
        }
    }
    for (auto& L : s->solos) {
        if (L.busy || L.req == 0) continue;
        Req& r = *s->reqs[L.req];
        const int n = std::min(s->cfg.quantum, r.steps - L.steps_done);
        int rc = dimgpu_enqueue_steps(L.s, n, r.cfl, r.dt_max);
        if (rc == DIMGPU_OK && cudaEventRecord(L.done, L.s->stream) != cudaSuccess) rc = DIMGPU_E_CUDA;
        if (rc == DIMGPU_OK) {
            L.steps_done += n;
            L.busy = true;
            s->quanta++;
            continue;
        }
        const std::string m = session_message(L.s);
        release_solo(s, L, r);
        finish(s, r, DIMGPU_REQ_FAILED, m);
    }
}

void serve_loop(dimgpu_server* s)
{
    std::unique_lock<std::mutex> lock(s->mu);
    while (!s->stop) {
        bool progressed = false;
        for (auto& G : s->groups)
            if (G.busy && batch_ready(G.batch)) {
                retire_batch(s, G);
                progressed = true;
            }
        for (auto& L : s->solos)
            if (L.busy && cudaEventQuery(L.done) != cudaErrorNotReady) {
                retire_solo(s, L);
                progressed = true;
            }
        cancel_resident(s);
        admit(s);
        enqueue_lanes(s);
        bool busy = false;
        for (auto& G : s->groups) busy = busy || G.busy;
        for (auto& L : s->solos) busy = busy || L.busy;
        if (progressed || !busy) s->cv.notify_all();
        if (busy) {
            if (!progressed) {
                // lanes are mid-quantum: look again shortly (no host sync)
                lock.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(50));
                lock.lock();
            }
            continue;
        }
        if (s->resident == 0 && !s->queue.empty()) {
            // nothing runs and the head still was not taken: it never fits
            Req& r = *s->reqs[s->queue.front()];
            finish(s, r, DIMGPU_REQ_FAILED, "the solve cannot be admitted within the server's limits");
            s->queue.pop_front();
            continue;
        }
        s->cv.wait(lock, [&] { return s->stop || !s->queue.empty(); });
    }
}

}  // namespace

extern "C" {

int dimgpu_server_create(const dimgpu_server_config* cfg, dimgpu_server** out)
{
    if (!cfg || !out) return sfail(nullptr, DIMGPU_E_INVALID_ARG, "dimgpu_server_create: null argument");
    *out = nullptr;
    if (!(cfg->hbm_budget_bytes > 0.0) || cfg->max_slots < 1 || cfg->quantum < 1 || cfg->max_steps_per_solve < 1)
        return sfail(nullptr, DIMGPU_E_INVALID_ARG,
                     "dimgpu_server_create: budget, slots, quantum and steps per solve must be positive");
    double sum = cfg->solo_share;
    if (!(cfg->solo_share >= 0.0) || cfg->solo_slots < 0 || cfg->solo_min_cells < 0)
        return sfail(nullptr, DIMGPU_E_INVALID_ARG, "dimgpu_server_create: negative solo setting");
    for (double f : cfg->dim_share) {
        if (!(f >= 0.0)) return sfail(nullptr, DIMGPU_E_INVALID_ARG, "dimgpu_server_create: negative budget share");
        sum += f;
    }
    if (!(sum > 0.0) || sum > 1.0 + 1e-12)
        return sfail(nullptr, DIMGPU_E_INVALID_ARG, "dimgpu_server_create: budget shares must add up to (0, 1]");
    if (cfg->solo_slots > 0 && cfg->solo_min_cells > 0 && cfg->max_steps_per_solve > kSoloHistCap)
        return sfail(nullptr, DIMGPU_E_INVALID_ARG,
                     "dimgpu_server_create: solo lanes keep at most 4096 steps per solve");
    auto* s = new dimgpu_server();
    s->cfg = *cfg;
    s->worker = std::thread(serve_loop, s);
    *out = s;
    return DIMGPU_OK;
}

int dimgpu_server_destroy(dimgpu_server* s)
{
    if (!s) return DIMGPU_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto& G : s->groups) dimgpu_batch_destroy(G.batch);
    for (auto& L : s->solos) {
        dimgpu_destroy(L.s);
        cudaEventDestroy(L.done);
    }
    cudaFree(s->solo_arena);
    delete s;
    return DIMGPU_OK;
}

const char* dimgpu_server_last_error(const dimgpu_server* s) { return s ? s->msg.c_str() : ""; }

int dimgpu_server_submit(dimgpu_server* s, const dimgpu_desc* desc, const double* soa, int steps, double cfl,
                         double dt_max, long long* request_id)
{
    if (!s || !desc || !soa || !request_id) return sfail(s, DIMGPU_E_INVALID_ARG, "dimgpu_server_submit: null argument");
    if (desc->dim < 1 || desc->dim > 3 || desc->nmat < 1 || desc->nmat > DIMGPU_MAX_MATERIALS)
        return sfail(s, DIMGPU_E_INVALID_ARG, "dimgpu_server_submit: bad dim or nmat");
    if (steps < 0 || steps > s->cfg.max_steps_per_solve)
        return sfail(s, DIMGPU_E_INVALID_ARG, "dimgpu_server_submit: step count beyond the server's limit");
    long long ncell = 1;
    for (int a = 0; a < desc->dim; ++a) {
        if (desc->N[a] < 1) return sfail(s, DIMGPU_E_INVALID_ARG, "dimgpu_server_submit: grid size must be positive");
        ncell *= desc->N[a];
        if (ncell > (1LL << 40)) return sfail(s, DIMGPU_E_OOM, "dimgpu_server_submit: grid too large");
    }
    const bool solo = is_solo(s, *desc, ncell);
    const double need = solo ? 8.0 * (double)session_grid_doubles(desc)
                             : bytes_per_cell(desc->nmat, desc->dim) * (double)ncell;
    const double share = solo ? s->cfg.solo_share : s->cfg.dim_share[desc->dim - 1];
    if (need > s->cfg.hbm_budget_bytes * share)
        return sfail(s, DIMGPU_E_OOM, "dimgpu_server_submit: the solve needs more device memory than its budget share");
    auto r = std::make_unique<Req>();
    r->desc = *desc;
    r->ncell = ncell;
    r->state.assign(soa, soa + (size_t)(2 * desc->nmat + desc->dim) * (size_t)ncell);
    r->steps = steps;
    r->cfl = cfl;
    r->dt_max = dt_max;
    r->submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        r->id = s->next_id++;
        *request_id = r->id;
        s->queue.push_back(r->id);
        s->reqs[r->id] = std::move(r);
        s->submitted++;
    }
    s->cv.notify_all();
    return DIMGPU_OK;
}

int dimgpu_server_poll(dimgpu_server* s, long long request_id, int* state, double* soa_out, size_t count,
                       double* dts_out, double* latency_s)
{
    if (!s || !state) return sfail(s, DIMGPU_E_INVALID_ARG, "dimgpu_server_poll: null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return sfail(s, DIMGPU_E_INVALID_ARG, "dimgpu_server_poll: unknown or collected request");
    Req& r = *it->second;
    *state = r.status;
    const bool final = r.status == DIMGPU_REQ_DONE || r.status == DIMGPU_REQ_CANCELLED || r.status == DIMGPU_REQ_FAILED;
    if (latency_s) *latency_s = final ? std::chrono::duration<double>(r.finished - r.submitted).count() : 0.0;
    if (!final) return DIMGPU_OK;
    if (r.status == DIMGPU_REQ_FAILED) {
        const std::string m = "request " + std::to_string(r.id) + ": " + r.msg;
        s->reqs.erase(it);
        return sfail(s, DIMGPU_E_NONFINITE, m);
    }
    if (r.status == DIMGPU_REQ_DONE && soa_out) {
        if (count != r.state.size()) return sfail(s, DIMGPU_E_INVALID_ARG, "dimgpu_server_poll: size mismatch");
        std::memcpy(soa_out, r.state.data(), sizeof(double) * r.state.size());
        if (dts_out) std::memcpy(dts_out, r.dts.data(), sizeof(double) * r.dts.size());
    }
    if (soa_out || r.status == DIMGPU_REQ_CANCELLED) s->reqs.erase(it);  // collected
    return DIMGPU_OK;
}

int dimgpu_server_cancel(dimgpu_server* s, long long request_id)
{
    if (!s) return sfail(nullptr, DIMGPU_E_INVALID_ARG, "dimgpu_server_cancel: null server");
    {
        std::lock_guard<std::mutex> lock(s->mu);
        auto it = s->reqs.find(request_id);
        if (it == s->reqs.end()) return sfail(s, DIMGPU_E_INVALID_ARG, "dimgpu_server_cancel: unknown request");
        it->second->cancel = true;
    }
    s->cv.notify_all();
    return DIMGPU_OK;
}

int dimgpu_server_drain(dimgpu_server* s)
{
    if (!s) return sfail(nullptr, DIMGPU_E_INVALID_ARG, "dimgpu_server_drain: null server");
    std::unique_lock<std::mutex> lock(s->mu);
    s->cv.wait(lock, [&] { return s->queue.empty() && s->resident == 0; });
    return DIMGPU_OK;
}

int dimgpu_server_stats(dimgpu_server* s, dimgpu_server_counters* out)
{
    if (!s || !out) return sfail(s, DIMGPU_E_INVALID_ARG, "dimgpu_server_stats: null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->cancelled = s->cancelled;
    out->failed = s->failed;
    out->quanta = s->quanta;
    out->queued = (long long)s->queue.size();
    out->resident = s->resident;
    out->peak_resident = s->peak_resident;
    out->peak_bytes = s->peak_bytes;
    return DIMGPU_OK;
}

}  // extern "C"
