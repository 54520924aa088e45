// dimgpu_server.cu — the continuous-batching serving loop behind the C-ABI
// (include/dimgpu.h: dimgpu_server_*).
//
// Requests (a grid, its initial state, a step budget) are submitted from any
// host thread and queue in arrival order.  A server thread runs the loop:
//
//   admit    first come first served, per (material count, dimension) group,
//            into that group's batch — an arena-mode dimgpu_batch whose
//            device memory was reserved once, so admission allocates and
//            synchronises nothing; a request that does not fit waits for
//            room (later requests of other groups may go ahead);
//   step     every group with resident solves enqueues one quantum of steps
//            on its own stream, so the groups' work overlaps on the device;
//   retire   after the quantum, finished solves are copied out and their
//            arena ranges returned, which is what lets the queue drain.
//
// Every solve's arithmetic is the single-grid step's: a result does not
// depend on what else was resident.  Latency is measured on the host from
// submission to the end of the quantum in which the solve finished.
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

using namespace dimgpu;

namespace {

using Clock = std::chrono::steady_clock;

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
    int group = -1;
    int inst = -1;
    Clock::time_point submitted, finished;
    std::string msg;
};

struct Group {
    int nmat = 0, dim = 0;
    dimgpu_batch* batch = nullptr;
    std::vector<long long> resident;  // request ids
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

void finish(dimgpu_server* s, Req& r, int status, const std::string& msg = "")
{
    r.status = status;
    r.msg = msg;
    r.finished = Clock::now();
    if (status == DIMGPU_REQ_DONE) s->completed++;
    else if (status == DIMGPU_REQ_CANCELLED) s->cancelled++;
    else if (status == DIMGPU_REQ_FAILED) s->failed++;
}

void release(dimgpu_server* s, Group& G, Req& r)
{
    dimgpu_batch_remove(G.batch, r.inst);
    G.resident.erase(std::find(G.resident.begin(), G.resident.end(), r.id));
    s->resident--;
    s->used_bytes -= bytes_per_cell(r.desc.nmat, r.desc.dim) * (double)r.ncell;
    r.inst = -1;
}

// Admission (lock held): first come first served within a group; a group
// whose head does not fit admits nothing more this round.
void admit(dimgpu_server* s)
{
    std::vector<char> blocked(s->groups.size() + 16, 0);
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
        std::string err;
        const int g = group_of(s, r.desc, &err);
        if (g < 0) {
            finish(s, r, DIMGPU_REQ_FAILED, err);
            it = s->queue.erase(it);
            continue;
        }
        if ((size_t)g >= blocked.size()) blocked.resize((size_t)g + 1, 0);
        if (blocked[(size_t)g]) {
            ++it;
            continue;
        }
        Group& G = s->groups[(size_t)g];
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
        r.status = DIMGPU_REQ_RUNNING;
        G.resident.push_back(r.id);
        s->resident++;
        s->peak_resident = std::max(s->peak_resident, s->resident);
        s->used_bytes += bytes_per_cell(r.desc.nmat, r.desc.dim) * (double)r.ncell;
        s->peak_bytes = std::max(s->peak_bytes, s->used_bytes);
        it = s->queue.erase(it);
    }
}

void serve_loop(dimgpu_server* s)
{
    std::unique_lock<std::mutex> lock(s->mu);
    while (true) {
        s->cv.wait(lock, [&] { return s->stop || !s->queue.empty() || s->resident > 0; });
        if (s->stop) break;
        // cancellations of resident solves
        for (auto& G : s->groups) {
            for (size_t k = 0; k < G.resident.size();) {
                Req& r = *s->reqs[G.resident[k]];
                if (r.cancel) {
                    release(s, G, r);
                    finish(s, r, DIMGPU_REQ_CANCELLED);
                }
                else {
                    ++k;
                }
            }
        }
        admit(s);
        if (s->resident == 0) {
            s->cv.notify_all();
            continue;
        }
        // one quantum on every group, each on its own stream, then wait for all
        std::vector<int> ran;
        for (size_t g = 0; g < s->groups.size(); ++g) {
            if (s->groups[g].resident.empty()) continue;
            if (dimgpu_batch_enqueue(s->groups[g].batch, s->cfg.quantum) == DIMGPU_OK) ran.push_back((int)g);
        }
        lock.unlock();
        std::vector<int> rcs(ran.size());
        for (size_t k = 0; k < ran.size(); ++k) rcs[k] = dimgpu_batch_wait(s->groups[(size_t)ran[k]].batch);
        lock.lock();
        s->quanta++;
        // retire finished solves (and fail the group's solves on an error)
        for (size_t k = 0; k < ran.size(); ++k) {
            Group& G = s->groups[(size_t)ran[k]];
            const std::string err = rcs[k] != DIMGPU_OK ? dimgpu_batch_last_error(G.batch) : "";
            for (size_t q = 0; q < G.resident.size();) {
                Req& r = *s->reqs[G.resident[q]];
                int done = 0, left = 0;
                dimgpu_batch_status(G.batch, r.inst, &done, &left);
                if (rcs[k] == DIMGPU_OK && left > 0) {
                    ++q;
                    continue;
                }
                int st = DIMGPU_REQ_FAILED;
                std::string m = err;
                if (rcs[k] == DIMGPU_OK) {
                    r.dts.assign((size_t)std::max(done, 1), 0.0);
                    const int rc = dimgpu_batch_download(G.batch, r.inst, r.state.data(), r.state.size(), r.dts.data());
                    r.dts.resize((size_t)done);
                    st = rc == DIMGPU_OK ? DIMGPU_REQ_DONE : DIMGPU_REQ_FAILED;
                    if (rc != DIMGPU_OK) m = dimgpu_batch_last_error(G.batch);
                }
                release(s, G, r);
                finish(s, r, st, m);
            }
        }
        s->cv.notify_all();
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
    double sum = 0.0;
    for (double f : cfg->dim_share) {
        if (!(f >= 0.0)) return sfail(nullptr, DIMGPU_E_INVALID_ARG, "dimgpu_server_create: negative budget share");
        sum += f;
    }
    if (!(sum > 0.0) || sum > 1.0 + 1e-12)
        return sfail(nullptr, DIMGPU_E_INVALID_ARG, "dimgpu_server_create: budget shares must add up to (0, 1]");
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
    const double need = bytes_per_cell(desc->nmat, desc->dim) * (double)ncell;
    if (need > s->cfg.hbm_budget_bytes * s->cfg.dim_share[desc->dim - 1])
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
