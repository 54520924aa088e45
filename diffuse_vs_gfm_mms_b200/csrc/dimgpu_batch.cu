// dimgpu_batch.cu — the batched form of the DIM step (include/dimgpu.h,
// dimgpu_batch_*): many independent grids of one material count and
// dimension, each with its own size, materials, boundaries, cfl, dt_max and
// step budget, advanced together by one set of persistent-grid launches per
// step (dim_batch.cuh) and replayed from a captured CUDA graph.
//
// Membership (instances added, finished, removed) lives in device tables;
// the launch geometry does not depend on it, so one captured graph of G steps
// serves every membership as long as the scratch and tables are not
// reallocated.  Each instance's arithmetic is exactly the single-grid step's,
// so an instance's result is the same alone, in any batch, and against the
// oracle.
#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "dim_launch.h"
#include "dimgpu.h"
#include "range_alloc.h"

using namespace dimgpu;

namespace {

constexpr int kGraphSteps = 8;  // steps per captured graph

struct HostInst {
    int id;
    dimgpu_desc desc;
    BInst dev;            // what is uploaded into the device table
    long long ncell;
    long long nbc;        // boundary cells
    int steps_total;
    int steps_left;       // host mirror (exact: every run advances min(n, left))
    long long cell_off;   // arena mode: first cell of its range (scratch items and state)
    long long dt_off;     // arena mode: first entry of its dt log range
};

long long boundary_cells(const dimgpu_desc& d)
{
    long long total = 0;
    for (int a = 0; a < d.dim; ++a) {
        if (d.N[a] <= 1) continue;
        long long c = 1;
        for (int b = 0; b < d.dim; ++b) {
            if (b == a) continue;
            c *= (b < a && d.N[b] != 1) ? (long long)(d.N[b] - 2) : (long long)d.N[b];
        }
        total += 2 * c;
    }
    return total;
}

}  // namespace

struct dimgpu_batch {
    int nmat = 0, dim = 0;
    std::vector<HostInst> inst;
    int next_id = 1;
    bool dirty = true;      // tables must be rebuilt before the next step
    // device
    BInst* tab = nullptr;
    long long* cell_prefix = nullptr;
    long long* bc_prefix = nullptr;
    double* blockmin = nullptr;
    double* scratch = nullptr;
    int* err = nullptr;
    long long tab_cap = 0, blockmin_cap = 0, scratch_cap = 0;
    int grid = 148 * 4;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::string msg;
    // arena mode (dimgpu_batch_reserve): everything allocated once
    bool arena = false;
    double* st_arena[2] = {nullptr, nullptr};
    double* dt_arena = nullptr;
    RangeAlloc cells, dts;
    BInst* tab_pinned = nullptr;           // host staging of the tables
    long long* prefix_pinned = nullptr;    // cell prefix, then bc prefix
    cudaEvent_t done = nullptr;            // after the last enqueued step
};

namespace {

int bfail(dimgpu_batch* b, int code, const std::string& m)
{
    if (b) b->msg = m;
    set_sessionless_error(m);
    return code;
}

int bcuda(dimgpu_batch* b, cudaError_t e, const char* what)
{
    if (e == cudaErrorMemoryAllocation) return bfail(b, DIMGPU_E_OOM, std::string(what) + ": out of device memory");
    return bfail(b, DIMGPU_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void drop_graphs(dimgpu_batch* b)
{
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

template<class T>
cudaError_t grow(T** p, long long* cap, long long need)
{
    if (need <= *cap && *p) return cudaSuccess;
    long long n = std::max<long long>(need, *cap * 3 / 2);
    n = std::max<long long>(n, 16);
    cudaFree(*p);
    *p = nullptr;
    cudaError_t e = cudaMalloc(p, sizeof(T) * (size_t)n);
    if (e == cudaSuccess) *cap = n;
    else *cap = 0;
    return e;
}

// The device-table entry of an instance as the device holds it after the
// steps enqueued so far: steps_done / steps_left from the host mirror;
// run = whether it ran in the last step enqueued; cur = its buffer at the
// start of that step (every instance starts in buffer 0 and a step moves it
// by D sweeps).
void sync_mirror(const dimgpu_batch* b, HostInst& h)
{
    const int done = h.steps_total - h.steps_left;
    h.dev.steps_done = done;
    h.dev.steps_left = h.steps_left;
    const int start = done - (h.dev.run ? 1 : 0);
    h.dev.cur = (int)(((long long)start * b->dim) & 1);
}

// The buffer that holds an instance's state after the steps enqueued so far.
int current_buffer(const dimgpu_batch* b, const HostInst& h)
{
    const long long done = h.steps_total - h.steps_left;
    return (int)((done * b->dim) & 1);
}

// Rebuild the device tables (and, outside arena mode, grow the scratch) for
// the current members.  Tables are padded to a capacity C (entries past the
// members have no work and no steps), and every launch is given C, so a
// captured graph stays valid across membership changes until a table or the
// scratch has to grow — which never happens in arena mode.
cudaError_t rebuild(dimgpu_batch* b)
{
    const int n = (int)b->inst.size();
    long long items = 0, cells_blocks = 0;
    for (int i = 0; i < n; ++i) {
        if (b->arena) {
            b->inst[i].dev.soff = b->inst[i].cell_off;
        }
        else {
            b->inst[i].dev.soff = items;
            items += b->inst[i].ncell;
        }
        cells_blocks += (b->inst[i].ncell + 255) / 256;
        sync_mirror(b, b->inst[i]);
    }
    cudaError_t e = cudaSuccess;
    if (!b->arena) {
        const int nrec = staged_scratch_doubles(b->nmat, b->dim);
        // A captured graph bakes in the launch arguments (buffer addresses and
        // the scratch capacity that strides every record): drop it whenever any
        // of them changes.  An address alone is not enough, since a regrown
        // buffer can come back at the address of the one it replaces.
        const long long caps_before[3] = {b->scratch_cap, b->blockmin_cap, b->tab_cap};
        const void* before[5] = {b->scratch, b->blockmin, b->tab, b->cell_prefix, b->bc_prefix};
        e = grow(&b->scratch, &b->scratch_cap, std::max<long long>(items, 1) * nrec);
        if (e == cudaSuccess) e = grow(&b->blockmin, &b->blockmin_cap, std::max<long long>(cells_blocks, 1));
        if (e == cudaSuccess && (n > b->tab_cap || !b->tab)) {
            const long long cap = std::max<long long>(std::max<long long>(16, n), b->tab_cap * 2);
            cudaFree(b->tab);
            cudaFree(b->cell_prefix);
            cudaFree(b->bc_prefix);
            b->tab = nullptr;
            b->cell_prefix = b->bc_prefix = nullptr;
            e = cudaMalloc(&b->tab, sizeof(BInst) * (size_t)cap);
            if (e == cudaSuccess) e = cudaMalloc(&b->cell_prefix, sizeof(long long) * (size_t)(cap + 1));
            if (e == cudaSuccess) e = cudaMalloc(&b->bc_prefix, sizeof(long long) * (size_t)(cap + 1));
            b->tab_cap = e == cudaSuccess ? cap : 0;
        }
        if (e != cudaSuccess) return e;
        const void* after[5] = {b->scratch, b->blockmin, b->tab, b->cell_prefix, b->bc_prefix};
        const long long caps_after[3] = {b->scratch_cap, b->blockmin_cap, b->tab_cap};
        if (std::memcmp(before, after, sizeof before) != 0 ||
            std::memcmp(caps_before, caps_after, sizeof caps_before) != 0)
            drop_graphs(b);
    }
    const long long C = b->tab_cap;
    std::vector<BInst> dev_v;
    std::vector<long long> pre_v;
    BInst* dev;
    long long* cp;
    if (b->arena) {
        dev = b->tab_pinned;
        cp = b->prefix_pinned;
    }
    else {
        dev_v.resize((size_t)C);
        pre_v.resize(2 * (size_t)(C + 1));
        dev = dev_v.data();
        cp = pre_v.data();
    }
    long long* bp = cp + (C + 1);
    std::memset(dev, 0, sizeof(BInst) * (size_t)C);
    cp[0] = bp[0] = 0;
    for (long long i = 0; i < C; ++i) {
        long long cb = 0, bb = 0;
        if (i < n) {
            dev[i] = b->inst[(size_t)i].dev;
            cb = (b->inst[(size_t)i].ncell + 255) / 256;
            bb = (b->inst[(size_t)i].nbc + 255) / 256;
        }
        cp[i + 1] = cp[i] + cb;
        bp[i + 1] = bp[i] + bb;
    }
    // Arena mode: the tables are staged in pinned memory, so the copies are
    // asynchronous; the host writes the staging again only after the steps
    // that read it have completed (a caller waits for every enqueued step
    // before it changes the membership again).  Otherwise: pageable staging
    // and a synchronisation.
    e = cudaMemcpyAsync(b->tab, dev, sizeof(BInst) * (size_t)C, cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->cell_prefix, cp, sizeof(long long) * (size_t)(C + 1), cudaMemcpyHostToDevice,
                            b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->bc_prefix, bp, sizeof(long long) * (size_t)(C + 1), cudaMemcpyHostToDevice,
                            b->stream);
    if (e == cudaSuccess && !b->arena) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return e;
    b->dirty = false;
    return cudaSuccess;
}

BatchLaunch launch_args(dimgpu_batch* b)
{
    BatchLaunch L;
    L.tab = b->tab;
    L.cell_prefix = b->cell_prefix;
    L.bc_prefix = b->bc_prefix;
    L.ninst = (int)b->tab_cap;
    L.blockmin = b->blockmin;
    L.scratch = b->scratch;
    L.cap = b->scratch_cap / staged_scratch_doubles(b->nmat, b->dim);
    L.err = b->err;
    L.grid = b->grid;
    return L;
}

cudaError_t one_step(dimgpu_batch* b, const BatchLaunch& L)
{
    cudaError_t e = cudaErrorInvalidValue;
    switch (b->nmat * 10 + b->dim) {
#define BATCH_CASE(NM, D) \
        case NM * 10 + D: e = batch_step<NM, D>(L, b->stream); break;
        BATCH_CASE(1, 1) BATCH_CASE(1, 2) BATCH_CASE(1, 3)
        BATCH_CASE(2, 1) BATCH_CASE(2, 2) BATCH_CASE(2, 3)
        BATCH_CASE(3, 1) BATCH_CASE(3, 2) BATCH_CASE(3, 3)
        BATCH_CASE(4, 1) BATCH_CASE(4, 2) BATCH_CASE(4, 3)
#undef BATCH_CASE
        default: break;
    }
    return e;
}

void free_instance(dimgpu_batch* b, HostInst& h)
{
    if (b->arena) {
        if (h.cell_off >= 0) b->cells.release(h.cell_off, h.ncell);
        if (h.dt_off >= 0) b->dts.release(h.dt_off, std::max(h.steps_total, 1));
        h.cell_off = h.dt_off = -1;
    }
    else {
        cudaFree(h.dev.st[0]);
        cudaFree(h.dev.st[1]);
        cudaFree(h.dev.dtlog);
    }
}

}  // namespace

namespace dimgpu {

// 1 when every enqueued step has finished (dimgpu_batch_wait then returns
// without blocking), 0 while steps run; no host synchronisation.
int batch_ready(dimgpu_batch* b)
{
    if (!b->done) return 1;
    const cudaError_t e = cudaEventQuery(b->done);
    if (e == cudaErrorNotReady) return 0;
    return 1;  // finished, or failed: dimgpu_batch_wait reports which
}

}  // namespace dimgpu

extern "C" {

int dimgpu_batch_create(int nmat, int dim, dimgpu_batch** out)
{
    if (!out) return bfail(nullptr, DIMGPU_E_INVALID_ARG, "null output pointer");
    *out = nullptr;
    if (nmat < 1 || nmat > DIMGPU_MAX_MATERIALS) return bfail(nullptr, DIMGPU_E_INVALID_ARG, "nmat must be 1..4");
    if (dim < 1 || dim > 3) return bfail(nullptr, DIMGPU_E_INVALID_ARG, "dim must be 1, 2 or 3");
    auto* b = new dimgpu_batch();
    b->nmat = nmat;
    b->dim = dim;
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&b->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(b->err, 0, sizeof(int), b->stream);
    int dev = 0, sms = 148;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        const int rc = bcuda(nullptr, e, "dimgpu_batch_create");
        dimgpu_batch_destroy(b);
        return rc;
    }
    b->grid = sms * DIMGPU_STAGED_MINB;
    b->own_stream = b->stream;
    *out = b;
    return DIMGPU_OK;
}

int dimgpu_batch_reserve(dimgpu_batch* b, long long max_cells, int max_instances, long long max_steps)
{
    if (!b) return bfail(nullptr, DIMGPU_E_INVALID_ARG, "null batch");
    if (!b->inst.empty() || b->arena)
        return bfail(b, DIMGPU_E_INVALID_ARG, "dimgpu_batch_reserve: only on a new, empty batch");
    if (max_cells < 1 || max_instances < 1 || max_steps < 1)
        return bfail(b, DIMGPU_E_INVALID_ARG, "dimgpu_batch_reserve: capacities must be positive");
    const int V = 2 * b->nmat + b->dim;
    const long long C = max_instances;
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 2 && e == cudaSuccess; ++k)
        e = cudaMalloc(&b->st_arena[k], sizeof(double) * (size_t)V * (size_t)max_cells);
    if (e == cudaSuccess) e = cudaMalloc(&b->dt_arena, sizeof(double) * (size_t)max_steps);
    if (e == cudaSuccess)
        e = cudaMalloc(&b->scratch, sizeof(double) * (size_t)staged_scratch_doubles(b->nmat, b->dim) *
                                        (size_t)max_cells);
    // every instance's work blocks round up to 256 cells: at most one extra block each
    const long long nblocks = (max_cells + 255) / 256 + C;
    if (e == cudaSuccess) e = cudaMalloc(&b->blockmin, sizeof(double) * (size_t)nblocks);
    if (e == cudaSuccess) e = cudaMalloc(&b->tab, sizeof(BInst) * (size_t)C);
    if (e == cudaSuccess) e = cudaMalloc(&b->cell_prefix, sizeof(long long) * (size_t)(C + 1));
    if (e == cudaSuccess) e = cudaMalloc(&b->bc_prefix, sizeof(long long) * (size_t)(C + 1));
    if (e == cudaSuccess) e = cudaMallocHost(&b->tab_pinned, sizeof(BInst) * (size_t)C);
    if (e == cudaSuccess) e = cudaMallocHost(&b->prefix_pinned, sizeof(long long) * 2 * (size_t)(C + 1));
    if (e != cudaSuccess) {
        for (auto& p : b->st_arena) { cudaFree(p); p = nullptr; }
        cudaFree(b->dt_arena); cudaFree(b->scratch); cudaFree(b->blockmin); cudaFree(b->tab);
        cudaFree(b->cell_prefix); cudaFree(b->bc_prefix);
        cudaFreeHost(b->tab_pinned); cudaFreeHost(b->prefix_pinned);
        b->dt_arena = b->scratch = b->blockmin = nullptr;
        b->tab = nullptr;
        b->cell_prefix = b->bc_prefix = b->prefix_pinned = nullptr;
        b->tab_pinned = nullptr;
        return bcuda(b, e, "dimgpu_batch_reserve");
    }
    b->scratch_cap = (long long)staged_scratch_doubles(b->nmat, b->dim) * max_cells;
    b->blockmin_cap = nblocks;
    b->tab_cap = C;
    b->arena = true;
    b->cells.reset(max_cells);
    b->dts.reset(max_steps);
    drop_graphs(b);
    b->dirty = true;
    return DIMGPU_OK;
}

int dimgpu_batch_destroy(dimgpu_batch* b)
{
    if (!b) return DIMGPU_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graphs(b);
    if (b->done) cudaEventDestroy(b->done);
    if (!b->arena)
        for (auto& h : b->inst) free_instance(b, h);
    for (auto& p : b->st_arena) cudaFree(p);
    cudaFree(b->dt_arena);
    cudaFreeHost(b->tab_pinned);
    cudaFreeHost(b->prefix_pinned);
    cudaFree(b->tab);
    cudaFree(b->cell_prefix);
    cudaFree(b->bc_prefix);
    cudaFree(b->blockmin);
    cudaFree(b->scratch);
    cudaFree(b->err);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    else if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return DIMGPU_OK;
}

const char* dimgpu_batch_last_error(const dimgpu_batch* b) { return b ? b->msg.c_str() : ""; }

int dimgpu_batch_add(dimgpu_batch* b, const dimgpu_desc* d, const double* soa, int steps, double cfl, double dt_max,
                     int* id)
{
    if (!b || !d || !soa || !id) return bfail(b, DIMGPU_E_INVALID_ARG, "null argument");
    if (d->nmat != b->nmat || d->dim != b->dim)
        return bfail(b, DIMGPU_E_INVALID_ARG, "instance nmat / dim differ from the batch's");
    if (d->time_update != DIMGPU_TIME_SPLIT) return bfail(b, DIMGPU_E_UNSUPPORTED, "the batch runs split steps only");
    if (d->precision != DIMGPU_PRECISION_FP64 && d->precision != DIMGPU_PRECISION_MIXED)
        return bfail(b, DIMGPU_E_INVALID_ARG, "precision must be DIMGPU_PRECISION_FP64 or _MIXED");
    if (d->model != DIMGPU_MODEL_DIM) return bfail(b, DIMGPU_E_UNSUPPORTED, "the batch runs the DIM step only");
    if (steps < 0) return bfail(b, DIMGPU_E_INVALID_ARG, "negative step count");
    if (!(cfl > 0.0) || !(dt_max > 0.0)) return bfail(b, DIMGPU_E_INVALID_ARG, "cfl and dt_max must be positive");
    long long ncell = 1;
    for (int a = 0; a < 3; ++a) {
        if (a < d->dim && d->N[a] < 1) return bfail(b, DIMGPU_E_INVALID_ARG, "grid size must be positive");
        if (a >= d->dim && d->N[a] != 1) return bfail(b, DIMGPU_E_INVALID_ARG, "unused axes must have N = 1");
        if (a < d->dim && !(d->dx[a] > 0.0)) return bfail(b, DIMGPU_E_INVALID_ARG, "grid spacing must be positive");
        if (a < d->dim && (d->N[a] == 2 || d->N[a] == 3))
            return bfail(b, DIMGPU_E_UNSUPPORTED, "the batch needs N = 1 or N >= 4 on every axis");
        ncell *= d->N[a];
        if (ncell > 0x7FFFFFFFLL) return bfail(b, DIMGPU_E_INVALID_ARG, "an instance holds at most 2^31 - 1 cells");
    }
    for (int k = 0; k < d->nmat; ++k) {
        if (d->mat[k].kind != DIMGPU_EOS_IDEAL_GAS && d->mat[k].kind != DIMGPU_EOS_STIFFENED_GAS)
            return bfail(b, DIMGPU_E_UNSUPPORTED_EOS, "only ideal_gas and stiffened_gas run on the GPU");
        if (!(d->mat[k].gamma > 1.0)) return bfail(b, DIMGPU_E_INVALID_ARG, "gamma must be > 1");
    }
    if (d->lambda_model < 0 || d->lambda_model > 2) return bfail(b, DIMGPU_E_INVALID_ARG, "unknown lambda model");
    if (b->arena && (long long)b->inst.size() >= b->tab_cap)
        return bfail(b, DIMGPU_E_OOM, "dimgpu_batch_add: the reserved instance table is full");

    HostInst h{};
    h.id = b->next_id++;
    h.desc = *d;
    h.ncell = ncell;
    h.nbc = boundary_cells(*d);
    h.steps_total = steps;
    h.steps_left = steps;
    h.cell_off = h.dt_off = -1;
    std::memset(&h.dev, 0, sizeof h.dev);
    BInst& I = h.dev;
    int kind[kMaxMat];
    double gam[kMaxMat], pinf[kMaxMat];
    for (int k = 0; k < d->nmat; ++k) {
        kind[k] = d->mat[k].kind;
        gam[k] = d->mat[k].gamma;
        pinf[k] = d->mat[k].p_inf;
    }
    fill_mats(I.M, d->nmat, kind, gam, pinf, d->lambda_model, d->alpha_source_floor);
    for (int a = 0; a < 3; ++a) {
        I.g.N[a] = d->N[a];
        I.g.dx[a] = d->dx[a];
        I.g.bc_lo[a] = d->bc_lo[a];
        I.g.bc_hi[a] = d->bc_hi[a];
    }
    I.g.ncell = ncell;
    I.g.stride[0] = 1;
    I.g.stride[1] = d->N[0];
    I.g.stride[2] = (long long)d->N[0] * d->N[1];
    for (int a = 0; a < 3; ++a) {
        I.nl[a] = (int)(ncell / d->N[a]);
        I.by_n[a].set((unsigned)d->N[a]);
        I.by_nl[a].set((unsigned)I.nl[a]);
    }
    I.by_n0.set((unsigned)d->N[0]);
    I.steps_left = steps;
    I.mixed = d->precision == DIMGPU_PRECISION_MIXED ? 1 : 0;
    I.cfl = cfl;
    I.dt_max = dt_max;
    const int V = 2 * d->nmat + d->dim;
    const size_t bytes = sizeof(double) * (size_t)V * (size_t)ncell;
    cudaError_t e = cudaSuccess;
    if (b->arena) {
        // no allocation, no synchronisation: ranges of the reserved arenas
        h.cell_off = b->cells.alloc(ncell);
        if (h.cell_off < 0) return bfail(b, DIMGPU_E_OOM, "dimgpu_batch_add: no room for the grid in the reserved cells");
        h.dt_off = b->dts.alloc(std::max(steps, 1));
        if (h.dt_off < 0) {
            b->cells.release(h.cell_off, ncell);
            return bfail(b, DIMGPU_E_OOM, "dimgpu_batch_add: no room for the steps in the reserved dt log");
        }
        I.st[0] = b->st_arena[0] + (size_t)V * (size_t)h.cell_off;
        I.st[1] = b->st_arena[1] + (size_t)V * (size_t)h.cell_off;
        I.dtlog = b->dt_arena + h.dt_off;
        e = cudaMemcpyAsync(I.st[0], soa, bytes, cudaMemcpyHostToDevice, b->stream);
    }
    else {
        e = cudaMalloc(&I.st[0], bytes);
        if (e == cudaSuccess) e = cudaMalloc(&I.st[1], bytes);
        if (e == cudaSuccess) e = cudaMalloc(&I.dtlog, sizeof(double) * (size_t)std::max(steps, 1));
        if (e == cudaSuccess) e = cudaMemcpyAsync(I.st[0], soa, bytes, cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    }
    if (e != cudaSuccess) {
        free_instance(b, h);
        return bcuda(b, e, "dimgpu_batch_add");
    }
    b->inst.push_back(h);
    b->dirty = true;
    *id = h.id;
    return DIMGPU_OK;
}

int dimgpu_batch_remove(dimgpu_batch* b, int id)
{
    if (!b) return bfail(nullptr, DIMGPU_E_INVALID_ARG, "null batch");
    for (size_t i = 0; i < b->inst.size(); ++i) {
        if (b->inst[i].id != id) continue;
        // Arena mode: the range is reused only by later work on the same
        // stream, which runs after every step already enqueued.
        if (!b->arena) cudaStreamSynchronize(b->stream);
        free_instance(b, b->inst[i]);
        b->inst.erase(b->inst.begin() + (long)i);
        b->dirty = true;
        return DIMGPU_OK;
    }
    return bfail(b, DIMGPU_E_INVALID_ARG, "no instance with this id");
}

// Enqueue up to n steps of every instance with steps left, without waiting.
int dimgpu_batch_enqueue(dimgpu_batch* b, int n)
{
    if (!b) return bfail(nullptr, DIMGPU_E_INVALID_ARG, "null batch");
    if (n < 0) return bfail(b, DIMGPU_E_INVALID_ARG, "negative step count");
    if (b->inst.empty() || n == 0) return DIMGPU_OK;
    cudaError_t e = cudaSuccess;
    if (b->dirty) {
        e = rebuild(b);
        if (e != cudaSuccess) return bcuda(b, e, "dimgpu_batch_enqueue");
    }
    const BatchLaunch L = launch_args(b);
    int done = 0;
    while (done < n && e == cudaSuccess) {
        if (n - done >= kGraphSteps) {
            if (!b->graph) {
                cudaGraph_t graph;
                e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
                for (int k = 0; k < kGraphSteps && e == cudaSuccess; ++k) e = one_step(b, L);
                cudaError_t e2 = cudaStreamEndCapture(b->stream, &graph);
                if (e == cudaSuccess) e = e2;
                if (e == cudaSuccess) {
                    e = cudaGraphInstantiate(&b->graph, graph, 0);
                    cudaGraphDestroy(graph);
                }
                if (e != cudaSuccess) break;
            }
            e = cudaGraphLaunch(b->graph, b->stream);
            count_launches((long long)kGraphSteps * (2 + 6 * b->dim));  // batch_step: cfl, finalize, 6 per axis
            done += kGraphSteps;
        }
        else {
            e = one_step(b, L);
            count_launches(2 + 6 * b->dim);
            done += 1;
        }
    }
    if (e == cudaSuccess && !b->done) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(b->done, b->stream);
    if (e != cudaSuccess) return bcuda(b, e, "dimgpu_batch_enqueue");
    // host mirror: an instance with L steps left ran min(n, L) of them, and
    // ran in the last one iff L >= n
    for (auto& h : b->inst) {
        h.dev.run = h.steps_left >= n ? 1 : 0;
        h.steps_left = std::max(0, h.steps_left - n);
    }
    return DIMGPU_OK;
}


// Wait for every enqueued step; report a non-finite state or time step.
int dimgpu_batch_wait(dimgpu_batch* b)
{
    if (!b) return bfail(nullptr, DIMGPU_E_INVALID_ARG, "null batch");
    int flag = 0;
    cudaError_t e = cudaMemcpyAsync(&flag, b->err, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return bcuda(b, e, "dimgpu_batch_wait");
    if (flag) {
        cudaMemsetAsync(b->err, 0, sizeof(int), b->stream);
        if (flag & kErrNonFinite)
            return bfail(b, DIMGPU_E_NONFINITE, "dim::hllc_flux_normal: invalid density or pressure (non-finite)");
        return bfail(b, DIMGPU_E_NONFINITE, "run_dim_case: non-positive timestep");
    }
    return DIMGPU_OK;
}

// Advance every instance with steps left by up to n steps and wait.
int dimgpu_batch_run(dimgpu_batch* b, int n)
{
    const int rc = dimgpu_batch_enqueue(b, n);
    if (rc != DIMGPU_OK) return rc;
    return dimgpu_batch_wait(b);
}

// Steps run and left for one instance (host-side mirror, no device sync).
int dimgpu_batch_status(dimgpu_batch* b, int id, int* steps_done, int* steps_left)
{
    if (!b) return bfail(nullptr, DIMGPU_E_INVALID_ARG, "null batch");
    for (auto& h : b->inst) {
        if (h.id != id) continue;
        if (steps_done) *steps_done = h.steps_total - h.steps_left;
        if (steps_left) *steps_left = h.steps_left;
        return DIMGPU_OK;
    }
    return bfail(b, DIMGPU_E_INVALID_ARG, "no instance with this id");
}

// State of one instance (count = V * ncell doubles) and, if dts is not NULL,
// the dt of each step it has run (room for steps_done doubles).
int dimgpu_batch_download(dimgpu_batch* b, int id, double* soa, size_t count, double* dts)
{
    if (!b) return bfail(nullptr, DIMGPU_E_INVALID_ARG, "null batch");
    for (auto& h : b->inst) {
        if (h.id != id) continue;
        const size_t want = (size_t)(2 * h.desc.nmat + h.desc.dim) * (size_t)h.ncell;
        if (soa && count != want) return bfail(b, DIMGPU_E_INVALID_ARG, "dimgpu_batch_download: size mismatch");
        cudaError_t e = cudaSuccess;
        if (soa)
            e = cudaMemcpyAsync(soa, h.dev.st[current_buffer(b, h)], sizeof(double) * want, cudaMemcpyDeviceToHost,
                                b->stream);
        const int ndone = h.steps_total - h.steps_left;
        if (e == cudaSuccess && dts && ndone > 0)
            e = cudaMemcpyAsync(dts, h.dev.dtlog, sizeof(double) * (size_t)ndone, cudaMemcpyDeviceToHost, b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        return e == cudaSuccess ? DIMGPU_OK : bcuda(b, e, "dimgpu_batch_download");
    }
    return bfail(b, DIMGPU_E_INVALID_ARG, "no instance with this id");
}

// Persistent grid size (CTAs per launch); 0 restores SMs x 4.
int dimgpu_batch_set_grid(dimgpu_batch* b, int ctas)
{
    if (!b) return bfail(nullptr, DIMGPU_E_INVALID_ARG, "null batch");
    if (ctas < 0) return bfail(b, DIMGPU_E_INVALID_ARG, "negative grid");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    b->grid = ctas ? ctas : sms * DIMGPU_STAGED_MINB;
    drop_graphs(b);
    return DIMGPU_OK;
}

int dimgpu_batch_size(const dimgpu_batch* b) { return b ? (int)b->inst.size() : 0; }

// Cells and dt-log entries in use in the reserved arenas (0 outside arena mode).
int dimgpu_batch_arena_used(const dimgpu_batch* b, long long* cells, long long* dt_entries)
{
    if (!b) return bfail(nullptr, DIMGPU_E_INVALID_ARG, "null batch");
    if (cells) *cells = b->arena ? b->cells.used() : 0;
    if (dt_entries) *dt_entries = b->arena ? b->dts.used() : 0;
    return DIMGPU_OK;
}

// Run on a caller-owned stream (NULL: the batch's own).  Captured graphs are
// kept: replaying them on another stream is valid.
int dimgpu_batch_set_stream(dimgpu_batch* b, void* cuda_stream)
{
    if (!b) return bfail(nullptr, DIMGPU_E_INVALID_ARG, "null batch");
    cudaStreamSynchronize(b->stream);
    if (!b->own_stream) b->own_stream = b->stream;
    b->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : b->own_stream;
    return DIMGPU_OK;
}

}  // extern "C"
