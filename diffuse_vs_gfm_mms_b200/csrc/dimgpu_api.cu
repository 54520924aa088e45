// dimgpu_api.cu — the C-ABI (include/dimgpu.h): sessions owning the
// device-resident SoA state, the step orchestration of dim::advance_one_step
// (src/dim/solver/advance_step.hpp:29-149) and the stateless drop-in call.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "dim_launch.h"
#include "dimgpu.h"
#include "dimgpu_session.h"
#include "dimgpu_validate.h"

using namespace dimgpu;

namespace {

constexpr int kMaxCflBlocks = 148 * 8;
constexpr int kHistCap = 4096;
constexpr int kTotalsBlocks = 1024;

enum Kind { kSweep = 0, kCfl = 1, kBoundary = 2, kOther = 3 };

thread_local std::string g_err = "";

int fail(std::string* where, int code, const std::string& msg)
{
    if (where) *where = msg;
    g_err = msg;
    return code;
}

#define DISPATCH_ND(nm, dim, ...)                                                   \
    switch ((nm) * 10 + (dim)) {                                                    \
        case 11: { constexpr int NM = 1, D = 1; __VA_ARGS__; } break;               \
        case 12: { constexpr int NM = 1, D = 2; __VA_ARGS__; } break;               \
        case 13: { constexpr int NM = 1, D = 3; __VA_ARGS__; } break;               \
        case 21: { constexpr int NM = 2, D = 1; __VA_ARGS__; } break;               \
        case 22: { constexpr int NM = 2, D = 2; __VA_ARGS__; } break;               \
        case 23: { constexpr int NM = 2, D = 3; __VA_ARGS__; } break;               \
        case 31: { constexpr int NM = 3, D = 1; __VA_ARGS__; } break;               \
        case 32: { constexpr int NM = 3, D = 2; __VA_ARGS__; } break;               \
        case 33: { constexpr int NM = 3, D = 3; __VA_ARGS__; } break;               \
        case 41: { constexpr int NM = 4, D = 1; __VA_ARGS__; } break;               \
        case 42: { constexpr int NM = 4, D = 2; __VA_ARGS__; } break;               \
        case 43: { constexpr int NM = 4, D = 3; __VA_ARGS__; } break;               \
        default: e = cudaErrorInvalidValue; break;                                  \
    }

#define DISPATCH_D(dim, ...)                                                        \
    switch (dim) {                                                                  \
        case 1: { constexpr int D = 1; __VA_ARGS__; } break;                        \
        case 2: { constexpr int D = 2; __VA_ARGS__; } break;                        \
        case 3: { constexpr int D = 3; __VA_ARGS__; } break;                        \
        default: e = cudaErrorInvalidValue; break;                                  \
    }

bool is_euler(const dimgpu_desc& d) { return d.model == DIMGPU_MODEL_EULER; }

__device__ __forceinline__ double warp_min_f(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// dt = std::min(dt_max, every candidate) (src/dim/solver/cfl.hpp:43-63): the
// min of non-NaN values is independent of the order.
__global__ void cfl_finalize_kernel(const double* __restrict__ blockmin, int nb, double dt_max,
                                    double* __restrict__ dt, double* __restrict__ hist, int* __restrict__ err)
{
    __shared__ double red[32];
    double v = HUGE_VAL;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) v = dmin(v, blockmin[i]);
    v = warp_min_f(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = dmin(m, red[w]);
        const double d = dmin(dt_max, m);
        dt[0] = d;
        if (hist) hist[0] = d;
        if (!(d > 0.0) || !fin(d)) atomicOr(err, kErrDt);
    }
}

}  // namespace

namespace dimgpu {

std::atomic<long long> g_launches{0};

void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

cudaError_t launch_cfl_finalize(const double* blockmin, int nblocks, double dt_max, double* dt, double* hist,
                                int* err, cudaStream_t s)
{
    cfl_finalize_kernel<<<1, 256, 0, s>>>(blockmin, nblocks, dt_max, dt, hist, err);
    count_launches(1);
    return cudaGetLastError();
}

int sweep_smem_doubles(int nmat, int dim) { return (2 * nmat + dim) + (2 * nmat + dim + 1); }

int staged_scratch_doubles(int nmat, int dim)
{
    const int pv = 2 * nmat + dim + 1, v = 2 * nmat + dim, fv = 2 * nmat + dim + 2;
    return 5 * pv + nmat + 2 * v + fv;
}

void set_sessionless_error(const std::string& msg) { g_err = msg; }

int session_fail(dimgpu_session* s, int code, const std::string& msg) { return fail(s ? &s->msg : nullptr, code, msg); }

}  // namespace dimgpu


namespace {

cudaEvent_t pool_get(dimgpu_session* s)
{
    if (!s->pool.empty()) {
        cudaEvent_t e = s->pool.back();
        s->pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

struct ProfScope {
    dimgpu_session* s;
    int kind;
    cudaEvent_t a = nullptr;
    ProfScope(dimgpu_session* s_, int k) : s(s_), kind(k)
    {
        if (s->profiling) {
            a = pool_get(s);
            cudaEventRecord(a, s->stream);
        }
    }
    ~ProfScope()
    {
        if (s->profiling) {
            cudaEvent_t b = pool_get(s);
            cudaEventRecord(b, s->stream);
            s->recs.push_back({kind, a, b});
        }
    }
};

void prof_drain(dimgpu_session* s)
{
    if (s->recs.empty()) return;
    cudaStreamSynchronize(s->stream);
    for (auto& r : s->recs) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        s->prof[2 * r.kind] += ms;
        s->prof[2 * r.kind + 1] += 1.0;
        s->pool.push_back(r.a);
        s->pool.push_back(r.b);
    }
    s->recs.clear();
}

int cuda_fail(dimgpu_session* s, cudaError_t e, const char* what)
{
    if (e == cudaErrorMemoryAllocation)
        return fail(s ? &s->msg : nullptr, DIMGPU_E_OOM, std::string(what) + ": out of device memory");
    return fail(s ? &s->msg : nullptr, DIMGPU_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int validate_desc(const dimgpu_desc* d, std::string* where)
{
    std::string msg;
    const int rc = check_desc(d, &msg);
    return rc ? fail(where, rc, msg) : DIMGPU_OK;
}

int check_err(dimgpu_session* s)
{
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, s->err, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_fail(s, e, "step");
    if (h) {
        cudaMemsetAsync(s->err, 0, sizeof(int), s->stream);
        if ((h & kErrNonFinite) && is_euler(s->desc))
            return fail(&s->msg, DIMGPU_E_NONFINITE,
                        "hllc_flux_normal: invalid star state, or non-finite density (require_positive)");
        if (h & kErrNonFinite)
            return fail(&s->msg, DIMGPU_E_NONFINITE, "dim::hllc_flux_normal: invalid density or pressure (non-finite)");
        if (h & kErrDt) return fail(&s->msg, DIMGPU_E_NONFINITE, "run_dim_case: non-positive timestep");
        if (h & kErrTimeout)
            return fail(&s->msg, DIMGPU_E_TIMEOUT, "sweep: the wait for a tile copy into shared memory ran out");
    }
    return DIMGPU_OK;
}

// CFL dt of buf[cur] into s->dt (and hist slot).
cudaError_t run_cfl(dimgpu_session* s, double cfl, double dt_max, double* hist)
{
    cudaError_t e = cudaSuccess;
    int nb = 1;
    {
        ProfScope p(s, kCfl);
        const bool unsplit = s->desc.time_update == DIMGPU_TIME_UNSPLIT;
        if (is_euler(s->desc)) {
            DISPATCH_D(s->desc.dim, e = launch_euler_cfl<D>(s->g, s->M, s->buf[s->cur], cfl, unsplit, s->blockmin,
                                                            kMaxCflBlocks, &nb, s->err, s->stream));
        }
        else {
            DISPATCH_ND(s->desc.nmat, s->desc.dim,
                        e = launch_cfl<NM, D>(s->g, s->M, s->buf[s->cur], cfl, unsplit, s->blockmin, kMaxCflBlocks,
                                              &nb, s->stream, s->desc.precision != DIMGPU_PRECISION_FP64));
        }
    }
    if (e != cudaSuccess) return e;
    ProfScope p(s, kOther);
    return launch_cfl_finalize(s->blockmin, nb, dt_max, s->dt, hist, s->err, s->stream);
}

constexpr long long kStagedChunkCells = 1LL << 24;

cudaError_t ensure_staged_scratch(dimgpu_session* s)
{
    if (s->staged) return cudaSuccess;
    long long cap = s->ncell < kStagedChunkCells ? s->ncell : kStagedChunkCells;
    for (int a = 0; a < 3; ++a)
        if (s->g.N[a] > cap) cap = s->g.N[a];
    const size_t bytes = sizeof(double) * (size_t)staged_scratch_doubles(s->desc.nmat, s->desc.dim) * (size_t)cap;
    cudaError_t e = cudaMalloc(&s->staged, bytes);
    if (e == cudaSuccess) s->staged_cap = cap;
    return e;
}

cudaError_t run_sweep(dimgpu_session* s, int dir, const double* in, double* out, const FusedStep* fused = nullptr,
                      int ends_copy = 0)
{
    cudaError_t e = cudaSuccess;
    const FusedStep off{0, 0, 0.0, 0.0, nullptr, nullptr, nullptr, nullptr};
    const FusedStep& fs = fused ? *fused : off;
    if (is_euler(s->desc)) {
        ProfScope p(s, kSweep);
        DISPATCH_D(s->desc.dim, e = launch_euler_sweep<D>(s->g, s->M, dir, s->tile[dir], in, out, s->dt, s->err,
                                                          ends_copy, s->stream));
        return e;
    }
    if (s->desc.precision != DIMGPU_PRECISION_FP64) {
        e = ensure_staged_scratch(s);
        if (e != cudaSuccess) return e;
        ProfScope p(s, kSweep);
        const bool twin = s->desc.precision == DIMGPU_PRECISION_MIXED_FP64;
        DISPATCH_ND(s->desc.nmat, s->desc.dim,
                    e = launch_sweep_mixed<NM, D>(s->g, s->M, dir, in, out, s->dt, s->err, s->staged,
                                                  s->staged_cap, fs, s->stream, twin));
        return e;
    }
    if (s->schedule[dir] == DIMGPU_SCHEDULE_STAGED) {
        e = ensure_staged_scratch(s);
        if (e != cudaSuccess) return e;
    }
    ProfScope p(s, kSweep);
    if (s->schedule[dir] == DIMGPU_SCHEDULE_STAGED) {
        DISPATCH_ND(s->desc.nmat, s->desc.dim,
                    e = launch_sweep_staged<NM, D>(s->g, s->M, dir, in, out, s->dt, s->err, s->staged,
                                                   s->staged_cap, fs, s->stream));
        return e;
    }
    DISPATCH_ND(s->desc.nmat, s->desc.dim,
                e = launch_sweep<NM, D>(s->g, s->M, dir, s->tile[dir], in, out, s->dt, s->err, s->stream));
    return e;
}

cudaError_t run_bc(dimgpu_session* s, double* st)
{
    cudaError_t e = cudaSuccess;
    ProfScope p(s, kBoundary);
    if (is_euler(s->desc)) {
        DISPATCH_D(s->desc.dim, e = launch_euler_bc<D>(s->g, s->M, st, s->stream));
        return e;
    }
    DISPATCH_ND(s->desc.nmat, s->desc.dim, e = launch_bc<NM, D>(s->g, s->M, st, s->stream));
    return e;
}

// The sweeps and boundary fills of one step, dt already in s->dt
// (advance_split_directions / advance_unsplit_directions,
// src/core/fv/directional_update.hpp:8-44).
cudaError_t run_directions(dimgpu_session* s)
{
    cudaError_t e = cudaSuccess;
    const int D = s->desc.dim;
    if (s->desc.time_update == DIMGPU_TIME_SPLIT) {
        for (int dir = 0; dir < D && e == cudaSuccess; ++dir) {
            if (s->g.N[dir] > 1) {  // a line of one cell is copied unchanged (sweep_core.hpp:35-38)
                e = run_sweep(s, dir, s->buf[s->cur], s->buf[1 - s->cur]);
                s->cur = 1 - s->cur;
            }
            if (e == cudaSuccess) e = run_bc(s, s->buf[s->cur]);
        }
        return e;
    }
    // unsplit: acc = base; per axis acc += sweep(base) - base, repair; one fill
    const int base = s->cur, acc = 1 - s->cur;
    const size_t bytes = sizeof(double) * (size_t)s->V * (size_t)s->ncell;
    e = cudaMemcpyAsync(s->buf[acc], s->buf[base], bytes, cudaMemcpyDeviceToDevice, s->stream);
    for (int dir = 0; dir < D && e == cudaSuccess; ++dir) {
        const double* dstate = s->buf[base];
        if (s->g.N[dir] > 1) {
            e = run_sweep(s, dir, s->buf[base], s->buf[2], nullptr, 1);
            dstate = s->buf[2];
        }
        if (e != cudaSuccess) break;
        ProfScope p(s, kOther);
        if (is_euler(s->desc)) {
            // advance_step.hpp:617-641: accumulate every axis, enforce once after the last
            DISPATCH_D(s->desc.dim, e = launch_euler_accumulate<D>(s->g, s->M, s->buf[acc], dstate, s->buf[base],
                                                                   dir == D - 1, s->stream));
        }
        else {
            DISPATCH_ND(s->desc.nmat, s->desc.dim,
                        e = launch_accumulate<NM, D>(s->g, s->M, s->buf[acc], dstate, s->buf[base], s->stream));
        }
    }
    if (e == cudaSuccess) e = run_bc(s, s->buf[acc]);
    s->cur = acc;
    return e;
}

// One time step: the CFL dt, then the directions.  When the first sweep is
// staged (or mixed), split and the grid fits one scratch chunk, the CFL
// minimum is reduced inside that sweep's stage A instead of by a separate
// recovery pass over the state.
cudaError_t run_step(dimgpu_session* s, double cfl, double dt_max, double* hist)
{
    const bool fusable = !is_euler(s->desc) && s->desc.time_update == DIMGPU_TIME_SPLIT && s->g.N[0] > 1 &&
                         s->cfl_slot &&
                         (s->desc.precision != DIMGPU_PRECISION_FP64 ||
                          s->schedule[0] == DIMGPU_SCHEDULE_STAGED) &&
                         s->ncell <= kStagedChunkCells;
    if (!fusable) {
        cudaError_t e = run_cfl(s, cfl, dt_max, hist);
        if (e == cudaSuccess) e = run_directions(s);
        return e;
    }
    cudaError_t e = ensure_staged_scratch(s);
    if (e != cudaSuccess) return e;
    if (s->ncell > s->staged_cap) {
        e = run_cfl(s, cfl, dt_max, hist);
        if (e == cudaSuccess) e = run_directions(s);
        return e;
    }
    const FusedStep fs{1, 0, cfl, dt_max, s->cfl_slot, s->dt, hist, s->err};
    e = run_sweep(s, 0, s->buf[s->cur], s->buf[1 - s->cur], &fs);
    s->cur = 1 - s->cur;
    if (e == cudaSuccess) e = run_bc(s, s->buf[s->cur]);
    for (int dir = 1; dir < s->desc.dim && e == cudaSuccess; ++dir) {
        if (s->g.N[dir] > 1) {
            e = run_sweep(s, dir, s->buf[s->cur], s->buf[1 - s->cur]);
            s->cur = 1 - s->cur;
        }
        if (e == cudaSuccess) e = run_bc(s, s->buf[s->cur]);
    }
    return e;
}

}  // namespace

namespace dimgpu {
int session_cuda_fail(dimgpu_session* s, cudaError_t e, const char* what) { return cuda_fail(s, e, what); }

cudaError_t session_cfl_range(dimgpu_session* s, double cfl, double dt_max, long long begin, long long end)
{
    int nb = 1;
    cudaError_t e = cudaSuccess;
    const bool unsplit = s->desc.time_update == DIMGPU_TIME_UNSPLIT;
    DISPATCH_ND(s->desc.nmat, s->desc.dim,
                e = launch_cfl<NM, D>(s->g, s->M, s->buf[s->cur], cfl, unsplit, s->blockmin, kMaxCflBlocks, &nb,
                                      s->stream, s->desc.precision != DIMGPU_PRECISION_FP64, begin, end));
    if (e != cudaSuccess) return e;
    return launch_cfl_finalize(s->blockmin, nb, dt_max, s->dt, nullptr, s->err, s->stream);
}

cudaError_t session_sweep(dimgpu_session* s, int dir)
{
    cudaError_t e = cudaSuccess;
    if (s->g.N[dir] > 1) {
        e = run_sweep(s, dir, s->buf[s->cur], s->buf[1 - s->cur]);
        s->cur = 1 - s->cur;
    }
    return e;
}

cudaError_t session_bc(dimgpu_session* s) { return run_bc(s, s->buf[s->cur]); }

int session_check(dimgpu_session* s) { return check_err(s); }
}  // namespace dimgpu

namespace {

// Grid, materials and tile defaults of a session from its descriptor.
void init_geometry(dimgpu_session* s, const dimgpu_desc* desc)
{
    s->desc = *desc;
    int kind[kMaxMat];
    double gam[kMaxMat], pinf[kMaxMat];
    for (int k = 0; k < desc->nmat; ++k) {
        kind[k] = desc->mat[k].kind;
        gam[k] = desc->mat[k].gamma;
        pinf[k] = desc->mat[k].p_inf;
    }
    fill_mats(s->M, desc->nmat, kind, gam, pinf, desc->lambda_model, desc->alpha_source_floor);
    s->V = 2 * desc->nmat + desc->dim;
    s->ncell = 1;
    for (int a = 0; a < 3; ++a) {
        s->g.N[a] = desc->N[a];
        s->g.dx[a] = desc->dx[a];
        s->g.bc_lo[a] = desc->bc_lo[a];
        s->g.bc_hi[a] = desc->bc_hi[a];
        s->ncell *= desc->N[a];
    }
    s->g.ncell = s->ncell;
    s->g.stride[0] = 1;
    s->g.stride[1] = desc->N[0];
    s->g.stride[2] = (long long)desc->N[0] * desc->N[1];
    // y / z sweeps of narrow grids: fewer lines per CTA, longer segments
    for (int dir = 1; dir < 3; ++dir)
        if (desc->N[0] < 4) s->tile[dir] = {128, 1};
    // Euler sweeps: the tile shapes measured fastest on a B200 (2D blast
    // 2048^2: y sweep 128 cells x 2 lines, 2.3 % less time per step than
    // 64 x 4; 3D blast 256^3: x sweep 64 cells x 2 lines, 4 % less than
    // 128 x 1).  Results do not depend on the tile.
    if (desc->model == DIMGPU_MODEL_EULER) {
        if (desc->dim == 2 && desc->N[0] >= 4) s->tile[1] = {128, 2};
        if (desc->dim == 3) s->tile[0] = {64, 2};
    }
}

// The session's stream and small device buffers (everything but the grid).
cudaError_t alloc_small(dimgpu_session* s)
{
    cudaError_t e = cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking);
    s->stream = s->own_stream;
    if (e == cudaSuccess) e = cudaMalloc(&s->blockmin, sizeof(double) * kMaxCflBlocks);
    if (e == cudaSuccess) e = cudaMalloc(&s->dt, sizeof(double) * 2);
    if (e == cudaSuccess) e = cudaMalloc(&s->hist, sizeof(double) * kHistCap);
    if (e == cudaSuccess) e = cudaMalloc(&s->partial, sizeof(double) * kTotalsBlocks * (DIMGPU_MAX_MATERIALS + 5));
    if (e == cudaSuccess) e = cudaMalloc(&s->err, sizeof(int));
    // the fused CFL slot (a double's bits, +inf when armed) and its block ticket counter
    if (e == cudaSuccess) e = cudaMalloc(&s->cfl_slot, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) {
        static const unsigned long long armed[2] = {0x7FF0000000000000ull, 0ull};  // +inf's bits, ticket 0
        e = cudaMemcpyAsync(s->cfl_slot, armed, sizeof armed, cudaMemcpyHostToDevice, s->stream);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(s->err, 0, sizeof(int), s->stream);
    return e;
}

}  // namespace

namespace dimgpu {

long long session_grid_doubles(const dimgpu_desc* d)
{
    long long ncell = 1;
    for (int a = 0; a < 3; ++a) ncell *= d->N[a];
    const long long V = 2 * d->nmat + d->dim;
    const long long nbuf = d->time_update == DIMGPU_TIME_UNSPLIT ? 3 : 2;
    long long cap = ncell < kStagedChunkCells ? ncell : kStagedChunkCells;
    for (int a = 0; a < 3; ++a)
        if (d->N[a] > cap) cap = d->N[a];
    return nbuf * V * ncell + (long long)staged_scratch_doubles(d->nmat, d->dim) * cap;
}

int session_shell_create(dimgpu_session** out)
{
    if (!out) return fail(nullptr, DIMGPU_E_INVALID_ARG, "null output pointer");
    auto* s = new dimgpu_session();
    s->borrowed = true;
    cudaError_t e = alloc_small(s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) {
        const int rc = cuda_fail(nullptr, e, "session_shell_create");
        dimgpu_destroy(s);
        return rc;
    }
    *out = s;
    return DIMGPU_OK;
}

int session_shell_bind(dimgpu_session* s, const dimgpu_desc* desc, double* mem)
{
    int rc = validate_desc(desc, nullptr);
    if (rc) return rc;
    if (!s || !s->borrowed || !mem) return fail(nullptr, DIMGPU_E_INVALID_ARG, "session_shell_bind: bad argument");
    s->tile[0] = {128, 1};
    s->tile[1] = {64, 4};
    s->tile[2] = {64, 4};
    for (int a = 0; a < 3; ++a) s->schedule[a] = DIMGPU_SCHEDULE_STAGED;
    init_geometry(s, desc);
    const int nbuf = desc->time_update == DIMGPU_TIME_UNSPLIT ? 3 : 2;
    const size_t n = (size_t)s->V * (size_t)s->ncell;
    for (int b = 0; b < 3; ++b) s->buf[b] = b < nbuf ? mem + (size_t)b * n : nullptr;
    long long cap = s->ncell < kStagedChunkCells ? s->ncell : kStagedChunkCells;
    for (int a = 0; a < 3; ++a)
        if (s->g.N[a] > cap) cap = s->g.N[a];
    s->staged = mem + (size_t)nbuf * n;
    s->staged_cap = cap;
    s->cur = 0;
    s->pending = 0;
    s->msg.clear();
    cudaError_t e = cudaMemsetAsync(s->err, 0, sizeof(int), s->stream);
    if (e != cudaSuccess) return cuda_fail(s, e, "session_shell_bind");
    return DIMGPU_OK;
}

}  // namespace dimgpu

extern "C" {

int dimgpu_components(const dimgpu_desc* desc) { return desc ? 2 * desc->nmat + desc->dim : 0; }

const char* dimgpu_last_error(const dimgpu_session* s)
{
    if (s) return s->msg.c_str();
    return g_err.c_str();
}

int dimgpu_create(const dimgpu_desc* desc, dimgpu_session** out)
{
    if (!out) return fail(nullptr, DIMGPU_E_INVALID_ARG, "null output pointer");
    *out = nullptr;
    int rc = validate_desc(desc, nullptr);
    if (rc) return rc;
    auto* s = new dimgpu_session();
    init_geometry(s, desc);
    const size_t bytes = sizeof(double) * (size_t)s->V * (size_t)s->ncell;
    cudaError_t e = alloc_small(s);
    const int nbuf = desc->time_update == DIMGPU_TIME_UNSPLIT ? 3 : 2;
    for (int b = 0; b < nbuf && e == cudaSuccess; ++b) e = cudaMalloc(&s->buf[b], bytes);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) {
        rc = cuda_fail(nullptr, e, "dimgpu_create");
        dimgpu_destroy(s);
        return rc;
    }
    *out = s;
    return DIMGPU_OK;
}

int dimgpu_destroy(dimgpu_session* s)
{
    if (!s) return DIMGPU_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto& r : s->recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto ev : s->pool) cudaEventDestroy(ev);
    if (!s->borrowed) {
        for (int b = 0; b < 3; ++b) cudaFree(s->buf[b]);
        cudaFree(s->staged);
    }
    cudaFree(s->blockmin);
    cudaFree(s->dt);
    cudaFree(s->hist);
    cudaFree(s->partial);
    cudaFree(s->err);
    cudaFree(s->cfl_slot);
    if (s->own_stream) cudaStreamDestroy(s->own_stream);
    delete s;
    return DIMGPU_OK;
}

int dimgpu_upload(dimgpu_session* s, const double* soa, size_t count)
{
    if (!s || !soa) return fail(s ? &s->msg : nullptr, DIMGPU_E_INVALID_ARG, "null argument");
    if (count != (size_t)s->V * (size_t)s->ncell)
        return fail(&s->msg, DIMGPU_E_INVALID_ARG, "dim::advance_one_step: grid size mismatch");
    cudaError_t e = cudaMemcpyAsync(s->buf[s->cur], soa, sizeof(double) * count, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return e == cudaSuccess ? DIMGPU_OK : cuda_fail(s, e, "dimgpu_upload");
}

int dimgpu_download(dimgpu_session* s, double* soa, size_t count)
{
    if (!s || !soa) return fail(s ? &s->msg : nullptr, DIMGPU_E_INVALID_ARG, "null argument");
    if (count != (size_t)s->V * (size_t)s->ncell)
        return fail(&s->msg, DIMGPU_E_INVALID_ARG, "dimgpu_download: buffer size mismatch");
    cudaError_t e = cudaMemcpyAsync(soa, s->buf[s->cur], sizeof(double) * count, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return e == cudaSuccess ? DIMGPU_OK : cuda_fail(s, e, "dimgpu_download");
}

int dimgpu_compute_dt_cfl(dimgpu_session* s, double cfl, double dt_max, double* dt_out)
{
    if (!s) return fail(nullptr, DIMGPU_E_INVALID_ARG, "null session");
    if (!(cfl > 0.0)) return fail(&s->msg, DIMGPU_E_INVALID_ARG, "dim::compute_dt_cfl: cfl must be positive");
    if (!(dt_max > 0.0)) return fail(&s->msg, DIMGPU_E_INVALID_ARG, "dim::compute_dt_cfl: dt_max must be positive");
    cudaError_t e = run_cfl(s, cfl, dt_max, nullptr);
    double h = 0.0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, s->dt, sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_fail(s, e, "dimgpu_compute_dt_cfl");
    cudaMemsetAsync(s->err, 0, sizeof(int), s->stream);  // dt <= 0 is the caller's decision here
    if (dt_out) *dt_out = h;
    return DIMGPU_OK;
}

int dimgpu_sweep_direction(dimgpu_session* s, int dir, double dt)
{
    if (!s) return fail(nullptr, DIMGPU_E_INVALID_ARG, "null session");
    if (dir < 0 || dir >= s->desc.dim) return fail(&s->msg, DIMGPU_E_INVALID_ARG, "sweep direction out of range");
    cudaError_t e = cudaMemcpyAsync(s->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess && s->g.N[dir] > 1) {
        e = run_sweep(s, dir, s->buf[s->cur], s->buf[1 - s->cur]);
        s->cur = 1 - s->cur;
    }
    if (e != cudaSuccess) return cuda_fail(s, e, "dimgpu_sweep_direction");
    return check_err(s);
}

int dimgpu_apply_boundary_conditions(dimgpu_session* s)
{
    if (!s) return fail(nullptr, DIMGPU_E_INVALID_ARG, "null session");
    cudaError_t e = run_bc(s, s->buf[s->cur]);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return e == cudaSuccess ? DIMGPU_OK : cuda_fail(s, e, "dimgpu_apply_boundary_conditions");
}

int dimgpu_step(dimgpu_session* s, double cfl, double dt_max, double* dt_out, dimgpu_phase_times* times)
{
    if (!s) return fail(nullptr, DIMGPU_E_INVALID_ARG, "null session");
    if (!(cfl > 0.0)) return fail(&s->msg, DIMGPU_E_INVALID_ARG, "dim::compute_dt_cfl: cfl must be positive");
    if (!(dt_max > 0.0)) return fail(&s->msg, DIMGPU_E_INVALID_ARG, "dim::compute_dt_cfl: dt_max must be positive");
    const bool was = s->profiling;
    double before[8];
    if (times) {
        prof_drain(s);
        std::memcpy(before, s->prof, sizeof before);
        s->profiling = true;
    }
    cudaError_t e = run_step(s, cfl, dt_max, nullptr);
    double h = 0.0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, s->dt, sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (times) {
        prof_drain(s);
        s->profiling = was;
        times->cfl_ms = s->prof[2 * kCfl] - before[2 * kCfl] + s->prof[2 * kOther] - before[2 * kOther];
        times->sweep_ms = s->prof[2 * kSweep] - before[2 * kSweep];
        times->boundary_ms = s->prof[2 * kBoundary] - before[2 * kBoundary];
        if (!was) std::memset(s->prof, 0, sizeof s->prof);
    }
    if (e != cudaSuccess) return cuda_fail(s, e, "dimgpu_step");
    if (dt_out) *dt_out = h;
    int hflag = 0;
    e = cudaMemcpyAsync(&hflag, s->err, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_fail(s, e, "dimgpu_step");
    if (hflag & kErrNonFinite) return check_err(s);
    if (hflag) cudaMemsetAsync(s->err, 0, sizeof(int), s->stream);  // dt <= 0: returned to the caller
    return DIMGPU_OK;
}

int dimgpu_enqueue_steps(dimgpu_session* s, int n, double cfl, double dt_max)
{
    if (!s) return fail(nullptr, DIMGPU_E_INVALID_ARG, "null session");
    if (n < 0) return fail(&s->msg, DIMGPU_E_INVALID_ARG, "negative step count");
    if (!(cfl > 0.0)) return fail(&s->msg, DIMGPU_E_INVALID_ARG, "dim::compute_dt_cfl: cfl must be positive");
    if (!(dt_max > 0.0)) return fail(&s->msg, DIMGPU_E_INVALID_ARG, "dim::compute_dt_cfl: dt_max must be positive");
    if (s->pending + n > kHistCap)
        return fail(&s->msg, DIMGPU_E_INVALID_ARG, "more than 4096 steps enqueued: call dimgpu_collect first");
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < n && e == cudaSuccess; ++k) {
        e = run_step(s, cfl, dt_max, s->hist + s->pending);
        if (e == cudaSuccess) ++s->pending;
    }
    return e == cudaSuccess ? DIMGPU_OK : cuda_fail(s, e, "dimgpu_enqueue_steps");
}

int dimgpu_collect(dimgpu_session* s, double* dt_out, int capacity, int* count)
{
    if (!s) return fail(nullptr, DIMGPU_E_INVALID_ARG, "null session");
    const int n = s->pending;
    s->pending = 0;
    if (count) *count = n;
    cudaError_t e = cudaSuccess;
    if (dt_out && n > 0) {
        if (capacity < n) return fail(&s->msg, DIMGPU_E_INVALID_ARG, "dimgpu_collect: dt_out too small");
        e = cudaMemcpyAsync(dt_out, s->hist, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream);
    }
    if (e != cudaSuccess) return cuda_fail(s, e, "dimgpu_collect");
    return check_err(s);
}

int dimgpu_steps(dimgpu_session* s, int n, double cfl, double dt_max, double* dt_out)
{
    if (!s) return fail(nullptr, DIMGPU_E_INVALID_ARG, "null session");
    if (n < 0) return fail(&s->msg, DIMGPU_E_INVALID_ARG, "negative step count");
    int rc = dimgpu_collect(s, nullptr, 0, nullptr);
    if (rc) return rc;
    for (int done = 0; done < n;) {
        const int chunk = (n - done < kHistCap) ? (n - done) : kHistCap;
        rc = dimgpu_enqueue_steps(s, chunk, cfl, dt_max);
        if (rc) return rc;
        rc = dimgpu_collect(s, dt_out ? dt_out + done : nullptr, chunk, nullptr);
        if (rc) return rc;
        done += chunk;
    }
    return DIMGPU_OK;
}

int dimgpu_totals(dimgpu_session* s, double* out)
{
    if (!s || !out) return fail(s ? &s->msg : nullptr, DIMGPU_E_INVALID_ARG, "null argument");
    double volume = 1.0;
    for (int a = 0; a < s->desc.dim; ++a) volume *= s->desc.dx[a];
    int nb = 1;
    cudaError_t e = cudaSuccess;
    DISPATCH_ND(s->desc.nmat, s->desc.dim,
                e = launch_totals<NM, D>(s->g, s->buf[s->cur], volume, s->partial, kTotalsBlocks, &nb, s->stream));
    const int NV = s->desc.nmat + 1 + s->desc.dim + 1;
    std::vector<double> h((size_t)nb * NV);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h.data(), s->partial, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_fail(s, e, "dimgpu_totals");
    for (int v = 0; v < NV; ++v) {
        double acc = 0.0;
        for (int b = 0; b < nb; ++b) acc += h[(size_t)b * NV + v];
        out[v] = acc;
    }
    return DIMGPU_OK;
}

int dimgpu_boundary_flux(dimgpu_session* s, double* out)
{
    if (!s || !out) return fail(s ? &s->msg : nullptr, DIMGPU_E_INVALID_ARG, "null argument");
    if (is_euler(s->desc))
        return fail(&s->msg, DIMGPU_E_UNSUPPORTED, "dimgpu_boundary_flux: the DIM model only");
    int nb = 1;
    cudaError_t e = cudaSuccess;
    DISPATCH_ND(s->desc.nmat, s->desc.dim,
                e = launch_boundary_flux<NM, D>(s->g, s->M, s->buf[s->cur], s->partial, kTotalsBlocks, &nb,
                                                s->stream));
    const int NV = s->desc.nmat + 1 + s->desc.dim + 1;
    std::vector<double> h((size_t)nb * NV);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h.data(), s->partial, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_fail(s, e, "dimgpu_boundary_flux");
    for (int v = 0; v < NV; ++v) {
        double acc = 0.0;
        for (int b = 0; b < nb; ++b) acc += h[(size_t)b * NV + v];
        out[v] = acc;
    }
    return DIMGPU_OK;
}

int dimgpu_set_stream(dimgpu_session* s, void* cuda_stream)
{
    if (!s) return fail(nullptr, DIMGPU_E_INVALID_ARG, "null session");
    cudaStreamSynchronize(s->stream);
    s->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : s->own_stream;
    return DIMGPU_OK;
}

int dimgpu_set_tile(dimgpu_session* s, int dir, int T, int W)
{
    if (!s) return fail(nullptr, DIMGPU_E_INVALID_ARG, "null session");
    if (dir < 0 || dir > 2 || T < 8 || W < 1 || T * W > 256 || (T * W) % 32 != 0)
        return fail(&s->msg, DIMGPU_E_INVALID_ARG, "tile must satisfy 8 <= T, T*W <= 256, T*W a multiple of 32");
    s->tile[dir] = {T, W};
    return DIMGPU_OK;
}

int dimgpu_set_schedule(dimgpu_session* s, int dir, int schedule)
{
    if (!s) return fail(nullptr, DIMGPU_E_INVALID_ARG, "null session");
    if (dir < 0 || dir > 2 || (schedule != DIMGPU_SCHEDULE_FUSED && schedule != DIMGPU_SCHEDULE_STAGED))
        return fail(&s->msg, DIMGPU_E_INVALID_ARG, "schedule must be DIMGPU_SCHEDULE_FUSED or _STAGED");
    s->schedule[dir] = schedule;
    return DIMGPU_OK;
}

int dimgpu_profile(dimgpu_session* s, int enable)
{
    if (!s) return fail(nullptr, DIMGPU_E_INVALID_ARG, "null session");
    prof_drain(s);
    std::memset(s->prof, 0, sizeof s->prof);
    s->profiling = enable != 0;
    return DIMGPU_OK;
}

long long dimgpu_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

int dimgpu_profile_read(dimgpu_session* s, double* out8)
{
    if (!s || !out8) return fail(s ? &s->msg : nullptr, DIMGPU_E_INVALID_ARG, "null argument");
    prof_drain(s);
    std::memcpy(out8, s->prof, sizeof s->prof);
    return DIMGPU_OK;
}

// One cached session per calling thread, rebuilt when the descriptor changes.
int dimgpu_advance_one_step(const dimgpu_desc* desc, const double* soa_in, double* soa_out, double cfl,
                            double dt_max, double* dt_out, dimgpu_phase_times* times)
{
    thread_local dimgpu_session* cached = nullptr;
    thread_local dimgpu_desc cached_desc;
    int rc = validate_desc(desc, nullptr);
    if (rc) return rc;
    if (!cached || std::memcmp(&cached_desc, desc, sizeof(dimgpu_desc)) != 0) {
        dimgpu_destroy(cached);
        cached = nullptr;
        rc = dimgpu_create(desc, &cached);
        if (rc) return rc;
        cached_desc = *desc;
    }
    const size_t count = (size_t)cached->V * (size_t)cached->ncell;
    if ((rc = dimgpu_upload(cached, soa_in, count))) { g_err = cached->msg; return rc; }
    if ((rc = dimgpu_step(cached, cfl, dt_max, dt_out, times))) { g_err = cached->msg; return rc; }
    if ((rc = dimgpu_download(cached, soa_out, count))) { g_err = cached->msg; return rc; }
    return DIMGPU_OK;
}

}  // extern "C"
