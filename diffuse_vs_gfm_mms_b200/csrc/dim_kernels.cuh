// dim_kernels.cuh — CUDA kernels of the DIM step for sm_100a.
//
// State: FP64 structure of arrays in HBM, component c of cell i at
// state[c * ncell + i], x-fastest.  One sweep kernel launch advances every
// line along one axis by the split MUSCL-Hancock / HLLC update; the CFL
// kernel reduces the step; the boundary kernel refills the boundary shell.
#pragma once

#include <cuda.h>
#include <cstring>
#include <utility>
#include <cuda_runtime.h>

#include "dim_launch.h"
#include "pdl.cuh"
#include "fastdiv.h"
#include "dim_line.h"
#include "dim_mixed.h"
#include "dimgpu.h"

namespace dimgpu {

// ---- SoA load / store ----------------------------------------------------------
template<int NM, int D>
__device__ __forceinline__ void load_cell(const double* __restrict__ s, long long ncell, long long i,
                                          State<NM, D>& U)
{
    int q = 0;
#pragma unroll
    for (int k = 0; k < NM; ++k) U.m[k] = __ldg(s + (q++) * ncell + i);
#pragma unroll
    for (int d = 0; d < D; ++d) U.mom[d] = __ldg(s + (q++) * ncell + i);
    U.E = __ldg(s + (q++) * ncell + i);
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) U.a[k] = __ldg(s + (q++) * ncell + i);
}

template<int NM, int D>
__device__ __forceinline__ void store_cell(double* __restrict__ s, long long ncell, long long i,
                                           const State<NM, D>& U)
{
    int q = 0;
#pragma unroll
    for (int k = 0; k < NM; ++k) s[(q++) * ncell + i] = U.m[k];
#pragma unroll
    for (int d = 0; d < D; ++d) s[(q++) * ncell + i] = U.mom[d];
    s[(q++) * ncell + i] = U.E;
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) s[(q++) * ncell + i] = U.a[k];
}

// ---- shared-memory records: variable v of slot t at sm[v * NT + t] -------------
template<int NM, int D>
__device__ __forceinline__ void sm_put(double* sm, int NT, int t, int v0, const Prim<NM, D>& P)
{
    int v = v0;
#pragma unroll
    for (int k = 0; k < NM; ++k) sm[(v++) * NT + t] = P.rho[k];
#pragma unroll
    for (int k = 0; k < NM; ++k) sm[(v++) * NT + t] = P.alpha[k];
#pragma unroll
    for (int d = 0; d < D; ++d) sm[(v++) * NT + t] = P.vel[d];
    sm[v * NT + t] = P.p;
}

template<int NM, int D>
__device__ __forceinline__ void sm_get(const double* sm, int NT, int t, int v0, Prim<NM, D>& P)
{
    int v = v0;
#pragma unroll
    for (int k = 0; k < NM; ++k) P.rho[k] = sm[(v++) * NT + t];
#pragma unroll
    for (int k = 0; k < NM; ++k) P.alpha[k] = sm[(v++) * NT + t];
#pragma unroll
    for (int d = 0; d < D; ++d) P.vel[d] = sm[(v++) * NT + t];
    P.p = sm[v * NT + t];
}

template<int NM, int D>
__device__ __forceinline__ void sm_put(double* sm, int NT, int t, int v0, const State<NM, D>& U)
{
    int v = v0;
#pragma unroll
    for (int k = 0; k < NM; ++k) sm[(v++) * NT + t] = U.m[k];
#pragma unroll
    for (int d = 0; d < D; ++d) sm[(v++) * NT + t] = U.mom[d];
    sm[(v++) * NT + t] = U.E;
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) sm[(v++) * NT + t] = U.a[k];
}

template<int NM, int D>
__device__ __forceinline__ void sm_get(const double* sm, int NT, int t, int v0, State<NM, D>& U)
{
    int v = v0;
#pragma unroll
    for (int k = 0; k < NM; ++k) U.m[k] = sm[(v++) * NT + t];
#pragma unroll
    for (int d = 0; d < D; ++d) U.mom[d] = sm[(v++) * NT + t];
    U.E = sm[(v++) * NT + t];
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) U.a[k] = sm[(v++) * NT + t];
}

template<int NM, int D>
__device__ __forceinline__ void sm_put(double* sm, int NT, int t, const FaceD<NM, D>& f)
{
    int v = 0;
#pragma unroll
    for (int k = 0; k < NM; ++k) sm[(v++) * NT + t] = f.F.m[k];
#pragma unroll
    for (int d = 0; d < D; ++d) sm[(v++) * NT + t] = f.F.mom[d];
    sm[(v++) * NT + t] = f.F.E;
    sm[(v++) * NT + t] = f.fv;
#pragma unroll
    for (int k = 0; k < NM; ++k) sm[(v++) * NT + t] = f.af[k];
}

template<int NM, int D>
__device__ __forceinline__ void sm_get(const double* sm, int NT, int t, FaceD<NM, D>& f)
{
    int v = 0;
#pragma unroll
    for (int k = 0; k < NM; ++k) f.F.m[k] = sm[(v++) * NT + t];
#pragma unroll
    for (int d = 0; d < D; ++d) f.F.mom[d] = sm[(v++) * NT + t];
    f.F.E = sm[(v++) * NT + t];
    f.fv = sm[(v++) * NT + t];
#pragma unroll
    for (int k = 0; k < NM; ++k) f.af[k] = sm[(v++) * NT + t];
}

__host__ __device__ constexpr int kPrimVars(int nm, int d) { return 2 * nm + d + 1; }
__host__ __device__ constexpr int kStateVars(int nm, int d) { return 2 * nm + d; }
// Largest live set between two stages: LS + PLS (stage C -> D).
__host__ __device__ constexpr int kSweepSmemVars(int nm, int d) { return kStateVars(nm, d) + kPrimVars(nm, d); }

__host__ __device__ constexpr int kStateVarsT(int nm, int d) { return 2 * nm + d; }

// ---- the sweep kernel ------------------------------------------------------------
//
// CTA = T*W threads over W lines x T consecutive cells of each line.  For the
// x sweep the T cells of a line are consecutive threads (coalesced); for the
// y / z sweeps the W lines are W consecutive x columns and sit in consecutive
// threads (coalesced across lines).  Cell positions pos = 0..T-1 map to line
// cells tile*(T-6) - 3 + pos; positions 3..T-4 are written, the rest is halo.
// Stage k+1 of a cell reads stage-k results of its two neighbours from shared
// memory, so every stage is separated by one __syncthreads.
//
// Input staging.  With `tma`, the CTA's whole input tile — its cells plus the
// 3-cell halo on each side, every component — arrives in shared memory in
// one TMA copy (cp.async.bulk.tensor, no multicast; the tensor map covers the
// input buffer of this GPU only), issued by thread 0 and awaited on an
// mbarrier; each thread then reads its cell from shared memory.  Tensor
// views (innermost first): x sweep (x, line, component), box (T + 2, W, V),
// its x start rounded down to an even cell so that it is 16-byte aligned;
// y sweep (x, y, z, component), box (W, T, 1, V); z sweep box (W, 1, T, V).
// Cells outside the grid arrive as zeros and are never read.  The wait is
// bounded: when it runs out, the CTA sets kErrTimeout, waits once more (also
// bounded) for the copy in flight, and returns without computing.
struct TileMap {
    CUtensorMap map;
};

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

// Thread 0 only: bounded wait for phase 0 of the barrier.  True if complete.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, long long limit)
{
    for (long long it = 0; it < limit; ++it) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(bar)
            : "memory");
        if (done) return true;
        __nanosleep(64);
    }
    return false;
}

template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, 2) sweep_kernel(const double* __restrict__ in, double* __restrict__ out,
                                                    __grid_constant__ const Grid g, __grid_constant__ const Mats M, int T, int W, int ntile, int ngx,
                                                    const double* __restrict__ dtp, int* __restrict__ err,
                                                    const __grid_constant__ TileMap tmap, int tma)
{
    extern __shared__ __align__(128) double sm_raw[];
    constexpr int V = kStateVarsT(NM, D);
    // TMA tile first (128-byte aligned), stage records after it
    const int tile_doubles = tma ? ((DIR == 0 ? (T + 2) : T) * W * V + 15) / 16 * 16 : 0;
    double* tile_sm = sm_raw;
    double* sm = sm_raw + tile_doubles;
    const int NT = T * W;
    const int t = threadIdx.x;
    const int n = g.N[DIR];
    const int OUT = T - 6;

    int pos, j, s;
    if (DIR == 0) { pos = t % T; j = t / T; s = 1; }
    else { j = t % W; pos = t / W; s = W; }

    // line of this thread and its base address
    long long bid = blockIdx.x;
    int tile;
    long long base;
    bool line_ok;
    long long sline;
    if (DIR == 0) {
        tile = (int)(bid % ntile);
        const long long L = (bid / ntile) * W + j;
        const long long nlines = g.ncell / g.N[0];
        line_ok = L < nlines;
        base = L * g.N[0];
        sline = 1;
    }
    else {
        const int gx = (int)(bid % ngx);
        const long long rest = bid / ngx;
        tile = (int)(rest % ntile);
        const long long other = rest / ntile;
        const int x = gx * W + j;
        line_ok = x < g.N[0];
        if (DIR == 1) base = x + other * g.stride[2];
        else base = x + other * g.stride[1];
        sline = g.stride[DIR];
    }
    const int gi = tile * OUT - 3 + pos;
    const bool valid = line_ok && gi >= 0 && gi < n;
    const bool first = gi == 0, last = gi == n - 1;
    const bool end = first || last || n < 3;
    const long long cell = base + (long long)gi * sline;

    const double dt = *dtp;
    const double dx = g.dx[DIR];

    // ---- input tile
    int xoff = 0;  // x sweep: this tile's first cell minus the aligned box start
    if (tma) {
        __shared__ __align__(8) unsigned long long bar;
        __shared__ int ok;
        const unsigned bar_a = smem_u32(&bar);
        if (t == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        int c0, c1, c2;  // box start: innermost coordinate first
        const int x0 = tile * OUT - 3;
        if (DIR == 0) {
            const int xa = x0 - (x0 & 1);
            xoff = x0 - xa;
            c0 = xa;
            c1 = (int)((bid / ntile) * W);
            c2 = 0;
        }
        else {
            const int gx = (int)(bid % ngx);
            const long long other = (bid / ngx) / ntile;
            c0 = gx * W;
            c1 = DIR == 1 ? x0 : (int)other;
            c2 = DIR == 1 ? (int)other : x0;
        }
        if (t == 0) {
            const unsigned bytes = (unsigned)((DIR == 0 ? (T + 2) : T) * W * V * 8);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(bytes) : "memory");
            const unsigned dst = smem_u32(tile_sm);
            const unsigned long long map = reinterpret_cast<unsigned long long>(&tmap.map);
            if (DIR == 0)
                asm volatile(
                    "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                    " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
                    "l"(map), "r"(c0), "r"(c1), "r"(0), "r"(bar_a)
                    : "memory");
            else
                asm volatile(
                    "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                    " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
                    "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(0), "r"(bar_a)
                    : "memory");
            bool done = mbar_wait_bounded(bar_a, 1LL << 22);
            if (!done) {
                atomicOr(err, kErrTimeout);
                mbar_wait_bounded(bar_a, 1LL << 22);
            }
            ok = done ? 1 : 0;
        }
        __syncthreads();
        if (!ok) return;
        mbar_wait_bounded(bar_a, 1);  // complete: this thread's acquire of the tile
    }

    // ---- stage A
    State<NM, D> U;
    CellA<NM, D> A;
    if (valid) {
        if (tma) {
            // shared-memory index of component 0 of this thread's cell
            const int rows = DIR == 0 ? (T + 2) : T;
            const int i0 = DIR == 0 ? (j * rows + xoff + pos) : (pos * W + j);
            const int cs = rows * W;  // component stride
            int q = 0;
#pragma unroll
            for (int k = 0; k < NM; ++k) U.m[k] = tile_sm[(q++) * cs + i0];
#pragma unroll
            for (int d = 0; d < D; ++d) U.mom[d] = tile_sm[(q++) * cs + i0];
            U.E = tile_sm[(q++) * cs + i0];
#pragma unroll
            for (int k = 0; k < NM - 1; ++k) U.a[k] = tile_sm[(q++) * cs + i0];
        }
        else {
            load_cell<NM, D>(in, g.ncell, cell, U);
        }
        stage_a<NM, D>(M, U, A);
        sm_put<NM, D>(sm, NT, t, 0, A.Pe);
    }
    __syncthreads();

    // ---- stage B
    const bool needB = valid && (end || (pos >= 1 && pos <= T - 2));
    State<NM, D> Uh;
    Prim<NM, D> Ph;
    if (needB) {
        Prim<NM, D> lo, hi;
        if (!end) {
            sm_get<NM, D>(sm, NT, t - s, 0, lo);
            sm_get<NM, D>(sm, NT, t + s, 0, hi);
        }
        stage_b<NM, D>(M, U, A, lo, hi, end, DIR, dt, dx, Uh, Ph);
    }
    __syncthreads();
    if (needB) sm_put<NM, D>(sm, NT, t, 0, Ph);
    __syncthreads();

    // ---- stage C
    auto needC_at = [&](int p, int gidx) {
        const bool v = line_ok && gidx >= 0 && gidx < n;
        const bool e = gidx == 0 || gidx == n - 1 || n < 3;
        return v && (e || (p >= 2 && p <= T - 3));
    };
    const bool needC = needC_at(pos, gi);
    State<NM, D> LS, RS;
    Prim<NM, D> PLS, PRS;
    if (needC) {
        Prim<NM, D> lo, hi;
        if (!end) {
            sm_get<NM, D>(sm, NT, t - s, 0, lo);
            sm_get<NM, D>(sm, NT, t + s, 0, hi);
        }
        stage_c<NM, D>(M, U, A, Ph, lo, hi, end, LS, RS, PLS, PRS);
    }
    __syncthreads();
    if (needC) {
        sm_put<NM, D>(sm, NT, t, 0, LS);
        sm_put<NM, D>(sm, NT, t, kStateVars(NM, D), PLS);
    }
    __syncthreads();

    // ---- stage D: face between this cell and the next one
    const bool needD = needC && pos + 1 <= T - 1 && gi + 1 < n && needC_at(pos + 1, gi + 1);
    FaceD<NM, D> fd;
    if (needD) {
        State<NM, D> UR;
        Prim<NM, D> PR;
        sm_get<NM, D>(sm, NT, t + s, 0, UR);
        sm_get<NM, D>(sm, NT, t + s, kStateVars(NM, D), PR);
        if (!stage_d<NM, D>(M, RS, PRS, UR, PR, DIR, fd)) atomicOr(err, kErrNonFinite);
    }
    __syncthreads();
    if (needD) sm_put<NM, D>(sm, NT, t, fd);
    __syncthreads();

    // ---- stage E: the outputs
    if (valid && pos >= 3 && pos <= T - 4) {
        FaceD<NM, D> lo;
        if (!first) sm_get<NM, D>(sm, NT, t - s, lo);
        State<NM, D> Un;
        stage_e<NM, D>(M, U, A, first ? nullptr : &lo, last ? nullptr : &fd, first, last, dt, dx, Un);
        store_cell<NM, D>(out, g.ncell, cell, Un);
    }
}

// ---- the staged sweep ---------------------------------------------------------------
//
// The same five stages as sweep_kernel, one kernel per stage over a chunk of
// whole lines, with the per-cell results handed between stages through a
// scratch area in global memory instead of shared memory.  Each kernel is
// small (fits the instruction cache), needs no CTA barrier and computes every
// cell exactly once (no tile halo); the price is the scratch traffic, about
// ten times the state traffic of the fused kernel, which the step's
// arithmetic intensity leaves room for.
//
// Work item t of a chunk of nl lines x n cells: for the x sweep t = line*n +
// i (cells of a line are consecutive threads), for y / z t = i*nl + line
// (consecutive threads are consecutive x columns).  Scratch record var v of
// item t sits at buf[v * cap + t]; the neighbour along the line is t +- s
// with s = 1 (x) or nl (y, z).
struct LineSet {
    long long L0;  // first line of the chunk
    int nl;        // lines in the chunk
    int n;         // cells per line
    // Dividers by n, nl and the grid's N[0], set on the host (item and line
    // indices stay below 2^32: a chunk holds at most max(2^24, longest
    // line) cells, a batch instance at most 2^31 - 1, and a grid's line
    // count is bounded by HBM far below 2^32).
    FastDiv by_n, by_nl, by_n0;
    __host__ void set_dividers(int n0)
    {
        by_n.set((unsigned)n);
        by_nl.set((unsigned)nl);
        by_n0.set((unsigned)n0);
    }
};

template<int NM, int D>
struct StagedBufs {
    double* P;    // cons_to_prim(U)             kPrimVars
    double* ck;   // alpha-RHS sound speeds       NM
    double* Pe;   // enforce(P)                   kPrimVars
    double* Ph;   // half-step primitive          kPrimVars
    double* LS;   // left face state              kStateVars
    double* RS;   // right face state             kStateVars
    double* PLS;  // cons_to_prim(LS)             kPrimVars
    double* PRS;  // cons_to_prim(RS)             kPrimVars
    double* F;    // face i|i+1: flux, s*, alpha flux   2*NM + D + 2
    long long cap;
};

__host__ __device__ constexpr int kFaceVars(int nm, int d) { return 2 * nm + d + 2; }
// P, Pe, Ph, PLS, PRS + ck + LS, RS + the face record
__host__ __device__ constexpr int kStagedVars(int nm, int d)
{
    return 5 * kPrimVars(nm, d) + nm + 2 * kStateVars(nm, d) + kFaceVars(nm, d);
}

template<int NM, int D>
__device__ __forceinline__ void g_put(double* b, long long cap, long long t, const Prim<NM, D>& P)
{
    int v = 0;
#pragma unroll
    for (int k = 0; k < NM; ++k) b[(v++) * cap + t] = P.rho[k];
#pragma unroll
    for (int k = 0; k < NM; ++k) b[(v++) * cap + t] = P.alpha[k];
#pragma unroll
    for (int d = 0; d < D; ++d) b[(v++) * cap + t] = P.vel[d];
    b[v * cap + t] = P.p;
}

template<int NM, int D>
__device__ __forceinline__ void g_get(const double* b, long long cap, long long t, Prim<NM, D>& P)
{
    int v = 0;
#pragma unroll
    for (int k = 0; k < NM; ++k) P.rho[k] = b[(v++) * cap + t];
#pragma unroll
    for (int k = 0; k < NM; ++k) P.alpha[k] = b[(v++) * cap + t];
#pragma unroll
    for (int d = 0; d < D; ++d) P.vel[d] = b[(v++) * cap + t];
    P.p = b[v * cap + t];
}

template<int NM, int D>
__device__ __forceinline__ void g_put(double* b, long long cap, long long t, const State<NM, D>& U)
{
    int v = 0;
#pragma unroll
    for (int k = 0; k < NM; ++k) b[(v++) * cap + t] = U.m[k];
#pragma unroll
    for (int d = 0; d < D; ++d) b[(v++) * cap + t] = U.mom[d];
    b[(v++) * cap + t] = U.E;
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) b[(v++) * cap + t] = U.a[k];
}

template<int NM, int D>
__device__ __forceinline__ void g_get(const double* b, long long cap, long long t, State<NM, D>& U)
{
    int v = 0;
#pragma unroll
    for (int k = 0; k < NM; ++k) U.m[k] = b[(v++) * cap + t];
#pragma unroll
    for (int d = 0; d < D; ++d) U.mom[d] = b[(v++) * cap + t];
    U.E = b[(v++) * cap + t];
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) U.a[k] = b[(v++) * cap + t];
}

template<int NM, int D>
__device__ __forceinline__ void g_put(double* b, long long cap, long long t, const FaceD<NM, D>& f)
{
    int v = 0;
#pragma unroll
    for (int k = 0; k < NM; ++k) b[(v++) * cap + t] = f.F.m[k];
#pragma unroll
    for (int d = 0; d < D; ++d) b[(v++) * cap + t] = f.F.mom[d];
    b[(v++) * cap + t] = f.F.E;
    b[(v++) * cap + t] = f.fv;
#pragma unroll
    for (int k = 0; k < NM; ++k) b[(v++) * cap + t] = f.af[k];
}

template<int NM, int D>
__device__ __forceinline__ void g_get(const double* b, long long cap, long long t, FaceD<NM, D>& f)
{
    int v = 0;
#pragma unroll
    for (int k = 0; k < NM; ++k) f.F.m[k] = b[(v++) * cap + t];
#pragma unroll
    for (int d = 0; d < D; ++d) f.F.mom[d] = b[(v++) * cap + t];
    f.F.E = b[(v++) * cap + t];
    f.fv = b[(v++) * cap + t];
#pragma unroll
    for (int k = 0; k < NM; ++k) f.af[k] = b[(v++) * cap + t];
}

// Stage A's enforced primitive of item t: the stored record, or (with
// DIMGPU_STAGED_NO_PE) the primitive P re-enforced on load — the same bits
// as stage A's enforce_positive_primitive, one record less written per cell.
template<int NM, int D>
__device__ __forceinline__ void get_pe(const StagedBufs<NM, D>& b, long long t, Prim<NM, D>& Pe)
{
    if (DIMGPU_STAGED_NO_PE) {
        g_get<NM, D>(b.P, b.cap, t, Pe);
        enforce_positive_primitive<NM, D>(Pe);
    }
    else {
        g_get<NM, D>(b.Pe, b.cap, t, Pe);
    }
}

// A face flux record (stage B's face fluxes, kept in the LS / RS slots until
// stage C writes the face states there).
template<int NM, int D>
__device__ __forceinline__ void g_put(double* b, long long cap, long long t, const Flux<NM, D>& F)
{
    int v = 0;
#pragma unroll
    for (int k = 0; k < NM; ++k) b[(v++) * cap + t] = F.m[k];
#pragma unroll
    for (int d = 0; d < D; ++d) b[(v++) * cap + t] = F.mom[d];
    b[v * cap + t] = F.E;
}

template<int NM, int D>
__device__ __forceinline__ void g_get(const double* b, long long cap, long long t, Flux<NM, D>& F)
{
    int v = 0;
#pragma unroll
    for (int k = 0; k < NM; ++k) F.m[k] = b[(v++) * cap + t];
#pragma unroll
    for (int d = 0; d < D; ++d) F.mom[d] = b[(v++) * cap + t];
    F.E = b[v * cap + t];
}

// Item t of a chunk: its cell index along the line, its cell in the grid and
// the scratch stride between neighbours along the line.
// FD: divide through the LineSet's dividers (set on the host: per chunk for
// a session's kernels, per instance in the batch's instance table) instead
// of 64-bit integer division.
template<int DIR, bool FD = DIMGPU_STAGED_FASTDIV>
struct StagedItem {
    int gi;
    long long cell;
    long long s;
    __device__ __forceinline__ StagedItem(const Grid& g, const LineSet& ls, long long t)
    {
        long long lrel;
        if (FD) {
            const unsigned u = (unsigned)t;
            if (DIR == 0) {
                const unsigned q = ls.by_n.div(u);
                lrel = q;
                gi = (int)(u - q * (unsigned)ls.n);
                s = 1;
            }
            else {
                const unsigned q = ls.by_nl.div(u);
                gi = (int)q;
                lrel = u - q * (unsigned)ls.nl;
                s = ls.nl;
            }
        }
        else if (DIR == 0) { lrel = t / ls.n; gi = (int)(t % ls.n); s = 1; }
        else { gi = (int)(t / ls.nl); lrel = t % ls.nl; s = ls.nl; }
        const long long L = ls.L0 + lrel;
        long long base;
        if (DIR == 0) base = L * g.N[0];
        else {
            long long lx, ly;
            if (FD) {
                const unsigned q = ls.by_n0.div((unsigned)L);
                ly = q;
                lx = (unsigned)L - q * (unsigned)g.N[0];
            }
            else {
                lx = L % g.N[0];
                ly = L / g.N[0];
            }
            base = lx + ly * g.stride[DIR == 1 ? 2 : 1];
        }
        cell = base + (long long)gi * g.stride[DIR];
    }
};


// Optional CFL reduction fused into stage A of the first sweep of a step:
// stage A recovers every cell's primitive from the very state the CFL
// minimum is taken over, so the candidate costs one sound speed, not a
// second recovery.  Block minima go to one slot by atomicMin on the bit
// pattern (every candidate is a non-negative double or +inf, which order
// like their bits).
// The last block to add its minimum (a ticket counter beside the slot)
// also finishes the reduction — dt = min(dt_max, slot), the dt log, the
// non-positive-dt flag — and re-arms slot and counter for the next step, so
// no separate finalize kernel runs (the threadFenceReduction pattern: no
// block waits for another).
struct FusedCfl {
    int on;
    int unsplit;
    double cfl;
    unsigned long long* slot;   // slot[0]: the minimum's bits; slot[1]: the block ticket counter
    double dt_max;
    double* dt;
    double* hist;
    int* err;
};

__device__ __forceinline__ void fused_cfl_reduce(double best, const FusedCfl& c)
{
    __shared__ double red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = dmin(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = dmin(m, red[w]);
        atomicMin(c.slot, (unsigned long long)__double_as_longlong(m));
        __threadfence();
        const unsigned long long ticket = atomicAdd(c.slot + 1, 1ull);
        if (ticket == (unsigned long long)gridDim.x - 1) {
            __threadfence();
            const double mm = __longlong_as_double((long long)atomicAdd(c.slot, 0ull));
            const double d = dmin(c.dt_max, mm);
            c.dt[0] = d;
            if (c.hist) c.hist[0] = d;
            if (!(d > 0.0) || !fin(d)) atomicOr(c.err, kErrDt);
            c.slot[0] = (unsigned long long)__double_as_longlong(HUGE_VAL);
            c.slot[1] = 0ull;
        }
    }
}

template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_A_MINB) staged_a(const double* __restrict__ in, __grid_constant__ const Grid g, __grid_constant__ const Mats M, LineSet ls,
                                                StagedBufs<NM, D> b, FusedCfl fc)
{
    pdl_enter();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double best = HUGE_VAL;
    if (t < (long long)ls.nl * ls.n) {
        const StagedItem<DIR> it(g, ls, t);
        State<NM, D> U;
        load_cell<NM, D>(in, g.ncell, it.cell, U);
        CellA<NM, D> A;
        stage_a<NM, D, true>(M, U, A);
        g_put<NM, D>(b.P, b.cap, t, A.P);
        if (!DIMGPU_STAGED_NO_PE) g_put<NM, D>(b.Pe, b.cap, t, A.Pe);
#pragma unroll
        for (int k = 0; k < NM; ++k) b.ck[k * b.cap + t] = A.ck[k];
        if (fc.on) best = cfl_candidate<NM, D, true>(M, U, A.P, g.dx, fc.cfl, fc.unsplit != 0, A.ck);
    }
    if (fc.on) fused_cfl_reduce(best, fc);
}

// Stage B in two kernels.  staged_bf: one thread per face state (2 per
// cell; the first half of the items are left faces, the second half right
// faces): reconstruct, build, repair, flux -> the LS / RS slots.  Each
// routine has one call site here, so all are inlined.
template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_FACE_MINB) staged_bf(__grid_constant__ const Grid g, __grid_constant__ const Mats M, LineSet ls,
                                                 StagedBufs<NM, D> b)
{
    pdl_enter();
    const long long N = (long long)ls.nl * ls.n;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * N) return;
    const bool right = t >= N;
    if (right) t -= N;
    const StagedItem<DIR> it(g, ls, t);
    const int n = ls.n;
    if (it.gi == 0 || it.gi == n - 1 || n < 3) return;  // end cells reconstruct nothing
    Prim<NM, D> lo, c, hi, Pl, Pr;
    get_pe<NM, D>(b, t - it.s, lo);
    get_pe<NM, D>(b, t, c);
    get_pe<NM, D>(b, t + it.s, hi);
    reconstruct_cell_faces<NM, D>(lo, c, hi, Pl, Pr);
    Flux<NM, D> F;
    face_flux<NM, D, true>(M, right ? Pr : Pl, DIR, F);
    g_put<NM, D>(right ? b.RS : b.LS, b.cap, t, F);
}

// staged_bu: one thread per cell, the half-step update from the two face
// fluxes (the face primitives are reconstructed again: the same values).
template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_BU_MINB) staged_bu(const double* __restrict__ in, __grid_constant__ const Grid g, __grid_constant__ const Mats M, LineSet ls,
                                                 StagedBufs<NM, D> b, const double* __restrict__ dtp)
{
    pdl_enter();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ls.nl * ls.n) return;
    const StagedItem<DIR> it(g, ls, t);
    const int n = ls.n;
    const bool end = it.gi == 0 || it.gi == n - 1 || n < 3;
    CellA<NM, D> A;
    get_pe<NM, D>(b, t, A.Pe);
    Prim<NM, D> Ph;
    if (end) {
        Ph = A.Pe;
    }
    else {
        State<NM, D> U;
        load_cell<NM, D>(in, g.ncell, it.cell, U);
#pragma unroll
        for (int k = 0; k < NM; ++k) A.ck[k] = b.ck[k * b.cap + t];
        Prim<NM, D> lo, hi, Pl, Pr;
        get_pe<NM, D>(b, t - it.s, lo);
        get_pe<NM, D>(b, t + it.s, hi);
        reconstruct_cell_faces<NM, D>(lo, A.Pe, hi, Pl, Pr);
        Flux<NM, D> FL, FR;
        g_get<NM, D>(b.LS, b.cap, t, FL);
        g_get<NM, D>(b.RS, b.cap, t, FR);
        State<NM, D> Uh;
        stage_b_update<NM, D, true>(M, U, A, Pl, Pr, FL, FR, DIR, *dtp, g.dx[DIR], Uh, Ph);
    }
    g_put<NM, D>(b.Ph, b.cap, t, Ph);
}

// Stage C: one thread per face state (left faces first, then right faces),
// all routines inlined.  End cells keep U and its primitive on both sides.
template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_FACE_MINB) staged_c(const double* __restrict__ in, __grid_constant__ const Grid g, __grid_constant__ const Mats M, LineSet ls,
                                                StagedBufs<NM, D> b)
{
    pdl_enter();
    const long long N = (long long)ls.nl * ls.n;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * N) return;
    const bool right = t >= N;
    if (right) t -= N;
    const StagedItem<DIR> it(g, ls, t);
    const int n = ls.n;
    const bool end = it.gi == 0 || it.gi == n - 1 || n < 3;
    State<NM, D> S;
    Prim<NM, D> P;
    if (end) {
        load_cell<NM, D>(in, g.ncell, it.cell, S);
        g_get<NM, D>(b.P, b.cap, t, P);
    }
    else {
        Prim<NM, D> Ph, lo, hi, Lh, Rh;
        g_get<NM, D>(b.Ph, b.cap, t, Ph);
        g_get<NM, D>(b.Ph, b.cap, t - it.s, lo);
        g_get<NM, D>(b.Ph, b.cap, t + it.s, hi);
        reconstruct_cell_faces<NM, D>(lo, Ph, hi, Lh, Rh);
        face_state<NM, D, true>(M, right ? Rh : Lh, S, P);
    }
    g_put<NM, D>(right ? b.RS : b.LS, b.cap, t, S);
    g_put<NM, D>(right ? b.PRS : b.PLS, b.cap, t, P);
}

template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_D_MINB) staged_d(__grid_constant__ const Grid g, __grid_constant__ const Mats M, LineSet ls, StagedBufs<NM, D> b,
                                                int* __restrict__ err)
{
    pdl_enter();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ls.nl * ls.n) return;
    const StagedItem<DIR> it(g, ls, t);
    if (it.gi >= ls.n - 1) return;  // face i|i+1 exists for i <= n-2
    State<NM, D> UL, UR;
    Prim<NM, D> PL, PR;
    g_get<NM, D>(b.RS, b.cap, t, UL);
    g_get<NM, D>(b.PRS, b.cap, t, PL);
    g_get<NM, D>(b.LS, b.cap, t + it.s, UR);
    g_get<NM, D>(b.PLS, b.cap, t + it.s, PR);
    FaceD<NM, D> f;
    if (!stage_d<NM, D, DIMGPU_STAGED_INLINE_DE>(M, UL, PL, UR, PR, DIR, f)) atomicOr(err, kErrNonFinite);
    g_put<NM, D>(b.F, b.cap, t, f);
}

template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_E_MINB) staged_e(const double* __restrict__ in, double* __restrict__ out, __grid_constant__ const Grid g,
                                                __grid_constant__ const Mats M, LineSet ls, StagedBufs<NM, D> b,
                                                const double* __restrict__ dtp)
{
    pdl_enter();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ls.nl * ls.n) return;
    const StagedItem<DIR> it(g, ls, t);
    const int n = ls.n;
    const bool first = it.gi == 0, last = it.gi == n - 1;
    State<NM, D> U;
    load_cell<NM, D>(in, g.ncell, it.cell, U);
    CellA<NM, D> A;
    g_get<NM, D>(b.P, b.cap, t, A.P);
#pragma unroll
    for (int k = 0; k < NM; ++k) A.ck[k] = b.ck[k * b.cap + t];
    FaceD<NM, D> lo, hi;
    if (!first) g_get<NM, D>(b.F, b.cap, t - it.s, lo);
    if (!last) g_get<NM, D>(b.F, b.cap, t, hi);
    State<NM, D> Un;
    stage_e<NM, D, DIMGPU_STAGED_INLINE_DE>(M, U, A, first ? nullptr : &lo, last ? nullptr : &hi, first, last, *dtp,
                                             g.dx[DIR], Un);
    store_cell<NM, D>(out, g.ncell, it.cell, Un);
}

// Stages D and E in one kernel.  A block owns a tile of TW lines x TH
// positions along them: every position gi >= 1 forms the face gi-1|gi
// (stage D of item gi-1) into shared memory, then the tile's first TH - 1
// positions update their cells from the faces on either side (stage E).
// Consecutive tiles along a line overlap by one position, so a face is
// formed twice only at tile seams (1 face in TH - 1).  The face records
// never reach HBM.  The x sweep puts the positions on the fast thread index
// (neighbouring items t and t+1), the other axes put the lines there.
template<int DIR>
struct DeTile {
    static constexpr int TW = DIR == 0 ? 8 : 16;   // lines per tile
    static constexpr int TH = DIR == 0 ? 32 : 16;  // positions per tile (TH - 1 cells updated)
};

template<int NM, int D, int DIR>
__host__ __device__ inline long long de_tiles_per_line(int n)
{
    return (n + DeTile<DIR>::TH - 2) / (DeTile<DIR>::TH - 1);
}

template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_DE_MINB) staged_de(const double* __restrict__ in, double* __restrict__ out,
                                                 __grid_constant__ const Grid g, __grid_constant__ const Mats M, LineSet ls,
                                                 StagedBufs<NM, D> b, const double* __restrict__ dtp,
                                                 int* __restrict__ err)
{
    constexpr int TW = DeTile<DIR>::TW, TH = DeTile<DIR>::TH, KF = kFaceVars(NM, D);
    static_assert(TW * TH == 256, "one thread per tile position");
    __shared__ double sf[KF][256];
    pdl_enter();
    const int tx = threadIdx.x;
    const int lo_ = DIR == 0 ? tx / TH : tx % TW;  // line within the tile
    const int po = DIR == 0 ? tx % TH : tx / TW;   // position within the tile
    const long long tpl = de_tiles_per_line<NM, D, DIR>(ls.n);
    const long long lrel = (long long)(blockIdx.x / tpl) * TW + lo_;
    const int gi = (int)(blockIdx.x % tpl) * (TH - 1) + po;
    const int n = ls.n;
    const bool live = lrel < ls.nl && gi < n;
    const long long t = DIR == 0 ? lrel * n + gi : (long long)gi * ls.nl + lrel;

    // Stage D: the face to the left of position gi (item gi-1's face).
    if (live && gi >= 1) {
        const long long s = DIR == 0 ? 1 : ls.nl;
        State<NM, D> UL, UR;
        Prim<NM, D> PL, PR;
        g_get<NM, D>(b.RS, b.cap, t - s, UL);
        g_get<NM, D>(b.PRS, b.cap, t - s, PL);
        g_get<NM, D>(b.LS, b.cap, t, UR);
        g_get<NM, D>(b.PLS, b.cap, t, PR);
        FaceD<NM, D> f;
        if (!stage_d<NM, D, DIMGPU_STAGED_INLINE_DE>(M, UL, PL, UR, PR, DIR, f)) atomicOr(err, kErrNonFinite);
        int v = 0;
#pragma unroll
        for (int k = 0; k < NM; ++k) sf[v++][tx] = f.F.m[k];
#pragma unroll
        for (int d = 0; d < D; ++d) sf[v++][tx] = f.F.mom[d];
        sf[v++][tx] = f.F.E;
        sf[v++][tx] = f.fv;
#pragma unroll
        for (int k = 0; k < NM; ++k) sf[v++][tx] = f.af[k];
    }
    __syncthreads();

    // Stage E on the tile's first TH - 1 positions.
    if (!live || po == TH - 1) return;
    const StagedItem<DIR> it(g, ls, t);
    const bool first = gi == 0, last = gi == n - 1;
    State<NM, D> U;
    load_cell<NM, D>(in, g.ncell, it.cell, U);
    CellA<NM, D> A;
    g_get<NM, D>(b.P, b.cap, t, A.P);
#pragma unroll
    for (int k = 0; k < NM; ++k) A.ck[k] = b.ck[k * b.cap + t];
    FaceD<NM, D> fl, fh;
    const int th = tx + (DIR == 0 ? 1 : TW);  // the next position's thread
    if (!first) {
        int v = 0;
#pragma unroll
        for (int k = 0; k < NM; ++k) fl.F.m[k] = sf[v++][tx];
#pragma unroll
        for (int d = 0; d < D; ++d) fl.F.mom[d] = sf[v++][tx];
        fl.F.E = sf[v++][tx];
        fl.fv = sf[v++][tx];
#pragma unroll
        for (int k = 0; k < NM; ++k) fl.af[k] = sf[v++][tx];
    }
    if (!last) {
        int v = 0;
#pragma unroll
        for (int k = 0; k < NM; ++k) fh.F.m[k] = sf[v++][th];
#pragma unroll
        for (int d = 0; d < D; ++d) fh.F.mom[d] = sf[v++][th];
        fh.F.E = sf[v++][th];
        fh.fv = sf[v++][th];
#pragma unroll
        for (int k = 0; k < NM; ++k) fh.af[k] = sf[v++][th];
    }
    State<NM, D> Un;
    stage_e<NM, D, DIMGPU_STAGED_INLINE_DE>(M, U, A, first ? nullptr : &fl, last ? nullptr : &fh, first, last, *dtp,
                                             g.dx[DIR], Un);
    store_cell<NM, D>(out, g.ncell, it.cell, Un);
}

// ---- the mixed-precision staged sweep (precision MIXED) ---------------------------
//
// Stage A is mixed_a (staged_a with the closed-form FP64 recovery), stage E
// is staged_e (FP64 cell update).  mixed_b is stage B with FP32-limited slopes and no face-state
// round trip; mixed_cd builds the two face states of face i|i+1 from the
// half-step primitives of cells i-1..i+2 and runs the FP32-increment HLLC,
// so the face states never reach HBM.  Scratch: P, ck, Pe, Ph and the face
// records, at the staged positions.
template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_MIXED_A_MINB) mixed_a(const double* __restrict__ in, __grid_constant__ const Grid g, __grid_constant__ const Mats M, LineSet ls,
                                               StagedBufs<NM, D> b, FusedCfl fc)
{
    pdl_enter();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double best = HUGE_VAL;
    if (t < (long long)ls.nl * ls.n) {
        const StagedItem<DIR> it(g, ls, t);
        State<NM, D> U;
        load_cell<NM, D>(in, g.ncell, it.cell, U);
        CellA<NM, D> A;
        stage_a_mixed<NM, D, DIMGPU_MIXED_INLINE>(M, U, A);
        g_put<NM, D>(b.P, b.cap, t, A.P);
        if (!DIMGPU_STAGED_NO_PE) g_put<NM, D>(b.Pe, b.cap, t, A.Pe);
#pragma unroll
        for (int k = 0; k < NM; ++k) b.ck[k * b.cap + t] = A.ck[k];
        if (fc.on) best = cfl_candidate<NM, D, DIMGPU_MIXED_INLINE>(M, U, A.P, g.dx, fc.cfl, fc.unsplit != 0, A.ck);
    }
    if (fc.on) fused_cfl_reduce(best, fc);
}

// mixed_b and mixed_cd run DIMGPU_MIXED_BCD_MINB blocks of 256 threads per
// SM (dim_launch.h) rather than the 2 that their ~100 registers allow: the
// FP64 chains are latency-bound, and the extra warps hide more of them than
// the few spills to L1 cost.
template<int NM, int D, int DIR, typename R = float>
__global__ void __launch_bounds__(256, DIMGPU_MIXED_BCD_MINB) mixed_b(const double* __restrict__ in, __grid_constant__ const Grid g, __grid_constant__ const Mats M, LineSet ls,
                                                  StagedBufs<NM, D> b, const double* __restrict__ dtp)
{
    pdl_enter();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ls.nl * ls.n) return;
    const StagedItem<DIR> it(g, ls, t);
    const int n = ls.n;
    const bool end = it.gi == 0 || it.gi == n - 1 || n < 3;
    CellA<NM, D> A;
    get_pe<NM, D>(b, t, A.Pe);
    Prim<NM, D> Ph;
    if (end) {
        Ph = A.Pe;
    }
    else {
        State<NM, D> U;
        load_cell<NM, D>(in, g.ncell, it.cell, U);
#pragma unroll
        for (int k = 0; k < NM; ++k) A.ck[k] = b.ck[k * b.cap + t];
        Prim<NM, D> lo, hi;
        get_pe<NM, D>(b, t - it.s, lo);
        get_pe<NM, D>(b, t + it.s, hi);
        stage_b_mixed<NM, D, R, DIMGPU_MIXED_INLINE>(M, U, A, lo, hi, false, DIR, *dtp, g.dx[DIR], Ph);
    }
    g_put<NM, D>(b.Ph, b.cap, t, Ph);
}

// Face state of cell item t on the given side (end cells: U and P).
template<int NM, int D, int DIR, typename R = float, bool FD = DIMGPU_STAGED_FASTDIV>
__device__ __forceinline__ void mixed_face(const double* __restrict__ in, const Grid& g, const Mats& M,
                                           const StagedBufs<NM, D>& b, const StagedItem<DIR, FD>& it, long long t, int n,
                                           bool right, State<NM, D>& Uf, Prim<NM, D>& Pf)
{
    const bool end = it.gi == 0 || it.gi == n - 1 || n < 3;
    if (end) {
        load_cell<NM, D>(in, g.ncell, it.cell, Uf);
        g_get<NM, D>(b.P, b.cap, t, Pf);
        return;
    }
    Prim<NM, D> lo, c, hi;
    g_get<NM, D>(b.Ph, b.cap, t - it.s, lo);
    g_get<NM, D>(b.Ph, b.cap, t, c);
    g_get<NM, D>(b.Ph, b.cap, t + it.s, hi);
    face_mixed<NM, D, R, DIMGPU_MIXED_INLINE>(M, lo, c, hi, right, Uf, Pf);
}

template<int NM, int D, int DIR, typename R = float>
__global__ void __launch_bounds__(256, DIMGPU_MIXED_BCD_MINB) mixed_cd(const double* __restrict__ in, __grid_constant__ const Grid g, __grid_constant__ const Mats M, LineSet ls,
                                                   StagedBufs<NM, D> b, int* __restrict__ err)
{
    pdl_enter();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ls.nl * ls.n) return;
    const StagedItem<DIR> it(g, ls, t);
    const int n = ls.n;
    if (it.gi >= n - 1) return;  // face i|i+1 exists for i <= n-2
    State<NM, D> UL, UR;
    Prim<NM, D> PL, PR;
    mixed_face<NM, D, DIR, R>(in, g, M, b, it, t, n, true, UL, PL);
    StagedItem<DIR> nx = it;
    nx.gi += 1;
    nx.cell += g.stride[DIR];
    mixed_face<NM, D, DIR, R>(in, g, M, b, nx, t + it.s, n, false, UR, PR);
    FaceD<NM, D> f;
    if (!stage_d_mixed<NM, D, R, DIMGPU_MIXED_INLINE>(M, UL, PL, UR, PR, DIR, f)) atomicOr(err, kErrNonFinite);
    g_put<NM, D>(b.F, b.cap, t, f);
}

// Stages C and D of the FP64 step fused, one thread per face i|i+1: the
// right face state of cell i and the left one of cell i+1 are built (stage
// C's reconstruction, build, repair, recovery, as face_state) and go
// straight into HLLC, so the four face-state records never reach HBM.  Each
// face state belongs to exactly one face, so nothing is computed twice.  The
// two face states run through one inlined copy of the routines (a loop of
// two, not unrolled); the first is parked in a small local array.
template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_STAGED_MINB) staged_cd(const double* __restrict__ in, __grid_constant__ const Grid g, __grid_constant__ const Mats M, LineSet ls,
                                                 StagedBufs<NM, D> b, int* __restrict__ err)
{
    pdl_enter();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ls.nl * ls.n) return;
    const StagedItem<DIR> it(g, ls, t);
    const int n = ls.n;
    if (it.gi >= n - 1) return;  // face i|i+1 exists for i <= n-2
    State<NM, D> S[2];
    Prim<NM, D> P[2];
#pragma unroll 1
    for (int side = 0; side < 2; ++side) {
        // side 0: cell i, its right face; side 1: cell i+1, its left face
        const long long tc = t + side * it.s;
        const int gi = it.gi + side;
        if (gi == 0 || gi == n - 1 || n < 3) {
            load_cell<NM, D>(in, g.ncell, it.cell + side * g.stride[DIR], S[side]);
            g_get<NM, D>(b.P, b.cap, tc, P[side]);
            continue;
        }
        Prim<NM, D> lo, c, hi, Lh, Rh;
        g_get<NM, D>(b.Ph, b.cap, tc - it.s, lo);
        g_get<NM, D>(b.Ph, b.cap, tc, c);
        g_get<NM, D>(b.Ph, b.cap, tc + it.s, hi);
        reconstruct_cell_faces<NM, D>(lo, c, hi, Lh, Rh);
        face_state<NM, D, true>(M, side == 0 ? Rh : Lh, S[side], P[side]);
    }
    FaceD<NM, D> f;
    if (!stage_d<NM, D, DIMGPU_STAGED_INLINE_DE>(M, S[0], P[0], S[1], P[1], DIR, f)) atomicOr(err, kErrNonFinite);
    g_put<NM, D>(b.F, b.cap, t, f);
}


// ---- CFL ------------------------------------------------------------------------
__device__ __forceinline__ double warp_min(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template<int NM, int D>
__global__ void __launch_bounds__(256) cfl_kernel(const double* __restrict__ st, __grid_constant__ const Grid g, __grid_constant__ const Mats M, double cfl,
                                                  int unsplit, int mixed, double* __restrict__ blockmin,
                                                  long long begin, long long end)
{
    __shared__ double red[32];
    double best = HUGE_VAL;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = begin + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < end; i += stride) {
        State<NM, D> U;
        Prim<NM, D> P;
        load_cell<NM, D>(st, g.ncell, i, U);
        if (mixed) cons_to_prim_mixed<NM, D>(M, U, P);  // the mixed step's own recovery
        else cons_to_prim<NM, D>(M, U, P);
        best = dmin(best, cfl_candidate<NM, D>(M, U, P, g.dx, cfl, unsplit != 0));
    }
    best = warp_min(best);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x < 32) {
        const int nw = blockDim.x >> 5;
        double v = threadIdx.x < nw ? red[threadIdx.x] : HUGE_VAL;
        v = warp_min(v);
        if (threadIdx.x == 0) blockmin[blockIdx.x] = v;
    }
}

// ---- boundary fill (dim::apply_boundary_conditions, src/dim/solver/advance/
// boundary.hpp:165-226) ----------------------------------------------------------
//
// Every boundary cell copies its source cell (each boundary axis shifted one
// cell inward), flipping the normal momentum on reflective sides; cells named
// nonreflective by boundary_name_for_cell (:23-41) take
// local_nonreflective_state (:113-163).  For axes with N >= 4 (N >= 3 without
// nonreflective sides) every cell read is an interior cell, so the
// reference's serial in-place loop is order-independent and one thread per
// boundary cell reproduces it; otherwise the host runs the serial variant.
template<int NM, int D>
__device__ void bc_cell(const Grid& g, const Mats& M, double* st, const int* idx, long long linear)
{
    int src[3] = {0, 0, 0};
    bool is_boundary = false;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        src[a] = idx[a];
        if (g.N[a] <= 1) continue;
        if (idx[a] == 0) { src[a] = 1; is_boundary = true; }
        else if (idx[a] == g.N[a] - 1) { src[a] = g.N[a] - 2; is_boundary = true; }
    }
    if (!is_boundary) return;
    int bc = DIMGPU_BC_TRANSMISSIVE;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        if (idx[a] == 0) { bc = g.bc_lo[a]; break; }
        if (idx[a] == g.N[a] - 1) { bc = g.bc_hi[a]; break; }
    }
    long long src_lin = 0;
#pragma unroll
    for (int a = 0; a < D; ++a) src_lin += (long long)src[a] * g.stride[a];
    State<NM, D> U;
    int q;
    if (bc == DIMGPU_BC_NONREFLECTIVE) {
        int second[3] = {src[0], src[1], src[2]};
#pragma unroll
        for (int a = 0; a < D; ++a) {
            if (idx[a] == 0 && g.N[a] > 2) second[a] = 2;
            else if (idx[a] == g.N[a] - 1 && g.N[a] > 2) second[a] = g.N[a] - 3;
        }
        long long sec_lin = 0;
#pragma unroll
        for (int a = 0; a < D; ++a) sec_lin += (long long)second[a] * g.stride[a];
        State<NM, D> first, sec, ex;
        // plain loads: the serial variant reads cells this launch rewrites
        q = 0;
#pragma unroll
        for (int k = 0; k < NM; ++k) { first.m[k] = st[q * g.ncell + src_lin]; sec.m[k] = st[q * g.ncell + sec_lin]; ++q; }
#pragma unroll
        for (int d = 0; d < D; ++d) { first.mom[d] = st[q * g.ncell + src_lin]; sec.mom[d] = st[q * g.ncell + sec_lin]; ++q; }
        first.E = st[q * g.ncell + src_lin]; sec.E = st[q * g.ncell + sec_lin]; ++q;
#pragma unroll
        for (int k = 0; k < NM - 1; ++k) { first.a[k] = st[q * g.ncell + src_lin]; sec.a[k] = st[q * g.ncell + sec_lin]; ++q; }
        U = first;
#pragma unroll
        for (int k = 0; k < NM; ++k) ex.m[k] = first.m[k] + (first.m[k] - sec.m[k]);
#pragma unroll
        for (int d = 0; d < D; ++d) ex.mom[d] = first.mom[d] + (first.mom[d] - sec.mom[d]);
        ex.E = first.E + (first.E - sec.E);
        int axis = 0;
#pragma unroll
        for (int a = D - 1; a >= 0; --a)
            if (idx[a] == 0 || idx[a] == g.N[a] - 1) axis = a;
        const int outward = (idx[axis] == 0) ? -1 : 1;
        const double ex_rho = dmax(total_density<NM, D>(ex), 1e-12);
        double ex_mom_axis = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d)
            if (d == axis) ex_mom_axis = ex.mom[d];
        const double ex_un = outward * safe_div(ex_mom_axis, ex_rho);
        if (ex_un > 0.0) {
            const double rho = dmax(total_density<NM, D>(U), 1e-12);
            double b = 0.0, af = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) b += U.mom[d] * U.mom[d];
#pragma unroll
            for (int d = 0; d < D; ++d)
                if (d == axis) U.mom[d] = ex.mom[d];
#pragma unroll
            for (int d = 0; d < D; ++d) af += U.mom[d] * U.mom[d];
            U.E += 0.5 * (af - b) / rho;
        }
        repair_state<NM, D>(M, U);
    }
    else {
        q = 0;
#pragma unroll
        for (int k = 0; k < NM; ++k) U.m[k] = st[(q++) * g.ncell + src_lin];
#pragma unroll
        for (int d = 0; d < D; ++d) U.mom[d] = st[(q++) * g.ncell + src_lin];
        U.E = st[(q++) * g.ncell + src_lin];
#pragma unroll
        for (int k = 0; k < NM - 1; ++k) U.a[k] = st[(q++) * g.ncell + src_lin];
#pragma unroll
        for (int a = 0; a < D; ++a) {
            if ((idx[a] == 0 && g.bc_lo[a] == DIMGPU_BC_REFLECTIVE) ||
                (idx[a] == g.N[a] - 1 && g.bc_hi[a] == DIMGPU_BC_REFLECTIVE))
                U.mom[a] *= -1.0;
        }
    }
    q = 0;
#pragma unroll
    for (int k = 0; k < NM; ++k) st[(q++) * g.ncell + linear] = U.m[k];
#pragma unroll
    for (int d = 0; d < D; ++d) st[(q++) * g.ncell + linear] = U.mom[d];
    st[(q++) * g.ncell + linear] = U.E;
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) st[(q++) * g.ncell + linear] = U.a[k];
}

// The boundary shell as planes: plane 2a+side holds the cells with
// idx[a] == (side ? N[a]-1 : 0) whose lower axes b < a are interior, so
// every boundary cell is visited exactly once.
template<int NM, int D>
__global__ void __launch_bounds__(256) bc_kernel(double* st, __grid_constant__ const Grid g, __grid_constant__ const Mats M, long long plane0, long long plane1,
                                                 long long plane2)
{
    pdl_enter();
    const long long count[3] = {plane0, plane1, plane2};
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int a = 0;
    while (a < D && i >= 2 * count[a]) { i -= 2 * count[a]; ++a; }
    if (a >= D) return;
    const int side = (int)(i / count[a]);
    long long r = i % count[a];
    int idx[3] = {0, 0, 0};
#pragma unroll
    for (int b = 0; b < D; ++b) {
        if (b == a) continue;
        // lower axes: interior cells only (an axis with N == 1 has no boundary)
        const bool inner = b < a && g.N[b] != 1;
        const int ext = inner ? (g.N[b] - 2) : g.N[b];
        idx[b] = (int)(r % ext) + (inner ? 1 : 0);
        r /= ext;
    }
    idx[a] = side ? g.N[a] - 1 : 0;
    long long linear = 0;
#pragma unroll
    for (int b = 0; b < D; ++b) linear += (long long)idx[b] * g.stride[b];
    bc_cell<NM, D>(g, M, st, idx, linear);
}

// The reference's literal serial order, for grids where it matters.
template<int NM, int D>
__global__ void bc_serial_kernel(double* st, __grid_constant__ const Grid g, __grid_constant__ const Mats M)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (long long linear = 0; linear < g.ncell; ++linear) {
        int idx[3] = {0, 0, 0};
        long long s = 1;
#pragma unroll
        for (int a = 0; a < D; ++a) {
            idx[a] = (int)((linear / s) % g.N[a]);
            s *= g.N[a];
        }
        bc_cell<NM, D>(g, M, st, idx, linear);
    }
}

// ---- unsplit accumulation (src/dim/solver/advance_step.hpp:77-101) -------------
template<int NM, int D>
__global__ void __launch_bounds__(256) accumulate_kernel(double* __restrict__ acc, const double* __restrict__ dir_state,
                                                         const double* __restrict__ base, __grid_constant__ const Grid g, __grid_constant__ const Mats M)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.ncell) return;
    State<NM, D> a, d, b;
    load_cell<NM, D>(acc, g.ncell, i, a);
    load_cell<NM, D>(dir_state, g.ncell, i, d);
    load_cell<NM, D>(base, g.ncell, i, b);
#pragma unroll
    for (int k = 0; k < NM; ++k) a.m[k] += d.m[k] - b.m[k];
#pragma unroll
    for (int q = 0; q < D; ++q) a.mom[q] += d.mom[q] - b.mom[q];
    a.E += d.E - b.E;
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) a.a[k] += d.a[k] - b.a[k];
    repair_state<NM, D>(M, a);
    store_cell<NM, D>(acc, g.ncell, i, a);
}

// ---- conservation totals (compute_dim_conservation_totals,
// src/app/io/conservation_report.hpp:188-218): per-block partial sums ------------
template<int NM, int D>
__global__ void __launch_bounds__(256) totals_kernel(const double* __restrict__ st, __grid_constant__ const Grid g, double volume,
                                                     double* __restrict__ partial)
{
    constexpr int NV = NM + 1 + D + 1;
    __shared__ double red[NV][256];
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.ncell; i += stride) {
        double cell_mass = 0.0;
#pragma unroll
        for (int k = 0; k < NM; ++k) {
            const double part = st[k * g.ncell + i] * volume;
            acc[k] += part;
            cell_mass += part;
        }
        acc[NM] += cell_mass;
#pragma unroll
        for (int d = 0; d < D; ++d) acc[NM + 1 + d] += st[(NM + d) * g.ncell + i] * volume;
        acc[NM + 1 + D] += st[(NM + D) * g.ncell + i] * volume;
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) red[v][threadIdx.x] = acc[v];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
#pragma unroll
            for (int v = 0; v < NV; ++v) red[v][threadIdx.x] += red[v][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) partial[(long long)blockIdx.x * NV + v] = red[v][0];
    }
}

// ---- launchers ---------------------------------------------------------------------
// The tensor map of a fused sweep's input tiles (see sweep_kernel), or false
// where the layout does not allow one: every global stride and the box's
// innermost extent must be multiples of 16 bytes (even N[0], even cell
// count, even W for the y / z sweeps) and every box extent at most 256.
inline bool make_tile_map(const Grid& g, int dir, int V, const double* base, int T, int W, CUtensorMap* out)
{
    using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static EncodeFn encode = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<EncodeFn>(fn);
    }
    if (!encode) return false;
    const long long nx = g.N[0], ny = g.N[1], nz = g.N[2];
    if ((nx & 1) || (g.ncell & 1) || V > 256 || W > 256) return false;
    if (dir == 0 && T + 2 > 256) return false;
    if (dir != 0 && ((W & 1) || T > 256)) return false;
    cuuint64_t dims[4], strides[3];
    cuuint32_t box[4], estr[4] = {1, 1, 1, 1};
    cuuint32_t rank;
    if (dir == 0) {
        rank = 3;
        dims[0] = (cuuint64_t)nx;
        dims[1] = (cuuint64_t)(g.ncell / nx);
        dims[2] = (cuuint64_t)V;
        strides[0] = (cuuint64_t)nx * 8;
        strides[1] = (cuuint64_t)g.ncell * 8;
        box[0] = (cuuint32_t)(T + 2);
        box[1] = (cuuint32_t)W;
        box[2] = (cuuint32_t)V;
    }
    else {
        rank = 4;
        dims[0] = (cuuint64_t)nx;
        dims[1] = (cuuint64_t)ny;
        dims[2] = (cuuint64_t)nz;
        dims[3] = (cuuint64_t)V;
        strides[0] = (cuuint64_t)nx * 8;
        strides[1] = (cuuint64_t)(nx * ny) * 8;
        strides[2] = (cuuint64_t)g.ncell * 8;
        box[0] = (cuuint32_t)W;
        box[1] = (cuuint32_t)(dir == 1 ? T : 1);
        box[2] = (cuuint32_t)(dir == 2 ? T : 1);
        box[3] = (cuuint32_t)V;
    }
    const CUresult r = encode(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, rank, const_cast<double*>(base), dims, strides,
                              box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template<int NM, int D, int DIR>
cudaError_t launch_sweep_dir(const Grid& g, const Mats& M, Tile tile, const double* in, double* out,
                             const double* dt, int* err, cudaStream_t s)
{
    const int n = g.N[DIR];
    const int T = tile.T, W = tile.W;
    const int ntile = (n + (T - 6) - 1) / (T - 6);
    long long nblocks;
    int ngx = 1;
    if (DIR == 0) {
        const long long nlines = g.ncell / g.N[0];
        nblocks = (long long)ntile * ((nlines + W - 1) / W);
    }
    else {
        ngx = (g.N[0] + W - 1) / W;
        const long long other = g.ncell / ((long long)g.N[0] * g.N[DIR]);
        nblocks = (long long)ngx * ntile * other;
    }
    TileMap tm;
    std::memset(&tm, 0, sizeof tm);
    const int V = kStateVarsT(NM, D);
    const int tma = make_tile_map(g, DIR, V, in, T, W, &tm.map) ? 1 : 0;
    const size_t tile_doubles = tma ? ((size_t)(DIR == 0 ? (T + 2) : T) * W * V + 15) / 16 * 16 : 0;
    const size_t smem = sizeof(double) * ((size_t)kSweepSmemVars(NM, D) * (size_t)(T * W) + tile_doubles);
    auto kern = sweep_kernel<NM, D, DIR>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)nblocks, T * W, smem, s>>>(in, out, g, M, T, W, ntile, ngx, dt, err, tm, tma);
    count_launches(1);
    return cudaGetLastError();
}

template<int NM, int D>
cudaError_t launch_sweep(const Grid& g, const Mats& M, int dir, Tile tile, const double* in, double* out,
                         const double* dt, int* err, cudaStream_t s)
{
    if (tile.T < 8 || tile.W < 1 || tile.T * tile.W > 256) return cudaErrorInvalidValue;
    if (dir == 0) return launch_sweep_dir<NM, D, 0>(g, M, tile, in, out, dt, err, s);
    if constexpr (D >= 2) {
        if (dir == 1) return launch_sweep_dir<NM, D, 1>(g, M, tile, in, out, dt, err, s);
    }
    if constexpr (D >= 3) {
        if (dir == 2) return launch_sweep_dir<NM, D, 2>(g, M, tile, in, out, dt, err, s);
    }
    return cudaErrorInvalidValue;
}

// Staged schedule: chunks of whole lines, at most `cap` cells each; scratch
// holds kStagedVars(NM, D) * cap doubles.
template<int NM, int D, int DIR>
cudaError_t launch_staged_dir(const Grid& g, const Mats& M, const double* in, double* out, const double* dt, int* err,
                              double* scratch, long long cap, const FusedStep& fs, cudaStream_t s)
{
    const int n = g.N[DIR];
    const long long nlines = g.ncell / n;
    long long per = cap / n;
    if (per < 1 || nlines > 0xFFFFFFFFLL || 2 * cap > 0xFFFFFFFFLL) return cudaErrorInvalidValue;
    StagedBufs<NM, D> b;
    b.cap = cap;
    double* p = scratch;
    b.P = p; p += kPrimVars(NM, D) * cap;
    b.ck = p; p += NM * cap;
    b.Pe = p; p += kPrimVars(NM, D) * cap;
    b.Ph = p; p += kPrimVars(NM, D) * cap;
    b.LS = p; p += kStateVars(NM, D) * cap;
    b.RS = p; p += kStateVars(NM, D) * cap;
    b.PLS = p; p += kPrimVars(NM, D) * cap;
    b.PRS = p; p += kPrimVars(NM, D) * cap;
    b.F = p;
    for (long long L0 = 0; L0 < nlines; L0 += per) {
        LineSet ls;
        ls.L0 = L0;
        ls.nl = (int)((nlines - L0 < per) ? (nlines - L0) : per);
        ls.n = n;
        ls.set_dividers(g.N[0]);
        const long long items = (long long)ls.nl * n;
        const unsigned blocks = (unsigned)((items + 255) / 256);
        FusedCfl fc{0, 0, 0.0, nullptr, 0.0, nullptr, nullptr, nullptr};
        if (fs.on) fc = FusedCfl{1, fs.unsplit, fs.cfl, fs.slot, fs.dt_max, fs.dt, fs.hist, fs.err};
        launch_stage(staged_a<NM, D, DIR>, blocks, s, in, g, M, ls, b, fc);
        count_launches(1);
        const unsigned blocks2 = (unsigned)((2 * items + 255) / 256);
        launch_stage(staged_bf<NM, D, DIR>, blocks2, s, g, M, ls, b);
        count_launches(1);
        launch_stage(staged_bu<NM, D, DIR>, blocks, s, in, g, M, ls, b, dt);
        count_launches(1);
        constexpr bool fuse_de = DIMGPU_STAGED_FUSE_DE && D >= 2 && !DIMGPU_STAGED_FUSE_CD;
        if (DIMGPU_STAGED_FUSE_CD) {
            launch_stage(staged_cd<NM, D, DIR>, blocks, s, in, g, M, ls, b, err);
            count_launches(1);
        }
        else {
            launch_stage(staged_c<NM, D, DIR>, blocks2, s, in, g, M, ls, b);
            count_launches(1);
            if constexpr (!fuse_de) {
                launch_stage(staged_d<NM, D, DIR>, blocks, s, g, M, ls, b, err);
                count_launches(1);
            }
        }
        if constexpr (fuse_de) {
            const long long tiles =
                ((ls.nl + DeTile<DIR>::TW - 1) / DeTile<DIR>::TW) * de_tiles_per_line<NM, D, DIR>(n);
            launch_stage(staged_de<NM, D, DIR>, (unsigned)tiles, s, in, out, g, M, ls, b, dt, err);
        }
        else {
            launch_stage(staged_e<NM, D, DIR>, blocks, s, in, out, g, M, ls, b, dt);
        }
        count_launches(1);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template<int NM, int D>
cudaError_t launch_sweep_staged(const Grid& g, const Mats& M, int dir, const double* in, double* out,
                                const double* dt, int* err, double* scratch, long long cap, const FusedStep& fs,
                                cudaStream_t s)
{
    if (fs.on && (long long)g.ncell > cap) return cudaErrorInvalidValue;  // fusion needs a single chunk
    if (dir == 0) return launch_staged_dir<NM, D, 0>(g, M, in, out, dt, err, scratch, cap, fs, s);
    if constexpr (D >= 2) {
        if (dir == 1) return launch_staged_dir<NM, D, 1>(g, M, in, out, dt, err, scratch, cap, fs, s);
    }
    if constexpr (D >= 3) {
        if (dir == 2) return launch_staged_dir<NM, D, 2>(g, M, in, out, dt, err, scratch, cap, fs, s);
    }
    return cudaErrorInvalidValue;
}

template<int NM, int D, int DIR>
cudaError_t launch_mixed_dir(const Grid& g, const Mats& M, const double* in, double* out, const double* dt, int* err,
                             double* scratch, long long cap, const FusedStep& fs, cudaStream_t s, bool twin)
{
    const int n = g.N[DIR];
    const long long nlines = g.ncell / n;
    const long long per = cap / n;
    if (per < 1 || nlines > 0xFFFFFFFFLL || 2 * cap > 0xFFFFFFFFLL) return cudaErrorInvalidValue;
    StagedBufs<NM, D> b;
    b.cap = cap;
    double* p = scratch;
    b.P = p; p += kPrimVars(NM, D) * cap;
    b.ck = p; p += NM * cap;
    b.Pe = p; p += kPrimVars(NM, D) * cap;
    b.Ph = p; p += kPrimVars(NM, D) * cap;
    b.F = p;
    b.LS = b.RS = nullptr;
    b.PLS = b.PRS = nullptr;
    for (long long L0 = 0; L0 < nlines; L0 += per) {
        LineSet ls;
        ls.L0 = L0;
        ls.nl = (int)((nlines - L0 < per) ? (nlines - L0) : per);
        ls.n = n;
        ls.set_dividers(g.N[0]);
        const long long items = (long long)ls.nl * n;
        const unsigned blocks = (unsigned)((items + 255) / 256);
        FusedCfl fc{0, 0, 0.0, nullptr, 0.0, nullptr, nullptr, nullptr};
        if (fs.on) fc = FusedCfl{1, fs.unsplit, fs.cfl, fs.slot, fs.dt_max, fs.dt, fs.hist, fs.err};
        launch_stage(mixed_a<NM, D, DIR>, blocks, s, in, g, M, ls, b, fc);
        count_launches(1);
        if (twin) {
            launch_stage(mixed_b<NM, D, DIR, double>, blocks, s, in, g, M, ls, b, dt);
            launch_stage(mixed_cd<NM, D, DIR, double>, blocks, s, in, g, M, ls, b, err);
        }
        else {
            launch_stage(mixed_b<NM, D, DIR>, blocks, s, in, g, M, ls, b, dt);
            launch_stage(mixed_cd<NM, D, DIR>, blocks, s, in, g, M, ls, b, err);
        }
        count_launches(2);
        launch_stage(staged_e<NM, D, DIR>, blocks, s, in, out, g, M, ls, b, dt);
        count_launches(1);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template<int NM, int D>
cudaError_t launch_sweep_mixed(const Grid& g, const Mats& M, int dir, const double* in, double* out,
                               const double* dt, int* err, double* scratch, long long cap, const FusedStep& fs,
                               cudaStream_t s, bool twin)
{
    if (fs.on && (long long)g.ncell > cap) return cudaErrorInvalidValue;
    if (dir == 0) return launch_mixed_dir<NM, D, 0>(g, M, in, out, dt, err, scratch, cap, fs, s, twin);
    if constexpr (D >= 2) {
        if (dir == 1) return launch_mixed_dir<NM, D, 1>(g, M, in, out, dt, err, scratch, cap, fs, s, twin);
    }
    if constexpr (D >= 3) {
        if (dir == 2) return launch_mixed_dir<NM, D, 2>(g, M, in, out, dt, err, scratch, cap, fs, s, twin);
    }
    return cudaErrorInvalidValue;
}

template<int NM, int D>
cudaError_t launch_cfl(const Grid& g, const Mats& M, const double* state, double cfl, bool unsplit,
                       double* blockmin, int max_blocks, int* nblocks, cudaStream_t s, bool mixed, long long begin,
                       long long end)
{
    if (end < 0) end = g.ncell;
    long long nb = (end - begin + 255) / 256;
    if (nb > max_blocks) nb = max_blocks;
    if (nb < 1) nb = 1;
    *nblocks = (int)nb;
    cfl_kernel<NM, D><<<(unsigned)nb, 256, 0, s>>>(state, g, M, cfl, unsplit ? 1 : 0, mixed ? 1 : 0, blockmin,
                                                   begin, end);
    count_launches(1);
    return cudaGetLastError();
}

template<int NM, int D>
cudaError_t launch_bc(const Grid& g, const Mats& M, double* state, cudaStream_t s)
{
    // N == 2 makes a source cell a boundary cell; with a nonreflective side,
    // N == 3 on any axis makes the extrapolation's second cell one.
    bool serial = false, nonreflective = false, three = false;
    for (int a = 0; a < D; ++a) {
        if (g.N[a] == 2) serial = true;
        if (g.N[a] == 3) three = true;
        if (g.bc_lo[a] == DIMGPU_BC_NONREFLECTIVE || g.bc_hi[a] == DIMGPU_BC_NONREFLECTIVE) nonreflective = true;
    }
    if (nonreflective && three) serial = true;
    if (serial) {
        bc_serial_kernel<NM, D><<<1, 1, 0, s>>>(state, g, M);
        count_launches(1);
        return cudaGetLastError();
    }
    long long plane[3] = {0, 0, 0};
    long long total = 0;
    for (int a = 0; a < D; ++a) {
        if (g.N[a] <= 1) continue;
        long long c = 1;
        for (int b = 0; b < D; ++b) {
            if (b == a) continue;
            c *= (b < a && g.N[b] != 1) ? (long long)(g.N[b] - 2) : (long long)g.N[b];
        }
        plane[a] = c;
        total += 2 * c;
    }
    if (total == 0) return cudaSuccess;
    launch_stage(bc_kernel<NM, D>, (unsigned)((total + 255) / 256), s, state, g, M, plane[0], plane[1], plane[2]);
    count_launches(1);
    return cudaGetLastError();
}

template<int NM, int D>
cudaError_t launch_accumulate(const Grid& g, const Mats& M, double* accum, const double* dir_state,
                              const double* base, cudaStream_t s)
{
    accumulate_kernel<NM, D><<<(unsigned)((g.ncell + 255) / 256), 256, 0, s>>>(accum, dir_state, base, g, M);
    count_launches(1);
    return cudaGetLastError();
}

template<int NM, int D>
cudaError_t launch_totals(const Grid& g, const double* state, double volume, double* partial, int max_blocks,
                          int* nblocks, cudaStream_t s)
{
    long long nb = (g.ncell + 255) / 256;
    if (nb > max_blocks) nb = max_blocks;
    if (nb < 1) nb = 1;
    *nblocks = (int)nb;
    totals_kernel<NM, D><<<(unsigned)nb, 256, 0, s>>>(state, g, volume, partial);
    count_launches(1);
    return cudaGetLastError();
}

// ---- boundary flux integrand (compute_dim_boundary_flux,
// src/app/io/conservation_report.hpp:253-305): per axis and transverse line,
// area * (F(right end cell) - F(left end cell)) with the physical normal flux
// of each end cell's own state; per-block partial sums ----------------------------
template<int NM, int D>
__global__ void __launch_bounds__(256) boundary_flux_kernel(const double* __restrict__ st, __grid_constant__ const Grid g, __grid_constant__ const Mats M,
                                                            long long lines0, long long lines1, double area0,
                                                            double area1, double area2,
                                                            double* __restrict__ partial)
{
    constexpr int NV = NM + 1 + D + 1;
    __shared__ double red[NV][256];
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = 0.0;
    const long long total_lines = g.ncell / g.N[0] + (D > 1 ? g.ncell / g.N[1] : 0) + (D > 2 ? g.ncell / g.N[2] : 0);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < total_lines; p += stride) {
        int dir = 0;
        long long line = p;
        if (line >= lines0) {
            line -= lines0;
            dir = 1;
            if (line >= lines1) {
                line -= lines1;
                dir = 2;
            }
        }
        const double area = dir == 0 ? area0 : (dir == 1 ? area1 : area2);
        int idx[3] = {0, 0, 0};
        long long tmp = line;
        for (int a = D - 1; a >= 0; --a) {
            if (a == dir) continue;
            idx[a] = (int)(tmp % g.N[a]);
            tmp /= g.N[a];
        }
        long long base = 0;
        for (int a = 0; a < D; ++a) base += (long long)idx[a] * g.stride[a];
        for (int side = 1; side >= 0; --side) {  // right end first, as the reference adds it
            const long long cell = base + (side ? (long long)(g.N[dir] - 1) * g.stride[dir] : 0);
            State<NM, D> U;
            Prim<NM, D> P;
            load_cell<NM, D>(st, g.ncell, cell, U);
            cons_to_prim<NM, D>(M, U, P);
            Flux<NM, D> F;
            flux_normal<NM, D>(U, P, dir, F);
            const double scale = side ? area : -area;
            double mass_flux = 0.0;
#pragma unroll
            for (int k = 0; k < NM; ++k) {
                const double v = scale * F.m[k];
                acc[k] += v;
                mass_flux += v;
            }
            acc[NM] += mass_flux;
#pragma unroll
            for (int d = 0; d < D; ++d) acc[NM + 1 + d] += scale * F.mom[d];
            acc[NM + 1 + D] += scale * F.E;
        }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) red[v][threadIdx.x] = acc[v];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
#pragma unroll
            for (int v = 0; v < NV; ++v) red[v][threadIdx.x] += red[v][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) partial[(long long)blockIdx.x * NV + v] = red[v][0];
    }
}

template<int NM, int D>
cudaError_t launch_boundary_flux(const Grid& g, const Mats& M, const double* state, double* partial, int max_blocks,
                                 int* nblocks, cudaStream_t s)
{
    long long lines[3] = {0, 0, 0};
    double area[3] = {1.0, 1.0, 1.0};
    long long total = 0;
    for (int a = 0; a < D; ++a) {
        lines[a] = g.ncell / g.N[a];
        total += lines[a];
        for (int b = 0; b < D; ++b)
            if (b != a) area[a] *= g.dx[b];
    }
    long long nb = (total + 255) / 256;
    if (nb > max_blocks) nb = max_blocks;
    if (nb < 1) nb = 1;
    *nblocks = (int)nb;
    boundary_flux_kernel<NM, D><<<(unsigned)nb, 256, 0, s>>>(state, g, M, lines[0], lines[1], area[0], area[1],
                                                            area[2], partial);
    count_launches(1);
    return cudaGetLastError();
}

#define DIMGPU_INSTANTIATE_D(NM, D)                                                                          \
    template cudaError_t launch_sweep<NM, D>(const Grid&, const Mats&, int, Tile, const double*, double*,    \
                                             const double*, int*, cudaStream_t);                             \
    template cudaError_t launch_sweep_staged<NM, D>(const Grid&, const Mats&, int, const double*, double*,   \
                                                    const double*, int*, double*, long long, const FusedStep&, \
                                                    cudaStream_t);                                           \
    template cudaError_t launch_sweep_mixed<NM, D>(const Grid&, const Mats&, int, const double*, double*,    \
                                                   const double*, int*, double*, long long, const FusedStep&, \
                                                   cudaStream_t, bool);                                      \
    template cudaError_t launch_cfl<NM, D>(const Grid&, const Mats&, const double*, double, bool, double*,   \
                                           int, int*, cudaStream_t, bool, long long, long long);             \
    template cudaError_t launch_bc<NM, D>(const Grid&, const Mats&, double*, cudaStream_t);                  \
    template cudaError_t launch_accumulate<NM, D>(const Grid&, const Mats&, double*, const double*,          \
                                                  const double*, cudaStream_t);                              \
    template cudaError_t launch_totals<NM, D>(const Grid&, const double*, double, double*, int, int*,        \
                                              cudaStream_t);                                                 \
    template cudaError_t launch_boundary_flux<NM, D>(const Grid&, const Mats&, const double*, double*, int,   \
                                                     int*, cudaStream_t);

#define DIMGPU_INSTANTIATE(NM)   \
    DIMGPU_INSTANTIATE_D(NM, 1)  \
    DIMGPU_INSTANTIATE_D(NM, 2)  \
    DIMGPU_INSTANTIATE_D(NM, 3)

}  // namespace dimgpu
