// dim_batch.cuh — kernels of the batched form: many independent DIM grids
// (different sizes, materials and time steps) advanced together.
//
// Every kernel is launched with a fixed grid (a multiple of the SM count) and
// walks "work blocks" of 256 items; work block wb belongs to the instance i
// with prefix[i] <= wb < prefix[i+1] (a device table, so membership can
// change without relaunch geometry changing: a captured CUDA graph stays
// valid).  Per instance: its Grid, Mats, two state buffers, a dt log and its
// remaining step count live in a device table of BInst.  Each instance keeps
// its own buffer parity: `cur` is its current buffer at the start of the
// step, sweep k of a step reads st[cur ^ (k & 1)] and writes the other one,
// and an instance that does not run in a step touches neither buffer.  The
// parity advances in the next step's finalize (by D if the instance ran), so
// no kernel of a step depends on another instance's progress.
#pragma once

#include "dim_kernels.cuh"

namespace dimgpu {



// Largest i with prefix[i] <= wb (prefix[0] = 0, prefix[ninst] = total).
__device__ __forceinline__ int batch_find(const long long* __restrict__ prefix, int ninst, long long wb)
{
    int lo = 0, hi = ninst;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(prefix + mid) <= wb) lo = mid;
        else hi = mid;
    }
    return lo;
}

// ---- CFL ----------------------------------------------------------------------------
// Current buffer at the start of this step: the previous step's start
// buffer, advanced by D sweeps if the instance ran in that step.
template<int D>
__device__ __forceinline__ int batch_cur(const BInst& I)
{
    return I.run ? (I.cur ^ (D & 1)) : I.cur;
}

template<int NM, int D>
__global__ void __launch_bounds__(256) batch_cfl(const BInst* __restrict__ tab, const long long* __restrict__ prefix,
                                                 int ninst, double* __restrict__ blockmin)
{
    pdl_enter_if<DIMGPU_BATCH_PDL>();
    __shared__ double red[8];
    const long long total = prefix[ninst];
    for (long long wb = blockIdx.x; wb < total; wb += gridDim.x) {
        const int i = batch_find(prefix, ninst, wb);
        const BInst& I = tab[i];
        double best = HUGE_VAL;
        const long long c = (wb - prefix[i]) * 256 + threadIdx.x;
        if (I.steps_left > 0 && c < I.g.ncell) {
            State<NM, D> U;
            Prim<NM, D> P;
            load_cell<NM, D>(I.st[batch_cur<D>(I)], I.g.ncell, c, U);
            if (I.mixed) cons_to_prim_mixed<NM, D>(I.M, U, P);
            else cons_to_prim<NM, D>(I.M, U, P);
            best = cfl_candidate<NM, D>(I.M, U, P, I.g.dx, I.cfl, false);
        }
        best = warp_min(best);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = red[0];
            for (int w = 1; w < 8; ++w) m = dmin(m, red[w]);
            blockmin[wb] = m;
        }
        __syncthreads();
    }
}

// One block per instance (strided): advances the instance's buffer parity
// past the previous step, then dt = min(dt_max, candidates), decides whether
// the instance runs this step and logs its dt.
template<int D>
__global__ void __launch_bounds__(256) batch_finalize(BInst* __restrict__ tab, const long long* __restrict__ prefix,
                                                      int ninst, const double* __restrict__ blockmin,
                                                      int* __restrict__ err)
{
    pdl_enter_if<DIMGPU_BATCH_PDL>();
    __shared__ double red[8];
    for (int i = blockIdx.x; i < ninst; i += gridDim.x) {
        double v = HUGE_VAL;
        for (long long wb = prefix[i] + threadIdx.x; wb < prefix[i + 1]; wb += blockDim.x) v = dmin(v, blockmin[wb]);
        v = warp_min(v);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            BInst& I = tab[i];
            double m = red[0];
            for (int w = 1; w < 8; ++w) m = dmin(m, red[w]);
            I.cur = batch_cur<D>(I);
            if (I.steps_left > 0) {
                const double d = dmin(I.dt_max, m);
                I.dt = d;
                I.run = 1;
                I.dtlog[I.steps_done] = d;
                I.steps_done += 1;
                I.steps_left -= 1;
                if (!(d > 0.0) || !fin(d)) atomicOr(err, kErrDt);
            }
            else {
                I.run = 0;
            }
        }
        __syncthreads();
    }
}

// ---- staged sweep over all instances ---------------------------------------------------
#define BATCH_LOOP_BEGIN                                                                   \
    const long long total = prefix[ninst];                                                 \
    for (long long wb = blockIdx.x; wb < total; wb += gridDim.x) {                         \
        const int inst = batch_find(prefix, ninst, wb);                                    \
        const BInst& I = tab[inst];                                                        \
        const long long t = (wb - prefix[inst]) * 256 + threadIdx.x;                       \
        if (t >= I.g.ncell) continue;                                                      \
        const int n = I.g.N[DIR];                                                          \
        LineSet ls;                                                                        \
        ls.L0 = 0;                                                                         \
        ls.n = n;                                                                          \
        ls.nl = I.nl[DIR];                                                                 \
        ls.by_n = I.by_n[DIR];                                                             \
        ls.by_nl = I.by_nl[DIR];                                                           \
        ls.by_n0 = I.by_n0;                                                                \
        const StagedItem<DIR, DIMGPU_STAGED_FASTDIV> it(I.g, ls, t);                       \
        const long long q = I.soff + t;                                                    \
        const double* in = I.st[I.cur ^ rel];                                              \
        (void)in;

#define BATCH_LOOP_END }

template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_STAGED_MINB) batch_a(const BInst* __restrict__ tab, const long long* __restrict__ prefix,
                                               int ninst, int rel, StagedBufs<NM, D> b)
{
    pdl_enter_if<DIMGPU_BATCH_PDL>();
    BATCH_LOOP_BEGIN
    if (!I.run || n == 1) continue;
    State<NM, D> U;
    load_cell<NM, D>(in, I.g.ncell, it.cell, U);
    CellA<NM, D> A;
    if (I.mixed) stage_a_mixed<NM, D>(I.M, U, A);
    else stage_a<NM, D, DIMGPU_BATCH_INLINE>(I.M, U, A);
    g_put<NM, D>(b.P, b.cap, q, A.P);
    g_put<NM, D>(b.Pe, b.cap, q, A.Pe);
#pragma unroll
    for (int k = 0; k < NM; ++k) b.ck[k * b.cap + q] = A.ck[k];
    BATCH_LOOP_END
}

template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_STAGED_MINB) batch_b(const BInst* __restrict__ tab, const long long* __restrict__ prefix,
                                               int ninst, int rel, StagedBufs<NM, D> b)
{
    pdl_enter_if<DIMGPU_BATCH_PDL>();
    BATCH_LOOP_BEGIN
    if (!I.run || n == 1) continue;
    const bool end = it.gi == 0 || it.gi == n - 1 || n < 3;
    CellA<NM, D> A;
    g_get<NM, D>(b.Pe, b.cap, q, A.Pe);
    Prim<NM, D> Ph;
    if (end) {
        Ph = A.Pe;
    }
    else {
        State<NM, D> U;
        load_cell<NM, D>(in, I.g.ncell, it.cell, U);
#pragma unroll
        for (int k = 0; k < NM; ++k) A.ck[k] = b.ck[k * b.cap + q];
        Prim<NM, D> lo, hi;
        g_get<NM, D>(b.Pe, b.cap, q - it.s, lo);
        g_get<NM, D>(b.Pe, b.cap, q + it.s, hi);
        if (I.mixed) {
            stage_b_mixed<NM, D>(I.M, U, A, lo, hi, false, DIR, I.dt, I.g.dx[DIR], Ph);
        }
        else {
            State<NM, D> Uh;
            stage_b<NM, D, DIMGPU_BATCH_INLINE>(I.M, U, A, lo, hi, false, DIR, I.dt, I.g.dx[DIR], Uh, Ph);
        }
    }
    g_put<NM, D>(b.Ph, b.cap, q, Ph);
    BATCH_LOOP_END
}

template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_STAGED_MINB) batch_c(const BInst* __restrict__ tab, const long long* __restrict__ prefix,
                                               int ninst, int rel, StagedBufs<NM, D> b)
{
    pdl_enter_if<DIMGPU_BATCH_PDL>();
    BATCH_LOOP_BEGIN
    if (!I.run || n == 1 || I.mixed) continue;  // mixed instances build their face states in batch_d
    const bool end = it.gi == 0 || it.gi == n - 1 || n < 3;
    State<NM, D> LS, RS;
    Prim<NM, D> PLS, PRS;
    if (end) {
        load_cell<NM, D>(in, I.g.ncell, it.cell, LS);
        RS = LS;
        g_get<NM, D>(b.P, b.cap, q, PLS);
        PRS = PLS;
    }
    else {
        CellA<NM, D> A;
        State<NM, D> U;
        Prim<NM, D> Ph, lo, hi;
        g_get<NM, D>(b.Ph, b.cap, q, Ph);
        g_get<NM, D>(b.Ph, b.cap, q - it.s, lo);
        g_get<NM, D>(b.Ph, b.cap, q + it.s, hi);
        stage_c<NM, D, DIMGPU_BATCH_INLINE>(I.M, U, A, Ph, lo, hi, false, LS, RS, PLS, PRS);
    }
    g_put<NM, D>(b.LS, b.cap, q, LS);
    g_put<NM, D>(b.RS, b.cap, q, RS);
    g_put<NM, D>(b.PLS, b.cap, q, PLS);
    g_put<NM, D>(b.PRS, b.cap, q, PRS);
    BATCH_LOOP_END
}

template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_STAGED_MINB) batch_d(const BInst* __restrict__ tab, const long long* __restrict__ prefix,
                                               int ninst, int rel, StagedBufs<NM, D> b, int* __restrict__ err)
{
    pdl_enter_if<DIMGPU_BATCH_PDL>();
    BATCH_LOOP_BEGIN
    if (!I.run || n == 1 || it.gi >= n - 1) continue;
    State<NM, D> UL, UR;
    Prim<NM, D> PL, PR;
    FaceD<NM, D> f;
    if (I.mixed) {
        // mixed_cd: both face states from the half-step primitives
        mixed_face<NM, D, DIR>(in, I.g, I.M, b, it, q, n, true, UL, PL);
        StagedItem<DIR, DIMGPU_STAGED_FASTDIV> nx = it;
        nx.gi += 1;
        nx.cell += I.g.stride[DIR];
        mixed_face<NM, D, DIR>(in, I.g, I.M, b, nx, q + it.s, n, false, UR, PR);
        if (!stage_d_mixed<NM, D>(I.M, UL, PL, UR, PR, DIR, f)) atomicOr(err, kErrNonFinite);
    }
    else {
        g_get<NM, D>(b.RS, b.cap, q, UL);
        g_get<NM, D>(b.PRS, b.cap, q, PL);
        g_get<NM, D>(b.LS, b.cap, q + it.s, UR);
        g_get<NM, D>(b.PLS, b.cap, q + it.s, PR);
        if (!stage_d<NM, D, DIMGPU_BATCH_INLINE>(I.M, UL, PL, UR, PR, DIR, f)) atomicOr(err, kErrNonFinite);
    }
    g_put<NM, D>(b.F, b.cap, q, f);
    BATCH_LOOP_END
}

// Stage E writes the other buffer; a running instance whose line along DIR
// is a single cell (no update along that axis) copies its state across.
template<int NM, int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_STAGED_MINB) batch_e(const BInst* __restrict__ tab, const long long* __restrict__ prefix,
                                               int ninst, int rel, StagedBufs<NM, D> b)
{
    pdl_enter_if<DIMGPU_BATCH_PDL>();
    BATCH_LOOP_BEGIN
    if (!I.run) continue;
    double* out = I.st[I.cur ^ rel ^ 1];
    State<NM, D> U;
    load_cell<NM, D>(in, I.g.ncell, it.cell, U);
    if (n == 1) {
        store_cell<NM, D>(out, I.g.ncell, it.cell, U);
        continue;
    }
    const bool first = it.gi == 0, last = it.gi == n - 1;
    CellA<NM, D> A;
    g_get<NM, D>(b.P, b.cap, q, A.P);
#pragma unroll
    for (int k = 0; k < NM; ++k) A.ck[k] = b.ck[k * b.cap + q];
    FaceD<NM, D> lo, hi;
    if (!first) g_get<NM, D>(b.F, b.cap, q - it.s, lo);
    if (!last) g_get<NM, D>(b.F, b.cap, q, hi);
    State<NM, D> Un;
    stage_e<NM, D, DIMGPU_BATCH_INLINE>(I.M, U, A, first ? nullptr : &lo, last ? nullptr : &hi, first, last, I.dt,
                                         I.g.dx[DIR], Un);
    store_cell<NM, D>(out, I.g.ncell, it.cell, Un);
    BATCH_LOOP_END
}

// Boundary fill of every running instance (one thread per boundary cell; the
// batch admits only grids whose fill is order-independent).
template<int NM, int D>
__global__ void __launch_bounds__(256) batch_bc(const BInst* __restrict__ tab, const long long* __restrict__ bprefix,
                                                int ninst, int rel)
{
    pdl_enter_if<DIMGPU_BATCH_PDL>();
    const long long total = bprefix[ninst];
    for (long long wb = blockIdx.x; wb < total; wb += gridDim.x) {
        const int inst = batch_find(bprefix, ninst, wb);
        const BInst& I = tab[inst];
        if (!I.run) continue;
        long long i = (wb - bprefix[inst]) * 256 + threadIdx.x;
        long long count[3] = {0, 0, 0};
        for (int a = 0; a < D; ++a) {
            if (I.g.N[a] <= 1) continue;
            long long c = 1;
            for (int bb = 0; bb < D; ++bb) {
                if (bb == a) continue;
                c *= (bb < a && I.g.N[bb] != 1) ? (long long)(I.g.N[bb] - 2) : (long long)I.g.N[bb];
            }
            count[a] = c;
        }
        int a = 0;
        while (a < D && i >= 2 * count[a]) { i -= 2 * count[a]; ++a; }
        if (a >= D) continue;
        const int side = (int)(i / count[a]);
        long long r = i % count[a];
        int idx[3] = {0, 0, 0};
        for (int bb = 0; bb < D; ++bb) {
            if (bb == a) continue;
            const bool inner = bb < a && I.g.N[bb] != 1;
            const int ext = inner ? (I.g.N[bb] - 2) : I.g.N[bb];
            idx[bb] = (int)(r % ext) + (inner ? 1 : 0);
            r /= ext;
        }
        idx[a] = side ? I.g.N[a] - 1 : 0;
        long long linear = 0;
        for (int bb = 0; bb < D; ++bb) linear += (long long)idx[bb] * I.g.stride[bb];
        bc_cell<NM, D>(I.g, I.M, I.st[I.cur ^ rel], idx, linear);
    }
}

// ---- launchers -----------------------------------------------------------------------


template<int NM, int D>
cudaError_t batch_step(const BatchLaunch& L, cudaStream_t s)
{
    StagedBufs<NM, D> b;
    b.cap = L.cap;
    double* p = L.scratch;
    b.P = p; p += kPrimVars(NM, D) * L.cap;
    b.ck = p; p += NM * L.cap;
    b.Pe = p; p += kPrimVars(NM, D) * L.cap;
    b.Ph = p; p += kPrimVars(NM, D) * L.cap;
    b.LS = p; p += kStateVars(NM, D) * L.cap;
    b.RS = p; p += kStateVars(NM, D) * L.cap;
    b.PLS = p; p += kPrimVars(NM, D) * L.cap;
    b.PRS = p; p += kPrimVars(NM, D) * L.cap;
    b.F = p;
    launch_chained<DIMGPU_BATCH_PDL>(batch_cfl<NM, D>, L.grid, 256u, 0, s, L.tab, L.cell_prefix, L.ninst, L.blockmin);
    launch_chained<DIMGPU_BATCH_PDL>(batch_finalize<D>, L.grid, 256u, 0, s, L.tab, L.cell_prefix, L.ninst, L.blockmin,
                                     L.err);
    // sweep k reads st[cur ^ (k & 1)]; the boundary fill after it works on the
    // buffer it wrote, st[cur ^ (k & 1) ^ 1]
#define BATCH_DIR(DIR)                                                                                   \
    launch_chained<DIMGPU_BATCH_PDL>(batch_a<NM, D, DIR>, L.grid, 256u, 0, s, L.tab, L.cell_prefix, L.ninst, DIR & 1, b); \
    launch_chained<DIMGPU_BATCH_PDL>(batch_b<NM, D, DIR>, L.grid, 256u, 0, s, L.tab, L.cell_prefix, L.ninst, DIR & 1, b); \
    launch_chained<DIMGPU_BATCH_PDL>(batch_c<NM, D, DIR>, L.grid, 256u, 0, s, L.tab, L.cell_prefix, L.ninst, DIR & 1, b); \
    launch_chained<DIMGPU_BATCH_PDL>(batch_d<NM, D, DIR>, L.grid, 256u, 0, s, L.tab, L.cell_prefix, L.ninst, DIR & 1, b,   \
                                     L.err);                                                            \
    launch_chained<DIMGPU_BATCH_PDL>(batch_e<NM, D, DIR>, L.grid, 256u, 0, s, L.tab, L.cell_prefix, L.ninst, DIR & 1, b); \
    launch_chained<DIMGPU_BATCH_PDL>(batch_bc<NM, D>, L.grid, 256u, 0, s, L.tab, L.bc_prefix, L.ninst, (DIR & 1) ^ 1);
    BATCH_DIR(0)
    if constexpr (D >= 2) { BATCH_DIR(1) }
    if constexpr (D >= 3) { BATCH_DIR(2) }
#undef BATCH_DIR
    return cudaGetLastError();
}

#define DIMGPU_INSTANTIATE_BATCH(NM)                                                        \
    template cudaError_t batch_step<NM, 1>(const BatchLaunch&, cudaStream_t);               \
    template cudaError_t batch_step<NM, 2>(const BatchLaunch&, cudaStream_t);               \
    template cudaError_t batch_step<NM, 3>(const BatchLaunch&, cudaStream_t);

}  // namespace dimgpu
