// euler_kernels.cuh — CUDA kernels of the single-material Euler step
// (DIMGPU_MODEL_EULER) for sm_100a: the fused tiled sweep, the CFL
// reduction, the boundary fill and the unsplit accumulation.
//
// State: FP64 SoA, components rho, mom[0..D-1], E (V = D + 2), x-fastest.
// The sweep uses the tile mapping of the DIM sweep_kernel: a CTA of T*W
// threads covers W lines x T cells, positions 3..T-4 are written and the
// rest is the radius-3 stencil halo.  The Euler step is closed form (no
// bisection), so one fused kernel with the stage results in shared memory
// keeps the sweep near its HBM traffic: the state is read once and written
// once per sweep.
#pragma once

#include <cuda_runtime.h>

#include "dim_launch.h"
#include "pdl.cuh"
#include "fastdiv.h"
#include "euler_physics.h"
#include "dimgpu.h"

namespace dimgpu {

template<int D>
__device__ __forceinline__ void e_load(const double* __restrict__ s, long long ncell, long long i, EState<D>& U)
{
    U.rho = __ldg(s + i);
#pragma unroll
    for (int d = 0; d < D; ++d) U.mom[d] = __ldg(s + (1 + d) * ncell + i);
    U.E = __ldg(s + (1 + D) * ncell + i);
}

template<int D>
__device__ __forceinline__ void e_load_plain(const double* s, long long ncell, long long i, EState<D>& U)
{
    U.rho = s[i];
#pragma unroll
    for (int d = 0; d < D; ++d) U.mom[d] = s[(1 + d) * ncell + i];
    U.E = s[(1 + D) * ncell + i];
}

template<int D>
__device__ __forceinline__ void e_store(double* s, long long ncell, long long i, const EState<D>& U)
{
    s[i] = U.rho;
#pragma unroll
    for (int d = 0; d < D; ++d) s[(1 + d) * ncell + i] = U.mom[d];
    s[(1 + D) * ncell + i] = U.E;
}

// shared-memory record of slot t: variable v at sm[v * NT + t]
template<int D>
__device__ __forceinline__ void e_put(double* sm, int NT, int t, const EState<D>& U)
{
    sm[t] = U.rho;
#pragma unroll
    for (int d = 0; d < D; ++d) sm[(1 + d) * NT + t] = U.mom[d];
    sm[(1 + D) * NT + t] = U.E;
}

template<int D>
__device__ __forceinline__ void e_get(const double* sm, int NT, int t, EState<D>& U)
{
    U.rho = sm[t];
#pragma unroll
    for (int d = 0; d < D; ++d) U.mom[d] = sm[(1 + d) * NT + t];
    U.E = sm[(1 + D) * NT + t];
}

template<int D>
__device__ __forceinline__ void e_put(double* sm, int NT, int t, const EPrim<D>& P)
{
    sm[t] = P.rho;
#pragma unroll
    for (int d = 0; d < D; ++d) sm[(1 + d) * NT + t] = P.vel[d];
    sm[(1 + D) * NT + t] = P.p;
}

template<int D>
__device__ __forceinline__ void e_get(const double* sm, int NT, int t, EPrim<D>& P)
{
    P.rho = sm[t];
#pragma unroll
    for (int d = 0; d < D; ++d) P.vel[d] = sm[(1 + d) * NT + t];
    P.p = sm[(1 + D) * NT + t];
}

// One split sweep along DIR (sweep_lines_flat + advance_line fast path,
// src/sim/solver/advance/sweep_core.hpp:65-111, 458-516).  Interior cells of
// every line get the update; the two end cells of a line get zeros when
// `ends_copy` is 0 (the split update sweeps into a value-initialised buffer,
// src/core/fv/directional_update.hpp:13-18) or their input state when it is
// 1 (the unsplit update sweeps into a copy of the base state, :34-38).
//
// Every stage result goes to shared memory as soon as it is formed, so no
// state stays in registers across a barrier (the cell state is re-read
// through the read-only cache where a later stage needs it).  Three record
// buffers of V = D + 2 doubles per slot: S0 holds P (A -> B), then RS
// (C -> D); S1 holds Ph (B -> C), then the face flux F (D -> E); S2 holds LS
// (C -> D).
//
// Launch bound: 4 blocks of 256 threads per SM (64 registers a thread).  The
// sweep is latency-bound on dependent FP64 chains; the extra warps hide more
// of that latency than the few spilled registers (L1-resident) cost.
// Launch-invariant dividers of the tile mapping (thread -> position and
// line in the tile, block -> tile and line group), set on the host, and
// the grid's line count along x.
struct EulerTileDiv {
    FastDiv by_T, by_W, by_ntile, by_ngx;
    long long nlines;
};

template<int D, int DIR>
__global__ void __launch_bounds__(256, DIMGPU_EULER_MINB) euler_sweep_kernel(const double* __restrict__ in, double* __restrict__ out,
                                                             __grid_constant__ const Grid g, __grid_constant__ const Mats M, int T, int W, int ntile, int ngx,
                                                             EulerTileDiv dv, const double* __restrict__ dtp,
                                                             int* __restrict__ err, int ends_copy)
{
    pdl_enter();
    extern __shared__ double sm[];
    const int NT = T * W;
    double* S0 = sm;
    double* S1 = sm + (D + 2) * NT;
    double* S2 = sm + 2 * (D + 2) * NT;
    const int t = threadIdx.x;
    const int n = g.N[DIR];
    const int OUT = T - 6;

    int pos, j, s;
    if (DIR == 0) { j = (int)dv.by_T.div((unsigned)t); pos = t - j * T; s = 1; }
    else { pos = (int)dv.by_W.div((unsigned)t); j = t - pos * W; s = W; }

    const unsigned bid = blockIdx.x;
    int tile;
    long long base, sline;
    bool line_ok;
    if (DIR == 0) {
        const unsigned q = dv.by_ntile.div(bid);
        tile = (int)(bid - q * (unsigned)ntile);
        const long long L = (long long)q * W + j;
        line_ok = L < dv.nlines;
        base = L * g.N[0];
        sline = 1;
    }
    else {
        const unsigned rest = dv.by_ngx.div(bid);
        const int gx = (int)(bid - rest * (unsigned)ngx);
        const unsigned other_u = dv.by_ntile.div(rest);
        tile = (int)(rest - other_u * (unsigned)ntile);
        const long long other = other_u;
        const int x = gx * W + j;
        line_ok = x < g.N[0];
        base = (DIR == 1) ? x + other * g.stride[2] : x + other * g.stride[1];
        sline = g.stride[DIR];
    }
    const int gi = tile * OUT - 3 + pos;
    const bool valid = line_ok && gi >= 0 && gi < n;
    const bool end = gi == 0 || gi == n - 1;
    const long long cell = base + (long long)gi * sline;
    const double dt = *dtp;
    const double dx = g.dx[DIR];
    bool ok = true;

    // A: P_i = enforce(cons_to_prim(U_i))
    if (valid) {
        EState<D> U;
        e_load<D>(in, g.ncell, cell, U);
        EPrim<D> P = e_cons_to_prim<D>(M, U);
        e_enforce_prim<D>(P);
        e_put<D>(S0, NT, t, P);
    }
    __syncthreads();

    // B: half step -> Ph_i
    if (valid && (end || (pos >= 1 && pos <= T - 2))) {
        EPrim<D> P, Ph;
        e_get<D>(S0, NT, t, P);
        if (end) {
            Ph = P;
        }
        else {
            EPrim<D> lo, hi;
            e_get<D>(S0, NT, t - s, lo);
            e_get<D>(S0, NT, t + s, hi);
            EState<D> U, Uh;
            e_load<D>(in, g.ncell, cell, U);
#if DIMGPU_EULER_FACE_LOOP
            // both face states through one inlined copy (a loop of two, not
            // unrolled): half the instruction footprint of two copies
            EState<D> Uf[2];
#pragma unroll 1
            for (int side = 0; side < 2; ++side) Uf[side] = e_face_state<D>(M, lo, P, hi, side == 1);
            ok &= e_hancock<D>(M, U, Uf[0], Uf[1], DIR, dt, dx, Uh);
#else
            const EState<D> Ul = e_face_state<D>(M, lo, P, hi, false);
            const EState<D> Ur = e_face_state<D>(M, lo, P, hi, true);
            ok &= e_hancock<D>(M, U, Ul, Ur, DIR, dt, dx, Uh);
#endif
            Ph = e_cons_to_prim<D>(M, Uh);
            e_enforce_prim<D>(Ph);
        }
        e_put<D>(S1, NT, t, Ph);
    }
    __syncthreads();

    // C: face states of the second reconstruction, each enforced once more
    auto needC_at = [&](int p, int gidx) {
        const bool v = line_ok && gidx >= 0 && gidx < n;
        const bool e = gidx == 0 || gidx == n - 1;
        return v && (e || (p >= 2 && p <= T - 3));
    };
    const bool needC = needC_at(pos, gi);
    if (needC) {
#if DIMGPU_EULER_FACE_LOOP
        EPrim<D> lo, c, hi;
        if (!end) {
            e_get<D>(S1, NT, t - s, lo);
            e_get<D>(S1, NT, t, c);
            e_get<D>(S1, NT, t + s, hi);
        }
#pragma unroll 1
        for (int side = 0; side < 2; ++side) {
            EState<D> X;
            if (end) e_load<D>(in, g.ncell, cell, X);
            else X = e_face_state<D>(M, lo, c, hi, side == 1);
            e_enforce<D>(M, X);
            e_put<D>(side == 0 ? S2 : S0, NT, t, X);
        }
#else
        EState<D> LS, RS;
        if (end) {
            e_load<D>(in, g.ncell, cell, LS);
            RS = LS;
        }
        else {
            EPrim<D> lo, c, hi;
            e_get<D>(S1, NT, t - s, lo);
            e_get<D>(S1, NT, t, c);
            e_get<D>(S1, NT, t + s, hi);
            LS = e_face_state<D>(M, lo, c, hi, false);
            RS = e_face_state<D>(M, lo, c, hi, true);
        }
        e_enforce<D>(M, LS);
        e_enforce<D>(M, RS);
        e_put<D>(S2, NT, t, LS);
        e_put<D>(S0, NT, t, RS);
#endif
    }
    __syncthreads();

    // D: face i|i+1
    if (needC && pos + 1 <= T - 1 && gi + 1 < n && needC_at(pos + 1, gi + 1)) {
        EState<D> UL, UR, F;
        e_get<D>(S0, NT, t, UL);
        e_get<D>(S2, NT, t + s, UR);
        ok &= e_hllc<D>(M, UL, UR, DIR, F);
        e_put<D>(S1, NT, t, F);
    }
    __syncthreads();

    // E: outputs
    if (valid && pos >= 3 && pos <= T - 4) {
        EState<D> Un;
        if (end) {
            if (ends_copy) e_load<D>(in, g.ncell, cell, Un);
            else {
                Un.rho = 0.0;
#pragma unroll
                for (int d = 0; d < D; ++d) Un.mom[d] = 0.0;
                Un.E = 0.0;
            }
        }
        else {
            EState<D> U, Flo, Fhi;
            e_load<D>(in, g.ncell, cell, U);
            e_get<D>(S1, NT, t - s, Flo);
            e_get<D>(S1, NT, t, Fhi);
            e_update<D>(M, U, Flo, Fhi, dt, dx, Un);
        }
        e_store<D>(out, g.ncell, cell, Un);
    }
    if (!ok) atomicOr(err, kErrNonFinite);
}

// CFL partial minima (compute_dt_cfl_materials[_unsplit],
// src/sim/solver/cfl.hpp:64-187), finished by the DIM finalize kernel.
template<int D>
__global__ void __launch_bounds__(256) euler_cfl_kernel(const double* __restrict__ st, __grid_constant__ const Grid g, __grid_constant__ const Mats M, double cfl,
                                                        int unsplit, double* __restrict__ blockmin,
                                                        int* __restrict__ err)
{
    pdl_enter();
    __shared__ double red[32];
    double best = HUGE_VAL;
    bool ok = true;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.ncell; i += stride) {
        EState<D> U;
        e_load<D>(st, g.ncell, i, U);
        double c;
        ok &= e_cfl_candidate<D>(M, U, g.dx, cfl, unsplit != 0, c);
        best = dmin(best, c);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = dmin(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x < 32) {
        const int nw = blockDim.x >> 5;
        double v = threadIdx.x < (unsigned)nw ? red[threadIdx.x] : HUGE_VAL;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0) blockmin[blockIdx.x] = v;
    }
    if (!ok) atomicOr(err, kErrNonFinite);
}

// ---- boundary fill (apply_boundary_conditions,
// src/sim/solver/advance/boundary.hpp:149-201) ------------------------------------
//
// Every boundary cell copies its source cell (each boundary axis one cell
// inward), flipping the normal momentum on reflective sides; nonreflective
// cells take local_nonreflective_state (:96-147), enforced.  With every
// axis N >= 4 (N >= 3 without nonreflective sides) all reads are interior
// cells, so one thread per boundary cell reproduces the reference's serial
// in-place loop; otherwise the serial kernel runs it in the linear order.
template<int D>
__device__ void euler_bc_cell(const Grid& g, const Mats& M, double* st, const int* idx, long long linear)
{
    int src[3] = {0, 0, 0};
    bool is_boundary = false;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        src[a] = idx[a];
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
    EState<D> U;
    e_load_plain<D>(st, g.ncell, src_lin, U);
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
        EState<D> S2, ex;
        e_load_plain<D>(st, g.ncell, sec_lin, S2);
        ex.rho = U.rho + (U.rho - S2.rho);
#pragma unroll
        for (int d = 0; d < D; ++d) ex.mom[d] = U.mom[d] + (U.mom[d] - S2.mom[d]);
        ex.E = U.E + (U.E - S2.E);
        int axis = 0;
#pragma unroll
        for (int a = D - 1; a >= 0; --a)
            if (idx[a] == 0 || idx[a] == g.N[a] - 1) axis = a;
        const int outward = (idx[axis] == 0) ? -1 : 1;
        double ex_mom_axis = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d)
            if (d == axis) ex_mom_axis = ex.mom[d];
        const double vn = outward * safe_div(ex_mom_axis, ex.rho);
        // has_physical_energy (:76-94)
        bool phys = fin(ex.rho) && ex.rho > 0.0 && fin(ex.E);
        double mom2 = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            phys = phys && fin(ex.mom[d]);
            mom2 += ex.mom[d] * ex.mom[d];
        }
        phys = phys && ex.E > 0.5 * mom2 / dmax(ex.rho, 1e-12);
        if (phys && vn > 0.0) {
            const double rho = dmax(U.rho, 1e-12);
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
        e_enforce<D>(M, U);
    }
    else {
#pragma unroll
        for (int a = 0; a < D; ++a) {
            if ((idx[a] == 0 && g.bc_lo[a] == DIMGPU_BC_REFLECTIVE) ||
                (idx[a] == g.N[a] - 1 && g.bc_hi[a] == DIMGPU_BC_REFLECTIVE))
                U.mom[a] *= -1.0;
        }
    }
    e_store<D>(st, g.ncell, linear, U);
}

// Boundary shell as planes (as bc_kernel): plane 2a+side holds the cells
// with idx[a] at that side whose lower axes are interior.
template<int D>
__global__ void __launch_bounds__(256) euler_bc_kernel(double* st, __grid_constant__ const Grid g, __grid_constant__ const Mats M, long long plane0,
                                                       long long plane1, long long plane2)
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
        const bool inner = b < a;
        const int ext = inner ? (g.N[b] - 2) : g.N[b];
        idx[b] = (int)(r % ext) + (inner ? 1 : 0);
        r /= ext;
    }
    idx[a] = side ? g.N[a] - 1 : 0;
    long long linear = 0;
#pragma unroll
    for (int b = 0; b < D; ++b) linear += (long long)idx[b] * g.stride[b];
    euler_bc_cell<D>(g, M, st, idx, linear);
}

template<int D>
__global__ void euler_bc_serial_kernel(double* st, __grid_constant__ const Grid g, __grid_constant__ const Mats M)
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
        euler_bc_cell<D>(g, M, st, idx, linear);
    }
}

// Unsplit: acc = acc + (dir - base) per axis (advance_step.hpp:617-623), then
// enforce every cell once (:626-641) before the boundary fill.
template<int D>
__global__ void __launch_bounds__(256) euler_accumulate_kernel(double* __restrict__ acc,
                                                               const double* __restrict__ dir_state,
                                                               const double* __restrict__ base, __grid_constant__ const Grid g, __grid_constant__ const Mats M,
                                                               int enforce)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.ncell) return;
    EState<D> a, d, b;
    e_load<D>(acc, g.ncell, i, a);
    e_load<D>(dir_state, g.ncell, i, d);
    e_load<D>(base, g.ncell, i, b);
    a.rho = a.rho + (d.rho - b.rho);
#pragma unroll
    for (int q = 0; q < D; ++q) a.mom[q] = a.mom[q] + (d.mom[q] - b.mom[q]);
    a.E = a.E + (d.E - b.E);
    if (enforce) e_enforce<D>(M, a);
    e_store<D>(acc, g.ncell, i, a);
}

// ---- launchers -------------------------------------------------------------------
template<int D, int DIR>
cudaError_t launch_euler_sweep_dir(const Grid& g, const Mats& M, Tile tile, const double* in, double* out,
                                   const double* dt, int* err, int ends_copy, cudaStream_t s)
{
    int T = tile.T, W = tile.W;
    const int n = g.N[DIR];
    if (DIR != 0 && g.N[0] < W) {  // narrow grids: fewer lines per CTA
        W = 1;
        T = 128;
    }
    const int OUT = T - 6;
    const int ntile = (n + OUT - 1) / OUT;
    long long nblocks;
    int ngx = 1;
    if (DIR == 0) {
        const long long nlines = g.ncell / g.N[0];
        nblocks = ((nlines + W - 1) / W) * ntile;
    }
    else {
        ngx = (g.N[0] + W - 1) / W;
        const long long other = g.ncell / ((long long)g.N[0] * n);
        nblocks = (long long)ngx * ntile * other;
    }
    const size_t smem = sizeof(double) * 3 * (size_t)(D + 2) * (size_t)(T * W);
    auto kern = euler_sweep_kernel<D, DIR>;
    const cudaError_t ea = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ea != cudaSuccess) return ea;
    if (nblocks > 0xFFFFFFFFLL) return cudaErrorInvalidValue;
    EulerTileDiv dv;
    dv.by_T.set((unsigned)T);
    dv.by_W.set((unsigned)W);
    dv.by_ntile.set((unsigned)ntile);
    dv.by_ngx.set((unsigned)ngx);
    dv.nlines = g.ncell / g.N[0];
    launch_stage_smem(kern, (unsigned)nblocks, (unsigned)(T * W), smem, s, in, out, g, M, T, W, ntile, ngx, dv, dt,
                      err, ends_copy);
    count_launches(1);
    return cudaGetLastError();
}

template<int D>
cudaError_t launch_euler_sweep(const Grid& g, const Mats& M, int dir, Tile tile, const double* in, double* out,
                               const double* dt, int* err, int ends_copy, cudaStream_t s)
{
    if (tile.T < 8 || tile.W < 1 || tile.T * tile.W > 256) return cudaErrorInvalidValue;
    if (dir == 0) return launch_euler_sweep_dir<D, 0>(g, M, tile, in, out, dt, err, ends_copy, s);
    if constexpr (D >= 2) {
        if (dir == 1) return launch_euler_sweep_dir<D, 1>(g, M, tile, in, out, dt, err, ends_copy, s);
    }
    if constexpr (D >= 3) {
        if (dir == 2) return launch_euler_sweep_dir<D, 2>(g, M, tile, in, out, dt, err, ends_copy, s);
    }
    return cudaErrorInvalidValue;
}

template<int D>
cudaError_t launch_euler_cfl(const Grid& g, const Mats& M, const double* state, double cfl, bool unsplit,
                             double* blockmin, int max_blocks, int* nblocks, int* err, cudaStream_t s)
{
    long long nb = (g.ncell + 255) / 256;
    if (nb > max_blocks) nb = max_blocks;
    if (nb < 1) nb = 1;
    *nblocks = (int)nb;
    launch_stage(euler_cfl_kernel<D>, (unsigned)nb, s, state, g, M, cfl, unsplit ? 1 : 0, blockmin, err);
    count_launches(1);
    return cudaGetLastError();
}

template<int D>
cudaError_t launch_euler_bc(const Grid& g, const Mats& M, double* state, cudaStream_t s)
{
    bool nonreflective = false, three = false;
    for (int a = 0; a < D; ++a) {
        if (g.N[a] == 3) three = true;
        if (g.bc_lo[a] == DIMGPU_BC_NONREFLECTIVE || g.bc_hi[a] == DIMGPU_BC_NONREFLECTIVE) nonreflective = true;
    }
    if (nonreflective && three) {
        euler_bc_serial_kernel<D><<<1, 1, 0, s>>>(state, g, M);
        count_launches(1);
        return cudaGetLastError();
    }
    long long plane[3] = {0, 0, 0};
    long long total = 0;
    for (int a = 0; a < D; ++a) {
        long long c = 1;
        for (int b = 0; b < D; ++b) {
            if (b == a) continue;
            c *= (b < a) ? (g.N[b] - 2) : g.N[b];
        }
        plane[a] = c;
        total += 2 * c;
    }
    if (total == 0) return cudaSuccess;
    launch_stage(euler_bc_kernel<D>, (unsigned)((total + 255) / 256), s, state, g, M, plane[0], plane[1], plane[2]);
    count_launches(1);
    return cudaGetLastError();
}

template<int D>
cudaError_t launch_euler_accumulate(const Grid& g, const Mats& M, double* acc, const double* dir_state,
                                    const double* base, bool enforce, cudaStream_t s)
{
    euler_accumulate_kernel<D><<<(unsigned)((g.ncell + 255) / 256), 256, 0, s>>>(acc, dir_state, base, g, M,
                                                                                enforce ? 1 : 0);
    count_launches(1);
    return cudaGetLastError();
}

#define DIMGPU_INSTANTIATE_EULER(D)                                                                               \
    template cudaError_t launch_euler_sweep<D>(const Grid&, const Mats&, int, Tile, const double*, double*,      \
                                               const double*, int*, int, cudaStream_t);                          \
    template cudaError_t launch_euler_cfl<D>(const Grid&, const Mats&, const double*, double, bool, double*, int, \
                                             int*, int*, cudaStream_t);                                          \
    template cudaError_t launch_euler_bc<D>(const Grid&, const Mats&, double*, cudaStream_t);                    \
    template cudaError_t launch_euler_accumulate<D>(const Grid&, const Mats&, double*, const double*,            \
                                                    const double*, bool, cudaStream_t);

}  // namespace dimgpu
