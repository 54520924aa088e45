// dim_launch.h — host-side declarations of the kernel launchers.  The
// launchers are templates over the material count NM and the dimension D,
// defined in dim_kernels.cuh and instantiated per NM in inst_nm*.cu.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "dim_physics.h"
#include "fastdiv.h"

struct dimgpu_batch;

// Resident blocks of 256 threads per SM that the staged kernels are compiled
// for (their register budget: 65536 / (256 * blocks), 85 registers at 3).
// Measured on a B200, 2D shock-bubble 1024x512, FP64: 0.736 ms per step at
// 2 blocks (112-128 registers), 0.675 at 3, 0.691 at 4 — the stages are
// latency-bound, and the third block's warps hide more of the dependent
// FP64 chains than its spills cost.
#ifndef DIMGPU_STAGED_MINB
#define DIMGPU_STAGED_MINB 3
#endif

// Per-kernel resident blocks per SM of stages A, B's cell update, D and E.
// Measured on a B200: A and B's update at 4 (64 registers) 1.9 % (c1) and
// 2.6 % (c2) less time per step than at 3 (on the build with FastDiv item
// indices: c1 0.575 against 0.587 ms, c2 216.2 against 222.8); D and E at
// 4 slower.
#ifndef DIMGPU_A_MINB
#define DIMGPU_A_MINB 4
#endif
#ifndef DIMGPU_BU_MINB
#define DIMGPU_BU_MINB 4
#endif
#ifndef DIMGPU_D_MINB
#define DIMGPU_D_MINB DIMGPU_STAGED_MINB
#endif
#ifndef DIMGPU_E_MINB
#define DIMGPU_E_MINB DIMGPU_STAGED_MINB
#endif

// Resident blocks per SM of the per-face-state kernels (staged_bf, staged_c),
// whose threads carry one face state each: 64 registers.  Measured on a
// B200: 3.5 % less time per step on c2 (512^3) than at 3 blocks, 0.3 % on c1;
// at 5 (51 registers) c1 0.590 against 0.575 ms, c2 222.5 against 216.2.
#ifndef DIMGPU_FACE_MINB
#define DIMGPU_FACE_MINB 4
#endif

// Resident 256-thread blocks per SM the Euler sweep is compiled for (its
// register budget).  Measured on a B200: 5 (51 registers) 1 % faster on e2
// than 4, 3 slower.
#ifndef DIMGPU_EULER_MINB
#define DIMGPU_EULER_MINB 5
#endif

// Whether the Euler sweep builds each cell's two face states through one
// inlined copy of the routines (a loop of two) instead of two copies.
// Measured on a B200: 3 % (e2) and 5 % (e3) slower, so off.
#ifndef DIMGPU_EULER_FACE_LOOP
#define DIMGPU_EULER_FACE_LOOP 0
#endif

// Resident blocks per SM mixed_a is compiled for.  Measured on a B200: at 3
// (80 registers instead of 90) the mixed step is 4 % faster on c1 and 5 %
// on c2 than uncapped.
#ifndef DIMGPU_MIXED_A_MINB
#define DIMGPU_MIXED_A_MINB 3
#endif

// Resident blocks per SM of mixed_b and mixed_cd.  Measured on a B200: at 4
// the mixed c2 step is 2.5 % faster than at 3, c1 unchanged.
#ifndef DIMGPU_MIXED_BCD_MINB
#define DIMGPU_MIXED_BCD_MINB 4
#endif

// Whether the mixed-precision kernels (mixed_a, mixed_b, mixed_cd) inline
// their recoveries, conversions, repairs and sound speeds.  Measured on a
// B200: 2 % less time per step on c1, 3 % on c2 (512^3) inlined.
#ifndef DIMGPU_MIXED_INLINE
#define DIMGPU_MIXED_INLINE true
#endif

// Whether the batch kernels inline the FP64 stages' routines (the mixed
// instances of a batch always call the out-of-line copies).  Measured on a
// B200: c3 1.3 % more solves/s inlined.
#ifndef DIMGPU_BATCH_INLINE
#define DIMGPU_BATCH_INLINE true
#endif

// Whether stage A stores only the primitive P and the stage B kernels
// re-enforce it on load, instead of storing the enforced copy as well.
// Measured on a B200: FP64 c1 unchanged, c2 3 % slower (the enforce's
// instructions cost more than the record's traffic saves), so off.
#ifndef DIMGPU_STAGED_NO_PE
#define DIMGPU_STAGED_NO_PE false
#endif

// Whether the kernels of a session's step (the staged and mixed stages, the
// fused-CFL finalize, the boundary fill) are launched with programmatic
// stream serialization: each may be scheduled while its predecessor drains
// and waits at its top for the predecessor's completion.  Measured on a
// B200: c1 3.7 % less time per step.
#ifndef DIMGPU_PDL
#define DIMGPU_PDL true
#endif

// Whether the batch step's kernels (captured into the batch's CUDA graph)
// form a programmatic launch chain as well.  Measured on a B200: no change
// on c3 (44.4 ms batched steps), so off.
#ifndef DIMGPU_BATCH_PDL
#define DIMGPU_BATCH_PDL false
#endif

// Whether the staged schedule runs stages C and D as one kernel per face
// (staged_cd) instead of staged_c + staged_d.
#ifndef DIMGPU_STAGED_FUSE_CD
#define DIMGPU_STAGED_FUSE_CD false
#endif

// Whether the staged kernels split their item index into line and position
// with precomputed multiply-high dividers (FastDiv) instead of 64-bit
// integer division.
#ifndef DIMGPU_STAGED_FASTDIV
#define DIMGPU_STAGED_FASTDIV true
#endif

// Whether the staged schedule of a 2D or 3D grid runs stages D and E as one
// kernel (staged_de: a tile's faces handed to its cells through shared
// memory) instead of staged_d + staged_e.  Measured on a B200: c1 0.601
// against 0.590 ms per step, c2 at 512^3 230.9 against 220.9 ms (the fused
// kernel spills at 80 registers, 0.617 ms at 2 blocks per SM, and its
// cells wait at the barrier for the tile's slowest face), so off.
#ifndef DIMGPU_STAGED_FUSE_DE
#define DIMGPU_STAGED_FUSE_DE false
#endif
#ifndef DIMGPU_DE_MINB
#define DIMGPU_DE_MINB DIMGPU_STAGED_MINB
#endif

// Whether the staged D and E kernels inline their sound speeds and repairs
// (two call sites each) instead of calling the out-of-line copies.
// Measured on a B200: 1.5 % less time per step on c1 and c2 inlined.
#ifndef DIMGPU_STAGED_INLINE_DE
#define DIMGPU_STAGED_INLINE_DE true
#endif

namespace dimgpu {

// Error bits written by the kernels into the session's flag word.
enum : int {
    kErrNonFinite = 1,  // hllc_flux_normal's require_positive would throw
    kErrDt = 2,         // CFL step is not positive and finite
    kErrTimeout = 4,    // a bounded wait for a copy into shared memory ran out
};

// Kernels launched by this library so far, process-wide (read with
// dimgpu_kernel_launches).  Every launch site adds its count; a batch adds,
// per step, the kernels one step holds, whether launched directly or
// replayed from a captured graph.
void count_launches(long long n);

struct Grid {
    int N[3];
    long long ncell;
    long long stride[3];  // 1, Nx, Nx*Ny
    double dx[3];
    int bc_lo[3], bc_hi[3];
};

// Tile shape of the sweep kernel: T cells along the line (T - 6 of them are
// outputs, the other 6 the stencil halo), W lines per CTA.
struct Tile {
    int T;
    int W;
};

template<int NM, int D>
cudaError_t launch_sweep(const Grid& g, const Mats& M, int dir, Tile tile, const double* in, double* out,
                         const double* dt, int* err, cudaStream_t s);

// CFL reduction fused into stage A of a staged / mixed sweep: when `on`, the
// launcher reduces the CFL minimum into `slot` during stage A and writes
// dt = min(dt_max, minimum) to dt[0] (and hist[0]) before stage B.  Needs
// the grid to fit one scratch chunk.
struct FusedStep {
    int on;
    int unsplit;
    double cfl;
    double dt_max;
    unsigned long long* slot;
    double* dt;
    double* hist;
    int* err;
};

// The staged schedule of the same sweep: stages A..E as separate kernels
// over chunks of whole lines of at most `cap` cells, intermediates in
// `scratch` (staged_scratch_doubles(nmat, dim) * cap doubles).
template<int NM, int D>
cudaError_t launch_sweep_staged(const Grid& g, const Mats& M, int dir, const double* in, double* out,
                                const double* dt, int* err, double* scratch, long long cap, const FusedStep& fs,
                                cudaStream_t s);

int staged_scratch_doubles(int nmat, int dim);

// Mixed-precision staged sweep (dim_mixed.h): same scratch as the staged one.
// twin: the same algorithm with its FP32 quantities in FP64
// (DIMGPU_PRECISION_MIXED_FP64).
template<int NM, int D>
cudaError_t launch_sweep_mixed(const Grid& g, const Mats& M, int dir, const double* in, double* out,
                               const double* dt, int* err, double* scratch, long long cap, const FusedStep& fs,
                               cudaStream_t s, bool twin = false);

// Per-block CFL minima into blockmin[0 .. nblocks-1]; nblocks <= max_blocks.
// `mixed`: recover the cells as the mixed-precision step does.  Cells
// [begin, end) only (end < 0: to the last cell).
template<int NM, int D>
cudaError_t launch_cfl(const Grid& g, const Mats& M, const double* state, double cfl, bool unsplit,
                       double* blockmin, int max_blocks, int* nblocks, cudaStream_t s, bool mixed = false,
                       long long begin = 0, long long end = -1);

// dt = min(dt_max, min(blockmin)), written to dt[0] and hist[0] (hist may be null).
cudaError_t launch_cfl_finalize(const double* blockmin, int nblocks, double dt_max, double* dt,
                                double* hist, int* err, cudaStream_t s);

template<int NM, int D>
cudaError_t launch_bc(const Grid& g, const Mats& M, double* state, cudaStream_t s);

// accum += dir - base, then repair_state, for the unsplit update.
template<int NM, int D>
cudaError_t launch_accumulate(const Grid& g, const Mats& M, double* accum, const double* dir_state,
                              const double* base, cudaStream_t s);

// Per-block partial conservation sums: nmat + 1 + D + 1 values per block.
template<int NM, int D>
cudaError_t launch_totals(const Grid& g, const double* state, double volume, double* partial,
                          int max_blocks, int* nblocks, cudaStream_t s);

// Per-block partial sums of the boundary flux integrand (same layout as
// launch_totals).
template<int NM, int D>
cudaError_t launch_boundary_flux(const Grid& g, const Mats& M, const double* state, double* partial, int max_blocks,
                                 int* nblocks, cudaStream_t s);

// ---- batched form (dim_batch.cuh) ----
// One entry per instance of a batch, in device memory.
struct BInst {
    Grid g;
    Mats M;
    double* st[2];      // ping-pong state buffers (SoA, ncell stride)
    double* dtlog;      // dt of every step run, capacity = steps requested
    long long soff;     // first scratch item of this instance
    int steps_left;     // steps still to run
    int steps_done;     // steps run so far
    int run;            // runs in the current step (set by the finalize kernel)
    int cur;            // current buffer at the start of the step that last ran finalize
    int mixed;          // DIMGPU_PRECISION_MIXED: mixed_b / mixed_cd arithmetic
    double cfl, dt_max;
    double dt;          // dt of the current step
    int nl[3];          // lines along each axis (ncell / N[a])
    FastDiv by_n[3], by_nl[3], by_n0;  // dividers of the staged item index (set on the host)
};

// Device tables and scratch of one batched step.
struct BatchLaunch {
    BInst* tab;
    const long long* cell_prefix;  // work blocks of 256 cells per instance
    const long long* bc_prefix;    // work blocks of 256 boundary cells per instance
    int ninst;
    double* blockmin;
    double* scratch;
    long long cap;                 // scratch items
    int* err;
    int grid;                      // persistent grid size
};

// One time step of every running instance: per-instance CFL, the staged
// sweeps and boundary fills, with a persistent grid of L.grid CTAs.
template<int NM, int D>
cudaError_t batch_step(const BatchLaunch& L, cudaStream_t s);

int sweep_smem_doubles(int nmat, int dim);

// ---- the single-material Euler step (euler_kernels.cuh) ----
// One split sweep (fused tile kernel); end cells of each line get zeros
// (ends_copy 0, the split update) or their input state (1, unsplit).
template<int D>
cudaError_t launch_euler_sweep(const Grid& g, const Mats& M, int dir, Tile tile, const double* in, double* out,
                               const double* dt, int* err, int ends_copy, cudaStream_t s);

// Per-block CFL minima (finished by launch_cfl_finalize).
template<int D>
cudaError_t launch_euler_cfl(const Grid& g, const Mats& M, const double* state, double cfl, bool unsplit,
                             double* blockmin, int max_blocks, int* nblocks, int* err, cudaStream_t s);

template<int D>
cudaError_t launch_euler_bc(const Grid& g, const Mats& M, double* state, cudaStream_t s);

// acc = acc + (dir - base); with `enforce`, then enforce_positive_conserved.
template<int D>
cudaError_t launch_euler_accumulate(const Grid& g, const Mats& M, double* acc, const double* dir_state,
                                    const double* base, bool enforce, cudaStream_t s);

// Message returned by dimgpu_last_error(NULL) on the calling thread.
void set_sessionless_error(const std::string& msg);

// 1 when every step enqueued on the batch has finished, 0 while steps run
// (cudaEventQuery; no host synchronisation).
int batch_ready(::dimgpu_batch* b);

}  // namespace dimgpu
