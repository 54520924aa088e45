/*
 * dimgpu.h — C-ABI of the B200-native Allaire five-equation diffuse-interface
 * (DIM) time step.
 *
 * The library replaces the header-only, OpenMP-parallel DIM step of
 * SegunOwoeye/diffuse_vs_GFM_MMS.  Every entry point below names the reference
 * function it stands in for (paths relative to the reference project root).
 * Signatures are plain C: pointers, sizes and POD structs only, so the
 * reference's C++ host (or ctypes, or any FFI) can bind them directly.
 *
 * State layout (host and device): structure of arrays, FP64, component-major.
 * Component c of cell `linear` lives at soa[c * ncell + linear], where the
 * linear index is x-fastest exactly as in the reference
 * (src/dim/solver/advance/geometry.hpp:26-53).  The components of one cell are
 * the fields of dim::State<DIM> (src/dim/state.hpp:9-15) in declaration order:
 *
 *     partial_mass[0 .. nmat-1], mom[0 .. DIM-1], E, alpha[0 .. nmat-2]
 *
 * so V = 2*nmat + DIM components per cell (V = 5, 6, 7 for two materials in
 * 1D, 2D, 3D).
 *
 * Status codes: every call returns DIMGPU_OK (0) or a positive error code;
 * dimgpu_last_error() gives a one-line message.  The reference throws
 * std::runtime_error in the same situations; the C++ drop-in header
 * (dimgpu_reference_shim.hpp) turns a non-zero status back into that throw.
 *
 * Threading: a session is not thread-safe; distinct sessions may be used from
 * distinct host threads.  All device work of a session is ordered on the
 * session's CUDA stream.
 */
#ifndef DIMGPU_H
#define DIMGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DIMGPU_MAX_MATERIALS 4

/* Status codes. */
enum {
    DIMGPU_OK = 0,
    DIMGPU_E_INVALID_ARG = 1,     /* bad sizes, dt_max <= 0, cfl <= 0, gamma <= 1, ... */
    DIMGPU_E_UNSUPPORTED_EOS = 2, /* an EoS kind other than ideal / stiffened gas      */
    DIMGPU_E_NONFINITE = 3,       /* a non-finite or non-positive time step             */
    DIMGPU_E_TIMEOUT = 4,         /* a bounded device-side wait ran out                 */
    DIMGPU_E_OOM = 5,             /* device allocation failed / admission refused       */
    DIMGPU_E_CUDA = 6,            /* any other CUDA runtime error                       */
    DIMGPU_E_UNSUPPORTED = 7      /* valid option that this build does not implement    */
};

/* EoS kinds: same numbering as the reference's EOSKind
 * (src/euler/eos_params.hpp:8-15).  Only the first two run on the GPU. */
enum {
    DIMGPU_EOS_IDEAL_GAS = 0,
    DIMGPU_EOS_STIFFENED_GAS = 1,
    DIMGPU_EOS_NOBLE_ABEL = 2,
    DIMGPU_EOS_PENG_ROBINSON = 3,
    DIMGPU_EOS_TAIT = 4,
    DIMGPU_EOS_MIE_GRUNEISEN = 5
};

/* Boundary kinds (Config::bc_lo / bc_hi strings, src/io/config.hpp:131-132).
 * Any name other than "reflective" / "nonreflective" behaves as transmissive
 * in the reference (src/dim/solver/advance/boundary.hpp:201-224). */
enum {
    DIMGPU_BC_TRANSMISSIVE = 0,
    DIMGPU_BC_REFLECTIVE = 1,
    DIMGPU_BC_NONREFLECTIVE = 2
};

/* Config::dim_lambda_model (src/io/config.hpp:124). */
enum {
    DIMGPU_LAMBDA_KAPILA = 0,
    DIMGPU_LAMBDA_ALLAIRE = 1,
    DIMGPU_LAMBDA_EQUAL_VELOCITY = 2
};

/* Arithmetic of the step. */
enum {
    DIMGPU_PRECISION_FP64 = 0,  /* bit-faithful to the reference's double run        */
    DIMGPU_PRECISION_MIXED = 1, /* FP32 reconstruction + HLLC, FP64 state/EoS/dt      */
    DIMGPU_PRECISION_MIXED_FP64 = 2  /* the mixed form's algorithm with its FP32 quantities
                                      * in FP64: (MIXED - this) is the cost of FP32 alone,
                                      * (this - FP64) the cost of the algorithm's shortcuts */
};

/* Sweep schedules (results are identical; speed differs by grid shape). */
enum {
    DIMGPU_SCHEDULE_FUSED = 0,   /* one kernel: all stages in a shared-memory tile      */
    DIMGPU_SCHEDULE_STAGED = 1   /* one kernel per stage, intermediates in HBM scratch   */
};

/* Config::time_update (src/io/config.hpp:112). */
enum {
    DIMGPU_TIME_SPLIT = 0,
    DIMGPU_TIME_UNSPLIT = 1
};

/* Which step a session runs. */
enum {
    DIMGPU_MODEL_DIM = 0,   /* dim::advance_one_step (src/dim/solver/advance_step.hpp:29) */
    DIMGPU_MODEL_EULER = 1  /* the single-material Euler step: advance_one_step<DIM, EOS>
                             * (src/sim/solver/advance_step.hpp:489) with one material
                             * and no level set; nmat = 1, V = 2 + DIM components
                             * (rho, mom[0..DIM-1], E: Conserved<DIM>,
                             * src/euler/state.hpp:8-12), every axis N >= 3 */
};

/* One material: the fields of ::EOSParams that the ideal and stiffened-gas
 * laws read (src/euler/eos_params.hpp:46-53). */
typedef struct dimgpu_material {
    int kind;
    double gamma;
    double p_inf;
} dimgpu_material;

/* Everything the reference's step reads from N, dx, dim::EOSParams and
 * Config<DIM> (src/dim/solver/advance_step.hpp:28-37). */
typedef struct dimgpu_desc {
    int dim;                        /* 1, 2 or 3                                  */
    int N[3];                       /* cells per axis; unused axes must be 1      */
    double dx[3];                   /* spacing per axis                           */
    int nmat;                       /* 1 .. DIMGPU_MAX_MATERIALS                  */
    dimgpu_material mat[DIMGPU_MAX_MATERIALS];
    int bc_lo[3];                   /* DIMGPU_BC_* per axis                       */
    int bc_hi[3];
    int lambda_model;               /* DIMGPU_LAMBDA_*                            */
    double alpha_source_floor;      /* Config::dim_alpha_source_floor             */
    int precision;                  /* DIMGPU_PRECISION_*                         */
    int time_update;                /* DIMGPU_TIME_*                              */
    int model;                      /* DIMGPU_MODEL_* (0: DIM)                    */
} dimgpu_desc;

/* Per-call phase timings, the device-side counterpart of SolverPhaseTimings
 * (src/core/phase_timings.hpp:4-12).  Milliseconds, from CUDA events. */
typedef struct dimgpu_phase_times {
    double cfl_ms;
    double sweep_ms;
    double boundary_ms;
} dimgpu_phase_times;

typedef struct dimgpu_session dimgpu_session;

/* Number of doubles per cell for a descriptor (2*nmat + dim). */
int dimgpu_components(const dimgpu_desc* desc);

/* Create a session: validates the descriptor (dim::EOSParams::validate,
 * src/dim/eos_params.hpp:16-28) and allocates the device-resident SoA state.
 * Unsupported EoS kinds give DIMGPU_E_UNSUPPORTED_EOS; there is no CPU path. */
int dimgpu_create(const dimgpu_desc* desc, dimgpu_session** out);

/* Free a session and all its device memory. */
int dimgpu_destroy(dimgpu_session* s);

/* Message of the last failing call on this session (or of the last failing
 * session-less call when s is NULL).  Never NULL. */
const char* dimgpu_last_error(const dimgpu_session* s);

/* Copy `count` doubles (must be V * ncell) from a host SoA buffer into the
 * session.  Replaces the caller's std::vector<dim::State<DIM>> argument of
 * dim::advance_one_step (src/dim/solver/advance_step.hpp:29-31). */
int dimgpu_upload(dimgpu_session* s, const double* soa, size_t count);

/* Copy the session state into a host SoA buffer of `count` doubles.
 * Replaces StepResult::U_new (src/dim/solver/advance_step.hpp:20-25, 147). */
int dimgpu_download(dimgpu_session* s, double* soa, size_t count);

/* One full time step on the resident state: CFL dt, then the split x, y, z
 * sweeps, each followed by the boundary fill.  Replaces
 * dim::advance_one_step (src/dim/solver/advance_step.hpp:29-149).
 * dt_out receives the step's dt; times may be NULL. */
int dimgpu_step(dimgpu_session* s, double cfl, double dt_max, double* dt_out,
                dimgpu_phase_times* times);

/* n consecutive steps with the same cfl and dt_max, no host synchronisation
 * between them (the CFL minimum of step k+1 is fused into step k's last
 * sweep).  dt_out (may be NULL) receives n doubles.  Equivalent to n calls of
 * dimgpu_step, i.e. to the time loop of run_dim_case with a constant dt_max
 * (src/app/solver/run_dim.hpp:88-111). */
int dimgpu_steps(dimgpu_session* s, int n, double cfl, double dt_max, double* dt_out);

/* Asynchronous form of dimgpu_steps: enqueue n steps on the session's stream
 * and return without waiting.  The dts stay on the device (at most 4096
 * enqueued steps between collections). */
int dimgpu_enqueue_steps(dimgpu_session* s, int n, double cfl, double dt_max);

/* Wait for the enqueued steps, copy their dts into dt_out (room for
 * `capacity` doubles; may be NULL), report how many in *count (may be NULL)
 * and return the first error any of them raised. */
int dimgpu_collect(dimgpu_session* s, double* dt_out, int capacity, int* count);

/* CFL time step of the resident state.  Replaces dim::compute_dt_cfl
 * (src/dim/solver/cfl.hpp:16-66) and, for DIMGPU_TIME_UNSPLIT sessions,
 * dim::compute_dt_cfl_unsplit (src/dim/solver/cfl.hpp:70-119). */
int dimgpu_compute_dt_cfl(dimgpu_session* s, double cfl, double dt_max, double* dt_out);

/* One split sweep along `dir` with time step dt, in place on the resident
 * state.  Replaces dim::sweep_direction_dispatch
 * (src/dim/solver/advance/sweep_core.hpp:151-202). */
int dimgpu_sweep_direction(dimgpu_session* s, int dir, double dt);

/* Boundary fill of the resident state.  Replaces
 * dim::apply_boundary_conditions (src/dim/solver/advance/boundary.hpp:165-226). */
int dimgpu_apply_boundary_conditions(dimgpu_session* s);

/* Conservation totals of the resident state: out receives nmat + dim + 2
 * doubles {material_mass[nmat], mass, momentum[dim], energy}, each the sum
 * over cells of the conserved variable times the cell volume.  Device
 * counterpart of compute_dim_conservation_totals
 * (src/app/io/conservation_report.hpp:188-218); the summation order differs,
 * so compare with a relative tolerance. */
int dimgpu_totals(dimgpu_session* s, double* out);

/* Boundary flux integrand of the resident state, the rate the conservation
 * report integrates over time: per axis and transverse line,
 * area * (F(last cell) - F(first cell)) with each end cell's own normal
 * flux.  out receives nmat + dim + 2 values laid out as dimgpu_totals.
 * Replaces app_io::compute_dim_boundary_flux
 * (src/app/io/conservation_report.hpp:253-305); the DIM model only. */
int dimgpu_boundary_flux(dimgpu_session* s, double* out);

/* Run the session's work on a caller-owned CUDA stream (a cudaStream_t cast
 * to void*; NULL restores the session's own stream).  The caller keeps the
 * stream alive while the session uses it. */
int dimgpu_set_stream(dimgpu_session* s, void* cuda_stream);

/* Tile shape of the sweep kernel along axis `dir`: T cells per line segment
 * (T - 6 of them are written, 6 are stencil halo) times W lines per CTA,
 * 8 <= T, T * W <= 256.  Results do not depend on the tile shape. */
int dimgpu_set_tile(dimgpu_session* s, int dir, int T, int W);

/* Sweep schedule along axis `dir` (DIMGPU_SCHEDULE_*).  The staged schedule
 * allocates its scratch (about 60 doubles per cell, at most 2^24 cells per
 * chunk) on first use. */
int dimgpu_set_schedule(dimgpu_session* s, int dir, int schedule);

/* Kernel timing: when enabled, every kernel the session launches is
 * bracketed by CUDA events on its stream.  dimgpu_profile_read synchronises
 * and writes {total_ms, launches} for the kinds sweep, cfl, boundary, other
 * (8 doubles), accumulated since profiling was last enabled. */
int dimgpu_profile(dimgpu_session* s, int enable);
int dimgpu_profile_read(dimgpu_session* s, double* out8);

/* Kernels this library has launched in the process so far (all sessions and
 * batches; a batch step replayed from a CUDA graph counts the kernels the
 * graph holds for it).  The difference of two reads brackets a region. */
long long dimgpu_kernel_launches(void);

/* CFL time step of a state that the caller keeps in its own device memory,
 * computed without allocating anything.  No counterpart in the reference: it
 * serves callers that own all device memory themselves (a serving process
 * holding the HBM budget for resident solves, a solver handing out buffers
 * from its own pool) and so cannot let a library call cudaMalloc — which may
 * fail for lack of memory and which synchronises the device — mid time loop.
 *
 * d_state: device pointer to the SoA state (layout above); the result is
 * written to the host double *dt_out; work runs on `cuda_stream` (a
 * cudaStream_t cast to void*, NULL for the default stream) and the call
 * returns once dt is on the host.  Same value as dimgpu_compute_dt_cfl, and
 * the same descriptor checks.  One difference: for the Euler model a
 * non-finite density returns DIMGPU_E_NONFINITE here (the reference's
 * compute_dt_cfl_materials throws there), where dimgpu_compute_dt_cfl
 * returns the dt and leaves the decision to the step that follows.
 *
 * Limits: at most 4 194 304 cells (larger grids return DIMGPU_E_INVALID_ARG
 * before any device work).  The scratch is one 128 KB array per GPU, static
 * to the library and kept until the process exits; the first call on a
 * device looks up its address and should come before any stream capture.
 * All calls share that array, so calls that overlap on the GPU race. */
int dimgpu_compute_dt_cfl_noalloc(const dimgpu_desc* desc, const double* d_state, double cfl,
                                  double dt_max, double* dt_out, void* cuda_stream);

/* Stateless drop-in for one call of dim::advance_one_step
 * (src/dim/solver/advance_step.hpp:29-149): host SoA in, host SoA out.
 * Uses a cached session per descriptor shape; the copies are part of the call. */
int dimgpu_advance_one_step(const dimgpu_desc* desc, const double* soa_in, double* soa_out,
                            double cfl, double dt_max, double* dt_out,
                            dimgpu_phase_times* times);

/* ---- batched form ------------------------------------------------------
 * Many independent grids (one material count and dimension per batch; each
 * with its own N, dx, materials, boundaries, cfl, dt_max and step budget)
 * advanced together: one set of persistent-grid launches per step for every
 * instance, replayed from a captured CUDA graph.  Each instance's results are
 * exactly those of a dimgpu_session run of the same grid.  Split steps, FP64,
 * N = 1 or N >= 4 on every axis.  No counterpart in the reference, which
 * runs one grid per process (src/app/solver/run_dim.hpp:20-178). */
typedef struct dimgpu_batch dimgpu_batch;

int dimgpu_batch_create(int nmat, int dim, dimgpu_batch** out);
int dimgpu_batch_destroy(dimgpu_batch* b);
const char* dimgpu_batch_last_error(const dimgpu_batch* b);

/* Add an instance: copies `soa` (V * ncell doubles) to the device; the
 * instance will run `steps` steps.  *id identifies it afterwards. */
int dimgpu_batch_add(dimgpu_batch* b, const dimgpu_desc* desc, const double* soa, int steps,
                     double cfl, double dt_max, int* id);

/* Remove an instance and free its device memory. */
int dimgpu_batch_remove(dimgpu_batch* b, int id);

/* Advance every instance that has steps left by up to n steps. */
int dimgpu_batch_run(dimgpu_batch* b, int n);

/* Steps run / left of an instance (no device synchronisation). */
int dimgpu_batch_status(dimgpu_batch* b, int id, int* steps_done, int* steps_left);

/* State of an instance (count = V * ncell) and, if dts is not NULL, the dt
 * of every step it has run. */
int dimgpu_batch_download(dimgpu_batch* b, int id, double* soa, size_t count, double* dts);

/* Persistent grid size in CTAs (0: 4 per SM). */
int dimgpu_batch_set_grid(dimgpu_batch* b, int ctas);

/* Number of instances in the batch. */
int dimgpu_batch_size(const dimgpu_batch* b);

/* Run the batch's work on a caller-owned CUDA stream (NULL: its own). */
int dimgpu_batch_set_stream(dimgpu_batch* b, void* cuda_stream);

/* Arena mode, for hosts that admit and retire solves continuously: reserve
 * once, on a new batch, device memory for at most `max_cells` cells over all
 * resident instances, `max_instances` instances and `max_steps` logged time
 * steps.  Afterwards dimgpu_batch_add and _remove allocate, free and
 * synchronise nothing (ranges of the reserved memory; the initial state is
 * copied asynchronously on the batch's stream), a full arena returns
 * DIMGPU_E_OOM, and the captured step graph stays valid across every join
 * and leave. */
int dimgpu_batch_reserve(dimgpu_batch* b, long long max_cells, int max_instances, long long max_steps);

/* Cells and dt-log entries of the arena in use. */
int dimgpu_batch_arena_used(const dimgpu_batch* b, long long* cells, long long* dt_entries);

/* dimgpu_batch_run without the wait: enqueue up to n steps of every instance
 * with steps left on the batch's stream and return.  dimgpu_batch_wait waits
 * for them and reports a non-finite state or time step of any of them. */
int dimgpu_batch_enqueue(dimgpu_batch* b, int n);
int dimgpu_batch_wait(dimgpu_batch* b);

/* ---- one grid over several GPUs --------------------------------------------
 * Slab decomposition of one DIM grid along its slowest axis (y in 2D, z in
 * 3D), one slab per listed device, driven from one process; replaces the
 * reference's MPI slab driver (src/app/dim_mpi_main.cpp:116-124 slabs,
 * :383-423 halo exchange, :758 MPI_Allreduce of dt).  Each slab holds three
 * ghost planes per internal cut (the split sweep's reach), refreshed by
 * device or peer copies before every sweep along the split axis, and dt is
 * the minimum over the slabs' owned cells: results are bit-identical to one
 * session on the whole grid.  `devices` may repeat a device (several slabs
 * on one GPU).  Split steps of the DIM model, 2D and 3D, at least three
 * planes per slab. */
typedef struct dimgpu_slabs dimgpu_slabs;

int dimgpu_slabs_create(const dimgpu_desc* desc, int nslabs, const int* devices, dimgpu_slabs** out);
int dimgpu_slabs_destroy(dimgpu_slabs* L);
const char* dimgpu_slabs_last_error(const dimgpu_slabs* L);
/* Whole-grid SoA state in (count = V * ncell of the whole grid). */
int dimgpu_slabs_upload(dimgpu_slabs* L, const double* soa, size_t count);
/* One time step of the whole grid (dim::advance_one_step); dt_out may be NULL. */
int dimgpu_slabs_step(dimgpu_slabs* L, double cfl, double dt_max, double* dt_out);
/* Whole-grid SoA state out, gathered from the slabs' owned planes. */
int dimgpu_slabs_download(dimgpu_slabs* L, double* soa, size_t count);

/* ---- the serving loop ----------------------------------------------------
 * Continuous batching of DIM solve requests.  No counterpart in the
 * reference, which runs one case per process (run_dim_case,
 * src/app/solver/run_dim.hpp:20-178).  Requests are submitted from any host
 * thread and queue in arrival order.  A server thread drives lanes, each on
 * its own stream: batch lanes (one per material count and dimension, an
 * arena batch reserved once from the budget, dimgpu_batch_reserve) for
 * small solves, and solo lanes (session shells over one reserved arena) for
 * solves of at least solo_min_cells cells, which fill the GPU alone and run
 * fastest as one grid.  Admission is first come first served per lane kind
 * and group and allocates and synchronises nothing.  Each lane advances its
 * solves a quantum at a time; when a lane's quantum ends (an event query)
 * it retires its finished solves, takes queued ones and starts its next
 * quantum while the other lanes run on.  A result is exactly the single-grid
 * step's. */
typedef struct dimgpu_server dimgpu_server;

typedef struct dimgpu_server_config {
    double hbm_budget_bytes;   /* device memory for resident solves (states + step scratch) */
    double dim_share[3];       /* fraction of the budget for 1D, 2D and 3D solves (sum <= 1) */
    int max_slots;             /* resident solves at most */
    int quantum;               /* steps per scheduling round */
    int max_steps_per_solve;   /* largest step budget a request may ask for */
    long long solo_min_cells;  /* solves of at least this many cells run alone on a solo lane (0: never) */
    double solo_share;         /* fraction of the budget for solo solves (sum with dim_share <= 1) */
    int solo_slots;            /* solo lanes (solves resident alone at once); 0: none */
} dimgpu_server_config;

enum {
    DIMGPU_REQ_QUEUED = 0,
    DIMGPU_REQ_RUNNING = 1,
    DIMGPU_REQ_DONE = 2,
    DIMGPU_REQ_CANCELLED = 3,
    DIMGPU_REQ_FAILED = 4
};

typedef struct dimgpu_server_counters {
    long long submitted, completed, cancelled, failed, quanta, queued;
    int resident, peak_resident;
    double peak_bytes;
} dimgpu_server_counters;

int dimgpu_server_create(const dimgpu_server_config* cfg, dimgpu_server** out);
int dimgpu_server_destroy(dimgpu_server* s);
const char* dimgpu_server_last_error(const dimgpu_server* s);

/* Queue a solve: the state (V * ncell doubles) is copied, so the caller's
 * buffer is free on return.  A solve larger than its dimension's share of
 * the budget returns DIMGPU_E_OOM. */
int dimgpu_server_submit(dimgpu_server* s, const dimgpu_desc* desc, const double* soa, int steps,
                         double cfl, double dt_max, long long* request_id);

/* State of a request (DIMGPU_REQ_*).  For a finished request, latency_s is
 * the time from submission to completion; with soa_out (count = V * ncell)
 * the result and, if dts_out is not NULL, the dt of every step are copied
 * out and the request is collected (forgotten).  A failed request returns
 * DIMGPU_E_NONFINITE with its message and is collected. */
int dimgpu_server_poll(dimgpu_server* s, long long request_id, int* state, double* soa_out, size_t count,
                       double* dts_out, double* latency_s);

/* Drop a queued or resident request; its room is freed at the next round. */
int dimgpu_server_cancel(dimgpu_server* s, long long request_id);

/* Wait until no request is queued or resident. */
int dimgpu_server_drain(dimgpu_server* s);

int dimgpu_server_stats(dimgpu_server* s, dimgpu_server_counters* out);

/* ---- initial fields generated on the device ------------------------------
 * The reference builds its initial field on the host cell by cell
 * (initialise_dim_from_config, src/setup/dim_initial_conditions.hpp:608-628)
 * with the tanh indicator 0.5 (1 - tanh(a s / thickness)) (smooth_indicator,
 * :224-236) across diffuse interfaces.  These entry points write the two
 * benchmark fields straight into a session's device state, so a 512^3 field
 * (7.5 GB) is never built on the host or copied.  The tanh is the library's
 * own (IEEE +, -, *, / and exact scaling), and the host generator in
 * diffuse_vs_gfm_mms_b200/workloads.py uses the same arithmetic: both give the
 * same bits. */

/* Shock-bubble (2D, two materials): material 1 in the disc of `radius`
 * around `center`, smeared by the indicator with `thickness` and
 * `sharpness`, its fraction set to 0 where the indicator is <= zero_below;
 * material 0 elsewhere, at (rho_post, u_post along x, p_post) for cell
 * centres x < shock_x and (rho_pre, at rest, p_pre) beyond.  Velocity and
 * pressure are the fraction-weighted mixes; the bubble is at rest at
 * (rho_bubble, p_bubble). */
typedef struct dimgpu_ic_shock_bubble {
    double center[2];
    double radius;
    double thickness;
    double sharpness;
    double shock_x;
    double zero_below;
    double rho_post, u_post, p_post;
    double rho_pre, p_pre;
    double rho_bubble, p_bubble;
} dimgpu_ic_shock_bubble;

int dimgpu_init_shock_bubble(dimgpu_session* s, const dimgpu_ic_shock_bubble* ic);

/* Bubble cloud (3D, two materials): material 1 (gas, density rho_gas) in
 * spheres; each sphere's indicator is evaluated in its box of cells
 * [box_lo, box_hi) only, and a cell's gas fraction is the largest of them (0
 * where <= zero_below); material 0 (liquid, rho_liquid) elsewhere; at rest,
 * pressure p_pulse for cell centres x < pulse_width and p_ambient beyond. */
typedef struct dimgpu_ic_bubble {
    double center[3];
    double radius;
    int box_lo[3];
    int box_hi[3];
} dimgpu_ic_bubble;

typedef struct dimgpu_ic_bubble_cloud {
    double thickness;
    double sharpness;
    double zero_below;
    double pulse_width;
    double rho_liquid, rho_gas;
    double p_ambient, p_pulse;
} dimgpu_ic_bubble_cloud;

int dimgpu_init_bubble_cloud(dimgpu_session* s, const dimgpu_ic_bubble_cloud* ic,
                             const dimgpu_ic_bubble* bubbles, int nbubbles);

/* ---- asynchronous CSV snapshot -------------------------------------------
 * Writes the session's current state as dim::write_csv does
 * (src/io/dim_write_csv.hpp:15-125): same header, one row per cell in linear
 * order, values printed as std::ostream prints a double ("%.6g"), cell
 * centres domain_min + (i + 0.5) (domain_max - domain_min) / N.  The call
 * copies the state into a device snapshot (ordered after the session's
 * pending work; the session's later work waits for the copy only) and
 * returns; a host thread then streams the per-cell values from the device
 * in chunks and formats them with `threads` threads (0: all cores) while the
 * session keeps stepping.  dimgpu_csv_wait joins the writer, frees it and
 * returns its status.  DIM model only. */
typedef struct dimgpu_csv_writer dimgpu_csv_writer;

int dimgpu_csv_write_async(dimgpu_session* s, const char* filename, const double* domain_min,
                           const double* domain_max, int threads, dimgpu_csv_writer** out);
int dimgpu_csv_wait(dimgpu_csv_writer* w);

#ifdef __cplusplus
}
#endif

#endif /* DIMGPU_H */
