// dimgpu_noalloc.cu — a CFL time-step entry point that allocates nothing.
//
// Who needs it: host programs that own every byte of device memory
// themselves — a serving process that reserves the HBM budget for resident
// solves up front, or a solver that hands out device buffers from its own
// pool — cannot let a library call cudaMalloc in the middle of a time loop:
// the memory may simply not be there, and cudaMalloc / cudaFree synchronise
// the device, stalling every other solve on it.  Such a caller keeps its
// state on the device and asks only for the step size.
//
// How: the CFL kernel's per-block minima, the final dt and the error flag
// live in one file-scope __device__ array (kScratchDoubles doubles, 128 KB
// per GPU that loads this library, held until the process exits).  One block
// of 256 cells writes one partial, so the grid may hold at most
// kScratchSlots * 256 = 4 194 304 cells; larger grids are refused before any
// device work.  Host code needs the array's device address, which
// cudaGetSymbolAddress gives once per device on the first call made with that
// device current; that first call should therefore come before any stream
// capture.  Every call reuses the same array: the error flag is cleared at
// the start of each call, and calls that overlap on the GPU (two host
// threads, or two streams, using the same device at once) race on it.
#include <cstring>
#include <mutex>
#include <string>

#include "dim_launch.h"
#include "dimgpu.h"
#include "dimgpu_validate.h"

using namespace dimgpu;

namespace {

constexpr int kScratchSlots = 16384;            // per-block CFL minima
constexpr int kScratchDoubles = kScratchSlots + 2;  // + dt + error flag
constexpr long long kMaxCells = (long long)kScratchSlots * 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Failures are reported through dimgpu_last_error(NULL), like every other
// session-less call.
int noalloc_fail(int code, const std::string& msg)
{
    set_sessionless_error(msg);
    return code;
}

// Device address of the scratch array for the current device (set-up on the
// first call per device).
int scratch_for_current_device(double** out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(DIMGPU_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(DIMGPU_E_UNSUPPORTED, "device index beyond 63");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return noalloc_fail(DIMGPU_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return DIMGPU_OK;
}

}  // namespace

extern "C" int dimgpu_compute_dt_cfl_noalloc(const dimgpu_desc* desc, const double* d_state, double cfl,
                                             double dt_max, double* dt_out, void* cuda_stream)
{
    if (!desc || !d_state || !dt_out) return noalloc_fail(DIMGPU_E_INVALID_ARG, "null argument");
    {
        std::string msg;
        const int rc = check_desc(desc, &msg);
        if (rc) return noalloc_fail(rc, msg);
    }
    // The cell count is checked against the limit axis by axis, so the
    // product never grows past kMaxCells * INT_MAX (no signed overflow).
    long long ncell = 1;
    for (int a = 0; a < 3; ++a) {
        ncell *= desc->N[a];
        if (ncell > kMaxCells)
            return noalloc_fail(DIMGPU_E_INVALID_ARG,
                                "grid " + std::to_string(desc->N[0]) + " x " + std::to_string(desc->N[1]) + " x " +
                                    std::to_string(desc->N[2]) + " exceeds the allocation-free limit of " +
                                    std::to_string(kMaxCells) + " cells");
    }
    if (!(cfl > 0.0)) return noalloc_fail(DIMGPU_E_INVALID_ARG, "cfl must be positive");
    if (!(dt_max > 0.0)) return noalloc_fail(DIMGPU_E_INVALID_ARG, "dt_max must be positive");

    double* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    double* blockmin = scratch;
    double* dt_dev = scratch + kScratchSlots;
    int* err = reinterpret_cast<int*>(scratch + kScratchSlots + 1);

    Mats M;
    int kind[kMaxMat];
    double gam[kMaxMat], pinf[kMaxMat];
    for (int k = 0; k < desc->nmat; ++k) {
        kind[k] = desc->mat[k].kind;
        gam[k] = desc->mat[k].gamma;
        pinf[k] = desc->mat[k].p_inf;
    }
    fill_mats(M, desc->nmat, kind, gam, pinf, desc->lambda_model, desc->alpha_source_floor);
    Grid g;
    std::memset(&g, 0, sizeof g);
    for (int a = 0; a < 3; ++a) {
        g.N[a] = desc->N[a];
        g.dx[a] = desc->dx[a];
        g.bc_lo[a] = desc->bc_lo[a];
        g.bc_hi[a] = desc->bc_hi[a];
    }
    g.ncell = ncell;
    g.stride[0] = 1;
    g.stride[1] = desc->N[0];
    g.stride[2] = (long long)desc->N[0] * desc->N[1];

    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), s);
    int nb = 1;
    const bool unsplit = desc->time_update == DIMGPU_TIME_UNSPLIT;
    if (e == cudaSuccess && desc->model == DIMGPU_MODEL_EULER) {
        switch (desc->dim) {
            case 1: e = launch_euler_cfl<1>(g, M, d_state, cfl, unsplit, blockmin, kScratchSlots, &nb, err, s); break;
            case 2: e = launch_euler_cfl<2>(g, M, d_state, cfl, unsplit, blockmin, kScratchSlots, &nb, err, s); break;
            case 3: e = launch_euler_cfl<3>(g, M, d_state, cfl, unsplit, blockmin, kScratchSlots, &nb, err, s); break;
            default: e = cudaErrorInvalidValue; break;
        }
    }
    else if (e == cudaSuccess) {
        switch (desc->nmat * 10 + desc->dim) {
#define NOALLOC_CASE(NM, D) \
            case NM * 10 + D: e = launch_cfl<NM, D>(g, M, d_state, cfl, unsplit, blockmin, kScratchSlots, &nb, s, \
                                                    desc->precision != DIMGPU_PRECISION_FP64); break;
            NOALLOC_CASE(1, 1) NOALLOC_CASE(1, 2) NOALLOC_CASE(1, 3)
            NOALLOC_CASE(2, 1) NOALLOC_CASE(2, 2) NOALLOC_CASE(2, 3)
            NOALLOC_CASE(3, 1) NOALLOC_CASE(3, 2) NOALLOC_CASE(3, 3)
            NOALLOC_CASE(4, 1) NOALLOC_CASE(4, 2) NOALLOC_CASE(4, 3)
#undef NOALLOC_CASE
            default: e = cudaErrorInvalidValue; break;
        }
    }
    if (e == cudaSuccess) e = launch_cfl_finalize(blockmin, nb, dt_max, dt_dev, nullptr, err, s);
    double dt_and_flag[2] = {0.0, 0.0};  // dt, then the error-flag slot
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt_and_flag, dt_dev, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return noalloc_fail(DIMGPU_E_CUDA, std::string("dimgpu_compute_dt_cfl_noalloc: ") +
                                                                 cudaGetErrorString(e));
    int flag = 0;
    std::memcpy(&flag, &dt_and_flag[1], sizeof flag);
    if (desc->model == DIMGPU_MODEL_EULER && (flag & kErrNonFinite))
        return noalloc_fail(DIMGPU_E_NONFINITE, "thermo: invalid density (non-finite)");
    *dt_out = dt_and_flag[0];
    return DIMGPU_OK;
}
