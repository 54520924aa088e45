// dimgpu_session.h — the session record behind the opaque dimgpu_session
// handle of include/dimgpu.h (internal; shared by the translation units that
// implement session entry points).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "dim_launch.h"
#include "dimgpu.h"

struct dimgpu_session {
    dimgpu_desc desc{};
    dimgpu::Mats M{};
    dimgpu::Grid g{};
    int V = 0;
    long long ncell = 0;
    double* buf[3] = {nullptr, nullptr, nullptr};
    int cur = 0;
    double* blockmin = nullptr;
    double* dt = nullptr;
    double* hist = nullptr;
    double* partial = nullptr;
    int* err = nullptr;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    dimgpu::Tile tile[3] = {{128, 1}, {64, 4}, {64, 4}};
    int schedule[3] = {DIMGPU_SCHEDULE_STAGED, DIMGPU_SCHEDULE_STAGED, DIMGPU_SCHEDULE_STAGED};
    double* staged = nullptr;  // scratch of the staged schedule (allocated on first use)
    unsigned long long* cfl_slot = nullptr;  // fused CFL: [0] minimum (a double's bits), [1] block ticket counter
    long long staged_cap = 0;
    std::string msg;
    // profiling
    bool profiling = false;
    struct Rec { int kind; cudaEvent_t a, b; };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    double prof[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int pending = 0;  // steps enqueued since the last collection
    bool borrowed = false;  // buf[] and staged point into a caller's arena (a shell)
};

namespace dimgpu {

// Records a failure on the session (or, with s == NULL, on the calling
// thread) and returns the status.
int session_fail(dimgpu_session* s, int code, const std::string& msg);
int session_cuda_fail(dimgpu_session* s, cudaError_t e, const char* what);

// Stream-ordered session operations without a host synchronisation (the
// slab solver drives several sessions at once with them):
//  * min(dt_max, CFL minimum over cells [begin, end) of the current state)
//    into s->dt;
//  * one sweep along `dir` with the dt held in s->dt on the device (the
//    current buffer flips);
//  * the boundary fill of the current state.
cudaError_t session_cfl_range(dimgpu_session* s, double cfl, double dt_max, long long begin, long long end);
cudaError_t session_sweep(dimgpu_session* s, int dir);
cudaError_t session_bc(dimgpu_session* s);
// Waits for the session's stream and turns its error flag into a status.
int session_check(dimgpu_session* s);

// Session shells (the serving loop's solo slots): a session with its stream
// and small device buffers but no grid memory; binding gives it a grid whose
// state buffers and staged scratch are a caller-owned device range of
// session_grid_doubles(desc) doubles, so a request is admitted without an
// allocation or a synchronisation.  Binding validates the descriptor.
long long session_grid_doubles(const dimgpu_desc* desc);
int session_shell_create(dimgpu_session** out);
int session_shell_bind(dimgpu_session* s, const dimgpu_desc* desc, double* mem);

}  // namespace dimgpu
