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
    unsigned long long* cfl_slot = nullptr;  // fused CFL minimum (bit pattern of a double)
    long long staged_cap = 0;
    std::string msg;
    // profiling
    bool profiling = false;
    struct Rec { int kind; cudaEvent_t a, b; };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    double prof[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int pending = 0;  // steps enqueued since the last collection
};

namespace dimgpu {

// Records a failure on the session (or, with s == NULL, on the calling
// thread) and returns the status.
int session_fail(dimgpu_session* s, int code, const std::string& msg);
int session_cuda_fail(dimgpu_session* s, cudaError_t e, const char* what);

}  // namespace dimgpu
