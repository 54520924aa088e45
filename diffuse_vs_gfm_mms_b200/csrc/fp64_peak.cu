// fp64_peak.cu — the FP64 throughput the sweep kernels are measured against
// (libdimprobe.so, loaded by bench.py only; not part of the C-ABI).
//
// Every thread runs kChains independent DFMA dependency chains for `iters`
// iterations, so the FP64 pipe never waits on a result: the kernel's rate is
// the pipe's issue limit.  A grid of 8 blocks of 256 threads per SM keeps
// every SM's schedulers busy.  The chains' results feed one conditional
// store, so the compiler cannot drop the arithmetic.
#include <cuda_runtime.h>

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) dfma_loop(double a, double b, int iters, double* __restrict__ sink)
{
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = 1.0 + 1e-3 * (threadIdx.x + c);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = __fma_rn(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 12345.678) sink[blockIdx.x] = s;  // never true for the inputs bench.py passes
}

}  // namespace

// Runs the loop `repeats` times after one warm-up launch and returns the best
// rate: DFMA thread instructions per second in *dfma_per_s and FP64 FLOP/s
// (2 per DFMA) in *flops.  Returns 0, or the CUDA error code.
extern "C" int dimprobe_fp64_peak(int repeats, double* dfma_per_s, double* flops)
{
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 8, threads = 256, iters = 4096;
    double* sink = nullptr;
    cudaError_t e = cudaMalloc(&sink, blocks * sizeof(double));
    if (e != cudaSuccess) return (int)e;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    double best = 0.0;
    dfma_loop<<<blocks, threads>>>(0.999999, 1e-7, iters, sink);
    for (int r = 0; r < repeats && e == cudaSuccess; ++r) {
        cudaEventRecord(t0);
        dfma_loop<<<blocks, threads>>>(0.999999, 1e-7, iters, sink);
        cudaEventRecord(t1);
        e = cudaEventSynchronize(t1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        const double n = (double)blocks * threads * kChains * iters;
        if (ms > 0.f && n / (ms * 1e-3) > best) best = n / (ms * 1e-3);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(sink);
    *dfma_per_s = best;
    *flops = 2.0 * best;
    return (int)e;
}
