// fastdiv.h — division of unsigned 32-bit indices by a divisor fixed for a
// launch, through a multiply-high (host-testable: tests/native/physics_host.cpp).
#pragma once

#ifdef __CUDACC__
#define FASTDIV_HD __host__ __device__ __forceinline__
#else
#define FASTDIV_HD inline
#endif

namespace dimgpu {

// Unsigned 32-bit division by a divisor fixed for a launch: one
// multiply-high, a subtract, an add and two shifts in place of the integer
// division routine (Granlund & Montgomery, "Division by invariant integers
// using multiplication", PLDI 1994, the round-up method of their Figure
// 4.1: l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1,
// q = (t + ((x - t) >> min(l, 1))) >> max(l - 1, 0) with t = mulhi(m, x)).
// Exact for every x < 2^32 and 1 <= d < 2^32.
struct FastDiv {
    unsigned m;
    int s1, s2;
    void set(unsigned d)
    {
        int l = 0;
        while ((1ull << l) < d) ++l;
        m = (unsigned)((((1ull << l) - d) << 32) / d + 1);
        s1 = l < 1 ? l : 1;
        s2 = l > 1 ? l - 1 : 0;
    }
    FASTDIV_HD unsigned div(unsigned x) const
    {
#ifdef __CUDA_ARCH__
        const unsigned t = __umulhi(m, x);
#else
        const unsigned t = (unsigned)(((unsigned long long)m * x) >> 32);
#endif
        return (t + ((x - t) >> s1)) >> s2;
    }
};

}  // namespace dimgpu
