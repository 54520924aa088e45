// Kernel instantiations for 1 material(s), all dimensions (compiled in
// parallel with the other material counts).
#include "dim_batch.cuh"
#include "dim_kernels.cuh"

namespace dimgpu {
DIMGPU_INSTANTIATE(1)
DIMGPU_INSTANTIATE_BATCH(1)
}  // namespace dimgpu
