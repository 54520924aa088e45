// Kernel instantiations for 2 material(s), all dimensions (compiled in
// parallel with the other material counts).
#include "dim_batch.cuh"
#include "dim_kernels.cuh"

namespace dimgpu {
DIMGPU_INSTANTIATE(2)
DIMGPU_INSTANTIATE_BATCH(2)
}  // namespace dimgpu
