// Kernel instantiations for 3 material(s), all dimensions (compiled in
// parallel with the other material counts).
#include "dim_batch.cuh"
#include "dim_kernels.cuh"

namespace dimgpu {
DIMGPU_INSTANTIATE(3)
DIMGPU_INSTANTIATE_BATCH(3)
}  // namespace dimgpu
