// Kernel instantiations for 4 material(s), all dimensions (compiled in
// parallel with the other material counts).
#include "dim_batch.cuh"
#include "dim_kernels.cuh"

namespace dimgpu {
DIMGPU_INSTANTIATE(4)
DIMGPU_INSTANTIATE_BATCH(4)
}  // namespace dimgpu
