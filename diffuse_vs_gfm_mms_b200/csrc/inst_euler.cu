// Kernel instantiations of the single-material Euler step, all dimensions.
#include "euler_kernels.cuh"

namespace dimgpu {
DIMGPU_INSTANTIATE_EULER(1)
DIMGPU_INSTANTIATE_EULER(2)
DIMGPU_INSTANTIATE_EULER(3)
}  // namespace dimgpu
