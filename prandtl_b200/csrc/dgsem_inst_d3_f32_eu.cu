// 3D, FP32-bulk, Euler: instantiation of the DGSEM kernels.
#include "dgsem_impl.cuh"

namespace prandtl {
PRANDTL_INSTANTIATE_RHS(3, float, false, false)
}   // namespace prandtl
