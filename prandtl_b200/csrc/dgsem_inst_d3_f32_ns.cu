// 3D, FP32-bulk, Navier-Stokes with lifted gradients (reference defects reproduced): instantiation of the DGSEM kernels.
#include "dgsem_impl.cuh"

namespace prandtl {
PRANDTL_INSTANTIATE_RHS(3, float, true, false)
PRANDTL_INSTANTIATE_LIFT(3, float, false)
}   // namespace prandtl
