// 3D, FP32-bulk, Navier-Stokes: instantiation of the DGSEM kernels.
#include "dgsem_impl.cuh"

namespace prandtl {
PRANDTL_INSTANTIATE_RHS(3, float, true)
PRANDTL_INSTANTIATE_LIFT(3, float)
}   // namespace prandtl
