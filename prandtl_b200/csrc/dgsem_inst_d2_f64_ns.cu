// 2D, FP64, Navier-Stokes: instantiation of the DGSEM kernels.
#include "dgsem_impl.cuh"

namespace prandtl {
PRANDTL_INSTANTIATE_RHS(2, double, true)
PRANDTL_INSTANTIATE_LIFT(2, double)
}   // namespace prandtl
