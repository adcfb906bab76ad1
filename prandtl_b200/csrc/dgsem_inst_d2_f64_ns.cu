// 2D, FP64, Navier-Stokes with lifted gradients (reference defects reproduced): instantiation of the DGSEM kernels.
#include "dgsem_impl.cuh"

namespace prandtl {
PRANDTL_INSTANTIATE_RHS(2, double, true, false)
PRANDTL_INSTANTIATE_LIFT(2, double, false)
}   // namespace prandtl
