// 3D, FP64, Euler: instantiation of the DGSEM kernels.
#include "dgsem_impl.cuh"

namespace prandtl {
PRANDTL_INSTANTIATE_RHS(3, double, false, false)
}   // namespace prandtl
