// 2D, FP32-bulk, Navier-Stokes with contravariant viscous fluxes: instantiation of the DGSEM kernels.
#include "dgsem_impl.cuh"

namespace prandtl {
PRANDTL_INSTANTIATE_RHS(2, float, true, true)
PRANDTL_INSTANTIATE_LIFT(2, float, true)
}   // namespace prandtl
