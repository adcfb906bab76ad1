// 3D, FP64, Navier-Stokes with contravariant viscous fluxes: instantiation of the DGSEM kernels.
#include "dgsem_impl.cuh"

namespace prandtl {
PRANDTL_INSTANTIATE_RHS(3, double, true, true)
PRANDTL_INSTANTIATE_LIFT(3, double, true)
}   // namespace prandtl
