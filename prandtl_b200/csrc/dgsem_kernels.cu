// dgsem_kernels.cu -- dispatch of the DGSEM kernels by dimension, working
// precision and physics to the dgsem_inst_*.cu translation units, and the
// batch step-end kernel.
#include "dgsem_kernels.cuh"

namespace prandtl {

bool order_supported(int dim, int order) {
    return (dim == 2 || dim == 3) && order >= 1 && order <= 5;
}

// Euler, Navier-Stokes with gradients, Navier-Stokes with contravariant viscous fluxes.
#define PRANDTL_DIM_PHYS(FN, REAL, NSV, VCV, ...)                                  \
    do {                                                                           \
        if (!(NSV)) {                                                              \
            if (dim == 2) return FN<2, REAL, false, false>(__VA_ARGS__);           \
            if (dim == 3) return FN<3, REAL, false, false>(__VA_ARGS__);           \
        } else if (VCV) {                                                          \
            if (dim == 2) return FN<2, REAL, true, true>(__VA_ARGS__);             \
            if (dim == 3) return FN<3, REAL, true, true>(__VA_ARGS__);             \
        } else {                                                                   \
            if (dim == 2) return FN<2, REAL, true, false>(__VA_ARGS__);            \
            if (dim == 3) return FN<3, REAL, true, false>(__VA_ARGS__);            \
        }                                                                          \
        return cudaErrorInvalidValue;                                              \
    } while (0)
#define PRANDTL_DIM_LIFT(FN, OUT, VCV, ...)                                        \
    do {                                                                           \
        if (VCV) {                                                                 \
            if (dim == 2) return FN<2, OUT, true>(__VA_ARGS__);                    \
            if (dim == 3) return FN<3, OUT, true>(__VA_ARGS__);                    \
        } else {                                                                   \
            if (dim == 2) return FN<2, OUT, false>(__VA_ARGS__);                   \
            if (dim == 3) return FN<3, OUT, false>(__VA_ARGS__);                   \
        }                                                                          \
        return cudaErrorInvalidValue;                                              \
    } while (0)

cudaError_t launch_rhs(int dim, int order, bool ns, const MeshDev &m, const RhsArgs &a,
                       const PhysParams &P, const OpTables &T, cudaStream_t s) {
    if (m.E <= 0) return cudaSuccess;
    PRANDTL_DIM_PHYS(rhs_dispatch, double, ns, use_vc(P), order, m, a, P, T, s);
}
cudaError_t launch_rhs_fp32(int dim, int order, bool ns, const MeshDev &m, const RhsArgs &a,
                            const PhysParams &P, const OpTables &T, cudaStream_t s) {
    if (m.E <= 0) return cudaSuccess;
    PRANDTL_DIM_PHYS(rhs_dispatch, float, ns, use_vc(P), order, m, a, P, T, s);
}
cudaError_t launch_lift(int dim, int order, const MeshDev &m, const LiftArgs &a,
                        const PhysParams &P, const OpTables &T, cudaStream_t s) {
    if (m.E <= 0) return cudaSuccess;
    PRANDTL_DIM_LIFT(lift_dispatch, double, use_vc(P), order, m, a, P, T, s);
}
cudaError_t launch_lift_fp32(int dim, int order, const MeshDev &m, const LiftArgs &a,
                             const PhysParams &P, const OpTables &T, cudaStream_t s) {
    if (m.E <= 0) return cudaSuccess;
    PRANDTL_DIM_LIFT(lift_dispatch, float, use_vc(P), order, m, a, P, T, s);
}

int batch_num_variants() { return 3; }

cudaError_t batch_prepare_rhs(int dim, int order, bool ns, bool vc, bool fp32, int variant, BatchKernelInfo *info) {
    if (fp32) PRANDTL_DIM_PHYS(rhs_batch_prepare, float, ns, vc, order, variant, info);
    PRANDTL_DIM_PHYS(rhs_batch_prepare, double, ns, vc, order, variant, info);
}
cudaError_t batch_prepare_lift(int dim, int order, bool vc, bool fp32, BatchKernelInfo *info) {
    if (fp32) PRANDTL_DIM_LIFT(lift_batch_prepare, float, vc, order, info);
    PRANDTL_DIM_LIFT(lift_batch_prepare, double, vc, order, info);
}
cudaError_t batch_launch_rhs(int dim, int order, bool ns, bool vc, bool fp32, int variant, int grid,
                             const BatchClassDev &c, const BatchStage &st, const OpTables &T, cudaStream_t s) {
    if (fp32) PRANDTL_DIM_PHYS(rhs_batch_launch, float, ns, vc, order, variant, grid, c, st, T, s);
    PRANDTL_DIM_PHYS(rhs_batch_launch, double, ns, vc, order, variant, grid, c, st, T, s);
}
cudaError_t batch_launch_lift(int dim, int order, bool vc, bool fp32, int grid, const BatchClassDev &c,
                              const BatchStage &st, const OpTables &T, cudaStream_t s) {
    if (fp32) PRANDTL_DIM_LIFT(lift_batch_launch, float, vc, order, grid, c, st, T, s);
    PRANDTL_DIM_LIFT(lift_batch_launch, double, vc, order, grid, c, st, T, s);
}

namespace {
// Simulation.cpp:1013-1018: dt = cfl * hmin / (lambda_max * (N+1)^2), here per
// solve from the largest |V|+c seen during its last step.
__global__ void batch_step_end_kernel(BatchInst *tab, const int *live, const int *n_live, int flip, int *left) {
    const int n = *n_live;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int id = live[q];
        BatchInst &I = tab[id];
        if (I.steps_left <= 0) continue;
        I.steps_left -= 1;
        left[id] = I.steps_left;
        I.steps_done += 1;
        I.cur ^= flip;
        const unsigned long long bits = I.lambda;
        I.lambda_last = bits;
        I.lambda = 0ull;
        const double lam = __longlong_as_double((long long)bits);
        if (I.cfl > 0.0 && lam > 0.0 && lam < 1e300) {
            const double np = double(I.order + 1);
            I.dt = I.cfl * I.hmin / (lam * np * np);
        }
    }
}
}   // namespace

cudaError_t batch_launch_step_end(BatchInst *tab, const int *live, const int *n_live, int flip, int *left,
                                  cudaStream_t s) {
    batch_step_end_kernel<<<8, 256, 0, s>>>(tab, live, n_live, flip, left);
    return cudaGetLastError();
}

}   // namespace prandtl
