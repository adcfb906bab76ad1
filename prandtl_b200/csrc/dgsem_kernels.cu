// dgsem_kernels.cu -- dispatch of the DGSEM kernels by dimension, working
// precision and physics to the dgsem_inst_*.cu translation units, and the
// batch step-end kernel.
#include "dgsem_kernels.cuh"

namespace prandtl {

bool order_supported(int dim, int order) {
    return (dim == 2 || dim == 3) && order >= 1 && order <= 5;
}

#define PRANDTL_DIM_NS(FN, REAL, ...)                                              \
    do {                                                                           \
        if (dim == 2) return ns ? FN<2, REAL, true>(__VA_ARGS__) : FN<2, REAL, false>(__VA_ARGS__); \
        if (dim == 3) return ns ? FN<3, REAL, true>(__VA_ARGS__) : FN<3, REAL, false>(__VA_ARGS__); \
        return cudaErrorInvalidValue;                                              \
    } while (0)
#define PRANDTL_DIM(FN, OUT, ...)                                                  \
    do {                                                                           \
        if (dim == 2) return FN<2, OUT>(__VA_ARGS__);                              \
        if (dim == 3) return FN<3, OUT>(__VA_ARGS__);                              \
        return cudaErrorInvalidValue;                                              \
    } while (0)

cudaError_t launch_rhs(int dim, int order, bool ns, const MeshDev &m, const RhsArgs &a,
                       const PhysParams &P, const OpTables &T, cudaStream_t s) {
    if (m.E <= 0) return cudaSuccess;
    PRANDTL_DIM_NS(rhs_dispatch, double, order, m, a, P, T, s);
}
cudaError_t launch_rhs_fp32(int dim, int order, bool ns, const MeshDev &m, const RhsArgs &a,
                            const PhysParams &P, const OpTables &T, cudaStream_t s) {
    if (m.E <= 0) return cudaSuccess;
    PRANDTL_DIM_NS(rhs_dispatch, float, order, m, a, P, T, s);
}
cudaError_t launch_lift(int dim, int order, const MeshDev &m, const LiftArgs &a,
                        const PhysParams &P, const OpTables &T, cudaStream_t s) {
    if (m.E <= 0) return cudaSuccess;
    PRANDTL_DIM(lift_dispatch, double, order, m, a, P, T, s);
}
cudaError_t launch_lift_fp32(int dim, int order, const MeshDev &m, const LiftArgs &a,
                             const PhysParams &P, const OpTables &T, cudaStream_t s) {
    if (m.E <= 0) return cudaSuccess;
    PRANDTL_DIM(lift_dispatch, float, order, m, a, P, T, s);
}

int batch_num_variants() { return 3; }

cudaError_t batch_prepare_rhs(int dim, int order, bool ns, bool fp32, int variant, BatchKernelInfo *info) {
    if (fp32) PRANDTL_DIM_NS(rhs_batch_prepare, float, order, variant, info);
    PRANDTL_DIM_NS(rhs_batch_prepare, double, order, variant, info);
}
cudaError_t batch_prepare_lift(int dim, int order, bool fp32, BatchKernelInfo *info) {
    if (fp32) PRANDTL_DIM(lift_batch_prepare, float, order, info);
    PRANDTL_DIM(lift_batch_prepare, double, order, info);
}
cudaError_t batch_launch_rhs(int dim, int order, bool ns, bool fp32, int variant, int grid,
                             const BatchClassDev &c, const BatchStage &st, const OpTables &T, cudaStream_t s) {
    if (fp32) PRANDTL_DIM_NS(rhs_batch_launch, float, order, variant, grid, c, st, T, s);
    PRANDTL_DIM_NS(rhs_batch_launch, double, order, variant, grid, c, st, T, s);
}
cudaError_t batch_launch_lift(int dim, int order, bool fp32, int grid, const BatchClassDev &c,
                              const BatchStage &st, const OpTables &T, cudaStream_t s) {
    if (fp32) PRANDTL_DIM(lift_batch_launch, float, order, grid, c, st, T, s);
    PRANDTL_DIM(lift_batch_launch, double, order, grid, c, st, T, s);
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
