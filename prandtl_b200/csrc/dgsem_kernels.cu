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
        if (I.health != 0u) {   // the state left the admissible set: stop here
            I.steps_left = 0;
            left[id] = 0;
            continue;
        }
        I.steps_left -= 1;
        I.steps_done += 1;
        I.cur ^= flip;
        I.t += I.dt;
        const unsigned long long bits = I.lambda;
        I.lambda_last = bits;
        I.lambda = 0ull;
        const double lam = __longlong_as_double((long long)bits);
        if (I.cfl > 0.0 && lam > 0.0 && lam < 1e300) {
            const double np = double(I.order + 1);
            I.dt = I.cfl * I.hmin / (lam * np * np);
        }
        if (I.t_final > 0.0) {   // dt_real = min(dt, t_final - t); done at t >= t_final - 1e-8 dt
            if (I.t >= I.t_final - 1e-8 * I.dt) I.steps_left = 0;
            else I.dt = fmin(I.dt, I.t_final - I.t);
        }
        left[id] = I.steps_left;
    }
}

// DGSEMOperator::RecoverStateFromWeighted (DGSEMOperator.cpp:161-470) with the
// low-order axis reconstruction the reference selects for "axis" boundaries
// (Simulation.cpp:520-530).  One thread per node: off the axis U = rU / r; at
// an axis node (or r <= 0) each field is d(rU)/dr from the two nearest
// off-axis nodes of the element at the same z (else the two nearest overall):
// the least-squares slope through the origin, limited by minmod against 1.5x
// each node's own slope and clamped to 10 |f1| / r1 (one node: its slope).  A
// density that is non-finite or below rho_floor, or a non-finite energy, takes
// the nearest off-axis node's U instead; radial momentum is 0 there.  Products and sums
// are rounded separately (no contraction) so the result is the host's bit
// for bit.
__device__ __forceinline__ double axi_sign(double a) { return (double)((a > 0) - (a < 0)); }
__device__ __forceinline__ double axi_minmod(double a, double b) {
    return __dmul_rn(a, b) <= 0.0 ? 0.0 : axi_sign(a) * fmin(fabs(a), fabs(b));
}
__device__ __forceinline__ double axi_clamp(double x, double m) {
    if (!isfinite(x)) return 0.0;
    return fabs(x) <= m ? x : axi_sign(x) * m;
}

__global__ void axi_recover_kernel(const double *__restrict__ rU, double *__restrict__ U,
                                   const double *__restrict__ xy, const unsigned char *__restrict__ axis,
                                   long long Ndof, int ND, double rho_floor) {
    constexpr int NF = 4;
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < Ndof;
         g += (long long)gridDim.x * blockDim.x) {
        const double *rr = xy + Ndof;
        const double r = rr[g];
        if (!axis[g] && r > 0.0) {
#pragma unroll
            for (int f = 0; f < NF; ++f) U[f * Ndof + g] = rU[f * Ndof + g] / r;
            continue;
        }
        const long long g0 = (g / ND) * ND;
        const double z_axis = xy[g];
        int j1 = -1, j2 = -1;
        double r1 = inf, r2 = inf;
        for (int pass = 0; pass < 2 && j1 < 0; ++pass)
            for (int j = 0; j < ND; ++j) {
                const double rj = rr[g0 + j];
                if (!(rj > 0.0)) continue;
                if (pass == 0 && !(fabs(xy[g0 + j] - z_axis) <= 1e-12)) continue;
                if (rj < r1) { r2 = r1; j2 = j1; r1 = rj; j1 = j; }
                else if (rj < r2) { r2 = rj; j2 = j; }
            }
        double d[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            const double *fe = rU + f * Ndof + g0;
            const double f_ref = j1 >= 0 ? fabs(fe[j1]) : 0.0;
            const double cap = (j1 >= 0 && !(f_ref < 1e-12)) ? __dmul_rn(10.0, f_ref) / fmax(r1, 1e-14) : inf;
            double v = 0.0;
            if (j1 >= 0 && j2 >= 0 && isfinite(r1) && isfinite(r2) && r1 > 0.0 && r2 > 0.0) {
                const double f1 = fe[j1], f2 = fe[j2];
                const double m = __dadd_rn(__dmul_rn(r1, f1), __dmul_rn(r2, f2)) /
                                 fmax(__dadd_rn(__dmul_rn(r1, r1), __dmul_rn(r2, r2)), 1e-14);
                const double s1 = f1 / r1, s2 = f2 / r2;
                v = axi_clamp(axi_minmod(m, axi_minmod(__dmul_rn(1.5, s1), __dmul_rn(1.5, s2))), cap);
            } else if (j1 >= 0 && isfinite(r1) && r1 > 0.0) {
                v = axi_clamp(fe[j1] / r1, cap);
            }
            d[f] = v;
        }
        if (!isfinite(d[0]) || d[0] < rho_floor || !isfinite(d[3])) {
            int nb = -1;
            double rn = -1.0;
            for (int j = 0; j < ND; ++j) {
                const double rj = rr[g0 + j];
                if (rj > 0.0 && (nb == -1 || rj < rn)) { rn = rj; nb = j; }
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) U[f * Ndof + g] = nb < 0 ? 0.0 : rU[f * Ndof + g0 + nb] / rn;
            U[2 * Ndof + g] = 0.0;
        } else {
            U[g] = d[0];
            U[Ndof + g] = d[1];
            U[2 * Ndof + g] = 0.0;
            U[3 * Ndof + g] = d[3];
        }
    }
}
}   // namespace

namespace {
struct Weights1D {
    double w[8];
};

// One thread per node (grid-stride), FP64 throughout; warp shuffles, then the
// block's warps in order, give one partial per block and output.
template <int NOUT>
__global__ void __launch_bounds__(BUDGET_THREADS) budget_kernel(const double *__restrict__ u,
                                                               const double *__restrict__ dudt,
                                                               const double *__restrict__ geo,
                                                               const double *__restrict__ ndetj, Weights1D W,
                                                               int dim, int np, int E, double gamma,
                                                               double *__restrict__ partials) {
    constexpr int MAXF = (NOUT - 2) / 2;
    const int nf = dim + 2, nd = dim == 2 ? np * np : np * np * np;
    const long long Ndof = (long long)E * nd;
    double acc[NOUT];
#pragma unroll
    for (int q = 0; q < NOUT; ++q) acc[q] = 0.0;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < Ndof;
         g += (long long)gridDim.x * blockDim.x) {
        const int e = (int)(g / nd), n = (int)(g - (long long)e * nd);
        double wn = W.w[n % np] * W.w[(n / np) % np];
        if (dim == 3) wn *= W.w[n / (np * np)];
        const double wJ = wn * fabs(ndetj ? ndetj[g] : geo[(long long)e * (dim * dim + 1) + dim * dim]);
        double s[MAXF], r[MAXF];
#pragma unroll
        for (int f = 0; f < MAXF; ++f) {
            s[f] = f < nf ? u[f * Ndof + g] : 0.0;
            r[f] = (f < nf && dudt) ? dudt[f * Ndof + g] : 0.0;
        }
        const double rho = s[0], E_ = s[nf - 1];
        double vv = 0.0;
#pragma unroll
        for (int d = 0; d < MAXF - 2; ++d)
            if (d < dim) vv += (s[1 + d] / rho) * (s[1 + d] / rho);
        const double p = (gamma - 1.0) * (E_ - 0.5 * rho * vv);
        const double ent = log(p) - gamma * log(rho);
        const double beta = rho / p;
#pragma unroll
        for (int f = 0; f < MAXF; ++f)
            if (f < nf) {
                acc[f] += wJ * s[f];
                acc[MAXF + 1 + f] += wJ * r[f];
            }
        acc[MAXF] += wJ * (-rho * ent / (gamma - 1.0));
        double vd = ((gamma - ent) / (gamma - 1.0) - 0.5 * beta * vv) * r[0] - beta * r[nf - 1];
#pragma unroll
        for (int d = 0; d < MAXF - 2; ++d)
            if (d < dim) vd += beta * (s[1 + d] / rho) * r[1 + d];
        acc[NOUT - 1] += wJ * vd;
    }
    __shared__ double red[BUDGET_THREADS / 32][NOUT];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NOUT; ++q) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[wid][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < NOUT) {
        double v = 0.0;
        for (int k = 0; k < BUDGET_THREADS / 32; ++k) v += red[k][threadIdx.x];
        partials[blockIdx.x * NOUT + threadIdx.x] = v;
    }
}

__global__ void budget_final_kernel(const double *__restrict__ partials, int blocks, int nout,
                                    double *__restrict__ out) {
    const int q = threadIdx.x;
    if (q >= nout) return;
    double v = 0.0;
    for (int b = 0; b < blocks; ++b) v += partials[b * nout + q];   // fixed order: deterministic
    out[q] = v;
}
}   // namespace

cudaError_t launch_budgets(const double *u, const double *dudt, const double *geo, const double *ndetj,
                           const double *w1d, int dim, int np, int E, double gamma, double *partials, double *out,
                           cudaStream_t s) {
    if (np < 2 || np > 8 || (dim != 2 && dim != 3) || E <= 0) return cudaErrorInvalidValue;
    Weights1D W{};
    for (int i = 0; i < np; ++i) W.w[i] = w1d[i];
    const long long Ndof = (long long)E * (dim == 2 ? np * np : np * np * np);
    long long blocks = (Ndof + BUDGET_THREADS - 1) / BUDGET_THREADS;
    if (blocks > BUDGET_BLOCKS) blocks = BUDGET_BLOCKS;
    // outputs: nf conserved integrals, entropy, nf rate integrals, entropy rate
    constexpr int NOUT = 2 * 5 + 2;
    budget_kernel<NOUT><<<(unsigned)blocks, BUDGET_THREADS, 0, s>>>(u, dudt, geo, ndetj, W, dim, np, E, gamma, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    budget_final_kernel<<<1, 32, 0, s>>>(partials, (int)blocks, NOUT, out);
    return cudaGetLastError();
}

cudaError_t launch_axi_recover(const double *rU, double *U, const double *xy, const unsigned char *axis,
                               long long Ndof, int ND, double rho_floor, cudaStream_t s) {
    if (Ndof <= 0) return cudaSuccess;
    const long long blocks = (Ndof + 255) / 256;
    axi_recover_kernel<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, s>>>(rU, U, xy, axis, Ndof, ND, rho_floor);
    return cudaGetLastError();
}

cudaError_t batch_launch_step_end(BatchInst *tab, const int *live, const int *n_live, int flip, int *left,
                                  cudaStream_t s) {
    batch_step_end_kernel<<<8, 256, 0, s>>>(tab, live, n_live, flip, left);
    return cudaGetLastError();
}

}   // namespace prandtl
