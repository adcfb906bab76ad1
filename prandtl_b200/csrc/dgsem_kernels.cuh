// dgsem_kernels.cuh -- launch interface of the DGSEM RHS kernels.
#pragma once

#include <cuda_runtime.h>

#include "dgsem_device.cuh"

namespace prandtl {

// Epilogue applied to the freshly computed element RHS L(u).
enum EpilogueMode : int {
    EPI_STORE = 0,   // dudt = L(u)
    EPI_LSRK = 1,    // du = A du + dt L(u);  u_out = u + B du   (2N-storage RK)
    EPI_SSP1 = 2,    // u_out = u + dt L(u)                      (RK3SSPSolver stage 1)
    EPI_SSP2 = 3,    // u_out = 3/4 x0 + 1/4 (u + dt L(u))       (stage 2)
    EPI_SSP3 = 4,    // u_out = 1/3 x0 + 2/3 (u + dt L(u))       (stage 3; u_out may be x0)
};

struct MeshDev {
    const double *geo;   // [E][DIM*DIM + 1]: adj(J) row-major, then det J
    const int4 *nbr;     // [E][2*DIM]: {neighbour elem, neighbour local face, face id, role}
    const double *fnor;  // [F][DIM] scaled normal, outward from elem1
    int E;
    long long Ndof;      // E * Np^DIM
};

struct RhsArgs {
    const double *u;        // stage input state (byNODES)
    const double *grad;     // NS: primitive gradients [DIM][NF][Ndof] (FP64 path)
    double *dudt;           // EPI_STORE output
    double *u_out;          // RK output state
    double *du;             // LSRK register
    const double *x0;       // SSP step-start state
    double *alpha;          // [E] blending coefficient out (may be null)
    unsigned long long *lambda;   // max |V|+c as ordered bits (may be null)
    double dt, rkA, rkB;
    int mode;
    const float *grad32;    // NS: primitive gradients, FP32-bulk form
};

struct LiftArgs {
    const double *u;
    double *grad;           // FP64 path
    float *grad32;          // FP32-bulk form
};

// Launchers (dispatch on dim and order).  Return cudaSuccess or the launch error.
cudaError_t launch_rhs(int dim, int order, bool ns, const MeshDev &m, const RhsArgs &a,
                       const PhysParams &P, const OpTables &T, cudaStream_t s);
cudaError_t launch_lift(int dim, int order, const MeshDev &m, const LiftArgs &a,
                        const PhysParams &P, const OpTables &T, cudaStream_t s);
// FP32-bulk form: flux work in FP32, primitives and RK update in FP64.
cudaError_t launch_rhs_fp32(int dim, int order, bool ns, const MeshDev &m, const RhsArgs &a,
                            const PhysParams &P, const OpTables &T, cudaStream_t s);
cudaError_t launch_lift_fp32(int dim, int order, const MeshDev &m, const LiftArgs &a,
                             const PhysParams &P, const OpTables &T, cudaStream_t s);
bool order_supported(int dim, int order);

}   // namespace prandtl
