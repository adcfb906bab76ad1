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
    const BcDev *bcs;    // boundary conditions (boundary faces: nbr = {-1, bc, face id, 0})
    // axisymmetric (z, r) form, 2D Euler (null otherwise)
    const double *rad;            // [Ndof] node radius
    const unsigned char *axis;    // [Ndof] 1 at axis nodes
    // non-affine (multilinear) elements, FP64 one-shot kernels (null otherwise):
    // the transformation at every node, [DIM*DIM + 1][Ndof] (adj(J) row-major,
    // then det J); the scaled normal at every face node, [F][Np^(DIM-1)][DIM]
    // (elem1's face node order); the subcell interface normals of every line,
    // [E][DIM][Np^(DIM-1)][Np-1][DIM] (interior interfaces 1..Np-1)
    const double *ngeo;
    const double *fnn;
    const double *snor;
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
    const double *u_rk;     // axisymmetric: the RK state r U (u holds the recovered U); else null
    unsigned int *health;   // RK modes: OR of the state-check bits of the new state (may be null)
};

struct LiftArgs {
    const double *u;
    double *grad;           // FP64 path
    float *grad32;          // FP32-bulk form
};

// ---------------------------------------------------------------- batches
// Device record of one resident solve in a batch.  The host writes it on
// admission; the step kernel advances steps_left / cur / dt; the RHS kernels
// fold max |V|+c into lambda.
enum BatchScheme : int { BATCH_SSPRK3 = 0, BATCH_LSRK45 = 1 };
constexpr int BATCH_CHUNK = 64;   // per-solve element ranges are padded to this in the work prefix

struct BatchInst {
    PhysParams P;
    const double *geo;          // [E][DIM*DIM + 1]
    const int4 *nbr;            // [E][2*DIM] (solve-local element and face ids)
    const double *fnor;         // [F][DIM]
    double *u[3];               // LSRK: state ping-pong u[0], u[1] and the register u[2];
                                // SSP-RK3: x, y1, y2
    void *grad;                 // NS gradients (double or float)
    double *alpha;              // [E] or null
    long long Ndof;             // E * Np^DIM
    int E, order;
    double dt;                  // current time step
    double cfl, hmin;           // cfl > 0: dt = cfl hmin / (lambda (N+1)^2) after every step
    int steps_left;             // > 0: the solve advances; 0: frozen
    int steps_done;
    int cur;                    // LSRK: u[cur] holds the state at the start of the step
    unsigned int health;        // state-check bits of the RK stages (sticky); non-zero freezes the solve
    const BcDev *bcs;           // boundary conditions (boundary faces)
    unsigned long long lambda;  // max |V|+c over the current step's stages (ordered bits)
    unsigned long long lambda_last;   // ... of the last completed step
    double t;                   // simulated time: the sum of the completed steps' dt
    double t_final;             // > 0: end time (the last step is shortened to reach it)
};
// One (dim, order, physics) class of a batch: its solves and the padded
// element prefix over them (prefix[s+1] - prefix[s] = E of slot s rounded up
// to BATCH_CHUNK).  hdr[0] = number of slots.
struct BatchClassDev {
    BatchInst *tab;
    const int *ids;
    const int *prefix;
    const int *hdr;
};
struct BatchStage {
    int scheme;                 // BatchScheme
    int stage;                  // stage index within the step
    double rkA, rkB;            // LSRK coefficients of the stage
};
struct BatchKernelInfo {
    int blocks_per_sm, threads, smem, regs, elems_per_item;
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

// Batch kernels of one class.  `variant` in [0, batch_num_variants()) picks the
// RHS launch shape.  `vc` selects the Navier-Stokes form that passes
// contravariant viscous fluxes from the lifting to the RHS (quirks = 1) instead
// of primitive gradients (quirks = 0).  prepare_* must run outside stream capture.
int batch_num_variants();
cudaError_t batch_prepare_rhs(int dim, int order, bool ns, bool vc, bool fp32, int variant, BatchKernelInfo *info);
cudaError_t batch_prepare_lift(int dim, int order, bool vc, bool fp32, BatchKernelInfo *info);
cudaError_t batch_launch_rhs(int dim, int order, bool ns, bool vc, bool fp32, int variant, int grid,
                             const BatchClassDev &c, const BatchStage &st, const OpTables &T, cudaStream_t s);
cudaError_t batch_launch_lift(int dim, int order, bool vc, bool fp32, int grid, const BatchClassDev &c,
                              const BatchStage &st, const OpTables &T, cudaStream_t s);
// End of a batch step: every live solve with steps left advances its counters,
// flips its LSRK parity, (cfl > 0) takes its next dt from lambda, and writes
// its remaining step count to left[id]; a solve whose state check failed
// (health != 0) is frozen instead: steps_left = 0.  With an end time the
// solve's time advances by the step's dt, the next dt is cut to reach t_final
// and the solve stops there (Simulation.cpp:1007-1024).
// FP64 budgets over the mesh (node weights w_i w_j (w_k) |J|): the integrals
// of the nf conserved fields and of the entropy function U = -rho s / (g-1),
// s = ln(p rho^-g); with dudt also the integrals of dudt_f and of v . dudt
// (v the entropy variables).  nout = 2 nf + 2 values; deterministic two-pass
// reduction through `partials` ([BUDGET_BLOCKS][nout]).  ndetj (non-affine
// elements, may be null): det J at every node instead of the element's.
constexpr int BUDGET_BLOCKS = 592;    // 4 per SM on 148 SMs (grid-stride beyond)
constexpr int BUDGET_THREADS = 256;
cudaError_t launch_budgets(const double *u, const double *dudt, const double *geo, const double *ndetj,
                           const double *w1d, int dim, int np, int E, double gamma, double *partials, double *out,
                           cudaStream_t s);

// Axisymmetric form: U recovered from the weighted state rU (2D, 4 fields).
cudaError_t launch_axi_recover(const double *rU, double *U, const double *xy, const unsigned char *axis,
                               long long Ndof, int ND, double rho_floor, cudaStream_t s);
cudaError_t batch_launch_step_end(BatchInst *tab, const int *live, const int *n_live, int flip, int *left,
                                  cudaStream_t s);

// Per-(dim, working precision, physics) dispatchers, one translation unit each.
// VC (Navier-Stokes only): the lifting emits the contravariant viscous fluxes
// adj * Fv^T, rows 1..NF-1, as [DIM][NF-1][Ndof] in the gradient buffer, and
// the RHS reads them instead of evaluating viscous fluxes from gradients.
template <int DIM, typename Real, bool NS, bool VC>
cudaError_t rhs_dispatch(int order, const MeshDev &m, const RhsArgs &a, const PhysParams &P,
                         const OpTables &T, cudaStream_t s);
template <int DIM, typename Out, bool VC>
cudaError_t lift_dispatch(int order, const MeshDev &m, const LiftArgs &a, const PhysParams &P,
                          const OpTables &T, cudaStream_t s);
template <int DIM, typename Real, bool NS, bool VC>
cudaError_t rhs_batch_prepare(int order, int variant, BatchKernelInfo *info);
template <int DIM, typename Real, bool NS, bool VC>
cudaError_t rhs_batch_launch(int order, int variant, int grid, const BatchClassDev &c, const BatchStage &st,
                             const OpTables &T, cudaStream_t s);
template <int DIM, typename Out, bool VC>
cudaError_t lift_batch_prepare(int order, BatchKernelInfo *info);
template <int DIM, typename Out, bool VC>
cudaError_t lift_batch_launch(int order, int grid, const BatchClassDev &c, const BatchStage &st,
                              const OpTables &T, cudaStream_t s);

// The Navier-Stokes form used for a configuration: contravariant viscous
// fluxes (VC) unless the reference's defects are reproduced (quirks == 0,
// whose volume and face viscous fluxes differ, Q1/Q8).
inline bool use_vc(const PhysParams &P) { return P.quirks != 0; }

}   // namespace prandtl
