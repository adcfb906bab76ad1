/*
 * prandtl_b200.h -- C ABI of the B200 (sm_100a) DGSEM right-hand side and
 * Runge-Kutta step of Prandtl.
 *
 * The reference exposes this hot path as
 *     class DGSEMOperator : public mfem::TimeDependentOperator
 *         void Mult(const Vector &u, Vector &dudt) const;      (src/Operators/DGSEMOperator.hpp:105)
 *         real_t GetMaxCharSpeed();                            (DGSEMOperator.hpp:106-109)
 *         real_t &GetTimeRef();                                (DGSEMOperator.hpp:111-114)
 * driven by mfem::ODESolver::Step (src/Simulation/Simulation.cpp:1010).  The
 * entry points below are what that surface binds to: plain pointers and
 * sizes, no C++ or CUDA types.  A header-only MFEM adapter
 * (prandtl_b200/shim/dgsem_operator_gpu.hpp) restores the class interface.
 *
 * Data layout (identical to the reference's mfem::Vector, Ordering::byNODES):
 *   u[f*Ndof + e*Np^dim + node], f = 0..dim+1 (rho, rho*v, E), node
 *   lexicographic with x fastest, Np = order + 1, Ndof = E*Np^dim.
 * State and RHS are FP64.
 *
 * Every call returns a prandtl_status; nothing aborts, traps or exits.
 * A handle owns one CUDA stream and its scratch buffers; calls on one handle
 * are serialised, different handles are independent.
 */
#ifndef PRANDTL_B200_H
#define PRANDTL_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum prandtl_status {
    PRANDTL_OK = 0,
    PRANDTL_EINVAL = 1,        /* bad argument or descriptor */
    PRANDTL_ENOMEM = 2,        /* device allocation failed */
    PRANDTL_ENONFINITE = 3,    /* the RK state left the admissible set: a non-finite value, or
                                  density or pressure <= 0 (the reference's NaN check,
                                  Simulation.cpp:1024-1035, extended to positivity) */
    PRANDTL_ETIMEDOUT = 4,     /* a bounded wait ran out */
    PRANDTL_ECUDA = 5,         /* CUDA runtime error (text in prandtl_last_error) */
    PRANDTL_EUNSUPPORTED = 6,  /* valid input outside what this build implements */
    PRANDTL_ETOOLARGE = 7      /* input larger than a fixed-size limit (prandtl_rhs_noalloc) */
} prandtl_status;

/* State-check bits behind PRANDTL_ENONFINITE: every RK stage checks every
 * node of the state it writes (the axisymmetric form checks finiteness only,
 * since its RK state r U vanishes on the axis). */
#define PRANDTL_HEALTH_NONFINITE 1u
#define PRANDTL_HEALTH_DENSITY 2u
#define PRANDTL_HEALTH_PRESSURE 4u

/* Pointer-location flags for the u / dudt arguments. */
#define PRANDTL_PTR_HOST 0     /* host memory: staged through the handle's device buffers */
#define PRANDTL_PTR_DEVICE 1   /* device memory on the handle's GPU: zero-copy */

/* Time-integration schemes of prandtl_step. */
#define PRANDTL_RK3SSP 0       /* Shu-Osher SSP-RK3, mfem::RK3SSPSolver operation order */
#define PRANDTL_LSRK45 1       /* Carpenter-Kennedy five-stage fourth-order 2N-storage RK */

/* Mesh in the form the DGSEM kernels consume.  Built by the caller from its
 * mfem::ParMesh (per element: ElementTransformation::AdjugateJacobian and
 * Weight of the affine map from [0,1]^dim; per interior face:
 * FaceElementTransformations Elem1No/Elem2No, local faces and CalcOrtho;
 * non-affine elements add the per-node values below). */
typedef struct prandtl_mesh_desc {
    int dim;                   /* 2 or 3 */
    int order;                 /* polynomial degree N (1..5); Np = N + 1 Gauss-Lobatto nodes */
    int num_elements;          /* E */
    int num_faces;             /* F faces: interior faces, then or mixed with boundary faces */
    const double *elem_adj;    /* [E][dim][dim] adjugate of the element Jacobian, row-major */
    const double *elem_detj;   /* [E] Jacobian determinant */
    const int *face_elems;     /* [F][4] elem1, lface1, elem2, lface2; lface = 2*dir + side,
                                  side 0 is the xi_dir = 0 face; traces aligned.  A boundary
                                  face is {elem1, lface1, -1, bc} with bc an index into
                                  prandtl_config.bcs (Euler only) */
    const double *face_nor;    /* [F][dim] scaled normal outward from elem1 (|n| = face measure) */
    /* Non-affine (multilinear) elements: all three set, or all three NULL for
     * affine meshes.  MFEM evaluates the transformation at every Gauss-Lobatto
     * node (ElementTransformation::SetIntPoint + AdjugateJacobian / Weight,
     * DGSEMIntegrator.cpp:254-267, LiftingBR1.cpp:184-186) and CalcOrtho at
     * every face point (DGSEMIntegrator.cpp:151-222); these arrays hold those
     * values.  prandtl_create takes them in the FP64 form and, for Euler, in
     * the FP32-bulk form; FP32-bulk Navier-Stokes, batches and
     * prandtl_rhs_noalloc return PRANDTL_EUNSUPPORTED.  elem_adj / elem_detj /
     * face_nor are still read
     * (validation, the element size) and may hold the element-centre values. */
    const double *node_adj;    /* [E][Np^dim][dim][dim] adj(J) at each node, row-major */
    const double *node_detj;   /* [E][Np^dim] det J at each node (> 0) */
    const double *face_node_nor; /* [F][Np^(dim-1)][dim] scaled normal at each face node,
                                    outward from elem1, in elem1's face node order */
} prandtl_mesh_desc;

/* Boundary conditions of boundary faces (Euler), each the reference's
 * boundary integrator of the same name with a constant state
 * (src/Integrators/BoundaryConditions/): */
#define PRANDTL_BC_STATE 0            /* SpecifiedState / SupersonicInflow: outer state = state */
#define PRANDTL_BC_OUTFLOW 1          /* SupersonicOutflow: outer state = inner state */
#define PRANDTL_BC_SLIP_WALL 2        /* SlipWall: pressure flux of the normal Riemann problem */
#define PRANDTL_BC_SYMMETRY 3         /* Symmetry: inner state with reflected normal momentum */
#define PRANDTL_BC_PRESSURE_OUTFLOW 4 /* SubsonicOutflowP: inner state at pressure p */
#define PRANDTL_BC_RIEMANN 5          /* RiemannInvariant: characteristic state from the outer
                                         primitive state (rho, V, p) in state[] */
#define PRANDTL_BC_INFLOW_RV 6        /* SubsonicInflowRV: density state[0], velocity state[1..dim],
                                         inner pressure */
#define PRANDTL_BC_INFLOW_PTTT 7      /* SubsonicInflowPtTtAng: total pressure pt, total temperature
                                         Tt, cp, flow angles theta, phi in degrees */
#define PRANDTL_BC_NOSLIP_ADIABATIC 8 /* NoSlipAdiabWall: wall velocity, normal heat flux */
#define PRANDTL_BC_NOSLIP_ISOTHERMAL 9 /* NoSlipIsothWall: wall velocity, wall temperature */
#define PRANDTL_BC_AXIS 10            /* the r = 0 axis of the axisymmetric form: the symmetry
                                         flux; marks the axis nodes (axisymmetric = 1 only) */
/* With parabolic = 1 every type but SLIP_WALL, SYMMETRY and INFLOW_PTTT is
 * accepted (the reference defines no viscous treatment for the first two), and
 * RIEMANN only with quirks = 1 (the reference's Riemann lifting reads a face
 * normal that is never set for it); in the Euler form the no-slip walls act as
 * slip walls, as in the reference. */
typedef struct prandtl_bc {
    int type;                  /* PRANDTL_BC_* */
    double state[5];           /* STATE: conserved outer state; RIEMANN: primitive outer state;
                                  INFLOW_RV: rho, V (dim+2 or dim+1 used) */
    double p;                  /* outflow pressure (PRANDTL_BC_PRESSURE_OUTFLOW) */
    double pt, Tt, cp;         /* PRANDTL_BC_INFLOW_PTTT */
    double theta, phi;         /*   flow direction (cos t, sin t) in 2D, (cos t sin f, sin t sin f, cos f) in 3D */
    double wall_vel[3];        /* NOSLIP_*: wall velocity (dim used) */
    double heat_flux;          /* NOSLIP_ADIABATIC: normal heat flux per unit face area */
    double wall_T;             /* NOSLIP_ISOTHERMAL: wall temperature (with the config's R_gas) */
} prandtl_bc;

/* Physics and switches.  Defaults (prandtl_config_default) match the
 * reference's Simulation::LoadConfig defaults (Simulation.cpp:153-157) and
 * PhysicsConstants (src/Physics/Physics.hpp:27-37). */
typedef struct prandtl_config {
    double gamma;              /* 1.4 */
    double Pr;                 /* 0.72 */
    double mu;                 /* 0.02, dynamic viscosity (constant unless sutherland) */
    double R_gas;              /* 287.05 */
    double alpha_max;          /* 0.5, blending cap (DGSEMOperator.hpp:99) */
    double alpha_min;          /* 0.001 */
    int parabolic;             /* 0: Euler; 1: Navier-Stokes with BR1 lifting (PARABOLIC) */
    int blending;              /* 1: modal indicator + subcell FV blending (SUBCELL_FV_BLENDING) */
    int sutherland;            /* 1: Sutherland viscosity (SUTHERLAND) */
    int quirks;                /* 0: reproduce the reference bit-for-bit in intent, including its
                                  known defects; 1: defects fixed (entropy-conservative 3D NS) */
    int surface_dissipation;   /* 1: reference surface flux; 0: entropy-conservative surface
                                  flux (verification switch, no reference counterpart) */
    int precision;             /* 0: FP64 throughout.  1: FP32 bulk -- two-point fluxes, flux
                                  differencing, surface fluxes and stored gradients in FP32;
                                  per-node primitives, entropy variables, lambda_max and the RK
                                  state and registers in FP64 (no reference counterpart) */
    double timeout_s;          /* bound on every host-side wait; 0 selects 120 s */
    int num_bcs;               /* boundary conditions the mesh's boundary faces index; */
    const prandtl_bc *bcs;     /*   copied at create (0 / NULL: periodic meshes only) */
    int axisymmetric;          /* 1: 2D Euler in (z, r) = (x, y) (AXISYMMETRIC): the state is r U,
                                  fluxes carry r, + p on the radial momentum; 0: planar */
    const double *node_coords; /* axisymmetric: [dim][Ndof] node coordinates (byNODES, the state's
                                  node order), copied at create; else ignored */
    double axis_rho_floor;     /* axisymmetric: density floor of the axis reconstruction; 0 selects
                                  1e-12 (DGSEMOperator.hpp:44).  The reference's driver raises it to
                                  max(1e-12, 1e-8 rho_inf) (SetAxisFloorsFromFreestream) */
} prandtl_config;

typedef struct prandtl_handle prandtl_handle;

/* Fill *cfg with the reference defaults. */
void prandtl_config_default(prandtl_config *cfg);

/* Build an operator for one mesh (DGSEMOperator ctor, DGSEMOperator.cpp:5-50,
 * plus DGSEMIntegrator ctor tables, DGSEMIntegrator.cpp:8-149).  Selects the
 * current CUDA device.  Allocates all device memory it will ever use.  The
 * first host-pointer call (prandtl_rhs / prandtl_step with PRANDTL_PTR_HOST)
 * on a state above 4 MB also allocates a 32 MB pinned host staging ring,
 * kept until prandtl_destroy, through which such calls copy the state in
 * 8 MB chunks filled and emptied by host threads. */
prandtl_status prandtl_create(const prandtl_mesh_desc *mesh, const prandtl_config *cfg,
                              prandtl_handle **out);

prandtl_status prandtl_destroy(prandtl_handle *h);

/* dudt = L(u): one RHS evaluation (DGSEMOperator::Mult, DGSEMOperator.cpp:537-591).
 * t is the operator time (TimeDependentOperator::SetTime); the periodic
 * problems here are autonomous.  lambda_max (may be NULL) receives the
 * largest |V|+c over all nodes of u (GetMaxCharSpeed with a per-call, not
 * running, maximum).  ptr_flags: PRANDTL_PTR_HOST or PRANDTL_PTR_DEVICE. */
prandtl_status prandtl_rhs(prandtl_handle *h, const double *u, double *dudt, double t,
                           double *lambda_max, int ptr_flags);

/* nsteps steps of size dt applied to u in place (ODESolver::Step,
 * Simulation.cpp:1010); each stage fuses the RK update into the RHS kernel.
 * Every stage checks the state it writes (PRANDTL_HEALTH_*) into a sticky
 * device flag of the handle.  With host pointers the call waits and returns
 * PRANDTL_ENONFINITE (state still copied back, reason in prandtl_last_error)
 * when any stage of these steps failed the check; with device pointers it
 * returns without waiting and the next prandtl_synchronize reports the flag.
 * Reporting clears the flag.  Runs of 8 or more steps replay a CUDA graph of
 * 4 steps (captured on the handle's own stream the first time for a given
 * state pointer, dt and scheme; launched on the handle's stream), with the
 * same results as step-by-step launches. */
prandtl_status prandtl_step(prandtl_handle *h, double *u, double t, double dt, int scheme,
                            int nsteps, int ptr_flags);

/* Per-element blending coefficient of the last RHS evaluation ([E] values;
 * the reference's `alpha` ParGridFunction on fes0). */
prandtl_status prandtl_get_alpha(prandtl_handle *h, double *alpha, int ptr_flags);

/* Axisymmetric form: the conserved state U recovered from the r-weighted state
 * rU ([4][Ndof] each), as every RHS evaluation sees it
 * (DGSEMOperator::RecoverStateFromWeighted, DGSEMOperator.cpp:161-470; the
 * reference's output fields are the primitives of this U, Simulation.cpp:1041-1044).
 * PRANDTL_EUNSUPPORTED for a planar operator. */
prandtl_status prandtl_recover_state(prandtl_handle *h, const double *rU, double *U, int ptr_flags);

/* FP64 budgets of a state on the device (planar forms): with nf = dim + 2,
 *   out[0 .. nf-1]       integrals of the conserved fields (mass, momentum, energy),
 *   out[nf]              integral of the entropy function U = -rho s / (gamma - 1),
 *                        s = ln(p rho^-gamma) (the entropy pair of the Chandrashekar flux),
 *   out[nf+1 .. 2nf]     integrals of dudt_f,
 *   out[2nf+1]           integral of v . dudt (v the entropy variables: the entropy production),
 * with the node weights w_i w_j (w_k) |J|; the last nf + 1 are 0 when dudt is NULL.
 * u and dudt follow ptr_flags; out is host memory of 2 nf + 2 doubles.  The sums are
 * deterministic (fixed-order two-pass reduction).  EUNSUPPORTED for the axisymmetric form. */
prandtl_status prandtl_budgets(prandtl_handle *h, const double *u, const double *dudt, double *out,
                               int ptr_flags);

/* CFL step dt = cfl*hmin/(lambda_max*(N+1)^2) (Simulation.cpp:906,1017). */
double prandtl_cfl_dt(double cfl, double hmin, double lambda_max, int order);

/* Use a caller-owned cudaStream_t (passed as void*) instead of the handle's. */
prandtl_status prandtl_set_stream(prandtl_handle *h, void *cuda_stream);

/* Wait for all work on the handle's stream, at most cfg->timeout_s; then
 * PRANDTL_ENONFINITE if a step since the last report failed the state check. */
prandtl_status prandtl_synchronize(prandtl_handle *h);

/* Number of kernels this handle has launched (instrumentation). */
long long prandtl_kernel_launches(const prandtl_handle *h);

/* Per-kernel CUDA-event timing (instrumentation, no reference counterpart).
 * While enabled, every launch is bracketed by events on the handle's stream;
 * prandtl_profile_read waits for the stream and returns the summed device
 * time and launch count of one kernel since the last reset. */
#define PRANDTL_KERNEL_RHS 0   /* fused volume + surface + RK-epilogue kernel */
#define PRANDTL_KERNEL_LIFT 1  /* BR1 lifting kernel (Navier-Stokes) */
#define PRANDTL_NUM_KERNELS 2
prandtl_status prandtl_profile(prandtl_handle *h, int enable);
prandtl_status prandtl_profile_read(prandtl_handle *h, int kernel, double *total_ms, long long *launches);
prandtl_status prandtl_profile_reset(prandtl_handle *h);

/* Bytes of device memory owned by the handle. */
size_t prandtl_device_bytes(const prandtl_handle *h);

/* Text of the last error on this handle ("" if none); h may be NULL for the
 * last error of a failed prandtl_create or prandtl_rhs_noalloc on this thread
 * (kept in a fixed thread-local buffer). */
const char *prandtl_last_error(const prandtl_handle *h);

const char *prandtl_version(void);

/* ---- Mesh ingestion (host only) ----
 * Replaces the reference's mesh setup, Simulation.cpp:271-336: `new
 * Mesh(file)` for MFEM v1.0 meshes (with a `nodes` section of L2_T1 corner
 * nodes, MFEM's form of periodic meshes) and Gmsh 2.2 ASCII meshes,
 * `UniformRefinement()` per `ser_ref_levels`, and "mesh_ordering": "Hilbert".
 * Quadrilaterals / hexahedra of structured topology: each element's local
 * frame is chosen so that neighbouring faces are aligned; other meshes get
 * PRANDTL_EUNSUPPORTED with the reason in prandtl_mesh_last_error().  A mesh
 * with any element that is not a parallelogram / parallelepiped is read with
 * multilinear elements (MFEM's order-1 map of the corners): the descriptor
 * then carries the per-node arrays (node_adj, node_detj, face_node_nor);
 * refinement splits each element in its reference coordinates. */
typedef struct prandtl_mesh prandtl_mesh;
prandtl_status prandtl_mesh_read(const char *path, int order, int refine_levels, int hilbert,
                                 prandtl_mesh **out);
/* Descriptor arrays, valid until prandtl_mesh_destroy.  Boundary faces are
 * {elem1, lface1, -1, attribute - 1} until prandtl_mesh_set_boundary_conditions.
 * hmin (may be NULL): smallest singular value of the element Jacobians at the
 * element centre, as MFEM's GetElementSize(e, 1). */
prandtl_status prandtl_mesh_describe(const prandtl_mesh *m, prandtl_mesh_desc *desc, double *hmin);
/* Boundary attribute of each descriptor face (0 for interior faces and for
 * boundary faces no boundary element names), num_faces entries. */
prandtl_status prandtl_mesh_face_attributes(const prandtl_mesh *m, int *attr);
/* Element attributes, num_elements entries. */
prandtl_status prandtl_mesh_element_attributes(const prandtl_mesh *m, int *attr);
/* Boundary faces of attribute a (1..num_attributes) take BC index
 * bc_of_attribute[a-1]; others take -1 (which prandtl_create rejects). */
prandtl_status prandtl_mesh_set_boundary_conditions(prandtl_mesh *m, const int *bc_of_attribute,
                                                    int num_attributes);
/* Attribute of a Gmsh physical group by entity dimension and name, -1 if none
 * (the reference's boundary names in "boundary_conditions"). */
int prandtl_mesh_attribute(const prandtl_mesh *m, int entity_dim, const char *name);
/* Physical coordinates of every node, [dim][E * (order+1)^dim], byNODES. */
prandtl_status prandtl_mesh_node_coords(const prandtl_mesh *m, double *xyz);
void prandtl_mesh_destroy(prandtl_mesh *m);
/* Text of this thread's last mesh-function error. */
const char *prandtl_mesh_last_error(void);

/* ---- Checkpoint/resume and ParaView output (host only) ----
 * The reference's checkpoint files (Simulation.cpp:1084-1116 save, :350-384
 * load): <folder>/Cycle<ti>/checkpoint_cycle_<ti>.<rank, 8 digits>.chk, an MFEM
 * GridFunction in text (L2_T1_<dim>D_P<order>, VDim dim+2), and
 * checkpoint_cycle_<ti>.json with {"time", "cycle"} (rank 0 writes it).
 * Values are written with 17 significant digits (exact round trip); the
 * loader accepts byNODES and byVDIM orderings and checks the meta file's
 * cycle.  u is byNODES, ndof nodes per field. */
prandtl_status prandtl_checkpoint_save(const char *folder, int cycle, double time, int rank, int dim, int order,
                                       long long ndof, const double *u);
prandtl_status prandtl_checkpoint_load(const char *folder, int cycle, int rank, int dim, int order,
                                       long long ndof, double *u, double *time);
/* ParaView collection as the reference's ParaViewDataCollection writes it
 * (Simulation.cpp:389-410, high-order output at the mesh order):
 * <dir>/<name>/<name>.pvd and Cycle<6 digits>/{data.pvtu, proc000000.vtu} with
 * VTK Lagrange cells and point fields Density, Horizontal/Vertical/Normal V,
 * Pressure, Blending Coeff.  coords: [dim][Ndof] node coordinates (as
 * prandtl_mesh_node_coords); alpha: per element or NULL; binary: base64 data. */
prandtl_status prandtl_paraview_save(const char *dir, const char *name, int cycle, double time, int dim, int order,
                                     int num_elements, const double *coords, const double *u, const double *alpha,
                                     double gamma, int binary);
const char *prandtl_io_last_error(void);

/* ---- RHS without any memory allocation (no counterpart in the reference) ----
 * For callers that cannot call cudaMalloc: code that runs inside another
 * framework's memory pool, embeddings with a fixed device footprint, or code
 * that must not change its footprint after start-up.  Computes the same
 * dudt = L(u) as prandtl_rhs without a handle and without allocating: mesh
 * arrays (the prandtl_mesh_desc pointers), u and dudt must already be in
 * device memory of the current device; everything else lives in one
 * file-scope device array of PRANDTL_NOALLOC_SCRATCH_BYTES that every GPU
 * which loads this library holds until the process exits.
 * Limit: dim*(dim+2)*Ndof doubles of gradients (Navier-Stokes only) plus
 * E*(dim*dim+1) doubles and E*2*dim int4 of tables must fit, each rounded up
 * to 256 bytes (3D N=3: about 4,200 elements); larger meshes return
 * PRANDTL_ETOOLARGE before any device work.
 * The first call on a device looks up the array's device address while that
 * device is current and creates the one CUDA event the call waits on; make
 * that first call before any stream capture.  Every call validates the mesh
 * on the device (faces in range, aligned, each element face listed once,
 * det J > 0), records that event behind the check on `cuda_stream` (a
 * cudaStream_t, NULL for the default stream) and waits for it on the host,
 * bounded by cfg->timeout_s (PRANDTL_ETIMEDOUT), reads the check's 4-byte
 * result, then enqueues the RHS kernels and returns without waiting for them.
 * A failed check returns PRANDTL_EUNSUPPORTED with the reason in
 * prandtl_last_error(NULL).  All calls share the scratch array, which keeps
 * the last call's contents; calls that overlap on the GPU (other streams or
 * host threads on the same device) race.  No lambda_max or
 * blending-coefficient output. */
#define PRANDTL_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
prandtl_status prandtl_rhs_noalloc(const prandtl_mesh_desc *mesh_dev, const prandtl_config *cfg,
                                   const double *u_dev, double *dudt_dev, void *cuda_stream);

/* ---- Batches: many independent solves in one device arena ----------------
 * Extends the reference's one-operator Mult/Step (DGSEMOperator.hpp:105,
 * Simulation.cpp:1010) to many operators at once.  Each solve has its own
 * periodic mesh, order, physics constants, time step and step count; all share
 * the batch's working precision and RK scheme.  Solves stay resident in one
 * device arena (admission by footprint; PRANDTL_ENOMEM when it has no room).
 * Per RK stage, each (dim, order, physics) class runs one persistent launch of
 * the lifting and one of the fused RHS + stage update over the work items of
 * all its solves; the step's launch sequence is captured in a CUDA graph once
 * and replayed.  Solve tables and work lists live in device memory, so solves
 * admitted or retired between advances need no new capture.  Calls on one
 * batch are serialised; batches are independent. */
typedef struct prandtl_batch prandtl_batch;

typedef struct {
    int precision;          /* 0: FP64, 1: FP32 bulk (as prandtl_config.precision) */
    int scheme;             /* PRANDTL_LSRK45 or PRANDTL_RK3SSP */
    size_t arena_bytes;     /* device memory for resident solves; 0: half of the free memory */
    int max_solves;         /* capacity of the solve table; 0: 4096 */
    int steps_per_graph;    /* steps per captured graph; 0: 4 */
    int use_graph;          /* 1: replay captured graphs; 0: launch stage by stage */
    double timeout_s;       /* bound on every host wait; <= 0: 120 s */
} prandtl_batch_config;

typedef struct {
    double dt;              /* time step (with cfl > 0: the first step's) */
    double cfl;             /* > 0: after each step dt = cfl*hmin/(lambda_max (N+1)^2),
                               lambda_max over that step's stages (Simulation.cpp:1013-1018) */
    double hmin;            /* smallest element size, for cfl > 0 */
    int nsteps;             /* steps to take (at most, with t_final) */
    double t_final;         /* > 0: end time; each step takes min(dt, t_final - t) and the solve
                               stops once t >= t_final - 1e-8 dt (Simulation.cpp:1007-1024);
                               0: no end time */
} prandtl_solve_desc;

void prandtl_batch_config_default(prandtl_batch_config *c);
prandtl_status prandtl_batch_create(const prandtl_batch_config *c, prandtl_batch **out);
prandtl_status prandtl_batch_destroy(prandtl_batch *b);
/* Arena bytes a solve of this mesh and physics takes. */
prandtl_status prandtl_batch_footprint(prandtl_batch *b, const prandtl_mesh_desc *mesh,
                                       const prandtl_config *cfg, size_t *bytes);
/* Admit a solve with initial state u0 (byNODES; host or device per ptr_flags).
 * cfg->precision is ignored (the batch's applies).  The mesh tables go up
 * through a 32 MB pinned host ring the first admission allocates (kept until
 * prandtl_batch_destroy); the class tables go up before the next launches. */
prandtl_status prandtl_batch_add(prandtl_batch *b, const prandtl_mesh_desc *mesh, const prandtl_config *cfg,
                                 const double *u0, int ptr_flags, const prandtl_solve_desc *solve, int *id);
/* prandtl_batch_add of n solves (mesh[k], cfg[k], u0[k], sd[k] -> ids[k]):
 * the mesh checks, neighbour tables and geometry rows are prepared on
 * several host threads, then the solves are admitted in order.  Stops at the
 * first solve that fails (its status is returned, the message names the
 * solve); ids of that solve and of those after it are -1, those before it
 * stay admitted. */
prandtl_status prandtl_batch_add_many(prandtl_batch *b, int n, const prandtl_mesh_desc *const *mesh,
                                      const prandtl_config *const *cfg, const double *const *u0, int ptr_flags,
                                      const prandtl_solve_desc *sd, int *ids);
/* Enqueue nsteps steps; each solve stops at its own step count.  Asynchronous. */
prandtl_status prandtl_batch_advance(prandtl_batch *b, int nsteps);
/* Wait (bounded) for the enqueued work. */
prandtl_status prandtl_batch_sync(prandtl_batch *b);
/* Waits, then lists up to `cap` resident solves with no steps left (including
 * solves stopped by a failed state check). */
prandtl_status prandtl_batch_finished(prandtl_batch *b, int *ids, int cap, int *count);
/* Waits, then reports one solve's progress, current dt and last-step lambda_max;
 * PRANDTL_ENONFINITE (outputs still filled) when an RK stage of the solve failed
 * the state check (PRANDTL_HEALTH_*): that solve alone stopped at the end of the
 * step, the others go on. */
prandtl_status prandtl_batch_query(prandtl_batch *b, int id, int *steps_left, int *steps_done,
                                   double *dt, double *lambda_max);
/* Waits, then reports the solve's simulated time (the sum of its steps' dt). */
prandtl_status prandtl_batch_time(prandtl_batch *b, int id, double *t);
/* Waits, then copies the solve's current state (byNODES) out; PRANDTL_ENONFINITE
 * (state still copied) for a solve stopped by the state check. */
prandtl_status prandtl_batch_read(prandtl_batch *b, int id, double *u, int ptr_flags);
/* prandtl_batch_read of n solves with two waits in all: solve ids[k] into
 * u[k].  Every state is copied; a solve stopped by the state check then
 * makes it return PRANDTL_ENONFINITE (the first such id in the message). */
prandtl_status prandtl_batch_read_many(prandtl_batch *b, int n, const int *ids, double *const *u, int ptr_flags);
/* Waits, then the FP64 budgets of the solve's current state, reduced on the device where it
 * resides: out[0 .. nf-1] the integrals of the conserved fields, out[nf] the integral of the
 * entropy function (host memory, nf + 1 doubles; as prandtl_budgets without the rates). */
prandtl_status prandtl_batch_budgets(prandtl_batch *b, int id, double *out);
/* Retire a solve and free its arena range (after the enqueued work). */
prandtl_status prandtl_batch_remove(prandtl_batch *b, int id);
/* Autotuner: per class with resident solves, time `reps` launches of each RHS
 * launch shape on the next step's first stage (which the step recomputes) and
 * keep the fastest. */
prandtl_status prandtl_batch_tune(prandtl_batch *b, int reps);
/* Autotuner inside the steps: the next n_variants steps that advances run
 * (n_variants as prandtl_batch_class_info reports it) time one RHS launch
 * shape each, step v running shape v in every class that has solves, with
 * events around every lifting and RHS launch; the host waits for each of
 * those steps (up to timeout_s).  After the last one each class keeps its
 * fastest shape and the step graphs are rebuilt.  The shapes give
 * bit-identical results, so the tuning does real steps instead of repeated
 * launches.  prandtl_batch_tune cancels a pending tuning in the steps. */
prandtl_status prandtl_batch_tune_in_steps(prandtl_batch *b);
/* Launch shape chosen for a class and the tuned times (ms per launch, -1 when
 * not timed) of each of the *n_variants RHS shapes and of the lifting launch;
 * ms and lift_ms may be NULL. */
prandtl_status prandtl_batch_class_info(prandtl_batch *b, int dim, int order, int parabolic,
                                        int *variant, int *n_variants, double *ms, double *lift_ms);
/* The CUDA stream (cudaStream_t) the batch enqueues on, for event timing. */
void *prandtl_batch_stream(const prandtl_batch *b);
size_t prandtl_batch_device_bytes(const prandtl_batch *b);   /* arena + tables */
size_t prandtl_batch_arena_bytes(const prandtl_batch *b);    /* arena only */
long long prandtl_batch_kernel_launches(const prandtl_batch *b);
const char *prandtl_batch_last_error(const prandtl_batch *b);

/* ---- Serving: a request loop over one batch ------------------------------
 * A worker thread admits submitted solves into a batch as arena room and
 * table slots free up (first come, first served), advances all resident
 * solves `steps_per_tick` steps at a time, and retires finished ones by
 * copying their final state to the caller's buffer.  Requests that arrive
 * while others run join the next tick: their stages share the launches of
 * the resident solves. */
typedef struct prandtl_server prandtl_server;

typedef struct {
    long long submitted, completed, rejected;
    long long steps;                /* batch steps the worker enqueued */
    double dof_updates;             /* sum over completed solves of nodes*fields*steps */
    double busy_s;                  /* wall time with at least one resident solve */
    int resident;                   /* solves resident now */
} prandtl_serve_stats;

prandtl_status prandtl_serve_create(const prandtl_batch_config *c, int steps_per_tick, prandtl_server **out);
/* Copies mesh, config and u0 (host memory); u_out (host, nf*Ndof doubles) receives
 * the final state and must stay valid until the request completes.  A request
 * that can never fit the arena is rejected with PRANDTL_ENOMEM. */
prandtl_status prandtl_serve_submit(prandtl_server *s, const prandtl_mesh_desc *mesh, const prandtl_config *cfg,
                                    const double *u0, const prandtl_solve_desc *solve, double *u_out,
                                    long long *ticket);
/* done = 1 when the result is in u_out; seconds = submit-to-result time. */
prandtl_status prandtl_serve_poll(prandtl_server *s, long long ticket, int *done, double *seconds);
/* Waits up to timeout_s for the request; PRANDTL_ETIMEDOUT otherwise. */
prandtl_status prandtl_serve_wait(prandtl_server *s, long long ticket, double timeout_s, double *seconds);
prandtl_status prandtl_serve_stats_get(prandtl_server *s, prandtl_serve_stats *st);
/* Stops the worker after the resident solves finish (bounded by the batch timeout) and frees everything. */
prandtl_status prandtl_serve_destroy(prandtl_server *s);
const char *prandtl_serve_last_error(prandtl_server *s);

#ifdef __cplusplus
}
#endif
#endif
