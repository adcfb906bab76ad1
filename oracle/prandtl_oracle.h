/*
 * prandtl_oracle.h -- CPU restatement of the Prandtl DGSEM right-hand side and
 * Runge-Kutta step, used ONLY as the test oracle and as the timed CPU baseline.
 *
 * This is test infrastructure.  Nothing in the product (prandtl_b200/, the
 * C-ABI library) links, loads or calls it; only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / --impl reference leg use it, as the checker.
 *
 * Parity status: pinned at the integrator level against the reference's own
 * sources compiled under oracle/_ref (see oracle/ref_harness/).  The MFEM
 * geometry pieces (Gauss-Lobatto rule, affine and multilinear element
 * transformations, face normals) are restated from their mathematics on both
 * sides.
 *
 * Layout conventions (identical to the product's C-ABI):
 *   state u: MFEM Ordering::byNODES, u[f*Ndof + e*Np^dim + node], node
 *            lexicographic with x fastest, Ndof = E*Np^dim, nf = dim+2 fields.
 *   local face lf = 2*dir + side, side 0 is the xi_dir = 0 face, side 1 the
 *            xi_dir = 1 face; face nodes enumerated lexicographically over the
 *            remaining directions (lower direction fastest).
 *   faces:   face_elems[f] = {elem1, lface1, elem2, lface2}; face_nor[f] is the
 *            scaled normal (outward from elem1, |n| = face measure on the
 *            [0,1] reference face), i.e. MFEM's CalcOrtho result.
 */
#ifndef PRANDTL_ORACLE_H
#define PRANDTL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_mesh {
    int dim;              /* 2 or 3 */
    int order;            /* polynomial degree N; Np = N + 1 nodes per direction */
    int num_elements;
    int num_faces;
    const double *elem_adj;   /* [E][dim][dim] adjugate of the (affine) element Jacobian */
    const double *elem_detj;  /* [E] Jacobian determinant */
    const int *face_elems;    /* [F][4] elem1, lface1, elem2, lface2 */
    const double *face_nor;   /* [F][dim] */
    /* Non-affine (multilinear) elements; all three NULL for affine meshes.
     * MFEM evaluates the element transformation at every Gauss-Lobatto node
     * (ElementTransformation::SetIntPoint + AdjugateJacobian / Weight,
     * DGSEMIntegrator.cpp:254-267) and the face transformation at every face
     * point (CalcOrtho, DGSEMIntegrator.cpp:151-222). */
    const double *node_adj;   /* [E][Np^dim][dim][dim] adjugate at each node */
    const double *node_detj;  /* [E][Np^dim] Jacobian determinant at each node */
    const double *face_node_nor; /* [F][Np^(dim-1)][dim] scaled normal at each face node
                                    (face node order of elem1's local face) */
} oracle_mesh;

/* Boundary conditions.  A boundary face is listed in face_elems as
 * {elem1, lface1, -1, bc} with bc an index into oracle_config.bcs.  With
 * parabolic = 1 the slip wall, symmetry and SubsonicInflowPtTtAng types are
 * rejected (the reference defines no viscous treatment for the first two). */
enum {
    ORACLE_BC_STATE = 0,            /* SpecifiedState / SupersonicInflow with a constant state */
    ORACLE_BC_OUTFLOW = 1,          /* SupersonicOutflow: outer state = inner state */
    ORACLE_BC_SLIP_WALL = 2,        /* SlipWall: pressure flux of the normal Riemann problem */
    ORACLE_BC_SYMMETRY = 3,         /* Symmetry: inner state with reflected normal momentum */
    ORACLE_BC_PRESSURE_OUTFLOW = 4, /* SubsonicOutflowP with a constant pressure */
    ORACLE_BC_RIEMANN = 5,          /* RiemannInvariant, constant outer primitive state */
    ORACLE_BC_INFLOW_RV = 6,        /* SubsonicInflowRV, constant density and velocity */
    ORACLE_BC_INFLOW_PTTT = 7,      /* SubsonicInflowPtTtAng, constant pt, Tt, angles */
    ORACLE_BC_NOSLIP_ADIABATIC = 8, /* NoSlipAdiabWall: wall velocity, normal heat flux */
    ORACLE_BC_NOSLIP_ISOTHERMAL = 9,/* NoSlipIsothWall: wall velocity, wall temperature */
    ORACLE_BC_AXIS = 10             /* "axis": the symmetry flux; its nodes at r = 0 are axis nodes */
};
typedef struct oracle_bc {
    int type;
    double state[5];    /* STATE: conserved outer state; RIEMANN: primitive (rho, V, p); INFLOW_RV: rho, V */
    double p;           /* outflow pressure (ORACLE_BC_PRESSURE_OUTFLOW) */
    double pt, Tt, cp;  /* ORACLE_BC_INFLOW_PTTT */
    double theta, phi;  /*   flow angles in degrees */
    double wall_vel[3]; /* NOSLIP_*: wall velocity */
    double heat_flux;   /* NOSLIP_ADIABATIC: normal heat flux per unit face measure */
    double wall_T;      /* NOSLIP_ISOTHERMAL: wall temperature (entropy variable -1/(R_gas T)) */
} oracle_bc;

typedef struct oracle_config {
    double gamma;
    double Pr;
    double mu;
    double R_gas;
    double alpha_max;
    double alpha_min;
    int parabolic;            /* Navier-Stokes: BR1 lifting + viscous fluxes */
    int blending;             /* Persson-Peraire indicator + subcell FV blending */
    int sutherland;           /* Sutherland viscosity law */
    int quirks;               /* 0: reproduce the reference exactly; 1: fixed */
    int surface_dissipation;  /* 1: as the reference; 0: EC surface flux (test switch) */
    int num_bcs;              /* boundary conditions referenced by boundary faces */
    const oracle_bc *bcs;
    int axisymmetric;         /* 2D Euler in (z, r): u is r U (AXISYMMETRIC build of the reference) */
    const double *node_coords;/* [dim][Ndof] node coordinates (axisymmetric: r = coordinate 1) */
    double axis_rho_floor;    /* axis density floor of the recovery; <= 0 selects 1e-12 */
} oracle_config;

/* Axisymmetric form: U recovered from the weighted state rU (the input every
 * axisymmetric oracle_rhs call takes).  Returns 0 on success. */
int oracle_recover_weighted(const oracle_mesh *m, const oracle_config *c, const double *rU, double *U);

/* One RHS evaluation dudt = L(u).  alpha (may be NULL) receives the per-element
 * blending coefficient, lambda_max (may be NULL) the largest |V|+c of any state
 * the fluxes saw.  grad (may be NULL; NS only) receives the lifted primitive
 * gradients [dim][nf*Ndof].  Returns 0 on success. */
int oracle_rhs(const oracle_mesh *m, const oracle_config *c, const double *u,
               double *dudt, double *alpha, double *lambda_max, double *grad,
               int nthreads);

/* nsteps explicit steps of size dt, in place.  scheme: 0 = SSP-RK3 (Shu-Osher,
 * MFEM RK3SSPSolver operation order), 1 = Carpenter-Kennedy LSRK4(5) 2N. */
int oracle_step(const oracle_mesh *m, const oracle_config *c, double *u,
                double t, double dt, int scheme, int nsteps, int nthreads);

/* Gauss-Lobatto nodes/weights on [0,1] and the derivative matrix D[i][l]
 * (Np*Np, row i = node) exactly as the oracle uses them. */
int oracle_gl(int order, double *nodes, double *weights, double *D);

/* Pointwise functions, exported for golden-vector tests. */
double oracle_log_mean(double x, double y);
double oracle_volume_flux(int dim, double gamma, const double *s1, const double *s2,
                          const double *m1, const double *m2, double *F);
double oracle_face_flux(int dim, double gamma, int quirks, int dissipation,
                        const double *s1, const double *s2, const double *nor, double *F);

#ifdef __cplusplus
}
#endif
#endif
