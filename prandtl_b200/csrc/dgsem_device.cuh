// dgsem_device.cuh -- point-wise DGSEM physics on the device (sm_100a).
//
// The two-point fluxes work on per-node primitives computed once per node
// (hoisted out of the O(Np) partner loops): 1/rho, velocity, p, beta = rho/(2p),
// 1/beta, |V|^2 and |V|+c.  Every division of the reference formulas becomes a
// multiplication by one of those reciprocals, and the logarithmic mean needs a
// single reciprocal on its series branch (it also returns 1/mean, which the
// enthalpy term needs).  Each function cites the reference routine whose
// arithmetic it restates; results agree with the reference formulas to a few
// ulp per evaluation.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace prandtl {

// Physics and switch parameters, passed by value to every kernel.
struct PhysParams {
    double gamma, gammaM1, gammaM1Inverse, PrInverse, mu, mu_bulk, R_gas;
    double mu0, T0, Ts, T0pTs;
    double alpha_max, alpha_min, modal_threshold;
    int sutherland;
    int quirks;        // 0: reproduce the reference; 1: fixed
    int dissipation;   // 1: reference surface flux; 0: entropy-conservative (test switch)
    int blending;
};

// A boundary condition (the layout of prandtl_bc).
// INFLOW_PTTT keeps pt, Tt, cp and the unit flow direction vc (formed on the
// host from theta, phi); the no-slip walls keep the wall velocity, the normal
// heat flux and vT = 1 / (R_gas T_wall).
enum BcType : int {
    BC_STATE = 0, BC_OUTFLOW = 1, BC_SLIP_WALL = 2, BC_SYMMETRY = 3, BC_PRESSURE_OUTFLOW = 4,
    BC_RIEMANN = 5, BC_INFLOW_RV = 6, BC_INFLOW_PTTT = 7, BC_NOSLIP_ADIABATIC = 8, BC_NOSLIP_ISOTHERMAL = 9,
    BC_AXIS = 10
};
struct BcDev {
    int type, pad;
    double state[5];
    double p;
    double pt, Tt, cp;
    double vc[3];
    double wall_vel[3];
    double heat_flux, vT;
};

// 1D operator tables for one polynomial order (NP <= 8), row-major [i][l].
struct OpTables {
    double D[64];       // D(i,l) = dL_l/dxi at node i        DGSEMIntegrator.cpp:58-69
    double Dhat[64];    // D + diag(1/w0, ..., -1/wN)         :71-74
    double Dhat2[64];   // 2D + diag(1/w0, ..., -1/wN)        :76-80
    double Vinv[64];    // inverse 1D shifted-Legendre Vandermonde, [mode][node]
    double w[8];        // Gauss-Lobatto weights on [0,1]
    double x[8];        // Gauss-Lobatto nodes on [0,1]
};

template <typename T> __device__ __forceinline__ T dmax(T a, T b) { return a > b ? a : b; }

// 1/x for positive normal x: hardware reciprocal estimate (PTX rcp.approx.ftz.f64)
// refined by two Newton-Raphson steps r <- r + r (1 - x r), each doubling the
// number of correct bits (Markstein, IBM J. Res. Dev. 34 (1990) 111-119).
// Within an ulp of the correctly rounded reciprocal; no special-value paths.
__device__ __forceinline__ double rcp(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}
// FP32 (the FP32-bulk form): the hardware reciprocal estimate alone
// (rcp.approx.ftz.f32, within an ulp), no refinement.
__device__ __forceinline__ float rcp(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Per-node primitives of a conserved state s = (rho, rho v, E).
template <int DIM, typename Real>
struct Prim {
    Real rho, rrho, v[DIM], vsq, beta, rbeta, lam;
    // pressure: p itself from primitives(); in the FP32-bulk form's working
    // copies p - p_ref, with p_ref a pressure of the evaluating element
    Real dp;
};

// ChandrashekarFlux.cpp:22-68 per node: v = m/rho, p = (g-1)(E - rho|v|^2/2),
// beta = rho/(2p), lambda = |v| + sqrt(g p / rho) (BasicOperations.cpp:53-56).
template <int DIM, typename Real>
__device__ __forceinline__ Prim<DIM, Real> primitives(const Real *s, Real gamma, Real gammaM1) {
    constexpr int NF = DIM + 2;
    Prim<DIM, Real> q;
    q.rho = s[0];
    q.rrho = rcp(s[0]);
    q.vsq = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        q.v[d] = s[1 + d] * q.rrho;
        q.vsq += q.v[d] * q.v[d];
    }
    const Real p = gammaM1 * (s[NF - 1] - Real(0.5) * q.rho * q.vsq);
    q.beta = Real(0.5) * q.rho * rcp(p);
    q.rbeta = Real(2) * p * q.rrho;
    q.lam = sqrt(q.vsq) + sqrt(gamma * p * q.rrho);
    q.dp = p;
    return q;
}

// FP32-bulk form: the same primitives in FP32, with the pressure relative to
// pref (dp = p - pref) formed in FP64 from the FP64 state, since it carries the
// low-Mach cancellation: 1/rho and |m|^2/(2 rho) in FP64, everything that only
// enters the O(Np^{d+1}) fluxes (v, beta, 1/beta, |v| + c) in FP32.
template <int DIM>
__device__ __forceinline__ Prim<DIM, float> primitives_mixed(const double *s, double gamma, double gammaM1,
                                                             double pref) {
    constexpr int NF = DIM + 2;
    Prim<DIM, float> q;
    const double rr = rcp(s[0]);
    double mm = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) mm += s[1 + d] * s[1 + d];
    const double p = gammaM1 * (s[NF - 1] - 0.5 * mm * rr);
    q.dp = float(p - pref);
    q.rho = float(s[0]);
    q.rrho = float(rr);
    q.vsq = 0.0f;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        q.v[d] = float(s[1 + d] * rr);
        q.vsq += q.v[d] * q.v[d];
    }
    const float pf = float(p);
    q.beta = 0.5f * q.rho * rcp(pf);
    q.rbeta = 2.0f * pf * q.rrho;
    q.lam = sqrtf(q.vsq) + sqrtf(float(gamma) * pf * q.rrho);
    return q;
}

// BasicOperations.cpp:6-12.  Logarithmic mean of x, y > 0 and its inverse.
// With f = (y-x)/(y+x) and u = f^2 the mean is ((x+y)/2) / P(u),
// P(u) = 1 + u/3 + u^2/5 + u^3/7, on the reference's series branch u < 1e-4
// (the reference writes it as (x+y)*52.5/(105+u(35+u(21+15u)))); there 1/P is
// expanded to third order in a = P-1 (a < 3.5e-5, truncation < 2e-18).
// Otherwise (y-x)/log(y/x), with y/x formed from the hoisted 1/x.
// rs returns 1/(x+y).
// FP32-bulk form: the series branch covers u < 0.04 (|f| < 0.2, ratios
// y/x in [2/3, 3/2]) with terms through u^5 (truncation u^6/13 < 4e-10, below
// FP32 rounding), so smooth flows never take the logarithm and a warp's lanes
// seldom split between the branches; 1/P is the reciprocal estimate.
template <typename Real>
__device__ __forceinline__ void log_mean(Real x, Real y, Real rx, Real &mean, Real &inv_mean, Real &rs) {
    const Real s = x + y, d = y - x;
    rs = rcp(s);
    const Real f = d * rs;
    const Real u = f * f;
    if constexpr (sizeof(Real) == 4) {
        if (u < 0.04f) {
            const float a = u * (1.0f / 3 + u * (1.0f / 5 + u * (1.0f / 7 + u * (1.0f / 9 + u * (1.0f / 11)))));
            inv_mean = 2.0f * rs * (1.0f + a);
            mean = 0.5f * s * rcp(1.0f + a);
            return;
        }
        const float L = log(y * rx);
        mean = d * rcp(L);
        inv_mean = L * rcp(d);
        return;
    }
    if (u < Real(1e-4)) {
        const Real a = u * (Real(1.0 / 3.0) + u * (Real(1.0 / 5.0) + u * Real(1.0 / 7.0)));
        inv_mean = Real(2) * rs * (Real(1) + a);
        mean = Real(0.5) * s * (Real(1) - a * (Real(1) - a * (Real(1) - a)));
    } else {
        const Real L = log(y * rx);
        mean = d * rcp(L);
        inv_mean = L * rcp(d);
    }
}

// ---- FP32-bulk form: two two-point fluxes at once on packed pairs of FP32
// lanes (the paired FADD2 / FMUL2 / FFMA2 instructions of sm_100: one issue
// slot for both).  The arithmetic is that of log_mean / volume_flux below for
// Real = float, applied to (x0, y0) and (x1, y1) side by side.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// Logarithmic means of (x.x, y.x) and (x.y, y.y) with their inverses and
// 1/(x+y): the series branch packed when both lanes take it, else each lane
// through the scalar log_mean.
__device__ __forceinline__ void log_mean2(float2 x, float2 y, float2 rx, float2 &mean, float2 &inv_mean, float2 &rs) {
    const float2 s = add2(x, y), d = sub2(y, x);
    rs = f2(rcp(s.x), rcp(s.y));
    const float2 f = mul2(d, rs);
    const float2 u = mul2(f, f);
    if (u.x < 0.04f && u.y < 0.04f) {
        const float2 a = mul2(u, fma2(u, fma2(u, fma2(u, fma2(u, f2(1.0f / 11), f2(1.0f / 9)), f2(1.0f / 7)),
                                               f2(1.0f / 5)), f2(1.0f / 3)));
        const float2 one_a = add2(f2(1.0f), a);
        inv_mean = mul2(mul2(f2(2.0f), rs), one_a);
        mean = mul2(mul2(f2(0.5f), s), f2(rcp(one_a.x), rcp(one_a.y)));
        return;
    }
    float m0, i0, r0, m1, i1, r1;
    log_mean<float>(x.x, y.x, rx.x, m0, i0, r0);
    log_mean<float>(x.y, y.y, rx.y, m1, i1, r1);
    mean = f2(m0, m1);
    inv_mean = f2(i0, i1);
    rs = f2(r0, r1);
}

// Pressure term of the momentum flux.  FP64: p_hat.  FP32-bulk form: the
// element's constant reference pressure is left out, p_hat - p_ref =
// (beta1 dp1 + beta2 dp2) / (beta1 + beta2) with dp = p - p_ref formed in FP64
// per node, so the O(1/Mach^2) constant that cancels in the flux differencing
// never enters the FP32 sums.  A constant pressure contributes nothing to
// the element's RHS (volume and surface terms cancel for affine elements),
// so this changes only the rounding.
template <int DIM, typename Real>
__device__ __forceinline__ Real momentum_pressure(const Prim<DIM, Real> &a, const Prim<DIM, Real> &b, Real p_hat,
                                                  Real rs_beta) {
    if constexpr (sizeof(Real) == 8) {
        return p_hat;
    } else {
        return fma(a.beta, a.dp, b.beta * b.dp) * rs_beta;
    }
}

// ChandrashekarFlux.cpp:11-83 with metric1 == metric2 == m (affine element,
// so ComputeMean returns m exactly).
template <int DIM, typename Real>
__device__ __forceinline__ void volume_flux(const Prim<DIM, Real> &a, const Prim<DIM, Real> &b,
                                            const Real *m, Real gammaM1Inverse, Real *F) {
    constexpr int NF = DIM + 2;
    Real rho_ln, irho_ln, rs_rho, beta_ln, ibeta_ln, rs_beta;
    log_mean(a.rho, b.rho, a.rrho, rho_ln, irho_ln, rs_rho);
    log_mean(a.beta, b.beta, a.rbeta, beta_ln, ibeta_ln, rs_beta);
    Real vm[DIM], Vn = 0, h = Real(-0.25) * (a.vsq + b.vsq);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        vm[d] = Real(0.5) * (a.v[d] + b.v[d]);
        Vn += vm[d] * m[d];
        h += vm[d] * vm[d];
    }
    const Real p_hat = Real(0.5) * (a.rho + b.rho) * rs_beta;   // 0.5(rho1+rho2)/(beta1+beta2)
    h += Real(0.5) * gammaM1Inverse * ibeta_ln + p_hat * irho_ln;
    const Real F0 = rho_ln * Vn;
    const Real p_mom = momentum_pressure(a, b, p_hat, rs_beta);
    F[0] = F0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) F[1 + d] = F0 * vm[d] + p_mom * m[d];
    F[NF - 1] = F0 * h;
}

// volume_flux (FP32-bulk form) of the pairs (a0, b0) and (a1, b1), each along
// the metric row m, on packed lanes.
template <int DIM>
__device__ __forceinline__ void volume_flux2(const Prim<DIM, float> &a0, const Prim<DIM, float> &b0,
                                             const Prim<DIM, float> &a1, const Prim<DIM, float> &b1,
                                             const float *m, float gammaM1Inverse, float *F0, float *F1) {
    constexpr int NF = DIM + 2;
    const float2 ar = f2(a0.rho, a1.rho), br = f2(b0.rho, b1.rho);
    const float2 ab = f2(a0.beta, a1.beta), bb = f2(b0.beta, b1.beta);
    float2 rho_ln, irho_ln, rs_rho, beta_ln, ibeta_ln, rs_beta;
    log_mean2(ar, br, f2(a0.rrho, a1.rrho), rho_ln, irho_ln, rs_rho);
    log_mean2(ab, bb, f2(a0.rbeta, a1.rbeta), beta_ln, ibeta_ln, rs_beta);
    float2 vm[DIM], Vn = f2(0.0f), h = mul2(f2(-0.25f), add2(f2(a0.vsq, a1.vsq), f2(b0.vsq, b1.vsq)));
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        vm[d] = mul2(f2(0.5f), add2(f2(a0.v[d], a1.v[d]), f2(b0.v[d], b1.v[d])));
        Vn = fma2(vm[d], f2(m[d]), Vn);
        h = fma2(vm[d], vm[d], h);
    }
    const float2 p_hat = mul2(mul2(f2(0.5f), add2(ar, br)), rs_beta);
    h = add2(h, fma2(mul2(f2(0.5f), f2(gammaM1Inverse)), ibeta_ln, mul2(p_hat, irho_ln)));
    const float2 Fm = mul2(rho_ln, Vn);
    // momentum_pressure (FP32): (beta1 dp1 + beta2 dp2) / (beta1 + beta2)
    const float2 p_mom = mul2(fma2(ab, f2(a0.dp, a1.dp), mul2(bb, f2(b0.dp, b1.dp))), rs_beta);
    F0[0] = Fm.x;
    F1[0] = Fm.y;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        const float2 Fd = fma2(Fm, vm[d], mul2(p_mom, f2(m[d])));
        F0[1 + d] = Fd.x;
        F1[1 + d] = Fd.y;
    }
    const float2 Fe = mul2(Fm, h);
    F0[NF - 1] = Fe.x;
    F1[NF - 1] = Fe.y;
}

// ChandrashekarFlux.cpp:85-161: entropy-conservative flux minus
// 0.5*lambda*jump*|n| (conserved jumps for mass and momentum, the entropy
// variable based `diss` for energy).  s1, s2 are the conserved inputs (for the
// momentum jumps); quirk3 reproduces `rho_mean * dw + w_mean` (:131) in 3D.
template <int DIM, typename Real>
__device__ __forceinline__ void face_flux(const Real *s1, const Prim<DIM, Real> &a, const Real *s2,
                                          const Prim<DIM, Real> &b, const Real *nor, Real gammaM1Inverse,
                                          bool quirk3, bool dissipation, Real *flux) {
    constexpr int NF = DIM + 2;
    Real nn = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) nn += nor[d] * nor[d];
    Real rho_ln, irho_ln, rs_rho, beta_ln, ibeta_ln, rs_beta;
    log_mean(a.rho, b.rho, a.rrho, rho_ln, irho_ln, rs_rho);
    log_mean(a.beta, b.beta, a.rbeta, beta_ln, ibeta_ln, rs_beta);
    const Real rho_mean = Real(0.5) * (a.rho + b.rho);
    const Real drho = b.rho - a.rho;
    Real vm[DIM], Vn = 0, h = Real(-0.25) * (a.vsq + b.vsq), diss = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        vm[d] = Real(0.5) * (a.v[d] + b.v[d]);
        const Real dv = b.v[d] - a.v[d];
        Vn += vm[d] * nor[d];
        h += vm[d] * vm[d];
        if (DIM == 3 && d == 2 && quirk3)
            diss += Real(0.5) * drho * a.v[d] * b.v[d] + rho_mean * dv + vm[d];
        else
            diss += Real(0.5) * drho * a.v[d] * b.v[d] + rho_mean * dv * vm[d];
    }
    const Real p_hat = rho_mean * rs_beta;
    h += Real(0.5) * gammaM1Inverse * ibeta_ln + p_hat * irho_ln;
    diss += Real(0.5) * drho * gammaM1Inverse * ibeta_ln + Real(0.5) * rho_mean * gammaM1Inverse * (b.rbeta - a.rbeta);
    const Real hl = dissipation ? Real(0.5) * dmax(a.lam, b.lam) * sqrt(nn) : Real(0);
    const Real F0 = rho_ln * Vn;
    const Real p_mom = momentum_pressure(a, b, p_hat, rs_beta);
    flux[0] = F0 - hl * drho;
#pragma unroll
    for (int d = 0; d < DIM; ++d) flux[1 + d] = F0 * vm[d] + p_mom * nor[d] - hl * (s2[1 + d] - s1[1 + d]);
    flux[NF - 1] = F0 * h - hl * diss;
}

// NavierStokesFlux.cpp:12-90 from primitives (rho, v, p): the stress tensor with
// the bulk coefficient mu_bulk = 2/3 and the heat flux lambda*cv grad T with
// lambda = mu gamma / Pr; row 0 (mass) is zero.  dq[c] = d(rho, v, p)/dx_c.
// Calls `emit(f, c, value)` for f = 1..NF-1, c = 0..DIM-1 so callers can
// project or store without holding the whole matrix.
template <int DIM, typename Real, typename Emit>
__device__ __forceinline__ void viscous_flux(Real rho, Real rrho, const Real *v, Real p,
                                             const Real (*dq)[DIM + 2], const PhysParams &P, Emit emit) {
    constexpr int NF = DIM + 2;
    Real mu = Real(P.mu);
    if (P.sutherland) {   // NavierStokesFlux.hpp:32-36
        const Real T = p * rrho * rcp(Real(P.R_gas));
        mu = Real(P.mu0) * Real(P.T0pTs) * rcp(T + Real(P.Ts)) * (T * rcp(Real(P.T0))) * sqrt(T * rcp(Real(P.T0)));
    }
    const Real lambda = mu * Real(P.gamma) * Real(P.PrInverse);
    Real div = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) div += dq[d][1 + d];
    const Real gm1i_r = Real(P.gammaM1Inverse) * rrho, pr = p * rrho, mub = Real(P.mu_bulk);
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
        Real e = 0;
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
            const Real tau = (r == c) ? mu * (Real(2) * dq[c][1 + r] - mub * div)
                                      : mu * (dq[c][1 + r] + dq[r][1 + c]);
            emit(1 + r, c, tau);
            e += v[r] * tau;
        }
        const Real cv_dT = gm1i_r * (dq[c][NF - 1] - pr * dq[c][0]);
        emit(NF - 1, c, e + lambda * cv_dT);
    }
}

// BasicOperations.cpp:81-104: entropy variables with beta = rho/p,
// s = log(p rho^-gamma) = log p - gamma log rho.
template <int DIM, typename Real>
__device__ __forceinline__ void conserv2entropy(const Real *s, const PhysParams &P, Real *v) {
    constexpr int NF = DIM + 2;
    const Real minv = rcp(s[0]);
    Real vel[DIM], vv = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        vel[d] = s[1 + d] * minv;
        vv += vel[d] * vel[d];
    }
    const Real v_sq = Real(0.5) * vv;
    const Real p = Real(P.gammaM1) * (s[NF - 1] - s[0] * v_sq);
    const Real beta = s[0] * rcp(p);
    const Real sent = log(p) - Real(P.gamma) * log(s[0]);
    v[0] = (Real(P.gamma) - sent) * Real(P.gammaM1Inverse) - beta * v_sq;
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[1 + d] = beta * vel[d];
    v[NF - 1] = -beta;
}

// FP32-bulk form: entropy variables relative to those of a reference node of
// the evaluating element.  Constants drop out of the lifted gradients (the
// derivative of a constant and the jump of a shared constant are zero), so
// only the O(1) variation is carried in FP32: s - s_ref = log1p(p/p_ref - 1) -
// gamma log1p(rho/rho_ref - 1) from ratios formed in FP64, and
// beta v^2/2 - (beta v^2/2)_ref, beta_ref - beta in FP64 before rounding.
struct EntropyRef {
    double rp, rrho, beta, bvsq;   // 1/p, 1/rho, rho/p, beta |v|^2 / 2 of the reference node
};
template <int DIM>
__device__ __forceinline__ EntropyRef entropy_ref(const double *s, const PhysParams &P) {
    constexpr int NF = DIM + 2;
    EntropyRef R;
    R.rrho = rcp(s[0]);
    double vv = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        const double vd = s[1 + d] * R.rrho;
        vv += vd * vd;
    }
    const double p = P.gammaM1 * (s[NF - 1] - s[0] * (0.5 * vv));
    R.rp = rcp(p);
    R.beta = s[0] * R.rp;
    R.bvsq = R.beta * (0.5 * vv);
    return R;
}
template <int DIM>
__device__ __forceinline__ void conserv2entropy_rel(const double *s, const PhysParams &P, const EntropyRef &R,
                                                    float *v) {
    constexpr int NF = DIM + 2;
    const double minv = rcp(s[0]);
    double vel[DIM], vv = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        vel[d] = s[1 + d] * minv;
        vv += vel[d] * vel[d];
    }
    const double v_sq = 0.5 * vv;
    const double p = P.gammaM1 * (s[NF - 1] - s[0] * v_sq);
    const double beta = s[0] * rcp(p);
    const float srel = log1pf(float(fma(p, R.rp, -1.0))) - float(P.gamma) * log1pf(float(fma(s[0], R.rrho, -1.0)));
    v[0] = -srel * float(P.gammaM1Inverse) - float(fma(beta, v_sq, -R.bvsq));
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[1 + d] = float(beta * vel[d]);
    v[NF - 1] = float(R.beta - beta);
}

// BasicOperations.cpp:126-170 for one node and one derivative direction.
// quirks == 0 keeps the reference's aliasing: `vel /= state(0)` turns the
// momentum slots of its state copy into velocity before the density-gradient
// line reads them.
template <int DIM, typename Real>
__device__ __forceinline__ void entropygrad2primgrad(const Real *s, const PhysParams &P, Real *g) {
    constexpr int NF = DIM + 2;
    const Real minv = rcp(s[0]);
    Real vel[DIM], vv = 0, gs[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) gs[f] = g[f];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        vel[d] = s[1 + d] * minv;
        vv += vel[d] * vel[d];
    }
    const Real v_sq = Real(0.5) * vv;
    const Real p = Real(P.gammaM1) * (s[NF - 1] - s[0] * v_sq);
    const Real KE = v_sq * s[0];
    const Real pr = p * minv, rp = s[0] * rcp(p);
    Real acc = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        g[1 + d] = pr * (gs[1 + d] + vel[d] * gs[NF - 1]);
        acc += ((P.quirks == 0) ? vel[d] : s[1 + d]) * g[1 + d];
    }
    g[0] = s[0] * gs[0] - gs[NF - 1] * (KE - p * Real(P.gammaM1Inverse)) + rp * acc;
    g[NF - 1] = pr * (g[0] + p * gs[NF - 1]);
}

}   // namespace prandtl
