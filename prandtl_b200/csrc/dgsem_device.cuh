// dgsem_device.cuh -- point-wise DGSEM physics on the device (sm_100a).
//
// Each function states the reference routine whose arithmetic it implements.
// Arithmetic is templated on the working type `Real` (double for the FP64
// path, float for the FP32-bulk form).
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

// BasicOperations.cpp:6-12: logarithmic mean with the series branch for
// u = ((xi-1)/(xi+1))^2 < 1e-4.
template <typename Real>
__device__ __forceinline__ Real log_mean(Real x, Real y) {
    const Real xi = y / x;
    const Real u = (xi * (xi - Real(2)) + Real(1)) / (xi * (xi + Real(2)) + Real(1));
    if (u < Real(1e-4))
        return (x + y) * Real(52.5) / (Real(105) + u * (Real(35) + u * (Real(21) + Real(15) * u)));
    return (y - x) / log(xi);
}

// ChandrashekarFlux.cpp:11-83 with metric1 == metric2 == m (affine element,
// so ComputeMean returns m exactly).  F has DIM+2 entries.
template <int DIM, typename Real>
__device__ __forceinline__ void volume_flux(const Real *s1, const Real *s2, const Real *m,
                                            Real gammaM1, Real gammaM1Inverse, Real *F) {
    constexpr int NF = DIM + 2;
    const Real rho1 = s1[0], rho2 = s2[0];
    const Real rho_ln = log_mean(rho1, rho2);
    Real vel1[DIM], vel2[DIM], vm[DIM];
    Real V_sq1 = 0, V_sq2 = 0, Vn = 0, h_hat = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        vel1[d] = s1[1 + d] / rho1;
        vel2[d] = s2[1 + d] / rho2;
        vm[d] = Real(0.5) * (vel1[d] + vel2[d]);
        V_sq1 += vel1[d] * vel1[d];
        V_sq2 += vel2[d] * vel2[d];
        Vn += vm[d] * m[d];
        h_hat += Real(-0.25) * (vel1[d] * vel1[d] + vel2[d] * vel2[d]) + vm[d] * vm[d];
    }
    const Real p1 = gammaM1 * (s1[NF - 1] - Real(0.5) * rho1 * V_sq1);
    const Real p2 = gammaM1 * (s2[NF - 1] - Real(0.5) * rho2 * V_sq2);
    const Real beta1 = Real(0.5) * rho1 / p1, beta2 = Real(0.5) * rho2 / p2;
    const Real beta_ln = log_mean(beta1, beta2);
    const Real p_hat = Real(0.5) * (rho1 + rho2) / (beta1 + beta2);
    h_hat += Real(0.5) / beta_ln * gammaM1Inverse + p_hat / rho_ln;
    F[0] = rho_ln * Vn;
#pragma unroll
    for (int d = 0; d < DIM; ++d) F[1 + d] = Vn * (rho_ln * vm[d]) + p_hat * m[d];
    F[NF - 1] = rho_ln * Vn * h_hat;
}

// ChandrashekarFlux.cpp:85-161: entropy-conservative flux minus the scalar
// dissipation 0.5*lambda*jump*|n|.  quirk3 reproduces `rho_mean * dw + w_mean`
// (:131) in 3D.
template <int DIM, typename Real>
__device__ __forceinline__ void face_flux(const Real *s1, const Real *s2, const Real *nor,
                                          Real gamma, Real gammaM1, Real gammaM1Inverse,
                                          bool quirk3, bool dissipation, Real *flux) {
    constexpr int NF = DIM + 2;
    Real nn = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) nn += nor[d] * nor[d];
    const Real nor_mag = sqrt(nn);
    const Real rho1 = s1[0], rho2 = s2[0];
    const Real rho_mean = Real(0.5) * (rho1 + rho2);
    const Real rho_ln = log_mean(rho1, rho2);
    const Real drho = rho2 - rho1;
    Real vm[DIM];
    Real V_sq1 = 0, V_sq2 = 0, Vn = 0, h_hat = 0, diss = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        const Real a1 = s1[1 + d] / rho1, a2 = s2[1 + d] / rho2;
        vm[d] = Real(0.5) * (a1 + a2);
        const Real da = a2 - a1;
        V_sq1 += a1 * a1;
        V_sq2 += a2 * a2;
        Vn += vm[d] * nor[d];
        h_hat += Real(-0.25) * (a1 * a1 + a2 * a2) + vm[d] * vm[d];
        if (DIM == 3 && d == 2 && quirk3)
            diss += Real(0.5) * drho * a1 * a2 + rho_mean * da + vm[d];
        else
            diss += Real(0.5) * drho * a1 * a2 + rho_mean * da * vm[d];
    }
    const Real p1 = gammaM1 * (s1[NF - 1] - Real(0.5) * rho1 * V_sq1);
    const Real p2 = gammaM1 * (s2[NF - 1] - Real(0.5) * rho2 * V_sq2);
    Real lambda = sqrt(V_sq1) + sqrt(gamma * p1 / rho1);
    lambda = dmax(lambda, sqrt(V_sq2) + sqrt(gamma * p2 / rho2));
    const Real beta1 = Real(0.5) * rho1 / p1, beta2 = Real(0.5) * rho2 / p2;
    const Real beta_ln = log_mean(beta1, beta2);
    const Real p_hat = Real(0.5) * (rho1 + rho2) / (beta1 + beta2);
    h_hat += Real(0.5) / beta_ln * gammaM1Inverse + p_hat / rho_ln;
    diss += Real(0.5) * drho * gammaM1Inverse / beta_ln +
            Real(0.5) * rho_mean * gammaM1Inverse * (Real(1) / beta2 - Real(1) / beta1);
    const Real hl = dissipation ? Real(0.5) * lambda * nor_mag : Real(0);
    flux[0] = rho_ln * Vn - hl * (rho2 - rho1);
#pragma unroll
    for (int d = 0; d < DIM; ++d)
        flux[1 + d] = Vn * (rho_ln * vm[d]) + p_hat * nor[d] - hl * (s2[1 + d] - s1[1 + d]);
    flux[NF - 1] = rho_ln * Vn * h_hat - hl * diss;
}

// NavierStokesFlux.cpp:12-90 (with Conserv2Prim, BasicOperations.cpp:172-186).
// As in the reference, ComputePressure overwrites the momentum slots of
// `state` with velocity (BasicOperations.cpp:33-34); callers that must not
// see that pass a copy.  Fv is [NF][DIM]; row 0 is zero.
template <int DIM, typename Real>
__device__ __forceinline__ void viscous_flux(Real *state, const Real (*dq)[DIM + 2],
                                             const PhysParams &P, Real (*Fv)[DIM]) {
    constexpr int NF = DIM + 2;
    Real prim[NF];
    prim[0] = state[0];
#pragma unroll
    for (int d = 0; d < DIM; ++d) prim[1 + d] = state[1 + d] / state[0];
    {
        const Real minv = Real(1) / state[0];
        Real vv = 0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) state[1 + d] *= minv;
#pragma unroll
        for (int d = 0; d < DIM; ++d) vv += state[1 + d] * state[1 + d];
        prim[NF - 1] = Real(P.gammaM1) * (state[NF - 1] - Real(0.5) * state[0] * vv);
    }
    Real mu = Real(P.mu);
    if (P.sutherland) {   // NavierStokesFlux.hpp:32-36
        const Real T = prim[NF - 1] / (prim[0] * Real(P.R_gas));
        mu = Real(P.mu0) * Real(P.T0pTs) / (T + Real(P.Ts)) * (T / Real(P.T0)) * sqrt(T / Real(P.T0));
    }
    const Real lambda = mu * Real(P.gamma) * Real(P.PrInverse);
    Real div = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) div += dq[d][1 + d];
    const Real gm1i = Real(P.gammaM1Inverse), mub = Real(P.mu_bulk);
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
        Fv[0][c] = 0;
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
            // tau(r, c): diagonal mu(2 du_r/dx_r - mu_bulk div), off-diagonal mu(du_r/dx_c + du_c/dx_r)
            if (r == c)
                Fv[1 + r][c] = mu * (Real(2) * dq[c][1 + r] - mub * div);
            else
                Fv[1 + r][c] = mu * (dq[c][1 + r] + dq[r][1 + c]);
        }
        const Real cv_dT = gm1i / prim[0] * (dq[c][NF - 1] - prim[NF - 1] / prim[0] * dq[c][0]);
        Real e = 0;
#pragma unroll
        for (int r = 0; r < DIM; ++r) e += prim[1 + r] * Fv[1 + r][c];
        Fv[NF - 1][c] = e + lambda * cv_dT;
    }
}

// BasicOperations.cpp:81-104 on a private copy of the node state.
template <int DIM, typename Real>
__device__ __forceinline__ void conserv2entropy(const Real *s, const PhysParams &P, Real *v) {
    constexpr int NF = DIM + 2;
    const Real minv = Real(1) / s[0];
    Real vel[DIM], vv = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) vel[d] = s[1 + d] * minv;
#pragma unroll
    for (int d = 0; d < DIM; ++d) vv += vel[d] * vel[d];
    const Real v_sq = Real(0.5) * vv;
    const Real p = Real(P.gammaM1) * (s[NF - 1] - s[0] * v_sq);
    const Real beta = s[0] / p;
    const Real sent = log(p * pow(s[0], -Real(P.gamma)));
    v[0] = (Real(P.gamma) - sent) * Real(P.gammaM1Inverse) - beta * v_sq;
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[1 + d] = beta * vel[d];
    v[NF - 1] = -beta;
}

// BasicOperations.cpp:126-170 for one node and one derivative direction.
// quirks == 0 keeps the reference's aliasing (`vel /= state(0)` turns the
// momentum slots of the state copy into velocity before the density-gradient
// line reads them).
template <int DIM, typename Real>
__device__ __forceinline__ void entropygrad2primgrad(const Real *s_in, const PhysParams &P, Real *g) {
    constexpr int NF = DIM + 2;
    Real s[NF], gs[NF], vel[DIM];
#pragma unroll
    for (int f = 0; f < NF; ++f) { s[f] = s_in[f]; gs[f] = g[f]; }
    const Real minv = Real(1) / s[0];
    Real vv = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) vel[d] = s[1 + d] * minv;
#pragma unroll
    for (int d = 0; d < DIM; ++d) vv += vel[d] * vel[d];
    if (P.quirks == 0) {
#pragma unroll
        for (int d = 0; d < DIM; ++d) s[1 + d] = vel[d];
    }
    const Real v_sq = Real(0.5) * vv;
    const Real p = Real(P.gammaM1) * (s[NF - 1] - s[0] * v_sq);
    const Real KE = v_sq * s[0];
    const Real pr = p / s[0];
    Real acc = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        g[1 + d] = pr * (gs[1 + d] + vel[d] * gs[NF - 1]);
        acc += s[1 + d] * g[1 + d];
    }
    g[0] = s[0] * gs[0] - gs[NF - 1] * (KE - p * Real(P.gammaM1Inverse)) + s[0] / p * acc;
    g[NF - 1] = pr * (g[0] + p * gs[NF - 1]);
}

}   // namespace prandtl
