// prandtl_oracle.cpp -- CPU restatement of the Prandtl DGSEM RHS (test oracle).
//
// TEST INFRASTRUCTURE ONLY: the product never links or calls this file.  It is
// the checker for the CUDA path and the timed CPU baseline ("port").
//
// Every routine follows the cited reference routine line by line, in the same
// floating-point operation order, including the reference's deterministic bugs
// (quirks == 0).  With quirks == 1 those bugs are fixed:
//   Q1  NS element viscous flux uses the state of local node Np^d-1
//       (stale member id1)                        DGSEMIntegrator.cpp:620,770
//   Q2  3D NS zeta loop stores g where h is meant DGSEMIntegrator.cpp:702
//   Q3  3D face-flux energy dissipation `rho_mean * dw + w_mean`
//                                                 ChandrashekarFlux.cpp:131
//   Q7  EntropyGrad2PrimGrad: `vel /= state(0)` aliases the state copy, so the
//       density gradient uses velocity where momentum is meant
//                                                 BasicOperations.cpp:137-138,165
//   Q8  ComputePressure aliases its const input (`V /= state(0)` through a
//       wrapping Vector), so after ComputeViscousFlux the NS face traces hold
//       velocity in the momentum slots when ComputeFaceFlux reads them
//                                                 BasicOperations.cpp:31-37,
//                                                 NavierStokesFlux.cpp:14,
//                                                 DGSEMIntegrator.cpp:471-481
// MFEM pieces (not vendored in the reference) are restated from their math:
// Gauss-Lobatto rule on [0,1], affine ElementTransformation (Weight, adjugate),
// CalcOrtho normals (given by the mesh descriptor), shifted Legendre
// Poly_1D::CalcLegendre, DenseMatrix::Invert, Vector ops (operator/= multiplies
// by the reciprocal), RK3SSPSolver operation order.
#include "prandtl_oracle.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kLogMeanEps = 1e-4;        // BasicOperations.hpp:9
constexpr double kSharpness = 9.21024;      // DGSEMOperator.hpp:50

// ---------------------------------------------------------------- pointwise
// BasicOperations.cpp:6-12
double log_mean(double x, double y) {
    double xi = y / x;
    double u = (xi * (xi - 2.0) + 1.0) / (xi * (xi + 2.0) + 1);
    double ln_mean = (u < kLogMeanEps)
                         ? (x + y) * 52.5 / (105.0 + u * (35.0 + u * (21.0 + 15.0 * u)))
                         : (y - x) / std::log(xi);
    return ln_mean;
}

// BasicOperations.cpp:53-56 with b = 0
double sound_speed(double p, double rho, double gamma) {
    return std::sqrt(gamma * p / (1.0 - 0.0 * rho) / rho);
}

// mfem::Vector::Norml2 for the small normals used here
double norml2(const double *v, int n) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += v[i] * v[i];
    return std::sqrt(s);
}

// ChandrashekarFlux.cpp:11-83
double volume_flux(int dim, double gamma, const double *s1, const double *s2,
                   const double *m1, const double *m2, double *F) {
    const int nf = dim + 2;
    const double gammaM1 = gamma - 1.0;
    const double gammaM1Inverse = 1.0 / gammaM1;
    double metric[3], mom[3];
    for (int d = 0; d < dim; ++d) {   // ComputeMean: mean = x; mean += y; mean *= 0.5
        metric[d] = m1[d];
        metric[d] += m2[d];
        metric[d] *= 0.5;
    }
    double rho1 = s1[0], rho2 = s2[0];
    double rho_ln = log_mean(rho1, rho2);
    double u1 = s1[1] / rho1, u2 = s2[1] / rho2;
    double u_mean = 0.5 * (u1 + u2);
    double V_sq1 = u1 * u1, V_sq2 = u2 * u2;
    double Vn = u_mean * metric[0];
    mom[0] = rho_ln * u_mean;
    double h_hat = -0.25 * (u1 * u1 + u2 * u2) + u_mean * u_mean;
    if (dim > 1) {
        double v1 = s1[2] / rho1, v2 = s2[2] / rho2;
        double v_mean = 0.5 * (v1 + v2);
        V_sq1 += v1 * v1;
        V_sq2 += v2 * v2;
        Vn += v_mean * metric[1];
        mom[1] = rho_ln * v_mean;
        h_hat += -0.25 * (v1 * v1 + v2 * v2) + v_mean * v_mean;
        if (dim > 2) {
            double w1 = s1[3] / rho1, w2 = s2[3] / rho2;
            double w_mean = 0.5 * (w1 + w2);
            V_sq1 += w1 * w1;
            V_sq2 += w2 * w2;
            Vn += w_mean * metric[2];
            mom[2] = rho_ln * w_mean;
            h_hat += -0.25 * (w1 * w1 + w2 * w2) + w_mean * w_mean;
        }
    }
    double p1 = gammaM1 * (s1[nf - 1] - 0.5 * rho1 * V_sq1);
    double p2 = gammaM1 * (s2[nf - 1] - 0.5 * rho2 * V_sq2);
    double lambda_max = std::sqrt(V_sq1) + sound_speed(p1, rho1, gamma);
    lambda_max = std::max(lambda_max, std::sqrt(V_sq2) + sound_speed(p2, rho2, gamma));
    double beta1 = 0.5 * rho1 / p1, beta2 = 0.5 * rho2 / p2;
    double beta_ln = log_mean(beta1, beta2);
    double p_hat = 0.5 * (rho1 + rho2) / (beta1 + beta2);
    h_hat += 0.5 / beta_ln * gammaM1Inverse + p_hat / rho_ln;
    F[0] = rho_ln * Vn;
    for (int d = 0; d < dim; ++d) F[1 + d] = Vn * mom[d] + p_hat * metric[d];
    F[1 + dim] = rho_ln * Vn * h_hat;
    return lambda_max;
}

// ChandrashekarFlux.cpp:85-161 (Q3 at :131)
double face_flux(int dim, double gamma, int quirks, int dissipation, const double *s1,
                 const double *s2, const double *nor, double *flux) {
    const int nf = dim + 2;
    const double gammaM1 = gamma - 1.0;
    const double gammaM1Inverse = 1.0 / gammaM1;
    double mom[3];
    double nor_mag = norml2(nor, dim);
    double rho1 = s1[0], rho2 = s2[0];
    double rho_mean = 0.5 * (rho1 + rho2);
    double rho_ln = log_mean(rho1, rho2);
    double drho = rho2 - rho1;
    double u1 = s1[1] / rho1, u2 = s2[1] / rho2;
    double u_mean = 0.5 * (u1 + u2);
    double du = u2 - u1;
    double V_sq1 = u1 * u1, V_sq2 = u2 * u2;
    double Vn = u_mean * nor[0];
    mom[0] = rho_ln * u_mean;
    double h_hat = -0.25 * (u1 * u1 + u2 * u2) + u_mean * u_mean;
    double diss = 0.5 * drho * u1 * u2 + rho_mean * du * u_mean;
    if (dim > 1) {
        double v1 = s1[2] / rho1, v2 = s2[2] / rho2;
        double v_mean = 0.5 * (v1 + v2);
        double dv = v2 - v1;
        V_sq1 += v1 * v1;
        V_sq2 += v2 * v2;
        Vn += v_mean * nor[1];
        mom[1] = rho_ln * v_mean;
        h_hat += -0.25 * (v1 * v1 + v2 * v2) + v_mean * v_mean;
        diss += 0.5 * drho * v1 * v2 + rho_mean * dv * v_mean;
        if (dim > 2) {
            double w1 = s1[3] / rho1, w2 = s2[3] / rho2;
            double w_mean = 0.5 * (w1 + w2);
            double dw = w2 - w1;
            V_sq1 += w1 * w1;
            V_sq2 += w2 * w2;
            Vn += w_mean * nor[2];
            mom[2] = rho_ln * w_mean;
            h_hat += -0.25 * (w1 * w1 + w2 * w2) + w_mean * w_mean;
            if (quirks == 0)
                diss += 0.5 * drho * w1 * w2 + rho_mean * dw + w_mean;   // Q3
            else
                diss += 0.5 * drho * w1 * w2 + rho_mean * dw * w_mean;
        }
    }
    double p1 = gammaM1 * (s1[nf - 1] - 0.5 * rho1 * V_sq1);
    double p2 = gammaM1 * (s2[nf - 1] - 0.5 * rho2 * V_sq2);
    double lambda_max = std::sqrt(V_sq1) + sound_speed(p1, rho1, gamma);
    lambda_max = std::max(lambda_max, std::sqrt(V_sq2) + sound_speed(p2, rho2, gamma));
    double beta1 = 0.5 * rho1 / p1, beta2 = 0.5 * rho2 / p2;
    double beta_ln = log_mean(beta1, beta2);
    double p_hat = 0.5 * (rho1 + rho2) / (beta1 + beta2);
    h_hat += 0.5 / beta_ln * gammaM1Inverse + p_hat / rho_ln;
    diss += 0.5 * drho * gammaM1Inverse / beta_ln +
            0.5 * rho_mean * gammaM1Inverse * (1.0 / beta2 - 1.0 / beta1);
    if (dissipation) {
        flux[0] = rho_ln * Vn - 0.5 * lambda_max * (rho2 - rho1) * nor_mag;
        for (int d = 0; d < dim; ++d)
            flux[1 + d] = Vn * mom[d] + p_hat * nor[d] -
                          0.5 * lambda_max * (s2[1 + d] - s1[1 + d]) * nor_mag;
        flux[1 + dim] = rho_ln * Vn * h_hat - 0.5 * lambda_max * diss * nor_mag;
    } else {
        flux[0] = rho_ln * Vn;
        for (int d = 0; d < dim; ++d) flux[1 + d] = Vn * mom[d] + p_hat * nor[d];
        flux[1 + dim] = rho_ln * Vn * h_hat;
    }
    return lambda_max;
}

// BasicOperations.cpp:31-37.  `Vector V(state.GetData()+1, ...)` wraps the
// caller's storage, so the momentum slots are overwritten with velocity (Q8).
double compute_pressure_inplace(double *state, int nf, double gammaM1) {
    const double m = 1.0 / state[0];   // Vector::operator/= multiplies by 1/c
    double vv = 0.0;
    for (int i = 1; i < nf - 1; ++i) state[i] *= m;
    for (int i = 1; i < nf - 1; ++i) vv += state[i] * state[i];
    return gammaM1 * (state[nf - 1] - 0.5 * state[0] * vv);
}

struct Phys {
    double gamma, gammaM1, gammaM1Inverse, PrInverse, mu, mu_bulk, R_gas, mu0, T0, Ts, T0pTs;
    int sutherland;
};

// NavierStokesFlux.cpp:12-58 (3D) / :60-90 (2D).  `state` is modified in place
// exactly as the reference's Conserv2Prim -> ComputePressure does (Q8).
// Fv is [nf][dim]; row 0 stays zero (the reference never writes it).
void viscous_flux(int dim, const Phys &P, double *state, const double *dqdx,
                  const double *dqdy, const double *dqdz, double *Fv) {
    const int nf = dim + 2;
    double prim[5];
    // BasicOperations.cpp:172-186
    prim[0] = state[0];
    prim[1] = state[1] / state[0];
    if (nf > 3) {
        prim[2] = state[2] / state[0];
        if (nf > 4) prim[3] = state[3] / state[0];
    }
    prim[nf - 1] = compute_pressure_inplace(state, nf, P.gammaM1);
    double mu = P.mu;
    if (P.sutherland) {   // NavierStokesFlux.hpp:32-36
        double T = prim[nf - 1] / (prim[0] * P.R_gas);
        mu = P.mu0 * P.T0pTs / (T + P.Ts) * (T / P.T0) * std::sqrt(T / P.T0);
    }
    double lambda = mu * P.gamma * P.PrInverse;
    for (int i = 0; i < nf * dim; ++i) Fv[i] = 0.0;
    if (dim == 3) {
        const double drdx = dqdx[0], dudx = dqdx[1], dvdx = dqdx[2], dwdx = dqdx[3], dpdx = dqdx[4];
        const double drdy = dqdy[0], dudy = dqdy[1], dvdy = dqdy[2], dwdy = dqdy[3], dpdy = dqdy[4];
        const double drdz = dqdz[0], dudz = dqdz[1], dvdz = dqdz[2], dwdz = dqdz[3], dpdz = dqdz[4];
        double div = dudx + dvdy + dwdz;
        double cv_dTdx = P.gammaM1Inverse / prim[0] * (dpdx - prim[4] / prim[0] * drdx);
        double cv_dTdy = P.gammaM1Inverse / prim[0] * (dpdy - prim[4] / prim[0] * drdy);
        double cv_dTdz = P.gammaM1Inverse / prim[0] * (dpdz - prim[4] / prim[0] * drdz);
        auto F = [&](int r, int c) -> double & { return Fv[r * 3 + c]; };
        F(1, 0) = mu * (2.0 * dudx - P.mu_bulk * div);
        F(2, 0) = mu * (dudy + dvdx);
        F(3, 0) = mu * (dudz + dwdx);
        F(4, 0) = prim[1] * F(1, 0) + prim[2] * F(2, 0) + prim[3] * F(3, 0) + lambda * cv_dTdx;
        F(1, 1) = mu * (dvdx + dudy);
        F(2, 1) = mu * (2.0 * dvdy - P.mu_bulk * div);
        F(3, 1) = mu * (dvdz + dwdy);
        F(4, 1) = prim[1] * F(1, 1) + prim[2] * F(2, 1) + prim[3] * F(3, 1) + lambda * cv_dTdy;
        F(1, 2) = mu * (dwdx + dudz);
        F(2, 2) = mu * (dwdy + dvdz);
        F(3, 2) = mu * (2.0 * dwdz - P.mu_bulk * div);
        F(4, 2) = prim[1] * F(1, 2) + prim[2] * F(2, 2) + prim[3] * F(3, 2) + lambda * cv_dTdz;
    } else {
        const double drdx = dqdx[0], dudx = dqdx[1], dvdx = dqdx[2], dpdx = dqdx[3];
        const double drdy = dqdy[0], dudy = dqdy[1], dvdy = dqdy[2], dpdy = dqdy[3];
        double div = dudx + dvdy;
        double cv_dTdx = P.gammaM1Inverse / prim[0] * (dpdx - prim[3] / prim[0] * drdx);
        double cv_dTdy = P.gammaM1Inverse / prim[0] * (dpdy - prim[3] / prim[0] * drdy);
        auto F = [&](int r, int c) -> double & { return Fv[r * 2 + c]; };
        F(1, 0) = mu * (2.0 * dudx - P.mu_bulk * div);
        F(2, 0) = mu * (dudy + dvdx);
        F(3, 0) = prim[1] * F(1, 0) + prim[2] * F(2, 0) + lambda * cv_dTdx;
        F(1, 1) = mu * (dvdx + dudy);
        F(2, 1) = mu * (2.0 * dvdy - P.mu_bulk * div);
        F(3, 1) = prim[1] * F(1, 1) + prim[2] * F(2, 1) + lambda * cv_dTdy;
    }
}

// BasicOperations.cpp:81-104 (on a copy of the state row)
void conserv2entropy(int nf, const Phys &P, const double *state_in, double *ent) {
    double state[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < nf; ++i) state[i] = state_in[i];
    const double m = 1.0 / state[0];
    double vv = 0.0;
    for (int i = 1; i < nf - 1; ++i) state[i] *= m;
    for (int i = 1; i < nf - 1; ++i) vv += state[i] * state[i];
    double v_sq = 0.5 * vv;
    double p = P.gammaM1 * (state[nf - 1] - state[0] * v_sq);
    double beta = state[0] / p;
    double s = std::log(p * std::pow(state[0], -P.gamma));
    ent[0] = (P.gamma - s) * P.gammaM1Inverse - beta * v_sq;
    ent[1] = beta * state[1];
    if (nf > 3) {
        ent[2] = beta * state[2];
        if (nf > 4) ent[3] = beta * state[3];
    }
    ent[nf - 1] = -beta;
}

// BasicOperations.cpp:126-170 for one node.  g holds the entropy-variable
// gradient on entry and the primitive gradient on exit.  Q7: `vel /= state(0)`
// aliases the state copy, so `state(1..dim)` below are velocities.
void entropygrad2primgrad(int dim, const Phys &P, int quirks, const double *state_in, double *g) {
    const int nf = dim + 2;
    double state[5], gs[5];
    for (int i = 0; i < nf; ++i) { state[i] = state_in[i]; gs[i] = g[i]; }
    const double m = 1.0 / state[0];
    double vel[3], vv = 0.0;
    for (int d = 0; d < dim; ++d) { vel[d] = state[1 + d] * m; }
    for (int d = 0; d < dim; ++d) vv += vel[d] * vel[d];
    if (quirks == 0)
        for (int d = 0; d < dim; ++d) state[1 + d] = vel[d];
    double v_sq = 0.5 * vv;
    double p = P.gammaM1 * (state[nf - 1] - state[0] * v_sq);
    double KE = v_sq * state[0];
    if (dim == 2) {
        g[1] = p / state[0] * (gs[1] + vel[0] * gs[3]);
        g[2] = p / state[0] * (gs[2] + vel[1] * gs[3]);
        g[0] = state[0] * gs[0] - gs[3] * (KE - p * P.gammaM1Inverse) +
               state[0] / p * (state[1] * g[1] + state[2] * g[2]);
        g[3] = p / state[0] * (g[0] + p * gs[3]);
    } else {
        g[1] = p / state[0] * (gs[1] + vel[0] * gs[4]);
        g[2] = p / state[0] * (gs[2] + vel[1] * gs[4]);
        g[3] = p / state[0] * (gs[3] + vel[2] * gs[4]);
        g[0] = state[0] * gs[0] - gs[4] * (KE - p * P.gammaM1Inverse) +
               state[0] / p * (state[1] * g[1] + state[2] * g[2] + state[3] * g[3]);
        g[4] = p / state[0] * (g[0] + p * gs[4]);
    }
}

// ----------------------------------------------------------- 1D GL machinery
long double legendre(int n, long double x, long double *dp) {
    long double p0 = 1.0L, p1 = x, dp0 = 0.0L, dp1 = 1.0L;
    if (n == 0) { *dp = 0.0L; return 1.0L; }
    for (int k = 1; k < n; ++k) {
        long double p2 = ((2 * k + 1) * x * p1 - k * p0) / (k + 1);
        long double dp2 = dp0 + (2 * k + 1) * p1;
        p0 = p1; p1 = p2; dp0 = dp1; dp1 = dp2;
    }
    *dp = dp1;
    return p1;
}

// Gauss-Lobatto nodes and weights on [0,1] (MFEM IntegrationRules(0,
// GaussLobatto), DGSEMIntegrator.cpp:18,22): interior nodes are the roots of
// P'_N on [-1,1], weights 2/(N(N+1) P_N(x)^2), mapped to [0,1].
void gauss_lobatto(int N, std::vector<double> &x, std::vector<double> &w) {
    const int Np = N + 1;
    x.assign(Np, 0.0);
    w.assign(Np, 0.0);
    std::vector<long double> xs(Np);
    const long double pi = 3.14159265358979323846264338327950288L;
    for (int i = 0; i < Np; ++i) {
        long double xi = -cosl(pi * i / N);
        if (i > 0 && i < N) {
            for (int it = 0; it < 100; ++it) {
                // Newton on (1-x^2) P'_N(x): derivative is -N(N+1) P_N(x)
                long double dP;
                long double P = legendre(N, xi, &dP);
                long double f = (1.0L - xi * xi) * dP;
                long double fp = -(long double)N * (N + 1) * P;
                long double dx = f / fp;
                xi -= dx;
                if (fabsl(dx) < 1e-30L) break;
            }
        }
        xs[i] = xi;
    }
    for (int i = 0; i < Np; ++i) {
        long double dP;
        long double P = legendre(N, xs[i], &dP);
        long double wi = 2.0L / ((long double)N * (N + 1) * P * P);
        x[i] = (double)((xs[i] + 1.0L) * 0.5L);
        w[i] = (double)(wi * 0.5L);
    }
    x[0] = 0.0;
    x[N] = 1.0;
}

// DGSEMIntegrator.cpp:45-82.  D[i*Np+l] = dL_l/dx at node i.
void diff_matrix(const std::vector<double> &x, std::vector<double> &D) {
    const int Np = (int)x.size();
    std::vector<double> wBary(Np, 1.0);
    for (int i = 1; i < Np; ++i)
        for (int j = 0; j < i; ++j) {
            wBary[j] *= (x[j] - x[i]);
            wBary[i] *= (x[i] - x[j]);
        }
    for (int i = 0; i < Np; ++i) wBary[i] = 1.0 / wBary[i];   // Vector::Reciprocal
    D.assign(Np * Np, 0.0);
    for (int iL = 0; iL < Np; ++iL)
        for (int i = 0; i < Np; ++i)
            if (iL != i) {
                D[i * Np + iL] = wBary[iL] / wBary[i] / (x[i] - x[iL]);
                D[i * Np + i] -= D[i * Np + iL];
            }
}

// MFEM Poly_1D::CalcLegendre: shifted Legendre P_n(2x-1), unnormalised.
void calc_legendre(int p, double x, double *u) {
    double z;
    u[0] = 1.0;
    if (p == 0) return;
    u[1] = z = 2.0 * x - 1.0;
    for (int n = 1; n < p; ++n) u[n + 1] = ((2 * n + 1) * z * u[n] - n * u[n - 1]) / (n + 1);
}

// Gauss-Jordan inverse with partial pivoting (DenseMatrix::Invert restated).
void invert(std::vector<double> &A, int n) {
    std::vector<double> I(n * n, 0.0);
    for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[r * n + c]) > std::fabs(A[piv * n + c])) piv = r;
        if (piv != c)
            for (int k = 0; k < n; ++k) {
                std::swap(A[c * n + k], A[piv * n + k]);
                std::swap(I[c * n + k], I[piv * n + k]);
            }
        double d = 1.0 / A[c * n + c];
        for (int k = 0; k < n; ++k) { A[c * n + k] *= d; I[c * n + k] *= d; }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            double f = A[r * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) {
                A[r * n + k] -= f * A[c * n + k];
                I[r * n + k] -= f * I[c * n + k];
            }
        }
    }
    A = I;
}

// ------------------------------------------------------------------ context
struct Ctx {
    int dim, N, Np, nd, nf, E, F;
    long Ndof;
    const double *adj, *detj, *fnor;
    const double *nadj, *ndetj, *fnn;   // per node / face node (multilinear elements), or null
    int nfn;                            // nodes per face
    const int *faces;
    Phys P;
    int parabolic, blending, quirks, dissipation;
    int num_bcs;
    const oracle_bc *bcs;
    int axi;                       // axisymmetric (z, r) form
    const double *xy;              // [dim][Ndof] node coordinates
    double axis_rho_floor;         // DGSEMOperator.hpp:44 rho_floor_abs
    std::vector<char> on_axis;     // [Ndof] axis nodes (DGSEMOperator::BuildAxisIndexFromMarker)
    double r(long g) const { return xy[Ndof + g]; }
    double alpha_max, alpha_min, modalThreshold;
    std::vector<double> x, w, D, Dhat, Dhat2;   // Dhat, Dhat2 as [i][l]
    std::vector<double> Vinv;                   // [nd][nd] modal basis inverse
    std::vector<int> ubdegs;                    // [nd][dim]
    int nx() const { return Np; }
    int ny() const { return dim > 1 ? Np : 1; }
    int nz() const { return dim > 2 ? Np : 1; }
    const double *A(int e) const { return adj + (long)e * dim * dim; }
    // the transformation at node n of element e (Tr.SetIntPoint + AdjugateJacobian /
    // Weight) and the scaled normal at face node a of face fc (CalcOrtho at the
    // face point); affine meshes have one value per element / face
    const double *An(int e, int n) const { return nadj ? nadj + ((long)e * nd + n) * dim * dim : A(e); }
    double Jn(int e, int n) const { return ndetj ? ndetj[(long)e * nd + n] : detj[e]; }
    const double *Nf(int fc, int a) const { return fnn ? fnn + ((long)fc * nfn + a) * dim : fnor + (long)fc * dim; }
};

void setup(Ctx &X, const oracle_mesh *m, const oracle_config *c) {
    X.dim = m->dim;
    X.N = m->order;
    X.Np = X.N + 1;
    X.nd = 1;
    for (int d = 0; d < X.dim; ++d) X.nd *= X.Np;
    X.nf = X.dim + 2;
    X.E = m->num_elements;
    X.F = m->num_faces;
    X.Ndof = (long)X.E * X.nd;
    X.adj = m->elem_adj;
    X.detj = m->elem_detj;
    X.fnor = m->face_nor;
    X.nadj = m->node_adj;
    X.ndetj = m->node_detj;
    X.fnn = m->face_node_nor;
    X.nfn = (X.dim == 2) ? X.Np : X.Np * X.Np;
    X.faces = m->face_elems;
    X.P.gamma = c->gamma;
    X.P.gammaM1 = c->gamma - 1.0;
    X.P.gammaM1Inverse = 1.0 / X.P.gammaM1;
    X.P.PrInverse = 1.0 / c->Pr;
    X.P.mu = c->mu;
    X.P.mu_bulk = 2.0 / 3.0;   // Physics.hpp:34
    X.P.R_gas = c->R_gas;
    X.P.mu0 = 1.716e-5;        // Physics.hpp:35-37
    X.P.T0 = 273.15;
    X.P.Ts = 110.4;
    X.P.T0pTs = X.P.T0 + X.P.Ts;
    X.P.sutherland = c->sutherland;
    X.parabolic = c->parabolic;
    X.blending = c->blending;
    X.quirks = c->quirks;
    X.num_bcs = c->num_bcs;
    X.bcs = c->bcs;
    X.axi = c->axisymmetric;
    X.xy = c->node_coords;
    X.axis_rho_floor = c->axis_rho_floor > 0.0 ? c->axis_rho_floor : 1e-12;
    if (X.axi) {   // DGSEMOperator.cpp:482-518: nodes at |r| <= 1e-14 of elements on "axis" boundaries
        X.on_axis.assign(X.Ndof, 0);
        for (int f = 0; f < X.F; ++f) {
            const int *fe = X.faces + 4 * f;
            if (fe[2] >= 0 || X.bcs[fe[3]].type != ORACLE_BC_AXIS) continue;
            for (int n = 0; n < X.nd; ++n) {
                const long g = (long)fe[0] * X.nd + n;
                if (std::abs(X.r(g)) <= 1e-14) X.on_axis[g] = 1;
            }
        }
    }
    X.dissipation = c->surface_dissipation;
    X.alpha_max = c->alpha_max;
    X.alpha_min = c->alpha_min;
    X.modalThreshold = 0.5 * std::pow(10.0, -1.8 * std::pow(X.N, 0.25));   // DGSEMOperator.cpp:25
    gauss_lobatto(X.N, X.x, X.w);
    diff_matrix(X.x, X.D);
    const int Np = X.Np;
    X.Dhat = X.D;   // DGSEMIntegrator.cpp:71-80 (stored untransposed, [i][l])
    X.Dhat[0] += 1.0 / X.w[0];
    X.Dhat[(Np - 1) * Np + Np - 1] -= 1.0 / X.w[Np - 1];
    X.Dhat2 = X.D;
    for (auto &v : X.Dhat2) v *= 2.0;
    X.Dhat2[0] += 1.0 / X.w[0];
    X.Dhat2[(Np - 1) * Np + Np - 1] -= 1.0 / X.w[Np - 1];
    if (X.blending) {
        // ModalBasis.cpp:42-135: ubdegs with the x-degree outermost, V(i,k) =
        // prod_j L_{deg(k,j)}(x_i,j), then inverted.
        const int nd = X.nd, dim = X.dim;
        X.ubdegs.assign(nd * dim, 0);
        int n = 0;
        if (dim == 2) {
            for (int i = 0; i < Np; ++i)
                for (int j = 0; j < Np; ++j) { X.ubdegs[n * 2] = i; X.ubdegs[n * 2 + 1] = j; ++n; }
        } else {
            for (int i = 0; i < Np; ++i)
                for (int j = 0; j < Np; ++j)
                    for (int k = 0; k < Np; ++k) {
                        X.ubdegs[n * 3] = i; X.ubdegs[n * 3 + 1] = j; X.ubdegs[n * 3 + 2] = k; ++n;
                    }
        }
        std::vector<double> V(nd * nd), L(Np);
        for (int i = 0; i < nd; ++i) {
            int ix[3] = {i % Np, (i / Np) % Np, i / (Np * Np)};
            for (int j = 0; j < dim; ++j) {
                calc_legendre(X.N, X.x[ix[j]], L.data());
                for (int k = 0; k < nd; ++k) {
                    double v = L[X.ubdegs[k * dim + j]];
                    V[i * nd + k] = (j == 0) ? v : V[i * nd + k] * v;
                }
            }
        }
        invert(V, nd);
        X.Vinv = V;
    }
}

inline int node_id(const Ctx &X, int i, int j, int k) { return k * X.ny() * X.nx() + j * X.nx() + i; }

// Outer state s2 of a boundary condition whose flux is the surface flux of
// (s1, s2) (ComputeOuterInviscidState of src/Integrators/BoundaryConditions/,
// constant data).  s1 takes the reference-mode aliasing the integrator applies
// to its inner trace.  Not for the wall types, which have their own flux.
void bdr_outer_state(const Ctx &X, const oracle_bc &bc, double *s1, const double *nor, double *s2) {
    const int dim = X.dim, nf = dim + 2;
    const double gamma = X.P.gamma, gammaM1 = X.P.gammaM1, gammaM1Inverse = X.P.gammaM1Inverse;
    switch (bc.type) {
    case ORACLE_BC_STATE:   // SpecifiedStateBdrFaceIntegrator.cpp:24-36 (constant)
        for (int f = 0; f < nf; ++f) s2[f] = bc.state[f];
        return;
    case ORACLE_BC_OUTFLOW:   // SupersonicOutflowBdrFaceIntegrator.cpp:11-14
        for (int f = 0; f < nf; ++f) s2[f] = s1[f];
        return;
    case ORACLE_BC_AXIS:
    case ORACLE_BC_SYMMETRY: {   // SymmetryBdrFaceIntegrator.cpp:11-32 (|nor| > 0)
        const double rn = 1.0 / norml2(nor, dim);
        double un[3], mn = 0.0;
        for (int d = 0; d < dim; ++d) un[d] = nor[d] * rn;
        for (int f = 0; f < nf; ++f) s2[f] = s1[f];
        for (int d = 0; d < dim; ++d) mn += s2[1 + d] * un[d];
        for (int d = 0; d < dim; ++d) s2[1 + d] += -2.0 * mn * un[d];
        return;
    }
    case ORACLE_BC_PRESSURE_OUTFLOW: {   // SubsonicOutflowPBdrFaceIntegrator.cpp:17-29
        // Q9: `Vector vel(state1.GetData() + 1, dim); vel /= state1(0);` wraps the
        // inner trace, so (reference) both traces carry velocity in the momentum slots
        double vel[3], vv = 0.0;
        const double r = 1.0 / s1[0];
        if (X.quirks == 0) {
            for (int d = 0; d < dim; ++d) s1[1 + d] *= r;
            for (int d = 0; d < dim; ++d) vel[d] = s1[1 + d];
        } else {
            for (int d = 0; d < dim; ++d) vel[d] = s1[1 + d] * r;
        }
        for (int d = 0; d < dim; ++d) vv += vel[d] * vel[d];
        for (int f = 0; f < nf; ++f) s2[f] = s1[f];
        s2[nf - 1] = bc.p * gammaM1Inverse + 0.5 * s1[0] * vv;
        return;
    }
    case ORACLE_BC_RIEMANN: {   // RiemannInvariantBdrFaceIntegrator.cpp:45-116 (constant state)
        const double gammaInverse = 1.0 / gamma;
        const double rho_o = bc.state[0], p_o = bc.state[nf - 1];
        double V_o[3], un[3], V_i[3];
        const double rn = 1.0 / norml2(nor, dim);   // Normalize: vec /= Norml2
        for (int d = 0; d < dim; ++d) { V_o[d] = bc.state[1 + d]; un[d] = nor[d] * rn; }
        const double r1 = 1.0 / s1[0];
        for (int d = 0; d < dim; ++d) V_i[d] = s1[1 + d] * r1;   // V_i /= state1(0)
        double Vn_i = 0.0, Vn_o = 0.0;
        for (int d = 0; d < dim; ++d) { Vn_i += V_i[d] * un[d]; Vn_o += V_o[d] * un[d]; }
        // Q10: V_i wraps state1, so the trace's momentum slots hold V_i; ComputePressure
        // then divides that wrapped range by rho once more (V_i = m / rho^2 afterwards).
        if (X.quirks == 0) {
            for (int d = 0; d < dim; ++d) { V_i[d] *= r1; s1[1 + d] = V_i[d]; }
        }
        double vv = 0.0;
        for (int d = 0; d < dim; ++d) vv += V_i[d] * V_i[d];
        const double p_i = gammaM1 * (s1[nf - 1] - 0.5 * s1[0] * vv);
        const double a_o = sound_speed(p_o, rho_o, gamma), a_i = sound_speed(p_i, s1[0], gamma);
        const double R_minus = (std::abs(Vn_o) >= a_o && Vn_i >= 0.0) ? Vn_i - 2.0 * a_i * gammaM1Inverse
                                                                      : Vn_o - 2.0 * a_o * gammaM1Inverse;
        const double R_plus = (std::abs(Vn_o) >= a_o && Vn_i < 0.0) ? Vn_o + 2.0 * a_o * gammaM1Inverse
                                                                    : Vn_i + 2.0 * a_i * gammaM1Inverse;
        const double Vn_b = 0.5 * (R_plus + R_minus), a_b = 0.25 * gammaM1 * (R_plus - R_minus);
        const double dVn_i = Vn_b - Vn_i, dVn_o = Vn_b - Vn_o;
        s2[0] = (Vn_i < 0.0) ? std::pow(a_b * a_b * gammaInverse * rho_o / p_o, gammaM1Inverse) * rho_o
                             : std::pow(a_b * a_b * gammaInverse * s1[0] / p_i, gammaM1Inverse) * s1[0];
        s2[nf - 1] = 0.0;
        for (int d = 0; d < dim; ++d) {
            s2[1 + d] = (Vn_i >= 0.0) ? s2[0] * (V_i[d] + dVn_i * un[d]) : s2[0] * (V_o[d] + dVn_o * un[d]);
            s2[nf - 1] += s2[1 + d] * s2[1 + d];
        }
        const double p_b = a_b * a_b * s2[0] * gammaInverse;
        s2[nf - 1] *= (0.5 / s2[0]);
        s2[nf - 1] += p_b * gammaM1Inverse;
        return;
    }
    case ORACLE_BC_INFLOW_RV: {   // SubsonicInflowRVBdrFaceIntegrator.cpp:19-49 (constant)
        const double r = bc.state[0];
        double dke = 0.0, uu = 0.0;
        s2[0] = r;
        for (int d = 0; d < dim; ++d) {
            s2[1 + d] = r * bc.state[1 + d];
            dke -= s1[1 + d] * s1[1 + d];
            uu += bc.state[1 + d] * bc.state[1 + d];
        }
        dke *= 0.5 / s1[0];
        dke += 0.5 * uu * r;
        s2[nf - 1] = s1[nf - 1] + dke;
        return;
    }
    case ORACLE_BC_INFLOW_PTTT: {   // SubsonicInflowPtTtAngBdrFaceIntegrator.cpp:15-79 (constant)
        // direction: (cos t, sin t) in 2D; in 3D the reference stores cos f one past
        // the end of its 3-vector and leaves the z component unset (Q11); cos f is used
        double vc[3] = {std::cos(bc.theta * M_PI / 180.0), std::sin(bc.theta * M_PI / 180.0), 0.0};
        if (dim > 2) {
            vc[0] *= std::sin(bc.phi * M_PI / 180.0);
            vc[1] *= std::sin(bc.phi * M_PI / 180.0);
            vc[2] = std::cos(bc.phi * M_PI / 180.0);
        }
        // ComputePressure(state1) wraps state1 (quirks 0: velocity stays in its momentum slots)
        const double r1 = 1.0 / s1[0];
        double v[3], vv = 0.0;
        for (int d = 0; d < dim; ++d) { v[d] = s1[1 + d] * r1; vv += v[d] * v[d]; }
        if (X.quirks == 0)
            for (int d = 0; d < dim; ++d) s1[1 + d] = v[d];
        const double p = gammaM1 * (s1[nf - 1] - 0.5 * s1[0] * vv);
        double V_sq = 2.0 * bc.cp * bc.Tt * (1.0 - std::pow(p / bc.pt, gammaM1 / gamma));
        V_sq = std::max(0.0, V_sq);
        s2[0] = gamma * gammaM1Inverse * p / (bc.cp * bc.Tt - 0.5 * V_sq);
        for (int d = 0; d < dim; ++d) s2[1 + d] = s2[0] * std::sqrt(V_sq) * vc[d];
        s2[nf - 1] = p * gammaM1Inverse + 0.5 * s2[0] * V_sq;
        return;
    }
    default:
        for (int f = 0; f < nf; ++f) s2[f] = s1[f];
        return;
    }
}

inline bool is_wall(int type) {
    return type == ORACLE_BC_SLIP_WALL || type == ORACLE_BC_NOSLIP_ADIABATIC || type == ORACLE_BC_NOSLIP_ISOTHERMAL;
}

// Boundary-face flux of trace s1 (BdrFaceIntegrator.cpp:61-138 with the
// integrators of src/Integrators/BoundaryConditions/).  The element receives
// -flux / (w0 J1) at the face node.  On return s1 and s2 are the inner and outer
// states the viscous boundary flux reads (NS).  Returns the largest |V|+c seen.
double bdr_face_flux(const Ctx &X, const oracle_bc &bc, double *s1, double *s2, const double *nor, double *flux) {
    const int dim = X.dim, nf = dim + 2;
    const double gamma = X.P.gamma, gammaM1 = X.P.gammaM1, gammaM1Inverse = X.P.gammaM1Inverse;
    if (is_wall(bc.type)) {
        // SlipWallBdrFaceIntegrator.cpp:16-59; the no-slip walls inherit it
        const double nn = norml2(nor, dim), rn = 1.0 / nn;
        const double gammaP1 = 1.0 + gamma, gammaP1Inverse = 1.0 / gammaP1;
        const double rho = s1[0];
        double mn = 0.0, vv = 0.0;
        for (int d = 0; d < dim; ++d) {
            mn += s1[1 + d] * (nor[d] * rn);
            const double v = s1[1 + d] / rho;
            vv += v * v;
        }
        const double u = mn / rho;   // normal velocity in the rotated frame
        const double p = gammaM1 * (s1[nf - 1] - 0.5 * rho * vv);
        const double an = sound_speed(p, rho, gamma);
        double p_star;
        if (u > 0.0)
            p_star = p + 0.25 * u * gammaP1 * rho *
                             (u + std::sqrt(u * u + 8.0 * gammaP1Inverse / rho * p * (gammaM1 * gammaP1Inverse + 1.0)));
        else
            p_star = p * std::pow(std::max(1.0 + 0.5 * gammaM1 * u / an, 0.0001), 2.0 * gamma * gammaM1Inverse);
        for (int f = 0; f < nf; ++f) flux[f] = 0.0;
        for (int d = 0; d < dim; ++d) flux[1 + d] = p_star * nor[d];
        for (int f = 0; f < nf; ++f) s2[f] = s1[f];
        return std::sqrt(vv) + an;
    }
    if ((bc.type == ORACLE_BC_SYMMETRY || bc.type == ORACLE_BC_AXIS) && norml2(nor, dim) == 0.0) {
        for (int f = 0; f < nf; ++f) { flux[f] = 0.0; s2[f] = s1[f]; }
        return 0.0;
    }
    bdr_outer_state(X, bc, s1, nor, s2);
    return face_flux(dim, gamma, X.quirks, X.dissipation, s1, s2, nor, flux);
}

// BasicOperations.cpp:106-124
void entropy2conserv(int dim, const Phys &P, const double *ent, double *state) {
    double vel[3], vv = 0.0;
    const double beta = -ent[dim + 1];
    const double rb = 1.0 / beta;   // vel /= beta
    for (int d = 0; d < dim; ++d) vel[d] = ent[1 + d] * rb;
    for (int d = 0; d < dim; ++d) vv += vel[d] * vel[d];
    const double s = P.gamma - (ent[0] + 0.5 * beta * vv) * P.gammaM1;
    state[0] = std::pow(std::exp(-s) / beta, P.gammaM1Inverse);
    for (int d = 0; d < dim; ++d) state[1 + d] = state[0] * vel[d];
    state[dim + 1] = state[0] * (1.0 / beta * P.gammaM1Inverse + 0.5 * vv);
}

// Lifting flux of a boundary face node (ComputeBdrFaceLiftingFlux): w1 is the
// inner trace's entropy variables; the gradient receives fluxN * nor / (w0 J1).
// Default (BdrFaceIntegrator.cpp:274-281): 1/2 (v(outer state of E2C(w1)) - w1)
// (reference mode: Q12).
// No-slip walls (NoSlip*WallBdrFaceIntegrator.cpp): v_wall - w1 with v_wall =
// (w1_0, V_wall * b, -b), b = -w1_last (adiabatic) or 1/(R_gas T_wall).
void bdr_lift_flux(const Ctx &X, const oracle_bc &bc, const double *w1, const double *nor, double *fluxN) {
    const int dim = X.dim, nf = dim + 2;
    if (bc.type == ORACLE_BC_NOSLIP_ADIABATIC || bc.type == ORACLE_BC_NOSLIP_ISOTHERMAL) {
        const double v = bc.type == ORACLE_BC_NOSLIP_ADIABATIC ? -w1[nf - 1] : 1.0 / (X.P.R_gas * bc.wall_T);
        fluxN[0] = w1[0];
        for (int d = 0; d < dim; ++d) fluxN[1 + d] = bc.wall_vel[d] * v;
        fluxN[nf - 1] = -v;
        for (int f = 0; f < nf; ++f) fluxN[f] -= w1[f];
        return;
    }
    double c[5] = {0, 0, 0, 0, 0}, s2[5] = {0, 0, 0, 0, 0}, w[5] = {0, 0, 0, 0, 0};
    for (int f = 0; f < nf; ++f) w[f] = w1[f];
    entropy2conserv(dim, X.P, w1, c);
    // Q12: Entropy2Conserv's `vel /= beta` wraps its const input, so (reference)
    // the trace's middle entries are velocities when `fluxN -= state1` reads them
    if (X.quirks == 0) {
        const double rb = 1.0 / -w1[nf - 1];
        for (int d = 0; d < dim; ++d) w[1 + d] = w1[1 + d] * rb;
    }
    bdr_outer_state(X, bc, c, nor, s2);
    conserv2entropy(nf, X.P, s2, fluxN);
    for (int f = 0; f < nf; ++f) fluxN[f] -= w[f];
    for (int f = 0; f < nf; ++f) fluxN[f] *= 0.5;
}

// Viscous boundary flux (ComputeBdrFaceViscousFlux) from the traces left by
// bdr_face_flux and the inner primitive gradients q[c][f]:
//   no-slip walls, supersonic outflow: Fv(inner state, q) . nor (outflow uses its
//   copy of the inner state); the adiabatic wall's energy row is V_wall . (mom rows)
//   + q_n |nor| (NoSlipAdiabWallBdrFaceIntegrator.cpp:17-31);
//   specified state, pressure outflow, Riemann invariants, inflow (rho, V):
//   Fv(outer state, 0) . nor = 0.
void bdr_viscous_flux(const Ctx &X, const oracle_bc &bc, double *s1, double *s2, const double (*q)[5],
                      const double *nor, double *fv) {
    const int dim = X.dim, nf = dim + 2;
    for (int f = 0; f < nf; ++f) fv[f] = 0.0;
    if (bc.type != ORACLE_BC_NOSLIP_ADIABATIC && bc.type != ORACLE_BC_NOSLIP_ISOTHERMAL &&
        bc.type != ORACLE_BC_OUTFLOW)
        return;
    double Fv[15];
    viscous_flux(dim, X.P, bc.type == ORACLE_BC_OUTFLOW ? s2 : s1, q[0], q[1], dim > 2 ? q[2] : nullptr, Fv);
    for (int f = 0; f < nf; ++f) {   // DenseMatrix::Mult(nor, fluxN)
        double t = 0.0;
        for (int c = 0; c < dim; ++c) t += Fv[f * dim + c] * nor[c];
        fv[f] = t;
    }
    if (bc.type == ORACLE_BC_NOSLIP_ADIABATIC) {
        double nn = 0.0;
        for (int c = 0; c < dim; ++c) nn += nor[c] * nor[c];
        const double qn = bc.heat_flux * std::sqrt(nn);
        double e = bc.wall_vel[0] * fv[1];
        for (int d = 1; d < dim; ++d) e += bc.wall_vel[d] * fv[1 + d];
        fv[nf - 1] = e + qn;
    }
}

// Element-local node on local face lf (= 2*dir + side) for face node a.
int face_node(const Ctx &X, int lf, int a) {
    const int d = lf >> 1, s = lf & 1, Np = X.Np;
    int c[3] = {0, 0, 0};
    c[d] = s * (Np - 1);
    if (X.dim == 2) {
        c[1 - d] = a;
    } else {
        int t0 = (d == 0) ? 1 : 0;
        int t1 = (d == 2) ? 1 : 2;
        c[t0] = a % Np;
        c[t1] = a / Np;
    }
    return node_id(X, c[0], c[1], X.dim > 2 ? c[2] : 0);
}

void gather(const Ctx &X, const double *u, int e, double *el) {   // el[node][f]
    for (int f = 0; f < X.nf; ++f)
        for (int n = 0; n < X.nd; ++n) el[n * X.nf + f] = u[f * X.Ndof + (long)e * X.nd + n];
}

// -------------------------------------------------------- blending (alpha)
// DGSEMOperator.cpp:60-80 + PerssonPeraireIndicator.cpp:21-58
double element_alpha(const Ctx &X, const double *el) {
    const int nd = X.nd, nf = X.nf, dim = X.dim;
    std::vector<double> rho_p(nd), modes(nd, 0.0), M1, M2;
    for (int i = 0; i < nd; ++i) {
        double state[5];
        for (int f = 0; f < nf; ++f) state[f] = el[i * nf + f];
        rho_p[i] = state[0] * compute_pressure_inplace(state, nf, X.P.gammaM1);
    }
    for (int r = 0; r < nd; ++r) {   // DenseMatrix::Mult, columns ascending
        double s = rho_p[0] * X.Vinv[r * nd + 0];
        for (int col = 1; col < nd; ++col) s += rho_p[col] * X.Vinv[r * nd + col];
        modes[r] = s;
    }
    M1 = modes;
    M2 = modes;
    for (int i = 0; i < nd; ++i)
        for (int j = 0; j < dim; ++j)
            if (X.ubdegs[i * dim + j] > X.N - 2) {
                M2[i] = 0.0;
                if (X.ubdegs[i * dim + j] > X.N - 1) M1[i] = 0.0;
            }
    double mm = 0, m1 = 0, m2 = 0;
    for (int i = 0; i < nd; ++i) { mm += modes[i] * modes[i]; m1 += M1[i] * M1[i]; m2 += M2[i] * M2[i]; }
    double eta = 1.0 - m1 / mm;
    eta = std::max(eta, 1.0 - m2 / m1);
    double a = 1.0 / (1.0 + std::exp(-kSharpness * (eta - X.modalThreshold) / X.modalThreshold));
    if (a < X.alpha_min) a = 0.0;
    else if (a > (1.0 - X.alpha_min)) a = 1.0;
    a = std::min(a, X.alpha_max);
    return a;
}

// ----------------------------------------------------------- subcell FV
// DGSEMIntegrator.cpp:1199-1304: subcell interface normal for direction dir at
// interface index i (0..Np) of the line whose nodes are base + m * stride:
// Ja_dir at the line's first node plus sum_{l<i} w_l sum_m D(l,m) Ja_dir(node m)
// (on an affine element the sums vanish and the normal is Ja_dir).
void subcell_normal(const Ctx &X, int e, int dir, int base, int stride, int i, double *nor) {
    const int dim = X.dim, Np = X.Np;
    const double *Ja0 = X.An(e, base) + dir * dim;
    double tmp[3];
    for (int c = 0; c < dim; ++c) nor[c] = Ja0[c];
    for (int l = 0; l < i; ++l) {
        for (int c = 0; c < dim; ++c) tmp[c] = 0.0;
        for (int m = 0; m < Np; ++m) {
            const double *Ja = X.An(e, base + m * stride) + dir * dim;
            for (int c = 0; c < dim; ++c) tmp[c] += Ja[c] * X.D[l * Np + m];
        }
        for (int c = 0; c < dim; ++c) tmp[c] *= X.w[l];
        for (int c = 0; c < dim; ++c) nor[c] += tmp[c];
    }
}

// DGSEMIntegrator.cpp:972-1196
void fv_fluxes(const Ctx &X, int e, const double *el, double alpha, double *el_dudt) {
    const int nf = X.nf, Np = X.Np;
    double s1[5], s2[5], nor[3], flux[5], dU[5];
    auto line = [&](int dir, int base, int stride, bool set) {
        for (int f = 0; f < nf; ++f) dU[f] = 0.0;
        int id1 = base;
        for (int f = 0; f < nf; ++f) s1[f] = el[id1 * nf + f];
        for (int i = 0; i < Np - 1; ++i) {
            int id2 = id1 + stride;
            for (int f = 0; f < nf; ++f) s2[f] = el[id2 * nf + f];
            subcell_normal(X, e, dir, base, stride, i + 1, nor);
            face_flux(X.dim, X.P.gamma, X.quirks, 1, s1, s2, nor, flux);
            if (X.axi) {   // DGSEMIntegrator.cpp:979-1031: times r at the nodes' reference midpoint
                const double rh = 0.5 * (X.r((long)e * X.nd + id1) + X.r((long)e * X.nd + id2));
                for (int f = 0; f < nf; ++f) flux[f] *= rh;
            }
            for (int f = 0; f < nf; ++f) dU[f] -= flux[f];
            const double m = 1.0 / (X.Jn(e, id1) * X.w[i]);   // Tr.Weight() at id1
            for (int f = 0; f < nf; ++f) dU[f] *= m;
            for (int f = 0; f < nf; ++f) {
                if (set) el_dudt[id1 * nf + f] = dU[f];
                else el_dudt[id1 * nf + f] += dU[f];
            }
            for (int f = 0; f < nf; ++f) { dU[f] = flux[f]; s1[f] = s2[f]; }
            id1 = id2;
        }
        const double m = 1.0 / (X.Jn(e, id1) * X.w[Np - 1]);
        for (int f = 0; f < nf; ++f) dU[f] *= m;
        for (int f = 0; f < nf; ++f) {
            if (set) el_dudt[id1 * nf + f] = dU[f];
            else el_dudt[id1 * nf + f] += dU[f];
        }
    };
    for (int k = 0; k < X.nz(); ++k)
        for (int j = 0; j < X.ny(); ++j) line(0, node_id(X, 0, j, k), 1, true);
    if (X.dim > 1) {
        for (int k = 0; k < X.nz(); ++k)
            for (int i = 0; i < X.nx(); ++i) line(1, node_id(X, i, 0, k), X.nx(), false);
        if (X.dim > 2)
            for (int j = 0; j < X.ny(); ++j)
                for (int i = 0; i < X.nx(); ++i) line(2, node_id(X, i, j, 0), X.nx() * X.ny(), false);
    }
    for (int n = 0; n < X.nd * nf; ++n) el_dudt[n] *= alpha;
}

// -------------------------------------------------------- element volume
// Euler: DGSEMIntegrator.cpp:224-433.  NS: :601-750 (3D), :752-864 (2D).
// el: [nd][nf] state, gq: [3][nd][nf] primitive gradients (NS), out [nd][nf].
void element_volume(const Ctx &X, int e, const double *el, const double *gq, double alpha,
                    double *el_dudt) {
    const int nf = X.nf, Np = X.Np, nd = X.nd, dim = X.dim;
    const bool ns = X.parabolic != 0;
    for (int n = 0; n < nd * nf; ++n) el_dudt[n] = 0.0;
    if (X.blending) fv_fluxes(X, e, el, alpha, el_dudt);
    // F/G/H_inviscid(node)(f, l): [node][f][l]
    std::vector<double> Fi(nd * nf * Np, 0.0), Gi(nd * nf * Np, 0.0), Hi(nd * nf * Np, 0.0);
    std::vector<double> Fv(nf * nd, 0.0), Gv(nf * nd, 0.0), Hv(nf * nd, 0.0);   // [f][node]
    auto setcol = [&](std::vector<double> &T, int node, int col, const double *v) {
        for (int f = 0; f < nf; ++f) T[(node * nf + f) * Np + col] = v[f];
    };
    if (ns) {
        // viscous flux per node, contravariant: flux_mat = adj * Fv^T
        const int idq1 = nd - 1;   // Q1: stale member id1 == Np^d - 1
        for (int i = 0; i < nd; ++i) {
            double state[5], fv[15];
            const double *adj = X.An(e, i);   // Tr.SetIntPoint(ip(i)), AdjugateJacobian
            const int src = (X.quirks == 0) ? idq1 : i;
            for (int f = 0; f < nf; ++f) state[f] = el[src * nf + f];
            const double *dqx = gq + (0 * nd + i) * nf;
            const double *dqy = gq + (1 * nd + i) * nf;
            const double *dqz = (dim > 2) ? gq + (2 * nd + i) * nf : nullptr;
            viscous_flux(dim, X.P, state, dqx, dqy, dqz, fv);
            for (int r = 0; r < dim; ++r)
                for (int f = 0; f < nf; ++f) {
                    double s = 0.0;
                    for (int cc = 0; cc < dim; ++cc) s += adj[r * dim + cc] * fv[f * dim + cc];
                    std::vector<double> &T = (r == 0) ? Fv : (r == 1) ? Gv : Hv;
                    T[f * nd + i] = s;
                }
        }
    }
    // metric row r at node n: adj1 / adj2 .GetRow(r) of the pair's nodes (ComputeMean in volume_flux)
    auto mrow = [&](int n, int r) { return X.An(e, n) + r * dim; };
    double f[5], g[5], h[5], s1[5], s2[5], dUi[5], dUv[5];
    for (int k = 0; k < X.nz(); ++k)
        for (int j = 0; j < X.ny(); ++j)
            for (int i = 0; i < X.nx(); ++i) {
                const int id1 = node_id(X, i, j, k);
                for (int q = 0; q < nf; ++q) s1[q] = el[id1 * nf + q];
                for (int q = 0; q < nf; ++q) f[q] = 0.0;
                setcol(Fi, id1, i, f);
                for (int m = i + 1; m < Np; ++m) {
                    const int id2 = node_id(X, m, j, k);
                    for (int q = 0; q < nf; ++q) s2[q] = el[id2 * nf + q];
                    volume_flux(dim, X.P.gamma, s1, s2, mrow(id1, 0), mrow(id2, 0), f);
                    if (X.axi) {   // DGSEMIntegrator.cpp:273-291: f *= r at the reference midpoint
                        const double rh = 0.5 * (X.r((long)e * nd + id1) + X.r((long)e * nd + id2));
                        for (int q = 0; q < nf; ++q) f[q] *= rh;
                    }
                    setcol(Fi, id1, m, f);
                    setcol(Fi, id2, i, f);
                }
                if (dim > 1) {
                    for (int q = 0; q < nf; ++q) g[q] = 0.0;
                    setcol(Gi, id1, j, g);
                    for (int m = j + 1; m < Np; ++m) {
                        const int id2 = node_id(X, i, m, k);
                        for (int q = 0; q < nf; ++q) s2[q] = el[id2 * nf + q];
                        volume_flux(dim, X.P.gamma, s1, s2, mrow(id1, 1), mrow(id2, 1), g);
                        if (X.axi) {   // :319-338
                            const double rh = 0.5 * (X.r((long)e * nd + id1) + X.r((long)e * nd + id2));
                            for (int q = 0; q < nf; ++q) g[q] *= rh;
                        }
                        setcol(Gi, id1, m, g);
                        setcol(Gi, id2, j, g);
                    }
                    if (dim > 2) {
                        for (int q = 0; q < nf; ++q) h[q] = 0.0;
                        setcol(Hi, id1, k, h);
                        for (int m = k + 1; m < Np; ++m) {
                            const int id2 = node_id(X, i, j, m);
                            for (int q = 0; q < nf; ++q) s2[q] = el[id2 * nf + q];
                            volume_flux(dim, X.P.gamma, s1, s2, mrow(id1, 2), mrow(id2, 2), h);
                            setcol(Hi, id1, m, h);
                            setcol(Hi, id2, k, (ns && X.quirks == 0) ? g : h);   // Q2
                        }
                    }
                }
                // dU_inviscid = F(id1) * Dhat2(i,:) (+ G * Dhat2(j,:) + H * Dhat2(k,:))
                auto mult = [&](const std::vector<double> &T, int row, bool add) {
                    for (int q = 0; q < nf; ++q) {
                        const double *c = &T[(id1 * nf + q) * Np];
                        double s = add ? dUi[q] : c[0] * X.Dhat2[row * Np + 0];
                        for (int l = add ? 0 : 1; l < Np; ++l) s += c[l] * X.Dhat2[row * Np + l];
                        dUi[q] = s;
                    }
                };
                auto visc = [&](const std::vector<double> &T, int row, int base, int stride) {
                    for (int l = 0; l < Np; ++l) {
                        const int n = base + l * stride;
                        for (int q = 0; q < nf; ++q) dUv[q] += T[q * nd + n] * X.Dhat[row * Np + l];
                    }
                };
                if (ns) for (int q = 0; q < nf; ++q) dUv[q] = 0.0;
                mult(Fi, i, false);
                if (ns) visc(Fv, i, node_id(X, 0, j, k), 1);
                if (dim > 1) {
                    mult(Gi, j, true);
                    if (ns) visc(Gv, j, node_id(X, i, 0, k), X.nx());
                    if (dim > 2) {
                        mult(Hi, k, true);
                        if (ns) visc(Hv, k, node_id(X, i, j, 0), X.nx() * X.ny());
                    }
                }
                for (int q = 0; q < nf; ++q) dUi[q] = -dUi[q];
                if (X.blending)
                    for (int q = 0; q < nf; ++q) dUi[q] *= (1.0 - alpha);
                const double mJ = 1.0 / X.Jn(e, id1);   // J = Tr.Weight() at id1
                if (X.axi) {   // DGSEMIntegrator.cpp:411-428: + p on the radial momentum
                    const double *st = el + id1 * nf;
                    const double ke = 0.5 * ((st[1] * st[1] + st[2] * st[2]) / st[0]);
                    el_dudt[id1 * nf + 2] += X.P.gammaM1 * (st[3] - ke);
                }
                if (ns) {
                    for (int q = 0; q < nf; ++q) el_dudt[id1 * nf + q] += (dUi[q] + dUv[q]) * mJ;
                } else {
                    for (int q = 0; q < nf; ++q) el_dudt[id1 * nf + q] += dUi[q] * mJ;
                }
            }
}

// --------------------------------------------------------------- lifting
// LiftingBR1.cpp:156-272 (element part), entropy variables in `v` [nd][nf].
void element_lift(const Ctx &X, int e, const double *v, double *gout /*[dim][nd][nf]*/) {
    const int nf = X.nf, Np = X.Np, nd = X.nd, dim = X.dim;
    for (int k = 0; k < X.nz(); ++k)
        for (int j = 0; j < X.ny(); ++j)
            for (int i = 0; i < X.nx(); ++i) {
                const int id = node_id(X, i, j, k);
                double g1[5][3];
                for (int q = 0; q < nf; ++q) for (int r = 0; r < 3; ++r) g1[q][r] = 0.0;
                for (int l = 0; l < Np; ++l) {
                    const double *a = v + node_id(X, l, j, k) * nf;
                    for (int q = 0; q < nf; ++q) g1[q][0] += a[q] * X.D[i * Np + l];
                    if (dim > 1) {
                        const double *b = v + node_id(X, i, l, k) * nf;
                        for (int q = 0; q < nf; ++q) g1[q][1] += b[q] * X.D[j * Np + l];
                    }
                    if (dim > 2) {
                        const double *c = v + node_id(X, i, j, l) * nf;
                        for (int q = 0; q < nf; ++q) g1[q][2] += c[q] * X.D[k * Np + l];
                    }
                }
                const double *adj = X.An(e, id);   // LiftingBR1.cpp:184-186: J, adj at the node
                const double mJ = 1.0 / X.Jn(e, id);
                for (int c = 0; c < dim; ++c)
                    for (int q = 0; q < nf; ++q) {
                        double s = 0.0;
                        for (int r = 0; r < dim; ++r) s += g1[q][r] * adj[r * dim + c];
                        gout[(c * nd + id) * nf + q] = s * mJ;
                    }
            }
}

// DGSEMOperator::RecoverStateFromWeighted (DGSEMOperator.cpp:161-470): U from
// the weighted state rU.  Off the axis U = rU / r.  At an axis node the
// reference's "axis" boundaries also select the low-order reconstruction
// (Simulation.cpp:520-530 sets SetLowOrderAxis(true)), so its high-order
// shape-derivative branch is never taken: U(0) = d(rU)/dr from the two nearest
// off-axis nodes at the same z (else the two nearest overall), a least-squares
// slope through the origin limited by minmod against theta_lim times each
// node's slope and clamped to cap = 10 |f1| / r1; one node: its slope; none:
// 0.  A non-finite or too small density or non-finite energy copies the
// nearest off-axis node's U instead.  Radial momentum is 0 on the axis.
int recover_weighted(const Ctx &X, const double *rU, double *U) {
    const int nd = X.nd, nf = X.nf;
    const long Ndof = X.Ndof;
    const double tiny = 1e-14, cap_mult = 10.0, z_tol = 1e-12, theta_lim = 1.5;
    const double rho_floor = X.axis_rho_floor;
    const double inf = std::numeric_limits<double>::infinity();
    auto sign = [](double a) { return (double)((a > 0) - (a < 0)); };
    auto minmod = [&](double a, double b) { return a * b <= 0.0 ? 0.0 : sign(a) * std::min(std::abs(a), std::abs(b)); };
    auto clamp = [&](double x, double m) {
        if (!std::isfinite(x)) return 0.0;
        return std::abs(x) <= m ? x : sign(x) * m;
    };
    int bad = 0;
    for (int e = 0; e < X.E; ++e) {
        const long g0 = (long)e * nd;
        for (int ld = 0; ld < nd; ++ld) {
            const long g = g0 + ld;
            const double r = X.r(g);
            if (!X.on_axis[g] && r > 0.0) {
                for (int f = 0; f < nf; ++f) U[f * Ndof + g] = rU[f * Ndof + g] / r;
                continue;
            }
            const double z_axis = X.xy[g];
            // nearest off-axis nodes at the same z, else overall (the same for every field)
            int j1 = -1, j2 = -1;
            double r1 = inf, r2 = inf;
            for (int pass = 0; pass < 2 && j1 < 0; ++pass)
                for (int j = 0; j < nd; ++j) {
                    const double rj = X.r(g0 + j);
                    if (!(rj > 0.0)) continue;
                    if (pass == 0 && !(std::abs(X.xy[g0 + j] - z_axis) <= z_tol)) continue;
                    if (rj < r1) { r2 = r1; j2 = j1; r1 = rj; j1 = j; }
                    else if (rj < r2) { r2 = rj; j2 = j; }
                }
            auto d_dr = [&](int f) {
                const double *fe = rU + f * Ndof + g0;
                const double f_ref = j1 >= 0 ? std::abs(fe[j1]) : 0.0;
                const double cap = (j1 >= 0 && !(f_ref < 1e-12)) ? cap_mult * f_ref / std::max(r1, tiny) : inf;
                if (j1 >= 0 && j2 >= 0 && std::isfinite(r1) && std::isfinite(r2) && r1 > 0.0 && r2 > 0.0) {
                    const double f1 = fe[j1], f2 = fe[j2];
                    const double m = (r1 * f1 + r2 * f2) / std::max(r1 * r1 + r2 * r2, tiny);
                    const double s1 = f1 / r1, s2 = f2 / r2;
                    return clamp(minmod(m, minmod(theta_lim * s1, theta_lim * s2)), cap);
                }
                if (j1 >= 0 && std::isfinite(r1) && r1 > 0.0) return clamp(fe[j1] / r1, cap);
                return 0.0;
            };
            const double rho_axis = d_dr(0), mz_axis = d_dr(1), E_axis = d_dr(3);
            if (!std::isfinite(rho_axis) || rho_axis < rho_floor || !std::isfinite(E_axis)) {
                int nb = -1;
                double rn = -1.0;
                for (int j = 0; j < nd; ++j) {
                    const double rj = X.r(g0 + j);
                    if (rj > 0.0 && (nb == -1 || rj < rn)) { rn = rj; nb = j; }
                }
                if (nb < 0) { ++bad; continue; }
                for (int f = 0; f < nf; ++f) U[f * Ndof + g] = rU[f * Ndof + g0 + nb] / rn;
                U[2 * Ndof + g] = 0.0;
            } else {
                U[g] = rho_axis;
                U[Ndof + g] = mz_axis;
                U[2 * Ndof + g] = 0.0;
                U[3 * Ndof + g] = E_axis;
            }
        }
    }
    return bad;
}

void run_rhs(const Ctx &X, const double *u_in, double *dudt, double *alpha_out, double *lambda_out,
             double *grad_out, int nthreads) {
    const int nf = X.nf, nd = X.nd, dim = X.dim, E = X.E;
    const long Ndof = X.Ndof;
    std::vector<double> Urec;
    const double *u = u_in;
    if (X.axi) {   // DGSEMOperator::Mult evaluates the fluxes on U recovered from rU
        Urec.assign((size_t)nf * Ndof, 0.0);
        recover_weighted(X, u_in, Urec.data());
        u = Urec.data();
    }
    std::vector<double> alpha(E, 0.0);
    if (X.blending) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
        for (int e = 0; e < E; ++e) {
            std::vector<double> el(nd * nf);
            gather(X, u, e, el.data());
            alpha[e] = element_alpha(X, el.data());
        }
    }
    if (alpha_out) std::memcpy(alpha_out, alpha.data(), sizeof(double) * E);
    if (lambda_out) {
        double lam = 0.0;
#pragma omp parallel for schedule(static) num_threads(nthreads) reduction(max : lam)
        for (long n = 0; n < Ndof; ++n) {
            double rho = u[n], vv = 0.0;
            for (int d = 0; d < dim; ++d) { double vd = u[(1 + d) * Ndof + n] / rho; vv += vd * vd; }
            double p = X.P.gammaM1 * (u[(nf - 1) * Ndof + n] - 0.5 * rho * vv);
            lam = std::max(lam, std::sqrt(vv) + sound_speed(p, rho, X.P.gamma));
        }
        *lambda_out = lam;
    }
    const double w0 = X.w[0];
    // ---- NS: entropy variables, BR1 lifting, primitive gradients
    std::vector<double> grad;   // [dim][nf][Ndof] byNODES like the reference's dudx/dudy/dudz
    if (X.parabolic) {
        std::vector<double> ent((size_t)nf * Ndof);
#pragma omp parallel for schedule(static) num_threads(nthreads)
        for (long n = 0; n < Ndof; ++n) {
            double s[5] = {0, 0, 0, 0, 0}, v[5];
            for (int f = 0; f < nf; ++f) s[f] = u[f * Ndof + n];
            conserv2entropy(nf, X.P, s, v);
            for (int f = 0; f < nf; ++f) ent[f * Ndof + n] = v[f];
        }
        grad.assign((size_t)dim * nf * Ndof, 0.0);
        // DGSEMNonlinearForm.cpp:424-491 element part
#pragma omp parallel for schedule(static) num_threads(nthreads)
        for (int e = 0; e < E; ++e) {
            std::vector<double> el(nd * nf), go(dim * nd * nf);
            gather(X, ent.data(), e, el.data());
            element_lift(X, e, el.data(), go.data());
            for (int c = 0; c < dim; ++c)
                for (int f = 0; f < nf; ++f)
                    for (int n = 0; n < nd; ++n)
                        grad[((size_t)c * nf + f) * Ndof + (long)e * nd + n] += go[(c * nd + n) * nf + f];
        }
        // faces, LiftingBR1.cpp:10-115, grouped by direction (no write conflicts)
        const int nfn = (dim == 2) ? X.Np : X.Np * X.Np;
        for (int dir = 0; dir < dim; ++dir) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
            for (int fc = 0; fc < X.F; ++fc) {
                const int *fe = X.faces + 4 * fc;
                if ((fe[1] >> 1) != dir || fe[2] < 0) continue;
                const int e1 = fe[0], lf1 = fe[1], e2 = fe[2], lf2 = fe[3];
                for (int a = 0; a < nfn; ++a) {
                    const int n1 = face_node(X, lf1, a), n2 = face_node(X, lf2, a);
                    const long g1 = (long)e1 * nd + n1, g2 = (long)e2 * nd + n2;
                    // LiftingBR1.cpp:40-49: J1, J2 at the face point, CalcOrtho there
                    const double *nor = X.Nf(fc, a);
                    const double a1 = 1.0 / (w0 * X.Jn(e1, n1)), a2 = 1.0 / (w0 * X.Jn(e2, n2));
                    double fj[5];
                    for (int f = 0; f < nf; ++f) fj[f] = 0.5 * (ent[f * Ndof + g2] - ent[f * Ndof + g1]);
                    for (int c = 0; c < dim; ++c)
                        for (int f = 0; f < nf; ++f) {
                            const double t = fj[f] * nor[c];
                            grad[((size_t)c * nf + f) * Ndof + g1] += a1 * t;
                            grad[((size_t)c * nf + f) * Ndof + g2] += a2 * t;
                        }
                }
            }
        }
        // boundary faces after the interior ones (DGSEMNonlinearForm.cpp:561-610 ->
        // LiftingBR1.cpp:311-407), element 1 only, grouped by direction
        for (int dir = 0; dir < dim; ++dir) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
            for (int fc = 0; fc < X.F; ++fc) {
                const int *fe = X.faces + 4 * fc;
                if ((fe[1] >> 1) != dir || fe[2] >= 0) continue;
                const int e1 = fe[0], lf1 = fe[1];
                for (int a = 0; a < nfn; ++a) {
                    const int n1 = face_node(X, lf1, a);
                    const long g1 = (long)e1 * nd + n1;
                    const double *nor = X.Nf(fc, a);
                    const double a1 = 1.0 / (w0 * X.Jn(e1, n1));
                    double w1[5], fj[5];
                    for (int f = 0; f < nf; ++f) w1[f] = ent[f * Ndof + g1];
                    bdr_lift_flux(X, X.bcs[fe[3]], w1, nor, fj);
                    for (int c = 0; c < dim; ++c)
                        for (int f = 0; f < nf; ++f) grad[((size_t)c * nf + f) * Ndof + g1] += a1 * (fj[f] * nor[c]);
                }
            }
        }
        // ComputeGlobalPrimitiveGradVector: DGSEMOperator.cpp:134-159
#pragma omp parallel for schedule(static) num_threads(nthreads)
        for (long n = 0; n < Ndof; ++n) {
            double s[5], g[5];
            for (int f = 0; f < nf; ++f) s[f] = u[f * Ndof + n];
            for (int c = 0; c < dim; ++c) {
                for (int f = 0; f < nf; ++f) g[f] = grad[((size_t)c * nf + f) * Ndof + n];
                entropygrad2primgrad(dim, X.P, X.quirks, s, g);
                for (int f = 0; f < nf; ++f) grad[((size_t)c * nf + f) * Ndof + n] = g[f];
            }
        }
        if (grad_out) std::memcpy(grad_out, grad.data(), sizeof(double) * grad.size());
    }
    // ---- element volume terms (DGSEMNonlinearForm.cpp:688-705 / :1351-1374)
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int e = 0; e < E; ++e) {
        std::vector<double> el(nd * nf), out(nd * nf), gq;
        gather(X, u, e, el.data());
        if (X.parabolic) {
            gq.resize(dim * nd * nf);
            for (int c = 0; c < dim; ++c)
                for (int f = 0; f < nf; ++f)
                    for (int n = 0; n < nd; ++n)
                        gq[(c * nd + n) * nf + f] = grad[((size_t)c * nf + f) * Ndof + (long)e * nd + n];
        }
        element_volume(X, e, el.data(), gq.data(), alpha[e], out.data());
        for (int f = 0; f < nf; ++f)
            for (int n = 0; n < nd; ++n) dudt[f * Ndof + (long)e * nd + n] = 0.0 + out[n * nf + f];
    }
    // ---- interior faces (DGSEMIntegrator.cpp:151-222 Euler, :435-549 NS)
    const int nfn = (dim == 2) ? X.Np : X.Np * X.Np;
    for (int dir = 0; dir < dim; ++dir) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
        for (int fc = 0; fc < X.F; ++fc) {
            const int *fe = X.faces + 4 * fc;
            if ((fe[1] >> 1) != dir) continue;
            const int e1 = fe[0], lf1 = fe[1], e2 = fe[2], lf2 = fe[3];
            if (e2 < 0) {   // boundary face (BdrFaceIntegrator::AssembleFaceVector)
                for (int a = 0; a < nfn; ++a) {
                    const int n1 = face_node(X, lf1, a);
                    const long g1 = (long)e1 * nd + n1;
                    const double *nor = X.Nf(fc, a);
                    const double a1 = 1.0 / (w0 * X.Jn(e1, n1));
                    double s1[5] = {0, 0, 0, 0, 0}, s2[5] = {0, 0, 0, 0, 0}, flux[5], d1[5];
                    for (int f = 0; f < nf; ++f) s1[f] = u[f * Ndof + g1];
                    bdr_face_flux(X, X.bcs[lf2], s1, s2, nor, flux);
                    if (X.axi)   // BdrFaceIntegrator.cpp:109-111: dU_face1 *= r
                        for (int f = 0; f < nf; ++f) flux[f] *= X.r(g1);
                    for (int f = 0; f < nf; ++f) d1[f] = -flux[f];
                    if (X.parabolic) {   // dU = -inviscid + viscous (BdrFaceIntegrator.cpp:170-186)
                        double q[3][5], fv[5];
                        for (int c = 0; c < dim; ++c)
                            for (int f = 0; f < nf; ++f) q[c][f] = grad[((size_t)c * nf + f) * Ndof + g1];
                        bdr_viscous_flux(X, X.bcs[lf2], s1, s2, q, nor, fv);
                        for (int f = 0; f < nf; ++f) d1[f] += fv[f];
                    }
                    for (int f = 0; f < nf; ++f) dudt[f * Ndof + g1] += a1 * d1[f];
                }
                continue;
            }
            for (int a = 0; a < nfn; ++a) {
                const int n1 = face_node(X, lf1, a), n2 = face_node(X, lf2, a);
                const long g1 = (long)e1 * nd + n1, g2 = (long)e2 * nd + n2;
                // DGSEMIntegrator.cpp:151-222: J1, J2 at the face point, CalcOrtho there
                const double *nor = X.Nf(fc, a);
                const double a1 = 1.0 / (w0 * X.Jn(e1, n1)), a2 = 1.0 / (w0 * X.Jn(e2, n2));
                double s1[5], s2[5], flux[5], d1[5], d2[5];
                for (int f = 0; f < nf; ++f) { s1[f] = u[f * Ndof + g1]; s2[f] = u[f * Ndof + g2]; }
                if (!X.parabolic) {
                    face_flux(dim, X.P.gamma, X.quirks, X.dissipation, s1, s2, nor, flux);
                    if (X.axi)   // DGSEMIntegrator.cpp:190-207: flux_num *= r at the face point
                        for (int f = 0; f < nf; ++f) flux[f] *= X.r(g1);
                    for (int f = 0; f < nf; ++f) { d1[f] = -flux[f]; d2[f] = flux[f]; }
                } else {
                    double q1[3][5], q2[3][5], fv1[15], fv2[15];
                    for (int c = 0; c < dim; ++c)
                        for (int f = 0; f < nf; ++f) {
                            q1[c][f] = grad[((size_t)c * nf + f) * Ndof + g1];
                            q2[c][f] = grad[((size_t)c * nf + f) * Ndof + g2];
                        }
                    double t1[5], t2[5];   // copies used only when the Q8 aliasing is fixed
                    for (int f = 0; f < nf; ++f) { t1[f] = s1[f]; t2[f] = s2[f]; }
                    double *v1 = (X.quirks == 0) ? s1 : t1;
                    double *v2 = (X.quirks == 0) ? s2 : t2;
                    viscous_flux(dim, X.P, v1, q1[0], q1[1], dim > 2 ? q1[2] : nullptr, fv1);
                    viscous_flux(dim, X.P, v2, q2[0], q2[1], dim > 2 ? q2[2] : nullptr, fv2);
                    face_flux(dim, X.P.gamma, X.quirks, X.dissipation, s1, s2, nor, flux);
                    for (int f = 0; f < nf; ++f) { d1[f] = -flux[f]; d2[f] = flux[f]; }
                    double fn[5];
                    for (int f = 0; f < nf; ++f) {
                        double s = 0.0;
                        for (int c = 0; c < dim; ++c) {
                            double fm = fv1[f * dim + c];
                            fm += fv2[f * dim + c];
                            fm *= 0.5;
                            s += fm * nor[c];
                        }
                        fn[f] = s;
                    }
                    for (int f = 0; f < nf; ++f) { d1[f] += fn[f]; d2[f] -= fn[f]; }
                }
                for (int f = 0; f < nf; ++f) {
                    dudt[f * Ndof + g1] += a1 * d1[f];
                    dudt[f * Ndof + g2] += a2 * d2[f];
                }
            }
        }
    }
    if (X.axi)   // DGSEMOperator::ZeroAxisRadialMom (DGSEMOperator.cpp:520-533)
        for (long g = 0; g < Ndof; ++g)
            if (X.on_axis[g]) dudt[2 * Ndof + g] = 0.0;
}

// Boundary faces need a valid BC index; the Navier-Stokes form has no viscous
// treatment for the slip wall, symmetry and pt/Tt inflow types, and in reference
// mode no defined Riemann-invariant lifting (RiemannInvariantBdrFaceIntegrator
// normalises the integrator's `nor`, which AssembleLiftingBdrFaceVector never sets).
bool bad_boundaries(const oracle_mesh *m, const oracle_config *c) {
    for (int f = 0; f < m->num_faces; ++f) {
        const int *fe = m->face_elems + 4 * f;
        if (fe[2] >= 0) continue;
        if (!c->bcs || fe[3] < 0 || fe[3] >= c->num_bcs) return true;
        const int t = c->bcs[fe[3]].type;
        if (c->parabolic && (t == ORACLE_BC_SLIP_WALL || t == ORACLE_BC_SYMMETRY || t == ORACLE_BC_INFLOW_PTTT))
            return true;
        // Q13: the reference's Riemann lifting reads a face normal only its face pass sets
        if (c->parabolic && c->quirks == 0 && t == ORACLE_BC_RIEMANN) return true;
        if (t == ORACLE_BC_AXIS && !c->axisymmetric) return true;
    }
    return false;
}
}   // namespace

extern "C" {

int oracle_rhs(const oracle_mesh *m, const oracle_config *c, const double *u, double *dudt,
               double *alpha, double *lambda_max, double *grad, int nthreads) {
    if (!m || !c || !u || !dudt) return 1;
    if (m->dim < 2 || m->dim > 3 || m->order < 1 || m->order > 9) return 1;
    if (nthreads <= 0) nthreads = 1;
    if (bad_boundaries(m, c)) return 1;
    if (c->axisymmetric && (m->dim != 2 || c->parabolic || !c->node_coords)) return 1;
    Ctx X;
    setup(X, m, c);
    run_rhs(X, u, dudt, alpha, lambda_max, grad, nthreads);
    return 0;
}

int oracle_recover_weighted(const oracle_mesh *m, const oracle_config *c, const double *rU, double *U) {
    if (!m || !c || !rU || !U || !c->axisymmetric || !c->node_coords || m->dim != 2) return 1;
    if (bad_boundaries(m, c)) return 1;
    Ctx X;
    setup(X, m, c);
    return recover_weighted(X, rU, U) == 0 ? 0 : 1;
}

int oracle_step(const oracle_mesh *m, const oracle_config *c, double *u, double t, double dt,
                int scheme, int nsteps, int nthreads) {
    if (!m || !c || !u) return 1;
    if (nthreads <= 0) nthreads = 1;
    if (bad_boundaries(m, c)) return 1;
    if (c->axisymmetric && (m->dim != 2 || c->parabolic || !c->node_coords)) return 1;
    Ctx X;
    setup(X, m, c);
    const long n = (long)X.nf * X.Ndof;
    std::vector<double> k(n), y(n);
    (void)t;
    for (int s = 0; s < nsteps; ++s) {
        if (scheme == 0) {
            // MFEM RK3SSPSolver::Step (Shu-Osher):
            //   y = x + dt*f(x); y += dt*f(y); y = 3/4 x + 1/4 y;
            //   y += dt*f(y); x = 1/3 x + 2/3 y
            run_rhs(X, u, k.data(), nullptr, nullptr, nullptr, nthreads);
            for (long i = 0; i < n; ++i) y[i] = u[i] + dt * k[i];
            run_rhs(X, y.data(), k.data(), nullptr, nullptr, nullptr, nthreads);
            for (long i = 0; i < n; ++i) y[i] += dt * k[i];
            for (long i = 0; i < n; ++i) y[i] = 3. / 4 * u[i] + 1. / 4 * y[i];
            run_rhs(X, y.data(), k.data(), nullptr, nullptr, nullptr, nthreads);
            for (long i = 0; i < n; ++i) y[i] += dt * k[i];
            for (long i = 0; i < n; ++i) u[i] = 1. / 3 * u[i] + 2. / 3 * y[i];
        } else if (scheme == 1) {
            // Carpenter & Kennedy (1994) five-stage fourth-order 2N-storage RK:
            //   du = A_i du + dt L(u);  u = u + B_i du
            static const double A[5] = {0.0, -567301805773.0 / 1357537059087.0,
                                        -2404267990393.0 / 2016746695238.0,
                                        -3550918686646.0 / 2091501179385.0,
                                        -1275806237668.0 / 842570457699.0};
            static const double B[5] = {1432997174477.0 / 9575080441755.0,
                                        5161836677717.0 / 13612068292357.0,
                                        1720146321549.0 / 2090206949498.0,
                                        3134564353537.0 / 4481467310338.0,
                                        2277821191437.0 / 14882151754819.0};
            std::fill(y.begin(), y.end(), 0.0);   // y holds du
            for (int st = 0; st < 5; ++st) {
                run_rhs(X, u, k.data(), nullptr, nullptr, nullptr, nthreads);
                for (long i = 0; i < n; ++i) y[i] = A[st] * y[i] + dt * k[i];
                for (long i = 0; i < n; ++i) u[i] = u[i] + B[st] * y[i];
            }
        } else {
            return 1;
        }
    }
    return 0;
}

int oracle_gl(int order, double *nodes, double *weights, double *D) {
    std::vector<double> x, w, Dm;
    gauss_lobatto(order, x, w);
    diff_matrix(x, Dm);
    for (int i = 0; i <= order; ++i) { nodes[i] = x[i]; weights[i] = w[i]; }
    if (D) std::memcpy(D, Dm.data(), sizeof(double) * Dm.size());
    return 0;
}

double oracle_log_mean(double x, double y) { return log_mean(x, y); }

double oracle_volume_flux(int dim, double gamma, const double *s1, const double *s2,
                          const double *m1, const double *m2, double *F) {
    return volume_flux(dim, gamma, s1, s2, m1, m2, F);
}

double oracle_face_flux(int dim, double gamma, int quirks, int dissipation, const double *s1,
                        const double *s2, const double *nor, double *F) {
    return face_flux(dim, gamma, quirks, dissipation, s1, s2, nor, F);
}

}   // extern "C"
