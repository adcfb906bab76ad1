// host_common.hpp -- host-side helpers shared by the operator handle, the
// no-allocation entry point and batches: the 1D operator tables, the physics
// constants and the validation of a mesh descriptor into the neighbour table.
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/prandtl_b200.h"
#include "dgsem_kernels.cuh"

namespace prandtl {
namespace host {

// ---- 1D tables (mirrors DGSEMIntegrator.cpp:41-82 and ModalBasis.cpp:110-135)
inline long double legendre_ld(int n, long double x, long double *dp) {
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

// Fixed-size arrays only (Np <= 8): the allocation-free entry point builds
// its tables with this function too.
inline void build_tables(int N, OpTables &T) {
    const int Np = N + 1;
    std::memset(&T, 0, sizeof(T));
    // Gauss-Lobatto nodes/weights on [0,1]
    const long double pi = 3.14159265358979323846264338327950288L;
    long double xs[8];
    for (int i = 0; i < Np; ++i) {
        long double xi = -cosl(pi * i / N);
        if (i > 0 && i < N)
            for (int it = 0; it < 100; ++it) {
                long double dP, P = legendre_ld(N, xi, &dP);
                long double dx = ((1.0L - xi * xi) * dP) / (-(long double)N * (N + 1) * P);
                xi -= dx;
                if (fabsl(dx) < 1e-30L) break;
            }
        xs[i] = xi;
    }
    for (int i = 0; i < Np; ++i) {
        long double dP, P = legendre_ld(N, xs[i], &dP);
        T.x[i] = (double)((xs[i] + 1.0L) * 0.5L);
        T.w[i] = (double)(2.0L / ((long double)N * (N + 1) * P * P) * 0.5L);
    }
    T.x[0] = 0.0;
    T.x[N] = 1.0;
    // barycentric differentiation matrix
    double wb[8];
    for (int i = 0; i < Np; ++i) wb[i] = 1.0;
    for (int i = 1; i < Np; ++i)
        for (int j = 0; j < i; ++j) {
            wb[j] *= (T.x[j] - T.x[i]);
            wb[i] *= (T.x[i] - T.x[j]);
        }
    for (int i = 0; i < Np; ++i) wb[i] = 1.0 / wb[i];
    for (int iL = 0; iL < Np; ++iL)
        for (int i = 0; i < Np; ++i)
            if (iL != i) {
                T.D[i * Np + iL] = wb[iL] / wb[i] / (T.x[i] - T.x[iL]);
                T.D[i * Np + i] -= T.D[i * Np + iL];
            }
    for (int q = 0; q < Np * Np; ++q) {
        T.Dhat[q] = T.D[q];
        T.Dhat2[q] = 2.0 * T.D[q];
    }
    T.Dhat[0] += 1.0 / T.w[0];
    T.Dhat[(Np - 1) * Np + Np - 1] -= 1.0 / T.w[Np - 1];
    T.Dhat2[0] += 1.0 / T.w[0];
    T.Dhat2[(Np - 1) * Np + Np - 1] -= 1.0 / T.w[Np - 1];
    // 1D Vandermonde of shifted Legendre P_a(2x-1): V[l][a], inverted (Gauss-Jordan)
    double V[64], I[64];
    for (int q = 0; q < Np * Np; ++q) I[q] = 0.0;
    for (int l = 0; l < Np; ++l) {
        double u[8], z = 2.0 * T.x[l] - 1.0;
        u[0] = 1.0;
        if (N >= 1) u[1] = z;
        for (int n = 1; n < N; ++n) u[n + 1] = ((2 * n + 1) * z * u[n] - n * u[n - 1]) / (n + 1);
        for (int a = 0; a < Np; ++a) V[l * Np + a] = u[a];
    }
    for (int i = 0; i < Np; ++i) I[i * Np + i] = 1.0;
    for (int c = 0; c < Np; ++c) {
        int piv = c;
        for (int r = c + 1; r < Np; ++r)
            if (std::fabs(V[r * Np + c]) > std::fabs(V[piv * Np + c])) piv = r;
        for (int k = 0; k < Np; ++k) {
            std::swap(V[c * Np + k], V[piv * Np + k]);
            std::swap(I[c * Np + k], I[piv * Np + k]);
        }
        const double d = 1.0 / V[c * Np + c];
        for (int k = 0; k < Np; ++k) { V[c * Np + k] *= d; I[c * Np + k] *= d; }
        for (int r = 0; r < Np; ++r) {
            if (r == c) continue;
            const double f = V[r * Np + c];
            for (int k = 0; k < Np; ++k) { V[r * Np + k] -= f * V[c * Np + k]; I[r * Np + k] -= f * I[c * Np + k]; }
        }
    }
    // I = V^{-1}: I[a][l] maps nodal values (l) to mode a
    for (int q = 0; q < Np * Np; ++q) T.Vinv[q] = I[q];
}

// Text of the calling thread's last failure outside a handle (prandtl_create,
// prandtl_rhs_noalloc), kept in a fixed thread-local buffer (no allocation);
// prandtl_last_error(NULL) returns it.  Defined in prandtl_api.cu.
void set_unbound_error(const char *msg);
const char *unbound_error();

// Room in a batch for one more solve of `bytes` (defined in prandtl_batch.cu).
bool batch_has_room(prandtl_batch *b, size_t bytes);

// Text for the state-check bits the RK epilogue sets (PRANDTL_HEALTH_*).
// Pause between polls of a device event (the host waits are all polls bounded
// by a timeout): yield for the first 200 us, so short waits end within a few
// microseconds of the event, then sleep 50 us at a time.
inline void poll_pause(double waited_s) {
    if (waited_s < 2e-4) std::this_thread::yield();
    else std::this_thread::sleep_for(std::chrono::microseconds(50));
}

inline std::string health_text(unsigned bits) {
    std::string t = "the state left the admissible set:";
    if (bits & PRANDTL_HEALTH_NONFINITE) t += " non-finite values;";
    if (bits & PRANDTL_HEALTH_DENSITY) t += " density <= 0;";
    if (bits & PRANDTL_HEALTH_PRESSURE) t += " pressure <= 0;";
    return t;
}

inline void build_phys(const prandtl_config &c, int N, PhysParams &P) {
    P.gamma = c.gamma;
    P.gammaM1 = c.gamma - 1.0;
    P.gammaM1Inverse = 1.0 / P.gammaM1;
    P.PrInverse = 1.0 / c.Pr;
    P.mu = c.mu;
    P.mu_bulk = 2.0 / 3.0;     // Physics.hpp:34
    P.R_gas = c.R_gas;
    P.mu0 = 1.716e-5;          // Physics.hpp:35-37
    P.T0 = 273.15;
    P.Ts = 110.4;
    P.T0pTs = P.T0 + P.Ts;
    P.alpha_max = c.alpha_max;
    P.alpha_min = c.alpha_min;
    P.modal_threshold = 0.5 * std::pow(10.0, -1.8 * std::pow((double)N, 0.25));   // DGSEMOperator.cpp:25
    P.sutherland = c.sutherland;
    P.quirks = c.quirks;
    P.dissipation = c.surface_dissipation;
    P.blending = c.blending;
}


// Checks a mesh descriptor and builds the neighbour table nbr[e][lf] =
// {neighbour element, its local face, face id, role (0: e is Elem1)}.  Every
// element face must be listed exactly once: as an interior face with the
// traces aligned (local faces 2*dir and 2*dir+1 of the same direction), or as
// a boundary face {elem1, lface1, -1, bc} with 0 <= bc < num_bcs, recorded as
// {-1, bc, face id, 0}.
inline prandtl_status validate_mesh(const prandtl_mesh_desc *md, std::vector<int4> &nbr, std::string &msg,
                                    int num_bcs = 0) {
    if (md->dim != 2 && md->dim != 3) { msg = "dim must be 2 or 3"; return PRANDTL_EUNSUPPORTED; }
    if (!order_supported(md->dim, md->order)) { msg = "order must be in 1..5"; return PRANDTL_EUNSUPPORTED; }
    if (md->num_elements <= 0 || md->num_faces < 0) { msg = "bad sizes"; return PRANDTL_EINVAL; }
    if (!md->elem_adj || !md->elem_detj || (md->num_faces > 0 && (!md->face_elems || !md->face_nor))) {
        msg = "mesh arrays missing";
        return PRANDTL_EINVAL;
    }
    const int NFACE = 2 * md->dim, E = md->num_elements, F = md->num_faces;
    constexpr int UNSET = -2;
    nbr.assign((size_t)E * NFACE, make_int4(UNSET, -1, -1, -1));
    for (int f = 0; f < F; ++f) {
        const int *fe = md->face_elems + 4 * f;
        const int e1 = fe[0], l1 = fe[1], e2 = fe[2], l2 = fe[3];
        if (e1 < 0 || e1 >= E || l1 < 0 || l1 >= NFACE) {
            msg = "face " + std::to_string(f) + " out of range";
            return PRANDTL_EINVAL;
        }
        int4 &a = nbr[(size_t)e1 * NFACE + l1];
        if (a.x != UNSET) {
            msg = "element face listed twice (face " + std::to_string(f) + ")";
            return PRANDTL_EINVAL;
        }
        if (e2 < 0) {   // boundary face
            if (e2 != -1 || l2 < 0 || l2 >= num_bcs) {
                msg = "boundary face " + std::to_string(f) + ": no boundary condition " + std::to_string(l2) +
                      " (" + std::to_string(num_bcs) + " given)";
                return PRANDTL_EINVAL;
            }
            a = make_int4(-1, l2, f, 0);
            continue;
        }
        if (e2 >= E || l2 < 0 || l2 >= NFACE) {
            msg = "face " + std::to_string(f) + " out of range";
            return PRANDTL_EINVAL;
        }
        if ((l1 >> 1) != (l2 >> 1) || (l1 ^ l2) != 1) {
            msg = "face " + std::to_string(f) + ": only aligned opposite faces are supported";
            return PRANDTL_EUNSUPPORTED;
        }
        int4 &b = nbr[(size_t)e2 * NFACE + l2];
        if (b.x != UNSET) {
            msg = "element face listed twice (face " + std::to_string(f) + ")";
            return PRANDTL_EINVAL;
        }
        a = make_int4(e2, l2, f, 0);
        b = make_int4(e1, l1, f, 1);
    }
    for (size_t q = 0; q < nbr.size(); ++q)
        if (nbr[q].x == UNSET) {
            msg = "element " + std::to_string(q / NFACE) + " has a face that is neither interior nor a boundary face";
            return PRANDTL_EUNSUPPORTED;
        }
    for (int e = 0; e < E; ++e)
        if (!(md->elem_detj[e] > 0.0)) { msg = "non-positive det J"; return PRANDTL_EINVAL; }
    return PRANDTL_OK;
}


// Device copy of the boundary conditions (BcDev has prandtl_bc's layout).
// Flow direction of SubsonicInflowPtTtAng (SubsonicInflowPtTtAngBdrFaceIntegrator.cpp
// constructors): (cos t, sin t) in 2D, (cos t sin f, sin t sin f, cos f) in 3D,
// angles in degrees.  The reference's 3D constructor stores cos f one slot past
// its dim-sized vector and leaves the z component unset; the intended value is
// used in both modes.
inline void inflow_direction(int dim, double theta, double phi, double vc[3]) {
    vc[0] = vc[1] = vc[2] = 0.0;
    vc[0] = std::cos(theta * M_PI / 180.0);
    vc[1] = std::sin(theta * M_PI / 180.0);
    if (dim > 2) {
        vc[0] *= std::sin(phi * M_PI / 180.0);
        vc[1] *= std::sin(phi * M_PI / 180.0);
        vc[2] = std::cos(phi * M_PI / 180.0);
    }
}

inline std::vector<BcDev> device_bcs(const prandtl_config *cfg, int dim) {
    std::vector<BcDev> out((size_t)(cfg->num_bcs > 0 && cfg->bcs ? cfg->num_bcs : 0));
    for (size_t k = 0; k < out.size(); ++k) {
        const prandtl_bc &b = cfg->bcs[k];
        BcDev &o = out[k];
        o.type = b.type;
        o.pad = 0;
        for (int f = 0; f < 5; ++f) o.state[f] = b.state[f];
        o.p = b.p;
        o.pt = b.pt;
        o.Tt = b.Tt;
        o.cp = b.cp;
        inflow_direction(dim, b.theta, b.phi, o.vc);
        for (int d = 0; d < 3; ++d) o.wall_vel[d] = b.wall_vel[d];
        o.heat_flux = b.heat_flux;
        o.vT = b.type == PRANDTL_BC_NOSLIP_ISOTHERMAL ? 1.0 / (cfg->R_gas * b.wall_T) : 0.0;
    }
    return out;
}

inline prandtl_status check_bcs(const prandtl_config *cfg, int dim, std::string &msg) {
    if (cfg->num_bcs < 0 || (cfg->num_bcs > 0 && !cfg->bcs)) { msg = "bad boundary-condition table"; return PRANDTL_EINVAL; }
    for (int k = 0; k < cfg->num_bcs; ++k) {
        const prandtl_bc &b = cfg->bcs[k];
        const std::string tag = "boundary condition " + std::to_string(k);
        if (b.type < PRANDTL_BC_STATE || b.type > PRANDTL_BC_AXIS) {
            msg = tag + ": unknown type";
            return PRANDTL_EINVAL;
        }
        if (b.type == PRANDTL_BC_AXIS && !cfg->axisymmetric) {
            msg = tag + ": the axis condition needs the axisymmetric form";
            return PRANDTL_EUNSUPPORTED;
        }
        if ((b.type == PRANDTL_BC_STATE || b.type == PRANDTL_BC_RIEMANN || b.type == PRANDTL_BC_INFLOW_RV) &&
            !(b.state[0] > 0.0)) {
            msg = tag + ": outer density must be positive";
            return PRANDTL_EINVAL;
        }
        if (b.type == PRANDTL_BC_RIEMANN && !(b.state[dim == 3 ? 4 : 3] > 0.0)) {
            msg = tag + ": outer pressure must be positive";
            return PRANDTL_EINVAL;
        }
        if (b.type == PRANDTL_BC_INFLOW_PTTT && !(b.pt > 0.0 && b.Tt > 0.0 && b.cp > 0.0)) {
            msg = tag + ": pt, Tt and cp must be positive";
            return PRANDTL_EINVAL;
        }
        if (b.type == PRANDTL_BC_NOSLIP_ISOTHERMAL && !(b.wall_T > 0.0 && cfg->R_gas > 0.0)) {
            msg = tag + ": wall temperature and R_gas must be positive";
            return PRANDTL_EINVAL;
        }
    }
    return PRANDTL_OK;
}

// The Navier-Stokes form has no treatment for the slip wall, symmetry and
// pt/Tt inflow (the reference defines none for the first two), and reference
// mode has no defined Riemann-invariant lifting: RiemannInvariantBdrFaceIntegrator
// normalises the integrator's face normal, which only its face pass sets.
// Checks the conditions boundary faces use (after validate_mesh).
inline prandtl_status check_viscous_bcs(const prandtl_mesh_desc *md, const prandtl_config *cfg, std::string &msg) {
    if (!cfg->parabolic) return PRANDTL_OK;
    for (int f = 0; f < md->num_faces; ++f) {
        const int *fe = md->face_elems + 4 * f;
        if (fe[2] >= 0) continue;
        const int t = cfg->bcs[fe[3]].type;
        const std::string tag = "boundary condition " + std::to_string(fe[3]);
        if (t == PRANDTL_BC_SLIP_WALL || t == PRANDTL_BC_SYMMETRY || t == PRANDTL_BC_INFLOW_PTTT) {
            msg = tag + ": slip wall, symmetry and pt/Tt inflow have no viscous treatment (parabolic = 1)";
            return PRANDTL_EUNSUPPORTED;
        }
        if (cfg->quirks == 0 && t == PRANDTL_BC_RIEMANN) {
            msg = tag + ": the reference's Riemann-invariant lifting is undefined (use quirks = 1)";
            return PRANDTL_EUNSUPPORTED;
        }
    }
    return PRANDTL_OK;
}

// For the Navier-Stokes form with contravariant viscous fluxes: every face's
// scaled normal must be the outward adjugate row of both its elements
// (Nanson's formula for affine elements): nor = s1 adj(J_e1)[d1] =
// -s2 adj(J_e2)[d2] with s = +1 on a local face 2d+1, -1 on 2d.
inline prandtl_status check_face_normals(const prandtl_mesh_desc *md, std::string &msg) {
    const int dim = md->dim;
    for (int f = 0; f < md->num_faces; ++f) {
        const int *fe = md->face_elems + 4 * f;
        const double *nor = md->face_nor + (size_t)f * dim;
        for (int side = 0; side < 2; ++side) {
            const int e = fe[2 * side], lf = fe[2 * side + 1], d = lf >> 1;
            if (e < 0) continue;   // boundary face: no element 2
            const double sg = ((lf & 1) ? 1.0 : -1.0) * (side == 0 ? 1.0 : -1.0);
            const double *row = md->elem_adj + ((size_t)e * dim + d) * dim;
            double err = 0, mag = 0;
            for (int c = 0; c < dim; ++c) {
                err = std::fmax(err, std::fabs(nor[c] - sg * row[c]));
                mag = std::fmax(mag, std::fabs(row[c]));
            }
            if (!(err <= 1e-9 * mag)) {
                msg = "face " + std::to_string(f) +
                      ": scaled normal differs from the element's adjugate row (non-affine or inconsistent mesh)";
                return PRANDTL_EUNSUPPORTED;
            }
        }
    }
    return PRANDTL_OK;
}

// ---- non-affine (multilinear) elements: per-node geometry
inline bool mesh_curved(const prandtl_mesh_desc *md) { return md->node_adj != nullptr; }

// All three per-node arrays or none; det J > 0 and every value finite.
inline prandtl_status check_curved(const prandtl_mesh_desc *md, std::string &msg) {
    const int n = (md->node_adj != nullptr) + (md->node_detj != nullptr) + (md->face_node_nor != nullptr);
    if (n == 0) return PRANDTL_OK;
    if (n != 3) {
        msg = "node_adj, node_detj and face_node_nor: all three or none";
        return PRANDTL_EINVAL;
    }
    const int dim = md->dim, Np = md->order + 1;
    int nd = 1;
    for (int d = 0; d < dim; ++d) nd *= Np;
    const int nfn = nd / Np;
    const size_t N = (size_t)md->num_elements * nd;
    for (size_t i = 0; i < N; ++i)
        if (!(md->node_detj[i] > 0.0) || !std::isfinite(md->node_detj[i])) {
            msg = "node_detj[" + std::to_string(i) + "] is not a positive finite value (inverted element)";
            return PRANDTL_EINVAL;
        }
    for (size_t i = 0; i < N * dim * dim; ++i)
        if (!std::isfinite(md->node_adj[i])) {
            msg = "node_adj holds a non-finite value";
            return PRANDTL_EINVAL;
        }
    for (size_t i = 0; i < (size_t)md->num_faces * nfn * dim; ++i)
        if (!std::isfinite(md->face_node_nor[i])) {
            msg = "face_node_nor holds a non-finite value";
            return PRANDTL_EINVAL;
        }
    return PRANDTL_OK;
}

// Element-local node of face node a on local face lf = 2 dir + side (face nodes
// lexicographic over the remaining directions, the lower one fastest).
inline int host_face_node(int dim, int Np, int lf, int a) {
    const int d = lf >> 1, s = lf & 1;
    int c[3] = {0, 0, 0};
    c[d] = s * (Np - 1);
    if (dim == 2) {
        c[1 - d] = a;
    } else {
        const int t0 = (d == 0) ? 1 : 0, t1 = (d == 2) ? 1 : 2;
        c[t0] = a % Np;
        c[t1] = a / Np;
    }
    return c[0] + Np * (c[1] + Np * c[2]);
}

// Per-node geometry, structure of arrays [dim*dim + 1][Ndof]: adj(J) entries
// (row-major index r*dim + q), then det J.
inline std::vector<double> node_geometry_soa(const prandtl_mesh_desc *md) {
    const int dim = md->dim, Np = md->order + 1, G = dim * dim + 1;
    int nd = 1;
    for (int d = 0; d < dim; ++d) nd *= Np;
    const size_t Ndof = (size_t)md->num_elements * nd;
    std::vector<double> g(G * Ndof);
    for (size_t n = 0; n < Ndof; ++n) {
        for (int c = 0; c < dim * dim; ++c) g[c * Ndof + n] = md->node_adj[n * dim * dim + c];
        g[(size_t)(dim * dim) * Ndof + n] = md->node_detj[n];
    }
    return g;
}

// Subcell interface normals (DGSEMIntegrator.cpp:1199-1304): for direction dir
// and line ln (the kernels' line_base numbering), interface i = 1..Np-1 has
// Ja_dir(first node) + sum_{l<i} w_l sum_m D(l,m) Ja_dir(node m), Ja_dir = row
// dir of adj(J).  Layout [E][dim][Np^(dim-1)][Np-1][dim].
inline std::vector<double> subcell_normals(const prandtl_mesh_desc *md, const OpTables &T) {
    const int dim = md->dim, Np = md->order + 1;
    int nd = 1;
    for (int d = 0; d < dim; ++d) nd *= Np;
    const int nline = nd / Np;
    std::vector<double> out((size_t)md->num_elements * dim * nline * (Np - 1) * dim);
    size_t o = 0;
    for (int e = 0; e < md->num_elements; ++e)
        for (int dir = 0; dir < dim; ++dir)
            for (int ln = 0; ln < nline; ++ln) {
                int base, stride;
                if (dir == 0) { base = ln * Np; stride = 1; }
                else if (dim == 2) { base = ln; stride = Np; }
                else if (dir == 1) { base = (ln / Np) * Np * Np + ln % Np; stride = Np; }
                else { base = ln; stride = Np * Np; }
                auto Ja = [&](int m, int c) {
                    return md->node_adj[(((size_t)e * nd + base + m * stride) * dim + dir) * dim + c];
                };
                for (int i = 1; i < Np; ++i) {
                    double nor[3], tmp[3];
                    for (int c = 0; c < dim; ++c) nor[c] = Ja(0, c);
                    for (int l = 0; l < i; ++l) {
                        for (int c = 0; c < dim; ++c) tmp[c] = 0.0;
                        for (int m = 0; m < Np; ++m)
                            for (int c = 0; c < dim; ++c) tmp[c] += Ja(m, c) * T.D[l * Np + m];
                        for (int c = 0; c < dim; ++c) nor[c] += tmp[c] * T.w[l];
                    }
                    for (int c = 0; c < dim; ++c) out[o++] = nor[c];
                }
            }
    return out;
}

// The contravariant viscous form takes Fv . n at a face node from the node's
// row of adj(J) Fv^T, which needs the face normal to be that row (Nanson's
// formula) on both sides: per face node on non-affine meshes.
inline prandtl_status check_face_node_normals(const prandtl_mesh_desc *md, std::string &msg) {
    const int dim = md->dim, Np = md->order + 1;
    int nd = 1;
    for (int d = 0; d < dim; ++d) nd *= Np;
    const int nfn = nd / Np;
    for (int f = 0; f < md->num_faces; ++f) {
        const int *fe = md->face_elems + 4 * f;
        for (int a = 0; a < nfn; ++a) {
            const double *nor = md->face_node_nor + ((size_t)f * nfn + a) * dim;
            for (int side = 0; side < 2; ++side) {
                const int e = fe[2 * side], lf = fe[2 * side + 1], d = lf >> 1;
                if (e < 0) continue;
                const double sg = ((lf & 1) ? 1.0 : -1.0) * (side == 0 ? 1.0 : -1.0);
                const int n = host_face_node(dim, Np, lf, a);
                const double *row = md->node_adj + (((size_t)e * nd + n) * dim + d) * dim;
                double err = 0, mag = 0;
                for (int c = 0; c < dim; ++c) {
                    err = std::fmax(err, std::fabs(nor[c] - sg * row[c]));
                    mag = std::fmax(mag, std::fabs(row[c]));
                }
                if (!(err <= 1e-9 * mag)) {
                    msg = "face " + std::to_string(f) + " node " + std::to_string(a) +
                          ": scaled normal differs from the element's adjugate row there";
                    return PRANDTL_EUNSUPPORTED;
                }
            }
        }
    }
    return PRANDTL_OK;
}

// Geometry rows [E][dim*dim + 1]: adj(J) row-major, then det J.
// (into an existing vector, whose capacity is reused across admissions)
inline void geometry_rows_into(const prandtl_mesh_desc *md, std::vector<double> &geo) {
    const int dim = md->dim, GEO = dim * dim + 1, E = md->num_elements;
    geo.resize((size_t)E * GEO);
    for (int e = 0; e < E; ++e) {
        for (int q = 0; q < dim * dim; ++q) geo[(size_t)e * GEO + q] = md->elem_adj[(size_t)e * dim * dim + q];
        geo[(size_t)e * GEO + dim * dim] = md->elem_detj[e];
    }
}
inline std::vector<double> geometry_rows(const prandtl_mesh_desc *md) {
    std::vector<double> geo;
    geometry_rows_into(md, geo);
    return geo;
}

}   // namespace host
}   // namespace prandtl
