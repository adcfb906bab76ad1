// ref_driver.cpp -- runs the reference's own integrator sources (compiled
// against mfem_standin/mfem.hpp) on a periodic affine mesh, to pin the CPU
// oracle.  TEST INFRASTRUCTURE ONLY: built into oracle/_ref/, never shipped.
//
// The per-element / per-face arithmetic comes from the reference sources
// themselves (DGSEMIntegrator, LiftingBR1, ChandrashekarFlux,
// NavierStokesFlux, BasicOperations, PerssonPeraireIndicator, ModalBasis).
// This file supplies what lives in MFEM or in classes that cannot be built
// without MFEM: the stand-in geometry, and the assembly loops of
// DGSEMOperator::Mult (DGSEMOperator.cpp:537-591, :60-159) and
// DGSEMNonlinearForm::Mult / MultLifting (DGSEMNonlinearForm.cpp:424-849,
// :1070-1545), restated for serial affine meshes (no shared faces, P =
// identity).  Boundary faces (Euler only) run the reference's own boundary
// integrators with constant states.
#include "mfem.hpp"

#include "BasicOperations.hpp"
#include "ChandrashekarFlux.hpp"
// The reference reads the member DGSEMIntegrator::id1 before writing it when
// SUBCELL_FV_BLENDING is off (DGSEMIntegrator.cpp:620, uninitialised on the
// first element of the first call).  The harness sets it to Np^d-1, the value
// every later element inherits from the previous element's loop, so it needs
// the member to be reachable; the class layout is unchanged.
#define private public
#include "DGSEMIntegrator.hpp"
#undef private
#include "LiftingBR1.hpp"
#include "ModalBasis.hpp"
#include "NavierStokesFlux.hpp"
#include "PerssonPeraireIndicator.hpp"
#include "Physics.hpp"
#include "SlipWallBdrFaceIntegrator.hpp"
#include "SpecifiedStateBdrFaceIntegrator.hpp"
#include "SubsonicOutflowPBdrFaceIntegrator.hpp"
#include "SupersonicOutflowBdrFaceIntegrator.hpp"
#include "SymmetryBdrFaceIntegrator.hpp"
#include "RiemannInvariantBdrFaceIntegrator.hpp"
#include "SubsonicInflowRVBdrFaceIntegrator.hpp"
#include "SubsonicInflowPtTtAngBdrFaceIntegrator.hpp"
#include "NoSlipAdiabWallBdrFaceIntegrator.hpp"
#include "NoSlipIsothWallBdrFaceIntegrator.hpp"
#include "prandtl_oracle.h"

namespace mfem {

void GaussLobattoRule(int n, std::vector<real_t> &x, std::vector<real_t> &w) {
    const int N = n - 1;
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    auto leg = [&](long double t, long double &dp) {
        long double p0 = 1.0L, p1 = t, dp0 = 0.0L, dp1 = 1.0L;
        if (N == 0) { dp = 0; return 1.0L; }
        for (int k = 1; k < N; ++k) {
            long double p2 = ((2 * k + 1) * t * p1 - k * p0) / (k + 1);
            long double dp2 = dp0 + (2 * k + 1) * p1;
            p0 = p1; p1 = p2; dp0 = dp1; dp1 = dp2;
        }
        dp = dp1;
        return p1;
    };
    const long double pi = 3.14159265358979323846264338327950288L;
    for (int i = 0; i < n; ++i) {
        long double t = -cosl(pi * i / N);
        if (i > 0 && i < N)
            for (int it = 0; it < 100; ++it) {
                long double dp, p = leg(t, dp);
                long double dx = ((1.0L - t * t) * dp) / (-(long double)N * (N + 1) * p);
                t -= dx;
                if (fabsl(dx) < 1e-30L) break;
            }
        long double dp, p = leg(t, dp);
        x[i] = (double)((t + 1.0L) * 0.5L);
        w[i] = (double)(2.0L / ((long double)N * (N + 1) * p * p) * 0.5L);
    }
    x[0] = 0.0;
    x[N] = 1.0;
}

const IntegrationRule &TensorGL(int geom, int n) {
    static std::map<std::pair<int, int>, std::unique_ptr<IntegrationRule>> cache;
    auto key = std::make_pair(geom, n);
    auto it = cache.find(key);
    if (it != cache.end()) return *it->second;
    std::vector<real_t> x, w;
    GaussLobattoRule(n, x, w);
    std::unique_ptr<IntegrationRule> ir;
    if (geom == Geometry::POINT) {
        ir.reset(new IntegrationRule(1));
        ir->IntPoint(0).weight = 1.0;
    } else if (geom == Geometry::SEGMENT) {
        ir.reset(new IntegrationRule(n));
        for (int i = 0; i < n; ++i) { ir->IntPoint(i).x = x[i]; ir->IntPoint(i).weight = w[i]; }
    } else if (geom == Geometry::SQUARE) {
        ir.reset(new IntegrationRule(n * n));
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                IntegrationPoint &p = ir->IntPoint(j * n + i);
                p.x = x[i]; p.y = x[j]; p.weight = w[i] * w[j];
            }
    } else {
        ir.reset(new IntegrationRule(n * n * n));
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    IntegrationPoint &p = ir->IntPoint((k * n + j) * n + i);
                    p.x = x[i]; p.y = x[j]; p.z = x[k]; p.weight = w[i] * w[j] * w[k];
                }
    }
    auto &ref = *ir;
    cache[key] = std::move(ir);
    return ref;
}

FiniteElement::FiniteElement(int dim, int order) : dim_(dim), order_(order) {
    std::vector<real_t> w;
    GaussLobattoRule(order + 1, x_, w);
    const int geom = dim == 1 ? Geometry::SEGMENT : dim == 2 ? Geometry::SQUARE : Geometry::CUBE;
    nodes_ = order > 0 ? TensorGL(geom, order + 1) : IntegrationRule(1);
    if (order == 0) { nodes_.IntPoint(0).x = nodes_.IntPoint(0).y = nodes_.IntPoint(0).z = 0.5; }
}

void FiniteElement::CalcShape(const IntegrationPoint &ip, Vector &shape) const {
    const int Np = order_ + 1;
    const real_t xi[3] = {ip.x, ip.y, ip.z};
    real_t l[3][16];
    for (int d = 0; d < dim_; ++d)
        for (int i = 0; i < Np; ++i) {
            real_t v = 1.0;
            for (int m = 0; m < Np; ++m)
                if (m != i) v *= (xi[d] - x_[m]) / (x_[i] - x_[m]);
            l[d][i] = v;
        }
    const int nd = GetDof();
    for (int n = 0; n < nd; ++n) {
        const int c[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
        real_t v = l[0][c[0]];
        for (int d = 1; d < dim_; ++d) v *= l[d][c[d]];
        shape(n) = v;
    }
}

void FaceElementTransformations::SetAllIntPoints(const IntegrationPoint *fip) {
    auto map = [&](int lf, IntegrationPoint &e) {
        const int d = lf >> 1, s = lf & 1;
        real_t c[3] = {0, 0, 0};
        c[d] = s;
        if (dim == 2) {
            c[1 - d] = fip->x;
        } else {
            const int t0 = (d == 0) ? 1 : 0, t1 = (d == 2) ? 1 : 2;
            c[t0] = fip->x;
            c[t1] = fip->y;
        }
        e.x = c[0]; e.y = c[1]; e.z = c[2];
    };
    map(lf1, eip1);
    T1->SetIntPoint(&eip1);
    if (T2) {   // boundary faces have no element 2
        map(lf2, eip2);
        T2->SetIntPoint(&eip2);
    }
    const int d = lf1 >> 1;
    Jf.SetSize(dim, dim - 1);
    if (dim == 2) {
        for (int r = 0; r < 2; ++r) Jf(r, 0) = orient * T1->J(r, 1 - d);
    } else {
        const int t0 = (d == 0) ? 1 : 0, t1 = (d == 2) ? 1 : 2;
        for (int r = 0; r < 3; ++r) { Jf(r, 0) = orient * T1->J(r, t0); Jf(r, 1) = T1->J(r, t1); }
    }
}

}   // namespace mfem

using namespace mfem;
using namespace Prandtl;

namespace {

// Stand-in ParMesh from the oracle descriptor: affine elements from the
// per-element adjugates, or (descriptor with per-node geometry) multilinear
// elements from their corner nodes, which the Gauss-Lobatto node coordinates
// include.
std::shared_ptr<ParMesh> make_mesh(const oracle_mesh *m, const double *coords = nullptr) {
    auto pm = std::make_shared<ParMesh>();
    const int dim = m->dim, Np = m->order + 1;
    int nd = 1;
    for (int d = 0; d < dim; ++d) nd *= Np;
    const long Ndof = (long)m->num_elements * nd;
    const bool multi = m->node_adj != nullptr;
    if (multi && !coords) throw std::runtime_error("multilinear elements need the node coordinates");
    pm->dim = dim;
    pm->trans.resize(m->num_elements);
    for (int e = 0; e < m->num_elements; ++e) {
        ElementTransformation &T = pm->trans[e];
        T.ElementNo = e;
        T.dim = dim;
        T.adj.SetSize(dim);
        T.J.SetSize(dim);
        if (multi) {
            T.multilinear = true;
            for (int b = 0; b < (1 << dim); ++b) {
                const int n = ((b & 1) + Np * ((b >> 1) & 1) + Np * Np * ((b >> 2) & 1)) * (Np - 1);
                for (int d = 0; d < dim; ++d) T.corner[b][d] = coords[d * Ndof + (long)e * nd + n];
            }
            continue;
        }
        const double *a = m->elem_adj + (size_t)e * dim * dim;
        for (int r = 0; r < dim; ++r)
            for (int c = 0; c < dim; ++c) T.adj(r, c) = a[r * dim + c];
        T.detJ = m->elem_detj[e];
        // J = det(J) adj(J)^{-1}
        DenseMatrix inv(T.adj);
        inv.Invert();
        for (int r = 0; r < dim; ++r)
            for (int c = 0; c < dim; ++c) T.J(r, c) = T.detJ * inv(r, c);
        if (coords)   // origin = node 0 of the element (xi = 0)
            for (int d = 0; d < dim; ++d) T.x0[d] = coords[d * Ndof + (long)e * nd];
    }
    for (int f = 0; f < m->num_faces; ++f) {
        const int *fe = m->face_elems + 4 * f;
        auto F = std::make_unique<FaceElementTransformations>();
        F->ElementNo = f;
        F->Elem1No = fe[0]; F->lf1 = fe[1];
        F->Elem2No = fe[2]; F->lf2 = fe[3];
        F->dim = dim;
        F->T1 = &pm->trans[fe[0]];
        F->T2 = fe[2] >= 0 ? &pm->trans[fe[2]] : nullptr;
        // orientation: CalcOrtho of element 1's tangential columns at the face
        // centre against the outward adjugate row there
        const int d = fe[1] >> 1, s = fe[1] & 1;
        IntegrationPoint c;
        c.x = 0.5; c.y = 0.5; c.z = 0.0;
        F->orient = 1.0;
        F->SetAllIntPoints(&c);
        Vector n(dim);
        CalcOrtho(F->Jf, n);
        real_t dot = 0.0;
        for (int q = 0; q < dim; ++q) dot += n(q) * F->T1->adj(d, q) * (s ? 1.0 : -1.0);
        if (dot < 0) F->orient = -1.0;
        F->SetAllIntPoints(&c);
        pm->faces.push_back(std::move(F));
    }
    return pm;
}

}   // namespace

extern "C" int ref_variant_parabolic() {
#ifdef PARABOLIC
    return 1;
#else
    return 0;
#endif
}
extern "C" int ref_variant_blending() {
#ifdef SUBCELL_FV_BLENDING
    return 1;
#else
    return 0;
#endif
}

// One RHS evaluation with the reference integrators.  Returns 0 on success.
extern "C" int ref_rhs(const oracle_mesh *md, const oracle_config *cfg, const double *u_in,
                       double *dudt_out, double *alpha_out, double *grad_out) {
    try {
        const int dim = md->dim, order = md->order, Np = order + 1, nf = dim + 2;
        PhysicsConstants pc(cfg->gamma, cfg->Pr, cfg->R_gas, cfg->mu);
        NavierStokesFlux flux(dim, pc.gamma, pc.Pr, pc.mu, pc.mu0, pc.mu_bulk, pc.R_gas, pc.Ts, pc.T0);
        ChandrashekarFlux rsolver(flux, pc.gamma);
        std::shared_ptr<LiftingScheme> lifting;
#ifdef PARABOLIC
        lifting = std::make_shared<LiftingBR1>();
#endif
        auto pmesh = make_mesh(md, cfg->node_coords);
        DG_FECollection fec(order, dim, BasisType::GaussLobatto), fec0(0, dim);
        auto vfes = std::make_shared<ParFiniteElementSpace>(pmesh.get(), &fec, nf);
        auto fes0 = std::make_shared<ParFiniteElementSpace>(pmesh.get(), &fec0, 1);
        auto eta = std::make_shared<ParGridFunction>(fes0.get());
        auto alpha = std::make_shared<ParGridFunction>(fes0.get());
        *alpha = 0.0;
        DGSEMIntegrator integ(pmesh, fes0, alpha, lifting, rsolver, Np, pc.gamma);
        const int NE = pmesh->GetNE(), Ndofs = vfes->GetFE(0)->GetDof();
        integ.id1 = Ndofs - 1;
        const int N = vfes->GetVSize();
        Vector u(const_cast<double *>(u_in), N), dudt(dudt_out, N);

#ifdef SUBCELL_FV_BLENDING
        {   // DGSEMOperator::ComputeBlendingCoefficient (DGSEMOperator.cpp:60-80)
            Geometry::Type gtype = (Geometry::Type)vfes->GetFE(0)->GetGeomType();
            PerssonPeraireIndicator ind(vfes, fes0, eta, std::make_shared<ModalBasis>(fec, gtype, order, dim),
                                        pc.gamma);
            ind.CheckSmoothness(u);
            const real_t thr = 0.5 * std::pow(10.0, -1.8 * std::pow(order, 0.25));
            Array<int> ind_indx;
            Vector ind_dof;
            for (int el = 0; el < NE; el++) {
                fes0->GetElementDofs(el, ind_indx);
                eta->GetSubVector(ind_indx, ind_dof);
                real_t a = 1.0 / (1.0 + std::exp(-9.21024 * (ind_dof(0) - thr) / thr));
                if (a < cfg->alpha_min) a = 0.0;
                else if (a > (1.0 - cfg->alpha_min)) a = 1.0;
                a = std::min(a, cfg->alpha_max);
                alpha->SetSubVector(ind_indx, a);
            }
        }
#endif
        if (alpha_out)
            for (int e = 0; e < NE; ++e) alpha_out[e] = (*alpha)(e);

        Array<int> vdofs, vdofs2;
        Vector el_u, el_dudt;
        const FiniteElement *fe = vfes->GetFE(0);
        dudt = 0.0;
        // the reference's boundary integrator of each condition (constant data;
        // the adiabatic wall through coefficient functions, as Simulation::LoadConfig
        // builds it, Simulation.cpp:540-632)
        std::vector<std::unique_ptr<BdrFaceIntegrator>> bdr;
        std::vector<std::unique_ptr<FunctionCoefficient>> scoef;
        std::vector<std::unique_ptr<VectorFunctionCoefficient>> vcoef;
        const real_t time = 0.0;
        for (int k = 0; k < cfg->num_bcs; ++k) {
            const oracle_bc &b = cfg->bcs[k];
            switch (b.type) {
            case ORACLE_BC_STATE: {
                Vector st(nf);
                for (int f = 0; f < nf; ++f) st(f) = b.state[f];
                bdr.emplace_back(new SpecifiedStateBdrFaceIntegrator(lifting, rsolver, Np, time, pc.gamma, st));
                break;
            }
            case ORACLE_BC_OUTFLOW:
                bdr.emplace_back(new SupersonicOutflowBdrFaceIntegrator(lifting, rsolver, Np, time, pc.gamma));
                break;
            case ORACLE_BC_SLIP_WALL:
                bdr.emplace_back(new SlipWallBdrFaceIntegrator(lifting, rsolver, Np, time, pc.gamma, true, false));
                break;
            case ORACLE_BC_SYMMETRY:
            case ORACLE_BC_AXIS:   // Simulation.cpp:520-530: "axis" adds the symmetry integrator
                bdr.emplace_back(new SymmetryBdrFaceIntegrator(lifting, rsolver, Np, time, pc.gamma, true, false));
                break;
            case ORACLE_BC_PRESSURE_OUTFLOW:
                bdr.emplace_back(new SubsonicOutflowPBdrFaceIntegrator(lifting, rsolver, Np, time, pc.gamma, b.p));
                break;
            case ORACLE_BC_RIEMANN: {
                Vector prim(nf);
                for (int f = 0; f < nf; ++f) prim(f) = b.state[f];
                bdr.emplace_back(new RiemannInvariantBdrFaceIntegrator(lifting, rsolver, Np, time, pc.gamma, prim));
                break;
            }
            case ORACLE_BC_INFLOW_RV: {
                Vector V(dim);
                for (int d = 0; d < dim; ++d) V(d) = b.state[1 + d];
                bdr.emplace_back(new SubsonicInflowRVBdrFaceIntegrator(lifting, rsolver, Np, time, pc.gamma,
                                                                       b.state[0], V));
                break;
            }
            case ORACLE_BC_INFLOW_PTTT:
                // the 3D constructor writes one past the end of its direction vector
                if (dim > 2) throw std::runtime_error("SubsonicInflowPtTtAng is not constructed in 3D");
                bdr.emplace_back(new SubsonicInflowPtTtAngBdrFaceIntegrator(lifting, rsolver, Np, time, pc.gamma, b.cp,
                                                                            b.pt, b.Tt, b.theta, b.phi));
                break;
            case ORACLE_BC_NOSLIP_ADIABATIC: {
                const double qn = b.heat_flux, v0 = b.wall_vel[0], v1 = b.wall_vel[1], v2 = b.wall_vel[2];
                scoef.emplace_back(new FunctionCoefficient([qn](const Vector &) { return qn; }));
                vcoef.emplace_back(new VectorFunctionCoefficient(dim, [v0, v1, v2, dim](const Vector &, Vector &v) {
                    v(0) = v0;
                    if (dim > 1) v(1) = v1;
                    if (dim > 2) v(2) = v2;
                }));
                bdr.emplace_back(new NoSlipAdiabWallBdrFaceIntegrator(lifting, rsolver, Np, time, pc.gamma,
                                                                      *scoef.back(), *vcoef.back(), false));
                break;
            }
            case ORACLE_BC_NOSLIP_ISOTHERMAL: {
                Vector V(dim);
                for (int d = 0; d < dim; ++d) V(d) = b.wall_vel[d];
                real_t T = b.wall_T;
                bdr.emplace_back(new NoSlipIsothWallBdrFaceIntegrator(lifting, rsolver, Np, time, pc.gamma,
                                                                      cfg->R_gas, T, V));
                break;
            }
            default:
                throw std::runtime_error("unknown boundary condition");
            }
        }
#ifdef PARABOLIC
        {
            // ComputeGlobalEntropyVector (DGSEMOperator.cpp:82-94)
            Vector ent(N), el_vdofs;
            DenseMatrix ent_mat(Ndofs, nf);
            for (int el = 0; el < NE; el++) {
                vfes->GetElementVDofs(el, vdofs);
                u.GetSubVector(vdofs, el_vdofs);
                DenseMatrix vdof_mat(el_vdofs.GetData(), Ndofs, nf);
                Conserv2Entropy(vdof_mat, ent_mat, pc.gamma, pc.gammaM1, pc.gammaM1Inverse);
                ent.SetSubVector(vdofs, ent_mat.GetData());
            }
            // MultLifting (DGSEMNonlinearForm.cpp:213-645), P = I
            std::vector<Vector> g(dim, Vector(N));
            for (auto &v : g) v = 0.0;
            std::vector<Vector> elg(3);
            for (int i = 0; i < NE; i++) {
                vfes->GetElementVDofs(i, vdofs);
                ent.GetSubVector(vdofs, el_u);
                if (dim == 3) integ.AssembleLiftingElementVector(*fe, *pmesh->GetElementTransformation(i), el_u, elg[0], elg[1], elg[2]);
                else integ.AssembleLiftingElementVector(*fe, *pmesh->GetElementTransformation(i), el_u, elg[0], elg[1]);
                for (int d = 0; d < dim; ++d) g[d].AddElementVector(vdofs, elg[d]);
            }
            for (int i = 0; i < pmesh->GetNumFaces(); i++) {
                FaceElementTransformations *tr = pmesh->GetInteriorFaceTransformations(i);
                if (tr->Elem2No < 0) continue;
                vfes->GetElementVDofs(tr->Elem1No, vdofs);
                vfes->GetElementVDofs(tr->Elem2No, vdofs2);
                vdofs.Append(vdofs2);
                ent.GetSubVector(vdofs, el_u);
                if (dim == 3) integ.AssembleLiftingFaceVector(*fe, *fe, *tr, el_u, elg[0], elg[1], elg[2]);
                else integ.AssembleLiftingFaceVector(*fe, *fe, *tr, el_u, elg[0], elg[1]);
                for (int d = 0; d < dim; ++d) g[d].AddElementVector(vdofs, elg[d]);
            }
            // boundary faces (DGSEMNonlinearForm.cpp:561-610)
            for (int i = 0; i < pmesh->GetNumFaces(); i++) {
                FaceElementTransformations *tr = pmesh->GetInteriorFaceTransformations(i);
                if (tr->Elem2No >= 0) continue;
                vfes->GetElementVDofs(tr->Elem1No, vdofs);
                ent.GetSubVector(vdofs, el_u);
                if (dim == 3) bdr.at(tr->lf2)->AssembleLiftingFaceVector(*fe, *fe, *tr, el_u, elg[0], elg[1], elg[2]);
                else bdr.at(tr->lf2)->AssembleLiftingFaceVector(*fe, *fe, *tr, el_u, elg[0], elg[1]);
                for (int d = 0; d < dim; ++d) g[d].AddElementVector(vdofs, elg[d]);
            }
            // ComputeGlobalPrimitiveGradVector (DGSEMOperator.cpp:112-159)
            Vector grad_vdofs;
            for (int el = 0; el < NE; el++) {
                vfes->GetElementVDofs(el, vdofs);
                u.GetSubVector(vdofs, el_vdofs);
                DenseMatrix vdof_mat(el_vdofs.GetData(), Ndofs, nf);
                for (int d = 0; d < dim; ++d) {
                    g[d].GetSubVector(vdofs, grad_vdofs);
                    DenseMatrix grad_mat(grad_vdofs.GetData(), Ndofs, nf);
                    EntropyGrad2PrimGrad(vdof_mat, grad_mat, pc.gammaM1, pc.gammaM1Inverse);
                    g[d].SetSubVector(vdofs, grad_mat.GetData());
                }
            }
            if (grad_out)
                for (int d = 0; d < dim; ++d) std::memcpy(grad_out + (size_t)d * N, g[d].GetData(), sizeof(double) * N);
            // Mult (DGSEMNonlinearForm.cpp:1070-1545)
            Vector gx, gy, gz;
            for (int i = 0; i < NE; i++) {
                vfes->GetElementVDofs(i, vdofs);
                u.GetSubVector(vdofs, el_u);
                g[0].GetSubVector(vdofs, gx);
                g[1].GetSubVector(vdofs, gy);
                if (dim == 3) {
                    g[2].GetSubVector(vdofs, gz);
                    integ.AssembleElementVector(*fe, *pmesh->GetElementTransformation(i), el_u, gx, gy, gz, el_dudt);
                } else {
                    integ.AssembleElementVector(*fe, *pmesh->GetElementTransformation(i), el_u, gx, gy, el_dudt);
                }
                dudt.AddElementVector(vdofs, el_dudt);
            }
            for (int i = 0; i < pmesh->GetNumFaces(); i++) {
                FaceElementTransformations *tr = pmesh->GetInteriorFaceTransformations(i);
                if (tr->Elem2No < 0) continue;
                vfes->GetElementVDofs(tr->Elem1No, vdofs);
                vfes->GetElementVDofs(tr->Elem2No, vdofs2);
                vdofs.Append(vdofs2);
                u.GetSubVector(vdofs, el_u);
                g[0].GetSubVector(vdofs, gx);
                g[1].GetSubVector(vdofs, gy);
                if (dim == 3) {
                    g[2].GetSubVector(vdofs, gz);
                    integ.AssembleFaceVector(*fe, *fe, *tr, el_u, gx, gy, gz, el_dudt);
                } else {
                    integ.AssembleFaceVector(*fe, *fe, *tr, el_u, gx, gy, el_dudt);
                }
                dudt.AddElementVector(vdofs, el_dudt);
            }
            // boundary faces (DGSEMNonlinearForm.cpp:1480-1525)
            for (int i = 0; i < pmesh->GetNumFaces(); i++) {
                FaceElementTransformations *tr = pmesh->GetInteriorFaceTransformations(i);
                if (tr->Elem2No >= 0) continue;
                vfes->GetElementVDofs(tr->Elem1No, vdofs);
                u.GetSubVector(vdofs, el_u);
                g[0].GetSubVector(vdofs, gx);
                g[1].GetSubVector(vdofs, gy);
                if (dim == 3) {
                    g[2].GetSubVector(vdofs, gz);
                    bdr.at(tr->lf2)->AssembleFaceVector(*fe, *fe, *tr, el_u, gx, gy, gz, el_dudt);
                } else {
                    bdr.at(tr->lf2)->AssembleFaceVector(*fe, *fe, *tr, el_u, gx, gy, el_dudt);
                }
                dudt.AddElementVector(vdofs, el_dudt);
            }
        }
#else
        // Mult (DGSEMNonlinearForm.cpp:647-849)
        for (int i = 0; i < NE; i++) {
            vfes->GetElementVDofs(i, vdofs);
            u.GetSubVector(vdofs, el_u);
            integ.AssembleElementVector(*fe, *pmesh->GetElementTransformation(i), el_u, el_dudt);
            dudt.AddElementVector(vdofs, el_dudt);
        }
        for (int i = 0; i < pmesh->GetNumFaces(); i++) {
            FaceElementTransformations *tr = pmesh->GetInteriorFaceTransformations(i);
            if (tr->Elem2No < 0) continue;
            vfes->GetElementVDofs(tr->Elem1No, vdofs);
            vfes->GetElementVDofs(tr->Elem2No, vdofs2);
            vdofs.Append(vdofs2);
            u.GetSubVector(vdofs, el_u);
            integ.AssembleFaceVector(*fe, *fe, *tr, el_u, el_dudt);
            dudt.AddElementVector(vdofs, el_dudt);
        }
        for (int i = 0; i < pmesh->GetNumFaces(); i++) {
            FaceElementTransformations *tr = pmesh->GetInteriorFaceTransformations(i);
            if (tr->Elem2No >= 0) continue;
            vfes->GetElementVDofs(tr->Elem1No, vdofs);
            u.GetSubVector(vdofs, el_u);
            bdr.at(tr->lf2)->AssembleFaceVector(*fe, *fe, *tr, el_u, el_dudt);
            dudt.AddElementVector(vdofs, el_dudt);
        }
#endif
#ifdef AXISYMMETRIC
        // u is the state recovered from r U (DGSEMOperator::Mult, restated by the
        // caller); DGSEMOperator::ZeroAxisRadialMom: zero radial-momentum rate at
        // the |r| <= 1e-14 nodes of elements on "axis" boundaries
        for (int f = 0; f < md->num_faces; ++f) {
            const int *fe4 = md->face_elems + 4 * f;
            if (fe4[2] >= 0 || cfg->bcs[fe4[3]].type != ORACLE_BC_AXIS) continue;
            for (int n = 0; n < Ndofs; ++n) {
                const long g = (long)fe4[0] * Ndofs + n;
                if (std::abs(cfg->node_coords[(long)NE * Ndofs + g]) <= 1e-14) dudt(2 * (long)NE * Ndofs + g) = 0.0;
            }
        }
#endif
        (void)grad_out;
        return 0;
    } catch (const std::exception &ex) {
        std::fprintf(stderr, "ref_rhs: %s\n", ex.what());
        return 1;
    }
}

// Reference point-wise routines, exported for golden vectors.
extern "C" double ref_log_mean(double x, double y) { return Prandtl::ComputeLogMean(x, y); }
