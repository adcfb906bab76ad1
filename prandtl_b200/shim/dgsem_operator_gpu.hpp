// dgsem_operator_gpu.hpp -- header-only MFEM adapter over the C ABI.
//
// Drop-in for Prandtl::DGSEMOperator (src/Operators/DGSEMOperator.hpp:15-141):
// the same mfem::TimeDependentOperator surface (Mult, GetMaxCharSpeed,
// GetTimeRef), so Simulation's ODESolver::Init / Step (Simulation.cpp:807,
// :1010) drive the sm_100a kernels unchanged.  The caller builds the
// prandtl_mesh_desc from its mesh: per element the adjugate and determinant of
// the affine Jacobian, per face Elem1/Elem2, their local faces and the
// CalcOrtho scaled normal.  mfem::Vector data are host arrays in
// Ordering::byNODES, exactly the layout the kernels use.
#pragma once

#include <stdexcept>
#include <string>

#include "prandtl_b200.h"

namespace prandtl {
namespace gpu {

class DGSEMOperatorGPU : public mfem::TimeDependentOperator {
public:
    DGSEMOperatorGPU(const prandtl_mesh_desc &mesh, const prandtl_config &cfg)
        : mfem::TimeDependentOperator((mesh.dim + 2) * mesh.num_elements * ipow(mesh.order + 1, mesh.dim)) {
        prandtl_status st = prandtl_create(&mesh, &cfg, &h_);
        if (st != PRANDTL_OK) throw std::runtime_error(std::string("prandtl_create: ") + prandtl_last_error(nullptr));
    }
    ~DGSEMOperatorGPU() override { prandtl_destroy(h_); }
    DGSEMOperatorGPU(const DGSEMOperatorGPU &) = delete;
    DGSEMOperatorGPU &operator=(const DGSEMOperatorGPU &) = delete;

    // DGSEMOperator::Mult (DGSEMOperator.cpp:537-591)
    void Mult(const mfem::Vector &u, mfem::Vector &dudt) const override {
        double lam = 0.0;
        check(prandtl_rhs(h_, u.GetData(), dudt.GetData(), t, &lam, PRANDTL_PTR_HOST));
        max_char_speed_ = lam;
    }
    double GetMaxCharSpeed() const { return max_char_speed_; }
    double &GetTimeRef() { return t; }

    // Whole RK steps on the device (one host<->device round trip per call).
    void Step(mfem::Vector &u, double &time, double dt, int scheme = PRANDTL_RK3SSP, int nsteps = 1) {
        check(prandtl_step(h_, u.GetData(), time, dt, scheme, nsteps, PRANDTL_PTR_HOST));
        time += nsteps * dt;
    }
    prandtl_handle *handle() const { return h_; }

private:
    static int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }
    void check(prandtl_status st) const {
        if (st != PRANDTL_OK) throw std::runtime_error(std::string("prandtl: ") + prandtl_last_error(h_));
    }
    prandtl_handle *h_ = nullptr;
    mutable double max_char_speed_ = -1.0;
};

}   // namespace gpu
}   // namespace prandtl
