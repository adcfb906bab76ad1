// Drives the MFEM adapter the way Simulation::Run drives DGSEMOperator:
// Mult for the initial CFL dt, then ODESolver-style steps.  Prints the max
// |dudt| and the final state checksum; exit code 0 on success, 2 without a GPU.
#include <cmath>
#include <cstdio>
#include <vector>

#include "mfem_compat.hpp"
#include "dgsem_operator_gpu.hpp"

int main() {
    // 2x2 periodic unit square, N = 2, free stream plus a bump (generated here)
    const int dim = 2, order = 2, n = 2, E = n * n, Np = order + 1, nd = Np * Np;
    const double h = 1.0 / n;
    std::vector<double> adj(E * 4), detj(E, h * h), nor;
    std::vector<int> faces;
    for (int e = 0; e < E; ++e) { adj[4 * e] = h; adj[4 * e + 1] = 0; adj[4 * e + 2] = 0; adj[4 * e + 3] = h; }
    for (int d = 0; d < 2; ++d)
        for (int e = 0; e < E; ++e) {
            int c[2] = {e % n, e / n};
            c[d] = (c[d] + 1) % n;
            const int eu = c[0] + n * c[1];
            if (e < eu) { faces.insert(faces.end(), {e, 2 * d + 1, eu, 2 * d}); nor.push_back(d == 0 ? h : 0); nor.push_back(d == 1 ? h : 0); }
            else { faces.insert(faces.end(), {eu, 2 * d, e, 2 * d + 1}); nor.push_back(d == 0 ? -h : 0); nor.push_back(d == 1 ? -h : 0); }
        }
    prandtl_mesh_desc md{dim, order, E, (int)faces.size() / 4, adj.data(), detj.data(), faces.data(), nor.data()};
    prandtl_config cfg;
    prandtl_config_default(&cfg);
    try {
        prandtl::gpu::DGSEMOperatorGPU op(md, cfg);
        const int N = (dim + 2) * E * nd;
        mfem::Vector u(N), k(N);
        for (int i = 0; i < E * nd; ++i) {
            const double rho = 1.0 + 0.1 * std::sin(0.3 * i);
            u(i) = rho; u(E * nd + i) = 0.2 * rho; u(2 * E * nd + i) = -0.1 * rho;
            u(3 * E * nd + i) = 1.0 / 0.4 + 0.5 * rho * 0.05;
        }
        op.SetTime(0.0);
        op.Mult(u, k);
        double mx = 0;
        for (int i = 0; i < N; ++i) mx = std::fmax(mx, std::fabs(k(i)));
        double t = 0.0;
        const double dt = prandtl_cfl_dt(0.5, h, op.GetMaxCharSpeed(), order);
        op.Step(u, t, dt, PRANDTL_RK3SSP, 3);
        double sum = 0;
        for (int i = 0; i < N; ++i) sum += u(i);
        std::printf("max|dudt| %.17g lambda %.17g t %.17g checksum %.17g\n", mx, op.GetMaxCharSpeed(), t, sum);
    } catch (const std::exception &ex) {
        std::printf("error: %s\n", ex.what());
        return 2;
    }
    return 0;
}
