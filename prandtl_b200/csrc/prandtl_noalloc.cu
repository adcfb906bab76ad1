// prandtl_noalloc.cu -- RHS entry point that allocates no memory.
//
// For callers that cannot call cudaMalloc: code running inside another
// framework's memory pool or a fixed-footprint embedding, or code that must
// keep the device footprint constant after start-up.  They pass the mesh
// arrays, the state and the output already in device memory; everything
// else this path needs (the derived geometry / neighbour tables and, for
// Navier-Stokes, the lifted gradients) lives in one file-scope device array of
// a fixed size, PRANDTL_NOALLOC_SCRATCH_BYTES, that every GPU which loads the
// library holds until the process exits.  The 1D operator tables are built on
// the host stack.
//
// The first call on a device looks the array's device address up with
// cudaGetSymbolAddress while that device is current, so that first call should
// be made before any stream capture.  All calls share the array and it keeps
// the previous call's contents; each call rebuilds what it reads.  Calls that
// overlap on the GPU (different streams, or different host threads on one
// device) race on the array.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <thread>

#include "../../include/prandtl_b200.h"
#include "dgsem_kernels.cuh"

using namespace prandtl;

namespace {

constexpr size_t kScratchBytes = PRANDTL_NOALLOC_SCRATCH_BYTES;
constexpr size_t kAlign = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_ptr[kMaxDevices] = {nullptr};

size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// The message documents the failure at the return site; callers get the status.
prandtl_status fail(prandtl_status st, const char *) { return st; }

// Device address of the scratch array on the current device (looked up once).
prandtl_status scratch_address(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(PRANDTL_EUNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return PRANDTL_OK;
}

// Legendre P_N(t) and P'_N(t) by the three-term recurrence.
__host__ long double legendre_ld(int N, long double t, long double &dp) {
    long double p0 = 1.0L, p1 = t, dp0 = 0.0L, dp1 = 1.0L;
    for (int k = 1; k < N; ++k) {
        long double p2 = ((2 * k + 1) * t * p1 - k * p0) / (k + 1);
        long double dp2 = dp0 + (2 * k + 1) * p1;
        p0 = p1; p1 = p2; dp0 = dp1; dp1 = dp2;
    }
    dp = dp1;
    return p1;
}

// 1D operator tables on fixed-size stack arrays (Gauss-Lobatto on [0,1],
// derivative matrices of DGSEMIntegrator.cpp:41-82, inverse Legendre
// Vandermonde of ModalBasis.cpp:110-135).
void tables_on_stack(int N, OpTables &T) {
    const int Np = N + 1;
    std::memset(&T, 0, sizeof(T));
    const long double pi = 3.14159265358979323846264338327950288L;
    long double xs[8];
    for (int i = 0; i < Np; ++i) {
        long double t = -cosl(pi * i / N);
        if (i > 0 && i < N)
            for (int it = 0; it < 100; ++it) {
                long double dp, p = legendre_ld(N, t, dp);
                long double dx = ((1.0L - t * t) * dp) / (-(long double)N * (N + 1) * p);
                t -= dx;
                if (fabsl(dx) < 1e-30L) break;
            }
        xs[i] = t;
    }
    for (int i = 0; i < Np; ++i) {
        long double dp, p = legendre_ld(N, xs[i], dp);
        T.x[i] = (double)((xs[i] + 1.0L) * 0.5L);
        T.w[i] = (double)(2.0L / ((long double)N * (N + 1) * p * p) * 0.5L);
    }
    T.x[0] = 0.0;
    T.x[N] = 1.0;
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
    double V[64], I[64];
    for (int l = 0; l < Np; ++l) {
        double u[8], z = 2.0 * T.x[l] - 1.0;
        u[0] = 1.0;
        u[1] = z;
        for (int n = 1; n < N; ++n) u[n + 1] = ((2 * n + 1) * z * u[n] - n * u[n - 1]) / (n + 1);
        for (int a = 0; a < Np; ++a) V[l * Np + a] = u[a];
    }
    for (int q = 0; q < Np * Np; ++q) I[q] = 0.0;
    for (int i = 0; i < Np; ++i) I[i * Np + i] = 1.0;
    for (int c = 0; c < Np; ++c) {
        int piv = c;
        for (int r = c + 1; r < Np; ++r)
            if (std::fabs(V[r * Np + c]) > std::fabs(V[piv * Np + c])) piv = r;
        for (int k = 0; k < Np; ++k) {
            double t0 = V[c * Np + k]; V[c * Np + k] = V[piv * Np + k]; V[piv * Np + k] = t0;
            double t1 = I[c * Np + k]; I[c * Np + k] = I[piv * Np + k]; I[piv * Np + k] = t1;
        }
        const double d = 1.0 / V[c * Np + c];
        for (int k = 0; k < Np; ++k) { V[c * Np + k] *= d; I[c * Np + k] *= d; }
        for (int r = 0; r < Np; ++r) {
            if (r == c) continue;
            const double f = V[r * Np + c];
            for (int k = 0; k < Np; ++k) { V[r * Np + k] -= f * V[c * Np + k]; I[r * Np + k] -= f * I[c * Np + k]; }
        }
    }
    for (int q = 0; q < Np * Np; ++q) T.Vinv[q] = I[q];
}

// geo[e] = {adj(J) row-major, det J}; neighbour slots start at -1.
__global__ void noalloc_geometry(const double *__restrict__ adj, const double *__restrict__ detj,
                                 double *__restrict__ geo, int4 *__restrict__ nbr, int E, int dim) {
    const int GEO = dim * dim + 1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < E;
         e += (long long)gridDim.x * blockDim.x) {
        for (int q = 0; q < dim * dim; ++q) geo[e * GEO + q] = adj[e * dim * dim + q];
        geo[e * GEO + dim * dim] = detj[e];
        for (int lf = 0; lf < 2 * dim; ++lf) nbr[e * 2 * dim + lf] = make_int4(-1, -1, -1, -1);
    }
}

// Scatter every face into its two element slots; count faces that are out of
// range, not aligned opposite faces, or land on an already-filled slot.
__global__ void noalloc_faces(const int *__restrict__ faces, int F, int E, int dim,
                              int4 *__restrict__ nbr, unsigned int *__restrict__ bad) {
    const int NFACE = 2 * dim;
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < F;
         f += (long long)gridDim.x * blockDim.x) {
        const int e1 = faces[4 * f], l1 = faces[4 * f + 1], e2 = faces[4 * f + 2], l2 = faces[4 * f + 3];
        const bool ok = e1 >= 0 && e1 < E && e2 >= 0 && e2 < E && l1 >= 0 && l1 < NFACE && l2 >= 0 &&
                        l2 < NFACE && (l1 >> 1) == (l2 >> 1) && (l1 ^ l2) == 1;
        if (!ok) {
            atomicAdd(bad, 1u);
            continue;
        }
        int *s1 = reinterpret_cast<int *>(&nbr[(long long)e1 * NFACE + l1]);
        int *s2 = reinterpret_cast<int *>(&nbr[(long long)e2 * NFACE + l2]);
        if (atomicCAS(s1, -1, e2) != -1) { atomicAdd(bad, 1u); continue; }
        if (atomicCAS(s2, -1, e1) != -1) { atomicAdd(bad, 1u); continue; }
        s1[1] = l2; s1[2] = (int)f; s1[3] = 0;
        s2[1] = l1; s2[2] = (int)f; s2[3] = 1;
    }
}

// Every slot filled (periodic mesh: no boundary faces).
__global__ void noalloc_check(const int4 *__restrict__ nbr, long long n, unsigned int *__restrict__ bad) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        if (nbr[i].x < 0) atomicAdd(bad, 1u);
}

prandtl_status wait_stream(cudaStream_t s, double limit_s) {
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaStreamQuery(s);
        if (e == cudaSuccess) return PRANDTL_OK;
        if (e != cudaErrorNotReady) return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit_s)
            return fail(PRANDTL_ETIMEDOUT, "wait for the mesh check timed out");
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

}   // namespace

extern "C" prandtl_status prandtl_rhs_noalloc(const prandtl_mesh_desc *m, const prandtl_config *cfg,
                                              const double *u, double *dudt, void *stream) {
    if (!m || !cfg || !u || !dudt) return fail(PRANDTL_EINVAL, "null argument");
    if (m->dim != 2 && m->dim != 3) return fail(PRANDTL_EUNSUPPORTED, "dim must be 2 or 3");
    if (!order_supported(m->dim, m->order)) return fail(PRANDTL_EUNSUPPORTED, "order must be in 1..5");
    if (m->num_elements <= 0 || m->num_faces <= 0) return fail(PRANDTL_EINVAL, "bad sizes");
    if (!m->elem_adj || !m->elem_detj || !m->face_elems || !m->face_nor)
        return fail(PRANDTL_EINVAL, "mesh arrays missing");
    if (cfg->precision != 0) return fail(PRANDTL_EUNSUPPORTED, "only precision 0 (FP64) is built");
    if (cfg->axisymmetric) return fail(PRANDTL_EUNSUPPORTED, "the axisymmetric form needs prandtl_create");
    if (!(cfg->gamma > 1.0) || !(cfg->Pr > 0.0)) return fail(PRANDTL_EINVAL, "bad gamma/Pr");

    const int dim = m->dim, E = m->num_elements, F = m->num_faces, NFACE = 2 * dim;
    int nd = 1;
    for (int d = 0; d < dim; ++d) nd *= m->order + 1;
    const long long Ndof = (long long)E * nd;
    const size_t grad_bytes = cfg->parabolic ? align_up((size_t)dim * (dim + 2) * Ndof * sizeof(double)) : 0;
    const size_t geo_bytes = align_up((size_t)E * (dim * dim + 1) * sizeof(double));
    const size_t nbr_bytes = align_up((size_t)E * NFACE * sizeof(int4));
    const size_t flag_bytes = kAlign;
    if (grad_bytes + geo_bytes + nbr_bytes + flag_bytes > kScratchBytes)
        return fail(PRANDTL_ETOOLARGE, "mesh needs more than PRANDTL_NOALLOC_SCRATCH_BYTES of scratch");

    void *base = nullptr;
    prandtl_status st = scratch_address(&base);
    if (st != PRANDTL_OK) return st;
    unsigned char *p = static_cast<unsigned char *>(base);
    double *grad = cfg->parabolic ? reinterpret_cast<double *>(p) : nullptr;
    double *geo = reinterpret_cast<double *>(p + grad_bytes);
    int4 *nbr = reinterpret_cast<int4 *>(p + grad_bytes + geo_bytes);
    unsigned int *bad = reinterpret_cast<unsigned int *>(p + grad_bytes + geo_bytes + nbr_bytes);
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    cudaError_t e;
    if ((e = cudaMemsetAsync(bad, 0, sizeof(unsigned int), s)) != cudaSuccess)
        return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
    const int tpb = 256;
    const int gE = (int)std::min<long long>((E + tpb - 1) / tpb, 4096);
    const int gF = (int)std::min<long long>((F + tpb - 1) / tpb, 4096);
    const long long nslots = (long long)E * NFACE;
    const int gS = (int)std::min<long long>((nslots + tpb - 1) / tpb, 4096);
    noalloc_geometry<<<gE, tpb, 0, s>>>(m->elem_adj, m->elem_detj, geo, nbr, E, dim);
    noalloc_faces<<<gF, tpb, 0, s>>>(m->face_elems, F, E, dim, nbr, bad);
    noalloc_check<<<gS, tpb, 0, s>>>(nbr, nslots, bad);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
    unsigned int nbad = 0;
    if ((e = cudaMemcpyAsync(&nbad, bad, sizeof(nbad), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
    st = wait_stream(s, cfg->timeout_s > 0 ? cfg->timeout_s : 120.0);
    if (st != PRANDTL_OK) return st;
    if (nbad != 0)
        return fail(PRANDTL_EUNSUPPORTED,
                    "mesh faces invalid, duplicated, or missing (only periodic meshes with aligned faces)");

    OpTables T;
    tables_on_stack(m->order, T);
    PhysParams P{};
    P.gamma = cfg->gamma;
    P.gammaM1 = cfg->gamma - 1.0;
    P.gammaM1Inverse = 1.0 / P.gammaM1;
    P.PrInverse = 1.0 / cfg->Pr;
    P.mu = cfg->mu;
    P.mu_bulk = 2.0 / 3.0;
    P.R_gas = cfg->R_gas;
    P.mu0 = 1.716e-5;
    P.T0 = 273.15;
    P.Ts = 110.4;
    P.T0pTs = P.T0 + P.Ts;
    P.alpha_max = cfg->alpha_max;
    P.alpha_min = cfg->alpha_min;
    P.modal_threshold = 0.5 * std::pow(10.0, -1.8 * std::pow((double)m->order, 0.25));
    P.sutherland = cfg->sutherland;
    P.quirks = cfg->quirks;
    P.dissipation = cfg->surface_dissipation;
    P.blending = cfg->blending;

    MeshDev md{};
    md.geo = geo;
    md.nbr = nbr;
    md.fnor = m->face_nor;
    md.E = E;
    md.Ndof = Ndof;
    md.bcs = nullptr;   // periodic meshes only: boundary faces fail the check above
    if (cfg->parabolic) {
        LiftArgs la{u, grad};
        if ((e = launch_lift(dim, m->order, md, la, P, T, s)) != cudaSuccess)
            return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
    }
    RhsArgs a{};
    a.u = u;
    a.grad = grad;
    a.dudt = dudt;
    a.mode = EPI_STORE;
    if ((e = launch_rhs(dim, m->order, cfg->parabolic != 0, md, a, P, T, s)) != cudaSuccess)
        return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
    return PRANDTL_OK;
}
