// prandtl_noalloc.cu -- RHS entry point that allocates no memory.
//
// For callers that cannot call cudaMalloc: code running inside another
// framework's memory pool or a fixed-footprint embedding, or code that must
// keep the device footprint constant after start-up.  They pass the mesh
// arrays, the state and the output already in device memory; everything
// else this path needs (the derived geometry / neighbour tables and, for
// Navier-Stokes, the lifted gradients) lives in one file-scope device array of
// a fixed size, PRANDTL_NOALLOC_SCRATCH_BYTES, that every GPU which loads the
// library holds until the process exits.  The 1D operator tables and the
// physics constants are built on the host stack by the same helpers the
// operator handle uses (host_common.hpp).
//
// The first call on a device looks the array's device address up with
// cudaGetSymbolAddress while that device is current, and creates the one
// CUDA event that bounds the wait for the mesh check; that first call should
// be made before any stream capture.  Every call then records that event
// behind the device-side mesh check and waits for it, bounded by
// cfg->timeout_s, before it enqueues the RHS kernels.  All calls share the
// array and it keeps the previous call's contents; each call rebuilds what it
// reads.  Calls that overlap on the GPU (different streams, or different host
// threads on one device) race on the array.
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
#include "host_common.hpp"

using namespace prandtl;

namespace {

constexpr size_t kScratchBytes = PRANDTL_NOALLOC_SCRATCH_BYTES;
constexpr size_t kAlign = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_ptr[kMaxDevices] = {nullptr};
cudaEvent_t g_check_done[kMaxDevices] = {nullptr};

size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// The message goes to the calling thread's fixed error buffer, which
// prandtl_last_error(NULL) returns (no allocation).
prandtl_status fail(prandtl_status st, const char *msg) {
    prandtl::host::set_unbound_error(msg);
    return st;
}

// Set-up of the current device, once: the device address of the scratch array
// and the event that marks the end of the mesh check.
prandtl_status device_setup(void **scratch, cudaEvent_t *check_done) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(PRANDTL_EUNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
        cudaEvent_t ev = nullptr;
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
        g_check_done[dev] = ev;
        g_scratch_ptr[dev] = p;
    }
    *scratch = g_scratch_ptr[dev];
    *check_done = g_check_done[dev];
    return PRANDTL_OK;
}

// geo[e] = {adj(J) row-major, det J}; neighbour slots start at -1.  Counts
// elements whose det J is not positive (the handle path rejects them too).
__global__ void noalloc_geometry(const double *__restrict__ adj, const double *__restrict__ detj,
                                 double *__restrict__ geo, int4 *__restrict__ nbr, int E, int dim,
                                 unsigned int *__restrict__ bad) {
    const int GEO = dim * dim + 1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < E;
         e += (long long)gridDim.x * blockDim.x) {
        for (int q = 0; q < dim * dim; ++q) geo[e * GEO + q] = adj[e * dim * dim + q];
        const double dj = detj[e];
        if (!(dj > 0.0)) atomicAdd(bad, 1u);
        geo[e * GEO + dim * dim] = dj;
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

// Waits for `ev` (recorded behind the mesh check), bounded by limit_s.
prandtl_status wait_event(cudaEvent_t ev, double limit_s) {
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaEventQuery(ev);
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
    prandtl::host::set_unbound_error("");
    if (!m || !cfg || !u || !dudt) return fail(PRANDTL_EINVAL, "null argument");
    if (m->dim != 2 && m->dim != 3) return fail(PRANDTL_EUNSUPPORTED, "dim must be 2 or 3");
    if (!order_supported(m->dim, m->order)) return fail(PRANDTL_EUNSUPPORTED, "order must be in 1..5");
    if (m->num_elements <= 0 || m->num_faces <= 0) return fail(PRANDTL_EINVAL, "bad sizes");
    if (!m->elem_adj || !m->elem_detj || !m->face_elems || !m->face_nor)
        return fail(PRANDTL_EINVAL, "mesh arrays missing");
    if (cfg->precision != 0) return fail(PRANDTL_EUNSUPPORTED, "only precision 0 (FP64) is built");
    if (cfg->axisymmetric) return fail(PRANDTL_EUNSUPPORTED, "the axisymmetric form needs prandtl_create");
    if (m->node_adj || m->node_detj || m->face_node_nor)
        return fail(PRANDTL_EUNSUPPORTED, "non-affine elements need prandtl_create");
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
    cudaEvent_t check_done = nullptr;
    prandtl_status st = device_setup(&base, &check_done);
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
    noalloc_geometry<<<gE, tpb, 0, s>>>(m->elem_adj, m->elem_detj, geo, nbr, E, dim, bad);
    noalloc_faces<<<gF, tpb, 0, s>>>(m->face_elems, F, E, dim, nbr, bad);
    noalloc_check<<<gS, tpb, 0, s>>>(nbr, nslots, bad);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
    // wait (bounded) for the check, then read its 4-byte count (a copy to
    // pageable memory returns once it has completed)
    if ((e = cudaEventRecord(check_done, s)) != cudaSuccess) return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
    st = wait_event(check_done, cfg->timeout_s > 0 ? cfg->timeout_s : 120.0);
    if (st != PRANDTL_OK) return st;
    unsigned int nbad = 0;
    if ((e = cudaMemcpyAsync(&nbad, bad, sizeof(nbad), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return fail(PRANDTL_ECUDA, cudaGetErrorString(e));
    if (nbad != 0)
        return fail(PRANDTL_EUNSUPPORTED,
                    "mesh invalid: faces out of range, duplicated or missing (only periodic meshes with aligned "
                    "faces), or a non-positive det J");

    OpTables T;
    prandtl::host::build_tables(m->order, T);
    PhysParams P{};
    prandtl::host::build_phys(*cfg, m->order, P);

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
