// dgsem_impl.cuh -- DGSEM RHS and BR1 lifting kernels for sm_100a (templates;
// each dgsem_inst_*.cu translation unit instantiates one dimension, working
// precision and physics).
//
// RHS: one lane group (a warp, or a power-of-two part of one for small
// elements) per element.  Everything an element needs stays in shared memory
// for the whole evaluation:
//   load state -> hoisted per-node primitives -> (blending coefficient) ->
//   two-point volume fluxes of all unique node pairs -> flux differencing ->
//   (subcell FV) -> surface fluxes of the element's own faces (neighbour
//   traces read from global/L2) -> epilogue (store dudt, or fuse the
//   Runge-Kutta stage update).
// Each interior face flux is evaluated by both neighbouring elements with the
// same operands in the same order, so both sides see bit-identical fluxes and
// no atomics or face buffers are needed.
//
// Two drivers share the element functions: one-shot kernels over one mesh
// (grid = ceil(E / elements per CTA)) and persistent batch kernels that walk
// the work items of many independent solves of one (dim, order, physics)
// class.
#pragma once

#include <atomic>
#include <cstdint>

#include "dgsem_kernels.cuh"

namespace prandtl {
namespace {


constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }
constexpr int cmax(int a, int b) { return a > b ? a : b; }

template <int DIM, int NP>
struct Shape {
    static constexpr int ND = ipow(NP, DIM);            // nodes per element
    static constexpr int NF = DIM + 2;                  // conserved fields
    static constexpr int NLINE = ND / NP;               // lines per direction
    static constexpr int PPL = NP * (NP - 1) / 2;       // unique pairs per line
    static constexpr int NFN = ND / NP;                 // nodes per face
    static constexpr int NFACE = 2 * DIM;
    static constexpr int NFI = NFACE * NFN;             // face-node items
    static constexpr int EPB = cmax(1, 128 / ND);       // elements per CTA
    static constexpr int THREADS = EPB * ND;
    static constexpr int TAB = 4 * NP * NP + 2 * NP;    // D, Dhat, Dhat2, Vinv, w, x
};

// Node coordinates (i, j, k) of element-local node n (x fastest).
template <int NP>
__device__ __forceinline__ void node_coords(int n, int c[3]) {
    c[0] = n % NP;
    c[1] = (n / NP) % NP;
    c[2] = n / (NP * NP);
}

// Line containing node coordinates c in direction dir, and its base/stride.
template <int DIM, int NP>
__device__ __forceinline__ int line_index(int dir, const int c[3]) {
    if (DIM == 2) return dir == 0 ? c[1] : c[0];
    return dir == 0 ? c[2] * NP + c[1] : (dir == 1 ? c[2] * NP + c[0] : c[1] * NP + c[0]);
}
template <int DIM, int NP>
__device__ __forceinline__ void line_base(int dir, int ln, int &base, int &stride) {
    if (DIM == 2) {
        if (dir == 0) { base = ln * NP; stride = 1; }
        else { base = ln; stride = NP; }
    } else {
        if (dir == 0) { base = ln * NP; stride = 1; }
        else if (dir == 1) { base = (ln / NP) * NP * NP + ln % NP; stride = NP; }
        else { base = ln; stride = NP * NP; }
    }
}
// Unique pair (a < b) <-> index, a-major.
template <int NP>
__device__ __forceinline__ int pair_index(int a, int b) {
    return a * NP - a * (a + 1) / 2 + (b - a - 1);
}
template <int NP>
__device__ __forceinline__ void pair_decode(int pp, int &a, int &b) {
    a = 0;
#pragma unroll
    for (int q = 0; q < NP - 1; ++q) {
        if (pp >= NP - 1 - a) { pp -= NP - 1 - a; ++a; }
    }
    b = a + 1 + pp;
}
// Element-local node of face node `a` on local face lf = 2*dir + side.
template <int DIM, int NP>
__device__ __forceinline__ int face_node(int lf, int a) {
    const int d = lf >> 1, s = lf & 1;
    int c[3] = {0, 0, 0};
    c[d] = s * (NP - 1);
    if (DIM == 2) {
        c[1 - d] = a;
        return c[1] * NP + c[0];
    }
    const int t0 = (d == 0) ? 1 : 0, t1 = (d == 2) ? 1 : 2;
    c[t0] = a % NP;
    c[t1] = a / NP;
    return (c[2] * NP + c[1]) * NP + c[0];
}
template <int DIM, int NP>
__device__ __forceinline__ int face_tangential(int d, const int c[3]) {
    if (DIM == 2) return c[1 - d];
    const int t0 = (d == 0) ? 1 : 0, t1 = (d == 2) ? 1 : 2;
    return c[t0] + NP * c[t1];
}

template <int NP, typename Real>
__device__ __forceinline__ void load_tables(const OpTables &T, Real *sT, int tid, int nthreads) {
    for (int q = tid; q < NP * NP; q += nthreads) {
        const int i = q / NP, l = q % NP;
        sT[q] = Real(T.D[i * NP + l]);
        sT[NP * NP + q] = Real(T.Dhat[i * NP + l]);
        sT[2 * NP * NP + q] = Real(T.Dhat2[i * NP + l]);
        sT[3 * NP * NP + q] = Real(T.Vinv[i * NP + l]);
    }
    for (int q = tid; q < NP; q += nthreads) {
        sT[4 * NP * NP + q] = Real(T.w[q]);
        sT[4 * NP * NP + NP + q] = Real(T.x[q]);
    }
}

// Node pairs of the flux-differencing phase, per direction: entry dir*NPD + p
// holds the element-local nodes (a, b), a < b along the line, of unique pair p
// (line-major, then pair-major) as a | b << 16.  Built once per CTA, so the
// pair loop does one shared load instead of decoding line and pair indices.
template <int DIM, int NP>
__device__ __forceinline__ void load_pair_table(uint32_t *sP, int tid, int nthreads) {
    constexpr int PPL = NP * (NP - 1) / 2, NPD = ipow(NP, DIM - 1) * PPL;
    for (int q = tid; q < DIM * NPD; q += nthreads) {
        const int dir = q / NPD, p = q - dir * NPD;
        const int ln = p / PPL, pp = p - ln * PPL;
        int pa, pb, base, stride;
        pair_decode<NP>(pp, pa, pb);
        line_base<DIM, NP>(dir, ln, base, stride);
        sP[q] = uint32_t(base + pa * stride) | (uint32_t(base + pb * stride) << 16);
    }
}

__device__ __forceinline__ void atomic_max_pos(unsigned long long *dst, double v) {
    // v >= 0 (or NaN): non-negative doubles order like their bit patterns.
    if (!(v >= 0.0)) v = __longlong_as_double(0x7ff0000000000000ll);   // NaN/negative -> +inf
    atomicMax(dst, (unsigned long long)__double_as_longlong(v));
}

// Block-wide max of per-thread values, one atomic per CTA.
template <int THREADS>
__device__ __forceinline__ void block_max_to(unsigned long long *dst, double v, double *sred) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sred[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = sred[0];
        for (int q = 1; q < (THREADS + 31) / 32; ++q) m = fmax(m, sred[q]);
        atomic_max_pos(dst, m);
    }
}

// Hoisted per-node primitive table in shared memory: H[k*ND + node].
// The FP32-bulk form also keeps dp = p - p_ref (slot DP).
template <int DIM>
struct HIdx {
    static constexpr int RHO = 0, RRHO = 1, V = 2, VSQ = 2 + DIM, BETA = 3 + DIM, RBETA = 4 + DIM,
                         LAM = 5 + DIM, K = 6 + DIM, DP = 6 + DIM;
};
template <int DIM, typename Real>
constexpr int hoisted_count() { return HIdx<DIM>::K + (sizeof(Real) == 4 ? 1 : 0); }
template <int DIM, int ND, typename Real>
__device__ __forceinline__ Prim<DIM, Real> load_prim(const Real *sH, int n) {
    using I = HIdx<DIM>;
    Prim<DIM, Real> q;
    q.rho = sH[I::RHO * ND + n];
    q.rrho = sH[I::RRHO * ND + n];
#pragma unroll
    for (int d = 0; d < DIM; ++d) q.v[d] = sH[(I::V + d) * ND + n];
    q.vsq = sH[I::VSQ * ND + n];
    q.beta = sH[I::BETA * ND + n];
    q.rbeta = sH[I::RBETA * ND + n];
    q.lam = sH[I::LAM * ND + n];
    if constexpr (sizeof(Real) == 4) q.dp = sH[I::DP * ND + n];
    return q;
}
template <int DIM, int ND, typename Real>
__device__ __forceinline__ void store_prim(Real *sH, int n, const Prim<DIM, double> &q, double pref) {
    using I = HIdx<DIM>;
    sH[I::RHO * ND + n] = Real(q.rho);
    sH[I::RRHO * ND + n] = Real(q.rrho);
#pragma unroll
    for (int d = 0; d < DIM; ++d) sH[(I::V + d) * ND + n] = Real(q.v[d]);
    sH[I::VSQ * ND + n] = Real(q.vsq);
    sH[I::BETA * ND + n] = Real(q.beta);
    sH[I::RBETA * ND + n] = Real(q.rbeta);
    sH[I::LAM * ND + n] = Real(q.lam);
    if constexpr (sizeof(Real) == 4) sH[I::DP * ND + n] = Real(q.dp - pref);
}
template <int DIM, int ND, typename Real>
__device__ __forceinline__ void store_prim_w(Real *sH, int n, const Prim<DIM, Real> &q) {
    using I = HIdx<DIM>;
    sH[I::RHO * ND + n] = q.rho;
    sH[I::RRHO * ND + n] = q.rrho;
#pragma unroll
    for (int d = 0; d < DIM; ++d) sH[(I::V + d) * ND + n] = q.v[d];
    sH[I::VSQ * ND + n] = q.vsq;
    sH[I::BETA * ND + n] = q.beta;
    sH[I::RBETA * ND + n] = q.rbeta;
    sH[I::LAM * ND + n] = q.lam;
    if constexpr (sizeof(Real) == 4) sH[I::DP * ND + n] = q.dp;
}
// Working-precision copy of primitives computed in FP64 (pressure relative
// to pref in the FP32-bulk form).
template <int DIM, typename Real>
__device__ __forceinline__ Prim<DIM, Real> cast_prim(const Prim<DIM, double> &q, double pref) {
    Prim<DIM, Real> r;
    r.rho = Real(q.rho);
    r.rrho = Real(q.rrho);
#pragma unroll
    for (int d = 0; d < DIM; ++d) r.v[d] = Real(q.v[d]);
    r.vsq = Real(q.vsq);
    r.beta = Real(q.beta);
    r.rbeta = Real(q.rbeta);
    r.lam = Real(q.lam);
    r.dp = sizeof(Real) == 4 ? Real(q.dp - pref) : Real(q.dp);
    return r;
}

constexpr int next_pow2(int v) { return v <= 1 ? 1 : 2 * next_pow2((v + 1) / 2); }

// Launch shape of the RHS kernel: warps per CTA and the minimum CTAs per SM the
// register allocation must allow (launch bounds).
#ifndef PRANDTL_NS_WARPS
#define PRANDTL_NS_WARPS 4
#endif
#ifndef PRANDTL_NS_MINB
#define PRANDTL_NS_MINB 3
#endif
#ifndef PRANDTL_EULER_WARPS
#define PRANDTL_EULER_WARPS 4
#endif
#ifndef PRANDTL_EULER_MINB
#define PRANDTL_EULER_MINB 5
#endif
#ifndef PRANDTL_NSVC_MINB
#define PRANDTL_NSVC_MINB 4
#endif
#ifndef PRANDTL_NSVC32_MINB
#define PRANDTL_NSVC32_MINB 4
#endif
#ifndef PRANDTL_NS32_MINB
#define PRANDTL_NS32_MINB 4
#endif
#ifndef PRANDTL_LINE_MAX_NP
#define PRANDTL_LINE_MAX_NP 5
#endif
#ifndef PRANDTL_EULER32_MINB
#define PRANDTL_EULER32_MINB 6
#endif
#ifndef PRANDTL_WIDE_MIN_ND
#define PRANDTL_WIDE_MIN_ND 125
#endif
#ifndef PRANDTL_LIFT64_MINB
#define PRANDTL_LIFT64_MINB 5
#endif

// Lane-group layout of the RHS kernel: one group of GS lanes owns one
// element.  GS = 32 (a warp), the next power of two >= Np^d for small
// elements (a warp then holds several elements), 64 (two warps) for large
// ones, or 128 for the FP32 Navier-Stokes 216-node elements.  Lane `li` of a
// group owns the nodes li, li+GS, ... and the pair / line / face / subcell
// items of the same stride.  Groups synchronise with __syncwarp, or with a
// named barrier when GS > 32.
//
// V selects the register budget (the batch autotuner times all of them): the
// launch bounds ask for MINB_BASE resident CTAs per SM (V = 0, also the
// one-shot kernels), one fewer (V = 1: more registers) or one more (V = 2:
// fewer registers, possibly spilling), always capped by what shared memory
// admits.  The group width is fixed per element size and form (measured:
// 64 lanes for >= 125 nodes, 128 for the FP32 Navier-Stokes 216-node form).
constexpr int NUM_VARIANTS = 3;
constexpr int CTX_RESERVE = 1280;   // bytes of per-item contexts reserved in every layout

template <int DIM, int NP, bool NS, typename Real, int V, bool VC>
struct RhsLayout {
    using S = Shape<DIM, NP>;
    static constexpr int ND = S::ND, NF = S::NF, NLINE = S::NLINE, PPL = S::PPL;
    static constexpr bool WIDE = ND >= PRANDTL_WIDE_MIN_ND;
    // FP32-bulk Navier-Stokes with contravariant viscous fluxes at Np = 6: 128
    // lanes, so that the 3 x 36 line tasks of the volume terms take one round
    static constexpr bool TASK128 = NS && VC && sizeof(Real) == 4 && ND >= 216;
    static constexpr int GS = TASK128 ? 128 : (WIDE ? 64 : (ND >= 32 ? 32 : next_pow2(ND)));
    static constexpr int EPW = GS >= 32 ? 1 : 32 / GS;  // elements per warp
    static constexpr int WPE = GS > 32 ? GS / 32 : 1;   // warps per element
    static constexpr int NPL = (ND + GS - 1) / GS;      // nodes per lane
    static constexpr int NPD = NLINE * PPL;             // pairs per direction
    static constexpr int NID = NLINE * (NP - 1);        // subcell interfaces per direction
    static constexpr int BUF = cmax(cmax(NPD, S::NFI), cmax(NID, (5 * ND + NF - 1) / NF)) * NF;
    static constexpr int K = hoisted_count<DIM, Real>();
    // per-element shared memory, in Real units: the hoisted primitives and the
    // work buffer (BODY, padded to 16 bytes), then (FP64) the element's
    // neighbour-table entries (2 DIM int4), and the whole a multiple of 4 words
    // so every element's area stays 16-byte aligned
    // Navier-Stokes viscous-flux buffer [DIM][VROWS][ND]: the line tasks keep
    // all NF rows (row 0 carries the direction's inviscid total), the pair form
    // only rows 1..NF-1 (the viscous mass flux is zero); the smaller footprint
    // leaves more of the SM's L1 to the face phase's loads (C2 FP64 RHS
    // 0.362 -> 0.335 ms)
    static constexpr bool LINE_FORM = NS && sizeof(Real) == 4 && (NP <= PRANDTL_LINE_MAX_NP || TASK128);
    static constexpr int VROWS = LINE_FORM ? NF : NF - 1;
    static constexpr int VOFF = NF - VROWS;             // buffer row of field f: f - VOFF
    static constexpr int BODY = (K * ND + cmax(BUF, NS ? DIM * VROWS * ND : 0) + 3) / 4 * 4;
    static constexpr int NBR_REALS = sizeof(Real) == 8 ? 2 * DIM * 16 / (int)sizeof(Real) : 0;
    static constexpr int PER_ELEM = (BODY + NBR_REALS + 3) / 4 * 4;
    static constexpr bool F64 = sizeof(Real) == 8;
    // (the Navier-Stokes form with contravariant viscous fluxes needs fewer
    // registers; in FP32 the 216-node elements of 128 lanes fit 4 CTAs of
    // 128 registers a thread; FP64 large elements are capped by shared
    // memory anyway)
    static constexpr int MINB_CFG = NS ? (F64 ? (VC ? PRANDTL_NSVC_MINB : PRANDTL_NS_MINB)
                                              : (VC ? (TASK128 ? 4 : PRANDTL_NSVC32_MINB) : PRANDTL_NS32_MINB))
                                       : (F64 ? PRANDTL_EULER_MINB : PRANDTL_EULER32_MINB);
    static constexpr int WARPS_CFG = NS ? PRANDTL_NS_WARPS : PRANDTL_EULER_WARPS;
    // warps per CTA: the configured count, reduced so the CTA's elements fit the
    // 227 KB shared-memory limit (whole elements, whole warps)
    static constexpr int SMEM_MAX = 227 * 1024;
    static constexpr int TAB_BYTES = (S::TAB * (int)sizeof(Real) + 15) / 16 * 16;
    static constexpr int PAIR_BYTES = (DIM * NPD * 4 + 15) / 16 * 16;   // load_pair_table
    static constexpr int FIXED_BYTES = TAB_BYTES + PAIR_BYTES + CTX_RESERVE;
    static constexpr int FIT_ELEMS = (SMEM_MAX - FIXED_BYTES) / (PER_ELEM * (int)sizeof(Real));
    static constexpr int FIT_WARPS = GS > 32 ? FIT_ELEMS * WPE : FIT_ELEMS / EPW;
    static constexpr int WARPS_FIT = FIT_WARPS < WARPS_CFG ? FIT_WARPS : WARPS_CFG;
    static constexpr int WARPS = cmax(WPE, WARPS_FIT / WPE * WPE);
    static constexpr int THREADS = WARPS * 32;
    static constexpr int EPB = THREADS / GS;            // elements per CTA
    // batch work items: one warp (EPW elements) or one two-warp group (1 element)
    static constexpr int ITEM_THREADS = GS > 32 ? GS : 32;
    static constexpr int ITEM_ELEMS = ITEM_THREADS / GS;
    static constexpr int ITEMS_PER_CTA = THREADS / ITEM_THREADS;
    static_assert(GS <= 32 || EPB < 16, "named barriers 1..15 identify the lane groups");
    static_assert(BATCH_CHUNK % ITEM_ELEMS == 0, "items must not straddle padded solve ranges");
    // resident CTAs the register budget is sized for: the variant's request,
    // capped by what shared memory admits (228 KB per SM, 1 KB reserved per CTA)
    static constexpr int CTA_SMEM = FIXED_BYTES + EPB * PER_ELEM * (int)sizeof(Real);
    static constexpr int SMEM_BLOCKS = cmax(1, (228 * 1024) / (CTA_SMEM + 1024));
    static constexpr int MINB_REQ = V == 1 ? cmax(1, MINB_CFG - 1) : (V == 2 ? MINB_CFG + 1 : MINB_CFG);
    static constexpr int MIN_BLOCKS = MINB_REQ < SMEM_BLOCKS ? MINB_REQ : SMEM_BLOCKS;
    // volume terms by line tasks (Navier-Stokes: the viscous-flux buffer holds
    // the per-direction results) or by pairs and node-wise sums.  Line tasks
    // were measured faster in the FP32-bulk form up to Np = 4 (3-4 %), at
    // Np = 5 on 64-lane groups (12 %, once the two-point fluxes of two partners
    // share paired FP32 instructions; 128 lanes: no gain) and with the 128-lane
    // groups at Np = 6 (17 %); slower in FP64.
    static constexpr bool LINE = NS && !F64 && (NP <= PRANDTL_LINE_MAX_NP || TASK128);
    static_assert(LINE == LINE_FORM, "viscous-buffer rows follow the volume form");
};

// Synchronise the GS lanes of lane group `gid` (its index within the CTA).
// A group narrower than a warp synchronises its own lanes only: groups of one
// warp take different paths (one element's subcell FV phase runs while its
// warp-mate's is skipped, and an inactive group returns early), so a
// full-warp mask would pair barriers of different groups and, once a group
// has exited, no longer order the other group's shared-memory accesses.
template <int GS>
__device__ __forceinline__ void group_sync(int gid) {
    if constexpr (GS < 32) {
        const unsigned base = (threadIdx.x & 31u) & ~unsigned(GS - 1);
        __syncwarp(((1u << GS) - 1u) << base);
    } else if constexpr (GS == 32) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(1 + gid), "n"(GS) : "memory");
    }
}

// Instance-local operands of one element evaluation (the one-shot kernels build
// it from their arguments, the batch kernels from the solve's table entry).
struct ElemIO {
    const double *u;            // stage input state (byNODES, field stride Ndof)
    void *grad;                 // NS primitive gradients [DIM][NF][Ndof], double or float
    double *dudt;               // EPI_STORE output
    double *u_out;              // RK output state
    double *du;                 // LSRK register
    const double *x0;           // SSP step-start state
    double *alpha;              // [E] blending coefficient (may be null)
    unsigned long long *lambda; // max |V|+c as ordered bits (may be null)
    const double *geo;          // [E][DIM*DIM + 1]
    const int4 *nbr;            // [E][2*DIM]
    const double *fnor;         // [F][DIM]
    long long Ndof;
    int E;
    int mode;
    double dt, rkA, rkB;
    const BcDev *bcs;           // boundary conditions (boundary faces)
    // axisymmetric (z, r) form, 2D Euler only; null otherwise
    const double *u_rk;         // the RK state r U (u is the U recovered from it)
    const double *rad;          // [Ndof] node radius r
    const unsigned char *axis;  // [Ndof] axis nodes
    unsigned int *health;       // RK modes: state-check bits (PRANDTL_HEALTH_*), may be null
    // non-affine elements (one-shot FP64 kernels; MeshDev), null otherwise
    const double *ngeo, *fnn, *snor;
};
// Per-warp (rhs) or per-CTA (lift) copy of the current solve's constants.
struct __align__(16) WarpCtx {
    PhysParams P;
    ElemIO io;
};
static_assert(4 * sizeof(WarpCtx) <= CTX_RESERVE, "context reserve too small");

__device__ __forceinline__ ElemIO io_from_args(const MeshDev &m, const RhsArgs &a) {
    ElemIO io;
    io.u = a.u;
    io.grad = a.grad32 ? (void *)a.grad32 : (void *)a.grad;
    io.dudt = a.dudt;
    io.u_out = a.u_out;
    io.du = a.du;
    io.x0 = a.x0;
    io.alpha = a.alpha;
    io.lambda = a.lambda;
    io.geo = m.geo;
    io.nbr = m.nbr;
    io.fnor = m.fnor;
    io.Ndof = m.Ndof;
    io.E = m.E;
    io.mode = a.mode;
    io.dt = a.dt;
    io.rkA = a.rkA;
    io.rkB = a.rkB;
    io.bcs = m.bcs;
    io.u_rk = a.u_rk;
    io.rad = m.rad;
    io.axis = m.axis;
    io.health = a.health;
    io.ngeo = m.ngeo;
    io.fnn = m.fnn;
    io.snor = m.snor;
    return io;
}

// Stage operands of solve I in a batch: the RK buffers the stage reads and
// writes follow the scheme, the stage index and (LSRK) the solve's ping-pong
// parity at the start of its current step.
__device__ __forceinline__ ElemIO io_from_batch(const BatchInst &I, BatchInst *Im, const BatchStage &st) {
    ElemIO io;
    io.grad = I.grad;
    io.dudt = nullptr;
    io.du = nullptr;
    io.x0 = nullptr;
    io.alpha = I.alpha;
    io.lambda = &Im->lambda;
    io.geo = I.geo;
    io.nbr = I.nbr;
    io.fnor = I.fnor;
    io.Ndof = I.Ndof;
    io.E = I.E;
    io.dt = I.dt;
    io.rkA = st.rkA;
    io.rkB = st.rkB;
    io.bcs = I.bcs;
    if (st.scheme == BATCH_LSRK45) {
        const int in = I.cur ^ (st.stage & 1);
        io.u = I.u[in];
        io.u_out = I.u[in ^ 1];
        io.du = I.u[2];
        io.mode = EPI_LSRK;
    } else {   // SSP-RK3 (Shu-Osher): x -> y1 -> y2 -> x
        io.u = I.u[st.stage];
        io.u_out = I.u[st.stage == 2 ? 0 : st.stage + 1];
        io.x0 = I.u[0];
        io.mode = st.stage == 0 ? EPI_SSP1 : (st.stage == 1 ? EPI_SSP2 : EPI_SSP3);
    }
    io.u_rk = nullptr;
    io.rad = nullptr;
    io.axis = nullptr;
    io.health = &Im->health;
    io.ngeo = io.fnn = io.snor = nullptr;
    return io;
}

// Locate the solve owning padded class element `first`: the last slot s with
// prefix[s] <= first (prefix holds each solve's element range rounded up to
// BATCH_CHUNK).
__device__ __forceinline__ int batch_slot(const int *prefix, int n, int first) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= first) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ bool bc_is_wall(int type) {
    return type == BC_SLIP_WALL || type == BC_NOSLIP_ADIABATIC || type == BC_NOSLIP_ISOTHERMAL;
}

// Outer state s2 of the conditions whose flux is the surface flux of (s1, s2)
// (ComputeOuterInviscidState of src/Integrators/BoundaryConditions/, constant
// data), in FP64.  s1 takes the reference-mode aliasing the integrator applies
// to its inner trace.  nn = |nor|.  Not for the wall types.
template <int DIM>
__device__ __forceinline__ void bc_outer_state(const BcDev &bc, double *s1, const double *nor, double nn,
                                               const PhysParams &P, double *s2) {
    constexpr int NF = DIM + 2;
    const double gamma = P.gamma, gm1 = P.gammaM1, gm1i = P.gammaM1Inverse;
    if (bc.type == BC_STATE) {   // SpecifiedStateBdrFaceIntegrator.cpp:24-36
#pragma unroll
        for (int f = 0; f < NF; ++f) s2[f] = bc.state[f];
    } else if (bc.type == BC_SYMMETRY || bc.type == BC_AXIS) {   // SymmetryBdrFaceIntegrator.cpp:11-32 (|nor| > 0)
        const double rn = 1.0 / nn;
        double mn = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) mn += s1[1 + d] * (nor[d] * rn);
#pragma unroll
        for (int f = 0; f < NF; ++f) s2[f] = s1[f];
#pragma unroll
        for (int d = 0; d < DIM; ++d) s2[1 + d] += -2.0 * mn * (nor[d] * rn);
    } else if (bc.type == BC_PRESSURE_OUTFLOW) {   // SubsonicOutflowPBdrFaceIntegrator.cpp:17-29
        // quirks == 0 (Q9): the reference's velocity vector wraps the inner
        // trace, so both traces carry velocity in their momentum slots
        const double r = 1.0 / s1[0];
        double vel[DIM], vv = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            vel[d] = s1[1 + d] * r;
            if (P.quirks == 0) s1[1 + d] = vel[d];
            vv += vel[d] * vel[d];
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) s2[f] = s1[f];
        s2[NF - 1] = bc.p * gm1i + 0.5 * s1[0] * vv;
    } else if (bc.type == BC_RIEMANN) {   // RiemannInvariantBdrFaceIntegrator.cpp:45-116
        const double rn = 1.0 / nn, r1 = 1.0 / s1[0], gi = 1.0 / gamma;
        const double rho_o = bc.state[0], p_o = bc.state[NF - 1];
        double un[DIM], vi[DIM], vn_i = 0.0, vn_o = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            un[d] = nor[d] * rn;
            vi[d] = s1[1 + d] * r1;
            vn_i += vi[d] * un[d];
            vn_o += bc.state[1 + d] * un[d];
        }
        // quirks == 0 (Q10): the inner velocity wraps the trace and the pressure
        // helper divides it once more, so the trace and vi end as m / rho^2
        double vv = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            if (P.quirks == 0) {
                vi[d] *= r1;
                s1[1 + d] = vi[d];
            }
            vv += vi[d] * vi[d];
        }
        const double p_i = gm1 * (s1[NF - 1] - 0.5 * s1[0] * vv);
        const double a_o = sqrt(gamma * p_o / rho_o), a_i = sqrt(gamma * p_i / s1[0]);
        const bool sup = fabs(vn_o) >= a_o;
        const double r_minus = (sup && vn_i >= 0.0) ? vn_i - 2.0 * a_i * gm1i : vn_o - 2.0 * a_o * gm1i;
        const double r_plus = (sup && vn_i < 0.0) ? vn_o + 2.0 * a_o * gm1i : vn_i + 2.0 * a_i * gm1i;
        const double vn_b = 0.5 * (r_plus + r_minus), a_b = 0.25 * gm1 * (r_plus - r_minus);
        s2[0] = vn_i < 0.0 ? pow(a_b * a_b * gi * rho_o / p_o, gm1i) * rho_o
                           : pow(a_b * a_b * gi * s1[0] / p_i, gm1i) * s1[0];
        double ke = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            s2[1 + d] = vn_i >= 0.0 ? s2[0] * (vi[d] + (vn_b - vn_i) * un[d])
                                    : s2[0] * (bc.state[1 + d] + (vn_b - vn_o) * un[d]);
            ke += s2[1 + d] * s2[1 + d];
        }
        s2[NF - 1] = ke * (0.5 / s2[0]) + a_b * a_b * s2[0] * gi * gm1i;
    } else if (bc.type == BC_INFLOW_RV) {   // SubsonicInflowRVBdrFaceIntegrator.cpp:19-49
        const double r = bc.state[0];
        double dke = 0.0, uu = 0.0;
        s2[0] = r;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            s2[1 + d] = r * bc.state[1 + d];
            dke -= s1[1 + d] * s1[1 + d];
            uu += bc.state[1 + d] * bc.state[1 + d];
        }
        dke *= 0.5 / s1[0];
        dke += 0.5 * uu * r;
        s2[NF - 1] = s1[NF - 1] + dke;
    } else if (bc.type == BC_INFLOW_PTTT) {   // SubsonicInflowPtTtAngBdrFaceIntegrator.cpp:55-79
        // quirks == 0: the pressure helper leaves velocity in the trace's momentum slots
        const double r1 = 1.0 / s1[0];
        double vv = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const double v = s1[1 + d] * r1;
            if (P.quirks == 0) s1[1 + d] = v;
            vv += v * v;
        }
        const double p = gm1 * (s1[NF - 1] - 0.5 * s1[0] * vv);
        double v_sq = 2.0 * bc.cp * bc.Tt * (1.0 - pow(p / bc.pt, gm1 / gamma));
        v_sq = fmax(0.0, v_sq);
        s2[0] = gamma * gm1i * p / (bc.cp * bc.Tt - 0.5 * v_sq);
        const double sv = sqrt(v_sq);
#pragma unroll
        for (int d = 0; d < DIM; ++d) s2[1 + d] = s2[0] * sv * bc.vc[d];
        s2[NF - 1] = p * gm1i + 0.5 * s2[0] * v_sq;
    } else {   // BC_OUTFLOW, SupersonicOutflowBdrFaceIntegrator.cpp:11-14
#pragma unroll
        for (int f = 0; f < NF; ++f) s2[f] = s1[f];
    }
}

// Boundary-face flux of the inner trace s_in (FP64 conserved state) along the
// element's outward scaled normal nor: the reference's boundary integrators
// with constant states (src/Integrators/BoundaryConditions/; the element is
// Elem1 and receives -flux / (w0 J), BdrFaceIntegrator.cpp:61-138).  Inviscid.
// The outer state is formed in FP64; the Chandrashekar surface flux runs in
// the working precision like the interior faces.
template <int DIM, typename Real>
__device__ __forceinline__ void boundary_flux(const BcDev &bc, const double *s_in, const double *nor,
                                              const PhysParams &P, double pref, Real *flux) {
    constexpr int NF = DIM + 2;
    const double gamma = P.gamma, gm1 = P.gammaM1, gm1i = P.gammaM1Inverse;
    double s1[NF], s2[NF], nn = 0.0;
#pragma unroll
    for (int f = 0; f < NF; ++f) s1[f] = s_in[f];
#pragma unroll
    for (int d = 0; d < DIM; ++d) nn += nor[d] * nor[d];
    nn = sqrt(nn);
    if (bc_is_wall(bc.type)) {   // SlipWallBdrFaceIntegrator.cpp:16-59 (the no-slip walls inherit it)
        const double rn = 1.0 / nn, gp1 = 1.0 + gamma, gp1i = 1.0 / gp1;
        const double rho = s1[0];
        double mn = 0.0, vv = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            mn += s1[1 + d] * (nor[d] * rn);
            const double v = s1[1 + d] / rho;
            vv += v * v;
        }
        const double un = mn / rho;   // normal velocity of the rotated state
        const double p = gm1 * (s1[NF - 1] - 0.5 * rho * vv);
        const double an = sqrt(gamma * p / rho);
        double p_star;
        if (un > 0.0)
            p_star = p + 0.25 * un * gp1 * rho * (un + sqrt(un * un + 8.0 * gp1i / rho * p * (gm1 * gp1i + 1.0)));
        else
            p_star = p * pow(fmax(1.0 + 0.5 * gm1 * un / an, 0.0001), 2.0 * gamma * gm1i);
        // the FP32-bulk form carries p - pref in every momentum flux (pref = 0 in FP64)
        flux[0] = 0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) flux[1 + d] = Real((p_star - pref) * nor[d]);
        flux[NF - 1] = 0;
        return;
    }
    if ((bc.type == BC_SYMMETRY || bc.type == BC_AXIS) && nn == 0.0) {
#pragma unroll
        for (int f = 0; f < NF; ++f) flux[f] = 0;
        return;
    }
    bc_outer_state<DIM>(bc, s1, nor, nn, P, s2);
    Real m1[NF], m2[NF], nr[DIM];
#pragma unroll
    for (int f = 0; f < NF; ++f) { m1[f] = Real(s1[f]); m2[f] = Real(s2[f]); }
#pragma unroll
    for (int d = 0; d < DIM; ++d) nr[d] = Real(nor[d]);
    face_flux<DIM, Real>(m1, cast_prim<DIM, Real>(primitives<DIM, double>(s1, gamma, gm1), pref), m2,
                         cast_prim<DIM, Real>(primitives<DIM, double>(s2, gamma, gm1), pref), nr, Real(gm1i),
                         P.quirks == 0, P.dissipation != 0, flux);
}

// ------------------------------------------------------------------- RHS
// Real is the working precision of the O(Np^{d+1}) work (two-point fluxes,
// flux differencing, surface fluxes, gradients): double for the plain FP64
// path, float for the FP32-bulk form.  Per-node primitives are always formed
// in FP64 from the FP64 state, and the RK stage update is FP64.
template <int DIM, int NP, bool NS, bool VC, typename Real, typename LY, bool CURV = false>
__device__ __forceinline__ void rhs_element(const ElemIO &a, const PhysParams &P, int e, bool active,
                                            const Real *sT, const uint32_t *sPair, Real *sH, int li, int lane,
                                            int gid) {
    static_assert(!CURV || sizeof(Real) == 8 || !NS, "non-affine elements: FP64, or FP32-bulk Euler");
    using S = Shape<DIM, NP>;
    constexpr int ND = S::ND, NF = S::NF, PPL = S::PPL;
    constexpr int NFN = S::NFN, NFI = S::NFI, GS = LY::GS, NPL = LY::NPL;
    constexpr int NPD = LY::NPD, NID = LY::NID;
    const Real *sDh = sT + NP * NP, *sDh2 = sT + 2 * NP * NP, *sVinv = sT + 3 * NP * NP;
    const Real *sW = sT + 4 * NP * NP;
    Real *sF = sH + LY::K * ND;                       // pairs / subcell / face items / modes
    Real *sV = sF;                                    // NS: contravariant viscous fluxes [DIM][NF][ND]
                                                      // (consumed before the pair phase reuses it)
    const Real *grad = nullptr;
    if constexpr (NS) grad = reinterpret_cast<const Real *>(a.grad);

    const long long Ndof = a.Ndof;
    const double gamma = P.gamma, gm1 = P.gammaM1;
    const Real gm1i = Real(P.gammaM1Inverse);
    const double *geo = a.geo + (long long)e * (DIM * DIM + 1);
    Real adj[DIM][DIM];
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int c2 = 0; c2 < DIM; ++c2) adj[r][c2] = Real(__ldg(geo + r * DIM + c2));
    const double J = __ldg(geo + DIM * DIM);
    const Real mJ = Real(1.0 / J);
    // non-affine elements: the transformation at node n, component c = r DIM + q
    // of adj(J) or c = DIM^2 for det J (Tr.SetIntPoint at the node,
    // DGSEMIntegrator.cpp:254-267); the affine path uses adj / J above
    auto ngeo = [&](int n, int c) -> double { return __ldg(a.ngeo + (long long)c * Ndof + (long long)e * ND + n); };

    // FP32-bulk form: reference pressure of the element (node 0), FP64.  The
    // shift cancels only where the volume operator annihilates a constant flux;
    // the reference's 3D Navier-Stokes volume term (quirks == 0) stores the eta
    // flux in the symmetric zeta slot (DGSEMIntegrator.cpp:702), so there pref = 0.
    // axisymmetric (z, r) form (DGSEMIntegrator.cpp AXISYMMETRIC parts): fluxes
    // weighted by r, a pressure source; r-weighting also breaks the constant-
    // pressure cancellation, so the FP32 shift is off there
    const double *rad = (DIM == 2 && !NS) ? a.rad : nullptr;
    double pref = 0.0;
    if constexpr (!LY::F64) {
        if (!(DIM == 3 && NS && P.quirks == 0) && !rad) {
            double s0[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) s0[f] = __ldg(a.u + f * Ndof + (long long)e * ND);
            pref = primitives<DIM, double>(s0, gamma, gm1).dp;
        }
    }

    // ---- own nodes: hoisted primitives (formed in FP64); largest |V|+c.  FP64:
    //      the element's neighbour-table entries are loaded with the own state
    //      and kept in shared memory, so the face phase's neighbour-trace loads
    //      do not wait on a table load first (C2 RHS -0.6 %).  FP32: the face
    //      phase loads them itself; holding the entry across the hoisting
    //      raised the N=4 kernels' spills (168-register budget: 12 -> 144 B)
    //      and their time by 11-40 %.
    constexpr bool NBR_SMEM = LY::F64;
    int4 *sNbr = reinterpret_cast<int4 *>(sH + LY::BODY);
    double lam = 0.0;
    {
        const int4 tn = NBR_SMEM && li < 2 * DIM ? __ldg(a.nbr + (long long)e * (2 * DIM) + li)
                                                 : make_int4(0, 0, 0, 0);
        double st[NPL][NF];   // every load in flight before the first use
#pragma unroll
        for (int k = 0; k < NPL; ++k) {
            const int n = li + k * GS;
#pragma unroll
            for (int f = 0; f < NF; ++f) st[k][f] = n < ND ? __ldg(a.u + f * Ndof + (long long)e * ND + n) : 1.0;
        }
#pragma unroll
        for (int k = 0; k < NPL; ++k) {
            const int n = li + k * GS;
            if (n < ND) {
                if constexpr (!LY::F64) {
                    const Prim<DIM, float> q = primitives_mixed<DIM>(st[k], gamma, gm1, pref);
                    store_prim_w<DIM, ND, Real>(sH, n, q);
                    lam = fmax(lam, double(q.lam));
                } else {
                    const Prim<DIM, double> q = primitives<DIM, double>(st[k], gamma, gm1);
                    store_prim<DIM, ND, Real>(sH, n, q, pref);
                    lam = fmax(lam, q.lam);
                }
            }
        }
        if (NBR_SMEM && li < 2 * DIM) sNbr[li] = tn;
    }
    if (a.lambda) {
        double v = active ? lam : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) atomic_max_pos(a.lambda, v);
    }
    group_sync<GS>(gid);

    // ---- blending coefficient (PerssonPeraireIndicator.cpp:21-58, DGSEMOperator.cpp:60-80)
    Real alpha = 0;
    if (P.blending) {
        Real *b0 = sF, *b1 = sF + ND;
#pragma unroll 1
        for (int k = 0; k < NPL; ++k) {
            const int n = li + k * GS;
            if (n < ND) {
                // rho * ComputePressure(state) with v = m * (1/rho)
                const Prim<DIM, Real> q = load_prim<DIM, ND, Real>(sH, n);
                b0[n] = q.rho * (Real(0.5) * q.rbeta * q.rho);
            }
        }
        group_sync<GS>(gid);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {   // modes = V^-1 (rho p), one direction per pass
            const Real *in = (d & 1) ? b1 : b0;
            Real *out = (d & 1) ? b0 : b1;
#pragma unroll 1
            for (int k = 0; k < NPL; ++k) {
                const int n = li + k * GS;
                if (n < ND) {
                    int c[3];
                    node_coords<NP>(n, c);
                    int base, stride;
                    line_base<DIM, NP>(d, line_index<DIM, NP>(d, c), base, stride);
                    Real s = 0;
#pragma unroll
                    for (int l = 0; l < NP; ++l) s += sVinv[c[d] * NP + l] * in[base + l * stride];
                    out[n] = s;
                }
            }
            group_sync<GS>(gid);
        }
        double e0 = 0, e1 = 0, e2 = 0;
#pragma unroll 1
        for (int k = 0; k < NPL; ++k) {
            const int n = li + k * GS;
            if (n < ND) {
                int c[3];
                node_coords<NP>(n, c);
                const double md = double(((DIM & 1) ? b1 : b0)[n]);
                int mx = c[0];
#pragma unroll
                for (int d = 1; d < DIM; ++d) mx = max(mx, c[d]);
                e0 += md * md;
                if (mx <= NP - 2) e1 += md * md;
                if (mx <= NP - 3) e2 += md * md;
            }
        }
        for (int o = (GS < 32 ? GS : 32) / 2; o > 0; o >>= 1) {
            e0 += __shfl_xor_sync(0xffffffffu, e0, o);
            e1 += __shfl_xor_sync(0xffffffffu, e1, o);
            e2 += __shfl_xor_sync(0xffffffffu, e2, o);
        }
        if constexpr (GS > 32) {
            // several warps per element: combine the warps' sums through
            // shared memory past the two mode buffers (8-byte aligned slots)
            double *xch = reinterpret_cast<double *>(sH + ((LY::K * ND + 2 * ND + 1) & ~1));
            if ((li & 31) == 0) {
                xch[3 * (li >> 5)] = e0;
                xch[3 * (li >> 5) + 1] = e1;
                xch[3 * (li >> 5) + 2] = e2;
            }
            group_sync<GS>(gid);
            e0 = xch[0];
            e1 = xch[1];
            e2 = xch[2];
#pragma unroll
            for (int w = 1; w < GS / 32; ++w) {
                e0 += xch[3 * w];
                e1 += xch[3 * w + 1];
                e2 += xch[3 * w + 2];
            }
        }
        double eta = 1.0 - e1 / e0;
        eta = fmax(eta, 1.0 - e2 / e1);
        const double thr = P.modal_threshold;
        double al = 1.0 / (1.0 + exp(-9.21024 * (eta - thr) / thr));
        if (al < P.alpha_min) al = 0.0;
        else if (al > 1.0 - P.alpha_min) al = 1.0;
        al = fmin(al, P.alpha_max);
        alpha = Real(al);
        if (li == 0 && a.alpha && active) a.alpha[e] = al;
        group_sync<GS>(gid);
    }

    Real dUi[NPL][NF], dUv[NPL][NF];
#pragma unroll
    for (int k = 0; k < NPL; ++k)
#pragma unroll
        for (int f = 0; f < NF; ++f) { dUi[k][f] = 0; dUv[k][f] = 0; }

    // ---- NS: contravariant viscous flux of every own node (flux_mat = adj * Fv^T, :632)
    if constexpr (NS && VC) {
        // formed by the lifting: rows f = 1..NF-1 of adj * Fv^T (the mass row is zero);
        // each lane's loads are all issued before the stores
        Real vrow[NPL][DIM][NF - 1];
#pragma unroll
        for (int k = 0; k < NPL; ++k) {
            const int n = li + k * GS;
#pragma unroll
            for (int r = 0; r < DIM; ++r)
#pragma unroll
                for (int f = 1; f < NF; ++f)
                    vrow[k][r][f - 1] = n < ND ? __ldg(grad + (r * (NF - 1) + f - 1) * Ndof + (long long)e * ND + n) : Real(0);
        }
#pragma unroll
        for (int k = 0; k < NPL; ++k) {
            const int n = li + k * GS;
            if (n < ND) {
#pragma unroll
                for (int r = 0; r < DIM; ++r)
#pragma unroll
                    for (int f = 1; f < NF; ++f) sV[(r * LY::VROWS + f - LY::VOFF) * ND + n] = vrow[k][r][f - 1];
            }
        }
    } else if constexpr (NS) {
#pragma unroll 1
        for (int k = 0; k < NPL; ++k) {
            const int n = li + k * GS;
            if (n < ND) {
                Real dq[DIM][NF];
#pragma unroll
                for (int d = 0; d < DIM; ++d)
#pragma unroll
                    for (int f = 0; f < NF; ++f)
                        dq[d][f] = __ldg(grad + (d * NF + f) * Ndof + (long long)e * ND + n);
                // Q1 (DGSEMIntegrator.cpp:620): the reference evaluates the volume
                // viscous flux with the state of node Np^d-1 (stale member id1).
                const int src = (P.quirks == 0) ? ND - 1 : n;
                const Prim<DIM, Real> q = load_prim<DIM, ND, Real>(sH, src);
                Real Vc[DIM][NF], an[DIM][DIM];   // adj(J) at node n (:620-633)
#pragma unroll
                for (int r = 0; r < DIM; ++r)
#pragma unroll
                    for (int c2 = 0; c2 < DIM; ++c2) an[r][c2] = CURV ? Real(ngeo(n, r * DIM + c2)) : adj[r][c2];
#pragma unroll
                for (int r = 0; r < DIM; ++r)
#pragma unroll
                    for (int f = 0; f < NF; ++f) Vc[r][f] = 0;
                viscous_flux<DIM, Real>(q.rho, q.rrho, q.v, Real(0.5) * q.rbeta * q.rho, dq, P,
                                        [&](int f, int cc, Real val) {
#pragma unroll
                                            for (int r = 0; r < DIM; ++r) Vc[r][f] += an[r][cc] * val;
                                        });
#pragma unroll
                for (int r = 0; r < DIM; ++r)
#pragma unroll
                    for (int f = LY::VOFF; f < NF; ++f) sV[(r * LY::VROWS + f - LY::VOFF) * ND + n] = Vc[r][f];
            }
        }
    }
    Real acc[NPL][NF];
    if constexpr (LY::LINE) {
        // ---- line tasks (DGSEMIntegrator.cpp:601-750): one lane per (direction,
        //      line) evaluates the line's Np(Np-1)/2 two-point fluxes once and
        //      accumulates both nodes' Dhat2 terms in registers, partners in
        //      ascending order as in the node-wise sum; adds the line's Dhat sums
        //      of the contravariant viscous fluxes and writes the direction's
        //      total over the line's own slots of that buffer (no other task
        //      reads them).  Q2 (quirks == 0, 3D): a zeta-line node's partners
        //      below it contribute the eta flux G(l) of DGSEMIntegrator.cpp:702.
        group_sync<GS>(gid);
        const Real blend = P.blending ? Real(1) - alpha : Real(1);
        for (int t = li; t < DIM * S::NLINE; t += GS) {
            const int dir = t / S::NLINE, ln = t - dir * S::NLINE;
            int base, stride;
            line_base<DIM, NP>(dir, ln, base, stride);
            Real mt[DIM], mg[DIM];
#pragma unroll
            for (int q = 0; q < DIM; ++q) {
                mt[q] = dir == 0 ? adj[0][q] : (dir == 1 ? adj[1][q] : adj[DIM - 1][q]);
                mg[q] = adj[1][q];
            }
            const bool useG = DIM == 3 && P.quirks == 0 && dir == 2;
            const bool gzero = ln / NP == NP - 1;   // zeta line at j = Np-1: G = 0
            Real al[NP][NF];
#pragma unroll
            for (int i = 0; i < NP; ++i)
#pragma unroll
                for (int f = 0; f < NF; ++f) al[i][f] = 0;
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                const Prim<DIM, Real> qi = load_prim<DIM, ND, Real>(sH, base + i * stride);
                Real G[NF];
#pragma unroll
                for (int f = 0; f < NF; ++f) G[f] = 0;
                if (i < NP - 1 && useG && !gzero)
                    volume_flux<DIM, Real>(qi, load_prim<DIM, ND, Real>(sH, ln % NP + (NP - 1) * NP + i * NP * NP),
                                           mg, gm1i, G);
                // FP32: partners l, l+1 on packed lanes (volume_flux2)
                constexpr int LSTEP = LY::F64 ? 1 : 2;
#pragma unroll
                for (int l = i + 1; l < NP; l += LSTEP) {
                    if constexpr (!LY::F64) {
                        if (l + 1 < NP) {
                            Real F[NF], F1[NF];
                            volume_flux2<DIM>(qi, load_prim<DIM, ND, Real>(sH, base + l * stride), qi,
                                              load_prim<DIM, ND, Real>(sH, base + (l + 1) * stride), mt, gm1i, F, F1);
                            const Real dil = sDh2[i * NP + l], dli = sDh2[l * NP + i];
                            const Real dil1 = sDh2[i * NP + l + 1], dl1i = sDh2[(l + 1) * NP + i];
#pragma unroll
                            for (int f = 0; f < NF; ++f) {
                                al[i][f] += dil * F[f];
                                al[l][f] += dli * (useG ? G[f] : F[f]);
                            }
#pragma unroll
                            for (int f = 0; f < NF; ++f) {
                                al[i][f] += dil1 * F1[f];
                                al[l + 1][f] += dl1i * (useG ? G[f] : F1[f]);
                            }
                            continue;
                        }
                    }
                    Real F[NF];
                    volume_flux<DIM, Real>(qi, load_prim<DIM, ND, Real>(sH, base + l * stride), mt, gm1i, F);
                    const Real dil = sDh2[i * NP + l], dli = sDh2[l * NP + i];
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        al[i][f] += dil * F[f];
                        al[l][f] += dli * (useG ? G[f] : F[f]);
                    }
                }
            }
            static_assert(LY::VROWS == NF, "line tasks use every row of the viscous buffer");
            Real vv[NP][NF - 1];
#pragma unroll
            for (int l = 0; l < NP; ++l)
#pragma unroll
                for (int f = 1; f < NF; ++f) vv[l][f - 1] = sV[(dir * NF + f) * ND + base + l * stride];
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                Real *out = sV + dir * NF * ND + base + i * stride;
                out[0] = -blend * al[i][0];
#pragma unroll
                for (int f = 1; f < NF; ++f) {
                    Real sv = 0;
#pragma unroll
                    for (int l = 0; l < NP; ++l) sv += vv[l][f - 1] * sDh[i * NP + l];
                    out[f * ND] = sv - blend * al[i][f];
                }
            }
        }
        group_sync<GS>(gid);
#pragma unroll
        for (int k = 0; k < NPL; ++k) {
            const int n = li + k * GS;
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                Real v = 0;
                if (n < ND) {
#pragma unroll
                    for (int d = 0; d < DIM; ++d) v += sV[(d * NF + f) * ND + n];
                }
                acc[k][f] = v * mJ;
            }
        }
        group_sync<GS>(gid);   // later phases overwrite the buffer
    } else {
        if constexpr (NS) {
            group_sync<GS>(gid);
            // sum_l Dhat(i,l) Fv_l along each direction (:710-738); the mass row is zero
#pragma unroll
            for (int k = 0; k < NPL; ++k) {
                const int n = li + k * GS;
                if (n < ND) {
                    int c[3];
                    node_coords<NP>(n, c);
#pragma unroll
                    for (int dir = 0; dir < DIM; ++dir) {
                        const int pos = c[dir];
                        int base, stride;
                        line_base<DIM, NP>(dir, line_index<DIM, NP>(dir, c), base, stride);
#pragma unroll
                        for (int l = 0; l < NP; ++l) {
                            const Real dh = sDh[pos * NP + l];
#pragma unroll
                            for (int f = 1; f < NF; ++f)
                                dUv[k][f] += sV[(dir * LY::VROWS + f - LY::VOFF) * ND + base + l * stride] * dh;
                        }
                    }
                }
            }
            group_sync<GS>(gid);   // the pair phase overwrites the buffer
        }

        // ---- inviscid flux differencing, one direction at a time:
        //      sum_l Dhat2(i,l) F#(i,l) with F#(i,i) = 0
#pragma unroll
        for (int dir = 0; dir < DIM; ++dir) {
            Real mt[DIM];
#pragma unroll
            for (int q = 0; q < DIM; ++q) mt[q] = adj[dir][q];
            for (int p = li; p < NPD; p += GS) {
                const uint32_t pr = sPair[dir * NPD + p];
                Real F[NF], mp[DIM];
                if constexpr (CURV) {   // ComputeMean(metric1, metric2) of the pair's nodes
#pragma unroll
                    for (int q = 0; q < DIM; ++q)
                        mp[q] = (Real(ngeo(int(pr & 0xffffu), dir * DIM + q)) + Real(ngeo(int(pr >> 16), dir * DIM + q))) *
                                Real(0.5);
                } else {
#pragma unroll
                    for (int q = 0; q < DIM; ++q) mp[q] = mt[q];
                }
                volume_flux<DIM, Real>(load_prim<DIM, ND, Real>(sH, int(pr & 0xffffu)),
                                       load_prim<DIM, ND, Real>(sH, int(pr >> 16)), mp, gm1i, F);
                if (rad) {   // f *= r at the pair's reference midpoint (:273-291, :319-338)
                    const Real rh = Real(0.5 * (__ldg(rad + (long long)e * ND + int(pr & 0xffffu)) +
                                                __ldg(rad + (long long)e * ND + int(pr >> 16))));
#pragma unroll
                    for (int f = 0; f < NF; ++f) F[f] *= rh;
                }
#pragma unroll
                for (int f = 0; f < NF; ++f) sF[f * NPD + p] = F[f];
            }
            group_sync<GS>(gid);
#pragma unroll
            for (int k = 0; k < NPL; ++k) {
                const int n = li + k * GS;
                if (n < ND) {
                    int c[3];
                    node_coords<NP>(n, c);
                    const int pos = c[dir];
                    const int ln = line_index<DIM, NP>(dir, c);
#pragma unroll
                    for (int l = 0; l < NP; ++l) {
                        if (l == pos) continue;
                        const Real dh = sDh2[pos * NP + l];
                        if (NS && DIM == 3 && dir == 2 && l < pos && P.quirks == 0) {
                            // Q2 (DGSEMIntegrator.cpp:702): H(id2)(:,k) = g, the last
                            // eta-pair flux of node (i,j,l): the pair (j, Np-1) on the
                            // eta line through (i, ., l); zero when j == Np-1.
                            if (c[1] != NP - 1) {
                                Real F[NF], mg[DIM];
                                const int na = (l * NP + c[1]) * NP + c[0], nb = (l * NP + NP - 1) * NP + c[0];
#pragma unroll
                                for (int q = 0; q < DIM; ++q)
                                    mg[q] = CURV ? (Real(ngeo(na, DIM + q)) + Real(ngeo(nb, DIM + q))) * Real(0.5)
                                                 : adj[1][q];
                                volume_flux<DIM, Real>(load_prim<DIM, ND, Real>(sH, na),
                                                       load_prim<DIM, ND, Real>(sH, nb), mg, gm1i, F);
#pragma unroll
                                for (int f = 0; f < NF; ++f) dUi[k][f] += dh * F[f];
                            }
                        } else {
                            const int pidx = ln * PPL + (l < pos ? pair_index<NP>(l, pos) : pair_index<NP>(pos, l));
#pragma unroll
                            for (int f = 0; f < NF; ++f) dUi[k][f] += dh * sF[f * NPD + pidx];
                        }
                    }
                }
            }
            group_sync<GS>(gid);
        }
#pragma unroll
        for (int k = 0; k < NPL; ++k) {
            const int n = li + k * GS;
            // J = Tr.Weight() at the node (dU /= J)
            const Real mJn = CURV ? Real(1.0 / (n < ND ? ngeo(n, DIM * DIM) : 1.0)) : mJ;
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                Real v = -dUi[k][f];
                if (P.blending) v *= (Real(1) - alpha);
                if (NS) v += dUv[k][f];
                acc[k][f] = v * mJn;
            }
        }
    }
    if (rad) {   // + p on the radial momentum (DGSEMIntegrator.cpp:411-428), not blended
#pragma unroll
        for (int k = 0; k < NPL; ++k) {
            const int n = li + k * GS;
            if (n < ND) {
                const Prim<DIM, Real> q = load_prim<DIM, ND, Real>(sH, n);
                if constexpr (LY::F64) acc[k][2] += Real(0.5) * q.rbeta * q.rho;
                else acc[k][2] += q.dp;   // pref = 0 here: dp is p
            }
        }
    }

    // ---- subcell first-order FV (DGSEMIntegrator.cpp:972-1196), skipped when alpha == 0
    if (P.blending && alpha != Real(0)) {
        Real fv[NPL][NF];
#pragma unroll
        for (int dir = 0; dir < DIM; ++dir) {
            Real nor[DIM];
#pragma unroll
            for (int q = 0; q < DIM; ++q) nor[q] = adj[dir][q];
            for (int it = li; it < NID; it += GS) {
                const int ln = it / (NP - 1), ii = it - ln * (NP - 1);
                int base, stride;
                line_base<DIM, NP>(dir, ln, base, stride);
                const int n1 = base + ii * stride, n2 = n1 + stride;
                const Prim<DIM, Real> q1 = load_prim<DIM, ND, Real>(sH, n1), q2 = load_prim<DIM, ND, Real>(sH, n2);
                Real s1[NF], s2[NF], F[NF], ni[DIM];
#pragma unroll
                for (int q = 0; q < DIM; ++q)   // non-affine: ComputeSubcellMetrics (:1199-1304)
                    ni[q] = CURV ? Real(__ldg(a.snor + (((long long)e * DIM + dir) * S::NLINE * (NP - 1) + it) * DIM + q))
                                 : nor[q];
#pragma unroll
                for (int d = 0; d < DIM; ++d) { s1[1 + d] = q1.rho * q1.v[d]; s2[1 + d] = q2.rho * q2.v[d]; }
                face_flux<DIM, Real>(s1, q1, s2, q2, ni, gm1i, P.quirks == 0, true, F);
                if (rad) {   // DGSEMIntegrator.cpp:979-1031, 1096-1111
                    const Real rh = Real(0.5 * (__ldg(rad + (long long)e * ND + n1) + __ldg(rad + (long long)e * ND + n2)));
#pragma unroll
                    for (int f = 0; f < NF; ++f) F[f] *= rh;
                }
#pragma unroll
                for (int f = 0; f < NF; ++f) sF[f * NID + it] = F[f];
            }
            group_sync<GS>(gid);
#pragma unroll
            for (int k = 0; k < NPL; ++k) {
                const int n = li + k * GS;
                if (n < ND) {
                    int c[3];
                    node_coords<NP>(n, c);
                    const int pos = c[dir];
                    const int ib = line_index<DIM, NP>(dir, c) * (NP - 1);
                    const Real mw = Real(1.0 / ((CURV ? ngeo(n, DIM * DIM) : J) * double(sW[pos])));
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        Real v;
                        if (pos == 0) v = -sF[f * NID + ib];
                        else if (pos == NP - 1) v = sF[f * NID + ib + pos - 1];
                        else v = sF[f * NID + ib + pos - 1] - sF[f * NID + ib + pos];
                        v *= mw;
                        fv[k][f] = (dir == 0) ? v : fv[k][f] + v;
                    }
                }
            }
            group_sync<GS>(gid);
        }
#pragma unroll
        for (int k = 0; k < NPL; ++k)
#pragma unroll
            for (int f = 0; f < NF; ++f) acc[k][f] = fv[k][f] * alpha + acc[k][f];
    }

    // ---- surface fluxes of the element's own faces; neighbour traces from global/L2.
    //      For N >= 3 a lane's face items go in pairs: both items' loads are in
    //      flight before either is evaluated.
    const Real aw = Real(1.0 / (double(sW[0]) * J));
    struct FaceIn {
        int4 t;
        double s[NF];                  // neighbour trace (interior face) or own trace (boundary)
        double nb[DIM];                // scaled normal
        Real vo[NF - 1], vn[NF - 1];   // VC form: own / neighbour contravariant viscous rows
    };
    auto face_load = [&](int it, FaceIn &x) {
        const int lf = it / NFN, fa = it - lf * NFN;
        const long long go = (long long)e * ND + face_node<DIM, NP>(lf, fa);
        x.t = NBR_SMEM ? sNbr[lf] : __ldg(a.nbr + (long long)e * (2 * DIM) + lf);
        const long long gs = x.t.x < 0 ? go : (long long)x.t.x * ND + face_node<DIM, NP>(x.t.y, fa);
#pragma unroll
        for (int f = 0; f < NF; ++f) x.s[f] = __ldg(a.u + f * Ndof + gs);
#pragma unroll
        for (int q = 0; q < DIM; ++q)   // non-affine: CalcOrtho at the face point
            x.nb[q] = CURV ? __ldg(a.fnn + ((long long)x.t.z * NFN + fa) * DIM + q)
                           : __ldg(a.fnor + (long long)x.t.z * DIM + q);
        if constexpr (NS && VC) {
            const int dd = lf >> 1, dn = x.t.x < 0 ? dd : x.t.y >> 1;
#pragma unroll
            for (int f = 1; f < NF; ++f) {
                x.vo[f - 1] = __ldg(grad + (dd * (NF - 1) + f - 1) * Ndof + go);
                x.vn[f - 1] = __ldg(grad + (dn * (NF - 1) + f - 1) * Ndof + gs);
            }
        }
    };
    constexpr int FB = NP >= 4 ? 2 : 1;   // face items whose loads go together
    for (int it0 = li; it0 < NFI; it0 += FB * GS) {
      FaceIn xin[FB];
#pragma unroll
      for (int q2 = 0; q2 < FB; ++q2)
          if (it0 + q2 * GS < NFI) face_load(it0 + q2 * GS, xin[q2]);
#pragma unroll
      for (int q2 = 0; q2 < FB; ++q2) {
        const int it = it0 + q2 * GS;
        if (it >= NFI) break;
        const FaceIn &x = xin[q2];
        const int lf = it / NFN, fa = it - lf * NFN;
        const int no = face_node<DIM, NP>(lf, fa);
        const int4 t = x.t;
        const long long go = (long long)e * ND + no;
        // 1 / (w0 J): non-affine elements take J at the face point (Elem1/Elem2 Weight())
        const Real awn = CURV ? Real(1.0 / (double(sW[0]) * ngeo(no, DIM * DIM))) : aw;
        if (t.x < 0) {   // boundary face: the element is Elem1 (BdrFaceIntegrator.cpp:61-186)
            double sb[NF], nb[DIM];
            Real fb[NF], fv[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) sb[f] = x.s[f];
#pragma unroll
            for (int q = 0; q < DIM; ++q) nb[q] = x.nb[q];
            const BcDev &bc = a.bcs[t.y];
            boundary_flux<DIM, Real>(bc, sb, nb, P, pref, fb);
            if (rad) {   // BdrFaceIntegrator.cpp:109-111
                const Real rr = Real(__ldg(rad + go));
#pragma unroll
                for (int f = 0; f < NF; ++f) fb[f] *= rr;
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) fv[f] = 0;
            if constexpr (NS) {
                // viscous boundary flux (ComputeBdrFaceViscousFlux): Fv(inner state,
                // inner gradients) . n for the no-slip walls and supersonic outflow;
                // the other accepted types evaluate Fv with zero gradients, i.e. 0
                if (bc.type == BC_NOSLIP_ADIABATIC || bc.type == BC_NOSLIP_ISOTHERMAL || bc.type == BC_OUTFLOW) {
                    if constexpr (VC) {
                        // n = sgo * row lf/2 of adj(J): Fv . n is a signed row of adj * Fv^T
                        const Real sgo = (lf & 1) ? Real(1) : Real(-1);
#pragma unroll
                        for (int f = 1; f < NF; ++f) fv[f] = sgo * x.vo[f - 1];
                    } else {
                        const Prim<DIM, Real> q = load_prim<DIM, ND, Real>(sH, no);
                        Real dq[DIM][NF], nr[DIM];
#pragma unroll
                        for (int d = 0; d < DIM; ++d) {
                            nr[d] = Real(nb[d]);
#pragma unroll
                            for (int f = 0; f < NF; ++f) dq[d][f] = __ldg(grad + (d * NF + f) * Ndof + go);
                        }
                        viscous_flux<DIM, Real>(q.rho, q.rrho, q.v, Real(0.5) * q.rbeta * q.rho, dq, P,
                                                [&](int f, int cc, Real val) { fv[f] += val * nr[cc]; });
                    }
                    if (bc.type == BC_NOSLIP_ADIABATIC) {   // NoSlipAdiabWallBdrFaceIntegrator.cpp:17-31
                        double nn = 0.0;
#pragma unroll
                        for (int q = 0; q < DIM; ++q) nn += nb[q] * nb[q];
                        Real e = 0;
#pragma unroll
                        for (int d = 0; d < DIM; ++d) e += Real(bc.wall_vel[d]) * fv[1 + d];
                        fv[NF - 1] = e + Real(bc.heat_flux * sqrt(nn));
                    }
                }
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) sF[f * NFI + it] = awn * (fv[f] - fb[f]);
            continue;
        }
        const long long gn = (long long)t.x * ND + face_node<DIM, NP>(t.y, fa);
        const bool own_is_1 = (t.w == 0);
        // the own trace's conserved state is read only by the gradient form
        // (its Q8 path rebuilds the trace from it); otherwise only its momentum
        // enters the surface flux, formed from the hoisted rho and v
        constexpr bool OWN_STATE = NS && !VC;
        double so[NF], sn[NF];
        Real nor[DIM], flux[NF], fn[NF], mo[NF], mn[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            if constexpr (OWN_STATE) so[f] = __ldg(a.u + f * Ndof + go);
            sn[f] = x.s[f];
        }
#pragma unroll
        for (int q = 0; q < DIM; ++q) nor[q] = Real(x.nb[q]);
        Prim<DIM, Real> po = load_prim<DIM, ND, Real>(sH, no);
        Prim<DIM, double> pn64;
        Prim<DIM, Real> pn;
        if constexpr (!LY::F64 && !(NS && !VC)) {
            pn = primitives_mixed<DIM>(sn, gamma, gm1, pref);
        } else {
            pn64 = primitives<DIM, double>(sn, gamma, gm1);
            pn = cast_prim<DIM, Real>(pn64, pref);
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) fn[f] = 0;
        if constexpr (NS && VC) {
            // 0.5 (Fv1 + Fv2) . n from the traces' contravariant viscous fluxes: for
            // affine elements the outward scaled normal of local face lf is
            // (lf odd ? +1 : -1) times row lf/2 of adj(J) (Nanson's formula), so
            // Fv . n_out is a signed row of adj * Fv^T.  fn is taken along nor.
            const Real sgo = (lf & 1) ? Real(1) : Real(-1), sgn = (t.y & 1) ? Real(1) : Real(-1);
#pragma unroll
            for (int f = 1; f < NF; ++f) {
                const Real vo = x.vo[f - 1];
                const Real vn = x.vn[f - 1];
                const Real avg = Real(0.5) * (sgo * vo - sgn * vn);
                fn[f] = own_is_1 ? avg : -avg;
            }
        } else if constexpr (NS) {
            // DGSEMIntegrator.cpp:435-549: 0.5 (Fv1 + Fv2) . n from each trace's
            // own state and lifted gradients
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const long long g = side == 0 ? go : gn;
                const Prim<DIM, Real> &q = side == 0 ? po : pn;
                Real dq[DIM][NF];
#pragma unroll
                for (int d = 0; d < DIM; ++d)
#pragma unroll
                    for (int f = 0; f < NF; ++f) dq[d][f] = __ldg(grad + (d * NF + f) * Ndof + g);
                viscous_flux<DIM, Real>(q.rho, q.rrho, q.v, Real(0.5) * q.rbeta * q.rho, dq, P,
                                        [&](int f, int cc, Real val) { fn[f] += (Real(0.5) * val) * nor[cc]; });
            }
            if (P.quirks == 0) {
                // Q8 (BasicOperations.cpp:33-34 via NavierStokesFlux.cpp:14): the face
                // Riemann flux reads states whose momentum slots now hold velocity.
                const Prim<DIM, double> po64 = primitives<DIM, double>(so, gamma, gm1);
#pragma unroll
                for (int d = 0; d < DIM; ++d) { so[1 + d] *= po64.rrho; sn[1 + d] *= pn64.rrho; }
                po = cast_prim<DIM, Real>(primitives<DIM, double>(so, gamma, gm1), pref);
                pn = cast_prim<DIM, Real>(primitives<DIM, double>(sn, gamma, gm1), pref);
            }
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) mn[f] = Real(sn[f]);
        if constexpr (OWN_STATE) {
#pragma unroll
            for (int f = 0; f < NF; ++f) mo[f] = Real(so[f]);
        } else {
            mo[0] = po.rho;
            mo[NF - 1] = 0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) mo[1 + d] = po.rho * po.v[d];
        }
        if (own_is_1)
            face_flux<DIM, Real>(mo, po, mn, pn, nor, gm1i, P.quirks == 0, P.dissipation != 0, flux);
        else
            face_flux<DIM, Real>(mn, pn, mo, po, nor, gm1i, P.quirks == 0, P.dissipation != 0, flux);
        if (rad) {   // DGSEMIntegrator.cpp:190-207: r at the face point, from element 1
            const Real rr = Real(__ldg(rad + (own_is_1 ? go : gn)));
#pragma unroll
            for (int f = 0; f < NF; ++f) flux[f] *= rr;
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) sF[f * NFI + it] = awn * (own_is_1 ? (fn[f] - flux[f]) : (flux[f] - fn[f]));
      }
    }
    group_sync<GS>(gid);

    // ---- gather face terms, epilogue (FP64 state update).  The stage's global
    //      operands of a lane's nodes (up to 4) are in flight before the gather.
    if (!active) return;
    const int mode = a.mode;
    const bool need_b = (mode == EPI_LSRK && a.rkA != 0.0) || mode == EPI_SSP2 || mode == EPI_SSP3;
    const double *pb = mode == EPI_LSRK ? a.du : a.x0;
    constexpr int KB = NPL <= 4 ? NPL : 1;   // nodes whose operands load together
#pragma unroll
    for (int k0 = 0; k0 < NPL; k0 += KB) {
        double ua[KB][NF], ub[KB][NF];
#pragma unroll
        for (int kk = 0; kk < KB; ++kk) {
            const int n = li + (k0 + kk) * GS;
            const long long gnode = (long long)e * ND + n;
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const long long g = f * Ndof + gnode;
                ua[kk][f] = (k0 + kk < NPL && n < ND && mode != EPI_STORE) ? __ldg((a.u_rk ? a.u_rk : a.u) + g) : 0.0;
                ub[kk][f] = (k0 + kk < NPL && n < ND && need_b) ? pb[g] : 0.0;
            }
        }
#pragma unroll
        for (int kk = 0; kk < KB; ++kk) {
            const int k = k0 + kk;
            const int n = li + k * GS;
            if (k >= NPL || n >= ND) continue;
            int c[3];
            node_coords<NP>(n, c);
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                int lf = -1;
                if (c[d] == 0) lf = 2 * d;
                else if (c[d] == NP - 1) lf = 2 * d + 1;
                if (lf >= 0) {
                    const int it = lf * NFN + face_tangential<DIM, NP>(d, c);
#pragma unroll
                    for (int f = 0; f < NF; ++f) acc[k][f] += sF[f * NFI + it];
                }
            }
            const long long gnode = (long long)e * ND + n;
            if (rad && a.axis && a.axis[gnode]) acc[k][2] = 0;   // DGSEMOperator::ZeroAxisRadialMom
            if (mode == EPI_STORE) {
#pragma unroll
                for (int f = 0; f < NF; ++f) a.dudt[f * Ndof + gnode] = double(acc[k][f]);
                continue;
            }
            // the node's new RK state, per scheme and stage, with the state check
            // (Simulation.cpp:1024-1035 checks rho for NaN) tracked field by field
            // as the values are stored: non-finite values anywhere, and (planar
            // form) rho <= 0 or p <= 0, where p = (gamma-1)(E - |m|^2 / (2 rho)) > 0
            // <=> 2 rho E - |m|^2 > 0 for rho > 0; one atomic per violating node,
            // none on healthy states.  (One loop per mode: a mode test inside one
            // loop over the fields raised the N=4 FP32 kernels' spills.)
            bool finite = true;
            double rho_n = 0.0, mm = 0.0, e_n = 0.0;
            auto track = [&](int f, double v) {
                finite = finite && isfinite(v);
                if (f == 0) rho_n = v;
                else if (f < NF - 1) mm += v * v;
                else e_n = v;
            };
            switch (mode) {
            case EPI_LSRK:
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    const long long g = f * Ndof + gnode;
                    const double L = double(acc[k][f]);
                    const double dv = (a.rkA == 0.0) ? a.dt * L : a.rkA * ub[kk][f] + a.dt * L;
                    a.du[g] = dv;
                    const double v = ua[kk][f] + a.rkB * dv;
                    a.u_out[g] = v;
                    track(f, v);
                }
                break;
            case EPI_SSP1:
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    const double v = ua[kk][f] + a.dt * double(acc[k][f]);
                    a.u_out[f * Ndof + gnode] = v;
                    track(f, v);
                }
                break;
            case EPI_SSP2:
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    const double y = ua[kk][f] + a.dt * double(acc[k][f]);
                    const double v = 3. / 4 * ub[kk][f] + 1. / 4 * y;
                    a.u_out[f * Ndof + gnode] = v;
                    track(f, v);
                }
                break;
            default:
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    const double y = ua[kk][f] + a.dt * double(acc[k][f]);
                    const double v = 1. / 3 * ub[kk][f] + 2. / 3 * y;
                    a.u_out[f * Ndof + gnode] = v;
                    track(f, v);
                }
                break;
            }
            if (a.health) {
                unsigned bad = finite ? 0u : 1u;
                if (rad == nullptr && finite) {   // the axisymmetric r U vanishes on the axis
                    if (!(rho_n > 0.0)) bad |= 2u;
                    else if (!(2.0 * rho_n * e_n - mm > 0.0)) bad |= 4u;
                }
                if (bad) atomicOr(a.health, bad);
            }
        }
    }
}

// One-shot kernel: grid = ceil(E / EPB), one element per lane group.  CURV:
// non-affine elements (per-node geometry; FP64, or FP32-bulk Euler).
template <int DIM, int NP, bool NS, bool VC, typename Real, bool CURV>
__global__ void __launch_bounds__(RhsLayout<DIM, NP, NS, Real, 0, VC>::THREADS, (RhsLayout<DIM, NP, NS, Real, 0, VC>::MIN_BLOCKS))
rhs_kernel(const MeshDev m, const RhsArgs a, const PhysParams P, const __grid_constant__ OpTables T) {
    using LY = RhsLayout<DIM, NP, NS, Real, 0, VC>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real *smem = reinterpret_cast<Real *>(smem_raw);
    uint32_t *sPair = reinterpret_cast<uint32_t *>(smem_raw + LY::TAB_BYTES);
    Real *sE = reinterpret_cast<Real *>(smem_raw + LY::TAB_BYTES + LY::PAIR_BYTES);
    load_tables<NP, Real>(T, smem, threadIdx.x, LY::THREADS);
    load_pair_table<DIM, NP>(sPair, threadIdx.x, LY::THREADS);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int grp = threadIdx.x / LY::GS;          // element slot within the CTA
    const int li = threadIdx.x - grp * LY::GS;     // lane within the group
    const int e_raw = blockIdx.x * LY::EPB + grp;
    const bool active = e_raw < m.E;
    const ElemIO io = io_from_args(m, a);
    rhs_element<DIM, NP, NS, VC, Real, LY, CURV>(io, P, active ? e_raw : m.E - 1, active, smem, sPair,
                                                 sE + grp * LY::PER_ELEM, li, lane, grp);
}

// Persistent batch kernel: a fixed grid walks the class's work items with a
// grid-stride loop.  An item is one warp's EPW elements, or one two-warp
// group's element, of one solve.  The item count and the solves are read from
// device memory, so a captured graph stays valid as solves are admitted and
// retired.  Items of finished solves and items wholly inside a solve's padding
// are skipped (uniformly over the item's lanes).
template <int DIM, int NP, bool NS, bool VC, typename Real, int V>
__global__ void __launch_bounds__(RhsLayout<DIM, NP, NS, Real, V, VC>::THREADS, (RhsLayout<DIM, NP, NS, Real, V, VC>::MIN_BLOCKS))
rhs_batch_kernel(const BatchClassDev c, const BatchStage st, const __grid_constant__ OpTables T) {
    using LY = RhsLayout<DIM, NP, NS, Real, V, VC>;
    static_assert(LY::ITEMS_PER_CTA * sizeof(WarpCtx) <= CTX_RESERVE, "per-item contexts exceed the reserve");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real *sT = reinterpret_cast<Real *>(smem_raw);
    uint32_t *sPair = reinterpret_cast<uint32_t *>(smem_raw + LY::TAB_BYTES);
    WarpCtx *ctxs = reinterpret_cast<WarpCtx *>(smem_raw + LY::TAB_BYTES + LY::PAIR_BYTES);
    Real *sE = reinterpret_cast<Real *>(smem_raw + LY::FIXED_BYTES);
    load_tables<NP, Real>(T, sT, threadIdx.x, LY::THREADS);
    load_pair_table<DIM, NP>(sPair, threadIdx.x, LY::THREADS);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int grp = threadIdx.x / LY::GS;              // element slot (lane group) in the CTA
    const int li = threadIdx.x - grp * LY::GS;
    const int slot = threadIdx.x / LY::ITEM_THREADS;   // item slot in the CTA
    const int il = threadIdx.x - slot * LY::ITEM_THREADS;
    const int gw = il / LY::GS;                        // element within the item
    WarpCtx *ctx = ctxs + slot;
    Real *sH = sE + grp * LY::PER_ELEM;
    const int n = c.hdr[0];
    const int total = n > 0 ? c.prefix[n] / LY::ITEM_ELEMS : 0;
    for (int item = blockIdx.x * LY::ITEMS_PER_CTA + slot; item < total; item += gridDim.x * LY::ITEMS_PER_CTA) {
        const int first = item * LY::ITEM_ELEMS;
        const int s = batch_slot(c.prefix, n, first);
        BatchInst *Im = c.tab + __ldg(c.ids + s);
        const int E = Im->E;
        const int e0 = first - __ldg(c.prefix + s);
        if (e0 >= E || Im->steps_left <= 0) continue;
        group_sync<LY::ITEM_THREADS>(slot);   // the previous item's reads of ctx are done
        {
            const int *src = reinterpret_cast<const int *>(&Im->P);
            int *dst = reinterpret_cast<int *>(&ctx->P);
            if (il < 32)
                for (int q = il; q < (int)(sizeof(PhysParams) / 4); q += 32) dst[q] = src[q];
            if (il == 0) ctx->io = io_from_batch(*Im, Im, st);
        }
        group_sync<LY::ITEM_THREADS>(slot);
        const int e_raw = e0 + gw;
        const bool active = e_raw < E;
        rhs_element<DIM, NP, NS, VC, Real, LY>(ctx->io, ctx->P, active ? e_raw : E - 1, active, sT, sPair, sH, li,
                                               lane, grp);
    }
}

// ------------------------------------------------------------ BR1 lifting
// Entropy variables (BasicOperations.cpp:81-104), element gradient
// (LiftingBR1.cpp:156-272), face lifting 1/2 (v2 - v1) n (LiftingBR1.cpp:10-115)
// and the chain rule to primitive gradients (BasicOperations.cpp:126-170), in
// the working precision W: double, or float for the FP32-bulk form, where the
// entropy variables are taken relative to the element's node 0 (constants
// drop out of the gradients) and only their logarithms of FP64 ratios are
// evaluated in FP32.
//
// The element function uses __syncthreads: every thread of the CTA calls it
// with the same control flow (n = node, sElem = this element's area).
// BR1 lifting at a boundary face node (LiftingBR1.cpp:311-407 with
// ComputeBdrFaceLiftingFlux): the gradient receives lf * nor / (w0 J) with
//   default: lf = 1/2 (v(outer state) - v1) (BdrFaceIntegrator.cpp:274-281),
//            the outer state formed from the trace itself (the reference forms
//            it from Entropy2Conserv(v1), the same state up to rounding);
//            reference mode (Q12): Entropy2Conserv's `vel /= beta` wraps v1, so
//            the middle entries of v1 in the jump are velocities;
//   no-slip walls: lf = v_wall - v1, v_wall = (v1_0, V_wall b, -b) with b = beta1
//            (adiabatic) or 1 / (R_gas T_wall) (NoSlip*WallBdrFaceIntegrator.cpp).
// The element's jump is 1/2 (vn - v1), so vn = v1 + 2 lf is returned (entropy
// variables of the lift's working form: absolute in FP64, relative to the
// element's node 0 in FP32 with absolute middle entries).
template <int DIM, typename W>
__device__ __forceinline__ void boundary_lift_trace(const ElemIO &a, const PhysParams &P, const EntropyRef &R,
                                                    long long g, const int4 t, W *vn, const double *nor) {
    constexpr int NF = DIM + 2;
    constexpr bool F64 = sizeof(W) == 8;
    const BcDev &bc = a.bcs[t.y];
    double s1[NF], nb[DIM], nn = 0.0;
#pragma unroll
    for (int f = 0; f < NF; ++f) s1[f] = __ldg(a.u + f * a.Ndof + g);
#pragma unroll
    for (int q = 0; q < DIM; ++q) {   // nor: the face's scaled normal (per face node on non-affine meshes)
        nb[q] = __ldg(nor + q);
        nn += nb[q] * nb[q];
    }
    nn = sqrt(nn);
    W v1[NF];
    if constexpr (F64) conserv2entropy<DIM, double>(s1, P, reinterpret_cast<double *>(v1));
    else conserv2entropy_rel<DIM>(s1, P, R, reinterpret_cast<float *>(v1));
    const double rr = 1.0 / s1[0];
    if (bc.type == BC_NOSLIP_ADIABATIC || bc.type == BC_NOSLIP_ISOTHERMAL) {
        double vv = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) vv += (s1[1 + d] * rr) * (s1[1 + d] * rr);
        const double beta1 = s1[0] * rcp(P.gammaM1 * (s1[NF - 1] - s1[0] * (0.5 * vv)));
        const bool adiab = bc.type == BC_NOSLIP_ADIABATIC;
        const double b = adiab ? beta1 : bc.vT;
        vn[0] = v1[0];
#pragma unroll
        for (int d = 0; d < DIM; ++d) vn[1 + d] = W(2.0 * (bc.wall_vel[d] * b)) - v1[1 + d];
        vn[NF - 1] = adiab ? v1[NF - 1] : W(2.0 * (F64 ? -bc.vT : R.beta - bc.vT)) - v1[NF - 1];
        return;
    }
    double c[NF], s2[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) c[f] = s1[f];
    bc_outer_state<DIM>(bc, c, nb, nn, P, s2);
    if constexpr (F64) conserv2entropy<DIM, double>(s2, P, reinterpret_cast<double *>(vn));
    else conserv2entropy_rel<DIM>(s2, P, R, reinterpret_cast<float *>(vn));
    if (P.quirks == 0) {
#pragma unroll
        for (int d = 0; d < DIM; ++d) vn[1 + d] += v1[1 + d] - W(s1[1 + d] * rr);
    }
}

// Per-node field rows of the lifting in shared memory, as 16-byte vectors:
// row group q holds fields q*VW .. q*VW+VW-1 of every node as one VW-wide
// vector per node ([NV][NITEM] vectors, VW = 4 floats or 2 doubles); the NF % VW
// remaining fields follow as scalar rows ([NR][NITEM]).  One node's NF values
// then take NV 16-byte accesses and NR scalar ones (FP32, 3D: 2 instead of 5).
// Consecutive items are 16 bytes apart, so a warp's accesses to distinct
// items are free of bank conflicts.  The base must be 16-byte aligned.
template <typename W, int NF, int NITEM>
struct FieldRows {
    static constexpr int VW = 16 / (int)sizeof(W);
    static constexpr int NV = NF / VW, NR = NF - NV * VW;
    static constexpr int SIZE = (NF * NITEM + VW - 1) / VW * VW;   // in W, a multiple of 16 bytes
    __device__ static __forceinline__ void store(W *s, int i, const W *v) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            if constexpr (VW == 4) {
                reinterpret_cast<float4 *>(s)[q * NITEM + i] =
                    make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            } else {
                reinterpret_cast<double2 *>(s)[q * NITEM + i] = make_double2(v[2 * q], v[2 * q + 1]);
            }
        }
#pragma unroll
        for (int r = 0; r < NR; ++r) s[NV * VW * NITEM + r * NITEM + i] = v[NV * VW + r];
    }
    __device__ static __forceinline__ void load(const W *s, int i, W *v) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            if constexpr (VW == 4) {
                const float4 t = reinterpret_cast<const float4 *>(s)[q * NITEM + i];
                v[4 * q] = t.x;
                v[4 * q + 1] = t.y;
                v[4 * q + 2] = t.z;
                v[4 * q + 3] = t.w;
            } else {
                const double2 t = reinterpret_cast<const double2 *>(s)[q * NITEM + i];
                v[2 * q] = t.x;
                v[2 * q + 1] = t.y;
            }
        }
#pragma unroll
        for (int r = 0; r < NR; ++r) v[NV * VW + r] = s[NV * VW * NITEM + r * NITEM + i];
    }
};

template <int DIM, int NP, typename W, bool VC, bool CURV = false>
__device__ __forceinline__ void lift_element(const ElemIO &a, const PhysParams &P, int e, bool active,
                                             const W *sT, W *sElem, int n) {
    using S = Shape<DIM, NP>;
    constexpr int ND = S::ND, NF = S::NF, NFN = S::NFN, NFI = S::NFI;
    constexpr bool F64 = sizeof(W) == 8;
    static_assert(!CURV || F64, "non-affine elements: FP64 kernels only");
    using VE = FieldRows<W, NF, ND>;
    using SJ = FieldRows<W, NF, NFI>;
    const W *sD = sT, *sW = sT + 4 * NP * NP;
    W *gout = reinterpret_cast<W *>(a.grad);
    W *sVe = sElem;                 // entropy variables, FieldRows over the nodes
    W *sS = sVe + VE::SIZE;         // face jumps, FieldRows over the face items
    W *sN = sS + SJ::SIZE;          // face normals [2 DIM][DIM] (one per local face);
                                    // non-affine: [NFI][DIM] (one per face node)
    const long long Ndof = a.Ndof;
    const long long gnode = (long long)e * ND + n;
    // FP64: this thread's face items' neighbour-table entries and interior
    // neighbour traces are loaded with the own state (measured 4 % faster).
    // The FP32 form loads them after the own entropy variables: earlier, the
    // longer live ranges spill and cost 10-20 %.
    constexpr int MAXIT = (NFI + ND - 1) / ND;   // face items per thread
    int4 tk[MAXIT];
    double snk[MAXIT][NF];
    if constexpr (F64) {
#pragma unroll
        for (int k = 0; k < MAXIT; ++k) {
            const int it = n + k * ND;
            tk[k] = it < NFI ? __ldg(a.nbr + (long long)e * (2 * DIM) + it / NFN) : make_int4(-1, 0, 0, 0);
        }
#pragma unroll
        for (int k = 0; k < MAXIT; ++k) {
            const int it = n + k * ND;
            if (it < NFI && tk[k].x >= 0) {
                const int fa = it - (it / NFN) * NFN;
                const long long gn = (long long)tk[k].x * ND + face_node<DIM, NP>(tk[k].y, fa);
#pragma unroll
                for (int f = 0; f < NF; ++f) snk[k][f] = __ldg(a.u + f * Ndof + gn);
            }
        }
    }
    double st[NF];
    W v[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) st[f] = __ldg(a.u + f * Ndof + gnode);
    EntropyRef R{};
    if constexpr (F64) {
        conserv2entropy<DIM, double>(st, P, reinterpret_cast<double *>(v));
    } else {
        double s0[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) s0[f] = __ldg(a.u + f * Ndof + (long long)e * ND);
        R = entropy_ref<DIM>(s0, P);
        conserv2entropy_rel<DIM>(st, P, R, reinterpret_cast<float *>(v));
    }
    VE::store(sVe, n, v);
    // the transformation: per element, or (non-affine) at this thread's node
    // (LiftingBR1.cpp:184-186: Tr.SetIntPoint, Weight, AdjugateJacobian)
    const double *geo = a.geo + (long long)e * (DIM * DIM + 1);
    W adj[DIM][DIM];
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int q = 0; q < DIM; ++q)
            adj[r][q] = W(CURV ? __ldg(a.ngeo + (long long)(r * DIM + q) * Ndof + gnode) : __ldg(geo + r * DIM + q));
    const double J = CURV ? __ldg(a.ngeo + (long long)(DIM * DIM) * Ndof + gnode) : __ldg(geo + DIM * DIM);
    int c[3];
    node_coords<NP>(n, c);

    // face part: the neighbour traces' entropy variables are formed before the
    // barrier (their loads overlap the own node's), the jumps after it:
    // +1/(w0 J) * 1/2 (v_elem2 - v_elem1) * n_c on both sides
    W vn[MAXIT][NF], nor[MAXIT][DIM];
    int no[MAXIT];
    bool own1[MAXIT];
#pragma unroll
    for (int k = 0; k < MAXIT; ++k) {
        const int it = n + k * ND;
        if (it < NFI) {
            const int lf = it / NFN, fa = it - lf * NFN;
            no[k] = face_node<DIM, NP>(lf, fa);
            const int4 t = F64 ? tk[k] : __ldg(a.nbr + (long long)e * (2 * DIM) + lf);
            // the scaled normal: per face, or (non-affine) CalcOrtho at this face point
            const double *fn = CURV ? a.fnn + ((long long)t.z * NFN + fa) * DIM : a.fnor + (long long)t.z * DIM;
#pragma unroll
            for (int q = 0; q < DIM; ++q) nor[k][q] = W(__ldg(fn + q));
            own1[k] = (t.w == 0);
            if (t.x < 0) {
                boundary_lift_trace<DIM, W>(a, P, R, e * (long long)ND + no[k], t, vn[k], fn);
                continue;
            }
            if constexpr (F64) {
                conserv2entropy<DIM, double>(snk[k], P, reinterpret_cast<double *>(vn[k]));
            } else {
                const long long gn = (long long)t.x * ND + face_node<DIM, NP>(t.y, fa);
                double sn[NF];
#pragma unroll
                for (int f = 0; f < NF; ++f) sn[f] = __ldg(a.u + f * Ndof + gn);
                conserv2entropy_rel<DIM>(sn, P, R, reinterpret_cast<float *>(vn[k]));
            }
        }
    }
    __syncthreads();   // tables and entropy variables complete
    const W aw = W(1.0 / (double(sW[0]) * J));
    // the jumps per face node and the normal per face; the face's nodes form
    // aw * (jump * n_q) themselves
#pragma unroll
    for (int k = 0; k < MAXIT; ++k) {
        const int it = n + k * ND;
        if (it < NFI) {
            W vo[NF], jf[NF];
            VE::load(sVe, no[k], vo);
#pragma unroll
            for (int f = 0; f < NF; ++f) jf[f] = own1[k] ? W(0.5) * (vn[k][f] - vo[f]) : W(0.5) * (vo[f] - vn[k][f]);
            SJ::store(sS, it, jf);
            if (CURV || it % NFN == 0) {
#pragma unroll
                for (int q = 0; q < DIM; ++q) sN[(CURV ? it : it / NFN) * DIM + q] = nor[k][q];
            }
        }
    }

    // element part: g1(f, r) = sum_l D(pos_r, l) v_l along direction r
    W g1[NF][DIM];
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int r = 0; r < DIM; ++r) g1[f][r] = 0;
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        int base, stride;
        line_base<DIM, NP>(r, line_index<DIM, NP>(r, c), base, stride);
#pragma unroll
        for (int l = 0; l < NP; ++l) {
            const W dl = sD[c[r] * NP + l];
            W vl[NF];
            VE::load(sVe, base + l * stride, vl);
#pragma unroll
            for (int f = 0; f < NF; ++f) g1[f][r] += vl[f] * dl;
        }
    }
    // grad_mat2 = grad_mat1 * adj, times 1/J (LiftingBR1.cpp:205-206)
    const W mJ = W(1.0 / J);
    W g[DIM][NF];
#pragma unroll
    for (int q = 0; q < DIM; ++q)
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            W s = 0;
#pragma unroll
            for (int r = 0; r < DIM; ++r) s += g1[f][r] * adj[r][q];
            g[q][f] = s * mJ;
        }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        int lf = -1;
        if (c[d] == 0) lf = 2 * d;
        else if (c[d] == NP - 1) lf = 2 * d + 1;
        if (lf >= 0) {
            const int it = lf * NFN + face_tangential<DIM, NP>(d, c);
            W jf[NF], nq[DIM];
            SJ::load(sS, it, jf);
#pragma unroll
            for (int q = 0; q < DIM; ++q) nq[q] = sN[(CURV ? it : lf) * DIM + q];
#pragma unroll
            for (int q = 0; q < DIM; ++q)
#pragma unroll
                for (int f = 0; f < NF; ++f) g[q][f] += aw * (jf[f] * nq[q]);
        }
    }
    if (!active) return;
    W sw[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) sw[f] = W(st[f]);
#pragma unroll
    for (int q = 0; q < DIM; ++q) entropygrad2primgrad<DIM, W>(sw, P, g[q]);
    if constexpr (VC) {
        // the node's contravariant viscous flux adj * Fv^T, rows f = 1..NF-1
        // (NavierStokesFlux.cpp:12-58 with this node's state and gradients;
        // flux_mat of DGSEMIntegrator.cpp:632), [DIM][NF-1][Ndof]
        const Prim<DIM, double> q64 = primitives<DIM, double>(st, P.gamma, P.gammaM1);
        W vel[DIM], Vc[DIM][NF];
#pragma unroll
        for (int d = 0; d < DIM; ++d) vel[d] = W(q64.v[d]);
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int f = 0; f < NF; ++f) Vc[r][f] = 0;
        viscous_flux<DIM, W>(W(q64.rho), W(q64.rrho), vel, W(q64.dp), g, P, [&](int f, int cc, W val) {
#pragma unroll
            for (int r = 0; r < DIM; ++r) Vc[r][f] += adj[r][cc] * val;
        });
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int f = 1; f < NF; ++f) gout[(r * (NF - 1) + f - 1) * Ndof + gnode] = Vc[r][f];
    } else {
#pragma unroll
        for (int q = 0; q < DIM; ++q)
#pragma unroll
            for (int f = 0; f < NF; ++f) gout[(q * NF + f) * Ndof + gnode] = g[q][f];
    }
}

// Shared memory of the lifting: the tables (rounded to 16 bytes), then per
// element the entropy variables, the face jumps and the normals, each element's
// part a multiple of 16 bytes (FieldRows wants 16-byte aligned rows).
template <int DIM, int NP, typename W, bool CURV = false>
struct LiftLayout {
    using S = Shape<DIM, NP>;
    static constexpr int VW = 16 / (int)sizeof(W);
    static constexpr int TABW = (S::TAB + VW - 1) / VW * VW;
    static constexpr int PER_ELEM = (FieldRows<W, S::NF, S::ND>::SIZE + FieldRows<W, S::NF, S::NFI>::SIZE +
                                     (CURV ? S::NFI * DIM : 2 * DIM * DIM) + VW - 1) / VW * VW;
};
constexpr int prev_pow2(int v) { return v <= 1 ? 1 : 2 * prev_pow2(v / 2); }
// Batch lift CTA: a power-of-two number of elements, so an item (one CTA's
// elements) never straddles two solves' BATCH_CHUNK-padded ranges.
template <int DIM, int NP, typename Out>
struct LiftBatchShape {
    static constexpr int ND = Shape<DIM, NP>::ND;
    // FP32 27-node elements (3D, N = 2): 8 per CTA (216 threads) fill 96 % of
    // the lanes against 84 % with 4 (measured on the one-shot FP32 lift: -14 %
    // at 4 resident CTAs)
    static constexpr bool WIDE27 = sizeof(Out) == 4 && ND == 27;
    static constexpr int EPB = WIDE27 ? 8 : prev_pow2(cmax(1, 128 / ND));
    static constexpr int THREADS = EPB * ND;
    // resident CTAs the FP32 lift's register budget is sized for (measured on the
    // 3D Navier-Stokes classes: 5 beats 4 by up to 13 %; 6 is better still at
    // Np = 5, N = 4; 4 for the 216-thread CTAs of N = 2); the FP64 lift keeps 4
    static constexpr int MIN_BLOCKS32 = WIDE27 ? 4 : ((DIM == 3 && NP == 5) ? 6 : 5);
    static_assert(BATCH_CHUNK % EPB == 0, "lift item must divide the padding chunk");
};

// Resident CTAs the one-shot lift's register budget is sized for (measured at
// 3D N=3: 5 beats 4 by 3.5 % in FP64 and 6 by -8 %, 6 beats 4 by 11 % in FP32;
// FP32 at N=4: 6 beats 4 by 7 %; FP32 at N=5 and FP64 at N >= 4 keep 4).
template <int NP, typename Out>
constexpr int lift_min_blocks() {
    return NP <= 4 ? (sizeof(Out) == 8 ? PRANDTL_LIFT64_MINB : 6) : ((NP == 5 && sizeof(Out) == 4) ? 6 : 4);
}

template <int DIM, int NP, typename Out, bool VC, bool CURV>
__global__ void __launch_bounds__(Shape<DIM, NP>::THREADS, lift_min_blocks<NP, Out>())
lift_kernel(const MeshDev m, const LiftArgs a, const PhysParams P, const __grid_constant__ OpTables T) {
    using S = Shape<DIM, NP>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Out *smem = reinterpret_cast<Out *>(smem_raw);
    load_tables<NP, Out>(T, smem, threadIdx.x, S::THREADS);
    const int el = threadIdx.x / S::ND;
    const int n = threadIdx.x - el * S::ND;
    const int e_raw = blockIdx.x * S::EPB + el;
    const bool active = e_raw < m.E;
    ElemIO io{};
    io.u = a.u;
    io.grad = sizeof(Out) == 8 ? (void *)a.grad : (void *)a.grad32;
    io.geo = m.geo;
    io.nbr = m.nbr;
    io.fnor = m.fnor;
    io.Ndof = m.Ndof;
    io.E = m.E;
    io.bcs = m.bcs;
    io.u_rk = nullptr;
    io.rad = nullptr;
    io.axis = nullptr;
    io.ngeo = m.ngeo;
    io.fnn = m.fnn;
    io.snor = nullptr;
    using LL = LiftLayout<DIM, NP, Out, CURV>;
    lift_element<DIM, NP, Out, VC, CURV>(io, P, active ? e_raw : m.E - 1, active, smem,
                                         smem + LL::TABW + el * LL::PER_ELEM, n);
}

// Persistent batch lift: CTA-level items of EPB elements of one solve.
template <int DIM, int NP, typename Out, bool VC>
__global__ void __launch_bounds__(LiftBatchShape<DIM, NP, Out>::THREADS,
                                  sizeof(Out) == 8 ? 4 : LiftBatchShape<DIM, NP, Out>::MIN_BLOCKS32)
lift_batch_kernel(const BatchClassDev c, const BatchStage st, const __grid_constant__ OpTables T) {
    using S = Shape<DIM, NP>;
    using LB = LiftBatchShape<DIM, NP, Out>;
    constexpr int TABB = (S::TAB * (int)sizeof(Out) + 15) / 16 * 16;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Out *sT = reinterpret_cast<Out *>(smem_raw);
    WarpCtx *ctx = reinterpret_cast<WarpCtx *>(smem_raw + TABB);
    Out *sE = reinterpret_cast<Out *>(smem_raw + TABB + CTX_RESERVE);
    load_tables<NP, Out>(T, sT, threadIdx.x, LB::THREADS);
    const int el = threadIdx.x / S::ND;
    const int nn = threadIdx.x - el * S::ND;
    const int n = c.hdr[0];
    const int total = n > 0 ? c.prefix[n] / LB::EPB : 0;
    for (int item = blockIdx.x; item < total; item += gridDim.x) {
        const int first = item * LB::EPB;
        const int s = batch_slot(c.prefix, n, first);
        BatchInst *Im = c.tab + __ldg(c.ids + s);
        const int E = Im->E;
        const int e0 = first - __ldg(c.prefix + s);
        if (e0 >= E || Im->steps_left <= 0) continue;   // CTA-uniform
        __syncthreads();   // the previous item's reads of ctx are complete
        {
            const int *src = reinterpret_cast<const int *>(&Im->P);
            int *dst = reinterpret_cast<int *>(&ctx->P);
            for (int q = threadIdx.x; q < (int)(sizeof(PhysParams) / 4); q += LB::THREADS) dst[q] = src[q];
            if (threadIdx.x == 0) ctx->io = io_from_batch(*Im, Im, st);
        }
        __syncthreads();
        const int e_raw = e0 + el;
        const bool active = e_raw < E;
        lift_element<DIM, NP, Out, VC>(ctx->io, ctx->P, active ? e_raw : E - 1, active, sT,
                                   sE + el * LiftLayout<DIM, NP, Out>::PER_ELEM, nn);
    }
}

template <int DIM, int NP, bool NS, bool VC, typename Real>
size_t rhs_smem() {
    using LY = RhsLayout<DIM, NP, NS, Real, 0, VC>;
    return LY::TAB_BYTES + LY::PAIR_BYTES + sizeof(Real) * (size_t)LY::EPB * LY::PER_ELEM;
}
template <int DIM, int NP, bool NS, bool VC, typename Real, int V>
size_t rhs_batch_smem() {
    using LY = RhsLayout<DIM, NP, NS, Real, V, VC>;
    return LY::FIXED_BYTES + sizeof(Real) * (size_t)LY::EPB * LY::PER_ELEM;
}
template <int DIM, int NP, typename Out, bool CURV>
size_t lift_smem() {
    using S = Shape<DIM, NP>;
    using LL = LiftLayout<DIM, NP, Out, CURV>;
    return sizeof(Out) * (LL::TABW + (size_t)S::EPB * LL::PER_ELEM);
}
template <int DIM, int NP, typename Out>
size_t lift_batch_smem() {
    using S = Shape<DIM, NP>;
    return (S::TAB * sizeof(Out) + 15) / 16 * 16 + CTX_RESERVE +
           sizeof(Out) * (size_t)LiftBatchShape<DIM, NP, Out>::EPB * LiftLayout<DIM, NP, Out>::PER_ELEM;
}

// The dynamic shared-memory limit of a kernel, raised once per device (the
// attribute is a property of the function in the device's context): a launch
// then costs only the launch.  `done` is the calling instantiation's bitmask
// of devices already set.
inline cudaError_t smem_attribute_once(const void *kernel, int bytes, std::atomic<unsigned> &done) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    const unsigned bit = dev < 32 ? 1u << dev : 0u;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (err == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return err;
}
// A launch refused for its shared memory (cudaErrorInvalidValue) after the
// attribute was recorded as set means the device's context was reset since:
// forget the device's bit so the next smem_attribute_once sets it again.
inline bool smem_attribute_lost(cudaError_t err, size_t bytes, std::atomic<unsigned> &done) {
    if (err != cudaErrorInvalidValue || bytes <= 48 * 1024) return false;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= 32) return false;
    done.fetch_and(~(1u << dev), std::memory_order_acq_rel);
    return true;
}

template <int DIM, int NP, bool NS, bool VC, typename Real, bool CURV>
cudaError_t rhs_launch_np(const MeshDev &m, const RhsArgs &a, const PhysParams &P, const OpTables &T,
                          cudaStream_t s) {
    using LY = RhsLayout<DIM, NP, NS, Real, 0, VC>;
    const int grid = (m.E + LY::EPB - 1) / LY::EPB;
    const size_t sm = rhs_smem<DIM, NP, NS, VC, Real>();
    static std::atomic<unsigned> smem_set{0u};
    for (int attempt = 0; attempt < 2; ++attempt) {
        cudaError_t err = smem_attribute_once((const void *)rhs_kernel<DIM, NP, NS, VC, Real, CURV>, (int)sm, smem_set);
        if (err != cudaSuccess) return err;
        rhs_kernel<DIM, NP, NS, VC, Real, CURV><<<grid, LY::THREADS, sm, s>>>(m, a, P, T);
        err = cudaGetLastError();
        if (!smem_attribute_lost(err, sm, smem_set)) return err;
    }
    return cudaErrorInvalidValue;
}
// non-affine meshes (m.ngeo set) run the per-node-geometry kernels (FP64, or FP32-bulk Euler)
template <int DIM, int NP, bool NS, bool VC, typename Real>
cudaError_t rhs_launch_any(const MeshDev &m, const RhsArgs &a, const PhysParams &P, const OpTables &T,
                           cudaStream_t s) {
    if (m.ngeo) {   // FP64, or the FP32-bulk Euler form (pair phase; no lifting)
        if constexpr (sizeof(Real) == 8 || !NS) return rhs_launch_np<DIM, NP, NS, VC, Real, true>(m, a, P, T, s);
        else return cudaErrorNotSupported;
    }
    return rhs_launch_np<DIM, NP, NS, VC, Real, false>(m, a, P, T, s);
}
template <int DIM, int NP, typename Out, bool VC, bool CURV>
cudaError_t lift_launch_np(const MeshDev &m, const LiftArgs &a, const PhysParams &P, const OpTables &T,
                           cudaStream_t s) {
    using S = Shape<DIM, NP>;
    const int grid = (m.E + S::EPB - 1) / S::EPB;
    const size_t sm = lift_smem<DIM, NP, Out, CURV>();
    static std::atomic<unsigned> smem_set{0u};
    for (int attempt = 0; attempt < 2; ++attempt) {
        cudaError_t err = smem_attribute_once((const void *)lift_kernel<DIM, NP, Out, VC, CURV>, (int)sm, smem_set);
        if (err != cudaSuccess) return err;
        lift_kernel<DIM, NP, Out, VC, CURV><<<grid, S::THREADS, sm, s>>>(m, a, P, T);
        err = cudaGetLastError();
        if (!smem_attribute_lost(err, sm, smem_set)) return err;
    }
    return cudaErrorInvalidValue;
}
template <int DIM, int NP, typename Out, bool VC>
cudaError_t lift_launch_any(const MeshDev &m, const LiftArgs &a, const PhysParams &P, const OpTables &T,
                            cudaStream_t s) {
    if (m.ngeo) {
        if constexpr (sizeof(Out) == 8) return lift_launch_np<DIM, NP, Out, VC, true>(m, a, P, T, s);
        else return cudaErrorNotSupported;
    }
    return lift_launch_np<DIM, NP, Out, VC, false>(m, a, P, T, s);
}

// Batch kernels: `prepare` sets the shared-memory attribute (outside any stream
// capture) and reports the resident CTAs per SM; `launch` only launches.
template <int DIM, int NP, bool NS, bool VC, typename Real, int V>
cudaError_t rhs_batch_prepare_np(BatchKernelInfo *info) {
    using LY = RhsLayout<DIM, NP, NS, Real, V, VC>;
    const size_t sm = rhs_batch_smem<DIM, NP, NS, VC, Real, V>();
    cudaError_t err = cudaFuncSetAttribute(rhs_batch_kernel<DIM, NP, NS, VC, Real, V>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (err != cudaSuccess) return err;
    int nb = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, rhs_batch_kernel<DIM, NP, NS, VC, Real, V>, LY::THREADS, sm);
    if (err != cudaSuccess) return err;
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, rhs_batch_kernel<DIM, NP, NS, VC, Real, V>);
    info->blocks_per_sm = nb;
    info->threads = LY::THREADS;
    info->smem = (int)sm;
    info->regs = fa.numRegs;
    info->elems_per_item = LY::ITEM_ELEMS;
    return cudaSuccess;
}
template <int DIM, int NP, bool NS, bool VC, typename Real, int V>
cudaError_t rhs_batch_launch_np(int grid, const BatchClassDev &c, const BatchStage &st, const OpTables &T,
                                cudaStream_t s) {
    using LY = RhsLayout<DIM, NP, NS, Real, V, VC>;
    rhs_batch_kernel<DIM, NP, NS, VC, Real, V><<<grid, LY::THREADS, rhs_batch_smem<DIM, NP, NS, VC, Real, V>(), s>>>(c, st, T);
    return cudaGetLastError();
}
template <int DIM, int NP, typename Out, bool VC>
cudaError_t lift_batch_prepare_np(BatchKernelInfo *info) {
    using S = LiftBatchShape<DIM, NP, Out>;
    const size_t sm = lift_batch_smem<DIM, NP, Out>();
    cudaError_t err = cudaFuncSetAttribute(lift_batch_kernel<DIM, NP, Out, VC>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (err != cudaSuccess) return err;
    int nb = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, lift_batch_kernel<DIM, NP, Out, VC>, S::THREADS, sm);
    if (err != cudaSuccess) return err;
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, lift_batch_kernel<DIM, NP, Out, VC>);
    info->blocks_per_sm = nb;
    info->threads = S::THREADS;
    info->smem = (int)sm;
    info->regs = fa.numRegs;
    info->elems_per_item = S::EPB;
    return cudaSuccess;
}
template <int DIM, int NP, typename Out, bool VC>
cudaError_t lift_batch_launch_np(int grid, const BatchClassDev &c, const BatchStage &st, const OpTables &T,
                                 cudaStream_t s) {
    using S = LiftBatchShape<DIM, NP, Out>;
    lift_batch_kernel<DIM, NP, Out, VC><<<grid, S::THREADS, lift_batch_smem<DIM, NP, Out>(), s>>>(c, st, T);
    return cudaGetLastError();
}

}   // namespace

#define PRANDTL_ORDER_SWITCH(CALL)                                       \
    switch (order) {                                                     \
    case 1: { constexpr int NP = 2; return CALL; }                       \
    case 2: { constexpr int NP = 3; return CALL; }                       \
    case 3: { constexpr int NP = 4; return CALL; }                       \
    case 4: { constexpr int NP = 5; return CALL; }                       \
    case 5: { constexpr int NP = 6; return CALL; }                       \
    default: return cudaErrorInvalidValue;                               \
    }
#define PRANDTL_VARIANT_SWITCH(CALLV)                                    \
    switch (variant) {                                                   \
    case 0: { constexpr int VV = 0; CALLV; }                             \
    case 1: { constexpr int VV = 1; CALLV; }                             \
    case 2: { constexpr int VV = 2; CALLV; }                             \
    default: return cudaErrorInvalidValue;                               \
    }

template <int DIM, typename Real, bool NS, bool VC>
cudaError_t rhs_dispatch(int order, const MeshDev &m, const RhsArgs &a, const PhysParams &P,
                         const OpTables &T, cudaStream_t s) {
    PRANDTL_ORDER_SWITCH((rhs_launch_any<DIM, NP, NS, VC, Real>(m, a, P, T, s)))
}
template <int DIM, typename Out, bool VC>
cudaError_t lift_dispatch(int order, const MeshDev &m, const LiftArgs &a, const PhysParams &P,
                          const OpTables &T, cudaStream_t s) {
    PRANDTL_ORDER_SWITCH((lift_launch_any<DIM, NP, Out, VC>(m, a, P, T, s)))
}
template <int DIM, typename Real, bool NS, bool VC>
cudaError_t rhs_batch_prepare(int order, int variant, BatchKernelInfo *info) {
    PRANDTL_ORDER_SWITCH(([&]() -> cudaError_t {
        PRANDTL_VARIANT_SWITCH(return (rhs_batch_prepare_np<DIM, NP, NS, VC, Real, VV>(info)))
    }()))
}
template <int DIM, typename Real, bool NS, bool VC>
cudaError_t rhs_batch_launch(int order, int variant, int grid, const BatchClassDev &c, const BatchStage &st,
                             const OpTables &T, cudaStream_t s) {
    PRANDTL_ORDER_SWITCH(([&]() -> cudaError_t {
        PRANDTL_VARIANT_SWITCH(return (rhs_batch_launch_np<DIM, NP, NS, VC, Real, VV>(grid, c, st, T, s)))
    }()))
}
template <int DIM, typename Out, bool VC>
cudaError_t lift_batch_prepare(int order, BatchKernelInfo *info) {
    PRANDTL_ORDER_SWITCH((lift_batch_prepare_np<DIM, NP, Out, VC>(info)))
}
template <int DIM, typename Out, bool VC>
cudaError_t lift_batch_launch(int order, int grid, const BatchClassDev &c, const BatchStage &st,
                              const OpTables &T, cudaStream_t s) {
    PRANDTL_ORDER_SWITCH((lift_batch_launch_np<DIM, NP, Out, VC>(grid, c, st, T, s)))
}

// One translation unit per (DIM, Real, physics) instantiates its share.
#define PRANDTL_INSTANTIATE_RHS(DIMV, REAL, NSV, VCV)                                                   \
    template cudaError_t rhs_dispatch<DIMV, REAL, NSV, VCV>(int, const MeshDev &, const RhsArgs &,      \
                                                            const PhysParams &, const OpTables &, cudaStream_t); \
    template cudaError_t rhs_batch_prepare<DIMV, REAL, NSV, VCV>(int, int, BatchKernelInfo *);          \
    template cudaError_t rhs_batch_launch<DIMV, REAL, NSV, VCV>(int, int, int, const BatchClassDev &,   \
                                                                const BatchStage &, const OpTables &, cudaStream_t);
#define PRANDTL_INSTANTIATE_LIFT(DIMV, OUT, VCV)                                                        \
    template cudaError_t lift_dispatch<DIMV, OUT, VCV>(int, const MeshDev &, const LiftArgs &,          \
                                                       const PhysParams &, const OpTables &, cudaStream_t); \
    template cudaError_t lift_batch_prepare<DIMV, OUT, VCV>(int, BatchKernelInfo *);                    \
    template cudaError_t lift_batch_launch<DIMV, OUT, VCV>(int, int, const BatchClassDev &, const BatchStage &, \
                                                           const OpTables &, cudaStream_t);

}   // namespace prandtl
