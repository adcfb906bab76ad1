// dgsem_kernels.cu -- element-per-thread-group DGSEM RHS kernels for sm_100a.
//
// One thread per volume node; EPB elements per CTA.  Everything an element
// needs stays in shared memory for the whole RHS evaluation:
//   load state -> (blending coefficient) -> two-point volume fluxes of all
//   unique node pairs -> flux differencing -> (subcell FV) -> surface fluxes of
//   the element's own faces (neighbour traces read from global/L2) -> epilogue
//   (store dudt, or fuse the Runge-Kutta stage update).
// Each interior face flux is evaluated by both neighbouring elements with the
// same operands in the same order, so both sides see bit-identical fluxes and
// no atomics or face buffers are needed.
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
    static constexpr int NPAIR = DIM * NLINE * PPL;     // unique volume pairs
    static constexpr int NFN = ND / NP;                 // nodes per face
    static constexpr int NFACE = 2 * DIM;
    static constexpr int NFI = NFACE * NFN;             // face-node items
    static constexpr int NIF = DIM * NLINE * (NP - 1);  // subcell FV interfaces
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

template <int NP>
__device__ __forceinline__ void load_tables(const OpTables &T, double *sT, int tid, int nthreads) {
    for (int q = tid; q < NP * NP; q += nthreads) {
        const int i = q / NP, l = q % NP;
        sT[q] = T.D[i * NP + l];
        sT[NP * NP + q] = T.Dhat[i * NP + l];
        sT[2 * NP * NP + q] = T.Dhat2[i * NP + l];
        sT[3 * NP * NP + q] = T.Vinv[i * NP + l];
    }
    for (int q = tid; q < NP; q += nthreads) {
        sT[4 * NP * NP + q] = T.w[q];
        sT[4 * NP * NP + NP + q] = T.x[q];
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
template <int DIM>
struct HIdx {
    static constexpr int RHO = 0, RRHO = 1, V = 2, VSQ = 2 + DIM, BETA = 3 + DIM, RBETA = 4 + DIM,
                         LAM = 5 + DIM, K = 6 + DIM;
};
template <int DIM, int ND>
__device__ __forceinline__ Prim<DIM, double> load_prim(const double *sH, int n) {
    using I = HIdx<DIM>;
    Prim<DIM, double> q;
    q.rho = sH[I::RHO * ND + n];
    q.rrho = sH[I::RRHO * ND + n];
#pragma unroll
    for (int d = 0; d < DIM; ++d) q.v[d] = sH[(I::V + d) * ND + n];
    q.vsq = sH[I::VSQ * ND + n];
    q.beta = sH[I::BETA * ND + n];
    q.rbeta = sH[I::RBETA * ND + n];
    q.lam = sH[I::LAM * ND + n];
    return q;
}
template <int DIM, int ND>
__device__ __forceinline__ void store_prim(double *sH, int n, const Prim<DIM, double> &q) {
    using I = HIdx<DIM>;
    sH[I::RHO * ND + n] = q.rho;
    sH[I::RRHO * ND + n] = q.rrho;
#pragma unroll
    for (int d = 0; d < DIM; ++d) sH[(I::V + d) * ND + n] = q.v[d];
    sH[I::VSQ * ND + n] = q.vsq;
    sH[I::BETA * ND + n] = q.beta;
    sH[I::RBETA * ND + n] = q.rbeta;
    sH[I::LAM * ND + n] = q.lam;
}

template <int DIM, int NP, bool NS>
struct RhsLayout {
    using S = Shape<DIM, NP>;
    static constexpr int ND = S::ND, NF = S::NF;
    static constexpr int NSCR = cmax(cmax(S::NPAIR, S::NIF), cmax(S::NFI, 5 * ND / NF + 1)) * NF;
    static constexpr int PER_ELEM = NF * ND + HIdx<DIM>::K * ND + NSCR + (NS ? DIM * NF * ND : 0);
    static constexpr int MIN_BLOCKS = NS ? 3 : 4;
};

// ------------------------------------------------------------------- RHS
template <int DIM, int NP, bool NS>
__global__ void __launch_bounds__(Shape<DIM, NP>::THREADS, (RhsLayout<DIM, NP, NS>::MIN_BLOCKS))
rhs_kernel(const MeshDev m, const RhsArgs a, const PhysParams P, const __grid_constant__ OpTables T) {
    using S = Shape<DIM, NP>;
    using LY = RhsLayout<DIM, NP, NS>;
    constexpr int ND = S::ND, NF = S::NF, NLINE = S::NLINE, PPL = S::PPL, NPAIR = S::NPAIR;
    constexpr int NFN = S::NFN, NFI = S::NFI, NIF = S::NIF, EPB = S::EPB;
    constexpr int NSCR = LY::NSCR, PER_ELEM = LY::PER_ELEM;

    extern __shared__ double smem[];
    __shared__ double sAlpha[EPB];
    __shared__ double sRed[(S::THREADS + 31) / 32];
    double *sT = smem;
    const double *sDh = sT + NP * NP, *sDh2 = sT + 2 * NP * NP, *sVinv = sT + 3 * NP * NP;
    const double *sW = sT + 4 * NP * NP;
    load_tables<NP>(T, sT, threadIdx.x, S::THREADS);

    const int el = threadIdx.x / ND;
    const int n = threadIdx.x - el * ND;
    const int e_raw = blockIdx.x * EPB + el;
    const bool active = e_raw < m.E;
    const int e = active ? e_raw : m.E - 1;
    double *sU = smem + S::TAB + el * PER_ELEM;    // conserved state [NF][ND]
    double *sH = sU + NF * ND;                     // hoisted primitives [K][ND]
    double *sS = sH + HIdx<DIM>::K * ND;           // scratch: pairs / FV / face items
    double *sV = sS + NSCR;                        // NS: contravariant viscous fluxes [DIM][NF][ND]

    const long long Ndof = m.Ndof;
    const long long gnode = (long long)e * ND + n;
    const double gamma = P.gamma, gm1 = P.gammaM1, gm1i = P.gammaM1Inverse;
    double st[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        st[f] = __ldg(a.u + f * Ndof + gnode);
        sU[f * ND + n] = st[f];
    }
    const Prim<DIM, double> me = primitives<DIM, double>(st, gamma, gm1);
    store_prim<DIM, ND>(sH, n, me);
    const double *geo = m.geo + (long long)e * (DIM * DIM + 1);
    double adj[DIM][DIM];
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int c2 = 0; c2 < DIM; ++c2) adj[r][c2] = __ldg(geo + r * DIM + c2);
    const double J = __ldg(geo + DIM * DIM);
    int c[3];
    node_coords<NP>(n, c);

    // ---- largest characteristic speed |V| + c of this state
    if (a.lambda) block_max_to<S::THREADS>(a.lambda, active ? me.lam : 0.0, sRed);

    // ---- blending coefficient (PerssonPeraireIndicator.cpp:21-58, DGSEMOperator.cpp:60-80)
    if (P.blending) {
        double *b0 = sS, *b1 = sS + ND;
        {
            double vv = 0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                const double vd = st[1 + d] * me.rrho;
                vv += vd * vd;
            }
            b0[n] = st[0] * (gm1 * (st[NF - 1] - 0.5 * st[0] * vv));
        }
        __syncthreads();
#pragma unroll
        for (int d = 0; d < DIM; ++d) {   // modes = V^-1 (rho p), one direction per pass
            const double *in = (d & 1) ? b1 : b0;
            double *out = (d & 1) ? b0 : b1;
            int base, stride;
            line_base<DIM, NP>(d, line_index<DIM, NP>(d, c), base, stride);
            double s = 0.0;
#pragma unroll
            for (int l = 0; l < NP; ++l) s += sVinv[c[d] * NP + l] * in[base + l * stride];
            out[n] = s;
            __syncthreads();
        }
        const double md = ((DIM & 1) ? b1 : b0)[n];
        int mx = c[0];
#pragma unroll
        for (int d = 1; d < DIM; ++d) mx = max(mx, c[d]);
        double *r0 = sS + 2 * ND, *r1 = r0 + ND, *r2 = r1 + ND;
        r0[n] = md * md;
        r1[n] = (mx <= NP - 2) ? md * md : 0.0;
        r2[n] = (mx <= NP - 3) ? md * md : 0.0;
        __syncthreads();
        if (n == 0) {
            double e0 = 0, e1 = 0, e2 = 0;
            for (int q = 0; q < ND; ++q) { e0 += r0[q]; e1 += r1[q]; e2 += r2[q]; }
            double eta = 1.0 - e1 / e0;
            eta = fmax(eta, 1.0 - e2 / e1);
            const double thr = P.modal_threshold;
            double al = 1.0 / (1.0 + exp(-9.21024 * (eta - thr) / thr));
            if (al < P.alpha_min) al = 0.0;
            else if (al > 1.0 - P.alpha_min) al = 1.0;
            al = fmin(al, P.alpha_max);
            sAlpha[el] = al;
            if (a.alpha && active) a.alpha[e] = al;
        }
    } else {
        if (n == 0) sAlpha[el] = 0.0;
    }

    // ---- NS: contravariant viscous flux of this node (flux_mat = adj * Fv^T, :632)
    if constexpr (NS) {
        double dq[DIM][NF];
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
            for (int f = 0; f < NF; ++f) dq[d][f] = __ldg(a.grad + (d * NF + f) * Ndof + gnode);
        __syncthreads();   // sU/sH complete: quirk Q1 reads another node
        // Q1 (DGSEMIntegrator.cpp:620): the reference evaluates the volume
        // viscous flux with the state of node Np^d-1 (stale member id1).
        const int src = (P.quirks == 0) ? ND - 1 : n;
        const Prim<DIM, double> q = load_prim<DIM, ND>(sH, src);
        double Vc[DIM][NF];
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int f = 0; f < NF; ++f) Vc[r][f] = 0.0;
        const double pq = q.rbeta * q.rho * 0.5;   // p = rho/(2 beta)
        viscous_flux<DIM, double>(q.rho, q.rrho, q.v, pq, dq, P, [&](int f, int cc, double val) {
#pragma unroll
            for (int r = 0; r < DIM; ++r) Vc[r][f] += adj[r][cc] * val;
        });
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int f = 0; f < NF; ++f) sV[(r * NF + f) * ND + n] = Vc[r][f];
    }
    __syncthreads();
    const double alpha = sAlpha[el];

    // ---- two-point volume fluxes of every unique node pair
    for (int p = n; p < NPAIR; p += ND) {
        const int dir = p / (NLINE * PPL);
        const int r = p - dir * NLINE * PPL;
        const int ln = r / PPL, pp = r - ln * PPL;
        int pa, pb, base, stride;
        pair_decode<NP>(pp, pa, pb);
        line_base<DIM, NP>(dir, ln, base, stride);
        const int n1 = base + pa * stride, n2 = base + pb * stride;
        double F[NF], mt[DIM];
#pragma unroll
        for (int q = 0; q < DIM; ++q) mt[q] = (dir == 0) ? adj[0][q] : (dir == 1 ? adj[1][q] : adj[DIM - 1][q]);
        volume_flux<DIM, double>(load_prim<DIM, ND>(sH, n1), load_prim<DIM, ND>(sH, n2), mt, gm1i, F);
#pragma unroll
        for (int f = 0; f < NF; ++f) sS[f * NPAIR + p] = F[f];
    }
    __syncthreads();

    // ---- flux differencing: sum_l Dhat2(i,l) F#(i,l) per direction (F#(i,i) = 0)
    double acc[NF];
    {
        double dUi[NF], dUv[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) { dUi[f] = 0.0; dUv[f] = 0.0; }
#pragma unroll
        for (int dir = 0; dir < DIM; ++dir) {
            const int pos = c[dir];
            const int ln = line_index<DIM, NP>(dir, c);
            const int pbase = dir * NLINE * PPL + ln * PPL;
#pragma unroll
            for (int l = 0; l < NP; ++l) {
                if (l == pos) continue;
                const double dh = sDh2[pos * NP + l];
                int pidx;
                bool zero = false;
                if (NS && DIM == 3 && dir == 2 && l < pos && P.quirks == 0) {
                    // Q2 (DGSEMIntegrator.cpp:702): H(id2)(:,k) = g, the last
                    // eta-pair flux of node (i,j,l): pair (j, Np-1) on the eta
                    // line through (i, ., l); zero when j == Np-1.
                    if (c[1] == NP - 1) zero = true;
                    pidx = 1 * NLINE * PPL + (l * NP + c[0]) * PPL + pair_index<NP>(c[1], NP - 1);
                } else {
                    pidx = pbase + (l < pos ? pair_index<NP>(l, pos) : pair_index<NP>(pos, l));
                }
                if (!zero) {
#pragma unroll
                    for (int f = 0; f < NF; ++f) dUi[f] += dh * sS[f * NPAIR + pidx];
                }
            }
            if constexpr (NS) {
                int base, stride;
                line_base<DIM, NP>(dir, ln, base, stride);
#pragma unroll
                for (int l = 0; l < NP; ++l) {
                    const double dh = sDh[pos * NP + l];
#pragma unroll
                    for (int f = 0; f < NF; ++f) dUv[f] += sV[(dir * NF + f) * ND + base + l * stride] * dh;
                }
            }
        }
        const double mJ = 1.0 / J;
        const double oma = 1.0 - alpha;
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            double v = -dUi[f];
            if (P.blending) v *= oma;
            if (NS) v += dUv[f];
            acc[f] = v * mJ;
        }
    }
    __syncthreads();

    // ---- subcell first-order FV (DGSEMIntegrator.cpp:972-1196), skipped when alpha == 0
    if (P.blending) {
        if (alpha != 0.0) {
            for (int it = n; it < NIF; it += ND) {
                const int dir = it / (NLINE * (NP - 1));
                const int r = it - dir * NLINE * (NP - 1);
                const int ln = r / (NP - 1), ii = r - ln * (NP - 1);
                int base, stride;
                line_base<DIM, NP>(dir, ln, base, stride);
                const int n1 = base + ii * stride, n2 = n1 + stride;
                double s1[NF], s2[NF], F[NF], nor[DIM];
#pragma unroll
                for (int f = 0; f < NF; ++f) { s1[f] = sU[f * ND + n1]; s2[f] = sU[f * ND + n2]; }
#pragma unroll
                for (int q = 0; q < DIM; ++q) nor[q] = (dir == 0) ? adj[0][q] : (dir == 1 ? adj[1][q] : adj[DIM - 1][q]);
                face_flux<DIM, double>(s1, load_prim<DIM, ND>(sH, n1), s2, load_prim<DIM, ND>(sH, n2), nor, gm1i,
                                       P.quirks == 0, true, F);
#pragma unroll
                for (int f = 0; f < NF; ++f) sS[f * NIF + it] = F[f];
            }
        }
        __syncthreads();
        if (alpha != 0.0) {
            double fv[NF];
#pragma unroll
            for (int dir = 0; dir < DIM; ++dir) {
                const int pos = c[dir];
                const int ln = line_index<DIM, NP>(dir, c);
                const int ib = dir * NLINE * (NP - 1) + ln * (NP - 1);
                const double mw = 1.0 / (J * sW[pos]);
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    double v;
                    if (pos == 0) v = -sS[f * NIF + ib];
                    else if (pos == NP - 1) v = sS[f * NIF + ib + pos - 1];
                    else v = sS[f * NIF + ib + pos - 1] - sS[f * NIF + ib + pos];
                    v *= mw;
                    fv[f] = (dir == 0) ? v : fv[f] + v;
                }
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) acc[f] = fv[f] * alpha + acc[f];
        }
        __syncthreads();
    }

    // ---- surface fluxes of the element's own faces
    const double aw = 1.0 / (sW[0] * J);
    for (int it = n; it < NFI; it += ND) {
        const int lf = it / NFN, fa = it - lf * NFN;
        const int no = face_node<DIM, NP>(lf, fa);
        const int4 t = __ldg(m.nbr + (long long)e * (2 * DIM) + lf);
        const int nn = face_node<DIM, NP>(t.y, fa);
        const long long gn = (long long)t.x * ND + nn;
        const bool own_is_1 = (t.w == 0);
        double so[NF], sn[NF], nor[DIM], flux[NF], d1[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) { so[f] = sU[f * ND + no]; sn[f] = __ldg(a.u + f * Ndof + gn); }
#pragma unroll
        for (int q = 0; q < DIM; ++q) nor[q] = __ldg(m.fnor + (long long)t.z * DIM + q);
        Prim<DIM, double> po = load_prim<DIM, ND>(sH, no);
        Prim<DIM, double> pn = primitives<DIM, double>(sn, gamma, gm1);
        double fn[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) fn[f] = 0.0;
        if constexpr (NS) {
            // DGSEMIntegrator.cpp:435-549: 0.5 (Fv1 + Fv2) . n from each trace's
            // own state and lifted gradients
            const long long go = (long long)e * ND + no;
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const long long g = side == 0 ? go : gn;
                const Prim<DIM, double> &q = side == 0 ? po : pn;
                double dq[DIM][NF];
#pragma unroll
                for (int d = 0; d < DIM; ++d)
#pragma unroll
                    for (int f = 0; f < NF; ++f) dq[d][f] = __ldg(a.grad + (d * NF + f) * Ndof + g);
                viscous_flux<DIM, double>(q.rho, q.rrho, q.v, 0.5 * q.rbeta * q.rho, dq, P,
                                          [&](int f, int cc, double val) { fn[f] += (0.5 * val) * nor[cc]; });
            }
            if (P.quirks == 0) {
                // Q8 (BasicOperations.cpp:33-34 via NavierStokesFlux.cpp:14): the face
                // Riemann flux reads states whose momentum slots now hold velocity.
#pragma unroll
                for (int d = 0; d < DIM; ++d) { so[1 + d] *= po.rrho; sn[1 + d] *= pn.rrho; }
                po = primitives<DIM, double>(so, gamma, gm1);
                pn = primitives<DIM, double>(sn, gamma, gm1);
            }
        }
        if (own_is_1)
            face_flux<DIM, double>(so, po, sn, pn, nor, gm1i, P.quirks == 0, P.dissipation != 0, flux);
        else
            face_flux<DIM, double>(sn, pn, so, po, nor, gm1i, P.quirks == 0, P.dissipation != 0, flux);
#pragma unroll
        for (int f = 0; f < NF; ++f) d1[f] = own_is_1 ? (-flux[f] + fn[f]) : (flux[f] - fn[f]);
#pragma unroll
        for (int f = 0; f < NF; ++f) sS[f * NFI + it] = aw * d1[f];
    }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        int lf = -1;
        if (c[d] == 0) lf = 2 * d;
        else if (c[d] == NP - 1) lf = 2 * d + 1;
        if (lf >= 0) {
            const int it = lf * NFN + face_tangential<DIM, NP>(d, c);
#pragma unroll
            for (int f = 0; f < NF; ++f) acc[f] += sS[f * NFI + it];
        }
    }

    // ---- epilogue
    if (!active) return;
    switch (a.mode) {
    case EPI_STORE:
#pragma unroll
        for (int f = 0; f < NF; ++f) a.dudt[f * Ndof + gnode] = acc[f];
        break;
    case EPI_LSRK:
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            const long long g = f * Ndof + gnode;
            const double dv = (a.rkA == 0.0) ? a.dt * acc[f] : a.rkA * a.du[g] + a.dt * acc[f];
            a.du[g] = dv;
            a.u_out[g] = st[f] + a.rkB * dv;
        }
        break;
    case EPI_SSP1:
#pragma unroll
        for (int f = 0; f < NF; ++f) a.u_out[f * Ndof + gnode] = st[f] + a.dt * acc[f];
        break;
    case EPI_SSP2:
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            const long long g = f * Ndof + gnode;
            const double y = st[f] + a.dt * acc[f];
            a.u_out[g] = 3. / 4 * a.x0[g] + 1. / 4 * y;
        }
        break;
    case EPI_SSP3:
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            const long long g = f * Ndof + gnode;
            const double y = st[f] + a.dt * acc[f];
            a.u_out[g] = 1. / 3 * a.x0[g] + 2. / 3 * y;
        }
        break;
    default:
        break;
    }
}

// ------------------------------------------------------------ BR1 lifting
// Entropy variables (BasicOperations.cpp:81-104), element gradient
// (LiftingBR1.cpp:156-272), face lifting 1/2 (v2 - v1) n (LiftingBR1.cpp:10-115)
// and the chain rule to primitive gradients (BasicOperations.cpp:126-170).
template <int DIM, int NP>
__global__ void __launch_bounds__(Shape<DIM, NP>::THREADS, 4)
lift_kernel(const MeshDev m, const LiftArgs a, const PhysParams P, const __grid_constant__ OpTables T) {
    using S = Shape<DIM, NP>;
    constexpr int ND = S::ND, NF = S::NF, NFN = S::NFN, NFI = S::NFI;
    constexpr int PER_ELEM = 2 * NF * ND + DIM * NF * NFI;
    extern __shared__ double smem[];
    double *sT = smem;
    const double *sD = sT, *sW = sT + 4 * NP * NP;
    load_tables<NP>(T, sT, threadIdx.x, S::THREADS);

    const int el = threadIdx.x / ND;
    const int n = threadIdx.x - el * ND;
    const int e_raw = blockIdx.x * S::EPB + el;
    const bool active = e_raw < m.E;
    const int e = active ? e_raw : m.E - 1;
    double *sU = smem + S::TAB + el * PER_ELEM;
    double *sVe = sU + NF * ND;
    double *sS = sVe + NF * ND;
    const long long Ndof = m.Ndof;
    const long long gnode = (long long)e * ND + n;
    double st[NF], v[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        st[f] = __ldg(a.u + f * Ndof + gnode);
        sU[f * ND + n] = st[f];
    }
    conserv2entropy<DIM, double>(st, P, v);
#pragma unroll
    for (int f = 0; f < NF; ++f) sVe[f * ND + n] = v[f];
    const double *geo = m.geo + (long long)e * (DIM * DIM + 1);
    double adj[DIM][DIM];
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int q = 0; q < DIM; ++q) adj[r][q] = __ldg(geo + r * DIM + q);
    const double J = __ldg(geo + DIM * DIM);
    int c[3];
    node_coords<NP>(n, c);

    // face part first (its neighbour loads overlap the element part):
    // +1/(w0 J) * 1/2 (v_elem2 - v_elem1) * n_c on both sides
    const double aw = 1.0 / (sW[0] * J);
    __syncthreads();
    for (int it = n; it < NFI; it += ND) {
        const int lf = it / NFN, fa = it - lf * NFN;
        const int no = face_node<DIM, NP>(lf, fa);
        const int4 t = __ldg(m.nbr + (long long)e * (2 * DIM) + lf);
        const int nn = face_node<DIM, NP>(t.y, fa);
        const long long gn = (long long)t.x * ND + nn;
        double sn[NF], vn[NF], nor[DIM];
#pragma unroll
        for (int f = 0; f < NF; ++f) sn[f] = __ldg(a.u + f * Ndof + gn);
        conserv2entropy<DIM, double>(sn, P, vn);
#pragma unroll
        for (int q = 0; q < DIM; ++q) nor[q] = __ldg(m.fnor + (long long)t.z * DIM + q);
        const bool own_is_1 = (t.w == 0);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            const double vo = sVe[f * ND + no];
            const double jf = own_is_1 ? 0.5 * (vn[f] - vo) : 0.5 * (vo - vn[f]);
#pragma unroll
            for (int q = 0; q < DIM; ++q) sS[(q * NF + f) * NFI + it] = aw * (jf * nor[q]);
        }
    }

    // element part: g1(f, r) = sum_l D(pos_r, l) v_l along direction r
    double g1[NF][DIM];
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int r = 0; r < DIM; ++r) g1[f][r] = 0.0;
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        int base, stride;
        line_base<DIM, NP>(r, line_index<DIM, NP>(r, c), base, stride);
#pragma unroll
        for (int l = 0; l < NP; ++l) {
            const double dl = sD[c[r] * NP + l];
#pragma unroll
            for (int f = 0; f < NF; ++f) g1[f][r] += sVe[f * ND + base + l * stride] * dl;
        }
    }
    // grad_mat2 = grad_mat1 * adj, times 1/J (LiftingBR1.cpp:205-206)
    const double mJ = 1.0 / J;
    double g[DIM][NF];
#pragma unroll
    for (int q = 0; q < DIM; ++q)
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            double s = 0.0;
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
#pragma unroll
            for (int q = 0; q < DIM; ++q)
#pragma unroll
                for (int f = 0; f < NF; ++f) g[q][f] += sS[(q * NF + f) * NFI + it];
        }
    }
    if (!active) return;
#pragma unroll
    for (int q = 0; q < DIM; ++q) {
        entropygrad2primgrad<DIM, double>(st, P, g[q]);
#pragma unroll
        for (int f = 0; f < NF; ++f) a.grad[(q * NF + f) * Ndof + gnode] = g[q][f];
    }
}

template <int DIM, int NP, bool NS>
size_t rhs_smem() {
    using S = Shape<DIM, NP>;
    return sizeof(double) * (S::TAB + (size_t)S::EPB * RhsLayout<DIM, NP, NS>::PER_ELEM);
}
template <int DIM, int NP>
size_t lift_smem() {
    using S = Shape<DIM, NP>;
    constexpr int PER_ELEM = 2 * S::NF * S::ND + DIM * S::NF * S::NFI;
    return sizeof(double) * (S::TAB + (size_t)S::EPB * PER_ELEM);
}

template <int DIM, int NP>
cudaError_t rhs_launch_t(bool ns, const MeshDev &m, const RhsArgs &a, const PhysParams &P,
                         const OpTables &T, cudaStream_t s) {
    using S = Shape<DIM, NP>;
    const int grid = (m.E + S::EPB - 1) / S::EPB;
    if (ns) {
        const size_t sm = rhs_smem<DIM, NP, true>();
        cudaError_t err = cudaFuncSetAttribute(rhs_kernel<DIM, NP, true>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (err != cudaSuccess) return err;
        rhs_kernel<DIM, NP, true><<<grid, S::THREADS, sm, s>>>(m, a, P, T);
    } else {
        const size_t sm = rhs_smem<DIM, NP, false>();
        cudaError_t err = cudaFuncSetAttribute(rhs_kernel<DIM, NP, false>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (err != cudaSuccess) return err;
        rhs_kernel<DIM, NP, false><<<grid, S::THREADS, sm, s>>>(m, a, P, T);
    }
    return cudaGetLastError();
}
template <int DIM, int NP>
cudaError_t lift_launch_t(const MeshDev &m, const LiftArgs &a, const PhysParams &P,
                          const OpTables &T, cudaStream_t s) {
    using S = Shape<DIM, NP>;
    const int grid = (m.E + S::EPB - 1) / S::EPB;
    const size_t sm = lift_smem<DIM, NP>();
    cudaError_t err = cudaFuncSetAttribute(lift_kernel<DIM, NP>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (err != cudaSuccess) return err;
    lift_kernel<DIM, NP><<<grid, S::THREADS, sm, s>>>(m, a, P, T);
    return cudaGetLastError();
}

}   // namespace

bool order_supported(int dim, int order) {
    return (dim == 2 || dim == 3) && order >= 1 && order <= 5;
}

#define PRANDTL_DISPATCH(DIMV, FN, ...)                                  \
    switch (order) {                                                     \
    case 1: return FN<DIMV, 2>(__VA_ARGS__);                             \
    case 2: return FN<DIMV, 3>(__VA_ARGS__);                             \
    case 3: return FN<DIMV, 4>(__VA_ARGS__);                             \
    case 4: return FN<DIMV, 5>(__VA_ARGS__);                             \
    case 5: return FN<DIMV, 6>(__VA_ARGS__);                             \
    default: return cudaErrorInvalidValue;                               \
    }

cudaError_t launch_rhs(int dim, int order, bool ns, const MeshDev &m, const RhsArgs &a,
                       const PhysParams &P, const OpTables &T, cudaStream_t s) {
    if (m.E <= 0) return cudaSuccess;
    if (dim == 2) { PRANDTL_DISPATCH(2, rhs_launch_t, ns, m, a, P, T, s) }
    if (dim == 3) { PRANDTL_DISPATCH(3, rhs_launch_t, ns, m, a, P, T, s) }
    return cudaErrorInvalidValue;
}

cudaError_t launch_lift(int dim, int order, const MeshDev &m, const LiftArgs &a,
                        const PhysParams &P, const OpTables &T, cudaStream_t s) {
    if (m.E <= 0) return cudaSuccess;
    if (dim == 2) { PRANDTL_DISPATCH(2, lift_launch_t, m, a, P, T, s) }
    if (dim == 3) { PRANDTL_DISPATCH(3, lift_launch_t, m, a, P, T, s) }
    return cudaErrorInvalidValue;
}

}   // namespace prandtl
