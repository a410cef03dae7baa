// k_fine.cu -- matrix-free fine-level operator: Gauss-Seidel colour sweeps,
// residuals (FP32 with fused per-case norms, and the refined FP64-solution form),
// the unit macro-strain right-hand side, and FP64 helpers of the refined mode.
//
// Reference behaviour restated (homo3d grid.cu):
//   gs_relaxation_otf_kernel (grid.cu:323-551): for each vertex of one colour,
//     sum over its 8 elements of (1e-9 + rho_e) * Ke[own rows][other nodes] * u,
//     then a 3x3 block Gauss-Seidel step on the components (x, then y, then z);
//     neighbours at the pinned origin count as zero; the origin stays zero.
//   update_residual_otf_kernel_1 (grid.cu:1277-1461): r = f - K(rho) u, r = 0 at
//     the pinned origin.
//   enforce_unit_macro_strain_kernel (grid.cu:1818-1919): f_i = K(rho) chi0_i.
//
// B200 design.  The element loop is reorganised per neighbour: for each of the 26
// neighbours the 3x3 coupling block sum_e rho_e Ke[a_e][b_e] is formed once (Ke
// entries are compile-time offsets into the kernel-parameter bank, so they are
// FFMA operands) and applied to the load cases, two cases at a time as packed
// FP32x2 lane pairs.  The colour sweep serves each vertex by one thread with all
// six cases (the block is built once per vertex; the sweep is bound by instruction
// issue, 128 registers, 4 CTAs/SM); the residuals serve it by three threads with
// two cases each in adjacent CTAs (fewer registers: the residual also writes r and
// reduces the norms), where the densities and neighbour rows the three share hit
// L1/L2, and all eight colours of a residual go in one launch (seven in a V-cycle,
// where the sweep's last colour launch writes colour 7's residual).  The operator is
// applied in difference form, sum_{d != 0} A_d (u_{v+d} - u_v), and the
// Gauss-Seidel step as u += D^-1 r with
// the components in the reference's order: the same iteration in exact
// arithmetic, and in FP32 it keeps rigid translations exact (see fine_apply).
#include <type_traits>

#include "h3d_internal.cuh"

namespace h3d {

constexpr int CPT = 2;            // load cases per thread of the FP32 residual (three threads per vertex)
constexpr int RES_MINB = 6;       // its CTAs per SM
constexpr int CPT64 = 2;          // load cases per thread of the FP64-solution residual
constexpr int MINB64 = 4;         // its CTAs per SM
constexpr int FBS = 128;          // threads per CTA

struct FineArgs {
    const float *__restrict__ rho;
    float *u;
    const float *__restrict__ f;
    float *r;
    int n[3];
    int h[3];
    long long nv;  // vertices
    long long P;   // vertices per colour plane
    float w;
    FastDiv dh0, dh1;  // division by h[0], h[1]
};

__device__ __forceinline__ void axis_nbrs(int i, int p, int h, int &im, int &ip) {
    if (p) { im = i; ip = (i + 1 == h) ? 0 : i + 1; }
    else { im = (i == 0) ? h - 1 : i - 1; ip = i; }
}

// (i, j, l) of index p (< 2^32) of a colour plane
__device__ __forceinline__ void plane_coords(const FineArgs &a, long long p, int &i, int &j, int &l) {
    const unsigned q = (unsigned)p;
    const unsigned t = a.dh0.div(q);
    i = (int)(q - t * (unsigned)a.h[0]);
    const unsigned z = a.dh1.div(t);
    j = (int)(t - z * (unsigned)a.h[1]);
    l = (int)z;
}

// first element (bit pattern w = ex | ey<<1 | ez<<2 of the element's offset from
// the vertex) shared by the vertex and its neighbour d, -1 if none
__host__ __device__ constexpr int first_shared(int d) {
    for (int w = 0; w < 8; ++w) {
        const int bx = 1 - (w & 1) + d % 3 - 1, by = 1 - ((w >> 1) & 1) + d / 3 % 3 - 1, bz = 1 - (w >> 2) + d / 9 - 1;
        if (bx >= 0 && bx <= 1 && by >= 0 && by <= 1 && bz >= 0 && bz <= 1) return w;
    }
    return -1;
}

// geometry of one colour-K vertex: its element densities and the offsets of its
// neighbours inside a colour plane (32-bit: a field plane holds < 2^31 vertices)
template <int KC>
struct VertexGeo {
    const int K;  // the colour: KC, or the run-time colour kr when KC < 0
    float rw[8];
    unsigned X[3], Y[3], Z[3];  // plane offsets of the neighbour rows: i, h0*j, h0*h1*l
    __device__ __forceinline__ VertexGeo(const FineArgs &a, long long p, int kr = KC) : K(KC >= 0 ? KC : kr) {
        const int px = (K & 1) ^ 1, py = ((K >> 1) & 1) ^ 1, pz = ((K >> 2) & 1) ^ 1;
        int i, j, l;
        plane_coords(a, p, i, j, l);
        const int x = 2 * i + px, y = 2 * j + py, z = 2 * l + pz;
        const int xe0 = x == 0 ? a.n[0] - 1 : x - 1;
        const int ye0 = y == 0 ? a.n[1] - 1 : y - 1;
        const int ze0 = z == 0 ? a.n[2] - 1 : z - 1;
        const unsigned n0 = (unsigned)a.n[0], n01 = (unsigned)a.n[0] * (unsigned)a.n[1];
#pragma unroll
        for (int w = 0; w < 8; ++w) {
            const unsigned ex = (w & 1) ? x : xe0, ey = ((w >> 1) & 1) ? y : ye0, ez = (w >> 2) ? z : ze0;
            rw[w] = RHO_PENAL_MIN + __ldg(&a.rho[ex + n0 * ey + n01 * ez]);
        }
        int ii[3], jj[3], ll[3];
        axis_nbrs(i, px, a.h[0], ii[0], ii[2]);
        axis_nbrs(j, py, a.h[1], jj[0], jj[2]);
        axis_nbrs(l, pz, a.h[2], ll[0], ll[2]);
        ii[1] = i; jj[1] = j; ll[1] = l;
        const unsigned h0 = (unsigned)a.h[0], h01 = (unsigned)a.h[0] * (unsigned)a.h[1];
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            X[t] = (unsigned)ii[t];
            Y[t] = h0 * (unsigned)jj[t];
            Z[t] = h01 * (unsigned)ll[t];
        }
    }
    // coupling block of neighbour d (compile-time d after unrolling):
    // sum over the shared elements e of rho_e Ke[a_e][b_e].  The shared elements
    // are mirror images of the first one across the axes where they differ, and
    // an isotropic Ke is invariant under the mirrors up to the sign of the
    // components mirrored, so entry (r,c) = Ke[a_0][b_0](r,c) * sum_e +-rho_e with
    // the sign set by whether r and c lie on the mirrored axes: four signed
    // density sums per block (signed_sums) instead of 9 FMAs per shared element.
    template <typename T>
    __device__ __forceinline__ void block_t(const T *kk, int d, T A[9]) const {
        const int dx = d % 3 - 1, dy = d / 3 % 3 - 1, dz = d / 9 - 1;
        const int w0 = first_shared(d);
        T cs[8];  // cs[m]: signed sum for the axis mask m = (1<<r) ^ (1<<c); m in {0, 3, 5, 6}
        signed_sums<T>(dx, dy, dz, w0, cs);
        const int an = 7 - w0;
        const int bn = (1 - (w0 & 1) + dx) + 2 * (1 - ((w0 >> 1) & 1) + dy) + 4 * (1 - (w0 >> 2) + dz);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) A[3 * r + c] = kk[(3 * an + r) * 24 + 3 * bn + c] * cs[(1 << r) ^ (1 << c)];
    }
    // The signed sums over the shared elements, folded one free axis at a time:
    // element pairs along the first free axis (their sum and difference), then
    // pairs of those along the next.  Along a free axis a the element with bit a
    // set enters with a minus sign when a lies in the mask m, so the sign of an
    // element is the parity of the mask axes on which it differs from w0.
    // 0 / 2 / 8 / 16 additions for a corner / edge / face neighbour / the vertex
    // itself, where the element-by-element sums took 4 / 8 / 16 / 32.
    template <typename T>
    __device__ __forceinline__ T rwv(int w) const { return (T)rw[w]; }
    template <typename T>
    __device__ __forceinline__ void signed_sums(int dx, int dy, int dz, int w0, T cs[8]) const {
        int fa[3], nf = 0;  // the free axes (offset 0), ascending
        if (dx == 0) fa[nf++] = 0;
        if (dy == 0) fa[nf++] = 1;
        if (dz == 0) fa[nf++] = 2;
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            if (m != 0 && m != 3 && m != 5 && m != 6) { cs[m] = T(0); continue; }
            if (nf == 0) {
                cs[m] = rwv<T>(w0);
            } else {
                const int a = fa[0];
                // level 1: pairs (w, w | a) for the 2^(nf-1) settings of the other free axes
                T v[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (k >= (1 << (nf - 1))) continue;
                    int w = w0;
                    if (nf > 1 && (k & 1)) w |= 1 << fa[1];
                    if (nf > 2 && (k & 2)) w |= 1 << fa[2];
                    v[k] = ((m >> a) & 1) ? rwv<T>(w) - rwv<T>(w | (1 << a)) : rwv<T>(w) + rwv<T>(w | (1 << a));
                }
                if (nf >= 2) {  // level 2: along fa[1]
                    const bool mb = (m >> fa[1]) & 1;
                    v[0] = mb ? v[0] - v[1] : v[0] + v[1];
                    if (nf == 3) v[2] = mb ? v[2] - v[3] : v[2] + v[3];
                }
                if (nf == 3) {  // level 3: along fa[2]
                    const bool mc = (m >> fa[2]) & 1;
                    v[0] = mc ? v[0] - v[2] : v[0] + v[2];
                }
                cs[m] = v[0];
            }
        }
    }
    __device__ __forceinline__ void block(const KeMat &ke, int d, float A[9]) const { block_t<float>(ke.k, d, A); }
    // the coupling block in FP64 from an FP64 element matrix (the exact refinement
    // residual): the same signed sums with FP64 densities and products
    __device__ __forceinline__ void block64(const KeMat64 &ke, int d, double A[9]) const {
        block_t<double>(ke.k, d, A);
    }
    // index of neighbour d in its colour plane set, and whether it is the pinned origin
    __device__ __forceinline__ unsigned nbr(const FineArgs &a, int d, int &Kn, bool &pinned) const {
        const int dx = d % 3 - 1, dy = d / 3 % 3 - 1, dz = d / 9 - 1;
        Kn = K ^ ((dx & 1) | ((dy & 1) << 1) | ((dz & 1) << 2));
        const unsigned off = X[dx + 1] + Y[dy + 1] + Z[dz + 1];
        pinned = (Kn == 7) && (off == 0u);
        return (unsigned)Kn * (unsigned)a.P + off;
    }
};

// acc[3c+r] (c < CPT, cases cb..cb+CPT-1) = (K u)_v in difference form,
// sum over the 26 neighbours of A_d (u_{v+d} - u_v), with u at the pinned origin
// counted as 0.  Equal to sum_d A_d u_{v+d} in exact arithmetic (the blocks of a
// row sum to zero), and exact for rigid translations in FP32 too, so the FP32
// operator agrees with the FP64 difference-form residual of the refined mode on
// the near-null translation mode of the pinned problem.
template <int K, int C>
__device__ __forceinline__ void fine_apply(const FineArgs &a, const KeMat &ke, const VertexGeo<K> &g, int cb,
                                           const float uv[3 * C], float acc[3 * C]) {
    constexpr int NP = C / 2;  // case pairs per thread
    constexpr int NS = C % 2;  // an odd last case, on scalar lanes
    // lane pair (case cb+2j, case cb+2j+1) of each component: Blackwell's packed
    // FP32x2 add and FMA do both cases in one instruction with the rounding of the
    // scalar forms, so the sums are the same as the scalar per-case loop (the odd
    // case runs the scalar forms in the same order)
    float2 acc2[3 * NP + 1], nuv2[3 * NP + 1];
    float acc1[3 * NS + 1], nuv1[3 * NS + 1];
#pragma unroll
    for (int j = 0; j < NP; ++j)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            acc2[3 * j + m] = make_float2(0.f, 0.f);
            nuv2[3 * j + m] = make_float2(-uv[6 * j + m], -uv[6 * j + 3 + m]);
        }
#pragma unroll
    for (int m = 0; m < 3 * NS; ++m) {
        acc1[m] = 0.f;
        nuv1[m] = -uv[6 * NP + m];
    }
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        if (d == 13) continue;
        int Kn;
        bool pinned;
        const unsigned nid = g.nbr(a, d, Kn, pinned);
        float A[9];
        g.block(ke, d, A);
        const float *up = a.u + fidx(3 * cb, nid);  // planes 3cb.. of the neighbour, FVB apart
#pragma unroll
        for (int j = 0; j < NP; ++j) {
            float2 dd[3];
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                const float2 un = pinned ? make_float2(0.f, 0.f)
                                         : make_float2(__ldg(up + (6 * j + m) * FVB), __ldg(up + (6 * j + 3 + m) * FVB));
                dd[m] = __fadd2_rn(un, nuv2[3 * j + m]);
            }
#pragma unroll
            for (int r = 0; r < 3; ++r)
                acc2[3 * j + r] = __ffma2_rn(make_float2(A[3 * r], A[3 * r]), dd[0],
                                             __ffma2_rn(make_float2(A[3 * r + 1], A[3 * r + 1]), dd[1],
                                                        __ffma2_rn(make_float2(A[3 * r + 2], A[3 * r + 2]), dd[2],
                                                                   acc2[3 * j + r])));
        }
        if (NS) {
            float dd[3];
#pragma unroll
            for (int m = 0; m < 3; ++m) dd[m] = __fadd_rn(pinned ? 0.f : __ldg(up + (6 * NP + m) * FVB), nuv1[m]);
#pragma unroll
            for (int r = 0; r < 3; ++r)
                acc1[r] = __fmaf_rn(A[3 * r], dd[0], __fmaf_rn(A[3 * r + 1], dd[1], __fmaf_rn(A[3 * r + 2], dd[2], acc1[r])));
        }
    }
#pragma unroll
    for (int j = 0; j < NP; ++j)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            acc[6 * j + m] = acc2[3 * j + m].x;
            acc[6 * j + 3 + m] = acc2[3 * j + m].y;
        }
#pragma unroll
    for (int m = 0; m < 3 * NS; ++m) acc[6 * NP + m] = acc1[m];
}

// thread -> (vertex p in the colour plane, first case cb) for C cases per thread;
// the NCASE / C case groups of a vertex block are adjacent CTAs
// vertex block are adjacent CTAs
template <int C>
__device__ __forceinline__ void thread_task(long long &p, int &cb, unsigned bid) {
    constexpr int NG = NCASE / C;
    cb = (int)(bid % NG) * C;
    p = (long long)(bid / NG) * blockDim.x + threadIdx.x;
}

// one vertex of the colour sweep; RES (the last colour of a sweep) also writes
// the residual of the updated vertex, whose neighbours (all of other colours) are
// final: with acc = sum_d A_d (u_{v+d} - u_v) taken before the update and the
// blocks of a row summing to zero, f - K u after u_v += e is (f - acc) - A_0 e,
// e the change actually stored.  nrm[c] gathers the weighted squared residual.
template <int K, int C, bool RES>
__device__ __forceinline__ void fine_gs_vertex(const FineArgs &a, const KeMat &ke, long long p, int cb,
                                               double nrm[C]) {
    const long long me = (long long)K * a.P + p;
    if (K == 7 && p == 0) {  // the pinned origin (grid.cu:445-447, 545)
#pragma unroll
        for (int q = 0; q < 3 * C; ++q) {
            a.u[fidx(3 * cb + q, me)] = 0.f;
            if (RES) a.r[fidx(3 * cb + q, me)] = 0.f;
        }
        return;
    }
    const VertexGeo<K> g(a, p);
    float uv[3 * C];
#pragma unroll
    for (int q = 0; q < 3 * C; ++q) uv[q] = a.u[fidx(3 * cb + q, me)];
    float acc[3 * C];
    fine_apply<K, C>(a, ke, g, cb, uv, acc);
    float ks[9];
    g.block(ke, 13, ks);
    const float w = a.w;
    double mult = 0;
    if (RES) {
        constexpr int px = (K & 1) ^ 1, py = ((K >> 1) & 1) ^ 1, pz = ((K >> 2) & 1) ^ 1;
        int i, j, l;
        plane_coords(a, p, i, j, l);
        mult = (double)(axis_mult(2 * i + px, a.n[0]) * axis_mult(2 * j + py, a.n[1]) * axis_mult(2 * l + pz, a.n[2]));
    }
    // the reference's component-wise block Gauss-Seidel step (x, then y, then z,
    // each with the relaxed values of the earlier components) written as an
    // update of u by the residual r = f - K u
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const long long o = fidx(3 * (cb + c), me);
        const float r0 = a.f[o] - acc[3 * c], r1 = a.f[o + FVB] - acc[3 * c + 1], r2 = a.f[o + 2 * FVB] - acc[3 * c + 2];
        const float d0 = w * r0 / ks[0];
        const float d1 = w * (r1 - ks[3] * d0) / ks[4];
        const float d2 = w * (r2 - ks[6] * d0 - ks[7] * d1) / ks[8];
        const float n0 = uv[3 * c] + d0, n1 = uv[3 * c + 1] + d1, n2 = uv[3 * c + 2] + d2;
        a.u[o] = n0;
        a.u[o + FVB] = n1;
        a.u[o + 2 * FVB] = n2;
        if (RES) {
            const float e0 = n0 - uv[3 * c], e1 = n1 - uv[3 * c + 1], e2 = n2 - uv[3 * c + 2];
            const float q0 = r0 - fmaf(ks[2], e2, fmaf(ks[1], e1, ks[0] * e0));
            const float q1 = r1 - fmaf(ks[5], e2, fmaf(ks[4], e1, ks[3] * e0));
            const float q2 = r2 - fmaf(ks[8], e2, fmaf(ks[7], e1, ks[6] * e0));
            a.r[o] = q0;
            a.r[o + FVB] = q1;
            a.r[o + 2 * FVB] = q2;
            nrm[c] += mult * ((double)q0 * q0 + (double)q1 * q1 + (double)q2 * q2);
        }
    }
}

// RES: the per-CTA norm partials go to the rows the residual of colour 7 would
// write (row 7 * (CTAs per colour of the residual) + CTA of the colour, one row
// per group of CPT cases, zeros for the other cases).  bid / nblk: the CTA's index
// and the CTA count of the design's launch (blockIdx.x / gridDim.x, or the slice
// of a batched launch, k_fine_gs_batch)
template <int K, int C, bool RES>
__device__ __forceinline__ void fine_gs_block(const FineArgs &a, const KeMat &ke, double *partial, unsigned bid,
                                              unsigned nblk) {
    long long p;
    int cb;
    thread_task<C>(p, cb, bid);
    double nrm[C];
#pragma unroll
    for (int c = 0; c < C; ++c) nrm[c] = 0;
    if (!RES) {
        if (p < a.P) fine_gs_vertex<K, C, false>(a, ke, p, cb, nrm);
        return;
    }
    static_assert(!RES || (K == 7 && C % CPT == 0), "the fused residual is the last colour's");
    if (p < a.P) fine_gs_vertex<K, C, RES>(a, ke, p, cb, nrm);
    __shared__ double sm[C][FBS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const double v = warp_sum(nrm[c]);
        if (lane == 0) sm[c][wid] = v;
    }
    __syncthreads();
    constexpr int NG = NCASE / C, NGR = NCASE / CPT;  // case groups of this launch / of the residual
    const long long pb = bid / NG, npb = nblk / NG;  // vertex block, vertex blocks
    if (threadIdx.x < (C / CPT) * NCASE) {
        const int gl = threadIdx.x / NCASE, q = threadIdx.x % NCASE;
        const int g = cb / CPT + gl;  // the residual's case group of this row
        double v = 0;
        if (q >= g * CPT && q < (g + 1) * CPT)
#pragma unroll
            for (int w = 0; w < FBS / 32; ++w) v += sm[q - cb][w];
        partial[((7 * npb + pb) * NGR + g) * NCASE + q] = v;
    }
}

template <int K, int C, int MINB, bool RES>
__global__ void __launch_bounds__(FBS, MINB) k_fine_gs(FineArgs a, const __grid_constant__ KeMat ke,
                                                    double *partial) {
    fine_gs_block<K, C, RES>(a, ke, partial, blockIdx.x, gridDim.x);
}

template <int KC>
__device__ __forceinline__ void fine_residual_vertex(const FineArgs &a, const KeMat &ke, long long p, int cb,
                                                     double nrm[CPT], int kr = KC) {
    const int K = KC >= 0 ? KC : kr;
    const long long me = (long long)K * a.P + p;
    if (K == 7 && p == 0) {
#pragma unroll
        for (int q = 0; q < 3 * CPT; ++q) a.r[fidx(3 * cb + q, me)] = 0.f;
        return;
    }
    const VertexGeo<KC> g(a, p, K);
    float uv[3 * CPT];
#pragma unroll
    for (int q = 0; q < 3 * CPT; ++q) uv[q] = __ldg(a.u + fidx(3 * cb + q, me));
    float acc[3 * CPT];
    fine_apply<KC, CPT>(a, ke, g, cb, uv, acc);
    const int px = (K & 1) ^ 1, py = ((K >> 1) & 1) ^ 1, pz = ((K >> 2) & 1) ^ 1;
    int i, j, l;
    plane_coords(a, p, i, j, l);
    const double mult = (double)(axis_mult(2 * i + px, a.n[0]) * axis_mult(2 * j + py, a.n[1]) *
                                 axis_mult(2 * l + pz, a.n[2]));
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        double s2 = 0;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            const long long o = fidx(3 * (cb + c) + m, me);
            const float rv = a.f[o] - acc[3 * c + m];
            a.r[o] = rv;
            s2 += (double)rv * rv;
        }
        nrm[c] += mult * s2;
    }
}

// The residual has no order between the colours, so all eight run in one launch
// with the colour the block index modulo the colour count (8, or 7 when the sweep
// before it wrote colour 7's residual): the eight CTAs of one
// vertex block cover a 2x2x2 neighbourhood of the grid and read each other's rows
// while they are in L2, where one launch per colour would stream the whole u
// field from HBM once per colour.  The colour is a run-time value of one code
// body (VertexGeo<-1>): eight compile-time colour bodies resident on an SM at
// once thrash the instruction cache (2.5x slower at 256^3), while the run-time
// colour costs a few integer operations per neighbour.  One thread per vertex
// (six cases) is slower here too: 3.55 against 3.11 ms per 256^3 residual.  The
// per-CTA norm partials of the CTA's two cases go to row colour * (CTAs per
// colour) + CTA of the colour, zeros for the other cases, as with one launch per
// colour, so the norms are summed in the same order.
template <int C>
__device__ __forceinline__ void colour_task(long long &p, int &cb, int &K, unsigned &bx, unsigned bid,
                                            unsigned ncol = 8) {
    constexpr int NG = NCASE / C;
    K = (int)(bid % ncol);
    bx = bid / ncol;
    cb = (int)(bx % NG) * C;
    p = (long long)(bx / NG) * blockDim.x + threadIdx.x;
}

template <unsigned NCOL>  // colours 0 .. NCOL-1 (8, or 7 after a sweep that did colour 7's)
__device__ __forceinline__ void fine_residual_block(const FineArgs &a, const KeMat &ke, double *partial, unsigned bid,
                                                    unsigned nblk) {
    constexpr unsigned ncol = NCOL;
    long long p;
    int cb, K;
    unsigned bx;
    colour_task<CPT>(p, cb, K, bx, bid, ncol);
    double nrm[CPT] = {};
    if (p < a.P) fine_residual_vertex<-1>(a, ke, p, cb, nrm, K);
    if (!partial) return;
    __shared__ double sm[CPT][FBS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        const double v = warp_sum(nrm[c]);
        if (lane == 0) sm[c][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < NCASE) {
        const int q = threadIdx.x;
        double v = 0;
        if (q >= cb && q < cb + CPT)
#pragma unroll
            for (int w = 0; w < FBS / 32; ++w) v += sm[q - cb][w];
        partial[((long long)K * (nblk / ncol) + bx) * NCASE + q] = v;
    }
}

template <unsigned NCOL>
__global__ void __launch_bounds__(FBS, RES_MINB) k_fine_residual(FineArgs a, const __grid_constant__ KeMat ke,
                                                       double *partial) {
    fine_residual_block<NCOL>(a, ke, partial, blockIdx.x, gridDim.x);
}

// ---- refined precision: residual of an FP64 solution ----------------------------
// K u at vertex v equals sum_{d != 0} A_d (u_{v+d} - u_v), because the assembled
// blocks of a row sum to zero (Ke annihilates rigid translations).  The
// differences are taken in FP64 and are O(1) where u itself is O(N), so the
// residual floor no longer grows with the grid size.  The pinned origin enters as
// an ordinary neighbour: its value is held fixed by the correction sweeps, so a
// nonzero value only translates the solution.  EXACT accumulates the products in
// FP64 too (the FP32-product form floors near 1e-6 of ||f||, independent of N).
template <int KC, bool EXACT, int C64 = CPT64>
__device__ __forceinline__ void fine_residual64_vertex(const FineArgs &a, const KeMat &ke, const KeMat64 &ke64,
                                                       const double *__restrict__ u64, long long p, int cb,
                                                       int kr = KC) {
    const int K = KC >= 0 ? KC : kr;
    const long long me = (long long)K * a.P + p;
    if (K == 7 && p == 0) {
#pragma unroll
        for (int q = 0; q < 3 * C64; ++q) a.r[fidx(3 * cb + q, me)] = 0.f;
        return;
    }
    const VertexGeo<KC> g(a, p, K);
    const double *uvp = u64 + fidx(3 * cb, me);
    double uv[3 * C64];
#pragma unroll
    for (int q = 0; q < 3 * C64; ++q) uv[q] = __ldg(uvp + q * FVB);
    using Acc = typename std::conditional<EXACT, double, float>::type;
    Acc acc[3 * C64];
#pragma unroll
    for (int q = 0; q < 3 * C64; ++q) acc[q] = 0;
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        if (d == 13) continue;
        int Kn;
        bool pinned;
        const unsigned nid = g.nbr(a, d, Kn, pinned);
        // EXACT: the block in FP64 (FP64 element matrix and densities, FP64
        // products): no per-entry FP32-to-FP64 conversions, which run on the narrow
        // conversion pipe; otherwise the FP32 block of the V-cycle operator
        Acc A[9];
        if (EXACT) {
            double A64[9];
            g.block64(ke64, d, A64);
#pragma unroll
            for (int k = 0; k < 9; ++k) A[k] = (Acc)A64[k];
        } else {
            float A32[9];
            g.block(ke, d, A32);
#pragma unroll
            for (int k = 0; k < 9; ++k) A[k] = (Acc)A32[k];
        }
        const double *up = u64 + fidx(3 * cb, nid);  // planes 3cb.. of the neighbour, FVB apart
#pragma unroll
        for (int c = 0; c < C64; ++c) {
            const Acc d0 = (Acc)(__ldg(up + (3 * c) * FVB) - uv[3 * c]);
            const Acc d1 = (Acc)(__ldg(up + (3 * c + 1) * FVB) - uv[3 * c + 1]);
            const Acc d2 = (Acc)(__ldg(up + (3 * c + 2) * FVB) - uv[3 * c + 2]);
            acc[3 * c + 0] = fma(A[0], d0, fma(A[1], d1, fma(A[2], d2, acc[3 * c + 0])));
            acc[3 * c + 1] = fma(A[3], d0, fma(A[4], d1, fma(A[5], d2, acc[3 * c + 1])));
            acc[3 * c + 2] = fma(A[6], d0, fma(A[7], d1, fma(A[8], d2, acc[3 * c + 2])));
        }
    }
#pragma unroll
    for (int q = 0; q < 3 * C64; ++q) {
        const long long o = fidx(3 * cb + q, me);
        a.r[o] = (float)((Acc)a.f[o] - acc[q]);
    }
}

// C64 load cases per thread (NCASE / C64 threads per vertex), MB CTAs per SM
template <bool EXACT, int C64 = CPT64, int MB = MINB64>
__global__ void __launch_bounds__(FBS, MB) k_fine_residual64(FineArgs a, const __grid_constant__ KeMat ke,
                                                         const __grid_constant__ KeMat64 ke64,
                                                         const double *__restrict__ u64) {
    long long p;
    int cb, K;
    unsigned bx;
    colour_task<C64>(p, cb, K, bx, blockIdx.x);  // all colours in one launch, colour-minor
    if (p >= a.P) return;
    fine_residual64_vertex<-1, EXACT, C64>(a, ke, ke64, u64, p, cb, K);
}

// f(case c) = sum_w (1e-9 + rho_w) * (Ke chi0_c)[rows of the vertex's local node in element w]
__global__ void __launch_bounds__(256) k_rhs(Planes P, const float *__restrict__ rho, float *f,
                                             const __grid_constant__ RhsTab g) {
    const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v >= P.nv) return;
    const int k = color_of_index(P, v);
    int x, y, z;
    vpos(P, k, v - P.base[k], x, y, z);
    const int n0 = P.n[0], n1 = P.n[1], n2 = P.n[2];
    const int xe0 = x == 0 ? n0 - 1 : x - 1, ye0 = y == 0 ? n1 - 1 : y - 1, ze0 = z == 0 ? n2 - 1 : z - 1;
    float acc[NF];
#pragma unroll
    for (int q = 0; q < NF; ++q) acc[q] = 0.f;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        const int ex = (w & 1) ? x : xe0, ey = ((w >> 1) & 1) ? y : ye0, ez = (w >> 2) ? z : ze0;
        const float rp = RHO_PENAL_MIN + __ldg(&rho[ex + (long long)n0 * (ey + (long long)n1 * ez)]);
        const int an = 7 - w;
#pragma unroll
        for (int c = 0; c < NCASE; ++c)
#pragma unroll
            for (int m = 0; m < 3; ++m) acc[3 * c + m] = fmaf(rp, g.g[c][3 * an + m], acc[3 * c + m]);
    }
#pragma unroll
    for (int q = 0; q < NF; ++q) f[fidx(q, v)] = acc[q];
}

static FineArgs make_args(const Level &L, const float *rho) {
    FineArgs a;
    a.rho = rho;
    a.u = L.u;
    a.f = L.f;
    a.r = L.r;
    for (int d = 0; d < 3; ++d) { a.n[d] = L.P.n[d]; a.h[d] = L.P.n[d] / 2; }
    a.nv = L.P.nv;
    a.P = L.P.nv / 8;
    a.w = 1.f;
    a.dh0 = FastDiv((unsigned)a.h[0]);
    a.dh1 = FastDiv((unsigned)a.h[1]);
    return a;
}

static unsigned task_blocks(const FineArgs &a, int cpt) { return (unsigned)(((a.P + FBS - 1) / FBS) * (NCASE / cpt)); }

int fine_residual_blocks(const Level &L) { return (int)(((L.P.nv / 8 + FBS - 1) / FBS) * (NCASE / CPT) * 8); }

// the colour sweep in launch shape v: 0 = one thread per vertex with all six
// cases (4 CTAs/SM), 1 = three threads per vertex with two cases each (5 CTAs/SM),
// 2 = three cases per thread (two threads per vertex, one case pair and one scalar
// case) at 5 CTAs/SM, 3 = two cases per thread at 6 CTAs/SM (fewer registers);
// all give the same result to the last bit
template <int C, int MINB>
static void fine_gs_sweep(const FineArgs &a, const KeMat &ke, cudaStream_t s) {
    const unsigned nb = task_blocks(a, C);
    k_fine_gs<0, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    k_fine_gs<1, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    k_fine_gs<2, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    k_fine_gs<3, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    k_fine_gs<4, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    k_fine_gs<5, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    k_fine_gs<6, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    k_fine_gs<7, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
}

void launch_fine_gs(const Level &L, const float *rho, const KeMat &ke, float w, cudaStream_t s) {
    FineArgs a = make_args(L, rho);
    a.w = w;
    switch (L.gs_shape) {
    case 1: fine_gs_sweep<2, 5>(a, ke, s); break;
    case 2: fine_gs_sweep<3, 5>(a, ke, s); break;
    case 3: fine_gs_sweep<2, 6>(a, ke, s); break;
    default: fine_gs_sweep<6, 4>(a, ke, s); break;
    }
}

// a sweep followed by the residual (the down leg of a V-cycle): the last colour's
// launch writes its own residual and norm partials, the residual launch covers
// the other seven colours
template <int C, int MINB>
static void fine_gs_sweep_res(const FineArgs &a, const KeMat &ke, double *partial, cudaStream_t s) {
    const unsigned nb = task_blocks(a, C);
    k_fine_gs<0, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    k_fine_gs<1, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    k_fine_gs<2, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    k_fine_gs<3, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    k_fine_gs<4, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    k_fine_gs<5, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    k_fine_gs<6, C, MINB, false><<<nb, FBS, 0, s>>>(a, ke, nullptr);
    // the last colour writes its residual with the norm partials of the residual's
    // case pairs: an odd case count per thread takes the six-case kernel for it
    constexpr int CR = (C % CPT == 0) ? C : 6, MR = (C % CPT == 0) ? MINB : 4;
    k_fine_gs<7, CR, MR, true><<<task_blocks(a, CR), FBS, 0, s>>>(a, ke, partial);
    k_fine_residual<7><<<task_blocks(a, CPT) * 7, FBS, 0, s>>>(a, ke, partial);
}

void launch_fine_gs_residual(const Level &L, const float *rho, const KeMat &ke, float w, double *norm_partial,
                             cudaStream_t s) {
    FineArgs a = make_args(L, rho);
    a.w = w;
    switch (L.gs_shape) {
    case 1: fine_gs_sweep_res<2, 5>(a, ke, norm_partial, s); break;
    case 2: fine_gs_sweep_res<3, 5>(a, ke, norm_partial, s); break;
    case 3: fine_gs_sweep_res<2, 6>(a, ke, norm_partial, s); break;
    default: fine_gs_sweep_res<6, 4>(a, ke, norm_partial, s); break;
    }
}

void launch_fine_residual(const Level &L, const float *rho, const KeMat &ke, double *norm_partial, int nblk_norm,
                          cudaStream_t s) {
    FineArgs a = make_args(L, rho);
    (void)nblk_norm;
    k_fine_residual<8><<<task_blocks(a, CPT) * 8, FBS, 0, s>>>(a, ke, norm_partial);
}

void launch_fine_residual64(const Level &L, const float *rho, const KeMat &ke, const KeMat64 &ke64, const float *f,
                            const double *u64,
                            float *r, bool exact, cudaStream_t s) {
    FineArgs a = make_args(L, rho);
    a.f = f;
    a.r = r;
    if (exact) k_fine_residual64<true><<<task_blocks(a, CPT64) * 8, FBS, 0, s>>>(a, ke, ke64, u64);
    else k_fine_residual64<false><<<task_blocks(a, CPT64) * 8, FBS, 0, s>>>(a, ke, ke64, u64);
}

void launch_rhs(const Level &L, const float *rho, const RhsTab &g, float *f, cudaStream_t s) {
    const int bs = 256;
    k_rhs<<<(unsigned)((L.P.nv + bs - 1) / bs), bs, 0, s>>>(L.P, rho, f, g);
}

// ---- FP64 helpers of the refined mode ---------------------------------------------
// u64 += e + T (T: the pending rigid translation of each of the 18 planes, see
// k_pin_deflate); the pinned origin (colour 7, first vertex) keeps its value
// Element-wise kernels over a blocked field run in storage order: one CTA of FVB
// threads per (128-vertex block, plane) chunk c, plane q = c % 18, vertex
// v = (c / 18) * FVB + thread (v >= nv in the padding of the last block).
__device__ __forceinline__ void field_elem(long long &o, int &q, long long &v) {
    const unsigned c = blockIdx.x;
    q = (int)(c % NF);
    v = (long long)(c / NF) * FVB + threadIdx.x;
    o = (long long)c * FVB + threadIdx.x;
}
static unsigned field_chunks(long long nv) { return (unsigned)(field_floats(nv) / FVB); }

__global__ void __launch_bounds__(FVB) k_update64(long long nv, double *u, const float *__restrict__ e,
                                                 const double *__restrict__ T, long long pin) {
    long long o, v;
    int q;
    field_elem(o, q, v);
    if (v >= nv || v == pin) return;
    u[o] += (double)e[o] + T[q];
}

// ---- rigid-translation deflation of the pinned problem -------------------------
// In the pinned system (rows v != origin, u_origin = 0) the rigid translation t'
// (1 on every vertex but the origin) is the lowest-energy mode: t'^T K t' is only
// the origin's 3x3 self block A_pp.  The FP16 coarse operators misjudge that tiny
// eigenvalue, and once the solution itself is small (near-uniform designs, where
// f nearly cancels) the V-cycle's error in this mode can grow from cycle to cycle.
// After every V-cycle of a solve the translation error is therefore removed
// exactly: s = sum_{v != origin} r_v = F + q with F = sum_{v != origin} f_v and
// q = sum_{d != 0} A_{p,d} u_{p+d} (because the columns of the periodic K sum to
// zero), alpha = A_pp^-1 s per case.  Instead of adding alpha to every vertex the
// shift is kept pending in T and folded into f (f_v += K_{v,p} alpha at the 26
// neighbours of the origin, F -= A_pp alpha), which is the same iteration; T joins
// the solution when it is next folded (k_update64, k_pin_fold).
// state[0..17] = F per (case, component), state[18..35] = T.
// One CTA of PIN_THREADS: thread (n, cr) with n < 26 the neighbour index (d = n,
// or n + 1 past the origin's own d = 13) and cr = 3c + r; the products of each
// neighbour are summed over d in ascending order by one thread per (c, r).
constexpr int PIN_THREADS = 26 * NF;
__device__ __forceinline__ void pin_deflate_block(const FineArgs &a, const KeMat &ke, double *state) {
    __shared__ double qpart[26][NF];
    __shared__ double al[NF];
    __shared__ double Ms[9];
    __shared__ int ok;
    const int tid = threadIdx.x;
    const int n = tid / NF, cr = tid % NF, c = cr / 3, r = cr % 3;
    const int d = n < 13 ? n : n + 1;
    const VertexGeo<7> g(a, 0);
    int Kn;
    bool pinned;
    const unsigned nid = g.nbr(a, d, Kn, pinned);
    float A[9];
    g.block(ke, d, A);
    {
        double t = 0;
        if (!pinned)
            for (int k = 0; k < 3; ++k) t += (double)A[3 * r + k] * (double)a.u[fidx(3 * c + k, nid)];
        qpart[n][cr] = t;
    }
    if (tid == 0) {
        float Af[9];
        g.block(ke, 13, Af);
        for (int k = 0; k < 9; ++k) Ms[k] = (double)Af[k];
    }
    __syncthreads();
    if (tid < NCASE) {
        const int cc = tid;
        const double *M = Ms;
        // inverse of the 3x3 self block by cofactors
        const double c00 = M[4] * M[8] - M[5] * M[7], c01 = M[5] * M[6] - M[3] * M[8], c02 = M[3] * M[7] - M[4] * M[6];
        const double det = M[0] * c00 + M[1] * c01 + M[2] * c02;
        if (cc == 0) ok = det > 0.0;
        if (det > 0.0) {  // otherwise not positive definite: leave the iterate alone
            const double inv[9] = {c00 / det, (M[2] * M[7] - M[1] * M[8]) / det, (M[1] * M[5] - M[2] * M[4]) / det,
                                   c01 / det, (M[0] * M[8] - M[2] * M[6]) / det, (M[2] * M[3] - M[0] * M[5]) / det,
                                   c02 / det, (M[1] * M[6] - M[0] * M[7]) / det, (M[0] * M[4] - M[1] * M[3]) / det};
            double sres[3];
            for (int rr = 0; rr < 3; ++rr) {
                double q = 0;
                for (int m = 0; m < 26; ++m) q += qpart[m][3 * cc + rr];
                sres[rr] = state[3 * cc + rr] + q;
            }
            double a3[3];
            for (int rr = 0; rr < 3; ++rr) a3[rr] = inv[3 * rr] * sres[0] + inv[3 * rr + 1] * sres[1] + inv[3 * rr + 2] * sres[2];
            for (int rr = 0; rr < 3; ++rr) {
                al[3 * cc + rr] = a3[rr];
                state[NF + 3 * cc + rr] += a3[rr];
                state[3 * cc + rr] -= M[3 * rr] * a3[0] + M[3 * rr + 1] * a3[1] + M[3 * rr + 2] * a3[2];
            }
        }
    }
    __syncthreads();
    if (!ok || pinned) return;
    // f at the origin's neighbours: K_{v,p} alpha = A_{p,d}^T alpha
    const double t = (double)A[r] * al[3 * c] + (double)A[3 + r] * al[3 * c + 1] + (double)A[6 + r] * al[3 * c + 2];
    float *fp = const_cast<float *>(a.f) + fidx(3 * c + r, nid);
    *fp = (float)((double)*fp + t);
}

__global__ void __launch_bounds__(PIN_THREADS) k_pin_deflate(FineArgs a, const __grid_constant__ KeMat ke,
                                                              double *state) {
    pin_deflate_block(a, ke, state);
}

// state: F = (plane sums of f) - f at the origin, T = 0
__global__ void k_pin_init(const double *__restrict__ sums, const float *__restrict__ f, long long nv, long long pin,
                           double *state) {
    const int i = threadIdx.x;
    if (i >= NF) return;
    state[i] = sums[i] - (double)f[fidx(i, pin)];
    state[NF + i] = 0.0;
}

// FP32 solutions: u += T on every vertex but the origin (grid-stride)
__global__ void k_pin_fold_u(long long nv, float *u, const double *__restrict__ state, long long pin) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv * NF;
         i += (long long)gridDim.x * blockDim.x) {
        const long long v = i % nv, q = i / nv;
        if (v != pin) u[fidx((int)q, v)] = (float)((double)u[fidx((int)q, v)] + state[NF + q]);
    }
}

// undo the fold of T into f at the origin's neighbours, then T = 0
__global__ void k_pin_restore_f(FineArgs a, const __grid_constant__ KeMat ke, double *state) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const VertexGeo<7> g(a, 0);
    for (int d = 0; d < 27; ++d) {
        if (d == 13) continue;
        int Kn;
        bool pinned;
        const unsigned nid = g.nbr(a, d, Kn, pinned);
        if (pinned) continue;
        float A[9];
        g.block(ke, d, A);
        for (int c = 0; c < NCASE; ++c)
            for (int r = 0; r < 3; ++r) {
                const double *T = state + NF + 3 * c;
                const double t = (double)A[r] * T[0] + (double)A[3 + r] * T[1] + (double)A[6 + r] * T[2];
                float *fp = const_cast<float *>(a.f) + fidx(3 * c + r, nid);
                *fp = (float)((double)*fp - t);
            }
    }
    for (int i = 0; i < NF; ++i) state[NF + i] = 0.0;
}

// FP32 field <-> FP64 field (both blocked)
__global__ void __launch_bounds__(FVB) k_f32_to_f64(long long nv, const float *__restrict__ s, double *d) {
    long long o, v;
    int q;
    field_elem(o, q, v);
    if (v < nv) d[o] = (double)s[o];
}

__global__ void __launch_bounds__(FVB) k_f64_to_f32(long long nv, const double *__restrict__ s, float *d) {
    long long o, v;
    int q;
    field_elem(o, q, v);
    if (v < nv) d[o] = (float)s[o];
}

void launch_update64(const Level &L, double *u64, const float *e, const double *T, cudaStream_t s) {
    k_update64<<<field_chunks(L.P.nv), FVB, 0, s>>>(L.P.nv, u64, e, T, L.P.base[7]);
}
void launch_pin_deflate(const Level &L, const float *rho, const KeMat &ke, double *state, cudaStream_t s) {
    k_pin_deflate<<<1, PIN_THREADS, 0, s>>>(make_args(L, rho), ke, state);
}
// level-0 f of a zero FP64 solution: f0 - K 0 = f0 on every vertex but the pinned
// origin, whose residual is 0 (what k_fine_residual64 computes for u64 = 0)
__global__ void __launch_bounds__(FVB) k_rhs_at_zero(long long nv, const float *__restrict__ f0, float *f,
                                                    long long pin) {
    long long o, v;
    int q;
    field_elem(o, q, v);
    if (v < nv) f[o] = v == pin ? 0.f : f0[o];
}
void launch_rhs_at_zero(const Level &L, const float *f0, float *f, cudaStream_t s) {
    k_rhs_at_zero<<<field_chunks(L.P.nv), FVB, 0, s>>>(L.P.nv, f0, f, L.P.base[7]);
}
void launch_pin_init(const Level &L, const double *sums, double *state, cudaStream_t s) {
    k_pin_init<<<1, 32, 0, s>>>(sums, L.f, L.P.nv, L.P.base[7], state);
}
void launch_pin_fold(const Level &L, const float *rho, const KeMat &ke, double *state, cudaStream_t s) {
    k_pin_fold_u<<<1184, 256, 0, s>>>(L.P.nv, L.u, state, L.P.base[7]);
    k_pin_restore_f<<<1, 32, 0, s>>>(make_args(L, rho), ke, state);
}
void launch_convert_field(long long nv, const float *src, double *dst, cudaStream_t s) {
    k_f32_to_f64<<<field_chunks(nv), FVB, 0, s>>>(nv, src, dst);
}
void launch_convert_field(long long nv, const double *src, float *dst, cudaStream_t s) {
    k_f64_to_f32<<<field_chunks(nv), FVB, 0, s>>>(nv, src, dst);
}

// ---- lockstep batches: the level 0 of several designs in one launch per step ----
// Each design owns a slice of the launch's CTAs (BatchSlices) and runs the same
// per-CTA body as its own launch would, with its CTA index inside the slice, so
// every design's fields and norm partials are those of its own launches, to the
// last bit.  A CTA copies its design's arguments to shared memory once; a design
// whose flag in `active` is 0 (converged) returns at once.  The sweep runs in
// launch shape 0 (six cases per thread, 4 CTAs/SM).
struct FineEnt {
    FineArgs a;
    double *partial;  // the design's norm partials
    double *state;    // its deflation state
    int design;       // its index in the active flags
};
struct FineBatchTab {
    BatchSlices gs;   // CTAs of one colour of the sweep, six cases per thread
    BatchSlices gs3;  // the same with three cases per thread
    BatchSlices res;  // CTAs of the seven-colour residual
    FineEnt e[BATCH_MAX];
};

// C cases per thread at MB CTAs per SM: launch shape 0 (C = 6, 4 CTAs/SM) or 1
// (C = 3, 5 CTAs/SM, one case pair and one scalar case per thread); the colour that
// writes the residual runs with six cases per thread in both
template <int K, bool RES, int C, int MB>
__global__ void __launch_bounds__(FBS, MB) k_fine_gs_batch(const FineBatchTab *__restrict__ t,
                                                         const int *__restrict__ active,
                                                         const __grid_constant__ KeMat ke) {
    static_assert(!RES || C == 6, "the residual-writing colour runs six cases per thread");
    __shared__ __align__(16) unsigned buf[(sizeof(FineArgs) + 3) / 4];
    const BatchSlices &sl = C == 6 ? t->gs : t->gs3;
    const int i = batch_slice(sl, blockIdx.x);
    const FineEnt &en = t->e[i];
    if (!__ldg(&active[en.design])) return;
    const FineArgs &a = stage_args(en.a, buf);
    const unsigned b0 = __ldg(&sl.start[i]), b1 = __ldg(&sl.start[i + 1]);
    fine_gs_block<K, C, RES>(a, ke, en.partial, blockIdx.x - b0, b1 - b0);
}

__global__ void __launch_bounds__(FBS, RES_MINB) k_fine_residual_batch(const FineBatchTab *__restrict__ t,
                                                                      const int *__restrict__ active,
                                                                      const __grid_constant__ KeMat ke) {
    __shared__ __align__(16) unsigned buf[(sizeof(FineArgs) + 3) / 4];
    const int i = batch_slice(t->res, blockIdx.x);
    const FineEnt &en = t->e[i];
    if (!__ldg(&active[en.design])) return;
    const FineArgs &a = stage_args(en.a, buf);
    const unsigned b0 = __ldg(&t->res.start[i]), b1 = __ldg(&t->res.start[i + 1]);
    fine_residual_block<7>(a, ke, en.partial, blockIdx.x - b0, b1 - b0);
}

// one CTA per design
__global__ void __launch_bounds__(PIN_THREADS) k_pin_deflate_batch(const FineBatchTab *__restrict__ t,
                                                                    const int *__restrict__ active,
                                                                    const __grid_constant__ KeMat ke) {
    __shared__ __align__(16) unsigned buf[(sizeof(FineArgs) + 3) / 4];
    const FineEnt &en = t->e[blockIdx.x];
    if (!__ldg(&active[en.design])) return;
    const FineArgs &a = stage_args(en.a, buf);
    pin_deflate_block(a, ke, en.state);
}

int fine_batch_create(const Level *const *lv0, const float *const *rho, double *const *partial,
                      double *const *state, const int *design, int n, bool scratch, BatchTab *out) {
    if (n < 1 || n > BATCH_MAX) return -1;
    FineBatchTab *t = new FineBatchTab();
    t->gs.n = t->gs3.n = t->res.n = n;
    t->gs.start[0] = t->gs3.start[0] = t->res.start[0] = 0;
    for (int i = 0; i < n; i++) {
        t->e[i].a = make_args(*lv0[i], rho[i]);
        if (scratch) t->e[i].a.u = t->e[i].a.r;
        t->e[i].partial = partial[i];
        t->e[i].state = state[i];
        t->e[i].design = design[i];
        t->gs.start[i + 1] = t->gs.start[i] + task_blocks(t->e[i].a, 6);
        t->gs3.start[i + 1] = t->gs3.start[i] + task_blocks(t->e[i].a, 3);
        t->res.start[i + 1] = t->res.start[i] + task_blocks(t->e[i].a, CPT) * 7;
    }
    void *d = nullptr;
    int rc = cudaMalloc(&d, sizeof(FineBatchTab)) == cudaSuccess ? 0 : -2;
    if (rc == 0 && cudaMemcpy(d, t, sizeof(FineBatchTab), cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
    if (rc == 0) {
        out->dev = d;
        out->n = n;
        out->grid[0] = t->gs.start[n];
        out->grid[1] = t->res.start[n];
        out->grid[2] = t->gs3.start[n];
    } else if (d) {
        cudaFree(d);
    }
    delete t;
    return rc;
}

template <int C, int MB>
static void fine_sweep_batch(const BatchTab &t, const KeMat &ke, const int *active, bool residual, cudaStream_t s) {
    const FineBatchTab *d = static_cast<const FineBatchTab *>(t.dev);
    const unsigned g = C == 6 ? t.grid[0] : t.grid[2];
    k_fine_gs_batch<0, false, C, MB><<<g, FBS, 0, s>>>(d, active, ke);
    k_fine_gs_batch<1, false, C, MB><<<g, FBS, 0, s>>>(d, active, ke);
    k_fine_gs_batch<2, false, C, MB><<<g, FBS, 0, s>>>(d, active, ke);
    k_fine_gs_batch<3, false, C, MB><<<g, FBS, 0, s>>>(d, active, ke);
    k_fine_gs_batch<4, false, C, MB><<<g, FBS, 0, s>>>(d, active, ke);
    k_fine_gs_batch<5, false, C, MB><<<g, FBS, 0, s>>>(d, active, ke);
    k_fine_gs_batch<6, false, C, MB><<<g, FBS, 0, s>>>(d, active, ke);
    if (residual) {
        k_fine_gs_batch<7, true, 6, 4><<<t.grid[0], FBS, 0, s>>>(d, active, ke);
        k_fine_residual_batch<<<t.grid[1], FBS, 0, s>>>(d, active, ke);
    } else {
        k_fine_gs_batch<7, false, C, MB><<<g, FBS, 0, s>>>(d, active, ke);
    }
}

void launch_fine_sweep_batch(const BatchTab &t, const KeMat &ke, const int *active, bool residual, int shape,
                             cudaStream_t s) {
    if (shape == 1) fine_sweep_batch<3, 5>(t, ke, active, residual, s);
    else fine_sweep_batch<6, 4>(t, ke, active, residual, s);
}

void launch_pin_deflate_batch(const BatchTab &t, const KeMat &ke, const int *active, cudaStream_t s) {
    k_pin_deflate_batch<<<t.n, PIN_THREADS, 0, s>>>(static_cast<const FineBatchTab *>(t.dev), active, ke);
}

// mean of each of the 18 planes over unique vertices, removed in place (FP64)
__global__ void __launch_bounds__(256) k_sum18_64(long long nv, const double *__restrict__ v, double *partial) {
    double s[NF];
#pragma unroll
    for (int q = 0; q < NF; ++q) s[q] = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int q = 0; q < NF; ++q) s[q] += v[fidx(q, i)];
    block_reduce<NF>(s, partial, blockIdx.x);
}

__global__ void __launch_bounds__(256) k_sum18_finish(const double *__restrict__ partial, int nblk, double *out) {
    double s[NF];
#pragma unroll
    for (int c = 0; c < NF; ++c) s[c] = 0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
        for (int c = 0; c < NF; ++c) s[c] += partial[(long long)b * NF + c];
    block_reduce<NF>(s, out, 0);
}

__global__ void k_sub_mean64(long long nv, double *v, const double *__restrict__ sum18) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const double inv = 1.0 / (double)nv;
#pragma unroll
    for (int q = 0; q < NF; ++q) v[fidx(q, i)] -= sum18[q] * inv;
}

void launch_remove_mean64(const Planes &P, double *v, double *partial, int nblk, cudaStream_t s) {
    double *tot = partial + (long long)nblk * NF;
    k_sum18_64<<<nblk, 256, 0, s>>>(P.nv, v, partial);
    k_sum18_finish<<<1, 256, 0, s>>>(partial, nblk, tot);
    k_sub_mean64<<<(unsigned)((P.nv + 255) / 256), 256, 0, s>>>(P.nv, v, tot);
}

}  // namespace h3d
