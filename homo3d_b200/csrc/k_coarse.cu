// k_coarse.cu -- coarse-level stencil sweeps and residuals, grid transfers,
// norms and layout conversions.
//
// Reference behaviour restated (homo3d grid.cu):
//   gs_relaxation_kernel (grid.cu:556-689): 27-point stencil of FP16 3x3 blocks,
//     FP32 accumulation, 3x3 block Gauss-Seidel on the components; no pin on
//     coarse levels (the pinned origin enters through the Galerkin stencils).
//   update_residual_kernel_1 (grid.cu:1465-1564): r = f - A u.
//   restrict_residual_kernel_1 (grid.cu:917-994): f_c(X) = sum_{|o|<r}
//     prod(r-|o|)/r^3 r_f(rX + o), periodic.
//   prolongate_correction_kernel_1 (grid.cu:1120-1190, homoCommon.cuh:350-385):
//     trilinear u_f += P u_c, the pinned fine origin is left unchanged.
//   v3_norm (grid.cu:1954-1966): norms over the padded periodic storage, i.e.
//     with the per-axis multiplicities of positions 0, 1 and n-1.
#include "h3d_internal.cuh"

namespace h3d {

struct CoarseArgs {
    float *u;
    const float *__restrict__ f;
    float *r;
    const uint4 *__restrict__ st;
    int n[3];
    int h[3];
    long long nv;
    long long P;
    float w;
    FastDiv dh0, dh1;  // division by h[0], h[1]
};

// (i, j, l) of index p (< 2^32) of a colour plane
__device__ __forceinline__ void cplane_coords(const CoarseArgs &a, long long p, int &i, int &j, int &l) {
    const unsigned q = (unsigned)p;
    const unsigned t = a.dh0.div(q);
    i = (int)(q - t * (unsigned)a.h[0]);
    const unsigned z = a.dh1.div(t);
    j = (int)(t - z * (unsigned)a.h[1]);
    l = (int)z;
}

__device__ __forceinline__ void axis_nbrs_c(int i, int p, int h, int &im, int &ip) {
    if (p) { im = i; ip = (i + 1 == h) ? 0 : i + 1; }
    else { im = (i == 0) ? h - 1 : i - 1; ip = i; }
}

// the 9 entries of neighbour block d of vertex me
template <int D, bool F32>
__device__ __forceinline__ void load_block(const CoarseArgs &a, long long me, float s[9]) {
    using S = StencilStore<F32>;
    constexpr int e0 = 9 * D, q0 = e0 / S::PER, q1 = (e0 + 8) / S::PER;
    float v[3 * S::PER];
#pragma unroll
    for (int q = q0; q <= q1; ++q) S::unpack(a.st[q * a.nv + me], v + (q - q0) * S::PER);
#pragma unroll
    for (int k = 0; k < 9; ++k) s[k] = v[e0 + k - S::PER * q0];
}

// Launch shapes of the coarse kernels (load cases per thread as packed FP32x2
// case pairs, CTAs per SM): shape 0 = three threads per vertex with two cases
// each, 6 CTAs/SM; shape 1 = one thread per vertex with all six, 4 CTAs/SM.  The
// threads of one vertex run in adjacent CTAs, so repeated stencil reads hit L2;
// shape 2 = two cases per thread at 4 CTAs/SM, shape 3 = six cases per thread at 3
// CTAs/SM.  All shapes give the same result to the last bit.

// KC: the vertex colour, or -1 for the run-time colour kr (one code body for all
// colours)
// CG: neighbour values through L2 only (ld.global.cg), for kernels that read values
// other CTAs wrote earlier in the same launch
template <int KC, bool SELF, bool F32, int C, bool CG = false>
__device__ __forceinline__ void coarse_apply(const CoarseArgs &a, long long me, int i, int j, int l, int cb,
                                             float acc[3 * C], int kr = KC) {
    static_assert(C % 2 == 0, "the load cases of a thread go in packed FP32x2 lane pairs");
    constexpr int NP = C / 2;
    const int K = KC >= 0 ? KC : kr;
    const int px = (K & 1) ^ 1, py = ((K >> 1) & 1) ^ 1, pz = ((K >> 2) & 1) ^ 1;
    int ii[3], jj[3], ll[3];
    axis_nbrs_c(i, px, a.h[0], ii[0], ii[2]);
    axis_nbrs_c(j, py, a.h[1], jj[0], jj[2]);
    axis_nbrs_c(l, pz, a.h[2], ll[0], ll[2]);
    ii[1] = i; jj[1] = j; ll[1] = l;
    // plane offsets of the neighbour rows (a colour plane holds < 2^32 vertices)
    unsigned X[3], Y[3], Z[3];
    const unsigned h0 = (unsigned)a.h[0], h01 = (unsigned)a.h[0] * (unsigned)a.h[1];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        X[t] = (unsigned)ii[t];
        Y[t] = h0 * (unsigned)jj[t];
        Z[t] = h01 * (unsigned)ll[t];
    }
    // lane pair (case cb+2j, case cb+2j+1): packed FP32x2 FMAs in the scalar per-case order
    float2 acc2[3 * NP];
#pragma unroll
    for (int q = 0; q < 3 * NP; ++q) acc2[q] = make_float2(0.f, 0.f);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        if (d == 13 && !SELF) continue;
        const int dx = d % 3 - 1, dy = d / 3 % 3 - 1, dz = d / 9 - 1;
        float s[9];
        switch (d) {  // compile-time block index for the chunk arithmetic
#define H3D_LB(D) case D: load_block<D, F32>(a, me, s); break;
            H3D_LB(0) H3D_LB(1) H3D_LB(2) H3D_LB(3) H3D_LB(4) H3D_LB(5) H3D_LB(6) H3D_LB(7) H3D_LB(8)
            H3D_LB(9) H3D_LB(10) H3D_LB(11) H3D_LB(12) H3D_LB(13) H3D_LB(14) H3D_LB(15) H3D_LB(16)
            H3D_LB(17) H3D_LB(18) H3D_LB(19) H3D_LB(20) H3D_LB(21) H3D_LB(22) H3D_LB(23) H3D_LB(24)
            H3D_LB(25) H3D_LB(26)
#undef H3D_LB
        }
        const int Kn = K ^ ((dx & 1) | ((dy & 1) << 1) | ((dz & 1) << 2));
        const unsigned nid = (unsigned)Kn * (unsigned)a.P + X[dx + 1] + Y[dy + 1] + Z[dz + 1];
        const float *up = a.u + fidx(3 * cb, nid);  // planes 3cb.. of the neighbour, FVB apart
#pragma unroll
        for (int jp = 0; jp < NP; ++jp) {
            float2 uu[3];
#pragma unroll
            for (int m = 0; m < 3; ++m)
                uu[m] = CG ? make_float2(__ldcg(up + (6 * jp + m) * FVB), __ldcg(up + (6 * jp + 3 + m) * FVB))
                           : make_float2(up[(6 * jp + m) * FVB], up[(6 * jp + 3 + m) * FVB]);
#pragma unroll
            for (int r = 0; r < 3; ++r)
                acc2[3 * jp + r] = __ffma2_rn(make_float2(s[3 * r], s[3 * r]), uu[0],
                                              __ffma2_rn(make_float2(s[3 * r + 1], s[3 * r + 1]), uu[1],
                                                         __ffma2_rn(make_float2(s[3 * r + 2], s[3 * r + 2]), uu[2],
                                                                    acc2[3 * jp + r])));
        }
    }
#pragma unroll
    for (int jp = 0; jp < NP; ++jp)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            acc[6 * jp + m] = acc2[3 * jp + m].x;
            acc[6 * jp + 3 + m] = acc2[3 * jp + m].y;
        }
}

// thread -> (vertex p, first load case cb) for C cases per thread: the NCASE / C
// CTAs of a case group cover the same 128 vertices with different load cases
template <int C>
__device__ __forceinline__ void coarse_task(long long &p, int &cb, unsigned bid) {
    constexpr int NG = NCASE / C;
    cb = (int)(bid % NG) * C;
    p = (long long)(bid / NG) * blockDim.x + threadIdx.x;
}

// RES (the last colour of a sweep, whose neighbours are final) also writes the
// residual of the updated vertex: r = f - acc - A_0 u with acc the neighbour sum.
// bid: the CTA's index in the design's launch (blockIdx.x, or its slice of a
// batched launch)
template <int K, bool F32, int CGS_CPT, bool RES>
__device__ __forceinline__ void coarse_gs_block(const CoarseArgs &a, unsigned bid) {
    long long p;
    int cb;
    coarse_task<CGS_CPT>(p, cb, bid);
    if (p >= a.P) return;
    const long long me = (long long)K * a.P + p;
    int i, j, l;
    cplane_coords(a, p, i, j, l);
    float acc[3 * CGS_CPT], ks[9];
    coarse_apply<K, false, F32, CGS_CPT>(a, me, i, j, l, cb, acc);
    load_block<13, F32>(a, me, ks);
    const float w = a.w;
#pragma unroll
    for (int c = 0; c < CGS_CPT; ++c) {
        float *u = a.u + fidx(3 * (cb + c), me);
        const float *f = a.f + fidx(3 * (cb + c), me);
        float u0 = u[0], u1 = u[FVB], u2 = u[2 * FVB];
        u0 = w * (f[0] - acc[3 * c] - ks[1] * u1 - ks[2] * u2) / ks[0] + (1.f - w) * u0;
        u1 = w * (f[FVB] - acc[3 * c + 1] - ks[3] * u0 - ks[5] * u2) / ks[4] + (1.f - w) * u1;
        u2 = w * (f[2 * FVB] - acc[3 * c + 2] - ks[6] * u0 - ks[7] * u1) / ks[8] + (1.f - w) * u2;
        u[0] = u0;
        u[FVB] = u1;
        u[2 * FVB] = u2;
        if (RES) {
            float *r = a.r + fidx(3 * (cb + c), me);
#pragma unroll
            for (int m = 0; m < 3; ++m)
                r[m * FVB] = f[m * FVB] - acc[3 * c + m] - fmaf(ks[3 * m + 2], u2, fmaf(ks[3 * m + 1], u1, ks[3 * m] * u0));
        }
    }
}

template <int K, bool F32, int CGS_CPT, int CGS_MINB, bool RES = false>
__global__ void __launch_bounds__(128, CGS_MINB) k_coarse_gs(CoarseArgs a) {
    coarse_gs_block<K, F32, CGS_CPT, RES>(a, blockIdx.x);
}

template <bool F32, int CRES_CPT>
__device__ __forceinline__ void coarse_res_vertex(const CoarseArgs &a, long long p, int cb, int K) {
    const long long me = (long long)K * a.P + p;
    int i, j, l;
    cplane_coords(a, p, i, j, l);
    float acc[3 * CRES_CPT];
    coarse_apply<-1, true, F32, CRES_CPT>(a, me, i, j, l, cb, acc, K);
#pragma unroll
    for (int q = 0; q < 3 * CRES_CPT; ++q) {
        const long long o = fidx(3 * cb + q, me);
        a.r[o] = a.f[o] - acc[q];
    }
}

// all colours in one launch (eight, or seven after a sweep whose last colour wrote
// its own residual), the colour the block index modulo NCOL and a run-time value
// of one code body: the CTAs of one vertex block read each other's neighbour rows
// while they are in L2, and a small level costs one launch instead of eight
template <bool F32, int CRES_CPT, unsigned NCOL>
__device__ __forceinline__ void coarse_residual_block(const CoarseArgs &a, unsigned bid) {
    constexpr int NG = NCASE / CRES_CPT;
    const int K = (int)(bid % NCOL);
    const unsigned bx = bid / NCOL;
    const int cb = (int)(bx % NG) * CRES_CPT;
    const long long p = (long long)(bx / NG) * blockDim.x + threadIdx.x;
    if (p >= a.P) return;
    coarse_res_vertex<F32, CRES_CPT>(a, p, cb, K);
}

template <bool F32, int CRES_CPT, int CRES_MINB, unsigned NCOL>
__global__ void __launch_bounds__(128, CRES_MINB) k_coarse_residual(CoarseArgs a) {
    coarse_residual_block<F32, CRES_CPT, NCOL>(a, blockIdx.x);
}

static CoarseArgs make_cargs(const Level &L) {
    CoarseArgs a;
    a.u = L.u;
    a.f = L.f;
    a.r = L.r;
    a.st = L.st;
    for (int d = 0; d < 3; ++d) { a.n[d] = L.P.n[d]; a.h[d] = L.P.n[d] / 2; }
    a.nv = L.P.nv;
    a.P = L.P.nv / 8;
    a.w = 1.f;
    a.dh0 = FastDiv((unsigned)a.h[0]);
    a.dh1 = FastDiv((unsigned)a.h[1]);
    return a;
}

template <bool F32, int C, int MINB>
static void coarse_gs_sweep(const CoarseArgs &a, cudaStream_t s) {
    const unsigned nb = (unsigned)((a.P + 127) / 128) * (NCASE / C);
    k_coarse_gs<0, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<1, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<2, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<3, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<4, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<5, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<6, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<7, F32, C, MINB><<<nb, 128, 0, s>>>(a);
}

void launch_coarse_gs(const Level &L, float w, cudaStream_t s) {
    CoarseArgs a = make_cargs(L);
    a.w = w;
    if (L.st32) {
        switch (L.gs_shape) {
        case 1: coarse_gs_sweep<true, 6, 4>(a, s); break;
        case 2: coarse_gs_sweep<true, 2, 4>(a, s); break;
        case 3: coarse_gs_sweep<true, 6, 3>(a, s); break;
        default: coarse_gs_sweep<true, 2, 6>(a, s); break;
        }
    } else {
        switch (L.gs_shape) {
        case 1: coarse_gs_sweep<false, 6, 4>(a, s); break;
        case 2: coarse_gs_sweep<false, 2, 4>(a, s); break;
        case 3: coarse_gs_sweep<false, 6, 3>(a, s); break;
        default: coarse_gs_sweep<false, 2, 6>(a, s); break;
        }
    }
}

template <bool F32, int C, int MINB, unsigned NCOL = 8>
static void coarse_residual_all(const CoarseArgs &a, cudaStream_t s) {
    const unsigned nb = (unsigned)((a.P + 127) / 128) * (NCASE / C);
    k_coarse_residual<F32, C, MINB, NCOL><<<nb * NCOL, 128, 0, s>>>(a);
}

template <unsigned NCOL>
static void coarse_residual_shape(const Level &L, const CoarseArgs &a, cudaStream_t s) {
    if (L.st32) {
        switch (L.res_shape) {
        case 1: coarse_residual_all<true, 6, 4, NCOL>(a, s); break;
        case 2: coarse_residual_all<true, 2, 4, NCOL>(a, s); break;
        case 3: coarse_residual_all<true, 6, 3, NCOL>(a, s); break;
        default: coarse_residual_all<true, 2, 6, NCOL>(a, s); break;
        }
    } else {
        switch (L.res_shape) {
        case 1: coarse_residual_all<false, 6, 4, NCOL>(a, s); break;
        case 2: coarse_residual_all<false, 2, 4, NCOL>(a, s); break;
        case 3: coarse_residual_all<false, 6, 3, NCOL>(a, s); break;
        default: coarse_residual_all<false, 2, 6, NCOL>(a, s); break;
        }
    }
}

void launch_coarse_residual(const Level &L, cudaStream_t s) { coarse_residual_shape<8>(L, make_cargs(L), s); }

// a sweep followed by the level's residual: the last colour's launch writes its
// own residual, the residual launch covers the other seven colours
template <bool F32, int C, int MINB>
static void coarse_gs_sweep_res(const CoarseArgs &a, cudaStream_t s) {
    const unsigned nb = (unsigned)((a.P + 127) / 128) * (NCASE / C);
    k_coarse_gs<0, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<1, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<2, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<3, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<4, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<5, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<6, F32, C, MINB><<<nb, 128, 0, s>>>(a);
    k_coarse_gs<7, F32, C, MINB, true><<<nb, 128, 0, s>>>(a);
}

void launch_coarse_gs_residual(const Level &L, float w, cudaStream_t s) {
    CoarseArgs a = make_cargs(L);
    a.w = w;
    if (L.st32) {
        switch (L.gs_shape) {
        case 1: coarse_gs_sweep_res<true, 6, 4>(a, s); break;
        case 2: coarse_gs_sweep_res<true, 2, 4>(a, s); break;
        case 3: coarse_gs_sweep_res<true, 6, 3>(a, s); break;
        default: coarse_gs_sweep_res<true, 2, 6>(a, s); break;
        }
    } else {
        switch (L.gs_shape) {
        case 1: coarse_gs_sweep_res<false, 6, 4>(a, s); break;
        case 2: coarse_gs_sweep_res<false, 2, 4>(a, s); break;
        case 3: coarse_gs_sweep_res<false, 6, 3>(a, s); break;
        default: coarse_gs_sweep_res<false, 2, 6>(a, s); break;
        }
    }
    coarse_residual_shape<7>(L, a, s);
}

// ---- transfers ---------------------------------------------------------------
// Restriction: one thread per (coarse vertex, load case) (blockIdx.y = case), three
// accumulators over the 27 (ratio 2) gathered fine vertices, so the large levels
// have enough independent loads in flight.  Prolongation: one thread per fine
// vertex and all 18 planes (at most 8 coarse parents, most with weight 0).
__global__ void __launch_bounds__(256) k_restrict(Planes F, Planes C, int r0, int r1, int r2,
                                                  const float *__restrict__ rf, float *fc) {
    const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v >= C.nv) return;
    const int c = blockIdx.y;
    const int k = color_of_index(C, v);
    int x, y, z;
    vpos(C, k, v - C.base[k], x, y, z);
    const float pr = (float)(r0 * r1 * r2);
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    for (int ox = -r0 + 1; ox < r0; ox++) {
        const int fx = wrap(r0 * x + ox, F.n[0]);
        for (int oy = -r1 + 1; oy < r1; oy++) {
            const int fy = wrap(r1 * y + oy, F.n[1]);
            for (int oz = -r2 + 1; oz < r2; oz++) {
                const int fz = wrap(r2 * z + oz, F.n[2]);
                const float w = (float)((r0 - abs(ox)) * (r1 - abs(oy)) * (r2 - abs(oz))) / pr;
                const float *src = rf + fidx(3 * c, vidx(F, fx, fy, fz));
                a0 = fmaf(__ldg(&src[0]), w, a0);
                a1 = fmaf(__ldg(&src[FVB]), w, a1);
                a2 = fmaf(__ldg(&src[2 * FVB]), w, a2);
            }
        }
    }
    float *dst = fc + fidx(3 * c, v);
    dst[0] = a0;
    dst[FVB] = a1;
    dst[2 * FVB] = a2;
}

__global__ void __launch_bounds__(256) k_prolong(Planes F, Planes C, int r0, int r1, int r2, int is_root,
                                                 const float *__restrict__ uc, float *uf) {
    const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v >= F.nv) return;
    const int k = color_of_index(F, v);
    int x, y, z;
    vpos(F, k, v - F.base[k], x, y, z);
    if (is_root && x == 0 && y == 0 && z == 0) return;
    const int rx = x % r0, ry = y % r1, rz = z % r2;
    const int bx = x / r0, by = y / r1, bz = z / r2;
    const float wc = (float)(r0 * r1 * r2);
    float acc[NF];
#pragma unroll
    for (int q = 0; q < NF; ++q) acc[q] = 0.f;
#pragma unroll
    for (int id = 0; id < 8; ++id) {
        const int ox = id & 1, oy = (id >> 1) & 1, oz = id >> 2;
        const float w = (float)((r0 - abs(ox * r0 - rx)) * (r1 - abs(oy * r1 - ry)) * (r2 - abs(oz * r2 - rz))) / wc;
        if (w == 0.f) continue;
        const long long ci = vidx(C, wrap(bx + ox, C.n[0]), wrap(by + oy, C.n[1]), wrap(bz + oz, C.n[2]));
#pragma unroll
        for (int q = 0; q < NF; ++q) acc[q] = fmaf(__ldg(&uc[fidx(q, ci)]), w, acc[q]);
    }
#pragma unroll
    for (int q = 0; q < NF; ++q) uf[fidx(q, v)] += acc[q];
}

// Ratio 2 on every axis (even grids): one thread per coarse vertex in
// lexicographic order, so that consecutive threads read consecutive fine vertices
// of each colour plane.  Fine vertex 2X + o has the colour of o's parities and, in
// that colour's plane, the coordinates X - [o < 0] (wrapped) per axis; the sums
// run in the general kernel's order, so the results are identical.
// thread t of case c; uc (or nullptr): the coarse solution, cleared at the vertex
__device__ __forceinline__ void restrict2_thread(const Planes &F, const Planes &C, const FastDiv &dn0,
                                                 const FastDiv &dn1, const float *__restrict__ rf, float *fc,
                                                 float *uc, long long t, int c) {
    if (t >= C.nv) return;
    const unsigned q = (unsigned)t, tq = dn0.div(q), zq = dn1.div(tq);
    const int x = (int)(q - tq * (unsigned)C.n[0]), y = (int)(tq - zq * (unsigned)C.n[1]), z = (int)zq;
    const int xm = x == 0 ? C.n[0] - 1 : x - 1, ym = y == 0 ? C.n[1] - 1 : y - 1, zm = z == 0 ? C.n[2] - 1 : z - 1;
    const long long cpl = F.nv / 8;  // vertices per fine colour plane
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
    for (int ox = -1; ox <= 1; ox++)
#pragma unroll
        for (int oy = -1; oy <= 1; oy++)
#pragma unroll
            for (int oz = -1; oz <= 1; oz++) {
                const float w = (float)((2 - abs(ox)) * (2 - abs(oy)) * (2 - abs(oz))) / 8.f;
                const int k = ((ox + 1) & 1) | (((oy + 1) & 1) << 1) | (((oz + 1) & 1) << 2);
                const long long fi = k * cpl + (ox < 0 ? xm : x) +
                                     (long long)C.n[0] * ((oy < 0 ? ym : y) + (long long)C.n[1] * (oz < 0 ? zm : z));
                const float *src = rf + fidx(3 * c, fi);
                a0 = fmaf(__ldg(&src[0]), w, a0);
                a1 = fmaf(__ldg(&src[FVB]), w, a1);
                a2 = fmaf(__ldg(&src[2 * FVB]), w, a2);
            }
    const long long cv = vidx(C, x, y, z);
    float *dst = fc + fidx(3 * c, cv);
    dst[0] = a0;
    dst[FVB] = a1;
    dst[2 * FVB] = a2;
    if (uc) {
        float *z0 = uc + fidx(3 * c, cv);
        z0[0] = 0.f;
        z0[FVB] = 0.f;
        z0[2 * FVB] = 0.f;
    }
}

__global__ void __launch_bounds__(256) k_restrict2(Planes F, Planes C, FastDiv dn0, FastDiv dn1,
                                                   const float *__restrict__ rf, float *fc) {
    restrict2_thread(F, C, dn0, dn1, rf, fc, nullptr, blockIdx.x * (long long)blockDim.x + threadIdx.x, blockIdx.y);
}

// Ratio 2: one thread per coarse cell X; its eight fine vertices 2X + e take
// their corrections from the cell's eight corners, read once per plane.  Fine
// vertex 2X + e sits at index X (lexicographic) of colour plane k(e).
__device__ __forceinline__ void prolong2_thread(const Planes &F, const Planes &C, const FastDiv &dn0,
                                                const FastDiv &dn1, int is_root, const float *__restrict__ uc,
                                                float *uf, long long t) {
    if (t >= C.nv) return;
    const unsigned q = (unsigned)t, tq = dn0.div(q), zq = dn1.div(tq);
    const int x = (int)(q - tq * (unsigned)C.n[0]), y = (int)(tq - zq * (unsigned)C.n[1]), z = (int)zq;
    const int xp = x + 1 == C.n[0] ? 0 : x + 1, yp = y + 1 == C.n[1] ? 0 : y + 1, zp = z + 1 == C.n[2] ? 0 : z + 1;
    long long ci[8];
#pragma unroll
    for (int id = 0; id < 8; ++id)
        ci[id] = vidx(C, (id & 1) ? xp : x, ((id >> 1) & 1) ? yp : y, (id >> 2) ? zp : z);
    const long long cpl = F.nv / 8;
    const bool root = is_root && t == 0;
#pragma unroll 2
    for (int pl = 0; pl < NF; ++pl) {
        // the eight fine values are loaded before any is stored: the compiler
        // cannot tell the eight colour planes apart, and read-add-write per vertex
        // would wait on one DRAM round trip after another
        float cv[8], fv[8];
#pragma unroll
        for (int id = 0; id < 8; ++id) cv[id] = __ldg(&uc[fidx(pl, ci[id])]);
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int ex = e & 1, ey = (e >> 1) & 1, ez = e >> 2;
            const int k = ((ex + 1) & 1) | (((ey + 1) & 1) << 1) | (((ez + 1) & 1) << 2);
            fv[e] = uf[fidx(pl, k * cpl + t)];
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            if (e == 0 && root) continue;  // the pinned origin keeps its value
            const int ex = e & 1, ey = (e >> 1) & 1, ez = e >> 2;
            float acc = 0.f;
#pragma unroll
            for (int id = 0; id < 8; ++id) {
                const int ox = id & 1, oy = (id >> 1) & 1, oz = id >> 2;
                const float w = (float)((2 - abs(ox * 2 - ex)) * (2 - abs(oy * 2 - ey)) * (2 - abs(oz * 2 - ez))) / 8.f;
                if (w == 0.f) continue;
                acc = fmaf(cv[id], w, acc);
            }
            // fine vertex (2x + ex, ...): colour of (ex, ey, ez), plane index t
            const int k = ((ex + 1) & 1) | (((ey + 1) & 1) << 1) | (((ez + 1) & 1) << 2);
            uf[fidx(pl, k * cpl + t)] = fv[e] + acc;
        }
    }
}

__global__ void __launch_bounds__(256) k_prolong2(Planes F, Planes C, FastDiv dn0, FastDiv dn1, int is_root,
                                                  const float *__restrict__ uc, float *uf) {
    prolong2_thread(F, C, dn0, dn1, is_root, uc, uf, blockIdx.x * (long long)blockDim.x + threadIdx.x);
}

static bool ratio2(const Level &C) { return C.ratio[0] == 2 && C.ratio[1] == 2 && C.ratio[2] == 2; }

void launch_restrict(const Level &F, const Level &C, cudaStream_t s) {
    const int bs = 256;
    const dim3 grid((unsigned)((C.P.nv + bs - 1) / bs), NCASE);
    if (ratio2(C) && F.P.even)
        k_restrict2<<<grid, bs, 0, s>>>(F.P, C.P, FastDiv((unsigned)C.P.n[0]), FastDiv((unsigned)C.P.n[1]), F.r, C.f);
    else
        k_restrict<<<grid, bs, 0, s>>>(F.P, C.P, C.ratio[0], C.ratio[1], C.ratio[2], F.r, C.f);
}

void launch_prolong(const Level &F, const Level &C, int is_root, cudaStream_t s) {
    const int bs = 256;
    if (ratio2(C) && F.P.even)
        k_prolong2<<<(unsigned)((C.P.nv + bs - 1) / bs), bs, 0, s>>>(F.P, C.P, FastDiv((unsigned)C.P.n[0]),
                                                                     FastDiv((unsigned)C.P.n[1]), is_root, C.u, F.u);
    else
        k_prolong<<<(unsigned)((F.P.nv + bs - 1) / bs), bs, 0, s>>>(F.P, C.P, C.ratio[0], C.ratio[1], C.ratio[2],
                                                                      is_root, C.u, F.u);
}

// ---- norms and means ---------------------------------------------------------
constexpr int NORM_BS = 256;

int norm_blocks(const Planes &P) {
    long long nb = (P.nv + NORM_BS - 1) / NORM_BS;
    return (int)(nb < 2048 ? nb : 2048);
}

__global__ void __launch_bounds__(NORM_BS) k_weighted_norm(Planes P, const float *__restrict__ v, double *partial) {
    double s[NCASE] = {0, 0, 0, 0, 0, 0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P.nv; i += (long long)gridDim.x * blockDim.x) {
        const int k = color_of_index(P, i);
        int x, y, z;
        vpos(P, k, i - P.base[k], x, y, z);
        const double m = (double)(axis_mult(x, P.n[0]) * axis_mult(y, P.n[1]) * axis_mult(z, P.n[2]));
#pragma unroll
        for (int c = 0; c < NCASE; ++c) {
            double a = 0;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const double t = v[fidx(3 * c + q, i)];
                a += t * t;
            }
            s[c] += m * a;
        }
    }
    block_reduce<NCASE>(s, partial, blockIdx.x);
}

void launch_weighted_norm(const Planes &P, const float *v, double *partial, int nblk, cudaStream_t s) {
    k_weighted_norm<<<nblk, NORM_BS, 0, s>>>(P, v, partial);
}

template <int N>
__device__ __forceinline__ void finish_block(const double *__restrict__ partial, int nblk, double *out) {
    double s[N];
#pragma unroll
    for (int c = 0; c < N; ++c) s[c] = 0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
        for (int c = 0; c < N; ++c) s[c] += partial[(long long)b * N + c];
    block_reduce<N>(s, out, 0);
}

template <int N>
__global__ void __launch_bounds__(256) k_finish(const double *__restrict__ partial, int nblk, double *out) {
    finish_block<N>(partial, nblk, out);
}

// first stage of a long reduction: CTA g sums the partials of blocks
// [g*per, (g+1)*per) into out[g*N + c]
template <int N>
__device__ __forceinline__ void finish_chunk_block(const double *__restrict__ partial, int nblk, int per,
                                                   double *out, int g) {
    const int b0 = g * per, b1 = min(nblk, b0 + per);
    double s[N];
#pragma unroll
    for (int c = 0; c < N; ++c) s[c] = 0;
    for (int b = b0 + threadIdx.x; b < b1; b += blockDim.x)
#pragma unroll
        for (int c = 0; c < N; ++c) s[c] += partial[(long long)b * N + c];
    block_reduce<N>(s, out, g);
}

template <int N>
__global__ void __launch_bounds__(256) k_finish_chunks(const double *__restrict__ partial, int nblk, int per,
                                                       double *out) {
    finish_chunk_block<N>(partial, nblk, per, out, blockIdx.x);
}

void launch_norm_finish(const double *partial, int nblk, double *out6, cudaStream_t s) {
    if (nblk <= NORM_FINISH_DIRECT) {
        k_finish<NCASE><<<1, 256, 0, s>>>(partial, nblk, out6);
        return;
    }
    // two stages; the first writes NORM_FINISH_CHUNKS x 6 sums behind the partials
    const int per = (nblk + NORM_FINISH_CHUNKS - 1) / NORM_FINISH_CHUNKS;
    double *mid = const_cast<double *>(partial) + (long long)nblk * NCASE;
    k_finish_chunks<NCASE><<<NORM_FINISH_CHUNKS, 256, 0, s>>>(partial, nblk, per, mid);
    k_finish<NCASE><<<1, 256, 0, s>>>(mid, NORM_FINISH_CHUNKS, out6);
}

__global__ void __launch_bounds__(NORM_BS) k_sum18(Planes P, const float *__restrict__ v, double *partial) {
    double s[NF];
#pragma unroll
    for (int q = 0; q < NF; ++q) s[q] = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P.nv; i += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int q = 0; q < NF; ++q) s[q] += v[fidx(q, i)];
    block_reduce<NF>(s, partial, blockIdx.x);
}

__global__ void __launch_bounds__(256) k_sub_mean(Planes P, float *v, const double *__restrict__ sum18) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= P.nv) return;
    const double inv = 1.0 / (double)P.nv;
#pragma unroll
    for (int q = 0; q < NF; ++q) v[fidx(q, i)] -= (float)(sum18[q] * inv);
}

void launch_mean_partial(const Planes &P, const float *v, double *partial, int nblk, cudaStream_t s) {
    k_sum18<<<nblk, NORM_BS, 0, s>>>(P, v, partial);
}

// the 18 plane sums of launch_mean_partial's partials into out
void launch_sum18_finish(const double *partial, int nblk, double *out, cudaStream_t s) {
    k_finish<NF><<<1, 256, 0, s>>>(partial, nblk, out);
}

// partial holds nblk rows of 18 sums; the total goes to partial[nblk*18 ..]
void launch_remove_mean(const Planes &P, float *v, const double *partial, int nblk, cudaStream_t s) {
    double *tot = const_cast<double *>(partial) + (long long)nblk * NF;
    k_finish<NF><<<1, 256, 0, s>>>(partial, nblk, tot);
    k_sub_mean<<<(unsigned)((P.nv + 255) / 256), 256, 0, s>>>(P, v, tot);
}

// ---- layout conversion: lexicographic [6][nv][3] <-> the blocked colour-ordered field ----
__global__ void k_field_lex(Planes P, const float *__restrict__ src, float *dst, int to_lex) {
    const long long lex = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (lex >= P.nv) return;
    const int x = (int)(lex % P.n[0]);
    const long long t = lex / P.n[0];
    const int y = (int)(t % P.n[1]), z = (int)(t / P.n[1]);
    const long long v = vidx(P, x, y, z);
#pragma unroll
    for (int c = 0; c < NCASE; ++c)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            const long long li = ((long long)c * P.nv + lex) * 3 + m, pi = fidx(3 * c + m, v);
            if (to_lex) dst[li] = src[pi];
            else dst[pi] = src[li];
        }
}

void launch_field_to_lex(const Planes &P, const float *src, float *dst_lex, cudaStream_t s) {
    k_field_lex<<<(unsigned)((P.nv + 255) / 256), 256, 0, s>>>(P, src, dst_lex, 1);
}
void launch_field_from_lex(const Planes &P, const float *src_lex, float *dst, cudaStream_t s) {
    k_field_lex<<<(unsigned)((P.nv + 255) / 256), 256, 0, s>>>(P, src_lex, dst, 0);
}

__global__ void k_stencil_lex(Planes P, const uint4 *st, float *lexf, const float *lexin, uint4 *stout, int f32) {
    const long long lex = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (lex >= P.nv) return;
    const int x = (int)(lex % P.n[0]);
    const long long t = lex / P.n[0];
    const int y = (int)(t % P.n[1]), z = (int)(t / P.n[1]);
    const long long v = vidx(P, x, y, z);
    for (int e = 0; e < 243; ++e) {
        if (lexf) lexf[lex * 243 + e] = f32 ? StencilStore<true>::get(st, P.nv, v, e) : StencilStore<false>::get(st, P.nv, v, e);
        else if (f32) StencilStore<true>::put(stout, P.nv, v, e, lexin[lex * 243 + e]);
        else StencilStore<false>::put(stout, P.nv, v, e, lexin[lex * 243 + e]);
    }
}

void launch_stencil_to_lex(const Level &L, float *dst_lex, cudaStream_t s) {
    k_stencil_lex<<<(unsigned)((L.P.nv + 127) / 128), 128, 0, s>>>(L.P, L.st, dst_lex, nullptr, nullptr, L.st32);
}
void launch_stencil_from_lex(const Level &L, const float *src_lex, cudaStream_t s) {
    k_stencil_lex<<<(unsigned)((L.P.nv + 127) / 128), 128, 0, s>>>(L.P, nullptr, nullptr, src_lex, L.st, L.st32);
}

// ---- the bottom of the V-cycle in one cooperative launch -------------------------
// The small levels cost a launch per colour (about 6 us each inside a graph,
// whatever the level's size).  k_vcycle_bottom runs the V-cycle's steps from the
// restriction into level `first` down to the coarsest solve and back up to the
// post-smoothing of level `first` as phases of one cooperative launch, separated by
// grid-wide barriers: per smoothed level on the way down, restriction (and the
// cleared correction), eight colours (the last with its residual), the residual of
// the other seven colours; at the bottom the restriction and the dense coarsest
// solve; per level on the way up, prolongation and eight colours.  Each phase runs
// the arithmetic of the separate kernels in the same order (two load cases per
// thread, ratio-2 transfers), so the results are the same to the last bit.  Values
// that other CTAs wrote earlier in the launch are read through L2 (ld.global.cg).
// The barrier is a counter and a generation number in global memory; a wait that
// runs out (it cannot, with all CTAs resident, but it is bounded) sets *flag and
// the CTA leaves the kernel, whose later waits then run out too.
constexpr int BOT_MAXLV = 8;
constexpr int BOT_T = 128;
constexpr long long BOT_WAIT_LIMIT = 1ll << 24;  // polls of the generation (L2 round trips)

struct BottomArgs {
    CoarseArgs lv[BOT_MAXLV + 1];  // lv[0]: the level above `first` (its residual, its u after the cycle)
    Planes P[BOT_MAXLV + 1];
    int nlv;                       // levels from `first` to the coarsest
    int project;                   // coarsest: remove the mean first
    int ndof;                      // coarsest unknowns
    const double *aug;             // coarsest [K | K^-1]
    unsigned *bar;                 // [0] arrivals, [1] generation
    int *flag;
};

__device__ __forceinline__ bool bottom_sync(unsigned *bar, int *flag) {
    __shared__ int gone;
    __syncthreads();
    if (threadIdx.x == 0) {
        gone = 0;
        volatile unsigned *gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long it = 0;
            while (*gen == g) {
                if (++it > BOT_WAIT_LIMIT) {
                    gone = 1;
                    atomicExch(flag, 1);
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return gone == 0;
}

// restriction (ratio 2) of F's residual into C's right-hand side, C's correction cleared
__device__ void bottom_restrict(const CoarseArgs &Fa, const Planes &F, const CoarseArgs &Ca, const Planes &C) {
    const long long total = C.nv * NCASE;
    for (long long t = blockIdx.x * (long long)BOT_T + threadIdx.x; t < total; t += (long long)gridDim.x * BOT_T) {
        const int c = (int)(t / C.nv);
        const long long v = t - (long long)c * C.nv;
        const int x = (int)(v % C.n[0]), y = (int)((v / C.n[0]) % C.n[1]), z = (int)(v / ((long long)C.n[0] * C.n[1]));
        const int xm = x == 0 ? C.n[0] - 1 : x - 1, ym = y == 0 ? C.n[1] - 1 : y - 1, zm = z == 0 ? C.n[2] - 1 : z - 1;
        const long long cpl = F.nv / 8;
        float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
        for (int ox = -1; ox <= 1; ox++)
#pragma unroll
            for (int oy = -1; oy <= 1; oy++)
#pragma unroll
                for (int oz = -1; oz <= 1; oz++) {
                    const float w = (float)((2 - abs(ox)) * (2 - abs(oy)) * (2 - abs(oz))) / 8.f;
                    const int k = ((ox + 1) & 1) | (((oy + 1) & 1) << 1) | (((oz + 1) & 1) << 2);
                    const long long fi = k * cpl + (ox < 0 ? xm : x) +
                                         (long long)C.n[0] * ((oy < 0 ? ym : y) + (long long)C.n[1] * (oz < 0 ? zm : z));
                    const float *src = Fa.r + fidx(3 * c, fi);
                    a0 = fmaf(__ldcg(&src[0]), w, a0);
                    a1 = fmaf(__ldcg(&src[FVB]), w, a1);
                    a2 = fmaf(__ldcg(&src[2 * FVB]), w, a2);
                }
        float *dst = const_cast<float *>(Ca.f) + fidx(3 * c, vidx(C, x, y, z));
        dst[0] = a0;
        dst[FVB] = a1;
        dst[2 * FVB] = a2;
    }
    const long long nu = field_floats(C.nv);
    for (long long t = blockIdx.x * (long long)BOT_T + threadIdx.x; t < nu; t += (long long)gridDim.x * BOT_T)
        Ca.u[t] = 0.f;
}

// trilinear prolongation (ratio 2) of C's correction into F's
__device__ void bottom_prolong(const CoarseArgs &Fa, const Planes &F, const CoarseArgs &Ca, const Planes &C) {
    for (long long t = blockIdx.x * (long long)BOT_T + threadIdx.x; t < C.nv; t += (long long)gridDim.x * BOT_T) {
        const int x = (int)(t % C.n[0]), y = (int)((t / C.n[0]) % C.n[1]), z = (int)(t / ((long long)C.n[0] * C.n[1]));
        const int xp = x + 1 == C.n[0] ? 0 : x + 1, yp = y + 1 == C.n[1] ? 0 : y + 1, zp = z + 1 == C.n[2] ? 0 : z + 1;
        long long ci[8];
#pragma unroll
        for (int id = 0; id < 8; ++id)
            ci[id] = vidx(C, (id & 1) ? xp : x, ((id >> 1) & 1) ? yp : y, (id >> 2) ? zp : z);
        const long long cpl = F.nv / 8;
        for (int pl = 0; pl < NF; ++pl) {
            float cv[8], fv[8];
#pragma unroll
            for (int id = 0; id < 8; ++id) cv[id] = __ldcg(&Ca.u[fidx(pl, ci[id])]);
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int ex = e & 1, ey = (e >> 1) & 1, ez = e >> 2;
                const int k = ((ex + 1) & 1) | (((ey + 1) & 1) << 1) | (((ez + 1) & 1) << 2);
                fv[e] = __ldcg(&Fa.u[fidx(pl, k * cpl + t)]);
            }
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int ex = e & 1, ey = (e >> 1) & 1, ez = e >> 2;
                float acc = 0.f;
#pragma unroll
                for (int id = 0; id < 8; ++id) {
                    const int ox = id & 1, oy = (id >> 1) & 1, oz = id >> 2;
                    const float w =
                        (float)((2 - abs(ox * 2 - ex)) * (2 - abs(oy * 2 - ey)) * (2 - abs(oz * 2 - ez))) / 8.f;
                    if (w == 0.f) continue;
                    acc = fmaf(cv[id], w, acc);
                }
                const int k = ((ex + 1) & 1) | (((ey + 1) & 1) << 1) | (((ez + 1) & 1) << 2);
                Fa.u[fidx(pl, k * cpl + t)] = fv[e] + acc;
            }
        }
    }
}

// one colour K of the sweep (two load cases per thread); RES: also the residual
template <bool F32, int K, bool RES>
__device__ void bottom_gs_k(const CoarseArgs &a) {
    constexpr int C = 2, NG = NCASE / C;
    constexpr bool res = RES;
    const long long nvb = (a.P + BOT_T - 1) / BOT_T * NG;
    for (long long b = blockIdx.x; b < nvb; b += gridDim.x) {
        const int cb = (int)(b % NG) * C;
        const long long p = (b / NG) * BOT_T + threadIdx.x;
        if (p >= a.P) continue;
        const long long me = (long long)K * a.P + p;
        int i, j, l;
        cplane_coords(a, p, i, j, l);
        float acc[3 * C], ks[9];
        coarse_apply<K, false, F32, C, true>(a, me, i, j, l, cb, acc);
        load_block<13, F32>(a, me, ks);
        const float w = a.w;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            float *u = a.u + fidx(3 * (cb + c), me);
            const float *f = a.f + fidx(3 * (cb + c), me);
            const float f0 = __ldcg(f), f1 = __ldcg(f + FVB), f2 = __ldcg(f + 2 * FVB);
            float u0 = __ldcg(u), u1 = __ldcg(u + FVB), u2 = __ldcg(u + 2 * FVB);
            u0 = w * (f0 - acc[3 * c] - ks[1] * u1 - ks[2] * u2) / ks[0] + (1.f - w) * u0;
            u1 = w * (f1 - acc[3 * c + 1] - ks[3] * u0 - ks[5] * u2) / ks[4] + (1.f - w) * u1;
            u2 = w * (f2 - acc[3 * c + 2] - ks[6] * u0 - ks[7] * u1) / ks[8] + (1.f - w) * u2;
            u[0] = u0;
            u[FVB] = u1;
            u[2 * FVB] = u2;
            if (res) {
                float *r = a.r + fidx(3 * (cb + c), me);
                const float ff[3] = {f0, f1, f2};
#pragma unroll
                for (int m = 0; m < 3; ++m)
                    r[m * FVB] = ff[m] - acc[3 * c + m] - fmaf(ks[3 * m + 2], u2, fmaf(ks[3 * m + 1], u1, ks[3 * m] * u0));
            }
        }
    }
}

template <bool F32>
__device__ void bottom_gs(const CoarseArgs &a, int K, bool res) {
    switch (K) {
    case 0: bottom_gs_k<F32, 0, false>(a); break;
    case 1: bottom_gs_k<F32, 1, false>(a); break;
    case 2: bottom_gs_k<F32, 2, false>(a); break;
    case 3: bottom_gs_k<F32, 3, false>(a); break;
    case 4: bottom_gs_k<F32, 4, false>(a); break;
    case 5: bottom_gs_k<F32, 5, false>(a); break;
    case 6: bottom_gs_k<F32, 6, false>(a); break;
    default:
        if (res) bottom_gs_k<F32, 7, true>(a);
        else bottom_gs_k<F32, 7, false>(a);
        break;
    }
}

// the residual of colours 0..6 (colour 7's came with its sweep)
template <bool F32>
__device__ void bottom_residual(const CoarseArgs &a) {
    constexpr int C = 2, NG = NCASE / C, NCOL = 7;
    const long long nvb = (a.P + BOT_T - 1) / BOT_T * NG * NCOL;
    for (long long b = blockIdx.x; b < nvb; b += gridDim.x) {
        const int K = (int)(b % NCOL);
        const long long bx = b / NCOL;
        const int cb = (int)(bx % NG) * C;
        const long long p = (bx / NG) * BOT_T + threadIdx.x;
        if (p >= a.P) continue;
        const long long me = (long long)K * a.P + p;
        int i, j, l;
        cplane_coords(a, p, i, j, l);
        float acc[3 * C];
        coarse_apply<-1, true, F32, C, true>(a, me, i, j, l, cb, acc, K);
#pragma unroll
        for (int q = 0; q < 3 * C; ++q) {
            const long long o = fidx(3 * cb + q, me);
            a.r[o] = __ldcg(a.f + o) - acc[q];
        }
    }
}

// the dense coarsest solve, one CTA per load case (the arithmetic of k_coarse_apply)
__device__ void bottom_coarsest(const BottomArgs &A, double *b) {
    const CoarseArgs &a = A.lv[A.nlv];
    const Planes &C = A.P[A.nlv];
    const int n = A.ndof;
    __shared__ double mean[3];
    for (int c = blockIdx.x; c < NCASE; c += gridDim.x) {
        for (int i = threadIdx.x; i < n; i += BOT_T) {
            const long long lex = i / 3;
            const int comp = i % 3;
            const int x = (int)(lex % C.n[0]), y = (int)((lex / C.n[0]) % C.n[1]),
                      z = (int)(lex / ((long long)C.n[0] * C.n[1]));
            b[i] = __ldcg(a.f + fidx(3 * c + comp, vidx(C, x, y, z)));
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            double sum = 0;
            if (A.project)
                for (int i = threadIdx.x; i < n; i += 3) sum += b[i];
            mean[threadIdx.x] = sum / (double)(n / 3);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += BOT_T) b[i] -= mean[i % 3];
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += BOT_T) {
            const double *row = A.aug + (long long)i * 2 * n + n;
            double sum = 0;
            for (int j = 0; j < n; j++) sum = fma(row[j], b[j], sum);
            const long long lex = i / 3;
            const int comp = i % 3;
            const int x = (int)(lex % C.n[0]), y = (int)((lex / C.n[0]) % C.n[1]),
                      z = (int)(lex / ((long long)C.n[0] * C.n[1]));
            a.u[fidx(3 * c + comp, vidx(C, x, y, z))] = (float)sum;
        }
        __syncthreads();
    }
}

template <bool F32>
__global__ void __launch_bounds__(BOT_T) k_vcycle_bottom(const __grid_constant__ BottomArgs A) {
    extern __shared__ double bot_b[];
    const int L = A.nlv;  // lv[1..L-1] smoothed, lv[L] the coarsest
    for (int l = 1; l < L; ++l) {
        bottom_restrict(A.lv[l - 1], A.P[l - 1], A.lv[l], A.P[l]);
        if (!bottom_sync(A.bar, A.flag)) return;
        for (int K = 0; K < 8; ++K) {
            bottom_gs<F32>(A.lv[l], K, K == 7);
            if (!bottom_sync(A.bar, A.flag)) return;
        }
        bottom_residual<F32>(A.lv[l]);
        if (!bottom_sync(A.bar, A.flag)) return;
    }
    bottom_restrict(A.lv[L - 1], A.P[L - 1], A.lv[L], A.P[L]);
    if (!bottom_sync(A.bar, A.flag)) return;
    bottom_coarsest(A, bot_b);
    if (!bottom_sync(A.bar, A.flag)) return;
    for (int l = L - 1; l >= 1; --l) {
        bottom_prolong(A.lv[l], A.P[l], A.lv[l + 1], A.P[l + 1]);
        if (!bottom_sync(A.bar, A.flag)) return;
        for (int K = 0; K < 8; ++K) {
            bottom_gs<F32>(A.lv[l], K, false);
            if (l > 1 || K < 7)
                if (!bottom_sync(A.bar, A.flag)) return;
        }
    }
}

// first: the first level of the bottom; levels first-1 .. nl-1 are passed
int launch_vcycle_bottom(const Level *lv, int first, int nl, const double *aug, int project, unsigned *bar, int *flag,
                         int nblk, cudaStream_t s) {
    BottomArgs A;
    A.nlv = nl - first;
    if (A.nlv < 1 || A.nlv > BOT_MAXLV || first < 1) return -1;
    for (int i = 0; i <= A.nlv; ++i) {
        A.lv[i] = make_cargs(lv[first - 1 + i]);
        A.P[i] = lv[first - 1 + i].P;
    }
    A.project = project;
    A.ndof = (int)(3 * lv[nl - 1].P.nv);
    A.aug = aug;
    A.bar = bar;
    A.flag = flag;
    const bool f32 = lv[first].st32;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.gridDim = dim3((unsigned)nblk);
    cfg.blockDim = dim3(BOT_T);
    cfg.dynamicSmemBytes = sizeof(double) * (size_t)A.ndof;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), s);
    const cudaError_t e = f32 ? cudaLaunchKernelEx(&cfg, k_vcycle_bottom<true>, A)
                              : cudaLaunchKernelEx(&cfg, k_vcycle_bottom<false>, A);
    return e == cudaSuccess ? 0 : -2;
}

// CTAs of the cooperative grid: all resident at once (blocks per SM from the
// occupancy query, at most four)
int vcycle_bottom_blocks(int num_sms, int ndof, bool f32) {
    int per = 0;
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per, f32 ? (const void *)k_vcycle_bottom<true> : (const void *)k_vcycle_bottom<false>, BOT_T,
        sizeof(double) * (size_t)ndof);
    if (e != cudaSuccess || per < 1) return 0;
    return num_sms;  // one CTA per SM: the fewest arrivals per barrier
}

// whether levels first..nl-2 can run in the bottom kernel: even smoothed levels,
// ratio 2 everywhere below `first - 1`, at most BOT_MAXLV levels
bool vcycle_bottom_fits(const Level *lv, int first, int nl) {
    if (first < 1 || nl - first < 1 || nl - first > BOT_MAXLV) return false;
    for (int l = first; l < nl; ++l) {
        if (lv[l].ratio[0] != 2 || lv[l].ratio[1] != 2 || lv[l].ratio[2] != 2) return false;
        if (!lv[l - 1].P.even) return false;
        if (l < nl - 1 && !lv[l].P.even) return false;
    }
    return true;
}

// ---- lockstep batches: a level (or a transfer) of several designs per launch ----
// Each design's CTAs run the body of its own launch with the CTA index inside its
// slice (BatchSlices), on its arguments staged in shared memory, so the results
// are those of the design's own launches to the last bit; designs whose flag in
// `active` is 0 return at once.  Sweeps and residuals in launch shape 0 (two cases
// per thread, 6 CTAs/SM).
constexpr int BATCH_CPT = 2, BATCH_MINB = 6;

struct CoarseEnt {
    CoarseArgs a;
    int design;
};
struct CoarseBatchTab {
    BatchSlices gs;   // CTAs of one colour of the sweep, two cases per thread
    BatchSlices gs6;  // the same with six cases per thread
    BatchSlices res;  // CTAs of the seven-colour residual
    CoarseEnt e[BATCH_MAX];
};

// C cases per thread at MB CTAs per SM: launch shape 0 (C = 2, 6 CTAs/SM) or 1
// (C = 6, 4 CTAs/SM)
template <int K, bool F32, bool RES, int C, int MB>
__global__ void __launch_bounds__(128, MB) k_coarse_gs_batch(const CoarseBatchTab *__restrict__ t,
                                                           const int *__restrict__ active) {
    __shared__ __align__(16) unsigned buf[sizeof(CoarseArgs) / 4];
    const BatchSlices &sl = C == BATCH_CPT ? t->gs : t->gs6;
    const int i = batch_slice(sl, blockIdx.x);
    const CoarseEnt &en = t->e[i];
    if (!__ldg(&active[en.design])) return;
    const CoarseArgs &a = stage_args(en.a, buf);
    coarse_gs_block<K, F32, C, RES>(a, blockIdx.x - __ldg(&sl.start[i]));
}

template <bool F32>
__global__ void __launch_bounds__(128, BATCH_MINB) k_coarse_residual_batch(const CoarseBatchTab *__restrict__ t,
                                                                         const int *__restrict__ active) {
    __shared__ __align__(16) unsigned buf[sizeof(CoarseArgs) / 4];
    const int i = batch_slice(t->res, blockIdx.x);
    const CoarseEnt &en = t->e[i];
    if (!__ldg(&active[en.design])) return;
    const CoarseArgs &a = stage_args(en.a, buf);
    coarse_residual_block<F32, BATCH_CPT, 7>(a, blockIdx.x - __ldg(&t->res.start[i]));
}

template <typename Tab>
static int upload_tab(const Tab &t, int n, BatchTab *out) {
    void *d = nullptr;
    if (cudaMalloc(&d, sizeof(Tab)) != cudaSuccess) return -2;
    if (cudaMemcpy(d, &t, sizeof(Tab), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d);
        return -2;
    }
    out->dev = d;
    out->n = n;
    return 0;
}

int coarse_batch_create(const Level *const *lv, const int *design, int n, bool scratch, BatchTab *out) {
    if (n < 1 || n > BATCH_MAX) return -1;
    CoarseBatchTab *t = new CoarseBatchTab();
    t->gs.n = t->gs6.n = t->res.n = n;
    t->gs.start[0] = t->gs6.start[0] = t->res.start[0] = 0;
    for (int i = 0; i < n; i++) {
        t->e[i].a = make_cargs(*lv[i]);
        if (scratch) t->e[i].a.u = t->e[i].a.r;
        t->e[i].design = design[i];
        const unsigned vb = (unsigned)((t->e[i].a.P + 127) / 128), nb = vb * (NCASE / BATCH_CPT);
        t->gs.start[i + 1] = t->gs.start[i] + nb;
        t->gs6.start[i + 1] = t->gs6.start[i] + vb;
        t->res.start[i + 1] = t->res.start[i] + nb * 7;
    }
    const int rc = upload_tab(*t, n, out);
    if (rc == 0) {
        out->grid[0] = t->gs.start[n];
        out->grid[1] = t->res.start[n];
        out->grid[2] = t->gs6.start[n];
    }
    delete t;
    return rc;
}

template <bool F32, int C, int MB>
static void coarse_sweep_batch(const BatchTab &t, const int *active, bool residual, cudaStream_t s) {
    const CoarseBatchTab *d = static_cast<const CoarseBatchTab *>(t.dev);
    const unsigned g = C == BATCH_CPT ? t.grid[0] : t.grid[2];
    k_coarse_gs_batch<0, F32, false, C, MB><<<g, 128, 0, s>>>(d, active);
    k_coarse_gs_batch<1, F32, false, C, MB><<<g, 128, 0, s>>>(d, active);
    k_coarse_gs_batch<2, F32, false, C, MB><<<g, 128, 0, s>>>(d, active);
    k_coarse_gs_batch<3, F32, false, C, MB><<<g, 128, 0, s>>>(d, active);
    k_coarse_gs_batch<4, F32, false, C, MB><<<g, 128, 0, s>>>(d, active);
    k_coarse_gs_batch<5, F32, false, C, MB><<<g, 128, 0, s>>>(d, active);
    k_coarse_gs_batch<6, F32, false, C, MB><<<g, 128, 0, s>>>(d, active);
    if (residual) {
        k_coarse_gs_batch<7, F32, true, C, MB><<<g, 128, 0, s>>>(d, active);
        k_coarse_residual_batch<F32><<<t.grid[1], 128, 0, s>>>(d, active);
    } else {
        k_coarse_gs_batch<7, F32, false, C, MB><<<g, 128, 0, s>>>(d, active);
    }
}

void launch_coarse_sweep_batch(const BatchTab &t, bool f32, const int *active, bool residual, int shape,
                               cudaStream_t s) {
    if (f32) {
        if (shape == 1) coarse_sweep_batch<true, 6, 4>(t, active, residual, s);
        else coarse_sweep_batch<true, BATCH_CPT, BATCH_MINB>(t, active, residual, s);
    } else {
        if (shape == 1) coarse_sweep_batch<false, 6, 4>(t, active, residual, s);
        else coarse_sweep_batch<false, BATCH_CPT, BATCH_MINB>(t, active, residual, s);
    }
}

// ratio-2 transfers: one slice of ceil(C.nv / 256) CTAs per design for both
struct TransferEnt {
    Planes F, C;
    FastDiv dn0, dn1;   // division by C.n[0], C.n[1]
    const float *rf;    // F.r
    float *fc, *uc;     // C.f, C.u
    float *uf;          // F.u
    int design;
    int pad;
};
struct TransferBatchTab {
    BatchSlices sl;
    TransferEnt e[BATCH_MAX];
};

__global__ void __launch_bounds__(256) k_restrict_batch(const TransferBatchTab *__restrict__ t,
                                                        const int *__restrict__ active) {
    __shared__ __align__(16) unsigned buf[sizeof(TransferEnt) / 4];
    const int i = batch_slice(t->sl, blockIdx.x);
    if (!__ldg(&active[t->e[i].design])) return;
    const TransferEnt &e = stage_args(t->e[i], buf);
    const long long tt = (long long)(blockIdx.x - __ldg(&t->sl.start[i])) * blockDim.x + threadIdx.x;
    restrict2_thread(e.F, e.C, e.dn0, e.dn1, e.rf, e.fc, e.uc, tt, blockIdx.y);
}

__global__ void __launch_bounds__(256) k_prolong_batch(const TransferBatchTab *__restrict__ t,
                                                       const int *__restrict__ active, int is_root) {
    __shared__ __align__(16) unsigned buf[sizeof(TransferEnt) / 4];
    const int i = batch_slice(t->sl, blockIdx.x);
    if (!__ldg(&active[t->e[i].design])) return;
    const TransferEnt &e = stage_args(t->e[i], buf);
    const long long tt = (long long)(blockIdx.x - __ldg(&t->sl.start[i])) * blockDim.x + threadIdx.x;
    prolong2_thread(e.F, e.C, e.dn0, e.dn1, is_root, e.uc, e.uf, tt);
}

int transfer_batch_create(const Level *const *F, const Level *const *C, const int *design, int n, BatchTab *out) {
    if (n < 1 || n > BATCH_MAX) return -1;
    TransferBatchTab *t = new TransferBatchTab();
    t->sl.n = n;
    t->sl.start[0] = 0;
    for (int i = 0; i < n; i++) {
        TransferEnt &e = t->e[i];
        e.F = F[i]->P;
        e.C = C[i]->P;
        e.dn0 = FastDiv((unsigned)C[i]->P.n[0]);
        e.dn1 = FastDiv((unsigned)C[i]->P.n[1]);
        e.rf = F[i]->r;
        e.fc = C[i]->f;
        e.uc = C[i]->u;
        e.uf = F[i]->u;
        e.design = design[i];
        t->sl.start[i + 1] = t->sl.start[i] + (unsigned)((C[i]->P.nv + 255) / 256);
    }
    const int rc = upload_tab(*t, n, out);
    if (rc == 0) out->grid[0] = t->sl.start[n];
    delete t;
    return rc;
}

void launch_restrict_batch(const BatchTab &t, const int *active, cudaStream_t s) {
    k_restrict_batch<<<dim3(t.grid[0], NCASE), 256, 0, s>>>(static_cast<const TransferBatchTab *>(t.dev), active);
}

void launch_prolong_batch(const BatchTab &t, const int *active, int is_root, cudaStream_t s) {
    k_prolong_batch<<<t.grid[0], 256, 0, s>>>(static_cast<const TransferBatchTab *>(t.dev), active, is_root);
}

// per-case norms: the first stage (NORM_FINISH_CHUNKS CTAs) for designs above
// NORM_FINISH_DIRECT partials, then one CTA per design
struct NormEnt {
    const double *partial;
    double *mid;  // the first stage's sums behind the partials (two-stage designs)
    int nblk, per, two, design;
};
struct NormBatchTab {
    BatchSlices chunks;  // first-stage CTAs (none for one-stage designs)
    NormEnt e[BATCH_MAX];
};

__global__ void __launch_bounds__(256) k_finish_chunks_batch(const NormBatchTab *__restrict__ t,
                                                             const int *__restrict__ active) {
    const int i = batch_slice(t->chunks, blockIdx.x);
    const NormEnt &e = t->e[i];
    if (!__ldg(&active[e.design])) return;
    finish_chunk_block<NCASE>(e.partial, e.nblk, e.per, e.mid, (int)(blockIdx.x - __ldg(&t->chunks.start[i])));
}

__global__ void __launch_bounds__(256) k_finish_batch(const NormBatchTab *__restrict__ t, const int *__restrict__ active,
                                                      double *out) {
    const NormEnt &e = t->e[blockIdx.x];
    if (!__ldg(&active[e.design])) return;
    if (e.two) finish_block<NCASE>(e.mid, NORM_FINISH_CHUNKS, out + (long long)NCASE * e.design);
    else finish_block<NCASE>(e.partial, e.nblk, out + (long long)NCASE * e.design);
}

int norm_batch_create(double *const *partial, const int *nblk, const int *design, int n, BatchTab *out) {
    if (n < 1 || n > BATCH_MAX) return -1;
    NormBatchTab *t = new NormBatchTab();
    t->chunks.n = n;
    t->chunks.start[0] = 0;
    for (int i = 0; i < n; i++) {
        NormEnt &e = t->e[i];
        e.partial = partial[i];
        e.nblk = nblk[i];
        e.two = nblk[i] > NORM_FINISH_DIRECT;
        e.per = (nblk[i] + NORM_FINISH_CHUNKS - 1) / NORM_FINISH_CHUNKS;
        e.mid = partial[i] + (long long)nblk[i] * NCASE;
        e.design = design[i];
        t->chunks.start[i + 1] = t->chunks.start[i] + (e.two ? NORM_FINISH_CHUNKS : 0);
    }
    const int rc = upload_tab(*t, n, out);
    if (rc == 0) out->grid[0] = t->chunks.start[n];
    delete t;
    return rc;
}

void launch_norm_finish_batch(const BatchTab &t, const int *active, double *out, cudaStream_t s) {
    const NormBatchTab *d = static_cast<const NormBatchTab *>(t.dev);
    if (t.grid[0] > 0) k_finish_chunks_batch<<<t.grid[0], 256, 0, s>>>(d, active);
    k_finish_batch<<<t.n, 256, 0, s>>>(d, active, out);
}

}  // namespace h3d
