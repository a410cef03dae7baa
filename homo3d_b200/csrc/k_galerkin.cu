// k_galerkin.cu -- Galerkin coarse operators and the coarsest-grid dense solve.
//
// Reference behaviour restated (homo3d):
//   restrict_stencil_otf_aos_kernel_1 (grid_ex.cu:936-1060): level-1 stencils
//     R K(rho) P computed from the fine densities (rho^p, no 1e-9 floor) for the
//     lexicographic vertices 0..n_c per axis, elements clipped to the domain, the
//     self block's diagonal clamped to >= 1e-4, stored FP16; the periodic images
//     of a vertex on a min face are then summed in FP16 (grid.cu:2741-2772 ->
//     grid.cu:3103-3176).  On B200 the triple loop over fine elements is replaced
//     by the exact refactoring into coarse element matrices
//     K_E = sum_s rho_s P_s^T Ke P_s (Q_s = P_s^T Ke P_s precomputed), and the
//     images become the subsets of the 8 coarse elements around the vertex.
//   restrict_stencil_arround_dirichelt_boundary (grid.cpp:1184-1325): the 27
//     coarse vertices around the pinned fine origin use the pinned fine operator
//     (identity at the origin node, 1e-9 floor) in double precision.  With
//     pin_identity = 0 the identity is left out, which makes the coarse operator
//     the exact Galerkin product of the pinned fine operator.
//   restrict_stencil_aos_kernel_1 (grid_ex.cu:1065-1160): deeper levels R A P
//     from the FP16 finer stencil.
//   solveHostEquation / assembleHostMatrix (grid.cpp:349-424): coarsest level.
//     Replaced by a dense FP64 inverse built on the device (Gauss-Jordan with
//     partial pivoting) and applied as a GEMV per load case.
#include "h3d_internal.cuh"

namespace h3d {

__device__ __forceinline__ int modp(int a, int n) { return ((a % n) + n) % n; }

// ---- level 1 from densities ---------------------------------------------------
// R = 2 on every axis is compiled with the sub-element loop unrolled; R = 0 is
// the generic path for ratio 4 (or mixed ratios).
template <int R, bool F32>
__global__ void __launch_bounds__(128) k_galerkin_l1(Planes F, Planes C, int r0, int r1, int r2,
                                                     const float *__restrict__ rho, const float *__restrict__ q,
                                                     int nsub, uint4 *st) {
    extern __shared__ float sq[];
    for (int i = threadIdx.x; i < nsub * 576; i += blockDim.x) sq[i] = q[i];
    __syncthreads();
    const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v >= C.nv) return;
    if (R == 2) { r0 = r1 = r2 = 2; nsub = 8; }
    const int k = color_of_index(C, v);
    int X[3];
    vpos(C, k, v - C.base[k], X[0], X[1], X[2]);
    const int bmask = (X[0] == 0 ? 4 : 0) | (X[1] == 0 ? 2 : 0) | (X[2] == 0 ? 1 : 0);
    // lexicographic index of fine element (E*r + s) for the coarse element E = X - l
    long long ebase[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        const int ex = wrap(X[0] - (l & 1), C.n[0]) * r0, ey = wrap(X[1] - ((l >> 1) & 1), C.n[1]) * r1,
                  ez = wrap(X[2] - (l >> 2), C.n[2]) * r2;
        ebase[l] = ex + (long long)F.n[0] * (ey + (long long)F.n[1] * ez);
    }
    uint32_t cbuf[4] = {0, 0, 0, 0};
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        const int dx = d % 3 - 1, dy = d / 3 % 3 - 1, dz = d / 9 - 1;
        // the images are summed in the storage precision (FP16: grid.cu:3103-3176)
        float res[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) res[e] = 0.f;
        for (int img = 0; img < 8; ++img) {
            if (img & ~bmask) continue;
            float p[9];
#pragma unroll
            for (int e = 0; e < 9; ++e) p[e] = 0.f;
#pragma unroll
            for (int l = 0; l < 8; ++l) {
                const int lx = l & 1, ly = (l >> 1) & 1, lz = l >> 2;
                const int mx = lx + dx, my = ly + dy, mz = lz + dz;
                if (mx < 0 || mx > 1 || my < 0 || my > 1 || mz < 0 || mz > 1) continue;
                const int m = mx + 2 * my + 4 * mz;
                const int limg = ((lx << 2) | (ly << 1) | lz) & bmask;
                if (limg != img) continue;
                if (R == 2) {
#pragma unroll
                    for (int s = 0; s < 8; ++s) {
                        const long long fe = ebase[l] + (s & 1) + (long long)F.n[0] * (((s >> 1) & 1) + (long long)F.n[1] * (s >> 2));
                        const float rp = __ldg(&rho[fe]);
                        const float *Q = sq + s * 576;
#pragma unroll
                        for (int i = 0; i < 3; ++i)
#pragma unroll
                            for (int j = 0; j < 3; ++j) p[3 * i + j] = fmaf(rp, Q[(3 * l + i) * 24 + 3 * m + j], p[3 * i + j]);
                    }
                } else {
                    for (int s = 0; s < nsub; ++s) {
                        const int sx = s % r0, sy = (s / r0) % r1, sz = s / (r0 * r1);
                        const long long fe = ebase[l] + sx + (long long)F.n[0] * (sy + (long long)F.n[1] * sz);
                        const float rp = __ldg(&rho[fe]);
                        const float *Q = sq + s * 576;
#pragma unroll
                        for (int i = 0; i < 3; ++i)
#pragma unroll
                            for (int j = 0; j < 3; ++j) p[3 * i + j] = fmaf(rp, Q[(3 * l + i) * 24 + 3 * m + j], p[3 * i + j]);
                    }
                }
            }
            if (d == 13) {
#pragma unroll
                for (int t = 0; t < 3; ++t)
                    if (fabsf(p[4 * t]) < 1e-4f) p[4 * t] = 1e-4f;
            }
#pragma unroll
            for (int e = 0; e < 9; ++e)
                res[e] = F32 ? res[e] + p[e] : __half2float(__hadd(__float2half_rn(res[e]), __float2half_rn(p[e])));
        }
        // stream the 9 entries into the packed chunks
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            const int g = 9 * d + e;
            if (F32) {
                cbuf[g & 3] = __float_as_uint(res[e]);
                if ((g & 3) == 3 || g == 242) {
                    if (g == 242) cbuf[3] = 0;  // entries 240..242 and the pad
                    st[(long long)(g >> 2) * C.nv + v] = make_uint4(cbuf[0], cbuf[1], cbuf[2], cbuf[3]);
                }
            } else {
                const uint32_t hv = (uint32_t)__half_as_ushort(__float2half_rn(res[e]));
                const int slot = (g & 7) >> 1;
                if (g & 1) cbuf[slot] |= hv << 16;
                else cbuf[slot] = hv;
                if ((g & 7) == 7 || g == 242) {
                    if (g == 242) { cbuf[1] &= 0xffffu; cbuf[2] = 0; cbuf[3] = 0; }
                    st[(long long)(g >> 3) * C.nv + v] = make_uint4(cbuf[0], cbuf[1], cbuf[2], cbuf[3]);
                }
            }
        }
    }
}

void launch_galerkin_l1(const Level &F, const Level &C, const float *rho, const float *q, int nsub, cudaStream_t s) {
    const int bs = 128;
    const unsigned nb = (unsigned)((C.P.nv + bs - 1) / bs);
    const size_t smem = (size_t)nsub * 576 * sizeof(float);
    if (C.ratio[0] == 2 && C.ratio[1] == 2 && C.ratio[2] == 2) {
        if (C.st32) k_galerkin_l1<2, true><<<nb, bs, smem, s>>>(F.P, C.P, 2, 2, 2, rho, q, nsub, C.st);
        else k_galerkin_l1<2, false><<<nb, bs, smem, s>>>(F.P, C.P, 2, 2, 2, rho, q, nsub, C.st);
    } else {
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k_galerkin_l1<0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            cudaFuncSetAttribute(k_galerkin_l1<0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            attr = true;
        }
        if (C.st32)
            k_galerkin_l1<0, true><<<nb, bs, smem, s>>>(F.P, C.P, C.ratio[0], C.ratio[1], C.ratio[2], rho, q, nsub, C.st);
        else
            k_galerkin_l1<0, false><<<nb, bs, smem, s>>>(F.P, C.P, C.ratio[0], C.ratio[1], C.ratio[2], rho, q, nsub,
                                                         C.st);
    }
}

// ---- the 27 coarse vertices around the pinned fine origin -----------------------
__device__ __forceinline__ double hat_w(int ox, int oy, int oz, int r0, int r1, int r2) {
    ox = abs(ox); oy = abs(oy); oz = abs(oz);
    if (ox >= r0 || oy >= r1 || oz >= r2) return 0.0;
    return (double)((r0 - ox) * (r1 - oy) * (r2 - oz)) / (double)(r0 * r1 * r2);
}

// one CTA per (coarse vertex offset vi in {-1,0,1}^3, neighbour d); its threads
// share the fine elements of the (2r)^3 box around the neighbour (one each for
// ratio 2 and 4, a fixed strided set above that) and the contributions are summed
// in a fixed tree order
constexpr int PATCH_MAX_THREADS = 512;
template <bool F32>
__global__ void __launch_bounds__(PATCH_MAX_THREADS) k_dirichlet_patch(Planes F, Planes C, int r0, int r1, int r2,
                                                                       const float *__restrict__ rho,
                                                                       const double *__restrict__ ked, int pin_identity,
                                                                       uint4 *st) {
    __shared__ double red[PATCH_MAX_THREADS][9];
    const int vi = blockIdx.x / 27, d = blockIdx.x % 27;
    const int vio[3] = {(vi % 3 - 1), (vi / 3 % 3 - 1), (vi / 9 - 1)};
    const int pi[3] = {vio[0] * r0, vio[1] * r1, vio[2] * r2};
    const int pj[3] = {pi[0] + (d % 3 - 1) * r0, pi[1] + (d / 3 % 3 - 1) * r1, pi[2] + (d / 9 - 1) * r2};
    const int tid = threadIdx.x;
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int e = tid; e < 8 * r0 * r1 * r2; e += blockDim.x) {  // this thread's elements, in order
    const int ex = e % (2 * r0) - r0, ey = (e / (2 * r0)) % (2 * r1) - r1, ez = e / (4 * r0 * r1) - r2;
    const int ep[3] = {pj[0] + ex, pj[1] + ey, pj[2] + ez};
    const int eo[3] = {ep[0] - pi[0], ep[1] - pi[1], ep[2] - pi[2]};
    if (!(eo[0] >= r0 || eo[0] < -r0 || eo[1] >= r1 || eo[1] < -r1 || eo[2] >= r2 || eo[2] < -r2)) {
        const long long fe =
            modp(ep[0], F.n[0]) + (long long)F.n[0] * (modp(ep[1], F.n[1]) + (long long)F.n[1] * modp(ep[2], F.n[2]));
        const double rp = 1e-9 + (double)rho[fe];
        for (int a = 0; a < 8; a++) {
            const int ap[3] = {ep[0] + (a & 1), ep[1] + ((a >> 1) & 1), ep[2] + (a >> 2)};
            const double wi = hat_w(ap[0] - pi[0], ap[1] - pi[1], ap[2] - pi[2], r0, r1, r2);
            if (wi == 0) continue;
            const bool ad = ap[0] == 0 && ap[1] == 0 && ap[2] == 0;
            for (int b = 0; b < 8; b++) {
                const int bp[3] = {ep[0] + (b & 1), ep[1] + ((b >> 1) & 1), ep[2] + (b >> 2)};
                const double wj = hat_w(bp[0] - pj[0], bp[1] - pj[1], bp[2] - pj[2], r0, r1, r2);
                if (wj == 0) continue;
                const bool bd = bp[0] == 0 && bp[1] == 0 && bp[2] == 0;
                if (ad || bd) {
                    if (a == b && pin_identity)
                        for (int i = 0; i < 3; i++) s[4 * i] += wi * wj;
                } else {
                    for (int i = 0; i < 3; i++)
                        for (int j = 0; j < 3; j++) s[3 * i + j] += wi * wj * rp * ked[(3 * a + i) * 24 + 3 * b + j];
                }
            }
        }
    }
    }
#pragma unroll
    for (int k = 0; k < 9; k++) red[tid][k] = s[k];
    __syncthreads();
    for (int half = blockDim.x / 2; half > 0; half /= 2) {  // blockDim.x is a power of two
        if (tid < half)
#pragma unroll
            for (int k = 0; k < 9; k++) red[tid][k] += red[tid + half][k];
        __syncthreads();
    }
    if (tid != 0) return;
    double t[9];
#pragma unroll
    for (int k = 0; k < 9; k++) t[k] = red[0][k];
    if (d == 13)
        for (int i = 0; i < 3; i++)
            if (fabs(t[4 * i]) < 1e-4) t[4 * i] = 1e-4;
    const long long v = vidx(C, modp(vio[0], C.n[0]), modp(vio[1], C.n[1]), modp(vio[2], C.n[2]));
    for (int e = 0; e < 9; e++) StencilStore<F32>::putd(st, C.nv, v, 9 * d + e, t[e]);
}

void launch_dirichlet_patch(const Level &F, const Level &C, const float *rho, const double *ked, int pin_identity,
                            cudaStream_t s) {
    int nt = 8 * C.ratio[0] * C.ratio[1] * C.ratio[2];  // (2r)^3 elements, a power of two
    if (nt > PATCH_MAX_THREADS) nt = PATCH_MAX_THREADS;
    if (C.st32)
        k_dirichlet_patch<true><<<27 * 27, nt, 0, s>>>(F.P, C.P, C.ratio[0], C.ratio[1], C.ratio[2], rho, ked,
                                                       pin_identity, C.st);
    else
        k_dirichlet_patch<false><<<27 * 27, nt, 0, s>>>(F.P, C.P, C.ratio[0], C.ratio[1], C.ratio[2], rho, ked,
                                                        pin_identity, C.st);
}

// ---- deeper levels: R A P from the finer stencil -----------------------------------
// the 9 entries of block J of fine vertex fv (compile-time J: fixed chunk slots)
template <int J, bool F32>
__device__ __forceinline__ void fine_block(const uint4 *__restrict__ st, long long nv, long long fv, float b[9]) {
    using S = StencilStore<F32>;
    constexpr int e0 = 9 * J, q0 = e0 / S::PER, q1 = (e0 + 8) / S::PER;
    float v[3 * S::PER];
#pragma unroll
    for (int q = q0; q <= q1; ++q) S::unpack(__ldg(st + q * nv + fv), v + (q - q0) * S::PER);
#pragma unroll
    for (int k = 0; k < 9; ++k) b[k] = v[e0 + k - S::PER * q0];
}

// One thread per (coarse vertex, coarse neighbour d): block d of the coarse
// stencil is sum over fine i in the support of the vertex and fine j in the
// support of neighbour d of w_i w_j A_ij.  The fine offsets are visited in the
// order x, y, z (z fastest) and the fine neighbours j in ascending order.  With
// dminor, d is the block index modulo 27, so the 27 CTAs of one block of coarse
// vertices run together and read the same fine stencil rows while they are in
// L2: for a finer stencil far larger than L2 (128^3 vertices, 1 GB) that is 9 %
// faster than d as the second grid dimension, which streams the finer stencil
// once per d; for smaller ones, where the stencil nearly fits in L2, it is slower
// (the 27 d of a vertex block have very different loop lengths).
template <bool F32>
__global__ void __launch_bounds__(128) k_galerkin(Planes F, Planes C, int r0, int r1, int r2,
                                                  const uint4 *__restrict__ fst, uint4 *cst, int dminor) {
    const int d = dminor ? (int)(blockIdx.x % 27u) : (int)blockIdx.y;
    const long long v = (dminor ? blockIdx.x / 27u : blockIdx.x) * (long long)blockDim.x + threadIdx.x;
    if (v >= C.nv) return;
    const int k = color_of_index(C, v);
    int X[3];
    vpos(C, k, v - C.base[k], X[0], X[1], X[2]);
    const float pr = (float)(r0 * r1 * r2);
    const int dj0 = r0 * (d % 3 - 1), dj1 = r1 * (d / 3 % 3 - 1), dj2 = r2 * (d / 9 - 1);
    float s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    // fine offsets oi from the coarse vertex with |oi| < r and |oi - dj| <= r
    const int a0 = max(-r0 + 1, dj0 - r0), b0 = min(r0 - 1, dj0 + r0);
    const int a1 = max(-r1 + 1, dj1 - r1), b1 = min(r1 - 1, dj1 + r1);
    const int a2 = max(-r2 + 1, dj2 - r2), b2 = min(r2 - 1, dj2 + r2);
    for (int o0 = a0; o0 <= b0; o0++)
        for (int o1 = a1; o1 <= b1; o1++)
            for (int o2 = a2; o2 <= b2; o2++) {
                const long long fv = vidx(F, modp(X[0] * r0 + o0, F.n[0]), modp(X[1] * r1 + o1, F.n[1]),
                                          modp(X[2] * r2 + o2, F.n[2]));
                const float wi = (float)((r0 - abs(o0)) * (r1 - abs(o1)) * (r2 - abs(o2))) / pr;
#pragma unroll
                for (int j = 0; j < 27; j++) {
                    const int q0 = abs(o0 + j % 3 - 1 - dj0), q1 = abs(o1 + j / 3 % 3 - 1 - dj1),
                              q2 = abs(o2 + j / 9 - 1 - dj2);
                    if (q0 >= r0 || q1 >= r1 || q2 >= r2) continue;
                    const float wj = (float)((r0 - q0) * (r1 - q1) * (r2 - q2)) / pr;
                    const float ww = wi * wj;
                    float bl[9];
                    switch (j) {  // compile-time block index for the chunk arithmetic
#define H3D_FB(J) case J: fine_block<J, F32>(fst, F.nv, fv, bl); break;
                        H3D_FB(0) H3D_FB(1) H3D_FB(2) H3D_FB(3) H3D_FB(4) H3D_FB(5) H3D_FB(6) H3D_FB(7) H3D_FB(8)
                        H3D_FB(9) H3D_FB(10) H3D_FB(11) H3D_FB(12) H3D_FB(13) H3D_FB(14) H3D_FB(15) H3D_FB(16)
                        H3D_FB(17) H3D_FB(18) H3D_FB(19) H3D_FB(20) H3D_FB(21) H3D_FB(22) H3D_FB(23) H3D_FB(24)
                        H3D_FB(25) H3D_FB(26)
#undef H3D_FB
                    }
#pragma unroll
                    for (int e = 0; e < 9; e++) s[e] = fmaf(ww, bl[e], s[e]);
                }
            }
    if (d == 13)
        for (int t = 0; t < 3; t++)
            if (fabsf(s[4 * t]) < 1e-4f) s[4 * t] = 1e-4f;
    for (int e = 0; e < 9; e++) StencilStore<F32>::put(cst, C.nv, v, 9 * d + e, s[e]);
}

void launch_galerkin(const Level &F, const Level &C, cudaStream_t s) {
    const int bs = 128;
    const unsigned nb = (unsigned)((C.P.nv + bs - 1) / bs);
    const int dminor = F.P.nv >= (1LL << 21);
    const dim3 grid = dminor ? dim3(nb * 27u, 1) : dim3(nb, 27);
    if (C.st32) k_galerkin<true><<<grid, bs, 0, s>>>(F.P, C.P, C.ratio[0], C.ratio[1], C.ratio[2], F.st, C.st, dminor);
    else k_galerkin<false><<<grid, bs, 0, s>>>(F.P, C.P, C.ratio[0], C.ratio[1], C.ratio[2], F.st, C.st, dminor);
}

// ---- coarsest level ---------------------------------------------------------------
// aug: [n][2n] row-major, left = K over unique DOFs (3*lexid + comp), right = I.
// One thread per row (vertex lex, component i) adds its 27 neighbour blocks in
// neighbour order d = 0..26, so entries that several periodic images of one
// neighbour fall on (grids of two or three cells per axis) are summed in a fixed
// order and the coarsest inverse is the same from run to run.
template <bool F32>
__global__ void k_coarse_assemble(Planes C, const uint4 *__restrict__ st, double *aug, int n) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= C.nv * 3) return;
    const long long lex = t / 3;
    const int i = (int)(t % 3);
    const int x = (int)(lex % C.n[0]);
    const int y = (int)((lex / C.n[0]) % C.n[1]), z = (int)(lex / ((long long)C.n[0] * C.n[1]));
    const long long v = vidx(C, x, y, z);
    double *row = aug + (3 * lex + i) * (2LL * n);
    for (int d = 0; d < 27; d++) {
        const int wx = wrap(x + d % 3 - 1, C.n[0]), wy = wrap(y + d / 3 % 3 - 1, C.n[1]), wz = wrap(z + d / 9 - 1, C.n[2]);
        const long long w = wx + (long long)C.n[0] * (wy + (long long)C.n[1] * wz);
        for (int j = 0; j < 3; j++) row[3 * w + j] += (double)StencilStore<F32>::get(st, C.nv, v, 9 * d + 3 * i + j);
    }
    row[n + 3 * lex + i] = 1.0;
}

void launch_coarse_assemble(const Level &C, double *aug, cudaStream_t s) {
    const int n = (int)(3 * C.P.nv);
    cudaMemsetAsync(aug, 0, sizeof(double) * (size_t)n * 2 * n, s);
    const long long nt = C.P.nv * 3;
    if (C.st32) k_coarse_assemble<true><<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(C.P, C.st, aug, n);
    else k_coarse_assemble<false><<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(C.P, C.st, aug, n);
}

// Gauss-Jordan elimination with partial pivoting on [K | I] (n rows, 2n columns,
// FP64; grid.cpp:385-424 inverts the same matrix on the host).  One launch per
// pivot column spreads the rank-1 update over every SM; the pivot search, row
// swap and scaling of the next column are done by whichever CTA of a launch
// finishes last (an arrival counter, no waiting), so a factorisation is n + 1
// launches.  Scratch behind the matrix: the n elimination factors of the current
// column and the arrival counter.
constexpr int GJ_THREADS = 256;
constexpr int GJ_TC = 64;                          // tile columns (lanes of a row)
constexpr int GJ_RPT = 8;                          // rows per thread
constexpr int GJ_TR = GJ_RPT * GJ_THREADS / GJ_TC; // tile rows

// pivot step of column k by one CTA: the row among k..n-1 with the largest |a_ik|
// (ties: the lowest row) swapped into row k and scaled by 1 / a_kk; col_i = a_ik
// (0 for the pivot row) for the elimination launch of column k
__device__ void gj_pivot(double *a, int n, int k, double *col, int *flag) {
    __shared__ double rmax[GJ_THREADS / 32];
    __shared__ int ridx[GJ_THREADS / 32];
    __shared__ int piv;
    const int tid = threadIdx.x, m = 2 * n;
    double best = -1.0;
    int bi = k;
    for (int i = k + tid; i < n; i += GJ_THREADS) {
        const double v = fabs(__ldcg(&a[(long long)i * m + k]));
        if (v > best) { best = v; bi = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if ((tid & 31) == 0) { rmax[tid >> 5] = best; ridx[tid >> 5] = bi; }
    __syncthreads();
    if (tid == 0) {
        double b = -1.0;
        int p = k;
        for (int w = 0; w < GJ_THREADS / 32; w++)
            if (rmax[w] > b || (rmax[w] == b && ridx[w] < p)) { b = rmax[w]; p = ridx[w]; }
        piv = p;
        if (!(b > 0.0)) *flag = 1;
    }
    __syncthreads();
    const int p = piv;
    if (p != k)
        for (int j = k + tid; j < m; j += GJ_THREADS) {
            const double t = __ldcg(&a[(long long)k * m + j]);
            a[(long long)k * m + j] = __ldcg(&a[(long long)p * m + j]);
            a[(long long)p * m + j] = t;
        }
    __syncthreads();
    const double inv = 1.0 / __ldcg(&a[(long long)k * m + k]);
    __syncthreads();
    for (int j = k + tid; j < m; j += GJ_THREADS) a[(long long)k * m + j] = __ldcg(&a[(long long)k * m + j]) * inv;
    for (int i = tid; i < n; i += GJ_THREADS) col[i] = (i == k) ? 0.0 : __ldcg(&a[(long long)i * m + k]);
}

__global__ void __launch_bounds__(GJ_THREADS) k_gj_first(double *a, int n, double *col, int *flag) {
    gj_pivot(a, n, 0, col, flag);
}

// elimination of column k from every other row over columns k..2n-1
// (a_ij -= col_i a_kj), then the pivot step of column k + 1 by the last CTA
__global__ void __launch_bounds__(GJ_THREADS) k_gj_step(double *a, int n, int k, double *col, int *flag,
                                                        unsigned *arrived) {
    const int m = 2 * n;
    const int j = k + blockIdx.x * GJ_TC + (threadIdx.x % GJ_TC);
    const int i0 = blockIdx.y * GJ_TR + threadIdx.x / GJ_TC;
    if (j < m) {
        const double akj = __ldcg(&a[(long long)k * m + j]);
#pragma unroll
        for (int r = 0; r < GJ_RPT; ++r) {
            const int i = i0 + r * (GJ_THREADS / GJ_TC);
            if (i < n && i != k) {
                double *e = &a[(long long)i * m + j];
                *e = fma(-__ldcg(&col[i]), akj, __ldcg(e));
            }
        }
    }
    if (k + 1 >= n) return;
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(arrived, 1u) == gridDim.x * gridDim.y - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    gj_pivot(a, n, k + 1, col, flag);
    if (threadIdx.x == 0) *arrived = 0u;
}

size_t gauss_jordan_doubles(int n) { return (size_t)n * 2 * n + n + 1; }

void launch_gauss_jordan(double *aug, int n, int *flag, cudaStream_t s) {
    double *col = aug + (size_t)n * 2 * n;
    unsigned *arrived = reinterpret_cast<unsigned *>(col + n);
    cudaMemsetAsync(arrived, 0, sizeof(unsigned), s);
    k_gj_first<<<1, GJ_THREADS, 0, s>>>(aug, n, col, flag);
    const unsigned gy = (unsigned)((n + GJ_TR - 1) / GJ_TR);
    for (int k = 0; k < n; k++) {
        const unsigned gx = (unsigned)((2 * n - k + GJ_TC - 1) / GJ_TC);
        k_gj_step<<<dim3(gx, gy), GJ_THREADS, 0, s>>>(aug, n, k, col, flag, arrived);
    }
}

// one block per load case c: b (optionally minus its mean per component), x = K^-1 b;
// b: n doubles of shared memory
__device__ __forceinline__ void coarse_apply_block(const Planes &C, const double *__restrict__ aug, int n, int project,
                                                   const float *__restrict__ f, float *u, int c, double *b) {
    __shared__ double mean[3];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const long long lex = i / 3;
        const int comp = i % 3;
        const int x = (int)(lex % C.n[0]), y = (int)((lex / C.n[0]) % C.n[1]), z = (int)(lex / ((long long)C.n[0] * C.n[1]));
        b[i] = f[fidx(3 * c + comp, vidx(C, x, y, z))];
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0;
        if (project)
            for (int i = threadIdx.x; i < n; i += 3) s += b[i];
        mean[threadIdx.x] = s / (double)(n / 3);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) b[i] -= mean[i % 3];
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double *row = aug + (long long)i * 2 * n + n;
        double s = 0;
        for (int j = 0; j < n; j++) s = fma(row[j], b[j], s);
        const long long lex = i / 3;
        const int comp = i % 3;
        const int x = (int)(lex % C.n[0]), y = (int)((lex / C.n[0]) % C.n[1]), z = (int)(lex / ((long long)C.n[0] * C.n[1]));
        u[fidx(3 * c + comp, vidx(C, x, y, z))] = (float)s;
    }
}

__global__ void __launch_bounds__(256) k_coarse_apply(Planes C, const double *__restrict__ aug, int n, int project,
                                                      const float *__restrict__ f, float *u) {
    extern __shared__ double b[];
    coarse_apply_block(C, aug, n, project, f, u, blockIdx.x, b);
}

void launch_coarse_apply(const Level &C, const double *aug, int project, cudaStream_t s) {
    const int n = (int)(3 * C.P.nv);
    k_coarse_apply<<<NCASE, 256, (size_t)n * sizeof(double), s>>>(C.P, aug, n, project, C.f, C.u);
}

// lockstep batches: the coarsest solves of several designs in one launch, six
// CTAs (one per load case) per design, each the CTA of the design's own launch
struct CoarsestEnt {
    Planes C;
    const double *aug;
    const float *f;
    float *u;
    int n, design;
};
struct CoarsestBatchTab {
    int n;
    CoarsestEnt e[BATCH_MAX];
};

__global__ void __launch_bounds__(256) k_coarse_apply_batch(const CoarsestBatchTab *__restrict__ t,
                                                            const int *__restrict__ active, int project) {
    extern __shared__ double b[];
    __shared__ __align__(16) unsigned buf[sizeof(CoarsestEnt) / 4];
    const int i = blockIdx.x / NCASE, c = blockIdx.x % NCASE;
    if (!__ldg(&active[t->e[i].design])) return;
    const CoarsestEnt &e = stage_args(t->e[i], buf);
    coarse_apply_block(e.C, e.aug, e.n, project, e.f, e.u, c, b);
}

int coarsest_batch_create(const Level *const *lv, const double *const *aug, const int *design, int n, BatchTab *out) {
    if (n < 1 || n > BATCH_MAX) return -1;
    CoarsestBatchTab *t = new CoarsestBatchTab();
    t->n = n;
    int nmax = 0;
    for (int i = 0; i < n; i++) {
        CoarsestEnt &e = t->e[i];
        e.C = lv[i]->P;
        e.aug = aug[i];
        e.f = lv[i]->f;
        e.u = lv[i]->u;
        e.n = (int)(3 * lv[i]->P.nv);
        e.design = design[i];
        nmax = e.n > nmax ? e.n : nmax;
    }
    void *d = nullptr;
    int rc = cudaMalloc(&d, sizeof(CoarsestBatchTab)) == cudaSuccess ? 0 : -2;
    if (rc == 0 && cudaMemcpy(d, t, sizeof(CoarsestBatchTab), cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
    if (rc == 0 && nmax * sizeof(double) + sizeof(CoarsestEnt) > 48 * 1024 &&
        cudaFuncSetAttribute(k_coarse_apply_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(nmax * sizeof(double))) != cudaSuccess)
        rc = -2;
    if (rc == 0) {
        out->dev = d;
        out->n = n;
        out->grid[0] = (unsigned)(n * NCASE);
        out->smem = (size_t)nmax * sizeof(double);
    } else if (d) {
        cudaFree(d);
    }
    delete t;
    return rc;
}

void launch_coarse_apply_batch(const BatchTab &t, const int *active, int project, cudaStream_t s) {
    k_coarse_apply_batch<<<t.grid[0], 256, t.smem, s>>>(static_cast<const CoarsestBatchTab *>(t.dev), active,
                                                         project);
}

}  // namespace h3d
