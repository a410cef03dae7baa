// k_fine_tc.cu -- level-0 residual r = f - K(rho) u element by element on the
// 5th-generation tensor cores (tcgen05, TF32 operands, FP32 accumulation in TMEM).
//
// Reference behaviour restated (homo3d grid.cu): update_residual_otf_kernel_1
// (grid.cu:1277-1461): r = f - K(rho) u with K(rho) = sum_e (1e-9 + rho_e) Ke over
// the eight elements of each vertex, u at the pinned origin counted as zero and
// r = 0 there.
//
// B200 design.  The contraction is the element product Ke U_e (24 x 24 times the
// element's 24 displacements, per load case), a GEMM with Ke as the shared operand:
//   rows    : 128 elements of a tile (one TMEM lane each),
//   K       : the element's 24 DOFs (three K = 8 steps of kind::tf32),
//   N       : the 24 output DOFs, 24 TMEM columns per tile.
// Precision.  U enters as differences from the element's node 0 (Ke annihilates
// rigid translations, so Ke U = Ke (U - u_0)), each split into a TF32 hi part and
// the FP32 remainder, Ke likewise, and the product is hi*Khi + lo*Khi + hi*Klo with
// FP32 accumulation: about 21 significant bits, near the FP32 operator's accuracy.
// One TF32 part alone keeps 11 bits, whose error floor (measured against an FP64
// emulation: 1.7e-3 of ||f|| at 64^3 on converged solutions, growing about like
// N^0.85) is above the 1e-3 drop a refinement step waits for at 256^3.
// Owned bricks.  A CTA owns a brick of 8 x 8 x 8 vertices and runs the (8+1)^3
// elements that touch it; the elements on a brick's faces are run by both bricks
// (729 elements for 512 vertices), their inputs staged once per brick and case.
// Every mbarrier wait is bounded: on timeout the kernel sets *flag, skips the rest
// of its work and still frees its TMEM.
#include <stdint.h>

#include "h3d_internal.cuh"

namespace h3d {

namespace {

constexpr int RT_M = 128;                       // elements per tile = TMEM lanes
constexpr int RT_T = 256;                       // threads: two per element row (halves of its DOFs)
constexpr int RT_B = 8;                         // owned vertices per brick edge
constexpr int RT_OWN = RT_B * RT_B * RT_B;      // owned vertices per brick
constexpr int RT_EL = (RT_B + 1) * (RT_B + 1) * (RT_B + 1);  // elements touching a brick
constexpr int RT_TILES = (RT_EL + RT_M - 1) / RT_M;          // 6
constexpr int RT_K = 24;                        // element DOFs
constexpr int RT_N = 24;                        // output DOFs
constexpr int RT_PART = RT_M * RT_K * 4;        // one TF32 operand tile: 12 KB
constexpr int RT_BPART = RT_N * RT_K * 4;       // Ke hi or lo: 2.25 KB
constexpr int RT_STAGE = (RT_B + 2) * (RT_B + 2) * (RT_B + 2);  // staged vertices of a brick
constexpr int RT_TMEM_COLS = 256;               // RT_TILES x 24 accumulator columns, rounded up
constexpr int RT_SMEM_USED = 2 * RT_PART + 2 * RT_BPART + 3 * RT_STAGE * 4 + RT_EL * RT_N * 4 + RT_EL * 4 + 64;
constexpr int RT_SMEM_REQUEST = RT_SMEM_USED + 128;  // + alignment slack
constexpr long long RT_WAIT_LIMIT = 1ll << 24;
constexpr int RT_MINB = 2;                      // CTAs per SM
static_assert(RT_TILES * RT_N <= RT_TMEM_COLS, "accumulators of a brick exceed the TMEM allocation");

// byte offset of (row, k) in a K-major, non-swizzled TF32 operand tile of K = 24:
// 8-row x 16-byte core matrices, K-chunks of 4 floats 128 B apart (leading
// offset), row groups 768 B apart (stride offset)
__host__ __device__ constexpr uint32_t rt_off(int row, int k) {
    return (uint32_t)((row >> 3) * 768 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ uint32_t rt_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t rt_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(768 >> 4) << 32) |
           ((uint64_t)1 << 46);
}

// instruction descriptor of kind::tf32: D FP32, A and B TF32 (format 2), both
// K-major, N = 24 (N >> 3 in bits 17-22), M = 128 (M >> 4 in bits 24-28)
constexpr uint32_t RT_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(RT_N >> 3) << 17) |
                              ((uint32_t)(RT_M >> 4) << 24);

__device__ __forceinline__ void rt_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(RT_IDESC), "r"(accumulate));
}

__device__ __forceinline__ void rt_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(rt_smem(bar))
                 : "memory");
}

__device__ __forceinline__ bool rt_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t a = rt_smem(bar);
    for (long long it = 0; it < RT_WAIT_LIMIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 12 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void rt_ld12(uint32_t taddr, float v[12]) {
    uint32_t r[12];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11])
                 : "r"(taddr + 8));
#pragma unroll
    for (int q = 0; q < 12; ++q) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

struct TcResArgs {
    const float *__restrict__ rho;
    const float *__restrict__ u;
    const float *__restrict__ f;
    float *r;
    Planes P;
    int nb[3];       // bricks per axis
    long long nbrick;
};

}  // namespace

// One CTA of 256 threads per brick at a time: threads t and t + 128 serve element
// row t % 128 of a tile, each with half of its 24 DOFs (corners 0-3 or 4-7) when
// gathering and half of its 24 outputs when reading TMEM.  Per load case (a pass):
//   1. stage the brick's vertices and one-vertex halo, the case's three planes;
//   2. per tile of 128 elements, the differences from corner 0 as TF32 hi + lo
//      parts into the A operand, and nine MMAs (three K steps of 8, each
//      hi*Khi + lo*Khi + hi*Klo) into the tile's 24 TMEM columns; the gather of the
//      next tile runs while the MMAs of this one do;
//   3. the weighted outputs (1e-9 + rho_e) KU_e of every element to shared memory;
//   4. per owned vertex, the sum of its eight element contributions in corner
//      order 0..7 (the same order every run), r = f - sum, and the weighted norm.
__global__ void __launch_bounds__(RT_T, RT_MINB) k_fine_residual_tc(TcResArgs a, const __grid_constant__ KeMat ke,
                                                                     double *partial, int *flag) {
    extern __shared__ __align__(128) unsigned char rt_smem_raw[];
    unsigned char *base = rt_smem_raw + ((128 - (rt_smem(rt_smem_raw) & 127)) & 127);
    unsigned char *Ahi = base, *Alo = base + RT_PART;
    unsigned char *Bhi = base + 2 * RT_PART, *Blo = Bhi + RT_BPART;
    float *stage = reinterpret_cast<float *>(Blo + RT_BPART);     // [3][(B+2)^3] the case's vertex values
    float *eo = stage + 3 * RT_STAGE;                               // [element][24] weighted outputs
    float *rhos = eo + RT_EL * RT_N;                                // [element] 1e-9 + rho
    uint64_t *bar = reinterpret_cast<uint64_t *>(rhos + RT_EL + ((RT_EL & 1) ? 1 : 0));
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int row = tid & (RT_M - 1), half = tid >> 7;   // element row, DOF half

    // Ke split into TF32 hi + lo as the B operand: B[n][k] = Ke[n][k]
    for (int q = tid; q < RT_N * RT_K; q += RT_T) {
        const int nn = q / RT_K, k = q % RT_K;
        const float v = ke.k[nn * 24 + k], h = tf32_hi(v);
        *reinterpret_cast<float *>(Bhi + rt_off(nn, k)) = h;
        *reinterpret_cast<float *>(Blo + rt_off(nn, k)) = v - h;
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(rt_smem(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(rt_smem(tslot)),
                     "r"(RT_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;
    // warps w and w + 4 read the same 32 lanes (rows), different column halves
    const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(12 * half);
    const uint32_t sAhi = rt_smem(Ahi), sAlo = rt_smem(Alo), sBhi = rt_smem(Bhi), sBlo = rt_smem(Blo);
    const int *n = a.P.n;

    double nrm[NCASE];
#pragma unroll
    for (int c = 0; c < NCASE; ++c) nrm[c] = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (long long brick = blockIdx.x; brick < a.nbrick && ok; brick += gridDim.x) {
        const int bxi = (int)(brick % a.nb[0]);
        const long long bt = brick / a.nb[0];
        const int byi = (int)(bt % a.nb[1]), bzi = (int)(bt / a.nb[1]);
        const int x0 = bxi * RT_B, y0 = byi * RT_B, z0 = bzi * RT_B;
        const int ox = min(RT_B, n[0] - x0), oy = min(RT_B, n[1] - y0), oz = min(RT_B, n[2] - z0);
        const int ex_n = ox + 1, ey_n = oy + 1;                  // elements per axis
        const int sx = ox + 2, sy = oy + 2;                      // staged vertices per axis
        const int nel = ex_n * ey_n * (oz + 1), nst = sx * sy * (oz + 2);
        const int ntile = (nel + RT_M - 1) / RT_M;
        for (int e = tid; e < nel; e += RT_T) {
            const int lx = e % ex_n, tt = e / ex_n, ly = tt % ey_n, lz = tt / ey_n;
            const int ex = wrap(x0 - 1 + lx, n[0]), ey = wrap(y0 - 1 + ly, n[1]), ez = wrap(z0 - 1 + lz, n[2]);
            rhos[e] = RHO_PENAL_MIN + __ldg(&a.rho[ex + (long long)n[0] * (ey + (long long)n[1] * ez)]);
        }
#pragma unroll 1
        for (int cs = 0; cs < NCASE && ok; ++cs) {
            // 1. the case's planes of the brick and its halo (the pinned origin as 0)
            for (int lv = tid; lv < nst; lv += RT_T) {
                const int lx = lv % sx, tt = lv / sx, ly = tt % sy, lz = tt / sy;
                const int x = wrap(x0 - 1 + lx, n[0]), y = wrap(y0 - 1 + ly, n[1]), z = wrap(z0 - 1 + lz, n[2]);
                const float *up = a.u + fidx(3 * cs, vidx(a.P, x, y, z));
                const bool origin = (x | y | z) == 0;
#pragma unroll
                for (int m = 0; m < 3; ++m) stage[m * RT_STAGE + lv] = origin ? 0.f : __ldg(up + m * FVB);
            }
            __syncthreads();
            // 2. tiles: gather (differences from corner 0, TF32 hi + lo) and MMAs
            for (int t = 0; t < ntile; ++t) {
                const int e = t * RT_M + row;
                const bool valid = e < nel;
                int s0 = 0;
                if (valid) {
                    const int lx = e % ex_n, tt = e / ex_n, ly = tt % ey_n, lz = tt / ey_n;
                    s0 = lx + sx * (ly + sy * lz);
                }
                float U[12];  // corners 4 half .. 4 half + 3, components 0..2
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    const float *sq = stage + m * RT_STAGE + s0;
                    const float u0 = sq[0];
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        const int c = 4 * half + cc;
                        U[3 * cc + m] = valid ? sq[(c & 1) + sx * (((c >> 1) & 1) + sy * (c >> 2))] - u0 : 0.f;
                    }
                }
                if (t > 0) {  // the MMAs of the previous tile have read A
                    const bool done = rt_wait(bar, phase);
                    if (__syncthreads_or(!done)) {
                        ok = false;
                        if (tid == 0) atomicExch(flag, 1);
                        break;
                    }
                    phase ^= 1u;
                }
#pragma unroll
                for (int k4 = 0; k4 < 3; ++k4) {
                    float4 h, l;
                    h.x = tf32_hi(U[4 * k4]);     l.x = U[4 * k4] - h.x;
                    h.y = tf32_hi(U[4 * k4 + 1]); l.y = U[4 * k4 + 1] - h.y;
                    h.z = tf32_hi(U[4 * k4 + 2]); l.z = U[4 * k4 + 2] - h.z;
                    h.w = tf32_hi(U[4 * k4 + 3]); l.w = U[4 * k4 + 3] - h.w;
                    *reinterpret_cast<float4 *>(Ahi + rt_off(row, 12 * half + 4 * k4)) = h;
                    *reinterpret_cast<float4 *>(Alo + rt_off(row, 12 * half + 4 * k4)) = l;
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncthreads();
                if (tid == 0) {
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t d = tmem + (uint32_t)(RT_N * t);
#pragma unroll
                    for (int st = 0; st < RT_K / 8; ++st) {
                        const uint32_t ko = (uint32_t)(st * 256);  // two 16-byte K-chunks per K step of 8
                        rt_mma(d, rt_desc(sAhi + ko), rt_desc(sBhi + ko), st > 0 ? 1u : 0u);
                        rt_mma(d, rt_desc(sAlo + ko), rt_desc(sBhi + ko), 1u);
                        rt_mma(d, rt_desc(sAhi + ko), rt_desc(sBlo + ko), 1u);
                    }
                    rt_commit(bar);
                }
            }
            if (!ok) break;
            {
                const bool done = rt_wait(bar, phase);
                if (__syncthreads_or(!done)) {
                    ok = false;
                    if (tid == 0) atomicExch(flag, 1);
                    break;
                }
                phase ^= 1u;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // 3. weighted outputs of every element to shared memory
            for (int t = 0; t < ntile; ++t) {
                float v[12];
                rt_ld12(lane_addr + (uint32_t)(RT_N * t), v);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                const int e = t * RT_M + row;
                if (e < nel) {
                    const float w = rhos[e];
                    float4 *dst = reinterpret_cast<float4 *>(eo + e * RT_N + 12 * half);
                    dst[0] = make_float4(v[0] * w, v[1] * w, v[2] * w, v[3] * w);
                    dst[1] = make_float4(v[4] * w, v[5] * w, v[6] * w, v[7] * w);
                    dst[2] = make_float4(v[8] * w, v[9] * w, v[10] * w, v[11] * w);
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            // 4. per owned vertex: the eight element contributions in corner order
            for (int ov = tid; ov < RT_OWN; ov += RT_T) {
                const int vx = ov % RT_B, vy = (ov / RT_B) % RT_B, vz = ov / (RT_B * RT_B);
                if (vx >= ox || vy >= oy || vz >= oz) continue;
                float sum[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    // the element with this vertex as corner c: element-local (v + 1 - bits of c)
                    const int e = (vx + 1 - (c & 1)) + ex_n * ((vy + 1 - ((c >> 1) & 1)) + ey_n * (vz + 1 - (c >> 2)));
                    const float *src = eo + e * RT_N + 3 * c;
                    sum[0] += src[0];
                    sum[1] += src[1];
                    sum[2] += src[2];
                }
                const int x = x0 + vx, y = y0 + vy, z = z0 + vz;
                const long long o = fidx(3 * cs, vidx(a.P, x, y, z));
                const bool origin = (x | y | z) == 0;
                const double mult = (double)(axis_mult(x, n[0]) * axis_mult(y, n[1]) * axis_mult(z, n[2]));
                double s2 = 0;
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    const float rv = origin ? 0.f : __ldg(a.f + o + m * FVB) - sum[m];
                    a.r[o + m * FVB] = rv;
                    s2 += (double)rv * rv;
                }
#pragma unroll
                for (int c = 0; c < NCASE; ++c)
                    if (c == cs) nrm[c] += mult * s2;
            }
            __syncthreads();  // stage, outputs and TMEM are reused by the next case
        }
    }
    if (partial) block_reduce<NCASE>(nrm, partial, blockIdx.x);
    // a wait that ran out leaves its MMAs in flight: let them finish (bounded) before
    // the TMEM they write is freed
    if (!ok) (void)rt_wait(bar, phase);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(RT_TMEM_COLS)
                     : "memory");
}

static_assert(RT_SMEM_REQUEST * RT_MINB <= 227 * 1024, "shared memory of RT_MINB CTAs exceeds an SM");
static_assert(RT_TMEM_COLS * RT_MINB <= 512, "TMEM columns of RT_MINB CTAs exceed an SM");

int fine_residual_tc_blocks(const Planes &P, int num_sms) {
    long long nb = 1;
    for (int d = 0; d < 3; ++d) nb *= (P.n[d] + RT_B - 1) / RT_B;
    const long long g = (long long)RT_MINB * num_sms;
    return (int)(nb < g ? nb : g);
}

int configure_fine_residual_tc() {
    return cudaFuncSetAttribute((const void *)k_fine_residual_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                RT_SMEM_REQUEST) == cudaSuccess
               ? 0
               : -1;
}

int launch_fine_residual_tc(const Level &L, const float *rho, const KeMat &ke, double *partial, int nblk,
                            int *flag, cudaStream_t s) {
    TcResArgs a;
    a.rho = rho;
    a.u = L.u;
    a.f = L.f;
    a.r = L.r;
    a.P = L.P;
    a.nbrick = 1;
    for (int d = 0; d < 3; ++d) {
        a.nb[d] = (L.P.n[d] + RT_B - 1) / RT_B;
        a.nbrick *= a.nb[d];
    }
    k_fine_residual_tc<<<nblk, RT_T, RT_SMEM_REQUEST, s>>>(a, ke, partial, flag);
    return 0;
}

}  // namespace h3d
