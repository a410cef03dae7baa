// k_homog_tc.cu -- homogenized elastic tensor and sensitivities, with the element
// contraction Ke x U on the 5th-generation tensor cores (tcgen05, TF32 inputs,
// FP32 accumulation in tensor memory).
//
// Reference behaviour restated (homo3d homogenization.cu):
//   elasticMatrix_kernel_opt (homogenization.cu:208-346), elasticMatrix
//   (:464-575): C_ij = (1/|Y|) sum_e (1e-9 + rho_e) (chi0_i - chi_i)^T Ke
//   (chi0_j - chi_j); Sensitivity_kernel_opt_2 (:697-858): per element
//   sum_{i<=j} (dC_ij + [i!=j] dC_ji) (chi0_i - chi_i)^T Ke (chi0_j - chi_j) / |Y|.
//
// B200 design.  A CTA owns a tile of 128 elements (one per thread and one per
// TMEM lane) and walks the six load cases j:
//   1. every thread gathers its element's 24 displacements U_j = chi0_j - chi_j
//      (FP64 chi taken relative to the element's node 0), splits each value into
//      TF32 hi + lo parts and stores both as the A operand (128 x 24, K-major,
//      no swizzle) in shared memory;
//   2. one thread issues nine tcgen05.mma kind::tf32 (three K-steps of 8, each
//      as hi*Khi + lo*Khi + hi*Klo: FP32-level accuracy from TF32 inputs) that
//      write KU_j = Ke U_j (128 x 24, FP32) into TMEM columns 24j..24j+23, and
//      commits them to an mbarrier;
//   3. after the mbarrier, each thread reads KU_i (i <= j) of its own lane and
//      forms E_ij = U_j . KU_i in FP32 (Ke is symmetric, so E_ij = E_ji).
// The 21 energies are weighted by (1e-9 + rho_e) and summed in FP64 (C), or
// contracted with dC (sensitivities).  TMEM: 256 columns per CTA, at most two
// CTAs per SM (the dynamic shared-memory request keeps a third off the SM).
// Every mbarrier wait is bounded; on timeout the kernel raises a flag, skips the
// rest of its work, and still frees its TMEM.
#include <stdint.h>

#include "h3d_internal.cuh"

namespace h3d {

constexpr int TC_M = 128;             // elements per tile (= threads per CTA = TMEM lanes)
constexpr int TC_K = 24;              // element DOFs
constexpr int TC_TILE_BYTES = TC_M * TC_K * 4;       // one 128 x 24 TF32 operand tile
constexpr int TC_B_BYTES = TC_K * TC_K * 4;          // Ke as a 24 x 24 TF32 tile
constexpr int TC_SMEM_USED = 4 * TC_TILE_BYTES + 2 * TC_B_BYTES + 64;  // A hi/lo double-buffered, B hi/lo
constexpr int TC_SMEM_REQUEST = 100 * 1024;          // > 227 KB / 3: at most two CTAs per SM
constexpr int TC_TMEM_COLS = 256;                    // 6 x 24 FP32 accumulator columns, rounded up
constexpr long long TC_WAIT_LIMIT = 1ll << 24;       // mbarrier polls before giving up

// byte offset of element (row, k) in a K-major, non-swizzled UMMA operand tile:
// 8-row x 16-byte core matrices, the six 16-byte K-chunks of a row group 128 B
// apart (leading offset), row groups 768 B apart (stride offset)
__host__ __device__ constexpr uint32_t tc_off(int row, int k) {
    return (uint32_t)((row >> 3) * 768 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

// shared-memory matrix descriptor (sm100 layout): start address >> 4 in bits
// [0,14), leading byte offset >> 4 in [16,30), stride byte offset >> 4 in
// [32,46), descriptor version 1 in [46,48), base offset 0, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(768 >> 4) << 32) |
           ((uint64_t)1 << 46);
}

// instruction descriptor of kind::tf32: D FP32, A and B TF32, both K-major,
// N = 24 (N >> 3 in bits [17,23)), M = 128 (M >> 4 in bits [24,29))
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_K >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// bounded wait for the mbarrier phase with the given parity; false on timeout
__device__ __forceinline__ bool tc_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (long long it = 0; it < TC_WAIT_LIMIT; ++it) {
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

// 8 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld8(uint32_t taddr, float v[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

// unit macro-strain displacement chi0 of local node a, case c, component m
// (homoCommon.cuh:455-519)
__host__ __device__ constexpr float tc_macro_disp(int a, int c, int m) {
    const int p0 = a & 1, p1 = (a >> 1) & 1, p2 = a >> 2;
    return c == 0 ? (m == 0 ? (float)p0 : 0.f)
         : c == 1 ? (m == 1 ? (float)p1 : 0.f)
         : c == 2 ? (m == 2 ? (float)p2 : 0.f)
         : c == 3 ? (m == 1 ? p2 * 0.5f : m == 2 ? p1 * 0.5f : 0.f)
         : c == 4 ? (m == 0 ? p2 * 0.5f : m == 2 ? p0 * 0.5f : 0.f)
                  : (m == 0 ? p1 * 0.5f : m == 1 ? p0 * 0.5f : 0.f);
}

struct TcDc { float w[21]; };  // (dC_ij + [i!=j] dC_ji) / |Y| for the 21 pairs

// SENS = false: per-block FP64 partial sums of (1e-9 + rho_e) E_ij (21 values);
// SENS = true: sens[x + (y + z*ny)*pitch] = sum_t dc_t E_t per element
// dcw (SENS only, may be null): the 21 weights read from device memory instead of dc
template <bool SENS>
__global__ void __launch_bounds__(TC_M) k_energy_tc(Planes P, const double *__restrict__ chi,
                                                    const float *__restrict__ rho, const __grid_constant__ KeMat ke,
                                                    double *partial, TcDc dc, const float *dcw, float *sens, int pitch,
                                                    int *flag) {
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    unsigned char *base = tc_smem + ((1024 - (smem_u32(tc_smem) & 1023)) & 1023);
    // A operand buffers b = 0, 1: hi at base + 2 b TILE, lo at base + (2 b + 1) TILE
    unsigned char *Bhi = base + 4 * TC_TILE_BYTES, *Blo = Bhi + TC_B_BYTES;
    uint64_t *bar = reinterpret_cast<uint64_t *>(Blo + TC_B_BYTES);  // one mbarrier per A buffer
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5;
    __shared__ float dcs[21];
    if (SENS && tid < 21) dcs[tid] = dcw ? dcw[tid] : dc.w[tid];

    // Ke split into TF32 hi + lo, as the 24 x 24 B operand (B[n][k] = Ke[n][k])
    for (int q = tid; q < TC_K * TC_K; q += TC_M) {
        const int n = q / TC_K, k = q % TC_K;
        const float v = ke.k[q], h = tf32_hi(v);
        *reinterpret_cast<float *>(Bhi + tc_off(n, k)) = h;
        *reinterpret_cast<float *>(Blo + tc_off(n, k)) = v - h;
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar + 1)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t sA = smem_u32(base), sBhi = smem_u32(Bhi), sBlo = smem_u32(Blo);

    double acc[21];
#pragma unroll
    for (int t = 0; t < 21; ++t) acc[t] = 0;
    uint32_t phase[2] = {0, 0};
    bool ok = true;
    const long long ntile = (P.nv + TC_M - 1) / TC_M;
    for (long long tile = blockIdx.x; tile < ntile && ok; tile += gridDim.x) {
        const long long e = tile * TC_M + tid;
        const bool valid = e < P.nv;
        int x = 0, y = 0, z = 0;
        if (valid) {
            x = (int)(e % P.n[0]);
            const long long tt = e / P.n[0];
            y = (int)(tt % P.n[1]);
            z = (int)(tt / P.n[1]);
        }
        long long vtx[8];
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int vx = (a & 1) ? (x + 1 == P.n[0] ? 0 : x + 1) : x;
            const int vy = ((a >> 1) & 1) ? (y + 1 == P.n[1] ? 0 : y + 1) : y;
            const int vz = (a >> 2) ? (z + 1 == P.n[2] ? 0 : z + 1) : z;
            vtx[a] = vidx(P, vx, vy, vz);
        }
        // case j: U_j = chi0_j - chi_j over the element's 24 DOFs (FP64 chi relative
        // to node 0), stored as TF32 hi / lo rows of A buffer j & 1
        auto gather = [&](int j, float U[TC_K]) {
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                const double c0 = valid ? __ldg(chi + fidx(3 * j + m, vtx[0])) : 0.0;
#pragma unroll
                for (int a = 0; a < 8; ++a)
                    U[3 * a + m] = valid ? tc_macro_disp(a, j, m) - (float)(__ldg(chi + fidx(3 * j + m, vtx[a])) - c0)
                                         : 0.f;
            }
            unsigned char *Ah = base + 2 * (j & 1) * TC_TILE_BYTES, *Al = Ah + TC_TILE_BYTES;
#pragma unroll
            for (int k4 = 0; k4 < TC_K / 4; ++k4) {
                float4 h, l;
                h.x = tf32_hi(U[4 * k4]);     l.x = U[4 * k4] - h.x;
                h.y = tf32_hi(U[4 * k4 + 1]); l.y = U[4 * k4 + 1] - h.y;
                h.z = tf32_hi(U[4 * k4 + 2]); l.z = U[4 * k4 + 2] - h.z;
                h.w = tf32_hi(U[4 * k4 + 3]); l.w = U[4 * k4 + 3] - h.w;
                *reinterpret_cast<float4 *>(Ah + tc_off(tid, 4 * k4)) = h;
                *reinterpret_cast<float4 *>(Al + tc_off(tid, 4 * k4)) = l;
            }
        };
        // KU_j = Ke U_j into TMEM columns 24j.. (lanes 0..127), committed to bar[j & 1]
        auto issue = [&](int j) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t d = tmem + (uint32_t)(TC_K * j);
            const uint32_t ahi = sA + (uint32_t)(2 * (j & 1) * TC_TILE_BYTES), alo = ahi + TC_TILE_BYTES;
#pragma unroll
            for (int st = 0; st < TC_K / 8; ++st) {
                const uint32_t ko = (uint32_t)(st * 256);  // two 16-byte K-chunks per K-step of 8
                tc_mma(d, tc_desc(ahi + ko), tc_desc(sBhi + ko), st > 0 ? 1u : 0u);
                tc_mma(d, tc_desc(alo + ko), tc_desc(sBhi + ko), 1u);
                tc_mma(d, tc_desc(ahi + ko), tc_desc(sBlo + ko), 1u);
            }
            tc_commit(bar + (j & 1));
        };
        // Pipeline (PIPE): the gather of case j + 1 and its MMAs run while the MMAs
        // of case j complete and case j's energies are read out of TMEM.  A buffer
        // (j+1) & 1 was last read by the MMAs of case j - 1, already waited for.
        // Without PIPE, case j is gathered, multiplied and read out before case
        // j + 1 starts.  Measured at 256^3: the pipeline makes the sensitivity form
        // faster (6.9 against 7.7 ms per call) and the C form, which keeps 21 FP64
        // sums per thread besides, 1.5 ms slower, so only the former uses it.
        constexpr bool PIPE = SENS;
        float E[21], Uc[TC_K], Un[TC_K];
        int waited = 0, issued = 0;
        if (PIPE) {
            gather(0, Uc);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) issue(0);
            issued = 1;
        }
#pragma unroll
        for (int j = 0; j < NCASE; ++j) {
            if (!ok) continue;
            if (PIPE && j + 1 < NCASE) gather(j + 1, Un);
            if (!PIPE) gather(j, Uc);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();  // the A buffer written; every thread past the previous case's TMEM reads
            if (PIPE ? j + 1 < NCASE : true) {
                if (tid == 0) issue(PIPE ? j + 1 : j);
                ++issued;
            }
            const bool done = tc_wait(bar + (j & 1), phase[j & 1]);
            phase[j & 1] ^= 1u;
            ++waited;
            if (__syncthreads_or(!done)) {  // uniform: every thread stops together
                ok = false;
                if (tid == 0) atomicExch(flag, 1);
                continue;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // E_ij = U_j . KU_i for i <= j (three 8-column loads, one wait)
#pragma unroll
            for (int i = 0; i <= j; ++i) {
                float ku[TC_K];
                tc_ld8(lane_addr + (uint32_t)(TC_K * i), ku);
                tc_ld8(lane_addr + (uint32_t)(TC_K * i + 8), ku + 8);
                tc_ld8(lane_addr + (uint32_t)(TC_K * i + 16), ku + 16);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                float sum = 0.f;
#pragma unroll
                for (int q = 0; q < TC_K; ++q) sum = fmaf(Uc[q], ku[q], sum);
                E[i * 6 - i * (i - 1) / 2 + (j - i)] = sum;
            }
            if (PIPE)
#pragma unroll
                for (int q = 0; q < TC_K; ++q) Uc[q] = Un[q];
        }
        // the next tile overwrites A and TMEM only after every thread is past its reads
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (!ok) {  // a wait ran out: let the MMAs still in flight finish (bounded) before TMEM is freed
            for (int k = waited; k < issued; ++k) {
                (void)tc_wait(bar + (k & 1), phase[k & 1]);
                phase[k & 1] ^= 1u;
            }
            break;
        }
        if (valid) {
            if (SENS) {
                float s = 0.f;
#pragma unroll
                for (int t = 0; t < 21; ++t) s = fmaf(E[t], dcs[t], s);
                sens[x + ((long long)y + (long long)z * P.n[1]) * pitch] = s;
            } else {
                const double rp = (double)(RHO_PENAL_MIN + rho[e]);
#pragma unroll
                for (int t = 0; t < 21; ++t) acc[t] += rp * (double)E[t];
            }
        }
    }
    if (!SENS) block_reduce<21>(acc, partial, blockIdx.x);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS)
                     : "memory");
}

static_assert(TC_SMEM_USED + 1024 <= TC_SMEM_REQUEST, "shared-memory layout exceeds the request");

// fixed-order sum of the per-block partials of C
template <int N>
__global__ void __launch_bounds__(256) k_finish_n(const double *__restrict__ partial, int nblk, double *out) {
    double s[N];
#pragma unroll
    for (int c = 0; c < N; ++c) s[c] = 0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
        for (int c = 0; c < N; ++c) s[c] += partial[(long long)b * N + c];
    block_reduce<N>(s, out, 0);
}

void launch_elastic_finish(const double *partial, int nblk, double *out21, cudaStream_t s) {
    k_finish_n<21><<<1, 256, 0, s>>>(partial, nblk, out21);
}

int energy_tc_blocks(const Planes &P, int num_sms) {
    const long long ntile = (P.nv + TC_M - 1) / TC_M;
    const long long nb = 2ll * num_sms;
    return (int)(ntile < nb ? ntile : nb);
}

static bool tc_configured(const void *fn) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM_REQUEST) == cudaSuccess;
}

int launch_elastic_tc(const Planes &P, const double *chi, const float *rho, const KeMat &ke, double *partial,
                      int nblk, int *flag, cudaStream_t s) {
    if (!tc_configured((const void *)k_energy_tc<false>)) return -1;
    TcDc dc{};
    k_energy_tc<false><<<nblk, TC_M, TC_SMEM_REQUEST, s>>>(P, chi, rho, ke, partial, dc, nullptr, nullptr, 0, flag);
    return 0;
}

int launch_sensitivity_tc(const Planes &P, const double *chi, const KeMat &ke, const float *dc36, float *sens,
                          int pitch, int nblk, int *flag, cudaStream_t s) {
    if (!tc_configured((const void *)k_energy_tc<true>)) return -1;
    TcDc dc{};
    const double vol = (double)P.nv;
    int t = 0;
    for (int i = 0; i < 6; i++)
        for (int j = i; j < 6; j++, t++) {
            const double w = dc36[i * 6 + j] + (i != j ? dc36[j * 6 + i] : 0.f);
            dc.w[t] = (float)(w / vol);
        }
    k_energy_tc<true><<<nblk, TC_M, TC_SMEM_REQUEST, s>>>(P, chi, nullptr, ke, nullptr, dc, nullptr, sens, pitch,
                                                           flag);
    return 0;
}

// the 21 weights (dC_ij + [i != j] dC_ji) / |Y| of the sensitivity for dC[36]
void sensitivity_weights(const Planes &P, const float *dc36, float w21[21]) {
    const double vol = (double)P.nv;
    int t = 0;
    for (int i = 0; i < 6; i++)
        for (int j = i; j < 6; j++, t++) {
            const double w = dc36[i * 6 + j] + (i != j ? dc36[j * 6 + i] : 0.f);
            w21[t] = (float)(w / vol);
        }
}

int configure_energy_tc() {
    return tc_configured((const void *)k_energy_tc<false>) && tc_configured((const void *)k_energy_tc<true>) ? 0 : -1;
}

void launch_sensitivity_tc_dev(const Planes &P, const double *chi, const KeMat &ke, const float *dcw, float *sens,
                               int pitch, int nblk, int *flag, cudaStream_t s) {
    TcDc dc{};
    k_energy_tc<true><<<nblk, TC_M, TC_SMEM_REQUEST, s>>>(P, chi, nullptr, ke, nullptr, dc, dcw, sens, pitch, flag);
}

}  // namespace h3d
