// k_static_norm.cu -- the padded-storage weighted norms of a level-0 vertex field
// with reduction scratch in a file-scope device array instead of the handle's
// scratch buffer (the kernels behind h3d_field_norms_static).
//
// Same arithmetic and the same fixed reduction order as k_weighted_norm +
// k_finish<6> in k_coarse.cu (v3_norm, grid.cu:1954-1966: per-case sums of
// squares with the multiplicities of positions 0, 1 and n-1 per axis).
//
// The scratch is one array per device, shared by every handle on that device:
// two calls that overlap in time (different host threads, or different streams
// without ordering between them) race on it.  Its address is looked up with
// cudaGetSymbolAddress once per device; that first lookup may load the module
// and must not happen while a stream is being captured.
#include <mutex>

#include "h3d_internal.cuh"

namespace h3d {

constexpr int STATIC_NORM_BS = 256;

// per-block partials (STATIC_NORM_MAX_BLOCKS x 6) followed by the 6 totals
__device__ __align__(256) double g_static_norm_scratch[STATIC_NORM_MAX_BLOCKS * NCASE + NCASE];

__global__ void __launch_bounds__(STATIC_NORM_BS) k_weighted_norm_static(Planes P, const float *__restrict__ v) {
    double s[NCASE] = {0, 0, 0, 0, 0, 0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P.nv;
         i += (long long)gridDim.x * blockDim.x) {
        const int k = color_of_index(P, i);
        int x, y, z;
        vpos(P, k, i - P.base[k], x, y, z);
        const double m = (double)(axis_mult(x, P.n[0]) * axis_mult(y, P.n[1]) * axis_mult(z, P.n[2]));
#pragma unroll
        for (int c = 0; c < NCASE; ++c) {
            double a = 0;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const double t = v[(3 * c + q) * P.nv + i];
                a += t * t;
            }
            s[c] += m * a;
        }
    }
    block_reduce<NCASE>(s, g_static_norm_scratch, blockIdx.x);
}

__global__ void __launch_bounds__(256) k_finish_static(int nblk) {
    double s[NCASE] = {0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
        for (int c = 0; c < NCASE; ++c) s[c] += g_static_norm_scratch[(long long)b * NCASE + c];
    block_reduce<NCASE>(s, g_static_norm_scratch + STATIC_NORM_MAX_BLOCKS * NCASE, 0);
}

const double *static_norm_totals(int device) {
    static std::mutex mu;
    static const double *addr[64] = {};
    if (device < 0 || device >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_static_norm_scratch) != cudaSuccess) return nullptr;
        addr[device] = static_cast<const double *>(p) + STATIC_NORM_MAX_BLOCKS * NCASE;
    }
    return addr[device];
}

int launch_weighted_norm_static(const Planes &P, const float *v, int nblk, cudaStream_t s) {
    if (nblk < 1 || nblk > STATIC_NORM_MAX_BLOCKS) return -1;
    k_weighted_norm_static<<<nblk, STATIC_NORM_BS, 0, s>>>(P, v);
    k_finish_static<<<1, 256, 0, s>>>(nblk);
    return 0;
}

}  // namespace h3d
