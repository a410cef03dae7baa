// k_static_norm.cu -- the padded-storage weighted norms of a level-0 vertex field
// with the reduction scratch in a fixed file-scope device array instead of memory
// the library allocates (the kernels behind h3d_field_norms_static).
//
// Who needs this: code that calls the solver from a context where it must not
// allocate device memory at call time -- for instance a caller whose device
// memory is fully owned by another allocator, or one that cannot accept the
// device-wide synchronisation a cudaMalloc / cudaFree can cause in the middle of
// its work.  The array is a fixed 2048 x 6 + 6 doubles (about 96 KB) that every
// GPU loading the library keeps until the process exits.
//
// Same arithmetic and the same fixed reduction order as k_weighted_norm +
// k_finish<6> in k_coarse.cu (v3_norm, grid.cu:1954-1966: per-case sums of
// squares with the multiplicities of positions 0, 1 and n-1 per axis), so the
// results are bit-identical to h3d_field_norms.
//
// The array is shared by every call on a device and keeps the last call's
// contents: each call overwrites every partial it later reads, so nothing needs
// clearing, but two calls that overlap in time on one GPU (different host
// threads, or streams without ordering between them) race on it.  Host code gets
// the array's device address from cudaGetSymbolAddress once per device, on that
// device's first call; that first call may load the module and should come
// before any stream capture.
#include <mutex>

#include "h3d_internal.cuh"

namespace h3d {

constexpr int STATIC_NORM_BS = 256;

// per-block partials (STATIC_NORM_MAX_BLOCKS x 6) followed by the 6 totals
static __device__ __align__(256) double g_static_norm_scratch[STATIC_NORM_MAX_BLOCKS * NCASE + NCASE];

__global__ void __launch_bounds__(STATIC_NORM_BS) k_weighted_norm_static(Planes P, const float *__restrict__ v,
                                                                        double *scratch) {
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
                const double t = v[fidx(3 * c + q, i)];
                a += t * t;
            }
            s[c] += m * a;
        }
    }
    block_reduce<NCASE>(s, scratch, blockIdx.x);
}

__global__ void __launch_bounds__(256) k_finish_static(int nblk, double *scratch) {
    double s[NCASE] = {0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
        for (int c = 0; c < NCASE; ++c) s[c] += scratch[(long long)b * NCASE + c];
    block_reduce<NCASE>(s, scratch + STATIC_NORM_MAX_BLOCKS * NCASE, 0);
}

// device address of the array on the current device (looked up once per device)
static double *static_norm_scratch(int device) {
    static std::mutex mu;
    static double *addr[64] = {};
    if (device < 0 || device >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        double *p = nullptr;
        if (cudaGetSymbolAddress((void **)&p, g_static_norm_scratch) != cudaSuccess) return nullptr;
        addr[device] = p;
    }
    return addr[device];
}

const double *static_norm_totals(int device) {
    double *p = static_norm_scratch(device);
    return p ? p + STATIC_NORM_MAX_BLOCKS * NCASE : nullptr;
}

int launch_weighted_norm_static(int device, const Planes &P, const float *v, int nblk, cudaStream_t s) {
    if (nblk < 1 || nblk > STATIC_NORM_MAX_BLOCKS) return -1;
    double *scratch = static_norm_scratch(device);
    if (!scratch) return -2;
    k_weighted_norm_static<<<nblk, STATIC_NORM_BS, 0, s>>>(P, v, scratch);
    k_finish_static<<<1, 256, 0, s>>>(nblk, scratch);
    return 0;
}

}  // namespace h3d
