// k_homog.cu -- homogenized elastic tensor and its density sensitivities.
//
// Reference behaviour restated (homo3d homogenization.cu):
//   elasticMatrix_kernel_opt (homogenization.cu:208-346) and elasticMatrix
//     (:464-575): C_ij = (1/|Y|) sum_e (1e-9 + rho_e) (chi0_i - chi_i)^T Ke
//     (chi0_j - chi_j) over the 21 pairs i <= j, |Y| = number of cells.
//   Sensitivity_kernel_opt_2 (homogenization.cu:697-858): per element
//     sum_{i<=j} (dC_ij + [i!=j] dC_ji) (chi0_i - chi_i)^T Ke (chi0_j - chi_j)
//     * p rho^(p-1) / |Y| with p = 1, written at x + (y + z*ny)*pitchT.
//   The reference rounds chi to FP16 before both reductions
//   (homogenization.cu:433-462) and sums in FP32; here chi is read in FP64,
//   taken relative to each element's node 0, and the reduction is FP64
//   (per-thread partials, then a fixed-order two-stage sum).
#include "h3d_internal.cuh"

namespace h3d {

// unit macro-strain displacement chi0 of local node a, strain case c, component m
// (homoCommon.cuh:455-519)
__host__ __device__ constexpr float macro_disp(int a, int c, int m) {
    const int p0 = a & 1, p1 = (a >> 1) & 1, p2 = a >> 2;
    return c == 0 ? (m == 0 ? (float)p0 : 0.f)
         : c == 1 ? (m == 1 ? (float)p1 : 0.f)
         : c == 2 ? (m == 2 ? (float)p2 : 0.f)
         : c == 3 ? (m == 1 ? p2 * 0.5f : m == 2 ? p1 * 0.5f : 0.f)
         : c == 4 ? (m == 0 ? p2 * 0.5f : m == 2 ? p0 * 0.5f : 0.f)
                  : (m == 0 ? p1 * 0.5f : m == 1 ? p0 * 0.5f : 0.f);
}

// E[t] for the 21 pairs (i <= j) of element e = (x,y,z)
// chi is FP64; the element's displacements are taken relative to its node 0
// (Ke annihilates translations), so the FP32 products see O(1) values even
// where chi itself is O(N)
__device__ __forceinline__ void element_energy(const Planes &P, const double *__restrict__ chi, const KeMat &ke,
                                               int x, int y, int z, float E[21]) {
    float U[NCASE][24];
    double c0[NF];
    {
        const long long v0 = vidx(P, x, y, z);
#pragma unroll
        for (int q = 0; q < NF; ++q) c0[q] = __ldg(&chi[q * P.nv + v0]);
    }
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const int vx = (a & 1) ? (x + 1 == P.n[0] ? 0 : x + 1) : x;
        const int vy = ((a >> 1) & 1) ? (y + 1 == P.n[1] ? 0 : y + 1) : y;
        const int vz = (a >> 2) ? (z + 1 == P.n[2] ? 0 : z + 1) : z;
        const long long v = vidx(P, vx, vy, vz);
#pragma unroll
        for (int c = 0; c < NCASE; ++c)
#pragma unroll
            for (int m = 0; m < 3; ++m)
                U[c][3 * a + m] = macro_disp(a, c, m) - (float)(__ldg(&chi[(3 * c + m) * P.nv + v]) - c0[3 * c + m]);
    }
    int t = 0;
#pragma unroll
    for (int j = 0; j < NCASE; ++j) {
        float KU[24];
#pragma unroll
        for (int r = 0; r < 24; ++r) {
            float s = 0.f;
#pragma unroll
            for (int q = 0; q < 24; ++q) s = fmaf(ke.k[r * 24 + q], U[j][q], s);
            KU[r] = s;
        }
#pragma unroll
        for (int i = 0; i <= j; ++i) {
            float s = 0.f;
#pragma unroll
            for (int r = 0; r < 24; ++r) s = fmaf(U[i][r], KU[r], s);
            // pair index of (i, j) with i <= j in row-major upper-triangle order
            E[i * 6 - i * (i - 1) / 2 + (j - i)] = s;
            ++t;
        }
    }
}

constexpr int EBS = 128;

int elastic_blocks(const Planes &P) {
    long long nb = (P.nv + EBS - 1) / EBS;
    return (int)(nb < 4096 ? nb : 4096);
}

__global__ void __launch_bounds__(EBS) k_elastic(Planes P, const double *__restrict__ chi, const float *__restrict__ rho,
                                                 const __grid_constant__ KeMat ke, double *partial) {
    double acc[21];
#pragma unroll
    for (int t = 0; t < 21; ++t) acc[t] = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < P.nv; e += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(e % P.n[0]);
        const long long tt = e / P.n[0];
        const int y = (int)(tt % P.n[1]), z = (int)(tt / P.n[1]);
        float E[21];
        element_energy(P, chi, ke, x, y, z, E);
        const double rp = (double)(RHO_PENAL_MIN + rho[e]);
#pragma unroll
        for (int t = 0; t < 21; ++t) acc[t] += rp * (double)E[t];
    }
    block_reduce<21>(acc, partial, blockIdx.x);
}

void launch_elastic_partials(const Planes &P, const double *chi, const float *rho, const KeMat &ke, double *partial,
                             int nblk, cudaStream_t s) {
    k_elastic<<<nblk, EBS, 0, s>>>(P, chi, rho, ke, partial);
}

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

struct DcTab { float w[21]; };  // (dC_ij + [i!=j] dC_ji) / |Y| for the 21 pairs

__global__ void __launch_bounds__(EBS) k_sensitivity(Planes P, const double *__restrict__ chi,
                                                     const __grid_constant__ KeMat ke, DcTab dc, float *sens,
                                                     int pitch) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= P.nv) return;
    const int x = (int)(e % P.n[0]);
    const long long tt = e / P.n[0];
    const int y = (int)(tt % P.n[1]), z = (int)(tt / P.n[1]);
    float E[21];
    element_energy(P, chi, ke, x, y, z, E);
    float s = 0.f;
#pragma unroll
    for (int t = 0; t < 21; ++t) s = fmaf(E[t], dc.w[t], s);
    sens[x + ((long long)y + (long long)z * P.n[1]) * pitch] = s;
}

void launch_sensitivity(const Planes &P, const double *chi, const KeMat &ke, const float *dc36, float *sens, int pitch,
                        cudaStream_t s) {
    DcTab t;
    const double vol = (double)P.nv;
    int q = 0;
    for (int i = 0; i < 6; ++i)
        for (int j = i; j < 6; ++j) {
            double w = dc36[i * 6 + j] + (i != j ? dc36[j * 6 + i] : 0.f);
            t.w[q++] = (float)(w / vol);
        }
    k_sensitivity<<<(unsigned)((P.nv + EBS - 1) / EBS), EBS, 0, s>>>(P, chi, ke, t, sens, pitch);
}

}  // namespace h3d
