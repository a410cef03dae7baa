// k_design.cu -- density input, OC update, sensitivity filter, symmetrisation.
//
// Reference behaviour restated (homo3d):
//   update_rho_kernel (grid.cu:4025-4064): pitched lexicographic density in.
//   OCOptimizer::update (OCOptimizer.cu:12-67): rho_new = clamp(rho *
//     max(-s/g, 0.01)^damp, rho +- step, [rho_min, 1]), 20 bisection steps on g
//     over [0, max|s|] until |vol - target| <= 1e-4.  Here the bisection state
//     lives on the device, so the update needs no host round trip per step.
//   OCOptimizer::filterSens (OCOptimizer.cu:76-152): s~_e = sum w rho s /
//     (sum w * rho_e), linear cone weight 1 - |d|/r on a (2*int(r+0.5)+1)^3
//     window, normalised by the full-window weight sum, optionally periodic.
//   symetrize_tensor_kernel (TensorExpression.cuh:72-): orbit averages with the
//     reference's FP32 summation order, so results are bit-identical.
#include "h3d_internal.cuh"

namespace h3d {

__global__ void k_density_in(int n0, int n1, int n2, const float *__restrict__ src, int pitch, float *dst) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long ne = (long long)n0 * n1 * n2;
    if (e >= ne) return;
    const int x = (int)(e % n0);
    const long long t = e / n0;
    const int y = (int)(t % n1), z = (int)(t / n1);
    dst[e] = src[x + ((long long)y + (long long)z * n1) * pitch];
}

// SIMP penalisation rho_phys = rho^p and its backward grad *= p rho^(p-1)
// (the reference builds these as the expression rho.pow(3), TensorExpression.h:517-531, 781-)
__global__ void k_penalize(long long n, const float *__restrict__ rho, float *out, float p, int backward) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float r = rho[i];
    if (backward) out[i] *= p * powf(r, p - 1.f);
    else out[i] = powf(r, p);
}

void launch_penalize(long long n, const float *rho, float *out, float p, int backward, cudaStream_t s) {
    k_penalize<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, rho, out, p, backward);
}

void launch_density_in(const int n[3], const float *src, int pitch, float *dst, cudaStream_t s) {
    const long long ne = (long long)n[0] * n[1] * n[2];
    k_density_in<<<(unsigned)((ne + 255) / 256), 256, 0, s>>>(n[0], n[1], n[2], src, pitch, dst);
}

// ---- OC ----------------------------------------------------------------------
// scratch layout: [0] lo, [1] hi, [2] done, [3] g, [4..] partial sums
constexpr int OC_BS = 256;
constexpr int OC_NB = 1184;  // 8 blocks per SM on 148 SMs

__global__ void __launch_bounds__(OC_BS) k_oc_maxabs(const float *__restrict__ s, long long n, double *partial) {
    double m = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmax(m, (double)fabsf(s[i]));
    __shared__ double sm[32];
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) partial[4 + blockIdx.x] = m;
    }
}

__global__ void k_oc_init(double *st, int nb) {
    if (threadIdx.x == 0) {
        double m = 0;
        for (int b = 0; b < nb; b++) m = fmax(m, st[4 + b]);
        st[0] = 0.0;
        st[1] = (double)(float)m;
        st[2] = 0.0;
    }
}

__global__ void __launch_bounds__(OC_BS) k_oc_step(const float *__restrict__ sens, const float *__restrict__ rho,
                                                   float *rho_new, long long n, float minrho, float step, float damp,
                                                   double *st) {
    if (st[2] != 0.0) return;  // converged in an earlier step: keep its densities
    const float g = ((float)st[1] + (float)st[0]) / 2;
    double s = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float r = rho[i];
        float B = -sens[i] / g;
        if (B < 0) B = 0.01f;
        float v = powf(B, damp) * r;
        if (v - r < -step) v = r - step;
        if (v - r > step) v = r + step;
        if (v < minrho) v = minrho;
        if (v > 1) v = 1;
        rho_new[i] = v;
        s += v;
    }
    double ss[1] = {s};
    block_reduce<1>(ss, st + 4, blockIdx.x);
}

__global__ void k_oc_decide(double *st, int nb, long long n, float vol) {
    if (threadIdx.x != 0 || st[2] != 0.0) return;
    double s = 0;
    for (int b = 0; b < nb; b++) s += st[4 + b];
    const float cur = (float)(s / (double)n);
    const float g = ((float)st[1] + (float)st[0]) / 2;
    if (cur < vol - 0.0001f) st[1] = g;
    else if (cur > vol + 0.0001f) st[0] = g;
    else st[2] = 1.0;
}

void launch_oc(const float *sens, float *rho, float *rho_new, long long n, float vol, float minrho, float step,
               float damp, double *scratch, cudaStream_t s) {
    k_oc_maxabs<<<OC_NB, OC_BS, 0, s>>>(sens, n, scratch);
    k_oc_init<<<1, 32, 0, s>>>(scratch, OC_NB);
    for (int it = 0; it < 20; ++it) {
        k_oc_step<<<OC_NB, OC_BS, 0, s>>>(sens, rho, rho_new, n, minrho, step, damp, scratch);
        k_oc_decide<<<1, 32, 0, s>>>(scratch, OC_NB, n, vol);
    }
    cudaMemcpyAsync(rho, rho_new, sizeof(float) * n, cudaMemcpyDeviceToDevice, s);
}

// ---- sensitivity filter ------------------------------------------------------
__global__ void __launch_bounds__(256) k_filter(int n0, int n1, int n2, int pitch, const float *__restrict__ sens,
                                                const float *__restrict__ rho, float *out, float radius, int hw,
                                                float wtot, int periodic) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long ne = (long long)n0 * n1 * n2;
    if (e >= ne) return;
    const int x = (int)(e % n0);
    const long long t = e / n0;
    const int y = (int)(t % n1), z = (int)(t / n1);
    float sum = 0.f, ws = 0.f;
    const int side = 2 * hw + 1;
    for (int id = 0; id < side * side * side; ++id) {
        const int ox = id % side - hw, oy = id / side % side - hw, oz = id / (side * side) - hw;
        const float r2 = (float)(ox * ox + oy * oy + oz * oz) / (radius * radius);
        float w = r2 < 1.f ? 1.f - sqrtf(r2) : 0.f;
        w /= wtot;
        int px = x + ox, py = y + oy, pz = z + oz;
        if (periodic) { px = (px + n0) % n0; py = (py + n1) % n1; pz = (pz + n2) % n2; }
        if (px < 0 || px >= n0 || py < 0 || py >= n1 || pz < 0 || pz >= n2) continue;
        const long long nid = px + ((long long)py + (long long)pz * n1) * pitch;
        sum += sens[nid] * rho[nid] * w;
        ws += w;
    }
    const long long me = x + ((long long)y + (long long)z * n1) * pitch;
    sum /= ws * rho[me];
    out[me] = sum;
}

void launch_filter(const int n[3], int pitch, const float *sens, const float *rho, float *out, float radius,
                   int periodic, cudaStream_t s) {
    const int hw = (int)(radius + 0.5f);
    float wtot = 0.f;
    const int side = 2 * hw + 1;
    for (int id = 0; id < side * side * side; ++id) {
        const int ox = id % side - hw, oy = id / side % side - hw, oz = id / (side * side) - hw;
        const float r2 = (float)(ox * ox + oy * oy + oz * oz) / (radius * radius);
        wtot += r2 < 1.f ? 1.f - sqrtf(r2) : 0.f;
    }
    const long long ne = (long long)n[0] * n[1] * n[2];
    k_filter<<<(unsigned)((ne + 255) / 256), 256, 0, s>>>(n[0], n[1], n[2], pitch, sens, rho, out, radius, hw, wtot,
                                                          periodic);
}

// ---- symmetrisation ------------------------------------------------------------
__device__ __forceinline__ long long lid(const int n[3], int a, int b, int c) {
    return a + (long long)n[0] * (b + (long long)n[1] * c);
}

__global__ void k_sym_reflect3(int n0, int n1, int n2, float *v) {
    const int n[3] = {n0, n1, n2}, h[3] = {n0 / 2, n1 / 2, n2 / 2};
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)h[0] * h[1] * h[2]) return;
    const int rp[3] = {(int)(t % h[0]), (int)(t / h[0] % h[1]), (int)(t / ((long long)h[0] * h[1]))};
    int orb[8][3];
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 3; j++) orb[i][j] = ((i >> j) & 1) ? n[j] - 1 - rp[j] : rp[j];
    float val = v[lid(n, orb[0][0], orb[0][1], orb[0][2])];
    for (int i = 1; i < 8; i++) val += v[lid(n, orb[i][0], orb[i][1], orb[i][2])];
    val /= 8;
    for (int i = 0; i < 8; i++) v[lid(n, orb[i][0], orb[i][1], orb[i][2])] = val;
}

__global__ void k_sym_reflect6(int n0, int h, float *v, long long nrep) {
    const int n[3] = {n0, n0, n0};
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= nrep) return;
    // representative x <= y <= z < h, enumerated tetrahedrally
    int z = (int)cbrtf(6.f * (float)t);
    while (z > 0 && (long long)z * (z + 1) * (z + 2) / 6 > t) z--;
    while ((long long)(z + 1) * (z + 2) * (z + 3) / 6 <= t) z++;
    long long rem = t - (long long)z * (z + 1) * (z + 2) / 6;
    int y = (int)sqrtf(2.f * (float)rem);
    while (y > 0 && (long long)y * (y + 1) / 2 > rem) y--;
    while ((long long)(y + 1) * (y + 2) / 2 <= rem) y++;
    const int x = (int)(rem - (long long)y * (y + 1) / 2);
    const int rp[3] = {x, y, z};
    float s = 0;
    for (int i = 0; i < 8; i++) {
        int o[3];
        for (int j = 0; j < 3; j++) o[j] = ((i >> j) & 1) ? n[j] - 1 - rp[j] : rp[j];
        s += v[lid(n, o[0], o[1], o[2])];
        s += v[lid(n, o[0], o[2], o[1])];
        s += v[lid(n, o[2], o[0], o[1])];
        s += v[lid(n, o[2], o[1], o[0])];
        s += v[lid(n, o[1], o[0], o[2])];
        s += v[lid(n, o[1], o[2], o[0])];
    }
    s /= 48;
    for (int i = 0; i < 8; i++) {
        int o[3];
        for (int j = 0; j < 3; j++) o[j] = ((i >> j) & 1) ? n[j] - 1 - rp[j] : rp[j];
        v[lid(n, o[0], o[1], o[2])] = s;
        v[lid(n, o[0], o[2], o[1])] = s;
        v[lid(n, o[2], o[0], o[1])] = s;
        v[lid(n, o[2], o[1], o[0])] = s;
        v[lid(n, o[1], o[0], o[2])] = s;
        v[lid(n, o[1], o[2], o[0])] = s;
    }
}

__global__ void k_sym_rotate3(int n0, int h, float *v, long long nrep) {
    const int n[3] = {n0, n0, n0};
    const int hh[3] = {h, h, h};
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= nrep) return;
    // representative z in [0,h), x, y in [0, z]
    int z = (int)cbrtf(3.f * (float)t);
    while (z > 0 && (long long)z * (z + 1) * (2 * z + 1) / 6 > t) z--;
    while ((long long)(z + 1) * (z + 2) * (2 * z + 3) / 6 <= t) z++;
    const long long rem = t - (long long)z * (z + 1) * (2 * z + 1) / 6;
    const int y = (int)(rem / (z + 1)), x = (int)(rem % (z + 1));
    const int rp[3] = {x, y, z};
    const int perm[6][3] = {{0, 2, 1}, {2, 1, 0}, {1, 0, 2}, {2, 0, 1}, {1, 2, 0}, {0, 1, 2}};
    const int fo[4][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 1}};
    const int fe[4][3] = {{0, 0, 0}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1}};
    // representatives with x, y <= z can share an orbit; the reference lets their
    // threads race, here each orbit is averaged once, by its first representative
    for (int i = 0; i < 6; i++) {
        const int o[3] = {rp[perm[i][0]], rp[perm[i][1]], rp[perm[i][2]]};
        for (int f = 0; f < 4; f++) {
            const int *fl = i < 3 ? fo[f] : fe[f];
            int q[3];
            for (int j = 0; j < 3; j++) q[j] = fl[j] ? -1 - o[j] : o[j];
            if (q[0] >= 0 && q[1] >= 0 && q[2] >= 0 && q[0] <= q[2] && q[1] <= q[2]) {
                const long long tq = (long long)q[2] * (q[2] + 1) * (2 * q[2] + 1) / 6 + (long long)q[1] * (q[2] + 1) + q[0];
                if (tq < t) return;
            }
        }
    }
    float s = 0;
    for (int i = 0; i < 6; i++) {
        const int o[3] = {rp[perm[i][0]], rp[perm[i][1]], rp[perm[i][2]]};
        for (int f = 0; f < 4; f++) {
            const int *fl = i < 3 ? fo[f] : fe[f];
            int p[3];
            for (int j = 0; j < 3; j++) p[j] = fl[j] ? hh[j] - 1 - o[j] : hh[j] + o[j];
            s += v[lid(n, p[0], p[1], p[2])];
        }
    }
    s /= 24;
    for (int i = 0; i < 6; i++) {
        const int o[3] = {rp[perm[i][0]], rp[perm[i][1]], rp[perm[i][2]]};
        for (int f = 0; f < 4; f++) {
            const int *fl = i < 3 ? fo[f] : fe[f];
            int p[3];
            for (int j = 0; j < 3; j++) p[j] = fl[j] ? hh[j] - 1 - o[j] : hh[j] + o[j];
            v[lid(n, p[0], p[1], p[2])] = s;
        }
    }
}

void launch_symmetrize(const int n[3], float *v, int sym, cudaStream_t s) {
    const int h = n[0] / 2;
    if (sym == 0) {
        const long long nr = (long long)(n[0] / 2) * (n[1] / 2) * (n[2] / 2);
        k_sym_reflect3<<<(unsigned)((nr + 255) / 256), 256, 0, s>>>(n[0], n[1], n[2], v);
    } else if (sym == 1) {
        const long long nr = (long long)h * (h + 1) * (h + 2) / 6;
        k_sym_reflect6<<<(unsigned)((nr + 255) / 256), 256, 0, s>>>(n[0], h, v, nr);
    } else if (sym == 2) {
        const long long nr = (long long)h * (h + 1) * (2 * h + 1) / 6;
        k_sym_rotate3<<<(unsigned)((nr + 255) / 256), 256, 0, s>>>(n[0], h, v, nr);
    }
}

// ---- the reference's trig-basis initial density -----------------------------------
// randTribase_sincos_kernel (Framework.cuh:106-222) and randTri (Framework.cuh:238-310):
// at voxel (x, y, z) with p = (x, y, z) / (dim - 1) (centred: p - 1/2 rotated by the
// unit quaternion of the four coefficients after the basis ones), with
// c[a][i] = cos(2 pi (i+1) p_a), s[a][i] = sin(2 pi (i+1) p_a), i < P:
//   first order,  6P terms:   coeff[i] c[i%3][i/3] for i < 3P, then
//                             coeff[i] s[j%3][j/3] with j = i - 3P;
//   second order, 36P^2 terms: coeff[6P + 6P j + k] v(j) v(k), j, k < 6P, where
//                             v(j) = c[j/P][j%P] for j < 3P, s[j/P-3][j%P] otherwise.
// One thread per voxel; its 6P basis values v(j) in shared memory (P <= 50).  The
// sum runs in FP64 and is rounded to FP32 (the reference sums eight FP32 partials of
// a warp-strided split).
struct TrigArgs {
    int n[3];
    int P;
    int centered;
    float rot[9];  // row-major rotation of the centred position
};

constexpr int TRIG_BS = 64;

__global__ void __launch_bounds__(TRIG_BS) k_trig_basis(TrigArgs a, const float *__restrict__ coeff, float *out) {
    extern __shared__ float tv[];  // [6P][TRIG_BS]
    const long long ne = (long long)a.n[0] * a.n[1] * a.n[2];
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int P = a.P, t = threadIdx.x;
    float p[3] = {0.f, 0.f, 0.f};
    if (e < ne) {
        const int x = (int)(e % a.n[0]);
        const long long tt = e / a.n[0];
        const int y = (int)(tt % a.n[1]), z = (int)(tt / a.n[1]);
        p[0] = (float)x / (float)(a.n[0] - 1);
        p[1] = (float)y / (float)(a.n[1] - 1);
        p[2] = (float)z / (float)(a.n[2] - 1);
        if (a.centered) {
            const float q[3] = {p[0] - 0.5f, p[1] - 0.5f, p[2] - 0.5f};
            for (int r = 0; r < 3; ++r) p[r] = a.rot[3 * r] * q[0] + a.rot[3 * r + 1] * q[1] + a.rot[3 * r + 2] * q[2];
        }
    }
    constexpr float pi2 = 3.1415926f * 2;  // the reference's constant (Framework.cuh:113)
    for (int j = 0; j < 3 * P; ++j) {
        const int ax = j / P, i = j % P;
        tv[j * TRIG_BS + t] = cosf(pi2 * (i + 1) * p[ax]);
        tv[(3 * P + j) * TRIG_BS + t] = sinf(pi2 * (i + 1) * p[ax]);
    }
    if (e >= ne) return;
    double sum = 0;
    for (int i = 0; i < 6 * P; ++i) {  // first order: component fastest
        const int j = i < 3 * P ? i : i - 3 * P;
        const int v = (j % 3) * P + j / 3 + (i < 3 * P ? 0 : 3 * P);
        sum += (double)coeff[i] * (double)tv[v * TRIG_BS + t];
    }
    const float *c2 = coeff + 6 * P;
    for (int j = 0; j < 6 * P; ++j) {
        const double vj = (double)tv[j * TRIG_BS + t];
        double inner = 0;
        for (int k = 0; k < 6 * P; ++k) inner += (double)c2[6 * P * j + k] * (double)tv[k * TRIG_BS + t];
        sum += vj * inner;
    }
    out[e] = (float)sum;
}

// level-set volume search of randTri: x = m + (M - m) / (1 + exp(-15 (v - t))),
// M = min(1.5 vol, 1), m = 0.001; t bisected on [-37 P^2, 37 P^2] for at most 60
// steps until the mean is within 1e-3 (relative) of vol.
// state: [0] t_l, [1] t_u, [2] done, [3] t, [4 ..] block partial sums
__device__ __forceinline__ float trig_level_map(float v, float t, float M) {
    const float sgm = 1.f / (1 + expf(-15.f * (v - t)));
    return sgm * (M - 0.001f) + 0.001f;
}

__global__ void k_level_init(double *st, float P) {
    if (threadIdx.x == 0) {
        const float tu = P * P * 37;
        st[0] = -tu;
        st[1] = tu;
        st[2] = 0.0;
        st[3] = 0.0;
    }
}

__global__ void __launch_bounds__(OC_BS) k_level_step(const float *__restrict__ v, long long n, float M, double *st) {
    if (st[2] != 0.0) return;
    const float t = ((float)st[1] + (float)st[0]) / 2;
    double s = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s += trig_level_map(v[i], t, M);
    double ss[1] = {s};
    block_reduce<1>(ss, st + 4, blockIdx.x);
}

__global__ void k_level_decide(double *st, int nb, long long n, float vol) {
    if (threadIdx.x != 0 || st[2] != 0.0) return;
    double s = 0;
    for (int b = 0; b < nb; b++) s += st[4 + b];
    const float mean = (float)(s / (double)n);
    const float t = ((float)st[1] + (float)st[0]) / 2;
    st[3] = t;
    if (fabsf(mean - vol) / vol < 1e-3f) {
        st[2] = 1.0;
        return;
    }
    if (mean > vol) st[0] = t;
    if (mean < vol) st[1] = t;
}

__global__ void k_level_apply(float *v, long long n, float M, const double *st) {
    const float t = (float)st[3];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[i] = trig_level_map(v[i], t, M);
}

int launch_trig_init(const int n[3], int P, const float *coeff_dev, int centered, const float rot[9], float vol, int sym,
                     float *rho, double *scratch, cudaStream_t s) {
    TrigArgs a;
    for (int d = 0; d < 3; ++d) a.n[d] = n[d];
    a.P = P;
    a.centered = centered;
    for (int i = 0; i < 9; ++i) a.rot[i] = rot[i];
    const long long ne = (long long)n[0] * n[1] * n[2];
    const size_t smem = sizeof(float) * 6 * P * TRIG_BS;
    if (cudaFuncSetAttribute((const void *)k_trig_basis, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return -1;
    k_trig_basis<<<(unsigned)((ne + TRIG_BS - 1) / TRIG_BS), TRIG_BS, smem, s>>>(a, coeff_dev, rho);
    if (sym >= 0) launch_symmetrize(n, rho, sym, s);
    const float M = fminf(vol * 1.5f, 1.f);
    k_level_init<<<1, 32, 0, s>>>(scratch, (float)P);
    for (int it = 0; it < 60; ++it) {
        k_level_step<<<OC_NB, OC_BS, 0, s>>>(rho, ne, M, scratch);
        k_level_decide<<<1, 32, 0, s>>>(scratch, OC_NB, ne, vol);
    }
    k_level_apply<<<OC_NB, OC_BS, 0, s>>>(rho, ne, M, scratch);
    return 0;
}

// ---- radial convolution of the expression layer ---------------------------------
// rho.conv(radial_convker_t<Spline4>(r)) (TensorExpression.h:946-1131,
// TensorExpression.cuh:288-369): window offsets |o_a| <= (int)(r + 0.5), weight
// w(o) = 1 - 6 q + 8 q^1.5 - 3 q^2 for q = |o|^2 / r^2 < 1 (0 otherwise); out(p) =
// sum_o w(o) in(p + o) / ws(p) over the offsets inside the grid (periodic: all,
// wrapped), ws(p) the sum of those weights.  The adjoint (the backward of the
// expression) is g_in(p) = sum_o w(o) g_out(p - o) / ws(p - o).
__device__ __forceinline__ float spline4_weight(int ox, int oy, int oz, float r) {
    const float q = (float)(ox * ox + oy * oy + oz * oz) / (r * r);
    const float rq = sqrtf(q);
    return q < 1.f ? 1.f - 6.f * q + 8.f * q * rq - 3.f * q * q : 0.f;
}

// mode 0: out = conv(in), ws = weight sums; mode 1: ws only; mode 2: out = adjoint(in) with ws
__global__ void __launch_bounds__(256) k_conv_radial(int n0, int n1, int n2, const float *__restrict__ in, float *out,
                                                     float *ws, float r, int hw, int periodic, int mode) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long ne = (long long)n0 * n1 * n2;
    if (e >= ne) return;
    const int x = (int)(e % n0);
    const long long t = e / n0;
    const int y = (int)(t % n1), z = (int)(t / n1);
    float sum = 0.f, wsum = 0.f;
    for (int oz = -hw; oz <= hw; ++oz)
        for (int oy = -hw; oy <= hw; ++oy)
            for (int ox = -hw; ox <= hw; ++ox) {
                const float w = spline4_weight(ox, oy, oz, r);
                // forward reads p + o, the adjoint p - o
                int px = mode == 2 ? x - ox : x + ox, py = mode == 2 ? y - oy : y + oy, pz = mode == 2 ? z - oz : z + oz;
                const bool inside = px >= 0 && px < n0 && py >= 0 && py < n1 && pz >= 0 && pz < n2;
                if (!inside && !periodic) continue;
                if (!inside) { px = (px + n0) % n0; py = (py + n1) % n1; pz = (pz + n2) % n2; }
                const long long q = px + (long long)n0 * (py + (long long)n1 * pz);
                wsum += w;
                if (mode == 0) sum += w * in[q];
                else if (mode == 2) sum += w * in[q] / ws[q];
            }
    if (mode == 0) { out[e] = sum / wsum; ws[e] = wsum; }
    else if (mode == 1) ws[e] = wsum;
    else out[e] = sum;
}

void launch_conv_radial(const int n[3], const float *in, float *out, float *ws, float radius, int periodic,
                        int adjoint, cudaStream_t s) {
    const int hw = (int)(radius + 0.5f);
    const long long ne = (long long)n[0] * n[1] * n[2];
    const unsigned nb = (unsigned)((ne + 255) / 256);
    if (!adjoint) {
        k_conv_radial<<<nb, 256, 0, s>>>(n[0], n[1], n[2], in, out, ws, radius, hw, periodic, 0);
    } else {
        k_conv_radial<<<nb, 256, 0, s>>>(n[0], n[1], n[2], in, out, ws, radius, hw, periodic, 1);
        k_conv_radial<<<nb, 256, 0, s>>>(n[0], n[1], n[2], in, out, ws, radius, hw, periodic, 2);
    }
}

}  // namespace h3d
