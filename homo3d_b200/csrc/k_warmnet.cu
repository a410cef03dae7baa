// k_warmnet.cu -- the learned warm start: a small periodic 3-D convolutional
// encoder-decoder that maps the density (averaged to an R^3 grid) to the six
// cell solutions chi_c / N at the R^3 coarse vertices, with hand-written forward,
// backward and Adam kernels, and the kernels that turn its prediction into the
// stored solutions a solve starts from.  No reference counterpart (the reference
// warm-starts only from the previous design's solutions, homogenization.cu:471-477).
//
// Network (R divisible by 8; channels 16, 32, 64, 64; every 3x3x3 convolution is
// periodic, i.e. circular padding, and followed by ReLU):
//   a0 = conv(x, 1->16)             at R        p1 = avgpool2(a0)
//   a1 = conv(p1, 16->32)           at R/2      p2 = avgpool2(a1)
//   a2 = conv(p2, 32->64)           at R/4      p3 = avgpool2(a2)
//   a3 = conv(p3, 64->64)           at R/8
//   d2 = conv(up2(a3) + a2, 64->32) at R/4
//   d1 = conv(up2(d2) + a1, 32->16) at R/2
//   d0 = conv(up2(d1) + a0, 16->16) at R
//   y  = W_out d0 + b_out (1x1, 16->18, linear)
// up2 is nearest-neighbour upsampling.  Activations are [batch][channel][R^3]
// FP32, voxel index x + R*(y + R*z).  Weights FP32, [cout][cin][27] with tap
// t = (dx+1) + 3(dy+1) + 9(dz+1).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/h3d.h"
#include "h3d_internal.cuh"

namespace h3d {

constexpr int WN_BS = 128;
constexpr int WN_CO = 8;  // output channels per thread in the convolution kernels

__device__ __forceinline__ int wn_wrap(int a, int r) { return a < 0 ? a + r : (a >= r ? a - r : a); }

// y[b][co][v] = bias[co] + sum_ci sum_t W[co][ci][t] x[b][ci][v + off(t)], then
// optionally ReLU.  TRANSPOSED computes the input gradient of a convolution:
// dx[b][ci][v] = sum_co sum_t W[co][ci][t] dy[b][co][v - off(t)] (the kernel's
// input channels are the convolution's outputs; taps mirrored; no bias).
template <bool TRANSPOSED>
__global__ void __launch_bounds__(WN_BS) k_wn_conv3(const float *__restrict__ x, const float *__restrict__ W,
                                                   const float *__restrict__ bias, float *y, int Cin, int Cout, int R,
                                                   int relu) {
    const int R3 = R * R * R;
    const int v = blockIdx.x * WN_BS + threadIdx.x;
    const int co0 = blockIdx.y * WN_CO, b = blockIdx.z;
    if (v >= R3) return;
    const int vx = v % R, vy = (v / R) % R, vz = v / (R * R);
    const int s = TRANSPOSED ? -1 : 1;
    int nb[27];
#pragma unroll
    for (int t = 0; t < 27; ++t) {
        const int dx = t % 3 - 1, dy = t / 3 % 3 - 1, dz = t / 9 - 1;
        nb[t] = wn_wrap(vx + s * dx, R) + R * (wn_wrap(vy + s * dy, R) + R * wn_wrap(vz + s * dz, R));
    }
    float acc[WN_CO];
#pragma unroll
    for (int q = 0; q < WN_CO; ++q) acc[q] = (!TRANSPOSED && bias && co0 + q < Cout) ? bias[co0 + q] : 0.f;
    const float *xb = x + (long long)b * Cin * R3;
    for (int ci = 0; ci < Cin; ++ci) {
        const float *xc = xb + (long long)ci * R3;
        float in[27];
#pragma unroll
        for (int t = 0; t < 27; ++t) in[t] = __ldg(xc + nb[t]);
#pragma unroll
        for (int q = 0; q < WN_CO; ++q) {
            const int co = co0 + q;
            if (co < Cout) {
                const float *w = TRANSPOSED ? W + ((long long)ci * Cout + co) * 27 : W + ((long long)co * Cin + ci) * 27;
                float a = acc[q];
#pragma unroll
                for (int t = 0; t < 27; ++t) a = fmaf(__ldg(w + t), in[t], a);
                acc[q] = a;
            }
        }
    }
    float *yb = y + (long long)b * Cout * R3;
#pragma unroll
    for (int q = 0; q < WN_CO; ++q) {
        const int co = co0 + q;
        if (co < Cout) yb[(long long)co * R3 + v] = relu ? fmaxf(acc[q], 0.f) : acc[q];
    }
}

// dW[co][ci][t] += sum_b sum_v dz[b][co][v] x[b][ci][v + off(t)], and for ci == 0
// db[co] += sum dz[b][co][v]; one block per (co, ci), fixed-order reduction
__global__ void __launch_bounds__(WN_BS) k_wn_conv3_wgrad(const float *__restrict__ x, const float *__restrict__ dz,
                                                         float *dW, float *db, int Cin, int Cout, int R, int B) {
    const int co = blockIdx.x / Cin, ci = blockIdx.x % Cin;
    const int R3 = R * R * R;
    float g[28];
#pragma unroll
    for (int t = 0; t < 28; ++t) g[t] = 0.f;
    for (int b = 0; b < B; ++b) {
        const float *xc = x + ((long long)b * Cin + ci) * R3;
        const float *dc = dz + ((long long)b * Cout + co) * R3;
        for (int v = threadIdx.x; v < R3; v += WN_BS) {
            const int vx = v % R, vy = (v / R) % R, vz = v / (R * R);
            const float d = __ldg(dc + v);
#pragma unroll
            for (int t = 0; t < 27; ++t) {
                const int dx = t % 3 - 1, dy = t / 3 % 3 - 1, dzz = t / 9 - 1;
                const int n = wn_wrap(vx + dx, R) + R * (wn_wrap(vy + dy, R) + R * wn_wrap(vz + dzz, R));
                g[t] = fmaf(d, __ldg(xc + n), g[t]);
            }
            g[27] += d;
        }
    }
    __shared__ float red[28][WN_BS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int t = 0; t < 28; ++t) {
        float v = g[t];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[t][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 28) {
        float v = 0.f;
        for (int w = 0; w < WN_BS / 32; ++w) v += red[threadIdx.x][w];
        if (threadIdx.x < 27) dW[((long long)co * Cin + ci) * 27 + threadIdx.x] += v;
        else if (ci == 0) db[co] += v;
    }
}

// 1x1 output layer: y[b][o][v] = bias[o] + sum_c W[o][c] x[b][c][v]
__global__ void k_wn_out_fwd(const float *__restrict__ x, const float *__restrict__ W, const float *__restrict__ bias,
                             float *y, int Cin, int Cout, int R3, int B) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * R3) return;
    const int b = (int)(i / R3), v = (int)(i % R3);
    const float *xb = x + (long long)b * Cin * R3 + v;
    for (int o = 0; o < Cout; ++o) {
        float s = bias[o];
        for (int c = 0; c < Cin; ++c) s = fmaf(W[o * Cin + c], xb[(long long)c * R3], s);
        y[((long long)b * Cout + o) * R3 + v] = s;
    }
}

// input gradient of the 1x1 layer, masked by the ReLU that produced its input x:
// dx[b][c][v] = (x > 0) * sum_o W[o][c] dy[b][o][v]
__global__ void k_wn_out_bwd(const float *__restrict__ dy, const float *__restrict__ W, const float *__restrict__ x,
                             float *dx, int Cin, int Cout, int R3, int B) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * R3) return;
    const int b = (int)(i / R3), v = (int)(i % R3);
    for (int c = 0; c < Cin; ++c) {
        float s = 0.f;
        for (int o = 0; o < Cout; ++o) s = fmaf(W[o * Cin + c], dy[((long long)b * Cout + o) * R3 + v], s);
        const long long k = ((long long)b * Cin + c) * R3 + v;
        dx[k] = x[k] > 0.f ? s : 0.f;
    }
}

// weight gradient of the 1x1 layer: one block per (o, c), c == Cin for the bias
__global__ void __launch_bounds__(WN_BS) k_wn_out_wgrad(const float *__restrict__ x, const float *__restrict__ dy,
                                                       float *dW, float *db, int Cin, int Cout, int R3, int B) {
    const int o = blockIdx.x / (Cin + 1), c = blockIdx.x % (Cin + 1);
    float s = 0.f;
    for (int b = 0; b < B; ++b)
        for (int v = threadIdx.x; v < R3; v += WN_BS) {
            const float d = dy[((long long)b * Cout + o) * R3 + v];
            s = fmaf(d, c < Cin ? x[((long long)b * Cin + c) * R3 + v] : 1.f, s);
        }
    __shared__ float red[WN_BS / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float v = 0.f;
        for (int w = 0; w < WN_BS / 32; ++w) v += red[w];
        if (c < Cin) dW[o * Cin + c] += v;
        else db[o] += v;
    }
}

// dz = dy * (y > 0), in place on dy
__global__ void k_wn_relu_bwd(float *dy, const float *__restrict__ y, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n && !(y[i] > 0.f)) dy[i] = 0.f;
}

// 2x average pooling of [B*C][R^3] to [B*C][(R/2)^3]
__global__ void k_wn_pool(const float *__restrict__ x, float *y, int R, long long BC) {
    const int h = R / 2, h3 = h * h * h;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= BC * h3) return;
    const long long bc = i / h3;
    const int v = (int)(i % h3), X = v % h, Y = (v / h) % h, Z = v / (h * h);
    const float *xc = x + bc * R * R * R;
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q)
        s += xc[(2 * X + (q & 1)) + R * ((2 * Y + ((q >> 1) & 1)) + R * (2 * Z + (q >> 2)))];
    y[i] = 0.125f * s;
}

// gradient of the pooling, added: gx[child] += gy[parent] / 8
__global__ void k_wn_pool_bwd_add(const float *__restrict__ gy, float *gx, int R, long long BC) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long R3 = (long long)R * R * R;
    if (i >= BC * R3) return;
    const long long bc = i / R3;
    const int v = (int)(i % R3), x = v % R, y = (v / R) % R, z = v / (R * R), h = R / 2;
    gx[i] += 0.125f * gy[bc * h * h * h + (x / 2) + h * ((y / 2) + h * (z / 2))];
}

// out = up2(c) + skip
__global__ void k_wn_up_add(const float *__restrict__ c, const float *__restrict__ skip, float *out, int R,
                            long long BC) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long R3 = (long long)R * R * R;
    if (i >= BC * R3) return;
    const long long bc = i / R3;
    const int v = (int)(i % R3), x = v % R, y = (v / R) % R, z = v / (R * R), h = R / 2;
    out[i] = c[bc * h * h * h + (x / 2) + h * ((y / 2) + h * (z / 2))] + skip[i];
}

// gradient of up2: gc[parent] = sum of g over its 8 children
__global__ void k_wn_up_bwd(const float *__restrict__ g, float *gc, int R, long long BC) {
    const int h = R / 2, h3 = h * h * h;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= BC * h3) return;
    const long long bc = i / h3;
    const int v = (int)(i % h3), X = v % h, Y = (v / h) % h, Z = v / (h * h);
    const float *gb = g + bc * R * R * R;
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q)
        s += gb[(2 * X + (q & 1)) + R * ((2 * Y + ((q >> 1) & 1)) + R * (2 * Z + (q >> 2)))];
    gc[i] = s;
}

// mean squared error: dy = 2 (y - t) / n, per-block FP64 partial sums of (y - t)^2
__global__ void __launch_bounds__(256) k_wn_mse(const float *__restrict__ y, const float *__restrict__ t, float *dy,
                                                long long n, double *partial) {
    double s = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float d = y[i] - t[i];
        dy[i] = 2.f * d / (float)n;
        s += (double)d * d;
    }
    double v[1] = {s};
    block_reduce<1>(v, partial, blockIdx.x);
}

__global__ void k_wn_sum(const double *__restrict__ partial, int nblk, double *out, double scale) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0;
        for (int b = 0; b < nblk; ++b) s += partial[b];
        out[0] = s * scale;
    }
}

// Adam (Kingma & Ba 2015): m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2,
// w -= lr (m / c1) / (sqrt(v / c2) + eps) with c1 = 1-b1^t, c2 = 1-b2^t; g cleared
__global__ void k_wn_adam(float *w, float *g, float *m, float *v, long long n, float lr, float b1, float b2, float c1,
                          float c2, float eps) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    g[i] = 0.f;
}

// network input from a handle's density: mean of rho_phys over the s^3 fine
// cells of each of the R^3 coarse cells (s = N / R)
__global__ void k_wn_density_pool(const float *__restrict__ rho, int N, int R, float *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int R3 = R * R * R;
    if (i >= R3) return;
    const int s = N / R, X = i % R, Y = (i / R) % R, Z = i / (R * R);
    double acc = 0;
    for (int dz = 0; dz < s; ++dz)
        for (int dy = 0; dy < s; ++dy)
            for (int dx = 0; dx < s; ++dx)
                acc += rho[(X * s + dx) + (long long)N * ((Y * s + dy) + (long long)N * (Z * s + dz))];
    out[i] = (float)(acc / ((double)s * s * s));
}

// stored solutions from the prediction: chi(case c, comp m, fine vertex) =
// N * periodic trilinear interpolation of y[3c+m] over the R^3 coarse vertices
__global__ void k_wn_to_chi(Planes P, const float *__restrict__ y, int R, double *chi) {
    const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v >= P.nv) return;
    const int k = color_of_index(P, v);
    int x, yy, z;
    vpos(P, k, v - P.base[k], x, yy, z);
    const int N = P.n[0], s = N / R, R3 = R * R * R;
    const int X0 = x / s, Y0 = yy / s, Z0 = z / s;
    const float fx = (float)(x % s) / s, fy = (float)(yy % s) / s, fz = (float)(z % s) / s;
    int idx[8];
    float w[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int ox = q & 1, oy = (q >> 1) & 1, oz = q >> 2;
        idx[q] = ((X0 + ox) % R) + R * (((Y0 + oy) % R) + R * ((Z0 + oz) % R));
        w[q] = (ox ? fx : 1.f - fx) * (oy ? fy : 1.f - fy) * (oz ? fz : 1.f - fz);
    }
    for (int q = 0; q < NF; ++q) {
        float a = 0.f;
#pragma unroll
        for (int t = 0; t < 8; ++t) a = fmaf(w[t], y[(long long)q * R3 + idx[t]], a);
        chi[fidx(q, v)] = (double)N * (double)a;
    }
}

}  // namespace h3d

// ---- host side: the network object and the C ABI -----------------------------
using namespace h3d;

namespace {

constexpr int WN_NCONV = 7;
// (cin, cout, level) of the seven 3x3x3 convolutions e0 e1 e2 e3 d2 d1 d0
constexpr int WN_LAYER[WN_NCONV][3] = {{1, 16, 0}, {16, 32, 1}, {32, 64, 2}, {64, 64, 3},
                                       {64, 32, 2}, {32, 16, 1}, {16, 16, 0}};
constexpr int WN_OUT_IN = 16, WN_OUT = NF;

}  // namespace

struct h3d_warmnet {
    int R = 0, maxB = 0, device = 0;
    cudaStream_t stream = nullptr;
    long long nparam = 0;
    long long woff[WN_NCONV + 1] = {}, boff[WN_NCONV + 1] = {};  // index WN_NCONV: output layer
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    // activations and their gradients, [maxB][C][R_l^3]
    float *a0, *p1, *a1, *p2, *a2, *p3, *a3, *u2, *d2, *u1, *d1, *u0, *d0, *y;
    float *ga0, *gp1, *ga1, *gp2, *ga2, *gp3, *ga3, *gu2, *gd2, *gu1, *gd1, *gu0, *gd0, *gy;
    float *act = nullptr;
    double *partial = nullptr, *d_loss = nullptr, *h_loss = nullptr;
    long long step = 0;
    std::string err;
    int lvl(int l) const { return R >> l; }
    long long vol(int l) const { const long long r = lvl(l); return r * r * r; }
};

namespace {

int wn_fail(h3d_warmnet *n, int code, const std::string &msg) {
    if (n) n->err = msg;
    return code;
}

#define WCK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return wn_fail(n, H3D_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

inline unsigned nblk(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

uint64_t splitmix(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void conv(h3d_warmnet *n, int layer, const float *x, float *y, int B, cudaStream_t s) {
    const int ci = WN_LAYER[layer][0], co = WN_LAYER[layer][1], R = n->lvl(WN_LAYER[layer][2]);
    const dim3 grid(nblk((long long)R * R * R, WN_BS), (co + WN_CO - 1) / WN_CO, B);
    k_wn_conv3<false><<<grid, WN_BS, 0, s>>>(x, n->w + n->woff[layer], n->w + n->boff[layer], y, ci, co, R, 1);
}

// input gradient of convolution `layer` from its (ReLU-masked) output gradient gz
void conv_bwd_data(h3d_warmnet *n, int layer, const float *gz, float *gx, int B, cudaStream_t s) {
    const int ci = WN_LAYER[layer][0], co = WN_LAYER[layer][1], R = n->lvl(WN_LAYER[layer][2]);
    const dim3 grid(nblk((long long)R * R * R, WN_BS), (ci + WN_CO - 1) / WN_CO, B);
    k_wn_conv3<true><<<grid, WN_BS, 0, s>>>(gz, n->w + n->woff[layer], nullptr, gx, co, ci, R, 0);
}

void conv_wgrad(h3d_warmnet *n, int layer, const float *x, const float *gz, int B, cudaStream_t s) {
    const int ci = WN_LAYER[layer][0], co = WN_LAYER[layer][1], R = n->lvl(WN_LAYER[layer][2]);
    k_wn_conv3_wgrad<<<co * ci, WN_BS, 0, s>>>(x, gz, n->g + n->woff[layer], n->g + n->boff[layer], ci, co, R, B);
}

void relu_bwd(float *g, const float *y, long long cnt, cudaStream_t s) {
    k_wn_relu_bwd<<<nblk(cnt, 256), 256, 0, s>>>(g, y, cnt);
}

int forward(h3d_warmnet *n, const float *x, int B, cudaStream_t s) {
    const long long b = B;
    conv(n, 0, x, n->a0, B, s);
    k_wn_pool<<<nblk(b * 16 * n->vol(1), 256), 256, 0, s>>>(n->a0, n->p1, n->lvl(0), b * 16);
    conv(n, 1, n->p1, n->a1, B, s);
    k_wn_pool<<<nblk(b * 32 * n->vol(2), 256), 256, 0, s>>>(n->a1, n->p2, n->lvl(1), b * 32);
    conv(n, 2, n->p2, n->a2, B, s);
    k_wn_pool<<<nblk(b * 64 * n->vol(3), 256), 256, 0, s>>>(n->a2, n->p3, n->lvl(2), b * 64);
    conv(n, 3, n->p3, n->a3, B, s);
    k_wn_up_add<<<nblk(b * 64 * n->vol(2), 256), 256, 0, s>>>(n->a3, n->a2, n->u2, n->lvl(2), b * 64);
    conv(n, 4, n->u2, n->d2, B, s);
    k_wn_up_add<<<nblk(b * 32 * n->vol(1), 256), 256, 0, s>>>(n->d2, n->a1, n->u1, n->lvl(1), b * 32);
    conv(n, 5, n->u1, n->d1, B, s);
    k_wn_up_add<<<nblk(b * 16 * n->vol(0), 256), 256, 0, s>>>(n->d1, n->a0, n->u0, n->lvl(0), b * 16);
    conv(n, 6, n->u0, n->d0, B, s);
    k_wn_out_fwd<<<nblk(b * n->vol(0), 128), 128, 0, s>>>(n->d0, n->w + n->woff[WN_NCONV], n->w + n->boff[WN_NCONV],
                                                         n->y, WN_OUT_IN, WN_OUT, (int)n->vol(0), B);
    return cudaGetLastError() == cudaSuccess ? (int)H3D_OK : wn_fail(n, H3D_ERR_CUDA, "forward launch failed");
}

// gradients of the mean squared error against target t, accumulated into g
int backward(h3d_warmnet *n, const float *x, const float *t, int B, cudaStream_t s) {
    const long long b = B, V0 = n->vol(0), V1 = n->vol(1), V2 = n->vol(2), V3 = n->vol(3);
    const long long ny = b * WN_OUT * V0;
    const int nb = 256;
    k_wn_mse<<<nb, 256, 0, s>>>(n->y, t, n->gy, ny, n->partial);
    k_wn_sum<<<1, 32, 0, s>>>(n->partial, nb, n->d_loss, 1.0 / (double)ny);
    k_wn_out_wgrad<<<WN_OUT * (WN_OUT_IN + 1), WN_BS, 0, s>>>(n->d0, n->gy, n->g + n->woff[WN_NCONV],
                                                             n->g + n->boff[WN_NCONV], WN_OUT_IN, WN_OUT, (int)V0, B);
    k_wn_out_bwd<<<nblk(b * V0, 128), 128, 0, s>>>(n->gy, n->w + n->woff[WN_NCONV], n->d0, n->gd0, WN_OUT_IN, WN_OUT,
                                                  (int)V0, B);
    // d0 = relu(conv6(u0)), u0 = up(d1) + a0
    conv_wgrad(n, 6, n->u0, n->gd0, B, s);
    conv_bwd_data(n, 6, n->gd0, n->gu0, B, s);
    k_wn_up_bwd<<<nblk(b * 16 * V1, 256), 256, 0, s>>>(n->gu0, n->gd1, n->lvl(0), b * 16);
    cudaMemcpyAsync(n->ga0, n->gu0, sizeof(float) * b * 16 * V0, cudaMemcpyDeviceToDevice, s);
    // d1 = relu(conv5(u1)), u1 = up(d2) + a1
    relu_bwd(n->gd1, n->d1, b * 16 * V1, s);
    conv_wgrad(n, 5, n->u1, n->gd1, B, s);
    conv_bwd_data(n, 5, n->gd1, n->gu1, B, s);
    k_wn_up_bwd<<<nblk(b * 32 * V2, 256), 256, 0, s>>>(n->gu1, n->gd2, n->lvl(1), b * 32);
    cudaMemcpyAsync(n->ga1, n->gu1, sizeof(float) * b * 32 * V1, cudaMemcpyDeviceToDevice, s);
    // d2 = relu(conv4(u2)), u2 = up(a3) + a2
    relu_bwd(n->gd2, n->d2, b * 32 * V2, s);
    conv_wgrad(n, 4, n->u2, n->gd2, B, s);
    conv_bwd_data(n, 4, n->gd2, n->gu2, B, s);
    k_wn_up_bwd<<<nblk(b * 64 * V3, 256), 256, 0, s>>>(n->gu2, n->ga3, n->lvl(2), b * 64);
    cudaMemcpyAsync(n->ga2, n->gu2, sizeof(float) * b * 64 * V2, cudaMemcpyDeviceToDevice, s);
    // a3 = relu(conv3(p3)), p3 = pool(a2)
    relu_bwd(n->ga3, n->a3, b * 64 * V3, s);
    conv_wgrad(n, 3, n->p3, n->ga3, B, s);
    conv_bwd_data(n, 3, n->ga3, n->gp3, B, s);
    k_wn_pool_bwd_add<<<nblk(b * 64 * V2, 256), 256, 0, s>>>(n->gp3, n->ga2, n->lvl(2), b * 64);
    // a2 = relu(conv2(p2)), p2 = pool(a1)
    relu_bwd(n->ga2, n->a2, b * 64 * V2, s);
    conv_wgrad(n, 2, n->p2, n->ga2, B, s);
    conv_bwd_data(n, 2, n->ga2, n->gp2, B, s);
    k_wn_pool_bwd_add<<<nblk(b * 32 * V1, 256), 256, 0, s>>>(n->gp2, n->ga1, n->lvl(1), b * 32);
    // a1 = relu(conv1(p1)), p1 = pool(a0)
    relu_bwd(n->ga1, n->a1, b * 32 * V1, s);
    conv_wgrad(n, 1, n->p1, n->ga1, B, s);
    conv_bwd_data(n, 1, n->ga1, n->gp1, B, s);
    k_wn_pool_bwd_add<<<nblk(b * 16 * V0, 256), 256, 0, s>>>(n->gp1, n->ga0, n->lvl(0), b * 16);
    // a0 = relu(conv0(x))
    relu_bwd(n->ga0, n->a0, b * 16 * V0, s);
    conv_wgrad(n, 0, x, n->ga0, B, s);
    return cudaGetLastError() == cudaSuccess ? (int)H3D_OK : wn_fail(n, H3D_ERR_CUDA, "backward launch failed");
}

int check_batch(h3d_warmnet *n, int B) {
    if (B < 1 || B > n->maxB) return wn_fail(n, H3D_ERR_ARG, "batch outside 1..max_batch");
    return H3D_OK;
}

}  // namespace

namespace h3d {
int warmnet_reso(const h3d_warmnet *n) { return n ? n->R : 0; }
int warmnet_device(const h3d_warmnet *n) { return n ? n->device : -1; }
// forward pass of one density on stream s; *y points at the network's output buffer
int warmnet_forward_on(h3d_warmnet *n, const float *x, cudaStream_t s, const float **y) {
    if (int e = forward(n, x, 1, s)) return e;
    *y = n->y;
    return H3D_OK;
}
void launch_warmnet_density_pool(const float *rho, int N, int R, float *out, cudaStream_t s) {
    k_wn_density_pool<<<nblk((long long)R * R * R, 128), 128, 0, s>>>(rho, N, R, out);
}
void launch_warmnet_to_chi(const Planes &P, const float *y, int R, double *chi, cudaStream_t s) {
    k_wn_to_chi<<<nblk(P.nv, 256), 256, 0, s>>>(P, y, R, chi);
}
}  // namespace h3d

extern "C" {

int h3d_warmnet_create(int reso, int max_batch, uint64_t seed, int device, h3d_warmnet **out) {
    if (!out) return H3D_ERR_ARG;
    *out = nullptr;
    if (reso < 8 || reso > 128 || reso % 8 != 0 || max_batch < 1 || max_batch > 64) return H3D_ERR_ARG;
    h3d_warmnet *n = new (std::nothrow) h3d_warmnet;
    if (!n) return H3D_ERR_NOMEM;
    n->R = reso;
    n->maxB = max_batch;
    n->device = device;
    auto bail = [&](int code) { h3d_warmnet_destroy(n); return code; };
    if (cudaSetDevice(device) != cudaSuccess) return bail(H3D_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(H3D_ERR_CUDA);
    long long off = 0;
    for (int l = 0; l < WN_NCONV; l++) {
        n->woff[l] = off;
        off += (long long)WN_LAYER[l][0] * WN_LAYER[l][1] * 27;
        n->boff[l] = off;
        off += WN_LAYER[l][1];
    }
    n->woff[WN_NCONV] = off;
    off += WN_OUT * WN_OUT_IN;
    n->boff[WN_NCONV] = off;
    off += WN_OUT;
    n->nparam = off;
    if (cudaMalloc(&n->w, sizeof(float) * 4 * off) != cudaSuccess) return bail(H3D_ERR_NOMEM);
    n->g = n->w + off;
    n->m = n->g + off;
    n->v = n->m + off;
    // per sample: a0 p1 a1 p2 a2 p3 a3 u2 d2 u1 d1 u0 d0 y, and the same again for gradients
    const long long B = max_batch, V0 = n->vol(0), V1 = n->vol(1), V2 = n->vol(2), V3 = n->vol(3);
    const long long sizes[14] = {16 * V0, 16 * V1, 32 * V1, 32 * V2, 64 * V2, 64 * V3, 64 * V3,
                                 64 * V2, 32 * V2, 32 * V1, 16 * V1, 16 * V0, 16 * V0, 18 * V0};
    long long tot = 0;
    for (long long sz : sizes) tot += sz;
    if (cudaMalloc(&n->act, sizeof(float) * 2 * B * tot) != cudaSuccess) return bail(H3D_ERR_NOMEM);
    float **fw[14] = {&n->a0, &n->p1, &n->a1, &n->p2, &n->a2, &n->p3, &n->a3,
                      &n->u2, &n->d2, &n->u1, &n->d1, &n->u0, &n->d0, &n->y};
    float **bw[14] = {&n->ga0, &n->gp1, &n->ga1, &n->gp2, &n->ga2, &n->gp3, &n->ga3,
                      &n->gu2, &n->gd2, &n->gu1, &n->gd1, &n->gu0, &n->gd0, &n->gy};
    float *p = n->act;
    for (int i = 0; i < 14; i++) { *fw[i] = p; p += B * sizes[i]; }
    for (int i = 0; i < 14; i++) { *bw[i] = p; p += B * sizes[i]; }
    if (cudaMalloc(&n->partial, sizeof(double) * 256) != cudaSuccess) return bail(H3D_ERR_NOMEM);
    if (cudaMalloc(&n->d_loss, sizeof(double)) != cudaSuccess) return bail(H3D_ERR_NOMEM);
    if (cudaMallocHost(&n->h_loss, sizeof(double)) != cudaSuccess) return bail(H3D_ERR_NOMEM);
    // He-normal weights (Box-Muller on SplitMix64 uniforms), zero biases; the
    // output layer starts small so that the first predictions are near zero
    std::vector<float> hw(off, 0.f);
    uint64_t st = seed;
    auto normal = [&]() {
        const double u1 = ((splitmix(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
        const double u2 = ((splitmix(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    };
    for (int l = 0; l <= WN_NCONV; l++) {
        const int fan_in = l < WN_NCONV ? WN_LAYER[l][0] * 27 : WN_OUT_IN;
        const double sd = l < WN_NCONV ? std::sqrt(2.0 / fan_in) : 0.1 / std::sqrt((double)fan_in);
        for (long long i = n->woff[l]; i < n->boff[l]; i++) hw[i] = (float)(sd * normal());
    }
    if (cudaMemcpy(n->w, hw.data(), sizeof(float) * off, cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(H3D_ERR_CUDA);
    if (cudaMemset(n->g, 0, sizeof(float) * 3 * off) != cudaSuccess) return bail(H3D_ERR_CUDA);
    *out = n;
    return H3D_OK;
}

int h3d_warmnet_destroy(h3d_warmnet *n) {
    if (!n) return H3D_OK;
    cudaSetDevice(n->device);
    if (n->stream) cudaStreamSynchronize(n->stream);
    cudaFree(n->w);
    cudaFree(n->act);
    cudaFree(n->partial);
    cudaFree(n->d_loss);
    cudaFreeHost(n->h_loss);
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
    return H3D_OK;
}

const char *h3d_warmnet_last_error(const h3d_warmnet *n) { return n ? n->err.c_str() : "null network"; }

int h3d_warmnet_num_params(const h3d_warmnet *n, int64_t *count) {
    if (!n || !count) return H3D_ERR_ARG;
    *count = n->nparam;
    return H3D_OK;
}

int h3d_warmnet_get_params(h3d_warmnet *n, float *host) {
    if (!n || !host) return H3D_ERR_ARG;
    WCK(cudaSetDevice(n->device));
    WCK(cudaMemcpyAsync(host, n->w, sizeof(float) * n->nparam, cudaMemcpyDeviceToHost, n->stream));
    WCK(cudaStreamSynchronize(n->stream));
    return H3D_OK;
}

// new weights; the Adam moments and step count restart
int h3d_warmnet_set_params(h3d_warmnet *n, const float *host) {
    if (!n || !host) return H3D_ERR_ARG;
    WCK(cudaSetDevice(n->device));
    WCK(cudaMemcpyAsync(n->w, host, sizeof(float) * n->nparam, cudaMemcpyHostToDevice, n->stream));
    WCK(cudaMemsetAsync(n->g, 0, sizeof(float) * 3 * n->nparam, n->stream));
    WCK(cudaStreamSynchronize(n->stream));
    n->step = 0;
    return H3D_OK;
}

int h3d_warmnet_get_grads(h3d_warmnet *n, float *host) {
    if (!n || !host) return H3D_ERR_ARG;
    WCK(cudaSetDevice(n->device));
    WCK(cudaMemcpyAsync(host, n->g, sizeof(float) * n->nparam, cudaMemcpyDeviceToHost, n->stream));
    WCK(cudaStreamSynchronize(n->stream));
    return H3D_OK;
}

int h3d_warmnet_forward(h3d_warmnet *n, const float *x_dev, int batch, float *y_dev) {
    if (!n || !x_dev || !y_dev) return H3D_ERR_ARG;
    if (int e = check_batch(n, batch)) return e;
    WCK(cudaSetDevice(n->device));
    if (int e = forward(n, x_dev, batch, n->stream)) return e;
    WCK(cudaMemcpyAsync(y_dev, n->y, sizeof(float) * batch * WN_OUT * n->vol(0), cudaMemcpyDeviceToDevice,
                        n->stream));
    WCK(cudaStreamSynchronize(n->stream));
    return H3D_OK;
}

int h3d_warmnet_gradients(h3d_warmnet *n, const float *x_dev, const float *t_dev, int batch, double *loss) {
    if (!n || !x_dev || !t_dev) return H3D_ERR_ARG;
    if (int e = check_batch(n, batch)) return e;
    WCK(cudaSetDevice(n->device));
    WCK(cudaMemsetAsync(n->g, 0, sizeof(float) * n->nparam, n->stream));
    if (int e = forward(n, x_dev, batch, n->stream)) return e;
    if (int e = backward(n, x_dev, t_dev, batch, n->stream)) return e;
    WCK(cudaMemcpyAsync(n->h_loss, n->d_loss, sizeof(double), cudaMemcpyDeviceToHost, n->stream));
    WCK(cudaStreamSynchronize(n->stream));
    if (loss) *loss = *n->h_loss;
    return H3D_OK;
}

int h3d_warmnet_train_step(h3d_warmnet *n, const float *x_dev, const float *t_dev, int batch, float lr,
                           double *loss) {
    if (int e = h3d_warmnet_gradients(n, x_dev, t_dev, batch, loss)) return e;
    n->step++;
    const float c1 = (float)(1.0 - std::pow(0.9, (double)n->step));
    const float c2 = (float)(1.0 - std::pow(0.999, (double)n->step));
    k_wn_adam<<<nblk(n->nparam, 256), 256, 0, n->stream>>>(n->w, n->g, n->m, n->v, n->nparam, lr, 0.9f, 0.999f, c1,
                                                           c2, 1e-8f);
    WCK(cudaGetLastError());
    WCK(cudaStreamSynchronize(n->stream));
    return H3D_OK;
}

}  // extern "C"
