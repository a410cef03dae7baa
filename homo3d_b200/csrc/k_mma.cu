// k_mma.cu -- the MMA design update (method of moving asymptotes) on the device,
// with its C ABI (h3d_mma_*).
//
// Reference behaviour restated (homo3d optimization/):
//   MMAOptimizer (mmaOptimizer.h:12-36, mmaOptimizer.cu:18-80): FP64 state
//     (xvar, xmin, xmax, xold1, xold2, low, upp), float design / gradients cast
//     in and the new design cast back out each update, a = 0, c = 1000, d = 1;
//   mmasub_ker (mmaOpt.cu:820-1019): asymptotes, move limits, p0/q0, P/Q, b;
//   subsolv_g (mmaOpt.cu:429-815): primal-dual Newton iteration on the MMA
//     subproblem with epsi = 1 .. 1e-7, the (m+1) x (m+1) reduced system, step
//     bound 1/max(1, 1.01 max ratio) and the halving line search;
//   mmasub_g (mmaOpt.cu:1021-1062): xold2 <- xold1 <- xvar <- new x.
//
// Design: every O(n) quantity of one Newton step is produced by ONE fused
// grid-stride kernel that also reduces what the host needs (residual sums and
// maxima, gvec, the m x m matrix GG diag(1/diagx) GG^T, step bounds) into
// fixed-order per-block partials; a one-block finisher sums them and a single
// small copy brings them to pinned host memory.  The O(m) logic, the (m+1)
// solve and the line-search control stay on the host, as in the reference.
// The reference instead runs ~40 expression-template kernels, cub reductions
// and host copies per Newton step.  m is at most 4 (the reference's callers use
// 1 and 2); the design vector may be up to 2^31 elements per kernel index.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/h3d.h"
#include "h3d_internal.cuh"

namespace h3d {

constexpr int MMA_MAXM = 4;
constexpr int MMA_BS = 256;
constexpr int MMA_NB = 1184;  // 8 blocks on each of 148 SMs
constexpr int MMA_MAXPART = 2 * MMA_MAXM + MMA_MAXM * (MMA_MAXM + 1) / 2 + 2;

constexpr double MMA_EPSIMIN = 1e-7, MMA_RAA0 = 1e-5, MMA_ALBEFA = 0.1;
constexpr double MMA_ASYINIT = 0.5, MMA_ASYINCR = 1.2, MMA_ASYDECR = 0.7;

struct MmaVecs {
    long long n;
    double *xvar, *xmin, *xmax, *xold1, *xold2, *low, *upp;
    double *alfa, *beta, *p0, *q0, *P, *Q;  // P, Q: [m][n]
    double *x, *xsi, *eta;                  // subproblem point
    double *xn, *xsin, *etan;               // line-search trial point
    double *dx, *dxsi, *deta;               // Newton direction
};

struct MmaIn {
    const float *x, *dfdx;
    const float *dgdx[MMA_MAXM];
};

struct MmaDual {
    double lam[MMA_MAXM], dlam[MMA_MAXM];
    double epsi, steg;
};

// reduce NS sums and NM maxima per block into partial[blk*(NS+NM) + ...] (fixed order)
template <int NS, int NM>
__device__ __forceinline__ void mma_block_reduce(const double *s, const double *mx, double *partial) {
    constexpr int N = NS + NM;
    __shared__ double sm[N > 0 ? N : 1][MMA_BS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < N; ++c) {
        double v = c < NS ? s[c] : mx[c - NS];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double w = __shfl_down_sync(0xffffffffu, v, o);
            v = c < NS ? v + w : fmax(v, w);
        }
        if (lane == 0) sm[c][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < N) {
        const int c = threadIdx.x;
        double v = sm[c][0];
        for (int w = 1; w < MMA_BS / 32; ++w) v = c < NS ? v + sm[c][w] : fmax(v, sm[c][w]);
        partial[(long long)blockIdx.x * N + c] = v;
    }
}

// sums (first ns) and maxima (next nm) over the blocks' partials
__global__ void k_mma_finish(const double *__restrict__ partial, int nblk, int ns, int nm, double *out) {
    const int c = threadIdx.x, N = ns + nm;
    if (c >= N) return;
    double v = partial[c];
    for (int b = 1; b < nblk; ++b) {
        const double w = partial[(long long)b * N + c];
        v = c < ns ? v + w : fmax(v, w);
    }
    out[c] = v;
}

// asymptotes, move limits and the subproblem data (mmaOpt.cu:848-990), then the
// starting point of the subproblem (mmaOpt.cu:437-455); partial sums of b
template <int M>
__global__ void __launch_bounds__(MMA_BS) k_mma_prep(MmaVecs V, MmaIn in, int itn, double move, double *partial) {
    double bs[M];
#pragma unroll
    for (int i = 0; i < M; ++i) bs[i] = 0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < V.n; j += (long long)gridDim.x * blockDim.x) {
        const double xv = (double)in.x[j];
        const double xmn = V.xmin[j], xmx = V.xmax[j], dxr = xmx - xmn;
        double l, u;
        if (itn <= 2) {
            l = xv - MMA_ASYINIT * dxr;
            u = xv + MMA_ASYINIT * dxr;
        } else {
            const double x1 = V.xold1[j], x2 = V.xold2[j];
            const double zzz = (xv - x1) * (x1 - x2);
            const double f = zzz > 0 ? MMA_ASYINCR : (zzz < 0 ? MMA_ASYDECR : 1.0);
            l = xv - f * (x1 - V.low[j]);
            u = xv + f * (V.upp[j] - x1);
            l = fmin(fmax(l, xv - 10 * dxr), xv - 0.01 * dxr);
            u = fmax(fmin(u, xv + 10 * dxr), xv + 0.01 * dxr);
        }
        V.xvar[j] = xv;
        V.low[j] = l;
        V.upp[j] = u;
        const double al = fmax(fmax(l + MMA_ALBEFA * (xv - l), xv - move * dxr), xmn);
        const double be = fmin(fmin(u - MMA_ALBEFA * (u - xv), xv + move * dxr), xmx);
        V.alfa[j] = al;
        V.beta[j] = be;
        const double xmamiinv = 1.0 / fmax(dxr, 1e-5);
        const double ux1 = u - xv, xl1 = xv - l, ux2 = ux1 * ux1, xl2 = xl1 * xl1;
        const double df = (double)in.dfdx[j];
        const double fp = fmax(df, 0.0), fm = fmax(-df, 0.0);
        const double pq0 = 1e-3 * (fp + fm) + MMA_RAA0 * xmamiinv;
        V.p0[j] = (fp + pq0) * ux2;
        V.q0[j] = (fm + pq0) * xl2;
#pragma unroll
        for (int i = 0; i < M; ++i) {
            const double g = (double)in.dgdx[i][j];
            const double p = fmax(g, 0.0), q = fmax(-g, 0.0);
            const double pq = 1e-3 * (p + q) + MMA_RAA0 * xmamiinv;
            const double Pij = (p + pq) * ux2, Qij = (q + pq) * xl2;
            V.P[i * V.n + j] = Pij;
            V.Q[i * V.n + j] = Qij;
            bs[i] += Pij / ux1 + Qij / xl1;
        }
        const double x0 = 0.5 * (al + be);
        V.x[j] = x0;
        V.xsi[j] = fmax(1.0 / (x0 - al), 1.0);
        V.eta[j] = fmax(1.0 / (be - x0), 1.0);
    }
    mma_block_reduce<M, 0>(bs, nullptr, partial);
}

// point of the subproblem: the current one, or (trial) old + steg * direction,
// which is then stored in the trial buffers
struct MmaPoint {
    double x, xsi, eta;
};

__device__ __forceinline__ MmaPoint mma_point(const MmaVecs &V, long long j, bool trial, double steg) {
    MmaPoint p{V.x[j], V.xsi[j], V.eta[j]};
    if (trial) {
        p.x += steg * V.dx[j];
        p.xsi += steg * V.dxsi[j];
        p.eta += steg * V.deta[j];
        V.xn[j] = p.x;
        V.xsin[j] = p.xsi;
        V.etan[j] = p.eta;
    }
    return p;
}

// the O(n) part of the KKT residual (mmaOpt.cu:557-575, 752-766): sum of squares
// and max |.| of rex, rexsi, reeta, and gvec_i = sum_j P_ij/(upp-x) + Q_ij/(x-low)
template <int M>
__global__ void __launch_bounds__(MMA_BS) k_mma_resid(MmaVecs V, MmaDual D, int trial, double *partial) {
    double s[1 + M], mx[1] = {0.0};
#pragma unroll
    for (int i = 0; i < 1 + M; ++i) s[i] = 0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < V.n; j += (long long)gridDim.x * blockDim.x) {
        const MmaPoint p = mma_point(V, j, trial != 0, D.steg);
        const double ux1 = V.upp[j] - p.x, xl1 = p.x - V.low[j];
        const double uxinv = 1.0 / ux1, xlinv = 1.0 / xl1;
        double plam = V.p0[j], qlam = V.q0[j];
#pragma unroll
        for (int i = 0; i < M; ++i) {
            const double Pij = V.P[i * V.n + j], Qij = V.Q[i * V.n + j];
            plam += Pij * D.lam[i];
            qlam += Qij * D.lam[i];
            s[1 + i] += Pij * uxinv + Qij * xlinv;
        }
        const double dpsidx = plam * uxinv * uxinv - qlam * xlinv * xlinv;
        const double rex = dpsidx - p.xsi + p.eta;
        const double rexsi = p.xsi * (p.x - V.alfa[j]) - D.epsi;
        const double reeta = p.eta * (V.beta[j] - p.x) - D.epsi;
        s[0] += rex * rex + rexsi * rexsi + reeta * reeta;
        mx[0] = fmax(mx[0], fmax(fabs(rex), fmax(fabs(rexsi), fabs(reeta))));
    }
    mma_block_reduce<1 + M, 1>(s, mx, partial);
}

// the O(n) part of one Newton step (mmaOpt.cu:585-660): gvec, GG (delx/diagx) and
// GG diag(1/diagx) GG^T (upper triangle, row by row)
template <int M>
__global__ void __launch_bounds__(MMA_BS) k_mma_newton(MmaVecs V, MmaDual D, double *partial) {
    constexpr int NT = M * (M + 1) / 2;
    double s[2 * M + NT];
#pragma unroll
    for (int i = 0; i < 2 * M + NT; ++i) s[i] = 0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < V.n; j += (long long)gridDim.x * blockDim.x) {
        const double x = V.x[j], xsi = V.xsi[j], eta = V.eta[j];
        const double xa = x - V.alfa[j], bx = V.beta[j] - x;
        const double ux1 = V.upp[j] - x, xl1 = x - V.low[j];
        const double uxinv1 = 1.0 / ux1, xlinv1 = 1.0 / xl1;
        const double uxinv2 = uxinv1 * uxinv1, xlinv2 = xlinv1 * xlinv1;
        double plam = V.p0[j], qlam = V.q0[j], gg[M];
#pragma unroll
        for (int i = 0; i < M; ++i) {
            const double Pij = V.P[i * V.n + j], Qij = V.Q[i * V.n + j];
            plam += Pij * D.lam[i];
            qlam += Qij * D.lam[i];
            s[i] += Pij * uxinv1 + Qij * xlinv1;
            gg[i] = Pij * uxinv2 - Qij * xlinv2;
        }
        const double dpsidx = plam * uxinv2 - qlam * xlinv2;
        const double delx = dpsidx - D.epsi / xa + D.epsi / bx;
        const double diagx = 2 * (plam * uxinv2 * uxinv1 + qlam * xlinv2 * xlinv1) + xsi / xa + eta / bx;
        const double dxinv = 1.0 / diagx, ddx = delx * dxinv;
        int t = 0;
#pragma unroll
        for (int i = 0; i < M; ++i) {
            s[M + i] += gg[i] * ddx;
#pragma unroll
            for (int q = i; q < M; ++q) s[2 * M + t++] += gg[i] * gg[q] * dxinv;
        }
    }
    mma_block_reduce<2 * M + NT, 0>(s, nullptr, partial);
}

// Newton direction of the O(n) unknowns (mmaOpt.cu:661-690) and the largest step
// ratio among them (mmaOpt.cu:706-716)
template <int M>
__global__ void __launch_bounds__(MMA_BS) k_mma_direction(MmaVecs V, MmaDual D, double *partial) {
    double mx[1] = {1.0};
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < V.n; j += (long long)gridDim.x * blockDim.x) {
        const double x = V.x[j], xsi = V.xsi[j], eta = V.eta[j];
        const double xa = x - V.alfa[j], bx = V.beta[j] - x;
        const double ux1 = V.upp[j] - x, xl1 = x - V.low[j];
        const double uxinv1 = 1.0 / ux1, xlinv1 = 1.0 / xl1;
        const double uxinv2 = uxinv1 * uxinv1, xlinv2 = xlinv1 * xlinv1;
        double plam = V.p0[j], qlam = V.q0[j], g = 0;
#pragma unroll
        for (int i = 0; i < M; ++i) {
            const double Pij = V.P[i * V.n + j], Qij = V.Q[i * V.n + j];
            plam += Pij * D.lam[i];
            qlam += Qij * D.lam[i];
            g += (Pij * uxinv2 - Qij * xlinv2) * D.dlam[i];
        }
        const double dpsidx = plam * uxinv2 - qlam * xlinv2;
        const double delx = dpsidx - D.epsi / xa + D.epsi / bx;
        const double diagx = 2 * (plam * uxinv2 * uxinv1 + qlam * xlinv2 * xlinv1) + xsi / xa + eta / bx;
        const double dx = -delx / diagx - g / diagx;
        const double dxsi = -xsi + D.epsi / xa - (xsi * dx) / xa;
        const double deta = -eta + D.epsi / bx + (eta * dx) / bx;
        V.dx[j] = dx;
        V.dxsi[j] = dxsi;
        V.deta[j] = deta;
        mx[0] = fmax(mx[0], fmax(fmax(-1.01 * dxsi / xsi, -1.01 * deta / eta),
                                 fmax(-1.01 * dx / xa, 1.01 * dx / bx)));
    }
    mma_block_reduce<0, 1>(nullptr, mx, partial);
}

// xold2 <- xold1 <- xvar, and the new design back to the caller's float array
// (mmaOpt.cu:1058-1060, mmaOptimizer.cu:78)
__global__ void k_mma_commit(MmaVecs V, float *x_out) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < V.n; j += (long long)gridDim.x * blockDim.x) {
        V.xold2[j] = V.xold1[j];
        V.xold1[j] = V.xvar[j];
        x_out[j] = (float)V.x[j];
    }
}

__global__ void k_mma_bounds(long long n, const float *xmin, const float *xmax, float smin, float smax,
                             double *dmin, double *dmax) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        dmin[j] = xmin ? (double)xmin[j] : (double)smin;
        dmax[j] = xmax ? (double)xmax[j] : (double)smax;
    }
}

}  // namespace h3d

// ---- host side: the optimiser object and the C ABI ----------------------------
using namespace h3d;

struct h3d_mma {
    int m = 0;
    long long n = 0;
    double a0 = 1, a = 0, c = 1000, d = 1;
    int device = 0;
    cudaStream_t stream = nullptr;
    MmaVecs V{};
    double *store = nullptr;         // all O(n) vectors in one allocation
    double *partial = nullptr, *d_small = nullptr, *h_small = nullptr;
    bool bounded = false;
    std::string err;
};

namespace {

int mma_fail(h3d_mma *o, int code, const std::string &msg) {
    if (o) o->err = msg;
    return code;
}

#define MCK(call)                                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return mma_fail(o, H3D_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// run the finisher over the last kernel's partials and copy the result to the host
int mma_collect(h3d_mma *o, int ns, int nm) {
    k_mma_finish<<<1, 64, 0, o->stream>>>(o->partial, MMA_NB, ns, nm, o->d_small);
    MCK(cudaGetLastError());
    MCK(cudaMemcpyAsync(o->h_small, o->d_small, sizeof(double) * (ns + nm), cudaMemcpyDeviceToHost, o->stream));
    MCK(cudaStreamSynchronize(o->stream));
    return H3D_OK;
}

// the O(m) state of the subproblem (host)
struct Small {
    double y[MMA_MAXM], lam[MMA_MAXM], mu[MMA_MAXM], s[MMA_MAXM];
    double z, zet;
};

// the full residual norm / max from the device sums and the O(m) terms
// (mmaOpt.cu:557-588)
void small_residual(int m, const double *gvec, double ss, double mxn, const Small &v, double a0, double a,
                    double c, double d, const double *b, double epsi, double &norm, double &mx) {
    double alam = 0;
    for (int i = 0; i < m; i++) alam += a * v.lam[i];
    const double rez = a0 - v.zet - alam, rezet = v.zet * v.z - epsi;
    ss += rez * rez + rezet * rezet;
    mx = std::max(mxn, std::max(std::fabs(rez), std::fabs(rezet)));
    for (int i = 0; i < m; i++) {
        const double rey = c + d * v.y[i] - v.mu[i] - v.lam[i];
        const double relam = gvec[i] - a * v.z - v.y[i] + v.s[i] - b[i];
        const double remu = v.mu[i] * v.y[i] - epsi;
        const double res = v.lam[i] * v.s[i] - epsi;
        ss += rey * rey + relam * relam + remu * remu + res * res;
        mx = std::max(mx, std::max(std::max(std::fabs(rey), std::fabs(relam)), std::max(std::fabs(remu), std::fabs(res))));
    }
    norm = std::sqrt(ss);
}

// dense (m+1) solve with partial pivoting
bool dense_solve(int k, double *A, double *b, double *x) {
    for (int c = 0; c < k; c++) {
        int p = c;
        for (int r = c + 1; r < k; r++)
            if (std::fabs(A[r * k + c]) > std::fabs(A[p * k + c])) p = r;
        if (A[p * k + c] == 0.0) return false;
        if (p != c) {
            for (int j = 0; j < k; j++) std::swap(A[c * k + j], A[p * k + j]);
            std::swap(b[c], b[p]);
        }
        for (int r = c + 1; r < k; r++) {
            const double f = A[r * k + c] / A[c * k + c];
            for (int j = c; j < k; j++) A[r * k + j] -= f * A[c * k + j];
            b[r] -= f * b[c];
        }
    }
    for (int r = k - 1; r >= 0; r--) {
        double s = b[r];
        for (int j = r + 1; j < k; j++) s -= A[r * k + j] * x[j];
        x[r] = s / A[r * k + r];
    }
    return true;
}

template <int M>
int mma_update_m(h3d_mma *o, int itn, float *x_dev, const float *dfdx_dev, const float *gval_dev,
                 const float *const *dgdx_dev, int *newton_out) {
    cudaStream_t st = o->stream;
    const int m = M;
    MmaVecs &V = o->V;
    MmaIn in{};
    in.x = x_dev;
    in.dfdx = dfdx_dev;
    for (int i = 0; i < M; i++) in.dgdx[i] = dgdx_dev[i];
    float gval_f[MMA_MAXM];
    MCK(cudaMemcpyAsync(gval_f, gval_dev, sizeof(float) * M, cudaMemcpyDeviceToHost, st));
    k_mma_prep<M><<<MMA_NB, MMA_BS, 0, st>>>(V, in, itn, 1.0, o->partial);
    MCK(cudaGetLastError());
    if (int e = mma_collect(o, M, 0)) return e;
    double b[MMA_MAXM];
    for (int i = 0; i < m; i++) b[i] = o->h_small[i] - (double)gval_f[i];

    Small v{};
    for (int i = 0; i < m; i++) { v.y[i] = 1; v.lam[i] = 1; v.mu[i] = std::max(1.0, 0.5 * o->c); v.s[i] = 1; }
    v.z = 1;
    v.zet = 1;
    MmaDual D{};
    double epsi = 1.0;
    int newton = 0;
    auto residual = [&](int trial, double steg, const Small &pt, double &norm, double &mx) -> int {
        for (int i = 0; i < m; i++) D.lam[i] = pt.lam[i];
        D.epsi = epsi;
        D.steg = steg;
        k_mma_resid<M><<<MMA_NB, MMA_BS, 0, st>>>(V, D, trial, o->partial);
        MCK(cudaGetLastError());
        if (int e = mma_collect(o, 1 + M, 1)) return e;
        small_residual(m, o->h_small + 1, o->h_small[0], o->h_small[1 + M], pt, o->a0, o->a, o->c, o->d, b, epsi,
                       norm, mx);
        return H3D_OK;
    };
    while (epsi > MMA_EPSIMIN) {
        double residunorm, residumax;
        if (int e = residual(0, 0.0, v, residunorm, residumax)) return e;
        int ittt = 0;
        while (residumax > 0.9 * epsi && ittt < 200) {
            ittt++;
            newton++;
            for (int i = 0; i < m; i++) D.lam[i] = v.lam[i];
            D.epsi = epsi;
            k_mma_newton<M><<<MMA_NB, MMA_BS, 0, st>>>(V, D, o->partial);
            MCK(cudaGetLastError());
            constexpr int NT = M * (M + 1) / 2;
            if (int e = mma_collect(o, 2 * M + NT, 0)) return e;
            const double *gvec = o->h_small, *ggx = o->h_small + M, *gtg = o->h_small + 2 * M;
            double alam = 0;
            for (int i = 0; i < m; i++) alam += o->a * v.lam[i];
            const double delz = o->a0 - alam - epsi / v.z;
            double dely[MMA_MAXM], diagy[MMA_MAXM], AA[(MMA_MAXM + 1) * (MMA_MAXM + 1)], bb[MMA_MAXM + 1],
                sol[MMA_MAXM + 1];
            const int k = m + 1;
            for (int i = 0; i < m; i++) {
                dely[i] = o->c + o->d * v.y[i] - v.lam[i] - epsi / v.y[i];
                const double dellam = gvec[i] - o->a * v.z - v.y[i] - b[i] + epsi / v.lam[i];
                diagy[i] = o->d + v.mu[i] / v.y[i];
                bb[i] = dellam + dely[i] / diagy[i] - ggx[i];
            }
            int t = 0;
            for (int i = 0; i < m; i++)
                for (int q = i; q < m; q++, t++) AA[i * k + q] = AA[q * k + i] = gtg[t];
            for (int i = 0; i < m; i++) {
                AA[i * k + i] += v.s[i] / v.lam[i] + 1.0 / diagy[i];
                AA[i * k + m] = o->a;
                AA[m * k + i] = o->a;
            }
            AA[m * k + m] = -v.zet / v.z;
            bb[m] = delz;
            if (!dense_solve(k, AA, bb, sol)) return mma_fail(o, H3D_ERR_SINGULAR, "MMA subproblem system is singular");
            const double dz = sol[m];
            Small dv{};
            for (int i = 0; i < m; i++) D.dlam[i] = dv.lam[i] = sol[i];
            k_mma_direction<M><<<MMA_NB, MMA_BS, 0, st>>>(V, D, o->partial);
            MCK(cudaGetLastError());
            if (int e = mma_collect(o, 0, 1)) return e;
            double stm = o->h_small[0];
            for (int i = 0; i < m; i++) {
                dv.y[i] = -dely[i] / diagy[i] + dv.lam[i] / diagy[i];
                dv.mu[i] = -v.mu[i] + epsi / v.y[i] - (v.mu[i] * dv.y[i]) / v.y[i];
                dv.s[i] = -v.s[i] + epsi / v.lam[i] - (v.s[i] * dv.lam[i]) / v.lam[i];
                stm = std::max(stm, -1.01 * dv.y[i] / v.y[i]);
                stm = std::max(stm, -1.01 * dv.lam[i] / v.lam[i]);
                stm = std::max(stm, -1.01 * dv.mu[i] / v.mu[i]);
                stm = std::max(stm, -1.01 * dv.s[i] / v.s[i]);
            }
            const double dzet = -v.zet + epsi / v.z - v.zet * dz / v.z;
            stm = std::max(stm, -1.01 * dz / v.z);
            stm = std::max(stm, -1.01 * dzet / v.zet);
            double steg = 1.0 / stm;
            // halving line search from the current point into the trial buffers
            const Small old = v;
            int itto = 0;
            double resinew = 2 * residunorm, rmax = residumax;
            while (resinew > residunorm && itto < 50) {
                itto++;
                for (int i = 0; i < m; i++) {
                    v.y[i] = old.y[i] + steg * dv.y[i];
                    v.lam[i] = old.lam[i] + steg * dv.lam[i];
                    v.mu[i] = old.mu[i] + steg * dv.mu[i];
                    v.s[i] = old.s[i] + steg * dv.s[i];
                }
                v.z = old.z + steg * dz;
                v.zet = old.zet + steg * dzet;
                if (int e = residual(1, steg, v, resinew, rmax)) return e;
                steg /= 2;
            }
            std::swap(V.x, V.xn);
            std::swap(V.xsi, V.xsin);
            std::swap(V.eta, V.etan);
            residunorm = resinew;
            residumax = rmax;
        }
        epsi *= 0.1;
    }
    k_mma_commit<<<MMA_NB, MMA_BS, 0, st>>>(V, x_dev);
    MCK(cudaGetLastError());
    MCK(cudaStreamSynchronize(st));
    if (newton_out) *newton_out = newton;
    return H3D_OK;
}

}  // namespace

extern "C" {

int h3d_mma_create(int m, int64_t n, double a0, double a, double c, double d, int device, h3d_mma **out) {
    if (!out) return H3D_ERR_ARG;
    *out = nullptr;
    if (m < 1 || m > MMA_MAXM || n < 1 || n > ((int64_t)1 << 31)) return H3D_ERR_ARG;
    h3d_mma *o = new (std::nothrow) h3d_mma;
    if (!o) return H3D_ERR_NOMEM;
    o->m = m; o->n = n; o->a0 = a0; o->a = a; o->c = c; o->d = d; o->device = device;
    auto bail = [&](int code) { h3d_mma_destroy(o); return code; };
    if (cudaSetDevice(device) != cudaSuccess) return bail(H3D_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&o->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(H3D_ERR_CUDA);
    const size_t nvec = 22 + 2 * (size_t)m;
    if (cudaMalloc(&o->store, sizeof(double) * nvec * (size_t)n) != cudaSuccess) return bail(H3D_ERR_NOMEM);
    double *p = o->store;
    auto take = [&](size_t k) { double *r = p; p += k * (size_t)n; return r; };
    MmaVecs &V = o->V;
    V.n = n;
    V.xvar = take(1); V.xmin = take(1); V.xmax = take(1); V.xold1 = take(1); V.xold2 = take(1);
    V.low = take(1); V.upp = take(1); V.alfa = take(1); V.beta = take(1); V.p0 = take(1); V.q0 = take(1);
    V.P = take(m); V.Q = take(m);
    V.x = take(1); V.xsi = take(1); V.eta = take(1); V.xn = take(1); V.xsin = take(1); V.etan = take(1);
    V.dx = take(1); V.dxsi = take(1); V.deta = take(1);
    if (cudaMemset(o->store, 0, sizeof(double) * nvec * (size_t)n) != cudaSuccess) return bail(H3D_ERR_CUDA);
    if (cudaMalloc(&o->partial, sizeof(double) * MMA_NB * MMA_MAXPART) != cudaSuccess) return bail(H3D_ERR_NOMEM);
    if (cudaMalloc(&o->d_small, sizeof(double) * 64) != cudaSuccess) return bail(H3D_ERR_NOMEM);
    if (cudaMallocHost(&o->h_small, sizeof(double) * 64) != cudaSuccess) return bail(H3D_ERR_NOMEM);
    *out = o;
    return H3D_OK;
}

int h3d_mma_destroy(h3d_mma *o) {
    if (!o) return H3D_OK;
    cudaSetDevice(o->device);
    if (o->stream) cudaStreamSynchronize(o->stream);
    cudaFree(o->store);
    cudaFree(o->partial);
    cudaFree(o->d_small);
    cudaFreeHost(o->h_small);
    if (o->stream) cudaStreamDestroy(o->stream);
    delete o;
    return H3D_OK;
}

const char *h3d_mma_last_error(const h3d_mma *o) { return o ? o->err.c_str() : "null MMA handle"; }

int h3d_mma_set_bounds(h3d_mma *o, const float *xmin_dev, const float *xmax_dev) {
    if (!o || !xmin_dev || !xmax_dev) return mma_fail(o, H3D_ERR_ARG, "bounds must be device arrays");
    MCK(cudaSetDevice(o->device));
    k_mma_bounds<<<MMA_NB, MMA_BS, 0, o->stream>>>(o->n, xmin_dev, xmax_dev, 0.f, 0.f, o->V.xmin, o->V.xmax);
    MCK(cudaGetLastError());
    MCK(cudaStreamSynchronize(o->stream));
    o->bounded = true;
    return H3D_OK;
}

int h3d_mma_set_bounds_scalar(h3d_mma *o, float xmin, float xmax) {
    if (!o) return H3D_ERR_ARG;
    MCK(cudaSetDevice(o->device));
    k_mma_bounds<<<MMA_NB, MMA_BS, 0, o->stream>>>(o->n, nullptr, nullptr, xmin, xmax, o->V.xmin, o->V.xmax);
    MCK(cudaGetLastError());
    MCK(cudaStreamSynchronize(o->stream));
    o->bounded = true;
    return H3D_OK;
}

int h3d_mma_update(h3d_mma *o, int itn, float *x_dev, const float *dfdx_dev, const float *gval_dev,
                   const float *const *dgdx_dev, int *newton_steps) {
    if (!o) return H3D_ERR_ARG;
    if (!x_dev || !dfdx_dev || !gval_dev || !dgdx_dev) return mma_fail(o, H3D_ERR_ARG, "null argument");
    for (int i = 0; i < o->m; i++)
        if (!dgdx_dev[i]) return mma_fail(o, H3D_ERR_ARG, "null constraint gradient");
    if (!o->bounded) return mma_fail(o, H3D_ERR_STATE, "bounds not set");
    MCK(cudaSetDevice(o->device));
    switch (o->m) {
    case 1: return mma_update_m<1>(o, itn, x_dev, dfdx_dev, gval_dev, dgdx_dev, newton_steps);
    case 2: return mma_update_m<2>(o, itn, x_dev, dfdx_dev, gval_dev, dgdx_dev, newton_steps);
    case 3: return mma_update_m<3>(o, itn, x_dev, dfdx_dev, gval_dev, dgdx_dev, newton_steps);
    default: return mma_update_m<4>(o, itn, x_dev, dfdx_dev, gval_dev, dgdx_dev, newton_steps);
    }
}

}  // extern "C"
