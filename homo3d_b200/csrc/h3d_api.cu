// h3d_api.cu -- host runtime and C ABI of libh3d.
//
// One handle = one periodic unit cell: its multigrid hierarchy, per-level
// fields, coarse stencils, the coarsest-grid inverse, the stored solutions of
// the six unit-strain cases, a CUDA stream, and a captured CUDA graph of one
// V-cycle (all levels, then the level-0 residual norms and their copy to pinned
// host memory).  The solve loop replays that graph and reads six doubles per
// cycle; nothing else crosses to the host.
//
// Reference call surface mirrored (homo3d): Homogenization::{build, update,
// elasticMatrix, Sensitivity} (homogenization.h:17-61), MG::{build, v_cycle,
// solveEquation, updateStencils} (MG.h:14-45), Grid::{gs_relaxation,
// update_residual, restrict_residual, prolongate_correction, solveHostEquation,
// enforce_unit_macro_strain} (grid.h:104-418), OCOptimizer::{update, filterSens}
// (OCOptimizer.h:16-19), Tensor::symmetrize (TensorExpression.h:425-445).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/h3d.h"
#include "h3d_internal.cuh"

using namespace h3d;

namespace {

constexpr int MAXLV = 16;

// element matrix for material matrix D by 2x2x2 Gauss quadrature on the unit
// cube, symmetrised (templateMatrix.cpp:95-165)
void ke_quadrature(const double D[6][6], double ke[576]) {
    const double p = std::sqrt(1.0 / 3.0);
    std::memset(ke, 0, sizeof(double) * 576);
    for (int g = 0; g < 8; g++) {
        const double gp[3] = {((2 * (g % 2) - 1) * p + 1) / 2, ((2 * (g / 2 % 2) - 1) * p + 1) / 2,
                              ((2 * (g / 4) - 1) * p + 1) / 2};
        double dn[8][3];
        for (int k = 0; k < 8; k++) {
            const int id[3] = {k % 2, k / 2 % 2, k / 4};
            double r[3];
            for (int a = 0; a < 3; a++) r[a] = id[a] ? gp[a] : 1 - gp[a];
            for (int a = 0; a < 3; a++) dn[k][a] = (id[a] ? 1.0 : -1.0) * r[(a + 1) % 3] * r[(a + 2) % 3];
        }
        double B[6][24] = {};
        for (int k = 0; k < 8; k++) {
            for (int a = 0; a < 3; a++) B[a][3 * k + a] = dn[k][a];
            B[3][3 * k + 1] = dn[k][2]; B[3][3 * k + 2] = dn[k][1];
            B[4][3 * k + 0] = dn[k][2]; B[4][3 * k + 2] = dn[k][0];
            B[5][3 * k + 0] = dn[k][1]; B[5][3 * k + 1] = dn[k][0];
        }
        for (int i = 0; i < 24; i++)
            for (int j = 0; j < 24; j++) {
                double s = 0;
                for (int a = 0; a < 6; a++)
                    for (int b = 0; b < 6; b++) s += B[a][i] * D[a][b] * B[b][j];
                ke[i * 24 + j] += s;
            }
    }
    for (int i = 0; i < 576; i++) ke[i] *= 0.125;
    for (int i = 0; i < 24; i++)
        for (int j = 0; j < i; j++) {
            const double s = 0.5 * (ke[i * 24 + j] + ke[j * 24 + i]);
            ke[i * 24 + j] = ke[j * 24 + i] = s;
        }
}

void element_matrix(double E, double nu, double ke[576]) {
    double D[6][6] = {};
    const double s = E / ((1 + nu) * (1 - 2 * nu));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) D[i][j] = s * (i == j ? 1 - nu : nu);
    for (int i = 3; i < 6; i++) D[i][i] = s * (1 - 2 * nu) / 2;
    ke_quadrature(D, ke);
}

double macro_disp_h(int a, int c, int m) {
    const int p[3] = {a & 1, (a >> 1) & 1, a >> 2};
    switch (c) {
    case 0: return m == 0 ? p[0] : 0;
    case 1: return m == 1 ? p[1] : 0;
    case 2: return m == 2 ? p[2] : 0;
    case 3: return m == 1 ? p[2] / 2.0 : m == 2 ? p[1] / 2.0 : 0;
    case 4: return m == 0 ? p[2] / 2.0 : m == 2 ? p[0] / 2.0 : 0;
    default: return m == 0 ? p[1] / 2.0 : m == 1 ? p[0] / 2.0 : 0;
    }
}

// resolution correction and coarsening ratios (grid.cpp:21-151)
int build_hierarchy(const int reso[3], int dims[MAXLV][3], int ratios[MAXLV][3]) {
    int avail[3], n[3];
    for (int a = 0; a < 3; a++) {
        if (reso[a] < 2 || reso[a] > 1024) return -1;
        const double l2 = std::log2((double)reso[a]);
        const double lcl = std::fmax(std::floor(l2) - 2, 0.);
        avail[a] = (int)std::ceil(std::pow(2, l2 - lcl));
        n[a] = (int)(avail[a] * std::pow(2, lcl));
    }
    for (int a = 0; a < 3; a++) { dims[0][a] = n[a]; ratios[0][a] = 0; }
    int nl = 1;
    while (nl < MAXLV) {
        int r[3], any = 0, all = 1;
        for (int a = 0; a < 3; a++) {
            const int c = dims[nl - 1][a];
            if (c <= avail[a]) { r[a] = 0; all = 0; }
            else if (c >= 256) { r[a] = 2; while (c / r[a] >= 256) r[a] *= 2; any = 1; }
            else { r[a] = 2; any = 1; }
        }
        if (!any) break;
        if (!all) return -2;
        for (int a = 0; a < 3; a++) { ratios[nl][a] = r[a]; dims[nl][a] = dims[nl - 1][a] / r[a]; }
        nl++;
    }
    return nl;
}

Planes make_planes(const int n[3]) {
    Planes P;
    for (int a = 0; a < 3; a++) P.n[a] = n[a];
    long long b = 0;
    for (int k = 0; k < 8; k++) {
        for (int a = 0; a < 3; a++) {
            const int par = ((k >> a) & 1) ^ 1;  // coordinate parity of colour k on axis a
            P.pn[k][a] = (n[a] - par + 1) / 2;
        }
        P.base[k] = b;
        b += (long long)P.pn[k][0] * P.pn[k][1] * P.pn[k][2];
    }
    P.nv = b;
    P.even = (n[0] % 2 == 0 && n[1] % 2 == 0 && n[2] % 2 == 0);
    return P;
}

}  // namespace

struct h3d_handle {
    h3d_config cfg;
    int device = 0;
    int nl = 0;
    Level lv[MAXLV];
    double ked[576];
    KeMat ke;
    KeMat64 ke64;
    RhsTab rhs;
    std::vector<float> qhost;
    int nsub = 0;
    float *rho = nullptr;       // physical density on level 0
    double *chi = nullptr;      // stored solutions [18][nv0], FP64
    double *u64 = nullptr;      // level-0 solution in the refined mode [18][nv0]
    float *f0 = nullptr;        // level-0 right-hand side of the refined mode [18][nv0]
    float *q = nullptr;         // level-1 Galerkin sub-element matrices
    double *d_ked = nullptr;
    double *aug = nullptr;      // coarsest [K | K^-1]
    int ndof = 0;
    int *d_flag = nullptr;
    double *partial = nullptr;  // reduction scratch
    size_t partial_n = 0;
    double *d_small = nullptr;  // 64 doubles: norms, C entries
    double *h_small = nullptr;  // pinned mirror
    float *tmp = nullptr;       // conversion / filter scratch
    size_t tmp_n = 0;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t vgraph = nullptr;   // one V-cycle on the level-0 field u
    cudaGraphExec_t rgraph = nullptr;   // refinement step: u64 += u, f = f0 - K u64 (FP32 products)
    cudaGraphExec_t xgraph = nullptr;   // the same with the FP64-accumulated residual
    cudaGraphExec_t sgraph = nullptr;   // a solve's V-cycle: vgraph + rigid-translation deflation
    cudaGraphExec_t fgraph = nullptr;   // coarsest assembly + Gauss-Jordan inverse (n + 1 launches)
    cudaGraphExec_t dgraph = nullptr;   // design step (h3d_design_step)
    float *d_dcw = nullptr, *h_dcw = nullptr;  // sensitivity weights: device copy, pinned host source
    h3d_design_params dkey{};           // parameters and buffers the design graph was captured for
    const float *dkey_rho = nullptr, *dkey_sens = nullptr;
    double *pin_state = nullptr;        // deflation: F[18], pending shift T[18], plane sums[18]
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool refine() const { return cfg.precision != H3D_PREC_FP32; }
    // the level-0 V-cycle residual on the tensor cores (k_fine_tc.cu)
    bool mixed() const { return cfg.precision == H3D_PREC_MIXED_TC; }
    // the refinement residual accumulated in FP32 down to relthres 2e-6
    bool fp32_refine() const { return cfg.precision == H3D_PREC_MIXED || cfg.precision == H3D_PREC_MIXED_TC; }
    int num_sms = 0;
    int *d_tcflag = nullptr;            // set by the tensor-core residual if an mbarrier wait timed out
    // cooperative bottom of the V-cycle: levels of at most bottom_nv vertices (0: off,
    // the default: its grid barriers cost more than the graph's launch boundaries)
    long long bottom_nv = 0;
    unsigned *d_bar = nullptr;          // its grid-barrier state
    int *d_botflag = nullptr;           // set if one of its barrier waits ran out
    bool have_density = false, have_stencils = false;
    bool tuned = false;  // launch shapes chosen (autotuner or h3d_set_tuning)
    // chi_zero: the stored solutions chi are all zero (allocation, h3d_reset_solutions,
    // no write since); u64_zero: the FP64 solution was set to zero by the last
    // elastic_prepare and nothing has written it since (a solve's start reads it)
    bool chi_zero = true, u64_zero = false;
    std::string err;
};

namespace {

int fail(h3d_handle *h, int code, const std::string &msg) {
    if (h) h->err = msg;
    return code;
}

#define CK(call)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return fail(h, e_ == cudaErrorMemoryAllocation ? H3D_ERR_NOMEM : H3D_ERR_CUDA,          \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                        \
    } while (0)

#define CKL()                                                                                       \
    do {                                                                                            \
        cudaError_t e_ = cudaGetLastError();                                                        \
        if (e_ != cudaSuccess) return fail(h, H3D_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
    } while (0)

int ensure_tmp(h3d_handle *h, size_t nfloat) {
    if (h->tmp_n >= nfloat) return H3D_OK;
    if (h->tmp) cudaFree(h->tmp);
    h->tmp = nullptr;
    h->tmp_n = 0;
    CK(cudaMalloc(&h->tmp, nfloat * sizeof(float)));
    h->tmp_n = nfloat;
    return H3D_OK;
}

// Q_s = P_s^T Ke P_s for every fine sub-element s of a coarse element (ratio r)
void build_q(const double ke[576], const int r[3], std::vector<float> &q, int &nsub) {
    nsub = r[0] * r[1] * r[2];
    q.assign((size_t)nsub * 576, 0.f);
    for (int s = 0; s < nsub; s++) {
        const int so[3] = {s % r[0], s / r[0] % r[1], s / (r[0] * r[1])};
        double P[8][8];
        for (int a = 0; a < 8; a++)
            for (int b = 0; b < 8; b++) {
                const int fo[3] = {so[0] + (a & 1), so[1] + ((a >> 1) & 1), so[2] + (a >> 2)};
                const int co[3] = {(b & 1) * r[0], ((b >> 1) & 1) * r[1], (b >> 2) * r[2]};
                double w = 1;
                for (int t = 0; t < 3; t++) {
                    const int o = std::abs(fo[t] - co[t]);
                    w *= o >= r[t] ? 0.0 : (double)(r[t] - o) / r[t];
                }
                P[a][b] = w;
            }
        for (int A = 0; A < 8; A++)
            for (int B = 0; B < 8; B++)
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) {
                        double v = 0;
                        for (int a = 0; a < 8; a++) {
                            if (P[a][A] == 0) continue;
                            for (int b = 0; b < 8; b++) v += P[a][A] * P[b][B] * ke[(3 * a + i) * 24 + 3 * b + j];
                        }
                        q[(size_t)s * 576 + (3 * A + i) * 24 + 3 * B + j] = (float)v;
                    }
    }
}

int destroy_graph(h3d_handle *h) {
    if (h->vgraph) { cudaGraphExecDestroy(h->vgraph); h->vgraph = nullptr; }
    if (h->rgraph) { cudaGraphExecDestroy(h->rgraph); h->rgraph = nullptr; }
    if (h->xgraph) { cudaGraphExecDestroy(h->xgraph); h->xgraph = nullptr; }
    if (h->sgraph) { cudaGraphExecDestroy(h->sgraph); h->sgraph = nullptr; }
    if (h->fgraph) { cudaGraphExecDestroy(h->fgraph); h->fgraph = nullptr; }
    if (h->dgraph) { cudaGraphExecDestroy(h->dgraph); h->dgraph = nullptr; }
    return H3D_OK;
}

// the V-cycle of MG::v_cycle (MG.cpp:46-70) on the handle's stream; the level-0
// residual of the down leg also yields the per-case norms (the stale residual the
// stopping test of MG.cpp:130-139 reads).  The refined solve runs the same cycle on
// the FP32 correction u, with level-0 f holding f0 - K u64.  Inside a solve the
// cycle ends with the rigid-translation deflation (launch_pin_deflate).
// the first level of the cooperative bottom (k_vcycle_bottom), or -1: the
// largest level of at most bottom_nv vertices, with a smoothed level below it
int bottom_first(const h3d_handle *h, float w) {
    if (h->bottom_nv <= 0 || w != 1.f) return -1;
    int first = -1;
    for (int l = h->nl - 2; l >= 1; l--)
        if (h->lv[l].P.nv <= h->bottom_nv) first = l;
    if (first < 0 || !vcycle_bottom_fits(h->lv, first, h->nl)) return -1;
    return first;
}

int enqueue_vcycle(h3d_handle *h, float w, bool deflate = false) {
    cudaStream_t s = h->stream;
    const int nblk_r = h->mixed() ? fine_residual_tc_blocks(h->lv[0].P, h->num_sms) : fine_residual_blocks(h->lv[0]);
    int bfirst = bottom_first(h, w);
    int bblk = 0;
    if (bfirst >= 0) {
        bblk = vcycle_bottom_blocks(h->num_sms, h->ndof, h->lv[bfirst].st32);
        if (bblk <= 0) bfirst = -1;
    }
    for (int l = 0; l < h->nl; l++) {
        if (l == bfirst) {  // restriction into `bfirst`, down to the coarsest solve and back up
            if (launch_vcycle_bottom(h->lv, bfirst, h->nl, h->aug, h->cfg.coarse_mode == H3D_COARSE_PROJECT, h->d_bar,
                                     h->d_botflag, bblk, s) != 0)
                return fail(h, H3D_ERR_CUDA, "cooperative V-cycle bottom could not be launched");
            break;
        }
        if (l > 0) {
            launch_restrict(h->lv[l - 1], h->lv[l], s);
            cudaMemsetAsync(h->lv[l].u, 0, sizeof(float) * field_floats(h->lv[l].P.nv), s);
        }
        if (l == h->nl - 1) {
            launch_coarse_apply(h->lv[l], h->aug, h->cfg.coarse_mode == H3D_COARSE_PROJECT, s);
        } else if (l == 0 && h->mixed()) {  // the sweep, then the residual on the tensor cores
            launch_fine_gs(h->lv[0], h->rho, h->ke, w, s);
            launch_fine_residual_tc(h->lv[0], h->rho, h->ke, h->partial, nblk_r, h->d_tcflag, s);
        } else if (l == 0) {
            launch_fine_gs_residual(h->lv[0], h->rho, h->ke, w, h->partial, s);
        } else {
            launch_coarse_gs_residual(h->lv[l], w, s);  // each level's residual comes with its sweep
        }
    }
    for (int l = (bfirst >= 0 ? bfirst : h->nl - 1) - 1; l >= 0; l--) {
        launch_prolong(h->lv[l], h->lv[l + 1], l == 0, s);
        if (l == 0) launch_fine_gs(h->lv[0], h->rho, h->ke, w, s);
        else launch_coarse_gs(h->lv[l], w, s);
    }
    if (deflate) launch_pin_deflate(h->lv[0], h->rho, h->ke, h->pin_state, s);
    launch_norm_finish(h->partial, nblk_r, h->d_small, s);
    cudaMemcpyAsync(h->h_small, h->d_small, sizeof(double) * NCASE, cudaMemcpyDeviceToHost, s);
    if (h->mixed()) cudaMemcpyAsync(&h->h_small[62], h->d_tcflag, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (bfirst >= 0) cudaMemcpyAsync(&h->h_small[61], h->d_botflag, sizeof(int), cudaMemcpyDeviceToHost, s);
    return H3D_OK;
}

// deflation state from the current level-0 f: F = sum of f over the vertices but
// the origin, pending shift T = 0
void enqueue_pin_init(h3d_handle *h, cudaStream_t s) {
    const Level &L0 = h->lv[0];
    const int nb = norm_blocks(L0.P);
    launch_mean_partial(L0.P, L0.f, h->partial, nb, s);
    launch_sum18_finish(h->partial, nb, h->pin_state + 2 * NF, s);
    launch_pin_init(L0, h->pin_state + 2 * NF, h->pin_state, s);
}
void enqueue_pin_init(h3d_handle *h) { enqueue_pin_init(h, h->stream); }

// the refinement step of the refined solve: fold the correction into the FP64
// solution (u64 += u + T, u = 0), recompute level-0 f = f0 - K u64 from it, read
// the per-case weighted norms of that (current, not stale) residual and restart
// the deflation state from it
int enqueue_refine(h3d_handle *h, bool exact) {
    cudaStream_t s = h->stream;
    const Level &L0 = h->lv[0];
    launch_update64(L0, h->u64, L0.u, h->pin_state + NF, s);
    cudaMemsetAsync(L0.u, 0, sizeof(float) * field_floats(L0.P.nv), s);
    launch_fine_residual64(L0, h->rho, h->ke, h->ke64, h->f0, h->u64, L0.f, exact, s);
    const int nb = norm_blocks(L0.P);
    launch_weighted_norm(L0.P, L0.f, h->partial, nb, s);
    launch_norm_finish(h->partial, nb, h->d_small, s);
    cudaMemcpyAsync(h->h_small, h->d_small, sizeof(double) * NCASE, cudaMemcpyDeviceToHost, s);
    enqueue_pin_init(h);
    return H3D_OK;
}

// the refinement step from a zero FP64 solution and correction (a solve's start
// without a guess): u64 += 0 changes nothing and f0 - K 0 is f0 with the pinned
// origin's entries 0, so level-0 f is set from f0 directly; the norms and the
// deflation state are those enqueue_refine would compute, to the last bit
int enqueue_zero_start(h3d_handle *h) {
    cudaStream_t s = h->stream;
    const Level &L0 = h->lv[0];
    launch_rhs_at_zero(L0, h->f0, L0.f, s);
    const int nb = norm_blocks(L0.P);
    launch_weighted_norm(L0.P, L0.f, h->partial, nb, s);
    launch_norm_finish(h->partial, nb, h->d_small, s);
    cudaMemcpyAsync(h->h_small, h->d_small, sizeof(double) * NCASE, cudaMemcpyDeviceToHost, s);
    enqueue_pin_init(h);
    return H3D_OK;
}

// vgraph: one V-cycle (h3d_v_cycle); sgraph: the same with the deflation (solves);
// rgraph / xgraph: the refinement step with FP32 / FP64 accumulation of the residual
enum GraphKind { G_VCYCLE, G_SOLVE, G_REFINE, G_REFINE_EXACT };
int build_graph(h3d_handle *h, GraphKind kind) {
    cudaGraphExec_t &ge = kind == G_VCYCLE ? h->vgraph : kind == G_SOLVE ? h->sgraph
                        : kind == G_REFINE_EXACT ? h->xgraph : h->rgraph;
    if (ge) return H3D_OK;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    if (kind == G_REFINE || kind == G_REFINE_EXACT) enqueue_refine(h, kind == G_REFINE_EXACT);
    else enqueue_vcycle(h, 1.f, kind == G_SOLVE);
    CK(cudaStreamEndCapture(h->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { ge = nullptr; return fail(h, H3D_ERR_CUDA, std::string("graph: ") + cudaGetErrorString(e)); }
    return H3D_OK;
}

int weighted_norms(h3d_handle *h, const Planes &P, const float *v, double out[6]) {
    const int nb = norm_blocks(P);
    launch_weighted_norm(P, v, h->partial, nb, h->stream);
    launch_norm_finish(h->partial, nb, h->d_small, h->stream);
    CKL();
    CK(cudaMemcpyAsync(h->h_small, h->d_small, sizeof(double) * NCASE, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int c = 0; c < NCASE; c++) out[c] = std::sqrt(h->h_small[c]);
    return H3D_OK;
}

int check_level(h3d_handle *h, int level, bool coarse_only = false) {
    if (!h) return H3D_ERR_ARG;
    if (level < 0 || level >= h->nl || (coarse_only && level == 0))
        return fail(h, H3D_ERR_ARG, "level out of range");
    return H3D_OK;
}

}  // namespace

namespace {

// Autotuner (no reference counterpart).  Per smoothed level, each launch shape of
// the colour sweep and, on the coarse levels, of the residual is timed with CUDA
// events on the handle's stream (one untimed launch sequence, then three timed)
// and the fastest is kept.  The sweeps iterate on the level's r, so u and f are
// untouched (r is scratch that the next residual overwrites).  The shapes give
// the same results to the last bit; tuning changes only the time.  Graphs
// captured with the old shapes are dropped and re-captured on demand.
int autotune(h3d_handle *h) {
    CK(cudaSetDevice(h->device));
    cudaStream_t s = h->stream;
    constexpr int NSHAPE = H3D_NUM_SHAPES, REPS = 3;
    for (int l = 0; l < h->nl - 1; l++) {
        Level &L = h->lv[l];
        for (int kind = 0; kind < (l > 0 ? 2 : 1); kind++) {  // 0: sweep, 1: residual
            float best = 0;
            int pick = 0;
            for (int v = 0; v < NSHAPE; v++) {
                Level T = L;
                T.gs_shape = T.res_shape = v;
                if (kind == 0) T.u = L.r;  // the sweep iterates on scratch
                auto run = [&]() {
                    if (kind == 1) launch_coarse_residual(T, s);
                    else if (l == 0) launch_fine_gs(T, h->rho, h->ke, 1.f, s);
                    else launch_coarse_gs(T, 1.f, s);
                };
                run();
                CK(cudaEventRecord(h->ev0, s));
                for (int r = 0; r < REPS; r++) run();
                CK(cudaEventRecord(h->ev1, s));
                CK(cudaEventSynchronize(h->ev1));
                CKL();
                float ms = 0;
                CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
                if (v == 0 || ms < best) { best = ms; pick = v; }
            }
            if (kind == 0) L.gs_shape = pick;
            else L.res_shape = pick;
        }
    }
    destroy_graph(h);
    h->tuned = true;
    return H3D_OK;
}

}  // namespace

namespace {

// The solve loop of MG::solveEquation (MG.cpp:113-203) as a resumable state
// machine: begin() enqueues the first step on the handle's stream; after that
// stream has drained, advance() reads the step's result and enqueues the next
// one, until finished().  h3d_solve drives one handle; h3d_batch_elastic_matrix
// drives several, each on its own stream, so their kernels overlap on the GPU.
//
// Refined mode: the FP32 V-cycles on the correction measure the stale residual
// accurately down to ~1e-6 N of the correction's right-hand side; the correction
// is folded into u64 and the residual recomputed exactly once the estimate has
// dropped by theta (10x above that floor) or reached the tolerance, and the solve
// only stops when that exact residual meets the tolerance too.
struct SolveRun {
    enum Pending { P_NONE, P_START_REFINE, P_CYCLE, P_TRIGGER_REFINE, P_FINAL_REFINE, P_DONE };
    h3d_handle *h = nullptr;
    int mask = 63, it = 0, nref = 0, status = H3D_OK, explode_left = 2, maxit = 200;
    double tol = 1e-2, theta = 1e-3;
    bool refine = false, exact = false, with_guess = false, fallback_tried = false, done_flag = false;
    bool u64_zero = false;
    double fn[6] = {}, rel[6] = {1, 1, 1, 1, 1, 1}, base[6] = {1, 1, 1, 1, 1, 1};
    // largest selected stale estimate of each cycle since the last refinement
    std::vector<double> since_refine;
    Pending pending = P_NONE;
    cudaGraphExec_t refine_step = nullptr;

    bool selected(int c) const { return ((mask >> c) & 1) != 0; }
    bool finished() const { return pending == P_DONE; }
    long long n18() const { return field_floats(h->lv[0].P.nv); }      // elements of an FP64 field
    long long nf32() const { return field_floats(h->lv[0].P.nv); }     // elements of an FP32 field

    int reset_solution() {
        if (refine) CK(cudaMemsetAsync(h->u64, 0, sizeof(double) * n18(), h->stream));
        else CK(cudaMemsetAsync(h->lv[0].u, 0, sizeof(float) * nf32(), h->stream));
        u64_zero = refine;
        return H3D_OK;
    }
    // every start refinement runs with the correction u and the pending shift at
    // 0; u64_zero: the FP64 solution too (reset, no V-cycle since)
    int launch_refine(Pending next) {
        nref++;
        since_refine.clear();
        if (next == P_START_REFINE && u64_zero) {
            if (int e = enqueue_zero_start(h)) return e;
            CKL();
        } else {
            CK(cudaGraphLaunch(refine_step, h->stream));
        }
        pending = next;
        return H3D_OK;
    }
    int launch_cycle() {
        u64_zero = false;
        if (it >= maxit) return finish(H3D_NOT_CONVERGED);
        CK(cudaGraphLaunch(h->sgraph, h->stream));
        pending = P_CYCLE;
        return H3D_OK;
    }
    void read_base() {
        for (int c = 0; c < NCASE; c++) base[c] = std::sqrt(h->h_small[c]) / (fn[c] + 1e-10);
    }
    // a solve that ends without converging still leaves its iterate in u64; the
    // FP32 solution takes the pending shift and f is restored
    int finish(int st) {
        status = st;
        if (refine && st != H3D_OK) return launch_refine(P_FINAL_REFINE);
        if (!refine) launch_pin_fold(h->lv[0], h->rho, h->ke, h->pin_state, h->stream);
        CK(cudaEventRecord(h->ev1, h->stream));
        pending = P_DONE;
        return H3D_OK;
    }

    int begin(h3d_handle *hh, int case_mask, double tolerance, int guess) {
        h = hh;
        if (!h) return H3D_ERR_ARG;
        if (!h->have_stencils) return fail(h, H3D_ERR_STATE, "no stencils");
        if (case_mask <= 0 || case_mask > 63) return fail(h, H3D_ERR_ARG, "case_mask must select load cases");
        CK(cudaSetDevice(h->device));
        mask = case_mask;
        tol = tolerance;
        with_guess = guess != 0;
        refine = h->refine();
        u64_zero = refine && with_guess && h->u64_zero;  // a guess that is all zero
        h->u64_zero = false;
        const Level &L0 = h->lv[0];
        if (!with_guess)
            if (int e = reset_solution()) return e;
        // balance the right-hand side: a periodic load has zero net force, and the few
        // ulps of net force left by FP32 rounding would, in the pinned problem, become
        // a point load at the origin; remove each plane's mean over the unique vertices
        {
            float *rhs = refine ? h->f0 : L0.f;
            const int nb = norm_blocks(L0.P);
            launch_mean_partial(L0.P, rhs, h->partial, nb, h->stream);
            launch_remove_mean(L0.P, rhs, h->partial, nb, h->stream);
            CKL();
        }
        if (!h->tuned)
            if (int e = autotune(h)) return e;
        if (int e = build_graph(h, G_SOLVE)) return e;
        // below ~1e-4 the FP32 products of the difference-form residual would floor
        // the iteration, so tight targets take the FP64-accumulating residual
        exact = refine && tol < (h->fp32_refine() ? 2e-6 : 1e-4);
        if (refine)
            if (int e = build_graph(h, exact ? G_REFINE_EXACT : G_REFINE)) return e;
        refine_step = exact ? h->xgraph : h->rgraph;
        {  // the reference norms, read by start() once the stream has drained
            const float *rhs = refine ? h->f0 : L0.f;
            const int nb = norm_blocks(L0.P);
            launch_weighted_norm(L0.P, rhs, h->partial, nb, h->stream);
            launch_norm_finish(h->partial, nb, h->d_small, h->stream);
            CKL();
            CK(cudaMemcpyAsync(h->h_small, h->d_small, sizeof(double) * NCASE, cudaMemcpyDeviceToHost, h->stream));
        }
        return H3D_OK;
    }

    // the first step, after begin(): a batch begins every design before it starts
    // any, so the designs' preparations overlap
    int start() {
        CK(cudaStreamSynchronize(h->stream));
        for (int c = 0; c < NCASE; c++) fn[c] = std::sqrt(h->h_small[c]);
        const Level &L0 = h->lv[0];
        const int nmax = std::max(L0.P.n[0], std::max(L0.P.n[1], L0.P.n[2]));
        theta = std::max(1e-3, 1e-5 * nmax);
        CK(cudaEventRecord(h->ev0, h->stream));
        CK(cudaMemsetAsync(h->pin_state + NF, 0, sizeof(double) * NF, h->stream));  // no pending shift
        CK(cudaMemsetAsync(h->d_botflag, 0, sizeof(int), h->stream));
        h->h_small[61] = 0.0;
        if (refine) {
            CK(cudaMemsetAsync(L0.u, 0, sizeof(float) * nf32(), h->stream));
            return launch_refine(P_START_REFINE);
        }
        enqueue_pin_init(h);
        return launch_cycle();
    }

    // the step enqueued last has completed on the handle's stream
    int advance() {
        switch (pending) {
        case P_START_REFINE: {
            read_base();
            // a starting guess worse than zero (relative residual above 1) is dropped
            bool worse = false;
            for (int c = 0; c < NCASE; c++)
                if (selected(c) && !(base[c] <= 1.0)) worse = true;
            if (with_guess && worse && !fallback_tried) {
                fallback_tried = true;
                if (int e = reset_solution()) return e;
                return launch_refine(P_START_REFINE);
            }
            return launch_cycle();
        }
        case P_CYCLE: {
            it++;
            if (h->mixed() && *reinterpret_cast<int *>(&h->h_small[62]))
                return fail(h, H3D_ERR_CUDA, "tensor-core residual: mbarrier wait timed out");
            if (*reinterpret_cast<int *>(&h->h_small[61]))
                return fail(h, H3D_ERR_CUDA, "cooperative V-cycle bottom: a grid barrier wait timed out");
            bool bad = false, done = true, trigger = true;
            double worst = 0;
            for (int c = 0; c < NCASE; c++) {
                rel[c] = std::sqrt(h->h_small[c]) / (fn[c] + 1e-10);
                if (!selected(c)) continue;
                if (!(rel[c] <= 10.0)) bad = true;
                if (!(rel[c] <= tol)) done = false;
                if (!(rel[c] <= tol || rel[c] <= theta * base[c])) trigger = false;
                worst = std::max(worst, rel[c]);
            }
            // a correction solve whose estimate fell by less than 2x over three
            // cycles has met the FP32 floor of its own equation (high-contrast
            // designs): refresh it from the exact residual instead of waiting for theta
            since_refine.push_back(worst);
            const size_t ns = since_refine.size();
            if (ns >= 4 && !(worst < 0.5 * since_refine[ns - 4])) trigger = true;
            if (bad) {  // MG.cpp:140-182: restart from zero once, then give up
                if (--explode_left <= 0) return finish(H3D_DIVERGED);
                if (!refine) launch_pin_fold(h->lv[0], h->rho, h->ke, h->pin_state, h->stream);  // restores f
                if (int e = reset_solution()) return e;
                CK(cudaMemsetAsync(h->pin_state + NF, 0, sizeof(double) * NF, h->stream));
                fallback_tried = true;
                if (refine) {
                    CK(cudaMemsetAsync(h->lv[0].u, 0, sizeof(float) * nf32(), h->stream));
                    return launch_refine(P_START_REFINE);
                }
                enqueue_pin_init(h);
                return launch_cycle();
            }
            if (refine && trigger) {
                done_flag = done;
                return launch_refine(P_TRIGGER_REFINE);
            }
            if (done) return finish(H3D_OK);
            return launch_cycle();
        }
        case P_TRIGGER_REFINE: {
            read_base();
            bool done = done_flag;
            if (done)
                for (int c = 0; c < NCASE; c++)
                    if (selected(c) && !(base[c] <= tol)) done = false;
            if (done) return finish(H3D_OK);
            return launch_cycle();
        }
        case P_FINAL_REFINE:
            read_base();
            CK(cudaEventRecord(h->ev1, h->stream));
            pending = P_DONE;
            return H3D_OK;
        default:
            return fail(h, H3D_ERR_STATE, "solve advanced in a wrong state");
        }
    }

    int end(h3d_solve_stats *stats) {
        CK(cudaEventSynchronize(h->ev1));
        if (stats) {
            stats->vcycles = it;
            stats->refinements = nref;
            stats->status = status;
            for (int c = 0; c < NCASE; c++) stats->rel_res[c] = rel[c];
            float ms = 0;
            cudaEventElapsedTime(&ms, h->ev0, h->ev1);
            stats->solve_ms = ms;
        }
        if (status != H3D_OK) return fail(h, status, status == H3D_DIVERGED ? "multigrid diverged" : "not converged");
        return H3D_OK;
    }
};


// the coarsest level's assembly and Gauss-Jordan inversion with the
// singular-matrix flag copied to the host; factor_coarsest_check reads it once
// the stream has drained
int factor_coarsest_enqueue(h3d_handle *h) {
    cudaStream_t s = h->stream;
    if (!h->fgraph) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        launch_coarse_assemble(h->lv[h->nl - 1], h->aug, s);
        cudaMemsetAsync(h->d_flag, 0, sizeof(int), s);
        launch_gauss_jordan(h->aug, h->ndof, h->d_flag, s);
        CK(cudaStreamEndCapture(s, &g));
        cudaError_t e = cudaGraphInstantiate(&h->fgraph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            h->fgraph = nullptr;
            return fail(h, H3D_ERR_CUDA, std::string("graph: ") + cudaGetErrorString(e));
        }
    }
    CK(cudaGraphLaunch(h->fgraph, s));
    CK(cudaMemcpyAsync(&h->h_small[63], h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    return H3D_OK;
}

int factor_coarsest_check(h3d_handle *h) {
    int flag = 0;
    std::memcpy(&flag, &h->h_small[63], sizeof(int));
    if (flag) return fail(h, H3D_ERR_SINGULAR, "coarsest-grid matrix is singular");
    h->have_stencils = true;
    return H3D_OK;
}

// right-hand sides and warm start from the stored solutions, mean removed
// (homogenization.cu:471-477, grid.cpp:1131-1141)
int elastic_prepare(h3d_handle *h) {
    Level &L = h->lv[0];
    cudaStream_t s = h->stream;
    const int nb = norm_blocks(L.P);
    if (h->refine()) {
        launch_rhs(L, h->rho, h->rhs, h->f0, s);
        if (h->chi_zero) {  // the copy and its (zero) mean removal would leave zeros
            CK(cudaMemsetAsync(h->u64, 0, sizeof(double) * field_floats(L.P.nv), s));
        } else {
            CK(cudaMemcpyAsync(h->u64, h->chi, sizeof(double) * field_floats(L.P.nv), cudaMemcpyDeviceToDevice, s));
            launch_remove_mean64(L.P, h->u64, h->partial, nb, s);
        }
        h->u64_zero = h->chi_zero;
    } else {
        launch_rhs(L, h->rho, h->rhs, L.f, s);
        launch_convert_field(L.P.nv, h->chi, L.u, s);
        launch_mean_partial(L.P, L.u, h->partial, nb, s);
        launch_remove_mean(L.P, L.u, h->partial, nb, s);
    }
    CKL();
    return H3D_OK;
}

// store the solutions as chi and enqueue the energy reduction of the 21 entries
// of C, with the results and the kernel's wait flag copied to the host
int elastic_enqueue_energy(h3d_handle *h) {
    Level &L = h->lv[0];
    cudaStream_t s = h->stream;
    if (h->refine())
        CK(cudaMemcpyAsync(h->chi, h->u64, sizeof(double) * field_floats(L.P.nv), cudaMemcpyDeviceToDevice, s));
    else launch_convert_field(L.P.nv, L.u, h->chi, s);
    h->chi_zero = false;
    int nsm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
    const int eb = energy_tc_blocks(L.P, nsm);
    CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), s));
    if (launch_elastic_tc(L.P, h->chi, h->rho, h->ke, h->partial, eb, h->d_flag, s) != 0)
        return fail(h, H3D_ERR_CUDA, "tensor-core energy kernel could not be configured");
    launch_elastic_finish(h->partial, eb, h->d_small, s);
    CKL();
    CK(cudaMemcpyAsync(h->h_small, h->d_small, sizeof(double) * 21, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&h->h_small[63], h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    return H3D_OK;
}

// C from the reduced energies once the stream has drained
int elastic_read(h3d_handle *h, double *C) {
    if (*reinterpret_cast<int *>(&h->h_small[63]))
        return fail(h, H3D_ERR_CUDA, "tensor-core energy kernel: mbarrier wait timed out");
    const double vol = (double)h->lv[0].P.nv;
    int t = 0;
    for (int i = 0; i < 6; i++)
        for (int j = i; j < 6; j++) {
            C[i * 6 + j] = C[j * 6 + i] = h->h_small[t] / vol;
            t++;
        }
    return H3D_OK;
}

// a batch drives each design's stream and host mirror separately, so a handle
// may appear only once
int distinct_handles(h3d_handle *const *hs, int n) {
    std::vector<const h3d_handle *> v(hs, hs + n);
    std::sort(v.begin(), v.end());
    for (int i = 1; i < n; i++)
        if (v[i] == v[i - 1]) return fail(hs[0], H3D_ERR_ARG, "a handle appears twice in the batch");
    return H3D_OK;
}

}  // namespace

extern "C" {

static int create_impl(h3d_handle *h, const h3d_config *cfg) {
    int dims[MAXLV][3], rat[MAXLV][3];
    const int nl = build_hierarchy(cfg->reso, dims, rat);
    if (nl < 2) return fail(h, H3D_ERR_ARG, "resolution gives fewer than two grid levels");
    if (!(cfg->youngs_modulus > 0) || !(cfg->poisson_ratio > -1.0 && cfg->poisson_ratio < 0.5))
        return fail(h, H3D_ERR_ARG, "invalid material");
    if (cfg->coarse_mode != H3D_COARSE_EXACT && cfg->coarse_mode != H3D_COARSE_PROJECT)
        return fail(h, H3D_ERR_ARG, "invalid coarse_mode");
    if (cfg->pin_mode != H3D_PIN_IDENTITY && cfg->pin_mode != H3D_PIN_GALERKIN)
        return fail(h, H3D_ERR_ARG, "invalid pin_mode");
    if (cfg->precision != H3D_PREC_REFINE && cfg->precision != H3D_PREC_FP32 && cfg->precision != H3D_PREC_MIXED &&
        cfg->precision != H3D_PREC_MIXED_TC)
        return fail(h, H3D_ERR_ARG, "invalid precision");
    if (cfg->stencil_precision != H3D_STENCIL_FP16 && cfg->stencil_precision != H3D_STENCIL_FP32)
        return fail(h, H3D_ERR_ARG, "invalid stencil_precision");
    h->cfg = *cfg;
    h->device = cfg->device;
    h->nl = nl;
    CK(cudaSetDevice(h->device));
    for (int l = 0; l < nl; l++) {
        Level &L = h->lv[l];
        L.P = make_planes(dims[l]);
        for (int a = 0; a < 3; a++) L.ratio[a] = rat[l][a];
        if (l < nl - 1 && !L.P.even) return fail(h, H3D_ERR_ARG, "every smoothed level needs even dimensions");
        const size_t bytes = sizeof(float) * (size_t)field_floats(L.P.nv);
        CK(cudaMalloc(&L.u, bytes));
        CK(cudaMalloc(&L.f, bytes));
        CK(cudaMalloc(&L.r, bytes));
        CK(cudaMemset(L.u, 0, bytes));
        CK(cudaMemset(L.f, 0, bytes));
        CK(cudaMemset(L.r, 0, bytes));
        if (l > 0) {
            L.st32 = cfg->stencil_precision == H3D_STENCIL_FP32;
            const size_t sb = sizeof(uint4) * (L.st32 ? NCHUNK32 : NCHUNK) * (size_t)L.P.nv;
            CK(cudaMalloc(&L.st, sb));
            CK(cudaMemset(L.st, 0, sb));
        }
    }
    const long long nv0 = h->lv[0].P.nv;
    CK(cudaMalloc(&h->rho, sizeof(float) * nv0));
    CK(cudaMalloc(&h->chi, sizeof(double) * field_floats(nv0)));
    CK(cudaMemset(h->chi, 0, sizeof(double) * field_floats(nv0)));
    if (h->refine()) {
        CK(cudaMalloc(&h->u64, sizeof(double) * field_floats(nv0)));
        CK(cudaMemset(h->u64, 0, sizeof(double) * field_floats(nv0)));
        CK(cudaMalloc(&h->f0, sizeof(float) * field_floats(nv0)));
        CK(cudaMemset(h->f0, 0, sizeof(float) * field_floats(nv0)));
    }
    // element matrix and derived tables
    element_matrix(cfg->youngs_modulus, cfg->poisson_ratio, h->ked);
    for (int i = 0; i < 576; i++) {
        h->ke.k[i] = (float)h->ked[i];
        h->ke64.k[i] = h->ked[i];
    }
    for (int c = 0; c < NCASE; c++)
        for (int a = 0; a < 24; a++) {
            double s = 0;
            for (int b = 0; b < 8; b++)
                for (int m = 0; m < 3; m++) s += h->ked[a * 24 + 3 * b + m] * macro_disp_h(b, c, m);
            h->rhs.g[c][a] = (float)s;
        }
    build_q(h->ked, h->lv[1].ratio, h->qhost, h->nsub);
    CK(cudaMalloc(&h->q, sizeof(float) * h->qhost.size()));
    CK(cudaMemcpy(h->q, h->qhost.data(), sizeof(float) * h->qhost.size(), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&h->d_ked, sizeof(double) * 576));
    CK(cudaMemcpy(h->d_ked, h->ked, sizeof(double) * 576, cudaMemcpyHostToDevice));
    const Level &C = h->lv[nl - 1];
    h->ndof = (int)(3 * C.P.nv);
    CK(cudaMalloc(&h->aug, sizeof(double) * gauss_jordan_doubles(h->ndof)));
    CK(cudaMalloc(&h->d_flag, sizeof(int)));
    CK(cudaMalloc(&h->d_tcflag, sizeof(int)));
    CK(cudaMemset(h->d_tcflag, 0, sizeof(int)));
    CK(cudaMalloc(&h->d_bar, 2 * sizeof(unsigned)));
    CK(cudaMemset(h->d_bar, 0, 2 * sizeof(unsigned)));
    CK(cudaMalloc(&h->d_botflag, sizeof(int)));
    CK(cudaMemset(h->d_botflag, 0, sizeof(int)));
    CK(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device));
    if (h->mixed() && configure_fine_residual_tc() != 0)
        return fail(h, H3D_ERR_CUDA, "tensor-core residual kernel could not be configured");
    // reduction scratch: residual partials, norms, C partials, means, OC
    size_t pn = ((size_t)fine_residual_blocks(h->lv[0]) + NORM_FINISH_CHUNKS) * NCASE;
    pn = std::max(pn, (size_t)4096 * 21);
    pn = std::max(pn, (size_t)2048 * NF + NF);
    pn = std::max(pn, (size_t)4 + 1184);
    h->partial_n = pn;
    CK(cudaMalloc(&h->partial, sizeof(double) * pn));
    CK(cudaMalloc(&h->d_small, sizeof(double) * 64));
    CK(cudaMallocHost(&h->h_small, sizeof(double) * 64));
    std::memset(h->h_small, 0, sizeof(double) * 64);
    CK(cudaMalloc(&h->pin_state, sizeof(double) * 3 * NF));
    CK(cudaMemset(h->pin_state, 0, sizeof(double) * 3 * NF));
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    return H3D_OK;
}

int h3d_create(const h3d_config *cfg, h3d_handle **out) {
    if (!cfg || !out) return H3D_ERR_ARG;
    *out = nullptr;
    h3d_handle *h = new (std::nothrow) h3d_handle();
    if (!h) return H3D_ERR_NOMEM;
    const int e = create_impl(h, cfg);
    if (e != H3D_OK) {
        h3d_destroy(h);
        return e;
    }
    *out = h;
    return H3D_OK;
}

int h3d_destroy(h3d_handle *h) {
    if (!h) return H3D_ERR_ARG;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    destroy_graph(h);
    for (int l = 0; l < h->nl; l++) {
        cudaFree(h->lv[l].u); cudaFree(h->lv[l].f); cudaFree(h->lv[l].r); cudaFree(h->lv[l].st);
    }
    cudaFree(h->rho); cudaFree(h->chi); cudaFree(h->u64); cudaFree(h->f0);
    cudaFree(h->q); cudaFree(h->d_ked); cudaFree(h->aug);
    cudaFree(h->d_dcw);
    cudaFree(h->d_bar);
    cudaFree(h->d_botflag);
    if (h->h_dcw) cudaFreeHost(h->h_dcw);
    cudaFree(h->d_flag); cudaFree(h->d_tcflag); cudaFree(h->partial); cudaFree(h->d_small); cudaFree(h->tmp); cudaFree(h->pin_state);
    if (h->h_small) cudaFreeHost(h->h_small);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return H3D_OK;
}

const char *h3d_last_error(const h3d_handle *h) { return h ? h->err.c_str() : "null handle"; }

int h3d_sync(h3d_handle *h) {
    if (!h) return H3D_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    return H3D_OK;
}

void *h3d_stream(h3d_handle *h) { return h ? (void *)h->stream : nullptr; }

int h3d_num_levels(const h3d_handle *h) { return h ? h->nl : -1; }

int h3d_level_dims(const h3d_handle *h, int level, int dims[3], int ratio[3]) {
    if (!h || level < 0 || level >= h->nl) return H3D_ERR_ARG;
    for (int a = 0; a < 3; a++) {
        if (dims) dims[a] = h->lv[level].P.n[a];
        if (ratio) ratio[a] = h->lv[level].ratio[a];
    }
    return H3D_OK;
}

int h3d_element_matrix(const h3d_handle *h, double ke[576]) {
    if (!h || !ke) return H3D_ERR_ARG;
    std::memcpy(ke, h->ked, sizeof(double) * 576);
    return H3D_OK;
}

int h3d_update_density(h3d_handle *h, const float *rho_dev, int pitchT) {
    if (!h || !rho_dev) return H3D_ERR_ARG;
    CK(cudaSetDevice(h->device));
    const int *n = h->lv[0].P.n;
    if (pitchT < 0) pitchT = n[0];
    if (pitchT < n[0]) return fail(h, H3D_ERR_ARG, "pitchT smaller than the x resolution");
    launch_density_in(n, rho_dev, pitchT, h->rho, h->stream);
    CKL();
    h->have_density = true;
    return h3d_update_stencils(h);
}

int h3d_restrict_stencil(h3d_handle *h, int coarse_level) {
    if (int e = check_level(h, coarse_level, true)) return e;
    CK(cudaSetDevice(h->device));
    if (coarse_level == 1) {
        if (!h->have_density) return fail(h, H3D_ERR_STATE, "no density");
        launch_galerkin_l1(h->lv[0], h->lv[1], h->rho, h->q, h->nsub, h->stream);
        launch_dirichlet_patch(h->lv[0], h->lv[1], h->rho, h->d_ked, h->cfg.pin_mode == H3D_PIN_IDENTITY,
                               h->stream);
    } else {
        launch_galerkin(h->lv[coarse_level - 1], h->lv[coarse_level], h->stream);
    }
    CKL();
    h->have_stencils = false;
    return H3D_OK;
}

int h3d_factor_coarsest(h3d_handle *h) {
    if (!h) return H3D_ERR_ARG;
    CK(cudaSetDevice(h->device));
    if (int e = factor_coarsest_enqueue(h)) return e;
    CK(cudaStreamSynchronize(h->stream));
    return factor_coarsest_check(h);
}

int h3d_update_stencils(h3d_handle *h) {
    if (!h) return H3D_ERR_ARG;
    if (!h->have_density) return fail(h, H3D_ERR_STATE, "no density");
    for (int l = 1; l < h->nl; l++)
        if (int e = h3d_restrict_stencil(h, l)) return e;
    return h3d_factor_coarsest(h);
}

int h3d_enforce_unit_macro_strain(h3d_handle *h) {
    if (!h) return H3D_ERR_ARG;
    if (!h->have_density) return fail(h, H3D_ERR_STATE, "no density");
    launch_rhs(h->lv[0], h->rho, h->rhs, h->lv[0].f, h->stream);
    if (h->refine())
        CK(cudaMemcpyAsync(h->f0, h->lv[0].f, sizeof(float) * field_floats(h->lv[0].P.nv), cudaMemcpyDeviceToDevice,
                           h->stream));
    CKL();
    return H3D_OK;
}

int h3d_gs_relaxation(h3d_handle *h, int level, float w, int times) {
    if (int e = check_level(h, level)) return e;
    if (level == h->nl - 1) return fail(h, H3D_ERR_ARG, "the coarsest level is solved directly");
    if (level == 0 && !h->have_density) return fail(h, H3D_ERR_STATE, "no density");
    if (level > 0 && !h->have_stencils) return fail(h, H3D_ERR_STATE, "no stencils");
    for (int t = 0; t < times; t++) {
        if (level == 0) launch_fine_gs(h->lv[0], h->rho, h->ke, w, h->stream);
        else launch_coarse_gs(h->lv[level], w, h->stream);
    }
    CKL();
    return H3D_OK;
}

int h3d_update_residual(h3d_handle *h, int level) {
    if (int e = check_level(h, level)) return e;
    if (level == 0) {
        if (!h->have_density) return fail(h, H3D_ERR_STATE, "no density");
        if (h->mixed()) {
            CK(cudaSetDevice(h->device));
            launch_fine_residual_tc(h->lv[0], h->rho, h->ke, nullptr, fine_residual_tc_blocks(h->lv[0].P, h->num_sms),
                                    h->d_tcflag, h->stream);
        } else {
            launch_fine_residual(h->lv[0], h->rho, h->ke, nullptr, 0, h->stream);
        }
    } else {
        if (!h->have_stencils) return fail(h, H3D_ERR_STATE, "no stencils");
        launch_coarse_residual(h->lv[level], h->stream);
    }
    CKL();
    return H3D_OK;
}

int h3d_restrict_residual(h3d_handle *h, int coarse_level) {
    if (int e = check_level(h, coarse_level, true)) return e;
    launch_restrict(h->lv[coarse_level - 1], h->lv[coarse_level], h->stream);
    CKL();
    return H3D_OK;
}

int h3d_prolongate_correction(h3d_handle *h, int fine_level) {
    if (int e = check_level(h, fine_level)) return e;
    if (fine_level == h->nl - 1) return fail(h, H3D_ERR_ARG, "no coarser level");
    launch_prolong(h->lv[fine_level], h->lv[fine_level + 1], fine_level == 0, h->stream);
    CKL();
    return H3D_OK;
}

int h3d_coarse_solve(h3d_handle *h) {
    if (!h) return H3D_ERR_ARG;
    if (!h->have_stencils) return fail(h, H3D_ERR_STATE, "no stencils");
    launch_coarse_apply(h->lv[h->nl - 1], h->aug, h->cfg.coarse_mode == H3D_COARSE_PROJECT, h->stream);
    CKL();
    return H3D_OK;
}

int h3d_reset_displacement(h3d_handle *h, int level) {
    if (!h) return H3D_ERR_ARG;
    for (int l = 0; l < h->nl; l++)
        if (level < 0 || level == l)
            CK(cudaMemsetAsync(h->lv[l].u, 0, sizeof(float) * field_floats(h->lv[l].P.nv), h->stream));
    return H3D_OK;
}

int h3d_field_norms(h3d_handle *h, int field, double out[6]) {
    if (!h || !out) return H3D_ERR_ARG;
    const Level &L = h->lv[0];
    if (field == H3D_FIELD_CHI || field == H3D_FIELD_SOLUTION) {
        const double *src = field == H3D_FIELD_CHI ? h->chi : h->u64;
        if (!src) return fail(h, H3D_ERR_ARG, "no FP64 solution in this precision mode");
        if (int e = ensure_tmp(h, (size_t)field_floats(L.P.nv))) return e;
        launch_convert_field(L.P.nv, src, h->tmp, h->stream);
        return weighted_norms(h, L.P, h->tmp, out);
    }
    const float *v = field == H3D_FIELD_U ? L.u : field == H3D_FIELD_F ? L.f : field == H3D_FIELD_R ? L.r : nullptr;
    if (!v) return fail(h, H3D_ERR_ARG, "field has no norm");
    return weighted_norms(h, L.P, v, out);
}

int h3d_v_cycle(h3d_handle *h, float w, int pre, int post) {
    if (!h) return H3D_ERR_ARG;
    if (!h->have_stencils) return fail(h, H3D_ERR_STATE, "no stencils");
    if (pre != 1 || post != 1) return fail(h, H3D_ERR_ARG, "only V(1,1) is supported");
    CK(cudaSetDevice(h->device));
    if (w == 1.f) {
        if (int e = build_graph(h, G_VCYCLE)) return e;
        CK(cudaGraphLaunch(h->vgraph, h->stream));
    } else {
        enqueue_vcycle(h, w);
        CKL();
    }
    return H3D_OK;
}

int h3d_solve(h3d_handle *h, int case_mask, double tol, int with_guess, h3d_solve_stats *stats) {
    SolveRun run;
    if (int e = run.begin(h, case_mask, tol, with_guess)) return e;
    if (int e = run.start()) return e;
    while (!run.finished()) {
        CK(cudaStreamSynchronize(h->stream));
        if (int e = run.advance()) return e;
    }
    return run.end(stats);
}

int h3d_autotune(h3d_handle *h) {
    if (!h) return H3D_ERR_ARG;
    if (!h->have_stencils) return fail(h, H3D_ERR_STATE, "no stencils");
    return autotune(h);
}

int h3d_get_tuning(const h3d_handle *h, int level, int shapes[2]) {
    if (!h || !shapes || level < 0 || level >= h->nl) return H3D_ERR_ARG;
    shapes[0] = h->lv[level].gs_shape;
    shapes[1] = h->lv[level].res_shape;
    return H3D_OK;
}

int h3d_set_tuning(h3d_handle *h, int level, int gs_shape, int res_shape) {
    if (!h) return H3D_ERR_ARG;
    if (level < 0 || level >= h->nl || gs_shape < 0 || gs_shape >= H3D_NUM_SHAPES || res_shape < 0 ||
        res_shape >= H3D_NUM_SHAPES)
        return fail(h, H3D_ERR_ARG, "level or launch shape out of range");
    h->lv[level].gs_shape = gs_shape;
    h->lv[level].res_shape = res_shape;
    destroy_graph(h);
    h->tuned = true;
    return H3D_OK;
}

int h3d_set_vcycle_bottom(h3d_handle *h, int64_t max_level_vertices) {
    if (!h || max_level_vertices < 0) return H3D_ERR_ARG;
    h->bottom_nv = max_level_vertices;
    destroy_graph(h);
    return H3D_OK;
}

int h3d_reset_solutions(h3d_handle *h) {
    if (!h) return H3D_ERR_ARG;
    CK(cudaMemsetAsync(h->chi, 0, sizeof(double) * field_floats(h->lv[0].P.nv), h->stream));
    h->chi_zero = true;
    return H3D_OK;
}

int h3d_elastic_matrix(h3d_handle *h, double tol, double C[36], h3d_solve_stats *stats) {
    if (!h || !C) return H3D_ERR_ARG;
    if (!h->have_stencils) return fail(h, H3D_ERR_STATE, "no stencils");
    CK(cudaSetDevice(h->device));
    if (int e = elastic_prepare(h)) return e;
    h3d_solve_stats st;
    int e = h3d_solve(h, 63, tol, 1, &st);
    if (stats) *stats = st;
    if (e != H3D_OK && e != H3D_NOT_CONVERGED) return e;
    if (int e2 = elastic_enqueue_energy(h)) return e2;
    CK(cudaStreamSynchronize(h->stream));
    if (int e2 = elastic_read(h, C)) return e2;
    return e;
}

int h3d_batch_update_density(h3d_handle *const *hs, const float *const *rho_dev, int n) {
    if (!hs || !rho_dev || n < 0) return H3D_ERR_ARG;
    for (int i = 0; i < n; i++)
        if (!hs[i] || !rho_dev[i]) return H3D_ERR_ARG;
    if (int e = distinct_handles(hs, n)) return e;
    // enqueue every design's assembly, then collect the singular-matrix flags, so
    // the assemblies of different designs run concurrently on their own streams
    int first = H3D_OK;
    for (int i = 0; i < n; i++) {
        h3d_handle *h = hs[i];
        int e = [&]() -> int {
            CK(cudaSetDevice(h->device));
            launch_density_in(h->lv[0].P.n, rho_dev[i], h->lv[0].P.n[0], h->rho, h->stream);
            CKL();
            h->have_density = true;
            for (int l = 1; l < h->nl; l++)
                if (int e2 = h3d_restrict_stencil(h, l)) return e2;
            return factor_coarsest_enqueue(h);
        }();
        if (e && first == H3D_OK) first = e;
    }
    for (int i = 0; i < n; i++) {
        h3d_handle *h = hs[i];
        int e = [&]() -> int {
            CK(cudaSetDevice(h->device));
            CK(cudaStreamSynchronize(h->stream));
            return factor_coarsest_check(h);
        }();
        if (e && first == H3D_OK) first = e;
    }
    return first;
}

int h3d_batch_elastic_matrix(h3d_handle *const *hs, int n, double tol, double *C, h3d_solve_stats *stats,
                             int *status) {
    if (!hs || !C || n < 0) return H3D_ERR_ARG;
    for (int i = 0; i < n; i++)
        if (!hs[i]) return H3D_ERR_ARG;
    if (int e = distinct_handles(hs, n)) return e;
    std::vector<SolveRun> runs(n);
    std::vector<int> st(n, H3D_OK);
    std::vector<char> live(n, 0);
    // start every solve (the graph captures happen here, before any polling)
    for (int i = 0; i < n; i++) {
        h3d_handle *h = hs[i];
        if (!h->have_stencils) { st[i] = fail(h, H3D_ERR_STATE, "no stencils"); continue; }
        st[i] = [&]() -> int {
            CK(cudaSetDevice(h->device));
            if (int e = elastic_prepare(h)) return e;
            return runs[i].begin(h, 63, tol, 1);
        }();
    }
    for (int i = 0; i < n; i++) {
        if (st[i] != H3D_OK) continue;
        h3d_handle *h = hs[i];
        st[i] = [&]() -> int {
            CK(cudaSetDevice(h->device));
            return runs[i].start();
        }();
        live[i] = st[i] == H3D_OK;
    }
    // advance whichever design's step has completed; each design's V-cycles and
    // refinements run on its own stream, so small designs fill the GPU together
    int nlive = 0;
    for (int i = 0; i < n; i++) nlive += live[i];
    while (nlive > 0) {
        bool progressed = false;
        for (int i = 0; i < n; i++) {
            if (!live[i]) continue;
            h3d_handle *h = hs[i];
            if (cudaSetDevice(h->device) != cudaSuccess) {  // the handles may sit on different GPUs
                st[i] = fail(h, H3D_ERR_CUDA, "cudaSetDevice failed");
                live[i] = 0;
                nlive--;
                continue;
            }
            cudaError_t q = cudaStreamQuery(h->stream);
            if (q == cudaErrorNotReady) continue;
            progressed = true;
            int e = q == cudaSuccess ? runs[i].advance() : fail(h, H3D_ERR_CUDA, cudaGetErrorString(q));
            if (e == H3D_OK && runs[i].finished()) {
                h3d_solve_stats s1;
                e = runs[i].end(&s1);
                if (stats) stats[i] = s1;
                if (e == H3D_OK || e == H3D_NOT_CONVERGED) {
                    const int e2 = elastic_enqueue_energy(h);
                    if (e2) e = e2;
                }
                st[i] = e;
                live[i] = 0;
                nlive--;
            } else if (e != H3D_OK) {
                st[i] = e;
                live[i] = 0;
                nlive--;
            }
        }
        if (!progressed) std::this_thread::yield();
    }
    int first = H3D_OK;
    for (int i = 0; i < n; i++) {
        h3d_handle *h = hs[i];
        if (st[i] == H3D_OK || st[i] == H3D_NOT_CONVERGED) {
            const int e = [&]() -> int {
                CK(cudaSetDevice(h->device));
                CK(cudaStreamSynchronize(h->stream));
                return elastic_read(h, C + 36 * (size_t)i);
            }();
            if (e) st[i] = e;
        }
        if (status) status[i] = st[i];
        if (st[i] != H3D_OK && first == H3D_OK) first = st[i];
    }
    return first;
}

}  // extern "C"

// ---- lockstep batches -------------------------------------------------------
// The V-cycle of enqueue_vcycle for all designs at once: level index l runs, for
// the designs that have it, the restriction into l (clearing l's solution), then
// the down leg's sweep and residual, or the coarsest solve where l is a design's
// last level; the up leg prolongs and sweeps; then the deflation and the norms.
// Each design sees its own launches' operations in its own order.
// one branch of the batch V-cycle graph: the tables of some of the batch's designs
struct LockGroup {
    std::vector<int> members;  // indices into the batch
    int lmax = 0;
    // launch shapes of the sweeps: level 0, and each coarse level (timed at creation)
    int fine_shape = 0;
    int coarse_shape[MAXLV] = {};
    BatchTab fine, norm;
    BatchTab coarse[MAXLV], xfer[MAXLV], coarsest[MAXLV];
    cudaStream_t stream = nullptr;  // capture stream of the branch (the batch stream for group 0)
    cudaEvent_t join = nullptr;
};

struct h3d_lockstep {
    std::vector<h3d_handle *> hs;
    int n = 0, device = 0, project = 0;
    bool f32 = false;
    KeMat ke;
    // the designs are split into groups whose V-cycle launches are parallel branches
    // of the one batch graph, so one group's launches fill the last partial wave of
    // another's
    std::vector<LockGroup> groups;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    cudaEvent_t ev0 = nullptr, fork = nullptr;
    int *d_active = nullptr, *h_active = nullptr;
    double *d_norms = nullptr, *h_norms = nullptr;
    std::string err;
};

namespace {

int lfail(h3d_lockstep *b, int code, const std::string &msg) {
    if (b) b->err = msg;
    return code;
}

#define LCK(call)                                                                                    \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            return lfail(b, e_ == cudaErrorMemoryAllocation ? H3D_ERR_NOMEM : H3D_ERR_CUDA,          \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                        \
    } while (0)

void lockstep_free(h3d_lockstep *b) {
    if (b->device >= 0) cudaSetDevice(b->device);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (LockGroup &g : b->groups) {
        batch_tab_free(g.fine);
        batch_tab_free(g.norm);
        for (int l = 0; l < MAXLV; l++) {
            batch_tab_free(g.coarse[l]);
            batch_tab_free(g.xfer[l]);
            batch_tab_free(g.coarsest[l]);
        }
        if (g.join) cudaEventDestroy(g.join);
        if (g.stream && g.stream != b->stream) cudaStreamDestroy(g.stream);
    }
    if (b->d_active) cudaFree(b->d_active);
    if (b->h_active) cudaFreeHost(b->h_active);
    if (b->d_norms) cudaFree(b->d_norms);
    if (b->h_norms) cudaFreeHost(b->h_norms);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
}

// one group's share of the batch V-cycle on stream s
void lockstep_enqueue_group(const h3d_lockstep *b, const LockGroup &g, cudaStream_t s) {
    launch_fine_sweep_batch(g.fine, b->ke, b->d_active, true, g.fine_shape, s);
    for (int l = 1; l < g.lmax; l++) {
        if (g.xfer[l].n) launch_restrict_batch(g.xfer[l], b->d_active, s);
        if (g.coarse[l].n) launch_coarse_sweep_batch(g.coarse[l], b->f32, b->d_active, true, g.coarse_shape[l], s);
        if (g.coarsest[l].n) launch_coarse_apply_batch(g.coarsest[l], b->d_active, b->project, s);
    }
    for (int l = g.lmax - 2; l >= 0; l--) {
        if (!g.xfer[l + 1].n) continue;
        launch_prolong_batch(g.xfer[l + 1], b->d_active, l == 0, s);
        if (l == 0) launch_fine_sweep_batch(g.fine, b->ke, b->d_active, false, g.fine_shape, s);
        else launch_coarse_sweep_batch(g.coarse[l], b->f32, b->d_active, false, g.coarse_shape[l], s);
    }
    launch_pin_deflate_batch(g.fine, b->ke, b->d_active, s);
    launch_norm_finish_batch(g.norm, b->d_active, b->d_norms, s);
}

// the batch V-cycle on b->stream (captured once): the active flags in, the groups
// as parallel branches, the norms out
void lockstep_enqueue(h3d_lockstep *b) {
    cudaStream_t s = b->stream;
    cudaMemcpyAsync(b->d_active, b->h_active, sizeof(int) * b->n, cudaMemcpyHostToDevice, s);
    cudaEventRecord(b->fork, s);
    for (size_t k = 1; k < b->groups.size(); k++) cudaStreamWaitEvent(b->groups[k].stream, b->fork, 0);
    for (const LockGroup &g : b->groups) lockstep_enqueue_group(b, g, g.stream);
    for (size_t k = 1; k < b->groups.size(); k++) {
        cudaEventRecord(b->groups[k].join, b->groups[k].stream);
        cudaStreamWaitEvent(s, b->groups[k].join, 0);
    }
    cudaMemcpyAsync(b->h_norms, b->d_norms, sizeof(double) * NCASE * b->n, cudaMemcpyDeviceToHost, s);
}

int lockstep_build_group(h3d_lockstep *b, LockGroup &grp) {
    std::vector<const Level *> a;
    std::vector<const float *> rho;
    std::vector<double *> part, state;
    std::vector<int> des, nblk;
    auto tab_rc = [&](int rc, const char *what) -> int {
        if (rc == 0) return H3D_OK;
        return lfail(b, rc == -2 ? H3D_ERR_NOMEM : H3D_ERR_ARG, std::string("lockstep table: ") + what);
    };
    for (int i : grp.members) {
        h3d_handle *h = b->hs[i];
        a.push_back(&h->lv[0]);
        rho.push_back(h->rho);
        part.push_back(h->partial);
        state.push_back(h->pin_state);
        des.push_back(i);
        nblk.push_back(fine_residual_blocks(h->lv[0]));
        grp.lmax = std::max(grp.lmax, h->nl);
    }
    const int m = (int)grp.members.size();
    if (int e = tab_rc(fine_batch_create(a.data(), rho.data(), part.data(), state.data(), des.data(), m, false,
                                         &grp.fine),
                       "level 0"))
        return e;
    if (int e = tab_rc(norm_batch_create(part.data(), nblk.data(), des.data(), m, &grp.norm), "norms")) return e;
    for (int l = 1; l < grp.lmax; l++) {
        std::vector<const Level *> F, Cl, S, Z;
        std::vector<int> dx, ds, dz;
        std::vector<const double *> az;
        for (int i : grp.members) {
            h3d_handle *h = b->hs[i];
            if (l >= h->nl) continue;
            F.push_back(&h->lv[l - 1]);
            Cl.push_back(&h->lv[l]);
            dx.push_back(i);
            if (l < h->nl - 1) {
                S.push_back(&h->lv[l]);
                ds.push_back(i);
            } else {
                Z.push_back(&h->lv[l]);
                az.push_back(h->aug);
                dz.push_back(i);
            }
        }
        if (!F.empty())
            if (int e = tab_rc(transfer_batch_create(F.data(), Cl.data(), dx.data(), (int)F.size(), &grp.xfer[l]),
                               "transfers"))
                return e;
        if (!S.empty())
            if (int e = tab_rc(coarse_batch_create(S.data(), ds.data(), (int)S.size(), false, &grp.coarse[l]),
                               "coarse level"))
                return e;
        if (!Z.empty())
            if (int e = tab_rc(coarsest_batch_create(Z.data(), az.data(), dz.data(), (int)Z.size(), &grp.coarsest[l]),
                               "coarsest level"))
                return e;
    }
    return H3D_OK;
}

// the batch V-cycle graph with the groups' current launch shapes
int lockstep_capture(h3d_lockstep *b) {
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t gr = nullptr;
    LCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    lockstep_enqueue(b);
    LCK(cudaStreamEndCapture(b->stream, &gr));
    const cudaError_t e = cudaGraphInstantiate(&b->graph, gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) {
        b->graph = nullptr;
        return lfail(b, H3D_ERR_CUDA, std::string("lockstep graph: ") + cudaGetErrorString(e));
    }
    return H3D_OK;
}

// the launch shape of the sweeps, level by level: both shapes timed with the
// sweeps of every group running together on the groups' streams, as in the batch
// graph, each iterating on its designs' residual fields (which every V-cycle
// rewrites before reading them); shape 1 is kept for all groups where it is at least
// 2 % faster.  The results do not depend on the choice
int lockstep_tune(h3d_lockstep *b) {
    cudaStream_t s = b->stream;
    const int ng = (int)b->groups.size();
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    LCK(cudaEventCreate(&t0));
    LCK(cudaEventCreate(&t1));
    LCK(cudaMemcpyAsync(b->d_active, b->h_active, sizeof(int) * b->n, cudaMemcpyHostToDevice, s));
    int lmax = 0;
    for (const LockGroup &g : b->groups) lmax = std::max(lmax, g.lmax);
    // scratch tables: level 0 and every coarse level of every group
    std::vector<BatchTab> fine(ng);
    std::vector<std::vector<BatchTab>> coarse(ng, std::vector<BatchTab>(MAXLV));
    int rc = H3D_OK;
    for (int k = 0; k < ng && rc == H3D_OK; k++) {
        const LockGroup &g = b->groups[k];
        std::vector<const Level *> a;
        std::vector<const float *> rho;
        std::vector<double *> part, state;
        std::vector<int> des;
        for (int i : g.members) {
            h3d_handle *h = b->hs[i];
            a.push_back(&h->lv[0]);
            rho.push_back(h->rho);
            part.push_back(h->partial);
            state.push_back(h->pin_state);
            des.push_back(i);
        }
        if (fine_batch_create(a.data(), rho.data(), part.data(), state.data(), des.data(), (int)a.size(), true,
                              &fine[k]) != 0)
            rc = lfail(b, H3D_ERR_NOMEM, "lockstep tuning table");
        for (int l = 1; l < g.lmax && rc == H3D_OK; l++) {
            if (!g.coarse[l].n) continue;
            std::vector<const Level *> S;
            std::vector<int> ds;
            for (int i : g.members)
                if (l < b->hs[i]->nl - 1) {
                    S.push_back(&b->hs[i]->lv[l]);
                    ds.push_back(i);
                }
            if (coarse_batch_create(S.data(), ds.data(), (int)S.size(), true, &coarse[k][l]) != 0)
                rc = lfail(b, H3D_ERR_NOMEM, "lockstep tuning table");
        }
    }
    // level l (0: the fine level) of every group together, in the given shape
    auto run = [&](int l, int shape) {
        cudaEventRecord(b->fork, s);
        for (int k = 1; k < ng; k++) cudaStreamWaitEvent(b->groups[k].stream, b->fork, 0);
        for (int k = 0; k < ng; k++) {
            cudaStream_t gs = b->groups[k].stream;
            if (l == 0) launch_fine_sweep_batch(fine[k], b->ke, b->d_active, false, shape, gs);
            else if (coarse[k][l].n) launch_coarse_sweep_batch(coarse[k][l], b->f32, b->d_active, false, shape, gs);
        }
        for (int k = 1; k < ng; k++) {
            cudaEventRecord(b->groups[k].join, b->groups[k].stream);
            cudaStreamWaitEvent(s, b->groups[k].join, 0);
        }
    };
    for (int l = 0; l < lmax - 1 && rc == H3D_OK; l++) {
        bool any = l == 0;
        for (int k = 0; k < ng; k++) any = any || coarse[k][l].n > 0;
        if (!any) continue;
        float best = 0;
        int pick = 0;
        for (int shape = 0; shape < 2 && rc == H3D_OK; shape++) {
            run(l, shape);
            if (cudaEventRecord(t0, s) != cudaSuccess) { rc = lfail(b, H3D_ERR_CUDA, "lockstep tuning"); break; }
            for (int r = 0; r < 10; r++) run(l, shape);
            if (cudaEventRecord(t1, s) != cudaSuccess || cudaEventSynchronize(t1) != cudaSuccess ||
                cudaGetLastError() != cudaSuccess) {
                rc = lfail(b, H3D_ERR_CUDA, "lockstep tuning launch failed");
                break;
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, t0, t1);
            // shape 1 only when clearly faster: the small levels time within the noise
            if (shape == 0) best = ms;
            else if (ms < 0.98f * best) pick = 1;
        }
        for (LockGroup &g : b->groups) {
            if (l == 0) g.fine_shape = pick;
            else g.coarse_shape[l] = pick;
        }
    }
    for (int k = 0; k < ng; k++) {
        batch_tab_free(fine[k]);
        for (BatchTab &t : coarse[k]) batch_tab_free(t);
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return rc;
}

// designs largest first, dealt round-robin to the groups (similar work per branch)
int lockstep_build(h3d_lockstep *b, int ngroups) {
    const int n = b->n;
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return b->hs[x]->lv[0].P.nv > b->hs[y]->lv[0].P.nv; });
    b->groups.resize(ngroups);
    for (int k = 0; k < n; k++) b->groups[k % ngroups].members.push_back(order[k]);
    for (LockGroup &g : b->groups) std::sort(g.members.begin(), g.members.end());
    LCK(cudaMalloc(&b->d_active, sizeof(int) * n));
    LCK(cudaMallocHost(&b->h_active, sizeof(int) * n));
    LCK(cudaMalloc(&b->d_norms, sizeof(double) * NCASE * n));
    LCK(cudaMallocHost(&b->h_norms, sizeof(double) * NCASE * n));
    LCK(cudaMemset(b->d_norms, 0, sizeof(double) * NCASE * n));
    std::memset(b->h_norms, 0, sizeof(double) * NCASE * n);
    for (int i = 0; i < n; i++) b->h_active[i] = 1;
    LCK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    LCK(cudaEventCreate(&b->ev0));
    LCK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    for (size_t k = 0; k < b->groups.size(); k++) {
        LockGroup &g = b->groups[k];
        if (int e = lockstep_build_group(b, g)) return e;
        if (k == 0) {
            g.stream = b->stream;
        } else {
            LCK(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
            LCK(cudaEventCreateWithFlags(&g.join, cudaEventDisableTiming));
        }
    }
    return lockstep_capture(b);
}

// one design of a lockstep solve: SolveRun's FP32 branch with the stale residual
// norms of each cycle read from the batch's host mirror, its other launches on
// the batch stream
struct LockRun {
    h3d_handle *h = nullptr;
    int it = 0, status = H3D_OK, explode_left = 2, maxit = 200;
    double tol = 1e-2, theta = 1e-3;
    double fn[6] = {}, rel[6] = {1, 1, 1, 1, 1, 1};
    bool live = false;

    // before the first batch cycle, on the design's stream: balanced right-hand
    // side, reference norms (to the host mirror), deflation state (SolveRun::begin
    // with a guess, FP32 mode); read_begin takes the norms once the stream drained
    int begin(h3d_handle *hh, double tolerance) {
        h = hh;
        tol = tolerance;
        const Level &L0 = h->lv[0];
        const int nb = norm_blocks(L0.P);
        launch_mean_partial(L0.P, L0.f, h->partial, nb, h->stream);
        launch_remove_mean(L0.P, L0.f, h->partial, nb, h->stream);
        launch_weighted_norm(L0.P, L0.f, h->partial, nb, h->stream);
        launch_norm_finish(h->partial, nb, h->d_small, h->stream);
        CKL();
        CK(cudaMemcpyAsync(h->h_small, h->d_small, sizeof(double) * NCASE, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemsetAsync(h->pin_state + NF, 0, sizeof(double) * NF, h->stream));
        enqueue_pin_init(h);
        CKL();
        return H3D_OK;
    }
    void read_begin() {
        for (int c = 0; c < NCASE; c++) fn[c] = std::sqrt(h->h_small[c]);
        const Level &L0 = h->lv[0];
        const int nmax = std::max(L0.P.n[0], std::max(L0.P.n[1], L0.P.n[2]));
        theta = std::max(1e-3, 1e-5 * nmax);
        live = true;
    }
    int finish(int st, cudaStream_t s) {
        status = st;
        launch_pin_fold(h->lv[0], h->rho, h->ke, h->pin_state, s);
        CK(cudaEventRecord(h->ev1, s));
        live = false;
        return H3D_OK;
    }
    // after a batch cycle; norms: this design's six stale residual norms squared
    int advance(const double *norms, cudaStream_t s) {
        it++;
        bool bad = false, done = true;
        for (int c = 0; c < NCASE; c++) {
            rel[c] = std::sqrt(norms[c]) / (fn[c] + 1e-10);
            if (!(rel[c] <= 10.0)) bad = true;
            if (!(rel[c] <= tol)) done = false;
        }
        if (bad) {  // MG.cpp:140-182: restart from zero once, then give up
            if (--explode_left <= 0) return finish(H3D_DIVERGED, s);
            launch_pin_fold(h->lv[0], h->rho, h->ke, h->pin_state, s);  // restores f
            CK(cudaMemsetAsync(h->lv[0].u, 0, sizeof(float) * field_floats(h->lv[0].P.nv), s));
            CK(cudaMemsetAsync(h->pin_state + NF, 0, sizeof(double) * NF, s));
            enqueue_pin_init(h, s);
            CKL();
        } else if (done) {
            return finish(H3D_OK, s);
        }
        if (it >= maxit) return finish(H3D_NOT_CONVERGED, s);
        return H3D_OK;
    }
};

}  // namespace

extern "C" {

int h3d_lockstep_create(h3d_handle *const *hs, int n, h3d_lockstep **out) {
    return h3d_lockstep_create_groups(hs, n, std::min(n, H3D_LOCKSTEP_DEFAULT_GROUPS), out);
}

int h3d_lockstep_create_groups(h3d_handle *const *hs, int n, int groups, h3d_lockstep **out) {
    if (!out) return H3D_ERR_ARG;
    *out = nullptr;
    if (!hs || n < 1 || n > H3D_LOCKSTEP_MAX) return H3D_ERR_ARG;
    if (groups < 1 || groups > n) return fail(hs[0], H3D_ERR_ARG, "lockstep: groups must be 1..n");
    for (int i = 0; i < n; i++)
        if (!hs[i]) return H3D_ERR_ARG;
    if (int e = distinct_handles(hs, n)) return e;
    h3d_handle *h0 = hs[0];
    for (int i = 0; i < n; i++) {
        h3d_handle *h = hs[i];
        if (h->device != h0->device) return fail(h0, H3D_ERR_ARG, "lockstep: handles on different devices");
        if (h->cfg.precision != H3D_PREC_FP32) return fail(h0, H3D_ERR_ARG, "lockstep: needs H3D_PREC_FP32 handles");
        if (std::memcmp(h->ke.k, h0->ke.k, sizeof(h->ke.k)) != 0)
            return fail(h0, H3D_ERR_ARG, "lockstep: handles with different materials");
        if (h->cfg.stencil_precision != h0->cfg.stencil_precision || h->cfg.coarse_mode != h0->cfg.coarse_mode)
            return fail(h0, H3D_ERR_ARG, "lockstep: different stencil precision or coarse mode");
        for (int l = 1; l < h->nl; l++)
            if (h->lv[l].ratio[0] != 2 || h->lv[l].ratio[1] != 2 || h->lv[l].ratio[2] != 2 || !h->lv[l - 1].P.even)
                return fail(h0, H3D_ERR_ARG, "lockstep: needs ratio-2 coarsening of even levels");
    }
    h3d_lockstep *b = new (std::nothrow) h3d_lockstep();
    if (!b) return H3D_ERR_NOMEM;
    b->hs.assign(hs, hs + n);
    b->n = n;
    b->device = h0->device;
    b->ke = h0->ke;
    b->f32 = h0->cfg.stencil_precision == H3D_STENCIL_FP32;
    b->project = h0->cfg.coarse_mode == H3D_COARSE_PROJECT;
    if (cudaSetDevice(b->device) != cudaSuccess) {
        delete b;
        return fail(h0, H3D_ERR_CUDA, "cudaSetDevice failed");
    }
    if (int e = lockstep_build(b, groups)) {
        fail(h0, e, b->err);
        lockstep_free(b);
        delete b;
        return e;
    }
    *out = b;
    return H3D_OK;
}

int h3d_lockstep_autotune(h3d_lockstep *b) {
    if (!b) return H3D_ERR_ARG;
    LCK(cudaSetDevice(b->device));
    LCK(cudaStreamSynchronize(b->stream));
    if (int e = lockstep_tune(b)) return e;
    return lockstep_capture(b);
}

int h3d_lockstep_set_shapes(h3d_lockstep *b, int fine_shape, int coarse_shape) {
    if (!b) return H3D_ERR_ARG;
    if (fine_shape < 0 || fine_shape > 1 || coarse_shape < 0 || coarse_shape > 1)
        return lfail(b, H3D_ERR_ARG, "lockstep launch shapes are 0 or 1");
    LCK(cudaSetDevice(b->device));
    LCK(cudaStreamSynchronize(b->stream));
    for (LockGroup &g : b->groups) {
        g.fine_shape = fine_shape;
        for (int l = 0; l < MAXLV; l++) g.coarse_shape[l] = coarse_shape;
    }
    return lockstep_capture(b);
}

int h3d_lockstep_destroy(h3d_lockstep *b) {
    if (!b) return H3D_ERR_ARG;
    lockstep_free(b);
    delete b;
    return H3D_OK;
}

const char *h3d_lockstep_last_error(const h3d_lockstep *b) { return b ? b->err.c_str() : "null lockstep batch"; }

int h3d_lockstep_elastic_matrix(h3d_lockstep *b, double tol, double *C, h3d_solve_stats *stats, int *status) {
    if (!b || !C) return H3D_ERR_ARG;
    LCK(cudaSetDevice(b->device));
    const int n = b->n;
    std::vector<LockRun> runs(n);
    std::vector<int> st(n, H3D_OK);
    for (int i = 0; i < n; i++) {
        h3d_handle *h = b->hs[i];
        if (!h->have_stencils) {
            st[i] = fail(h, H3D_ERR_STATE, "no stencils");
            continue;
        }
        st[i] = elastic_prepare(h);
        if (st[i] == H3D_OK) st[i] = runs[i].begin(h, tol);
    }
    // the designs' own streams hold their preparation: drain them before the
    // batch stream takes over
    for (int i = 0; i < n; i++) {
        if (cudaStreamSynchronize(b->hs[i]->stream) != cudaSuccess && st[i] == H3D_OK)
            st[i] = fail(b->hs[i], H3D_ERR_CUDA, "stream synchronisation failed");
        if (st[i] == H3D_OK) runs[i].read_begin();
        else runs[i].live = false;
    }
    LCK(cudaEventRecord(b->ev0, b->stream));
    for (int i = 0; i < n; i++)
        if (runs[i].live) LCK(cudaEventRecord(b->hs[i]->ev0, b->stream));
    for (;;) {
        int nlive = 0;
        for (int i = 0; i < n; i++) {
            b->h_active[i] = runs[i].live ? 1 : 0;
            nlive += b->h_active[i];
        }
        if (!nlive) break;
        LCK(cudaGraphLaunch(b->graph, b->stream));
        LCK(cudaStreamSynchronize(b->stream));
        for (int i = 0; i < n; i++) {
            if (!b->h_active[i]) continue;
            const int e = runs[i].advance(b->h_norms + NCASE * i, b->stream);
            if (e != H3D_OK) {
                st[i] = e;
                runs[i].live = false;
            }
        }
    }
    LCK(cudaStreamSynchronize(b->stream));
    for (int i = 0; i < n; i++) {
        h3d_handle *h = b->hs[i];
        if (st[i] != H3D_OK) continue;
        if (stats) {
            h3d_solve_stats &s1 = stats[i];
            s1.vcycles = runs[i].it;
            s1.refinements = 0;
            s1.status = runs[i].status;
            for (int c = 0; c < NCASE; c++) s1.rel_res[c] = runs[i].rel[c];
            float ms = 0;
            cudaEventElapsedTime(&ms, h->ev0, h->ev1);
            s1.solve_ms = ms;
        }
        st[i] = runs[i].status;
        if (st[i] != H3D_OK && st[i] != H3D_NOT_CONVERGED) {
            fail(h, st[i], "multigrid diverged");
            continue;
        }
        if (int e = elastic_enqueue_energy(h)) st[i] = e;
    }
    int first = H3D_OK;
    for (int i = 0; i < n; i++) {
        h3d_handle *h = b->hs[i];
        if (st[i] == H3D_OK || st[i] == H3D_NOT_CONVERGED) {
            if (cudaStreamSynchronize(h->stream) != cudaSuccess) st[i] = fail(h, H3D_ERR_CUDA, "stream synchronisation failed");
            else if (int e = elastic_read(h, C + 36 * (size_t)i)) st[i] = e;
        }
        if (status) status[i] = st[i];
        if (st[i] != H3D_OK && first == H3D_OK) {
            first = st[i];
            b->err = h->err;
        }
    }
    return first;
}

}  // extern "C"

extern "C" {

int h3d_sensitivity(h3d_handle *h, const float dC[36], float *sens_dev, int pitchT) {
    if (!h || !dC || !sens_dev) return H3D_ERR_ARG;
    CK(cudaSetDevice(h->device));
    const Planes &P = h->lv[0].P;
    if (pitchT < 0) pitchT = P.n[0];
    if (pitchT < P.n[0]) return fail(h, H3D_ERR_ARG, "pitchT smaller than the x resolution");
    CK(cudaMemsetAsync(sens_dev, 0, sizeof(float) * (size_t)pitchT * P.n[1] * P.n[2], h->stream));
    int nsm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
    CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
    if (launch_sensitivity_tc(P, h->chi, h->ke, dC, sens_dev, pitchT, energy_tc_blocks(P, nsm), h->d_flag,
                              h->stream) != 0)
        return fail(h, H3D_ERR_CUDA, "tensor-core energy kernel could not be configured");
    CKL();
    CK(cudaMemcpyAsync(&h->h_small[63], h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (*reinterpret_cast<int *>(&h->h_small[63]))
        return fail(h, H3D_ERR_CUDA, "tensor-core energy kernel: mbarrier wait timed out");
    return H3D_OK;
}

int h3d_penalize(h3d_handle *h, const float *rho_dev, float *rho_phys_dev, int64_t n, float p) {
    if (!h || !rho_dev || !rho_phys_dev || n <= 0) return H3D_ERR_ARG;
    CK(cudaSetDevice(h->device));
    launch_penalize(n, rho_dev, rho_phys_dev, p, 0, h->stream);
    CKL();
    return H3D_OK;
}

int h3d_penalize_backward(h3d_handle *h, const float *rho_dev, float *grad_dev, int64_t n, float p) {
    if (!h || !rho_dev || !grad_dev || n <= 0) return H3D_ERR_ARG;
    CK(cudaSetDevice(h->device));
    launch_penalize(n, rho_dev, grad_dev, p, 1, h->stream);
    CKL();
    return H3D_OK;
}

int h3d_oc_update(h3d_handle *h, const float *sens_dev, float *rho_dev, int64_t n, float volratio, float min_rho,
                  float step_limit, float damp) {
    if (!h || !sens_dev || !rho_dev || n <= 0) return H3D_ERR_ARG;
    CK(cudaSetDevice(h->device));
    if (int e = ensure_tmp(h, (size_t)n)) return e;
    launch_oc(sens_dev, rho_dev, h->tmp, n, volratio, min_rho, step_limit, damp, h->partial, h->stream);
    CKL();
    return H3D_OK;
}

int h3d_oc_filter(h3d_handle *h, float *sens_dev, const float *rho_dev, const int reso[3], int pitchT, float radius,
                  int periodic) {
    if (!h || !sens_dev || !rho_dev || !reso) return H3D_ERR_ARG;
    CK(cudaSetDevice(h->device));
    if (pitchT < 0) pitchT = reso[0];
    const size_t n = (size_t)pitchT * reso[1] * reso[2];
    if (int e = ensure_tmp(h, n)) return e;
    CK(cudaMemsetAsync(h->tmp, 0, sizeof(float) * n, h->stream));
    launch_filter(reso, pitchT, sens_dev, rho_dev, h->tmp, radius, periodic, h->stream);
    CKL();
    CK(cudaMemcpyAsync(sens_dev, h->tmp, sizeof(float) * n, cudaMemcpyDeviceToDevice, h->stream));
    return H3D_OK;
}

int h3d_symmetrize(h3d_handle *h, float *field_dev, const int reso[3], int sym) {
    if (!h || !field_dev || !reso || sym < 0 || sym > 2) return H3D_ERR_ARG;
    if (sym > 0 && (reso[0] != reso[1] || reso[1] != reso[2]))
        return fail(h, H3D_ERR_ARG, "reflect6 and rotate3 need a cubic grid");
    CK(cudaSetDevice(h->device));
    launch_symmetrize(reso, field_dev, sym, h->stream);
    CKL();
    return H3D_OK;
}

int h3d_init_density_trig(h3d_handle *h, float *rho_dev, const int reso[3], int n_period, const float *coeff,
                          int ncoeff, int centered, float volratio, int sym) {
    if (!h || !rho_dev || !reso || !coeff) return H3D_ERR_ARG;
    if (n_period < 1 || n_period > 50) return fail(h, H3D_ERR_ARG, "n_period outside 1..50");
    const int nbasis = 6 * n_period + 36 * n_period * n_period;
    if (ncoeff != nbasis + (centered ? 4 : 0))
        return fail(h, H3D_ERR_ARG, "coefficient count must be 6 P + 36 P^2 (+ 4 when centred)");
    if (!(volratio > 0 && volratio <= 1)) return fail(h, H3D_ERR_ARG, "volratio outside (0, 1]");
    if (sym < -1 || sym > 2) return fail(h, H3D_ERR_ARG, "sym must be -1, 0, 1 or 2");
    if (sym > 0 && (reso[0] != reso[1] || reso[1] != reso[2]))
        return fail(h, H3D_ERR_ARG, "reflect6 and rotate3 need a cubic grid");
    for (int d = 0; d < 3; d++)
        if (reso[d] < 2) return fail(h, H3D_ERR_ARG, "each axis needs at least two cells");
    // rotation of the unit quaternion (w, x, y, z) of the four extra coefficients
    float rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (centered) {
        double q[4] = {coeff[nbasis], coeff[nbasis + 1], coeff[nbasis + 2], coeff[nbasis + 3]};
        const double qn = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        if (!(qn > 0)) return fail(h, H3D_ERR_ARG, "zero quaternion");
        for (double &v : q) v /= qn;
        const double w = q[0], x = q[1], y = q[2], z = q[3];
        const double R[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - w * z),     2 * (x * z + w * y),
                             2 * (x * y + w * z),     1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                             2 * (x * z - w * y),     2 * (y * z + w * x),     1 - 2 * (x * x + y * y)};
        for (int i = 0; i < 9; i++) rot[i] = (float)R[i];
    }
    CK(cudaSetDevice(h->device));
    float *dcoeff = nullptr;
    CK(cudaMalloc(&dcoeff, sizeof(float) * ncoeff));
    cudaError_t e = cudaMemcpyAsync(dcoeff, coeff, sizeof(float) * ncoeff, cudaMemcpyHostToDevice, h->stream);
    int rc = H3D_OK;
    if (e != cudaSuccess) rc = fail(h, H3D_ERR_CUDA, cudaGetErrorString(e));
    else if (launch_trig_init(reso, n_period, dcoeff, centered, rot, volratio, sym, rho_dev, h->partial, h->stream) != 0)
        rc = fail(h, H3D_ERR_CUDA, "trig-basis kernel could not be configured");
    e = cudaStreamSynchronize(h->stream);
    cudaFree(dcoeff);
    if (rc == H3D_OK && e != cudaSuccess) rc = fail(h, H3D_ERR_CUDA, cudaGetErrorString(e));
    if (rc == H3D_OK) {
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(h, H3D_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    }
    return rc;
}

int h3d_conv_radial(h3d_handle *h, const float *in_dev, float *out_dev, const int reso[3], float radius, int periodic,
                    int adjoint) {
    if (!h || !in_dev || !out_dev || !reso) return H3D_ERR_ARG;
    if (in_dev == out_dev) return fail(h, H3D_ERR_ARG, "input and output must not overlap");
    if (!(radius > 0) || radius > 32) return fail(h, H3D_ERR_ARG, "radius outside (0, 32]");
    for (int d = 0; d < 3; d++)
        if (reso[d] < 1) return fail(h, H3D_ERR_ARG, "empty grid");
    const int hw = (int)(radius + 0.5f);
    if (periodic && (reso[0] <= 2 * hw || reso[1] <= 2 * hw || reso[2] <= 2 * hw))
        return fail(h, H3D_ERR_ARG, "periodic window wider than the grid");
    CK(cudaSetDevice(h->device));
    const size_t ne = (size_t)reso[0] * reso[1] * reso[2];
    if (int e = ensure_tmp(h, ne)) return e;
    launch_conv_radial(reso, in_dev, out_dev, h->tmp, radius, periodic, adjoint, h->stream);
    CKL();
    return H3D_OK;
}

int h3d_design_step(h3d_handle *h, const float dC[36], float *rho_dev, float *sens_dev, const h3d_design_params *prm) {
    if (!h || !dC || !rho_dev || !sens_dev || !prm) return H3D_ERR_ARG;
    const Planes &P = h->lv[0].P;
    const int *n = P.n;
    if (prm->sym < -1 || prm->sym > 2) return fail(h, H3D_ERR_ARG, "sym must be -1, 0, 1 or 2");
    if (prm->sym > 0 && (n[0] != n[1] || n[1] != n[2]))
        return fail(h, H3D_ERR_ARG, "reflect6 and rotate3 need a cubic grid");
    if (!(prm->volratio > 0 && prm->volratio <= 1)) return fail(h, H3D_ERR_ARG, "volratio outside (0, 1]");
    CK(cudaSetDevice(h->device));
    const long long ne = (long long)n[0] * n[1] * n[2];
    if (int e = ensure_tmp(h, (size_t)ne)) return e;
    if (!h->d_dcw) CK(cudaMalloc(&h->d_dcw, sizeof(float) * 32));
    if (!h->h_dcw) CK(cudaMallocHost(&h->h_dcw, sizeof(float) * 32));
    if (h->dgraph && (h->dkey_rho != rho_dev || h->dkey_sens != sens_dev ||
                      std::memcmp(&h->dkey, prm, sizeof(h3d_design_params)) != 0)) {
        cudaGraphExecDestroy(h->dgraph);
        h->dgraph = nullptr;
    }
    if (!h->dgraph) {
        if (configure_energy_tc() != 0) return fail(h, H3D_ERR_CUDA, "tensor-core energy kernel could not be configured");
        int nsm = 0;
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
        cudaStream_t s = h->stream;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        cudaMemcpyAsync(h->d_dcw, h->h_dcw, sizeof(float) * 21, cudaMemcpyHostToDevice, s);
        cudaMemsetAsync(h->d_flag, 0, sizeof(int), s);
        cudaMemsetAsync(sens_dev, 0, sizeof(float) * ne, s);
        launch_sensitivity_tc_dev(P, h->chi, h->ke, h->d_dcw, sens_dev, n[0], energy_tc_blocks(P, nsm), h->d_flag, s);
        launch_penalize(ne, rho_dev, sens_dev, prm->penal, 1, s);
        if (prm->sym >= 0) launch_symmetrize(n, sens_dev, prm->sym, s);
        if (prm->filter_radius > 0) {
            cudaMemsetAsync(h->tmp, 0, sizeof(float) * ne, s);
            launch_filter(n, n[0], sens_dev, rho_dev, h->tmp, prm->filter_radius, prm->filter_periodic, s);
            cudaMemcpyAsync(sens_dev, h->tmp, sizeof(float) * ne, cudaMemcpyDeviceToDevice, s);
        }
        launch_oc(sens_dev, rho_dev, h->tmp, ne, prm->volratio, prm->min_rho, prm->step_limit, prm->damp, h->partial,
                  s);
        if (prm->sym >= 0) launch_symmetrize(n, rho_dev, prm->sym, s);
        cudaMemcpyAsync(&h->h_small[63], h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s);
        CK(cudaStreamEndCapture(s, &g));
        cudaError_t e = cudaGraphInstantiate(&h->dgraph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            h->dgraph = nullptr;
            return fail(h, H3D_ERR_CUDA, std::string("graph: ") + cudaGetErrorString(e));
        }
        h->dkey = *prm;
        h->dkey_rho = rho_dev;
        h->dkey_sens = sens_dev;
    }
    sensitivity_weights(P, dC, h->h_dcw);
    CK(cudaGraphLaunch(h->dgraph, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (*reinterpret_cast<int *>(&h->h_small[63]))
        return fail(h, H3D_ERR_CUDA, "tensor-core energy kernel: mbarrier wait timed out");
    return H3D_OK;
}

int h3d_get_field(h3d_handle *h, int level, int field, float *host) {
    if (int e = check_level(h, level)) return e;
    if (!host) return H3D_ERR_ARG;
    CK(cudaSetDevice(h->device));
    const Level &L = h->lv[level];
    if (field == H3D_FIELD_STENCIL) {
        if (level == 0) return fail(h, H3D_ERR_ARG, "level 0 has no stored stencil");
        if (int e = ensure_tmp(h, (size_t)243 * L.P.nv)) return e;
        launch_stencil_to_lex(L, h->tmp, h->stream);
        CKL();
        CK(cudaMemcpyAsync(host, h->tmp, sizeof(float) * 243 * L.P.nv, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        return H3D_OK;
    }
    const size_t n18 = (size_t)NF * L.P.nv, nf = (size_t)field_floats(L.P.nv);
    if (field == H3D_FIELD_CHI || field == H3D_FIELD_SOLUTION) {
        const double *src = level != 0 ? nullptr : field == H3D_FIELD_CHI ? h->chi : h->u64;
        if (!src) return fail(h, H3D_ERR_ARG, "no such FP64 field on this level / precision mode");
        if (int e = ensure_tmp(h, n18 + nf)) return e;
        launch_convert_field(L.P.nv, src, h->tmp + n18, h->stream);
        launch_field_to_lex(L.P, h->tmp + n18, h->tmp, h->stream);
    } else {
        const float *src = field == H3D_FIELD_U ? L.u : field == H3D_FIELD_F ? L.f : field == H3D_FIELD_R ? L.r : nullptr;
        if (!src) return fail(h, H3D_ERR_ARG, "unknown field");
        if (int e = ensure_tmp(h, n18)) return e;
        launch_field_to_lex(L.P, src, h->tmp, h->stream);
    }
    CKL();
    CK(cudaMemcpyAsync(host, h->tmp, sizeof(float) * n18, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return H3D_OK;
}

int h3d_set_field(h3d_handle *h, int level, int field, const float *host) {
    if (int e = check_level(h, level)) return e;
    if (!host) return H3D_ERR_ARG;
    CK(cudaSetDevice(h->device));
    Level &L = h->lv[level];
    if (field == H3D_FIELD_STENCIL) {
        if (level == 0) return fail(h, H3D_ERR_ARG, "level 0 has no stored stencil");
        if (int e = ensure_tmp(h, (size_t)243 * L.P.nv)) return e;
        CK(cudaMemcpyAsync(h->tmp, host, sizeof(float) * 243 * L.P.nv, cudaMemcpyHostToDevice, h->stream));
        launch_stencil_from_lex(L, h->tmp, h->stream);
        CKL();
        CK(cudaStreamSynchronize(h->stream));
        return H3D_OK;
    }
    const size_t n18 = (size_t)NF * L.P.nv, nf = (size_t)field_floats(L.P.nv);
    if (field == H3D_FIELD_CHI || field == H3D_FIELD_SOLUTION) {
        double *dst = level != 0 ? nullptr : field == H3D_FIELD_CHI ? h->chi : h->u64;
        if (!dst) return fail(h, H3D_ERR_ARG, "no such FP64 field on this level / precision mode");
        if (field == H3D_FIELD_CHI) h->chi_zero = false;
        else h->u64_zero = false;
        if (int e = ensure_tmp(h, n18 + nf)) return e;
        CK(cudaMemcpyAsync(h->tmp, host, sizeof(float) * n18, cudaMemcpyHostToDevice, h->stream));
        launch_field_from_lex(L.P, h->tmp, h->tmp + n18, h->stream);
        launch_convert_field(L.P.nv, h->tmp + n18, dst, h->stream);
    } else {
        float *dst = field == H3D_FIELD_U ? L.u : field == H3D_FIELD_F ? L.f : field == H3D_FIELD_R ? L.r : nullptr;
        if (!dst) return fail(h, H3D_ERR_ARG, "unknown field");
        if (int e = ensure_tmp(h, n18)) return e;
        CK(cudaMemcpyAsync(h->tmp, host, sizeof(float) * n18, cudaMemcpyHostToDevice, h->stream));
        launch_field_from_lex(L.P, h->tmp, dst, h->stream);
        // in the refined mode the solve reads its right-hand side from f0
        if (field == H3D_FIELD_F && level == 0 && h->refine())
            CK(cudaMemcpyAsync(h->f0, dst, sizeof(float) * nf, cudaMemcpyDeviceToDevice, h->stream));
    }
    CKL();
    CK(cudaStreamSynchronize(h->stream));
    return H3D_OK;
}

int h3d_warm_start_learned(h3d_handle *h, h3d_warmnet *net) {
    if (!h || !net) return H3D_ERR_ARG;
    const Level &L = h->lv[0];
    const int N = L.P.n[0], R = warmnet_reso(net);
    if (L.P.n[1] != N || L.P.n[2] != N || N % R != 0)
        return fail(h, H3D_ERR_ARG, "learned warm start needs a cubic grid whose size is a multiple of the network's");
    if (warmnet_device(net) != h->device) return fail(h, H3D_ERR_ARG, "network and handle on different devices");
    if (!h->rho) return fail(h, H3D_ERR_STATE, "no density");
    CK(cudaSetDevice(h->device));
    if (int e = ensure_tmp(h, (size_t)R * R * R)) return e;
    launch_warmnet_density_pool(h->rho, N, R, h->tmp, h->stream);
    const float *y = nullptr;
    if (warmnet_forward_on(net, h->tmp, h->stream, &y) != H3D_OK) return fail(h, H3D_ERR_CUDA, "network forward failed");
    launch_warmnet_to_chi(L.P, y, R, h->chi, h->stream);
    h->chi_zero = false;
    CKL();
    CK(cudaStreamSynchronize(h->stream));
    return H3D_OK;
}

// h3d_field_norms for the FP32 level-0 fields for callers that must not have
// device memory allocated (or the handle's scratch touched) during the call: the
// reduction runs in a fixed file-scope device array (k_static_norm.cu).  Calls on
// one device share that array, so calls that overlap in time race; the first call
// on a device looks up the array's address and should precede any stream capture.
int h3d_field_norms_static(h3d_handle *h, int field, double out[6]) {
    if (!h || !out) return H3D_ERR_ARG;
    CK(cudaSetDevice(h->device));
    const Level &L = h->lv[0];
    const float *v = field == H3D_FIELD_U ? L.u : field == H3D_FIELD_F ? L.f : field == H3D_FIELD_R ? L.r : nullptr;
    if (!v) return fail(h, H3D_ERR_ARG, "static-scratch norms take the FP32 fields U, F, R");
    const int nb = norm_blocks(L.P);
    if (nb > STATIC_NORM_MAX_BLOCKS)
        return fail(h, H3D_ERR_ARG, "field needs more norm blocks than the static scratch holds (2048)");
    const double *tot = static_norm_totals(h->device);
    if (!tot) return fail(h, H3D_ERR_CUDA, "cudaGetSymbolAddress of the static norm scratch failed");
    const int rc = launch_weighted_norm_static(h->device, L.P, v, nb, h->stream);
    if (rc == -1) return fail(h, H3D_ERR_ARG, "norm block count outside 1..2048 for the static scratch");
    if (rc != 0) return fail(h, H3D_ERR_CUDA, "cudaGetSymbolAddress of the static norm scratch failed");
    CKL();
    double sums[NCASE];
    CK(cudaMemcpyAsync(sums, tot, sizeof(double) * NCASE, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int c = 0; c < NCASE; c++) out[c] = std::sqrt(sums[c]);
    return H3D_OK;
}

}  // extern "C"
