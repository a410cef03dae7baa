// h3d_internal.cuh -- shared device layout and kernel launch declarations.
//
// Layout in HBM (every level):
//   A vertex field holds the six load cases and three components as 18 planes
//   (q = 3c + m for case c, component m), interleaved in blocks of 128
//   vertices: value(q, v) = field[fidx(q, v)] (FP32 and FP64 fields alike).
//   Vertices are ordered by Gauss-Seidel colour, then lexicographically inside
//   the colour: a vertex (x,y,z) has colour k = ((x+1)&1) | ((y+1)&1)<<1 |
//   ((z+1)&1)<<2 (the reference's padded-position parity, grid.cu:143-200) and
//   index base[k] + (x>>1) + pn[k][0]*((y>>1) + pn[k][1]*(z>>1)).  A colour
//   sweep therefore reads and writes contiguous runs, and the 26 neighbours of a
//   vertex sit in the other colour planes at unit-stride offsets.
//   Coarse stencils: 243 FP16 entries per vertex (27 neighbours x 3x3) packed
//   eight to a uint4 chunk, chunk-major: st[q * nv + v], q = 0..30; or, with
//   FP32 stencil storage, four to a chunk, q = 0..60.
//   Density: float, lexicographic cells (the fine level only).
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace h3d {

constexpr int NCASE = 6;
constexpr int NF = 18;          // floats per vertex (6 cases x 3 components)
constexpr int NCHUNK = 31;      // uint4 chunks per stencil (243 halves -> 248)
constexpr int NCHUNK32 = 61;    // the same with FP32 entries (243 floats -> 244)
constexpr float RHO_PENAL_MIN = 1e-9f;  // grid.h:425

// Vertex fields (u, f, r of every level in FP32; the refined solution and the
// stored solutions chi in FP64): the 18 planes interleaved in blocks of FVB
// vertices, value(plane q, vertex v) at fidx(q, v); the planes a thread reads for
// one vertex are then immediate offsets from one address.  A field holds
// field_floats(nv) elements (nv rounded up to a multiple of FVB).
constexpr int FVB = 128;
static_assert(FVB == 128, "fidx shifts by log2(FVB) = 7");
__host__ __device__ inline long long fidx(int q, long long v) {
    return ((v >> 7) * NF + q) * FVB + (v & (FVB - 1));
}
__host__ __device__ inline long long field_floats(long long nv) { return ((nv + FVB - 1) / FVB) * FVB * NF; }

struct Planes {
    int n[3];        // vertices (= cells) per axis
    int pn[8][3];    // plane dims of each colour
    long long base[8];
    long long nv;
    int even;        // all axes even: pn uniform, base[k] = k * nv / 8
};

__host__ __device__ inline int color_of(int x, int y, int z) {
    return ((x + 1) & 1) | (((y + 1) & 1) << 1) | (((z + 1) & 1) << 2);
}

__host__ __device__ inline long long vidx(const Planes &P, int x, int y, int z) {
    int k = color_of(x, y, z);
    return P.base[k] + (x >> 1) + (long long)P.pn[k][0] * ((y >> 1) + (long long)P.pn[k][1] * (z >> 1));
}

// inverse of vidx for the vertex with plane offset p in colour k
// unsigned 32-bit division by a divisor fixed at launch, as a multiply-high, an
// add and a shift (Granlund and Montgomery's round-up method with the 33-bit
// multiplier 2^32 + m, l = ceil(log2 d)); exact for every 32-bit dividend
struct FastDiv {
    unsigned d = 1, m = 1;
    int l = 0;
    FastDiv() = default;
    __host__ explicit FastDiv(unsigned div) : d(div) {
        l = 0;
        while (l < 32 && (1ull << l) < div) ++l;
        m = (unsigned)((((1ull << 32) * ((1ull << l) - div)) / div) + 1);
    }
    __device__ __forceinline__ unsigned div(unsigned n) const {
        return (unsigned)(((unsigned long long)__umulhi(m, n) + n) >> l);
    }
};

// position of index p (< 2^32) of colour plane k
__host__ __device__ inline void vpos(const Planes &P, int k, long long p, int &x, int &y, int &z) {
    const unsigned q = (unsigned)p, a = (unsigned)P.pn[k][0], b = (unsigned)P.pn[k][1];
    const unsigned t = q / a;
    const int i = (int)(q - t * a);
    const int l = (int)(t / b);
    const int j = (int)(t - (unsigned)l * b);
    x = 2 * i + ((k & 1) ^ 1);
    y = 2 * j + (((k >> 1) & 1) ^ 1);
    z = 2 * l + (((k >> 2) & 1) ^ 1);
}

__host__ __device__ inline int wrap(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

#ifdef __CUDACC__
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// block-reduce N per-thread values into partial[blk*N + i] in a fixed order;
// every thread of the block must call it
template <int N>
__device__ __forceinline__ void block_reduce(const double *s, double *partial, long long blk) {
    __shared__ double sm[N][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int c = 0; c < N; ++c) {
        double v = warp_sum(s[c]);
        if (lane == 0) sm[c][wid] = v;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int c = 0; c < N; ++c) {
            double v = lane < nw ? sm[c][lane] : 0.0;
            v = warp_sum(v);
            if (lane == 0) partial[blk * N + c] = v;
        }
    }
}

// multiplicity of a unique vertex in the reference's padded periodic storage
// (positions 0, 1 and n-1 are stored twice per axis, grid.cpp:155-198)
__device__ __forceinline__ int axis_mult(int x, int n) { return (x == 0 || x == 1 || x == n - 1) ? 2 : 1; }

__device__ __forceinline__ int color_of_index(const Planes &P, long long v) {
    int k = 0;
#pragma unroll
    for (int q = 1; q < 8; ++q) k += (v >= P.base[q]) ? 1 : 0;
    return k;
}
#endif

// ---- lockstep batches of designs (h3d_batch_*): one launch per step over a level
// of several designs.  Design slot i of a batched launch owns its CTAs
// [start[i], start[i+1]); tables live in device memory, built once per batch.
constexpr int BATCH_MAX = 64;  // designs per batch
struct BatchSlices {
    int n;
    unsigned start[BATCH_MAX + 1];
};
#ifdef __CUDACC__
// the slot whose slice holds CTA b (the last slot starting at or before b, so
// empty slices are skipped)
__device__ __forceinline__ int batch_slice(const BatchSlices &s, unsigned b) {
    int lo = 0, hi = __ldg(&s.n) - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&s.start[mid]) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
// a design's launch arguments copied to shared memory by the CTA (argument structs
// with default member initialisers cannot be __shared__ objects themselves); every
// thread of the CTA must call it
template <typename T>
__device__ __forceinline__ const T &stage_args(const T &src, unsigned *buf) {
    static_assert(sizeof(T) % 4 == 0, "copied as 32-bit words");
    const unsigned *w = reinterpret_cast<const unsigned *>(&src);
    for (int i = threadIdx.x; i < (int)(sizeof(T) / 4); i += blockDim.x) buf[i] = __ldg(w + i);
    __syncthreads();
    return *reinterpret_cast<const T *>(buf);
}
#endif
// host view of one device table: its address, slot count and launch sizes
struct BatchTab {
    void *dev = nullptr;
    int n = 0;
    unsigned grid[4] = {0, 0, 0, 0};
    size_t smem = 0;
};
inline void batch_tab_free(BatchTab &t) {
    if (t.dev) cudaFree(t.dev);
    t = BatchTab();
}

struct KeMat { float k[576]; };        // element matrix, row-major, FP32
struct KeMat64 { double k[576]; };     // the same in FP64 (exact refinement residual)
struct RhsTab { float g[NCASE][24]; }; // Ke * chi0_c for the six unit strains

struct Level {
    Planes P;
    int ratio[3];          // coarsening ratio from the finer level (0 on level 0)
    float *u = nullptr, *f = nullptr, *r = nullptr;
    uint4 *st = nullptr;   // coarse levels
    bool st32 = false;     // FP32 stencil entries (FP16 otherwise)
    // launch shapes of the level's sweep and residual (see the launchers); set by
    // the autotuner, results do not depend on them
    int gs_shape = 0, res_shape = 0;
};

#ifdef __CUDACC__
// coarse-stencil storage: entry e of vertex v in chunk e / PER, slot e % PER
template <bool F32>
struct StencilStore;
template <>
struct StencilStore<false> {
    static constexpr int PER = 8, CHUNKS = NCHUNK;
    __device__ static float get(const uint4 *st, long long nv, long long v, int e) {
        return __half2float(reinterpret_cast<const __half *>(st + (long long)(e >> 3) * nv + v)[e & 7]);
    }
    __device__ static void put(uint4 *st, long long nv, long long v, int e, float x) {
        reinterpret_cast<__half *>(st + (long long)(e >> 3) * nv + v)[e & 7] = __float2half_rn(x);
    }
    __device__ static void putd(uint4 *st, long long nv, long long v, int e, double x) {
        reinterpret_cast<__half *>(st + (long long)(e >> 3) * nv + v)[e & 7] = __double2half(x);
    }
    __device__ __forceinline__ static void unpack(const uint4 &c, float *o) {
        const __half2 *h = reinterpret_cast<const __half2 *>(&c);
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const float2 q = __half22float2(h[t]);
            o[2 * t] = q.x;
            o[2 * t + 1] = q.y;
        }
    }
};
template <>
struct StencilStore<true> {
    static constexpr int PER = 4, CHUNKS = NCHUNK32;
    __device__ static float get(const uint4 *st, long long nv, long long v, int e) {
        return reinterpret_cast<const float *>(st + (long long)(e >> 2) * nv + v)[e & 3];
    }
    __device__ static void put(uint4 *st, long long nv, long long v, int e, float x) {
        reinterpret_cast<float *>(st + (long long)(e >> 2) * nv + v)[e & 3] = x;
    }
    __device__ static void putd(uint4 *st, long long nv, long long v, int e, double x) {
        reinterpret_cast<float *>(st + (long long)(e >> 2) * nv + v)[e & 3] = (float)x;
    }
    __device__ __forceinline__ static void unpack(const uint4 &c, float *o) {
        o[0] = __uint_as_float(c.x);
        o[1] = __uint_as_float(c.y);
        o[2] = __uint_as_float(c.z);
        o[3] = __uint_as_float(c.w);
    }
};
#endif

// ---- launch wrappers (kernels in the .cu files) --------------------------
// fine level (k_fine.cu)
void launch_fine_gs(const Level &L, const float *rho, const KeMat &ke, float w, cudaStream_t s);
// a colour sweep followed by the level-0 residual and its norm partials (the last
// colour's launch computes its own vertices' residual)
void launch_fine_gs_residual(const Level &L, const float *rho, const KeMat &ke, float w, double *norm_partial,
                             cudaStream_t s);
void launch_fine_residual(const Level &L, const float *rho, const KeMat &ke, double *norm_partial,
                          int nblk_norm, cudaStream_t s);
// number of per-block norm partials launch_fine_residual writes
int fine_residual_blocks(const Level &L);
void launch_rhs(const Level &L, const float *rho, const RhsTab &g, float *f, cudaStream_t s);
// r = f - K u with u in FP64, the operator in difference form (refined precision)
void launch_fine_residual64(const Level &L, const float *rho, const KeMat &ke, const KeMat64 &ke64, const float *f,
                            const double *u64,
                            float *r, bool exact, cudaStream_t s);
// u64 += e + T over the level-0 vertices but the pinned origin
void launch_update64(const Level &L, double *u64, const float *e, const double *T, cudaStream_t s);
// rigid-translation deflation of the pinned level-0 problem (k_fine.cu); state is
// 36 doubles: F (sum of f over the vertices but the origin) and the pending shift T
void launch_pin_deflate(const Level &L, const float *rho, const KeMat &ke, double *state, cudaStream_t s);
// state from the 18 plane sums of level-0 f: F = sums - f(origin), T = 0
void launch_pin_init(const Level &L, const double *sums, double *state, cudaStream_t s);
// f = f0 - K 0 on level 0 (f0 with the pinned origin's entries 0)
void launch_rhs_at_zero(const Level &L, const float *f0, float *f, cudaStream_t s);
// FP32 solutions: u += T (but the origin), f restored near the origin, T = 0
void launch_pin_fold(const Level &L, const float *rho, const KeMat &ke, double *state, cudaStream_t s);
// FP32 field of nv vertices <-> FP64 field
void launch_convert_field(long long nv, const float *src, double *dst, cudaStream_t s);
void launch_convert_field(long long nv, const double *src, float *dst, cudaStream_t s);
void launch_remove_mean64(const Planes &P, double *v, double *partial, int nblk, cudaStream_t s);
// coarse levels and transfers (k_coarse.cu)
void launch_coarse_gs(const Level &L, float w, cudaStream_t s);
void launch_coarse_residual(const Level &L, cudaStream_t s);
// a coarse colour sweep followed by the level's residual (the last colour's launch
// computes its own vertices' residual)
void launch_coarse_gs_residual(const Level &L, float w, cudaStream_t s);
void launch_restrict(const Level &F, const Level &C, cudaStream_t s);
void launch_prolong(const Level &F, const Level &C, int is_root, cudaStream_t s);
void launch_weighted_norm(const Planes &P, const float *v, double *partial, int nblk, cudaStream_t s);
int norm_blocks(const Planes &P);
// sums nblk x 6 partials into out6; above NORM_FINISH_DIRECT blocks it runs in two
// stages and needs NORM_FINISH_CHUNKS x 6 doubles of scratch behind the partials
constexpr int NORM_FINISH_DIRECT = 4096;
constexpr int NORM_FINISH_CHUNKS = 592;
void launch_norm_finish(const double *partial, int nblk, double *out6, cudaStream_t s);
void launch_mean_partial(const Planes &P, const float *v, double *partial, int nblk, cudaStream_t s);
void launch_remove_mean(const Planes &P, float *v, const double *partial, int nblk, cudaStream_t s);
void launch_sum18_finish(const double *partial, int nblk, double *out, cudaStream_t s);
// Galerkin and coarsest solve (k_galerkin.cu)
void launch_galerkin_l1(const Level &F, const Level &C, const float *rho, const float *q, int nsub,
                        cudaStream_t s);
void launch_dirichlet_patch(const Level &F, const Level &C, const float *rho, const double *ked, int pin_identity,
                            cudaStream_t s);
void launch_galerkin(const Level &F, const Level &C, cudaStream_t s);
void launch_coarse_assemble(const Level &C, double *aug, cudaStream_t s);
// aug must hold gauss_jordan_doubles(n) doubles: the [n][2n] matrix and the
// elimination scratch behind it
size_t gauss_jordan_doubles(int n);
void launch_gauss_jordan(double *aug, int n, int *flag, cudaStream_t s);
void launch_coarse_apply(const Level &C, const double *aug, int project, cudaStream_t s);
// the V-cycle from the restriction into level `first` to the post-smoothing of
// that level in one cooperative launch of nblk CTAs (k_coarse.cu); bar: two
// unsigned of barrier state, *flag set if a grid barrier's wait ran out; -1 if the
// levels do not fit (vcycle_bottom_fits), -2 if the launch failed
int launch_vcycle_bottom(const Level *lv, int first, int nl, const double *aug, int project, unsigned *bar, int *flag,
                         int nblk, cudaStream_t s);
int vcycle_bottom_blocks(int num_sms, int ndof, bool f32);
bool vcycle_bottom_fits(const Level *lv, int first, int nl);
// level-0 residual on the tensor cores (k_fine_tc.cu): element products Ke U with
// TF32 hi + lo operands and FP32 accumulation; a persistent grid of
// fine_residual_tc_blocks CTAs writing one row of six norm partials each (partial
// may be null); *flag is set if an mbarrier wait timed out.
// configure_fine_residual_tc (once per device, before any launch or stream
// capture) returns -1 when the kernel's shared memory cannot be granted
int configure_fine_residual_tc();
int fine_residual_tc_blocks(const Planes &P, int num_sms);
int launch_fine_residual_tc(const Level &L, const float *rho, const KeMat &ke, double *partial, int nblk,
                            int *flag, cudaStream_t s);
// homogenized tensor and sensitivities on the tensor cores (k_homog_tc.cu):
// a persistent grid of energy_tc_blocks CTAs; *flag is set if an mbarrier wait
// timed out; the launchers return -1 when the kernel cannot be configured
int energy_tc_blocks(const Planes &P, int num_sms);
int launch_elastic_tc(const Planes &P, const double *chi, const float *rho, const KeMat &ke, double *partial,
                      int nblk, int *flag, cudaStream_t s);
int launch_sensitivity_tc(const Planes &P, const double *chi, const KeMat &ke, const float *dc36, float *sens,
                          int pitch, int nblk, int *flag, cudaStream_t s);
void launch_elastic_finish(const double *partial, int nblk, double *out21, cudaStream_t s);
// the same sensitivity with its 21 weights (sensitivity_weights) read from device
// memory at run time, for captured graphs; configure_energy_tc first (outside any
// capture), -1 if the kernels cannot be configured
void sensitivity_weights(const Planes &P, const float *dc36, float w21[21]);
int configure_energy_tc();
void launch_sensitivity_tc_dev(const Planes &P, const double *chi, const KeMat &ke, const float *dcw, float *sens,
                               int pitch, int nblk, int *flag, cudaStream_t s);
// design (k_design.cu)
void launch_density_in(const int n[3], const float *src, int pitch, float *dst, cudaStream_t s);
void launch_penalize(long long n, const float *rho, float *out, float p, int backward, cudaStream_t s);
void launch_oc(const float *sens, float *rho, float *rho_new, long long n, float vol, float minrho, float step,
               float damp, double *scratch, cudaStream_t s);
void launch_filter(const int n[3], int pitch, const float *sens, const float *rho, float *out, float radius,
                   int periodic, cudaStream_t s);
void launch_symmetrize(const int n[3], float *v, int sym, cudaStream_t s);
// radial Spline4 convolution of the expression layer (k_design.cu): forward out =
// conv(in) with ws = the in-grid weight sums, or adjoint out = conv^T(in) (ws is
// recomputed); ws holds nx ny nz floats
void launch_conv_radial(const int n[3], const float *in, float *out, float *ws, float radius, int periodic,
                        int adjoint, cudaStream_t s);
// the reference's trig-basis initial density (randTri): basis sum with P periods,
// symmetrised (sym >= 0), level-set mapped to volume vol; scratch holds 4 + 1184
// doubles; -1 if the kernel's shared memory (6 P x 64 floats) cannot be granted
int launch_trig_init(const int n[3], int P, const float *coeff_dev, int centered, const float rot[9], float vol, int sym,
                     float *rho, double *scratch, cudaStream_t s);
// weighted norms with file-scope device scratch (k_static_norm.cu), on the
// current device: the launcher returns -1 when nblk exceeds STATIC_NORM_MAX_BLOCKS
// and -2 when the array's address cannot be looked up; the totals pointer is the
// device address of the six sums (nullptr if the lookup failed)
constexpr int STATIC_NORM_MAX_BLOCKS = 2048;
int launch_weighted_norm_static(int device, const Planes &P, const float *v, int nblk, cudaStream_t s);
const double *static_norm_totals(int device);
// learned warm start (k_warmnet.cu)
}  // namespace h3d
struct h3d_warmnet;
namespace h3d {
int warmnet_reso(const h3d_warmnet *n);
int warmnet_device(const h3d_warmnet *n);
int warmnet_forward_on(h3d_warmnet *n, const float *x, cudaStream_t s, const float **y);
void launch_warmnet_density_pool(const float *rho, int N, int R, float *out, cudaStream_t s);
void launch_warmnet_to_chi(const Planes &P, const float *y, int R, double *chi, cudaStream_t s);
// lockstep batches (k_fine.cu, k_coarse.cu, k_galerkin.cu).  The create functions
// copy a table to the device (not inside a stream capture) and return 0, -1 for a
// slot count outside 1..BATCH_MAX, -2 if the device table cannot be allocated.
// design[i]: slot i's index in the `active` flags the launches read.
// level 0 of each design: the sweep (launch shape 0: six cases per thread, 1: three),
// the seven-colour residual and the deflation (state: the design's deflation
// state); scratch: the sweeps iterate on each design's r instead of u (timing)
int fine_batch_create(const Level *const *lv0, const float *const *rho, double *const *partial,
                      double *const *state, const int *design, int n, bool scratch, BatchTab *out);
void launch_fine_sweep_batch(const BatchTab &t, const KeMat &ke, const int *active, bool residual, int shape,
                             cudaStream_t s);
void launch_pin_deflate_batch(const BatchTab &t, const KeMat &ke, const int *active, cudaStream_t s);
// one coarse level of each design (all with the same stencil precision): the
// sweep (launch shape 0: two cases per thread, 1: six), with residual the down
// leg's sweep and residual; scratch as for level 0
int coarse_batch_create(const Level *const *lv, const int *design, int n, bool scratch, BatchTab *out);
void launch_coarse_sweep_batch(const BatchTab &t, bool f32, const int *active, bool residual, int shape,
                               cudaStream_t s);
// ratio-2 transfers between levels F[i] (even) and C[i]: restriction of F.r into
// C.f with C.u cleared, prolongation of C.u into F.u (is_root: F is level 0)
int transfer_batch_create(const Level *const *F, const Level *const *C, const int *design, int n, BatchTab *out);
void launch_restrict_batch(const BatchTab &t, const int *active, cudaStream_t s);
void launch_prolong_batch(const BatchTab &t, const int *active, int is_root, cudaStream_t s);
// the per-case norms of each design from its nblk[i] partials into out + 6 * design[i]
// (the same two-stage order as launch_norm_finish above NORM_FINISH_DIRECT blocks)
int norm_batch_create(double *const *partial, const int *nblk, const int *design, int n, BatchTab *out);
void launch_norm_finish_batch(const BatchTab &t, const int *active, double *out, cudaStream_t s);
// the coarsest solve of each design (aug[i]: its [K | K^-1])
int coarsest_batch_create(const Level *const *lv, const double *const *aug, const int *design, int n, BatchTab *out);
void launch_coarse_apply_batch(const BatchTab &t, const int *active, int project, cudaStream_t s);
// field conversion (k_coarse.cu)
void launch_field_to_lex(const Planes &P, const float *src, float *dst_lex, cudaStream_t s);
void launch_field_from_lex(const Planes &P, const float *src_lex, float *dst, cudaStream_t s);
void launch_stencil_to_lex(const Level &L, float *dst_lex, cudaStream_t s);
void launch_stencil_from_lex(const Level &L, const float *src_lex, cudaStream_t s);

}  // namespace h3d
