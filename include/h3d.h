/*
 * h3d.h -- C ABI of the B200 periodic-homogenization solver (libh3d.so).
 *
 * The library replaces the hot path of lavenklau/homo3d: the multigrid grid
 * operations, the V-cycle, the homogenized elastic tensor and its sensitivities,
 * and the OC design update.  Every entry point returns an h3d_status; none
 * exits, throws or prints.  Device pointers passed in are owned by the caller;
 * all solver memory is owned by the handle.  Calls on one handle are ordered on
 * the handle's CUDA stream; calls that return host data synchronise that stream.
 * Distinct handles are independent and may be used from different threads.
 *
 * Data formats at this boundary
 *   density / sensitivity : float, lexicographic cell order, element (x,y,z) at
 *                           x + (y + z*ny)*pitchT  (pitchT >= nx; -1 means nx)
 *   vertex fields         : float [6][nz][ny][nx][3]  (load case, vertex, comp)
 *   stencils              : float [nz][ny][nx][27][9], neighbour d = (dx+1) +
 *                           3(dy+1) + 9(dz+1), entry 3*row + col
 *   elastic tensor C      : double[36] row-major, Voigt order xx yy zz yz xz xy
 *                           with engineering shear strains
 */
#ifndef H3D_H
#define H3D_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define H3D_API __attribute__((visibility("default")))
#else
#define H3D_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct h3d_handle h3d_handle;

typedef enum {
    H3D_OK = 0,
    H3D_ERR_ARG = 1,          /* invalid argument or unsupported size */
    H3D_ERR_CUDA = 2,         /* a CUDA call failed; see h3d_last_error */
    H3D_ERR_NOMEM = 3,        /* device allocation failed */
    H3D_NOT_CONVERGED = 4,    /* iteration cap reached above the tolerance */
    H3D_DIVERGED = 5,         /* relative residual above 10 twice, or NaN */
    H3D_ERR_STATE = 6,        /* call order violated (e.g. solve before density) */
    H3D_ERR_SINGULAR = 7      /* coarsest-grid matrix could not be inverted */
} h3d_status;

/* how the coarsest-grid right-hand side is treated before the dense solve */
typedef enum {
    H3D_COARSE_EXACT = 0,       /* solve the pinned Galerkin system as is */
    H3D_COARSE_PROJECT = 1      /* first remove the mean (rigid translations) */
} h3d_coarse_mode;

/* how the pinned origin vertex enters the level-1 Galerkin operator */
typedef enum {
    H3D_PIN_IDENTITY = 0,       /* identity block at the pinned node, as the reference does */
    H3D_PIN_GALERKIN = 1        /* exact Galerkin product of the pinned fine operator */
} h3d_pin_mode;

/* where the level-0 solution lives and how its residual is formed */
typedef enum {
    H3D_PREC_REFINE = 0,        /* FP64 solution; FP32 V-cycles on the correction, folded
                                   in with an FP64-exact residual in translation-invariant
                                   difference form whenever the stale residual has dropped
                                   by max(1e-3, 1e-5 N) or met the tolerance (iterative
                                   refinement) */
    H3D_PREC_FP32 = 1,          /* FP32 solution swept directly, as the reference does; its
                                   relative residual floors near 1e-6 * N */
    H3D_PREC_MIXED = 2,         /* H3D_PREC_REFINE with the refinement residual accumulated
                                   in FP32 (FP64 differences, FP32 products and sums) down
                                   to relthres 2e-6, below which it accumulates in FP64;
                                   that residual's floor is ~1e-6 of ||f|| at any grid
                                   size (no reference counterpart) */
    H3D_PREC_MIXED_TC = 3       /* H3D_PREC_MIXED with the level-0 residual of every V-cycle
                                   formed element by element on the tensor cores: element
                                   displacement differences and Ke as TF32 hi + lo parts,
                                   FP32 accumulation (no reference counterpart) */
} h3d_precision;

/* storage of the Galerkin coarse-level stencils */
typedef enum {
    H3D_STENCIL_FP16 = 0,       /* FP16 entries, images summed in FP16, as the reference does */
    H3D_STENCIL_FP32 = 1        /* FP32 entries (twice the stencil bytes); keeps the V-cycle
                                   convergent on high-contrast designs where FP16 rounding of
                                   the coarse operators stalls or diverges it */
} h3d_stencil_precision;

typedef struct {
    int reso[3];                /* requested cells per axis; corrected like the reference */
    double youngs_modulus;      /* E of the base material */
    double poisson_ratio;       /* nu of the base material */
    int coarse_mode;            /* h3d_coarse_mode */
    int pin_mode;               /* h3d_pin_mode */
    int precision;              /* h3d_precision */
    int device;                 /* CUDA device ordinal */
    int stencil_precision;      /* h3d_stencil_precision (0 = FP16) */
} h3d_config;

typedef struct {
    int vcycles;                /* V-cycles run (max over the active load cases) */
    int status;                 /* h3d_status of the solve */
    double rel_res[6];          /* final ||r||/||f|| per load case */
    double solve_ms;            /* device time of the V-cycle loop */
    int refinements;            /* refinement steps (u64 += u, exact residual) of the refined mode */
} h3d_solve_stats;

/* fields addressable through h3d_get_field / h3d_set_field */
typedef enum {
    H3D_FIELD_U = 0,            /* displacement */
    H3D_FIELD_F = 1,            /* right-hand side */
    H3D_FIELD_R = 2,            /* residual */
    H3D_FIELD_STENCIL = 3,      /* coarse-level stencil (levels >= 1) */
    H3D_FIELD_CHI = 4,          /* stored solutions of the six cases (level 0, FP64) */
    H3D_FIELD_SOLUTION = 5      /* the refined mode's FP64 solution (level 0); in that
                                   mode level-0 U holds the last correction */
} h3d_field;

/* ---- lifetime (homogenization.cpp:40-66 Homogenization::build) ---------- */
H3D_API int h3d_create(const h3d_config *cfg, h3d_handle **out);
H3D_API int h3d_destroy(h3d_handle *h);
H3D_API const char *h3d_last_error(const h3d_handle *h);
H3D_API int h3d_sync(h3d_handle *h);
/* the handle's CUDA stream (cudaStream_t) for callers that order their own work */
H3D_API void *h3d_stream(h3d_handle *h);

/* ---- hierarchy queries (grid.cpp:21-151 buildRoot / coarse2) -------------- */
H3D_API int h3d_num_levels(const h3d_handle *h);
H3D_API int h3d_level_dims(const h3d_handle *h, int level, int dims[3], int ratio[3]);
/* the 24x24 element matrix in double, row-major (templateMatrix.cpp:95-201) */
H3D_API int h3d_element_matrix(const h3d_handle *h, double ke[576]);

/* ---- design input (homogenization.cpp:79-85 Homogenization::update) ------- */
/* rho_dev: physical density rho^p on the device (grid.cu:4208-4240 Grid::update) */
H3D_API int h3d_update_density(h3d_handle *h, const float *rho_dev, int pitchT);
/* Galerkin coarse operators + coarsest factorisation (MG.cpp:341-354) */
H3D_API int h3d_update_stencils(h3d_handle *h);
/* one coarse level's stencil from the next finer level (grid.cu:2383-2439);
 * coarse_level 1 is built from the densities */
H3D_API int h3d_restrict_stencil(h3d_handle *h, int coarse_level);
/* dense inverse of the coarsest-level operator (grid.cpp:385-424) */
H3D_API int h3d_factor_coarsest(h3d_handle *h);

/* ---- grid entry points, all six load cases at once (grid.h:225-275) ------ */
H3D_API int h3d_enforce_unit_macro_strain(h3d_handle *h);            /* grid.cu:1921 */
H3D_API int h3d_gs_relaxation(h3d_handle *h, int level, float w, int times); /* grid.cu:1192 */
H3D_API int h3d_update_residual(h3d_handle *h, int level);           /* grid.cu:1566 */
H3D_API int h3d_restrict_residual(h3d_handle *h, int coarse_level);  /* grid.cu:1257 */
H3D_API int h3d_prolongate_correction(h3d_handle *h, int fine_level);/* grid.cu:1238 */
H3D_API int h3d_coarse_solve(h3d_handle *h);                         /* grid.cpp:349 */
H3D_API int h3d_reset_displacement(h3d_handle *h, int level);        /* grid.h:246; -1 = all */
/* per-case norm of a level-0 field with the reference's padded-storage
 * multiplicities (grid.cu:1954-1966 v3_norm) */
H3D_API int h3d_field_norms(h3d_handle *h, int field, double out[6]);
/* No reference counterpart.  h3d_field_norms for the FP32 fields U, F, R, for
 * callers that must not have device memory allocated during the call (their
 * device memory is owned by another allocator, or they cannot take the device
 * synchronisation of cudaMalloc / cudaFree): the reduction runs in a fixed device
 * array of 2048 x 6 + 6 doubles (about 96 KB, held by every GPU that loads the
 * library until exit) and nothing is allocated; H3D_ERR_ARG if a field would need
 * more than 2048 blocks.  Calls on one device share the array, so overlapping
 * calls race; the first call on a device looks up the array's address and should
 * come before any stream capture. */
H3D_API int h3d_field_norms_static(h3d_handle *h, int field, double out[6]);

/* ---- multigrid (MG.cpp:46-203) ------------------------------------------- */
H3D_API int h3d_v_cycle(h3d_handle *h, float w, int pre, int post);
/* V-cycles until every case in case_mask has ||r||/||f|| <= tol; with_guess = 0
 * starts from zero (MG::solveEquation) */
H3D_API int h3d_solve(h3d_handle *h, int case_mask, double tol, int with_guess, h3d_solve_stats *stats);

/* ---- homogenization (homogenization.cu:464-948) -------------------------- */
/* the six solves (warm-started from the previous design's solutions, mean
 * removed) followed by C; tol is the relative residual threshold */
H3D_API int h3d_elastic_matrix(h3d_handle *h, double tol, double C[36], h3d_solve_stats *stats);
/* sens = d obj / d rho_phys from dC = d obj / d C (float[36] row-major) */
H3D_API int h3d_sensitivity(h3d_handle *h, const float dC[36], float *sens_dev, int pitchT);
/* forget the stored solutions (warm start).  The next h3d_elastic_matrix then
 * starts from zero without copying, centring or taking the FP64 residual of the
 * zero solution (same results to the last bit, about 6 ms less at 256^3);
 * writing the solutions through h3d_set_field, even with zeros, takes the full
 * path */
H3D_API int h3d_reset_solutions(h3d_handle *h);

/* ---- autotuner (no reference counterpart) ----------------------------------
 * Each smoothed level has H3D_NUM_SHAPES launch shapes for its colour sweep and
 * (coarse levels) its residual: load cases per thread (all six, or two as three
 * threads per vertex) times CTAs per SM (the register budget per thread).  Level 0:
 * shape 0 / 1 / 2 / 3 = six cases at 4 CTAs/SM / two at 5 / three at 5 / two at 6;
 * coarse levels: two at 6 / six at 4 / two at 4 / six at 3.  All give the same
 * results to the last bit.  The first solve of a handle times them (CUDA events,
 * a few sweeps per shape, iterating on the level's scratch residual field) and
 * keeps the fastest; h3d_autotune re-runs that now, h3d_set_tuning fixes the
 * shapes (and turns the automatic tuning off), h3d_get_tuning reads them:
 * shapes[0] = sweep, shapes[1] = residual. */
#define H3D_NUM_SHAPES 4
H3D_API int h3d_autotune(h3d_handle *h);
/* The V-cycle's levels of at most max_level_vertices vertices (0, the default: none)
 * run from the restriction into the largest of them to its post-smoothing in one
 * cooperative kernel launch (no reference counterpart; the reference launches every
 * colour and transfer of every level): per level and colour a phase separated by a
 * grid-wide barrier, the same arithmetic as the separate launches, the same results
 * to the last bit.  Levels with other than ratio-2 coarsening below it fall back to
 * separate launches.  Off by default: on B200 a grid barrier costs about as much
 * as a kernel boundary inside the captured V-cycle graph, and the bottom measured
 * slower (256^3: 12.70 against 12.41 ms per V-cycle with levels up to 32^3). */
H3D_API int h3d_set_vcycle_bottom(h3d_handle *h, int64_t max_level_vertices);
H3D_API int h3d_get_tuning(const h3d_handle *h, int level, int shapes[2]);
H3D_API int h3d_set_tuning(h3d_handle *h, int level, int gs_shape, int res_shape);

/* ---- batched designs (no reference counterpart: the reference homogenizes one
 * design per process) -------------------------------------------------------- */
/* h3d_update_density on n distinct handles (lexicographic rho_phys, unpadded),
 * with the stencil assemblies of all designs enqueued before any is waited on.
 * Returns the first error; every handle is attempted. */
H3D_API int h3d_batch_update_density(h3d_handle *const *hs, const float *const *rho_dev, int n);
/* h3d_elastic_matrix on n distinct handles, solved together: each design's
 * V-cycles run on its own stream and the host advances whichever design's step
 * has completed.  C holds n row-major 6x6 blocks; stats (n entries) and status
 * (n codes, H3D_NOT_CONVERGED keeps its C) may be NULL.  The handles may differ
 * in resolution and precision mode.  Returns the first non-OK status. */
H3D_API int h3d_batch_elastic_matrix(h3d_handle *const *hs, int n, double tol, double *C,
                                     h3d_solve_stats *stats, int *status);
/* Lockstep batches: the designs step through their V-cycles together.  Every
 * step of a batch V-cycle (a colour of a level's sweep, a residual, a transfer,
 * the coarsest solves, the deflation, the norms) is one launch over all designs
 * of that level, each design owning a slice of its CTAs; the batch V-cycle is one
 * captured CUDA graph, and the host decides once per cycle which designs are still
 * running (a converged design's CTAs return at once).  Requirements: 1 to
 * H3D_LOCKSTEP_MAX distinct H3D_PREC_FP32 handles on one device with the same
 * material, stencil precision and coarse mode, and ratio-2 coarsening on every
 * level (resolutions below 512); otherwise H3D_ERR_ARG.  The batch holds the
 * handles' buffer addresses: destroy it before any of its handles.
 * h3d_lockstep_elastic_matrix is h3d_batch_elastic_matrix over the batch's
 * handles, with the same C, statistics and status as h3d_elastic_matrix on each
 * handle to the last bit (solve_ms: from the batch's start to the design's end). */
#define H3D_LOCKSTEP_MAX 64
typedef struct h3d_lockstep h3d_lockstep;
/* h3d_lockstep_create_groups with min(n, H3D_LOCKSTEP_DEFAULT_GROUPS) groups */
#define H3D_LOCKSTEP_DEFAULT_GROUPS 4
H3D_API int h3d_lockstep_create(h3d_handle *const *hs, int n, h3d_lockstep **out);
/* groups (1..n): the designs, largest first, are dealt round-robin to groups whose
 * launches are parallel branches of the batch V-cycle graph, so one group's
 * launches fill the last partial wave of another's; results do not depend on it */
H3D_API int h3d_lockstep_create_groups(h3d_handle *const *hs, int n, int groups, h3d_lockstep **out);
H3D_API int h3d_lockstep_elastic_matrix(h3d_lockstep *b, double tol, double *C, h3d_solve_stats *stats,
                                        int *status);
/* The sweeps of each group and level run in one of two launch shapes (level 0: six
 * or three load cases per thread; coarse levels: two or six), shape 0 by default;
 * results do not depend on the shapes.  h3d_lockstep_set_shapes forces every group
 * and level to fine_shape / coarse_shape (0 or 1); h3d_lockstep_autotune times both
 * shapes level by level with the sweeps of all groups running together on scratch
 * fields (each design's residual field) and keeps shape 1 where it is at least 2 %
 * faster.  Both recapture the batch graph.  Measured for 24-64 designs of
 * 16^3-128^3: the tuned choice within 0.6 % of the fixed default. */
H3D_API int h3d_lockstep_set_shapes(h3d_lockstep *b, int fine_shape, int coarse_shape);
H3D_API int h3d_lockstep_autotune(h3d_lockstep *b);
H3D_API int h3d_lockstep_destroy(h3d_lockstep *b);
H3D_API const char *h3d_lockstep_last_error(const h3d_lockstep *b);

/* ---- SIMP penalisation, the expression rho.pow(p) (TensorExpression.h:517-531) */
/* rho_phys = rho^p */
H3D_API int h3d_penalize(h3d_handle *h, const float *rho_dev, float *rho_phys_dev, int64_t n, float p);
/* grad *= p rho^(p-1): d obj / d rho_phys -> d obj / d rho */
H3D_API int h3d_penalize_backward(h3d_handle *h, const float *rho_dev, float *grad_dev, int64_t n, float p);

/* ---- design update (OCOptimizer.cu:38-247, TensorExpression.cuh:72-) ----- */
H3D_API int h3d_oc_update(h3d_handle *h, const float *sens_dev, float *rho_dev, int64_t n, float volratio,
                  float min_rho, float step_limit, float damp);
H3D_API int h3d_oc_filter(h3d_handle *h, float *sens_dev, const float *rho_dev, const int reso[3], int pitchT,
                  float radius, int periodic);
/* sym: 0 reflect3, 1 reflect6, 2 rotate3; lexicographic, pitch nx */
H3D_API int h3d_symmetrize(h3d_handle *h, float *field_dev, const int reso[3], int sym);

/* ---- the reference's trig-basis initial density (Framework.cuh:106-310 randTri with
 * randTribase_sincos_kernel; -init random / randcenter) -------------------------
 * rho_dev[x + nx (y + ny z)] = the basis sum of n_period periods per axis with the
 * caller's coefficients (6 P + 36 P^2 of them, the reference draws them uniformly
 * in [-1, 1) from a clock-seeded generator; centered = 1 takes four more, a
 * quaternion rotating the centred position), symmetrised (sym as h3d_symmetrize,
 * -1 none), then mapped through the level set m + (M - m) sigmoid(15 (v - t)),
 * M = min(1.5 volratio, 1), m = 0.001, with t bisected until the mean volume is
 * within 1e-3 of volratio.  1 <= n_period <= 50. */
H3D_API int h3d_init_density_trig(h3d_handle *h, float *rho_dev, const int reso[3], int n_period, const float *coeff,
                                  int ncoeff, int centered, float volratio, int sym);

/* ---- radial convolution of the expression layer (AutoDiff/TensorExpression.h:946-1131,
 * rho.conv(radial_convker_t<float, Spline4>(radius)), TensorExpression.cuh:288-369) ---
 * out[p] = sum_o w(o) in[p + o] / sum_o w(o) over the window offsets |o_a| <=
 * (int)(radius + 0.5) that stay inside the grid (periodic = 1: all of them,
 * wrapped), w(o) = 1 - 6 q + 8 q^1.5 - 3 q^2 for q = |o|^2 / radius^2 < 1; with
 * adjoint = 1 the transpose of that map (the expression's backward).  in and out
 * are lexicographic device arrays of nx ny nz floats and must not overlap. */
H3D_API int h3d_conv_radial(h3d_handle *h, const float *in_dev, float *out_dev, const int reso[3], float radius,
                            int periodic, int adjoint);

/* ---- one design update after a solve, on the device (testAutoDiff.cu:298-327,
 * the body of optiBulk / optiShear / optiNpr after objective.eval()) ---------------
 * sens = dObj/drho_phys from dC (as h3d_sensitivity), times p rho^(p-1) (the SIMP
 * backward, homoExpression.h:89-119 through rho.pow(p)); symmetrised
 * (symmetrizeField, Framework.cuh:222-236); filtered (OCOptimizer::filterSens,
 * OCOptimizer.cu:134-152) unless filter_radius <= 0; the OC update of rho
 * (OCOptimizer::update, OCOptimizer.cu:38-67); rho symmetrised.  rho_dev and
 * sens_dev are the caller's lexicographic density and sensitivity (pitch nx).  The
 * sequence is captured once per (rho, sens, parameters) as a CUDA graph on the
 * handle's stream and replayed; dC is read from host memory when it runs, so no
 * step waits on the host.  The call returns after the graph has run (the energy
 * kernel's wait flag is checked then). */
typedef struct {
    float penal;                /* SIMP exponent p of rho_phys = rho^p */
    int sym;                    /* 0 reflect3, 1 reflect6, 2 rotate3, -1 none */
    float filter_radius;        /* cone filter radius; <= 0: no filter */
    int filter_periodic;        /* periodic filter window */
    float volratio;             /* target volume fraction */
    float min_rho;              /* lower density bound (0.001 in the reference) */
    float step_limit;           /* OC move limit */
    float damp;                 /* OC damping exponent */
} h3d_design_params;
H3D_API int h3d_design_step(h3d_handle *h, const float dC[36], float *rho_dev, float *sens_dev,
                            const h3d_design_params *prm);

/* ---- MMA optimiser (MMAOptimizer, mmaOptimizer.h:12-36, mmaOpt.cu:429-1062) -
 * Method of moving asymptotes with m constraints g_i(x) <= 0 (1 <= m <= 4) on n
 * design variables; FP64 state on the device, float design and gradients at the
 * boundary.  An MMA handle has its own stream and is independent of h3d_handle. */
typedef struct h3d_mma h3d_mma;
/* MMAOptimizer(m, n, a0, a, c, d) (mmaOptimizer.h:20-25) */
H3D_API int h3d_mma_create(int m, int64_t n, double a0, double a, double c, double d, int device, h3d_mma **out);
H3D_API int h3d_mma_destroy(h3d_mma *o);
H3D_API const char *h3d_mma_last_error(const h3d_mma *o);
/* MMAOptimizer::setBound(float *xmin, float *xmax) (mmaOptimizer.cu:44-48), device arrays */
H3D_API int h3d_mma_set_bounds(h3d_mma *o, const float *xmin_dev, const float *xmax_dev);
/* MMAOptimizer::setBound(float xmin, float xmax) (mmaOptimizer.cu:50-54) */
H3D_API int h3d_mma_set_bounds_scalar(h3d_mma *o, float xmin, float xmax);
/* MMAOptimizer::update(itn, x, dfdx, gval, dgdx) (mmaOptimizer.cu:61-78): x_dev is
 * replaced by the new design; gval_dev holds m floats, dgdx_dev is a host array of
 * m device pointers to n floats; newton_steps (may be NULL) receives the Newton
 * steps of the subproblem solve */
H3D_API int h3d_mma_update(h3d_mma *o, int itn, float *x_dev, const float *dfdx_dev, const float *gval_dev,
                           const float *const *dgdx_dev, int *newton_steps);

/* ---- learned warm start (no reference counterpart) ------------------------
 * A periodic 3-D convolutional encoder-decoder (channels 16-32-64-64, ~0.26 M
 * FP32 parameters) from the density averaged to reso^3 cells to the six cell
 * solutions chi / N at the reso^3 coarse vertices, trained with its own CUDA
 * forward / backward / Adam kernels.  Tensors are float [batch][channel][reso^3],
 * voxel x + reso*(y + reso*z); targets have 18 channels (case, component). */
typedef struct h3d_warmnet h3d_warmnet;
/* reso: multiple of 8 in 8..128; max_batch: 1..64 */
H3D_API int h3d_warmnet_create(int reso, int max_batch, uint64_t seed, int device, h3d_warmnet **out);
H3D_API int h3d_warmnet_destroy(h3d_warmnet *n);
H3D_API const char *h3d_warmnet_last_error(const h3d_warmnet *n);
H3D_API int h3d_warmnet_num_params(const h3d_warmnet *n, int64_t *count);
H3D_API int h3d_warmnet_get_params(h3d_warmnet *n, float *host);
H3D_API int h3d_warmnet_set_params(h3d_warmnet *n, const float *host);
H3D_API int h3d_warmnet_get_grads(h3d_warmnet *n, float *host);
H3D_API int h3d_warmnet_forward(h3d_warmnet *n, const float *x_dev, int batch, float *y_dev);
/* gradients of the mean squared error of one batch (replacing stored gradients) */
H3D_API int h3d_warmnet_gradients(h3d_warmnet *n, const float *x_dev, const float *t_dev, int batch, double *loss);
/* one Adam step on one batch; *loss = the batch's error before the step */
H3D_API int h3d_warmnet_train_step(h3d_warmnet *n, const float *x_dev, const float *t_dev, int batch, float lr,
                                   double *loss);
/* replace the handle's stored solutions (the starting point of the next
 * h3d_elastic_matrix) by the network's prediction for the handle's density, on
 * cubic grids whose size is a multiple of the network's reso.  In the refined
 * precision mode a solve whose starting residual exceeds that of a zero start
 * restarts from zero. */
H3D_API int h3d_warm_start_learned(h3d_handle *h, h3d_warmnet *net);

/* ---- data exchange (host pointers) ---------------------------------------- */
H3D_API int h3d_get_field(h3d_handle *h, int level, int field, float *host);
H3D_API int h3d_set_field(h3d_handle *h, int level, int field, const float *host);

#ifdef __cplusplus
}
#endif
#endif /* H3D_H */
