// h3d.hpp -- header-only C++ shim that restores the homo3d class names on top of
// the C ABI in h3d.h, so code written against the reference's hot path
// (homogenization.h, MG.h, grid.h, OCOptimizer.h) compiles against libh3d with
// little change.  Errors are reported as std::runtime_error, as the reference's
// own code paths do (MG.cpp:153, grid.cpp:26).
#pragma once
#include <array>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "h3d.h"

namespace homo {

inline void h3d_check(h3d_handle *h, int code) {
    if (code != H3D_OK && code != H3D_NOT_CONVERGED)
        throw std::runtime_error(std::string("h3d: ") + h3d_last_error(h));
}

struct HomoConfig {               // the fields of cfg::HomoConfig this path reads
    int reso[3] = {64, 64, 64};
    double youngsModulu = 1e1;
    double poissonRatio = 0.3;
    double femRelThres = 1e-2;
    int coarseMode = H3D_COARSE_EXACT;
    int pinMode = H3D_PIN_IDENTITY;
    int precision = H3D_PREC_REFINE;
    int device = 0;
    int stencilPrecision = H3D_STENCIL_FP16;
};

// one level of the hierarchy (grid.h:104-418); operates on all six load cases
struct Grid {
    h3d_handle *h;
    int level;
    std::array<int, 3> cellReso{};
    void gs_relaxation(float w_SOR = 1.f, int times_ = 1) { h3d_check(h, h3d_gs_relaxation(h, level, w_SOR, times_)); }
    void update_residual() { h3d_check(h, h3d_update_residual(h, level)); }
    void restrict_residual() { h3d_check(h, h3d_restrict_residual(h, level)); }
    void prolongate_correction() { h3d_check(h, h3d_prolongate_correction(h, level)); }
    void restrict_stencil() { h3d_check(h, h3d_restrict_stencil(h, level)); }
    bool solveHostEquation() { return h3d_coarse_solve(h) == H3D_OK; }
    void assembleHostMatrix() { h3d_check(h, h3d_factor_coarsest(h)); }
    void enforce_unit_macro_strain(int /*all six at once*/) { h3d_check(h, h3d_enforce_unit_macro_strain(h)); }
    void reset_displacement() { h3d_check(h, h3d_reset_displacement(h, level)); }
};

// multigrid driver (MG.h:14-45)
struct MG {
    h3d_handle *h = nullptr;
    std::vector<std::shared_ptr<Grid>> grids;
    void v_cycle(float w_SOR = 1.f, int pre = 1, int post = 1) { h3d_check(h, h3d_v_cycle(h, w_SOR, pre, post)); }
    double solveEquation(double tol = 1e-2, bool with_guess = true) {
        h3d_solve_stats st{};
        h3d_check(h, h3d_solve(h, 63, tol, with_guess ? 1 : 0, &st));
        double r = 0;
        for (double v : st.rel_res) r = v > r ? v : r;
        return r;
    }
    void updateStencils() { h3d_check(h, h3d_update_stencils(h)); }
    void reset_displacement() { h3d_check(h, h3d_reset_displacement(h, -1)); }
    std::shared_ptr<Grid> getRootGrid() { return grids.at(0); }
};

// homogenized elastic tensor and its sensitivities (homogenization.h:17-61)
struct Homogenization {
    HomoConfig config;
    h3d_handle *h = nullptr;
    std::unique_ptr<MG> mg_;
    std::shared_ptr<Grid> grid;

    Homogenization() = default;
    explicit Homogenization(const HomoConfig &c) { build(c); }
    Homogenization(int xreso, int yreso, int zreso, double youngsModu = 1e6, double poissonRatio = 0.3) {
        HomoConfig c;
        c.reso[0] = xreso; c.reso[1] = yreso; c.reso[2] = zreso;
        c.youngsModulu = youngsModu; c.poissonRatio = poissonRatio;
        build(c);
    }
    Homogenization(const Homogenization &) = delete;
    Homogenization &operator=(const Homogenization &) = delete;
    ~Homogenization() { if (h) h3d_destroy(h); }

    void build(const HomoConfig &c) {
        config = c;
        h3d_config cfg{};
        for (int i = 0; i < 3; i++) cfg.reso[i] = c.reso[i];
        cfg.youngs_modulus = c.youngsModulu;
        cfg.poisson_ratio = c.poissonRatio;
        cfg.coarse_mode = c.coarseMode;
        cfg.pin_mode = c.pinMode;
        cfg.precision = c.precision;
        cfg.device = c.device;
        cfg.stencil_precision = c.stencilPrecision;
        if (h3d_create(&cfg, &h) != H3D_OK) throw std::runtime_error("h3d_create failed");
        mg_.reset(new MG());
        mg_->h = h;
        for (int l = 0; l < h3d_num_levels(h); l++) {
            auto g = std::make_shared<Grid>();
            g->h = h;
            g->level = l;
            int d[3], r[3];
            h3d_level_dims(h, l, d, r);
            g->cellReso = {d[0], d[1], d[2]};
            mg_->grids.push_back(g);
        }
        grid = mg_->grids[0];
    }
    std::shared_ptr<Grid> getGrid() { return grid; }
    // rho: physical density on the device, lexicographic with row pitch pitchT
    void update(float *rho = nullptr, int pitchT = -1) {
        if (rho) h3d_check(h, h3d_update_density(h, rho, pitchT));
        else h3d_check(h, h3d_update_stencils(h));
    }
    void elasticMatrix(double C[6][6]) {
        h3d_check(h, h3d_elastic_matrix(h, config.femRelThres, &C[0][0], nullptr));
    }
    void elasticMatrix(float C[6][6]) {
        double c[6][6];
        elasticMatrix(c);
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 6; j++) C[i][j] = (float)c[i][j];
    }
    // lexiOrder is always true here: sens is written lexicographically with pitchT
    void Sensitivity(float dC[6][6], float *sens, int pitchT, bool /*lexiOrder*/ = true) {
        h3d_check(h, h3d_sensitivity(h, &dC[0][0], sens, pitchT));
    }
};

// optimality-criteria update and sensitivity filter (OCOptimizer.h:16-19)
struct OCOptimizer {
    h3d_handle *h;
    int ne;
    float step_limit = 0.02f, damp = 0.5f, minRho = 0.001f;
    OCOptimizer(Homogenization &hom, int Ne, float min_density, float stepLimit, float dampExponent)
        : h(hom.h), ne(Ne), step_limit(stepLimit), damp(dampExponent), minRho(min_density) {}
    void filterSens(float *sens, const float *rho, size_t pitchT, int reso[3], float radius = 2, bool periodic = false) {
        h3d_check(h, h3d_oc_filter(h, sens, rho, reso, (int)pitchT, radius, periodic ? 1 : 0));
    }
    void update(const float *sens, float *rho, float volratio) {
        h3d_check(h, h3d_oc_update(h, sens, rho, ne, volratio, minRho, step_limit, damp));
    }
};

// method of moving asymptotes (mmaOptimizer.h:12-36); device pointers throughout
struct MMAOptimizer {
    h3d_mma *o = nullptr;
    int n, m;
    MMAOptimizer(int nconstrain, int nvar, double a0_, double a_, double c_, double d_, int device = 0)
        : n(nvar), m(nconstrain) {
        if (h3d_mma_create(nconstrain, nvar, a0_, a_, c_, d_, device, &o) != H3D_OK)
            throw std::runtime_error("h3d_mma_create failed");
    }
    ~MMAOptimizer() { h3d_mma_destroy(o); }
    MMAOptimizer(const MMAOptimizer &) = delete;
    MMAOptimizer &operator=(const MMAOptimizer &) = delete;
    void check(int st) {
        if (st != H3D_OK) throw std::runtime_error(h3d_mma_last_error(o));
    }
    void setBound(float *xmin, float *xmax) { check(h3d_mma_set_bounds(o, xmin, xmax)); }
    void setBound(float xmin, float xmax) { check(h3d_mma_set_bounds_scalar(o, xmin, xmax)); }
    void update(int itn, float *x, float *dfdx, float *gval, float **dgdx) {
        check(h3d_mma_update(o, itn, x, dfdx, gval, dgdx, nullptr));
    }
};

enum TensorSym { Reflection3 = 0, Reflection6 = 1, Rotate3 = 2 };
inline void symmetrize(Homogenization &hom, float *field, const int reso[3], TensorSym sym) {
    h3d_check(hom.h, h3d_symmetrize(hom.h, field, reso, (int)sym));
}

}  // namespace homo
