/*
 * mma_oracle.c -- FP64 CPU restatement of the reference's MMA update
 * (Svanberg's method of moving asymptotes, the 2007 mmasub/subsolv scheme).
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle for the CUDA MMA update in
 * homo3d_b200/csrc/k_mma.cu; nothing in the product links it.
 *
 * Follows lavenklau/homo3d optimization/mmaOpt.cu:
 *   mmasub_ker (mmaOpt.cu:820-1019): asymptotes low/upp (asyinit 0.5, asyincr 1.2,
 *     asydecr 0.7, clamps at 0.01 and 10 times xmax-xmin), move limits alfa/beta
 *     (albefa 0.1), p0/q0 and P/Q with 1e-3 (p+q) + raa0/xmami (raa0 1e-5),
 *     b = P/(upp-x) + Q/(x-low) summed over the variables, minus gval;
 *   subsolv_g (mmaOpt.cu:429-815): primal-dual interior point on the MMA
 *     subproblem, epsi from 1 down to epsimin 1e-7 by factors of 10, Newton steps
 *     while max|residual| > 0.9 epsi (at most 200 per epsi), the (m+1) x (m+1)
 *     system of the m < n branch, step length 1/max(1, 1.01 * largest ratio),
 *     halving line search on the residual 2-norm (at most 50 halvings);
 *   mmasub_g (mmaOpt.cu:1021-1062): xold2 <- xold1, xold1 <- x, x <- new x.
 * The (m+1) system is solved by Gaussian elimination with partial pivoting (the
 * reference calls Eigen's ColPivHouseholderQR, mmaOpt.cpp:49-73; the two agree to
 * rounding for the well-conditioned systems met here).  Parity status: pinned by
 * optimality (KKT) checks of converged toy problems, not by reference outputs.
 *
 * Arrays: x-like vectors double[n]; dgdx row-major double[m][n].
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MMA_EPSIMIN 1e-7
#define MMA_RAA0 1e-5
#define MMA_ALBEFA 0.1
#define MMA_ASYINIT 0.5
#define MMA_ASYINCR 1.2
#define MMA_ASYDECR 0.7

static double dmax(double a, double b) { return a > b ? a : b; }
static double dmin(double a, double b) { return a < b ? a : b; }

/* solve A x = b for a dense k x k system (row-major), partial pivoting */
static int dense_solve(int k, double *A, double *b, double *x) {
    for (int c = 0; c < k; c++) {
        int p = c;
        for (int r = c + 1; r < k; r++)
            if (fabs(A[r * k + c]) > fabs(A[p * k + c])) p = r;
        if (A[p * k + c] == 0.0) return -1;
        if (p != c) {
            for (int j = 0; j < k; j++) { double t = A[c * k + j]; A[c * k + j] = A[p * k + j]; A[p * k + j] = t; }
            double t = b[c]; b[c] = b[p]; b[p] = t;
        }
        for (int r = c + 1; r < k; r++) {
            double f = A[r * k + c] / A[c * k + c];
            for (int j = c; j < k; j++) A[r * k + j] -= f * A[c * k + j];
            b[r] -= f * b[c];
        }
    }
    for (int r = k - 1; r >= 0; r--) {
        double s = b[r];
        for (int j = r + 1; j < k; j++) s -= A[r * k + j] * x[j];
        x[r] = s / A[r * k + r];
    }
    return 0;
}

typedef struct {
    int m;
    long n;
    const double *low, *upp, *alfa, *beta, *p0, *q0, *P, *Q, *a, *b, *c, *d;
    double a0;
} mma_sub;

typedef struct {
    double *x, *xsi, *eta; /* n */
    double *y, *lam, *mu, *s; /* m */
    double z, zet;
} mma_pt;

/* residual of the perturbed KKT system at point v; returns the 2-norm, max abs in *mx */
static double kkt_residual(const mma_sub *S, const mma_pt *v, double epsi, double *mx) {
    const int m = S->m;
    const long n = S->n;
    double ss = 0, mxa = 0;
    double *gvec = calloc(m, sizeof(double));
    for (long j = 0; j < n; j++) {
        const double ux1 = S->upp[j] - v->x[j], xl1 = v->x[j] - S->low[j];
        double plam = S->p0[j], qlam = S->q0[j];
        for (int i = 0; i < m; i++) {
            plam += S->P[i * n + j] * v->lam[i];
            qlam += S->Q[i * n + j] * v->lam[i];
            gvec[i] += S->P[i * n + j] / ux1 + S->Q[i * n + j] / xl1;
        }
        const double dpsidx = plam / (ux1 * ux1) - qlam / (xl1 * xl1);
        const double rex = dpsidx - v->xsi[j] + v->eta[j];
        const double rexsi = v->xsi[j] * (v->x[j] - S->alfa[j]) - epsi;
        const double reeta = v->eta[j] * (S->beta[j] - v->x[j]) - epsi;
        ss += rex * rex + rexsi * rexsi + reeta * reeta;
        mxa = dmax(mxa, dmax(fabs(rex), dmax(fabs(rexsi), fabs(reeta))));
    }
    double alam = 0;
    for (int i = 0; i < m; i++) alam += S->a[i] * v->lam[i];
    const double rez = S->a0 - v->zet - alam, rezet = v->zet * v->z - epsi;
    ss += rez * rez + rezet * rezet;
    mxa = dmax(mxa, dmax(fabs(rez), fabs(rezet)));
    for (int i = 0; i < m; i++) {
        const double rey = S->c[i] + S->d[i] * v->y[i] - v->mu[i] - v->lam[i];
        const double relam = gvec[i] - S->a[i] * v->z - v->y[i] + v->s[i] - S->b[i];
        const double remu = v->mu[i] * v->y[i] - epsi;
        const double res = v->lam[i] * v->s[i] - epsi;
        ss += rey * rey + relam * relam + remu * remu + res * res;
        mxa = dmax(mxa, dmax(dmax(fabs(rey), fabs(relam)), dmax(fabs(remu), fabs(res))));
    }
    free(gvec);
    *mx = mxa;
    return sqrt(ss);
}

static void pt_alloc(mma_pt *v, int m, long n) {
    v->x = malloc(sizeof(double) * n);
    v->xsi = malloc(sizeof(double) * n);
    v->eta = malloc(sizeof(double) * n);
    v->y = malloc(sizeof(double) * m);
    v->lam = malloc(sizeof(double) * m);
    v->mu = malloc(sizeof(double) * m);
    v->s = malloc(sizeof(double) * m);
}
static void pt_free(mma_pt *v) {
    free(v->x); free(v->xsi); free(v->eta); free(v->y); free(v->lam); free(v->mu); free(v->s);
}

/* subsolv_g (mmaOpt.cu:429-815); returns the number of Newton steps, x_out = new x */
static int subsolve(const mma_sub *S, double *x_out) {
    const int m = S->m;
    const long n = S->n;
    mma_pt v, o, dv;
    pt_alloc(&v, m, n); pt_alloc(&o, m, n); pt_alloc(&dv, m, n);
    for (long j = 0; j < n; j++) {
        v.x[j] = 0.5 * (S->alfa[j] + S->beta[j]);
        v.xsi[j] = dmax(1.0 / (v.x[j] - S->alfa[j]), 1.0);
        v.eta[j] = dmax(1.0 / (S->beta[j] - v.x[j]), 1.0);
    }
    for (int i = 0; i < m; i++) { v.y[i] = 1; v.lam[i] = 1; v.mu[i] = dmax(0.5 * S->c[i], 1.0); v.s[i] = 1; }
    v.z = 1; v.zet = 1;
    double *delx = malloc(sizeof(double) * n), *diagx = malloc(sizeof(double) * n);
    double *GG = malloc(sizeof(double) * m * n);
    double *gvec = malloc(sizeof(double) * m), *dely = malloc(sizeof(double) * m);
    double *dellam = malloc(sizeof(double) * m), *diagy = malloc(sizeof(double) * m);
    double *blam = malloc(sizeof(double) * (m + 1)), *AA = malloc(sizeof(double) * (m + 1) * (m + 1));
    double *sol = malloc(sizeof(double) * (m + 1));
    double epsi = 1.0;
    int newton = 0;
    while (epsi > MMA_EPSIMIN) {
        double residumax;
        double residunorm = kkt_residual(S, &v, epsi, &residumax);
        int ittt = 0;
        while (residumax > 0.9 * epsi && ittt < 200) {
            ittt++;
            newton++;
            for (int i = 0; i < m; i++) gvec[i] = 0;
            for (long j = 0; j < n; j++) {
                const double ux1 = S->upp[j] - v.x[j], xl1 = v.x[j] - S->low[j];
                const double ux2 = ux1 * ux1, xl2 = xl1 * xl1, ux3 = ux1 * ux2, xl3 = xl1 * xl2;
                double plam = S->p0[j], qlam = S->q0[j];
                for (int i = 0; i < m; i++) {
                    plam += S->P[i * n + j] * v.lam[i];
                    qlam += S->Q[i * n + j] * v.lam[i];
                    gvec[i] += S->P[i * n + j] / ux1 + S->Q[i * n + j] / xl1;
                    GG[i * n + j] = S->P[i * n + j] / ux2 - S->Q[i * n + j] / xl2;
                }
                const double dpsidx = plam / ux2 - qlam / xl2;
                delx[j] = dpsidx - epsi / (v.x[j] - S->alfa[j]) + epsi / (S->beta[j] - v.x[j]);
                diagx[j] = 2 * (plam / ux3 + qlam / xl3) + v.xsi[j] / (v.x[j] - S->alfa[j]) +
                           v.eta[j] / (S->beta[j] - v.x[j]);
            }
            double alam = 0;
            for (int i = 0; i < m; i++) alam += S->a[i] * v.lam[i];
            const double delz = S->a0 - alam - epsi / v.z;
            for (int i = 0; i < m; i++) {
                dely[i] = S->c[i] + S->d[i] * v.y[i] - v.lam[i] - epsi / v.y[i];
                dellam[i] = gvec[i] - S->a[i] * v.z - v.y[i] - S->b[i] + epsi / v.lam[i];
                diagy[i] = S->d[i] + v.mu[i] / v.y[i];
            }
            /* [Alam a; a' -zet/z] [dlam; dz] = [blam; delz] */
            const int k = m + 1;
            for (int i = 0; i < m; i++) {
                double gx = 0;
                for (long j = 0; j < n; j++) gx += GG[i * n + j] * (delx[j] / diagx[j]);
                blam[i] = dellam[i] + dely[i] / diagy[i] - gx;
                for (int q = 0; q < m; q++) {
                    double sum = 0;
                    for (long j = 0; j < n; j++) sum += GG[i * n + j] * GG[q * n + j] / diagx[j];
                    AA[i * k + q] = sum;
                }
                AA[i * k + i] += v.s[i] / v.lam[i] + 1.0 / diagy[i];
                AA[i * k + m] = S->a[i];
                AA[m * k + i] = S->a[i];
            }
            AA[m * k + m] = -v.zet / v.z;
            blam[m] = delz;
            dense_solve(k, AA, blam, sol);
            const double dz = sol[m];
            for (int i = 0; i < m; i++) dv.lam[i] = sol[i];
            double stm = 1.0;
            for (long j = 0; j < n; j++) {
                double g = 0;
                for (int i = 0; i < m; i++) g += GG[i * n + j] * dv.lam[i];
                const double dx = -delx[j] / diagx[j] - g / diagx[j];
                const double xa = v.x[j] - S->alfa[j], bx = S->beta[j] - v.x[j];
                dv.x[j] = dx;
                dv.xsi[j] = -v.xsi[j] + epsi / xa - (v.xsi[j] * dx) / xa;
                dv.eta[j] = -v.eta[j] + epsi / bx + (v.eta[j] * dx) / bx;
                stm = dmax(stm, -1.01 * dv.xsi[j] / v.xsi[j]);
                stm = dmax(stm, -1.01 * dv.eta[j] / v.eta[j]);
                stm = dmax(stm, -1.01 * dx / xa);
                stm = dmax(stm, 1.01 * dx / bx);
            }
            for (int i = 0; i < m; i++) {
                dv.y[i] = -dely[i] / diagy[i] + dv.lam[i] / diagy[i];
                dv.mu[i] = -v.mu[i] + epsi / v.y[i] - (v.mu[i] * dv.y[i]) / v.y[i];
                dv.s[i] = -v.s[i] + epsi / v.lam[i] - (v.s[i] * dv.lam[i]) / v.lam[i];
                stm = dmax(stm, -1.01 * dv.y[i] / v.y[i]);
                stm = dmax(stm, -1.01 * dv.lam[i] / v.lam[i]);
                stm = dmax(stm, -1.01 * dv.mu[i] / v.mu[i]);
                stm = dmax(stm, -1.01 * dv.s[i] / v.s[i]);
            }
            const double dzet = -v.zet + epsi / v.z - v.zet * dz / v.z;
            stm = dmax(stm, -1.01 * dz / v.z);
            stm = dmax(stm, -1.01 * dzet / v.zet);
            double steg = 1.0 / stm;
            /* line search from the saved point */
            memcpy(o.x, v.x, sizeof(double) * n); memcpy(o.xsi, v.xsi, sizeof(double) * n);
            memcpy(o.eta, v.eta, sizeof(double) * n);
            memcpy(o.y, v.y, sizeof(double) * m); memcpy(o.lam, v.lam, sizeof(double) * m);
            memcpy(o.mu, v.mu, sizeof(double) * m); memcpy(o.s, v.s, sizeof(double) * m);
            o.z = v.z; o.zet = v.zet;
            int itto = 0;
            double resinew = 2 * residunorm, rmax = residumax;
            while (resinew > residunorm && itto < 50) {
                itto++;
                for (long j = 0; j < n; j++) {
                    v.x[j] = o.x[j] + steg * dv.x[j];
                    v.xsi[j] = o.xsi[j] + steg * dv.xsi[j];
                    v.eta[j] = o.eta[j] + steg * dv.eta[j];
                }
                for (int i = 0; i < m; i++) {
                    v.y[i] = o.y[i] + steg * dv.y[i];
                    v.lam[i] = o.lam[i] + steg * dv.lam[i];
                    v.mu[i] = o.mu[i] + steg * dv.mu[i];
                    v.s[i] = o.s[i] + steg * dv.s[i];
                }
                v.z = o.z + steg * dz;
                v.zet = o.zet + steg * dzet;
                resinew = kkt_residual(S, &v, epsi, &rmax);
                steg /= 2;
            }
            residunorm = resinew;
            residumax = rmax;
        }
        epsi *= 0.1;
    }
    memcpy(x_out, v.x, sizeof(double) * n);
    pt_free(&v); pt_free(&o); pt_free(&dv);
    free(delx); free(diagx); free(GG); free(gvec); free(dely); free(dellam); free(diagy);
    free(blam); free(AA); free(sol);
    return newton;
}

/* one MMA update (mmasub_g): xvar is replaced by the new design, xold1/xold2 and
 * low/upp are updated in place.  a/c/d are m-vectors, dgdx is [m][n], gval[m].
 * Returns the number of Newton steps of the subproblem. */
int ora_mma_update(int m, long n, int itn, double *xvar, const double *xmin, const double *xmax, double *xold1,
                   double *xold2, const double *df0dx, const double *gval, const double *dgdx, double *low,
                   double *upp, double a0, const double *a, const double *c, const double *d, double move) {
    double *alfa = malloc(sizeof(double) * n), *beta = malloc(sizeof(double) * n);
    double *p0 = malloc(sizeof(double) * n), *q0 = malloc(sizeof(double) * n);
    double *P = malloc(sizeof(double) * m * n), *Q = malloc(sizeof(double) * m * n);
    double *b = calloc(m, sizeof(double));
    for (long j = 0; j < n; j++) {
        const double dx = xmax[j] - xmin[j];
        if (itn <= 2) {
            low[j] = xvar[j] - MMA_ASYINIT * dx;
            upp[j] = xvar[j] + MMA_ASYINIT * dx;
        } else {
            const double zzz = (xvar[j] - xold1[j]) * (xold1[j] - xold2[j]);
            const double f = zzz > 0 ? MMA_ASYINCR : (zzz < 0 ? MMA_ASYDECR : 1.0);
            double l = xvar[j] - f * (xold1[j] - low[j]);
            double u = xvar[j] + f * (upp[j] - xold1[j]);
            l = dmin(dmax(l, xvar[j] - 10 * dx), xvar[j] - 0.01 * dx);
            u = dmax(dmin(u, xvar[j] + 10 * dx), xvar[j] + 0.01 * dx);
            low[j] = l;
            upp[j] = u;
        }
        alfa[j] = dmax(dmax(low[j] + MMA_ALBEFA * (xvar[j] - low[j]), xvar[j] - move * dx), xmin[j]);
        beta[j] = dmin(dmin(upp[j] - MMA_ALBEFA * (upp[j] - xvar[j]), xvar[j] + move * dx), xmax[j]);
        const double xmamiinv = 1.0 / dmax(dx, 1e-5);
        const double ux1 = upp[j] - xvar[j], xl1 = xvar[j] - low[j];
        const double ux2 = ux1 * ux1, xl2 = xl1 * xl1;
        const double fp = dmax(df0dx[j], 0), fm = dmax(-df0dx[j], 0);
        const double pq0 = 1e-3 * (fp + fm) + MMA_RAA0 * xmamiinv;
        p0[j] = (fp + pq0) * ux2;
        q0[j] = (fm + pq0) * xl2;
        for (int i = 0; i < m; i++) {
            const double g = dgdx[(long)i * n + j];
            const double p = dmax(g, 0), q = dmax(-g, 0);
            const double pq = 1e-3 * (p + q) + MMA_RAA0 * xmamiinv;
            P[(long)i * n + j] = (p + pq) * ux2;
            Q[(long)i * n + j] = (q + pq) * xl2;
            b[i] += P[(long)i * n + j] / ux1 + Q[(long)i * n + j] / xl1;
        }
    }
    for (int i = 0; i < m; i++) b[i] -= gval[i];
    mma_sub S = {m, n, low, upp, alfa, beta, p0, q0, P, Q, a, b, c, d, a0};
    double *xnew = malloc(sizeof(double) * n);
    const int newton = subsolve(&S, xnew);
    memcpy(xold2, xold1, sizeof(double) * n);
    memcpy(xold1, xvar, sizeof(double) * n);
    memcpy(xvar, xnew, sizeof(double) * n);
    free(alfa); free(beta); free(p0); free(q0); free(P); free(Q); free(b); free(xnew);
    return newton;
}
