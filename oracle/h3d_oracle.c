/*
 * h3d_oracle.c -- FP64 CPU restatement of the homo3d periodic-homogenization hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle for the CUDA library
 * (homo3d_b200/csrc) and the timed CPU baseline of bench.py.  Nothing in the
 * product links it or calls it.
 *
 * Parity status: partially pinned.  The reference (lavenklau/homo3d) cannot be
 * built here (it needs Eigen 3.4, glm 0.9.9, gflags and OpenVDB, none of which are
 * installed), and it ships no golden outputs.  What pins this restatement:
 *   - the 24x24 element matrix is checked against the integer lambda/mu tables
 *     that the reference hard-codes (homogenization/templateMatrix.cpp:8-61),
 *     through the fixture tests/golden/ke_lame72.json;
 *   - analytic known answers (rigid-body null space of Ke, homogeneous density
 *     gives the base-material C, laminates, cubic symmetry, FD sensitivities);
 *   - the symmetrisation orbit maps are restated bit for bit.
 * The coarsest-grid solve (Eigen FullPivLU kernel + BiCGSTAB/ILUT in the
 * reference, grid.cpp:349-424) is not pinned: it is replaced by a dense LU solve
 * after removing the three rigid translations from the right-hand side.
 *
 * Conventions shared with the CUDA library:
 *   vertex / element (x,y,z), 0 <= x < nx, lexicographic id x + nx*(y + ny*z);
 *   element e has local nodes i = 0..7 at e + (i%2, i/2%2, i/4) (periodic wrap);
 *   local DOF 3*i + comp  (templateMatrix.cpp:137-158);
 *   Gauss-Seidel colour of a vertex k = ((x+1)&1) | ((y+1)&1)<<1 | ((z+1)&1)<<2,
 *   swept in order k = 0..7 (grid.cu:1206-1231: colour = parity of the padded
 *   position, padded position = position + 1);
 *   vertex fields are double [nv][6][3] (vertex, load case, component);
 *   stencils are double [nv][27][9], neighbour d = (dx+1) + 3(dy+1) + 9(dz+1),
 *   entry k = 3*row + col (row: force component of the vertex, col: displacement
 *   component of the neighbour).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <omp.h>

#define NCASE 6
#define NF (NCASE * 3)
#define MAXLV 16

static const double RHO_PENAL_MIN = 1e-9; /* grid.h:425 */

static inline int wrapi(int a, int n) { a %= n; return a < 0 ? a + n : a; }
static inline long lexid(int x, int y, int z, const int n[3]) {
    return (long)x + (long)n[0] * ((long)y + (long)n[1] * (long)z);
}
static inline int vcolor(int x, int y, int z) {
    return ((x + 1) & 1) | (((y + 1) & 1) << 1) | (((z + 1) & 1) << 2);
}
static inline double to_half(double v) { return (double)(_Float16)v; }
/* fp16 == 3: FP32 storage of the coarse stencils (not the reference's scheme;
 * used to show that FP16 storage is what makes the V-cycle diverge on
 * high-contrast designs) */
static void round_row_f32(double *st) {
    for (int q = 0; q < 243; q++) st[q] = (double)(float)st[q];
}

/* ------------------------------------------------------------------------- */
/* element matrix (templateMatrix.cpp:95-201)                                 */
/* ------------------------------------------------------------------------- */

/* Ke for material matrix D by 2x2x2 Gauss quadrature on the unit cube */
static void ke_quadrature(const double D[6][6], double ke[576]) {
    double p = sqrt(1. / 3);
    memset(ke, 0, sizeof(double) * 576);
    for (int g = 0; g < 8; g++) {
        double gp[3] = {((2 * (g % 2) - 1) * p + 1) / 2, ((2 * (g / 2 % 2) - 1) * p + 1) / 2,
                        ((2 * (g / 4) - 1) * p + 1) / 2};
        double dn[8][3];
        for (int k = 0; k < 8; k++) {
            int id[3] = {k % 2, k / 2 % 2, k / 4};
            double r[3];
            for (int a = 0; a < 3; a++) r[a] = id[a] ? gp[a] : 1 - gp[a];
            for (int a = 0; a < 3; a++) dn[k][a] = (id[a] ? 1.0 : -1.0) * r[(a + 1) % 3] * r[(a + 2) % 3];
        }
        double B[6][24];
        memset(B, 0, sizeof(B));
        for (int k = 0; k < 8; k++) {
            for (int a = 0; a < 3; a++) B[a][3 * k + a] = dn[k][a];
            B[3][3 * k + 1] = dn[k][2]; B[3][3 * k + 2] = dn[k][1]; /* yz */
            B[4][3 * k + 0] = dn[k][2]; B[4][3 * k + 2] = dn[k][0]; /* xz */
            B[5][3 * k + 0] = dn[k][1]; B[5][3 * k + 1] = dn[k][0]; /* xy */
        }
        double DB[6][24];
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 24; j++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += D[i][k] * B[k][j];
                DB[i][j] = s;
            }
        for (int i = 0; i < 24; i++)
            for (int j = 0; j < 24; j++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += B[k][i] * DB[k][j];
                ke[i * 24 + j] += s;
            }
    }
    for (int i = 0; i < 576; i++) ke[i] *= 1.0 / 8.0;
    for (int i = 0; i < 24; i++)
        for (int j = 0; j < i; j++) {
            double s = 0.5 * (ke[i * 24 + j] + ke[j * 24 + i]);
            ke[i * 24 + j] = ke[j * 24 + i] = s;
        }
}

/* Ke = lambda*Klam + mu*Kmu;  72*Klam and 72*Kmu are integer tables */
void ora_ke_lame(double klam[576], double kmu[576]) {
    double Dl[6][6], Dm[6][6];
    memset(Dl, 0, sizeof(Dl));
    memset(Dm, 0, sizeof(Dm));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Dl[i][j] = 1;
    for (int i = 0; i < 3; i++) Dm[i][i] = 2;
    for (int i = 3; i < 6; i++) Dm[i][i] = 1;
    ke_quadrature(Dl, klam);
    ke_quadrature(Dm, kmu);
}

/* Ke for Young's modulus E and Poisson ratio nu (templateMatrix.cpp:95-165) */
void ora_ke(double E, double nu, double ke[576]) {
    double D[6][6];
    memset(D, 0, sizeof(D));
    double s = E / ((1 + nu) * (1 - 2 * nu));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) D[i][j] = s * (i == j ? 1 - nu : nu);
    for (int i = 3; i < 6; i++) D[i][i] = s * (1 - 2 * nu) / 2;
    ke_quadrature(D, ke);
}

/* unit macro-strain displacement of local node i for strain case c
 * (homoCommon.cuh:455-519, engineering shear split in halves) */
static void macro_disp(int i, int c, double u[3]) {
    int p[3] = {i % 2, i / 2 % 2, i / 4};
    u[0] = u[1] = u[2] = 0;
    switch (c) {
    case 0: u[0] = p[0]; break;
    case 1: u[1] = p[1]; break;
    case 2: u[2] = p[2]; break;
    case 3: u[1] = p[2] / 2.; u[2] = p[1] / 2.; break;
    case 4: u[0] = p[2] / 2.; u[2] = p[0] / 2.; break;
    case 5: u[0] = p[1] / 2.; u[1] = p[0] / 2.; break;
    }
}

/* ------------------------------------------------------------------------- */
/* hierarchy (grid.cpp:21-151)                                                */
/* ------------------------------------------------------------------------- */
int ora_hierarchy(const int reso[3], int dims[MAXLV][3], int ratios[MAXLV][3]) {
    int avail[3], n[3];
    for (int a = 0; a < 3; a++) {
        if (reso[a] < 2 || reso[a] > 1024) return -1;
        double l2 = log2((double)reso[a]);
        double lcl = fmax(floor(l2) - 2, 0.);
        double xc = l2 - lcl;
        avail[a] = (int)ceil(pow(2, xc));
        n[a] = (int)(avail[a] * pow(2, lcl));
    }
    int nl = 0;
    for (int a = 0; a < 3; a++) { dims[0][a] = n[a]; ratios[0][a] = 0; }
    nl = 1;
    while (nl < MAXLV) {
        int r[3], any = 0, all = 1;
        for (int a = 0; a < 3; a++) {
            int c = dims[nl - 1][a];
            if (c <= avail[a]) { r[a] = 0; all = 0; }
            else if (c >= 256) { r[a] = 2; while (c / r[a] >= 256) r[a] *= 2; any = 1; }
            else { r[a] = 2; any = 1; }
        }
        if (!any) break;
        if (!all) return -2; /* axes that stop coarsening at different depths */
        for (int a = 0; a < 3; a++) { ratios[nl][a] = r[a]; dims[nl][a] = dims[nl - 1][a] / r[a]; }
        nl++;
    }
    return nl;
}

/* ------------------------------------------------------------------------- */
/* multigrid context                                                          */
/* ------------------------------------------------------------------------- */
typedef struct {
    int n[3];
    long nv;
    int ratio[3]; /* ratio to the finer level (0 on level 0) */
    double *u, *f, *r;
    double *st; /* coarse levels: [nv][27][9] */
} ora_level;

typedef struct {
    int nl;
    ora_level lv[MAXLV];
    double ke[576];
    double E, nu;
    double *rho; /* physical density rho^p on level 0, lexicographic */
    /* coarsest dense LU */
    int ndof;
    double *lu;
    int *piv;
    int fp16; /* coarse stencil storage: 1 FP16 (the reference's), 0 FP64, 3 FP32 */
    int project; /* remove rigid translations from the coarsest right-hand side */
    int pin_identity; /* add the identity block at the pinned node (reference patch) */
} ora_mg;

ora_mg *ora_mg_create(const int reso[3], double E, double nu) {
    int dims[MAXLV][3], rat[MAXLV][3];
    int nl = ora_hierarchy(reso, dims, rat);
    if (nl < 2) return NULL;
    ora_mg *m = (ora_mg *)calloc(1, sizeof(ora_mg));
    m->nl = nl;
    m->E = E; m->nu = nu;
    m->fp16 = 1;
    m->project = 0;
    m->pin_identity = 1;
    ora_ke(E, nu, m->ke);
    for (int l = 0; l < nl; l++) {
        ora_level *L = &m->lv[l];
        for (int a = 0; a < 3; a++) { L->n[a] = dims[l][a]; L->ratio[a] = rat[l][a]; }
        L->nv = (long)L->n[0] * L->n[1] * L->n[2];
        L->u = (double *)calloc(L->nv * NF, sizeof(double));
        L->f = (double *)calloc(L->nv * NF, sizeof(double));
        L->r = (double *)calloc(L->nv * NF, sizeof(double));
        if (l > 0) L->st = (double *)calloc(L->nv * 243, sizeof(double));
    }
    m->rho = (double *)calloc(m->lv[0].nv, sizeof(double));
    ora_level *C = &m->lv[nl - 1];
    m->ndof = (int)(3 * C->nv);
    m->lu = (double *)calloc((size_t)m->ndof * m->ndof, sizeof(double));
    m->piv = (int *)calloc(m->ndof, sizeof(int));
    return m;
}

void ora_mg_destroy(ora_mg *m) {
    if (!m) return;
    for (int l = 0; l < m->nl; l++) {
        free(m->lv[l].u); free(m->lv[l].f); free(m->lv[l].r); free(m->lv[l].st);
    }
    free(m->rho); free(m->lu); free(m->piv);
    free(m);
}

int ora_mg_nlevels(const ora_mg *m) { return m->nl; }
void ora_mg_level_info(const ora_mg *m, int l, int dims[3], int ratio[3]) {
    for (int a = 0; a < 3; a++) { dims[a] = m->lv[l].n[a]; ratio[a] = m->lv[l].ratio[a]; }
}
double *ora_mg_field(ora_mg *m, int l, int which) {
    ora_level *L = &m->lv[l];
    return which == 0 ? L->u : which == 1 ? L->f : which == 2 ? L->r : L->st;
}
void ora_mg_ke(const ora_mg *m, double ke[576]) { memcpy(ke, m->ke, sizeof(double) * 576); }
void ora_mg_set_fp16(ora_mg *m, int on) { m->fp16 = on; }
void ora_mg_set_project(ora_mg *m, int on) { m->project = on; }
void ora_mg_set_pin_identity(ora_mg *m, int on) { m->pin_identity = on; }
void ora_mg_set_density(ora_mg *m, const double *rho) {
    memcpy(m->rho, rho, sizeof(double) * m->lv[0].nv);
}

/* ------------------------------------------------------------------------- */
/* right-hand side: f_i = K(rho) chi0_i (grid.cu:1818-1919)                    */
/* ------------------------------------------------------------------------- */
void ora_mg_rhs(ora_mg *m) {
    ora_level *L = &m->lv[0];
    const int *n = L->n;
    double g[NCASE][24]; /* Ke * chi0_c */
    for (int c = 0; c < NCASE; c++)
        for (int a = 0; a < 24; a++) {
            double s = 0;
            for (int b = 0; b < 8; b++) {
                double ub[3];
                macro_disp(b, c, ub);
                for (int k = 0; k < 3; k++) s += m->ke[a * 24 + 3 * b + k] * ub[k];
            }
            g[c][a] = s;
        }
#pragma omp parallel for collapse(2)
    for (int z = 0; z < n[2]; z++)
        for (int y = 0; y < n[1]; y++)
            for (int x = 0; x < n[0]; x++) {
                double acc[NF] = {0};
                for (int w = 0; w < 8; w++) {
                    int ex = wrapi(x - 1 + w % 2, n[0]), ey = wrapi(y - 1 + w / 2 % 2, n[1]),
                        ez = wrapi(z - 1 + w / 4, n[2]);
                    double rp = RHO_PENAL_MIN + m->rho[lexid(ex, ey, ez, n)];
                    int a = 7 - w;
                    for (int c = 0; c < NCASE; c++)
                        for (int k = 0; k < 3; k++) acc[c * 3 + k] += rp * g[c][3 * a + k];
                }
                memcpy(&L->f[lexid(x, y, z, n) * NF], acc, sizeof(acc));
            }
}

/* ------------------------------------------------------------------------- */
/* fine level: matrix-free Gauss-Seidel and residual (grid.cu:323-551, 1277-1461) */
/* ------------------------------------------------------------------------- */
static inline int is_origin(int x, int y, int z) { return x == 0 && y == 0 && z == 0; }

/* sum over the 8 elements of vertex (x,y,z): rho_e * Ke[row block of v][nodes]
 * applied to u; with_self selects whether the vertex's own node is included;
 * returns the 3x3 self block in ks when non-NULL */
static void fine_apply(const ora_mg *m, const double *u, int x, int y, int z, int with_self,
                       double acc[NF], double ks[9]) {
    const int *n = m->lv[0].n;
    memset(acc, 0, sizeof(double) * NF);
    if (ks) memset(ks, 0, sizeof(double) * 9);
    for (int w = 0; w < 8; w++) {
        int e0[3] = {x - 1 + w % 2, y - 1 + w / 2 % 2, z - 1 + w / 4};
        int ex = wrapi(e0[0], n[0]), ey = wrapi(e0[1], n[1]), ez = wrapi(e0[2], n[2]);
        double rp = RHO_PENAL_MIN + m->rho[lexid(ex, ey, ez, n)];
        int a = 7 - w;
        double ku[NF] = {0};
        for (int b = 0; b < 8; b++) {
            if (b == a && !with_self) continue;
            int vx = wrapi(e0[0] + b % 2, n[0]), vy = wrapi(e0[1] + b / 2 % 2, n[1]),
                vz = wrapi(e0[2] + b / 4, n[2]);
            if (is_origin(vx, vy, vz)) continue; /* Dirichlet pin: u = 0 */
            const double *un = &u[lexid(vx, vy, vz, n) * NF];
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) {
                    double k = m->ke[(3 * a + r) * 24 + 3 * b + c];
                    for (int q = 0; q < NCASE; q++) ku[q * 3 + r] += k * un[q * 3 + c];
                }
        }
        for (int i = 0; i < NF; i++) acc[i] += rp * ku[i];
        if (ks)
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) ks[3 * r + c] += rp * m->ke[(3 * a + r) * 24 + 3 * a + c];
    }
}

static void block_gs_update(double *uv, const double *fv, const double acc[NF], const double ks[9], double w) {
    for (int q = 0; q < NCASE; q++) {
        double *u = uv + 3 * q;
        const double *f = fv + 3 * q;
        const double *a = acc + 3 * q;
        u[0] = w * (f[0] - a[0] - ks[1] * u[1] - ks[2] * u[2]) / ks[0] + (1 - w) * u[0];
        u[1] = w * (f[1] - a[1] - ks[3] * u[0] - ks[5] * u[2]) / ks[4] + (1 - w) * u[1];
        u[2] = w * (f[2] - a[2] - ks[6] * u[0] - ks[7] * u[1]) / ks[8] + (1 - w) * u[2];
    }
}

static void fine_gs(ora_mg *m, double w) {
    ora_level *L = &m->lv[0];
    const int *n = L->n;
    for (int col = 0; col < 8; col++) {
        int px = ((col & 1) ^ 1), py = (((col >> 1) & 1) ^ 1), pz = (((col >> 2) & 1) ^ 1);
#pragma omp parallel for collapse(2)
        for (int z = pz; z < n[2]; z += 2)
            for (int y = py; y < n[1]; y += 2)
                for (int x = px; x < n[0]; x += 2) {
                    double *uv = &L->u[lexid(x, y, z, n) * NF];
                    if (is_origin(x, y, z)) { memset(uv, 0, sizeof(double) * NF); continue; }
                    double acc[NF], ks[9];
                    fine_apply(m, L->u, x, y, z, 0, acc, ks);
                    block_gs_update(uv, &L->f[lexid(x, y, z, n) * NF], acc, ks, w);
                }
    }
}

static void fine_residual(ora_mg *m) {
    ora_level *L = &m->lv[0];
    const int *n = L->n;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < n[2]; z++)
        for (int y = 0; y < n[1]; y++)
            for (int x = 0; x < n[0]; x++) {
                long v = lexid(x, y, z, n);
                double *rv = &L->r[v * NF];
                if (is_origin(x, y, z)) { memset(rv, 0, sizeof(double) * NF); continue; }
                double acc[NF];
                fine_apply(m, L->u, x, y, z, 1, acc, NULL);
                for (int i = 0; i < NF; i++) rv[i] = L->f[v * NF + i] - acc[i];
            }
}

/* ------------------------------------------------------------------------- */
/* coarse levels: stored 27-point stencils (grid.cu:556-689, 1465-1564)        */
/* ------------------------------------------------------------------------- */
static void stencil_apply(const ora_level *L, int x, int y, int z, int with_self, double acc[NF]) {
    const int *n = L->n;
    const double *st = &L->st[lexid(x, y, z, n) * 243];
    memset(acc, 0, sizeof(double) * NF);
    for (int d = 0; d < 27; d++) {
        if (d == 13 && !with_self) continue;
        int vx = wrapi(x + d % 3 - 1, n[0]), vy = wrapi(y + d / 3 % 3 - 1, n[1]),
            vz = wrapi(z + d / 9 - 1, n[2]);
        const double *un = &L->u[lexid(vx, vy, vz, n) * NF];
        const double *s = st + 9 * d;
        for (int q = 0; q < NCASE; q++)
            for (int r = 0; r < 3; r++)
                acc[q * 3 + r] += s[3 * r] * un[q * 3] + s[3 * r + 1] * un[q * 3 + 1] + s[3 * r + 2] * un[q * 3 + 2];
    }
}

static void coarse_gs(ora_mg *m, int l, double w) {
    ora_level *L = &m->lv[l];
    const int *n = L->n;
    for (int col = 0; col < 8; col++) {
        int px = ((col & 1) ^ 1), py = (((col >> 1) & 1) ^ 1), pz = (((col >> 2) & 1) ^ 1);
#pragma omp parallel for collapse(2)
        for (int z = pz; z < n[2]; z += 2)
            for (int y = py; y < n[1]; y += 2)
                for (int x = px; x < n[0]; x += 2) {
                    long v = lexid(x, y, z, n);
                    double acc[NF];
                    stencil_apply(L, x, y, z, 0, acc);
                    block_gs_update(&L->u[v * NF], &L->f[v * NF], acc, &L->st[v * 243 + 9 * 13], w);
                }
    }
}

static void coarse_residual(ora_mg *m, int l) {
    ora_level *L = &m->lv[l];
    const int *n = L->n;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < n[2]; z++)
        for (int y = 0; y < n[1]; y++)
            for (int x = 0; x < n[0]; x++) {
                long v = lexid(x, y, z, n);
                double acc[NF];
                stencil_apply(L, x, y, z, 1, acc);
                for (int i = 0; i < NF; i++) L->r[v * NF + i] = L->f[v * NF + i] - acc[i];
            }
}

void ora_mg_gs(ora_mg *m, int l, double w) { if (l == 0) fine_gs(m, w); else coarse_gs(m, l, w); }
void ora_mg_residual(ora_mg *m, int l) { if (l == 0) fine_residual(m); else coarse_residual(m, l); }

/* ------------------------------------------------------------------------- */
/* transfers (grid.cu:917-994, 1120-1190, homoCommon.cuh:350-385)             */
/* ------------------------------------------------------------------------- */
/* full weighting: f_c(X) = sum_{|o|<r} prod(r-|o|)/r^3 * r_f(r X + o)  on level lc */
void ora_mg_restrict(ora_mg *m, int lc) {
    ora_level *C = &m->lv[lc], *F = &m->lv[lc - 1];
    const int *r = C->ratio;
    double pr = (double)r[0] * r[1] * r[2];
#pragma omp parallel for collapse(2)
    for (int z = 0; z < C->n[2]; z++)
        for (int y = 0; y < C->n[1]; y++)
            for (int x = 0; x < C->n[0]; x++) {
                double acc[NF] = {0};
                for (int ox = -r[0] + 1; ox < r[0]; ox++)
                    for (int oy = -r[1] + 1; oy < r[1]; oy++)
                        for (int oz = -r[2] + 1; oz < r[2]; oz++) {
                            double w = (double)(r[0] - abs(ox)) * (r[1] - abs(oy)) * (r[2] - abs(oz)) / pr;
                            long fv = lexid(wrapi(r[0] * x + ox, F->n[0]), wrapi(r[1] * y + oy, F->n[1]),
                                            wrapi(r[2] * z + oz, F->n[2]), F->n);
                            for (int i = 0; i < NF; i++) acc[i] += w * F->r[fv * NF + i];
                        }
                memcpy(&C->f[lexid(x, y, z, C->n) * NF], acc, sizeof(acc));
            }
}

/* trilinear prolongation u_f += P u_c on level lf (Dirichlet origin skipped on level 0) */
void ora_mg_prolong(ora_mg *m, int lf) {
    ora_level *F = &m->lv[lf], *C = &m->lv[lf + 1];
    const int *r = C->ratio;
    double pr = (double)r[0] * r[1] * r[2];
#pragma omp parallel for collapse(2)
    for (int z = 0; z < F->n[2]; z++)
        for (int y = 0; y < F->n[1]; y++)
            for (int x = 0; x < F->n[0]; x++) {
                if (lf == 0 && is_origin(x, y, z)) continue;
                int p[3] = {x, y, z}, rem[3], base[3];
                for (int a = 0; a < 3; a++) { rem[a] = p[a] % r[a]; base[a] = p[a] / r[a]; }
                double acc[NF] = {0};
                for (int id = 0; id < 8; id++) {
                    int o[3] = {id % 2, id / 2 % 2, id / 4};
                    double w = 1;
                    for (int a = 0; a < 3; a++) w *= (double)(r[a] - abs(o[a] * r[a] - rem[a]));
                    w /= pr;
                    if (w == 0) continue;
                    long cv = lexid(wrapi(base[0] + o[0], C->n[0]), wrapi(base[1] + o[1], C->n[1]),
                                    wrapi(base[2] + o[2], C->n[2]), C->n);
                    for (int i = 0; i < NF; i++) acc[i] += w * C->u[cv * NF + i];
                }
                double *uf = &F->u[lexid(x, y, z, F->n) * NF];
                for (int i = 0; i < NF; i++) uf[i] += acc[i];
            }
}

/* ------------------------------------------------------------------------- */
/* Galerkin coarse operators (grid_ex.cu:936-1160, grid.cu:2383-2439,          */
/* grid.cu:3103-3176, grid.cpp:1184-1325)                                      */
/* ------------------------------------------------------------------------- */
static inline double hat_w(const int off[3], const int r[3]) {
    /* prod (r - |off|) / r^3, zero outside |off| < r */
    double w = 1;
    for (int a = 0; a < 3; a++) {
        int o = abs(off[a]);
        if (o >= r[a]) return 0;
        w *= (double)(r[a] - o);
    }
    return w / ((double)r[0] * r[1] * r[2]);
}

static void clamp_diag(double s[9]) {
    for (int k = 0; k < 3; k++)
        if (fabs(s[4 * k]) < 1e-4) s[4 * k] = 1e-4;
}

/* stencil of coarse lexicographic vertex X (coordinates may equal n_c, the
 * periodic image of 0) from fine elements clipped to [0, n_f): the reference's
 * level-1 kernel (grid_ex.cu:936-1060), rho_penal = rho^p without the 1e-9 floor */
static void l1_partial(const ora_mg *m, int lc, const int X[3], double st[243]) {
    const ora_level *F = &m->lv[lc - 1], *C = &m->lv[lc];
    const int *r = C->ratio, *nf = F->n;
    int vi[3] = {X[0] * r[0], X[1] * r[1], X[2] * r[2]};
    memset(st, 0, sizeof(double) * 243);
    for (int d = 0; d < 27; d++) {
        int dj[3] = {r[0] * (d % 3 - 1), r[1] * (d / 3 % 3 - 1), r[2] * (d / 9 - 1)};
        double *s = st + 9 * d;
        for (int ex = -r[0]; ex < r[0]; ex++)
            for (int ey = -r[1]; ey < r[1]; ey++)
                for (int ez = -r[2]; ez < r[2]; ez++) {
                    int eo[3] = {dj[0] + ex, dj[1] + ey, dj[2] + ez};
                    if (eo[0] < -r[0] || eo[0] >= r[0] || eo[1] < -r[1] || eo[1] >= r[1] || eo[2] < -r[2] ||
                        eo[2] >= r[2])
                        continue;
                    int ep[3] = {vi[0] + eo[0], vi[1] + eo[1], vi[2] + eo[2]};
                    if (ep[0] < 0 || ep[0] >= nf[0] || ep[1] < 0 || ep[1] >= nf[1] || ep[2] < 0 || ep[2] >= nf[2])
                        continue;
                    double rp = m->rho[lexid(ep[0], ep[1], ep[2], nf)];
                    for (int a = 0; a < 8; a++) {
                        int ao[3] = {eo[0] + a % 2, eo[1] + a / 2 % 2, eo[2] + a / 4};
                        double wi = hat_w(ao, r);
                        if (wi == 0) continue;
                        for (int b = 0; b < 8; b++) {
                            int bo[3] = {eo[0] + b % 2 - dj[0], eo[1] + b / 2 % 2 - dj[1], eo[2] + b / 4 - dj[2]};
                            double wj = hat_w(bo, r);
                            if (wj == 0) continue;
                            double ww = wi * rp * wj;
                            for (int i = 0; i < 3; i++)
                                for (int j = 0; j < 3; j++) s[3 * i + j] += ww * m->ke[(3 * a + i) * 24 + 3 * b + j];
                        }
                    }
                }
    }
}

/* periodic image combination of the level-1 partial stencils: each partial is
 * diagonal-clamped and FP16-rounded by itself, then the images are summed in
 * FP16 in the order x-image, y-image, z-image (grid.cu:3103-3176) */
static void l1_combine(const ora_mg *m, int lc, int x, int y, int z, double out[243],
                       void (*partial)(const ora_mg *, int, const int *, double *)) {
    const ora_level *C = &m->lv[lc];
    int nimg[3] = {x == 0 ? 2 : 1, y == 0 ? 2 : 1, z == 0 ? 2 : 1};
    double acc[243];
    for (int k = 0; k < 243; k++) acc[k] = 0;
    int first = 1;
    for (int i = 0; i < nimg[0]; i++)
        for (int j = 0; j < nimg[1]; j++)
            for (int k = 0; k < nimg[2]; k++) {
                int X[3] = {x + i * C->n[0], y + j * C->n[1], z + k * C->n[2]};
                double p[243];
                partial(m, lc, X, p);
                clamp_diag(p + 9 * 13);
                if (m->fp16 == 1) {
                    for (int q = 0; q < 243; q++) {
                        p[q] = to_half(p[q]);
                        /* FP16 accumulation: each sum correctly rounded to half (native
                         * half add); the double sum of two halves is exact */
                        acc[q] = to_half(acc[q] + p[q]);
                    }
                } else {
                    for (int q = 0; q < 243; q++) acc[q] += p[q];
                }
                first = 0;
            }
    (void)first;
    if (m->fp16 == 3) round_row_f32(acc);
    memcpy(out, acc, sizeof(acc));
}

/* the 27 coarse vertices around the pinned fine origin, recomputed with the
 * pinned fine operator (identity at the origin node, 1e-9 floor on rho) in
 * double and rounded once (grid.cpp:1184-1325) */
static void l1_dirichlet_patch(const ora_mg *m, int lc, const int Xoff[3], double st[243]) {
    const ora_level *F = &m->lv[lc - 1];
    const int *r = m->lv[lc].ratio, *nf = F->n;
    int vi[3] = {Xoff[0] * r[0], Xoff[1] * r[1], Xoff[2] * r[2]};
    memset(st, 0, sizeof(double) * 243);
    for (int d = 0; d < 27; d++) {
        int vj[3] = {vi[0] + (d % 3 - 1) * r[0], vi[1] + (d / 3 % 3 - 1) * r[1], vi[2] + (d / 9 - 1) * r[2]};
        double *s = st + 9 * d;
        for (int ex = -r[0]; ex < r[0]; ex++)
            for (int ey = -r[1]; ey < r[1]; ey++)
                for (int ez = -r[2]; ez < r[2]; ez++) {
                    int ep[3] = {vj[0] + ex, vj[1] + ey, vj[2] + ez};
                    int eoi[3] = {ep[0] - vi[0], ep[1] - vi[1], ep[2] - vi[2]};
                    if (eoi[0] >= r[0] || eoi[0] < -r[0] || eoi[1] >= r[1] || eoi[1] < -r[1] || eoi[2] >= r[2] ||
                        eoi[2] < -r[2])
                        continue;
                    double rp = RHO_PENAL_MIN +
                                m->rho[lexid(wrapi(ep[0], nf[0]), wrapi(ep[1], nf[1]), wrapi(ep[2], nf[2]), nf)];
                    for (int a = 0; a < 8; a++) {
                        int ap[3] = {ep[0] + a % 2, ep[1] + a / 2 % 2, ep[2] + a / 4};
                        int ao[3] = {ap[0] - vi[0], ap[1] - vi[1], ap[2] - vi[2]};
                        double wi = hat_w(ao, r);
                        if (wi == 0) continue;
                        int ad = ap[0] == 0 && ap[1] == 0 && ap[2] == 0;
                        for (int b = 0; b < 8; b++) {
                            int bp[3] = {ep[0] + b % 2, ep[1] + b / 2 % 2, ep[2] + b / 4};
                            int bo[3] = {bp[0] - vj[0], bp[1] - vj[1], bp[2] - vj[2]};
                            double wj = hat_w(bo, r);
                            if (wj == 0) continue;
                            int bd = bp[0] == 0 && bp[1] == 0 && bp[2] == 0;
                            if (ad || bd) {
                                if (a == b && m->pin_identity)
                                    for (int i = 0; i < 3; i++) s[4 * i] += wi * wj;
                            } else {
                                for (int i = 0; i < 3; i++)
                                    for (int j = 0; j < 3; j++)
                                        s[3 * i + j] += wi * wj * rp * m->ke[(3 * a + i) * 24 + 3 * b + j];
                            }
                        }
                    }
                }
    }
    clamp_diag(st + 9 * 13);
    if (m->fp16 == 1)
        for (int q = 0; q < 243; q++) st[q] = to_half(st[q]);
    else if (m->fp16 == 3)
        round_row_f32(st);
}

/* fast restatement of l1_partial: coarse element matrices
 * K_E = sum_s rho_s P_s^T Ke P_s (exact algebraic refactoring of the same sum) */
static double *g_q = NULL; /* [nsub][576] for the current ratio */
static int g_qr[3] = {0, 0, 0};
static double g_qke[576];
static void build_q(const ora_mg *m, const int r[3]) {
    if (g_q && g_qr[0] == r[0] && g_qr[1] == r[1] && g_qr[2] == r[2] && !memcmp(g_qke, m->ke, sizeof(g_qke))) return;
    free(g_q);
    int ns = r[0] * r[1] * r[2];
    g_q = (double *)calloc((size_t)ns * 576, sizeof(double));
    memcpy(g_qr, r, sizeof(g_qr));
    memcpy(g_qke, m->ke, sizeof(g_qke));
    for (int s = 0; s < ns; s++) {
        int so[3] = {s % r[0], s / r[0] % r[1], s / (r[0] * r[1])};
        double P[8][8]; /* P[fine node][coarse node] */
        for (int a = 0; a < 8; a++)
            for (int b = 0; b < 8; b++) {
                int fo[3] = {so[0] + a % 2, so[1] + a / 2 % 2, so[2] + a / 4};
                int co[3] = {(b % 2) * r[0], (b / 2 % 2) * r[1], (b / 4) * r[2]};
                int off[3] = {fo[0] - co[0], fo[1] - co[1], fo[2] - co[2]};
                double w = 1;
                for (int q = 0; q < 3; q++) {
                    int o = abs(off[q]);
                    w *= o >= r[q] ? 0 : (double)(r[q] - o) / r[q];
                }
                P[a][b] = w;
            }
        double *Q = g_q + (size_t)s * 576;
        for (int A = 0; A < 8; A++)
            for (int B = 0; B < 8; B++)
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) {
                        double v = 0;
                        for (int a = 0; a < 8; a++) {
                            if (P[a][A] == 0) continue;
                            for (int b = 0; b < 8; b++)
                                v += P[a][A] * P[b][B] * m->ke[(3 * a + i) * 24 + 3 * b + j];
                        }
                        Q[(3 * A + i) * 24 + 3 * B + j] = v;
                    }
    }
}

static void l1_partial_fast(const ora_mg *m, int lc, const int X[3], double st[243]) {
    const ora_level *F = &m->lv[lc - 1], *C = &m->lv[lc];
    const int *r = C->ratio, *nf = F->n, *nc = C->n;
    int ns = r[0] * r[1] * r[2];
    memset(st, 0, sizeof(double) * 243);
    for (int l = 0; l < 8; l++) {            /* local node of X in coarse element E = X - l */
        int E[3] = {X[0] - l % 2, X[1] - l / 2 % 2, X[2] - l / 4};
        if (E[0] < 0 || E[0] >= nc[0] || E[1] < 0 || E[1] >= nc[1] || E[2] < 0 || E[2] >= nc[2]) continue;
        for (int mm = 0; mm < 8; mm++) {
            int d[3] = {mm % 2 - l % 2, mm / 2 % 2 - l / 2 % 2, mm / 4 - l / 4};
            double *s = st + 9 * ((d[0] + 1) + 3 * (d[1] + 1) + 9 * (d[2] + 1));
            for (int q = 0; q < ns; q++) {
                int so[3] = {q % r[0], q / r[0] % r[1], q / (r[0] * r[1])};
                double rp = m->rho[lexid(E[0] * r[0] + so[0], E[1] * r[1] + so[1], E[2] * r[2] + so[2], nf)];
                const double *Q = g_q + (size_t)q * 576;
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) s[3 * i + j] += rp * Q[(3 * l + i) * 24 + 3 * mm + j];
            }
        }
    }
}

static int near_origin(int x, int n) { return x == 0 || x == 1 || x == n - 1; }

/* level-1 stencils; method 0 = reference loop nest, 1 = coarse-element refactoring */
void ora_mg_galerkin_l1(ora_mg *m, int method) {
    ora_level *C = &m->lv[1];
    const int *n = C->n;
    build_q(m, C->ratio);
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int z = 0; z < n[2]; z++)
        for (int y = 0; y < n[1]; y++)
            for (int x = 0; x < n[0]; x++) {
                double *st = &C->st[lexid(x, y, z, n) * 243];
                if (near_origin(x, n[0]) && near_origin(y, n[1]) && near_origin(z, n[2])) {
                    int off[3] = {x == n[0] - 1 ? -1 : x, y == n[1] - 1 ? -1 : y, z == n[2] - 1 ? -1 : z};
                    l1_dirichlet_patch(m, 1, off, st);
                } else {
                    l1_combine(m, 1, x, y, z, st, method ? l1_partial_fast : l1_partial);
                }
            }
}

/* deeper levels: R A P from the stored finer stencil (grid_ex.cu:1065-1160) */
void ora_mg_galerkin(ora_mg *m, int lc) {
    ora_level *C = &m->lv[lc], *F = &m->lv[lc - 1];
    const int *r = C->ratio;
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int z = 0; z < C->n[2]; z++)
        for (int y = 0; y < C->n[1]; y++)
            for (int x = 0; x < C->n[0]; x++) {
                double *st = &C->st[lexid(x, y, z, C->n) * 243];
                for (int d = 0; d < 27; d++) {
                    int dj[3] = {r[0] * (d % 3 - 1), r[1] * (d / 3 % 3 - 1), r[2] * (d / 9 - 1)};
                    double s[9] = {0};
                    for (int fx = -r[0]; fx <= r[0]; fx++)
                        for (int fy = -r[1]; fy <= r[1]; fy++)
                            for (int fz = -r[2]; fz <= r[2]; fz++) {
                                int oi[3] = {fx + dj[0], fy + dj[1], fz + dj[2]};
                                double wi = hat_w(oi, r);
                                if (wi == 0) continue;
                                long fv = lexid(wrapi(r[0] * x + oi[0], F->n[0]), wrapi(r[1] * y + oi[1], F->n[1]),
                                                wrapi(r[2] * z + oi[2], F->n[2]), F->n);
                                const double *fst = &F->st[fv * 243];
                                for (int j = 0; j < 27; j++) {
                                    int oj[3] = {oi[0] + j % 3 - 1 - dj[0], oi[1] + j / 3 % 3 - 1 - dj[1],
                                                 oi[2] + j / 9 - 1 - dj[2]};
                                    double wj = hat_w(oj, r);
                                    if (wj == 0) continue;
                                    for (int k = 0; k < 9; k++) s[k] += wi * wj * fst[9 * j + k];
                                }
                            }
                    if (d == 13) clamp_diag(s);
                    for (int k = 0; k < 9; k++) st[9 * d + k] = m->fp16 == 1 ? to_half(s[k]) : s[k];
                }
                if (m->fp16 == 3) round_row_f32(st);
            }
}

/* ------------------------------------------------------------------------- */
/* coarsest level: dense LU, right-hand side with rigid translations removed   */
/* ------------------------------------------------------------------------- */
static int lu_factor(double *A, int n, int *piv) {
    for (int k = 0; k < n; k++) {
        int p = k;
        double mx = fabs(A[(size_t)k * n + k]);
        for (int i = k + 1; i < n; i++)
            if (fabs(A[(size_t)i * n + k]) > mx) { mx = fabs(A[(size_t)i * n + k]); p = i; }
        piv[k] = p;
        if (mx == 0) return -1;
        if (p != k)
            for (int j = 0; j < n; j++) {
                double t = A[(size_t)k * n + j]; A[(size_t)k * n + j] = A[(size_t)p * n + j]; A[(size_t)p * n + j] = t;
            }
        double inv = 1.0 / A[(size_t)k * n + k];
        for (int i = k + 1; i < n; i++) {
            double l = A[(size_t)i * n + k] * inv;
            A[(size_t)i * n + k] = l;
            if (l != 0)
                for (int j = k + 1; j < n; j++) A[(size_t)i * n + j] -= l * A[(size_t)k * n + j];
        }
    }
    return 0;
}
static void lu_solve(const double *A, int n, const int *piv, double *b) {
    for (int k = 0; k < n; k++) { int p = piv[k]; if (p != k) { double t = b[k]; b[k] = b[p]; b[p] = t; } }
    for (int i = 0; i < n; i++) { double s = b[i]; for (int j = 0; j < i; j++) s -= A[(size_t)i * n + j] * b[j]; b[i] = s; }
    for (int i = n - 1; i >= 0; i--) {
        double s = b[i];
        for (int j = i + 1; j < n; j++) s -= A[(size_t)i * n + j] * b[j];
        b[i] = s / A[(size_t)i * n + i];
    }
}

/* dense matrix of the coarsest stencil over unique DOFs (grid.cpp:844-915) */
void ora_mg_coarse_matrix(ora_mg *m, double *K) {
    ora_level *C = &m->lv[m->nl - 1];
    int nd = m->ndof;
    memset(K, 0, sizeof(double) * nd * nd);
    for (int z = 0; z < C->n[2]; z++)
        for (int y = 0; y < C->n[1]; y++)
            for (int x = 0; x < C->n[0]; x++) {
                long v = lexid(x, y, z, C->n);
                for (int d = 0; d < 27; d++) {
                    long w = lexid(wrapi(x + d % 3 - 1, C->n[0]), wrapi(y + d / 3 % 3 - 1, C->n[1]),
                                   wrapi(z + d / 9 - 1, C->n[2]), C->n);
                    for (int i = 0; i < 3; i++)
                        for (int j = 0; j < 3; j++) K[(3 * v + i) * nd + 3 * w + j] += C->st[v * 243 + 9 * d + 3 * i + j];
                }
            }
}

int ora_mg_coarse_factor(ora_mg *m) {
    ora_mg_coarse_matrix(m, m->lu);
    return lu_factor(m->lu, m->ndof, m->piv);
}

void ora_mg_coarse_solve(ora_mg *m) {
    ora_level *C = &m->lv[m->nl - 1];
    int nd = m->ndof;
    long nv = C->nv;
    double *b = (double *)malloc(sizeof(double) * nd);
    for (int q = 0; q < NCASE; q++) {
        double mean[3] = {0, 0, 0};
        for (long v = 0; v < nv; v++)
            for (int i = 0; i < 3; i++) mean[i] += C->f[v * NF + 3 * q + i];
        for (int i = 0; i < 3; i++) mean[i] = m->project ? mean[i] / (double)nv : 0;
        for (long v = 0; v < nv; v++)
            for (int i = 0; i < 3; i++) b[3 * v + i] = C->f[v * NF + 3 * q + i] - mean[i];
        lu_solve(m->lu, nd, m->piv, b);
        for (long v = 0; v < nv; v++)
            for (int i = 0; i < 3; i++) C->u[v * NF + 3 * q + i] = b[3 * v + i];
    }
    free(b);
}

void ora_mg_update_stencils(ora_mg *m, int l1_method) {
    ora_mg_galerkin_l1(m, l1_method);
    for (int l = 2; l < m->nl; l++) ora_mg_galerkin(m, l);
    ora_mg_coarse_factor(m);
}

/* ------------------------------------------------------------------------- */
/* V-cycle and solve (MG.cpp:46-70, 113-203)                                   */
/* ------------------------------------------------------------------------- */
void ora_mg_vcycle(ora_mg *m, double w) {
    for (int l = 0; l < m->nl; l++) {
        if (l > 0) {
            ora_mg_residual(m, l - 1);
            ora_mg_restrict(m, l);
            memset(m->lv[l].u, 0, sizeof(double) * m->lv[l].nv * NF);
        }
        if (l == m->nl - 1) ora_mg_coarse_solve(m);
        else ora_mg_gs(m, l, w);
    }
    for (int l = m->nl - 2; l >= 0; l--) {
        ora_mg_prolong(m, l);
        ora_mg_gs(m, l, w);
    }
}

/* multiplicity of a unique vertex in the reference's padded periodic storage:
 * positions 0, 1 and n-1 appear twice per axis (grid.cpp:155-198) */
static inline int axis_mult(int x, int n) { return (x == 0 || x == 1 || x == n - 1) ? 2 : 1; }

/* per-case norms with the padded-storage multiplicities */
void ora_weighted_norm(const int n[3], const double *v, double out[NCASE]) {
    double s[NCASE] = {0};
    for (int z = 0; z < n[2]; z++)
        for (int y = 0; y < n[1]; y++)
            for (int x = 0; x < n[0]; x++) {
                double w = axis_mult(x, n[0]) * axis_mult(y, n[1]) * axis_mult(z, n[2]);
                const double *p = &v[lexid(x, y, z, n) * NF];
                for (int q = 0; q < NCASE; q++)
                    s[q] += w * (p[3 * q] * p[3 * q] + p[3 * q + 1] * p[3 * q + 1] + p[3 * q + 2] * p[3 * q + 2]);
            }
    for (int q = 0; q < NCASE; q++) out[q] = sqrt(s[q]);
}

/* remove the mean displacement over unique vertices (grid.cpp:1131-1141) */
void ora_mg_remove_mean(ora_mg *m) {
    ora_level *L = &m->lv[0];
    double mean[NF] = {0};
    for (long v = 0; v < L->nv; v++)
        for (int i = 0; i < NF; i++) mean[i] += L->u[v * NF + i];
    for (int i = 0; i < NF; i++) mean[i] /= (double)L->nv;
    for (long v = 0; v < L->nv; v++)
        for (int i = 0; i < NF; i++) L->u[v * NF + i] -= mean[i];
}

/* repeat V-cycles until every case has ||r||/||f|| <= tol (stale residual taken
 * after pre-smoothing, as the reference does); returns the number of cycles;
 * hist receives [cycle][6] relative residuals (up to maxit rows) */
/* Rigid-translation deflation after each V-cycle of a solve (the CUDA library's
 * k_pin_deflate): in the pinned system the translation t' (1 on every vertex but
 * the origin) has energy t'^T K t' = A_pp, the origin's unpinned self block, and
 * the residual's translation component is s = sum_{v != 0} f_v + (K u)_origin
 * (the columns of the periodic operator sum to zero).  u += A_pp^-1 s on every
 * vertex but the origin removes the error in that mode exactly.  The reference
 * has no such step (it projects the translations out of the coarsest right-hand
 * side, grid.cpp:349-374). */
static void pin_deflate(ora_mg *m) {
    ora_level *L = &m->lv[0];
    const int *n = L->n;
    double F[NF] = {0};
    for (long v = 1; v < L->nv; v++)
        for (int i = 0; i < NF; i++) F[i] += L->f[v * NF + i];
    double q[NF], A[9];
    fine_apply(m, L->u, 0, 0, 0, 0, q, A);
    const double c00 = A[4] * A[8] - A[5] * A[7], c01 = A[5] * A[6] - A[3] * A[8], c02 = A[3] * A[7] - A[4] * A[6];
    const double det = A[0] * c00 + A[1] * c01 + A[2] * c02;
    if (!(det > 0)) return;
    const double inv[9] = {c00 / det, (A[2] * A[7] - A[1] * A[8]) / det, (A[1] * A[5] - A[2] * A[4]) / det,
                           c01 / det, (A[0] * A[8] - A[2] * A[6]) / det, (A[2] * A[3] - A[0] * A[5]) / det,
                           c02 / det, (A[1] * A[6] - A[0] * A[7]) / det, (A[0] * A[4] - A[1] * A[3]) / det};
    double al[NF];
    for (int c = 0; c < NCASE; c++)
        for (int r = 0; r < 3; r++) {
            al[3 * c + r] = 0;
            for (int k = 0; k < 3; k++) al[3 * c + r] += inv[3 * r + k] * (F[3 * c + k] + q[3 * c + k]);
        }
#pragma omp parallel for
    for (long v = 1; v < L->nv; v++)
        for (int i = 0; i < NF; i++) L->u[v * NF + i] += al[i];
    (void)n;
}

int ora_mg_solve(ora_mg *m, double tol, int maxit, double *hist) {
    ora_level *L = &m->lv[0];
    double fn[NCASE], rn[NCASE];
    /* balanced right-hand side (zero net force per case and component), as the
     * CUDA library enforces before every solve */
    {
        double mean[NF] = {0};
        for (long v = 0; v < L->nv; v++)
            for (int i = 0; i < NF; i++) mean[i] += L->f[v * NF + i];
        for (int i = 0; i < NF; i++) mean[i] /= (double)L->nv;
        for (long v = 0; v < L->nv; v++)
            for (int i = 0; i < NF; i++) L->f[v * NF + i] -= mean[i];
    }
    ora_weighted_norm(L->n, L->f, fn);
    int it = 0;
    for (;;) {
        int done = 1;
        if (it > 0) {
            for (int q = 0; q < NCASE; q++) if (rn[q] / (fn[q] + 1e-10) > tol) done = 0;
            if (done) break;
        }
        if (it >= maxit) break;
        ora_mg_vcycle(m, 1.0);
        pin_deflate(m);
        it++;
        /* the level-0 residual left by the down leg */
        ora_weighted_norm(L->n, L->r, rn);
        if (hist)
            for (int q = 0; q < NCASE; q++) hist[(it - 1) * NCASE + q] = rn[q] / (fn[q] + 1e-10);
    }
    return it;
}

/* ------------------------------------------------------------------------- */
/* homogenized tensor and sensitivities (homogenization.cu:208-346, 697-948)  */
/* ------------------------------------------------------------------------- */
static void element_chi(const ora_mg *m, const double *chi, int x, int y, int z, double U[NCASE][24]) {
    const int *n = m->lv[0].n;
    for (int a = 0; a < 8; a++) {
        long v = lexid(wrapi(x + a % 2, n[0]), wrapi(y + a / 2 % 2, n[1]), wrapi(z + a / 4, n[2]), n);
        for (int q = 0; q < NCASE; q++) {
            double u0[3];
            macro_disp(a, q, u0);
            for (int k = 0; k < 3; k++) U[q][3 * a + k] = u0[k] - chi[v * NF + 3 * q + k];
        }
    }
}

static void element_energy(const ora_mg *m, double U[NCASE][24], double E[NCASE][NCASE]) {
    double KU[NCASE][24];
    for (int q = 0; q < NCASE; q++)
        for (int i = 0; i < 24; i++) {
            double s = 0;
            for (int j = 0; j < 24; j++) s += m->ke[i * 24 + j] * U[q][j];
            KU[q][i] = s;
        }
    for (int p = 0; p < NCASE; p++)
        for (int q = 0; q < NCASE; q++) {
            double s = 0;
            for (int i = 0; i < 24; i++) s += U[p][i] * KU[q][i];
            E[p][q] = s;
        }
}

/* C_ij = (1/N^3) sum_e (1e-9 + rho_e) (chi0_i - chi_i)^T Ke (chi0_j - chi_j) */
void ora_mg_elastic_matrix(ora_mg *m, const double *chi, double C[36]) {
    const int *n = m->lv[0].n;
    if (!chi) chi = m->lv[0].u;
    double acc[36] = {0};
#pragma omp parallel
    {
        double loc[36] = {0};
#pragma omp for collapse(2)
        for (int z = 0; z < n[2]; z++)
            for (int y = 0; y < n[1]; y++)
                for (int x = 0; x < n[0]; x++) {
                    double U[NCASE][24], E[NCASE][NCASE];
                    element_chi(m, chi, x, y, z, U);
                    element_energy(m, U, E);
                    double rp = RHO_PENAL_MIN + m->rho[lexid(x, y, z, n)];
                    for (int i = 0; i < 36; i++) loc[i] += rp * E[i / 6][i % 6];
                }
#pragma omp critical
        for (int i = 0; i < 36; i++) acc[i] += loc[i];
    }
    double vol = (double)m->lv[0].nv;
    for (int i = 0; i < 36; i++) C[i] = acc[i] / vol;
}

/* d obj / d rho_phys per element, written at x + (y + z*ny)*pitch (exponent 1) */
void ora_mg_sensitivity(ora_mg *m, const double *chi, const double dC[36], double *sens, int pitch) {
    const int *n = m->lv[0].n;
    if (!chi) chi = m->lv[0].u;
    double vol = (double)m->lv[0].nv;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < n[2]; z++)
        for (int y = 0; y < n[1]; y++)
            for (int x = 0; x < n[0]; x++) {
                double U[NCASE][24], E[NCASE][NCASE];
                element_chi(m, chi, x, y, z, U);
                element_energy(m, U, E);
                double s = 0;
                for (int i = 0; i < NCASE; i++)
                    for (int j = i; j < NCASE; j++) {
                        double dc = dC[i * 6 + j] + (i != j ? dC[j * 6 + i] : 0);
                        s += E[i][j] * dc;
                    }
                sens[x + ((long)y + (long)z * n[1]) * pitch] = s / vol;
            }
}

/* ------------------------------------------------------------------------- */
/* design update (OCOptimizer.cu:12-152, TensorExpression.h:945-1047)          */
/* ------------------------------------------------------------------------- */
/* OC bisection; returns the number of bisection steps taken */
int ora_oc_update(long ne, const double *sens, double *rho, double volratio, double minrho, double step,
                  double damp) {
    double mx = 0;
    for (long i = 0; i < ne; i++) if (fabs(sens[i]) > mx) mx = fabs(sens[i]);
    double lo = 0, hi = mx;
    double *nr = (double *)malloc(sizeof(double) * ne);
    int it;
    for (it = 0; it < 20; it++) {
        double g = (hi + lo) / 2;
        double sum = 0;
#pragma omp parallel for reduction(+ : sum)
        for (long i = 0; i < ne; i++) {
            double r = rho[i];
            double B = -sens[i] / g;
            if (B < 0) B = 0.01;
            double v = pow(B, damp) * r;
            if (v - r < -step) v = r - step;
            if (v - r > step) v = r + step;
            if (v < minrho) v = minrho;
            if (v > 1) v = 1;
            nr[i] = v;
            sum += v;
        }
        double vol = sum / (double)ne;
        if (vol < volratio - 0.0001) hi = g;
        else if (vol > volratio + 0.0001) lo = g;
        else { it++; break; }
    }
    memcpy(rho, nr, sizeof(double) * ne);
    free(nr);
    return it;
}

/* linear cone filter of sensitivities, radius r, window int(r+0.5), optional wrap */
void ora_filter_sens(const int n[3], const double *sens, const double *rho, double *out, double radius, int periodic) {
    int h = (int)(radius + 0.5);
#pragma omp parallel for collapse(2)
    for (int z = 0; z < n[2]; z++)
        for (int y = 0; y < n[1]; y++)
            for (int x = 0; x < n[0]; x++) {
                double s = 0, ws = 0;
                for (int dz = -h; dz <= h; dz++)
                    for (int dy = -h; dy <= h; dy++)
                        for (int dx = -h; dx <= h; dx++) {
                            double d2 = (double)(dx * dx + dy * dy + dz * dz) / (radius * radius);
                            double w = d2 < 1 ? 1 - sqrt(d2) : 0;
                            int p[3] = {x + dx, y + dy, z + dz};
                            if (periodic) for (int a = 0; a < 3; a++) p[a] = wrapi(p[a], n[a]);
                            if (p[0] < 0 || p[0] >= n[0] || p[1] < 0 || p[1] >= n[1] || p[2] < 0 || p[2] >= n[2])
                                continue;
                            long id = lexid(p[0], p[1], p[2], n);
                            s += sens[id] * rho[id] * w;
                            ws += w;
                        }
                long id = lexid(x, y, z, n);
                out[id] = s / (ws * rho[id]);
            }
}

/* symmetrisation, FP32 arithmetic in the reference's summation order
 * (TensorExpression.cuh:72-): type 0 = reflect3, 1 = reflect6, 2 = rotate3 */
static inline long sidx(const int n[3], int a, int b, int c) { return lexid(a, b, c, n); }
void ora_symmetrize_f32(const int n[3], float *v, int type) {
    int h[3] = {n[0] / 2, n[1] / 2, n[2] / 2};
    if (type == 0) {
        for (int z = 0; z < h[2]; z++)
            for (int y = 0; y < h[1]; y++)
                for (int x = 0; x < h[0]; x++) {
                    int rp[3] = {x, y, z}, orb[8][3];
                    for (int i = 0; i < 8; i++)
                        for (int j = 0; j < 3; j++) orb[i][j] = ((i >> j) & 1) ? n[j] - 1 - rp[j] : rp[j];
                    float val = v[sidx(n, orb[0][0], orb[0][1], orb[0][2])];
                    for (int i = 1; i < 8; i++) val += v[sidx(n, orb[i][0], orb[i][1], orb[i][2])];
                    val /= 8;
                    for (int i = 0; i < 8; i++) v[sidx(n, orb[i][0], orb[i][1], orb[i][2])] = val;
                }
    } else if (type == 1) {
        for (int z = 0; z < h[2]; z++)
            for (int y = 0; y <= z; y++)
                for (int x = 0; x <= y; x++) {
                    int rp[3] = {x, y, z};
                    float s = 0;
                    for (int i = 0; i < 8; i++) {
                        int o[3];
                        for (int j = 0; j < 3; j++) o[j] = ((i >> j) & 1) ? n[j] - 1 - rp[j] : rp[j];
                        s += v[sidx(n, o[0], o[1], o[2])];
                        s += v[sidx(n, o[0], o[2], o[1])];
                        s += v[sidx(n, o[2], o[0], o[1])];
                        s += v[sidx(n, o[2], o[1], o[0])];
                        s += v[sidx(n, o[1], o[0], o[2])];
                        s += v[sidx(n, o[1], o[2], o[0])];
                    }
                    s /= 48;
                    for (int i = 0; i < 8; i++) {
                        int o[3];
                        for (int j = 0; j < 3; j++) o[j] = ((i >> j) & 1) ? n[j] - 1 - rp[j] : rp[j];
                        v[sidx(n, o[0], o[1], o[2])] = s;
                        v[sidx(n, o[0], o[2], o[1])] = s;
                        v[sidx(n, o[2], o[0], o[1])] = s;
                        v[sidx(n, o[2], o[1], o[0])] = s;
                        v[sidx(n, o[1], o[0], o[2])] = s;
                        v[sidx(n, o[1], o[2], o[0])] = s;
                    }
                }
    } else if (type == 2) {
        /* rotate3: the 24 proper rotations of the cube about its centre; odd axis
         * permutations take an odd number of mirror flips, even ones an even number */
        static const int perm[6][3] = {{0, 2, 1}, {2, 1, 0}, {1, 0, 2}, {2, 0, 1}, {1, 2, 0}, {0, 1, 2}};
        static const int flips_odd[4][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 1}};
        static const int flips_even[4][3] = {{0, 0, 0}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1}};
        for (int z = 0; z < h[2]; z++)
            for (int y = 0; y <= z; y++)
                for (int x = 0; x <= z; x++) {
                    int rp[3] = {x, y, z};
                    /* representatives with x, y <= z can share an orbit (e.g. (0,1,1) and
                     * (1,0,1)); average each orbit once, at its first representative */
                    long t = (long)z * (z + 1) * (2 * z + 1) / 6 + (long)y * (z + 1) + x, tmin = t;
                    for (int i = 0; i < 6; i++) {
                        int o[3] = {rp[perm[i][0]], rp[perm[i][1]], rp[perm[i][2]]};
                        for (int f = 0; f < 4; f++) {
                            const int *fl = i < 3 ? flips_odd[f] : flips_even[f];
                            int q[3];
                            for (int j = 0; j < 3; j++) q[j] = fl[j] ? -1 - o[j] : o[j];
                            if (q[0] >= 0 && q[1] >= 0 && q[2] >= 0 && q[0] <= q[2] && q[1] <= q[2]) {
                                long tq = (long)q[2] * (q[2] + 1) * (2 * q[2] + 1) / 6 + (long)q[1] * (q[2] + 1) + q[0];
                                if (tq < tmin) tmin = tq;
                            }
                        }
                    }
                    if (tmin < t) continue;
                    float s = 0;
                    for (int i = 0; i < 6; i++) {
                        int o[3] = {rp[perm[i][0]], rp[perm[i][1]], rp[perm[i][2]]};
                        for (int f = 0; f < 4; f++) {
                            const int *fl = i < 3 ? flips_odd[f] : flips_even[f];
                            int p[3];
                            for (int j = 0; j < 3; j++) p[j] = fl[j] ? h[j] - 1 - o[j] : h[j] + o[j];
                            s += v[sidx(n, p[0], p[1], p[2])];
                        }
                    }
                    s /= 24;
                    for (int i = 0; i < 6; i++) {
                        int o[3] = {rp[perm[i][0]], rp[perm[i][1]], rp[perm[i][2]]};
                        for (int f = 0; f < 4; f++) {
                            const int *fl = i < 3 ? flips_odd[f] : flips_even[f];
                            int p[3];
                            for (int j = 0; j < 3; j++) p[j] = fl[j] ? h[j] - 1 - o[j] : h[j] + o[j];
                            v[sidx(n, p[0], p[1], p[2])] = s;
                        }
                    }
                }
    }
}
