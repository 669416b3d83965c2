/* terrain_open_oracle.c - TEST INFRASTRUCTURE ONLY (never linked by the
 * product).  CPU restatement, one binary32 operation at a time in the
 * reference's order, of the terrain + all-open psolver=3 acoustic RK stage:
 *
 *   cpu_psolver3_terrain_open_stage_inplace   src/cm1core/cuda_psolver3_terrain_open.py:774-894
 *     _prepare_coefficients                   :300-390
 *     _terrain_pressure_gradient              :393-479
 *     _transformed_velocity_terms             :482-541
 *     _initial_fpk                            :544-592
 *     _pressure_advection                     :595-675
 *     _implicit_and_pressure_update           :678-745
 *     _average_velocities                     :748-771
 *   cpu_ssopen_terrain_all_inplace            src/cm1core/cuda_terrain_open_boundary.py:720-850
 *   _interp_u_at_w                            :666-684
 *   cpu_bcwsfc_terrain_physical_inplace       :687-708
 *   terrain_coordinate_profiles (uniform)     :486-560
 *   cpu_bcp/bcs/bcu/bcv/bcw_open_inplace      src/cm1core/cuda_sound3_open_boundary.py:249-335
 *   cpu_radiation4_composed_inplace           :424-442
 *   cpu_radiation4_inplace                    src/cm1core/cuda_lateral_closure.py:390-472
 *   fornberg_extrapolation_weights            src/cm1core/cm1_vertical_grid.py:387-454
 *
 * Layout (C order, CM1 index i maps to padded column i+2 on the ng=3 lane):
 *   pressure family (nk+2, nj+2, ni+2); u (nk+2, nj+6, ni+7); v (nk+2, nj+7,
 *   ni+6); w (nk+3, nj+6, ni+6); scalar (nk+2, nj+6, ni+6); radbcw/e
 *   (nk+2, nj+6); radbcs/n (nk+2, ni+6); metrics as terrain_static_shapes.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "real.h"  /* before the header: its array structs take the working precision */
#include "../include/gm1b.h"

int oracle_stage_schedule(float dt, int nsound, int nrk, int *nloop, float *dts);
float oracle_rk_stage_dt(float dt, int nrk);

typedef struct TosArrays {
    float *ppi, *pp3d, *ppx, *ppd, *piadv, *ppterm, *ppten, *thv, *qk, *pk1, *pk2, *mm, *fpk, *divh, *hadvp, *dum3,
        *elim_c, *elim_d, *tri_aa, *tri_bb, *tri_cc, *tri_dd, *tri_pivot, *tri_residual;
    float *ua, *u3d, *uten, *rru, *va, *v3d, *vten, *rrv, *wa, *w3d, *wten, *rrw;
    float *radbcw, *radbce, *radbcs, *radbcn, *uh, *vh, *ruf, *rvf, *scalar;
} TosArrays;

typedef struct TosMetrics {
    const float *rho0_3d, *rr0, *rf0, *rrf0, *c1, *c2, *gz, *rgzu, *rgzv, *dzdx, *dzdy, *gx, *gxu, *gy, *gyv;
} TosMetrics;

enum {
    ABL_OPEN = 1, ABL_PGRAD = 2, ABL_DIV = 4, ABL_PADV = 8, ABL_IMPLICIT = 16, ABL_PFILL = 32, ABL_RADIATION = 64,
    ABL_FILLS = 128
};

typedef struct G {
    int ni, nj, nk;
} G;

static inline size_t P(const G *g, int k, int j, int i) { return ((size_t)k * (g->nj + 2) + j) * (g->ni + 2) + i; }
static inline size_t U(const G *g, int k, int y, int x) { return ((size_t)k * (g->nj + 6) + y) * (g->ni + 7) + x; }
static inline size_t V(const G *g, int k, int y, int x) { return ((size_t)k * (g->nj + 7) + y) * (g->ni + 6) + x; }
static inline size_t W(const G *g, int k, int y, int x) { return ((size_t)k * (g->nj + 6) + y) * (g->ni + 6) + x; }
static inline size_t M(const G *g, int k0, int j0, int i0) { return ((size_t)k0 * g->nj + j0) * g->ni + i0; }
static inline size_t H(const G *g, int j0, int i0) { return (size_t)j0 * g->ni + i0; }
static inline int X(int i) { return i + 2; }
static inline int Y(int j) { return j + 2; }

/* numpy.minimum / numpy.maximum: NaN propagates, ties return the second */
static inline float np_min(float a, float b) { return a != a ? a : (b != b ? b : (a < b ? a : b)); }
static inline float np_max(float a, float b) { return a != a ? a : (b != b ? b : (a > b ? a : b)); }

/* ---------------------------------------------------------------------- */
/* vertical coordinate of the uniform terrain column                      */
/* ---------------------------------------------------------------------- */
typedef struct Prof {
    float *sigma, *sigmaf, *rds, *rdsf;
    float cgs[3], cgt[3];
} Prof;

/* Fornberg (1988) weights of the three-point value stencil at x0 from four
 * nodes, in double precision (delta[n][m+1][nu], m = -1..4). */
static void fornberg3(const double alpha[4], double x0, double out[3]) {
    double delta[4][6][4];
    memset(delta, 0, sizeof delta);
    delta[0][1][0] = 1.0;
    double c1 = 1.0;
    for (int n = 1; n < 4; ++n) {
        double c2 = 1.0;
        for (int nu = 0; nu < n; ++nu) {
            const double c3 = alpha[n] - alpha[nu];
            c2 = c2 * c3;
            delta[n - 1][n + 1][nu] = 0.0;
            const int mmax = n < 4 ? n : 4;
            for (int m = 0; m <= mmax; ++m)
                delta[n][m + 1][nu] = ((alpha[n] - x0) * delta[n - 1][m + 1][nu] - m * delta[n - 1][m][nu]) / c3;
        }
        const int mmax = n < 4 ? n : 4;
        for (int m = 0; m <= mmax; ++m)
            delta[n][m + 1][n] =
                (c1 / c2) * (m * delta[n - 1][m][n - 1] - (alpha[n - 1] - x0) * delta[n - 1][m + 1][n - 1]);
        c1 = c2;
    }
    for (int nu = 0; nu < 3; ++nu) out[nu] = delta[2][1][nu];
}

static void edge_weights(const float *sigma, const float *sigmaf, int nk, int top, float out[3]) {
    float den, num;
    float nodes[4];
    if (top) {
        den = sigmaf[nk + 1] - sigmaf[nk];
        num = sigmaf[nk + 1];
        for (int q = 0; q < 4; ++q) nodes[q] = sigma[nk - q];
    } else {
        den = sigmaf[2] - sigmaf[1];
        num = sigmaf[1];
        for (int q = 0; q < 4; ++q) nodes[q] = sigma[1 + q];
    }
    const double x0 = (double)(num / den);
    double alpha[4], w[3];
    for (int q = 0; q < 4; ++q) alpha[q] = (double)(nodes[q] / den);
    fornberg3(alpha, x0, w);
    for (int q = 0; q < 3; ++q) out[q] = (float)w[q];
}

static void make_profiles(Prof *p, int nk, float dz32) {
    const size_t n = (size_t)nk + 2;
    p->sigma = calloc(n, sizeof(float));
    p->sigmaf = calloc(n, sizeof(float));
    p->rds = calloc(n, sizeof(float));
    p->rdsf = calloc(n, sizeof(float));
    for (int k = 1; k <= nk; ++k) p->sigma[k] = ((float)k - 0.5f) * dz32;
    for (int k = 1; k <= nk + 1; ++k) p->sigmaf[k] = (float)(k - 1) * dz32;
    for (int k = 2; k <= nk; ++k) p->rds[k] = 1.0f / (p->sigma[k] - p->sigma[k - 1]);
    for (int k = 1; k <= nk; ++k) p->rdsf[k] = 1.0f / (p->sigmaf[k + 1] - p->sigmaf[k]);
    edge_weights(p->sigma, p->sigmaf, nk, 0, p->cgs);
    edge_weights(p->sigma, p->sigmaf, nk, 1, p->cgt);
}

static void free_profiles(Prof *p) {
    free(p->sigma);
    free(p->sigmaf);
    free(p->rds);
    free(p->rdsf);
}

/* the six Fornberg words, for the product's host side to compare against */
void oracle_terrain_edge_weights(int nk, float dz, float cgs[3], float cgt[3]) {
    Prof p;
    make_profiles(&p, nk, dz);
    memcpy(cgs, p.cgs, sizeof p.cgs);
    memcpy(cgt, p.cgt, sizeof p.cgt);
    free_profiles(&p);
}

/* ---------------------------------------------------------------------- */
/* lateral boundary operators                                             */
/* ---------------------------------------------------------------------- */
static float interp_at_w(const float *q, size_t (*ix)(const G *, int, int, int), const G *g, const Prof *p, int kf,
                         int y, int x) {
    const int nk = g->nk;
    if (kf == 1) return (p->cgs[0] * q[ix(g, 1, y, x)] + p->cgs[1] * q[ix(g, 2, y, x)]) + p->cgs[2] * q[ix(g, 3, y, x)];
    if (kf == nk + 1)
        return (p->cgt[0] * q[ix(g, nk, y, x)] + p->cgt[1] * q[ix(g, nk - 1, y, x)]) + p->cgt[2] * q[ix(g, nk - 2, y, x)];
    const float r2 = (p->sigmaf[kf] - p->sigma[kf - 1]) * p->rds[kf];
    const float r1 = 1.0f - r2;
    return r1 * q[ix(g, kf - 1, y, x)] + r2 * q[ix(g, kf, y, x)];
}

/* the four terrain ssopenbc operators in source order (west, east, south,
 * north); each side snapshots its two w-level interpolations first */
static void ssopen_terrain(TosArrays *a, const TosMetrics *m, const G *g, const Prof *p, float dts, float rdx,
                           float rdy) {
    const int ni = g->ni, nj = g->nj, nk = g->nk;
    const float half = 0.5f;
    float *snap = malloc(sizeof(float) * (size_t)(nk + 1) * (size_t)(ni > nj ? ni : nj) * 2);
#define SN(kf, l, q) snap[(((size_t)(kf) - 1) * L + (l)) * 2 + (q)]
    size_t L = (size_t)nj;
    for (int side = 0; side < 2; ++side) {  /* west, east */
        const int xa = side == 0 ? X(1) : X(ni), xb = side == 0 ? X(2) : X(ni + 1);
        for (int kf = 1; kf <= nk + 1; ++kf)
            for (int j0 = 0; j0 < nj; ++j0) {
                SN(kf, j0, 0) = interp_at_w(a->u3d, U, g, p, kf, Y(j0 + 1), xa);
                SN(kf, j0, 1) = interp_at_w(a->u3d, U, g, p, kf, Y(j0 + 1), xb);
            }
        for (int k = 1; k <= nk; ++k)
            for (int j0 = 0; j0 < nj; ++j0) {
                const int y = Y(j0 + 1);
                const float lo0 = SN(k, j0, 0), lo1 = SN(k, j0, 1), hi0 = SN(k + 1, j0, 0), hi1 = SN(k + 1, j0, 1);
                if (side == 0) {
                    float hz = m->gz[H(g, j0, 0)] * (a->u3d[U(g, k, y, X(2))] * m->rgzu[(size_t)j0 * (ni + 1) + 1] -
                                                     a->u3d[U(g, k, y, X(1))] * m->rgzu[(size_t)j0 * (ni + 1) + 0]);
                    hz = (hz * rdx) * a->uh[X(1)];
                    float vt = m->gx[M(g, k, j0, 0)] * (hi1 + hi0) - m->gx[M(g, k - 1, j0, 0)] * (lo1 + lo0);
                    vt = (half * vt) * p->rdsf[k];
                    const float rad = (-a->radbcw[(size_t)k * (nj + 6) + y]) * (hz + vt);
                    const float ten = rad + a->uten[U(g, k, y, X(1))];
                    a->u3d[U(g, k, y, X(1))] = a->u3d[U(g, k, y, X(1))] + dts * ten;
                } else {
                    float hz = m->gz[H(g, j0, ni - 1)] *
                               (a->u3d[U(g, k, y, X(ni + 1))] * m->rgzu[(size_t)j0 * (ni + 1) + ni] -
                                a->u3d[U(g, k, y, X(ni))] * m->rgzu[(size_t)j0 * (ni + 1) + ni - 1]);
                    hz = (hz * rdx) * a->uh[X(ni)];
                    float vt = m->gx[M(g, k, j0, ni - 1)] * (hi1 + hi0) - m->gx[M(g, k - 1, j0, ni - 1)] * (lo1 + lo0);
                    vt = (half * vt) * p->rdsf[k];
                    const float rad = (-a->radbce[(size_t)k * (nj + 6) + y]) * (hz + vt);
                    const float ten = rad + a->uten[U(g, k, y, X(ni + 1))];
                    a->u3d[U(g, k, y, X(ni + 1))] = a->u3d[U(g, k, y, X(ni + 1))] + dts * ten;
                }
            }
    }
    L = (size_t)ni;
    for (int side = 0; side < 2; ++side) {  /* south, north */
        const int ya = side == 0 ? Y(1) : Y(nj), yb = side == 0 ? Y(2) : Y(nj + 1);
        for (int kf = 1; kf <= nk + 1; ++kf)
            for (int i0 = 0; i0 < ni; ++i0) {
                SN(kf, i0, 0) = interp_at_w(a->v3d, V, g, p, kf, ya, X(i0 + 1));
                SN(kf, i0, 1) = interp_at_w(a->v3d, V, g, p, kf, yb, X(i0 + 1));
            }
        for (int k = 1; k <= nk; ++k)
            for (int i0 = 0; i0 < ni; ++i0) {
                const int x = X(i0 + 1);
                const float lo0 = SN(k, i0, 0), lo1 = SN(k, i0, 1), hi0 = SN(k + 1, i0, 0), hi1 = SN(k + 1, i0, 1);
                if (side == 0) {
                    float hz = m->gz[H(g, 0, i0)] * (a->v3d[V(g, k, Y(2), x)] * m->rgzv[(size_t)1 * ni + i0] -
                                                     a->v3d[V(g, k, Y(1), x)] * m->rgzv[i0]);
                    hz = (hz * rdy) * a->vh[Y(1)];
                    float vt = m->gy[M(g, k, 0, i0)] * (hi1 + hi0) - m->gy[M(g, k - 1, 0, i0)] * (lo1 + lo0);
                    vt = (half * vt) * p->rdsf[k];
                    const float rad = (-a->radbcs[(size_t)k * (ni + 6) + x]) * (hz + vt);
                    const float ten = rad + a->vten[V(g, k, Y(1), x)];
                    a->v3d[V(g, k, Y(1), x)] = a->v3d[V(g, k, Y(1), x)] + dts * ten;
                } else {
                    float hz = m->gz[H(g, nj - 1, i0)] *
                               (a->v3d[V(g, k, Y(nj + 1), x)] * m->rgzv[(size_t)nj * ni + i0] -
                                a->v3d[V(g, k, Y(nj), x)] * m->rgzv[(size_t)(nj - 1) * ni + i0]);
                    hz = (hz * rdy) * a->vh[Y(nj)];
                    float vt = m->gy[M(g, k, nj - 1, i0)] * (hi1 + hi0) - m->gy[M(g, k - 1, nj - 1, i0)] * (lo1 + lo0);
                    vt = (half * vt) * p->rdsf[k];
                    const float rad = (-a->radbcn[(size_t)k * (ni + 6) + x]) * (hz + vt);
                    const float ten = rad + a->vten[V(g, k, Y(nj + 1), x)];
                    a->v3d[V(g, k, Y(nj + 1), x)] = a->v3d[V(g, k, Y(nj + 1), x)] + dts * ten;
                }
            }
    }
#undef SN
    free(snap);
}

/* bc.F:1151-1178 on the physical bottom faces */
static void bcwsfc(TosArrays *a, const TosMetrics *m, const G *g) {
    for (int j0 = 0; j0 < g->nj; ++j0)
        for (int i0 = 0; i0 < g->ni; ++i0) {
            const int y = Y(j0 + 1), x = X(i0 + 1);
            const float ut = (a->u3d[U(g, 1, y, x)] + a->u3d[U(g, 1, y, x + 1)]) * m->dzdx[H(g, j0, i0)];
            const float vt = (a->v3d[V(g, 1, y, x)] + a->v3d[V(g, 1, y + 1, x)]) * m->dzdy[H(g, j0, i0)];
            a->w3d[W(g, 1, y, x)] = (0.5f * (ut + vt)) * m->gz[H(g, j0, i0)];
        }
}

static void bcp_open(float *q, const G *g) {
    const int ni = g->ni, nj = g->nj;
    for (int k = 1; k <= g->nk; ++k) {
        for (int j = 0; j <= nj + 1; ++j) q[P(g, k, j, 0)] = q[P(g, k, j, 1)];
        for (int j = 0; j <= nj + 1; ++j) q[P(g, k, j, ni + 1)] = q[P(g, k, j, ni)];
        for (int i = 0; i <= ni + 1; ++i) q[P(g, k, 0, i)] = q[P(g, k, 1, i)];
        for (int i = 0; i <= ni + 1; ++i) q[P(g, k, nj + 1, i)] = q[P(g, k, nj, i)];
    }
}

/* scalar (S) and w (W) share a layout */
static void bcs_open(float *q, const G *g, int k0, int k1) {
    const int ni = g->ni, nj = g->nj;
    for (int k = k0; k <= k1; ++k) {
        for (int j = 0; j <= nj + 1; ++j)
            for (int i = -2; i <= 0; ++i) q[W(g, k, Y(j), X(i))] = q[W(g, k, Y(j), X(1))];
        for (int j = 0; j <= nj + 1; ++j)
            for (int i = ni + 1; i <= ni + 3; ++i) q[W(g, k, Y(j), X(i))] = q[W(g, k, Y(j), X(ni))];
        for (int j = -2; j <= 0; ++j)
            for (int i = 0; i <= ni + 1; ++i) q[W(g, k, Y(j), X(i))] = q[W(g, k, Y(1), X(i))];
        for (int j = nj + 1; j <= nj + 3; ++j)
            for (int i = 0; i <= ni + 1; ++i) q[W(g, k, Y(j), X(i))] = q[W(g, k, Y(nj), X(i))];
    }
}

static void bcu_open(float *q, const G *g) {
    const int ni = g->ni, nj = g->nj;
    for (int k = 1; k <= g->nk; ++k) {
        for (int j = 0; j <= nj + 1; ++j)
            for (int i = -2; i <= 0; ++i) q[U(g, k, Y(j), X(i))] = q[U(g, k, Y(j), X(1))];
        for (int j = 0; j <= nj + 1; ++j)
            for (int i = ni + 2; i <= ni + 4; ++i) q[U(g, k, Y(j), X(i))] = q[U(g, k, Y(j), X(ni + 1))];
        for (int j = -2; j <= 0; ++j)
            for (int i = 0; i <= ni + 2; ++i) q[U(g, k, Y(j), X(i))] = q[U(g, k, Y(1), X(i))];
        for (int j = nj + 1; j <= nj + 3; ++j)
            for (int i = 0; i <= ni + 2; ++i) q[U(g, k, Y(j), X(i))] = q[U(g, k, Y(nj), X(i))];
    }
}

static void bcv_open(float *q, const G *g) {
    const int ni = g->ni, nj = g->nj;
    for (int k = 1; k <= g->nk; ++k) {
        for (int j = -2; j <= 0; ++j)
            for (int i = 0; i <= ni + 1; ++i) q[V(g, k, Y(j), X(i))] = q[V(g, k, Y(1), X(i))];
        for (int j = nj + 2; j <= nj + 4; ++j)
            for (int i = 0; i <= ni + 1; ++i) q[V(g, k, Y(j), X(i))] = q[V(g, k, Y(nj + 1), X(i))];
        for (int j = 0; j <= nj + 2; ++j)
            for (int i = -2; i <= 0; ++i) q[V(g, k, Y(j), X(i))] = q[V(g, k, Y(j), X(1))];
        for (int j = 0; j <= nj + 2; ++j)
            for (int i = ni + 1; i <= ni + 3; ++i) q[V(g, k, Y(j), X(i))] = q[V(g, k, Y(j), X(ni))];
    }
}

static void bcw_open_flag1(float *q, const G *g) {
    bcs_open(q, g, 2, g->nk);
    for (int j = 0; j <= g->nj + 1; ++j)
        for (int i = 0; i <= g->ni + 1; ++i) {
            q[W(g, 1, Y(j), X(i))] = 0.0f;
            q[W(g, g->nk + 1, Y(j), X(i))] = 0.0f;
        }
}

/* radbcew4 / radbcns4 (Durran-Klemp phase speeds averaged over the column) */
static void radiation4(TosArrays *a, const G *g, float dx, float dy, float dttmp) {
    const int ni = g->ni, nj = g->nj, nk = g->nk;
    const float eps = 1.0e-10f, zero = 0.0f, limit = 350.0f;
    for (int j0 = 0; j0 < nj; ++j0) {
        const int y = Y(j0 + 1);
        float avgw = 0.0f, avge = 0.0f;
        for (int k = 1; k <= nk; ++k) {
            float foo = a->ua[U(g, k, y, X(3))] - a->ua[U(g, k, y, X(2))];
            float num = dx * a->ruf[X(2)];
            num = num * (a->ua[U(g, k, y, X(2))] - a->u3d[U(g, k, y, X(2))]);
            float den = dttmp * (copysignf(eps, foo) + foo);
            float c = num / den;
            avgw = avgw + np_max(np_min(c, zero), -limit);
            foo = a->ua[U(g, k, y, X(ni))] - a->ua[U(g, k, y, X(ni - 1))];
            num = dx * a->ruf[X(ni)];
            num = num * (a->ua[U(g, k, y, X(ni))] - a->u3d[U(g, k, y, X(ni))]);
            den = dttmp * (copysignf(eps, foo) + foo);
            c = num / den;
            avge = avge + np_min(np_max(c, zero), limit);
        }
        avgw = avgw / (float)nk;
        avge = avge / (float)nk;
        for (int k = 1; k <= nk; ++k) {
            a->radbcw[(size_t)k * (nj + 6) + y] = avgw;
            a->radbce[(size_t)k * (nj + 6) + y] = avge;
        }
    }
    for (int i0 = 0; i0 < ni; ++i0) {
        const int x = X(i0 + 1);
        float avgs = 0.0f, avgn = 0.0f;
        for (int k = 1; k <= nk; ++k) {
            float foo = a->va[V(g, k, Y(3), x)] - a->va[V(g, k, Y(2), x)];
            float num = dy * a->rvf[Y(2)];
            num = num * (a->va[V(g, k, Y(2), x)] - a->v3d[V(g, k, Y(2), x)]);
            float den = dttmp * (copysignf(eps, foo) + foo);
            float c = num / den;
            avgs = avgs + np_max(np_min(c, zero), -limit);
            foo = a->va[V(g, k, Y(nj), x)] - a->va[V(g, k, Y(nj - 1), x)];
            num = dy * a->rvf[Y(nj)];
            num = num * (a->va[V(g, k, Y(nj), x)] - a->v3d[V(g, k, Y(nj), x)]);
            den = dttmp * (copysignf(eps, foo) + foo);
            c = num / den;
            avgn = avgn + np_min(np_max(c, zero), limit);
        }
        avgs = avgs / (float)nk;
        avgn = avgn / (float)nk;
        for (int k = 1; k <= nk; ++k) {
            a->radbcs[(size_t)k * (ni + 6) + x] = avgs;
            a->radbcn[(size_t)k * (ni + 6) + x] = avgn;
        }
    }
}

/* ---------------------------------------------------------------------- */
/* the acoustic stage                                                     */
/* ---------------------------------------------------------------------- */
#define NSCRATCH 16

static void prepare(TosArrays *a, const TosMetrics *m, const G *g, const Prof *p, float dts) {
    const int ni = g->ni, nj = g->nj, nk = g->nk;
    const size_t np = (size_t)(nk + 2) * (nj + 2) * (ni + 2);
    float *scratch[NSCRATCH] = {a->qk, a->pk1, a->pk2, a->mm, a->fpk, a->divh, a->hadvp, a->dum3,
                                a->elim_c, a->elim_d, a->tri_aa, a->tri_bb, a->tri_cc, a->tri_dd, a->tri_pivot,
                                a->tri_residual};
    for (int s = 0; s < NSCRATCH; ++s) memset(scratch[s], 0, np * sizeof(float));
    const float cp = 1005.7f;
    for (int k = 1; k <= nk; ++k)
        for (int j0 = 0; j0 < nj; ++j0)
            for (int i0 = 0; i0 < ni; ++i0) {
                const int j = j0 + 1, i = i0 + 1;
                const size_t c = P(g, k, j, i);
                const float gz = m->gz[H(g, j0, i0)];
                const float tem = dts * p->rdsf[k];
                a->qk[c] = (tem * a->ppterm[c]) * gz;
                const float tem2 = ((dts * gz) * p->rdsf[k]) * m->rr0[M(g, k - 1, j0, i0)];
                const float b2 = (-m->c2[M(g, k, j0, i0)]) * a->piadv[P(g, k + 1, j, i)] +
                                 (1.0f - m->c1[M(g, k, j0, i0)]) * a->piadv[c];
                a->pk2[c] = (tem2 * m->rf0[M(g, k, j0, i0)]) * b2;
                const float b1 = m->c1[M(g, k - 1, j0, i0)] * a->piadv[P(g, k - 1, j, i)] +
                                 (m->c2[M(g, k - 1, j0, i0)] - 1.0f) * a->piadv[c];
                a->pk1[c] = (tem2 * m->rf0[M(g, k - 1, j0, i0)]) * b1;
                if (k >= 2) {
                    const float tem1 = (dts * p->rds[k]) * cp;
                    const float th = m->c2[M(g, k - 1, j0, i0)] * a->thv[c] + m->c1[M(g, k - 1, j0, i0)] * a->thv[P(g, k - 1, j, i)];
                    a->mm[c] = (tem1 * th) * gz;
                } else {
                    a->dum3[P(g, 1, j, i)] = 0.0f;
                    a->dum3[P(g, nk + 1, j, i)] = 0.0f;
                }
                if (k == 1) a->pk1[c] = 0.0f;
                if (k == nk) a->pk2[c] = 0.0f;
            }
}

static void pressure_gradient(TosArrays *a, const TosMetrics *m, const G *g, const Prof *p, float dts, float rdx,
                              float rdy) {
    const int ni = g->ni, nj = g->nj, nk = g->nk;
    float *vert = a->hadvp;
    memset(vert, 0, sizeof(float) * (size_t)(nk + 2) * (nj + 2) * (ni + 2));
    for (int k = 2; k <= nk; ++k)
        for (int j = 0; j <= nj + 1; ++j)
            for (int i = 0; i <= ni + 1; ++i)
                vert[P(g, k, j, i)] = (a->ppd[P(g, k, j, i)] - a->ppd[P(g, k - 1, j, i)]) * p->rds[k];
    const float halfcp = 1005.7f * 0.5f, eighth = 0.125f;
    for (int k = 1; k <= nk; ++k) {
        for (int j0 = 0; j0 < nj; ++j0) {
            const int j = j0 + 1, y = Y(j);
            for (int f = 2; f <= ni; ++f) {
                const int i0 = f - 1;
                const float th = a->thv[P(g, k, j, f)] + a->thv[P(g, k, j, f - 1)];
                const float hz = (a->ppd[P(g, k, j, f)] - a->ppd[P(g, k, j, f - 1)]) * rdx;
                const float vs = (vert[P(g, k + 1, j, f)] + vert[P(g, k + 1, j, f - 1)]) +
                                 (vert[P(g, k, j, f)] + vert[P(g, k, j, f - 1)]);
                const float tr = (eighth * vs) * (m->gxu[((size_t)(k - 1) * nj + j0) * (ni + 1) + i0] +
                                                  m->gxu[((size_t)k * nj + j0) * (ni + 1) + i0]);
                const float pg = (halfcp * th) * (hz + tr);
                const size_t q = U(g, k, y, X(f));
                a->u3d[q] = a->u3d[q] + dts * (a->uten[q] - pg);
            }
        }
        for (int f = 2; f <= nj; ++f) {
            const int j0 = f - 1, y = Y(f);
            for (int i0 = 0; i0 < ni; ++i0) {
                const int i = i0 + 1;
                const float th = a->thv[P(g, k, f, i)] + a->thv[P(g, k, f - 1, i)];
                const float hz = (a->ppd[P(g, k, f, i)] - a->ppd[P(g, k, f - 1, i)]) * rdy;
                const float vs = (vert[P(g, k + 1, f, i)] + vert[P(g, k + 1, f - 1, i)]) +
                                 (vert[P(g, k, f, i)] + vert[P(g, k, f - 1, i)]);
                const float tr = (eighth * vs) * (m->gyv[((size_t)(k - 1) * (nj + 1) + j0) * ni + i0] +
                                                  m->gyv[((size_t)k * (nj + 1) + j0) * ni + i0]);
                const float pg = (halfcp * th) * (hz + tr);
                const size_t q = V(g, k, y, X(i));
                a->v3d[q] = a->v3d[q] + dts * (a->vten[q] - pg);
            }
        }
    }
}

/* xu (nk+2, nj, ni+1) and yv (nk+2, nj+1, ni) = u*rgzu, v*rgzv; dum3 */
static void transformed_terms(TosArrays *a, const TosMetrics *m, const G *g, const Prof *p, float zt, float rzt,
                              float *xu, float *yv) {
    const int ni = g->ni, nj = g->nj, nk = g->nk;
#define XU(k, j0, f) xu[((size_t)(k) * nj + (j0)) * (ni + 1) + (f)]
#define YV(k, f, i0) yv[((size_t)(k) * (nj + 1) + (f)) * ni + (i0)]
    memset(xu, 0, sizeof(float) * (size_t)(nk + 2) * nj * (ni + 1));
    memset(yv, 0, sizeof(float) * (size_t)(nk + 2) * (nj + 1) * ni);
    for (int k = 1; k <= nk; ++k) {
        for (int j0 = 0; j0 < nj; ++j0)
            for (int f = 0; f <= ni; ++f)
                XU(k, j0, f) = a->u3d[U(g, k, Y(j0 + 1), X(f + 1))] * m->rgzu[(size_t)j0 * (ni + 1) + f];
        for (int f = 0; f <= nj; ++f)
            for (int i0 = 0; i0 < ni; ++i0) YV(k, f, i0) = a->v3d[V(g, k, Y(f + 1), X(i0 + 1))] * m->rgzv[(size_t)f * ni + i0];
    }
    memset(a->dum3, 0, sizeof(float) * (size_t)(nk + 2) * (nj + 2) * (ni + 2));
    for (int kf = 2; kf <= nk; ++kf) {
        const float r2 = (p->sigmaf[kf] - p->sigma[kf - 1]) * p->rds[kf];
        const float r1 = 1.0f - r2;
        const float height = (p->sigmaf[kf] - zt) * rzt;
        for (int j0 = 0; j0 < nj; ++j0)
            for (int i0 = 0; i0 < ni; ++i0) {
                const float uh = XU(kf, j0, i0) + XU(kf, j0, i0 + 1), ul = XU(kf - 1, j0, i0) + XU(kf - 1, j0, i0 + 1);
                const float vh = YV(kf, j0, i0) + YV(kf, j0 + 1, i0), vl = YV(kf - 1, j0, i0) + YV(kf - 1, j0 + 1, i0);
                const float xt = (r2 * uh + r1 * ul) * m->dzdx[H(g, j0, i0)];
                const float yt = (r2 * vh + r1 * vl) * m->dzdy[H(g, j0, i0)];
                float v = 0.5f * (xt + yt);
                v = (v * height) * m->gz[H(g, j0, i0)];
                a->dum3[P(g, kf, j0 + 1, i0 + 1)] = v;
            }
    }
}

static void initial_fpk(TosArrays *a, const TosMetrics *m, const G *g, const Prof *p, const float *xu,
                        const float *yv, float dts, float rdx, float rdy, float beta, int do_div) {
    const int ni = g->ni, nj = g->nj, nk = g->nk;
    const float smeps = 1.0e-20f;
    for (int k = 1; k <= nk; ++k)
        for (int j0 = 0; j0 < nj; ++j0)
            for (int i0 = 0; i0 < ni; ++i0) {
                const int j = j0 + 1, i = i0 + 1;
                const size_t c = P(g, k, j, i);
                float div = 0.0f;
                if (do_div) {
                    const float hz = (XU(k, j0, i0 + 1) - XU(k, j0, i0)) * rdx + (YV(k, j0 + 1, i0) - YV(k, j0, i0)) * rdy;
                    const float vt = (a->dum3[P(g, k + 1, j, i)] - a->dum3[c]) * p->rdsf[k];
                    div = m->gz[H(g, j0, i0)] * (hz + vt);
                    if (fabsf(div) < smeps) div = 0.0f;
                }
                a->divh[c] = div;
                const float w1 = k == 1 ? 0.0f : a->w3d[W(g, k, Y(j), X(i))];
                const float w2 = k == nk ? 0.0f : a->w3d[W(g, k + 1, Y(j), X(i))];
                const float src = dts * (a->ppten[c] - a->ppterm[c] * div);
                const float qp = (-a->qk[c]) * (w2 - w1);
                a->fpk[c] = src + beta * qp;
            }
}

/* rho0p == NULL: the uniform operator's base density rho0_3d(k, 1, 1) on
 * every face.  Otherwise each face's own average of the padded base density
 * (nk+2, nj+6, ni+6), the stretched terrain column's xurho / yvrho
 * (cuda_gm1_child_psolver3_open.py:199-205, sound.F:604-613). */
static void pressure_advection(TosArrays *a, const TosMetrics *m, const G *g, const Prof *p, float *xu, float *yv,
                               float dts, float rdx, float rdy, float beta, float zt, float rzt, const float *rho0p) {
    const int ni = g->ni, nj = g->nj, nk = g->nk;
    const size_t pw = (size_t)ni + 6, pp = (size_t)(nj + 6) * pw;
    for (int k = 1; k <= nk; ++k) {
        const float rho = m->rho0_3d[M(g, k - 1, 0, 0)];
        const float *r = rho0p ? rho0p + (size_t)k * pp : NULL;
        for (int j0 = 0; j0 < nj; ++j0)
            for (int f = 0; f <= ni; ++f) {
                const size_t o = (size_t)(j0 + 3) * pw + (size_t)(f + 2);
                const float dens = r ? 0.5f * (r[o] + r[o + 1]) : rho;
                XU(k, j0, f) = dens * XU(k, j0, f);
            }
        for (int f = 0; f <= nj; ++f)
            for (int i0 = 0; i0 < ni; ++i0) {
                const size_t o = (size_t)(f + 2) * pw + (size_t)(i0 + 3);
                const float dens = r ? 0.5f * (r[o] + r[o + pw]) : rho;
                YV(k, f, i0) = dens * YV(k, f, i0);
            }
    }
    memset(a->hadvp, 0, sizeof(float) * (size_t)(nk + 2) * (nj + 2) * (ni + 2));
    for (int kf = 2; kf <= nk; ++kf) {
        const float r2 = (p->sigmaf[kf] - p->sigma[kf - 1]) * p->rds[kf];
        const float r1 = 1.0f - r2;
        const float height = (p->sigmaf[kf] - zt) * rzt;
        for (int j0 = 0; j0 < nj; ++j0)
            for (int i0 = 0; i0 < ni; ++i0) {
                const float uh = XU(kf, j0, i0) + XU(kf, j0, i0 + 1), ul = XU(kf - 1, j0, i0) + XU(kf - 1, j0, i0 + 1);
                const float vh = YV(kf, j0, i0) + YV(kf, j0 + 1, i0), vl = YV(kf - 1, j0, i0) + YV(kf - 1, j0 + 1, i0);
                const float xt = (r2 * uh + r1 * ul) * m->dzdx[H(g, j0, i0)];
                const float yt = (r2 * vh + r1 * vl) * m->dzdy[H(g, j0, i0)];
                float v = 0.5f * (xt + yt);
                v = ((v * height) * m->gz[H(g, j0, i0)]) * m->rrf0[M(g, kf - 1, j0, i0)];
                a->hadvp[P(g, kf, j0 + 1, i0 + 1)] = v;
            }
    }
    const float temx = (dts * 0.5f) * rdx, temy = (dts * 0.5f) * rdy;
    for (int k = 1; k <= nk; ++k)
        for (int j0 = 0; j0 < nj; ++j0)
            for (int i0 = 0; i0 < ni; ++i0) {
                const int j = j0 + 1, i = i0 + 1;
                const size_t c = P(g, k, j, i);
                const float u2 = temx * XU(k, j0, i0 + 1), u1 = temx * XU(k, j0, i0);
                const float v2 = temy * YV(k, j0 + 1, i0), v1 = temy * YV(k, j0, i0);
                const float w2 = a->hadvp[P(g, k + 1, j, i)] + beta * a->w3d[W(g, k + 1, Y(j), X(i))];
                const float w1 = a->hadvp[c] + beta * a->w3d[W(g, k, Y(j), X(i))];
                const float pc = a->piadv[c];
                const float xa = u2 * (a->piadv[P(g, k, j, i + 1)] - pc) + u1 * (pc - a->piadv[P(g, k, j, i - 1)]);
                const float ya = v2 * (a->piadv[P(g, k, j + 1, i)] - pc) + v1 * (pc - a->piadv[P(g, k, j - 1, i)]);
                float hz = (-(xa + ya)) * m->rr0[M(g, k - 1, j0, i0)];
                hz = hz * m->gz[H(g, j0, i0)];
                const float vt = w1 * a->pk1[c] + w2 * a->pk2[c];
                a->fpk[c] = a->fpk[c] + (hz + vt);
            }
}
#undef XU
#undef YV

/* flat != 0: the flat column's update (sound.F:742-765) keeps w(1) and
 * w(nk+1) as they are and filters with cm1.F:311's smeps 1.0e-30 */
static void implicit_and_update(TosArrays *a, const G *g, float dts, int nrk, int n, int nloop, float alph, float beta,
                                float kdiv, int implicit, int flat) {
    const int ni = g->ni, nj = g->nj, nk = g->nk;
    const float asq = alph * alph, smeps = flat ? 1.0e-30f : 1.0e-20f;
    for (int j0 = 0; j0 < nj; ++j0)
        for (int i0 = 0; i0 < ni; ++i0) {
            const int j = j0 + 1, i = i0 + 1, y = Y(j), x = X(i);
#define C(k) P(g, (k), j, i)
#define WW(k) a->w3d[W(g, (k), y, x)]
            if (implicit) {
                for (int k = 2; k <= nk; ++k) {
                    float aa = 0.0f, cc = 0.0f;
                    if (k >= 3) aa = (-asq) * (a->mm[C(k)] * (a->pk1[C(k - 1)] + a->qk[C(k - 1)]));
                    if (k < nk) cc = (-asq) * ((-a->mm[C(k)]) * (a->pk2[C(k)] - a->qk[C(k)]));
                    const float diag = (-(a->pk1[C(k)] + a->qk[C(k)])) + (a->pk2[C(k - 1)] - a->qk[C(k - 1)]);
                    const float bb = 1.0f - asq * (a->mm[C(k)] * diag);
                    const float pdl = a->pp3d[C(k)] - a->pp3d[C(k - 1)];
                    const float fwk = dts * a->wten[W(g, k, y, x)] + beta * ((-a->mm[C(k)]) * pdl);
                    const float upd = (a->pp3d[C(k)] + a->fpk[C(k)]) - (a->pp3d[C(k - 1)] + a->fpk[C(k - 1)]);
                    const float dd = (WW(k) + fwk) + alph * ((-a->mm[C(k)]) * upd);
                    const float piv = k == 2 ? bb : aa * a->elim_c[C(k - 1)] + bb;
                    const float inv = 1.0f / piv;
                    a->tri_aa[C(k)] = aa;
                    a->tri_bb[C(k)] = bb;
                    a->tri_cc[C(k)] = cc;
                    a->tri_dd[C(k)] = dd;
                    a->tri_pivot[C(k)] = piv;
                    if (k < nk) {
                        a->elim_c[C(k)] = (-cc) * inv;
                        const float num = k == 2 ? dd : dd - aa * a->elim_d[C(k - 1)];
                        a->elim_d[C(k)] = num * inv;
                    } else {
                        WW(k) = (dd - aa * a->elim_d[C(k - 1)]) * inv;
                    }
                }
                for (int k = nk - 1; k >= 2; --k) WW(k) = a->elim_c[C(k)] * WW(k + 1) + a->elim_d[C(k)];
                for (int k = 2; k <= nk; ++k) {
                    float lhs = a->tri_aa[C(k)] * WW(k - 1) + a->tri_bb[C(k)] * WW(k);
                    lhs = lhs + a->tri_cc[C(k)] * WW(k + 1);
                    a->tri_residual[C(k)] = lhs - a->tri_dd[C(k)];
                }
            }
            for (int k = 1; k <= nk; ++k) {
                const float w1 = (k == 1 && !flat) ? 0.0f : WW(k), w2 = (k == nk && !flat) ? 0.0f : WW(k + 1);
                const float old = a->pp3d[C(k)];
                const float vt = w1 * (a->pk1[C(k)] + a->qk[C(k)]) + w2 * (a->pk2[C(k)] - a->qk[C(k)]);
                float up = (old + a->fpk[C(k)]) + alph * vt;
                if (fabsf(up) < smeps) up = 0.0f;
                a->pp3d[C(k)] = up;
                const float tend = kdiv * (up - old);
                a->elim_c[C(k)] = tend;
                a->ppd[C(k)] = up + tend;
                if (nrk == 3 && n == nloop) a->ppx[C(k)] = tend;
            }
#undef C
#undef WW
        }
}

static void average_velocities(TosArrays *a, const G *g, int n, int nloop, float alph) {
    const float tavg = 1.0f / (float)nloop;
    for (int k = 1; k <= g->nk; ++k)
        for (int j = 1; j <= g->nj + 1; ++j)
            for (int i = 1; i <= g->ni + 1; ++i) {
                const int y = Y(j), x = X(i);
                const size_t qu = U(g, k, y, x), qv = V(g, k, y, x), qw = W(g, k, y, x);
                float v = a->rru[qu] + a->u3d[qu];
                a->rru[qu] = n < nloop ? v : v * tavg;
                v = a->rrv[qv] + a->v3d[qv];
                a->rrv[qv] = n < nloop ? v : v * tavg;
                const float add = n < nloop ? a->w3d[qw] : a->w3d[qw] * alph;
                v = a->rrw[qw] + add;
                a->rrw[qw] = n < nloop ? v : v * tavg;
            }
}

/* One terrain/open acoustic RK stage.  dz and the lid height zt = nk*dz are
 * taken in double (the reference forms zt as float32(nk * dz) with a Python
 * float dz); everything else is binary32.  diag[0] = nloop, diag[1] = dts,
 * diag[2] = max |tri_residual| over the physical levels 2..nk. */
static int stage_impl(TosArrays *a, const TosMetrics *m, int ni, int nj, int nk, int nrk, float dt, int nsound,
                      float dx, float dy, const Prof *pp, float zt, const float *rho0p, float alph, float kdiv,
                      unsigned ablations, float *diag);

int oracle_terrain_open_stage(TosArrays *a, const TosMetrics *m, int ni, int nj, int nk, int nrk, float dt,
                              int nsound, float dx, float dy, double dz, float alph, float kdiv, unsigned ablations,
                              float *diag) {
    if (ni < 3 || nj < 3 || nk < 4 || nrk < 1 || nrk > 3) return -1;
    Prof p;
    make_profiles(&p, nk, (float)dz);
    const int rc = stage_impl(a, m, ni, nj, nk, nrk, dt, nsound, dx, dy, &p, (float)((double)nk * dz), NULL, alph,
                              kdiv, ablations, diag);
    free_profiles(&p);
    return rc;
}

/* The stage on a stretched terrain column (cuda_gm1_child_psolver3_open.py:
 * 152-330 patching the uniform texts): the caller's CM1-indexed sigma (nk+2),
 * sigmaf (nk+3), rds (nk+2), rdsf (nk+3) in place of the in-kernel uniform
 * coordinate, the lid ztop in place of nk*dz, face-averaged padded base
 * density in the pressure advection, and the open-boundary text's literal
 * 1.875 / -1.25 / 0.375 edge-face weights (cuda_terrain_open_boundary.py:
 * 845-850, untouched by the patch) in place of the column's own. */
int oracle_terrain_open_stage_column(TosArrays *a, const TosMetrics *m, int ni, int nj, int nk, int nrk, float dt,
                                     int nsound, float dx, float dy, const float *sigma, const float *sigmaf,
                                     const float *rds, const float *rdsf, float ztop, const float *rho0p, float alph,
                                     float kdiv, unsigned ablations, float *diag) {
    if (ni < 3 || nj < 3 || nk < 4 || nrk < 1 || nrk > 3 || !rho0p) return -1;
    Prof p;
    p.sigma = (float *)sigma, p.sigmaf = (float *)sigmaf, p.rds = (float *)rds, p.rdsf = (float *)rdsf;
    const float w[3] = {1.875f, -1.25f, 0.375f};
    for (int q = 0; q < 3; ++q) p.cgs[q] = p.cgt[q] = w[q];
    return stage_impl(a, m, ni, nj, nk, nrk, dt, nsound, dx, dy, &p, ztop, rho0p, alph, kdiv, ablations, diag);
}

static int stage_impl(TosArrays *a, const TosMetrics *m, int ni, int nj, int nk, int nrk, float dt, int nsound,
                      float dx, float dy, const Prof *pp, float zt, const float *rho0p, float alph, float kdiv,
                      unsigned ablations, float *diag) {
    const G g = {ni, nj, nk};
    int nloop;
    float dts;
    if (oracle_stage_schedule(dt, nsound, nrk, &nloop, &dts) != 0) return -1;
    const Prof p = *pp;
    const float rzt = 1.0f / zt;
    const float beta = 1.0f - alph;
    const float rdx = 1.0f / dx, rdy = 1.0f / dy;
    float *xu = malloc(sizeof(float) * (size_t)(nk + 2) * nj * (ni + 1));
    float *yv = malloc(sizeof(float) * (size_t)(nk + 2) * (nj + 1) * ni);

    prepare(a, m, &g, &p, dts);
    for (int k = 1; k <= nk; ++k)
        for (int j = 0; j <= nj + 1; ++j)
            for (int i = 0; i <= ni + 1; ++i) {
                a->ppd[P(&g, k, j, i)] = a->ppx[P(&g, k, j, i)];
                if (nrk != 1) a->pp3d[P(&g, k, j, i)] = a->ppi[P(&g, k, j, i)];
            }
    for (int k = 1; k <= nk; ++k)
        for (int j = 0; j <= nj + 1; ++j)
            for (int i = 0; i <= ni + 1; ++i) {
                const int y = Y(j), x = X(i);
                a->rru[U(&g, k, y, x)] = 0.0f;
                a->rrv[V(&g, k, y, x)] = 0.0f;
                a->rrw[W(&g, k, y, x)] = a->wa[W(&g, k, y, x)] * beta;
                if (nrk != 1) {
                    a->u3d[U(&g, k, y, x)] = a->ua[U(&g, k, y, x)];
                    a->v3d[V(&g, k, y, x)] = a->va[V(&g, k, y, x)];
                    a->w3d[W(&g, k, y, x)] = a->wa[W(&g, k, y, x)];
                }
            }
    for (int n = 1; n <= nloop; ++n) {
        if (ablations & ABL_OPEN) ssopen_terrain(a, m, &g, &p, dts, rdx, rdy);
        if (ablations & ABL_PGRAD) pressure_gradient(a, m, &g, &p, dts, rdx, rdy);
        transformed_terms(a, m, &g, &p, zt, rzt, xu, yv);
        initial_fpk(a, m, &g, &p, xu, yv, dts, rdx, rdy, beta, (ablations & ABL_DIV) != 0);
        bcwsfc(a, m, &g);
        if (ablations & ABL_PADV) pressure_advection(a, m, &g, &p, xu, yv, dts, rdx, rdy, beta, zt, rzt, rho0p);
        implicit_and_update(a, &g, dts, nrk, n, nloop, alph, beta, kdiv, (ablations & ABL_IMPLICIT) != 0, 0);
        if (n < nloop && (ablations & ABL_PFILL)) bcp_open(a->ppd, &g);
        average_velocities(a, &g, n, nloop, alph);
    }
    if (ablations & ABL_RADIATION) radiation4(a, &g, dx, dy, oracle_rk_stage_dt(dt, nrk));
    if (ablations & ABL_FILLS) {
        bcu_open(a->u3d, &g);
        bcv_open(a->v3d, &g);
        bcw_open_flag1(a->w3d, &g);
        bcwsfc(a, m, &g);
        if (nrk < 3) {
            bcp_open(a->pp3d, &g);
            bcs_open(a->scalar, &g, 1, nk);
        }
    }
    float rmax = 0.0f;
    for (int k = 2; k <= nk; ++k)
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                const float r = fabsf(a->tri_residual[P(&g, k, j, i)]);
                if (r > rmax) rmax = r;
            }
    if (diag) {
        diag[0] = (float)nloop;
        diag[1] = dts;
        diag[2] = rmax;
    }
    free(xu);
    free(yv);
    return 0;
}

/* the open-lateral fills on their own (GM1B_FILL_* kinds) */
void oracle_open_fill(int ni, int nj, int nk, int kind, float *q) {
    const G g = {ni, nj, nk};
    switch (kind) {
        case 0: bcp_open(q, &g); break;
        case 1: bcs_open(q, &g, 1, nk); break;
        case 2: bcu_open(q, &g); break;
        case 3: bcv_open(q, &g); break;
        case 4: bcw_open_flag1(q, &g); break;
        case 5: bcs_open(q, &g, 2, nk); break;
        default: break;
    }
}

/* ---------------------------------------------------------------------- */
/* the flat stretched column (terrain_flag=.false.)                        */
/* cuda_gm1_child_psolver3_open.py:343-507 (the flat texts) and :1618-1795 */
/* (their order): the terrain stage's substeps less the u/v reconstruction */
/* before the open-edge update and every bcwsfc.                           */
/* ---------------------------------------------------------------------- */

/* sound.F:119-143: qk, pk1, pk2 and mm from rdz*mh(k) / rdz*mf(k) and the
 * column's base state at CM1's (1,1,k); mm at every level */
static void prepare_flat(TosArrays *a, const TosMetrics *m, const G *g, const float *mh, const float *mf, float rdz,
                         float dts) {
    const int ni = g->ni, nj = g->nj, nk = g->nk;
    const size_t np = (size_t)(nk + 2) * (nj + 2) * (ni + 2);
    float *scratch[NSCRATCH] = {a->qk, a->pk1, a->pk2, a->mm, a->fpk, a->divh, a->hadvp, a->dum3,
                                a->elim_c, a->elim_d, a->tri_aa, a->tri_bb, a->tri_cc, a->tri_dd, a->tri_pivot,
                                a->tri_residual};
    for (int s = 0; s < NSCRATCH; ++s) memset(scratch[s], 0, np * sizeof(float));
    const float cp = 1005.7f;
    for (int k = 1; k <= nk; ++k) {
        const float t0 = (dts * rdz) * mh[k];
        const float rr = m->rr0[M(g, k - 1, 0, 0)];
        const float r2 = (t0 * rr) * m->rf0[M(g, k, 0, 0)];
        const float r1 = (t0 * rr) * m->rf0[M(g, k - 1, 0, 0)];
        const float tem1 = ((dts * rdz) * cp) * mf[k];
        const float c1a = m->c1[M(g, k - 1, 0, 0)], c1b = m->c1[M(g, k, 0, 0)];
        const float c2a = m->c2[M(g, k - 1, 0, 0)], c2b = m->c2[M(g, k, 0, 0)];
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                const size_t c = P(g, k, j, i);
                a->qk[c] = t0 * a->ppterm[c];
                a->pk2[c] = r2 * ((-c2b) * a->piadv[P(g, k + 1, j, i)] + (1.0f - c1b) * a->piadv[c]);
                a->pk1[c] = r1 * (c1a * a->piadv[P(g, k - 1, j, i)] + (c2a - 1.0f) * a->piadv[c]);
                a->mm[c] = tem1 * (c2a * a->thv[c] + c1a * a->thv[P(g, k - 1, j, i)]);
                if (k == 1) a->pk1[c] = 0.0f;
                if (k == nk) a->pk2[c] = 0.0f;
            }
    }
}

/* bc.F:2410-2419 and its three twins: u(1) = u(1) + dts*(((-radbcw*(u(2)-u(1)))
 * *rdx)*uh(1) + uten(1)) on each open side (code 2 in the side's nibble) */
static void ssopen_flat(TosArrays *a, const G *g, float dts, float rdx, float rdy, unsigned obc) {
    const int ni = g->ni, nj = g->nj, nk = g->nk;
    const size_t ry = (size_t)nj + 6, rx = (size_t)ni + 6;
    for (int k = 1; k <= nk; ++k)
        for (int j0 = 0; j0 < nj; ++j0) {
            const int y = j0 + 3;
            if ((obc & 15u) == 2u) {
                const size_t b = U(g, k, y, 3);
                const float t = (((-a->radbcw[k * ry + y]) * (a->u3d[U(g, k, y, 4)] - a->u3d[b])) * rdx) * a->uh[3] +
                                a->uten[b];
                a->u3d[b] = a->u3d[b] + dts * t;
            }
            if (((obc >> 4) & 15u) == 2u) {
                const size_t b = U(g, k, y, ni + 3);
                const float t = (((-a->radbce[k * ry + y]) * (a->u3d[b] - a->u3d[U(g, k, y, ni + 2)])) * rdx) *
                                    a->uh[ni + 2] + a->uten[b];
                a->u3d[b] = a->u3d[b] + dts * t;
            }
        }
    for (int k = 1; k <= nk; ++k)
        for (int i0 = 0; i0 < ni; ++i0) {
            const int x = i0 + 3;
            if (((obc >> 8) & 15u) == 2u) {
                const size_t b = V(g, k, 3, x);
                const float t = (((-a->radbcs[k * rx + x]) * (a->v3d[V(g, k, 4, x)] - a->v3d[b])) * rdy) * a->vh[3] +
                                a->vten[b];
                a->v3d[b] = a->v3d[b] + dts * t;
            }
            if (((obc >> 12) & 15u) == 2u) {
                const size_t b = V(g, k, nj + 3, x);
                const float t = (((-a->radbcn[k * rx + x]) * (a->v3d[b] - a->v3d[V(g, k, nj + 2, x)])) * rdy) *
                                    a->vh[nj + 2] + a->vten[b];
                a->v3d[b] = a->v3d[b] + dts * t;
            }
        }
}

/* sound.F:318-342: every face i = 1..ni+1, j = 1..nj+1 takes u + (dts*dtu0)*
 * (uten - pgrad), dtu0 = 1 on the faces param.F:9182-9219 admits (a
 * periodic side's boundary face included), 0 elsewhere */
static void pgrad_flat(TosArrays *a, const G *g, float dts, float rdx, float rdy, unsigned obc) {
    const int ni = g->ni, nj = g->nj, nk = g->nk;
    const float cp = 1005.7f, tem1 = (rdx * cp) * 0.5f, tem2 = (rdy * cp) * 0.5f;
    const int pw = (obc & 15u) == 1u, pe = ((obc >> 4) & 15u) == 1u;
    const int ps = ((obc >> 8) & 15u) == 1u, pn = ((obc >> 12) & 15u) == 1u;
    for (int k = 1; k <= nk; ++k)
        for (int j = 1; j <= nj + 1; ++j)
            for (int i = 1; i <= ni + 1; ++i) {
                const float wu = (j <= nj && (i > 1 || pw) && (i < ni + 1 || pe)) ? 1.0f : 0.0f;
                const float wv = (i <= ni && (j > 1 || ps) && (j < nj + 1 || pn)) ? 1.0f : 0.0f;
                const size_t c = P(g, k, j, i);
                float pu = tem1 * (a->ppd[c] - a->ppd[P(g, k, j, i - 1)]);
                pu = pu * (a->thv[c] + a->thv[P(g, k, j, i - 1)]);
                const size_t xu = U(g, k, j + 2, i + 2);
                a->u3d[xu] = a->u3d[xu] + (dts * wu) * (a->uten[xu] - pu);
                float pv = tem2 * (a->ppd[c] - a->ppd[P(g, k, j - 1, i)]);
                pv = pv * (a->thv[c] + a->thv[P(g, k, j - 1, i)]);
                const size_t xv = V(g, k, j + 2, i + 2);
                a->v3d[xv] = a->v3d[xv] + (dts * wv) * (a->vten[xv] - pv);
            }
}

/* sound.F:491-509: fpk = ((dts*(ppten - ppterm*div)) + H) + beta*W with the
 * flat divergence and pressure advection */
static void initial_flat(TosArrays *a, const G *g, float dts, float rdx, float rdy, float beta, int do_div) {
    const int ni = g->ni, nj = g->nj, nk = g->nk;
    const float temx = (dts * 0.5f) * rdx, temy = (dts * 0.5f) * rdy;
    for (int k = 1; k <= nk; ++k)
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                const int y = Y(j), x = X(i);
                const size_t c = P(g, k, j, i);
                const float uw = a->u3d[U(g, k, y, x)], ue = a->u3d[U(g, k, y, x + 1)];
                const float vs = a->v3d[V(g, k, y, x)], vn = a->v3d[V(g, k, y + 1, x)];
                float div = 0.0f;
                if (do_div) {
                    div = (ue - uw) * rdx + (vn - vs) * rdy;
                    if (fabsf(div) < 1.0e-30f) div = 0.0f;
                }
                const float pc = a->piadv[c];
                float hx = uw * (pc - a->piadv[P(g, k, j, i - 1)]) + ue * (a->piadv[P(g, k, j, i + 1)] - pc);
                hx = (-hx) * temx;
                float hy = vs * (pc - a->piadv[P(g, k, j - 1, i)]) + vn * (a->piadv[P(g, k, j + 1, i)] - pc);
                hy = (-hy) * temy;
                const float hp = hx + hy;
                const float vert = a->w3d[W(g, k, y, x)] * (a->pk1[c] + a->qk[c]) +
                                   a->w3d[W(g, k + 1, y, x)] * (a->pk2[c] - a->qk[c]);
                a->divh[c] = div;
                a->hadvp[c] = hp;
                a->fpk[c] = ((dts * (a->ppten[c] - a->ppterm[c] * div)) + hp) + beta * vert;
            }
}

int oracle_terrain_open_stage_flat(TosArrays *a, const TosMetrics *m, int ni, int nj, int nk, int nrk, float dt,
                                   int nsound, float dx, float dy, const float *mh, const float *mf, float rdz,
                                   unsigned obc, float alph, float kdiv, unsigned ablations, float *diag) {
    if (ni < 3 || nj < 3 || nk < 4 || nrk < 1 || nrk > 3 || !mh || !mf) return -1;
    const G g = {ni, nj, nk};
    int nloop;
    float dts;
    if (oracle_stage_schedule(dt, nsound, nrk, &nloop, &dts) != 0) return -1;
    const float beta = 1.0f - alph;
    const float rdx = 1.0f / dx, rdy = 1.0f / dy;
    prepare_flat(a, m, &g, mh, mf, rdz, dts);
    for (int k = 1; k <= nk; ++k)
        for (int j = 0; j <= nj + 1; ++j)
            for (int i = 0; i <= ni + 1; ++i) {
                a->ppd[P(&g, k, j, i)] = a->ppx[P(&g, k, j, i)];
                if (nrk != 1) a->pp3d[P(&g, k, j, i)] = a->ppi[P(&g, k, j, i)];
            }
    for (int k = 1; k <= nk; ++k)
        for (int j = 0; j <= nj + 1; ++j)
            for (int i = 0; i <= ni + 1; ++i) {
                const int y = Y(j), x = X(i);
                a->rru[U(&g, k, y, x)] = 0.0f;
                a->rrv[V(&g, k, y, x)] = 0.0f;
                a->rrw[W(&g, k, y, x)] = a->wa[W(&g, k, y, x)] * beta;
                if (nrk != 1) {
                    a->u3d[U(&g, k, y, x)] = a->ua[U(&g, k, y, x)];
                    a->v3d[V(&g, k, y, x)] = a->va[V(&g, k, y, x)];
                    a->w3d[W(&g, k, y, x)] = a->wa[W(&g, k, y, x)];
                }
            }
    for (int n = 1; n <= nloop; ++n) {
        if (ablations & ABL_OPEN) ssopen_flat(a, &g, dts, rdx, rdy, obc);
        if (ablations & ABL_PGRAD) pgrad_flat(a, &g, dts, rdx, rdy, obc);
        initial_flat(a, &g, dts, rdx, rdy, beta, (ablations & ABL_DIV) != 0);
        implicit_and_update(a, &g, dts, nrk, n, nloop, alph, beta, kdiv, (ablations & ABL_IMPLICIT) != 0, 1);
        if (n < nloop && (ablations & ABL_PFILL)) bcp_open(a->ppd, &g);
        average_velocities(a, &g, n, nloop, alph);
    }
    if (ablations & ABL_RADIATION) radiation4(a, &g, dx, dy, oracle_rk_stage_dt(dt, nrk));
    if (ablations & ABL_FILLS) {
        bcu_open(a->u3d, &g);
        bcv_open(a->v3d, &g);
        bcw_open_flag1(a->w3d, &g);
        if (nrk < 3) {
            bcp_open(a->pp3d, &g);
            bcs_open(a->scalar, &g, 1, nk);
        }
    }
    if (diag) {
        diag[0] = (float)nloop;
        diag[1] = dts;
        diag[2] = 0.0f;
    }
    return 0;
}
