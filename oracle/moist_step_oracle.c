/* moist_step_oracle.c - TEST INFRASTRUCTURE ONLY (never linked by the
 * product).  CPU restatement, one binary32 operation at a time in the
 * reference's order, of the pieces that join the operators of the moist
 * large step (their reference counterparts exist as CUDA source only):
 *
 *   moist buoyancy, getdiv, getdivx      src/cm1core/cuda_moist_stage_bridge.py:160-194
 *   final-stage moisture pdef chain      src/cm1core/cuda_scalar_moist_rk.py:560-700
 *   held-tendency composition            src/cm1core/cuda_gm1_child_step_composer.py:547-556
 *   solve3 density                       src/cm1core/cuda_gm1_forecast.py:548
 *
 * The interior of the pdef candidate/correction pair is the reference's CPU
 * twin cpu_pdef_direction_inplace (pinned in rk_oracle.c); the rest follows
 * the kernel source word for word.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include "real.h"

typedef struct {
    int ni, nj, nk;
} Ln;

static inline size_t S(const Ln *L, int k, int y, int x) { return ((size_t)k * (L->nj + 6) + y) * (L->ni + 6) + x; }
static inline size_t Uu(const Ln *L, int k, int y, int x) { return ((size_t)k * (L->nj + 6) + y) * (L->ni + 7) + x; }
static inline size_t Vv(const Ln *L, int k, int y, int x) { return ((size_t)k * (L->nj + 7) + y) * (L->ni + 6) + x; }
static inline size_t Mm(const Ln *L, int k0, int j0, int i0) { return ((size_t)k0 * L->nj + j0) * L->ni + i0; }

/* ------------------------------------------------------------------ */
static float buoy_face(const float *dum8, const float *c1, const float *c2, const Ln *L, int kf, int j, int i) {
    if (kf == 1 || kf == L->nk + 1) return 0.0f;
    const size_t p = Mm(L, kf - 1, j, i);
    return c1[p] * dum8[S(L, kf - 1, j + 3, i + 3)] + c2[p] * dum8[S(L, kf, j + 3, i + 3)];
}

/* the flat column's buoyancy (launch_cuda_gm1_flat_stretched_buoyancy,
 * src/cm1core/cuda_gm1_child_stretched_moist.py:240): wten only */
void oracle_moist_buoyancy_flat(int ni, int nj, int nk, const float *dum8, const float *c1, const float *c2,
                                float *wten) {
    const Ln L = {ni, nj, nk};
    for (int kf = 2; kf <= nk; ++kf)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                const size_t p = Mm(&L, kf - 1, j, i);
                const float add = c1[p] * dum8[S(&L, kf - 1, j + 3, i + 3)] + c2[p] * dum8[S(&L, kf, j + 3, i + 3)];
                const size_t d = S(&L, kf, j + 3, i + 3);
                wten[d] = wten[d] + add;
            }
}

void oracle_moist_buoyancy(int ni, int nj, int nk, const float *dum8, const float *c1, const float *c2,
                           const float *gxu, const float *gyv, float *uten, float *vten, float *wten) {
    const Ln L = {ni, nj, nk};
    oracle_moist_buoyancy_flat(ni, nj, nk, dum8, c1, c2, wten);
    for (int k = 1; k <= nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int f = 1; f < ni; ++f) {
                float t = (buoy_face(dum8, c1, c2, &L, k + 1, j, f) + buoy_face(dum8, c1, c2, &L, k + 1, j, f - 1)) +
                          (buoy_face(dum8, c1, c2, &L, k, j, f) + buoy_face(dum8, c1, c2, &L, k, j, f - 1));
                t = 0.125f * t;
                t = t - 0.25f * (dum8[S(&L, k, j + 3, f + 3)] + dum8[S(&L, k, j + 3, f + 2)]);
                t = t * (gxu[((size_t)(k - 1) * nj + j) * (ni + 1) + f] + gxu[((size_t)k * nj + j) * (ni + 1) + f]);
                const size_t d = Uu(&L, k, j + 3, f + 3);
                uten[d] = uten[d] + t;
            }
    for (int k = 1; k <= nk; ++k)
        for (int f = 1; f < nj; ++f)
            for (int i = 0; i < ni; ++i) {
                float t = (buoy_face(dum8, c1, c2, &L, k + 1, f, i) + buoy_face(dum8, c1, c2, &L, k + 1, f - 1, i)) +
                          (buoy_face(dum8, c1, c2, &L, k, f, i) + buoy_face(dum8, c1, c2, &L, k, f - 1, i));
                t = 0.125f * t;
                t = t - 0.25f * (dum8[S(&L, k, f + 3, i + 3)] + dum8[S(&L, k, f + 2, i + 3)]);
                t = t * (gyv[((size_t)(k - 1) * (nj + 1) + f) * ni + i] + gyv[((size_t)k * (nj + 1) + f) * ni + i]);
                const size_t d = Vv(&L, k, f + 3, i + 3);
                vten[d] = vten[d] + t;
            }
}

/* ------------------------------------------------------------------ */
typedef struct {
    float *rru, *rrv, *rrw;
    const float *rgzu, *rgzv, *dzdx, *dzdy, *gz, *rho0_3d, *rf0, *thterm;
    float *divergence, *theta_divergence_term, *divx;
} post_arrays;

/* the post-acoustic column: mode 0 uniform; 1 terrain branch on a stretched
 * column (sigma/sigmaf/rds/rdsf, physical top, padded base density); 2 flat
 * column (rdz*mh, rho0p(k,3,3), rf0(1,1,k), no terrain w, no rgzu/rgzv) -
 * cuda_gm1_child_stretched_moist.py:35-110 */
typedef struct {
    int mode;
    const float *rho0p, *sigma, *sigmaf, *rds, *rdsf, *mh;
    float ztop, rdz;
} post_column;
static const post_column kUniformPost = {0, 0, 0, 0, 0, 0, 0, 0.0f, 0.0f};

static float gd_xu(const post_arrays *a, const Ln *L, int k, int j, int f, const post_column *c) {
    if (c->mode == 2) return a->rru[Uu(L, k, j + 3, f + 3)];
    return a->rru[Uu(L, k, j + 3, f + 3)] * a->rgzu[(size_t)j * (L->ni + 1) + f];
}
static float gd_yv(const post_arrays *a, const Ln *L, int k, int f, int i, const post_column *c) {
    if (c->mode == 2) return a->rrv[Vv(L, k, f + 3, i + 3)];
    return a->rrv[Vv(L, k, f + 3, i + 3)] * a->rgzv[(size_t)f * L->ni + i];
}
static float gd_wt(const post_arrays *a, const Ln *L, int kf, int j, int i, float dz, const post_column *c) {
    if (kf == 1 || kf == L->nk + 1) return 0.0f;
    if (c->mode == 2) return a->rrw[S(L, kf, j + 3, i + 3)];
    const int pr = c->mode == 1;
    const float rds = pr ? c->rds[kf] : 1.0f / dz;
    const float sf = pr ? c->sigmaf[kf] : (float)(kf - 1) * dz, sm = pr ? c->sigma[kf - 1] : ((float)(kf - 1) - 0.5f) * dz;
    float r2 = (sf - sm) * rds;
    const float r1 = 0.5f * (1.0f - r2);
    r2 = 0.5f * r2;
    const float ux = r2 * (gd_xu(a, L, kf, j, i, c) + gd_xu(a, L, kf, j, i + 1, c)) +
                     r1 * (gd_xu(a, L, kf - 1, j, i, c) + gd_xu(a, L, kf - 1, j, i + 1, c));
    const float vy = r2 * (gd_yv(a, L, kf, j, i, c) + gd_yv(a, L, kf, j + 1, i, c)) +
                     r1 * (gd_yv(a, L, kf - 1, j, i, c) + gd_yv(a, L, kf - 1, j + 1, i, c));
    float terrain = ux * a->dzdx[(size_t)j * L->ni + i] + vy * a->dzdy[(size_t)j * L->ni + i];
    const float zt = pr ? c->ztop : (float)L->nk * dz;
    terrain = ((terrain * (sf - zt)) * a->gz[(size_t)j * L->ni + i]) * (1.0f / zt);
    return a->rrw[S(L, kf, j + 3, i + 3)] + terrain;
}

static void post_acoustic_impl(int ni, int nj, int nk, const post_arrays *a, float dx, float dy, float dz,
                               const post_column *c) {
    const Ln L = {ni, nj, nk};
    const int flat = c->mode == 2, pr = c->mode == 1;
    const float smeps = flat ? 1.0e-30f : 1.0e-20f;
    const float rdx = 1.0f / dx, rdy = 1.0f / dy, rdsf = 1.0f / dz;
    size_t z = 0;
    for (int k = 1; k <= nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i, ++z) {
                float d = (gd_xu(a, &L, k, j, i + 1, c) - gd_xu(a, &L, k, j, i, c)) * rdx +
                          (gd_yv(a, &L, k, j + 1, i, c) - gd_yv(a, &L, k, j, i, c)) * rdy;
                const float dw = gd_wt(a, &L, k + 1, j, i, dz, c) - gd_wt(a, &L, k, j, i, dz, c);
                d = d + (flat ? (dw * c->rdz) * c->mh[k] : dw * (pr ? c->rdsf[k] : rdsf));
                if (fabsf(d) < smeps) d = 0.0f;
                a->divergence[z] = d;
                a->theta_divergence_term[z] = d * a->thterm[z];
            }
    for (int k = 1; k <= nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int f = 0; f <= ni; ++f) {
                const size_t p = Uu(&L, k, j + 3, f + 3);
                if (flat) {
                    a->rru[p] = a->rru[p] * c->rho0p[S(&L, k, 3, 3)];
                    continue;
                }
                const int l = f == 0 ? 0 : f - 1, r = f == ni ? ni - 1 : f;
                const float den = pr ? 0.5f * (c->rho0p[S(&L, k, j + 3, f + 2)] + c->rho0p[S(&L, k, j + 3, f + 3)])
                                     : 0.5f * (a->rho0_3d[Mm(&L, k - 1, j, l)] + a->rho0_3d[Mm(&L, k - 1, j, r)]);
                a->rru[p] = (den * a->rru[p]) * a->rgzu[(size_t)j * (ni + 1) + f];
            }
    for (int k = 1; k <= nk; ++k)
        for (int f = 0; f <= nj; ++f)
            for (int i = 0; i < ni; ++i) {
                const size_t p = Vv(&L, k, f + 3, i + 3);
                if (flat) {
                    a->rrv[p] = a->rrv[p] * c->rho0p[S(&L, k, 3, 3)];
                    continue;
                }
                const int s = f == 0 ? 0 : f - 1, n = f == nj ? nj - 1 : f;
                const float den = pr ? 0.5f * (c->rho0p[S(&L, k, f + 2, i + 3)] + c->rho0p[S(&L, k, f + 3, i + 3)])
                                     : 0.5f * (a->rho0_3d[Mm(&L, k - 1, s, i)] + a->rho0_3d[Mm(&L, k - 1, n, i)]);
                a->rrv[p] = (den * a->rrv[p]) * a->rgzv[(size_t)f * ni + i];
            }
    const float rds = 1.0f / dz, zt = pr ? c->ztop : (float)nk * dz, rzt = 1.0f / zt;
    for (int kf = 1; kf <= nk + 1; ++kf)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                const size_t p = S(&L, kf, j + 3, i + 3);
                if (kf == 1 || kf == nk + 1) {
                    a->rrw[p] = 0.0f;
                    continue;
                }
                if (flat) {
                    a->rrw[p] = a->rrw[p] * a->rf0[Mm(&L, kf - 1, 0, 0)];
                    continue;
                }
                const float sf = pr ? c->sigmaf[kf] : (float)(kf - 1) * dz, sm = pr ? c->sigma[kf - 1] : ((float)(kf - 1) - 0.5f) * dz;
                float r2 = (sf - sm) * (pr ? c->rds[kf] : rds);
                const float r1 = 0.5f * (1.0f - r2);
                r2 = 0.5f * r2;
                const float ux = r2 * (a->rru[Uu(&L, kf, j + 3, i + 3)] + a->rru[Uu(&L, kf, j + 3, i + 4)]) +
                                 r1 * (a->rru[Uu(&L, kf - 1, j + 3, i + 3)] + a->rru[Uu(&L, kf - 1, j + 3, i + 4)]);
                const float vy = r2 * (a->rrv[Vv(&L, kf, j + 3, i + 3)] + a->rrv[Vv(&L, kf, j + 4, i + 3)]) +
                                 r1 * (a->rrv[Vv(&L, kf - 1, j + 3, i + 3)] + a->rrv[Vv(&L, kf - 1, j + 4, i + 3)]);
                float terrain = ux * a->dzdx[(size_t)j * ni + i] + vy * a->dzdy[(size_t)j * ni + i];
                terrain = ((terrain * (sf - zt)) * a->gz[(size_t)j * ni + i]) * rzt;
                a->rrw[p] = a->rf0[Mm(&L, kf - 1, j, i)] * a->rrw[p] + terrain;
            }
    z = 0;
    for (int k = 1; k <= nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i, ++z) {
                float d = (a->rru[Uu(&L, k, j + 3, i + 4)] - a->rru[Uu(&L, k, j + 3, i + 3)]) * rdx +
                          (a->rrv[Vv(&L, k, j + 4, i + 3)] - a->rrv[Vv(&L, k, j + 3, i + 3)]) * rdy;
                const float dw = a->rrw[S(&L, k + 1, j + 3, i + 3)] - a->rrw[S(&L, k, j + 3, i + 3)];
                d = d + (flat ? (dw * c->rdz) * c->mh[k] : dw * (pr ? c->rdsf[k] : rdsf));
                a->divx[z] = fabsf(d) < smeps ? 0.0f : d;
            }
}

void oracle_post_acoustic_flux(int ni, int nj, int nk, const post_arrays *a, float dx, float dy, float dz) {
    post_acoustic_impl(ni, nj, nk, a, dx, dy, dz, &kUniformPost);
}

/* launch_cuda_gm1_child_stretched_post_acoustic (src/cm1core/cuda_gm1_child_stretched_moist.py:286) */
void oracle_post_acoustic_flux_column(int ni, int nj, int nk, const post_arrays *a, float dx, float dy, int flat,
                                      const float *rho0p, const float *sigma, const float *sigmaf, const float *rds,
                                      const float *rdsf, float ztop, const float *mh, float rdz) {
    const post_column c = {flat ? 2 : 1, rho0p, sigma, sigmaf, rds, rdsf, mh, ztop, rdz};
    post_acoustic_impl(ni, nj, nk, a, dx, dy, 1.0f, &c);
}

/* ------------------------------------------------------------------ */
/* final-stage moisture pdef chain                                     */
/* ------------------------------------------------------------------ */
static const float kC13_12 = 0x1.155556p+0f, kCm7_6 = -0x1.2aaaaap+0f, kC11_6 = 0x1.d55556p+0f;
static const float kF3_1 = -0x1.555556p-3f, kF3_2 = 0x1.aaaaaap-1f, kF3_3 = 0x1.555556p-2f, kC1_6 = 0x1.555556p-3f;

static double dmin30(double x) { return x < 1.0e30 ? x : 1.0e30; }
static float weno5(float s1, float s2, float s3, float s4, float s5, double eps) {
    const float d1 = (s1 - 2.0f * s2) + s3, e1 = (s1 - 4.0f * s2) + 3.0f * s3;
    const float b1r = kC13_12 * (d1 * d1) + 0.25f * (e1 * e1);
    const float d2 = (s2 - 2.0f * s3) + s4, e2 = s2 - s4;
    const float b2r = kC13_12 * (d2 * d2) + 0.25f * (e2 * e2);
    const float d3 = (s3 - 2.0f * s4) + s5, e3 = (3.0f * s3 - 4.0f * s4) + s5;
    const float b3r = kC13_12 * (d3 * d3) + 0.25f * (e3 * e3);
    const double b1 = b1r, b2 = b2r, b3 = b3r, tau = fabs(b1 - b3);
    const double q1 = dmin30(tau / (b1 + eps)), q2 = dmin30(tau / (b2 + eps)), q3 = dmin30(tau / (b3 + eps));
    const double w1 = (double)0.1f * (1.0 + q1 * q1), w2 = (double)0.6f * (1.0 + q2 * q2),
                 w3 = (double)0.3f * (1.0 + q3 * q3);
    const float p1 = (kF3_3 * s1 + kCm7_6 * s2) + kC11_6 * s3;
    const float p2 = (kF3_1 * s2 + kF3_2 * s3) + kF3_3 * s4;
    const float p3 = (kF3_3 * s3 + kF3_2 * s4) + kF3_1 * s5;
    return (float)((w1 * (double)p1 + w2 * (double)p2 + w3 * (double)p3) / (w1 + w2 + w3));
}
static float upstrpd(float s1, float s2, float s3, float weps) {
    const float dd = s2 - s1;
    const float se = copysignf(fabsf(weps), dd);
    const float rr = (s3 - s2) / (se + dd);
    const float cand = kC1_6 + kF3_3 * rr;
    const float phi = fmaxf(0.0f, fminf(rr, fminf(cand, 1.0f)));
    return s2 + phi * (s2 - s1);
}
static float max5abs(float a, float b, float c, float d, float e) {
    return fmaxf(fmaxf(fabsf(a), fabsf(b)), fmaxf(fabsf(c), fmaxf(fabsf(d), fabsf(e))));
}
static unsigned obc_side(unsigned obc, unsigned side) { return (obc >> (4u * side)) & 15u; }
static int inflow_lo(int i, unsigned obc, unsigned side, float m) { return i == 0 && obc_side(obc, side) == 2u && m >= 0.0f; }
static int inflow_hi(int i, int n, unsigned obc, unsigned side, float m) {
    return i + 1 == n && obc_side(obc, side) == 2u && m <= 0.0f;
}
static long long pdef_cell(long long c, long long n, unsigned lo, unsigned hi) {
    if (c < 0) return lo == 1u ? c + n : (lo == 2u ? 0 : -c - 1);
    if (c >= n) return hi == 1u ? c - n : (hi == 2u ? n - 1 : 2 * n - 1 - c);
    return c;
}
static float pdef_at(const float *d, long long base, long long stride, long long c, long long n, unsigned lo, unsigned hi) {
    return d[base + pdef_cell(c, n, lo, hi) * stride];
}
static float pdef_ratio(const float *d, long long base, long long stride, long long c, long long n, unsigned lo,
                        unsigned hi) {
    const float v = pdef_at(d, base, stride, c, n, lo, hi);
    if (v >= 0.0f) return 0.0f;
    const float f1 = fmaxf(0.0f, pdef_at(d, base, stride, c - 1, n, lo, hi));
    const float f2 = fmaxf(0.0f, pdef_at(d, base, stride, c + 1, n, lo, hi));
    const float sum = f1 + f2;
    return sum > 1.0e-30f ? fmaxf(v, -sum) / sum : 0.0f;
}
static void pdef_row_mass(const float *d, long long base, long long stride, long long c, long long n, unsigned lo,
                          unsigned hi, float *mass, int *flag) {
    const float v = pdef_at(d, base, stride, c, n, lo, hi);
    if (v < 0.0f) {
        const float r = pdef_ratio(d, base, stride, c, n, lo, hi);
        if (r != 0.0f) {
            const float sum = fmaxf(0.0f, pdef_at(d, base, stride, c - 1, n, lo, hi)) +
                              fmaxf(0.0f, pdef_at(d, base, stride, c + 1, n, lo, hi));
            *mass = 0.0f - sum * r;
            *flag = 1;
        }
    } else if (v > 1.0e-30f) {
        const float rl = pdef_ratio(d, base, stride, c - 1, n, lo, hi), rr = pdef_ratio(d, base, stride, c + 1, n, lo, hi);
        if (rl != 0.0f) *mass = *mass + v * rl, *flag = 1;
        if (rr != 0.0f) *mass = *mass + v * rr, *flag = 1;
    }
}
static float ratio1(const float *d, long long c, long long lo, long long hi, long long stride) {
    if (c <= lo || c >= hi || d[c] >= 0.0f) return 0.0f;
    const float f1 = fmaxf(0.0f, d[c - stride]), f2 = fmaxf(0.0f, d[c + stride]);
    const float sum = f1 + f2;
    return sum > 1.0e-30f ? fmaxf(d[c], -sum) / sum : 0.0f;
}
static float zval(const float *d, long long q, int k, size_t slab, int nk) {
    return (k < 0 || k >= nk) ? 0.0f : d[q + (long long)k * (long long)slab];
}
static float zratio(const float *d, long long base, int k, size_t slab, int nk) {
    const float c = zval(d, base, k, slab, nk);
    if (c >= 0.0f) return 0.0f;
    const float f1 = fmaxf(0.0f, zval(d, base, k - 1, slab, nk)), f2 = fmaxf(0.0f, zval(d, base, k + 1, slab, nk));
    const float sum = f1 + f2;
    return sum > 1.0e-30f ? fmaxf(c, -sum) / sum : 0.0f;
}

typedef struct {
    const float *scalar_a, *scalar_padded, *rho0_3d, *gz, *rgz, *rr0, *c1, *c2, *divx, *rru, *rrv, *rrw;
    float *fx, *fy, *fz, *advx, *advy, *advz, *candidate, *advection;
} chain_arrays;

/* the chain's vertical column: mode 0 uniform (rdz = 1/dz), mode 1 terrain
 * branch with rdsf(k), mode 2 flat column with (x*rdz)*mh(k), the column's
 * rho0(k) / rr0(k) and no gz or rgz (cuda_gm1_child_stretched_scalar.py:160-255,
 * :355-470; pdef.F:37-47, 146-178, 263-275, 381-411, 477-486, 548-557) */
typedef struct {
    int mode;
    const float *rdsf, *mh;
    float rdz;
} chain_column;

static inline float zterm(const chain_column *vc, float x, int k) {
    if (vc->mode == 2) return (x * vc->rdz) * vc->mh[k];
    return x * (vc->mode == 1 ? vc->rdsf[k] : vc->rdz);
}

static void chain_impl(int ni, int nj, int nk, const chain_arrays *a, float dttmp, float dx, float dy,
                       const chain_column *vc, double weps, unsigned obc, int pdefweno, int stop_after_directional) {
    const Ln L = {ni, nj, nk};
    const float *s = a->scalar_padded;
    const float ew = (float)weps;
    const float rdx = 1.0f / dx, rdy = 1.0f / dy, rdt = 1.0f / dttmp;
    const int flat = vc->mode == 2;
    for (int k = 1; k <= nk; ++k)
        for (int j = 0; j <= nj; ++j)
            for (int i = 0; i <= ni; ++i) {
                const int x = i + 3, y = j + 3;
                if (j < nj) {
                    const float m = a->rru[Uu(&L, k, y, x)];
                    float s1, s2, s3, s4, s5;
                    if (m >= 0.0f) s1 = s[S(&L, k, y, x - 3)], s2 = s[S(&L, k, y, x - 2)], s3 = s[S(&L, k, y, x - 1)],
                                   s4 = s[S(&L, k, y, x)], s5 = s[S(&L, k, y, x + 1)];
                    else s1 = s[S(&L, k, y, x + 2)], s2 = s[S(&L, k, y, x + 1)], s3 = s[S(&L, k, y, x)],
                         s4 = s[S(&L, k, y, x - 1)], s5 = s[S(&L, k, y, x - 2)];
                    a->fx[Uu(&L, k, y, x)] = (double)max5abs(s1, s2, s3, s4, s5) > weps ? m * weno5(s1, s2, s3, s4, s5, weps) : 0.0f;
                }
                if (i < ni) {
                    const float m = a->rrv[Vv(&L, k, y, x)];
                    float s1, s2, s3, s4, s5;
                    if (m >= 0.0f) s1 = s[S(&L, k, y - 3, x)], s2 = s[S(&L, k, y - 2, x)], s3 = s[S(&L, k, y - 1, x)],
                                   s4 = s[S(&L, k, y, x)], s5 = s[S(&L, k, y + 1, x)];
                    else s1 = s[S(&L, k, y + 2, x)], s2 = s[S(&L, k, y + 1, x)], s3 = s[S(&L, k, y, x)],
                         s4 = s[S(&L, k, y - 1, x)], s5 = s[S(&L, k, y - 2, x)];
                    a->fy[Vv(&L, k, y, x)] = (double)max5abs(s1, s2, s3, s4, s5) > weps ? m * weno5(s1, s2, s3, s4, s5, weps) : 0.0f;
                }
            }
    for (int k = 2; k <= nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                const int x = i + 3, y = j + 3;
                const float m = a->rrw[S(&L, k, y, x)];
                const size_t cm = ((size_t)(k - 1) * nj + j) * ni + i;
                float r;
                if (k == 2) {
                    r = m >= 0.0f ? a->c1[cm] * s[S(&L, k - 1, y, x)] + a->c2[cm] * s[S(&L, k, y, x)]
                                  : upstrpd(s[S(&L, k + 1, y, x)], s[S(&L, k, y, x)], s[S(&L, k - 1, y, x)], ew);
                } else if (k == nk) {
                    r = m > 0.0f ? upstrpd(s[S(&L, k - 2, y, x)], s[S(&L, k - 1, y, x)], s[S(&L, k, y, x)], ew)
                                 : a->c1[cm] * s[S(&L, k - 1, y, x)] + a->c2[cm] * s[S(&L, k, y, x)];
                } else {
                    const int low = (k == 3 && (pdefweno ? m > 0.0f : m >= 0.0f)) || (k == nk - 1 && m < 0.0f);
                    if (low) {
                        r = k == 3 ? upstrpd(s[S(&L, k - 2, y, x)], s[S(&L, k - 1, y, x)], s[S(&L, k, y, x)], ew)
                                   : upstrpd(s[S(&L, k + 1, y, x)], s[S(&L, k, y, x)], s[S(&L, k - 1, y, x)], ew);
                    } else {
                        float s1, s2, s3, s4, s5;
                        if (m >= 0.0f) s1 = s[S(&L, k - 3, y, x)], s2 = s[S(&L, k - 2, y, x)], s3 = s[S(&L, k - 1, y, x)],
                                       s4 = s[S(&L, k, y, x)], s5 = s[S(&L, k + 1, y, x)];
                        else s1 = s[S(&L, k + 2, y, x)], s2 = s[S(&L, k + 1, y, x)], s3 = s[S(&L, k, y, x)],
                             s4 = s[S(&L, k - 1, y, x)], s5 = s[S(&L, k - 2, y, x)];
                        if (pdefweno && (double)max5abs(s1, s2, s3, s4, s5) <= weps) {
                            a->fz[S(&L, k, y, x)] = 0.0f;
                            continue;
                        }
                        r = weno5(s1, s2, s3, s4, s5, weps);
                    }
                }
                a->fz[S(&L, k, y, x)] = m * r;
            }
    const size_t slab = (size_t)ni * nj, n = slab * nk;
    for (size_t q = 0; q < n; ++q) {
        const int i = (int)(q % ni), j = (int)((q / ni) % nj), k = (int)(q / slab) + 1, x = i + 3, y = j + 3;
        float fw = a->fx[Uu(&L, k, y, x)], fe = a->fx[Uu(&L, k, y, x + 1)], fs = a->fy[Vv(&L, k, y, x)],
              fn = a->fy[Vv(&L, k, y + 1, x)];
        const float uw = a->rru[Uu(&L, k, y, x)], ue = a->rru[Uu(&L, k, y, x + 1)];
        const float vs = a->rrv[Vv(&L, k, y, x)], vn = a->rrv[Vv(&L, k, y + 1, x)];
        const int iw = inflow_lo(i, obc, 0u, uw), ie = inflow_hi(i, ni, obc, 1u, ue);
        const int js = inflow_lo(j, obc, 2u, vs), jn = inflow_hi(j, nj, obc, 3u, vn);
        if (iw) fw = fe;
        if (ie) fe = fw;
        if (js) fs = fn;
        if (jn) fn = fs;
        float axv = (fw - fe) * rdx, ayv = (fs - fn) * rdy;
        if (iw || ie || js || jn) {
            const float sv = s[S(&L, k, y, x)];
            if (iw) axv = axv - (sv * (ue - uw)) * rdx;
            if (ie) axv = axv - (sv * (ue - uw)) * rdx;
            if (js) ayv = ayv - (sv * (vn - vs)) * rdy;
            if (jn) ayv = ayv - (sv * (vn - vs)) * rdy;
        }
        a->advx[q] = axv;
        a->advy[q] = ayv;
        a->advz[q] = k == 1 ? zterm(vc, -a->fz[S(&L, 2, y, x)], k)
                            : (k == nk ? zterm(vc, a->fz[S(&L, nk, y, x)], k)
                                       : zterm(vc, a->fz[S(&L, k, y, x)] - a->fz[S(&L, k + 1, y, x)], k));
    }
    if (stop_after_directional) return;
    for (int axis = 0; axis < 3; ++axis) {
        float *dir = axis == 0 ? a->advx : axis == 1 ? a->advy : a->advz;
        const float rsp = axis == 0 ? rdx : rdy;  /* x and y spacing; z goes through zterm */
        float *d = a->candidate;
        for (size_t q = 0; q < n; ++q) {
            const int i = (int)(q % ni), j = (int)((q / ni) % nj), k = (int)(q / slab) + 1, x = i + 3, y = j + 3;
            float m0, m1;
            int inflow = 0;
            if (axis == 0) {
                m0 = a->rru[Uu(&L, k, y, x)], m1 = a->rru[Uu(&L, k, y, x + 1)];
                inflow = inflow_lo(i, obc, 0u, m0) || inflow_hi(i, ni, obc, 1u, m1);
            } else if (axis == 1) {
                m0 = a->rrv[Vv(&L, k, y, x)], m1 = a->rrv[Vv(&L, k, y + 1, x)];
                inflow = inflow_lo(j, obc, 2u, m0) || inflow_hi(j, nj, obc, 3u, m1);
            } else {
                m0 = a->rrw[S(&L, k, y, x)], m1 = a->rrw[S(&L, k + 1, y, x)];
            }
            const float dm = m1 - m0;
            const float r0a = (flat ? a->rho0_3d[(size_t)(k - 1) * slab] : a->rho0_3d[q]) * a->scalar_a[q];
            const float sdm = s[S(&L, k, y, x)] * dm;
            const float inc = dttmp * (dir[q] + (axis == 2 ? zterm(vc, sdm, k) : sdm * rsp));
            d[q] = inflow ? r0a : (flat ? r0a + inc : r0a + inc * a->gz[(size_t)j * ni + i]);
        }
        for (size_t q = 0; q < n; ++q) {
            const int i = (int)(q % ni), j = (int)((q / ni) % nj), k0 = (int)(q / slab);
            float mass = 0.0f;
            int flag = 0;
            if (axis == 2) {
                const long long base = (long long)(q - (size_t)k0 * slab);
                const float cur = d[q];
                if (cur < 0.0f) {
                    const float r = zratio(d, base, k0, slab, nk);
                    if (r != 0.0f) {
                        const float sum = fmaxf(0.0f, zval(d, base, k0 - 1, slab, nk)) + fmaxf(0.0f, zval(d, base, k0 + 1, slab, nk));
                        mass = 0.0f - sum * r;
                        flag = 1;
                    }
                } else if (cur > 1.0e-30f) {
                    const float rl = zratio(d, base, k0 - 1, slab, nk), rr = zratio(d, base, k0 + 1, slab, nk);
                    if (rl != 0.0f) mass = mass + cur * rl, flag = 1;
                    if (rr != 0.0f) mass = mass + cur * rr, flag = 1;
                }
            } else {
                const int c = axis == 0 ? i : j, nn = axis == 0 ? ni : nj;
                const long long stride = axis == 0 ? 1 : (long long)ni;
                const long long base = (long long)q - (long long)c * stride;
                if (obc != 0u) {
                    pdef_row_mass(d, base, stride, c, nn, obc_side(obc, axis == 0 ? 0u : 2u), obc_side(obc, axis == 0 ? 1u : 3u),
                                  &mass, &flag);
                } else if (c > 0 && c + 1 < nn) {
                    const long long lo = base, hi = base + (long long)(nn - 1) * stride;
                    if (d[q] < 0.0f) {
                        const float r = ratio1(d, (long long)q, lo, hi, stride);
                        if (r != 0.0f) {
                            const float sum = fmaxf(0.0f, d[q - stride]) + fmaxf(0.0f, d[q + stride]);
                            mass = 0.0f - sum * r;
                            flag = 1;
                        }
                    } else if (d[q] > 1.0e-30f) {
                        const float rl = ratio1(d, (long long)q - stride, lo, hi, stride);
                        const float rr = ratio1(d, (long long)q + stride, lo, hi, stride);
                        if (rl != 0.0f) mass = mass + d[q] * rl, flag = 1;
                        if (rr != 0.0f) mass = mass + d[q] * rr, flag = 1;
                    }
                }
            }
            if (flag) {
                const int k = k0 + 1, x = i + 3, y = j + 3;
                const float r0 = flat ? a->rho0_3d[(size_t)k0 * slab] : a->rho0_3d[q];
                float first = ((d[q] + mass) - r0 * a->scalar_a[q]) * rdt;
                if (!flat) first = first * a->rgz[(size_t)j * ni + i];
                float dm;
                if (axis == 0) dm = a->rru[Uu(&L, k, y, x + 1)] - a->rru[Uu(&L, k, y, x)];
                else if (axis == 1) dm = a->rrv[Vv(&L, k, y + 1, x)] - a->rrv[Vv(&L, k, y, x)];
                else dm = a->rrw[S(&L, k + 1, y, x)] - a->rrw[S(&L, k, y, x)];
                const float sdm = s[S(&L, k, y, x)] * dm;
                dir[q] = first - (axis == 2 ? zterm(vc, sdm, k) : sdm * rsp);
            }
        }
    }
    for (size_t q = 0; q < n; ++q) {
        const int i = (int)(q % ni), j = (int)((q / ni) % nj), k = (int)(q / slab) + 1;
        if (!(obc != 0u || (i >= 3 && i + 3 < ni && j >= 3 && j + 3 < nj))) continue;
        float t = (a->advx[q] + a->advy[q]) + a->advz[q];
        t = t + s[S(&L, k, j + 3, i + 3)] * a->divx[q];
        a->advection[q] = flat ? t * a->rr0[(size_t)(k - 1) * slab] : (t * a->rr0[q]) * a->gz[(size_t)j * ni + i];
    }
}

void oracle_pdef_moisture_chain(int ni, int nj, int nk, const chain_arrays *a, float dttmp, float dx, float dy,
                                float dz, double weps, unsigned obc, int pdefweno) {
    const chain_column vc = {0, 0, 0, 1.0f / dz};
    chain_impl(ni, nj, nk, a, dttmp, dx, dy, &vc, weps, obc, pdefweno, 0);
}

/* the chain up to the directional advection (before any repair) */
void oracle_pdef_moisture_directional(int ni, int nj, int nk, const chain_arrays *a, float dttmp, float dx, float dy,
                                      float dz, double weps, unsigned obc, int pdefweno) {
    const chain_column vc = {0, 0, 0, 1.0f / dz};
    chain_impl(ni, nj, nk, a, dttmp, dx, dy, &vc, weps, obc, pdefweno, 1);
}

/* launch_cuda_gm1_child_stretched_pdef_moisture
 * (src/cm1core/cuda_gm1_child_stretched_scalar.py:851): the chain on a
 * stretched column, mode 1 (terrain branch, rdsf(k)) or mode 2 (flat
 * column, rdz*mh(k) with the column's base state). */
void oracle_pdef_moisture_chain_column(int ni, int nj, int nk, const chain_arrays *a, float dttmp, float dx, float dy,
                                       double weps, unsigned obc, int pdefweno, int mode, const float *rdsf,
                                       const float *mh, float rdz) {
    const chain_column vc = {mode, rdsf, mh, rdz};
    chain_impl(ni, nj, nk, a, dttmp, dx, dy, &vc, weps, obc, pdefweno, 0);
}

/* ------------------------------------------------------------------ */
typedef struct {
    const float *th0, *pi0, *rho, *ppi, *tha, *qa, *qpten, *qtten, *qvten, *qcten;
    float *thheld, *qheld, *ppten;
} held_arrays;

void oracle_held_compose(int ni, int nj, int nk, const held_arrays *h, float dt) {
    const size_t n = (size_t)ni * nj * nk;
    const float rd = 287.04f, rv = 461.5f, rp00 = 1.0f / 100000.0f, rddcv = 287.04f / (1005.7f - 287.04f);
    const float tem = 0.0001f * 0.0001f, qsmall = 1.0e-14f;
    for (size_t q = 0; q < n; ++q) {
        const int i = (int)(q % ni), j = (int)((q / ni) % nj), k = (int)(q / ((size_t)ni * nj));
        const size_t pp = ((size_t)(k + 1) * (nj + 2) + (j + 1)) * (size_t)(ni + 2) + (i + 1);
        const float ht = h->thheld[q], qvt = h->qheld[q];
        if (fabsf(dt * ht) > tem || fabsf(dt * qvt) > qsmall) {
            const float thnew = h->tha[q] + dt * ht, qvnew = h->qa[q] + dt * qvt;
            float base = (h->rho[q] * (h->th0[q] + thnew)) * (rd + rv * qvnew);
            base = base * rp00;
            const float pinew = powf(base, rddcv) - h->pi0[q];
            h->ppten[pp] = (pinew - h->ppi[q]) / dt + h->qpten[q];
        } else {
            h->ppten[pp] = h->qpten[q];
        }
        h->thheld[q] = ht + h->qtten[q];
        h->qheld[q] = qvt + h->qvten[q];
        h->qheld[n + q] = h->qheld[n + q] + h->qcten[q];
    }
}

void oracle_solve3_density(int ni, int nj, int nk, const float *rho, const float *c1, const float *c2, float *rr,
                           float *rf) {
    const size_t plane = (size_t)ni * nj, n = plane * nk;
    for (size_t z = 0; z < n; ++z) rr[z] = 1.0f / rho[z];
    for (size_t z = 0; z < plane * (nk + 1); ++z) {
        const size_t h = z % plane;
        const int f = (int)(z / plane);
        if (f == 0) rf[z] = (1.875f * rho[h] + (-1.25f) * rho[plane + h]) + 0.375f * rho[2 * plane + h];
        else if (f == nk)
            rf[z] = (1.875f * rho[(size_t)(nk - 1) * plane + h] + (-1.25f) * rho[(size_t)(nk - 2) * plane + h]) +
                    0.375f * rho[(size_t)(nk - 3) * plane + h];
        else rf[z] = c1[z] * rho[(size_t)(f - 1) * plane + h] + c2[z] * rho[(size_t)f * plane + h];
    }
}

void oracle_pack_scalar(int ni, int nj, int nk, const float *s, float *padded) {
    const Ln L = {ni, nj, nk};
    size_t q = 0;
    for (int k = 1; k <= nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i, ++q) padded[S(&L, k, j + 3, i + 3)] = s[q];
}

void oracle_bcwsfc(int ni, int nj, int nk, const float *u, const float *v, float *w, const float *gz, const float *dzdx,
                   const float *dzdy) {
    const Ln L = {ni, nj, nk};
    for (int j0 = 0; j0 < nj; ++j0)
        for (int i0 = 0; i0 < ni; ++i0) {
            const size_t q = (size_t)j0 * ni + i0;
            const int y = j0 + 3, x = i0 + 3;
            const float ut = (u[Uu(&L, 1, y, x)] + u[Uu(&L, 1, y, x + 1)]) * dzdx[q];
            const float vt = (v[Vv(&L, 1, y, x)] + v[Vv(&L, 1, y + 1, x)]) * dzdy[q];
            w[S(&L, 1, y, x)] = (0.5f * (ut + vt)) * gz[q];
        }
}

void oracle_w_level1_fill(int ni, int nj, int nk, float *w) {
    const int nx = ni + 6, ny = nj + 6;
    float *s = w + (size_t)nx * ny;
    (void)nk;
    for (int y = 0; y < ny; ++y)
        for (int h = 0; h < 3; ++h) s[(size_t)y * nx + h] = s[(size_t)y * nx + 3];
    for (int y = 0; y < ny; ++y)
        for (int h = 0; h < 3; ++h) s[(size_t)y * nx + 3 + ni + h] = s[(size_t)y * nx + 3 + ni - 1];
    for (int h = 0; h < 3; ++h)
        for (int x = 0; x < nx; ++x) s[(size_t)h * nx + x] = s[(size_t)3 * nx + x];
    for (int h = 0; h < 3; ++h)
        for (int x = 0; x < nx; ++x) s[(size_t)(3 + nj + h) * nx + x] = s[(size_t)(3 + nj - 1) * nx + x];
}
