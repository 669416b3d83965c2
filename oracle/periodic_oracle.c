/*
 * periodic_oracle.c - CPU restatement of the reference's NumPy twins for the
 * serial-periodic flat dry lane.  TEST INFRASTRUCTURE ONLY: the checker for
 * the CUDA library, never linked into it or called by it.
 *
 * Arithmetic contract: binary32 storage and binary32 arithmetic, one
 * operation at a time, in the statement order of the NumPy twins, with no
 * contraction (built with -ffp-contract=off) - the same contract as the
 * reference (src/cm1core/records/CM1-ARITHMETIC-CONTRACT.md; NVRTC options
 * src/cm1core/cuda_sound3_periodic.py:1097-1112).  Results are expected to
 * be bit-identical to the NumPy twins; tests/golden holds vectors made by
 * running the reference itself that pin this file.
 *
 * Followed functions (reference file:line):
 *   sound3_stage_schedule_f32        src/cm1core/cuda_sound3_column.py:391-417
 *   rk_stage_dt_f32                  src/cm1core/cuda_sound3_column.py:420-424
 *   fill_periodic_scalar_inplace     src/cm1core/cuda_sound3_periodic.py:506-516
 *   fill_periodic_uv_inplace         src/cm1core/cuda_sound3_periodic.py:519-532
 *   cpu_sound3_periodic_stage_inplace src/cm1core/cuda_sound3_periodic.py:672-1064
 *   _prepare_stage_cpu               src/cm1core/cuda_psolver3_trajectory.py:456-471
 *   _instant_mass_flux_cpu           src/cm1core/cuda_psolver3_trajectory.py:474-493
 *   _scale_averages_cpu              src/cm1core/cuda_psolver3_trajectory.py:496-512
 *   _divergence_cpu                  src/cm1core/cuda_psolver3_trajectory.py:515-533
 *   _momentum_tendencies_cpu         src/cm1core/cuda_psolver3_trajectory.py:536-660
 *   _theta_tendency_update_cpu       src/cm1core/cuda_psolver3_trajectory.py:663-726
 *   _post_step_cpu                   src/cm1core/cuda_psolver3_trajectory.py:735-758
 *   cpu_psolver3_trajectory_inplace  src/cm1core/cuda_psolver3_trajectory.py:761-901
 *   flux helpers _flx3/_flx5/...     src/cm1core/cuda_psolver3_trajectory.py:282-426
 *
 * Loops over independent columns or cells may run on several OpenMP threads;
 * each output word is still produced by the same scalar operation sequence,
 * so the thread count never changes a bit.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "real.h"  /* before the header: its array structs take the working precision */
#include "../include/gm1b.h"

typedef gm1b_periodic_arrays A;

/* binary32 constants, each the correctly rounded float32 quotient the NumPy
 * twins form at run time */
#define F5_1 0x1.111112p-5f  /*   2/60 */
#define F5_2 -0x1.bbbbbcp-3f /* -13/60 */
#define F5_3 0x1.911112p-1f  /*  47/60 */
#define F5_4 0x1.ccccccp-2f  /*  27/60 */
#define F5_5 -0x1.99999ap-5f /*  -3/60 */
#define F3_1 -0x1.555556p-3f /*  -1/6 */
#define F3_2 0x1.aaaaaap-1f  /*   5/6 */
#define F3_3 0x1.555556p-2f  /*   2/6 */
#define RDDCV 0x1.98fef2p-2f /* 287.04 / (1005.7 - 287.04) */
#define GRAV 0x1.39eb86p+3f  /* 9.81 */
#define TH0R 300.0f
#define SMEPS 0x1.4484cp-100f /* 1e-30 */

#define S(p, k, j, i) (p)[((size_t)(k) * (nj + 2) + (size_t)(j)) * (ni + 2) + (size_t)(i)]
#define U(p, k, j, f) (p)[((size_t)(k) * (nj + 2) + (size_t)(j)) * (ni + 1) + (size_t)(f)]
#define V(p, k, g, i) (p)[((size_t)(k) * (nj + 1) + (size_t)(g)) * (ni + 2) + (size_t)(i)]
#define W(p, k, j, i) (p)[((size_t)(k) * nj + (size_t)(j)) * ni + (size_t)(i)]

static inline int pmod(int x, int n) { return ((x % n) + n) % n; }

static size_t scalar_words(int ni, int nj, int nk) { return (size_t)(nk + 2) * (nj + 2) * (ni + 2); }
static size_t u_words(int ni, int nj, int nk) { return (size_t)(nk + 2) * (nj + 2) * (ni + 1); }
static size_t v_words(int ni, int nj, int nk) { return (size_t)(nk + 2) * (nj + 1) * (ni + 2); }
static size_t w_words(int ni, int nj, int nk) { return (size_t)(nk + 2) * nj * ni; }

static void zero(float *p, size_t n) { memset(p, 0, n * sizeof(float)); }

/* --------------------------------------------------------------------- */
/* schedule                                                              */
/* --------------------------------------------------------------------- */

int oracle_stage_schedule(float dt, int nsound, int nrk, int *nloop, float *dts) {
    if (nsound < 4 || (nsound % 2) != 0 || nrk < 1 || nrk > 3) return -1;
    if (nrk == 1) {
        int n = (int)floorf((float)nsound / 3.0f + 0.5f);
        float den = (float)n * 3.0f;
        float d = dt / den;
        float target = dt / (float)nsound;
        if (d > target) {
            n += 1;
            den = (float)n * 3.0f;
            d = dt / den;
        }
        *nloop = n;
        *dts = d;
    } else if (nrk == 2) {
        *nloop = nsound / 2;
        *dts = dt / (float)nsound;
    } else {
        *nloop = nsound;
        *dts = dt / (float)nsound;
    }
    return 0;
}

float oracle_rk_stage_dt(float dt, int nrk) { return dt / (float)(4 - nrk); }

/* --------------------------------------------------------------------- */
/* periodic fills                                                        */
/* --------------------------------------------------------------------- */

void oracle_fill_periodic_scalar(float *p, int ni, int nj, int nk) {
    for (int k = 1; k <= nk; ++k) {
        for (int j = 0; j < nj + 2; ++j) {
            S(p, k, j, 0) = S(p, k, j, ni);
            S(p, k, j, ni + 1) = S(p, k, j, 1);
        }
        for (int i = 0; i < ni + 2; ++i) {
            S(p, k, 0, i) = S(p, k, nj, i);
            S(p, k, nj + 1, i) = S(p, k, 1, i);
        }
    }
}

static void fill_periodic_uv(float *u, float *v, int ni, int nj, int nk) {
    for (int k = 1; k <= nk; ++k) {
        for (int f = 0; f < ni + 1; ++f) {
            U(u, k, 0, f) = U(u, k, nj, f);
            U(u, k, nj + 1, f) = U(u, k, 1, f);
        }
        for (int g = 0; g < nj + 1; ++g) {
            V(v, k, g, 0) = V(v, k, g, ni);
            V(v, k, g, ni + 1) = V(v, k, g, 1);
        }
    }
}

/* --------------------------------------------------------------------- */
/* acoustic stage: cpu_sound3_periodic_stage_inplace                     */
/* --------------------------------------------------------------------- */

int oracle_sound3_periodic_stage(const A *a, int ni, int nj, int nk, float dt, int nsound,
                                 int nrk, float rdx, float rdy, float rdz, float cp,
                                 float alph, float kdiv, float smeps) {
    int nloop;
    float dts;
    if (oracle_stage_schedule(dt, nsound, nrk, &nloop, &dts) != 0) return -1;
    const float beta = 1.0f - alph;
    const float asq = alph * alph;
    const size_t sw = scalar_words(ni, nj, nk);
    float *scratch[] = {a->qk,     a->pk1,    a->pk2,    a->mm,     a->fpk,
                        a->divh,   a->hadvp,  a->elim_c, a->elim_d, a->tri_aa,
                        a->tri_bb, a->tri_cc, a->tri_dd, a->tri_pivot, a->tri_residual};
    for (size_t s = 0; s < sizeof(scratch) / sizeof(scratch[0]); ++s) zero(scratch[s], sw);
    const size_t plane = (size_t)(nj + 2) * (ni + 2);
    memcpy(a->ppd + plane, a->ppx + plane, (size_t)nk * plane * sizeof(float));
    zero(a->rru, u_words(ni, nj, nk));
    zero(a->rrv, v_words(ni, nj, nk));
    if (nrk != 1) {
        memcpy(a->u3d, a->ua, u_words(ni, nj, nk) * sizeof(float));
        memcpy(a->v3d, a->va, v_words(ni, nj, nk) * sizeof(float));
        memcpy(a->pp3d + plane, a->ppi + plane, (size_t)nk * plane * sizeof(float));
    }
#pragma omp parallel for schedule(static)
    for (int j0 = 0; j0 < nj; ++j0) {
        const int j = j0 + 1;
        for (int i0 = 0; i0 < ni; ++i0) {
            const int i = i0 + 1;
            for (int k = 1; k <= nk; ++k) {
                float tem = (dts * rdz) * S(a->mh, k, j, i);
                float r2 = (dts * rdz) * S(a->mh, k, j, i);
                r2 = r2 * S(a->rr0, k, j, i);
                r2 = r2 * S(a->rf0, k + 1, j, i);
                float r1 = (dts * rdz) * S(a->mh, k, j, i);
                r1 = r1 * S(a->rr0, k, j, i);
                r1 = r1 * S(a->rf0, k, j, i);
                float tem1 = ((dts * rdz) * cp) * S(a->mf, k, j, i);
                S(a->qk, k, j, i) = tem * S(a->ppterm, k, j, i);
                S(a->pk2, k, j, i) =
                    r2 * ((-S(a->c2, k + 1, j, i)) * S(a->piadv, k + 1, j, i) +
                          (1.0f - S(a->c1, k + 1, j, i)) * S(a->piadv, k, j, i));
                S(a->pk1, k, j, i) =
                    r1 * (S(a->c1, k, j, i) * S(a->piadv, k - 1, j, i) +
                          (S(a->c2, k, j, i) - 1.0f) * S(a->piadv, k, j, i));
                S(a->mm, k, j, i) = tem1 * (S(a->c2, k, j, i) * S(a->thv, k, j, i) +
                                            S(a->c1, k, j, i) * S(a->thv, k - 1, j, i));
                W(a->rrw, k, j0, i0) = W(a->wa, k, j0, i0) * beta;
                if (nrk != 1) W(a->w3d, k, j0, i0) = W(a->wa, k, j0, i0);
            }
            S(a->pk1, 1, j, i) = 0.0f;
            S(a->pk2, nk, j, i) = 0.0f;
        }
    }
    const float tem1x = (rdx * cp) * 0.5f;
    const float tem2y = (rdy * cp) * 0.5f;
    const float temx = (dts * 0.5f) * rdx;
    const float temy = (dts * 0.5f) * rdy;
    const float tavg = 1.0f / (float)nloop;
    for (int n = 1; n <= nloop; ++n) {
#pragma omp parallel for schedule(static)
        for (int k = 1; k <= nk; ++k) {
            for (int j = 1; j < nj + 2; ++j)
                for (int f = 0; f < ni + 1; ++f) {
                    float pg = tem1x * (S(a->ppd, k, j, f + 1) - S(a->ppd, k, j, f));
                    pg = pg * a->uf[f + 1];
                    pg = pg * (S(a->thv, k, j, f + 1) + S(a->thv, k, j, f));
                    U(a->u3d, k, j, f) = U(a->u3d, k, j, f) +
                                         (dts * a->dtu0[(size_t)j * (ni + 1) + f]) *
                                             (U(a->uten, k, j, f) - pg);
                }
            for (int f = 0; f < nj + 1; ++f)
                for (int i = 1; i < ni + 2; ++i) {
                    float pg = tem2y * (S(a->ppd, k, f + 1, i) - S(a->ppd, k, f, i));
                    pg = pg * a->vf[f + 1];
                    pg = pg * (S(a->thv, k, f + 1, i) + S(a->thv, k, f, i));
                    V(a->v3d, k, f, i) = V(a->v3d, k, f, i) +
                                         (dts * a->dtv0[(size_t)f * (ni + 2) + i]) *
                                             (V(a->vten, k, f, i) - pg);
                }
        }
#pragma omp parallel for schedule(static)
        for (int j0 = 0; j0 < nj; ++j0) {
            const int j = j0 + 1;
            for (int i0 = 0; i0 < ni; ++i0) {
                const int i = i0 + 1;
                for (int k = 1; k <= nk; ++k) {
                    float du = ((U(a->u3d, k, j, i) - U(a->u3d, k, j, i - 1)) * rdx) * a->uh[i];
                    float dv = ((V(a->v3d, k, j, i) - V(a->v3d, k, j - 1, i)) * rdy) * a->vh[j];
                    float div = du + dv;
                    if (fabsf(div) < smeps) div = 0.0f;
                    S(a->divh, k, j, i) = div;
                    float gxw = S(a->piadv, k, j, i) - S(a->piadv, k, j, i - 1);
                    float gxe = S(a->piadv, k, j, i + 1) - S(a->piadv, k, j, i);
                    float gys = S(a->piadv, k, j, i) - S(a->piadv, k, j - 1, i);
                    float gyn = S(a->piadv, k, j + 1, i) - S(a->piadv, k, j, i);
                    float hx = U(a->u3d, k, j, i - 1) * gxw + U(a->u3d, k, j, i) * gxe;
                    hx = ((-hx) * temx) * a->uh[i];
                    float hy = V(a->v3d, k, j - 1, i) * gys + V(a->v3d, k, j, i) * gyn;
                    hy = ((-hy) * temy) * a->vh[j];
                    float hp = hx + hy;
                    S(a->hadvp, k, j, i) = hp;
                    float src = dts * (S(a->ppten, k, j, i) - S(a->ppterm, k, j, i) * div);
                    float vert = W(a->w3d, k, j0, i0) * (S(a->pk1, k, j, i) + S(a->qk, k, j, i)) +
                                 W(a->w3d, k + 1, j0, i0) * (S(a->pk2, k, j, i) - S(a->qk, k, j, i));
                    S(a->fpk, k, j, i) = (src + hp) + beta * vert;
                }
                for (int k = 2; k <= nk; ++k) {
                    float aa = 0.0f, cc = 0.0f;
                    if (k >= 3)
                        aa = (-asq) *
                             (S(a->mm, k, j, i) * (S(a->pk1, k - 1, j, i) + S(a->qk, k - 1, j, i)));
                    if (k < nk)
                        cc = (-asq) *
                             ((-S(a->mm, k, j, i)) * (S(a->pk2, k, j, i) - S(a->qk, k, j, i)));
                    float diag = (-(S(a->pk1, k, j, i) + S(a->qk, k, j, i))) +
                                 (S(a->pk2, k - 1, j, i) - S(a->qk, k - 1, j, i));
                    float bb = 1.0f - asq * (S(a->mm, k, j, i) * diag);
                    float pd = S(a->pp3d, k, j, i) - S(a->pp3d, k - 1, j, i);
                    float fwk = dts * W(a->wten, k, j0, i0) + beta * ((-S(a->mm, k, j, i)) * pd);
                    float upd = (S(a->pp3d, k, j, i) + S(a->fpk, k, j, i)) -
                                (S(a->pp3d, k - 1, j, i) + S(a->fpk, k - 1, j, i));
                    float dd = (W(a->w3d, k, j0, i0) + fwk) + alph * ((-S(a->mm, k, j, i)) * upd);
                    float pivot = (k < 3) ? bb : (aa * S(a->elim_c, k - 1, j, i) + bb);
                    float inv = 1.0f / pivot;
                    S(a->tri_aa, k, j, i) = aa;
                    S(a->tri_bb, k, j, i) = bb;
                    S(a->tri_cc, k, j, i) = cc;
                    S(a->tri_dd, k, j, i) = dd;
                    S(a->tri_pivot, k, j, i) = pivot;
                    if (k < nk) {
                        S(a->elim_c, k, j, i) = (-cc) * inv;
                        float num = (k < 3) ? dd : (dd - aa * S(a->elim_d, k - 1, j, i));
                        S(a->elim_d, k, j, i) = num * inv;
                    } else {
                        W(a->w3d, k, j0, i0) = (dd - aa * S(a->elim_d, k - 1, j, i)) * inv;
                    }
                }
                for (int k = nk - 1; k >= 2; --k)
                    W(a->w3d, k, j0, i0) =
                        S(a->elim_c, k, j, i) * W(a->w3d, k + 1, j0, i0) + S(a->elim_d, k, j, i);
                for (int k = 2; k <= nk; ++k) {
                    float lhs = S(a->tri_aa, k, j, i) * W(a->w3d, k - 1, j0, i0);
                    lhs = lhs + S(a->tri_bb, k, j, i) * W(a->w3d, k, j0, i0);
                    lhs = lhs + S(a->tri_cc, k, j, i) * W(a->w3d, k + 1, j0, i0);
                    S(a->tri_residual, k, j, i) = lhs - S(a->tri_dd, k, j, i);
                }
                for (int k = 1; k <= nk; ++k) {
                    float old = S(a->pp3d, k, j, i);
                    float vert = W(a->w3d, k, j0, i0) * (S(a->pk1, k, j, i) + S(a->qk, k, j, i)) +
                                 W(a->w3d, k + 1, j0, i0) * (S(a->pk2, k, j, i) - S(a->qk, k, j, i));
                    float upd = (old + S(a->fpk, k, j, i)) + alph * vert;
                    if (fabsf(upd) < smeps) upd = 0.0f;
                    S(a->pp3d, k, j, i) = upd;
                    S(a->elim_c, k, j, i) = kdiv * (upd - old);
                    S(a->ppd, k, j, i) = upd + S(a->elim_c, k, j, i);
                    if (nrk == 3 && n == nloop) S(a->ppx, k, j, i) = S(a->elim_c, k, j, i);
                    if (n < nloop)
                        W(a->rrw, k, j0, i0) = W(a->rrw, k, j0, i0) + W(a->w3d, k, j0, i0);
                    else
                        W(a->rrw, k, j0, i0) =
                            (W(a->rrw, k, j0, i0) + W(a->w3d, k, j0, i0) * alph) * (1.0f / (float)nloop);
                }
            }
        }
        if (n < nloop) oracle_fill_periodic_scalar(a->ppd, ni, nj, nk);
#pragma omp parallel for schedule(static)
        for (int k = 1; k <= nk; ++k) {
            for (int j = 1; j < nj + 2; ++j)
                for (int f = 0; f < ni + 1; ++f)
                    U(a->rru, k, j, f) = (n < nloop)
                                             ? U(a->rru, k, j, f) + U(a->u3d, k, j, f)
                                             : (U(a->rru, k, j, f) + U(a->u3d, k, j, f)) * tavg;
            for (int f = 0; f < nj + 1; ++f)
                for (int i = 1; i < ni + 2; ++i)
                    V(a->rrv, k, f, i) = (n < nloop)
                                             ? V(a->rrv, k, f, i) + V(a->v3d, k, f, i)
                                             : (V(a->rrv, k, f, i) + V(a->v3d, k, f, i)) * tavg;
        }
    }
    fill_periodic_uv(a->u3d, a->v3d, ni, nj, nk);
    if (nrk < 3) oracle_fill_periodic_scalar(a->pp3d, ni, nj, nk);
    return nloop;
}

/* --------------------------------------------------------------------- */
/* fifth-order flux helpers                                              */
/* --------------------------------------------------------------------- */

static inline float flx3(float s1, float s2, float s3) {
    float r = F3_1 * s1;
    r = r + F3_2 * s2;
    return r + F3_3 * s3;
}

static inline float flx5(float s1, float s2, float s3, float s4, float s5) {
    float r = F5_1 * s1;
    r = r + F5_2 * s2;
    r = r + F5_3 * s3;
    r = r + F5_4 * s4;
    return r + F5_5 * s5;
}

/* A view of a field restricted to its live block, indexed (k, j, i) from 0,
 * with modulo wrap in x and y where the twin applies it. */
typedef struct {
    const float *p;
    int nz, ny, nx;           /* view extents */
    size_t sz, sy;            /* strides of the padded array */
    int oz, oy, ox;           /* offsets into the padded array */
} view3;

static inline float vat(const view3 *v, int k, int j, int i) {
    return v->p[(size_t)(k + v->oz) * v->sz + (size_t)(j + v->oy) * v->sy + (size_t)(i + v->ox)];
}

/* _scalar_x_flux: state[k, j, i % nx] */
static float scalar_x_flux(const view3 *s, float vel, int face, int j, int k) {
    int q0, q1, q2, q3, q4;
    if (vel >= 0.0f) { q0 = face - 3; q1 = face - 2; q2 = face - 1; q3 = face; q4 = face + 1; }
    else { q0 = face + 2; q1 = face + 1; q2 = face; q3 = face - 1; q4 = face - 2; }
    int n = s->nx;
    float r = flx5(vat(s, k, j, pmod(q0, n)), vat(s, k, j, pmod(q1, n)), vat(s, k, j, pmod(q2, n)),
                   vat(s, k, j, pmod(q3, n)), vat(s, k, j, pmod(q4, n)));
    return vel * r;
}

/* _scalar_y_flux: state[k, j % ny, i] */
static float scalar_y_flux(const view3 *s, float vel, int i, int face, int k) {
    int q0, q1, q2, q3, q4;
    if (vel >= 0.0f) { q0 = face - 3; q1 = face - 2; q2 = face - 1; q3 = face; q4 = face + 1; }
    else { q0 = face + 2; q1 = face + 1; q2 = face; q3 = face - 1; q4 = face - 2; }
    int n = s->ny;
    float r = flx5(vat(s, k, pmod(q0, n), i), vat(s, k, pmod(q1, n), i), vat(s, k, pmod(q2, n), i),
                   vat(s, k, pmod(q3, n), i), vat(s, k, pmod(q4, n), i));
    return vel * r;
}

static float centered_x_flux(const view3 *s, float vel, int b, int j, int k) {
    int q0, q1, q2, q3, q4;
    if (vel >= 0.0f) { q0 = b - 2; q1 = b - 1; q2 = b; q3 = b + 1; q4 = b + 2; }
    else { q0 = b + 3; q1 = b + 2; q2 = b + 1; q3 = b; q4 = b - 1; }
    int n = s->nx;
    float r = flx5(vat(s, k, j, pmod(q0, n)), vat(s, k, j, pmod(q1, n)), vat(s, k, j, pmod(q2, n)),
                   vat(s, k, j, pmod(q3, n)), vat(s, k, j, pmod(q4, n)));
    return vel * r;
}

static float centered_y_flux(const view3 *s, float vel, int i, int b, int k) {
    int q0, q1, q2, q3, q4;
    if (vel >= 0.0f) { q0 = b - 2; q1 = b - 1; q2 = b; q3 = b + 1; q4 = b + 2; }
    else { q0 = b + 3; q1 = b + 2; q2 = b + 1; q3 = b; q4 = b - 1; }
    int n = s->ny;
    float r = flx5(vat(s, k, pmod(q0, n), i), vat(s, k, pmod(q1, n), i), vat(s, k, pmod(q2, n), i),
                   vat(s, k, pmod(q3, n), i), vat(s, k, pmod(q4, n), i));
    return vel * r;
}

/* _vertical_mass_flux: CM1 stag=1/2/3 flux at Fortran face `face`, nk = nz */
static float vertical_mass_flux(const view3 *s, float v, int face, int j, int i, float c1, float c2) {
    const int nk = s->nz;
#define SZ(z) vat(s, (z), j, i)
    float recon;
    if (face == 2) {
        recon = (v >= 0.0f) ? (c1 * SZ(0) + c2 * SZ(1)) : flx3(SZ(2), SZ(1), SZ(0));
    } else if (face == 3) {
        recon = (v >= 0.0f) ? flx3(SZ(0), SZ(1), SZ(2)) : flx5(SZ(4), SZ(3), SZ(2), SZ(1), SZ(0));
    } else if (face == nk - 1) {
        recon = (v >= 0.0f) ? flx5(SZ(nk - 5), SZ(nk - 4), SZ(nk - 3), SZ(nk - 2), SZ(nk - 1))
                            : flx3(SZ(nk - 1), SZ(nk - 2), SZ(nk - 3));
    } else if (face == nk) {
        recon = (v >= 0.0f) ? flx3(SZ(nk - 3), SZ(nk - 2), SZ(nk - 1))
                            : (c1 * SZ(nk - 2) + c2 * SZ(nk - 1));
    } else {
        if (v >= 0.0f)
            recon = flx5(SZ(face - 4), SZ(face - 3), SZ(face - 2), SZ(face - 1), SZ(face));
        else
            recon = flx5(SZ(face + 1), SZ(face), SZ(face - 1), SZ(face - 2), SZ(face - 3));
    }
#undef SZ
    return v * recon;
}

/* _vertical_w_flux: CM1 stag=4 flux at mass level `level` (1..nk), nk = nz-1 */
static float vertical_w_flux(const view3 *s, float v, int level, int j, int i) {
    const int nk = s->nz - 1;
#define SZ(z) vat(s, (z), j, i)
    float recon;
    if (level == 1) {
        recon = (v >= 0.0f) ? (0.5f * (SZ(0) + SZ(1))) : flx3(SZ(2), SZ(1), SZ(0));
    } else if (level == 2) {
        recon = (v >= 0.0f) ? flx3(SZ(0), SZ(1), SZ(2)) : flx5(SZ(5), SZ(4), SZ(3), SZ(2), SZ(1));
    } else if (level == nk - 1) {
        recon = (v >= 0.0f) ? flx5(SZ(nk - 4), SZ(nk - 3), SZ(nk - 2), SZ(nk - 1), SZ(nk))
                            : flx3(SZ(nk), SZ(nk - 1), SZ(nk - 2));
    } else if (level == nk) {
        recon = (v >= 0.0f) ? flx3(SZ(nk - 2), SZ(nk - 1), SZ(nk)) : (0.5f * (SZ(nk - 1) + SZ(nk)));
    } else {
        if (v >= 0.0f)
            recon = flx5(SZ(level - 3), SZ(level - 2), SZ(level - 1), SZ(level), SZ(level + 1));
        else
            recon = flx5(SZ(level + 2), SZ(level + 1), SZ(level), SZ(level - 1), SZ(level - 2));
    }
#undef SZ
    return v * recon;
}

/* --------------------------------------------------------------------- */
/* trajectory pieces                                                     */
/* --------------------------------------------------------------------- */

void oracle_traj_prepare(const A *a, int ni, int nj, int nk) {
    for (int k = 1; k <= nk; ++k)
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                S(a->thv, k, j, i) = S(a->th0, k, j, i) + S(a->th3d, k, j, i);
                S(a->piadv, k, j, i) = S(a->pi0, k, j, i) + S(a->pp3d, k, j, i);
                S(a->ppterm, k, j, i) = S(a->piadv, k, j, i) * RDDCV;
            }
    oracle_fill_periodic_scalar(a->thv, ni, nj, nk);
    oracle_fill_periodic_scalar(a->piadv, ni, nj, nk);
    size_t sw = scalar_words(ni, nj, nk);
    zero(a->ppten, sw);
    zero(a->thten, sw);
    zero(a->uten, u_words(ni, nj, nk));
    zero(a->vten, v_words(ni, nj, nk));
    zero(a->wten, w_words(ni, nj, nk));
}

void oracle_traj_instant_mass_flux(const A *a, int ni, int nj, int nk) {
    zero(a->rru, u_words(ni, nj, nk));
    zero(a->rrv, v_words(ni, nj, nk));
    zero(a->rrw, w_words(ni, nj, nk));
    for (int k = 1; k <= nk; ++k) {
        for (int j = 1; j <= nj; ++j)
            for (int f = 0; f < ni + 1; ++f)
                U(a->rru, k, j, f) = S(a->rho0, k, j, 1) * U(a->u3d, k, j, f);
        for (int f = 0; f < nj + 1; ++f)
            for (int i = 1; i <= ni; ++i)
                V(a->rrv, k, f, i) = S(a->rho0, k, 1, i) * V(a->v3d, k, f, i);
    }
    for (int q = 2; q <= nk; ++q)
        for (int j0 = 0; j0 < nj; ++j0)
            for (int i0 = 0; i0 < ni; ++i0)
                W(a->rrw, q, j0, i0) = S(a->rf0, q, j0 + 1, i0 + 1) * W(a->w3d, q, j0, i0);
}

void oracle_traj_scale_averages(const A *a, int ni, int nj, int nk) {
    for (int k = 1; k <= nk; ++k) {
        for (int j = 1; j <= nj; ++j)
            for (int f = 0; f < ni + 1; ++f)
                U(a->rru, k, j, f) = U(a->rru, k, j, f) * S(a->rho0, k, j, 1);
        for (int f = 0; f < nj + 1; ++f)
            for (int i = 1; i <= ni; ++i)
                V(a->rrv, k, f, i) = V(a->rrv, k, f, i) * S(a->rho0, k, 1, i);
    }
    for (int q = 2; q <= nk; ++q)
        for (int j0 = 0; j0 < nj; ++j0)
            for (int i0 = 0; i0 < ni; ++i0)
                W(a->rrw, q, j0, i0) = W(a->rrw, q, j0, i0) * S(a->rf0, q, j0 + 1, i0 + 1);
    memset(&W(a->rrw, 1, 0, 0), 0, (size_t)nj * ni * sizeof(float));
    memset(&W(a->rrw, nk + 1, 0, 0), 0, (size_t)nj * ni * sizeof(float));
}

void oracle_traj_divergence(const A *a, int ni, int nj, int nk, float rdx, float rdy, float rdz) {
    zero(a->divx, scalar_words(ni, nj, nk));
    for (int k = 1; k <= nk; ++k)
        for (int j0 = 0; j0 < nj; ++j0)
            for (int i0 = 0; i0 < ni; ++i0) {
                int j = j0 + 1, i = i0 + 1;
                float dx = (U(a->rru, k, j, i0 + 1) - U(a->rru, k, j, i0)) * rdx;
                float dy = (V(a->rrv, k, j0 + 1, i) - V(a->rrv, k, j0, i)) * rdy;
                float dz = (W(a->rrw, k + 1, j0, i0) - W(a->rrw, k, j0, i0)) * rdz;
                float value = (dx + dy) + dz;
                if (fabsf(value) < SMEPS) value = 0.0f;
                S(a->divx, k, j, i) = value;
            }
}

void oracle_traj_momentum(const A *a, int ni, int nj, int nk, float rdx, float rdy, float rdz,
                          int momentum_advection, int buoyancy) {
    const size_t ssz = (size_t)(nj + 2) * (ni + 2), ssy = (size_t)(ni + 2);
    const size_t usz = (size_t)(nj + 2) * (ni + 1), usy = (size_t)(ni + 1);
    const size_t vsz = (size_t)(nj + 1) * (ni + 2), vsy = (size_t)(ni + 2);
    const size_t wsz = (size_t)nj * ni, wsy = (size_t)ni;
    const view3 u = {a->u3d, nk, nj, ni, usz, usy, 1, 1, 0};
    const view3 v = {a->v3d, nk, nj, ni, vsz, vsy, 1, 0, 1};
    const view3 w = {a->w3d, nk + 1, nj, ni, wsz, wsy, 1, 0, 0};
    const view3 rru = {a->rru, nk, nj, ni, usz, usy, 1, 1, 0};
    const view3 rrv = {a->rrv, nk, nj, ni, vsz, vsy, 1, 0, 1};
    const view3 rrw = {a->rrw, nk + 1, nj, ni, wsz, wsy, 1, 0, 0};
    const view3 dv = {a->divx, nk, nj, ni, ssz, ssy, 1, 1, 1};
    if (momentum_advection) {
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nk; ++k) {
            const int ks = k + 1;
            for (int j = 0; j < nj; ++j) {
                const int js = j + 1;
                for (int f = 0; f < ni + 1; ++f) {
                    const int fu = f % ni;
                    const int fm = pmod(fu - 1, ni), fp = (fu + 1) % ni;
                    float east_v = 0.5f * (vat(&rru, k, j, fu) + vat(&rru, k, j, fp));
                    float west_v = 0.5f * (vat(&rru, k, j, fm) + vat(&rru, k, j, fu));
                    float fx_e = centered_x_flux(&u, east_v, fu, j, k);
                    float fx_w = centered_x_flux(&u, west_v, fu - 1, j, k);
                    const int jn = (j + 1) % nj;
                    float south_v = 0.5f * (vat(&rrv, k, j, fu) + vat(&rrv, k, j, fm));
                    float north_v = 0.5f * (vat(&rrv, k, jn, fu) + vat(&rrv, k, jn, fm));
                    float fy_s = scalar_y_flux(&u, south_v, fu, j, k);
                    float fy_n = scalar_y_flux(&u, north_v, fu, j + 1, k);
                    float advx = (-(fx_e - fx_w)) * rdx;
                    float advy = (-(fy_n - fy_s)) * rdy;
                    float advz = 0.0f;
                    if (nk >= 6) {
                        if (k == 0) {
                            float vv = 0.5f * (vat(&rrw, 1, j, fu) + vat(&rrw, 1, j, fm));
                            float top = vertical_mass_flux(&u, vv, 2, j, fu, S(a->c1, 2, js, fu + 1),
                                                           S(a->c2, 2, js, fu + 1));
                            advz = (-top) * rdz;
                        } else if (k == nk - 1) {
                            float vv = 0.5f * (vat(&rrw, nk - 1, j, fu) + vat(&rrw, nk - 1, j, fm));
                            float bottom = vertical_mass_flux(&u, vv, nk, j, fu, S(a->c1, nk, js, fu + 1),
                                                              S(a->c2, nk, js, fu + 1));
                            advz = bottom * rdz;
                        } else {
                            const int lo = k + 1, hi = k + 2;
                            float vlo = 0.5f * (vat(&rrw, lo - 1, j, fu) + vat(&rrw, lo - 1, j, fm));
                            float vhi = 0.5f * (vat(&rrw, hi - 1, j, fu) + vat(&rrw, hi - 1, j, fm));
                            float flo = vertical_mass_flux(&u, vlo, lo, j, fu, S(a->c1, lo, js, fu + 1),
                                                           S(a->c2, lo, js, fu + 1));
                            float fhi = vertical_mass_flux(&u, vhi, hi, j, fu, S(a->c1, hi, js, fu + 1),
                                                           S(a->c2, hi, js, fu + 1));
                            advz = (-(fhi - flo)) * rdz;
                        }
                    }
                    float corr = vat(&u, k, j, fu) * (0.5f * (vat(&dv, k, j, fu) + vat(&dv, k, j, fm)));
                    float total = (((advx + advy) + advz) + corr) * S(a->rr0, ks, js, fu + 1);
                    U(a->uten, ks, js, f) = total;
                }
            }
            for (int g = 0; g < nj + 1; ++g) {
                const int gv = g % nj;
                const int gm = pmod(gv - 1, nj), gp = (gv + 1) % nj;
                for (int i = 0; i < ni; ++i) {
                    const int is = i + 1, ip = (i + 1) % ni;
                    float west_v = 0.5f * (vat(&rru, k, gv, i) + vat(&rru, k, gm, i));
                    float east_v = 0.5f * (vat(&rru, k, gv, ip) + vat(&rru, k, gm, ip));
                    float fx_w = scalar_x_flux(&v, west_v, i, gv, k);
                    float fx_e = scalar_x_flux(&v, east_v, i + 1, gv, k);
                    float south_v = 0.5f * (vat(&rrv, k, gm, i) + vat(&rrv, k, gv, i));
                    float north_v = 0.5f * (vat(&rrv, k, gv, i) + vat(&rrv, k, gp, i));
                    float fy_s = centered_y_flux(&v, south_v, i, gv - 1, k);
                    float fy_n = centered_y_flux(&v, north_v, i, gv, k);
                    float advx = (-(fx_e - fx_w)) * rdx;
                    float advy = (-(fy_n - fy_s)) * rdy;
                    float advz = 0.0f;
                    if (nk >= 6) {
                        if (k == 0) {
                            float vv = 0.5f * (vat(&rrw, 1, gv, i) + vat(&rrw, 1, gm, i));
                            advz = (-vertical_mass_flux(&v, vv, 2, gv, i, S(a->c1, 2, gv + 1, is),
                                                        S(a->c2, 2, gv + 1, is))) * rdz;
                        } else if (k == nk - 1) {
                            float vv = 0.5f * (vat(&rrw, nk - 1, gv, i) + vat(&rrw, nk - 1, gm, i));
                            advz = vertical_mass_flux(&v, vv, nk, gv, i, S(a->c1, nk, gv + 1, is),
                                                      S(a->c2, nk, gv + 1, is)) * rdz;
                        } else {
                            const int lo = k + 1, hi = k + 2;
                            float vlo = 0.5f * (vat(&rrw, lo - 1, gv, i) + vat(&rrw, lo - 1, gm, i));
                            float vhi = 0.5f * (vat(&rrw, hi - 1, gv, i) + vat(&rrw, hi - 1, gm, i));
                            float flo = vertical_mass_flux(&v, vlo, lo, gv, i, S(a->c1, lo, gv + 1, is),
                                                           S(a->c2, lo, gv + 1, is));
                            float fhi = vertical_mass_flux(&v, vhi, hi, gv, i, S(a->c1, hi, gv + 1, is),
                                                           S(a->c2, hi, gv + 1, is));
                            advz = (-(fhi - flo)) * rdz;
                        }
                    }
                    float corr = vat(&v, k, gv, i) * (0.5f * (vat(&dv, k, gv, i) + vat(&dv, k, gm, i)));
                    V(a->vten, ks, g, is) = (((advx + advy) + advz) + corr) * S(a->rr0, ks, gv + 1, is);
                }
            }
        }
#pragma omp parallel for schedule(static)
        for (int q = 1; q < nk; ++q) {
            const int qs = q + 1;
            for (int j = 0; j < nj; ++j) {
                const int js = j + 1;
                for (int i = 0; i < ni; ++i) {
                    const int is = i + 1;
                    const float c2 = S(a->c2, qs, js, is);
                    const float c1 = 1.0f - c2;
                    const int i1 = (i + 1) % ni, j1 = (j + 1) % nj;
                    float ux_w = c2 * vat(&rru, q, j, i) + c1 * vat(&rru, q - 1, j, i);
                    float ux_e = c2 * vat(&rru, q, j, i1) + c1 * vat(&rru, q - 1, j, i1);
                    float vy_s = c2 * vat(&rrv, q, j, i) + c1 * vat(&rrv, q - 1, j, i);
                    float vy_n = c2 * vat(&rrv, q, j1, i) + c1 * vat(&rrv, q - 1, j1, i);
                    float fx_w = scalar_x_flux(&w, ux_w, i, j, q);
                    float fx_e = scalar_x_flux(&w, ux_e, i + 1, j, q);
                    float fy_s = scalar_y_flux(&w, vy_s, i, j, q);
                    float fy_n = scalar_y_flux(&w, vy_n, i, j + 1, q);
                    float advx = (-(fx_e - fx_w)) * rdx;
                    float advy = (-(fy_n - fy_s)) * rdy;
                    float vlo = 0.5f * (vat(&rrw, q - 1, j, i) + vat(&rrw, q, j, i));
                    float vhi = 0.5f * (vat(&rrw, q, j, i) + vat(&rrw, q + 1, j, i));
                    float flo = vertical_w_flux(&w, vlo, q, j, i);
                    float fhi = vertical_w_flux(&w, vhi, q + 1, j, i);
                    float advz = (-(fhi - flo)) * rdz;
                    float corr = vat(&w, q, j, i) * (c2 * vat(&dv, q, j, i) + c1 * vat(&dv, q - 1, j, i));
                    W(a->wten, qs, j, i) = (((advx + advy) + advz) + corr) * S(a->rrf0, qs, js, is);
                }
            }
        }
    }
    if (buoyancy) {
        for (int q = 1; q < nk; ++q) {
            const int qs = q + 1;
            for (int j = 0; j < nj; ++j)
                for (int i = 0; i < ni; ++i) {
                    const int js = j + 1, is = i + 1;
                    float lower = GRAV * (S(a->th3d, q, js, is) * S(a->rth0, q, js, is));
                    float upper = GRAV * (S(a->th3d, q + 1, js, is) * S(a->rth0, q + 1, js, is));
                    float b = S(a->c1, qs, js, is) * lower + S(a->c2, qs, js, is) * upper;
                    W(a->wten, qs, j, i) = W(a->wten, qs, j, i) + b;
                }
        }
    }
}

void oracle_traj_theta(const A *a, int ni, int nj, int nk, float rdx, float rdy, float rdz,
                       float dttmp, int enabled, int include_base_theta) {
    zero(a->sadv, scalar_words(ni, nj, nk));
    for (int k = 1; k <= nk; ++k)
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                float base = include_base_theta ? (S(a->th0, k, j, i) - TH0R) : 0.0f;
                S(a->sadv, k, j, i) = base + S(a->th3d, k, j, i);
            }
    oracle_fill_periodic_scalar(a->sadv, ni, nj, nk);
    const size_t ssz = (size_t)(nj + 2) * (ni + 2), ssy = (size_t)(ni + 2);
    const size_t usz = (size_t)(nj + 2) * (ni + 1), usy = (size_t)(ni + 1);
    const size_t vsz = (size_t)(nj + 1) * (ni + 2), vsy = (size_t)(ni + 2);
    const size_t wsz = (size_t)nj * ni, wsy = (size_t)ni;
    const view3 th = {a->sadv, nk, nj, ni, ssz, ssy, 1, 1, 1};
    const view3 rru = {a->rru, nk, nj, ni, usz, usy, 1, 1, 0};
    const view3 rrv = {a->rrv, nk, nj, ni, vsz, vsy, 1, 0, 1};
    const view3 rrw = {a->rrw, nk + 1, nj, ni, wsz, wsy, 1, 0, 0};
    const view3 dv = {a->divx, nk, nj, ni, ssz, ssy, 1, 1, 1};
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nk; ++k) {
        const int ks = k + 1;
        for (int j = 0; j < nj; ++j) {
            const int js = j + 1;
            for (int i = 0; i < ni; ++i) {
                const int is = i + 1;
                float tendency = 0.0f;
                if (enabled) {
                    float fx_w = scalar_x_flux(&th, vat(&rru, k, j, i), i, j, k);
                    float fx_e = scalar_x_flux(&th, vat(&rru, k, j, (i + 1) % ni), i + 1, j, k);
                    float fy_s = scalar_y_flux(&th, vat(&rrv, k, j, i), i, j, k);
                    float fy_n = scalar_y_flux(&th, vat(&rrv, k, (j + 1) % nj, i), i, j + 1, k);
                    float advx = (-(fx_e - fx_w)) * rdx;
                    float advy = (-(fy_n - fy_s)) * rdy;
                    float advz;
                    if (k == 0) {
                        advz = (-vertical_mass_flux(&th, vat(&rrw, 1, j, i), 2, j, i, S(a->c1, 2, js, is),
                                                    S(a->c2, 2, js, is))) * rdz;
                    } else if (k == nk - 1) {
                        advz = vertical_mass_flux(&th, vat(&rrw, nk - 1, j, i), nk, j, i,
                                                  S(a->c1, nk, js, is), S(a->c2, nk, js, is)) * rdz;
                    } else {
                        const int lo = k + 1, hi = k + 2;
                        float flo = vertical_mass_flux(&th, vat(&rrw, lo - 1, j, i), lo, j, i,
                                                       S(a->c1, lo, js, is), S(a->c2, lo, js, is));
                        float fhi = vertical_mass_flux(&th, vat(&rrw, hi - 1, j, i), hi, j, i,
                                                       S(a->c1, hi, js, is), S(a->c2, hi, js, is));
                        advz = (-(fhi - flo)) * rdz;
                    }
                    float corr = vat(&th, k, j, i) * vat(&dv, k, j, i);
                    tendency = (((advx + advy) + advz) + corr) * S(a->rr0, ks, js, is);
                }
                S(a->thten, ks, js, is) = tendency;
                float updated = S(a->tha, ks, js, is) + dttmp * tendency;
                if (fabsf(updated) < SMEPS) updated = 0.0f;
                S(a->th3d, ks, js, is) = updated;
            }
        }
    }
}

void oracle_traj_post_step(const A *a, int ni, int nj, int nk, int post_step_ppx, int promotion) {
    oracle_fill_periodic_scalar(a->pp3d, ni, nj, nk);
    oracle_fill_periodic_scalar(a->th3d, ni, nj, nk);
    if (post_step_ppx) {
        for (int k = 1; k <= nk; ++k)
            for (int j = 1; j <= nj; ++j)
                for (int i = 1; i <= ni; ++i) S(a->ppx, k, j, i) = S(a->pp3d, k, j, i) + S(a->ppx, k, j, i);
        oracle_fill_periodic_scalar(a->ppx, ni, nj, nk);
    }
    if (promotion) {
        memcpy(a->ua, a->u3d, u_words(ni, nj, nk) * sizeof(float));
        memcpy(a->va, a->v3d, v_words(ni, nj, nk) * sizeof(float));
        memcpy(a->wa, a->w3d, w_words(ni, nj, nk) * sizeof(float));
        memcpy(a->ppi, a->pp3d, scalar_words(ni, nj, nk) * sizeof(float));
        memcpy(a->tha, a->th3d, scalar_words(ni, nj, nk) * sizeof(float));
    }
}

/* One RK stage of the dry trajectory (the body of the nrk loop of
 * cpu_psolver3_trajectory_inplace, :830-863).  Returns nloop or -1. */
int oracle_traj_stage(const A *a, int ni, int nj, int nk, float dt, int nsound, int nrk,
                      float dx, float dy, float dz, unsigned ablations) {
    const float rdx = 1.0f / dx, rdy = 1.0f / dy, rdz = 1.0f / dz;
    oracle_traj_prepare(a, ni, nj, nk);
    oracle_traj_instant_mass_flux(a, ni, nj, nk);
    oracle_traj_divergence(a, ni, nj, nk, rdx, rdy, rdz);
    oracle_traj_momentum(a, ni, nj, nk, rdx, rdy, rdz, !(ablations & GM1B_ABLATE_MOMENTUM_ADVECTION),
                         !(ablations & GM1B_ABLATE_BUOYANCY));
    int nloop = oracle_sound3_periodic_stage(a, ni, nj, nk, dt, nsound, nrk, rdx, rdy, rdz,
                                             0x1.f6d99ap+9f /* 1005.7 */, 0x1.333334p-1f /* 0.6 */,
                                             0x1.99999ap-4f /* 0.1 */, SMEPS);
    if (nloop < 0) return -1;
    oracle_traj_scale_averages(a, ni, nj, nk);
    oracle_traj_divergence(a, ni, nj, nk, rdx, rdy, rdz);
    float dttmp = oracle_rk_stage_dt(dt, nrk);
    oracle_traj_theta(a, ni, nj, nk, rdx, rdy, rdz, dttmp, !(ablations & GM1B_ABLATE_SCALAR_ADVECTION),
                      !(ablations & GM1B_ABLATE_BASE_THETA_ADVECTION));
    if (nrk < 3) oracle_fill_periodic_scalar(a->th3d, ni, nj, nk);
    return nloop;
}

int oracle_traj_steps(const A *a, int ni, int nj, int nk, int steps, float dt, int nsound,
                      float dx, float dy, float dz, unsigned ablations) {
    for (int s = 0; s < steps; ++s) {
        for (int nrk = 1; nrk <= 3; ++nrk)
            if (oracle_traj_stage(a, ni, nj, nk, dt, nsound, nrk, dx, dy, dz, ablations) < 0) return -1;
        oracle_traj_post_step(a, ni, nj, nk, !(ablations & GM1B_ABLATE_POST_STEP_PPX),
                              !(ablations & GM1B_ABLATE_CARRIER_PROMOTION));
    }
    return 0;
}
