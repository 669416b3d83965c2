/* Oracle (test infrastructure only): CPU restatement of the terrain/open
 * fifth-order momentum advection of the padded lane,
 * cpu_terrain_open_momentum_advection5_inplace
 * (src/cm1core/cuda_momentum_advection5.py:753-1068): the mass fluxes rru,
 * rrv, rrw (with the terrain term) on every face, the divergence divx, and
 * the advu / advv / advw increments added into uten / vten / wten, with
 * CM1's lateral families (periodic sides wrap, open sides substitute the
 * inner face flux for inflow and apply the inflow edits).
 *
 * Padded arrays (ng = 3): u-shaped (nk+2, nj+6, ni+7), v-shaped
 * (nk+2, nj+7, ni+6), w-shaped (nk+3, nj+6, ni+6); uh (ni+6), vh (nj+6);
 * metrics rho0_3d (nk, nj, ni), rf0/rrf0/c2 (nk+1, nj, ni), gz/dzdx/dzdy
 * (nj, ni), gzu/rgzu (nj, ni+1), gzv/rgzv (nj+1, ni); divx (nk, nj, ni).
 * sides = (wbc, ebc, sbc, nbc), 1 periodic, 2 open, 3/4 walls.
 * Binary32 one operation at a time.
 */
#include <math.h>
#include <stdint.h>
#include "real.h"

#define NG 3

typedef struct {
  float *u3d, *uten, *rru, *v3d, *vten, *rrv, *w3d, *wten, *rrw;
  const float *uh, *vh;
  const float *rho0_3d, *rf0, *rrf0, *c2, *gz, *gzu, *gzv, *rgzu, *rgzv, *dzdx, *dzdy;
  float* divx;
} mom_arrays;

typedef struct {
  int ni, nj, nk;
  int side[4];
  const mom_arrays* a;
  /* vertical column: 0 uniform; 1 terrain branch on a stretched column
   * (sigma/sigmaf/rds/rdsf, ztop, padded base density); 2 flat column
   * (rdz*mh / rdz*mf, the column's base state) -
   * cuda_gm1_child_stretched_momentum.py:56-330 */
  int vmode;
  const float *rho0p, *sigma, *sigmaf, *rds, *rdsf, *mh, *mf, *rr0;
  float ztop, rdzm;
} mom_ctx;

#define UX(c) ((c)->ni + 1 + 2 * NG)
#define UY(c) ((c)->nj + 2 * NG)
#define VX(c) ((c)->ni + 2 * NG)
#define VY(c) ((c)->nj + 1 + 2 * NG)
#define U_(c, p, k, y, x) (p)[(((int64_t)(k)) * UY(c) + (y)) * UX(c) + (x)]
#define V_(c, p, k, y, x) (p)[(((int64_t)(k)) * VY(c) + (y)) * VX(c) + (x)]
#define W_(c, p, k, y, x) (p)[(((int64_t)(k)) * UY(c) + (y)) * VX(c) + (x)]
#define C3(c, p, k, j, i) (p)[(((int64_t)(k)) * (c)->nj + (j)) * (c)->ni + (i)]

static int clampi(int x, int n) { return x < 0 ? 0 : (x >= n ? n - 1 : x); }
static int per(const mom_ctx* c, int s) { return c->side[s] == 1; }
static int opn(const mom_ctx* c, int s) { return c->side[s] == 2; }
static int cx(const mom_ctx* c, int i) {
  if (per(c, 0) && i < 0) return i + c->ni;
  if (per(c, 1) && i >= c->ni) return i - c->ni;
  return i;
}
static int fx(const mom_ctx* c, int i) {
  if (per(c, 0) && i < 0) return i + c->ni;
  if (per(c, 1) && i > c->ni) return i - c->ni;
  return i;
}
static int cy(const mom_ctx* c, int j) {
  if (per(c, 2) && j < 0) return j + c->nj;
  if (per(c, 3) && j >= c->nj) return j - c->nj;
  return j;
}
static int fy(const mom_ctx* c, int j) {
  if (per(c, 2) && j < 0) return j + c->nj;
  if (per(c, 3) && j > c->nj) return j - c->nj;
  return j;
}
/* face-level metric at Fortran face kface (1-based), clamped column */
static float met(const mom_ctx* c, const float* p, int kface, int j, int i) {
  return p[((int64_t)(kface - 1) * c->nj + clampi(j, c->nj)) * c->ni + clampi(i, c->ni)];
}

static float flx3m(float a, float b, float d) {
  float r = (-1.0f / 6.0f) * a;
  r = r + (5.0f / 6.0f) * b;
  return r + (2.0f / 6.0f) * d;
}
static float flx5m(float a, float b, float d, float e, float f) {
  float r = (2.0f / 60.0f) * a;
  r = r + (-13.0f / 60.0f) * b;
  r = r + (47.0f / 60.0f) * d;
  r = r + (27.0f / 60.0f) * e;
  return r + (-3.0f / 60.0f) * f;
}

static float u_fx(const mom_ctx* c, int k, int j, int face) {
  const mom_arrays* a = c->a;
  const int y = j + NG, x = face + NG;
  const float mass = 0.5f * (U_(c, a->rru, k, y, fx(c, face) + NG) + U_(c, a->rru, k, y, fx(c, face + 1) + NG));
  const float* u = a->u3d;
  const float r = mass >= 0.0f
                      ? flx5m(U_(c, u, k, y, x - 2), U_(c, u, k, y, x - 1), U_(c, u, k, y, x), U_(c, u, k, y, x + 1), U_(c, u, k, y, x + 2))
                      : flx5m(U_(c, u, k, y, x + 3), U_(c, u, k, y, x + 2), U_(c, u, k, y, x + 1), U_(c, u, k, y, x), U_(c, u, k, y, x - 1));
  return mass * r;
}

static float u_fy_base(const mom_ctx* c, int k, int face, int i_face) {
  const mom_arrays* a = c->a;
  const int y = face + NG, x = i_face + NG;
  const float mass = 0.5f * (V_(c, a->rrv, k, y, cx(c, i_face) + NG) + V_(c, a->rrv, k, y, cx(c, i_face - 1) + NG));
  const float* u = a->u3d;
  const float r = mass >= 0.0f
                      ? flx5m(U_(c, u, k, y - 3, x), U_(c, u, k, y - 2, x), U_(c, u, k, y - 1, x), U_(c, u, k, y, x), U_(c, u, k, y + 1, x))
                      : flx5m(U_(c, u, k, y + 2, x), U_(c, u, k, y + 1, x), U_(c, u, k, y, x), U_(c, u, k, y - 1, x), U_(c, u, k, y - 2, x));
  return mass * r;
}

static float u_fy(const mom_ctx* c, int k, int face, int i_face) {
  const mom_arrays* a = c->a;
  const int y = face + NG;
  const float mt = V_(c, a->rrv, k, y, cx(c, i_face) + NG) + V_(c, a->rrv, k, y, cx(c, i_face - 1) + NG);
  if (face == 0 && opn(c, 2) && mt >= 0.0f) return u_fy_base(c, k, 1, i_face);
  if (face == c->nj && opn(c, 3) && mt <= 0.0f) return u_fy_base(c, k, c->nj - 1, i_face);
  return u_fy_base(c, k, face, i_face);
}

static float v_fx_base(const mom_ctx* c, int k, int j_face, int face) {
  const mom_arrays* a = c->a;
  const int y = j_face + NG, x = face + NG;
  const float mass = 0.5f * (U_(c, a->rru, k, cy(c, j_face) + NG, x) + U_(c, a->rru, k, cy(c, j_face - 1) + NG, x));
  const float* v = a->v3d;
  const float r = mass >= 0.0f
                      ? flx5m(V_(c, v, k, y, x - 3), V_(c, v, k, y, x - 2), V_(c, v, k, y, x - 1), V_(c, v, k, y, x), V_(c, v, k, y, x + 1))
                      : flx5m(V_(c, v, k, y, x + 2), V_(c, v, k, y, x + 1), V_(c, v, k, y, x), V_(c, v, k, y, x - 1), V_(c, v, k, y, x - 2));
  return mass * r;
}

static float v_fx(const mom_ctx* c, int k, int j_face, int face) {
  const mom_arrays* a = c->a;
  const int x = face + NG;
  const float mt = U_(c, a->rru, k, cy(c, j_face) + NG, x) + U_(c, a->rru, k, cy(c, j_face - 1) + NG, x);
  if (face == 0 && opn(c, 0) && mt >= 0.0f) return v_fx_base(c, k, j_face, 1);
  if (face == c->ni && opn(c, 1) && mt <= 0.0f) return v_fx_base(c, k, j_face, c->ni - 1);
  return v_fx_base(c, k, j_face, face);
}

static float v_fy(const mom_ctx* c, int k, int face, int i) {
  const mom_arrays* a = c->a;
  const int y = face + NG, x = i + NG;
  const float mass = 0.5f * (V_(c, a->rrv, k, fy(c, face) + NG, x) + V_(c, a->rrv, k, fy(c, face + 1) + NG, x));
  const float* v = a->v3d;
  const float r = mass >= 0.0f
                      ? flx5m(V_(c, v, k, y - 2, x), V_(c, v, k, y - 1, x), V_(c, v, k, y, x), V_(c, v, k, y + 1, x), V_(c, v, k, y + 2, x))
                      : flx5m(V_(c, v, k, y + 3, x), V_(c, v, k, y + 2, x), V_(c, v, k, y + 1, x), V_(c, v, k, y, x), V_(c, v, k, y - 1, x));
  return mass * r;
}

/* vertical flux of u (is_u) or v at Fortran face kface of column (j, i) */
static float uv_z(const mom_ctx* c, int is_u, int kface, int j, int i) {
  const mom_arrays* a = c->a;
  const int y = j + NG, x = i + NG, nk = c->nk;
  float mass, c2;
  if (is_u) {
    mass = 0.5f * (W_(c, a->rrw, kface, y, cx(c, i) + NG) + W_(c, a->rrw, kface, y, cx(c, i - 1) + NG));
    c2 = 0.5f * (met(c, a->c2, kface, j, i - 1) + met(c, a->c2, kface, j, i));
  } else {
    mass = 0.5f * (W_(c, a->rrw, kface, cy(c, j) + NG, x) + W_(c, a->rrw, kface, cy(c, j - 1) + NG, x));
    c2 = 0.5f * (met(c, a->c2, kface, j - 1, i) + met(c, a->c2, kface, j, i));
  }
  const float c1 = 1.0f - c2;
#define Q(l) (is_u ? U_(c, a->u3d, (l), y, x) : V_(c, a->v3d, (l), y, x))
  float r;
  if (kface == 2) {
    r = mass >= 0.0f ? c1 * Q(1) + c2 * Q(2) : flx3m(Q(3), Q(2), Q(1));
  } else if (kface == nk) {
    r = mass >= 0.0f ? flx3m(Q(nk - 2), Q(nk - 1), Q(nk)) : c1 * Q(nk - 1) + c2 * Q(nk);
  } else if (kface == 3) {
    r = mass >= 0.0f ? flx3m(Q(1), Q(2), Q(3)) : flx5m(Q(5), Q(4), Q(3), Q(2), Q(1));
  } else if (kface == nk - 1) {
    r = mass >= 0.0f ? flx5m(Q(kface - 3), Q(kface - 2), Q(kface - 1), Q(kface), Q(kface + 1))
                     : flx3m(Q(kface + 1), Q(kface), Q(kface - 1));
  } else if (mass >= 0.0f) {
    r = flx5m(Q(kface - 3), Q(kface - 2), Q(kface - 1), Q(kface), Q(kface + 1));
  } else {
    r = flx5m(Q(kface + 2), Q(kface + 1), Q(kface), Q(kface - 1), Q(kface - 2));
  }
#undef Q
  return mass * r;
}

static float w_fx_base(const mom_ctx* c, int kface, int j, int face) {
  const mom_arrays* a = c->a;
  const int y = j + NG, x = face + NG;
  const float c2 = 0.5f * (met(c, a->c2, kface, j, face - 1) + met(c, a->c2, kface, j, face)), c1 = 1.0f - c2;
  const float mass = c2 * U_(c, a->rru, kface, y, x) + c1 * U_(c, a->rru, kface - 1, y, x);
  const float* w = a->w3d;
  const float r = mass >= 0.0f
                      ? flx5m(W_(c, w, kface, y, x - 3), W_(c, w, kface, y, x - 2), W_(c, w, kface, y, x - 1), W_(c, w, kface, y, x), W_(c, w, kface, y, x + 1))
                      : flx5m(W_(c, w, kface, y, x + 2), W_(c, w, kface, y, x + 1), W_(c, w, kface, y, x), W_(c, w, kface, y, x - 1), W_(c, w, kface, y, x - 2));
  return mass * r;
}

static float w_fx(const mom_ctx* c, int kface, int j, int face) {
  const mom_arrays* a = c->a;
  const int y = j + NG, x = face + NG;
  const float c2 = 0.5f * (met(c, a->c2, kface, j, face - 1) + met(c, a->c2, kface, j, face)), c1 = 1.0f - c2;
  const float mass = c2 * U_(c, a->rru, kface, y, x) + c1 * U_(c, a->rru, kface - 1, y, x);
  if (face == 0 && opn(c, 0) && mass >= 0.0f) return w_fx_base(c, kface, j, 1);
  if (face == c->ni && opn(c, 1) && mass <= 0.0f) return w_fx_base(c, kface, j, c->ni - 1);
  return w_fx_base(c, kface, j, face);
}

static float w_fy_base(const mom_ctx* c, int kface, int face, int i) {
  const mom_arrays* a = c->a;
  const int y = face + NG, x = i + NG;
  const float c2 = 0.5f * (met(c, a->c2, kface, face - 1, i) + met(c, a->c2, kface, face, i)), c1 = 1.0f - c2;
  const float mass = c2 * V_(c, a->rrv, kface, y, x) + c1 * V_(c, a->rrv, kface - 1, y, x);
  const float* w = a->w3d;
  const float r = mass >= 0.0f
                      ? flx5m(W_(c, w, kface, y - 3, x), W_(c, w, kface, y - 2, x), W_(c, w, kface, y - 1, x), W_(c, w, kface, y, x), W_(c, w, kface, y + 1, x))
                      : flx5m(W_(c, w, kface, y + 2, x), W_(c, w, kface, y + 1, x), W_(c, w, kface, y, x), W_(c, w, kface, y - 1, x), W_(c, w, kface, y - 2, x));
  return mass * r;
}

static float w_fy(const mom_ctx* c, int kface, int face, int i) {
  const mom_arrays* a = c->a;
  const int y = face + NG, x = i + NG;
  const float c2 = 0.5f * (met(c, a->c2, kface, face - 1, i) + met(c, a->c2, kface, face, i)), c1 = 1.0f - c2;
  const float mass = c2 * V_(c, a->rrv, kface, y, x) + c1 * V_(c, a->rrv, kface - 1, y, x);
  if (face == 0 && opn(c, 2) && mass >= 0.0f) return w_fy_base(c, kface, 1, i);
  if (face == c->nj && opn(c, 3) && mass <= 0.0f) return w_fy_base(c, kface, c->nj - 1, i);
  return w_fy_base(c, kface, face, i);
}

static float w_z(const mom_ctx* c, int k, int j, int i) {
  const mom_arrays* a = c->a;
  const int y = j + NG, x = i + NG, nk = c->nk;
  const float mass = 0.5f * (W_(c, a->rrw, k, y, x) + W_(c, a->rrw, k + 1, y, x));
#define Q(l) W_(c, a->w3d, (l), y, x)
  float r;
  if (k == 1) {
    r = mass >= 0.0f ? 0.5f * (Q(1) + Q(2)) : flx3m(Q(3), Q(2), Q(1));
  } else if (k == 2) {
    r = mass >= 0.0f ? flx3m(Q(1), Q(2), Q(3)) : flx5m(Q(5), Q(4), Q(3), Q(2), Q(1));
  } else if (k == nk - 1) {
    r = mass >= 0.0f ? flx5m(Q(k - 2), Q(k - 1), Q(k), Q(k + 1), Q(k + 2)) : flx3m(Q(k + 2), Q(k + 1), Q(k));
  } else if (k == nk) {
    r = mass >= 0.0f ? flx3m(Q(k - 1), Q(k), Q(k + 1)) : 0.5f * (Q(k) + Q(k + 1));
  } else if (mass >= 0.0f) {
    r = flx5m(Q(k - 2), Q(k - 1), Q(k), Q(k + 1), Q(k + 2));
  } else {
    r = flx5m(Q(k + 3), Q(k + 2), Q(k + 1), Q(k), Q(k - 1));
  }
#undef Q
  return mass * r;
}

#define P_(c, p, k, y, x) (p)[(((int64_t)(k)) * UY(c) + (y)) * VX(c) + (x)]

static float zmass(const mom_ctx* c, float x, int k, float rdz) {
  if (c->vmode == 2) return (x * c->rdzm) * c->mh[k];
  return x * (c->vmode == 1 ? c->rdsf[k] : rdz);
}
static float zface(const mom_ctx* c, float x, int kf, float rdz) {
  if (c->vmode == 2) return (x * c->rdzm) * c->mf[kf];
  return x * (c->vmode == 1 ? c->rds[kf] : rdz);
}
static float bcorr(const mom_ctx* c, float q, float cr, float r, float h) {
  return c->vmode == 2 ? ((q * cr) * r) * h : q * (cr * (r * h));
}

/* phase bit 1: mass fluxes and divx; bit 2: advu/advv/advw from them */
static int mom_phase(const mom_ctx* c, float dx, float dy, float dz, int phase) {
  const int ni = c->ni, nj = c->nj, nk = c->nk;
  const mom_arrays* a = c->a;
  const float half = 0.5f;
  if (phase & 1) {
  /* horizontal mass fluxes on every face */
  for (int k0 = 0; k0 < nk; ++k0) {
    const int k = k0 + 1;
    for (int j = 0; j < nj; ++j) {
      const int y = j + NG;
      for (int face = 0; face <= ni; ++face) {
        if (c->vmode == 2) {
          U_(c, a->rru, k, y, face + NG) = P_(c, c->rho0p, k, NG, NG) * U_(c, a->u3d, k, y, face + NG);
          continue;
        }
        const int l = face - 1 < 0 ? 0 : face - 1, r = face < ni - 1 ? face : ni - 1;
        const float density = c->vmode == 1 ? P_(c, c->rho0p, k, y, face + NG - 1) + P_(c, c->rho0p, k, y, face + NG)
                                            : C3(c, a->rho0_3d, k0, j, l) + C3(c, a->rho0_3d, k0, j, r);
        U_(c, a->rru, k, y, face + NG) = (half * density) * (U_(c, a->u3d, k, y, face + NG) * a->rgzu[(int64_t)j * (ni + 1) + face]);
      }
    }
    for (int face = 0; face <= nj; ++face) {
      const int s = face - 1 < 0 ? 0 : face - 1, n = face < nj - 1 ? face : nj - 1;
      const int y = face + NG;
      for (int i = 0; i < ni; ++i) {
        if (c->vmode == 2) {
          V_(c, a->rrv, k, y, i + NG) = P_(c, c->rho0p, k, NG, NG) * V_(c, a->v3d, k, y, i + NG);
          continue;
        }
        const float density = c->vmode == 1 ? P_(c, c->rho0p, k, y - 1, i + NG) + P_(c, c->rho0p, k, y, i + NG)
                                            : C3(c, a->rho0_3d, k0, s, i) + C3(c, a->rho0_3d, k0, n, i);
        V_(c, a->rrv, k, y, i + NG) = (half * density) * (V_(c, a->v3d, k, y, i + NG) * a->rgzv[(int64_t)face * ni + i]);
      }
    }
  }
  /* vertical mass flux with the terrain term */
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i < ni; ++i) {
      W_(c, a->rrw, 1, j + NG, i + NG) = 0.0f;
      W_(c, a->rrw, nk + 1, j + NG, i + NG) = 0.0f;
    }
  const float zt = c->vmode == 1 ? c->ztop : (float)nk * dz, rzt = 1.0f / zt, rdz0 = 1.0f / dz;
  for (int k = 2; k <= nk; ++k) {
    if (c->vmode == 2) {
      for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i)
          W_(c, a->rrw, k, j + NG, i + NG) = a->rf0[(int64_t)(k - 1) * nj * ni] * W_(c, a->w3d, k, j + NG, i + NG);
      continue;
    }
    const float sigmaf = c->vmode == 1 ? c->sigmaf[k] : (float)(k - 1) * dz;
    const float sigma = c->vmode == 1 ? c->sigma[k - 1] : (float)((double)k - 1.5) * dz;
    float r2 = (sigmaf - sigma) * (c->vmode == 1 ? c->rds[k] : rdz0);
    const float r1 = half * (1.0f - r2);
    r2 = half * r2;
    for (int j = 0; j < nj; ++j) {
      const int y = j + NG;
      for (int i = 0; i < ni; ++i) {
        const int x = i + NG;
        const float ux = r2 * (U_(c, a->rru, k, y, x) + U_(c, a->rru, k, y, x + 1)) +
                         r1 * (U_(c, a->rru, k - 1, y, x) + U_(c, a->rru, k - 1, y, x + 1));
        const float vy = r2 * (V_(c, a->rrv, k, y, x) + V_(c, a->rrv, k, y + 1, x)) +
                         r1 * (V_(c, a->rrv, k - 1, y, x) + V_(c, a->rrv, k - 1, y + 1, x));
        float terrain = ux * a->dzdx[(int64_t)j * ni + i] + vy * a->dzdy[(int64_t)j * ni + i];
        terrain = terrain * (sigmaf - zt);
        terrain = terrain * a->gz[(int64_t)j * ni + i];
        terrain = terrain * rzt;
        W_(c, a->rrw, k, y, x) = a->rf0[((int64_t)(k - 1) * nj + j) * ni + i] * W_(c, a->w3d, k, y, x) + terrain;
      }
    }
  }
  const float rdx = 1.0f / dx, rdy = 1.0f / dy, rdz = 1.0f / dz;
  for (int k0 = 0; k0 < nk; ++k0) {
    const int k = k0 + 1;
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const int y = j + NG, x = i + NG;
        float value = (U_(c, a->rru, k, y, x + 1) - U_(c, a->rru, k, y, x)) * rdx +
                      (V_(c, a->rrv, k, y + 1, x) - V_(c, a->rrv, k, y, x)) * rdy;
        value = value + zmass(c, W_(c, a->rrw, k + 1, y, x) - W_(c, a->rrw, k, y, x), k, rdz);
        C3(c, a->divx, k0, j, i) = fabsf(value) < (c->vmode == 2 ? 1.0e-30f : 1.0e-20f) ? 0.0f : value;
      }
  }
  }
  if (!(phase & 2)) return 0;
  const float rdx = 1.0f / dx, rdy = 1.0f / dy, rdz = 1.0f / dz;
  /* advu */
  const int first_face = per(c, 0) ? 0 : 1, last_face = per(c, 1) ? ni : ni - 1;
  const int first_row = per(c, 2) ? 0 : 1, last_row = per(c, 3) ? nj : nj - 1;
  for (int k0 = 0; k0 < nk; ++k0) {
    const int k = k0 + 1;
    for (int j = 0; j < nj; ++j) {
      const int y = j + NG;
      for (int f = first_face; f <= last_face; ++f) {
        const int x = f + NG, west = cx(c, f - 1), east = cx(c, f);
        const float advx = -(u_fx(c, k, j, f) - u_fx(c, k, j, f - 1)) * rdx;
        float advy = -(u_fy(c, k, j + 1, f) - u_fy(c, k, j, f)) * rdy;
        const float uc = U_(c, a->u3d, k, y, x);
        if (j == 0 && opn(c, 2)) {
          const float mass = V_(c, a->rrv, k, NG, east + NG) + V_(c, a->rrv, k, NG, west + NG);
          if (mass >= 0.0f) {
            const float corr = (V_(c, a->rrv, k, NG + 1, west + NG) - V_(c, a->rrv, k, NG, west + NG)) +
                               (V_(c, a->rrv, k, NG + 1, east + NG) - V_(c, a->rrv, k, NG, east + NG));
            advy = advy - bcorr(c, uc * half, corr, rdy, a->vh[y]);
          }
        } else if (j == nj - 1 && opn(c, 3)) {
          const float mass = V_(c, a->rrv, k, NG + nj, east + NG) + V_(c, a->rrv, k, NG + nj, west + NG);
          if (mass <= 0.0f) {
            const float corr = (V_(c, a->rrv, k, y + 1, west + NG) - V_(c, a->rrv, k, y, west + NG)) +
                               (V_(c, a->rrv, k, y + 1, east + NG) - V_(c, a->rrv, k, y, east + NG));
            advy = advy - bcorr(c, uc * half, corr, rdy, a->vh[y]);
          }
        }
        float advz;
        if (k == 1) advz = zmass(c, -uv_z(c, 1, 2, j, f), k, rdz);
        else if (k == nk) advz = zmass(c, uv_z(c, 1, nk, j, f), k, rdz);
        else advz = zmass(c, -(uv_z(c, 1, k + 1, j, f) - uv_z(c, 1, k, j, f)), k, rdz);
        float total = (advx + advy) + advz;
        total = total + uc * (half * (C3(c, a->divx, k0, j, east) + C3(c, a->divx, k0, j, west)));
        const float scale = c->vmode == 2 ? C3(c, c->rr0, k0, 0, 0)
                                          : a->gzu[(int64_t)j * (ni + 1) + f] /
                                                (half * (C3(c, a->rho0_3d, k0, j, west) + C3(c, a->rho0_3d, k0, j, east)));
        U_(c, a->uten, k, y, x) = U_(c, a->uten, k, y, x) + total * scale;
      }
    }
  }
  /* advv */
  for (int k0 = 0; k0 < nk; ++k0) {
    const int k = k0 + 1;
    for (int g = first_row; g <= last_row; ++g) {
      const int y = g + NG, south = cy(c, g - 1), north = cy(c, g);
      for (int i = 0; i < ni; ++i) {
        const int x = i + NG;
        float advx = -(v_fx(c, k, g, i + 1) - v_fx(c, k, g, i)) * rdx;
        const float advy = -(v_fy(c, k, g, i) - v_fy(c, k, g - 1, i)) * rdy;
        const float vc = V_(c, a->v3d, k, y, x);
        if (i == 0 && opn(c, 0)) {
          const float mass = U_(c, a->rru, k, north + NG, NG) + U_(c, a->rru, k, south + NG, NG);
          if (mass >= 0.0f) {
            const float corr = (U_(c, a->rru, k, south + NG, NG + 1) - U_(c, a->rru, k, south + NG, NG)) +
                               (U_(c, a->rru, k, north + NG, NG + 1) - U_(c, a->rru, k, north + NG, NG));
            advx = advx - bcorr(c, vc * half, corr, rdx, a->uh[NG]);
          }
        } else if (i == ni - 1 && opn(c, 1)) {
          const float mass = U_(c, a->rru, k, north + NG, NG + ni) + U_(c, a->rru, k, south + NG, NG + ni);
          if (mass <= 0.0f) {
            const float corr = (U_(c, a->rru, k, south + NG, x + 1) - U_(c, a->rru, k, south + NG, x)) +
                               (U_(c, a->rru, k, north + NG, x + 1) - U_(c, a->rru, k, north + NG, x));
            advx = advx - bcorr(c, vc * half, corr, rdx, a->uh[x]);
          }
        }
        float advz;
        if (k == 1) advz = zmass(c, -uv_z(c, 0, 2, g, i), k, rdz);
        else if (k == nk) advz = zmass(c, uv_z(c, 0, nk, g, i), k, rdz);
        else advz = zmass(c, -(uv_z(c, 0, k + 1, g, i) - uv_z(c, 0, k, g, i)), k, rdz);
        float total = (advx + advy) + advz;
        total = total + vc * (half * (C3(c, a->divx, k0, north, i) + C3(c, a->divx, k0, south, i)));
        const float scale = c->vmode == 2 ? C3(c, c->rr0, k0, 0, 0)
                                          : a->gzv[(int64_t)g * ni + i] /
                                                (half * (C3(c, a->rho0_3d, k0, south, i) + C3(c, a->rho0_3d, k0, north, i)));
        V_(c, a->vten, k, y, x) = V_(c, a->vten, k, y, x) + total * scale;
      }
    }
  }
  /* advw */
  for (int kf = 2; kf <= nk; ++kf)
    for (int j = 0; j < nj; ++j) {
      const int y = j + NG;
      for (int i = 0; i < ni; ++i) {
        const int x = i + NG;
        const float dfx = -(w_fx(c, kf, j, i + 1) - w_fx(c, kf, j, i)), dfy = -(w_fy(c, kf, j + 1, i) - w_fy(c, kf, j, i));
        float advx = c->vmode == 2 ? (dfx * rdx) * a->uh[x] : dfx * (rdx * a->uh[x]);
        float advy = c->vmode == 2 ? (dfy * rdy) * a->vh[y] : dfy * (rdy * a->vh[y]);
        const float c2 = a->c2[((int64_t)(kf - 1) * nj + j) * ni + i], c1 = 1.0f - c2;
        const float wc = W_(c, a->w3d, kf, y, x);
        if (i == 0 && opn(c, 0)) {
          const float mass = c2 * U_(c, a->rru, kf, y, NG) + c1 * U_(c, a->rru, kf - 1, y, NG);
          if (mass >= 0.0f) {
            const float corr = c1 * (U_(c, a->rru, kf - 1, y, NG + 1) - U_(c, a->rru, kf - 1, y, NG)) +
                               c2 * (U_(c, a->rru, kf, y, NG + 1) - U_(c, a->rru, kf, y, NG));
            advx = advx - bcorr(c, wc, corr, rdx, a->uh[x]);
          }
        } else if (i == ni - 1 && opn(c, 1)) {
          const float mass = c2 * U_(c, a->rru, kf, y, NG + ni) + c1 * U_(c, a->rru, kf - 1, y, NG + ni);
          if (mass <= 0.0f) {
            const float corr = c1 * (U_(c, a->rru, kf - 1, y, x + 1) - U_(c, a->rru, kf - 1, y, x)) +
                               c2 * (U_(c, a->rru, kf, y, x + 1) - U_(c, a->rru, kf, y, x));
            advx = advx - bcorr(c, wc, corr, rdx, a->uh[x]);
          }
        }
        if (j == 0 && opn(c, 2)) {
          const float mass = c2 * V_(c, a->rrv, kf, NG, x) + c1 * V_(c, a->rrv, kf - 1, NG, x);
          if (mass >= 0.0f) {
            const float corr = c1 * (V_(c, a->rrv, kf - 1, NG + 1, x) - V_(c, a->rrv, kf - 1, NG, x)) +
                               c2 * (V_(c, a->rrv, kf, NG + 1, x) - V_(c, a->rrv, kf, NG, x));
            advy = advy - bcorr(c, wc, corr, rdy, a->vh[y]);
          }
        } else if (j == nj - 1 && opn(c, 3)) {
          const float mass = c2 * V_(c, a->rrv, kf, NG + nj, x) + c1 * V_(c, a->rrv, kf - 1, NG + nj, x);
          if (mass <= 0.0f) {
            const float corr = c1 * (V_(c, a->rrv, kf - 1, y + 1, x) - V_(c, a->rrv, kf - 1, y, x)) +
                               c2 * (V_(c, a->rrv, kf, y + 1, x) - V_(c, a->rrv, kf, y, x));
            advy = advy - bcorr(c, wc, corr, rdy, a->vh[y]);
          }
        }
        const float advz = zface(c, -(w_z(c, kf, j, i) - w_z(c, kf - 1, j, i)), kf, rdz);
        float total = (advx + advy) + advz;
        total = total + wc * (c2 * C3(c, a->divx, kf - 1, j, i) + c1 * C3(c, a->divx, kf - 2, j, i));
        const float scale = c->vmode == 2 ? a->rrf0[(int64_t)(kf - 1) * nj * ni]
                                          : a->rrf0[((int64_t)(kf - 1) * nj + j) * ni + i] * a->gz[(int64_t)j * ni + i];
        W_(c, a->wten, kf, y, x) = W_(c, a->wten, kf, y, x) + total * scale;
      }
    }
  return 0;
}

int oracle_momentum_advection5_phase(int ni, int nj, int nk, const mom_arrays* a, const int* sides, float dx,
                                     float dy, float dz, int phase) {
  if (ni < 7 || nj < 7 || nk < 8) return -1;
  mom_ctx cc = {ni, nj, nk, {sides[0], sides[1], sides[2], sides[3]}, a, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0.0f, 0.0f};
  return mom_phase(&cc, dx, dy, dz, phase);
}

/* launch_cuda_gm1_child_stretched_momentum5
 * (src/cm1core/cuda_gm1_child_stretched_momentum.py:540-780): flat = 0 the
 * terrain branch (sigma, sigmaf, rds, rdsf, ztop, padded rho0); flat = 1 the
 * flat column (mh, mf, rdz, the column's padded rho0, rf0, rr0, rrf0). */
int oracle_momentum_advection5_column_phase(int ni, int nj, int nk, const mom_arrays* a, const int* sides, float dx,
                                            float dy, int phase, int flat, const float* rho0p, const float* sigma,
                                            const float* sigmaf, const float* rds, const float* rdsf, float ztop,
                                            const float* mh, const float* mf, const float* rr0, float rdz) {
  if (ni < 7 || nj < 7 || nk < 8) return -1;
  mom_ctx cc = {ni, nj, nk, {sides[0], sides[1], sides[2], sides[3]}, a, flat ? 2 : 1, rho0p, sigma, sigmaf, rds,
                rdsf, mh, mf, rr0, ztop, rdz};
  return mom_phase(&cc, dx, dy, 1.0f, phase);
}

int oracle_momentum_advection5(int ni, int nj, int nk, const mom_arrays* a, const int* sides, float dx, float dy,
                               float dz) {
  return oracle_momentum_advection5_phase(ni, nj, nk, a, sides, dx, dy, dz, 3);
}
