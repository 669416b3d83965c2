/* Oracle (test infrastructure only): CPU restatement of the TKE evolution of
 * the terrain lane, cpu_tke_evolution_inplace
 * (src/cm1core/cuda_tke_evolution.py:206-327):
 *
 *   oracle_tke_diffusion   turbt: horizontal TKE flux divergence with the
 *                          terrain correction and the vertically implicit
 *                          diffusion (Thomas), added into tketen (:210-250)
 *   oracle_tke_rk_stage    one RK stage: flux-form fifth-order (WENO5 at
 *                          nrk = 3) advection with the open-side edits, the
 *                          divergence correction and the tendency, from the
 *                          stage-start field cur into nxt (:251-326)
 *
 * Shapes: face fields (nk+1, nj, ni): tke, tkea, tketen, kmh, kmv, rf, mf,
 * c1, c2, rrf0; mass fields (nk, nj, ni): rho, mh, divx; gz, rgz (nj, ni),
 * rgzu (nj, ni+1), rgzv (nj+1, ni); padded rru (nk+2, nj+6, ni+7), rrv
 * (nk+2, nj+7, ni+6), rrw (nk+3, nj+6, ni+6).  Horizontal neighbours beyond
 * the domain take the nearest column (constant extension).  Binary32 one
 * operation at a time, binary64 WENO weights.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include "real.h"

#define NG 3
#define I3(k, j, i, ny, nx) ((((int64_t)(k)) * (ny) + (j)) * (nx) + (i))

static int cl(int x, int n) { return x < 0 ? 0 : (x >= n ? n - 1 : x); }

typedef struct {
  int ni, nj, nk;
  const float *kmh, *kmv, *rho, *rf, *mh, *mf, *gz, *rgz, *rgzu, *rgzv, *c1, *c2, *rrf0, *rru, *rrv, *rrw, *divx;
} tke_grid;

static float CELL(const tke_grid* g, const float* a, int k, int j, int i) {
  return a[I3(k, cl(j, g->nj), cl(i, g->ni), g->nj, g->ni)];
}
static float G2(const tke_grid* g, const float* a, int j, int i) { return a[(int64_t)cl(j, g->nj) * g->ni + cl(i, g->ni)]; }

/* sm(m) = 0.5*(t(m) + t(m+1)) at a clamped column */
static float SM(const tke_grid* g, const float* t, int m, int j, int i) {
  return 0.5f * (CELL(g, t, m, j, i) + CELL(g, t, m + 1, j, i));
}

/* tx at face level f (1..nk-1), row j, u face `face` (0..ni); 0 elsewhere */
static float TX(const tke_grid* g, const float* t, int f, int j, int face, float rdx, float rdz, float dz) {
  if (f <= 0 || f >= g->nk) return 0.0f;
  const int l = face - 1, r = face;
  const float zt = (float)g->nk * dz;
  const float den = G2(g, g->gz, j, r) * CELL(g, g->rf, f, j, r) + G2(g, g->gz, j, l) * CELL(g, g->rf, f, j, l);
  const float kval = CELL(g, g->kmh, f, j, r) + CELL(g, g->kmh, f, j, l);
  float term = (CELL(g, t, f, j, r) * G2(g, g->rgz, j, r) - CELL(g, t, f, j, l) * G2(g, g->rgz, j, l)) * rdx;
  const float up = (zt - ((float)f + 0.5f) * dz) * (SM(g, t, f, j, l) + SM(g, t, f, j, r));
  const float lo = (zt - ((float)f - 0.5f) * dz) * (SM(g, t, f - 1, j, l) + SM(g, t, f - 1, j, r));
  term = term + 0.5f * ((up - lo) * (rdz * ((G2(g, g->rgz, j, r) - G2(g, g->rgz, j, l)) * rdx)));
  return -0.25f * (den * (2.0f * (kval * term)));
}

/* ty at face level f, v face `face` (0..nj), column i */
static float TY(const tke_grid* g, const float* t, int f, int face, int i, float rdy, float rdz, float dz) {
  if (f <= 0 || f >= g->nk) return 0.0f;
  const int s = face - 1, n = face;
  const float zt = (float)g->nk * dz;
  const float den = G2(g, g->gz, n, i) * CELL(g, g->rf, f, n, i) + G2(g, g->gz, s, i) * CELL(g, g->rf, f, s, i);
  const float kval = CELL(g, g->kmh, f, n, i) + CELL(g, g->kmh, f, s, i);
  float term = (CELL(g, t, f, n, i) * G2(g, g->rgz, n, i) - CELL(g, t, f, s, i) * G2(g, g->rgz, s, i)) * rdy;
  const float up = (zt - ((float)f + 0.5f) * dz) * (SM(g, t, f, s, i) + SM(g, t, f, n, i));
  const float lo = (zt - ((float)f - 0.5f) * dz) * (SM(g, t, f - 1, s, i) + SM(g, t, f - 1, n, i));
  term = term + 0.5f * ((up - lo) * (rdz * ((G2(g, g->rgz, n, i) - G2(g, g->rgz, s, i)) * rdy)));
  return -0.25f * (den * (2.0f * (kval * term)));
}

/* sx(m) = 0.5*(tx(m) + tx(m+1)), sy likewise */
static float SX(const tke_grid* g, const float* t, int m, int j, int face, float rdx, float rdz, float dz) {
  return 0.5f * (TX(g, t, m, j, face, rdx, rdz, dz) + TX(g, t, m + 1, j, face, rdx, rdz, dz));
}
static float SY(const tke_grid* g, const float* t, int m, int face, int i, float rdy, float rdz, float dz) {
  return 0.5f * (TY(g, t, m, face, i, rdy, rdz, dz) + TY(g, t, m + 1, face, i, rdy, rdz, dz));
}

int oracle_tke_diffusion(int ni, int nj, int nk, const float* t, const float* kmh, const float* kmv, const float* rho,
                         const float* rf, const float* mh, const float* mf, const float* gz, const float* rgz,
                         const float* rgzu, const float* rgzv, float* tketen, float dx, float dy, float dz, float dt) {
  if (ni < 3 || nj < 3 || nk < 4) return -1;
  tke_grid g = {ni, nj, nk, kmh, kmv, rho, rf, mh, mf, gz, rgz, rgzu, rgzv, 0, 0, 0, 0, 0, 0, 0};
  const float rdx = 1.0f / dx, rdy = 1.0f / dy, rdz = 1.0f / dz;
  const float zt = (float)nk * dz;
  const int n = nk - 1;
  float* cp = malloc(sizeof(float) * n);
  float* dp = malloc(sizeof(float) * n);
  float* sol = malloc(sizeof(float) * n);
  if (!cp || !dp || !sol) return -2;
  const float tema = -1.0f * (dt * (rdz * rdz));
  const float rdt = 1.0f / dt;
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i < ni; ++i) {
      const float gzji = gz[(int64_t)j * ni + i];
      const float ru1 = rgzu[(int64_t)j * (ni + 1) + i + 1], ru0 = rgzu[(int64_t)j * (ni + 1) + i];
      const float rv1 = rgzv[(int64_t)(j + 1) * ni + i], rv0 = rgzv[(int64_t)j * ni + i];
      /* vertically implicit diffusion */
      int f = 1;
      float rrf = mf[I3(f, j, i, nj, ni)] / rf[I3(f, j, i, nj, ni)];
      float r2 = (kmv[I3(f, j, i, nj, ni)] + kmv[I3(f + 1, j, i, nj, ni)]) *
                 (mh[I3(f, j, i, nj, ni)] * (rho[I3(f, j, i, nj, ni)] * rrf));
      float cfc = tema * r2, cfb = 1.0f - cfc, inv = 1.0f / cfb;
      cp[0] = -1.0f * (cfc * inv);
      dp[0] = t[I3(f, j, i, nj, ni)] * inv;
      for (int p = 1; p < n - 1; ++p) {
        f = p + 1;
        rrf = mf[I3(f, j, i, nj, ni)] / rf[I3(f, j, i, nj, ni)];
        const float r1 = (kmv[I3(f - 1, j, i, nj, ni)] + kmv[I3(f, j, i, nj, ni)]) *
                         (mh[I3(f - 1, j, i, nj, ni)] * (rho[I3(f - 1, j, i, nj, ni)] * rrf));
        r2 = (kmv[I3(f, j, i, nj, ni)] + kmv[I3(f + 1, j, i, nj, ni)]) *
             (mh[I3(f, j, i, nj, ni)] * (rho[I3(f, j, i, nj, ni)] * rrf));
        const float cfa = tema * r1;
        cfc = tema * r2;
        cfb = (1.0f - cfa) - cfc;
        inv = 1.0f / (cfa * cp[p - 1] + cfb);
        cp[p] = -1.0f * (cfc * inv);
        dp[p] = (t[I3(f, j, i, nj, ni)] - cfa * dp[p - 1]) * inv;
      }
      {
        const int p = n - 1;
        f = nk - 1;
        rrf = mf[I3(f, j, i, nj, ni)] / rf[I3(f, j, i, nj, ni)];
        const float r1 = (kmv[I3(f - 1, j, i, nj, ni)] + kmv[I3(f, j, i, nj, ni)]) *
                         (mh[I3(f - 1, j, i, nj, ni)] * (rho[I3(f - 1, j, i, nj, ni)] * rrf));
        const float cfa = tema * r1;
        cfb = 1.0f - cfa;
        sol[p] = (t[I3(f, j, i, nj, ni)] - cfa * dp[p - 1]) * (1.0f / (cfa * cp[p - 1] + cfb));
      }
      for (int p = n - 2; p >= 0; --p) sol[p] = cp[p] * sol[p + 1] + dp[p];
      for (int p = 0; p < n; ++p) {
        f = p + 1;
        /* horizontal divergence with the terrain correction */
        float x = -1.0f * ((TX(&g, t, f, j, i + 1, rdx, rdz, dz) * ru1 - TX(&g, t, f, j, i, rdx, rdz, dz) * ru0) *
                           (gzji * rdx));
        float up = (zt - ((float)f + 0.5f) * dz) * (SX(&g, t, f, j, i, rdx, rdz, dz) + SX(&g, t, f, j, i + 1, rdx, rdz, dz));
        float lo = (zt - ((float)f - 0.5f) * dz) *
                   (SX(&g, t, f - 1, j, i, rdx, rdz, dz) + SX(&g, t, f - 1, j, i + 1, rdx, rdz, dz));
        x = x - 0.5f * ((up - lo) * (rdz * ((ru1 - ru0) * (gzji * rdx))));
        float y = -1.0f * ((TY(&g, t, f, j + 1, i, rdy, rdz, dz) * rv1 - TY(&g, t, f, j, i, rdy, rdz, dz) * rv0) *
                           (gzji * rdy));
        up = (zt - ((float)f + 0.5f) * dz) * (SY(&g, t, f, j, i, rdy, rdz, dz) + SY(&g, t, f, j + 1, i, rdy, rdz, dz));
        lo = (zt - ((float)f - 0.5f) * dz) * (SY(&g, t, f - 1, j, i, rdy, rdz, dz) + SY(&g, t, f - 1, j + 1, i, rdy, rdz, dz));
        y = y - 0.5f * ((up - lo) * (rdz * ((rv1 - rv0) * (gzji * rdy))));
        const float hx = (i == 0 || i == ni - 1) ? 0.0f : x;
        const float hy = (j == 0 || j == nj - 1) ? 0.0f : y;
        const int64_t z = I3(f, j, i, nj, ni);
        const float vz = rf[z] * ((sol[p] - t[z]) * rdt);
        tketen[z] = tketen[z] + ((hx + hy) + vz) / rf[z];
      }
    }
  free(cp);
  free(dp);
  free(sol);
  return 0;
}

/* ------------------------------------------------------------- RK stage */

static float flx3o(float a, float b, float c) {
  float r = (-1.0f / 6.0f) * a;
  r = r + (5.0f / 6.0f) * b;
  return r + (2.0f / 6.0f) * c;
}
static float flx5o(float a, float b, float c, float d, float e) {
  float r = (2.0f / 60.0f) * a;
  r = r + (-13.0f / 60.0f) * b;
  r = r + (47.0f / 60.0f) * c;
  r = r + (27.0f / 60.0f) * d;
  return r + (-3.0f / 60.0f) * e;
}
static double dmin(double a, double b) { return a < b ? a : b; }
static float weno5o(float s1, float s2, float s3, float s4, float s5, double eps) {
  const float d1 = (s1 - 2.0f * s2) + s3, e1 = (s1 - 4.0f * s2) + 3.0f * s3;
  const float b1 = (13.0f / 12.0f) * (d1 * d1) + 0.25f * (e1 * e1);
  const float d2 = (s2 - 2.0f * s3) + s4, e2 = s2 - s4;
  const float b2 = (13.0f / 12.0f) * (d2 * d2) + 0.25f * (e2 * e2);
  const float d3 = (s3 - 2.0f * s4) + s5, e3 = (3.0f * s3 - 4.0f * s4) + s5;
  const float b3 = (13.0f / 12.0f) * (d3 * d3) + 0.25f * (e3 * e3);
  const double tau = fabs((double)b1 - (double)b3);
  const double q1 = dmin(1e30, tau / ((double)b1 + eps)), q2 = dmin(1e30, tau / ((double)b2 + eps)),
               q3 = dmin(1e30, tau / ((double)b3 + eps));
  const double w1 = (double)0.1f * (1 + q1 * q1), w2 = (double)0.6f * (1 + q2 * q2), w3 = (double)0.3f * (1 + q3 * q3);
  const float p1 = ((2.0f / 6.0f) * s1 + (-7.0f / 6.0f) * s2) + (11.0f / 6.0f) * s3;
  const float p2 = ((-1.0f / 6.0f) * s2 + (5.0f / 6.0f) * s3) + (2.0f / 6.0f) * s4;
  const float p3 = ((2.0f / 6.0f) * s3 + (5.0f / 6.0f) * s4) + (-1.0f / 6.0f) * s5;
  return (float)((w1 * p1 + w2 * p2 + w3 * p3) / (w1 + w2 + w3));
}
static float upstrpdo(float s1, float s2, float s3, float weps) {
  const float dd = s2 - s1;
  const float se = copysignf(fabsf(weps), dd);
  const float rr = (s3 - s2) / (se + dd);
  const float cand = (1.0f / 6.0f) + (2.0f / 6.0f) * rr;
  float m = cand < 1.0f ? cand : 1.0f;
  m = rr < m ? rr : m;
  const float phi = m > 0.0f ? m : 0.0f;
  return s2 + phi * (s2 - s1);
}
static float rec5(const float* v, int w, double eps) {
  return w ? weno5o(v[0], v[1], v[2], v[3], v[4], eps) : flx5o(v[0], v[1], v[2], v[3], v[4]);
}

#define RRU(k, j, f) g->rru[I3((k), (j) + NG, (f) + NG, g->nj + 2 * NG, g->ni + 1 + 2 * NG)]
#define RRV(k, f, i) g->rrv[I3((k), (f) + NG, (i) + NG, g->nj + 1 + 2 * NG, g->ni + 2 * NG)]
#define RRW(k, j, i) g->rrw[I3((k), (j) + NG, (i) + NG, g->nj + 2 * NG, g->ni + 2 * NG)]

/* horizontal face flux (cuda_tke_evolution.py:172-191): axis 0 = x face
 * `face` of row `row`, axis 1 = y face `face` of column `row` */
static float hflux(const tke_grid* g, const float* q, int f, int row, int face, int axis, int w, double eps, int ov,
                   float* mass_out) {
  float c2, mass;
  if (axis == 0) {
    c2 = 0.5f * (CELL(g, g->c2, f, row, face - 1) + CELL(g, g->c2, f, row, face));
    mass = c2 * RRU(f + 1, row, face) + (1.0f - c2) * RRU(f, row, face);
  } else {
    c2 = 0.5f * (CELL(g, g->c2, f, face - 1, row) + CELL(g, g->c2, f, face, row));
    mass = c2 * RRV(f + 1, face, row) + (1.0f - c2) * RRV(f, face, row);
  }
  *mass_out = mass;
  const int n = axis == 0 ? g->ni : g->nj;
  float dummy;
  if (ov && face == 0 && mass >= 0.0f) return hflux(g, q, f, row, 1, axis, w, eps, 0, &dummy);
  if (ov && face == n && mass <= 0.0f) return hflux(g, q, f, row, n - 1, axis, w, eps, 0, &dummy);
  static const int up[5] = {-3, -2, -1, 0, 1}, dn[5] = {2, 1, 0, -1, -2};
  const int* ids = mass >= 0.0f ? up : dn;
  float v[5];
  for (int s = 0; s < 5; ++s) v[s] = axis == 0 ? CELL(g, q, f, row, face + ids[s]) : CELL(g, q, f, face + ids[s], row);
  return mass * rec5(v, w, eps);
}

/* vertical flux at face-level-stagger index ks (cuda_tke_evolution.py:194-203) */
static float vflux(const tke_grid* g, const float* q, int ks, int j, int i, int w, double eps) {
  const int nk = g->nk;
  const float mass = 0.5f * (RRW(ks, j, i) + RRW(ks + 1, j, i));
#define Q(k) q[I3((k), j, i, g->nj, g->ni)]
  const float wf = (float)eps;
  float r, v[5];
  if (ks == 1) {
    r = mass >= 0.0f ? 0.5f * (Q(0) + Q(1)) : (w ? upstrpdo(Q(2), Q(1), Q(0), wf) : flx3o(Q(2), Q(1), Q(0)));
  } else if (ks == 2) {
    if (mass >= 0.0f) {
      r = w ? upstrpdo(Q(0), Q(1), Q(2), wf) : flx3o(Q(0), Q(1), Q(2));
    } else {
      for (int s = 0; s < 5; ++s) v[s] = Q(4 - s);
      r = rec5(v, w, eps);
    }
  } else if (ks == nk - 1) {
    if (w ? mass > 0.0f : mass >= 0.0f) {
      for (int s = 0; s < 5; ++s) v[s] = Q(ks - 3 + s);
      r = rec5(v, w, eps);
    } else {
      r = w ? upstrpdo(Q(ks + 1), Q(ks), Q(ks - 1), wf) : flx3o(Q(ks + 1), Q(ks), Q(ks - 1));
    }
  } else if (ks == nk) {
    r = (w ? mass > 0.0f : mass >= 0.0f) ? (w ? upstrpdo(Q(nk - 2), Q(nk - 1), Q(nk), wf) : flx3o(Q(nk - 2), Q(nk - 1), Q(nk)))
                                         : 0.5f * (Q(nk - 1) + Q(nk));
  } else if (mass >= 0.0f) {
    for (int s = 0; s < 5; ++s) v[s] = Q(ks - 3 + s);
    r = rec5(v, w, eps);
  } else {
    for (int s = 0; s < 5; ++s) v[s] = Q(ks + 2 - s);
    r = rec5(v, w, eps);
  }
#undef Q
  return mass * r;
}

int oracle_tke_rk_stage(int ni, int nj, int nk, const float* cur, const float* tkea, const float* tketen,
                        const float* c1, const float* c2, const float* rrf0, const float* gz, const float* rru,
                        const float* rrv, const float* rrw, const float* divx, float* nxt, int nrk, float dx, float dy,
                        float dz, float dt) {
  (void)c1;
  if (ni < 3 || nj < 3 || nk < 6 || nrk < 1 || nrk > 3) return -1;
  tke_grid gg = {ni, nj, nk, 0, 0, 0, 0, 0, 0, gz, 0, 0, 0, c1, c2, rrf0, rru, rrv, rrw, divx};
  const tke_grid* g = &gg;
  const float rdx = 1.0f / dx, rdy = 1.0f / dy, rdz = 1.0f / dz;
  const float dttmp = dt / (float)(4 - nrk);
  const int w = nrk == 3;
  const double eps = (double)(100.0f * 1e-18f);
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i < ni; ++i) {
      nxt[I3(0, j, i, nj, ni)] = 0.0f;
      nxt[I3(nk, j, i, nj, ni)] = 0.0f;
    }
  for (int f = 1; f < nk; ++f)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        float mw, me, ms, mn;
        const float fx0 = hflux(g, cur, f, j, i, 0, w, eps, 1, &mw);
        const float fx1 = hflux(g, cur, f, j, i + 1, 0, w, eps, 1, &me);
        const float fy0 = hflux(g, cur, f, i, j, 1, w, eps, 1, &ms);
        const float fy1 = hflux(g, cur, f, i, j + 1, 1, w, eps, 1, &mn);
        float ax = -1.0f * ((fx1 - fx0) * rdx);
        float ay = -1.0f * ((fy1 - fy0) * rdy);
        const int64_t z = I3(f, j, i, nj, ni);
        const float cc2 = c2[z], cc1 = 1.0f - cc2;
        const float q = cur[z];
        if ((i == 0 && mw >= 0.0f) || (i == ni - 1 && me <= 0.0f)) {
          const float du = cc1 * (RRU(f, j, i + 1) - RRU(f, j, i)) + cc2 * (RRU(f + 1, j, i + 1) - RRU(f + 1, j, i));
          ax = ax - q * (du * rdx);
        }
        if ((j == 0 && ms >= 0.0f) || (j == nj - 1 && mn <= 0.0f)) {
          const float dv = cc1 * (RRV(f, j + 1, i) - RRV(f, j, i)) + cc2 * (RRV(f + 1, j + 1, i) - RRV(f + 1, j, i));
          ay = ay - q * (dv * rdy);
        }
        const float az = -1.0f * ((vflux(g, cur, f + 1, j, i, w, eps) - vflux(g, cur, f, j, i, w, eps)) * rdz);
        float total = (ax + ay) + az;
        total = total + q * (cc2 * divx[I3(f, j, i, nj, ni)] + cc1 * divx[I3(f - 1, j, i, nj, ni)]);
        const float wten = tketen[z] + total * (rrf0[z] * gz[(int64_t)j * ni + i]);
        const float value = tkea[z] + dttmp * wten;
        nxt[z] = value < 1e-10f ? 0.0f : value;
      }
  return 0;
}

/* ---- flat (terrain_flag=.false.) stretched column --------------------- */

/* turbt, gm1_flat_turbt_v1 (src/cm1core/cuda_gm1_flat_stretched_closure.py:314-359;
 * turbtend.F:729-1044): per column, the x/y face fluxes at each face level,
 * the implicit diffusion with the coordinate's reference rdz and the 3-D mh
 * (mass) and mf (face), added into tketen. */
static float tfx_flat(const tke_grid* g, const float* t, int f, int j, int a, float rdx) {
  float r = 0.25f * (CELL(g, g->rf, f, j, a) + CELL(g, g->rf, f, j, a - 1));
  r = r * 2.0f;
  r = r * (CELL(g, g->kmh, f, j, a) + CELL(g, g->kmh, f, j, a - 1));
  r = r * (CELL(g, t, f, j, a) - CELL(g, t, f, j, a - 1));
  return -(r * rdx);
}
static float tfy_flat(const tke_grid* g, const float* t, int f, int b, int i, float rdy) {
  float r = 0.25f * (CELL(g, g->rf, f, b, i) + CELL(g, g->rf, f, b - 1, i));
  r = r * 2.0f;
  r = r * (CELL(g, g->kmh, f, b, i) + CELL(g, g->kmh, f, b - 1, i));
  r = r * (CELL(g, t, f, b, i) - CELL(g, t, f, b - 1, i));
  return -(r * rdy);
}

int oracle_tke_diffusion_flat(int ni, int nj, int nk, const float* t, const float* kmh, const float* kmv,
                              const float* rho, const float* rf, const float* mh, const float* mf, float* ten,
                              float dx, float dy, float rdz, float dt) {
  if (ni < 3 || nj < 3 || nk < 6) return -1;
  tke_grid gg = {ni, nj, nk, kmh, kmv, rho, rf, mh, mf, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const tke_grid* g = &gg;
  const float rdx = 1.0f / dx, rdy = 1.0f / dy, rdt = 1.0f / dt;
  const float tema = (((-1.0f * dt) * 1.0f) * rdz) * rdz, temb = ((dt * 0.0f) * rdz) * rdz;
  float *hx = malloc(sizeof(float) * (nk + 1)), *hy = malloc(sizeof(float) * (nk + 1));
  float *d1 = malloc(sizeof(float) * (nk + 1)), *d2 = malloc(sizeof(float) * (nk + 1));
  float *d3 = malloc(sizeof(float) * (nk + 1)), *tz = malloc(sizeof(float) * (nk + 1));
  if (!hx || !hy || !d1 || !d2 || !d3 || !tz) return -2;
#define TF(f) t[I3((f), j, i, nj, ni)]
#define PF(a, f) a[I3((f), j, i, nj, ni)]
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i < ni; ++i) {
      for (int f = 1; f < nk; ++f) {
        hx[f] = -((tfx_flat(g, t, f, j, i + 1, rdx) - tfx_flat(g, t, f, j, i, rdx)) * rdx);
        hy[f] = -((tfy_flat(g, t, f, j + 1, i, rdy) - tfy_flat(g, t, f, j, i, rdy)) * rdy);
        if (i == 0 || i == ni - 1) hx[f] = 0.0f;
        if (j == 0 || j == nj - 1) hy[f] = 0.0f;
      }
      {
        const int f = 1;
        const float rrf = PF(mf, f) / PF(rf, f);
        const float r2 = (((PF(kmv, f) + PF(kmv, f + 1)) * PF(mh, f)) * PF(rho, f)) * rrf;
        const float cfc = tema * r2, cfb = 1.0f - cfc;
        const float cfd = TF(f) + temb * ((r2 * TF(f + 1)) - (r2 * TF(f)));
        const float inv = 1.0f / cfb;
        d1[f] = -(cfc * inv);
        d2[f] = cfd * inv;
      }
      for (int f = 2; f < nk - 1; ++f) {
        const float rrf = PF(mf, f) / PF(rf, f);
        const float r1 = (((PF(kmv, f - 1) + PF(kmv, f)) * PF(mh, f - 1)) * PF(rho, f - 1)) * rrf;
        const float r2 = (((PF(kmv, f) + PF(kmv, f + 1)) * PF(mh, f)) * PF(rho, f)) * rrf;
        const float cfa = tema * r1, cfc = tema * r2, cfb = (1.0f - cfa) - cfc;
        const float cfd = TF(f) + temb * (((r2 * TF(f + 1)) - ((r1 + r2) * TF(f))) + (r1 * TF(f - 1)));
        const float inv = 1.0f / (cfa * d1[f - 1] + cfb);
        d1[f] = -(cfc * inv);
        d2[f] = (cfd - cfa * d2[f - 1]) * inv;
      }
      {
        const int f = nk - 1;
        const float rrf = PF(mf, f) / PF(rf, f);
        const float r1 = (((PF(kmv, f - 1) + PF(kmv, f)) * PF(mh, f - 1)) * PF(rho, f - 1)) * rrf;
        const float cfa = tema * r1, cfb = 1.0f - cfa;
        const float cfd = TF(f) + temb * ((-(r1 * TF(f))) + (r1 * TF(f - 1)));
        const float inv = 1.0f / (cfa * d1[f - 1] + cfb);
        d3[f] = (cfd - cfa * d2[f - 1]) * inv;
        tz[f] = (PF(rf, f) * (d3[f] - TF(f))) * rdt;
      }
      for (int f = nk - 2; f >= 1; --f) {
        d3[f] = d1[f] * d3[f + 1] + d2[f];
        tz[f] = (PF(rf, f) * (d3[f] - TF(f))) * rdt;
      }
      for (int f = 1; f < nk; ++f) {
        const int64_t p = I3(f, j, i, nj, ni);
        ten[p] = ten[p] + ((hx[f] + hy[f]) + tz[f]) / rf[p];
      }
    }
#undef TF
#undef PF
  free(hx);
  free(hy);
  free(d1);
  free(d2);
  free(d3);
  free(tz);
  return 0;
}

/* One RK stage on a flat column, gm1_flat_tke_advw_rk_v1 (the stretched TKE
 * advw text with the flat patches of
 * src/cm1core/cuda_gm1_flat_stretched_closure.py:401-449): vertical
 * divergence -(dumz(k)-dumz(k-1))*rdz*mfp(k) (mfp the nk+3 mf profile,
 * CM1-indexed), the column's c2 (its (k, 0, 0) word) in the divergence
 * correction and its rrf0, the cell's c2 in the open-side pieces (q*d)*rdx,
 * no gz. */
int oracle_tke_rk_stage_flat(int ni, int nj, int nk, const float* cur, const float* tkea, const float* tketen,
                             const float* c2, const float* rrf0, const float* rru, const float* rrv, const float* rrw,
                             const float* divx, const float* mfp, float* nxt, int nrk, float dx, float dy, float rdz,
                             float dt) {
  if (ni < 3 || nj < 3 || nk < 6 || nrk < 1 || nrk > 3) return -1;
  tke_grid gg = {ni, nj, nk, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, c2, rrf0, rru, rrv, rrw, divx};
  const tke_grid* g = &gg;
  const float rdx = 1.0f / dx, rdy = 1.0f / dy;
  const float dttmp = dt / (float)(4 - nrk);
  const int w = nrk == 3;
  const double eps = (double)(100.0f * 1e-18f);
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i < ni; ++i) {
      nxt[I3(0, j, i, nj, ni)] = 0.0f;
      nxt[I3(nk, j, i, nj, ni)] = 0.0f;
    }
  for (int f = 1; f < nk; ++f)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        float mw, me, ms, mn;
        const float fx0 = hflux(g, cur, f, j, i, 0, w, eps, 1, &mw);
        const float fx1 = hflux(g, cur, f, j, i + 1, 0, w, eps, 1, &me);
        const float fy0 = hflux(g, cur, f, i, j, 1, w, eps, 1, &ms);
        const float fy1 = hflux(g, cur, f, i, j + 1, 1, w, eps, 1, &mn);
        float ax = -1.0f * ((fx1 - fx0) * rdx);
        float ay = -1.0f * ((fy1 - fy0) * rdy);
        const int64_t z = I3(f, j, i, nj, ni);
        const float cc2 = c2[z], cc1 = 1.0f - cc2;
        const float c2c = c2[I3(f, 0, 0, nj, ni)], c1c = 1.0f - c2c;
        const float q = cur[z];
        if ((i == 0 && mw >= 0.0f) || (i == ni - 1 && me <= 0.0f)) {
          const float d = cc1 * (RRU(f, j, i + 1) - RRU(f, j, i)) + cc2 * (RRU(f + 1, j, i + 1) - RRU(f + 1, j, i));
          ax = ax - (q * d) * rdx;
        }
        if ((j == 0 && ms >= 0.0f) || (j == nj - 1 && mn <= 0.0f)) {
          const float d = cc1 * (RRV(f, j + 1, i) - RRV(f, j, i)) + cc2 * (RRV(f + 1, j + 1, i) - RRV(f + 1, j, i));
          ay = ay - (q * d) * rdy;
        }
        const float dv = vflux(g, cur, f + 1, j, i, w, eps) - vflux(g, cur, f, j, i, w, eps);
        const float az = ((-dv) * rdz) * mfp[f + 1];
        float total = (ax + ay) + az;
        total = total + q * (c2c * divx[I3(f, j, i, nj, ni)] + c1c * divx[I3(f - 1, j, i, nj, ni)]);
        const float wten = tketen[z] + total * rrf0[I3(f, 0, 0, nj, ni)];
        const float value = tkea[z] + dttmp * wten;
        nxt[z] = value < 1e-10f ? 0.0f : value;
      }
  return 0;
}
