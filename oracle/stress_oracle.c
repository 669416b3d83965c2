/* Oracle (test infrastructure only): CPU restatement of the SGS stress
 * tendencies of the flat (terrain_flag=.false.) stretched column.
 *
 *   gettau, free-slip lower and upper faces
 *       enqueue_flat_gettau               src/cm1core/cuda_gm1_flat_stretched_closure.py:551-571
 *       texts gm1_flat_gettau_normal_v1 / _t12_v1 / _t13_v1 / _t23_v1       :134-161
 *       (CM1 turb.F:4094-4190, :4281-4433, :4536-4545)
 *   turbu/turbuz, turbv/turbvz, turbw (two-part block off, ntwk = 0)
 *       enqueue_flat_momentum_stress      src/cm1core/cuda_gm1_flat_stretched_closure.py:574-618
 *       texts gm1_flat_turbu_v1 / _turbv_v1 / _turbw_v1, COLUMN_IMPLICIT   :163-292
 *       (CM1 turbtend.F:1095-1361, :1438-1560, :1860-2128, :2194-2310, :2508-2885)
 *
 * The reference has no NumPy twin of these texts: this restates the CUDA
 * source statement by statement (binary32, one operation at a time, built
 * with -ffp-contract=off; the literal zero factors of vibeta = 0 are formed
 * so signed zeros stay what they are), pinned word for word to those texts
 * compiled and run on the host (tests/golden/make_kernel_text_golden.py).  Open sides are index clamps (CM1's
 * zero-gradient halo).  Shapes (C order): s11/s22/s33/t11/t22/t33/rho/mh
 * (nk, nj, ni); s12/t12 (nk, nj+1, ni+1); s13/t13 (nk+1, nj, ni+1);
 * s23/t23 (nk+1, nj+1, ni); kmh/kmv/rf/mf/w/wten (nk+1, nj, ni);
 * u/uten (nk, nj, ni+1); v/vten (nk, nj+1, ni).  The tendencies are added
 * into uten, vten and wten (wten at faces 1..nk-1).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include "real.h"

#define I3(k, j, i, ny, nx) ((((int64_t)(k)) * (ny) + (j)) * (nx) + (i))

static int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

/* a mass- or face-shaped (.., nj, ni) carrier at a clamped column */
static float cell(const float* a, int k, int j, int i, int nj, int ni) {
  return a[I3(k, clampi(j, 0, nj - 1), clampi(i, 0, ni - 1), nj, ni)];
}

int oracle_flat_gettau(int ni, int nj, int nk, const float* s11, const float* s22, const float* s33, const float* s12,
                       const float* s13, const float* s23, const float* kmh, const float* kmv, float* t11, float* t22,
                       float* t33, float* t12, float* t13, float* t23) {
  if (ni < 3 || nj < 3 || nk < 3) return -1;
  const int64_t z = (int64_t)ni * nj;
  for (int64_t q = 0; q < (int64_t)nk * z; ++q) {
    const float m = kmh[q] + kmh[q + z];
    t11[q] = s11[q] * m;
    t22[q] = s22[q] * m;
    t33[q] = s33[q] * m;
  }
  for (int k = 0; k < nk; ++k)
    for (int jc = 0; jc <= nj; ++jc)
      for (int ic = 0; ic <= ni; ++ic) {
        const int ii = clampi(ic, 1, ni - 1), jj = clampi(jc, 1, nj - 1);
        const float lo = (kmh[I3(k, jj - 1, ii - 1, nj, ni)] + kmh[I3(k, jj, ii, nj, ni)]) +
                         (kmh[I3(k, jj, ii - 1, nj, ni)] + kmh[I3(k, jj - 1, ii, nj, ni)]);
        const float hi = (kmh[I3(k + 1, jj - 1, ii - 1, nj, ni)] + kmh[I3(k + 1, jj, ii, nj, ni)]) +
                         (kmh[I3(k + 1, jj, ii - 1, nj, ni)] + kmh[I3(k + 1, jj - 1, ii, nj, ni)]);
        t12[I3(k, jc, ic, nj + 1, ni + 1)] = (s12[I3(k, jj, ii, nj + 1, ni + 1)] * 0.25f) * (lo + hi);
      }
  for (int f = 0; f <= nk; ++f) {
    const int ff = f == 0 ? 1 : (f == nk ? nk - 1 : f);
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i <= ni; ++i)
        t13[I3(f, j, i, nj, ni + 1)] =
            s13[I3(ff, j, i, nj, ni + 1)] * (cell(kmv, ff, j, i - 1, nj, ni) + cell(kmv, ff, j, i, nj, ni));
    for (int j = 0; j <= nj; ++j)
      for (int i = 0; i < ni; ++i)
        t23[I3(f, j, i, nj + 1, ni)] =
            s23[I3(ff, j, i, nj + 1, ni)] * (cell(kmv, ff, j - 1, i, nj, ni) + cell(kmv, ff, j, i, nj, ni));
  }
  return 0;
}

/* one u- or v-point column of turbuz/turbvz (COLUMN_IMPLICIT): the cells
 * either side are (ja, ia) and (jb, ib); q is the column's wind at mass
 * levels (stride qs), top13 its t13/t23 at face levels (stride ts), rd the
 * horizontal 1/spacing across the pair.  Writes the vertical term tz[k]. */
static void column_implicit(int nk, int nj, int ni, int ja, int ia, int jb, int ib, const float* q, int64_t qs,
                            const float* top13, int64_t ts, const float* kmv, const float* rho, const float* rf,
                            const float* mh, const float* mf, const float* w, float rd, float rdz, float dt,
                            float* d1, float* d2, float* d3, float* d7, float* tz) {
#define PAIR(a, k) (cell(a, k, ja, ia, nj, ni) + cell(a, k, jb, ib, nj, ni))
#define QK(k) q[(int64_t)(k) * qs]
  const int K = nk;
  const float rdt = 0.5f / dt;
  const float tema = (((-0.0625f * dt) * 1.0f) * rdz) * rdz;
  const float temb = (((0.0625f * dt) * 0.0f) * rdz) * rdz;
  const float temc = (0.5f * dt) * rdz;
  {
    const int k = 0;
    const float rr0 = 1.0f / (0.5f * PAIR(rho, k));
    const float tem = PAIR(mh, k) * rr0;
    const float r2 = ((PAIR(kmv, k + 1) * PAIR(mf, k + 1)) * PAIR(rf, k + 1)) * tem;
    const float cfc = tema * r2, cfb = 1.0f - cfc, qk = QK(k), qp = QK(k + 1);
    const float cfd = (qk + temb * (r2 * qp - r2 * qk)) - ((temc * top13[0]) * PAIR(mh, 0)) * rr0;
    const float inv = 1.0f / cfb;
    d1[0] = -(cfc * inv);
    d2[0] = cfd * inv;
    d7[0] = 0.0f;
  }
  for (int k = 1; k < K - 1; ++k) {
    const float rr0 = 1.0f / (0.5f * PAIR(rho, k));
    const float tem = PAIR(mh, k) * rr0;
    const float r1 = ((PAIR(kmv, k) * PAIR(mf, k)) * PAIR(rf, k)) * tem;
    const float r2 = ((PAIR(kmv, k + 1) * PAIR(mf, k + 1)) * PAIR(rf, k + 1)) * tem;
    const float cfa = tema * r1, cfc = tema * r2, cfb = (1.0f - cfa) - cfc;
    const float qk = QK(k), qp = QK(k + 1), qm = QK(k - 1);
    const float cfd = qk + temb * ((r2 * qp - (r1 + r2) * qk) + r1 * qm);
    const float inv = 1.0f / (cfa * d1[k - 1] + cfb);
    d1[k] = -(cfc * inv);
    d2[k] = (cfd - cfa * d2[k - 1]) * inv;
    d7[k] = ((((cell(w, k, jb, ib, nj, ni) - cell(w, k, ja, ia, nj, ni)) * rd) * 0.25f) * PAIR(kmv, k)) * PAIR(rf, k);
  }
  {
    const int k = K - 1;
    const float rr0 = 1.0f / (0.5f * PAIR(rho, k));
    const float tem = PAIR(mh, k) * rr0;
    const float r1 = ((PAIR(kmv, k) * PAIR(mf, k)) * PAIR(rf, k)) * tem;
    const float cfa = tema * r1, cfb = 1.0f - cfa, qk = QK(k), qm = QK(k - 1);
    const float cfd = (qk + temb * (-(r1 * qk) + r1 * qm)) + ((temc * top13[(int64_t)K * ts]) * PAIR(mh, k)) * rr0;
    const float inv = 1.0f / (cfa * d1[k - 1] + cfb);
    d3[k] = (cfd - cfa * d2[k - 1]) * inv;
    tz[k] = (PAIR(rho, k) * (d3[k] - qk)) * rdt;
    d7[k] = ((((cell(w, k, jb, ib, nj, ni) - cell(w, k, ja, ia, nj, ni)) * rd) * 0.25f) * PAIR(kmv, k)) * PAIR(rf, k);
    tz[k] = tz[k] + (((0.0f - d7[k]) * rdz) * 0.5f) * PAIR(mh, k);
  }
  for (int k = K - 2; k >= 0; --k) {
    d3[k] = d1[k] * d3[k + 1] + d2[k];
    tz[k] = (PAIR(rho, k) * (d3[k] - QK(k))) * rdt;
    tz[k] = tz[k] + (((d7[k + 1] - d7[k]) * rdz) * 0.5f) * PAIR(mh, k);
  }
#undef QK
}

int oracle_flat_momentum_stress(int ni, int nj, int nk, const float* t11, const float* t22, const float* t33,
                                const float* t12, const float* t13, const float* t23, const float* kmh,
                                const float* kmv, const float* rho, const float* rf, const float* mh, const float* mf,
                                const float* u, const float* v, const float* w, float dx, float dy, float rdz, float dt,
                                float* uten, float* vten, float* wten) {
  if (ni < 3 || nj < 3 || nk < 3) return -1;
  const float rdx = 1.0f / dx, rdy = 1.0f / dy;
  const int K = nk;
  float* buf = malloc(sizeof(float) * 7 * (size_t)(nk + 1));
  if (!buf) return -2;
  float *hx = buf, *hy = buf + (nk + 1), *d1 = buf + 2 * (nk + 1), *d2 = buf + 3 * (nk + 1);
  float *d3 = buf + 4 * (nk + 1), *d7 = buf + 5 * (nk + 1), *tz = buf + 6 * (nk + 1);
  const int ux = ni + 1, vy = nj + 1;
  /* turbu: one column per u point (j, f), f in [0, ni] */
  for (int j = 0; j < nj; ++j)
    for (int f = 0; f <= ni; ++f) {
      const int ia = f - 1, ib = f, ja = j, jb = j;
      for (int k = 0; k < K; ++k) {
        hx[k] = (cell(t11, k, j, ib, nj, ni) - cell(t11, k, j, ia, nj, ni)) * rdx;
        hy[k] = (t12[I3(k, j + 1, f, vy, ux)] - t12[I3(k, j, f, vy, ux)]) * rdy;
        if (f == 0 || f == ni) hx[k] = 0.0f;
        if (j == 0 || j == nj - 1) hy[k] = 0.0f;
      }
      column_implicit(nk, nj, ni, ja, ia, jb, ib, &u[I3(0, j, f, nj, ux)], (int64_t)nj * ux,
                      &t13[I3(0, j, f, nj, ux)], (int64_t)nj * ux, kmv, rho, rf, mh, mf, w, rdx, rdz, dt, d1, d2, d3,
                      d7, tz);
      for (int k = 0; k < K; ++k) {
        const float rr0 = 1.0f / (0.5f * PAIR(rho, k));
        const int64_t p = I3(k, j, f, nj, ux);
        uten[p] = uten[p] + ((hx[k] + hy[k]) + tz[k]) * rr0;
      }
    }
  /* turbv: one column per v point (f, i), f in [0, nj] */
  for (int f = 0; f <= nj; ++f)
    for (int i = 0; i < ni; ++i) {
      const int ia = i, ib = i, ja = f - 1, jb = f;
      for (int k = 0; k < K; ++k) {
        hx[k] = (t12[I3(k, f, i + 1, vy, ux)] - t12[I3(k, f, i, vy, ux)]) * rdx;
        hy[k] = (cell(t22, k, jb, i, nj, ni) - cell(t22, k, ja, i, nj, ni)) * rdy;
        if (i == 0 || i == ni - 1) hx[k] = 0.0f;
        if (f == 0 || f == nj) hy[k] = 0.0f;
      }
      column_implicit(nk, nj, ni, ja, ia, jb, ib, &v[I3(0, f, i, vy, ni)], (int64_t)vy * ni,
                      &t23[I3(0, f, i, vy, ni)], (int64_t)vy * ni, kmv, rho, rf, mh, mf, w, rdy, rdz, dt, d1, d2, d3,
                      d7, tz);
      for (int k = 0; k < K; ++k) {
        const float rr0 = 1.0f / (0.5f * PAIR(rho, k));
        const int64_t p = I3(k, f, i, vy, ni);
        vten[p] = vten[p] + ((hx[k] + hy[k]) + tz[k]) * rr0;
      }
    }
#undef PAIR
  /* turbw: one column per mass column (j, i), faces 1..nk-1 */
  {
    const float rdt = 1.0f / dt;
    const float tema = (((-1.0f * dt) * 1.0f) * rdz) * rdz;
    const float temb = ((dt * 0.0f) * rdz) * rdz;
    const float temc = dt * rdz;
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
#define WF(f) w[I3(f, j, i, nj, ni)]
#define PF(a, f) a[I3(f, j, i, nj, ni)]
        for (int f = 1; f < K; ++f) {
          hx[f] = (t13[I3(f, j, i + 1, nj, ux)] - t13[I3(f, j, i, nj, ux)]) * rdx;
          hy[f] = (t23[I3(f, j + 1, i, vy, ni)] - t23[I3(f, j, i, vy, ni)]) * rdy;
          if (i == 0 || i == ni - 1) hx[f] = 0.0f;
          if (j == 0 || j == nj - 1) hy[f] = 0.0f;
        }
        {
          const int f = 1;
          const float rrf = PF(mf, f) / PF(rf, f);
          const float r2 = (((PF(kmh, f) + PF(kmh, f + 1)) * PF(mh, f)) * PF(rho, f)) * rrf;
          const float cfc = tema * r2, cfb = 1.0f - cfc;
          const float cfd = (WF(f) + temb * (r2 * WF(f + 1) - r2 * WF(f))) - (temc * PF(t33, f - 1)) * rrf;
          const float inv = 1.0f / cfb;
          d1[f] = -(cfc * inv);
          d2[f] = cfd * inv;
        }
        for (int f = 2; f < K - 1; ++f) {
          const float rrf = PF(mf, f) / PF(rf, f);
          const float r1 = (((PF(kmh, f - 1) + PF(kmh, f)) * PF(mh, f - 1)) * PF(rho, f - 1)) * rrf;
          const float r2 = (((PF(kmh, f) + PF(kmh, f + 1)) * PF(mh, f)) * PF(rho, f)) * rrf;
          const float cfa = tema * r1, cfc = tema * r2, cfb = (1.0f - cfa) - cfc;
          const float cfd = WF(f) + temb * ((r2 * WF(f + 1) - (r1 + r2) * WF(f)) + r1 * WF(f - 1));
          const float inv = 1.0f / (cfa * d1[f - 1] + cfb);
          d1[f] = -(cfc * inv);
          d2[f] = (cfd - cfa * d2[f - 1]) * inv;
        }
        {
          const int f = K - 1;
          const float rrf = PF(mf, f) / PF(rf, f);
          const float r1 = (((PF(kmh, f - 1) + PF(kmh, f)) * PF(mh, f - 1)) * PF(rho, f - 1)) * rrf;
          const float cfa = tema * r1, cfb = 1.0f - cfa;
          const float cfd = (WF(f) + temb * (-(r1 * WF(f)) + r1 * WF(f - 1))) + (temc * PF(t33, f)) * rrf;
          const float inv = 1.0f / (cfa * d1[f - 1] + cfb);
          d3[f] = (cfd - cfa * d2[f - 1]) * inv;
          tz[f] = (PF(rf, f) * (d3[f] - WF(f))) * rdt;
        }
        for (int f = K - 2; f >= 1; --f) {
          d3[f] = d1[f] * d3[f + 1] + d2[f];
          tz[f] = (PF(rf, f) * (d3[f] - WF(f))) * rdt;
        }
        for (int f = 1; f < K; ++f) {
          const int64_t p = I3(f, j, i, nj, ni);
          wten[p] = wten[p] + ((hx[f] + hy[f]) + tz[f]) / rf[p];
        }
#undef WF
#undef PF
      }
  }
  free(buf);
  return 0;
}

/* ------------------------------------------------------------------------
 * turbs on the flat column (numq moisture rows after theta), the four open
 * sides, no surface flux (iflux = 0):
 *   the open-halo copies        gm1_turbs_pad_static_open_v1 / _pack_scalar_open_v1
 *                               src/cm1core/cuda_gm1_scalar_turbulence.py:453-466
 *                               (theta is (th0 - 300) + tha, bc.F:180-364)
 *   the flat fluxes and turbsz  gm1_flat_turbs_xy_flux_v1 / _implicit_apply_v1
 *                               src/cm1core/cuda_gm1_flat_stretched_closure.py:335-381
 *                               (turbtend.F:60-434, :442-692; solve1.F:1169-1233)
 * th0 (nk), tha/rho/rr/mh (nk, nj, ni), qa and qten (rows of nk*nj*ni),
 * rf/mf/khh/khv (nk+1, nj, ni).  The tendencies are ADDED into thten and
 * the first numq rows of qten.  dz is the coordinate's reference spacing.
 */
typedef struct {
  int ni, nj, nk;
  const float *th0, *tha, *q; /* q != NULL: a moisture row, else theta */
} scalar_src;

/* the open-halo scalar at a clamped cell */
static float sval(const scalar_src* s, int k, int j, int i) {
  const int64_t p = I3(k, clampi(j, 0, s->nj - 1), clampi(i, 0, s->ni - 1), s->nj, s->ni);
  if (s->q) return s->q[p];
  return (s->th0[k] - 300.0f) + s->tha[p];
}

/* x flux through the face between cells f-1 and f (f in [0, ni]) */
static float flux_x(const scalar_src* s, const float* rho, const float* khh, int k, int j, int f, float rx) {
  const int nj = s->nj, ni = s->ni;
  const float den = cell(rho, k, j, f, nj, ni) + cell(rho, k, j, f - 1, nj, ni);
  const float kh = (cell(khh, k, j, f, nj, ni) + cell(khh, k, j, f - 1, nj, ni)) +
                   (cell(khh, k + 1, j, f, nj, ni) + cell(khh, k + 1, j, f - 1, nj, ni));
  return (((-0.125f * den) * kh) * (sval(s, k, j, f) - sval(s, k, j, f - 1))) * rx;
}

/* y flux through the face between rows f-1 and f (f in [0, nj]) */
static float flux_y(const scalar_src* s, const float* rho, const float* khh, int k, int f, int i, float ry) {
  const int nj = s->nj, ni = s->ni;
  const float den = cell(rho, k, f, i, nj, ni) + cell(rho, k, f - 1, i, nj, ni);
  const float kh = (cell(khh, k, f, i, nj, ni) + cell(khh, k, f - 1, i, nj, ni)) +
                   (cell(khh, k + 1, f, i, nj, ni) + cell(khh, k + 1, f - 1, i, nj, ni));
  return (((-0.125f * den) * kh) * (sval(s, k, f, i) - sval(s, k, f - 1, i))) * ry;
}

static void turbs_one(const scalar_src* s, const float* rho, const float* rr, const float* rf, const float* mh,
                      const float* mf, const float* khh, const float* khv, float dx, float dy, float dz, float dt,
                      float* target, float* cp, float* dp) {
  const int ni = s->ni, nj = s->nj, nk = s->nk;
  const float rx = 1.0f / dx, ry = 1.0f / dy, rz = 1.0f / dz, rdt = 1.0f / dt;
  const float tema = (((-1.0f * dt) * 1.0f) * rz) * rz;
  const float temb = ((dt * 0.0f) * rz) * rz;
  const float temc = dt * rz;
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i < ni; ++i) {
#define SC(k) sval(s, k, j, i)
#define COEF(F, K) \
  ((((khv[I3(F, j, i, nj, ni)] * mf[I3(F, j, i, nj, ni)]) * rf[I3(F, j, i, nj, ni)]) * mh[I3(K, j, i, nj, ni)]) * \
   rr[I3(K, j, i, nj, ni)])
      const int64_t col = I3(0, j, i, nj, ni);
      float r2 = COEF(1, 0);
      float cfc = tema * r2, cfb = 1.0f - cfc;
      float ex = (-r2) * SC(0) + r2 * SC(1);
      float bc = ((temc * 0.0f) * mh[col]) * rr[col];
      float cfd = (SC(0) + temb * ex) + bc;
      float tem = 1.0f / cfb;
      cp[0] = (-cfc) * tem;
      dp[0] = cfd * tem;
      for (int k = 1; k + 1 < nk; ++k) {
        const float r1 = COEF(k, k);
        r2 = COEF(k + 1, k);
        const float cfa = tema * r1;
        cfc = tema * r2;
        cfb = (1.0f - cfa) - cfc;
        ex = (r1 * SC(k - 1) - (r1 + r2) * SC(k)) + r2 * SC(k + 1);
        cfd = SC(k) + temb * ex;
        tem = 1.0f / (cfa * cp[k - 1] + cfb);
        cp[k] = (-cfc) * tem;
        dp[k] = (cfd - cfa * dp[k - 1]) * tem;
      }
      const int k = nk - 1;
      const int64_t top = I3(k, j, i, nj, ni);
      const float r1 = COEF(k, k), cfa = tema * r1;
      cfb = 1.0f - cfa;
      ex = r1 * SC(k - 1) - r1 * SC(k);
      bc = ((temc * 0.0f) * mh[top]) * rr[top];
      cfd = (SC(k) + temb * ex) - bc;
      tem = 1.0f / (cfa * cp[k - 1] + cfb);
      float sol = (cfd - cfa * dp[k - 1]) * tem;
      for (int kk = nk - 1; kk >= 0; --kk) {
        const int64_t mass = I3(kk, j, i, nj, ni);
        if (kk != nk - 1) sol = cp[kk] * sol + dp[kk];
        const float tz = (rho[mass] * (sol - SC(kk))) * rdt;
        float tx = -((flux_x(s, rho, khh, kk, j, i + 1, rx) - flux_x(s, rho, khh, kk, j, i, rx)) * rx);
        if (i == 0 || i + 1 == ni) tx = 0.0f;
        float ty = -((flux_y(s, rho, khh, kk, j + 1, i, ry) - flux_y(s, rho, khh, kk, j, i, ry)) * ry);
        if (j == 0 || j + 1 == nj) ty = 0.0f;
        target[mass] = target[mass] + ((tx + ty) + tz) * rr[mass];
      }
#undef SC
#undef COEF
    }
}

int oracle_flat_scalar_turbulence(int ni, int nj, int nk, int numq, const float* th0, const float* tha,
                                  const float* qa, const float* rho, const float* rr, const float* rf,
                                  const float* mh, const float* mf, const float* khh, const float* khv, float dx,
                                  float dy, float dz, float dt, float* thten, float* qten) {
  if (ni < 3 || nj < 3 || nk < 3 || numq < 0) return -1;
  float* buf = malloc(sizeof(float) * 2 * (size_t)nk);
  if (!buf) return -2;
  const int64_t n = (int64_t)ni * nj * nk;
  scalar_src s = {ni, nj, nk, th0, tha, NULL};
  turbs_one(&s, rho, rr, rf, mh, mf, khh, khv, dx, dy, dz, dt, thten, buf, buf + nk);
  for (int q = 0; q < numq; ++q) {
    s.q = qa + q * n;
    turbs_one(&s, rho, rr, rf, mh, mf, khh, khv, dx, dy, dz, dt, qten + q * n, buf, buf + nk);
  }
  free(buf);
  return 0;
}

/* ------------------------------------------------------------------------
 * Upper Rayleigh damping, irdamp = 1 (cpu_rayleigh_held_inplace and its
 * kernel cm1_rayleigh_held_physical_f32_v1,
 * src/cm1core/cuda_rayleigh_held.py:213-254, :419-488; CM1 solve1.F:412-454):
 *   uten1 = ((-rdalpha*0.5)*(tauh(i-1)+tauh(i)))*(ua - u0(k)), vten1 the
 *   same across j, wten1 = (-rdalpha*tauf)*wa, thten1 = (-rdalpha*taus)*tha.
 * profiles = 0: tauh/taus (nk, nj+2, ni+2) and tauf (nk+1, nj+2, ni+2) with
 * one horizontal halo (the reference's layout); profiles = 1: tauh/taus
 * (nk) and tauf (nk+1) column profiles.  add_momentum = 1 adds the damping
 * into the momentum outputs (uten1 = damping + uten1, the closure's held
 * sum cuda_cartesian_closure.py:1289-1291) and assigns thten1.
 */
static float tau_at(const float* tau, int profiles, int k, int jh, int ih, int nj, int ni) {
  return profiles ? tau[k] : tau[I3(k, jh, ih, nj + 2, ni + 2)];
}

int oracle_rayleigh_held(int ni, int nj, int nk, const float* tauh, const float* taus, const float* tauf,
                         const float* u0, const float* v0, const float* ua, const float* va, const float* wa,
                         const float* tha, int profiles, int add_momentum, float rdalpha, float* uten1,
                         float* vten1, float* wten1, float* thten1) {
  if (ni < 1 || nj < 1 || nk < 1) return -1;
  const float neg = -rdalpha, negh = neg * 0.5f;
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int f = 0; f <= ni; ++f) {
        const float pair = tau_at(tauh, profiles, k, j + 1, f, nj, ni) + tau_at(tauh, profiles, k, j + 1, f + 1, nj, ni);
        const int64_t z = I3(k, j, f, nj, ni + 1);
        const float d = (negh * pair) * (ua[z] - u0[k]);
        uten1[z] = add_momentum ? d + uten1[z] : d;
      }
  for (int k = 0; k < nk; ++k)
    for (int f = 0; f <= nj; ++f)
      for (int i = 0; i < ni; ++i) {
        const float pair = tau_at(tauh, profiles, k, f, i + 1, nj, ni) + tau_at(tauh, profiles, k, f + 1, i + 1, nj, ni);
        const int64_t z = I3(k, f, i, nj + 1, ni);
        const float d = (negh * pair) * (va[z] - v0[k]);
        vten1[z] = add_momentum ? d + vten1[z] : d;
      }
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const int64_t z = I3(k, j, i, nj, ni);
        const float dw = (neg * tau_at(tauf, profiles, k, j + 1, i + 1, nj, ni)) * wa[z];
        wten1[z] = add_momentum ? dw + wten1[z] : dw;
        thten1[z] = (neg * tau_at(taus, profiles, k, j + 1, i + 1, nj, ni)) * tha[z];
      }
  return 0;
}

/* ------------------------------------------------------------------------
 * Dissipative heating, idiss = 1 (cpu_idiss_cell_f32 and the consumer
 * Eqtset2IdissConsumer.apply, src/cm1core/eqtset2_energy_terms.py:176-215,
 * :375-470; CM1 solve1.F:744-848, :917-975): per cell
 *   cvm = ((cv + cvv*qv) + cpl*(qc+qr)) + cpi*((qi+qs)+qg)
 *   thten1 += (0.5*(dissten(k)+dissten(k+1))) / ((cpdcv*cvm)*(pi0+ppi))
 * dissten (nk+1, nj, ni), pi0 (nk), ppi/thten1 (nk, nj, ni), qa six rows of
 * nk*nj*ni words (qv qc qr qi qs qg).
 */
int oracle_dissipative_heating(int ni, int nj, int nk, const float* dissten, const float* pi0, const float* ppi,
                               const float* qa, float* thten1) {
  if (ni < 1 || nj < 1 || nk < 1) return -1;
  const float rd = 287.04f, cp = 1005.7f, cpv = 1870.0f, rv = 461.5f, cpl = 4190.0f, cpi = 2106.0f;
  const float cv = cp - rd, cvv = cpv - rv, cpdcv = cp / cv;
  const int64_t n = (int64_t)ni * nj * nk, plane = (int64_t)ni * nj;
  for (int64_t q = 0; q < n; ++q) {
    const int k = (int)(q / plane);
    const float ql = qa[n + q] + qa[2 * n + q];
    const float qice = (qa[3 * n + q] + qa[4 * n + q]) + qa[5 * n + q];
    float cvm = cv + cvv * qa[q];
    cvm = cvm + cpl * ql;
    cvm = cvm + cpi * qice;
    const float epsd = 0.5f * (dissten[q] + dissten[q + plane]);
    const float den = (cpdcv * cvm) * (pi0[k] + ppi[q]);
    thten1[q] = thten1[q] + epsd / den;
  }
  return 0;
}
