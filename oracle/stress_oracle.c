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
 * so signed zeros stay what they are).  Open sides are index clamps (CM1's
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
