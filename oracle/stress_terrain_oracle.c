/* Oracle (test infrastructure only): CPU restatement of the SGS stress and
 * the scalar diffusion of the terrain texts the uniform column runs.
 *
 *   gettau and turbu/turbuz, turbv/turbvz, turbw (four open sides, doimpl = 1,
 *   free-slip bottom and top)
 *       cpu_sgs_stress_tendency_inplace   src/cm1core/cuda_sgs_stress_tendency.py:292-449
 *       (CM1 turb.F:4065-4506, :4536-4545; turbtend.F:1052-2885)
 *   turbs of theta ((th0 - 300) + tha) and numq moisture rows, no surface flux
 *       cpu_gm1_scalar_turbulence_inplace src/cm1core/cuda_gm1_scalar_turbulence.py:230-430
 *       (turbtend.F:18-434, :442-692; solve1.F:1169-1227)
 *
 * Binary32 one operation at a time in the twins' statement order (built with
 * -ffp-contract=off); open sides are index clamps (the twins' edge padding).
 * Shapes as gm1b_terrain_stress_arrays / gm1b_terrain_scalar_turbulence_arrays
 * declare them; the tendencies are ADDED into uten/vten/wten (wten on faces
 * 1..nk-1), thten and the first numq rows of qten.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include "real.h"

#define I3(k, j, i, ny, nx) ((((int64_t)(k)) * (ny) + (j)) * (nx) + (i))

static int cl(int x, int n) { return x < 0 ? 0 : (x >= n ? n - 1 : x); }
/* a (.., nj, ni) carrier at a clamped column; a 2-D (nj, ni) one at k = 0 */
static float cell3(const float* a, int k, int j, int i, int nj, int ni) { return a[I3(k, cl(j, nj), cl(i, ni), nj, ni)]; }
static float cell2(const float* a, int j, int i, int nj, int ni) { return a[(int64_t)cl(j, nj) * ni + cl(i, ni)]; }

/* the face-level average of a mass carrier at a clamped column, with the
 * second-order extrapolation at the bottom and top faces */
static float atw_c(const float* a, int f, int j, int i, int nk, int nj, int ni) {
  if (f == 0) return (1.875f * cell3(a, 0, j, i, nj, ni) + (-1.25f) * cell3(a, 1, j, i, nj, ni)) + 0.375f * cell3(a, 2, j, i, nj, ni);
  if (f == nk)
    return (1.875f * cell3(a, nk - 1, j, i, nj, ni) + (-1.25f) * cell3(a, nk - 2, j, i, nj, ni)) +
           0.375f * cell3(a, nk - 3, j, i, nj, ni);
  return 0.5f * (cell3(a, f - 1, j, i, nj, ni) + cell3(a, f, j, i, nj, ni));
}
/* the same on a t12-shaped (nk, nj+1, ni+1) carrier at corner (jf, iface) */
static float atw_xy(const float* a, int f, int jf, int iface, int nk, int nj, int ni) {
  const int ny = nj + 1, nx = ni + 1;
  if (f == 0) return (1.875f * a[I3(0, jf, iface, ny, nx)] + (-1.25f) * a[I3(1, jf, iface, ny, nx)]) + 0.375f * a[I3(2, jf, iface, ny, nx)];
  if (f == nk)
    return (1.875f * a[I3(nk - 1, jf, iface, ny, nx)] + (-1.25f) * a[I3(nk - 2, jf, iface, ny, nx)]) +
           0.375f * a[I3(nk - 3, jf, iface, ny, nx)];
  return 0.5f * (a[I3(f - 1, jf, iface, ny, nx)] + a[I3(f, jf, iface, ny, nx)]);
}

int oracle_terrain_gettau(int ni, int nj, int nk, const float* s11, const float* s22, const float* s33,
                          const float* s12, const float* s13, const float* s23, const float* kmh, const float* kmv,
                          float* t11, float* t22, float* t33, float* t12, float* t13, float* t23) {
  if (ni < 3 || nj < 3 || nk < 3) return -1;
  for (int k = 0; k < nk; ++k) {
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const int64_t p = I3(k, j, i, nj, ni);
        const float tem = kmh[p] + kmh[I3(k + 1, j, i, nj, ni)];
        t11[p] = s11[p] * tem;
        t22[p] = s22[p] * tem;
        t33[p] = s33[p] * tem;
      }
    for (int jf = 0; jf <= nj; ++jf)
      for (int iface = 0; iface <= ni; ++iface) {
        float total = 0.0f;
        for (int kf = k; kf <= k + 1; ++kf)
          for (int jj = jf - 1; jj <= jf; ++jj)
            for (int ii = iface - 1; ii <= iface; ++ii) total = total + cell3(kmh, kf, jj, ii, nj, ni);
        const int64_t q = I3(k, jf, iface, nj + 1, ni + 1);
        t12[q] = s12[q] * (0.25f * total);
      }
  }
  for (int f = 1; f < nk; ++f) {
    for (int j = 0; j < nj; ++j)
      for (int iface = 0; iface <= ni; ++iface)
        t13[I3(f, j, iface, nj, ni + 1)] =
            s13[I3(f, j, iface, nj, ni + 1)] * (cell3(kmv, f, j, iface - 1, nj, ni) + cell3(kmv, f, j, iface, nj, ni));
    for (int jf = 0; jf <= nj; ++jf)
      for (int i = 0; i < ni; ++i)
        t23[I3(f, jf, i, nj + 1, ni)] =
            s23[I3(f, jf, i, nj + 1, ni)] * (cell3(kmv, f, jf - 1, i, nj, ni) + cell3(kmv, f, jf, i, nj, ni));
  }
  for (int64_t q = 0; q < (int64_t)nj * (ni + 1); ++q) {
    t13[q] = t13[(int64_t)nj * (ni + 1) + q];
    t13[(int64_t)nk * nj * (ni + 1) + q] = t13[(int64_t)(nk - 1) * nj * (ni + 1) + q];
  }
  for (int64_t q = 0; q < (int64_t)(nj + 1) * ni; ++q) {
    t23[q] = t23[(int64_t)(nj + 1) * ni + q];
    t23[(int64_t)nk * (nj + 1) * ni + q] = t23[(int64_t)(nk - 1) * (nj + 1) * ni + q];
  }
  return 0;
}

/* one u or v column's implicit solve and tendency: the pair (ja, ia)/(jb,
 * ib), its wind q (stride qs), its t13/t23 (stride ts), h[k] its horizontal
 * terms, rd the horizontal 1/spacing across the pair, rgp the pair's rgz
 * difference (rg_b - rg_a) and the pair's rgz words; out (stride qs). */
static void terrain_uv_column(int nk, int nj, int ni, int ja, int ia, int jb, int ib, const float* q, int64_t qs,
                              const float* top, const float* h, const float* kmv, const float* rho, const float* rf,
                              const float* mh, const float* mf, const float* gz, const float* rgz, const float* w,
                              float rd, float dz, float dt, float* out, float* cp, float* dp, float* sol,
                              float* cross) {
#define PAIR(a, k) (cell3(a, k, ja, ia, nj, ni) + cell3(a, k, jb, ib, nj, ni))
#define WA(k) w[I3(k, cl(ja, nj), cl(ia, ni), nj, ni)]
#define WB(k) w[I3(k, cl(jb, nj), cl(ib, ni), nj, ni)]
  const float rdz = 1.0f / dz, zt = (float)nk * dz;
  const float tema = -0.0625f * (dt * (rdz * rdz)), temc = 0.5f * (dt * rdz), rdt = 0.5f / dt;
  const float rg_a = cell2(rgz, ja, ia, nj, ni), rg_b = cell2(rgz, jb, ib, nj, ni);
  const float gza = cell2(gz, ja, ia, nj, ni), gzb = cell2(gz, jb, ib, nj, ni);
  for (int k = 0; k <= nk; ++k) cross[k] = 0.0f;
  {
    const float rr0 = 1.0f / (0.5f * PAIR(rho, 0)), mhp = PAIR(mh, 0);
    const float r2v = PAIR(kmv, 1) * (PAIR(mf, 1) * (PAIR(rf, 1) * (mhp * rr0)));
    const float cfc = tema * r2v, cfb = 1.0f - cfc;
    const float cfd = q[0] - temc * (top[0] * (mhp * rr0));
    const float inv = 1.0f / cfb;
    cp[0] = -1.0f * (cfc * inv);
    dp[0] = cfd * inv;
  }
  for (int k = 1; k < nk - 1; ++k) {
    const float rr0 = 1.0f / (0.5f * PAIR(rho, k)), common = PAIR(mh, k) * rr0;
    const float r1v = PAIR(kmv, k) * (PAIR(mf, k) * (PAIR(rf, k) * common));
    const float r2v = PAIR(kmv, k + 1) * (PAIR(mf, k + 1) * (PAIR(rf, k + 1) * common));
    const float cfa = tema * r1v, cfc = tema * r2v, cfb = (1.0f - cfa) - cfc;
    const float inv = 1.0f / (cfa * cp[k - 1] + cfb);
    cp[k] = -1.0f * (cfc * inv);
    dp[k] = (q[(int64_t)k * qs] - cfa * dp[k - 1]) * inv;
  }
  for (int k = 1; k < nk; ++k) {
    const float wm = 0.5f * (WB(k) + WB(k + 1)), wl = 0.5f * (WA(k) + WA(k + 1));
    const float grad = (WB(k) * rg_b - WA(k) * rg_a) * rd;
    const float below = 0.5f * (WB(k - 1) + WB(k)) + 0.5f * (WA(k - 1) + WA(k));
    const float terrain =
        0.5f * (((zt - ((float)k + 0.5f) * dz) * (wm + wl) - (zt - ((float)k - 0.5f) * dz) * below) * (rdz * ((rg_b - rg_a) * rd)));
    cross[k] = (grad + terrain) * (0.25f * (PAIR(kmv, k) * (gza * cell3(rf, k, ja, ia, nj, ni) + gzb * cell3(rf, k, jb, ib, nj, ni))));
  }
  {
    const int k = nk - 1;
    const float rr0 = 1.0f / (0.5f * PAIR(rho, k)), mhp = PAIR(mh, k);
    const float r1v = PAIR(kmv, k) * (PAIR(mf, k) * (PAIR(rf, k) * (mhp * rr0)));
    const float cfa = tema * r1v, cfb = 1.0f - cfa;
    const float cfd = q[(int64_t)k * qs] + temc * (top[(int64_t)nk * qs] * (mhp * rr0));
    sol[k] = (cfd - cfa * dp[k - 1]) * (1.0f / (cfa * cp[k - 1] + cfb));
  }
  for (int k = nk - 2; k >= 0; --k) sol[k] = cp[k] * sol[k + 1] + dp[k];
  for (int k = 0; k < nk; ++k) {
    const float rho_p = PAIR(rho, k), mhp = PAIR(mh, k);
    float vert = rho_p * ((sol[k] - q[(int64_t)k * qs]) * rdt);
    vert = vert + ((k + 1 < nk ? cross[k + 1] : 0.0f) - cross[k]) * (rdz * (0.5f * mhp));
    out[(int64_t)k * qs] = out[(int64_t)k * qs] + (h[k] + vert) / (0.5f * rho_p);
  }
#undef PAIR
#undef WA
#undef WB
}

int oracle_terrain_momentum_stress(int ni, int nj, int nk, const float* t11, const float* t22, const float* t33,
                                   const float* t12, const float* t13, const float* t23, const float* kmh,
                                   const float* kmv, const float* rho, const float* rf, const float* mh,
                                   const float* mf, const float* gz, const float* rgz, const float* gzu,
                                   const float* rgzu, const float* gzv, const float* rgzv, const float* gxu,
                                   const float* gyv, const float* u, const float* v, const float* w, float dx,
                                   float dy, float dz, float dt, float* uten, float* vten, float* wten) {
  if (ni < 3 || nj < 3 || nk < 3) return -1;
  const float rdx = 1.0f / dx, rdy = 1.0f / dy, rdz = 1.0f / dz, zt = (float)nk * dz;
  float* buf = malloc(sizeof(float) * 5 * (size_t)(nk + 1));
  if (!buf) return -2;
  float *h = buf, *cp = buf + (nk + 1), *dp = buf + 2 * (nk + 1), *sol = buf + 3 * (nk + 1), *cross = buf + 4 * (nk + 1);
  const int ux = ni + 1, vy = nj + 1;
  /* turbu/turbuz: one column per u point (j, iface) */
  for (int j = 0; j < nj; ++j)
    for (int iface = 0; iface <= ni; ++iface) {
      const int left = iface - 1, right = iface;
      const float rg_l = cell2(rgz, j, left, nj, ni), rg_r = cell2(rgz, j, right, nj, ni);
      const float g = gzu[j * ux + iface];
      const float r1 = 0.25f * ((cell2(rgz, j - 1, left, nj, ni) + cell2(rgz, j, right, nj, ni)) +
                                (cell2(rgz, j, left, nj, ni) + cell2(rgz, j - 1, right, nj, ni)));
      const float r2 = 0.25f * ((cell2(rgz, j + 1, left, nj, ni) + cell2(rgz, j, right, nj, ni)) +
                                (cell2(rgz, j, left, nj, ni) + cell2(rgz, j + 1, right, nj, ni)));
      for (int k = 0; k < nk; ++k) {
        const float x = g * ((cell3(t11, k, j, right, nj, ni) * rg_r - cell3(t11, k, j, left, nj, ni) * rg_l) * rdx);
        const float up = gxu[I3(k + 1, j, iface, nj, ux)] * (atw_c(t11, k + 1, j, left, nk, nj, ni) + atw_c(t11, k + 1, j, right, nk, nj, ni));
        const float lo = gxu[I3(k, j, iface, nj, ux)] * (atw_c(t11, k, j, left, nk, nj, ni) + atw_c(t11, k, j, right, nk, nj, ni));
        float hx = x + 0.5f * ((up - lo) * rdz);
        const float y = g * ((t12[I3(k, j + 1, iface, vy, ux)] * r2 - t12[I3(k, j, iface, vy, ux)] * r1) * rdy);
        const float su = (zt - (float)(k + 1) * dz) * (atw_xy(t12, k + 1, j, iface, nk, nj, ni) + atw_xy(t12, k + 1, j + 1, iface, nk, nj, ni));
        const float sl = (zt - (float)k * dz) * (atw_xy(t12, k, j, iface, nk, nj, ni) + atw_xy(t12, k, j + 1, iface, nk, nj, ni));
        float hy = y + 0.5f * ((su - sl) * (g * ((r2 - r1) * (rdy * rdz))));
        if (iface == 0 || iface == ni) hx = 0.0f;
        if (j == 0 || j == nj - 1) hy = 0.0f;
        h[k] = hx + hy;
      }
      terrain_uv_column(nk, nj, ni, j, left, j, right, &u[I3(0, j, iface, nj, ux)], (int64_t)nj * ux,
                        &t13[I3(0, j, iface, nj, ux)], h, kmv, rho, rf, mh, mf, gz, rgz, w, rdx, dz, dt,
                        &uten[I3(0, j, iface, nj, ux)], cp, dp, sol, cross);
    }
  /* turbv/turbvz: one column per v point (jface, i) */
  for (int jface = 0; jface <= nj; ++jface)
    for (int i = 0; i < ni; ++i) {
      const int south = jface - 1, north = jface;
      const float g = gzv[jface * ni + i];
      const float r1 = 0.25f * ((cell2(rgz, south, i - 1, nj, ni) + cell2(rgz, north, i, nj, ni)) +
                                (cell2(rgz, north, i - 1, nj, ni) + cell2(rgz, south, i, nj, ni)));
      const float r2 = 0.25f * ((cell2(rgz, south, i + 1, nj, ni) + cell2(rgz, north, i, nj, ni)) +
                                (cell2(rgz, north, i + 1, nj, ni) + cell2(rgz, south, i, nj, ni)));
      const float rg_s = cell2(rgz, south, i, nj, ni), rg_n = cell2(rgz, north, i, nj, ni);
      for (int k = 0; k < nk; ++k) {
        const float x = g * ((t12[I3(k, jface, i + 1, vy, ux)] * r2 - t12[I3(k, jface, i, vy, ux)] * r1) * rdx);
        const float su = (zt - (float)(k + 1) * dz) * (atw_xy(t12, k + 1, jface, i, nk, nj, ni) + atw_xy(t12, k + 1, jface, i + 1, nk, nj, ni));
        const float sl = (zt - (float)k * dz) * (atw_xy(t12, k, jface, i, nk, nj, ni) + atw_xy(t12, k, jface, i + 1, nk, nj, ni));
        float hx = x + 0.5f * ((su - sl) * (g * ((r2 - r1) * (rdx * rdz))));
        const float y = g * ((cell3(t22, k, north, i, nj, ni) * rg_n - cell3(t22, k, south, i, nj, ni) * rg_s) * rdy);
        const float up = gyv[I3(k + 1, jface, i, vy, ni)] * (atw_c(t22, k + 1, south, i, nk, nj, ni) + atw_c(t22, k + 1, north, i, nk, nj, ni));
        const float lo = gyv[I3(k, jface, i, vy, ni)] * (atw_c(t22, k, south, i, nk, nj, ni) + atw_c(t22, k, north, i, nk, nj, ni));
        float hy = y + 0.5f * ((up - lo) * rdz);
        if (i == 0 || i == ni - 1) hx = 0.0f;
        if (jface == 0 || jface == nj) hy = 0.0f;
        h[k] = hx + hy;
      }
      terrain_uv_column(nk, nj, ni, south, i, north, i, &v[I3(0, jface, i, vy, ni)], (int64_t)vy * ni,
                        &t23[I3(0, jface, i, vy, ni)], h, kmv, rho, rf, mh, mf, gz, rgz, w, rdy, dz, dt,
                        &vten[I3(0, jface, i, vy, ni)], cp, dp, sol, cross);
    }
  /* turbw with its implicit solve on faces 1..nk-1 */
  {
    const float tema = -1.0f * (dt * (rdz * rdz)), temc = dt * rdz, rdt = 1.0f / dt;
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
#define T13(f, ii) t13[I3(f, j, ii, nj, ux)]
#define T23(f, jj) t23[I3(f, jj, i, vy, ni)]
#define PF(a, f) a[I3(f, j, i, nj, ni)]
        const float g = gz[j * ni + i];
        for (int f = 1; f < nk; ++f) {
          const float d1 = 0.25f * ((T13(f + 1, i) + T13(f + 1, i + 1)) + (T13(f, i) + T13(f, i + 1)));
          const float d0 = 0.25f * ((T13(f, i) + T13(f, i + 1)) + (T13(f - 1, i) + T13(f - 1, i + 1)));
          float x = g * ((T13(f, i + 1) * rgzu[j * ux + i + 1] - T13(f, i) * rgzu[j * ux + i]) * rdx);
          x = x + ((zt - ((float)f + 0.5f) * dz) * d1 - (zt - ((float)f - 0.5f) * dz) * d0) *
                      (g * ((rgzu[j * ux + i + 1] - rgzu[j * ux + i]) * (rdx * rdz)));
          const float e1 = 0.25f * ((T23(f + 1, j) + T23(f + 1, j + 1)) + (T23(f, j) + T23(f, j + 1)));
          const float e0 = 0.25f * ((T23(f, j) + T23(f, j + 1)) + (T23(f - 1, j) + T23(f - 1, j + 1)));
          float y = g * ((T23(f, j + 1) * rgzv[(j + 1) * ni + i] - T23(f, j) * rgzv[j * ni + i]) * rdy);
          y = y + ((zt - ((float)f + 0.5f) * dz) * e1 - (zt - ((float)f - 0.5f) * dz) * e0) *
                      (g * ((rgzv[(j + 1) * ni + i] - rgzv[j * ni + i]) * (rdy * rdz)));
          h[f] = (i == 0 || i == ni - 1 ? 0.0f : x) + (j == 0 || j == nj - 1 ? 0.0f : y);
        }
        {
          const int f = 1;
          const float rrf = PF(mf, f) / PF(rf, f);
          const float r2v = (PF(kmh, f) + PF(kmh, f + 1)) * (PF(mh, f) * (PF(rho, f) * rrf));
          const float cfc = tema * r2v, cfb = 1.0f - cfc, cfd = PF(w, f) - temc * (PF(t33, 0) * rrf);
          const float inv = 1.0f / cfb;
          cp[0] = -1.0f * (cfc * inv);
          dp[0] = cfd * inv;
        }
        for (int f = 2; f < nk - 1; ++f) {
          const int p = f - 1;
          const float rrf = PF(mf, f) / PF(rf, f);
          const float r1v = (PF(kmh, f - 1) + PF(kmh, f)) * (PF(mh, f - 1) * (PF(rho, f - 1) * rrf));
          const float r2v = (PF(kmh, f) + PF(kmh, f + 1)) * (PF(mh, f) * (PF(rho, f) * rrf));
          const float cfa = tema * r1v, cfc = tema * r2v, cfb = (1.0f - cfa) - cfc;
          const float inv = 1.0f / (cfa * cp[p - 1] + cfb);
          cp[p] = -1.0f * (cfc * inv);
          dp[p] = (PF(w, f) - cfa * dp[p - 1]) * inv;
        }
        {
          const int f = nk - 1, p = nk - 2;
          const float rrf = PF(mf, f) / PF(rf, f);
          const float r1v = (PF(kmh, f - 1) + PF(kmh, f)) * (PF(mh, f - 1) * (PF(rho, f - 1) * rrf));
          const float cfa = tema * r1v, cfb = 1.0f - cfa, cfd = PF(w, f) + temc * (PF(t33, nk - 1) * rrf);
          sol[p] = (cfd - cfa * dp[p - 1]) * (1.0f / (cfa * cp[p - 1] + cfb));
        }
        for (int p = nk - 3; p >= 0; --p) sol[p] = cp[p] * sol[p + 1] + dp[p];
        for (int f = 1; f < nk; ++f) {
          const float vert = PF(rf, f) * ((sol[f - 1] - PF(w, f)) * rdt);
          wten[I3(f, j, i, nj, ni)] = wten[I3(f, j, i, nj, ni)] + (h[f] + vert) / PF(rf, f);
        }
#undef T13
#undef T23
#undef PF
      }
  }
  free(buf);
  return 0;
}

/* ------------------------------------------------------------------------
 * turbs on the terrain texts (one scalar at a time, as the twin) */
typedef struct {
  int ni, nj, nk;
  const float *th0, *tha, *q;
} tsrc;

static float tsv(const tsrc* s, int k, int j, int i) {
  const int64_t p = I3(k, cl(j, s->nj), cl(i, s->ni), s->nj, s->ni);
  return s->q ? s->q[p] : (s->th0[k] - 300.0f) + s->tha[p];
}
/* the scalar at w face f of a clamped column: the twin's _at_w */
static float tsw(const tsrc* s, int f, int j, int i) {
  const int nk = s->nk;
  if (f == 0) return (1.875f * tsv(s, 0, j, i) + (-1.25f) * tsv(s, 1, j, i)) + 0.375f * tsv(s, 2, j, i);
  if (f == nk) return (1.875f * tsv(s, nk - 1, j, i) + (-1.25f) * tsv(s, nk - 2, j, i)) + 0.375f * tsv(s, nk - 3, j, i);
  return 0.5f * tsv(s, f - 1, j, i) + 0.5f * tsv(s, f, j, i);
}
static float interp_w(const float* col, int64_t stride, int f, int nk) {
  if (f == 0) return (1.875f * col[0] + (-1.25f) * col[stride]) + 0.375f * col[2 * stride];
  if (f == nk) return (1.875f * col[(nk - 1) * stride] + (-1.25f) * col[(nk - 2) * stride]) + 0.375f * col[(nk - 3) * stride];
  return 0.5f * col[(f - 1) * stride] + 0.5f * col[f * stride];
}

static void terrain_turbs_one(const tsrc* s, const float* rho, const float* rr, const float* rf, const float* mh,
                              const float* mf, const float* khh, const float* khv, const float* gz, const float* rgz,
                              const float* rgzu, const float* rgzv, const float* gx, const float* gxu,
                              const float* gy, const float* gyv, float dx, float dy, float dz, float dt,
                              float* target, float* fx, float* fy, float* cp, float* dp) {
  const int ni = s->ni, nj = s->nj, nk = s->nk, ux = ni + 1, vy = nj + 1;
  const float rdx = 1.0f / dx, rdy = 1.0f / dy, rdz = 1.0f / dz;
  for (int k = 0; k < nk; ++k) {
    for (int j = 0; j < nj; ++j)
      for (int face = 0; face <= ni; ++face) {
        const int il = face - 1, ir = face; /* real columns either side */
        const float den = cell2(gz, j, ir, nj, ni) * cell3(rho, k, j, ir, nj, ni) + cell2(gz, j, il, nj, ni) * cell3(rho, k, j, il, nj, ni);
        const float dif = (cell3(khh, k, j, ir, nj, ni) + cell3(khh, k, j, il, nj, ni)) +
                          (cell3(khh, k + 1, j, ir, nj, ni) + cell3(khh, k + 1, j, il, nj, ni));
        const float hor = (tsv(s, k, j, ir) * cell2(rgz, j, ir, nj, ni) - tsv(s, k, j, il) * cell2(rgz, j, il, nj, ni)) * rdx;
        const float up = gxu[I3(k + 1, j, face, nj, ux)] * (tsw(s, k + 1, j, ir) + tsw(s, k + 1, j, il));
        const float lo = gxu[I3(k, j, face, nj, ux)] * (tsw(s, k, j, ir) + tsw(s, k, j, il));
        const float ter = ((0.5f * (up - lo)) * rdz) * rgzu[j * ux + face];
        fx[I3(k, j, face, nj, ux)] = ((-0.125f * den) * dif) * (hor + ter);
      }
    for (int face = 0; face <= nj; ++face)
      for (int i = 0; i < ni; ++i) {
        const int js = face - 1, jn = face;
        const float den = cell2(gz, jn, i, nj, ni) * cell3(rho, k, jn, i, nj, ni) + cell2(gz, js, i, nj, ni) * cell3(rho, k, js, i, nj, ni);
        const float dif = (cell3(khh, k, jn, i, nj, ni) + cell3(khh, k, js, i, nj, ni)) +
                          (cell3(khh, k + 1, jn, i, nj, ni) + cell3(khh, k + 1, js, i, nj, ni));
        const float hor = (tsv(s, k, jn, i) * cell2(rgz, jn, i, nj, ni) - tsv(s, k, js, i) * cell2(rgz, js, i, nj, ni)) * rdy;
        const float up = gyv[I3(k + 1, face, i, vy, ni)] * (tsw(s, k + 1, jn, i) + tsw(s, k + 1, js, i));
        const float lo = gyv[I3(k, face, i, vy, ni)] * (tsw(s, k, jn, i) + tsw(s, k, js, i));
        const float ter = ((0.5f * (up - lo)) * rdz) * rgzv[face * ni + i];
        fy[I3(k, face, i, vy, ni)] = ((-0.125f * den) * dif) * (hor + ter);
      }
  }
  const float rdt = 1.0f / dt, tema = (((-1.0f * dt) * 1.0f) * rdz) * rdz, temb = ((dt * 0.0f) * rdz) * rdz;
  const float temc = dt * rdz;
  const int64_t zu = (int64_t)nj * ux, zv = (int64_t)vy * ni;
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i < ni; ++i) {
#define SC(k) tsv(s, k, j, i)
#define COEF(F, K) ((((khv[I3(F, j, i, nj, ni)] * mf[I3(F, j, i, nj, ni)]) * rf[I3(F, j, i, nj, ni)]) * mh[I3(K, j, i, nj, ni)]) * rr[I3(K, j, i, nj, ni)])
      float r2 = COEF(1, 0);
      float cfc = tema * r2, cfb = 1.0f - cfc;
      float ex = (-r2) * SC(0) + r2 * SC(1);
      float bc = ((temc * 0.0f) * mh[I3(0, j, i, nj, ni)]) * rr[I3(0, j, i, nj, ni)];
      float cfd = (SC(0) + temb * ex) + bc;
      float tem = 1.0f / cfb;
      cp[0] = (-cfc) * tem;
      dp[0] = cfd * tem;
      for (int k = 1; k < nk - 1; ++k) {
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
      const int kt = nk - 1;
      const float r1 = COEF(kt, kt), cfa = tema * r1;
      cfb = 1.0f - cfa;
      ex = r1 * SC(kt - 1) - r1 * SC(kt);
      bc = ((temc * 0.0f) * mh[I3(kt, j, i, nj, ni)]) * rr[I3(kt, j, i, nj, ni)];
      cfd = (SC(kt) + temb * ex) - bc;
      tem = 1.0f / (cfa * cp[kt - 1] + cfb);
      float sol = (cfd - cfa * dp[kt - 1]) * tem;
      const float g = gz[j * ni + i];
      for (int kk = nk - 1; kk >= 0; --kk) {
        if (kk != nk - 1) sol = cp[kk] * sol + dp[kk];
        const int64_t m = I3(kk, j, i, nj, ni);
        const float turbz = (rho[m] * (sol - SC(kk))) * rdt;
        const float right = fx[I3(kk, j, i + 1, nj, ux)] * rgzu[j * ux + i + 1], left = fx[I3(kk, j, i, nj, ux)] * rgzu[j * ux + i];
        const float tx0 = ((-g) * (right - left)) * rdx;
        const float* cxi = &fx[I3(0, j, i, nj, ux)];
        const float upx = gx[I3(kk + 1, j, i, nj, ni)] * (interp_w(cxi, zu, kk + 1, nk) + interp_w(cxi + 1, zu, kk + 1, nk));
        const float lox = gx[I3(kk, j, i, nj, ni)] * (interp_w(cxi, zu, kk, nk) + interp_w(cxi + 1, zu, kk, nk));
        float tx = tx0 + ((-(upx - lox)) * 0.5f) * rdz;
        if (i == 0 || i == ni - 1) tx = 0.0f;
        const float north = fy[I3(kk, j + 1, i, vy, ni)] * rgzv[(j + 1) * ni + i], south = fy[I3(kk, j, i, vy, ni)] * rgzv[j * ni + i];
        const float ty0 = ((-g) * (north - south)) * rdy;
        const float* cyj = &fy[I3(0, j, i, vy, ni)];
        const float upy = gy[I3(kk + 1, j, i, nj, ni)] * (interp_w(cyj, zv, kk + 1, nk) + interp_w(cyj + ni, zv, kk + 1, nk));
        const float loy = gy[I3(kk, j, i, nj, ni)] * (interp_w(cyj, zv, kk, nk) + interp_w(cyj + ni, zv, kk, nk));
        float ty = ty0 + ((-(upy - loy)) * 0.5f) * rdz;
        if (j == 0 || j == nj - 1) ty = 0.0f;
        target[m] = target[m] + ((tx + ty) + turbz) * rr[m];
      }
#undef SC
#undef COEF
    }
}

int oracle_terrain_scalar_turbulence(int ni, int nj, int nk, int numq, const float* th0, const float* tha,
                                     const float* qa, const float* rho, const float* rr, const float* rf,
                                     const float* mh, const float* mf, const float* khh, const float* khv,
                                     const float* gz, const float* rgz, const float* rgzu, const float* rgzv,
                                     const float* gx, const float* gxu, const float* gy, const float* gyv, float dx,
                                     float dy, float dz, float dt, float* thten, float* qten) {
  if (ni < 3 || nj < 3 || nk < 3 || numq < 0) return -1;
  const int64_t n = (int64_t)ni * nj * nk;
  float* fx = malloc(sizeof(float) * (size_t)nk * nj * (ni + 1));
  float* fy = malloc(sizeof(float) * (size_t)nk * (nj + 1) * ni);
  float* cd = malloc(sizeof(float) * 2 * (size_t)nk);
  if (!fx || !fy || !cd) return -2;
  tsrc s = {ni, nj, nk, th0, tha, NULL};
  terrain_turbs_one(&s, rho, rr, rf, mh, mf, khh, khv, gz, rgz, rgzu, rgzv, gx, gxu, gy, gyv, dx, dy, dz, dt, thten, fx,
                    fy, cd, cd + nk);
  for (int q = 0; q < numq; ++q) {
    s.q = qa + q * n;
    terrain_turbs_one(&s, rho, rr, rf, mh, mf, khh, khv, gz, rgz, rgzu, rgzv, gx, gxu, gy, gyv, dx, dy, dz, dt,
                      qten + q * n, fx, fy, cd, cd + nk);
  }
  free(fx);
  free(fy);
  free(cd);
  return 0;
}
