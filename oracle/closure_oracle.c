/* Oracle (test infrastructure only): CPU restatement of the two closure
 * inputs of the TKE source, deformation and moist N^2.
 *
 *   calcdef, Cartesian terrain branch, four open sides
 *       cpu_terrain_deformation_inplace   src/cm1core/cuda_terrain_deformation.py:234-736
 *       (CM1 turb.F:4711-5423)
 *   calcnm, six-species ice-aware branch
 *       cpu_moist_nm_inplace              src/cm1core/cuda_moist_nm.py:292-396
 *       (CM1 turb.F:5432-5685; rslf/rsif cm1libs.F:16-115)
 *
 * Binary32 one operation at a time (built with -ffp-contract=off); expf/logf
 * are the C library's.  Shapes (C order):
 *   u (nk, nj, ni+1), v (nk, nj+1, ni), w/rf/c1/c2/gx/gy/mf/defv/defh/nm
 *   (nk+1, nj, ni), rho/prs/pp3d/th3d (nk, nj, ni), q3d (6, nk, nj, ni),
 *   gz/rgz (nj, ni), rgzu (nj, ni+1), rgzv (nj+1, ni), pi0/th0 (nk).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include "real.h"

#define I3(k, j, i, ny, nx) ((((int64_t)(k)) * (ny) + (j)) * (nx) + (i))

static int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

/* face-level average of a u- or v-shaped field at column (j, i) of a layout
 * with row length nx and rows per level ny (cuda_terrain_deformation.py:210) */
static float atw(const float* q, int kf, int j, int i, int nk, int ny, int nx) {
  if (kf == 0) {
    float r = 1.875f * q[I3(0, j, i, ny, nx)];
    r = r + (-1.25f) * q[I3(1, j, i, ny, nx)];
    return r + 0.375f * q[I3(2, j, i, ny, nx)];
  }
  if (kf == nk) {
    float r = 1.875f * q[I3(nk - 1, j, i, ny, nx)];
    r = r + (-1.25f) * q[I3(nk - 2, j, i, ny, nx)];
    return r + 0.375f * q[I3(nk - 3, j, i, ny, nx)];
  }
  return 0.5f * (q[I3(kf - 1, j, i, ny, nx)] + q[I3(kf, j, i, ny, nx)]);
}

/* the six strain carriers rho*Sij of the terrain calcdef (its mass and face
 * passes, cpu_terrain_deformation_inplace): s11/s22/s33 (nk, nj, ni), s12
 * (nk, nj+1, ni+1) at every corner from the nearest interior corner, s13
 * (nk+1, nj, ni+1) and s23 (nk+1, nj+1, ni) on face levels 1..nk-1 (levels
 * 0 and nk left as they are) */
int oracle_terrain_strain(int ni, int nj, int nk, const float* u, const float* v, const float* w, const float* rho,
                          const float* rf, const float* gz, const float* rgz, const float* rgzu, const float* rgzv,
                          const float* gx, const float* gy, float dx, float dy, float dz, float* s11, float* s22,
                          float* s33, float* s12, float* s13, float* s23) {
  if (ni < 3 || nj < 3 || nk < 3) return -1;
  const float rdx = 1.0f / dx, rdy = 1.0f / dy, rds = 1.0f / dz;
  const float half = 0.5f, quarter = 0.25f;
  const float zt = (float)nk * dz;
  const int ux = ni + 1, vy = nj + 1;
  for (int k = 0; k < nk; ++k) {
    const float sig_lo = (float)k * dz, sig_hi = (float)(k + 1) * dz;
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const int64_t p = I3(k, j, i, nj, ni);
        const float g = gz[j * ni + i];
        float hor = g * (u[I3(k, j, i + 1, nj, ux)] * rgzu[j * ux + i + 1] - u[I3(k, j, i, nj, ux)] * rgzu[j * ux + i]);
        hor = hor * rdx;
        float up = gx[I3(k + 1, j, i, nj, ni)] * (atw(u, k + 1, j, i, nk, nj, ux) + atw(u, k + 1, j, i + 1, nk, nj, ux));
        float lo = gx[I3(k, j, i, nj, ni)] * (atw(u, k, j, i, nk, nj, ux) + atw(u, k, j, i + 1, nk, nj, ux));
        float vert = ((up - lo) * half) * rds;
        s11[p] = (hor + vert) * rho[p];
        hor = g * (v[I3(k, j + 1, i, vy, ni)] * rgzv[(j + 1) * ni + i] - v[I3(k, j, i, vy, ni)] * rgzv[j * ni + i]);
        hor = hor * rdy;
        up = gy[I3(k + 1, j, i, nj, ni)] * (atw(v, k + 1, j, i, nk, vy, ni) + atw(v, k + 1, j + 1, i, nk, vy, ni));
        lo = gy[I3(k, j, i, nj, ni)] * (atw(v, k, j, i, nk, vy, ni) + atw(v, k, j + 1, i, nk, vy, ni));
        vert = ((up - lo) * half) * rds;
        s22[p] = (hor + vert) * rho[p];
        s33[p] = (((w[I3(k + 1, j, i, nj, ni)] - w[I3(k, j, i, nj, ni)]) * rds) * g) * rho[p];
      }
    for (int jc = 0; jc <= nj; ++jc) {
      const int jj = clampi(jc, 1, nj - 1);
      for (int ic = 0; ic <= ni; ++ic) {
        const int ii = clampi(ic, 1, ni - 1);
        float r1 = (rho[I3(k, jj - 1, ii - 1, nj, ni)] * gz[(jj - 1) * ni + ii - 1] +
                    rho[I3(k, jj, ii, nj, ni)] * gz[jj * ni + ii]) +
                   (rho[I3(k, jj, ii - 1, nj, ni)] * gz[jj * ni + ii - 1] +
                    rho[I3(k, jj - 1, ii, nj, ni)] * gz[(jj - 1) * ni + ii]);
        r1 = quarter * r1;
        const float x1 =
            (r1 * (u[I3(k, jj, ii, nj, ux)] * rgzu[jj * ux + ii] - u[I3(k, jj - 1, ii, nj, ux)] * rgzu[(jj - 1) * ux + ii])) *
            rdy;
        const float xu = (zt - sig_hi) * (atw(u, k + 1, jj - 1, ii, nk, nj, ux) + atw(u, k + 1, jj, ii, nk, nj, ux));
        const float xl = (zt - sig_lo) * (atw(u, k, jj - 1, ii, nk, nj, ux) + atw(u, k, jj, ii, nk, nj, ux));
        const float x2 = ((((half * (xu - xl)) * rds) * r1) * (rgzu[jj * ux + ii] - rgzu[(jj - 1) * ux + ii])) * rdy;
        const float y1 =
            (r1 * (v[I3(k, jj, ii, vy, ni)] * rgzv[jj * ni + ii] - v[I3(k, jj, ii - 1, vy, ni)] * rgzv[jj * ni + ii - 1])) *
            rdx;
        const float yu = (zt - sig_hi) * (atw(v, k + 1, jj, ii - 1, nk, vy, ni) + atw(v, k + 1, jj, ii, nk, vy, ni));
        const float yl = (zt - sig_lo) * (atw(v, k, jj, ii - 1, nk, vy, ni) + atw(v, k, jj, ii, nk, vy, ni));
        const float y2 = ((((half * (yu - yl)) * rds) * r1) * (rgzv[jj * ni + ii] - rgzv[jj * ni + ii - 1])) * rdx;
        s12[I3(k, jc, ic, nj + 1, ni + 1)] = half * ((x1 + x2) + (y1 + y2));
      }
    }
  }
  for (int kf = 1; kf < nk; ++kf) {
    const float sig_l = ((float)kf - half) * dz, sig_u = ((float)kf + half) * dz;
    for (int j = 0; j < nj; ++j)
      for (int ic = 0; ic <= ni; ++ic) {
        const int il = ic - 1 < 0 ? 0 : ic - 1, ir = ic < ni - 1 ? ic : ni - 1;
        const float du = (u[I3(kf, j, ic, nj, ux)] - u[I3(kf - 1, j, ic, nj, ux)]) * rds;
        const float hw =
            (w[I3(kf, j, ir, nj, ni)] * rgz[j * ni + ir] - w[I3(kf, j, il, nj, ni)] * rgz[j * ni + il]) * rdx;
        const float wu = (zt - sig_u) * (half * (w[I3(kf, j, ir, nj, ni)] + w[I3(kf + 1, j, ir, nj, ni)]) +
                                         half * (w[I3(kf, j, il, nj, ni)] + w[I3(kf + 1, j, il, nj, ni)]));
        const float wl = (zt - sig_l) * (half * (w[I3(kf - 1, j, ir, nj, ni)] + w[I3(kf, j, ir, nj, ni)]) +
                                         half * (w[I3(kf - 1, j, il, nj, ni)] + w[I3(kf, j, il, nj, ni)]));
        const float terrain = (((half * rds) * (wu - wl)) * (rgz[j * ni + ir] - rgz[j * ni + il])) * rdx;
        const float strain = half * ((du + hw) + terrain);
        const float density =
            half * (gz[j * ni + il] * rf[I3(kf, j, il, nj, ni)] + gz[j * ni + ir] * rf[I3(kf, j, ir, nj, ni)]);
        s13[I3(kf, j, ic, nj, ni + 1)] = strain * density;
      }
    for (int jc = 0; jc <= nj; ++jc) {
      const int jb = jc - 1 < 0 ? 0 : jc - 1, jt = jc < nj - 1 ? jc : nj - 1;
      for (int i = 0; i < ni; ++i) {
        const float dv = (v[I3(kf, jc, i, vy, ni)] - v[I3(kf - 1, jc, i, vy, ni)]) * rds;
        const float hw =
            (w[I3(kf, jt, i, nj, ni)] * rgz[jt * ni + i] - w[I3(kf, jb, i, nj, ni)] * rgz[jb * ni + i]) * rdy;
        const float wu = (zt - sig_u) * (half * (w[I3(kf, jt, i, nj, ni)] + w[I3(kf + 1, jt, i, nj, ni)]) +
                                         half * (w[I3(kf, jb, i, nj, ni)] + w[I3(kf + 1, jb, i, nj, ni)]));
        const float wl = (zt - sig_l) * (half * (w[I3(kf - 1, jt, i, nj, ni)] + w[I3(kf, jt, i, nj, ni)]) +
                                         half * (w[I3(kf - 1, jb, i, nj, ni)] + w[I3(kf, jb, i, nj, ni)]));
        const float terrain = (((half * rds) * (wu - wl)) * (rgz[jt * ni + i] - rgz[jb * ni + i])) * rdy;
        const float strain = half * ((dv + hw) + terrain);
        const float density =
            half * (gz[jb * ni + i] * rf[I3(kf, jb, i, nj, ni)] + gz[jt * ni + i] * rf[I3(kf, jt, i, nj, ni)]);
        s23[I3(kf, jc, i, nj + 1, ni)] = strain * density;
      }
    }
  }
  return 0;
}

int oracle_calcdef(int ni, int nj, int nk, const float* u, const float* v, const float* w, const float* rho,
                   const float* rf, const float* c1, const float* c2, const float* gz, const float* rgz,
                   const float* rgzu, const float* rgzv, const float* gx, const float* gy, float dx, float dy,
                   float dz, float* defv, float* defh) {
  if (ni < 3 || nj < 3 || nk < 3) return -1;
  const float half = 0.5f, quarter = 0.25f;
  const int64_t ncell = (int64_t)nk * nj * ni;
  float* s11 = calloc(ncell, sizeof(float));
  float* s22 = calloc(ncell, sizeof(float));
  float* s33 = calloc(ncell, sizeof(float));
  float* s12 = calloc((int64_t)nk * (nj + 1) * (ni + 1), sizeof(float));
  float* s13 = calloc((int64_t)(nk + 1) * nj * (ni + 1), sizeof(float));
  float* s23 = calloc((int64_t)(nk + 1) * (nj + 1) * ni, sizeof(float));
  if (!s11 || !s22 || !s33 || !s12 || !s13 || !s23) return -2;
  oracle_terrain_strain(ni, nj, nk, u, v, w, rho, rf, gz, rgz, rgzu, rgzv, gx, gy, dx, dy, dz, s11, s22, s33, s12, s13,
                        s23);
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i < ni; ++i) {
      defv[I3(0, j, i, nj, ni)] = 0.0f;
      defh[I3(0, j, i, nj, ni)] = 0.0f;
      defv[I3(nk, j, i, nj, ni)] = 0.0f;
      defh[I3(nk, j, i, nj, ni)] = 0.0f;
    }
#define SQ(x) ((x) * (x))
  for (int kf = 1; kf < nk; ++kf)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const int64_t p = I3(kf, j, i, nj, ni), lo = I3(kf - 1, j, i, nj, ni), hi = I3(kf, j, i, nj, ni);
        const float a = c1[p], b = c2[p];
        const float t11 = a * SQ(s11[lo]) + b * SQ(s11[hi]);
        const float t22 = a * SQ(s22[lo]) + b * SQ(s22[hi]);
        const float t33 = a * SQ(s33[lo]) + b * SQ(s33[hi]);
        const float* L = s12 + I3(kf - 1, 0, 0, nj + 1, ni + 1);
        const float* H = s12 + I3(kf, 0, 0, nj + 1, ni + 1);
        const int X = ni + 1;
        const float lo12 = (SQ(L[j * X + i]) + SQ(L[(j + 1) * X + i + 1])) + (SQ(L[(j + 1) * X + i]) + SQ(L[j * X + i + 1]));
        const float hi12 = (SQ(H[j * X + i]) + SQ(H[(j + 1) * X + i + 1])) + (SQ(H[(j + 1) * X + i]) + SQ(H[j * X + i + 1]));
        const float t12 = quarter * (a * lo12 + b * hi12);
        const float t13 = half * (SQ(s13[I3(kf, j, i, nj, ni + 1)]) + SQ(s13[I3(kf, j, i + 1, nj, ni + 1)]));
        const float t23 = half * (SQ(s23[I3(kf, j, i, nj + 1, ni)]) + SQ(s23[I3(kf, j + 1, i, nj + 1, ni)]));
        const float rrf = 1.0f / (rf[p] * rf[p]);
        defv[p] = (4.0f * (t13 + t23)) * rrf;
        defh[p] = ((2.0f * ((t11 + t22) + t33)) + 4.0f * t12) * rrf;
      }
#undef SQ
  free(s11);
  free(s22);
  free(s33);
  free(s12);
  free(s13);
  free(s23);
  return 0;
}

/* ---------------------------------------------------------------- calcnm */

typedef struct {
  float g, rd, cp, cpv, cpl, cpi, eps, reps, lv1, lv2, ls1, ls2;
} nm_consts;

static nm_consts nm_constants(void) {
  nm_consts c;
  c.g = 9.81f;
  c.rd = 287.04f;
  const float rv = 461.5f;
  c.cp = 1005.7f;
  c.cpv = 1870.0f;
  c.cpl = 4190.0f;
  c.cpi = 2106.0f;
  const float xlv = 2501000.0f, xls = 2834000.0f, to = 273.15f;
  c.eps = c.rd / rv;
  c.reps = rv / c.rd;
  c.lv1 = xlv + (c.cpl - c.cpv) * to;
  c.lv2 = c.cpl - c.cpv;
  c.ls1 = xls + (c.cpi - c.cpv) * to;
  c.ls2 = c.cpi - c.cpv;
  return c;
}

static float nm_rslf(float p, float t, float eps) {
  const float x = (17.67f * (t - 273.15f)) / (t - 29.65f);
  float es = 611.2f * expf(x);
  const float h = p * 0.5f;
  if (h < es) es = h;
  return (eps * es) / (p - es);
}

static float nm_rsif(float p, float t, float eps) {
  const float x = (21.8745584f * (t - 273.15f)) / (t - 7.66f);
  float es = 611.2f * expf(x);
  const float h = p * 0.5f;
  if (h < es) es = h;
  return (eps * es) / (p - es);
}

static float nm_saturated(const nm_consts* c, float upper_t, float lower_t, float upper_qt, float lower_qt, float tavg,
                          float qtavg, float qvs, float ql, float qi, float qv, float mrdz, int ice) {
  float cpml = c->cp + c->cpv * qv;
  cpml = cpml + c->cpl * ql;
  if (qi != 0.0f) cpml = cpml + c->cpi * qi;
  float lh, drdt, den;
  if (ice) {
    lh = c->ls1 - c->ls2 * tavg;
    drdt = 21.8745584f * (273.15f - 7.66f);
    den = (tavg - 7.66f) * (tavg - 7.66f);
  } else {
    lh = c->lv1 - c->lv2 * tavg;
    drdt = 17.67f * (273.15f - 29.65f);
    den = (tavg - 29.65f) * (tavg - 29.65f);
  }
  drdt = (drdt * qvs) / den;
  float gamma = c->g * (1.0f + qtavg);
  gamma = gamma * (1.0f + (lh * qvs) / (c->rd * tavg));
  gamma = gamma / (cpml + lh * drdt);
  float first = logf(upper_t / lower_t) * mrdz;
  first = first + gamma / tavg;
  float second = tavg * drdt;
  second = second / (c->eps + qvs);
  first = first * (1.0f + second);
  float moist = logf((1.0f + upper_qt) / (1.0f + lower_qt));
  moist = moist * mrdz;
  return c->g * (first - moist);
}

/* counts[4]: saturated, liquid, mixed, ice words */
int oracle_moist_nm(int ni, int nj, int nk, const float* c1, const float* c2, const float* mf, const float* pi0,
                    const float* th0, const float* prs, const float* pp3d, const float* th3d, const float* q3d,
                    float dz, float* nm, float* temperature, float* qt, float* thv, float* qvci, uint8_t* mask,
                    int64_t* counts) {
  if (ni < 1 || nj < 1 || nk < 2) return -1;
  const nm_consts c = nm_constants();
  const float rdz = 1.0f / dz;
  const int64_t cells = (int64_t)nk * nj * ni;
  for (int q = 0; q < 4; ++q) counts[q] = 0;
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const int64_t p = I3(k, j, i, nj, ni);
        const float qv = q3d[p], qc = q3d[cells + p], qi = q3d[3 * cells + p];
        qvci[p] = (qv + qc) + qi;
        float t = 0.0f;
        for (int s = 0; s < 6; ++s) t = t + q3d[s * cells + p];
        qt[p] = t;
        const float theta = th0[k] + th3d[p];
        const float exner = pi0[k] + pp3d[p];
        temperature[p] = theta * exner;
        float tv = theta * (1.0f + c.reps * qv);
        thv[p] = tv / (1.0f + t);
        mask[p] = 0;
      }
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i < ni; ++i) {
      nm[I3(0, j, i, nj, ni)] = 0.0f;
      nm[I3(nk, j, i, nj, ni)] = 0.0f;
      for (int k = 1; k < nk; ++k) {
        const int64_t f = I3(k, j, i, nj, ni), m = I3(k, j, i, nj, ni), l = I3(k - 1, j, i, nj, ni);
        const float mrdz = rdz * mf[f];
        float value = c.g * (logf(thv[m] / thv[l]) * mrdz);
        const float a = c1[f], b = c2[f];
        const float pavg = a * prs[l] + b * prs[m];
        const float tavg = a * temperature[l] + b * temperature[m];
        const float qtavg = a * qt[l] + b * qt[m];
        const float qvciavg = a * qvci[l] + b * qvci[m];
        if (tavg >= 273.15f) {
          const float qvs = nm_rslf(pavg, tavg, c.eps);
          float ql = qvciavg - qvs;
          if (!(ql > 0.0f)) ql = 0.0f; /* max(x, 0) */
          if (ql > 1.0e-10f) {
            float qvv = qvciavg - ql;
            if (!(qvv > 0.0f)) qvv = 0.0f;
            value = nm_saturated(&c, temperature[m], temperature[l], qt[m], qt[l], tavg, qtavg, qvs, ql, 0.0f, qvv,
                                 mrdz, 0);
            mask[m] = 1;
            counts[0]++;
            counts[1]++;
          }
        } else if (tavg <= 233.15f) {
          const float qvs = nm_rsif(pavg, tavg, c.eps);
          float qii = qvciavg - qvs;
          if (!(qii > 0.0f)) qii = 0.0f;
          if (qii > 1.0e-10f) {
            float qvv = qvciavg - qii;
            if (!(qvv > 0.0f)) qvv = 0.0f;
            value = nm_saturated(&c, temperature[m], temperature[l], qt[m], qt[l], tavg, qtavg, qvs, 0.0f, qii, qvv,
                                 mrdz, 1);
            mask[m] = 1;
            counts[0]++;
            counts[3]++;
          }
        } else {
          const float ff = (tavg - 233.15f) / (273.15f - 233.15f);
          const float qvsl = nm_rslf(pavg, tavg, c.eps), qvsi = nm_rsif(pavg, tavg, c.eps);
          const float om = 1.0f - ff;
          const float qvs = ff * qvsl + om * qvsi;
          const float ex = qvciavg - qvs;
          float qii = om * ex;
          if (!(qii > 0.0f)) qii = 0.0f;
          float ql = ff * ex;
          if (!(ql > 0.0f)) ql = 0.0f;
          if (ql + qii > 1.0e-10f) {
            float qvv = (qvciavg - ql) - qii;
            if (!(qvv > 0.0f)) qvv = 0.0f;
            const float nml = nm_saturated(&c, temperature[m], temperature[l], qt[m], qt[l], tavg, qtavg, qvsl, ql, qii,
                                           qvv, mrdz, 0);
            const float nmi = nm_saturated(&c, temperature[m], temperature[l], qt[m], qt[l], tavg, qtavg, qvsi, ql, qii,
                                           qvv, mrdz, 1);
            value = ff * nml + om * nmi;
            mask[m] = 1;
            counts[0]++;
            counts[2]++;
          }
        }
        nm[f] = value;
      }
    }
  return 0;
}

/* calcdef on a flat (terrain_flag=.false.) stretched column, three passes as
 * the reference's texts gm1_flat_calcdef_mass_v1 / _face_v1 / _reduce_v1
 * (src/cm1core/cuda_gm1_flat_stretched_closure.py:76-136; turb.F:4772-4786,
 * :4880-4895, :5361-5385), with the zero fill of defv/defh before them
 * (cuda_cartesian_closure.py:1130-1131).  mhp is the mh profile (nk+2,
 * CM1-indexed: mhp[k+1] belongs to mass level k); mf is the 3-D face array;
 * rdz the coordinate's reference 1/dz.  Open sides are index clamps. */
/* the six strain carriers rho*Sij of the flat calcdef (its mass and face
 * passes): s11/s22/s33 (nk, nj, ni), s12 (nk, nj+1, ni+1) with every corner
 * written (open sides take the nearest interior corner), s13 (nk+1, nj, ni+1)
 * and s23 (nk+1, nj+1, ni) on face levels 1..nk-1 (levels 0 and nk left as
 * they are) */
int oracle_flat_strain(int ni, int nj, int nk, const float* u, const float* v, const float* w, const float* rho,
                       const float* rf, const float* mf, const float* mhp, float dx, float dy, float rdz, float* s11,
                       float* s22, float* s33, float* s12, float* s13, float* s23) {
  if (ni < 3 || nj < 3 || nk < 3) return -1;
  const float rdx = 1.0f / dx, rdy = 1.0f / dy;
  const int ux = ni + 1, vy = nj + 1;
  /* mass pass: s11, s22, s33 at cells, s12 at corners */
  for (int k = 0; k < nk; ++k)
    for (int jc = 0; jc <= nj; ++jc)
      for (int ic = 0; ic <= ni; ++ic) {
        if (ic < ni && jc < nj) {
          const int64_t p = I3(k, jc, ic, nj, ni);
          const float r = rho[p];
          float d = u[I3(k, jc, ic + 1, nj, ux)] - u[I3(k, jc, ic, nj, ux)];
          s11[p] = (r * d) * rdx;
          d = v[I3(k, jc + 1, ic, vy, ni)] - v[I3(k, jc, ic, vy, ni)];
          s22[p] = (r * d) * rdy;
          d = w[I3(k + 1, jc, ic, nj, ni)] - w[I3(k, jc, ic, nj, ni)];
          const float m = rdz * mhp[k + 1];
          s33[p] = (r * d) * m;
        }
        const int ii = clampi(ic, 1, ni - 1), jj = clampi(jc, 1, nj - 1);
        const float x = (u[I3(k, jj, ii, nj, ux)] - u[I3(k, jj - 1, ii, nj, ux)]) * rdy;
        const float y = (v[I3(k, jj, ii, vy, ni)] - v[I3(k, jj, ii - 1, vy, ni)]) * rdx;
        float rs = rho[I3(k, jj - 1, ii - 1, nj, ni)] + rho[I3(k, jj, ii, nj, ni)];
        rs = rs + (rho[I3(k, jj, ii - 1, nj, ni)] + rho[I3(k, jj - 1, ii, nj, ni)]);
        s12[I3(k, jc, ic, vy, ux)] = ((0.5f * (x + y)) * 0.25f) * rs;
      }
  /* face pass: s13 on u-face columns, s23 on v-face rows, face levels 1..nk-1 */
  for (int kf = 1; kf < nk; ++kf)
    for (int jc = 0; jc <= nj; ++jc)
      for (int ic = 0; ic <= ni; ++ic) {
        if (jc < nj) {
          const int il = clampi(ic - 1, 0, ni - 1), ir = clampi(ic, 0, ni - 1);
          const float dw = (w[I3(kf, jc, ir, nj, ni)] - w[I3(kf, jc, il, nj, ni)]) * rdx;
          float du = (u[I3(kf, jc, ic, nj, ux)] - u[I3(kf - 1, jc, ic, nj, ux)]) * rdz;
          du = (du * 0.5f) * (mf[I3(kf, jc, il, nj, ni)] + mf[I3(kf, jc, ir, nj, ni)]);
          const float dens = rf[I3(kf, jc, il, nj, ni)] + rf[I3(kf, jc, ir, nj, ni)];
          s13[I3(kf, jc, ic, nj, ux)] = ((0.5f * (dw + du)) * 0.5f) * dens;
        }
        if (ic < ni) {
          const int js = clampi(jc - 1, 0, nj - 1), jn = clampi(jc, 0, nj - 1);
          const float dw = (w[I3(kf, jn, ic, nj, ni)] - w[I3(kf, js, ic, nj, ni)]) * rdy;
          float dv = (v[I3(kf, jc, ic, vy, ni)] - v[I3(kf - 1, jc, ic, vy, ni)]) * rdz;
          dv = (dv * 0.5f) * (mf[I3(kf, js, ic, nj, ni)] + mf[I3(kf, jn, ic, nj, ni)]);
          const float dens = rf[I3(kf, js, ic, nj, ni)] + rf[I3(kf, jn, ic, nj, ni)];
          s23[I3(kf, jc, ic, vy, ni)] = ((0.5f * (dw + dv)) * 0.5f) * dens;
        }
      }
  return 0;
}

int oracle_flat_calcdef(int ni, int nj, int nk, const float* u, const float* v, const float* w, const float* rho,
                        const float* rf, const float* mf, const float* c1, const float* c2, const float* mhp,
                        float dx, float dy, float rdz, float* defv, float* defh) {
  if (ni < 3 || nj < 3 || nk < 3) return -1;
  const int64_t ncell = (int64_t)nk * nj * ni;
  float* s11 = calloc(ncell, sizeof(float));
  float* s22 = calloc(ncell, sizeof(float));
  float* s33 = calloc(ncell, sizeof(float));
  float* s12 = calloc((int64_t)nk * (nj + 1) * (ni + 1), sizeof(float));
  float* s13 = calloc((int64_t)(nk + 1) * nj * (ni + 1), sizeof(float));
  float* s23 = calloc((int64_t)(nk + 1) * (nj + 1) * ni, sizeof(float));
  if (!s11 || !s22 || !s33 || !s12 || !s13 || !s23) return -2;
  for (int64_t q = 0; q < (int64_t)(nk + 1) * nj * ni; ++q) {
    defv[q] = 0.0f;
    defh[q] = 0.0f;
  }
  const int ux = ni + 1, vy = nj + 1;
  oracle_flat_strain(ni, nj, nk, u, v, w, rho, rf, mf, mhp, dx, dy, rdz, s11, s22, s33, s12, s13, s23);
  /* reduction (the pass both branches share) */
  for (int kf = 1; kf < nk; ++kf)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const int64_t p = I3(kf, j, i, nj, ni), lo = I3(kf - 1, j, i, nj, ni);
        const float a = c1[p], b = c2[p];
        const float t11 = a * (s11[lo] * s11[lo]) + b * (s11[p] * s11[p]);
        const float t22 = a * (s22[lo] * s22[lo]) + b * (s22[p] * s22[p]);
        const float t33 = a * (s33[lo] * s33[lo]) + b * (s33[p] * s33[p]);
        const float l00 = s12[I3(kf - 1, j, i, vy, ux)], l11 = s12[I3(kf - 1, j + 1, i + 1, vy, ux)];
        const float l10 = s12[I3(kf - 1, j + 1, i, vy, ux)], l01 = s12[I3(kf - 1, j, i + 1, vy, ux)];
        const float h00 = s12[I3(kf, j, i, vy, ux)], h11 = s12[I3(kf, j + 1, i + 1, vy, ux)];
        const float h10 = s12[I3(kf, j + 1, i, vy, ux)], h01 = s12[I3(kf, j, i + 1, vy, ux)];
        const float lsum = (l00 * l00 + l11 * l11) + (l10 * l10 + l01 * l01);
        const float hsum = (h00 * h00 + h11 * h11) + (h10 * h10 + h01 * h01);
        const float t12 = 0.25f * (a * lsum + b * hsum);
        const float x0 = s13[I3(kf, j, i, nj, ux)], x1 = s13[I3(kf, j, i + 1, nj, ux)];
        const float y0 = s23[I3(kf, j, i, vy, ni)], y1 = s23[I3(kf, j + 1, i, vy, ni)];
        const float t13 = 0.5f * (x0 * x0 + x1 * x1), t23 = 0.5f * (y0 * y0 + y1 * y1);
        const float rrf = 1.0f / (rf[p] * rf[p]);
        defv[p] = (4.0f * (t13 + t23)) * rrf;
        defh[p] = ((2.0f * ((t11 + t22) + t33)) + 4.0f * t12) * rrf;
      }
  free(s11);
  free(s22);
  free(s33);
  free(s12);
  free(s13);
  free(s23);
  return 0;
}
