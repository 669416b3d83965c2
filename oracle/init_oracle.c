/* Oracle (test infrastructure only): CPU restatement of the CM1 r21.1
 * analytic initial state used by the moist storm configurations.
 *
 *   - Weisman-Klemp (1982) base column, CM1 isnd=5 (base.F:363-450), as the
 *     reference restates it in binary32 in
 *     rust/cm1-state/src/storm_initialization.rs:187-350
 *     (weisman_klemp_column_with_iterations) with the surface words of
 *     :67-80 and rslf of rust/cm1-state/src/idealized_initialization.rs:984.
 *   - iwnd=2 quarter-circle base wind (base.F:2321-2360), reference
 *     storm_initialization.rs:354-389 (analytic_shear_u / analytic_shear_v).
 *   - iinit=1 warm bubble (init3d.F:450-482), reference
 *     rust/cm1-state/src/initial_perturbation.rs:449-466.
 *
 * Arithmetic is binary32 one operation at a time (built with
 * -ffp-contract=off), transcendental calls go to the C library's
 * powf/expf/cosf/sinf/sqrtf as gfortran's do, so the column can be compared
 * word for word with CM1's own output.  Only tests and the benchmark's CPU
 * baseline call this file.
 */
#include <math.h>
#include <stdint.h>
#include "real.h"

/* CM1 constants.F binary32 words */
#define K_G 9.81f
#define K_CP 1005.7f
#define K_RD 287.04f
#define K_RV 461.5f
#define K_P00 100000.0f
/* base.F:369-374 */
#define WK_Z_TROP 12000.0f
#define WK_TH_TROP 343.0f
#define WK_T_TROP 213.0f
#define WK_TH_SFC 300.0f
#define WK_PRS_SFC 100000.0f
#define WK_QV_PBL 0.014f

/* CM1 rslf (Bolton liquid saturation mixing ratio with the p/2 clamp),
 * idealized_initialization.rs:984-989. */
static float oracle_rslf(float p, float t) {
  const float eps = K_RD / K_RV;
  float x = 17.67f * (t - 273.15f);
  x = x / (t - 29.65f);
  float es = 611.2f * expf(x);
  const float half_p = p * 0.5f;
  if (half_p < es) es = half_p;
  return eps * es / (p - es);
}

/* Surface pi, qv and theta_v (base.F:378-380, storm_initialization.rs:67-80). */
void oracle_wk_surface(float out3[3]) {
  const float reps = K_RV / K_RD;
  const float pi = powf(WK_PRS_SFC / K_P00, K_RD / K_CP);
  const float qv = oracle_rslf(WK_PRS_SFC, WK_TH_SFC * pi);
  const float thv = WK_TH_SFC * (1.0f + qv * reps) / (1.0f + qv);
  out3[0] = pi;
  out3[1] = qv;
  out3[2] = thv;
}

/* The isnd=5 column on mass heights zh[0..nk) (m, strictly increasing above
 * 0).  imoist 0/1; iterations = 20 for CM1.  Outputs are nk words each; any
 * output pointer may be NULL except th0, qv0, pi0 and prs0.
 * Returns 0, or -1 on bad arguments (storm_initialization.rs:194-226). */
int oracle_wk_column(int nk, const float* zh, int imoist, int iterations, float* th0, float* qv0,
                     float* thv0, float* pi0, float* prs0, float* t0, float* rh0) {
  if (nk < 1 || (imoist != 0 && imoist != 1) || iterations < 1) return -1;
  for (int k = 0; k < nk; ++k) {
    const float below = k == 0 ? 0.0f : zh[k - 1];
    if (!(zh[k] > below) || !isfinite(zh[k])) return -1;
  }
  const float reps = K_RV / K_RD;
  float sfc[3];
  oracle_wk_surface(sfc);
  float rh[nk], thv[nk];
  /* theta and relative humidity (base.F:385-397) */
  for (int k = 0; k < nk; ++k) {
    if (zh[k] < WK_Z_TROP) {
      const float shape = powf(zh[k] / WK_Z_TROP, 1.25f);
      th0[k] = WK_TH_SFC + (WK_TH_TROP - WK_TH_SFC) * shape;
      rh[k] = imoist == 1 ? 1.0f - 0.75f * shape : 0.0f;
    } else {
      const float rate = K_G / (WK_T_TROP * K_CP);
      th0[k] = WK_TH_TROP * expf(rate * (zh[k] - WK_Z_TROP));
      rh[k] = imoist == 1 ? 0.25f : 0.0f;
    }
    qv0[k] = 0.0f;
  }
  /* 20-sweep hydrostatic fixed point (base.F:405-429) */
  const float cpdrd = K_CP / K_RD;
  for (int it = 0; it < iterations; ++it) {
    for (int k = 0; k < nk; ++k) thv[k] = th0[k] * (1.0f + reps * qv0[k]) / (1.0f + qv0[k]);
    for (int k = 0; k < nk; ++k) {
      const float pi_below = k == 0 ? sfc[0] : pi0[k - 1];
      const float thv_below = k == 0 ? sfc[2] : thv[k - 1];
      const float dz = k == 0 ? zh[0] : zh[k] - zh[k - 1];
      const float denom = K_CP * 0.5f * (thv[k] + thv_below);
      pi0[k] = pi_below - K_G * dz / denom;
    }
    for (int k = 0; k < nk; ++k) prs0[k] = K_P00 * powf(pi0[k], cpdrd);
    for (int k = 0; k < nk; ++k) {
      float q = rh[k] * oracle_rslf(prs0[k], th0[k] * pi0[k]);
      qv0[k] = q > WK_QV_PBL ? WK_QV_PBL : q;
    }
  }
  /* diagnostics (base.F:411-413 last sweep, :433-435) */
  for (int k = 0; k < nk; ++k) {
    if (thv0) thv0[k] = thv[k];
    if (rh0) rh0[k] = qv0[k] / oracle_rslf(prs0[k], th0[k] * pi0[k]);
    if (t0) t0[k] = th0[k] * pi0[k];
  }
  return 0;
}

/* iwnd=2 on face heights (base.F:2331-2357; storm_initialization.rs:354-389). */
void oracle_analytic_shear(int n, const float* zu, const float* zv, float* u, float* v) {
  const float pi = 3.14159265358979f;
  const float udep1 = 2000.0f, udep2 = 6000.0f, umax1 = 7.0f, umax2 = 31.0f;
  for (int k = 0; k < n; ++k) {
    if (u) {
      const float z = zu[k];
      if (z <= udep1) {
        const float angle = 90.0f * (z / udep1) * (pi / 180.0f);
        u[k] = umax1 - umax1 * cosf(angle);
      } else if (z <= udep2) {
        u[k] = umax1 + (z - udep1) * (umax2 - umax1) / (udep2 - udep1);
      } else {
        u[k] = umax2;
      }
    }
    if (v) {
      const float z = zv[k];
      if (z <= udep1) {
        const float angle = 90.0f * (z / udep1) * (pi / 180.0f);
        v[k] = umax1 * sinf(angle);
      } else {
        v[k] = umax1;
      }
    }
  }
}

/* iinit=1 cos^2 bubble into tha[nk][nj][ni] on mass points xh[ni], yh[nj],
 * zh[nk] (flat grid) (init3d.F:450-482; initial_perturbation.rs:449-466). */
void oracle_theta_bubble(int ni, int nj, int nk, const float* xh, const float* yh, const float* zh,
                         float xc, float yc, float zc, float hrad, float zrad, float amp,
                         float* tha) {
  const float pi = 3.14159265358979f;
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const float rx = (xh[i] - xc) / hrad;
        const float ry = (yh[j] - yc) / hrad;
        const float rz = (zh[k] - zc) / zrad;
        const float beta = sqrtf(rx * rx + ry * ry + rz * rz);
        float value = 0.0f;
        if (beta < 1.0f) {
          const float c = cosf(0.5f * pi * beta);
          value = amp * (c * c);
        }
        tha[((int64_t)k * nj + j) * ni + i] = value;
      }
}
