/* Oracle (test infrastructure only): CPU restatement of CM1's limits and
 * advective Courant number as the reference forms them.
 *
 *   cm1_acoustic_small_step_limit_s   src/cm1core/gm1_runtime.py:249-268
 *   cm1_diagnostic_acoustic_substeps  src/cm1core/gm1_runtime.py:284-302
 *   cm1_advective_courant             src/cm1core/gm1_runtime.py:458-489
 *   _reduce_courant, advective_courant_number
 *                                     src/cm1core/storm_diagnostics.py:195-297
 *
 * The domain reduction walks the levels in order, takes each level's maximum
 * with NumPy's amax rule (a NaN in the level makes the level NaN) and folds
 * them with Python's max(largest, level) rule (only a greater value
 * replaces the running maximum, so a NaN level never does).
 */
#include <math.h>
#include <stdint.h>
#include "real.h"

double oracle_small_step_limit(double dx, double dy) { return 0.60 * (dx < dy ? dx : dy) / 360.0; }

int oracle_diagnostic_substeps(double dt, double dx, double dy) {
  const double limit = oracle_small_step_limit(dx, dy);
  const double r = dt / limit;
  long long n = r >= 0 ? (long long)floor(r + 0.5) : -(long long)floor(-r + 0.5);
  if (n < 4) n = 4;
  if (n % 2) n += 1;
  if (dt / (double)n > limit) n += 2;
  return (int)n;
}

double oracle_advective_courant(double dt, double dx, double dy, double dz, double u, double v, double w) {
  const double a = u * dt / dx, b = v * dt / dy, c = w * dt / dz;
  return sqrt((a * a + b * b) + c * c);
}

/* u (nk, nj, ni+1), v (nk, nj+1, ni), w (nk+1, nj, ni); level_max[nk] out */
float oracle_courant_max(int ni, int nj, int nk, const float* u, const float* v, const float* w, const float* uh,
                         const float* vh, const float* mh, float dtdx, float dtdy, float dtdz, float* level_max) {
  const int64_t plane = (int64_t)ni * nj;
  float largest = 0.0f;
  for (int k = 0; k < nk; ++k) {
    float m = -1.0f;
    int has_nan = 0;
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const int64_t fu = ((int64_t)k * nj + j) * (ni + 1) + i;
        const int64_t fv = ((int64_t)k * (nj + 1) + j) * ni + i;
        const int64_t fw = ((int64_t)k * nj + j) * ni + i;
        float t = u[fu] + u[fu + 1];
        t = t * dtdx;
        t = t * uh[i];
        float acc = t * t;
        t = v[fv] + v[fv + ni];
        t = t * dtdy;
        t = t * vh[j];
        t = t * t;
        acc = acc + t;
        t = w[fw] + w[fw + plane];
        t = t * dtdz;
        t = t * mh[k];
        t = t * t;
        acc = acc + t;
        const float s = sqrtf(acc);
        if (isnan(s)) has_nan = 1;
        else if (s > m) m = s;
      }
    const float lv = has_nan ? NAN : m;
    if (level_max) level_max[k] = lv;
    if (lv > largest) largest = lv;
  }
  return largest;
}
