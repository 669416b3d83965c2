/* vertical_oracle.c - TEST INFRASTRUCTURE ONLY.  CPU restatement of the
 * reference's CM1 vertical-coordinate generator for stretch_z = 0 and 1:
 *
 *   derive_stretch_z1      src/cm1core/cuda_stretch_z1.py:130-201
 *                          (param.F:7814-7914 feasibility and c1/c2)
 *   build_stretch_z1_grid  src/cm1core/cuda_stretch_z1.py:204-263
 *                          (param.F:7916-7953, 8162-8209)
 *   _rds_rdsf              src/cm1core/cm1_vertical_grid.py:599-613 (init_terrain.F:292-298)
 *   fornberg_extrapolation_weights  src/cm1core/cm1_vertical_grid.py:387-454
 *   build_vertical_levels  src/cm1core/cm1_vertical_grid.py:780-927 (stretch_z 0 / 1 only)
 *
 * Binary32 one operation at a time (the twins' np.float32 helpers), binary64
 * for the Fornberg table.  Returns 0, or a negative code for a refused set:
 * -1 argument shape, -2 infeasible segments, -3 non-positive spacing,
 * -4 duplicated Fornberg nodes, -5 uniform top not dz*nk, -6 stretch_z not
 * built. */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include "real.h"

typedef struct {
    int32_t nk1, nk2, nk3;
    float nominal, c1, c2;
} oracle_z1_derived;

static int nint_positive(float v) { return (int)floor((double)v + 0.5); }

int oracle_derive_stretch_z1(int nk, float dz, float ztop, float str_bot, float str_top, float dz_bot, float dz_top,
                             oracle_z1_derived *out) {
    if (nk < 4) return -1;
    if (!isfinite(dz) || !isfinite(ztop) || !isfinite(str_bot) || !isfinite(str_top) || !isfinite(dz_bot) ||
        !isfinite(dz_top))
        return -1;
    if (dz <= 0.0f || ztop <= 0.0f || dz_bot <= 0.0f || dz_top <= 0.0f) return -1;
    if (str_bot < 0.0f || str_top <= str_bot || str_top > ztop) return -1;
    const float nominal = 0.5f * (dz_bot + dz_top);
    const int nk1 = nint_positive(str_bot / dz_bot);
    const int nk3 = nint_positive((ztop - str_top) / dz_top);
    const int nk2 = nk - (nk1 + nk3);
    if (nk1 < 0 || nk2 < 2 || nk3 < 0) return -2;
    const double bottom = fabs((double)((float)nk1 * dz_bot - str_bot));
    const double middle = fabs((double)((float)nk2 * nominal - (str_top - str_bot)));
    const double top = fabs((double)((float)nk3 * dz_top - (ztop - str_top)));
    if (bottom > 0.01 || middle >= 0.01 || top > 0.01) return -2;
    const float c2 = (nominal - dz_bot) / ((nominal * nominal) * (float)(nk2 - 1));
    const float c1 = dz_bot / nominal - c2 * nominal;
    const float len = (dz_bot * (float)nk1 + nominal * (float)nk2) + dz_top * (float)nk3;
    if (fabs((double)(ztop - len)) > (double)(1.0e-6f * ztop)) return -2;
    out->nk1 = nk1;
    out->nk2 = nk2;
    out->nk3 = nk3;
    out->nominal = nominal;
    out->c1 = c1;
    out->c2 = c2;
    return 0;
}

/* profiles: zf, sigmaf, mf, rmf, rdsf (nk+3); zh, sigma, mh, rmh, rds (nk+2) */
int oracle_stretch_z1_grid(int nk, float dz, float ztop, float str_bot, float str_top, float dz_bot, float dz_top,
                           float *zf, float *zh, float *sigmaf, float *sigma, float *mh, float *mf, float *rmh,
                           float *rmf, float *rds, float *rdsf, oracle_z1_derived *derived) {
    oracle_z1_derived d;
    const int rc = oracle_derive_stretch_z1(nk, dz, ztop, str_bot, str_top, dz_bot, dz_top, &d);
    if (rc != 0) return rc;
    if (derived) *derived = d;
    memset(zf, 0, sizeof(float) * (size_t)(nk + 3));
    memset(sigmaf, 0, sizeof(float) * (size_t)(nk + 3));
    for (int k = 1; k <= d.nk1 + 1; ++k) {
        zf[k] = (float)(k - 1) * dz_bot;
        sigmaf[k] = zf[k];
    }
    for (int k = d.nk1 + 1; k <= d.nk1 + d.nk2 + 1; ++k) {
        const float delta = (float)(k - 1 - d.nk1);
        const float factor = d.c1 + (d.c2 * delta) * d.nominal;
        const float distance = (factor * delta) * d.nominal;
        zf[k] = zf[d.nk1 + 1] + distance;
        sigmaf[k] = zf[k];
    }
    for (int k = d.nk1 + d.nk2 + 2; k <= nk + 1; ++k) {
        zf[k] = zf[k - 1] + dz_top;
        sigmaf[k] = zf[k];
    }
    zf[0] = -zf[2];
    zf[nk + 2] = zf[nk + 1] + (zf[nk + 1] - zf[nk]);
    sigmaf[0] = -sigmaf[2];
    sigmaf[nk + 2] = sigmaf[nk + 1] + (sigmaf[nk + 1] - sigmaf[nk]);
    for (int k = 0; k <= nk + 1; ++k) {
        zh[k] = 0.5f * (zf[k + 1] + zf[k]);
        mh[k] = dz / (zf[k + 1] - zf[k]);
    }
    zh[0] = -zh[1];
    zh[nk + 1] = zh[nk] + 2.0f * (zf[nk + 1] - zh[nk]);
    for (int k = 1; k <= nk + 1; ++k) mf[k] = dz / (zh[k] - zh[k - 1]);
    mf[0] = mf[1];
    mf[nk + 2] = mf[nk + 1];
    for (int k = 0; k <= nk + 1; ++k) sigma[k] = 0.5f * (sigmaf[k] + sigmaf[k + 1]);
    for (int k = 0; k <= nk + 1; ++k) rmh[k] = 1.0f / mh[k];
    for (int k = 0; k <= nk + 2; ++k) rmf[k] = 1.0f / mf[k];
    for (int k = 1; k <= nk; ++k)
        if (!(zf[k + 1] > zf[k])) return -3;
    memset(rds, 0, sizeof(float) * (size_t)(nk + 2));
    memset(rdsf, 0, sizeof(float) * (size_t)(nk + 3));
    for (int k = 2; k <= nk; ++k) rds[k] = 1.0f / (sigma[k] - sigma[k - 1]);
    for (int k = 1; k <= nk; ++k) rdsf[k] = 1.0f / (sigmaf[k + 1] - sigmaf[k]);
    return 0;
}

/* Fornberg (1988) table with bigm = 4, bign = 3 (param.F:9016-9035); the
 * value weights delta(2, 0, nu) */
int oracle_fornberg_weights(int nk, const float *sigma, const float *sigmaf, int top, float out[3]) {
    if (nk < 4) return -1;
    float den, num, nodes[4];
    if (top) {
        den = sigmaf[nk + 1] - sigmaf[nk];
        num = sigmaf[nk + 1];
        for (int q = 0; q < 4; ++q) nodes[q] = sigma[nk - q];
    } else {
        den = sigmaf[2] - sigmaf[1];
        num = sigmaf[1];
        for (int q = 0; q < 4; ++q) nodes[q] = sigma[1 + q];
    }
    if (!isfinite(den) || !(den > 0.0f)) return -1;
    const double x0 = (double)(num / den);
    double alpha[4];
    for (int q = 0; q < 4; ++q) alpha[q] = (double)(nodes[q] / den);
    double t[4][6][4];
    memset(t, 0, sizeof t);
    t[0][1][0] = 1.0;
    double b1 = 1.0;
    for (int n = 1; n < 4; ++n) {
        double b2 = 1.0;
        for (int nu = 0; nu < n; ++nu) {
            const double b3 = alpha[n] - alpha[nu];
            if (!isfinite(b3) || b3 == 0.0) return -4;
            b2 = b2 * b3;
            t[n - 1][n + 1][nu] = 0.0;
            for (int m = 0; m <= (n < 4 ? n : 4); ++m)
                t[n][m + 1][nu] = ((alpha[n] - x0) * t[n - 1][m + 1][nu] - m * t[n - 1][m][nu]) / b3;
        }
        for (int m = 0; m <= (n < 4 ? n : 4); ++m)
            t[n][m + 1][n] = (b1 / b2) * (m * t[n - 1][m][n - 1] - (alpha[n - 1] - x0) * t[n - 1][m + 1][n - 1]);
        b1 = b2;
    }
    for (int nu = 0; nu < 3; ++nu) out[nu] = (float)t[2][1][nu];
    return 0;
}

/* build_vertical_levels for stretch_z 0 and 1: profiles, rds/rdsf, cgs/cgt */
int oracle_vertical_levels(int stretch_z, int nk, float dz, float ztop, float str_bot, float str_top, float dz_bot,
                           float dz_top, float *zf, float *zh, float *sigmaf, float *sigma, float *mh, float *mf,
                           float *rmh, float *rmf, float *rds, float *rdsf, float cgs[3], float cgt[3]) {
    if (stretch_z != 0 && stretch_z != 1) return -6;
    if (nk < 4) return -1;
    if (stretch_z == 0) {
        const float expected = dz * (float)nk;
        if (ztop != expected) return -5;
        str_bot = 0.0f;
        str_top = expected;
        dz_bot = dz_top = dz;
        ztop = expected;
    }
    int rc = oracle_stretch_z1_grid(nk, dz, ztop, str_bot, str_top, dz_bot, dz_top, zf, zh, sigmaf, sigma, mh, mf,
                                    rmh, rmf, rds, rdsf, 0);
    if (rc != 0) return rc;
    rc = oracle_fornberg_weights(nk, sigma, sigmaf, 0, cgs);
    if (rc != 0) return rc;
    return oracle_fornberg_weights(nk, sigma, sigmaf, 1, cgt);
}
