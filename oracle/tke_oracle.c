/*
 * tke_oracle.c - CPU restatement of the reference's Deardorff SGS/TKE local
 * algebra: tkekm (grid scale, length scale, Km, Kh, dissipation), the
 * free-slip lower face tkebc, and the pre-turbt TKE source.
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library.
 *
 * Followed functions (reference file:line):
 *   sgs_constants_f32    src/cm1core/cuda_sgs_tke.py:187-208
 *   cpu_sgs_tke_inplace  src/cm1core/cuda_sgs_tke.py:220-357
 *
 * Arithmetic: binary32 one operation at a time (-ffp-contract=off).  The grid
 * scale (dx dy dz)^0.33333333 goes through powf, so every word that depends
 * on it agrees with the twin (NumPy's power) and the CUDA library (CUDA's
 * powf) within a few ULPs, not bit for bit.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include "real.h"

typedef struct {
    const float *ruh, *rvh, *rmf, *nm, *defv, *defh;
    float *tkea, *tk, *grdscl, *rgrdscl, *lenscl, *dissten, *cme, *ce1, *ce2, *csm, *kmh, *kmv, *khh, *khv, *tketen;
} sgs_tke_arrays;

void oracle_sgs_constants(float out[4]) {
    const float cme = 0.10f, c_l = 0.8165f, ri_c = 0.25f, pi = 3.1415926535897932384626433f;
    float ce1 = cme * c_l;
    ce1 = ce1 * c_l;
    ce1 = ce1 * (1.0f / ri_c - 1.0f);
    float ce2 = (cme * pi) * pi - ce1;
    ce2 = ce2 > 0.0f ? ce2 : 0.0f;
    const float numerator = (cme * cme) * cme;
    const float csm = powf(numerator / (ce1 + ce2), 0.25f);
    out[0] = cme;
    out[1] = ce1;
    out[2] = ce2;
    out[3] = csm;
}

#define W(p, k, j, i) (p)[((size_t)(k) * nj + (size_t)(j)) * ni + (size_t)(i)]

/* returns the number of clipped (tke <= 1e-10) words */
int oracle_sgs_tke(const sgs_tke_arrays *a, int ni, int nj, int nk, float dx, float dy, float dz) {
    float c[4];
    oracle_sgs_constants(c);
    const float c_l = 0.8165f, exponent = 0.33333333f, tke_min = 1.0e-10f, nm_min = 1.0e-6f, small = 0.001f;
    int clipped = 0;
    for (int k = 1; k < nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                float grid = dx * a->ruh[i];
                grid = grid * (dy * a->rvh[j]);
                grid = grid * (dz * W(a->rmf, k, j, i));
                grid = powf(grid, exponent);
                const float reciprocal = 1.0f / grid;
                float tk, length;
                const float nm = W(a->nm, k, j, i);
                if (W(a->tkea, k, j, i) <= tke_min) {
                    tk = tke_min;
                    length = small * grid;
                    clipped += 1;
                } else {
                    tk = W(a->tkea, k, j, i);
                    length = grid;
                    if (nm > nm_min) {
                        length = c_l * sqrtf(tk / nm);
                        length = fminf(length, grid);
                        length = fmaxf(length, small * grid);
                    }
                }
                W(a->grdscl, k, j, i) = grid;
                W(a->rgrdscl, k, j, i) = reciprocal;
                W(a->tk, k, j, i) = tk;
                W(a->lenscl, k, j, i) = length;
                W(a->cme, k, j, i) = c[0];
                W(a->ce1, k, j, i) = c[1];
                W(a->ce2, k, j, i) = c[2];
                W(a->csm, k, j, i) = c[3];
                const float sqrt_tk = sqrtf(tk);
                float df = c[2] * length;
                df = df * reciprocal;
                df = c[1] + df;
                float diss = df * tk;
                diss = diss * sqrt_tk;
                diss = diss / length;
                W(a->dissten, k, j, i) = W(a->dissten, k, j, i) + diss;
                float km = c[0] * sqrt_tk;
                km = km * length;
                W(a->kmh, k, j, i) = km;
                W(a->kmv, k, j, i) = km;
                float prinv = 3.0f;
                if (nm > nm_min) {
                    const float cand = 1.0f + 2.0f * (length * reciprocal);
                    prinv = fminf(cand, 3.0f);
                }
                const float kh = km * prinv;
                W(a->khh, k, j, i) = kh;
                W(a->khv, k, j, i) = kh;
                const float buoy = (-kh) * nm;
                float source = buoy - W(a->dissten, k, j, i);
                float deform = W(a->defv, k, j, i) + W(a->defh, k, j, i);
                deform = fmaxf(0.0f, deform);
                source = source + km * deform;
                W(a->tketen, k, j, i) = source;
            }
    for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i) {
            W(a->tkea, 0, j, i) = 0.0f;
            W(a->kmh, 0, j, i) = 0.0f;
            W(a->kmv, 0, j, i) = W(a->kmh, 0, j, i);
            float ratio = W(a->khv, 1, j, i) / (1.0e-10f + W(a->kmv, 1, j, i));
            W(a->khv, 0, j, i) = W(a->kmv, 0, j, i) * ratio;
            ratio = W(a->khh, 1, j, i) / (1.0e-10f + W(a->kmh, 1, j, i));
            W(a->khh, 0, j, i) = W(a->kmh, 0, j, i) * ratio;
        }
    return clipped;
}
