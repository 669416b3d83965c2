/*
 * advection_oracle.c - CPU restatement of the reference's fifth-order/WENO5
 * scalar advection and terrain mass flux on the padded (ng = 3) lane.
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library.
 *
 * Followed functions (reference file:line):
 *   _flx3_f32, _flx5_f32, _weno5_f32, _upstrpd_f32
 *                                   src/cm1core/cuda_advection5.py:170-245
 *   cpu_terrain_mass_flux5_inplace  src/cm1core/cuda_advection5.py:271-437
 *   cpu_scalar_advection5_inplace   src/cm1core/cuda_advection5.py:440-579
 *   tendency with CM1 lateral sides (whole-domain launch, open-side inflow
 *   edits of adv.F:86-98,214-340) - the reference CUDA kernel
 *   cm1_adv5_scalar_tendency_v1     src/cm1core/cuda_advection5.py:669
 *   (the CPU twin covers only the tile-local launch, lateral code 0)
 *
 * Arithmetic: binary32 one operation at a time (-ffp-contract=off); the WENO
 * smoothness weights in binary64 exactly as the twin's Python floats.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include "real.h"

#define NG 3

#define F5_1 0x1.111112p-5f
#define F5_2 -0x1.bbbbbcp-3f
#define F5_3 0x1.911112p-1f
#define F5_4 0x1.ccccccp-2f
#define F5_5 -0x1.99999ap-5f
#define F3_1 -0x1.555556p-3f
#define F3_2 0x1.aaaaaap-1f
#define F3_3 0x1.555556p-2f
#define C13_12 0x1.155556p+0f
#define CM7_6 -0x1.2aaaaap+0f
#define C11_6 0x1.d55556p+0f
#define C1_6 0x1.555556p-3f

typedef struct {
    const float *u3d, *v3d, *w3d;
    float *rru, *rrv, *rrw;
    const float *rho0_3d, *rf0, *rgzu, *rgzv, *dzdx, *dzdy, *gz;
    float *divx;
} mass_flux_arrays;

typedef struct {
    const float *scalar, *rru, *rrv, *rrw;
    const float *c1, *c2, *rr0, *gz, *divx;
    float *tendency, *flux_x, *flux_y, *flux_z;
} scalar_adv_arrays;

/* padded shapes: scalar (nk+2, nj+6, ni+6); u (nk+2, nj+6, ni+7);
 * v (nk+2, nj+7, ni+6); w (nk+3, nj+6, ni+6) */
#define PS(p, k, y, x) (p)[((size_t)(k) * (nj + 2 * NG) + (size_t)(y)) * (ni + 2 * NG) + (size_t)(x)]
#define PU(p, k, y, x) (p)[((size_t)(k) * (nj + 2 * NG) + (size_t)(y)) * (ni + 1 + 2 * NG) + (size_t)(x)]
#define PV(p, k, y, x) (p)[((size_t)(k) * (nj + 1 + 2 * NG) + (size_t)(y)) * (ni + 2 * NG) + (size_t)(x)]
#define PW PS
/* unpadded (nk', nj, ni) and 2-D metrics */
#define C3(p, k, j, i) (p)[((size_t)(k) * nj + (size_t)(j)) * ni + (size_t)(i)]
#define M2(p, j, i, nx) (p)[(size_t)(j) * (nx) + (size_t)(i)]

static inline float flx3(float s1, float s2, float s3) {
    float r = F3_1 * s1;
    r = r + F3_2 * s2;
    return r + F3_3 * s3;
}

static inline float flx5(float s1, float s2, float s3, float s4, float s5) {
    float r = F5_1 * s1;
    r = r + F5_2 * s2;
    r = r + F5_3 * s3;
    r = r + F5_4 * s4;
    return r + F5_5 * s5;
}

static inline double dmin30(double x) { return x < 1.0e30 ? x : 1.0e30; }

float oracle_weno5(float s1, float s2, float s3, float s4, float s5, double eps) {
    float d1 = (s1 - 2.0f * s2) + s3;
    float e1 = (s1 - 4.0f * s2) + 3.0f * s3;
    float b1r = C13_12 * (d1 * d1) + 0.25f * (e1 * e1);
    float d2 = (s2 - 2.0f * s3) + s4;
    float e2 = s2 - s4;
    float b2r = C13_12 * (d2 * d2) + 0.25f * (e2 * e2);
    float d3 = (s3 - 2.0f * s4) + s5;
    float e3 = (3.0f * s3 - 4.0f * s4) + s5;
    float b3r = C13_12 * (d3 * d3) + 0.25f * (e3 * e3);
    double b1 = b1r, b2 = b2r, b3 = b3r;
    double tau = fabs(b1 - b3);
    double q1 = dmin30(tau / (b1 + eps));
    double q2 = dmin30(tau / (b2 + eps));
    double q3 = dmin30(tau / (b3 + eps));
    double w1 = (double)0.1f * (1.0 + q1 * q1);
    double w2 = (double)0.6f * (1.0 + q2 * q2);
    double w3 = (double)0.3f * (1.0 + q3 * q3);
    float p1 = (F3_3 * s1 + CM7_6 * s2) + C11_6 * s3;
    float p2 = (F3_1 * s2 + F3_2 * s3) + F3_3 * s4;
    float p3 = (F3_3 * s3 + F3_2 * s4) + F3_1 * s5;
    return (float)((w1 * (double)p1 + w2 * (double)p2 + w3 * (double)p3) / (w1 + w2 + w3));
}

static inline float upstrpd(float s1, float s2, float s3, float weps) {
    float dd = s2 - s1;
    float se = copysignf(fabsf(weps), dd);
    float rr = (s3 - s2) / (se + dd);
    float cand = C1_6 + F3_3 * rr;
    float inner = fminf(cand, 1.0f);
    float phi = fmaxf(0.0f, fminf(rr, inner));
    return s2 + phi * (s2 - s1);
}

static inline float recon(float s1, float s2, float s3, float s4, float s5, int weno, double eps) {
    return weno ? oracle_weno5(s1, s2, s3, s4, s5, eps) : flx5(s1, s2, s3, s4, s5);
}

void oracle_terrain_mass_flux5(const mass_flux_arrays *a, int ni, int nj, int nk, float dx, float dy, float dz) {
    const float half = 0.5f;
    for (int k0 = 0; k0 < nk; ++k0) {
        const int k = k0 + 1;
        for (int j = 0; j < nj; ++j) {
            const int y = j + NG;
            for (int face = 1; face < ni; ++face) {
                const int x = face + NG;
                float density = C3(a->rho0_3d, k0, j, face - 1) + C3(a->rho0_3d, k0, j, face);
                PU(a->rru, k, y, x) = (half * density) * (PU(a->u3d, k, y, x) * M2(a->rgzu, j, face, ni + 1));
            }
        }
        for (int face = 1; face < nj; ++face) {
            const int y = face + NG;
            for (int i = 0; i < ni; ++i) {
                const int x = i + NG;
                float density = C3(a->rho0_3d, k0, face - 1, i) + C3(a->rho0_3d, k0, face, i);
                PV(a->rrv, k, y, x) = (half * density) * (PV(a->v3d, k, y, x) * M2(a->rgzv, face, i, ni));
            }
        }
    }
    for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i) {
            PW(a->rrw, 1, j + NG, i + NG) = 0.0f;
            PW(a->rrw, nk + 1, j + NG, i + NG) = 0.0f;
        }
    const float zt = (float)nk * dz;
    const float rzt = 1.0f / zt;
    for (int k = 2; k <= nk; ++k) {
        const float sigmaf = (float)(k - 1) * dz;
        const float sigma = (float)((double)k - 1.5) * dz;
        float r2 = (sigmaf - sigma) * (1.0f / dz);
        const float r1 = half * (1.0f - r2);
        r2 = half * r2;
        for (int j = 1; j < nj - 1; ++j) {
            const int y = j + NG;
            for (int i = 1; i < ni - 1; ++i) {
                const int x = i + NG;
                float ux = r2 * (PU(a->rru, k, y, x) + PU(a->rru, k, y, x + 1)) +
                           r1 * (PU(a->rru, k - 1, y, x) + PU(a->rru, k - 1, y, x + 1));
                float vy = r2 * (PV(a->rrv, k, y, x) + PV(a->rrv, k, y + 1, x)) +
                           r1 * (PV(a->rrv, k - 1, y, x) + PV(a->rrv, k - 1, y + 1, x));
                float terrain = ux * M2(a->dzdx, j, i, ni) + vy * M2(a->dzdy, j, i, ni);
                terrain = terrain * (sigmaf - zt);
                terrain = terrain * M2(a->gz, j, i, ni);
                terrain = terrain * rzt;
                PW(a->rrw, k, y, x) = C3(a->rf0, k - 1, j, i) * PW(a->w3d, k, y, x) + terrain;
            }
        }
    }
    const float rdx = 1.0f / dx, rdy = 1.0f / dy, rdsf = 1.0f / dz;
    for (int k0 = 0; k0 < nk; ++k0) {
        const int k = k0 + 1;
        for (int j = 1; j < nj - 1; ++j) {
            const int y = j + NG;
            for (int i = 1; i < ni - 1; ++i) {
                const int x = i + NG;
                float value = (PU(a->rru, k, y, x + 1) - PU(a->rru, k, y, x)) * rdx +
                              (PV(a->rrv, k, y + 1, x) - PV(a->rrv, k, y, x)) * rdy;
                value = value + (PW(a->rrw, k + 1, y, x) - PW(a->rrw, k, y, x)) * rdsf;
                C3(a->divx, k0, j, i) = (fabs((double)value) < 1.0e-20) ? 0.0f : value;
            }
        }
    }
}

/* Vertical column of the tendency: mode 0 uniform (rdsf = 1/dz); mode 1
 * terrain-following stretched, rdsf(k) per level
 * (cuda_gm1_child_stretched_scalar.py:138-153); mode 2 flat stretched,
 * ((d*rdz)*mh(k)) and the column's rr0(k) without gz
 * (cuda_gm1_child_stretched_scalar.py:324-348; adv.F:555-572, 646-656). */
typedef struct {
    int mode;
    const float *rdsf; /* (nk+3,) CM1-indexed, mode 1 */
    const float *mh;   /* (nk+2,) CM1-indexed, mode 2 */
    float rdz;         /* mode 2 */
} vertical_column;

static const vertical_column kUniformColumn = {0, 0, 0, 0.0f};

/* One cell of the tendency with CM1 lateral side codes (0 = tile-local). */
static float tendency_cell(const scalar_adv_arrays *a, const float *fx, const float *fy, const float *fz, int ni,
                           int nj, int nk, int k, int j, int i, unsigned obc, float rdx, float rdy, float rdsf,
                           const vertical_column *vc) {
    const int x = i + NG, y = j + NG;
    float fw = PU(fx, k, y, x), fe = PU(fx, k, y, x + 1);
    float fs = PV(fy, k, y, x), fn = PV(fy, k, y + 1, x);
    const float sv = PS(a->scalar, k, y, x);
    const float uw = PU(a->rru, k, y, x), ue = PU(a->rru, k, y, x + 1);
    const float vs = PV(a->rrv, k, y, x), vn = PV(a->rrv, k, y + 1, x);
    const int iw = (i == 0) && (((obc >> 0) & 15u) == 2u) && uw >= 0.0f;
    const int ie = (i + 1 == ni) && (((obc >> 4) & 15u) == 2u) && ue <= 0.0f;
    const int js = (j == 0) && (((obc >> 8) & 15u) == 2u) && vs >= 0.0f;
    const int jn = (j + 1 == nj) && (((obc >> 12) & 15u) == 2u) && vn <= 0.0f;
    if (iw) fw = fe;
    if (ie) fe = fw;
    if (js) fs = fn;
    if (jn) fn = fs;
    float ax = (fw - fe) * rdx;
    float ay = (fs - fn) * rdy;
    if (iw) ax = ax - (sv * (ue - uw)) * rdx;
    if (ie) ax = ax - (sv * (ue - uw)) * rdx;
    if (js) ay = ay - (sv * (vn - vs)) * rdy;
    if (jn) ay = ay - (sv * (vn - vs)) * rdy;
    float az;
    if (vc->mode == 2) {
        if (k == 1)
            az = ((-PW(fz, 2, y, x)) * vc->rdz) * vc->mh[k];
        else if (k == nk)
            az = (PW(fz, nk, y, x) * vc->rdz) * vc->mh[k];
        else
            az = ((-(PW(fz, k + 1, y, x) - PW(fz, k, y, x))) * vc->rdz) * vc->mh[k];
    } else {
        const float r = vc->mode == 1 ? vc->rdsf[k] : rdsf;
        if (k == 1)
            az = (-PW(fz, 2, y, x)) * r;
        else if (k == nk)
            az = PW(fz, nk, y, x) * r;
        else
            az = (PW(fz, k, y, x) - PW(fz, k + 1, y, x)) * r;
    }
    float total = (ax + ay) + az;
    total = total + sv * C3(a->divx, k - 1, j, i);
    if (vc->mode == 2) return total * C3(a->rr0, k - 1, 0, 0);
    return (total * C3(a->rr0, k - 1, j, i)) * M2(a->gz, j, i, ni);
}

static void scalar_advection5_column(const scalar_adv_arrays *a, int ni, int nj, int nk, int use_weno, float dx,
                                     float dy, float dz, double weps, unsigned obc, const vertical_column *vc) {
    float *fx = a->flux_x, *fy = a->flux_y, *fz = a->flux_z;
    const float *s = a->scalar;
    for (int k = 1; k <= nk; ++k) {
        for (int j = 0; j < nj; ++j) {
            const int y = j + NG;
            for (int face = 0; face <= ni; ++face) {
                const int x = face + NG;
                const float m = PU(a->rru, k, y, x);
                float r;
                if (m >= 0.0f)
                    r = recon(PS(s, k, y, x - 3), PS(s, k, y, x - 2), PS(s, k, y, x - 1), PS(s, k, y, x),
                              PS(s, k, y, x + 1), use_weno, weps);
                else
                    r = recon(PS(s, k, y, x + 2), PS(s, k, y, x + 1), PS(s, k, y, x), PS(s, k, y, x - 1),
                              PS(s, k, y, x - 2), use_weno, weps);
                PU(fx, k, y, x) = m * r;
            }
        }
        for (int face = 0; face <= nj; ++face) {
            const int y = face + NG;
            for (int i = 0; i < ni; ++i) {
                const int x = i + NG;
                const float m = PV(a->rrv, k, y, x);
                float r;
                if (m >= 0.0f)
                    r = recon(PS(s, k, y - 3, x), PS(s, k, y - 2, x), PS(s, k, y - 1, x), PS(s, k, y, x),
                              PS(s, k, y + 1, x), use_weno, weps);
                else
                    r = recon(PS(s, k, y + 2, x), PS(s, k, y + 1, x), PS(s, k, y, x), PS(s, k, y - 1, x),
                              PS(s, k, y - 2, x), use_weno, weps);
                PV(fy, k, y, x) = m * r;
            }
        }
    }
    for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i) {
            PW(fz, 1, j + NG, i + NG) = 0.0f;
            PW(fz, nk + 1, j + NG, i + NG) = 0.0f;
        }
    const float wepsf = (float)weps;
    for (int k = 2; k <= nk; ++k) {
        for (int j = 0; j < nj; ++j) {
            const int y = j + NG;
            for (int i = 0; i < ni; ++i) {
                const int x = i + NG;
                const float m = PW(a->rrw, k, y, x);
#define SK(kk) PS(s, (kk), y, x)
                float r;
                const float c1 = C3(a->c1, k - 1, j, i), c2 = C3(a->c2, k - 1, j, i);
                if (k == 2) {
                    if (m >= 0.0f)
                        r = c1 * SK(k - 1) + c2 * SK(k);
                    else if (use_weno)
                        r = upstrpd(SK(k + 1), SK(k), SK(k - 1), wepsf);
                    else
                        r = flx3(SK(k + 1), SK(k), SK(k - 1));
                } else if (k == nk) {
                    int up = use_weno ? (m > 0.0f) : (m >= 0.0f);
                    if (up)
                        r = use_weno ? upstrpd(SK(k - 2), SK(k - 1), SK(k), wepsf) : flx3(SK(k - 2), SK(k - 1), SK(k));
                    else
                        r = c1 * SK(k - 1) + c2 * SK(k);
                } else if (k == 3) {
                    if (m >= 0.0f)
                        r = use_weno ? upstrpd(SK(k - 2), SK(k - 1), SK(k), wepsf) : flx3(SK(k - 2), SK(k - 1), SK(k));
                    else
                        r = recon(SK(k + 2), SK(k + 1), SK(k), SK(k - 1), SK(k - 2), use_weno, weps);
                } else if (k == nk - 1) {
                    if (m >= 0.0f)
                        r = recon(SK(k - 3), SK(k - 2), SK(k - 1), SK(k), SK(k + 1), use_weno, weps);
                    else if (use_weno)
                        r = upstrpd(SK(k + 1), SK(k), SK(k - 1), wepsf);
                    else
                        r = flx3(SK(k + 1), SK(k), SK(k - 1));
                } else {
                    if (m >= 0.0f)
                        r = recon(SK(k - 3), SK(k - 2), SK(k - 1), SK(k), SK(k + 1), use_weno, weps);
                    else
                        r = recon(SK(k + 2), SK(k + 1), SK(k), SK(k - 1), SK(k - 2), use_weno, weps);
                }
#undef SK
                PW(fz, k, y, x) = m * r;
            }
        }
    }
    const float rdx = 1.0f / dx, rdy = 1.0f / dy, rdsf = 1.0f / dz;
    for (int k = 1; k <= nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                const int owned = obc != 0u || (i >= 3 && i + 3 < ni && j >= 3 && j + 3 < nj);
                if (!owned) continue;
                C3(a->tendency, k - 1, j, i) =
                    tendency_cell(a, fx, fy, fz, ni, nj, nk, k, j, i, obc, rdx, rdy, rdsf, vc);
            }
}

void oracle_scalar_advection5(const scalar_adv_arrays *a, int ni, int nj, int nk, int use_weno, float dx, float dy,
                              float dz, double weps, unsigned obc) {
    scalar_advection5_column(a, ni, nj, nk, use_weno, dx, dy, dz, weps, obc, &kUniformColumn);
}

/* launch_cuda_gm1_child_stretched_scalar_advection5
 * (src/cm1core/cuda_gm1_child_stretched_scalar.py:666-842): the same face
 * fluxes with the tendency's vertical derivative on a stretched column,
 * mode 1 (terrain branch, rdsf(k)) or mode 2 (flat, rdz*mh(k), rr0(k)). */
void oracle_scalar_advection5_column(const scalar_adv_arrays *a, int ni, int nj, int nk, int use_weno, float dx,
                                     float dy, double weps, unsigned obc, int mode, const float *rdsf,
                                     const float *mh, float rdz) {
    const vertical_column vc = {mode, rdsf, mh, rdz};
    scalar_advection5_column(a, ni, nj, nk, use_weno, dx, dy, 1.0f, weps, obc, &vc);
}
