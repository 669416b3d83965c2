/*
 * kessler_oracle.c - CPU restatement of the reference's complete Kessler
 * warm-rain operator (ptype = 1, efall = 0): pdefq(qv, qc, qr), rain fall
 * speed and rain-energy budget, fallout sub-stepping, local conversion
 * (autoconversion, accretion, evaporation) and saturation adjustment, with
 * the FP64 budgets.  TEST INFRASTRUCTURE ONLY: the checker for the CUDA
 * library.
 *
 * Followed functions (reference file:line):
 *   _constants                      src/cm1core/cuda_gm1_kessler_driver.py:277-297
 *   _cpu_pdefq                      src/cm1core/cuda_gm1_kessler_driver.py:300-335
 *   _cpu_satadj                     src/cm1core/cuda_gm1_kessler_driver.py:337-428
 *   cpu_gm1_kessler_driver_inplace  src/cm1core/cuda_gm1_kessler_driver.py:431-559
 *   cpu_gm1_kessler_local_inplace   src/cm1core/cuda_gm1_kessler_local.py:251-432
 *
 * Arithmetic: binary32 one operation at a time (-ffp-contract=off), FP64
 * budget sums in the twin's loop order.  powf/expf are the C library's; the
 * twin's are NumPy's, and the CUDA library's are CUDA's, so words that pass
 * through a power or an exponential agree within a few ULPs, not bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "real.h"

typedef struct {
    /* inputs */
    const float *ruh, *rvh, *rmh, *mh, *pi0, *th0, *rr;
    /* in/out */
    float *rho, *pp3d, *th3d, *prs, *qv, *qc, *qr, *fall_velocity, *rain, *prate;
    double *asq, *qbudget;
    /* optional outputs (may be NULL) */
    uint32_t *satadj_iterations;
} kessler_arrays;

#define CELL(p, k, j, i) (p)[((size_t)(k) * nj + (size_t)(j)) * ni + (size_t)(i)]

typedef struct {
    float rd, cp, cpv, rv, xlv, cv, cvv, rovcp, eps, reps, cpl, lv2, lv1, rp00, cpdcv, rddcv, cpdrd, p00;
} kconst;

static kconst constants(void) {
    kconst c;
    c.rd = 287.04f;
    c.cp = 1005.7f;
    c.cpv = 1870.0f;
    c.rv = 461.5f;
    c.xlv = 2501000.0f;
    c.cv = c.cp - c.rd;
    c.cvv = c.cpv - c.rv;
    c.rovcp = c.rd / c.cp;
    c.eps = c.rd / c.rv;
    c.reps = c.rv / c.rd;
    c.cpl = 4190.0f;
    c.lv2 = c.cpl - c.cpv;
    c.lv1 = c.xlv + c.lv2 * 273.15f;
    c.p00 = 1.0e5f;
    c.rp00 = 1.0f / c.p00;
    c.cpdcv = c.cp / c.cv;
    c.rddcv = c.rd / c.cv;
    c.cpdrd = c.cp / c.rd;
    return c;
}

static inline float fmaxf_py(float a, float b) { return (b > a) ? b : a; } /* Python max(a, b) */
static inline float fminf_py(float a, float b) { return (b < a) ? b : a; } /* Python min(a, b) */

static void pdefq(const kessler_arrays *a, float *q, float rmax, int ni, int nj, int nk, double volume,
                  double *asq_slot) {
    for (int j = 0; j < nj; ++j) {
        double budj = 0.0;
        for (int i = 0; i < ni; ++i) {
            double t1 = 0.0, t2 = 0.0, a1 = 0.0, a2 = 0.0;
            for (int k = 0; k < nk; ++k) {
                const float rho = CELL(a->rho, k, j, i);
                float rq = rho * CELL(q, k, j, i);
                t1 += (double)rq;
                float cell = (((rho * CELL(q, k, j, i)) * a->ruh[i]) * a->rvh[j]) * CELL(a->rmh, k, j, i);
                a1 += (double)cell;
                if (CELL(q, k, j, i) < rmax) CELL(q, k, j, i) = 0.0f;
                t2 += (double)(rho * CELL(q, k, j, i));
            }
            double t3 = (t1 + 1.0e-20) / (t2 + 1.0e-20);
            if (t3 < 0.0) t3 = 1.0;
            for (int k = 0; k < nk; ++k) {
                const float rho = CELL(a->rho, k, j, i);
                CELL(q, k, j, i) = (float)(t3 * (double)CELL(q, k, j, i));
                float cell = (((rho * CELL(q, k, j, i)) * a->ruh[i]) * a->rvh[j]) * CELL(a->rmh, k, j, i);
                a2 += (double)cell;
            }
            budj += a2 - a1;
        }
        *asq_slot += budj * volume;
    }
}

/* saturation vapour pressure (Bolton) capped at half the pressure */
static inline float esl_capped(float t, float prs) {
    float esl = 611.2f * expf((17.67f * (t - 273.15f)) / (t - 29.65f));
    return fminf_py(esl, prs * 0.5f);
}

/* returns the number of cells that failed to converge */
static int local_and_satadj(const kessler_arrays *a, int ni, int nj, int nk, float dx, float dy, float dz, float dt,
                            int eqtset) {
    const kconst c = constants();
    double *bud = calloc((size_t)5 * nk, sizeof(double));
    int failures = 0;
    /* local conversion over every cell (cpu_gm1_kessler_local_inplace) */
    for (int k = 0; k < nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                float pisum = CELL(a->pi0, k, j, i) + CELL(a->pp3d, k, j, i);
                const float tmp = (CELL(a->th0, k, j, i) + CELL(a->th3d, k, j, i)) * pisum;
                float qvnew = CELL(a->qv, k, j, i), qcnew = CELL(a->qc, k, j, i), qrnew = CELL(a->qr, k, j, i);
                float ar = 0.0f, cr = 0.0f, er = 0.0f;
                const float prs = CELL(a->prs, k, j, i), rho = CELL(a->rho, k, j, i);
                if (qcnew > 0.0f) {
                    ar = fmaxf_py(0.001f * (qcnew - 0.001f), 0.0f);
                    ar = ar * dt;
                }
                if (qcnew > 0.0f && qrnew > 0.0f) cr = ((2.2f * qcnew) * powf(qrnew, 0.875f)) * dt;
                if (qrnew > 0.0f) {
                    const float esl = esl_capped(tmp, prs);
                    const float qvs = (c.eps * esl) / (prs - esl);
                    if (qvnew < qvs) {
                        const float rhoqr = rho * qrnew;
                        const float vent = 1.6f + 30.3922f * powf(rhoqr, 0.2046f);
                        const float deficit = 1.0f - qvnew / qvs;
                        const float num = (vent * deficit) * powf(rhoqr, 0.525f);
                        const float den = (2.03e4f + 9.584e6f / (qvs * prs)) * rho;
                        er = fminf_py((num / den) * dt, qrnew);
                        if (qvnew + er > qvs) er = qvs - qvnew;
                    }
                }
                if (ar + cr > qcnew) {
                    const float term1 = ar + cr;
                    ar = (qcnew * ar) / term1;
                    cr = (qcnew * cr) / term1;
                }
                qvnew = qvnew + er;
                qcnew = qcnew - (ar + cr);
                qrnew = qrnew + ((ar + cr) - er);
                if (er > 1.0e-7f) {
                    if (eqtset == 2) {
                        const float cpml = (c.cp + c.cpv * qvnew) + c.cpl * (qcnew + qrnew);
                        const float cvml = (c.cv + c.cvv * qvnew) + c.cpl * (qcnew + qrnew);
                        const float rm = c.rd + c.rv * qvnew;
                        const float latent = c.lv1 - c.lv2 * tmp;
                        const float first = latent / ((c.cpdcv * cvml) * pisum);
                        const float second = ((CELL(a->th0, k, j, i) + CELL(a->th3d, k, j, i)) * (c.rv / cvml)) *
                                             (1.0f - (c.rovcp * cpml) / rm);
                        CELL(a->th3d, k, j, i) = CELL(a->th3d, k, j, i) - er * (first - second);
                        const float base = ((rho * rm) * (CELL(a->th0, k, j, i) + CELL(a->th3d, k, j, i))) * c.rp00;
                        CELL(a->pp3d, k, j, i) = powf(base, c.rddcv) - CELL(a->pi0, k, j, i);
                        pisum = CELL(a->pi0, k, j, i) + CELL(a->pp3d, k, j, i);
                        CELL(a->prs, k, j, i) = c.p00 * powf(pisum, c.cpdrd);
                    } else {
                        const float latent = c.lv1 - c.lv2 * tmp;
                        CELL(a->th3d, k, j, i) = CELL(a->th3d, k, j, i) - er * (latent / (c.cp * pisum));
                        const float den = ((c.rd * (CELL(a->th0, k, j, i) + CELL(a->th3d, k, j, i))) * pisum) *
                                          (1.0f + qvnew * c.reps);
                        CELL(a->rho, k, j, i) = prs / den;
                    }
                }
                const float tem = (a->ruh[i] * a->rvh[j]) * CELL(a->rmh, k, j, i);
                const float rr = CELL(a->rr, k, j, i);
                bud[0 * nk + k] += (double)((rr * ar) * tem);
                bud[1 * nk + k] += (double)((rr * cr) * tem);
                bud[2 * nk + k] += (double)((rr * er) * tem);
                CELL(a->qv, k, j, i) = qvnew;
                CELL(a->qc, k, j, i) = qcnew;
                CELL(a->qr, k, j, i) = qrnew;
            }
    const double volume = (double)((dx * dy) * dz);
    for (int p = 0; p < 3; ++p)
        for (int k = 0; k < nk; ++k) a->qbudget[2 + p] = a->qbudget[2 + p] + bud[p * nk + k] * volume;
    /* saturation adjustment over every cell (_cpu_satadj) */
    const float converge = 2.0f * 0.0001f;
    for (int k = 0; k < nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                const float old_qv = CELL(a->qv, k, j, i), old_qc = CELL(a->qc, k, j, i);
                float qvnew = old_qv, qcnew = old_qc;
                const float prs = CELL(a->prs, k, j, i), rho = CELL(a->rho, k, j, i);
                float tnew = (CELL(a->th0, k, j, i) + CELL(a->th3d, k, j, i)) *
                             (CELL(a->pi0, k, j, i) + CELL(a->pp3d, k, j, i));
                float esl = esl_capped(tnew, prs);
                float qvs = (c.eps * esl) / (prs - esl);
                uint32_t iterations = 0;
                if (eqtset == 2) {
                    if (old_qc > 1.0e-12f || old_qv > qvs) {
                        const float ql = fmaxf_py(old_qc + CELL(a->qr, k, j, i), 0.0f);
                        const float cvml = (c.cv + c.cvv * qvnew) + c.cpl * ql;
                        const float lhv = c.lv1 - c.lv2 * tnew;
                        const float t1 = (lhv - c.rv * tnew) / cvml;
                        const float d1 = (t1 * 17.67f) * 243.5f;
                        float tlast = tnew, pnew = prs;
                        int n = 0;
                        for (;;) {
                            n += 1;
                            const float denom = 1.0f + (d1 * qvs) / ((tnew - 29.65f) * (tnew - 29.65f));
                            float dqv = (qvs - qvnew) / denom;
                            dqv = fminf_py(dqv, qcnew);
                            if (qvnew + dqv < 1.0e-20f) dqv = 1.0e-20f - qvnew;
                            qvnew = qvnew + dqv;
                            qcnew = qcnew - dqv;
                            tnew = tnew - dqv * t1;
                            pnew = (rho * (c.rd + c.rv * qvnew)) * tnew;
                            const int conv = fabs((double)(tnew - tlast)) <= (double)converge;
                            if (!conv) {
                                tlast = tnew;
                                esl = esl_capped(tnew, prs);
                                qvs = (c.eps * esl) / (pnew - esl);
                            }
                            if (n == 100) { /* the twin fails at the 100th pass, converged or not */
                                failures += 1;
                                break;
                            }
                            if (conv) break;
                        }
                        iterations = (uint32_t)n;
                        CELL(a->prs, k, j, i) = pnew;
                        CELL(a->pp3d, k, j, i) = powf(pnew * c.rp00, c.rovcp) - CELL(a->pi0, k, j, i);
                        CELL(a->th3d, k, j, i) =
                            tnew / (CELL(a->pi0, k, j, i) + CELL(a->pp3d, k, j, i)) - CELL(a->th0, k, j, i);
                        CELL(a->qv, k, j, i) = qvnew;
                        CELL(a->qc, k, j, i) = qcnew;
                    }
                } else {
                    const float lhv = c.lv1 - c.lv2 * tnew;
                    const float square = (tnew - 29.65f) * (tnew - 29.65f);
                    const float numerator = ((lhv * qvs) * 17.67f) * 243.5f;
                    float dqv = (qvs - qvnew) / (1.0f + numerator / (c.cp * square));
                    if (qvnew + dqv < 1.0e-20f) dqv = 1.0e-20f - qvnew;
                    dqv = fminf_py(dqv, fmaxf_py(0.0f, qcnew));
                    qvnew = qvnew + dqv;
                    qcnew = qcnew - dqv;
                    iterations = 1;
                    CELL(a->th3d, k, j, i) =
                        CELL(a->th3d, k, j, i) -
                        dqv * (lhv / (c.cp * (CELL(a->pi0, k, j, i) + CELL(a->pp3d, k, j, i))));
                    CELL(a->qv, k, j, i) = qvnew;
                    CELL(a->qc, k, j, i) = qcnew;
                    const float den = ((c.rd * (CELL(a->th0, k, j, i) + CELL(a->th3d, k, j, i))) *
                                       (CELL(a->pi0, k, j, i) + CELL(a->pp3d, k, j, i))) *
                                      (1.0f + qvnew * c.reps);
                    CELL(a->rho, k, j, i) = CELL(a->prs, k, j, i) / den;
                }
                if (a->satadj_iterations) CELL(a->satadj_iterations, k, j, i) = iterations;
                const float cond = fmaxf_py(qcnew - old_qc, 0.0f);
                const float evac = fmaxf_py(qvnew - old_qv, 0.0f);
                const float tem = (a->ruh[i] * a->rvh[j]) * CELL(a->rmh, k, j, i);
                bud[3 * nk + k] += (double)((CELL(a->rr, k, j, i) * cond) * tem);
                bud[4 * nk + k] += (double)((CELL(a->rr, k, j, i) * evac) * tem);
            }
    for (int k = 0; k < nk; ++k) a->qbudget[0] += bud[3 * nk + k] * volume;
    for (int k = 0; k < nk; ++k) a->qbudget[1] += bud[4 * nk + k] * volume;
    free(bud);
    return failures;
}

/* Returns the largest fallout sub-step count (>= 1), or -1 (bad arguments),
 * or -(100 + failures) when saturation adjustment did not converge. */
int oracle_kessler_driver(const kessler_arrays *a, int ni, int nj, int nk, float dx, float dy, float dz, float dt,
                          int eqtset, int32_t *nfall_out) {
    if (ni < 1 || nj < 1 || nk < 1 || (eqtset != 1 && eqtset != 2)) return -1;
    const kconst c = constants();
    float *temperature = malloc((size_t)ni * nj * nk * sizeof(float));
    for (int k = 0; k < nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i)
                CELL(temperature, k, j, i) = (CELL(a->th0, k, j, i) + CELL(a->th3d, k, j, i)) *
                                             (CELL(a->pi0, k, j, i) + CELL(a->pp3d, k, j, i));
    const double pdef_volume = (double)((dx * dy) * dz);
    pdefq(a, a->qv, 0.0f, ni, nj, nk, pdef_volume, &a->asq[0]);
    pdefq(a, a->qc, 1.0e-14f, ni, nj, nk, pdef_volume, &a->asq[1]);
    pdefq(a, a->qr, 1.0e-14f, ni, nj, nk, pdef_volume, &a->asq[2]);
    for (int k = 0; k < nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                float velocity = 0.0f;
                const float rho = CELL(a->rho, k, j, i), qr = CELL(a->qr, k, j, i);
                if (qr > 1.0e-12f) velocity = (14.34f * powf(rho * qr, 0.1346f)) * sqrtf(1.15f / rho);
                CELL(a->fall_velocity, k, j, i) = velocity;
            }
    for (int j = 0; j < nj; ++j) {
        double bud = 0.0;
        for (int i = 0; i < ni; ++i) {
            float term = dt * CELL(a->fall_velocity, 0, j, i);
            term = term * CELL(a->rr, 0, j, i);
            term = term * CELL(a->qr, 0, j, i);
            term = term * (c.cpl * CELL(temperature, 0, j, i) - c.lv1);
            term = term * a->ruh[i];
            term = term * a->rvh[j];
            bud += (double)term;
        }
        a->qbudget[6] += bud * (double)dx * (double)dy;
    }
    const float rdz = 1.0f / dz;
    int max_nfall = 1;
    const double area = (double)(dx * dy);
    float *rq = malloc((size_t)(nk + 1) * sizeof(float));
    for (int j = 0; j < nj; ++j) {
        double bud = 0.0;
        for (int i = 0; i < ni; ++i) {
            float crmax = 0.0f;
            for (int k = 0; k < nk; ++k)
                crmax = fmaxf_py(crmax, ((CELL(a->fall_velocity, k, j, i) * dt) * rdz) * CELL(a->mh, k, j, i));
            int nfall = (int)(crmax + 1.0f);
            if (nfall < 1) nfall = 1;
            if (nfall_out) nfall_out[(size_t)j * ni + i] = nfall;
            if (nfall > max_nfall) max_nfall = nfall;
            for (int k = nk - 2; k >= 0; --k)
                if (CELL(a->qr, k, j, i) < 1.0e-8f) CELL(a->fall_velocity, k, j, i) = CELL(a->fall_velocity, k + 1, j, i);
            const float dtfall = dt / (float)nfall;
            for (int n = 0; n < nfall; ++n) {
                for (int k = 0; k < nk; ++k)
                    rq[k] = (CELL(a->rho, k, j, i) * CELL(a->fall_velocity, k, j, i)) *
                            fmaxf_py(0.0f, CELL(a->qr, k, j, i));
                rq[nk] = 0.0f;
                for (int k = 0; k < nk; ++k) {
                    const float delta =
                        (((dtfall * (rq[k + 1] - rq[k])) * rdz) * CELL(a->mh, k, j, i)) / CELL(a->rho, k, j, i);
                    CELL(a->qr, k, j, i) = CELL(a->qr, k, j, i) + delta;
                }
                a->rain[(size_t)j * ni + i] = a->rain[(size_t)j * ni + i] + (0.1f * dtfall) * rq[0];
                a->prate[(size_t)j * ni + i] = rq[0];
                float term = dtfall * CELL(a->rr, 0, j, i);
                term = term * CELL(a->fall_velocity, 0, j, i);
                term = term * fmaxf_py(0.0f, CELL(a->qr, 0, j, i));
                term = term * a->ruh[i];
                term = term * a->rvh[j];
                bud += (double)term;
            }
        }
        a->qbudget[5] += bud * area;
    }
    free(rq);
    free(temperature);
    const int failures = local_and_satadj(a, ni, nj, nk, dx, dy, dz, dt, eqtset);
    if (failures) return -(100 + failures);
    return max_nfall;
}

/* cpu_gm1_kessler_large_step_inplace (src/cm1core/cuda_gm1_kessler_large_step.py:183-292):
 * equation-set-2 held remove/snapshot, pre-physics EOS (numpy float32 power:
 * libm powf), rr = rho, the driver, held recapture.  held[0..3] = qpten,
 * qtten, qvten, qcten (ignored for equation set 1).  Returns the driver's
 * result. */
/* ---------------------------------------------------------------------------
 * The final-RK dry-air mass correction, apmasscon = 1: cpu_initial_dry_mass
 * and cpu_apmasscon_inplace (src/cm1core/cuda_apmasscon.py:190-325): per
 * level the twin's serial binary64 sums of ((rho*ruh)*rvh)*rmh and of
 * pi0 + pp3d, the levels summed in order, the binary64 correction, then
 * pp3d += correction and prs, rho from the equation of state.
 * ------------------------------------------------------------------------- */
static void mass_layers(const float *rho, const float *ruh, const float *rvh, const float *rmh, const float *pi0,
                        const float *pp3d, int ni, int nj, int nk, double *dry, double *pis) {
    for (int k = 0; k < nk; ++k) {
        double d = 0.0, p = 0.0;
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                const size_t q = ((size_t)k * nj + j) * ni + i;
                float term = rho[q] * ruh[i];
                term = term * rvh[j];
                term = term * rmh[q];
                d = d + (double)term;
                if (pis != NULL) p = p + (double)(pi0[q] + pp3d[q]);
            }
        dry[k] = d;
        if (pis != NULL) pis[k] = p;
    }
}

double oracle_dry_mass(const float *rho, const float *ruh, const float *rvh, const float *rmh, int ni, int nj,
                       int nk) {
    double *dry = malloc(sizeof(double) * (size_t)nk);
    if (dry == NULL) return -1.0;
    mass_layers(rho, ruh, rvh, rmh, NULL, NULL, ni, nj, nk, dry, NULL);
    double total = 0.0;
    for (int k = 0; k < nk; ++k) total = total + dry[k];
    free(dry);
    return total;
}

/* diag: mass2, the Exner sum, the binary64 correction, mass1 */
int oracle_apmasscon(const float *ruh, const float *rvh, const float *rmh, const float *pi0, const float *th0,
                     const float *th3d, const float *qv, float *pp3d, float *prs, float *rho, float *rr, int ni,
                     int nj, int nk, double mass1, double *diag) {
    double *dry = malloc(sizeof(double) * (size_t)nk), *pis = malloc(sizeof(double) * (size_t)nk);
    if (dry == NULL || pis == NULL) {
        free(dry);
        free(pis);
        return -1;
    }
    mass_layers(rho, ruh, rvh, rmh, pi0, pp3d, ni, nj, nk, dry, pis);
    double mass2 = 0.0, psum = 0.0;
    for (int k = 0; k < nk; ++k) {
        mass2 = mass2 + dry[k];
        psum = psum + pis[k];
    }
    free(dry);
    free(pis);
    const float cp = 1005.7f, rd = 287.04f, rv = 461.5f;
    const float cv = cp - rd;
    const float rddcv = rd / cv;
    const float cpdrd = cp / rd;
    double value = pow(mass1 / mass2, (double)rddcv) - 1.0;
    value = value * psum;
    value = value / (double)((size_t)ni * nj * nk);
    const float corr = (float)value;
    if (diag != NULL) {
        diag[0] = mass2;
        diag[1] = psum;
        diag[2] = value;
        diag[3] = mass1;
    }
    const size_t n = (size_t)ni * nj * nk;
    for (size_t q = 0; q < n; ++q) {
        pp3d[q] = pp3d[q] + corr;
        const float pi = pi0[q] + pp3d[q];
        const float pressure = 100000.0f * powf(pi, cpdrd);
        const float theta = th0[q] + th3d[q];
        float vapor = qv[q] > 0.0f ? qv[q] : 0.0f;
        if (qv[q] != qv[q]) vapor = qv[q];
        const float gas = rd + vapor * rv;
        float den = theta * pi;
        den = den * gas;
        prs[q] = pressure;
        rho[q] = pressure / den;
        if (rr != NULL) rr[q] = rho[q];
    }
    return 0;
}

int oracle_kessler_large_step_mass(const kessler_arrays *a, float *const held[4], int ni, int nj, int nk, float dx,
                                   float dy, float dz, float dt, int eqtset, int *nfall, const double *mass1,
                                   double *diag);

/* the Kessler large step with the mass correction between the pre-physics
 * equation of state and the driver */
int oracle_kessler_large_step_apmasscon(const kessler_arrays *a, float *const held[4], int ni, int nj, int nk,
                                        float dx, float dy, float dz, float dt, int eqtset, int *nfall,
                                        const double *mass1, double *diag) {
    return oracle_kessler_large_step_mass(a, held, ni, nj, nk, dx, dy, dz, dt, eqtset, nfall, mass1, diag);
}

int oracle_kessler_large_step(const kessler_arrays *a, float *const held[4], int ni, int nj, int nk, float dx,
                              float dy, float dz, float dt, int eqtset, int *nfall) {
    return oracle_kessler_large_step_mass(a, held, ni, nj, nk, dx, dy, dz, dt, eqtset, nfall, NULL, NULL);
}

int oracle_kessler_large_step_mass(const kessler_arrays *a, float *const held[4], int ni, int nj, int nk, float dx,
                                   float dy, float dz, float dt, int eqtset, int *nfall, const double *mass1,
                                   double *diag) {
    const size_t n = (size_t)ni * nj * nk;
    float *state[4] = {a->pp3d, a->th3d, a->qv, a->qc};
    if (eqtset == 2)
        for (int s = 0; s < 4; ++s)
            for (size_t q = 0; q < n; ++q) {
                const float w = held[s][q] * dt;
                state[s][q] = state[s][q] - w;
                held[s][q] = state[s][q];
            }
    const float cpdrd = (float)((double)1005.7f / (double)287.04f);
    for (size_t q = 0; q < n; ++q) {
        const float pi = a->pi0[q] + a->pp3d[q];
        float prs = powf(pi, cpdrd);
        prs = prs * 100000.0f;
        float rho = a->th0[q] + a->th3d[q];
        rho = rho * pi;
        float w = a->qv[q] > 0.0f ? a->qv[q] : 0.0f;
        if (a->qv[q] != a->qv[q]) w = a->qv[q];
        w = w * 461.5f;
        w = w + 287.04f;
        rho = rho * w;
        rho = prs / rho;
        a->prs[q] = prs;
        a->rho[q] = rho;
        ((float *)a->rr)[q] = rho;
    }
    if (mass1 != NULL && oracle_apmasscon(a->ruh, a->rvh, a->rmh, a->pi0, a->th0, a->th3d, a->qv, a->pp3d, a->prs,
                                          a->rho, (float *)a->rr, ni, nj, nk, *mass1, diag) != 0)
        return -1;
    const int r = oracle_kessler_driver(a, ni, nj, nk, dx, dy, dz, dt, eqtset, nfall);
    if (r < 0 || eqtset != 2) return r;
    for (int s = 0; s < 4; ++s)
        for (size_t q = 0; q < n; ++q) held[s][q] = (state[s][q] - held[s][q]) / dt;
    return r;
}
