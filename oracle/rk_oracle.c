/*
 * rk_oracle.c - CPU restatement of the reference's scalar/moisture RK stage
 * pieces on the padded (ng = 3) lane: the theta transport packing, the
 * A-anchored RK composition and one positive-definite (pdef) direction pass.
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library.
 *
 * Followed functions (reference file:line):
 *   cpu_theta_transport_scalar_inplace          src/cm1core/cuda_scalar_moist_rk.py:255-280
 *   cpu_compose_scalar_moist_rk_stage_inplace   src/cm1core/cuda_scalar_moist_rk.py:283-349
 *   cpu_pdef_direction_inplace                  src/cm1core/cuda_scalar_moist_rk.py:352-518
 *
 * Arithmetic: binary32 one operation at a time (-ffp-contract=off).  The pdef
 * line repair is restated in the twin's own sequential form (one pass along
 * each line in index order).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "real.h"

#define NG 3
#define SMEPS 0x1.4484cp-100f /* 1e-30 */

void oracle_theta_pack(const float *th0, const float *th3d, float *padded, int ni, int nj, int nk) {
    const size_t sx = (size_t)ni + 2 * NG, sy = (size_t)nj + 2 * NG;
    for (int k = 0; k < nk; ++k) {
        const float base = th0[k] - 300.0f;
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i)
                padded[((size_t)(k + 1) * sy + (size_t)(j + NG)) * sx + (size_t)(i + NG)] =
                    base + th3d[((size_t)k * nj + j) * ni + i];
    }
}

void oracle_rk_compose(const float *theta_a, const float *theta_held, const float *theta_divterm,
                       const float *theta_adv, float *theta_cur, const float *q_a, const float *q_held,
                       const float *q_adv, float *q_cur, size_t cells, int nq, float dttmp) {
    for (size_t p = 0; p < cells; ++p) {
        const float seed = theta_held[p] - theta_divterm[p];
        const float total = seed + theta_adv[p];
        float out = theta_a[p] + dttmp * total;
        if (fabsf(out) < SMEPS) out = 0.0f;
        theta_cur[p] = out;
    }
    for (size_t p = 0; p < cells * (size_t)nq; ++p) {
        const float total = q_held[p] + q_adv[p];
        float out = q_a[p] + dttmp * total;
        if (fabsf(out) < SMEPS) out = 0.0f;
        q_cur[p] = out;
    }
}

/* axis: 0 = x, 1 = y, 2 = z */
void oracle_pdef_direction(const float *scalar_a, const float *scalar_padded, const float *rho0, const float *gz,
                           const float *rgz, const float *mass_flux, float *directional, float *candidate, int ni,
                           int nj, int nk, int axis, float dt, float spacing) {
    const size_t sx = (size_t)ni + 2 * NG, sy = (size_t)nj + 2 * NG;
    const size_t ux = (size_t)ni + 1 + 2 * NG, vy = (size_t)nj + 1 + 2 * NG;
    const float rdt = 1.0f / dt;
    const float rs = 1.0f / spacing;
#define C3(k, j, i) (((size_t)(k) * nj + (size_t)(j)) * ni + (size_t)(i))
#define SP(k, y, x) scalar_padded[((size_t)(k) * sy + (size_t)(y)) * sx + (size_t)(x)]
    /* face difference of the mass flux along the axis at cell (k, j, i) */
#define DIFF(k, j, i)                                                                                         \
    (axis == 0 ? mass_flux[((size_t)((k) + 1) * sy + (size_t)((j) + NG)) * ux + (size_t)((i) + NG + 1)] -       \
                     mass_flux[((size_t)((k) + 1) * sy + (size_t)((j) + NG)) * ux + (size_t)((i) + NG)]       \
     : axis == 1 ? mass_flux[((size_t)((k) + 1) * vy + (size_t)((j) + NG + 1)) * sx + (size_t)((i) + NG)] -     \
                       mass_flux[((size_t)((k) + 1) * vy + (size_t)((j) + NG)) * sx + (size_t)((i) + NG)]     \
                 : mass_flux[((size_t)((k) + 2) * sy + (size_t)((j) + NG)) * sx + (size_t)((i) + NG)] -       \
                       mass_flux[((size_t)((k) + 1) * sy + (size_t)((j) + NG)) * sx + (size_t)((i) + NG)])
    for (int k = 0; k < nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                const float difference = DIFF(k, j, i);
                const float divergence = (SP(k + 1, j + NG, i + NG) * difference) * rs;
                const float total = directional[C3(k, j, i)] + divergence;
                const float increment = (dt * total) * gz[(size_t)j * ni + i];
                candidate[C3(k, j, i)] = rho0[C3(k, j, i)] * scalar_a[C3(k, j, i)] + increment;
            }
    const int length = axis == 0 ? ni : (axis == 1 ? nj : nk);
    const int nlines = axis == 0 ? nk * nj : (axis == 1 ? nk * ni : nj * ni);
    float *values = malloc((size_t)length * sizeof(float));
    float *mass = malloc((size_t)length * sizeof(float));
    unsigned char *flags = malloc((size_t)length);
    for (int line = 0; line < nlines; ++line) {
        int a0, a1;
        if (axis == 0) { a0 = line / nj; a1 = line % nj; }       /* k, j */
        else if (axis == 1) { a0 = line / ni; a1 = line % ni; }  /* k, i */
        else { a0 = line / ni; a1 = line % ni; }                 /* j, i */
#define LINE_CELL(idx) (axis == 0 ? C3(a0, a1, (idx)) : axis == 1 ? C3(a0, (idx), a1) : C3((idx), a0, a1))
        for (int q = 0; q < length; ++q) {
            values[q] = candidate[LINE_CELL(q)];
            mass[q] = 0.0f;
            flags[q] = 0;
        }
        const int start = axis == 2 ? 0 : 1;
        const int stop = axis == 2 ? length : length - 1;
        for (int index = start; index < stop; ++index) {
            const float center = values[index];
            if (center >= 0.0f) continue;
            const float left = index == 0 ? 0.0f : fmaxf(0.0f, values[index - 1]);
            const float right = index + 1 == length ? 0.0f : fmaxf(0.0f, values[index + 1]);
            const float donor = left + right;
            if (donor <= SMEPS) continue;
            const float ratio = fmaxf(center, 0.0f - donor) / donor;
            if (index > 0) {
                mass[index - 1] = mass[index - 1] + left * ratio;
                if (values[index - 1] > SMEPS) flags[index - 1] = 1;
            }
            mass[index] = mass[index] - donor * ratio;
            flags[index] = 1;
            if (index + 1 < length) {
                mass[index + 1] = mass[index + 1] + right * ratio;
                if (values[index + 1] > SMEPS) flags[index + 1] = 1;
            }
        }
        for (int q = 0; q < length; ++q) {
            if (!flags[q]) continue;
            int k, j, i;
            if (axis == 0) { k = a0; j = a1; i = q; }
            else if (axis == 1) { k = a0; j = q; i = a1; }
            else { k = q; j = a0; i = a1; }
            const float difference = DIFF(k, j, i);
            const float divergence = (SP(k + 1, j + NG, i + NG) * difference) * rs;
            float adjusted = (candidate[C3(k, j, i)] + mass[q]) - rho0[C3(k, j, i)] * scalar_a[C3(k, j, i)];
            adjusted = (adjusted * rdt) * rgz[(size_t)j * ni + i];
            directional[C3(k, j, i)] = adjusted - divergence;
        }
#undef LINE_CELL
    }
    free(values);
    free(mass);
    free(flags);
#undef DIFF
#undef SP
#undef C3
}

/*
 * eqtset=2 stage terms of one cell (cpu_eqtset2_cell_f32,
 * src/cm1core/cuda_moist_stage_bridge.py:62-139): buoyancy, theta-rho,
 * theta and pressure energy terms.  q = {qv, qc, qr, qi, qs, qg}.
 */
void oracle_eqtset2_cell(float th0, float qv0, float pi0, float qc0, float qi0, float th3d, float pp3d,
                         const float q[6], float out[4]) {
    const float rd = 287.04f, rv = 461.5f, cp = 1005.7f, cpv = 1870.0f, cpl = 4190.0f, cpi = 2106.0f, g = 9.81f;
    const float cv = cp - rd, cvv = cpv - rv, rovcp = rd / cp, reps = rv / rd;
    const float repsm1 = reps - 1.0f;
    const float qv = fmaxf(q[0], 0.0f);
    const float liquid = q[1] + q[2];
    const float ice = (q[3] + q[4]) + q[5];
    const float qli = fmaxf(liquid + ice, 0.0f);
    const float cpli = cpl * fmaxf(liquid, 0.0f) + cpi * fmaxf(ice, 0.0f);
    const float theta = th0 + th3d;
    float b = th3d * (1.0f / th0) + repsm1 * (qv - qv0);
    b = g * (b - ((qli - qc0) - qi0));
    const float theta_rho = (theta * (1.0f + reps * qv)) / ((1.0f + qv) + qli);
    const float cpm = (cp + cpv * qv) + cpli;
    const float cvm = 1.0f / ((cv + cvv * qv) + cpli);
    const float theta_term = (theta * ((rd + rv * qv) - rovcp * cpm)) * cvm;
    const float pressure_term = (((pi0 + pp3d) * rovcp) * cpm) * cvm;
    out[0] = b;
    out[1] = theta_rho;
    out[2] = theta_term;
    out[3] = pressure_term;
}

/* the eqtset=2 stage-terms pass over the padded lane
 * (launch_cuda_eqtset2_stage_terms, src/cm1core/cuda_moist_stage_bridge.py:378-430):
 * live cells give buoyancy (scalar layout), thv and ppterm (pressure box)
 * and thterm (compact); every cell of the pressure box gets piadv from the
 * nearest live base-state column.  Base profiles (nk), qc0 = qi0 = 0. */
void oracle_eqtset2_stage_terms(int ni, int nj, int nk, const float *th0, const float *qv0, const float *pi0,
                                const float *th3d, const float *q3d, const float *pp3d, float *thv, float *ppterm,
                                float *buoyancy, float *thterm, float *piadv) {
    const size_t n = (size_t)ni * nj * nk;
    for (int k = 0; k < nk; ++k)
        for (int y = 0; y < nj + 2; ++y)
            for (int x = 0; x < ni + 2; ++x) {
                const size_t pp = ((size_t)(k + 1) * (nj + 2) + y) * (size_t)(ni + 2) + x;
                piadv[pp] = pi0[k] + pp3d[pp];
                if (x < 1 || x > ni || y < 1 || y > nj) continue;
                const size_t cell = ((size_t)k * nj + (y - 1)) * (size_t)ni + (x - 1);
                float q[6];
                for (int r = 0; r < 6; ++r) q[r] = q3d[(size_t)r * n + cell];
                float out[4];
                oracle_eqtset2_cell(th0[k], qv0[k], pi0[k], 0.0f, 0.0f, th3d[cell], pp3d[pp], q, out);
                buoyancy[((size_t)(k + 1) * (nj + 6) + (y + 2)) * (size_t)(ni + 6) + (x + 2)] = out[0];
                thv[pp] = out[1];
                thterm[cell] = out[2];
                ppterm[pp] = out[3];
            }
}
