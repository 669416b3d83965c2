// weno.cuh - the fifth-order WENO-Z reconstruction and the positive-definite
// third-order upwind closure shared by the scalar and the TKE advection.
//
// Behaviour followed (reference file:line):
//   WENO5 with binary64 smoothness weights   src/cm1core/cuda_advection5.py:440-579,
//                                            src/cm1core/cuda_tke_evolution.py:157-165
//   upstrpd                                  src/cm1core/cuda_tke_evolution.py:168-169
// binary32 operations in the reference's order; the weights, their sum and
// the final quotient in binary64 as the reference forms them.
#pragma once

#include "gm1b_common.cuh"

namespace gm1b {

constexpr float kC13_12 = 0x1.155556p+0f;   // 13/12
constexpr float kCm7_6 = -0x1.2aaaaap+0f;   // -7/6
constexpr float kC11_6 = 0x1.d55556p+0f;    // 11/6
constexpr float kC1_6 = 0x1.555556p-3f;     // 1/6

__device__ __forceinline__ double dmin30(double x) { return x < 1.0e30 ? x : 1.0e30; }

__device__ __forceinline__ float weno5(float s1, float s2, float s3, float s4, float s5, double eps) {
    const float d1 = (s1 - 2.0f * s2) + s3;
    const float e1 = (s1 - 4.0f * s2) + 3.0f * s3;
    const float b1r = kC13_12 * (d1 * d1) + 0.25f * (e1 * e1);
    const float d2 = (s2 - 2.0f * s3) + s4;
    const float e2 = s2 - s4;
    const float b2r = kC13_12 * (d2 * d2) + 0.25f * (e2 * e2);
    const float d3 = (s3 - 2.0f * s4) + s5;
    const float e3 = (3.0f * s3 - 4.0f * s4) + s5;
    const float b3r = kC13_12 * (d3 * d3) + 0.25f * (e3 * e3);
    const double b1 = b1r, b2 = b2r, b3 = b3r;
    const double tau = fabs(b1 - b3);
    const double q1 = dmin30(tau / (b1 + eps));
    const double q2 = dmin30(tau / (b2 + eps));
    const double q3 = dmin30(tau / (b3 + eps));
    const double w1 = (double)0.1f * (1.0 + q1 * q1);
    const double w2 = (double)0.6f * (1.0 + q2 * q2);
    const double w3 = (double)0.3f * (1.0 + q3 * q3);
    const float p1 = (kF3_3 * s1 + kCm7_6 * s2) + kC11_6 * s3;
    const float p2 = (kF3_1 * s2 + kF3_2 * s3) + kF3_3 * s4;
    const float p3 = (kF3_3 * s3 + kF3_2 * s4) + kF3_1 * s5;
    return (float)((w1 * (double)p1 + w2 * (double)p2 + w3 * (double)p3) / (w1 + w2 + w3));
}

__device__ __forceinline__ float upstrpd(float s1, float s2, float s3, float weps) {
    const float dd = s2 - s1;
    const float se = copysignf(fabsf(weps), dd);
    const float rr = (s3 - s2) / (se + dd);
    const float cand = kC1_6 + kF3_3 * rr;
    const float phi = fmaxf(0.0f, fminf(rr, fminf(cand, 1.0f)));
    return s2 + phi * (s2 - s1);
}

}  // namespace gm1b
