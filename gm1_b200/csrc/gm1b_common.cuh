// gm1b_common.cuh - shared device/host helpers of libgm1b.so.
//
// Arithmetic contract (all translation units): binary32 storage, binary32
// arithmetic one operation at a time, no fused multiply-add (the library is
// compiled with --fmad=false), IEEE division (-prec-div=true), no flush to
// zero.  This is the contract of the reference kernels
// (src/cm1core/cuda_sound3_periodic.py:1097-1112, --fmad=false --ftz=false
// --prec-div=true) and lets the kernels reproduce the reference's CPU twins
// word for word.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gm1b.h"

namespace gm1b {

// binary32 constants, each the correctly rounded float32 quotient the
// reference forms at run time (src/cm1core/cuda_psolver3_trajectory.py:282-302)
constexpr float kF5_1 = 0x1.111112p-5f;   //   2/60
constexpr float kF5_2 = -0x1.bbbbbcp-3f;  // -13/60
constexpr float kF5_3 = 0x1.911112p-1f;   //  47/60
constexpr float kF5_4 = 0x1.ccccccp-2f;   //  27/60
constexpr float kF5_5 = -0x1.99999ap-5f;  //  -3/60
constexpr float kF3_1 = -0x1.555556p-3f;  //  -1/6
constexpr float kF3_2 = 0x1.aaaaaap-1f;   //   5/6
constexpr float kF3_3 = 0x1.555556p-2f;   //   2/6
constexpr float kRddcv = 0x1.98fef2p-2f;  // 287.04 / (1005.7 - 287.04)
constexpr float kGrav = 0x1.39eb86p+3f;   // 9.81
constexpr float kTh0r = 300.0f;
constexpr float kSmeps = 0x1.4484cp-100f;  // 1e-30
constexpr float kCp = 0x1.f6d99ap+9f;      // 1005.7
constexpr float kAlph = 0x1.333334p-1f;    // 0.60
constexpr float kKdiv = 0x1.99999ap-4f;    // 0.10

__device__ __forceinline__ float flx3(float s1, float s2, float s3) {
    float r = kF3_1 * s1;
    r = r + kF3_2 * s2;
    return r + kF3_3 * s3;
}

// Correctly rounded binary32 reciprocal on the short path: the hardware's
// approximate reciprocal (PTX rcp.approx.ftz.f32, at most 1 ulp from 1/b)
// refined by one FMA Newton-Raphson step in Markstein's form (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990): e = 1 - b*y exactly, then
// y + y*e rounded once.  Used where |b| lies in [2^-125, 2^125]; elsewhere
// (subnormal-adjacent, huge, zero, inf, NaN) it defers to __frcp_rn.
// gm1b_selftest_reciprocal compares it with __frcp_rn on every one of the
// 2^32 binary32 words.
__device__ __forceinline__ float rcp_rn(float b) {
    const float ab = fabsf(b);
    if (!(ab >= 0x1p-125f && ab <= 0x1p125f)) return __frcp_rn(b);
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(b));
    const float e = fmaf(-b, y, 1.0f);
    return fmaf(y, e, y);
}

__device__ __forceinline__ float flx5(float s1, float s2, float s3, float s4, float s5) {
    float r = kF5_1 * s1;
    r = r + kF5_2 * s2;
    r = r + kF5_3 * s3;
    r = r + kF5_4 * s4;
    return r + kF5_5 * s5;
}

// Padded-lane extents with the index helpers of the four staggered shapes.
struct Dims {
    int ni, nj, nk;
    __host__ __device__ __forceinline__ size_t s(int k, int j, int i) const {
        return ((size_t)k * (nj + 2) + (size_t)j) * (size_t)(ni + 2) + (size_t)i;
    }
    __host__ __device__ __forceinline__ size_t u(int k, int j, int f) const {
        return ((size_t)k * (nj + 2) + (size_t)j) * (size_t)(ni + 1) + (size_t)f;
    }
    __host__ __device__ __forceinline__ size_t v(int k, int g, int i) const {
        return ((size_t)k * (nj + 1) + (size_t)g) * (size_t)(ni + 2) + (size_t)i;
    }
    __host__ __device__ __forceinline__ size_t w(int k, int j, int i) const {
        return ((size_t)k * nj + (size_t)j) * (size_t)ni + (size_t)i;
    }
    __host__ __device__ __forceinline__ size_t scalar_words() const { return (size_t)(nk + 2) * (nj + 2) * (ni + 2); }
    __host__ __device__ __forceinline__ size_t u_words() const { return (size_t)(nk + 2) * (nj + 2) * (ni + 1); }
    __host__ __device__ __forceinline__ size_t v_words() const { return (size_t)(nk + 2) * (nj + 1) * (ni + 2); }
    __host__ __device__ __forceinline__ size_t w_words() const { return (size_t)(nk + 2) * nj * ni; }
};

__device__ __forceinline__ int wrap(int x, int n) {  // periodic halo index -> live index
    return x == 0 ? n : (x == n + 1 ? 1 : x);
}

// Python modulo for x in [-n, 2n), the only range the stencils produce
// (n >= 5 and offsets of at most +-4 around an index in [-1, n+1]).
__device__ __forceinline__ int pmod(int x, int n) { return x < 0 ? x + n : (x >= n ? x - n : x); }

// Brackets one kernel launch with profiler events when the profiler is on.
class ProfScope {
  public:
    ProfScope(const char *name, cudaStream_t st);
    void stop();

  private:
    const char *name_;
    cudaStream_t st_;
    cudaEvent_t start_;
};

}  // namespace gm1b

// thread-local error message of the last failed entry point
void gm1b_set_error(const char *fmt, ...);
