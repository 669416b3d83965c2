// limits.cu - CM1's time-step limits and its advective Courant number.
//
// Behaviour followed (reference file:line):
//   cm1_acoustic_small_step_limit_s    src/cm1core/gm1_runtime.py:249-268 (misclibs.F:867)
//   cm1_diagnostic_acoustic_substeps   src/cm1core/gm1_runtime.py:284-302 (misclibs.F:883-885)
//   cm1_advective_courant              src/cm1core/gm1_runtime.py:458-489 (misclibs.F:2747-2765)
//   _reduce_courant / advective_courant_number
//                                      src/cm1core/storm_diagnostics.py:195-297 (calccflquick)
//
// Design (B200): the three scalars are binary64 host arithmetic in the
// reference's order.  The domain Courant number, which the reference forms as
// about fifteen elementwise launches per model level plus a device-to-host
// read per level, is one pass here: every thread forms the binary32 cell
// value in the reference's operation order, the block reduces it, and one
// atomicMax per block and level lands in a per-level word (cfl(k) of CM1);
// a one-warp fold then takes the maximum over levels with the reference's
// Python max() rule (a NaN level never replaces the running maximum).  The
// pass reads u, v and w once: 12 bytes per cell.
#include <cmath>

#include "gm1b_common.cuh"

namespace gm1b {
namespace {

constexpr double kAcousticSpeed = 360.0;   // CM1_PSOLVER3_ACOUSTIC_SPEED_M_S
constexpr double kAcousticCourant = 0.60;  // CM1_PSOLVER3_ACOUSTIC_COURANT
constexpr int kMinSubsteps = 4;            // CM1_MIN_ACOUSTIC_SUBSTEPS
constexpr int kCflThreads = 256;

bool positive_finite(double x) { return std::isfinite(x) && x > 0.0; }

double small_step_limit(double dx, double dy) { return kAcousticCourant * (dx < dy ? dx : dy) / kAcousticSpeed; }

// Fortran nint: half away from zero
long long fortran_nint(double x) {
    return x >= 0.0 ? (long long)std::floor(x + 0.5) : -(long long)std::floor(-x + 0.5);
}

// Order key of a non-negative-or-NaN binary32: NaN sorts above everything
__device__ __forceinline__ unsigned int cfl_key(float x) { return isnan(x) ? 0xffffffffu : __float_as_uint(x); }

__global__ void __launch_bounds__(kCflThreads) courant_level_kernel(const float *__restrict__ u,
                                                                    const float *__restrict__ v,
                                                                    const float *__restrict__ w,
                                                                    const float *__restrict__ uh,
                                                                    const float *__restrict__ vh,
                                                                    const float *__restrict__ mh, int ni, int nj,
                                                                    float dtdx, float dtdy, float dtdz,
                                                                    unsigned int *__restrict__ level_key) {
    const int k = blockIdx.y;
    const size_t plane = (size_t)ni * nj;
    unsigned int best = 0u;
    const float mk = mh[k];
    for (size_t p = (size_t)blockIdx.x * kCflThreads + threadIdx.x; p < plane; p += (size_t)gridDim.x * kCflThreads) {
        const int j = (int)(p / (size_t)ni);
        const int i = (int)(p - (size_t)j * ni);
        // u (nk, nj, ni+1), v (nk, nj+1, ni), w (nk+1, nj, ni)
        const size_t fu = ((size_t)k * nj + j) * (size_t)(ni + 1) + i;
        const size_t fv = ((size_t)k * (nj + 1) + j) * (size_t)ni + i;
        const size_t fw = ((size_t)k * nj + j) * (size_t)ni + i;
        float term = u[fu] + u[fu + 1];
        term = term * dtdx;
        term = term * uh[i];
        float acc = term * term;
        term = v[fv] + v[fv + ni];
        term = term * dtdy;
        term = term * vh[j];
        term = term * term;
        acc = acc + term;
        term = w[fw] + w[fw + plane];
        term = term * dtdz;
        term = term * mk;
        term = term * term;
        acc = acc + term;
        const unsigned int key = cfl_key(sqrtf(acc));
        best = key > best ? key : best;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned int o = __shfl_xor_sync(0xffffffffu, best, off);
        best = o > best ? o : best;
    }
    __shared__ unsigned int s_best[kCflThreads / 32];
    if ((threadIdx.x & 31) == 0) s_best[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x < 32) {
        best = threadIdx.x < kCflThreads / 32 ? s_best[threadIdx.x] : 0u;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const unsigned int o = __shfl_xor_sync(0xffffffffu, best, off);
            best = o > best ? o : best;
        }
        if (threadIdx.x == 0 && best != 0u) atomicMax(&level_key[k], best);
    }
}

// largest = max(largest, level) in level order with Python's rule: the level
// replaces the running value only if it compares greater (NaN never does)
__global__ void courant_fold_kernel(const unsigned int *__restrict__ level_key, int nk, float *__restrict__ out) {
    if (threadIdx.x != 0) return;
    float largest = 0.0f;
    for (int k = 0; k < nk; ++k) {
        const unsigned int key = level_key[k];
        const float m = key == 0xffffffffu ? __uint_as_float(0x7fc00000u) : __uint_as_float(key);
        if (m > largest) largest = m;
    }
    *out = largest;
}

bool launch_ok(const char *what) {
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        cudaGetLastError();
        gm1b_set_error("%s: %s", what, cudaGetErrorString(e));
        return false;
    }
    return true;
}

}  // namespace
}  // namespace gm1b

using namespace gm1b;

extern "C" double gm1b_acoustic_small_step_limit(double dx, double dy) {
    if (!positive_finite(dx) || !positive_finite(dy)) {
        gm1b_set_error("gm1b_acoustic_small_step_limit: dx_m and dy_m must be finite and positive");
        return __builtin_nan("");
    }
    return small_step_limit(dx, dy);
}

extern "C" int32_t gm1b_diagnostic_acoustic_substeps(double dt, double dx, double dy, int32_t *nsound) {
    if (nsound == nullptr || !positive_finite(dt) || !positive_finite(dx) || !positive_finite(dy)) {
        gm1b_set_error("gm1b_diagnostic_acoustic_substeps: dt_s, dx_m and dy_m must be finite and positive");
        return GM1B_ERR_ARGUMENT;
    }
    const double limit = small_step_limit(dx, dy);
    const double ratio = dt / limit;
    if (!(ratio < 2.0e9)) {
        gm1b_set_error("gm1b_diagnostic_acoustic_substeps: dt_s/dtsm = %g does not fit an acoustic substep count",
                       ratio);
        return GM1B_ERR_ARGUMENT;
    }
    long long n = fortran_nint(ratio);
    if (n < kMinSubsteps) n = kMinSubsteps;
    if (n % 2) n += 1;
    if (dt / (double)n > limit) n += 2;
    *nsound = (int32_t)n;
    return GM1B_OK;
}

extern "C" int32_t gm1b_advective_courant(double dt, double dx, double dy, double dz, double u, double v, double w,
                                          double *out) {
    if (out == nullptr || !positive_finite(dt) || !positive_finite(dx) || !positive_finite(dy) ||
        !positive_finite(dz)) {
        gm1b_set_error("gm1b_advective_courant: dt_s, dx_m, dy_m and dz_m must be finite and positive");
        return GM1B_ERR_ARGUMENT;
    }
    if (!std::isfinite(u) || !std::isfinite(v) || !std::isfinite(w)) {
        gm1b_set_error("gm1b_advective_courant: u_m_s, v_m_s and w_m_s must be finite");
        return GM1B_ERR_ARGUMENT;
    }
    const double cu = u * dt / dx, cv = v * dt / dy, cw = w * dt / dz;
    const double horizontal = cu * cu + cv * cv;
    *out = std::sqrt(horizontal + cw * cw);
    return GM1B_OK;
}

extern "C" int32_t gm1b_courant_max(int32_t ni, int32_t nj, int32_t nk, const float *u, const float *v, const float *w,
                                    const float *uh, const float *vh, const float *mh, float dtdx, float dtdy,
                                    float dtdz, uint32_t *level_keys, float *out, void *stream) {
    if (ni < 1 || nj < 1 || nk < 1 || !u || !v || !w || !uh || !vh || !mh || !level_keys || !out) {
        gm1b_set_error("gm1b_courant_max: need ni, nj, nk >= 1 and every array");
        return GM1B_ERR_ARGUMENT;
    }
    if (nk > 65535) {
        gm1b_set_error("gm1b_courant_max: nk=%d exceeds one grid dimension", nk);
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(level_keys, 0, (size_t)nk * sizeof(uint32_t), st);
    if (e != cudaSuccess) {
        gm1b_set_error("cudaMemsetAsync: %s", cudaGetErrorString(e));
        return GM1B_ERR_CUDA;
    }
    const size_t plane = (size_t)ni * nj;
    // about 8 cells per thread, and at least 2 x 148 blocks over the volume
    size_t bx = (plane + 8 * kCflThreads - 1) / (8 * kCflThreads);
    const size_t want = (2 * 148 + nk - 1) / nk;
    if (bx < want) bx = want;
    const size_t cap = (plane + kCflThreads - 1) / kCflThreads;
    if (bx > cap) bx = cap;
    {
        ProfScope ps("courant_level_kernel", st);
        courant_level_kernel<<<dim3((unsigned)bx, nk), kCflThreads, 0, st>>>(u, v, w, uh, vh, mh, ni, nj, dtdx, dtdy,
                                                                            dtdz, level_keys);
        ps.stop();
    }
    if (!launch_ok("courant_level_kernel")) return GM1B_ERR_CUDA;
    courant_fold_kernel<<<1, 32, 0, st>>>(level_keys, nk, out);
    return launch_ok("courant_fold_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}
