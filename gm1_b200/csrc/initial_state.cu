// initial_state.cu - the analytic initial state of the moist storm
// configurations: the Weisman-Klemp base column (CM1 isnd=5), the iwnd=2
// quarter-circle base wind, and the iinit=1 warm-bubble theta perturbation.
//
// Behaviour followed (reference file:line):
//   weisman_klemp_column_with_iterations   rust/cm1-state/src/storm_initialization.rs:194-350
//   WeismanKlempSurface::official          rust/cm1-state/src/storm_initialization.rs:67-80
//   rslf                                   rust/cm1-state/src/idealized_initialization.rs:984-989
//   analytic_shear_u / analytic_shear_v    rust/cm1-state/src/storm_initialization.rs:354-389
//   build_theta_perturbation, iinit = 1    rust/cm1-state/src/initial_perturbation.rs:449-466
//
// Design (B200): the base column is nk words computed once, by a 20-sweep
// serial recurrence in k; it runs on the host in binary32 one operation at a
// time with the C library's powf/expf (the functions CM1's gfortran build
// calls), so th0, qv0 and pi0 come out word-identical to CM1 r21.1's own
// output.  The bubble is a 3-D field of the whole domain (39 M words at
// 640x768x80) and is written straight into the device-resident scalar lane
// by one elementwise kernel, so the state never crosses PCIe.
#include <cmath>
#include <vector>

#include "gm1b_common.cuh"

namespace gm1b {
namespace {

// CM1 constants.F words (binary32); kCp is the shared 1005.7
constexpr float kG = 9.81f, kRd = 287.04f, kRv = 461.5f, kP00 = 100000.0f;
// base.F:369-374
constexpr float kZTrop = 12000.0f, kThTrop = 343.0f, kTTrop = 213.0f, kThSfc = 300.0f, kPrsSfc = 100000.0f;
constexpr float kQvPbl = 0.014f;
// constants.F pi as a default REAL, and base.F:2323-2326 / :2344
constexpr float kPi = 3.14159265358979f;
constexpr float kUdep1 = 2000.0f, kUdep2 = 6000.0f, kUmax1 = 7.0f, kUmax2 = 31.0f;

// Host arithmetic must not be contracted into fused multiply-adds: each
// statement below is one rounded binary32 operation, as in CM1.
float host_rslf(float p, float t) {
    volatile float eps = kRd / kRv;
    float x = 17.67f * (t - 273.15f);
    x = x / (t - 29.65f);
    float es = 611.2f * std::exp(x);
    const float half_p = p * 0.5f;
    if (half_p < es) es = half_p;
    const float num = eps * es;
    return num / (p - es);
}

__global__ void theta_bubble_kernel(const float *__restrict__ xh, const float *__restrict__ yh,
                                    const float *__restrict__ zh, float *__restrict__ tha, int ni, int nj,
                                    int nk, int ng, int gz, float xc, float yc, float zc, float hrad, float zrad,
                                    float amp) {
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= ni || j >= nj) return;
    const float rx = (xh[i] - xc) / hrad;
    const float ry = (yh[j] - yc) / hrad;
    const float rz = (zh[k] - zc) / zrad;
    const float r2 = rx * rx + ry * ry + rz * rz;
    const float beta = sqrtf(r2);
    float value = 0.0f;
    if (beta < 1.0f) {
        const float c = cosf(0.5f * kPi * beta);
        value = amp * (c * c);
    }
    const size_t sx = (size_t)ni + 2 * ng, sy = (size_t)nj + 2 * ng;
    tha[((size_t)(k + gz) * sy + (size_t)(j + ng)) * sx + (size_t)(i + ng)] = value;
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

extern "C" int32_t gm1b_wk_base_column(int32_t nk, const float *zh, int32_t imoist, int32_t iterations, float *th0,
                                       float *qv0, float *thv0, float *pi0, float *prs0, float *t0, float *rh0) {
    if (nk < 1 || zh == nullptr || th0 == nullptr || qv0 == nullptr || pi0 == nullptr || prs0 == nullptr) {
        gm1b_set_error("gm1b_wk_base_column: analytic sounding column requires nk>=1 and the th0, qv0, pi0, prs0 "
                       "outputs");
        return GM1B_ERR_ARGUMENT;
    }
    if (imoist != 0 && imoist != 1) {
        gm1b_set_error("gm1b_wk_base_column: base.F:389-397 branches on imoist=0 or 1 only; got imoist=%d", imoist);
        return GM1B_ERR_ARGUMENT;
    }
    if (iterations < 1) {
        gm1b_set_error("gm1b_wk_base_column: the analytic hydrostatic fixed point requires at least one iteration");
        return GM1B_ERR_ARGUMENT;
    }
    for (int k = 0; k < nk; ++k) {
        const float below = k == 0 ? 0.0f : zh[k - 1];
        if (!std::isfinite(zh[k]) || !(zh[k] > below)) {
            gm1b_set_error("gm1b_wk_base_column: analytic sounding mass heights must be strictly increasing above "
                           "z=0; level %d is %g m after %g m",
                           k, (double)zh[k], (double)below);
            return GM1B_ERR_ARGUMENT;
        }
    }
    volatile float reps_v = kRv / kRd, cpdrd_v = kCp / kRd, rovcp_v = kRd / kCp;
    const float reps = reps_v, cpdrd = cpdrd_v;
    // surface words (base.F:378-380)
    const float pi_sfc = std::pow(kPrsSfc / kP00, (float)rovcp_v);
    const float qv_sfc = host_rslf(kPrsSfc, kThSfc * pi_sfc);
    float thv_sfc = kThSfc * (1.0f + qv_sfc * reps);
    thv_sfc = thv_sfc / (1.0f + qv_sfc);

    std::vector<float> rh(nk), thv(nk);
    for (int k = 0; k < nk; ++k) {
        if (zh[k] < kZTrop) {
            const float shape = std::pow(zh[k] / kZTrop, 1.25f);
            const float rise = (kThTrop - kThSfc) * shape;
            th0[k] = kThSfc + rise;
            const float dry = 0.75f * shape;
            rh[k] = imoist == 1 ? 1.0f - dry : 0.0f;
        } else {
            volatile float rate_v = kG / (kTTrop * kCp);
            const float arg = rate_v * (zh[k] - kZTrop);
            th0[k] = kThTrop * std::exp(arg);
            rh[k] = imoist == 1 ? 0.25f : 0.0f;
        }
        qv0[k] = 0.0f;
    }
    for (int it = 0; it < iterations; ++it) {
        for (int k = 0; k < nk; ++k) {
            const float num = th0[k] * (1.0f + reps * qv0[k]);
            thv[k] = num / (1.0f + qv0[k]);
        }
        for (int k = 0; k < nk; ++k) {
            const float pi_below = k == 0 ? pi_sfc : pi0[k - 1];
            const float thv_below = k == 0 ? thv_sfc : thv[k - 1];
            const float dz = k == 0 ? zh[0] : zh[k] - zh[k - 1];
            const float half_cp = kCp * 0.5f;
            const float denom = half_cp * (thv[k] + thv_below);
            const float gdz = kG * dz;
            pi0[k] = pi_below - gdz / denom;
        }
        for (int k = 0; k < nk; ++k) prs0[k] = kP00 * std::pow(pi0[k], cpdrd);
        for (int k = 0; k < nk; ++k) {
            const float tk = th0[k] * pi0[k];
            const float q = rh[k] * host_rslf(prs0[k], tk);
            qv0[k] = q > kQvPbl ? kQvPbl : q;
        }
    }
    for (int k = 0; k < nk; ++k) {
        const float tk = th0[k] * pi0[k];
        const float sat = host_rslf(prs0[k], tk);
        if (thv0) thv0[k] = thv[k];
        if (rh0) rh0[k] = qv0[k] / sat;
        if (t0) t0[k] = tk;
        const bool finite = std::isfinite(th0[k]) && std::isfinite(qv0[k]) && std::isfinite(pi0[k]) &&
                            std::isfinite(prs0[k]) && std::isfinite(thv[k]);
        if (!finite || !(th0[k] > 0.0f) || !(pi0[k] > 0.0f) || !(prs0[k] > 0.0f) || qv0[k] < 0.0f) {
            gm1b_set_error("gm1b_wk_base_column: analytic sounding column is non-physical at level %d: the requested "
                           "mass heights leave the interval where base.F:363-450 produces a positive hydrostatic "
                           "base state",
                           k);
            return GM1B_ERR_ARGUMENT;
        }
    }
    return GM1B_OK;
}

extern "C" int32_t gm1b_analytic_shear(int32_t n, const float *zu, const float *zv, float *u, float *v) {
    if (n < 0 || (u != nullptr && zu == nullptr) || (v != nullptr && zv == nullptr)) {
        gm1b_set_error("gm1b_analytic_shear: need n >= 0 and a height array for every requested profile");
        return GM1B_ERR_ARGUMENT;
    }
    volatile float deg_v = kPi / 180.0f;
    const float deg = deg_v;
    for (int k = 0; k < n; ++k) {
        if (u) {
            const float z = zu[k];
            if (z <= kUdep1) {
                const float angle = 90.0f * (z / kUdep1) * deg;
                const float c = kUmax1 * std::cos(angle);
                u[k] = kUmax1 - c;
            } else if (z <= kUdep2) {
                const float ramp = (z - kUdep1) * (kUmax2 - kUmax1);
                u[k] = kUmax1 + ramp / (kUdep2 - kUdep1);
            } else {
                u[k] = kUmax2;
            }
        }
        if (v) {
            const float z = zv[k];
            if (z <= kUdep1) {
                const float angle = 90.0f * (z / kUdep1) * deg;
                v[k] = kUmax1 * std::sin(angle);
            } else {
                v[k] = kUmax1;
            }
        }
    }
    return GM1B_OK;
}

extern "C" int32_t gm1b_theta_bubble(int32_t ni, int32_t nj, int32_t nk, int32_t ng, const float *xh,
                                     const float *yh, const float *zh, float center_x, float center_y,
                                     float center_z, float horizontal_radius, float vertical_radius, float amplitude,
                                     float *tha, void *stream) {
    if (ni < 1 || nj < 1 || nk < 1 || ng < 0 || ng > 3 || !xh || !yh || !zh || !tha) {
        gm1b_set_error("gm1b_theta_bubble: need ni, nj, nk >= 1, ng in 0..3 and device xh, yh, zh, tha");
        return GM1B_ERR_ARGUMENT;
    }
    if (!(horizontal_radius > 0.0f) || !(vertical_radius > 0.0f) || !std::isfinite(amplitude)) {
        gm1b_set_error("gm1b_theta_bubble: bubble radii must be positive and the amplitude finite");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int gz = ng > 0 ? 1 : 0;
    ProfScope ps("theta_bubble_kernel", st);
    theta_bubble_kernel<<<dim3((ni + 31) / 32, (nj + 7) / 8, nk), dim3(32, 8), 0, st>>>(
        xh, yh, zh, tha, ni, nj, nk, ng, gz, center_x, center_y, center_z, horizontal_radius, vertical_radius,
        amplitude);
    ps.stop();
    return launch_ok("theta_bubble_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}
