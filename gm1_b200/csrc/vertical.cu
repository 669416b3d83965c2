// vertical.cu - CM1 vertical coordinates for stretch_z = 0 and 1: the
// Wilhelmson-Chen level generator, the mh/mf metrics and their inverses, the
// terrain-coordinate reciprocals rds/rdsf and the Fornberg boundary weights.
//
// Behaviour followed (reference file:line):
//   derive_stretch_z1       src/cm1core/cuda_stretch_z1.py:130-201 (param.F:7814-7914)
//   build_stretch_z1_grid   src/cm1core/cuda_stretch_z1.py:204-263 (param.F:7916-7953, 8162-8209)
//   launch_cuda_stretch_z1  src/cm1core/cuda_stretch_z1.py:418-470
//   _rds_rdsf               src/cm1core/cm1_vertical_grid.py:599-613 (init_terrain.F:292-298)
//   fornberg_extrapolation_weights  src/cm1core/cm1_vertical_grid.py:387-454 (param.F:8985-9035)
//   build_vertical_levels   src/cm1core/cm1_vertical_grid.py:780-927 (stretch_z 0 and 1)
//
// One generator, compiled for the host and the device, forms every word in
// binary32 one operation at a time (no contraction on either side), so the
// host profiles and the device profiles are the same words.  The device
// entry runs it in one thread: the column is a few hundred words, formed
// once per run.
#include <cmath>
#include <vector>

#include "gm1b_common.cuh"

namespace gm1b {
namespace {

struct Z1 {
    int nk, nk1, nk2, nk3;
    float dz, dz_bot, dz_top, nominal, c1, c2;
};

__host__ __device__ void z1_profiles(const Z1 &z, float *zf, float *zh, float *sigmaf, float *sigma, float *mh,
                                     float *mf, float *rmh, float *rmf, float *rds, float *rdsf) {
    const int nk = z.nk;
    for (int k = 0; k < nk + 3; ++k) zf[k] = sigmaf[k] = 0.0f;
    for (int k = 1; k <= z.nk1 + 1; ++k) zf[k] = sigmaf[k] = (float)(k - 1) * z.dz_bot;
    const float base = zf[z.nk1 + 1];
    for (int k = z.nk1 + 1; k <= z.nk1 + z.nk2 + 1; ++k) {
        const float delta = (float)(k - 1 - z.nk1);
        const float factor = z.c1 + (z.c2 * delta) * z.nominal;
        const float distance = (factor * delta) * z.nominal;
        zf[k] = sigmaf[k] = base + distance;
    }
    for (int k = z.nk1 + z.nk2 + 2; k <= nk + 1; ++k) zf[k] = sigmaf[k] = zf[k - 1] + z.dz_top;
    zf[0] = sigmaf[0] = -zf[2];
    zf[nk + 2] = sigmaf[nk + 2] = zf[nk + 1] + (zf[nk + 1] - zf[nk]);
    for (int k = 0; k <= nk + 1; ++k) {
        zh[k] = 0.5f * (zf[k + 1] + zf[k]);
        mh[k] = z.dz / (zf[k + 1] - zf[k]);
    }
    zh[0] = -zh[1];
    zh[nk + 1] = zh[nk] + 2.0f * (zf[nk + 1] - zh[nk]);
    for (int k = 1; k <= nk + 1; ++k) mf[k] = z.dz / (zh[k] - zh[k - 1]);
    mf[0] = mf[1];
    mf[nk + 2] = mf[nk + 1];
    for (int k = 0; k <= nk + 1; ++k) sigma[k] = 0.5f * (sigmaf[k] + sigmaf[k + 1]);
    for (int k = 0; k <= nk + 1; ++k) rmh[k] = 1.0f / mh[k];
    for (int k = 0; k <= nk + 2; ++k) rmf[k] = 1.0f / mf[k];
    if (rds != nullptr) {
        for (int k = 0; k < nk + 2; ++k) rds[k] = 0.0f;
        for (int k = 2; k <= nk; ++k) rds[k] = 1.0f / (sigma[k] - sigma[k - 1]);
    }
    if (rdsf != nullptr) {
        for (int k = 0; k < nk + 3; ++k) rdsf[k] = 0.0f;
        for (int k = 1; k <= nk; ++k) rdsf[k] = 1.0f / (sigmaf[k + 1] - sigmaf[k]);
    }
}

__global__ void stretch_z1_kernel(Z1 z, gm1b_vertical_profiles p) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    z1_profiles(z, p.zf, p.zh, p.sigmaf, p.sigma, p.mh, p.mf, p.rmh, p.rmf, p.rds, p.rdsf);
}

int nint_positive(float v) { return (int)std::floor((double)v + 0.5); }

// derive_stretch_z1's checks and coefficients; false with the message set
bool derive(const char *who, int nk, float dz, float ztop, float str_bot, float str_top, float dz_bot, float dz_top,
            Z1 &z) {
    if (nk < 4) {
        gm1b_set_error("%s: nk must be an integer >= 4", who);
        return false;
    }
    if (!std::isfinite(dz) || !std::isfinite(ztop) || !std::isfinite(str_bot) || !std::isfinite(str_top) ||
        !std::isfinite(dz_bot) || !std::isfinite(dz_top)) {
        gm1b_set_error("%s: stretch_z=1 parameters must be finite", who);
        return false;
    }
    if (dz <= 0.0f || ztop <= 0.0f || dz_bot <= 0.0f || dz_top <= 0.0f) {
        gm1b_set_error("%s: dz, ztop, dz_bot, and dz_top must be positive", who);
        return false;
    }
    if (str_bot < 0.0f || str_top <= str_bot || str_top > ztop) {
        gm1b_set_error("%s: require 0 <= str_bot < str_top <= ztop", who);
        return false;
    }
    const float nominal = 0.5f * (dz_bot + dz_top);
    const int nk1 = nint_positive(str_bot / dz_bot);
    const int nk3 = nint_positive((ztop - str_top) / dz_top);
    const int nk2 = nk - (nk1 + nk3);
    if (nk1 < 0 || nk2 < 2 || nk3 < 0) {
        gm1b_set_error("%s: stretch_z=1 requires nk1>=0, nk2>=2, and nk3>=0 (nk1=%d nk2=%d nk3=%d)", who, nk1, nk2,
                       nk3);
        return false;
    }
    const double bottom = std::fabs((double)((float)nk1 * dz_bot - str_bot));
    const double middle = std::fabs((double)((float)nk2 * nominal - (str_top - str_bot)));
    const double top = std::fabs((double)((float)nk3 * dz_top - (ztop - str_top)));
    if (bottom > 0.01 || middle >= 0.01 || top > 0.01) {
        gm1b_set_error("%s: stretch_z=1 segment depths must satisfy the official 0.01 m feasibility checks", who);
        return false;
    }
    const float c2 = (nominal - dz_bot) / ((nominal * nominal) * (float)(nk2 - 1));
    const float c1 = dz_bot / nominal - c2 * nominal;
    const float len = (dz_bot * (float)nk1 + nominal * (float)nk2) + dz_top * (float)nk3;
    if (std::fabs((double)(ztop - len)) > (double)(1.0e-6f * ztop)) {
        gm1b_set_error("%s: stretch_z=1 total length fails the official relative feasibility check", who);
        return false;
    }
    z = Z1{nk, nk1, nk2, nk3, dz, dz_bot, dz_top, nominal, c1, c2};
    return true;
}

// the generator on the host, then the reference's positive-spacing refusal
bool host_profiles(const char *who, const Z1 &z, float *zf, float *zh, float *sigmaf, float *sigma, float *mh,
                   float *mf, float *rmh, float *rmf, float *rds, float *rdsf) {
    z1_profiles(z, zf, zh, sigmaf, sigma, mh, mf, rmh, rmf, rds, rdsf);
    for (int k = 1; k <= z.nk; ++k)
        if (!(zf[k + 1] > zf[k])) {
            gm1b_set_error("%s: stretch_z=1 generated nonpositive physical spacing at level %d", who, k);
            return false;
        }
    return true;
}

// Fornberg (1988) table, bigm = 4, bign = 3 (param.F:9016-9035), value row
bool fornberg(const char *who, int nk, const float *sigma, const float *sigmaf, bool top, float out[3]) {
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
    if (!std::isfinite(den) || !(den > 0.0f)) {
        gm1b_set_error("%s: Fornberg extrapolation spacing is not positive and finite", who);
        return false;
    }
    const double x0 = (double)(num / den);
    double alpha[4];
    for (int q = 0; q < 4; ++q) alpha[q] = (double)(nodes[q] / den);
    double t[4][6][4] = {};
    t[0][1][0] = 1.0;
    double b1 = 1.0;
    for (int n = 1; n < 4; ++n) {
        double b2 = 1.0;
        for (int nu = 0; nu < n; ++nu) {
            const double b3 = alpha[n] - alpha[nu];
            if (!std::isfinite(b3) || b3 == 0.0) {
                gm1b_set_error("%s: Fornberg extrapolation nodes are duplicated", who);
                return false;
            }
            b2 = b2 * b3;
            t[n - 1][n + 1][nu] = 0.0;
            for (int m = 0; m <= n; ++m)
                t[n][m + 1][nu] = ((alpha[n] - x0) * t[n - 1][m + 1][nu] - m * t[n - 1][m][nu]) / b3;
        }
        for (int m = 0; m <= n; ++m)
            t[n][m + 1][n] = (b1 / b2) * (m * t[n - 1][m][n - 1] - (alpha[n - 1] - x0) * t[n - 1][m + 1][n - 1]);
        b1 = b2;
    }
    for (int nu = 0; nu < 3; ++nu) out[nu] = (float)t[2][1][nu];
    return true;
}

bool profiles_present(const gm1b_vertical_profiles *p) {
    return p != nullptr && p->zf && p->zh && p->sigmaf && p->sigma && p->mh && p->mf && p->rmh && p->rmf;
}

}  // namespace
}  // namespace gm1b

using namespace gm1b;

extern "C" int32_t gm1b_stretch_z1_derive(int32_t nk, float dz, float ztop, float str_bot, float str_top, float dz_bot,
                                          float dz_top, gm1b_stretch_z1_derived *out) {
    Z1 z;
    if (!derive("gm1b_stretch_z1_derive", nk, dz, ztop, str_bot, str_top, dz_bot, dz_top, z)) return GM1B_ERR_ARGUMENT;
    if (out != nullptr) *out = gm1b_stretch_z1_derived{z.nk1, z.nk2, z.nk3, z.nominal, z.c1, z.c2};
    return GM1B_OK;
}

extern "C" int32_t gm1b_vertical_levels(int32_t stretch_z, int32_t nk, float dz, float ztop, float str_bot,
                                        float str_top, float dz_bot, float dz_top, const gm1b_vertical_profiles *host,
                                        float cgs[3], float cgt[3]) {
    const char *who = "gm1b_vertical_levels";
    if (stretch_z != 0 && stretch_z != 1) {
        gm1b_set_error("%s: stretch_z=%d is not built (stretch_z 0 and 1 are)", who, stretch_z);
        return GM1B_ERR_ARGUMENT;
    }
    if (!profiles_present(host)) {
        gm1b_set_error("%s: every profile but rds/rdsf is required", who);
        return GM1B_ERR_ARGUMENT;
    }
    if (nk < 4) {
        gm1b_set_error("%s: nk must be an integer >= 4", who);
        return GM1B_ERR_ARGUMENT;
    }
    if (stretch_z == 0) {  // param.F:2608: the top of an unstretched column is dz*nk
        const float expected = dz * (float)nk;
        if (!(ztop == expected)) {
            gm1b_set_error("%s: stretch_z=0 fixes the model top at dz*nk = %g m (param.F:2608); %g m was declared", who,
                           (double)expected, (double)ztop);
            return GM1B_ERR_ARGUMENT;
        }
        str_bot = 0.0f;
        str_top = expected;
        dz_bot = dz_top = dz;
    }
    Z1 z;
    if (!derive(who, nk, dz, ztop, str_bot, str_top, dz_bot, dz_top, z)) return GM1B_ERR_ARGUMENT;
    if (!host_profiles(who, z, host->zf, host->zh, host->sigmaf, host->sigma, host->mh, host->mf, host->rmh, host->rmf,
                       host->rds, host->rdsf))
        return GM1B_ERR_ARGUMENT;
    if (cgs != nullptr && !fornberg(who, nk, host->sigma, host->sigmaf, false, cgs)) return GM1B_ERR_ARGUMENT;
    if (cgt != nullptr && !fornberg(who, nk, host->sigma, host->sigmaf, true, cgt)) return GM1B_ERR_ARGUMENT;
    return GM1B_OK;
}

extern "C" int32_t gm1b_stretch_z1(int32_t nk, float dz, float ztop, float str_bot, float str_top, float dz_bot,
                                   float dz_top, const gm1b_vertical_profiles *device, void *stream) {
    const char *who = "gm1b_stretch_z1";
    if (!profiles_present(device)) {
        gm1b_set_error("%s: every profile but rds/rdsf is required", who);
        return GM1B_ERR_ARGUMENT;
    }
    Z1 z;
    if (!derive(who, nk, dz, ztop, str_bot, str_top, dz_bot, dz_top, z)) return GM1B_ERR_ARGUMENT;
    // the positive-spacing refusal is decided on the host before any launch
    std::vector<float> h((size_t)10 * (size_t)(nk + 3));
    float *b = h.data();
    const size_t L = (size_t)nk + 3;
    if (!host_profiles(who, z, b, b + L, b + 2 * L, b + 3 * L, b + 4 * L, b + 5 * L, b + 6 * L, b + 7 * L, b + 8 * L,
                       b + 9 * L))
        return GM1B_ERR_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    {
        ProfScope ps("stretch_z1_kernel", st);
        stretch_z1_kernel<<<1, 1, 0, st>>>(z, *device);
        ps.stop();
    }
    const cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        cudaGetLastError();
        gm1b_set_error("%s: %s", who, cudaGetErrorString(e));
        return GM1B_ERR_CUDA;
    }
    return GM1B_OK;
}
