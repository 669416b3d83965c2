// scalar_rk.cu - sm_100a kernels of the scalar/moisture RK stage pieces on
// the padded (ng = 3) lane: theta transport packing, the A-anchored RK
// composition, and one positive-definite (pdef) direction pass.
//
// Behaviour followed (reference file:line):
//   cpu_theta_transport_scalar_inplace          src/cm1core/cuda_scalar_moist_rk.py:255-280
//   cpu_compose_scalar_moist_rk_stage_inplace   src/cm1core/cuda_scalar_moist_rk.py:283-349
//   cpu_pdef_direction_inplace                  src/cm1core/cuda_scalar_moist_rk.py:352-518
//
// Design (B200): all three are elementwise passes with x fastest.  The pdef
// line repair, which the reference runs as one sequential sweep per line, is
// cell-parallel here: the mass correction of cell m only receives
// contributions from the negative centres m-1, m and m+1 (in that order),
// each a function of the candidates m-2..m+2, so each thread forms its own
// correction from five neighbouring candidates in the sweep's order.
#include "gm1b_common.cuh"

namespace gm1b {
namespace {

constexpr int NG = 3;
constexpr int kRX = 32, kRY = 4;

__global__ void __launch_bounds__(kRX *kRY) theta_pack_kernel(const float *th0, const float *th3d, float *padded,
                                                              int ni, int nj) {
    const int i = blockIdx.x * kRX + threadIdx.x;
    const int j = blockIdx.y * kRY + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= ni || j >= nj) return;
    const size_t sx = (size_t)ni + 2 * NG, sy = (size_t)nj + 2 * NG;
    const float base = th0[k] - 300.0f;
    padded[((size_t)(k + 1) * sy + (j + NG)) * sx + (i + NG)] = base + th3d[((size_t)k * nj + j) * ni + i];
}

__global__ void rk_compose_kernel(gm1b_scalar_rk_compose_arrays a, size_t cells, int nq, float dttmp) {
    const size_t n = cells * (size_t)(1 + nq);
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        float out;
        if (p < cells) {
            const float seed = a.theta_held[p] - a.theta_divterm[p];
            const float total = seed + a.theta_adv[p];
            out = a.theta_a[p] + dttmp * total;
            if (fabsf(out) < kSmeps) out = 0.0f;
            a.theta_cur[p] = out;
        } else {
            const size_t q = p - cells;
            const float total = a.q_held[q] + a.q_adv[q];
            out = a.q_a[q] + dttmp * total;
            if (fabsf(out) < kSmeps) out = 0.0f;
            a.q_cur[q] = out;
        }
    }
}

struct PdefGeom {
    int ni, nj, nk, axis;
    __device__ __forceinline__ size_t c3(int k, int j, int i) const {
        return ((size_t)k * nj + (size_t)j) * (size_t)ni + (size_t)i;
    }
    // mass-flux difference along the axis at cell (k, j, i)
    __device__ __forceinline__ float diff(const float *mf, int k, int j, int i) const {
        const size_t sx = (size_t)ni + 2 * NG, sy = (size_t)nj + 2 * NG;
        if (axis == 0) {
            const size_t ux = (size_t)ni + 1 + 2 * NG;
            const size_t r = ((size_t)(k + 1) * sy + (j + NG)) * ux + (i + NG);
            return mf[r + 1] - mf[r];
        }
        if (axis == 1) {
            const size_t vy = (size_t)nj + 1 + 2 * NG;
            const size_t r = ((size_t)(k + 1) * vy + (j + NG)) * sx + (i + NG);
            return mf[r + sx] - mf[r];
        }
        const size_t r = ((size_t)(k + 1) * sy + (j + NG)) * sx + (i + NG);
        return mf[r + sx * sy] - mf[r];
    }
    __device__ __forceinline__ float padded(const float *sp, int k, int j, int i) const {
        const size_t sx = (size_t)ni + 2 * NG, sy = (size_t)nj + 2 * NG;
        return sp[((size_t)(k + 1) * sy + (j + NG)) * sx + (i + NG)];
    }
};

__global__ void __launch_bounds__(kRX *kRY) pdef_candidate_kernel(gm1b_pdef_arrays a, PdefGeom g, float dt, float rs) {
    const int i = blockIdx.x * kRX + threadIdx.x;
    const int j = blockIdx.y * kRY + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.ni || j >= g.nj) return;
    const size_t c = g.c3(k, j, i);
    const float divergence = (g.padded(a.scalar_padded, k, j, i) * g.diff(a.mass_flux, k, j, i)) * rs;
    const float total = a.directional[c] + divergence;
    const float increment = (dt * total) * a.gz[(size_t)j * g.ni + i];
    a.candidate[c] = a.rho0[c] * a.scalar_a[c] + increment;
}

__global__ void __launch_bounds__(kRX *kRY) pdef_repair_kernel(gm1b_pdef_arrays a, PdefGeom g, float rdt, float rs) {
    const int i = blockIdx.x * kRX + threadIdx.x;
    const int j = blockIdx.y * kRY + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.ni || j >= g.nj) return;
    const int length = g.axis == 0 ? g.ni : (g.axis == 1 ? g.nj : g.nk);
    const int m = g.axis == 0 ? i : (g.axis == 1 ? j : k);
    const int start = g.axis == 2 ? 0 : 1;
    const int stop = g.axis == 2 ? length : length - 1;
    // candidate at line index m + off (0 outside the line: never read there)
    auto v = [&](int off) -> float {
        const int q = m + off;
        if (q < 0 || q >= length) return 0.0f;
        const size_t c = g.axis == 0 ? g.c3(k, j, q) : (g.axis == 1 ? g.c3(k, q, i) : g.c3(q, j, i));
        return a.candidate[c];
    };
    const float vm2 = v(-2), vm1 = v(-1), v0 = v(0), vp1 = v(1), vp2 = v(2);
    float mass = 0.0f;
    bool flag = false;
    if (m - 1 >= start && m - 1 < stop && vm1 < 0.0f) {  // centre m-1, this cell its right neighbour
        const float left = (m - 1 == 0) ? 0.0f : fmaxf(0.0f, vm2);
        const float right = fmaxf(0.0f, v0);
        const float donor = left + right;
        if (donor > kSmeps) {
            const float ratio = fmaxf(vm1, 0.0f - donor) / donor;
            mass = mass + right * ratio;
            if (v0 > kSmeps) flag = true;
        }
    }
    if (m >= start && m < stop && v0 < 0.0f) {  // this cell as the centre
        const float left = (m == 0) ? 0.0f : fmaxf(0.0f, vm1);
        const float right = (m + 1 == length) ? 0.0f : fmaxf(0.0f, vp1);
        const float donor = left + right;
        if (donor > kSmeps) {
            const float ratio = fmaxf(v0, 0.0f - donor) / donor;
            mass = mass - donor * ratio;
            flag = true;
        }
    }
    if (m + 1 >= start && m + 1 < stop && vp1 < 0.0f) {  // centre m+1, this cell its left neighbour
        const float left = fmaxf(0.0f, v0);
        const float right = (m + 2 == length) ? 0.0f : fmaxf(0.0f, vp2);
        const float donor = left + right;
        if (donor > kSmeps) {
            const float ratio = fmaxf(vp1, 0.0f - donor) / donor;
            mass = mass + left * ratio;
            if (v0 > kSmeps) flag = true;
        }
    }
    if (!flag) return;
    const size_t c = g.c3(k, j, i);
    const float divergence = (g.padded(a.scalar_padded, k, j, i) * g.diff(a.mass_flux, k, j, i)) * rs;
    float adjusted = (v0 + mass) - a.rho0[c] * a.scalar_a[c];
    adjusted = (adjusted * rdt) * a.rgz[(size_t)j * g.ni + i];
    a.directional[c] = adjusted - divergence;
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

extern "C" int32_t gm1b_theta_transport_pack(int32_t ni, int32_t nj, int32_t nk, const float *th0, const float *th3d,
                                            float *padded, void *stream) {
    if (ni < 1 || nj < 1 || nk < 1 || th0 == nullptr || th3d == nullptr || padded == nullptr) {
        gm1b_set_error("gm1b_theta_transport_pack: need arrays and ni, nj, nk >= 1");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("theta_pack_kernel", st);
    theta_pack_kernel<<<dim3((ni + kRX - 1) / kRX, (nj + kRY - 1) / kRY, nk), dim3(kRX, kRY), 0, st>>>(th0, th3d,
                                                                                                     padded, ni, nj);
    ps.stop();
    return launch_ok("theta_pack_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_scalar_moist_rk_compose(size_t cells, int32_t nq, const gm1b_scalar_rk_compose_arrays *arrays,
                                               int32_t nrk, float dt, void *stream) {
    if (arrays == nullptr || cells == 0 || nq < 0 || nrk < 1 || nrk > 3 || !(dt > 0.0f)) {
        gm1b_set_error("gm1b_scalar_moist_rk_compose: need arrays, cells > 0, nq >= 0, nrk 1..3, dt > 0");
        return GM1B_ERR_ARGUMENT;
    }
    const gm1b_scalar_rk_compose_arrays &a = *arrays;
    if (!a.theta_a || !a.theta_held || !a.theta_divterm || !a.theta_adv || !a.theta_cur ||
        (nq > 0 && (!a.q_a || !a.q_held || !a.q_adv || !a.q_cur))) {
        gm1b_set_error("gm1b_scalar_moist_rk_compose: a required array is NULL");
        return GM1B_ERR_ARGUMENT;
    }
    const float dttmp = dt / (float)(4 - nrk);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = cells * (size_t)(1 + nq);
    const int blocks = (int)((n + 255) / 256 < (size_t)(148 * 16) ? (n + 255) / 256 : (size_t)(148 * 16));
    ProfScope ps("rk_compose_kernel", st);
    rk_compose_kernel<<<blocks, 256, 0, st>>>(a, cells, nq, dttmp);
    ps.stop();
    return launch_ok("rk_compose_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_pdef_direction(int32_t ni, int32_t nj, int32_t nk, const gm1b_pdef_arrays *arrays,
                                      int32_t axis, float dt, float spacing, void *stream) {
    if (arrays == nullptr || ni < 1 || nj < 1 || nk < 1 || axis < 0 || axis > 2) {
        gm1b_set_error("gm1b_pdef_direction: need arrays, ni, nj, nk >= 1 and axis 0 (x), 1 (y) or 2 (z)");
        return GM1B_ERR_ARGUMENT;
    }
    if (!(dt > 0.0f) || !isfinite(dt) || !(spacing > 0.0f) || !isfinite(spacing)) {
        gm1b_set_error("gm1b_pdef_direction: dt and spacing must be finite and > 0");
        return GM1B_ERR_ARGUMENT;
    }
    const float *const *p = reinterpret_cast<const float *const *>(arrays);
    for (size_t q = 0; q < sizeof(gm1b_pdef_arrays) / sizeof(float *); ++q)
        if (p[q] == nullptr) {
            gm1b_set_error("gm1b_pdef_direction: array #%zu is NULL", q);
            return GM1B_ERR_ARGUMENT;
        }
    const PdefGeom g{ni, nj, nk, axis};
    const float rdt = 1.0f / dt, rs = 1.0f / spacing;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const dim3 grid((ni + kRX - 1) / kRX, (nj + kRY - 1) / kRY, nk), blk(kRX, kRY);
    {
        ProfScope ps("pdef_candidate_kernel", st);
        pdef_candidate_kernel<<<grid, blk, 0, st>>>(*arrays, g, dt, rs);
        ps.stop();
    }
    if (!launch_ok("pdef_candidate_kernel")) return GM1B_ERR_CUDA;
    {
        ProfScope ps("pdef_repair_kernel", st);
        pdef_repair_kernel<<<grid, blk, 0, st>>>(*arrays, g, rdt, rs);
        ps.stop();
    }
    return launch_ok("pdef_repair_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}
