// SGS stress and scalar diffusion of the terrain texts (the uniform column's
// operator family): calcdef's strain carriers, gettau, turbu/turbv/turbw with
// their implicit vertical solves, and turbs of theta and the moisture rows.
//
// Behaviour followed (reference file:line):
//   the strain carriers rho*Sij   cpu_terrain_deformation_inplace
//       src/cm1core/cuda_terrain_deformation.py:234-736 (turb.F:4711-5423)
//   gettau and the momentum stress (four open sides, doimpl = 1, free-slip
//   bottom and top)               cpu_sgs_stress_tendency_inplace
//       src/cm1core/cuda_sgs_stress_tendency.py:292-449 (turb.F:4065-4506,
//       :4536-4545; turbtend.F:1052-2885)
//   turbs, no surface flux        cpu_gm1_scalar_turbulence_inplace and its
//       kernels src/cm1core/cuda_gm1_scalar_turbulence.py:230-430, :453-510
//       (turbtend.F:18-434, :442-692; solve1.F:1169-1227)
//
// Binary32 one operation at a time in the twins' statement order
// (--fmad=false); open sides are index clamps (the twins' edge padding).
//
// Design as csrc/stress.cu: elementwise grid-stride passes for the strain
// and gettau, one thread per staggered column (32 x 4 columns per CTA, the
// Thomas coefficients in shared memory [level][thread]) for the implicit
// solves, the horizontal terms and the cross term formed in the back
// substitution; turbs forms its x/y fluxes of every scalar in one pass into
// the workspace (their w-level interpolation is read back there), then solves
// each column.
#include "gm1b_common.cuh"

namespace gm1b {
namespace {

constexpr int kCX = 32, kCY = 4, kCT = kCX * kCY;
constexpr int kEW = 256;

#define TRY(x)                        \
    do {                              \
        const int r_ = (x);           \
        if (r_ != GM1B_OK) return r_; \
    } while (0)

bool launch_ok(const char *what) {
    const cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        cudaGetLastError();
        gm1b_set_error("%s: %s", what, cudaGetErrorString(e));
        return false;
    }
    return true;
}

struct TArgs {
    const float *u, *v, *w, *rho, *rf, *mh, *mf, *kmh, *kmv, *gz, *rgz, *gzu, *rgzu, *gzv, *rgzv, *gx, *gy, *gxu, *gyv;
    float *s11, *s22, *s33, *s12, *s13, *s23, *t11, *t22, *t33, *t12, *t13, *t23, *uten, *vten, *wten;
    int ni, nj, nk;
    float dx, dy, dz, dt;
};

__device__ __forceinline__ int cl(int x, int n) { return x < 0 ? 0 : (x >= n ? n - 1 : x); }
__device__ __forceinline__ int clr(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }
__device__ __forceinline__ unsigned o3(int k, int j, int i, int ny, int nx) {
    return ((unsigned)k * (unsigned)ny + (unsigned)j) * (unsigned)nx + (unsigned)i;
}
__device__ __forceinline__ float c3(const TArgs &a, const float *p, int k, int j, int i) {
    return p[o3(k, cl(j, a.nj), cl(i, a.ni), a.nj, a.ni)];
}
__device__ __forceinline__ float c2(const TArgs &a, const float *p, int j, int i) {
    return p[(unsigned)cl(j, a.nj) * (unsigned)a.ni + (unsigned)cl(i, a.ni)];
}
// face average of a (.., ny, nx) field at (j, i), the bottom/top faces extrapolated
// (calcdef's form: ((1.875a - 1.25b) + 0.375c) accumulated left to right)
__device__ __forceinline__ float atw_s(const float *q, int f, int j, int i, int nk, int ny, int nx) {
    if (f == 0) {
        float r = 1.875f * q[o3(0, j, i, ny, nx)];
        r = r + (-1.25f) * q[o3(1, j, i, ny, nx)];
        return r + 0.375f * q[o3(2, j, i, ny, nx)];
    }
    if (f == nk) {
        float r = 1.875f * q[o3(nk - 1, j, i, ny, nx)];
        r = r + (-1.25f) * q[o3(nk - 2, j, i, ny, nx)];
        return r + 0.375f * q[o3(nk - 3, j, i, ny, nx)];
    }
    return 0.5f * (q[o3(f - 1, j, i, ny, nx)] + q[o3(f, j, i, ny, nx)]);
}
// the stress twin's face average of a mass carrier at a clamped column
__device__ __forceinline__ float atw_c(const TArgs &a, const float *p, int f, int j, int i) {
    const int nk = a.nk;
    if (f == 0) return (1.875f * c3(a, p, 0, j, i) + (-1.25f) * c3(a, p, 1, j, i)) + 0.375f * c3(a, p, 2, j, i);
    if (f == nk)
        return (1.875f * c3(a, p, nk - 1, j, i) + (-1.25f) * c3(a, p, nk - 2, j, i)) + 0.375f * c3(a, p, nk - 3, j, i);
    return 0.5f * (c3(a, p, f - 1, j, i) + c3(a, p, f, j, i));
}
// the same on t12 (nk, nj+1, ni+1) at corner (jf, iface)
__device__ __forceinline__ float atw_xy(const TArgs &a, int f, int jf, int iface) {
    const int nk = a.nk, ny = a.nj + 1, nx = a.ni + 1;
    const float *q = a.t12;
    if (f == 0) return (1.875f * q[o3(0, jf, iface, ny, nx)] + (-1.25f) * q[o3(1, jf, iface, ny, nx)]) + 0.375f * q[o3(2, jf, iface, ny, nx)];
    if (f == nk)
        return (1.875f * q[o3(nk - 1, jf, iface, ny, nx)] + (-1.25f) * q[o3(nk - 2, jf, iface, ny, nx)]) +
               0.375f * q[o3(nk - 3, jf, iface, ny, nx)];
    return 0.5f * (q[o3(f - 1, jf, iface, ny, nx)] + q[o3(f, jf, iface, ny, nx)]);
}

// ---------------------------------------------------------------- strain
__global__ void __launch_bounds__(kEW) terrain_strain_kernel(TArgs a) {
    const int ni = a.ni, nj = a.nj, nk = a.nk, ux = ni + 1, vy = nj + 1;
    const float rdx = 1.0f / a.dx, rdy = 1.0f / a.dy, rds = 1.0f / a.dz, dz = a.dz;
    const float half = 0.5f, quarter = 0.25f, zt = (float)nk * dz;
    const size_t total = (size_t)(nk + 1) * vy * ux;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int ic = (int)(q % ux), jc = (int)((q / ux) % vy), k = (int)(q / ((size_t)ux * vy));
        if (k < nk) {
            if (ic < ni && jc < nj) {
                const int j = jc, i = ic;
                const unsigned p = o3(k, j, i, nj, ni);
                const float g = a.gz[j * ni + i];
                float hor = g * (a.u[o3(k, j, i + 1, nj, ux)] * a.rgzu[j * ux + i + 1] - a.u[o3(k, j, i, nj, ux)] * a.rgzu[j * ux + i]);
                hor = hor * rdx;
                float up = a.gx[o3(k + 1, j, i, nj, ni)] * (atw_s(a.u, k + 1, j, i, nk, nj, ux) + atw_s(a.u, k + 1, j, i + 1, nk, nj, ux));
                float lo = a.gx[o3(k, j, i, nj, ni)] * (atw_s(a.u, k, j, i, nk, nj, ux) + atw_s(a.u, k, j, i + 1, nk, nj, ux));
                float vert = ((up - lo) * half) * rds;
                a.s11[p] = (hor + vert) * a.rho[p];
                hor = g * (a.v[o3(k, j + 1, i, vy, ni)] * a.rgzv[(j + 1) * ni + i] - a.v[o3(k, j, i, vy, ni)] * a.rgzv[j * ni + i]);
                hor = hor * rdy;
                up = a.gy[o3(k + 1, j, i, nj, ni)] * (atw_s(a.v, k + 1, j, i, nk, vy, ni) + atw_s(a.v, k + 1, j + 1, i, nk, vy, ni));
                lo = a.gy[o3(k, j, i, nj, ni)] * (atw_s(a.v, k, j, i, nk, vy, ni) + atw_s(a.v, k, j + 1, i, nk, vy, ni));
                vert = ((up - lo) * half) * rds;
                a.s22[p] = (hor + vert) * a.rho[p];
                a.s33[p] = (((a.w[o3(k + 1, j, i, nj, ni)] - a.w[o3(k, j, i, nj, ni)]) * rds) * g) * a.rho[p];
            }
            const float sig_lo = (float)k * dz, sig_hi = (float)(k + 1) * dz;
            const int jj = clr(jc, 1, nj - 1), ii = clr(ic, 1, ni - 1);
            float r1 = (a.rho[o3(k, jj - 1, ii - 1, nj, ni)] * a.gz[(jj - 1) * ni + ii - 1] + a.rho[o3(k, jj, ii, nj, ni)] * a.gz[jj * ni + ii]) +
                       (a.rho[o3(k, jj, ii - 1, nj, ni)] * a.gz[jj * ni + ii - 1] + a.rho[o3(k, jj - 1, ii, nj, ni)] * a.gz[(jj - 1) * ni + ii]);
            r1 = quarter * r1;
            const float x1 = (r1 * (a.u[o3(k, jj, ii, nj, ux)] * a.rgzu[jj * ux + ii] - a.u[o3(k, jj - 1, ii, nj, ux)] * a.rgzu[(jj - 1) * ux + ii])) * rdy;
            const float xu = (zt - sig_hi) * (atw_s(a.u, k + 1, jj - 1, ii, nk, nj, ux) + atw_s(a.u, k + 1, jj, ii, nk, nj, ux));
            const float xl = (zt - sig_lo) * (atw_s(a.u, k, jj - 1, ii, nk, nj, ux) + atw_s(a.u, k, jj, ii, nk, nj, ux));
            const float x2 = ((((half * (xu - xl)) * rds) * r1) * (a.rgzu[jj * ux + ii] - a.rgzu[(jj - 1) * ux + ii])) * rdy;
            const float y1 = (r1 * (a.v[o3(k, jj, ii, vy, ni)] * a.rgzv[jj * ni + ii] - a.v[o3(k, jj, ii - 1, vy, ni)] * a.rgzv[jj * ni + ii - 1])) * rdx;
            const float yu = (zt - sig_hi) * (atw_s(a.v, k + 1, jj, ii - 1, nk, vy, ni) + atw_s(a.v, k + 1, jj, ii, nk, vy, ni));
            const float yl = (zt - sig_lo) * (atw_s(a.v, k, jj, ii - 1, nk, vy, ni) + atw_s(a.v, k, jj, ii, nk, vy, ni));
            const float y2 = ((((half * (yu - yl)) * rds) * r1) * (a.rgzv[jj * ni + ii] - a.rgzv[jj * ni + ii - 1])) * rdx;
            a.s12[o3(k, jc, ic, vy, ux)] = half * ((x1 + x2) + (y1 + y2));
        }
        if (k >= 1 && k < nk) {
            const int kf = k;
            const float sig_l = ((float)kf - half) * dz, sig_u = ((float)kf + half) * dz;
            if (jc < nj) {
                const int j = jc, il = ic - 1 < 0 ? 0 : ic - 1, ir = ic < ni - 1 ? ic : ni - 1;
                const float du = (a.u[o3(kf, j, ic, nj, ux)] - a.u[o3(kf - 1, j, ic, nj, ux)]) * rds;
                const float hw = (a.w[o3(kf, j, ir, nj, ni)] * a.rgz[j * ni + ir] - a.w[o3(kf, j, il, nj, ni)] * a.rgz[j * ni + il]) * rdx;
                const float wu = (zt - sig_u) * (half * (a.w[o3(kf, j, ir, nj, ni)] + a.w[o3(kf + 1, j, ir, nj, ni)]) +
                                                 half * (a.w[o3(kf, j, il, nj, ni)] + a.w[o3(kf + 1, j, il, nj, ni)]));
                const float wl = (zt - sig_l) * (half * (a.w[o3(kf - 1, j, ir, nj, ni)] + a.w[o3(kf, j, ir, nj, ni)]) +
                                                 half * (a.w[o3(kf - 1, j, il, nj, ni)] + a.w[o3(kf, j, il, nj, ni)]));
                const float terrain = (((half * rds) * (wu - wl)) * (a.rgz[j * ni + ir] - a.rgz[j * ni + il])) * rdx;
                const float strain = half * ((du + hw) + terrain);
                const float density = half * (a.gz[j * ni + il] * a.rf[o3(kf, j, il, nj, ni)] + a.gz[j * ni + ir] * a.rf[o3(kf, j, ir, nj, ni)]);
                a.s13[o3(kf, j, ic, nj, ux)] = strain * density;
            }
            if (ic < ni) {
                const int i = ic, jb = jc - 1 < 0 ? 0 : jc - 1, jt = jc < nj - 1 ? jc : nj - 1;
                const float dv = (a.v[o3(kf, jc, i, vy, ni)] - a.v[o3(kf - 1, jc, i, vy, ni)]) * rds;
                const float hw = (a.w[o3(kf, jt, i, nj, ni)] * a.rgz[jt * ni + i] - a.w[o3(kf, jb, i, nj, ni)] * a.rgz[jb * ni + i]) * rdy;
                const float wu = (zt - sig_u) * (half * (a.w[o3(kf, jt, i, nj, ni)] + a.w[o3(kf + 1, jt, i, nj, ni)]) +
                                                 half * (a.w[o3(kf, jb, i, nj, ni)] + a.w[o3(kf + 1, jb, i, nj, ni)]));
                const float wl = (zt - sig_l) * (half * (a.w[o3(kf - 1, jt, i, nj, ni)] + a.w[o3(kf, jt, i, nj, ni)]) +
                                                 half * (a.w[o3(kf - 1, jb, i, nj, ni)] + a.w[o3(kf, jb, i, nj, ni)]));
                const float terrain = (((half * rds) * (wu - wl)) * (a.rgz[jt * ni + i] - a.rgz[jb * ni + i])) * rdy;
                const float strain = half * ((dv + hw) + terrain);
                const float density = half * (a.gz[jb * ni + i] * a.rf[o3(kf, jb, i, nj, ni)] + a.gz[jt * ni + i] * a.rf[o3(kf, jt, i, nj, ni)]);
                a.s23[o3(kf, jc, i, vy, ni)] = strain * density;
            }
        }
    }
}

// ---------------------------------------------------------------- gettau
__global__ void __launch_bounds__(kEW) terrain_gettau_kernel(TArgs a) {
    const int ni = a.ni, nj = a.nj, nk = a.nk, ux = ni + 1, vy = nj + 1;
    const size_t total = (size_t)(nk + 1) * vy * ux;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int ic = (int)(q % ux), jc = (int)((q / ux) % vy), k = (int)(q / ((size_t)ux * vy));
        if (k < nk) {
            if (ic < ni && jc < nj) {
                const unsigned p = o3(k, jc, ic, nj, ni);
                const float tem = a.kmh[p] + a.kmh[o3(k + 1, jc, ic, nj, ni)];
                a.t11[p] = a.s11[p] * tem;
                a.t22[p] = a.s22[p] * tem;
                a.t33[p] = a.s33[p] * tem;
            }
            float total12 = 0.0f;
            for (int kf = k; kf <= k + 1; ++kf)
                for (int jj = jc - 1; jj <= jc; ++jj)
                    for (int ii = ic - 1; ii <= ic; ++ii) total12 = total12 + c3(a, a.kmh, kf, jj, ii);
            const unsigned p12 = o3(k, jc, ic, vy, ux);
            a.t12[p12] = a.s12[p12] * (0.25f * total12);
        }
        const int ff = k == 0 ? 1 : (k == nk ? nk - 1 : k);
        if (jc < nj)
            a.t13[o3(k, jc, ic, nj, ux)] = a.s13[o3(ff, jc, ic, nj, ux)] * (c3(a, a.kmv, ff, jc, ic - 1) + c3(a, a.kmv, ff, jc, ic));
        if (ic < ni)
            a.t23[o3(k, jc, ic, vy, ni)] = a.s23[o3(ff, jc, ic, vy, ni)] * (c3(a, a.kmv, ff, jc - 1, ic) + c3(a, a.kmv, ff, jc, ic));
    }
}

// ------------------------------------------------------- turbu and turbv
template <int DIR>
__global__ void __launch_bounds__(kCT) terrain_turb_uv_kernel(TArgs a) {
    extern __shared__ float s_col[];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kCX + tx;
    const int ni = a.ni, nj = a.nj, nk = a.nk, ux = ni + 1, vy = nj + 1;
    const int cx = blockIdx.x * kCX + tx, cy = blockIdx.y * kCY + ty;
    if (DIR == 0 ? (cx > ni || cy >= nj) : (cx >= ni || cy > nj)) return;
    // DIR 0: u column (j = cy, iface = cx), cells (j, cx-1), (j, cx); DIR 1: v column (jface = cy, i = cx)
    const int ja = DIR == 0 ? cy : cy - 1, jb = cy, ia = DIR == 0 ? cx - 1 : cx, ib = cx;
    const float *q = DIR == 0 ? a.u : a.v, *top = DIR == 0 ? a.t13 : a.t23;
    float *ten = DIR == 0 ? a.uten : a.vten;
    const unsigned col = DIR == 0 ? (unsigned)cy * ux + cx : (unsigned)cy * ni + cx;
    const unsigned lev = DIR == 0 ? (unsigned)nj * ux : (unsigned)vy * ni;
    const float rdx = 1.0f / a.dx, rdy = 1.0f / a.dy, dz = a.dz, dt = a.dt, rdz = 1.0f / dz, zt = (float)nk * dz;
    const float rd = DIR == 0 ? rdx : rdy;
    const float tema = -0.0625f * (dt * (rdz * rdz)), temc = 0.5f * (dt * rdz), rdt = 0.5f / dt;
    float *cp = s_col, *dp = s_col + (size_t)nk * kCT;
#define CP(k) cp[(unsigned)(k) * kCT + tid]
#define DP(k) dp[(unsigned)(k) * kCT + tid]
#define PAIR(p, k) (c3(a, p, k, ja, ia) + c3(a, p, k, jb, ib))
#define QK(k) q[(unsigned)(k) * lev + col]
#define WA(k) a.w[o3(k, cl(ja, nj), cl(ia, ni), nj, ni)]
#define WB(k) a.w[o3(k, cl(jb, nj), cl(ib, ni), nj, ni)]
    const float rg_a = c2(a, a.rgz, ja, ia), rg_b = c2(a, a.rgz, jb, ib);
    const float gza = c2(a, a.gz, ja, ia), gzb = c2(a, a.gz, jb, ib);
    // forward elimination
    float kmv_u = PAIR(a.kmv, 1), mf_u = PAIR(a.mf, 1), rf_u = PAIR(a.rf, 1);
    {
        const float rr0 = 1.0f / (0.5f * PAIR(a.rho, 0)), mhp = PAIR(a.mh, 0);
        const float r2v = kmv_u * (mf_u * (rf_u * (mhp * rr0)));
        const float cfc = tema * r2v, cfb = 1.0f - cfc, cfd = QK(0) - temc * (top[col] * (mhp * rr0));
        const float inv = 1.0f / cfb;
        CP(0) = -1.0f * (cfc * inv);
        DP(0) = cfd * inv;
    }
    float cprev = CP(0), dprev = DP(0);
    #pragma unroll 4
    for (int k = 1; k < nk - 1; ++k) {
        const float rr0 = 1.0f / (0.5f * PAIR(a.rho, k)), common = PAIR(a.mh, k) * rr0;
        const float r1v = kmv_u * (mf_u * (rf_u * common));
        kmv_u = PAIR(a.kmv, k + 1);
        mf_u = PAIR(a.mf, k + 1);
        rf_u = PAIR(a.rf, k + 1);
        const float r2v = kmv_u * (mf_u * (rf_u * common));
        const float cfa = tema * r1v, cfc = tema * r2v, cfb = (1.0f - cfa) - cfc;
        const float inv = 1.0f / (cfa * cprev + cfb);
        cprev = -1.0f * (cfc * inv);
        dprev = (QK(k) - cfa * dprev) * inv;
        CP(k) = cprev;
        DP(k) = dprev;
    }
    float sol;
    {
        const int k = nk - 1;
        const float rr0 = 1.0f / (0.5f * PAIR(a.rho, k)), mhp = PAIR(a.mh, k);
        const float r1v = kmv_u * (mf_u * (rf_u * (mhp * rr0)));
        const float cfa = tema * r1v, cfb = 1.0f - cfa;
        const float cfd = QK(k) + temc * (top[(unsigned)nk * lev + col] * (mhp * rr0));
        sol = (cfd - cfa * dprev) * (1.0f / (cfa * cprev + cfb));
    }
    // back substitution, the cross term and the tendency per level
    float r1 = 0.0f, r2 = 0.0f;
    if (DIR == 0) {
        r1 = 0.25f * ((c2(a, a.rgz, cy - 1, ia) + c2(a, a.rgz, cy, ib)) + (c2(a, a.rgz, cy, ia) + c2(a, a.rgz, cy - 1, ib)));
        r2 = 0.25f * ((c2(a, a.rgz, cy + 1, ia) + c2(a, a.rgz, cy, ib)) + (c2(a, a.rgz, cy, ia) + c2(a, a.rgz, cy + 1, ib)));
    } else {
        r1 = 0.25f * ((c2(a, a.rgz, ja, cx - 1) + c2(a, a.rgz, jb, cx)) + (c2(a, a.rgz, jb, cx - 1) + c2(a, a.rgz, ja, cx)));
        r2 = 0.25f * ((c2(a, a.rgz, ja, cx + 1) + c2(a, a.rgz, jb, cx)) + (c2(a, a.rgz, jb, cx + 1) + c2(a, a.rgz, ja, cx)));
    }
    const float g = DIR == 0 ? a.gzu[(unsigned)cy * ux + cx] : a.gzv[(unsigned)cy * ni + cx];
    float cross_up = 0.0f;  // cross(k+1); zero above the top level
    #pragma unroll 4
    for (int k = nk - 1; k >= 0; --k) {
        if (k < nk - 1) sol = CP(k) * sol + DP(k);
        float cross = 0.0f;
        if (k >= 1) {
            const float wm = 0.5f * (WB(k) + WB(k + 1)), wl = 0.5f * (WA(k) + WA(k + 1));
            const float grad = (WB(k) * rg_b - WA(k) * rg_a) * rd;
            const float below = 0.5f * (WB(k - 1) + WB(k)) + 0.5f * (WA(k - 1) + WA(k));
            const float terrain = 0.5f * (((zt - ((float)k + 0.5f) * dz) * (wm + wl) - (zt - ((float)k - 0.5f) * dz) * below) *
                                          (rdz * ((rg_b - rg_a) * rd)));
            cross = (grad + terrain) * (0.25f * (PAIR(a.kmv, k) * (gza * c3(a, a.rf, k, ja, ia) + gzb * c3(a, a.rf, k, jb, ib))));
        }
        float hx, hy;
        if (DIR == 0) {
            const float x = g * ((c3(a, a.t11, k, cy, ib) * rg_b - c3(a, a.t11, k, cy, ia) * rg_a) * rdx);
            const float up = a.gxu[o3(k + 1, cy, cx, nj, ux)] * (atw_c(a, a.t11, k + 1, cy, ia) + atw_c(a, a.t11, k + 1, cy, ib));
            const float lo = a.gxu[o3(k, cy, cx, nj, ux)] * (atw_c(a, a.t11, k, cy, ia) + atw_c(a, a.t11, k, cy, ib));
            hx = x + 0.5f * ((up - lo) * rdz);
            const float y = g * ((a.t12[o3(k, cy + 1, cx, vy, ux)] * r2 - a.t12[o3(k, cy, cx, vy, ux)] * r1) * rdy);
            const float su = (zt - (float)(k + 1) * dz) * (atw_xy(a, k + 1, cy, cx) + atw_xy(a, k + 1, cy + 1, cx));
            const float sl = (zt - (float)k * dz) * (atw_xy(a, k, cy, cx) + atw_xy(a, k, cy + 1, cx));
            hy = y + 0.5f * ((su - sl) * (g * ((r2 - r1) * (rdy * rdz))));
            if (cx == 0 || cx == ni) hx = 0.0f;
            if (cy == 0 || cy == nj - 1) hy = 0.0f;
        } else {
            const float x = g * ((a.t12[o3(k, cy, cx + 1, vy, ux)] * r2 - a.t12[o3(k, cy, cx, vy, ux)] * r1) * rdx);
            const float su = (zt - (float)(k + 1) * dz) * (atw_xy(a, k + 1, cy, cx) + atw_xy(a, k + 1, cy, cx + 1));
            const float sl = (zt - (float)k * dz) * (atw_xy(a, k, cy, cx) + atw_xy(a, k, cy, cx + 1));
            hx = x + 0.5f * ((su - sl) * (g * ((r2 - r1) * (rdx * rdz))));
            const float y = g * ((c3(a, a.t22, k, jb, cx) * rg_b - c3(a, a.t22, k, ja, cx) * rg_a) * rdy);
            const float up = a.gyv[o3(k + 1, cy, cx, vy, ni)] * (atw_c(a, a.t22, k + 1, ja, cx) + atw_c(a, a.t22, k + 1, jb, cx));
            const float lo = a.gyv[o3(k, cy, cx, vy, ni)] * (atw_c(a, a.t22, k, ja, cx) + atw_c(a, a.t22, k, jb, cx));
            hy = y + 0.5f * ((up - lo) * rdz);
            if (cx == 0 || cx == ni - 1) hx = 0.0f;
            if (cy == 0 || cy == nj) hy = 0.0f;
        }
        const float rho_p = PAIR(a.rho, k), mhp = PAIR(a.mh, k);
        float vert = rho_p * ((sol - QK(k)) * rdt);
        vert = vert + (cross_up - cross) * (rdz * (0.5f * mhp));
        cross_up = cross;
        const unsigned p = (unsigned)k * lev + col;
        ten[p] = ten[p] + ((hx + hy) + vert) / (0.5f * rho_p);
    }
#undef CP
#undef DP
#undef PAIR
#undef QK
#undef WA
#undef WB
}

// ----------------------------------------------------------------- turbw
__global__ void __launch_bounds__(kCT) terrain_turbw_kernel(TArgs a) {
    extern __shared__ float s_col[];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kCX + tx;
    const int ni = a.ni, nj = a.nj, nk = a.nk, ux = ni + 1, vy = nj + 1;
    const int i = blockIdx.x * kCX + tx, j = blockIdx.y * kCY + ty;
    if (i >= ni || j >= nj) return;
    const unsigned col = (unsigned)j * ni + i, lev = (unsigned)nj * ni;
    const float rdx = 1.0f / a.dx, rdy = 1.0f / a.dy, dz = a.dz, dt = a.dt, rdz = 1.0f / dz, zt = (float)nk * dz;
    const float tema = -1.0f * (dt * (rdz * rdz)), temc = dt * rdz, rdt = 1.0f / dt;
    float *cp = s_col, *dp = s_col + (size_t)nk * kCT;
#define CP(p) cp[(unsigned)(p) * kCT + tid]
#define DP(p) dp[(unsigned)(p) * kCT + tid]
#define PF(p, f) p[(unsigned)(f) * lev + col]
#define T13(f, ii) a.t13[o3(f, j, ii, nj, ux)]
#define T23(f, jj) a.t23[o3(f, jj, i, vy, ni)]
    {
        const int f = 1;
        const float rrf = PF(a.mf, f) / PF(a.rf, f);
        const float r2v = (PF(a.kmh, f) + PF(a.kmh, f + 1)) * (PF(a.mh, f) * (PF(a.rho, f) * rrf));
        const float cfc = tema * r2v, cfb = 1.0f - cfc, cfd = PF(a.w, f) - temc * (PF(a.t33, 0) * rrf);
        const float inv = 1.0f / cfb;
        CP(0) = -1.0f * (cfc * inv);
        DP(0) = cfd * inv;
    }
    float cprev = CP(0), dprev = DP(0);
    #pragma unroll 4
    for (int f = 2; f < nk - 1; ++f) {
        const float rrf = PF(a.mf, f) / PF(a.rf, f);
        const float r1v = (PF(a.kmh, f - 1) + PF(a.kmh, f)) * (PF(a.mh, f - 1) * (PF(a.rho, f - 1) * rrf));
        const float r2v = (PF(a.kmh, f) + PF(a.kmh, f + 1)) * (PF(a.mh, f) * (PF(a.rho, f) * rrf));
        const float cfa = tema * r1v, cfc = tema * r2v, cfb = (1.0f - cfa) - cfc;
        const float inv = 1.0f / (cfa * cprev + cfb);
        cprev = -1.0f * (cfc * inv);
        dprev = (PF(a.w, f) - cfa * dprev) * inv;
        CP(f - 1) = cprev;
        DP(f - 1) = dprev;
    }
    float sol;
    {
        const int f = nk - 1;
        const float rrf = PF(a.mf, f) / PF(a.rf, f);
        const float r1v = (PF(a.kmh, f - 1) + PF(a.kmh, f)) * (PF(a.mh, f - 1) * (PF(a.rho, f - 1) * rrf));
        const float cfa = tema * r1v, cfb = 1.0f - cfa, cfd = PF(a.w, f) + temc * (PF(a.t33, nk - 1) * rrf);
        sol = (cfd - cfa * dprev) * (1.0f / (cfa * cprev + cfb));
    }
    const float g = a.gz[col];
    #pragma unroll 4
    for (int f = nk - 1; f >= 1; --f) {
        if (f < nk - 1) sol = CP(f - 1) * sol + DP(f - 1);
        const float d1 = 0.25f * ((T13(f + 1, i) + T13(f + 1, i + 1)) + (T13(f, i) + T13(f, i + 1)));
        const float d0 = 0.25f * ((T13(f, i) + T13(f, i + 1)) + (T13(f - 1, i) + T13(f - 1, i + 1)));
        float x = g * ((T13(f, i + 1) * a.rgzu[j * ux + i + 1] - T13(f, i) * a.rgzu[j * ux + i]) * rdx);
        x = x + ((zt - ((float)f + 0.5f) * dz) * d1 - (zt - ((float)f - 0.5f) * dz) * d0) *
                    (g * ((a.rgzu[j * ux + i + 1] - a.rgzu[j * ux + i]) * (rdx * rdz)));
        const float e1 = 0.25f * ((T23(f + 1, j) + T23(f + 1, j + 1)) + (T23(f, j) + T23(f, j + 1)));
        const float e0 = 0.25f * ((T23(f, j) + T23(f, j + 1)) + (T23(f - 1, j) + T23(f - 1, j + 1)));
        float y = g * ((T23(f, j + 1) * a.rgzv[(j + 1) * ni + i] - T23(f, j) * a.rgzv[j * ni + i]) * rdy);
        y = y + ((zt - ((float)f + 0.5f) * dz) * e1 - (zt - ((float)f - 0.5f) * dz) * e0) *
                    (g * ((a.rgzv[(j + 1) * ni + i] - a.rgzv[j * ni + i]) * (rdy * rdz)));
        const float h = (i == 0 || i == ni - 1 ? 0.0f : x) + (j == 0 || j == nj - 1 ? 0.0f : y);
        const float rff = PF(a.rf, f);
        const float vert = rff * ((sol - PF(a.w, f)) * rdt);
        const unsigned p = (unsigned)f * lev + col;
        a.wten[p] = a.wten[p] + (h + vert) / rff;
    }
#undef CP
#undef DP
#undef PF
#undef T13
#undef T23
}

// --------------------------------------------------------- turbs (terrain)
struct SArgs {
    const float *th0, *tha, *qa, *rho, *rr, *rf, *mh, *mf, *khh, *khv, *gz, *rgz, *rgzu, *rgzv, *gx, *gxu, *gy, *gyv;
    float *thten, *qten, *work;
    int ni, nj, nk, nsc;
    float dx, dy, dz, dt;
};

__device__ __forceinline__ float sc3(const SArgs &a, const float *p, int k, int j, int i) {
    return p[o3(k, cl(j, a.nj), cl(i, a.ni), a.nj, a.ni)];
}
__device__ __forceinline__ float sc2(const SArgs &a, const float *p, int j, int i) {
    return p[(unsigned)cl(j, a.nj) * (unsigned)a.ni + (unsigned)cl(i, a.ni)];
}
__device__ __forceinline__ float sv(const SArgs &a, int sc, int k, int j, int i) {
    const unsigned p = o3(k, cl(j, a.nj), cl(i, a.ni), a.nj, a.ni);
    if (sc > 0) return a.qa[(size_t)(sc - 1) * ((size_t)a.ni * a.nj * a.nk) + p];
    return (a.th0[k] - 300.0f) + a.tha[p];
}
// the scalar at w face f (the twin's _at_w)
__device__ __forceinline__ float sw(const SArgs &a, int sc, int f, int j, int i) {
    const int nk = a.nk;
    if (f == 0) return (1.875f * sv(a, sc, 0, j, i) + (-1.25f) * sv(a, sc, 1, j, i)) + 0.375f * sv(a, sc, 2, j, i);
    if (f == nk) return (1.875f * sv(a, sc, nk - 1, j, i) + (-1.25f) * sv(a, sc, nk - 2, j, i)) + 0.375f * sv(a, sc, nk - 3, j, i);
    return 0.5f * sv(a, sc, f - 1, j, i) + 0.5f * sv(a, sc, f, j, i);
}

// workspace of scalar sc: fx (nk, nj, ni+1) then fy (nk, nj+1, ni)
__device__ __forceinline__ float *fx_of(const SArgs &a, int sc) {
    const size_t per = (size_t)a.nk * a.nj * (a.ni + 1) + (size_t)a.nk * (a.nj + 1) * a.ni;
    return a.work + (size_t)sc * per;
}
__device__ __forceinline__ float *fy_of(const SArgs &a, int sc) { return fx_of(a, sc) + (size_t)a.nk * a.nj * (a.ni + 1); }

__global__ void __launch_bounds__(kEW) terrain_turbs_flux_kernel(SArgs a) {
    const int ni = a.ni, nj = a.nj, nk = a.nk, ux = ni + 1, vy = nj + 1;
    const float rdx = 1.0f / a.dx, rdy = 1.0f / a.dy, rdz = 1.0f / a.dz;
    const size_t nxf = (size_t)nk * nj * ux, nyf = (size_t)nk * vy * ni, total = nxf + nyf;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        if (q < nxf) {
            const int face = (int)(q % ux), j = (int)((q / ux) % nj), k = (int)(q / ((size_t)ux * nj));
            const int il = face - 1, ir = face;
            const float den = sc2(a, a.gz, j, ir) * sc3(a, a.rho, k, j, ir) + sc2(a, a.gz, j, il) * sc3(a, a.rho, k, j, il);
            const float dif = (sc3(a, a.khh, k, j, ir) + sc3(a, a.khh, k, j, il)) + (sc3(a, a.khh, k + 1, j, ir) + sc3(a, a.khh, k + 1, j, il));
            const float fac = (-0.125f * den) * dif;
            const float rr_ = sc2(a, a.rgz, j, ir), rl_ = sc2(a, a.rgz, j, il);
            const float gu = a.gxu[o3(k + 1, j, face, nj, ux)], gl = a.gxu[o3(k, j, face, nj, ux)], rzu = a.rgzu[j * ux + face];
            for (int sc = 0; sc < a.nsc; ++sc) {
                const float hor = (sv(a, sc, k, j, ir) * rr_ - sv(a, sc, k, j, il) * rl_) * rdx;
                const float up = gu * (sw(a, sc, k + 1, j, ir) + sw(a, sc, k + 1, j, il));
                const float lo = gl * (sw(a, sc, k, j, ir) + sw(a, sc, k, j, il));
                const float ter = ((0.5f * (up - lo)) * rdz) * rzu;
                fx_of(a, sc)[q] = fac * (hor + ter);
            }
        } else {
            const size_t z = q - nxf;
            const int i = (int)(z % ni), face = (int)((z / ni) % vy), k = (int)(z / ((size_t)ni * vy));
            const int js = face - 1, jn = face;
            const float den = sc2(a, a.gz, jn, i) * sc3(a, a.rho, k, jn, i) + sc2(a, a.gz, js, i) * sc3(a, a.rho, k, js, i);
            const float dif = (sc3(a, a.khh, k, jn, i) + sc3(a, a.khh, k, js, i)) + (sc3(a, a.khh, k + 1, jn, i) + sc3(a, a.khh, k + 1, js, i));
            const float fac = (-0.125f * den) * dif;
            const float rn_ = sc2(a, a.rgz, jn, i), rs_ = sc2(a, a.rgz, js, i);
            const float gu = a.gyv[o3(k + 1, face, i, vy, ni)], gl = a.gyv[o3(k, face, i, vy, ni)], rzv = a.rgzv[face * ni + i];
            for (int sc = 0; sc < a.nsc; ++sc) {
                const float hor = (sv(a, sc, k, jn, i) * rn_ - sv(a, sc, k, js, i) * rs_) * rdy;
                const float up = gu * (sw(a, sc, k + 1, jn, i) + sw(a, sc, k + 1, js, i));
                const float lo = gl * (sw(a, sc, k, jn, i) + sw(a, sc, k, js, i));
                const float ter = ((0.5f * (up - lo)) * rdz) * rzv;
                fy_of(a, sc)[z] = fac * (hor + ter);
            }
        }
    }
}

// a flux column's value at w face f (the twin's _interpolate_flux)
__device__ __forceinline__ float fw(const float *col, size_t stride, int f, int nk) {
    if (f == 0) return (1.875f * col[0] + (-1.25f) * col[stride]) + 0.375f * col[2 * stride];
    if (f == nk) return (1.875f * col[(nk - 1) * stride] + (-1.25f) * col[(nk - 2) * stride]) + 0.375f * col[(nk - 3) * stride];
    return 0.5f * col[(f - 1) * stride] + 0.5f * col[f * stride];
}

__global__ void __launch_bounds__(kCT) terrain_turbs_column_kernel(SArgs a) {
    extern __shared__ float s_col[];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kCX + tx;
    const int ni = a.ni, nj = a.nj, nk = a.nk, ux = ni + 1, vy = nj + 1;
    const int i = blockIdx.x * kCX + tx, j = blockIdx.y * kCY + ty;
    if (i >= ni || j >= nj) return;
    const size_t n = (size_t)ni * nj * nk, zu = (size_t)nj * ux, zv = (size_t)vy * ni;
    const unsigned col = (unsigned)j * ni + i, lev = (unsigned)nj * ni;
    float *cp = s_col, *dp = s_col + (size_t)nk * kCT;
#define CP(k) cp[(unsigned)(k) * kCT + tid]
#define DP(k) dp[(unsigned)(k) * kCT + tid]
#define PF(p, k) p[(unsigned)(k) * lev + col]
#define COEF(F, K) ((((PF(a.khv, F) * PF(a.mf, F)) * PF(a.rf, F)) * PF(a.mh, K)) * PF(a.rr, K))
    const float rdx = 1.0f / a.dx, rdy = 1.0f / a.dy, rdz = 1.0f / a.dz, dt = a.dt, rdt = 1.0f / dt;
    const float tema = (((-1.0f * dt) * 1.0f) * rdz) * rdz;
    const float temb = ((dt * 0.0f) * rdz) * rdz;
    const float temc = dt * rdz;
    const float g = a.gz[col];
    for (int sc = 0; sc < a.nsc; ++sc) {
        float *target = sc == 0 ? a.thten : a.qten + (size_t)(sc - 1) * n;
        const float *fxc = fx_of(a, sc) + (size_t)j * ux + i, *fyc = fy_of(a, sc) + (size_t)j * ni + i;
#define SC(k) sv(a, sc, k, j, i)
        float sm = SC(0), sk = SC(1);
        float r2 = COEF(1, 0);
        float cfc = tema * r2, cfb = 1.0f - cfc;
        float ex = (-r2) * sm + r2 * sk;
        float bc = ((temc * 0.0f) * PF(a.mh, 0)) * PF(a.rr, 0);
        float cfd = (sm + temb * ex) + bc;
        float tem = 1.0f / cfb;
        float cprev = (-cfc) * tem, dprev = cfd * tem;
        CP(0) = cprev;
        DP(0) = dprev;
        #pragma unroll 4
        for (int k = 1; k + 1 < nk; ++k) {
            const float r1 = COEF(k, k);
            r2 = COEF(k + 1, k);
            const float cfa = tema * r1;
            cfc = tema * r2;
            cfb = (1.0f - cfa) - cfc;
            const float sp1 = SC(k + 1);
            ex = (r1 * sm - (r1 + r2) * sk) + r2 * sp1;
            cfd = sk + temb * ex;
            tem = 1.0f / (cfa * cprev + cfb);
            cprev = (-cfc) * tem;
            dprev = (cfd - cfa * dprev) * tem;
            CP(k) = cprev;
            DP(k) = dprev;
            sm = sk;
            sk = sp1;
        }
        float sol;
        {
            const int k = nk - 1;
            const float r1 = COEF(k, k), cfa = tema * r1;
            cfb = 1.0f - cfa;
            ex = r1 * sm - r1 * sk;
            bc = ((temc * 0.0f) * PF(a.mh, k)) * PF(a.rr, k);
            cfd = (sk + temb * ex) - bc;
            tem = 1.0f / (cfa * cprev + cfb);
            sol = (cfd - cfa * dprev) * tem;
        }
        #pragma unroll 4
        for (int k = nk - 1; k >= 0; --k) {
            if (k != nk - 1) sol = CP(k) * sol + DP(k);
            const float turbz = (PF(a.rho, k) * (sol - SC(k))) * rdt;
            const float right = fxc[(size_t)k * zu + 1] * a.rgzu[j * ux + i + 1], left = fxc[(size_t)k * zu] * a.rgzu[j * ux + i];
            const float tx0 = ((-g) * (right - left)) * rdx;
            const float upx = a.gx[o3(k + 1, j, i, nj, ni)] * (fw(fxc, zu, k + 1, nk) + fw(fxc + 1, zu, k + 1, nk));
            const float lox = a.gx[o3(k, j, i, nj, ni)] * (fw(fxc, zu, k, nk) + fw(fxc + 1, zu, k, nk));
            float txv = tx0 + ((-(upx - lox)) * 0.5f) * rdz;
            if (i == 0 || i == ni - 1) txv = 0.0f;
            const float north = fyc[(size_t)k * zv + ni] * a.rgzv[(j + 1) * ni + i], south = fyc[(size_t)k * zv] * a.rgzv[j * ni + i];
            const float ty0 = ((-g) * (north - south)) * rdy;
            const float upy = a.gy[o3(k + 1, j, i, nj, ni)] * (fw(fyc, zv, k + 1, nk) + fw(fyc + ni, zv, k + 1, nk));
            const float loy = a.gy[o3(k, j, i, nj, ni)] * (fw(fyc, zv, k, nk) + fw(fyc + ni, zv, k, nk));
            float tyv = ty0 + ((-(upy - loy)) * 0.5f) * rdz;
            if (j == 0 || j == nj - 1) tyv = 0.0f;
            const unsigned p = (unsigned)k * lev + col;
            target[p] = target[p] + ((txv + tyv) + turbz) * PF(a.rr, k);
        }
#undef SC
    }
#undef CP
#undef DP
#undef PF
#undef COEF
}

bool all_set(std::initializer_list<const void *> ps) {
    for (const void *p : ps)
        if (p == nullptr) return false;
    return true;
}

unsigned ew_blocks(size_t total) {
    const size_t want = (total + kEW - 1) / kEW, cap = (size_t)148 * 16;
    return (unsigned)(want < cap ? want : cap);
}

template <typename Kernel>
int configure(Kernel kernel, size_t smem, const char *name) {
    if (smem <= 48 * 1024) return GM1B_OK;
    const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
        cudaGetLastError();
        gm1b_set_error("cudaFuncSetAttribute(%s): %s", name, cudaGetErrorString(e));
        return GM1B_ERR_CUDA;
    }
    return GM1B_OK;
}

int check_grid(int ni, int nj, int nk, float dx, float dy, float dz, float dt, const char *what) {
    if (ni < 3 || nj < 3 || nk < 3 || nk > 200) {
        gm1b_set_error("%s: need ni >= 3, nj >= 3 and 3 <= nk <= 200", what);
        return GM1B_ERR_ARGUMENT;
    }
    if ((double)(nk + 1) * (nj + 1) * (ni + 1) >= 2147483648.0) {
        gm1b_set_error("%s: a %dx%dx%d grid reaches 2^31 words; the kernels index with 32-bit offsets", what, ni, nj, nk);
        return GM1B_ERR_ARGUMENT;
    }
    if (!(dx > 0.0f && dy > 0.0f && dz > 0.0f && dt > 0.0f) || !isfinite(dx) || !isfinite(dy) || !isfinite(dz) ||
        !isfinite(dt)) {
        gm1b_set_error("%s: dx, dy, dz, dt must be finite and > 0", what);
        return GM1B_ERR_ARGUMENT;
    }
    return GM1B_OK;
}

TArgs targs(int ni, int nj, int nk, const gm1b_terrain_stress_arrays *s, float dx, float dy, float dz, float dt) {
    return TArgs{s->u3d, s->v3d, s->w3d, s->rho, s->rf, s->mh,  s->mf,  s->kmh, s->kmv, s->gz,  s->rgz,  s->gzu,
                 s->rgzu, s->gzv, s->rgzv, s->gx, s->gy, s->gxu, s->gyv, s->s11, s->s22, s->s33, s->s12, s->s13,
                 s->s23, s->t11, s->t22, s->t33, s->t12, s->t13, s->t23, s->uten, s->vten, s->wten, ni,  nj,
                 nk,  dx,  dy,  dz,  dt};
}

}  // namespace
}  // namespace gm1b

using namespace gm1b;

extern "C" int32_t gm1b_terrain_strain(int32_t ni, int32_t nj, int32_t nk, const gm1b_terrain_stress_arrays *arrays,
                                       float dx, float dy, float dz, void *stream) {
    if (arrays == nullptr) {
        gm1b_set_error("gm1b_terrain_strain: NULL arrays");
        return GM1B_ERR_ARGUMENT;
    }
    TRY(check_grid(ni, nj, nk, dx, dy, dz, 1.0f, "gm1b_terrain_strain"));
    const TArgs a = targs(ni, nj, nk, arrays, dx, dy, dz, 1.0f);
    if (!all_set({a.u, a.v, a.w, a.rho, a.rf, a.gz, a.rgz, a.rgzu, a.rgzv, a.gx, a.gy, a.s11, a.s22, a.s33, a.s12, a.s13,
                  a.s23})) {
        gm1b_set_error("gm1b_terrain_strain: a required array is NULL");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("terrain_strain_kernel", st);
    terrain_strain_kernel<<<ew_blocks((size_t)(nk + 1) * (nj + 1) * (ni + 1)), kEW, 0, st>>>(a);
    ps.stop();
    return launch_ok("terrain_strain_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_terrain_stress(int32_t ni, int32_t nj, int32_t nk, const gm1b_terrain_stress_arrays *arrays,
                                       float dx, float dy, float dz, float dt, void *stream) {
    if (arrays == nullptr) {
        gm1b_set_error("gm1b_terrain_stress: NULL arrays");
        return GM1B_ERR_ARGUMENT;
    }
    TRY(check_grid(ni, nj, nk, dx, dy, dz, dt, "gm1b_terrain_stress"));
    const TArgs a = targs(ni, nj, nk, arrays, dx, dy, dz, dt);
    if (!all_set({a.s11, a.s22, a.s33, a.s12, a.s13, a.s23, a.kmh, a.kmv, a.t11, a.t22, a.t33, a.t12, a.t13, a.t23,
                  a.rho, a.rf, a.mh, a.mf, a.gz, a.rgz, a.gzu, a.rgzu, a.gzv, a.rgzv, a.gxu, a.gyv, a.u, a.v, a.w,
                  a.uten, a.vten, a.wten})) {
        gm1b_set_error("gm1b_terrain_stress: a required array is NULL");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    {
        ProfScope ps("terrain_gettau_kernel", st);
        terrain_gettau_kernel<<<ew_blocks((size_t)(nk + 1) * (nj + 1) * (ni + 1)), kEW, 0, st>>>(a);
        ps.stop();
        if (!launch_ok("terrain_gettau_kernel")) return GM1B_ERR_CUDA;
    }
    const size_t smem = (size_t)2 * nk * kCT * sizeof(float);
    TRY(configure(terrain_turb_uv_kernel<0>, smem, "terrain_turb_uv_kernel<0>"));
    TRY(configure(terrain_turb_uv_kernel<1>, smem, "terrain_turb_uv_kernel<1>"));
    TRY(configure(terrain_turbw_kernel, smem, "terrain_turbw_kernel"));
    {
        ProfScope ps("terrain_turbu_kernel", st);
        terrain_turb_uv_kernel<0><<<dim3((ni + 1 + kCX - 1) / kCX, (nj + kCY - 1) / kCY), dim3(kCX, kCY), smem, st>>>(a);
        ps.stop();
        if (!launch_ok("terrain_turbu_kernel")) return GM1B_ERR_CUDA;
    }
    {
        ProfScope ps("terrain_turbv_kernel", st);
        terrain_turb_uv_kernel<1><<<dim3((ni + kCX - 1) / kCX, (nj + 1 + kCY - 1) / kCY), dim3(kCX, kCY), smem, st>>>(a);
        ps.stop();
        if (!launch_ok("terrain_turbv_kernel")) return GM1B_ERR_CUDA;
    }
    ProfScope ps("terrain_turbw_kernel", st);
    terrain_turbw_kernel<<<dim3((ni + kCX - 1) / kCX, (nj + kCY - 1) / kCY), dim3(kCX, kCY), smem, st>>>(a);
    ps.stop();
    return launch_ok("terrain_turbw_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_terrain_sgs_stress(int32_t ni, int32_t nj, int32_t nk, const gm1b_terrain_stress_arrays *arrays,
                                           float dx, float dy, float dz, float dt, void *stream) {
    TRY(gm1b_terrain_strain(ni, nj, nk, arrays, dx, dy, dz, stream));
    return gm1b_terrain_stress(ni, nj, nk, arrays, dx, dy, dz, dt, stream);
}

extern "C" int64_t gm1b_terrain_scalar_turbulence_workspace_words(int32_t ni, int32_t nj, int32_t nk, int32_t numq) {
    if (ni < 1 || nj < 1 || nk < 1 || numq < 0) return 0;
    return (int64_t)(numq + 1) * ((int64_t)nk * nj * (ni + 1) + (int64_t)nk * (nj + 1) * ni);
}

extern "C" int32_t gm1b_terrain_scalar_turbulence(int32_t ni, int32_t nj, int32_t nk, int32_t numq,
                                                  const gm1b_terrain_scalar_turbulence_arrays *arrays, float dx,
                                                  float dy, float dz, float dt, void *stream) {
    const gm1b_terrain_scalar_turbulence_arrays *s = arrays;
    if (s == nullptr || numq < 0 || numq > 6) {
        gm1b_set_error("gm1b_terrain_scalar_turbulence: need arrays and numq in 0..6");
        return GM1B_ERR_ARGUMENT;
    }
    TRY(check_grid(ni, nj, nk, dx, dy, dz, dt, "gm1b_terrain_scalar_turbulence"));
    if (!all_set({s->th0, s->tha, s->rho, s->rr, s->rf, s->mh, s->mf, s->khh, s->khv, s->gz, s->rgz, s->rgzu, s->rgzv,
                  s->gx, s->gxu, s->gy, s->gyv, s->thten, s->workspace}) ||
        (numq > 0 && !all_set({s->qa, s->qten}))) {
        gm1b_set_error("gm1b_terrain_scalar_turbulence: a required array (or the workspace) is NULL");
        return GM1B_ERR_ARGUMENT;
    }
    const SArgs a{s->th0, s->tha, s->qa, s->rho, s->rr, s->rf, s->mh, s->mf, s->khh, s->khv, s->gz, s->rgz,
                  s->rgzu, s->rgzv, s->gx, s->gxu, s->gy, s->gyv, s->thten, s->qten, s->workspace, ni, nj, nk,
                  numq + 1, dx, dy, dz, dt};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    {
        ProfScope ps("terrain_turbs_flux_kernel", st);
        terrain_turbs_flux_kernel<<<ew_blocks((size_t)nk * nj * (ni + 1) + (size_t)nk * (nj + 1) * ni), kEW, 0, st>>>(a);
        ps.stop();
        if (!launch_ok("terrain_turbs_flux_kernel")) return GM1B_ERR_CUDA;
    }
    const size_t smem = (size_t)2 * nk * kCT * sizeof(float);
    TRY(configure(terrain_turbs_column_kernel, smem, "terrain_turbs_column_kernel"));
    ProfScope ps("terrain_turbs_column_kernel", st);
    terrain_turbs_column_kernel<<<dim3((ni + kCX - 1) / kCX, (nj + kCY - 1) / kCY), dim3(kCX, kCY), smem, st>>>(a);
    ps.stop();
    return launch_ok("terrain_turbs_column_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}
