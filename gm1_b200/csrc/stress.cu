// SGS stress tendencies of the flat (terrain_flag=.false.) stretched column:
// CM1 gettau and the momentum stress divergence turbu/turbv/turbw with their
// implicit vertical solves.
//
// Behaviour followed (reference file:line):
//   the strain carriers rho*Sij of calcdef's mass and face passes
//       gm1_flat_calcdef_mass_v1 / _face_v1
//       src/cm1core/cuda_gm1_flat_stretched_closure.py:76-114 (turb.F:4772-4786,
//       :4880-4895)
//   gettau with the free-slip lower and upper faces (enqueue_flat_gettau)
//       src/cm1core/cuda_gm1_flat_stretched_closure.py:134-161, :551-571
//       (turb.F:4094-4190, :4281-4433, :4536-4545)
//   turbu/turbuz, turbv/turbvz, turbw (enqueue_flat_momentum_stress, the
//   two-part block off)
//       src/cm1core/cuda_gm1_flat_stretched_closure.py:163-292, :574-618
//       (turbtend.F:1095-1361, :1438-1560, :1860-2128, :2194-2310, :2508-2885)
//
// Binary32 one operation at a time in the reference's statement order
// (--fmad=false; the literal zero factors of vibeta = 0 are formed, so signed
// zeros are what the reference's are).  Open sides are index clamps.
//
//   turbs for theta and the moisture rows (the flat fluxes and turbsz, the
//   open-halo pad/pack copies as index clamps; no surface flux)
//       src/cm1core/cuda_gm1_scalar_turbulence.py:453-466 (pad, pack)
//       src/cm1core/cuda_gm1_flat_stretched_closure.py:335-381 (flux, apply)
//       src/cm1core/cuda_cartesian_closure.py:1566-1633 (the per-scalar loop)
//       (turbtend.F:60-434, :442-692; solve1.F:1169-1233)
//   the dissipative heating, idiss = 1
//       src/cm1core/eqtset2_energy_terms.py:176-215, :375-470 (solve1.F:744-848, :917-975)
//   the upper Rayleigh damping held tendencies, irdamp = 1
//       src/cm1core/cuda_rayleigh_held.py:213-254, :419-488 (solve1.F:412-454)
//
// Design: the strain and gettau passes are grid-stride elementwise kernels
// over the union of their index spaces (one launch each).  The three column
// solves run one thread per staggered column, 32 x 4 columns per CTA with
// consecutive threads on consecutive columns of a row (every level's loads
// coalesce); the forward sweep keeps the face pairs of the level above in
// registers for the next level and parks the Thomas coefficients in shared
// memory ([level][thread], conflict-free); the back substitution recomputes
// the horizontal divergence and the cross term at each level and adds the
// tendency there, so no column array beyond the two coefficient rows exists.
#include "gm1b_common.cuh"

namespace gm1b {
namespace {

constexpr int kCX = 32, kCY = 4, kCT = kCX * kCY;  // column tile
constexpr int kEW = 256;                            // elementwise block

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

struct StressArgs {
    const float *u, *v, *w, *rho, *rf, *mh, *mf, *mhp, *kmh, *kmv;
    float *s11, *s22, *s33, *s12, *s13, *s23;
    float *t11, *t22, *t33, *t12, *t13, *t23;
    float *uten, *vten, *wten;
    int ni, nj, nk;
    float rdx, rdy, rdz, dt;
};

__device__ __forceinline__ int clampi(int x, int n) { return x < 0 ? 0 : (x >= n ? n - 1 : x); }
__device__ __forceinline__ int clampr(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }
// (k, j, i) of a layout with rows of nx words and ny rows per level
__device__ __forceinline__ unsigned o3(int k, int j, int i, int ny, int nx) {
    return ((unsigned)k * (unsigned)ny + (unsigned)j) * (unsigned)nx + (unsigned)i;
}
// a (.., nj, ni) carrier at a clamped column
__device__ __forceinline__ float cell(const StressArgs &a, const float *p, int k, int j, int i) {
    return p[o3(k, clampi(j, a.nj), clampi(i, a.ni), a.nj, a.ni)];
}

// ---------------------------------------------------------------- strain
__global__ void __launch_bounds__(kEW) flat_strain_kernel(StressArgs a) {
    const int ni = a.ni, nj = a.nj, nk = a.nk, ux = ni + 1, vy = nj + 1;
    const size_t total = (size_t)(nk + 1) * vy * ux;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int ic = (int)(q % ux), jc = (int)((q / ux) % vy), k = (int)(q / ((size_t)ux * vy));
        if (k < nk) {
            if (ic < ni && jc < nj) {
                const unsigned p = o3(k, jc, ic, nj, ni);
                const float r = a.rho[p];
                a.s11[p] = (r * (a.u[o3(k, jc, ic + 1, nj, ux)] - a.u[o3(k, jc, ic, nj, ux)])) * a.rdx;
                a.s22[p] = (r * (a.v[o3(k, jc + 1, ic, vy, ni)] - a.v[o3(k, jc, ic, vy, ni)])) * a.rdy;
                a.s33[p] = (r * (a.w[o3(k + 1, jc, ic, nj, ni)] - a.w[o3(k, jc, ic, nj, ni)])) * (a.rdz * a.mhp[k + 1]);
            }
            const int ii = clampr(ic, 1, ni - 1), jj = clampr(jc, 1, nj - 1);
            const float x = (a.u[o3(k, jj, ii, nj, ux)] - a.u[o3(k, jj - 1, ii, nj, ux)]) * a.rdy;
            const float y = (a.v[o3(k, jj, ii, vy, ni)] - a.v[o3(k, jj, ii - 1, vy, ni)]) * a.rdx;
            const float rs = (a.rho[o3(k, jj - 1, ii - 1, nj, ni)] + a.rho[o3(k, jj, ii, nj, ni)]) +
                             (a.rho[o3(k, jj, ii - 1, nj, ni)] + a.rho[o3(k, jj - 1, ii, nj, ni)]);
            a.s12[o3(k, jc, ic, vy, ux)] = ((0.5f * (x + y)) * 0.25f) * rs;
        }
        if (k >= 1 && k < nk) {
            const int kf = k;
            if (jc < nj) {
                const int il = clampi(ic - 1, ni), ir = clampi(ic, ni);
                const float dw = (a.w[o3(kf, jc, ir, nj, ni)] - a.w[o3(kf, jc, il, nj, ni)]) * a.rdx;
                const float du = (((a.u[o3(kf, jc, ic, nj, ux)] - a.u[o3(kf - 1, jc, ic, nj, ux)]) * a.rdz) * 0.5f) *
                                 (a.mf[o3(kf, jc, il, nj, ni)] + a.mf[o3(kf, jc, ir, nj, ni)]);
                a.s13[o3(kf, jc, ic, nj, ux)] =
                    ((0.5f * (dw + du)) * 0.5f) * (a.rf[o3(kf, jc, il, nj, ni)] + a.rf[o3(kf, jc, ir, nj, ni)]);
            }
            if (ic < ni) {
                const int js = clampi(jc - 1, nj), jn = clampi(jc, nj);
                const float dw = (a.w[o3(kf, jn, ic, nj, ni)] - a.w[o3(kf, js, ic, nj, ni)]) * a.rdy;
                const float dv = (((a.v[o3(kf, jc, ic, vy, ni)] - a.v[o3(kf - 1, jc, ic, vy, ni)]) * a.rdz) * 0.5f) *
                                 (a.mf[o3(kf, js, ic, nj, ni)] + a.mf[o3(kf, jn, ic, nj, ni)]);
                a.s23[o3(kf, jc, ic, vy, ni)] =
                    ((0.5f * (dw + dv)) * 0.5f) * (a.rf[o3(kf, js, ic, nj, ni)] + a.rf[o3(kf, jn, ic, nj, ni)]);
            }
        }
    }
}

// ---------------------------------------------------------------- gettau
__global__ void __launch_bounds__(kEW) flat_gettau_kernel(StressArgs a) {
    const int ni = a.ni, nj = a.nj, nk = a.nk, ux = ni + 1, vy = nj + 1;
    const size_t total = (size_t)(nk + 1) * vy * ux;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int ic = (int)(q % ux), jc = (int)((q / ux) % vy), k = (int)(q / ((size_t)ux * vy));
        if (k < nk) {
            if (ic < ni && jc < nj) {
                const unsigned p = o3(k, jc, ic, nj, ni), pu = o3(k + 1, jc, ic, nj, ni);
                const float m = a.kmh[p] + a.kmh[pu];
                a.t11[p] = a.s11[p] * m;
                a.t22[p] = a.s22[p] * m;
                a.t33[p] = a.s33[p] * m;
            }
            const int ii = clampr(ic, 1, ni - 1), jj = clampr(jc, 1, nj - 1);
            const float lo = (a.kmh[o3(k, jj - 1, ii - 1, nj, ni)] + a.kmh[o3(k, jj, ii, nj, ni)]) +
                             (a.kmh[o3(k, jj, ii - 1, nj, ni)] + a.kmh[o3(k, jj - 1, ii, nj, ni)]);
            const float hi = (a.kmh[o3(k + 1, jj - 1, ii - 1, nj, ni)] + a.kmh[o3(k + 1, jj, ii, nj, ni)]) +
                             (a.kmh[o3(k + 1, jj, ii - 1, nj, ni)] + a.kmh[o3(k + 1, jj - 1, ii, nj, ni)]);
            a.t12[o3(k, jc, ic, vy, ux)] = (a.s12[o3(k, jj, ii, vy, ux)] * 0.25f) * (lo + hi);
        }
        const int f = k, ff = f == 0 ? 1 : (f == nk ? nk - 1 : f);
        if (jc < nj)
            a.t13[o3(f, jc, ic, nj, ux)] =
                a.s13[o3(ff, jc, ic, nj, ux)] * (cell(a, a.kmv, ff, jc, ic - 1) + cell(a, a.kmv, ff, jc, ic));
        if (ic < ni)
            a.t23[o3(f, jc, ic, vy, ni)] =
                a.s23[o3(ff, jc, ic, vy, ni)] * (cell(a, a.kmv, ff, jc - 1, ic) + cell(a, a.kmv, ff, jc, ic));
    }
}

// ------------------------------------------------------- turbu and turbv
// DIR 0: a u column (j, f), f in [0, ni]; DIR 1: a v column (f, i), f in [0, nj];
// the cells either side of it are (ja, ia) and (jb, ib).
template <int DIR>
__global__ void __launch_bounds__(kCT) flat_turb_uv_kernel(StressArgs a) {
    extern __shared__ float s_col[];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kCX + tx;
    const int ni = a.ni, nj = a.nj, K = a.nk, ux = ni + 1, vy = nj + 1;
    const int cx = blockIdx.x * kCX + tx, cy = blockIdx.y * kCY + ty;
    // DIR 0: column (j = cy, f = cx); DIR 1: column (f = cy, i = cx)
    if (DIR == 0 ? (cx > ni || cy >= nj) : (cx >= ni || cy > nj)) return;
    const int ja = DIR == 0 ? cy : cy - 1, jb = cy, ia = DIR == 0 ? cx - 1 : cx, ib = cx;
    const float *q = DIR == 0 ? a.u : a.v;       // the column's wind
    const float *top = DIR == 0 ? a.t13 : a.t23;  // its t13/t23 (face levels)
    float *ten = DIR == 0 ? a.uten : a.vten;
    const unsigned col = DIR == 0 ? (unsigned)cy * ux + cx : (unsigned)cy * ni + cx;
    const unsigned lev = DIR == 0 ? (unsigned)nj * ux : (unsigned)vy * ni;
    const float rd = DIR == 0 ? a.rdx : a.rdy, rdz = a.rdz, dt = a.dt;
    float *cp = s_col, *dp = s_col + (size_t)K * kCT;
#define CP(k) cp[(unsigned)(k) * kCT + tid]
#define DP(k) dp[(unsigned)(k) * kCT + tid]
#define PAIR(p, k) (cell(a, p, k, ja, ia) + cell(a, p, k, jb, ib))
#define QK(k) q[(unsigned)(k) * lev + col]
#define D7(k) (((((cell(a, a.w, k, jb, ib) - cell(a, a.w, k, ja, ia)) * rd) * 0.25f) * PAIR(a.kmv, k)) * PAIR(a.rf, k))
    const float rdt = 0.5f / dt;
    const float tema = (((-0.0625f * dt) * 1.0f) * rdz) * rdz;
    const float temb = (((0.0625f * dt) * 0.0f) * rdz) * rdz;
    const float temc = (0.5f * dt) * rdz;
    // k = 0
    float rr0 = 1.0f / (0.5f * PAIR(a.rho, 0));
    float mhp = PAIR(a.mh, 0);
    float tem = mhp * rr0;
    float kmv_u = PAIR(a.kmv, 1), mf_u = PAIR(a.mf, 1), rf_u = PAIR(a.rf, 1);  // face above
    float r2 = ((kmv_u * mf_u) * rf_u) * tem;
    float cfc = tema * r2, cfb = 1.0f - cfc;
    float qm = QK(0), qk = QK(1);  // q(k-1), q(k) of the next level
    float cfd = (qm + temb * (r2 * qk - r2 * qm)) - ((temc * top[col]) * mhp) * rr0;
    float inv = 1.0f / cfb;
    float cprev = -(cfc * inv), dprev = cfd * inv;
    CP(0) = cprev;
    DP(0) = dprev;
    #pragma unroll 4
    for (int k = 1; k < K - 1; ++k) {
        rr0 = 1.0f / (0.5f * PAIR(a.rho, k));
        tem = PAIR(a.mh, k) * rr0;
        const float r1 = ((kmv_u * mf_u) * rf_u) * tem;
        kmv_u = PAIR(a.kmv, k + 1);
        mf_u = PAIR(a.mf, k + 1);
        rf_u = PAIR(a.rf, k + 1);
        r2 = ((kmv_u * mf_u) * rf_u) * tem;
        const float cfa = tema * r1;
        cfc = tema * r2;
        cfb = (1.0f - cfa) - cfc;
        const float qp = QK(k + 1);
        cfd = qk + temb * ((r2 * qp - (r1 + r2) * qk) + r1 * qm);
        inv = 1.0f / (cfa * cprev + cfb);
        cprev = -(cfc * inv);
        dprev = (cfd - cfa * dprev) * inv;
        CP(k) = cprev;
        DP(k) = dprev;
        qm = qk;
        qk = qp;
    }
    float sol;
    {
        const int k = K - 1;
        rr0 = 1.0f / (0.5f * PAIR(a.rho, k));
        mhp = PAIR(a.mh, k);
        tem = mhp * rr0;
        const float r1 = ((kmv_u * mf_u) * rf_u) * tem;
        const float cfa = tema * r1;
        cfb = 1.0f - cfa;
        cfd = (qk + temb * (-(r1 * qk) + r1 * qm)) + ((temc * top[(unsigned)K * lev + col]) * mhp) * rr0;
        inv = 1.0f / (cfa * cprev + cfb);
        sol = (cfd - cfa * dprev) * inv;
    }
    // back substitution, the vertical term and the tendency per level
    float d7_up = 0.0f;
    #pragma unroll 4
    for (int k = K - 1; k >= 0; --k) {
        if (k < K - 1) sol = CP(k) * sol + DP(k);
        const float rho_p = PAIR(a.rho, k);
        float tz = (rho_p * (sol - QK(k))) * rdt;
        const float d7 = k == 0 ? 0.0f : D7(k);
        tz = tz + (((d7_up - d7) * rdz) * 0.5f) * PAIR(a.mh, k);
        d7_up = d7;
        float hx, hy;
        if (DIR == 0) {
            hx = (cell(a, a.t11, k, cy, ib) - cell(a, a.t11, k, cy, ia)) * a.rdx;
            hy = (a.t12[o3(k, cy + 1, cx, vy, ux)] - a.t12[o3(k, cy, cx, vy, ux)]) * a.rdy;
            if (cx == 0 || cx == ni) hx = 0.0f;
            if (cy == 0 || cy == nj - 1) hy = 0.0f;
        } else {
            hx = (a.t12[o3(k, cy, cx + 1, vy, ux)] - a.t12[o3(k, cy, cx, vy, ux)]) * a.rdx;
            hy = (cell(a, a.t22, k, jb, cx) - cell(a, a.t22, k, ja, cx)) * a.rdy;
            if (cx == 0 || cx == ni - 1) hx = 0.0f;
            if (cy == 0 || cy == nj) hy = 0.0f;
        }
        const float rrk = 1.0f / (0.5f * rho_p);
        const unsigned p = (unsigned)k * lev + col;
        ten[p] = ten[p] + ((hx + hy) + tz) * rrk;
    }
#undef CP
#undef DP
#undef PAIR
#undef QK
#undef D7
}

// ----------------------------------------------------------------- turbw
__global__ void __launch_bounds__(kCT) flat_turbw_kernel(StressArgs a) {
    extern __shared__ float s_col[];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kCX + tx;
    const int ni = a.ni, nj = a.nj, K = a.nk, ux = ni + 1, vy = nj + 1;
    const int i = blockIdx.x * kCX + tx, j = blockIdx.y * kCY + ty;
    if (i >= ni || j >= nj) return;
    const unsigned col = (unsigned)j * ni + i, lev = (unsigned)nj * ni;
    const float rdz = a.rdz, dt = a.dt;
    float *cp = s_col, *dp = s_col + (size_t)K * kCT;
#define CP(p) cp[(unsigned)(p) * kCT + tid]
#define DP(p) dp[(unsigned)(p) * kCT + tid]
#define PF(p, f) p[(unsigned)(f) * lev + col]
    const float rdt = 1.0f / dt;
    const float tema = (((-1.0f * dt) * 1.0f) * rdz) * rdz;
    const float temb = ((dt * 0.0f) * rdz) * rdz;
    const float temc = dt * rdz;
    // face 1
    float rrf = PF(a.mf, 1) / PF(a.rf, 1);
    float kmh_m = PF(a.kmh, 1), kmh_u = PF(a.kmh, 2);
    float r2 = (((kmh_m + kmh_u) * PF(a.mh, 1)) * PF(a.rho, 1)) * rrf;
    float cfc = tema * r2, cfb = 1.0f - cfc;
    float wm = PF(a.w, 1), wk = PF(a.w, 2);  // w(f-1), w(f) of the next face
    float cfd = (wm + temb * (r2 * wk - r2 * wm)) - (temc * PF(a.t33, 0)) * rrf;
    float inv = 1.0f / cfb;
    float cprev = -(cfc * inv), dprev = cfd * inv;
    CP(0) = cprev;
    DP(0) = dprev;
    #pragma unroll 4
    for (int f = 2; f < K - 1; ++f) {
        rrf = PF(a.mf, f) / PF(a.rf, f);
        const float r1 = (((kmh_m + kmh_u) * PF(a.mh, f - 1)) * PF(a.rho, f - 1)) * rrf;
        kmh_m = kmh_u;
        kmh_u = PF(a.kmh, f + 1);
        r2 = (((kmh_m + kmh_u) * PF(a.mh, f)) * PF(a.rho, f)) * rrf;
        const float cfa = tema * r1;
        cfc = tema * r2;
        cfb = (1.0f - cfa) - cfc;
        const float wp = PF(a.w, f + 1);
        cfd = wk + temb * ((r2 * wp - (r1 + r2) * wk) + r1 * wm);
        inv = 1.0f / (cfa * cprev + cfb);
        cprev = -(cfc * inv);
        dprev = (cfd - cfa * dprev) * inv;
        CP(f - 1) = cprev;
        DP(f - 1) = dprev;
        wm = wk;
        wk = wp;
    }
    float sol;
    {
        const int f = K - 1;
        rrf = PF(a.mf, f) / PF(a.rf, f);
        const float r1 = (((kmh_m + kmh_u) * PF(a.mh, f - 1)) * PF(a.rho, f - 1)) * rrf;
        const float cfa = tema * r1;
        cfb = 1.0f - cfa;
        cfd = (wk + temb * (-(r1 * wk) + r1 * wm)) + (temc * PF(a.t33, f)) * rrf;
        inv = 1.0f / (cfa * cprev + cfb);
        sol = (cfd - cfa * dprev) * inv;
    }
    #pragma unroll 4
    for (int f = K - 1; f >= 1; --f) {
        if (f < K - 1) sol = CP(f - 1) * sol + DP(f - 1);
        const float rff = PF(a.rf, f);
        const float tz = (rff * (sol - PF(a.w, f))) * rdt;
        float hx = (a.t13[o3(f, j, i + 1, nj, ux)] - a.t13[o3(f, j, i, nj, ux)]) * a.rdx;
        float hy = (a.t23[o3(f, j + 1, i, vy, ni)] - a.t23[o3(f, j, i, vy, ni)]) * a.rdy;
        if (i == 0 || i == ni - 1) hx = 0.0f;
        if (j == 0 || j == nj - 1) hy = 0.0f;
        const unsigned p = (unsigned)f * lev + col;
        a.wten[p] = a.wten[p] + ((hx + hy) + tz) / rff;
    }
#undef CP
#undef DP
#undef PF
}


// ---------------------------------------------------------- turbs (flat)
// theta ((th0 - 300) + tha) and numq moisture rows.  The open-halo copies of
// the reference's pad/pack texts are index clamps here, so no halo array is
// written.  Two passes: the horizontal pass forms, per cell, the x and y
// flux divergence tx + ty of every scalar into the workspace (each face's
// factor (-0.125*(rho_l + rho_r))*(the four khh) formed once and shared by
// all scalars); the column pass solves turbsz's tridiagonal for each scalar
// and adds ((tx + ty) + tz)*rr, the reference's sum in its order.
struct TurbsArgs {
    const float *th0, *tha, *qa, *rho, *rr, *rf, *mh, *mf, *khh, *khv;
    float *thten, *qten, *work;
    int ni, nj, nk, nsc;
    float dx, dy, dz, dt;
};

__device__ __forceinline__ float tcell(const TurbsArgs &a, const float *p, int k, int j, int i) {
    return p[o3(k, clampi(j, a.nj), clampi(i, a.ni), a.nj, a.ni)];
}
// the open-halo scalar sc (0 theta, 1.. the moisture rows) at a clamped cell
__device__ __forceinline__ float sval(const TurbsArgs &a, int sc, int k, int j, int i) {
    const unsigned p = o3(k, clampi(j, a.nj), clampi(i, a.ni), a.nj, a.ni);
    if (sc > 0) return a.qa[(size_t)(sc - 1) * ((size_t)a.ni * a.nj * a.nk) + p];
    return (a.th0[k] - 300.0f) + a.tha[p];
}
// the face factor (-0.125*(rho(a)+rho(a-1)))*((khh(k)+khh(k)) + (khh(k+1)+khh(k+1)))
// across x face f (cells f-1, f) or y face f (rows f-1, f)
__device__ __forceinline__ float fac_x(const TurbsArgs &a, int k, int j, int f) {
    const float den = tcell(a, a.rho, k, j, f) + tcell(a, a.rho, k, j, f - 1);
    const float kh = (tcell(a, a.khh, k, j, f) + tcell(a, a.khh, k, j, f - 1)) +
                     (tcell(a, a.khh, k + 1, j, f) + tcell(a, a.khh, k + 1, j, f - 1));
    return (-0.125f * den) * kh;
}
__device__ __forceinline__ float fac_y(const TurbsArgs &a, int k, int f, int i) {
    const float den = tcell(a, a.rho, k, f, i) + tcell(a, a.rho, k, f - 1, i);
    const float kh = (tcell(a, a.khh, k, f, i) + tcell(a, a.khh, k, f - 1, i)) +
                     (tcell(a, a.khh, k + 1, f, i) + tcell(a, a.khh, k + 1, f - 1, i));
    return (-0.125f * den) * kh;
}

__global__ void __launch_bounds__(kCT) flat_turbs_horizontal_kernel(TurbsArgs a) {
    const int i = blockIdx.x * kCX + threadIdx.x, j = blockIdx.y * kCY + threadIdx.y, k = blockIdx.z;
    const int ni = a.ni, nj = a.nj;
    if (i >= ni || j >= nj) return;
    const size_t n = (size_t)ni * nj * a.nk, p = o3(k, j, i, nj, ni);
    const float rx = 1.0f / a.dx, ry = 1.0f / a.dy;
    const bool xin = !(i == 0 || i + 1 == ni), yin = !(j == 0 || j + 1 == nj);
    float fw = 0.0f, fe = 0.0f, fs = 0.0f, fn = 0.0f;
    if (xin) {
        fw = fac_x(a, k, j, i);
        fe = fac_x(a, k, j, i + 1);
    }
    if (yin) {
        fs = fac_y(a, k, j, i);
        fn = fac_y(a, k, j + 1, i);
    }
    for (int sc = 0; sc < a.nsc; ++sc) {
        float tx = 0.0f, ty = 0.0f;
        const float s0 = sval(a, sc, k, j, i);
        if (xin) {
            const float xw = (fw * (s0 - sval(a, sc, k, j, i - 1))) * rx;
            const float xe = (fe * (sval(a, sc, k, j, i + 1) - s0)) * rx;
            tx = -((xe - xw) * rx);
        }
        if (yin) {
            const float ys = (fs * (s0 - sval(a, sc, k, j - 1, i))) * ry;
            const float yn = (fn * (sval(a, sc, k, j + 1, i) - s0)) * ry;
            ty = -((yn - ys) * ry);
        }
        a.work[(size_t)sc * n + p] = tx + ty;
    }
}

__global__ void __launch_bounds__(kCT) flat_turbs_column_kernel(TurbsArgs a) {
    extern __shared__ float s_col[];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kCX + tx;
    const int ni = a.ni, nj = a.nj, nk = a.nk;
    const int i = blockIdx.x * kCX + tx, j = blockIdx.y * kCY + ty;
    if (i >= ni || j >= nj) return;
    const size_t n = (size_t)ni * nj * nk;
    const unsigned col = (unsigned)j * ni + i, lev = (unsigned)nj * ni;
    float *cp = s_col, *dp = s_col + (size_t)nk * kCT;
#define CP(k) cp[(unsigned)(k) * kCT + tid]
#define DP(k) dp[(unsigned)(k) * kCT + tid]
#define PF(p, k) p[(unsigned)(k) * lev + col]
#define COEF(F, K) ((((PF(a.khv, F) * PF(a.mf, F)) * PF(a.rf, F)) * PF(a.mh, K)) * PF(a.rr, K))
    const float rz = 1.0f / a.dz, dt = a.dt, rdt = 1.0f / dt;
    const float tema = (((-1.0f * dt) * 1.0f) * rz) * rz;
    const float temb = ((dt * 0.0f) * rz) * rz;
    const float temc = dt * rz;
    for (int sc = 0; sc < a.nsc; ++sc) {
        float *target = sc == 0 ? a.thten : a.qten + (size_t)(sc - 1) * n;
        const float *h = a.work + (size_t)sc * n;
#define SC(k) sval(a, sc, k, j, i)
        float sm = SC(0), sk = SC(1);  // scalar at k-1 and k of the next level
        float r2 = COEF(1, 0);
        float cfc = tema * r2, cfb = 1.0f - cfc;
        float ex = (-r2) * sm + r2 * sk;
        float bc = ((temc * 0.0f) * PF(a.mh, 0)) * PF(a.rr, 0);
        float cfd = (sm + temb * ex) + bc;
        float tem = 1.0f / cfb;
        float cprev = (-cfc) * tem, dprev = cfd * tem;
        CP(0) = cprev;
        DP(0) = dprev;
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
        for (int k = nk - 1; k >= 0; --k) {
            if (k != nk - 1) sol = CP(k) * sol + DP(k);
            const float tz = (PF(a.rho, k) * (sol - SC(k))) * rdt;
            const unsigned p = (unsigned)k * lev + col;
            target[p] = target[p] + (h[p] + tz) * PF(a.rr, k);
        }
#undef SC
    }
#undef CP
#undef DP
#undef PF
#undef COEF
}

// ------------------------------------------------------ Rayleigh (upper)
// irdamp = 1: uten1 = ((-rdalpha*0.5)*(tauh(i-1)+tauh(i)))*(ua - u0(k)), vten1
// across j, wten1 = (-rdalpha*tauf)*wa, thten1 = (-rdalpha*taus)*tha.  tau
// as one-halo 3-D arrays (the reference's layout) or as column profiles;
// add_momentum adds the damping into the momentum outputs (the closure's
// held sum uten1 + uten) and assigns thten1.
struct RayArgs {
    const float *tauh, *taus, *tauf, *u0, *v0, *ua, *va, *wa, *tha;
    float *uten1, *vten1, *wten1, *thten1;
    int ni, nj, nk;
    float rdalpha;
    int profiles, add_momentum;
};

__device__ __forceinline__ float tau_at(const RayArgs &a, const float *tau, int k, int jh, int ih) {
    return a.profiles ? tau[k] : tau[((size_t)k * (a.nj + 2) + jh) * (size_t)(a.ni + 2) + ih];
}

__global__ void __launch_bounds__(kEW) rayleigh_held_kernel(RayArgs a) {
    const int ni = a.ni, nj = a.nj, nk = a.nk;
    const size_t first = (size_t)blockIdx.x * blockDim.x + threadIdx.x, step = (size_t)gridDim.x * blockDim.x;
    const size_t nu = (size_t)nk * nj * (ni + 1), nv = (size_t)nk * (nj + 1) * ni, ns = (size_t)nk * nj * ni;
    const float neg = -a.rdalpha, negh = neg * 0.5f;
    for (size_t z = first; z < nu; z += step) {
        const int f = (int)(z % (ni + 1)), j = (int)((z / (ni + 1)) % nj), k = (int)(z / ((size_t)(ni + 1) * nj));
        const float pair = tau_at(a, a.tauh, k, j + 1, f) + tau_at(a, a.tauh, k, j + 1, f + 1);
        const float d = (negh * pair) * (a.ua[z] - a.u0[k]);
        a.uten1[z] = a.add_momentum ? d + a.uten1[z] : d;
    }
    for (size_t z = first; z < nv; z += step) {
        const int i = (int)(z % ni), f = (int)((z / ni) % (nj + 1)), k = (int)(z / ((size_t)ni * (nj + 1)));
        const float pair = tau_at(a, a.tauh, k, f, i + 1) + tau_at(a, a.tauh, k, f + 1, i + 1);
        const float d = (negh * pair) * (a.va[z] - a.v0[k]);
        a.vten1[z] = a.add_momentum ? d + a.vten1[z] : d;
    }
    for (size_t z = first; z < ns; z += step) {
        const int i = (int)(z % ni), j = (int)((z / ni) % nj), k = (int)(z / ((size_t)ni * nj));
        const float dw = (neg * tau_at(a, a.tauf, k, j + 1, i + 1)) * a.wa[z];
        a.wten1[z] = a.add_momentum ? dw + a.wten1[z] : dw;
        a.thten1[z] = (neg * tau_at(a, a.taus, k, j + 1, i + 1)) * a.tha[z];
    }
}


// ---------------------------------------------------- dissipative heating
// idiss = 1: thten1 += (0.5*(dissten(k)+dissten(k+1))) /
// ((cpdcv*cvm)*(pi0+ppi)), cvm = ((cv + cvv*qv) + cpl*ql) + cpi*qice.
struct DissArgs {
    const float *dissten, *pi0, *ppi, *qa;
    float *thten1;
    int ni, nj, nk;
};

__global__ void __launch_bounds__(kEW) dissipative_heating_kernel(DissArgs a) {
    const float rd = 287.04f, cp = 1005.7f, cpv = 1870.0f, rv = 461.5f, cpl = 4190.0f, cpi = 2106.0f;
    const float cv = cp - rd, cvv = cpv - rv, cpdcv = cp / cv;
    const size_t plane = (size_t)a.ni * a.nj, n = plane * a.nk;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(q / plane);
        const float ql = a.qa[n + q] + a.qa[2 * n + q];
        const float qice = (a.qa[3 * n + q] + a.qa[4 * n + q]) + a.qa[5 * n + q];
        float cvm = cv + cvv * a.qa[q];
        cvm = cvm + cpl * ql;
        cvm = cvm + cpi * qice;
        const float epsd = 0.5f * (a.dissten[q] + a.dissten[q + plane]);
        const float den = (cpdcv * cvm) * (a.pi0[k] + a.ppi[q]);
        a.thten1[q] = a.thten1[q] + epsd / den;
    }
}

// ------------------------------------------------------------------ host
int stress_args(int32_t ni, int32_t nj, int32_t nk, const gm1b_flat_stress_arrays *s, float dx, float dy, float rdz,
                float dt, bool need_dt, StressArgs &a, const char *what) {
    if (s == nullptr || ni < 3 || nj < 3 || nk < 3) {
        gm1b_set_error("%s: need arrays, ni >= 3, nj >= 3, nk >= 3", what);
        return GM1B_ERR_ARGUMENT;
    }
    if ((double)(nk + 1) * (nj + 1) * (ni + 1) >= 2147483648.0) {
        gm1b_set_error("%s: a %dx%dx%d grid reaches 2^31 words; the kernels index with 32-bit offsets", what, ni, nj,
                       nk);
        return GM1B_ERR_ARGUMENT;
    }
    if (!(dx > 0.0f && dy > 0.0f && rdz > 0.0f) || !isfinite(dx) || !isfinite(dy) || !isfinite(rdz) ||
        (need_dt && !(dt > 0.0f && isfinite(dt)))) {
        gm1b_set_error("%s: dx, dy, rdz%s must be finite and > 0", what, need_dt ? ", dt" : "");
        return GM1B_ERR_ARGUMENT;
    }
    a = StressArgs{};
    a.u = s->u3d;
    a.v = s->v3d;
    a.w = s->w3d;
    a.rho = s->rho;
    a.rf = s->rf;
    a.mh = s->mh;
    a.mf = s->mf;
    a.mhp = s->mh_profile;
    a.kmh = s->kmh;
    a.kmv = s->kmv;
    a.s11 = s->s11;
    a.s22 = s->s22;
    a.s33 = s->s33;
    a.s12 = s->s12;
    a.s13 = s->s13;
    a.s23 = s->s23;
    a.t11 = s->t11;
    a.t22 = s->t22;
    a.t33 = s->t33;
    a.t12 = s->t12;
    a.t13 = s->t13;
    a.t23 = s->t23;
    a.uten = s->uten;
    a.vten = s->vten;
    a.wten = s->wten;
    a.ni = ni;
    a.nj = nj;
    a.nk = nk;
    a.rdx = 1.0f / dx;
    a.rdy = 1.0f / dy;
    a.rdz = rdz;
    a.dt = dt;
    return GM1B_OK;
}

bool all_set(std::initializer_list<const void *> ps) {
    for (const void *p : ps)
        if (p == nullptr) return false;
    return true;
}

unsigned ew_blocks(int ni, int nj, int nk) {
    const size_t total = (size_t)(nk + 1) * (nj + 1) * (ni + 1);
    const size_t want = (total + kEW - 1) / kEW, cap = (size_t)148 * 16;
    return (unsigned)(want < cap ? want : cap);
}

int enqueue_strain(const StressArgs &a, cudaStream_t st) {
    ProfScope ps("flat_strain_kernel", st);
    flat_strain_kernel<<<ew_blocks(a.ni, a.nj, a.nk), kEW, 0, st>>>(a);
    ps.stop();
    return launch_ok("flat_strain_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

int enqueue_gettau(const StressArgs &a, cudaStream_t st) {
    ProfScope ps("flat_gettau_kernel", st);
    flat_gettau_kernel<<<ew_blocks(a.ni, a.nj, a.nk), kEW, 0, st>>>(a);
    ps.stop();
    return launch_ok("flat_gettau_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
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

int enqueue_momentum(const StressArgs &a, cudaStream_t st) {
    const size_t smem = (size_t)2 * a.nk * kCT * sizeof(float);
    if (smem > 200 * 1024) {
        gm1b_set_error("gm1b_flat_momentum_stress: nk=%d exceeds the column solves' shared memory (nk <= 200)", a.nk);
        return GM1B_ERR_ARGUMENT;
    }
    TRY(configure(flat_turb_uv_kernel<0>, smem, "flat_turb_uv_kernel<0>"));
    TRY(configure(flat_turb_uv_kernel<1>, smem, "flat_turb_uv_kernel<1>"));
    TRY(configure(flat_turbw_kernel, smem, "flat_turbw_kernel"));
    {
        ProfScope ps("flat_turbu_kernel", st);
        flat_turb_uv_kernel<0><<<dim3((a.ni + 1 + kCX - 1) / kCX, (a.nj + kCY - 1) / kCY), dim3(kCX, kCY), smem, st>>>(a);
        ps.stop();
        if (!launch_ok("flat_turbu_kernel")) return GM1B_ERR_CUDA;
    }
    {
        ProfScope ps("flat_turbv_kernel", st);
        flat_turb_uv_kernel<1><<<dim3((a.ni + kCX - 1) / kCX, (a.nj + 1 + kCY - 1) / kCY), dim3(kCX, kCY), smem, st>>>(a);
        ps.stop();
        if (!launch_ok("flat_turbv_kernel")) return GM1B_ERR_CUDA;
    }
    ProfScope ps("flat_turbw_kernel", st);
    flat_turbw_kernel<<<dim3((a.ni + kCX - 1) / kCX, (a.nj + kCY - 1) / kCY), dim3(kCX, kCY), smem, st>>>(a);
    ps.stop();
    return launch_ok("flat_turbw_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

}  // namespace
}  // namespace gm1b

using namespace gm1b;

extern "C" int32_t gm1b_flat_strain(int32_t ni, int32_t nj, int32_t nk, const gm1b_flat_stress_arrays *arrays,
                                    float dx, float dy, float rdz, void *stream) {
    StressArgs a;
    TRY(stress_args(ni, nj, nk, arrays, dx, dy, rdz, 1.0f, false, a, "gm1b_flat_strain"));
    if (!all_set({a.u, a.v, a.w, a.rho, a.rf, a.mf, a.mhp, a.s11, a.s22, a.s33, a.s12, a.s13, a.s23})) {
        gm1b_set_error("gm1b_flat_strain: a required array is NULL");
        return GM1B_ERR_ARGUMENT;
    }
    return enqueue_strain(a, static_cast<cudaStream_t>(stream));
}

extern "C" int32_t gm1b_flat_gettau(int32_t ni, int32_t nj, int32_t nk, const gm1b_flat_stress_arrays *arrays,
                                    void *stream) {
    StressArgs a;
    TRY(stress_args(ni, nj, nk, arrays, 1.0f, 1.0f, 1.0f, 1.0f, false, a, "gm1b_flat_gettau"));
    if (!all_set({a.s11, a.s22, a.s33, a.s12, a.s13, a.s23, a.kmh, a.kmv, a.t11, a.t22, a.t33, a.t12, a.t13, a.t23})) {
        gm1b_set_error("gm1b_flat_gettau: a required array is NULL");
        return GM1B_ERR_ARGUMENT;
    }
    return enqueue_gettau(a, static_cast<cudaStream_t>(stream));
}

extern "C" int32_t gm1b_flat_momentum_stress(int32_t ni, int32_t nj, int32_t nk,
                                             const gm1b_flat_stress_arrays *arrays, float dx, float dy, float rdz,
                                             float dt, void *stream) {
    StressArgs a;
    TRY(stress_args(ni, nj, nk, arrays, dx, dy, rdz, dt, true, a, "gm1b_flat_momentum_stress"));
    if (!all_set({a.t11, a.t22, a.t33, a.t12, a.t13, a.t23, a.kmh, a.kmv, a.rho, a.rf, a.mh, a.mf, a.u, a.v, a.w,
                  a.uten, a.vten, a.wten})) {
        gm1b_set_error("gm1b_flat_momentum_stress: a required array is NULL");
        return GM1B_ERR_ARGUMENT;
    }
    return enqueue_momentum(a, static_cast<cudaStream_t>(stream));
}

extern "C" int32_t gm1b_flat_sgs_stress(int32_t ni, int32_t nj, int32_t nk, const gm1b_flat_stress_arrays *arrays,
                                        float dx, float dy, float rdz, float dt, void *stream) {
    TRY(gm1b_flat_strain(ni, nj, nk, arrays, dx, dy, rdz, stream));
    TRY(gm1b_flat_gettau(ni, nj, nk, arrays, stream));
    return gm1b_flat_momentum_stress(ni, nj, nk, arrays, dx, dy, rdz, dt, stream);
}

extern "C" int64_t gm1b_flat_scalar_turbulence_workspace_words(int32_t ni, int32_t nj, int32_t nk, int32_t numq) {
    if (ni < 1 || nj < 1 || nk < 1 || numq < 0) return 0;
    return (int64_t)(numq + 1) * ni * nj * nk;
}

extern "C" int32_t gm1b_flat_scalar_turbulence(int32_t ni, int32_t nj, int32_t nk, int32_t numq,
                                               const gm1b_flat_scalar_turbulence_arrays *arrays, float dx, float dy,
                                               float dz, float dt, void *stream) {
    const gm1b_flat_scalar_turbulence_arrays *s = arrays;
    if (s == nullptr || ni < 3 || nj < 3 || nk < 3 || numq < 0 || numq > 6) {
        gm1b_set_error("gm1b_flat_scalar_turbulence: need arrays, ni >= 3, nj >= 3, nk >= 3, numq in 0..6");
        return GM1B_ERR_ARGUMENT;
    }
    if ((double)(nk + 1) * nj * ni >= 2147483648.0) {
        gm1b_set_error("gm1b_flat_scalar_turbulence: a %dx%dx%d grid is too large for 32-bit offsets", ni, nj, nk);
        return GM1B_ERR_ARGUMENT;
    }
    if (!(dx > 0.0f && dy > 0.0f && dz > 0.0f && dt > 0.0f) || !isfinite(dx) || !isfinite(dy) || !isfinite(dz) ||
        !isfinite(dt)) {
        gm1b_set_error("gm1b_flat_scalar_turbulence: dx, dy, dz, dt must be finite and > 0");
        return GM1B_ERR_ARGUMENT;
    }
    if (!all_set({s->th0, s->tha, s->rho, s->rr, s->rf, s->mh, s->mf, s->khh, s->khv, s->thten, s->workspace}) ||
        (numq > 0 && !all_set({s->qa, s->qten}))) {
        gm1b_set_error("gm1b_flat_scalar_turbulence: a required array (or the workspace) is NULL");
        return GM1B_ERR_ARGUMENT;
    }
    const size_t smem = (size_t)2 * nk * kCT * sizeof(float);
    if (smem > 200 * 1024) {
        gm1b_set_error("gm1b_flat_scalar_turbulence: nk=%d exceeds the column solve's shared memory (nk <= 200)", nk);
        return GM1B_ERR_ARGUMENT;
    }
    TRY(configure(flat_turbs_column_kernel, smem, "flat_turbs_column_kernel"));
    TurbsArgs a{s->th0, s->tha, s->qa, s->rho, s->rr, s->rf, s->mh, s->mf, s->khh, s->khv, s->thten, s->qten,
                s->workspace, ni, nj, nk, numq + 1, dx, dy, dz, dt};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const dim3 tile(kCX, kCY), cols((ni + kCX - 1) / kCX, (nj + kCY - 1) / kCY);
    {
        ProfScope ps("flat_turbs_horizontal_kernel", st);
        flat_turbs_horizontal_kernel<<<dim3(cols.x, cols.y, nk), tile, 0, st>>>(a);
        ps.stop();
        if (!launch_ok("flat_turbs_horizontal_kernel")) return GM1B_ERR_CUDA;
    }
    ProfScope ps("flat_turbs_column_kernel", st);
    flat_turbs_column_kernel<<<cols, tile, smem, st>>>(a);
    ps.stop();
    return launch_ok("flat_turbs_column_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_rayleigh_held(int32_t ni, int32_t nj, int32_t nk, const gm1b_rayleigh_held_arrays *arrays,
                                      int32_t profiles, int32_t add_momentum, float rdalpha, void *stream) {
    const gm1b_rayleigh_held_arrays *s = arrays;
    if (s == nullptr || ni < 1 || nj < 1 || nk < 1 || (profiles != 0 && profiles != 1) ||
        (add_momentum != 0 && add_momentum != 1)) {
        gm1b_set_error("gm1b_rayleigh_held: need arrays, ni, nj, nk >= 1, profiles and add_momentum 0 or 1");
        return GM1B_ERR_ARGUMENT;
    }
    if (!(rdalpha >= 0.0f) || !isfinite(rdalpha)) {
        gm1b_set_error("gm1b_rayleigh_held: rdalpha must be finite and >= 0");
        return GM1B_ERR_ARGUMENT;
    }
    if (!all_set({s->tauh, s->taus, s->tauf, s->u0, s->v0, s->ua, s->va, s->wa, s->tha, s->uten1, s->vten1, s->wten1,
                  s->thten1})) {
        gm1b_set_error("gm1b_rayleigh_held: a required array is NULL");
        return GM1B_ERR_ARGUMENT;
    }
    RayArgs a{s->tauh, s->taus, s->tauf, s->u0,    s->v0,    s->ua,    s->va,    s->wa, s->tha,
              s->uten1, s->vten1, s->wten1, s->thten1, ni, nj, nk, rdalpha, profiles, add_momentum};
    const size_t most = (size_t)nk * (nj + 1) * (ni + 1);
    const size_t want = (most + kEW - 1) / kEW, cap = (size_t)148 * 16;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("rayleigh_held_kernel", st);
    rayleigh_held_kernel<<<(unsigned)(want < cap ? want : cap), kEW, 0, st>>>(a);
    ps.stop();
    return launch_ok("rayleigh_held_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_dissipative_heating(int32_t ni, int32_t nj, int32_t nk,
                                            const gm1b_dissipative_heating_arrays *arrays, void *stream) {
    const gm1b_dissipative_heating_arrays *s = arrays;
    if (s == nullptr || ni < 1 || nj < 1 || nk < 1) {
        gm1b_set_error("gm1b_dissipative_heating: need arrays and ni, nj, nk >= 1");
        return GM1B_ERR_ARGUMENT;
    }
    if (!all_set({s->dissten, s->pi0, s->ppi, s->qa, s->thten1})) {
        gm1b_set_error("gm1b_dissipative_heating: a required array is NULL");
        return GM1B_ERR_ARGUMENT;
    }
    DissArgs a{s->dissten, s->pi0, s->ppi, s->qa, s->thten1, ni, nj, nk};
    const size_t n = (size_t)ni * nj * nk, want = (n + kEW - 1) / kEW, cap = (size_t)148 * 16;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("dissipative_heating_kernel", st);
    dissipative_heating_kernel<<<(unsigned)(want < cap ? want : cap), kEW, 0, st>>>(a);
    ps.stop();
    return launch_ok("dissipative_heating_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}
