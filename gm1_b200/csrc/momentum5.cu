// momentum5.cu - sm_100a kernels of the terrain/open fifth-order momentum
// advection of the padded (ng = 3) lane: the mass fluxes rru, rrv, rrw (with
// the terrain term), the divergence divx, and the advu / advv / advw
// increments of uten / vten / wten, for CM1's lateral families.
//
// Behaviour followed (reference file:line):
//   cpu_terrain_open_momentum_advection5_inplace
//       src/cm1core/cuda_momentum_advection5.py:753-1068
//   lateral families (periodic wrap, open-side inflow substitution and
//   edits)  :103-208
//
// Design (B200): three launches instead of the reference's six.  (1) every
// u and v face's mass flux; (2) rrw and divx together (each cell forms the
// two rrw words its divergence needs, writing its own); (3) one momentum
// pass where a thread owns the u face, the v face and the w face at its
// (k, y, x).  Upwind face fluxes read the six points that hold both upwind
// stencils before the mass-flux sign is known, so no load waits on it.
// Binary32 one operation at a time in the reference's order: word-identical.
#include "gm1b_common.cuh"

namespace gm1b {
namespace {

constexpr int G = 3;

struct MomArgs {
    const float *u3d, *v3d, *w3d, *uh, *vh;
    const float *rho0, *rf0, *rrf0, *c2, *gz, *gzu, *gzv, *rgzu, *rgzv, *dzdx, *dzdy;
    float *uten, *vten, *wten, *rru, *rrv, *rrw, *divx;
    int ni, nj, nk;
    int per[4], opn[4];  // west, east, south, north
    float rdx, rdy, rdz, dz;
    // vertical column: 0 uniform (dz); 1 terrain branch on a stretched column
    // (sigma, sigmaf, rds, rdsf profiles, physical top ztop, base density from
    // the padded rho0p); 2 flat column (rdz*mh / rdz*mf, the column's rho0p,
    // rf0, rr0, rrf0; no terrain terms), cuda_gm1_child_stretched_momentum.py:56-330
    int vmode;
    const float *rho0p, *sigma, *sigmaf, *rds, *rdsf, *mh, *mf, *rr0;
    float ztop, rdzm;
};

// 32-bit element offsets (the host refuses grids whose padded arrays reach
// 2^31 words)
__device__ __forceinline__ unsigned iu(const MomArgs &a, int k, int y, int x) {
    return ((unsigned)k * (unsigned)(a.nj + 2 * G) + (unsigned)y) * (unsigned)(a.ni + 1 + 2 * G) + (unsigned)x;
}
__device__ __forceinline__ unsigned iv(const MomArgs &a, int k, int y, int x) {
    return ((unsigned)k * (unsigned)(a.nj + 1 + 2 * G) + (unsigned)y) * (unsigned)(a.ni + 2 * G) + (unsigned)x;
}
__device__ __forceinline__ unsigned iw(const MomArgs &a, int k, int y, int x) {
    return ((unsigned)k * (unsigned)(a.nj + 2 * G) + (unsigned)y) * (unsigned)(a.ni + 2 * G) + (unsigned)x;
}
__device__ __forceinline__ unsigned ic(const MomArgs &a, int k, int j, int i) {
    return ((unsigned)k * (unsigned)a.nj + (unsigned)j) * (unsigned)a.ni + (unsigned)i;
}
__device__ __forceinline__ int clampn(int x, int n) { return x < 0 ? 0 : (x >= n ? n - 1 : x); }
// periodic wraps of a cell (c*) and a face (f*) index
__device__ __forceinline__ int cxw(const MomArgs &a, int i) {
    return (a.per[0] && i < 0) ? i + a.ni : ((a.per[1] && i >= a.ni) ? i - a.ni : i);
}
__device__ __forceinline__ int fxw(const MomArgs &a, int i) {
    return (a.per[0] && i < 0) ? i + a.ni : ((a.per[1] && i > a.ni) ? i - a.ni : i);
}
__device__ __forceinline__ int cyw(const MomArgs &a, int j) {
    return (a.per[2] && j < 0) ? j + a.nj : ((a.per[3] && j >= a.nj) ? j - a.nj : j);
}
__device__ __forceinline__ int fyw(const MomArgs &a, int j) {
    return (a.per[2] && j < 0) ? j + a.nj : ((a.per[3] && j > a.nj) ? j - a.nj : j);
}
// face-level c2 at Fortran face kface, clamped column
__device__ __forceinline__ float c2m(const MomArgs &a, int kface, int j, int i) {
    return __ldg(a.c2 + ic(a, kface - 1, clampn(j, a.nj), clampn(i, a.ni)));
}

// x * the column's vertical reciprocal at mass level k (uniform rdz, the
// terrain branch's rdsf(k), or the flat column's (x*rdz)*mh(k))
__device__ __forceinline__ float zmass(const MomArgs &a, float x, int k) {
    if (a.vmode == 2) return (x * a.rdzm) * __ldg(a.mh + k);
    return x * (a.vmode == 1 ? __ldg(a.rdsf + k) : a.rdz);
}
// the same at w level kf (rds(kf) / (x*rdz)*mf(kf))
__device__ __forceinline__ float zface(const MomArgs &a, float x, int kf) {
    if (a.vmode == 2) return (x * a.rdzm) * __ldg(a.mf + kf);
    return x * (a.vmode == 1 ? __ldg(a.rds + kf) : a.rdz);
}
// a boundary correction: uniform and terrain ((q*c)*(r*h)) as adv.F is
// grouped in the uniform text; the flat text groups it ((q*c)*r)*h
__device__ __forceinline__ float bcorr(const MomArgs &a, float q, float c, float r, float h) {
    return a.vmode == 2 ? ((q * c) * r) * h : q * (c * (r * h));
}

__device__ __forceinline__ float up5(float m, float s0, float s1, float s2, float s3, float s4, float s5) {
    const bool pos = m >= 0.0f;
    const float r = flx5(pos ? s0 : s5, pos ? s1 : s4, pos ? s2 : s3, pos ? s3 : s2, pos ? s4 : s1);
    return m * r;
}

#define LU(k, y, x) __ldg(a.u3d + iu(a, (k), (y), (x)))
#define LV(k, y, x) __ldg(a.v3d + iv(a, (k), (y), (x)))
#define LW(k, y, x) __ldg(a.w3d + iw(a, (k), (y), (x)))
#define RU(k, y, x) a.rru[iu(a, (k), (y), (x))]
#define RV(k, y, x) a.rrv[iv(a, (k), (y), (x))]
#define RW(k, y, x) a.rrw[iw(a, (k), (y), (x))]

__device__ float u_fx(const MomArgs &a, int k, int j, int face) {
    const int y = j + G, x = face + G;
    const float m = 0.5f * (RU(k, y, fxw(a, face) + G) + RU(k, y, fxw(a, face + 1) + G));
    return up5(m, LU(k, y, x - 2), LU(k, y, x - 1), LU(k, y, x), LU(k, y, x + 1), LU(k, y, x + 2), LU(k, y, x + 3));
}

__device__ float u_fy_base(const MomArgs &a, int k, int face, int i_face) {
    const int y = face + G, x = i_face + G;
    const float m = 0.5f * (RV(k, y, cxw(a, i_face) + G) + RV(k, y, cxw(a, i_face - 1) + G));
    return up5(m, LU(k, y - 3, x), LU(k, y - 2, x), LU(k, y - 1, x), LU(k, y, x), LU(k, y + 1, x), LU(k, y + 2, x));
}

__device__ float u_fy(const MomArgs &a, int k, int face, int i_face) {
    const int y = face + G;
    const float mt = RV(k, y, cxw(a, i_face) + G) + RV(k, y, cxw(a, i_face - 1) + G);
    if (face == 0 && a.opn[2] && mt >= 0.0f) return u_fy_base(a, k, 1, i_face);
    if (face == a.nj && a.opn[3] && mt <= 0.0f) return u_fy_base(a, k, a.nj - 1, i_face);
    return u_fy_base(a, k, face, i_face);
}

__device__ float v_fx_base(const MomArgs &a, int k, int j_face, int face) {
    const int y = j_face + G, x = face + G;
    const float m = 0.5f * (RU(k, cyw(a, j_face) + G, x) + RU(k, cyw(a, j_face - 1) + G, x));
    return up5(m, LV(k, y, x - 3), LV(k, y, x - 2), LV(k, y, x - 1), LV(k, y, x), LV(k, y, x + 1), LV(k, y, x + 2));
}

__device__ float v_fx(const MomArgs &a, int k, int j_face, int face) {
    const int x = face + G;
    const float mt = RU(k, cyw(a, j_face) + G, x) + RU(k, cyw(a, j_face - 1) + G, x);
    if (face == 0 && a.opn[0] && mt >= 0.0f) return v_fx_base(a, k, j_face, 1);
    if (face == a.ni && a.opn[1] && mt <= 0.0f) return v_fx_base(a, k, j_face, a.ni - 1);
    return v_fx_base(a, k, j_face, face);
}

__device__ float v_fy(const MomArgs &a, int k, int face, int i) {
    const int y = face + G, x = i + G;
    const float m = 0.5f * (RV(k, fyw(a, face) + G, x) + RV(k, fyw(a, face + 1) + G, x));
    return up5(m, LV(k, y - 2, x), LV(k, y - 1, x), LV(k, y, x), LV(k, y + 1, x), LV(k, y + 2, x), LV(k, y + 3, x));
}

__device__ float w_fx_base(const MomArgs &a, int kf, int j, int face) {
    const int y = j + G, x = face + G;
    const float c2 = 0.5f * (c2m(a, kf, j, face - 1) + c2m(a, kf, j, face)), c1 = 1.0f - c2;
    const float m = c2 * RU(kf, y, x) + c1 * RU(kf - 1, y, x);
    return up5(m, LW(kf, y, x - 3), LW(kf, y, x - 2), LW(kf, y, x - 1), LW(kf, y, x), LW(kf, y, x + 1),
               LW(kf, y, x + 2));
}

__device__ float w_fx(const MomArgs &a, int kf, int j, int face) {
    const int y = j + G, x = face + G;
    const float c2 = 0.5f * (c2m(a, kf, j, face - 1) + c2m(a, kf, j, face)), c1 = 1.0f - c2;
    const float m = c2 * RU(kf, y, x) + c1 * RU(kf - 1, y, x);
    if (face == 0 && a.opn[0] && m >= 0.0f) return w_fx_base(a, kf, j, 1);
    if (face == a.ni && a.opn[1] && m <= 0.0f) return w_fx_base(a, kf, j, a.ni - 1);
    return w_fx_base(a, kf, j, face);
}

__device__ float w_fy_base(const MomArgs &a, int kf, int face, int i) {
    const int y = face + G, x = i + G;
    const float c2 = 0.5f * (c2m(a, kf, face - 1, i) + c2m(a, kf, face, i)), c1 = 1.0f - c2;
    const float m = c2 * RV(kf, y, x) + c1 * RV(kf - 1, y, x);
    return up5(m, LW(kf, y - 3, x), LW(kf, y - 2, x), LW(kf, y - 1, x), LW(kf, y, x), LW(kf, y + 1, x),
               LW(kf, y + 2, x));
}

__device__ float w_fy(const MomArgs &a, int kf, int face, int i) {
    const int y = face + G, x = i + G;
    const float c2 = 0.5f * (c2m(a, kf, face - 1, i) + c2m(a, kf, face, i)), c1 = 1.0f - c2;
    const float m = c2 * RV(kf, y, x) + c1 * RV(kf - 1, y, x);
    if (face == 0 && a.opn[2] && m >= 0.0f) return w_fy_base(a, kf, 1, i);
    if (face == a.nj && a.opn[3] && m <= 0.0f) return w_fy_base(a, kf, a.nj - 1, i);
    return w_fy_base(a, kf, face, i);
}

// vertical flux of u (is_u) or v at Fortran face kface of column (j, i)
__device__ float uv_z(const MomArgs &a, bool is_u, int kface, int j, int i) {
    const int y = j + G, x = i + G, nk = a.nk;
    float m, c2;
    if (is_u) {
        m = 0.5f * (RW(kface, y, cxw(a, i) + G) + RW(kface, y, cxw(a, i - 1) + G));
        c2 = 0.5f * (c2m(a, kface, j, i - 1) + c2m(a, kface, j, i));
    } else {
        m = 0.5f * (RW(kface, cyw(a, j) + G, x) + RW(kface, cyw(a, j - 1) + G, x));
        c2 = 0.5f * (c2m(a, kface, j - 1, i) + c2m(a, kface, j, i));
    }
    const float c1 = 1.0f - c2;
#define Q(l) (is_u ? LU((l), y, x) : LV((l), y, x))
    float r;
    if (kface == 2) {
        r = m >= 0.0f ? c1 * Q(1) + c2 * Q(2) : flx3(Q(3), Q(2), Q(1));
    } else if (kface == nk) {
        r = m >= 0.0f ? flx3(Q(nk - 2), Q(nk - 1), Q(nk)) : c1 * Q(nk - 1) + c2 * Q(nk);
    } else if (kface == 3) {
        r = m >= 0.0f ? flx3(Q(1), Q(2), Q(3)) : flx5(Q(5), Q(4), Q(3), Q(2), Q(1));
    } else if (kface == nk - 1) {
        r = m >= 0.0f ? flx5(Q(kface - 3), Q(kface - 2), Q(kface - 1), Q(kface), Q(kface + 1))
                      : flx3(Q(kface + 1), Q(kface), Q(kface - 1));
    } else {
        return up5(m, Q(kface - 3), Q(kface - 2), Q(kface - 1), Q(kface), Q(kface + 1), Q(kface + 2));
    }
#undef Q
    return m * r;
}

__device__ float w_z(const MomArgs &a, int k, int j, int i) {
    const int y = j + G, x = i + G, nk = a.nk;
    const float m = 0.5f * (RW(k, y, x) + RW(k + 1, y, x));
#define Q(l) LW((l), y, x)
    float r;
    if (k == 1) {
        r = m >= 0.0f ? 0.5f * (Q(1) + Q(2)) : flx3(Q(3), Q(2), Q(1));
    } else if (k == 2) {
        r = m >= 0.0f ? flx3(Q(1), Q(2), Q(3)) : flx5(Q(5), Q(4), Q(3), Q(2), Q(1));
    } else if (k == nk - 1) {
        r = m >= 0.0f ? flx5(Q(k - 2), Q(k - 1), Q(k), Q(k + 1), Q(k + 2)) : flx3(Q(k + 2), Q(k + 1), Q(k));
    } else if (k == nk) {
        r = m >= 0.0f ? flx3(Q(k - 1), Q(k), Q(k + 1)) : 0.5f * (Q(k) + Q(k + 1));
    } else {
        return up5(m, Q(k - 2), Q(k - 1), Q(k), Q(k + 1), Q(k + 2), Q(k + 3));
    }
#undef Q
    return m * r;
}

// (1) horizontal mass fluxes; grid: x over 0..ni, y over 0..nj, z over k = 1..nk
__global__ void __launch_bounds__(128) mom5_mass_kernel(MomArgs a) {
    const int x = blockIdx.x * 32 + threadIdx.x, yy = blockIdx.y * 4 + threadIdx.y, k = blockIdx.z + 1;
    const int ni = a.ni, nj = a.nj, k0 = k - 1;
    if (x > ni || yy > nj) return;
    if (a.vmode == 2) {  // flat column: rho0(1,1,k) u and rho0(1,1,k) v
        const float r0 = __ldg(a.rho0p + iw(a, k, G, G));
        if (yy < nj) RU(k, yy + G, x + G) = r0 * LU(k, yy + G, x + G);
        if (x < ni) RV(k, yy + G, x + G) = r0 * LV(k, yy + G, x + G);
        return;
    }
    if (yy < nj) {  // u face (row yy, face x)
        const int j = yy, l = x - 1 < 0 ? 0 : x - 1, r = x < ni - 1 ? x : ni - 1;
        const float density = a.vmode == 1 ? __ldg(a.rho0p + iw(a, k, j + G, x + G - 1)) + __ldg(a.rho0p + iw(a, k, j + G, x + G))
                                           : __ldg(a.rho0 + ic(a, k0, j, l)) + __ldg(a.rho0 + ic(a, k0, j, r));
        RU(k, j + G, x + G) = (0.5f * density) * (LU(k, j + G, x + G) * __ldg(a.rgzu + (size_t)j * (ni + 1) + x));
    }
    if (x < ni) {  // v face (face yy, column x)
        const int s = yy - 1 < 0 ? 0 : yy - 1, n = yy < nj - 1 ? yy : nj - 1;
        const float density = a.vmode == 1 ? __ldg(a.rho0p + iw(a, k, yy + G - 1, x + G)) + __ldg(a.rho0p + iw(a, k, yy + G, x + G))
                                           : __ldg(a.rho0 + ic(a, k0, s, x)) + __ldg(a.rho0 + ic(a, k0, n, x));
        RV(k, yy + G, x + G) = (0.5f * density) * (LV(k, yy + G, x + G) * __ldg(a.rgzv + (size_t)yy * ni + x));
    }
}

// rrw at level k (2..nk) of cell (j, i); 0 at levels 1 and nk+1
__device__ __forceinline__ float rrw_value(const MomArgs &a, int k, int j, int i) {
    if (k <= 1 || k >= a.nk + 1) return 0.0f;
    if (a.vmode == 2) return __ldg(a.rf0 + ic(a, k - 1, 0, 0)) * LW(k, j + G, i + G);
    const bool pr = a.vmode == 1;
    const float zt = pr ? a.ztop : (float)a.nk * a.dz, rzt = 1.0f / zt, rdz0 = 1.0f / a.dz;
    const float sigmaf = pr ? __ldg(a.sigmaf + k) : (float)(k - 1) * a.dz;
    const float sigma = pr ? __ldg(a.sigma + k - 1) : ((float)k - 1.5f) * a.dz;
    float r2 = (sigmaf - sigma) * (pr ? __ldg(a.rds + k) : rdz0);
    const float r1 = 0.5f * (1.0f - r2);
    r2 = 0.5f * r2;
    const int y = j + G, x = i + G;
    const float ux = r2 * (RU(k, y, x) + RU(k, y, x + 1)) + r1 * (RU(k - 1, y, x) + RU(k - 1, y, x + 1));
    const float vy = r2 * (RV(k, y, x) + RV(k, y + 1, x)) + r1 * (RV(k - 1, y, x) + RV(k - 1, y + 1, x));
    const size_t c2d = (size_t)j * a.ni + i;
    float terrain = ux * __ldg(a.dzdx + c2d) + vy * __ldg(a.dzdy + c2d);
    terrain = terrain * (sigmaf - zt);
    terrain = terrain * __ldg(a.gz + c2d);
    terrain = terrain * rzt;
    return __ldg(a.rf0 + ic(a, k - 1, j, i)) * LW(k, y, x) + terrain;
}

// (2) rrw and divx; grid: x over i, y over j, z over k0 = 0..nk-1
__global__ void __launch_bounds__(128) mom5_rrw_divx_kernel(MomArgs a) {
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 4 + threadIdx.y, k0 = blockIdx.z, k = k0 + 1;
    if (i >= a.ni || j >= a.nj) return;
    const int y = j + G, x = i + G;
    const float lo = rrw_value(a, k, j, i), hi = rrw_value(a, k + 1, j, i);
    RW(k, y, x) = lo;
    if (k == a.nk) RW(k + 1, y, x) = hi;
    float value = (RU(k, y, x + 1) - RU(k, y, x)) * a.rdx + (RV(k, y + 1, x) - RV(k, y, x)) * a.rdy;
    if (a.vmode == 2) {  // the flat column's ((d*rdz)*mh(k)) with cm1.F's smeps 1e-30
        value = value + ((hi - lo) * a.rdzm) * __ldg(a.mh + k);
        a.divx[ic(a, k0, j, i)] = fabsf(value) < 1.0e-30f ? 0.0f : value;
        return;
    }
    value = value + (hi - lo) * (a.vmode == 1 ? __ldg(a.rdsf + k) : a.rdz);
    a.divx[ic(a, k0, j, i)] = fabsf(value) < 1.0e-20f ? 0.0f : value;
}

// (3) advu / advv / advw; grid: x over 0..ni, y over 0..nj, z over k = 1..nk
__global__ void __launch_bounds__(128) mom5_adv_kernel(MomArgs a) {
    const int xx = blockIdx.x * 32 + threadIdx.x, yy = blockIdx.y * 4 + threadIdx.y, k = blockIdx.z + 1;
    const int ni = a.ni, nj = a.nj, nk = a.nk, k0 = k - 1;
    if (xx > ni || yy > nj) return;
    // advu at face f = xx of row j = yy
    const int ff = a.per[0] ? 0 : 1, lf = a.per[1] ? ni : ni - 1;
    if (yy < nj && xx >= ff && xx <= lf) {
        const int j = yy, f = xx, y = j + G, x = f + G, west = cxw(a, f - 1), east = cxw(a, f);
        const float advx = -(u_fx(a, k, j, f) - u_fx(a, k, j, f - 1)) * a.rdx;
        float advy = -(u_fy(a, k, j + 1, f) - u_fy(a, k, j, f)) * a.rdy;
        const float uc = LU(k, y, x);
        if (j == 0 && a.opn[2]) {
            const float m = RV(k, G, east + G) + RV(k, G, west + G);
            if (m >= 0.0f) {
                const float corr = (RV(k, G + 1, west + G) - RV(k, G, west + G)) + (RV(k, G + 1, east + G) - RV(k, G, east + G));
                advy = advy - bcorr(a, uc * 0.5f, corr, a.rdy, __ldg(a.vh + y));
            }
        } else if (j == nj - 1 && a.opn[3]) {
            const float m = RV(k, G + nj, east + G) + RV(k, G + nj, west + G);
            if (m <= 0.0f) {
                const float corr = (RV(k, y + 1, west + G) - RV(k, y, west + G)) + (RV(k, y + 1, east + G) - RV(k, y, east + G));
                advy = advy - bcorr(a, uc * 0.5f, corr, a.rdy, __ldg(a.vh + y));
            }
        }
        float advz;
        if (k == 1) advz = zmass(a, -uv_z(a, true, 2, j, f), k);
        else if (k == nk) advz = zmass(a, uv_z(a, true, nk, j, f), k);
        else advz = zmass(a, -(uv_z(a, true, k + 1, j, f) - uv_z(a, true, k, j, f)), k);
        float total = (advx + advy) + advz;
        total = total + uc * (0.5f * (a.divx[ic(a, k0, j, east)] + a.divx[ic(a, k0, j, west)]));
        const float scale = a.vmode == 2 ? __ldg(a.rr0 + ic(a, k0, 0, 0))
                                         : __ldg(a.gzu + (size_t)j * (ni + 1) + f) /
                                               (0.5f * (__ldg(a.rho0 + ic(a, k0, j, west)) + __ldg(a.rho0 + ic(a, k0, j, east))));
        const unsigned p = iu(a, k, y, x);
        a.uten[p] = a.uten[p] + total * scale;
    }
    // advv at face g = yy of column i = xx
    const int fr = a.per[2] ? 0 : 1, lr = a.per[3] ? nj : nj - 1;
    if (xx < ni && yy >= fr && yy <= lr) {
        const int g = yy, i = xx, y = g + G, x = i + G, south = cyw(a, g - 1), north = cyw(a, g);
        float advx = -(v_fx(a, k, g, i + 1) - v_fx(a, k, g, i)) * a.rdx;
        const float advy = -(v_fy(a, k, g, i) - v_fy(a, k, g - 1, i)) * a.rdy;
        const float vc = LV(k, y, x);
        if (i == 0 && a.opn[0]) {
            const float m = RU(k, north + G, G) + RU(k, south + G, G);
            if (m >= 0.0f) {
                const float corr = (RU(k, south + G, G + 1) - RU(k, south + G, G)) + (RU(k, north + G, G + 1) - RU(k, north + G, G));
                advx = advx - bcorr(a, vc * 0.5f, corr, a.rdx, __ldg(a.uh + G));
            }
        } else if (i == ni - 1 && a.opn[1]) {
            const float m = RU(k, north + G, G + ni) + RU(k, south + G, G + ni);
            if (m <= 0.0f) {
                const float corr = (RU(k, south + G, x + 1) - RU(k, south + G, x)) + (RU(k, north + G, x + 1) - RU(k, north + G, x));
                advx = advx - bcorr(a, vc * 0.5f, corr, a.rdx, __ldg(a.uh + x));
            }
        }
        float advz;
        if (k == 1) advz = zmass(a, -uv_z(a, false, 2, g, i), k);
        else if (k == nk) advz = zmass(a, uv_z(a, false, nk, g, i), k);
        else advz = zmass(a, -(uv_z(a, false, k + 1, g, i) - uv_z(a, false, k, g, i)), k);
        float total = (advx + advy) + advz;
        total = total + vc * (0.5f * (a.divx[ic(a, k0, north, i)] + a.divx[ic(a, k0, south, i)]));
        const float scale = a.vmode == 2 ? __ldg(a.rr0 + ic(a, k0, 0, 0))
                                         : __ldg(a.gzv + (size_t)g * ni + i) /
                                               (0.5f * (__ldg(a.rho0 + ic(a, k0, south, i)) + __ldg(a.rho0 + ic(a, k0, north, i))));
        const unsigned p = iv(a, k, y, x);
        a.vten[p] = a.vten[p] + total * scale;
    }
    // advw at Fortran face kf = k + 1 (2..nk) of column (yy, xx)
    if (xx < ni && yy < nj && k < nk) {
        const int kf = k + 1, j = yy, i = xx, y = j + G, x = i + G;
        const float dfx = -(w_fx(a, kf, j, i + 1) - w_fx(a, kf, j, i)), dfy = -(w_fy(a, kf, j + 1, i) - w_fy(a, kf, j, i));
        float advx = a.vmode == 2 ? (dfx * a.rdx) * __ldg(a.uh + x) : dfx * (a.rdx * __ldg(a.uh + x));
        float advy = a.vmode == 2 ? (dfy * a.rdy) * __ldg(a.vh + y) : dfy * (a.rdy * __ldg(a.vh + y));
        const float c2 = __ldg(a.c2 + ic(a, kf - 1, j, i)), c1 = 1.0f - c2;
        const float wc = LW(kf, y, x);
        if (i == 0 && a.opn[0]) {
            const float m = c2 * RU(kf, y, G) + c1 * RU(kf - 1, y, G);
            if (m >= 0.0f) {
                const float corr = c1 * (RU(kf - 1, y, G + 1) - RU(kf - 1, y, G)) + c2 * (RU(kf, y, G + 1) - RU(kf, y, G));
                advx = advx - bcorr(a, wc, corr, a.rdx, __ldg(a.uh + x));
            }
        } else if (i == ni - 1 && a.opn[1]) {
            const float m = c2 * RU(kf, y, G + ni) + c1 * RU(kf - 1, y, G + ni);
            if (m <= 0.0f) {
                const float corr = c1 * (RU(kf - 1, y, x + 1) - RU(kf - 1, y, x)) + c2 * (RU(kf, y, x + 1) - RU(kf, y, x));
                advx = advx - bcorr(a, wc, corr, a.rdx, __ldg(a.uh + x));
            }
        }
        if (j == 0 && a.opn[2]) {
            const float m = c2 * RV(kf, G, x) + c1 * RV(kf - 1, G, x);
            if (m >= 0.0f) {
                const float corr = c1 * (RV(kf - 1, G + 1, x) - RV(kf - 1, G, x)) + c2 * (RV(kf, G + 1, x) - RV(kf, G, x));
                advy = advy - bcorr(a, wc, corr, a.rdy, __ldg(a.vh + y));
            }
        } else if (j == nj - 1 && a.opn[3]) {
            const float m = c2 * RV(kf, G + nj, x) + c1 * RV(kf - 1, G + nj, x);
            if (m <= 0.0f) {
                const float corr = c1 * (RV(kf - 1, y + 1, x) - RV(kf - 1, y, x)) + c2 * (RV(kf, y + 1, x) - RV(kf, y, x));
                advy = advy - bcorr(a, wc, corr, a.rdy, __ldg(a.vh + y));
            }
        }
        const float advz = zface(a, -(w_z(a, kf, j, i) - w_z(a, kf - 1, j, i)), kf);
        float total = (advx + advy) + advz;
        total = total + wc * (c2 * a.divx[ic(a, kf - 1, j, i)] + c1 * a.divx[ic(a, kf - 2, j, i)]);
        const float scale = a.vmode == 2 ? __ldg(a.rrf0 + ic(a, kf - 1, 0, 0))
                                         : __ldg(a.rrf0 + ic(a, kf - 1, j, i)) * __ldg(a.gz + (size_t)j * ni + i);
        const unsigned p = iw(a, kf, y, x);
        a.wten[p] = a.wten[p] + total * scale;
    }
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

namespace {

int mom_args(int ni, int nj, int nk, const gm1b_momentum5_arrays *s, uint32_t lateral_obc, float dx, float dy,
             float dz, MomArgs &a, const char *what) {
    a.vmode = 0;
    a.rho0p = a.sigma = a.sigmaf = a.rds = a.rdsf = a.mh = a.mf = a.rr0 = nullptr;
    a.ztop = a.rdzm = 0.0f;
    if (s == nullptr || ni < 7 || nj < 7 || nk < 8) {
        gm1b_set_error("%s: need arrays, ni >= 7, nj >= 7, nk >= 8", what);
        return GM1B_ERR_ARGUMENT;
    }
    if ((size_t)(nk + 3) * (size_t)(nj + 7) * (size_t)(ni + 7) >= ((size_t)1 << 31)) {
        gm1b_set_error("%s: a %dx%dx%d grid's padded arrays reach 2^31 words; the kernels index with 32-bit offsets",
                       what, ni, nj, nk);
        return GM1B_ERR_ARGUMENT;
    }
    if (!(dx > 0.0f) || !(dy > 0.0f) || !(dz > 0.0f) || !isfinite(dx) || !isfinite(dy) || !isfinite(dz)) {
        gm1b_set_error("%s: dx, dy, dz must be finite and > 0", what);
        return GM1B_ERR_ARGUMENT;
    }
    int side[4];
    for (int q = 0; q < 4; ++q) {
        side[q] = (int)((lateral_obc >> (4 * q)) & 15u);
        if (side[q] < 1 || side[q] > 4) {
            gm1b_set_error("%s: lateral side codes must be 1..4 (wbc|ebc<<4|sbc<<8|nbc<<12)", what);
            return GM1B_ERR_ARGUMENT;
        }
    }
    if ((side[0] == 1) != (side[1] == 1) || (side[2] == 1) != (side[3] == 1)) {
        gm1b_set_error("%s: a direction cannot be periodic on one side only", what);
        return GM1B_ERR_ARGUMENT;
    }
    const void *need[] = {s->u3d, s->uten, s->rru, s->v3d, s->vten, s->rrv, s->w3d, s->wten, s->rrw, s->uh, s->vh,
                          s->rho0_3d, s->rf0, s->rrf0, s->c2, s->gz, s->gzu, s->gzv, s->rgzu, s->rgzv, s->dzdx,
                          s->dzdy, s->divx};
    for (const void *q : need)
        if (q == nullptr) {
            gm1b_set_error("%s: a required array is NULL", what);
            return GM1B_ERR_ARGUMENT;
        }
    a.u3d = s->u3d;
    a.v3d = s->v3d;
    a.w3d = s->w3d;
    a.uh = s->uh;
    a.vh = s->vh;
    a.rho0 = s->rho0_3d;
    a.rf0 = s->rf0;
    a.rrf0 = s->rrf0;
    a.c2 = s->c2;
    a.gz = s->gz;
    a.gzu = s->gzu;
    a.gzv = s->gzv;
    a.rgzu = s->rgzu;
    a.rgzv = s->rgzv;
    a.dzdx = s->dzdx;
    a.dzdy = s->dzdy;
    a.uten = s->uten;
    a.vten = s->vten;
    a.wten = s->wten;
    a.rru = s->rru;
    a.rrv = s->rrv;
    a.rrw = s->rrw;
    a.divx = s->divx;
    a.ni = ni;
    a.nj = nj;
    a.nk = nk;
    for (int q = 0; q < 4; ++q) {
        a.per[q] = side[q] == 1;
        a.opn[q] = side[q] == 2;
    }
    a.rdx = 1.0f / dx;
    a.rdy = 1.0f / dy;
    a.rdz = 1.0f / dz;
    a.dz = dz;
    return GM1B_OK;
}

int enqueue_mass(const MomArgs &a, cudaStream_t st) {
    const dim3 blk(32, 4);
    const dim3 g_face((a.ni + 1 + 31) / 32, (a.nj + 1 + 3) / 4, a.nk), g_cell((a.ni + 31) / 32, (a.nj + 3) / 4, a.nk);
    {
        ProfScope ps("mom5_mass_kernel", st);
        mom5_mass_kernel<<<g_face, blk, 0, st>>>(a);
        ps.stop();
    }
    if (!launch_ok("mom5_mass_kernel")) return GM1B_ERR_CUDA;
    {
        ProfScope ps("mom5_rrw_divx_kernel", st);
        mom5_rrw_divx_kernel<<<g_cell, blk, 0, st>>>(a);
        ps.stop();
    }
    return launch_ok("mom5_rrw_divx_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

int enqueue_transport(const MomArgs &a, cudaStream_t st) {
    const dim3 g_face((a.ni + 1 + 31) / 32, (a.nj + 1 + 3) / 4, a.nk);
    ProfScope ps("mom5_adv_kernel", st);
    mom5_adv_kernel<<<g_face, dim3(32, 4), 0, st>>>(a);
    ps.stop();
    return launch_ok("mom5_adv_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

}  // namespace

extern "C" int32_t gm1b_momentum_mass_flux5(int32_t ni, int32_t nj, int32_t nk, const gm1b_momentum5_arrays *s,
                                            uint32_t lateral_obc, float dx, float dy, float dz, void *stream) {
    MomArgs a;
    const int r = mom_args(ni, nj, nk, s, lateral_obc, dx, dy, dz, a, "gm1b_momentum_mass_flux5");
    return r != GM1B_OK ? r : enqueue_mass(a, static_cast<cudaStream_t>(stream));
}

extern "C" int32_t gm1b_momentum_transport5(int32_t ni, int32_t nj, int32_t nk, const gm1b_momentum5_arrays *s,
                                            uint32_t lateral_obc, float dx, float dy, float dz, void *stream) {
    MomArgs a;
    const int r = mom_args(ni, nj, nk, s, lateral_obc, dx, dy, dz, a, "gm1b_momentum_transport5");
    return r != GM1B_OK ? r : enqueue_transport(a, static_cast<cudaStream_t>(stream));
}

extern "C" int32_t gm1b_momentum_advection5(int32_t ni, int32_t nj, int32_t nk, const gm1b_momentum5_arrays *s,
                                            uint32_t lateral_obc, float dx, float dy, float dz, void *stream) {
    MomArgs a;
    const int r = mom_args(ni, nj, nk, s, lateral_obc, dx, dy, dz, a, "gm1b_momentum_advection5");
    if (r != GM1B_OK) return r;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int m = enqueue_mass(a, st);
    return m != GM1B_OK ? m : enqueue_transport(a, st);
}

// ---------------------------------------------------------------------------
// the same operator on a stretched column (launch_cuda_gm1_child_stretched_momentum5,
// src/cm1core/cuda_gm1_child_stretched_momentum.py:540-780): terrain branch
// (rdsf / rds / sigma / sigmaf and the physical top) or flat column
// (rdz*mh / rdz*mf and the column's base state)
// ---------------------------------------------------------------------------
namespace {
int column_args(int ni, int nj, int nk, const gm1b_momentum5_arrays *s, uint32_t lateral_obc, float dx, float dy,
                const gm1b_momentum_column *c, MomArgs &a, const char *what) {
    if (c == nullptr || (c->flat != 0 && c->flat != 1) || c->rho0_padded == nullptr) {
        gm1b_set_error("%s: need a column with flat = 0 or 1 and the padded base density", what);
        return GM1B_ERR_ARGUMENT;
    }
    if (c->flat ? (c->mh == nullptr || c->mf == nullptr || c->rr0 == nullptr || !(c->rdz > 0.0f) ||
                   !isfinite(c->rdz))
                : (c->sigma == nullptr || c->sigmaf == nullptr || c->rds == nullptr || c->rdsf == nullptr ||
                   !(c->ztop > 0.0f) || !isfinite(c->ztop))) {
        gm1b_set_error("%s: a flat column needs mh, mf, rr0 and rdz > 0; a terrain column sigma, sigmaf, rds, rdsf "
                       "and ztop > 0", what);
        return GM1B_ERR_ARGUMENT;
    }
    // dz forms only the uniform reciprocals, which a stretched column never reads
    const int r = mom_args(ni, nj, nk, s, lateral_obc, dx, dy, 1.0f, a, what);
    if (r != GM1B_OK) return r;
    a.vmode = c->flat ? 2 : 1;
    a.rho0p = c->rho0_padded, a.sigma = c->sigma, a.sigmaf = c->sigmaf, a.rds = c->rds, a.rdsf = c->rdsf;
    a.mh = c->mh, a.mf = c->mf, a.rr0 = c->rr0, a.ztop = c->ztop, a.rdzm = c->rdz;
    return GM1B_OK;
}
}  // namespace

extern "C" int32_t gm1b_momentum_mass_flux5_column(int32_t ni, int32_t nj, int32_t nk, const gm1b_momentum5_arrays *s,
                                                   uint32_t lateral_obc, float dx, float dy,
                                                   const gm1b_momentum_column *column, void *stream) {
    MomArgs a;
    const int r = column_args(ni, nj, nk, s, lateral_obc, dx, dy, column, a, "gm1b_momentum_mass_flux5_column");
    return r != GM1B_OK ? r : enqueue_mass(a, static_cast<cudaStream_t>(stream));
}

extern "C" int32_t gm1b_momentum_transport5_column(int32_t ni, int32_t nj, int32_t nk, const gm1b_momentum5_arrays *s,
                                                   uint32_t lateral_obc, float dx, float dy,
                                                   const gm1b_momentum_column *column, void *stream) {
    MomArgs a;
    const int r = column_args(ni, nj, nk, s, lateral_obc, dx, dy, column, a, "gm1b_momentum_transport5_column");
    return r != GM1B_OK ? r : enqueue_transport(a, static_cast<cudaStream_t>(stream));
}

extern "C" int32_t gm1b_momentum_advection5_column(int32_t ni, int32_t nj, int32_t nk, const gm1b_momentum5_arrays *s,
                                                   uint32_t lateral_obc, float dx, float dy,
                                                   const gm1b_momentum_column *column, void *stream) {
    MomArgs a;
    const int r = column_args(ni, nj, nk, s, lateral_obc, dx, dy, column, a, "gm1b_momentum_advection5_column");
    if (r != GM1B_OK) return r;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int m = enqueue_mass(a, st);
    return m != GM1B_OK ? m : enqueue_transport(a, st);
}
