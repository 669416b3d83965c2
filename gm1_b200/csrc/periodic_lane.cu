// periodic_lane.cu - sm_100a kernels of the flat serial-periodic dry lane:
// the psolver=3 acoustic RK stage and the dry RK3 trajectory around it.
//
// Behaviour followed (reference file:line):
//   acoustic stage   src/cm1core/cuda_sound3_periodic.py:672-1064 (CPU twin),
//                    launch order :1216-1400
//   dry trajectory   src/cm1core/cuda_psolver3_trajectory.py:456-901 (CPU twin),
//                    launch order :1460-1700
//
// Design (B200): every pass is one grid over the padded arrays with x fastest
// (coalesced rows); periodic halo fills are fused into the producing pass
// (each live cell also writes the halo words that mirror it), so no
// single-thread fill kernels exist.  The vertically implicit w-pi' solve runs
// one CTA per 32-column row tile: the k-parallel parts (divergence, pi'
// advection, fpk, tridiagonal coefficients, pressure update) use all warps,
// and the sequential Thomas sweep runs on one warp out of shared memory.
#include <cstdint>
#include <cstdio>

#include "gm1b_common.cuh"

namespace gm1b {
namespace {

using Arr = gm1b_periodic_arrays;

constexpr int kTX = 32;  // x extent of a 3-D elementwise block
constexpr int kTY = 4;   // y extent
constexpr int kColWarps = 16;  // warps of the column CTA
constexpr int kColArrays = 11;  // shared-memory column arrays of the column CTA

// ---------------------------------------------------------------------------
// trajectory: stage preparation, instant mass flux and divergence
// (_prepare_stage_cpu :456-471, _instant_mass_flux_cpu :474-493,
//  _divergence_cpu :515-533)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTX *kTY) traj_prepare_kernel(Arr a, Dims d, float rdx, float rdy,
                                                                float rdz) {
    const int i = blockIdx.x * kTX + threadIdx.x;
    const int j = blockIdx.y * kTY + threadIdx.y;
    const int k = blockIdx.z;
    const int ni = d.ni, nj = d.nj, nk = d.nk;
    if (i >= ni + 2 || j >= nj + 2) return;
    const bool klive = k >= 1 && k <= nk;
    if (klive) {
        const int jw = wrap(j, nj), iw = wrap(i, ni);
        const size_t sw = d.s(k, jw, iw);
        a.thv[d.s(k, j, i)] = a.th0[sw] + a.th3d[sw];
        const float piadv = a.pi0[sw] + a.pp3d[sw];
        a.piadv[d.s(k, j, i)] = piadv;
        if (jw == j && iw == i) a.ppterm[d.s(k, j, i)] = piadv * kRddcv;
    }
    if (i <= ni) {
        a.rru[d.u(k, j, i)] = (klive && j >= 1 && j <= nj) ? a.rho0[d.s(k, j, 1)] * a.u3d[d.u(k, j, i)] : 0.0f;
    }
    if (j <= nj) {
        a.rrv[d.v(k, j, i)] = (klive && i >= 1 && i <= ni) ? a.rho0[d.s(k, 1, i)] * a.v3d[d.v(k, j, i)] : 0.0f;
    }
    if (j < nj && i < ni) {
        a.rrw[d.w(k, j, i)] = (k >= 2 && k <= nk) ? a.rf0[d.s(k, j + 1, i + 1)] * a.w3d[d.w(k, j, i)] : 0.0f;
    }
    float div = 0.0f;
    if (klive && j >= 1 && j <= nj && i >= 1 && i <= ni) {
        const float rhox = a.rho0[d.s(k, j, 1)];
        const float ue = rhox * a.u3d[d.u(k, j, i)];
        const float uw = rhox * a.u3d[d.u(k, j, i - 1)];
        const float vn = a.rho0[d.s(k, 1, i)] * a.v3d[d.v(k, j, i)];
        const float vs = a.rho0[d.s(k, 1, i)] * a.v3d[d.v(k, j - 1, i)];
        const float wt = (k + 1 <= nk) ? a.rf0[d.s(k + 1, j, i)] * a.w3d[d.w(k + 1, j - 1, i - 1)] : 0.0f;
        const float wb = (k >= 2) ? a.rf0[d.s(k, j, i)] * a.w3d[d.w(k, j - 1, i - 1)] : 0.0f;
        const float dx = (ue - uw) * rdx;
        const float dy = (vn - vs) * rdy;
        const float dz = (wt - wb) * rdz;
        div = (dx + dy) + dz;
        if (fabsf(div) < kSmeps) div = 0.0f;
    }
    a.divx[d.s(k, j, i)] = div;
}

// ---------------------------------------------------------------------------
// trajectory: fifth-order momentum advection and dry buoyancy
// (_momentum_tendencies_cpu :536-660 with the flux helpers :305-426)
// ---------------------------------------------------------------------------

// A field restricted to its live block, indexed from 0 with the strides and
// offsets of its padded array.
struct View {
    const float *p;
    int sz, sy, oz, oy, ox;
    // 32-bit offsets: every periodic-lane array holds fewer than 2^31 words
    // (the entry points reject larger grids)
    __device__ __forceinline__ float at(int k, int j, int i) const {
        return __ldg(p + ((k + oz) * sz + (j + oy) * sy + (i + ox)));
    }
};

// Upwind fifth-order face value from the six points lo..lo+5 that hold both
// upwind stencils: vel >= 0 uses lo..lo+4, vel < 0 uses lo+5..lo+1 (the same
// flx5 operand order as the reference's two branches).  All six points are
// read before the sign of vel is known, so no load waits on the velocity.
__device__ __forceinline__ float upwind5(float vel, float s0, float s1, float s2, float s3, float s4, float s5) {
    const bool pos = vel >= 0.0f;
    const float r = flx5(pos ? s0 : s5, pos ? s1 : s4, pos ? s2 : s3, pos ? s3 : s2, pos ? s4 : s1);
    return vel * r;
}

// x flux at the face between points face-1 and face (stencil face-3..face+2)
__device__ __forceinline__ float x_flux5(const View &s, float vel, int face, int j, int k, int n) {
    return upwind5(vel, s.at(k, j, pmod(face - 3, n)), s.at(k, j, pmod(face - 2, n)), s.at(k, j, pmod(face - 1, n)),
                   s.at(k, j, pmod(face, n)), s.at(k, j, pmod(face + 1, n)), s.at(k, j, pmod(face + 2, n)));
}

__device__ __forceinline__ float y_flux5(const View &s, float vel, int i, int face, int k, int n) {
    return upwind5(vel, s.at(k, pmod(face - 3, n), i), s.at(k, pmod(face - 2, n), i), s.at(k, pmod(face - 1, n), i),
                   s.at(k, pmod(face, n), i), s.at(k, pmod(face + 1, n), i), s.at(k, pmod(face + 2, n), i));
}

// flux at the face between points b and b+1 (stencil b-2..b+3)
__device__ __forceinline__ float x_flux5c(const View &s, float vel, int b, int j, int k, int n) {
    return upwind5(vel, s.at(k, j, pmod(b - 2, n)), s.at(k, j, pmod(b - 1, n)), s.at(k, j, pmod(b, n)),
                   s.at(k, j, pmod(b + 1, n)), s.at(k, j, pmod(b + 2, n)), s.at(k, j, pmod(b + 3, n)));
}

__device__ __forceinline__ float y_flux5c(const View &s, float vel, int i, int b, int k, int n) {
    return upwind5(vel, s.at(k, pmod(b - 2, n), i), s.at(k, pmod(b - 1, n), i), s.at(k, pmod(b, n), i),
                   s.at(k, pmod(b + 1, n), i), s.at(k, pmod(b + 2, n), i), s.at(k, pmod(b + 3, n), i));
}

// CM1 stag=1/2/3 vertical flux at Fortran face `face`; nk levels in the view
__device__ __forceinline__ float z_flux_mass(const View &s, float v, int face, int j, int i, float c1, float c2,
                                             int nk) {
    float recon;
    if (face == 2) {
        recon = (v >= 0.0f) ? (c1 * s.at(0, j, i) + c2 * s.at(1, j, i))
                            : flx3(s.at(2, j, i), s.at(1, j, i), s.at(0, j, i));
    } else if (face == 3) {
        recon = (v >= 0.0f) ? flx3(s.at(0, j, i), s.at(1, j, i), s.at(2, j, i))
                            : flx5(s.at(4, j, i), s.at(3, j, i), s.at(2, j, i), s.at(1, j, i), s.at(0, j, i));
    } else if (face == nk - 1) {
        recon = (v >= 0.0f) ? flx5(s.at(nk - 5, j, i), s.at(nk - 4, j, i), s.at(nk - 3, j, i), s.at(nk - 2, j, i),
                                   s.at(nk - 1, j, i))
                            : flx3(s.at(nk - 1, j, i), s.at(nk - 2, j, i), s.at(nk - 3, j, i));
    } else if (face == nk) {
        recon = (v >= 0.0f) ? flx3(s.at(nk - 3, j, i), s.at(nk - 2, j, i), s.at(nk - 1, j, i))
                            : (c1 * s.at(nk - 2, j, i) + c2 * s.at(nk - 1, j, i));
    } else {
        return upwind5(v, s.at(face - 4, j, i), s.at(face - 3, j, i), s.at(face - 2, j, i), s.at(face - 1, j, i),
                       s.at(face, j, i), s.at(face + 1, j, i));
    }
    return v * recon;
}

// CM1 stag=4 vertical flux at mass level `level`; the view holds nk+1 levels
__device__ __forceinline__ float z_flux_w(const View &s, float v, int level, int j, int i, int nk) {
    float recon;
    if (level == 1) {
        recon = (v >= 0.0f) ? (0.5f * (s.at(0, j, i) + s.at(1, j, i)))
                            : flx3(s.at(2, j, i), s.at(1, j, i), s.at(0, j, i));
    } else if (level == 2) {
        recon = (v >= 0.0f) ? flx3(s.at(0, j, i), s.at(1, j, i), s.at(2, j, i))
                            : flx5(s.at(5, j, i), s.at(4, j, i), s.at(3, j, i), s.at(2, j, i), s.at(1, j, i));
    } else if (level == nk - 1) {
        recon = (v >= 0.0f) ? flx5(s.at(nk - 4, j, i), s.at(nk - 3, j, i), s.at(nk - 2, j, i), s.at(nk - 1, j, i),
                                   s.at(nk, j, i))
                            : flx3(s.at(nk, j, i), s.at(nk - 1, j, i), s.at(nk - 2, j, i));
    } else if (level == nk) {
        recon = (v >= 0.0f) ? flx3(s.at(nk - 2, j, i), s.at(nk - 1, j, i), s.at(nk, j, i))
                            : (0.5f * (s.at(nk - 1, j, i) + s.at(nk, j, i)));
    } else {
        return upwind5(v, s.at(level - 3, j, i), s.at(level - 2, j, i), s.at(level - 1, j, i), s.at(level, j, i),
                       s.at(level + 1, j, i), s.at(level + 2, j, i));
    }
    return v * recon;
}

// grid: x over faces/cells 0..ni, y over 0..nj, z over k = 0..nk-1 (view level)
__global__ void __launch_bounds__(kTX *kTY) traj_momentum_kernel(Arr a, Dims d, float rdx, float rdy, float rdz,
                                                                 int advect, int buoyancy) {
    const int x = blockIdx.x * kTX + threadIdx.x;
    const int y = blockIdx.y * kTY + threadIdx.y;
    const int k = blockIdx.z;
    const int ni = d.ni, nj = d.nj, nk = d.nk;
    if (x > ni || y > nj) return;
    const int ssz = (nj + 2) * (ni + 2), ssy = ni + 2;
    const int usz = (nj + 2) * (ni + 1), usy = ni + 1;
    const int vsz = (nj + 1) * (ni + 2), vsy = ni + 2;
    const int wsz = nj * ni, wsy = ni;
    const View u{a.u3d, usz, usy, 1, 1, 0};
    const View v{a.v3d, vsz, vsy, 1, 0, 1};
    const View w{a.w3d, wsz, wsy, 1, 0, 0};
    const View rru{a.rru, usz, usy, 1, 1, 0};
    const View rrv{a.rrv, vsz, vsy, 1, 0, 1};
    const View rrw{a.rrw, wsz, wsy, 1, 0, 0};
    const View dv{a.divx, ssz, ssy, 1, 1, 1};
    const int ks = k + 1;

    // u at face f = x of row j = y
    if (y < nj && advect) {
        const int j = y, js = y + 1, f = x;
        const int fu = f == ni ? 0 : f;
        const int fm = pmod(fu - 1, ni), fp = pmod(fu + 1, ni);
        const float east_v = 0.5f * (rru.at(k, j, fu) + rru.at(k, j, fp));
        const float west_v = 0.5f * (rru.at(k, j, fm) + rru.at(k, j, fu));
        const float fx_e = x_flux5c(u, east_v, fu, j, k, ni);
        const float fx_w = x_flux5c(u, west_v, fu - 1, j, k, ni);
        const int jn = pmod(j + 1, nj);
        const float south_v = 0.5f * (rrv.at(k, j, fu) + rrv.at(k, j, fm));
        const float north_v = 0.5f * (rrv.at(k, jn, fu) + rrv.at(k, jn, fm));
        const float fy_s = y_flux5(u, south_v, fu, j, k, nj);
        const float fy_n = y_flux5(u, north_v, fu, j + 1, k, nj);
        const float advx = (-(fx_e - fx_w)) * rdx;
        const float advy = (-(fy_n - fy_s)) * rdy;
        float advz = 0.0f;
        if (nk >= 6) {
            if (k == 0) {
                const float vv = 0.5f * (rrw.at(1, j, fu) + rrw.at(1, j, fm));
                const float top =
                    z_flux_mass(u, vv, 2, j, fu, a.c1[d.s(2, js, fu + 1)], a.c2[d.s(2, js, fu + 1)], nk);
                advz = (-top) * rdz;
            } else if (k == nk - 1) {
                const float vv = 0.5f * (rrw.at(nk - 1, j, fu) + rrw.at(nk - 1, j, fm));
                const float bottom =
                    z_flux_mass(u, vv, nk, j, fu, a.c1[d.s(nk, js, fu + 1)], a.c2[d.s(nk, js, fu + 1)], nk);
                advz = bottom * rdz;
            } else {
                const int lo = k + 1, hi = k + 2;
                const float vlo = 0.5f * (rrw.at(lo - 1, j, fu) + rrw.at(lo - 1, j, fm));
                const float vhi = 0.5f * (rrw.at(hi - 1, j, fu) + rrw.at(hi - 1, j, fm));
                const float flo =
                    z_flux_mass(u, vlo, lo, j, fu, a.c1[d.s(lo, js, fu + 1)], a.c2[d.s(lo, js, fu + 1)], nk);
                const float fhi =
                    z_flux_mass(u, vhi, hi, j, fu, a.c1[d.s(hi, js, fu + 1)], a.c2[d.s(hi, js, fu + 1)], nk);
                advz = (-(fhi - flo)) * rdz;
            }
        }
        const float corr = u.at(k, j, fu) * (0.5f * (dv.at(k, j, fu) + dv.at(k, j, fm)));
        a.uten[d.u(ks, js, f)] = (((advx + advy) + advz) + corr) * a.rr0[d.s(ks, js, fu + 1)];
    }
    // v at face g = y of column i = x
    if (x < ni && advect) {
        const int i = x, is = x + 1, g = y;
        const int gv = g == nj ? 0 : g;
        const int gm = pmod(gv - 1, nj), gp = pmod(gv + 1, nj), ip = pmod(i + 1, ni);
        const float west_v = 0.5f * (rru.at(k, gv, i) + rru.at(k, gm, i));
        const float east_v = 0.5f * (rru.at(k, gv, ip) + rru.at(k, gm, ip));
        const float fx_w = x_flux5(v, west_v, i, gv, k, ni);
        const float fx_e = x_flux5(v, east_v, i + 1, gv, k, ni);
        const float south_v = 0.5f * (rrv.at(k, gm, i) + rrv.at(k, gv, i));
        const float north_v = 0.5f * (rrv.at(k, gv, i) + rrv.at(k, gp, i));
        const float fy_s = y_flux5c(v, south_v, i, gv - 1, k, nj);
        const float fy_n = y_flux5c(v, north_v, i, gv, k, nj);
        const float advx = (-(fx_e - fx_w)) * rdx;
        const float advy = (-(fy_n - fy_s)) * rdy;
        float advz = 0.0f;
        if (nk >= 6) {
            if (k == 0) {
                const float vv = 0.5f * (rrw.at(1, gv, i) + rrw.at(1, gm, i));
                advz = (-z_flux_mass(v, vv, 2, gv, i, a.c1[d.s(2, gv + 1, is)], a.c2[d.s(2, gv + 1, is)], nk)) * rdz;
            } else if (k == nk - 1) {
                const float vv = 0.5f * (rrw.at(nk - 1, gv, i) + rrw.at(nk - 1, gm, i));
                advz = z_flux_mass(v, vv, nk, gv, i, a.c1[d.s(nk, gv + 1, is)], a.c2[d.s(nk, gv + 1, is)], nk) * rdz;
            } else {
                const int lo = k + 1, hi = k + 2;
                const float vlo = 0.5f * (rrw.at(lo - 1, gv, i) + rrw.at(lo - 1, gm, i));
                const float vhi = 0.5f * (rrw.at(hi - 1, gv, i) + rrw.at(hi - 1, gm, i));
                const float flo =
                    z_flux_mass(v, vlo, lo, gv, i, a.c1[d.s(lo, gv + 1, is)], a.c2[d.s(lo, gv + 1, is)], nk);
                const float fhi =
                    z_flux_mass(v, vhi, hi, gv, i, a.c1[d.s(hi, gv + 1, is)], a.c2[d.s(hi, gv + 1, is)], nk);
                advz = (-(fhi - flo)) * rdz;
            }
        }
        const float corr = v.at(k, gv, i) * (0.5f * (dv.at(k, gv, i) + dv.at(k, gm, i)));
        a.vten[d.v(ks, g, is)] = (((advx + advy) + advz) + corr) * a.rr0[d.s(ks, gv + 1, is)];
    }
    // w at face q = k (1..nk-1) of column (y, x)
    if (k >= 1 && k < nk && x < ni && y < nj) {
        const int q = k, qs = k + 1, i = x, j = y, js = y + 1, is = x + 1;
        float wt = 0.0f;
        if (advect) {
            const float c2 = a.c2[d.s(qs, js, is)];
            const float c1 = 1.0f - c2;
            const int i1 = pmod(i + 1, ni), j1 = pmod(j + 1, nj);
            const float ux_w = c2 * rru.at(q, j, i) + c1 * rru.at(q - 1, j, i);
            const float ux_e = c2 * rru.at(q, j, i1) + c1 * rru.at(q - 1, j, i1);
            const float vy_s = c2 * rrv.at(q, j, i) + c1 * rrv.at(q - 1, j, i);
            const float vy_n = c2 * rrv.at(q, j1, i) + c1 * rrv.at(q - 1, j1, i);
            const float fx_w = x_flux5(w, ux_w, i, j, q, ni);
            const float fx_e = x_flux5(w, ux_e, i + 1, j, q, ni);
            const float fy_s = y_flux5(w, vy_s, i, j, q, nj);
            const float fy_n = y_flux5(w, vy_n, i, j + 1, q, nj);
            const float advx = (-(fx_e - fx_w)) * rdx;
            const float advy = (-(fy_n - fy_s)) * rdy;
            const float vlo = 0.5f * (rrw.at(q - 1, j, i) + rrw.at(q, j, i));
            const float vhi = 0.5f * (rrw.at(q, j, i) + rrw.at(q + 1, j, i));
            const float flo = z_flux_w(w, vlo, q, j, i, nk);
            const float fhi = z_flux_w(w, vhi, q + 1, j, i, nk);
            const float advz = (-(fhi - flo)) * rdz;
            const float corr = w.at(q, j, i) * (c2 * dv.at(q, j, i) + c1 * dv.at(q - 1, j, i));
            wt = (((advx + advy) + advz) + corr) * a.rrf0[d.s(qs, js, is)];
        }
        if (buoyancy) {
            const float lower = kGrav * (a.th3d[d.s(q, js, is)] * a.rth0[d.s(q, js, is)]);
            const float upper = kGrav * (a.th3d[d.s(q + 1, js, is)] * a.rth0[d.s(q + 1, js, is)]);
            const float b = a.c1[d.s(qs, js, is)] * lower + a.c2[d.s(qs, js, is)] * upper;
            wt = wt + b;
        }
        if (advect || buoyancy) a.wten[d.w(qs, j, i)] = wt;
    }
}

// ---------------------------------------------------------------------------
// acoustic stage: preparation (cpu_sound3_periodic_stage_inplace :690-822)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTX *kTY) sound_prep_kernel(Arr a, Dims d, int nrk, float dts, float rdz, float cp,
                                                              float beta, int scratch_outputs, int fused_reset) {
    const int i = blockIdx.x * kTX + threadIdx.x;
    const int j = blockIdx.y * kTY + threadIdx.y;
    const int k = blockIdx.z;
    const int ni = d.ni, nj = d.nj, nk = d.nk;
    if (i >= ni + 2 || j >= nj + 2) return;
    if (fused_reset && i == 0 && j == 0 && k == 0) {
        // grid-barrier counter of the fused stage kernel; its error word only
        // on the call's first fused stage (fused_reset == 2)
        *reinterpret_cast<unsigned long long *>(a.tri_residual) = 0ull;
        if (fused_reset == 2) reinterpret_cast<int *>(a.tri_residual)[2] = 0;
    }
    const size_t c = d.s(k, j, i);
    const bool klive = k >= 1 && k <= nk;
    if (klive) {
        a.ppd[c] = a.ppx[c];
        if (nrk != 1) a.pp3d[c] = a.ppi[c];
    }
    if (i <= ni) {
        const size_t fu = d.u(k, j, i);
        if (nrk != 1) a.u3d[fu] = a.ua[fu];
        a.rru[fu] = 0.0f;
    }
    if (j <= nj) {
        const size_t fv = d.v(k, j, i);
        if (nrk != 1) a.v3d[fv] = a.va[fv];
        a.rrv[fv] = 0.0f;
    }
    float qk = 0.0f, pk1 = 0.0f, pk2 = 0.0f, mm = 0.0f;
    if (klive && j >= 1 && j <= nj && i >= 1 && i <= ni) {
        const float mh = a.mh[c];
        const float tem = (dts * rdz) * mh;
        float r2 = (dts * rdz) * mh;
        r2 = r2 * a.rr0[c];
        r2 = r2 * a.rf0[d.s(k + 1, j, i)];
        float r1 = (dts * rdz) * mh;
        r1 = r1 * a.rr0[c];
        r1 = r1 * a.rf0[c];
        const float tem1 = ((dts * rdz) * cp) * a.mf[c];
        qk = tem * a.ppterm[c];
        if (k < nk) {
            const size_t up = d.s(k + 1, j, i);
            pk2 = r2 * ((-a.c2[up]) * a.piadv[up] + (1.0f - a.c1[up]) * a.piadv[c]);
        }
        if (k > 1) {
            pk1 = r1 * (a.c1[c] * a.piadv[d.s(k - 1, j, i)] + (a.c2[c] - 1.0f) * a.piadv[c]);
        }
        mm = tem1 * (a.c2[c] * a.thv[c] + a.c1[c] * a.thv[d.s(k - 1, j, i)]);
        const size_t wc = d.w(k, j - 1, i - 1);
        const float wa = a.wa[wc];
        a.rrw[wc] = wa * beta;
        if (nrk != 1) a.w3d[wc] = wa;
    }
    a.qk[c] = qk;
    a.pk1[c] = pk1;
    a.pk2[c] = pk2;
    a.mm[c] = mm;
    if (scratch_outputs) {
        a.fpk[c] = 0.0f;
        a.divh[c] = 0.0f;
        a.hadvp[c] = 0.0f;
        a.elim_c[c] = 0.0f;
        a.elim_d[c] = 0.0f;
        a.tri_aa[c] = 0.0f;
        a.tri_bb[c] = 0.0f;
        a.tri_cc[c] = 0.0f;
        a.tri_dd[c] = 0.0f;
        a.tri_pivot[c] = 0.0f;
        a.tri_residual[c] = 0.0f;
    }
}

// ---------------------------------------------------------------------------
// acoustic small step, part 1: horizontal pressure-gradient update of u and v
// and the running rru/rrv averages (:824-858 and :1005-1027)
// grid: x over 0..ni+1, y over 0..nj+1, z over k = 1..nk
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTX *kTY) sound_uv_kernel(Arr a, Dims d, float dts, float tem1x, float tem2y,
                                                            int last, float tavg) {
    const int x = blockIdx.x * kTX + threadIdx.x;
    const int y = blockIdx.y * kTY + threadIdx.y;
    const int k = blockIdx.z + 1;
    const int ni = d.ni, nj = d.nj;
    if (x >= ni + 2 || y >= nj + 2) return;
    if (y >= 1 && x <= ni) {  // u face (j = y in 1..nj+1, f = x in 0..ni)
        float pg = tem1x * (a.ppd[d.s(k, y, x + 1)] - a.ppd[d.s(k, y, x)]);
        pg = pg * a.uf[x + 1];
        pg = pg * (a.thv[d.s(k, y, x + 1)] + a.thv[d.s(k, y, x)]);
        const size_t fu = d.u(k, y, x);
        const float un = a.u3d[fu] + (dts * a.dtu0[(size_t)y * (ni + 1) + x]) * (a.uten[fu] - pg);
        a.u3d[fu] = un;
        a.rru[fu] = last ? (a.rru[fu] + un) * tavg : a.rru[fu] + un;
    }
    if (y <= nj && x >= 1) {  // v face (g = y in 0..nj, i = x in 1..ni+1)
        float pg = tem2y * (a.ppd[d.s(k, y + 1, x)] - a.ppd[d.s(k, y, x)]);
        pg = pg * a.vf[y + 1];
        pg = pg * (a.thv[d.s(k, y + 1, x)] + a.thv[d.s(k, y, x)]);
        const size_t fv = d.v(k, y, x);
        const float vn = a.v3d[fv] + (dts * a.dtv0[(size_t)y * (ni + 2) + x]) * (a.vten[fv] - pg);
        a.v3d[fv] = vn;
        a.rrv[fv] = last ? (a.rrv[fv] + vn) * tavg : a.rrv[fv] + vn;
    }
}

// ---------------------------------------------------------------------------
// acoustic small step, part 2: per column divergence, pi' advection, fpk,
// implicit w solve, pi' update with the kdiv filter, ppd, ppx and the rrw
// average (:859-1003), with the stage-end periodic fills fused in.
// One CTA = kTX consecutive columns of one row j; blockDim = (kTX, kColWarps).
// ---------------------------------------------------------------------------
struct ColumnArgs {
    int nrk, n, nloop;
    float dts, rdx, rdy, alph, beta, asq, kdiv, smeps, temx, temy, rnloop;
    int scratch_outputs;
    int fill_pp3d;   // write pp3d halos at the last small step
    int post_ppx;    // trajectory post-step ppx completion fused at nrk=3
    // fast mode (no scratch outputs): the first small step stores 1/pivot in
    // tri_pivot and the elimination coefficients in tri_cc, later small
    // steps of the stage read them back
    int store_consts, use_consts;
};

__global__ void __launch_bounds__(kTX *kColWarps, 1) sound_column_kernel(Arr a, Dims d, ColumnArgs p) {
    extern __shared__ float smem[];
    const int ni = d.ni, nj = d.nj, nk = d.nk;
    const int lane = threadIdx.x;
    const int wy = threadIdx.y;
    const int i = blockIdx.x * kTX + lane + 1;  // live column index 1..ni
    const int j = blockIdx.y + 1;               // live row 1..nj
    const bool live = i <= ni;
    const int L = nk + 2;
    float *s_fpk = smem;
    float *s_w = s_fpk + L * kTX;
    float *s_pp = s_w + L * kTX;
    float *s_a1 = s_pp + L * kTX;
    float *s_a2 = s_a1 + L * kTX;
    float *s_mm = s_a2 + L * kTX;
    float *s_aa = s_mm + L * kTX;
    float *s_bb = s_aa + L * kTX;
    float *s_cc = s_bb + L * kTX;
    float *s_dd = s_cc + L * kTX;
    float *s_ed = s_dd + L * kTX;
#define SM(arr, k) arr[(k) * kTX + lane]
    const int last = p.n == p.nloop;

    // phase A: k-parallel divergence, pressure advection and fpk
    if (live) {
#pragma unroll 2
        for (int k = 1 + wy; k <= nk + 1; k += kColWarps) {
            SM(s_w, k) = a.w3d[d.w(k, j - 1, i - 1)];
            if (k > nk) continue;
            const size_t c = d.s(k, j, i);
            const float uE = a.u3d[d.u(k, j, i)], uW = a.u3d[d.u(k, j, i - 1)];
            const float vN = a.v3d[d.v(k, j, i)], vS = a.v3d[d.v(k, j - 1, i)];
            const float du = ((uE - uW) * p.rdx) * a.uh[i];
            const float dv = ((vN - vS) * p.rdy) * a.vh[j];
            float div = du + dv;
            if (fabsf(div) < p.smeps) div = 0.0f;
            const float pc = a.piadv[c];
            const float gxw = pc - a.piadv[c - 1];
            const float gxe = a.piadv[c + 1] - pc;
            const float gys = pc - a.piadv[d.s(k, j - 1, i)];
            const float gyn = a.piadv[d.s(k, j + 1, i)] - pc;
            float hx = uW * gxw + uE * gxe;
            hx = ((-hx) * p.temx) * a.uh[i];
            float hy = vS * gys + vN * gyn;
            hy = ((-hy) * p.temy) * a.vh[j];
            const float hp = hx + hy;
            const float src = p.dts * (a.ppten[c] - a.ppterm[c] * div);
            const float qk = a.qk[c];
            const float a1 = a.pk1[c] + qk;
            const float a2 = a.pk2[c] - qk;
            const float vert = a.w3d[d.w(k, j - 1, i - 1)] * a1 + a.w3d[d.w(k + 1, j - 1, i - 1)] * a2;
            const float fpk = (src + hp) + p.beta * vert;
            SM(s_fpk, k) = fpk;
            SM(s_a1, k) = a1;
            SM(s_a2, k) = a2;
            SM(s_mm, k) = a.mm[c];
            SM(s_pp, k) = a.pp3d[c];
            if (p.scratch_outputs && last) {
                a.divh[c] = div;
                a.hadvp[c] = hp;
                a.fpk[c] = fpk;
            }
        }
    }
    __syncthreads();
    // phase A2: tridiagonal coefficients and right-hand side, k = 2..nk
    if (live) {
#pragma unroll 2
        for (int k = 2 + wy; k <= nk; k += kColWarps) {
            const float mm = SM(s_mm, k);
            const float aa = (k >= 3) ? (-p.asq) * (mm * SM(s_a1, k - 1)) : 0.0f;
            const float pd = SM(s_pp, k) - SM(s_pp, k - 1);
            const float fwk = p.dts * a.wten[d.w(k, j - 1, i - 1)] + p.beta * ((-mm) * pd);
            const float upd = (SM(s_pp, k) + SM(s_fpk, k)) - (SM(s_pp, k - 1) + SM(s_fpk, k - 1));
            const float dd = (SM(s_w, k) + fwk) + p.alph * ((-mm) * upd);
            SM(s_aa, k) = aa;
            SM(s_dd, k) = dd;
            if (p.use_consts) {
                // stage-constant 1/pivot and elimination coefficient stored by
                // the first small step of this stage (identical words)
                const size_t c = d.s(k, j, i);
                SM(s_bb, k) = a.tri_pivot[c];
                SM(s_cc, k) = (k < nk) ? a.tri_cc[c] : 0.0f;
                continue;
            }
            const float cc = (k < nk) ? (-p.asq) * ((-mm) * SM(s_a2, k)) : 0.0f;
            const float diag = (-SM(s_a1, k)) + SM(s_a2, k - 1);
            const float bb = 1.0f - p.asq * (mm * diag);
            SM(s_bb, k) = bb;
            SM(s_cc, k) = cc;
            if (p.scratch_outputs && last) {
                const size_t c = d.s(k, j, i);
                a.tri_aa[c] = aa;
                a.tri_bb[c] = bb;
                a.tri_cc[c] = cc;
                a.tri_dd[c] = dd;
            }
        }
    }
    __syncthreads();
    // phase B: Thomas sweep, one lane per column, out of shared memory
    if (wy == 0 && live && p.use_consts) {
        // forward elimination of the right-hand side only: no division
        float ed = 0.0f;
        for (int k = 2; k <= nk; ++k) {
            const float aa = SM(s_aa, k), dd = SM(s_dd, k), inv = SM(s_bb, k);
            if (k < nk) {
                const float num = (k < 3) ? dd : (dd - aa * ed);
                ed = num * inv;
                SM(s_ed, k) = ed;
            } else {
                SM(s_w, k) = (dd - aa * ed) * inv;
            }
        }
        for (int k = nk - 1; k >= 2; --k) SM(s_w, k) = SM(s_cc, k) * SM(s_w, k + 1) + SM(s_ed, k);
    } else if (wy == 0 && live) {
        float ec = 0.0f, ed = 0.0f;
        for (int k = 2; k <= nk; ++k) {
            const float aa = SM(s_aa, k), bb = SM(s_bb, k), cc = SM(s_cc, k), dd = SM(s_dd, k);
            const float pivot = (k < 3) ? bb : (aa * ec + bb);
            const float inv = 1.0f / pivot;
            if (p.scratch_outputs && last) a.tri_pivot[d.s(k, j, i)] = pivot;
            if (p.store_consts) a.tri_pivot[d.s(k, j, i)] = inv;
            if (k < nk) {
                const float num = (k < 3) ? dd : (dd - aa * ed);
                ec = (-cc) * inv;
                ed = num * inv;
                SM(s_cc, k) = ec;  // elimination coefficient replaces cc
                SM(s_ed, k) = ed;
                if (p.scratch_outputs && last) a.elim_d[d.s(k, j, i)] = ed;
                if (p.store_consts) a.tri_cc[d.s(k, j, i)] = ec;
            } else {
                SM(s_w, k) = (dd - aa * ed) * inv;
            }
        }
        for (int k = nk - 1; k >= 2; --k) SM(s_w, k) = SM(s_cc, k) * SM(s_w, k + 1) + SM(s_ed, k);
    }
    __syncthreads();
    // phase C: pressure update, filter, averages and fused fills, k = 1..nk
    if (live) {
        const bool wrap_j0 = j == nj, wrap_j1 = j == 1, wrap_i0 = i == ni, wrap_i1 = i == 1;
        const int rows[3] = {j, wrap_j0 ? 0 : -1, wrap_j1 ? nj + 1 : -1};
        const int cols[3] = {i, wrap_i0 ? 0 : -1, wrap_i1 ? ni + 1 : -1};
        const bool halo_cell = wrap_j0 || wrap_j1 || wrap_i0 || wrap_i1;
#pragma unroll 2
        for (int k = 1 + wy; k <= nk; k += kColWarps) {
            const size_t c = d.s(k, j, i);
            const float wk = SM(s_w, k), wk1 = SM(s_w, k + 1);
            if (p.scratch_outputs && last && k >= 2) {
                float lhs = SM(s_aa, k) * SM(s_w, k - 1);
                lhs = lhs + SM(s_bb, k) * wk;
                // s_cc holds elimination coefficients for k < nk; recompute cc
                const float cc = (k < nk) ? (-p.asq) * ((-SM(s_mm, k)) * SM(s_a2, k)) : 0.0f;
                lhs = lhs + cc * wk1;
                a.tri_residual[c] = lhs - SM(s_dd, k);
            }
            if (k >= 2) a.w3d[d.w(k, j - 1, i - 1)] = wk;
            const float old = SM(s_pp, k);
            const float vert = wk * SM(s_a1, k) + wk1 * SM(s_a2, k);
            float upd = (old + SM(s_fpk, k)) + p.alph * vert;
            if (fabsf(upd) < p.smeps) upd = 0.0f;
            const float ek = p.kdiv * (upd - old);
            const float ppd = upd + ek;
            a.pp3d[c] = upd;
            a.ppd[c] = ppd;
            if (p.scratch_outputs && last) a.elim_c[c] = ek;
            const bool write_ppx = p.nrk == 3 && last;
            const float ppx = p.post_ppx ? (upd + ek) : ek;
            if (write_ppx) a.ppx[c] = ppx;
            const size_t wc = d.w(k, j - 1, i - 1);
            a.rrw[wc] = last ? (a.rrw[wc] + wk * p.alph) * p.rnloop : a.rrw[wc] + wk;
            if (halo_cell) {
                _Pragma("unroll") for (int r = 0; r < 3; ++r) {
                    if (rows[r] < 0) continue;
                    _Pragma("unroll") for (int q = 0; q < 3; ++q) {
                        if (cols[q] < 0 || (r == 0 && q == 0)) continue;
                        const size_t h = d.s(k, rows[r], cols[q]);
                        if (!last) a.ppd[h] = ppd;
                        if (last && p.fill_pp3d) a.pp3d[h] = upd;
                        if (write_ppx && p.post_ppx) a.ppx[h] = ppx;
                    }
                }
            }
            if (last) {  // stage-end u/v periodic fill (fill_periodic_uv_inplace)
                if (wrap_j0) {
                    a.u3d[d.u(k, 0, i)] = a.u3d[d.u(k, nj, i)];
                    if (i == 1) a.u3d[d.u(k, 0, 0)] = a.u3d[d.u(k, nj, 0)];
                }
                if (wrap_j1) {
                    a.u3d[d.u(k, nj + 1, i)] = a.u3d[d.u(k, 1, i)];
                    if (i == 1) a.u3d[d.u(k, nj + 1, 0)] = a.u3d[d.u(k, 1, 0)];
                }
                if (wrap_i0) {
                    a.v3d[d.v(k, j, 0)] = a.v3d[d.v(k, j, ni)];
                    if (j == 1) a.v3d[d.v(k, 0, 0)] = a.v3d[d.v(k, 0, ni)];
                }
                if (wrap_i1) {
                    a.v3d[d.v(k, j, ni + 1)] = a.v3d[d.v(k, j, 1)];
                    if (j == 1) a.v3d[d.v(k, 0, ni + 1)] = a.v3d[d.v(k, 0, 1)];
                }
            }
        }
    }
#undef SM
}

#include "periodic_stage_fused.cuh"

// ---------------------------------------------------------------------------
// trajectory: averaged-flux rescale and the advected theta carrier
// (_scale_averages_cpu :496-512, sadv part of _theta_tendency_update_cpu)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTX *kTY) traj_theta_prep_kernel(Arr a, Dims d, int include_base) {
    const int i = blockIdx.x * kTX + threadIdx.x;
    const int j = blockIdx.y * kTY + threadIdx.y;
    const int k = blockIdx.z;
    const int ni = d.ni, nj = d.nj, nk = d.nk;
    if (i >= ni + 2 || j >= nj + 2) return;
    const bool klive = k >= 1 && k <= nk;
    if (i <= ni && klive && j >= 1 && j <= nj) {
        const size_t f = d.u(k, j, i);
        a.rru[f] = a.rru[f] * a.rho0[d.s(k, j, 1)];
    }
    if (j <= nj && klive && i >= 1 && i <= ni) {
        const size_t f = d.v(k, j, i);
        a.rrv[f] = a.rrv[f] * a.rho0[d.s(k, 1, i)];
    }
    if (j < nj && i < ni) {
        const size_t f = d.w(k, j, i);
        if (k >= 2 && k <= nk)
            a.rrw[f] = a.rrw[f] * a.rf0[d.s(k, j + 1, i + 1)];
        else if (k == 1 || k == nk + 1)
            a.rrw[f] = 0.0f;
    }
    float s = 0.0f;
    if (klive) {
        const size_t sw = d.s(k, wrap(j, nj), wrap(i, ni));
        const float base = include_base ? (a.th0[sw] - kTh0r) : 0.0f;
        s = base + a.th3d[sw];
    }
    a.sadv[d.s(k, j, i)] = s;
}

// ---------------------------------------------------------------------------
// trajectory: averaged-flux divergence, theta advection and RK update
// (_divergence_cpu, _theta_tendency_update_cpu :663-726) with the periodic
// th3d fill of the stage end / post step fused in
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTX *kTY) traj_theta_kernel(Arr a, Dims d, float rdx, float rdy, float rdz,
                                                              float dttmp, int enabled) {
    const int x = blockIdx.x * kTX + threadIdx.x;
    const int y = blockIdx.y * kTY + threadIdx.y;
    const int kk = blockIdx.z;
    const int ni = d.ni, nj = d.nj, nk = d.nk;
    if (x >= ni + 2 || y >= nj + 2) return;
    const bool live = kk >= 1 && kk <= nk && y >= 1 && y <= nj && x >= 1 && x <= ni;
    if (!live) {
        a.divx[d.s(kk, y, x)] = 0.0f;
        return;
    }
    const int ks = kk, js = y, is = x;
    const int k = kk - 1, j = y - 1, i = x - 1;
    const int ssz = (nj + 2) * (ni + 2), ssy = ni + 2;
    const int usz = (nj + 2) * (ni + 1), usy = ni + 1;
    const int vsz = (nj + 1) * (ni + 2), vsy = ni + 2;
    const int wsz = nj * ni, wsy = ni;
    const View th{a.sadv, ssz, ssy, 1, 1, 1};
    const View rru{a.rru, usz, usy, 1, 1, 0};
    const View rrv{a.rrv, vsz, vsy, 1, 0, 1};
    const View rrw{a.rrw, wsz, wsy, 1, 0, 0};
    // divergence of the scaled averaged fluxes
    const float ddx = (a.rru[d.u(ks, js, is)] - a.rru[d.u(ks, js, is - 1)]) * rdx;
    const float ddy = (a.rrv[d.v(ks, js, is)] - a.rrv[d.v(ks, js - 1, is)]) * rdy;
    const float ddz = (a.rrw[d.w(ks + 1, j, i)] - a.rrw[d.w(ks, j, i)]) * rdz;
    float div = (ddx + ddy) + ddz;
    if (fabsf(div) < kSmeps) div = 0.0f;
    const size_t c = d.s(ks, js, is);
    a.divx[c] = div;
    float tendency = 0.0f;
    if (enabled) {
        const float fx_w = x_flux5(th, rru.at(k, j, i), i, j, k, ni);
        const float fx_e = x_flux5(th, rru.at(k, j, pmod(i + 1, ni)), i + 1, j, k, ni);
        const float fy_s = y_flux5(th, rrv.at(k, j, i), i, j, k, nj);
        const float fy_n = y_flux5(th, rrv.at(k, pmod(j + 1, nj), i), i, j + 1, k, nj);
        const float advx = (-(fx_e - fx_w)) * rdx;
        const float advy = (-(fy_n - fy_s)) * rdy;
        float advz;
        if (k == 0) {
            advz = (-z_flux_mass(th, rrw.at(1, j, i), 2, j, i, a.c1[d.s(2, js, is)], a.c2[d.s(2, js, is)], nk)) * rdz;
        } else if (k == nk - 1) {
            advz = z_flux_mass(th, rrw.at(nk - 1, j, i), nk, j, i, a.c1[d.s(nk, js, is)], a.c2[d.s(nk, js, is)], nk) *
                   rdz;
        } else {
            const int lo = k + 1, hi = k + 2;
            const float flo =
                z_flux_mass(th, rrw.at(lo - 1, j, i), lo, j, i, a.c1[d.s(lo, js, is)], a.c2[d.s(lo, js, is)], nk);
            const float fhi =
                z_flux_mass(th, rrw.at(hi - 1, j, i), hi, j, i, a.c1[d.s(hi, js, is)], a.c2[d.s(hi, js, is)], nk);
            advz = (-(fhi - flo)) * rdz;
        }
        const float corr = th.at(k, j, i) * div;
        tendency = (((advx + advy) + advz) + corr) * a.rr0[c];
    }
    a.thten[c] = tendency;
    float updated = a.tha[c] + dttmp * tendency;
    if (fabsf(updated) < kSmeps) updated = 0.0f;
    a.th3d[c] = updated;
    // periodic th3d halos mirrored from this live cell
    const int rows[3] = {js, js == nj ? 0 : -1, js == 1 ? nj + 1 : -1};
    const int cols[3] = {is, is == ni ? 0 : -1, is == 1 ? ni + 1 : -1};
    _Pragma("unroll") for (int r = 0; r < 3; ++r) {
        if (rows[r] < 0) continue;
        _Pragma("unroll") for (int q = 0; q < 3; ++q) {
            if (cols[q] < 0 || (r == 0 && q == 0)) continue;
            a.th3d[d.s(ks, rows[r], cols[q])] = updated;
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
dim3 box_grid(int nx, int ny, int nz) { return dim3((nx + kTX - 1) / kTX, (ny + kTY - 1) / kTY, nz); }

size_t column_smem_bytes(int nk) { return (size_t)kColArrays * (nk + 2) * kTX * sizeof(float); }

bool check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        gm1b_set_error("%s: %s", what, cudaGetErrorString(e));
        return false;
    }
    return true;
}

int schedule(float dt, int nsound, int nrk, int *nloop, float *dts) {
    if (nsound < 4 || (nsound % 2) != 0 || nrk < 1 || nrk > 3) return -1;
    if (nrk == 1) {
        int n = (int)floorf((float)nsound / 3.0f + 0.5f);
        float den = (float)n * 3.0f;
        float dd = dt / den;
        const float target = dt / (float)nsound;
        if (dd > target) {
            n += 1;
            den = (float)n * 3.0f;
            dd = dt / den;
        }
        *nloop = n;
        *dts = dd;
    } else if (nrk == 2) {
        *nloop = nsound / 2;
        *dts = dt / (float)nsound;
    } else {
        *nloop = nsound;
        *dts = dt / (float)nsound;
    }
    return 0;
}

bool prepare_column_kernel(int nk) {
    const size_t bytes = column_smem_bytes(nk);
    if (bytes > 227 * 1024) {
        gm1b_set_error("nk=%d exceeds the column kernel's shared-memory capacity", nk);
        return false;
    }
    // set once per device (and again only for a larger need), so a call
    // under stream capture makes no attribute call
    static size_t configured[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess && dev >= 0 && dev < 64 && configured[dev] >= bytes) return true;
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(sound_column_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) {
        gm1b_set_error("cudaFuncSetAttribute(sound_column_kernel): %s", cudaGetErrorString(e));
        return false;
    }
    if (dev >= 0 && dev < 64) configured[dev] = bytes;
    return true;
}

// Whether the fused stage kernel can run this stage: benchmark path (no
// scratch outputs, multi-launch not forced), at least two small steps, the
// stage state within one CTA's shared memory, every row-tile CTA co-resident
// (cooperative launch), and an 8-byte aligned barrier word.  Attributes are
// set once per device.
bool fused_stage_eligible(const Arr &a, const Dims &d, int nloop, uint32_t flags) {
    if ((flags & (GM1B_FLAG_SCRATCH_OUTPUTS | GM1B_FLAG_MULTI_LAUNCH_STAGE)) != 0 || nloop < 2) return false;
    if ((reinterpret_cast<uintptr_t>(a.tri_residual) & 7u) != 0) return false;
    // the kernel's fixed-trip loops cover (kFusedMaxNk + 1) levels
    static_assert(34 * (kFusedMaxNk + 1) <= kLoadTrips * kFusedThreads, "stage-load trips");
    static_assert(kFusedMaxNk + 1 <= kLoadTrips * kColWarps, "level trips");
    if (d.nk > kFusedMaxNk) return false;
    const size_t bytes = fused_smem_floats(d.nk) * sizeof(float);
    if (bytes > 227 * 1024) return false;
    static int capacity[64] = {};  // co-resident CTAs per device, -1 = unusable
    static size_t configured[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    if (configured[dev] < bytes) {
        int coop = 0, sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaError_t e =
            cudaFuncSetAttribute(sound_stage_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sound_stage_fused_kernel, kFusedThreads, bytes);
        if (e != cudaSuccess || !coop) {
            cudaGetLastError();
            capacity[dev] = -1;
        } else {
            capacity[dev] = per_sm * sms;
        }
        configured[dev] = bytes;
    }
    const long long ctas = (long long)((d.ni + kTX - 1) / kTX) * d.nj;
    return capacity[dev] > 0 && ctas <= capacity[dev];
}

int launch_fused_stage(const Arr &a, const Dims &d, const FusedArgs &p, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((d.ni + kTX - 1) / kTX, d.nj);
    cfg.blockDim = dim3(kTX, kColWarps);
    cfg.dynamicSmemBytes = fused_smem_floats(d.nk) * sizeof(float);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    ProfScope ps_("sound_stage_fused_kernel", st);
    cudaError_t e = cudaLaunchKernelEx(&cfg, sound_stage_fused_kernel, a, d, p);
    ps_.stop();
    if (e != cudaSuccess) {
        cudaGetLastError();
        gm1b_set_error("sound_stage_fused_kernel (cooperative launch): %s", cudaGetErrorString(e));
        return GM1B_ERR_CUDA;
    }
    return check_launch("sound_stage_fused_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

// Per-call control of the fused stage's grid barrier: the spin limit, the
// caller's status word, and whether a fused stage of this call has run yet.
struct BarrierControl {
    int spin_limit = kSpinLimit;
    int32_t *status = nullptr;
    bool fused_seen = false;
};

// One acoustic RK stage; returns nloop, or a negative status.
int enqueue_sound_stage(const Arr &a, const Dims &d, float dt, int nsound, int nrk, float rdx, float rdy, float rdz,
                        float cp, float alph, float kdiv, uint32_t flags, int trajectory, int post_ppx,
                        BarrierControl &bc, cudaStream_t st) {
    const int scratch_outputs = (flags & GM1B_FLAG_SCRATCH_OUTPUTS) ? 1 : 0;
    int nloop;
    float dts;
    if (schedule(dt, nsound, nrk, &nloop, &dts) != 0) {
        gm1b_set_error("invalid acoustic schedule: nsound=%d (even, >= 4 required), nrk=%d", nsound, nrk);
        return GM1B_ERR_SCHEDULE;
    }
    const float beta = 1.0f - alph;
    const float asq = alph * alph;
    const bool fused = fused_stage_eligible(a, d, nloop, flags);
    const int fused_reset = fused ? (bc.fused_seen ? 1 : 2) : 0;
    if (fused) bc.fused_seen = true;
    {
            ProfScope ps_("sound_prep_kernel", st);
            sound_prep_kernel<<<box_grid(d.ni + 2, d.nj + 2, d.nk + 2), dim3(kTX, kTY), 0, st>>>(a, d, nrk, dts, rdz, cp, beta,
                                                                                        scratch_outputs, fused_reset);
            ps_.stop();
        }
    if (!check_launch("sound_prep_kernel")) return GM1B_ERR_CUDA;
    const float tem1x = (rdx * cp) * 0.5f;
    const float tem2y = (rdy * cp) * 0.5f;
    if (fused) {
        FusedArgs f;
        f.nrk = nrk;
        f.nloop = nloop;
        f.dts = dts;
        f.rdx = rdx;
        f.rdy = rdy;
        f.alph = alph;
        f.beta = beta;
        f.asq = asq;
        f.kdiv = kdiv;
        f.smeps = kSmeps;
        f.temx = (dts * 0.5f) * rdx;
        f.temy = (dts * 0.5f) * rdy;
        f.rnloop = 1.0f / (float)nloop;
        f.tem1x = tem1x;
        f.tem2y = tem2y;
        f.tavg = 1.0f / (float)nloop;
        f.fill_pp3d = (nrk < 3) || trajectory;
        f.post_ppx = post_ppx;
        f.spin_limit = bc.spin_limit;
        f.status = bc.status;
        const int r = launch_fused_stage(a, d, f, st);
        return r < 0 ? r : nloop;
    }
    ColumnArgs p;
    p.nrk = nrk;
    p.nloop = nloop;
    p.dts = dts;
    p.rdx = rdx;
    p.rdy = rdy;
    p.alph = alph;
    p.beta = beta;
    p.asq = asq;
    p.kdiv = kdiv;
    p.smeps = kSmeps;
    p.temx = (dts * 0.5f) * rdx;
    p.temy = (dts * 0.5f) * rdy;
    p.rnloop = 1.0f / (float)nloop;
    p.scratch_outputs = scratch_outputs;
    p.fill_pp3d = (nrk < 3) || trajectory;
    p.post_ppx = post_ppx;
    const float tavg = 1.0f / (float)nloop;
    const dim3 col_grid((d.ni + kTX - 1) / kTX, d.nj);
    const size_t smem = column_smem_bytes(d.nk);
    for (int n = 1; n <= nloop; ++n) {
        const int last = n == nloop;
        {
                    ProfScope ps_("sound_uv_kernel", st);
                    sound_uv_kernel<<<box_grid(d.ni + 2, d.nj + 2, d.nk), dim3(kTX, kTY), 0, st>>>(a, d, dts, tem1x, tem2y, last,
                                                                                      tavg);
                    ps_.stop();
                }
        if (!check_launch("sound_uv_kernel")) return GM1B_ERR_CUDA;
        p.n = n;
        p.store_consts = (!scratch_outputs && n == 1) ? 1 : 0;
        p.use_consts = (!scratch_outputs && n > 1) ? 1 : 0;
        {
                    ProfScope ps_("sound_column_kernel", st);
                    sound_column_kernel<<<col_grid, dim3(kTX, kColWarps), smem, st>>>(a, d, p);
                    ps_.stop();
                }
        if (!check_launch("sound_column_kernel")) return GM1B_ERR_CUDA;
    }
    return nloop;
}

bool arrays_present(const Arr *a, bool trajectory) {
    const float *const *p = reinterpret_cast<const float *const *>(a);
    const size_t n = trajectory ? sizeof(Arr) / sizeof(float *) : 47;
    for (size_t q = 0; q < n; ++q)
        if (p[q] == nullptr) {
            gm1b_set_error("array #%zu of gm1b_periodic_arrays is NULL", q);
            return false;
        }
    return true;
}

}  // namespace
}  // namespace gm1b

using namespace gm1b;

extern "C" int32_t gm1b_sound3_stage_schedule(float dt, int32_t nsound, int32_t nrk, int32_t *nloop, float *dts) {
    if (nloop == nullptr || dts == nullptr) {
        gm1b_set_error("gm1b_sound3_stage_schedule: NULL output pointer");
        return GM1B_ERR_ARGUMENT;
    }
    int n;
    float s;
    if (schedule(dt, nsound, nrk, &n, &s) != 0) {
        gm1b_set_error("invalid acoustic schedule: nsound=%d (even, >= 4 required), nrk=%d", nsound, nrk);
        return GM1B_ERR_SCHEDULE;
    }
    *nloop = n;
    *dts = s;
    return GM1B_OK;
}

extern "C" float gm1b_rk_stage_dt(float dt, int32_t nrk) {
    if (nrk < 1 || nrk > 3) return __builtin_nanf("");
    return dt / (float)(4 - nrk);
}

namespace {
// Barrier control of one call: spin_limit <= 0 takes the default; the status
// word (when given) is cleared on the stream before the call's first launch.
bool barrier_control(BarrierControl *bc, int32_t spin_limit, int32_t *status_dev, cudaStream_t st) {
    bc->spin_limit = spin_limit > 0 ? spin_limit : kSpinLimit;
    bc->status = status_dev;
    if (status_dev != nullptr) {
        const cudaError_t e = cudaMemsetAsync(status_dev, 0, sizeof(int32_t), st);
        if (e != cudaSuccess) {
            cudaGetLastError();
            gm1b_set_error("cudaMemsetAsync (barrier status word): %s", cudaGetErrorString(e));
            return false;
        }
    }
    return true;
}
}  // namespace

extern "C" int32_t gm1b_sound3_periodic_three_stage_checked(int32_t ni, int32_t nj, int32_t nk,
                                                           const gm1b_periodic_arrays *arrays, float dt,
                                                           int32_t nsound, float rdx, float rdy, float rdz, float cp,
                                                           float alph, float kdiv, uint32_t flags, int32_t spin_limit,
                                                           int32_t *status_dev, void *stream) {
    if (arrays == nullptr || ni < 3 || nj < 3 || nk < 3) {
        gm1b_set_error("gm1b_sound3_periodic_three_stage: need arrays and ni, nj, nk >= 3");
        return GM1B_ERR_ARGUMENT;
    }
    if (!arrays_present(arrays, false)) return GM1B_ERR_ARGUMENT;
    if (!prepare_column_kernel(nk)) return GM1B_ERR_CUDA;
    const Dims d{ni, nj, nk};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    BarrierControl bc;
    if (!barrier_control(&bc, spin_limit, status_dev, st)) return GM1B_ERR_CUDA;
    for (int nrk = 1; nrk <= 3; ++nrk) {
        int r = enqueue_sound_stage(*arrays, d, dt, nsound, nrk, rdx, rdy, rdz, cp, alph, kdiv, flags, 0, 0, bc, st);
        if (r < 0) return r;
    }
    return GM1B_OK;
}

extern "C" int32_t gm1b_sound3_periodic_three_stage(int32_t ni, int32_t nj, int32_t nk,
                                                   const gm1b_periodic_arrays *arrays, float dt, int32_t nsound,
                                                   float rdx, float rdy, float rdz, float cp, float alph, float kdiv,
                                                   uint32_t flags, void *stream) {
    return gm1b_sound3_periodic_three_stage_checked(ni, nj, nk, arrays, dt, nsound, rdx, rdy, rdz, cp, alph, kdiv,
                                                    flags, 0, nullptr, stream);
}

extern "C" int32_t gm1b_psolver3_trajectory(int32_t ni, int32_t nj, int32_t nk, const gm1b_periodic_arrays *arrays,
                                           int32_t steps, float dt, int32_t nsound, float dx, float dy, float dz,
                                           uint32_t ablations, uint32_t flags, void *stream) {
    return gm1b_psolver3_trajectory_checked(ni, nj, nk, arrays, steps, dt, nsound, dx, dy, dz, ablations, flags, 0,
                                            nullptr, stream);
}

extern "C" int32_t gm1b_psolver3_trajectory_checked(int32_t ni, int32_t nj, int32_t nk,
                                                   const gm1b_periodic_arrays *arrays, int32_t steps, float dt,
                                                   int32_t nsound, float dx, float dy, float dz, uint32_t ablations,
                                                   uint32_t flags, int32_t spin_limit, int32_t *status_dev,
                                                   void *stream) {
    if (arrays == nullptr || ni < 5 || nj < 5 || nk < 6 || steps < 1) {
        gm1b_set_error("gm1b_psolver3_trajectory: need arrays, ni >= 5, nj >= 5, nk >= 6, steps >= 1");
        return GM1B_ERR_ARGUMENT;
    }
    if ((double)(nk + 2) * (nj + 2) * (ni + 2) >= 2147483647.0) {
        gm1b_set_error("gm1b_psolver3_trajectory: arrays of 2^31 or more words are not supported");
        return GM1B_ERR_ARGUMENT;
    }
    if (!(dt > 0.0f) || !(dx > 0.0f) || !(dy > 0.0f) || !(dz > 0.0f)) {
        gm1b_set_error("gm1b_psolver3_trajectory: dt, dx, dy, dz must be finite and positive");
        return GM1B_ERR_ARGUMENT;
    }
    for (int nrk = 1; nrk <= 3; ++nrk) {
        int n;
        float s;
        if (schedule(dt, nsound, nrk, &n, &s) != 0) {
            gm1b_set_error("invalid acoustic schedule: nsound=%d (even, >= 4 required)", nsound);
            return GM1B_ERR_SCHEDULE;
        }
    }
    if (!arrays_present(arrays, true)) return GM1B_ERR_ARGUMENT;
    if (!prepare_column_kernel(nk)) return GM1B_ERR_CUDA;
    const Arr &a = *arrays;
    const Dims d{ni, nj, nk};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    BarrierControl bc;
    if (!barrier_control(&bc, spin_limit, status_dev, st)) return GM1B_ERR_CUDA;
    const float rdx = 1.0f / dx, rdy = 1.0f / dy, rdz = 1.0f / dz;
    const int advect = !(ablations & GM1B_ABLATE_MOMENTUM_ADVECTION);
    const int buoy = !(ablations & GM1B_ABLATE_BUOYANCY);
    const int theta_adv = !(ablations & GM1B_ABLATE_SCALAR_ADVECTION);
    const int base_theta = !(ablations & GM1B_ABLATE_BASE_THETA_ADVECTION);
    const int post_ppx = !(ablations & GM1B_ABLATE_POST_STEP_PPX);
    const int promote = !(ablations & GM1B_ABLATE_CARRIER_PROMOTION);
    // tendencies whose halo words stay zero (the twin zero-fills them every
    // stage and never writes their halos)
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMemsetAsync(a.ppten, 0, d.scalar_words() * sizeof(float), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.thten, 0, d.scalar_words() * sizeof(float), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.uten, 0, d.u_words() * sizeof(float), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.vten, 0, d.v_words() * sizeof(float), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.wten, 0, d.w_words() * sizeof(float), st);
    if (e != cudaSuccess) {
        gm1b_set_error("cudaMemsetAsync: %s", cudaGetErrorString(e));
        return GM1B_ERR_CUDA;
    }
    const dim3 blk(kTX, kTY);
    const dim3 g_box = box_grid(ni + 2, nj + 2, nk + 2);
    const dim3 g_mom = box_grid(ni + 1, nj + 1, nk);
    for (int step = 0; step < steps; ++step) {
        for (int nrk = 1; nrk <= 3; ++nrk) {
            {
                            ProfScope ps_("traj_prepare_kernel", st);
                            traj_prepare_kernel<<<g_box, blk, 0, st>>>(a, d, rdx, rdy, rdz);
                            ps_.stop();
                        }
            if (!check_launch("traj_prepare_kernel")) return GM1B_ERR_CUDA;
            {
                            ProfScope ps_("traj_momentum_kernel", st);
                            traj_momentum_kernel<<<g_mom, blk, 0, st>>>(a, d, rdx, rdy, rdz, advect, buoy);
                            ps_.stop();
                        }
            if (!check_launch("traj_momentum_kernel")) return GM1B_ERR_CUDA;
            int r = enqueue_sound_stage(a, d, dt, nsound, nrk, rdx, rdy, rdz, kCp, kAlph, kKdiv, flags, 1,
                                        post_ppx, bc, st);
            if (r < 0) return r;
            {
                            ProfScope ps_("traj_theta_prep_kernel", st);
                            traj_theta_prep_kernel<<<g_box, blk, 0, st>>>(a, d, base_theta);
                            ps_.stop();
                        }
            if (!check_launch("traj_theta_prep_kernel")) return GM1B_ERR_CUDA;
            const float dttmp = dt / (float)(4 - nrk);
            {
                            ProfScope ps_("traj_theta_kernel", st);
                            traj_theta_kernel<<<g_box, blk, 0, st>>>(a, d, rdx, rdy, rdz, dttmp, theta_adv);
                            ps_.stop();
                        }
            if (!check_launch("traj_theta_kernel")) return GM1B_ERR_CUDA;
        }
        if (promote) {
            const struct {
                float *dst;
                const float *src;
                size_t n;
            } copies[5] = {{a.ua, a.u3d, d.u_words()},
                           {a.va, a.v3d, d.v_words()},
                           {a.wa, a.w3d, d.w_words()},
                           {a.ppi, a.pp3d, d.scalar_words()},
                           {a.tha, a.th3d, d.scalar_words()}};
            for (const auto &cp : copies) {
                e = cudaMemcpyAsync(cp.dst, cp.src, cp.n * sizeof(float), cudaMemcpyDeviceToDevice, st);
                if (e != cudaSuccess) {
                    gm1b_set_error("cudaMemcpyAsync (carrier promotion): %s", cudaGetErrorString(e));
                    return GM1B_ERR_CUDA;
                }
            }
        }
    }
    return GM1B_OK;
}
