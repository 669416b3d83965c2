// terrain_open.cu - sm_100a kernels of the terrain + all-open psolver=3
// acoustic RK stage on the padded (ng = 3) lane.
//
// Behaviour followed (reference file:line):
//   cpu_psolver3_terrain_open_stage_inplace   src/cm1core/cuda_psolver3_terrain_open.py:774-894
//     (_prepare_coefficients :300, _terrain_pressure_gradient :393,
//      _transformed_velocity_terms :482, _initial_fpk :544,
//      _pressure_advection :595, _implicit_and_pressure_update :678,
//      _average_velocities :748)
//   cpu_ssopen_terrain_all_inplace, _interp_u_at_w, cpu_bcwsfc_terrain_physical_inplace
//                                             src/cm1core/cuda_terrain_open_boundary.py:666-850
//   terrain_coordinate_profiles (uniform)     :486-560
//   cpu_bc{p,s,u,v,w}_open_inplace            src/cm1core/cuda_sound3_open_boundary.py:249-335
//   cpu_radiation4_inplace                    src/cm1core/cuda_lateral_closure.py:390-472
//
// Design (B200).  Per stage: one prepare pass.  Per small step: three
// launches - (1) the four open edges (a CTA per boundary line snapshots both
// w-level interpolations of its two face columns in shared memory, then
// advances every level at once), (2) the terrain pressure gradient on the
// interior faces (a 32x4 tile marching up the column, each vertical ppd
// difference formed once), (3) one column pass per 32 columns of a row that
// keeps the whole column in shared memory: transformed divergence, surface
// w, pi' advection and fpk, the tridiagonal coefficients, the Thomas sweep,
// the pi' update with the kdiv filter, the ppd halo copy between small steps
// and the rru/rrv/rrw averages (the reference takes eight launches and
// global elimination scratch for the same small step).  After the last small
// step: the radiation histories (one warp per boundary line, the column sum
// in level order) and the stage fills in two ordered passes (the first
// direction of every fill, then the second).  Scratch arrays are written only
// at the last small step, and only under GM1B_TOS_DIAGNOSTICS: their final
// words are the CPU twin's.  The vertical coordinate is formed in-kernel with
// the twin's own float32 operations.  Binary32 one operation at a time in the
// reference's order: word-identical.
#include "gm1b_common.cuh"

namespace gm1b {
namespace {

constexpr int kTosWarps = 8;     // k-parallel warps of the column pass
constexpr int kTosMaxNk = 160;   // column pass keeps 10 words per level per column in shared memory
constexpr int kTosArrays = 7;
constexpr int kPgLevels = 4;     // levels whose loads the pressure-gradient march issues together
constexpr int kA2Levels = 2;     // levels per warp whose column-pass loads are issued together (phase A2)
constexpr int kColLevels = 2;    // the same for phases A3 and C
constexpr int kThomasChunk = 8;  // back-substitution levels whose coefficients are read together

struct TosArgs {
    gm1b_terrain_open_arrays a;
    gm1b_terrain_metrics m;
    int ni, nj, nk, nrk, n, nloop;
    unsigned abl, diag;
    float dts, rdx, rdy, dz, alph, beta, asq, kdiv, temx, temy, tavg, zt, rzt, halfcp;
    float cgs[3], cgt[3];
    // the stretched terrain column (vmode 1): CM1-indexed sigma (nk+2),
    // sigmaf (nk+3), rds (nk+2), rdsf (nk+3) and the source-valid padded base
    // density (nk+2, nj+6, ni+6); unused on the uniform column (vmode 0)
    int vmode;
    const float *sgm, *sgmf, *rdsp, *rdsfp, *rho0p;
    // the flat stretched column (vmode 2): mh (nk+2), mf (nk+3), rdz and the
    // packed lateral code wbc | ebc << 4 | sbc << 8 | nbc << 12
    const float *mhp, *mfp;
    float rdz;
    unsigned obc;
};

// 32-bit element offsets: the host refuses grids whose largest padded
// array reaches 2^31 words, so every offset below fits (a 640x768x80 padded
// scalar is 41 M words)
struct Ix {
    int ni, nj;
    __device__ __forceinline__ unsigned p(int k, int j, int i) const {
        return ((unsigned)k * (unsigned)(nj + 2) + (unsigned)j) * (unsigned)(ni + 2) + (unsigned)i;
    }
    __device__ __forceinline__ unsigned u(int k, int y, int x) const {
        return ((unsigned)k * (unsigned)(nj + 6) + (unsigned)y) * (unsigned)(ni + 7) + (unsigned)x;
    }
    __device__ __forceinline__ unsigned v(int k, int y, int x) const {
        return ((unsigned)k * (unsigned)(nj + 7) + (unsigned)y) * (unsigned)(ni + 6) + (unsigned)x;
    }
    __device__ __forceinline__ unsigned w(int k, int y, int x) const {
        return ((unsigned)k * (unsigned)(nj + 6) + (unsigned)y) * (unsigned)(ni + 6) + (unsigned)x;
    }
    __device__ __forceinline__ unsigned m(int k0, int j0, int i0) const {
        return ((unsigned)k0 * (unsigned)nj + (unsigned)j0) * (unsigned)ni + (unsigned)i0;
    }
    __device__ __forceinline__ unsigned h(int j0, int i0) const { return (unsigned)j0 * (unsigned)ni + (unsigned)i0; }
};

// uniform terrain coordinate, the twin's float32 words (terrain_coordinate_profiles)
__device__ __forceinline__ float sig(int k, float dz) { return ((float)k - 0.5f) * dz; }
__device__ __forceinline__ float sigf(int k, float dz) { return (float)(k - 1) * dz; }
__device__ __forceinline__ float rds(int k, float dz) { return rcp_rn(sig(k, dz) - sig(k - 1, dz)); }
__device__ __forceinline__ float rdsf(int k, float dz) { return rcp_rn(sigf(k + 1, dz) - sigf(k, dz)); }

// The column's vertical coordinate: formed in-kernel on the uniform column
// (VM 0), read from the bound profiles at CM1's indices on the stretched
// terrain column (VM 1): rds(dz) -> rds[k] / rdsf[k], sig/sigf -> sigma /
// sigmaf, the lid nk*dz -> ztop (cuda_gm1_child_psolver3_open.py:152-280)
template <int VM> __device__ __forceinline__ float col_rds(const TosArgs &p, int k) {
    return VM ? __ldg(p.rdsp + k) : rds(k, p.dz);
}
template <int VM> __device__ __forceinline__ float col_rdsf(const TosArgs &p, int k) {
    return VM ? __ldg(p.rdsfp + k) : rdsf(k, p.dz);
}
template <int VM> __device__ __forceinline__ float col_sigf(const TosArgs &p, int kf) {
    return VM ? __ldg(p.sgmf + kf) : sigf(kf, p.dz);
}
// r2 of the face-to-level interpolation r2*q(kf) + (1-r2)*q(kf-1)
template <int VM> __device__ __forceinline__ float col_r2(const TosArgs &p, int kf) {
    return VM ? (__ldg(p.sgmf + kf) - __ldg(p.sgm + kf - 1)) * __ldg(p.rdsp + kf)
              : (sigf(kf, p.dz) - sig(kf - 1, p.dz)) * rds(kf, p.dz);
}
__device__ __forceinline__ float vrds(const TosArgs &p, int k) { return p.vmode ? col_rds<1>(p, k) : col_rds<0>(p, k); }
__device__ __forceinline__ float vrdsf(const TosArgs &p, int k) {
    return p.vmode ? col_rdsf<1>(p, k) : col_rdsf<0>(p, k);
}
__device__ __forceinline__ float vr2(const TosArgs &p, int kf) { return p.vmode ? col_r2<1>(p, kf) : col_r2<0>(p, kf); }

// numpy.minimum / numpy.maximum: NaN propagates, a tie returns the second
__device__ __forceinline__ float np_min(float a, float b) { return a != a ? a : (b != b ? b : (a < b ? a : b)); }
__device__ __forceinline__ float np_max(float a, float b) { return a != a ? a : (b != b ? b : (a > b ? a : b)); }

// ---------------------------------------------------------------------------
// stage start: coefficients, carriers, accumulators (and scratch zeroing)
// one thread per (k = 1..nk, j = 0..nj+1, i = 0..ni+1)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) tos_prepare_kernel(TosArgs p) {
    const Ix X{p.ni, p.nj};
    const int ni = p.ni, nj = p.nj, nk = p.nk;
    const size_t plane = (size_t)(nj + 2) * (ni + 2), total = plane * nk;
    const gm1b_terrain_open_arrays &a = p.a;
    const gm1b_terrain_metrics &m = p.m;
    for (size_t z = (size_t)blockIdx.x * blockDim.x + threadIdx.x; z < total; z += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(z % (ni + 2));
        const int j = (int)((z / (ni + 2)) % (nj + 2));
        const int k = (int)(z / plane) + 1;
        const unsigned c = X.p(k, j, i);
        a.ppd[c] = a.ppx[c];
        if (p.nrk != 1) a.pp3d[c] = a.ppi[c];
        const int y = j + 2, x = i + 2;
        const unsigned qu = X.u(k, y, x), qv = X.v(k, y, x), qw = X.w(k, y, x);
        a.rru[qu] = 0.0f;
        a.rrv[qv] = 0.0f;
        a.rrw[qw] = a.wa[qw] * p.beta;
        if (p.nrk != 1) {
            a.u3d[qu] = a.ua[qu];
            a.v3d[qv] = a.va[qv];
            a.w3d[qw] = a.wa[qw];
        }
        const bool phys = j >= 1 && j <= nj && i >= 1 && i <= ni;
        if (phys && p.vmode == 2) {
            // sound.F:119-143 on the flat column: rdz*mh(k), rdz*mf(k) and the
            // base state at CM1's (1,1,k); mm at every level
            // (cuda_gm1_child_psolver3_open.py:374-385)
            const float t0 = (p.dts * p.rdz) * __ldg(p.mhp + k);
            const float rr = m.rr0[X.m(k - 1, 0, 0)];
            const float r2 = (t0 * rr) * m.rf0[X.m(k, 0, 0)];
            const float r1 = (t0 * rr) * m.rf0[X.m(k - 1, 0, 0)];
            const float tem1 = ((p.dts * p.rdz) * 1005.7f) * __ldg(p.mfp + k);
            const float c1a = m.c1[X.m(k - 1, 0, 0)], c1b = m.c1[X.m(k, 0, 0)];
            const float c2a = m.c2[X.m(k - 1, 0, 0)], c2b = m.c2[X.m(k, 0, 0)];
            const float pc = a.piadv[c];
            a.qk[c] = t0 * a.ppterm[c];
            a.pk2[c] = k == nk ? 0.0f : r2 * ((-c2b) * a.piadv[X.p(k + 1, j, i)] + (1.0f - c1b) * pc);
            a.pk1[c] = k == 1 ? 0.0f : r1 * (c1a * a.piadv[X.p(k - 1, j, i)] + (c2a - 1.0f) * pc);
            a.mm[c] = tem1 * (c2a * a.thv[c] + c1a * a.thv[X.p(k - 1, j, i)]);
        } else if (phys) {
            const int j0 = j - 1, i0 = i - 1;
            const float gz = m.gz[X.h(j0, i0)];
            const float tem = p.dts * vrdsf(p, k);
            a.qk[c] = (tem * a.ppterm[c]) * gz;
            const float tem2 = ((p.dts * gz) * vrdsf(p, k)) * m.rr0[X.m(k - 1, j0, i0)];
            const float pc = a.piadv[c];
            const float b2 = (-m.c2[X.m(k, j0, i0)]) * a.piadv[X.p(k + 1, j, i)] + (1.0f - m.c1[X.m(k, j0, i0)]) * pc;
            const float b1 = m.c1[X.m(k - 1, j0, i0)] * a.piadv[X.p(k - 1, j, i)] + (m.c2[X.m(k - 1, j0, i0)] - 1.0f) * pc;
            a.pk2[c] = k == nk ? 0.0f : (tem2 * m.rf0[X.m(k, j0, i0)]) * b2;
            a.pk1[c] = k == 1 ? 0.0f : (tem2 * m.rf0[X.m(k - 1, j0, i0)]) * b1;
            float mmv = 0.0f;
            if (k >= 2) {
                const float tem1 = (p.dts * vrds(p, k)) * 1005.7f;
                const float th = m.c2[X.m(k - 1, j0, i0)] * a.thv[c] + m.c1[X.m(k - 1, j0, i0)] * a.thv[X.p(k - 1, j, i)];
                mmv = (tem1 * th) * gz;
            }
            if (k >= 2 || p.diag) a.mm[c] = mmv;
        }
        if (p.diag) {
            float *zero[] = {a.fpk, a.divh, a.hadvp, a.dum3, a.elim_c, a.elim_d, a.tri_aa, a.tri_bb, a.tri_cc,
                             a.tri_dd, a.tri_pivot, a.tri_residual, a.qk, a.pk1, a.pk2, a.mm};
            const int nz = phys ? 12 : 16;  // the coefficients of a live cell were just written
#pragma unroll 1
            for (int q = 0; q < nz; ++q) zero[q][c] = 0.0f;
            if (k == 1 || k == nk) {
                const unsigned e = X.p(k == 1 ? 0 : nk + 1, j, i);
#pragma unroll 1
                for (int q = 0; q < 16; ++q) zero[q][e] = 0.0f;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// open-side normal velocity (ssopenbc*): one CTA per boundary line
// lines: [0, nj) west, [nj, 2nj) east, [2nj, 2nj+ni) south, [.., 2nj+2ni) north
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) tos_edge_kernel(TosArgs p) {
    extern __shared__ float sh[];
    const Ix X{p.ni, p.nj};
    const int ni = p.ni, nj = p.nj, nk = p.nk, L = nk + 2;
    float *q0 = sh, *q1 = sh + L, *s0 = sh + 2 * L, *s1 = sh + 3 * L;
    const gm1b_terrain_open_arrays &a = p.a;
    const gm1b_terrain_metrics &m = p.m;
    int line = blockIdx.x, side;
    if (line < nj) side = 0;
    else if (line < 2 * nj) side = 1, line -= nj;
    else if (line < 2 * nj + ni) side = 2, line -= 2 * nj;
    else side = 3, line -= 2 * nj + ni;
    const bool ew = side < 2;
    // face columns: q0 at (y0, x0), q1 at (y1, x1); the updated one is q0
    // on the west/south side and q1 on the east/north side
    int y0, x0, y1, x1;
    if (side == 0) y0 = y1 = line + 3, x0 = 3, x1 = 4;
    else if (side == 1) y0 = y1 = line + 3, x0 = ni + 2, x1 = ni + 3;
    else if (side == 2) x0 = x1 = line + 3, y0 = 3, y1 = 4;
    else x0 = x1 = line + 3, y0 = nj + 2, y1 = nj + 3;
    const float *q = ew ? a.u3d : a.v3d;
    for (int k = 1 + threadIdx.x; k <= nk; k += blockDim.x) {
        q0[k] = q[ew ? X.u(k, y0, x0) : X.v(k, y0, x0)];
        q1[k] = q[ew ? X.u(k, y1, x1) : X.v(k, y1, x1)];
    }
    __syncthreads();
    for (int kf = 1 + threadIdx.x; kf <= nk + 1; kf += blockDim.x) {
        float r0, r1v;
        if (kf == 1) {
            r0 = (p.cgs[0] * q0[1] + p.cgs[1] * q0[2]) + p.cgs[2] * q0[3];
            r1v = (p.cgs[0] * q1[1] + p.cgs[1] * q1[2]) + p.cgs[2] * q1[3];
        } else if (kf == nk + 1) {
            r0 = (p.cgt[0] * q0[nk] + p.cgt[1] * q0[nk - 1]) + p.cgt[2] * q0[nk - 2];
            r1v = (p.cgt[0] * q1[nk] + p.cgt[1] * q1[nk - 1]) + p.cgt[2] * q1[nk - 2];
        } else {
            const float r2 = vr2(p, kf);
            const float r1 = 1.0f - r2;
            r0 = r1 * q0[kf - 1] + r2 * q0[kf];
            r1v = r1 * q1[kf - 1] + r2 * q1[kf];
        }
        s0[kf] = r0;
        s1[kf] = r1v;
    }
    __syncthreads();
    const int j0 = ew ? line : (side == 2 ? 0 : nj - 1);   // metric row of the edge cell
    const int i0 = ew ? (side == 0 ? 0 : ni - 1) : line;   // metric column of the edge cell
    const float gz = m.gz[X.h(j0, i0)];
    float rg0, rg1, hmet, rd;
    const float *gmet;
    const float *rad;
    const float *ten;
    if (side == 0) rg0 = m.rgzu[(size_t)j0 * (ni + 1)], rg1 = m.rgzu[(size_t)j0 * (ni + 1) + 1], hmet = a.uh[3];
    else if (side == 1) rg0 = m.rgzu[(size_t)j0 * (ni + 1) + ni - 1], rg1 = m.rgzu[(size_t)j0 * (ni + 1) + ni], hmet = a.uh[ni + 2];
    else if (side == 2) rg0 = m.rgzv[i0], rg1 = m.rgzv[(size_t)ni + i0], hmet = a.vh[3];
    else rg0 = m.rgzv[(size_t)(nj - 1) * ni + i0], rg1 = m.rgzv[(size_t)nj * ni + i0], hmet = a.vh[nj + 2];
    rd = ew ? p.rdx : p.rdy;
    gmet = ew ? m.gx : m.gy;
    rad = side == 0 ? a.radbcw : side == 1 ? a.radbce : side == 2 ? a.radbcs : a.radbcn;
    ten = ew ? a.uten : a.vten;
    const bool upd0 = side == 0 || side == 2;
    const int yu = upd0 ? y0 : y1, xu = upd0 ? x0 : x1;
    const size_t radstride = ew ? (size_t)(nj + 6) : (size_t)(ni + 6);
    const int radpos = ew ? yu : xu;
    float *qout = ew ? a.u3d : a.v3d;
    for (int k = 1 + threadIdx.x; k <= nk; k += blockDim.x) {
        float hz = gz * (q1[k] * rg1 - q0[k] * rg0);
        hz = (hz * rd) * hmet;
        float vt = gmet[X.m(k, j0, i0)] * (s1[k + 1] + s0[k + 1]) - gmet[X.m(k - 1, j0, i0)] * (s1[k] + s0[k]);
        vt = (0.5f * vt) * vrdsf(p, k);
        const float r = (-rad[(size_t)k * radstride + radpos]) * (hz + vt);
        const size_t o = ew ? X.u(k, yu, xu) : X.v(k, yu, xu);
        const float tnd = r + ten[o];
        qout[o] = (upd0 ? q0[k] : q1[k]) + p.dts * tnd;
    }
}

// ---------------------------------------------------------------------------
// flat column, open-side normal velocity (bc.F:2410-2419 and its three
// twins): one thread per (k, row) of the west/east faces, then per (k,
// column) of the south/north faces; only sides whose code is 2 (open)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) tos_flat_edge_kernel(TosArgs p) {
    const Ix X{p.ni, p.nj};
    const int ni = p.ni, nj = p.nj, nk = p.nk;
    const gm1b_terrain_open_arrays &a = p.a;
    const unsigned we = (unsigned)nk * (unsigned)nj, total = we + (unsigned)nk * (unsigned)ni;
    for (unsigned z = blockIdx.x * blockDim.x + threadIdx.x; z < total; z += gridDim.x * blockDim.x) {
        if (z < we) {
            const int k = (int)(z / (unsigned)nj) + 1, y = (int)(z % (unsigned)nj) + 3;
            const size_t r = (size_t)k * (nj + 6) + y;
            if ((p.obc & 15u) == 2u) {
                const unsigned b = X.u(k, y, 3);
                const float t = (((-a.radbcw[r]) * (a.u3d[X.u(k, y, 4)] - a.u3d[b])) * p.rdx) * a.uh[3] + a.uten[b];
                a.u3d[b] = a.u3d[b] + p.dts * t;
            }
            if (((p.obc >> 4) & 15u) == 2u) {
                const unsigned b = X.u(k, y, ni + 3);
                const float t =
                    (((-a.radbce[r]) * (a.u3d[b] - a.u3d[X.u(k, y, ni + 2)])) * p.rdx) * a.uh[ni + 2] + a.uten[b];
                a.u3d[b] = a.u3d[b] + p.dts * t;
            }
        } else {
            const unsigned q = z - we;
            const int k = (int)(q / (unsigned)ni) + 1, x = (int)(q % (unsigned)ni) + 3;
            const size_t r = (size_t)k * (ni + 6) + x;
            if (((p.obc >> 8) & 15u) == 2u) {
                const unsigned b = X.v(k, 3, x);
                const float t = (((-a.radbcs[r]) * (a.v3d[X.v(k, 4, x)] - a.v3d[b])) * p.rdy) * a.vh[3] + a.vten[b];
                a.v3d[b] = a.v3d[b] + p.dts * t;
            }
            if (((p.obc >> 12) & 15u) == 2u) {
                const unsigned b = X.v(k, nj + 3, x);
                const float t =
                    (((-a.radbcn[r]) * (a.v3d[b] - a.v3d[X.v(k, nj + 2, x)])) * p.rdy) * a.vh[nj + 2] + a.vten[b];
                a.v3d[b] = a.v3d[b] + p.dts * t;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// flat column pressure gradient (sound.F:318-342): every face i = 1..ni+1,
// j = 1..nj+1 takes u + (dts*dtu0)*(uten - pgrad), dtu0 = 1 on the faces
// param.F:9182-9219 admits (a periodic side's boundary face included), 0
// elsewhere; one thread per (j, i), marching k
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) tos_flat_pgrad_kernel(TosArgs p) {
    const Ix X{p.ni, p.nj};
    const int ni = p.ni, nj = p.nj, nk = p.nk;
    const int i = blockIdx.x * 32 + threadIdx.x + 1;
    const int j = blockIdx.y * 4 + threadIdx.y + 1;
    if (i > ni + 1 || j > nj + 1) return;
    const gm1b_terrain_open_arrays &a = p.a;
    const bool pw = (p.obc & 15u) == 1u, pe = ((p.obc >> 4) & 15u) == 1u;
    const bool ps = ((p.obc >> 8) & 15u) == 1u, pn = ((p.obc >> 12) & 15u) == 1u;
    const float wu = (j <= nj && (i > 1 || pw) && (i < ni + 1 || pe)) ? 1.0f : 0.0f;
    const float wv = (i <= ni && (j > 1 || ps) && (j < nj + 1 || pn)) ? 1.0f : 0.0f;
    const float tem1 = (p.rdx * 1005.7f) * 0.5f, tem2 = (p.rdy * 1005.7f) * 0.5f;
    const float du = p.dts * wu, dv = p.dts * wv;
    for (int k = 1; k <= nk; ++k) {
        const unsigned c = X.p(k, j, i);
        const float pc = __ldg(a.ppd + c), tc = __ldg(a.thv + c);
        float pu = tem1 * (pc - __ldg(a.ppd + X.p(k, j, i - 1)));
        pu = pu * (tc + __ldg(a.thv + X.p(k, j, i - 1)));
        const unsigned xu = X.u(k, j + 2, i + 2);
        a.u3d[xu] = a.u3d[xu] + du * (__ldg(a.uten + xu) - pu);
        float pv = tem2 * (pc - __ldg(a.ppd + X.p(k, j - 1, i)));
        pv = pv * (tc + __ldg(a.thv + X.p(k, j - 1, i)));
        const unsigned xv = X.v(k, j + 2, i + 2);
        a.v3d[xv] = a.v3d[xv] + dv * (__ldg(a.vten + xv) - pv);
    }
}

// ---------------------------------------------------------------------------
// terrain pressure gradient on the interior faces (u faces 2..ni of the
// physical rows, v faces 2..nj of the physical columns).  One thread per
// pressure point (j, i), j = 0..nj+1, i = 0..ni+1, marching k = 1..nk with
// the vertical ppd differences of its own, west and south points carried in
// registers.  Under diagnostics with the pi' advection ablated, the last
// small step leaves those differences in hadvp, as the twin does.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) tos_pgrad_kernel(TosArgs p) {
    const Ix X{p.ni, p.nj};
    const int ni = p.ni, nj = p.nj, nk = p.nk;
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 4 + threadIdx.y;
    if (i > ni + 1 || j > nj + 1) return;
    const gm1b_terrain_open_arrays &a = p.a;
    const gm1b_terrain_metrics &m = p.m;
    const bool du = j >= 1 && j <= nj && i >= 2 && i <= ni;
    const bool dv = j >= 2 && j <= nj && i >= 1 && i <= ni;
    const bool dh = p.diag && p.n == p.nloop && !(p.abl & GM1B_TOS_PRESSURE_ADVECTION);
    if (!du && !dv && !dh) return;
    const int iw = du ? i - 1 : i, js = dv ? j - 1 : j;   // neighbour points (own point when unused)
    float pc = __ldg(a.ppd + X.p(1, j, i)), pw = __ldg(a.ppd + X.p(1, j, iw)), ps = __ldg(a.ppd + X.p(1, js, i));
    float vc = 0.0f, vw = 0.0f, vs = 0.0f;  // vertical difference at level k (zero at k = 1)
    float gxu_lo = du ? __ldg(m.gxu + (size_t)(j - 1) * (ni + 1) + (i - 1)) : 0.0f;
    float gyv_lo = dv ? __ldg(m.gyv + (size_t)(j - 1) * ni + (i - 1)) : 0.0f;
    // Levels go in chunks of kPgLevels: every load of a chunk is issued before
    // its first store, so the chunk's loads are in flight together (the
    // stores to u3d/v3d would otherwise order each level's loads behind the
    // previous level's stores).
    for (int k0 = 1; k0 <= nk; k0 += kPgLevels) {
        float lp[kPgLevels], lw[kPgLevels], ls[kPgLevels], lth[kPgLevels], lthw[kPgLevels], lths[kPgLevels];
        float lgx[kPgLevels], lgy[kPgLevels], lut[kPgLevels], luu[kPgLevels], lvt[kPgLevels], lvv[kPgLevels];
#pragma unroll
        for (int q = 0; q < kPgLevels; ++q) {
            const int k = k0 + q;
            lp[q] = lw[q] = ls[q] = lth[q] = lthw[q] = lths[q] = 0.0f;
            lgx[q] = lgy[q] = lut[q] = luu[q] = lvt[q] = lvv[q] = 0.0f;
            if (k > nk) continue;
            if (k < nk) {
                lp[q] = __ldg(a.ppd + X.p(k + 1, j, i));
                lw[q] = __ldg(a.ppd + X.p(k + 1, j, iw));
                ls[q] = __ldg(a.ppd + X.p(k + 1, js, i));
            }
            lth[q] = __ldg(a.thv + X.p(k, j, i));
            if (du) {
                const unsigned o = X.u(k, j + 2, i + 2);
                lthw[q] = __ldg(a.thv + X.p(k, j, iw));
                lgx[q] = __ldg(m.gxu + ((unsigned)k * (unsigned)nj + (unsigned)(j - 1)) * (unsigned)(ni + 1) + (unsigned)(i - 1));
                lut[q] = __ldg(a.uten + o);
                luu[q] = a.u3d[o];
            }
            if (dv) {
                const unsigned o = X.v(k, j + 2, i + 2);
                lths[q] = __ldg(a.thv + X.p(k, js, i));
                lgy[q] = __ldg(m.gyv + ((unsigned)k * (unsigned)(nj + 1) + (unsigned)(j - 1)) * (unsigned)ni + (unsigned)(i - 1));
                lvt[q] = __ldg(a.vten + o);
                lvv[q] = a.v3d[o];
            }
        }
#pragma unroll
        for (int q = 0; q < kPgLevels; ++q) {
            const int k = k0 + q;
            if (k > nk) break;
            float vc1 = 0.0f, vw1 = 0.0f, vs1 = 0.0f;
            const float pc1 = lp[q], pw1 = lw[q], ps1 = ls[q];
            if (k < nk) {
                const float r = vrds(p, k + 1);
                vc1 = (pc1 - pc) * r;
                vw1 = (pw1 - pw) * r;
                vs1 = (ps1 - ps) * r;
            }
            if (dh && k >= 2) a.hadvp[X.p(k, j, i)] = vc;
            const float thc = lth[q];
            if (du) {
                const float gxu_hi = lgx[q];
                const float th = thc + lthw[q];
                const float hz = (pc - pw) * p.rdx;
                const float vsum = (vc1 + vw1) + (vc + vw);
                const float tr = (0.125f * vsum) * (gxu_lo + gxu_hi);
                const float pg = (p.halfcp * th) * (hz + tr);
                a.u3d[X.u(k, j + 2, i + 2)] = luu[q] + p.dts * (lut[q] - pg);
                gxu_lo = gxu_hi;
            }
            if (dv) {
                const float gyv_hi = lgy[q];
                const float th = thc + lths[q];
                const float hz = (pc - ps) * p.rdy;
                const float vsum = (vc1 + vs1) + (vc + vs);
                const float tr = (0.125f * vsum) * (gyv_lo + gyv_hi);
                const float pg = (p.halfcp * th) * (hz + tr);
                a.v3d[X.v(k, j + 2, i + 2)] = lvv[q] + p.dts * (lvt[q] - pg);
                gyv_lo = gyv_hi;
            }
            pc = pc1, pw = pw1, ps = ps1;
            vc = vc1, vw = vw1, vs = vs1;
        }
    }
}

// ---------------------------------------------------------------------------
// column pass of one small step.  CTA = 32 consecutive columns of row j,
// kTosWarps warps sharing the levels; three CTAs per SM so that one's serial
// Thomas sweep overlaps the others' loads.  Shared memory holds, per level
// and column: the four transformed face velocities (later aa, bb, cc/ec,
// dd), w, fpk and the eliminated right-hand side ed; pk1+qk, pk2-qk and
// pp3d are re-read from global memory (L2-resident) where they are used.
// dum3 and hadvp are formed where they are used (levels k and k+1), with
// the same operations as the twin; read-only fields take the non-coherent
// path so the unrolled level loops keep several levels' loads in flight.
// ---------------------------------------------------------------------------
// global words one level of phase A2 reads (zero where the level or the
// pi' advection does not use them)
struct A2Load {
    float rk, rl, rk1, rrf_k, rrf_k1, qk, pk1, pk2, ppten, ppterm, pc, pe, pw, pn, ps, rr0;
    __device__ __forceinline__ void load(const gm1b_terrain_open_arrays &a, const gm1b_terrain_metrics &m,
                                         const Ix &X, int k, int nk, int j, int i, bool adv, bool flat) {
        rk = rl = rk1 = rrf_k = rrf_k1 = qk = pk1 = pk2 = ppten = ppterm = 0.0f;
        pc = pe = pw = pn = ps = rr0 = 0.0f;
        if (k > nk) return;
        const int j0 = j - 1, i0 = i - 1;
        const unsigned c = X.p(k, j, i);
        if (flat) {  // the flat column's pi' advection reads piadv only
            pc = __ldg(a.piadv + c);
            pe = __ldg(a.piadv + c + 1);
            pw = __ldg(a.piadv + c - 1);
            pn = __ldg(a.piadv + X.p(k, j + 1, i));
            ps = __ldg(a.piadv + X.p(k, j - 1, i));
        } else if (adv) {
            rk = __ldg(m.rho0_3d + X.m(k - 1, 0, 0));
            if (k >= 2) rl = __ldg(m.rho0_3d + X.m(k - 2, 0, 0));
            if (k < nk) rk1 = __ldg(m.rho0_3d + X.m(k, 0, 0));
            if (k >= 2) rrf_k = __ldg(m.rrf0 + X.m(k - 1, j0, i0));
            if (k < nk) rrf_k1 = __ldg(m.rrf0 + X.m(k, j0, i0));
            pc = __ldg(a.piadv + c);
            pe = __ldg(a.piadv + c + 1);
            pw = __ldg(a.piadv + c - 1);
            pn = __ldg(a.piadv + X.p(k, j + 1, i));
            ps = __ldg(a.piadv + X.p(k, j - 1, i));
            rr0 = __ldg(m.rr0 + X.m(k - 1, j0, i0));
        }
        qk = __ldg(a.qk + c);
        pk1 = __ldg(a.pk1 + c);
        pk2 = __ldg(a.pk2 + c);
        ppten = __ldg(a.ppten + c);
        ppterm = __ldg(a.ppterm + c);
    }
};

template <int VM>
__device__ __forceinline__ void tos_level_terms(const float *s_xw, const float *s_xe, const float *s_ys,
                                                const float *s_yn, const float *s_r, int lane, int kf,
                                                const TosArgs &p, float dzdx, float dzdy, float gz, float rk,
                                                float rl, float rrf0, bool adv, float &d3, float &ha) {
    const float r2 = col_r2<VM>(p, kf);
    const float r1 = 1.0f - r2;
    const float height = (col_sigf<VM>(p, kf) - p.zt) * p.rzt;
    const float xw = s_xw[kf * 32 + lane], xe = s_xe[kf * 32 + lane];
    const float xwl = s_xw[(kf - 1) * 32 + lane], xel = s_xe[(kf - 1) * 32 + lane];
    const float ys = s_ys[kf * 32 + lane], yn = s_yn[kf * 32 + lane];
    const float ysl = s_ys[(kf - 1) * 32 + lane], ynl = s_yn[(kf - 1) * 32 + lane];
    {
        const float uh = xw + xe, ul = xwl + xel, vh = ys + yn, vl = ysl + ynl;
        const float xt = (r2 * uh + r1 * ul) * dzdx;
        const float yt = (r2 * vh + r1 * vl) * dzdy;
        d3 = ((0.5f * (xt + yt)) * height) * gz;
    }
    ha = 0.0f;
    if (adv) {
        float uh, ul, vh, vl;
        if (VM) {
            // face-averaged base density times the face velocity, formed in
            // phase A1 (s_r: west, east, south, north arrays of L*32 words)
            const int L32 = (p.nk + 2) * 32, o = kf * 32 + lane, ol = (kf - 1) * 32 + lane;
            uh = s_r[o] + s_r[L32 + o], ul = s_r[ol] + s_r[L32 + ol];
            vh = s_r[2 * L32 + o] + s_r[3 * L32 + o], vl = s_r[2 * L32 + ol] + s_r[3 * L32 + ol];
        } else {
            uh = rk * xw + rk * xe, ul = rl * xwl + rl * xel;
            vh = rk * ys + rk * yn, vl = rl * ysl + rl * ynl;
        }
        const float xt = (r2 * uh + r1 * ul) * dzdx;
        const float yt = (r2 * vh + r1 * vl) * dzdy;
        ha = (((0.5f * (xt + yt)) * height) * gz) * rrf0;
    }
}

template <int VM>
__global__ void __launch_bounds__(32 * kTosWarps, 3) tos_column_kernel(TosArgs p) {
    extern __shared__ float sh[];
    const Ix X{p.ni, p.nj};
    const int ni = p.ni, nj = p.nj, nk = p.nk, L = nk + 2;
    const int lane = threadIdx.x, wy = threadIdx.y;
    const int i = blockIdx.x * 32 + lane + 1;
    const int j = blockIdx.y + 1;
    const bool live = i <= ni;
    const int i0 = i - 1, j0 = j - 1, y = j + 2, x = i + 2;
    const gm1b_terrain_open_arrays &a = p.a;
    const gm1b_terrain_metrics &m = p.m;
    const bool last = p.n == p.nloop;
    const bool dlast = p.diag && last;
    const bool do_div = p.abl & GM1B_TOS_TRANSFORMED_DIVERGENCE;
    const bool do_adv = p.abl & GM1B_TOS_PRESSURE_ADVECTION;
    const bool do_imp = p.abl & GM1B_TOS_IMPLICIT_SOLVE;
    float *s_xw = sh, *s_xe = s_xw + L * 32, *s_ys = s_xe + L * 32, *s_yn = s_ys + L * 32;
    float *s_w = s_yn + L * 32, *s_fpk = s_w + L * 32, *s_ed = s_fpk + L * 32;
    float *s_aa = s_xw, *s_bb = s_xe, *s_cc = s_ys, *s_dd = s_yn;
    // VM 1: the four rho-weighted face velocities (west, east, south, north),
    // read only in phases A1-A2; the west array shares its words with ed,
    // which phase B first writes (three more arrays per level, so two CTAs
    // share an SM at nk = 80)
    float *s_r = s_ed, *s_re = s_r + L * 32, *s_rs = s_re + L * 32, *s_rn = s_rs + L * 32;
#define SM(arr, k) arr[(k) * 32 + lane]
    float gz = 0.0f, dzdx = 0.0f, dzdy = 0.0f;
    if (live) {
        gz = __ldg(m.gz + X.h(j0, i0));
        dzdx = __ldg(m.dzdx + X.h(j0, i0));
        dzdy = __ldg(m.dzdy + X.h(j0, i0));
    }
    // A1: face velocities over the terrain factor, w, and the surface w
    if (live) {
        const float rgw = __ldg(m.rgzu + (size_t)j0 * (ni + 1) + i0), rge = __ldg(m.rgzu + (size_t)j0 * (ni + 1) + i0 + 1);
        const float rgs = __ldg(m.rgzv + (size_t)j0 * ni + i0), rgn = __ldg(m.rgzv + (size_t)(j0 + 1) * ni + i0);
#pragma unroll 4
        for (int k = 1 + wy; k <= nk + 1; k += kTosWarps) {
            const float wv = a.w3d[X.w(k, y, x)];
            if (k > nk) {
                SM(s_w, k) = wv;
                continue;
            }
            const float uw = __ldg(a.u3d + X.u(k, y, x)), ue = __ldg(a.u3d + X.u(k, y, x + 1));
            const float vs = __ldg(a.v3d + X.v(k, y, x)), vn = __ldg(a.v3d + X.v(k, y + 1, x));
            if (VM == 2) {  // flat column: the face velocities and w as they are
                SM(s_xw, k) = uw;
                SM(s_xe, k) = ue;
                SM(s_ys, k) = vs;
                SM(s_yn, k) = vn;
                SM(s_w, k) = wv;
                continue;
            }
            SM(s_xw, k) = uw * rgw;
            SM(s_xe, k) = ue * rge;
            SM(s_ys, k) = vs * rgs;
            SM(s_yn, k) = vn * rgn;
            // bc.F:1151-1178: the surface w of this small step (stored in phase C)
            SM(s_w, k) = k == 1 ? (0.5f * ((uw + ue) * dzdx + (vs + vn) * dzdy)) * gz : wv;
            if (VM && do_adv) {
                // xurho / yvrho: the face's own average of the padded base
                // density (sound.F:604-613; cuda_gm1_child_psolver3_open.py:199-205)
                const float rc = __ldg(p.rho0p + X.w(k, y, x));
                const float rw = __ldg(p.rho0p + X.w(k, y, x - 1)), re = __ldg(p.rho0p + X.w(k, y, x + 1));
                const float rs = __ldg(p.rho0p + X.w(k, y - 1, x)), rn = __ldg(p.rho0p + X.w(k, y + 1, x));
                SM(s_r, k) = (0.5f * (rw + rc)) * SM(s_xw, k);
                SM(s_re, k) = (0.5f * (rc + re)) * SM(s_xe, k);
                SM(s_rs, k) = (0.5f * (rs + rc)) * SM(s_ys, k);
                SM(s_rn, k) = (0.5f * (rc + rn)) * SM(s_yn, k);
            }
        }
    }
    // Each phase's first chunk of global loads is issued before the barrier
    // that opens the phase (they read nothing the earlier phases write), so
    // their latency overlaps the other warps' remaining work.
    A2Load ld[kA2Levels];
    if (live) {
#pragma unroll
        for (int q = 0; q < kA2Levels; ++q) ld[q].load(a, m, X, 1 + wy + q * kTosWarps, nk, j, i, do_adv, VM == 2);
    }
    __syncthreads();
    // A2: divergence, fpk (initial + pi' advection), column coefficients
    if (live) {
        for (int kb = 1 + wy; kb <= nk; kb += kTosWarps * kA2Levels) {
            if (kb != 1 + wy) {
#pragma unroll
                for (int q = 0; q < kA2Levels; ++q) ld[q].load(a, m, X, kb + q * kTosWarps, nk, j, i, do_adv, VM == 2);
            }
#pragma unroll
            for (int q = 0; q < kA2Levels; ++q) {
            const int k = kb + q * kTosWarps;
            if (k > nk) break;
            const unsigned c = X.p(k, j, i);
            const float rk = ld[q].rk, rl = ld[q].rl, rk1 = ld[q].rk1, rrf_k = ld[q].rrf_k, rrf_k1 = ld[q].rrf_k1;
            const float qk = ld[q].qk, pk1 = ld[q].pk1, pk2 = ld[q].pk2;
            const float ppten = ld[q].ppten, ppterm = ld[q].ppterm;
            const float pc = ld[q].pc, pe = ld[q].pe, pw = ld[q].pw, pn = ld[q].pn, ps = ld[q].ps, rr0 = ld[q].rr0;
            if (VM == 2) {
                // sound.F:491-509 (cuda_gm1_child_psolver3_open.py:407-419):
                // fpk = ((dts*(ppten - ppterm*div)) + H) + beta*W, the flat
                // divergence (smeps 1e-30) and pressure advection, W with
                // w(k) and w(k+1) as they are
                const float xw = SM(s_xw, k), xe = SM(s_xe, k), ys = SM(s_ys, k), yn = SM(s_yn, k);
                float div = 0.0f;
                if (do_div) {
                    div = (xe - xw) * p.rdx + (yn - ys) * p.rdy;
                    if (fabsf(div) < 1.0e-30f) div = 0.0f;
                }
                float hx = xw * (pc - pw) + xe * (pe - pc);
                hx = (-hx) * p.temx;
                float hy = ys * (pc - ps) + yn * (pn - pc);
                hy = (-hy) * p.temy;
                const float hp = hx + hy;
                const float vert = SM(s_w, k) * (pk1 + qk) + SM(s_w, k + 1) * (pk2 - qk);
                const float fpk = ((p.dts * (ppten - ppterm * div)) + hp) + p.beta * vert;
                if (dlast) {
                    a.divh[c] = div;
                    a.hadvp[c] = hp;
                    a.fpk[c] = fpk;
                }
                SM(s_fpk, k) = fpk;
                continue;
            }
            float d3k = 0.0f, d3k1 = 0.0f, hak = 0.0f, hak1 = 0.0f;
            if (k >= 2)
                tos_level_terms<VM>(s_xw, s_xe, s_ys, s_yn, s_r, lane, k, p, dzdx, dzdy, gz, rk, rl, rrf_k, do_adv,
                                    d3k, hak);
            if (k < nk)
                tos_level_terms<VM>(s_xw, s_xe, s_ys, s_yn, s_r, lane, k + 1, p, dzdx, dzdy, gz, rk1, rk, rrf_k1,
                                    do_adv, d3k1, hak1);
            if (dlast && k >= 2) {
                a.dum3[c] = d3k;
                if (do_adv) a.hadvp[c] = hak;
            }
            const float xw = SM(s_xw, k), xe = SM(s_xe, k), ys = SM(s_ys, k), yn = SM(s_yn, k);
            float div = 0.0f;
            if (do_div) {
                const float hz = (xe - xw) * p.rdx + (yn - ys) * p.rdy;
                const float vt = (d3k1 - d3k) * col_rdsf<VM>(p, k);
                div = gz * (hz + vt);
                if (fabsf(div) < 1.0e-20f) div = 0.0f;
            }
            const float wk = SM(s_w, k), wk1 = SM(s_w, k + 1);
            const float w1 = k == 1 ? 0.0f : wk, w2 = k == nk ? 0.0f : wk1;
            const float src = p.dts * (ppten - ppterm * div);
            float fpk = src + p.beta * ((-qk) * (w2 - w1));
            if (dlast) a.divh[c] = div;
            if (do_adv) {
                float rxe, rxw, ryn, rys;
                if (VM) {
                    rxw = SM(s_r, k), rxe = SM(s_re, k);
                    rys = SM(s_rs, k), ryn = SM(s_rn, k);
                } else {
                    rxe = rk * xe, rxw = rk * xw, ryn = rk * yn, rys = rk * ys;
                }
                const float u2 = p.temx * rxe, u1 = p.temx * rxw;
                const float v2 = p.temy * ryn, v1 = p.temy * rys;
                const float ww2 = hak1 + p.beta * wk1;
                const float ww1 = hak + p.beta * wk;
                const float xa = u2 * (pe - pc) + u1 * (pc - pw);
                const float ya = v2 * (pn - pc) + v1 * (pc - ps);
                float hz = (-(xa + ya)) * rr0;
                hz = hz * gz;
                const float vt = ww1 * pk1 + ww2 * pk2;
                fpk = fpk + (hz + vt);
            }
            if (dlast) a.fpk[c] = fpk;
            SM(s_fpk, k) = fpk;
            }
        }
    }
    // A3 reads pk1 + qk, pk2 - qk and pp3d of levels k and k-1 again from
    // global memory (L2-resident after A2) instead of keeping them in shared
    // memory: seven shared words per level let three CTAs share an SM
    float lmm[kColLevels], lwt[kColLevels], lq[kColLevels], lp1[kColLevels], lp2[kColLevels], lpp[kColLevels];
    float lqm[kColLevels], lp1m[kColLevels], lp2m[kColLevels], lppm[kColLevels];
    auto a3_loads = [&](int kb) {
#pragma unroll
        for (int q = 0; q < kColLevels; ++q) {
            const int k = kb + q * kTosWarps;
            lmm[q] = lwt[q] = lq[q] = lp1[q] = lp2[q] = lpp[q] = lqm[q] = lp1m[q] = lp2m[q] = lppm[q] = 0.0f;
            if (k > nk) continue;
            const unsigned c = X.p(k, j, i), cm = X.p(k - 1, j, i);
            lmm[q] = __ldg(a.mm + c);
            lwt[q] = __ldg(a.wten + X.w(k, y, x));
            lq[q] = __ldg(a.qk + c);
            lp1[q] = __ldg(a.pk1 + c);
            lp2[q] = __ldg(a.pk2 + c);
            lpp[q] = a.pp3d[c];
            lqm[q] = __ldg(a.qk + cm);
            lp1m[q] = __ldg(a.pk1 + cm);
            lp2m[q] = __ldg(a.pk2 + cm);
            lppm[q] = a.pp3d[cm];
        }
    };
    if (live && do_imp) a3_loads(2 + wy);
    __syncthreads();
    // A3: tridiagonal coefficients and right-hand side, k = 2..nk
    if (live && do_imp) {
        for (int kb = 2 + wy; kb <= nk; kb += kTosWarps * kColLevels) {
            if (kb != 2 + wy) a3_loads(kb);
#pragma unroll
            for (int q = 0; q < kColLevels; ++q) {
            const int k = kb + q * kTosWarps;
            if (k > nk) break;
            const unsigned c = X.p(k, j, i);
            const float mmk = lmm[q];
            const float wt = lwt[q];
            const float a1k = lp1[q] + lq[q], a2k = lp2[q] - lq[q];
            const float a1m = lp1m[q] + lqm[q], a2m = lp2m[q] - lqm[q];
            const float aa = k >= 3 ? (-p.asq) * (mmk * a1m) : 0.0f;
            const float cc = k < nk ? (-p.asq) * ((-mmk) * a2k) : 0.0f;
            const float dg = (-a1k) + a2m;
            const float bb = 1.0f - p.asq * (mmk * dg);
            const float pd = lpp[q] - lppm[q];
            const float fwk = p.dts * wt + p.beta * ((-mmk) * pd);
            const float ud = (lpp[q] + SM(s_fpk, k)) - (lppm[q] + SM(s_fpk, k - 1));
            const float dd = (SM(s_w, k) + fwk) + p.alph * ((-mmk) * ud);
            SM(s_aa, k) = aa;
            SM(s_bb, k) = bb;
            SM(s_cc, k) = cc;
            SM(s_dd, k) = dd;
            if (dlast) {
                a.tri_aa[c] = aa;
                a.tri_bb[c] = bb;
                a.tri_cc[c] = cc;
                a.tri_dd[c] = dd;
            }
            }
        }
    }
    // phase C's first chunk, in flight while warp 0 runs the Thomas sweep
    // (pp3d of level k is read here before this thread writes it in C)
    float luu[kColLevels], lvv[kColLevels], lru[kColLevels], lrv[kColLevels], lrw[kColLevels];
    float cpp[kColLevels], ca1[kColLevels], ca2[kColLevels];
    auto c_loads = [&](int kb) {
#pragma unroll
        for (int q = 0; q < kColLevels; ++q) {
            const int k = kb + q * kTosWarps;
            luu[q] = lvv[q] = lru[q] = lrv[q] = lrw[q] = cpp[q] = ca1[q] = ca2[q] = 0.0f;
            if (k > nk) continue;
            const unsigned qu = X.u(k, y, x), qv = X.v(k, y, x), qw = X.w(k, y, x), c = X.p(k, j, i);
            luu[q] = __ldg(a.u3d + qu);
            lvv[q] = __ldg(a.v3d + qv);
            lru[q] = a.rru[qu];
            lrv[q] = a.rrv[qv];
            lrw[q] = a.rrw[qw];
            cpp[q] = a.pp3d[c];
            const float qk = __ldg(a.qk + c);
            ca1[q] = __ldg(a.pk1 + c) + qk;
            ca2[q] = __ldg(a.pk2 + c) - qk;
        }
    };
    if (live) c_loads(1 + wy);
    __syncthreads();
    // B: Thomas sweep, one lane per column (1/pivot by the correctly rounded
    // reciprocal rcp_rn, the same word as 1.0f / pivot)
    // The next level's coefficients are read while this level eliminates, and
    // the back substitution carries w(k+1) in a register and reads its
    // coefficients kThomasChunk levels at a time, so shared-memory latency
    // stays off the sweep's dependency chain (same operations, same order).
    if (live && do_imp && wy == 0) {
        float ec = 0.0f, ed = 0.0f;
        float aa = SM(s_aa, 2), bb = SM(s_bb, 2), cc = SM(s_cc, 2), dd = SM(s_dd, 2);
        float wtop = 0.0f;
        for (int k = 2; k <= nk; ++k) {
            float naa = 0.0f, nbb = 0.0f, ncc = 0.0f, ndd = 0.0f;
            if (k < nk) {
                naa = SM(s_aa, k + 1);
                nbb = SM(s_bb, k + 1);
                ncc = SM(s_cc, k + 1);
                ndd = SM(s_dd, k + 1);
            }
            const float piv = k == 2 ? bb : aa * ec + bb;
            const float inv = rcp_rn(piv);
            if (dlast) a.tri_pivot[X.p(k, j, i)] = piv;
            if (k < nk) {
                ec = (-cc) * inv;
                ed = (k == 2 ? dd : dd - aa * ed) * inv;
                SM(s_cc, k) = ec;
                SM(s_ed, k) = ed;
                if (dlast) a.elim_d[X.p(k, j, i)] = ed;
            } else {
                wtop = (dd - aa * ed) * inv;
                SM(s_w, k) = wtop;
            }
            aa = naa, bb = nbb, cc = ncc, dd = ndd;
        }
        float wn = wtop;
        for (int kb = nk - 1; kb >= 2; kb -= kThomasChunk) {
            float ce[kThomasChunk], ee[kThomasChunk];
#pragma unroll
            for (int q = 0; q < kThomasChunk; ++q) {
                const int k = kb - q;
                ce[q] = k >= 2 ? SM(s_cc, k) : 0.0f;
                ee[q] = k >= 2 ? SM(s_ed, k) : 0.0f;
            }
#pragma unroll
            for (int q = 0; q < kThomasChunk; ++q) {
                const int k = kb - q;
                if (k < 2) break;
                wn = ce[q] * wn + ee[q];
                SM(s_w, k) = wn;
            }
        }
    }
    __syncthreads();
    // C: pressure update, filter, halo copy, averages
    if (live) {
        const bool fill = p.n < p.nloop && (p.abl & GM1B_TOS_BETWEEN_STEP_FILL);
        const bool east = i == ni, north = j == nj;
        for (int kb = 1 + wy; kb <= nk; kb += kTosWarps * kColLevels) {
            if (kb != 1 + wy) c_loads(kb);
#pragma unroll
            for (int q = 0; q < kColLevels; ++q) {
            const int k = kb + q * kTosWarps;
            if (k > nk) break;
            const unsigned c = X.p(k, j, i);
            const unsigned qu = X.u(k, y, x), qv = X.v(k, y, x), qw = X.w(k, y, x);
            const float uu = luu[q], vv = lvv[q];
            const float ru = lru[q], rv = lrv[q], rw = lrw[q];
            const float wk = SM(s_w, k), wk1 = SM(s_w, k + 1);
            if (k == 1) a.w3d[qw] = wk;
            if (do_imp && k >= 2) {
                a.w3d[qw] = wk;
                if (dlast) {
                    float lhs = SM(s_aa, k) * SM(s_w, k - 1) + SM(s_bb, k) * wk;
                    const float cc = k < nk ? (-p.asq) * ((-__ldg(a.mm + c)) * ca2[q]) : 0.0f;
                    lhs = lhs + cc * wk1;
                    a.tri_residual[c] = lhs - SM(s_dd, k);
                }
            }
            // the flat column keeps w(1) and w(nk+1) and filters at 1e-30
            const float w1 = (k == 1 && VM != 2) ? 0.0f : wk, w2 = (k == nk && VM != 2) ? 0.0f : wk1;
            const float old = cpp[q];
            const float vt = w1 * ca1[q] + w2 * ca2[q];
            float up = (old + SM(s_fpk, k)) + p.alph * vt;
            if (fabsf(up) < (VM == 2 ? 1.0e-30f : 1.0e-20f)) up = 0.0f;
            const float tend = p.kdiv * (up - old);
            const float pd = up + tend;
            a.pp3d[c] = up;
            a.ppd[c] = pd;
            if (dlast) a.elim_c[c] = tend;
            if (p.nrk == 3 && last) a.ppx[c] = tend;
            if (fill) {  // bcp: the halo takes its clamped interior neighbour
                const int rows[3] = {j, j == 1 ? 0 : -1, north ? nj + 1 : -1};
                const int cols[3] = {i, i == 1 ? 0 : -1, east ? ni + 1 : -1};
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    if (rows[r] < 0) continue;
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        if (cols[q] < 0 || (r == 0 && q == 0)) continue;
                        a.ppd[X.p(k, rows[r], cols[q])] = pd;
                    }
                }
            }
            // rru/rrv/rrw over faces 1..ni+1 and rows 1..nj+1
            {
                const float su = ru + uu, sv = rv + vv, sw = rw + (last ? wk * p.alph : wk);
                a.rru[qu] = last ? su * p.tavg : su;
                a.rrv[qv] = last ? sv * p.tavg : sv;
                a.rrw[qw] = last ? sw * p.tavg : sw;
            }
            if (east || north) {
#pragma unroll
                for (int e = 1; e < 4; ++e) {
                    const int dx = e & 1, dy = e >> 1;
                    if ((dx && !east) || (dy && !north)) continue;
                    const unsigned eu = X.u(k, y + dy, x + dx), ev = X.v(k, y + dy, x + dx), ew = X.w(k, y + dy, x + dx);
                    const float su = a.rru[eu] + __ldg(a.u3d + eu), sv = a.rrv[ev] + __ldg(a.v3d + ev);
                    const float wv = a.w3d[ew];
                    const float sw = a.rrw[ew] + (last ? wv * p.alph : wv);
                    a.rru[eu] = last ? su * p.tavg : su;
                    a.rrv[ev] = last ? sv * p.tavg : sv;
                    a.rrw[ew] = last ? sw * p.tavg : sw;
                }
            }
            }
        }
    }
#undef SM
}

// ---------------------------------------------------------------------------
// radiation histories (radbcew4/radbcns4): one warp per boundary line, the
// clamped phase speeds of all levels in parallel, their column mean summed
// in level order by lane 0
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) tos_radiation_kernel(TosArgs p, float dx, float dy, float dttmp) {
    extern __shared__ float sh[];
    const Ix X{p.ni, p.nj};
    const int ni = p.ni, nj = p.nj, nk = p.nk;
    const int lane = threadIdx.x, wy = threadIdx.y;
    int line = blockIdx.x * 4 + wy;
    const int lines = 2 * nj + 2 * ni;
    if (line >= lines) return;
    float *s = sh + wy * (nk + 1);
    const gm1b_terrain_open_arrays &a = p.a;
    int side;
    if (line < nj) side = 0;
    else if (line < 2 * nj) side = 1, line -= nj;
    else if (line < 2 * nj + ni) side = 2, line -= 2 * nj;
    else side = 3, line -= 2 * nj + ni;
    const float eps = 1.0e-10f, limit = 350.0f;
    for (int k = 1 + lane; k <= nk; k += 32) {
        float foo, num, c;
        if (side == 0) {
            const int yy = line + 3;
            foo = a.ua[X.u(k, yy, 5)] - a.ua[X.u(k, yy, 4)];
            num = (dx * a.ruf[4]) * (a.ua[X.u(k, yy, 4)] - a.u3d[X.u(k, yy, 4)]);
        } else if (side == 1) {
            const int yy = line + 3;
            foo = a.ua[X.u(k, yy, ni + 2)] - a.ua[X.u(k, yy, ni + 1)];
            num = (dx * a.ruf[ni + 2]) * (a.ua[X.u(k, yy, ni + 2)] - a.u3d[X.u(k, yy, ni + 2)]);
        } else if (side == 2) {
            const int xx = line + 3;
            foo = a.va[X.v(k, 5, xx)] - a.va[X.v(k, 4, xx)];
            num = (dy * a.rvf[4]) * (a.va[X.v(k, 4, xx)] - a.v3d[X.v(k, 4, xx)]);
        } else {
            const int xx = line + 3;
            foo = a.va[X.v(k, nj + 2, xx)] - a.va[X.v(k, nj + 1, xx)];
            num = (dy * a.rvf[nj + 2]) * (a.va[X.v(k, nj + 2, xx)] - a.v3d[X.v(k, nj + 2, xx)]);
        }
        const float den = dttmp * (copysignf(eps, foo) + foo);
        c = num / den;
        s[k - 1] = (side == 0 || side == 2) ? np_max(np_min(c, 0.0f), -limit) : np_min(np_max(c, 0.0f), limit);
    }
    __syncwarp();
    if (lane == 0) {
        float avg = 0.0f;
        for (int k = 0; k < nk; ++k) avg = avg + s[k];
        s[nk] = avg / (float)nk;
    }
    __syncwarp();
    const float avg = s[nk];
    float *rad = side == 0 ? a.radbcw : side == 1 ? a.radbce : side == 2 ? a.radbcs : a.radbcn;
    const size_t stride = side < 2 ? (size_t)(nj + 6) : (size_t)(ni + 6);
    for (int k = 1 + lane; k <= nk; k += 32) rad[(size_t)k * stride + line + 3] = avg;
}

// ---------------------------------------------------------------------------
// stage fills, pass 1: bcu west/east, bcv south/north, bcw west/east on
// k = 2..nk with the flag-1 zero of w levels 1 and nk+1, and (nrk < 3) bcp
// west/east of pp3d and bcs west/east of the scalar
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) tos_fill1_kernel(TosArgs p) {
    const Ix X{p.ni, p.nj};
    const int ni = p.ni, nj = p.nj, nk = p.nk;
    const gm1b_terrain_open_arrays &a = p.a;
    const bool more = p.nrk < 3;
    const size_t nA = (size_t)nk * (nj + 2) * 6;           // u W/E, rows 0..nj+1
    const size_t nB = (size_t)nk * 6 * (ni + 2);           // v S/N, columns 0..ni+1
    const size_t nC = (size_t)(nk - 1) * (nj + 2) * 6;     // w W/E, k = 2..nk
    const size_t nD = (size_t)2 * (nj + 2) * (ni + 2);     // w levels 1 and nk+1
    const size_t nE = more ? (size_t)nk * (nj + 2) * 2 : 0;  // pp3d W/E
    const size_t nF = more ? (size_t)nk * (nj + 2) * 6 : 0;  // scalar W/E
    const size_t total = nA + nB + nC + nD + nE + nF;
    for (size_t z = (size_t)blockIdx.x * blockDim.x + threadIdx.x; z < total; z += (size_t)gridDim.x * blockDim.x) {
        size_t q = z;
        if (q < nA) {
            const int h = (int)(q % 6), j = (int)((q / 6) % (nj + 2)), k = (int)(q / (6 * (size_t)(nj + 2))) + 1;
            const int y = j + 2;
            if (h < 3) a.u3d[X.u(k, y, h)] = a.u3d[X.u(k, y, 3)];
            else a.u3d[X.u(k, y, ni + 1 + h)] = a.u3d[X.u(k, y, ni + 3)];
            continue;
        }
        q -= nA;
        if (q < nB) {
            const int i = (int)(q % (ni + 2)), h = (int)((q / (ni + 2)) % 6), k = (int)(q / (6 * (size_t)(ni + 2))) + 1;
            const int x = i + 2;
            if (h < 3) a.v3d[X.v(k, h, x)] = a.v3d[X.v(k, 3, x)];
            else a.v3d[X.v(k, nj + 1 + h, x)] = a.v3d[X.v(k, nj + 3, x)];
            continue;
        }
        q -= nB;
        if (q < nC) {
            const int h = (int)(q % 6), j = (int)((q / 6) % (nj + 2)), k = (int)(q / (6 * (size_t)(nj + 2))) + 2;
            const int y = j + 2;
            if (h < 3) a.w3d[X.w(k, y, h)] = a.w3d[X.w(k, y, 3)];
            else a.w3d[X.w(k, y, ni + h)] = a.w3d[X.w(k, y, ni + 2)];
            continue;
        }
        q -= nC;
        if (q < nD) {
            const int i = (int)(q % (ni + 2)), j = (int)((q / (ni + 2)) % (nj + 2));
            const int k = q / ((size_t)(ni + 2) * (nj + 2)) == 0 ? 1 : nk + 1;
            a.w3d[X.w(k, j + 2, i + 2)] = 0.0f;
            continue;
        }
        q -= nD;
        if (q < nE) {
            const int e = (int)(q % 2), j = (int)((q / 2) % (nj + 2)), k = (int)(q / (2 * (size_t)(nj + 2))) + 1;
            if (e == 0) a.pp3d[X.p(k, j, 0)] = a.pp3d[X.p(k, j, 1)];
            else a.pp3d[X.p(k, j, ni + 1)] = a.pp3d[X.p(k, j, ni)];
            continue;
        }
        q -= nE;
        {
            const int h = (int)(q % 6), j = (int)((q / 6) % (nj + 2)), k = (int)(q / (6 * (size_t)(nj + 2))) + 1;
            const int y = j + 2;
            if (h < 3) a.scalar[X.w(k, y, h)] = a.scalar[X.w(k, y, 3)];
            else a.scalar[X.w(k, y, ni + h)] = a.scalar[X.w(k, y, ni + 2)];
        }
    }
}

// ---------------------------------------------------------------------------
// stage fills, pass 2: bcu south/north, bcv west/east, bcw south/north on
// k = 2..nk, the surface w (bcwsfc), and (nrk < 3) bcp south/north of pp3d
// and bcs south/north of the scalar
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) tos_fill2_kernel(TosArgs p) {
    const Ix X{p.ni, p.nj};
    const int ni = p.ni, nj = p.nj, nk = p.nk;
    const gm1b_terrain_open_arrays &a = p.a;
    const gm1b_terrain_metrics &m = p.m;
    const bool more = p.nrk < 3;
    const size_t nA = (size_t)nk * 6 * (ni + 3);           // u S/N, faces 0..ni+2
    const size_t nB = (size_t)nk * (nj + 3) * 6;           // v W/E, rows 0..nj+2
    const size_t nC = (size_t)(nk - 1) * 6 * (ni + 2);     // w S/N, k = 2..nk
    const size_t nD = p.vmode == 2 ? 0 : (size_t)nj * ni;  // bcwsfc (none on the flat column)
    const size_t nE = more ? (size_t)nk * 2 * (ni + 2) : 0;  // pp3d S/N
    const size_t nF = more ? (size_t)nk * 6 * (ni + 2) : 0;  // scalar S/N
    const size_t total = nA + nB + nC + nD + nE + nF;
    for (size_t z = (size_t)blockIdx.x * blockDim.x + threadIdx.x; z < total; z += (size_t)gridDim.x * blockDim.x) {
        size_t q = z;
        if (q < nA) {
            const int i = (int)(q % (ni + 3)), h = (int)((q / (ni + 3)) % 6), k = (int)(q / (6 * (size_t)(ni + 3))) + 1;
            const int x = i + 2;
            if (h < 3) a.u3d[X.u(k, h, x)] = a.u3d[X.u(k, 3, x)];
            else a.u3d[X.u(k, nj + h, x)] = a.u3d[X.u(k, nj + 2, x)];
            continue;
        }
        q -= nA;
        if (q < nB) {
            const int h = (int)(q % 6), j = (int)((q / 6) % (nj + 3)), k = (int)(q / (6 * (size_t)(nj + 3))) + 1;
            const int y = j + 2;
            if (h < 3) a.v3d[X.v(k, y, h)] = a.v3d[X.v(k, y, 3)];
            else a.v3d[X.v(k, y, ni + h)] = a.v3d[X.v(k, y, ni + 2)];
            continue;
        }
        q -= nB;
        if (q < nC) {
            const int i = (int)(q % (ni + 2)), h = (int)((q / (ni + 2)) % 6), k = (int)(q / (6 * (size_t)(ni + 2))) + 2;
            const int x = i + 2;
            if (h < 3) a.w3d[X.w(k, h, x)] = a.w3d[X.w(k, 3, x)];
            else a.w3d[X.w(k, nj + h, x)] = a.w3d[X.w(k, nj + 2, x)];
            continue;
        }
        q -= nC;
        if (q < nD) {
            const int i0 = (int)(q % ni), j0 = (int)(q / ni);
            const int y = j0 + 3, x = i0 + 3;
            const float ut = (a.u3d[X.u(1, y, x)] + a.u3d[X.u(1, y, x + 1)]) * m.dzdx[X.h(j0, i0)];
            const float vt = (a.v3d[X.v(1, y, x)] + a.v3d[X.v(1, y + 1, x)]) * m.dzdy[X.h(j0, i0)];
            a.w3d[X.w(1, y, x)] = (0.5f * (ut + vt)) * m.gz[X.h(j0, i0)];
            continue;
        }
        q -= nD;
        if (q < nE) {
            const int i = (int)(q % (ni + 2)), e = (int)((q / (ni + 2)) % 2), k = (int)(q / (2 * (size_t)(ni + 2))) + 1;
            if (e == 0) a.pp3d[X.p(k, 0, i)] = a.pp3d[X.p(k, 1, i)];
            else a.pp3d[X.p(k, nj + 1, i)] = a.pp3d[X.p(k, nj, i)];
            continue;
        }
        q -= nE;
        {
            const int i = (int)(q % (ni + 2)), h = (int)((q / (ni + 2)) % 6), k = (int)(q / (6 * (size_t)(ni + 2))) + 1;
            const int x = i + 2;
            if (h < 3) a.scalar[X.w(k, h, x)] = a.scalar[X.w(k, 3, x)];
            else a.scalar[X.w(k, nj + h, x)] = a.scalar[X.w(k, nj + 2, x)];
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
bool launch_ok(const char *what) {
    const cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        cudaGetLastError();
        gm1b_set_error("%s: %s", what, cudaGetErrorString(e));
        return false;
    }
    return true;
}

// Fornberg (1988): weights of the three-point value stencil at x0 from the
// first three of four nodes, in double precision (param.F:9016-9035).
void fornberg_value_weights(const double alpha[4], double x0, double out[3]) {
    double d[4][6][4] = {};
    d[0][1][0] = 1.0;
    double c1 = 1.0;
    for (int n = 1; n < 4; ++n) {
        double c2 = 1.0;
        for (int nu = 0; nu < n; ++nu) {
            const double c3 = alpha[n] - alpha[nu];
            c2 = c2 * c3;
            d[n - 1][n + 1][nu] = 0.0;
            for (int mo = 0; mo <= n; ++mo)
                d[n][mo + 1][nu] = ((alpha[n] - x0) * d[n - 1][mo + 1][nu] - mo * d[n - 1][mo][nu]) / c3;
        }
        for (int mo = 0; mo <= n; ++mo)
            d[n][mo + 1][n] = (c1 / c2) * (mo * d[n - 1][mo][n - 1] - (alpha[n - 1] - x0) * d[n - 1][mo + 1][n - 1]);
        c1 = c2;
    }
    for (int nu = 0; nu < 3; ++nu) out[nu] = d[2][1][nu];
}

// cgs (ground) / cgt (lid) of the uniform column, float32 levels as the twin
// forms them (fornberg_extrapolation_weights, cm1_vertical_grid.py:422-454)
bool edge_weights(int nk, float dz, bool top, float out[3]) {
    auto sg = [dz](int k) { return ((float)k - 0.5f) * dz; };
    auto sf = [dz](int k) { return (float)(k - 1) * dz; };
    float den, num, nodes[4];
    if (top) {
        den = sf(nk + 1) - sf(nk);
        num = sf(nk + 1);
        for (int q = 0; q < 4; ++q) nodes[q] = sg(nk - q);
    } else {
        den = sf(2) - sf(1);
        num = sf(1);
        for (int q = 0; q < 4; ++q) nodes[q] = sg(1 + q);
    }
    if (!(den > 0.0f) || !std::isfinite(den)) return false;
    double alpha[4], w[3];
    for (int q = 0; q < 4; ++q) alpha[q] = (double)(nodes[q] / den);
    for (int q = 0; q < 4; ++q)
        for (int r = 0; r < q; ++r)
            if (alpha[q] == alpha[r]) return false;
    fornberg_value_weights(alpha, (double)(num / den), w);
    for (int q = 0; q < 3; ++q) out[q] = (float)w[q];
    return true;
}

unsigned grid_for(size_t work, int block) {
    const size_t want = (work + (size_t)block - 1) / (size_t)block;
    const size_t cap = (size_t)148 * 16;
    return (unsigned)std::max<size_t>(1, std::min(want, cap));
}

}  // namespace
}  // namespace gm1b

using namespace gm1b;

namespace gm1b {
namespace {

// one stage on the uniform column (col == nullptr, dz) or on the stretched
// terrain column bound in col
int32_t terrain_open_stage(int32_t ni, int32_t nj, int32_t nk, int32_t nrk, float dt, int32_t nsound, float dx,
                           float dy, double dz, float alph, float kdiv, uint32_t ablations, uint32_t flags,
                           uint32_t obc, const gm1b_terrain_open_arrays *arrays, const gm1b_terrain_metrics *metrics,
                           const gm1b_momentum_column *col, void *stream) {
    if (arrays == nullptr || metrics == nullptr || ni < 3 || nj < 3 || nk < 4 || nk > kTosMaxNk || nrk < 1 ||
        nrk > 3) {
        gm1b_set_error("gm1b_terrain_open_stage: need arrays and metrics, ni >= 3, nj >= 3, 4 <= nk <= %d, "
                       "nrk in 1..3", kTosMaxNk);
        return GM1B_ERR_ARGUMENT;
    }
    if ((size_t)(nk + 3) * (size_t)(nj + 7) * (size_t)(ni + 7) >= ((size_t)1 << 31)) {
        gm1b_set_error("gm1b_terrain_open_stage: a %dx%dx%d grid's padded arrays reach 2^31 words; the kernels "
                       "index with 32-bit offsets", ni, nj, nk);
        return GM1B_ERR_ARGUMENT;
    }
    if (col != nullptr && col->flat) {
        if (col->mh == nullptr || col->mf == nullptr || !(col->rdz > 0.0f) || !std::isfinite(col->rdz)) {
            gm1b_set_error("gm1b_terrain_open_stage_column: the flat column needs mh, mf and a finite rdz > 0");
            return GM1B_ERR_ARGUMENT;
        }
        for (int side = 0; side < 4; ++side) {
            const unsigned code = (obc >> (4 * side)) & 15u;
            if (code < 1u || code > 4u) {
                gm1b_set_error("gm1b_terrain_open_stage_column: lateral code 0x%x: each side is 1..4", obc);
                return GM1B_ERR_ARGUMENT;
            }
        }
        if ((obc >> 16) != 0u || (((obc & 15u) == 1u) != (((obc >> 4) & 15u) == 1u)) ||
            ((((obc >> 8) & 15u) == 1u) != (((obc >> 12) & 15u) == 1u))) {
            gm1b_set_error("gm1b_terrain_open_stage_column: lateral code 0x%x: a periodic direction is periodic on "
                           "both sides (param.F:2562-2588)", obc);
            return GM1B_ERR_ARGUMENT;
        }
        dz = 1.0;  // the scalar spacing is not used on a bound column
    } else if (col != nullptr) {
        if (obc != 0x2222u) {
            gm1b_set_error("gm1b_terrain_open_stage_column: lateral code 0x%x: the terrain column's stage runs "
                           "ssopenbc on all four sides (0x2222)", obc);
            return GM1B_ERR_ARGUMENT;
        }
        if (col->sigma == nullptr || col->sigmaf == nullptr || col->rds == nullptr || col->rdsf == nullptr ||
            col->rho0_padded == nullptr || !(col->ztop > 0.0f) || !std::isfinite(col->ztop)) {
            gm1b_set_error("gm1b_terrain_open_stage_column: the terrain column needs sigma, sigmaf, rds, rdsf, "
                           "rho0_padded and a finite ztop > 0");
            return GM1B_ERR_ARGUMENT;
        }
        dz = 1.0;  // the scalar spacing is not used on a bound column
    }
    if (!(dx > 0.0f) || !(dy > 0.0f) || !(dz > 0.0) || !std::isfinite(dx) || !std::isfinite(dy) ||
        !std::isfinite(dz) || !(dt > 0.0f) || !std::isfinite(dt)) {
        gm1b_set_error("gm1b_terrain_open_stage: dt, dx, dy, dz must be finite and > 0");
        return GM1B_ERR_ARGUMENT;
    }
    if (!(alph >= 0.0f && alph <= 1.0f) || !(kdiv >= 0.0f && kdiv <= 1.0f)) {
        gm1b_set_error("gm1b_terrain_open_stage: alph and kdiv must lie in [0, 1]");
        return GM1B_ERR_ARGUMENT;
    }
    if (ablations & ~GM1B_TOS_ALL) {
        gm1b_set_error("gm1b_terrain_open_stage: unknown ablation bits 0x%x", ablations & ~GM1B_TOS_ALL);
        return GM1B_ERR_ARGUMENT;
    }
    const float *const *mp = reinterpret_cast<const float *const *>(metrics);
    for (size_t q = 0; q < sizeof(gm1b_terrain_metrics) / sizeof(float *); ++q)
        if (mp[q] == nullptr) {
            gm1b_set_error("gm1b_terrain_open_stage: a metric pointer is NULL");
            return GM1B_ERR_ARGUMENT;
        }
    float *const *ap = reinterpret_cast<float *const *>(arrays);
    for (size_t q = 0; q < sizeof(gm1b_terrain_open_arrays) / sizeof(float *); ++q)
        if (ap[q] == nullptr) {
            gm1b_set_error("gm1b_terrain_open_stage: an array pointer is NULL");
            return GM1B_ERR_ARGUMENT;
        }
    int32_t nloop = 0;
    float dts = 0.0f;
    if (gm1b_sound3_stage_schedule(dt, nsound, nrk, &nloop, &dts) != GM1B_OK) return GM1B_ERR_ARGUMENT;
    TosArgs p{};
    p.a = *arrays;
    p.m = *metrics;
    p.ni = ni, p.nj = nj, p.nk = nk, p.nrk = nrk, p.nloop = nloop;
    p.abl = ablations;
    p.diag = (flags & GM1B_TOS_DIAGNOSTICS) ? 1u : 0u;
    p.dts = dts;
    p.rdx = 1.0f / dx;
    p.rdy = 1.0f / dy;
    p.dz = (float)dz;
    p.alph = alph;
    p.beta = 1.0f - alph;
    p.asq = alph * alph;
    p.kdiv = kdiv;
    p.temx = (dts * 0.5f) * p.rdx;
    p.temy = (dts * 0.5f) * p.rdy;
    p.tavg = 1.0f / (float)nloop;
    p.zt = (float)((double)nk * dz);
    p.rzt = 1.0f / p.zt;
    p.halfcp = 1005.7f * 0.5f;
    p.obc = obc;
    if (col != nullptr && col->flat) {
        p.vmode = 2;
        p.mhp = col->mh, p.mfp = col->mf, p.rdz = col->rdz;
    } else if (col != nullptr) {
        // the lid is the bound top; the edge-face extrapolation keeps the
        // open-boundary text's own 1.875 / -1.25 / 0.375 weights, which the
        // profile patch leaves in place (cuda_terrain_open_boundary.py:845-850,
        // cuda_gm1_child_psolver3_open.py:289-330)
        p.vmode = 1;
        p.sgm = col->sigma, p.sgmf = col->sigmaf, p.rdsp = col->rds, p.rdsfp = col->rdsf;
        p.rho0p = col->rho0_padded;
        p.zt = col->ztop;
        p.rzt = 1.0f / p.zt;
        const float w[3] = {1.875f, -1.25f, 0.375f};
        for (int q = 0; q < 3; ++q) p.cgs[q] = p.cgt[q] = w[q];
    } else if (!edge_weights(nk, p.dz, false, p.cgs) || !edge_weights(nk, p.dz, true, p.cgt)) {
        gm1b_set_error("gm1b_terrain_open_stage: degenerate vertical levels for dz=%g", dz);
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int col_arrays = kTosArrays + (p.vmode == 1 ? 3 : 0);
    const size_t col_smem = (size_t)col_arrays * (size_t)(nk + 2) * 32 * sizeof(float);
    static bool attr_set[64] = {};  // per device: the attribute belongs to each device's context
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        gm1b_set_error("gm1b_terrain_open_stage: no usable current device");
        return GM1B_ERR_CUDA;
    }
    if (!attr_set[dev]) {
        cudaError_t e = cudaFuncSetAttribute(tos_column_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)((size_t)kTosArrays * (kTosMaxNk + 2) * 32 * sizeof(float)));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(tos_column_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)((size_t)(kTosArrays + 3) * (kTosMaxNk + 2) * 32 * sizeof(float)));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(tos_column_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)((size_t)kTosArrays * (kTosMaxNk + 2) * 32 * sizeof(float)));
        if (e != cudaSuccess) {
            gm1b_set_error("cudaFuncSetAttribute(tos_column_kernel): %s", cudaGetErrorString(e));
            return GM1B_ERR_CUDA;
        }
        attr_set[dev] = true;
    }
    {
        ProfScope ps("tos_prepare_kernel", st);
        tos_prepare_kernel<<<grid_for((size_t)nk * (nj + 2) * (ni + 2), 256), 256, 0, st>>>(p);
        ps.stop();
    }
    if (!launch_ok("tos_prepare_kernel")) return GM1B_ERR_CUDA;
    const dim3 pg_grid((ni + 2 + 31) / 32, (nj + 2 + 3) / 4), col_grid((ni + 31) / 32, nj);
    for (int n = 1; n <= nloop; ++n) {
        p.n = n;
        if ((ablations & GM1B_TOS_OPEN_CONSUMPTION) && p.vmode == 2) {
            ProfScope ps("tos_flat_edge_kernel", st);
            tos_flat_edge_kernel<<<grid_for((size_t)nk * (nj + ni), 256), 256, 0, st>>>(p);
            ps.stop();
            if (!launch_ok("tos_flat_edge_kernel")) return GM1B_ERR_CUDA;
        } else if (ablations & GM1B_TOS_OPEN_CONSUMPTION) {
            ProfScope ps("tos_edge_kernel", st);
            tos_edge_kernel<<<2 * nj + 2 * ni, 128, 4 * (size_t)(nk + 2) * sizeof(float), st>>>(p);
            ps.stop();
            if (!launch_ok("tos_edge_kernel")) return GM1B_ERR_CUDA;
        }
        if ((ablations & GM1B_TOS_PRESSURE_GRADIENT) && p.vmode == 2) {
            ProfScope ps("tos_flat_pgrad_kernel", st);
            tos_flat_pgrad_kernel<<<dim3((ni + 1 + 31) / 32, (nj + 1 + 3) / 4), dim3(32, 4), 0, st>>>(p);
            ps.stop();
            if (!launch_ok("tos_flat_pgrad_kernel")) return GM1B_ERR_CUDA;
        } else if (ablations & GM1B_TOS_PRESSURE_GRADIENT) {
            ProfScope ps("tos_pgrad_kernel", st);
            tos_pgrad_kernel<<<pg_grid, dim3(32, 4), 0, st>>>(p);
            ps.stop();
            if (!launch_ok("tos_pgrad_kernel")) return GM1B_ERR_CUDA;
        }
        {
            ProfScope ps("tos_column_kernel", st);
            if (p.vmode == 2)
                tos_column_kernel<2><<<col_grid, dim3(32, kTosWarps), col_smem, st>>>(p);
            else if (p.vmode == 1)
                tos_column_kernel<1><<<col_grid, dim3(32, kTosWarps), col_smem, st>>>(p);
            else
                tos_column_kernel<0><<<col_grid, dim3(32, kTosWarps), col_smem, st>>>(p);
            ps.stop();
            if (!launch_ok("tos_column_kernel")) return GM1B_ERR_CUDA;
        }
    }
    if (ablations & GM1B_TOS_RADIATION) {
        const int lines = 2 * nj + 2 * ni;
        ProfScope ps("tos_radiation_kernel", st);
        tos_radiation_kernel<<<(lines + 3) / 4, dim3(32, 4), 4 * (size_t)(nk + 1) * sizeof(float), st>>>(
            p, dx, dy, gm1b_rk_stage_dt(dt, nrk));
        ps.stop();
        if (!launch_ok("tos_radiation_kernel")) return GM1B_ERR_CUDA;
    }
    if (ablations & GM1B_TOS_STAGE_FILLS) {
        const size_t w1 = (size_t)nk * (nj + 2) * 6 * 3 + (size_t)nk * 6 * (ni + 2) + (size_t)2 * (nj + 2) * (ni + 2);
        const size_t w2 = (size_t)nk * 6 * (ni + 3) * 2 + (size_t)nk * (nj + 3) * 6 + (size_t)nj * ni;
        {
            ProfScope ps("tos_fill1_kernel", st);
            tos_fill1_kernel<<<grid_for(w1, 256), 256, 0, st>>>(p);
            ps.stop();
        }
        if (!launch_ok("tos_fill1_kernel")) return GM1B_ERR_CUDA;
        {
            ProfScope ps("tos_fill2_kernel", st);
            tos_fill2_kernel<<<grid_for(w2, 256), 256, 0, st>>>(p);
            ps.stop();
        }
        if (!launch_ok("tos_fill2_kernel")) return GM1B_ERR_CUDA;
    }
    return GM1B_OK;
}

}  // namespace
}  // namespace gm1b

extern "C" int32_t gm1b_terrain_open_stage(int32_t ni, int32_t nj, int32_t nk, int32_t nrk, float dt, int32_t nsound,
                                           float dx, float dy, double dz, float alph, float kdiv, uint32_t ablations,
                                           uint32_t flags, const gm1b_terrain_open_arrays *arrays,
                                           const gm1b_terrain_metrics *metrics, void *stream) {
    return terrain_open_stage(ni, nj, nk, nrk, dt, nsound, dx, dy, dz, alph, kdiv, ablations, flags, 0x2222u, arrays,
                              metrics, nullptr, stream);
}

extern "C" int32_t gm1b_terrain_open_stage_column(int32_t ni, int32_t nj, int32_t nk, int32_t nrk, float dt,
                                                  int32_t nsound, float dx, float dy, float alph, float kdiv,
                                                  uint32_t ablations, uint32_t flags, uint32_t lateral_obc,
                                                  const gm1b_terrain_open_arrays *arrays,
                                                  const gm1b_terrain_metrics *metrics,
                                                  const gm1b_momentum_column *column, void *stream) {
    if (column == nullptr) {
        gm1b_set_error("gm1b_terrain_open_stage_column: column is NULL");
        return GM1B_ERR_ARGUMENT;
    }
    return terrain_open_stage(ni, nj, nk, nrk, dt, nsound, dx, dy, 1.0, alph, kdiv, ablations, flags, lateral_obc,
                              arrays, metrics, column, stream);
}
