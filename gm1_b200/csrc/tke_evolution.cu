// tke_evolution.cu - sm_100a kernels of the TKE evolution on the terrain
// lane: turbt (horizontal TKE flux divergence with the terrain correction
// and the vertically implicit diffusion) and the flux-form RK stages.
//
// Behaviour followed (reference file:line):
//   cpu_tke_evolution_inplace   src/cm1core/cuda_tke_evolution.py:206-327
//   launch_cuda_tke_diffusion / _rk_stage / _commit / _evolution   :421-492
//   flat column: gm1_flat_turbt_v1 and gm1_flat_tke_advw_rk_v1
//               src/cm1core/cuda_gm1_flat_stretched_closure.py:314-359, :401-449
//               (enqueue_flat_turbt :631; CartesianClosure.tke_rk, cuda_cartesian_closure.py:1658-1663)
//
// Design (B200):
//  * turbt is one kernel per 32 x 4 column tile.  Each thread first solves
//    its column's implicit diffusion (Thomas) with the elimination arrays in
//    shared memory (the reference's thread-per-column kernel keeps five local
//    arrays of 74 words, which spill); then the tile walks the face levels
//    upwards with a three-level ring of the x and y TKE face fluxes (33 x 4
//    and 32 x 5 per level) in shared memory, so every face flux is formed
//    once, and each cell adds its horizontal divergence and vertical
//    diffusion to tketen.  No device scratch.
//  * an RK stage is elementwise over the face levels: each cell forms its six
//    face fluxes (fifth order, WENO5 at nrk = 3) from the stage-start field.
//  * binary32 one operation at a time in the reference's order, binary64
//    WENO weights: word-identical to the reference twin.
#include "gm1b_common.cuh"
#include "weno.cuh"

namespace gm1b {
namespace {

constexpr int kTTX = 32, kTTY = 4, kTT = kTTX * kTTY;  // turbt tile
constexpr int kTTChunk = 8;  // levels whose column-solve loads turbt issues together
constexpr int kG = 3;                                    // padded-lane halo of rru/rrv/rrw

struct TkeArgs {
    const float *t, *kmh, *kmv, *rho, *rf, *mh, *mf, *gz, *rgz, *rgzu, *rgzv;
    const float *tkea, *c2, *rrf0, *rru, *rrv, *rrw, *divx;
    const float *mfp;  // flat column: the mf profile (nk+3, CM1-indexed)
    float *tketen;
    int ni, nj, nk;
    float rdx, rdy, rdz, dz, zt;  // flat column: rdz is the coordinate's reference 1/dz
};

__device__ __forceinline__ int clampi(int x, int n) { return x < 0 ? 0 : (x >= n ? n - 1 : x); }
// 32-bit element offsets (the entry points refuse grids whose padded arrays
// reach 2^31 words)
__device__ __forceinline__ unsigned f3(const TkeArgs &a, int k, int j, int i) {
    return ((unsigned)k * (unsigned)a.nj + (unsigned)j) * (unsigned)a.ni + (unsigned)i;
}
// value at a clamped column (constant extension beyond the open sides)
__device__ __forceinline__ float cellc(const TkeArgs &a, const float *p, int k, int j, int i) {
    return p[f3(a, k, clampi(j, a.nj), clampi(i, a.ni))];
}
__device__ __forceinline__ float g2c(const TkeArgs &a, const float *p, int j, int i) {
    return p[(unsigned)clampi(j, a.nj) * (unsigned)a.ni + (unsigned)clampi(i, a.ni)];
}
__device__ __forceinline__ float tsm(const TkeArgs &a, int m, int j, int i) {
    return 0.5f * (cellc(a, a.t, m, j, i) + cellc(a, a.t, m + 1, j, i));
}

// x TKE flux at face level f (1..nk-1), row j, u face `face`; 0 elsewhere
__device__ float tke_tx(const TkeArgs &a, int f, int j, int face) {
    if (f <= 0 || f >= a.nk) return 0.0f;
    const int l = face - 1, r = face;
    const float den = g2c(a, a.gz, j, r) * cellc(a, a.rf, f, j, r) + g2c(a, a.gz, j, l) * cellc(a, a.rf, f, j, l);
    const float kval = cellc(a, a.kmh, f, j, r) + cellc(a, a.kmh, f, j, l);
    const float gr = g2c(a, a.rgz, j, r), gl = g2c(a, a.rgz, j, l);
    float term = (cellc(a, a.t, f, j, r) * gr - cellc(a, a.t, f, j, l) * gl) * a.rdx;
    const float up = (a.zt - ((float)f + 0.5f) * a.dz) * (tsm(a, f, j, l) + tsm(a, f, j, r));
    const float lo = (a.zt - ((float)f - 0.5f) * a.dz) * (tsm(a, f - 1, j, l) + tsm(a, f - 1, j, r));
    term = term + 0.5f * ((up - lo) * (a.rdz * ((gr - gl) * a.rdx)));
    return -0.25f * (den * (2.0f * (kval * term)));
}

// y TKE flux at face level f, v face `face`, column i
__device__ float tke_ty(const TkeArgs &a, int f, int face, int i) {
    if (f <= 0 || f >= a.nk) return 0.0f;
    const int s = face - 1, n = face;
    const float den = g2c(a, a.gz, n, i) * cellc(a, a.rf, f, n, i) + g2c(a, a.gz, s, i) * cellc(a, a.rf, f, s, i);
    const float kval = cellc(a, a.kmh, f, n, i) + cellc(a, a.kmh, f, s, i);
    const float gn = g2c(a, a.rgz, n, i), gs = g2c(a, a.rgz, s, i);
    float term = (cellc(a, a.t, f, n, i) * gn - cellc(a, a.t, f, s, i) * gs) * a.rdy;
    const float up = (a.zt - ((float)f + 0.5f) * a.dz) * (tsm(a, f, s, i) + tsm(a, f, n, i));
    const float lo = (a.zt - ((float)f - 0.5f) * a.dz) * (tsm(a, f - 1, s, i) + tsm(a, f - 1, n, i));
    term = term + 0.5f * ((up - lo) * (a.rdz * ((gn - gs) * a.rdy)));
    return -0.25f * (den * (2.0f * (kval * term)));
}

// dynamic shared memory: cp and dp (the latter becomes the solution), each
// (nk-1) levels x kTT columns
__global__ void __launch_bounds__(kTT) tke_turbt_kernel(TkeArgs a, float dt) {
    extern __shared__ float s_col[];
    __shared__ float s_tx[4][kTTY][kTTX + 1];
    __shared__ float s_ty[4][kTTY + 1][kTTX];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTTX + tx;
    const int i0 = blockIdx.x * kTTX, j0 = blockIdx.y * kTTY;
    const int i = i0 + tx, j = j0 + ty;
    const int ni = a.ni, nj = a.nj, nk = a.nk, n = nk - 1;
    const bool own = i < ni && j < nj;
    float *cp = s_col, *dp = s_col + (size_t)n * kTT;
#define CP(p) cp[(unsigned)(p) * kTT + tid]
#define DP(p) dp[(unsigned)(p) * kTT + tid]
    const float rdt = 1.0f / dt;
    // ---- vertically implicit diffusion of the own column -------------------
    if (own) {
        const float tema = -1.0f * (dt * (a.rdz * a.rdz));
        int f = 1;
        unsigned z = f3(a, f, j, i);
        float rrf = a.mf[z] / a.rf[z];
        float r2 = (a.kmv[z] + a.kmv[f3(a, f + 1, j, i)]) * (a.mh[f3(a, f, j, i)] * (a.rho[f3(a, f, j, i)] * rrf));
        float cfc = tema * r2, cfb = 1.0f - cfc, inv = rcp_rn(cfb);
        float cprev = -1.0f * (cfc * inv), dprev = a.t[z] * inv;
        CP(0) = cprev;
        DP(0) = dprev;
        // kmv(f-1), kmv(f), mh(f-1) and rho(f-1) of the level being
        // eliminated ride in registers; each chunk of kTTChunk levels issues
        // all of its loads before its first elimination, so their latency is
        // paid once per chunk rather than once per level (same operations,
        // same order)
        float km1 = a.kmv[z], k0 = a.kmv[f3(a, 2, j, i)], mhm = a.mh[z], rhom = a.rho[z];
        for (int p0 = 1; p0 < n - 1; p0 += kTTChunk) {
            float lkn[kTTChunk], lmh[kTTChunk], lrho[kTTChunk], lmf[kTTChunk], lrf[kTTChunk], lt[kTTChunk];
#pragma unroll
            for (int q = 0; q < kTTChunk; ++q) {
                lkn[q] = lmh[q] = lrho[q] = lt[q] = 0.0f;
                lmf[q] = lrf[q] = 1.0f;
                if (p0 + q >= n - 1) continue;
                const unsigned zq = f3(a, p0 + q + 1, j, i);
                lkn[q] = a.kmv[f3(a, p0 + q + 2, j, i)];
                lmh[q] = a.mh[zq];
                lrho[q] = a.rho[zq];
                lmf[q] = a.mf[zq];
                lrf[q] = a.rf[zq];
                lt[q] = a.t[zq];
            }
#pragma unroll
            for (int q = 0; q < kTTChunk; ++q) {
                const int p = p0 + q;
                if (p >= n - 1) break;
                rrf = lmf[q] / lrf[q];
                const float r1 = (km1 + k0) * (mhm * (rhom * rrf));
                r2 = (k0 + lkn[q]) * (lmh[q] * (lrho[q] * rrf));
                const float cfa = tema * r1;
                cfc = tema * r2;
                cfb = (1.0f - cfa) - cfc;
                inv = rcp_rn(cfa * cprev + cfb);
                cprev = -1.0f * (cfc * inv);
                dprev = (lt[q] - cfa * dprev) * inv;
                CP(p) = cprev;
                DP(p) = dprev;
                km1 = k0, k0 = lkn[q], mhm = lmh[q], rhom = lrho[q];
            }
        }
        f = nk - 1;
        z = f3(a, f, j, i);
        rrf = a.mf[z] / a.rf[z];
        const float r1 = (km1 + k0) * (mhm * (rhom * rrf));
        const float cfa = tema * r1;
        cfb = 1.0f - cfa;
        float sol = (a.t[z] - cfa * DP(n - 2)) * rcp_rn(cfa * CP(n - 2) + cfb);
        DP(n - 1) = sol;
        for (int p = n - 2; p >= 0; --p) {
            sol = CP(p) * sol + DP(p);
            DP(p) = sol;
        }
    }
    // ---- horizontal divergence, walking the face levels --------------------
    // Four level slots: while level f is formed from slots f-1, f, f+1, this
    // thread's share of level f+2's face terms is evaluated into registers
    // (its loads in flight during the level's arithmetic) and stored into the
    // fourth slot, which no thread reads until after the closing barrier.
    constexpr int kXF = kTTY * (kTTX + 1), kYF = (kTTY + 1) * kTTX;
    constexpr int kXE = (kXF + kTT - 1) / kTT, kYE = (kYF + kTT - 1) / kTT;
    float rx[kXE], ry[kYE];
    auto eval = [&](int lev) {
#pragma unroll
        for (int q2 = 0; q2 < kXE; ++q2) {
            const int e = tid + q2 * kTT, r = e / (kTTX + 1), q = e - r * (kTTX + 1);
            rx[q2] = (e < kXF && j0 + r < nj && i0 + q <= ni) ? tke_tx(a, lev, j0 + r, i0 + q) : 0.0f;
        }
#pragma unroll
        for (int q2 = 0; q2 < kYE; ++q2) {
            const int e = tid + q2 * kTT, r = e / kTTX, q = e - r * kTTX;
            ry[q2] = (e < kYF && j0 + r <= nj && i0 + q < ni) ? tke_ty(a, lev, j0 + r, i0 + q) : 0.0f;
        }
    };
    auto store = [&](int lev) {
        const int slot = lev % 4;
#pragma unroll
        for (int q2 = 0; q2 < kXE; ++q2) {
            const int e = tid + q2 * kTT, r = e / (kTTX + 1), q = e - r * (kTTX + 1);
            if (e < kXF) s_tx[slot][r][q] = rx[q2];
        }
#pragma unroll
        for (int q2 = 0; q2 < kYE; ++q2) {
            const int e = tid + q2 * kTT, r = e / kTTX, q = e - r * kTTX;
            if (e < kYF) s_ty[slot][r][q] = ry[q2];
        }
    };
    for (int lev = 0; lev <= 2 && lev <= nk; ++lev) {
        eval(lev);
        store(lev);
    }
    __syncthreads();
    float gzji = 0.0f, ru0 = 0.0f, ru1 = 0.0f, rv0 = 0.0f, rv1 = 0.0f;
    if (own) {
        gzji = a.gz[(size_t)j * ni + i];
        ru0 = a.rgzu[(size_t)j * (ni + 1) + i];
        ru1 = a.rgzu[(size_t)j * (ni + 1) + i + 1];
        rv0 = a.rgzv[(size_t)j * ni + i];
        rv1 = a.rgzv[(size_t)(j + 1) * ni + i];
    }
    for (int f = 1; f < nk; ++f) {
        const bool ahead = f + 2 <= nk;
        if (ahead) eval(f + 2);
        if (own) {
            const int cm = (f - 1) % 4, c0 = f % 4, cpl = (f + 1) % 4;
            const float x0 = s_tx[c0][ty][tx], x1 = s_tx[c0][ty][tx + 1];
            float x = -1.0f * ((x1 * ru1 - x0 * ru0) * (gzji * a.rdx));
            const float sxf0 = 0.5f * (x0 + s_tx[cpl][ty][tx]), sxf1 = 0.5f * (x1 + s_tx[cpl][ty][tx + 1]);
            const float sxm0 = 0.5f * (s_tx[cm][ty][tx] + x0), sxm1 = 0.5f * (s_tx[cm][ty][tx + 1] + x1);
            float up = (a.zt - ((float)f + 0.5f) * a.dz) * (sxf0 + sxf1);
            float lo = (a.zt - ((float)f - 0.5f) * a.dz) * (sxm0 + sxm1);
            x = x - 0.5f * ((up - lo) * (a.rdz * ((ru1 - ru0) * (gzji * a.rdx))));
            const float y0 = s_ty[c0][ty][tx], y1 = s_ty[c0][ty + 1][tx];
            float y = -1.0f * ((y1 * rv1 - y0 * rv0) * (gzji * a.rdy));
            const float syf0 = 0.5f * (y0 + s_ty[cpl][ty][tx]), syf1 = 0.5f * (y1 + s_ty[cpl][ty + 1][tx]);
            const float sym0 = 0.5f * (s_ty[cm][ty][tx] + y0), sym1 = 0.5f * (s_ty[cm][ty + 1][tx] + y1);
            up = (a.zt - ((float)f + 0.5f) * a.dz) * (syf0 + syf1);
            lo = (a.zt - ((float)f - 0.5f) * a.dz) * (sym0 + sym1);
            y = y - 0.5f * ((up - lo) * (a.rdz * ((rv1 - rv0) * (gzji * a.rdy))));
            const float hx = (i == 0 || i == ni - 1) ? 0.0f : x;
            const float hy = (j == 0 || j == nj - 1) ? 0.0f : y;
            const unsigned z = f3(a, f, j, i);
            const float rfz = a.rf[z];
            const float vz = rfz * ((DP(f - 1) - a.t[z]) * rdt);
            a.tketen[z] = a.tketen[z] + ((hx + hy) + vz) / rfz;
        }
        if (ahead) store(f + 2);
        __syncthreads();
    }
#undef CP
#undef DP
}

// ------------------------------------------------- turbt, flat column
// gm1_flat_turbt_v1 (src/cm1core/cuda_gm1_flat_stretched_closure.py:314-359;
// turbtend.F:729-1044 with terrain_flag=.false.): the x/y face fluxes
// -0.25*(rf(a)+rf(a-1))*2*(kmh(a)+kmh(a-1))*(t(a)-t(a-1))*rdx, no terrain
// correction, and the implicit diffusion with rdz and the 3-D mh/mf.  One
// CTA per 32 x 4 column tile: the own column's Thomas in shared memory, then
// per face level the tile's face fluxes (each formed once) in shared memory.

// x face flux at face level f, row j, between cells face-1 and face
__device__ __forceinline__ float tke_tx_flat(const TkeArgs &a, int f, int j, int face) {
    const float rs = cellc(a, a.rf, f, j, face) + cellc(a, a.rf, f, j, face - 1);
    const float ks = cellc(a, a.kmh, f, j, face) + cellc(a, a.kmh, f, j, face - 1);
    const float dt = cellc(a, a.t, f, j, face) - cellc(a, a.t, f, j, face - 1);
    return -(((((0.25f * rs) * 2.0f) * ks) * dt) * a.rdx);
}
__device__ __forceinline__ float tke_ty_flat(const TkeArgs &a, int f, int face, int i) {
    const float rs = cellc(a, a.rf, f, face, i) + cellc(a, a.rf, f, face - 1, i);
    const float ks = cellc(a, a.kmh, f, face, i) + cellc(a, a.kmh, f, face - 1, i);
    const float dt = cellc(a, a.t, f, face, i) - cellc(a, a.t, f, face - 1, i);
    return -(((((0.25f * rs) * 2.0f) * ks) * dt) * a.rdy);
}

__global__ void __launch_bounds__(kTT) tke_turbt_flat_kernel(TkeArgs a, float dt) {
    extern __shared__ float s_col[];
    __shared__ float s_tx[kTTY][kTTX + 1];
    __shared__ float s_ty[kTTY + 1][kTTX];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTTX + tx;
    const int i0 = blockIdx.x * kTTX, j0 = blockIdx.y * kTTY;
    const int i = i0 + tx, j = j0 + ty;
    const int ni = a.ni, nj = a.nj, nk = a.nk, n = nk - 1;
    const bool own = i < ni && j < nj;
    float *cp = s_col, *dp = s_col + (size_t)n * kTT;
#define CP(p) cp[(unsigned)(p) * kTT + tid]
#define DP(p) dp[(unsigned)(p) * kTT + tid]
    const float rdt = 1.0f / dt;
    if (own) {
        const float tema = (((-1.0f * dt) * 1.0f) * a.rdz) * a.rdz;
        const float temb = ((dt * 0.0f) * a.rdz) * a.rdz;
        // level f = 1
        unsigned z = f3(a, 1, j, i);
        float tprev = a.t[z], tcur = a.t[f3(a, 2, j, i)];
        float rrf = a.mf[z] / a.rf[z];
        float kprev = a.kmv[z], kcur = a.kmv[f3(a, 2, j, i)];
        float r2 = (((kprev + kcur) * a.mh[z]) * a.rho[z]) * rrf;
        float cfc = tema * r2, cfb = 1.0f - cfc;
        float cfd = tprev + temb * ((r2 * tcur) - (r2 * tprev));
        float inv = rcp_rn(cfb);
        float cprev = -(cfc * inv), dprev = cfd * inv;
        CP(0) = cprev;
        DP(0) = dprev;
        float tm = tprev;  // t(f-1)
        // levels f = 2 .. nk-2
        for (int f = 2; f < nk - 1; ++f) {
            const unsigned zf = f3(a, f, j, i), zm = f3(a, f - 1, j, i);
            const float tp = a.t[f3(a, f + 1, j, i)];
            const float knext = a.kmv[f3(a, f + 1, j, i)];
            rrf = a.mf[zf] / a.rf[zf];
            const float r1 = (((kprev + kcur) * a.mh[zm]) * a.rho[zm]) * rrf;
            r2 = (((kcur + knext) * a.mh[zf]) * a.rho[zf]) * rrf;
            const float cfa = tema * r1;
            cfc = tema * r2;
            cfb = (1.0f - cfa) - cfc;
            const float tf = tcur;
            cfd = tf + temb * (((r2 * tp) - ((r1 + r2) * tf)) + (r1 * tm));
            inv = rcp_rn(cfa * cprev + cfb);
            cprev = -(cfc * inv);
            dprev = (cfd - cfa * dprev) * inv;
            CP(f - 1) = cprev;
            DP(f - 1) = dprev;
            tm = tf;
            tcur = tp;
            kprev = kcur;
            kcur = knext;
        }
        // level f = nk-1
        {
            const int f = nk - 1;
            const unsigned zf = f3(a, f, j, i), zm = f3(a, f - 1, j, i);
            rrf = a.mf[zf] / a.rf[zf];
            const float r1 = (((kprev + kcur) * a.mh[zm]) * a.rho[zm]) * rrf;
            const float cfa = tema * r1;
            cfb = 1.0f - cfa;
            const float tf = tcur;
            cfd = tf + temb * ((-(r1 * tf)) + (r1 * tm));
            inv = rcp_rn(cfa * cprev + cfb);
            float sol = (cfd - cfa * dprev) * inv;
            DP(n - 1) = sol;
            for (int p = n - 2; p >= 0; --p) {
                sol = CP(p) * sol + DP(p);
                DP(p) = sol;
            }
        }
    }
    constexpr int kXF = kTTY * (kTTX + 1), kYF = (kTTY + 1) * kTTX;
    for (int f = 1; f < nk; ++f) {
        for (int e = tid; e < kXF; e += kTT) {
            const int r = e / (kTTX + 1), q = e - r * (kTTX + 1);
            if (j0 + r < nj && i0 + q <= ni) s_tx[r][q] = tke_tx_flat(a, f, j0 + r, i0 + q);
        }
        for (int e = tid; e < kYF; e += kTT) {
            const int r = e / kTTX, q = e - r * kTTX;
            if (j0 + r <= nj && i0 + q < ni) s_ty[r][q] = tke_ty_flat(a, f, j0 + r, i0 + q);
        }
        __syncthreads();
        if (own) {
            const float hx = (i == 0 || i == ni - 1) ? 0.0f : -((s_tx[ty][tx + 1] - s_tx[ty][tx]) * a.rdx);
            const float hy = (j == 0 || j == nj - 1) ? 0.0f : -((s_ty[ty + 1][tx] - s_ty[ty][tx]) * a.rdy);
            const unsigned z = f3(a, f, j, i);
            const float rfz = a.rf[z];
            const float tz = (rfz * (DP(f - 1) - a.t[z])) * rdt;
            a.tketen[z] = a.tketen[z] + ((hx + hy) + tz) / rfz;
        }
        __syncthreads();
    }
#undef CP
#undef DP
}

// ------------------------------------------------------------- RK stage
__device__ __forceinline__ float rru_at(const TkeArgs &a, int k, int j, int f) {
    return a.rru[((unsigned)k * (unsigned)(a.nj + 2 * kG) + (unsigned)(j + kG)) * (unsigned)(a.ni + 1 + 2 * kG) +
                 (unsigned)(f + kG)];
}
__device__ __forceinline__ float rrv_at(const TkeArgs &a, int k, int f, int i) {
    return a.rrv[((unsigned)k * (unsigned)(a.nj + 1 + 2 * kG) + (unsigned)(f + kG)) * (unsigned)(a.ni + 2 * kG) +
                 (unsigned)(i + kG)];
}
__device__ __forceinline__ float rrw_at(const TkeArgs &a, int k, int j, int i) {
    return a.rrw[((unsigned)k * (unsigned)(a.nj + 2 * kG) + (unsigned)(j + kG)) * (unsigned)(a.ni + 2 * kG) +
                 (unsigned)(i + kG)];
}

// mass flux through x face `face` of row j (axis 0) or y face `face` of
// column `row` (axis 1) at face level f
__device__ __forceinline__ float face_mass(const TkeArgs &a, int axis, int f, int row, int face) {
    if (axis == 0) {
        const float c2 = 0.5f * (cellc(a, a.c2, f, row, face - 1) + cellc(a, a.c2, f, row, face));
        return c2 * rru_at(a, f + 1, row, face) + (1.0f - c2) * rru_at(a, f, row, face);
    }
    const float c2 = 0.5f * (cellc(a, a.c2, f, face - 1, row) + cellc(a, a.c2, f, face, row));
    return c2 * rrv_at(a, f + 1, face, row) + (1.0f - c2) * rrv_at(a, f, face, row);
}

template <bool W>
__device__ __forceinline__ float rec5(float s1, float s2, float s3, float s4, float s5, double eps) {
    if (W) return weno5(s1, s2, s3, s4, s5, eps);
    return flx5(s1, s2, s3, s4, s5);
}

// face flux with its own mass (no open-side substitution)
template <bool W>
__device__ float face_flux_plain(const TkeArgs &a, const float *q, int axis, int f, int row, int face, double eps) {
    const float m = face_mass(a, axis, f, row, face);
    float v[5];
    const int sgn = m >= 0.0f ? 1 : -1;
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        const int off = sgn > 0 ? s - 3 : 2 - s;
        v[s] = axis == 0 ? cellc(a, q, f, row, face + off) : cellc(a, q, f, face + off, row);
    }
    return m * rec5<W>(v[0], v[1], v[2], v[3], v[4], eps);
}

// face flux with the open-side substitution: inflow through the first face
// (or the last face) takes the flux of its inner neighbour face; the mass
// returned is the face's own
template <bool W>
__device__ float face_flux(const TkeArgs &a, const float *q, int axis, int f, int row, int face, double eps,
                           float *mass) {
    const int n = axis == 0 ? a.ni : a.nj;
    const float m = face_mass(a, axis, f, row, face);
    *mass = m;
    if (face == 0 && m >= 0.0f) return face_flux_plain<W>(a, q, axis, f, row, 1, eps);
    if (face == n && m <= 0.0f) return face_flux_plain<W>(a, q, axis, f, row, n - 1, eps);
    float v[5];
    const int sgn = m >= 0.0f ? 1 : -1;
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        const int off = sgn > 0 ? s - 3 : 2 - s;
        v[s] = axis == 0 ? cellc(a, q, f, row, face + off) : cellc(a, q, f, face + off, row);
    }
    return m * rec5<W>(v[0], v[1], v[2], v[3], v[4], eps);
}

// vertical flux at staggered index ks (cuda_tke_evolution.py:194-203)
template <bool W>
__device__ float vert_flux(const TkeArgs &a, const float *q, int ks, int j, int i, double eps) {
    const int nk = a.nk;
    const float m = 0.5f * (rrw_at(a, ks, j, i) + rrw_at(a, ks + 1, j, i));
    const float wf = (float)eps;
#define Q(k) q[f3(a, (k), j, i)]
    float r;
    if (ks == 1) {
        r = m >= 0.0f ? 0.5f * (Q(0) + Q(1)) : (W ? upstrpd(Q(2), Q(1), Q(0), wf) : flx3(Q(2), Q(1), Q(0)));
    } else if (ks == 2) {
        r = m >= 0.0f ? (W ? upstrpd(Q(0), Q(1), Q(2), wf) : flx3(Q(0), Q(1), Q(2)))
                      : rec5<W>(Q(4), Q(3), Q(2), Q(1), Q(0), eps);
    } else if (ks == nk - 1) {
        r = (W ? m > 0.0f : m >= 0.0f) ? rec5<W>(Q(ks - 3), Q(ks - 2), Q(ks - 1), Q(ks), Q(ks + 1), eps)
                                       : (W ? upstrpd(Q(ks + 1), Q(ks), Q(ks - 1), wf) : flx3(Q(ks + 1), Q(ks), Q(ks - 1)));
    } else if (ks == nk) {
        r = (W ? m > 0.0f : m >= 0.0f) ? (W ? upstrpd(Q(nk - 2), Q(nk - 1), Q(nk), wf) : flx3(Q(nk - 2), Q(nk - 1), Q(nk)))
                                       : 0.5f * (Q(nk - 1) + Q(nk));
    } else if (m >= 0.0f) {
        r = rec5<W>(Q(ks - 3), Q(ks - 2), Q(ks - 1), Q(ks), Q(ks + 1), eps);
    } else {
        r = rec5<W>(Q(ks + 2), Q(ks + 1), Q(ks), Q(ks - 1), Q(ks - 2), eps);
    }
#undef Q
    return m * r;
}

// grid: x over i, y over j, z over face level f = 0..nk; nxt2 optional.
// FLAT: the flat column's advw (gm1_flat_tke_advw_rk_v1,
// src/cm1core/cuda_gm1_flat_stretched_closure.py:401-449; adv.F:3252-3355
// with terrain_flag=.false.): vertical divergence -(dumz(k)-dumz(k-1))*rdz
// *mf(k), the column's c1/c2 in the divergence correction and its rrf0, the
// open-side divergence piece (q*d)*rdx evaluated left to right, no gz.
template <bool W, bool FLAT>
__global__ void __launch_bounds__(128) tke_rk_stage_kernel(TkeArgs a, const float *__restrict__ cur,
                                                           float *__restrict__ nxt, float *__restrict__ nxt2,
                                                           float dttmp, double eps) {
    // The x face fluxes pass to the next lane by warp shuffle and the y face
    // fluxes to the next warp row through shared memory (the last lane or row
    // forms its outer one itself): each face flux is formed once, by the same
    // function of the same arguments.
    __shared__ float s_fy[4][32], s_my[4][32];
    const int lane = threadIdx.x, row = threadIdx.y;
    const int i = blockIdx.x * 32 + lane, j = blockIdx.y * 4 + row, f = blockIdx.z;
    const int ni = a.ni, nj = a.nj, nk = a.nk;
    const bool inner = f > 0 && f < nk;  // uniform over the block
    float mw = 0.0f, me = 0.0f, ms = 0.0f, mn = 0.0f, fx0 = 0.0f, fx1 = 0.0f, fy0 = 0.0f, fy1 = 0.0f;
    if (inner) {
        if (j < nj && i <= ni) fx0 = face_flux<W>(a, cur, 0, f, j, i, eps, &mw);
        fx1 = __shfl_down_sync(0xffffffffu, fx0, 1);
        me = __shfl_down_sync(0xffffffffu, mw, 1);
        if (lane == 31 && j < nj && i < ni) fx1 = face_flux<W>(a, cur, 0, f, j, i + 1, eps, &me);
        if (i < ni && j <= nj) fy0 = face_flux<W>(a, cur, 1, f, i, j, eps, &ms);
        s_fy[row][lane] = fy0;
        s_my[row][lane] = ms;
    }
    __syncthreads();
    if (inner && row < 3) {
        fy1 = s_fy[row + 1][lane];
        mn = s_my[row + 1][lane];
    }
    if (i >= ni || j >= nj) return;
    const unsigned z = f3(a, f, j, i);
    if (!inner) {
        nxt[z] = 0.0f;
        if (nxt2) nxt2[z] = 0.0f;
        return;
    }
    if (row == 3) fy1 = face_flux<W>(a, cur, 1, f, i, j + 1, eps, &mn);
    float ax = -1.0f * ((fx1 - fx0) * a.rdx);
    float ay = -1.0f * ((fy1 - fy0) * a.rdy);
    const float c2 = a.c2[z], c1 = 1.0f - c2;
    const float q = cur[z];
    if ((i == 0 && mw >= 0.0f) || (i == ni - 1 && me <= 0.0f)) {
        const float du = c1 * (rru_at(a, f, j, i + 1) - rru_at(a, f, j, i)) +
                         c2 * (rru_at(a, f + 1, j, i + 1) - rru_at(a, f + 1, j, i));
        ax = FLAT ? ax - ((q * du) * a.rdx) : ax - q * (du * a.rdx);
    }
    if ((j == 0 && ms >= 0.0f) || (j == nj - 1 && mn <= 0.0f)) {
        const float dv = c1 * (rrv_at(a, f, j + 1, i) - rrv_at(a, f, j, i)) +
                         c2 * (rrv_at(a, f + 1, j + 1, i) - rrv_at(a, f + 1, j, i));
        ay = FLAT ? ay - ((q * dv) * a.rdy) : ay - q * (dv * a.rdy);
    }
    const float dvf = vert_flux<W>(a, cur, f + 1, j, i, eps) - vert_flux<W>(a, cur, f, j, i, eps);
    const float az = FLAT ? ((-dvf) * a.rdz) * a.mfp[f + 1] : -1.0f * (dvf * a.rdz);
    float total = (ax + ay) + az;
    // the divergence correction: the flat text reads the column's c2 here
    // (the open-side pieces above read the cell's)
    const float c2d = FLAT ? a.c2[f3(a, f, 0, 0)] : c2, c1d = FLAT ? 1.0f - c2d : c1;
    total = total + q * (c2d * a.divx[f3(a, f, j, i)] + c1d * a.divx[f3(a, f - 1, j, i)]);
    const float wten = FLAT ? a.tketen[z] + total * a.rrf0[f3(a, f, 0, 0)]
                            : a.tketen[z] + total * (a.rrf0[z] * a.gz[(size_t)j * ni + i]);
    const float value = a.tkea[z] + dttmp * wten;
    const float out = value < 1e-10f ? 0.0f : value;
    nxt[z] = out;
    if (nxt2) nxt2[z] = out;
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

int tke_args(int ni, int nj, int nk, const gm1b_tke_evolution_arrays *s, float dx, float dy, float dz, float dt,
             TkeArgs &a, const char *what) {
    if (s == nullptr || ni < 3 || nj < 3 || nk < 6) {
        gm1b_set_error("%s: need arrays, ni >= 3, nj >= 3, nk >= 6", what);
        return GM1B_ERR_ARGUMENT;
    }
    if ((size_t)(nk + 3) * (size_t)(nj + 7) * (size_t)(ni + 7) >= ((size_t)1 << 31)) {
        gm1b_set_error("%s: a %dx%dx%d grid's padded arrays reach 2^31 words; the kernels index with 32-bit offsets",
                       what, ni, nj, nk);
        return GM1B_ERR_ARGUMENT;
    }
    const float v[4] = {dx, dy, dz, dt};
    for (float x : v)
        if (!(x > 0.0f) || !isfinite(x)) {
            gm1b_set_error("%s: dx, dy, dz, dt must be finite and > 0", what);
            return GM1B_ERR_ARGUMENT;
        }
    const void *need[] = {s->tkea, s->tke3d, s->tketen, s->kmh, s->kmv, s->rho, s->rf, s->mh, s->mf, s->gz,
                          s->rgz, s->rgzu, s->rgzv, s->c1, s->c2, s->rrf0, s->rru, s->rrv, s->rrw, s->divx};
    for (const void *q : need)
        if (q == nullptr) {
            gm1b_set_error("%s: a required array is NULL", what);
            return GM1B_ERR_ARGUMENT;
        }
    a.t = s->tke3d;
    a.kmh = s->kmh;
    a.kmv = s->kmv;
    a.rho = s->rho;
    a.rf = s->rf;
    a.mh = s->mh;
    a.mf = s->mf;
    a.gz = s->gz;
    a.rgz = s->rgz;
    a.rgzu = s->rgzu;
    a.rgzv = s->rgzv;
    a.tkea = s->tkea;
    a.c2 = s->c2;
    a.rrf0 = s->rrf0;
    a.rru = s->rru;
    a.rrv = s->rrv;
    a.rrw = s->rrw;
    a.divx = s->divx;
    a.tketen = s->tketen;
    a.ni = ni;
    a.nj = nj;
    a.nk = nk;
    a.rdx = 1.0f / dx;
    a.rdy = 1.0f / dy;
    a.rdz = 1.0f / dz;
    a.dz = dz;
    a.zt = (float)nk * dz;
    return GM1B_OK;
}

size_t turbt_smem(int nk) { return (size_t)2 * (nk - 1) * kTT * sizeof(float); }

int enqueue_diffusion(const TkeArgs &a, float dt, cudaStream_t st) {
    const size_t smem = turbt_smem(a.nk);
    if (smem > 200 * 1024) {
        gm1b_set_error("gm1b_tke_diffusion: nk=%d exceeds the column solve's shared memory (nk <= 201)", a.nk);
        return GM1B_ERR_ARGUMENT;
    }
    static size_t configured[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64 && configured[dev] < smem) {
        const cudaError_t e =
            cudaFuncSetAttribute(tke_turbt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) {
            cudaGetLastError();
            gm1b_set_error("cudaFuncSetAttribute(tke_turbt_kernel): %s", cudaGetErrorString(e));
            return GM1B_ERR_CUDA;
        }
        configured[dev] = 200 * 1024;
    }
    ProfScope ps("tke_turbt_kernel", st);
    tke_turbt_kernel<<<dim3((a.ni + kTTX - 1) / kTTX, (a.nj + kTTY - 1) / kTTY), dim3(kTTX, kTTY), smem, st>>>(a, dt);
    ps.stop();
    return launch_ok("tke_turbt_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

int enqueue_stage(const TkeArgs &a, const float *cur, float *nxt, float *nxt2, int nrk, float dt, cudaStream_t st) {
    const float dttmp = dt / (float)(4 - nrk);
    const double eps = (double)(100.0f * 1e-18f);
    const dim3 grid((a.ni + 31) / 32, (a.nj + 3) / 4, a.nk + 1), block(32, 4);
    ProfScope ps("tke_rk_stage_kernel", st);
    if (nrk == 3)
        tke_rk_stage_kernel<true, false><<<grid, block, 0, st>>>(a, cur, nxt, nxt2, dttmp, eps);
    else
        tke_rk_stage_kernel<false, false><<<grid, block, 0, st>>>(a, cur, nxt, nxt2, dttmp, eps);
    ps.stop();
    return launch_ok("tke_rk_stage_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

int enqueue_stage_flat(const TkeArgs &a, const float *cur, float *nxt, int nrk, float dt, cudaStream_t st) {
    const float dttmp = dt / (float)(4 - nrk);
    const double eps = (double)(100.0f * 1e-18f);
    const dim3 grid((a.ni + 31) / 32, (a.nj + 3) / 4, a.nk + 1), block(32, 4);
    ProfScope ps("tke_rk_stage_flat_kernel", st);
    if (nrk == 3)
        tke_rk_stage_kernel<true, true><<<grid, block, 0, st>>>(a, cur, nxt, nullptr, dttmp, eps);
    else
        tke_rk_stage_kernel<false, true><<<grid, block, 0, st>>>(a, cur, nxt, nullptr, dttmp, eps);
    ps.stop();
    return launch_ok("tke_rk_stage_flat_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

// Flat column arguments: the arrays the flat turbt and RK stage read.
int tke_args_flat(int ni, int nj, int nk, const gm1b_tke_evolution_arrays *s, float dx, float dy, float rdz,
                  float dt, TkeArgs &a, bool stage, const float *mf_profile, const char *what) {
    if (s == nullptr || ni < 3 || nj < 3 || nk < 6) {
        gm1b_set_error("%s: need arrays, ni >= 3, nj >= 3, nk >= 6", what);
        return GM1B_ERR_ARGUMENT;
    }
    if ((size_t)(nk + 3) * (size_t)(nj + 7) * (size_t)(ni + 7) >= ((size_t)1 << 31)) {
        gm1b_set_error("%s: a %dx%dx%d grid's padded arrays reach 2^31 words; the kernels index with 32-bit offsets",
                       what, ni, nj, nk);
        return GM1B_ERR_ARGUMENT;
    }
    const float v[4] = {dx, dy, rdz, dt};
    for (float x : v)
        if (!(x > 0.0f) || !isfinite(x)) {
            gm1b_set_error("%s: dx, dy, rdz, dt must be finite and > 0", what);
            return GM1B_ERR_ARGUMENT;
        }
    const void *turbt_need[] = {s->tke3d, s->tketen, s->kmh, s->kmv, s->rho, s->rf, s->mh, s->mf};
    const void *stage_need[] = {s->tkea, s->tketen, s->c2, s->rrf0, s->rru, s->rrv, s->rrw, s->divx, mf_profile};
    if (stage) {
        for (const void *q : stage_need)
            if (q == nullptr) {
                gm1b_set_error("%s: a required array is NULL", what);
                return GM1B_ERR_ARGUMENT;
            }
    } else {
        for (const void *q : turbt_need)
            if (q == nullptr) {
                gm1b_set_error("%s: a required array is NULL", what);
                return GM1B_ERR_ARGUMENT;
            }
    }
    a = TkeArgs{};
    a.t = s->tke3d;
    a.kmh = s->kmh;
    a.kmv = s->kmv;
    a.rho = s->rho;
    a.rf = s->rf;
    a.mh = s->mh;
    a.mf = s->mf;
    a.tkea = s->tkea;
    a.c2 = s->c2;
    a.rrf0 = s->rrf0;
    a.rru = s->rru;
    a.rrv = s->rrv;
    a.rrw = s->rrw;
    a.divx = s->divx;
    a.tketen = s->tketen;
    a.mfp = mf_profile;
    a.ni = ni;
    a.nj = nj;
    a.nk = nk;
    a.rdx = 1.0f / dx;
    a.rdy = 1.0f / dy;
    a.rdz = rdz;
    return GM1B_OK;
}

}  // namespace

extern "C" int32_t gm1b_tke_diffusion(int32_t ni, int32_t nj, int32_t nk, const gm1b_tke_evolution_arrays *arrays,
                                      float dx, float dy, float dz, float dt, void *stream) {
    TkeArgs a;
    const int r = tke_args(ni, nj, nk, arrays, dx, dy, dz, dt, a, "gm1b_tke_diffusion");
    if (r != GM1B_OK) return r;
    return enqueue_diffusion(a, dt, static_cast<cudaStream_t>(stream));
}

extern "C" int32_t gm1b_tke_diffusion_flat(int32_t ni, int32_t nj, int32_t nk,
                                           const gm1b_tke_evolution_arrays *arrays, float dx, float dy, float rdz,
                                           float dt, void *stream) {
    TkeArgs a;
    const int r = tke_args_flat(ni, nj, nk, arrays, dx, dy, rdz, dt, a, false, nullptr, "gm1b_tke_diffusion_flat");
    if (r != GM1B_OK) return r;
    const size_t smem = turbt_smem(nk);
    if (smem > 200 * 1024) {
        gm1b_set_error("gm1b_tke_diffusion_flat: nk=%d exceeds the column solve's shared memory (nk <= 201)", nk);
        return GM1B_ERR_ARGUMENT;
    }
    static size_t configured[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64 && configured[dev] < smem) {
        const cudaError_t e =
            cudaFuncSetAttribute(tke_turbt_flat_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) {
            cudaGetLastError();
            gm1b_set_error("cudaFuncSetAttribute(tke_turbt_flat_kernel): %s", cudaGetErrorString(e));
            return GM1B_ERR_CUDA;
        }
        configured[dev] = 200 * 1024;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("tke_turbt_flat_kernel", st);
    tke_turbt_flat_kernel<<<dim3((ni + kTTX - 1) / kTTX, (nj + kTTY - 1) / kTTY), dim3(kTTX, kTTY), smem, st>>>(a, dt);
    ps.stop();
    return launch_ok("tke_turbt_flat_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_tke_rk_stage_flat(int32_t ni, int32_t nj, int32_t nk,
                                          const gm1b_tke_evolution_arrays *arrays, const float *mf_profile,
                                          const float *cur, float *nxt, int32_t nrk, float dx, float dy, float rdz,
                                          float dt, void *stream) {
    TkeArgs a;
    const int r = tke_args_flat(ni, nj, nk, arrays, dx, dy, rdz, dt, a, true, mf_profile, "gm1b_tke_rk_stage_flat");
    if (r != GM1B_OK) return r;
    if (cur == nullptr || nxt == nullptr || cur == nxt || nrk < 1 || nrk > 3) {
        gm1b_set_error("gm1b_tke_rk_stage_flat: need distinct cur and nxt and nrk in 1..3");
        return GM1B_ERR_ARGUMENT;
    }
    return enqueue_stage_flat(a, cur, nxt, nrk, dt, static_cast<cudaStream_t>(stream));
}

extern "C" int32_t gm1b_tke_rk_stage(int32_t ni, int32_t nj, int32_t nk, const gm1b_tke_evolution_arrays *arrays,
                                     const float *cur, float *nxt, int32_t nrk, float dx, float dy, float dz, float dt,
                                     void *stream) {
    TkeArgs a;
    const int r = tke_args(ni, nj, nk, arrays, dx, dy, dz, dt, a, "gm1b_tke_rk_stage");
    if (r != GM1B_OK) return r;
    if (cur == nullptr || nxt == nullptr || cur == nxt || nrk < 1 || nrk > 3) {
        gm1b_set_error("gm1b_tke_rk_stage: need distinct cur and nxt and nrk in 1..3");
        return GM1B_ERR_ARGUMENT;
    }
    return enqueue_stage(a, cur, nxt, nullptr, nrk, dt, static_cast<cudaStream_t>(stream));
}

extern "C" int32_t gm1b_tke_evolution(int32_t ni, int32_t nj, int32_t nk, const gm1b_tke_evolution_arrays *arrays,
                                      float *workspace, float dx, float dy, float dz, float dt, void *stream) {
    TkeArgs a;
    const int r = tke_args(ni, nj, nk, arrays, dx, dy, dz, dt, a, "gm1b_tke_evolution");
    if (r != GM1B_OK) return r;
    if (workspace == nullptr) {
        gm1b_set_error("gm1b_tke_evolution: need a workspace of (nk+1)*nj*ni floats");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float *tke3d = arrays->tke3d, *tkea = arrays->tkea;
    int s = enqueue_diffusion(a, dt, st);
    // stage 1: tke3d -> workspace; stage 2: workspace -> tke3d; stage 3:
    // tke3d -> tkea (each cell reads only its own tkea word) and workspace
    if (s == GM1B_OK) s = enqueue_stage(a, tke3d, workspace, nullptr, 1, dt, st);
    if (s == GM1B_OK) s = enqueue_stage(a, workspace, tke3d, nullptr, 2, dt, st);
    if (s == GM1B_OK) s = enqueue_stage(a, tke3d, workspace, tkea, 3, dt, st);
    if (s != GM1B_OK) return s;
    const size_t bytes = (size_t)(nk + 1) * nj * ni * sizeof(float);
    const cudaError_t e = cudaMemcpyAsync(tke3d, workspace, bytes, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) {
        gm1b_set_error("gm1b_tke_evolution: commit copy: %s", cudaGetErrorString(e));
        return GM1B_ERR_CUDA;
    }
    return GM1B_OK;
}
