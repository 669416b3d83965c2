// periodic_stage_fused.cuh - the whole acoustic RK stage of the periodic lane
// (all nloop small steps: horizontal PGF of u and v, then the column solve)
// as ONE persistent cooperative kernel.  Included inside periodic_lane.cu's
// anonymous namespace; used for the benchmark path (no scratch outputs) when
// the grid of row tiles is co-resident and the stage state fits in shared
// memory (nk <= 44).
//
// Behaviour: identical, word for word, to sound_uv_kernel followed by
// sound_column_kernel for n = 1..nloop (cpu_sound3_periodic_stage_inplace,
// src/cm1core/cuda_sound3_periodic.py:824-1027): every float is formed by the
// same binary32 operations in the same order.
//
// Design (B200):
//  * one CTA owns the 32 columns (i0..i0+31) of one row j for the whole stage
//    and keeps their state in shared memory: u faces x = i0-1..i0+31, the v
//    faces north (y = j) and south (y = j-1) of its columns, w, pi', the rru /
//    rrv / rrw running sums, and every stage-constant input;
//  * the west u face and the south v faces belong to neighbouring CTAs; each
//    CTA carries its own copy of them, advanced with the same operations as the
//    owner's, so no CTA ever reads a face another CTA writes during the stage;
//  * the only data that crosses CTAs per small step is ppd (the filtered pi'
//    the next step's PGF reads at i-1, i+1, j-1, j+1).  It is double-buffered
//    through two acoustic scratch arrays (tri_aa, tri_bb), so one grid barrier
//    per small step orders it; the stage-final ppd (and its halo words, which
//    the multi-launch path leaves at the previous small step's values) goes
//    to ppd at the last small step;
//  * the faces CM1 also updates on halo rows / columns (u on row nj+1, v on
//    column ni+1, and v on row 0) are carried by the edge CTAs in shared
//    memory and only their rru / rrv words are written, since the stage-end
//    periodic fill overwrites their u / v words;
//  * the grid barrier is an arrive counter (64-bit, reset by sound_prep_kernel
//    in tri_residual words 0-1) with a bounded spin: after spin_limit polls
//    (a launch argument, kSpinLimit by default) a CTA records 1 in
//    tri_residual word 2 and in the caller's status word (when one is given),
//    and every CTA leaves the kernel at its next barrier.  The error word is
//    cleared only by the first fused stage of a library call, so after a
//    failure every later stage of the same call leaves at its first barrier.
//    The launch is cooperative, so all CTAs are co-resident.
//
// Shared-memory layout: arrays of L = nk+2 levels, 32 lanes (columns
// i0+lane), 33 faces (x = i0-1+q) or 34 columns (x = i0-1+q).

constexpr int kFusedThreads = kTX * kColWarps;  // 512
constexpr int kSpinLimit = 1 << 21;              // L2 round-trip polls: a second or more
constexpr int kFusedMaxNk = 44;                  // stage state of nk <= 44 fits one CTA
constexpr int kLoadTrips = 3;                    // ceil(34 * (kFusedMaxNk + 1) / kFusedThreads)

struct FusedArgs {
    int nrk, nloop;
    float dts, rdx, rdy, alph, beta, asq, kdiv, smeps, temx, temy, rnloop, tem1x, tem2y, tavg;
    int fill_pp3d, post_ppx;
    int spin_limit;  // barrier polls before a CTA gives up
    int *status;     // caller's status word (device, may be null): 1 once a barrier gave up
};

__host__ __device__ constexpr size_t fused_smem_floats(int nk) {
    return (size_t)(nk + 2) * (8 * 33 + 8 * 32 + 4 * 34 + 18 * 32 + 8);
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_volatile_i32(const int *p) { return *reinterpret_cast<const volatile int *>(p); }

// Bounded grid barrier; returns false (all threads) once any CTA gave up.
__device__ __forceinline__ bool fused_grid_sync(unsigned long long *ctr, int *err, unsigned long long target,
                                                int spin_limit, int *status) {
    __shared__ int s_fail;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        int fail = 0;
        __threadfence();
        atomicAdd(ctr, 1ull);
        for (int it = 0;; ++it) {
            if (ld_acquire_u64(ctr) >= target) break;
            if (ld_volatile_i32(err) != 0) {
                fail = 1;
                break;
            }
            if (it >= spin_limit) {
                atomicExch(err, 1);
                if (status != nullptr) atomicExch(status, 1);
                fail = 1;
                break;
            }
        }
        __threadfence();
        s_fail = fail;
    }
    __syncthreads();
    return s_fail == 0;
}

// Thomas sweep of one column whose levels sit 32 words apart in shared
// memory (pointers already offset to the column's lane), levels 2..nk
// (nk >= 3), in the operation order of the multi-launch column kernel.
// first: inv holds bb and ec holds cc on entry; the sweep replaces them with
// 1/pivot and the elimination coefficient, the stage constants that later
// small steps (first = false) reuse.  The reciprocal is rcp_rn (the word of __frcp_rn), the
// correctly rounded 1/x, i.e. the same word as 1.0f / x under IEEE division.
// Each level's operands are read one level ahead of its dependent chain.
__device__ __forceinline__ void column_sweep(int nk, bool first, const float *aa, float *inv, float *ec,
                                             const float *dd, float *ed, float *w) {
    constexpr int S = kTX;  // level stride
    float e;                // elimination right-hand side of the previous level
    if (first) {
        float c;  // elimination coefficient of the previous level
        {
            const float iv = rcp_rn(inv[2 * S]);
            inv[2 * S] = iv;
            c = (-ec[2 * S]) * iv;
            e = dd[2 * S] * iv;
            ec[2 * S] = c;
            ed[2 * S] = e;
        }
        float a_n = aa[3 * S], b_n = inv[3 * S], c_n = ec[3 * S], d_n = dd[3 * S];
        for (int k = 3; k < nk; ++k) {
            const float a_k = a_n, b_k = b_n, c_k = c_n, d_k = d_n;
            a_n = aa[(k + 1) * S];
            b_n = inv[(k + 1) * S];
            c_n = ec[(k + 1) * S];
            d_n = dd[(k + 1) * S];
            const float pivot = a_k * c + b_k;
            const float iv = rcp_rn(pivot);
            inv[k * S] = iv;
            const float num = d_k - a_k * e;
            c = (-c_k) * iv;
            e = num * iv;
            ec[k * S] = c;
            ed[k * S] = e;
        }
        const float pivot = a_n * c + b_n;
        const float iv = rcp_rn(pivot);
        inv[nk * S] = iv;
        w[nk * S] = (d_n - a_n * e) * iv;
    } else {
        e = dd[2 * S] * inv[2 * S];
        ed[2 * S] = e;
        float a_n = aa[3 * S], d_n = dd[3 * S], v_n = inv[3 * S];
#pragma unroll 4
        for (int k = 3; k < nk; ++k) {
            const float a_k = a_n, d_k = d_n, v_k = v_n;
            a_n = aa[(k + 1) * S];
            d_n = dd[(k + 1) * S];
            v_n = inv[(k + 1) * S];
            const float num = d_k - a_k * e;
            e = num * v_k;
            ed[k * S] = e;
        }
        w[nk * S] = (d_n - a_n * e) * v_n;
    }
    float wn = w[nk * S];
    float c_n = ec[(nk - 1) * S], e_n = ed[(nk - 1) * S];
#pragma unroll 4
    for (int k = nk - 1; k >= 2; --k) {
        const float c_k = c_n, e_k = e_n;
        c_n = ec[(k - 1) * S];
        e_n = ed[(k - 1) * S];
        wn = c_k * wn + e_k;
        w[k * S] = wn;
    }
}

__global__ void __launch_bounds__(kFusedThreads, 1) sound_stage_fused_kernel(Arr a, Dims d, FusedArgs p) {
    extern __shared__ float smem[];
    const int ni = d.ni, nj = d.nj, nk = d.nk;
    const int lane = threadIdx.x, wy = threadIdx.y;
    const int tid = wy * kTX + lane;
    const int i0 = blockIdx.x * kTX + 1;  // first live column of the tile
    const int j = blockIdx.y + 1;         // live row
    const int i = i0 + lane;
    const bool live = i <= ni;
    const bool first_tile = i0 == 1;
    const bool last_tile = i0 + kTX > ni;  // holds column ni
    const bool top_row = j == nj, bottom_row = j == 1;
    const int L = nk + 2;
    const int nlive = (ni - i0 + 1) < kTX ? (ni - i0 + 1) : kTX;  // live columns of the tile

    float *q33 = smem;
    float *sU = q33, *sUten = sU + L * 33, *sRru = sUten + L * 33, *sTu = sRru + L * 33;
    float *sUx = sTu + L * 33, *sUxten = sUx + L * 33, *sRrux = sUxten + L * 33, *sTux = sRrux + L * 33;
    float *q32 = sTux + L * 33;
    float *sV = q32, *sVten = sV + L * 32, *sRrv = sVten + L * 32, *sTv = sRrv + L * 32;
    float *sVs = sTv + L * 32, *sVsten = sVs + L * 32, *sRrvs = sVsten + L * 32, *sTvs = sRrvs + L * 32;
    float *q34 = sTvs + L * 32;
    float *sPpd = q34, *sPpdN = sPpd + L * 34, *sPpdS = sPpdN + L * 34, *sPia = sPpdS + L * 34;
    float *c32 = sPia + L * 34;
    float *sPiaN = c32, *sPiaS = sPiaN + L * 32, *sPpten = sPiaS + L * 32, *sPpterm = sPpten + L * 32;
    float *sA1 = sPpterm + L * 32, *sA2 = sA1 + L * 32, *sMm = sA2 + L * 32, *sWten = sMm + L * 32;
    float *sW = sWten + L * 32, *sPp = sW + L * 32, *sRrw = sPp + L * 32, *sFpk = sRrw + L * 32;
    float *sAa = sFpk + L * 32, *sDd = sAa + L * 32, *sInv = sDd + L * 32, *sEc = sInv + L * 32;
    float *sEd = sEc + L * 32, *sPpdPrev = sEd + L * 32;
    float *sVx = sPpdPrev + L * 32;  // [k*2 + r]: r = 0 row j, r = 1 row 0 (bottom row only)
    float *sVxten = sVx + L * 2, *sRrvx = sVxten + L * 2, *sTvx = sRrvx + L * 2;
#define F33(arr, k, q) arr[(k) * 33 + (q)]
#define F34(arr, k, q) arr[(k) * 34 + (q)]
#define F32(arr, k) arr[(k) * 32 + lane]
#define FX(arr, k, r) arr[(k) * 2 + (r)]

    unsigned long long *ctr = reinterpret_cast<unsigned long long *>(a.tri_residual);
    int *err = reinterpret_cast<int *>(a.tri_residual) + 2;

    // ---- stage load: stage constants and the stage-start state -------------
    // Fixed-trip unrolled loops, so every load of a thread is in flight at
    // once (global loads and shared stores never alias).
    // u faces of row j (and row nj+1 on the top row), x = i0-1+q
#pragma unroll
    for (int t = 0; t < kLoadTrips; ++t) {
        const int e = tid + t * kFusedThreads;
        if (e >= nk * 33) continue;
        const int k = 1 + e / 33, q = e - (k - 1) * 33;
        const int x = i0 - 1 + q;
        if (x > ni) continue;
        const size_t fu = d.u(k, j, x);
        F33(sU, k, q) = a.u3d[fu];
        F33(sUten, k, q) = a.uten[fu];
        F33(sRru, k, q) = a.rru[fu];
        F33(sTu, k, q) = a.thv[d.s(k, j, x + 1)] + a.thv[d.s(k, j, x)];
        if (top_row) {
            const size_t fx = d.u(k, nj + 1, x);
            F33(sUx, k, q) = a.u3d[fx];
            F33(sUxten, k, q) = a.uten[fx];
            F33(sRrux, k, q) = a.rru[fx];
            F33(sTux, k, q) = a.thv[d.s(k, nj + 1, x + 1)] + a.thv[d.s(k, nj + 1, x)];
        }
    }
    // 34-wide piadv row; 32-wide column state
#pragma unroll
    for (int t = 0; t < kLoadTrips; ++t) {
        const int e = tid + t * kFusedThreads;
        if (e >= nk * 34) continue;
        const int k = 1 + e / 34, q = e - (k - 1) * 34;
        const int x = i0 - 1 + q;
        if (x > ni + 1) continue;
        F34(sPia, k, q) = a.piadv[d.s(k, j, x)];
    }
    if (live) {
#pragma unroll
        for (int t = 0; t < kLoadTrips; ++t) {
            const int k = 1 + wy + t * kColWarps;
            if (k > nk + 1) continue;
            F32(sW, k) = a.w3d[d.w(k, j - 1, i - 1)];
            if (k > nk) continue;
            const size_t c = d.s(k, j, i);
            const size_t fv = d.v(k, j, i), fs = d.v(k, j - 1, i);
            F32(sV, k) = a.v3d[fv];
            F32(sVten, k) = a.vten[fv];
            F32(sRrv, k) = a.rrv[fv];
            F32(sTv, k) = a.thv[d.s(k, j + 1, i)] + a.thv[c];
            F32(sVs, k) = a.v3d[fs];
            F32(sVsten, k) = a.vten[fs];
            F32(sRrvs, k) = a.rrv[fs];
            F32(sTvs, k) = a.thv[c] + a.thv[d.s(k, j - 1, i)];
            F32(sPiaN, k) = a.piadv[d.s(k, j + 1, i)];
            F32(sPiaS, k) = a.piadv[d.s(k, j - 1, i)];
            F32(sPpten, k) = a.ppten[c];
            F32(sPpterm, k) = a.ppterm[c];
            const float qk = a.qk[c];
            F32(sA1, k) = a.pk1[c] + qk;
            F32(sA2, k) = a.pk2[c] - qk;
            F32(sMm, k) = a.mm[c];
            F32(sWten, k) = a.wten[d.w(k, j - 1, i - 1)];
            F32(sPp, k) = a.pp3d[c];
            F32(sRrw, k) = a.rrw[d.w(k, j - 1, i - 1)];
        }
    }
    // v faces on column ni+1 (last tile): rows j and, on the bottom row, 0
    if (last_tile && wy == 0) {
        for (int k = 1 + lane; k <= nk; k += kTX) {
            for (int r = 0; r < (bottom_row ? 2 : 1); ++r) {
                const int y = r == 0 ? j : 0;
                const size_t fv = d.v(k, y, ni + 1);
                FX(sVx, k, r) = a.v3d[fv];
                FX(sVxten, k, r) = a.vten[fv];
                FX(sRrvx, k, r) = a.rrv[fv];
                FX(sTvx, k, r) = a.thv[d.s(k, y + 1, ni + 1)] + a.thv[d.s(k, y, ni + 1)];
            }
        }
    }
    __syncthreads();
    // tridiagonal lower coefficient (stage constant)
    if (live) {
        for (int k = 2 + wy; k <= nk; k += kColWarps)
            F32(sAa, k) = (k >= 3) ? (-p.asq) * (F32(sMm, k) * F32(sA1, k - 1)) : 0.0f;
    }
    // per-thread face constants: dts*dtu0, uf of own face (q = lane+1) and,
    // on lane 0, of the west face (q = 0); dts*dtv0 and vf of the v faces
    const int xo = i0 + lane;  // own u face
    const float cu_own = live ? p.dts * a.dtu0[(size_t)j * (ni + 1) + xo] : 0.0f;
    const float uf_own = live ? a.uf[xo + 1] : 0.0f;
    const float cu_w = p.dts * a.dtu0[(size_t)j * (ni + 1) + (i0 - 1)];
    const float uf_w = a.uf[i0];
    const float cux_own = (live && top_row) ? p.dts * a.dtu0[(size_t)(nj + 1) * (ni + 1) + xo] : 0.0f;
    const float cux_w = top_row ? p.dts * a.dtu0[(size_t)(nj + 1) * (ni + 1) + (i0 - 1)] : 0.0f;
    const float cv_n = live ? p.dts * a.dtv0[(size_t)j * (ni + 2) + i] : 0.0f;
    const float cv_s = live ? p.dts * a.dtv0[(size_t)(j - 1) * (ni + 2) + i] : 0.0f;
    const float vf_n = a.vf[j + 1], vf_s = a.vf[j];
    const float cvx0 = last_tile ? p.dts * a.dtv0[(size_t)j * (ni + 2) + (ni + 1)] : 0.0f;
    const float cvx1 = (last_tile && bottom_row) ? p.dts * a.dtv0[(size_t)(ni + 1)] : 0.0f;
    const float vf_x1 = a.vf[1];
    const float uh_i = live ? a.uh[i] : 0.0f, vh_j = a.vh[j];

    for (int n = 1; n <= p.nloop; ++n) {
        const bool last = n == p.nloop;
        // Each warp loads the ppd words of its own levels: column q = lane+1
        // on every live lane, q = 0 on lane 0 and q = nlive+1 on the last live
        // lane, so the PGF below reads only words of its own warp.
        const float *rd = n == 1 ? a.ppd : ((n - 1) & 1 ? a.tri_aa : a.tri_bb);
#pragma unroll
        for (int t = 0; t < kLoadTrips; ++t) {
            const int k = 1 + wy + t * kColWarps;
            if (k > nk) continue;
            if (live) {
                const int q = lane + 1;
                F34(sPpd, k, q) = __ldcg(rd + d.s(k, j, i));
                F34(sPpdN, k, q) = __ldcg(rd + d.s(k, j + 1, i));
                F34(sPpdS, k, q) = __ldcg(rd + d.s(k, j - 1, i));
            }
            if (lane == 0 || lane == nlive - 1) {
                const int q = lane == 0 ? 0 : nlive + 1;
                const int x = i0 - 1 + q;
                F34(sPpd, k, q) = __ldcg(rd + d.s(k, j, x));
                F34(sPpdN, k, q) = __ldcg(rd + d.s(k, j + 1, x));
                F34(sPpdS, k, q) = __ldcg(rd + d.s(k, j - 1, x));
            }
            if (nlive == 1 && lane == 0) {  // a one-column tile: lane 0 also holds q = 2
                F34(sPpd, k, 2) = __ldcg(rd + d.s(k, j, i0 + 1));
                F34(sPpdN, k, 2) = __ldcg(rd + d.s(k, j + 1, i0 + 1));
                F34(sPpdS, k, 2) = __ldcg(rd + d.s(k, j - 1, i0 + 1));
            }
        }
        __syncwarp();
        // ---- part 1: horizontal PGF of u and v (sound_uv_kernel) -----------
        for (int k = 1 + wy; k <= nk; k += kColWarps) {
            if (live) {
                const int q = lane + 1;
                {  // own u face x = i
                    float pg = p.tem1x * (F34(sPpd, k, q + 1) - F34(sPpd, k, q));
                    pg = pg * uf_own;
                    pg = pg * F33(sTu, k, q);
                    const float un = F33(sU, k, q) + cu_own * (F33(sUten, k, q) - pg);
                    F33(sU, k, q) = un;
                    const float r = F33(sRru, k, q);
                    F33(sRru, k, q) = last ? (r + un) * p.tavg : r + un;
                }
                if (top_row) {  // u face on halo row nj+1
                    float pg = p.tem1x * (F34(sPpdN, k, q + 1) - F34(sPpdN, k, q));
                    pg = pg * uf_own;
                    pg = pg * F33(sTux, k, q);
                    const float un = F33(sUx, k, q) + cux_own * (F33(sUxten, k, q) - pg);
                    F33(sUx, k, q) = un;
                    const float r = F33(sRrux, k, q);
                    F33(sRrux, k, q) = last ? (r + un) * p.tavg : r + un;
                }
                {  // north v face y = j
                    float pg = p.tem2y * (F34(sPpdN, k, q) - F34(sPpd, k, q));
                    pg = pg * vf_n;
                    pg = pg * F32(sTv, k);
                    const float vn = F32(sV, k) + cv_n * (F32(sVten, k) - pg);
                    F32(sV, k) = vn;
                    const float r = F32(sRrv, k);
                    F32(sRrv, k) = last ? (r + vn) * p.tavg : r + vn;
                }
                {  // south v face y = j-1 (own on the bottom row, else a private copy)
                    float pg = p.tem2y * (F34(sPpd, k, q) - F34(sPpdS, k, q));
                    pg = pg * vf_s;
                    pg = pg * F32(sTvs, k);
                    const float vn = F32(sVs, k) + cv_s * (F32(sVsten, k) - pg);
                    F32(sVs, k) = vn;
                    const float r = F32(sRrvs, k);
                    F32(sRrvs, k) = last ? (r + vn) * p.tavg : r + vn;
                }
            }
            if (lane == 0) {  // west u face x = i0-1 (own when it is face 0)
                float pg = p.tem1x * (F34(sPpd, k, 1) - F34(sPpd, k, 0));
                pg = pg * uf_w;
                pg = pg * F33(sTu, k, 0);
                const float un = F33(sU, k, 0) + cu_w * (F33(sUten, k, 0) - pg);
                F33(sU, k, 0) = un;
                const float r = F33(sRru, k, 0);
                F33(sRru, k, 0) = last ? (r + un) * p.tavg : r + un;
                if (top_row && first_tile) {  // face 0 of halo row nj+1
                    float pgx = p.tem1x * (F34(sPpdN, k, 1) - F34(sPpdN, k, 0));
                    pgx = pgx * uf_w;
                    pgx = pgx * F33(sTux, k, 0);
                    const float ux = F33(sUx, k, 0) + cux_w * (F33(sUxten, k, 0) - pgx);
                    F33(sUx, k, 0) = ux;
                    const float rx = F33(sRrux, k, 0);
                    F33(sRrux, k, 0) = last ? (rx + ux) * p.tavg : rx + ux;
                }
            }
            if (last_tile && lane < (bottom_row ? 2 : 1)) {  // v faces on column ni+1
                const int r = lane;
                const int qx = ni + 1 - (i0 - 1);
                const float up = r == 0 ? F34(sPpdN, k, qx) : F34(sPpd, k, qx);
                const float dn = r == 0 ? F34(sPpd, k, qx) : F34(sPpdS, k, qx);
                float pg = p.tem2y * (up - dn);
                pg = pg * (r == 0 ? vf_n : vf_x1);
                pg = pg * FX(sTvx, k, r);
                const float vn = FX(sVx, k, r) + (r == 0 ? cvx0 : cvx1) * (FX(sVxten, k, r) - pg);
                FX(sVx, k, r) = vn;
                const float rr = FX(sRrvx, k, r);
                FX(sRrvx, k, r) = last ? (rr + vn) * p.tavg : rr + vn;
            }
        }
        __syncwarp();  // phase A reads the west face of lane-1 at the same level
        // ---- part 2, phase A: divergence, pi' advection, fpk ---------------
        if (live) {
            for (int k = 1 + wy; k <= nk; k += kColWarps) {
                const int q = lane + 1;
                const float uE = F33(sU, k, q), uW = F33(sU, k, q - 1);
                const float vN = F32(sV, k), vS = F32(sVs, k);
                const float du = ((uE - uW) * p.rdx) * uh_i;
                const float dv = ((vN - vS) * p.rdy) * vh_j;
                float div = du + dv;
                if (fabsf(div) < p.smeps) div = 0.0f;
                const float pc = F34(sPia, k, q);
                const float gxw = pc - F34(sPia, k, q - 1);
                const float gxe = F34(sPia, k, q + 1) - pc;
                const float gys = pc - F32(sPiaS, k);
                const float gyn = F32(sPiaN, k) - pc;
                float hx = uW * gxw + uE * gxe;
                hx = ((-hx) * p.temx) * uh_i;
                float hy = vS * gys + vN * gyn;
                hy = ((-hy) * p.temy) * vh_j;
                const float hp = hx + hy;
                const float src = p.dts * (F32(sPpten, k) - F32(sPpterm, k) * div);
                const float a1 = F32(sA1, k), a2 = F32(sA2, k);
                const float vert = F32(sW, k) * a1 + F32(sW, k + 1) * a2;
                F32(sFpk, k) = (src + hp) + p.beta * vert;
            }
        }
        __syncthreads();
        // ---- phase A2: right-hand side (and, at n = 1, bb and cc) ----------
        if (live) {
            for (int k = 2 + wy; k <= nk; k += kColWarps) {
                const float mm = F32(sMm, k);
                const float pd = F32(sPp, k) - F32(sPp, k - 1);
                const float fwk = p.dts * F32(sWten, k) + p.beta * ((-mm) * pd);
                const float upd = (F32(sPp, k) + F32(sFpk, k)) - (F32(sPp, k - 1) + F32(sFpk, k - 1));
                F32(sDd, k) = (F32(sW, k) + fwk) + p.alph * ((-mm) * upd);
                if (n == 1) {
                    F32(sEc, k) = (k < nk) ? (-p.asq) * ((-mm) * F32(sA2, k)) : 0.0f;  // cc
                    const float diag = (-F32(sA1, k)) + F32(sA2, k - 1);
                    F32(sInv, k) = 1.0f - p.asq * (mm * diag);  // bb
                }
            }
        }
        __syncthreads();
        // ---- phase B: Thomas sweep, one lane per column ---------------------
        if (wy == 0 && live)
            column_sweep(nk, n == 1, &F32(sAa, 0), &F32(sInv, 0), &F32(sEc, 0), &F32(sDd, 0), &F32(sEd, 0),
                         &F32(sW, 0));
        __syncthreads();
        // ---- phase C: pressure update, kdiv filter, averages, ppd exchange -
        if (live) {
            float *wr = last ? a.ppd : ((n & 1) ? a.tri_aa : a.tri_bb);
            const bool wrap_j0 = j == nj, wrap_j1 = j == 1, wrap_i0 = i == ni, wrap_i1 = i == 1;
            const int rows[3] = {j, wrap_j0 ? 0 : -1, wrap_j1 ? nj + 1 : -1};
            const int cols[3] = {i, wrap_i0 ? 0 : -1, wrap_i1 ? ni + 1 : -1};
            const bool halo_cell = wrap_j0 || wrap_j1 || wrap_i0 || wrap_i1;
            const bool write_ppx = p.nrk == 3 && last;
            for (int k = 1 + wy; k <= nk; k += kColWarps) {
                const size_t c = d.s(k, j, i);
                const float wk = F32(sW, k), wk1 = F32(sW, k + 1);
                const float old = F32(sPp, k);
                const float vert = wk * F32(sA1, k) + wk1 * F32(sA2, k);
                float upd = (old + F32(sFpk, k)) + p.alph * vert;
                if (fabsf(upd) < p.smeps) upd = 0.0f;
                const float ek = p.kdiv * (upd - old);
                const float ppd = upd + ek;
                F32(sPp, k) = upd;
                const float r = F32(sRrw, k);
                const float rrw = last ? (r + wk * p.alph) * p.rnloop : r + wk;
                F32(sRrw, k) = rrw;
                wr[c] = ppd;
                const float ppx = p.post_ppx ? (upd + ek) : ek;
                if (last) {
                    a.pp3d[c] = upd;
                    if (k >= 2) a.w3d[d.w(k, j - 1, i - 1)] = wk;
                    a.rrw[d.w(k, j - 1, i - 1)] = rrw;
                    if (write_ppx) a.ppx[c] = ppx;
                }
                if (halo_cell) {
                    const float prev = F32(sPpdPrev, k);
                    _Pragma("unroll") for (int rr = 0; rr < 3; ++rr) {
                        if (rows[rr] < 0) continue;
                        _Pragma("unroll") for (int qq = 0; qq < 3; ++qq) {
                            if (cols[qq] < 0 || (rr == 0 && qq == 0)) continue;
                            const size_t h = d.s(k, rows[rr], cols[qq]);
                            if (!last) {
                                wr[h] = ppd;
                            } else {
                                a.ppd[h] = prev;
                                if (p.fill_pp3d) a.pp3d[h] = upd;
                                if (write_ppx && p.post_ppx) a.ppx[h] = ppx;
                            }
                        }
                    }
                }
                F32(sPpdPrev, k) = ppd;
            }
        }
        if (!last) {
            const unsigned long long target = (unsigned long long)n * (gridDim.x * gridDim.y);
            if (!fused_grid_sync(ctr, err, target, p.spin_limit, p.status)) return;
        }
    }
    // ---- stage end: u, v, rru, rrv and the stage-end periodic u/v fill -----
    for (int k = 1 + wy; k <= nk; k += kColWarps) {
        if (live) {
            const int q = lane + 1;
            a.u3d[d.u(k, j, i)] = F33(sU, k, q);
            a.rru[d.u(k, j, i)] = F33(sRru, k, q);
            a.v3d[d.v(k, j, i)] = F32(sV, k);
            a.rrv[d.v(k, j, i)] = F32(sRrv, k);
            if (bottom_row) {
                a.v3d[d.v(k, 0, i)] = F32(sVs, k);
                a.rrv[d.v(k, 0, i)] = F32(sRrvs, k);
            }
            if (top_row) a.rru[d.u(k, nj + 1, i)] = F33(sRrux, k, q);
            // fill_periodic_uv_inplace, from the stage-final own faces
            if (j == nj) a.u3d[d.u(k, 0, i)] = F33(sU, k, q);
            if (j == 1) a.u3d[d.u(k, nj + 1, i)] = F33(sU, k, q);
            if (i == ni) a.v3d[d.v(k, j, 0)] = F32(sV, k);
            if (i == 1) a.v3d[d.v(k, j, ni + 1)] = F32(sV, k);
            if (i == ni && j == 1) a.v3d[d.v(k, 0, 0)] = F32(sVs, k);
            if (i == 1 && j == 1) a.v3d[d.v(k, 0, ni + 1)] = F32(sVs, k);
        }
        if (lane == 0 && first_tile) {  // face 0
            a.u3d[d.u(k, j, 0)] = F33(sU, k, 0);
            a.rru[d.u(k, j, 0)] = F33(sRru, k, 0);
            if (top_row) a.rru[d.u(k, nj + 1, 0)] = F33(sRrux, k, 0);
            if (j == nj) a.u3d[d.u(k, 0, 0)] = F33(sU, k, 0);
            if (j == 1) a.u3d[d.u(k, nj + 1, 0)] = F33(sU, k, 0);
        }
        if (last_tile && lane < (bottom_row ? 2 : 1)) {
            const int y = lane == 0 ? j : 0;
            a.rrv[d.v(k, y, ni + 1)] = FX(sRrvx, k, lane);
        }
    }
#undef F33
#undef F34
#undef F32
#undef FX
}
