// closure.cu - sm_100a kernels of the two inputs of the TKE source:
// deformation (CM1 calcdef, Cartesian terrain branch, four open sides) and
// the moist squared buoyancy frequency (CM1 calcnm, six-species ice-aware
// branch).
//
// Behaviour followed (reference file:line):
//   cpu_terrain_deformation_inplace   src/cm1core/cuda_terrain_deformation.py:234-736
//   enqueue_flat_calcdef (flat column) src/cm1core/cuda_gm1_flat_stretched_closure.py:524-553, texts :76-136
//   cpu_moist_nm_inplace              src/cm1core/cuda_moist_nm.py:292-396
//
// Design (B200):
//  * calcdef is one z-marching tiled kernel.  A 32 x 8 CTA owns a tile of
//    output columns and walks the face levels upwards; the strain components
//    at its cells (s11, s22, s33) ride in registers from one level to the
//    next, the corner shear s12 of the tile's 33 x 9 corners is built in
//    shared memory (two level buffers), and the face shears s13 (33 x 8) and
//    s23 (32 x 9) of the current face level are built in shared memory before
//    the tile's defv and defh are combined.  Every strain word is formed once
//    and nothing goes through device memory between stages (the reference
//    stores six scratch volumes and runs three launches).
//  * calcnm is elementwise per face level: each thread forms the cell
//    diagnostics of its own level and of the level below and the face value
//    between them, so columns need no serial walk; the branch counts are
//    reduced per CTA with __syncthreads_count before one atomicAdd.
//  * Arithmetic is binary32 one operation at a time in the reference's
//    order (the library is built with --fmad=false), so calcdef is
//    word-identical to the reference; calcnm passes through logf/expf.
#include "gm1b_common.cuh"

namespace gm1b {
namespace {

constexpr int kDX = 32, kDY = 8;  // calcdef tile

struct DefArgs {
    const float *u, *v, *w, *rho, *rf, *c1, *c2, *gz, *rgz, *rgzu, *rgzv, *gx, *gy;
    const float *mf3, *mhp;  // flat column: face mf (nk+1, nj, ni) and the mh profile (nk+2, CM1-indexed)
    float *defv, *defh;
    int ni, nj, nk;
    float rdx, rdy, rds, zt, dz;
    float rdz;  // flat column: the vertical coordinate's reference 1/dz
};

// 32-bit element offsets (the entry points refuse grids whose arrays reach
// 2^31 words)
__device__ __forceinline__ unsigned i3(int k, int j, int i, int ny, int nx) {
    return ((unsigned)k * (unsigned)ny + (unsigned)j) * (unsigned)nx + (unsigned)i;
}

// face-level value of a u- or v-shaped field (levels nk, rows ny, row nx)
__device__ __forceinline__ float atw(const float *q, int kf, int j, int i, int nk, int ny, int nx) {
    if (kf == 0) {
        float r = 1.875f * q[i3(0, j, i, ny, nx)];
        r = r + (-1.25f) * q[i3(1, j, i, ny, nx)];
        return r + 0.375f * q[i3(2, j, i, ny, nx)];
    }
    if (kf == nk) {
        float r = 1.875f * q[i3(nk - 1, j, i, ny, nx)];
        r = r + (-1.25f) * q[i3(nk - 2, j, i, ny, nx)];
        return r + 0.375f * q[i3(nk - 3, j, i, ny, nx)];
    }
    return 0.5f * (q[i3(kf - 1, j, i, ny, nx)] + q[i3(kf, j, i, ny, nx)]);
}

// s11, s22, s33 at mass level k, cell (j, i)
__device__ __forceinline__ void strain_diag(const DefArgs &p, int k, int j, int i, float &s11, float &s22, float &s33) {
    const int ni = p.ni, nj = p.nj, nk = p.nk, ux = ni + 1, vy = nj + 1;
    const unsigned c = i3(k, j, i, nj, ni);
    const float g = p.gz[(unsigned)j * ni + i], r = p.rho[c];
    float hor = g * (p.u[i3(k, j, i + 1, nj, ux)] * p.rgzu[(unsigned)j * ux + i + 1] -
                     p.u[i3(k, j, i, nj, ux)] * p.rgzu[(unsigned)j * ux + i]);
    hor = hor * p.rdx;
    float up = p.gx[i3(k + 1, j, i, nj, ni)] * (atw(p.u, k + 1, j, i, nk, nj, ux) + atw(p.u, k + 1, j, i + 1, nk, nj, ux));
    float lo = p.gx[c] * (atw(p.u, k, j, i, nk, nj, ux) + atw(p.u, k, j, i + 1, nk, nj, ux));
    float vert = ((up - lo) * 0.5f) * p.rds;
    s11 = (hor + vert) * r;
    hor = g * (p.v[i3(k, j + 1, i, vy, ni)] * p.rgzv[(unsigned)(j + 1) * ni + i] -
               p.v[i3(k, j, i, vy, ni)] * p.rgzv[(unsigned)j * ni + i]);
    hor = hor * p.rdy;
    up = p.gy[i3(k + 1, j, i, nj, ni)] * (atw(p.v, k + 1, j, i, nk, vy, ni) + atw(p.v, k + 1, j + 1, i, nk, vy, ni));
    lo = p.gy[c] * (atw(p.v, k, j, i, nk, vy, ni) + atw(p.v, k, j + 1, i, nk, vy, ni));
    vert = ((up - lo) * 0.5f) * p.rds;
    s22 = (hor + vert) * r;
    s33 = (((p.w[i3(k + 1, j, i, nj, ni)] - p.w[c]) * p.rds) * g) * r;
}

// s12 at mass level k, corner (jc, ic) in [0, nj] x [0, ni]; the open sides
// use the nearest interior corner (constant extension)
__device__ __forceinline__ float strain_s12(const DefArgs &p, int k, int jc, int ic) {
    const int ni = p.ni, nj = p.nj, nk = p.nk, ux = ni + 1, vy = nj + 1;
    const int jj = jc < 1 ? 1 : (jc > nj - 1 ? nj - 1 : jc);
    const int ii = ic < 1 ? 1 : (ic > ni - 1 ? ni - 1 : ic);
    const float sig_lo = (float)k * p.dz, sig_hi = (float)(k + 1) * p.dz;
    float r1 = p.rho[i3(k, jj - 1, ii - 1, nj, ni)] * p.gz[(unsigned)(jj - 1) * ni + ii - 1] +
               p.rho[i3(k, jj, ii, nj, ni)] * p.gz[(unsigned)jj * ni + ii];
    r1 = r1 + (p.rho[i3(k, jj, ii - 1, nj, ni)] * p.gz[(unsigned)jj * ni + ii - 1] +
               p.rho[i3(k, jj - 1, ii, nj, ni)] * p.gz[(unsigned)(jj - 1) * ni + ii]);
    r1 = 0.25f * r1;
    const float rgzu_t = p.rgzu[(unsigned)jj * ux + ii], rgzu_b = p.rgzu[(unsigned)(jj - 1) * ux + ii];
    const float x1 = (r1 * (p.u[i3(k, jj, ii, nj, ux)] * rgzu_t - p.u[i3(k, jj - 1, ii, nj, ux)] * rgzu_b)) * p.rdy;
    const float xu = (p.zt - sig_hi) * (atw(p.u, k + 1, jj - 1, ii, nk, nj, ux) + atw(p.u, k + 1, jj, ii, nk, nj, ux));
    const float xl = (p.zt - sig_lo) * (atw(p.u, k, jj - 1, ii, nk, nj, ux) + atw(p.u, k, jj, ii, nk, nj, ux));
    const float x2 = ((((0.5f * (xu - xl)) * p.rds) * r1) * (rgzu_t - rgzu_b)) * p.rdy;
    const float rgzv_r = p.rgzv[(unsigned)jj * ni + ii], rgzv_l = p.rgzv[(unsigned)jj * ni + ii - 1];
    const float y1 = (r1 * (p.v[i3(k, jj, ii, vy, ni)] * rgzv_r - p.v[i3(k, jj, ii - 1, vy, ni)] * rgzv_l)) * p.rdx;
    const float yu = (p.zt - sig_hi) * (atw(p.v, k + 1, jj, ii - 1, nk, vy, ni) + atw(p.v, k + 1, jj, ii, nk, vy, ni));
    const float yl = (p.zt - sig_lo) * (atw(p.v, k, jj, ii - 1, nk, vy, ni) + atw(p.v, k, jj, ii, nk, vy, ni));
    const float y2 = ((((0.5f * (yu - yl)) * p.rds) * r1) * (rgzv_r - rgzv_l)) * p.rdx;
    return 0.5f * ((x1 + x2) + (y1 + y2));
}

// s13 at face level kf (1..nk-1), row j, u-face column ic in [0, ni]
__device__ __forceinline__ float strain_s13(const DefArgs &p, int kf, int j, int ic) {
    const int ni = p.ni, nj = p.nj, ux = ni + 1;
    const int il = ic - 1 < 0 ? 0 : ic - 1, ir = ic < ni - 1 ? ic : ni - 1;
    const float sig_l = ((float)kf - 0.5f) * p.dz, sig_u = ((float)kf + 0.5f) * p.dz;
    const float wr = p.w[i3(kf, j, ir, nj, ni)], wl = p.w[i3(kf, j, il, nj, ni)];
    const float rgr = p.rgz[(unsigned)j * ni + ir], rgl = p.rgz[(unsigned)j * ni + il];
    const float du = (p.u[i3(kf, j, ic, nj, ux)] - p.u[i3(kf - 1, j, ic, nj, ux)]) * p.rds;
    const float hw = (wr * rgr - wl * rgl) * p.rdx;
    const float upper = (p.zt - sig_u) * (0.5f * (wr + p.w[i3(kf + 1, j, ir, nj, ni)]) +
                                          0.5f * (wl + p.w[i3(kf + 1, j, il, nj, ni)]));
    const float lower = (p.zt - sig_l) * (0.5f * (p.w[i3(kf - 1, j, ir, nj, ni)] + wr) +
                                          0.5f * (p.w[i3(kf - 1, j, il, nj, ni)] + wl));
    const float terrain = (((0.5f * p.rds) * (upper - lower)) * (rgr - rgl)) * p.rdx;
    const float strain = 0.5f * ((du + hw) + terrain);
    const float density = 0.5f * (p.gz[(unsigned)j * ni + il] * p.rf[i3(kf, j, il, nj, ni)] +
                                  p.gz[(unsigned)j * ni + ir] * p.rf[i3(kf, j, ir, nj, ni)]);
    return strain * density;
}

// s23 at face level kf (1..nk-1), v-face row jc in [0, nj], column i
__device__ __forceinline__ float strain_s23(const DefArgs &p, int kf, int jc, int i) {
    const int ni = p.ni, nj = p.nj, vy = nj + 1;
    const int jb = jc - 1 < 0 ? 0 : jc - 1, jt = jc < nj - 1 ? jc : nj - 1;
    const float sig_l = ((float)kf - 0.5f) * p.dz, sig_u = ((float)kf + 0.5f) * p.dz;
    const float wt = p.w[i3(kf, jt, i, nj, ni)], wb = p.w[i3(kf, jb, i, nj, ni)];
    const float rgt = p.rgz[(unsigned)jt * ni + i], rgb = p.rgz[(unsigned)jb * ni + i];
    const float dv = (p.v[i3(kf, jc, i, vy, ni)] - p.v[i3(kf - 1, jc, i, vy, ni)]) * p.rds;
    const float hw = (wt * rgt - wb * rgb) * p.rdy;
    const float upper = (p.zt - sig_u) * (0.5f * (wt + p.w[i3(kf + 1, jt, i, nj, ni)]) +
                                          0.5f * (wb + p.w[i3(kf + 1, jb, i, nj, ni)]));
    const float lower = (p.zt - sig_l) * (0.5f * (p.w[i3(kf - 1, jt, i, nj, ni)] + wt) +
                                          0.5f * (p.w[i3(kf - 1, jb, i, nj, ni)] + wb));
    const float terrain = (((0.5f * p.rds) * (upper - lower)) * (rgt - rgb)) * p.rdy;
    const float strain = 0.5f * ((dv + hw) + terrain);
    const float density = 0.5f * (p.gz[(unsigned)jb * ni + i] * p.rf[i3(kf, jb, i, nj, ni)] +
                                  p.gz[(unsigned)jt * ni + i] * p.rf[i3(kf, jt, i, nj, ni)]);
    return strain * density;
}

// ---- flat column (terrain_flag=.false.) strains: rdz*mh(k) / rdz*mf(k)
// (gm1_flat_calcdef_mass_v1 / _face_v1, src/cm1core/cuda_gm1_flat_stretched_closure.py:76-112;
// turb.F:4772-4786, :4880-4895)

// s11, s22, s33 at mass level k, cell (j, i)
__device__ __forceinline__ void strain_diag_flat(const DefArgs &p, int k, int j, int i, float &s11, float &s22,
                                                 float &s33) {
    const int ni = p.ni, nj = p.nj, ux = ni + 1, vy = nj + 1;
    const unsigned c = i3(k, j, i, nj, ni);
    const float r = p.rho[c];
    s11 = (r * (p.u[i3(k, j, i + 1, nj, ux)] - p.u[i3(k, j, i, nj, ux)])) * p.rdx;
    s22 = (r * (p.v[i3(k, j + 1, i, vy, ni)] - p.v[i3(k, j, i, vy, ni)])) * p.rdy;
    s33 = (r * (p.w[i3(k + 1, j, i, nj, ni)] - p.w[c])) * (p.rdz * p.mhp[k + 1]);
}

// s12 at mass level k, corner (jc, ic); open sides take the nearest interior corner
__device__ __forceinline__ float strain_s12_flat(const DefArgs &p, int k, int jc, int ic) {
    const int ni = p.ni, nj = p.nj, ux = ni + 1, vy = nj + 1;
    const int jj = jc < 1 ? 1 : (jc > nj - 1 ? nj - 1 : jc);
    const int ii = ic < 1 ? 1 : (ic > ni - 1 ? ni - 1 : ic);
    const float x = (p.u[i3(k, jj, ii, nj, ux)] - p.u[i3(k, jj - 1, ii, nj, ux)]) * p.rdy;
    const float y = (p.v[i3(k, jj, ii, vy, ni)] - p.v[i3(k, jj, ii - 1, vy, ni)]) * p.rdx;
    const float rs = (p.rho[i3(k, jj - 1, ii - 1, nj, ni)] + p.rho[i3(k, jj, ii, nj, ni)]) +
                     (p.rho[i3(k, jj, ii - 1, nj, ni)] + p.rho[i3(k, jj - 1, ii, nj, ni)]);
    return ((0.5f * (x + y)) * 0.25f) * rs;
}

// s13 at face level kf (1..nk-1), row j, u-face column ic in [0, ni]
__device__ __forceinline__ float strain_s13_flat(const DefArgs &p, int kf, int j, int ic) {
    const int ni = p.ni, nj = p.nj, ux = ni + 1;
    const int il = ic - 1 < 0 ? 0 : ic - 1, ir = ic < ni - 1 ? ic : ni - 1;
    const float dw = (p.w[i3(kf, j, ir, nj, ni)] - p.w[i3(kf, j, il, nj, ni)]) * p.rdx;
    const float du = (((p.u[i3(kf, j, ic, nj, ux)] - p.u[i3(kf - 1, j, ic, nj, ux)]) * p.rdz) * 0.5f) *
                     (p.mf3[i3(kf, j, il, nj, ni)] + p.mf3[i3(kf, j, ir, nj, ni)]);
    return ((0.5f * (dw + du)) * 0.5f) * (p.rf[i3(kf, j, il, nj, ni)] + p.rf[i3(kf, j, ir, nj, ni)]);
}

// s23 at face level kf (1..nk-1), v-face row jc in [0, nj], column i
__device__ __forceinline__ float strain_s23_flat(const DefArgs &p, int kf, int jc, int i) {
    const int ni = p.ni, nj = p.nj, vy = nj + 1;
    const int js = jc - 1 < 0 ? 0 : jc - 1, jn = jc < nj - 1 ? jc : nj - 1;
    const float dw = (p.w[i3(kf, jn, i, nj, ni)] - p.w[i3(kf, js, i, nj, ni)]) * p.rdy;
    const float dv = (((p.v[i3(kf, jc, i, vy, ni)] - p.v[i3(kf - 1, jc, i, vy, ni)]) * p.rdz) * 0.5f) *
                     (p.mf3[i3(kf, js, i, nj, ni)] + p.mf3[i3(kf, jn, i, nj, ni)]);
    return ((0.5f * (dw + dv)) * 0.5f) * (p.rf[i3(kf, js, i, nj, ni)] + p.rf[i3(kf, jn, i, nj, ni)]);
}

template <bool FLAT>
__device__ __forceinline__ void strain_diag_t(const DefArgs &p, int k, int j, int i, float &a, float &b, float &c) {
    if (FLAT) strain_diag_flat(p, k, j, i, a, b, c);
    else strain_diag(p, k, j, i, a, b, c);
}
template <bool FLAT>
__device__ __forceinline__ float strain_s12_t(const DefArgs &p, int k, int jc, int ic) {
    return FLAT ? strain_s12_flat(p, k, jc, ic) : strain_s12(p, k, jc, ic);
}
template <bool FLAT>
__device__ __forceinline__ float strain_s13_t(const DefArgs &p, int kf, int j, int ic) {
    return FLAT ? strain_s13_flat(p, kf, j, ic) : strain_s13(p, kf, j, ic);
}
template <bool FLAT>
__device__ __forceinline__ float strain_s23_t(const DefArgs &p, int kf, int jc, int i) {
    return FLAT ? strain_s23_flat(p, kf, jc, i) : strain_s23(p, kf, jc, i);
}

__device__ __forceinline__ float sq(float x) { return x * x; }

// One CTA = a 32 x 8 tile of columns, walking face levels 1..nk-1; FLAT
// selects the flat column's strain texts (the deformation reduction of
// turb.F:5361-5385 is the same in both branches).
template <bool FLAT>
__global__ void __launch_bounds__(kDX *kDY) calcdef_tile_kernel(DefArgs p) {
    __shared__ float s12[2][kDY + 1][kDX + 1];
    __shared__ float s13[kDY][kDX + 1];
    __shared__ float s23[kDY + 1][kDX];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kDX + tx;
    const int i0 = blockIdx.x * kDX, j0 = blockIdx.y * kDY;
    const int i = i0 + tx, j = j0 + ty;
    const int ni = p.ni, nj = p.nj, nk = p.nk;
    const bool own = i < ni && j < nj;
    constexpr int kCorners = (kDY + 1) * (kDX + 1), kXFaces = kDY * (kDX + 1), kYFaces = (kDY + 1) * kDX;

    float p11 = 0.0f, p22 = 0.0f, p33 = 0.0f;  // mass level kf-1 at the own cell
    if (own) strain_diag_t<FLAT>(p, 0, j, i, p11, p22, p33);
    for (int e = tid; e < kCorners; e += kDX * kDY) {
        const int r = e / (kDX + 1), q = e - r * (kDX + 1);
        if (j0 + r <= nj && i0 + q <= ni) s12[0][r][q] = strain_s12_t<FLAT>(p, 0, j0 + r, i0 + q);
    }
    for (int kf = 1; kf < nk; ++kf) {
        const int cur = kf & 1;
        float c11 = 0.0f, c22 = 0.0f, c33 = 0.0f;
        if (own) strain_diag_t<FLAT>(p, kf, j, i, c11, c22, c33);
        for (int e = tid; e < kCorners; e += kDX * kDY) {
            const int r = e / (kDX + 1), q = e - r * (kDX + 1);
            if (j0 + r <= nj && i0 + q <= ni) s12[cur][r][q] = strain_s12_t<FLAT>(p, kf, j0 + r, i0 + q);
        }
        for (int e = tid; e < kXFaces; e += kDX * kDY) {
            const int r = e / (kDX + 1), q = e - r * (kDX + 1);
            if (j0 + r < nj && i0 + q <= ni) s13[r][q] = strain_s13_t<FLAT>(p, kf, j0 + r, i0 + q);
        }
        for (int e = tid; e < kYFaces; e += kDX * kDY) {
            const int r = e / kDX, q = e - r * kDX;
            if (j0 + r <= nj && i0 + q < ni) s23[r][q] = strain_s23_t<FLAT>(p, kf, j0 + r, i0 + q);
        }
        __syncthreads();
        if (own) {
            const unsigned f = i3(kf, j, i, nj, ni);
            const float a = p.c1[f], b = p.c2[f];
            const float t11 = a * sq(p11) + b * sq(c11);
            const float t22 = a * sq(p22) + b * sq(c22);
            const float t33 = a * sq(p33) + b * sq(c33);
            const float(*L)[kDX + 1] = s12[cur ^ 1];
            const float(*H)[kDX + 1] = s12[cur];
            const float lo12 = (sq(L[ty][tx]) + sq(L[ty + 1][tx + 1])) + (sq(L[ty + 1][tx]) + sq(L[ty][tx + 1]));
            const float hi12 = (sq(H[ty][tx]) + sq(H[ty + 1][tx + 1])) + (sq(H[ty + 1][tx]) + sq(H[ty][tx + 1]));
            const float t12 = 0.25f * (a * lo12 + b * hi12);
            const float t13 = 0.5f * (sq(s13[ty][tx]) + sq(s13[ty][tx + 1]));
            const float t23 = 0.5f * (sq(s23[ty][tx]) + sq(s23[ty + 1][tx]));
            const float rfv = p.rf[f];
            const float rrf = rcp_rn(rfv * rfv);
            p.defv[f] = (4.0f * (t13 + t23)) * rrf;
            p.defh[f] = ((2.0f * ((t11 + t22) + t33)) + 4.0f * t12) * rrf;
        }
        p11 = c11;
        p22 = c22;
        p33 = c33;
        __syncthreads();
    }
    if (own) {
        p.defv[i3(0, j, i, nj, ni)] = 0.0f;
        p.defh[i3(0, j, i, nj, ni)] = 0.0f;
        p.defv[i3(nk, j, i, nj, ni)] = 0.0f;
        p.defh[i3(nk, j, i, nj, ni)] = 0.0f;
    }
}

// ---------------------------------------------------------------- calcnm
struct NmConsts {
    float g, rd, cp, cpv, cpl, cpi, eps, reps, lv1, lv2, ls1, ls2;
};

struct NmArgs {
    const float *c1, *c2, *mf, *pi0, *th0, *prs, *pp3d, *th3d, *q3d;
    float *nm, *temperature, *qt, *thv, *qvci;
    uint8_t *mask;
    unsigned long long *counts;
    int ni, nj, nk;
    float rdz;
    NmConsts c;
};

struct NmCell {
    float t, qt, thv, qvci;
};

__device__ __forceinline__ NmCell nm_cell(const NmArgs &a, int k, unsigned p) {
    const unsigned cells = (unsigned)a.nk * a.nj * a.ni;
    NmCell r;
    const float qv = a.q3d[p];
    r.qvci = (qv + a.q3d[cells + p]) + a.q3d[3 * cells + p];
    float t = 0.0f;
#pragma unroll
    for (int s = 0; s < 6; ++s) t = t + a.q3d[s * cells + p];
    r.qt = t;
    const float theta = a.th0[k] + a.th3d[p];
    const float exner = a.pi0[k] + a.pp3d[p];
    r.t = theta * exner;
    const float tv = theta * (1.0f + a.c.reps * qv);
    r.thv = tv / (1.0f + t);
    return r;
}

__device__ __forceinline__ float sat_liquid(float p, float t, float eps) {
    const float x = (17.67f * (t - 273.15f)) / (t - 29.65f);
    float es = 611.2f * expf(x);
    const float h = p * 0.5f;
    if (h < es) es = h;
    return (eps * es) / (p - es);
}

__device__ __forceinline__ float sat_ice(float p, float t, float eps) {
    const float x = (21.8745584f * (t - 273.15f)) / (t - 7.66f);
    float es = 611.2f * expf(x);
    const float h = p * 0.5f;
    if (h < es) es = h;
    return (eps * es) / (p - es);
}

__device__ __forceinline__ float nm_saturated(const NmConsts &c, const NmCell &up, const NmCell &lo, float tavg,
                                              float qtavg, float qvs, float ql, float qi, float qv, float mrdz,
                                              bool ice) {
    float cpml = c.cp + c.cpv * qv;
    cpml = cpml + c.cpl * ql;
    if (qi != 0.0f) cpml = cpml + c.cpi * qi;
    float lh, drdt, den;
    if (ice) {
        lh = c.ls1 - c.ls2 * tavg;
        drdt = 21.8745584f * (273.15f - 7.66f);
        den = (tavg - 7.66f) * (tavg - 7.66f);
    } else {
        lh = c.lv1 - c.lv2 * tavg;
        drdt = 17.67f * (273.15f - 29.65f);
        den = (tavg - 29.65f) * (tavg - 29.65f);
    }
    drdt = (drdt * qvs) / den;
    float gamma = c.g * (1.0f + qtavg);
    gamma = gamma * (1.0f + (lh * qvs) / (c.rd * tavg));
    gamma = gamma / (cpml + lh * drdt);
    float first = logf(up.t / lo.t) * mrdz;
    first = first + gamma / tavg;
    float second = tavg * drdt;
    second = second / (c.eps + qvs);
    first = first * (1.0f + second);
    float moist = logf((1.0f + up.qt) / (1.0f + lo.qt));
    moist = moist * mrdz;
    return c.g * (first - moist);
}

// grid: x over i, y over j, z over face level kf = 0..nk
__global__ void __launch_bounds__(128) moist_nm_kernel(NmArgs a) {
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 4 + threadIdx.y;
    const int kf = blockIdx.z;
    const int ni = a.ni, nj = a.nj, nk = a.nk;
    const bool in = i < ni && j < nj;
    int sat = 0, liq = 0, mix = 0, ice = 0;
    if (in) {
        const unsigned col = (unsigned)j * ni + i, plane = (unsigned)nj * ni;
        const unsigned m = (unsigned)kf * plane + col, f = m;
        NmCell up{}, lo{};
        if (kf < nk) {
            up = nm_cell(a, kf, m);
            a.qvci[m] = up.qvci;
            a.qt[m] = up.qt;
            a.temperature[m] = up.t;
            a.thv[m] = up.thv;
        }
        float value = 0.0f;
        if (kf >= 1 && kf < nk) {
            const unsigned l = m - plane;
            lo = nm_cell(a, kf - 1, l);
            const NmConsts &c = a.c;
            const float mrdz = a.rdz * a.mf[f];
            value = c.g * (logf(up.thv / lo.thv) * mrdz);
            const float w1 = a.c1[f], w2 = a.c2[f];
            const float pavg = w1 * a.prs[l] + w2 * a.prs[m];
            const float tavg = w1 * lo.t + w2 * up.t;
            const float qtavg = w1 * lo.qt + w2 * up.qt;
            const float qvciavg = w1 * lo.qvci + w2 * up.qvci;
            if (tavg >= 273.15f) {
                const float qvs = sat_liquid(pavg, tavg, c.eps);
                float ql = qvciavg - qvs;
                if (!(ql > 0.0f)) ql = 0.0f;
                if (ql > 1.0e-10f) {
                    float qv = qvciavg - ql;
                    if (!(qv > 0.0f)) qv = 0.0f;
                    value = nm_saturated(c, up, lo, tavg, qtavg, qvs, ql, 0.0f, qv, mrdz, false);
                    sat = liq = 1;
                }
            } else if (tavg <= 233.15f) {
                const float qvs = sat_ice(pavg, tavg, c.eps);
                float qi = qvciavg - qvs;
                if (!(qi > 0.0f)) qi = 0.0f;
                if (qi > 1.0e-10f) {
                    float qv = qvciavg - qi;
                    if (!(qv > 0.0f)) qv = 0.0f;
                    value = nm_saturated(c, up, lo, tavg, qtavg, qvs, 0.0f, qi, qv, mrdz, true);
                    sat = ice = 1;
                }
            } else {
                const float ff = (tavg - 233.15f) / (273.15f - 233.15f);
                const float qvsl = sat_liquid(pavg, tavg, c.eps), qvsi = sat_ice(pavg, tavg, c.eps);
                const float om = 1.0f - ff;
                const float qvs = ff * qvsl + om * qvsi;
                const float ex = qvciavg - qvs;
                float qi = om * ex;
                if (!(qi > 0.0f)) qi = 0.0f;
                float ql = ff * ex;
                if (!(ql > 0.0f)) ql = 0.0f;
                if (ql + qi > 1.0e-10f) {
                    float qv = (qvciavg - ql) - qi;
                    if (!(qv > 0.0f)) qv = 0.0f;
                    const float nml = nm_saturated(c, up, lo, tavg, qtavg, qvsl, ql, qi, qv, mrdz, false);
                    const float nmi = nm_saturated(c, up, lo, tavg, qtavg, qvsi, ql, qi, qv, mrdz, true);
                    value = ff * nml + om * nmi;
                    sat = mix = 1;
                }
            }
        }
        a.nm[f] = value;
        if (kf < nk) a.mask[m] = (uint8_t)sat;
    }
    if (a.counts != nullptr) {
        const int n0 = __syncthreads_count(sat), n1 = __syncthreads_count(liq);
        const int n2 = __syncthreads_count(mix), n3 = __syncthreads_count(ice);
        if (threadIdx.x == 0 && threadIdx.y == 0 && n0 > 0) {
            atomicAdd(&a.counts[0], (unsigned long long)n0);
            if (n1) atomicAdd(&a.counts[1], (unsigned long long)n1);
            if (n2) atomicAdd(&a.counts[2], (unsigned long long)n2);
            if (n3) atomicAdd(&a.counts[3], (unsigned long long)n3);
        }
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

extern "C" int32_t gm1b_terrain_deformation(int32_t ni, int32_t nj, int32_t nk,
                                            const gm1b_deformation_arrays *arrays, float dx, float dy, float dz,
                                            void *stream) {
    if (arrays == nullptr || ni < 3 || nj < 3 || nk < 3) {
        gm1b_set_error("gm1b_terrain_deformation: need arrays and ni, nj, nk >= 3");
        return GM1B_ERR_ARGUMENT;
    }
    if (!(dx > 0.0f) || !(dy > 0.0f) || !(dz > 0.0f) || !isfinite(dx) || !isfinite(dy) || !isfinite(dz)) {
        gm1b_set_error("gm1b_terrain_deformation: dx, dy, dz must be finite and > 0");
        return GM1B_ERR_ARGUMENT;
    }
    const gm1b_deformation_arrays &s = *arrays;
    const void *need[] = {s.u3d, s.v3d, s.w3d, s.rho, s.rf, s.c1, s.c2, s.gz, s.rgz, s.rgzu, s.rgzv, s.gx, s.gy,
                          s.defv, s.defh};
    for (const void *q : need)
        if (q == nullptr) {
            gm1b_set_error("gm1b_terrain_deformation: a required array is NULL");
            return GM1B_ERR_ARGUMENT;
        }
    if ((size_t)(nk + 3) * (size_t)(nj + 7) * (size_t)(ni + 7) >= ((size_t)1 << 31)) {
        gm1b_set_error("gm1b_terrain_deformation: grid too large (the kernels index with 32-bit offsets)");
        return GM1B_ERR_ARGUMENT;
    }
    DefArgs p;
    p.u = s.u3d;
    p.v = s.v3d;
    p.w = s.w3d;
    p.rho = s.rho;
    p.rf = s.rf;
    p.c1 = s.c1;
    p.c2 = s.c2;
    p.gz = s.gz;
    p.rgz = s.rgz;
    p.rgzu = s.rgzu;
    p.rgzv = s.rgzv;
    p.gx = s.gx;
    p.gy = s.gy;
    p.defv = s.defv;
    p.defh = s.defh;
    p.ni = ni;
    p.nj = nj;
    p.nk = nk;
    p.rdx = 1.0f / dx;
    p.rdy = 1.0f / dy;
    p.rds = 1.0f / dz;
    p.zt = (float)nk * dz;
    p.dz = dz;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("calcdef_tile_kernel", st);
    calcdef_tile_kernel<false><<<dim3((ni + kDX - 1) / kDX, (nj + kDY - 1) / kDY), dim3(kDX, kDY), 0, st>>>(p);
    ps.stop();
    return launch_ok("calcdef_tile_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_flat_deformation(int32_t ni, int32_t nj, int32_t nk, const gm1b_flat_deformation_arrays *arrays,
                                         float dx, float dy, float rdz, void *stream) {
    if (arrays == nullptr || ni < 3 || nj < 3 || nk < 3) {
        gm1b_set_error("gm1b_flat_deformation: need arrays and ni, nj, nk >= 3");
        return GM1B_ERR_ARGUMENT;
    }
    if (!(dx > 0.0f) || !(dy > 0.0f) || !(rdz > 0.0f) || !isfinite(dx) || !isfinite(dy) || !isfinite(rdz)) {
        gm1b_set_error("gm1b_flat_deformation: dx, dy, rdz must be finite and > 0");
        return GM1B_ERR_ARGUMENT;
    }
    const gm1b_flat_deformation_arrays &s = *arrays;
    const void *need[] = {s.u3d, s.v3d, s.w3d, s.rho, s.rf, s.mf, s.c1, s.c2, s.mh_profile, s.defv, s.defh};
    for (const void *q : need)
        if (q == nullptr) {
            gm1b_set_error("gm1b_flat_deformation: a required array is NULL");
            return GM1B_ERR_ARGUMENT;
        }
    if ((size_t)(nk + 3) * (size_t)(nj + 7) * (size_t)(ni + 7) >= ((size_t)1 << 31)) {
        gm1b_set_error("gm1b_flat_deformation: grid too large (the kernels index with 32-bit offsets)");
        return GM1B_ERR_ARGUMENT;
    }
    DefArgs p{};
    p.u = s.u3d;
    p.v = s.v3d;
    p.w = s.w3d;
    p.rho = s.rho;
    p.rf = s.rf;
    p.c1 = s.c1;
    p.c2 = s.c2;
    p.mf3 = s.mf;
    p.mhp = s.mh_profile;
    p.defv = s.defv;
    p.defh = s.defh;
    p.ni = ni;
    p.nj = nj;
    p.nk = nk;
    p.rdx = 1.0f / dx;
    p.rdy = 1.0f / dy;
    p.rdz = rdz;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("calcdef_flat_tile_kernel", st);
    calcdef_tile_kernel<true><<<dim3((ni + kDX - 1) / kDX, (nj + kDY - 1) / kDY), dim3(kDX, kDY), 0, st>>>(p);
    ps.stop();
    return launch_ok("calcdef_flat_tile_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_moist_nm(int32_t ni, int32_t nj, int32_t nk, const gm1b_moist_nm_arrays *arrays, float dz,
                                 void *stream) {
    if (arrays == nullptr || ni < 1 || nj < 1 || nk < 2 || nk > 65534) {
        gm1b_set_error("gm1b_moist_nm: need arrays, ni >= 1, nj >= 1 and 2 <= nk <= 65534");
        return GM1B_ERR_ARGUMENT;
    }
    if ((size_t)(nk + 3) * (size_t)(nj + 7) * (size_t)(ni + 7) >= ((size_t)1 << 31)) {
        gm1b_set_error("gm1b_moist_nm: grid too large (the kernels index with 32-bit offsets)");
        return GM1B_ERR_ARGUMENT;
    }
    if (!(dz > 0.0f) || !isfinite(dz)) {
        gm1b_set_error("gm1b_moist_nm: dz must be finite and > 0");
        return GM1B_ERR_ARGUMENT;
    }
    const gm1b_moist_nm_arrays &s = *arrays;
    const void *need[] = {s.c1, s.c2, s.mf, s.pi0, s.th0, s.prs, s.pp3d, s.th3d, s.q3d, s.nm, s.temperature,
                          s.qt, s.thv, s.qvci, s.saturation_mask};
    for (const void *q : need)
        if (q == nullptr) {
            gm1b_set_error("gm1b_moist_nm: a required array is NULL");
            return GM1B_ERR_ARGUMENT;
        }
    NmArgs a;
    a.c1 = s.c1;
    a.c2 = s.c2;
    a.mf = s.mf;
    a.pi0 = s.pi0;
    a.th0 = s.th0;
    a.prs = s.prs;
    a.pp3d = s.pp3d;
    a.th3d = s.th3d;
    a.q3d = s.q3d;
    a.nm = s.nm;
    a.temperature = s.temperature;
    a.qt = s.qt;
    a.thv = s.thv;
    a.qvci = s.qvci;
    a.mask = s.saturation_mask;
    a.counts = reinterpret_cast<unsigned long long *>(s.counts);
    a.ni = ni;
    a.nj = nj;
    a.nk = nk;
    a.rdz = 1.0f / dz;
    // CM1 constants.F words and the derived latent-heat coefficients, formed
    // in binary32 as the reference forms them (cuda_moist_nm.py:179-204)
    volatile float rv = 461.5f, to = 273.15f;
    NmConsts &c = a.c;
    c.g = 9.81f;
    c.rd = 287.04f;
    c.cp = 1005.7f;
    c.cpv = 1870.0f;
    c.cpl = 4190.0f;
    c.cpi = 2106.0f;
    c.eps = c.rd / rv;
    c.reps = rv / c.rd;
    const float dl = c.cpl - c.cpv, di = c.cpi - c.cpv;
    const float tl = dl * to, ti = di * to;
    c.lv1 = 2501000.0f + tl;
    c.lv2 = dl;
    c.ls1 = 2834000.0f + ti;
    c.ls2 = di;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("moist_nm_kernel", st);
    moist_nm_kernel<<<dim3((ni + 31) / 32, (nj + 3) / 4, nk + 1), dim3(32, 4), 0, st>>>(a);
    ps.stop();
    return launch_ok("moist_nm_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}
