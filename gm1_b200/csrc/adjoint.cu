// adjoint.cu - hand-written adjoint (reverse-mode) kernels of the large
// step's operators, for gradients of a scalar objective with respect to the
// model state.
//
//   scalar advection5 / WENO5 adjoint   the tendency of gm1b_scalar_advection5
//       (cpu_scalar_advection5_inplace, src/cm1core/cuda_advection5.py:440-579,
//       :669) differentiated with respect to the padded scalar, the mass
//       fluxes held fixed; the WENO-Z weights differentiated at their
//       epsilon-regularised form (the 1e30 cap and |b1 - b3| at b1 = b3 take
//       the subgradient 0), upstrpd's min/max limiter by its active branch.
//   open-fill adjoint                   the transpose of the scalar open
//       fill (bcs open, src/cm1core/cuda_sound3_open_boundary.py:249-335):
//       halo adjoints fold back onto the edge cells they copy.
//   transposed tridiagonal solve        the adjoint of the acoustic column's
//       vertically implicit solve a(k) x(k-1) + b(k) x(k) + c(k) x(k+1) = d(k)
//       (cpu_sound3_periodic_stage_inplace's w-pi' system,
//       src/cm1core/cuda_sound3_periodic.py:824-1027): A^T y = g per column,
//       the Thomas sweep of the transposed system.
//   Kessler collection and its adjoint  autoconversion max(0.001(qc-0.001), 0)
//       dt and accretion 2.2 qc qr^0.875 dt with the qc limiter
//       (cpu_gm1_kessler_local_inplace, src/cm1core/cuda_gm1_kessler_local.py:
//       251; the driver's local step, cuda_gm1_kessler_driver.py:636-653):
//       the subgradient 0 at the autoconversion switch qc = 0.001 and at
//       qr = 0, where qr^0.875 has no derivative.
//   single-pass saturation adjustment    the equation-set-1 branch of the
//       Kessler operator's _cpu_satadj (src/cm1core/cuda_gm1_kessler_driver.py:
//       337-428), forward and adjoint, each limiter by its taken branch.
//
// Design (B200): every adjoint is a gather - one thread per output word
// sums the contributions of the forward words that read it, recomputing the
// forward's local derivative - so there are no atomics and the result is
// deterministic.  binary32 storage, binary64 for the WENO weight derivatives.
#include <algorithm>

#include "gm1b_common.cuh"
#include "weno.cuh"

namespace gm1b {
namespace {

constexpr int kNg = 3;

// Python-style max (the Kessler operator's: b when b > a, else a)
__device__ __forceinline__ float pymax(float a, float b) { return (b > a) ? b : a; }

// d weno5 / d s_k (k = 0..4), the binary64 derivative of the function the
// forward evaluates (its own rounded stencil differences as the point)
__device__ void weno5_grad(const float s[5], double eps, double g[5]) {
    const double d1 = (double)((s[0] - 2.0f * s[1]) + s[2]);
    const double e1 = (double)((s[0] - 4.0f * s[1]) + 3.0f * s[2]);
    const double d2 = (double)((s[1] - 2.0f * s[2]) + s[3]);
    const double e2 = (double)(s[1] - s[3]);
    const double d3 = (double)((s[2] - 2.0f * s[3]) + s[4]);
    const double e3 = (double)((3.0f * s[2] - 4.0f * s[3]) + s[4]);
    const double c13 = (double)kC13_12;
    const double b1 = (double)(kC13_12 * (float)(d1 * d1) + 0.25f * (float)(e1 * e1));
    const double b2 = (double)(kC13_12 * (float)(d2 * d2) + 0.25f * (float)(e2 * e2));
    const double b3 = (double)(kC13_12 * (float)(d3 * d3) + 0.25f * (float)(e3 * e3));
    // gradients of the smoothness indicators
    const double dd1[5] = {1, -2, 1, 0, 0}, de1[5] = {1, -4, 3, 0, 0};
    const double dd2[5] = {0, 1, -2, 1, 0}, de2[5] = {0, 1, 0, -1, 0};
    const double dd3[5] = {0, 0, 1, -2, 1}, de3[5] = {0, 0, 3, -4, 1};
    double gb1[5], gb2[5], gb3[5];
    for (int k = 0; k < 5; ++k) {
        gb1[k] = 2.0 * c13 * d1 * dd1[k] + 0.5 * e1 * de1[k];
        gb2[k] = 2.0 * c13 * d2 * dd2[k] + 0.5 * e2 * de2[k];
        gb3[k] = 2.0 * c13 * d3 * dd3[k] + 0.5 * e3 * de3[k];
    }
    const double diff = b1 - b3;
    const double tau = fabs(diff);
    const double sg = diff > 0.0 ? 1.0 : (diff < 0.0 ? -1.0 : 0.0);
    const double den1 = b1 + eps, den2 = b2 + eps, den3 = b3 + eps;
    const double q1r = tau / den1, q2r = tau / den2, q3r = tau / den3;
    const double q1 = dmin30(q1r), q2 = dmin30(q2r), q3 = dmin30(q3r);
    const double gam1 = (double)0.1f, gam2 = (double)0.6f, gam3 = (double)0.3f;
    const double w1 = gam1 * (1.0 + q1 * q1), w2 = gam2 * (1.0 + q2 * q2), w3 = gam3 * (1.0 + q3 * q3);
    const double W = w1 + w2 + w3;
    const double p1 = (double)((kF3_3 * s[0] + kCm7_6 * s[1]) + kC11_6 * s[2]);
    const double p2 = (double)((kF3_1 * s[1] + kF3_2 * s[2]) + kF3_3 * s[3]);
    const double p3 = (double)((kF3_3 * s[2] + kF3_2 * s[3]) + kF3_1 * s[4]);
    const double rW = 1.0 / W, rden1 = 1.0 / den1, rden2 = 1.0 / den2, rden3 = 1.0 / den3;
    const double f = (w1 * p1 + w2 * p2 + w3 * p3) * rW;
    const double gp1[5] = {(double)kF3_3, (double)kCm7_6, (double)kC11_6, 0, 0};
    const double gp2[5] = {0, (double)kF3_1, (double)kF3_2, (double)kF3_3, 0};
    const double gp3[5] = {0, 0, (double)kF3_3, (double)kF3_2, (double)kF3_1};
    for (int k = 0; k < 5; ++k) {
        const double gtau = sg * (gb1[k] - gb3[k]);
        const double gq1 = q1r < 1.0e30 ? (gtau - q1r * gb1[k]) * rden1 : 0.0;
        const double gq2 = q2r < 1.0e30 ? (gtau - q2r * gb2[k]) * rden2 : 0.0;
        const double gq3 = q3r < 1.0e30 ? (gtau - q3r * gb3[k]) * rden3 : 0.0;
        const double gw1 = gam1 * 2.0 * q1 * gq1, gw2 = gam2 * 2.0 * q2 * gq2, gw3 = gam3 * 2.0 * q3 * gq3;
        g[k] = ((w1 * gp1[k] + w2 * gp2[k] + w3 * gp3[k]) + ((p1 - f) * gw1 + (p2 - f) * gw2 + (p3 - f) * gw3)) * rW;
    }
}

// d upstrpd(s1, s2, s3) / d s_k: the limiter's active branch
__device__ void upstrpd_grad(float s1, float s2, float s3, float weps, double g[3]) {
    const float dd = s2 - s1;
    const float se = copysignf(fabsf(weps), dd);
    const float den = se + dd;
    const float num = s3 - s2;
    const float rr = num / den;
    const float cand = kC1_6 + kF3_3 * rr;
    const float inner = fminf(cand, 1.0f);
    const float mn = fminf(rr, inner);
    const float phi = fmaxf(0.0f, mn);
    const double dn = den, nm = num;
    const double grr[3] = {nm / (dn * dn), (-dn - nm) / (dn * dn), 1.0 / dn};  // d rr / d (s1, s2, s3)
    double gphi[3] = {0.0, 0.0, 0.0};
    if (mn > 0.0f) {
        if (rr <= inner) {
            for (int k = 0; k < 3; ++k) gphi[k] = grr[k];
        } else if (cand < 1.0f) {
            for (int k = 0; k < 3; ++k) gphi[k] = (double)kF3_3 * grr[k];
        }
    }
    g[0] = -(double)phi + (double)dd * gphi[0];
    g[1] = 1.0 + (double)phi + (double)dd * gphi[1];
    g[2] = (double)dd * gphi[2];
}

struct AdvAdjArgs {
    const float *s, *rru, *rrv, *rrw, *c1, *c2, *rr0, *gz, *divx, *lam;  // lam: tendency adjoint (nk, nj, ni)
    float *out;         // padded (or compact) scalar adjoint
    const float *base;  // compact form: added to the gathered adjoint (NULL: nothing)
    float *sum_out;     // compact form: when set, out = gathered and sum_out = base + gathered
    int compact_scalar; // s is the compact (nk, nj, ni) scalar, read through the open carrier's map
    float lam_scale;    // lam enters as lam_scale * lam
    // face coefficient scratch: six slots per face, slot o + 3 holding
    // (face adjoint) * (mass flux) * d(face value)/d(scalar at face + o),
    // o = -3..2 along the face's axis
    float *cx, *cy, *cz;
    int ni, nj, nk, weno;
    unsigned obc;
    float rdx, rdy, rdz;
    double eps;
};

// 32-bit offsets: the launcher refuses grids whose largest array (the
// face-coefficient scratch, 6 (nk+1)(nj+1)(ni+1) words) reaches 2^31 words
__device__ __forceinline__ int pidx(const AdvAdjArgs &a, int k, int y, int x) {
    return (k * (a.nj + 2 * kNg) + y) * (a.ni + 2 * kNg) + x;
}
__device__ __forceinline__ int uidx(const AdvAdjArgs &a, int k, int y, int x) {
    return (k * (a.nj + 2 * kNg) + y) * (a.ni + 1 + 2 * kNg) + x;
}
__device__ __forceinline__ int vidx(const AdvAdjArgs &a, int k, int y, int x) {
    return (k * (a.nj + 1 + 2 * kNg) + y) * (a.ni + 2 * kNg) + x;
}
__device__ __forceinline__ int cidx(const AdvAdjArgs &a, int k, int j, int i) { return (k * a.nj + j) * a.ni + i; }
// scratch slots: x faces (nk levels, nj rows, ni+1 faces), y faces (nk,
// nj+1, ni), z faces (K = 1..nk+1 at index K-1, nj, ni)
__device__ __forceinline__ int cxi(const AdvAdjArgs &a, int o, int k, int j, int f) {
    return (((o + 3) * a.nk + (k - 1)) * a.nj + j) * (a.ni + 1) + f;
}
__device__ __forceinline__ int cyi(const AdvAdjArgs &a, int o, int k, int f, int i) {
    return (((o + 3) * a.nk + (k - 1)) * (a.nj + 1) + f) * a.ni + i;
}
__device__ __forceinline__ int czi(const AdvAdjArgs &a, int o, int K, int j, int i) {
    return (((o + 3) * (a.nk + 1) + (K - 1)) * a.nj + j) * a.ni + i;
}

// the carrier word (k, y, x): the padded scalar itself, or, for a compact
// scalar, the open-filled carrier's word computed from the compact field
// (the map of scalar_carrier_open_kernel)
__device__ __forceinline__ float carrier(const AdvAdjArgs &a, int k, int y, int x) {
    if (!a.compact_scalar) return a.s[pidx(a, k, y, x)];
    const int x0 = kNg, xl = kNg + a.ni - 1, y0 = kNg, yl = kNg + a.nj - 1;
    if (k < 1 || k > a.nk || !((y >= y0 && y <= yl) || (x >= x0 - 1 && x <= xl + 1))) return 0.0f;
    return __ldg(a.s + cidx(a, k - 1, min(max(y, y0), yl) - kNg, min(max(x, x0), xl) - kNg));
}

// the adjoint of the tendency's "total" (before the rr0*gz scale) at cell
// (level k = 1..nk, j, i), zero outside the domain
__device__ __forceinline__ float lam_total(const AdvAdjArgs &a, int k, int j, int i) {
    if (k < 1 || k > a.nk || j < 0 || j >= a.nj || i < 0 || i >= a.ni) return 0.0f;
    const int c = cidx(a, k - 1, j, i);
    return ((a.lam_scale * a.lam[c]) * a.rr0[c]) * a.gz[j * a.ni + i];
}

// open-side inflow edit of cell (k, j, i) along x / y: its face fluxes are
// replaced and the divergence piece s*(ue-uw)*rdx added
__device__ __forceinline__ bool x_edit(const AdvAdjArgs &a, int k, int j, int i) {
    const int y = j + kNg, x = i + kNg;
    const bool iw = i == 0 && ((a.obc >> 0) & 15u) == 2u && a.rru[uidx(a, k, y, x)] >= 0.0f;
    const bool ie = i + 1 == a.ni && ((a.obc >> 4) & 15u) == 2u && a.rru[uidx(a, k, y, x + 1)] <= 0.0f;
    return iw || ie;
}
__device__ __forceinline__ bool y_edit(const AdvAdjArgs &a, int k, int j, int i) {
    const int y = j + kNg, x = i + kNg;
    const bool js = j == 0 && ((a.obc >> 8) & 15u) == 2u && a.rrv[vidx(a, k, y, x)] >= 0.0f;
    const bool jn = j + 1 == a.nj && ((a.obc >> 12) & 15u) == 2u && a.rrv[vidx(a, k, y + 1, x)] <= 0.0f;
    return js || jn;
}

// the 5-point reconstruction's derivatives at its stencil
__device__ __forceinline__ void recon_grad5_all(const AdvAdjArgs &a, const float st[5], double g[5]) {
    if (!a.weno) {
        g[0] = kF5_1;
        g[1] = kF5_2;
        g[2] = kF5_3;
        g[3] = kF5_4;
        g[4] = kF5_5;
        return;
    }
    weno5_grad(st, a.eps, g);
}

// horizontal face (axis 0: x face f = 0..ni of row j; axis 1: y face f =
// 0..nj of column i) at level k: its six slots
__device__ void hface_coefficients(const AdvAdjArgs &a, int axis, int k, int line, int f, float slot[6]) {
    for (int o = 0; o < 6; ++o) slot[o] = 0.0f;
    const bool xa = axis == 0;
    const int F = f + kNg, L = line + kNg;
    const float m = xa ? a.rru[uidx(a, k, L, F)] : a.rrv[vidx(a, k, F, L)];
    // face adjoint: + rd * lam(cell right/north of the face), - rd * lam(cell left/south)
    const float rd = xa ? a.rdx : a.rdy;
    const int n = xa ? a.ni : a.nj;
    float g = 0.0f;
    if (xa) {
        if (f < n && !x_edit(a, k, line, f)) g += lam_total(a, k, line, f) * rd;
        if (f - 1 >= 0 && !x_edit(a, k, line, f - 1)) g -= lam_total(a, k, line, f - 1) * rd;
    } else {
        if (f < n && !y_edit(a, k, f, line)) g += lam_total(a, k, f, line) * rd;
        if (f - 1 >= 0 && !y_edit(a, k, f - 1, line)) g -= lam_total(a, k, f - 1, line) * rd;
    }
    if (g == 0.0f) return;
    const bool up = m >= 0.0f;
    float st[5];
    for (int q = 0; q < 5; ++q) {
        const int pp = up ? F - 3 + q : F + 2 - q;
        st[q] = xa ? carrier(a, k, L, pp) : carrier(a, k, pp, L);
    }
    double d[5];
    recon_grad5_all(a, st, d);
    const double gm = (double)g * (double)m;
    for (int q = 0; q < 5; ++q) {
        const int o = up ? q - 3 : 2 - q;  // the point's offset from the face
        slot[o + 3] = (float)(gm * d[q]);
    }
}

// vertical face K (2..nk) of column (j, i): its six slots, following the
// forward's boundary-closure branches in its order
__device__ void zface_coefficients(const AdvAdjArgs &a, int K, int j, int i, float slot[6]) {
    for (int o = 0; o < 6; ++o) slot[o] = 0.0f;
    const int nk = a.nk;
    if (K < 2 || K > nk) return;
    const int y = j + kNg, x = i + kNg;
    const float m = a.rrw[pidx(a, K, y, x)];
    const float g = (lam_total(a, K, j, i) - lam_total(a, K - 1, j, i)) * a.rdz;
    if (g == 0.0f) return;
    const double gm = (double)g * (double)m;
    const float c1 = a.c1[cidx(a, K - 1, j, i)], c2 = a.c2[cidx(a, K - 1, j, i)];
    const float wepsf = (float)a.eps;
    auto S = [&](int kk) { return carrier(a, kk, y, x); };
    auto put = [&](int level, double d) { slot[level - K + 3] = (float)(gm * d); };
    auto lin2 = [&]() {  // c1*s(K-1) + c2*s(K)
        put(K - 1, c1);
        put(K, c2);
    };
    auto three = [&](int k1, int k2, int k3) {  // flx3 / upstrpd(s(k1), s(k2), s(k3))
        double gg[3];
        if (a.weno) {
            upstrpd_grad(S(k1), S(k2), S(k3), wepsf, gg);
        } else {
            gg[0] = kF3_1;
            gg[1] = kF3_2;
            gg[2] = kF3_3;
        }
        put(k1, gg[0]);
        put(k2, gg[1]);
        put(k3, gg[2]);
    };
    auto five = [&](int k1, int step) {  // recon(s(k1), s(k1+step), ...)
        float st[5];
        for (int q = 0; q < 5; ++q) st[q] = S(k1 + step * q);
        double d[5];
        recon_grad5_all(a, st, d);
        for (int q = 0; q < 5; ++q) put(k1 + step * q, d[q]);
    };
    if (K == 2) {
        if (m >= 0.0f) lin2();
        else three(K + 1, K, K - 1);
    } else if (K == nk) {
        const bool up = a.weno ? (m > 0.0f) : (m >= 0.0f);
        if (up) three(K - 2, K - 1, K);
        else lin2();
    } else if (K == 3) {
        if (m >= 0.0f) three(K - 2, K - 1, K);
        else five(K + 2, -1);
    } else if (K == nk - 1) {
        if (m >= 0.0f) five(K - 3, 1);
        else three(K + 1, K, K - 1);
    } else {
        if (m >= 0.0f) five(K - 3, 1);
        else five(K + 2, -1);
    }
}

// pass 1: grid (ceil((ni+1)/32), ceil((nj+1)/8), nk+1); one thread per
// face site (column i = 0..ni, row j = 0..nj, level L = 0..nk) writes the
// slots of its x face, y face and z face (K = L + 1)
__global__ void __launch_bounds__(256) advection_adjoint_faces_kernel(const __grid_constant__ AdvAdjArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, L = blockIdx.z;
    if (i > a.ni || j > a.nj) return;
    {
        float slot[6];
        if (L < a.nk && j < a.nj) {
            hface_coefficients(a, 0, L + 1, j, i, slot);
            for (int o = -3; o <= 2; ++o) a.cx[cxi(a, o, L + 1, j, i)] = slot[o + 3];
        }
        if (L < a.nk && i < a.ni) {
            hface_coefficients(a, 1, L + 1, i, j, slot);
            for (int o = -3; o <= 2; ++o) a.cy[cyi(a, o, L + 1, j, i)] = slot[o + 3];
        }
        if (i < a.ni && j < a.nj) {
            zface_coefficients(a, L + 1, j, i, slot);
            for (int o = -3; o <= 2; ++o) a.cz[czi(a, o, L + 1, j, i)] = slot[o + 3];
        }
    }
}

// dJ/d(padded word (k, y, x)): the slots of every face whose stencil reads
// it, plus the divergence and open-side terms of its own cell
__device__ double padded_adjoint(const AdvAdjArgs &a, int k, int y, int x) {
    if (k < 1 || k > a.nk) return 0.0;
    const int i = x - kNg, j = y - kNg;
    double acc = 0.0;
    if (j >= 0 && j < a.nj) {
        for (int o = -3; o <= 2; ++o) {
            const int f = i - o;
            if (f >= 0 && f <= a.ni) acc += (double)a.cx[cxi(a, o, k, j, f)];
        }
    }
    if (i >= 0 && i < a.ni) {
        for (int o = -3; o <= 2; ++o) {
            const int f = j - o;
            if (f >= 0 && f <= a.nj) acc += (double)a.cy[cyi(a, o, k, f, i)];
        }
        if (j >= 0 && j < a.nj) {
            for (int o = -3; o <= 2; ++o) {
                const int K = k - o;
                if (K >= 2 && K <= a.nk) acc += (double)a.cz[czi(a, o, K, j, i)];
            }
            // the s*divx term and the open-side divergence pieces
            const float lt = lam_total(a, k, j, i);
            acc += (double)lt * (double)a.divx[cidx(a, k - 1, j, i)];
            if (x_edit(a, k, j, i)) {
                const float du = a.rru[uidx(a, k, y, x + 1)] - a.rru[uidx(a, k, y, x)];
                acc -= (double)lt * (double)du * (double)a.rdx;
            }
            if (y_edit(a, k, j, i)) {
                const float dv = a.rrv[vidx(a, k, y + 1, x)] - a.rrv[vidx(a, k, y, x)];
                acc -= (double)lt * (double)dv * (double)a.rdy;
            }
        }
    }
    return acc;
}

// pass 2, padded output: grid (ceil((ni+6)/32), ceil((nj+6)/8), nk+2), one
// thread per padded word
__global__ void __launch_bounds__(256) advection_adjoint_gather_kernel(const __grid_constant__ AdvAdjArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (x >= a.ni + 2 * kNg || y >= a.nj + 2 * kNg) return;
    a.out[pidx(a, k, y, x)] = (float)padded_adjoint(a, k, y, x);
}

// The open-filled carrier's map from padded word (y, x) to the compact cell
// it holds: (clamp(y), clamp(x)) when y is an interior row or x lies in
// x0-1..xl+1, nothing otherwise (bcs fills the west/east halo columns of rows
// y0-1..yl+1 first, then the south/north halo rows of columns x0-1..xl+1).
// pass 2, compact output: one thread per compact cell sums the padded
// adjoints of its preimage words (one word inside, up to 16 at a corner)
__device__ __noinline__ double edge_preimage_adjoint(const AdvAdjArgs &a, int k, int j, int i) {
    const int x0 = kNg, xl = kNg + a.ni - 1, y0 = kNg, yl = kNg + a.nj - 1;
    const int xa = i == 0 ? 0 : i + kNg, xb = i == a.ni - 1 ? xl + kNg : i + kNg;
    const int ya = j == 0 ? 0 : j + kNg, yb = j == a.nj - 1 ? yl + kNg : j + kNg;
    double acc = 0.0;
    for (int y = ya; y <= yb; ++y) {
        const bool row_in = y >= y0 && y <= yl;
        for (int x = xa; x <= xb; ++x)
            if (row_in || (x >= x0 - 1 && x <= xl + 1)) acc += padded_adjoint(a, k, y, x);
    }
    return acc;
}

// grid (ceil(ni/32), ceil(nj/8), nk)
__global__ void __launch_bounds__(256, 4) advection_adjoint_gather_compact_kernel(const __grid_constant__ AdvAdjArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i >= a.ni || j >= a.nj) return;
    const int q = cidx(a, k - 1, j, i);
    const bool edge = i == 0 || j == 0 || i == a.ni - 1 || j == a.nj - 1;
    const double acc = edge ? edge_preimage_adjoint(a, k, j, i) : padded_adjoint(a, k, j + kNg, i + kNg);
    if (a.sum_out != nullptr) {
        a.out[q] = (float)acc;
        a.sum_out[q] = a.base[q] + (float)acc;
    } else {
        a.out[q] = a.base != nullptr ? a.base[q] + (float)acc : (float)acc;
    }
}

// the open-filled carrier in one pass: the compact scalar inside, each halo
// word by the map above, levels 0 and nk+1 and the unfilled corner words 0
// grid (ceil((ni+6)/32), ceil((nj+6)/8), nk+2)
__global__ void scalar_carrier_open_kernel(const float *__restrict__ scalar, float *__restrict__ padded, int ni, int nj,
                                           int nk) {
    const int px = ni + 2 * kNg, py = nj + 2 * kNg;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (x >= px || y >= py) return;
    const int x0 = kNg, xl = kNg + ni - 1, y0 = kNg, yl = kNg + nj - 1;
    float v = 0.0f;
    if (k >= 1 && k <= nk && ((y >= y0 && y <= yl) || (x >= x0 - 1 && x <= xl + 1))) {
        const int cx = min(max(x, x0), xl) - kNg, cy = min(max(y, y0), yl) - kNg;
        v = __ldg(scalar + ((k - 1) * nj + cy) * ni + cx);
    }
    padded[(k * py + y) * px + x] = v;
}

// transpose of the scalar open fill: halo adjoints fold onto the edge cells
// they were copied from, the halo words become zero.  pass 1: the south /
// north halo rows (columns x0-1..xl+1), pass 2: the west / east halo
// columns (rows y0-1..yl+1) - the reverse of the fill's order.
__global__ void open_fill_adjoint_kernel(float *q, int ni, int nj, int nk, int pass) {
    const int px = ni + 2 * kNg, py = nj + 2 * kNg;
    const int lines = pass == 1 ? ni + 2 : nj + 2;
    const int total = nk * lines * 2;
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < total; z += gridDim.x * blockDim.x) {
        const int side = z % 2, l = (z / 2) % lines, k = 1 + z / (2 * lines);
        float *lev = q + (size_t)k * py * px;
        if (pass == 1) {
            const int x = kNg - 1 + l;
            const int src = side == 0 ? kNg : kNg + nj - 1;
            float sum = 0.0f;
            for (int h = 1; h <= kNg; ++h) {
                const int y = side == 0 ? src - h : src + h;
                sum += lev[(size_t)y * px + x];
                lev[(size_t)y * px + x] = 0.0f;
            }
            lev[(size_t)src * px + x] += sum;
        } else {
            const int y = kNg - 1 + l;
            const int src = side == 0 ? kNg : kNg + ni - 1;
            float sum = 0.0f;
            for (int h = 1; h <= kNg; ++h) {
                const int x = side == 0 ? src - h : src + h;
                sum += lev[(size_t)y * px + x];
                lev[(size_t)y * px + x] = 0.0f;
            }
            lev[(size_t)y * px + src] += sum;
        }
    }
}

// forward and transposed tridiagonal solves, one thread per column; levels
// are `stride` words apart (column-major over the plane)
__global__ void tridiagonal_kernel(const float *a, const float *b, const float *c, const float *d, float *x,
                                   float *work, int n, size_t ncol, int transposed) {
    const size_t col = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
#define L(p, k) p[(size_t)(k) * ncol + col]
    // A x = d with A(k, k-1) = a(k), A(k, k) = b(k), A(k, k+1) = c(k);
    // transposed: A^T has sub-diagonal c(k-1), super-diagonal a(k+1)
    float cprev = 0.0f, dprev = 0.0f;
    for (int k = 0; k < n; ++k) {
        const float lo = k == 0 ? 0.0f : (transposed ? L(c, k - 1) : L(a, k));
        const float up = k == n - 1 ? 0.0f : (transposed ? L(a, k + 1) : L(c, k));
        const float piv = L(b, k) - lo * cprev;
        const float inv = 1.0f / piv;
        cprev = up * inv;
        dprev = (L(d, k) - lo * dprev) * inv;
        L(work, k) = cprev;
        L(x, k) = dprev;
    }
    for (int k = n - 2; k >= 0; --k) L(x, k) = L(x, k) - L(work, k) * L(x, k + 1);
#undef L
}

// autoconversion + accretion with the qc limiter, and its adjoint
__device__ __forceinline__ void collection(float qc, float qr, float dt, float &ar, float &cr) {
    ar = 0.0f;
    cr = 0.0f;
    if (qc > 0.0f) ar = pymax(0.001f * (qc - 0.001f), 0.0f) * dt;
    if (qc > 0.0f && qr > 0.0f) cr = ((2.2f * qc) * powf(qr, 0.875f)) * dt;
    if (ar + cr > qc) {
        const float t = ar + cr;
        ar = (qc * ar) / t;
        cr = (qc * cr) / t;
    }
}

__global__ void kessler_collection_kernel(float *qc, float *qr, size_t n, float dt) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        float ar, cr;
        const float c = qc[p], r = qr[p];
        collection(c, r, dt, ar, cr);
        qc[p] = c - (ar + cr);
        qr[p] = r + (ar + cr);
    }
}

// given the forward inputs qc, qr and the output adjoints gc, gr, overwrite
// gc, gr with the input adjoints.  The converted amount t is ar + cr, or qc
// when the limiter is active (the binary32 forward's own branch decides);
// qc' = qc - t, qr' = qr + t.
__device__ __forceinline__ void collection_adjoint_cell(float c, float r, float dt, float &gc, float &gr) {
    double dt_dc = 0.0, dt_dr = 0.0;
    // autoconversion: subgradient 0 at the switch qc = 0.001
    if (c > 0.0f && 0.001f * (c - 0.001f) > 0.0f) dt_dc += 0.001 * (double)dt;
    // accretion: qr^0.875 has no derivative at qr = 0, where it is gated off
    if (c > 0.0f && r > 0.0f) {
        const double rp = pow((double)r, 0.875);
        dt_dc += 2.2 * rp * (double)dt;
        dt_dr += 2.2 * (double)c * 0.875 * pow((double)r, -0.125) * (double)dt;
    }
    float ar32 = 0.0f, cr32 = 0.0f;
    if (c > 0.0f) ar32 = pymax(0.001f * (c - 0.001f), 0.0f) * dt;
    if (c > 0.0f && r > 0.0f) cr32 = ((2.2f * c) * powf(r, 0.875f)) * dt;
    if (ar32 + cr32 > c) {
        dt_dc = 1.0;
        dt_dr = 0.0;
    }
    const double g_c = gc, g_r = gr;
    const double gt = g_r - g_c;
    gc = (float)(g_c + gt * dt_dc);
    gr = (float)(g_r + gt * dt_dr);
}

__global__ void kessler_collection_adjoint_kernel(const float *qc, const float *qr, float *gc, float *gr, size_t n,
                                                  float dt) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        float a = gc[p], b = gr[p];
        collection_adjoint_cell(qc[p], qr[p], dt, a, b);
        gc[p] = a;
        gr[p] = b;
    }
}

// ---- single-pass saturation adjustment (equation set 1) --------------------
// The eqtset = 1 branch of the Kessler operator's saturation adjustment
// (_cpu_satadj, src/cm1core/cuda_gm1_kessler_driver.py:337-428): one
// Newton-like step towards saturation at the frozen pressure, limited to the
// available cloud water, with its latent heating of theta'.
struct SatConst {
    float cp, eps, lv1, lv2;
};

__host__ SatConst sat_constants() {
    const float rd = 287.04f, rv = 461.5f, cpv = 1870.0f, cpl = 4190.0f, xlv = 2501000.0f;
    SatConst c;
    c.cp = 1005.7f;
    c.eps = rd / rv;
    c.lv2 = cpl - cpv;
    c.lv1 = xlv + c.lv2 * 273.15f;
    return c;
}

__device__ __forceinline__ float pymin(float a, float b) { return (b < a) ? b : a; }

// the forward on one cell, in place on th3d, qv, qc
__device__ __forceinline__ void satadj1_cell(const SatConst &c, float th0, float pi0, float pp3d, float pr, float &th3d,
                                             float &qv, float &qc) {
    const float pisum = pi0 + pp3d;
    const float tnew = (th0 + th3d) * pisum;
    float esl = 611.2f * expf((17.67f * (tnew - 273.15f)) / (tnew - 29.65f));
    esl = pymin(esl, pr * 0.5f);
    const float qvs = (c.eps * esl) / (pr - esl);
    const float lhv = c.lv1 - c.lv2 * tnew;
    const float square = (tnew - 29.65f) * (tnew - 29.65f);
    const float numerator = ((lhv * qvs) * 17.67f) * 243.5f;
    const float qvn = qv, qcn = qc;
    float dqv = (qvs - qvn) / (1.0f + numerator / (c.cp * square));
    if (qvn + dqv < 1.0e-20f) dqv = 1.0e-20f - qvn;
    dqv = pymin(dqv, pymax(0.0f, qcn));
    qv = qvn + dqv;
    qc = qcn - dqv;
    th3d = th3d - dqv * (lhv / (c.cp * pisum));
}

__global__ void satadj1_kernel(const float *th0, const float *pi0, const float *pp3d, const float *prs, float *th3d,
                               float *qv, float *qc, size_t n, SatConst c) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        float t = th3d[p], v = qv[p], w = qc[p];
        satadj1_cell(c, th0[p], pi0[p], pp3d[p], prs[p], t, v, w);
        th3d[p] = t;
        qv[p] = v;
        qc[p] = w;
    }
}

// adjoint on one cell: the forward's inputs (th3d, qv, qc before the step)
// and the output adjoints in g_th, g_qv, g_qc, overwritten with the input
// adjoints.  Branches are the binary32 forward's own; the cap of esl at half
// the pressure, the 1e-20 floor and the cloud-water limit each
// differentiate as the branch they took (subgradient of the limiter at
// equality: the unlimited branch's when dqv <= qc).
__device__ __forceinline__ void satadj1_adjoint_cell(const SatConst &c, float th0, float pi0, float pp3d, float pr,
                                                     float th3d, float qvn, float qcn, float &g_th, float &g_qv,
                                                     float &g_qc) {
    const float pisum = pi0 + pp3d;
    const float tnew = (th0 + th3d) * pisum;
    const float eraw = 611.2f * expf((17.67f * (tnew - 273.15f)) / (tnew - 29.65f));
    const bool capped = (pr * 0.5f < eraw);  // the branch pymin(eraw, half) takes
    const float esl = pymin(eraw, pr * 0.5f);
    const float qvs = (c.eps * esl) / (pr - esl);
    const float lhv = c.lv1 - c.lv2 * tnew;
    const float square = (tnew - 29.65f) * (tnew - 29.65f);
    const float numerator = ((lhv * qvs) * 17.67f) * 243.5f;
    const float den = 1.0f + numerator / (c.cp * square);
    float dqv = (qvs - qvn) / den;
    int branch = 0;  // 0 raw, 1 floor, 2 cloud-water limit
    if (qvn + dqv < 1.0e-20f) {
        dqv = 1.0e-20f - qvn;
        branch = 1;
    }
    const float lim = pymax(0.0f, qcn);
    if (lim < dqv) {
        dqv = lim;
        branch = 2;
    }
    // derivatives of the raw dqv with respect to T and qv (binary64)
    const double T = tnew, P = pr, tm = T - 29.65, E = esl;
    const double dE = capped ? 0.0 : (double)eraw * (17.67 * 243.5) / (tm * tm);
    const double dqvs = (double)c.eps * P * dE / ((P - E) * (P - E));
    const double dlhv = -(double)c.lv2;
    const double sq = tm * tm, dsq = 2.0 * tm;
    const double num = (double)lhv * (double)qvs * 17.67 * 243.5;
    const double dnum = 17.67 * 243.5 * (dlhv * (double)qvs + (double)lhv * dqvs);
    const double D = (double)den, dD = (dnum * sq - num * dsq) / ((double)c.cp * sq * sq);
    const double raw = ((double)qvs - (double)qvn);
    double ddq_dT = (dqvs * D - raw * dD) / (D * D), ddq_dqv = -1.0 / D, ddq_dqc = 0.0;
    if (branch == 1) {
        ddq_dT = 0.0;
        ddq_dqv = -1.0;
    } else if (branch == 2) {
        ddq_dT = 0.0;
        ddq_dqv = 0.0;
        ddq_dqc = qcn > 0.0f ? 1.0 : 0.0;
    }
    const double pis = pisum;
    const double L = (double)lhv / ((double)c.cp * pis), dL_dT = dlhv / ((double)c.cp * pis);
    const double gth = g_th, gv = g_qv, gcc = g_qc;
    const double gd = gv - gcc - gth * L;  // adjoint of dqv
    // th3d_out = th3d - dqv * L(T), T = (th0 + th3d) * pisum
    g_th = (float)(gth + (gd * ddq_dT - gth * (double)dqv * dL_dT) * pis);
    g_qv = (float)(gv + gd * ddq_dqv);
    g_qc = (float)(gcc + gd * ddq_dqc);
}

__global__ void satadj1_adjoint_kernel(const float *th0, const float *pi0, const float *pp3d, const float *prs,
                                       const float *th3d, const float *qv, const float *qc, float *g_th, float *g_qv,
                                       float *g_qc, size_t n, SatConst c) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        float a = g_th[p], b = g_qv[p], d = g_qc[p];
        satadj1_adjoint_cell(c, th0[p], pi0[p], pp3d[p], prs[p], th3d[p], qv[p], qc[p], a, b, d);
        g_th[p] = a;
        g_qv[p] = b;
        g_qc[p] = d;
    }
}

// The cell step of the warm-rain transport model after its transport:
// qc, qr clipped at 0 (x < 0 ? 0 : x, NaN kept), collection, satadj1 -
// the words of those three pieces run one after another.  state: th3d,
// qv, qc, qr (4 arrays of n words); out likewise.
struct WarmRainArgs {
    const float *th0, *pi0, *pp3d, *prs;
    const float *s[4];
    const float *lam[4];  // adjoint only: dJ/d(out)
    float *out[4];
    size_t n;
    float dt;
    SatConst c;
};

__device__ __forceinline__ float clip0(float x) { return x < 0.0f ? 0.0f : x; }

__global__ void warm_rain_cell_kernel(const __grid_constant__ WarmRainArgs a) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += (size_t)gridDim.x * blockDim.x) {
        float th = a.s[0][p], qv = a.s[1][p];
        const float c = clip0(a.s[2][p]), r = clip0(a.s[3][p]);
        float ar, cr;
        collection(c, r, a.dt, ar, cr);
        float qc = c - (ar + cr);
        const float qr = r + (ar + cr);
        satadj1_cell(a.c, a.th0[p], a.pi0[p], a.pp3d[p], a.prs[p], th, qv, qc);
        a.out[0][p] = th;
        a.out[1][p] = qv;
        a.out[2][p] = qc;
        a.out[3][p] = qr;
    }
}

// its adjoint: from the transported state s and dJ/d(out), dJ/d(s); the
// clip passes the adjoint where s >= 0 (as g * (s >= 0))
__global__ void warm_rain_cell_adjoint_kernel(const __grid_constant__ WarmRainArgs a) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += (size_t)gridDim.x * blockDim.x) {
        const float th = a.s[0][p], qv = a.s[1][p], qc0 = a.s[2][p], qr0 = a.s[3][p];
        const float c = clip0(qc0), r = clip0(qr0);
        float ar, cr;
        collection(c, r, a.dt, ar, cr);
        const float qc1 = c - (ar + cr);
        float g_th = a.lam[0][p], g_qv = a.lam[1][p], g_qc = a.lam[2][p], g_qr = a.lam[3][p];
        satadj1_adjoint_cell(a.c, a.th0[p], a.pi0[p], a.pp3d[p], a.prs[p], th, qv, qc1, g_th, g_qv, g_qc);
        collection_adjoint_cell(c, r, a.dt, g_qc, g_qr);
        a.out[0][p] = g_th;
        a.out[1][p] = g_qv;
        a.out[2][p] = g_qc * (float)(qc0 >= 0.0f);
        a.out[3][p] = g_qr * (float)(qr0 >= 0.0f);
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

unsigned grid_for(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 32); }

}  // namespace
}  // namespace gm1b

using namespace gm1b;

namespace {
size_t adjoint_face_words(int ni, int nj, int nk) {
    return 6 * ((size_t)nk * nj * (ni + 1) + (size_t)nk * (nj + 1) * ni + (size_t)(nk + 1) * nj * ni);
}

int32_t advection_adjoint_launch(const char *who, int32_t ni, int32_t nj, int32_t nk,
                                 const gm1b_scalar_advection5_adjoint_arrays *arrays, int32_t nrk, int32_t wflag,
                                 float dx, float dy, float dz, double weps, uint32_t lateral_obc, void *workspace,
                                 bool compact, float lam_scale, const float *base, float *sum_out, void *stream) {
    if (arrays == nullptr || ni < 8 || nj < 8 || nk < 8 || nrk < 1 || nrk > 3) {
        gm1b_set_error("%s: need arrays, ni, nj, nk >= 8 and nrk in 1..3", who);
        return GM1B_ERR_ARGUMENT;
    }
    if (lateral_obc == 0u) {
        gm1b_set_error("%s: the whole-domain operator only (lateral_obc != 0)", who);
        return GM1B_ERR_ARGUMENT;
    }
    if (compact && lateral_obc != 0x2222u) {
        gm1b_set_error("%s: the compact form folds the all-open carrier fill (lateral_obc 0x2222)", who);
        return GM1B_ERR_ARGUMENT;
    }
    const gm1b_scalar_advection5_adjoint_arrays &s = *arrays;
    const void *need[] = {s.scalar, s.rru, s.rrv, s.rrw, s.c1, s.c2, s.rr0, s.gz, s.divx, s.tendency_adjoint,
                          s.scalar_adjoint, workspace};
    for (const void *p : need)
        if (p == nullptr) {
            gm1b_set_error("%s: a required array or the workspace is NULL", who);
            return GM1B_ERR_ARGUMENT;
        }
    if (!(dx > 0.0f) || !(dy > 0.0f) || !(dz > 0.0f)) {
        gm1b_set_error("%s: dx, dy, dz must be > 0", who);
        return GM1B_ERR_ARGUMENT;
    }
    if (adjoint_face_words(ni, nj, nk) >= (size_t)1 << 31 || nk + 2 > 65535) {
        gm1b_set_error("%s: the face scratch must hold fewer than 2^31 words (32-bit offsets)", who);
        return GM1B_ERR_ARGUMENT;
    }
    AdvAdjArgs a;
    a.s = s.scalar;
    a.rru = s.rru;
    a.rrv = s.rrv;
    a.rrw = s.rrw;
    a.c1 = s.c1;
    a.c2 = s.c2;
    a.rr0 = s.rr0;
    a.gz = s.gz;
    a.divx = s.divx;
    a.lam = s.tendency_adjoint;
    a.out = s.scalar_adjoint;
    a.base = base;
    a.sum_out = sum_out;
    a.lam_scale = lam_scale;
    if (sum_out != nullptr && base == nullptr) {
        gm1b_set_error("%s: a running sum needs the accumulate input", who);
        return GM1B_ERR_ARGUMENT;
    }
    a.compact_scalar = compact ? 1 : 0;
    a.cx = static_cast<float *>(workspace);
    a.cy = a.cx + 6 * (size_t)nk * nj * (ni + 1);
    a.cz = a.cy + 6 * (size_t)nk * (nj + 1) * ni;
    a.ni = ni;
    a.nj = nj;
    a.nk = nk;
    a.weno = (wflag && nrk == 3) ? 1 : 0;
    a.obc = lateral_obc;
    a.rdx = 1.0f / dx;
    a.rdy = 1.0f / dy;
    a.rdz = 1.0f / dz;
    a.eps = weps;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    {
        ProfScope ps(a.weno ? "advection_adjoint_faces_weno_kernel" : "advection_adjoint_faces_kernel", st);
        advection_adjoint_faces_kernel<<<dim3((ni + 1 + 31) / 32, (nj + 1 + 7) / 8, nk + 1), dim3(32, 8), 0, st>>>(a);
        ps.stop();
        if (!launch_ok("advection_adjoint_faces_kernel")) return GM1B_ERR_CUDA;
    }
    if (compact) {
        ProfScope ps("advection_adjoint_gather_compact_kernel", st);
        advection_adjoint_gather_compact_kernel<<<dim3((ni + 31) / 32, (nj + 7) / 8, nk), dim3(32, 8), 0, st>>>(a);
        ps.stop();
        return launch_ok("advection_adjoint_gather_compact_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
    }
    ProfScope ps("advection_adjoint_gather_kernel", st);
    advection_adjoint_gather_kernel<<<dim3((ni + 6 + 31) / 32, (nj + 6 + 7) / 8, nk + 2), dim3(32, 8), 0, st>>>(a);
    ps.stop();
    return launch_ok("advection_adjoint_gather_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}
}  // namespace

extern "C" size_t gm1b_scalar_advection5_adjoint_workspace_bytes(int32_t ni, int32_t nj, int32_t nk) {
    if (ni < 1 || nj < 1 || nk < 1) return 0;
    return 4 * adjoint_face_words(ni, nj, nk);
}

extern "C" int32_t gm1b_scalar_advection5_adjoint(int32_t ni, int32_t nj, int32_t nk,
                                                  const gm1b_scalar_advection5_adjoint_arrays *arrays, int32_t nrk,
                                                  int32_t wflag, float dx, float dy, float dz, double weps,
                                                  uint32_t lateral_obc, void *workspace, void *stream) {
    return advection_adjoint_launch("gm1b_scalar_advection5_adjoint", ni, nj, nk, arrays, nrk, wflag, dx, dy, dz,
                                    weps, lateral_obc, workspace, false, 1.0f, nullptr, nullptr, stream);
}

extern "C" int32_t gm1b_scalar_advection5_adjoint_open(int32_t ni, int32_t nj, int32_t nk,
                                                       const gm1b_scalar_advection5_adjoint_arrays *arrays,
                                                       int32_t nrk, int32_t wflag, float dx, float dy, float dz,
                                                       double weps, float adjoint_scale, const float *accumulate,
                                                       float *running_sum, void *workspace, void *stream) {
    return advection_adjoint_launch("gm1b_scalar_advection5_adjoint_open", ni, nj, nk, arrays, nrk, wflag, dx, dy,
                                    dz, weps, 0x2222u, workspace, true, adjoint_scale, accumulate, running_sum, stream);
}

extern "C" int32_t gm1b_scalar_carrier_open(int32_t ni, int32_t nj, int32_t nk, const float *scalar, float *padded,
                                            void *stream) {
    if (scalar == nullptr || padded == nullptr || ni < 1 || nj < 1 || nk < 1) {
        gm1b_set_error("gm1b_scalar_carrier_open: need scalar, padded and ni, nj, nk >= 1");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("scalar_carrier_open_kernel", st);
    if ((size_t)(nk + 2) * (nj + 6) * (ni + 6) >= (size_t)1 << 31 || nk + 2 > 65535) {
        gm1b_set_error("gm1b_scalar_carrier_open: the carrier must hold fewer than 2^31 words, nk <= 65533");
        return GM1B_ERR_ARGUMENT;
    }
    scalar_carrier_open_kernel<<<dim3((ni + 6 + 31) / 32, (nj + 6 + 7) / 8, nk + 2), dim3(32, 8), 0, st>>>(scalar, padded,
                                                                                                          ni, nj, nk);
    ps.stop();
    return launch_ok("scalar_carrier_open_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_open_fill_scalar_adjoint(int32_t ni, int32_t nj, int32_t nk, float *q, void *stream) {
    if (q == nullptr || ni < 1 || nj < 1 || nk < 1) {
        gm1b_set_error("gm1b_open_fill_scalar_adjoint: need q and ni, nj, nk >= 1");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (int pass = 1; pass <= 2; ++pass) {
        const size_t total = (size_t)nk * (pass == 1 ? ni + 2 : nj + 2) * 2;
        ProfScope ps("open_fill_adjoint_kernel", st);
        open_fill_adjoint_kernel<<<grid_for(total), 256, 0, st>>>(q, ni, nj, nk, pass);
        ps.stop();
        if (!launch_ok("open_fill_adjoint_kernel")) return GM1B_ERR_CUDA;
    }
    return GM1B_OK;
}

extern "C" int32_t gm1b_tridiagonal_solve(int32_t n, size_t columns, const float *a, const float *b, const float *c,
                                          const float *d, float *x, float *work, int32_t transposed, void *stream) {
    if (n < 2 || columns < 1 || !a || !b || !c || !d || !x || !work) {
        gm1b_set_error("gm1b_tridiagonal_solve: need n >= 2, columns >= 1 and every array");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps(transposed ? "tridiagonal_adjoint_kernel" : "tridiagonal_kernel", st);
    tridiagonal_kernel<<<(unsigned)((columns + 127) / 128), 128, 0, st>>>(a, b, c, d, x, work, n, columns,
                                                                           transposed ? 1 : 0);
    ps.stop();
    return launch_ok("tridiagonal_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_kessler_collection(size_t cells, float *qc, float *qr, float dt, void *stream) {
    if (!qc || !qr || cells < 1 || !(dt > 0.0f)) {
        gm1b_set_error("gm1b_kessler_collection: need qc, qr, cells >= 1 and dt > 0");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("kessler_collection_kernel", st);
    kessler_collection_kernel<<<grid_for(cells), 256, 0, st>>>(qc, qr, cells, dt);
    ps.stop();
    return launch_ok("kessler_collection_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_kessler_collection_adjoint(size_t cells, const float *qc, const float *qr, float *gc,
                                                   float *gr, float dt, void *stream) {
    if (!qc || !qr || !gc || !gr || cells < 1 || !(dt > 0.0f)) {
        gm1b_set_error("gm1b_kessler_collection_adjoint: need every array, cells >= 1 and dt > 0");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("kessler_collection_adjoint_kernel", st);
    kessler_collection_adjoint_kernel<<<grid_for(cells), 256, 0, st>>>(qc, qr, gc, gr, cells, dt);
    ps.stop();
    return launch_ok("kessler_collection_adjoint_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_satadj1(size_t cells, const float *th0, const float *pi0, const float *pp3d, const float *prs,
                                float *th3d, float *qv, float *qc, void *stream) {
    if (!th0 || !pi0 || !pp3d || !prs || !th3d || !qv || !qc || cells < 1) {
        gm1b_set_error("gm1b_satadj1: need every array and cells >= 1");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("satadj1_kernel", st);
    satadj1_kernel<<<grid_for(cells), 256, 0, st>>>(th0, pi0, pp3d, prs, th3d, qv, qc, cells, sat_constants());
    ps.stop();
    return launch_ok("satadj1_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_satadj1_adjoint(size_t cells, const float *th0, const float *pi0, const float *pp3d,
                                        const float *prs, const float *th3d, const float *qv, const float *qc,
                                        float *g_th, float *g_qv, float *g_qc, void *stream) {
    if (!th0 || !pi0 || !pp3d || !prs || !th3d || !qv || !qc || !g_th || !g_qv || !g_qc || cells < 1) {
        gm1b_set_error("gm1b_satadj1_adjoint: need every array and cells >= 1");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("satadj1_adjoint_kernel", st);
    satadj1_adjoint_kernel<<<grid_for(cells), 256, 0, st>>>(th0, pi0, pp3d, prs, th3d, qv, qc, g_th, g_qv, g_qc, cells,
                                                            sat_constants());
    ps.stop();
    return launch_ok("satadj1_adjoint_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

namespace {
int32_t warm_rain_launch(bool adjoint, size_t cells, const float *th0, const float *pi0, const float *pp3d,
                         const float *prs, const float *const *state, const float *const *lam, float *const *out,
                         float dt, void *stream) {
    const char *who = adjoint ? "gm1b_warm_rain_cell_adjoint" : "gm1b_warm_rain_cell";
    if (!th0 || !pi0 || !pp3d || !prs || !state || !out || (adjoint && !lam) || cells < 1 || !(dt > 0.0f)) {
        gm1b_set_error("%s: need every array, cells >= 1 and dt > 0", who);
        return GM1B_ERR_ARGUMENT;
    }
    WarmRainArgs a;
    a.th0 = th0;
    a.pi0 = pi0;
    a.pp3d = pp3d;
    a.prs = prs;
    for (int q = 0; q < 4; ++q) {
        a.s[q] = state[q];
        a.lam[q] = adjoint ? lam[q] : nullptr;
        a.out[q] = out[q];
        if (!a.s[q] || !a.out[q] || (adjoint && !a.lam[q])) {
            gm1b_set_error("%s: a state, adjoint or output array is NULL", who);
            return GM1B_ERR_ARGUMENT;
        }
    }
    a.n = cells;
    a.dt = dt;
    a.c = sat_constants();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps(adjoint ? "warm_rain_cell_adjoint_kernel" : "warm_rain_cell_kernel", st);
    if (adjoint)
        warm_rain_cell_adjoint_kernel<<<grid_for(cells), 256, 0, st>>>(a);
    else
        warm_rain_cell_kernel<<<grid_for(cells), 256, 0, st>>>(a);
    ps.stop();
    return launch_ok(who) ? GM1B_OK : GM1B_ERR_CUDA;
}
}  // namespace

extern "C" int32_t gm1b_warm_rain_cell(size_t cells, const float *th0, const float *pi0, const float *pp3d,
                                       const float *prs, const float *const *state, float *const *out, float dt,
                                       void *stream) {
    return warm_rain_launch(false, cells, th0, pi0, pp3d, prs, state, nullptr, out, dt, stream);
}

extern "C" int32_t gm1b_warm_rain_cell_adjoint(size_t cells, const float *th0, const float *pi0, const float *pp3d,
                                               const float *prs, const float *const *state,
                                               const float *const *out_adjoint, float *const *state_adjoint, float dt,
                                               void *stream) {
    return warm_rain_launch(true, cells, th0, pi0, pp3d, prs, state, out_adjoint, state_adjoint, dt, stream);
}
