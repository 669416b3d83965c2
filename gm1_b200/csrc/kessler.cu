// kessler.cu - sm_100a kernels of the complete Kessler warm-rain operator
// (ptype = 1, efall = 0): pdefq(qv, qc, qr), rain fall speed and rain-energy
// budget, fallout sub-stepping, local conversion and saturation adjustment,
// with the FP64 budgets.
//
// Behaviour followed (reference file:line):
//   cpu_gm1_kessler_driver_inplace  src/cm1core/cuda_gm1_kessler_driver.py:431-559
//   _cpu_pdefq                      src/cm1core/cuda_gm1_kessler_driver.py:300-335
//   _cpu_satadj                     src/cm1core/cuda_gm1_kessler_driver.py:337-428
//   cpu_gm1_kessler_local_inplace   src/cm1core/cuda_gm1_kessler_local.py:251-432
//
// Design (B200): the reference runs its column phases one thread per j ROW
// (serial over i, k and the fallout sub-steps) and its budget finishes on a
// single thread.  Here every COLUMN is a thread (pdefq x3, fall speed,
// nfall, the fallout sub-steps marching up k with the flux of the level
// above carried in a register), every CELL is a thread for the local
// conversion fused with the saturation adjustment, and the FP64 budgets are
// reduced in a fixed order: per-column sums in the twin's k order, row sums
// in its i order, then a short ordered finish.  The budget scratch lives in a
// caller-provided workspace; its first 16 bytes are status words.
#include <mutex>

#include "gm1b_common.cuh"

namespace gm1b {
namespace {

constexpr int kMaxFallSubsteps = 1 << 14;  // bound of the fallout sub-steps of one column
constexpr int kKX = 128;  // cell-kernel CTA: a run of 128 cells of one row at one level
constexpr int kCX = 32, kCY = 4;

struct KConst {
    float rd, cp, cpv, rv, xlv, cv, cvv, rovcp, eps, reps, cpl, lv2, lv1, rp00, cpdcv, rddcv, cpdrd, p00;
};

__host__ KConst make_constants() {
    KConst c;
    c.rd = 287.04f;
    c.cp = 1005.7f;
    c.cpv = 1870.0f;
    c.rv = 461.5f;
    c.xlv = 2501000.0f;
    c.cv = c.cp - c.rd;
    c.cvv = c.cpv - c.rv;
    c.rovcp = c.rd / c.cp;
    c.eps = c.rd / c.rv;
    c.reps = c.rv / c.rd;
    c.cpl = 4190.0f;
    c.lv2 = c.cpl - c.cpv;
    c.lv1 = c.xlv + c.lv2 * 273.15f;
    c.p00 = 1.0e5f;
    c.rp00 = 1.0f / c.p00;
    c.cpdcv = c.cp / c.cv;
    c.rddcv = c.rd / c.cv;
    c.cpdrd = c.cp / c.rd;
    return c;
}

__device__ __forceinline__ float pymax(float a, float b) { return (b > a) ? b : a; }
__device__ __forceinline__ float pymin(float a, float b) { return (b < a) ? b : a; }

__device__ __forceinline__ float esl_capped(float t, float prs) {
    const float esl = 611.2f * expf((17.67f * (t - 273.15f)) / (t - 29.65f));
    return pymin(esl, prs * 0.5f);
}

struct KDims {
    int ni, nj, nk;
    __device__ __forceinline__ size_t c(int k, int j, int i) const {
        return ((size_t)k * nj + (size_t)j) * (size_t)ni + (size_t)i;
    }
};

// workspace layout (doubles after a 16-byte status block)
struct KWork {
    int32_t *status;   // [0] satadj non-converged cells, [1] max fallout sub-steps,
                       // [2] columns whose fall Courant number was not finite or >= kMaxFallSubsteps
    double *colterm;   // [5][nj*ni]
    double *rows;      // [5][nj]
    double *partial;   // [5][nk][nj][nbx]
    int nbx;
};

__host__ size_t workspace_bytes(int ni, int nj, int nk) {
    const size_t ncol = (size_t)ni * nj;
    const size_t nbx = (size_t)((ni + kKX - 1) / kKX);
    return 16 + sizeof(double) * (5 * ncol + 5 * (size_t)nj + 5 * (size_t)nk * nj * nbx);
}

__host__ KWork carve(void *ws, int ni, int nj, int nk) {
    KWork w;
    char *p = static_cast<char *>(ws);
    w.status = reinterpret_cast<int32_t *>(p);
    w.colterm = reinterpret_cast<double *>(p + 16);
    w.rows = w.colterm + 5 * (size_t)ni * nj;
    w.partial = w.rows + 5 * (size_t)nj;
    w.nbx = (ni + kKX - 1) / kKX;
    return w;
}

// pdefq of one column: returns a2 - a1 and rescales q in place
__device__ __forceinline__ double pdefq_column(const gm1b_kessler_arrays &a, float *q, float rmax, const KDims &d,
                                               int j, int i) {
    double t1 = 0.0, t2 = 0.0, a1 = 0.0, a2 = 0.0;
    const float ruh = a.ruh[i], rvh = a.rvh[j];
    for (int k = 0; k < d.nk; ++k) {
        const size_t p = d.c(k, j, i);
        const float rho = a.rho[p], qk = q[p], rmh = a.rmh[p];
        const float rq = rho * qk;
        t1 += (double)rq;
        const float cell = (((rho * qk) * ruh) * rvh) * rmh;
        a1 += (double)cell;
        const float qc = (qk < rmax) ? 0.0f : qk;
        t2 += (double)(rho * qc);
    }
    double t3 = (t1 + 1.0e-20) / (t2 + 1.0e-20);
    if (t3 < 0.0) t3 = 1.0;
    for (int k = 0; k < d.nk; ++k) {
        const size_t p = d.c(k, j, i);
        const float rho = a.rho[p];
        const float qk0 = q[p];
        const float qc = (qk0 < rmax) ? 0.0f : qk0;
        const float qn = (float)(t3 * (double)qc);
        q[p] = qn;
        const float cell = (((rho * qn) * ruh) * rvh) * a.rmh[p];
        a2 += (double)cell;
    }
    return a2 - a1;
}

// grid (ceil(ni/32), ceil(nj/4)): one thread per column
__global__ void __launch_bounds__(kCX *kCY)
    kessler_column_kernel(gm1b_kessler_arrays a, KDims d, KWork w, KConst c, float dt, float rdz) {
    const int i = blockIdx.x * kCX + threadIdx.x;
    const int j = blockIdx.y * kCY + threadIdx.y;
    if (i >= d.ni || j >= d.nj) return;
    const int nk = d.nk;
    const size_t col = (size_t)j * d.ni + i;
    const size_t ncol = (size_t)d.ni * d.nj;
    const size_t p0 = d.c(0, j, i);
    const float temp0 = (a.th0[p0] + a.th3d[p0]) * (a.pi0[p0] + a.pp3d[p0]);
    w.colterm[0 * ncol + col] = pdefq_column(a, a.qv, 0.0f, d, j, i);
    w.colterm[1 * ncol + col] = pdefq_column(a, a.qc, 1.0e-14f, d, j, i);
    w.colterm[2 * ncol + col] = pdefq_column(a, a.qr, 1.0e-14f, d, j, i);
    // rain fall speed and the largest Courant number of the column
    float crmax = 0.0f;
    for (int k = 0; k < nk; ++k) {
        const size_t p = d.c(k, j, i);
        const float rho = a.rho[p], qr = a.qr[p];
        float v = 0.0f;
        if (qr > 1.0e-12f) v = (14.34f * powf(rho * qr, 0.1346f)) * sqrtf(1.15f / rho);
        a.fall_velocity[p] = v;
        crmax = pymax(crmax, ((v * dt) * rdz) * a.mh[p]);
    }
    const float ruh = a.ruh[i], rvh = a.rvh[j];
    {
        float term = dt * a.fall_velocity[p0];
        term = term * a.rr[p0];
        term = term * a.qr[p0];
        term = term * (c.cpl * temp0 - c.lv1);
        term = term * ruh;
        term = term * rvh;
        w.colterm[3 * ncol + col] = (double)term;
    }
    int nfall = (int)(crmax + 1.0f);
    if (nfall < 1) nfall = 1;
    // A column whose fall Courant number is not finite or above
    // kMaxFallSubsteps holds no physical state (rain or density already blew
    // up); int(crmax + 1) would reach 2^31 sub-steps.  It is counted in
    // status[2] and takes one sub-step, so the launch stays bounded and the
    // caller refuses the step.
    if (!(crmax < (float)kMaxFallSubsteps)) {
        atomicAdd(&w.status[2], 1);
        nfall = 1;
    }
    if (a.nfall != nullptr) a.nfall[col] = nfall;
    atomicMax(&w.status[1], nfall);
    // below-threshold rain takes the fall speed of the level above
    for (int k = nk - 2; k >= 0; --k) {
        const size_t p = d.c(k, j, i);
        if (a.qr[p] < 1.0e-8f) a.fall_velocity[p] = a.fall_velocity[d.c(k + 1, j, i)];
    }
    const float dtfall = dt / (float)nfall;
    double bud = 0.0;
    for (int n = 0; n < nfall; ++n) {
        float rq_k = (a.rho[p0] * a.fall_velocity[p0]) * pymax(0.0f, a.qr[p0]);
        const float rq0 = rq_k;
        for (int k = 0; k < nk; ++k) {
            const size_t p = d.c(k, j, i);
            float rq_up = 0.0f;
            if (k + 1 < nk) {
                const size_t pu = d.c(k + 1, j, i);
                rq_up = (a.rho[pu] * a.fall_velocity[pu]) * pymax(0.0f, a.qr[pu]);
            }
            const float delta = (((dtfall * (rq_up - rq_k)) * rdz) * a.mh[p]) / a.rho[p];
            a.qr[p] = a.qr[p] + delta;
            rq_k = rq_up;
        }
        a.rain[col] = a.rain[col] + (0.1f * dtfall) * rq0;
        a.prate[col] = rq0;
        float term = dtfall * a.rr[p0];
        term = term * a.fall_velocity[p0];
        term = term * pymax(0.0f, a.qr[p0]);
        term = term * ruh;
        term = term * rvh;
        bud += (double)term;
    }
    w.colterm[4 * ncol + col] = bud;
}

__device__ __forceinline__ double block_sum(double v, double *smem) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += smem[q];
    __syncthreads();
    return s;
}

// grid (nbx, nj, nk): one thread per cell; local conversion then satadj
__global__ void __launch_bounds__(kKX)
    kessler_cell_kernel(gm1b_kessler_arrays a, KDims d, KWork w, KConst c, float dt, int eqtset) {
    __shared__ double s_red[kKX / 32];
    const int i = blockIdx.x * kKX + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    double terms[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < d.ni) {
        const size_t p = d.c(k, j, i);
        const float th0 = a.th0[p], pi0 = a.pi0[p], rr = a.rr[p];
        float th3d = a.th3d[p], pp3d = a.pp3d[p], prs = a.prs[p], rho = a.rho[p];
        float qvnew = a.qv[p], qcnew = a.qc[p], qrnew = a.qr[p];
        const float tem = (a.ruh[i] * a.rvh[j]) * a.rmh[p];
        // --- local conversion ---
        {
            float pisum = pi0 + pp3d;
            const float tmp = (th0 + th3d) * pisum;
            float ar = 0.0f, cr = 0.0f, er = 0.0f;
            if (qcnew > 0.0f) {
                ar = pymax(0.001f * (qcnew - 0.001f), 0.0f);
                ar = ar * dt;
            }
            if (qcnew > 0.0f && qrnew > 0.0f) cr = ((2.2f * qcnew) * powf(qrnew, 0.875f)) * dt;
            if (qrnew > 0.0f) {
                const float esl = esl_capped(tmp, prs);
                const float qvs = (c.eps * esl) / (prs - esl);
                if (qvnew < qvs) {
                    const float rhoqr = rho * qrnew;
                    const float vent = 1.6f + 30.3922f * powf(rhoqr, 0.2046f);
                    const float deficit = 1.0f - qvnew / qvs;
                    const float num = (vent * deficit) * powf(rhoqr, 0.525f);
                    const float den = (2.03e4f + 9.584e6f / (qvs * prs)) * rho;
                    er = pymin((num / den) * dt, qrnew);
                    if (qvnew + er > qvs) er = qvs - qvnew;
                }
            }
            if (ar + cr > qcnew) {
                const float term1 = ar + cr;
                ar = (qcnew * ar) / term1;
                cr = (qcnew * cr) / term1;
            }
            qvnew = qvnew + er;
            qcnew = qcnew - (ar + cr);
            qrnew = qrnew + ((ar + cr) - er);
            if (er > 1.0e-7f) {
                if (eqtset == 2) {
                    const float cpml = (c.cp + c.cpv * qvnew) + c.cpl * (qcnew + qrnew);
                    const float cvml = (c.cv + c.cvv * qvnew) + c.cpl * (qcnew + qrnew);
                    const float rm = c.rd + c.rv * qvnew;
                    const float latent = c.lv1 - c.lv2 * tmp;
                    const float first = latent / ((c.cpdcv * cvml) * pisum);
                    const float second = ((th0 + th3d) * (c.rv / cvml)) * (1.0f - (c.rovcp * cpml) / rm);
                    th3d = th3d - er * (first - second);
                    const float base = ((rho * rm) * (th0 + th3d)) * c.rp00;
                    pp3d = powf(base, c.rddcv) - pi0;
                    pisum = pi0 + pp3d;
                    prs = c.p00 * powf(pisum, c.cpdrd);
                } else {
                    const float latent = c.lv1 - c.lv2 * tmp;
                    th3d = th3d - er * (latent / (c.cp * pisum));
                    const float den = ((c.rd * (th0 + th3d)) * pisum) * (1.0f + qvnew * c.reps);
                    rho = prs / den;
                }
            }
            terms[0] = (double)((rr * ar) * tem);
            terms[1] = (double)((rr * cr) * tem);
            terms[2] = (double)((rr * er) * tem);
        }
        // --- saturation adjustment ---
        {
            const float old_qv = qvnew, old_qc = qcnew;
            float tnew = (th0 + th3d) * (pi0 + pp3d);
            float esl = esl_capped(tnew, prs);
            float qvs = (c.eps * esl) / (prs - esl);
            uint32_t iterations = 0;
            if (eqtset == 2) {
                if (old_qc > 1.0e-12f || old_qv > qvs) {
                    const float ql = pymax(old_qc + qrnew, 0.0f);
                    const float cvml = (c.cv + c.cvv * qvnew) + c.cpl * ql;
                    const float lhv = c.lv1 - c.lv2 * tnew;
                    const float t1 = (lhv - c.rv * tnew) / cvml;
                    const float d1 = (t1 * 17.67f) * 243.5f;
                    const float converge = 2.0f * 0.0001f;
                    float tlast = tnew, pnew = prs;
                    int n = 0;
                    for (;;) {  // bounded: leaves at the 100th pass at the latest
                        n += 1;
                        const float denom = 1.0f + (d1 * qvs) / ((tnew - 29.65f) * (tnew - 29.65f));
                        float dqv = (qvs - qvnew) / denom;
                        dqv = pymin(dqv, qcnew);
                        if (qvnew + dqv < 1.0e-20f) dqv = 1.0e-20f - qvnew;
                        qvnew = qvnew + dqv;
                        qcnew = qcnew - dqv;
                        tnew = tnew - dqv * t1;
                        pnew = (rho * (c.rd + c.rv * qvnew)) * tnew;
                        const bool conv = fabsf(tnew - tlast) <= converge;
                        if (!conv) {
                            tlast = tnew;
                            esl = esl_capped(tnew, prs);
                            qvs = (c.eps * esl) / (pnew - esl);
                        }
                        if (n == 100) {
                            atomicAdd(&w.status[0], 1);
                            break;
                        }
                        if (conv) break;
                    }
                    iterations = (uint32_t)n;
                    prs = pnew;
                    pp3d = powf(pnew * c.rp00, c.rovcp) - pi0;
                    th3d = tnew / (pi0 + pp3d) - th0;
                }
            } else {
                const float lhv = c.lv1 - c.lv2 * tnew;
                const float square = (tnew - 29.65f) * (tnew - 29.65f);
                const float numerator = ((lhv * qvs) * 17.67f) * 243.5f;
                float dqv = (qvs - qvnew) / (1.0f + numerator / (c.cp * square));
                if (qvnew + dqv < 1.0e-20f) dqv = 1.0e-20f - qvnew;
                dqv = pymin(dqv, pymax(0.0f, qcnew));
                qvnew = qvnew + dqv;
                qcnew = qcnew - dqv;
                iterations = 1;
                th3d = th3d - dqv * (lhv / (c.cp * (pi0 + pp3d)));
                const float den = ((c.rd * (th0 + th3d)) * (pi0 + pp3d)) * (1.0f + qvnew * c.reps);
                rho = prs / den;
            }
            if (a.satadj_iterations != nullptr) a.satadj_iterations[p] = iterations;
            const float cond = pymax(qcnew - old_qc, 0.0f);
            const float evac = pymax(qvnew - old_qv, 0.0f);
            terms[3] = (double)((rr * cond) * tem);
            terms[4] = (double)((rr * evac) * tem);
        }
        a.th3d[p] = th3d;
        a.pp3d[p] = pp3d;
        a.prs[p] = prs;
        a.rho[p] = rho;
        a.qv[p] = qvnew;
        a.qc[p] = qcnew;
        a.qr[p] = qrnew;
    }
    const size_t slot = ((size_t)k * d.nj + j) * w.nbx + blockIdx.x;
    const size_t plane = (size_t)d.nk * d.nj * w.nbx;
#pragma unroll
    for (int t = 0; t < 5; ++t) {
        const double s = block_sum(terms[t], s_red);
        if (threadIdx.x == 0) w.partial[t * plane + slot] = s;
    }
}

// one thread per (budget type, row): row sums of the column terms in i order
__global__ void kessler_rows_kernel(KDims d, KWork w) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= 5 * d.nj) return;
    const int t = q / d.nj, j = q % d.nj;
    const size_t ncol = (size_t)d.ni * d.nj;
    double s = 0.0;
    for (int i = 0; i < d.ni; ++i) s += w.colterm[t * ncol + (size_t)j * d.ni + i];
    w.rows[(size_t)t * d.nj + j] = s;
}

// grid (nk, 5): block (k, t) sums the nj*nbx cell-kernel partials of budget
// term t at level k (strided per thread, then a fixed warp/block tree, so the
// result is the same on every run) and leaves the level total in the level's
// first slot, where the finish kernel reads it.
constexpr int kLevelThreads = 256;
__global__ void __launch_bounds__(kLevelThreads) kessler_levels_kernel(KDims d, KWork w) {
    __shared__ double s_red[kLevelThreads / 32];
    const int k = blockIdx.x, t = blockIdx.y;
    const size_t n = (size_t)d.nj * w.nbx;
    double *level = w.partial + (size_t)t * d.nk * n + (size_t)k * n;
    double s = 0.0;
    for (size_t q = threadIdx.x; q < n; q += kLevelThreads) s += level[q];
    s = block_sum(s, s_red);
    if (threadIdx.x == 0) level[0] = s;
}

// single thread: ordered finish of every budget (row sums of asq in j order,
// level totals of qbudget in k order)
__global__ void kessler_finish_kernel(gm1b_kessler_arrays a, KDims d, KWork w, double volume, double dxd,
                                      double dyd, double area) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    // Each budget accumulates in a register in the same order as a running
    // sum in memory would, and is stored once: the row and level totals are
    // then independent loads that can all be in flight together.
    const double *rows = w.rows;
    for (int s = 0; s < 3; ++s) {
        double acc = a.asq[s];
        for (int j = 0; j < d.nj; ++j) acc += rows[(size_t)s * d.nj + j] * volume;
        a.asq[s] = acc;
    }
    double q6 = a.qbudget[6], q5 = a.qbudget[5];
    for (int j = 0; j < d.nj; ++j) q6 += rows[(size_t)3 * d.nj + j] * dxd * dyd;
    for (int j = 0; j < d.nj; ++j) q5 += rows[(size_t)4 * d.nj + j] * area;
    a.qbudget[6] = q6;
    a.qbudget[5] = q5;
    const size_t n = (size_t)d.nj * w.nbx, plane = (size_t)d.nk * n;
    for (int p = 0; p < 3; ++p) {
        double acc = a.qbudget[2 + p];
        for (int k = 0; k < d.nk; ++k) acc = acc + w.partial[p * plane + (size_t)k * n] * volume;
        a.qbudget[2 + p] = acc;
    }
    for (int p = 3; p < 5; ++p) {
        double acc = a.qbudget[p - 3];
        for (int k = 0; k < d.nk; ++k) acc += w.partial[p * plane + (size_t)k * n] * volume;
        a.qbudget[p - 3] = acc;
    }
}

bool launched(const char *what) {
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

extern "C" size_t gm1b_kessler_workspace_bytes(int32_t ni, int32_t nj, int32_t nk) {
    if (ni < 1 || nj < 1 || nk < 1) return 0;
    return workspace_bytes(ni, nj, nk);
}

extern "C" int32_t gm1b_kessler_driver(int32_t ni, int32_t nj, int32_t nk, const gm1b_kessler_arrays *arrays,
                                      float dx, float dy, float dz, float dt, int32_t equation_set, int32_t efall,
                                      void *workspace, size_t workspace_size, void *stream) {
    if (arrays == nullptr || ni < 1 || nj < 1 || nk < 1) {
        gm1b_set_error("gm1b_kessler_driver: need arrays and ni, nj, nk >= 1");
        return GM1B_ERR_ARGUMENT;
    }
    if (equation_set != 1 && equation_set != 2) {
        gm1b_set_error("gm1b_kessler_driver: equation_set must be 1 or 2");
        return GM1B_ERR_ARGUMENT;
    }
    if (efall != 0) {
        gm1b_set_error("gm1b_kessler_driver: only efall=0 (no precipitation-energy fallout) is built");
        return GM1B_ERR_ARGUMENT;
    }
    if (!(dx > 0.0f) || !(dy > 0.0f) || !(dz > 0.0f) || !(dt > 0.0f) || !isfinite(dx) || !isfinite(dy) ||
        !isfinite(dz) || !isfinite(dt)) {
        gm1b_set_error("gm1b_kessler_driver: dx, dy, dz, dt must be finite and > 0");
        return GM1B_ERR_ARGUMENT;
    }
    const gm1b_kessler_arrays &a = *arrays;
    const void *required[] = {a.ruh, a.rvh, a.rmh, a.mh, a.pi0, a.th0, a.rr, a.rho, a.pp3d, a.th3d, a.prs,
                              a.qv,  a.qc,  a.qr,  a.fall_velocity, a.rain, a.prate, a.asq, a.qbudget};
    for (const void *p : required)
        if (p == nullptr) {
            gm1b_set_error("gm1b_kessler_driver: a required array is NULL");
            return GM1B_ERR_ARGUMENT;
        }
    if (workspace == nullptr || workspace_size < workspace_bytes(ni, nj, nk) ||
        (reinterpret_cast<uintptr_t>(workspace) & 15u) != 0u) {
        gm1b_set_error("gm1b_kessler_driver: workspace must be 16-byte aligned and hold %zu bytes",
                       workspace_bytes(ni, nj, nk));
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const KDims d{ni, nj, nk};
    const KWork w = carve(workspace, ni, nj, nk);
    const KConst c = make_constants();
    if (cudaMemsetAsync(w.status, 0, 16, st) != cudaSuccess) {
        gm1b_set_error("gm1b_kessler_driver: status reset failed");
        return GM1B_ERR_CUDA;
    }
    const float rdz = 1.0f / dz;
    {
        ProfScope ps("kessler_column_kernel", st);
        kessler_column_kernel<<<dim3((ni + kCX - 1) / kCX, (nj + kCY - 1) / kCY), dim3(kCX, kCY), 0, st>>>(a, d, w, c,
                                                                                                         dt, rdz);
        ps.stop();
    }
    if (!launched("kessler_column_kernel")) return GM1B_ERR_CUDA;
    {
        ProfScope ps("kessler_cell_kernel", st);
        kessler_cell_kernel<<<dim3(w.nbx, nj, nk), kKX, 0, st>>>(a, d, w, c, dt, equation_set);
        ps.stop();
    }
    if (!launched("kessler_cell_kernel")) return GM1B_ERR_CUDA;
    {
        ProfScope ps("kessler_rows_kernel", st);
        kessler_rows_kernel<<<(5 * nj + 127) / 128, 128, 0, st>>>(d, w);
        ps.stop();
    }
    if (!launched("kessler_rows_kernel")) return GM1B_ERR_CUDA;
    {
        ProfScope ps("kessler_levels_kernel", st);
        kessler_levels_kernel<<<dim3(nk, 5), kLevelThreads, 0, st>>>(d, w);
        ps.stop();
    }
    if (!launched("kessler_levels_kernel")) return GM1B_ERR_CUDA;
    const double volume = (double)((dx * dy) * dz);
    const double area = (double)(dx * dy);
    {
        ProfScope ps("kessler_finish_kernel", st);
        kessler_finish_kernel<<<1, 1, 0, st>>>(a, d, w, volume, (double)dx, (double)dy, area);
        ps.stop();
    }
    if (!launched("kessler_finish_kernel")) return GM1B_ERR_CUDA;
    return GM1B_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant.  Some callers cannot allocate device memory of
// their own: a host model that hands this library only its state arrays
// (for instance a Fortran or C model bound through this C ABI whose device
// memory belongs to another runtime's pool), or a process whose device
// memory is reserved up front by another framework's allocator.  They
// cannot supply the workspace gm1b_kessler_driver needs, so this entry point
// keeps that scratch in a file-scope device array instead.  Every GPU that
// loads the library holds the array until the process exits; every call on
// a device shares it and finds the previous call's contents there.
// ---------------------------------------------------------------------------
namespace {

static __device__ __align__(256) unsigned char g_kessler_static_scratch[GM1B_KESSLER_STATIC_SCRATCH_BYTES];

std::mutex g_static_mu;
void *g_static_ptr[64] = {};  // device address of the array, per device ordinal

// Device address of the scratch array on the current device, resolved once
// per device (host code may not use the symbol itself: on the host it names
// a stand-in, not device memory).
// The cached address stays valid for the life of the device's primary
// context; a caller that resets the device (cudaDeviceReset) must not call
// this entry point again in the same process.
void *static_scratch_address(int dev) {
    std::lock_guard<std::mutex> g(g_static_mu);
    if (g_static_ptr[dev] == nullptr) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_kessler_static_scratch) != cudaSuccess) return nullptr;
        g_static_ptr[dev] = p;
    }
    return g_static_ptr[dev];
}

}  // namespace

extern "C" int32_t gm1b_kessler_driver_static(int32_t ni, int32_t nj, int32_t nk, const gm1b_kessler_arrays *arrays,
                                             float dx, float dy, float dz, float dt, int32_t equation_set,
                                             int32_t efall, int32_t *status_out, void *stream) {
    if (ni < 1 || nj < 1 || nk < 1) {
        gm1b_set_error("gm1b_kessler_driver_static: need ni, nj, nk >= 1");
        return GM1B_ERR_ARGUMENT;
    }
    const size_t need = workspace_bytes(ni, nj, nk);
    if (need > (size_t)GM1B_KESSLER_STATIC_SCRATCH_BYTES) {
        gm1b_set_error("gm1b_kessler_driver_static: a %dx%dx%d grid needs %zu bytes of scratch, more than the %u-byte "
                       "static array; use gm1b_kessler_driver with a caller workspace",
                       ni, nj, nk, need, (unsigned)GM1B_KESSLER_STATIC_SCRATCH_BYTES);
        return GM1B_ERR_ARGUMENT;
    }
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        gm1b_set_error("gm1b_kessler_driver_static: no current CUDA device");
        return GM1B_ERR_CUDA;
    }
    if (dev < 0 || dev >= 64) {
        gm1b_set_error("gm1b_kessler_driver_static: device ordinal %d is beyond the 64 devices this entry point "
                       "serves; use gm1b_kessler_driver with a caller workspace", dev);
        return GM1B_ERR_ARGUMENT;
    }
    void *scratch = static_scratch_address(dev);
    if (scratch == nullptr) {
        cudaGetLastError();
        gm1b_set_error("gm1b_kessler_driver_static: cudaGetSymbolAddress of the static scratch failed");
        return GM1B_ERR_CUDA;
    }
    // gm1b_kessler_driver clears the status words and overwrites every
    // partial sum it reads, so leftover contents of a previous call are inert.
    const int32_t rc = gm1b_kessler_driver(ni, nj, nk, arrays, dx, dy, dz, dt, equation_set, efall, scratch,
                                           (size_t)GM1B_KESSLER_STATIC_SCRATCH_BYTES, stream);
    if (rc != GM1B_OK) return rc;
    if (status_out != nullptr) {
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (cudaMemcpyAsync(status_out, scratch, 2 * sizeof(int32_t), cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
            cudaGetLastError();
            gm1b_set_error("gm1b_kessler_driver_static: status copy failed");
            return GM1B_ERR_CUDA;
        }
    }
    return GM1B_OK;
}

// ---------------------------------------------------------------------------
// once-per-large-step Kessler transition (cpu_gm1_kessler_large_step_inplace,
// src/cm1core/cuda_gm1_kessler_large_step.py:183-292): with equation set 2
// the previous held rates are removed from pp3d/th3d/qv/qc and each carrier
// takes the pre-physics state (solve2.F:1561-1579); the pre-physics pressure
// and moist density follow (solve2.F:1582-1595), rr takes the density, the
// driver runs, and the carriers become the next step's held rates
// (solve3.F:319-337).  Two elementwise launches around the driver.
// ---------------------------------------------------------------------------
namespace gm1b {
namespace {

struct KesslerEos {
    float cpdrd, p00, rd, rv;
};

__global__ void __launch_bounds__(256) kessler_pre_physics_kernel(gm1b_kessler_arrays a, gm1b_kessler_held h,
                                                                  size_t n, float dt, int eqt2, KesslerEos c) {
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        float pp = a.pp3d[q], th = a.th3d[q], qv = a.qv[q];
        if (eqt2) {
            float *state[4] = {&pp, &th, &qv, nullptr};
            float *rate[4] = {h.qpten, h.qtten, h.qvten, h.qcten};
            float qc = a.qc[q];
            state[3] = &qc;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const float w = rate[s][q] * dt;
                *state[s] = *state[s] - w;
                rate[s][q] = *state[s];
            }
            a.pp3d[q] = pp;
            a.th3d[q] = th;
            a.qv[q] = qv;
            a.qc[q] = qc;
        }
        const float pi = a.pi0[q] + pp;
        float prs = powf(pi, c.cpdrd);
        prs = prs * c.p00;
        float rho = a.th0[q] + th;
        rho = rho * pi;
        float w = fmaxf(qv, 0.0f);
        w = w * c.rv;
        w = w + c.rd;
        rho = rho * w;
        rho = prs / rho;
        a.prs[q] = prs;
        a.rho[q] = rho;
        const_cast<float *>(a.rr)[q] = rho;
    }
}

__global__ void __launch_bounds__(256) kessler_recapture_kernel(gm1b_kessler_arrays a, gm1b_kessler_held h, size_t n,
                                                                float dt) {
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        h.qpten[q] = (a.pp3d[q] - h.qpten[q]) / dt;
        h.qtten[q] = (a.th3d[q] - h.qtten[q]) / dt;
        h.qvten[q] = (a.qv[q] - h.qvten[q]) / dt;
        h.qcten[q] = (a.qc[q] - h.qcten[q]) / dt;
    }
}

}  // namespace
}  // namespace gm1b

// ---------------------------------------------------------------------------
// final-RK dry-air mass correction, apmasscon = 1 (cpu_initial_dry_mass and
// cpu_apmasscon_inplace, src/cm1core/cuda_apmasscon.py:190-325; CM1
// init3d.F:2483-2527, solve2.F:1616-1656 and :1972-2030): per level the dry
// mass ((rho*ruh)*rvh)*rmh and the Exner words pi0 + pp3d summed in binary64,
// the levels summed in order, the uniform Exner correction
// ((mass1/mass2)^rddcv - 1) * sum(pi) / cells in binary64 and rounded to
// binary32, then pp3d += correction and prs, rho rebuilt from the equation
// of state.  The level sums are formed in a fixed order: 16 CTAs per level
// (each thread a strided binary64 partial, then a shared-memory tree per
// CTA, as the reference's one-CTA-per-level CUDA reduction does per block),
// the level adding its 16 partials in order; the twin sums each level
// serially, so the two ledgers agree to binary64 rounding.
// ---------------------------------------------------------------------------
namespace gm1b {
namespace {

struct MassArgs {
    const float *ruh, *rvh, *rmh, *pi0, *th0, *th3d, *qv;
    float *pp3d, *prs, *rho, *rr;
    int ni, nj, nk;
    // the ledger's cells: columns i0..i1-1 of rows j0..j1-1 (the whole plane
    // unless a decomposed run sums its interior only)
    int i0, i1, j0, j1;
};

constexpr int kMassThreads = 256;
constexpr int kMassChunks = 16;  // CTAs per level: chunk c sums cells ij = c*256 + t + m*16*256

// grid (nk, kMassChunks): each CTA a fixed share of one level, its binary64
// partial sums at partials[(k * kMassChunks + c)] (dry) and at the same
// index + nk * kMassChunks (Exner)
__global__ void __launch_bounds__(kMassThreads) apmasscon_levels_kernel(MassArgs a, double *partials, int pressure) {
    __shared__ double s_dry[kMassThreads], s_pi[kMassThreads];
    const int k = blockIdx.x, c = blockIdx.y;
    const int wi = a.i1 - a.i0;
    const size_t nw = (size_t)wi * (a.j1 - a.j0), base = (size_t)k * a.ni * a.nj;
    double dry = 0.0, pis = 0.0;
    for (size_t ij = (size_t)c * kMassThreads + threadIdx.x; ij < nw; ij += (size_t)kMassChunks * kMassThreads) {
        const int i = a.i0 + (int)(ij % wi), j = a.j0 + (int)(ij / wi);
        const size_t q = base + (size_t)j * a.ni + i;
        float term = a.rho[q] * __ldg(a.ruh + i);
        term = term * __ldg(a.rvh + j);
        term = term * __ldg(a.rmh + q);
        dry += (double)term;
        if (pressure) pis += (double)(__ldg(a.pi0 + q) + a.pp3d[q]);
    }
    s_dry[threadIdx.x] = dry;
    s_pi[threadIdx.x] = pis;
    __syncthreads();
    for (int stride = kMassThreads / 2; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride) {
            s_dry[threadIdx.x] += s_dry[threadIdx.x + stride];
            s_pi[threadIdx.x] += s_pi[threadIdx.x + stride];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partials[(size_t)k * kMassChunks + c] = s_dry[0];
        partials[(size_t)(a.nk + k) * kMassChunks + c] = s_pi[0];
    }
}

// the level sums: each level's chunk partials added in chunk order
__device__ __forceinline__ double level_sum(const double *partials, int row) {
    double v = 0.0;
    for (int c = 0; c < kMassChunks; ++c) v += partials[(size_t)row * kMassChunks + c];
    return v;
}

// the dry-mass ledger (levels in order) into mass[0]; with only_if_unset a
// non-zero mass[0] (a ledger already held, e.g. restored) is kept
__global__ void dry_mass_finish_kernel(const double *layers, int nk, double *mass, int only_if_unset) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    if (only_if_unset && mass[0] != 0.0) return;
    double total = 0.0;
    for (int k = 0; k < nk; ++k) total += level_sum(layers, k);
    mass[0] = total;
}

// diag: mass2, the Exner sum, the binary64 correction, mass1
__global__ void apmasscon_finish_kernel(const double *layers, int nk, const double *mass1, double cells, float rddcv,
                                        float *correction, double *diag) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double mass2 = 0.0, pis = 0.0;
    for (int k = 0; k < nk; ++k) {
        mass2 += level_sum(layers, k);
        pis += level_sum(layers, nk + k);
    }
    double value = pow(mass1[0] / mass2, (double)rddcv) - 1.0;
    value = value * pis;
    value = value / cells;
    correction[0] = (float)value;
    if (diag != nullptr) {
        diag[0] = mass2;
        diag[1] = pis;
        diag[2] = value;
        diag[3] = mass1[0];
    }
}

__global__ void __launch_bounds__(256) apmasscon_apply_kernel(MassArgs a, const float *correction, size_t n,
                                                              KesslerEos c) {
    const float corr = correction[0];
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const float pp = a.pp3d[q] + corr;
        const float pi = __ldg(a.pi0 + q) + pp;
        const float prs = c.p00 * powf(pi, c.cpdrd);
        const float theta = __ldg(a.th0 + q) + __ldg(a.th3d + q);
        const float vapor = fmaxf(0.0f, __ldg(a.qv + q));
        const float gas = c.rd + vapor * c.rv;
        float den = theta * pi;
        den = den * gas;
        const float rho = prs / den;
        a.pp3d[q] = pp;
        a.prs[q] = prs;
        a.rho[q] = rho;
        if (a.rr != nullptr) a.rr[q] = rho;
    }
}

KesslerEos mass_eos() {
    const float cp = 1005.7f, rd = 287.04f;
    return KesslerEos{(float)((double)cp / (double)rd), 100000.0f, rd, 461.5f};
}

float mass_rddcv() {
    const float cp = 1005.7f, rd = 287.04f;
    const float cv = cp - rd;
    return rd / cv;
}

size_t mass_workspace_bytes(int nk) { return sizeof(double) * (2 * (size_t)nk * kMassChunks + 2); }

int32_t mass_partials(const MassArgs &m, double *partials, int pressure, cudaStream_t st) {
    ProfScope ps("apmasscon_levels_kernel", st);
    apmasscon_levels_kernel<<<dim3(m.nk, kMassChunks), kMassThreads, 0, st>>>(m, partials, pressure);
    ps.stop();
    return launched("apmasscon_levels_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

// the correction from level partials already formed (and, in a decomposed
// run, added over the subdomains), then the EOS rebuild of every cell
int32_t mass_apply(const MassArgs &m, const double *partials, const double *mass1, double cells, double *diag,
                   void *workspace, cudaStream_t st) {
    double *layers = static_cast<double *>(workspace);
    float *corr = reinterpret_cast<float *>(layers + 2 * (size_t)m.nk * kMassChunks);
    const size_t n = (size_t)m.ni * m.nj * m.nk;
    apmasscon_finish_kernel<<<1, 1, 0, st>>>(partials, m.nk, mass1, cells, mass_rddcv(), corr, diag);
    if (!launched("apmasscon_finish_kernel")) return GM1B_ERR_CUDA;
    const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)148 * 8);
    {
        ProfScope ps("apmasscon_apply_kernel", st);
        apmasscon_apply_kernel<<<grid, 256, 0, st>>>(m, corr, n, mass_eos());
        ps.stop();
    }
    return launched("apmasscon_apply_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

int32_t mass_correction(const MassArgs &m, const double *mass1, double *diag, void *workspace, cudaStream_t st) {
    double *layers = static_cast<double *>(workspace);
    const int32_t rc = mass_partials(m, layers, 1, st);
    if (rc != GM1B_OK) return rc;
    return mass_apply(m, layers, mass1, (double)((size_t)m.ni * m.nj * m.nk), diag, workspace, st);
}

bool mass_grid_ok(const char *who, int32_t ni, int32_t nj, int32_t nk) {
    if (ni < 1 || nj < 1 || nk < 1 || nk > 65535) {
        gm1b_set_error("%s: need ni, nj >= 1 and 1 <= nk <= 65535", who);
        return false;
    }
    return true;
}

}  // namespace
}  // namespace gm1b

extern "C" size_t gm1b_apmasscon_workspace_bytes(int32_t nk) { return nk < 1 ? 0 : mass_workspace_bytes(nk); }

extern "C" int32_t gm1b_dry_mass(int32_t ni, int32_t nj, int32_t nk, const float *rho, const float *ruh,
                                 const float *rvh, const float *rmh, double *mass, int32_t only_if_unset,
                                 void *workspace, void *stream) {
    if (!mass_grid_ok("gm1b_dry_mass", ni, nj, nk)) return GM1B_ERR_ARGUMENT;
    if (rho == nullptr || ruh == nullptr || rvh == nullptr || rmh == nullptr || mass == nullptr ||
        workspace == nullptr) {
        gm1b_set_error("gm1b_dry_mass: rho, ruh, rvh, rmh, mass and the workspace are required");
        return GM1B_ERR_ARGUMENT;
    }
    MassArgs m{ruh, rvh, rmh, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, const_cast<float *>(rho), nullptr,
               ni, nj, nk, 0, ni, 0, nj};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double *layers = static_cast<double *>(workspace);
    apmasscon_levels_kernel<<<dim3(nk, kMassChunks), kMassThreads, 0, st>>>(m, layers, 0);
    if (!launched("apmasscon_levels_kernel")) return GM1B_ERR_CUDA;
    dry_mass_finish_kernel<<<1, 1, 0, st>>>(layers, nk, mass, only_if_unset ? 1 : 0);
    return launched("dry_mass_finish_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_apmasscon(int32_t ni, int32_t nj, int32_t nk, const gm1b_apmasscon_arrays *arrays,
                                  const double *mass1, double *diagnostics, void *workspace, void *stream) {
    if (!mass_grid_ok("gm1b_apmasscon", ni, nj, nk)) return GM1B_ERR_ARGUMENT;
    if (arrays == nullptr || mass1 == nullptr || workspace == nullptr) {
        gm1b_set_error("gm1b_apmasscon: arrays, mass1 and the workspace are required");
        return GM1B_ERR_ARGUMENT;
    }
    const gm1b_apmasscon_arrays &a = *arrays;
    const void *need[] = {a.ruh, a.rvh, a.rmh, a.pi0, a.th0, a.th3d, a.qv, a.pp3d, a.prs, a.rho};
    for (const void *q : need)
        if (q == nullptr) {
            gm1b_set_error("gm1b_apmasscon: a required array is NULL");
            return GM1B_ERR_ARGUMENT;
        }
    const MassArgs m{a.ruh, a.rvh, a.rmh, a.pi0, a.th0, a.th3d, a.qv, a.pp3d, a.prs, a.rho, nullptr, ni, nj, nk,
                     0, ni, 0, nj};
    return mass_correction(m, mass1, diagnostics, workspace, static_cast<cudaStream_t>(stream));
}

namespace {
// phase 0: the whole transition; with the dry-mass correction split for a
// decomposed run, phase 1 (held removal, pre-physics EOS, the level partials
// of the window into partials) and phase 2 (the correction from partials
// already added over the subdomains, for `cells` cells, then the driver and
// the recapture)
int32_t kessler_large_step(int32_t ni, int32_t nj, int32_t nk, const gm1b_kessler_arrays *arrays,
                           const gm1b_kessler_held *held, float dx, float dy, float dz, float dt, int32_t equation_set,
                           int32_t efall, void *workspace, size_t workspace_size, const double *mass1,
                           double *mass_diagnostics, void *mass_workspace, void *stream, int phase = 0,
                           const int32_t *window = nullptr, double *partials = nullptr, double cells = 0.0) {
    if (arrays == nullptr || ni < 1 || nj < 1 || nk < 2) {
        gm1b_set_error("gm1b_kessler_large_step: need arrays, ni >= 1, nj >= 1, nk >= 2");
        return GM1B_ERR_ARGUMENT;
    }
    const bool eqt2 = equation_set == 2;
    if (eqt2 && (held == nullptr || held->qpten == nullptr || held->qtten == nullptr || held->qvten == nullptr ||
                 held->qcten == nullptr)) {
        gm1b_set_error("gm1b_kessler_large_step: equation set 2 needs the four held-rate carriers");
        return GM1B_ERR_ARGUMENT;
    }
    if (!(dt > 0.0f) || !isfinite(dt)) {
        gm1b_set_error("gm1b_kessler_large_step: dt must be finite and > 0");
        return GM1B_ERR_ARGUMENT;
    }
    const gm1b_kessler_held none{nullptr, nullptr, nullptr, nullptr};
    const gm1b_kessler_held h = eqt2 ? *held : none;
    const size_t n = (size_t)ni * nj * nk;
    // CM1 constants.F: cpdrd = cp / rd of the default-real operands
    const float cp = 1005.7f, rd = 287.04f;
    const KesslerEos c{(float)((double)cp / (double)rd), 100000.0f, rd, 461.5f};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)148 * 8);
    const gm1b_kessler_arrays &k = *arrays;
    MassArgs m{k.ruh, k.rvh, k.rmh, k.pi0, k.th0, k.th3d, k.qv, k.pp3d, k.prs, k.rho,
               const_cast<float *>(k.rr), ni, nj, nk, 0, ni, 0, nj};
    if (phase != 2) {
        {
            ProfScope ps("kessler_pre_physics_kernel", st);
            kessler_pre_physics_kernel<<<grid, 256, 0, st>>>(*arrays, h, n, dt, eqt2 ? 1 : 0, c);
            ps.stop();
        }
        if (!launched("kessler_pre_physics_kernel")) return GM1B_ERR_CUDA;
        if (phase == 1) {  // the window's level partials of the dry-mass ledger
            m.i0 = window[0], m.i1 = window[1], m.j0 = window[2], m.j1 = window[3];
            return mass_partials(m, partials, 1, st);
        }
        if (mass1 != nullptr) {  // apmasscon between the pre-physics EOS and the driver
            const int32_t mrc = mass_correction(m, mass1, mass_diagnostics, mass_workspace, st);
            if (mrc != GM1B_OK) return mrc;
        }
    } else {
        const int32_t mrc = mass_apply(m, partials, mass1, cells, mass_diagnostics, mass_workspace, st);
        if (mrc != GM1B_OK) return mrc;
    }
    const int32_t rc = gm1b_kessler_driver(ni, nj, nk, arrays, dx, dy, dz, dt, equation_set, efall, workspace,
                                           workspace_size, stream);
    if (rc != GM1B_OK || !eqt2) return rc;
    {
        ProfScope ps("kessler_recapture_kernel", st);
        kessler_recapture_kernel<<<grid, 256, 0, st>>>(*arrays, h, n, dt);
        ps.stop();
    }
    return launched("kessler_recapture_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}
}  // namespace

extern "C" int32_t gm1b_kessler_large_step(int32_t ni, int32_t nj, int32_t nk, const gm1b_kessler_arrays *arrays,
                                           const gm1b_kessler_held *held, float dx, float dy, float dz, float dt,
                                           int32_t equation_set, int32_t efall, void *workspace,
                                           size_t workspace_size, void *stream) {
    return kessler_large_step(ni, nj, nk, arrays, held, dx, dy, dz, dt, equation_set, efall, workspace,
                              workspace_size, nullptr, nullptr, nullptr, stream);
}

extern "C" int32_t gm1b_kessler_large_step_apmasscon(int32_t ni, int32_t nj, int32_t nk,
                                                     const gm1b_kessler_arrays *arrays, const gm1b_kessler_held *held,
                                                     float dx, float dy, float dz, float dt, int32_t equation_set,
                                                     int32_t efall, void *workspace, size_t workspace_size,
                                                     const double *mass1, double *mass_diagnostics,
                                                     void *mass_workspace, void *stream) {
    if (mass1 == nullptr || mass_workspace == nullptr || arrays == nullptr || arrays->ruh == nullptr ||
        arrays->rvh == nullptr || arrays->rmh == nullptr) {
        gm1b_set_error("gm1b_kessler_large_step_apmasscon: mass1, the mass workspace and ruh, rvh, rmh are required");
        return GM1B_ERR_ARGUMENT;
    }
    if (nk > 65535) {
        gm1b_set_error("gm1b_kessler_large_step_apmasscon: nk <= 65535");
        return GM1B_ERR_ARGUMENT;
    }
    return kessler_large_step(ni, nj, nk, arrays, held, dx, dy, dz, dt, equation_set, efall, workspace,
                              workspace_size, mass1, mass_diagnostics, mass_workspace, stream);
}

extern "C" size_t gm1b_apmasscon_partials_words(int32_t nk) { return nk < 1 ? 0 : 2 * (size_t)nk * kMassChunks; }

namespace {
bool window_ok(const char *who, int32_t ni, int32_t nj, const int32_t *w) {
    if (w == nullptr || w[0] < 0 || w[1] > ni || w[0] >= w[1] || w[2] < 0 || w[3] > nj || w[2] >= w[3]) {
        gm1b_set_error("%s: the window (i0, i1, j0, j1) must be a non-empty part of the %dx%d plane", who, ni, nj);
        return false;
    }
    return true;
}
}  // namespace

extern "C" int32_t gm1b_apmasscon_partials(int32_t ni, int32_t nj, int32_t nk, const float *rho, const float *ruh,
                                           const float *rvh, const float *rmh, const float *pi0, const float *pp3d,
                                           const int32_t *window, int32_t pressure, double *partials, void *stream) {
    if (!mass_grid_ok("gm1b_apmasscon_partials", ni, nj, nk) || !window_ok("gm1b_apmasscon_partials", ni, nj, window))
        return GM1B_ERR_ARGUMENT;
    if (rho == nullptr || ruh == nullptr || rvh == nullptr || rmh == nullptr || partials == nullptr ||
        (pressure && (pi0 == nullptr || pp3d == nullptr))) {
        gm1b_set_error("gm1b_apmasscon_partials: rho, ruh, rvh, rmh, partials (and pi0, pp3d for the Exner sum) "
                       "are required");
        return GM1B_ERR_ARGUMENT;
    }
    const MassArgs m{ruh, rvh, rmh, pi0, nullptr, nullptr, nullptr, const_cast<float *>(pp3d), nullptr,
                     const_cast<float *>(rho), nullptr, ni, nj, nk, window[0], window[1], window[2], window[3]};
    return mass_partials(m, partials, pressure ? 1 : 0, static_cast<cudaStream_t>(stream));
}

extern "C" int32_t gm1b_dry_mass_from_partials(int32_t nk, const double *partials, double *mass, int32_t only_if_unset,
                                               void *stream) {
    if (nk < 1 || partials == nullptr || mass == nullptr) {
        gm1b_set_error("gm1b_dry_mass_from_partials: need nk >= 1, partials and mass");
        return GM1B_ERR_ARGUMENT;
    }
    dry_mass_finish_kernel<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(partials, nk, mass, only_if_unset ? 1 : 0);
    return launched("dry_mass_finish_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

extern "C" int32_t gm1b_kessler_large_step_apmasscon_begin(int32_t ni, int32_t nj, int32_t nk,
                                                           const gm1b_kessler_arrays *arrays,
                                                           const gm1b_kessler_held *held, float dt,
                                                           int32_t equation_set, const int32_t *window,
                                                           double *partials, void *stream) {
    const char *who = "gm1b_kessler_large_step_apmasscon_begin";
    if (arrays == nullptr || arrays->ruh == nullptr || arrays->rvh == nullptr || arrays->rmh == nullptr ||
        partials == nullptr || !mass_grid_ok(who, ni, nj, nk) || !window_ok(who, ni, nj, window)) {
        if (arrays == nullptr || partials == nullptr) gm1b_set_error("%s: arrays and partials are required", who);
        return GM1B_ERR_ARGUMENT;
    }
    return kessler_large_step(ni, nj, nk, arrays, held, 1.0f, 1.0f, 1.0f, dt, equation_set, 0, nullptr, 0, nullptr,
                              nullptr, nullptr, stream, 1, window, partials, 0.0);
}

extern "C" int32_t gm1b_kessler_large_step_apmasscon_end(int32_t ni, int32_t nj, int32_t nk,
                                                         const gm1b_kessler_arrays *arrays,
                                                         const gm1b_kessler_held *held, float dx, float dy, float dz,
                                                         float dt, int32_t equation_set, int32_t efall,
                                                         void *workspace, size_t workspace_size,
                                                         const double *partials, double cells, const double *mass1,
                                                         double *mass_diagnostics, void *mass_workspace,
                                                         void *stream) {
    if (partials == nullptr || mass1 == nullptr || mass_workspace == nullptr || !(cells > 0.0)) {
        gm1b_set_error("gm1b_kessler_large_step_apmasscon_end: partials, mass1, the mass workspace and cells > 0 "
                       "are required");
        return GM1B_ERR_ARGUMENT;
    }
    return kessler_large_step(ni, nj, nk, arrays, held, dx, dy, dz, dt, equation_set, efall, workspace,
                              workspace_size, mass1, mass_diagnostics, mass_workspace, stream, 2, nullptr,
                              const_cast<double *>(partials), cells);
}
