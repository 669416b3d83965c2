// moist_large_step.cu - the composed moist RK3 large step behind one C entry
// point (gm1b_moist_large_step): the operators of this library enqueued in
// the reference's large-step schedule (StepPhase / large_step_schedule,
// src/cm1core/gm1_runtime.py:611-627, :1969-2007), the phase bindings of the
// Cartesian runtime (CartesianDynamics, src/cm1core/cuda_cartesian_dynamics.py:
// 1014-1317; CartesianClosure, src/cm1core/cuda_cartesian_closure.py:1118-1200,
// :1635-1685; the Kessler transition, src/cm1core/cuda_gm1_kessler_large_step.py:183;
// solve3, src/cm1core/cuda_cartesian_finish.py:739).
//
// The same launches in the same order as the package's Python composition
// (gm1_b200.moist_step.MoistLargeStep), so the two give the same words; the
// uniform column runs the terrain operator family on flat metrics, a
// stretched column the flat (terrain_flag=.false.) family.  Each RK stage's
// theta and moisture advection, momentum/pressure boundaries and TKE stage
// touch disjoint fields and run on side streams when the step is concurrent
// (forked from and joined back to the caller's stream with events, so a
// captured step keeps the dependencies).  Nothing is allocated and nothing
// synchronises inside a step.
#include <algorithm>
#include <cstring>
#include <vector>

#include "gm1b_common.cuh"

namespace gm1b {
namespace {

// copy of a (nz, ny, nx) box between two arrays of different row and level
// strides (compact <-> padded sub-box): one warp per row, rows grid-strided
constexpr int kCopyRows = 8;  // rows (warps) per CTA
__global__ void __launch_bounds__(32 * kCopyRows)
    box_copy_kernel(float *__restrict__ dst, size_t dst_sy, size_t dst_sz, const float *__restrict__ src,
                    size_t src_sy, size_t src_sz, int nx, int ny, int nz) {
    const size_t rows = (size_t)ny * nz;
    for (size_t r = (size_t)blockIdx.x * kCopyRows + threadIdx.y; r < rows; r += (size_t)gridDim.x * kCopyRows) {
        const size_t j = r % ny, k = r / ny;
        float *d = dst + k * dst_sz + j * dst_sy;
        const float *s = src + k * src_sz + j * src_sy;
        for (int i = threadIdx.x; i < nx; i += 32) d[i] = s[i];
    }
}

__global__ void add_inplace_kernel(float *__restrict__ acc, const float *__restrict__ x, size_t n) {
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        acc[q] = acc[q] + x[q];
}

bool ok(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return true;
    cudaGetLastError();
    gm1b_set_error("gm1b_moist_large_step: %s: %s", what, cudaGetErrorString(e));
    return false;
}

}  // namespace
}  // namespace gm1b

using namespace gm1b;

struct gm1b_moist_step {
    gm1b_moist_step_config c{};
    gm1b_moist_state s{};
    gm1b_moist_metrics m{};
    int device = 0;
    cudaStream_t side[6] = {};
    cudaEvent_t ev[16] = {};
    void *kessler_ws = nullptr;
    size_t kessler_ws_bytes = 0;
    void *mass_ws = nullptr;  // the dry-mass correction's level sums
    float *stress_buf = nullptr;     // the SGS stress scratch (strains, stresses, held tendencies)
    float *turbs_work = nullptr;     // the scalar turbulence's workspace
    gm1b_flat_stress_arrays stress{};
    int32_t *status_acc = nullptr;  // 8 words
    float *courant = nullptr;       // 1 word
    uint32_t *courant_keys = nullptr;
    float *ones_i = nullptr, *ones_j = nullptr, *mh_col = nullptr;
    float rdz = 0.0f;
    uint32_t obc = 0;
};

namespace {

using Step = gm1b_moist_step;
constexpr int kNumq = 3;

int box_copy(float *dst, size_t dst_sy, size_t dst_sz, const float *src, size_t src_sy, size_t src_sz, int nx, int ny,
             int nz, cudaStream_t st) {
    const size_t rows = (size_t)ny * nz, want = (rows + kCopyRows - 1) / kCopyRows, cap = (size_t)148 * 32;
    ProfScope ps("box_copy_kernel", st);
    box_copy_kernel<<<(unsigned)(want < cap ? want : cap), dim3(32, kCopyRows), 0, st>>>(dst, dst_sy, dst_sz, src,
                                                                                         src_sy, src_sz, nx, ny, nz);
    ps.stop();
    return ok(cudaPeekAtLastError(), "box_copy_kernel") ? GM1B_OK : GM1B_ERR_CUDA;
}

// compact copies of the interior winds (the closure's u/v/w inputs)
int compact_winds(Step &h, cudaStream_t st) {
    const gm1b_moist_state &s = h.s;
    const int ni = h.c.ni, nj = h.c.nj, nk = h.c.nk;
    const size_t uy = ni + 7, uz = (size_t)(nj + 6) * uy;
    const size_t vy = ni + 6, vz = (size_t)(nj + 7) * vy;
    const size_t wy = ni + 6, wz = (size_t)(nj + 6) * wy;
    int r = box_copy(s.uc, ni + 1, (size_t)nj * (ni + 1), s.u3d + uz + 3 * uy + 3, uy, uz, ni + 1, nj, nk, st);
    if (r == GM1B_OK)
        r = box_copy(s.vc, ni, (size_t)(nj + 1) * ni, s.v3d + vz + 3 * vy + 3, vy, vz, ni, nj + 1, nk, st);
    if (r == GM1B_OK) r = box_copy(s.wc, ni, (size_t)nj * ni, s.w3d + wz + 3 * wy + 3, wy, wz, ni, nj, nk + 1, st);
    return r;
}

// pp3d interior <-> the compact pp3d_c
int pp3d_compact(Step &h, bool to_compact, cudaStream_t st) {
    const int ni = h.c.ni, nj = h.c.nj, nk = h.c.nk;
    const size_t py = ni + 2, pz = (size_t)(nj + 2) * py;
    float *interior = h.s.pp3d + pz + py + 1;
    if (to_compact) return box_copy(h.s.pp3d_c, ni, (size_t)nj * ni, interior, py, pz, ni, nj, nk, st);
    return box_copy(interior, py, pz, h.s.pp3d_c, ni, (size_t)nj * ni, ni, nj, nk, st);
}

int zero(void *p, size_t bytes, cudaStream_t st, const char *what) {
    return ok(cudaMemsetAsync(p, 0, bytes, st), what) ? GM1B_OK : GM1B_ERR_CUDA;
}

int copy(void *dst, const void *src, size_t bytes, cudaStream_t st, const char *what) {
    return ok(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st), what) ? GM1B_OK : GM1B_ERR_CUDA;
}

// sizes in words
struct Sizes {
    size_t mass, face, u, v, w, scalar, pr;
    explicit Sizes(const gm1b_moist_step_config &c) {
        const size_t ni = c.ni, nj = c.nj, nk = c.nk;
        mass = nk * nj * ni;
        face = (nk + 1) * nj * ni;
        u = (nk + 2) * (nj + 6) * (ni + 7);
        v = (nk + 2) * (nj + 7) * (ni + 6);
        w = (nk + 3) * (nj + 6) * (ni + 6);
        scalar = (nk + 2) * (nj + 6) * (ni + 6);
        pr = (nk + 2) * (nj + 2) * (ni + 2);
    }
};

#define TRY(x)                      \
    do {                            \
        const int r_ = (x);         \
        if (r_ != GM1B_OK) return r_; \
    } while (0)

gm1b_momentum_column flat_column(const Step &h) {
    gm1b_momentum_column col{};
    col.flat = 1;
    col.rho0_padded = h.m.rho0_padded;
    col.mh = h.m.mh_profile;
    col.mf = h.m.mf_profile;
    col.rr0 = h.m.rr0;
    col.rdz = h.rdz;
    return col;
}

gm1b_vertical_column flat_vertical(const Step &h) {
    gm1b_vertical_column col{};
    col.flat = 1;
    col.mh = h.m.mh_profile;
    col.rdz = h.rdz;
    return col;
}

gm1b_tke_evolution_arrays tke_arrays(const Step &h) {
    const gm1b_moist_state &s = h.s;
    const gm1b_moist_metrics &m = h.m;
    gm1b_tke_evolution_arrays a{};
    a.tkea = s.tkea;
    a.tke3d = s.tke3d;
    a.tketen = s.tketen;
    a.kmh = s.kmh;
    a.kmv = s.kmv;
    a.rho = s.rho;
    a.rf = s.rf;
    a.mh = m.mh;
    a.mf = m.mf;
    a.gz = m.gz;
    a.rgz = m.rgz;
    a.rgzu = m.rgzu;
    a.rgzv = m.rgzv;
    a.c1 = m.c1;
    a.c2 = m.c2;
    a.rrf0 = m.rrf0;
    a.rru = s.rru;
    a.rrv = s.rrv;
    a.rrw = s.rrw;
    a.divx = s.divx;
    return a;
}

int fold(Step &h, const int32_t *kessler_status, const float *courant, cudaStream_t st) {
    return gm1b_step_status_fold(kessler_status, courant, h.status_acc, st);
}

int fold_courant(Step &h, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    // dtdx = (0.5*dt)*f32(1/dx) in binary32, as storm_diagnostics.py:278-280
    const float half_dt = 0.5f * c.dt;
    const float dtdx = half_dt * (float)(1.0 / (double)c.dx);
    const float dtdy = half_dt * (float)(1.0 / (double)c.dy);
    const float dtdz = half_dt * (float)(1.0 / (double)c.dz);
    TRY(gm1b_courant_max(c.ni, c.nj, c.nk, h.s.uc, h.s.vc, h.s.wc, h.ones_i, h.ones_j, h.mh_col, dtdx, dtdy, dtdz,
                         h.courant_keys, h.courant, st));
    return fold(h, nullptr, h.courant, st);
}

// ---- phases (cf. MoistLargeStep) ------------------------------------------
int closure(Step &h, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    const gm1b_moist_state &s = h.s;
    const gm1b_moist_metrics &m = h.m;
    TRY(compact_winds(h, st));
    TRY(pp3d_compact(h, true, st));
    TRY(fold_courant(h, st));
    gm1b_moist_nm_arrays nm{m.c1, m.c2, m.mf, s.pi0, s.th0, s.prs, s.pp3d_c, s.th3d, s.q3d,
                            s.nm, s.temperature, s.qt, s.thv_c, s.qvci, s.saturation_mask, nullptr};
    TRY(gm1b_moist_nm(c.ni, c.nj, c.nk, &nm, c.dz, st));
    if (c.stretched) {
        gm1b_flat_deformation_arrays d{s.uc, s.vc, s.wc, s.rho, s.rf, m.mf, m.c1, m.c2, m.mh_profile, s.defv, s.defh};
        TRY(gm1b_flat_deformation(c.ni, c.nj, c.nk, &d, c.dx, c.dy, h.rdz, st));
    } else {
        gm1b_deformation_arrays d{s.uc,  s.vc,  s.wc,   s.rho,  s.rf, m.c1, m.c2,   m.gz,
                                  m.rgz, m.rgzu, m.rgzv, m.gx, m.gy, s.defv, s.defh};
        TRY(gm1b_terrain_deformation(c.ni, c.nj, c.nk, &d, c.dx, c.dy, c.dz, st));
    }
    gm1b_sgs_tke_arrays g{s.ruh, s.rvh, m.rmf, s.nm, s.defv, s.defh, s.tkea, s.tk, s.grdscl, s.rgrdscl, s.lenscl,
                          s.dissten, s.cme, s.ce1, s.ce2, s.csm, s.kmh, s.kmv, s.khh, s.khv, s.tketen, nullptr};
    TRY(gm1b_sgs_tke(c.ni, c.nj, c.nk, &g, c.dx, c.dy, c.dz, st));
    TRY(copy(s.tke3d, s.tkea, Sizes(c).face * sizeof(float), st, "tke3d <- tkea"));
    gm1b_tke_evolution_arrays t = tke_arrays(h);
    if (c.stretched)
        TRY(gm1b_tke_diffusion_flat(c.ni, c.nj, c.nk, &t, c.dx, c.dy, h.rdz, c.dt, st));
    else
        TRY(gm1b_tke_diffusion(c.ni, c.nj, c.nk, &t, c.dx, c.dy, c.dz, c.dt, st));
    if (!c.sgs_diffusion && !c.rayleigh) return GM1B_OK;
    // the held momentum tendencies: zeroed, then the SGS stress added (the
    // Rayleigh damping joins them in the held phase)
    const Sizes z(c);
    TRY(zero(h.stress.uten, (size_t)c.nk * c.nj * (c.ni + 1) * sizeof(float), st, "zero held u"));
    TRY(zero(h.stress.vten, (size_t)c.nk * (c.nj + 1) * c.ni * sizeof(float), st, "zero held v"));
    TRY(zero(h.stress.wten, z.face * sizeof(float), st, "zero held w"));
    if (!c.sgs_diffusion) return GM1B_OK;
    if (c.stretched) return gm1b_flat_sgs_stress(c.ni, c.nj, c.nk, &h.stress, c.dx, c.dy, h.rdz, c.dt, st);
    // the uniform column: the terrain texts on its flat metrics
    const gm1b_flat_stress_arrays &f = h.stress;
    const gm1b_terrain_stress_arrays ta{f.u3d, f.v3d, f.w3d, f.rho, f.rf,  f.mh,  f.mf,  f.kmh, f.kmv, m.gz,
                                        m.rgz, m.gzu, m.rgzu, m.gzv, m.rgzv, m.gx, m.gy, m.gxu, m.gyv, f.s11,
                                        f.s22, f.s33, f.s12, f.s13, f.s23, f.t11, f.t22, f.t33, f.t12, f.t13,
                                        f.t23, f.uten, f.vten, f.wten};
    return gm1b_terrain_sgs_stress(c.ni, c.nj, c.nk, &ta, c.dx, c.dy, c.dz, c.dt, st);
}

// the held momentum into the physical cells of the zeroed stage tendencies
// (pack_cartesian_held_momentum, cuda_cartesian_dynamics.py:206)
int seed_held_momentum(Step &h, cudaStream_t st) {
    const gm1b_moist_state &s = h.s;
    const int ni = h.c.ni, nj = h.c.nj, nk = h.c.nk;
    const size_t uy = ni + 7, uz = (size_t)(nj + 6) * uy;
    const size_t vy = ni + 6, vz = (size_t)(nj + 7) * vy;
    const size_t wy = ni + 6, wz = (size_t)(nj + 6) * wy;
    TRY(box_copy(s.uten + uz + 3 * uy + 3, uy, uz, h.stress.uten, ni + 1, (size_t)nj * (ni + 1), ni + 1, nj, nk, st));
    TRY(box_copy(s.vten + vz + 3 * vy + 3, vy, vz, h.stress.vten, ni, (size_t)(nj + 1) * ni, ni, nj + 1, nk, st));
    return box_copy(s.wten + wz + 3 * wy + 3, wy, wz, h.stress.wten, ni, (size_t)nj * ni, ni, nj, nk + 1, st);
}

int held_tendencies(Step &h, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    const gm1b_moist_state &s = h.s;
    const Sizes z(c);
    TRY(zero(s.thheld, z.mass * sizeof(float), st, "zero thheld"));
    TRY(zero(s.qheld, kNumq * z.mass * sizeof(float), st, "zero qheld"));
    if (c.rayleigh) {
        // the damping added into the held momentum (uten1 + uten) and
        // assigned to the held theta before the scalar diffusion adds to it
        const gm1b_moist_metrics &m = h.m;
        const gm1b_rayleigh_held_arrays ra{m.tauh, m.taus, m.tauf, m.u0, m.v0, s.uc, s.vc, s.wc, s.tha,
                                           h.stress.uten, h.stress.vten, h.stress.wten, s.thheld};
        TRY(gm1b_rayleigh_held(c.ni, c.nj, c.nk, &ra, 1, 1, c.rdalpha, st));
    }
    if (c.dissipative_heating) {
        // idiss after the damping and before the subgrid turbulence
        // (solve1.F:917-975)
        const gm1b_dissipative_heating_arrays da{s.dissten, s.pi0, s.pp3d_c, s.qa, s.thheld};
        TRY(gm1b_dissipative_heating(c.ni, c.nj, c.nk, &da, st));
    }
    if (c.sgs_diffusion) {
        // turbs for theta and the moisture rows into the held thten1/qten the
        // eqtset 2 composition then reads (solve1.F:1169-1233)
        const gm1b_moist_metrics &m = h.m;
        if (c.stretched) {
            const gm1b_flat_scalar_turbulence_arrays ta{s.th0, s.tha, s.qa, s.rho, s.rr, s.rf, m.mh, m.mf,
                                                        s.khh, s.khv, s.thheld, s.qheld, h.turbs_work};
            TRY(gm1b_flat_scalar_turbulence(c.ni, c.nj, c.nk, kNumq, &ta, c.dx, c.dy, c.dz, c.dt, st));
        } else {
            const gm1b_terrain_scalar_turbulence_arrays ta{
                s.th0, s.tha, s.qa,   s.rho,  s.rr, s.rf,  m.mh, m.mf,     s.khh, s.khv, m.gz,
                m.rgz, m.rgzu, m.rgzv, m.gx, m.gxu, m.gy, m.gyv, s.thheld, s.qheld, h.turbs_work};
            TRY(gm1b_terrain_scalar_turbulence(c.ni, c.nj, c.nk, kNumq, &ta, c.dx, c.dy, c.dz, c.dt, st));
        }
    }
    gm1b_held_arrays a{s.th0_3d, s.pi0_3d, s.rho, s.pp3d_c, s.tha, s.qa, s.qpten, s.qtten, s.qvten, s.qcten,
                       s.thheld, s.qheld, s.ppten};
    return gm1b_held_compose(c.ni, c.nj, c.nk, &a, c.dt, st);
}

gm1b_momentum5_arrays momentum_arrays(const Step &h) {
    const gm1b_moist_state &s = h.s;
    const gm1b_moist_metrics &m = h.m;
    gm1b_momentum5_arrays a{};
    a.u3d = s.u3d;
    a.uten = s.uten;
    a.rru = s.rru;
    a.v3d = s.v3d;
    a.vten = s.vten;
    a.rrv = s.rrv;
    a.w3d = s.w3d;
    a.wten = s.wten;
    a.rrw = s.rrw;
    a.uh = s.uh;
    a.vh = s.vh;
    a.rho0_3d = m.rho0_3d;
    a.rf0 = m.rf0;
    a.rrf0 = m.rrf0;
    a.c2 = m.c2;
    a.gz = m.gz;
    a.gzu = m.gzu;
    a.gzv = m.gzv;
    a.rgzu = m.rgzu;
    a.rgzv = m.rgzv;
    a.dzdx = m.dzdx;
    a.dzdy = m.dzdy;
    a.divx = s.divx;
    return a;
}

int pre_acoustic(Step &h, int nrk, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    const gm1b_moist_state &s = h.s;
    const gm1b_moist_metrics &m = h.m;
    const Sizes z(c);
    gm1b_eqtset2_arrays e{s.th0, s.qv0, s.pi0, nullptr, nullptr, s.th3d, s.q3d, s.pp3d,
                          s.thv, s.ppterm, s.dum8, s.thterm, s.piadv};
    TRY(gm1b_eqtset2_stage_terms(c.ni, c.nj, c.nk, &e, 0, st));
    TRY(gm1b_open_fill(c.ni, c.nj, c.nk, 0, s.thv, st));   // pressure
    TRY(gm1b_open_fill(c.ni, c.nj, c.nk, 1, s.dum8, st));  // scalar
    TRY(zero(s.uten, z.u * sizeof(float), st, "zero uten"));
    TRY(zero(s.vten, z.v * sizeof(float), st, "zero vten"));
    TRY(zero(s.wten, z.w * sizeof(float), st, "zero wten"));
    if (c.sgs_diffusion || c.rayleigh) TRY(seed_held_momentum(h, st));
    gm1b_momentum5_arrays a = momentum_arrays(h);
    if (c.stretched) {
        // solve2.F:484-487 (bcwsfc, bc2d of w(1)) and :575 (bcw(rrw,0)) are
        // terrain_flag statements: a flat column runs neither
        const gm1b_momentum_column col = flat_column(h);
        TRY(gm1b_momentum_advection5_column(c.ni, c.nj, c.nk, &a, h.obc, c.dx, c.dy, &col, st));
        return gm1b_moist_buoyancy_flat(c.ni, c.nj, c.nk, s.dum8, m.c1, m.c2, s.wten, st);
    }
    if (nrk >= 2) {
        TRY(gm1b_bcwsfc(c.ni, c.nj, c.nk, s.u3d, s.v3d, s.w3d, m.gz, m.dzdx, m.dzdy, st));
        TRY(gm1b_w_level1_fill(c.ni, c.nj, c.nk, s.w3d, st));
    }
    TRY(gm1b_momentum_mass_flux5(c.ni, c.nj, c.nk, &a, h.obc, c.dx, c.dy, c.dz, st));
    TRY(gm1b_open_fill(c.ni, c.nj, c.nk, 5, s.rrw, st));  // w, ends kept
    TRY(gm1b_momentum_transport5(c.ni, c.nj, c.nk, &a, h.obc, c.dx, c.dy, c.dz, st));
    return gm1b_moist_buoyancy(c.ni, c.nj, c.nk, s.dum8, m.c1, m.c2, m.gxu, m.gyv, s.uten, s.vten, s.wten, st);
}

int acoustic(Step &h, int nrk, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    const gm1b_moist_state &s = h.s;
    const gm1b_moist_metrics &m = h.m;
    gm1b_terrain_open_arrays a{s.ppi,    s.pp3d,   s.ppx,    s.ppd,    s.piadv,  s.ppterm,   s.ppten,  s.thv,
                               s.qk,     s.pk1,    s.pk2,    s.mm,     s.fpk,    s.divh,     s.hadvp,  s.dum3,
                               s.elim_c, s.elim_d, s.tri_aa, s.tri_bb, s.tri_cc, s.tri_dd,   s.tri_pivot,
                               s.tri_residual,
                               s.ua,     s.u3d,    s.uten,   s.rru,    s.va,     s.v3d,      s.vten,   s.rrv,
                               s.wa,     s.w3d,    s.wten,   s.rrw,    s.radbcw, s.radbce,   s.radbcs, s.radbcn,
                               s.uh,     s.vh,     s.ruf,    s.rvf,    s.scalar};
    gm1b_terrain_metrics tm{m.rho0_3d, m.rr0, m.rf0, m.rrf0, m.c1, m.c2, m.gz, m.rgzu, m.rgzv, m.dzdx, m.dzdy,
                            m.gx, m.gxu, m.gy, m.gyv};
    const uint32_t stage_without_fills = GM1B_TOS_ALL & ~GM1B_TOS_STAGE_FILLS;
    if (c.stretched) {
        const gm1b_momentum_column col = flat_column(h);
        return gm1b_terrain_open_stage_column(c.ni, c.nj, c.nk, nrk, c.dt, c.nsound, c.dx, c.dy, c.alph, c.kdiv,
                                              stage_without_fills, 0, h.obc, &a, &tm, &col, st);
    }
    return gm1b_terrain_open_stage(c.ni, c.nj, c.nk, nrk, c.dt, c.nsound, c.dx, c.dy, (double)c.dz, c.alph, c.kdiv,
                                   stage_without_fills, 0, &a, &tm, st);
}

int post_acoustic(Step &h, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    const gm1b_moist_state &s = h.s;
    const gm1b_moist_metrics &m = h.m;
    gm1b_post_acoustic_arrays a{s.rru, s.rrv, s.rrw, m.rgzu, m.rgzv, m.dzdx, m.dzdy, m.gz, m.rho0_3d, m.rf0,
                                s.thterm, s.divergence, s.theta_div, s.divx};
    if (c.stretched) {
        const gm1b_momentum_column col = flat_column(h);
        return gm1b_post_acoustic_flux_column(c.ni, c.nj, c.nk, &a, c.dx, c.dy, &col, st);
    }
    return gm1b_post_acoustic_flux(c.ni, c.nj, c.nk, &a, c.dx, c.dy, c.dz, st);
}

// the weps words of the WENO weights (binary64 of binary32 products)
double weps_of(float mag) { return (double)(mag * 1.0e-18f); }

int advect(Step &h, float *padded, float *tendency, double weps, int nrk, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    const gm1b_moist_state &s = h.s;
    const gm1b_moist_metrics &m = h.m;
    gm1b_scalar_advection5_arrays a{padded, s.rru, s.rrv, s.rrw, m.c1, m.c2, m.rr0, m.gz, s.divx,
                                    tendency, nullptr, nullptr, nullptr};
    if (c.stretched) {
        const gm1b_vertical_column col = flat_vertical(h);
        return gm1b_scalar_advection5_column(c.ni, c.nj, c.nk, &a, nrk, 1, c.dx, c.dy, weps, h.obc, 0, &col, st);
    }
    return gm1b_scalar_advection5(c.ni, c.nj, c.nk, &a, nrk, 1, c.dx, c.dy, c.dz, weps, h.obc, 0, st);
}

int theta_advection(Step &h, int nrk, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    const gm1b_moist_state &s = h.s;
    TRY(gm1b_theta_transport_pack(c.ni, c.nj, c.nk, s.th0, s.th3d, s.theta_padded, st));
    TRY(gm1b_open_fill(c.ni, c.nj, c.nk, 1, s.theta_padded, st));
    TRY(zero(s.theta_adv, Sizes(c).mass * sizeof(float), st, "zero theta_adv"));
    return advect(h, s.theta_padded, s.theta_adv, weps_of(10.0f), nrk, st);
}

struct Species {
    float *padded, *fx, *fy, *fz, *advx, *advy, *advz, *candidate;
};

Species species(const Step &h, int r) {
    const gm1b_moist_state &s = h.s;
    if (r == 1)
        return {s.moisture_padded_1, s.fx_1, s.fy_1, s.fz_1, s.advx_1, s.advy_1, s.advz_1, s.candidate_1};
    if (r == 2)
        return {s.moisture_padded_2, s.fx_2, s.fy_2, s.fz_2, s.advx_2, s.advy_2, s.advz_2, s.candidate_2};
    return {s.moisture_padded, s.fx, s.fy, s.fz, s.advx, s.advy, s.advz, s.candidate};
}

int species_advection(Step &h, int r, int nrk, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    const gm1b_moist_state &s = h.s;
    const gm1b_moist_metrics &m = h.m;
    const Sizes z(c);
    const Species sp = species(h, r);
    float *q = s.q3d + (size_t)r * z.mass;
    float *adv = s.moist_adv + (size_t)r * z.mass;
    TRY(gm1b_pack_scalar(c.ni, c.nj, c.nk, q, sp.padded, st));
    TRY(gm1b_open_fill(c.ni, c.nj, c.nk, 1, sp.padded, st));
    TRY(zero(adv, z.mass * sizeof(float), st, "zero moist_adv"));
    const double weps = weps_of(1.0e-2f);
    if (nrk < 3) return advect(h, sp.padded, adv, weps, nrk, st);
    gm1b_pdef_chain_arrays a{s.qa + (size_t)r * z.mass, sp.padded, m.rho0_3d, m.gz, m.rgz, m.rr0, m.c1, m.c2,
                             s.divx, s.rru, s.rrv, s.rrw, sp.fx, sp.fy, sp.fz, sp.advx, sp.advy, sp.advz,
                             sp.candidate, adv};
    const float dttmp = c.dt / (float)(4 - nrk);
    if (c.stretched) {
        const gm1b_vertical_column col = flat_vertical(h);
        return gm1b_pdef_moisture_chain_column(c.ni, c.nj, c.nk, &a, dttmp, c.dx, c.dy, weps, h.obc, r == 0 ? 0 : 1,
                                               &col, st);
    }
    return gm1b_pdef_moisture_chain(c.ni, c.nj, c.nk, &a, dttmp, c.dx, c.dy, c.dz, weps, h.obc, r == 0 ? 0 : 1, st);
}

int record_wait(cudaEvent_t ev, cudaStream_t from, cudaStream_t to) {
    if (!ok(cudaEventRecord(ev, from), "cudaEventRecord")) return GM1B_ERR_CUDA;
    return ok(cudaStreamWaitEvent(to, ev, 0), "cudaStreamWaitEvent") ? GM1B_OK : GM1B_ERR_CUDA;
}

int scalar_moist(Step &h, int nrk, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    const gm1b_moist_state &s = h.s;
    if (c.concurrent) {
        // fork the theta and species lanes from st, join them back
        TRY(ok(cudaEventRecord(h.ev[0], st), "cudaEventRecord") ? GM1B_OK : GM1B_ERR_CUDA);
        for (int q = 0; q < 1 + kNumq; ++q)
            TRY(ok(cudaStreamWaitEvent(h.side[q], h.ev[0], 0), "cudaStreamWaitEvent") ? GM1B_OK : GM1B_ERR_CUDA);
        TRY(theta_advection(h, nrk, h.side[0]));
        for (int r = 0; r < kNumq; ++r) TRY(species_advection(h, r, nrk, h.side[1 + r]));
        for (int q = 0; q < 1 + kNumq; ++q) TRY(record_wait(h.ev[1 + q], h.side[q], st));
    } else {
        TRY(theta_advection(h, nrk, st));
        for (int r = 0; r < kNumq; ++r) TRY(species_advection(h, r, nrk, st));
    }
    const Sizes z(c);
    gm1b_scalar_rk_compose_arrays a{s.tha, s.thheld, s.theta_div, s.theta_adv, s.th3d,
                                    s.qa,  s.qheld,  s.moist_adv, s.q3d};
    return gm1b_scalar_moist_rk_compose(z.mass, kNumq, &a, nrk, c.dt, st);
}

int momentum_boundaries(Step &h, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    const gm1b_moist_state &s = h.s;
    const gm1b_moist_metrics &m = h.m;
    TRY(gm1b_open_fill(c.ni, c.nj, c.nk, 2, s.u3d, st));
    TRY(gm1b_open_fill(c.ni, c.nj, c.nk, 3, s.v3d, st));
    TRY(gm1b_open_fill(c.ni, c.nj, c.nk, 4, s.w3d, st));
    if (c.stretched) return GM1B_OK;  // solve2.F:1676: bcwsfc is a terrain_flag statement
    return gm1b_bcwsfc(c.ni, c.nj, c.nk, s.u3d, s.v3d, s.w3d, m.gz, m.dzdx, m.dzdy, st);
}

int scalar_boundaries(Step &h, cudaStream_t st) { return gm1b_open_fill(h.c.ni, h.c.nj, h.c.nk, 0, h.s.pp3d, st); }

int tke_rk(Step &h, int nrk, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    const gm1b_moist_state &s = h.s;
    gm1b_tke_evolution_arrays t = tke_arrays(h);
    if (c.stretched)
        TRY(gm1b_tke_rk_stage_flat(c.ni, c.nj, c.nk, &t, h.m.mf_profile, s.tke3d, s.tke_workspace, nrk, c.dx, c.dy,
                                   h.rdz, c.dt, st));
    else
        TRY(gm1b_tke_rk_stage(c.ni, c.nj, c.nk, &t, s.tke3d, s.tke_workspace, nrk, c.dx, c.dy, c.dz, c.dt, st));
    return copy(s.tke3d, s.tke_workspace, Sizes(c).face * sizeof(float), st, "tke3d <- stage");
}

// the stage tail: scalar/moisture on st (forking its own lanes), momentum
// and pressure boundaries on one side stream, TKE on another, joined
int stage_tail(Step &h, int nrk, cudaStream_t st) {
    if (!h.c.concurrent) {
        TRY(scalar_moist(h, nrk, st));
        TRY(momentum_boundaries(h, st));
        if (nrk < 3) TRY(scalar_boundaries(h, st));
        return tke_rk(h, nrk, st);
    }
    cudaStream_t bnd = h.side[1 + kNumq], tke = h.side[2 + kNumq];
    TRY(ok(cudaEventRecord(h.ev[8], st), "cudaEventRecord") ? GM1B_OK : GM1B_ERR_CUDA);
    TRY(ok(cudaStreamWaitEvent(bnd, h.ev[8], 0), "cudaStreamWaitEvent") ? GM1B_OK : GM1B_ERR_CUDA);
    TRY(ok(cudaStreamWaitEvent(tke, h.ev[8], 0), "cudaStreamWaitEvent") ? GM1B_OK : GM1B_ERR_CUDA);
    TRY(scalar_moist(h, nrk, st));
    TRY(momentum_boundaries(h, bnd));
    if (nrk < 3) TRY(scalar_boundaries(h, bnd));
    TRY(tke_rk(h, nrk, tke));
    TRY(record_wait(h.ev[9], bnd, st));
    return record_wait(h.ev[10], tke, st);
}

int microphysics(Step &h, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    const gm1b_moist_state &s = h.s;
    const gm1b_moist_metrics &m = h.m;
    const Sizes z(c);
    TRY(pp3d_compact(h, true, st));
    gm1b_kessler_arrays k{};
    k.ruh = s.ruh;
    k.rvh = s.rvh;
    k.rmh = m.rmh;
    k.mh = m.mh;
    k.pi0 = s.pi0_3d;
    k.th0 = s.th0_3d;
    k.rr = s.kessler_rr;
    k.rho = s.rho;
    k.pp3d = s.pp3d_c;
    k.th3d = s.th3d;
    k.prs = s.prs;
    k.qv = s.q3d;
    k.qc = s.q3d + z.mass;
    k.qr = s.q3d + 2 * z.mass;
    k.fall_velocity = s.fall_velocity;
    k.rain = s.rain;
    k.prate = s.prate;
    k.asq = s.asq;
    k.qbudget = s.qbudget;
    gm1b_kessler_held held{s.qpten, s.qtten, s.qvten, s.qcten};
    if (c.apmasscon)
        TRY(gm1b_kessler_large_step_apmasscon(c.ni, c.nj, c.nk, &k, &held, c.dx, c.dy, c.dz, c.dt, 2, 0,
                                              h.kessler_ws, h.kessler_ws_bytes, s.mass1, nullptr, h.mass_ws, st));
    else
        TRY(gm1b_kessler_large_step(c.ni, c.nj, c.nk, &k, &held, c.dx, c.dy, c.dz, c.dt, 2, 0, h.kessler_ws,
                                    h.kessler_ws_bytes, st));
    TRY(fold(h, static_cast<const int32_t *>(h.kessler_ws), nullptr, st));
    return pp3d_compact(h, false, st);
}

int solve3(Step &h, cudaStream_t st) {
    const gm1b_moist_step_config &c = h.c;
    const gm1b_moist_state &s = h.s;
    const gm1b_moist_metrics &m = h.m;
    const Sizes z(c);
    {
        ProfScope ps("add_inplace_kernel", st);
        add_inplace_kernel<<<(unsigned)std::min<size_t>((z.pr + 255) / 256, 4096), 256, 0, st>>>(s.ppx, s.pp3d, z.pr);
        ps.stop();
        if (!ok(cudaPeekAtLastError(), "add_inplace_kernel")) return GM1B_ERR_CUDA;
    }
    const struct {
        float *dst;
        const float *src;
        size_t words;
    } promote[7] = {{s.ua, s.u3d, z.u},     {s.va, s.v3d, z.v},          {s.wa, s.w3d, z.w},
                    {s.ppi, s.pp3d, z.pr},  {s.tha, s.th3d, z.mass},     {s.qa, s.q3d, 6 * z.mass},
                    {s.tkea, s.tke3d, z.face}};
    for (const auto &p : promote) TRY(copy(p.dst, p.src, p.words * sizeof(float), st, "carrier promotion"));
    return gm1b_solve3_density(c.ni, c.nj, c.nk, s.rho, m.c1, m.c2, s.rr, s.rf, st);
}

void release(Step *h) {
    for (auto &q : h->side)
        if (q) cudaStreamDestroy(q);
    for (auto &e : h->ev)
        if (e) cudaEventDestroy(e);
    void *bufs[] = {h->kessler_ws, h->status_acc, h->courant, h->courant_keys, h->ones_i, h->ones_j, h->mh_col,
                    h->mass_ws, h->stress_buf, h->turbs_work};
    for (void *b : bufs)
        if (b) cudaFree(b);
    delete h;
}

}  // namespace

extern "C" int32_t gm1b_moist_step_create(const gm1b_moist_step_config *config, const gm1b_moist_state *state,
                                          const gm1b_moist_metrics *metrics, gm1b_moist_step **out) {
    if (config == nullptr || state == nullptr || metrics == nullptr || out == nullptr) {
        gm1b_set_error("gm1b_moist_step_create: NULL argument");
        return GM1B_ERR_ARGUMENT;
    }
    *out = nullptr;
    const gm1b_moist_step_config &c = *config;
    if (c.ni < 8 || c.nj < 8 || c.nk < 8) {
        gm1b_set_error("gm1b_moist_step_create: need ni, nj, nk >= 8");
        return GM1B_ERR_ARGUMENT;
    }
    const float v[5] = {c.dx, c.dy, c.dz, c.dt, 1.0f};
    for (float x : v)
        if (!(x > 0.0f) || !isfinite(x)) {
            gm1b_set_error("gm1b_moist_step_create: dx, dy, dz, dt must be finite and > 0");
            return GM1B_ERR_ARGUMENT;
        }
    for (int q = 0; q < 4; ++q)
        if (c.lateral_sides[q] < 1 || c.lateral_sides[q] > 15) {
            gm1b_set_error("gm1b_moist_step_create: lateral side codes must be 1..15");
            return GM1B_ERR_ARGUMENT;
        }
    const void *const *sp = reinterpret_cast<const void *const *>(state);
    for (size_t q = 0; q < sizeof(gm1b_moist_state) / sizeof(void *); ++q)
        if (sp[q] == nullptr) {
            gm1b_set_error("gm1b_moist_step_create: state array #%zu is NULL", q);
            return GM1B_ERR_ARGUMENT;
        }
    const void *const *mp = reinterpret_cast<const void *const *>(metrics);
    const size_t all = sizeof(gm1b_moist_metrics) / sizeof(void *);
    for (size_t q = 0; q < all; ++q)
        if (mp[q] == nullptr && (q < 25 || (q < 28 && c.stretched) || (q >= 28 && c.rayleigh))) {
            gm1b_set_error("gm1b_moist_step_create: metric #%zu is NULL%s", q,
                           q >= 28   ? " (the Rayleigh damping needs u0, v0, tauh, taus and tauf)"
                           : q >= 25 ? " (a stretched column needs mh_profile, mf_profile and rho0_padded)"
                                     : "");
            return GM1B_ERR_ARGUMENT;
        }
    if (c.rayleigh && (!(c.rdalpha >= 0.0f) || !isfinite(c.rdalpha))) {
        gm1b_set_error("gm1b_moist_step_create: the Rayleigh damping needs a finite rdalpha >= 0");
        return GM1B_ERR_ARGUMENT;
    }
    if (c.sgs_diffusion && c.nk > 200) {
        gm1b_set_error("gm1b_moist_step_create: the SGS diffusion's column solves take nk <= 200");
        return GM1B_ERR_ARGUMENT;
    }
    Step *h = new Step;
    h->c = c;
    h->s = *state;
    h->m = *metrics;
    h->obc = (uint32_t)c.lateral_sides[0] | ((uint32_t)c.lateral_sides[1] << 4) |
             ((uint32_t)c.lateral_sides[2] << 8) | ((uint32_t)c.lateral_sides[3] << 12);
    h->rdz = 1.0f / c.dz;
    bool good = ok(cudaGetDevice(&h->device), "cudaGetDevice");
    for (auto &q : h->side)
        if (good) good = ok(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
    for (auto &e : h->ev)
        if (good) good = ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreateWithFlags");
    h->kessler_ws_bytes = gm1b_kessler_workspace_bytes(c.ni, c.nj, c.nk);
    if (good) good = ok(cudaMalloc(&h->kessler_ws, h->kessler_ws_bytes), "cudaMalloc (Kessler workspace)");
    if (good) good = ok(cudaMalloc(&h->status_acc, 8 * sizeof(int32_t)), "cudaMalloc (status)");
    if (good) good = ok(cudaMalloc(&h->courant, sizeof(float)), "cudaMalloc (courant)");
    if (good) good = ok(cudaMalloc(&h->courant_keys, (size_t)c.nk * sizeof(uint32_t)), "cudaMalloc (courant keys)");
    if (good) good = ok(cudaMalloc(&h->ones_i, (size_t)c.ni * sizeof(float)), "cudaMalloc");
    if (good) good = ok(cudaMalloc(&h->ones_j, (size_t)c.nj * sizeof(float)), "cudaMalloc");
    if (good) good = ok(cudaMalloc(&h->mh_col, (size_t)c.nk * sizeof(float)), "cudaMalloc");
    if (good && c.apmasscon)
        good = ok(cudaMalloc(&h->mass_ws, gm1b_apmasscon_workspace_bytes(c.nk)), "cudaMalloc (mass workspace)");
    if (good && c.sgs_diffusion)
        good = ok(cudaMalloc(&h->turbs_work,
                             (size_t)(c.stretched ? gm1b_flat_scalar_turbulence_workspace_words(c.ni, c.nj, c.nk, kNumq)
                                                  : gm1b_terrain_scalar_turbulence_workspace_words(c.ni, c.nj, c.nk, kNumq)) *
                                 sizeof(float)),
                  "cudaMalloc (scalar turbulence workspace)");
    if (good && (c.sgs_diffusion || c.rayleigh)) {
        // strains and stresses, then the held u, v, w (the layouts of
        // gm1b_flat_stress_arrays), carved from one allocation
        const size_t ni = c.ni, nj = c.nj, nk = c.nk;
        const size_t cell = nk * nj * ni, corner = nk * (nj + 1) * (ni + 1), s13 = (nk + 1) * nj * (ni + 1),
                     s23 = (nk + 1) * (nj + 1) * ni, heldu = nk * nj * (ni + 1), heldv = nk * (nj + 1) * ni,
                     heldw = (nk + 1) * nj * ni;
        const size_t words[15] = {cell, cell, cell, corner, s13, s23, cell, cell, cell, corner, s13, s23,
                                  heldu, heldv, heldw};
        size_t total = 0;
        for (size_t w : words) total += (w + 31) / 32 * 32;  // 128-byte aligned pieces
        good = ok(cudaMalloc(&h->stress_buf, total * sizeof(float)), "cudaMalloc (SGS stress scratch)") &&
               ok(cudaMemset(h->stress_buf, 0, total * sizeof(float)), "SGS stress scratch");
        if (good) {
            float *piece[15];
            float *p = h->stress_buf;
            for (int q = 0; q < 15; ++q) {
                piece[q] = p;
                p += (words[q] + 31) / 32 * 32;
            }
            gm1b_flat_stress_arrays &a = h->stress;
            a.u3d = state->uc;
            a.v3d = state->vc;
            a.w3d = state->wc;
            a.rho = state->rho;
            a.rf = state->rf;
            a.mh = metrics->mh;
            a.mf = metrics->mf;
            a.mh_profile = metrics->mh_profile;
            a.kmh = state->kmh;
            a.kmv = state->kmv;
            float **dst[15] = {&a.s11, &a.s22, &a.s33, &a.s12, &a.s13, &a.s23, &a.t11, &a.t22,
                               &a.t33, &a.t12, &a.t13, &a.t23, &a.uten, &a.vten, &a.wten};
            for (int q = 0; q < 15; ++q) *dst[q] = piece[q];
        }
    }
    if (good) {
        // uh = vh = 1 (uniform horizontal grid) and the mh column (the first
        // column of the 3-D mh), the Courant reduction's metric inputs
        std::vector<float> ones((size_t)std::max(c.ni, c.nj), 1.0f);
        good = ok(cudaMemcpy(h->ones_i, ones.data(), (size_t)c.ni * sizeof(float), cudaMemcpyHostToDevice), "ones") &&
               ok(cudaMemcpy(h->ones_j, ones.data(), (size_t)c.nj * sizeof(float), cudaMemcpyHostToDevice), "ones") &&
               ok(cudaMemcpy2D(h->mh_col, sizeof(float), metrics->mh, (size_t)c.nj * c.ni * sizeof(float),
                               sizeof(float), (size_t)c.nk, cudaMemcpyDeviceToDevice),
                  "mh column") &&
               ok(cudaMemset(h->status_acc, 0, 8 * sizeof(int32_t)), "status") &&
               ok(cudaMemset(h->kessler_ws, 0, h->kessler_ws_bytes), "Kessler workspace") &&
               ok(cudaDeviceSynchronize(), "set-up");
    }
    if (good && c.apmasscon) {
        // init3d.F:2483-2527: the initial dry-air mass of the state, unless it
        // carries one already
        good = gm1b_dry_mass(c.ni, c.nj, c.nk, state->rho, state->ruh, state->rvh, metrics->rmh, state->mass1, 1,
                             h->mass_ws, nullptr) == GM1B_OK &&
               ok(cudaDeviceSynchronize(), "dry-mass ledger");
    }
    if (!good) {
        release(h);
        return GM1B_ERR_CUDA;
    }
    *out = h;
    return GM1B_OK;
}

extern "C" int32_t gm1b_moist_large_step(gm1b_moist_step *step, void *stream) {
    if (step == nullptr) {
        gm1b_set_error("gm1b_moist_large_step: NULL step");
        return GM1B_ERR_ARGUMENT;
    }
    Step &h = *step;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    TRY(closure(h, st));
    TRY(held_tendencies(h, st));
    for (int nrk = 1; nrk <= 3; ++nrk) {
        TRY(pre_acoustic(h, nrk, st));
        TRY(acoustic(h, nrk, st));
        TRY(post_acoustic(h, st));
        TRY(stage_tail(h, nrk, st));
    }
    TRY(microphysics(h, st));
    return solve3(h, st);
}

extern "C" int32_t gm1b_moist_step_status(gm1b_moist_step *step, int32_t *out, int32_t reset, void *stream) {
    if (step == nullptr || out == nullptr) {
        gm1b_set_error("gm1b_moist_step_status: NULL argument");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!ok(cudaMemcpyAsync(out, step->status_acc, 8 * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "status read") ||
        !ok(cudaStreamSynchronize(st), "status read"))
        return GM1B_ERR_CUDA;
    if (reset && !ok(cudaMemsetAsync(step->status_acc, 0, 8 * sizeof(int32_t), st), "status reset"))
        return GM1B_ERR_CUDA;
    if (out[0] != 0 || out[2] != 0) return GM1B_STATUS_SATADJ;
    float courant;
    memcpy(&courant, &out[3], sizeof(float));
    if (out[4] != 0 && (!isfinite(courant) || courant >= 1.5f)) return GM1B_STATUS_COURANT;
    return GM1B_OK;
}

extern "C" int32_t gm1b_moist_step_destroy(gm1b_moist_step *step) {
    if (step == nullptr) return GM1B_OK;
    cudaSetDevice(step->device);
    cudaDeviceSynchronize();
    release(step);
    return GM1B_OK;
}
