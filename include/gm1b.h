/*
 * gm1b.h - C ABI of the B200 (sm_100a) dynamical-core library libgm1b.so.
 *
 * Every entry point takes plain device pointers, sizes and scalars, enqueues
 * its kernels on the given CUDA stream (a cudaStream_t passed as void*, NULL
 * for the legacy default stream), returns without synchronising, and reports
 * argument errors through its int32_t return value (GM1B_OK on success).
 * The message of the last failure on the calling thread is available from
 * gm1b_last_error().
 *
 * Arrays are float32, C order (z, y, x), with the padded shapes and names of
 * the reference operator API:
 *
 *   scalar  (nk+2, nj+2, ni+2)   u (nk+2, nj+2, ni+1)
 *   v       (nk+2, nj+1, ni+2)   w (nk+2, nj,   ni  )
 *   dtu0    (nj+2, ni+1)         dtv0 (nj+1, ni+2)
 *   uf, uh  (ni+2)               vf, vh (nj+2)
 *
 * (src/cm1core/cuda_sound3_periodic.py:449-491,
 *  src/cm1core/cuda_psolver3_trajectory.py:93-126).
 * The caller owns every array; the library allocates no device memory in
 * these entry points.
 */
#ifndef GM1B_H
#define GM1B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GM1B_ABI_VERSION 1

#if defined(__GNUC__)
#define GM1B_API __attribute__((visibility("default")))
#else
#define GM1B_API
#endif

/* Return codes: 0 ok, negative = argument or launch error. */
#define GM1B_OK 0
#define GM1B_ERR_ARGUMENT (-1)
#define GM1B_ERR_SCHEDULE (-2)
#define GM1B_ERR_CUDA (-3)

/* flags for the acoustic stage and the trajectory */
/* Write the reference-semantics acoustic scratch outputs of the last small
 * step (fpk, divh, hadvp, elim_c, elim_d, tri_aa, tri_bb, tri_cc, tri_dd,
 * tri_pivot, tri_residual).  Without it those arrays are scratch. */
#define GM1B_FLAG_SCRATCH_OUTPUTS 1u
/* Without scratch outputs, each acoustic stage normally runs as one
 * persistent cooperative kernel (all small steps, one bounded grid barrier
 * per small step) when its row tiles are co-resident and nk <= 44; that
 * kernel uses tri_aa/tri_bb as a double buffer of ppd and tri_residual
 * words 0-2 as its barrier counter and status (word 2 nonzero = a grid
 * barrier gave up and the stage was abandoned).  This flag forces the
 * multi-launch stage (two kernels per small step) instead; both produce the
 * same words in every non-scratch array. */
#define GM1B_FLAG_MULTI_LAUNCH_STAGE 2u

/* ablation bits of the dry trajectory
 * (src/cm1core/cuda_psolver3_trajectory.py:429-436 TrajectoryAblations);
 * a set bit DISABLES the term. */
#define GM1B_ABLATE_MOMENTUM_ADVECTION 1u
#define GM1B_ABLATE_SCALAR_ADVECTION 2u
#define GM1B_ABLATE_BASE_THETA_ADVECTION 4u
#define GM1B_ABLATE_BUOYANCY 8u
#define GM1B_ABLATE_POST_STEP_PPX 16u
#define GM1B_ABLATE_CARRIER_PROMOTION 32u

/*
 * Arrays of the serial-periodic flat lane.  Field order is the reference's
 * ALL_ARRAY_NAMES order: the acoustic-stage arrays of
 * src/cm1core/cuda_sound3_periodic.py:51-99 followed by the trajectory
 * extras of src/cm1core/cuda_psolver3_trajectory.py:93-104.  The acoustic
 * entry point ignores the trailing trajectory fields.
 */
typedef struct gm1b_periodic_arrays {
    /* scalar shape */
    float *mh, *rr0, *rf0, *c1, *c2, *mf, *piadv, *ppterm, *thv, *ppten;
    float *ppi, *pp3d, *ppx, *ppd, *qk, *pk1, *pk2, *mm, *fpk, *divh;
    float *hadvp, *elim_c, *elim_d, *tri_aa, *tri_bb, *tri_cc, *tri_dd;
    float *tri_pivot, *tri_residual;
    /* w shape */
    float *wten, *wa, *w3d, *rrw;
    /* u shape */
    float *ua, *u3d, *uten, *rru;
    /* v shape */
    float *va, *v3d, *vten, *rrv;
    /* metrics */
    float *dtu0, *dtv0, *uf, *vf, *uh, *vh;
    /* trajectory extras, scalar shape */
    float *pi0, *rho0, *rrf0, *th0, *rth0, *tha, *th3d, *sadv, *thten, *divx;
} gm1b_periodic_arrays;

/* ABI version of the loaded library (GM1B_ABI_VERSION at build time). */
GM1B_API int32_t gm1b_abi_version(void);

/* Message of the last failed call on this thread ("" if none). */
GM1B_API const char *gm1b_last_error(void);

/*
 * Small-step count and small time step of one RK stage.
 * Replaces sound3_stage_schedule_f32 (src/cm1core/cuda_sound3_column.py:391-417):
 * nsound must be even and >= 4, nrk in {1,2,3}.
 */
GM1B_API int32_t gm1b_sound3_stage_schedule(float dt, int32_t nsound, int32_t nrk,
                                   int32_t *nloop, float *dts);

/* RK stage time step dt/(4-nrk) in float32
 * (src/cm1core/cuda_sound3_column.py:420-424).  Returns NaN for a bad nrk. */
GM1B_API float gm1b_rk_stage_dt(float dt, int32_t nrk);

/*
 * Three psolver=3 acoustic RK stages (nrk = 1, 2, 3) of the serial-periodic
 * flat lane on device arrays, in place.
 * Replaces launch_cuda_sound3_periodic_three_stage
 * (src/cm1core/cuda_sound3_periodic.py:1216) and its CPU twin
 * cpu_sound3_periodic_three_stage_inplace (:1071).
 */
GM1B_API int32_t gm1b_sound3_periodic_three_stage(
    int32_t ni, int32_t nj, int32_t nk, const gm1b_periodic_arrays *arrays,
    float dt, int32_t nsound, float rdx, float rdy, float rdz, float cp,
    float alph, float kdiv, uint32_t flags, void *stream);

/*
 * `steps` dry RK3 large steps of the flat serial-periodic rigid-lid
 * trajectory (prepare, mass flux, divergence, fifth-order momentum advection
 * with buoyancy, the psolver=3 acoustic stage, averaged-flux theta advection
 * and update, ppx completion and carrier promotion), in place.
 * Replaces launch_cuda_psolver3_trajectory
 * (src/cm1core/cuda_psolver3_trajectory.py:1460) and its CPU twin
 * cpu_psolver3_trajectory_inplace (:761).
 */
GM1B_API int32_t gm1b_psolver3_trajectory(
    int32_t ni, int32_t nj, int32_t nk, const gm1b_periodic_arrays *arrays,
    int32_t steps, float dt, int32_t nsound, float dx, float dy, float dz,
    uint32_t ablations, uint32_t flags, void *stream);

/*
 * gm1b_psolver3_trajectory and gm1b_sound3_periodic_three_stage with the
 * persistent acoustic stage's grid-barrier status surfaced.  When a stage
 * runs as the one persistent cooperative kernel (no scratch outputs, nk <= 44,
 * the row tiles co-resident), each small step ends at a grid barrier whose
 * wait is bounded: after spin_limit polls (<= 0: the default, about a second
 * of L2 round trips) a CTA gives up, writes 1 into status_dev[0] and every
 * CTA leaves the kernel, so the fields of that call are invalid but the
 * context stays usable.  status_dev (one device int32, or NULL) is cleared
 * on the stream before the call's first launch.  The reference reads its
 * device status words back and refuses (cuda_graphs.read_device,
 * src/cm1core/cuda_graphs.py:197); the caller does that here by reading
 * status_dev after the stream's work.
 */
GM1B_API int32_t gm1b_psolver3_trajectory_checked(
    int32_t ni, int32_t nj, int32_t nk, const gm1b_periodic_arrays *arrays,
    int32_t steps, float dt, int32_t nsound, float dx, float dy, float dz,
    uint32_t ablations, uint32_t flags, int32_t spin_limit, int32_t *status_dev, void *stream);
GM1B_API int32_t gm1b_sound3_periodic_three_stage_checked(
    int32_t ni, int32_t nj, int32_t nk, const gm1b_periodic_arrays *arrays,
    float dt, int32_t nsound, float rdx, float rdy, float rdz, float cp,
    float alph, float kdiv, uint32_t flags, int32_t spin_limit, int32_t *status_dev, void *stream);


/* ------------------------------------------------------------------------
 * Padded lane (ng = 3 lateral ghost cells, CM1_OPEN_NGXY): shapes
 *   scalar (nk+2, nj+6, ni+6)   u/rru (nk+2, nj+6, ni+7)
 *   v/rrv  (nk+2, nj+7, ni+6)   w/rrw (nk+3, nj+6, ni+6)
 *   cell fields (nk, nj, ni), face-level fields (nk+1, nj, ni),
 *   rgzu (nj, ni+1), rgzv (nj+1, ni), dzdx/dzdy/gz (nj, ni)
 * (src/cm1core/cuda_advection5.py:293-300,987-995;
 *  src/cm1core/cuda_terrain_open_boundary.py:429-459).
 * ---------------------------------------------------------------------- */

typedef struct gm1b_mass_flux5_arrays {
    const float *u3d, *v3d, *w3d;
    float *rru, *rrv, *rrw;
    const float *rho0_3d, *rf0, *rgzu, *rgzv, *dzdx, *dzdy, *gz;
    float *divx;
} gm1b_mass_flux5_arrays;

/*
 * Terrain mass flux rru/rrv on interior faces, rrw (with the terrain term)
 * and the interior divergence divx of one RK stage.
 * Replaces launch_cuda_terrain_mass_flux5
 * (src/cm1core/cuda_advection5.py:849) and its CPU twin
 * cpu_terrain_mass_flux5_inplace (:271).  ni, nj, nk >= 8.
 */
GM1B_API int32_t gm1b_terrain_mass_flux5(int32_t ni, int32_t nj, int32_t nk,
                                         const gm1b_mass_flux5_arrays *arrays,
                                         float dx, float dy, float dz, void *stream);

typedef struct gm1b_scalar_advection5_arrays {
    const float *scalar, *rru, *rrv, *rrw;
    const float *c1, *c2, *rr0, *gz, *divx;
    float *tendency;
    /* face fluxes (shapes of rru, rrv, rrw); NULL = not written */
    float *flux_x, *flux_y, *flux_z;
} gm1b_scalar_advection5_arrays;

/*
 * Fifth-order (nrk = 1, 2) or WENO5-Z (nrk = 3 with wflag) flux-divergence
 * tendency of one scalar.  lateral_obc packs CM1's lateral side codes
 * wbc | ebc<<4 | sbc<<8 | nbc<<12 (1 periodic, 2 open, 3 rigid, 4 ...) for a
 * whole-domain call, or 0 for a tile-local call that leaves the outer three
 * cells unwritten.  levels_per_chunk sets the z-chunk of the marching CTAs
 * (<= 0: default).
 * Replaces launch_cuda_scalar_advection5 (src/cm1core/cuda_advection5.py:948)
 * and its CPU twin cpu_scalar_advection5_inplace (:440).  ni, nj, nk >= 8.
 */
GM1B_API int32_t gm1b_scalar_advection5(int32_t ni, int32_t nj, int32_t nk,
                                        const gm1b_scalar_advection5_arrays *arrays,
                                        int32_t nrk, int32_t wflag, float dx, float dy,
                                        float dz, double weps, uint32_t lateral_obc,
                                        int32_t levels_per_chunk, void *stream);

/*
 * The stretched-column scalar advection of
 * launch_cuda_gm1_child_stretched_scalar_advection5
 * (src/cm1core/cuda_gm1_child_stretched_scalar.py:666-842): the same face
 * fluxes, with the tendency's vertical derivative taken on a stretched
 * column.  flat = 0: CM1's terrain branch, -(d*rdsf(k)) with rdsf the
 * (nk+3,) CM1-indexed profile (:89-153); flat = 1: the flat column,
 * -((d*rdz)*mh(k)) with mh the (nk+2,) profile and the tendency scaled by
 * the column's rr0(k) without gz (:262-352; adv.F:555-572, 646-656).
 */
typedef struct gm1b_vertical_column {
    int32_t flat;
    const float *rdsf; /* flat = 0 */
    const float *mh;   /* flat = 1 */
    float rdz;         /* flat = 1: 1/dz of the metric reference */
} gm1b_vertical_column;

GM1B_API int32_t gm1b_scalar_advection5_column(int32_t ni, int32_t nj, int32_t nk,
                                               const gm1b_scalar_advection5_arrays *arrays, int32_t nrk,
                                               int32_t wflag, float dx, float dy, double weps,
                                               uint32_t lateral_obc, int32_t levels_per_chunk,
                                               const gm1b_vertical_column *column, void *stream);

/* ------------------------------------------------------------------------
 * eqtset=2 moist stage terms
 * ---------------------------------------------------------------------- */
typedef struct gm1b_eqtset2_arrays {
    /* base state: (nk) profiles, or (nk, nj, ni) with base3d; qc0/qi0 may be
     * NULL (base condensate exactly zero) */
    const float *th0, *qv0, *pi0, *qc0, *qi0;
    const float *th3d;  /* (nk, nj, ni) */
    const float *q3d;   /* (6, nk, nj, ni): qv, qc, qr, qi, qs, qg */
    const float *pp3d;  /* (nk+2, nj+2, ni+2) */
    float *thv, *ppterm; /* (nk+2, nj+2, ni+2), live cells written */
    float *buoyancy;     /* padded-lane scalar (nk+2, nj+6, ni+6), live cells written */
    float *thterm;       /* (nk, nj, ni) */
    float *piadv;        /* (nk+2, nj+2, ni+2), levels 1..nk incl. halos */
} gm1b_eqtset2_arrays;

/*
 * Moist buoyancy g*(th3d/th0 + (Rv/Rd-1)(qv-qv0) - (ql+qi-qc0-qi0)),
 * theta-rho, the theta and pressure energy terms of eqtset=2, and piadv.
 * Replaces the cell algebra of cpu_eqtset2_cell_f32
 * (src/cm1core/cuda_moist_stage_bridge.py:62) as applied by
 * launch_cuda_eqtset2_stage_terms (:378); the open-boundary halo fills that
 * launch adds are the boundary family's, not this operator's.
 */
GM1B_API int32_t gm1b_eqtset2_stage_terms(int32_t ni, int32_t nj, int32_t nk,
                                          const gm1b_eqtset2_arrays *arrays, int32_t base3d,
                                          void *stream);

/* ------------------------------------------------------------------------
 * Scalar/moisture RK stage pieces (padded lane)
 * ---------------------------------------------------------------------- */

/*
 * Theta transport carrier: padded[k+1, j+3, i+3] = (th0[k] - 300) + th3d[k, j, i]
 * (th0 (nk), th3d (nk, nj, ni), padded scalar shape; halos untouched).
 * Replaces cpu_theta_transport_scalar_inplace
 * (src/cm1core/cuda_scalar_moist_rk.py:255) and the packing kernel
 * cm1_rk_pack_theta_v1 (:587).
 */
GM1B_API int32_t gm1b_theta_transport_pack(int32_t ni, int32_t nj, int32_t nk, const float *th0,
                                           const float *th3d, float *padded, void *stream);

typedef struct gm1b_scalar_rk_compose_arrays {
    /* theta: `cells` words each */
    const float *theta_a, *theta_held, *theta_divterm, *theta_adv;
    float *theta_cur;
    /* moisture: nq * cells words each (species-major) */
    const float *q_a, *q_held, *q_adv;
    float *q_cur;
} gm1b_scalar_rk_compose_arrays;

/*
 * A-anchored RK update of theta and nq moisture species, dttmp = dt/(4-nrk):
 * theta = A + dttmp*((held - t11*thterm) + adv), q = A + dttmp*(held + adv),
 * |x| < 1e-30 flushed to 0.
 * Replaces cpu_compose_scalar_moist_rk_stage_inplace
 * (src/cm1core/cuda_scalar_moist_rk.py:283) and cm1_rk_compose_{theta,moisture}_v1.
 */
GM1B_API int32_t gm1b_scalar_moist_rk_compose(size_t cells, int32_t nq,
                                              const gm1b_scalar_rk_compose_arrays *arrays,
                                              int32_t nrk, float dt, void *stream);

typedef struct gm1b_pdef_arrays {
    const float *scalar_a;      /* (nk, nj, ni) */
    const float *scalar_padded; /* padded scalar shape */
    const float *rho0;          /* (nk, nj, ni) */
    const float *gz, *rgz;      /* (nj, ni) */
    const float *mass_flux;     /* rru (axis x), rrv (y) or rrw (z) shape */
    float *directional;         /* (nk, nj, ni), in/out */
    float *candidate;           /* (nk, nj, ni), out */
} gm1b_pdef_arrays;

/*
 * One terrain positive-definite direction pass (pdef x, y or z; axis 0/1/2):
 * candidate = rho0*A + dt*(directional + s*div(mass flux))*gz, then the
 * donor-cell repair of negative candidates along each line and the matching
 * update of `directional`.
 * Replaces cpu_pdef_direction_inplace (src/cm1core/cuda_scalar_moist_rk.py:352)
 * and cm1_rk_pdef_{directional,candidate_*,correct_*}_v1.
 */
GM1B_API int32_t gm1b_pdef_direction(int32_t ni, int32_t nj, int32_t nk, const gm1b_pdef_arrays *arrays,
                                     int32_t axis, float dt, float spacing, void *stream);

/* ------------------------------------------------------------------------
 * Kessler warm rain (compact mass arrays (nk, nj, ni), no halos)
 * ---------------------------------------------------------------------- */
typedef struct gm1b_kessler_arrays {
    /* inputs: ruh (ni), rvh (nj), rmh/mh/pi0/th0/rr mass-shaped */
    const float *ruh, *rvh, *rmh, *mh, *pi0, *th0, *rr;
    /* in/out, mass-shaped except rain (1, nj, ni) and prate (nj, ni) */
    float *rho, *pp3d, *th3d, *prs, *qv, *qc, *qr, *fall_velocity, *rain, *prate;
    /* in/out FP64 budgets: asq[3] (pdefq of qv, qc, qr), qbudget[10] */
    double *asq, *qbudget;
    /* optional outputs (NULL = not written): saturation-adjustment
     * iterations per cell (uint32, mass-shaped) and fallout sub-steps per
     * column (int32, (nj, ni)) */
    uint32_t *satadj_iterations;
    int32_t *nfall;
} gm1b_kessler_arrays;

/* Bytes of device workspace gm1b_kessler_driver needs for this grid. */
GM1B_API size_t gm1b_kessler_workspace_bytes(int32_t ni, int32_t nj, int32_t nk);

/*
 * The complete Kessler operator, in place: pdefq(qv, qc, qr), rain fall
 * speed, rain-energy budget, fallout sub-stepping, local conversion and
 * saturation adjustment (equation_set 1 or 2; efall must be 0).
 * `workspace` (16-byte aligned, gm1b_kessler_workspace_bytes) holds the
 * budget partial sums; its first three int32 words are set by the call to
 * the number of cells whose saturation adjustment did not converge within
 * 100 iterations (the reference raises on any), the largest fallout
 * sub-step count, and the number of columns whose fall Courant number was
 * not finite or reached 16384 (a blown-up state: such a column takes one
 * sub-step instead of int(crmax + 1), which would reach 2^31).
 * Replaces launch_cuda_gm1_kessler_driver
 * (src/cm1core/cuda_gm1_kessler_driver.py:907) and its CPU twin
 * cpu_gm1_kessler_driver_inplace (:431).
 */
GM1B_API int32_t gm1b_kessler_driver(int32_t ni, int32_t nj, int32_t nk,
                                     const gm1b_kessler_arrays *arrays, float dx, float dy,
                                     float dz, float dt, int32_t equation_set, int32_t efall,
                                     void *workspace, size_t workspace_size, void *stream);

/* Held-rate carriers of the equation-set-2 Kessler lifecycle, mass-shaped
 * (Gm1KesslerHeldCarriers, src/cm1core/cuda_gm1_kessler_large_step.py:112). */
typedef struct gm1b_kessler_held {
    float *qpten, *qtten, *qvten, *qcten;
} gm1b_kessler_held;

/*
 * The once-per-large-step Kessler transition, in place: with equation set 2
 * remove the held rates from pp3d, th3d, qv, qc and snapshot the result into
 * the carriers, form the pre-physics prs and rho (and rr = rho), run
 * gm1b_kessler_driver, then turn the carriers into the next step's rates
 * (state - snapshot) / dt.  held may be NULL for equation set 1.  Replaces
 * CudaGm1KesslerLargeStepTransition.apply (cuda_gm1_kessler_large_step.py:392)
 * and its CPU twin cpu_gm1_kessler_large_step_inplace (:183).
 */
GM1B_API int32_t gm1b_kessler_large_step(int32_t ni, int32_t nj, int32_t nk, const gm1b_kessler_arrays *arrays,
                                         const gm1b_kessler_held *held, float dx, float dy, float dz, float dt,
                                         int32_t equation_set, int32_t efall, void *workspace, size_t workspace_size,
                                         void *stream);

/*
 * The final-RK dry-air mass correction, apmasscon = 1 (replaces
 * launch_cuda_apmasscon, src/cm1core/cuda_apmasscon.py:596, and its CPU twin
 * cpu_apmasscon_inplace :256; CM1 solve2.F:1616-1656, :1972-2030): the
 * dry-mass ledger mass2 = sum over levels of the binary64 level sums of
 * ((rho*ruh)*rvh)*rmh and the Exner sum of pi0 + pp3d, the binary64
 * correction ((mass1/mass2)^rddcv - 1) * sum / cells rounded to binary32,
 * then pp3d += correction and prs = p00 * pi^(cp/rd), rho = prs / ((theta *
 * pi) * (rd + max(qv, 0) * rv)) rebuilt.  mass1 is a device word (the
 * initial ledger, gm1b_dry_mass); diagnostics (device, 4 doubles, may be
 * NULL) receive mass2, the Exner sum, the binary64 correction and mass1.
 * Arrays mass-shaped (nk, nj, ni) except ruh (ni) and rvh (nj); workspace
 * gm1b_apmasscon_workspace_bytes(nk).  Allocation-free; graph-capturable.
 */
typedef struct gm1b_apmasscon_arrays {
    const float *ruh, *rvh, *rmh, *pi0, *th0, *th3d, *qv;
    float *pp3d, *prs, *rho;
} gm1b_apmasscon_arrays;

GM1B_API size_t gm1b_apmasscon_workspace_bytes(int32_t nk);
GM1B_API int32_t gm1b_apmasscon(int32_t ni, int32_t nj, int32_t nk, const gm1b_apmasscon_arrays *arrays,
                                const double *mass1, double *diagnostics, void *workspace, void *stream);
/* The dry-mass ledger of a state into mass[0] (cpu_initial_dry_mass,
 * cuda_apmasscon.py:226; CM1 init3d.F:2483-2527); with only_if_unset a
 * non-zero mass[0] is kept (a ledger already held, e.g. restored). */
GM1B_API int32_t gm1b_dry_mass(int32_t ni, int32_t nj, int32_t nk, const float *rho, const float *ruh, const float *rvh,
                               const float *rmh, double *mass, int32_t only_if_unset, void *workspace, void *stream);
/* gm1b_kessler_large_step with the dry-mass correction between the
 * pre-physics equation of state and the driver (where the reference's
 * finish runs it, after remove-held-EOS and before pdefq: its
 * large_step_schedule MASS_BEGIN / MASS_FINISH, gm1_runtime.py:1969-2007);
 * rr takes the corrected rho.  The ruh, rvh and rmh of arrays weigh the
 * ledger. */
GM1B_API int32_t gm1b_kessler_large_step_apmasscon(int32_t ni, int32_t nj, int32_t nk,
                                                   const gm1b_kessler_arrays *arrays, const gm1b_kessler_held *held,
                                                   float dx, float dy, float dz, float dt, int32_t equation_set,
                                                   int32_t efall, void *workspace, size_t workspace_size,
                                                   const double *mass1, double *mass_diagnostics,
                                                   void *mass_workspace, void *stream);

/* The correction of a domain split over subdomains (each a widened block of
 * the domain, stepped on its own): the level partials of the dry-mass
 * ledger and of the Exner sum over a window of cells (columns i0..i1-1 of
 * rows j0..j1-1: the subdomain's own cells), gm1b_apmasscon_partials_words
 * doubles; the subdomains' partials added word by word (in a fixed order, or
 * by an all-reduce) give the domain's, from which every subdomain forms the
 * same correction.  _begin runs the transition up to the ledger (held rates,
 * pre-physics EOS, the window's partials), _end the rest from the added
 * partials and the domain's cell count.  gm1b_dry_mass_from_partials turns
 * added dry-mass partials (pressure = 0) into the ledger mass1. */
GM1B_API size_t gm1b_apmasscon_partials_words(int32_t nk);
GM1B_API int32_t gm1b_apmasscon_partials(int32_t ni, int32_t nj, int32_t nk, const float *rho, const float *ruh,
                                         const float *rvh, const float *rmh, const float *pi0, const float *pp3d,
                                         const int32_t *window, int32_t pressure, double *partials, void *stream);
GM1B_API int32_t gm1b_dry_mass_from_partials(int32_t nk, const double *partials, double *mass, int32_t only_if_unset,
                                             void *stream);
GM1B_API int32_t gm1b_kessler_large_step_apmasscon_begin(int32_t ni, int32_t nj, int32_t nk,
                                                         const gm1b_kessler_arrays *arrays,
                                                         const gm1b_kessler_held *held, float dt,
                                                         int32_t equation_set, const int32_t *window,
                                                         double *partials, void *stream);
GM1B_API int32_t gm1b_kessler_large_step_apmasscon_end(int32_t ni, int32_t nj, int32_t nk,
                                                       const gm1b_kessler_arrays *arrays,
                                                       const gm1b_kessler_held *held, float dx, float dy, float dz,
                                                       float dt, int32_t equation_set, int32_t efall, void *workspace,
                                                       size_t workspace_size, const double *partials, double cells,
                                                       const double *mass1, double *mass_diagnostics,
                                                       void *mass_workspace, void *stream);

/*
 * gm1b_kessler_driver without a workspace argument, for callers that cannot
 * allocate device memory of their own (for instance a Fortran or C host
 * model bound through this ABI whose device memory belongs to another
 * runtime's pool, or a process whose device memory another framework
 * reserves up front): the budget scratch lives in a static device array of
 * GM1B_KESSLER_STATIC_SCRATCH_BYTES (8 MiB), which every GPU that loads the
 * library holds until the process exits.  No counterpart in the reference
 * (its launcher always allocates a workspace).
 *
 * - Grids whose scratch exceeds 8 MiB are rejected with GM1B_ERR_ARGUMENT.
 *   The scratch is gm1b_kessler_workspace_bytes(ni, nj, nk) =
 *   16 + 8 * (5*ni*nj + 5*nj + 5*nk*nj*ceil(ni/128)) bytes: 4.27 MB at
 *   256x256x80 and 8.20 MB at 480x256x80 fit; 8.53 MB at 512x256x80 and
 *   32 MB at 640x768x80 are refused.
 * - Device ordinals 0..63 are served; a higher ordinal is refused.
 * - The first call on a device resolves the array's device address for that
 *   device (cudaGetSymbolAddress, with the device current); make that first
 *   call before any stream capture.
 * - All calls on a device share the one array: calls that overlap on the GPU
 *   (different streams, or other threads) race and must be serialised by the
 *   caller.  Each call clears the status words it uses.
 * - status_out (device pointer to 2 int32 words, or NULL) receives the
 *   non-converged saturation-adjustment cell count and the largest fallout
 *   sub-step count, stream-ordered after the operator.
 * - The call allocates no device memory and calls no allocator.
 */
#define GM1B_KESSLER_STATIC_SCRATCH_BYTES (8u * 1024u * 1024u)
GM1B_API int32_t gm1b_kessler_driver_static(int32_t ni, int32_t nj, int32_t nk,
                                            const gm1b_kessler_arrays *arrays, float dx, float dy,
                                            float dz, float dt, int32_t equation_set, int32_t efall,
                                            int32_t *status_out, void *stream);

/* ------------------------------------------------------------------------
 * SGS/TKE local algebra: every array (nk+1, nj, ni) (w levels) except
 * ruh (ni) and rvh (nj)
 * ---------------------------------------------------------------------- */
typedef struct gm1b_sgs_tke_arrays {
    const float *ruh, *rvh, *rmf, *nm, *defv, *defh;
    float *tkea, *tk, *grdscl, *rgrdscl, *lenscl, *dissten;
    float *cme, *ce1, *ce2, *csm, *kmh, *kmv, *khh, *khv, *tketen;
    /* optional (NULL = not written): count of clipped TKE words */
    uint32_t *clip_count;
} gm1b_sgs_tke_arrays;

/*
 * Deardorff tkekm on levels 1..nk-1 (grid and length scales, Km = Kh/Pr,
 * dissipation added into dissten), the free-slip lower face (tkebc) and the
 * pre-turbt TKE source tketen = -Kh N^2 - dissten + Km max(0, defv + defh).
 * Replaces launch_cuda_sgs_tke (src/cm1core/cuda_sgs_tke.py:637) and its CPU
 * twin cpu_sgs_tke_inplace (:220).
 */
GM1B_API int32_t gm1b_sgs_tke(int32_t ni, int32_t nj, int32_t nk, const gm1b_sgs_tke_arrays *arrays,
                              float dx, float dy, float dz, void *stream);

/* ------------------------------------------------------------------------
 * Terrain/open fifth-order momentum advection of the padded lane (shapes as
 * above; uh (ni+6), vh (nj+6); rho0_3d (nk, nj, ni); rf0, rrf0, c2
 * (nk+1, nj, ni); gz, dzdx, dzdy (nj, ni); gzu, rgzu (nj, ni+1); gzv, rgzv
 * (nj+1, ni); divx (nk, nj, ni)).
 * ---------------------------------------------------------------------- */
typedef struct gm1b_momentum5_arrays {
    const float *u3d;
    float *uten, *rru;
    const float *v3d;
    float *vten, *rrv;
    const float *w3d;
    float *wten, *rrw;
    const float *uh, *vh, *rho0_3d, *rf0, *rrf0, *c2, *gz, *gzu, *gzv, *rgzu, *rgzv, *dzdx, *dzdy;
    float *divx;
} gm1b_momentum5_arrays;

/* Mass fluxes rru, rrv (every face) and rrw (with the terrain term), the
 * divergence divx, and the advu / advv / advw increments added into uten,
 * vten, wten.  lateral_obc packs CM1's (wbc, ebc, sbc, nbc) as
 * wbc|ebc<<4|sbc<<8|nbc<<12 (1 periodic on both sides of a direction, 2
 * open, 3/4 walls).  Replaces launch_cuda_terrain_open_momentum_advection5
 * (src/cm1core/cuda_momentum_advection5.py:1173) and its CPU twin
 * cpu_terrain_open_momentum_advection5_inplace (:753).  ni, nj >= 7, nk >= 8. */
GM1B_API int32_t gm1b_momentum_advection5(int32_t ni, int32_t nj, int32_t nk, const gm1b_momentum5_arrays *arrays,
                                          uint32_t lateral_obc, float dx, float dy, float dz, void *stream);

/*
 * The momentum advection on a stretched column
 * (launch_cuda_gm1_child_stretched_momentum5,
 * src/cm1core/cuda_gm1_child_stretched_momentum.py:540-780).  flat = 0: CM1's
 * terrain branch with the column's sigma (nk+2), sigmaf (nk+3), rds (nk+2)
 * and rdsf (nk+3) profiles, the physical top ztop and the base density from
 * rho0_padded ((nk+2, nj+6, ni+6)); flat = 1: the flat column
 * (solve2.F:493-520, 605-617; adv.F's rdz*mh / rdz*mf statements) with mh
 * (nk+2), mf (nk+3), rdz, and the column's rho0_padded(k, 3, 3), rf0, rr0 and
 * rrf0 words.  The split entries place a hook (an rrw fill) between the mass
 * fluxes and the transport as the uniform ones do.
 */
typedef struct gm1b_momentum_column {
    int32_t flat;
    const float *rho0_padded;
    const float *sigma, *sigmaf, *rds, *rdsf; /* flat = 0 */
    float ztop;                               /* flat = 0 */
    const float *mh, *mf, *rr0;               /* flat = 1 (rr0 compact (nk, nj, ni)) */
    float rdz;                                /* flat = 1 */
} gm1b_momentum_column;

GM1B_API int32_t gm1b_momentum_advection5_column(int32_t ni, int32_t nj, int32_t nk, const gm1b_momentum5_arrays *s,
                                                 uint32_t lateral_obc, float dx, float dy,
                                                 const gm1b_momentum_column *column, void *stream);
GM1B_API int32_t gm1b_momentum_mass_flux5_column(int32_t ni, int32_t nj, int32_t nk, const gm1b_momentum5_arrays *s,
                                                 uint32_t lateral_obc, float dx, float dy,
                                                 const gm1b_momentum_column *column, void *stream);
GM1B_API int32_t gm1b_momentum_transport5_column(int32_t ni, int32_t nj, int32_t nk, const gm1b_momentum5_arrays *s,
                                                 uint32_t lateral_obc, float dx, float dy,
                                                 const gm1b_momentum_column *column, void *stream);

/* ------------------------------------------------------------------------
 * Terrain + all-open psolver=3 acoustic RK stage (padded ng = 3 lane).
 * Replaces launch_cuda_psolver3_terrain_open_stage / _three_stage
 * (src/cm1core/cuda_psolver3_terrain_open.py:1436, :1217) and their CPU twin
 * cpu_psolver3_terrain_open_stage_inplace (:774).  Shapes as
 * terrain_open_sound_shapes (:162): pressure family (nk+2, nj+2, ni+2),
 * u (nk+2, nj+6, ni+7), v (nk+2, nj+7, ni+6), w (nk+3, nj+6, ni+6), scalar
 * (nk+2, nj+6, ni+6), radbcw/e (nk+2, nj+6), radbcs/n (nk+2, ni+6), uh
 * (ni+6), vh (nj+6), ruf (ni+7), rvf (nj+7); metrics as terrain_static_shapes
 * (src/cm1core/cuda_terrain_open_boundary.py:429).  ni, nj >= 3, nk >= 4.
 * ------------------------------------------------------------------------ */
typedef struct gm1b_terrain_open_arrays {
    float *ppi, *pp3d, *ppx, *ppd, *piadv, *ppterm, *ppten, *thv, *qk, *pk1, *pk2, *mm, *fpk, *divh, *hadvp, *dum3,
        *elim_c, *elim_d, *tri_aa, *tri_bb, *tri_cc, *tri_dd, *tri_pivot, *tri_residual;
    float *ua, *u3d, *uten, *rru, *va, *v3d, *vten, *rrv, *wa, *w3d, *wten, *rrw;
    float *radbcw, *radbce, *radbcs, *radbcn, *uh, *vh, *ruf, *rvf, *scalar;
} gm1b_terrain_open_arrays;

typedef struct gm1b_terrain_metrics {
    const float *rho0_3d, *rr0, *rf0, *rrf0, *c1, *c2, *gz, *rgzu, *rgzv, *dzdx, *dzdy, *gx, *gxu, *gy, *gyv;
} gm1b_terrain_metrics;

/* TerrainOpenSoundAblations (:276): a set bit runs that phase */
#define GM1B_TOS_OPEN_CONSUMPTION 1u
#define GM1B_TOS_PRESSURE_GRADIENT 2u
#define GM1B_TOS_TRANSFORMED_DIVERGENCE 4u
#define GM1B_TOS_PRESSURE_ADVECTION 8u
#define GM1B_TOS_IMPLICIT_SOLVE 16u
#define GM1B_TOS_BETWEEN_STEP_FILL 32u
#define GM1B_TOS_RADIATION 64u
#define GM1B_TOS_STAGE_FILLS 128u
#define GM1B_TOS_ALL 255u
/* flags: leave every scratch array (qk .. tri_residual) as the CPU twin
 * does; without it only the prognostic and radiation arrays are written
 * (qk, pk1, pk2, mm hold this stage's coefficients) */
#define GM1B_TOS_DIAGNOSTICS 1u

/* One RK stage nrk (1..3).  dz is double because the lid height is
 * float32(nk * dz) of a double dz (:528).  Allocation-free; graph-capturable. */
GM1B_API int32_t gm1b_terrain_open_stage(int32_t ni, int32_t nj, int32_t nk, int32_t nrk, float dt, int32_t nsound,
                                         float dx, float dy, double dz, float alph, float kdiv, uint32_t ablations,
                                         uint32_t flags, const gm1b_terrain_open_arrays *arrays,
                                         const gm1b_terrain_metrics *metrics, void *stream);

/* The same stage on a stretched column (replaces
 * launch_cuda_gm1_child_psolver3_open_stage, cuda_gm1_child_psolver3_open.py:848).
 * Terrain column (column->flat = 0): sigma/sigmaf/rds/rdsf at CM1's indices,
 * the lid ztop and the padded base density rho0_padded (nk+2, nj+6, ni+6);
 * lateral_obc must be all-open 0x2222.  Flat column (flat = 1): sound.F's
 * terrain_flag=.false. statements on mh (nk+2), mf (nk+3) and rdz, the base
 * state at CM1's (1,1,k), no bcwsfc; lateral_obc = wbc | ebc << 4 |
 * sbc << 8 | nbc << 12 (the pressure gradient's dtu0/dtv0 mask, ssopenbc on
 * the open sides).  No dz: every vertical derivative reads the profiles.
 * Allocation-free; graph-capturable. */
GM1B_API int32_t gm1b_terrain_open_stage_column(int32_t ni, int32_t nj, int32_t nk, int32_t nrk, float dt,
                                                int32_t nsound, float dx, float dy, float alph, float kdiv,
                                                uint32_t ablations, uint32_t flags, uint32_t lateral_obc,
                                                const gm1b_terrain_open_arrays *arrays,
                                                const gm1b_terrain_metrics *metrics,
                                                const gm1b_momentum_column *column, void *stream);

/* ------------------------------------------------------------------------
 * Pieces that join the operators of the moist large step on the open lane.
 * ------------------------------------------------------------------------ */
/* Open-lateral halo fills in the reference's two ordered passes
 * (cpu_bcp/bcs/bcu/bcv/bcw_open_inplace, src/cm1core/cuda_sound3_open_boundary.py:249-335). */
#define GM1B_FILL_PRESSURE 0     /* bcp: (nk+2, nj+2, ni+2), levels 1..nk */
#define GM1B_FILL_SCALAR 1       /* bcs: (nk+2, nj+6, ni+6), levels 1..nk */
#define GM1B_FILL_U 2            /* bcu: (nk+2, nj+6, ni+7) */
#define GM1B_FILL_V 3            /* bcv: (nk+2, nj+7, ni+6) */
#define GM1B_FILL_W 4            /* bcw flag 1: (nk+3, nj+6, ni+6), levels 2..nk, then w(1) = w(nk+1) = 0 */
#define GM1B_FILL_W_KEEP_ENDS 5  /* bcw flag 0 */
GM1B_API int32_t gm1b_open_fill(int32_t ni, int32_t nj, int32_t nk, int32_t kind, float *q, void *stream);

/* Moist buoyancy into the live tendencies: wten += c1 dum8 + c2 dum8 on the
 * interior w levels, uten/vten += the terrain-horizontal part
 * (launch_cuda_moist_buoyancy, src/cm1core/cuda_moist_stage_bridge.py:433;
 * kernel cm1_msb_buoyancy_v1 in that file's source).  dum8 is the scalar
 * layout (nk+2, nj+6, ni+6) with open halos; c1, c2 (nk+1, nj, ni); gxu
 * (nk+1, nj, ni+1); gyv (nk+1, nj+1, ni). */
GM1B_API int32_t gm1b_moist_buoyancy(int32_t ni, int32_t nj, int32_t nk, const float *dum8, const float *c1,
                                     const float *c2, const float *gxu, const float *gyv, float *uten, float *vten,
                                     float *wten, void *stream);

/* launch_cuda_gm1_flat_stretched_buoyancy (src/cm1core/cuda_gm1_child_stretched_moist.py:240):
 * the flat column's buoyancy, added to wten only. */
GM1B_API int32_t gm1b_moist_buoyancy_flat(int32_t ni, int32_t nj, int32_t nk, const float *dum8, const float *c1,
                                          const float *c2, float *wten, void *stream);

/* Post-acoustic getdiv on the acoustic-averaged velocities (divergence and
 * theta_divergence_term = divergence * thterm, compact), then getdivx in
 * place: rru/rrv/rrw become mass fluxes and divx their divergence
 * (launch_cuda_post_acoustic_flux_bridge, cuda_moist_stage_bridge.py:461). */
typedef struct gm1b_post_acoustic_arrays {
    float *rru, *rrv, *rrw;
    const float *rgzu, *rgzv, *dzdx, *dzdy, *gz, *rho0_3d, *rf0, *thterm;
    float *divergence, *theta_divergence_term, *divx;
} gm1b_post_acoustic_arrays;
GM1B_API int32_t gm1b_post_acoustic_flux(int32_t ni, int32_t nj, int32_t nk, const gm1b_post_acoustic_arrays *arrays,
                                         float dx, float dy, float dz, void *stream);

/* The post-acoustic getdiv/getdivx on a stretched column
 * (launch_cuda_gm1_child_stretched_post_acoustic,
 * src/cm1core/cuda_gm1_child_stretched_moist.py:286; the flat texts :83-110):
 * flat = 0, the terrain branch with the column's sigma/sigmaf/rds/rdsf, its
 * physical top and the padded base density; flat = 1, the flat column's
 * rdz*mh(k), rho0_padded(k, 3, 3) and rf0(1,1,k), no terrain w.  Reads only
 * the column fields named there. */
GM1B_API int32_t gm1b_post_acoustic_flux_column(int32_t ni, int32_t nj, int32_t nk,
                                                const gm1b_post_acoustic_arrays *arrays, float dx, float dy,
                                                const gm1b_momentum_column *column, void *stream);

/* The final-stage positive-definite moisture chain of one species: WENO
 * face fluxes (horizontal, vertical with the lower/upper closures), the
 * directional advection with the open-side inflow edits, the pdef
 * candidate/correction in x, y and z (boundary-family repair rows when
 * lateral_obc != 0), and the total advection (launch_cuda_scalar_moist_rk_stage
 * final stage, src/cm1core/cuda_scalar_moist_rk.py:1336-1500).  pdefweno is 0
 * for qv and 1 for the other species. */
typedef struct gm1b_pdef_chain_arrays {
    const float *scalar_a, *scalar_padded, *rho0_3d, *gz, *rgz, *rr0, *c1, *c2, *divx, *rru, *rrv, *rrw;
    float *fx, *fy, *fz, *advx, *advy, *advz, *candidate, *advection;
} gm1b_pdef_chain_arrays;
GM1B_API int32_t gm1b_pdef_moisture_chain(int32_t ni, int32_t nj, int32_t nk, const gm1b_pdef_chain_arrays *arrays,
                                          float dttmp, float dx, float dy, float dz, double weps, uint32_t lateral_obc,
                                          int32_t pdefweno, void *stream);

/* The chain on a stretched column (launch_cuda_gm1_child_stretched_pdef_moisture,
 * src/cm1core/cuda_gm1_child_stretched_scalar.py:851): flat = 0, the
 * terrain branch's rdsf(k) in every vertical derivative; flat = 1, the flat
 * column's rdz*mh(k) with the column's rho0(k) and rr0(k) and no gz or rgz. */
GM1B_API int32_t gm1b_pdef_moisture_chain_column(int32_t ni, int32_t nj, int32_t nk, const gm1b_pdef_chain_arrays *a,
                                                 float dttmp, float dx, float dy, double weps, uint32_t lateral_obc,
                                                 int32_t pdefweno, const gm1b_vertical_column *column, void *stream);

/* Held-tendency composition once per large step: ppten from the held theta
 * and qv tendencies (or the microphysics pressure rate alone), then the
 * microphysics rates join the held theta/qv/qc tendencies
 * (gm1_child_predict_and_compose_held_base3d_v1,
 * src/cm1core/cuda_gm1_child_step_composer.py:547-556).  Mass-shaped except
 * ppten (nk+2, nj+2, ni+2) and qheld (2+, nk, nj, ni). */
typedef struct gm1b_held_arrays {
    const float *th0, *pi0, *rho, *ppi, *tha, *qa, *qpten, *qtten, *qvten, *qcten;
    float *thheld, *qheld, *ppten;
} gm1b_held_arrays;
GM1B_API int32_t gm1b_held_compose(int32_t ni, int32_t nj, int32_t nk, const gm1b_held_arrays *arrays, float dt,
                                   void *stream);

/* solve3 density: rr = 1/rho, rf = face average (c1, c2) with the uniform
 * Fornberg ends (gm1_solve3_density_v1, src/cm1core/cuda_gm1_forecast.py:548). */
GM1B_API int32_t gm1b_solve3_density(int32_t ni, int32_t nj, int32_t nk, const float *rho, const float *c1,
                                     const float *c2, float *rr, float *rf, void *stream);

/* Surface w on the physical bottom faces from u, v and the terrain slopes
 * (cpu_bcwsfc_terrain_physical_inplace, src/cm1core/cuda_terrain_open_boundary.py:687);
 * gz, dzdx, dzdy are (nj, ni). */
GM1B_API int32_t gm1b_bcwsfc(int32_t ni, int32_t nj, int32_t nk, const float *u3d, const float *v3d, float *w3d,
                             const float *gz, const float *dzdx, const float *dzdy, void *stream);

/* The open halo of the w(1) slab: west/east over every row, then
 * south/north over every column (cm1_momentum_rk_bc2d_open_v1,
 * src/cm1core/cuda_momentum_rk.py, directions 0..3). */
GM1B_API int32_t gm1b_w_level1_fill(int32_t ni, int32_t nj, int32_t nk, float *w3d, void *stream);

/* Copy a compact (nk, nj, ni) scalar into the interior of its padded
 * (nk+2, nj+6, ni+6) carrier (cm1_rk_pack_scalar_v1). */
GM1B_API int32_t gm1b_pack_scalar(int32_t ni, int32_t nj, int32_t nk, const float *scalar, float *padded,
                                  void *stream);

/* The two halves of gm1b_momentum_advection5, for a caller that edits the
 * fluxes or divx between them (the reference's post_divergence_hook seam):
 * the mass fluxes and divx, then the advu / advv / advw increments from the
 * fluxes and divx already formed (_cpu_momentum_transport5,
 * src/cm1core/cuda_momentum_advection5.py:871). */
GM1B_API int32_t gm1b_momentum_mass_flux5(int32_t ni, int32_t nj, int32_t nk, const gm1b_momentum5_arrays *arrays,
                                          uint32_t lateral_obc, float dx, float dy, float dz, void *stream);
GM1B_API int32_t gm1b_momentum_transport5(int32_t ni, int32_t nj, int32_t nk, const gm1b_momentum5_arrays *arrays,
                                          uint32_t lateral_obc, float dx, float dy, float dz, void *stream);

/* ------------------------------------------------------------------------
 * TKE evolution on the terrain lane: turbt and the flux-form RK stages.
 * Face fields (nk+1, nj, ni): tkea, tke3d, tketen, kmh, kmv, rf, mf, c1, c2,
 * rrf0; mass fields (nk, nj, ni): rho, mh, divx; gz, rgz (nj, ni), rgzu
 * (nj, ni+1), rgzv (nj+1, ni); padded mass fluxes rru (nk+2, nj+6, ni+7),
 * rrv (nk+2, nj+7, ni+6), rrw (nk+3, nj+6, ni+6).
 * ---------------------------------------------------------------------- */
typedef struct gm1b_tke_evolution_arrays {
    float *tkea, *tke3d, *tketen;
    const float *kmh, *kmv, *rho, *rf, *mh, *mf, *gz, *rgz, *rgzu, *rgzv, *c1, *c2, *rrf0, *rru, *rrv, *rrw, *divx;
} gm1b_tke_evolution_arrays;

/* turbt: the horizontal TKE flux divergence with the terrain correction
 * (zero on the outermost columns) and the vertically implicit diffusion,
 * added into tketen.  Replaces launch_cuda_tke_diffusion
 * (src/cm1core/cuda_tke_evolution.py:421).  nk <= 201. */
GM1B_API int32_t gm1b_tke_diffusion(int32_t ni, int32_t nj, int32_t nk, const gm1b_tke_evolution_arrays *arrays,
                                    float dx, float dy, float dz, float dt, void *stream);

/* One RK stage nrk (1..3) from the stage-start field cur into nxt (distinct
 * face volumes): fifth-order (WENO5 at nrk = 3) flux-form advection with the
 * open-side edits and the divergence correction, tkea + dt/(4-nrk) *
 * tendency, words below 1e-10 set to zero.  Replaces
 * launch_cuda_tke_rk_stage (src/cm1core/cuda_tke_evolution.py:430). */
GM1B_API int32_t gm1b_tke_rk_stage(int32_t ni, int32_t nj, int32_t nk, const gm1b_tke_evolution_arrays *arrays,
                                   const float *cur, float *nxt, int32_t nrk, float dx, float dy, float dz, float dt,
                                   void *stream);

/* turbt on a flat (terrain_flag=.false.) stretched column: the face fluxes
 * -0.25*(rf(a)+rf(a-1))*2*(kmh(a)+kmh(a-1))*(t(a)-t(a-1))*rdx (no terrain
 * correction; zero divergence on the outermost columns) and the implicit
 * diffusion with the coordinate's reference rdz and the 3-D mh (mass) and
 * mf (face), added into tketen.  Reads tke3d, kmh, kmv, rho, rf, mh, mf,
 * tketen.  Replaces enqueue_flat_turbt
 * (src/cm1core/cuda_gm1_flat_stretched_closure.py:631).  nk <= 201. */
GM1B_API int32_t gm1b_tke_diffusion_flat(int32_t ni, int32_t nj, int32_t nk, const gm1b_tke_evolution_arrays *arrays,
                                         float dx, float dy, float rdz, float dt, void *stream);

/* One RK stage on a flat stretched column: gm1b_tke_rk_stage with the
 * vertical divergence -(dumz(k)-dumz(k-1))*rdz*mf(k) (mf_profile: nk+3
 * words, CM1-indexed), the column's c2 and rrf0 (their (k, 0, 0) words),
 * and the open-side divergence piece (q*d)*rdx.  Reads tkea, tketen, c2,
 * rrf0, rru, rrv, rrw, divx.  Replaces the flat branch of
 * CartesianClosure.tke_rk (src/cm1core/cuda_cartesian_closure.py:1658-1663,
 * kernel gm1_flat_tke_advw_rk_v1 of cuda_gm1_flat_stretched_closure.py). */
GM1B_API int32_t gm1b_tke_rk_stage_flat(int32_t ni, int32_t nj, int32_t nk, const gm1b_tke_evolution_arrays *arrays,
                                        const float *mf_profile, const float *cur, float *nxt, int32_t nrk, float dx,
                                        float dy, float rdz, float dt, void *stream);

/* The whole operator: turbt, the three RK stages from tke3d, and the commit
 * tke3d = tkea = result.  workspace: one face volume.  Replaces
 * launch_cuda_tke_evolution (src/cm1core/cuda_tke_evolution.py:481) and the
 * CPU twin cpu_tke_evolution_inplace (:206). */
GM1B_API int32_t gm1b_tke_evolution(int32_t ni, int32_t nj, int32_t nk, const gm1b_tke_evolution_arrays *arrays,
                                    float *workspace, float dx, float dy, float dz, float dt, void *stream);

/* ------------------------------------------------------------------------
 * TKE source inputs: deformation and moist N^2 (compact physical arrays)
 * ---------------------------------------------------------------------- */

/* u3d (nk, nj, ni+1), v3d (nk, nj+1, ni), w3d/rf/c1/c2/gx/gy/defv/defh
 * (nk+1, nj, ni), rho (nk, nj, ni), gz/rgz (nj, ni), rgzu (nj, ni+1),
 * rgzv (nj+1, ni).  The reference's gzu and gzv enter no formula of this
 * branch and are not passed. */
typedef struct gm1b_deformation_arrays {
    const float *u3d, *v3d, *w3d, *rho, *rf, *c1, *c2, *gz, *rgz, *rgzu, *rgzv, *gx, *gy;
    float *defv, *defh;
} gm1b_deformation_arrays;

/*
 * CM1 calcdef, Cartesian terrain branch with four open sides: defv and
 * defh on face levels 1..nk-1 (levels 0 and nk are zero).  One kernel, no
 * device scratch.  Replaces launch_cuda_terrain_deformation
 * (src/cm1core/cuda_terrain_deformation.py:914) and its CPU twin
 * cpu_terrain_deformation_inplace (:234).  ni, nj, nk >= 3.
 */
GM1B_API int32_t gm1b_terrain_deformation(int32_t ni, int32_t nj, int32_t nk, const gm1b_deformation_arrays *arrays,
                                          float dx, float dy, float dz, void *stream);

/* u3d (nk, nj, ni+1), v3d (nk, nj+1, ni), w3d/rf/mf/c1/c2/defv/defh
 * (nk+1, nj, ni), rho (nk, nj, ni), mh_profile (nk+2, CM1-indexed: word k+1
 * is the mh of mass level k). */
typedef struct gm1b_flat_deformation_arrays {
    const float *u3d, *v3d, *w3d, *rho, *rf, *mf, *c1, *c2, *mh_profile;
    float *defv, *defh;
} gm1b_flat_deformation_arrays;

/*
 * CM1 calcdef on a flat (terrain_flag=.false.) stretched column: the strains
 * with rdz*mh(k) and rdz*mf(k), the open sides as an index clamp, and the
 * deformation reduction; defv and defh on face levels 1..nk-1, levels 0 and
 * nk zero.  One kernel, no device scratch.  rdz is the vertical coordinate's
 * reference 1/dz.  Replaces enqueue_flat_calcdef
 * (src/cm1core/cuda_gm1_flat_stretched_closure.py:524) with the zero fill
 * of defv/defh before it (cuda_cartesian_closure.py:1130-1131).
 */
GM1B_API int32_t gm1b_flat_deformation(int32_t ni, int32_t nj, int32_t nk, const gm1b_flat_deformation_arrays *arrays,
                                       float dx, float dy, float rdz, void *stream);

/* The SGS stress of the flat (terrain_flag=.false.) stretched column.
 * Shapes (C order): u3d/uten (nk, nj, ni+1), v3d/vten (nk, nj+1, ni),
 * w3d/wten/rf/mf/kmh/kmv (nk+1, nj, ni), rho/mh/s11/s22/s33/t11/t22/t33
 * (nk, nj, ni), s12/t12 (nk, nj+1, ni+1), s13/t13 (nk+1, nj, ni+1), s23/t23
 * (nk+1, nj+1, ni), mh_profile (nk+2, CM1-indexed: word k+1 is the mh of
 * mass level k).  Each entry point reads and writes only the arrays it
 * names below; the others may be NULL. */
typedef struct gm1b_flat_stress_arrays {
    const float *u3d, *v3d, *w3d, *rho, *rf, *mh, *mf, *mh_profile, *kmh, *kmv;
    float *s11, *s22, *s33, *s12, *s13, *s23;
    float *t11, *t22, *t33, *t12, *t13, *t23;
    float *uten, *vten, *wten;
} gm1b_flat_stress_arrays;

/*
 * The strain carriers rho*Sij of the flat calcdef's mass and face passes:
 * s11/s22/s33 at cells, s12 at every corner (an open side takes the nearest
 * interior corner), s13/s23 on face levels 1..nk-1 (levels 0 and nk not
 * written).  Reads u3d, v3d, w3d, rho, rf, mf, mh_profile.  Replaces the
 * strain half of enqueue_flat_calcdef (gm1_flat_calcdef_mass_v1 / _face_v1,
 * src/cm1core/cuda_gm1_flat_stretched_closure.py:76-114, :524-548).
 */
GM1B_API int32_t gm1b_flat_strain(int32_t ni, int32_t nj, int32_t nk, const gm1b_flat_stress_arrays *arrays,
                                  float dx, float dy, float rdz, void *stream);

/*
 * CM1 gettau with the free-slip lower and upper faces: t11/t22/t33 =
 * s*(kmh(k)+kmh(k+1)), t12 from the clamped interior corner and the eight
 * surrounding kmh, t13/t23 on every face level (levels 0 and nk copy levels
 * 1 and nk-1).  Reads s11..s23, kmh, kmv.  Replaces enqueue_flat_gettau
 * (src/cm1core/cuda_gm1_flat_stretched_closure.py:551).
 */
GM1B_API int32_t gm1b_flat_gettau(int32_t ni, int32_t nj, int32_t nk, const gm1b_flat_stress_arrays *arrays,
                                  void *stream);

/*
 * CM1 turbu/turbuz, turbv/turbvz and turbw with their implicit vertical
 * solves (doimpl = 1, the two-part block off), ADDED into uten, vten and
 * wten (wten on faces 1..nk-1).  Reads t11..t23, kmh, kmv, rho, rf, mh, mf,
 * u3d, v3d, w3d.  nk <= 200 (the column solves' shared memory).  Replaces
 * enqueue_flat_momentum_stress with two_part=None
 * (src/cm1core/cuda_gm1_flat_stretched_closure.py:574).
 */
GM1B_API int32_t gm1b_flat_momentum_stress(int32_t ni, int32_t nj, int32_t nk, const gm1b_flat_stress_arrays *arrays,
                                           float dx, float dy, float rdz, float dt, void *stream);

/* gm1b_flat_strain, gm1b_flat_gettau and gm1b_flat_momentum_stress in that
 * order on one stream (the stress block of cuda_cartesian_closure.py:1293-1317
 * with the strain carriers its calcdef left). */
GM1B_API int32_t gm1b_flat_sgs_stress(int32_t ni, int32_t nj, int32_t nk, const gm1b_flat_stress_arrays *arrays,
                                      float dx, float dy, float rdz, float dt, void *stream);

/* th0 (nk); tha/rho/rr/mh/thten (nk, nj, ni); qa/qten rows of nk*nj*ni words
 * (moisture row q at word q*nk*nj*ni); rf/mf/khh/khv (nk+1, nj, ni);
 * workspace gm1b_flat_scalar_turbulence_workspace_words() words of device
 * scratch (the horizontal flux divergence of every scalar). */
typedef struct gm1b_flat_scalar_turbulence_arrays {
    const float *th0, *tha, *qa, *rho, *rr, *rf, *mh, *mf, *khh, *khv;
    float *thten, *qten, *workspace;
} gm1b_flat_scalar_turbulence_arrays;

/* Words of the scalar turbulence's workspace: (numq + 1)*nk*nj*ni. */
GM1B_API int64_t gm1b_flat_scalar_turbulence_workspace_words(int32_t ni, int32_t nj, int32_t nk, int32_t numq);

/*
 * CM1 turbs on the flat stretched column for theta ((th0 - 300) + tha) and
 * then moisture rows 0..numq-1: the x/y diffusive fluxes with khh on the
 * open-halo copies (index clamps) and the implicit vertical diffusion with
 * khv, mh and mf, zero surface flux; ADDED into thten and the first numq
 * rows of qten.  dz is the coordinate's reference spacing; nk <= 200.
 * Replaces the scalar loop of the closure's held phase on the flat lane
 * (cuda_cartesian_closure.py:1566-1633: gm1_turbs_pad_static_open_v1,
 * gm1_turbs_pack_scalar_open_v1, gm1_flat_turbs_xy_flux_v1,
 * gm1_flat_turbs_implicit_apply_v1).
 */
GM1B_API int32_t gm1b_flat_scalar_turbulence(int32_t ni, int32_t nj, int32_t nk, int32_t numq,
                                             const gm1b_flat_scalar_turbulence_arrays *arrays, float dx, float dy,
                                             float dz, float dt, void *stream);

/* The terrain texts' stress (the uniform column's family): compact arrays,
 * shapes as gm1b_flat_stress_arrays, plus the column metrics gz/rgz (nj,
 * ni), gzu/rgzu (nj, ni+1), gzv/rgzv (nj+1, ni) and the slopes gx/gy (nk+1,
 * nj, ni), gxu (nk+1, nj, ni+1), gyv (nk+1, nj+1, ni). */
typedef struct gm1b_terrain_stress_arrays {
    const float *u3d, *v3d, *w3d, *rho, *rf, *mh, *mf, *kmh, *kmv;
    const float *gz, *rgz, *gzu, *rgzu, *gzv, *rgzv, *gx, *gy, *gxu, *gyv;
    float *s11, *s22, *s33, *s12, *s13, *s23;
    float *t11, *t22, *t33, *t12, *t13, *t23;
    float *uten, *vten, *wten;
} gm1b_terrain_stress_arrays;

/*
 * The strain carriers rho*Sij of the terrain calcdef: s11/s22/s33 at cells,
 * s12 at every corner (an open side takes the nearest interior corner),
 * s13/s23 on face levels 1..nk-1.  Reads u3d, v3d, w3d, rho, rf, gz, rgz,
 * rgzu, rgzv, gx, gy.  Replaces the strain half of
 * cpu_terrain_deformation_inplace
 * (src/cm1core/cuda_terrain_deformation.py:234-736).
 */
GM1B_API int32_t gm1b_terrain_strain(int32_t ni, int32_t nj, int32_t nk, const gm1b_terrain_stress_arrays *arrays,
                                     float dx, float dy, float dz, void *stream);

/*
 * CM1 gettau (t13/t23 levels 0 and nk copy levels 1 and nk-1, the eight-kmh
 * t12 at the clamped corner columns) and turbu/turbuz, turbv/turbvz and
 * turbw on the terrain texts with their implicit vertical solves (doimpl =
 * 1, four open sides, free-slip bottom and top), ADDED into uten, vten and
 * wten (wten on faces 1..nk-1).  nk <= 200.  Replaces
 * cpu_sgs_stress_tendency_inplace and its kernels
 * (src/cm1core/cuda_sgs_stress_tendency.py:292-449).
 */
GM1B_API int32_t gm1b_terrain_stress(int32_t ni, int32_t nj, int32_t nk, const gm1b_terrain_stress_arrays *arrays,
                                     float dx, float dy, float dz, float dt, void *stream);

/* gm1b_terrain_strain then gm1b_terrain_stress on one stream. */
GM1B_API int32_t gm1b_terrain_sgs_stress(int32_t ni, int32_t nj, int32_t nk,
                                         const gm1b_terrain_stress_arrays *arrays, float dx, float dy, float dz,
                                         float dt, void *stream);

/* As gm1b_flat_scalar_turbulence_arrays with the terrain column metrics of
 * gm1b_terrain_stress_arrays (gz, rgz, rgzu, rgzv, gx, gxu, gy, gyv) and
 * gm1b_terrain_scalar_turbulence_workspace_words() words of workspace (the
 * x and y fluxes of every scalar). */
typedef struct gm1b_terrain_scalar_turbulence_arrays {
    const float *th0, *tha, *qa, *rho, *rr, *rf, *mh, *mf, *khh, *khv;
    const float *gz, *rgz, *rgzu, *rgzv, *gx, *gxu, *gy, *gyv;
    float *thten, *qten, *workspace;
} gm1b_terrain_scalar_turbulence_arrays;

/* Words of the terrain scalar turbulence's workspace:
 * (numq + 1)*(nk*nj*(ni+1) + nk*(nj+1)*ni). */
GM1B_API int64_t gm1b_terrain_scalar_turbulence_workspace_words(int32_t ni, int32_t nj, int32_t nk, int32_t numq);

/*
 * CM1 turbs on the terrain texts for theta ((th0 - 300) + tha) and moisture
 * rows 0..numq-1 (numq <= 6): the x/y fluxes with their terrain terms, the
 * implicit vertical diffusion with khv, zero surface flux; ADDED into thten
 * and the first numq rows of qten.  nk <= 200.  Replaces
 * cpu_gm1_scalar_turbulence_inplace and its kernels
 * (src/cm1core/cuda_gm1_scalar_turbulence.py:230-430, :453-510).
 */
GM1B_API int32_t gm1b_terrain_scalar_turbulence(int32_t ni, int32_t nj, int32_t nk, int32_t numq,
                                                const gm1b_terrain_scalar_turbulence_arrays *arrays, float dx,
                                                float dy, float dz, float dt, void *stream);

/* tauh/taus (nk, nj+2, ni+2) and tauf (nk+1, nj+2, ni+2) with one
 * horizontal halo, or (profiles = 1) tauh/taus (nk) and tauf (nk+1)
 * columns; u0/v0 (nk); ua/uten1 (nk, nj, ni+1); va/vten1 (nk, nj+1, ni);
 * wa/tha/wten1/thten1 (nk, nj, ni) (wa the w faces 0..nk-1). */
typedef struct gm1b_rayleigh_held_arrays {
    const float *tauh, *taus, *tauf, *u0, *v0, *ua, *va, *wa, *tha;
    float *uten1, *vten1, *wten1, *thten1;
} gm1b_rayleigh_held_arrays;

/*
 * CM1's upper Rayleigh damping (irdamp = 1) held tendencies: uten1 =
 * ((-rdalpha*0.5)*(tauh(i-1)+tauh(i)))*(ua - u0), vten1 the same across j,
 * wten1 = (-rdalpha*tauf)*wa, thten1 = (-rdalpha*taus)*tha.  add_momentum
 * = 0 assigns all four (cm1_rayleigh_held_physical_f32_v1); add_momentum = 1
 * adds the damping into uten1/vten1/wten1 (the held sum uten1 + uten of
 * cuda_cartesian_closure.py:1289-1291) and assigns thten1.  Replaces
 * launch_cuda_rayleigh_held (src/cm1core/cuda_rayleigh_held.py:523).
 */
GM1B_API int32_t gm1b_rayleigh_held(int32_t ni, int32_t nj, int32_t nk, const gm1b_rayleigh_held_arrays *arrays,
                                    int32_t profiles, int32_t add_momentum, float rdalpha, void *stream);

/* dissten (nk+1, nj, ni), pi0 (nk), ppi/thten1 (nk, nj, ni), qa six rows of
 * nk*nj*ni words (qv qc qr qi qs qg). */
typedef struct gm1b_dissipative_heating_arrays {
    const float *dissten, *pi0, *ppi, *qa;
    float *thten1;
} gm1b_dissipative_heating_arrays;

/*
 * CM1's dissipative heating (idiss = 1), ADDED into thten1: per cell
 * (0.5*(dissten(k)+dissten(k+1))) / ((cpdcv*cvm)*(pi0+ppi)) with the moist
 * heat capacity cvm = ((cv + cvv*qv) + cpl*(qc+qr)) + cpi*((qi+qs)+qg).
 * Replaces Eqtset2IdissConsumer.apply (src/cm1core/eqtset2_energy_terms.py:375).
 */
GM1B_API int32_t gm1b_dissipative_heating(int32_t ni, int32_t nj, int32_t nk,
                                          const gm1b_dissipative_heating_arrays *arrays, void *stream);

/* c1/c2/mf/nm (nk+1, nj, ni), pi0/th0 (nk), prs/pp3d/th3d and the cell
 * outputs (nk, nj, ni), q3d (6, nk, nj, ni) in the order qv qc qr qi qs qg,
 * saturation_mask uint8 (nk, nj, ni).  counts (optional, NULL = not
 * written): four uint64 words ADDED to, saturated, liquid, mixed and ice
 * face words. */
typedef struct gm1b_moist_nm_arrays {
    const float *c1, *c2, *mf, *pi0, *th0, *prs, *pp3d, *th3d, *q3d;
    float *nm, *temperature, *qt, *thv, *qvci;
    uint8_t *saturation_mask;
    uint64_t *counts;
} gm1b_moist_nm_arrays;

/*
 * CM1 calcnm, six-species ice-aware branch (liquid at T >= 273.15 K, ice at
 * T <= 233.15 K, a linear blend between): nm on face levels 1..nk-1 (0 at
 * levels 0 and nk) and the cell diagnostics.  Replaces launch_cuda_moist_nm
 * (src/cm1core/cuda_moist_nm.py:542) and its CPU twin cpu_moist_nm_inplace
 * (:292).  ni, nj >= 1, nk >= 2.
 */
GM1B_API int32_t gm1b_moist_nm(int32_t ni, int32_t nj, int32_t nk, const gm1b_moist_nm_arrays *arrays, float dz,
                               void *stream);

/* ------------------------------------------------------------------------
 * CM1 limits: small-step bound, substep count, advective Courant number
 * ---------------------------------------------------------------------- */

/* 0.60*min(dx,dy)/360 in binary64 (misclibs.F:867).  Replaces
 * cm1_acoustic_small_step_limit_s (src/cm1core/gm1_runtime.py:249); returns
 * NaN (message in gm1b_last_error) unless dx, dy are finite and positive. */
GM1B_API double gm1b_acoustic_small_step_limit(double dx, double dy);

/* The nsound CM1 would choose for dt on this grid (misclibs.F:883-885).
 * Replaces cm1_diagnostic_acoustic_substeps (src/cm1core/gm1_runtime.py:284). */
GM1B_API int32_t gm1b_diagnostic_acoustic_substeps(double dt, double dx, double dy, int32_t *nsound);

/* Scalar advective Courant number of one wind vector, binary64
 * (misclibs.F:2747-2765).  Replaces cm1_advective_courant
 * (src/cm1core/gm1_runtime.py:458). */
GM1B_API int32_t gm1b_advective_courant(double dt, double dx, double dy, double dz, double u, double v, double w,
                                        double *out);

/*
 * Domain advective Courant number (CM1 calccflquick) of DEVICE winds u
 * (nk, nj, ni+1), v (nk, nj+1, ni), w (nk+1, nj, ni) with stretching
 * factors uh (ni), vh (nj), mh (nk) and dtdx = 0.5*dt*rdx etc. as binary32.
 * level_keys (nk words, device) receives each level's maximum as an order
 * key (float bits; 0xffffffff = a NaN in that level); *out (device) the
 * maximum over levels, a NaN level never replacing the running maximum.
 * Replaces advective_courant_number / _reduce_courant
 * (src/cm1core/storm_diagnostics.py:249,195).
 */
GM1B_API int32_t gm1b_courant_max(int32_t ni, int32_t nj, int32_t nk, const float *u, const float *v, const float *w,
                                  const float *uh, const float *vh, const float *mh, float dtdx, float dtdy,
                                  float dtdz, uint32_t *level_keys, float *out, void *stream);

/*
 * Fold one step's failure words into a device accumulator of 8 int32
 * (zeroed by the caller once): [0] += Kessler status[0] (cells whose
 * saturation adjustment did not converge), [1] = max(Kessler status[1])
 * (fallout sub-steps), [2] += Kessler status[2] (blown-up fall columns),
 * [3] = the largest *courant (float bits; a NaN is kept), [4] counts the
 * Courant folds, [5] the Kessler folds.  Either input may be NULL.  One
 * single-thread launch, stream-ordered, so a captured step folds its words
 * without a host read; the caller reads acc and refuses as the reference
 * does after a step (satadj non-convergence,
 * src/cm1core/cuda_cartesian_finish.py:638-639; Courant >= 1.5 or not
 * finite, src/cm1core/gm1_runtime.py:518-549).
 */
GM1B_API int32_t gm1b_step_status_fold(const int32_t *kessler_status, const float *courant, int32_t *acc,
                                       void *stream);

/* ------------------------------------------------------------------------
 * Analytic initial state (host, once per run, except the bubble field)
 * ---------------------------------------------------------------------- */

/*
 * Weisman-Klemp base column (CM1 isnd=5) on nk HOST mass heights zh (m,
 * strictly increasing above 0): th0, qv0, pi0, prs0 required; thv0, t0,
 * rh0 optional (NULL = not written).  imoist 0 or 1; iterations = 20 is
 * CM1's count.  Binary32, one operation at a time, on the host.  Replaces
 * weisman_klemp_column_with_iterations
 * (rust/cm1-state/src/storm_initialization.rs:194) and the error cases it
 * refuses (nk < 1, imoist outside {0,1}, zero iterations, non-increasing
 * heights, non-physical column).
 */
GM1B_API int32_t gm1b_wk_base_column(int32_t nk, const float *zh, int32_t imoist, int32_t iterations, float *th0,
                                     float *qv0, float *thv0, float *pi0, float *prs0, float *t0, float *rh0);

/*
 * iwnd=2 quarter-circle base wind on n HOST face heights: u on zu, v on zv
 * (either output may be NULL).  Replaces analytic_shear_u / analytic_shear_v
 * (rust/cm1-state/src/storm_initialization.rs:354,379).
 */
GM1B_API int32_t gm1b_analytic_shear(int32_t n, const float *zu, const float *zv, float *u, float *v);

/*
 * iinit=1 cos^2 warm bubble written into the interior of the DEVICE scalar
 * lane tha: ng = 0 dense (nk, nj, ni); ng = 1 periodic lane (nk+2, nj+2,
 * ni+2); ng = 3 padded lane (nk+2, nj+6, ni+6).  xh (ni), yh (nj), zh (nk)
 * are device mass-point coordinates (m).  Halo words are not written.
 * Replaces build_theta_perturbation for iinit=1
 * (rust/cm1-state/src/initial_perturbation.rs:425,449-466).
 */
GM1B_API int32_t gm1b_theta_bubble(int32_t ni, int32_t nj, int32_t nk, int32_t ng, const float *xh, const float *yh,
                                   const float *zh, float center_x, float center_y, float center_z,
                                   float horizontal_radius, float vertical_radius, float amplitude, float *tha,
                                   void *stream);

/*
 * CM1 vertical coordinates (stretch_z = 0 uniform, stretch_z = 1
 * Wilhelmson-Chen stretching), CM1-indexed float32 profiles: zf, sigmaf, mf,
 * rmf and rdsf hold nk + 3 words, zh, sigma, mh, rmh and rds nk + 2.  rds and
 * rdsf are init_terrain.F:292-298's 1/(sigma(k)-sigma(k-1)) (k = 2..nk) and
 * 1/(sigmaf(k+1)-sigmaf(k)) (k = 1..nk), zero elsewhere.
 */
typedef struct gm1b_stretch_z1_derived {
    int32_t nk1, nk2, nk3; /* layers below str_bot, stretched, above str_top */
    float nominal, c1, c2; /* (dz_bot + dz_top) / 2 and the quadratic's coefficients */
} gm1b_stretch_z1_derived;

typedef struct gm1b_vertical_profiles {
    float *zf, *zh, *sigmaf, *sigma, *mh, *mf, *rmh, *rmf, *rds, *rdsf;
} gm1b_vertical_profiles;

/* derive_stretch_z1 (src/cm1core/cuda_stretch_z1.py:130-201): the segment
 * counts and c1/c2 of a stretch_z = 1 column, with the reference's
 * feasibility refusals (param.F:7814-7914).  Host only. */
GM1B_API int32_t gm1b_stretch_z1_derive(int32_t nk, float dz, float ztop, float str_bot, float str_top, float dz_bot,
                                        float dz_top, gm1b_stretch_z1_derived *out);

/* build_vertical_levels for stretch_z 0 and 1 (src/cm1core/cm1_vertical_grid.py:780-927):
 * every profile into HOST memory plus the Fornberg boundary weights cgs/cgt
 * (fornberg_extrapolation_weights, :422-454).  stretch_z = 0 requires
 * ztop == dz * nk in float32 (param.F:2608) and ignores the stretch words.
 * rds/rdsf may be NULL.  Host only. */
GM1B_API int32_t gm1b_vertical_levels(int32_t stretch_z, int32_t nk, float dz, float ztop, float str_bot,
                                      float str_top, float dz_bot, float dz_top, const gm1b_vertical_profiles *host,
                                      float cgs[3], float cgt[3]);

/* launch_cuda_stretch_z1 (src/cm1core/cuda_stretch_z1.py:418): the same
 * profiles written into DEVICE memory by one device thread on `stream`
 * (rds/rdsf may be NULL).  The parameters are checked on the host first. */
GM1B_API int32_t gm1b_stretch_z1(int32_t nk, float dz, float ztop, float str_bot, float str_top, float dz_bot,
                                 float dz_top, const gm1b_vertical_profiles *device, void *stream);

/*
 * Self-check of the short-path correctly rounded reciprocal the column
 * solves use (the hardware approximate reciprocal refined by one FMA
 * Newton-Raphson step, used for |b| in [2^-125, 2^125]): compares it with
 * CUDA's __frcp_rn on all 2^32 binary32 words on `stream`.  device_counts[0]
 * receives the number of differing words, device_counts[1] the number of
 * words on the short path; device_first_mismatch the smallest differing word
 * (0xffffffff when none).  No host synchronisation.
 */
GM1B_API int32_t gm1b_selftest_reciprocal(unsigned long long *device_counts, uint32_t *device_first_mismatch,
                                          void *stream);

/*
 * Launch profiler.  While enabled, every kernel launch of the library is
 * bracketed by a pair of CUDA events recorded on its own stream (the
 * per-phase device timing of src/cm1core/runtime_profiler.py:1-48, per
 * kernel).  gm1b_profiler_collect waits for the recorded events, returns
 * per-kernel launch counts and total device milliseconds (sorted by total,
 * descending) and clears the record.  Events are created once and reused;
 * no device memory is allocated.
 */
typedef struct gm1b_kernel_stat {
    char name[48];
    int32_t launches;
    double total_ms;
} gm1b_kernel_stat;

GM1B_API int32_t gm1b_profiler_enable(int32_t on);
GM1B_API int32_t gm1b_profiler_collect(gm1b_kernel_stat *out, int32_t capacity, int32_t *count);

/* ------------------------------------------------------------------------
 * Adjoint (reverse-mode) kernels.  The reference has no adjoint; these are
 * the transposes of this library's forward operators, for gradients of a
 * scalar objective J with respect to the state.
 * ---------------------------------------------------------------------- */
typedef struct gm1b_scalar_advection5_adjoint_arrays {
    /* the forward's inputs (padded scalar, mass fluxes, metrics, divx) */
    const float *scalar, *rru, *rrv, *rrw, *c1, *c2, *rr0, *gz, *divx;
    /* dJ/d tendency (nk, nj, ni) in; dJ/d scalar (padded) out */
    const float *tendency_adjoint;
    float *scalar_adjoint;
} gm1b_scalar_advection5_adjoint_arrays;

/*
 * dJ/d scalar of gm1b_scalar_advection5's tendency (the whole-domain
 * operator, lateral_obc != 0) with the mass fluxes held fixed: every padded
 * scalar word receives the sum over the faces whose stencils read it of
 * (face adjoint) * (mass flux) * d(reconstruction)/d(word), plus its
 * divergence and open-side terms.  The WENO-Z weights are differentiated at
 * their epsilon-regularised form (subgradient 0 for |b1 - b3| at b1 = b3
 * and beyond the 1e30 cap), upstrpd by its active limiter branch.
 * Differentiates cpu_scalar_advection5_inplace (src/cm1core/cuda_advection5.py:
 * 440) / cm1_adv5_scalar_tendency_v1 (:669).  Two passes, no atomics: each
 * face writes its six coefficients (face adjoint x mass flux x the
 * reconstruction's derivative at each stencil point) into the workspace
 * (gm1b_scalar_advection5_adjoint_workspace_bytes), then each word gathers
 * the coefficients of the faces that read it.  scalar_adjoint: the padded
 * (nk+2, nj+6, ni+6) dJ/d(carrier word).
 */
GM1B_API size_t gm1b_scalar_advection5_adjoint_workspace_bytes(int32_t ni, int32_t nj, int32_t nk);
GM1B_API int32_t gm1b_scalar_advection5_adjoint(int32_t ni, int32_t nj, int32_t nk,
                                                const gm1b_scalar_advection5_adjoint_arrays *arrays, int32_t nrk,
                                                int32_t wflag, float dx, float dy, float dz, double weps,
                                                uint32_t lateral_obc, void *workspace, void *stream);
/* The same through the all-open carrier: scalar is the COMPACT (nk, nj, ni)
 * scalar (its open-filled carrier, the words gm1b_scalar_carrier_open
 * makes, is read through the fill's index map, never stored),
 * scalar_adjoint the compact dJ/d scalar (the fill's transpose folded into
 * the gather), for
 * the tendency adjoint adjoint_scale * tendency_adjoint.  accumulate
 * (compact, may be NULL, may equal scalar_adjoint) is added to the result;
 * with running_sum (compact, needs accumulate) the result is written bare
 * and running_sum = accumulate + result (the RK stage chain's two outputs). */
GM1B_API int32_t gm1b_scalar_advection5_adjoint_open(int32_t ni, int32_t nj, int32_t nk,
                                                     const gm1b_scalar_advection5_adjoint_arrays *arrays, int32_t nrk,
                                                     int32_t wflag, float dx, float dy, float dz, double weps,
                                                     float adjoint_scale, const float *accumulate, float *running_sum,
                                                     void *workspace, void *stream);
/* The compact (nk, nj, ni) scalar packed into its padded (nk+2, nj+6, ni+6)
 * carrier with the all-open halo fill in one pass: the same words as
 * zeroing, gm1b_pack_scalar and gm1b_open_fill(GM1B_FILL_SCALAR) in turn
 * (cm1_rk_pack_scalar_v1 and bcs, src/cm1core/cuda_sound3_open_boundary.py:
 * 249-335). */
GM1B_API int32_t gm1b_scalar_carrier_open(int32_t ni, int32_t nj, int32_t nk, const float *scalar, float *padded,
                                          void *stream);

/* The transpose of gm1b_open_fill's scalar kind (bcs on open sides,
 * src/cm1core/cuda_sound3_open_boundary.py:249-335), in place on a padded
 * adjoint: each halo word's adjoint folds onto the edge word it copied, the
 * halo words become zero. */
GM1B_API int32_t gm1b_open_fill_scalar_adjoint(int32_t ni, int32_t nj, int32_t nk, float *q, void *stream);

/*
 * One tridiagonal solve per column (columns independent; level k of every
 * column at word k*columns + col): a(k) x(k-1) + b(k) x(k) + c(k) x(k+1) =
 * d(k), a(0) and c(n-1) unused; transposed = 1 solves A^T x = d (the adjoint
 * of the acoustic column's vertically implicit w-pi' solve,
 * cpu_sound3_periodic_stage_inplace, src/cm1core/cuda_sound3_periodic.py:
 * 824-1027: dJ/dd = A^-T dJ/dx).  work: n*columns words.
 */
GM1B_API int32_t gm1b_tridiagonal_solve(int32_t n, size_t columns, const float *a, const float *b, const float *c,
                                        const float *d, float *x, float *work, int32_t transposed, void *stream);

/*
 * Kessler collection in place: autoconversion max(0.001(qc - 0.001), 0) dt
 * and accretion 2.2 qc qr^0.875 dt, limited to the available qc, moved from
 * qc to qr (the first part of the local conversion of
 * cpu_gm1_kessler_local_inplace, src/cm1core/cuda_gm1_kessler_local.py:251).
 * qc, qr >= 0, the reference's own precondition (with qc < 0 the limiter
 * divides 0 by 0).  The adjoint takes the forward's inputs qc, qr and dJ/d(outputs) in gc, gr,
 * and overwrites gc, gr with dJ/d(inputs); it takes the subgradient 0 at
 * the autoconversion switch qc = 0.001 and at qr = 0.
 */
GM1B_API int32_t gm1b_kessler_collection(size_t cells, float *qc, float *qr, float dt, void *stream);
GM1B_API int32_t gm1b_kessler_collection_adjoint(size_t cells, const float *qc, const float *qr, float *gc, float *gr,
                                                 float dt, void *stream);

/*
 * Single-pass saturation adjustment, in place (the equation-set-1 branch of
 * the Kessler operator's _cpu_satadj, src/cm1core/cuda_gm1_kessler_driver.py:
 * 337-428): at the frozen pressure prs and Exner pi0 + pp3d, one step
 * dqv = (qvs - qv) / (1 + L qvs 17.67 243.5 / (cp (T - 29.65)^2)), floored
 * so that qv stays >= 1e-20 and limited to the cloud water; qv += dqv,
 * qc -= dqv, th3d -= dqv L / (cp pi).  All arrays `cells` words.  The adjoint
 * takes the forward's inputs and dJ/d(outputs) in g_th, g_qv, g_qc, and
 * overwrites them with dJ/d(inputs), each limiter differentiated as the
 * branch the binary32 forward took (the saturation switch: the cloud-water
 * limit's subgradient is the unlimited branch's at equality).
 */
GM1B_API int32_t gm1b_satadj1(size_t cells, const float *th0, const float *pi0, const float *pp3d, const float *prs,
                              float *th3d, float *qv, float *qc, void *stream);
GM1B_API int32_t gm1b_satadj1_adjoint(size_t cells, const float *th0, const float *pi0, const float *pp3d,
                                      const float *prs, const float *th3d, const float *qv, const float *qc,
                                      float *g_th, float *g_qv, float *g_qc, void *stream);

/*
 * The cell step of the warm-rain transport model after its transport, in one
 * pass: qc and qr clipped at 0, collection (gm1b_kessler_collection), then
 * satadj1 - the same words as those pieces run in turn.  state and out: four
 * host arrays of device pointers (th3d, qv, qc, qr), cells words each.  The
 * adjoint takes the transported state and dJ/d(out) and writes dJ/d(state);
 * the clip passes the adjoint where the state is >= 0.
 */
GM1B_API int32_t gm1b_warm_rain_cell(size_t cells, const float *th0, const float *pi0, const float *pp3d,
                                     const float *prs, const float *const *state, float *const *out, float dt,
                                     void *stream);
GM1B_API int32_t gm1b_warm_rain_cell_adjoint(size_t cells, const float *th0, const float *pi0, const float *pp3d,
                                             const float *prs, const float *const *state,
                                             const float *const *out_adjoint, float *const *state_adjoint, float dt,
                                             void *stream);

/* ------------------------------------------------------------------------
 * The whole moist RK3 large step behind one entry point.
 *
 * Every array of the composed state, device pointers in this order (the
 * arrays of the step's Python mirror, gm1_b200.moist_step.moist_state_shapes):
 * padded winds u/v (nk+2, nj+6, ni+7 / nj+7, ni+6) and w (nk+3, nj+6, ni+6)
 * with their tendencies, mass fluxes and scratch fluxes; the pressure-lane
 * arrays (nk+2, nj+2, ni+2) and the six column diagnostics (one word each);
 * the radiation histories and boundary profiles; the padded scalars
 * (nk+2, nj+6, ni+6); the mass fields (nk, nj, ni); q3d/qa (6, nk, nj, ni),
 * qheld/moist_adv (3, nk, nj, ni); the face fields (nk+1, nj, ni); the
 * compact winds uc (nk, nj, ni+1), vc (nk, nj+1, ni), wc (nk+1, nj, ni); the
 * base profiles th0/pi0/qv0 (nk); rain (1, nj, ni), prate (nj, ni); ruh
 * (ni), rvh (nj); saturation_mask (uint8, mass); asq (3) and qbudget (10)
 * FP64; and the scratch of moisture species 1 and 2 (each padded scalar,
 * fx, fy, fz, advx, advy, advz, candidate), which lets the three species
 * advect concurrently (species 0 uses the state's own).  The caller owns
 * every array.
 * ---------------------------------------------------------------------- */
typedef struct gm1b_moist_state {
    float *ua, *u3d, *uten, *rru, *va, *v3d, *vten, *rrv, *wa, *w3d, *wten, *rrw, *fz, *fx, *fy;
    float *ppi, *pp3d, *ppx, *ppd, *piadv, *ppterm, *ppten, *thv, *qk, *pk1, *pk2, *mm, *fpk, *divh, *hadvp, *dum3,
        *elim_c, *elim_d;
    float *tri_aa, *tri_bb, *tri_cc, *tri_dd, *tri_pivot, *tri_residual;
    float *radbcw, *radbce, *radbcs, *radbcn, *uh, *vh, *ruf, *rvf, *scalar, *dum8, *theta_padded, *moisture_padded;
    float *th3d, *tha, *thterm, *divergence, *theta_div, *divx, *pp3d_c, *prs, *rho, *rr, *kessler_rr, *thheld, *qpten,
        *qtten, *qvten, *qcten, *theta_adv, *advx, *advy, *advz, *candidate, *temperature, *qt, *thv_c, *qvci,
        *pi0_3d, *th0_3d, *fall_velocity, *ones_mass;
    float *q3d, *qa, *qheld, *moist_adv;
    float *rf, *nm, *defv, *defh, *tke3d, *tkea, *tketen, *tk, *grdscl, *rgrdscl, *lenscl, *dissten, *cme, *ce1,
        *ce2, *csm, *kmh, *kmv, *khh, *khv, *tke_workspace;
    float *uc, *vc, *wc, *th0, *pi0, *qv0, *rain, *prate, *ruh, *rvh;
    uint8_t *saturation_mask;
    double *asq, *qbudget;
    float *moisture_padded_1, *fx_1, *fy_1, *fz_1, *advx_1, *advy_1, *advz_1, *candidate_1;
    float *moisture_padded_2, *fx_2, *fy_2, *fz_2, *advx_2, *advy_2, *advz_2, *candidate_2;
    /* the dry-air mass ledger mass1 (one double; with apmasscon, computed
     * from the state at create when it holds 0, else kept - a restored
     * ledger) */
    double *mass1;
} gm1b_moist_state;

/* The metrics: the 25 terrain metrics of the padded lane (flat: gz = 1,
 * zero slopes) and, for a stretched column, its mh (nk+2) and mf (nk+3)
 * profiles (CM1-indexed) and the padded base density (nk+2, nj+6, ni+6);
 * the last three may be NULL on a uniform column. */
typedef struct gm1b_moist_metrics {
    const float *terrain_msl, *zh, *zf, *mh, *rmh, *mf, *rmf, *c1, *c2, *rho0_3d, *rr0, *rf0, *rrf0, *gz, *rgz, *gzu,
        *rgzu, *gzv, *rgzv, *dzdx, *dzdy, *gx, *gxu, *gy, *gyv;
    const float *mh_profile, *mf_profile, *rho0_padded;
    /* the upper Rayleigh damping (read when the configuration turns it on):
     * the base-state winds u0/v0 (nk) and the damping profiles tauh/taus
     * (nk) and tauf (nk+1) */
    const float *u0, *v0, *tauh, *taus, *tauf;
} gm1b_moist_metrics;

/* dz: the uniform layer depth, or a stretched column's reference dz
 * (rdz = 1/dz).  lateral_sides: CM1's wbc, ebc, sbc, nbc.  stretched = 1
 * selects the flat (terrain_flag=.false.) operator family on the column the
 * metrics describe.  concurrent = 1 runs each RK stage's scalar, boundary and
 * TKE work on side streams (the same words as concurrent = 0). */
typedef struct gm1b_moist_step_config {
    int32_t ni, nj, nk;
    float dx, dy, dz, dt;
    int32_t nsound;
    float alph, kdiv;
    int32_t lateral_sides[4];
    int32_t stretched;
    int32_t concurrent;
    /* the final-RK dry-air mass correction (CM1 apmasscon = 1, the
     * supercell namelist's): between the pre-physics equation of state and
     * the Kessler driver, against the state's mass1 ledger */
    int32_t apmasscon;
    /* the SGS stress and scalar diffusion held tendencies (gettau and
     * turbu/turbv/turbw once per large step, added into the momentum
     * tendencies of every RK stage; turbs of theta and the moisture rows
     * into thheld/qheld before the eqtset 2 composition); stretched columns
     * only.  The handle allocates the stress scratch. */
    int32_t sgs_diffusion;
    /* CM1's upper Rayleigh damping, irdamp = 1 (the held u, v, w and theta
     * tendencies of solve1.F:412-454 at rate rdalpha on the metrics' tau
     * profiles); stretched columns only */
    int32_t rayleigh;
    float rdalpha;
    /* CM1's dissipative heating, idiss = 1 (the TKE closure's dissipation
     * rate into the held theta, solve1.F:917-975) */
    int32_t dissipative_heating;
} gm1b_moist_step_config;

typedef struct gm1b_moist_step gm1b_moist_step;

/*
 * Bind a composed moist step to a device state.  The handle keeps the
 * pointers (the arrays stay the caller's), creates the side streams and
 * events of the concurrent stage tail, and allocates its own small device
 * words: the Kessler workspace (gm1b_kessler_workspace_bytes), the folded
 * status words and the Courant reduction's scratch.  Call with the state's
 * device current.  Replaces the construction of CudaCartesianRuntime
 * (src/cm1core/cuda_cartesian_runtime.py) for this step's phases.
 */
GM1B_API int32_t gm1b_moist_step_create(const gm1b_moist_step_config *config, const gm1b_moist_state *state,
                                        const gm1b_moist_metrics *metrics, gm1b_moist_step **out);

/*
 * One moist RK3 large step on `stream` in the reference's large-step
 * schedule (StepPhase / large_step_schedule, src/cm1core/gm1_runtime.py:
 * 611-627, :1969-2007; CartesianBackend.execute, :2010-2014): closure and
 * held tendencies, three RK stages of pre-acoustic, acoustic, post-acoustic,
 * scalar/moisture, boundaries and TKE, the Kessler transition and solve3;
 * the step's failure words (satadj non-convergence, blown-up fall columns,
 * the advective Courant number of the state entering the step) are folded
 * on the device.  No host synchronisation and no allocation: the step can
 * be captured in a CUDA graph on `stream`.
 */
GM1B_API int32_t gm1b_moist_large_step(gm1b_moist_step *step, void *stream);

/* The folded failure words of every step since creation (or the last
 * reset), after waiting for `stream`: out[0] non-converged satadj cells,
 * out[1] largest fallout sub-step count, out[2] blown-up fall columns,
 * out[3] the largest Courant number (float bits), out[4] Courant samples,
 * out[5] Kessler samples.  Returns GM1B_STATUS_SATADJ (1) or
 * GM1B_STATUS_COURANT (2) when the reference would refuse the run
 * (cuda_cartesian_finish.py:638-639; gm1_runtime.py:518-549), else 0. */
#define GM1B_STATUS_SATADJ 1
#define GM1B_STATUS_COURANT 2
GM1B_API int32_t gm1b_moist_step_status(gm1b_moist_step *step, int32_t *out, int32_t reset, void *stream);

GM1B_API int32_t gm1b_moist_step_destroy(gm1b_moist_step *step);

#ifdef __cplusplus
}
#endif

#endif /* GM1B_H */
