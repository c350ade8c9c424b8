/*
 * qj.h -- C ABI of libqj, the B200 (sm_100a) implementation of quantum-jax's
 * kick-drift-kick Schroedinger-Poisson step.
 *
 * The reference (pmocz/quantum-jax) has no native interface: its boundary is
 * the Python signature of the per-script functions that a jitted fori_loop
 * calls, with every physical constant captured from module globals.  Each
 * entry point below replaces one of those functions; the constants travel in
 * a plan.  Paths are the reference's files.
 *
 * Conventions
 *  - Arrays are C-order [nx][ny][nz] (z fastest), as built by the reference's
 *    meshgrid(..., indexing="ij") (quantum-stars.py:139,145).
 *  - Precision QJ_PLAIN_F64: psi complex128, real fields / particles float64.
 *    Precision QJ_FUSED_F32: psi complex64, real fields / particles float32
 *    (phase arguments, the k=0 mode, mean density and reductions in FP64).
 *  - Particle arrays are [n][3] (x, y, z), like the reference's pos / vel.
 *  - All pointers are device pointers unless stated otherwise.  Every call is
 *    asynchronous on `stream` (a cudaStream_t; NULL = legacy default stream).
 *  - Status: 0 on success, a QJ_ERR_* code otherwise; qj_last_error() gives a
 *    thread-local message.  No call aborts, exits or traps on the device.
 *  - A plan is not safe for concurrent use from several streams; make one
 *    plan per stream.  The plan owns its device workspace and tables.
 */
#ifndef QJ_H
#define QJ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QJ_OK 0
#define QJ_ERR_ARG 1       /* invalid argument / unsupported size */
#define QJ_ERR_CUDA 2      /* a CUDA runtime call failed */
#define QJ_ERR_NONFINITE 3 /* non-finite value detected in the state */
#define QJ_ERR_TIMEOUT 4   /* a bounded device wait gave up */
#define QJ_ERR_ALLOC 5     /* device allocation failed */

#define QJ_PLAIN_F64 0 /* unfused float64 kernels, op for op with the reference */
#define QJ_FUSED_F32 1 /* fused pencil-pass kernels, complex64 bulk */

typedef struct qj_plan qj_plan;

/* Grid: quantum-stars.py:73-80 (nx, ny, nz, Lx, Ly, Lz). */
typedef struct qj_grid {
  int32_t nx, ny, nz;
  double Lx, Ly, Lz;
} qj_grid;

/* Physical constants the reference reads from module globals:
 * m_per_hbar (quantum-stars.py:109), G (:103), rho_bar (:83 or set in main,
 * quantum-gas-bh.py:680-681), b_coeff (:117-125; 0 disables the
 * self-interaction term), cs (quantum-gas-bh.py:74), c_light (:86). */
typedef struct qj_phys {
  double m_per_hbar;
  double G;
  double rho_bar;
  double b_coeff;
  double cs;
  double c_light;
} qj_phys;

/* The scalar part of the stars state dict (quantum-stars.py:434-440):
 * t, a_max, dt_s.  Lives in DEVICE memory; qj_kdk_step updates it in place. */
typedef struct qj_diag {
  double t;
  double a_max;
  double dt_s;
} qj_diag;

/* Create / destroy a plan.  Replaces the module-level set-up of
 * quantum-stars.py:61-157 (grid, k-grid, constants).  Supported lengths per
 * axis: 16, 32, 64, 96, 128, 256, 512; nz must be a multiple of 16.
 * max_particles bounds n_s of later calls (workspace is sized for it). */
int qj_plan_create(qj_plan **plan, const qj_grid *grid, const qj_phys *phys,
                   int precision, int max_particles);
int qj_plan_destroy(qj_plan *plan);
/* A batched plan holds nbox independent boxes of one grid (QJ_FUSED_F32 only;
 * the IC-ensemble form of the step, one script run per box in the reference).
 * Its qj_kdk_step takes psi [nbox][nx][ny][nz], pos / vel [nbox][n_s][3] and
 * nbox qj_diag records; every pass launch covers all boxes.  The other entry
 * points need nbox == 1. */
int qj_plan_create_batched(qj_plan **plan, const qj_grid *grid,
                           const qj_phys *phys, int precision,
                           int max_particles, int nbox);
/* Update rho_bar / b_coeff / G / m_per_hbar / cs of an existing plan. */
int qj_plan_set_phys(qj_plan *plan, const qj_phys *phys);

/* Thread-local message of the last failing call on this thread. */
const char *qj_last_error(void);

/* get_potential(rho) -> V.  quantum-stars.py:189-193 (also gas-bh :159-163,
 * tidal :168-172, cosmo :142-146).  rho, V: real [nx][ny][nz] of the plan's
 * real type.  self_interaction != 0 adds b_coeff * rho (:193). */
int qj_get_potential(qj_plan *plan, const void *rho, void *V,
                     int self_interaction, void *stream);

/* bin_stars(pos) -> rho_s.  quantum-stars.py:212-247 / bin_particles
 * quantum-gas-bh.py:414-449.  masses: per-particle mass array [n] (device,
 * real type) or NULL to use m_s for every particle.  Deterministic: each
 * cell sums its contributions in (particle, corner) order, like the
 * reference's sequential fori_loop. */
int qj_bin_stars(qj_plan *plan, const void *pos, int n, double m_s,
                 const void *masses, void *rho_s, void *stream);

/* get_acceleration(pos, rho) -> (acc [n][3], a_max).  quantum-stars.py:250-288.
 * a_max: device pointer to one double. */
int qj_get_acceleration(qj_plan *plan, const void *pos, int n, const void *rho,
                        void *acc, double *a_max, void *stream);

/* nsteps x compute_step(psi, pos, vel, t, a_max, dt_s), quantum-stars.py:295-330
 * (the body of `update`, :333-351, iterated like fori_loop at :454).
 * psi, pos, vel and diag are updated in place.  n_s may be 0 (no stars).
 * self_interaction as in qj_get_potential.  v_ext: optional static external
 * potential [nx][ny][nz] (real type) added to V at each kick
 * (quantum-tidal.py:191,201); NULL for none. */
int qj_kdk_step(qj_plan *plan, void *psi, void *pos, void *vel, int n_s,
                double m_s, double dt, int nsteps, int self_interaction,
                const void *v_ext, qj_diag *diag, void *stream);

/* nsteps x compute_step(psi, rho, vx, vy, vz, m_bh, pos, vel, t) of
 * quantum-gas-bh.py:537-578: Schroedinger-Poisson + isothermal gas (MUSCL-
 * Hancock, Rusanov; solve_hydro :269-337, apply_grav_accel :255-266) + black
 * holes (CIC with per-particle masses m_bh [n_bh], do_accretion :497-530 of
 * black hole 0).  rho == NULL drops the gas (quantum-bh.py:346-381).
 * sigma_v: velocity floor of the accretion rate (cs in quantum-gas-bh.py:510,
 * sigma in quantum-bh.py:319).  dm_accretion != 0 enables do_accretion.
 * bondi_r_acc_mult > 0 adds the isothermal Bondi gas sink of
 * quantum-fluid-accretion-test.py:454-494 after the hydro and black-hole
 * drift (:534-536), with r_acc = bondi_r_acc_mult * dx.  Cubic grid and box
 * only (as the reference).  Fields are updated in place; t_io (HOST, may be
 * NULL) is advanced by nsteps * dt. */
int qj_kdk_gas_bh_step(qj_plan *plan, void *psi, void *rho, void *vx, void *vy,
                       void *vz, void *m_bh, void *pos, void *vel, int n_bh,
                       double dt, int nsteps, double sigma_v, int dm_accretion,
                       double bondi_r_acc_mult, double *t_io, void *stream);

/* Gradient of the KDK step with respect to psi (particles as a fixed source:
 * optional self-interaction, static V_ext, and rho_s, a given density added to
 * |psi|^2 wherever the step builds its density -- the star density of
 * quantum-stars.py:298-299 / :315-316 with the stars held fixed; NULL for
 * none).  The reference claims differentiability (README.md:7) but has no
 * jax.grad call site; this is the reverse sweep of qj_kdk_step.
 * qj_kdk_forward_ckpt: advances psi by nsteps in chunks of K steps (one
 * qj_kdk_step call each) and copies psi at the start of chunk j into
 * ckpt + j (ckpt: ceil(nsteps / K) complex [nx][ny][nz] arrays).
 * qj_kdk_adjoint: g holds dL/dRe psi_T + i dL/dIm psi_T on entry and
 * dL/dRe psi_0 + i dL/dIm psi_0 on return; it recomputes each chunk from its
 * checkpoint and runs the adjoint kicks (two Poisson solves each) and drifts
 * backwards.  v_ext and rho_s: real [nx][ny][nz] of the plan's real type. */
int qj_kdk_forward_ckpt(qj_plan *plan, void *psi, int nsteps, int K, void *ckpt,
                        double dt, int self_interaction, const void *v_ext,
                        const void *rho_s, void *stream);
int qj_kdk_adjoint(qj_plan *plan, const void *ckpt, void *g, int nsteps, int K,
                   double dt, int self_interaction, const void *v_ext,
                   const void *rho_s, void *stream);

/* nsteps x compute_step(psi, a) of the comoving script, quantum-cosmo.py:169-196:
 * per step dt = compute_dt(a, da) (:149-162, evaluated in float64 on the
 * host), kin_fac and pot_fac (:173-174) scale the drift and kick phases;
 * a += da.  No particles.  a_io: HOST pointer to the scale factor, advanced
 * by nsteps * da on success. */
int qj_kdk_cosmo(qj_plan *plan, void *psi, double *a_io, double da, double H0,
                 double omega_m, double omega_l, int nsteps, void *stream);

/* 3-D FFT of a complex [nx][ny][nz] array with the plan's pencil kernels
 * (direction -1 forward, unnormalised; +1 inverse, scaled by 1/(nx ny nz)),
 * i.e. jnp.fft.fftn / ifftn as called at quantum-stars.py:191-192,307-309.
 * in == out is allowed. */
int qj_fft3d(qj_plan *plan, const void *in, void *out, int direction,
             void *stream);

/* get_potential in single precision that allocates no device memory.  No
 * counterpart in the reference: it exists for callers that must not call
 * cudaMalloc, such as a JAX / XLA FFI handler (XLA reserves most of the device
 * memory up front, and cudaMalloc / cudaFree would also synchronise the device
 * inside XLA's asynchronous schedule) or a host with a fixed memory budget.
 * Same result as qj_get_potential on a QJ_FUSED_F32 plan, without a plan.
 * rho, V: float32 device arrays [nx][ny][nz]; each axis 16, 32 or 64 cells
 * (at most QJ_NOALLOC_MAX_CELLS), nz a multiple of 16; other sizes return
 * QJ_ERR_ARG.  Its scratch is a fixed 2 MiB array held by every GPU that
 * loads libqj until the process exits; the first call on a device (and the
 * first after a cudaDeviceReset, which frees the array) looks up that array's
 * device address, so make that first call before any stream capture.  All
 * calls on a device share the array: calls that overlap on the
 * GPU (unordered streams) race; calls on one stream are safe. */
#define QJ_NOALLOC_MAX_AXIS 64
#define QJ_NOALLOC_MAX_CELLS (64 * 64 * 64)
int qj_get_potential_f32_noalloc(const qj_grid *grid, const qj_phys *phys,
                                 const float *rho, float *V,
                                 int self_interaction, void *stream);

/* Ensembles of uneven boxes (no reference counterpart: the reference runs one
 * box per process).  One batched plan per box size; qj_ensemble_step advances
 * every plan's boxes by nsteps, joined on `stream`, each plan on its own
 * stream.  With use_graph, the `chunk`-step body is captured once into a CUDA
 * graph (recaptured when pointers, sizes or the launch form change) and
 * replayed nsteps / chunk times; a remainder runs directly.  Arrays are
 * indexed by plan: psi[i], pos[i], vel[i] (device), n_s[i], m_s[i], dt[i]
 * (host), diag[i] (device, nbox records).
 * qj_ensemble_set_merge(ens, 1) runs each fused pass of the step as one
 * launch over all plans' boxes instead, whose CTAs claim each box's tiles
 * from a device counter (a small buffer of the ensemble, sized before any
 * capture), when the plans are cubes of distinct sizes among 64, 96 and 128
 * with the default radix plan and tile (tuning fields 10, 11 zero).  The
 * bits are the same; the per-plan streams measured faster, so they are the
 * default (merge 0).  qj_ensemble_merged returns 1 when steps use the single
 * launches, else 0. */
typedef struct qj_ensemble qj_ensemble;
int qj_ensemble_create(qj_ensemble **ens, qj_plan *const *plans, int nplans);
int qj_ensemble_destroy(qj_ensemble *ens);
int qj_ensemble_set_merge(qj_ensemble *ens, int on);
int qj_ensemble_merged(const qj_ensemble *ens);
int qj_ensemble_step(qj_ensemble *ens, void *const *psi, void *const *pos,
                     void *const *vel, const int *n_s, const double *m_s,
                     const double *dt, qj_diag *const *diag, int nsteps,
                     int chunk, int use_graph, void *stream);

/* Bytes of device workspace the plan holds. */
int64_t qj_plan_workspace_bytes(const qj_plan *plan);

/* bh_bondi_step_ambient (quantum-fluid-accretion.py:440-510): fixed-grid sink
 * of radius r_acc_mult dx around x_bh with the ambient density sampled in
 * the shell [max(ann_lo r_acc, r_acc + dx/4), max(ann_hi r_acc, r_lo + dx/2)].
 * rho (the plan's real type) is updated in place.  vx/vy/vz (may be NULL)
 * add the BHL term with the black-hole velocity v_bh.  fmax <= 0: no cap
 * beyond the sink's mass.  out (device, 7 doubles) = dMdt_target, rho_inf,
 * rB, dM_cap, r_acc, M_avail, dM_uncl.  The shell must fit the grid
 * (2 ceil(r_hi / dx) + 3 <= n), else QJ_ERR_ARG. */
int qj_bondi_ambient(qj_plan *plan, void *rho, const void *vx, const void *vy, const void *vz,
                     const double *x_bh, const double *v_bh, double M_bh, double dt,
                     double r_acc_mult, double lam, double fmax, double ann_lo, double ann_hi,
                     double *out, void *stream);

/* compute_step of quantum-fluid-accretion.py (:695-870): kick-drift-kick
 * with a black hole that is placed at the (smoothed) dark-matter peak at
 * t >= bh_inject_t, grows by a tanh seed ramp plus ambient-shell Bondi
 * accretion, moves under a low-pass-filtered force, and gravitates through a
 * Gaussian-softened CIC density; hydro of that script (limited pressure
 * gradient, local c^2 flux); dt_eff = min(dt, hydro CFL) per step.
 * Plain float64 plans only (the reference runs with x64).  The black-hole
 * state lives on the host (state), as the reference's control flow depends
 * on it: each step synchronises the stream.  diag (host, may be NULL)
 * receives the last step's diagnostics. */
typedef struct {
  double t, M_acc, x_bh[3], v_bh[3], placed;
} qj_facc_state;
typedef struct {
  double cs, hydro_cfl;
  int bh_on, bh_grav, bh_move, bh_accretion;
  double bh_init_m, bh_inject_t;
  int ramp_on;
  double ramp_center, ramp_w, r_acc_mult, lam, fmax, ann_lo, ann_hi, k_cut_frac;
  int inject_smooth_on;
  double inject_smooth_kpc, rho_gas;
} qj_facc_params;
typedef struct {
  double dMdt, rho_inf, r_B, dMdt_real, cap_ratio, r_acc_eff, M_bh_eff_out, dt_eff;
} qj_facc_diag;
int qj_fluid_accretion_step(qj_plan *plan, void *psi, void *rho, void *vx, void *vy, void *vz,
                            qj_facc_state *state, const qj_facc_params *params, double dt,
                            int nsteps, qj_facc_diag *diag, void *stream);

/* Hydro CFL step, quantum-fluid-accretion.py:697-701 (constant sound speed
 * cs, cs2_local :248-250): dt_out (device double) = min(dt, cfl dx /
 * max(cs + |v|)). */
int qj_hydro_cfl_dt(qj_plan *plan, const void *vx, const void *vy, const void *vz, double cs,
                    double cfl, double dt, double *dt_out, void *stream);

/* Launch tuning of a plan: QJ_TUNE_N integers.
 *   [0..7]  CTAs per SM of the persistent fused passes, by pass (0 density,
 *           1 forward FFT y, 2 Poisson, 3 inverse FFT y, 4 kick, 5 drift y,
 *           6 drift + density, 7 deposit); 0 = the occupancy maximum.
 *   [8]     CTA slots the passes leave free for the star stream; -1 = 2.
 *   [9]     threads per block of the hydro kernels; 0 = 256.
 *   [10]    FFT radix plan of the passes along axes of length 128 and 256,
 *           a bit mask: bit m = pass m of [0..6] along x or y, bit 8 + m =
 *           pass m along z (the first density build follows bits 6 and 14):
 *           0 = 16 elements per thread (radix 16 x 16 for 256, 16 x 8 for
 *           128), 1 = 8 elements per thread (8 x 8 x 4, and 8 x 4 x 4), twice
 *           the threads per pencil.
 *   [11]    pencil tile of those passes, a bit mask like [10]: 0 = a CTA holds
 *           256 threads' worth of z pencils, or a 16-column tile of x / y
 *           pencils; 1 = half of that (128 threads' worth, 8 columns).
 * [0..9] change launch shapes only: results are bit-identical for every
 * setting.  [10] and [11] change the order of the floating-point work (the
 * transforms' rounding, the grouping of the density's partial sums): results
 * stay within the single-precision bars, not bit for bit.
 * qj_autotune_kdk times qj_kdk_step on a copy of the given state (probe_steps
 * steps per trial; psi/pos/vel are not modified) and keeps the fastest
 * setting in the plan: with QJ_AUTOTUNE_SHAPES in flags it first picks, per
 * pass and orientation, the radix plan and tile ([10], [11]) among the four
 * combinations, timing that pass alone (CUDA events around its launches,
 * unless qj_profile_enable is on, when it times whole steps), then, as
 * without it, the CTA counts [0..8].  No reference counterpart (XLA
 * picks its own launch shapes and FFT plans). */
#define QJ_TUNE_N 12
#define QJ_TUNE_RADIX 10
#define QJ_TUNE_TILE 11
#define QJ_AUTOTUNE_SHAPES 1
int qj_plan_get_tuning(const qj_plan *plan, int32_t *tune, int n);
int qj_plan_set_tuning(qj_plan *plan, const int32_t *tune, int n);
int qj_autotune_kdk(qj_plan *plan, const void *psi, const void *pos, const void *vel, int n_s,
                    double m_s, double dt, int probe_steps, int flags, void *stream);

/* qj_plan_status: waits for the device, then returns QJ_ERR_TIMEOUT (and
 * clears the flag) if a fused pass of this plan gave up a bounded wait for
 * one of its tile copies since the last call, else QJ_OK.  No reference
 * counterpart: the reference's XLA kernels have no device-side waits. */
int qj_plan_status(qj_plan *plan);

/* qj_plan_selftest_wait: exercises the failure report without a fault.  One
 * warp waits, with the fused passes' bounded wait and a limit of limit_ns
 * (1 ms .. 2 s), for an mbarrier that nothing completes; when the wait gives
 * up it sets the plan's error word, so the next qj_plan_status returns
 * QJ_ERR_TIMEOUT (and clears it).  No reference counterpart. */
int qj_plan_selftest_wait(qj_plan *plan, int64_t limit_ns, void *stream);

/* ---- XLA custom-call targets (the JAX binding) ----
 * Inside a jitted JAX program the reference's step (the `update` body that
 * jax.lax.fori_loop runs, quantum-stars.py:333-351, :454) and get_potential
 * (:189-193) become XLA custom calls to these targets.  They use XLA's GPU
 * custom-call convention, status-returning form (custom_call api_version 2;
 * jax.ffi.register_ffi_target(name, capsule, platform="CUDA",
 * api_version=0)): buffers = operands' device pointers, then the results';
 * opaque = the call's backend_config, one of the packed descriptors below.
 *
 * qj_xla_kdk_step_f32: operands psi complex64 [nx][ny][nz], pos float32
 *   [n_s][3], vel float32 [n_s][3], diag float64 [3] (t, a_max, dt_s), then
 *   v_ext float32 [nx][ny][nz] if has_v_ext; results psi, pos, vel, diag
 *   after nsteps steps (qj_kdk_step on a cached QJ_FUSED_F32 plan).  Results
 *   may alias their operands; unaliased operands are copied first.
 * qj_xla_get_potential_f32: operand rho float32 [nx][ny][nz], result V.
 *   Grids of 16 / 32 / 64 cells per axis run allocation-free
 *   (qj_get_potential_f32_noalloc); larger ones on a cached plan.
 * Plans are created on a configuration's first call on a device (outside
 * stream capture) and kept until qj_xla_release_plans().  A failing call
 * reports through the status function set by qj_xla_set_status_fn (the
 * binding passes jaxlib's XlaCustomCallStatusSetFailure; libqj does not link
 * jaxlib) when status is non-null, and always to qj_xla_last_status() (the
 * QJ_* code of the last target call) and qj_last_error(). */
#define QJ_XLA_DESC_VERSION 1
typedef struct qj_xla_kdk_desc {
  int32_t version; /* QJ_XLA_DESC_VERSION */
  int32_t nsteps;
  int32_t n_s;
  int32_t self_interaction;
  int32_t has_v_ext;
  int32_t reserved;
  qj_grid grid;
  qj_phys phys;
  double m_s;
  double dt;
} qj_xla_kdk_desc;
typedef struct qj_xla_poisson_desc {
  int32_t version; /* QJ_XLA_DESC_VERSION */
  int32_t self_interaction;
  qj_grid grid;
  qj_phys phys;
} qj_xla_poisson_desc;
typedef void (*qj_xla_status_fn)(void *status, const char *message, size_t message_len);
void qj_xla_kdk_step_f32(void *stream, void **buffers, const char *opaque, size_t opaque_len,
                         void *status);
void qj_xla_get_potential_f32(void *stream, void **buffers, const char *opaque,
                              size_t opaque_len, void *status);
void qj_xla_set_status_fn(qj_xla_status_fn fn);
int qj_xla_last_status(void);
int qj_xla_release_plans(void);

/* qj_selftest_sincos: sin_cos[2 i], sin_cos[2 i + 1] = sin and cos of
 * theta[i] (device float64 in, device float32 pairs out) by the kick pass's
 * own routine (float64 quadrant reduction, float32 series), so that its
 * accuracy can be tested directly.  No reference counterpart (the reference
 * takes exp(-1j V dt / 2) of a complex64 array, quantum-stars.py:300). */
int qj_selftest_sincos(const double *theta, float *sin_cos, int n, void *stream);

/* Instrumentation (no reference counterpart; used by the benchmark).
 * qj_launch_count: kernels libqj has launched in this process.
 * qj_profile_enable(1) clears and starts per-pass CUDA-event timing;
 * qj_profile_read fills ms[b] / count[b] for buckets b < nbuckets
 * (0 density, 1 forward FFT, 2 Poisson, 3 inverse FFT, 4 kick, 5 drift,
 * 6 drift + density, 7 deposit sort, 8 particle gather / update); it waits
 * for the recorded events. */
int64_t qj_launch_count(void);
int qj_profile_enable(int on);
int qj_profile_read(double *ms, int64_t *count, int nbuckets);

#ifdef __cplusplus
}
#endif

#endif /* QJ_H */
