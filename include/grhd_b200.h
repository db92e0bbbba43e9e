/*
 * grhd_b200.h -- C ABI of the B200 (sm_100a) fixed-background Valencia GRHD
 * operator.
 *
 * The entry points replace the methods of the reference's operator classes
 * (GRDzhadzha Source/Matter/GRHD/FixedBGFArrayBoxFiniteVolume.hpp):
 *
 *   FixedBGLevelDataFiniteVolumeOperator<eos_t, background_t>       :446-614
 *   TimeDependentFixedBGLevelDataFiniteVolumeOperator<eos_t, fac_t> :677-830
 *
 * One call works on one box of a level (one Chombo FArrayBox): the caller
 * owns every array; the library holds only parameters and its own scratch.
 *
 * Storage (the FArrayBox layout of the reference, Chombo Fortran order):
 *   the state array covers the ghosted box  glo = lo - ghost, ghi = hi + ghost,
 *   value(i,j,k,c) = state[c * state_comp_stride
 *                          + (i-glo0) + nx*((j-glo1) + ny*(k-glo2))]
 *   nx = ghi0-glo0+1, ny = ghi1-glo1+1, state_comp_stride >= nx*ny*nz,
 *   components in the order of the reference UserVariables
 *   (Tests/GRHDFixedBGTest/UserVariables.hpp:24-40) counted from c_GRHD_D:
 *     0 D, 1 S1, 2 S2, 3 S3, 4 tau, 5 rho, 6 eps, 7 pressure, 8 v1, 9 v2, 10 v3
 *   so a caller holding a full GRChombo FAB passes &fab(lo, c_GRHD_D).
 * Right-hand sides cover the interior box only (the reference's rhs
 * LevelData has zero ghosts): 5 components D, S1, S2, S3, tau.
 *
 * All pointers are device pointers (cudaMalloc'd or managed).  `stream` is a
 * cudaStream_t passed as void* (NULL = legacy default stream).  Every call is
 * ordered on that stream; calls that return host values (diagnostics, dt,
 * status) synchronise the stream before returning.  A context may be used by
 * one thread at a time; distinct contexts are independent.
 *
 * Error behaviour mirrors the reference's exceptions: a con2prim failure on
 * an RHS, boundary or CFL path (the reference throws std::runtime_error,
 * :48-55, :157-164, :272-279, :383-390) returns GRHD_ERR_RECOVERY and
 * grhd_last_error() gives the failing cell and residual; cfl <= 0 or dx <= 0
 * (std::invalid_argument, :549-550, FixedBGLevelDataDriver.hpp:36-38)
 * returns GRHD_ERR_INVALID_ARG.  After an error the state is unspecified.
 */
#ifndef GRHD_B200_H_
#define GRHD_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GRHD_B200_ABI_VERSION 1

typedef struct grhd_ctx grhd_ctx;

typedef enum grhd_status
{
    GRHD_OK = 0,
    GRHD_ERR_RECOVERY = 1,    /* con2prim failed where the reference throws */
    GRHD_ERR_INVALID_ARG = 2, /* bad argument (cfl, dx, box, pointer)       */
    GRHD_ERR_CUDA = 3,        /* CUDA runtime error                          */
    GRHD_ERR_SETUP = 4        /* initial data could not be constructed       */
} grhd_status;

typedef enum grhd_background_kind
{
    GRHD_BG_KERR_SCHILD = 0, /* Source/Background/KerrSchild.hpp        */
    GRHD_BG_BINARY_PN = 1    /* Source/Background/CircularBinaryPN.hpp  */
} grhd_background_kind;

/* Where a recovery failure happened (the reference's message variants). */
typedef enum grhd_error_where
{
    GRHD_WHERE_NONE = 0,
    GRHD_WHERE_OUTFLOW_SOURCE = 1,    /* boundary fill,  :157-164 */
    GRHD_WHERE_GHOSTED_RECOVERY = 2,  /* ghosted box,    :48-55   */
    GRHD_WHERE_METRIC_SOURCES = 3,    /* sources,        :272-279 */
    GRHD_WHERE_CFL = 4                /* CFL speed,      :383-390 */
} grhd_error_where;

/* Arithmetic of the operator (new; the reference is FP64 throughout).
 * FP64: every quantity in FP64, the reference's algorithm (parity path).
 * MIXED: reconstruction, HLLE, metric and sources in FP32; con2prim (FP64
 * Newton started from the previous stage's pressure), the metric within
 * three gravitational radii of a Kerr-Schild hole, the volume-time source
 * and the conserved state / RK accumulation in FP64. */
typedef enum grhd_precision
{
    GRHD_PRECISION_FP64 = 0,
    GRHD_PRECISION_MIXED = 1
} grhd_precision;

/* Operator parameters: the constructor arguments of the reference operators
 * (:450-464 and :681-700) with the EOS (IdealGasEOS.hpp:13-16), background
 * params_t (KerrSchild.hpp:26-31, CircularBinaryPN.hpp:32-42),
 * AtmosphereOptions (Atmosphere.hpp:16-22) and RecoveryOptions
 * (Valencia.hpp:17-23) flattened in.  grhd_default_params() fills the
 * reference defaults.  Fields marked "new" have no reference counterpart. */
typedef struct grhd_params
{
    int background; /* grhd_background_kind */
    double ks_mass, ks_spin;
    double pn_mass_1, pn_mass_2, pn_separation, pn_angular_velocity,
        pn_phase, pn_time, pn_softening_radius;
    double adiabatic_index;
    double dx;
    double center[3];
    double rho_floor, pressure_floor, max_velocity_squared,
        metric_source_atmosphere_factor;
    int recovery_max_iterations;
    double recovery_tolerance, recovery_pressure_floor,
        recovery_max_velocity_squared;
    double limiter_theta;
    int use_reconstruction, use_static_metric_sources,
        use_metric_volume_time_sources;
    double metric_time_derivative_step;
    double excision_radius; /* new: cells with coordinate radius below this
                               are frozen and get a zero RHS; <= 0 disables */
    double accretion_radius; /* new: > 0 turns on the rest-mass accretion
                                rate through the sphere r < R (see
                                grhd_accretion) */
    int precision;           /* new: grhd_precision */
} grhd_params;

/* One box of the level.  lo/hi: the box's valid cells (inclusive); ghost:
 * ghost width of its storage (>= 2); domain_lo/hi: the non-periodic
 * problem domain.  Ghost cells outside the domain are physical boundaries
 * (outflow); ghost cells inside it are the caller's (exchange). */
typedef struct grhd_box
{
    int lo[3], hi[3];
    int ghost;
    int domain_lo[3], domain_hi[3];
} grhd_box;

/* AtmosphereResetDiagnostics, FArrayBoxFiniteVolume.hpp:78-92.  Every entry
 * point that takes a `diag` adds its counts to it (as the reference's
 * operator += does, :104-110): zero it before the first call. */
typedef struct grhd_diagnostics
{
    long long num_cells, num_failed_recoveries, num_floored_primitives,
        num_conserved_resets;
} grhd_diagnostics;

typedef struct grhd_error
{
    int status;    /* grhd_status of the failing call */
    int where;     /* grhd_error_where */
    int cell[3];   /* failing cell (level index space) */
    double residual;
    char message[256];
} grhd_error;

/* ---- context ---- */
void grhd_default_params(grhd_params *params);
/* Creates a context for `params` on the current CUDA device.  Replaces the
 * operator constructor (:450-464 / :681-700). */
int grhd_create(const grhd_params *params, grhd_ctx **out);
void grhd_destroy(grhd_ctx *ctx);
int grhd_last_error(const grhd_ctx *ctx, grhd_error *out);
const char *grhd_status_string(int status);
int grhd_abi_version(void);

/* ---- operator methods ---- */

/* compute_rhs(rhs, state, domain, inverse_dx_U[, time]), :468-477 / :702-720.
 * Fills the physical ghosts of `state` (conserved and primitive components),
 * then writes the flux-divergence + static-metric (+ volume-time) RHS over
 * the interior.  `time` is ignored by the static Kerr-Schild background. */
int grhd_compute_rhs(grhd_ctx *ctx, double *rhs, int64_t rhs_comp_stride,
                     double *state, int64_t state_comp_stride,
                     const grhd_box *box, const double inverse_dx[3],
                     double time, void *stream);

/* grhd_compute_rhs with no device allocation: the same RHS, its scratch
 * taken from one fixed device array (about 5 MiB) instead of buffers the
 * context grows with cudaMalloc.  No counterpart in the reference.  For
 * hosts that cannot let a library allocate device memory mid-run (their
 * pool holds the memory; cudaFree would wait for the whole device).
 * Limits: at most 65536 ghosted and 32768 interior cells (e.g. a 32^3 box
 * with 2 ghosts); larger boxes return GRHD_ERR_INVALID_ARG.  The first
 * call on each device looks the array up (cudaGetSymbolAddress with that
 * device current) and caches its address for the life of the process:
 * make that first call before any stream capture begins on the device,
 * and make no call after a reset of the device (cudaDeviceReset), which
 * leaves the cached address stale.  All calls on a device share the
 * array, so calls that overlap in time there (other streams, threads or
 * contexts) race: issue them one after another.  Like grhd_compute_rhs,
 * the call synchronizes `stream` to read the status word, so it cannot be
 * captured in a CUDA graph.  Its kernels
 * count in the context's launch counter but not in the per-kernel
 * profile (grhd_profile_read). */
int grhd_compute_rhs_static(grhd_ctx *ctx, double *rhs,
                            int64_t rhs_comp_stride, double *state,
                            int64_t state_comp_stride, const grhd_box *box,
                            const double inverse_dx[3], double time,
                            void *stream);

/* Test support for grhd_compute_rhs_static (no counterpart in the
 * reference): sets every word of its fixed array on the context's device
 * to `value` and synchronizes `stream`.  Lets a test show that the RHS
 * does not depend on what earlier calls left in the array. */
int grhd_static_scratch_fill(grhd_ctx *ctx, double value, void *stream);

/* recover_primitives(state[, time]) -> AtmosphereResetDiagnostics,
 * :506-520 / :728-743.  `diag` may be NULL. */
int grhd_recover_primitives(grhd_ctx *ctx, double *state,
                            int64_t state_comp_stride, const grhd_box *box,
                            double time, grhd_diagnostics *diag, void *stream);

/* update_conserved(state, rhs, dt[, recovery_time], recover), :522-533 /
 * :745-757.  `diag` may be NULL. */
int grhd_update_conserved(grhd_ctx *ctx, double *state,
                          int64_t state_comp_stride, const double *rhs,
                          int64_t rhs_comp_stride, const grhd_box *box,
                          double dt, double recovery_time, int recover,
                          grhd_diagnostics *diag, void *stream);

/* compute_max_inverse_dt(state, domain_box, inverse_dx_U[, time]),
 * :535-542 / :759-767. */
int grhd_compute_max_inverse_dt(grhd_ctx *ctx, const double *state,
                                int64_t state_comp_stride,
                                const grhd_box *box,
                                const double inverse_dx[3], double time,
                                double *out, void *stream);

/* compute_stable_dt(state, domain_box, inverse_dx_U, cfl[, time]),
 * :544-555 / :769-780. */
int grhd_compute_stable_dt(grhd_ctx *ctx, const double *state,
                           int64_t state_comp_stride, const grhd_box *box,
                           const double inverse_dx[3], double cfl,
                           double time, double *out, void *stream);

/* advance_ssprk2(state, domain, inverse_dx_U, [time,] dt), :563-589 /
 * :782-809.  `diag` (may be NULL) accumulates the recovery counts of both
 * post-update recoveries. */
int grhd_advance_ssprk2(grhd_ctx *ctx, double *state,
                        int64_t state_comp_stride, const grhd_box *box,
                        const double inverse_dx[3], double time, double dt,
                        grhd_diagnostics *diag, void *stream);

/* advance_ssprk2 (:563-589 / :782-809) cut at its two RHS evaluations, for
 * a level of several boxes or ranks whose ghosts the caller exchanges
 * before each stage (the reference's compute_rhs exchanges inside):
 *   stage 1: stage_state = state + dt L(state), recovered at time + dt;
 *   stage 2: state = (state + stage_state + dt L(stage_state)) / 2
 *            (combine_ssprk2_conserved_state), recovered.
 * state and stage_state are ghosted states of the same box. */
int grhd_ssprk2_stage(grhd_ctx *ctx, int stage, double *state,
                      int64_t state_comp_stride, double *stage_state,
                      int64_t stage_comp_stride, const grhd_box *box,
                      const double inverse_dx[3], double time, double dt,
                      grhd_diagnostics *diag, void *stream);

/* New (no reference counterpart; the reference integrates with SSPRK2
 * only): classic four-stage RK4 with the reference's post-update recovery
 * after every stage, stage times t, t+dt/2, t+dt/2, t+dt. */
int grhd_advance_rk4(grhd_ctx *ctx, double *state, int64_t state_comp_stride,
                     const grhd_box *box, const double inverse_dx[3],
                     double time, double dt, grhd_diagnostics *diag,
                     void *stream);

/* New: one RK4 step whose dt comes from the CFL condition, as a driver's
 * compute_stable_dt + advance pair does (dt = min(cfl / max_inverse_dt,
 * max_dt); max_dt <= 0 means no cap).  *max_inverse_dt is in/out: pass the
 * value this call returned for the same, unmodified state (or <= 0 to have
 * it computed from `state` first); on return it holds the max inverse dt
 * of the new state, computed inside the step's last stage.  *dt_used (may
 * be NULL) receives the step taken. */
int grhd_advance_rk4_cfl(grhd_ctx *ctx, double *state,
                         int64_t state_comp_stride, const grhd_box *box,
                         const double inverse_dx[3], double time, double cfl,
                         double max_dt, double *max_inverse_dt,
                         double *dt_used, grhd_diagnostics *diag,
                         void *stream);

/* New: `steps` calls of grhd_advance_rk4_cfl in one (each step's dt from
 * the CFL speed of its input state, capped by max_dt; *max_inverse_dt in
 * and out as there), for a driver that advances several steps between
 * looks at the state: the last stage of each step also does the per-cell
 * pass (con2prim, sources) of the next step's first RHS, which a separate
 * call has to redo.  time_out (may be NULL) receives the time reached;
 * `diag` (may be NULL) the counts of every recovery of every step. */
int grhd_advance_rk4_cfl_steps(grhd_ctx *ctx, double *state,
                               int64_t state_comp_stride,
                               const grhd_box *box,
                               const double inverse_dx[3], double time,
                               double cfl, double max_dt, int steps,
                               double *max_inverse_dt, double *time_out,
                               grhd_diagnostics *diag, void *stream);

/* New: grhd_advance_rk4_cfl of a state held in HOST memory (host_state:
 * the whole-domain box's 11 components at host_state + c * stride; pinned
 * memory copies fastest).  The call copies to the device what the step
 * reads -- the 5 conserved components of every cell, the primitive
 * components of the z planes that hold excised cells, and in mixed
 * precision the pressure -- runs the step there (the same kernels as
 * grhd_advance_rk4_cfl, same results bit for bit) and copies all 11
 * components back; the other primitive components on input are ignored.
 * h2d_bytes / d2h_bytes (may be NULL) receive the bytes moved each way.
 * The device copy of the state lives in the context.  Synchronous.
 * With *max_inverse_dt > 0 (the previous call's value) and no accretion
 * sphere, the step runs as a wavefront over z chunks of the box on the
 * given stream and two streams of the context, copies in and out
 * overlapping the computation; otherwise the state is copied in, stepped
 * and copied back in turn.  On a recovery failure every copy has finished
 * when the call returns; in the wavefront the chunks already copied back
 * then hold the new state. */
int grhd_advance_rk4_cfl_host(grhd_ctx *ctx, double *host_state,
                              int64_t state_comp_stride,
                              const grhd_box *box,
                              const double inverse_dx[3], double time,
                              double cfl, double max_dt,
                              double *max_inverse_dt, double *dt_used,
                              grhd_diagnostics *diag, long long *h2d_bytes,
                              long long *d2h_bytes, void *stream);

/* ---- pointwise kernels for verification ---- */

/* ADM background vars at n points (xyz[3n], positions relative to the
 * operator centre) at operator time `time`, laid out per point as
 * gamma[9], K_tensor[9], K, lapse, shift[3], d1_gamma[27] ([i][j][k] =
 * d_k gamma_ij), d1_lapse[3], d1_shift[9] ([i][j] = d_j shift^i): 64
 * doubles.  Same quantities as KerrSchild/CircularBinaryPN::
 * compute_metric_background (KerrSchild.hpp:64-166,
 * CircularBinaryPN.hpp:70-189).  Device pointers. */
int grhd_eval_background(grhd_ctx *ctx, int64_t n, const double *xyz,
                         double time, double *out, void *stream);

/* recover_primitive (Valencia.hpp:116-228) at n points: cons[5n] (D,S,tau),
 * gUU[9n]; writes prim[6n] (rho,eps,p,v), ok[n], iterations[n],
 * residual[n].  Device pointers. */
int grhd_eval_con2prim(grhd_ctx *ctx, int64_t n, const double *cons,
                       const double *gUU, double *prim, int *ok,
                       int *iterations, double *residual, void *stream);

/* The face pass's z-march length (planes per block) for an nx x ny x nz
 * interior on a device with `resident_blocks` face blocks resident at once
 * (SMs x blocks per SM): of 32, 16, 8, 6 and 4 planes, the one whose blocks
 * list-scheduled in launch order finish first, a block costing its planes
 * plus two lead-in planes.  The kernels choose it this way whenever their
 * caller gives no z-march length; the RHS does not depend on it.  Host
 * only (no device call).  New (the reference has no face kernel). */
int grhd_face_zchunk(int nx, int ny, int nz, int resident_blocks,
                     int *zchunk);

/* The FP64 division, reciprocal, square root and reciprocal square root
 * the kernels compute with, at n points: out[4n] = (a/b, 1/b, sqrt(a),
 * 1/sqrt(a)) per point (about one ulp from IEEE for normal operands and
 * results, and 0 for the square root; a zero divisor or an overflowing
 * quotient gives NaN).  New (the reference
 * uses IEEE operations).  Device pointers. */
int grhd_eval_arith(grhd_ctx *ctx, int64_t n, const double *a,
                    const double *b, double *out, void *stream);

/* ---- initial data (setup, not part of a step) ---- */

/* FixedBGTorusConfig, Source/Matter/GRHD/FixedBGTorus.hpp:20-34 */
typedef struct grhd_torus_config
{
    double total_mass, inner_radius, pressure_max_radius, rho_peak,
        max_velocity_squared, radial_derivative_fraction,
        radial_derivative_min_step, angular_momentum_min_factor,
        angular_momentum_max_factor;
    int angular_momentum_samples, angular_momentum_bisection_iterations;
    double angular_momentum_tolerance;
} grhd_torus_config;

/* FixedBGTorusParameters, FixedBGTorus.hpp:36-42 */
typedef struct grhd_torus_params
{
    double ell, surface_potential, polytropic_constant, max_enthalpy;
} grhd_torus_params;

void grhd_default_torus_config(grhd_torus_config *config);

/* make_fixed_bg_torus_parameters + fill_fixed_bg_torus_level_data
 * (FixedBGTorus.hpp:291-409) on the device: the angular-momentum solve, the
 * maximum enthalpy over the box interior and the primitive + conserved fill
 * of the whole ghosted box, with the operator's EOS, background (at `time`)
 * and atmosphere.  `out` may be NULL.  Returns GRHD_ERR_SETUP when the
 * torus has no pressure-supported region. */
int grhd_torus_initial_data(grhd_ctx *ctx, double *state,
                            int64_t state_comp_stride, const grhd_box *box,
                            const grhd_torus_config *config, double time,
                            grhd_torus_params *out, void *stream);

/* MichelConfig of Tests/GRHDLevelDataMichelAccretion (:32-45); the EOS
 * index is the operator's.  The operator's background must be the
 * Kerr-Schild hole of the same mass with zero spin. */
typedef struct grhd_michel_config
{
    double mass, sonic_radius, sonic_density, atmosphere_radius,
        root_tolerance;
} grhd_michel_config;

/* fill_michel_state (GRHDLevelDataMichelAccretion.cpp:312-372) on the
 * device: analytic Michel primitives outside atmosphere_radius (Bernoulli
 * root solve per cell), atmosphere inside, floors, conserved variables. */
int grhd_michel_initial_data(grhd_ctx *ctx, double *state,
                             int64_t state_comp_stride, const grhd_box *box,
                             const grhd_michel_config *config, void *stream);

/* New: rho *= 1 + amplitude * u with u uniform in [-1, 1) from a
 * counter-based hash of (seed, cell); pressure and velocity kept, eps and
 * the conserved variables recomputed (whole ghosted box). */
int grhd_perturb_density(grhd_ctx *ctx, double *state,
                         int64_t state_comp_stride, const grhd_box *box,
                         double amplitude, uint64_t seed, double time,
                         void *stream);

/* ---- accretion rate (new) ---- */

/* With params.accretion_radius = R > 0 every RHS evaluation also computes
 * the rest-mass accretion rate through the voxelised sphere r < R,
 *   Mdot = - sum over the faces between a cell inside and a cell outside
 *          sqrt(det gamma_face) F_D . n_out dx^2,
 * from the scheme's own HLLE face fluxes (so Mdot is the discrete rest-mass
 * budget of the sphere), and the integrators accumulate its time integral
 * with their stage weights (RK4: dt/6 (1,2,2,1); SSPRK2: dt/2, dt/2).
 * Reads Mdot of the last RHS evaluation and the integral (either may be
 * NULL) and, with reset != 0, zeroes the integral.  Synchronous. */
int grhd_accretion(grhd_ctx *ctx, double *mdot_last, double *integral,
                   int reset);

/* ---- instrumentation ---- */

/* Kernel classes timed by the profiler. */
typedef enum grhd_kernel_class
{
    GRHD_K_GHOSTS = 0, /* physical ghost fill                         */
    GRHD_K_CELLS = 1,  /* per-cell con2prim + sources                 */
    GRHD_K_FACES = 2,  /* face fluxes + divergence                    */
    GRHD_K_STAGE = 3,  /* update / RK stage / recovery                */
    GRHD_K_CFL = 4,    /* max inverse dt reduction                    */
    GRHD_K_NUM_CLASSES = 5
} grhd_kernel_class;

/* Enables (1) or disables (0) CUDA-event timing of every kernel the
 * context launches, on the stream it is launched on. */
int grhd_profile_enable(grhd_ctx *ctx, int enable);
/* Synchronises the recorded events and returns, per kernel class, the
 * summed device time in ms and the number of launches since the last
 * read; then clears them. */
int grhd_profile_read(grhd_ctx *ctx, double ms[GRHD_K_NUM_CLASSES],
                      long long launches[GRHD_K_NUM_CLASSES]);
/* Total number of kernels this context has launched. */
long long grhd_launch_count(const grhd_ctx *ctx);

/* ---- binary-PN disk driver source terms ----
 * The source terms the reference's production driver adds to the operator
 * (Examples/GRHDLevelDataBinaryPNKITPDisk/
 * Main_GRHDLevelDataBinaryPNKITPDisk.cpp): its SimulationConfig fields
 * (:63, :67-71).  They need the binary-PN operator (body masses and orbit
 * from its params at the given operator time). */
typedef struct grhd_kitp_config
{
    double alpha_viscosity, viscosity_beta, rho_floor, sink_size, sink_rate,
        sink_shape;
} grhd_kitp_config;

void grhd_default_kitp_config(grhd_kitp_config *config);
/* add_kitp_viscous_rhs (:772-806): rhs (interior, 5 components) -= the
 * central difference in x and y of the alpha-viscosity stress flux
 * (viscous_flux_for_cell, :700-770) built from the state's stored
 * primitives; neighbours clamped to the problem domain (:664-674). */
int grhd_kitp_viscous_rhs(grhd_ctx *ctx, double *rhs, int64_t rhs_comp_stride,
                          const double *state, int64_t state_comp_stride,
                          const grhd_box *box, const grhd_kitp_config *config,
                          double time, void *stream);
/* add_kitp_sink_rhs (:567-610): rhs -= rate * conserved where the stored
 * density is above 10 x the atmosphere floor. */
int grhd_kitp_sink_rhs(grhd_ctx *ctx, double *rhs, int64_t rhs_comp_stride,
                       const double *state, int64_t state_comp_stride,
                       const grhd_box *box, const grhd_kitp_config *config,
                       double time, void *stream);
/* apply_kitp_sink_decay (:612-662): conserved *= exp(-rate dt) with the
 * bodies at operator time `time` (the driver passes the step's mid time,
 * :874). */
int grhd_kitp_sink_decay(grhd_ctx *ctx, double *state,
                         int64_t state_comp_stride, const grhd_box *box,
                         const grhd_kitp_config *config, double time,
                         double dt, void *stream);

/* advance_kitp_ssprk2 (:842-876), the disk driver's step, on one box
 * covering the domain: SSPRK2 whose RHS is the operator's plus the viscous
 * stress divergence (the sink term enters as the decay, not the RHS), the
 * stage recovered at time + dt, the combination, the sink decay at
 * time + dt/2, the recovery at time + dt.  FP64; needs the binary PN
 * background.  `diag` (may be NULL) accumulates both recoveries. */
int grhd_kitp_advance_ssprk2(grhd_ctx *ctx, double *state,
                             int64_t state_comp_stride, const grhd_box *box,
                             const double inverse_dx[3],
                             const grhd_kitp_config *config, double time,
                             double dt, grhd_diagnostics *diag, void *stream);

/* ---- example drivers' diagnostics and checkpoints ---- */

/* compute_diagnostics of the example drivers
 * (Examples/GRHDLevelDataKerrSchildDisk/Main_GRHDLevelDataKerrSchildDisk.cpp:
 * 223-290): out = mass, disk_mass (cells denser than 10 x the atmosphere
 * floor), tau (proper-volume sums of D and tau), max rho, max pressure,
 * max |v|, max W over the box interior, from the stored primitives.
 * Synchronous. */
int grhd_disk_diagnostics(grhd_ctx *ctx, const double *state,
                          int64_t state_comp_stride, const grhd_box *box,
                          double time, double out[7], void *stream);

/* LevelData<FArrayBox>::exchange() of one level on the device (the
 * reference calls it before every RHS, FixedBGFArrayBoxFiniteVolume.hpp:
 * 322-363): every box's ghost cells inside the (non-periodic) problem
 * domain receive all 11 components from the box whose interior holds
 * them.  boxes / states / strides: the `count` boxes of the level (a
 * disjoint layout sharing one domain) and their device states.  Ghosts
 * outside the domain are left to compute_rhs's outflow fill.  Ordered on
 * `stream`; err (may be NULL) receives a message on error. */
int grhd_level_exchange(const grhd_box *boxes, double *const *states,
                        const int64_t *state_comp_strides, int count,
                        char *err, int err_cap, void *stream);
/* The same for states of `ncomp` components (1..256), e.g. the
 * GRHD_CCZ4_NUM_VARS of the operator on CCZ4-stored geometry, whose
 * geometry the exchange must move as well. */
int grhd_level_exchange_components(const grhd_box *boxes,
                                   double *const *states,
                                   const int64_t *state_comp_strides,
                                   int count, int ncomp, char *err,
                                   int err_cap, void *stream);

/* ---- The operator on CCZ4-stored geometry ----
 * LevelDataFiniteVolumeOperator (Source/Matter/GRHD/FArrayBoxFiniteVolume.hpp:
 * 1215-1364): the same Valencia operator for a metric that the grid holds
 * (dynamical-spacetime coupling).  The state has GRHD_CCZ4_NUM_VARS
 * components of state_comp_stride doubles each: GRChombo's 25 CCZ4
 * variables (chi, h11 h12 h13 h22 h23 h33, K, A11 A12 A13 A22 A23 A33,
 * Theta, Gamma1..3, lapse, shift1..3, B1..3), then the 11 GRHD components
 * in the order of the fixed-background state (Tests/GRHDFixedBGTest/
 * UserVariables.hpp:24-40).  Geometry per cell: gamma = h / chi,
 * gamma^-1 = chi h^-1, K_ij = A_ij / chi + gamma_ij K / 3, lapse, shift
 * (load_ccz4_geometry, :168-192); the sources take their metric
 * derivatives as finite differences of it (:219-427).  FP64 whatever the
 * context's precision; the context's background, dx, centre, excision and
 * accretion settings do not apply.  Physical ghosts copy the conserved
 * variables and chi, h, lapse, shift of their source cell (:430-519). */
#define GRHD_CCZ4_NUM_VARS 36
#define GRHD_CCZ4_GRHD_OFFSET 25

/* compute_rhs (:1232-1240): rhs (5 comps over the interior) = flux
 * divergence + sources. */
int grhd_ccz4_compute_rhs(grhd_ctx *ctx, double *rhs, int64_t rhs_comp_stride,
                          double *state, int64_t state_comp_stride,
                          const grhd_box *box, const double inverse_dx[3],
                          void *stream);
/* recover_primitives (:1272-1285). */
int grhd_ccz4_recover_primitives(grhd_ctx *ctx, double *state,
                                 int64_t state_comp_stride,
                                 const grhd_box *box, grhd_diagnostics *diag,
                                 void *stream);
/* update_conserved (:1288-1299). */
int grhd_ccz4_update_conserved(grhd_ctx *ctx, double *state,
                               int64_t state_comp_stride, const double *rhs,
                               int64_t rhs_comp_stride, const grhd_box *box,
                               double dt, int recover, grhd_diagnostics *diag,
                               void *stream);
/* compute_max_inverse_dt (:1301-1307). */
int grhd_ccz4_compute_max_inverse_dt(grhd_ctx *ctx, const double *state,
                                     int64_t state_comp_stride,
                                     const grhd_box *box,
                                     const double inverse_dx[3], double *out,
                                     void *stream);
/* advance_ssprk2 (:1323-1348) cut at its two RHS evaluations, for a level
 * of several boxes or ranks whose ghosts (all 36 components) the caller
 * exchanges before each stage, as grhd_ssprk2_stage for the fixed
 * background: stage 1 copies the state into stage_state and adds dt L(state)
 * (recovered); stage 2 sets state = (state + stage_state + dt
 * L(stage_state)) / 2 (recovered). */
int grhd_ccz4_ssprk2_stage(grhd_ctx *ctx, int stage, double *state,
                           int64_t state_comp_stride, double *stage_state,
                           int64_t stage_comp_stride, const grhd_box *box,
                           const double inverse_dx[3], double dt,
                           grhd_diagnostics *diag, void *stream);
/* advance_ssprk2 (:1323-1348); the box must be the whole domain. */
int grhd_ccz4_advance_ssprk2(grhd_ctx *ctx, double *state,
                             int64_t state_comp_stride, const grhd_box *box,
                             const double inverse_dx[3], double dt,
                             grhd_diagnostics *diag, void *stream);

/* The halo message of a level split over ranks (LevelData::exchange()
 * across MPI ranks in the reference): the 11 components of the cells
 * [lo, hi] (inside the ghosted box) into a packed device buffer laid out
 * [component][k][j][i] (pack != 0), or from it into the state (pack == 0).
 * Ordered on `stream`. */
int grhd_region_copy(int pack, double *state, int64_t state_comp_stride,
                     const grhd_box *box, const int lo[3], const int hi[3],
                     double *buffer, void *stream);
/* The same for states of `ncomp` components (1..256); the buffer holds
 * ncomp x cells values. */
int grhd_region_copy_components(int pack, double *state,
                                int64_t state_comp_stride,
                                const grhd_box *box, const int lo[3],
                                const int hi[3], int ncomp, double *buffer,
                                void *stream);

/* The binary disk drivers' Keplerian disk (kitp_primitive +
 * fill_kitp_level_data, Main_GRHDLevelDataBinaryPNKITPDisk.cpp:398-555),
 * the initial data of the benchmark's binary-disk configuration: the
 * SimulationConfig disk settings (:56-61) and, new, azimuthal density
 * modes m = 1..4 (surface density times 1 + sum_m A_m cos(m phi + phase_m)).
 * The operator's background must be the binary PN one; its binary
 * (masses, separation, orbital frequency, phase, time, softening) and
 * atmosphere floors are the disk's. */
typedef struct grhd_kitp_disk_config
{
    double mach, aspect_ratio, cavity_radius_factor, cavity_delta,
        outer_cutoff_radius, rho_peak;
    double mode_amplitude[4], mode_phase[4];
} grhd_kitp_disk_config;
/* The driver's defaults (mach 10, H/R 0.1, cavity 2.5 separations with
 * floor 1e-5, no outer cut-off, rho_peak 4e-5), no modes. */
void grhd_default_kitp_disk_config(grhd_kitp_disk_config *config);
/* Primitives and conserved variables over the ghosted box at `time`. */
int grhd_kitp_disk_initial_data(grhd_ctx *ctx, double *state,
                                int64_t state_comp_stride,
                                const grhd_box *box,
                                const grhd_kitp_disk_config *config,
                                double time, void *stream);

/* The header of a KITPCHK1 checkpoint (write_checkpoint /
 * read_checkpoint_header, Examples/GRHDLevelDataBinaryPNKITPDisk/
 * Main_GRHDLevelDataBinaryPNKITPDisk.cpp:1289-1505).  num_components is
 * the driver's NUM_VARS (its GRHD components are the last 11, after the
 * CCZ4 slots, which the writer fills with zeros and the reader ignores). */
typedef struct grhd_checkpoint_header
{
    int num_components, num_cells, num_z_cells, num_ghosts, steps,
        frame_index;
    double time, next_output_time, next_checkpoint_time;
    long long recovery_totals[4]; /* cells, failed, floored, resets */
    double diagnostics[7];        /* as grhd_disk_diagnostics */
    long long diagnostic_counts[3];
} grhd_checkpoint_header;

/* Writes the device state (11 components over the ghosted box, which must
 * be the checkpoint's domain num_cells^2 x num_z_cells grown by
 * num_ghosts) as a KITPCHK1 file the reference driver restarts from;
 * `signature` is the driver's config_signature (:1203-1223).  On error
 * err (err_cap bytes, may be NULL) receives the reference's message. */
int grhd_checkpoint_write(const char *path,
                          const grhd_checkpoint_header *header,
                          const char *signature, const double *state,
                          int64_t state_comp_stride, const grhd_box *box,
                          char *err, int err_cap, void *stream);
/* Reads a KITPCHK1 file: the header, and (state non-NULL) the GRHD
 * components into the device state; expected_signature (may be NULL)
 * must equal the file's. */
int grhd_checkpoint_read(const char *path, grhd_checkpoint_header *header,
                         const char *expected_signature, double *state,
                         int64_t state_comp_stride, const grhd_box *box,
                         char *err, int err_cap, void *stream);

/* ---- batched ensemble (new; no reference counterpart) ----
 * Many independent single-box problems on Kerr-Schild backgrounds, of any
 * sizes, spins, EOS and floors, advanced together: every call runs `steps`
 * classic RK4 steps of every member (the grhd_advance_rk4_cfl step: dt =
 * min(cfl / max inverse dt, max_dt) per member, post-stage recovery,
 * excision, accretion rate) in ONE persistent kernel launch whose phases
 * (ghost fill, face pass, stage) hand out the work items of all members
 * between grid-wide barriers.  The launch can be replayed from a CUDA
 * graph.  Each member's arithmetic is that of the single-box entry points
 * (FP64 members reproduce grhd_advance_rk4_cfl to rounding, 1e-13 of the
 * state's scale).  The ensemble runs on its own stream, ordered after and
 * before `stream`. */
typedef struct grhd_ensemble grhd_ensemble;

typedef struct grhd_ensemble_member
{
    grhd_params params; /* Kerr-Schild; the same precision for all members */
    grhd_box box;       /* the member's whole domain (box == domain)       */
    double *state;      /* device, 11 components over the ghosted box      */
    int64_t state_comp_stride;
    double inverse_dx[3];
    double cfl;    /* > 0 */
    double max_dt; /* <= 0: no cap */
    double time;   /* initial member time */
} grhd_ensemble_member;

/* Launch shape of the persistent kernel: the z extent of a face tile and
 * the resident blocks per SM; ms_per_step is what the autotuner measured
 * (0 when set by hand). */
typedef struct grhd_ensemble_tuning
{
    int zchunk;
    int blocks_per_sm;
    double ms_per_step;
} grhd_ensemble_tuning;

/* Allocates the scratch of every member (the states stay the caller's).
 * On error *out is still set (read the message, then destroy it). */
int grhd_ensemble_create(const grhd_ensemble_member *members, int count,
                         grhd_ensemble **out);
void grhd_ensemble_destroy(grhd_ensemble *ens);
int grhd_ensemble_last_error(const grhd_ensemble *ens, grhd_error *out);
int grhd_ensemble_get_tuning(const grhd_ensemble *ens,
                             grhd_ensemble_tuning *tuning,
                             int *max_blocks_per_sm);
int grhd_ensemble_set_tuning(grhd_ensemble *ens,
                             const grhd_ensemble_tuning *tuning);
/* Times `trial_steps` steps of every candidate launch shape (z chunks 8,
 * 16, 32, 64 x 1..max blocks per SM) on the real members, keeps the
 * fastest and restores the states, times, accretion integrals and
 * counters as they were. */
int grhd_ensemble_autotune(grhd_ensemble *ens, int trial_steps,
                           grhd_ensemble_tuning *best, void *stream);
/* `steps` RK4 steps of every member in one launch; use_graph = 1 replays a
 * CUDA graph captured for this step count (captured at its first use).
 * Synchronises; a recovery failure returns GRHD_ERR_RECOVERY naming the
 * member and cell. */
int grhd_ensemble_advance(grhd_ensemble *ens, int steps, int use_graph,
                          void *stream);
/* Member time, CFL speed of its current state (0 before the first
 * advance), Mdot of its last RHS, the Mdot time integral and the
 * cumulative recovery counters. */
int grhd_ensemble_member_info(grhd_ensemble *ens, int member, double *time,
                              double *max_inverse_dt, double *mdot,
                              double *mdot_integral, grhd_diagnostics *diag);
int grhd_ensemble_reset_accretion(grhd_ensemble *ens);
/* The member states were changed outside the ensemble: the next advance
 * recomputes the CFL speed from them. */
int grhd_ensemble_invalidate(grhd_ensemble *ens);
/* Test hook: grid barriers wait for `extra_arrivals` more blocks than the
 * grid has (none arrive, so every wait runs out after timeout_seconds and
 * advance returns GRHD_ERR_CUDA); 0 and the default 4 s restore normal
 * operation. */
int grhd_ensemble_set_barrier_test(grhd_ensemble *ens,
                                   unsigned int extra_arrivals,
                                   double timeout_seconds);
long long grhd_ensemble_launch_count(const grhd_ensemble *ens);


/* ---- discrete adjoint (new; no reference counterpart) ----
 * Reverse-mode kernels of the FP64 Kerr-Schild operator (one box covering
 * the domain, ghost width 2): the RHS, one RK4 step with its post-update
 * recoveries, and a checkpointed forward/backward pair for
 *   J = integral over the run of the rest-mass accretion rate through the
 *       sphere r < params.accretion_radius (grhd_accretion's quantity),
 * as a function of the eight parameters of a torus initial state.  The
 * backward replays the MUSCL limiter branches recorded by the forward,
 * runs the HLLE flux in reverse, differentiates con2prim by the implicit
 * function theorem at the converged pressure, and gets spin derivatives
 * of the analytic metric in dual numbers.  The step size is fixed (dt), so
 * J is differentiated along a fixed step sequence. */
typedef struct grhd_adjoint grhd_adjoint;

/* Initial data: the constant-angular-momentum torus of
 * FixedBGTorus.hpp:291-409 (inner edge, pressure maximum, velocity cap of
 * the potential) with density and pressure scaled by `amplitude`,
 * polytropic constant `entropy` (<= 0: the value giving density 1 at the
 * pressure maximum), Kerr-Schild spin `spin` (also the operator's), and
 * density modes rho *= 1 + sum_m mode_amplitude[m-1] cos(m phi +
 * mode_phase[m-1]), m = 1..5.  The gradient is ordered
 *   [amplitude, entropy, spin, mode_amplitude[0..4]]. */
typedef struct grhd_adjoint_torus
{
    double amplitude, entropy, spin;
    double mode_amplitude[5], mode_phase[5];
    double inner_radius, pressure_max_radius, max_velocity_squared;
} grhd_adjoint_torus;

void grhd_default_adjoint_torus(grhd_adjoint_torus *torus);
/* The entropy (polytropic constant) that gives density 1 at the pressure
 * maximum for these radii and spin. */
int grhd_adjoint_unit_entropy(const grhd_params *params,
                              const grhd_adjoint_torus *torus, double *K);
/* params: FP64 Kerr-Schild operator (its spin is replaced by the torus
 * spin of each forward); box == domain.  Allocates the tape of
 * `checkpoint_every` steps (about 1.6 KB per cell per step) and one
 * checkpoint per segment.  On error *out is still set. */
int grhd_adjoint_create(const grhd_params *params, const grhd_box *box,
                        int steps, int checkpoint_every, double dt,
                        grhd_adjoint **out);
void grhd_adjoint_destroy(grhd_adjoint *adj);
int grhd_adjoint_last_error(const grhd_adjoint *adj, grhd_error *out);
long long grhd_adjoint_launch_count(const grhd_adjoint *adj);
/* The initial state of `torus` (11 components over the ghosted box, may be
 * NULL) and/or its tangents dU0/dtheta_k (8 x 5 components over the
 * interior, component (k, c) at tangent + (5k + c) * stride; may be
 * NULL).  Device pointers; synchronous. */
int grhd_adjoint_initial_data(grhd_adjoint *adj,
                              const grhd_adjoint_torus *torus, double *state,
                              int64_t state_cs, double *tangent,
                              int64_t tangent_comp_stride, void *stream);
/* Forward: the initial state of `torus`, `steps` RK4 steps of size dt,
 * checkpoints every `checkpoint_every` steps; *J receives J.
 * Synchronous. */
int grhd_adjoint_forward(grhd_adjoint *adj, const grhd_adjoint_torus *torus,
                         double *J, void *stream);
/* Backward of the last forward: grad[8] = dJ/dtheta; lambda0 (device, 5
 * components over the interior, may be NULL) = dJ/dU0.  Synchronous. */
int grhd_adjoint_backward(grhd_adjoint *adj, double grad[8], double *lambda0,
                          int64_t lambda_comp_stride, void *stream);
/* Tangent-linear sweep (forward mode): J and dJ = sum_k direction[k]
 * dJ/dtheta_k for the torus `torus`, along the same taped forward steps
 * as grhd_adjoint_forward, with the same recorded limiter branches and the
 * same branch decisions as the backward sweep, so that dJ equals the
 * gradient's projection <grad, direction> to rounding for every direction
 * -- the check of the adjoint that needs no finite-difference step.
 * Overwrites the last forward's tape (call grhd_adjoint_forward again
 * before a backward).  Allocates its buffers per call.  Synchronous. */
int grhd_adjoint_tangent(grhd_adjoint *adj, const grhd_adjoint_torus *torus,
                         const double direction[8], double *J, double *dJ,
                         void *stream);
/* Vector-Jacobian product of one RHS evaluation (grhd_compute_rhs of the
 * FP64 operator with the adjoint's parameters, spin = params.ks_spin):
 * state_bar = (dRHS/dU)^T rhs_bar + mdot_bar dMdot/dU over the interior
 * conserved variables; *spin_bar = the same product's spin derivative.
 * Fills the physical ghosts of `state` as compute_rhs does. */
int grhd_adjoint_rhs_vjp(grhd_adjoint *adj, double *state, int64_t state_cs,
                         const double *rhs_bar, int64_t rhs_bar_cs,
                         double mdot_bar, double *state_bar,
                         int64_t state_bar_cs, double *spin_bar,
                         void *stream);
/* Vector-Jacobian product of one RK4 step of size dt (grhd_advance_rk4):
 * given the adjoint of U^{n+1} and the weight of the step's accretion
 * integral, the adjoint of U^n and the spin derivative. */
int grhd_adjoint_step_vjp(grhd_adjoint *adj, const double *state,
                          int64_t state_cs, const double *state_bar_next,
                          int64_t next_cs, double mdot_integral_bar,
                          double *state_bar, int64_t state_bar_cs,
                          double *spin_bar, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* GRHD_B200_H_ */
