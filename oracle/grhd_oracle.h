/*
 * grhd_oracle.h -- CPU restatement of GRDzhadzha's fixed-background Valencia
 * GRHD path, used ONLY as the test checker and as the timed CPU baseline.
 *
 * TEST INFRASTRUCTURE.  Nothing in the product library links, loads or calls
 * this code.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may use it.
 *
 * Every function restates one reference function and cites it as
 * path:line relative to the GRDzhadzha source tree.  Floating-point operation
 * order follows the reference expressions so that, built with
 * -ffp-contract=off, the results are the reference's own up to libm.
 *
 * Storage: one ghosted box per call, structure of arrays, x fastest:
 *   value(i,j,k,c) = data[c*comp_stride + (i-glo0) + nx*((j-glo1) + ny*(k-glo2))]
 * with components in the reference UserVariables order
 *   0 D, 1 S1, 2 S2, 3 S3, 4 tau, 5 rho, 6 eps, 7 pressure, 8 v1, 9 v2, 10 v3
 * (Tests/GRHDFixedBGTest/UserVariables.hpp:24-40, conserved first).
 */
#ifndef GRHD_ORACLE_H_
#define GRHD_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum
{
    ORC_D = 0,
    ORC_S1,
    ORC_S2,
    ORC_S3,
    ORC_TAU,
    ORC_RHO,
    ORC_EPS,
    ORC_PRESS,
    ORC_V1,
    ORC_V2,
    ORC_V3,
    ORC_NCOMP
};

enum
{
    ORC_BG_KERR_SCHILD = 0,
    ORC_BG_BINARY_PN = 1
};

enum
{
    ORC_OK = 0,
    ORC_ERR_RECOVERY = 1,     /* con2prim failure on an RHS/CFL/boundary path */
    ORC_ERR_INVALID_ARG = 2,  /* cfl <= 0, dx <= 0, bad box */
    ORC_ERR_SETUP = 3         /* initial-data construction failed */
};

/* Error location kinds, mirroring the reference's runtime_error messages. */
enum
{
    ORC_WHERE_NONE = 0,
    ORC_WHERE_OUTFLOW_SOURCE = 1, /* FixedBGFArrayBoxFiniteVolume.hpp:157-164 */
    ORC_WHERE_GHOSTED_RECOVERY = 2, /* :48-55 */
    ORC_WHERE_METRIC_SOURCES = 3, /* :272-279 */
    ORC_WHERE_CFL = 4             /* :383-390 */
};

/* Operator parameters: the union of the constructor arguments of
 * FixedBGLevelDataFiniteVolumeOperator / TimeDependent... (reference
 * FixedBGFArrayBoxFiniteVolume.hpp:450-464, 681-700), the background
 * params_t structs (KerrSchild.hpp:26-31, CircularBinaryPN.hpp:32-42),
 * AtmosphereOptions (Atmosphere.hpp:16-22) and RecoveryOptions
 * (Valencia.hpp:17-23).  New fields are marked. */
typedef struct orc_params
{
    int background;            /* ORC_BG_* */
    double ks_mass, ks_spin;   /* KerrSchild::params_t */
    double pn_mass_1, pn_mass_2, pn_separation, pn_angular_velocity,
        pn_phase, pn_time, pn_softening_radius; /* CircularBinaryPN::params_t */
    double gamma;              /* IdealGasEOS adiabatic index */
    double dx;                 /* m_dx */
    double center[3];          /* m_center (Coordinates origin) */
    double atmo_rho_floor, atmo_pressure_floor, atmo_max_velocity_squared,
        atmo_metric_source_atmosphere_factor;
    int rec_max_iterations;
    double rec_tolerance, rec_pressure_floor, rec_max_velocity_squared;
    double limiter_theta;
    int use_reconstruction, use_static_metric_sources,
        use_metric_volume_time_sources;
    double metric_time_derivative_step;
    double excision_radius;    /* new: <= 0 disables excision */
    double accretion_radius;   /* new: sphere of the Mdot diagnostic */
} orc_params;

/* A box of the level: interior cell range (inclusive, Chombo Box), the
 * ghosted storage range of the array that holds it, and the problem domain
 * (non-periodic).  comp_stride is the distance between components. */
typedef struct orc_box
{
    int lo[3], hi[3];
    int glo[3], ghi[3];
    int dlo[3], dhi[3];
    int64_t comp_stride;
} orc_box;

typedef struct orc_diag
{
    long long num_cells, num_failed_recoveries, num_floored_primitives,
        num_conserved_resets;
} orc_diag;

typedef struct orc_error
{
    int code;
    int where;
    int cell[3];
    double residual;
} orc_error;

void orc_default_params(orc_params *p);

/* ---- pointwise helpers (exposed for unit tests) ---- */
/* ADM vars at a position relative to the operator centre, time offset t:
 * out = gamma[9], K_tensor[9], K, lapse, shift[3], d1_gamma[27] ([i][j][k],
 * derivative last), d1_lapse[3], d1_shift[9] ([i][j] = d_j shift^i). */
void orc_background_vars(const orc_params *p, double t, double x, double y,
                         double z, double *out_64);
/* Valencia p2c for one cell: prim = rho,eps,p,v^i; gLL[9]. */
void orc_compute_conserved(const orc_params *p, const double *prim6,
                           const double *gLL9, double *cons5);
/* con2prim: returns success; writes prim6, iterations, residual. */
int orc_recover_primitive(const orc_params *p, const double *cons5,
                          const double *gUU9, double *prim6, int *iterations,
                          double *residual);
/* The full face flux: MUSCL reconstruct + floors + p2c + HLLE. */
void orc_muscl_hlle_flux(const orc_params *p, const double *left_prim6,
                         const double *right_prim6, const double *left_slope6,
                         const double *right_slope6, const double *gLL9,
                         const double *gUU9, double lapse,
                         const double *shift3, int direction, double *flux5);

/* ---- box operators (single box; ghosts 2) ---- */
int orc_compute_rhs(const orc_params *p, const orc_box *box, double *state,
                    double *rhs, int64_t rhs_comp_stride,
                    const double inv_dx[3], double time, orc_error *err);
int orc_recover_primitives(const orc_params *p, const orc_box *box,
                           double *state, double time, orc_diag *diag);
int orc_compute_max_inverse_dt(const orc_params *p, const orc_box *box,
                               const double *state, const double inv_dx[3],
                               double time, double *out, orc_error *err);
int orc_compute_stable_dt(const orc_params *p, const orc_box *box,
                          const double *state, const double inv_dx[3],
                          double cfl, double time, double *out,
                          orc_error *err);
int orc_update_conserved(const orc_params *p, const orc_box *box,
                         double *state, const double *rhs,
                         int64_t rhs_comp_stride, double dt,
                         double recovery_time, int recover, orc_diag *diag);
int orc_advance_ssprk2(const orc_params *p, const orc_box *box, double *state,
                       const double inv_dx[3], double time, double dt,
                       orc_diag *diag, orc_error *err);
/* New: the RHS plus the rest-mass accretion rate through the voxelised
 * sphere r < accretion_radius: Mdot = - sum over its boundary faces of
 * sqrt(det gamma_face) F_D . n_out dx^2, with the scheme's HLLE face
 * fluxes. */
int orc_compute_rhs_mdot(const orc_params *p, const orc_box *box,
                         double *state, double *rhs, int64_t rhs_comp_stride,
                         const double inv_dx[3], double time, double *mdot,
                         orc_error *err);
int orc_advance_ssprk2_mdot(const orc_params *p, const orc_box *box,
                            double *state, const double inv_dx[3],
                            double time, double dt, orc_diag *diag,
                            orc_error *err, double *mdot_integral);
int orc_advance_rk4_mdot(const orc_params *p, const orc_box *box,
                         double *state, const double inv_dx[3], double time,
                         double dt, orc_diag *diag, orc_error *err,
                         double *mdot_integral);
/* New: classic RK4 with post-stage recovery. */
int orc_advance_rk4(const orc_params *p, const orc_box *box, double *state,
                    const double inv_dx[3], double time, double dt,
                    orc_diag *diag, orc_error *err);

/* ---- multi-box CPU baseline: z-slab boxes, one thread per box ---- */
int orc_compute_rhs_slabs(const orc_params *p, const orc_box *box,
                          double *state, double *rhs, int64_t rhs_comp_stride,
                          const double inv_dx[3], double time, int num_slabs,
                          orc_error *err);

/* ---- initial data ---- */
typedef struct orc_torus_config
{
    double total_mass, inner_radius, pressure_max_radius, rho_peak,
        max_velocity_squared, radial_derivative_fraction,
        radial_derivative_min_step, angular_momentum_min_factor,
        angular_momentum_max_factor;
    int angular_momentum_samples, angular_momentum_bisection_iterations;
    double angular_momentum_tolerance;
} orc_torus_config;

typedef struct orc_torus_params
{
    double ell, surface_potential, polytropic_constant, max_enthalpy;
} orc_torus_params;

void orc_default_torus_config(orc_torus_config *c);
int orc_make_torus_parameters(const orc_params *p, const orc_torus_config *c,
                              const orc_box *box, double time,
                              orc_torus_params *out);
int orc_fill_torus(const orc_params *p, const orc_torus_config *c,
                   const orc_torus_params *t, const orc_box *box,
                   double *state, double time);

typedef struct orc_michel_config
{
    double mass, gamma, sonic_radius, sonic_density, atmosphere_radius,
        root_tolerance;
} orc_michel_config;

/* Michel constants: polytropic_K, mass_flux, bernoulli, sonic_ur, cs2. */
void orc_michel_constants(const orc_michel_config *c, double *out5);
/* Michel point at radius: rho, pressure, eps, ur, vr. */
int orc_michel_point(const orc_params *p, const orc_michel_config *c,
                     double radius, double *out5);
int orc_fill_michel(const orc_params *p, const orc_michel_config *c,
                    const orc_box *box, double *state);

/* Number of threads the setup passes (initial data, recovery) use. */
void orc_set_threads(int n);

/* conserved components of the whole ghosted box from its primitives */
void orc_fill_conserved_from_primitives(const orc_params *p,
                                        const orc_box *box, double *state,
                                        double time);

/* ---- diagnostics (example drivers) ---- */
/* out: mass, disk_mass, tau, max_rho, max_pressure, max_velocity,
 * max_lorentz_factor (Main_GRHDLevelDataKerrSchildDisk.cpp:223-290) over
 * the cell range [lo,hi] of the box. */
void orc_disk_diagnostics(const orc_params *p, const orc_box *box,
                          const int lo[3], const int hi[3],
                          const double *state, double time, double *out7);


/* ---- KITP disk driver source terms (the binary-PN production driver) ----
 * Examples/GRHDLevelDataBinaryPNKITPDisk/Main_GRHDLevelDataBinaryPNKITPDisk.cpp
 * SimulationConfig fields (:67-71) and rho_floor (:63) used by them. */
typedef struct orc_kitp_config
{
    double alpha_viscosity, viscosity_beta, rho_floor, sink_size, sink_rate,
        sink_shape;
} orc_kitp_config;
/* add_kitp_viscous_rhs (:772-806): rhs (interior, 5 comps) -= the central
 * difference of the alpha-viscosity stress flux in x and y, from the
 * state's stored primitives, binary at operator time t. */
void orc_kitp_viscous_rhs(const orc_params *p, const orc_kitp_config *k,
                          const orc_box *box, const double *state,
                          double *rhs, int64_t rhs_comp_stride, double t);
/* add_kitp_sink_rhs (:567-610): rhs -= rate * conserved. */
void orc_kitp_sink_rhs(const orc_params *p, const orc_kitp_config *k,
                       const orc_box *box, const double *state, double *rhs,
                       int64_t rhs_comp_stride, double t);
/* apply_kitp_sink_decay (:612-662): conserved *= exp(-rate dt) at binary
 * time t (the driver passes the step's mid time). */
void orc_kitp_sink_decay(const orc_params *p, const orc_kitp_config *k,
                         const orc_box *box, double *state, double t,
                         double dt);

/* ---- the binary disk drivers' Keplerian disk (kitp_primitive,
 * Main_GRHDLevelDataBinaryPNKITPDisk.cpp:398-555; SimulationConfig :56-61)
 * with azimuthal density modes m = 1..4 (new) ---- */
typedef struct orc_kitp_disk
{
    double mach, aspect_ratio, cavity_radius_factor, cavity_delta,
        outer_cutoff_radius, rho_peak;
    double mode_amplitude[4], mode_phase[4];
} orc_kitp_disk;
/* Primitives and conserved variables over the ghosted box at time t (the
 * operator's binary and atmosphere floors). */
void orc_fill_kitp_disk(const orc_params *p, const orc_kitp_disk *k,
                        const orc_box *box, double *state, double t);

/* ---- the operator on CCZ4-stored geometry (LevelDataFiniteVolumeOperator,
 * Source/Matter/GRHD/FArrayBoxFiniteVolume.hpp:681-1364) ----
 * state: 36 components of comp_stride each, GRChombo's 25 CCZ4 variables
 * (chi, h11 h12 h13 h22 h23 h33, K, A11..A33, Theta, Gamma1..3, lapse,
 * shift1..3, B1..3) then the 11 GRHD ones. */
#define ORC_CCZ4_NUM_VARS 36
#define ORC_CCZ4_GRHD_OFFSET 25
int orc_ccz4_compute_rhs(const orc_params *p, const orc_box *box,
                         double *state, double *rhs, int64_t rhs_comp_stride,
                         const double inv_dx[3], orc_error *err);
void orc_ccz4_recover_primitives(const orc_params *p, const orc_box *box,
                                 double *state, orc_diag *diag);
int orc_ccz4_compute_max_inverse_dt(const orc_params *p, const orc_box *box,
                                    const double *state,
                                    const double inv_dx[3], double *out,
                                    orc_error *err);
void orc_ccz4_fill_from_background(const orc_params *p, const orc_box *box,
                                   double *state, double t);

#ifdef __cplusplus
}
#endif

#endif /* GRHD_ORACLE_H_ */
