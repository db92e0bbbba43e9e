// grhd_kitp.cuh -- source terms of the reference's binary-PN disk production
// driver (Examples/GRHDLevelDataBinaryPNKITPDisk/
// Main_GRHDLevelDataBinaryPNKITPDisk.cpp): the alpha-viscosity stress
// divergence (:676-806) and the two point-mass sinks (:557-662), on the
// device, FP64.
#pragma once

#include "grhd_kernels.cuh"

namespace grhd {

// The driver's SimulationConfig fields these terms read (:63, :67-71), the
// binary's masses and body positions at the evaluation time, and the
// atmosphere floor that switches them off.
struct KitpDev
{
    double alpha, beta, rho_floor_cfg, sink_size, sink_rate, sink_shape;
    double mass[2];
    double body[2][3];
    double atmo_rho_floor;
};

// rhs (interior, 5 components, stride rcs) -= d/dx F_x + d/dy F_y of the
// viscous stress flux (add_kitp_viscous_rhs, :772-806).
void launch_kitp_viscous_rhs(double *rhs, int64_t rcs, const double *state,
                             const BoxDev &b, const Options &o,
                             const KitpDev &k, cudaStream_t s);
// rhs -= rate * conserved (add_kitp_sink_rhs, :567-610).
void launch_kitp_sink_rhs(double *rhs, int64_t rcs, const double *state,
                          const BoxDev &b, const Options &o, const KitpDev &k,
                          cudaStream_t s);
// conserved *= exp(-rate dt) (apply_kitp_sink_decay, :612-662).
void launch_kitp_sink_decay(double *state, const BoxDev &b, const Options &o,
                            const KitpDev &k, double dt, cudaStream_t s);

// combine_ssprk2_conserved_state (FArrayBoxFiniteVolume.hpp:942-969) on the
// interior conserved variables, without a recovery: s = (s + u1 + dt k) / 2
// (the disk driver decays its sinks between the combination and the
// recovery, advance_kitp_ssprk2 :842-876).
void launch_kitp_combine(double *state, const BoxDev &b, const double *u1,
                         int64_t u1_cs, const double *k, int64_t rcs,
                         double dt, cudaStream_t s);

// The disk drivers' Keplerian disk (kitp_primitive, :398-520) with the
// azimuthal density modes m = 1..4 (new): the binary (masses, separation,
// softening, orbital frequency, body positions at the fill time) and the
// disk settings of SimulationConfig (:56-61).
struct KitpDiskDev
{
    double mach, aspect, cavity_factor, cavity_delta, outer_cutoff, rho_peak;
    double amp[4], phase[4];
    double sep, mass[2], soft, omega_bin;
    double body[2][3];
};

// Primitives and conserved variables of every ghosted cell.
void launch_kitp_disk_fill(double *state, const BoxDev &b,
                           const Background &bg, const Options &o,
                           const KitpDiskDev &k, cudaStream_t s);

} // namespace grhd
