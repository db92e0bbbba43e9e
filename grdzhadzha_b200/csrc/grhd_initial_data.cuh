// grhd_initial_data.cuh -- device initial data (torus, Michel, perturbation).
#pragma once

#include "grhd_kernels.cuh"

#include <math_constants.h>

namespace grhd {

// FixedBGTorusConfig, Source/Matter/GRHD/FixedBGTorus.hpp:20-34
struct TorusConfigDev
{
    double total_mass, inner_radius, pressure_max_radius, rho_peak,
        max_velocity_squared, radial_derivative_fraction,
        radial_derivative_min_step, angular_momentum_min_factor,
        angular_momentum_max_factor;
    int angular_momentum_samples, angular_momentum_bisection_iterations;
    double angular_momentum_tolerance;
};

// MichelConfig, Tests/GRHDLevelDataMichelAccretion/
// GRHDLevelDataMichelAccretion.cpp:32-45
struct MichelConfigDev
{
    double mass, gamma, sonic_radius, sonic_density, atmosphere_radius,
        root_tolerance;
};

// out = ell, surface potential, polytropic constant, max enthalpy.
cudaError_t torus_initial_data(double *state, const BoxDev &b,
                               const Background &bg, const Options &o,
                               const TorusConfigDev &c, double *scratch4,
                               double out[4], cudaStream_t s);
cudaError_t michel_initial_data(double *state, const BoxDev &b,
                                const Options &o, const MichelConfigDev &c,
                                int *bad_flag, cudaStream_t s);
cudaError_t perturb_density(double *state, const BoxDev &b,
                            const Background &bg, const Options &o,
                            double amplitude, uint64_t seed, cudaStream_t s);

} // namespace grhd
