// A compiled C++ caller of the C ABI (include/grhd_b200.h): the drop-in
// class INTEGRATION.md gives for the reference operator
// FixedBGLevelDataFiniteVolumeOperator<IdealGasEOS, KerrSchild>
// (Source/Matter/GRHD/FixedBGFArrayBoxFiniteVolume.hpp:446-614), with the
// reference's method names and exception types, driven on one box.
//
// Built by tests/test_gpu_cxx_dropin.py with g++ against the header and
// linked to libgrhd_b200.so.  Usage:
//   cxx_dropin <params.txt> <state.bin> <out_dir>
// params.txt: "name value" lines (grhd_params fields, box, time, dt, cfl);
// state.bin: the ghosted box's 11 components, FP64, x fastest.
// Writes out_dir/rhs.bin (compute_rhs), out_dir/ssprk2.bin (the state after
// advance_ssprk2 from the input state), out_dir/stable_dt.txt and prints
// "invalid_argument ok" when compute_stable_dt(cfl = 0) throws
// std::invalid_argument, as the reference's does (:549-550).
#include "grhd_b200.h"

#include <cuda_runtime.h>

#include <array>
#include <cstdio>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

// The reference's option structs (Atmosphere.hpp:16-22, Valencia.hpp:17-23)
// as a caller holds them; the field names and defaults are the reference's.
namespace GRHD
{
struct AtmosphereOptions
{
    double rho_floor = 1.0e-12;
    double pressure_floor = 1.0e-12;
    double max_velocity_squared = 1.0 - 1.0e-12;
    double metric_source_atmosphere_factor = 1.0 + 1.0e-12;
};
struct RecoveryOptions
{
    int max_iterations = 50;
    double tolerance = 1.0e-12;
    double pressure_floor = 1.0e-12;
    double max_velocity_squared = 1.0 - 1.0e-12;
};
} // namespace GRHD

// KerrSchild::params_t (Source/Background/KerrSchild.hpp)
struct KerrSchildParams
{
    double mass = 1.0;
    double spin = 0.0;
};

class B200FixedBGOperator
{
  public:
    B200FixedBGOperator(double gamma, const KerrSchildParams &bg, double dx,
                        const std::array<double, 3> &center,
                        const GRHD::AtmosphereOptions &atmo = {},
                        double limiter_theta = 1.5,
                        const GRHD::RecoveryOptions &rec = {},
                        bool use_reconstruction = true,
                        bool use_static_metric_sources = true)
    {
        grhd_params p;
        grhd_default_params(&p);
        p.background = GRHD_BG_KERR_SCHILD;
        p.ks_mass = bg.mass;
        p.ks_spin = bg.spin;
        p.adiabatic_index = gamma;
        p.dx = dx;
        for (int d = 0; d < 3; ++d)
            p.center[d] = center[d];
        p.rho_floor = atmo.rho_floor;
        p.pressure_floor = atmo.pressure_floor;
        p.max_velocity_squared = atmo.max_velocity_squared;
        p.metric_source_atmosphere_factor =
            atmo.metric_source_atmosphere_factor;
        p.recovery_max_iterations = rec.max_iterations;
        p.recovery_tolerance = rec.tolerance;
        p.recovery_pressure_floor = rec.pressure_floor;
        p.recovery_max_velocity_squared = rec.max_velocity_squared;
        p.limiter_theta = limiter_theta;
        p.use_reconstruction = use_reconstruction;
        p.use_static_metric_sources = use_static_metric_sources;
        if (grhd_create(&p, &m_ctx) != GRHD_OK)
            throw std::runtime_error("grhd_create failed");
    }
    ~B200FixedBGOperator() { grhd_destroy(m_ctx); }
    B200FixedBGOperator(const B200FixedBGOperator &) = delete;
    B200FixedBGOperator &operator=(const B200FixedBGOperator &) = delete;

    // compute_rhs(rhs, state, domain, inverse_dx_U), :468-477; one box of
    // the level (after state.exchange() for a level of several boxes)
    void compute_rhs(double *rhs, int64_t rhs_stride, double *state,
                     int64_t state_stride, const grhd_box &box,
                     const double inv_dx[3], cudaStream_t s) const
    {
        check(grhd_compute_rhs(m_ctx, rhs, rhs_stride, state, state_stride,
                               &box, inv_dx, 0.0, s));
    }

    // recover_primitives(state), :506-520
    grhd_diagnostics recover_primitives(double *state, int64_t state_stride,
                                        const grhd_box &box,
                                        cudaStream_t s) const
    {
        grhd_diagnostics d{};
        check(grhd_recover_primitives(m_ctx, state, state_stride, &box, 0.0,
                                      &d, s));
        return d;
    }

    // update_conserved(state, rhs, dt, recover), :522-533
    grhd_diagnostics update_conserved(double *state, int64_t state_stride,
                                      const double *rhs, int64_t rhs_stride,
                                      const grhd_box &box, double dt,
                                      bool recover, cudaStream_t s) const
    {
        grhd_diagnostics d{};
        check(grhd_update_conserved(m_ctx, state, state_stride, rhs,
                                    rhs_stride, &box, dt, 0.0, recover, &d,
                                    s));
        return d;
    }

    // compute_stable_dt(state, domain_box, inverse_dx_U, cfl), :544-555
    double compute_stable_dt(const double *state, int64_t state_stride,
                             const grhd_box &box, const double inv_dx[3],
                             double cfl, cudaStream_t s) const
    {
        double dt = 0.0;
        check(grhd_compute_stable_dt(m_ctx, state, state_stride, &box,
                                     inv_dx, cfl, 0.0, &dt, s));
        return dt;
    }

    // advance_ssprk2(state, domain, inverse_dx_U, dt), :563-589
    grhd_diagnostics advance_ssprk2(double *state, int64_t state_stride,
                                    const grhd_box &box,
                                    const double inv_dx[3], double dt,
                                    cudaStream_t s) const
    {
        grhd_diagnostics d{};
        check(grhd_advance_ssprk2(m_ctx, state, state_stride, &box, inv_dx,
                                  0.0, dt, &d, s));
        return d;
    }

  private:
    // the reference's exception types: std::invalid_argument for bad
    // arguments (:549-550), std::runtime_error for a failed recovery
    // (:48-55, :157-164, :272-279, :383-390)
    void check(int status) const
    {
        if (status == GRHD_OK)
            return;
        grhd_error e;
        grhd_last_error(m_ctx, &e);
        if (status == GRHD_ERR_INVALID_ARG)
            throw std::invalid_argument(e.message);
        throw std::runtime_error(e.message);
    }
    grhd_ctx *m_ctx = nullptr;
};

// ------------------------------------------------------------------ driver

static void cuda_check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " +
                                 cudaGetErrorString(e));
}

static std::map<std::string, std::vector<double>>
read_params(const char *path)
{
    std::map<std::string, std::vector<double>> out;
    std::ifstream in(path);
    std::string line;
    while (std::getline(in, line))
    {
        std::istringstream ls(line);
        std::string key;
        if (!(ls >> key))
            continue;
        double v;
        while (ls >> v)
            out[key].push_back(v);
    }
    return out;
}

static void write_bin(const std::string &path, const std::vector<double> &v)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(v.data()),
            (std::streamsize)(v.size() * sizeof(double)));
}

int main(int argc, char **argv)
{
    if (argc != 4)
    {
        std::fprintf(stderr, "usage: %s params.txt state.bin out_dir\n",
                     argv[0]);
        return 2;
    }
    try
    {
        auto P = read_params(argv[1]);
        auto v = [&](const char *k) { return P.at(k).at(0); };
        grhd_box box;
        for (int d = 0; d < 3; ++d)
        {
            box.lo[d] = (int)P.at("lo").at(d);
            box.hi[d] = (int)P.at("hi").at(d);
            box.domain_lo[d] = (int)P.at("domain_lo").at(d);
            box.domain_hi[d] = (int)P.at("domain_hi").at(d);
        }
        box.ghost = (int)v("ghost");
        int64_t stride = 1, interior = 1;
        for (int d = 0; d < 3; ++d)
        {
            stride *= box.hi[d] - box.lo[d] + 1 + 2 * box.ghost;
            interior *= box.hi[d] - box.lo[d] + 1;
        }
        std::vector<double> host(11 * stride);
        {
            std::ifstream f(argv[2], std::ios::binary);
            f.read(reinterpret_cast<char *>(host.data()),
                   (std::streamsize)(host.size() * sizeof(double)));
            if (!f)
                throw std::runtime_error("short state file");
        }
        GRHD::AtmosphereOptions atmo;
        atmo.rho_floor = v("rho_floor");
        atmo.pressure_floor = v("pressure_floor");
        atmo.max_velocity_squared = v("max_velocity_squared");
        atmo.metric_source_atmosphere_factor =
            v("metric_source_atmosphere_factor");
        GRHD::RecoveryOptions rec;
        rec.max_iterations = (int)v("recovery_max_iterations");
        rec.tolerance = v("recovery_tolerance");
        rec.pressure_floor = v("recovery_pressure_floor");
        rec.max_velocity_squared = v("recovery_max_velocity_squared");
        const double dx = v("dx");
        const std::array<double, 3> center = {P.at("center").at(0),
                                              P.at("center").at(1),
                                              P.at("center").at(2)};
        const B200FixedBGOperator op(
            v("adiabatic_index"), KerrSchildParams{v("ks_mass"), v("ks_spin")},
            dx, center, atmo, v("limiter_theta"), rec,
            v("use_reconstruction") != 0.0,
            v("use_static_metric_sources") != 0.0);
        const double inv_dx[3] = {1.0 / dx, 1.0 / dx, 1.0 / dx};

        cudaStream_t s;
        cuda_check(cudaStreamCreate(&s), "cudaStreamCreate");
        double *state = nullptr, *rhs = nullptr;
        cuda_check(cudaMalloc(&state, host.size() * sizeof(double)),
                   "cudaMalloc state");
        cuda_check(cudaMalloc(&rhs, 5 * interior * sizeof(double)),
                   "cudaMalloc rhs");
        const std::string out = argv[3];

        // compute_rhs of the input state
        cuda_check(cudaMemcpy(state, host.data(), host.size() * sizeof(double),
                              cudaMemcpyHostToDevice),
                   "copy state");
        op.compute_rhs(rhs, interior, state, stride, box, inv_dx, s);
        std::vector<double> r(5 * interior);
        cuda_check(cudaMemcpy(r.data(), rhs, r.size() * sizeof(double),
                              cudaMemcpyDeviceToHost),
                   "copy rhs");
        write_bin(out + "/rhs.bin", r);

        // compute_stable_dt, then one advance_ssprk2 from the input state
        cuda_check(cudaMemcpy(state, host.data(), host.size() * sizeof(double),
                              cudaMemcpyHostToDevice),
                   "copy state");
        const double dt =
            op.compute_stable_dt(state, stride, box, inv_dx, v("cfl"), s);
        {
            std::ofstream f(out + "/stable_dt.txt");
            char buf[64];
            std::snprintf(buf, sizeof buf, "%.17g\n", dt);
            f << buf;
        }
        const grhd_diagnostics d =
            op.advance_ssprk2(state, stride, box, inv_dx, v("dt"), s);
        std::vector<double> after(host.size());
        cuda_check(cudaMemcpy(after.data(), state,
                              after.size() * sizeof(double),
                              cudaMemcpyDeviceToHost),
                   "copy state back");
        write_bin(out + "/ssprk2.bin", after);
        std::printf("ssprk2_diag %lld %lld %lld %lld\n",
                    d.num_cells, d.num_failed_recoveries,
                    d.num_floored_primitives, d.num_conserved_resets);

        // the reference's argument check: cfl <= 0 is invalid_argument
        try
        {
            op.compute_stable_dt(state, stride, box, inv_dx, 0.0, s);
            std::printf("no exception for cfl = 0\n");
        }
        catch (const std::invalid_argument &e)
        {
            std::printf("invalid_argument ok: %s\n", e.what());
        }
        cudaFree(state);
        cudaFree(rhs);
        cudaStreamDestroy(s);
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
