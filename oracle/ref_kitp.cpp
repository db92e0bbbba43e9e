/*
 * ref_kitp.cpp -- TEST INFRASTRUCTURE: the reference's KITP disk driver
 * (Examples/GRHDLevelDataBinaryPNKITPDisk/Main_GRHDLevelDataBinaryPNKITPDisk
 * .cpp) behind C entry points with the oracle's types, for the parity of
 * the oracle's restatement of its source terms, initial data and step.
 *
 * The driver's source file is compiled unmodified as part of this
 * translation unit (its `main` renamed by the preprocessor; its functions
 * live in an anonymous namespace, visible here), against oracle/shim, by
 * oracle/Makefile into oracle/_ref/libref_kitp.so.  The driver's
 * SimulationConfig (:36-84) is assembled from orc_params (binary, EOS-side
 * floors, limiter, metric-source switches), orc_kitp_config (viscosity,
 * sinks) and orc_kitp_disk (the disk; the reference has no azimuthal
 * modes, so they must be zero).
 */
#include "grhd_oracle.h"

#define main kitp_reference_main
#include "Main_GRHDLevelDataBinaryPNKITPDisk.cpp"
#undef main

#include <cstring>

namespace
{

SimulationConfig config_of(const orc_params *p, const orc_kitp_config *k,
                           const orc_kitp_disk *d)
{
    SimulationConfig c;
    c.mass_1 = p->pn_mass_1;
    c.mass_2 = p->pn_mass_2;
    c.separation = p->pn_separation;
    c.binary_phase = p->pn_phase;
    c.binary_time = p->pn_time;
    c.binary_angular_velocity = p->pn_angular_velocity;
    c.softening_radius = p->pn_softening_radius;
    c.metric_time_derivative_step = p->metric_time_derivative_step;
    c.rho_floor = p->atmo_rho_floor;
    c.pressure_floor = p->atmo_pressure_floor;
    c.max_velocity_squared = p->atmo_max_velocity_squared;
    c.limiter_theta = p->limiter_theta;
    c.use_reconstruction = p->use_reconstruction != 0;
    c.use_static_metric_sources = p->use_static_metric_sources != 0;
    c.use_metric_volume_time_sources =
        p->use_metric_volume_time_sources != 0;
    if (k)
    {
        c.alpha_viscosity = k->alpha_viscosity;
        c.viscosity_beta = k->viscosity_beta;
        c.rho_floor = k->rho_floor;
        c.sink_size = k->sink_size;
        c.sink_rate = k->sink_rate;
        c.sink_shape = k->sink_shape;
    }
    if (d)
    {
        c.mach = d->mach;
        c.aspect_ratio = d->aspect_ratio;
        c.cavity_radius_factor = d->cavity_radius_factor;
        c.cavity_delta = d->cavity_delta;
        c.outer_cutoff_radius = d->outer_cutoff_radius;
        c.rho_peak = d->rho_peak;
    }
    return c;
}

BinaryPNFactory factory_of(const orc_params *p)
{
    BinaryPNFactory f;
    f.params.mass_1 = p->pn_mass_1;
    f.params.mass_2 = p->pn_mass_2;
    f.params.separation = p->pn_separation;
    f.params.angular_velocity = p->pn_angular_velocity;
    f.params.phase = p->pn_phase;
    f.params.time = p->pn_time;
    f.params.softening_radius = p->pn_softening_radius;
    f.params.center = {{0.0, 0.0, 0.0}};
    f.dx = p->dx;
    return f;
}

GRHD::AtmosphereOptions atmo_of(const orc_params *p)
{
    GRHD::AtmosphereOptions a;
    a.rho_floor = p->atmo_rho_floor;
    a.pressure_floor = p->atmo_pressure_floor;
    a.max_velocity_squared = p->atmo_max_velocity_squared;
    a.metric_source_atmosphere_factor =
        p->atmo_metric_source_atmosphere_factor;
    return a;
}

GRHD::RecoveryOptions rec_of(const orc_params *p)
{
    GRHD::RecoveryOptions r;
    r.max_iterations = p->rec_max_iterations;
    r.tolerance = p->rec_tolerance;
    r.pressure_floor = p->rec_pressure_floor;
    r.max_velocity_squared = p->rec_max_velocity_squared;
    return r;
}

std::array<double, CH_SPACEDIM> centre_of(const orc_params *p)
{
    return {p->center[0], p->center[1], p->center[2]};
}

bool usable(const orc_params *p, const orc_box *b)
{
    if (!p || !b || p->background != ORC_BG_BINARY_PN || !(p->dx > 0.0))
        return false;
    for (int d = 0; d < 3; ++d)
        if (b->lo[d] - b->glo[d] != 2 || b->ghi[d] - b->hi[d] != 2)
            return false;
    return true;
}

bool no_modes(const orc_kitp_disk *d)
{
    for (int m = 0; m < 4; ++m)
        if (d->mode_amplitude[m] != 0.0)
            return false;
    return true;
}

/* the caller's ghosted box as a one-box level of NUM_VARS components */
struct Lv
{
    Box domain_box, interior;
    ProblemDomain domain;
    DisjointBoxLayout grids;
    LevelData<FArrayBox> state;
    const orc_box *b;

    explicit Lv(const orc_box *bb) : b(bb)
    {
        domain_box = Box(IntVect(b->dlo[0], b->dlo[1], b->dlo[2]),
                         IntVect(b->dhi[0], b->dhi[1], b->dhi[2]));
        interior = Box(IntVect(b->lo[0], b->lo[1], b->lo[2]),
                       IntVect(b->hi[0], b->hi[1], b->hi[2]));
        domain = ProblemDomain(domain_box);
        Vector<Box> boxes(1, interior);
        Vector<int> procs(1, 0);
        grids = DisjointBoxLayout(boxes, procs, domain);
        state.define(grids, NUM_VARS, 2 * IntVect::Unit);
    }
    FArrayBox &fab() { return state[DataIndex(0)]; }
    int64_t at(const IntVect &iv) const
    {
        const int64_t nx = b->ghi[0] - b->glo[0] + 1;
        const int64_t ny = b->ghi[1] - b->glo[1] + 1;
        return (iv[0] - b->glo[0]) +
               nx * ((iv[1] - b->glo[1]) + ny * (int64_t)(iv[2] - b->glo[2]));
    }
    void load(const double *s)
    {
        for (BoxIterator bit(fab().box()); bit.ok(); ++bit)
            for (int c = 0; c < ORC_NCOMP; ++c)
                fab()(bit(), c_GRHD_D + c) = s[c * b->comp_stride + at(bit())];
    }
    void store(double *s)
    {
        for (BoxIterator bit(fab().box()); bit.ok(); ++bit)
            for (int c = 0; c < ORC_NCOMP; ++c)
                s[c * b->comp_stride + at(bit())] = fab()(bit(), c_GRHD_D + c);
    }
    int64_t iat(const IntVect &iv) const
    {
        const int64_t nx = b->hi[0] - b->lo[0] + 1;
        const int64_t ny = b->hi[1] - b->lo[1] + 1;
        return (iv[0] - b->lo[0]) +
               nx * ((iv[1] - b->lo[1]) + ny * (int64_t)(iv[2] - b->lo[2]));
    }
};

} // namespace

extern "C" {

/* fill_kitp_level_data (:521-565) at time t over the ghosted box. */
int ref_kitp_fill(const orc_params *p, const orc_kitp_disk *d,
                  const orc_box *b, double *state, double t)
{
    if (!usable(p, b) || !d || !no_modes(d))
        return ORC_ERR_INVALID_ARG;
    Lv lv(b);
    lv.load(state);
    fill_kitp_level_data(lv.state, factory_of(p), IdealGasEOS(p->gamma), t,
                         p->dx, centre_of(p), config_of(p, nullptr, d),
                         atmo_of(p));
    lv.store(state);
    return ORC_OK;
}

/* rhs (interior, 5 components, stride rcs) += add_kitp_viscous_rhs
 * (:772-806) or add_kitp_sink_rhs (:567-610) at time t (which = 0 / 1). */
int ref_kitp_source_rhs(const orc_params *p, const orc_kitp_config *k,
                        const orc_box *b, const double *state, double *rhs,
                        int64_t rcs, double t, int which)
{
    if (!usable(p, b) || !k)
        return ORC_ERR_INVALID_ARG;
    Lv lv(b);
    lv.load(state);
    FArrayBox r(lv.interior, NUM_VARS);
    r.setVal(0.0);
    for (BoxIterator bit(lv.interior); bit.ok(); ++bit)
        for (int c = 0; c < 5; ++c)
            r(bit(), c_GRHD_D + c) = rhs[c * rcs + lv.iat(bit())];
    const SimulationConfig c = config_of(p, k, nullptr);
    const BinaryState binary = make_binary_state(c, t);
    if (which == 0)
        add_kitp_viscous_rhs(r, lv.fab(), lv.interior, lv.domain_box, p->dx,
                             centre_of(p), binary, c, IdealGasEOS(p->gamma),
                             atmo_of(p));
    else
        add_kitp_sink_rhs(r, lv.fab(), lv.interior, p->dx, centre_of(p),
                          binary, c, atmo_of(p));
    for (BoxIterator bit(lv.interior); bit.ok(); ++bit)
        for (int c5 = 0; c5 < 5; ++c5)
            rhs[c5 * rcs + lv.iat(bit())] = r(bit(), c_GRHD_D + c5);
    return ORC_OK;
}

/* apply_kitp_sink_decay (:612-662). */
int ref_kitp_sink_decay(const orc_params *p, const orc_kitp_config *k,
                        const orc_box *b, double *state, double t, double dt)
{
    if (!usable(p, b) || !k)
        return ORC_ERR_INVALID_ARG;
    Lv lv(b);
    lv.load(state);
    apply_kitp_sink_decay(lv.state, t, dt, p->dx, centre_of(p),
                          config_of(p, k, nullptr));
    lv.store(state);
    return ORC_OK;
}

/* advance_kitp_ssprk2 (:842-876) with the driver's operator
 * (TimeDependentFixedBGLevelDataFiniteVolumeOperator, :1715-1721). */
int ref_kitp_advance_ssprk2(const orc_params *p, const orc_kitp_config *k,
                            const orc_box *b, double *state, double t,
                            double dt, orc_error *err)
{
    if (err)
        std::memset(err, 0, sizeof(*err));
    if (!usable(p, b) || !k)
        return ORC_ERR_INVALID_ARG;
    try
    {
        Lv lv(b);
        lv.load(state);
        const SimulationConfig c = config_of(p, k, nullptr);
        const IdealGasEOS eos(p->gamma);
        GRHD::TimeDependentFixedBGLevelDataFiniteVolumeOperator<
            IdealGasEOS, BinaryPNFactory>
            op(eos, factory_of(p), p->dx, centre_of(p), atmo_of(p),
               p->limiter_theta, p->use_reconstruction != 0, rec_of(p),
               p->use_static_metric_sources != 0,
               p->use_metric_volume_time_sources != 0,
               p->metric_time_derivative_step);
        Tensor<1, double> inv;
        FOR(dir) { inv[dir] = 1.0 / p->dx; }
        advance_kitp_ssprk2(op, lv.state, lv.domain, inv, t, dt, p->dx,
                            centre_of(p), c, eos, atmo_of(p));
        lv.store(state);
    }
    catch (const std::runtime_error &)
    {
        if (err)
            err->code = ORC_ERR_RECOVERY;
        return ORC_ERR_RECOVERY;
    }
    return ORC_OK;
}

} // extern "C"
