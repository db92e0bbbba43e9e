/*
 * ref_capi.cpp -- TEST INFRASTRUCTURE: GRDzhadzha's own GRHD operator
 * behind the oracle's C interface (grhd_oracle.h types, `ref_` names).
 *
 * The reference's headers (Source/Matter/GRHD, Source/Background) are
 * compiled unmodified, in place, against oracle/shim (the Chombo and
 * GRChombo names they use, written here from their call sites) by
 * oracle/Makefile into oracle/_ref/.  Nothing in the product library links,
 * loads or calls this code: it is the parity checker's reference and the
 * CPU baseline's reference implementation.
 *
 * A call copies the caller's 11-component ghosted box (grhd_oracle.h
 * layout) into a one-box LevelData<FArrayBox> of NUM_VARS components (the
 * GRHD components at c_GRHD_D.., Tests/GRHDFixedBGTest/UserVariables.hpp),
 * runs the reference operator's method
 * (FixedBGLevelDataFiniteVolumeOperator, FixedBGFArrayBoxFiniteVolume.hpp:
 * 446-614, or TimeDependentFixedBGLevelDataFiniteVolumeOperator, :677-830,
 * for the binary; LevelDataFiniteVolumeOperator, FArrayBoxFiniteVolume.hpp:
 * 1215-1364, for CCZ4-stored geometry) and copies the box back.  The
 * reference has no excision or accretion-rate diagnostic: calls with
 * those set return ORC_ERR_INVALID_ARG.
 *
 * The *_ranks entry points cut the box into z slabs and run one slab per
 * thread as its own one-box level, exchanging the slab ghosts between the
 * RHS evaluations as the reference's LevelData::exchange() does between
 * MPI ranks: the reference's parallel structure on the host cores.
 */
#include "grhd_oracle.h"

#include "CircularBinaryPN.hpp"
#include "FixedBGFArrayBoxFiniteVolume.hpp"
#include "IdealGasEOS.hpp"
#include "KerrSchild.hpp"
#include "UserVariables.hpp"

#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

namespace
{

struct BinaryFactory
{
    CircularBinaryPN::params_t params;
    double dx = 1.0;
    CircularBinaryPN operator()(double time) const
    {
        auto p = params;
        p.time += time;
        return CircularBinaryPN(p, dx);
    }
};

using StaticOp = GRHD::FixedBGLevelDataFiniteVolumeOperator<IdealGasEOS,
                                                            KerrSchild>;
using TimeOp =
    GRHD::TimeDependentFixedBGLevelDataFiniteVolumeOperator<IdealGasEOS,
                                                            BinaryFactory>;
using CCZ4Op = GRHD::LevelDataFiniteVolumeOperator<IdealGasEOS>;

std::array<double, CH_SPACEDIM> center_of(const orc_params *p)
{
    return {p->center[0], p->center[1], p->center[2]};
}

GRHD::AtmosphereOptions atmosphere_of(const orc_params *p)
{
    GRHD::AtmosphereOptions a;
    a.rho_floor = p->atmo_rho_floor;
    a.pressure_floor = p->atmo_pressure_floor;
    a.max_velocity_squared = p->atmo_max_velocity_squared;
    a.metric_source_atmosphere_factor =
        p->atmo_metric_source_atmosphere_factor;
    return a;
}

GRHD::RecoveryOptions recovery_of(const orc_params *p)
{
    GRHD::RecoveryOptions r;
    r.max_iterations = p->rec_max_iterations;
    r.tolerance = p->rec_tolerance;
    r.pressure_floor = p->rec_pressure_floor;
    r.max_velocity_squared = p->rec_max_velocity_squared;
    return r;
}

StaticOp static_op(const orc_params *p)
{
    KerrSchild::params_t k;
    k.mass = p->ks_mass;
    k.spin = p->ks_spin;
    k.center = center_of(p);
    return StaticOp(IdealGasEOS(p->gamma), KerrSchild(k, p->dx), p->dx,
                    center_of(p), atmosphere_of(p), p->limiter_theta,
                    p->use_reconstruction != 0, recovery_of(p),
                    p->use_static_metric_sources != 0);
}

TimeOp time_op(const orc_params *p)
{
    BinaryFactory f;
    f.params.mass_1 = p->pn_mass_1;
    f.params.mass_2 = p->pn_mass_2;
    f.params.separation = p->pn_separation;
    f.params.angular_velocity = p->pn_angular_velocity;
    f.params.phase = p->pn_phase;
    f.params.time = p->pn_time;
    f.params.softening_radius = p->pn_softening_radius;
    f.params.center = center_of(p);
    f.dx = p->dx;
    return TimeOp(IdealGasEOS(p->gamma), f, p->dx, center_of(p),
                  atmosphere_of(p), p->limiter_theta,
                  p->use_reconstruction != 0, recovery_of(p),
                  p->use_static_metric_sources != 0,
                  p->use_metric_volume_time_sources != 0,
                  p->metric_time_derivative_step);
}

CCZ4Op ccz4_op(const orc_params *p)
{
    return CCZ4Op(IdealGasEOS(p->gamma), atmosphere_of(p), p->limiter_theta,
                  p->use_reconstruction != 0, recovery_of(p),
                  p->use_static_metric_sources != 0);
}

/* The caller's box as a level: interior lo..hi, ghosts lo - glo (equal on
 * every side), domain dlo..dhi. */
struct Level
{
    Box domain_box;
    ProblemDomain domain;
    DisjointBoxLayout grids;
    IntVect ghost;

    explicit Level(const orc_box *b)
    {
        domain_box = Box(IntVect(b->dlo[0], b->dlo[1], b->dlo[2]),
                         IntVect(b->dhi[0], b->dhi[1], b->dhi[2]));
        domain = ProblemDomain(domain_box);
        Vector<Box> boxes(1);
        boxes[0] = Box(IntVect(b->lo[0], b->lo[1], b->lo[2]),
                       IntVect(b->hi[0], b->hi[1], b->hi[2]));
        Vector<int> procs(1, 0);
        grids = DisjointBoxLayout(boxes, procs, domain);
        ghost = IntVect(b->lo[0] - b->glo[0], b->lo[1] - b->glo[1],
                        b->lo[2] - b->glo[2]);
    }
};

bool box_ok(const orc_box *b)
{
    if (!b)
        return false;
    for (int d = 0; d < 3; ++d)
    {
        if (b->lo[d] > b->hi[d] || b->lo[d] - b->glo[d] != b->lo[0] - b->glo[0] ||
            b->ghi[d] - b->hi[d] != b->lo[0] - b->glo[0] ||
            b->lo[d] - b->glo[d] < 2)
            return false;
    }
    return true;
}

bool params_ok(const orc_params *p)
{
    return p && p->dx > 0.0 && !(p->excision_radius > 0.0) &&
           !(p->accretion_radius > 0.0);
}

int64_t cell_index(const orc_box *b, const IntVect &iv)
{
    const int64_t nx = b->ghi[0] - b->glo[0] + 1;
    const int64_t ny = b->ghi[1] - b->glo[1] + 1;
    return (iv[0] - b->glo[0]) + nx * ((iv[1] - b->glo[1]) +
                                       ny * (int64_t)(iv[2] - b->glo[2]));
}

/* components [c0, c0 + nc) of the caller's box <-> the level's fab from
 * component f0 on (every cell of the ghosted box) */
void load(const orc_box *b, const double *s, FArrayBox &fab, int c0, int nc,
          int f0)
{
    for (BoxIterator bit(fab.box()); bit.ok(); ++bit)
    {
        const int64_t i = cell_index(b, bit());
        for (int c = 0; c < nc; ++c)
            fab(bit(), f0 + c) = s[(c0 + c) * b->comp_stride + i];
    }
}

void store(const orc_box *b, double *s, const FArrayBox &fab, int c0, int nc,
           int f0)
{
    for (BoxIterator bit(fab.box()); bit.ok(); ++bit)
    {
        const int64_t i = cell_index(b, bit());
        for (int c = 0; c < nc; ++c)
            s[(c0 + c) * b->comp_stride + i] = fab(bit(), f0 + c);
    }
}

/* components [c0, c0 + nc) of `region` only */
void store_region(const orc_box *b, double *s, const FArrayBox &fab,
                  const Box &region, int c0, int nc, int f0)
{
    for (BoxIterator bit(region); bit.ok(); ++bit)
    {
        const int64_t i = cell_index(b, bit());
        for (int c = 0; c < nc; ++c)
            s[(c0 + c) * b->comp_stride + i] = fab(bit(), f0 + c);
    }
}

/* the 5 conserved RHS components over the interior, x fastest, stride rcs */
void store_rhs(const orc_box *b, double *rhs, int64_t rcs,
               const FArrayBox &fab, int f0)
{
    const Box interior(IntVect(b->lo[0], b->lo[1], b->lo[2]),
                       IntVect(b->hi[0], b->hi[1], b->hi[2]));
    const int64_t nx = b->hi[0] - b->lo[0] + 1, ny = b->hi[1] - b->lo[1] + 1;
    for (BoxIterator bit(interior); bit.ok(); ++bit)
    {
        const IntVect &iv = bit();
        const int64_t i = (iv[0] - b->lo[0]) +
                          nx * ((iv[1] - b->lo[1]) + ny * (iv[2] - b->lo[2]));
        for (int c = 0; c < 5; ++c)
            rhs[c * rcs + i] = fab(iv, f0 + c);
    }
}

void load_rhs(const orc_box *b, const double *rhs, int64_t rcs, FArrayBox &fab,
              int f0)
{
    fab.setVal(0.0);
    const Box interior(IntVect(b->lo[0], b->lo[1], b->lo[2]),
                       IntVect(b->hi[0], b->hi[1], b->hi[2]));
    const int64_t nx = b->hi[0] - b->lo[0] + 1, ny = b->hi[1] - b->lo[1] + 1;
    for (BoxIterator bit(interior); bit.ok(); ++bit)
    {
        const IntVect &iv = bit();
        const int64_t i = (iv[0] - b->lo[0]) +
                          nx * ((iv[1] - b->lo[1]) + ny * (iv[2] - b->lo[2]));
        for (int c = 0; c < 5; ++c)
            fab(iv, f0 + c) = rhs[c * rcs + i];
    }
}

/* "GRHD primitive recovery failed at (i,j,k) ... residual r": the
 * reference's exception as the oracle's error record */
int recovery_error(const std::exception &e, orc_error *err)
{
    if (!err)
        return ORC_ERR_RECOVERY;
    const std::string m = e.what();
    err->code = ORC_ERR_RECOVERY;
    err->where = m.find("outflow source") != std::string::npos
                     ? ORC_WHERE_OUTFLOW_SOURCE
                 : m.find("metric sources") != std::string::npos
                     ? ORC_WHERE_METRIC_SOURCES
                 : m.find("CFL") != std::string::npos
                     ? ORC_WHERE_CFL
                     : ORC_WHERE_GHOSTED_RECOVERY;
    const std::size_t at = m.find('(');
    if (at != std::string::npos)
        std::sscanf(m.c_str() + at, "(%d,%d,%d)", &err->cell[0],
                    &err->cell[1], &err->cell[2]);
    const std::size_t r = m.rfind("residual ");
    if (r != std::string::npos)
        err->residual = std::strtod(m.c_str() + r + 9, nullptr);
    return ORC_ERR_RECOVERY;
}

Tensor<1, double> inverse_dx(const double inv[3])
{
    Tensor<1, double> t;
    FOR(d) { t[d] = inv[d]; }
    return t;
}

void to_diag(const GRHD::AtmosphereResetDiagnostics &a, orc_diag *d)
{
    if (!d)
        return;
    d->num_cells += a.num_cells;
    d->num_failed_recoveries += a.num_failed_recoveries;
    d->num_floored_primitives += a.num_floored_primitives;
    d->num_conserved_resets += a.num_conserved_resets;
}

/* ---- the operator's methods on one level (the state in `st`) ---- */

void level_rhs(const orc_params *p, const Level &lv, LevelData<FArrayBox> &st,
               LevelData<FArrayBox> &rhs, const Tensor<1, double> &inv,
               double time)
{
    if (p->background == ORC_BG_BINARY_PN)
        time_op(p).compute_rhs(rhs, st, lv.domain, inv, time);
    else
        static_op(p).compute_rhs(rhs, st, lv.domain, inv);
}

GRHD::AtmosphereResetDiagnostics level_recover(const orc_params *p,
                                               LevelData<FArrayBox> &st,
                                               double time)
{
    if (p->background == ORC_BG_BINARY_PN)
        return time_op(p).recover_primitives(st, time);
    return static_op(p).recover_primitives(st);
}

double level_max_inverse_dt(const orc_params *p, const Level &lv,
                            const LevelData<FArrayBox> &st,
                            const Tensor<1, double> &inv, double time)
{
    if (p->background == ORC_BG_BINARY_PN)
        return time_op(p).compute_max_inverse_dt(st, lv.domain_box, inv,
                                                 time);
    return static_op(p).compute_max_inverse_dt(st, lv.domain_box, inv);
}

/* state += dt * rhs over the valid cells (add_scaled_conserved_rhs), then
 * the recovery when asked: the operator's update_conserved */
GRHD::AtmosphereResetDiagnostics
level_update(const orc_params *p, LevelData<FArrayBox> &st,
             const LevelData<FArrayBox> &rhs, double dt, double recovery_time,
             bool recover)
{
    const DisjointBoxLayout &grids = st.disjointBoxLayout();
    for (DataIterator dit = grids.dataIterator(); dit.ok(); ++dit)
        GRHD::add_scaled_conserved_rhs(st[dit], rhs[dit], grids[dit], dt);
    if (!recover)
        return GRHD::AtmosphereResetDiagnostics();
    return level_recover(p, st, recovery_time);
}

/* A reusable barrier for the rank threads; a rank that fails aborts it,
 * after which every wait returns false at once. */
class Barrier
{
  public:
    explicit Barrier(int n) : m_n(n) {}
    bool wait()
    {
        std::unique_lock<std::mutex> lock(m_mutex);
        if (m_aborted)
            return false;
        const long long gen = m_generation;
        if (++m_count == m_n)
        {
            m_count = 0;
            ++m_generation;
            m_cv.notify_all();
            return true;
        }
        m_cv.wait(lock, [&] { return gen != m_generation || m_aborted; });
        return !m_aborted;
    }
    void abort()
    {
        std::lock_guard<std::mutex> lock(m_mutex);
        m_aborted = true;
        m_cv.notify_all();
    }

  private:
    std::mutex m_mutex;
    std::condition_variable m_cv;
    int m_n, m_count = 0;
    long long m_generation = 0;
    bool m_aborted = false;
};

/* z slab s of n of the caller's box, as its own orc_box over the same
 * ghosted storage */
orc_box slab_of(const orc_box *b, int s, int n)
{
    orc_box x = *b;
    const int nz = b->hi[2] - b->lo[2] + 1;
    x.lo[2] = b->lo[2] + (int)((int64_t)nz * s / n);
    x.hi[2] = b->lo[2] + (int)((int64_t)nz * (s + 1) / n) - 1;
    x.glo[2] = x.lo[2] - (b->lo[2] - b->glo[2]);
    x.ghi[2] = x.hi[2] + (b->ghi[2] - b->hi[2]);
    return x;
}

/* One rank per z slab: every slab a one-box level of its own. */
struct Ranks
{
    const orc_params *p;
    const orc_box *b;
    int n;
    std::vector<orc_box> slab;
    std::vector<Level> level;
    std::vector<LevelData<FArrayBox>> state, stage, acc, k;
    Barrier barrier;
    std::vector<int> status;
    std::vector<orc_error> err;
    std::vector<orc_diag> diag;
    std::vector<double> maxinv;

    Ranks(const orc_params *pp, const orc_box *bb, int nn)
        : p(pp), b(bb), n(nn), barrier(nn), status(nn, ORC_OK), err(nn),
          diag(nn), maxinv(nn, 0.0)
    {
        for (int s = 0; s < n; ++s)
        {
            slab.push_back(slab_of(b, s, n));
            level.emplace_back(&slab[s]);
        }
        state.resize(n);
        stage.resize(n);
        acc.resize(n);
        k.resize(n);
        std::memset(err.data(), 0, sizeof(orc_error) * n);
        std::memset(diag.data(), 0, sizeof(orc_diag) * n);
    }

    /* ghost planes of slab s from its neighbours' valid planes (the other
     * ranks' part of LevelData::exchange()) */
    void exchange(std::vector<LevelData<FArrayBox>> &v, int s)
    {
        FArrayBox &mine = v[s][DataIndex(0)];
        for (int o = s - 1; o <= s + 1; o += 2)
        {
            if (o < 0 || o >= n)
                continue;
            const Box valid = level[o].grids[DataIndex(0)];
            const Box overlap = mine.box() & valid;
            if (!overlap.isEmpty())
                mine.copy(v[o][DataIndex(0)], overlap, 0, 0, NUM_VARS);
        }
    }
};

template <class F> int run_ranks(Ranks &r, F &&body)
{
    std::vector<std::thread> threads;
    for (int s = 0; s < r.n; ++s)
        threads.emplace_back([&r, &body, s] {
            try
            {
                body(s);
            }
            catch (const std::runtime_error &e)
            {
                r.status[s] = recovery_error(e, &r.err[s]);
                r.barrier.abort();
            }
        });
    for (auto &t : threads)
        t.join();
    for (int s = 0; s < r.n; ++s)
        if (r.status[s])
            return s;
    return -1;
}

} // namespace

extern "C" {

int ref_compute_rhs(const orc_params *p, const orc_box *b, double *state,
                    double *rhs, int64_t rcs, const double inv_dx[3],
                    double time, orc_error *err)
{
    if (err)
        std::memset(err, 0, sizeof(*err));
    if (!params_ok(p) || !box_ok(b))
        return ORC_ERR_INVALID_ARG;
    try
    {
        const Level lv(b);
        LevelData<FArrayBox> st(lv.grids, NUM_VARS, lv.ghost);
        LevelData<FArrayBox> r(lv.grids, NUM_VARS, IntVect::Zero);
        load(b, state, st[DataIndex(0)], 0, ORC_NCOMP, c_GRHD_D);
        level_rhs(p, lv, st, r, inverse_dx(inv_dx), time);
        store(b, state, st[DataIndex(0)], 0, ORC_NCOMP, c_GRHD_D);
        store_rhs(b, rhs, rcs, r[DataIndex(0)], c_GRHD_D);
    }
    catch (const std::runtime_error &e)
    {
        return recovery_error(e, err);
    }
    return ORC_OK;
}

int ref_recover_primitives(const orc_params *p, const orc_box *b,
                           double *state, double time, orc_diag *diag)
{
    if (diag)
        std::memset(diag, 0, sizeof(*diag));
    if (!params_ok(p) || !box_ok(b))
        return ORC_ERR_INVALID_ARG;
    const Level lv(b);
    LevelData<FArrayBox> st(lv.grids, NUM_VARS, lv.ghost);
    load(b, state, st[DataIndex(0)], 0, ORC_NCOMP, c_GRHD_D);
    to_diag(level_recover(p, st, time), diag);
    store(b, state, st[DataIndex(0)], 0, ORC_NCOMP, c_GRHD_D);
    return ORC_OK;
}

int ref_compute_max_inverse_dt(const orc_params *p, const orc_box *b,
                               const double *state, const double inv_dx[3],
                               double time, double *out, orc_error *err)
{
    if (err)
        std::memset(err, 0, sizeof(*err));
    if (!params_ok(p) || !box_ok(b) || !out)
        return ORC_ERR_INVALID_ARG;
    try
    {
        const Level lv(b);
        LevelData<FArrayBox> st(lv.grids, NUM_VARS, lv.ghost);
        load(b, state, st[DataIndex(0)], 0, ORC_NCOMP, c_GRHD_D);
        *out = level_max_inverse_dt(p, lv, st, inverse_dx(inv_dx), time);
    }
    catch (const std::runtime_error &e)
    {
        return recovery_error(e, err);
    }
    return ORC_OK;
}

int ref_update_conserved(const orc_params *p, const orc_box *b,
                         double *state, const double *rhs, int64_t rcs,
                         double dt, double recovery_time, int recover,
                         orc_diag *diag)
{
    if (diag)
        std::memset(diag, 0, sizeof(*diag));
    if (!params_ok(p) || !box_ok(b))
        return ORC_ERR_INVALID_ARG;
    const Level lv(b);
    LevelData<FArrayBox> st(lv.grids, NUM_VARS, lv.ghost);
    LevelData<FArrayBox> r(lv.grids, NUM_VARS, IntVect::Zero);
    load(b, state, st[DataIndex(0)], 0, ORC_NCOMP, c_GRHD_D);
    load_rhs(b, rhs, rcs, r[DataIndex(0)], c_GRHD_D);
    to_diag(level_update(p, st, r, dt, recovery_time, recover != 0), diag);
    store(b, state, st[DataIndex(0)], 0, ORC_NCOMP, c_GRHD_D);
    return ORC_OK;
}

int ref_advance_ssprk2(const orc_params *p, const orc_box *b, double *state,
                       const double inv_dx[3], double time, double dt,
                       orc_diag *diag, orc_error *err)
{
    if (diag)
        std::memset(diag, 0, sizeof(*diag));
    if (err)
        std::memset(err, 0, sizeof(*err));
    if (!params_ok(p) || !box_ok(b))
        return ORC_ERR_INVALID_ARG;
    try
    {
        const Level lv(b);
        LevelData<FArrayBox> st(lv.grids, NUM_VARS, lv.ghost);
        load(b, state, st[DataIndex(0)], 0, ORC_NCOMP, c_GRHD_D);
        if (p->background == ORC_BG_BINARY_PN)
            time_op(p).advance_ssprk2(st, lv.domain, inverse_dx(inv_dx), time,
                                      dt);
        else
            static_op(p).advance_ssprk2(st, lv.domain, inverse_dx(inv_dx),
                                        dt);
        store(b, state, st[DataIndex(0)], 0, ORC_NCOMP, c_GRHD_D);
    }
    catch (const std::runtime_error &e)
    {
        return recovery_error(e, err);
    }
    return ORC_OK;
}

/* The CFL bound and one classic RK4 step built from the operator's public
 * methods (compute_rhs, update_conserved), one z slab per thread, the slab
 * ghosts exchanged before every RHS: U_s = U^n + c_s dt k_s recovered at
 * the stage time for s = 1..3, then U^n + dt (k1 + 2 k2 + 2 k3 + k4) / 6
 * recovered at t + dt.  *max_inverse_dt receives the bound of U^n and dt
 * = cfl / that bound (capped by max_dt when max_dt > 0); at most nz / ghost
 * slabs (each at least as thick as the ghost layer).  The valid cells
 * of the box are updated; its ghost cells keep their input values. */
int ref_advance_rk4_cfl_ranks(const orc_params *p, const orc_box *b,
                              double *state, const double inv_dx[3],
                              double time, double cfl, double max_dt,
                              int ranks, double *max_inverse_dt,
                              double *dt_used, orc_diag *diag, orc_error *err)
{
    if (diag)
        std::memset(diag, 0, sizeof(*diag));
    if (err)
        std::memset(err, 0, sizeof(*err));
    // every slab at least as thick as the ghost layer: the reference fills
    // a ghost outside the domain from its own box's edge plane
    // (FixedBGFArrayBoxFiniteVolume.hpp:131-145), so a thinner box at a
    // domain edge would change the result with the slab count
    const int nz = b ? b->hi[2] - b->lo[2] + 1 : 0;
    const int ghost = b ? b->lo[2] - b->glo[2] : 1;
    if (!params_ok(p) || !box_ok(b) || ranks < 1 || ranks > nz / ghost ||
        !(cfl > 0.0))
        return ORC_ERR_INVALID_ARG;
    Ranks r(p, b, ranks);
    const Tensor<1, double> inv = inverse_dx(inv_dx);
    double dt = 0.0;
    const int bad = run_ranks(r, [&](int s) {
        const Level &lv = r.level[s];
        r.state[s].define(lv.grids, NUM_VARS, lv.ghost);
        r.stage[s].define(lv.grids, NUM_VARS, lv.ghost);
        r.acc[s].define(lv.grids, NUM_VARS, IntVect::Zero);
        r.k[s].define(lv.grids, NUM_VARS, IntVect::Zero);
        // the slab's ghosted box out of the caller's array (the caller's
        // box geometry indexes it)
        load(b, state, r.state[s][DataIndex(0)], 0, ORC_NCOMP, c_GRHD_D);
        // the stage state starts as U^n, ghosts included: ghosts inside the
        // domain but outside the caller's box keep the caller's values
        r.stage[s][DataIndex(0)].copy(r.state[s][DataIndex(0)]);
        r.maxinv[s] = level_max_inverse_dt(p, lv, r.state[s], inv, time);
        if (!r.barrier.wait())
            return;
        double mi = 0.0;
        for (int o = 0; o < r.n; ++o)
            mi = std::max(mi, r.maxinv[o]);
        double h = cfl / std::max(mi, 1.0e-14);
        if (max_dt > 0.0)
            h = std::min(h, max_dt);
        if (s == 0)
            dt = h;
        const double c[3] = {0.5 * h, 0.5 * h, h};
        const double w[4] = {h / 6.0, h / 3.0, h / 3.0, h / 6.0};
        const double ts[4] = {time, time + 0.5 * h, time + 0.5 * h, time + h};
        r.acc[s][DataIndex(0)].setVal(0.0);
        GRHD::AtmosphereResetDiagnostics d;
        for (int q = 0; q < 4; ++q)
        {
            LevelData<FArrayBox> &in = q == 0 ? r.state[s] : r.stage[s];
            level_rhs(p, lv, in, r.k[s], inv, ts[q]);
            // acc += w_q k_q over the valid cells
            const Box valid = lv.grids[DataIndex(0)];
            FArrayBox &a = r.acc[s][DataIndex(0)];
            const FArrayBox &kq = r.k[s][DataIndex(0)];
            for (BoxIterator bit(valid); bit.ok(); ++bit)
                for (int v = c_GRHD_D; v <= c_GRHD_tau; ++v)
                    a(bit(), v) += w[q] * kq(bit(), v);
            if (q < 3)
            {
                r.state[s].copyTo(r.stage[s]);
                d.add(level_update(p, r.stage[s], r.k[s], c[q], ts[q + 1],
                                   true));
                // every rank's stage is recovered before the exchange
                if (!r.barrier.wait())
                    return;
                r.exchange(r.stage, s);
                if (!r.barrier.wait())
                    return;
            }
        }
        d.add(level_update(p, r.state[s], r.acc[s], 1.0, time + h, true));
        GRHD::AtmosphereResetDiagnostics dd = d;
        orc_diag od{};
        to_diag(dd, &od);
        r.diag[s] = od;
        // each slab writes back its valid cells only; the caller's ghost
        // cells keep their input values
        store_region(b, state, r.state[s][DataIndex(0)],
                     lv.grids[DataIndex(0)], 0, ORC_NCOMP, c_GRHD_D);
    });
    if (bad >= 0)
    {
        if (err)
            *err = r.err[bad];
        return r.status[bad];
    }
    double mi = 0.0;
    for (int s = 0; s < r.n; ++s)
    {
        mi = std::max(mi, r.maxinv[s]);
        if (diag)
        {
            diag->num_cells += r.diag[s].num_cells;
            diag->num_failed_recoveries += r.diag[s].num_failed_recoveries;
            diag->num_floored_primitives += r.diag[s].num_floored_primitives;
            diag->num_conserved_resets += r.diag[s].num_conserved_resets;
        }
    }
    if (max_inverse_dt)
        *max_inverse_dt = mi;
    if (dt_used)
        *dt_used = dt;
    return ORC_OK;
}

/* ---- the operator on CCZ4-stored geometry (36 components: the 25 CCZ4
 * variables, then the 11 GRHD ones) ---- */

int ref_ccz4_compute_rhs(const orc_params *p, const orc_box *b, double *state,
                         double *rhs, int64_t rcs, const double inv_dx[3],
                         orc_error *err)
{
    if (err)
        std::memset(err, 0, sizeof(*err));
    if (!p || !(p->dx > 0.0) || !box_ok(b))
        return ORC_ERR_INVALID_ARG;
    try
    {
        const Level lv(b);
        LevelData<FArrayBox> st(lv.grids, NUM_VARS, lv.ghost);
        LevelData<FArrayBox> r(lv.grids, NUM_VARS, IntVect::Zero);
        load(b, state, st[DataIndex(0)], 0, NUM_VARS, 0);
        ccz4_op(p).compute_rhs(r, st, lv.domain, inverse_dx(inv_dx));
        store(b, state, st[DataIndex(0)], 0, NUM_VARS, 0);
        store_rhs(b, rhs, rcs, r[DataIndex(0)], c_GRHD_D);
    }
    catch (const std::runtime_error &e)
    {
        return recovery_error(e, err);
    }
    return ORC_OK;
}

int ref_ccz4_recover_primitives(const orc_params *p, const orc_box *b,
                                double *state, orc_diag *diag)
{
    if (diag)
        std::memset(diag, 0, sizeof(*diag));
    if (!p || !box_ok(b))
        return ORC_ERR_INVALID_ARG;
    const Level lv(b);
    LevelData<FArrayBox> st(lv.grids, NUM_VARS, lv.ghost);
    load(b, state, st[DataIndex(0)], 0, NUM_VARS, 0);
    to_diag(ccz4_op(p).recover_primitives(st), diag);
    store(b, state, st[DataIndex(0)], 0, NUM_VARS, 0);
    return ORC_OK;
}

int ref_ccz4_compute_max_inverse_dt(const orc_params *p, const orc_box *b,
                                    const double *state,
                                    const double inv_dx[3], double *out,
                                    orc_error *err)
{
    if (err)
        std::memset(err, 0, sizeof(*err));
    if (!p || !box_ok(b) || !out)
        return ORC_ERR_INVALID_ARG;
    try
    {
        const Level lv(b);
        LevelData<FArrayBox> st(lv.grids, NUM_VARS, lv.ghost);
        load(b, state, st[DataIndex(0)], 0, NUM_VARS, 0);
        *out = ccz4_op(p).compute_max_inverse_dt(st, lv.domain_box,
                                                 inverse_dx(inv_dx));
    }
    catch (const std::runtime_error &e)
    {
        return recovery_error(e, err);
    }
    return ORC_OK;
}

} // extern "C"
