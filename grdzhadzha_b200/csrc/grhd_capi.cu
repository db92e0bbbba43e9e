// grhd_capi.cu -- the extern "C" boundary (include/grhd_b200.h): context,
// scratch management, status/error reporting and the operator methods of
// the reference's FixedBGLevelDataFiniteVolumeOperator /
// TimeDependentFixedBGLevelDataFiniteVolumeOperator
// (Source/Matter/GRHD/FixedBGFArrayBoxFiniteVolume.hpp:446-830).
#include "grhd_b200.h"
#include "grhd_initial_data.cuh"
#include "grhd_kernels.cuh"
#include "grhd_io.cuh"
#include "grhd_kitp.cuh"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <mutex>
#include <new>
#include <vector>

using namespace grhd;

struct grhd_ctx
{
    grhd_params params;
    Options opt;
    int device;
    // scratch, grown on demand
    double *prim = nullptr;  // 5 comps over the ghosted box
    size_t prim_cap = 0;     // doubles
    double *src = nullptr;   // 5 comps over the interior
    double *kbuf = nullptr;  // 5 comps over the interior
    double *acc = nullptr;   // 5 comps over the interior
    size_t int_cap = 0;      // doubles per interior buffer
    double *stage = nullptr; // 11 comps over the ghosted box
    size_t stage_cap = 0;
    double *diag_part = nullptr;  // diagnostics: per-block partial results
    size_t diag_cap = 0;
    double *ccz4_geo = nullptr;   // CCZ4 operator: geometry cache (16 comps)
    size_t ccz4_geo_cap = 0;
    double *ccz4_stage = nullptr; // CCZ4 operator: SSPRK2 stage (36 comps)
    size_t ccz4_stage_cap = 0;
    double *host_state = nullptr; // device copy of a host-held state
    size_t host_state_cap = 0;
    double *prim2 = nullptr; // host-buffer step: second primitive cache
    size_t prim2_cap = 0;
    cudaStream_t h2d = nullptr, d2h = nullptr; // host-buffer step copies
    std::vector<cudaEvent_t> pipe_events;
    double *mdot_part = nullptr; // per face-kernel block accretion sums
    size_t mdot_cap = 0;
    double *mdot_acc = nullptr;  // [Mdot of the last RHS, time integral]
    DevStatus *status = nullptr;   // device
    DevStatus *status_h = nullptr; // pinned host mirror
    double *probe = nullptr;       // device scalars: probe + torus setup
    int *flag = nullptr;           // device flag (initial-data failures)
    int zchunk = 0; // face kernel z march: chosen per box (face_zchunk)
    grhd_error last_error;
    // instrumentation
    long long launches = 0;
    bool prof_on = false;
    struct ProfRec
    {
        cudaEvent_t a, b;
        int cls;
    };
    std::vector<ProfRec> prof_pending;
    std::vector<cudaEvent_t> event_pool;
};

namespace {

const unsigned long long kNoError = ~0ull;

cudaEvent_t take_event(grhd_ctx *ctx)
{
    if (!ctx->event_pool.empty())
    {
        cudaEvent_t e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Brackets one kernel launch: counts it and, when profiling is on, records
// a pair of events on its stream.
struct Timed
{
    grhd_ctx *ctx;
    cudaStream_t s;
    grhd_ctx::ProfRec rec;
    Timed(grhd_ctx *c, int cls, cudaStream_t st) : ctx(c), s(st)
    {
        ++ctx->launches;
        rec.cls = cls;
        rec.a = rec.b = nullptr;
        if (ctx->prof_on)
        {
            rec.a = take_event(ctx);
            rec.b = take_event(ctx);
            cudaEventRecord(rec.a, s);
        }
    }
    ~Timed()
    {
        if (rec.a)
        {
            cudaEventRecord(rec.b, s);
            ctx->prof_pending.push_back(rec);
        }
    }
};

int set_error(grhd_ctx *ctx, int status, int where, const int cell[3],
              double residual, const char *msg)
{
    grhd_error &e = ctx->last_error;
    e.status = status;
    e.where = where;
    for (int d = 0; d < 3; ++d)
        e.cell[d] = cell ? cell[d] : 0;
    e.residual = residual;
    std::snprintf(e.message, sizeof(e.message), "%s", msg ? msg : "");
    return status;
}

int cuda_error(grhd_ctx *ctx, cudaError_t err, const char *what)
{
    char buf[256];
    std::snprintf(buf, sizeof(buf), "CUDA error in %s: %s", what,
                  cudaGetErrorString(err));
    return set_error(ctx, GRHD_ERR_CUDA, GRHD_WHERE_NONE, nullptr, 0.0, buf);
}

#define GRHD_CUDA(ctx, call)                                                  \
    do                                                                        \
    {                                                                         \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess)                                                \
            return cuda_error((ctx), e_, #call);                              \
    } while (0)

Options make_options(const grhd_params &p)
{
    Options o;
    o.G = p.adiabatic_index;
    o.rho_floor = p.rho_floor;
    o.p_floor = p.pressure_floor;
    o.atmo_vmax2 = p.max_velocity_squared;
    o.src_atmo_factor = p.metric_source_atmosphere_factor;
    o.rec_maxit = p.recovery_max_iterations;
    o.rec_tol = p.recovery_tolerance;
    o.rec_pfloor = p.recovery_pressure_floor;
    o.rec_vmax2 = p.recovery_max_velocity_squared;
    o.theta = p.limiter_theta;
    o.use_recon = p.use_reconstruction;
    o.use_src = p.use_static_metric_sources;
    o.use_vol = p.use_metric_volume_time_sources;
    o.excision_radius = p.excision_radius;
    o.accretion_radius = p.accretion_radius;
    o.dx = p.dx;
    for (int d = 0; d < 3; ++d)
        o.center[d] = p.center[d];
    return o;
}

// CircularBinaryPN::compute_state (:219-250) at operator time t; the
// reference's background factory adds t to params.time
// (Tests/GRHDFixedBGTest/GRHDFixedBGTest.cpp:440-445).
void pn_state(const grhd_params &p, double t, double p1[3], double p2[3],
              double v1[3], double v2[3])
{
    const double total = p.pn_mass_1 + p.pn_mass_2;
    const double omega =
        p.pn_angular_velocity != 0.0
            ? p.pn_angular_velocity
            : std::sqrt(total / (p.pn_separation * p.pn_separation *
                                 p.pn_separation));
    const double phase = p.pn_phase + omega * (p.pn_time + t);
    const double c = std::cos(phase), s = std::sin(phase);
    const double r1 = p.pn_mass_2 / total * p.pn_separation;
    const double r2 = p.pn_mass_1 / total * p.pn_separation;
    for (int i = 0; i < 3; ++i)
        p1[i] = p2[i] = v1[i] = v2[i] = 0.0;
    p1[0] = r1 * c;
    p1[1] = r1 * s;
    p2[0] = -r2 * c;
    p2[1] = -r2 * s;
    v1[0] = -omega * r1 * s;
    v1[1] = omega * r1 * c;
    v2[0] = omega * r2 * s;
    v2[1] = -omega * r2 * c;
}

Background make_background(const grhd_params &p, double t)
{
    Background bg;
    std::memset(&bg, 0, sizeof(bg));
    bg.kind = p.background;
    bg.M = p.ks_mass;
    bg.a = p.ks_spin;
    if (p.background == GRHD_BG_BINARY_PN)
    {
        bg.m1 = p.pn_mass_1;
        bg.m2 = p.pn_mass_2;
        bg.soft2 = p.pn_softening_radius * p.pn_softening_radius;
        pn_state(p, t, bg.p1, bg.p2, bg.v1, bg.v2);
        // fixed_background_log_sqrt_det_time_derivative, :616-631
        const double h = std::fmax(p.metric_time_derivative_step, 1.0e-12);
        bg.fd_h = h;
        double vv1[3], vv2[3];
        pn_state(p, t + h, bg.p1p, bg.p2p, vv1, vv2);
        pn_state(p, t - h, bg.p1m, bg.p2m, vv1, vv2);
    }
    return bg;
}

bool valid_box(const grhd_box *b)
{
    if (!b || b->ghost < 2)
        return false;
    for (int d = 0; d < 3; ++d)
        if (b->lo[d] > b->hi[d] || b->domain_lo[d] > b->domain_hi[d])
            return false;
    return true;
}

BoxDev make_box(const grhd_box *b, int64_t state_cs)
{
    BoxDev x;
    for (int d = 0; d < 3; ++d)
    {
        x.lo[d] = b->lo[d];
        x.hi[d] = b->hi[d];
        x.glo[d] = b->lo[d] - b->ghost;
        x.ghi[d] = b->hi[d] + b->ghost;
        x.dlo[d] = b->domain_lo[d];
        x.dhi[d] = b->domain_hi[d];
        x.gn[d] = x.ghi[d] - x.glo[d] + 1;
        x.in[d] = x.hi[d] - x.lo[d] + 1;
    }
    x.cs = state_cs;
    x.rcs = x.ivol();
    x.pcs = x.gvol();
    return x;
}

int check_strides(grhd_ctx *ctx, const BoxDev &b, int64_t state_cs,
                  int64_t rhs_cs)
{
    const int cell[3] = {0, 0, 0};
    if (state_cs < b.gvol())
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, cell, 0.0,
                         "state component stride is smaller than the "
                         "ghosted box volume");
    if (rhs_cs >= 0 && rhs_cs < b.ivol())
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, cell, 0.0,
                         "rhs component stride is smaller than the interior "
                         "box volume");
    return GRHD_OK;
}

int grow(grhd_ctx *ctx, double **ptr, size_t *cap, size_t need)
{
    if (*cap >= need)
        return GRHD_OK;
    if (*ptr)
        cudaFree(*ptr);
    *ptr = nullptr;
    *cap = 0;
    GRHD_CUDA(ctx, cudaMalloc((void **)ptr, need * sizeof(double)));
    *cap = need;
    return GRHD_OK;
}

// blocks of one face-kernel launch over box b (its z march as chosen for
// the context's precision)
int64_t face_blocks(const grhd_ctx *ctx, const BoxDev &b)
{
    return face_kernel_blocks(b, ctx->zchunk,
                              ctx->params.precision == GRHD_PRECISION_MIXED);
}

int ensure_scratch(grhd_ctx *ctx, const BoxDev &b, bool need_stage)
{
    int st = grow(ctx, &ctx->prim, &ctx->prim_cap, 5 * (size_t)b.gvol());
    if (st)
        return st;
    const size_t ni = 5 * (size_t)b.ivol();
    if (ctx->int_cap < ni)
    {
        size_t c1 = ctx->int_cap, c2 = ctx->int_cap, c3 = ctx->int_cap;
        if ((st = grow(ctx, &ctx->src, &c1, ni)) ||
            (st = grow(ctx, &ctx->kbuf, &c2, ni)) ||
            (st = grow(ctx, &ctx->acc, &c3, ni)))
            return st;
        ctx->int_cap = ni;
    }
    if (need_stage &&
        (st = grow(ctx, &ctx->stage, &ctx->stage_cap,
                   kStateComps * (size_t)b.gvol())))
        return st;
    if (ctx->params.accretion_radius > 0.0)
        st = grow(ctx, &ctx->mdot_part, &ctx->mdot_cap,
                  (size_t)face_blocks(ctx, b));
    return st;
}

int reset_status(grhd_ctx *ctx, cudaStream_t s)
{
    DevStatus init;
    init.err_key = kNoError;
    for (int q = 0; q < 4; ++q)
        init.counts[q] = 0;
    init.maxinv_bits = 0;
    *ctx->status_h = init;
    GRHD_CUDA(ctx, cudaMemcpyAsync(ctx->status, ctx->status_h,
                                   sizeof(DevStatus), cudaMemcpyHostToDevice,
                                   s));
    return GRHD_OK;
}

// Reads the device status back (synchronising the stream) and converts a
// recorded recovery failure into the reference's exception data.
int finish_status(grhd_ctx *ctx, const BoxDev &b, const double *state,
                  const Background &bg, cudaStream_t s)
{
    GRHD_CUDA(ctx, cudaGetLastError());
    GRHD_CUDA(ctx, cudaMemcpyAsync(ctx->status_h, ctx->status,
                                   sizeof(DevStatus), cudaMemcpyDeviceToHost,
                                   s));
    GRHD_CUDA(ctx, cudaStreamSynchronize(s));
    const unsigned long long key = ctx->status_h->err_key;
    if (key == kNoError)
        return GRHD_OK;
    const int where = (int)(key >> 56);
    const int64_t order = (int64_t)(key & ((1ull << 56) - 1));
    int cell[3];
    int probe[3];
    if (where == GRHD_WHERE_CFL)
    {
        cell[0] = b.lo[0] + (int)(order % b.in[0]);
        cell[1] = b.lo[1] + (int)((order / b.in[0]) % b.in[1]);
        cell[2] = b.lo[2] + (int)(order / ((int64_t)b.in[0] * b.in[1]));
    }
    else
    {
        cell[0] = b.glo[0] + (int)(order % b.gn[0]);
        cell[1] = b.glo[1] + (int)((order / b.gn[0]) % b.gn[1]);
        cell[2] = b.glo[2] + (int)(order / ((int64_t)b.gn[0] * b.gn[1]));
    }
    for (int d = 0; d < 3; ++d)
        probe[d] = cell[d];
    if (where == GRHD_WHERE_OUTFLOW_SOURCE)
    {
        // the failing con2prim is at the clamped interior source cell
        for (int d = 0; d < 3; ++d)
        {
            if (cell[d] < b.dlo[d])
                probe[d] = b.lo[d];
            else if (cell[d] > b.dhi[d])
                probe[d] = b.hi[d];
        }
    }
    double residual = 0.0;
    launch_residual_probe(state, b, bg, ctx->opt, probe[0], probe[1],
                          probe[2], ctx->probe, s);
    GRHD_CUDA(ctx, cudaMemcpyAsync(&residual, ctx->probe, sizeof(double),
                                   cudaMemcpyDeviceToHost, s));
    GRHD_CUDA(ctx, cudaStreamSynchronize(s));
    char msg[256];
    const char *what =
        where == GRHD_WHERE_OUTFLOW_SOURCE
            ? "GRHD primitive recovery failed at outflow source (%d,%d,%d) "
              "while filling fixed-background boundary, residual %g"
        : where == GRHD_WHERE_CFL
            ? "GRHD primitive recovery failed at (%d,%d,%d) while computing "
              "fixed-background CFL speed, residual %g"
            : "GRHD primitive recovery failed at (%d,%d,%d) with residual %g "
              "on fixed background";
    std::snprintf(msg, sizeof(msg), what, probe[0], probe[1], probe[2],
                  residual);
    return set_error(ctx, GRHD_ERR_RECOVERY, where, probe, residual, msg);
}

void read_diag(const grhd_ctx *ctx, grhd_diagnostics *d)
{
    if (!d)
        return;
    d->num_cells += (long long)ctx->status_h->counts[0];
    d->num_failed_recoveries += (long long)ctx->status_h->counts[1];
    d->num_floored_primitives += (long long)ctx->status_h->counts[2];
    d->num_conserved_resets += (long long)ctx->status_h->counts[3];
}

// One RHS evaluation on the device (no synchronisation).  With
// `prepared` the interior primitive cache and sources were already
// written by the previous fused stage kernel for this state and time.
// `mdot_weight` is the weight of this RHS's accretion rate in the time
// integral (the stage weight times dt).
// The scratch buffers are allocated in doubles; the mixed path (T = float)
// uses their first half.
template <typename T> T *scratch(double *p) { return reinterpret_cast<T *>(p); }

template <typename T>
void enqueue_rhs(grhd_ctx *ctx, T *rhs, double *state, const BoxDev &b,
                 const Background &bg, const double inv_dx[3], cudaStream_t s,
                 bool prepared = false, double mdot_weight = 0.0)
{
    T *prim = scratch<T>(ctx->prim), *src = scratch<T>(ctx->src);
    {
        Timed t_(ctx, GRHD_K_GHOSTS, s);
        launch_fill_ghosts<T>(state, prim, b, bg, ctx->opt, ctx->status, s);
    }
    if (!prepared)
    {
        Timed t_(ctx, GRHD_K_CELLS, s);
        launch_cells<T>(state, prim, src, b, bg, ctx->opt, ctx->status, s);
    }
    {
        Timed t_(ctx, GRHD_K_FACES, s);
        launch_faces<T>(prim, src, rhs, b, bg, ctx->opt, inv_dx, ctx->zchunk,
                        ctx->mdot_part, s);
    }
    if (ctx->params.accretion_radius > 0.0)
    {
        ++ctx->launches;
        launch_mdot_sum(ctx->mdot_part, face_blocks(ctx, b),
                        mdot_weight, ctx->mdot_acc, s);
    }
}

bool box_is_domain(const grhd_box *b)
{
    for (int d = 0; d < 3; ++d)
        if (b->lo[d] != b->domain_lo[d] || b->hi[d] != b->domain_hi[d])
            return false;
    return true;
}

int common_checks(grhd_ctx *ctx, const void *state, const grhd_box *box)
{
    const int cell[3] = {0, 0, 0};
    if (!ctx)
        return GRHD_ERR_INVALID_ARG;
    std::memset(&ctx->last_error, 0, sizeof(ctx->last_error));
    if (!state || !valid_box(box))
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, cell, 0.0,
                         "invalid state pointer or box");
    if (!(ctx->params.dx > 0.0))
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, cell, 0.0,
                         "GRHD grid spacing must be positive");
    GRHD_CUDA(ctx, cudaSetDevice(ctx->device));
    return GRHD_OK;
}

} // namespace

extern "C" {

int grhd_abi_version(void) { return GRHD_B200_ABI_VERSION; }

void grhd_default_params(grhd_params *p)
{
    std::memset(p, 0, sizeof(*p));
    p->background = GRHD_BG_KERR_SCHILD;
    p->ks_mass = 1.0;
    p->ks_spin = 0.0;
    p->pn_mass_1 = 0.5;
    p->pn_mass_2 = 0.5;
    p->pn_separation = 10.0;
    p->pn_angular_velocity = 0.0;
    p->pn_phase = 0.0;
    p->pn_time = 0.0;
    p->pn_softening_radius = 0.5;
    p->adiabatic_index = 5.0 / 3.0;
    p->dx = 1.0;
    p->rho_floor = 1.0e-12;
    p->pressure_floor = 1.0e-12;
    p->max_velocity_squared = 1.0 - 1.0e-12;
    p->metric_source_atmosphere_factor = 1.0 + 1.0e-12;
    p->recovery_max_iterations = 50;
    p->recovery_tolerance = 1.0e-12;
    p->recovery_pressure_floor = 1.0e-12;
    p->recovery_max_velocity_squared = 1.0 - 1.0e-12;
    p->limiter_theta = 1.5;
    p->use_reconstruction = 1;
    p->use_static_metric_sources = 1;
    p->use_metric_volume_time_sources = 0;
    p->metric_time_derivative_step = 1.0e-3;
    p->excision_radius = 0.0;
    p->accretion_radius = 0.0;
    p->precision = GRHD_PRECISION_FP64;
}

const char *grhd_status_string(int status)
{
    switch (status)
    {
    case GRHD_OK:
        return "ok";
    case GRHD_ERR_RECOVERY:
        return "primitive recovery failed";
    case GRHD_ERR_INVALID_ARG:
        return "invalid argument";
    case GRHD_ERR_CUDA:
        return "CUDA error";
    case GRHD_ERR_SETUP:
        return "setup failed";
    default:
        return "unknown status";
    }
}

int grhd_create(const grhd_params *params, grhd_ctx **out)
{
    if (!params || !out)
        return GRHD_ERR_INVALID_ARG;
    *out = nullptr;
    if (!(params->dx > 0.0))
        return GRHD_ERR_INVALID_ARG;
    if (params->background == GRHD_BG_KERR_SCHILD &&
        (params->ks_spin > params->ks_mass ||
         params->ks_spin < -params->ks_mass))
        return GRHD_ERR_INVALID_ARG; // KerrSchild.hpp:81-90
    if (params->background == GRHD_BG_BINARY_PN &&
        (params->pn_mass_1 <= 0.0 || params->pn_mass_2 <= 0.0 ||
         params->pn_separation <= 0.0 || params->pn_softening_radius < 0.0))
        return GRHD_ERR_INVALID_ARG; // CircularBinaryPN.hpp:49-57
    if (params->background != GRHD_BG_KERR_SCHILD &&
        params->background != GRHD_BG_BINARY_PN)
        return GRHD_ERR_INVALID_ARG;
    if (params->precision != GRHD_PRECISION_FP64 &&
        params->precision != GRHD_PRECISION_MIXED)
        return GRHD_ERR_INVALID_ARG;
    grhd_ctx *ctx = new (std::nothrow) grhd_ctx();
    if (!ctx)
        return GRHD_ERR_SETUP;
    ctx->params = *params;
    ctx->opt = make_options(*params);
    std::memset(&ctx->last_error, 0, sizeof(ctx->last_error));
    if (cudaGetDevice(&ctx->device) != cudaSuccess ||
        configure_kernels() != cudaSuccess ||
        cudaMalloc((void **)&ctx->status, sizeof(DevStatus)) != cudaSuccess ||
        cudaMallocHost((void **)&ctx->status_h, sizeof(DevStatus)) !=
            cudaSuccess ||
        cudaMalloc((void **)&ctx->probe, 8 * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void **)&ctx->flag, sizeof(int)) != cudaSuccess ||
        cudaMalloc((void **)&ctx->mdot_acc, 2 * sizeof(double)) !=
            cudaSuccess ||
        cudaMemset(ctx->mdot_acc, 0, 2 * sizeof(double)) != cudaSuccess)
    {
        grhd_destroy(ctx);
        return GRHD_ERR_CUDA;
    }
    *out = ctx;
    return GRHD_OK;
}

void grhd_destroy(grhd_ctx *ctx)
{
    if (!ctx)
        return;
    cudaFree(ctx->prim);
    cudaFree(ctx->src);
    cudaFree(ctx->kbuf);
    cudaFree(ctx->acc);
    cudaFree(ctx->stage);
    cudaFree(ctx->status);
    cudaFree(ctx->probe);
    cudaFree(ctx->flag);
    cudaFree(ctx->mdot_part);
    cudaFree(ctx->mdot_acc);
    cudaFree(ctx->diag_part);
    cudaFree(ctx->ccz4_geo);
    cudaFree(ctx->ccz4_stage);
    cudaFree(ctx->host_state);
    cudaFree(ctx->prim2);
    if (ctx->h2d)
        cudaStreamDestroy(ctx->h2d);
    if (ctx->d2h)
        cudaStreamDestroy(ctx->d2h);
    for (cudaEvent_t e : ctx->pipe_events)
        cudaEventDestroy(e);
    if (ctx->status_h)
        cudaFreeHost(ctx->status_h);
    for (auto &r : ctx->prof_pending)
    {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (cudaEvent_t e : ctx->event_pool)
        cudaEventDestroy(e);
    delete ctx;
}

int grhd_last_error(const grhd_ctx *ctx, grhd_error *out)
{
    if (!ctx || !out)
        return GRHD_ERR_INVALID_ARG;
    *out = ctx->last_error;
    return GRHD_OK;
}

int grhd_compute_rhs(grhd_ctx *ctx, double *rhs, int64_t rhs_cs,
                     double *state, int64_t state_cs, const grhd_box *box,
                     const double inverse_dx[3], double time, void *stream)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    if (!rhs || !inverse_dx)
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "null rhs or inverse_dx");
    cudaStream_t s = (cudaStream_t)stream;
    const BoxDev b = make_box(box, state_cs);
    if ((st = check_strides(ctx, b, state_cs, rhs_cs)) ||
        (st = ensure_scratch(ctx, b, false)) || (st = reset_status(ctx, s)))
        return st;
    const Background bg = make_background(ctx->params, time);
    // the face kernel writes with the interior-volume stride; a caller
    // stride that differs, or the mixed path's FP32 RHS, goes through the
    // k scratch buffer
    if (ctx->params.precision == GRHD_PRECISION_MIXED)
    {
        enqueue_rhs<float>(ctx, scratch<float>(ctx->kbuf), state, b, bg,
                           inverse_dx, s);
        ++ctx->launches;
        launch_widen(scratch<float>(ctx->kbuf), b.ivol(), rhs, rhs_cs, s);
    }
    else if (rhs_cs == b.ivol())
        enqueue_rhs<double>(ctx, rhs, state, b, bg, inverse_dx, s);
    else
    {
        enqueue_rhs<double>(ctx, ctx->kbuf, state, b, bg, inverse_dx, s);
        for (int c = 0; c < 5; ++c)
            GRHD_CUDA(ctx, cudaMemcpyAsync(rhs + c * rhs_cs,
                                           ctx->kbuf + c * b.ivol(),
                                           b.ivol() * sizeof(double),
                                           cudaMemcpyDeviceToDevice, s));
    }
    return finish_status(ctx, b, state, bg, s);
}

int grhd_recover_primitives(grhd_ctx *ctx, double *state, int64_t state_cs,
                            const grhd_box *box, double time,
                            grhd_diagnostics *diag, void *stream)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    cudaStream_t s = (cudaStream_t)stream;
    const BoxDev b = make_box(box, state_cs);
    if ((st = check_strides(ctx, b, state_cs, -1)) ||
        (st = reset_status(ctx, s)))
        return st;
    const Background bg = make_background(ctx->params, time);
    {
        Timed t_(ctx, GRHD_K_STAGE, s);
        launch_recover(state, b, bg, ctx->opt, ctx->status, s);
    }
    st = finish_status(ctx, b, state, bg, s);
    read_diag(ctx, diag);
    return st;
}

int grhd_update_conserved(grhd_ctx *ctx, double *state, int64_t state_cs,
                          const double *rhs, int64_t rhs_cs,
                          const grhd_box *box, double dt,
                          double recovery_time, int recover,
                          grhd_diagnostics *diag, void *stream)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    if (!rhs)
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "null rhs");
    cudaStream_t s = (cudaStream_t)stream;
    BoxDev b = make_box(box, state_cs);
    b.rcs = rhs_cs;
    if ((st = check_strides(ctx, b, state_cs, rhs_cs)) ||
        (st = reset_status(ctx, s)))
        return st;
    const Background bg = make_background(ctx->params, recovery_time);
    {
        Timed t_(ctx, GRHD_K_STAGE, s);
        launch_update(state, b.cs, state, b.cs, rhs, b, bg, ctx->opt, dt,
                      recover, ctx->status, s);
    }
    st = finish_status(ctx, b, state, bg, s);
    read_diag(ctx, diag);
    return st;
}

int grhd_compute_max_inverse_dt(grhd_ctx *ctx, const double *state,
                                int64_t state_cs, const grhd_box *box,
                                const double inverse_dx[3], double time,
                                double *out, void *stream)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    if (!out || !inverse_dx)
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "null output or inverse_dx");
    cudaStream_t s = (cudaStream_t)stream;
    const BoxDev b = make_box(box, state_cs);
    if ((st = check_strides(ctx, b, state_cs, -1)) ||
        (st = reset_status(ctx, s)))
        return st;
    const Background bg = make_background(ctx->params, time);
    {
        Timed t_(ctx, GRHD_K_CFL, s);
        launch_max_inv_dt(state, b, bg, ctx->opt, inverse_dx, ctx->status,
                          ctx->params.precision == GRHD_PRECISION_MIXED, s);
    }
    st = finish_status(ctx, b, state, bg, s);
    if (st)
        return st;
    double v;
    const unsigned long long bits = ctx->status_h->maxinv_bits;
    std::memcpy(&v, &bits, sizeof(v));
    *out = v;
    return GRHD_OK;
}

int grhd_compute_stable_dt(grhd_ctx *ctx, const double *state,
                           int64_t state_cs, const grhd_box *box,
                           const double inverse_dx[3], double cfl,
                           double time, double *out, void *stream)
{
    if (ctx && !(cfl > 0.0))
    {
        std::memset(&ctx->last_error, 0, sizeof(ctx->last_error));
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "GRHD CFL number must be positive");
    }
    double m = 0.0;
    int st = grhd_compute_max_inverse_dt(ctx, state, state_cs, box,
                                         inverse_dx, time, &m, stream);
    if (st)
        return st;
    *out = cfl / std::fmax(m, 1.0e-14);
    return GRHD_OK;
}

} // extern "C"

namespace {

int advance_checks(grhd_ctx *ctx, double *state, int64_t state_cs,
                   const grhd_box *box, const double inverse_dx[3],
                   BoxDev &b, cudaStream_t s)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    if (!inverse_dx || !box_is_domain(box))
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "advance needs the box to cover the whole domain");
    b = make_box(box, state_cs);
    if ((st = check_strides(ctx, b, state_cs, -1)) ||
        (st = ensure_scratch(ctx, b, true)) || (st = reset_status(ctx, s)))
        return st;
    return GRHD_OK;
}

double bits_to_double(unsigned long long bits)
{
    double v;
    std::memcpy(&v, &bits, sizeof(v));
    return v;
}

// advance_ssprk2 (:563-589 / :782-809): rhs_initial = L(state); stage =
// state + dt rhs_initial recovered at t + dt, fused with the primitive
// cache and sources of L(stage); then the SSPRK2 combination.
template <typename T>
void enqueue_ssprk2(grhd_ctx *ctx, double *state, const BoxDev &b,
                    const double inverse_dx[3], double time, double dt,
                    cudaStream_t s)
{
    BoxDev sb = b; // the stage buffer is packed: stride = ghosted volume
    sb.cs = b.gvol();
    const Background bg0 = make_background(ctx->params, time);
    const Background bg1 = make_background(ctx->params, time + dt);
    T *k = scratch<T>(ctx->kbuf), *prim = scratch<T>(ctx->prim),
      *src = scratch<T>(ctx->src);
    enqueue_rhs<T>(ctx, k, state, b, bg0, inverse_dx, s, false, 0.5 * dt);
    {
        Timed t_(ctx, GRHD_K_STAGE, s);
        launch_stage<T>(1, state, b.cs, nullptr, 0, ctx->stage, sb.cs, k,
                        nullptr, prim, src, true, b, bg1, ctx->opt, 0, dt,
                        false, inverse_dx, ctx->status, s);
    }
    enqueue_rhs<T>(ctx, k, ctx->stage, sb, bg1, inverse_dx, s, true, 0.5 * dt);
    {
        Timed t_(ctx, GRHD_K_STAGE, s);
        launch_stage<T>(2, state, b.cs, ctx->stage, sb.cs, state, b.cs, k,
                        nullptr, prim, nullptr, false, b, bg1, ctx->opt, 0, dt,
                        false, inverse_dx, ctx->status, s);
    }
}

// Classic RK4 (new): stage RHS times t, t+dt/2, t+dt/2, t+dt; every stage
// combination is fused with the post-update recovery at the next RHS time
// and with that RHS's per-cell work; the last stage optionally computes the
// next CFL speed.  No host synchronisation.
// prepped_in: the primitive cache and sources already hold the first
// RHS's per-cell pass (done by the previous step's last stage); prep_out:
// the last stage does that pass for the next step.
template <typename T>
void enqueue_rk4(grhd_ctx *ctx, double *state, const BoxDev &b,
                 const double inverse_dx[3], double time, double dt,
                 bool want_cfl, cudaStream_t s, bool prepped_in = false,
                 bool prep_out = false)
{
    BoxDev sb = b;
    sb.cs = b.gvol();
    const Background bgs[4] = {
        make_background(ctx->params, time),
        make_background(ctx->params, time + 0.5 * dt),
        make_background(ctx->params, time + 0.5 * dt),
        make_background(ctx->params, time + dt)};
    T *k = scratch<T>(ctx->kbuf), *prim = scratch<T>(ctx->prim),
      *src = scratch<T>(ctx->src);
    for (int stage = 0; stage < 4; ++stage)
    {
        const double w = (dt / 6.0) * ((stage == 1 || stage == 2) ? 2.0 : 1.0);
        if (stage == 0)
            enqueue_rhs<T>(ctx, k, state, b, bgs[0], inverse_dx, s,
                           prepped_in, w);
        else
            enqueue_rhs<T>(ctx, k, ctx->stage, sb, bgs[stage], inverse_dx, s,
                           true, w);
        Timed t_(ctx, GRHD_K_STAGE, s);
        if (stage < 3)
            launch_stage<T>(0, state, b.cs, nullptr, 0, ctx->stage, sb.cs, k,
                            ctx->acc, prim, src, true, b, bgs[stage + 1],
                            ctx->opt, stage, dt, false, inverse_dx,
                            ctx->status, s);
        else
            launch_stage<T>(0, state, b.cs, nullptr, 0, state, b.cs, k,
                            ctx->acc, prim, prep_out ? src : nullptr,
                            prep_out ? 3 : 0, b, bgs[3], ctx->opt, stage, dt,
                            want_cfl, inverse_dx, ctx->status, s);
    }
}

void enqueue_rk4_any(grhd_ctx *ctx, double *state, const BoxDev &b,
                     const double inverse_dx[3], double time, double dt,
                     bool want_cfl, cudaStream_t s, bool prepped_in = false,
                     bool prep_out = false)
{
    if (ctx->params.precision == GRHD_PRECISION_MIXED)
        enqueue_rk4<float>(ctx, state, b, inverse_dx, time, dt, want_cfl, s,
                           prepped_in, prep_out);
    else
        enqueue_rk4<double>(ctx, state, b, inverse_dx, time, dt, want_cfl, s,
                            prepped_in, prep_out);
}

// advance_ssprk2 (:563-589) cut at its two RHS evaluations, for a level
// whose ghosts the caller exchanges in between: stage 1 stage_state =
// state + dt L(state), recovered at t + dt; stage 2 state = (state +
// stage_state + dt L(stage_state)) / 2 (combine_ssprk2_conserved_state),
// recovered.  The same kernels as the fused single-box step, without the
// fusion of the stage with the next RHS's per-cell pass.
template <typename T>
void enqueue_ssprk2_stage(grhd_ctx *ctx, int stage, double *state,
                          const BoxDev &b, double *stage_state,
                          const BoxDev &sb, const Background &bg0,
                          const Background &bg1, const double inverse_dx[3],
                          double dt, cudaStream_t s)
{
    T *k = scratch<T>(ctx->kbuf), *prim = scratch<T>(ctx->prim),
      *src = scratch<T>(ctx->src);
    if (stage == 1)
    {
        enqueue_rhs<T>(ctx, k, state, b, bg0, inverse_dx, s, false, 0.5 * dt);
        Timed t_(ctx, GRHD_K_STAGE, s);
        launch_stage<T>(1, state, b.cs, nullptr, 0, stage_state, sb.cs, k,
                        nullptr, prim, src, false, b, bg1, ctx->opt, 0, dt,
                        false, inverse_dx, ctx->status, s);
    }
    else
    {
        enqueue_rhs<T>(ctx, k, stage_state, sb, bg1, inverse_dx, s, false,
                       0.5 * dt);
        Timed t_(ctx, GRHD_K_STAGE, s);
        launch_stage<T>(2, state, b.cs, stage_state, sb.cs, state, b.cs, k,
                        nullptr, prim, nullptr, false, b, bg1, ctx->opt, 0, dt,
                        false, inverse_dx, ctx->status, s);
    }
}

// ---- the operator on CCZ4-stored geometry (LevelDataFiniteVolumeOperator,
// FArrayBoxFiniteVolume.hpp:1215-1364)

// The device status of a CCZ4 call as the reference's exceptions.
int ccz4_finish(grhd_ctx *ctx, const BoxDev &b, const double *state,
                cudaStream_t s)
{
    GRHD_CUDA(ctx, cudaGetLastError());
    GRHD_CUDA(ctx, cudaMemcpyAsync(ctx->status_h, ctx->status,
                                   sizeof(DevStatus), cudaMemcpyDeviceToHost,
                                   s));
    GRHD_CUDA(ctx, cudaStreamSynchronize(s));
    const unsigned long long key = ctx->status_h->err_key;
    if (key == kNoError)
        return GRHD_OK;
    const int where = (int)(key >> 56);
    const int64_t order = (int64_t)(key & ((1ull << 56) - 1));
    int cell[3];
    if (where == GRHD_WHERE_CFL)
    {
        cell[0] = b.lo[0] + (int)(order % b.in[0]);
        cell[1] = b.lo[1] + (int)((order / b.in[0]) % b.in[1]);
        cell[2] = b.lo[2] + (int)(order / ((int64_t)b.in[0] * b.in[1]));
    }
    else
    {
        cell[0] = b.glo[0] + (int)(order % b.gn[0]);
        cell[1] = b.glo[1] + (int)((order / b.gn[0]) % b.gn[1]);
        cell[2] = b.glo[2] + (int)(order / ((int64_t)b.gn[0] * b.gn[1]));
    }
    double residual = 0.0;
    launch_ccz4_probe(state, b, ctx->opt, cell[0], cell[1], cell[2],
                      ctx->probe, s);
    GRHD_CUDA(ctx, cudaMemcpyAsync(&residual, ctx->probe, sizeof(double),
                                   cudaMemcpyDeviceToHost, s));
    GRHD_CUDA(ctx, cudaStreamSynchronize(s));
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  where == GRHD_WHERE_CFL
                      ? "GRHD primitive recovery failed at (%d,%d,%d) while "
                        "computing CFL speed, residual %g"
                      : "GRHD primitive recovery failed at (%d,%d,%d) with "
                        "residual %g",
                  cell[0], cell[1], cell[2], residual);
    return set_error(ctx, GRHD_ERR_RECOVERY, where, cell, residual, msg);
}

int ccz4_checks(grhd_ctx *ctx, const double *state, int64_t state_cs,
                const grhd_box *box, int64_t rhs_cs, BoxDev &b,
                cudaStream_t s)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    b = make_box(box, state_cs);
    if ((st = check_strides(ctx, b, state_cs, rhs_cs)) ||
        (st = ensure_scratch(ctx, b, false)) ||
        (st = grow(ctx, &ctx->ccz4_geo, &ctx->ccz4_geo_cap,
                   16 * (size_t)b.gvol())) ||
        (st = reset_status(ctx, s)))
        return st;
    return GRHD_OK;
}

// compute_leveldata_flux_rhs_from_ccz4_geometry (:1047-1090) on one box:
// the fills, the ghosted-box recovery into the caches, then one kernel for
// the three directional flux differences and the sources.
void enqueue_ccz4_rhs(grhd_ctx *ctx, double *rhs, int64_t rhs_cs,
                      double *state, const BoxDev &b,
                      const double inverse_dx[3], cudaStream_t s)
{
    launch_ccz4_fill(state, b, true, s);
    launch_ccz4_cells(state, b, ctx->opt, ctx->prim, ctx->ccz4_geo,
                      ctx->status, s);
    launch_ccz4_rhs(state, b, ctx->opt, ctx->prim, ctx->ccz4_geo, rhs, rhs_cs,
                    inverse_dx, ctx->status, s);
    ctx->launches += 3;
}

// ---- the host-buffer RK4 step as a wavefront over z chunks

// Chunk c of n: interior planes k0(c)..k1(c) (len planes from lo[2]); its
// copies carry the ghosted planes plo(c)..phi(c) (the ghost planes below
// and above the interior go with the first and the last chunk).  About 24
// chunks of at least 8 planes: the copy out of the first chunk starts
// after 4 of them have been through the stages, the last chunk's copy out
// is all that follows the computation (measured on B200 at 256^3 FP64:
// 48.4 ms per step with 8 chunks, 46.5 with 24, 55.3 with 32; mixed 40.7,
// 36.0, 34.4 with 8, 16, 32).
struct ZChunks
{
    int lo2, hi2, glo2, ghi2, len, n;
    int k0(int c) const { return lo2 + c * len; }
    int k1(int c) const { return std::min(lo2 + (c + 1) * len - 1, hi2); }
    int plo(int c) const { return c == 0 ? glo2 : k0(c); }
    int phi(int c) const { return c == n - 1 ? ghi2 : k1(c); }
};

ZChunks make_zchunks(const BoxDev &b)
{
    ZChunks z;
    z.lo2 = b.lo[2];
    z.hi2 = b.hi[2];
    z.glo2 = b.glo[2];
    z.ghi2 = b.ghi[2];
    z.len = std::max(8, (b.in[2] + 23) / 24);
    z.n = (b.in[2] + z.len - 1) / z.len;
    return z;
}

// The interior planes k0..k1 of b as a box of their own (BoxDev::t0).
BoxDev chunk_view(const BoxDev &b, int k0, int k1)
{
    BoxDev v = b;
    v.lo[2] = k0;
    v.hi[2] = k1;
    v.in[2] = k1 - k0 + 1;
    v.t0 = b.t0 + (int64_t)(k0 - b.lo[2]) * b.in[0] * b.in[1];
    return v;
}

int pipe_setup(grhd_ctx *ctx, int nchunks)
{
    if (!ctx->h2d)
        GRHD_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->h2d,
                                                 cudaStreamNonBlocking));
    if (!ctx->d2h)
        GRHD_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->d2h,
                                                 cudaStreamNonBlocking));
    while (ctx->pipe_events.size() < 2 * (size_t)nchunks + 1)
    {
        cudaEvent_t e;
        GRHD_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->pipe_events.push_back(e);
    }
    return GRHD_OK;
}

// One RK4 step (the kernels of enqueue_rk4, want_cfl) of the state in
// pinned host memory `host` through its device copy `dev`, as a wavefront
// over z chunks.  Iteration w copies chunk w in (on its own stream, all
// chunks queued at once), computes its con2prim and sources once its copy
// has landed, then runs RK stage s on chunk w-1-s for s = 0..3: the
// ghost cells of the chunk's planes, its fluxes, its stage kernel.  Stage
// s on chunk j reads stage-s primitives two planes into chunks j-1 and
// j+1; those were written earlier in the same or the previous iteration,
// and the stages alternate between two primitive caches (stage s reads
// one and prepares stage s+1's in the other) so that no chunk's stage-s
// primitives are overwritten before its neighbour's stage-s fluxes have
// read them.  Chunk j's copy out (every component of its ghosted planes)
// starts as soon as its last stage is done.  Every cell sees exactly the
// arithmetic of the whole-box step: the result is bit-identical.  The
// excised planes ek0..ek1 carry their primitives in (empty when ek0 > ek1).
template <typename T>
int enqueue_rk4_host_pipelined(grhd_ctx *ctx, double *host, double *dev,
                               const BoxDev &b, const double inv_dx[3],
                               double time, double dt, int ek0, int ek1,
                               cudaStream_t s, long long &in, long long &out)
{
    const ZChunks z = make_zchunks(b);
    int st = pipe_setup(ctx, z.n);
    if (st)
        return st;
    cudaEvent_t *ev_in = ctx->pipe_events.data();
    cudaEvent_t *ev_out = ev_in + z.n;
    cudaEvent_t ev_start = ev_in[2 * z.n];
    const bool mixed = sizeof(T) != sizeof(double);
    const size_t cs = (size_t)b.cs;
    const size_t plane = (size_t)b.gn[0] * b.gn[1];
    GRHD_CUDA(ctx, cudaEventRecord(ev_start, s));
    GRHD_CUDA(ctx, cudaStreamWaitEvent(ctx->h2d, ev_start, 0));
    for (int c = 0; c < z.n; ++c)
    {
        const int p0 = z.plo(c), p1 = z.phi(c);
        for (int q = 0; q < kStateComps; ++q)
        {
            int q0 = p0, q1 = p1;
            if (q >= 5 && !(mixed && q == kPress))
            {
                q0 = std::max(ek0, p0);
                q1 = std::min(ek1, p1);
                if (q0 > q1)
                    continue;
            }
            const size_t off = (size_t)(q0 - b.glo[2]) * plane;
            const size_t n = (size_t)(q1 - q0 + 1) * plane;
            GRHD_CUDA(ctx, cudaMemcpyAsync(dev + q * cs + off,
                                           host + q * cs + off,
                                           n * sizeof(double),
                                           cudaMemcpyHostToDevice, ctx->h2d));
            in += (long long)(n * sizeof(double));
        }
        GRHD_CUDA(ctx, cudaEventRecord(ev_in[c], ctx->h2d));
    }
    BoxDev sb = b;
    sb.cs = b.gvol();
    const Background bgs[4] = {
        make_background(ctx->params, time),
        make_background(ctx->params, time + 0.5 * dt),
        make_background(ctx->params, time + 0.5 * dt),
        make_background(ctx->params, time + dt)};
    T *P[2] = {scratch<T>(ctx->prim), scratch<T>(ctx->prim2)};
    T *k = scratch<T>(ctx->kbuf), *src = scratch<T>(ctx->src);
    double *acc = ctx->acc;
    // the z march of each chunk's face blocks chosen for the chunk
    const int zc = ctx->zchunk;
    for (int w = 0; w < z.n + 4; ++w)
    {
        if (w < z.n)
        {
            GRHD_CUDA(ctx, cudaStreamWaitEvent(s, ev_in[w], 0));
            const BoxDev v = chunk_view(b, z.k0(w), z.k1(w));
            Timed t_(ctx, GRHD_K_CELLS, s);
            launch_cells<T>(dev, P[0], src + v.t0, v, bgs[0], ctx->opt,
                            ctx->status, s);
        }
        for (int sg = 0; sg < 4; ++sg)
        {
            const int j = w - 1 - sg;
            if (j < 0 || j >= z.n)
                continue;
            T *pin = P[sg % 2], *pout = P[(sg + 1) % 2];
            const BoxDev v = chunk_view(b, z.k0(j), z.k1(j));
            {
                Timed t_(ctx, GRHD_K_GHOSTS, s);
                launch_fill_ghost_planes<T>(sg == 0 ? dev : ctx->stage, pin,
                                            sg == 0 ? b : sb, bgs[sg],
                                            ctx->opt, ctx->status, z.plo(j),
                                            z.phi(j), s);
            }
            {
                Timed t_(ctx, GRHD_K_FACES, s);
                launch_faces<T>(pin, src + v.t0, k + v.t0, v, bgs[sg],
                                ctx->opt, inv_dx, zc, nullptr, s);
            }
            {
                Timed t_(ctx, GRHD_K_STAGE, s);
                if (sg < 3)
                    launch_stage<T>(0, dev, b.cs, nullptr, 0, ctx->stage, sb.cs,
                                    k + v.t0, acc + v.t0, pout, src + v.t0, 1,
                                    v, bgs[sg + 1], ctx->opt, sg, dt, false,
                                    inv_dx, ctx->status, s, pin);
                else
                    launch_stage<T>(0, dev, b.cs, nullptr, 0, dev, b.cs,
                                    k + v.t0, acc + v.t0, pout, nullptr, 0, v,
                                    bgs[3], ctx->opt, 3, dt, true, inv_dx,
                                    ctx->status, s, pin);
            }
            if (sg == 3)
            {
                GRHD_CUDA(ctx, cudaEventRecord(ev_out[j], s));
                GRHD_CUDA(ctx, cudaStreamWaitEvent(ctx->d2h, ev_out[j], 0));
                const size_t off = (size_t)(z.plo(j) - b.glo[2]) * plane;
                const size_t n = (size_t)(z.phi(j) - z.plo(j) + 1) * plane;
                for (int q = 0; q < kStateComps; ++q)
                {
                    GRHD_CUDA(ctx, cudaMemcpyAsync(host + q * cs + off,
                                                   dev + q * cs + off,
                                                   n * sizeof(double),
                                                   cudaMemcpyDeviceToHost,
                                                   ctx->d2h));
                    out += (long long)(n * sizeof(double));
                }
            }
        }
    }
    return GRHD_OK;
}

} // namespace

extern "C" {

int grhd_ccz4_compute_rhs(grhd_ctx *ctx, double *rhs, int64_t rhs_cs,
                          double *state, int64_t state_cs,
                          const grhd_box *box, const double inverse_dx[3],
                          void *stream)
{
    if (ctx && (!rhs || !inverse_dx))
    {
        std::memset(&ctx->last_error, 0, sizeof(ctx->last_error));
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "null rhs or inverse_dx");
    }
    cudaStream_t s = (cudaStream_t)stream;
    BoxDev b;
    int st = ccz4_checks(ctx, state, state_cs, box, rhs_cs, b, s);
    if (st)
        return st;
    enqueue_ccz4_rhs(ctx, rhs, rhs_cs, state, b, inverse_dx, s);
    return ccz4_finish(ctx, b, state, s);
}

int grhd_ccz4_recover_primitives(grhd_ctx *ctx, double *state,
                                 int64_t state_cs, const grhd_box *box,
                                 grhd_diagnostics *diag, void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    BoxDev b;
    int st = ccz4_checks(ctx, state, state_cs, box, -1, b, s);
    if (st)
        return st;
    launch_ccz4_recover(state, b, ctx->opt, ctx->status, s);
    ++ctx->launches;
    st = ccz4_finish(ctx, b, state, s);
    read_diag(ctx, diag);
    return st;
}

int grhd_ccz4_update_conserved(grhd_ctx *ctx, double *state,
                               int64_t state_cs, const double *rhs,
                               int64_t rhs_cs, const grhd_box *box, double dt,
                               int recover, grhd_diagnostics *diag,
                               void *stream)
{
    if (ctx && !rhs)
    {
        std::memset(&ctx->last_error, 0, sizeof(ctx->last_error));
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "null rhs");
    }
    cudaStream_t s = (cudaStream_t)stream;
    BoxDev b;
    int st = ccz4_checks(ctx, state, state_cs, box, rhs_cs, b, s);
    if (st)
        return st;
    launch_ccz4_update(state, nullptr, 0, rhs, rhs_cs, b, dt, 0, s);
    ++ctx->launches;
    if (recover)
    {
        launch_ccz4_recover(state, b, ctx->opt, ctx->status, s);
        ++ctx->launches;
    }
    st = ccz4_finish(ctx, b, state, s);
    read_diag(ctx, diag);
    return st;
}

int grhd_ccz4_compute_max_inverse_dt(grhd_ctx *ctx, const double *state,
                                     int64_t state_cs, const grhd_box *box,
                                     const double inverse_dx[3], double *out,
                                     void *stream)
{
    if (ctx && (!out || !inverse_dx))
    {
        std::memset(&ctx->last_error, 0, sizeof(ctx->last_error));
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "null output or inverse_dx");
    }
    cudaStream_t s = (cudaStream_t)stream;
    BoxDev b;
    int st = ccz4_checks(ctx, state, state_cs, box, -1, b, s);
    if (st)
        return st;
    launch_ccz4_max_inv_dt(state, b, ctx->opt, inverse_dx, ctx->status, s);
    ++ctx->launches;
    st = ccz4_finish(ctx, b, state, s);
    if (st == GRHD_OK)
        *out = bits_to_double(ctx->status_h->maxinv_bits);
    return st;
}

int grhd_ccz4_advance_ssprk2(grhd_ctx *ctx, double *state, int64_t state_cs,
                             const grhd_box *box, const double inverse_dx[3],
                             double dt, grhd_diagnostics *diag, void *stream)
{
    if (ctx && (!inverse_dx || !box_is_domain(box)))
    {
        std::memset(&ctx->last_error, 0, sizeof(ctx->last_error));
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "advance needs inverse_dx and the box to cover the "
                         "whole domain");
    }
    cudaStream_t s = (cudaStream_t)stream;
    BoxDev b;
    int st = ccz4_checks(ctx, state, state_cs, box, -1, b, s);
    if (st)
        return st;
    const int64_t gv = b.gvol();
    if ((st = grow(ctx, &ctx->ccz4_stage, &ctx->ccz4_stage_cap,
                   (size_t)GRHD_CCZ4_NUM_VARS * gv)))
        return st;
    BoxDev sb = b;
    sb.cs = gv;
    double *stage = ctx->ccz4_stage;
    double *k0 = ctx->kbuf, *k1 = ctx->src; // rhs_initial, rhs_stage
    // advance_ssprk2 (:1323-1348): stage = state; rhs_initial = L(state);
    // stage += dt rhs_initial, recovered; rhs_stage = L(stage);
    // state = (state + stage + dt rhs_stage) / 2, recovered
    GRHD_CUDA(ctx, cudaMemcpy2DAsync(stage, gv * sizeof(double), state,
                                     state_cs * sizeof(double),
                                     gv * sizeof(double), GRHD_CCZ4_NUM_VARS,
                                     cudaMemcpyDeviceToDevice, s));
    enqueue_ccz4_rhs(ctx, k0, b.ivol(), state, b, inverse_dx, s);
    launch_ccz4_update(stage, nullptr, 0, k0, b.ivol(), sb, dt, 0, s);
    launch_ccz4_recover(stage, sb, ctx->opt, ctx->status, s);
    enqueue_ccz4_rhs(ctx, k1, b.ivol(), stage, sb, inverse_dx, s);
    launch_ccz4_update(state, stage, gv, k1, b.ivol(), b, dt, 1, s);
    launch_ccz4_recover(state, b, ctx->opt, ctx->status, s);
    ctx->launches += 4;
    st = ccz4_finish(ctx, b, state, s);
    read_diag(ctx, diag);
    return st;
}

int grhd_ccz4_ssprk2_stage(grhd_ctx *ctx, int stage, double *state,
                           int64_t state_cs, double *stage_state,
                           int64_t stage_cs, const grhd_box *box,
                           const double inverse_dx[3], double dt,
                           grhd_diagnostics *diag, void *stream)
{
    if (ctx && (!inverse_dx || !stage_state || (stage != 1 && stage != 2)))
    {
        std::memset(&ctx->last_error, 0, sizeof(ctx->last_error));
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "ssprk2 stage is 1 or 2 and needs a stage state and "
                         "inverse_dx");
    }
    cudaStream_t s = (cudaStream_t)stream;
    BoxDev b;
    int st = ccz4_checks(ctx, state, state_cs, box, -1, b, s);
    if (st)
        return st;
    const BoxDev sb = make_box(box, stage_cs);
    if ((st = check_strides(ctx, sb, stage_cs, -1)))
        return st;
    const int64_t gv = b.gvol();
    if (stage == 1)
    {
        // stage = state (all components); rhs_initial = L(state); stage +=
        // dt rhs_initial, recovered
        GRHD_CUDA(ctx, cudaMemcpy2DAsync(stage_state, stage_cs * sizeof(double),
                                         state, state_cs * sizeof(double),
                                         gv * sizeof(double),
                                         GRHD_CCZ4_NUM_VARS,
                                         cudaMemcpyDeviceToDevice, s));
        enqueue_ccz4_rhs(ctx, ctx->kbuf, b.ivol(), state, b, inverse_dx, s);
        launch_ccz4_update(stage_state, nullptr, 0, ctx->kbuf, b.ivol(), sb,
                           dt, 0, s);
        launch_ccz4_recover(stage_state, sb, ctx->opt, ctx->status, s);
    }
    else
    {
        // rhs_stage = L(stage); state = (state + stage + dt rhs_stage) / 2,
        // recovered
        enqueue_ccz4_rhs(ctx, ctx->kbuf, b.ivol(), stage_state, sb,
                         inverse_dx, s);
        launch_ccz4_update(state, stage_state, stage_cs, ctx->kbuf, b.ivol(),
                           b, dt, 1, s);
        launch_ccz4_recover(state, b, ctx->opt, ctx->status, s);
    }
    ctx->launches += 2;
    st = stage == 1 ? ccz4_finish(ctx, sb, stage_state, s)
                    : ccz4_finish(ctx, b, state, s);
    read_diag(ctx, diag);
    return st;
}

int grhd_advance_ssprk2(grhd_ctx *ctx, double *state, int64_t state_cs,
                        const grhd_box *box, const double inverse_dx[3],
                        double time, double dt, grhd_diagnostics *diag,
                        void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    BoxDev b;
    int st = advance_checks(ctx, state, state_cs, box, inverse_dx, b, s);
    if (st)
        return st;
    if (ctx->params.precision == GRHD_PRECISION_MIXED)
        enqueue_ssprk2<float>(ctx, state, b, inverse_dx, time, dt, s);
    else
        enqueue_ssprk2<double>(ctx, state, b, inverse_dx, time, dt, s);
    st = finish_status(ctx, b, state, make_background(ctx->params, time), s);
    read_diag(ctx, diag);
    return st;
}

int grhd_ssprk2_stage(grhd_ctx *ctx, int stage, double *state,
                      int64_t state_cs, double *stage_state,
                      int64_t stage_cs, const grhd_box *box,
                      const double inverse_dx[3], double time, double dt,
                      grhd_diagnostics *diag, void *stream)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    if (!stage_state || !inverse_dx || (stage != 1 && stage != 2))
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "ssprk2 stage is 1 or 2 and needs a stage state and "
                         "inverse_dx");
    cudaStream_t s = (cudaStream_t)stream;
    const BoxDev b = make_box(box, state_cs);
    const BoxDev sb = make_box(box, stage_cs);
    if ((st = check_strides(ctx, b, state_cs, -1)) ||
        (st = check_strides(ctx, sb, stage_cs, -1)) ||
        (st = ensure_scratch(ctx, b, false)) || (st = reset_status(ctx, s)))
        return st;
    const Background bg0 = make_background(ctx->params, time);
    const Background bg1 = make_background(ctx->params, time + dt);
    if (ctx->params.precision == GRHD_PRECISION_MIXED)
        enqueue_ssprk2_stage<float>(ctx, stage, state, b, stage_state, sb,
                                    bg0, bg1, inverse_dx, dt, s);
    else
        enqueue_ssprk2_stage<double>(ctx, stage, state, b, stage_state, sb,
                                     bg0, bg1, inverse_dx, dt, s);
    st = stage == 1 ? finish_status(ctx, b, state, bg0, s)
                    : finish_status(ctx, sb, stage_state, bg1, s);
    read_diag(ctx, diag);
    return st;
}

int grhd_advance_rk4(grhd_ctx *ctx, double *state, int64_t state_cs,
                     const grhd_box *box, const double inverse_dx[3],
                     double time, double dt, grhd_diagnostics *diag,
                     void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    BoxDev b;
    int st = advance_checks(ctx, state, state_cs, box, inverse_dx, b, s);
    if (st)
        return st;
    enqueue_rk4_any(ctx, state, b, inverse_dx, time, dt, false, s);
    st = finish_status(ctx, b, state, make_background(ctx->params, time), s);
    read_diag(ctx, diag);
    return st;
}

int grhd_advance_rk4_cfl(grhd_ctx *ctx, double *state, int64_t state_cs,
                         const grhd_box *box, const double inverse_dx[3],
                         double time, double cfl, double max_dt,
                         double *max_inverse_dt, double *dt_used,
                         grhd_diagnostics *diag, void *stream)
{
    if (ctx && (!(cfl > 0.0) || !max_inverse_dt))
    {
        std::memset(&ctx->last_error, 0, sizeof(ctx->last_error));
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "GRHD CFL number must be positive");
    }
    cudaStream_t s = (cudaStream_t)stream;
    BoxDev b;
    int st = advance_checks(ctx, state, state_cs, box, inverse_dx, b, s);
    if (st)
        return st;
    const Background bg0 = make_background(ctx->params, time);
    double mi = *max_inverse_dt;
    if (!(mi > 0.0))
    {
        {
            Timed t_(ctx, GRHD_K_CFL, s);
            launch_max_inv_dt(state, b, bg0, ctx->opt, inverse_dx,
                              ctx->status,
                              ctx->params.precision == GRHD_PRECISION_MIXED,
                              s);
        }
        if ((st = finish_status(ctx, b, state, bg0, s)))
            return st;
        mi = bits_to_double(ctx->status_h->maxinv_bits);
        if ((st = reset_status(ctx, s)))
            return st;
    }
    double dt = cfl / std::fmax(mi, 1.0e-14);
    if (max_dt > 0.0)
        dt = std::fmin(dt, max_dt);
    enqueue_rk4_any(ctx, state, b, inverse_dx, time, dt, true, s);
    st = finish_status(ctx, b, state, bg0, s);
    read_diag(ctx, diag);
    if (st)
        return st;
    *max_inverse_dt = bits_to_double(ctx->status_h->maxinv_bits);
    if (dt_used)
        *dt_used = dt;
    return GRHD_OK;
}

// One grhd_advance_rk4_cfl step of a state held in host memory.  Host ->
// device goes what the step reads: the conserved components of every cell
// (the box is the whole domain, so every ghost is physical and refilled
// from the interior), the primitives of the z planes that hold excised
// cells (frozen stencil neighbours), and in mixed precision the pressure
// (con2prim's starting point).  Device -> host goes the whole state.
// With the CFL speed given (*max_inverse_dt > 0, as every call after the
// first passes it) and no accretion-rate integral, the copies overlap the
// step (enqueue_rk4_host_pipelined); otherwise the state is copied in,
// stepped and copied out in turn.
int grhd_advance_rk4_cfl_host(grhd_ctx *ctx, double *host_state,
                              int64_t state_cs, const grhd_box *box,
                              const double inverse_dx[3], double time,
                              double cfl, double max_dt,
                              double *max_inverse_dt, double *dt_used,
                              grhd_diagnostics *diag, long long *h2d_bytes,
                              long long *d2h_bytes, void *stream)
{
    if (!ctx)
        return GRHD_ERR_INVALID_ARG;
    std::memset(&ctx->last_error, 0, sizeof(ctx->last_error));
    if (!host_state || !box || !valid_box(box) || !box_is_domain(box))
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "host step needs a host state and a box covering "
                         "the whole domain");
    if (!(cfl > 0.0) || !max_inverse_dt)
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "GRHD CFL number must be positive");
    GRHD_CUDA(ctx, cudaSetDevice(ctx->device));
    const BoxDev b = make_box(box, state_cs);
    int st = check_strides(ctx, b, state_cs, -1);
    if (st)
        return st;
    if ((st = grow(ctx, &ctx->host_state, &ctx->host_state_cap,
                   kStateComps * (size_t)state_cs)))
        return st;
    cudaStream_t s = (cudaStream_t)stream;
    double *dev = ctx->host_state;
    const size_t cs = (size_t)state_cs;
    const bool mixed = ctx->params.precision == GRHD_PRECISION_MIXED;
    // ghosted z planes with a cell centre inside |z| < R, one plane of
    // margin each side (empty: ek0 > ek1)
    int ek0 = 1, ek1 = 0;
    const double R = ctx->params.excision_radius;
    if (R > 0.0)
    {
        const double dx = ctx->params.dx, cz = ctx->params.center[2];
        const int k0 = (int)std::floor((cz - R) / dx - 0.5) - 1;
        const int k1 = (int)std::ceil((cz + R) / dx - 0.5) + 1;
        ek0 = std::max(k0, b.glo[2]);
        ek1 = std::min(k1, b.ghi[2]);
    }
    long long in = 0, out = 0;
    if (*max_inverse_dt > 0.0 && !(ctx->params.accretion_radius > 0.0))
    {
        BoxDev bb;
        if ((st = advance_checks(ctx, dev, state_cs, box, inverse_dx, bb, s)) ||
            (st = grow(ctx, &ctx->prim2, &ctx->prim2_cap,
                       5 * (size_t)bb.gvol())))
            return st;
        double dt = cfl / std::fmax(*max_inverse_dt, 1.0e-14);
        if (max_dt > 0.0)
            dt = std::fmin(dt, max_dt);
        st = mixed ? enqueue_rk4_host_pipelined<float>(
                         ctx, host_state, dev, bb, inverse_dx, time, dt, ek0,
                         ek1, s, in, out)
                   : enqueue_rk4_host_pipelined<double>(
                         ctx, host_state, dev, bb, inverse_dx, time, dt, ek0,
                         ek1, s, in, out);
        // no copy into the caller's memory may outlive the call
        const cudaError_t e_out = cudaStreamSynchronize(ctx->d2h);
        const cudaError_t e_in = cudaStreamSynchronize(ctx->h2d);
        if (st)
            return st;
        GRHD_CUDA(ctx, e_out);
        GRHD_CUDA(ctx, e_in);
        st = finish_status(ctx, bb, dev, make_background(ctx->params, time),
                           s);
        read_diag(ctx, diag);
        if (st)
            return st;
        *max_inverse_dt = bits_to_double(ctx->status_h->maxinv_bits);
        if (dt_used)
            *dt_used = dt;
        if (h2d_bytes)
            *h2d_bytes = in;
        if (d2h_bytes)
            *d2h_bytes = out;
        return GRHD_OK;
    }
    GRHD_CUDA(ctx, cudaMemcpyAsync(dev, host_state, 5 * cs * sizeof(double),
                                   cudaMemcpyHostToDevice, s));
    in += 5 * cs * sizeof(double);
    if (mixed)
    {
        GRHD_CUDA(ctx, cudaMemcpyAsync(dev + kPress * cs,
                                       host_state + kPress * cs,
                                       cs * sizeof(double),
                                       cudaMemcpyHostToDevice, s));
        in += cs * sizeof(double);
    }
    if (ek0 <= ek1)
    {
        const size_t plane = (size_t)b.gn[0] * b.gn[1];
        const size_t off = (size_t)(ek0 - b.glo[2]) * plane;
        const size_t n = (size_t)(ek1 - ek0 + 1) * plane;
        for (int c = 5; c < kStateComps; ++c)
        {
            if (mixed && c == kPress)
                continue;
            GRHD_CUDA(ctx, cudaMemcpyAsync(dev + c * cs + off,
                                           host_state + c * cs + off,
                                           n * sizeof(double),
                                           cudaMemcpyHostToDevice, s));
            in += n * sizeof(double);
        }
    }
    st = grhd_advance_rk4_cfl(ctx, dev, state_cs, box, inverse_dx, time, cfl,
                              max_dt, max_inverse_dt, dt_used, diag, stream);
    if (st)
        return st;
    GRHD_CUDA(ctx, cudaMemcpyAsync(host_state, dev,
                                   kStateComps * cs * sizeof(double),
                                   cudaMemcpyDeviceToHost, s));
    GRHD_CUDA(ctx, cudaStreamSynchronize(s));
    if (h2d_bytes)
        *h2d_bytes = in;
    if (d2h_bytes)
        *d2h_bytes = (long long)(kStateComps * cs * sizeof(double));
    return GRHD_OK;
}

int grhd_advance_rk4_cfl_steps(grhd_ctx *ctx, double *state,
                               int64_t state_cs, const grhd_box *box,
                               const double inverse_dx[3], double time,
                               double cfl, double max_dt, int steps,
                               double *max_inverse_dt, double *time_out,
                               grhd_diagnostics *diag, void *stream)
{
    if (ctx && (!(cfl > 0.0) || !max_inverse_dt || steps < 0))
    {
        std::memset(&ctx->last_error, 0, sizeof(ctx->last_error));
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "GRHD CFL number must be positive");
    }
    cudaStream_t s = (cudaStream_t)stream;
    BoxDev b;
    int st = advance_checks(ctx, state, state_cs, box, inverse_dx, b, s);
    if (st)
        return st;
    grhd_diagnostics total{};
    double mi = *max_inverse_dt;
    if (!(mi > 0.0) && steps > 0)
    {
        const Background bg0 = make_background(ctx->params, time);
        {
            Timed t_(ctx, GRHD_K_CFL, s);
            launch_max_inv_dt(state, b, bg0, ctx->opt, inverse_dx,
                              ctx->status,
                              ctx->params.precision == GRHD_PRECISION_MIXED,
                              s);
        }
        if ((st = finish_status(ctx, b, state, bg0, s)))
            return st;
        mi = bits_to_double(ctx->status_h->maxinv_bits);
        if ((st = reset_status(ctx, s)))
            return st;
    }
    for (int n = 0; n < steps; ++n)
    {
        double dt = cfl / std::fmax(mi, 1.0e-14);
        if (max_dt > 0.0)
            dt = std::fmin(dt, max_dt);
        enqueue_rk4_any(ctx, state, b, inverse_dx, time, dt, true, s, n > 0,
                        n + 1 < steps);
        st = finish_status(ctx, b, state, make_background(ctx->params, time),
                           s);
        grhd_diagnostics d{};
        read_diag(ctx, &d);
        total.num_cells += d.num_cells;
        total.num_failed_recoveries += d.num_failed_recoveries;
        total.num_floored_primitives += d.num_floored_primitives;
        total.num_conserved_resets += d.num_conserved_resets;
        if (st)
            break;
        mi = bits_to_double(ctx->status_h->maxinv_bits);
        time += dt;
        if (n + 1 < steps && (st = reset_status(ctx, s)))
            break;
    }
    if (diag)
        *diag = total;
    if (st)
        return st;
    *max_inverse_dt = mi;
    if (time_out)
        *time_out = time;
    return GRHD_OK;
}

int grhd_eval_background(grhd_ctx *ctx, int64_t n, const double *xyz,
                         double time, double *out, void *stream)
{
    if (!ctx || n < 0 || (n > 0 && (!xyz || !out)))
        return GRHD_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const Background bg = make_background(ctx->params, time);
    launch_eval_background(n, xyz, bg, out, s);
    GRHD_CUDA(ctx, cudaGetLastError());
    GRHD_CUDA(ctx, cudaStreamSynchronize(s));
    return GRHD_OK;
}

int grhd_eval_con2prim(grhd_ctx *ctx, int64_t n, const double *cons,
                       const double *gUU, double *prim, int *ok,
                       int *iterations, double *residual, void *stream)
{
    if (!ctx || n < 0 ||
        (n > 0 && (!cons || !gUU || !prim || !ok || !iterations || !residual)))
        return GRHD_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    launch_eval_con2prim(n, cons, gUU, ctx->opt, prim, ok, iterations,
                         residual, s);
    GRHD_CUDA(ctx, cudaGetLastError());
    GRHD_CUDA(ctx, cudaStreamSynchronize(s));
    return GRHD_OK;
}

int grhd_face_zchunk(int nx, int ny, int nz, int resident_blocks,
                     int *zchunk)
{
    if (nx < 1 || ny < 1 || nz < 1 || resident_blocks < 1 || !zchunk)
        return GRHD_ERR_INVALID_ARG;
    *zchunk = face_zchunk_model(nx, ny, nz, resident_blocks);
    return GRHD_OK;
}

int grhd_eval_arith(grhd_ctx *ctx, int64_t n, const double *a,
                    const double *b, double *out, void *stream)
{
    if (!ctx || n < 0 || (n > 0 && (!a || !b || !out)))
        return GRHD_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    launch_eval_arith(n, a, b, out, s);
    GRHD_CUDA(ctx, cudaGetLastError());
    GRHD_CUDA(ctx, cudaStreamSynchronize(s));
    return GRHD_OK;
}

void grhd_default_torus_config(grhd_torus_config *c)
{
    // FixedBGTorusConfig defaults, FixedBGTorus.hpp:20-34
    c->total_mass = 1.0;
    c->inner_radius = 0.0;
    c->pressure_max_radius = 0.0;
    c->rho_peak = 1.0;
    c->max_velocity_squared = 1.0 - 1.0e-12;
    c->radial_derivative_fraction = 1.0e-3;
    c->radial_derivative_min_step = 1.0e-4;
    c->angular_momentum_min_factor = 0.25;
    c->angular_momentum_max_factor = 4.0;
    c->angular_momentum_samples = 120;
    c->angular_momentum_bisection_iterations = 80;
    c->angular_momentum_tolerance = 1.0e-13;
}

int grhd_torus_initial_data(grhd_ctx *ctx, double *state, int64_t state_cs,
                            const grhd_box *box,
                            const grhd_torus_config *config, double time,
                            grhd_torus_params *out, void *stream)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    if (!config)
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "null torus config");
    cudaStream_t s = (cudaStream_t)stream;
    const BoxDev b = make_box(box, state_cs);
    if ((st = check_strides(ctx, b, state_cs, -1)))
        return st;
    TorusConfigDev c;
    static_assert(sizeof(TorusConfigDev) == sizeof(grhd_torus_config),
                  "torus config layout");
    std::memcpy(&c, config, sizeof(c));
    const Background bg = make_background(ctx->params, time);
    double res[4] = {0, 0, 0, 0};
    ctx->launches += 3;
    const cudaError_t e = torus_initial_data(state, b, bg, ctx->opt, c,
                                             ctx->probe, res, s);
    if (out)
    {
        out->ell = res[0];
        out->surface_potential = res[1];
        out->polytropic_constant = res[2];
        out->max_enthalpy = res[3];
    }
    if (e == cudaErrorInvalidValue)
        return set_error(ctx, GRHD_ERR_SETUP, 0, nullptr, 0.0,
                         "torus has no pressure-supported region or an "
                         "invalid surface potential");
    GRHD_CUDA(ctx, e);
    GRHD_CUDA(ctx, cudaStreamSynchronize(s));
    return GRHD_OK;
}

int grhd_michel_initial_data(grhd_ctx *ctx, double *state, int64_t state_cs,
                             const grhd_box *box,
                             const grhd_michel_config *config, void *stream)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    if (!config)
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "null Michel config");
    cudaStream_t s = (cudaStream_t)stream;
    const BoxDev b = make_box(box, state_cs);
    if ((st = check_strides(ctx, b, state_cs, -1)))
        return st;
    MichelConfigDev c;
    c.mass = config->mass;
    c.gamma = ctx->params.adiabatic_index;
    c.sonic_radius = config->sonic_radius;
    c.sonic_density = config->sonic_density;
    c.atmosphere_radius = config->atmosphere_radius;
    c.root_tolerance = config->root_tolerance;
    ++ctx->launches;
    GRHD_CUDA(ctx, michel_initial_data(state, b, ctx->opt, c, ctx->flag, s));
    int bad = 0;
    GRHD_CUDA(ctx, cudaMemcpyAsync(&bad, ctx->flag, sizeof(int),
                                   cudaMemcpyDeviceToHost, s));
    GRHD_CUDA(ctx, cudaStreamSynchronize(s));
    if (bad)
        return set_error(ctx, GRHD_ERR_SETUP, 0, nullptr, 0.0,
                         "Michel profile has no root or an invalid Lorentz "
                         "factor outside the atmosphere radius");
    return GRHD_OK;
}

int grhd_perturb_density(grhd_ctx *ctx, double *state, int64_t state_cs,
                         const grhd_box *box, double amplitude, uint64_t seed,
                         double time, void *stream)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    cudaStream_t s = (cudaStream_t)stream;
    const BoxDev b = make_box(box, state_cs);
    if ((st = check_strides(ctx, b, state_cs, -1)))
        return st;
    const Background bg = make_background(ctx->params, time);
    ++ctx->launches;
    GRHD_CUDA(ctx, perturb_density(state, b, bg, ctx->opt, amplitude, seed, s));
    GRHD_CUDA(ctx, cudaStreamSynchronize(s));
    return GRHD_OK;
}

int grhd_profile_enable(grhd_ctx *ctx, int enable)
{
    if (!ctx)
        return GRHD_ERR_INVALID_ARG;
    ctx->prof_on = enable != 0;
    return GRHD_OK;
}

int grhd_profile_read(grhd_ctx *ctx, double ms[GRHD_K_NUM_CLASSES],
                      long long launches[GRHD_K_NUM_CLASSES])
{
    if (!ctx || !ms || !launches)
        return GRHD_ERR_INVALID_ARG;
    for (int q = 0; q < GRHD_K_NUM_CLASSES; ++q)
    {
        ms[q] = 0.0;
        launches[q] = 0;
    }
    for (auto &r : ctx->prof_pending)
    {
        GRHD_CUDA(ctx, cudaEventSynchronize(r.b));
        float t = 0.0f;
        GRHD_CUDA(ctx, cudaEventElapsedTime(&t, r.a, r.b));
        if (r.cls >= 0 && r.cls < GRHD_K_NUM_CLASSES)
        {
            ms[r.cls] += t;
            launches[r.cls] += 1;
        }
        ctx->event_pool.push_back(r.a);
        ctx->event_pool.push_back(r.b);
    }
    ctx->prof_pending.clear();
    return GRHD_OK;
}

int grhd_accretion(grhd_ctx *ctx, double *mdot_last, double *integral,
                   int reset)
{
    if (!ctx)
        return GRHD_ERR_INVALID_ARG;
    double h[2];
    GRHD_CUDA(ctx, cudaSetDevice(ctx->device));
    GRHD_CUDA(ctx, cudaMemcpy(h, ctx->mdot_acc, 2 * sizeof(double),
                              cudaMemcpyDeviceToHost));
    if (mdot_last)
        *mdot_last = h[0];
    if (integral)
        *integral = h[1];
    if (reset)
        GRHD_CUDA(ctx, cudaMemset(ctx->mdot_acc + 1, 0, sizeof(double)));
    return GRHD_OK;
}

long long grhd_launch_count(const grhd_ctx *ctx)
{
    return ctx ? ctx->launches : 0;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Source terms of the binary-PN disk driver (grhd_kitp.cuh).
namespace {

int kitp_setup(grhd_ctx *ctx, const void *state, const grhd_box *box,
               int64_t state_cs, const grhd_kitp_config *cfg, double time,
               BoxDev &b, KitpDev &k)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    if (!cfg)
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, nullptr,
                         0.0, "null source-term configuration");
    if (ctx->params.background != GRHD_BG_BINARY_PN)
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, nullptr,
                         0.0, "the disk driver's source terms need the "
                              "binary post-Newtonian background");
    b = make_box(box, state_cs);
    if (state_cs < b.gvol())
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, nullptr,
                         0.0, "state stride smaller than the ghosted box");
    k.alpha = cfg->alpha_viscosity;
    k.beta = cfg->viscosity_beta;
    k.rho_floor_cfg = cfg->rho_floor;
    k.sink_size = cfg->sink_size;
    k.sink_rate = cfg->sink_rate;
    k.sink_shape = cfg->sink_shape;
    k.mass[0] = ctx->params.pn_mass_1;
    k.mass[1] = ctx->params.pn_mass_2;
    double v1[3], v2[3];
    pn_state(ctx->params, time, k.body[0], k.body[1], v1, v2);
    k.atmo_rho_floor = ctx->params.rho_floor;
    return GRHD_OK;
}

} // namespace

extern "C" {

void grhd_default_kitp_config(grhd_kitp_config *c)
{
    if (!c)
        return;
    // SimulationConfig defaults, Main_GRHDLevelDataBinaryPNKITPDisk.cpp:63-71
    c->alpha_viscosity = 0.03;
    c->viscosity_beta = 0.0;
    c->rho_floor = 1.0e-10;
    c->sink_size = 1.0;
    c->sink_rate = 1.0e4;
    c->sink_shape = 4.0;
}

int grhd_kitp_viscous_rhs(grhd_ctx *ctx, double *rhs, int64_t rhs_cs,
                          const double *state, int64_t state_cs,
                          const grhd_box *box, const grhd_kitp_config *cfg,
                          double time, void *stream)
{
    BoxDev b;
    KitpDev k;
    int st = kitp_setup(ctx, state, box, state_cs, cfg, time, b, k);
    if (st)
        return st;
    if (!rhs || rhs_cs < b.ivol())
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, nullptr,
                         0.0, "null rhs or rhs stride too small");
    if (cfg->alpha_viscosity == 0.0)
        return GRHD_OK;
    cudaStream_t s = (cudaStream_t)stream;
    ++ctx->launches;
    launch_kitp_viscous_rhs(rhs, rhs_cs, state, b, ctx->opt, k, s);
    GRHD_CUDA(ctx, cudaGetLastError());
    return GRHD_OK;
}

int grhd_kitp_sink_rhs(grhd_ctx *ctx, double *rhs, int64_t rhs_cs,
                       const double *state, int64_t state_cs,
                       const grhd_box *box, const grhd_kitp_config *cfg,
                       double time, void *stream)
{
    BoxDev b;
    KitpDev k;
    int st = kitp_setup(ctx, state, box, state_cs, cfg, time, b, k);
    if (st)
        return st;
    if (!rhs || rhs_cs < b.ivol())
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, nullptr,
                         0.0, "null rhs or rhs stride too small");
    if (cfg->sink_rate == 0.0 || cfg->sink_size <= 0.0)
        return GRHD_OK;
    cudaStream_t s = (cudaStream_t)stream;
    ++ctx->launches;
    launch_kitp_sink_rhs(rhs, rhs_cs, state, b, ctx->opt, k, s);
    GRHD_CUDA(ctx, cudaGetLastError());
    return GRHD_OK;
}

int grhd_kitp_sink_decay(grhd_ctx *ctx, double *state, int64_t state_cs,
                         const grhd_box *box, const grhd_kitp_config *cfg,
                         double time, double dt, void *stream)
{
    BoxDev b;
    KitpDev k;
    int st = kitp_setup(ctx, state, box, state_cs, cfg, time, b, k);
    if (st)
        return st;
    if (cfg->sink_rate == 0.0 || cfg->sink_size <= 0.0)
        return GRHD_OK;
    cudaStream_t s = (cudaStream_t)stream;
    ++ctx->launches;
    launch_kitp_sink_decay(state, b, ctx->opt, k, dt, s);
    GRHD_CUDA(ctx, cudaGetLastError());
    return GRHD_OK;
}

int grhd_kitp_advance_ssprk2(grhd_ctx *ctx, double *state, int64_t state_cs,
                             const grhd_box *box, const double inverse_dx[3],
                             const grhd_kitp_config *cfg, double time,
                             double dt, grhd_diagnostics *diag, void *stream)
{
    if (ctx && ctx->params.precision != GRHD_PRECISION_FP64)
    {
        std::memset(&ctx->last_error, 0, sizeof(ctx->last_error));
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "the disk driver's step runs in FP64");
    }
    cudaStream_t s = (cudaStream_t)stream;
    BoxDev b, bk;
    KitpDev k0, k1, kh;
    int st;
    if ((st = kitp_setup(ctx, state, box, state_cs, cfg, time, bk, k0)) ||
        (st = kitp_setup(ctx, state, box, state_cs, cfg, time + dt, bk, k1)) ||
        (st = kitp_setup(ctx, state, box, state_cs, cfg, time + 0.5 * dt, bk,
                         kh)) ||
        (st = advance_checks(ctx, state, state_cs, box, inverse_dx, b, s)))
        return st;
    BoxDev sb = b;
    sb.cs = b.gvol();
    const Background bg0 = make_background(ctx->params, time);
    const Background bg1 = make_background(ctx->params, time + dt);
    double *k = ctx->kbuf;
    const bool visc = cfg->alpha_viscosity != 0.0;
    // advance_kitp_ssprk2 (Main_GRHDLevelDataBinaryPNKITPDisk.cpp:842-876):
    // rhs = L(state) + viscous(state); stage = state + dt rhs, recovered at
    // t + dt (its primitives kept: the viscous stress reads them);
    // rhs = L(stage) + viscous(stage); state = (state + stage + dt rhs) / 2;
    // sink decay at t + dt/2; recovery at t + dt
    enqueue_rhs<double>(ctx, k, state, b, bg0, inverse_dx, s, false, 0.5 * dt);
    if (visc)
        launch_kitp_viscous_rhs(k, b.ivol(), state, b, ctx->opt, k0, s);
    launch_stage<double>(1, state, b.cs, nullptr, 0, ctx->stage, sb.cs, k,
                         nullptr, ctx->prim, ctx->src, 3, b, bg1, ctx->opt, 0,
                         dt, false, inverse_dx, ctx->status, s);
    enqueue_rhs<double>(ctx, k, ctx->stage, sb, bg1, inverse_dx, s, true,
                        0.5 * dt);
    if (visc)
        launch_kitp_viscous_rhs(k, b.ivol(), ctx->stage, sb, ctx->opt, k1, s);
    launch_kitp_combine(state, b, ctx->stage, sb.cs, k, b.ivol(), dt, s);
    if (cfg->sink_rate != 0.0 && cfg->sink_size > 0.0)
        launch_kitp_sink_decay(state, b, ctx->opt, kh, dt, s);
    launch_recover(state, b, bg1, ctx->opt, ctx->status, s);
    ctx->launches += 4 + (visc ? 2 : 0);
    st = finish_status(ctx, b, state, bg0, s);
    read_diag(ctx, diag);
    return st;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Diagnostics and checkpoints of the example drivers (grhd_io.cuh).
namespace {

int io_error(char *err, int cap, const char *msg, int status)
{
    if (err && cap > 0)
        std::snprintf(err, (size_t)cap, "%s", msg);
    return status;
}

template <typename V> void put(std::FILE *f, const V &v, bool &ok)
{
    ok = ok && std::fwrite(&v, sizeof(V), 1, f) == 1;
}

template <typename V> bool get(std::FILE *f, V &v)
{
    return std::fread(&v, sizeof(V), 1, f) == 1;
}

// The header fields of read_checkpoint_header
// (Main_GRHDLevelDataBinaryPNKITPDisk.cpp:1289-1345) up to the state.
int read_header(std::FILE *f, grhd_checkpoint_header &h, std::string &sig,
                uint64_t &count, char *err, int cap)
{
    char magic[8];
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "KITPCHK1", 8))
        return io_error(err, cap, "not a KITP checkpoint",
                        GRHD_ERR_INVALID_ARG);
    uint32_t version;
    int32_t nc, ncell, nz, ng, steps, frame;
    if (!get(f, version) || !get(f, nc) || !get(f, ncell) || !get(f, nz) ||
        !get(f, ng))
        return io_error(err, cap, "checkpoint ended unexpectedly",
                        GRHD_ERR_INVALID_ARG);
    if (version != 1 || nc < kStateComps)
        return io_error(err, cap, "unsupported KITP checkpoint format",
                        GRHD_ERR_INVALID_ARG);
    h.num_components = nc;
    h.num_cells = ncell;
    h.num_z_cells = nz;
    h.num_ghosts = ng;
    bool ok = get(f, steps) && get(f, frame) && get(f, h.time) &&
              get(f, h.next_output_time) && get(f, h.next_checkpoint_time);
    h.steps = steps;
    h.frame_index = frame;
    for (int q = 0; q < 4 && ok; ++q)
    {
        uint64_t v;
        ok = get(f, v);
        h.recovery_totals[q] = (long long)v;
    }
    for (int q = 0; q < 7 && ok; ++q)
        ok = get(f, h.diagnostics[q]);
    for (int q = 0; q < 3 && ok; ++q)
    {
        uint64_t v;
        ok = get(f, v);
        h.diagnostic_counts[q] = (long long)v;
    }
    uint64_t ssize = 0;
    ok = ok && get(f, ssize);
    if (!ok)
        return io_error(err, cap, "checkpoint ended unexpectedly",
                        GRHD_ERR_INVALID_ARG);
    if (ssize > 16384)
        return io_error(err, cap,
                        "invalid checkpoint configuration signature",
                        GRHD_ERR_INVALID_ARG);
    sig.assign((size_t)ssize, '\0');
    if ((ssize && std::fread(&sig[0], 1, (size_t)ssize, f) != ssize) ||
        !get(f, count))
        return io_error(err, cap, "checkpoint ended unexpectedly",
                        GRHD_ERR_INVALID_ARG);
    return GRHD_OK;
}

// The box must be the checkpoint's storage box: the domain (num_cells^2 x
// num_z_cells) grown by num_ghosts (checkpoint_storage_box, :1358-1363).
bool storage_matches(const grhd_box *box, int ncell, int nz, int ng)
{
    if (!valid_box(box) || !box_is_domain(box) || box->ghost != ng)
        return false;
    const int n[3] = {ncell, ncell, nz};
    for (int d = 0; d < 3; ++d)
        if (box->hi[d] - box->lo[d] + 1 != n[d])
            return false;
    return true;
}

} // namespace

extern "C" {

int grhd_disk_diagnostics(grhd_ctx *ctx, const double *state,
                          int64_t state_cs, const grhd_box *box, double time,
                          double out[7], void *stream)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    if (!out)
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, nullptr,
                         0.0, "null output");
    const BoxDev b = make_box(box, state_cs);
    if (state_cs < b.gvol())
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, nullptr,
                         0.0, "state stride smaller than the ghosted box");
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = diagnostics_blocks(b);
    // the partial results live in the context (grown once), so that a call
    // allocates nothing after the first on a box of its size
    if ((st = grow(ctx, &ctx->diag_part, &ctx->diag_cap, (size_t)7 * nb)))
        return st;
    double *part = ctx->diag_part;
    ++ctx->launches;
    launch_diagnostics(state, b, make_background(ctx->params, time),
                       ctx->opt, part, s);
    std::vector<double> h((size_t)7 * nb);
    cudaError_t e = cudaMemcpyAsync(h.data(), part, sizeof(double) * 7 * nb,
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return cuda_error(ctx, e, "grhd_disk_diagnostics");
    double r[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0};
    for (int q = 0; q < nb; ++q)
    {
        for (int c = 0; c < 3; ++c)
            r[c] += h[(size_t)q * 7 + c];
        for (int c = 3; c < 7; ++c)
            r[c] = std::fmax(r[c], h[(size_t)q * 7 + c]);
    }
    for (int c = 0; c < 7; ++c)
        out[c] = r[c];
    return GRHD_OK;
}

int grhd_level_exchange(const grhd_box *boxes, double *const *states,
                        const int64_t *strides, int count, char *err,
                        int err_cap, void *stream)
{
    return grhd_level_exchange_components(boxes, states, strides, count,
                                          kStateComps, err, err_cap, stream);
}

int grhd_level_exchange_components(const grhd_box *boxes,
                                   double *const *states,
                                   const int64_t *strides, int count,
                                   int ncomp, char *err, int err_cap,
                                   void *stream)
{
    if (count < 0 || (count > 0 && (!boxes || !states || !strides)))
        return io_error(err, err_cap, "null level arrays",
                        GRHD_ERR_INVALID_ARG);
    if (ncomp < 1 || ncomp > 256)
        return io_error(err, err_cap, "component count out of range",
                        GRHD_ERR_INVALID_ARG);
    std::vector<BoxDev> b((size_t)count);
    for (int q = 0; q < count; ++q)
    {
        if (!valid_box(&boxes[q]) || !states[q])
            return io_error(err, err_cap, "invalid box or state",
                            GRHD_ERR_INVALID_ARG);
        b[q] = make_box(&boxes[q], strides[q]);
        if (strides[q] < b[q].gvol())
            return io_error(err, err_cap, "state stride too small",
                            GRHD_ERR_INVALID_ARG);
        for (int d = 0; d < 3; ++d)
            if (boxes[q].domain_lo[d] != boxes[0].domain_lo[d] ||
                boxes[q].domain_hi[d] != boxes[0].domain_hi[d])
                return io_error(err, err_cap,
                                "the boxes of a level share one domain",
                                GRHD_ERR_INVALID_ARG);
    }
    // a DisjointBoxLayout: interiors do not overlap
    for (int p = 0; p < count; ++p)
        for (int q = p + 1; q < count; ++q)
        {
            bool overlap = true;
            for (int d = 0; d < 3; ++d)
                overlap = overlap && b[p].lo[d] <= b[q].hi[d] &&
                          b[q].lo[d] <= b[p].hi[d];
            if (overlap)
                return io_error(err, err_cap, "box interiors overlap",
                                GRHD_ERR_INVALID_ARG);
        }
    cudaStream_t s = (cudaStream_t)stream;
    for (int a = 0; a < count; ++a)
        for (int q = 0; q < count; ++q)
        {
            if (q == a)
                continue;
            // ghosted box of a, inside the domain, intersected with the
            // interior of q (disjoint from a's interior)
            int lo[3], hi[3];
            bool any = true;
            for (int d = 0; d < 3; ++d)
            {
                lo[d] = std::max(std::max(b[a].glo[d], b[a].dlo[d]),
                                 b[q].lo[d]);
                hi[d] = std::min(std::min(b[a].ghi[d], b[a].dhi[d]),
                                 b[q].hi[d]);
                any = any && lo[d] <= hi[d];
            }
            if (any)
                launch_copy_region(states[a], b[a], states[q], b[q], lo, hi,
                                   ncomp, s);
        }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return io_error(err, err_cap, cudaGetErrorString(e), GRHD_ERR_CUDA);
    return GRHD_OK;
}

int grhd_region_copy(int pack, double *state, int64_t state_cs,
                     const grhd_box *box, const int lo[3], const int hi[3],
                     double *buffer, void *stream)
{
    return grhd_region_copy_components(pack, state, state_cs, box, lo, hi,
                                       kStateComps, buffer, stream);
}

int grhd_region_copy_components(int pack, double *state, int64_t state_cs,
                                const grhd_box *box, const int lo[3],
                                const int hi[3], int ncomp, double *buffer,
                                void *stream)
{
    if (!state || !buffer || !lo || !hi || !valid_box(box) || ncomp < 1 ||
        ncomp > 256)
        return GRHD_ERR_INVALID_ARG;
    const BoxDev b = make_box(box, state_cs);
    if (state_cs < b.gvol())
        return GRHD_ERR_INVALID_ARG;
    for (int d = 0; d < 3; ++d)
        if (lo[d] > hi[d] || lo[d] < b.glo[d] || hi[d] > b.ghi[d])
            return GRHD_ERR_INVALID_ARG;
    launch_region(pack != 0, state, b, buffer, lo, hi, ncomp,
                  (cudaStream_t)stream);
    return cudaGetLastError() == cudaSuccess ? GRHD_OK : GRHD_ERR_CUDA;
}

void grhd_default_kitp_disk_config(grhd_kitp_disk_config *c)
{
    if (!c)
        return;
    // SimulationConfig, Main_GRHDLevelDataBinaryPNKITPDisk.cpp:56-61
    c->mach = 10.0;
    c->aspect_ratio = 0.1;
    c->cavity_radius_factor = 2.5;
    c->cavity_delta = 1.0e-5;
    c->outer_cutoff_radius = 1.0e10;
    c->rho_peak = 4.0e-5;
    for (int m = 0; m < 4; ++m)
        c->mode_amplitude[m] = c->mode_phase[m] = 0.0;
}

int grhd_kitp_disk_initial_data(grhd_ctx *ctx, double *state,
                                int64_t state_cs, const grhd_box *box,
                                const grhd_kitp_disk_config *cfg, double time,
                                void *stream)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    if (!cfg || !(cfg->mach > 0.0) || !(cfg->rho_peak > 0.0))
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, nullptr,
                         0.0, "disk configuration needs mach > 0 and "
                              "rho_peak > 0");
    if (ctx->params.background != GRHD_BG_BINARY_PN)
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, nullptr,
                         0.0, "the disk needs the binary post-Newtonian "
                              "background");
    const BoxDev b = make_box(box, state_cs);
    if ((st = check_strides(ctx, b, state_cs, -1)))
        return st;
    const grhd_params &p = ctx->params;
    KitpDiskDev k;
    k.mach = cfg->mach;
    k.aspect = cfg->aspect_ratio;
    k.cavity_factor = cfg->cavity_radius_factor;
    k.cavity_delta = cfg->cavity_delta;
    k.outer_cutoff = cfg->outer_cutoff_radius;
    k.rho_peak = cfg->rho_peak;
    for (int m = 0; m < 4; ++m)
    {
        k.amp[m] = cfg->mode_amplitude[m];
        k.phase[m] = cfg->mode_phase[m];
    }
    k.sep = p.pn_separation;
    k.mass[0] = p.pn_mass_1;
    k.mass[1] = p.pn_mass_2;
    k.soft = p.pn_softening_radius;
    const double total = p.pn_mass_1 + p.pn_mass_2;
    k.omega_bin = p.pn_angular_velocity != 0.0
                      ? p.pn_angular_velocity
                      : std::sqrt(total / (p.pn_separation * p.pn_separation *
                                           p.pn_separation));
    double v1[3], v2[3];
    pn_state(p, time, k.body[0], k.body[1], v1, v2);
    cudaStream_t s = (cudaStream_t)stream;
    ++ctx->launches;
    launch_kitp_disk_fill(state, b, make_background(p, time), ctx->opt, k, s);
    GRHD_CUDA(ctx, cudaGetLastError());
    GRHD_CUDA(ctx, cudaStreamSynchronize(s));
    return GRHD_OK;
}

int grhd_checkpoint_write(const char *path, const grhd_checkpoint_header *h,
                          const char *signature, const double *state,
                          int64_t state_cs, const grhd_box *box, char *err,
                          int err_cap, void *stream)
{
    if (!path || !h || !signature || !state)
        return io_error(err, err_cap, "null argument", GRHD_ERR_INVALID_ARG);
    if (h->num_components < kStateComps)
        return io_error(err, err_cap, "fewer components than the GRHD state",
                        GRHD_ERR_INVALID_ARG);
    if (!storage_matches(box, h->num_cells, h->num_z_cells, h->num_ghosts))
        return io_error(err, err_cap,
                        "box is not the checkpoint's domain and ghosts",
                        GRHD_ERR_INVALID_ARG);
    const BoxDev b = make_box(box, state_cs);
    if (state_cs < b.gvol())
        return io_error(err, err_cap, "state stride too small",
                        GRHD_ERR_INVALID_ARG);
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t count = (uint64_t)h->num_components * (uint64_t)b.gvol();
    std::vector<double> host((size_t)count);
    double *dev = nullptr;
    cudaError_t e = cudaMalloc((void **)&dev, count * sizeof(double));
    if (e == cudaSuccess)
    {
        launch_state_to_checkpoint(state, b, h->num_components, dev, s);
        e = cudaMemcpyAsync(host.data(), dev, count * sizeof(double),
                            cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s);
        cudaFree(dev);
    }
    if (e != cudaSuccess)
        return io_error(err, err_cap, cudaGetErrorString(e), GRHD_ERR_CUDA);
    // write_checkpoint, :1385-1505: a temporary file renamed into place
    const std::string tmp = std::string(path) + ".tmp";
    std::FILE *f = std::fopen(tmp.c_str(), "wb");
    if (!f)
        return io_error(err, err_cap, "could not create checkpoint",
                        GRHD_ERR_SETUP);
    bool ok = std::fwrite("KITPCHK1", 1, 8, f) == 8;
    put(f, (uint32_t)1, ok);
    put(f, (int32_t)h->num_components, ok);
    put(f, (int32_t)h->num_cells, ok);
    put(f, (int32_t)h->num_z_cells, ok);
    put(f, (int32_t)h->num_ghosts, ok);
    put(f, (int32_t)h->steps, ok);
    put(f, (int32_t)h->frame_index, ok);
    put(f, h->time, ok);
    put(f, h->next_output_time, ok);
    put(f, h->next_checkpoint_time, ok);
    for (int q = 0; q < 4; ++q)
        put(f, (uint64_t)h->recovery_totals[q], ok);
    for (int q = 0; q < 7; ++q)
        put(f, h->diagnostics[q], ok);
    for (int q = 0; q < 3; ++q)
        put(f, (uint64_t)h->diagnostic_counts[q], ok);
    const uint64_t ssize = std::strlen(signature);
    put(f, ssize, ok);
    ok = ok && std::fwrite(signature, 1, (size_t)ssize, f) == ssize;
    put(f, count, ok);
    ok = ok && std::fwrite(host.data(), sizeof(double), (size_t)count, f) ==
                   count;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok)
        return io_error(err, err_cap, "failed while writing checkpoint",
                        GRHD_ERR_SETUP);
    if (std::rename(tmp.c_str(), path) != 0)
        return io_error(err, err_cap, "could not finalize checkpoint",
                        GRHD_ERR_SETUP);
    return GRHD_OK;
}

int grhd_checkpoint_read(const char *path, grhd_checkpoint_header *h,
                         const char *expected_signature, double *state,
                         int64_t state_cs, const grhd_box *box, char *err,
                         int err_cap, void *stream)
{
    if (!path || !h)
        return io_error(err, err_cap, "null argument", GRHD_ERR_INVALID_ARG);
    std::FILE *f = std::fopen(path, "rb");
    if (!f)
        return io_error(err, err_cap, "could not open checkpoint",
                        GRHD_ERR_INVALID_ARG);
    std::string sig;
    uint64_t count = 0;
    int st = read_header(f, *h, sig, count, err, err_cap);
    if (st == GRHD_OK && expected_signature && sig != expected_signature)
        st = io_error(err, err_cap,
                      "checkpoint configuration does not match this run",
                      GRHD_ERR_INVALID_ARG);
    if (st != GRHD_OK || !state)
    {
        std::fclose(f);
        return st;
    }
    if (!storage_matches(box, h->num_cells, h->num_z_cells, h->num_ghosts))
    {
        std::fclose(f);
        return io_error(err, err_cap, "checkpoint grid does not match this run",
                        GRHD_ERR_INVALID_ARG);
    }
    const BoxDev b = make_box(box, state_cs);
    if (state_cs < b.gvol() ||
        count != (uint64_t)h->num_components * (uint64_t)b.gvol())
    {
        std::fclose(f);
        return io_error(err, err_cap,
                        "checkpoint state size does not match the grid",
                        GRHD_ERR_INVALID_ARG);
    }
    std::vector<double> host((size_t)count);
    const bool ok =
        std::fread(host.data(), sizeof(double), (size_t)count, f) == count;
    std::fclose(f);
    if (!ok)
        return io_error(err, err_cap, "checkpoint state data is incomplete",
                        GRHD_ERR_INVALID_ARG);
    cudaStream_t s = (cudaStream_t)stream;
    double *dev = nullptr;
    cudaError_t e = cudaMalloc((void **)&dev, count * sizeof(double));
    if (e == cudaSuccess)
    {
        e = cudaMemcpyAsync(dev, host.data(), count * sizeof(double),
                            cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            launch_checkpoint_to_state(dev, b, h->num_components, state, s);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s);
        cudaFree(dev);
    }
    if (e != cudaSuccess)
        return io_error(err, err_cap, cudaGetErrorString(e), GRHD_ERR_CUDA);
    return GRHD_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// grhd_compute_rhs_static: grhd_compute_rhs with its scratch in a fixed
// device array instead of context buffers grown by cudaMalloc.
//
// Some callers cannot let a library allocate device memory during a run:
// a host code whose own pool already holds the device memory it budgets
// (a cudaMalloc there fails or fragments that pool), and a per-box loop
// that must not stall because cudaFree waits for the whole device.  For
// them this entry point takes every scratch word from `g_rhs_scratch`, a
// file-scope device array of fixed size, and allocates nothing.
//
// The array is sized for one box of at most kStaticGhostedCells ghosted
// cells and kStaticInteriorCells interior cells; larger boxes are rejected
// with GRHD_ERR_INVALID_ARG.  Every call on a device shares the one array,
// so calls that overlap in time on that device (two streams, two host
// threads or two contexts) race on it: issue them one after another.
// Nothing in the array has to start at zero: each word a kernel reads was
// written earlier in the same call (ghost and interior primitives, sources,
// the FP32 or strided RHS copy, one accretion partial per face block).
namespace {

constexpr int64_t kStaticGhostedCells = 65536;  // e.g. 36^3 = 46656
constexpr int64_t kStaticInteriorCells = 32768; // e.g. 32^3
constexpr int64_t kStaticMdotBlocks = 4096;
constexpr int64_t kStaticPrimOff = 0;
constexpr int64_t kStaticSrcOff = 5 * kStaticGhostedCells;
constexpr int64_t kStaticKOff = kStaticSrcOff + 5 * kStaticInteriorCells;
constexpr int64_t kStaticMdotOff = kStaticKOff + 5 * kStaticInteriorCells;
constexpr int64_t kStaticDoubles = kStaticMdotOff + kStaticMdotBlocks;
static_assert(kStaticSrcOff % 32 == 0 && kStaticKOff % 32 == 0 &&
                  kStaticMdotOff % 32 == 0,
              "static scratch regions start on 256-byte boundaries");

static __device__ __align__(256) double g_rhs_scratch[kStaticDoubles];

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mutex;
double *g_static_addr[kStaticMaxDevices] = {};

// The address of g_rhs_scratch on the current device, looked up once per
// device.  The first call on a device makes this lookup (which may load the
// module on that device); later calls only read the cached pointer.
int static_scratch(grhd_ctx *ctx, double **out)
{
    if (ctx->device < 0 || ctx->device >= kStaticMaxDevices)
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, nullptr,
                         0.0, "device ordinal outside the static scratch "
                              "table");
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (!g_static_addr[ctx->device])
    {
        void *p = nullptr;
        GRHD_CUDA(ctx, cudaGetSymbolAddress(&p, g_rhs_scratch));
        g_static_addr[ctx->device] = static_cast<double *>(p);
    }
    *out = g_static_addr[ctx->device];
    return GRHD_OK;
}

__global__ void k_static_scratch_fill(double v)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
         q < kStaticDoubles; q += (int64_t)gridDim.x * blockDim.x)
        g_rhs_scratch[q] = v;
}

// The three RHS launches count in the context's launch counter; they are
// not timed by the per-kernel profile (that would take events from the
// context's pool).
template <typename T>
void enqueue_rhs_static(grhd_ctx *ctx, T *rhs, double *state, const BoxDev &b,
                        const Background &bg, const double inv_dx[3],
                        double *base, cudaStream_t s)
{
    T *prim = scratch<T>(base + kStaticPrimOff);
    T *src = scratch<T>(base + kStaticSrcOff);
    double *mdot_part = base + kStaticMdotOff;
    launch_fill_ghosts<T>(state, prim, b, bg, ctx->opt, ctx->status, s);
    launch_cells<T>(state, prim, src, b, bg, ctx->opt, ctx->status, s);
    launch_faces<T>(prim, src, rhs, b, bg, ctx->opt, inv_dx, ctx->zchunk,
                    mdot_part, s);
    ctx->launches += 3;
    if (ctx->params.accretion_radius > 0.0)
    {
        ++ctx->launches;
        launch_mdot_sum(mdot_part, face_blocks(ctx, b), 0.0,
                        ctx->mdot_acc, s);
    }
}

} // namespace

extern "C" int grhd_compute_rhs_static(grhd_ctx *ctx, double *rhs,
                                       int64_t rhs_cs, double *state,
                                       int64_t state_cs, const grhd_box *box,
                                       const double inverse_dx[3], double time,
                                       void *stream)
{
    int st = common_checks(ctx, state, box);
    if (st)
        return st;
    if (!rhs || !inverse_dx)
        return set_error(ctx, GRHD_ERR_INVALID_ARG, 0, nullptr, 0.0,
                         "null rhs or inverse_dx");
    cudaStream_t s = (cudaStream_t)stream;
    const BoxDev b = make_box(box, state_cs);
    if ((st = check_strides(ctx, b, state_cs, rhs_cs)))
        return st;
    if (b.gvol() > kStaticGhostedCells || b.ivol() > kStaticInteriorCells)
    {
        char msg[200];
        std::snprintf(msg, sizeof(msg),
                      "box too large for the static RHS scratch: %lld "
                      "ghosted / %lld interior cells (limits %lld / %lld)",
                      (long long)b.gvol(), (long long)b.ivol(),
                      (long long)kStaticGhostedCells,
                      (long long)kStaticInteriorCells);
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, nullptr,
                         0.0, msg);
    }
    if (face_blocks(ctx, b) > kStaticMdotBlocks)
    {
        char msg[200];
        std::snprintf(msg, sizeof(msg),
                      "box too large for the static RHS scratch: its face "
                      "pass needs %lld accretion partials (limit %lld)",
                      (long long)face_blocks(ctx, b),
                      (long long)kStaticMdotBlocks);
        return set_error(ctx, GRHD_ERR_INVALID_ARG, GRHD_WHERE_NONE, nullptr,
                         0.0, msg);
    }
    double *base = nullptr;
    if ((st = static_scratch(ctx, &base)) || (st = reset_status(ctx, s)))
        return st;
    const Background bg = make_background(ctx->params, time);
    double *kbuf = base + kStaticKOff;
    if (ctx->params.precision == GRHD_PRECISION_MIXED)
    {
        enqueue_rhs_static<float>(ctx, scratch<float>(kbuf), state, b, bg,
                                  inverse_dx, base, s);
        ++ctx->launches;
        launch_widen(scratch<float>(kbuf), b.ivol(), rhs, rhs_cs, s);
    }
    else if (rhs_cs == b.ivol())
        enqueue_rhs_static<double>(ctx, rhs, state, b, bg, inverse_dx, base,
                                   s);
    else
    {
        enqueue_rhs_static<double>(ctx, kbuf, state, b, bg, inverse_dx, base,
                                   s);
        for (int c = 0; c < 5; ++c)
            GRHD_CUDA(ctx, cudaMemcpyAsync(rhs + c * rhs_cs,
                                           kbuf + c * b.ivol(),
                                           b.ivol() * sizeof(double),
                                           cudaMemcpyDeviceToDevice, s));
    }
    return finish_status(ctx, b, state, bg, s);
}

// Test support: sets every word of the fixed array on the context's device
// to `value`, so that a test can show that no word of it has to hold any
// particular value before a grhd_compute_rhs_static call.
extern "C" int grhd_static_scratch_fill(grhd_ctx *ctx, double value,
                                        void *stream)
{
    if (!ctx)
        return GRHD_ERR_INVALID_ARG;
    GRHD_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    k_static_scratch_fill<<<148, 256, 0, s>>>(value);
    GRHD_CUDA(ctx, cudaGetLastError());
    GRHD_CUDA(ctx, cudaStreamSynchronize(s));
    return GRHD_OK;
}

// Host helpers shared with the ensemble driver (grhd_ensemble.cu).
namespace grhd {
namespace host {
Options options_of(const grhd_params &p) { return make_options(p); }
Background background_of(const grhd_params &p, double t)
{
    return make_background(p, t);
}
BoxDev box_of(const grhd_box *b, int64_t state_cs)
{
    return make_box(b, state_cs);
}
bool box_valid(const grhd_box *b) { return valid_box(b); }
bool box_whole_domain(const grhd_box *b) { return box_is_domain(b); }
} // namespace host
} // namespace grhd
