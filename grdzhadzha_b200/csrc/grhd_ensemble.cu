// grhd_ensemble.cu -- batched ensemble of independent boxes (new; the
// reference advances one level at a time): many Kerr-Schild members of
// different sizes and parameters advanced by RK4 in one persistent launch,
// optionally replayed from a CUDA graph, with the launch shape picked by a
// measuring autotuner.  C ABI in include/grhd_b200.h.
#include "grhd_b200.h"
#include "grhd_host.cuh"
#include "grhd_kernels.cuh"

#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <vector>

using namespace grhd;

namespace {

const unsigned long long kNoErrorKey = ~0ull;
constexpr int kMinZChunk = 4;
constexpr int kMaxZChunk = 256;
constexpr double kDefaultBarrierTimeout = 4.0; // seconds per barrier wait

// Per-member values the kernel updates, in one device block.
struct alignas(64) MemberState
{
    double time;
    double mdot_acc[2];
    unsigned long long mi_bits[2];
    DevStatus st;
};

size_t align_up(size_t n) { return (n + 255) & ~(size_t)255; }

} // namespace

struct grhd_ensemble
{
    int n = 0;
    bool mixed = false;
    int device = 0;
    int num_sms = 0;
    std::vector<grhd_ensemble_member> host_members;
    std::vector<EnsMember> desc;   // without the tiling fields filled
    std::vector<int64_t> off;      // [3][n+1] ghost, cell, tile prefix sums
    unsigned char *arena = nullptr; // all per-member scratch
    MemberState *mstate = nullptr;  // device [n]
    MemberState *mstate_h = nullptr; // pinned mirror
    EnsMember *d_desc = nullptr;
    int64_t *d_off = nullptr;
    EnsControl *ctl = nullptr;
    EnsControl *ctl_h = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    grhd_ensemble_tuning tuning = {32, 1, 0.0};
    int max_bps = 1;
    unsigned int bar_extra = 0;
    double bar_timeout = kDefaultBarrierTimeout;
    std::map<int, cudaGraphExec_t> graphs; // by step count
    long long launches = 0;
    grhd_error last_error;
};

namespace {

int ens_error(grhd_ensemble *e, int status, const char *msg, int where = 0,
              const int *cell = nullptr, double residual = 0.0)
{
    grhd_error &x = e->last_error;
    x.status = status;
    x.where = where;
    for (int d = 0; d < 3; ++d)
        x.cell[d] = cell ? cell[d] : 0;
    x.residual = residual;
    std::snprintf(x.message, sizeof(x.message), "%s", msg);
    return status;
}

int ens_cuda(grhd_ensemble *e, cudaError_t err, const char *what)
{
    char buf[256];
    std::snprintf(buf, sizeof(buf), "CUDA error in %s: %s", what,
                  cudaGetErrorString(err));
    return ens_error(e, GRHD_ERR_CUDA, buf);
}

#define ENS_CUDA(e, call)                                                     \
    do                                                                        \
    {                                                                         \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess)                                                \
            return ens_cuda((e), e_, #call);                                  \
    } while (0)

void drop_graphs(grhd_ensemble *e)
{
    for (auto &g : e->graphs)
        cudaGraphExecDestroy(g.second);
    e->graphs.clear();
}

// Face tiles of member m along x, y, z for a z chunk.
void member_tiles(const BoxDev &b, int zchunk, int t[3])
{
    t[0] = (b.in[0] + kTC - 1) / kTC;
    t[1] = (b.in[1] + kTC - 1) / kTC;
    t[2] = (b.in[2] + zchunk - 1) / zchunk;
}

// Fills the tiling fields of the descriptors and the prefix tables for the
// current tuning and uploads both.
int upload_layout(grhd_ensemble *e)
{
    const int n = e->n;
    e->off.assign(3 * (size_t)(n + 1), 0);
    int64_t *og = e->off.data(), *oc = og + (n + 1), *ot = oc + (n + 1);
    for (int m = 0; m < n; ++m)
    {
        EnsMember &d = e->desc[m];
        member_tiles(d.b, e->tuning.zchunk, d.tiles);
        const int64_t items = (d.b.ivol() + kEnsItemCells - 1) / kEnsItemCells;
        const int64_t gitems = (d.nshell + kEnsItemCells - 1) / kEnsItemCells;
        og[m + 1] = og[m] + gitems;
        oc[m + 1] = oc[m] + items;
        ot[m + 1] = ot[m] + (int64_t)d.tiles[0] * d.tiles[1] * d.tiles[2];
    }
    ENS_CUDA(e, cudaMemcpy(e->d_desc, e->desc.data(),
                           sizeof(EnsMember) * (size_t)n,
                           cudaMemcpyHostToDevice));
    ENS_CUDA(e, cudaMemcpy(e->d_off, e->off.data(),
                           sizeof(int64_t) * e->off.size(),
                           cudaMemcpyHostToDevice));
    drop_graphs(e);
    return GRHD_OK;
}

EnsLaunch launch_args(grhd_ensemble *e, int steps)
{
    EnsLaunch a;
    a.m = e->d_desc;
    a.nm = e->n;
    a.off_ghost = e->d_off;
    a.off_cell = e->d_off + (e->n + 1);
    a.off_tile = e->d_off + 2 * (e->n + 1);
    a.ctl = e->ctl;
    a.steps = steps;
    a.zchunk = e->tuning.zchunk;
    a.nblocks = (unsigned)(e->tuning.blocks_per_sm * e->num_sms);
    a.bar_extra = e->bar_extra;
    a.bar_timeout_ns = (unsigned long long)(e->bar_timeout * 1.0e9);
    return a;
}

// Enqueues one launch on e->s: reset of the per-launch control words, then
// the persistent kernel.
cudaError_t enqueue_launch(grhd_ensemble *e, int steps)
{
    cudaError_t err = cudaMemsetAsync(e->ctl, 0,
                                      offsetof(EnsControl, steps_done), e->s);
    if (err != cudaSuccess)
        return err;
    const EnsLaunch a = launch_args(e, steps);
    const int grid = (int)a.nblocks;
    ++e->launches;
    return e->mixed ? launch_ensemble<float>(a, grid, e->s)
                    : launch_ensemble<double>(a, grid, e->s);
}

// Reads back the control block and member states and converts a barrier
// time-out or a recorded recovery failure into the error record.
int finish(grhd_ensemble *e)
{
    ENS_CUDA(e, cudaMemcpyAsync(e->ctl_h, e->ctl, sizeof(EnsControl),
                                cudaMemcpyDeviceToHost, e->s));
    ENS_CUDA(e, cudaMemcpyAsync(e->mstate_h, e->mstate,
                                sizeof(MemberState) * (size_t)e->n,
                                cudaMemcpyDeviceToHost, e->s));
    ENS_CUDA(e, cudaStreamSynchronize(e->s));
    if (e->ctl_h->error)
    {
        char msg[160];
        std::snprintf(msg, sizeof(msg),
                      "ensemble grid barrier wait ran out in phase %d "
                      "(state unspecified)",
                      e->ctl_h->error_phase);
        e->ctl_h->error = 0;
        return ens_error(e, GRHD_ERR_CUDA, msg);
    }
    for (int m = 0; m < e->n; ++m)
    {
        const unsigned long long key = e->mstate_h[m].st.err_key;
        if (key == kNoErrorKey)
            continue;
        const int where = (int)(key >> 56);
        const long long order = (long long)(key & ((1ull << 56) - 1));
        const EnsMember &d = e->desc[m];
        int cell[3];
        // where 4 (CFL) indexes the interior, the others the ghosted box
        const int *lo = where == GRHD_WHERE_CFL ? d.b.lo : d.b.glo;
        const int *nn = where == GRHD_WHERE_CFL ? d.b.in : d.b.gn;
        cell[0] = lo[0] + (int)(order % nn[0]);
        cell[1] = lo[1] + (int)((order / nn[0]) % nn[1]);
        cell[2] = lo[2] + (int)(order / ((long long)nn[0] * nn[1]));
        static const char *const what[5] = {
            "", " (outflow source of the boundary fill)",
            " (ghosted recovery)", " (metric sources)", " (CFL speed)"};
        char msg[200];
        std::snprintf(msg, sizeof(msg),
                      "ensemble member %d: GRHD primitive recovery failed at "
                      "cell (%d, %d, %d)%s",
                      m, cell[0], cell[1], cell[2],
                      (where >= 0 && where < 5) ? what[where] : "");
        // clear the keys so that the ensemble stays usable
        for (int q = 0; q < e->n; ++q)
            e->mstate_h[q].st.err_key = kNoErrorKey;
        ENS_CUDA(e, cudaMemcpy(e->mstate, e->mstate_h,
                               sizeof(MemberState) * (size_t)e->n,
                               cudaMemcpyHostToDevice));
        return ens_error(e, GRHD_ERR_RECOVERY, msg, where, cell);
    }
    return GRHD_OK;
}

int run(grhd_ensemble *e, int steps, bool use_graph, cudaStream_t user)
{
    ENS_CUDA(e, cudaEventRecord(e->ev_in, user));
    ENS_CUDA(e, cudaStreamWaitEvent(e->s, e->ev_in, 0));
    if (use_graph)
    {
        auto it = e->graphs.find(steps);
        if (it == e->graphs.end())
        {
            cudaGraph_t g = nullptr;
            ENS_CUDA(e, cudaStreamBeginCapture(e->s,
                                               cudaStreamCaptureModeThreadLocal));
            const cudaError_t le = enqueue_launch(e, steps);
            const cudaError_t ce = cudaStreamEndCapture(e->s, &g);
            if (le != cudaSuccess)
            {
                if (g)
                    cudaGraphDestroy(g);
                return ens_cuda(e, le, "ensemble launch under capture");
            }
            ENS_CUDA(e, ce);
            cudaGraphExec_t x = nullptr;
            const cudaError_t ie = cudaGraphInstantiate(&x, g, 0);
            cudaGraphDestroy(g);
            ENS_CUDA(e, ie);
            it = e->graphs.emplace(steps, x).first;
            --e->launches; // counted again at replay
        }
        ++e->launches;
        ENS_CUDA(e, cudaGraphLaunch(it->second, e->s));
    }
    else
        ENS_CUDA(e, enqueue_launch(e, steps));
    ENS_CUDA(e, cudaGetLastError());
    ENS_CUDA(e, cudaEventRecord(e->ev_out, e->s));
    ENS_CUDA(e, cudaStreamWaitEvent(user, e->ev_out, 0));
    return finish(e);
}

int validate_member(grhd_ensemble *e, const grhd_ensemble_member &m, int idx)
{
    char msg[200];
    const grhd_params &p = m.params;
    const char *why = nullptr;
    if (!m.state)
        why = "null state pointer";
    else if (!host::box_valid(&m.box) || !host::box_whole_domain(&m.box))
        why = "box must be valid and cover its whole domain";
    else if (p.background != GRHD_BG_KERR_SCHILD)
        why = "ensemble members must use the Kerr-Schild background";
    else if (p.ks_spin > p.ks_mass || p.ks_spin < -p.ks_mass)
        why = "Kerr-Schild spin must satisfy |a| <= M";
    else if (!(p.dx > 0.0))
        why = "GRHD grid spacing must be positive";
    else if (!(m.cfl > 0.0))
        why = "GRHD CFL number must be positive";
    else if (p.precision != e->host_members[0].params.precision)
        why = "all members must use the same precision";
    else if (m.state_comp_stride <
             host::box_of(&m.box, m.state_comp_stride).gvol())
        why = "state component stride is smaller than the ghosted box volume";
    if (!why)
        return GRHD_OK;
    std::snprintf(msg, sizeof(msg), "ensemble member %d: %s", idx, why);
    return ens_error(e, GRHD_ERR_INVALID_ARG, msg);
}

int build(grhd_ensemble *e)
{
    const int n = e->n;
    e->mixed = e->host_members[0].params.precision == GRHD_PRECISION_MIXED;
    const size_t tsz = e->mixed ? sizeof(float) : sizeof(double);
    for (int m = 0; m < n; ++m)
    {
        int st = validate_member(e, e->host_members[m], m);
        if (st)
            return st;
    }
    ENS_CUDA(e, cudaGetDevice(&e->device));
    ENS_CUDA(e, configure_kernels());
    ENS_CUDA(e, cudaDeviceGetAttribute(&e->num_sms,
                                       cudaDevAttrMultiProcessorCount,
                                       e->device));
    int bps = 0;
    ENS_CUDA(e, e->mixed ? ensemble_occupancy<float>(&bps)
                         : ensemble_occupancy<double>(&bps));
    if (bps < 1)
        return ens_error(e, GRHD_ERR_CUDA,
                         "the ensemble kernel does not fit on an SM");
    e->max_bps = bps;
    e->tuning.blocks_per_sm = 1;

    // scratch arena
    std::vector<size_t> base(n);
    size_t total = 0;
    e->desc.assign(n, EnsMember());
    for (int m = 0; m < n; ++m)
    {
        const grhd_ensemble_member &hm = e->host_members[m];
        const BoxDev b = host::box_of(&hm.box, hm.state_comp_stride);
        int t[3];
        member_tiles(b, kMinZChunk, t);
        base[m] = total;
        total += align_up(5 * (size_t)b.gvol() * tsz);         // prim
        total += 2 * align_up(5 * (size_t)b.ivol() * tsz);     // src, k
        total += align_up(5 * (size_t)b.ivol() * 8);           // acc
        total += align_up((size_t)kStateComps * b.gvol() * 8); // stage
        total += align_up((size_t)t[0] * t[1] * t[2] * 8);     // mdot parts
    }
    ENS_CUDA(e, cudaMalloc((void **)&e->arena, total));
    ENS_CUDA(e, cudaMalloc((void **)&e->mstate, sizeof(MemberState) * n));
    ENS_CUDA(e, cudaMallocHost((void **)&e->mstate_h, sizeof(MemberState) * n));
    ENS_CUDA(e, cudaMalloc((void **)&e->d_desc, sizeof(EnsMember) * n));
    ENS_CUDA(e, cudaMalloc((void **)&e->d_off, sizeof(int64_t) * 3 * (n + 1)));
    ENS_CUDA(e, cudaMalloc((void **)&e->ctl, sizeof(EnsControl)));
    ENS_CUDA(e, cudaMallocHost((void **)&e->ctl_h, sizeof(EnsControl)));
    ENS_CUDA(e, cudaStreamCreateWithFlags(&e->s, cudaStreamNonBlocking));
    ENS_CUDA(e, cudaEventCreateWithFlags(&e->ev_in, cudaEventDisableTiming));
    ENS_CUDA(e, cudaEventCreateWithFlags(&e->ev_out, cudaEventDisableTiming));

    for (int m = 0; m < n; ++m)
    {
        const grhd_ensemble_member &hm = e->host_members[m];
        EnsMember &d = e->desc[m];
        std::memset(&d, 0, sizeof(d));
        d.b = host::box_of(&hm.box, hm.state_comp_stride);
        d.sb = d.b;
        d.sb.cs = d.b.gvol();
        d.bg = host::background_of(hm.params, 0.0);
        d.o = host::options_of(hm.params);
        for (int q = 0; q < 3; ++q)
            d.inv[q] = hm.inverse_dx[q];
        d.cfl = hm.cfl;
        d.max_dt = hm.max_dt;
        d.state = hm.state;
        unsigned char *p = e->arena + base[m];
        d.prim = p;
        p += align_up(5 * (size_t)d.b.gvol() * tsz);
        d.src = p;
        p += align_up(5 * (size_t)d.b.ivol() * tsz);
        d.k = p;
        p += align_up(5 * (size_t)d.b.ivol() * tsz);
        d.acc = reinterpret_cast<double *>(p);
        p += align_up(5 * (size_t)d.b.ivol() * 8);
        d.stage = reinterpret_cast<double *>(p);
        p += align_up((size_t)kStateComps * d.b.gvol() * 8);
        d.mdot_part = reinterpret_cast<double *>(p);
        d.has_mdot = hm.params.accretion_radius > 0.0;
        d.nshell = d.b.gvol() - d.b.ivol();
        MemberState *ms = e->mstate + m;
        d.time = &ms->time;
        d.mdot_acc = ms->mdot_acc;
        d.mi_bits = ms->mi_bits;
        d.st = &ms->st;
        MemberState &h = e->mstate_h[m];
        std::memset(&h, 0, sizeof(h));
        h.time = hm.time;
        h.st.err_key = kNoErrorKey;
    }
    ENS_CUDA(e, cudaMemcpy(e->mstate, e->mstate_h, sizeof(MemberState) * n,
                           cudaMemcpyHostToDevice));
    std::memset(e->ctl_h, 0, sizeof(EnsControl));
    e->ctl_h->need_cfl = 1;
    ENS_CUDA(e, cudaMemcpy(e->ctl, e->ctl_h, sizeof(EnsControl),
                           cudaMemcpyHostToDevice));
    return upload_layout(e);
}

bool valid_tuning(const grhd_ensemble *e, const grhd_ensemble_tuning &t)
{
    return t.zchunk >= kMinZChunk && t.zchunk <= kMaxZChunk &&
           t.blocks_per_sm >= 1 && t.blocks_per_sm <= e->max_bps;
}

// Copies of everything a trial launch changes: the member states, the
// per-member device block and the carried control words.
struct Snapshot
{
    std::vector<double *> states;
    std::vector<size_t> bytes;
    MemberState *mstate = nullptr;
    EnsControl ctl;
};

size_t state_bytes(const grhd_ensemble_member &m)
{
    const BoxDev b = host::box_of(&m.box, m.state_comp_stride);
    return ((size_t)(kStateComps - 1) * (size_t)m.state_comp_stride +
            (size_t)b.gvol()) *
           sizeof(double);
}

int snapshot_take(grhd_ensemble *e, Snapshot &sn)
{
    sn.states.assign(e->n, nullptr);
    sn.bytes.assign(e->n, 0);
    for (int m = 0; m < e->n; ++m)
    {
        sn.bytes[m] = state_bytes(e->host_members[m]);
        ENS_CUDA(e, cudaMalloc((void **)&sn.states[m], sn.bytes[m]));
        ENS_CUDA(e, cudaMemcpyAsync(sn.states[m], e->host_members[m].state,
                                    sn.bytes[m], cudaMemcpyDeviceToDevice,
                                    e->s));
    }
    ENS_CUDA(e, cudaMalloc((void **)&sn.mstate, sizeof(MemberState) * e->n));
    ENS_CUDA(e, cudaMemcpyAsync(sn.mstate, e->mstate,
                                sizeof(MemberState) * e->n,
                                cudaMemcpyDeviceToDevice, e->s));
    ENS_CUDA(e, cudaMemcpyAsync(&sn.ctl, e->ctl, sizeof(EnsControl),
                                cudaMemcpyDeviceToHost, e->s));
    ENS_CUDA(e, cudaStreamSynchronize(e->s));
    return GRHD_OK;
}

int snapshot_restore(grhd_ensemble *e, const Snapshot &sn)
{
    for (int m = 0; m < e->n; ++m)
        ENS_CUDA(e, cudaMemcpyAsync(e->host_members[m].state, sn.states[m],
                                    sn.bytes[m], cudaMemcpyDeviceToDevice,
                                    e->s));
    ENS_CUDA(e, cudaMemcpyAsync(e->mstate, sn.mstate,
                                sizeof(MemberState) * e->n,
                                cudaMemcpyDeviceToDevice, e->s));
    *e->ctl_h = sn.ctl;
    ENS_CUDA(e, cudaMemcpyAsync(e->ctl, e->ctl_h, sizeof(EnsControl),
                                cudaMemcpyHostToDevice, e->s));
    ENS_CUDA(e, cudaStreamSynchronize(e->s));
    return GRHD_OK;
}

void snapshot_free(Snapshot &sn)
{
    for (double *p : sn.states)
        cudaFree(p);
    sn.states.clear();
    cudaFree(sn.mstate);
    sn.mstate = nullptr;
}

} // namespace

extern "C" {

int grhd_ensemble_create(const grhd_ensemble_member *members, int count,
                         grhd_ensemble **out)
{
    if (!out || !members || count < 1)
        return GRHD_ERR_INVALID_ARG;
    *out = nullptr;
    grhd_ensemble *e = new (std::nothrow) grhd_ensemble();
    if (!e)
        return GRHD_ERR_CUDA;
    std::memset(&e->last_error, 0, sizeof(e->last_error));
    e->n = count;
    e->host_members.assign(members, members + count);
    const int st = build(e);
    *out = e; // returned even on error so that the message can be read
    return st;
}

void grhd_ensemble_destroy(grhd_ensemble *e)
{
    if (!e)
        return;
    cudaSetDevice(e->device);
    if (e->s)
        cudaStreamSynchronize(e->s);
    drop_graphs(e);
    cudaFree(e->arena);
    cudaFree(e->mstate);
    cudaFreeHost(e->mstate_h);
    cudaFree(e->d_desc);
    cudaFree(e->d_off);
    cudaFree(e->ctl);
    cudaFreeHost(e->ctl_h);
    if (e->ev_in)
        cudaEventDestroy(e->ev_in);
    if (e->ev_out)
        cudaEventDestroy(e->ev_out);
    if (e->s)
        cudaStreamDestroy(e->s);
    delete e;
}

int grhd_ensemble_last_error(const grhd_ensemble *e, grhd_error *out)
{
    if (!e || !out)
        return GRHD_ERR_INVALID_ARG;
    *out = e->last_error;
    return GRHD_OK;
}

int grhd_ensemble_get_tuning(const grhd_ensemble *e, grhd_ensemble_tuning *t,
                             int *max_blocks_per_sm)
{
    if (!e || !t)
        return GRHD_ERR_INVALID_ARG;
    *t = e->tuning;
    if (max_blocks_per_sm)
        *max_blocks_per_sm = e->max_bps;
    return GRHD_OK;
}

int grhd_ensemble_set_tuning(grhd_ensemble *e, const grhd_ensemble_tuning *t)
{
    if (!e || !t)
        return GRHD_ERR_INVALID_ARG;
    std::memset(&e->last_error, 0, sizeof(e->last_error));
    if (!valid_tuning(e, *t))
        return ens_error(e, GRHD_ERR_INVALID_ARG,
                         "tuning out of range (zchunk in [4, 256], "
                         "blocks_per_sm in [1, occupancy limit])");
    ENS_CUDA(e, cudaSetDevice(e->device));
    e->tuning = *t;
    return upload_layout(e);
}

int grhd_ensemble_advance(grhd_ensemble *e, int steps, int use_graph,
                          void *stream)
{
    if (!e)
        return GRHD_ERR_INVALID_ARG;
    std::memset(&e->last_error, 0, sizeof(e->last_error));
    if (steps < 0)
        return ens_error(e, GRHD_ERR_INVALID_ARG, "negative step count");
    ENS_CUDA(e, cudaSetDevice(e->device));
    return run(e, steps, use_graph != 0, (cudaStream_t)stream);
}

int grhd_ensemble_autotune(grhd_ensemble *e, int trial_steps,
                           grhd_ensemble_tuning *best, void *stream)
{
    if (!e)
        return GRHD_ERR_INVALID_ARG;
    std::memset(&e->last_error, 0, sizeof(e->last_error));
    if (trial_steps < 1)
        return ens_error(e, GRHD_ERR_INVALID_ARG, "trial_steps must be >= 1");
    ENS_CUDA(e, cudaSetDevice(e->device));
    cudaStream_t user = (cudaStream_t)stream;
    ENS_CUDA(e, cudaStreamSynchronize(user));
    Snapshot sn;
    int st = snapshot_take(e, sn);
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    grhd_ensemble_tuning win = e->tuning;
    win.ms_per_step = 0.0;
    if (!st && (cudaEventCreate(&t0) != cudaSuccess ||
                cudaEventCreate(&t1) != cudaSuccess))
        st = ens_error(e, GRHD_ERR_CUDA, "event creation failed");
    const int zs[] = {8, 16, 32, 64};
    for (int zi = 0; !st && zi < 4; ++zi)
        for (int bps = 1; !st && bps <= e->max_bps; ++bps)
        {
            grhd_ensemble_tuning t = {zs[zi], bps, 0.0};
            e->tuning = t;
            if ((st = upload_layout(e)) || (st = snapshot_restore(e, sn)) ||
                (st = run(e, 1, false, user)))
                break;
            if (cudaEventRecord(t0, e->s) != cudaSuccess ||
                enqueue_launch(e, trial_steps) != cudaSuccess ||
                cudaEventRecord(t1, e->s) != cudaSuccess ||
                cudaEventSynchronize(t1) != cudaSuccess)
            {
                st = ens_error(e, GRHD_ERR_CUDA, "autotune trial failed");
                break;
            }
            if ((st = finish(e)))
                break;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, t0, t1);
            t.ms_per_step = ms / trial_steps;
            if (win.ms_per_step == 0.0 || t.ms_per_step < win.ms_per_step)
                win = t;
        }
    if (t0)
        cudaEventDestroy(t0);
    if (t1)
        cudaEventDestroy(t1);
    if (!st)
    {
        e->tuning = win;
        if (!(st = upload_layout(e)))
            st = snapshot_restore(e, sn);
    }
    snapshot_free(sn);
    if (!st && best)
        *best = win;
    return st;
}

int grhd_ensemble_member_info(grhd_ensemble *e, int member, double *time,
                              double *max_inverse_dt, double *mdot,
                              double *mdot_integral, grhd_diagnostics *diag)
{
    if (!e || member < 0 || member >= e->n)
        return GRHD_ERR_INVALID_ARG;
    ENS_CUDA(e, cudaSetDevice(e->device));
    ENS_CUDA(e, cudaStreamSynchronize(e->s));
    MemberState h;
    EnsControl c;
    ENS_CUDA(e, cudaMemcpy(&h, e->mstate + member, sizeof(h),
                           cudaMemcpyDeviceToHost));
    ENS_CUDA(e, cudaMemcpy(&c, e->ctl, sizeof(c), cudaMemcpyDeviceToHost));
    if (time)
        *time = h.time;
    if (max_inverse_dt)
    {
        double v;
        std::memcpy(&v, &h.mi_bits[c.steps_done & 1ull], sizeof(v));
        *max_inverse_dt = c.need_cfl ? 0.0 : v;
    }
    if (mdot)
        *mdot = h.mdot_acc[0];
    if (mdot_integral)
        *mdot_integral = h.mdot_acc[1];
    if (diag)
    {
        diag->num_cells = (long long)h.st.counts[0];
        diag->num_failed_recoveries = (long long)h.st.counts[1];
        diag->num_floored_primitives = (long long)h.st.counts[2];
        diag->num_conserved_resets = (long long)h.st.counts[3];
    }
    return GRHD_OK;
}

int grhd_ensemble_reset_accretion(grhd_ensemble *e)
{
    if (!e)
        return GRHD_ERR_INVALID_ARG;
    ENS_CUDA(e, cudaSetDevice(e->device));
    ENS_CUDA(e, cudaStreamSynchronize(e->s));
    for (int m = 0; m < e->n; ++m)
        ENS_CUDA(e, cudaMemset(&e->mstate[m].mdot_acc[1], 0, sizeof(double)));
    return GRHD_OK;
}

int grhd_ensemble_invalidate(grhd_ensemble *e)
{
    if (!e)
        return GRHD_ERR_INVALID_ARG;
    ENS_CUDA(e, cudaSetDevice(e->device));
    ENS_CUDA(e, cudaStreamSynchronize(e->s));
    EnsControl c;
    ENS_CUDA(e, cudaMemcpy(&c, e->ctl, sizeof(c), cudaMemcpyDeviceToHost));
    for (int m = 0; m < e->n; ++m)
        ENS_CUDA(e, cudaMemset(&e->mstate[m].mi_bits[c.steps_done & 1ull], 0,
                               sizeof(unsigned long long)));
    c.need_cfl = 1;
    ENS_CUDA(e, cudaMemcpy(e->ctl, &c, sizeof(c), cudaMemcpyHostToDevice));
    return GRHD_OK;
}

int grhd_ensemble_set_barrier_test(grhd_ensemble *e,
                                   unsigned int extra_arrivals,
                                   double timeout_seconds)
{
    if (!e || !(timeout_seconds > 0.0) || timeout_seconds > 60.0)
        return GRHD_ERR_INVALID_ARG;
    e->bar_extra = extra_arrivals;
    e->bar_timeout = timeout_seconds;
    drop_graphs(e);
    return GRHD_OK;
}

long long grhd_ensemble_launch_count(const grhd_ensemble *e)
{
    return e ? e->launches : 0;
}

} // extern "C"
