// grhd_adjoint.cu -- discrete adjoint of the FP64 Kerr-Schild operator
// (new; the reference has no adjoint): reverse-mode kernels of one RHS
// evaluation and of one RK4 step, a checkpointed forward/backward driver
// for J = time integral of the rest-mass accretion rate, and the gradient
// of J with respect to the eight parameters of the torus initial data
// (amplitude, polytropic constant, spin, five azimuthal modes).
//
// Forward sweep.  The RK4 step is the operator's own (grhd_advance_rk4
// arithmetic): the RHS runs the library's ghost-fill, cell and face
// kernels; the stage combination + post-update recovery runs here so that
// it can record, per cell, the pre-recovery state Y, its con2prim pressure
// and which recovery branch was taken.  A bits pass records the MUSCL
// limiter branch of every cell, direction and primitive.  Checkpoints of
// the whole state are kept every `checkpoint_every` steps; the tape (the
// stage states, primitive caches, limiter bits, Y, pressures, branches) of
// one checkpoint segment is rebuilt from its checkpoint when the backward
// sweep reaches it.
//
// Reverse sweep of one RHS evaluation (lambda_k = adjoint of the RHS):
//   face kernels (one per direction): per face, lambda_F = (lambda_k[R] -
//     lambda_k[L]) / dx (+ the accretion weight on sphere faces), then the
//     reverse of the MUSCL-HLLE face with the recorded limiter branches;
//     writes the adjoints of the two reconstructed face states;
//   shell kernel: per physical ghost cell, the adjoint of its primitive
//     cache gathered from the faces, through the ghost's floors back to the
//     con2prim of its source cell;
//   cell kernel: per interior cell, gathers the face-state adjoints through
//     the replayed slopes, adds the ghosts it fed, reverses the sources and
//     con2prim (implicit function theorem), and continues straight into the
//     reverse of the RK4 stage combination and of the recovery.
// Every face is reversed once; the cell gather reads the four faces whose
// stencil contains the cell.  Spin adjoints are the metric-field adjoints
// contracted with the dual-number spin derivative of the metric; block
// sums go to per-block slots summed in a fixed order (deterministic).
#include "grhd_adjoint.cuh"
#include "grhd_adjoint_items.cuh"
#include "grhd_b200.h"
#include "grhd_tangent.cuh"
#include "grhd_host.cuh"
#include "grhd_kernels.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <utility>
#include <vector>

using namespace grhd;
using namespace grhd::adj;

namespace {

constexpr int kAdjThreads = 128;
constexpr int kSpinSlots = 8; // kernel classes with spin partials
const unsigned long long kNoErr = ~0ull;

// ----------------------------------------------------------- kernels

__device__ inline void block_add(double v, double *slot)
{
    __shared__ double red[32];
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, off);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        red[w] = v;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double s = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q)
            s += red[q];
        slot[blockIdx.x] += s;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256)
    k_adj_bits(BoxDev b, Options o, const double *P, unsigned *bits)
{
    const int64_t n = b.gvol();
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n;
         g += (int64_t)gridDim.x * blockDim.x)
        bits_item(b, o, P, bits, g);
}

__global__ void __launch_bounds__(256)
    k_adj_stage(BoxDev b, Options o, double M, double a, const double *un,
                const double *kv, double *acc, int stage, double dt,
                double *out, double *Y, double *pY, unsigned char *br)
{
    const int64_t n = b.ivol();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        stage_tape_item(b, o, M, a, un, kv, acc, stage, dt, out, Y, pY, br,
                        t);
}

// three resident blocks per SM (168 registers, small spills)
__global__ void __launch_bounds__(kAdjThreads, 3)
    k_adj_faces(AdjRhs A, int d, double *slot)
{
    int n[3] = {A.b.in[0], A.b.in[1], A.b.in[2]};
    n[d] += 1;
    const int64_t nf = (int64_t)n[0] * n[1] * n[2];
    double spin = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nf;
         t += (int64_t)gridDim.x * blockDim.x)
        spin += face_rev_item(A, d, t);
    block_add(spin, slot);
}

__global__ void __launch_bounds__(256) k_adj_shell(AdjRhs A, double *slot)
{
    const int64_t n = A.b.gvol();
    double spin = 0.0;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n;
         g += (int64_t)gridDim.x * blockDim.x)
        spin += shell_rev_item(A, g);
    block_add(spin, slot);
}

__global__ void __launch_bounds__(kAdjThreads)
    k_adj_cells(AdjRhs A, AdjStage S, double *slot)
{
    const int64_t n = A.b.ivol();
    double spin = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        spin += cell_rev_item(A, S, t);
    block_add(spin, slot);
}

__global__ void __launch_bounds__(256)
    k_adj_proj(BoxDev b, Options o, double M, double a, double dt,
               const double *lam, const double *Y, const double *pY,
               const unsigned char *br, double *A, double *acc, double *lamk,
               double *slot)
{
    const int64_t n = b.ivol();
    double spin = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        spin += proj_rev_item(b, o, M, a, dt, lam, Y, pY, br, A, acc, lamk, t);
    block_add(spin, slot);
}

__global__ void __launch_bounds__(256)
    k_adj_torus_fill(TorusArgs T, double *state)
{
    const int64_t n = T.b.gvol();
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n;
         g += (int64_t)gridDim.x * blockDim.x)
        torus_fill_item(T, state, g);
}

__global__ void __launch_bounds__(kAdjThreads)
    k_adj_torus_tangent(TorusArgs T, const double *lam, double *tangent,
                        int64_t tcs, double *slots /* [8][grid] */)
{
    const int64_t n = T.b.ivol();
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        torus_tangent_item(T, lam, tangent, tcs, t, acc);
    for (int p = 0; p < 8; ++p)
        block_add(acc[p], slots + (int64_t)p * gridDim.x);
}

// ------------------------------------------------ tangent-linear kernels

__global__ void __launch_bounds__(kAdjThreads) k_tan_cells(TanRhs A)
{
    const int64_t n = A.b.ivol();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        tan_cell_item(A, t);
}

__global__ void __launch_bounds__(256) k_tan_ghosts(TanRhs A)
{
    const int64_t n = A.b.gvol();
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n;
         g += (int64_t)gridDim.x * blockDim.x)
        tan_ghost_item(A, g);
}

__global__ void __launch_bounds__(kAdjThreads) k_tan_rhs(TanRhs A,
                                                         double *slot)
{
    const int64_t n = A.b.ivol();
    double m = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        m += tan_rhs_item(A, t);
    block_add(m, slot);
}

__global__ void __launch_bounds__(256)
    k_tan_stage(BoxDev b, Options o, double M, double a, double da, int stage,
                double dt, const double *dUn, const double *dk, double *dacc,
                const double *Y, const double *pY, const unsigned char *br,
                double *out)
{
    const int64_t n = b.ivol();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        tan_stage_item(b, o, M, a, da, stage, dt, dUn, dk, dacc, Y, pY, br,
                       out, t);
}

struct Direction
{
    double v[8];
};

// dU0 = sum_k v_k dU0/dtheta_k over the interior (tan0: [8][5][n]).
__global__ void __launch_bounds__(256)
    k_tan_combine(int64_t n, const double *tan0, Direction v, double *dU)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        for (int q = 0; q < 5; ++q)
        {
            double s = 0.0;
            for (int k = 0; k < 8; ++k)
                s += v.v[k] * tan0[((int64_t)k * 5 + q) * n + t];
            dU[q * n + t] = s;
        }
}

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

} // namespace

// ------------------------------------------------------------- driver

struct grhd_adjoint
{
    grhd_params params;
    grhd_box box;
    Options o;
    Background bg;
    BoxDev b; // cs = pcs = gvol, rcs = ivol
    int device = 0;
    int steps = 0, every = 1, nseg = 0;
    double dt = 0.0;
    double inv_dx[3];
    int grid = 0; // blocks of the reverse kernels
    // memory
    unsigned char *arena = nullptr;
    struct Slot
    {
        double *U[4], *P[4], *Y[4], *pY[4];
        unsigned *bits[4];
        unsigned char *br[4];
    };
    std::vector<Slot> slots;
    double *ckpt = nullptr; // [nseg][11][gvol]
    double *Xend = nullptr;
    double *kbuf = nullptr, *accbuf = nullptr, *src = nullptr;
    double *mdot_part = nullptr, *mdot_acc = nullptr;
    DevStatus *status = nullptr;
    double *fb = nullptr, *gbuf = nullptr;
    double *lam = nullptr, *lamA = nullptr, *lamAcc = nullptr,
           *lamK = nullptr;
    double *spin_slots = nullptr; // [kSpinSlots][grid]
    double *tan_slots = nullptr;  // [8][grid]
    // last forward
    bool have_forward = false;
    bool tape_is_last_segment = false;
    grhd_adjoint_torus torus;
    TorusSetup setup;
    double J = 0.0;
    long long launches = 0;
    grhd_error last_error;
};

namespace {

int adj_error(grhd_adjoint *a, int status, const char *msg)
{
    grhd_error &e = a->last_error;
    e.status = status;
    e.where = 0;
    e.cell[0] = e.cell[1] = e.cell[2] = 0;
    e.residual = 0.0;
    std::snprintf(e.message, sizeof(e.message), "%s", msg);
    return status;
}

#define ADJ_CUDA(a, call)                                                     \
    do                                                                        \
    {                                                                         \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess)                                                \
        {                                                                     \
            char m_[200];                                                     \
            std::snprintf(m_, sizeof(m_), "CUDA error in %s: %s", #call,      \
                          cudaGetErrorString(e_));                            \
            return adj_error((a), GRHD_ERR_CUDA, m_);                         \
        }                                                                     \
    } while (0)

int grid_of(int64_t n, int threads, int cap)
{
    int64_t g = (n + threads - 1) / threads;
    if (g > cap)
        g = cap;
    return (int)(g < 1 ? 1 : g);
}

// The taped forward RK4 step of slot sl from sl.U[0] into `next`.
void forward_step(grhd_adjoint *a, grhd_adjoint::Slot &sl, double *next,
                  cudaStream_t s)
{
    const BoxDev &b = a->b;
    const int gi = grid_of(b.ivol(), 256, 148 * 16);
    const int gg = grid_of(b.gvol(), 256, 148 * 16);
    for (int st = 0; st < 4; ++st)
    {
        double *U = sl.U[st];
        launch_fill_ghosts<double>(U, sl.P[st], b, a->bg, a->o, a->status, s);
        launch_cells<double>(U, sl.P[st], a->src, b, a->bg, a->o, a->status,
                             s);
        launch_faces<double>(sl.P[st], a->src, a->kbuf, b, a->bg, a->o,
                             a->inv_dx, 0, a->mdot_part, s);
        if (a->o.accretion_radius > 0.0)
            launch_mdot_sum(a->mdot_part, face_kernel_blocks(b, 0),
                            a->dt / 6.0 * stage_weight(st), a->mdot_acc, s);
        k_adj_bits<<<gg, 256, 0, s>>>(b, a->o, sl.P[st], sl.bits[st]);
        double *out = (st < 3) ? sl.U[st + 1] : next;
        k_adj_stage<<<gi, 256, 0, s>>>(b, a->o, a->bg.M, a->bg.a, sl.U[0],
                                       a->kbuf, a->accbuf, st, a->dt, out,
                                       sl.Y[st], sl.pY[st], sl.br[st]);
        a->launches += 6;
    }
}

AdjRhs rhs_args(grhd_adjoint *a, const grhd_adjoint::Slot &sl, int st,
                double mu)
{
    AdjRhs A;
    A.b = a->b;
    A.o = a->o;
    A.M = a->bg.M;
    A.a = a->bg.a;
    for (int d = 0; d < 3; ++d)
        A.inv_dx[d] = a->inv_dx[d];
    A.U = sl.U[st];
    A.P = sl.P[st];
    A.bits = sl.bits[st];
    A.lamk = a->lamK;
    A.mu = mu;
    A.fb = a->fb;
    A.gbuf = a->gbuf;
    return A;
}

// Reverse of one RHS evaluation at stage st of slot sl and of the stage
// combination (S.stage = st) or RHS only (S.stage = -1).
void reverse_rhs(grhd_adjoint *a, const grhd_adjoint::Slot &sl, int st,
                 double mu, const AdjStage &S, cudaStream_t s)
{
    const AdjRhs A = rhs_args(a, sl, st, mu);
    for (int d = 0; d < 3; ++d)
        k_adj_faces<<<a->grid, kAdjThreads, 0, s>>>(
            A, d, a->spin_slots + (int64_t)d * a->grid);
    k_adj_shell<<<a->grid, 256, 0, s>>>(A, a->spin_slots +
                                               (int64_t)3 * a->grid);
    k_adj_cells<<<a->grid, kAdjThreads, 0, s>>>(
        A, S, a->spin_slots + (int64_t)4 * a->grid);
    a->launches += 5;
}

// Reverse of one taped RK4 step: lam (adjoint of U^{n+1}) -> lam (of U^n).
// mu_scale multiplies the accretion weights (1 for J).
void reverse_step(grhd_adjoint *a, const grhd_adjoint::Slot &sl,
                  double mu_scale, cudaStream_t s)
{
    const BoxDev &b = a->b;
    k_adj_proj<<<a->grid, 256, 0, s>>>(
        b, a->o, a->bg.M, a->bg.a, a->dt, a->lam, sl.Y[3], sl.pY[3], sl.br[3],
        a->lamA, a->lamAcc, a->lamK, a->spin_slots + (int64_t)5 * a->grid);
    ++a->launches;
    for (int st = 3; st >= 0; --st)
    {
        AdjStage S;
        S.stage = st;
        S.dt = a->dt;
        S.Y = st >= 1 ? sl.Y[st - 1] : nullptr;
        S.pY = st >= 1 ? sl.pY[st - 1] : nullptr;
        S.br = st >= 1 ? sl.br[st - 1] : nullptr;
        S.A = a->lamA;
        S.acc = a->lamAcc;
        S.lamk = a->lamK;
        S.out = a->lam;
        reverse_rhs(a, sl, st, mu_scale * a->dt / 6.0 * stage_weight(st), S,
                    s);
    }
}

int check_status(grhd_adjoint *a, cudaStream_t s)
{
    DevStatus st;
    ADJ_CUDA(a, cudaMemcpyAsync(&st, a->status, sizeof(st),
                                cudaMemcpyDeviceToHost, s));
    ADJ_CUDA(a, cudaStreamSynchronize(s));
    if (st.err_key != kNoErr)
        return adj_error(a, GRHD_ERR_RECOVERY,
                         "con2prim failed in the adjoint's forward sweep");
    return GRHD_OK;
}

int reset_status(grhd_adjoint *a, cudaStream_t s)
{
    DevStatus st;
    std::memset(&st, 0, sizeof(st));
    st.err_key = kNoErr;
    ADJ_CUDA(a, cudaMemcpyAsync(a->status, &st, sizeof(st),
                                cudaMemcpyHostToDevice, s));
    return GRHD_OK;
}

// Sum of the per-block slots in a fixed order.
int sum_slots(grhd_adjoint *a, const double *dev, int count, double *out,
              cudaStream_t s)
{
    std::vector<double> h((size_t)count);
    ADJ_CUDA(a, cudaMemcpyAsync(h.data(), dev, sizeof(double) * count,
                                cudaMemcpyDeviceToHost, s));
    ADJ_CUDA(a, cudaStreamSynchronize(s));
    double t = 0.0;
    for (int i = 0; i < count; ++i)
        t += h[i];
    *out = t;
    return GRHD_OK;
}

int make_torus_args(grhd_adjoint *a, const grhd_adjoint_torus *tp,
                    TorusArgs &T)
{
    TorusSetup S;
    if (!torus_setup(a->params.ks_mass, tp->spin, tp->inner_radius,
                     tp->pressure_max_radius, tp->max_velocity_squared,
                     a->o.G, S))
        return adj_error(a, GRHD_ERR_SETUP,
                         "no torus for these radii and spin");
    a->setup = S;
    const double K = tp->entropy > 0.0 ? tp->entropy : S.K_unit;
    T.b = a->b;
    T.o = a->o;
    T.M = a->params.ks_mass;
    T.th.A = tp->amplitude;
    T.th.K = K;
    T.th.a = tp->spin;
    for (int m = 0; m < 5; ++m)
    {
        T.th.eps[m] = tp->mode_amplitude[m];
        T.phase[m] = tp->mode_phase[m];
    }
    T.th.ell = S.ell;
    T.th.W_in = S.W_in;
    for (int p = 0; p < 8; ++p)
    {
        TorusThetaT<Dual> &d = T.thd[p];
        d.A = Dual(tp->amplitude, p == 0 ? 1.0 : 0.0);
        d.K = Dual(K, p == 1 ? 1.0 : 0.0);
        d.a = Dual(tp->spin, p == 2 ? 1.0 : 0.0);
        for (int m = 0; m < 5; ++m)
            d.eps[m] = Dual(tp->mode_amplitude[m], p == 3 + m ? 1.0 : 0.0);
        d.ell = Dual(S.ell, p == 2 ? S.dell_da : 0.0);
        d.W_in = Dual(S.W_in, p == 2 ? S.dWin_da : 0.0);
    }
    T.r_in = tp->inner_radius;
    T.vmax2 = tp->max_velocity_squared;
    return GRHD_OK;
}

int copy_state_in(grhd_adjoint *a, double *dst, const double *src,
                  int64_t cs, cudaStream_t s)
{
    const int64_t gv = a->b.gvol();
    for (int c = 0; c < kStateComps; ++c)
        ADJ_CUDA(a, cudaMemcpyAsync(dst + c * gv, src + c * cs,
                                    gv * sizeof(double),
                                    cudaMemcpyDeviceToDevice, s));
    return GRHD_OK;
}

int copy5(grhd_adjoint *a, double *dst, int64_t dcs, const double *src,
          int64_t scs, int64_t n, cudaStream_t s)
{
    for (int c = 0; c < 5; ++c)
        ADJ_CUDA(a, cudaMemcpyAsync(dst + c * dcs, src + c * scs,
                                    n * sizeof(double),
                                    cudaMemcpyDeviceToDevice, s));
    return GRHD_OK;
}

// The whole forward sweep from the state in slots[0].U[0]: J, checkpoints.
int run_forward(grhd_adjoint *a, cudaStream_t s)
{
    const int64_t gv = a->b.gvol();
    int rc = reset_status(a, s);
    if (rc)
        return rc;
    ADJ_CUDA(a, cudaMemsetAsync(a->mdot_acc, 0, 2 * sizeof(double), s));
    for (int n = 0; n < a->steps; ++n)
    {
        const int j = n % a->every, seg = n / a->every;
        grhd_adjoint::Slot &sl = a->slots[j];
        if (j == 0)
            ADJ_CUDA(a, cudaMemcpyAsync(a->ckpt + (int64_t)seg * kStateComps *
                                                      gv,
                                        sl.U[0],
                                        kStateComps * gv * sizeof(double),
                                        cudaMemcpyDeviceToDevice, s));
        const bool last_in_seg = (j == a->every - 1) || (n == a->steps - 1);
        double *next = last_in_seg ? a->Xend : a->slots[j + 1].U[0];
        forward_step(a, sl, next, s);
        if (last_in_seg && n < a->steps - 1)
            ADJ_CUDA(a, cudaMemcpyAsync(a->slots[0].U[0], a->Xend,
                                        kStateComps * gv * sizeof(double),
                                        cudaMemcpyDeviceToDevice, s));
    }
    double acc[2];
    ADJ_CUDA(a, cudaMemcpyAsync(acc, a->mdot_acc, sizeof(acc),
                                cudaMemcpyDeviceToHost, s));
    rc = check_status(a, s);
    if (rc)
        return rc;
    a->J = acc[1];
    a->tape_is_last_segment = true;
    return GRHD_OK;
}

} // namespace

extern "C" {

void grhd_default_adjoint_torus(grhd_adjoint_torus *t)
{
    std::memset(t, 0, sizeof(*t));
    t->amplitude = 1.0;
    t->entropy = 0.0; // 0: the value giving density 1 at the maximum
    t->spin = 0.7;
    const double amp[5] = {1.0e-2, 8.0e-3, 6.0e-3, 4.0e-3, 2.0e-3};
    const double ph[5] = {0.3, 1.1, 2.0, 4.0, 5.5};
    for (int m = 0; m < 5; ++m)
    {
        t->mode_amplitude[m] = amp[m];
        t->mode_phase[m] = ph[m];
    }
    t->inner_radius = 3.5;
    t->pressure_max_radius = 6.0;
    t->max_velocity_squared = 0.8;
}

int grhd_adjoint_unit_entropy(const grhd_params *params,
                              const grhd_adjoint_torus *t, double *K)
{
    if (!params || !t || !K)
        return GRHD_ERR_INVALID_ARG;
    TorusSetup S;
    if (!torus_setup(params->ks_mass, t->spin, t->inner_radius,
                     t->pressure_max_radius, t->max_velocity_squared,
                     params->adiabatic_index, S))
        return GRHD_ERR_SETUP;
    *K = S.K_unit;
    return GRHD_OK;
}

int grhd_adjoint_create(const grhd_params *params, const grhd_box *box,
                        int steps, int checkpoint_every, double dt,
                        grhd_adjoint **out)
{
    if (!out)
        return GRHD_ERR_INVALID_ARG;
    *out = nullptr;
    if (!params || !box)
        return GRHD_ERR_INVALID_ARG;
    grhd_adjoint *a = new (std::nothrow) grhd_adjoint();
    if (!a)
        return GRHD_ERR_CUDA;
    std::memset(&a->last_error, 0, sizeof(a->last_error));
    *out = a;
    a->params = *params;
    a->box = *box;
    if (params->background != GRHD_BG_KERR_SCHILD ||
        params->precision != GRHD_PRECISION_FP64)
        return adj_error(a, GRHD_ERR_INVALID_ARG,
                         "the adjoint supports the FP64 Kerr-Schild operator");
    if (!host::box_valid(box) || !host::box_whole_domain(box) ||
        box->ghost != 2)
        return adj_error(a, GRHD_ERR_INVALID_ARG,
                         "the adjoint needs one box covering the domain, "
                         "ghost width 2");
    if (!(params->dx > 0.0) || steps < 1 || checkpoint_every < 1 ||
        !(dt > 0.0))
        return adj_error(a, GRHD_ERR_INVALID_ARG,
                         "dx, dt, steps and checkpoint_every must be "
                         "positive");
    ADJ_CUDA(a, cudaGetDevice(&a->device));
    ADJ_CUDA(a, configure_kernels());
    a->o = host::options_of(*params);
    a->bg = host::background_of(*params, 0.0);
    const BoxDev b0 = host::box_of(box, 1);
    a->b = b0;
    a->b.cs = b0.gvol();
    a->steps = steps;
    a->every = checkpoint_every < steps ? checkpoint_every : steps;
    a->nseg = (steps + a->every - 1) / a->every;
    a->dt = dt;
    for (int d = 0; d < 3; ++d)
        a->inv_dx[d] = 1.0 / params->dx;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, a->device);
    // a whole number of waves for the reverse cell kernel (2 blocks of 128
    // threads per SM) and the reverse face kernels (3 per SM)
    a->grid = sms * 6;

    const size_t gv = (size_t)a->b.gvol(), iv = (size_t)a->b.ivol();
    const size_t nfb = (size_t)face_kernel_blocks(a->b, 0);
    size_t off = 0;
    std::vector<size_t> offs;
    auto take = [&](size_t bytes) {
        offs.push_back(off);
        off += align256(bytes);
    };
    // slots
    for (int j = 0; j < a->every; ++j)
        for (int st = 0; st < 4; ++st)
        {
            take(kStateComps * gv * 8); // U
            take(5 * gv * 8);           // P
            take(5 * iv * 8);           // Y
            take(iv * 8);               // pY
            take(gv * 4);               // bits
            take(iv);                   // br
        }
    take((size_t)a->nseg * kStateComps * gv * 8); // ckpt
    take(kStateComps * gv * 8);                   // Xend
    take(5 * iv * 8);                             // kbuf
    take(5 * iv * 8);                             // accbuf
    take(5 * iv * 8);                             // src
    take(nfb * 8);                                // mdot_part
    take(2 * 8);                                  // mdot_acc
    take(sizeof(DevStatus));                      // status
    take(30 * gv * 8);                            // fb
    take(5 * gv * 8);                             // gbuf
    take(5 * iv * 8);                             // lam
    take(5 * iv * 8);                             // lamA
    take(5 * iv * 8);                             // lamAcc
    take(5 * iv * 8);                             // lamK
    take((size_t)kSpinSlots * a->grid * 8);       // spin
    take((size_t)8 * a->grid * 8);                // tangent slots
    ADJ_CUDA(a, cudaMalloc(&a->arena, off));
    size_t q = 0;
    auto P = [&](size_t i) { return a->arena + offs[i]; };
    a->slots.resize(a->every);
    for (int j = 0; j < a->every; ++j)
        for (int st = 0; st < 4; ++st)
        {
            grhd_adjoint::Slot &sl = a->slots[j];
            sl.U[st] = (double *)P(q++);
            sl.P[st] = (double *)P(q++);
            sl.Y[st] = (double *)P(q++);
            sl.pY[st] = (double *)P(q++);
            sl.bits[st] = (unsigned *)P(q++);
            sl.br[st] = (unsigned char *)P(q++);
        }
    a->ckpt = (double *)P(q++);
    a->Xend = (double *)P(q++);
    a->kbuf = (double *)P(q++);
    a->accbuf = (double *)P(q++);
    a->src = (double *)P(q++);
    a->mdot_part = (double *)P(q++);
    a->mdot_acc = (double *)P(q++);
    a->status = (DevStatus *)P(q++);
    a->fb = (double *)P(q++);
    a->gbuf = (double *)P(q++);
    a->lam = (double *)P(q++);
    a->lamA = (double *)P(q++);
    a->lamAcc = (double *)P(q++);
    a->lamK = (double *)P(q++);
    a->spin_slots = (double *)P(q++);
    a->tan_slots = (double *)P(q++);
    // the face kernels leave the faces they do not own untouched
    ADJ_CUDA(a, cudaMemset(a->fb, 0, 30 * gv * 8));
    ADJ_CUDA(a, cudaMemset(a->gbuf, 0, 5 * gv * 8));
    return GRHD_OK;
}

void grhd_adjoint_destroy(grhd_adjoint *a)
{
    if (!a)
        return;
    if (a->arena)
    {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(a->device);
        cudaFree(a->arena);
        cudaSetDevice(prev);
    }
    delete a;
}

int grhd_adjoint_last_error(const grhd_adjoint *a, grhd_error *out)
{
    if (!a || !out)
        return GRHD_ERR_INVALID_ARG;
    *out = a->last_error;
    return GRHD_OK;
}

long long grhd_adjoint_launch_count(const grhd_adjoint *a)
{
    return a ? a->launches : 0;
}

int grhd_adjoint_initial_data(grhd_adjoint *a, const grhd_adjoint_torus *t,
                              double *state, int64_t state_cs,
                              double *tangent, int64_t tangent_comp_stride,
                              void *stream)
{
    if (!a || !t || (!state && !tangent))
        return GRHD_ERR_INVALID_ARG;
    if (!a->arena)
        return adj_error(a, GRHD_ERR_INVALID_ARG, "adjoint not created");
    cudaStream_t s = (cudaStream_t)stream;
    ADJ_CUDA(a, cudaSetDevice(a->device));
    TorusArgs T;
    int rc = make_torus_args(a, t, T);
    if (rc)
        return rc;
    if (state)
    {
        if (state_cs < a->b.gvol())
            return adj_error(a, GRHD_ERR_INVALID_ARG, "state stride too small");
        T.b.cs = state_cs;
        k_adj_torus_fill<<<grid_of(a->b.gvol(), 256, 148 * 16), 256, 0, s>>>(
            T, state);
        ++a->launches;
    }
    if (tangent)
    {
        if (tangent_comp_stride < a->b.ivol())
            return adj_error(a, GRHD_ERR_INVALID_ARG,
                             "tangent stride too small");
        T.b = a->b;
        k_adj_torus_tangent<<<a->grid, kAdjThreads, 0, s>>>(
            T, nullptr, tangent, tangent_comp_stride, a->tan_slots);
        ++a->launches;
    }
    ADJ_CUDA(a, cudaGetLastError());
    ADJ_CUDA(a, cudaStreamSynchronize(s));
    return GRHD_OK;
}

int grhd_adjoint_forward(grhd_adjoint *a, const grhd_adjoint_torus *t,
                         double *J, void *stream)
{
    if (!a || !t)
        return GRHD_ERR_INVALID_ARG;
    if (!a->arena)
        return adj_error(a, GRHD_ERR_INVALID_ARG, "adjoint not created");
    cudaStream_t s = (cudaStream_t)stream;
    ADJ_CUDA(a, cudaSetDevice(a->device));
    TorusArgs T;
    int rc = make_torus_args(a, t, T);
    if (rc)
        return rc;
    a->bg.a = t->spin; // the torus's hole is the operator's background
    k_adj_torus_fill<<<grid_of(a->b.gvol(), 256, 148 * 16), 256, 0, s>>>(
        T, a->slots[0].U[0]);
    ++a->launches;
    rc = run_forward(a, s);
    if (rc)
        return rc;
    a->torus = *t;
    a->have_forward = true;
    if (J)
        *J = a->J;
    return GRHD_OK;
}

int grhd_adjoint_backward(grhd_adjoint *a, double grad[8], double *lambda0,
                          int64_t lambda_comp_stride, void *stream)
{
    if (!a || !grad)
        return GRHD_ERR_INVALID_ARG;
    if (!a->have_forward)
        return adj_error(a, GRHD_ERR_INVALID_ARG,
                         "backward needs a forward first");
    cudaStream_t s = (cudaStream_t)stream;
    ADJ_CUDA(a, cudaSetDevice(a->device));
    const int64_t gv = a->b.gvol(), iv = a->b.ivol();
    ADJ_CUDA(a, cudaMemsetAsync(a->lam, 0, 5 * iv * 8, s));
    ADJ_CUDA(a, cudaMemsetAsync(a->spin_slots, 0,
                                (size_t)kSpinSlots * a->grid * 8, s));
    int rc = reset_status(a, s);
    if (rc)
        return rc;
    for (int seg = a->nseg - 1; seg >= 0; --seg)
    {
        const int n0 = seg * a->every;
        const int n1 = (n0 + a->every < a->steps) ? n0 + a->every : a->steps;
        if (!(seg == a->nseg - 1 && a->tape_is_last_segment))
        {
            ADJ_CUDA(a, cudaMemcpyAsync(a->slots[0].U[0],
                                        a->ckpt + (int64_t)seg * kStateComps *
                                                      gv,
                                        kStateComps * gv * sizeof(double),
                                        cudaMemcpyDeviceToDevice, s));
            for (int n = n0; n < n1; ++n)
            {
                const int j = n - n0;
                double *next =
                    (n == n1 - 1) ? a->Xend : a->slots[j + 1].U[0];
                forward_step(a, a->slots[j], next, s);
            }
        }
        for (int n = n1 - 1; n >= n0; --n)
            reverse_step(a, a->slots[n - n0], 1.0, s);
    }
    a->tape_is_last_segment = false;
    ADJ_CUDA(a, cudaGetLastError());
    rc = check_status(a, s);
    if (rc)
        return rc;
    // initial-data tangents contracted with lambda0
    TorusArgs T;
    rc = make_torus_args(a, &a->torus, T);
    if (rc)
        return rc;
    ADJ_CUDA(a, cudaMemsetAsync(a->tan_slots, 0, (size_t)8 * a->grid * 8, s));
    k_adj_torus_tangent<<<a->grid, kAdjThreads, 0, s>>>(T, a->lam, nullptr, 0,
                                                        a->tan_slots);
    ++a->launches;
    ADJ_CUDA(a, cudaGetLastError());
    for (int p = 0; p < 8; ++p)
    {
        rc = sum_slots(a, a->tan_slots + (int64_t)p * a->grid, a->grid,
                       &grad[p], s);
        if (rc)
            return rc;
    }
    double spin;
    rc = sum_slots(a, a->spin_slots, kSpinSlots * a->grid, &spin, s);
    if (rc)
        return rc;
    grad[2] += spin;
    if (lambda0)
    {
        if (lambda_comp_stride < iv)
            return adj_error(a, GRHD_ERR_INVALID_ARG,
                             "lambda stride too small");
        rc = copy5(a, lambda0, lambda_comp_stride, a->lam, iv, iv, s);
        if (rc)
            return rc;
        ADJ_CUDA(a, cudaStreamSynchronize(s));
    }
    return GRHD_OK;
}

// Tangent-linear sweep: J and dJ = (dJ/dtheta) . direction along the same
// taped forward steps as grhd_adjoint_forward (each step's tape rebuilt and
// differentiated in forward mode, no checkpoints needed).  The buffers of
// the sweep are allocated and freed per call.
int grhd_adjoint_tangent(grhd_adjoint *a, const grhd_adjoint_torus *t,
                         const double direction[8], double *J, double *dJ,
                         void *stream)
{
    if (!a || !t || !direction || !dJ)
        return GRHD_ERR_INVALID_ARG;
    if (!a->arena)
        return adj_error(a, GRHD_ERR_INVALID_ARG, "adjoint not created");
    cudaStream_t s = (cudaStream_t)stream;
    ADJ_CUDA(a, cudaSetDevice(a->device));
    TorusArgs T;
    int rc = make_torus_args(a, t, T);
    if (rc)
        return rc;
    a->bg.a = t->spin;
    // the previous forward's tape and checkpoints are overwritten
    a->have_forward = false;
    const BoxDev &b = a->b;
    const int64_t ni = b.ivol(), gv = b.gvol();
    const size_t n5 = 5 * (size_t)ni;
    double *buf = nullptr;
    const size_t total = 8 * n5 + 6 * n5 + 5 * (size_t)gv + a->grid;
    ADJ_CUDA(a, cudaMalloc((void **)&buf, total * sizeof(double)));
    double *tan0 = buf;
    double *dUn = tan0 + 8 * n5, *dUs = dUn + n5, *dUx = dUs + n5;
    double *dS = dUx + n5, *dk = dS + n5, *dacc = dk + n5;
    double *dP = dacc + n5;
    double *slots = dP + 5 * (size_t)gv;
    auto fail = [&](int code) {
        cudaFree(buf);
        return code;
    };
    k_adj_torus_fill<<<grid_of(gv, 256, 148 * 16), 256, 0, s>>>(
        T, a->slots[0].U[0]);
    k_adj_torus_tangent<<<a->grid, kAdjThreads, 0, s>>>(T, nullptr, tan0, ni,
                                                        a->tan_slots);
    Direction v;
    for (int k = 0; k < 8; ++k)
        v.v[k] = direction[k];
    const int gi = grid_of(ni, 256, 148 * 16), gg = grid_of(gv, 256, 148 * 16);
    k_tan_combine<<<gi, 256, 0, s>>>(ni, tan0, v, dUn);
    a->launches += 3;
    if (cudaMemsetAsync(slots, 0, a->grid * sizeof(double), s) != cudaSuccess ||
        cudaMemsetAsync(a->mdot_acc, 0, 2 * sizeof(double), s) != cudaSuccess)
        return fail(adj_error(a, GRHD_ERR_CUDA, "tangent set-up failed"));
    if ((rc = reset_status(a, s)))
        return fail(rc);
    grhd_adjoint::Slot &sl = a->slots[0];
    for (int n = 0; n < a->steps; ++n)
    {
        forward_step(a, sl, a->Xend, s);
        for (int st = 0; st < 4; ++st)
        {
            TanRhs R;
            R.b = b;
            R.o = a->o;
            R.M = a->bg.M;
            R.a = a->bg.a;
            R.da = direction[2];
            for (int d = 0; d < 3; ++d)
                R.inv_dx[d] = a->inv_dx[d];
            R.U = sl.U[st];
            R.P = sl.P[st];
            R.bits = sl.bits[st];
            R.dU = st == 0 ? dUn : dUs;
            R.dP = dP;
            R.dS = dS;
            R.dk = dk;
            R.mu = a->dt / 6.0 * stage_weight(st);
            k_tan_cells<<<a->grid, kAdjThreads, 0, s>>>(R);
            k_tan_ghosts<<<gg, 256, 0, s>>>(R);
            k_tan_rhs<<<a->grid, kAdjThreads, 0, s>>>(R, slots);
            k_tan_stage<<<gi, 256, 0, s>>>(b, a->o, a->bg.M, a->bg.a,
                                           direction[2], st, a->dt, dUn, dk,
                                           dacc, sl.Y[st], sl.pY[st],
                                           sl.br[st], st < 3 ? dUs : dUx);
            a->launches += 4;
        }
        if (cudaMemcpyAsync(sl.U[0], a->Xend,
                            kStateComps * gv * sizeof(double),
                            cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            return fail(adj_error(a, GRHD_ERR_CUDA, "tangent step copy"));
        std::swap(dUn, dUx);
    }
    if (cudaGetLastError() != cudaSuccess)
        return fail(adj_error(a, GRHD_ERR_CUDA, "tangent kernel launch"));
    double acc[2];
    if (cudaMemcpyAsync(acc, a->mdot_acc, sizeof(acc), cudaMemcpyDeviceToHost,
                        s) != cudaSuccess)
        return fail(adj_error(a, GRHD_ERR_CUDA, "tangent read-back"));
    if ((rc = check_status(a, s)))
        return fail(rc);
    double d = 0.0;
    if ((rc = sum_slots(a, slots, a->grid, &d, s)))
        return fail(rc);
    cudaFree(buf);
    if (J)
        *J = acc[1];
    *dJ = d;
    return GRHD_OK;
}

int grhd_adjoint_rhs_vjp(grhd_adjoint *a, double *state, int64_t state_cs,
                         const double *rhs_bar, int64_t rhs_bar_cs,
                         double mdot_bar, double *state_bar,
                         int64_t state_bar_cs, double *spin_bar, void *stream)
{
    if (!a || !state || !rhs_bar || !state_bar)
        return GRHD_ERR_INVALID_ARG;
    const int64_t gv = a->b.gvol(), iv = a->b.ivol();
    if (state_cs < gv || rhs_bar_cs < iv || state_bar_cs < iv)
        return adj_error(a, GRHD_ERR_INVALID_ARG, "stride too small");
    cudaStream_t s = (cudaStream_t)stream;
    ADJ_CUDA(a, cudaSetDevice(a->device));
    a->have_forward = false;
    a->bg.a = a->params.ks_spin;
    a->tape_is_last_segment = false;
    grhd_adjoint::Slot &sl = a->slots[0];
    int rc = copy_state_in(a, sl.U[0], state, state_cs, s);
    if (rc)
        return rc;
    rc = reset_status(a, s);
    if (rc)
        return rc;
    const BoxDev &b = a->b;
    launch_fill_ghosts<double>(sl.U[0], sl.P[0], b, a->bg, a->o, a->status, s);
    launch_cells<double>(sl.U[0], sl.P[0], a->src, b, a->bg, a->o, a->status,
                         s);
    k_adj_bits<<<grid_of(gv, 256, 148 * 16), 256, 0, s>>>(b, a->o, sl.P[0],
                                                          sl.bits[0]);
    a->launches += 3;
    rc = copy5(a, a->lamK, iv, rhs_bar, rhs_bar_cs, iv, s);
    if (rc)
        return rc;
    ADJ_CUDA(a, cudaMemsetAsync(a->spin_slots, 0,
                                (size_t)kSpinSlots * a->grid * 8, s));
    AdjStage S;
    std::memset(&S, 0, sizeof(S));
    S.stage = -1;
    S.out = a->lam;
    reverse_rhs(a, sl, 0, mdot_bar, S, s);
    ADJ_CUDA(a, cudaGetLastError());
    rc = check_status(a, s);
    if (rc)
        return rc;
    rc = copy5(a, state_bar, state_bar_cs, a->lam, iv, iv, s);
    if (rc)
        return rc;
    // the caller's state gets its physical ghosts, as compute_rhs does
    for (int c = 0; c < kStateComps; ++c)
        ADJ_CUDA(a, cudaMemcpyAsync(state + c * state_cs, sl.U[0] + c * gv,
                                    gv * sizeof(double),
                                    cudaMemcpyDeviceToDevice, s));
    double spin = 0.0;
    rc = sum_slots(a, a->spin_slots, kSpinSlots * a->grid, &spin, s);
    if (rc)
        return rc;
    if (spin_bar)
        *spin_bar = spin;
    return GRHD_OK;
}

int grhd_adjoint_step_vjp(grhd_adjoint *a, const double *state,
                          int64_t state_cs, const double *state_bar_next,
                          int64_t next_cs, double mdot_integral_bar,
                          double *state_bar, int64_t state_bar_cs,
                          double *spin_bar, void *stream)
{
    if (!a || !state || !state_bar_next || !state_bar)
        return GRHD_ERR_INVALID_ARG;
    const int64_t gv = a->b.gvol(), iv = a->b.ivol();
    if (state_cs < gv || next_cs < iv || state_bar_cs < iv)
        return adj_error(a, GRHD_ERR_INVALID_ARG, "stride too small");
    cudaStream_t s = (cudaStream_t)stream;
    ADJ_CUDA(a, cudaSetDevice(a->device));
    a->have_forward = false;
    a->bg.a = a->params.ks_spin;
    a->tape_is_last_segment = false;
    grhd_adjoint::Slot &sl = a->slots[0];
    int rc = copy_state_in(a, sl.U[0], state, state_cs, s);
    if (rc)
        return rc;
    rc = reset_status(a, s);
    if (rc)
        return rc;
    ADJ_CUDA(a, cudaMemsetAsync(a->mdot_acc, 0, 2 * sizeof(double), s));
    forward_step(a, sl, a->Xend, s);
    rc = copy5(a, a->lam, iv, state_bar_next, next_cs, iv, s);
    if (rc)
        return rc;
    ADJ_CUDA(a, cudaMemsetAsync(a->spin_slots, 0,
                                (size_t)kSpinSlots * a->grid * 8, s));
    reverse_step(a, sl, mdot_integral_bar, s);
    ADJ_CUDA(a, cudaGetLastError());
    rc = check_status(a, s);
    if (rc)
        return rc;
    rc = copy5(a, state_bar, state_bar_cs, a->lam, iv, iv, s);
    if (rc)
        return rc;
    double spin = 0.0;
    rc = sum_slots(a, a->spin_slots, kSpinSlots * a->grid, &spin, s);
    if (rc)
        return rc;
    if (spin_bar)
        *spin_bar = spin;
    return GRHD_OK;
}

} // extern "C"
