// grhd_kernels.cuh -- kernels of the fixed-background GRHD operator and the
// small host-side descriptors they take.
#pragma once

#include "grhd_device.cuh"

namespace grhd {

// One box of the level on the device: interior [lo,hi], ghosted storage
// [glo,ghi], non-periodic domain [dlo,dhi]; cs / rcs / pcs are the
// component strides of the state (11 components over the ghosted box), of
// interior-box arrays (5 components) and of the primitive cache (5
// components over the ghosted box).
struct BoxDev
{
    int lo[3], hi[3], glo[3], ghi[3], dlo[3], dhi[3];
    int gn[3], in[3];
    int64_t cs;  // state component stride
    int64_t rcs; // interior array component stride
    int64_t pcs; // primitive cache component stride (ghosted volume)
    // interior index, within the box it views, of this box's first
    // interior cell: 0 for a whole box; a z range of planes of a box (the
    // same ghosted layout and strides, its own lo/hi/in in z) starts at
    // the index of its first plane
    int64_t t0 = 0;

    __host__ __device__ int64_t gidx(int i, int j, int k) const
    {
        return (int64_t)(i - glo[0]) +
               (int64_t)gn[0] * ((int64_t)(j - glo[1]) +
                                 (int64_t)gn[1] * (int64_t)(k - glo[2]));
    }
    __host__ __device__ int64_t iidx(int i, int j, int k) const
    {
        return (int64_t)(i - lo[0]) +
               (int64_t)in[0] * ((int64_t)(j - lo[1]) +
                                 (int64_t)in[1] * (int64_t)(k - lo[2]));
    }
    __host__ __device__ int64_t gvol() const
    {
        return (int64_t)gn[0] * gn[1] * gn[2];
    }
    __host__ __device__ int64_t ivol() const
    {
        return (int64_t)in[0] * in[1] * in[2];
    }
};

// The cells of the ghosted planes k0..k1 of box b that lie outside its
// interior: whole planes below lo[2] and above hi[2], and the ring
// "ghosted plane minus interior plane" of the planes in between.  Cell t
// of that set in plane order (x fastest; in a ring the rows outside the
// interior first, then the x margins of the interior rows).
__host__ __device__ inline int64_t plane_shell_count(const BoxDev &b, int k0,
                                                     int k1)
{
    const int64_t P = (int64_t)b.gn[0] * b.gn[1];
    const int64_t R = P - (int64_t)b.in[0] * b.in[1];
    const int nb = max(0, min(k1, b.lo[2] - 1) - k0 + 1);
    const int nm = max(0, min(k1, b.hi[2]) - max(k0, b.lo[2]) + 1);
    const int nt = max(0, k1 - max(k0, b.hi[2] + 1) + 1);
    return (int64_t)(nb + nt) * P + (int64_t)nm * R;
}

__host__ __device__ inline void plane_shell_cell(const BoxDev &b, int k0,
                                                 int k1, int64_t t, int &i,
                                                 int &j, int &k)
{
    const int64_t gx = b.gn[0];
    const int64_t P = gx * b.gn[1];
    const int64_t R = P - (int64_t)b.in[0] * b.in[1];
    const int nb = max(0, min(k1, b.lo[2] - 1) - k0 + 1);
    const int nm = max(0, min(k1, b.hi[2]) - max(k0, b.lo[2]) + 1);
    const int64_t n1 = (int64_t)nb * P, n2 = (int64_t)nm * R;
    if (t < n1 || t >= n1 + n2)
    {
        // a whole ghost plane below or above the interior
        const int kb = t < n1 ? k0 : max(k0, b.hi[2] + 1);
        const int64_t u = t < n1 ? t : t - n1 - n2;
        k = kb + (int)(u / P);
        const int64_t r = u % P;
        j = b.glo[1] + (int)(r / gx);
        i = b.glo[0] + (int)(r % gx);
        return;
    }
    const int64_t u = t - n1;
    k = max(k0, b.lo[2]) + (int)(u / R);
    int64_t r = u % R;
    const int64_t ylo = b.lo[1] - b.glo[1];
    const int64_t ny_out = b.gn[1] - b.in[1];
    if (r < ny_out * gx)
    {
        const int64_t jj = r / gx;
        j = (jj < ylo) ? b.glo[1] + (int)jj : b.hi[1] + 1 + (int)(jj - ylo);
        i = b.glo[0] + (int)(r % gx);
        return;
    }
    r -= ny_out * gx;
    const int64_t xlo = b.lo[0] - b.glo[0];
    const int64_t nx_out = b.gn[0] - b.in[0];
    j = b.lo[1] + (int)(r / nx_out);
    const int64_t ii = r % nx_out;
    i = (ii < xlo) ? b.glo[0] + (int)ii : b.hi[0] + 1 + (int)(ii - xlo);
}

// Device-side status of one call: the first recovery failure in the
// reference's iteration order (key = where << 56 | linear index), the
// atmosphere-reset counters, and the CFL maximum (bit pattern of a
// non-negative double, so integer max == floating max).
struct DevStatus
{
    unsigned long long err_key;
    unsigned long long counts[4];
    unsigned long long maxinv_bits;
};

enum : int
{
    kStateComps = 11,
    kCcz4GrhdOffset = 25, // GRHD components after GRChombo's CCZ4 ones
    kD = 0,
    kS1 = 1,
    kTau = 4,
    kRho = 5,
    kEps = 6,
    kPress = 7,
    kV1 = 8
};

// Face kernel tiling: 16x16 threads own a 15x15 cell tile in (x, y) and
// march along z.
constexpr int kTB = 16;
constexpr int kTC = 15;
constexpr int kPW = kTC + 4; // primitive tile width (2 halo each side)
constexpr int kGW = kTC + 2; // geometry tile width (1 halo each side)
constexpr int kGeoFields = 16;

// Per-device kernel attributes (dynamic shared memory of the face kernels).
cudaError_t configure_kernels();
// z-march length (planes per block) of the face kernel for box b: zchunk
// when positive; otherwise face_zchunk_model with the device's resident
// face blocks (SMs x the occupancy query's blocks per SM).
int face_zchunk(const BoxDev &b, int zchunk, bool fp32);
// Of 32, 16, 8, 6 and 4 planes, the one whose launch has the shortest
// makespan when its blocks -- every full z block of every (x,y) tile, then
// the short last z row -- are list-scheduled in launch order on `slots`
// resident blocks, a block costing its planes plus its two lead-in planes
// (ties keep the longer march).  Host only; the RHS does not depend on the
// choice.
int face_zchunk_model(int nx, int ny, int nz, int64_t slots);
int64_t face_kernel_blocks(const BoxDev &b, int zchunk, bool fp32 = false);

// T is the arithmetic type of the primitive cache, sources and RHS:
// double (FP64 path) or float (mixed path).

// Physical ghost fill of the shell, then con2prim of every shell cell into
// the primitive cache.
template <typename T>
void launch_fill_ghosts(double *state, T *prim, const BoxDev &b,
                        const Background &bg, const Options &o, DevStatus *st,
                        cudaStream_t s);
// The same fill restricted to the ghosted planes k0..k1 (their cells
// outside the interior).
template <typename T>
void launch_fill_ghost_planes(double *state, T *prim, const BoxDev &b,
                              const Background &bg, const Options &o,
                              DevStatus *st, int k0, int k1, cudaStream_t s);
// Interior con2prim into the primitive cache + sources.
template <typename T>
void launch_cells(const double *state, T *prim, T *src, const BoxDev &b,
                  const Background &bg, const Options &o, DevStatus *st,
                  cudaStream_t s);
// Face fluxes + divergence + sources -> rhs.  mdot_part (one double per
// block) receives the block sums of the accretion-rate faces when
// o.accretion_radius > 0.
template <typename T>
void launch_faces(const T *prim, const T *src, T *rhs, const BoxDev &b,
                  const Background &bg, const Options &o,
                  const double inv_dx[3], int zchunk, double *mdot_part,
                  cudaStream_t s);
// acc[0] = sum of part[0..n); acc[1] += weight * acc[0]
void launch_mdot_sum(const double *part, int64_t n, double weight,
                     double *acc, cudaStream_t s);
// update_conserved (FP64): dst = src + dt rhs, then recovery when asked.
void launch_update(double *dst, int64_t dcs, const double *src_state,
                   int64_t scs, const double *rhs, const BoxDev &b,
                   const Background &bg, const Options &o, double dt,
                   int recover, DevStatus *st, cudaStream_t s);
void launch_recover(double *state, const BoxDev &b, const Background &bg,
                    const Options &o, DevStatus *st, cudaStream_t s);
// Integrator stage fused with the post-update recovery; mode 0 RK4 stage
// `stage`, 1 Euler update, 2 SSPRK2 combine.  With prep the stage also
// prepares the next RHS (primitive cache and sources); the mixed path
// reads its con2prim start from `prim_in` (`prim` when null) either way.
// With cfl it accumulates the next max inverse dt into st->maxinv_bits.
template <typename T>
void launch_stage(int mode, const double *un, int64_t ucs, const double *us,
                  int64_t tcs, double *out, int64_t ocs, const T *k,
                  double *acc, T *prim, T *src, int prep, const BoxDev &b,
                  const Background &bg, const Options &o, int stage,
                  double dt, bool cfl, const double inv_dx[3], DevStatus *st,
                  cudaStream_t s, const T *prim_in = nullptr);
// The CFL speed in the FP64 metric and arithmetic, or (mixed) in those of
// the mixed path's fused stage.
void launch_max_inv_dt(const double *state, const BoxDev &b,
                       const Background &bg, const Options &o,
                       const double inv_dx[3], DevStatus *st, bool mixed,
                       cudaStream_t s);
void launch_residual_probe(const double *state, const BoxDev &b,
                           const Background &bg, const Options &o, int i,
                           int j, int k, double *out, cudaStream_t s);
// FP32 5-component interior array into an FP64 one with stride ocs.
void launch_widen(const float *in, int64_t n, double *out, int64_t ocs,
                  cudaStream_t s);
void launch_eval_background(int64_t n, const double *xyz,
                            const Background &bg, double *out,
                            cudaStream_t s);
void launch_eval_con2prim(int64_t n, const double *cons, const double *gUU,
                          const Options &o, double *prim, int *ok, int *iters,
                          double *resid, cudaStream_t s);
void launch_eval_arith(int64_t n, const double *a, const double *b,
                       double *out, cudaStream_t s);

// ------------------------------------------------------------ ensemble
// Many independent boxes (members) advanced by one persistent launch: each
// phase (ghost fill, face pass, stage) runs the work items of every member,
// handed out by an atomic counter, between grid-wide barriers.

// Cells per cell-wise work item (one per thread of a 16x16 block).
constexpr int kEnsItemCells = kTB * kTB;

// One member, as the persistent kernel reads it.  prim/src/k hold the
// ensemble's arithmetic type T.
struct EnsMember
{
    BoxDev b;  // the member's state box (caller's component stride)
    BoxDev sb; // the same box over the RK stage buffer (stride = volume)
    Background bg;
    Options o;
    double inv[3];
    double cfl, max_dt;
    double *state, *stage, *acc;
    void *prim, *src, *k;
    double *mdot_part;           // one partial per face tile
    double *mdot_acc;            // [Mdot of the last RHS, time integral]
    double *time;                // member time
    unsigned long long *mi_bits; // [2] max inverse dt by step parity
    DevStatus *st;
    int tiles[3];   // face tiles along x, y, z
    int has_mdot;
    int64_t nshell; // ghost shell cells
};

// Control block of a launch (zeroed by the host before each launch, except
// steps_done and need_cfl, which carry over between launches).
struct EnsControl
{
    unsigned long long ctr[3]; // work counters, by phase number mod 3
    unsigned int bar_count, bar_gen;
    int error;       // 1: a grid barrier wait ran out
    int error_phase; // phase number of that barrier
    unsigned long long steps_done;
    int need_cfl; // the first phase computes the CFL speed
    int pad_;
};

struct EnsLaunch
{
    const EnsMember *m;
    int nm;
    // per-member prefix sums of work items, [nm + 1] each
    const int64_t *off_ghost, *off_cell, *off_tile;
    EnsControl *ctl;
    int steps;
    int zchunk;
    unsigned int nblocks;
    unsigned int bar_extra; // arrivals beyond the grid a barrier waits for
    unsigned long long bar_timeout_ns;
};

// Dynamic shared memory and resident blocks per SM of the ensemble kernel.
template <typename T> size_t ensemble_smem();
template <typename T> cudaError_t ensemble_occupancy(int *blocks_per_sm);
// One persistent launch of `grid` blocks (all resident; cooperative).
template <typename T>
cudaError_t launch_ensemble(const EnsLaunch &a, int grid, cudaStream_t s);

// The operator on CCZ4-stored geometry (grhd_kernels.cu): state of 36
// components (25 CCZ4, then 11 GRHD), stride b.cs; the geometry cache holds
// gLL[6] gUU[6] lapse shift[3] over the ghosted box.
void launch_ccz4_fill(double *s, const BoxDev &b, bool conserved,
                      cudaStream_t st);
void launch_ccz4_cells(const double *s, const BoxDev &b, const Options &o,
                       double *prim, double *gc, DevStatus *st,
                       cudaStream_t stream);
void launch_ccz4_rhs(const double *s, const BoxDev &b, const Options &o,
                     const double *prim, const double *gc, double *rhs,
                     int64_t rcs, const double inv[3], DevStatus *st,
                     cudaStream_t stream);
void launch_ccz4_recover(double *s, const BoxDev &b, const Options &o,
                         DevStatus *st, cudaStream_t stream);
void launch_ccz4_max_inv_dt(const double *s, const BoxDev &b,
                            const Options &o, const double inv[3],
                            DevStatus *st, cudaStream_t stream);
void launch_ccz4_update(double *s, const double *u1, int64_t ucs,
                        const double *rhs, int64_t rcs, const BoxDev &b,
                        double dt, int mode, cudaStream_t stream);
void launch_ccz4_probe(const double *s, const BoxDev &b, const Options &o,
                       int i, int j, int k, double *out, cudaStream_t stream);

} // namespace grhd
