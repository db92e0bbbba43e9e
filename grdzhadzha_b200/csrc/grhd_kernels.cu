// grhd_kernels.cu -- sm_100a kernels of the fixed-background Valencia GRHD
// operator.
//
// The kernels are templated on the arithmetic type T of the primitive
// cache, the face fluxes, the sources and the RHS: T = double is the FP64
// path, T = float the mixed path (the conserved state, the RK accumulator
// and con2prim stay FP64 in both).
//
// One RHS evaluation is three launches:
//   fill_ghosts : physical (outflow) ghost cells of the box, as
//                 fill_conserved_outflow_boundaries_from_fixed_background
//                 (FixedBGFArrayBoxFiniteVolume.hpp:113-177), then the
//                 ghost cells' con2prim into the primitive cache;
//   cells       : interior cells: metric + con2prim into the primitive
//                 cache (recover_primitives_from_fixed_background, :33-58)
//                 and the static-metric and volume-time sources (:255-298,
//                 :616-675);
//   faces       : the face fluxes -- MUSCL slopes, floors, p2c, HLLE --
//                 with the flux divergence and the sources written straight
//                 to the RHS (:179-253, :300-363).
// Inside the RK integrators the per-cell work of the next RHS is fused into
// the stage kernel, so `cells` runs once per step.  The reference evaluates
// every face twice and every direction in a separate pass over the box;
// here the interface states never leave registers / shared memory.
#include "grhd_kernels.cuh"

#include <atomic>

namespace grhd {

namespace {

constexpr int kWhereShift = 56;

__device__ __forceinline__ void record_error(DevStatus *st, int where,
                                             int64_t order)
{
    const unsigned long long key =
        ((unsigned long long)where << kWhereShift) | (unsigned long long)order;
    atomicMin(&st->err_key, key);
}

// Resident blocks per SM the register budget is sized for: the FP32
// (mixed) kernels fit three 256-thread blocks (80 registers, small
// spills; measured 13 % faster than two), the FP64 ones two (the FP64 face
// tile's 108 KB of shared memory allows no more).
template <typename T> constexpr int kMinBlocks = sizeof(T) == 4 ? 3 : 2;

// Loads of data that a persistent launch wrote itself in an earlier phase
// (CG = true) go through L2 (ld.global.cg): the non-coherent read-only path
// (__ldg) is only valid for data left unchanged for a whole launch.
template <bool CG, typename T> __device__ __forceinline__ T rd(const T *p)
{
    return CG ? __ldcg(p) : *p;
}
template <bool CG, typename T> __device__ __forceinline__ T rdro(const T *p)
{
    return CG ? __ldcg(p) : __ldg(p);
}

template <bool CG = false>
__device__ __forceinline__ Cons load_cons(const double *s, int64_t cs,
                                          int64_t idx)
{
    Cons c;
    c.D = rd<CG>(&s[kD * cs + idx]);
    c.S[0] = rd<CG>(&s[(kS1 + 0) * cs + idx]);
    c.S[1] = rd<CG>(&s[(kS1 + 1) * cs + idx]);
    c.S[2] = rd<CG>(&s[(kS1 + 2) * cs + idx]);
    c.tau = rd<CG>(&s[kTau * cs + idx]);
    return c;
}

__device__ __forceinline__ void store_cons(double *s, int64_t cs, int64_t idx,
                                           const Cons &c)
{
    s[kD * cs + idx] = c.D;
    s[(kS1 + 0) * cs + idx] = c.S[0];
    s[(kS1 + 1) * cs + idx] = c.S[1];
    s[(kS1 + 2) * cs + idx] = c.S[2];
    s[kTau * cs + idx] = c.tau;
}

__device__ __forceinline__ void store_prim(double *s, int64_t cs, int64_t idx,
                                           const Prim &p)
{
    s[kRho * cs + idx] = p.rho;
    s[kEps * cs + idx] = p.eps;
    s[kPress * cs + idx] = p.p;
    s[(kV1 + 0) * cs + idx] = p.v[0];
    s[(kV1 + 1) * cs + idx] = p.v[1];
    s[(kV1 + 2) * cs + idx] = p.v[2];
}

template <bool CG = false>
__device__ __forceinline__ Prim load_prim(const double *s, int64_t cs,
                                          int64_t idx)
{
    Prim p;
    p.rho = rd<CG>(&s[kRho * cs + idx]);
    p.eps = rd<CG>(&s[kEps * cs + idx]);
    p.p = rd<CG>(&s[kPress * cs + idx]);
    p.v[0] = rd<CG>(&s[(kV1 + 0) * cs + idx]);
    p.v[1] = rd<CG>(&s[(kV1 + 1) * cs + idx]);
    p.v[2] = rd<CG>(&s[(kV1 + 2) * cs + idx]);
    return p;
}

__device__ __forceinline__ bool primitive_differs(const Prim &a, const Prim &b)
{
    return a.rho != b.rho || a.eps != b.eps || a.p != b.p ||
           a.v[0] != b.v[0] || a.v[1] != b.v[1] || a.v[2] != b.v[2];
}

template <typename T>
__device__ __forceinline__ void store_pv(T *prim, int64_t pcs, int64_t g,
                                         const Prim &pr)
{
    prim[0 * pcs + g] = T(pr.rho);
    prim[1 * pcs + g] = T(pr.p);
    prim[2 * pcs + g] = T(pr.v[0]);
    prim[3 * pcs + g] = T(pr.v[1]);
    prim[4 * pcs + g] = T(pr.v[2]);
}

template <typename T>
__device__ __forceinline__ void store_src(T *src, int64_t rcs, int64_t ri,
                                          const ConsT<T> &s)
{
    src[0 * rcs + ri] = s.D;
    src[1 * rcs + ri] = s.S[0];
    src[2 * rcs + ri] = s.S[1];
    src[3 * rcs + ri] = s.S[2];
    src[4 * rcs + ri] = s.tau;
}

template <typename T> __device__ __forceinline__ ConsT<T> zero_cons()
{
    ConsT<T> z;
    z.D = z.tau = z.S[0] = z.S[1] = z.S[2] = T(0);
    return z;
}

// con2prim of a cell: the reference's bracketed solve (FP64 path) or the
// warm-started FP64 solve from a nearby pressure (mixed path).
template <typename T>
__device__ __forceinline__ bool cell_con2prim(const Options &o, const Cons &c,
                                              const GeoT<T> &g, double p_guess,
                                              Prim &out)
{
    double gUU[6];
#pragma unroll
    for (int q = 0; q < 6; ++q)
        gUU[q] = double(g.gUU[q]);
    if (sizeof(T) == sizeof(double))
        return con2prim(o, c, gUU, out, nullptr, nullptr);
    return con2prim_warm(o, c, gUU, p_guess, out);
}

template <typename T>
__device__ __forceinline__ void gLL_double(const GeoT<T> &g, double out[6])
{
#pragma unroll
    for (int q = 0; q < 6; ++q)
        out[q] = double(g.gLL[q]);
}

// The metric of a cell for its con2prim, floors and p2c, widened to FP64
// for the solve: the FP64 metric, or the mixed path's, so that every
// con2prim of a cell within one path sees the same gamma (a state the
// stage recovery accepted at the velocity cap is accepted again by the
// next RHS's boundary fill and CFL speed).
template <typename T>
__device__ __forceinline__ void cell_metric_d(const Background &bg, double x,
                                              double y, double z,
                                              double gLL[6], double gUU[6])
{
    GeoT<T> g;
    metric_T<T, false>(bg, x, y, z, g, nullptr);
#pragma unroll
    for (int q = 0; q < 6; ++q)
    {
        gLL[q] = double(g.gLL[q]);
        gUU[q] = double(g.gUU[q]);
    }
}

// ------------------------------------------------------------ ghost fill

// Enumerates the shell "ghosted box minus interior box" as three slabs:
// z outside the interior; z inside, y outside; z and y inside, x outside.
__device__ __forceinline__ bool shell_cell(const BoxDev &b, int64_t t, int &i,
                                           int &j, int &k)
{
    const int64_t gx = b.gn[0], gy = b.gn[1];
    const int64_t zlo = b.lo[2] - b.glo[2];
    const int64_t nz_out = b.gn[2] - b.in[2];
    const int64_t n1 = nz_out * gx * gy;
    if (t < n1)
    {
        const int64_t kk = t / (gx * gy);
        const int64_t r = t - kk * gx * gy;
        k = (kk < zlo) ? b.glo[2] + (int)kk : b.hi[2] + 1 + (int)(kk - zlo);
        j = b.glo[1] + (int)(r / gx);
        i = b.glo[0] + (int)(r % gx);
        return true;
    }
    t -= n1;
    const int64_t ylo = b.lo[1] - b.glo[1];
    const int64_t ny_out = b.gn[1] - b.in[1];
    const int64_t n2 = (int64_t)b.in[2] * ny_out * gx;
    if (t < n2)
    {
        const int64_t kk = t / (ny_out * gx);
        const int64_t r = t - kk * ny_out * gx;
        const int64_t jj = r / gx;
        k = b.lo[2] + (int)kk;
        j = (jj < ylo) ? b.glo[1] + (int)jj : b.hi[1] + 1 + (int)(jj - ylo);
        i = b.glo[0] + (int)(r % gx);
        return true;
    }
    t -= n2;
    const int64_t xlo = b.lo[0] - b.glo[0];
    const int64_t nx_out = b.gn[0] - b.in[0];
    const int64_t n3 = (int64_t)b.in[2] * b.in[1] * nx_out;
    if (t < n3)
    {
        const int64_t kj = t / nx_out;
        const int64_t ii = t - kj * nx_out;
        k = b.lo[2] + (int)(kj / b.in[1]);
        j = b.lo[1] + (int)(kj % b.in[1]);
        i = (ii < xlo) ? b.glo[0] + (int)ii : b.hi[0] + 1 + (int)(ii - xlo);
        return true;
    }
    return false;
}

// Physical (outflow) ghost fill of the shell "ghosted box minus box"
// (fill_conserved_outflow_boundaries_from_fixed_background, :113-177),
// then, for every shell cell, the ghosted-box con2prim of the RHS into the
// primitive cache (recover_primitives_from_fixed_background, :33-58).  The
// fill itself is FP64 in both paths.  Shell cells inside the domain hold
// the owning boxes' values (after grhd_level_exchange); an excised one of
// them keeps its frozen primitives, as it does as an interior cell, so a
// level's RHS does not depend on how it is cut into boxes.
template <typename T, bool CG = false>
__device__ __forceinline__ void ghost_at(double *__restrict__ state,
                                         T *__restrict__ prim,
                                         const BoxDev &b, const Background &bg,
                                         const Options &o, DevStatus *st,
                                         int i, int j, int k)
{
    {
        const int iv[3] = {i, j, k};
        int srcc[3] = {i, j, k};
        bool ghost = false;
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            if (iv[d] < b.dlo[d])
            {
                ghost = true;
                srcc[d] = b.lo[d];
            }
            else if (iv[d] > b.dhi[d])
            {
                ghost = true;
                srcc[d] = b.hi[d];
            }
        }
        double x, y, z;
        const int64_t idx = b.gidx(i, j, k);
        cell_xyz(o, i, j, k, x, y, z);
        double tLL[6], tUU[6];
        cell_metric_d<T>(bg, x, y, z, tLL, tUU);
        Cons c;
        if (ghost)
        {
            double sx, sy, sz;
            cell_xyz(o, srcc[0], srcc[1], srcc[2], sx, sy, sz);
            double sLL[6], sUU[6];
            cell_metric_d<T>(bg, sx, sy, sz, sLL, sUU);
            const Cons sc = load_cons<CG>(state, b.cs,
                                          b.gidx(srcc[0], srcc[1], srcc[2]));
            Prim pr;
            if (!con2prim(o, sc, sUU, pr, nullptr, nullptr))
            {
                record_error(st, 1, idx);
                return;
            }
            floors(o, pr, tLL);
            store_prim(state, b.cs, idx, pr);
            c = p2c(pr, tLL);
            store_cons(state, b.cs, idx, c);
        }
        else if (excised(o, i, j, k))
        {
            // a ghost that another box of the level owns: frozen like the
            // owner's interior cell
            store_pv(prim, b.pcs, idx, load_prim<CG>(state, b.cs, idx));
            return;
        }
        else
            c = load_cons<CG>(state, b.cs, idx);
        Prim pr;
        if (!con2prim(o, c, tUU, pr, nullptr, nullptr))
        {
            record_error(st, 2, idx);
            pr.rho = pr.p = 1.0;
            pr.v[0] = pr.v[1] = pr.v[2] = 0.0;
        }
        store_pv(prim, b.pcs, idx, pr);
    }
}

template <typename T, bool CG = false>
__device__ __forceinline__ void ghost_item(double *__restrict__ state,
                                           T *__restrict__ prim,
                                           const BoxDev &b,
                                           const Background &bg,
                                           const Options &o, DevStatus *st,
                                           int64_t t)
{
    int i, j, k;
    if (shell_cell(b, t, i, j, k))
        ghost_at<T, CG>(state, prim, b, bg, o, st, i, j, k);
}

template <typename T>
__global__ void __launch_bounds__(256)
    k_fill_ghosts(double *__restrict__ state, T *__restrict__ prim, BoxDev b,
                  Background bg, Options o, DevStatus *st, int64_t nshell)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
         t < nshell; t += (int64_t)gridDim.x * blockDim.x)
        ghost_item<T>(state, prim, b, bg, o, st, t);
}

// The shell cells of the ghosted planes k0..k1 only (plane_shell_cell).
template <typename T>
__global__ void __launch_bounds__(256)
    k_fill_ghost_planes(double *__restrict__ state, T *__restrict__ prim,
                        BoxDev b, Background bg, Options o, DevStatus *st,
                        int k0, int k1, int64_t n)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        int i, j, k;
        plane_shell_cell(b, k0, k1, t, i, j, k);
        ghost_at<T>(state, prim, b, bg, o, st, i, j, k);
    }
}

// Static-metric sources (:255-298) from the floored primitives and, for
// the binary, the volume-time source (:616-675, FP64 in both paths); `pr`
// is the cell's unfloored con2prim result.
template <typename T>
__device__ __forceinline__ ConsT<T> cell_sources(const Options &o,
                                                 const Background &bg,
                                                 double x, double y, double z,
                                                 const Prim &pr, const Cons &c,
                                                 const GeoFullT<T> &f)
{
    ConsT<T> s = zero_cons<T>();
    if (o.use_src)
    {
        // floors and the atmosphere test in FP64 for both paths, so that
        // which cells count as atmosphere does not depend on the type
        double gLL[6];
        gLL_double(f.g, gLL);
        Prim fd = pr;
        floors(o, fd, gLL);
        if (!is_atmo(o, fd, o.src_atmo_factor))
            s = static_sources(convert_prim<double, T>(fd),
                               convert_cons<double, T>(c), f);
    }
    if (o.use_vol && bg.kind == 1)
    {
        const double pos[3] = {x, y, z};
        const double Up = pn_scalar(bg.m1, bg.m2, bg.soft2, bg.p1p, bg.p2p, pos);
        const double Um = pn_scalar(bg.m1, bg.m2, bg.soft2, bg.p1m, bg.p2m, pos);
        const double dl =
            __dadd_rn(pn_log_sqrt_det(__dadd_rn(1.0, 2.0 * Up)),
                      -pn_log_sqrt_det(__dadd_rn(1.0, 2.0 * Um))) /
            (2.0 * bg.fd_h);
        s.D = T(double(s.D) + (0.0 - c.D * dl));
        s.tau = T(double(s.tau) + (0.0 - c.tau * dl));
#pragma unroll
        for (int m = 0; m < 3; ++m)
            s.S[m] = T(double(s.S[m]) + (0.0 - c.S[m] * dl));
    }
    return s;
}

// ------------------------------------------------------- per-cell pass

// Interior cells: con2prim into the primitive cache (the ghosted-box
// recovery of the RHS restricted to the interior; the shell is done by
// k_fill_ghosts) and the sources into the source scratch.  Excised cells
// keep their frozen primitives and get no source.  The mixed path starts
// con2prim from the state's stored pressure.
template <typename T, bool CG = false>
__device__ __forceinline__ void cells_item(const double *__restrict__ state,
                                           T *__restrict__ prim,
                                           T *__restrict__ src,
                                           const BoxDev &b,
                                           const Background &bg,
                                           const Options &o, DevStatus *st,
                                           int64_t t)
{
    {
        const int i = b.lo[0] + (int)(t % b.in[0]);
        const int64_t r = t / b.in[0];
        const int j = b.lo[1] + (int)(r % b.in[1]);
        const int k = b.lo[2] + (int)(r / b.in[1]);
        const int64_t g = b.gidx(i, j, k);
        ConsT<T> s = zero_cons<T>();
        if (excised(o, i, j, k))
        {
            store_pv(prim, b.pcs, g, load_prim<CG>(state, b.cs, g));
            store_src(src, b.rcs, t, s);
            return;
        }
        double x, y, z;
        cell_xyz(o, i, j, k, x, y, z);
        GeoFullT<T> f;
        if (o.use_src)
            metric_T<T, true>(bg, x, y, z, f.g, &f);
        else
            metric_T<T, false>(bg, x, y, z, f.g, nullptr);
        const Cons c = load_cons<CG>(state, b.cs, g);
        Prim pr;
        if (!cell_con2prim(o, c, f.g, rd<CG>(&state[kPress * b.cs + g]), pr))
        {
            record_error(st, 2, g);
            pr.rho = pr.p = 1.0;
            pr.v[0] = pr.v[1] = pr.v[2] = 0.0;
            pr.eps = 1.0;
        }
        else
            s = cell_sources<T>(o, bg, x, y, z, pr, c, f);
        store_pv(prim, b.pcs, g, pr);
        store_src(src, b.rcs, t, s);
    }
}

template <typename T>
__global__ void __launch_bounds__(256, kMinBlocks<T>)
    k_cells(const double *__restrict__ state, T *__restrict__ prim,
            T *__restrict__ src, BoxDev b, Background bg, Options o,
            DevStatus *st)
{
    const int64_t n = b.ivol();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        cells_item<T>(state, prim, src, b, bg, o, st, t);
}

// ----------------------------------------------------------- face pass

template <typename T>
__device__ __forceinline__ void geo_store(T *g, int n, int cell,
                                          const GeoT<T> &v)
{
#pragma unroll
    for (int s = 0; s < 6; ++s)
    {
        g[s * n + cell] = v.gLL[s];
        g[(6 + s) * n + cell] = v.gUU[s];
    }
    g[12 * n + cell] = v.lapse;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        g[(13 + i) * n + cell] = v.shift[i];
}

template <typename T>
__device__ __forceinline__ void geo_load(const T *g, int n, int cell,
                                         GeoT<T> &v)
{
#pragma unroll
    for (int s = 0; s < 6; ++s)
    {
        v.gLL[s] = g[s * n + cell];
        v.gUU[s] = g[(6 + s) * n + cell];
    }
    v.lapse = g[12 * n + cell];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        v.shift[i] = g[(13 + i) * n + cell];
}

template <typename T>
__device__ __forceinline__ void geo_avg_smem(const T *g, int n, int ca, int cb,
                                             GeoT<T> &v)
{
#pragma unroll
    for (int s = 0; s < 6; ++s)
    {
        v.gLL[s] = T(0.5) * (g[s * n + ca] + g[s * n + cb]);
        v.gUU[s] = T(0.5) * (g[(6 + s) * n + ca] + g[(6 + s) * n + cb]);
    }
    v.lapse = T(0.5) * (g[12 * n + ca] + g[12 * n + cb]);
#pragma unroll
    for (int i = 0; i < 3; ++i)
        v.shift[i] = T(0.5) * (g[(13 + i) * n + ca] + g[(13 + i) * n + cb]);
}

template <typename T, bool CG = false>
__device__ __forceinline__ PVT<T> load_pv_global(const T *__restrict__ prim,
                                                 int64_t pcs, int64_t idx)
{
    PVT<T> p;
#pragma unroll
    for (int c = 0; c < 5; ++c)
        p.q[c] = rdro<CG>(&prim[c * pcs + idx]);
    return p;
}

template <typename T>
__device__ __forceinline__ PVT<T> load_pv_smem(const T *P, int cell)
{
    constexpr int n = kPW * kPW;
    PVT<T> p;
#pragma unroll
    for (int c = 0; c < 5; ++c)
        p.q[c] = P[c * n + cell];
    return p;
}

// Asynchronous global -> shared copy of one element (cp.async, 4 or 8
// bytes, cached in L1) and the wait for all of this thread's copies.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d),
                     "l"(src)
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d),
                     "l"(src)
                     : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// The primitive cross tile of a z march at plane k (clamped to the
// ghosted box): synchronous loads, or (ASYNC) cp.async copies completed by
// cp_async_wait_all before the next barrier.
template <typename T, bool CG, bool ASYNC>
__device__ __forceinline__ void load_p_tile(T *P, const T *__restrict__ prim,
                                            const BoxDev &b, int i0, int j0,
                                            int k, int tid)
{
    constexpr int nP = kPW * kPW;
    for (int idx = tid; idx < nP; idx += kTB * kTB)
    {
        const int u = idx % kPW, v = idx / kPW;
        if ((u < 2 || u > kPW - 3) && (v < 2 || v > kPW - 3))
            continue;
        const int gi = min(max(i0 - 2 + u, b.glo[0]), b.ghi[0]);
        const int gj = min(max(j0 - 2 + v, b.glo[1]), b.ghi[1]);
        const int64_t g = b.gidx(gi, gj, k);
#pragma unroll
        for (int c = 0; c < 5; ++c)
        {
            if constexpr (ASYNC)
                cp_async_elem(&P[c * nP + idx], &prim[c * b.pcs + g]);
            else
                P[c * nP + idx] = rdro<CG>(&prim[c * b.pcs + g]);
        }
    }
}

// Geometry of the cross-shaped (x,y) neighbourhood of a tile at plane kk.
template <typename T, int BGK = -1>
__device__ __forceinline__ void tile_geometry(T *G, const Background &bg,
                                              const Options &o, int i0,
                                              int j0, int kk, int tid)
{
    constexpr int n = kGW * kGW;
    for (int idx = tid; idx < n; idx += kTB * kTB)
    {
        const int u = idx % kGW, v = idx / kGW;
        if ((u == 0 || u == kGW - 1) && (v == 0 || v == kGW - 1))
            continue;
        double x, y, z;
        cell_xyz(o, i0 - 1 + u, j0 - 1 + v, kk, x, y, z);
        GeoT<T> g;
        metric_T<T, false, BGK>(bg, x, y, z, g, nullptr);
        geo_store(G, n, idx, g);
    }
}

// Rest-mass flux of one face through the voxelised sphere r < R (new):
// the face between cells L and R (R = L + e_d) lies on the sphere's
// boundary when exactly one of them is inside; the outward flux is
// +sqrt(gamma_face) F_D dA when L is inside, and Mdot counts the inward
// flux.
template <typename T>
__device__ __forceinline__ double mdot_face(const Options &o, int il, int jl,
                                            int kl, int d, const GeoT<T> &gf,
                                            T FD)
{
    double x, y, z;
    cell_xyz(o, il, jl, kl, x, y, z);
    const bool in_l = sqrt(x * x + y * y + z * z) < o.accretion_radius;
    cell_xyz(o, il + (d == 0), jl + (d == 1), kl + (d == 2), x, y, z);
    const bool in_r = sqrt(x * x + y * y + z * z) < o.accretion_radius;
    if (in_l == in_r)
        return 0.0;
    double g[6];
    gLL_double(gf, g);
    const double det = g[0] * (g[3] * g[5] - g[4] * g[4]) -
                       g[1] * (g[1] * g[5] - g[4] * g[2]) +
                       g[2] * (g[1] * g[4] - g[3] * g[2]);
    return (in_l ? -1.0 : 1.0) * sqrt(det) * double(FD) * (o.dx * o.dx);
}

// Block sum of `v` into part[block] (fixed order within the block).
__device__ __forceinline__ void block_partial(double v, double *scratch,
                                              double *part, int tid, int nt,
                                              int64_t block)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, off);
    if ((tid & 31) == 0)
        scratch[tid >> 5] = v;
    __syncthreads();
    if (tid == 0)
    {
        double sum = 0.0;
        for (int w = 0; w < nt / 32; ++w)
            sum += scratch[w];
        part[block] = sum;
    }
}

// 16x16 threads own a 15x15 (x,y) cell tile and march along z over a chunk
// of planes.  Per plane: the primitive cross tile (2-cell halo) and the
// geometry cross tile (1-cell halo) in shared memory, geometry double
// buffered by plane; x and y faces from shared memory (each tile also
// evaluates its two boundary faces per row), the z face from a 4-plane
// register window (each z face once); divergence + sources to the RHS.
// One tile (bx, by, bz) of the face pass; 16x16 threads, `smem_raw` holds
// faces_smem<T>() bytes; the tile's accretion sum goes to mdot_part[part].
template <typename T, bool MDOT, bool CG = false, int BGK = -1>
__device__ __forceinline__ void
faces_tile(const T *__restrict__ prim, const T *__restrict__ src,
           T *__restrict__ rhs, const BoxDev &b, const Background &bg,
           const Options &o, double idx0_, double idx1_, double idx2_,
           int zchunk, int bx, int by, int bz, unsigned char *smem_raw,
           double *__restrict__ mdot_part, int64_t part)
{
    T *smem = reinterpret_cast<T *>(smem_raw);
    constexpr int nP = kPW * kPW;
    constexpr int nG = kGW * kGW;
    constexpr int nFx = kTB * kTC; // x faces: a in [0,16), b in [0,15)
    T *P = smem;                       // [5][nP]
    T *Gb = P + 5 * nP;                // [2][16][nG]
    T *Fx = Gb + 2 * kGeoFields * nG;  // [5][nFx]
    T *Fy = Fx + 5 * nFx;              // [5][nFx]
    const T idx0 = T(idx0_), idx1 = T(idx1_), idx2 = T(idx2_);

    const int a = threadIdx.x, bb = threadIdx.y;
    const int tid = bb * kTB + a;
    const int i0 = b.lo[0] + bx * kTC;
    const int j0 = b.lo[1] + by * kTC;
    const int k0 = b.lo[2] + bz * zchunk;
    const int k1 = min(k0 + zchunk - 1, b.hi[2]);
    const int ci = i0 + a, cj = j0 + bb; // this thread's cell column
    const bool col_ok = a < kTC && bb < kTC && ci <= b.hi[0] && cj <= b.hi[1];
    const int ci_c = min(ci, b.hi[0]), cj_c = min(cj, b.hi[1]);

    // The z march starts two planes below k0: plane k0-2 only computes
    // the tile geometry of plane k0-1, plane k0-1 only the z face below
    // k0.  Every plane's geometry and every z face thus come from the same
    // code as in the rest of the march, so the face below k0 equals the
    // block below's upper face bit for bit: the RHS does not depend on
    // where the z blocks start.  w0..w3 is this column's window
    // P(k-1 .. k+2) of the z face above plane k.
    PVT<T> w0, w1, w2, w3;
    ConsT<T> Flo = zero_cons<T>();
    double macc = 0.0;
    w0 = load_pv_global<T, CG>(prim, b.pcs, b.gidx(ci_c, cj_c, k0 - 2));
    w1 = load_pv_global<T, CG>(prim, b.pcs, b.gidx(ci_c, cj_c, k0 - 1));
    w2 = load_pv_global<T, CG>(prim, b.pcs, b.gidx(ci_c, cj_c, k0));

    int cur = 0;
#pragma unroll 1
    for (int k = k0 - 2; k <= k1; ++k)
    {
        T *Gc = Gb + cur * kGeoFields * nG;
        T *Gn = Gb + (cur ^ 1) * kGeoFields * nG;
        const bool zface = k >= k0 - 1; // the z face above plane k
        const bool cells = k >= k0;     // plane k's x/y faces and RHS
        if (zface)
            w3 = load_pv_global<T, CG>(prim, b.pcs, b.gidx(ci_c, cj_c, k + 2));
        // primitive cross tile at plane k: issued after the previous
        // plane's faces (asynchronous copies, overlapping that plane's
        // output and this plane's geometry), or loaded here (the ensemble's
        // coherent loads)
        if (cells && CG)
            load_p_tile<T, CG, false>(P, prim, b, i0, j0, k, tid);
        tile_geometry<T, BGK>(Gn, bg, o, i0, j0, k + 1, tid);
        if (cells && !CG)
            cp_async_wait_all();
        __syncthreads();

        // x face between cells (i0+a-1, i0+a) in row j0+bb
        if (cells && bb < kTC && cj <= b.hi[1] && i0 + a - 1 <= b.hi[0])
        {
            const int row = (bb + 2) * kPW;
            GeoT<T> gf;
            geo_avg_smem(Gc, nG, (bb + 1) * kGW + a, (bb + 1) * kGW + a + 1, gf);
            const ConsT<T> f = face_flux(o, load_pv_smem(P, row + a),
                                         load_pv_smem(P, row + a + 1),
                                         load_pv_smem(P, row + a + 2),
                                         load_pv_smem(P, row + a + 3), gf, 0);
            const int fi = bb * kTB + a;
            if (MDOT && a < kTC && i0 + a <= b.hi[0])
                macc += mdot_face(o, i0 + a - 1, cj, k, 0, gf, f.D);
            Fx[0 * nFx + fi] = f.D;
            Fx[1 * nFx + fi] = f.S[0];
            Fx[2 * nFx + fi] = f.S[1];
            Fx[3 * nFx + fi] = f.S[2];
            Fx[4 * nFx + fi] = f.tau;
        }
        // y face between rows (j0+bb-1, j0+bb) in column i0+a
        if (cells && a < kTC && ci <= b.hi[0] && j0 + bb - 1 <= b.hi[1])
        {
            GeoT<T> gf;
            geo_avg_smem(Gc, nG, bb * kGW + a + 1, (bb + 1) * kGW + a + 1, gf);
            const int col = a + 2;
            const ConsT<T> f = face_flux(o, load_pv_smem(P, bb * kPW + col),
                                         load_pv_smem(P, (bb + 1) * kPW + col),
                                         load_pv_smem(P, (bb + 2) * kPW + col),
                                         load_pv_smem(P, (bb + 3) * kPW + col),
                                         gf, 1);
            const int fi = a * kTB + bb;
            if (MDOT && bb < kTC && j0 + bb <= b.hi[1])
                macc += mdot_face(o, ci, j0 + bb - 1, k, 1, gf, f.D);
            Fy[0 * nFx + fi] = f.D;
            Fy[1 * nFx + fi] = f.S[0];
            Fy[2 * nFx + fi] = f.S[1];
            Fy[3 * nFx + fi] = f.S[2];
            Fy[4 * nFx + fi] = f.tau;
        }
        // z face at k+1/2 for this column
        ConsT<T> Fhi = zero_cons<T>();
        if (zface && col_ok)
        {
            GeoT<T> gf, gA, gB;
            const int cell = (bb + 1) * kGW + a + 1;
            geo_load(Gc, nG, cell, gA);
            geo_load(Gn, nG, cell, gB);
            average_geo(gA, gB, gf);
            Fhi = face_flux(o, w0, w1, w2, w3, gf, 2);
            // a box counts the sphere faces whose upper cell it holds, in
            // every direction, so the boxes of a level count each once
            if (MDOT && (cells ? k < b.hi[2] : k0 == b.lo[2]))
                macc += mdot_face(o, ci, cj, k, 2, gf, Fhi.D);
        }
        __syncthreads();
        // the x/y faces have read plane k's tile: fetch plane k+1's
        if (!CG && k + 1 >= k0 && k + 1 <= k1)
            load_p_tile<T, CG, true>(P, prim, b, i0, j0, k + 1, tid);

        if (cells && col_ok)
        {
            const int fxl = bb * kTB + a, fxh = bb * kTB + a + 1;
            const int fyl = a * kTB + bb, fyh = a * kTB + bb + 1;
            const int64_t ri = b.iidx(ci, cj, k);
            T out[5];
            const T fl[5] = {Flo.D, Flo.S[0], Flo.S[1], Flo.S[2], Flo.tau};
            const T fh[5] = {Fhi.D, Fhi.S[0], Fhi.S[1], Fhi.S[2], Fhi.tau};
#pragma unroll
            for (int c = 0; c < 5; ++c)
            {
                const T rx = -idx0 * (Fx[c * nFx + fxh] - Fx[c * nFx + fxl]);
                const T ry = -idx1 * (Fy[c * nFx + fyh] - Fy[c * nFx + fyl]);
                const T rz = -idx2 * (fh[c] - fl[c]);
                out[c] = ((rx + ry) + rz) + rdro<CG>(&src[c * b.rcs + ri]);
            }
            if (excised(o, ci, cj, k))
            {
#pragma unroll
                for (int c = 0; c < 5; ++c)
                    out[c] = T(0);
            }
#pragma unroll
            for (int c = 0; c < 5; ++c)
                rhs[c * b.rcs + ri] = out[c];
        }
        Flo = Fhi;
        if (zface)
        {
            w0 = w1;
            w1 = w2;
            w2 = w3;
        }
        cur ^= 1;
        __syncthreads();
    }
    if (MDOT)
        block_partial(macc, reinterpret_cast<double *>(smem_raw), mdot_part,
                      tid, kTB * kTB, part);
}

template <typename T, bool MDOT, int BGK>
__global__ void __launch_bounds__(kTB *kTB, kMinBlocks<T>)
    k_faces(const T *__restrict__ prim, const T *__restrict__ src,
            T *__restrict__ rhs, BoxDev b, Background bg, Options o,
            double idx0_, double idx1_, double idx2_, int zchunk,
            double *__restrict__ mdot_part)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    faces_tile<T, MDOT, false, BGK>(prim, src, rhs, b, bg, o, idx0_, idx1_,
                                    idx2_, zchunk,
                        blockIdx.x, blockIdx.y, blockIdx.z, smem_raw,
                        mdot_part,
                        blockIdx.x + (int64_t)gridDim.x *
                                         (blockIdx.y + (int64_t)gridDim.y *
                                                           blockIdx.z));
}

// Mdot of one RHS evaluation: the block partials summed in a fixed order;
// acc[0] = Mdot, acc[1] += weight * Mdot (the time integral).
__global__ void k_mdot_sum(const double *__restrict__ part, int64_t n,
                           double weight, double *acc)
{
    __shared__ double w[32];
    double v = 0.0;
    for (int64_t q = threadIdx.x; q < n; q += blockDim.x)
        v += part[q];
    block_partial(v, w, w + 8, threadIdx.x, blockDim.x, 0);
    if (threadIdx.x == 0)
    {
        acc[0] = w[8];
        acc[1] += weight * w[8];
    }
}

// ---------------------------------------------- post-update recovery

// recover_primitives_and_apply_atmosphere_from_fixed_background for one
// cell (FixedBGFArrayBoxFiniteVolume.hpp:60-110); c is the updated
// conserved state.  Writes prims (and reset conserved) to `out`.
__device__ __forceinline__ void recover_cell(const Options &o, const Geo &g,
                                             Cons c, double *out, int64_t cs,
                                             int64_t idx,
                                             unsigned long long cnt[4])
{
    Prim pr;
    const bool ok = con2prim(o, c, g.gUU, pr, nullptr, nullptr);
    bool reset = !ok;
    cnt[0] += 1;
    if (ok)
    {
        Prim fl = pr;
        floors(o, fl, g.gLL);
        reset = primitive_differs(pr, fl);
        if (reset)
            cnt[2] += 1;
        pr = fl;
    }
    else
    {
        cnt[1] += 1;
        pr = atmosphere(o);
    }
    store_prim(out, cs, idx, pr);
    if (reset)
    {
        cnt[3] += 1;
        c = p2c(pr, g.gLL);
    }
    store_cons(out, cs, idx, c);
}

// Lane of the calling thread in its warp (blocks may be 2-D).
__device__ __forceinline__ int lane_id()
{
    return (int)((threadIdx.x + blockDim.x * threadIdx.y) & 31u);
}

__device__ __forceinline__ void flush_counts(DevStatus *st,
                                             unsigned long long cnt[4])
{
#pragma unroll
    for (int q = 0; q < 4; ++q)
    {
        unsigned long long v = cnt[q];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane_id() == 0 && v)
            atomicAdd(&st->counts[q], v);
    }
}

__device__ __forceinline__ void interior_cell(const BoxDev &b, int64_t t,
                                              int &i, int &j, int &k)
{
    i = b.lo[0] + (int)(t % b.in[0]);
    const int64_t r = t / b.in[0];
    j = b.lo[1] + (int)(r % b.in[1]);
    k = b.lo[2] + (int)(r / b.in[1]);
}

// update_conserved: dst = src + dt * rhs on the interior
// (add_scaled_conserved_rhs, FArrayBoxFiniteVolume.hpp:927-940), then the
// post-update recovery when `recover` is set.
__global__ void __launch_bounds__(256)
    k_update(double *dst, int64_t dcs, const double *srcs, int64_t scs,
             const double *__restrict__ rhs, BoxDev b, Background bg,
             Options o, double dt, int recover, DevStatus *st)
{
    unsigned long long cnt[4] = {0, 0, 0, 0};
    const int64_t n = b.ivol();
    const int64_t n_pad = (n + blockDim.x - 1) / blockDim.x * blockDim.x;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_pad;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        if (t < n)
        {
            int i, j, k;
            interior_cell(b, t, i, j, k);
            const int64_t g = b.gidx(i, j, k);
            if (excised(o, i, j, k))
            {
                if (dst != srcs)
                    for (int c = 0; c < kStateComps; ++c)
                        dst[c * dcs + g] = srcs[c * scs + g];
            }
            else
            {
                Cons c = load_cons(srcs, scs, g);
                c.D += dt * rhs[0 * b.rcs + t];
                c.tau += dt * rhs[4 * b.rcs + t];
                c.S[0] += dt * rhs[1 * b.rcs + t];
                c.S[1] += dt * rhs[2 * b.rcs + t];
                c.S[2] += dt * rhs[3 * b.rcs + t];
                if (recover)
                {
                    double x, y, z;
                    cell_xyz(o, i, j, k, x, y, z);
                    Geo geo;
                    background_metric<false>(bg, x, y, z, geo, nullptr);
                    recover_cell(o, geo, c, dst, dcs, g, cnt);
                }
                else
                {
                    store_cons(dst, dcs, g, c);
                    if (dst != srcs)
                        store_prim(dst, dcs, g, load_prim(srcs, scs, g));
                }
            }
        }
        flush_counts(st, cnt);
        cnt[0] = cnt[1] = cnt[2] = cnt[3] = 0;
    }
}

__global__ void __launch_bounds__(256)
    k_recover(double *__restrict__ state, BoxDev b, Background bg, Options o,
              DevStatus *st)
{
    unsigned long long cnt[4] = {0, 0, 0, 0};
    const int64_t n = b.ivol();
    const int64_t n_pad = (n + blockDim.x - 1) / blockDim.x * blockDim.x;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_pad;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        if (t < n)
        {
            int i, j, k;
            interior_cell(b, t, i, j, k);
            if (!excised(o, i, j, k))
            {
                const int64_t g = b.gidx(i, j, k);
                double x, y, z;
                cell_xyz(o, i, j, k, x, y, z);
                Geo geo;
                background_metric<false>(bg, x, y, z, geo, nullptr);
                recover_cell(o, geo, load_cons(state, b.cs, g), state, b.cs,
                             g, cnt);
            }
        }
        flush_counts(st, cnt);
        cnt[0] = cnt[1] = cnt[2] = cnt[3] = 0;
    }
}

// Characteristic-speed CFL contribution of one cell, sum_d max|lambda|/dx_d
// (compute_max_inverse_dt_from_fixed_background, :398-409) for floored
// primitives that are not atmosphere.
template <typename T>
__device__ __forceinline__ double cell_inverse_dt(const Options &o,
                                                  const PrimT<T> &fp,
                                                  const GeoT<T> &g,
                                                  const double inv[3])
{
    double cell = 0.0;
    if (!is_atmo(o, fp, 1.0 + 1.0e-12))
    {
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            T lo, hi;
            char_speeds(o, fp, g, d, lo, hi);
            cell += double(max_(abs_(lo), abs_(hi))) * inv[d];
        }
    }
    return cell;
}

// The CFL speed of a cell from its FP64 con2prim result: floors, the
// atmosphere test and the characteristic speeds in FP64 for both paths
// (the mixed path's metric widened), so that the step size does not hinge
// on whether a near-floor cell rounds to the floor in FP32.
template <typename T>
__device__ __forceinline__ double cfl_speed(const Options &o, const Prim &pr,
                                            const GeoT<T> &g,
                                            const double inv[3])
{
    Geo gd;
#pragma unroll
    for (int q = 0; q < 6; ++q)
    {
        gd.gLL[q] = double(g.gLL[q]);
        gd.gUU[q] = double(g.gUU[q]);
    }
    gd.lapse = double(g.lapse);
#pragma unroll
    for (int q = 0; q < 3; ++q)
        gd.shift[q] = double(g.shift[q]);
    Prim fp = pr;
    floors(o, fp, gd.gLL);
    return cell_inverse_dt(o, fp, gd, inv);
}

__device__ __forceinline__ void flush_max_to(unsigned long long *bits,
                                             double v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
    if (lane_id() == 0 && v > 0.0)
        atomicMax(bits, (unsigned long long)__double_as_longlong(v));
}

__device__ __forceinline__ void flush_max(DevStatus *st, double v)
{
    flush_max_to(&st->maxinv_bits, v);
}

// One stage of an integrator fused with the post-update recovery
// (update_conserved / recover_primitives_and_apply_atmosphere,
// FixedBGFArrayBoxFiniteVolume.hpp:60-110, 522-533) and, optionally, with
// the per-cell work of the next RHS evaluation and of the next CFL speed,
// which both start from con2prim of the state this stage writes:
//   * prep: the next RHS's con2prim (unfloored, :33-58) into the primitive
//     cache and its sources (:255-298, :616-675) into the source scratch;
//   * cfl : the next compute_max_inverse_dt (:364-412) as a device max.
// For a cell whose conserved variables were reset, the next con2prim runs
// on the reset state, as the reference's next call would.
// Modes: 0 RK4 stage `stage` (new): stages 0..2 out = U^n + c dt k with
// acc = k1 (+ 2 k2 + 2 k3), stage 3 out = U^n + dt/6 (acc + k4);
// 1 Euler update out = U^n + dt k (advance_ssprk2 stage, :578);
// 2 SSPRK2 combine out = (U^n + U^1 + dt k)/2 (FArrayBoxFiniteVolume.hpp:
// 942-969).  The stage input k, the primitive cache and the sources are of
// type T; U, the accumulator and con2prim are FP64.  The mixed path starts
// con2prim from the primitive cache's pressure of the same cell.
template <int MODE, typename T, bool CG = false, int BGK = -1>
__device__ __forceinline__ void
stage_item(const double *un, int64_t ucs, const double *us, int64_t tcs,
           double *out, int64_t ocs, const T *__restrict__ kv,
           double *__restrict__ acc, T *__restrict__ prim,
           T *__restrict__ src, const BoxDev &b, const Background &bg,
           const Options &o, int stage, double dt, bool prep, bool store_p,
           bool cfl, const double inv[3], DevStatus *st, int64_t t,
           unsigned long long cnt[4], double &cell_inv,
           const T *__restrict__ prim_in = nullptr)
{
    const double cst = (stage == 2) ? dt : 0.5 * dt;
    const double dt6 = dt / 6.0;
    const bool mixed = sizeof(T) != sizeof(double);
    int i, j, k;
    interior_cell(b, t, i, j, k);
    const int64_t g = b.gidx(i, j, k);
    if (excised(o, i, j, k))
    {
        if (out != un)
            for (int c = 0; c < kStateComps; ++c)
                out[c * ocs + g] = rd<CG>(&un[c * ucs + g]);
        if (prep)
        {
            store_pv(prim, b.pcs, g, load_prim<CG>(un, ucs, g));
            store_src(src, b.rcs, t, zero_cons<T>());
        }
    }
    else
    {
        const int comp_of[5] = {kD, kS1, kS1 + 1, kS1 + 2, kTau};
        double u[5];
#pragma unroll
        for (int c = 0; c < 5; ++c)
        {
            const double kk = double(rd<CG>(&kv[c * b.rcs + t]));
            const double u0 = rd<CG>(&un[comp_of[c] * ucs + g]);
            if (MODE == 0)
            {
                double a = (stage == 0) ? kk : rd<CG>(&acc[c * b.rcs + t]);
                if (stage == 1 || stage == 2)
                    a = a + 2.0 * kk;
                if (stage < 3)
                {
                    acc[c * b.rcs + t] = a;
                    u[c] = u0 + cst * kk;
                }
                else
                    u[c] = u0 + dt6 * (a + kk);
            }
            else if (MODE == 1)
                u[c] = u0 + dt * kk;
            else
                u[c] = 0.5 * (u0 + rd<CG>(&us[comp_of[c] * tcs + g]) + dt * kk);
        }
        Cons c;
        c.D = u[0];
        c.S[0] = u[1];
        c.S[1] = u[2];
        c.S[2] = u[3];
        c.tau = u[4];
        double x, y, z;
        cell_xyz(o, i, j, k, x, y, z);
        GeoFullT<T> f;
        if (prep && o.use_src)
            metric_T<T, true, BGK>(bg, x, y, z, f.g, &f);
        else
            metric_T<T, false, BGK>(bg, x, y, z, f.g, nullptr);
        double gLL[6];
        gLL_double(f.g, gLL);
        const T *pg = prim_in ? prim_in : prim;
        const double p_guess =
            (mixed && pg) ? double(rd<CG>(&pg[1 * b.pcs + g])) : 0.0;
        // recovery with atmosphere (:60-110)
        Prim pr;
        const bool ok = cell_con2prim(o, c, f.g, p_guess, pr);
        bool reset = !ok;
        Prim stored;
        cnt[0] += 1;
        if (ok)
        {
            stored = pr;
            floors(o, stored, gLL);
            reset = primitive_differs(pr, stored);
            if (reset)
                cnt[2] += 1;
        }
        else
        {
            cnt[1] += 1;
            stored = atmosphere(o);
        }
        if (reset)
        {
            cnt[3] += 1;
            c = p2c(stored, gLL);
        }
        // the RK stage buffer (prep) carries conserved variables
        // only: its primitive components are never read
        if (store_p)
            store_prim(out, ocs, g, stored);
        store_cons(out, ocs, g, c);
        if (prep || cfl)
        {
            // con2prim of the state just written (unchanged cells:
            // the same solve on the same input gives pr again).  The mixed
            // path takes the primitives of a cell reset to the atmosphere
            // or to the density / pressure floors as they are: con2prim of
            // their p2c returns them to within its residual tolerance, far
            // below the FP32 rounding of the primitive cache.  The FP64
            // path re-solves, as the reference's next con2prim does.
            Prim pn = pr;
            bool okn = ok;
            if (reset)
            {
                if (mixed && (!ok || (stored.v[0] == pr.v[0] &&
                                      stored.v[1] == pr.v[1] &&
                                      stored.v[2] == pr.v[2])))
                {
                    pn = stored;
                    okn = true;
                }
                else
                    okn = cell_con2prim(o, c, f.g, stored.p, pn);
            }
            if (!okn)
            {
                record_error(st, cfl && !prep ? 4 : 2,
                             cfl && !prep ? b.t0 + t : g);
                pn.rho = pn.p = 1.0;
                pn.v[0] = pn.v[1] = pn.v[2] = 0.0;
                pn.eps = 1.0;
            }
            if (prep)
            {
                store_pv(prim, b.pcs, g, pn);
                ConsT<T> s = zero_cons<T>();
                if (okn)
                    s = cell_sources<T>(o, bg, x, y, z, pn, c, f);
                store_src(src, b.rcs, t, s);
            }
            if (cfl && okn)
                cell_inv = cfl_speed<T>(o, pn, f.g, inv);
        }
    }
}

template <int MODE, typename T, int BGK>
__global__ void __launch_bounds__(256, kMinBlocks<T>)
    k_stage(const double *un, int64_t ucs, const double *us, int64_t tcs,
            double *out, int64_t ocs, const T *__restrict__ kv,
            double *__restrict__ acc, T *__restrict__ prim,
            T *__restrict__ src, BoxDev b, Background bg, Options o,
            int stage, double dt, int prep_flag, int cfl, double i0,
            double i1, double i2, DevStatus *st, const T *__restrict__ prim_in)
{
    unsigned long long cnt[4] = {0, 0, 0, 0};
    const int64_t n = b.ivol();
    const int64_t n_pad = (n + blockDim.x - 1) / blockDim.x * blockDim.x;
    const double inv[3] = {i0, i1, i2};
    // prep_flag bit 0: the next RHS's per-cell pass; bit 1: the output
    // keeps its primitives even so (the last RK4 stage of a multi-step call)
    const bool prep = (prep_flag & 1) && prim != nullptr;
    const bool store_p = !prep || (prep_flag & 2);
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_pad;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        double cell_inv = 0.0;
        if (t < n)
            stage_item<MODE, T, false, BGK>(un, ucs, us, tcs, out, ocs, kv, acc,
                                            prim, src,
                                b, bg, o, stage, dt, prep, store_p, cfl != 0,
                                inv, st, t, cnt, cell_inv, prim_in);
        flush_counts(st, cnt);
        cnt[0] = cnt[1] = cnt[2] = cnt[3] = 0;
        if (cfl)
            flush_max(st, cell_inv);
    }
}

// compute_max_inverse_dt_from_fixed_background (:364-412): per cell
// con2prim + floors, skip atmosphere, sum_d max|lambda| / dx_d; block max by
// warp shuffles, one atomicMax per warp on the bit pattern.
// One cell of the CFL speed in the metric and arithmetic of type T (the
// FP64 path, or the mixed path as the fused stage computes it).
template <typename T, bool CG = false>
__device__ __forceinline__ double cfl_item(const double *__restrict__ state,
                                           const BoxDev &b,
                                           const Background &bg,
                                           const Options &o,
                                           const double inv[3], DevStatus *st,
                                           int64_t t)
{
    double cell = 0.0;
    int i, j, k;
    interior_cell(b, t, i, j, k);
    if (!excised(o, i, j, k))
    {
        double x, y, z;
        cell_xyz(o, i, j, k, x, y, z);
        GeoT<T> geo;
        metric_T<T, false>(bg, x, y, z, geo, nullptr);
        double gUU[6];
#pragma unroll
        for (int q = 0; q < 6; ++q)
            gUU[q] = double(geo.gUU[q]);
        Prim pr;
        if (!con2prim(o, load_cons<CG>(state, b.cs, b.gidx(i, j, k)), gUU, pr,
                      nullptr, nullptr))
            record_error(st, 4, b.t0 + t);
        else
            cell = cfl_speed<T>(o, pr, geo, inv);
    }
    return cell;
}

template <typename T>
__global__ void __launch_bounds__(256)
    k_max_inv_dt(const double *__restrict__ state, BoxDev b, Background bg,
                 Options o, double i0, double i1, double i2, DevStatus *st)
{
    const int64_t n = b.ivol();
    const int64_t n_pad = (n + blockDim.x - 1) / blockDim.x * blockDim.x;
    const double inv[3] = {i0, i1, i2};
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_pad;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        double cell = 0.0;
        if (t < n)
            cell = cfl_item<T>(state, b, bg, o, inv, st, t);
        flush_max(st, cell);
    }
}

// Residual of the failing con2prim at one cell (error reporting only).
__global__ void k_residual_probe(const double *__restrict__ state, BoxDev b,
                                 Background bg, Options o, int i, int j,
                                 int k, double *out)
{
    double x, y, z;
    cell_xyz(o, i, j, k, x, y, z);
    Geo g;
    background_metric<false>(bg, x, y, z, g, nullptr);
    Prim pr;
    double res = 0.0;
    con2prim(o, load_cons(state, b.cs, b.gidx(i, j, k)), g.gUU, pr, nullptr,
             &res);
    *out = res;
}

// float RHS of the mixed path into the caller's FP64 array
__global__ void k_widen(const float *__restrict__ in, int64_t n, double *out,
                        int64_t ocs)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
         t < 5 * n; t += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t c = t / n, r = t - c * n;
        out[c * ocs + r] = double(in[t]);
    }
}

__global__ void k_eval_background(int64_t n, const double *__restrict__ xyz,
                                  Background bg, double *__restrict__ out)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    GeoFull f;
    background_metric<true>(bg, xyz[3 * t], xyz[3 * t + 1], xyz[3 * t + 2],
                            f.g, &f);
    double *o = out + 64 * t;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
        {
            o[3 * i + j] = f.g.gLL[sym(i, j)];
            o[9 + 3 * i + j] = f.K[sym(i, j)];
        }
    double K = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            K += f.g.gUU[sym(i, j)] * f.K[sym(i, j)];
    o[18] = K;
    o[19] = f.g.lapse;
    for (int i = 0; i < 3; ++i)
        o[20 + i] = f.g.shift[i];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                o[23 + 9 * i + 3 * j + k] = f.dgamma[k][sym(i, j)];
    for (int i = 0; i < 3; ++i)
        o[50 + i] = f.dlapse[i];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            o[53 + 3 * i + j] = f.dshift[i][j];
    o[62] = 0.0;
    o[63] = 0.0;
}

__global__ void k_eval_con2prim(int64_t n, const double *__restrict__ cons,
                                const double *__restrict__ gUU9, Options o,
                                double *__restrict__ prim, int *ok,
                                int *iters, double *resid)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    Cons c;
    c.D = cons[5 * t];
    c.S[0] = cons[5 * t + 1];
    c.S[1] = cons[5 * t + 2];
    c.S[2] = cons[5 * t + 3];
    c.tau = cons[5 * t + 4];
    double g[6];
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j)
            g[sym(i, j)] = gUU9[9 * t + 3 * i + j];
    Prim pr;
    pr.rho = pr.eps = pr.p = pr.v[0] = pr.v[1] = pr.v[2] = 0.0;
    int it;
    double r;
    ok[t] = con2prim(o, c, g, pr, &it, &r) ? 1 : 0;
    iters[t] = it;
    resid[t] = r;
    prim[6 * t] = pr.rho;
    prim[6 * t + 1] = pr.eps;
    prim[6 * t + 2] = pr.p;
    for (int i = 0; i < 3; ++i)
        prim[6 * t + 3 + i] = pr.v[i];
}

// The FP64 division, reciprocal, square root and reciprocal square root
// of the kernels at n points: out[4t .. 4t+3] = a/b, 1/b, sqrt(a),
// 1/sqrt(a).
__global__ void k_eval_arith(int64_t n, const double *__restrict__ a,
                             const double *__restrict__ b,
                             double *__restrict__ out)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    out[4 * t] = div_(a[t], b[t]);
    out[4 * t + 1] = rcp_(b[t]);
    out[4 * t + 2] = sqrt_(a[t]);
    out[4 * t + 3] = rsqrt_(a[t]);
}

// ------------------------------------------------------------- ensemble

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier of the persistent ensemble launch (every block is
// resident: the launch is cooperative and sized by the occupancy query).
// Thread 0 of each block arrives on a counter; the last arrival resets it
// and advances the generation the others wait on.  Each wait is bounded by
// bar_timeout_ns: a block whose wait runs out sets ctl->error (recording
// the phase) and every block leaves the kernel.  False on error.
__device__ bool ens_barrier(const EnsLaunch &a, int phase)
{
    EnsControl *c = a.ctl;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0)
    {
        volatile unsigned int *gen = &c->bar_gen;
        volatile int *err = &c->error;
        const unsigned int g = *gen;
        __threadfence();
        const unsigned int arrived = atomicAdd(&c->bar_count, 1u) + 1u;
        if (arrived == a.nblocks + a.bar_extra)
        {
            atomicExch(&c->bar_count, 0u);
            __threadfence();
            atomicAdd(&c->bar_gen, 1u);
        }
        else
        {
            const unsigned long long t0 = global_ns();
            while (*gen == g && *err == 0)
            {
                if (global_ns() - t0 > a.bar_timeout_ns)
                {
                    if (atomicCAS(&c->error, 0, 1) == 0)
                        c->error_phase = phase;
                    break;
                }
                __nanosleep(128);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int *)&a.ctl->error == 0;
}

// Next work item of phase `phase` for this block.
__device__ __forceinline__ int64_t ens_next(EnsControl *c, int phase,
                                            int64_t *sh)
{
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0)
        *sh = (int64_t)atomicAdd(&c->ctr[phase % 3], 1ull);
    __syncthreads();
    return *sh;
}

// Member owning item `it` of a prefix-sum table off[0..nm].
__device__ __forceinline__ int ens_find(const int64_t *off, int nm,
                                        int64_t it)
{
    int lo = 0, hi = nm;
    while (hi - lo > 1)
    {
        const int mid = (lo + hi) >> 1;
        if (__ldg(&off[mid]) <= it)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// dt of a member's step from the CFL speed of the step's input state, as
// the host driver computes it (cfl / max(speed, 1e-14), capped by max_dt).
__device__ __forceinline__ double ens_dt(const EnsMember &m,
                                         unsigned long long step)
{
    const double mi =
        __longlong_as_double((long long)__ldcg(&m.mi_bits[step & 1ull]));
    double dt = m.cfl / fmax(mi, 1.0e-14);
    if (m.max_dt > 0.0)
        dt = fmin(dt, m.max_dt);
    return dt;
}

// The persistent ensemble kernel: `steps` RK4 steps of every member.
// Phase 0: the CFL speed (when need_cfl), interior con2prim + sources and
// the ghost fill of every state.  Each stage: ghost fill of the stage input
// (not before the first stage of the launch), face pass into k, stage
// combination with post-stage recovery, the next RHS's con2prim + sources
// and (last stage) the next CFL speed; per member one bookkeeping item sums
// the accretion partials and advances the member time.  The arithmetic of
// every item is that of the single-box kernels.
template <typename T>
__global__ void __launch_bounds__(kEnsItemCells, kMinBlocks<T>)
    k_ensemble(EnsLaunch a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // raw storage: the member record is copied in word by word below
    __shared__ __align__(16) unsigned char ms_raw[sizeof(EnsMember)];
    EnsMember &ms = *reinterpret_cast<EnsMember *>(ms_raw);
    __shared__ int64_t item_sh;
    const int tid = threadIdx.y * kTB + threadIdx.x;
    EnsControl *ctl = a.ctl;
    const bool lead = blockIdx.x == 0 && tid == 0;
    const unsigned long long step0 = __ldcg(&ctl->steps_done);
    const bool need_cfl = __ldcg(&ctl->need_cfl) != 0;
    const int64_t ncell = __ldg(&a.off_cell[a.nm]);
    const int64_t nghost = __ldg(&a.off_ghost[a.nm]);
    const int64_t ntile = __ldg(&a.off_tile[a.nm]);
    int cur = -1;
    int ph = 0;
    auto load = [&](int m) {
        if (m != cur)
        {
            const unsigned long long *src =
                reinterpret_cast<const unsigned long long *>(a.m + m);
            unsigned long long *dst =
                reinterpret_cast<unsigned long long *>(&ms);
            for (int w = tid; w < (int)(sizeof(EnsMember) / 8);
                 w += kEnsItemCells)
                dst[w] = __ldg(&src[w]);
            __syncthreads();
            cur = m;
        }
    };
    auto zero_next_mi = [&](unsigned long long step) {
        for (int m = 0; m < a.nm; ++m)
            a.m[m].mi_bits[(step + 1ull) & 1ull] = 0ull;
    };

    // ---- phase 0
    {
        const int64_t ncfl = need_cfl ? ncell : 0;
        if (lead)
        {
            ctl->ctr[(ph + 1) % 3] = 0ull;
            zero_next_mi(step0);
        }
        for (;;)
        {
            int64_t it = ens_next(ctl, ph, &item_sh);
            if (it >= ncfl + ncell + nghost)
                break;
            if (it < ncfl)
            {
                const int m = ens_find(a.off_cell, a.nm, it);
                load(m);
                const int64_t t =
                    (it - __ldg(&a.off_cell[m])) * kEnsItemCells + tid;
                double v = 0.0;
                if (t < ms.b.ivol())
                    v = cfl_item<T, true>(ms.state, ms.b, ms.bg, ms.o, ms.inv,
                                          ms.st, t);
                flush_max_to(&ms.mi_bits[step0 & 1ull], v);
            }
            else if (it < ncfl + ncell)
            {
                it -= ncfl;
                const int m = ens_find(a.off_cell, a.nm, it);
                load(m);
                const int64_t t =
                    (it - __ldg(&a.off_cell[m])) * kEnsItemCells + tid;
                if (t < ms.b.ivol())
                    cells_item<T, true>(ms.state, static_cast<T *>(ms.prim),
                                        static_cast<T *>(ms.src), ms.b, ms.bg,
                                        ms.o, ms.st, t);
            }
            else
            {
                it -= ncfl + ncell;
                const int m = ens_find(a.off_ghost, a.nm, it);
                load(m);
                const int64_t t =
                    (it - __ldg(&a.off_ghost[m])) * kEnsItemCells + tid;
                if (t < ms.nshell)
                    ghost_item<T, true>(ms.state, static_cast<T *>(ms.prim),
                                        ms.b, ms.bg, ms.o, ms.st, t);
            }
        }
        if (!ens_barrier(a, ph++))
            return;
    }

    for (int n = 0; n < a.steps; ++n)
    {
        const unsigned long long step = step0 + (unsigned long long)n;
        for (int s = 0; s < 4; ++s)
        {
            // ---- ghost fill of the stage input
            if (n > 0 || s > 0)
            {
                if (lead)
                {
                    ctl->ctr[(ph + 1) % 3] = 0ull;
                    if (s == 0)
                        zero_next_mi(step);
                }
                for (;;)
                {
                    const int64_t it = ens_next(ctl, ph, &item_sh);
                    if (it >= nghost)
                        break;
                    const int m = ens_find(a.off_ghost, a.nm, it);
                    load(m);
                    const int64_t t =
                        (it - __ldg(&a.off_ghost[m])) * kEnsItemCells + tid;
                    if (t < ms.nshell)
                        ghost_item<T, true>(s == 0 ? ms.state : ms.stage,
                                            static_cast<T *>(ms.prim),
                                            s == 0 ? ms.b : ms.sb, ms.bg,
                                            ms.o, ms.st, t);
                }
                if (!ens_barrier(a, ph++))
                    return;
            }
            // ---- face pass
            if (lead)
                ctl->ctr[(ph + 1) % 3] = 0ull;
            for (;;)
            {
                const int64_t it = ens_next(ctl, ph, &item_sh);
                if (it >= ntile)
                    break;
                const int m = ens_find(a.off_tile, a.nm, it);
                load(m);
                const int64_t local = it - __ldg(&a.off_tile[m]);
                const int bx = (int)(local % ms.tiles[0]);
                const int64_t r = local / ms.tiles[0];
                const int by = (int)(r % ms.tiles[1]);
                const int bz = (int)(r / ms.tiles[1]);
                if (ms.has_mdot)
                    faces_tile<T, true, true>(
                        static_cast<const T *>(ms.prim),
                        static_cast<const T *>(ms.src), static_cast<T *>(ms.k),
                        ms.b, ms.bg, ms.o, ms.inv[0], ms.inv[1], ms.inv[2],
                        a.zchunk, bx, by, bz, smem_raw, ms.mdot_part, local);
                else
                    faces_tile<T, false, true>(
                        static_cast<const T *>(ms.prim),
                        static_cast<const T *>(ms.src), static_cast<T *>(ms.k),
                        ms.b, ms.bg, ms.o, ms.inv[0], ms.inv[1], ms.inv[2],
                        a.zchunk, bx, by, bz, smem_raw, nullptr, local);
            }
            if (!ens_barrier(a, ph++))
                return;
            // ---- stage combination (+ bookkeeping items)
            if (lead)
                ctl->ctr[(ph + 1) % 3] = 0ull;
            for (;;)
            {
                const int64_t it = ens_next(ctl, ph, &item_sh);
                if (it >= ncell + a.nm)
                    break;
                if (it < ncell)
                {
                    const int m = ens_find(a.off_cell, a.nm, it);
                    load(m);
                    const int64_t t =
                        (it - __ldg(&a.off_cell[m])) * kEnsItemCells + tid;
                    const double dt = ens_dt(ms, step);
                    unsigned long long cnt[4] = {0ull, 0ull, 0ull, 0ull};
                    double ci = 0.0;
                    if (t < ms.b.ivol())
                        stage_item<0, T, true>(
                            ms.state, ms.b.cs, nullptr, 0,
                            s < 3 ? ms.stage : ms.state,
                            s < 3 ? ms.sb.cs : ms.b.cs,
                            static_cast<const T *>(ms.k), ms.acc,
                            static_cast<T *>(ms.prim),
                            static_cast<T *>(ms.src), ms.b, ms.bg, ms.o, s,
                            dt, true, s == 3, s == 3, ms.inv, ms.st, t, cnt,
                            ci);
                    flush_counts(ms.st, cnt);
                    if (s == 3)
                        flush_max_to(&ms.mi_bits[(step + 1ull) & 1ull], ci);
                }
                else
                {
                    const int m = (int)(it - ncell);
                    load(m);
                    const double dt = ens_dt(ms, step);
                    if (ms.has_mdot)
                    {
                        // the single-box k_mdot_sum, 256 threads
                        const int64_t np = (int64_t)ms.tiles[0] *
                                           ms.tiles[1] * ms.tiles[2];
                        double v = 0.0;
                        for (int64_t q = tid; q < np; q += kEnsItemCells)
                            v += __ldcg(&ms.mdot_part[q]);
                        double *w = reinterpret_cast<double *>(smem_raw);
                        block_partial(v, w, w + 8, tid, kEnsItemCells, 0);
                        if (tid == 0)
                        {
                            const double wgt =
                                (dt / 6.0) * ((s == 1 || s == 2) ? 2.0 : 1.0);
                            ms.mdot_acc[0] = w[8];
                            ms.mdot_acc[1] += wgt * w[8];
                        }
                    }
                    if (s == 3 && tid == 0)
                        *ms.time += dt;
                }
            }
            if (!ens_barrier(a, ph++))
                return;
        }
    }
    if (lead)
    {
        ctl->steps_done = step0 + (unsigned long long)a.steps;
        ctl->need_cfl = 0;
    }
}

int grid_for(int64_t n, int threads)
{
    int64_t blocks = (n + threads - 1) / threads;
    const int64_t cap = 148 * 32; // grid-stride beyond ~32 waves
    if (blocks > cap)
        blocks = cap;
    return (int)(blocks < 1 ? 1 : blocks);
}

template <typename T> size_t faces_smem()
{
    return sizeof(T) *
           (5 * kPW * kPW + 2 * kGeoFields * kGW * kGW + 2 * 5 * kTB * kTC);
}

// ---------------------------------------------- CCZ4-stored geometry
// LevelDataFiniteVolumeOperator (Source/Matter/GRHD/FArrayBoxFiniteVolume.hpp:
// 1215-1364): the same Valencia operator with the geometry of every cell
// read from GRChombo's CCZ4 variables of the state (chi, h_ij, A_ij, K,
// lapse, shift; components 0..24, the GRHD ones from 25) and the metric
// derivatives of the sources as finite differences.  FP64 only.

constexpr int kCzChi = 0, kCzH = 1, kCzK = 7, kCzA = 8, kCzLapse = 18,
              kCzShift = 19;

// load_ccz4_geometry (:168-192): gamma = h / chi, gamma^-1 = chi h^-1 (the
// symmetric cofactor inverse of GRChombo's TensorAlgebra), K_ij = A_ij /
// chi + gamma_ij K / 3.
__device__ __forceinline__ void ccz4_geo(const double *__restrict__ s,
                                         int64_t cs, int64_t g, Geo &geo,
                                         double *K)
{
    const double chi = s[kCzChi * cs + g];
    double h[6], hu[6];
#pragma unroll
    for (int q = 0; q < 6; ++q)
        h[q] = s[(kCzH + q) * cs + g];
    const double det = h[0] * h[3] * h[5] + 2 * h[1] * h[2] * h[4] -
                       h[0] * h[4] * h[4] - h[3] * h[2] * h[2] -
                       h[5] * h[1] * h[1];
    hu[0] = (h[3] * h[5] - h[4] * h[4]) / det;
    hu[1] = (h[2] * h[4] - h[1] * h[5]) / det;
    hu[2] = (h[1] * h[4] - h[2] * h[3]) / det;
    hu[3] = (h[0] * h[5] - h[2] * h[2]) / det;
    hu[4] = (h[1] * h[2] - h[0] * h[4]) / det;
    hu[5] = (h[0] * h[3] - h[1] * h[1]) / det;
#pragma unroll
    for (int q = 0; q < 6; ++q)
    {
        geo.gLL[q] = h[q] / chi;
        geo.gUU[q] = chi * hu[q];
    }
    if (K)
    {
        const double trK = s[kCzK * cs + g];
#pragma unroll
        for (int q = 0; q < 6; ++q)
            K[q] = s[(kCzA + q) * cs + g] / chi + geo.gLL[q] * trK / 3.0;
    }
    geo.lapse = s[kCzLapse * cs + g];
#pragma unroll
    for (int d = 0; d < 3; ++d)
        geo.shift[d] = s[(kCzShift + d) * cs + g];
}

// The geometry cache: gLL[6] gUU[6] lapse shift[3] per ghosted cell.
__device__ __forceinline__ void geo_put(double *gc, int64_t n, int64_t g,
                                        const Geo &v)
{
#pragma unroll
    for (int q = 0; q < 6; ++q)
    {
        gc[q * n + g] = v.gLL[q];
        gc[(6 + q) * n + g] = v.gUU[q];
    }
    gc[12 * n + g] = v.lapse;
#pragma unroll
    for (int d = 0; d < 3; ++d)
        gc[(13 + d) * n + g] = v.shift[d];
}

__device__ __forceinline__ Geo geo_get(const double *__restrict__ gc,
                                       int64_t n, int64_t g)
{
    Geo v;
#pragma unroll
    for (int q = 0; q < 6; ++q)
    {
        v.gLL[q] = gc[q * n + g];
        v.gUU[q] = gc[(6 + q) * n + g];
    }
    v.lapse = gc[12 * n + g];
#pragma unroll
    for (int d = 0; d < 3; ++d)
        v.shift[d] = gc[(13 + d) * n + g];
    return v;
}

__device__ __forceinline__ void ghosted_cell(const BoxDev &b, int64_t t,
                                             int &i, int &j, int &k)
{
    i = b.glo[0] + (int)(t % b.gn[0]);
    const int64_t r = t / b.gn[0];
    j = b.glo[1] + (int)(r % b.gn[1]);
    k = b.glo[2] + (int)(r / b.gn[1]);
}

// fill_conserved_outflow_boundaries (:484-519) and
// fill_ccz4_geometry_outflow_boundaries (:430-473): a physical ghost copies
// the conserved variables (when `conserved`) and chi, h_ij, lapse, shift of
// its source cell (the box's end in each direction it lies outside in).
__global__ void __launch_bounds__(256)
    k_ccz4_fill(double *__restrict__ s, BoxDev b, int conserved)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
         t < b.gvol(); t += (int64_t)gridDim.x * blockDim.x)
    {
        int iv[3];
        ghosted_cell(b, t, iv[0], iv[1], iv[2]);
        int src[3] = {iv[0], iv[1], iv[2]};
        bool ghost = false;
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            if (iv[d] < b.dlo[d])
            {
                ghost = true;
                src[d] = b.lo[d];
            }
            else if (iv[d] > b.dhi[d])
            {
                ghost = true;
                src[d] = b.hi[d];
            }
        }
        if (!ghost)
            continue;
        const int64_t g = t, sg = b.gidx(src[0], src[1], src[2]);
        if (conserved)
            for (int c = 0; c < 5; ++c)
                s[(kCcz4GrhdOffset + c) * b.cs + g] =
                    s[(kCcz4GrhdOffset + c) * b.cs + sg];
        for (int q = 0; q < 7; ++q) // chi, h
            s[q * b.cs + g] = s[q * b.cs + sg];
        for (int q = kCzLapse; q < kCzLapse + 4; ++q) // lapse, shift
            s[q * b.cs + g] = s[q * b.cs + sg];
    }
}

// recover_primitives_from_ccz4_geometry over the ghosted box (:681-702):
// the primitive cache (rho, p, v) and the geometry cache of every cell.
__global__ void __launch_bounds__(256)
    k_ccz4_cells(const double *__restrict__ s, BoxDev b, Options o,
                 double *__restrict__ prim, double *__restrict__ gc,
                 DevStatus *st)
{
    const double *q = s + kCcz4GrhdOffset * b.cs;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
         t < b.gvol(); t += (int64_t)gridDim.x * blockDim.x)
    {
        Geo geo;
        ccz4_geo(s, b.cs, t, geo, nullptr);
        geo_put(gc, b.gvol(), t, geo);
        Prim pr;
        if (!con2prim(o, load_cons(q, b.cs, t), geo.gUU, pr, nullptr,
                      nullptr))
        {
            record_error(st, 2, t);
            pr.rho = pr.p = 1.0;
            pr.v[0] = pr.v[1] = pr.v[2] = 0.0;
        }
        store_pv(prim, b.gvol(), t, pr);
    }
}

__device__ __forceinline__ double log_sqrt_det6(const double *g)
{
    const double det = g[0] * g[3] * g[5] + 2 * g[1] * g[2] * g[4] -
                       g[0] * g[4] * g[4] - g[3] * g[2] * g[2] -
                       g[5] * g[1] * g[1];
    return (det <= 0.0 || !isfinite(det)) ? 0.0 : 0.5 * log(det);
}

// The RHS of one interior cell: per direction the two faces of the cell
// (compute_directional_flux_rhs_from_ccz4_geometry, :784-833, every face
// twice as the reference computes it), then the static-metric sources with
// finite-difference derivatives (add_static_metric_sources_to_conserved_rhs,
// :367-427; one-sided where a neighbour's stored primitives are metric-
// source atmosphere, make_metric_source_derivative_stencil, :283-322).
__global__ void __launch_bounds__(256, 2)
    k_ccz4_rhs(const double *__restrict__ s, BoxDev b, Options o,
               const double *__restrict__ prim, const double *__restrict__ gc,
               double *__restrict__ rhs, int64_t rcs, double inv0,
               double inv1, double inv2, DevStatus *st)
{
    const int64_t n = b.gvol();
    const double *q = s + kCcz4GrhdOffset * b.cs;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
         t < b.ivol(); t += (int64_t)gridDim.x * blockDim.x)
    {
        int i, j, k;
        interior_cell(b, t, i, j, k);
        const int64_t g = b.gidx(i, j, k);
        const double inv[3] = {inv0, inv1, inv2};
        const int64_t step[3] = {1, (int64_t)b.gn[0],
                                 (int64_t)b.gn[0] * b.gn[1]};
        Cons r;
        r.D = r.tau = 0.0;
        r.S[0] = r.S[1] = r.S[2] = 0.0;
        for (int d = 0; d < 3; ++d)
        {
            const int64_t so = step[d];
            Cons f[2];
            for (int side = 0; side < 2; ++side)
            {
                const int64_t L = g - so + side * so, R = L + so;
                Geo gf;
                average_geo(geo_get(gc, n, L), geo_get(gc, n, R), gf);
                f[side] = face_flux(o, load_pv_global<double>(prim, n, L - so),
                                    load_pv_global<double>(prim, n, L),
                                    load_pv_global<double>(prim, n, R),
                                    load_pv_global<double>(prim, n, R + so),
                                    gf, d);
            }
            r.D += -inv[d] * (f[1].D - f[0].D);
            r.tau += -inv[d] * (f[1].tau - f[0].tau);
#pragma unroll
            for (int m = 0; m < 3; ++m)
                r.S[m] += -inv[d] * (f[1].S[m] - f[0].S[m]);
        }
        if (o.use_src)
        {
            GeoFull fg;
            ccz4_geo(s, b.cs, g, fg.g, fg.K);
            const PV pv = load_pv_global<double>(prim, n, g);
            Prim pr;
            pr.rho = pv.q[0];
            pr.p = pv.q[1];
            pr.v[0] = pv.q[2];
            pr.v[1] = pv.q[3];
            pr.v[2] = pv.q[4];
            floors(o, pr, fg.g.gLL);
            if (!is_atmo(o, pr, o.src_atmo_factor))
            {
                for (int d = 0; d < 3; ++d)
                {
                    fg.dlapse[d] = fg.dlnsqrtg[d] = 0.0;
#pragma unroll
                    for (int q6 = 0; q6 < 6; ++q6)
                        fg.dgamma[d][q6] = 0.0;
#pragma unroll
                    for (int m = 0; m < 3; ++m)
                        fg.dshift[m][d] = 0.0;
                    const int64_t lo_i = g - step[d], hi_i = g + step[d];
                    Prim pl, pu;
                    pl.rho = q[kRho * b.cs + lo_i];
                    pl.p = q[kPress * b.cs + lo_i];
                    pu.rho = q[kRho * b.cs + hi_i];
                    pu.p = q[kPress * b.cs + hi_i];
                    const bool la = !is_atmo(o, pl, o.src_atmo_factor);
                    const bool ua = !is_atmo(o, pu, o.src_atmo_factor);
                    int64_t lc, uc;
                    double coef;
                    if (la && ua)
                    {
                        lc = lo_i;
                        uc = hi_i;
                        coef = 0.5 * inv[d];
                    }
                    else if (ua)
                    {
                        lc = g;
                        uc = hi_i;
                        coef = inv[d];
                    }
                    else if (la)
                    {
                        lc = lo_i;
                        uc = g;
                        coef = inv[d];
                    }
                    else
                        continue;
                    const Geo gu = geo_get(gc, n, uc), gl = geo_get(gc, n, lc);
                    fg.dlapse[d] = coef * (gu.lapse - gl.lapse);
                    fg.dlnsqrtg[d] =
                        coef * (log_sqrt_det6(gu.gLL) - log_sqrt_det6(gl.gLL));
#pragma unroll
                    for (int q6 = 0; q6 < 6; ++q6)
                        fg.dgamma[d][q6] = coef * (gu.gLL[q6] - gl.gLL[q6]);
#pragma unroll
                    for (int m = 0; m < 3; ++m)
                        fg.dshift[m][d] = coef * (gu.shift[m] - gl.shift[m]);
                }
                const Cons c = load_cons(q, b.cs, g);
                const Cons src = static_sources(pr, c, fg);
                r.D += src.D;
                r.tau += src.tau;
#pragma unroll
                for (int m = 0; m < 3; ++m)
                    r.S[m] += src.S[m];
            }
        }
        rhs[0 * rcs + t] = r.D;
        rhs[1 * rcs + t] = r.S[0];
        rhs[2 * rcs + t] = r.S[1];
        rhs[3 * rcs + t] = r.S[2];
        rhs[4 * rcs + t] = r.tau;
    }
}

// recover_primitives_and_apply_atmosphere_from_ccz4_geometry (:713-761).
__global__ void __launch_bounds__(256)
    k_ccz4_recover(double *__restrict__ s, BoxDev b, Options o, DevStatus *st)
{
    double *q = s + kCcz4GrhdOffset * b.cs;
    unsigned long long cnt[4] = {0, 0, 0, 0};
    const int64_t n = b.ivol();
    const int64_t n_pad = (n + blockDim.x - 1) / blockDim.x * blockDim.x;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_pad;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        if (t < n)
        {
            int i, j, k;
            interior_cell(b, t, i, j, k);
            const int64_t g = b.gidx(i, j, k);
            Geo geo;
            ccz4_geo(s, b.cs, g, geo, nullptr);
            recover_cell(o, geo, load_cons(q, b.cs, g), q, b.cs, g, cnt);
        }
        flush_counts(st, cnt);
        cnt[0] = cnt[1] = cnt[2] = cnt[3] = 0;
    }
}

// compute_max_inverse_dt_from_ccz4_geometry (:1139-1183).
__global__ void __launch_bounds__(256)
    k_ccz4_max_inv_dt(const double *__restrict__ s, BoxDev b, Options o,
                      double inv0, double inv1, double inv2, DevStatus *st)
{
    const double *q = s + kCcz4GrhdOffset * b.cs;
    const int64_t n = b.ivol();
    const int64_t n_pad = (n + blockDim.x - 1) / blockDim.x * blockDim.x;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_pad;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        double cell = 0.0;
        if (t < n)
        {
            int i, j, k;
            interior_cell(b, t, i, j, k);
            const int64_t g = b.gidx(i, j, k);
            Geo geo;
            ccz4_geo(s, b.cs, g, geo, nullptr);
            Prim pr;
            if (!con2prim(o, load_cons(q, b.cs, g), geo.gUU, pr, nullptr,
                          nullptr))
                record_error(st, 4, t); // GRHD_WHERE_CFL
            else
            {
                floors(o, pr, geo.gLL);
                if (!is_atmo(o, pr, 1.0 + 1.0e-12))
                {
                    const double inv[3] = {inv0, inv1, inv2};
                    for (int d = 0; d < 3; ++d)
                    {
                        double lo, hi;
                        char_speeds(o, pr, geo, d, lo, hi);
                        cell += fmax(fabs(lo), fabs(hi)) * inv[d];
                    }
                }
            }
        }
        flush_max(st, cell);
    }
}

// add_scaled_conserved_rhs (:927-940) and combine_ssprk2_conserved_state
// (:942-969) on the GRHD components: mode 0 s += dt rhs; mode 1
// s = (s + u1 + dt rhs) / 2.
__global__ void __launch_bounds__(256)
    k_ccz4_update(double *__restrict__ s, const double *__restrict__ u1,
                  int64_t ucs, const double *__restrict__ rhs, int64_t rcs,
                  BoxDev b, double dt, int mode)
{
    double *q = s + kCcz4GrhdOffset * b.cs;
    const double *u = u1 ? u1 + kCcz4GrhdOffset * ucs : nullptr;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
         t < b.ivol(); t += (int64_t)gridDim.x * blockDim.x)
    {
        int i, j, k;
        interior_cell(b, t, i, j, k);
        const int64_t g = b.gidx(i, j, k);
        for (int c = 0; c < 5; ++c)
        {
            const double x = rhs[c * rcs + t];
            if (mode == 0)
                q[c * b.cs + g] += dt * x;
            else
                q[c * b.cs + g] = 0.5 * (q[c * b.cs + g] + u[c * ucs + g] +
                                         dt * x);
        }
    }
}

__global__ void k_ccz4_probe(const double *__restrict__ s, BoxDev b,
                             Options o, int i, int j, int k, double *out)
{
    const int64_t g = b.gidx(i, j, k);
    Geo geo;
    ccz4_geo(s, b.cs, g, geo, nullptr);
    Prim pr;
    double res = 0.0;
    con2prim(o, load_cons(s + kCcz4GrhdOffset * b.cs, b.cs, g), geo.gUU, pr,
             nullptr, &res);
    *out = res;
}

} // namespace

cudaError_t configure_kernels()
{
    cudaError_t e = cudaSuccess;
    const cudaFuncAttribute attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
    const int d = (int)faces_smem<double>(), f = (int)faces_smem<float>();
    const void *fp64[] = {(const void *)k_faces<double, false, 0>,
                          (const void *)k_faces<double, true, 0>,
                          (const void *)k_faces<double, false, 1>,
                          (const void *)k_faces<double, true, 1>};
    const void *fp32[] = {(const void *)k_faces<float, false, 0>,
                          (const void *)k_faces<float, true, 0>,
                          (const void *)k_faces<float, false, 1>,
                          (const void *)k_faces<float, true, 1>};
    for (const void *k : fp64)
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k, attr, d);
    for (const void *k : fp32)
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k, attr, f);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_ensemble<double>, attr,
                                 (int)faces_smem<double>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_ensemble<float>, attr,
                                 (int)faces_smem<float>());
    return e;
}

template <typename T> size_t ensemble_smem() { return faces_smem<T>(); }

template <typename T> cudaError_t ensemble_occupancy(int *blocks_per_sm)
{
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        blocks_per_sm, k_ensemble<T>, kEnsItemCells, faces_smem<T>());
}

template <typename T>
cudaError_t launch_ensemble(const EnsLaunch &a, int grid, cudaStream_t s)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kTB, kTB);
    cfg.dynamicSmemBytes = faces_smem<T>();
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_ensemble<T>, a);
}

template size_t ensemble_smem<double>();
template size_t ensemble_smem<float>();
template cudaError_t ensemble_occupancy<double>(int *);
template cudaError_t ensemble_occupancy<float>(int *);
template cudaError_t launch_ensemble<double>(const EnsLaunch &, int,
                                             cudaStream_t);
template cudaError_t launch_ensemble<float>(const EnsLaunch &, int,
                                            cudaStream_t);

namespace
{
// resident face-kernel blocks of the current device (SMs x blocks per SM
// at the kernel's registers and shared memory), per precision
int face_slots(bool fp32)
{
    static std::atomic<int> cache[64][2];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return fp32 ? 3 * 148 : 2 * 148;
    std::atomic<int> &c = cache[dev][fp32 ? 1 : 0];
    const int have = c.load(std::memory_order_relaxed);
    if (have > 0)
        return have;
    int sms = 148, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const cudaError_t e =
        fp32 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                   &per, k_faces<float, false, 0>, kTB * kTB,
                   faces_smem<float>())
             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                   &per, k_faces<double, false, 0>, kTB * kTB,
                   faces_smem<double>());
    if (e != cudaSuccess || per < 1)
    {
        (void)cudaGetLastError();
        per = fp32 ? 3 : 2;
    }
    c.store(sms * per, std::memory_order_relaxed);
    return sms * per;
}
} // namespace

// Makespan (in plane-times) of nf blocks of df planes followed by np of dp
// planes on `slots` resident blocks, each block started on the slot that
// frees first in launch order (the last z row of a launch holds the short
// blocks): whole waves of full blocks, then the short blocks on the slots
// left free in the last full wave and on the others as they free.
int64_t face_makespan(int64_t nf, int64_t df, int64_t np, int64_t dp,
                      int64_t slots)
{
    const int64_t t1 = (nf / slots) * df, rem = nf % slots;
    int64_t ta = t1, na = slots - rem;           // free at t1
    int64_t tb = t1 + (rem ? df : 0), nb = rem;  // free after the last full
    int64_t end = rem ? tb : t1;
    for (int64_t left = np; left > 0;)
    {
        if (nb == 0 || ta <= tb)
        {
            left -= std::min(left, na);
            ta += dp;
            end = std::max(end, ta);
        }
        else
        {
            left -= std::min(left, nb);
            tb += dp;
            end = std::max(end, tb);
        }
    }
    return end;
}

int face_zchunk(const BoxDev &b, int zchunk, bool fp32)
{
    if (zchunk > 0)
        return zchunk;
    return face_zchunk_model(b.in[0], b.in[1], b.in[2], face_slots(fp32));
}

int face_zchunk_model(int nx, int ny, int nz, int64_t slots)
{
    const int64_t tiles =
        (int64_t)((nx + kTC - 1) / kTC) * ((ny + kTC - 1) / kTC);
    const int cand[5] = {32, 16, 8, 6, 4};
    int best = cand[0];
    int64_t best_cost = -1;
    for (int z : cand)
    {
        // nz / z full blocks per column of tiles, then one of nz % z
        // planes; every block also marches two lead-in planes
        const int r = nz % z;
        const int64_t cost = face_makespan(tiles * (nz / z), z + 2,
                                           r ? tiles : 0, r + 2, slots);
        if (best_cost < 0 || cost < best_cost)
        {
            best = z;
            best_cost = cost;
        }
    }
    return best;
}

int64_t face_kernel_blocks(const BoxDev &b, int zchunk, bool fp32)
{
    zchunk = face_zchunk(b, zchunk, fp32);
    return (int64_t)((b.in[0] + kTC - 1) / kTC) * ((b.in[1] + kTC - 1) / kTC) *
           ((b.in[2] + zchunk - 1) / zchunk);
}

template <typename T>
void launch_fill_ghosts(double *state, T *prim, const BoxDev &b,
                        const Background &bg, const Options &o, DevStatus *st,
                        cudaStream_t s)
{
    const int64_t nshell = b.gvol() - b.ivol();
    if (nshell <= 0)
        return;
    k_fill_ghosts<T><<<grid_for(nshell, 256), 256, 0, s>>>(state, prim, b, bg,
                                                          o, st, nshell);
}

template <typename T>
void launch_fill_ghost_planes(double *state, T *prim, const BoxDev &b,
                              const Background &bg, const Options &o,
                              DevStatus *st, int k0, int k1, cudaStream_t s)
{
    const int64_t n = plane_shell_count(b, k0, k1);
    if (n <= 0)
        return;
    k_fill_ghost_planes<T><<<grid_for(n, 256), 256, 0, s>>>(state, prim, b, bg,
                                                           o, st, k0, k1, n);
}

template <typename T>
void launch_cells(const double *state, T *prim, T *src, const BoxDev &b,
                  const Background &bg, const Options &o, DevStatus *st,
                  cudaStream_t s)
{
    k_cells<T><<<grid_for(b.ivol(), 256), 256, 0, s>>>(state, prim, src, b, bg,
                                                       o, st);
}

template <typename T>
void launch_faces(const T *prim, const T *src, T *rhs, const BoxDev &b,
                  const Background &bg, const Options &o,
                  const double inv_dx[3], int zchunk, double *mdot_part,
                  cudaStream_t s)
{
    zchunk = face_zchunk(b, zchunk, sizeof(T) == sizeof(float));
    dim3 grid((b.in[0] + kTC - 1) / kTC, (b.in[1] + kTC - 1) / kTC,
              (b.in[2] + zchunk - 1) / zchunk);
    dim3 block(kTB, kTB);
    // one instantiation per background kind: each carries only its own
    // metric code
    const bool md = o.accretion_radius > 0.0 && mdot_part;
    auto go = [&](auto kern) {
        kern<<<grid, block, faces_smem<T>(), s>>>(
            prim, src, rhs, b, bg, o, inv_dx[0], inv_dx[1], inv_dx[2], zchunk,
            md ? mdot_part : nullptr);
    };
    if (bg.kind == 1)
        md ? go(k_faces<T, true, 1>) : go(k_faces<T, false, 1>);
    else
        md ? go(k_faces<T, true, 0>) : go(k_faces<T, false, 0>);
}

void launch_mdot_sum(const double *part, int64_t n, double weight,
                     double *acc, cudaStream_t s)
{
    k_mdot_sum<<<1, 256, 0, s>>>(part, n, weight, acc);
}

void launch_update(double *dst, int64_t dcs, const double *src_state,
                   int64_t scs, const double *rhs, const BoxDev &b,
                   const Background &bg, const Options &o, double dt,
                   int recover, DevStatus *st, cudaStream_t s)
{
    k_update<<<grid_for(b.ivol(), 256), 256, 0, s>>>(
        dst, dcs, src_state, scs, rhs, b, bg, o, dt, recover, st);
}

void launch_recover(double *state, const BoxDev &b, const Background &bg,
                    const Options &o, DevStatus *st, cudaStream_t s)
{
    k_recover<<<grid_for(b.ivol(), 256), 256, 0, s>>>(state, b, bg, o, st);
}

template <typename T>
void launch_stage(int mode, const double *un, int64_t ucs, const double *us,
                  int64_t tcs, double *out, int64_t ocs, const T *k,
                  double *acc, T *prim, T *src, int prep, const BoxDev &b,
                  const Background &bg, const Options &o, int stage,
                  double dt, bool cfl, const double inv_dx[3], DevStatus *st,
                  cudaStream_t s, const T *prim_in)
{
    const int grid = grid_for(b.ivol(), 256);
    const double i0 = inv_dx ? inv_dx[0] : 0.0, i1 = inv_dx ? inv_dx[1] : 0.0,
                 i2 = inv_dx ? inv_dx[2] : 0.0;
    const int pf = prep, cf = cfl ? 1 : 0;
    auto go = [&](auto kern) {
        kern<<<grid, 256, 0, s>>>(un, ucs, us, tcs, out, ocs, k, acc, prim, src,
                                  b, bg, o, stage, dt, pf, cf, i0, i1, i2, st,
                                  prim_in);
    };
    // one instantiation per background kind (only its own metric code)
    const bool pn = bg.kind == 1;
    if (mode == 0)
        pn ? go(k_stage<0, T, 1>) : go(k_stage<0, T, 0>);
    else if (mode == 1)
        pn ? go(k_stage<1, T, 1>) : go(k_stage<1, T, 0>);
    else
        pn ? go(k_stage<2, T, 1>) : go(k_stage<2, T, 0>);
}

void launch_max_inv_dt(const double *state, const BoxDev &b,
                       const Background &bg, const Options &o,
                       const double inv_dx[3], DevStatus *st, bool mixed,
                       cudaStream_t s)
{
    if (mixed)
        k_max_inv_dt<float><<<grid_for(b.ivol(), 256), 256, 0, s>>>(
            state, b, bg, o, inv_dx[0], inv_dx[1], inv_dx[2], st);
    else
        k_max_inv_dt<double><<<grid_for(b.ivol(), 256), 256, 0, s>>>(
            state, b, bg, o, inv_dx[0], inv_dx[1], inv_dx[2], st);
}

void launch_residual_probe(const double *state, const BoxDev &b,
                           const Background &bg, const Options &o, int i,
                           int j, int k, double *out, cudaStream_t s)
{
    k_residual_probe<<<1, 1, 0, s>>>(state, b, bg, o, i, j, k, out);
}

void launch_widen(const float *in, int64_t n, double *out, int64_t ocs,
                  cudaStream_t s)
{
    k_widen<<<grid_for(5 * n, 256), 256, 0, s>>>(in, n, out, ocs);
}

void launch_eval_background(int64_t n, const double *xyz,
                            const Background &bg, double *out, cudaStream_t s)
{
    if (n <= 0)
        return;
    k_eval_background<<<(int)((n + 127) / 128), 128, 0, s>>>(n, xyz, bg, out);
}

void launch_eval_con2prim(int64_t n, const double *cons, const double *gUU,
                          const Options &o, double *prim, int *ok, int *iters,
                          double *resid, cudaStream_t s)
{
    if (n <= 0)
        return;
    k_eval_con2prim<<<(int)((n + 127) / 128), 128, 0, s>>>(n, cons, gUU, o,
                                                           prim, ok, iters,
                                                           resid);
}

void launch_eval_arith(int64_t n, const double *a, const double *b,
                       double *out, cudaStream_t s)
{
    if (n <= 0)
        return;
    k_eval_arith<<<(int)((n + 255) / 256), 256, 0, s>>>(n, a, b, out);
}

void launch_ccz4_fill(double *s, const BoxDev &b, bool conserved,
                      cudaStream_t st)
{
    k_ccz4_fill<<<grid_for(b.gvol(), 256), 256, 0, st>>>(s, b,
                                                          conserved ? 1 : 0);
}

void launch_ccz4_cells(const double *s, const BoxDev &b, const Options &o,
                       double *prim, double *gc, DevStatus *st,
                       cudaStream_t stream)
{
    k_ccz4_cells<<<grid_for(b.gvol(), 256), 256, 0, stream>>>(s, b, o, prim,
                                                               gc, st);
}

void launch_ccz4_rhs(const double *s, const BoxDev &b, const Options &o,
                     const double *prim, const double *gc, double *rhs,
                     int64_t rcs, const double inv[3], DevStatus *st,
                     cudaStream_t stream)
{
    k_ccz4_rhs<<<grid_for(b.ivol(), 256), 256, 0, stream>>>(
        s, b, o, prim, gc, rhs, rcs, inv[0], inv[1], inv[2], st);
}

void launch_ccz4_recover(double *s, const BoxDev &b, const Options &o,
                         DevStatus *st, cudaStream_t stream)
{
    k_ccz4_recover<<<grid_for(b.ivol(), 256), 256, 0, stream>>>(s, b, o, st);
}

void launch_ccz4_max_inv_dt(const double *s, const BoxDev &b,
                            const Options &o, const double inv[3],
                            DevStatus *st, cudaStream_t stream)
{
    k_ccz4_max_inv_dt<<<grid_for(b.ivol(), 256), 256, 0, stream>>>(
        s, b, o, inv[0], inv[1], inv[2], st);
}

void launch_ccz4_update(double *s, const double *u1, int64_t ucs,
                        const double *rhs, int64_t rcs, const BoxDev &b,
                        double dt, int mode, cudaStream_t stream)
{
    k_ccz4_update<<<grid_for(b.ivol(), 256), 256, 0, stream>>>(
        s, u1, ucs, rhs, rcs, b, dt, mode);
}

void launch_ccz4_probe(const double *s, const BoxDev &b, const Options &o,
                       int i, int j, int k, double *out, cudaStream_t stream)
{
    k_ccz4_probe<<<1, 1, 0, stream>>>(s, b, o, i, j, k, out);
}

#define GRHD_INSTANTIATE(T)                                                   \
    template void launch_fill_ghosts<T>(double *, T *, const BoxDev &,        \
                                        const Background &, const Options &,  \
                                        DevStatus *, cudaStream_t);           \
    template void launch_fill_ghost_planes<T>(                                \
        double *, T *, const BoxDev &, const Background &, const Options &,   \
        DevStatus *, int, int, cudaStream_t);                                 \
    template void launch_cells<T>(const double *, T *, T *, const BoxDev &,   \
                                  const Background &, const Options &,        \
                                  DevStatus *, cudaStream_t);                 \
    template void launch_faces<T>(const T *, const T *, T *, const BoxDev &,  \
                                  const Background &, const Options &,        \
                                  const double *, int, double *,              \
                                  cudaStream_t);                              \
    template void launch_stage<T>(int, const double *, int64_t,               \
                                  const double *, int64_t, double *, int64_t, \
                                  const T *, double *, T *, T *, int,         \
                                  const BoxDev &, const Background &,         \
                                  const Options &, int, double, bool,         \
                                  const double *, DevStatus *, cudaStream_t,  \
                                  const T *);

GRHD_INSTANTIATE(double)
GRHD_INSTANTIATE(float)

} // namespace grhd
