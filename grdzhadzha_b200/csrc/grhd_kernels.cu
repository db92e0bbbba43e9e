// grhd_kernels.cu -- sm_100a kernels of the fixed-background Valencia GRHD
// operator (FP64).
//
// One RHS evaluation is three launches:
//   fill_ghosts : physical (outflow) ghost cells of the box, as
//                 fill_conserved_outflow_boundaries_from_fixed_background
//                 (FixedBGFArrayBoxFiniteVolume.hpp:113-177);
//   cells       : per cell of the ghosted box, metric + con2prim into the
//                 primitive scratch (recover_primitives_from_fixed_background,
//                 :33-58), and for interior cells the static-metric and
//                 volume-time sources (:255-298, :616-675);
//   faces       : every face of the box computed once -- MUSCL slopes,
//                 floors, p2c, HLLE -- with the flux divergence and the
//                 sources written straight to the RHS (:179-253, :300-363).
// The reference evaluates each face twice and every direction in a
// separate pass over the box; here each face is evaluated once and the
// interface states never leave registers / shared memory.
#include "grhd_kernels.cuh"

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

__device__ __forceinline__ Cons load_cons(const double *s, int64_t cs,
                                          int64_t idx)
{
    Cons c;
    c.D = s[kD * cs + idx];
    c.S[0] = s[(kS1 + 0) * cs + idx];
    c.S[1] = s[(kS1 + 1) * cs + idx];
    c.S[2] = s[(kS1 + 2) * cs + idx];
    c.tau = s[kTau * cs + idx];
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

__device__ __forceinline__ Prim load_prim(const double *s, int64_t cs,
                                          int64_t idx)
{
    Prim p;
    p.rho = s[kRho * cs + idx];
    p.eps = s[kEps * cs + idx];
    p.p = s[kPress * cs + idx];
    p.v[0] = s[(kV1 + 0) * cs + idx];
    p.v[1] = s[(kV1 + 1) * cs + idx];
    p.v[2] = s[(kV1 + 2) * cs + idx];
    return p;
}

__device__ __forceinline__ bool primitive_differs(const Prim &a, const Prim &b)
{
    return a.rho != b.rho || a.eps != b.eps || a.p != b.p ||
           a.v[0] != b.v[0] || a.v[1] != b.v[1] || a.v[2] != b.v[2];
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

__device__ __forceinline__ void store_pv(double *prim, int64_t pcs,
                                         int64_t g, const Prim &pr)
{
    prim[0 * pcs + g] = pr.rho;
    prim[1 * pcs + g] = pr.p;
    prim[2 * pcs + g] = pr.v[0];
    prim[3 * pcs + g] = pr.v[1];
    prim[4 * pcs + g] = pr.v[2];
}

// Physical (outflow) ghost fill of the shell "ghosted box minus box"
// (fill_conserved_outflow_boundaries_from_fixed_background, :113-177),
// then, for every shell cell, the ghosted-box con2prim of the RHS into the
// primitive cache (recover_primitives_from_fixed_background, :33-58).
__global__ void __launch_bounds__(256)
    k_fill_ghosts(double *__restrict__ state, double *__restrict__ prim,
                  BoxDev b, Background bg, Options o, DevStatus *st,
                  int64_t nshell)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
         t < nshell; t += (int64_t)gridDim.x * blockDim.x)
    {
        int i, j, k;
        if (!shell_cell(b, t, i, j, k))
            continue;
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
        Geo tg;
        background_metric<false>(bg, x, y, z, tg, nullptr);
        Cons c;
        if (ghost)
        {
            double sx, sy, sz;
            cell_xyz(o, srcc[0], srcc[1], srcc[2], sx, sy, sz);
            Geo sg;
            background_metric<false>(bg, sx, sy, sz, sg, nullptr);
            const Cons sc =
                load_cons(state, b.cs, b.gidx(srcc[0], srcc[1], srcc[2]));
            Prim pr;
            if (!con2prim(o, sc, sg.gUU, pr, nullptr, nullptr))
            {
                record_error(st, 1, idx);
                continue;
            }
            floors(o, pr, tg.gLL);
            store_prim(state, b.cs, idx, pr);
            c = p2c(pr, tg.gLL);
            store_cons(state, b.cs, idx, c);
        }
        else
            c = load_cons(state, b.cs, idx);
        Prim pr;
        if (!con2prim(o, c, tg.gUU, pr, nullptr, nullptr))
        {
            record_error(st, 2, idx);
            pr.rho = pr.p = 1.0;
            pr.v[0] = pr.v[1] = pr.v[2] = 0.0;
        }
        store_pv(prim, b.pcs, idx, pr);
    }
}

// Static-metric sources (:255-298) from the floored primitives and, for
// the binary, the volume-time source (:616-675); `pr` is the cell's
// unfloored con2prim result.
__device__ __forceinline__ Cons cell_sources(const Options &o,
                                             const Background &bg, double x,
                                             double y, double z,
                                             const Prim &pr, const Cons &c,
                                             const GeoFull &f)
{
    Cons s;
    s.D = s.tau = s.S[0] = s.S[1] = s.S[2] = 0.0;
    if (o.use_src)
    {
        Prim fp = pr;
        floors(o, fp, f.g.gLL);
        if (!is_atmo(o, fp, o.src_atmo_factor))
            s = static_sources(fp, c, f);
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
        s.D += 0.0 - c.D * dl;
        s.tau += 0.0 - c.tau * dl;
#pragma unroll
        for (int m = 0; m < 3; ++m)
            s.S[m] += 0.0 - c.S[m] * dl;
    }
    return s;
}

__device__ __forceinline__ void store_src(double *src, int64_t rcs,
                                          int64_t ri, const Cons &s)
{
    src[0 * rcs + ri] = s.D;
    src[1 * rcs + ri] = s.S[0];
    src[2 * rcs + ri] = s.S[1];
    src[3 * rcs + ri] = s.S[2];
    src[4 * rcs + ri] = s.tau;
}

// ------------------------------------------------------- per-cell pass

// Interior cells: con2prim into the primitive cache (the ghosted-box
// recovery of the RHS restricted to the interior; the shell is done by
// k_fill_ghosts) and the sources into the source scratch.  Excised cells
// keep their frozen primitives and get no source.
__global__ void __launch_bounds__(256, 2)
    k_cells(const double *__restrict__ state, double *__restrict__ prim,
            double *__restrict__ src, BoxDev b, Background bg, Options o,
            DevStatus *st)
{
    const int64_t n = b.ivol();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = b.lo[0] + (int)(t % b.in[0]);
        const int64_t r = t / b.in[0];
        const int j = b.lo[1] + (int)(r % b.in[1]);
        const int k = b.lo[2] + (int)(r / b.in[1]);
        const int64_t g = b.gidx(i, j, k);
        Cons s;
        s.D = s.tau = s.S[0] = s.S[1] = s.S[2] = 0.0;
        if (excised(o, i, j, k))
        {
            store_pv(prim, b.pcs, g, load_prim(state, b.cs, g));
            store_src(src, b.rcs, t, s);
            continue;
        }
        double x, y, z;
        cell_xyz(o, i, j, k, x, y, z);
        GeoFull f;
        if (o.use_src)
            background_metric<true>(bg, x, y, z, f.g, &f);
        else
            background_metric<false>(bg, x, y, z, f.g, nullptr);
        const Cons c = load_cons(state, b.cs, g);
        Prim pr;
        if (!con2prim(o, c, f.g.gUU, pr, nullptr, nullptr))
        {
            record_error(st, 2, g);
            pr.rho = pr.p = 1.0;
            pr.v[0] = pr.v[1] = pr.v[2] = 0.0;
            pr.eps = 1.0;
        }
        else
            s = cell_sources(o, bg, x, y, z, pr, c, f);
        store_pv(prim, b.pcs, g, pr);
        store_src(src, b.rcs, t, s);
    }
}

// ----------------------------------------------------------- face pass

__device__ __forceinline__ void geo_store(double *g, int n, int cell,
                                          const Geo &v)
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

__device__ __forceinline__ void geo_load(const double *g, int n, int cell,
                                         Geo &v)
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

__device__ __forceinline__ void geo_avg_smem(const double *g, int n, int ca,
                                             int cb, Geo &v)
{
#pragma unroll
    for (int s = 0; s < 6; ++s)
    {
        v.gLL[s] = 0.5 * (g[s * n + ca] + g[s * n + cb]);
        v.gUU[s] = 0.5 * (g[(6 + s) * n + ca] + g[(6 + s) * n + cb]);
    }
    v.lapse = 0.5 * (g[12 * n + ca] + g[12 * n + cb]);
#pragma unroll
    for (int i = 0; i < 3; ++i)
        v.shift[i] = 0.5 * (g[(13 + i) * n + ca] + g[(13 + i) * n + cb]);
}

__device__ __forceinline__ PV load_pv_global(const double *__restrict__ prim,
                                             int64_t pcs, int64_t idx)
{
    PV p;
#pragma unroll
    for (int c = 0; c < 5; ++c)
        p.q[c] = __ldg(&prim[c * pcs + idx]);
    return p;
}

__device__ __forceinline__ PV load_pv_smem(const double *P, int cell)
{
    constexpr int n = kPW * kPW;
    PV p;
#pragma unroll
    for (int c = 0; c < 5; ++c)
        p.q[c] = P[c * n + cell];
    return p;
}

// Geometry of the cross-shaped (x,y) neighbourhood of a tile at plane kk.
__device__ __forceinline__ void tile_geometry(double *G, const Background &bg,
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
        Geo g;
        background_metric<false>(bg, x, y, z, g, nullptr);
        geo_store(G, n, idx, g);
    }
}

__global__ void __launch_bounds__(kTB *kTB, 2)
    k_faces(const double *__restrict__ prim, const double *__restrict__ src,
            double *__restrict__ rhs, BoxDev b, Background bg, Options o,
            double idx0, double idx1, double idx2, int zchunk)
{
    extern __shared__ double smem[];
    constexpr int nP = kPW * kPW;
    constexpr int nG = kGW * kGW;
    constexpr int nFx = kTB * kTC; // x faces: a in [0,16), b in [0,15)
    double *P = smem;                       // [5][nP]
    double *Gb = P + 5 * nP;                // [2][16][nG]
    double *Fx = Gb + 2 * kGeoFields * nG;  // [5][nFx]
    double *Fy = Fx + 5 * nFx;              // [5][nFx]

    const int a = threadIdx.x, bb = threadIdx.y;
    const int tid = bb * kTB + a;
    const int i0 = b.lo[0] + blockIdx.x * kTC;
    const int j0 = b.lo[1] + blockIdx.y * kTC;
    const int k0 = b.lo[2] + blockIdx.z * zchunk;
    const int k1 = min(k0 + zchunk - 1, b.hi[2]);
    const int ci = i0 + a, cj = j0 + bb; // this thread's cell column
    const bool col_ok = a < kTC && bb < kTC && ci <= b.hi[0] && cj <= b.hi[1];
    const int ci_c = min(ci, b.hi[0]), cj_c = min(cj, b.hi[1]);

    // own-column z window P(k-1..k+2) and the z face below k0
    PV w0, w1, w2, w3;
    Cons Flo;
    tile_geometry(Gb, bg, o, i0, j0, k0, tid);
    __syncthreads();
    Flo.D = Flo.tau = Flo.S[0] = Flo.S[1] = Flo.S[2] = 0.0;
    {
        w0 = load_pv_global(prim, b.pcs, b.gidx(ci_c, cj_c, k0 - 2));
        w1 = load_pv_global(prim, b.pcs, b.gidx(ci_c, cj_c, k0 - 1));
        w2 = load_pv_global(prim, b.pcs, b.gidx(ci_c, cj_c, k0));
        w3 = load_pv_global(prim, b.pcs, b.gidx(ci_c, cj_c, k0 + 1));
        if (col_ok)
        {
            double x, y, z;
            cell_xyz(o, ci, cj, k0 - 1, x, y, z);
            Geo gl, gr, gf;
            background_metric<false>(bg, x, y, z, gl, nullptr);
            geo_load(Gb, nG, (bb + 1) * kGW + (a + 1), gr);
            average_geo(gl, gr, gf);
            Flo = face_flux(o, w0, w1, w2, w3, gf, 2);
        }
        // shift so that w0..w3 = P(k0-1 .. k0+2) after the next load
        w0 = w1;
        w1 = w2;
        w2 = w3;
    }

    int cur = 0;
    for (int k = k0; k <= k1; ++k)
    {
        double *Gc = Gb + cur * kGeoFields * nG;
        double *Gn = Gb + (cur ^ 1) * kGeoFields * nG;
        w3 = load_pv_global(prim, b.pcs, b.gidx(ci_c, cj_c, k + 2));
        // primitive cross tile at plane k (clamped to the ghosted box)
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
                P[c * nP + idx] = __ldg(&prim[c * b.pcs + g]);
        }
        tile_geometry(Gn, bg, o, i0, j0, k + 1, tid);
        __syncthreads();

        // x face between cells (i0+a-1, i0+a) in row j0+bb
        if (bb < kTC && cj <= b.hi[1] && i0 + a - 1 <= b.hi[0])
        {
            const int row = (bb + 2) * kPW;
            Geo gf;
            geo_avg_smem(Gc, nG, (bb + 1) * kGW + a, (bb + 1) * kGW + a + 1, gf);
            const Cons f = face_flux(o, load_pv_smem(P, row + a),
                                     load_pv_smem(P, row + a + 1),
                                     load_pv_smem(P, row + a + 2),
                                     load_pv_smem(P, row + a + 3), gf, 0);
            const int fi = bb * kTB + a;
            Fx[0 * nFx + fi] = f.D;
            Fx[1 * nFx + fi] = f.S[0];
            Fx[2 * nFx + fi] = f.S[1];
            Fx[3 * nFx + fi] = f.S[2];
            Fx[4 * nFx + fi] = f.tau;
        }
        // y face between rows (j0+bb-1, j0+bb) in column i0+a
        if (a < kTC && ci <= b.hi[0] && j0 + bb - 1 <= b.hi[1])
        {
            Geo gf;
            geo_avg_smem(Gc, nG, bb * kGW + a + 1, (bb + 1) * kGW + a + 1, gf);
            const int col = a + 2;
            const Cons f = face_flux(o, load_pv_smem(P, bb * kPW + col),
                                     load_pv_smem(P, (bb + 1) * kPW + col),
                                     load_pv_smem(P, (bb + 2) * kPW + col),
                                     load_pv_smem(P, (bb + 3) * kPW + col), gf,
                                     1);
            const int fi = a * kTB + bb;
            Fy[0 * nFx + fi] = f.D;
            Fy[1 * nFx + fi] = f.S[0];
            Fy[2 * nFx + fi] = f.S[1];
            Fy[3 * nFx + fi] = f.S[2];
            Fy[4 * nFx + fi] = f.tau;
        }
        // z face at k+1/2 for this column
        Cons Fhi;
        if (col_ok)
        {
            Geo gf;
            const int cell = (bb + 1) * kGW + a + 1;
            Geo gA, gB;
            geo_load(Gc, nG, cell, gA);
            geo_load(Gn, nG, cell, gB);
            average_geo(gA, gB, gf);
            Fhi = face_flux(o, w0, w1, w2, w3, gf, 2);
        }
        __syncthreads();

        if (col_ok)
        {
            const int fxl = bb * kTB + a, fxh = bb * kTB + a + 1;
            const int fyl = a * kTB + bb, fyh = a * kTB + bb + 1;
            const int64_t ri = b.iidx(ci, cj, k);
            double out[5];
            const double fl[5] = {Flo.D, Flo.S[0], Flo.S[1], Flo.S[2], Flo.tau};
            const double fh[5] = {Fhi.D, Fhi.S[0], Fhi.S[1], Fhi.S[2], Fhi.tau};
#pragma unroll
            for (int c = 0; c < 5; ++c)
            {
                const double rx = -idx0 * (Fx[c * nFx + fxh] - Fx[c * nFx + fxl]);
                const double ry = -idx1 * (Fy[c * nFx + fyh] - Fy[c * nFx + fyl]);
                const double rz = -idx2 * (fh[c] - fl[c]);
                out[c] = ((rx + ry) + rz) + __ldg(&src[c * b.rcs + ri]);
            }
            if (excised(o, ci, cj, k))
            {
#pragma unroll
                for (int c = 0; c < 5; ++c)
                    out[c] = 0.0;
            }
#pragma unroll
            for (int c = 0; c < 5; ++c)
                rhs[c * b.rcs + ri] = out[c];
        }
        Flo = Fhi;
        w0 = w1;
        w1 = w2;
        w2 = w3;
        cur ^= 1;
        __syncthreads();
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
        if ((threadIdx.x & 31) == 0 && v)
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
__device__ __forceinline__ double cell_inverse_dt(const Options &o,
                                                  const Prim &fp,
                                                  const Geo &g,
                                                  const double inv[3])
{
    double cell = 0.0;
    if (!is_atmo(o, fp, 1.0 + 1.0e-12))
    {
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            double lo, hi;
            char_speeds(o, fp, g, d, lo, hi);
            cell += fmax(fabs(lo), fabs(hi)) * inv[d];
        }
    }
    return cell;
}

__device__ __forceinline__ void flush_max(DevStatus *st, double v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0 && v > 0.0)
        atomicMax(&st->maxinv_bits, (unsigned long long)__double_as_longlong(v));
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
// 942-969).
template <int MODE>
__global__ void __launch_bounds__(256, 2)
    k_stage(const double *un, int64_t ucs, const double *us, int64_t tcs,
            double *out, int64_t ocs, const double *__restrict__ kv,
            double *__restrict__ acc, double *__restrict__ prim,
            double *__restrict__ src, BoxDev b, Background bg, Options o,
            int stage, double dt, int cfl, double i0, double i1, double i2,
            DevStatus *st)
{
    unsigned long long cnt[4] = {0, 0, 0, 0};
    const int64_t n = b.ivol();
    const int64_t n_pad = (n + blockDim.x - 1) / blockDim.x * blockDim.x;
    const double cst = (stage == 2) ? dt : 0.5 * dt;
    const double dt6 = dt / 6.0;
    const double inv[3] = {i0, i1, i2};
    const bool prep = prim != nullptr;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_pad;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        double cell_inv = 0.0;
        if (t < n)
        {
            int i, j, k;
            interior_cell(b, t, i, j, k);
            const int64_t g = b.gidx(i, j, k);
            if (excised(o, i, j, k))
            {
                if (out != un)
                    for (int c = 0; c < kStateComps; ++c)
                        out[c * ocs + g] = un[c * ucs + g];
                if (prep)
                {
                    store_pv(prim, b.pcs, g, load_prim(un, ucs, g));
                    Cons z0;
                    z0.D = z0.tau = z0.S[0] = z0.S[1] = z0.S[2] = 0.0;
                    store_src(src, b.rcs, t, z0);
                }
            }
            else
            {
                const int comp_of[5] = {kD, kS1, kS1 + 1, kS1 + 2, kTau};
                double u[5];
#pragma unroll
                for (int c = 0; c < 5; ++c)
                {
                    const double kk = kv[c * b.rcs + t];
                    const double u0 = un[comp_of[c] * ucs + g];
                    if (MODE == 0)
                    {
                        double a = (stage == 0) ? kk : acc[c * b.rcs + t];
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
                        u[c] = 0.5 * (u0 + us[comp_of[c] * tcs + g] + dt * kk);
                }
                Cons c;
                c.D = u[0];
                c.S[0] = u[1];
                c.S[1] = u[2];
                c.S[2] = u[3];
                c.tau = u[4];
                double x, y, z;
                cell_xyz(o, i, j, k, x, y, z);
                GeoFull f;
                if (prep && o.use_src)
                    background_metric<true>(bg, x, y, z, f.g, &f);
                else
                    background_metric<false>(bg, x, y, z, f.g, nullptr);
                // recovery with atmosphere (:60-110)
                Prim pr;
                const bool ok = con2prim(o, c, f.g.gUU, pr, nullptr, nullptr);
                bool reset = !ok;
                Prim stored;
                cnt[0] += 1;
                if (ok)
                {
                    stored = pr;
                    floors(o, stored, f.g.gLL);
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
                    c = p2c(stored, f.g.gLL);
                }
                store_prim(out, ocs, g, stored);
                store_cons(out, ocs, g, c);
                if (prep || cfl)
                {
                    // con2prim of the state just written (unchanged cells:
                    // the same solve on the same input gives pr again)
                    Prim pn = pr;
                    bool okn = ok;
                    if (reset)
                        okn = con2prim(o, c, f.g.gUU, pn, nullptr, nullptr);
                    if (!okn)
                    {
                        record_error(st, cfl && !prep ? 4 : 2,
                                     cfl && !prep ? t : g);
                        pn.rho = pn.p = 1.0;
                        pn.v[0] = pn.v[1] = pn.v[2] = 0.0;
                        pn.eps = 1.0;
                    }
                    if (prep)
                    {
                        store_pv(prim, b.pcs, g, pn);
                        Cons s;
                        s.D = s.tau = s.S[0] = s.S[1] = s.S[2] = 0.0;
                        if (okn)
                            s = cell_sources(o, bg, x, y, z, pn, c, f);
                        store_src(src, b.rcs, t, s);
                    }
                    if (cfl && okn)
                    {
                        Prim fp = pn;
                        floors(o, fp, f.g.gLL);
                        cell_inv = cell_inverse_dt(o, fp, f.g, inv);
                    }
                }
            }
        }
        flush_counts(st, cnt);
        cnt[0] = cnt[1] = cnt[2] = cnt[3] = 0;
        if (cfl)
            flush_max(st, cell_inv);
    }
}

// compute_max_inverse_dt_from_fixed_background (:364-412): per cell
// con2prim + floors, skip atmosphere, sum_d max|lambda| / dx_d; block max by
// warp shuffles, one atomicMax per warp on the bit pattern.
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
        {
            int i, j, k;
            interior_cell(b, t, i, j, k);
            if (!excised(o, i, j, k))
            {
                double x, y, z;
                cell_xyz(o, i, j, k, x, y, z);
                Geo geo;
                background_metric<false>(bg, x, y, z, geo, nullptr);
                Prim pr;
                if (!con2prim(o, load_cons(state, b.cs, b.gidx(i, j, k)),
                              geo.gUU, pr, nullptr, nullptr))
                    record_error(st, 4, t);
                else
                {
                    floors(o, pr, geo.gLL);
                    cell = cell_inverse_dt(o, pr, geo, inv);
                }
            }
        }
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

int grid_for(int64_t n, int threads)
{
    int64_t blocks = (n + threads - 1) / threads;
    const int64_t cap = 148 * 32; // grid-stride beyond ~32 waves
    if (blocks > cap)
        blocks = cap;
    return (int)(blocks < 1 ? 1 : blocks);
}

} // namespace

cudaError_t configure_kernels()
{
    return cudaFuncSetAttribute(k_faces,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)face_kernel_smem_bytes());
}

size_t face_kernel_smem_bytes()
{
    return sizeof(double) *
           (5 * kPW * kPW + 2 * kGeoFields * kGW * kGW + 2 * 5 * kTB * kTC);
}

void launch_fill_ghosts(double *state, double *prim, const BoxDev &b,
                        const Background &bg, const Options &o, DevStatus *st,
                        cudaStream_t s)
{
    const int64_t nshell = b.gvol() - b.ivol();
    if (nshell <= 0)
        return;
    k_fill_ghosts<<<grid_for(nshell, 256), 256, 0, s>>>(state, prim, b, bg, o,
                                                       st, nshell);
}

void launch_cells(const double *state, double *prim, double *src,
                  const BoxDev &b, const Background &bg, const Options &o,
                  DevStatus *st, cudaStream_t s)
{
    k_cells<<<grid_for(b.ivol(), 256), 256, 0, s>>>(state, prim, src, b, bg,
                                                    o, st);
}

void launch_faces(const double *prim, const double *src, double *rhs,
                  const BoxDev &b, const Background &bg, const Options &o,
                  const double inv_dx[3], int zchunk, cudaStream_t s)
{
    const size_t smem = face_kernel_smem_bytes();
    if (zchunk < 1)
        zchunk = 1;
    dim3 grid((b.in[0] + kTC - 1) / kTC, (b.in[1] + kTC - 1) / kTC,
              (b.in[2] + zchunk - 1) / zchunk);
    dim3 block(kTB, kTB);
    k_faces<<<grid, block, smem, s>>>(prim, src, rhs, b, bg, o, inv_dx[0],
                                      inv_dx[1], inv_dx[2], zchunk);
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

void launch_stage(int mode, const double *un, int64_t ucs, const double *us,
                  int64_t tcs, double *out, int64_t ocs, const double *k,
                  double *acc, double *prim, double *src, const BoxDev &b,
                  const Background &bg, const Options &o, int stage,
                  double dt, bool cfl, const double inv_dx[3], DevStatus *st,
                  cudaStream_t s)
{
    const int grid = grid_for(b.ivol(), 256);
    const double i0 = inv_dx ? inv_dx[0] : 0.0, i1 = inv_dx ? inv_dx[1] : 0.0,
                 i2 = inv_dx ? inv_dx[2] : 0.0;
    if (mode == 0)
        k_stage<0><<<grid, 256, 0, s>>>(un, ucs, us, tcs, out, ocs, k, acc,
                                        prim, src, b, bg, o, stage, dt,
                                        cfl ? 1 : 0, i0, i1, i2, st);
    else if (mode == 1)
        k_stage<1><<<grid, 256, 0, s>>>(un, ucs, us, tcs, out, ocs, k, acc,
                                        prim, src, b, bg, o, stage, dt,
                                        cfl ? 1 : 0, i0, i1, i2, st);
    else
        k_stage<2><<<grid, 256, 0, s>>>(un, ucs, us, tcs, out, ocs, k, acc,
                                        prim, src, b, bg, o, stage, dt,
                                        cfl ? 1 : 0, i0, i1, i2, st);
}

void launch_max_inv_dt(const double *state, const BoxDev &b,
                       const Background &bg, const Options &o,
                       const double inv_dx[3], DevStatus *st, cudaStream_t s)
{
    k_max_inv_dt<<<grid_for(b.ivol(), 256), 256, 0, s>>>(
        state, b, bg, o, inv_dx[0], inv_dx[1], inv_dx[2], st);
}

void launch_residual_probe(const double *state, const BoxDev &b,
                           const Background &bg, const Options &o, int i,
                           int j, int k, double *out, cudaStream_t s)
{
    k_residual_probe<<<1, 1, 0, s>>>(state, b, bg, o, i, j, k, out);
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

} // namespace grhd
