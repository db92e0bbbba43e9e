// grhd_io.cu -- device side of the example drivers' diagnostics and of the
// KITPCHK1 checkpoint layout (grhd_io.cuh).
#include "grhd_io.cuh"

namespace grhd {

namespace {

constexpr int kDiagThreads = 256;

__device__ __forceinline__ void warp_sum_max(double v[7])
{
    for (int off = 16; off > 0; off >>= 1)
    {
        for (int q = 0; q < 3; ++q)
            v[q] += __shfl_down_sync(0xffffffffu, v[q], off);
        for (int q = 3; q < 7; ++q)
            v[q] = fmax(v[q], __shfl_down_sync(0xffffffffu, v[q], off));
    }
}

// compute_diagnostics, Main_GRHDLevelDataKerrSchildDisk.cpp:223-290; the
// per-cell quantities as the reference forms them (proper volume
// exp(log sqrt(det gamma)) dx^3, |v| = sqrt(max(0, v^2)), W).
__global__ void __launch_bounds__(kDiagThreads)
    k_diagnostics(const double *__restrict__ s, BoxDev b, Background bg,
                  Options o, double *__restrict__ partial)
{
    __shared__ double red[kDiagThreads / 32][7];
    double v[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0};
    const double vol = o.dx * o.dx * o.dx;
    const int64_t n = b.ivol();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = b.lo[0] + (int)(t % b.in[0]);
        const int64_t r = t / b.in[0];
        const int j = b.lo[1] + (int)(r % b.in[1]);
        const int k = b.lo[2] + (int)(r / b.in[1]);
        const int64_t g = b.gidx(i, j, k);
        double x, y, z;
        cell_xyz(o, i, j, k, x, y, z);
        Geo geo;
        background_metric<false>(bg, x, y, z, geo, nullptr);
        const double *G = geo.gLL;
        const double det = G[0] * G[3] * G[5] + 2.0 * G[1] * G[2] * G[4] -
                           G[0] * G[4] * G[4] - G[3] * G[2] * G[2] -
                           G[5] * G[1] * G[1];
        const double lsd =
            (det <= 0.0 || !isfinite(det)) ? 0.0 : 0.5 * log(det);
        const double pv = exp(lsd) * vol;
        const double D = s[kD * b.cs + g], tau = s[kTau * b.cs + g];
        const double rho = s[kRho * b.cs + g], p = s[kPress * b.cs + g];
        const double vel[3] = {s[kV1 * b.cs + g], s[(kV1 + 1) * b.cs + g],
                               s[(kV1 + 2) * b.cs + g]};
        v[0] += D * pv;
        v[2] += tau * pv;
        if (rho > 10.0 * o.rho_floor)
            v[1] += D * pv;
        v[3] = fmax(v[3], rho);
        v[4] = fmax(v[4], p);
        const double v2 = vsq(vel, G);
        v[5] = fmax(v[5], sqrt(fmax(0.0, v2)));
        v[6] = fmax(v[6], 1.0 / sqrt(1.0 - v2));
    }
    warp_sum_max(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int q = 0; q < 7; ++q)
            red[w][q] = v[q];
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double out[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0};
        for (int ww = 0; ww < kDiagThreads / 32; ++ww)
        {
            for (int q = 0; q < 3; ++q)
                out[q] += red[ww][q];
            for (int q = 3; q < 7; ++q)
                out[q] = fmax(out[q], red[ww][q]);
        }
        for (int q = 0; q < 7; ++q)
            partial[(int64_t)blockIdx.x * 7 + q] = out[q];
    }
}

// One thread per ghosted cell: its 11 components into / out of the
// interleaved record of `ncomp` values.
__global__ void __launch_bounds__(256)
    k_to_checkpoint(const double *__restrict__ s, BoxDev b, int ncomp,
                    double *__restrict__ out)
{
    const int64_t n = b.gvol();
    const int off = ncomp - kStateComps;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n;
         g += (int64_t)gridDim.x * blockDim.x)
    {
        double *rec = out + g * ncomp;
        for (int c = 0; c < off; ++c)
            rec[c] = 0.0;
        for (int c = 0; c < kStateComps; ++c)
            rec[off + c] = s[c * b.cs + g];
    }
}

__global__ void __launch_bounds__(256)
    k_from_checkpoint(const double *__restrict__ in, BoxDev b, int ncomp,
                      double *__restrict__ s)
{
    const int64_t n = b.gvol();
    const int off = ncomp - kStateComps;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n;
         g += (int64_t)gridDim.x * blockDim.x)
    {
        const double *rec = in + g * ncomp;
        for (int c = 0; c < kStateComps; ++c)
            s[c * b.cs + g] = rec[off + c];
    }
}

__global__ void __launch_bounds__(256)
    k_copy_region(double *__restrict__ dst, BoxDev db,
                  const double *__restrict__ src, BoxDev sb, int lo0, int lo1,
                  int lo2, int n0, int n1, int n2, int ncomp)
{
    const int64_t n = (int64_t)n0 * n1 * n2;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = lo0 + (int)(t % n0);
        const int64_t r = t / n0;
        const int j = lo1 + (int)(r % n1);
        const int k = lo2 + (int)(r / n1);
        const int64_t gd = db.gidx(i, j, k), gs = sb.gidx(i, j, k);
        for (int c = 0; c < ncomp; ++c)
            dst[c * db.cs + gd] = src[c * sb.cs + gs];
    }
}

// One region [lo, lo + n) of the ghosted box to / from a packed buffer
// [component][k][j][i] (halo messages between ranks).
template <bool PACK>
__global__ void __launch_bounds__(256)
    k_region(double *__restrict__ state, BoxDev b, double *__restrict__ buf,
             int lo0, int lo1, int lo2, int n0, int n1, int n2, int ncomp)
{
    const int64_t n = (int64_t)n0 * n1 * n2;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = lo0 + (int)(t % n0);
        const int64_t r = t / n0;
        const int j = lo1 + (int)(r % n1);
        const int k = lo2 + (int)(r / n1);
        const int64_t g = b.gidx(i, j, k);
        for (int c = 0; c < ncomp; ++c)
        {
            if (PACK)
                buf[c * n + t] = state[c * b.cs + g];
            else
                state[c * b.cs + g] = buf[c * n + t];
        }
    }
}

int grid_of(int64_t n)
{
    int64_t g = (n + 255) / 256;
    if (g > 148 * 16)
        g = 148 * 16;
    return (int)(g < 1 ? 1 : g);
}

} // namespace

int diagnostics_blocks(const BoxDev &b) { return grid_of(b.ivol()); }

void launch_diagnostics(const double *state, const BoxDev &b,
                        const Background &bg, const Options &o,
                        double *partial, cudaStream_t s)
{
    k_diagnostics<<<diagnostics_blocks(b), kDiagThreads, 0, s>>>(state, b, bg,
                                                                o, partial);
}

void launch_state_to_checkpoint(const double *state, const BoxDev &b,
                                int ncomp, double *out, cudaStream_t s)
{
    k_to_checkpoint<<<grid_of(b.gvol()), 256, 0, s>>>(state, b, ncomp, out);
}

void launch_checkpoint_to_state(const double *in, const BoxDev &b, int ncomp,
                                double *state, cudaStream_t s)
{
    k_from_checkpoint<<<grid_of(b.gvol()), 256, 0, s>>>(in, b, ncomp, state);
}

void launch_copy_region(double *dst, const BoxDev &db, const double *src,
                        const BoxDev &sb, const int lo[3], const int hi[3],
                        int ncomp, cudaStream_t s)
{
    const int n0 = hi[0] - lo[0] + 1, n1 = hi[1] - lo[1] + 1,
              n2 = hi[2] - lo[2] + 1;
    k_copy_region<<<grid_of((int64_t)n0 * n1 * n2), 256, 0, s>>>(
        dst, db, src, sb, lo[0], lo[1], lo[2], n0, n1, n2, ncomp);
}

void launch_region(bool pack, double *state, const BoxDev &b, double *buf,
                   const int lo[3], const int hi[3], int ncomp,
                   cudaStream_t s)
{
    const int n0 = hi[0] - lo[0] + 1, n1 = hi[1] - lo[1] + 1,
              n2 = hi[2] - lo[2] + 1;
    const int g = grid_of((int64_t)n0 * n1 * n2);
    if (pack)
        k_region<true><<<g, 256, 0, s>>>(state, b, buf, lo[0], lo[1], lo[2],
                                         n0, n1, n2, ncomp);
    else
        k_region<false><<<g, 256, 0, s>>>(state, b, buf, lo[0], lo[1], lo[2],
                                          n0, n1, n2, ncomp);
}

} // namespace grhd
