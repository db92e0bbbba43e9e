// grhd_initial_data.cu -- initial data on the device:
//   * constant-specific-angular-momentum torus on the analytic background
//     (Source/Matter/GRHD/FixedBGTorus.hpp:20-409);
//   * Michel (Bondi) inflow onto a Schwarzschild hole in Kerr-Schild
//     coordinates (Tests/GRHDLevelDataMichelAccretion/
//     GRHDLevelDataMichelAccretion.cpp:183-372);
//   * a seeded relative density perturbation.
// Setup work, not part of the timed step.
#include "grhd_initial_data.cuh"

#include <cfloat>

namespace grhd {

namespace {

// ------------------------------------------------------------------ torus

// fixed_bg_torus_{azimuthal_metric, covariant_azimuthal_shift,
// coordinate_angular_velocity, eulerian_velocity...}, FixedBGTorus.hpp:44-121
struct TorusMetric
{
    double gpp, gtp, gtt;
};

__device__ __forceinline__ TorusMetric torus_metric(double x, double y,
                                                    const Geo &g)
{
    const double b[3] = {-y, x, 0.0};
    double gpp = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            gpp += g.gLL[sym(i, j)] * b[i] * b[j];
    double gtp = 0.0, bb = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        double sL = 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j)
            sL += g.gLL[sym(i, j)] * g.shift[j];
        gtp += sL * b[i];
        bb += sL * g.shift[i];
    }
    TorusMetric t;
    t.gpp = gpp;
    t.gtp = gtp;
    t.gtt = -g.lapse * g.lapse + bb;
    return t;
}

__device__ __forceinline__ double torus_omega(const TorusMetric &t,
                                              double ell)
{
    const double den = ell * t.gtp + t.gpp;
    if (fabs(den) < 1.0e-300)
        return CUDART_NAN;
    return -(ell * t.gtt + t.gtp) / den;
}

// fixed_bg_torus_potential_from_geometry, FixedBGTorus.hpp:152-187
__device__ double torus_potential_geo(double x, double y, double ell,
                                      const Geo &g, double vmax2)
{
    const TorusMetric t = torus_metric(x, y, g);
    const double om = torus_omega(t, ell);
    if (!isfinite(om))
        return CUDART_INF;
    const double b[3] = {-y, x, 0.0};
    double v[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        v[i] = (om * b[i] + g.shift[i]) / g.lapse;
    const double v2 = vsq(v, g.gLL);
    if (v2 >= vmax2 || v2 >= 1.0)
        return CUDART_INF;
    const double norm = -t.gtt - 2.0 * om * t.gtp - om * om * t.gpp;
    if (norm <= 0.0)
        return CUDART_INF;
    const double mut = -(t.gtt + om * t.gtp) / sqrt(norm);
    if (mut <= 0.0)
        return CUDART_INF;
    return log(mut);
}

__device__ double torus_potential(const Background &bg, double x, double y,
                                  double z, double ell, double vmax2)
{
    Geo g;
    background_metric<false>(bg, x, y, z, g, nullptr);
    return torus_potential_geo(x, y, ell, g, vmax2);
}

// fixed_bg_torus_radial_potential_derivative, :200-216
__device__ double torus_dWdr(const Background &bg, const TorusConfigDev &c,
                             double R, double ell)
{
    const double dr =
        fmax(c.radial_derivative_fraction * R, c.radial_derivative_min_step);
    const double rm = fmax(R - dr, 1.0e-6);
    const double wp = torus_potential(bg, R + dr, 0.0, 0.0, ell,
                                      c.max_velocity_squared);
    const double wm =
        torus_potential(bg, rm, 0.0, 0.0, ell, c.max_velocity_squared);
    if (!isfinite(wp) || !isfinite(wm))
        return CUDART_NAN;
    return (wp - wm) / (R + dr - rm);
}

// fixed_bg_torus_pressure_max_specific_angular_momentum, :218-281, and the
// surface potential of make_fixed_bg_torus_parameters, :297-304.  One
// thread: a scan of `samples` values plus a bounded bisection.
__global__ void k_torus_setup(Background bg, TorusConfigDev c,
                              double *out /* ell, surface potential, ok */)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    out[2] = 0.0;
    if (c.pressure_max_radius <= 3.0 * c.total_mass)
        return;
    const double guess =
        sqrt(c.total_mass * c.pressure_max_radius) /
        (1.0 - 2.0 * c.total_mass / c.pressure_max_radius);
    double ell = guess;
    double prev_ell = c.angular_momentum_min_factor * guess;
    double prev_d = torus_dWdr(bg, c, c.pressure_max_radius, prev_ell);
    bool done = false;
    for (int s = 1; s <= c.angular_momentum_samples && !done; ++s)
    {
        const double frac = (double)s / c.angular_momentum_samples;
        const double e = guess * (c.angular_momentum_min_factor +
                                  frac * (c.angular_momentum_max_factor -
                                          c.angular_momentum_min_factor));
        const double d = torus_dWdr(bg, c, c.pressure_max_radius, e);
        if (!isfinite(d))
            continue;
        if (isfinite(prev_d) && prev_d * d <= 0.0)
        {
            double lower = prev_ell, upper = e, f_lower = prev_d;
            ell = 0.5 * (lower + upper);
            for (int it = 0; it < c.angular_momentum_bisection_iterations;
                 ++it)
            {
                const double mid = 0.5 * (lower + upper);
                const double fm = torus_dWdr(bg, c, c.pressure_max_radius, mid);
                if (!isfinite(fm))
                {
                    ell = 0.5 * (lower + upper);
                    break;
                }
                if (fabs(fm) < c.angular_momentum_tolerance)
                {
                    ell = mid;
                    break;
                }
                if (f_lower * fm <= 0.0)
                    upper = mid;
                else
                {
                    lower = mid;
                    f_lower = fm;
                }
                ell = 0.5 * (lower + upper);
            }
            done = true;
        }
        prev_ell = e;
        prev_d = d;
    }
    out[0] = ell;
    out[1] = torus_potential(bg, c.inner_radius, 0.0, 0.0, ell,
                             c.max_velocity_squared);
    out[2] = isfinite(out[1]) ? 1.0 : 0.0;
}

// max specific enthalpy over the domain box (:306-321)
__global__ void __launch_bounds__(256)
    k_torus_max_enthalpy(BoxDev b, Background bg, Options o,
                         TorusConfigDev c, const double *setup,
                         unsigned long long *max_bits)
{
    const double ell = setup[0], ws = setup[1];
    const int64_t n = b.ivol();
    const int64_t n_pad = (n + blockDim.x - 1) / blockDim.x * blockDim.x;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_pad;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        double h = 1.0;
        if (t < n)
        {
            const int i = b.lo[0] + (int)(t % b.in[0]);
            const int64_t r = t / b.in[0];
            const int j = b.lo[1] + (int)(r % b.in[1]);
            const int k = b.lo[2] + (int)(r / b.in[1]);
            double x, y, z;
            cell_xyz(o, i, j, k, x, y, z);
            if (sqrt(x * x + y * y) >= c.inner_radius)
            {
                const double W =
                    torus_potential(bg, x, y, z, ell, c.max_velocity_squared);
                if (isfinite(W))
                    h = exp(ws - W);
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            h = fmax(h, __shfl_down_sync(0xffffffffu, h, off));
        if ((threadIdx.x & 31) == 0)
            atomicMax(max_bits, (unsigned long long)__double_as_longlong(h));
    }
}

// fixed_bg_torus_primitive + fill_fixed_bg_torus_level_data, :333-409
__global__ void __launch_bounds__(256)
    k_torus_fill(double *state, BoxDev b, Background bg, Options o,
                 TorusConfigDev c, double ell, double ws, double K)
{
    const int64_t n = b.gvol();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = b.glo[0] + (int)(t % b.gn[0]);
        const int64_t r = t / b.gn[0];
        const int j = b.glo[1] + (int)(r % b.gn[1]);
        const int k = b.glo[2] + (int)(r / b.gn[1]);
        double x, y, z;
        cell_xyz(o, i, j, k, x, y, z);
        Geo g;
        background_metric<false>(bg, x, y, z, g, nullptr);
        Prim pr = atmosphere(o);
        if (sqrt(x * x + y * y) >= c.inner_radius)
        {
            const double W =
                torus_potential_geo(x, y, ell, g, c.max_velocity_squared);
            const double h = isfinite(W) ? exp(ws - W) : 1.0;
            if (h > 1.0)
            {
                const double G = o.G;
                pr.rho = pow((h - 1.0) * (G - 1.0) / (G * K), 1.0 / (G - 1.0));
                pr.p = K * pow(pr.rho, G);
                pr.eps = pr.p / ((G - 1.0) * pr.rho);
                const TorusMetric tm = torus_metric(x, y, g);
                const double om = torus_omega(tm, ell);
                const double bvec[3] = {-y, x, 0.0};
#pragma unroll
                for (int q = 0; q < 3; ++q)
                    pr.v[q] = (om * bvec[q] + g.shift[q]) / g.lapse;
                floors(o, pr, g.gLL);
            }
        }
        const Cons cc = p2c(pr, g.gLL);
        state[kD * b.cs + t] = cc.D;
        state[(kS1 + 0) * b.cs + t] = cc.S[0];
        state[(kS1 + 1) * b.cs + t] = cc.S[1];
        state[(kS1 + 2) * b.cs + t] = cc.S[2];
        state[kTau * b.cs + t] = cc.tau;
        state[kRho * b.cs + t] = pr.rho;
        state[kEps * b.cs + t] = pr.eps;
        state[kPress * b.cs + t] = pr.p;
        state[(kV1 + 0) * b.cs + t] = pr.v[0];
        state[(kV1 + 1) * b.cs + t] = pr.v[1];
        state[(kV1 + 2) * b.cs + t] = pr.v[2];
    }
}

// ----------------------------------------------------------------- Michel

// make_constants, GRHDLevelDataMichelAccretion.cpp:196-214
struct MichelConst
{
    double K, mass_flux, bernoulli;
};

__device__ __forceinline__ double mi_enthalpy(const MichelConfigDev &c,
                                              const MichelConst &k,
                                              double rho)
{
    const double p = k.K * pow(rho, c.gamma);
    return 1.0 + c.gamma * p / ((c.gamma - 1.0) * rho);
}

__device__ __forceinline__ double mi_residual(const MichelConfigDev &c,
                                              const MichelConst &k, double r,
                                              double rho)
{
    const double f = 1.0 - 2.0 * c.mass / r;
    const double ur = k.mass_flux / (r * r * rho);
    const double h = mi_enthalpy(c, k, rho);
    return h * h * (f + ur * ur) - k.bernoulli * k.bernoulli;
}

// solve_density + bisect_density_root, :230-310 (bounded loops)
__device__ double mi_density_sweep(const MichelConfigDev &c,
                                   const MichelConst &k, double r, bool &ok)
{
    if (fabs(r - c.sonic_radius) < 1.0e-12)
        return c.sonic_density;
    const double log_min = log(c.sonic_density * 1.0e-6);
    const double log_max = log(c.sonic_density * 1.0e6);
    const int samples = 6000;
    const bool inner = r < c.sonic_radius;
    double flo = 0, fhi = 0, slo = 0, shi = 0;
    bool have_first = false, have_sel = false;
    double last_rho = exp(log_min);
    double last_v = mi_residual(c, k, r, last_rho);
    for (int i = 1; i <= samples; ++i)
    {
        const double w = (double)i / samples;
        const double rho = exp(log_min + w * (log_max - log_min));
        const double v = mi_residual(c, k, r, rho);
        if (last_v == 0.0 || v == 0.0 || last_v * v < 0.0)
        {
            const double mid = 0.5 * (last_rho + rho);
            if (!have_first)
            {
                have_first = true;
                flo = last_rho;
                fhi = rho;
            }
            if (!have_sel &&
                (inner ? mid > c.sonic_density : mid < c.sonic_density))
            {
                have_sel = true;
                slo = last_rho;
                shi = rho;
            }
        }
        last_rho = rho;
        last_v = v;
    }
    if (!have_first)
    {
        ok = false;
        return 0.0;
    }
    if (!have_sel)
    {
        slo = flo;
        shi = fhi;
    }
    double lower = slo, upper = shi;
    double fl = mi_residual(c, k, r, lower);
    const double fu = mi_residual(c, k, r, upper);
    if (fl == 0.0)
        return lower;
    if (fu == 0.0)
        return upper;
    if (fl * fu > 0.0)
    {
        ok = false;
        return 0.0;
    }
    for (int it = 0; it < 200; ++it)
    {
        const double mid = 0.5 * (lower + upper);
        const double fm = mi_residual(c, k, r, mid);
        if (fabs(fm) < c.root_tolerance ||
            fabs(upper - lower) <= c.root_tolerance * fmax(1.0e-300, fabs(mid)))
            return mid;
        if (fl * fm <= 0.0)
            upper = mid;
        else
        {
            lower = mid;
            fl = fm;
        }
    }
    return 0.5 * (lower + upper);
}

// Relative half-width of the band around the sonic radius where the
// sweep above can miss the root (new; no reference counterpart).
constexpr double kSonicBand = 5.0e-3;

// The sweep's density, or, where the sweep finds no sign change within
// kSonicBand of the sonic radius (the two density roots meet there, closer
// than one sample of the sweep), the density of the branch the sweep
// selects on that side (the root above rho_s inside r_s, below it
// outside), from the quadratic through the sonic point and that branch's
// sweep solutions at r_s (1 +- kSonicBand) and r_s (1 +- 2 kSonicBand).
// New: the reference fails at such radii.
__device__ double mi_density(const MichelConfigDev &c, const MichelConst &k,
                             double r, bool &ok)
{
    const double rho = mi_density_sweep(c, k, r, ok);
    const double x = r / c.sonic_radius - 1.0;
    if (ok || !(fabs(x) < kSonicBand))
        return rho;
    const double sg = x < 0.0 ? -1.0 : 1.0;
    bool o1 = true, o2 = true;
    const double p1 =
        mi_density_sweep(c, k, c.sonic_radius * (1.0 + sg * kSonicBand), o1);
    const double p2 = mi_density_sweep(
        c, k, c.sonic_radius * (1.0 + 2.0 * sg * kSonicBand), o2);
    ok = o1 && o2;
    const double t = fabs(x) / kSonicBand;
    return 0.5 * (t - 1.0) * (t - 2.0) * c.sonic_density -
           t * (t - 2.0) * p1 + 0.5 * t * (t - 1.0) * p2;
}

// make_point + primitive_from_radius + fill_michel_state, :312-372
__global__ void __launch_bounds__(128)
    k_michel_fill(double *state, BoxDev b, Options o, MichelConfigDev c,
                  MichelConst k, int *bad)
{
    const int64_t n = b.gvol();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = b.glo[0] + (int)(t % b.gn[0]);
        const int64_t rr = t / b.gn[0];
        const int j = b.glo[1] + (int)(rr % b.gn[1]);
        const int kk = b.glo[2] + (int)(rr / b.gn[1]);
        double x, y, z;
        cell_xyz(o, i, j, kk, x, y, z);
        const double radius = sqrt(x * x + y * y + z * z);
        Geo g;
        ks_metric<double, false>(c.mass, 0.0, x, y, z, g, nullptr);
        Prim pr;
        if (radius < c.atmosphere_radius)
            pr = atmosphere(o);
        else
        {
            bool ok = (1.0 - 2.0 * c.mass / radius) > 0.0;
            const double rho = ok ? mi_density(c, k, radius, ok) : 0.0;
            // Michel velocity on the +x axis in Kerr-Schild coordinates
            Geo ga;
            ks_metric<double, false>(c.mass, 0.0, radius, 0.0, 0.0, ga, nullptr);
            double W = 0.0, vr = 0.0;
            if (ok)
            {
                const double f = 1.0 - 2.0 * c.mass / radius;
                const double ur = k.mass_flux / (radius * radius * rho);
                double sL0 = ga.gLL[0] * ga.shift[0] + ga.gLL[1] * ga.shift[1] +
                             ga.gLL[2] * ga.shift[2];
                double s2 = 0.0;
#pragma unroll
                for (int q = 0; q < 3; ++q)
                {
                    double sLq = 0.0;
#pragma unroll
                    for (int m = 0; m < 3; ++m)
                        sLq += ga.gLL[sym(q, m)] * ga.shift[m];
                    s2 += sLq * ga.shift[q];
                }
                const double gtt = -ga.lapse * ga.lapse + s2;
                const double u_t = -sqrt(f + ur * ur);
                const double ut = (u_t - sL0 * ur) / gtt;
                W = ga.lapse * ut;
                ok = (W > 1.0) && isfinite(W);
                vr = ur / W + ga.shift[0] / ga.lapse;
            }
            if (!ok)
            {
                atomicExch(bad, 1);
                pr = atmosphere(o);
            }
            else
            {
                pr.rho = rho;
                pr.p = k.K * pow(rho, c.gamma);
                pr.eps = pr.p / ((c.gamma - 1.0) * rho);
                pr.v[0] = vr * x / radius;
                pr.v[1] = vr * y / radius;
                pr.v[2] = vr * z / radius;
                floors(o, pr, g.gLL);
            }
        }
        const Cons cc = p2c(pr, g.gLL);
        state[kD * b.cs + t] = cc.D;
        state[(kS1 + 0) * b.cs + t] = cc.S[0];
        state[(kS1 + 1) * b.cs + t] = cc.S[1];
        state[(kS1 + 2) * b.cs + t] = cc.S[2];
        state[kTau * b.cs + t] = cc.tau;
        state[kRho * b.cs + t] = pr.rho;
        state[kEps * b.cs + t] = pr.eps;
        state[kPress * b.cs + t] = pr.p;
        state[(kV1 + 0) * b.cs + t] = pr.v[0];
        state[(kV1 + 1) * b.cs + t] = pr.v[1];
        state[(kV1 + 2) * b.cs + t] = pr.v[2];
    }
}

// -------------------------------------------------------- perturbation

__device__ __forceinline__ uint64_t splitmix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// rho *= 1 + A u, u uniform in [-1, 1) from a counter-based hash of
// (seed, cell index in the level); pressure and velocity kept, eps and the
// conserved variables recomputed with the cell metric.
__global__ void __launch_bounds__(256)
    k_perturb_density(double *state, BoxDev b, Background bg, Options o,
                      double amp, uint64_t seed)
{
    const int64_t n = b.gvol();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = b.glo[0] + (int)(t % b.gn[0]);
        const int64_t r = t / b.gn[0];
        const int j = b.glo[1] + (int)(r % b.gn[1]);
        const int k = b.glo[2] + (int)(r / b.gn[1]);
        const uint64_t key =
            ((uint64_t)(uint32_t)(i + (1 << 20)) << 42) ^
            ((uint64_t)(uint32_t)(j + (1 << 20)) << 21) ^
            (uint64_t)(uint32_t)(k + (1 << 20));
        const uint64_t h = splitmix64(seed ^ splitmix64(key));
        const double u = (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
        Prim pr;
        pr.rho = state[kRho * b.cs + t] * (1.0 + amp * u);
        pr.p = state[kPress * b.cs + t];
        pr.v[0] = state[(kV1 + 0) * b.cs + t];
        pr.v[1] = state[(kV1 + 1) * b.cs + t];
        pr.v[2] = state[(kV1 + 2) * b.cs + t];
        pr.eps = pr.p / ((o.G - 1.0) * pr.rho);
        double x, y, z;
        cell_xyz(o, i, j, k, x, y, z);
        Geo g;
        background_metric<false>(bg, x, y, z, g, nullptr);
        const Cons cc = p2c(pr, g.gLL);
        state[kD * b.cs + t] = cc.D;
        state[(kS1 + 0) * b.cs + t] = cc.S[0];
        state[(kS1 + 1) * b.cs + t] = cc.S[1];
        state[(kS1 + 2) * b.cs + t] = cc.S[2];
        state[kTau * b.cs + t] = cc.tau;
        state[kRho * b.cs + t] = pr.rho;
        state[kEps * b.cs + t] = pr.eps;
    }
}

int grid_of(int64_t n, int threads)
{
    int64_t blocks = (n + threads - 1) / threads;
    if (blocks > 148 * 32)
        blocks = 148 * 32;
    return (int)(blocks < 1 ? 1 : blocks);
}

} // namespace

cudaError_t torus_initial_data(double *state, const BoxDev &b,
                               const Background &bg, const Options &o,
                               const TorusConfigDev &c, double *scratch4,
                               double out[4], cudaStream_t s)
{
    // scratch4: device doubles [ell, ws, ok, max_enthalpy bits]
    k_torus_setup<<<1, 1, 0, s>>>(bg, c, scratch4);
    cudaMemsetAsync(scratch4 + 3, 0, sizeof(double), s);
    k_torus_max_enthalpy<<<grid_of(b.ivol(), 256), 256, 0, s>>>(
        b, bg, o, c, scratch4, (unsigned long long *)(scratch4 + 3));
    double h[4];
    cudaError_t e = cudaMemcpyAsync(h, scratch4, 4 * sizeof(double),
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return e;
    out[0] = h[0];
    out[1] = h[1];
    out[3] = (h[3] > 1.0) ? h[3] : 1.0;
    if (h[2] != 1.0 || !(out[3] > 1.0))
    {
        out[2] = 0.0;
        return cudaErrorInvalidValue;
    }
    const double G = o.G;
    out[2] = (out[3] - 1.0) * (G - 1.0) / (G * pow(c.rho_peak, G - 1.0));
    k_torus_fill<<<grid_of(b.gvol(), 256), 256, 0, s>>>(state, b, bg, o, c,
                                                       out[0], out[1], out[2]);
    return cudaGetLastError();
}

cudaError_t michel_initial_data(double *state, const BoxDev &b,
                                const Options &o, const MichelConfigDev &c,
                                int *bad_flag, cudaStream_t s)
{
    MichelConst k;
    // make_constants, GRHDLevelDataMichelAccretion.cpp:196-214
    const double cs2 = c.mass / (2.0 * c.sonic_radius - 3.0 * c.mass);
    const double ur_s = -sqrt(c.mass / (2.0 * c.sonic_radius));
    const double q = cs2 / (c.gamma - cs2 * c.gamma / (c.gamma - 1.0));
    k.K = q / pow(c.sonic_density, c.gamma - 1.0);
    const double ps = k.K * pow(c.sonic_density, c.gamma);
    const double hc = 1.0 + c.gamma * ps / ((c.gamma - 1.0) * c.sonic_density);
    const double fc = 1.0 - 2.0 * c.mass / c.sonic_radius;
    k.bernoulli = hc * sqrt(fc + ur_s * ur_s);
    k.mass_flux = c.sonic_radius * c.sonic_radius * c.sonic_density * ur_s;
    cudaMemsetAsync(bad_flag, 0, sizeof(int), s);
    k_michel_fill<<<grid_of(b.gvol(), 128), 128, 0, s>>>(state, b, o, c, k,
                                                        bad_flag);
    return cudaGetLastError();
}

cudaError_t perturb_density(double *state, const BoxDev &b,
                            const Background &bg, const Options &o,
                            double amplitude, uint64_t seed, cudaStream_t s)
{
    k_perturb_density<<<grid_of(b.gvol(), 256), 256, 0, s>>>(
        state, b, bg, o, amplitude, seed);
    return cudaGetLastError();
}

} // namespace grhd
