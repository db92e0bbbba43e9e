// grhd_kitp.cu -- device kernels of the binary-PN disk driver's source terms
// (alpha viscosity, point-mass sinks); see grhd_kitp.cuh.  One thread per
// interior cell; the stencil reads go through L1 (each cell's primitives
// are read by up to nine viscous-flux evaluations of its neighbours).
#include "grhd_kitp.cuh"

namespace grhd {

namespace {

__device__ __forceinline__ void cell_of_interior(const BoxDev &b, int64_t t,
                                                 int &i, int &j, int &k)
{
    i = b.lo[0] + (int)(t % b.in[0]);
    const int64_t r = t / b.in[0];
    j = b.lo[1] + (int)(r % b.in[1]);
    k = b.lo[2] + (int)(r / b.in[1]);
}

// sink_kernel (:557-565) summed over both bodies (:584-597)
__device__ double sink_rate(const KitpDev &k, double x, double y, double z)
{
    const double pos[3] = {x, y, z};
    double rate = 0.0;
    for (int body = 0; body < 2; ++body)
    {
        double r2 = 0.0;
        for (int d = 0; d < 3; ++d)
        {
            const double dd = pos[d] - k.body[body][d];
            r2 += dd * dd;
        }
        const double radius = k.sink_size * k.mass[body];
        double kern = 0.0;
        if (radius > 0.0 && k.sink_rate != 0.0)
            kern = exp(-pow(r2 / (radius * radius), 0.5 * k.sink_shape));
        rate += k.sink_rate * kern;
    }
    return rate;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi)
{
    return v < lo ? lo : (v > hi ? hi : v);
}

// alpha_dynamic_viscosity (:676-698)
__device__ double dynamic_viscosity(const KitpDev &k, const Options &o,
                                    double rho, double p, const double pos[3])
{
    if (k.alpha == 0.0)
        return 0.0;
    double omega2 = 0.0;
    for (int body = 0; body < 2; ++body)
    {
        double r2 = 1.0e-10;
        for (int d = 0; d < 3; ++d)
        {
            const double dd = pos[d] - k.body[body][d];
            r2 += dd * dd;
        }
        omega2 += k.mass[body] * pow(r2, -1.5);
    }
    const double cs2 = o.G * p / fmax(rho, k.rho_floor_cfg);
    return rho * k.alpha * cs2 / sqrt(fmax(omega2, 1.0e-300));
}

// viscous_flux_for_cell (:700-770) of cell (i,j,l) in direction dir:
// f[0], f[1] the S_x, S_y fluxes, f[2] the tau flux.
__device__ void viscous_flux(const double *__restrict__ s, const BoxDev &b,
                             const Options &o, const KitpDev &k, int i, int j,
                             int l, int dir, double f[3])
{
    f[0] = f[1] = f[2] = 0.0;
    const int64_t g = b.gidx(i, j, l);
    const double rho = __ldg(&s[kRho * b.cs + g]);
    if (rho <= 10.0 * k.atmo_rho_floor)
        return;
    double x, y, z;
    cell_xyz(o, i, j, l, x, y, z);
    const double pos[3] = {x, y, z};
    const double mu =
        dynamic_viscosity(k, o, rho, __ldg(&s[kPress * b.cs + g]), pos);
    if (mu == 0.0)
        return;
    const int iv[3] = {i, j, l};
    double gradv[2][2];
    for (int c = 0; c < 2; ++c)
    {
        int m[3] = {i, j, l}, q[3] = {i, j, l};
        m[c] = clampi(iv[c] - 1, b.dlo[c], b.dhi[c]);
        q[c] = clampi(iv[c] + 1, b.dlo[c], b.dhi[c]);
        const int span = q[c] - m[c];
        const double den = (span > 1 ? span : 1) * o.dx;
        const int64_t gm = b.gidx(m[0], m[1], m[2]);
        const int64_t gq = b.gidx(q[0], q[1], q[2]);
        for (int v = 0; v < 2; ++v)
            gradv[v][c] = (__ldg(&s[(kV1 + v) * b.cs + gq]) -
                           __ldg(&s[(kV1 + v) * b.cs + gm])) /
                          den;
    }
    const double divergence = gradv[0][0] + gradv[1][1];
    double tau[2][2];
    for (int a = 0; a < 2; ++a)
        for (int c = 0; c < 2; ++c)
            tau[a][c] = mu * (gradv[a][c] + gradv[c][a] +
                              (k.beta - 2.0 / 3.0) * (double)(a == c) *
                                  divergence);
    const double vx = __ldg(&s[kV1 * b.cs + g]);
    const double vy = __ldg(&s[(kV1 + 1) * b.cs + g]);
    f[0] = -tau[dir][0];
    f[1] = -tau[dir][1];
    f[2] = -tau[dir][0] * vx - tau[dir][1] * vy;
}

__global__ void __launch_bounds__(256)
    k_kitp_viscous(double *__restrict__ rhs, int64_t rcs,
                   const double *__restrict__ s, BoxDev b, Options o,
                   KitpDev k)
{
    const int64_t n = b.ivol();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        int i, j, l;
        cell_of_interior(b, t, i, j, l);
        const int iv[3] = {i, j, l};
        for (int d = 0; d < 2; ++d)
        {
            int lo[3] = {i, j, l}, hi[3] = {i, j, l};
            lo[d] = clampi(iv[d] - 1, b.dlo[d], b.dhi[d]);
            hi[d] = clampi(iv[d] + 1, b.dlo[d], b.dhi[d]);
            double fl[3], fh[3];
            viscous_flux(s, b, o, k, lo[0], lo[1], lo[2], d, fl);
            viscous_flux(s, b, o, k, hi[0], hi[1], hi[2], d, fh);
            rhs[4 * rcs + t] -= (fh[2] - fl[2]) / (2.0 * o.dx);
            rhs[1 * rcs + t] -= (fh[0] - fl[0]) / (2.0 * o.dx);
            rhs[2 * rcs + t] -= (fh[1] - fl[1]) / (2.0 * o.dx);
        }
    }
}

__global__ void __launch_bounds__(256)
    k_kitp_sink_rhs(double *__restrict__ rhs, int64_t rcs,
                    const double *__restrict__ s, BoxDev b, Options o,
                    KitpDev k)
{
    const int64_t n = b.ivol();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        int i, j, l;
        cell_of_interior(b, t, i, j, l);
        const int64_t g = b.gidx(i, j, l);
        if (s[kRho * b.cs + g] <= 10.0 * k.atmo_rho_floor)
            continue;
        double x, y, z;
        cell_xyz(o, i, j, l, x, y, z);
        const double rate = sink_rate(k, x, y, z);
        if (rate == 0.0)
            continue;
        rhs[0 * rcs + t] -= rate * s[kD * b.cs + g];
        rhs[4 * rcs + t] -= rate * s[kTau * b.cs + g];
        for (int d = 0; d < 3; ++d)
            rhs[(1 + d) * rcs + t] -= rate * s[(kS1 + d) * b.cs + g];
    }
}

__global__ void __launch_bounds__(256)
    k_kitp_sink_decay(double *__restrict__ s, BoxDev b, Options o, KitpDev k,
                      double dt)
{
    const int64_t n = b.ivol();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        int i, j, l;
        cell_of_interior(b, t, i, j, l);
        const int64_t g = b.gidx(i, j, l);
        if (s[kD * b.cs + g] <= 0.0)
            continue;
        double x, y, z;
        cell_xyz(o, i, j, l, x, y, z);
        const double rate = sink_rate(k, x, y, z);
        if (rate == 0.0)
            continue;
        const double decay = exp(-rate * dt);
        s[kD * b.cs + g] *= decay;
        s[kTau * b.cs + g] *= decay;
        for (int d = 0; d < 3; ++d)
            s[(kS1 + d) * b.cs + g] *= decay;
    }
}

// kitp_primitive (:465-520); the modes scale the midplane surface density.
__device__ Prim kitp_disk_prim(const KitpDiskDev &k, const Options &o,
                               const double pos[3], const Geo &g)
{
    Prim pr = atmosphere(o);
    const double radius = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
    if (radius <= 1.0e-12)
        return pr;
    const double phi = atan2(pos[1], pos[0]);
    const double h = fmax(k.aspect * radius, 1.0e-12);
    const double vprof = exp(-0.5 * (pos[2] / h) * (pos[2] / h));
    const double zero_sigma = o.rho_floor / k.rho_peak;
    // kitp_sigma_midplane (:408-418) with stable_logistic_cutoff (:398-406)
    const double safe_r = fmax(radius, 1.0e-12);
    const double cavity = k.cavity_factor * k.sep;
    const double cprof =
        (1.0 - k.cavity_delta) * exp(-pow(cavity / safe_r, 12.0)) +
        k.cavity_delta;
    const double arg = -2.0 * (radius - k.outer_cutoff);
    const double cut =
        arg > 700.0 ? 1.0 : (arg < -700.0 ? 0.0 : 1.0 - 1.0 / (1.0 + exp(arg)));
    double sigma = cprof * cut;
    double modes = 1.0;
    for (int m = 0; m < 4; ++m)
        modes += k.amp[m] * cos((m + 1) * phi + k.phase[m]);
    sigma *= modes;
    pr.rho = fmax(o.rho_floor, k.rho_peak * (sigma * vprof + zero_sigma));
    // binary_point_mass_potential (:444-463)
    double pot = 0.0;
    for (int b = 0; b < 2; ++b)
    {
        double r2 = k.soft * k.soft;
        for (int d = 0; d < 3; ++d)
        {
            const double dd = pos[d] - k.body[b][d];
            r2 += dd * dd;
        }
        pot -= k.mass[b] / sqrt(r2);
    }
    const double cs2 =
        fmax(o.p_floor / pr.rho, -pot / (k.mach * k.mach));
    pr.p = fmax(o.p_floor, pr.rho * cs2 / o.G);
    pr.eps = pr.p / ((o.G - 1.0) * pr.rho);
    // kitp_radial_velocity (:420-427), kitp_phi_velocity (:429-442)
    const double v0 = 1.0e-4 * k.omega_bin * k.sep;
    const double vr = v0 * sin(phi) * (radius / k.sep) *
                      exp(-pow(radius / (3.5 * k.sep), 6.0));
    const double total = k.mass[0] + k.mass[1];
    const double wg = sqrt(total / (safe_r * safe_r * safe_r) *
                           fmax(0.0, 1.0 - 1.0 / (k.mach * k.mach)));
    double vphi = 0.0;
    if (wg > 0.0)
        vphi = pow(pow(k.omega_bin, -4.0) + pow(wg, -4.0), -0.25) * safe_r;
    const double cv[3] = {vr * cos(phi) - vphi * sin(phi),
                          vr * sin(phi) + vphi * cos(phi), 0.0};
    for (int d = 0; d < 3; ++d)
        pr.v[d] = (cv[d] + g.shift[d]) / g.lapse;
    floors(o, pr, g.gLL);
    return pr;
}

// fill_kitp_level_data (:522-555): every ghosted cell.
__global__ void __launch_bounds__(256)
    k_kitp_disk_fill(double *__restrict__ s, BoxDev b, Background bg,
                     Options o, KitpDiskDev k)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
         t < b.gvol(); t += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = b.glo[0] + (int)(t % b.gn[0]);
        const int64_t r = t / b.gn[0];
        const int j = b.glo[1] + (int)(r % b.gn[1]);
        const int l = b.glo[2] + (int)(r / b.gn[1]);
        double pos[3];
        cell_xyz(o, i, j, l, pos[0], pos[1], pos[2]);
        Geo g;
        background_metric<false>(bg, pos[0], pos[1], pos[2], g, nullptr);
        const Prim pr = kitp_disk_prim(k, o, pos, g);
        s[kRho * b.cs + t] = pr.rho;
        s[kEps * b.cs + t] = pr.eps;
        s[kPress * b.cs + t] = pr.p;
        for (int d = 0; d < 3; ++d)
            s[(kV1 + d) * b.cs + t] = pr.v[d];
        const Cons c = p2c(pr, g.gLL);
        s[kD * b.cs + t] = c.D;
        s[kTau * b.cs + t] = c.tau;
        for (int d = 0; d < 3; ++d)
            s[(kS1 + d) * b.cs + t] = c.S[d];
    }
}

__global__ void __launch_bounds__(256)
    k_kitp_combine(double *__restrict__ s, BoxDev b,
                   const double *__restrict__ u1, int64_t ucs,
                   const double *__restrict__ k, int64_t rcs, double dt)
{
    const int64_t n = b.ivol();
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
    {
        int i, j, l;
        cell_of_interior(b, t, i, j, l);
        const int64_t g = b.gidx(i, j, l);
        // RHS components D, S1..3, tau are the state's first five
        for (int c = 0; c < 5; ++c)
            s[c * b.cs + g] =
                0.5 * (s[c * b.cs + g] + u1[c * ucs + g] + dt * k[c * rcs + t]);
    }
}

int blocks_for(int64_t n)
{
    int64_t g = (n + 255) / 256;
    if (g > 148 * 32)
        g = 148 * 32;
    return (int)(g < 1 ? 1 : g);
}

} // namespace

void launch_kitp_viscous_rhs(double *rhs, int64_t rcs, const double *state,
                             const BoxDev &b, const Options &o,
                             const KitpDev &k, cudaStream_t s)
{
    k_kitp_viscous<<<blocks_for(b.ivol()), 256, 0, s>>>(rhs, rcs, state, b, o,
                                                        k);
}

void launch_kitp_sink_rhs(double *rhs, int64_t rcs, const double *state,
                          const BoxDev &b, const Options &o, const KitpDev &k,
                          cudaStream_t s)
{
    k_kitp_sink_rhs<<<blocks_for(b.ivol()), 256, 0, s>>>(rhs, rcs, state, b,
                                                         o, k);
}

void launch_kitp_sink_decay(double *state, const BoxDev &b, const Options &o,
                            const KitpDev &k, double dt, cudaStream_t s)
{
    k_kitp_sink_decay<<<blocks_for(b.ivol()), 256, 0, s>>>(state, b, o, k,
                                                           dt);
}

void launch_kitp_disk_fill(double *state, const BoxDev &b,
                           const Background &bg, const Options &o,
                           const KitpDiskDev &k, cudaStream_t s)
{
    k_kitp_disk_fill<<<blocks_for(b.gvol()), 256, 0, s>>>(state, b, bg, o, k);
}

void launch_kitp_combine(double *state, const BoxDev &b, const double *u1,
                         int64_t u1_cs, const double *k, int64_t rcs,
                         double dt, cudaStream_t s)
{
    k_kitp_combine<<<blocks_for(b.ivol()), 256, 0, s>>>(state, b, u1, u1_cs, k,
                                                        rcs, dt);
}

} // namespace grhd
