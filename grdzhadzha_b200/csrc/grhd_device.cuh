// grhd_device.cuh -- pointwise device physics of the fixed-background
// Valencia GRHD operator (FP64).
//
// Each function names the reference function whose result it reproduces
// (paths relative to the GRDzhadzha source tree).  The metric is evaluated
// in closed form rather than through the reference's generic symmetric
// inverse + Christoffel route; the two agree to rounding.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace grhd {

// Symmetric 3x3 packing: 00 01 02 11 12 22.
__host__ __device__ constexpr int sym(int i, int j)
{
    return (i <= j) ? (i == 0 ? j : (i == 1 ? 2 + j : 5))
                    : (j == 0 ? i : (j == 1 ? 2 + i : 5));
}

struct Prim
{
    double rho, eps, p, v[3];
};

struct Cons
{
    double D, S[3], tau;
};

// Face / cell geometry needed by con2prim, floors and the HLLE flux
// (the members of CellGeometryData, StaticMetric.hpp:19-40, minus K).
struct Geo
{
    double gLL[6], gUU[6], lapse, shift[3];
};

// Everything the static-metric sources need
// (make_static_metric_derivatives_from_adm, FixedBGMetric.hpp:31-53).
struct GeoFull
{
    Geo g;
    double K[6];
    double dlapse[3];
    double dlnsqrtg[3];
    double dgamma[3][6]; // [direction][sym(i,j)]
    double dshift[3][3]; // [i][direction] = d_direction shift^i
};

// Background constants for one evaluation time.  For the binary the
// orbital state (positions, velocities) is evaluated on the host once per
// call, as CircularBinaryPN::compute_state does per cell (:219-250).
struct Background
{
    int kind; // 0 Kerr-Schild, 1 binary PN
    double M, a;
    double m1, m2, soft2;
    double p1[3], p2[3], v1[3], v2[3];
    // positions at t + h and t - h for the volume-time source FD
    double p1p[3], p2p[3], p1m[3], p2m[3];
    double fd_h;
};

struct Options
{
    double G;           // adiabatic index
    double rho_floor, p_floor, atmo_vmax2, src_atmo_factor;
    int rec_maxit;
    double rec_tol, rec_pfloor, rec_vmax2;
    double theta;
    int use_recon, use_src, use_vol;
    double excision_radius;
    double dx, center[3];
};

// ---------------------------------------------------------------- metric

// Kerr-Schild metric of mass M, spin a at (x,y,z) relative to the hole:
// gamma_ij = delta_ij + 2 H l_i l_j, lapse (1+2H)^-1/2, shift 2H l^i/(1+2H l.l)
// (KerrSchild.hpp:64-166; derivatives as get_KS_derivs, :171-242).
template <bool FULL>
__device__ __forceinline__ void ks_metric(double M, double a, double x,
                                          double y, double z, Geo &g,
                                          GeoFull *f)
{
    const double a2 = a * a;
    const double rho = fmax(sqrt(x * x + y * y + z * z), 1.0e-6);
    const double rho2 = rho * rho;
    const double A = rho2 - a2;
    const double Q = sqrt(0.25 * A * A + a2 * z * z);
    const double r2 = 0.5 * A + Q;
    const double r = sqrt(r2);
    const double inv_r = 1.0 / r;
    const double ct = z * inv_r;
    const double Sigma = r2 + a2 * ct * ct;
    const double H = M * r / Sigma;
    const double inv_ra = 1.0 / (r2 + a2);
    const double l[3] = {(r * x + a * y) * inv_ra, (r * y - a * x) * inv_ra,
                         z * inv_r};
    const double ll = l[0] * l[0] + l[1] * l[1] + l[2] * l[2];
    const double twoH = 2.0 * H;
    const double den = 1.0 + twoH * ll;
    const double c = twoH / den; // Sherman-Morrison coefficient
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
        {
            const double ll_ij = l[i] * l[j];
            g.gLL[sym(i, j)] = (i == j ? 1.0 : 0.0) + twoH * ll_ij;
            g.gUU[sym(i, j)] = (i == j ? 1.0 : 0.0) - c * ll_ij;
        }
    g.lapse = rsqrt(1.0 + twoH);
#pragma unroll
    for (int i = 0; i < 3; ++i)
        g.shift[i] = c * l[i];
    if (!FULL)
        return;

    // derivatives of r, cos(theta), H and l (derivative index last)
    const double inv_2Q = 0.5 / Q;
    const double xs[3] = {x, y, z};
    double dr[3], dH[3], dl[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        const double drho = xs[i] / rho;
        dr[i] = 0.5 * inv_r *
                (rho * drho + inv_2Q * (drho * rho * A +
                                        (i == 2 ? 2.0 * a2 * z : 0.0)));
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        const double dct = -z * inv_r * inv_r * dr[i] + (i == 2 ? inv_r : 0.0);
        dH[i] = H * (dr[i] * inv_r -
                     2.0 / Sigma * (r * dr[i] + a2 * ct * dct));
    }
    const double nx = r * x + a * y, ny = r * y - a * x;
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        const double two_r_dr = 2.0 * r * dr[i];
        dl[0][i] = (x * dr[i] + (i == 0 ? r : 0.0) + (i == 1 ? a : 0.0) -
                    two_r_dr * nx * inv_ra) * inv_ra;
        dl[1][i] = (y * dr[i] + (i == 1 ? r : 0.0) - (i == 0 ? a : 0.0) -
                    two_r_dr * ny * inv_ra) * inv_ra;
        dl[2][i] = -z * dr[i] * inv_r * inv_r + (i == 2 ? inv_r : 0.0);
    }
    const double lapse = g.lapse;
    const double lapse2 = lapse * lapse;
    const double lapse3 = lapse2 * lapse;
    // d_k gamma_ij, d ln sqrt(gamma) = 1/2 gUU^ij d gamma_ij
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        double trace = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = i; j < 3; ++j)
            {
                const double d = 2.0 * (l[i] * l[j] * dH[k] +
                                        H * l[i] * dl[j][k] +
                                        H * l[j] * dl[i][k]);
                f->dgamma[k][sym(i, j)] = d;
                trace += (i == j ? 1.0 : 2.0) * g.gUU[sym(i, j)] * d;
            }
        f->dlnsqrtg[k] = 0.5 * trace;
        f->dlapse[k] = -lapse3 * dH[k];
    }
    // d_j shift^i with shift^i = 2 H lapse^2 l^i (KerrSchild.hpp:177-184)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            f->dshift[i][j] = 2.0 * dH[j] * lapse2 * l[i] +
                              4.0 * H * lapse * f->dlapse[j] * l[i] +
                              2.0 * H * lapse2 * dl[i][j];
    // K_ij = (D_i beta_j + D_j beta_i) / (2 lapse):
    //   sum_k gamma_kj d_i b^k + gamma_ki d_j b^k + (d_j g_ki + d_i g_kj) b^k
    //         - b^m (d_i g_mj + d_j g_mi - d_m g_ij)
    // which is the reference's Christoffel form (KerrSchild.hpp:186-207).
    const double *b = g.shift;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
        {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                s += g.gLL[sym(k, j)] * f->dshift[k][i] +
                     g.gLL[sym(k, i)] * f->dshift[k][j];
                s += b[k] * f->dgamma[k][sym(i, j)];
            }
            f->K[sym(i, j)] = s * (0.5 / lapse);
        }
    f->g = g;
}

// Softened circular-binary potentials at `pos` (add_point_potential,
// CircularBinaryPN.hpp:252-297).
__device__ __forceinline__ void pn_add_point(double mass, double soft2,
                                             const double *sp,
                                             const double *sv,
                                             const double *pos, double &U,
                                             double &dUdt, double dU[3],
                                             double V[3], double dV[3][3])
{
    double d[3];
    double r2 = soft2;
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        d[i] = pos[i] - sp[i];
        r2 += d[i] * d[i];
    }
    const double ir = 1.0 / sqrt(r2);
    const double ir3 = ir * ir * ir;
    U += mass * ir;
    dUdt += mass * (d[0] * sv[0] + d[1] * sv[1] + d[2] * sv[2]) * ir3;
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        dU[i] += -mass * d[i] * ir3;
        V[i] += mass * sv[i] * ir;
#pragma unroll
        for (int j = 0; j < 3; ++j)
            dV[i][j] += -mass * sv[i] * d[j] * ir3;
    }
}

// Scalar potential only, for the volume-time source.  The reference takes
// a central difference in time of ln sqrt(det gamma) with step h
// (FixedBGFArrayBoxFiniteVolume.hpp:616-631), which amplifies the rounding
// of U by ~1/h; the sums here are written with round-to-nearest intrinsics
// so that no multiply-add is fused and U rounds exactly as the reference's
// expression does.
__device__ __forceinline__ double pn_scalar(double m1, double m2,
                                            double soft2, const double *p1,
                                            const double *p2,
                                            const double *pos)
{
    double r1 = soft2, r2 = soft2;
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        const double d1 = __dadd_rn(pos[i], -p1[i]);
        const double d2 = __dadd_rn(pos[i], -p2[i]);
        r1 = __dadd_rn(r1, __dmul_rn(d1, d1));
        r2 = __dadd_rn(r2, __dmul_rn(d2, d2));
    }
    return __dadd_rn(__dmul_rn(m1, 1.0 / sqrt(r1)),
                     __dmul_rn(m2, 1.0 / sqrt(r2)));
}

// CircularBinaryPN::compute_metric_background, CircularBinaryPN.hpp:70-189:
// conformally flat gamma = psi delta with psi = 1 + 2U, lapse^2 =
// 1 - 2U + 2U^2 + 16 V^2/psi, shift = -4 V/psi, and
// K_ij = [psi (d_i b^j + d_j b^i) + delta_ij (b.grad psi - d_t psi)]/(2 lapse).
template <bool FULL>
__device__ __forceinline__ void pn_metric(const Background &bg, double x,
                                          double y, double z, Geo &g,
                                          GeoFull *f)
{
    const double pos[3] = {x, y, z};
    double U = 0.0, dUdt = 0.0, dU[3] = {0, 0, 0}, V[3] = {0, 0, 0};
    double dV[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    pn_add_point(bg.m1, bg.soft2, bg.p1, bg.v1, pos, U, dUdt, dU, V, dV);
    pn_add_point(bg.m2, bg.soft2, bg.p2, bg.v2, pos, U, dUdt, dU, V, dV);
    const double psi = 1.0 + 2.0 * U;
    const double ipsi = 1.0 / psi;
    const double V2 = V[0] * V[0] + V[1] * V[1] + V[2] * V[2];
    const double lapse2 = 1.0 - 2.0 * U + 2.0 * U * U + 16.0 * V2 * ipsi;
    const double lapse = sqrt(lapse2);
#pragma unroll
    for (int s = 0; s < 6; ++s)
    {
        g.gLL[s] = 0.0;
        g.gUU[s] = 0.0;
    }
    g.gLL[0] = g.gLL[3] = g.gLL[5] = psi;
    g.gUU[0] = g.gUU[3] = g.gUU[5] = ipsi;
    g.lapse = lapse;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        g.shift[i] = -4.0 * V[i] * ipsi;
    if (!FULL)
        return;
    double bgradpsi = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        const double dpsi = 2.0 * dU[d];
        bgradpsi += g.shift[d] * dpsi;
#pragma unroll
        for (int s = 0; s < 6; ++s)
            f->dgamma[d][s] = (s == 0 || s == 3 || s == 5) ? dpsi : 0.0;
        f->dlnsqrtg[d] = 1.5 * dpsi * ipsi;
        double dV2 = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c)
        {
            dV2 += 2.0 * V[c] * dV[c][d];
            f->dshift[c][d] = -4.0 * (dV[c][d] * ipsi - V[c] * dpsi * ipsi * ipsi);
        }
        const double dl2 = (-2.0 + 4.0 * U) * dU[d] +
                           16.0 * (dV2 * ipsi - V2 * dpsi * ipsi * ipsi);
        f->dlapse[d] = 0.5 * dl2 / lapse;
    }
    const double dpsidt = 2.0 * dUdt;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
        {
            double s = psi * (f->dshift[j][i] + f->dshift[i][j]);
            if (i == j)
                s += bgradpsi - dpsidt;
            f->K[sym(i, j)] = s * (0.5 / lapse);
        }
    f->g = g;
}

template <bool FULL>
__device__ __forceinline__ void background_metric(const Background &bg,
                                                  double x, double y,
                                                  double z, Geo &g,
                                                  GeoFull *f)
{
    if (bg.kind == 1)
        pn_metric<FULL>(bg, x, y, z, g, f);
    else
        ks_metric<FULL>(bg.M, bg.a, x, y, z, g, f);
}

// Coordinates<double>: cell centre (i + 1/2) dx - centre, rounded as the
// reference's separate multiply and subtract (no fused multiply-add), so
// that positions -- and everything the time-difference volume source
// amplifies -- match the reference bit for bit.
__device__ __forceinline__ void cell_xyz(const Options &o, int i, int j,
                                         int k, double &x, double &y,
                                         double &z)
{
    x = __dadd_rn(__dmul_rn(i + 0.5, o.dx), -o.center[0]);
    y = __dadd_rn(__dmul_rn(j + 0.5, o.dx), -o.center[1]);
    z = __dadd_rn(__dmul_rn(k + 0.5, o.dx), -o.center[2]);
}

__device__ __forceinline__ bool excised(const Options &o, int i, int j, int k)
{
    if (!(o.excision_radius > 0.0))
        return false;
    double x, y, z;
    cell_xyz(o, i, j, k, x, y, z);
    return sqrt(x * x + y * y + z * z) < o.excision_radius;
}

// spatial_metric_log_sqrt_det for the binary (det = psi^3),
// StaticMetric.hpp:293-302.
__device__ __forceinline__ double pn_log_sqrt_det(double psi)
{
    const double det = __dmul_rn(__dmul_rn(psi, psi), psi);
    if (det <= 0.0 || !isfinite(det))
        return 0.0;
    return 0.5 * log(det);
}

// --------------------------------------------------------- Valencia, EOS

__device__ __forceinline__ double vsq(const double v[3], const double gLL[6])
{
    return gLL[0] * v[0] * v[0] + gLL[3] * v[1] * v[1] + gLL[5] * v[2] * v[2] +
           2.0 * (gLL[1] * v[0] * v[1] + gLL[2] * v[0] * v[2] +
                  gLL[4] * v[1] * v[2]);
}

// compute_conserved, Valencia.hpp:55-73
__device__ __forceinline__ Cons p2c(const Prim &pr, const double gLL[6])
{
    Cons c;
    const double vL0 = gLL[0] * pr.v[0] + gLL[1] * pr.v[1] + gLL[2] * pr.v[2];
    const double vL1 = gLL[1] * pr.v[0] + gLL[3] * pr.v[1] + gLL[4] * pr.v[2];
    const double vL2 = gLL[2] * pr.v[0] + gLL[4] * pr.v[1] + gLL[5] * pr.v[2];
    const double v2 = vL0 * pr.v[0] + vL1 * pr.v[1] + vL2 * pr.v[2];
    const double W = 1.0 / sqrt(1.0 - v2);
    const double h = 1.0 + pr.eps + pr.p / pr.rho;
    const double rhw = pr.rho * h * W * W;
    c.D = pr.rho * W;
    c.tau = rhw - pr.p - c.D;
    c.S[0] = rhw * vL0;
    c.S[1] = rhw * vL1;
    c.S[2] = rhw * vL2;
    return c;
}

// detail::pressure_residual (+ derivative), Valencia.hpp:79-108.
__device__ __forceinline__ double c2p_residual(double p, double D,
                                               double tau, double S2,
                                               double G, double Gfac,
                                               double vmax2, double *deriv)
{
    const double e = tau + D + p;
    double v2 = S2 / (e * e);
    if (v2 > vmax2)
        v2 = vmax2;
    const double W = 1.0 / sqrt(1.0 - v2);
    const double W2 = W * W;
    if (deriv)
    {
        const double dW = -W2 * W * v2 / e;
        *deriv = D * dW + Gfac * (W2 + p * 2.0 * W * dW) - 1.0;
    }
    return D * W + Gfac * p * W2 - e;
}

// recover_primitive, Valencia.hpp:116-228 (bounded loops throughout).
__device__ __forceinline__ bool con2prim(const Options &o, const Cons &c,
                                         const double gUU[6], Prim &out,
                                         int *iters_out, double *resid_out)
{
    int iters = 0;
    double resid = 0.0;
    bool ok = false;
    if (c.D > 0.0)
    {
        const double G = o.G;
        const double Gfac = G / (G - 1.0);
        const double vmax2 = o.rec_vmax2;
        const double tol = o.rec_tol;
        const double S2 = gUU[0] * c.S[0] * c.S[0] + gUU[3] * c.S[1] * c.S[1] +
                          gUU[5] * c.S[2] * c.S[2] +
                          2.0 * (gUU[1] * c.S[0] * c.S[1] +
                                 gUU[2] * c.S[0] * c.S[2] +
                                 gUU[4] * c.S[1] * c.S[2]);
        double lower = o.rec_pfloor;
        const double f_lower =
            c2p_residual(lower, c.D, c.tau, S2, G, Gfac, vmax2, nullptr);
        bool bracket_ok = !(f_lower >= 0.0 && fabs(f_lower) > tol);
        double upper = lower;
        if (bracket_ok && f_lower < 0.0)
        {
            upper = fmax(1.0, fabs(c.tau) + c.D);
            double f_upper =
                c2p_residual(upper, c.D, c.tau, S2, G, Gfac, vmax2, nullptr);
            for (int b = 0; f_upper <= 0.0 && b < o.rec_maxit; ++b)
            {
                upper *= 2.0;
                f_upper =
                    c2p_residual(upper, c.D, c.tau, S2, G, Gfac, vmax2, nullptr);
            }
            bracket_ok = f_upper > 0.0;
        }
        if (bracket_ok)
        {
            double p = (fabs(f_lower) <= tol)
                           ? lower
                           : fmin(fmax(c.tau * (G - 1.0), lower), upper);
            double dres;
            double r = c2p_residual(p, c.D, c.tau, S2, G, Gfac, vmax2, &dres);
            for (int it = 0; it < o.rec_maxit; ++it)
            {
                iters = it + 1;
                if (fabs(r) < tol)
                    break;
                if (f_lower < 0.0)
                {
                    if (r > 0.0)
                        upper = p;
                    else
                        lower = p;
                }
                double np = p - r / dres;
                if (!isfinite(np) || np <= lower || np >= upper)
                    np = 0.5 * (lower + upper);
                p = np;
                r = c2p_residual(p, c.D, c.tau, S2, G, Gfac, vmax2, &dres);
            }
            resid = r;
            if (fabs(r) < tol)
            {
                const double e = c.tau + c.D + p;
                const double v2 = S2 / (e * e);
                if (v2 < vmax2)
                {
                    const double W = 1.0 / sqrt(1.0 - v2);
                    out.rho = c.D / W;
                    out.p = p;
                    out.eps = p / ((G - 1.0) * out.rho);
                    const double ie = 1.0 / e;
                    out.v[0] = (gUU[0] * c.S[0] + gUU[1] * c.S[1] + gUU[2] * c.S[2]) * ie;
                    out.v[1] = (gUU[1] * c.S[0] + gUU[3] * c.S[1] + gUU[4] * c.S[2]) * ie;
                    out.v[2] = (gUU[2] * c.S[0] + gUU[4] * c.S[1] + gUU[5] * c.S[2]) * ie;
                    ok = true;
                }
            }
        }
    }
    if (iters_out)
        *iters_out = iters;
    if (resid_out)
        *resid_out = resid;
    return ok;
}

// enforce_primitive_floors, Atmosphere.hpp:24-46 (eps recomputed always)
__device__ __forceinline__ void floors(const Options &o, Prim &pr,
                                       const double gLL[6])
{
    pr.rho = fmax(pr.rho, o.rho_floor);
    pr.p = fmax(pr.p, o.p_floor);
    const double v2 = vsq(pr.v, gLL);
    if (v2 >= o.atmo_vmax2)
    {
        const double s = sqrt(o.atmo_vmax2 / v2);
        pr.v[0] *= s;
        pr.v[1] *= s;
        pr.v[2] *= s;
    }
    pr.eps = pr.p / ((o.G - 1.0) * pr.rho);
}

// make_atmosphere_primitive, Atmosphere.hpp:48-60
__device__ __forceinline__ Prim atmosphere(const Options &o)
{
    Prim pr;
    pr.rho = o.rho_floor;
    pr.p = o.p_floor;
    pr.eps = pr.p / ((o.G - 1.0) * pr.rho);
    pr.v[0] = pr.v[1] = pr.v[2] = 0.0;
    return pr;
}

// is_atmosphere_primitive, FArrayBoxFiniteVolume.hpp:118-126
__device__ __forceinline__ bool is_atmo(const Options &o, const Prim &pr,
                                        double factor)
{
    const double f = fmax(1.0, factor);
    return pr.rho <= f * o.rho_floor && pr.p <= f * o.p_floor;
}

// compute_flux, Valencia.hpp:230-259
__device__ __forceinline__ Cons phys_flux(const Prim &pr, const Cons &c, int d,
                                          double lapse, const double shift[3])
{
    Cons f;
    const double tv = lapse * pr.v[d] - shift[d];
    const double ap = lapse * pr.p;
    f.D = c.D * tv;
    f.tau = c.tau * tv + ap * pr.v[d];
#pragma unroll
    for (int j = 0; j < 3; ++j)
        f.S[j] = c.S[j] * tv + (j == d ? ap : 0.0);
    return f;
}

// compute_characteristic_speeds (shifted), RiemannSolvers.hpp:23-67
__device__ __forceinline__ void char_speeds(const Options &o, const Prim &pr,
                                            const Geo &g, int d, double &lo,
                                            double &hi)
{
    const double v2 = vsq(pr.v, g.gLL);
    const double h = 1.0 + pr.eps + pr.p / pr.rho;
    const double cs2 = o.G * pr.p / (pr.rho * h);
    const double cs = sqrt(cs2);
    const double vel = pr.v[d];
    const double den = 1.0 - v2 * cs2;
    const double rad =
        (1.0 - v2) * (g.gUU[sym(d, d)] * den - vel * vel * (1.0 - cs2));
    const double root = cs * sqrt(fmax(0.0, rad));
    const double base = vel * (1.0 - cs2);
    const double iden = 1.0 / den;
    lo = g.lapse * ((base - root) * iden) - g.shift[d];
    hi = g.lapse * ((base + root) * iden) - g.shift[d];
}

// minmod / compute_limited_slope, Reconstruction.hpp:16-37
__device__ __forceinline__ double minmod2(double l, double r)
{
    if (l * r <= 0.0)
        return 0.0;
    return l > 0.0 ? fmin(l, r) : fmax(l, r);
}

__device__ __forceinline__ double limited_slope(double l, double c, double r,
                                                double theta)
{
    return minmod2(theta * (c - l), minmod2(0.5 * (r - l), theta * (r - c)));
}

// Cell primitives as stored for the stencil: rho, p, v (eps is always
// recomputed by the floors before use, Atmosphere.hpp:43-45).
struct PV
{
    double q[5]; // rho, p, v0, v1, v2
};

// One MUSCL-HLLE face flux between cells L and R (compute_muscl_hlle_flux,
// FiniteVolume.hpp:63-98, with the face geometry of average_geometry,
// FArrayBoxFiniteVolume.hpp:194-216).  LL, L, R, RR are the cells
// i-1, i, i+1, i+2 around face i+1/2.
__device__ __forceinline__ Cons face_flux(const Options &o, const PV &LL,
                                          const PV &L, const PV &R,
                                          const PV &RR, const Geo &g, int d)
{
    Prim lp, rp;
    double ql[5], qr[5];
#pragma unroll
    for (int c = 0; c < 5; ++c)
    {
        if (o.use_recon)
        {
            const double sl = limited_slope(LL.q[c], L.q[c], R.q[c], o.theta);
            const double sr = limited_slope(L.q[c], R.q[c], RR.q[c], o.theta);
            ql[c] = L.q[c] + 0.5 * sl;
            qr[c] = R.q[c] - 0.5 * sr;
        }
        else
        {
            ql[c] = L.q[c];
            qr[c] = R.q[c];
        }
    }
    lp.rho = ql[0];
    lp.p = ql[1];
    rp.rho = qr[0];
    rp.p = qr[1];
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        lp.v[i] = ql[2 + i];
        rp.v[i] = qr[2 + i];
    }
    floors(o, lp, g.gLL);
    floors(o, rp, g.gLL);
    const Cons lc = p2c(lp, g.gLL);
    const Cons rc = p2c(rp, g.gLL);
    // compute_hlle_flux, RiemannSolvers.hpp:69-118
    const Cons lf = phys_flux(lp, lc, d, g.lapse, g.shift);
    const Cons rf = phys_flux(rp, rc, d, g.lapse, g.shift);
    double llo, lhi, rlo, rhi;
    char_speeds(o, lp, g, d, llo, lhi);
    char_speeds(o, rp, g, d, rlo, rhi);
    const double sl = fmin(0.0, fmin(llo, rlo));
    const double su = fmax(0.0, fmax(lhi, rhi));
    if (sl >= 0.0)
        return lf;
    if (su <= 0.0)
        return rf;
    const double inv = 1.0 / (su - sl);
    const double ss = sl * su;
    Cons f;
    f.D = (su * lf.D - sl * rf.D + ss * (rc.D - lc.D)) * inv;
    f.tau = (su * lf.tau - sl * rf.tau + ss * (rc.tau - lc.tau)) * inv;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        f.S[i] = (su * lf.S[i] - sl * rf.S[i] + ss * (rc.S[i] - lc.S[i])) * inv;
    return f;
}

__device__ __forceinline__ void average_geo(const Geo &a, const Geo &b, Geo &g)
{
#pragma unroll
    for (int s = 0; s < 6; ++s)
    {
        g.gLL[s] = 0.5 * (a.gLL[s] + b.gLL[s]);
        g.gUU[s] = 0.5 * (a.gUU[s] + b.gUU[s]);
    }
    g.lapse = 0.5 * (a.lapse + b.lapse);
#pragma unroll
    for (int i = 0; i < 3; ++i)
        g.shift[i] = 0.5 * (a.shift[i] + b.shift[i]);
}

// compute_static_metric_source_terms, StaticMetric.hpp:193-275
__device__ __forceinline__ Cons static_sources(const Prim &pr, const Cons &c,
                                               const GeoFull &f)
{
    const Geo &g = f.g;
    const double W = 1.0 / sqrt(1.0 - vsq(pr.v, g.gLL));
    const double h = 1.0 + pr.eps + pr.p / pr.rho;
    const double rhw = pr.rho * h * W * W;
    double st[6];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
            st[sym(i, j)] = rhw * pr.v[i] * pr.v[j] + pr.p * g.gUU[sym(i, j)];
    const double E = c.D + c.tau;
    double mU[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        mU[i] = g.gUU[sym(i, 0)] * c.S[0] + g.gUU[sym(i, 1)] * c.S[1] +
                g.gUU[sym(i, 2)] * c.S[2];
    Cons F[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
        F[d] = phys_flux(pr, c, d, g.lapse, g.shift);
    Cons s;
    s.D = 0.0;
    s.tau = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        s.D -= F[d].D * f.dlnsqrtg[d];
        s.tau -= F[d].tau * f.dlnsqrtg[d];
        s.tau -= mU[d] * f.dlapse[d];
    }
    double sk = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            sk += st[sym(i, j)] * f.K[sym(i, j)];
    s.tau += g.lapse * sk;
#pragma unroll
    for (int m = 0; m < 3; ++m)
    {
        double ms = -E * f.dlapse[m];
        double sg = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                sg += st[sym(i, j)] * f.dgamma[m][sym(i, j)];
        ms += 0.5 * g.lapse * sg;
#pragma unroll
        for (int sd = 0; sd < 3; ++sd)
            ms += c.S[sd] * f.dshift[sd][m];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            ms -= F[d].S[m] * f.dlnsqrtg[d];
        s.S[m] = ms;
    }
    return s;
}

} // namespace grhd
