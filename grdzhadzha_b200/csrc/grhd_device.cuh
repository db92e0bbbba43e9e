// grhd_device.cuh -- pointwise device physics of the fixed-background
// Valencia GRHD operator, templated on the arithmetic type T.
//
// T = double is the FP64 path (parity with the reference); T = float is the
// arithmetic of the mixed path's reconstruction, Riemann solver, metric and
// sources.  The con2prim root solve is FP64 in both paths.  Each function
// names the reference function whose result it reproduces (paths relative
// to the GRDzhadzha source tree).  The metric is evaluated in closed form
// rather than through the reference's generic symmetric inverse +
// Christoffel route; the two agree to rounding.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// Pointwise functions of the FP64 path are also host-callable (the host
// test of the adjoint's reverse-mode functions runs them on the CPU); the
// FP32 overloads use device intrinsics and stay device-only.
#define GRHD_HD __host__ __device__

namespace grhd {

// Symmetric 3x3 packing: 00 01 02 11 12 22.
__host__ __device__ constexpr int sym(int i, int j)
{
    return (i <= j) ? (i == 0 ? j : (i == 1 ? 2 + j : 5))
                    : (j == 0 ? i : (j == 1 ? 2 + i : 5));
}

// ------------------------------------------------------------- arithmetic
// FP64 on the device: division, reciprocal and square root from the
// hardware's approximate reciprocal (square root) refined by Newton-Raphson
// steps, within about one ulp of the IEEE result (checked against it by
// grhd_eval_arith's test) and without the IEEE operations' special-case
// branches, which the face and stage kernels pay on every call.  Their
// domain is that of the quantities they are used on -- densities,
// enthalpies, metric functions, speed differences and squared norms:
// normal numbers up to 2^1021, and 0 for the square root; a zero divisor
// or a quotient that overflows gives NaN (not +-inf), and a subnormal
// operand is flushed to zero.  The oracle and the host keep IEEE
// division, as does the binary's volume-time source (pn_scalar), whose
// time difference is rounded as the reference's.  FP32: the SFU
// reciprocal / reciprocal square root (a few ulp), which is what makes the
// FP32 path cheap.

#ifdef __CUDA_ARCH__
// 1/a: the approximate reciprocal (rcp.approx.ftz.f64, about 20 correct
// bits) and two Newton-Raphson steps y <- y + y (1 - a y), each of which
// squares the relative error.
__device__ __forceinline__ double rcp_newton(double a)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
#pragma unroll
    for (int it = 0; it < 2; ++it)
        y = fma(y, fma(-a, y, 1.0), y);
    return y;
}
#endif

// a / b: the quotient q = a y with y ~ 1/b, corrected once by its exact
// residual r = a - b q (one fused multiply-add): q + r y (Markstein's
// correction, IBM J. Res. Dev. 34 (1990) 111-119).
GRHD_HD __forceinline__ double div_(double a, double b)
{
#ifdef __CUDA_ARCH__
    const double y = rcp_newton(b);
    const double q = a * y;
    return fma(fma(-b, q, a), y, q);
#else
    return a / b;
#endif
}
__device__ __forceinline__ float div_(float a, float b)
{
    return __fdividef(a, b);
}
GRHD_HD __forceinline__ double rcp_(double a)
{
#ifdef __CUDA_ARCH__
    const double y = rcp_newton(a);
    return fma(y, fma(-a, y, 1.0), y);
#else
    return 1.0 / a;
#endif
}
__device__ __forceinline__ float rcp_(float a) { return __fdividef(1.0f, a); }
// FP64 reciprocal square root: the hardware's approximate rsqrt
// (rsqrt.approx.ftz.f64, a few ulp of FP32 accuracy) refined by two
// Newton-Raphson steps y <- y + y (1 - a y^2) / 2, each of which squares
// the relative error; the result is within a few ulp of 1/sqrt(a), for
// one MUFU operation and eight FP64 ones instead of an IEEE square root
// followed by an IEEE division.  a > 0 (the callers pass 1 - v^2 with v^2
// below its cap, or a squared norm).
GRHD_HD __forceinline__ double rsqrt_(double a)
{
#ifdef __CUDA_ARCH__
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
#pragma unroll
    for (int it = 0; it < 2; ++it)
    {
        const double e = fma(-(a * y), y, 1.0);
        y = fma(0.5 * y, e, y);
    }
    return y;
#else
    return 1.0 / sqrt(a);
#endif
}
__device__ __forceinline__ float rsqrt_(float a) { return rsqrtf(a); }
// sqrt(a) = a / sqrt(a): s = a y with y ~ 1/sqrt(a) (rsqrt_), corrected by
// one Newton step on s^2 = a, s + (a - s^2) y / 2; a = 0 returns 0 and a
// negative a NaN.
GRHD_HD __forceinline__ double sqrt_(double a)
{
#ifdef __CUDA_ARCH__
    const double y = rsqrt_(a);
    const double s = a * y;
    const double r = fma(0.5 * y, fma(-s, s, a), s);
    return a > 0.0 ? r
                   : (a == 0.0 ? a : __longlong_as_double(0x7ff8000000000000ll));
#else
    return sqrt(a);
#endif
}
__device__ __forceinline__ float sqrt_(float a) { return sqrtf(a); }
GRHD_HD __forceinline__ double max_(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float max_(float a, float b) { return fmaxf(a, b); }
GRHD_HD __forceinline__ double min_(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float min_(float a, float b) { return fminf(a, b); }
GRHD_HD __forceinline__ double abs_(double a) { return fabs(a); }
__device__ __forceinline__ float abs_(float a) { return fabsf(a); }
// the lapse (1 + 2H)^-1/2 of the Kerr-Schild metric
GRHD_HD __forceinline__ double lapse_rsqrt(double a)
{
#ifdef __CUDA_ARCH__
    return rsqrt(a);
#else
    return 1.0 / sqrt(a);
#endif
}
__device__ __forceinline__ float lapse_rsqrt(float a) { return rsqrtf(a); }

template <typename T> struct PrimT
{
    T rho, eps, p, v[3];
};

template <typename T> struct ConsT
{
    T D, S[3], tau;
};

// Face / cell geometry needed by con2prim, floors and the HLLE flux
// (the members of CellGeometryData, StaticMetric.hpp:19-40, minus K).
template <typename T> struct GeoT
{
    T gLL[6], gUU[6], lapse, shift[3];
};

// Everything the static-metric sources need
// (make_static_metric_derivatives_from_adm, FixedBGMetric.hpp:31-53).
template <typename T> struct GeoFullT
{
    GeoT<T> g;
    T K[6];
    T dlapse[3];
    T dlnsqrtg[3];
    T dgamma[3][6]; // [direction][sym(i,j)]
    T dshift[3][3]; // [i][direction] = d_direction shift^i
};

// Cell primitives as stored for the stencil: rho, p, v (eps is always
// recomputed by the floors before use, Atmosphere.hpp:43-45).
template <typename T> struct PVT
{
    T q[5]; // rho, p, v0, v1, v2
};

using Prim = PrimT<double>;
using Cons = ConsT<double>;
using Geo = GeoT<double>;
using GeoFull = GeoFullT<double>;
using PV = PVT<double>;

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
    double accretion_radius; // > 0: Mdot through the sphere r < R (new)
    double dx, center[3];
};

// ---------------------------------------------------------------- metric

// Kerr-Schild metric of mass M, spin a at (x,y,z) relative to the hole:
// gamma_ij = delta_ij + 2 H l_i l_j, lapse (1+2H)^-1/2,
// shift^i = 2H l^i/(1 + 2H l.l), gamma^ij by Sherman-Morrison
// (KerrSchild.hpp:64-166; derivatives as get_KS_derivs, :171-242).
template <typename T, bool FULL>
GRHD_HD __forceinline__ void ks_metric(T M, T a, T x, T y, T z,
                                          GeoT<T> &g, GeoFullT<T> *f)
{
    const T a2 = a * a;
    const T rho = max_(sqrt_(x * x + y * y + z * z), T(1.0e-6));
    const T rho2 = rho * rho;
    const T A = rho2 - a2;
    const T Q = sqrt_(T(0.25) * A * A + a2 * z * z);
    const T r2 = T(0.5) * A + Q;
    const T r = sqrt_(r2);
    const T inv_r = rcp_(r);
    const T ct = z * inv_r;
    const T Sigma = r2 + a2 * ct * ct;
    const T H = div_(M * r, Sigma);
    const T inv_ra = rcp_(r2 + a2);
    const T l[3] = {(r * x + a * y) * inv_ra, (r * y - a * x) * inv_ra,
                    z * inv_r};
    const T ll = l[0] * l[0] + l[1] * l[1] + l[2] * l[2];
    const T twoH = T(2) * H;
    const T den = T(1) + twoH * ll;
    const T c = div_(twoH, den); // Sherman-Morrison coefficient
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
        {
            const T ll_ij = l[i] * l[j];
            g.gLL[sym(i, j)] = (i == j ? T(1) : T(0)) + twoH * ll_ij;
            g.gUU[sym(i, j)] = (i == j ? T(1) : T(0)) - c * ll_ij;
        }
    g.lapse = lapse_rsqrt(T(1) + twoH);
#pragma unroll
    for (int i = 0; i < 3; ++i)
        g.shift[i] = c * l[i];
    if (!FULL)
        return;

    // derivatives of r, cos(theta), H and l (derivative index last)
    const T inv_2Q = div_(T(0.5), Q);
    const T xs[3] = {x, y, z};
    T dr[3], dH[3], dl[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        const T drho = div_(xs[i], rho);
        dr[i] = T(0.5) * inv_r *
                (rho * drho + inv_2Q * (drho * rho * A +
                                        (i == 2 ? T(2) * a2 * z : T(0))));
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        const T dct = -z * inv_r * inv_r * dr[i] + (i == 2 ? inv_r : T(0));
        dH[i] = H * (dr[i] * inv_r -
                     div_(T(2), Sigma) * (r * dr[i] + a2 * ct * dct));
    }
    const T nx = r * x + a * y, ny = r * y - a * x;
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        const T two_r_dr = T(2) * r * dr[i];
        dl[0][i] = (x * dr[i] + (i == 0 ? r : T(0)) + (i == 1 ? a : T(0)) -
                    two_r_dr * nx * inv_ra) * inv_ra;
        dl[1][i] = (y * dr[i] + (i == 1 ? r : T(0)) - (i == 0 ? a : T(0)) -
                    two_r_dr * ny * inv_ra) * inv_ra;
        dl[2][i] = -z * dr[i] * inv_r * inv_r + (i == 2 ? inv_r : T(0));
    }
    const T lapse = g.lapse;
    const T lapse2 = lapse * lapse;
    const T lapse3 = lapse2 * lapse;
    // d_k gamma_ij, d ln sqrt(gamma) = 1/2 gUU^ij d gamma_ij
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        T trace = T(0);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = i; j < 3; ++j)
            {
                const T d = T(2) * (l[i] * l[j] * dH[k] + H * l[i] * dl[j][k] +
                                    H * l[j] * dl[i][k]);
                f->dgamma[k][sym(i, j)] = d;
                trace += (i == j ? T(1) : T(2)) * g.gUU[sym(i, j)] * d;
            }
        f->dlnsqrtg[k] = T(0.5) * trace;
        f->dlapse[k] = -lapse3 * dH[k];
    }
    // d_j shift^i with shift^i = 2 H lapse^2 l^i (KerrSchild.hpp:177-184)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            f->dshift[i][j] = T(2) * dH[j] * lapse2 * l[i] +
                              T(4) * H * lapse * f->dlapse[j] * l[i] +
                              T(2) * H * lapse2 * dl[i][j];
    // K_ij = (D_i beta_j + D_j beta_i) / (2 lapse), which for a static
    // metric is the Lie derivative of gamma along beta over 2 lapse:
    //   sum_k gamma_kj d_i b^k + gamma_ki d_j b^k + b^k d_k gamma_ij
    // (the reference's Christoffel form, KerrSchild.hpp:186-207, reduces
    // to this identically).
    const T *b = g.shift;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
        {
            T s = T(0);
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                s += g.gLL[sym(k, j)] * f->dshift[k][i] +
                     g.gLL[sym(k, i)] * f->dshift[k][j];
                s += b[k] * f->dgamma[k][sym(i, j)];
            }
            f->K[sym(i, j)] = s * div_(T(0.5), lapse);
        }
    f->g = g;
}

// Softened circular-binary potentials at `pos` (add_point_potential,
// CircularBinaryPN.hpp:252-297).
template <typename T>
__device__ __forceinline__ void pn_add_point(T mass, T soft2, const double *sp,
                                             const double *sv, const T *pos,
                                             T &U, T &dUdt, T dU[3], T V[3],
                                             T dV[3][3])
{
    T d[3];
    T r2 = soft2;
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        d[i] = pos[i] - T(sp[i]);
        r2 += d[i] * d[i];
    }
    const T ir = rsqrt_(r2);
    const T ir3 = ir * ir * ir;
    U += mass * ir;
    dUdt += mass * (d[0] * T(sv[0]) + d[1] * T(sv[1]) + d[2] * T(sv[2])) * ir3;
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        dU[i] += -mass * d[i] * ir3;
        V[i] += mass * T(sv[i]) * ir;
#pragma unroll
        for (int j = 0; j < 3; ++j)
            dV[i][j] += -mass * T(sv[i]) * d[j] * ir3;
    }
}

// Scalar potential only, for the volume-time source (FP64 in both paths).
// The reference takes a central difference in time of ln sqrt(det gamma)
// with step h (FixedBGFArrayBoxFiniteVolume.hpp:616-631), which amplifies
// the rounding of U by ~1/h; the sums here are written with
// round-to-nearest intrinsics so that no multiply-add is fused and U rounds
// exactly as the reference's expression does.
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
template <typename T, bool FULL>
__device__ __forceinline__ void pn_metric(const Background &bg, T x, T y, T z,
                                          GeoT<T> &g, GeoFullT<T> *f)
{
    const T pos[3] = {x, y, z};
    T U = T(0), dUdt = T(0), dU[3] = {T(0), T(0), T(0)},
      V[3] = {T(0), T(0), T(0)};
    T dV[3][3] = {{T(0), T(0), T(0)}, {T(0), T(0), T(0)}, {T(0), T(0), T(0)}};
    pn_add_point<T>(T(bg.m1), T(bg.soft2), bg.p1, bg.v1, pos, U, dUdt, dU, V,
                    dV);
    pn_add_point<T>(T(bg.m2), T(bg.soft2), bg.p2, bg.v2, pos, U, dUdt, dU, V,
                    dV);
    const T psi = T(1) + T(2) * U;
    const T ipsi = rcp_(psi);
    const T V2 = V[0] * V[0] + V[1] * V[1] + V[2] * V[2];
    const T lapse2 = T(1) - T(2) * U + T(2) * U * U + T(16) * V2 * ipsi;
    const T lapse = sqrt_(lapse2);
#pragma unroll
    for (int s = 0; s < 6; ++s)
    {
        g.gLL[s] = T(0);
        g.gUU[s] = T(0);
    }
    g.gLL[0] = g.gLL[3] = g.gLL[5] = psi;
    g.gUU[0] = g.gUU[3] = g.gUU[5] = ipsi;
    g.lapse = lapse;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        g.shift[i] = T(-4) * V[i] * ipsi;
    if (!FULL)
        return;
    T bgradpsi = T(0);
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        const T dpsi = T(2) * dU[d];
        bgradpsi += g.shift[d] * dpsi;
#pragma unroll
        for (int s = 0; s < 6; ++s)
            f->dgamma[d][s] = (s == 0 || s == 3 || s == 5) ? dpsi : T(0);
        f->dlnsqrtg[d] = T(1.5) * dpsi * ipsi;
        T dV2 = T(0);
#pragma unroll
        for (int c = 0; c < 3; ++c)
        {
            dV2 += T(2) * V[c] * dV[c][d];
            f->dshift[c][d] =
                T(-4) * (dV[c][d] * ipsi - V[c] * dpsi * ipsi * ipsi);
        }
        const T dl2 = (T(-2) + T(4) * U) * dU[d] +
                      T(16) * (dV2 * ipsi - V2 * dpsi * ipsi * ipsi);
        f->dlapse[d] = div_(T(0.5) * dl2, lapse);
    }
    const T dpsidt = T(2) * dUdt;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
        {
            T s = psi * (f->dshift[j][i] + f->dshift[i][j]);
            if (i == j)
                s += bgradpsi - dpsidt;
            f->K[sym(i, j)] = s * div_(T(0.5), lapse);
        }
    f->g = g;
}

// BGK: the background kind when known at compile time (0 Kerr-Schild,
// 1 binary PN), -1 to read it from bg.kind.
template <bool FULL, int BGK = -1>
__device__ __forceinline__ void background_metric(const Background &bg,
                                                  double x, double y,
                                                  double z, Geo &g,
                                                  GeoFull *f)
{
    if (BGK == 1 || (BGK < 0 && bg.kind == 1))
        pn_metric<double, FULL>(bg, x, y, z, g, f);
    else
        ks_metric<double, FULL>(bg.M, bg.a, x, y, z, g, f);
}

template <typename A, typename B>
GRHD_HD __forceinline__ void convert_geo(const GeoT<A> &s, GeoT<B> &d)
{
#pragma unroll
    for (int q = 0; q < 6; ++q)
    {
        d.gLL[q] = B(s.gLL[q]);
        d.gUU[q] = B(s.gUU[q]);
    }
    d.lapse = B(s.lapse);
#pragma unroll
    for (int q = 0; q < 3; ++q)
        d.shift[q] = B(s.shift[q]);
}

// FP64 Kerr-Schild geometry rounded to FP32 (mixed path, r < 3M).
template <bool FULL>
__device__ __noinline__ void ks_metric_fp64_to_fp32(double M, double a,
                                                    double x, double y,
                                                    double z, GeoT<float> &g,
                                                    GeoFullT<float> *f)
{
    GeoFull fd;
    ks_metric<double, FULL>(M, a, x, y, z, fd.g, FULL ? &fd : nullptr);
    convert_geo(fd.g, g);
    if (FULL)
    {
#pragma unroll
        for (int q = 0; q < 6; ++q)
            f->K[q] = float(fd.K[q]);
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            f->dlapse[d] = float(fd.dlapse[d]);
            f->dlnsqrtg[d] = float(fd.dlnsqrtg[d]);
#pragma unroll
            for (int q = 0; q < 6; ++q)
                f->dgamma[d][q] = float(fd.dgamma[d][q]);
#pragma unroll
            for (int q = 0; q < 3; ++q)
                f->dshift[d][q] = float(fd.dshift[d][q]);
        }
        f->g = g;
    }
}

// Mixed-path geometry: FP32 closed forms, except within three gravitational
// radii of a Kerr-Schild hole where the metric (and so its determinant and
// inverse) is evaluated in FP64 -- there r^2 = (rho^2 - a^2)/2 + ... and
// 1 + 2H lose too many FP32 digits.
template <bool FULL, int BGK = -1>
__device__ __forceinline__ void background_metric_mixed(const Background &bg,
                                                        double x, double y,
                                                        double z,
                                                        GeoT<float> &g,
                                                        GeoFullT<float> *f)
{
    if (BGK == 1 || (BGK < 0 && bg.kind == 1))
        pn_metric<float, FULL>(bg, float(x), float(y), float(z), g, f);
    else if (x * x + y * y + z * z < 9.0 * bg.M * bg.M)
        ks_metric_fp64_to_fp32<FULL>(bg.M, bg.a, x, y, z, g, f);
    else
        ks_metric<float, FULL>(float(bg.M), float(bg.a), float(x), float(y),
                               float(z), g, f);
}

template <typename T, bool FULL, int BGK = -1>
__device__ __forceinline__ void metric_T(const Background &bg, double x,
                                         double y, double z, GeoT<T> &g,
                                         GeoFullT<T> *f)
{
    if constexpr (sizeof(T) == sizeof(double))
        background_metric<FULL, BGK>(bg, x, y, z, g, f);
    else
        background_metric_mixed<FULL, BGK>(bg, x, y, z, g, f);
}

// Coordinates<double>: cell centre (i + 1/2) dx - centre, rounded as the
// reference's separate multiply and subtract (no fused multiply-add), so
// that positions -- and everything the time-difference volume source
// amplifies -- match the reference bit for bit.
GRHD_HD __forceinline__ void cell_xyz(const Options &o, int i, int j,
                                         int k, double &x, double &y,
                                         double &z)
{
#ifdef __CUDA_ARCH__
    x = __dadd_rn(__dmul_rn(i + 0.5, o.dx), -o.center[0]);
    y = __dadd_rn(__dmul_rn(j + 0.5, o.dx), -o.center[1]);
    z = __dadd_rn(__dmul_rn(k + 0.5, o.dx), -o.center[2]);
#else
    // host: a separately rounded multiply and subtract (build the host
    // code without floating-point contraction)
    const volatile double px = (i + 0.5) * o.dx, py = (j + 0.5) * o.dx,
                          pz = (k + 0.5) * o.dx;
    x = px - o.center[0];
    y = py - o.center[1];
    z = pz - o.center[2];
#endif
}

GRHD_HD __forceinline__ bool excised(const Options &o, int i, int j, int k)
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

template <typename T>
GRHD_HD __forceinline__ T vsq(const T v[3], const T gLL[6])
{
    return gLL[0] * v[0] * v[0] + gLL[3] * v[1] * v[1] + gLL[5] * v[2] * v[2] +
           T(2) * (gLL[1] * v[0] * v[1] + gLL[2] * v[0] * v[2] +
                   gLL[4] * v[1] * v[2]);
}

// compute_conserved, Valencia.hpp:55-73
template <typename T>
GRHD_HD __forceinline__ ConsT<T> p2c(const PrimT<T> &pr, const T gLL[6])
{
    ConsT<T> c;
    const T vL0 = gLL[0] * pr.v[0] + gLL[1] * pr.v[1] + gLL[2] * pr.v[2];
    const T vL1 = gLL[1] * pr.v[0] + gLL[3] * pr.v[1] + gLL[4] * pr.v[2];
    const T vL2 = gLL[2] * pr.v[0] + gLL[4] * pr.v[1] + gLL[5] * pr.v[2];
    const T v2 = vL0 * pr.v[0] + vL1 * pr.v[1] + vL2 * pr.v[2];
    const T W = rsqrt_(T(1) - v2);
    const T h = T(1) + pr.eps + div_(pr.p, pr.rho);
    const T rhw = pr.rho * h * W * W;
    c.D = pr.rho * W;
    c.tau = rhw - pr.p - c.D;
    c.S[0] = rhw * vL0;
    c.S[1] = rhw * vL1;
    c.S[2] = rhw * vL2;
    return c;
}

// detail::pressure_residual (+ derivative), Valencia.hpp:79-108.  The
// recovery divides with div_ / rcp_ / sqrt_ like the rest of the device
// code; e = tau + D + p equal to zero (which IEEE division would turn into
// a capped v^2) gives a NaN residual and so a failed recovery.
GRHD_HD __forceinline__ double c2p_residual(double p, double D,
                                               double tau, double S2,
                                               double G, double Gfac,
                                               double vmax2, double *deriv)
{
    const double e = tau + D + p;
    const double ie = rcp_(e);
    double v2 = S2 * ie * ie;
    if (v2 > vmax2)
        v2 = vmax2;
    const double W = rsqrt_(1.0 - v2);
    const double W2 = W * W;
    if (deriv)
    {
        const double dW = -W2 * W * v2 * ie;
        *deriv = D * dW + Gfac * (W2 + p * 2.0 * W * dW) - 1.0;
    }
    return D * W + Gfac * p * W2 - e;
}

GRHD_HD __forceinline__ double c2p_S2(const Cons &c, const double gUU[6])
{
    return gUU[0] * c.S[0] * c.S[0] + gUU[3] * c.S[1] * c.S[1] +
           gUU[5] * c.S[2] * c.S[2] +
           2.0 * (gUU[1] * c.S[0] * c.S[1] + gUU[2] * c.S[0] * c.S[2] +
                  gUU[4] * c.S[1] * c.S[2]);
}

// The primitives of a converged pressure, Valencia.hpp:213-226; false when
// the velocity reaches the cap.
GRHD_HD __forceinline__ bool c2p_finish(const Options &o, const Cons &c,
                                           const double gUU[6], double S2,
                                           double p, Prim &out)
{
    const double e = c.tau + c.D + p;
    const double v2 = div_(S2, e * e);
    if (!(v2 < o.rec_vmax2))
        return false;
    // W rounded as the reference's 1 / sqrt(1 - v^2) (sqrt_ and rcp_ give
    // the IEEE results, rsqrt_ is up to two ulp off): rho = D / W decides
    // the atmosphere and floor tests bit for bit, and an ulp there switches
    // a cell's sources on or off
    const double W = rcp_(sqrt_(1.0 - v2));
    out.rho = div_(c.D, W);
    out.p = p;
    out.eps = div_(p, (o.G - 1.0) * out.rho);
    const double ie = rcp_(e);
    out.v[0] = (gUU[0] * c.S[0] + gUU[1] * c.S[1] + gUU[2] * c.S[2]) * ie;
    out.v[1] = (gUU[1] * c.S[0] + gUU[3] * c.S[1] + gUU[4] * c.S[2]) * ie;
    out.v[2] = (gUU[2] * c.S[0] + gUU[4] * c.S[1] + gUU[5] * c.S[2]) * ie;
    return true;
}

// recover_primitive, Valencia.hpp:116-228 (bounded loops throughout).
GRHD_HD __forceinline__ bool con2prim(const Options &o, const Cons &c,
                                         const double gUU[6], Prim &out,
                                         int *iters_out, double *resid_out)
{
    int iters = 0;
    double resid = 0.0;
    bool ok = false;
    if (c.D > 0.0)
    {
        const double G = o.G;
        const double Gfac = div_(G, G - 1.0);
        const double vmax2 = o.rec_vmax2;
        const double tol = o.rec_tol;
        const double S2 = c2p_S2(c, gUU);
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
                double np = p - div_(r, dres);
                if (!isfinite(np) || np <= lower || np >= upper)
                    np = 0.5 * (lower + upper);
                p = np;
                r = c2p_residual(p, c.D, c.tau, S2, G, Gfac, vmax2, &dres);
            }
            resid = r;
            if (fabs(r) < tol)
                ok = c2p_finish(o, c, gUU, S2, p, out);
        }
    }
    if (iters_out)
        *iters_out = iters;
    if (resid_out)
        *resid_out = resid;
    return ok;
}

// Mixed path: the same FP64 root solve started from a known nearby
// pressure (the previous stage's), safeguarded Newton on the monotone
// residual; falls back to the full bracketed solve when the guess is not
// usable or a step leaves (p_floor, inf).  Converges to the same root to
// the solver tolerance.
GRHD_HD __forceinline__ bool con2prim_warm(const Options &o, const Cons &c,
                                              const double gUU[6],
                                              double p_guess, Prim &out)
{
    if (c.D > 0.0 && !(p_guess > o.rec_pfloor))
    {
        // a guess at (or rounded below) the recovery floor: the full solve
        // returns the floor itself when the residual there is within
        // tolerance; test that first
        const double G = o.G;
        const double S2 = c2p_S2(c, gUU);
        const double r = c2p_residual(o.rec_pfloor, c.D, c.tau, S2, G,
                                      div_(G, G - 1.0), o.rec_vmax2, nullptr);
        if (fabs(r) <= o.rec_tol)
            return c2p_finish(o, c, gUU, S2, o.rec_pfloor, out) ||
                   con2prim(o, c, gUU, out, nullptr, nullptr);
    }
    if (c.D > 0.0 && p_guess > o.rec_pfloor && isfinite(p_guess))
    {
        const double G = o.G;
        const double Gfac = div_(G, G - 1.0);
        const double S2 = c2p_S2(c, gUU);
        double p = p_guess, dres;
        double r = c2p_residual(p, c.D, c.tau, S2, G, Gfac, o.rec_vmax2, &dres);
        for (int it = 0; it < 6; ++it)
        {
            if (fabs(r) < o.rec_tol)
                return c2p_finish(o, c, gUU, S2, p, out) ||
                       con2prim(o, c, gUU, out, nullptr, nullptr);
            const double np = p - div_(r, dres);
            if (!isfinite(np) || !(np > o.rec_pfloor))
                break;
            p = np;
            r = c2p_residual(p, c.D, c.tau, S2, G, Gfac, o.rec_vmax2, &dres);
        }
    }
    return con2prim(o, c, gUU, out, nullptr, nullptr);
}

// enforce_primitive_floors, Atmosphere.hpp:24-46 (eps recomputed always)
template <typename T>
GRHD_HD __forceinline__ void floors(const Options &o, PrimT<T> &pr,
                                       const T gLL[6])
{
    pr.rho = max_(pr.rho, T(o.rho_floor));
    pr.p = max_(pr.p, T(o.p_floor));
    const T v2 = vsq(pr.v, gLL);
    if (v2 >= T(o.atmo_vmax2))
    {
        const T s = sqrt_(div_(T(o.atmo_vmax2), v2));
        pr.v[0] *= s;
        pr.v[1] *= s;
        pr.v[2] *= s;
    }
    pr.eps = div_(pr.p, (T(o.G) - T(1)) * pr.rho);
}

// make_atmosphere_primitive, Atmosphere.hpp:48-60
GRHD_HD __forceinline__ Prim atmosphere(const Options &o)
{
    Prim pr;
    pr.rho = o.rho_floor;
    pr.p = o.p_floor;
    pr.eps = pr.p / ((o.G - 1.0) * pr.rho);
    pr.v[0] = pr.v[1] = pr.v[2] = 0.0;
    return pr;
}

// is_atmosphere_primitive, FArrayBoxFiniteVolume.hpp:118-126
template <typename T>
GRHD_HD __forceinline__ bool is_atmo(const Options &o, const PrimT<T> &pr,
                                        double factor)
{
    const double f = fmax(1.0, factor);
    return pr.rho <= T(f * o.rho_floor) && pr.p <= T(f * o.p_floor);
}

// compute_flux, Valencia.hpp:230-259
template <typename T>
GRHD_HD __forceinline__ ConsT<T> phys_flux(const PrimT<T> &pr,
                                              const ConsT<T> &c, int d,
                                              T lapse, const T shift[3])
{
    ConsT<T> f;
    const T tv = lapse * pr.v[d] - shift[d];
    const T ap = lapse * pr.p;
    f.D = c.D * tv;
    f.tau = c.tau * tv + ap * pr.v[d];
#pragma unroll
    for (int j = 0; j < 3; ++j)
        f.S[j] = c.S[j] * tv + (j == d ? ap : T(0));
    return f;
}

// compute_characteristic_speeds (shifted), RiemannSolvers.hpp:23-67
template <typename T>
GRHD_HD __forceinline__ void char_speeds(const Options &o,
                                            const PrimT<T> &pr,
                                            const GeoT<T> &g, int d, T &lo,
                                            T &hi)
{
    const T v2 = vsq(pr.v, g.gLL);
    const T h = T(1) + pr.eps + div_(pr.p, pr.rho);
    const T cs2 = div_(T(o.G) * pr.p, pr.rho * h);
    const T cs = sqrt_(cs2);
    const T vel = pr.v[d];
    const T den = T(1) - v2 * cs2;
    const T rad =
        (T(1) - v2) * (g.gUU[sym(d, d)] * den - vel * vel * (T(1) - cs2));
    const T root = cs * sqrt_(max_(T(0), rad));
    const T base = vel * (T(1) - cs2);
    const T iden = rcp_(den);
    lo = g.lapse * ((base - root) * iden) - g.shift[d];
    hi = g.lapse * ((base + root) * iden) - g.shift[d];
}

// minmod / compute_limited_slope, Reconstruction.hpp:16-37
template <typename T> GRHD_HD __forceinline__ T minmod2(T l, T r)
{
    if (l * r <= T(0))
        return T(0);
    return l > T(0) ? min_(l, r) : max_(l, r);
}

template <typename T>
GRHD_HD __forceinline__ T limited_slope(T l, T c, T r, T theta)
{
    return minmod2(theta * (c - l), minmod2(T(0.5) * (r - l), theta * (r - c)));
}

// One MUSCL-HLLE face flux between cells L and R (compute_muscl_hlle_flux,
// FiniteVolume.hpp:63-98, with the face geometry of average_geometry,
// FArrayBoxFiniteVolume.hpp:194-216).  LL, L, R, RR are the cells
// i-1, i, i+1, i+2 around face i+1/2.
template <typename T>
GRHD_HD __forceinline__ ConsT<T> face_flux(const Options &o,
                                              const PVT<T> &LL,
                                              const PVT<T> &L,
                                              const PVT<T> &R,
                                              const PVT<T> &RR,
                                              const GeoT<T> &g, int d)
{
    PrimT<T> lp, rp;
    T ql[5], qr[5];
    const T theta = T(o.theta);
#pragma unroll
    for (int c = 0; c < 5; ++c)
    {
        if (o.use_recon)
        {
            const T sl = limited_slope(LL.q[c], L.q[c], R.q[c], theta);
            const T sr = limited_slope(L.q[c], R.q[c], RR.q[c], theta);
            ql[c] = L.q[c] + T(0.5) * sl;
            qr[c] = R.q[c] - T(0.5) * sr;
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
    const ConsT<T> lc = p2c(lp, g.gLL);
    const ConsT<T> rc = p2c(rp, g.gLL);
    // compute_hlle_flux, RiemannSolvers.hpp:69-118
    const ConsT<T> lf = phys_flux(lp, lc, d, g.lapse, g.shift);
    const ConsT<T> rf = phys_flux(rp, rc, d, g.lapse, g.shift);
    T llo, lhi, rlo, rhi;
    char_speeds(o, lp, g, d, llo, lhi);
    char_speeds(o, rp, g, d, rlo, rhi);
    const T sl = min_(T(0), min_(llo, rlo));
    const T su = max_(T(0), max_(lhi, rhi));
    if (sl >= T(0))
        return lf;
    if (su <= T(0))
        return rf;
    const T inv = rcp_(su - sl);
    const T ss = sl * su;
    ConsT<T> f;
    f.D = (su * lf.D - sl * rf.D + ss * (rc.D - lc.D)) * inv;
    f.tau = (su * lf.tau - sl * rf.tau + ss * (rc.tau - lc.tau)) * inv;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        f.S[i] = (su * lf.S[i] - sl * rf.S[i] + ss * (rc.S[i] - lc.S[i])) * inv;
    return f;
}

template <typename T>
GRHD_HD __forceinline__ void average_geo(const GeoT<T> &a, const GeoT<T> &b,
                                            GeoT<T> &g)
{
#pragma unroll
    for (int s = 0; s < 6; ++s)
    {
        g.gLL[s] = T(0.5) * (a.gLL[s] + b.gLL[s]);
        g.gUU[s] = T(0.5) * (a.gUU[s] + b.gUU[s]);
    }
    g.lapse = T(0.5) * (a.lapse + b.lapse);
#pragma unroll
    for (int i = 0; i < 3; ++i)
        g.shift[i] = T(0.5) * (a.shift[i] + b.shift[i]);
}

// compute_static_metric_source_terms, StaticMetric.hpp:193-275
template <typename T>
GRHD_HD __forceinline__ ConsT<T> static_sources(const PrimT<T> &pr,
                                                   const ConsT<T> &c,
                                                   const GeoFullT<T> &f)
{
    const GeoT<T> &g = f.g;
    const T W = rsqrt_(T(1) - vsq(pr.v, g.gLL));
    const T h = T(1) + pr.eps + div_(pr.p, pr.rho);
    const T rhw = pr.rho * h * W * W;
    T st[6];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
            st[sym(i, j)] = rhw * pr.v[i] * pr.v[j] + pr.p * g.gUU[sym(i, j)];
    const T E = c.D + c.tau;
    T mU[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        mU[i] = g.gUU[sym(i, 0)] * c.S[0] + g.gUU[sym(i, 1)] * c.S[1] +
                g.gUU[sym(i, 2)] * c.S[2];
    ConsT<T> F[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
        F[d] = phys_flux(pr, c, d, g.lapse, g.shift);
    ConsT<T> s;
    s.D = T(0);
    s.tau = T(0);
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        s.D -= F[d].D * f.dlnsqrtg[d];
        s.tau -= F[d].tau * f.dlnsqrtg[d];
        s.tau -= mU[d] * f.dlapse[d];
    }
    T sk = T(0);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            sk += st[sym(i, j)] * f.K[sym(i, j)];
    s.tau += g.lapse * sk;
#pragma unroll
    for (int m = 0; m < 3; ++m)
    {
        T ms = -E * f.dlapse[m];
        T sg = T(0);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                sg += st[sym(i, j)] * f.dgamma[m][sym(i, j)];
        ms += T(0.5) * g.lapse * sg;
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

template <typename A, typename B>
GRHD_HD __forceinline__ PrimT<B> convert_prim(const PrimT<A> &s)
{
    PrimT<B> d;
    d.rho = B(s.rho);
    d.eps = B(s.eps);
    d.p = B(s.p);
    d.v[0] = B(s.v[0]);
    d.v[1] = B(s.v[1]);
    d.v[2] = B(s.v[2]);
    return d;
}

template <typename A, typename B>
GRHD_HD __forceinline__ ConsT<B> convert_cons(const ConsT<A> &s)
{
    ConsT<B> d;
    d.D = B(s.D);
    d.S[0] = B(s.S[0]);
    d.S[1] = B(s.S[1]);
    d.S[2] = B(s.S[2]);
    d.tau = B(s.tau);
    return d;
}

} // namespace grhd
