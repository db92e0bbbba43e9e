/*
 * grhd_oracle.c -- CPU restatement of GRDzhadzha's fixed-background Valencia
 * GRHD path (TEST INFRASTRUCTURE ONLY; see grhd_oracle.h).
 *
 * Paths cited below are relative to the GRDzhadzha source tree.  The
 * GRChombo helpers the reference calls (TensorAlgebra, Coordinates) are not
 * part of that tree; their arithmetic is restated from its mathematics here
 * (symmetric 3x3 determinant/inverse by cofactors, Christoffel symbols of the
 * second kind, index contractions; cell centre (i+1/2)dx - centre and a
 * coordinate radius clamped below at 1e-6).
 *
 * Build with -ffp-contract=off so that no fused multiply-add changes the
 * rounding of the reference expressions.
 */
#include "grhd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

/* ------------------------------------------------------------------------ */
/* small value types                                                         */
/* ------------------------------------------------------------------------ */

typedef struct
{
    double rho, eps, p, v[3];
} Prim;

typedef struct
{
    double D, S[3], tau;
} Cons;

typedef Cons Flux;

typedef struct
{
    double gLL[3][3], gUU[3][3], lapse, shift[3], K[3][3];
} Geom;

typedef struct
{
    double dlapse[3];
    double dlnsqrtg[3];
    double dgamma[3][3][3]; /* [direction][i][j] */
    double dshift[3][3];    /* [i][direction]   */
} Derivs;

typedef struct
{
    double gamma[3][3], K_tensor[3][3], K, lapse, shift[3];
    double d1_gamma[3][3][3]; /* [i][j][k] = d_k gamma_ij */
    double d1_lapse[3];
    double d1_shift[3][3];    /* [i][j] = d_j shift^i */
} ADM;

static double delta(int i, int j) { return i == j ? 1.0 : 0.0; }
static double dmax(double a, double b) { return a > b ? a : b; }
static double dmin(double a, double b) { return a < b ? a : b; }

/* ------------------------------------------------------------------------ */
/* tensor algebra (GRChombo TensorAlgebra, restated)                          */
/* ------------------------------------------------------------------------ */

static double det_sym(const double m[3][3])
{
    return m[0][0] * m[1][1] * m[2][2] + 2 * m[0][1] * m[0][2] * m[1][2] -
           m[0][0] * m[1][2] * m[1][2] - m[1][1] * m[0][2] * m[0][2] -
           m[2][2] * m[0][1] * m[0][1];
}

static void inverse_sym(const double m[3][3], double out[3][3])
{
    const double det = det_sym(m);
    out[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[1][2]) / det;
    out[0][1] = (m[0][2] * m[1][2] - m[0][1] * m[2][2]) / det;
    out[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) / det;
    out[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[0][2]) / det;
    out[1][2] = (m[0][1] * m[0][2] - m[0][0] * m[1][2]) / det;
    out[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[0][1]) / det;
    out[1][0] = out[0][1];
    out[2][0] = out[0][2];
    out[2][1] = out[1][2];
}

/* Gamma^i_jk = gUU^il * 1/2 (d_k g_lj + d_j g_lk - d_l g_jk) */
static void christoffel_ULL(const double d1[3][3][3], const double gUU[3][3],
                            double ULL[3][3][3])
{
    double LLL[3][3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                LLL[i][j][k] =
                    0.5 * (d1[j][i][k] + d1[k][i][j] - d1[j][k][i]);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
            {
                ULL[i][j][k] = 0;
                for (int l = 0; l < 3; ++l)
                    ULL[i][j][k] += gUU[i][l] * LLL[l][j][k];
            }
}

static double trace_sym(const double gUU[3][3], const double m[3][3])
{
    double t = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            t += gUU[i][j] * m[i][j];
    return t;
}

static double dot_metric(const double a[3], const double b[3],
                         const double g[3][3])
{
    double d = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            d += a[i] * b[j] * g[i][j];
    return d;
}

/* ------------------------------------------------------------------------ */
/* analytic backgrounds                                                      */
/* ------------------------------------------------------------------------ */

/* Coordinates<double>::get_radius: coordinate radius, clamped at 1e-6. */
static double coord_radius(double x, double y, double z)
{
    const double r = sqrt(x * x + y * y + z * z);
    return dmax(r, 1.0e-6);
}

/* KerrSchild::get_KS_derivs, Source/Background/KerrSchild.hpp:171-242 */
static void ks_derivs(double M, double a, double x0, double x1, double x2,
                      double H, double dHdx[3], double dldx[3][3],
                      double dltdx[3])
{
    (void)M;
    const double a2 = a * a;
    const double x[3] = {x0, x1, x2};
    const double z = x2;
    const double rho = coord_radius(x0, x1, x2);
    const double rho2 = rho * rho;
    const double r2 =
        0.5 * (rho2 - a2) + sqrt(0.25 * (rho2 - a2) * (rho2 - a2) + a2 * z * z);
    const double r = sqrt(r2);
    const double cos_theta = z / r;
    const double cos_theta2 = cos_theta * cos_theta;

    double drhodx[3], drdx[3], dcosthetadx[3];
    for (int i = 0; i < 3; ++i)
        drhodx[i] = x[i] / rho;
    for (int i = 0; i < 3; ++i)
        drdx[i] = 0.5 / r *
                  (rho * drhodx[i] +
                   0.5 / sqrt(0.25 * (rho2 - a2) * (rho2 - a2) + a2 * z * z) *
                       (drhodx[i] * rho * (rho2 - a2) +
                        delta(i, 2) * 2.0 * a2 * z));
    for (int i = 0; i < 3; ++i)
        dcosthetadx[i] = -z / r2 * drdx[i] + delta(i, 2) / r;
    for (int i = 0; i < 3; ++i)
        dHdx[i] = H * (drdx[i] / r -
                       2.0 / (r2 + a2 * cos_theta2) *
                           (r * drdx[i] + a2 * cos_theta * dcosthetadx[i]));
    for (int i = 0; i < 3; ++i)
    {
        dldx[0][i] = (x[0] * drdx[i] + r * delta(i, 0) + a * delta(i, 1) -
                      2.0 * r * drdx[i] * (r * x[0] + a * x[1]) / (r2 + a2)) /
                     (r2 + a2);
        dldx[1][i] = (x[1] * drdx[i] + r * delta(i, 1) - a * delta(i, 0) -
                      2.0 * r * drdx[i] * (r * x[1] - a * x[0]) / (r2 + a2)) /
                     (r2 + a2);
        dldx[2][i] = -x[2] * drdx[i] / r2 + delta(i, 2) / r;
    }
    for (int i = 0; i < 3; ++i)
        dltdx[i] = 0.0;
}

/* KerrSchild::compute_metric_background, KerrSchild.hpp:64-166 */
static void ks_metric(double M, double a, double x, double y, double z,
                      ADM *v)
{
    const double a2 = a * a;
    const double rho = coord_radius(x, y, z);
    const double rho2 = rho * rho;
    const double r2 =
        0.5 * (rho2 - a2) + sqrt(0.25 * (rho2 - a2) * (rho2 - a2) + a2 * z * z);
    const double r = sqrt(r2);
    const double cos_theta = z / r;
    const double H = M * r / (r2 + a2 * cos_theta * cos_theta);
    const double el[3] = {(r * x + a * y) / (r2 + a2),
                          (r * y - a * x) / (r2 + a2), z / r};
    const double el_t = 1.0;

    double dHdx[3], dldx[3][3], dltdx[3];
    ks_derivs(M, a, x, y, z, H, dHdx, dldx, dltdx);

    v->lapse = pow(1.0 + 2.0 * H * el_t * el_t, -0.5);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            v->gamma[i][j] = delta(i, j) + 2.0 * H * el[i] * el[j];
    double gUU[3][3];
    inverse_sym(v->gamma, gUU);
    for (int i = 0; i < 3; ++i)
    {
        v->shift[i] = 0;
        for (int j = 0; j < 3; ++j)
            v->shift[i] += gUU[i][j] * 2.0 * H * el[j] * el_t;
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                v->d1_gamma[i][j][k] =
                    2.0 * (el[i] * el[j] * dHdx[k] + H * el[i] * dldx[j][k] +
                           H * el[j] * dldx[i][k]);
    for (int i = 0; i < 3; ++i)
        v->d1_lapse[i] = -pow(v->lapse, 3.0) * el_t *
                         (el_t * dHdx[i] + 2.0 * H * dltdx[i]);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            v->d1_shift[i][j] =
                2.0 * el_t * dHdx[j] * pow(v->lapse, 2.0) * el[i] +
                4.0 * el_t * H * v->lapse * v->d1_lapse[j] * el[i] +
                2.0 * el_t * H * pow(v->lapse, 2.0) * dldx[i][j] +
                2.0 * dltdx[j] * H * pow(v->lapse, 2.0) * el[i];

    double ULL[3][3][3];
    christoffel_ULL(v->d1_gamma, gUU, ULL);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
        {
            v->K_tensor[i][j] = 0.0;
            for (int k = 0; k < 3; ++k)
            {
                v->K_tensor[i][j] +=
                    v->gamma[k][j] * v->d1_shift[k][i] +
                    v->gamma[k][i] * v->d1_shift[k][j] +
                    (v->d1_gamma[k][i][j] + v->d1_gamma[k][j][i]) *
                        v->shift[k];
                for (int m = 0; m < 3; ++m)
                    v->K_tensor[i][j] +=
                        -2.0 * ULL[k][i][j] * v->gamma[k][m] * v->shift[m];
            }
            v->K_tensor[i][j] *= 0.5 / v->lapse;
        }
    v->K = trace_sym(gUU, v->K_tensor);
}

typedef struct
{
    double scalar, scalar_time_derivative, scalar_derivative[3], vector[3],
        vector_derivative[3][3];
} PNPotentials;

/* CircularBinaryPN::add_point_potential, CircularBinaryPN.hpp:252-297 */
static void pn_add_point(PNPotentials *pt, double softening, double mass,
                         const double sp[3], const double sv[3],
                         const double fp[3])
{
    double disp[3];
    double r2 = softening * softening;
    for (int i = 0; i < 3; ++i)
    {
        disp[i] = fp[i] - sp[i];
        r2 += disp[i] * disp[i];
    }
    const double inv_r = 1.0 / sqrt(r2);
    const double inv_r3 = inv_r * inv_r * inv_r;
    pt->scalar += mass * inv_r;
    double ddv = 0.0;
    for (int i = 0; i < 3; ++i)
        ddv += disp[i] * sv[i];
    pt->scalar_time_derivative += mass * ddv * inv_r3;
    for (int d = 0; d < 3; ++d)
        pt->scalar_derivative[d] += -mass * disp[d] * inv_r3;
    for (int c = 0; c < 3; ++c)
        for (int d = 0; d < 3; ++d)
            pt->vector_derivative[c][d] += -mass * sv[c] * disp[d] * inv_r3;
    for (int c = 0; c < 3; ++c)
        pt->vector[c] += mass * sv[c] * inv_r;
}

/* CircularBinaryPN::angular_velocity / compute_state, :209-250 */
static void pn_state(const orc_params *p, double t, double p1[3],
                     double p2[3], double v1[3], double v2[3])
{
    const double total = p->pn_mass_1 + p->pn_mass_2;
    const double omega =
        p->pn_angular_velocity != 0.0
            ? p->pn_angular_velocity
            : sqrt(total / (p->pn_separation * p->pn_separation *
                            p->pn_separation));
    const double phase = p->pn_phase + omega * (p->pn_time + t);
    const double c = cos(phase), s = sin(phase);
    const double r1 = p->pn_mass_2 / total * p->pn_separation;
    const double r2 = p->pn_mass_1 / total * p->pn_separation;
    for (int i = 0; i < 3; ++i)
        p1[i] = p2[i] = v1[i] = v2[i] = 0.0;
    p1[0] = r1 * c;
    p1[1] = r1 * s;
    p2[0] = -r2 * c;
    p2[1] = -r2 * s;
    v1[0] = -omega * r1 * s;
    v1[1] = omega * r1 * c;
    v2[0] = omega * r2 * s;
    v2[1] = -omega * r2 * c;
}

/* CircularBinaryPN::compute_metric_background, CircularBinaryPN.hpp:70-189.
 * The reference's background factory adds the operator time to params.time
 * (Tests/GRHDFixedBGTest/GRHDFixedBGTest.cpp:440-445). */
static void pn_metric(const orc_params *p, double t, double x, double y,
                      double z, ADM *v)
{
    const double pos[3] = {x, y, z};
    double p1[3], p2[3], v1[3], v2[3];
    pn_state(p, t, p1, p2, v1, v2);
    PNPotentials pt;
    memset(&pt, 0, sizeof(pt));
    pn_add_point(&pt, p->pn_softening_radius, p->pn_mass_1, p1, v1, pos);
    pn_add_point(&pt, p->pn_softening_radius, p->pn_mass_2, p2, v2, pos);

    const double U = pt.scalar;
    const double dpsi_dt = 2.0 * pt.scalar_time_derivative;
    const double psi = 1.0 + 2.0 * U;
    double V2 = 0.0;
    for (int i = 0; i < 3; ++i)
        V2 += pt.vector[i] * pt.vector[i];
    const double lapse2 = 1.0 - 2.0 * U + 2.0 * U * U + 16.0 * V2 / psi;

    memset(v, 0, sizeof(*v));
    v->lapse = sqrt(lapse2);
    for (int i = 0; i < 3; ++i)
    {
        v->gamma[i][i] = psi;
        v->shift[i] = -4.0 * pt.vector[i] / psi;
    }
    double gUU[3][3];
    inverse_sym(v->gamma, gUU);
    for (int d = 0; d < 3; ++d)
    {
        const double dU = pt.scalar_derivative[d];
        const double dpsi = 2.0 * dU;
        for (int m = 0; m < 3; ++m)
            v->d1_gamma[m][m][d] = dpsi;
        double dV2 = 0.0;
        for (int c = 0; c < 3; ++c)
        {
            dV2 += 2.0 * pt.vector[c] * pt.vector_derivative[c][d];
            v->d1_shift[c][d] =
                -4.0 * (pt.vector_derivative[c][d] / psi -
                        pt.vector[c] * dpsi / (psi * psi));
        }
        const double dlapse2 =
            (-2.0 + 4.0 * U) * dU +
            16.0 * (dV2 / psi - V2 * dpsi / (psi * psi));
        v->d1_lapse[d] = 0.5 * dlapse2 / v->lapse;
    }
    double ULL[3][3][3];
    christoffel_ULL(v->d1_gamma, gUU, ULL);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
        {
            for (int k = 0; k < 3; ++k)
            {
                v->K_tensor[i][j] +=
                    v->gamma[k][j] * v->d1_shift[k][i] +
                    v->gamma[k][i] * v->d1_shift[k][j] +
                    (v->d1_gamma[k][i][j] + v->d1_gamma[k][j][i]) *
                        v->shift[k];
                for (int m = 0; m < 3; ++m)
                    v->K_tensor[i][j] +=
                        -2.0 * ULL[k][i][j] * v->gamma[k][m] * v->shift[m];
            }
            if (i == j)
                v->K_tensor[i][j] -= dpsi_dt;
            v->K_tensor[i][j] *= 0.5 / v->lapse;
        }
    v->K = trace_sym(gUU, v->K_tensor);
}

static void background_adm(const orc_params *p, double t, double x, double y,
                           double z, ADM *v)
{
    if (p->background == ORC_BG_BINARY_PN)
        pn_metric(p, t, x, y, z, v);
    else
        ks_metric(p->ks_mass, p->ks_spin, x, y, z, v);
}

/* make_cell_geometry_from_adm, Source/Matter/GRHD/FixedBGMetric.hpp:17-29 */
static void geom_from_adm(const ADM *v, Geom *g)
{
    memcpy(g->gLL, v->gamma, sizeof(g->gLL));
    inverse_sym(v->gamma, g->gUU);
    g->lapse = v->lapse;
    for (int i = 0; i < 3; ++i)
        g->shift[i] = v->shift[i];
    memcpy(g->K, v->K_tensor, sizeof(g->K));
}

/* make_static_metric_derivatives_from_adm, FixedBGMetric.hpp:31-53 */
static void derivs_from_adm(const ADM *v, Derivs *d)
{
    memset(d, 0, sizeof(*d));
    for (int i = 0; i < 3; ++i)
        d->dlapse[i] = v->d1_lapse[i];
    memcpy(d->dshift, v->d1_shift, sizeof(d->dshift));
    double gUU[3][3];
    inverse_sym(v->gamma, gUU);
    for (int dir = 0; dir < 3; ++dir)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
            {
                d->dgamma[dir][i][j] = v->d1_gamma[i][j][dir];
                d->dlnsqrtg[dir] += 0.5 * gUU[i][j] * v->d1_gamma[i][j][dir];
            }
}

static void cell_position(const orc_params *p, int i, int j, int k,
                          double *x, double *y, double *z)
{
    *x = (i + 0.5) * p->dx - p->center[0];
    *y = (j + 0.5) * p->dx - p->center[1];
    *z = (k + 0.5) * p->dx - p->center[2];
}

/* load_fixed_background_geometry, FixedBGFArrayBoxFiniteVolume.hpp:15-22 */
static void load_geometry(const orc_params *p, double t, int i, int j, int k,
                          Geom *g)
{
    double x, y, z;
    cell_position(p, i, j, k, &x, &y, &z);
    ADM v;
    background_adm(p, t, x, y, z, &v);
    geom_from_adm(&v, g);
}

/* load_fixed_background_metric_derivatives, :24-31 */
static void load_derivs(const orc_params *p, double t, int i, int j, int k,
                        Derivs *d)
{
    double x, y, z;
    cell_position(p, i, j, k, &x, &y, &z);
    ADM v;
    background_adm(p, t, x, y, z, &v);
    derivs_from_adm(&v, d);
}

/* average_geometry, FArrayBoxFiniteVolume.hpp:194-216 */
static void average_geometry(const Geom *l, const Geom *r, Geom *g)
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
        {
            g->gLL[i][j] = 0.5 * (l->gLL[i][j] + r->gLL[i][j]);
            g->gUU[i][j] = 0.5 * (l->gUU[i][j] + r->gUU[i][j]);
            g->K[i][j] = 0.5 * (l->K[i][j] + r->K[i][j]);
        }
    g->lapse = 0.5 * (l->lapse + r->lapse);
    for (int i = 0; i < 3; ++i)
        g->shift[i] = 0.5 * (l->shift[i] + r->shift[i]);
}

/* spatial_metric_log_sqrt_det, StaticMetric.hpp:293-302 */
static double log_sqrt_det(const Geom *g)
{
    const double det = det_sym(g->gLL);
    if (det <= 0.0 || !isfinite(det))
        return 0.0;
    return 0.5 * log(det);
}

/* ------------------------------------------------------------------------ */
/* EOS and Valencia (IdealGasEOS.hpp, Valencia.hpp)                          */
/* ------------------------------------------------------------------------ */

static double eos_enthalpy(double rho, double eps, double p)
{
    return 1.0 + eps + p / rho;
}
static double eos_cs2(double G, double rho, double eps, double p)
{
    const double h = eos_enthalpy(rho, eps, p);
    return G * p / (rho * h);
}

/* compute_velocity_squared, Valencia.hpp:33-43 */
static double velocity_squared(const double v[3], const double g[3][3])
{
    double v2 = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            v2 += g[i][j] * v[i] * v[j];
    return v2;
}

/* compute_conserved, Valencia.hpp:55-73 */
static Cons p2c(double G, const Prim *pr, const double g[3][3])
{
    (void)G;
    Cons c;
    double vL[3];
    for (int i = 0; i < 3; ++i)
    {
        vL[i] = 0;
        for (int j = 0; j < 3; ++j)
            vL[i] += g[i][j] * pr->v[j];
    }
    const double W = 1.0 / sqrt(1.0 - velocity_squared(pr->v, g));
    const double h = eos_enthalpy(pr->rho, pr->eps, pr->p);
    const double rhw = pr->rho * h * W * W;
    c.D = pr->rho * W;
    c.tau = rhw - pr->p - c.D;
    for (int i = 0; i < 3; ++i)
        c.S[i] = rhw * vL[i];
    return c;
}

static double sq(double x) { return x * x; }

/* detail::pressure_residual, Valencia.hpp:79-91 */
static double pres_residual(double p, double D, double tau, double S2,
                            double G, double vmax2)
{
    const double e = tau + D + p;
    double v2 = S2 / sq(e);
    if (v2 > vmax2)
        v2 = vmax2;
    const double W = 1.0 / sqrt(1.0 - v2);
    return D * W + G * p * W * W / (G - 1.0) - e;
}

/* detail::pressure_residual_derivative, Valencia.hpp:93-108 */
static double pres_residual_deriv(double p, double D, double tau, double S2,
                                  double G, double vmax2)
{
    const double e = tau + D + p;
    double v2 = S2 / sq(e);
    if (v2 > vmax2)
        v2 = vmax2;
    const double W = 1.0 / sqrt(1.0 - v2);
    const double dW = -W * W * W * v2 / e;
    const double dW2 = 2.0 * W * dW;
    return D * dW + G * (W * W + p * dW2) / (G - 1.0) - 1.0;
}

/* recover_primitive, Valencia.hpp:116-228 */
static int con2prim(const orc_params *o, const Cons *c, const double gUU[3][3],
                    Prim *out, int *iters, double *resid)
{
    *iters = 0;
    *resid = 0.0;
    if (c->D <= 0.0)
        return 0;
    const double G = o->gamma;
    const double vmax2 = o->rec_max_velocity_squared;
    const double tol = o->rec_tolerance;
    const int maxit = o->rec_max_iterations;
    const double S2 = dot_metric(c->S, c->S, gUU);

    double lower = o->rec_pressure_floor;
    double f_lower = pres_residual(lower, c->D, c->tau, S2, G, vmax2);
    if (f_lower >= 0.0 && fabs(f_lower) > tol)
        return 0;
    double upper = lower;
    double f_upper = f_lower;
    if (f_lower < 0.0)
    {
        upper = dmax(1.0, fabs(c->tau) + c->D);
        f_upper = pres_residual(upper, c->D, c->tau, S2, G, vmax2);
        int b = 0;
        while (f_upper <= 0.0 && b < maxit)
        {
            upper *= 2.0;
            f_upper = pres_residual(upper, c->D, c->tau, S2, G, vmax2);
            ++b;
        }
        if (f_upper <= 0.0)
            return 0;
    }
    double p = (fabs(f_lower) <= tol)
                   ? lower
                   : dmin(dmax(c->tau * (G - 1.0), lower), upper);
    double r = pres_residual(p, c->D, c->tau, S2, G, vmax2);
    for (int it = 0; it < maxit; ++it)
    {
        *iters = it + 1;
        if (fabs(r) < tol)
            break;
        if (f_lower < 0.0)
        {
            if (r > 0.0)
                upper = p;
            else
                lower = p;
        }
        const double dr = pres_residual_deriv(p, c->D, c->tau, S2, G, vmax2);
        double np = p - r / dr;
        if (!isfinite(np) || np <= lower || np >= upper)
            np = 0.5 * (lower + upper);
        p = np;
        r = pres_residual(p, c->D, c->tau, S2, G, vmax2);
    }
    *resid = r;
    if (fabs(r) >= tol)
        return 0;
    const double e = c->tau + c->D + p;
    const double v2 = S2 / sq(e);
    if (v2 >= vmax2)
        return 0;
    const double W = 1.0 / sqrt(1.0 - v2);
    out->rho = c->D / W;
    out->p = p;
    out->eps = p / ((G - 1.0) * out->rho);
    for (int i = 0; i < 3; ++i)
    {
        out->v[i] = 0.0;
        for (int j = 0; j < 3; ++j)
            out->v[i] += gUU[i][j] * c->S[j] / e;
    }
    return 1;
}

/* compute_flux, Valencia.hpp:230-259 */
static Flux phys_flux(const Prim *pr, const Cons *c, int d, double lapse,
                      const double shift[3])
{
    Flux f;
    const double tv = lapse * pr->v[d] - shift[d];
    f.D = c->D * tv;
    f.tau = c->tau * tv + lapse * pr->p * pr->v[d];
    for (int j = 0; j < 3; ++j)
    {
        f.S[j] = c->S[j] * tv;
        if (j == d)
            f.S[j] += lapse * pr->p;
    }
    return f;
}

/* ------------------------------------------------------------------------ */
/* atmosphere (Atmosphere.hpp, FArrayBoxFiniteVolume.hpp:118-134,704-711)    */
/* ------------------------------------------------------------------------ */

static void enforce_floors(const orc_params *o, Prim *pr, const double g[3][3])
{
    pr->rho = dmax(pr->rho, o->atmo_rho_floor);
    pr->p = dmax(pr->p, o->atmo_pressure_floor);
    const double v2 = velocity_squared(pr->v, g);
    if (v2 >= o->atmo_max_velocity_squared)
    {
        const double s = sqrt(o->atmo_max_velocity_squared / v2);
        for (int i = 0; i < 3; ++i)
            pr->v[i] *= s;
    }
    pr->eps = pr->p / ((o->gamma - 1.0) * pr->rho);
}

static Prim atmosphere_prim(const orc_params *o)
{
    Prim pr;
    pr.rho = o->atmo_rho_floor;
    pr.p = o->atmo_pressure_floor;
    pr.eps = pr.p / ((o->gamma - 1.0) * pr.rho);
    pr.v[0] = pr.v[1] = pr.v[2] = 0.0;
    return pr;
}

static int is_atmosphere(const orc_params *o, const Prim *pr, double factor)
{
    const double f = dmax(1.0, factor);
    return pr->rho <= f * o->atmo_rho_floor &&
           pr->p <= f * o->atmo_pressure_floor;
}

static int prim_differs(const Prim *a, const Prim *b)
{
    int d = a->rho != b->rho || a->eps != b->eps || a->p != b->p;
    for (int i = 0; i < 3; ++i)
        d = d || a->v[i] != b->v[i];
    return d;
}

/* ------------------------------------------------------------------------ */
/* reconstruction and Riemann solver                                         */
/* ------------------------------------------------------------------------ */

/* Reconstruction.hpp:16-27 */
static double minmod2(double l, double r)
{
    if (l * r <= 0.0)
        return 0.0;
    return l > 0.0 ? dmin(l, r) : dmax(l, r);
}

/* compute_limited_slope, Reconstruction.hpp:29-37 */
static double limited_slope(double l, double c, double r, double theta)
{
    return minmod2(theta * (c - l), minmod2(0.5 * (r - l), theta * (r - c)));
}

static Prim prim_slope(const Prim *l, const Prim *c, const Prim *r,
                       double theta)
{
    Prim s;
    s.rho = limited_slope(l->rho, c->rho, r->rho, theta);
    s.eps = limited_slope(l->eps, c->eps, r->eps, theta);
    s.p = limited_slope(l->p, c->p, r->p, theta);
    for (int i = 0; i < 3; ++i)
        s.v[i] = limited_slope(l->v[i], c->v[i], r->v[i], theta);
    return s;
}

/* add_scaled, Reconstruction.hpp:59-69 */
static Prim prim_add_scaled(const Prim *pr, const Prim *s, double scale)
{
    Prim o;
    o.rho = pr->rho + scale * s->rho;
    o.eps = pr->eps + scale * s->eps;
    o.p = pr->p + scale * s->p;
    for (int i = 0; i < 3; ++i)
        o.v[i] = pr->v[i] + scale * s->v[i];
    return o;
}

/* compute_characteristic_speeds (+ shifted), RiemannSolvers.hpp:23-67 */
static void char_speeds(double G, const Prim *pr, const double gLL[3][3],
                        const double gUU[3][3], int d, double lapse,
                        const double shift[3], double *lo, double *hi)
{
    const double v2 = velocity_squared(pr->v, gLL);
    const double cs2 = eos_cs2(G, pr->rho, pr->eps, pr->p);
    const double cs = sqrt(cs2);
    const double vel = pr->v[d];
    const double den = 1.0 - v2 * cs2;
    const double rad = (1.0 - v2) * (gUU[d][d] * (1.0 - v2 * cs2) -
                                     vel * vel * (1.0 - cs2));
    const double root = cs * sqrt(dmax(0.0, rad));
    const double l = (vel * (1.0 - cs2) - root) / den;
    const double u = (vel * (1.0 - cs2) + root) / den;
    *lo = lapse * l - shift[d];
    *hi = lapse * u - shift[d];
}

/* compute_hlle_flux, RiemannSolvers.hpp:69-118 */
static Flux hlle(double G, const Prim *lp, const Prim *rp, const Cons *lc,
                 const Cons *rc, const double gLL[3][3],
                 const double gUU[3][3], int d, double lapse,
                 const double shift[3])
{
    const Flux lf = phys_flux(lp, lc, d, lapse, shift);
    const Flux rf = phys_flux(rp, rc, d, lapse, shift);
    double llo, lhi, rlo, rhi;
    char_speeds(G, lp, gLL, gUU, d, lapse, shift, &llo, &lhi);
    char_speeds(G, rp, gLL, gUU, d, lapse, shift, &rlo, &rhi);
    const double sl = dmin(0.0, dmin(llo, rlo));
    const double su = dmax(0.0, dmax(lhi, rhi));
    if (sl >= 0.0)
        return lf;
    if (su <= 0.0)
        return rf;
    Flux f;
    const double inv = 1.0 / (su - sl);
    f.D = (su * lf.D - sl * rf.D + sl * su * (rc->D - lc->D)) * inv;
    f.tau = (su * lf.tau - sl * rf.tau + sl * su * (rc->tau - lc->tau)) * inv;
    for (int i = 0; i < 3; ++i)
        f.S[i] = (su * lf.S[i] - sl * rf.S[i] + sl * su * (rc->S[i] - lc->S[i])) *
                 inv;
    return f;
}

/* compute_muscl_hlle_flux, FiniteVolume.hpp:63-98 */
static Flux muscl_hlle(const orc_params *o, const Prim *lcell,
                       const Prim *rcell, const Prim *lslope,
                       const Prim *rslope, const Geom *g, int d)
{
    Prim lp = *lcell, rp = *rcell;
    if (o->use_reconstruction)
    {
        lp = prim_add_scaled(lcell, lslope, 0.5);
        rp = prim_add_scaled(rcell, rslope, -0.5);
    }
    enforce_floors(o, &lp, g->gLL);
    enforce_floors(o, &rp, g->gLL);
    const Cons lc = p2c(o->gamma, &lp, g->gLL);
    const Cons rc = p2c(o->gamma, &rp, g->gLL);
    return hlle(o->gamma, &lp, &rp, &lc, &rc, g->gLL, g->gUU, d, g->lapse,
                g->shift);
}

/* ------------------------------------------------------------------------ */
/* geometric sources (StaticMetric.hpp:193-291)                               */
/* ------------------------------------------------------------------------ */

static void stress_UU(double G, const Prim *pr, const Geom *g,
                      double out[3][3])
{
    (void)G;
    const double W = 1.0 / sqrt(1.0 - velocity_squared(pr->v, g->gLL));
    const double h = eos_enthalpy(pr->rho, pr->eps, pr->p);
    const double rhw = pr->rho * h * W * W;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            out[i][j] = rhw * pr->v[i] * pr->v[j] + pr->p * g->gUU[i][j];
}

static Cons static_sources(double G, const Prim *pr, const Cons *c,
                           const Geom *g, const Derivs *dv)
{
    Cons s;
    memset(&s, 0, sizeof(s));
    double st[3][3];
    stress_UU(G, pr, g, st);
    const double E = c->D + c->tau;
    double mU[3] = {0, 0, 0};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            mU[i] += g->gUU[i][j] * c->S[j];
    Flux F[3];
    for (int d = 0; d < 3; ++d)
        F[d] = phys_flux(pr, c, d, g->lapse, g->shift);
    for (int d = 0; d < 3; ++d)
    {
        s.D -= F[d].D * dv->dlnsqrtg[d];
        s.tau -= F[d].tau * dv->dlnsqrtg[d];
        s.tau -= mU[d] * dv->dlapse[d];
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            s.tau += g->lapse * st[i][j] * g->K[i][j];
    for (int m = 0; m < 3; ++m)
    {
        double ms = -E * dv->dlapse[m];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                ms += 0.5 * g->lapse * st[i][j] * dv->dgamma[m][i][j];
        for (int sd = 0; sd < 3; ++sd)
            ms += c->S[sd] * dv->dshift[sd][m];
        for (int d = 0; d < 3; ++d)
            ms -= F[d].S[m] * dv->dlnsqrtg[d];
        s.S[m] += ms;
    }
    return s;
}

/* ------------------------------------------------------------------------ */
/* FAB access                                                                */
/* ------------------------------------------------------------------------ */

static int64_t fab_index(const orc_box *b, int i, int j, int k)
{
    const int64_t nx = b->ghi[0] - b->glo[0] + 1;
    const int64_t ny = b->ghi[1] - b->glo[1] + 1;
    return (i - b->glo[0]) + nx * ((j - b->glo[1]) + ny * (int64_t)(k - b->glo[2]));
}

static Cons load_cons(const orc_box *b, const double *s, int64_t idx)
{
    Cons c;
    const int64_t cs = b->comp_stride;
    c.D = s[ORC_D * cs + idx];
    c.S[0] = s[ORC_S1 * cs + idx];
    c.S[1] = s[ORC_S2 * cs + idx];
    c.S[2] = s[ORC_S3 * cs + idx];
    c.tau = s[ORC_TAU * cs + idx];
    return c;
}

static void store_cons(const orc_box *b, double *s, int64_t idx,
                       const Cons *c)
{
    const int64_t cs = b->comp_stride;
    s[ORC_D * cs + idx] = c->D;
    s[ORC_S1 * cs + idx] = c->S[0];
    s[ORC_S2 * cs + idx] = c->S[1];
    s[ORC_S3 * cs + idx] = c->S[2];
    s[ORC_TAU * cs + idx] = c->tau;
}

static Prim load_prim(const orc_box *b, const double *s, int64_t idx)
{
    Prim p;
    const int64_t cs = b->comp_stride;
    p.rho = s[ORC_RHO * cs + idx];
    p.eps = s[ORC_EPS * cs + idx];
    p.p = s[ORC_PRESS * cs + idx];
    p.v[0] = s[ORC_V1 * cs + idx];
    p.v[1] = s[ORC_V2 * cs + idx];
    p.v[2] = s[ORC_V3 * cs + idx];
    return p;
}

static void store_prim(const orc_box *b, double *s, int64_t idx,
                       const Prim *p)
{
    const int64_t cs = b->comp_stride;
    s[ORC_RHO * cs + idx] = p->rho;
    s[ORC_EPS * cs + idx] = p->eps;
    s[ORC_PRESS * cs + idx] = p->p;
    s[ORC_V1 * cs + idx] = p->v[0];
    s[ORC_V2 * cs + idx] = p->v[1];
    s[ORC_V3 * cs + idx] = p->v[2];
}

/* New: a cell is excised when its coordinate radius (relative to the
 * operator centre) is below excision_radius; semantics follow
 * Source/Background/ExcisionEvolution.hpp:37-50 (RHS := 0 inside), with the
 * state held frozen so the cell still serves as a stencil neighbour. */
static int is_excised(const orc_params *p, int i, int j, int k)
{
    if (!(p->excision_radius > 0.0))
        return 0;
    double x, y, z;
    cell_position(p, i, j, k, &x, &y, &z);
    return sqrt(x * x + y * y + z * z) < p->excision_radius;
}

static void set_error(orc_error *err, int code, int where, int i, int j,
                      int k, double residual)
{
    if (!err || err->code != ORC_OK)
        return;
    err->code = code;
    err->where = where;
    err->cell[0] = i;
    err->cell[1] = j;
    err->cell[2] = k;
    err->residual = residual;
}

/* ------------------------------------------------------------------------ */
/* box operators                                                             */
/* ------------------------------------------------------------------------ */

/* fill_conserved_outflow_boundaries_from_fixed_background,
 * FixedBGFArrayBoxFiniteVolume.hpp:113-177.  The ghosted box of a box of
 * the level is the box grown by the storage ghost width. */
static int fill_outflow(const orc_params *o, const orc_box *b,
                        const int lo[3], const int hi[3], const int glo[3],
                        const int ghi[3], double *state, double t,
                        orc_error *err)
{
    for (int k = glo[2]; k <= ghi[2]; ++k)
        for (int j = glo[1]; j <= ghi[1]; ++j)
            for (int i = glo[0]; i <= ghi[0]; ++i)
            {
                const int iv[3] = {i, j, k};
                int src[3] = {i, j, k};
                int ghost = 0;
                for (int d = 0; d < 3; ++d)
                {
                    if (iv[d] < b->dlo[d])
                    {
                        ghost = 1;
                        src[d] = lo[d];
                    }
                    else if (iv[d] > b->dhi[d])
                    {
                        ghost = 1;
                        src[d] = hi[d];
                    }
                }
                if (!ghost)
                    continue;
                Geom sg, tg;
                load_geometry(o, t, src[0], src[1], src[2], &sg);
                const Cons sc =
                    load_cons(b, state, fab_index(b, src[0], src[1], src[2]));
                Prim pr;
                int it;
                double res;
                if (!con2prim(o, &sc, sg.gUU, &pr, &it, &res))
                {
                    set_error(err, ORC_ERR_RECOVERY, ORC_WHERE_OUTFLOW_SOURCE,
                              src[0], src[1], src[2], res);
                    return ORC_ERR_RECOVERY;
                }
                load_geometry(o, t, i, j, k, &tg);
                enforce_floors(o, &pr, tg.gLL);
                const int64_t idx = fab_index(b, i, j, k);
                store_prim(b, state, idx, &pr);
                const Cons c = p2c(o->gamma, &pr, tg.gLL);
                store_cons(b, state, idx, &c);
            }
    return ORC_OK;
}

/* One box's flux RHS plus sources: compute_leveldata_flux_rhs_from_fixed_
 * background for a single box (FixedBGFArrayBoxFiniteVolume.hpp:199-253,
 * 255-298, 322-363), with the time-dependent volume source of :616-675.
 * lo/hi: the box's interior; glo/ghi: its ghosted box; rhs is indexed over
 * the interior box of the whole array `b` via rhs_index. */
static int inside_sphere(const orc_params *o, int i, int j, int k)
{
    double x, y, z;
    cell_position(o, i, j, k, &x, &y, &z);
    return sqrt(x * x + y * y + z * z) < o->accretion_radius;
}

static int box_rhs(const orc_params *o, const orc_box *b, const int lo[3],
                   const int hi[3], double *state, double *rhs,
                   int64_t rcs, const orc_box *rb, const double inv_dx[3],
                   double t, int do_outflow, orc_error *err, double *mdot)
{
    int glo[3], ghi[3];
    for (int d = 0; d < 3; ++d)
    {
        glo[d] = lo[d] - 2;
        ghi[d] = hi[d] + 2;
    }
    const int gnx = ghi[0] - glo[0] + 1, gny = ghi[1] - glo[1] + 1,
              gnz = ghi[2] - glo[2] + 1;
    const int64_t gvol = (int64_t)gnx * gny * gnz;
#define GIDX(i, j, k)                                                         \
    ((int64_t)((i)-glo[0]) + gnx * ((int64_t)((j)-glo[1]) + gny * ((k)-glo[2])))
#define RIDX(i, j, k)                                                         \
    ((int64_t)((i)-rb->lo[0]) +                                               \
     (int64_t)(rb->hi[0] - rb->lo[0] + 1) *                                   \
         ((int64_t)((j)-rb->lo[1]) +                                          \
          (int64_t)(rb->hi[1] - rb->lo[1] + 1) * ((k)-rb->lo[2])))

    Prim *prims = (Prim *)calloc(gvol, sizeof(Prim));
    Prim *slopes = (Prim *)calloc(gvol, sizeof(Prim));
    double *drhs = (double *)calloc(5 * (size_t)gvol, sizeof(double));
    int status = ORC_OK;

    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i)
            {
                const int64_t r = RIDX(i, j, k);
                for (int c = 0; c < 5; ++c)
                    rhs[c * rcs + r] = 0.0;
            }

    for (int dir = 0; dir < 3 && status == ORC_OK; ++dir)
    {
        if (do_outflow)
        {
            status = fill_outflow(o, b, lo, hi, glo, ghi, state, t, err);
            if (status != ORC_OK)
                break;
        }
        /* recover_primitives_from_fixed_background over the ghosted box,
         * :33-58 (no floors; failure throws). */
        for (int k = glo[2]; k <= ghi[2] && status == ORC_OK; ++k)
            for (int j = glo[1]; j <= ghi[1] && status == ORC_OK; ++j)
                for (int i = glo[0]; i <= ghi[0]; ++i)
                {
                    const int64_t sidx = fab_index(b, i, j, k);
                    if (is_excised(o, i, j, k) && i >= b->lo[0] &&
                        i <= b->hi[0] && j >= b->lo[1] && j <= b->hi[1] &&
                        k >= b->lo[2] && k <= b->hi[2])
                    {
                        prims[GIDX(i, j, k)] = load_prim(b, state, sidx);
                        continue;
                    }
                    Geom g;
                    load_geometry(o, t, i, j, k, &g);
                    const Cons c = load_cons(b, state, sidx);
                    int it;
                    double res;
                    if (!con2prim(o, &c, g.gUU, &prims[GIDX(i, j, k)], &it,
                                  &res))
                    {
                        set_error(err, ORC_ERR_RECOVERY,
                                  ORC_WHERE_GHOSTED_RECOVERY, i, j, k, res);
                        status = ORC_ERR_RECOVERY;
                        break;
                    }
                }
        if (status != ORC_OK)
            break;

        /* compute_primitive_slopes on the ghosted box shrunk along dir,
         * FArrayBoxFiniteVolume.hpp:573-589 */
        memset(slopes, 0, gvol * sizeof(Prim));
        const int off[3] = {dir == 0, dir == 1, dir == 2};
        for (int k = glo[2] + off[2]; k <= ghi[2] - off[2]; ++k)
            for (int j = glo[1] + off[1]; j <= ghi[1] - off[1]; ++j)
                for (int i = glo[0] + off[0]; i <= ghi[0] - off[0]; ++i)
                    slopes[GIDX(i, j, k)] = prim_slope(
                        &prims[GIDX(i - off[0], j - off[1], k - off[2])],
                        &prims[GIDX(i, j, k)],
                        &prims[GIDX(i + off[0], j + off[1], k + off[2])],
                        o->limiter_theta);

        /* hot loop, FixedBGFArrayBoxFiniteVolume.hpp:229-252 */
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i)
                {
                    Flux fx[2];
                    for (int side = 0; side < 2; ++side)
                    {
                        /* side 0: face i+1/2 (left = iv); side 1: i-1/2 */
                        const int li = i - (side ? off[0] : 0);
                        const int lj = j - (side ? off[1] : 0);
                        const int lk = k - (side ? off[2] : 0);
                        const int ri = li + off[0], rj = lj + off[1],
                                  rk = lk + off[2];
                        Geom gl, gr, gf;
                        load_geometry(o, t, li, lj, lk, &gl);
                        load_geometry(o, t, ri, rj, rk, &gr);
                        average_geometry(&gl, &gr, &gf);
                        fx[side] = muscl_hlle(
                            o, &prims[GIDX(li, lj, lk)],
                            &prims[GIDX(ri, rj, rk)],
                            &slopes[GIDX(li, lj, lk)],
                            &slopes[GIDX(ri, rj, rk)], &gf, dir);
                        /* new: rest-mass flux through the faces of the
                         * voxelised sphere r < R, each face once (as the
                         * high face of its left cell) */
                        if (mdot && side == 0 && o->accretion_radius > 0.0)
                        {
                            const int in_l = inside_sphere(o, li, lj, lk);
                            const int in_r = inside_sphere(o, ri, rj, rk);
                            if (in_l != in_r)
                            {
                                const double sg = sqrt(det_sym(gf.gLL));
                                const double dA = o->dx * o->dx;
                                /* outward normal +d when the left cell is
                                 * inside; Mdot = - outward flux */
                                *mdot += (in_l ? -1.0 : 1.0) * sg *
                                         fx[side].D * dA;
                            }
                        }
                    }
                    const int64_t g = GIDX(i, j, k);
                    const double idx_d = inv_dx[dir];
                    double cr[5];
                    cr[0] = -idx_d * (fx[0].D - fx[1].D);
                    cr[4] = -idx_d * (fx[0].tau - fx[1].tau);
                    for (int m = 0; m < 3; ++m)
                        cr[1 + m] = -idx_d * (fx[0].S[m] - fx[1].S[m]);
                    for (int c = 0; c < 5; ++c)
                        drhs[c * gvol + g] = cr[c];
                }
        /* add_conserved_rhs, FArrayBoxFiniteVolume.hpp:912-925 */
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i)
                {
                    const int64_t r = RIDX(i, j, k), g = GIDX(i, j, k);
                    for (int c = 0; c < 5; ++c)
                        rhs[c * rcs + r] += drhs[c * gvol + g];
                }
    }

    /* add_static_metric_sources_from_fixed_background_to_conserved_rhs,
     * FixedBGFArrayBoxFiniteVolume.hpp:255-298 */
    if (status == ORC_OK && o->use_static_metric_sources)
    {
        for (int k = lo[2]; k <= hi[2] && status == ORC_OK; ++k)
            for (int j = lo[1]; j <= hi[1] && status == ORC_OK; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i)
                {
                    if (is_excised(o, i, j, k))
                        continue;
                    Geom g;
                    load_geometry(o, t, i, j, k, &g);
                    const Cons c = load_cons(b, state, fab_index(b, i, j, k));
                    Prim pr;
                    int it;
                    double res;
                    if (!con2prim(o, &c, g.gUU, &pr, &it, &res))
                    {
                        set_error(err, ORC_ERR_RECOVERY,
                                  ORC_WHERE_METRIC_SOURCES, i, j, k, res);
                        status = ORC_ERR_RECOVERY;
                        break;
                    }
                    enforce_floors(o, &pr, g.gLL);
                    if (is_atmosphere(o, &pr,
                                      o->atmo_metric_source_atmosphere_factor))
                        continue;
                    Derivs dv;
                    load_derivs(o, t, i, j, k, &dv);
                    const Cons s = static_sources(o->gamma, &pr, &c, &g, &dv);
                    const int64_t r = RIDX(i, j, k);
                    rhs[0 * rcs + r] += s.D;
                    rhs[4 * rcs + r] += s.tau;
                    for (int m = 0; m < 3; ++m)
                        rhs[(1 + m) * rcs + r] += s.S[m];
                }
    }

    /* add_metric_volume_time_sources_from_fixed_background_to_conserved_rhs,
     * :633-657, with fixed_background_log_sqrt_det_time_derivative :616-631 */
    if (status == ORC_OK && o->use_metric_volume_time_sources)
    {
        const double h = dmax(o->metric_time_derivative_step, 1.0e-12);
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i)
                {
                    if (is_excised(o, i, j, k))
                        continue;
                    Geom gp, gm;
                    load_geometry(o, t + h, i, j, k, &gp);
                    load_geometry(o, t - h, i, j, k, &gm);
                    const double dl =
                        (log_sqrt_det(&gp) - log_sqrt_det(&gm)) / (2.0 * h);
                    const Cons c = load_cons(b, state, fab_index(b, i, j, k));
                    const int64_t r = RIDX(i, j, k);
                    rhs[0 * rcs + r] += 0.0 - c.D * dl;
                    rhs[4 * rcs + r] += 0.0 - c.tau * dl;
                    for (int m = 0; m < 3; ++m)
                        rhs[(1 + m) * rcs + r] += 0.0 - c.S[m] * dl;
                }
    }

    /* new: excised cells have a zero right-hand side */
    if (status == ORC_OK && o->excision_radius > 0.0)
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i)
                    if (is_excised(o, i, j, k))
                    {
                        const int64_t r = RIDX(i, j, k);
                        for (int c = 0; c < 5; ++c)
                            rhs[c * rcs + r] = 0.0;
                    }
#undef GIDX
#undef RIDX
    free(prims);
    free(slopes);
    free(drhs);
    return status;
}

static int check_box(const orc_box *b)
{
    for (int d = 0; d < 3; ++d)
        if (b->lo[d] > b->hi[d] || b->glo[d] > b->lo[d] - 2 ||
            b->ghi[d] < b->hi[d] + 2)
            return 0;
    return 1;
}

int orc_compute_rhs(const orc_params *p, const orc_box *box, double *state,
                    double *rhs, int64_t rcs, const double inv_dx[3],
                    double time, orc_error *err)
{
    if (err)
        memset(err, 0, sizeof(*err));
    if (!check_box(box) || !(p->dx > 0.0))
        return ORC_ERR_INVALID_ARG;
    return box_rhs(p, box, box->lo, box->hi, state, rhs, rcs, box, inv_dx,
                   time, 1, err, NULL);
}

typedef struct
{
    const orc_params *p;
    const orc_box *box;
    double *state, *rhs;
    int64_t rcs;
    const double *inv_dx;
    double time;
    int lo[3], hi[3];
    int status;
    orc_error err;
} SlabJob;

/* One reference box per worker thread: the box's own ghosted-box recovery,
 * slopes, faces and sources, as one MPI rank would run it. */
static void *slab_worker(void *arg)
{
    SlabJob *j = (SlabJob *)arg;
    memset(&j->err, 0, sizeof(j->err));
    j->status = box_rhs(j->p, j->box, j->lo, j->hi, j->state, j->rhs, j->rcs,
                        j->box, j->inv_dx, j->time, 0, &j->err, NULL);
    return NULL;
}

int orc_compute_rhs_mdot(const orc_params *p, const orc_box *box,
                         double *state, double *rhs, int64_t rcs,
                         const double inv_dx[3], double time, double *mdot,
                         orc_error *err)
{
    if (err)
        memset(err, 0, sizeof(*err));
    if (!check_box(box) || !(p->dx > 0.0))
        return ORC_ERR_INVALID_ARG;
    *mdot = 0.0;
    return box_rhs(p, box, box->lo, box->hi, state, rhs, rcs, box, inv_dx,
                   time, 1, err, mdot);
}

int orc_compute_rhs_slabs(const orc_params *p, const orc_box *box,
                          double *state, double *rhs, int64_t rcs,
                          const double inv_dx[3], double time, int num_slabs,
                          orc_error *err)
{
    if (err)
        memset(err, 0, sizeof(*err));
    if (!check_box(box) || num_slabs < 1)
        return ORC_ERR_INVALID_ARG;
    /* Physical ghosts are filled once for the whole level (each box of the
     * reference fills the physical ghosts of its own ghosted box with the
     * same values); internal ghosts are the neighbours' interior, as after
     * LevelData::exchange(). */
    int glo[3], ghi[3];
    for (int d = 0; d < 3; ++d)
    {
        glo[d] = box->lo[d] - 2;
        ghi[d] = box->hi[d] + 2;
    }
    int st = fill_outflow(p, box, box->lo, box->hi, glo, ghi, state, time, err);
    if (st != ORC_OK)
        return st;
    const int nz = box->hi[2] - box->lo[2] + 1;
    if (num_slabs > nz)
        num_slabs = nz;
    SlabJob *jobs = (SlabJob *)calloc(num_slabs, sizeof(SlabJob));
    pthread_t *threads = (pthread_t *)calloc(num_slabs, sizeof(pthread_t));
    for (int s = 0; s < num_slabs; ++s)
    {
        SlabJob *j = &jobs[s];
        j->p = p;
        j->box = box;
        j->state = state;
        j->rhs = rhs;
        j->rcs = rcs;
        j->inv_dx = inv_dx;
        j->time = time;
        j->lo[0] = box->lo[0];
        j->lo[1] = box->lo[1];
        j->lo[2] = box->lo[2] + (nz * s) / num_slabs;
        j->hi[0] = box->hi[0];
        j->hi[1] = box->hi[1];
        j->hi[2] = box->lo[2] + (nz * (s + 1)) / num_slabs - 1;
        pthread_create(&threads[s], NULL, slab_worker, j);
    }
    int status = ORC_OK;
    for (int s = 0; s < num_slabs; ++s)
    {
        pthread_join(threads[s], NULL);
        if (status == ORC_OK && jobs[s].status != ORC_OK)
        {
            status = jobs[s].status;
            if (err)
                *err = jobs[s].err;
        }
    }
    free(jobs);
    free(threads);
    return status;
}

/* ------------------------------------------------------------------------ */
/* z-parallel loops for the setup passes (initial data, recovery).  Cells   */
/* are independent in these passes, so splitting k changes no result.      */
/* ------------------------------------------------------------------------ */

static int g_threads = 1;

void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

typedef void (*zrange_fn)(void *ctx, int k0, int k1, int slot);

typedef struct
{
    zrange_fn fn;
    void *ctx;
    int k0, k1, slot;
} ZJob;

static void *zjob_run(void *arg)
{
    ZJob *j = (ZJob *)arg;
    j->fn(j->ctx, j->k0, j->k1, j->slot);
    return NULL;
}

/* Runs fn over [klo, khi] split into at most g_threads contiguous chunks;
 * returns the number of slots used. */
static int parallel_z(int klo, int khi, zrange_fn fn, void *ctx, int max_slots)
{
    const int nz = khi - klo + 1;
    int n = g_threads < max_slots ? g_threads : max_slots;
    if (n > nz)
        n = nz;
    if (n <= 1)
    {
        fn(ctx, klo, khi, 0);
        return 1;
    }
    ZJob jobs[256];
    pthread_t th[256];
    for (int s = 0; s < n; ++s)
    {
        jobs[s].fn = fn;
        jobs[s].ctx = ctx;
        jobs[s].k0 = klo + (nz * s) / n;
        jobs[s].k1 = klo + (nz * (s + 1)) / n - 1;
        jobs[s].slot = s;
        pthread_create(&th[s], NULL, zjob_run, &jobs[s]);
    }
    for (int s = 0; s < n; ++s)
        pthread_join(th[s], NULL);
    return n;
}

static void recover_range(const orc_params *o, const orc_box *b,
                          double *state, double t, int k0, int k1,
                          orc_diag *out);

typedef struct
{
    const orc_params *o;
    const orc_box *b;
    double *state;
    double t;
    orc_diag d[256];
} RecoverCtx;

static void recover_job(void *ctx, int k0, int k1, int slot)
{
    RecoverCtx *c = (RecoverCtx *)ctx;
    recover_range(c->o, c->b, c->state, c->t, k0, k1, &c->d[slot]);
}

/* recover_primitives_and_apply_atmosphere_from_fixed_background,
 * FixedBGFArrayBoxFiniteVolume.hpp:60-110 */
int orc_recover_primitives(const orc_params *o, const orc_box *b,
                           double *state, double t, orc_diag *diag)
{
    RecoverCtx *c = (RecoverCtx *)calloc(1, sizeof(RecoverCtx));
    c->o = o;
    c->b = b;
    c->state = state;
    c->t = t;
    const int n = parallel_z(b->lo[2], b->hi[2], recover_job, c, 256);
    if (diag)
        for (int s = 0; s < n; ++s)
        {
            diag->num_cells += c->d[s].num_cells;
            diag->num_failed_recoveries += c->d[s].num_failed_recoveries;
            diag->num_floored_primitives += c->d[s].num_floored_primitives;
            diag->num_conserved_resets += c->d[s].num_conserved_resets;
        }
    free(c);
    return ORC_OK;
}

static void recover_range(const orc_params *o, const orc_box *b,
                          double *state, double t, int k0, int k1,
                          orc_diag *diag)
{
    orc_diag dg;
    memset(&dg, 0, sizeof(dg));
    for (int k = k0; k <= k1; ++k)
        for (int j = b->lo[1]; j <= b->hi[1]; ++j)
            for (int i = b->lo[0]; i <= b->hi[0]; ++i)
            {
                if (is_excised(o, i, j, k))
                    continue;
                ++dg.num_cells;
                Geom g;
                load_geometry(o, t, i, j, k, &g);
                const int64_t idx = fab_index(b, i, j, k);
                const Cons c = load_cons(b, state, idx);
                Prim pr;
                int it;
                double res;
                const int ok = con2prim(o, &c, g.gUU, &pr, &it, &res);
                int reset = !ok;
                if (ok)
                {
                    Prim fl = pr;
                    enforce_floors(o, &fl, g.gLL);
                    reset = prim_differs(&pr, &fl);
                    if (reset)
                        ++dg.num_floored_primitives;
                    pr = fl;
                }
                else
                {
                    ++dg.num_failed_recoveries;
                    pr = atmosphere_prim(o);
                }
                store_prim(b, state, idx, &pr);
                if (reset)
                {
                    ++dg.num_conserved_resets;
                    const Cons nc = p2c(o->gamma, &pr, g.gLL);
                    store_cons(b, state, idx, &nc);
                }
            }
    *diag = dg;
}

/* compute_max_inverse_dt_from_fixed_background, :364-412 */
/* compute_max_inverse_dt of a box (:364-444), over the z planes k0..k1. */
typedef struct
{
    const orc_params *o;
    const orc_box *b;
    const double *state;
    const double *inv_dx;
    double t;
    double mx[256];
    int status[256];
    orc_error err[256];
} CflJob;

static void cfl_job(void *ctx, int k0, int k1, int slot)
{
    CflJob *c = (CflJob *)ctx;
    const orc_params *o = c->o;
    const orc_box *b = c->b;
    double mx = 0.0;
    c->status[slot] = ORC_OK;
    memset(&c->err[slot], 0, sizeof(orc_error));
    for (int k = k0; k <= k1; ++k)
        for (int j = b->lo[1]; j <= b->hi[1]; ++j)
            for (int i = b->lo[0]; i <= b->hi[0]; ++i)
            {
                if (is_excised(o, i, j, k))
                    continue;
                Geom g;
                load_geometry(o, c->t, i, j, k, &g);
                const Cons cs = load_cons(b, c->state, fab_index(b, i, j, k));
                Prim pr;
                int it;
                double res;
                if (!con2prim(o, &cs, g.gUU, &pr, &it, &res))
                {
                    set_error(&c->err[slot], ORC_ERR_RECOVERY, ORC_WHERE_CFL,
                              i, j, k, res);
                    c->status[slot] = ORC_ERR_RECOVERY;
                    c->mx[slot] = mx;
                    return;
                }
                enforce_floors(o, &pr, g.gLL);
                if (is_atmosphere(o, &pr, 1.0 + 1.0e-12))
                    continue;
                double cell = 0.0;
                for (int d = 0; d < 3; ++d)
                {
                    double lo, hi;
                    char_speeds(o->gamma, &pr, g.gLL, g.gUU, d, g.lapse,
                                g.shift, &lo, &hi);
                    cell += dmax(fabs(lo), fabs(hi)) * c->inv_dx[d];
                }
                mx = dmax(mx, cell);
            }
    c->mx[slot] = mx;
}

/* The maximum is exact, so splitting the planes over threads changes no
 * result; the error reported is the first failing cell in the box's
 * iteration order (the lowest failing slot's first failure). */
int orc_compute_max_inverse_dt(const orc_params *o, const orc_box *b,
                               const double *state, const double inv_dx[3],
                               double t, double *out, orc_error *err)
{
    if (err)
        memset(err, 0, sizeof(*err));
    CflJob *c = (CflJob *)calloc(1, sizeof(CflJob));
    c->o = o;
    c->b = b;
    c->state = state;
    c->inv_dx = inv_dx;
    c->t = t;
    const int n = parallel_z(b->lo[2], b->hi[2], cfl_job, c, 256);
    double mx = 0.0;
    int status = ORC_OK;
    for (int s = 0; s < n; ++s)
    {
        if (c->status[s] != ORC_OK)
        {
            status = c->status[s];
            if (err)
                *err = c->err[s];
            break;
        }
        mx = dmax(mx, c->mx[s]);
    }
    free(c);
    if (status != ORC_OK)
        return status;
    *out = mx;
    return ORC_OK;
}

/* compute_stable_dt, :544-555 */
int orc_compute_stable_dt(const orc_params *o, const orc_box *b,
                          const double *state, const double inv_dx[3],
                          double cfl, double t, double *out, orc_error *err)
{
    if (err)
        memset(err, 0, sizeof(*err));
    if (cfl <= 0.0)
    {
        if (err)
            err->code = ORC_ERR_INVALID_ARG;
        return ORC_ERR_INVALID_ARG;
    }
    double m;
    int st = orc_compute_max_inverse_dt(o, b, state, inv_dx, t, &m, err);
    if (st != ORC_OK)
        return st;
    *out = cfl / dmax(m, 1.0e-14);
    return ORC_OK;
}

/* update_conserved: add_scaled_conserved_rhs (FArrayBoxFiniteVolume.hpp:
 * 927-940) then recover_primitives, FixedBGFArrayBoxFiniteVolume.hpp:522-533 */
int orc_update_conserved(const orc_params *o, const orc_box *b,
                         double *state, const double *rhs, int64_t rcs,
                         double dt, double recovery_time, int recover,
                         orc_diag *diag)
{
    const int64_t nx = b->hi[0] - b->lo[0] + 1, ny = b->hi[1] - b->lo[1] + 1;
    for (int k = b->lo[2]; k <= b->hi[2]; ++k)
        for (int j = b->lo[1]; j <= b->hi[1]; ++j)
            for (int i = b->lo[0]; i <= b->hi[0]; ++i)
            {
                const int64_t s = fab_index(b, i, j, k);
                const int64_t r =
                    (i - b->lo[0]) + nx * ((j - b->lo[1]) + ny * (int64_t)(k - b->lo[2]));
                state[ORC_D * b->comp_stride + s] += dt * rhs[0 * rcs + r];
                state[ORC_TAU * b->comp_stride + s] += dt * rhs[4 * rcs + r];
                state[ORC_S1 * b->comp_stride + s] += dt * rhs[1 * rcs + r];
                state[ORC_S2 * b->comp_stride + s] += dt * rhs[2 * rcs + r];
                state[ORC_S3 * b->comp_stride + s] += dt * rhs[3 * rcs + r];
            }
    if (recover)
        return orc_recover_primitives(o, b, state, recovery_time, diag);
    return ORC_OK;
}

static size_t box_state_doubles(const orc_box *b)
{
    return (size_t)b->comp_stride * ORC_NCOMP;
}

static size_t box_interior_cells(const orc_box *b)
{
    return (size_t)(b->hi[0] - b->lo[0] + 1) * (b->hi[1] - b->lo[1] + 1) *
           (b->hi[2] - b->lo[2] + 1);
}

/* The RHS of an integrator stage: the single reference box, or -- when
 * several threads are set and no accretion integral is wanted -- the same
 * box cut into z-slab boxes, one thread each (orc_compute_rhs_slabs).  The
 * two give the same RHS bit for bit: the slabs fill the level's physical
 * ghosts with the single box's values, and every cell's faces and sources
 * read the same neighbours. */
static int stage_rhs(const orc_params *o, const orc_box *b, double *state,
                     double *rhs, int64_t nr, const double inv_dx[3],
                     double t, double *mdot, orc_error *err)
{
    if (g_threads > 1 && mdot == NULL)
        return orc_compute_rhs_slabs(o, b, state, rhs, nr, inv_dx, t,
                                     g_threads, err);
    double m = 0.0;
    const int st = orc_compute_rhs_mdot(o, b, state, rhs, nr, inv_dx, t, &m,
                                        err);
    if (mdot)
        *mdot = m;
    return st;
}

/* advance_ssprk2 of the time-dependent operator, :782-809 (the static
 * operator, :563-589, is the same with time ignored by the background). */
int orc_advance_ssprk2(const orc_params *o, const orc_box *b, double *state,
                       const double inv_dx[3], double t, double dt,
                       orc_diag *diag, orc_error *err)
{
    return orc_advance_ssprk2_mdot(o, b, state, inv_dx, t, dt, diag, err,
                                   NULL);
}

/* SSPRK2 with the time integral of the accretion rate: U^{n+1} = U^n +
 * dt/2 L(U^n) + dt/2 L(U^1), so each stage's Mdot carries weight dt/2. */
int orc_advance_ssprk2_mdot(const orc_params *o, const orc_box *b,
                            double *state, const double inv_dx[3], double t,
                            double dt, orc_diag *diag, orc_error *err,
                            double *mdot_integral)
{
    const size_t ns = box_state_doubles(b);
    const size_t nr = box_interior_cells(b);
    double *old_state = (double *)malloc(ns * sizeof(double));
    double *stage = (double *)malloc(ns * sizeof(double));
    double *r0 = (double *)malloc(5 * nr * sizeof(double));
    double *r1 = (double *)malloc(5 * nr * sizeof(double));
    memcpy(old_state, state, ns * sizeof(double));
    memcpy(stage, state, ns * sizeof(double));
    double m0 = 0.0, m1 = 0.0;
    int st = stage_rhs(o, b, state, r0, nr, inv_dx, t,
                       mdot_integral ? &m0 : NULL, err);
    if (st == ORC_OK)
    {
        orc_update_conserved(o, b, stage, r0, nr, dt, t + dt, 1, diag);
        st = stage_rhs(o, b, stage, r1, nr, inv_dx, t + dt,
                       mdot_integral ? &m1 : NULL, err);
    }
    if (mdot_integral)
        *mdot_integral += 0.5 * dt * m0 + 0.5 * dt * m1;
    if (st == ORC_OK)
    {
        /* combine_ssprk2_conserved_state, FArrayBoxFiniteVolume.hpp:942-969 */
        const int64_t nx = b->hi[0] - b->lo[0] + 1, ny = b->hi[1] - b->lo[1] + 1;
        for (int k = b->lo[2]; k <= b->hi[2]; ++k)
            for (int j = b->lo[1]; j <= b->hi[1]; ++j)
                for (int i = b->lo[0]; i <= b->hi[0]; ++i)
                {
                    const int64_t s = fab_index(b, i, j, k);
                    const int64_t r = (i - b->lo[0]) +
                                      nx * ((j - b->lo[1]) + ny * (int64_t)(k - b->lo[2]));
                    for (int c = 0; c < 5; ++c)
                    {
                        const int64_t q = c * b->comp_stride + s;
                        state[q] = 0.5 * (old_state[q] + stage[q] +
                                          dt * r1[c * nr + r]);
                    }
                }
        orc_recover_primitives(o, b, state, t + dt, diag);
    }
    free(old_state);
    free(stage);
    free(r0);
    free(r1);
    return st;
}

/* New: classic four-stage Runge-Kutta with the reference's post-update
 * recovery (update_conserved semantics) after every stage.
 *   k1 = L(U^n, t)          U1 = U^n + (dt/2) k1   recover at t + dt/2
 *   k2 = L(U1, t + dt/2)    U2 = U^n + (dt/2) k2   recover at t + dt/2
 *   k3 = L(U2, t + dt/2)    U3 = U^n + dt k3       recover at t + dt
 *   k4 = L(U3, t + dt)      U^{n+1} = U^n + (dt/6)(((k1 + 2 k2) + 2 k3) + k4)
 *                                                  recover at t + dt       */
int orc_advance_rk4(const orc_params *o, const orc_box *b, double *state,
                    const double inv_dx[3], double t, double dt,
                    orc_diag *diag, orc_error *err)
{
    return orc_advance_rk4_mdot(o, b, state, inv_dx, t, dt, diag, err, NULL);
}

/* RK4 with the time integral of the accretion rate, weights dt/6 (1, 2, 2,
 * 1) -- the weights the stage fluxes carry in U^{n+1}. */
int orc_advance_rk4_mdot(const orc_params *o, const orc_box *b, double *state,
                         const double inv_dx[3], double t, double dt,
                         orc_diag *diag, orc_error *err,
                         double *mdot_integral)
{
    const size_t ns = box_state_doubles(b);
    const size_t nr = box_interior_cells(b);
    double *stage = (double *)malloc(ns * sizeof(double));
    double *k = (double *)malloc(5 * nr * sizeof(double));
    double *acc = (double *)malloc(5 * nr * sizeof(double));
    const double c_stage[3] = {0.5 * dt, 0.5 * dt, dt};
    const double t_stage[4] = {t, t + 0.5 * dt, t + 0.5 * dt, t + dt};
    const int64_t nx = b->hi[0] - b->lo[0] + 1, ny = b->hi[1] - b->lo[1] + 1;
    int st = ORC_OK;
    memcpy(stage, state, ns * sizeof(double));
    for (int s = 0; s < 4 && st == ORC_OK; ++s)
    {
        double ms = 0.0;
        st = stage_rhs(o, b, s == 0 ? state : stage, k, nr, inv_dx,
                       t_stage[s], mdot_integral ? &ms : NULL, err);
        if (st != ORC_OK)
            break;
        if (mdot_integral)
            *mdot_integral += (dt / 6.0) * ((s == 1 || s == 2) ? 2.0 : 1.0) * ms;
        for (int kk = b->lo[2]; kk <= b->hi[2]; ++kk)
            for (int j = b->lo[1]; j <= b->hi[1]; ++j)
                for (int i = b->lo[0]; i <= b->hi[0]; ++i)
                {
                    const int64_t q = fab_index(b, i, j, kk);
                    const int64_t r = (i - b->lo[0]) +
                                      nx * ((j - b->lo[1]) + ny * (int64_t)(kk - b->lo[2]));
                    for (int c = 0; c < 5; ++c)
                    {
                        const double kv = k[c * nr + r];
                        const double un = state[c * b->comp_stride + q];
                        double *a = &acc[c * nr + r];
                        if (s == 0)
                            *a = kv;
                        else if (s < 3)
                            *a = *a + 2.0 * kv;
                        if (s < 3)
                            stage[c * b->comp_stride + q] = un + c_stage[s] * kv;
                        else
                            stage[c * b->comp_stride + q] =
                                un + (dt / 6.0) * (*a + kv);
                    }
                }
        orc_recover_primitives(o, b, stage, s < 2 ? t + 0.5 * dt : t + dt,
                               diag);
    }
    if (st == ORC_OK)
    {
        /* copy the new interior (conserved and primitives) back; the ghosts
         * of `state` keep the physical-ghost fill of the first stage, as in
         * the reference's advance_ssprk2. */
        for (int kk = b->lo[2]; kk <= b->hi[2]; ++kk)
            for (int j = b->lo[1]; j <= b->hi[1]; ++j)
                for (int i = b->lo[0]; i <= b->hi[0]; ++i)
                {
                    const int64_t q = fab_index(b, i, j, kk);
                    for (int c = 0; c < ORC_NCOMP; ++c)
                        state[c * b->comp_stride + q] =
                            stage[c * b->comp_stride + q];
                }
    }
    free(stage);
    free(k);
    free(acc);
    return st;
}

/* ------------------------------------------------------------------------ */
/* pointwise exports                                                         */
/* ------------------------------------------------------------------------ */

void orc_default_params(orc_params *p)
{
    memset(p, 0, sizeof(*p));
    p->background = ORC_BG_KERR_SCHILD;
    p->ks_mass = 1.0;
    p->ks_spin = 0.0;
    p->pn_mass_1 = 0.5;
    p->pn_mass_2 = 0.5;
    p->pn_separation = 10.0;
    p->pn_softening_radius = 0.5;
    p->gamma = 5.0 / 3.0;
    p->dx = 1.0;
    p->atmo_rho_floor = 1.0e-12;
    p->atmo_pressure_floor = 1.0e-12;
    p->atmo_max_velocity_squared = 1.0 - 1.0e-12;
    p->atmo_metric_source_atmosphere_factor = 1.0 + 1.0e-12;
    p->rec_max_iterations = 50;
    p->rec_tolerance = 1.0e-12;
    p->rec_pressure_floor = 1.0e-12;
    p->rec_max_velocity_squared = 1.0 - 1.0e-12;
    p->limiter_theta = 1.5;
    p->use_reconstruction = 1;
    p->use_static_metric_sources = 1;
    p->use_metric_volume_time_sources = 0;
    p->metric_time_derivative_step = 1.0e-3;
    p->excision_radius = 0.0;
    p->accretion_radius = 0.0;
}

void orc_background_vars(const orc_params *p, double t, double x, double y,
                         double z, double *o)
{
    ADM v;
    background_adm(p, t, x, y, z, &v);
    int n = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            o[n++] = v.gamma[i][j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            o[n++] = v.K_tensor[i][j];
    o[n++] = v.K;
    o[n++] = v.lapse;
    for (int i = 0; i < 3; ++i)
        o[n++] = v.shift[i];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                o[n++] = v.d1_gamma[i][j][k];
    for (int i = 0; i < 3; ++i)
        o[n++] = v.d1_lapse[i];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            o[n++] = v.d1_shift[i][j];
}

static Prim prim_from6(const double *a)
{
    Prim p;
    p.rho = a[0];
    p.eps = a[1];
    p.p = a[2];
    for (int i = 0; i < 3; ++i)
        p.v[i] = a[3 + i];
    return p;
}

static void g33(const double *a, double g[3][3])
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            g[i][j] = a[3 * i + j];
}

void orc_compute_conserved(const orc_params *p, const double *prim6,
                           const double *gLL9, double *cons5)
{
    double g[3][3];
    g33(gLL9, g);
    const Prim pr = prim_from6(prim6);
    const Cons c = p2c(p->gamma, &pr, g);
    cons5[0] = c.D;
    cons5[1] = c.S[0];
    cons5[2] = c.S[1];
    cons5[3] = c.S[2];
    cons5[4] = c.tau;
}

int orc_recover_primitive(const orc_params *p, const double *cons5,
                          const double *gUU9, double *prim6, int *iterations,
                          double *residual)
{
    double g[3][3];
    g33(gUU9, g);
    Cons c;
    c.D = cons5[0];
    c.S[0] = cons5[1];
    c.S[1] = cons5[2];
    c.S[2] = cons5[3];
    c.tau = cons5[4];
    Prim pr;
    memset(&pr, 0, sizeof(pr));
    const int ok = con2prim(p, &c, g, &pr, iterations, residual);
    prim6[0] = pr.rho;
    prim6[1] = pr.eps;
    prim6[2] = pr.p;
    for (int i = 0; i < 3; ++i)
        prim6[3 + i] = pr.v[i];
    return ok;
}

void orc_muscl_hlle_flux(const orc_params *p, const double *lp6,
                         const double *rp6, const double *ls6,
                         const double *rs6, const double *gLL9,
                         const double *gUU9, double lapse,
                         const double *shift3, int direction, double *flux5)
{
    Geom g;
    memset(&g, 0, sizeof(g));
    g33(gLL9, g.gLL);
    g33(gUU9, g.gUU);
    g.lapse = lapse;
    for (int i = 0; i < 3; ++i)
        g.shift[i] = shift3[i];
    const Prim lp = prim_from6(lp6), rp = prim_from6(rp6),
               ls = prim_from6(ls6), rs = prim_from6(rs6);
    const Flux f = muscl_hlle(p, &lp, &rp, &ls, &rs, &g, direction);
    flux5[0] = f.D;
    flux5[1] = f.S[0];
    flux5[2] = f.S[1];
    flux5[3] = f.S[2];
    flux5[4] = f.tau;
}

/* ------------------------------------------------------------------------ */
/* torus initial data, Source/Matter/GRHD/FixedBGTorus.hpp                   */
/* ------------------------------------------------------------------------ */

void orc_default_torus_config(orc_torus_config *c)
{
    c->total_mass = 1.0;
    c->inner_radius = 0.0;
    c->pressure_max_radius = 0.0;
    c->rho_peak = 1.0;
    c->max_velocity_squared = 1.0 - 1.0e-12;
    c->radial_derivative_fraction = 1.0e-3;
    c->radial_derivative_min_step = 1.0e-4;
    c->angular_momentum_min_factor = 0.25;
    c->angular_momentum_max_factor = 4.0;
    c->angular_momentum_samples = 120;
    c->angular_momentum_bisection_iterations = 80;
    c->angular_momentum_tolerance = 1.0e-13;
}

/* geometry at an arbitrary point (fixed_bg_torus_geometry_at, :144-150) */
static void geometry_at_point(const orc_params *p, double t, double x,
                              double y, double z, Geom *g)
{
    ADM v;
    background_adm(p, t, x, y, z, &v);
    geom_from_adm(&v, g);
}

/* :44-105 */
static double torus_gphiphi(double x, double y, const Geom *g)
{
    const double b[3] = {-y, x, 0.0};
    double s = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            s += g->gLL[i][j] * b[i] * b[j];
    return s;
}

static double torus_gtphi(double x, double y, const Geom *g)
{
    const double b[3] = {-y, x, 0.0};
    double sL[3] = {0, 0, 0};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            sL[i] += g->gLL[i][j] * g->shift[j];
    double bp = 0.0;
    for (int i = 0; i < 3; ++i)
        bp += sL[i] * b[i];
    return bp;
}

static double torus_gtt(const Geom *g)
{
    return -g->lapse * g->lapse + dot_metric(g->shift, g->shift, g->gLL);
}

static double torus_omega(double x, double y, double ell, const Geom *g)
{
    const double gpp = torus_gphiphi(x, y, g);
    const double gtp = torus_gtphi(x, y, g);
    const double gtt = torus_gtt(g);
    const double den = ell * gtp + gpp;
    if (fabs(den) < 1.0e-300)
        return NAN;
    return -(ell * gtt + gtp) / den;
}

static void torus_velocity(double x, double y, double omega, const Geom *g,
                           double v[3])
{
    const double b[3] = {-y, x, 0.0};
    for (int i = 0; i < 3; ++i)
        v[i] = (omega * b[i] + g->shift[i]) / g->lapse;
}

/* fixed_bg_torus_potential_from_geometry, :152-187 */
static double torus_potential_geom(double x, double y, double ell,
                                   const Geom *g, const orc_torus_config *c)
{
    const double om = torus_omega(x, y, ell, g);
    if (!isfinite(om))
        return INFINITY;
    double v[3];
    torus_velocity(x, y, om, g, v);
    const double v2 = velocity_squared(v, g->gLL);
    if (v2 >= c->max_velocity_squared || v2 >= 1.0)
        return INFINITY;
    const double gpp = torus_gphiphi(x, y, g);
    const double gtp = torus_gtphi(x, y, g);
    const double gtt = torus_gtt(g);
    const double norm = -gtt - 2.0 * om * gtp - om * om * gpp;
    if (norm <= 0.0)
        return INFINITY;
    const double mut = -(gtt + om * gtp) / sqrt(norm);
    if (mut <= 0.0)
        return INFINITY;
    return log(mut);
}

static double torus_potential(const orc_params *p, double t, double x,
                              double y, double z, double ell,
                              const orc_torus_config *c)
{
    Geom g;
    geometry_at_point(p, t, x, y, z, &g);
    return torus_potential_geom(x, y, ell, &g, c);
}

/* :200-216 */
static double torus_dWdr(const orc_params *p, double t, double radius,
                         double ell, const orc_torus_config *c)
{
    const double dr = dmax(c->radial_derivative_fraction * radius,
                           c->radial_derivative_min_step);
    const double rm = dmax(radius - dr, 1.0e-6);
    const double wp = torus_potential(p, t, radius + dr, 0.0, 0.0, ell, c);
    const double wm = torus_potential(p, t, rm, 0.0, 0.0, ell, c);
    if (!isfinite(wp) || !isfinite(wm))
        return NAN;
    return (wp - wm) / (radius + dr - rm);
}

/* :218-281 */
static double torus_ell(const orc_params *p, double t,
                        const orc_torus_config *c, int *ok)
{
    *ok = 1;
    if (c->pressure_max_radius <= 3.0 * c->total_mass)
    {
        *ok = 0;
        return NAN;
    }
    const double guess = sqrt(c->total_mass * c->pressure_max_radius) /
                         (1.0 - 2.0 * c->total_mass / c->pressure_max_radius);
    double prev_ell = c->angular_momentum_min_factor * guess;
    double prev_d = torus_dWdr(p, t, c->pressure_max_radius, prev_ell, c);
    for (int s = 1; s <= c->angular_momentum_samples; ++s)
    {
        const double frac = (double)s / c->angular_momentum_samples;
        const double ell =
            guess * (c->angular_momentum_min_factor +
                     frac * (c->angular_momentum_max_factor -
                             c->angular_momentum_min_factor));
        const double d = torus_dWdr(p, t, c->pressure_max_radius, ell, c);
        if (!isfinite(d))
            continue;
        if (isfinite(prev_d) && prev_d * d <= 0.0)
        {
            double lower = prev_ell, upper = ell, f_lower = prev_d;
            for (int it = 0; it < c->angular_momentum_bisection_iterations;
                 ++it)
            {
                const double mid = 0.5 * (lower + upper);
                const double fm =
                    torus_dWdr(p, t, c->pressure_max_radius, mid, c);
                if (!isfinite(fm))
                    break;
                if (fabs(fm) < c->angular_momentum_tolerance)
                    return mid;
                if (f_lower * fm <= 0.0)
                    upper = mid;
                else
                {
                    lower = mid;
                    f_lower = fm;
                }
            }
            return 0.5 * (lower + upper);
        }
        prev_ell = ell;
        prev_d = d;
    }
    return guess;
}

static double torus_enthalpy(double W, const orc_torus_params *t)
{
    if (!isfinite(W))
        return 1.0;
    return exp(t->surface_potential - W);
}

typedef struct
{
    const orc_params *p;
    const orc_torus_config *c;
    const orc_box *b;
    double t;
    const orc_torus_params *tp;
    double hmax[256];
} TorusMaxCtx;

/* the maximum specific enthalpy over cells with R >= inner radius */
static void torus_max_job(void *ctx, int k0, int k1, int slot)
{
    TorusMaxCtx *m = (TorusMaxCtx *)ctx;
    double h = 1.0;
    for (int k = k0; k <= k1; ++k)
        for (int j = m->b->lo[1]; j <= m->b->hi[1]; ++j)
            for (int i = m->b->lo[0]; i <= m->b->hi[0]; ++i)
            {
                double x, y, z;
                cell_position(m->p, i, j, k, &x, &y, &z);
                const double R = sqrt(x * x + y * y);
                if (R < m->c->inner_radius)
                    continue;
                const double W =
                    torus_potential(m->p, m->t, x, y, z, m->tp->ell, m->c);
                h = dmax(h, torus_enthalpy(W, m->tp));
            }
    m->hmax[slot] = h;
}

typedef struct
{
    const orc_params *p;
    const orc_torus_config *c;
    const orc_torus_params *t;
    const orc_box *b;
    double *state;
    double time;
} TorusFillCtx;

static void torus_fill_job(void *ctx, int k0, int k1, int slot);

/* make_fixed_bg_torus_parameters, :291-331 (domain = the box interior) */
int orc_make_torus_parameters(const orc_params *p, const orc_torus_config *c,
                              const orc_box *b, double t,
                              orc_torus_params *out)
{
    int ok;
    out->ell = torus_ell(p, t, c, &ok);
    if (!ok)
        return ORC_ERR_SETUP;
    out->max_enthalpy = 1.0;
    out->polytropic_constant = 0.0;
    out->surface_potential =
        torus_potential(p, t, c->inner_radius, 0.0, 0.0, out->ell, c);
    if (!isfinite(out->surface_potential))
        return ORC_ERR_SETUP;
    TorusMaxCtx *mc = (TorusMaxCtx *)calloc(1, sizeof(TorusMaxCtx));
    mc->p = p;
    mc->c = c;
    mc->b = b;
    mc->t = t;
    mc->tp = out;
    const int n = parallel_z(b->lo[2], b->hi[2], torus_max_job, mc, 256);
    for (int s = 0; s < n; ++s)
        out->max_enthalpy = dmax(out->max_enthalpy, mc->hmax[s]);
    free(mc);
    if (out->max_enthalpy <= 1.0)
        return ORC_ERR_SETUP;
    const double G = p->gamma;
    out->polytropic_constant = (out->max_enthalpy - 1.0) * (G - 1.0) /
                               (G * pow(c->rho_peak, G - 1.0));
    return ORC_OK;
}

/* fixed_bg_torus_primitive, :333-374 */
static Prim torus_prim(const orc_params *p, double x, double y, const Geom *g,
                       const orc_torus_params *t, const orc_torus_config *c)
{
    Prim pr = atmosphere_prim(p);
    const double R = sqrt(x * x + y * y);
    if (R < c->inner_radius)
        return pr;
    const double W = torus_potential_geom(x, y, t->ell, g, c);
    const double h = torus_enthalpy(W, t);
    if (h <= 1.0)
        return pr;
    const double G = p->gamma;
    pr.rho = pow((h - 1.0) * (G - 1.0) / (G * t->polytropic_constant),
                 1.0 / (G - 1.0));
    pr.p = t->polytropic_constant * pow(pr.rho, G);
    pr.eps = pr.p / ((G - 1.0) * pr.rho);
    const double om = torus_omega(x, y, t->ell, g);
    torus_velocity(x, y, om, g, pr.v);
    enforce_floors(p, &pr, g->gLL);
    return pr;
}

/* fill_fixed_bg_torus_level_data, :376-409 (ghosted box) */
int orc_fill_torus(const orc_params *p, const orc_torus_config *c,
                   const orc_torus_params *t, const orc_box *b,
                   double *state, double time)
{
    TorusFillCtx f = {p, c, t, b, state, time};
    parallel_z(b->glo[2], b->ghi[2], torus_fill_job, &f, 256);
    return ORC_OK;
}

static void torus_fill_job(void *ctx, int k0, int k1, int slot)
{
    (void)slot;
    const TorusFillCtx *f = (const TorusFillCtx *)ctx;
    const orc_box *b = f->b;
    for (int k = k0; k <= k1; ++k)
        for (int j = b->glo[1]; j <= b->ghi[1]; ++j)
            for (int i = b->glo[0]; i <= b->ghi[0]; ++i)
            {
                double x, y, z;
                cell_position(f->p, i, j, k, &x, &y, &z);
                Geom g;
                load_geometry(f->p, f->time, i, j, k, &g);
                const Prim pr = torus_prim(f->p, x, y, &g, f->t, f->c);
                const int64_t idx = fab_index(b, i, j, k);
                store_prim(b, f->state, idx, &pr);
                const Cons cc = p2c(f->p->gamma, &pr, g.gLL);
                store_cons(b, f->state, idx, &cc);
            }
}

/* ------------------------------------------------------------------------ */
/* Michel initial data, Tests/GRHDLevelDataMichelAccretion/                  */
/* GRHDLevelDataMichelAccretion.cpp:183-380 (and Tests/GRHDMichelAccretion)  */
/* ------------------------------------------------------------------------ */

static double mi_pressure(const double *k, const orc_michel_config *c,
                          double rho)
{
    return k[0] * pow(rho, c->gamma);
}

static double mi_enthalpy(const double *k, const orc_michel_config *c,
                          double rho)
{
    const double p = mi_pressure(k, c, rho);
    return 1.0 + c->gamma * p / ((c->gamma - 1.0) * rho);
}

void orc_michel_constants(const orc_michel_config *c, double *k)
{
    /* k: polytropic_K, mass_flux, bernoulli, sonic_ur, sonic cs2 */
    k[4] = c->mass / (2.0 * c->sonic_radius - 3.0 * c->mass);
    k[3] = -sqrt(c->mass / (2.0 * c->sonic_radius));
    const double q = k[4] / (c->gamma - k[4] * c->gamma / (c->gamma - 1.0));
    k[0] = q / pow(c->sonic_density, c->gamma - 1.0);
    const double hc = mi_enthalpy(k, c, c->sonic_density);
    const double fc = 1.0 - 2.0 * c->mass / c->sonic_radius;
    k[2] = hc * sqrt(fc + k[3] * k[3]);
    k[1] = c->sonic_radius * c->sonic_radius * c->sonic_density * k[3];
}

static double mi_residual(const double *k, const orc_michel_config *c,
                          double radius, double rho)
{
    const double f = 1.0 - 2.0 * c->mass / radius;
    const double ur = k[1] / (radius * radius * rho);
    const double h = mi_enthalpy(k, c, rho);
    return h * h * (f + ur * ur) - k[2] * k[2];
}

static double mi_bisect(const double *k, const orc_michel_config *c,
                        double radius, double lower, double upper, int *ok)
{
    double fl = mi_residual(k, c, radius, lower);
    const double fu = mi_residual(k, c, radius, upper);
    if (fl == 0.0)
        return lower;
    if (fu == 0.0)
        return upper;
    if (fl * fu > 0.0)
    {
        *ok = 0;
        return NAN;
    }
    for (int it = 0; it < 200; ++it)
    {
        const double mid = 0.5 * (lower + upper);
        const double fm = mi_residual(k, c, radius, mid);
        if (fabs(fm) < c->root_tolerance ||
            fabs(upper - lower) <= c->root_tolerance * dmax(1.0e-300, fabs(mid)))
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

static double mi_density_sweep(const double *k, const orc_michel_config *c,
                               double radius, int *ok)
{
    if (fabs(radius - c->sonic_radius) < 1.0e-12)
        return c->sonic_density;
    const double log_min = log(c->sonic_density * 1.0e-6);
    const double log_max = log(c->sonic_density * 1.0e6);
    const int samples = 6000;
    const int inner = radius < c->sonic_radius;
    double first_lo = NAN, first_hi = NAN, sel_lo = NAN, sel_hi = NAN;
    int have_first = 0, have_sel = 0;
    double last_rho = exp(log_min);
    double last_v = mi_residual(k, c, radius, last_rho);
    for (int i = 1; i <= samples; ++i)
    {
        const double w = (double)i / samples;
        const double rho = exp(log_min + w * (log_max - log_min));
        const double v = mi_residual(k, c, radius, rho);
        if (last_v == 0.0 || v == 0.0 || last_v * v < 0.0)
        {
            const double mid = 0.5 * (last_rho + rho);
            if (!have_first)
            {
                have_first = 1;
                first_lo = last_rho;
                first_hi = rho;
            }
            if (!have_sel && (inner ? mid > c->sonic_density
                                    : mid < c->sonic_density))
            {
                have_sel = 1;
                sel_lo = last_rho;
                sel_hi = rho;
            }
        }
        last_rho = rho;
        last_v = v;
    }
    if (!have_first)
    {
        *ok = 0;
        return NAN;
    }
    if (!have_sel)
    {
        sel_lo = first_lo;
        sel_hi = first_hi;
    }
    return mi_bisect(k, c, radius, sel_lo, sel_hi, ok);
}

/* New (no reference counterpart): within MI_SONIC_BAND (relative) of the
 * sonic radius the two density roots meet closer than one sample of the
 * sweep, which then finds no sign change and the reference fails.  There
 * the density is that of the branch the sweep selects on that side (the
 * root above rho_s inside r_s, below it outside), from the quadratic
 * through the sonic point and that branch's sweep solutions at
 * r_s (1 +- MI_SONIC_BAND) and r_s (1 +- 2 MI_SONIC_BAND). */
#define MI_SONIC_BAND 5.0e-3

static double mi_density(const double *k, const orc_michel_config *c,
                         double radius, int *ok)
{
    const double rho = mi_density_sweep(k, c, radius, ok);
    const double x = radius / c->sonic_radius - 1.0;
    if (*ok || !(fabs(x) < MI_SONIC_BAND))
        return rho;
    const double sg = x < 0.0 ? -1.0 : 1.0;
    int o1 = 1, o2 = 1;
    const double p1 = mi_density_sweep(
        k, c, c->sonic_radius * (1.0 + sg * MI_SONIC_BAND), &o1);
    const double p2 = mi_density_sweep(
        k, c, c->sonic_radius * (1.0 + 2.0 * sg * MI_SONIC_BAND), &o2);
    *ok = o1 && o2;
    const double t = fabs(x) / MI_SONIC_BAND;
    return 0.5 * (t - 1.0) * (t - 2.0) * c->sonic_density -
           t * (t - 2.0) * p1 + 0.5 * t * (t - 1.0) * p2;
}

int orc_michel_point(const orc_params *p, const orc_michel_config *c,
                     double radius, double *out)
{
    double k[5];
    orc_michel_constants(c, k);
    const double f = 1.0 - 2.0 * c->mass / radius;
    if (f <= 0.0)
        return ORC_ERR_SETUP;
    int ok = 1;
    const double rho = mi_density(k, c, radius, &ok);
    if (!ok)
        return ORC_ERR_SETUP;
    const double pressure = mi_pressure(k, c, rho);
    const double eps = pressure / ((c->gamma - 1.0) * rho);
    const double ur = k[1] / (radius * radius * rho);
    /* geometry on the +x axis of a KS black hole of mass c->mass, spin 0 */
    orc_params q = *p;
    q.background = ORC_BG_KERR_SCHILD;
    q.ks_mass = c->mass;
    q.ks_spin = 0.0;
    Geom g;
    geometry_at_point(&q, 0.0, radius, 0.0, 0.0, &g);
    double sL[3] = {0, 0, 0};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            sL[i] += g.gLL[i][j] * g.shift[j];
    const double s2 = dot_metric(g.shift, g.shift, g.gLL);
    const double gtt = -g.lapse * g.lapse + s2;
    const double u_t = -sqrt(f + ur * ur);
    const double ut = (u_t - sL[0] * ur) / gtt;
    const double W = g.lapse * ut;
    if (!(W > 1.0) || !isfinite(W))
        return ORC_ERR_SETUP;
    out[0] = rho;
    out[1] = pressure;
    out[2] = eps;
    out[3] = ur;
    out[4] = ur / W + g.shift[0] / g.lapse;
    return ORC_OK;
}

/* fill_michel_state, GRHDLevelDataMichelAccretion.cpp:331-372 (ghosted) */
typedef struct
{
    const orc_params *p;
    const orc_michel_config *c;
    const orc_box *b;
    double *state;
    int status[256];
} MichelFill;

static void michel_fill_job(void *ctx, int k0, int k1, int slot)
{
    MichelFill *f = (MichelFill *)ctx;
    const orc_params *p = f->p;
    const orc_michel_config *c = f->c;
    const orc_box *b = f->b;
    f->status[slot] = ORC_OK;
    for (int k = k0; k <= k1; ++k)
        for (int j = b->glo[1]; j <= b->ghi[1]; ++j)
            for (int i = b->glo[0]; i <= b->ghi[0]; ++i)
            {
                double x, y, z;
                cell_position(p, i, j, k, &x, &y, &z);
                const double pos[3] = {x, y, z};
                const double radius = sqrt(x * x + y * y + z * z);
                Geom g;
                load_geometry(p, 0.0, i, j, k, &g);
                Prim pr;
                if (radius < c->atmosphere_radius)
                    pr = atmosphere_prim(p);
                else
                {
                    double pt[5];
                    if (orc_michel_point(p, c, radius, pt) != ORC_OK)
                    {
                        f->status[slot] = ORC_ERR_SETUP;
                        return;
                    }
                    pr.rho = pt[0];
                    pr.eps = pt[2];
                    pr.p = pt[1];
                    for (int d = 0; d < 3; ++d)
                        pr.v[d] = pt[4] * pos[d] / radius;
                    enforce_floors(p, &pr, g.gLL);
                }
                const int64_t idx = fab_index(b, i, j, k);
                store_prim(b, f->state, idx, &pr);
                const Cons cc = p2c(p->gamma, &pr, g.gLL);
                store_cons(b, f->state, idx, &cc);
            }
}

/* fill_michel_state (Tests/GRHDLevelDataMichelAccretion/...cpp:312-372)
 * over the ghosted box; cells are independent, so the z planes are split
 * over the setup threads (orc_set_threads). */
int orc_fill_michel(const orc_params *p, const orc_michel_config *c,
                    const orc_box *b, double *state)
{
    MichelFill *f = (MichelFill *)calloc(1, sizeof(MichelFill));
    f->p = p;
    f->c = c;
    f->b = b;
    f->state = state;
    const int n = parallel_z(b->glo[2], b->ghi[2], michel_fill_job, f, 256);
    int status = ORC_OK;
    for (int q = 0; q < n && status == ORC_OK; ++q)
        status = f->status[q];
    free(f);
    return status;
}

/* compute_diagnostics, Examples/GRHDLevelDataKerrSchildDisk/
 * Main_GRHDLevelDataKerrSchildDisk.cpp:223-290 */
void orc_disk_diagnostics(const orc_params *p, const orc_box *b,
                          const int lo[3], const int hi[3],
                          const double *state, double t, double *out)
{
    double mass = 0, disk = 0, tau = 0, mrho = 0, mp = 0, mv = 0, mW = 1.0;
    const double vol = pow(p->dx, 3);
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i)
            {
                const int64_t idx = fab_index(b, i, j, k);
                const Cons c = load_cons(b, state, idx);
                const Prim pr = load_prim(b, state, idx);
                Geom g;
                load_geometry(p, t, i, j, k, &g);
                const double pv = exp(log_sqrt_det(&g)) * vol;
                mass += c.D * pv;
                tau += c.tau * pv;
                if (pr.rho > 10.0 * p->atmo_rho_floor)
                    disk += c.D * pv;
                mrho = dmax(mrho, pr.rho);
                mp = dmax(mp, pr.p);
                const double v2 = velocity_squared(pr.v, g.gLL);
                mv = dmax(mv, sqrt(dmax(0.0, v2)));
                mW = dmax(mW, 1.0 / sqrt(1.0 - v2));
            }
    out[0] = mass;
    out[1] = disk;
    out[2] = tau;
    out[3] = mrho;
    out[4] = mp;
    out[5] = mv;
    out[6] = mW;
}

/* Conserved variables of every cell of the ghosted box from the primitive
 * components already stored there (the fixture fill of
 * Tests/GRHDFixedBGTest/GRHDFixedBGTest.cpp:136-160). */
typedef struct
{
    const orc_params *p;
    const orc_box *b;
    double *state;
    double t;
} ConsFillCtx;

static void cons_fill_job(void *ctx, int k0, int k1, int slot);

void orc_fill_conserved_from_primitives(const orc_params *p, const orc_box *b,
                                        double *state, double t)
{
    ConsFillCtx f = {p, b, state, t};
    parallel_z(b->glo[2], b->ghi[2], cons_fill_job, &f, 256);
}

static void cons_fill_job(void *ctx, int k0, int k1, int slot)
{
    (void)slot;
    const ConsFillCtx *f = (const ConsFillCtx *)ctx;
    const orc_params *p = f->p;
    const orc_box *b = f->b;
    double *state = f->state;
    const double t = f->t;
    for (int k = k0; k <= k1; ++k)
        for (int j = b->glo[1]; j <= b->ghi[1]; ++j)
            for (int i = b->glo[0]; i <= b->ghi[0]; ++i)
            {
                Geom g;
                load_geometry(p, t, i, j, k, &g);
                const int64_t idx = fab_index(b, i, j, k);
                const Prim pr = load_prim(b, state, idx);
                const Cons c = p2c(p->gamma, &pr, g.gLL);
                store_cons(b, state, idx, &c);
            }
}

/* ------------------------------------------------------------------------ */
/* KITP disk driver source terms,                                            */
/* Examples/GRHDLevelDataBinaryPNKITPDisk/Main_GRHDLevelDataBinaryPNKITPDisk.cpp */
/* ------------------------------------------------------------------------ */

/* sink_kernel, :557-565 */
static double kitp_sink_kernel(double r2, double sink_radius,
                               const orc_kitp_config *k)
{
    if (sink_radius <= 0.0 || k->sink_rate == 0.0)
        return 0.0;
    const double size2 = sink_radius * sink_radius;
    return exp(-pow(r2 / size2, 0.5 * k->sink_shape));
}

/* the summed sink rate of both bodies at a cell (:584-597, :633-650) */
static double kitp_sink_rate(const orc_params *p, const orc_kitp_config *k,
                             const double bp[2][3], int i, int j, int l)
{
    double x, y, z;
    cell_position(p, i, j, l, &x, &y, &z);
    const double pos[3] = {x, y, z};
    const double mass[2] = {p->pn_mass_1, p->pn_mass_2};
    double rate = 0.0;
    for (int b = 0; b < 2; ++b)
    {
        double r2 = 0.0;
        for (int d = 0; d < 3; ++d)
        {
            const double dd = pos[d] - bp[b][d];
            r2 += dd * dd;
        }
        rate += k->sink_rate * kitp_sink_kernel(r2, k->sink_size * mass[b], k);
    }
    return rate;
}

static void kitp_bodies(const orc_params *p, double t, double bp[2][3])
{
    double v1[3], v2[3];
    pn_state(p, t, bp[0], bp[1], v1, v2);
}

/* add_kitp_sink_rhs, :567-610 */
void orc_kitp_sink_rhs(const orc_params *p, const orc_kitp_config *k,
                       const orc_box *b, const double *state, double *rhs,
                       int64_t rcs, double t)
{
    if (k->sink_rate == 0.0 || k->sink_size <= 0.0)
        return;
    double bp[2][3];
    kitp_bodies(p, t, bp);
    const int nx = b->hi[0] - b->lo[0] + 1, ny = b->hi[1] - b->lo[1] + 1;
    for (int l = b->lo[2]; l <= b->hi[2]; ++l)
        for (int j = b->lo[1]; j <= b->hi[1]; ++j)
            for (int i = b->lo[0]; i <= b->hi[0]; ++i)
            {
                const int64_t g = fab_index(b, i, j, l);
                const Prim pr = load_prim(b, state, g);
                if (pr.rho <= 10.0 * p->atmo_rho_floor)
                    continue;
                const double rate = kitp_sink_rate(p, k, bp, i, j, l);
                if (rate == 0.0)
                    continue;
                const Cons c = load_cons(b, state, g);
                const int64_t r = (i - b->lo[0]) +
                                  (int64_t)nx * ((j - b->lo[1]) +
                                                 (int64_t)ny * (l - b->lo[2]));
                rhs[0 * rcs + r] -= rate * c.D;
                rhs[4 * rcs + r] -= rate * c.tau;
                for (int d = 0; d < 3; ++d)
                    rhs[(1 + d) * rcs + r] -= rate * c.S[d];
            }
}

/* apply_kitp_sink_decay, :612-662 (one box) */
void orc_kitp_sink_decay(const orc_params *p, const orc_kitp_config *k,
                         const orc_box *b, double *state, double t, double dt)
{
    if (k->sink_rate == 0.0 || k->sink_size <= 0.0)
        return;
    double bp[2][3];
    kitp_bodies(p, t, bp);
    const int64_t cs = b->comp_stride;
    for (int l = b->lo[2]; l <= b->hi[2]; ++l)
        for (int j = b->lo[1]; j <= b->hi[1]; ++j)
            for (int i = b->lo[0]; i <= b->hi[0]; ++i)
            {
                const int64_t g = fab_index(b, i, j, l);
                if (state[ORC_D * cs + g] <= 0.0)
                    continue;
                const double rate = kitp_sink_rate(p, k, bp, i, j, l);
                if (rate == 0.0)
                    continue;
                const double decay = exp(-rate * dt);
                state[ORC_D * cs + g] *= decay;
                state[ORC_TAU * cs + g] *= decay;
                state[ORC_S1 * cs + g] *= decay;
                state[ORC_S2 * cs + g] *= decay;
                state[ORC_S3 * cs + g] *= decay;
            }
}

/* clamped_neighbor, :664-674 (clamped to the problem domain) */
static int kitp_clamp(int v, int lo, int hi)
{
    return v < lo ? lo : (v > hi ? hi : v);
}

/* alpha_dynamic_viscosity, :676-698 */
static double kitp_mu(const orc_params *p, const orc_kitp_config *k,
                      const Prim *pr, const double pos[3],
                      const double bp[2][3])
{
    if (k->alpha_viscosity == 0.0)
        return 0.0;
    const double mass[2] = {p->pn_mass_1, p->pn_mass_2};
    double omega2 = 0.0;
    for (int b = 0; b < 2; ++b)
    {
        double r2 = 1.0e-10;
        for (int d = 0; d < 3; ++d)
        {
            const double dd = pos[d] - bp[b][d];
            r2 += dd * dd;
        }
        omega2 += mass[b] * pow(r2, -1.5);
    }
    const double cs2 = p->gamma * pr->p / dmax(pr->rho, k->rho_floor);
    return pr->rho * k->alpha_viscosity * cs2 / sqrt(dmax(omega2, 1.0e-300));
}

/* viscous_flux_for_cell, :700-770; flux[0..2] = S_x, S_y, tau */
static void kitp_viscous_flux(const orc_params *p, const orc_kitp_config *k,
                              const orc_box *b, const double *state, int i,
                              int j, int l, int dir, const double bp[2][3],
                              double flux[3])
{
    flux[0] = flux[1] = flux[2] = 0.0;
    const Prim pr = load_prim(b, state, fab_index(b, i, j, l));
    if (pr.rho <= 10.0 * p->atmo_rho_floor)
        return;
    double x, y, z;
    cell_position(p, i, j, l, &x, &y, &z);
    const double pos[3] = {x, y, z};
    const double mu = kitp_mu(p, k, &pr, pos, bp);
    if (mu == 0.0)
        return;
    double gradv[2][2];
    const int iv[3] = {i, j, l};
    for (int c = 0; c < 2; ++c)
    {
        int m[3] = {i, j, l}, q[3] = {i, j, l};
        m[c] = kitp_clamp(iv[c] - 1, b->dlo[c], b->dhi[c]);
        q[c] = kitp_clamp(iv[c] + 1, b->dlo[c], b->dhi[c]);
        const int span = q[c] - m[c];
        const double den = (span > 1 ? span : 1) * p->dx;
        const Prim pm = load_prim(b, state, fab_index(b, m[0], m[1], m[2]));
        const Prim pq = load_prim(b, state, fab_index(b, q[0], q[1], q[2]));
        for (int v = 0; v < 2; ++v)
            gradv[v][c] = (pq.v[v] - pm.v[v]) / den;
    }
    const double divergence = gradv[0][0] + gradv[1][1];
    double tau[2][2];
    for (int a = 0; a < 2; ++a)
        for (int c = 0; c < 2; ++c)
            tau[a][c] = mu * (gradv[a][c] + gradv[c][a] +
                              (k->viscosity_beta - 2.0 / 3.0) *
                                  (double)(a == c) * divergence);
    flux[0] = -tau[dir][0];
    flux[1] = -tau[dir][1];
    flux[2] = -tau[dir][0] * pr.v[0] - tau[dir][1] * pr.v[1];
}

/* add_kitp_viscous_rhs, :772-806 */
void orc_kitp_viscous_rhs(const orc_params *p, const orc_kitp_config *k,
                          const orc_box *b, const double *state, double *rhs,
                          int64_t rcs, double t)
{
    if (k->alpha_viscosity == 0.0)
        return;
    double bp[2][3];
    kitp_bodies(p, t, bp);
    const int nx = b->hi[0] - b->lo[0] + 1, ny = b->hi[1] - b->lo[1] + 1;
    for (int l = b->lo[2]; l <= b->hi[2]; ++l)
        for (int j = b->lo[1]; j <= b->hi[1]; ++j)
            for (int i = b->lo[0]; i <= b->hi[0]; ++i)
            {
                const int64_t r = (i - b->lo[0]) +
                                  (int64_t)nx * ((j - b->lo[1]) +
                                                 (int64_t)ny * (l - b->lo[2]));
                const int iv[3] = {i, j, l};
                for (int d = 0; d < 2; ++d)
                {
                    int lo[3] = {i, j, l}, hi[3] = {i, j, l};
                    lo[d] = kitp_clamp(iv[d] - 1, b->dlo[d], b->dhi[d]);
                    hi[d] = kitp_clamp(iv[d] + 1, b->dlo[d], b->dhi[d]);
                    double fl[3], fh[3];
                    kitp_viscous_flux(p, k, b, state, lo[0], lo[1], lo[2], d,
                                      bp, fl);
                    kitp_viscous_flux(p, k, b, state, hi[0], hi[1], hi[2], d,
                                      bp, fh);
                    rhs[4 * rcs + r] -= (fh[2] - fl[2]) / (2.0 * p->dx);
                    rhs[1 * rcs + r] -= (fh[0] - fl[0]) / (2.0 * p->dx);
                    rhs[2 * rcs + r] -= (fh[1] - fl[1]) / (2.0 * p->dx);
                }
            }
}


/* ------------------------------------------------------------------------ */
/* The operator on CCZ4-stored geometry (LevelDataFiniteVolumeOperator,      */
/* Source/Matter/GRHD/FArrayBoxFiniteVolume.hpp:136-192, 219-542, 681-1364). */
/* The state holds GRChombo's 25 CCZ4 variables, then the 11 GRHD ones       */
/* (Tests/GRHDFixedBGTest/UserVariables.hpp:24-40); the geometry is read      */
/* from chi, h_ij, A_ij, K, lapse and shift, and the metric derivatives of    */
/* the sources are finite differences of it.                                 */
/* ------------------------------------------------------------------------ */

enum
{
    CZ_CHI = 0,
    CZ_H = 1,      /* h11 h12 h13 h22 h23 h33 */
    CZ_K = 7,
    CZ_A = 8,      /* A11 A12 A13 A22 A23 A33 */
    CZ_LAPSE = 18,
    CZ_SHIFT = 19, /* shift1..3 */
    CZ_GRHD = 25
};

static const int CZ_SYM[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};

/* load_ccz4_geometry, :168-192 */
static void ccz4_geometry(const orc_box *b, const double *s, int64_t idx,
                          Geom *g)
{
    const int64_t cs = b->comp_stride;
    const double chi = s[CZ_CHI * cs + idx];
    double h[3][3], A[3][3], hUU[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
        {
            h[i][j] = s[(CZ_H + CZ_SYM[i][j]) * cs + idx];
            A[i][j] = s[(CZ_A + CZ_SYM[i][j]) * cs + idx];
        }
    inverse_sym(h, hUU);
    const double trK = s[CZ_K * cs + idx];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
        {
            g->gLL[i][j] = h[i][j] / chi;
            g->gUU[i][j] = chi * hUU[i][j];
            g->K[i][j] = A[i][j] / chi + g->gLL[i][j] * trK / 3.0;
        }
    g->lapse = s[CZ_LAPSE * cs + idx];
    for (int i = 0; i < 3; ++i)
        g->shift[i] = s[(CZ_SHIFT + i) * cs + idx];
}

/* Outflow source of a physical ghost (interior_box ends), or -1. */
static int64_t ccz4_outflow_source(const orc_box *b, int i, int j, int k)
{
    const int iv[3] = {i, j, k};
    int src[3] = {i, j, k};
    int ghost = 0;
    for (int d = 0; d < 3; ++d)
    {
        if (iv[d] < b->dlo[d])
        {
            ghost = 1;
            src[d] = b->lo[d];
        }
        else if (iv[d] > b->dhi[d])
        {
            ghost = 1;
            src[d] = b->hi[d];
        }
    }
    return ghost ? fab_index(b, src[0], src[1], src[2]) : -1;
}

/* fill_conserved_outflow_boundaries (:484-519) and
 * fill_ccz4_geometry_outflow_boundaries (:430-473): the physical ghosts
 * copy the five conserved variables and chi, h_ij, lapse, shift of their
 * source cell (the other CCZ4 variables and the primitives stay). */
static void ccz4_fill_outflow(const orc_box *b, double *s, int conserved)
{
    const int64_t cs = b->comp_stride;
    static const int geo[11] = {CZ_CHI, 1, 2, 3, 4, 5, 6, CZ_LAPSE,
                                CZ_SHIFT, CZ_SHIFT + 1, CZ_SHIFT + 2};
    for (int k = b->glo[2]; k <= b->ghi[2]; ++k)
        for (int j = b->glo[1]; j <= b->ghi[1]; ++j)
            for (int i = b->glo[0]; i <= b->ghi[0]; ++i)
            {
                const int64_t src = ccz4_outflow_source(b, i, j, k);
                if (src < 0)
                    continue;
                const int64_t dst = fab_index(b, i, j, k);
                if (conserved)
                    for (int c = 0; c < 5; ++c)
                        s[(CZ_GRHD + c) * cs + dst] =
                            s[(CZ_GRHD + c) * cs + src];
                for (int q = 0; q < 11; ++q)
                    s[geo[q] * cs + dst] = s[geo[q] * cs + src];
            }
}

static Cons ccz4_cons(const orc_box *b, const double *s, int64_t idx)
{
    return load_cons(b, s + CZ_GRHD * b->comp_stride, idx);
}

static Prim ccz4_prim(const orc_box *b, const double *s, int64_t idx)
{
    return load_prim(b, s + CZ_GRHD * b->comp_stride, idx);
}

/* compute_leveldata_flux_rhs_from_ccz4_geometry (:1047-1090) on one box:
 * per direction the outflow fills, the ghosted-box recovery
 * (recover_primitives_from_ccz4_geometry, :681-702), the MC slopes and the
 * interior face pairs (:784-833, every face twice), summed into rhs; then
 * the geometry fill and add_static_metric_sources_to_conserved_rhs
 * (:367-427) with the one-sided stencils of
 * make_metric_source_derivative_stencil (:283-322). */
int orc_ccz4_compute_rhs(const orc_params *p, const orc_box *b, double *s,
                         double *rhs, int64_t rcs, const double inv_dx[3],
                         orc_error *err)
{
    if (err)
        memset(err, 0, sizeof(*err));
    if (!check_box(b))
        return ORC_ERR_INVALID_ARG;
    const int gnx = b->ghi[0] - b->glo[0] + 1, gny = b->ghi[1] - b->glo[1] + 1,
              gnz = b->ghi[2] - b->glo[2] + 1;
    const int64_t gvol = (int64_t)gnx * gny * gnz;
    const int nx = b->hi[0] - b->lo[0] + 1, ny = b->hi[1] - b->lo[1] + 1;
#define CZ_RIDX(i, j, k)                                                      \
    ((int64_t)((i)-b->lo[0]) +                                                \
     (int64_t)nx * ((int64_t)((j)-b->lo[1]) + (int64_t)ny * ((k)-b->lo[2])))
    for (int k = b->lo[2]; k <= b->hi[2]; ++k)
        for (int j = b->lo[1]; j <= b->hi[1]; ++j)
            for (int i = b->lo[0]; i <= b->hi[0]; ++i)
                for (int c = 0; c < 5; ++c)
                    rhs[c * rcs + CZ_RIDX(i, j, k)] = 0.0;
    Prim *prims = (Prim *)calloc(gvol, sizeof(Prim));
    Geom *geo = (Geom *)calloc(gvol, sizeof(Geom));
    int status = ORC_OK;
    /* the fills and the recovery give the same values in every direction */
    ccz4_fill_outflow(b, s, 1);
    for (int k = b->glo[2]; k <= b->ghi[2] && status == ORC_OK; ++k)
        for (int j = b->glo[1]; j <= b->ghi[1] && status == ORC_OK; ++j)
            for (int i = b->glo[0]; i <= b->ghi[0]; ++i)
            {
                const int64_t idx = fab_index(b, i, j, k);
                ccz4_geometry(b, s, idx, &geo[idx]);
                const Cons c = ccz4_cons(b, s, idx);
                int it;
                double res;
                if (!con2prim(p, &c, geo[idx].gUU, &prims[idx], &it, &res))
                {
                    set_error(err, ORC_ERR_RECOVERY,
                              ORC_WHERE_GHOSTED_RECOVERY, i, j, k, res);
                    status = ORC_ERR_RECOVERY;
                    break;
                }
            }
    for (int dir = 0; dir < 3 && status == ORC_OK; ++dir)
    {
        const int off[3] = {dir == 0, dir == 1, dir == 2};
        const int64_t so = fab_index(b, b->lo[0] + off[0], b->lo[1] + off[1],
                                     b->lo[2] + off[2]) -
                           fab_index(b, b->lo[0], b->lo[1], b->lo[2]);
        for (int k = b->lo[2]; k <= b->hi[2]; ++k)
            for (int j = b->lo[1]; j <= b->hi[1]; ++j)
                for (int i = b->lo[0]; i <= b->hi[0]; ++i)
                {
                    const int64_t c0 = fab_index(b, i, j, k);
                    Flux f[2];
                    for (int side = 0; side < 2; ++side)
                    {
                        /* face between L = c0 - so + side*so and L + so */
                        const int64_t L = c0 - so + side * so, R = L + so;
                        const Prim sl = prim_slope(&prims[L - so], &prims[L],
                                                   &prims[R], p->limiter_theta);
                        const Prim sr = prim_slope(&prims[L], &prims[R],
                                                   &prims[R + so],
                                                   p->limiter_theta);
                        Geom g;
                        average_geometry(&geo[L], &geo[R], &g);
                        f[side] = muscl_hlle(p, &prims[L], &prims[R], &sl,
                                             &sr, &g, dir);
                    }
                    const int64_t r = CZ_RIDX(i, j, k);
                    const double idx_ = inv_dx[dir];
                    rhs[0 * rcs + r] += -idx_ * (f[1].D - f[0].D);
                    rhs[4 * rcs + r] += -idx_ * (f[1].tau - f[0].tau);
                    for (int m = 0; m < 3; ++m)
                        rhs[(1 + m) * rcs + r] += -idx_ * (f[1].S[m] - f[0].S[m]);
                }
    }
    if (status == ORC_OK && p->use_static_metric_sources)
    {
        ccz4_fill_outflow(b, s, 0);
        for (int k = b->lo[2]; k <= b->hi[2] && status == ORC_OK; ++k)
            for (int j = b->lo[1]; j <= b->hi[1] && status == ORC_OK; ++j)
                for (int i = b->lo[0]; i <= b->hi[0]; ++i)
                {
                    const int64_t idx = fab_index(b, i, j, k);
                    Geom g;
                    ccz4_geometry(b, s, idx, &g);
                    const Cons c = ccz4_cons(b, s, idx);
                    Prim pr;
                    int it;
                    double res;
                    if (!con2prim(p, &c, g.gUU, &pr, &it, &res))
                    {
                        set_error(err, ORC_ERR_RECOVERY,
                                  ORC_WHERE_METRIC_SOURCES, i, j, k, res);
                        status = ORC_ERR_RECOVERY;
                        break;
                    }
                    enforce_floors(p, &pr, g.gLL);
                    if (is_atmosphere(p, &pr,
                                      p->atmo_metric_source_atmosphere_factor))
                        continue;
                    Derivs dv;
                    memset(&dv, 0, sizeof(dv));
                    for (int dir = 0; dir < 3; ++dir)
                    {
                        const int off[3] = {dir == 0, dir == 1, dir == 2};
                        const int64_t lo_i = fab_index(b, i - off[0], j - off[1],
                                                       k - off[2]);
                        const int64_t hi_i = fab_index(b, i + off[0], j + off[1],
                                                       k + off[2]);
                        const Prim pl = ccz4_prim(b, s, lo_i);
                        const Prim pu = ccz4_prim(b, s, hi_i);
                        const double f = p->atmo_metric_source_atmosphere_factor;
                        const int la = !is_atmosphere(p, &pl, f);
                        const int ua = !is_atmosphere(p, &pu, f);
                        int64_t lo_c, up_c;
                        double coef;
                        if (la && ua)
                        {
                            lo_c = lo_i;
                            up_c = hi_i;
                            coef = 0.5 * inv_dx[dir];
                        }
                        else if (ua)
                        {
                            lo_c = idx;
                            up_c = hi_i;
                            coef = inv_dx[dir];
                        }
                        else if (la)
                        {
                            lo_c = lo_i;
                            up_c = idx;
                            coef = inv_dx[dir];
                        }
                        else
                            continue;
                        Geom gu, gl;
                        ccz4_geometry(b, s, up_c, &gu);
                        ccz4_geometry(b, s, lo_c, &gl);
                        const int64_t cs = b->comp_stride;
                        dv.dlapse[dir] = coef * (s[CZ_LAPSE * cs + up_c] -
                                                 s[CZ_LAPSE * cs + lo_c]);
                        dv.dlnsqrtg[dir] =
                            coef * (log_sqrt_det(&gu) - log_sqrt_det(&gl));
                        for (int a = 0; a < 3; ++a)
                            for (int bb = 0; bb < 3; ++bb)
                                dv.dgamma[dir][a][bb] =
                                    coef * (gu.gLL[a][bb] - gl.gLL[a][bb]);
                        for (int sd = 0; sd < 3; ++sd)
                            dv.dshift[sd][dir] =
                                coef * (s[(CZ_SHIFT + sd) * cs + up_c] -
                                        s[(CZ_SHIFT + sd) * cs + lo_c]);
                    }
                    const Cons src = static_sources(p->gamma, &pr, &c, &g, &dv);
                    const int64_t r = CZ_RIDX(i, j, k);
                    rhs[0 * rcs + r] += src.D;
                    rhs[4 * rcs + r] += src.tau;
                    for (int m = 0; m < 3; ++m)
                        rhs[(1 + m) * rcs + r] += src.S[m];
                }
    }
#undef CZ_RIDX
    free(prims);
    free(geo);
    return status;
}

/* recover_primitives_and_apply_atmosphere_from_ccz4_geometry (:713-761)
 * over the interior. */
void orc_ccz4_recover_primitives(const orc_params *p, const orc_box *b,
                                 double *s, orc_diag *diag)
{
    memset(diag, 0, sizeof(*diag));
    double *q = s + CZ_GRHD * b->comp_stride;
    for (int k = b->lo[2]; k <= b->hi[2]; ++k)
        for (int j = b->lo[1]; j <= b->hi[1]; ++j)
            for (int i = b->lo[0]; i <= b->hi[0]; ++i)
            {
                ++diag->num_cells;
                const int64_t idx = fab_index(b, i, j, k);
                Geom g;
                ccz4_geometry(b, s, idx, &g);
                const Cons c = load_cons(b, q, idx);
                Prim pr;
                int it;
                double res;
                int reset = !con2prim(p, &c, g.gUU, &pr, &it, &res);
                if (!reset)
                {
                    Prim fl = pr;
                    enforce_floors(p, &fl, g.gLL);
                    reset = prim_differs(&pr, &fl);
                    if (reset)
                        ++diag->num_floored_primitives;
                    pr = fl;
                }
                else
                {
                    ++diag->num_failed_recoveries;
                    pr = atmosphere_prim(p);
                }
                store_prim(b, q, idx, &pr);
                if (reset)
                {
                    ++diag->num_conserved_resets;
                    const Cons nc = p2c(p->gamma, &pr, g.gLL);
                    store_cons(b, q, idx, &nc);
                }
            }
}

/* compute_max_inverse_dt_from_ccz4_geometry (:1139-1183). */
int orc_ccz4_compute_max_inverse_dt(const orc_params *p, const orc_box *b,
                                    const double *s, const double inv_dx[3],
                                    double *out, orc_error *err)
{
    if (err)
        memset(err, 0, sizeof(*err));
    double m = 0.0;
    for (int k = b->lo[2]; k <= b->hi[2]; ++k)
        for (int j = b->lo[1]; j <= b->hi[1]; ++j)
            for (int i = b->lo[0]; i <= b->hi[0]; ++i)
            {
                const int64_t idx = fab_index(b, i, j, k);
                Geom g;
                ccz4_geometry(b, s, idx, &g);
                const Cons c = ccz4_cons(b, s, idx);
                Prim pr;
                int it;
                double res;
                if (!con2prim(p, &c, g.gUU, &pr, &it, &res))
                {
                    set_error(err, ORC_ERR_RECOVERY, ORC_WHERE_CFL, i, j, k,
                              res);
                    return ORC_ERR_RECOVERY;
                }
                enforce_floors(p, &pr, g.gLL);
                if (is_atmosphere(p, &pr, 1.0 + 1.0e-12))
                    continue;
                double cell = 0.0;
                for (int d = 0; d < 3; ++d)
                {
                    double lo, hi;
                    char_speeds(p->gamma, &pr, g.gLL, g.gUU, d, g.lapse,
                                g.shift, &lo, &hi);
                    cell += dmax(fabs(lo), fabs(hi)) * inv_dx[d];
                }
                m = dmax(m, cell);
            }
    *out = m;
    return ORC_OK;
}

/* The CCZ4 variables of a fixed background (the reference's fixed-BG vs
 * CCZ4-geometry test fills them from the analytic metric,
 * store_ccz4_background_vars, Tests/GRHDFixedBGTest/GRHDFixedBGTest.cpp:
 * 97-134): chi = det(gamma)^(-1/3), h = gamma chi, A = K_ij chi - K h / 3,
 * trace K, lapse, shift, over the
 * ghosted box; the GRHD components are left as they are. */
void orc_ccz4_fill_from_background(const orc_params *p, const orc_box *b,
                                   double *s, double t)
{
    const int64_t cs = b->comp_stride;
    for (int k = b->glo[2]; k <= b->ghi[2]; ++k)
        for (int j = b->glo[1]; j <= b->ghi[1]; ++j)
            for (int i = b->glo[0]; i <= b->ghi[0]; ++i)
            {
                const int64_t idx = fab_index(b, i, j, k);
                double x, y, z;
                cell_position(p, i, j, k, &x, &y, &z);
                ADM v;
                background_adm(p, t, x, y, z, &v);
                const double chi = pow(det_sym(v.gamma), -1.0 / 3.0);
                for (int q = 0; q < CZ_GRHD; ++q)
                    s[q * cs + idx] = 0.0;
                s[CZ_CHI * cs + idx] = chi;
                for (int a = 0; a < 3; ++a)
                    for (int c = a; c < 3; ++c)
                    {
                        const double h = v.gamma[a][c] * chi;
                        s[(CZ_H + CZ_SYM[a][c]) * cs + idx] = h;
                        s[(CZ_A + CZ_SYM[a][c]) * cs + idx] =
                            v.K_tensor[a][c] * chi - v.K * h / 3.0;
                    }
                s[CZ_K * cs + idx] = v.K;
                s[CZ_LAPSE * cs + idx] = v.lapse;
                for (int a = 0; a < 3; ++a)
                    s[(CZ_SHIFT + a) * cs + idx] = v.shift[a];
            }
}

/* ------------------------------------------------------------------------ */
/* The binary disk drivers' Keplerian disk (kitp_primitive and               */
/* fill_kitp_level_data, Examples/GRHDLevelDataBinaryPNKITPDisk/             */
/* Main_GRHDLevelDataBinaryPNKITPDisk.cpp:398-555), on the operator's binary */
/* (masses, separation, phase, time, softening of orc_params) and its        */
/* atmosphere floors, plus the azimuthal density modes m = 1..4 of the       */
/* benchmark's binary-disk configuration (new).                              */
/* ------------------------------------------------------------------------ */

/* stable_logistic_cutoff, :398-406 */
static double kitp_cutoff(double radius, double outer_radius)
{
    const double arg = -2.0 * (radius - outer_radius);
    if (arg > 700.0)
        return 1.0;
    if (arg < -700.0)
        return 0.0;
    return 1.0 - 1.0 / (1.0 + exp(arg));
}

static double kitp_omega_bin(const orc_params *p)
{
    const double total = p->pn_mass_1 + p->pn_mass_2;
    return p->pn_angular_velocity != 0.0
               ? p->pn_angular_velocity
               : sqrt(total / (p->pn_separation * p->pn_separation *
                               p->pn_separation));
}

/* kitp_primitive, :465-520, with the modes applied to the density profile
 * (1 + sum_m A_m cos(m phi + phase_m)) before the floor. */
static Prim kitp_disk_prim(const orc_params *p, const orc_kitp_disk *k,
                           const double pos[3], const double body[2][3],
                           const Geom *g)
{
    Prim pr = atmosphere_prim(p);
    const double radius = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
    if (radius <= 1.0e-12)
        return pr;
    const double phi = atan2(pos[1], pos[0]);
    const double h = dmax(k->aspect_ratio * radius, 1.0e-12);
    const double vprof = exp(-0.5 * (pos[2] / h) * (pos[2] / h));
    const double zero_sigma = p->atmo_rho_floor / k->rho_peak;
    /* kitp_sigma_midplane, :408-418 */
    const double safe_r = dmax(radius, 1.0e-12);
    const double cavity = k->cavity_radius_factor * p->pn_separation;
    const double cprof =
        (1.0 - k->cavity_delta) * exp(-pow(cavity / safe_r, 12.0)) +
        k->cavity_delta;
    double sigma = cprof * kitp_cutoff(radius, k->outer_cutoff_radius);
    double modes = 1.0;
    for (int m = 0; m < 4; ++m)
        modes += k->mode_amplitude[m] * cos((m + 1) * phi + k->mode_phase[m]);
    sigma *= modes;
    const double dscale = sigma * vprof + zero_sigma;
    pr.rho = dmax(p->atmo_rho_floor, k->rho_peak * dscale);
    /* binary_point_mass_potential, :444-463 */
    const double masses[2] = {p->pn_mass_1, p->pn_mass_2};
    double pot = 0.0;
    for (int b = 0; b < 2; ++b)
    {
        double r2 = p->pn_softening_radius * p->pn_softening_radius;
        for (int d = 0; d < 3; ++d)
        {
            const double dd = pos[d] - body[b][d];
            r2 += dd * dd;
        }
        pot -= masses[b] / sqrt(r2);
    }
    const double cs2 = dmax(p->atmo_pressure_floor / pr.rho,
                            -pot / (k->mach * k->mach));
    pr.p = dmax(p->atmo_pressure_floor, pr.rho * cs2 / p->gamma);
    pr.eps = pr.p / ((p->gamma - 1.0) * pr.rho);
    /* kitp_radial_velocity, :420-427; kitp_phi_velocity, :429-442 */
    const double wb = kitp_omega_bin(p);
    const double sep = p->pn_separation;
    const double v0 = 1.0e-4 * wb * sep;
    const double vr = v0 * sin(phi) * (radius / sep) *
                      exp(-pow(radius / (3.5 * sep), 6.0));
    const double total = p->pn_mass_1 + p->pn_mass_2;
    const double wg = sqrt(total / (safe_r * safe_r * safe_r) *
                           dmax(0.0, 1.0 - 1.0 / (k->mach * k->mach)));
    double vphi = 0.0;
    if (wg > 0.0)
        vphi = pow(pow(wb, -4.0) + pow(wg, -4.0), -0.25) * safe_r;
    const double cv[3] = {vr * cos(phi) - vphi * sin(phi),
                          vr * sin(phi) + vphi * cos(phi), 0.0};
    for (int d = 0; d < 3; ++d)
        pr.v[d] = (cv[d] + g->shift[d]) / g->lapse;
    enforce_floors(p, &pr, g->gLL);
    return pr;
}

void orc_fill_kitp_disk(const orc_params *p, const orc_kitp_disk *k,
                        const orc_box *b, double *state, double t)
{
    double body[2][3], v1[3], v2[3];
    pn_state(p, t, body[0], body[1], v1, v2);
    for (int kk = b->glo[2]; kk <= b->ghi[2]; ++kk)
        for (int j = b->glo[1]; j <= b->ghi[1]; ++j)
            for (int i = b->glo[0]; i <= b->ghi[0]; ++i)
            {
                double pos[3];
                cell_position(p, i, j, kk, &pos[0], &pos[1], &pos[2]);
                Geom g;
                load_geometry(p, t, i, j, kk, &g);
                const Prim pr = kitp_disk_prim(p, k, pos, body, &g);
                const int64_t idx = fab_index(b, i, j, kk);
                store_prim(b, state, idx, &pr);
                const Cons c = p2c(p->gamma, &pr, g.gLL);
                store_cons(b, state, idx, &c);
            }
}
