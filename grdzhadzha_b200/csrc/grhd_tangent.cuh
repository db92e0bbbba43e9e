// grhd_tangent.cuh -- forward-mode (tangent-linear) versions of the FP64
// pointwise physics, the counterpart of the reverse-mode functions of
// grhd_adjoint.cuh, and the work items of the tangent-linear sweep.  No
// counterpart in the reference.
//
// A value and its directional derivative travel together as a Dual.  Every
// branch is taken exactly as the matching *_rev function takes it (same
// tests on the same double values, same tie rules), and every MUSCL
// limiter branch comes from the bits the forward sweep recorded, so that
// the tangent-linear map and the adjoint are transposes of one linear map
// and <lambda, J v> = <J^T lambda, v> holds to rounding.
#pragma once

#include "grhd_adjoint.cuh"
#include "grhd_adjoint_items.cuh"

namespace grhd {
namespace adj {

GRHD_HD inline Dual dual_sqrt_nz(Dual a)
{
    // sqrt with a zero derivative where the value is zero (char_speeds_rev
    // passes no adjoint through sqrt(max(0, rad)) when rad <= 0)
    const double s = sqrt(a.v);
    return Dual(s, s > 0.0 ? a.d / (2.0 * s) : 0.0);
}

GRHD_HD inline Cons values_of(const ConsT<Dual> &a)
{
    Cons c;
    c.D = a.D.v;
    c.tau = a.tau.v;
    for (int i = 0; i < 3; ++i)
        c.S[i] = a.S[i].v;
    return c;
}

// Metric tangents along a direction whose spin component is da: the
// dual-number spin derivative scaled by da.
GRHD_HD inline void scale_tangent(GeoT<Dual> &g, double da)
{
    for (int q = 0; q < 6; ++q)
    {
        g.gLL[q].d *= da;
        g.gUU[q].d *= da;
    }
    g.lapse.d *= da;
    for (int i = 0; i < 3; ++i)
        g.shift[i].d *= da;
}

GRHD_HD inline void scale_tangent(GeoFullT<Dual> &f, double da)
{
    scale_tangent(f.g, da);
    for (int q = 0; q < 6; ++q)
        f.K[q].d *= da;
    for (int d = 0; d < 3; ++d)
    {
        f.dlapse[d].d *= da;
        f.dlnsqrtg[d].d *= da;
        for (int q = 0; q < 6; ++q)
            f.dgamma[d][q].d *= da;
        for (int q = 0; q < 3; ++q)
            f.dshift[d][q].d *= da;
    }
}

// recover_primitive (Valencia.hpp:116-228) at its converged pressure p, in
// tangent form (con2prim_rev transposed): dp = -(f_D dD + f_tau dtau +
// f_S2 dS2) / f_p by the implicit function theorem, zero for a pressure
// pinned at the recovery floor; the primitives are the closed forms of
// (D, S, tau, gamma^ij, p).
GRHD_HD inline PrimT<Dual> con2prim_tan(const Options &o, const ConsT<Dual> &c,
                                        const Dual gUU[6], double p)
{
    Dual S2 = Dual(0.0);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            S2 += gUU[sym(i, j)] * c.S[i] * c.S[j];
    const double gm1 = o.G - 1.0;
    double dp = 0.0;
    if (p > o.rec_pfloor)
    {
        const double e = c.tau.v + c.D.v + p;
        const double v2 = S2.v / (e * e);
        const double W = 1.0 / sqrt(1.0 - v2);
        const double Gfac = o.G / gm1;
        const double fW = c.D.v + 2.0 * Gfac * p * W;
        const double dWdv2 = 0.5 * W * W * W;
        const double dv2de = -2.0 * v2 / e;
        const double f_p = Gfac * W * W + fW * dWdv2 * dv2de - 1.0;
        const double f_D = W + fW * dWdv2 * dv2de - 1.0;
        const double f_tau = fW * dWdv2 * dv2de - 1.0;
        const double f_S2 = fW * dWdv2 / (e * e);
        dp = -(f_D * c.D.d + f_tau * c.tau.d + f_S2 * S2.d) / f_p;
    }
    const Dual pd(p, dp);
    const Dual e = c.tau + c.D + pd;
    const Dual v2 = S2 / (e * e);
    const Dual W = 1.0 / sqrt_(1.0 - v2);
    PrimT<Dual> out;
    out.rho = c.D / W;
    out.p = pd;
    out.eps = pd / (gm1 * out.rho);
    for (int i = 0; i < 3; ++i)
    {
        Dual m = Dual(0.0);
        for (int j = 0; j < 3; ++j)
            m += gUU[sym(i, j)] * c.S[j];
        out.v[i] = m / e;
    }
    return out;
}

// enforce_primitive_floors (Atmosphere.hpp:24-46) in tangent form; `in`
// holds the double input on which floors_rev decides (eps unused).
GRHD_HD inline PrimT<Dual> floors_tan(const Options &o, const Prim &in,
                                      const PrimT<Dual> &ind,
                                      const Dual G[6])
{
    PrimT<Dual> out;
    out.rho = in.rho > o.rho_floor ? ind.rho : Dual(fmax(in.rho, o.rho_floor));
    out.p = in.p > o.p_floor ? ind.p : Dual(fmax(in.p, o.p_floor));
    double Gv[6];
    for (int q = 0; q < 6; ++q)
        Gv[q] = G[q].v;
    const double v2 = vsq(in.v, Gv);
    if (v2 >= o.atmo_vmax2)
    {
        const Dual v2d = vsq(ind.v, G);
        const Dual s = sqrt_(o.atmo_vmax2 / v2d);
        for (int k = 0; k < 3; ++k)
            out.v[k] = ind.v[k] * s;
    }
    else
        for (int k = 0; k < 3; ++k)
            out.v[k] = ind.v[k];
    out.eps = out.p / ((o.G - 1.0) * out.rho);
    return out;
}

// rad of compute_characteristic_speeds in double, computed as
// char_speeds_rev computes it (its sign decides whether sqrt passes a
// derivative).
GRHD_HD inline double char_rad(const Options &o, const Prim &pr,
                               const Geo &g, int d)
{
    const double v2 = vsq(pr.v, g.gLL);
    const double h = 1.0 + pr.eps + pr.p / pr.rho;
    const double cs2 = o.G * pr.p / (pr.rho * h);
    const double vel = pr.v[d];
    const double den = 1.0 - v2 * cs2;
    const double Q = g.gUU[sym(d, d)] * den - vel * vel * (1.0 - cs2);
    return (1.0 - v2) * Q;
}

// compute_characteristic_speeds (shifted), RiemannSolvers.hpp:23-67, as
// char_speeds_rev differentiates it; rad_pos: char_rad(...) > 0.
GRHD_HD inline void char_speeds_tan(const Options &o, const PrimT<Dual> &pr,
                                    const GeoT<Dual> &g, int d, bool rad_pos,
                                    Dual &lo, Dual &hi)
{
    const Dual v2 = vsq(pr.v, g.gLL);
    const Dual h = 1.0 + pr.eps + pr.p / pr.rho;
    const Dual cs2 = o.G * pr.p / (pr.rho * h);
    const Dual cs = sqrt_(cs2);
    const Dual vel = pr.v[d];
    const Dual den = 1.0 - v2 * cs2;
    const Dual Q = g.gUU[sym(d, d)] * den - vel * vel * (1.0 - cs2);
    const Dual rad = (1.0 - v2) * Q;
    const Dual sr = rad_pos ? dual_sqrt_nz(rad) : Dual(0.0);
    const Dual root = cs * sr;
    const Dual base = vel * (1.0 - cs2);
    const Dual iden = 1.0 / den;
    lo = g.lapse * ((base - root) * iden) - g.shift[d];
    hi = g.lapse * ((base + root) * iden) - g.shift[d];
}

// The MUSCL-HLLE face flux (FiniteVolume.hpp:63-98, RiemannSolvers.hpp:
// 69-118) in tangent form with the recorded limiter branches, as
// face_flux_rev reverses it.  LL..RR: rho, p, v of cells i-1..i+2 and
// dLL..dRR their tangents; g: the face geometry with its tangent.
GRHD_HD inline ConsT<Dual> face_flux_tan(
    const Options &o, const double LL[5], const double L[5],
    const double R[5], const double RR[5], const double dLL[5],
    const double dL[5], const double dR[5], const double dRR[5],
    unsigned bitsL, unsigned bitsR, const GeoT<Dual> &g, int d)
{
    double ql[5], qr[5], dql[5], dqr[5];
    for (int c = 0; c < 5; ++c)
    {
        if (o.use_recon)
        {
            const int bl = bits_of(bitsL, c), br = bits_of(bitsR, c);
            const double sl = slope_value(bl, LL[c], L[c], R[c], o.theta);
            const double sr = slope_value(br, L[c], R[c], RR[c], o.theta);
            double wl, wc, wr;
            slope_weights(bl, o.theta, wl, wc, wr);
            const double dsl = wl * dLL[c] + wc * dL[c] + wr * dR[c];
            slope_weights(br, o.theta, wl, wc, wr);
            const double dsr = wl * dL[c] + wc * dR[c] + wr * dRR[c];
            ql[c] = L[c] + 0.5 * sl;
            qr[c] = R[c] - 0.5 * sr;
            dql[c] = dL[c] + 0.5 * dsl;
            dqr[c] = dR[c] - 0.5 * dsr;
        }
        else
        {
            ql[c] = L[c];
            qr[c] = R[c];
            dql[c] = dL[c];
            dqr[c] = dR[c];
        }
    }
    Prim lq, rq;
    PrimT<Dual> lqd, rqd;
    lq.rho = ql[0];
    lq.p = ql[1];
    rq.rho = qr[0];
    rq.p = qr[1];
    lq.eps = rq.eps = 0.0;
    lqd.rho = Dual(ql[0], dql[0]);
    lqd.p = Dual(ql[1], dql[1]);
    rqd.rho = Dual(qr[0], dqr[0]);
    rqd.p = Dual(qr[1], dqr[1]);
    lqd.eps = rqd.eps = Dual(0.0);
    for (int i = 0; i < 3; ++i)
    {
        lq.v[i] = ql[2 + i];
        rq.v[i] = qr[2 + i];
        lqd.v[i] = Dual(ql[2 + i], dql[2 + i]);
        rqd.v[i] = Dual(qr[2 + i], dqr[2 + i]);
    }
    // the double primal of face_flux_rev, which takes every decision
    Geo gv;
    values_of(g, gv);
    Prim lpv = lq, rpv = rq;
    floors(o, lpv, gv.gLL);
    floors(o, rpv, gv.gLL);
    double llov, lhiv, rlov, rhiv;
    char_speeds(o, lpv, gv, d, llov, lhiv);
    char_speeds(o, rpv, gv, d, rlov, rhiv);
    const bool lpos = char_rad(o, lpv, gv, d) > 0.0;
    const bool rpos = char_rad(o, rpv, gv, d) > 0.0;

    const PrimT<Dual> lp = floors_tan(o, lq, lqd, g.gLL);
    const PrimT<Dual> rp = floors_tan(o, rq, rqd, g.gLL);
    const ConsT<Dual> lc = p2c(lp, g.gLL);
    const ConsT<Dual> rc = p2c(rp, g.gLL);
    const ConsT<Dual> lf = phys_flux(lp, lc, d, g.lapse, g.shift);
    const ConsT<Dual> rf = phys_flux(rp, rc, d, g.lapse, g.shift);
    Dual llo, lhi, rlo, rhi;
    char_speeds_tan(o, lp, g, d, lpos, llo, lhi);
    char_speeds_tan(o, rp, g, d, rpos, rlo, rhi);
    const double slv = fmin(0.0, fmin(llov, rlov));
    const double suv = fmax(0.0, fmax(lhiv, rhiv));
    if (slv >= 0.0)
        return lf;
    if (suv <= 0.0)
        return rf;
    const Dual sl = llov <= rlov ? llo : rlo;
    const Dual su = lhiv >= rhiv ? lhi : rhi;
    const Dual inv = 1.0 / (su - sl);
    const Dual ss = sl * su;
    ConsT<Dual> f;
    f.D = (su * lf.D - sl * rf.D + ss * (rc.D - lc.D)) * inv;
    f.tau = (su * lf.tau - sl * rf.tau + ss * (rc.tau - lc.tau)) * inv;
    for (int i = 0; i < 3; ++i)
        f.S[i] = (su * lf.S[i] - sl * rf.S[i] + ss * (rc.S[i] - lc.S[i])) * inv;
    return f;
}

// The post-update recovery of one cell in tangent form, with the branch
// the forward sweep recorded (recovery_rev transposed): 0 kept Y, 1
// replaced it by p2c of the floored con2prim result at pressure pY, 2 by
// the atmosphere (v = 0: p2c of it does not depend on the metric).
GRHD_HD inline ConsT<Dual> recovery_tan(const Options &o, const ConsT<Dual> &Y,
                                        int br, double pY,
                                        const GeoT<Dual> &g)
{
    if (br == 0)
        return Y;
    Geo gv;
    values_of(g, gv);
    if (br != 1)
    {
        const Cons c = p2c(atmosphere(o), gv.gLL);
        ConsT<Dual> z;
        z.D = Dual(c.D);
        z.tau = Dual(c.tau);
        for (int i = 0; i < 3; ++i)
            z.S[i] = Dual(c.S[i]);
        return z;
    }
    const PrimT<Dual> pr = con2prim_tan(o, Y, g.gUU, pY);
    const Prim prv = c2p_at(o, values_of(Y), gv.gUU, pY);
    const PrimT<Dual> fl = floors_tan(o, prv, pr, g.gLL);
    return p2c(fl, g.gLL);
}

// ------------------------------------------------------------ work items

// One RHS evaluation of the tangent-linear sweep: the forward tape's state,
// primitive cache and limiter bits at this stage, the tangent of the
// state's conserved variables (interior) and the spin component da of the
// direction.
struct TanRhs
{
    BoxDev b; // cs = pcs = ghosted volume, rcs = interior volume
    Options o;
    double M, a, da;
    double inv_dx[3];
    const double *U;      // RHS input state (11 comps)
    const double *P;      // its primitive cache (rho, p, v)
    const unsigned *bits; // limiter branches, 10 bits per direction
    const double *dU;     // tangent of U's conserved variables (5, interior)
    double *dP;           // tangent of the primitive cache (5, ghosted)
    double *dS;           // tangent of the sources (5, interior)
    double *dk;           // out: tangent of the RHS (5, interior)
    double mu;            // weight of this RHS's Mdot in J
};

__host__ __device__ inline void ks_geo_tan(const TanRhs &A, const int c[3],
                                           GeoT<Dual> &g)
{
    double x, y, z;
    cell_xyz(A.o, c[0], c[1], c[2], x, y, z);
    ks_metric_spin<false>(A.M, A.a, x, y, z, g, nullptr);
    scale_tangent(g, A.da);
}

// Interior cell t: the tangent of its primitive cache (con2prim at the
// taped pressure, implicit function theorem) and of its static sources
// (cell_rev_item's forward half, transposed).
__host__ __device__ inline void tan_cell_item(const TanRhs &A, int64_t t)
{
    const BoxDev &b = A.b;
    const Options &o = A.o;
    int c[3];
    c[0] = b.lo[0] + (int)(t % b.in[0]);
    const int64_t r = t / b.in[0];
    c[1] = b.lo[1] + (int)(r % b.in[1]);
    c[2] = b.lo[2] + (int)(r / b.in[1]);
    const int64_t g = b.gidx(c[0], c[1], c[2]);
    if (excised(o, c[0], c[1], c[2]))
    {
        for (int q = 0; q < 5; ++q)
        {
            A.dP[q * b.pcs + g] = 0.0;
            A.dS[q * b.rcs + t] = 0.0;
        }
        return;
    }
    double x, y, z;
    cell_xyz(o, c[0], c[1], c[2], x, y, z);
    GeoFullT<Dual> fd;
    ks_metric_spin<true>(A.M, A.a, x, y, z, fd.g, &fd);
    scale_tangent(fd, A.da);
    const Cons Uv = load_cons5(A.U, b.cs, g);
    ConsT<Dual> cu;
    cu.D = Dual(Uv.D, A.dU[0 * b.rcs + t]);
    for (int i = 0; i < 3; ++i)
        cu.S[i] = Dual(Uv.S[i], A.dU[(1 + i) * b.rcs + t]);
    cu.tau = Dual(Uv.tau, A.dU[4 * b.rcs + t]);
    double q5[5];
    load5(A.P, b.pcs, g, q5);
    const PrimT<Dual> pr = con2prim_tan(o, cu, fd.g.gUU, q5[1]);
    A.dP[0 * b.pcs + g] = pr.rho.d;
    A.dP[1 * b.pcs + g] = pr.p.d;
    for (int i = 0; i < 3; ++i)
        A.dP[(2 + i) * b.pcs + g] = pr.v[i].d;
    double ds[5] = {0, 0, 0, 0, 0};
    if (o.use_src)
    {
        Prim pv;
        pv.rho = q5[0];
        pv.p = q5[1];
        pv.eps = pv.p / ((o.G - 1.0) * pv.rho);
        for (int i = 0; i < 3; ++i)
            pv.v[i] = q5[2 + i];
        Geo gv;
        values_of(fd.g, gv);
        Prim fl = pv;
        floors(o, fl, gv.gLL);
        if (!is_atmo(o, fl, o.src_atmo_factor))
        {
            const PrimT<Dual> fld = floors_tan(o, pv, pr, fd.g.gLL);
            const ConsT<Dual> sv = static_sources(fld, cu, fd);
            ds[0] = sv.D.d;
            ds[1] = sv.S[0].d;
            ds[2] = sv.S[1].d;
            ds[3] = sv.S[2].d;
            ds[4] = sv.tau.d;
        }
    }
    for (int q = 0; q < 5; ++q)
        A.dS[q * b.rcs + t] = ds[q];
}

// Physical ghost cell g (outside the interior in exactly one direction):
// the tangent of its primitive cache, its source cell's con2prim tangent
// through the ghost's floors (shell_rev_item transposed).  Other shell
// cells feed no face and get zero.
__host__ __device__ inline void tan_ghost_item(const TanRhs &A, int64_t g)
{
    const BoxDev &b = A.b;
    int c[3];
    cell_of(b, g, c);
    int out = 0, d0 = -1;
    for (int d = 0; d < 3; ++d)
        if (c[d] < b.lo[d] || c[d] > b.hi[d])
        {
            ++out;
            d0 = d;
        }
    if (out == 0)
        return;
    if (out != 1)
    {
        for (int q = 0; q < 5; ++q)
            A.dP[q * b.pcs + g] = 0.0;
        return;
    }
    int s[3] = {c[0], c[1], c[2]};
    s[d0] = c[d0] < b.lo[d0] ? b.lo[d0] : b.hi[d0];
    const int64_t sg = b.gidx(s[0], s[1], s[2]);
    double sq[5];
    load5(A.P, b.pcs, sg, sq);
    Prim in;
    in.rho = sq[0];
    in.p = sq[1];
    in.eps = 0.0;
    for (int i = 0; i < 3; ++i)
        in.v[i] = sq[2 + i];
    PrimT<Dual> ind;
    ind.rho = Dual(sq[0], A.dP[0 * b.pcs + sg]);
    ind.p = Dual(sq[1], A.dP[1 * b.pcs + sg]);
    ind.eps = Dual(0.0);
    for (int i = 0; i < 3; ++i)
        ind.v[i] = Dual(sq[2 + i], A.dP[(2 + i) * b.pcs + sg]);
    GeoT<Dual> gd;
    ks_geo_tan(A, c, gd);
    const PrimT<Dual> o2 = floors_tan(A.o, in, ind, gd.gLL);
    A.dP[0 * b.pcs + g] = o2.rho.d;
    A.dP[1 * b.pcs + g] = o2.p.d;
    for (int i = 0; i < 3; ++i)
        A.dP[(2 + i) * b.pcs + g] = o2.v[i].d;
}

// The face between L and R = L + e_d in tangent form; gf receives the
// face geometry.
__host__ __device__ inline ConsT<Dual> tan_face(const TanRhs &A, int d,
                                                const int L[3],
                                                GeoT<Dual> &gf)
{
    const BoxDev &b = A.b;
    const int64_t sd = stride_of(b, d);
    const int64_t gL = b.gidx(L[0], L[1], L[2]);
    int R[3] = {L[0], L[1], L[2]};
    R[d] += 1;
    GeoT<Dual> gl, gr;
    ks_geo_tan(A, L, gl);
    ks_geo_tan(A, R, gr);
    average_geo(gl, gr, gf);
    double q[4][5], dq[4][5];
    for (int m = 0; m < 4; ++m)
    {
        const int64_t gm = gL + (m - 1) * sd;
        load5(A.P, b.pcs, gm, q[m]);
        load5(A.dP, b.pcs, gm, dq[m]);
    }
    const unsigned bL = (A.bits[gL] >> (10 * d)) & 0x3ffu;
    const unsigned bR = (A.bits[gL + sd] >> (10 * d)) & 0x3ffu;
    return face_flux_tan(A.o, q[0], q[1], q[2], q[3], dq[0], dq[1], dq[2],
                         dq[3], bL, bR, gf, d);
}

// Interior cell t: the tangent of its RHS, -(dF_hi - dF_lo) / dx summed
// over the directions plus its source tangent; returns mu times the
// tangent of the accretion-sphere faces whose lower cell it is (each face
// of the voxelised sphere between two interior cells counted once, as the
// forward counts it).
__host__ __device__ inline double tan_rhs_item(const TanRhs &A, int64_t t)
{
    const BoxDev &b = A.b;
    const Options &o = A.o;
    int c[3];
    c[0] = b.lo[0] + (int)(t % b.in[0]);
    const int64_t r = t / b.in[0];
    c[1] = b.lo[1] + (int)(r % b.in[1]);
    c[2] = b.lo[2] + (int)(r / b.in[1]);
    if (excised(o, c[0], c[1], c[2]))
    {
        for (int q = 0; q < 5; ++q)
            A.dk[q * b.rcs + t] = 0.0;
        return 0.0;
    }
    double dk[5];
    for (int q = 0; q < 5; ++q)
        dk[q] = A.dS[q * b.rcs + t];
    double dm = 0.0;
    for (int d = 0; d < 3; ++d)
    {
        int L[3] = {c[0], c[1], c[2]};
        L[d] -= 1;
        GeoT<Dual> gf;
        const ConsT<Dual> flo = tan_face(A, d, L, gf);
        const ConsT<Dual> fhi = tan_face(A, d, c, gf);
        const double fl[5] = {flo.D.d, flo.S[0].d, flo.S[1].d, flo.S[2].d,
                              flo.tau.d};
        const double fh[5] = {fhi.D.d, fhi.S[0].d, fhi.S[1].d, fhi.S[2].d,
                              fhi.tau.d};
        for (int q = 0; q < 5; ++q)
            dk[q] -= A.inv_dx[d] * (fh[q] - fl[q]);
        int R[3] = {c[0], c[1], c[2]};
        R[d] += 1;
        if (A.mu != 0.0 && o.accretion_radius > 0.0 && R[d] <= b.hi[d])
        {
            const bool il = radius_of(o, c) < o.accretion_radius;
            const bool ir = radius_of(o, R) < o.accretion_radius;
            if (il != ir)
            {
                const Dual m = sqrt_det(gf.gLL) * fhi.D;
                dm += (il ? -1.0 : 1.0) * o.dx * o.dx * A.mu * m.d;
            }
        }
    }
    for (int q = 0; q < 5; ++q)
        A.dk[q * b.rcs + t] = dk[q];
    return dm;
}

// The RK4 stage combination and post-update recovery of interior cell t in
// tangent form (stage_tape_item's arithmetic, recorded recovery branch).
// dUn: tangent of U^n; dk: of this stage's RHS; dacc: of the accumulator;
// out: of the stage's output state.
__host__ __device__ inline void tan_stage_item(
    const BoxDev &b, const Options &o, double M, double a, double da,
    int stage, double dt, const double *dUn, const double *dk, double *dacc,
    const double *Y, const double *pY, const unsigned char *br, double *out,
    int64_t t)
{
    const int i = b.lo[0] + (int)(t % b.in[0]);
    const int64_t r = t / b.in[0];
    const int j = b.lo[1] + (int)(r % b.in[1]);
    const int k = b.lo[2] + (int)(r / b.in[1]);
    if (excised(o, i, j, k))
    {
        for (int q = 0; q < 5; ++q)
            out[q * b.rcs + t] = dUn[q * b.rcs + t];
        return;
    }
    const double cst = (stage == 2) ? dt : 0.5 * dt;
    const double dt6 = dt / 6.0;
    double dy[5];
    for (int q = 0; q < 5; ++q)
    {
        const double kk = dk[q * b.rcs + t];
        const double u0 = dUn[q * b.rcs + t];
        double av = (stage == 0) ? kk : dacc[q * b.rcs + t];
        if (stage == 1 || stage == 2)
            av = av + 2.0 * kk;
        if (stage < 3)
        {
            dacc[q * b.rcs + t] = av;
            dy[q] = u0 + cst * kk;
        }
        else
            dy[q] = u0 + dt6 * (av + kk);
    }
    ConsT<Dual> Yd;
    Yd.D = Dual(Y[0 * b.rcs + t], dy[0]);
    for (int m = 0; m < 3; ++m)
        Yd.S[m] = Dual(Y[(1 + m) * b.rcs + t], dy[1 + m]);
    Yd.tau = Dual(Y[4 * b.rcs + t], dy[4]);
    double x, y, z;
    cell_xyz(o, i, j, k, x, y, z);
    GeoT<Dual> gd;
    ks_metric_spin<false>(M, a, x, y, z, gd, nullptr);
    scale_tangent(gd, da);
    const ConsT<Dual> U = recovery_tan(o, Yd, br[t], pY[t], gd);
    out[0 * b.rcs + t] = U.D.d;
    for (int m = 0; m < 3; ++m)
        out[(1 + m) * b.rcs + t] = U.S[m].d;
    out[4 * b.rcs + t] = U.tau.d;
}

} // namespace adj
} // namespace grhd
