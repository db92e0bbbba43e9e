// grhd_adjoint.cuh -- reverse-mode (discrete adjoint) versions of the FP64
// pointwise physics in grhd_device.cuh.  No counterpart in the reference.
//
// Each *_rev function takes the forward inputs and the adjoint of the
// forward outputs ("bar" values) and ADDS the adjoints of the inputs:
// x_bar += (d out / d x)^T out_bar.  The forward quantities are recomputed
// from the inputs inside each function, so they need no tape; branches of
// the forward (floors, velocity caps, the HLLE wave-speed cases) are taken
// again from the same inputs, and the MUSCL limiter branch comes from the
// bits recorded in the forward sweep (slope_branch).
//
// Geometry adjoints are accumulated field by field (GeoBar / GeoFullBar:
// the adjoint of each stored component, symmetric tensors in the packed
// 00 01 02 11 12 22 order, an off-diagonal entry collecting both of its
// uses); contracting them with the spin derivative of the same fields
// (the metric evaluated in dual numbers) gives the spin adjoint.
#pragma once

#include "grhd_device.cuh"
#include "grhd_dual.cuh"

namespace grhd {
namespace adj {

struct PrimBar
{
    double rho, eps, p, v[3];
};
struct ConsBar
{
    double D, S[3], tau;
};
struct GeoBar
{
    double gLL[6], gUU[6], lapse, shift[3];
};
struct GeoFullBar
{
    GeoBar g;
    double K[6], dlapse[3], dlnsqrtg[3], dgamma[3][6], dshift[3][3];
};

GRHD_HD inline PrimBar zero_prim_bar()
{
    PrimBar b;
    b.rho = b.eps = b.p = 0.0;
    b.v[0] = b.v[1] = b.v[2] = 0.0;
    return b;
}
GRHD_HD inline ConsBar zero_cons_bar()
{
    ConsBar b;
    b.D = b.tau = 0.0;
    b.S[0] = b.S[1] = b.S[2] = 0.0;
    return b;
}
GRHD_HD inline void zero(GeoBar &g)
{
    for (int q = 0; q < 6; ++q)
        g.gLL[q] = g.gUU[q] = 0.0;
    g.lapse = 0.0;
    g.shift[0] = g.shift[1] = g.shift[2] = 0.0;
}
GRHD_HD inline void zero(GeoFullBar &f)
{
    zero(f.g);
    for (int q = 0; q < 6; ++q)
        f.K[q] = 0.0;
    for (int d = 0; d < 3; ++d)
    {
        f.dlapse[d] = f.dlnsqrtg[d] = 0.0;
        for (int q = 0; q < 6; ++q)
            f.dgamma[d][q] = 0.0;
        for (int q = 0; q < 3; ++q)
            f.dshift[d][q] = 0.0;
    }
}

// Symmetric-matrix adjoint of a bilinear use G_ij a_i b_j summed over all
// ordered pairs: the packed entry q = sym(i,j) collects every (i,j).
GRHD_HD inline void sym_outer_add(double Gbar[6], double w, const double a[3],
                                  const double b[3])
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            Gbar[sym(i, j)] += w * a[i] * b[j];
}

GRHD_HD inline void lower(const double G[6], const double v[3], double vL[3])
{
    vL[0] = G[0] * v[0] + G[1] * v[1] + G[2] * v[2];
    vL[1] = G[1] * v[0] + G[3] * v[1] + G[4] * v[2];
    vL[2] = G[2] * v[0] + G[4] * v[1] + G[5] * v[2];
}

// v2 = v^T G v
GRHD_HD inline void vsq_rev(const double v[3], const double G[6],
                            double v2bar, double vbar[3], double Gbar[6])
{
    double vL[3];
    lower(G, v, vL);
    for (int i = 0; i < 3; ++i)
        vbar[i] += 2.0 * v2bar * vL[i];
    sym_outer_add(Gbar, v2bar, v, v);
}

// compute_conserved (p2c), Valencia.hpp:55-73
GRHD_HD inline void p2c_rev(const Prim &pr, const double G[6],
                            const ConsBar &cb, PrimBar &pb, double Gbar[6])
{
    double vL[3];
    lower(G, pr.v, vL);
    const double v2 = vL[0] * pr.v[0] + vL[1] * pr.v[1] + vL[2] * pr.v[2];
    const double W = 1.0 / sqrt(1.0 - v2);
    const double h = 1.0 + pr.eps + pr.p / pr.rho;
    const double rhw = pr.rho * h * W * W;
    const double rhwbar =
        cb.tau + cb.S[0] * vL[0] + cb.S[1] * vL[1] + cb.S[2] * vL[2];
    double vLbar[3];
    for (int i = 0; i < 3; ++i)
        vLbar[i] = cb.S[i] * rhw;
    const double Dbar = cb.D - cb.tau; // tau = rhw - p - D
    double Wbar = Dbar * pr.rho;
    pb.rho += Dbar * W;
    pb.p -= cb.tau;
    pb.rho += rhwbar * h * W * W;
    const double hbar = rhwbar * pr.rho * W * W;
    Wbar += rhwbar * pr.rho * h * 2.0 * W;
    pb.eps += hbar;
    pb.p += hbar / pr.rho;
    pb.rho -= hbar * pr.p / (pr.rho * pr.rho);
    const double v2bar = Wbar * 0.5 * W * W * W;
    // vL = G v
    double t[3];
    lower(G, vLbar, t);
    for (int j = 0; j < 3; ++j)
        pb.v[j] += t[j];
    sym_outer_add(Gbar, 1.0, vLbar, pr.v);
    vsq_rev(pr.v, G, v2bar, pb.v, Gbar);
}

// enforce_primitive_floors, Atmosphere.hpp:24-46.  `in` is the input of
// the floors (eps unused: the floors recompute it); `ob` the adjoint of
// their output (eps included); adds the adjoint of rho, p, v of the input.
GRHD_HD inline void floors_rev(const Options &o, const Prim &in,
                               const double G[6], const PrimBar &ob,
                               PrimBar &ib, double Gbar[6])
{
    const double rho1 = fmax(in.rho, o.rho_floor);
    const double p1 = fmax(in.p, o.p_floor);
    const double gm1 = o.G - 1.0;
    double rho1bar = ob.rho, p1bar = ob.p;
    p1bar += ob.eps / (gm1 * rho1);
    rho1bar -= ob.eps * p1 / (gm1 * rho1 * rho1);
    if (in.rho > o.rho_floor)
        ib.rho += rho1bar;
    if (in.p > o.p_floor)
        ib.p += p1bar;
    const double v2 = vsq(in.v, G);
    if (v2 >= o.atmo_vmax2)
    {
        const double s = sqrt(o.atmo_vmax2 / v2);
        const double sbar =
            ob.v[0] * in.v[0] + ob.v[1] * in.v[1] + ob.v[2] * in.v[2];
        for (int k = 0; k < 3; ++k)
            ib.v[k] += s * ob.v[k];
        vsq_rev(in.v, G, -0.5 * s / v2 * sbar, ib.v, Gbar);
    }
    else
    {
        for (int k = 0; k < 3; ++k)
            ib.v[k] += ob.v[k];
    }
}

// compute_flux, Valencia.hpp:230-259
GRHD_HD inline void phys_flux_rev(const Prim &pr, const Cons &c, int d,
                                  double lapse, const double shift[3],
                                  const ConsBar &fb, PrimBar &pb, ConsBar &cb,
                                  double &lapse_bar, double shift_bar[3])
{
    const double tv = lapse * pr.v[d] - shift[d];
    const double ap = lapse * pr.p;
    cb.D += fb.D * tv;
    cb.tau += fb.tau * tv;
    for (int j = 0; j < 3; ++j)
        cb.S[j] += fb.S[j] * tv;
    const double tvbar = fb.D * c.D + fb.tau * c.tau + fb.S[0] * c.S[0] +
                         fb.S[1] * c.S[1] + fb.S[2] * c.S[2];
    const double apbar = fb.tau * pr.v[d] + fb.S[d];
    pb.v[d] += fb.tau * ap + tvbar * lapse;
    pb.p += apbar * lapse;
    lapse_bar += tvbar * pr.v[d] + apbar * pr.p;
    shift_bar[d] -= tvbar;
}

// compute_characteristic_speeds (shifted), RiemannSolvers.hpp:23-67
GRHD_HD inline void char_speeds_rev(const Options &o, const Prim &pr,
                                    const Geo &g, int d, double lobar,
                                    double hibar, PrimBar &pb, GeoBar &gb)
{
    const double v2 = vsq(pr.v, g.gLL);
    const double h = 1.0 + pr.eps + pr.p / pr.rho;
    const double cs2 = o.G * pr.p / (pr.rho * h);
    const double cs = sqrt(cs2);
    const double vel = pr.v[d];
    const double den = 1.0 - v2 * cs2;
    const double gdd = g.gUU[sym(d, d)];
    const double Q = gdd * den - vel * vel * (1.0 - cs2);
    const double rad = (1.0 - v2) * Q;
    const double sr = sqrt(fmax(0.0, rad));
    const double root = cs * sr;
    const double base = vel * (1.0 - cs2);
    const double iden = 1.0 / den;

    gb.shift[d] -= lobar + hibar;
    gb.lapse += lobar * (base - root) * iden + hibar * (base + root) * iden;
    const double qlo = g.lapse * lobar, qhi = g.lapse * hibar;
    const double basebar = (qlo + qhi) * iden;
    const double rootbar = (qhi - qlo) * iden;
    const double idenbar = qlo * (base - root) + qhi * (base + root);
    double denbar = -idenbar * iden * iden;
    double velbar = basebar * (1.0 - cs2);
    double cs2bar = -basebar * vel;
    double csbar = rootbar * sr;
    double radbar = (rad > 0.0) ? rootbar * cs / (2.0 * sr) : 0.0;
    double v2bar = -radbar * Q;
    const double Qbar = radbar * (1.0 - v2);
    gb.gUU[sym(d, d)] += Qbar * den;
    denbar += Qbar * gdd;
    velbar -= Qbar * 2.0 * vel * (1.0 - cs2);
    cs2bar += Qbar * vel * vel;
    v2bar -= denbar * cs2;
    cs2bar -= denbar * v2;
    cs2bar += csbar / (2.0 * cs);
    // cs2 = G p / (rho h)
    pb.p += cs2bar * o.G / (pr.rho * h);
    pb.rho -= cs2bar * cs2 / pr.rho;
    const double hbar = -cs2bar * cs2 / h;
    pb.eps += hbar;
    pb.p += hbar / pr.rho;
    pb.rho -= hbar * pr.p / (pr.rho * pr.rho);
    pb.v[d] += velbar;
    vsq_rev(pr.v, g.gLL, v2bar, pb.v, gb.gLL);
}

// ---------------------------------------------------------------- limiter

// Which argument compute_limited_slope (Reconstruction.hpp:16-37) selects:
// 0 none (zero slope), 1 theta (c - l), 2 (r - l)/2, 3 theta (r - c).
GRHD_HD inline int slope_branch(double l, double c, double r, double theta)
{
    const double A = theta * (c - l), B = 0.5 * (r - l), C = theta * (r - c);
    int ib;
    double iv;
    if (B * C <= 0.0)
    {
        ib = 0;
        iv = 0.0;
    }
    else if (B > 0.0)
    {
        ib = (B <= C) ? 2 : 3;
        iv = fmin(B, C);
    }
    else
    {
        ib = (B >= C) ? 2 : 3;
        iv = fmax(B, C);
    }
    if (A * iv <= 0.0)
        return 0;
    if (A > 0.0)
        return (A <= iv) ? 1 : ib;
    return (A >= iv) ? 1 : ib;
}

GRHD_HD inline double slope_value(int br, double l, double c, double r,
                                  double theta)
{
    switch (br)
    {
    case 1:
        return theta * (c - l);
    case 2:
        return 0.5 * (r - l);
    case 3:
        return theta * (r - c);
    default:
        return 0.0;
    }
}

// d slope / d (l, c, r) of a recorded branch
GRHD_HD inline void slope_weights(int br, double theta, double &wl,
                                  double &wc, double &wr)
{
    wl = wc = wr = 0.0;
    if (br == 1)
    {
        wl = -theta;
        wc = theta;
    }
    else if (br == 2)
    {
        wl = -0.5;
        wr = 0.5;
    }
    else if (br == 3)
    {
        wc = -theta;
        wr = theta;
    }
}

// The limiter branches of one cell in one direction, 2 bits per
// primitive component (rho, p, v0, v1, v2).
GRHD_HD inline unsigned slope_bits(const double l[5], const double c[5],
                                   const double r[5], double theta)
{
    unsigned bits = 0;
    for (int q = 0; q < 5; ++q)
        bits |= (unsigned)slope_branch(l[q], c[q], r[q], theta) << (2 * q);
    return bits;
}

GRHD_HD inline int bits_of(unsigned bits, int q) { return (bits >> (2 * q)) & 3; }

// ------------------------------------------------------------- face flux

// Reverse of face_flux (FiniteVolume.hpp:63-98 with the HLLE of
// RiemannSolvers.hpp:69-118) for the face between cells L and R in
// direction d.  LL..RR hold rho, p, v0, v1, v2 of cells i-1..i+2; bitsL /
// bitsR the recorded limiter branches of L and R in direction d.  Given
// Fbar, writes the adjoints of the two reconstructed face states before
// the floors (qlbar, qrbar, rho p v order) and adds the face-geometry
// adjoint.  Returns F_D (the forward rest-mass flux) for the accretion
// term.
GRHD_HD inline double face_flux_rev(const Options &o, const double LL[5],
                                    const double L[5], const double R[5],
                                    const double RR[5], unsigned bitsL,
                                    unsigned bitsR, const Geo &g, int d,
                                    const ConsBar &Fb, double qlbar[5],
                                    double qrbar[5], GeoBar &gb)
{
    double ql[5], qr[5];
    for (int c = 0; c < 5; ++c)
    {
        if (o.use_recon)
        {
            const double sl =
                slope_value(bits_of(bitsL, c), LL[c], L[c], R[c], o.theta);
            const double sr =
                slope_value(bits_of(bitsR, c), L[c], R[c], RR[c], o.theta);
            ql[c] = L[c] + 0.5 * sl;
            qr[c] = R[c] - 0.5 * sr;
        }
        else
        {
            ql[c] = L[c];
            qr[c] = R[c];
        }
    }
    Prim lq, rq;
    lq.rho = ql[0];
    lq.p = ql[1];
    rq.rho = qr[0];
    rq.p = qr[1];
    lq.eps = rq.eps = 0.0;
    for (int i = 0; i < 3; ++i)
    {
        lq.v[i] = ql[2 + i];
        rq.v[i] = qr[2 + i];
    }
    Prim lp = lq, rp = rq;
    floors(o, lp, g.gLL);
    floors(o, rp, g.gLL);
    const Cons lc = p2c(lp, g.gLL);
    const Cons rc = p2c(rp, g.gLL);
    const Cons lf = phys_flux(lp, lc, d, g.lapse, g.shift);
    const Cons rf = phys_flux(rp, rc, d, g.lapse, g.shift);
    double llo, lhi, rlo, rhi;
    char_speeds(o, lp, g, d, llo, lhi);
    char_speeds(o, rp, g, d, rlo, rhi);
    const double sl = fmin(0.0, fmin(llo, rlo));
    const double su = fmax(0.0, fmax(lhi, rhi));

    ConsBar lfb = zero_cons_bar(), rfb = zero_cons_bar();
    ConsBar lcb = zero_cons_bar(), rcb = zero_cons_bar();
    double llob = 0.0, lhib = 0.0, rlob = 0.0, rhib = 0.0;
    double FD;
    if (sl >= 0.0)
    {
        lfb = Fb;
        FD = lf.D;
    }
    else if (su <= 0.0)
    {
        rfb = Fb;
        FD = rf.D;
    }
    else
    {
        const double inv = 1.0 / (su - sl);
        const double ss = sl * su;
        const double lfv[5] = {lf.D, lf.S[0], lf.S[1], lf.S[2], lf.tau};
        const double rfv[5] = {rf.D, rf.S[0], rf.S[1], rf.S[2], rf.tau};
        const double lcv[5] = {lc.D, lc.S[0], lc.S[1], lc.S[2], lc.tau};
        const double rcv[5] = {rc.D, rc.S[0], rc.S[1], rc.S[2], rc.tau};
        const double fbv[5] = {Fb.D, Fb.S[0], Fb.S[1], Fb.S[2], Fb.tau};
        double lfbv[5], rfbv[5], lcbv[5], rcbv[5];
        double subar = 0.0, slbar = 0.0;
        FD = (su * lf.D - sl * rf.D + ss * (rc.D - lc.D)) * inv;
        for (int q = 0; q < 5; ++q)
        {
            const double F =
                (su * lfv[q] - sl * rfv[q] + ss * (rcv[q] - lcv[q])) * inv;
            lfbv[q] = su * inv * fbv[q];
            rfbv[q] = -sl * inv * fbv[q];
            rcbv[q] = ss * inv * fbv[q];
            lcbv[q] = -ss * inv * fbv[q];
            subar += fbv[q] * (lfv[q] + sl * (rcv[q] - lcv[q]) - F) * inv;
            slbar += fbv[q] * (-rfv[q] + su * (rcv[q] - lcv[q]) + F) * inv;
        }
        lfb.D = lfbv[0];
        lfb.S[0] = lfbv[1];
        lfb.S[1] = lfbv[2];
        lfb.S[2] = lfbv[3];
        lfb.tau = lfbv[4];
        rfb.D = rfbv[0];
        rfb.S[0] = rfbv[1];
        rfb.S[1] = rfbv[2];
        rfb.S[2] = rfbv[3];
        rfb.tau = rfbv[4];
        lcb.D = lcbv[0];
        lcb.S[0] = lcbv[1];
        lcb.S[1] = lcbv[2];
        lcb.S[2] = lcbv[3];
        lcb.tau = lcbv[4];
        rcb.D = rcbv[0];
        rcb.S[0] = rcbv[1];
        rcb.S[1] = rcbv[2];
        rcb.S[2] = rcbv[3];
        rcb.tau = rcbv[4];
        // sl = min(llo, rlo) < 0, su = max(lhi, rhi) > 0
        if (llo <= rlo)
            llob = slbar;
        else
            rlob = slbar;
        if (lhi >= rhi)
            lhib = subar;
        else
            rhib = subar;
    }
    PrimBar lpb = zero_prim_bar(), rpb = zero_prim_bar();
    phys_flux_rev(lp, lc, d, g.lapse, g.shift, lfb, lpb, lcb, gb.lapse,
                  gb.shift);
    phys_flux_rev(rp, rc, d, g.lapse, g.shift, rfb, rpb, rcb, gb.lapse,
                  gb.shift);
    char_speeds_rev(o, lp, g, d, llob, lhib, lpb, gb);
    char_speeds_rev(o, rp, g, d, rlob, rhib, rpb, gb);
    p2c_rev(lp, g.gLL, lcb, lpb, gb.gLL);
    p2c_rev(rp, g.gLL, rcb, rpb, gb.gLL);
    PrimBar lqb = zero_prim_bar(), rqb = zero_prim_bar();
    floors_rev(o, lq, g.gLL, lpb, lqb, gb.gLL);
    floors_rev(o, rq, g.gLL, rpb, rqb, gb.gLL);
    qlbar[0] = lqb.rho;
    qlbar[1] = lqb.p;
    qrbar[0] = rqb.rho;
    qrbar[1] = rqb.p;
    for (int i = 0; i < 3; ++i)
    {
        qlbar[2 + i] = lqb.v[i];
        qrbar[2 + i] = rqb.v[i];
    }
    return FD;
}

// ------------------------------------------------------------- con2prim

// Reverse of recover_primitive (Valencia.hpp:116-228) at its converged
// pressure p: the primitives are closed forms of (D, S, tau, gamma^ij, p)
// and p is the root of the pressure residual f, so by the implicit
// function theorem dp = -(f_D dD + f_tau dtau + f_S2 dS2) / f_p.  A
// pressure pinned at the recovery floor (the solve returns the floor when
// the residual there is within tolerance) does not move.  pb: adjoint of
// (rho, eps, p, v); adds the adjoint of the conserved variables and of
// gamma^ij.
GRHD_HD inline void con2prim_rev(const Options &o, const Cons &c,
                                 const double gUU[6], double p,
                                 const PrimBar &pb, ConsBar &cb,
                                 double gUUbar[6])
{
    const double S2 = c2p_S2(c, gUU);
    const double e = c.tau + c.D + p;
    const double v2 = div_(S2, e * e);
    const double W = rcp_(sqrt_(1.0 - v2));
    const double rho = div_(c.D, W);
    const double gm1 = o.G - 1.0;
    const double eps = div_(p, gm1 * rho);
    double m[3];
    lower(gUU, c.S, m);
    double pbar = pb.p + div_(pb.eps, gm1 * rho);
    const double rhobar = pb.rho - div_(pb.eps * eps, rho);
    cb.D += div_(rhobar, W);
    const double Wbar = div_(-rhobar * rho, W);
    const double ie = rcp_(e);
    double mbar[3], ebar = 0.0;
    for (int i = 0; i < 3; ++i)
    {
        mbar[i] = pb.v[i] * ie;
        ebar -= pb.v[i] * m[i] * ie * ie;
    }
    const double v2bar = Wbar * 0.5 * W * W * W;
    double S2bar = v2bar * ie * ie;
    ebar -= 2.0 * v2bar * v2 * ie;
    cb.tau += ebar;
    cb.D += ebar;
    pbar += ebar;
    if (p > o.rec_pfloor)
    {
        const double Gfac = div_(o.G, gm1);
        const double fW = c.D + 2.0 * Gfac * p * W;
        const double dWdv2 = 0.5 * W * W * W;
        const double dv2de = -2.0 * v2 * ie;
        const double f_p = Gfac * W * W + fW * dWdv2 * dv2de - 1.0;
        const double f_D = W + fW * dWdv2 * dv2de - 1.0;
        const double f_tau = fW * dWdv2 * dv2de - 1.0;
        const double f_S2 = fW * dWdv2 * ie * ie;
        const double q = div_(-pbar, f_p);
        cb.D += q * f_D;
        cb.tau += q * f_tau;
        S2bar += q * f_S2;
    }
    // S2 = S^T gUU S, m = gUU S
    for (int j = 0; j < 3; ++j)
        cb.S[j] += 2.0 * S2bar * m[j];
    sym_outer_add(gUUbar, S2bar, c.S, c.S);
    double t[3];
    lower(gUU, mbar, t);
    for (int j = 0; j < 3; ++j)
        cb.S[j] += t[j];
    sym_outer_add(gUUbar, 1.0, mbar, c.S);
}

// The primitives of recover_primitive at a known converged pressure p
// (c2p_finish without the velocity check).
GRHD_HD inline Prim c2p_at(const Options &o, const Cons &c,
                           const double gUU[6], double p)
{
    Prim out;
    const double S2 = c2p_S2(c, gUU);
    const double e = c.tau + c.D + p;
    const double v2 = div_(S2, e * e);
    const double W = rcp_(sqrt_(1.0 - v2));
    out.rho = div_(c.D, W);
    out.p = p;
    out.eps = div_(p, (o.G - 1.0) * out.rho);
    const double ie = rcp_(e);
    out.v[0] = (gUU[0] * c.S[0] + gUU[1] * c.S[1] + gUU[2] * c.S[2]) * ie;
    out.v[1] = (gUU[1] * c.S[0] + gUU[3] * c.S[1] + gUU[4] * c.S[2]) * ie;
    out.v[2] = (gUU[2] * c.S[0] + gUU[4] * c.S[1] + gUU[5] * c.S[2]) * ie;
    return out;
}

// -------------------------------------------------------------- sources

// compute_static_metric_source_terms, StaticMetric.hpp:193-275, reversed.
// pr: the floored primitives the forward used; c: conserved variables.
GRHD_HD inline void static_sources_rev(const Prim &pr, const Cons &c,
                                       const GeoFull &f, const ConsBar &sb,
                                       PrimBar &pb, ConsBar &cb,
                                       GeoFullBar &fb)
{
    const Geo &g = f.g;
    double vL[3];
    lower(g.gLL, pr.v, vL);
    const double v2 = vL[0] * pr.v[0] + vL[1] * pr.v[1] + vL[2] * pr.v[2];
    const double W = rsqrt_(1.0 - v2);
    const double h = 1.0 + pr.eps + div_(pr.p, pr.rho);
    const double rhw = pr.rho * h * W * W;
    double st[6];
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j)
            st[sym(i, j)] = rhw * pr.v[i] * pr.v[j] + pr.p * g.gUU[sym(i, j)];
    const double E = c.D + c.tau;
    double mU[3];
    lower(g.gUU, c.S, mU);
    Cons F[3];
    for (int d = 0; d < 3; ++d)
        F[d] = phys_flux(pr, c, d, g.lapse, g.shift);
    const double sS[3] = {sb.S[0], sb.S[1], sb.S[2]};

    // flux terms and their d ln sqrt(gamma) weights
    ConsBar Fb[3];
    for (int d = 0; d < 3; ++d)
    {
        Fb[d].D = -sb.D * f.dlnsqrtg[d];
        Fb[d].tau = -sb.tau * f.dlnsqrtg[d];
        for (int m = 0; m < 3; ++m)
            Fb[d].S[m] = -sS[m] * f.dlnsqrtg[d];
        fb.dlnsqrtg[d] -= sb.D * F[d].D + sb.tau * F[d].tau +
                          sS[0] * F[d].S[0] + sS[1] * F[d].S[1] +
                          sS[2] * F[d].S[2];
    }
    // tau: - mU . d lapse + lapse st:K
    double stK = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            stK += st[sym(i, j)] * f.K[sym(i, j)];
    double mUbar[3], stbar[6] = {0, 0, 0, 0, 0, 0};
    for (int d = 0; d < 3; ++d)
    {
        mUbar[d] = -sb.tau * f.dlapse[d];
        fb.dlapse[d] -= sb.tau * mU[d];
    }
    fb.g.lapse += sb.tau * stK;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
        {
            stbar[sym(i, j)] += sb.tau * g.lapse * f.K[sym(i, j)];
            fb.K[sym(i, j)] += sb.tau * g.lapse * st[sym(i, j)];
        }
    // S_m: -E d_m lapse + lapse/2 st:d_m gamma + S_j d_m shift^j
    double Ebar = 0.0;
    for (int m = 0; m < 3; ++m)
    {
        Ebar -= sS[m] * f.dlapse[m];
        fb.dlapse[m] -= sS[m] * E;
        double sg = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
            {
                sg += st[sym(i, j)] * f.dgamma[m][sym(i, j)];
                stbar[sym(i, j)] += sS[m] * 0.5 * g.lapse *
                                    f.dgamma[m][sym(i, j)];
                fb.dgamma[m][sym(i, j)] +=
                    sS[m] * 0.5 * g.lapse * st[sym(i, j)];
            }
        fb.g.lapse += sS[m] * 0.5 * sg;
        for (int sd = 0; sd < 3; ++sd)
        {
            cb.S[sd] += sS[m] * f.dshift[sd][m];
            fb.dshift[sd][m] += sS[m] * c.S[sd];
        }
    }
    cb.D += Ebar;
    cb.tau += Ebar;
    // mU = gUU S
    double t[3];
    lower(g.gUU, mUbar, t);
    for (int j = 0; j < 3; ++j)
        cb.S[j] += t[j];
    sym_outer_add(fb.g.gUU, 1.0, mUbar, c.S);
    // st_q = rhw v_i v_j + p gUU_q (q = sym(i,j), computed once per q)
    double rhwbar = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j)
        {
            const int q = sym(i, j);
            rhwbar += stbar[q] * pr.v[i] * pr.v[j];
            pb.v[i] += stbar[q] * rhw * pr.v[j];
            pb.v[j] += stbar[q] * rhw * pr.v[i];
            pb.p += stbar[q] * g.gUU[q];
            fb.g.gUU[q] += stbar[q] * pr.p;
        }
    // rhw = rho h W^2
    pb.rho += rhwbar * h * W * W;
    const double hbar = rhwbar * pr.rho * W * W;
    const double Wbar = rhwbar * pr.rho * h * 2.0 * W;
    pb.eps += hbar;
    pb.p += div_(hbar, pr.rho);
    pb.rho -= div_(hbar * pr.p, pr.rho * pr.rho);
    vsq_rev(pr.v, g.gLL, Wbar * 0.5 * W * W * W, pb.v, fb.g.gLL);
    for (int d = 0; d < 3; ++d)
        phys_flux_rev(pr, c, d, g.lapse, g.shift, Fb[d], pb, cb, fb.g.lapse,
                      fb.g.shift);
}

// ------------------------------------------------- spin contractions

GRHD_HD inline double contract(const GeoBar &b, const GeoT<Dual> &g)
{
    double s = b.lapse * g.lapse.d;
    for (int q = 0; q < 6; ++q)
        s += b.gLL[q] * g.gLL[q].d + b.gUU[q] * g.gUU[q].d;
    for (int q = 0; q < 3; ++q)
        s += b.shift[q] * g.shift[q].d;
    return s;
}

GRHD_HD inline double contract(const GeoFullBar &b, const GeoFullT<Dual> &f)
{
    double s = contract(b.g, f.g);
    for (int q = 0; q < 6; ++q)
        s += b.K[q] * f.K[q].d;
    for (int d = 0; d < 3; ++d)
    {
        s += b.dlapse[d] * f.dlapse[d].d + b.dlnsqrtg[d] * f.dlnsqrtg[d].d;
        for (int q = 0; q < 6; ++q)
            s += b.dgamma[d][q] * f.dgamma[d][q].d;
        for (int q = 0; q < 3; ++q)
            s += b.dshift[d][q] * f.dshift[d][q].d;
    }
    return s;
}

GRHD_HD inline void values_of(const GeoT<Dual> &a, Geo &g)
{
    for (int q = 0; q < 6; ++q)
    {
        g.gLL[q] = a.gLL[q].v;
        g.gUU[q] = a.gUU[q].v;
    }
    g.lapse = a.lapse.v;
    for (int q = 0; q < 3; ++q)
        g.shift[q] = a.shift[q].v;
}

GRHD_HD inline void values_of(const GeoFullT<Dual> &a, GeoFull &f)
{
    values_of(a.g, f.g);
    for (int q = 0; q < 6; ++q)
        f.K[q] = a.K[q].v;
    for (int d = 0; d < 3; ++d)
    {
        f.dlapse[d] = a.dlapse[d].v;
        f.dlnsqrtg[d] = a.dlnsqrtg[d].v;
        for (int q = 0; q < 6; ++q)
            f.dgamma[d][q] = a.dgamma[d][q].v;
        for (int q = 0; q < 3; ++q)
            f.dshift[d][q] = a.dshift[d][q].v;
    }
}

// Kerr-Schild geometry at a point with its spin derivative.
template <bool FULL>
GRHD_HD inline void ks_metric_spin(double M, double a, double x, double y,
                                   double z, GeoT<Dual> &g,
                                   GeoFullT<Dual> *f)
{
    ks_metric<Dual, FULL>(Dual(M), Dual(a, 1.0), Dual(x), Dual(y), Dual(z),
                          g, f);
}

// sqrt(det gamma) of packed gamma_ij in dual numbers (the accretion
// face weight, as mdot_face evaluates it).
GRHD_HD inline Dual sqrt_det(const Dual g[6])
{
    const Dual det = g[0] * (g[3] * g[5] - g[4] * g[4]) -
                     g[1] * (g[1] * g[5] - g[4] * g[2]) +
                     g[2] * (g[1] * g[4] - g[3] * g[2]);
    return sqrt_(det);
}

} // namespace adj
} // namespace grhd

namespace grhd {
namespace adj {

// Whether the floors or atmosphere changed the primitives
// (primitive_differs, FArrayBoxFiniteVolume.hpp:704-711).
GRHD_HD inline bool differs(const Prim &a, const Prim &b)
{
    return a.rho != b.rho || a.eps != b.eps || a.p != b.p ||
           a.v[0] != b.v[0] || a.v[1] != b.v[1] || a.v[2] != b.v[2];
}

// Reverse of the post-update recovery of one cell
// (recover_primitives_and_apply_atmosphere_from_fixed_background,
// FixedBGFArrayBoxFiniteVolume.hpp:60-110) as recorded by the forward
// sweep: branch 0 kept the updated state Y, 1 replaced it by p2c of the
// floored con2prim result (converged pressure pY), 2 by the atmosphere.
GRHD_HD inline ConsBar recovery_rev(const Options &o, const Cons &Y, int br,
                                    double pY, const Geo &g,
                                    const ConsBar &Ub, GeoBar &gb)
{
    if (br == 0)
        return Ub;
    ConsBar Yb = zero_cons_bar();
    if (br != 1)
        return Yb;
    const Prim pr = c2p_at(o, Y, g.gUU, pY);
    Prim fl = pr;
    floors(o, fl, g.gLL);
    PrimBar flb = zero_prim_bar(), prb = zero_prim_bar();
    p2c_rev(fl, g.gLL, Ub, flb, gb.gLL);
    floors_rev(o, pr, g.gLL, flb, prb, gb.gLL);
    con2prim_rev(o, Y, g.gUU, pY, prb, Yb, gb.gUU);
    return Yb;
}

// ----------------------------------------------- torus initial data
// The constant-specific-angular-momentum torus of FixedBGTorus.hpp
// (fixed_bg_torus_primitive, :333-374) with eight parameters: an amplitude
// A scaling the equilibrium density and pressure (the test-fluid
// equilibrium is invariant under it), the polytropic constant K, the spin
// a of the Kerr-Schild hole (metric and torus), and five azimuthal density
// modes rho *= 1 + sum_m eps_m cos(m phi + phase_m).  Templated so that
// the same code gives the state (double) and its derivative along one
// parameter (Dual).

template <typename T> struct TorusThetaT
{
    T A, K, a, eps[5];
    T ell, W_in; // angular momentum and surface potential of spin a
};

template <typename T>
GRHD_HD inline bool torus_potential_T(T x, T y, T ell, const GeoT<T> &g,
                                      double vmax2, T &W)
{
    const T b[3] = {-y, x, T(0.0)};
    T gpp = T(0.0), gtp = T(0.0), bb = T(0.0);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            gpp += g.gLL[sym(i, j)] * b[i] * b[j];
    for (int i = 0; i < 3; ++i)
    {
        T sL = T(0.0);
        for (int j = 0; j < 3; ++j)
            sL += g.gLL[sym(i, j)] * g.shift[j];
        gtp += sL * b[i];
        bb += sL * g.shift[i];
    }
    const T gtt = bb - g.lapse * g.lapse;
    const T den = ell * gtp + gpp;
    if (fabs(val(den)) < 1.0e-300)
        return false;
    const T om = -(ell * gtt + gtp) / den;
    T v[3];
    for (int i = 0; i < 3; ++i)
        v[i] = (om * b[i] + g.shift[i]) / g.lapse;
    const T v2 = vsq(v, g.gLL);
    if (val(v2) >= vmax2 || val(v2) >= 1.0)
        return false;
    const T norm = -gtt - T(2.0) * om * gtp - om * om * gpp;
    if (val(norm) <= 0.0)
        return false;
    const T mut = -(gtt + om * gtp) / sqrt_(norm);
    if (val(mut) <= 0.0)
        return false;
    W = log_(mut);
    return true;
}

template <typename T>
GRHD_HD inline void torus_velocity_T(T x, T y, T ell, const GeoT<T> &g,
                                     T v[3])
{
    const T b[3] = {-y, x, T(0.0)};
    T gpp = T(0.0), gtp = T(0.0), bb = T(0.0);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            gpp += g.gLL[sym(i, j)] * b[i] * b[j];
    for (int i = 0; i < 3; ++i)
    {
        T sL = T(0.0);
        for (int j = 0; j < 3; ++j)
            sL += g.gLL[sym(i, j)] * g.shift[j];
        gtp += sL * b[i];
        bb += sL * g.shift[i];
    }
    const T gtt = bb - g.lapse * g.lapse;
    const T om = -(ell * gtt + gtp) / (ell * gtp + gpp);
    for (int i = 0; i < 3; ++i)
        v[i] = (om * b[i] + g.shift[i]) / g.lapse;
}

// Primitives and conserved variables of one cell centre (x, y, z) relative
// to the hole.  r_in: the torus's inner edge (cylindrical radius below
// which the atmosphere is kept, as the reference's fill does); vmax2: the
// torus configuration's velocity cap of the potential.
template <typename T>
GRHD_HD inline ConsT<T> torus_cell_T(const Options &o, double M,
                                     const TorusThetaT<T> &th,
                                     const double phase[5], double r_in,
                                     double vmax2, double x, double y,
                                     double z, PrimT<T> &pr)
{
    GeoT<T> g;
    ks_metric<T, false>(T(M), th.a, T(x), T(y), T(z), g, nullptr);
    const double G = o.G;
    pr.rho = T(o.rho_floor);
    pr.p = T(o.p_floor);
    pr.v[0] = pr.v[1] = pr.v[2] = T(0.0);
    pr.eps = pr.p / (T(G - 1.0) * pr.rho);
    if (sqrt(x * x + y * y) >= r_in)
    {
        T W;
        if (torus_potential_T(T(x), T(y), th.ell, g, vmax2, W))
        {
            const T h = exp_(th.W_in - W);
            if (val(h) > 1.0)
            {
                const T rho_eq =
                    pow_((h - T(1.0)) * T(G - 1.0) / (T(G) * th.K),
                         1.0 / (G - 1.0));
                const T p_eq = th.K * pow_(rho_eq, G);
                const double phi = atan2(y, x);
                T pert = T(1.0);
                for (int m = 0; m < 5; ++m)
                    pert += th.eps[m] * cos((m + 1) * phi + phase[m]);
                pr.rho = th.A * rho_eq * pert;
                pr.p = th.A * p_eq;
                pr.eps = pr.p / (T(G - 1.0) * pr.rho);
                torus_velocity_T(T(x), T(y), th.ell, g, pr.v);
            }
        }
    }
    floors(o, pr, g.gLL);
    return p2c(pr, g.gLL);
}

// d W / d R at R on the x axis by the centred difference of
// fixed_bg_torus_radial_potential_derivative (FixedBGTorus.hpp:200-216);
// false when the potential is not finite there.
template <typename T>
GRHD_HD inline bool torus_dWdr_T(double M, T a, T ell, double R,
                                 double vmax2, T &out)
{
    const double dr = fmax(1.0e-3 * R, 1.0e-4);
    const double rm = fmax(R - dr, 1.0e-6);
    GeoT<T> gp, gm;
    ks_metric<T, false>(T(M), a, T(R + dr), T(0.0), T(0.0), gp, nullptr);
    ks_metric<T, false>(T(M), a, T(rm), T(0.0), T(0.0), gm, nullptr);
    T wp, wm;
    if (!torus_potential_T(T(R + dr), T(0.0), ell, gp, vmax2, wp) ||
        !torus_potential_T(T(rm), T(0.0), ell, gm, vmax2, wm))
        return false;
    out = (wp - wm) / T(R + dr - rm);
    return true;
}

// Torus constants of spin a with their spin derivatives: the angular
// momentum ell whose potential is stationary at the pressure maximum
// (fixed_bg_torus_pressure_max_specific_angular_momentum,
// FixedBGTorus.hpp:218-281: a scan of 120 values in [0.25, 4] x the
// Schwarzschild guess, then bisection to |dW/dR| < 1e-13), the surface
// potential W_in at the inner edge, and the polytropic constant K that
// gives density 1 at the pressure maximum.  d ell / d a follows from the
// implicit function theorem on dW/dR(ell, a) = 0.  False when no torus
// exists for these radii.
struct TorusSetup
{
    double ell, dell_da, W_in, dWin_da, K_unit;
};

GRHD_HD inline bool torus_setup(double M, double a, double r_in,
                                double r_max, double vmax2, double G,
                                TorusSetup &out)
{
    if (r_max <= 3.0 * M)
        return false;
    const double guess = sqrt(M * r_max) / (1.0 - 2.0 * M / r_max);
    double ell = guess;
    double prev_ell = 0.25 * guess, prev_d = 0.0;
    bool prev_ok = torus_dWdr_T<double>(M, a, prev_ell, r_max, vmax2, prev_d);
    for (int s = 1; s <= 120; ++s)
    {
        const double e = guess * (0.25 + (double)s / 120.0 * 3.75);
        double d;
        if (!torus_dWdr_T<double>(M, a, e, r_max, vmax2, d))
            continue;
        if (prev_ok && prev_d * d <= 0.0)
        {
            double lo = prev_ell, hi = e, flo = prev_d;
            ell = 0.5 * (lo + hi);
            for (int it = 0; it < 80; ++it)
            {
                const double mid = 0.5 * (lo + hi);
                double fm;
                if (!torus_dWdr_T<double>(M, a, mid, r_max, vmax2, fm))
                    break;
                ell = mid;
                if (fabs(fm) < 1.0e-13)
                    break;
                if (flo * fm <= 0.0)
                    hi = mid;
                else
                {
                    lo = mid;
                    flo = fm;
                }
                ell = 0.5 * (lo + hi);
            }
            break;
        }
        prev_ell = e;
        prev_d = d;
        prev_ok = true;
    }
    Dual ge, ga;
    if (!torus_dWdr_T<Dual>(M, Dual(a), Dual(ell, 1.0), r_max, vmax2, ge) ||
        !torus_dWdr_T<Dual>(M, Dual(a, 1.0), Dual(ell), r_max, vmax2, ga))
        return false;
    out.ell = ell;
    out.dell_da = -ga.d / ge.d;
    GeoT<Dual> g;
    ks_metric<Dual, false>(Dual(M), Dual(a, 1.0), Dual(r_in), Dual(0.0),
                           Dual(0.0), g, nullptr);
    Dual W;
    if (!torus_potential_T<Dual>(Dual(r_in), Dual(0.0),
                                 Dual(ell, out.dell_da), g, vmax2, W))
        return false;
    out.W_in = W.v;
    out.dWin_da = W.d;
    Geo gc;
    ks_metric<double, false>(M, a, r_max, 0.0, 0.0, gc, nullptr);
    double Wc;
    if (!torus_potential_T<double>(r_max, 0.0, ell, gc, vmax2, Wc))
        return false;
    const double hc = exp(out.W_in - Wc);
    if (!(hc > 1.0))
        return false;
    out.K_unit = (hc - 1.0) * (G - 1.0) / G;
    return true;
}

} // namespace adj
} // namespace grhd
