// grhd_adjoint_items.cuh -- per-cell and per-face work items of the
// discrete adjoint (grhd_adjoint.cu launches them as kernels; the host
// check of the adjoint runs the same items in host loops).
#pragma once

#include "grhd_adjoint.cuh"
#include "grhd_kernels.cuh"

namespace grhd {
namespace adj {

// RK4 stage weights of the accretion integral (dt/6) (1, 2, 2, 1)
__host__ __device__ inline double stage_weight(int s)
{
    return (s == 1 || s == 2) ? 2.0 : 1.0;
}

struct AdjRhs
{
    BoxDev b;   // cs = pcs = ghosted volume, rcs = interior volume
    Options o;
    double M, a;
    double inv_dx[3];
    const double *U;      // RHS input state (11 comps)
    const double *P;      // primitive cache (rho, p, v) of that state
    const unsigned *bits; // limiter branches, 10 bits per direction
    const double *lamk;   // adjoint of the RHS (5 comps, interior)
    double mu;            // weight of this RHS's Mdot in J
    double *fb;           // face-state adjoints [3][10][gvol]
    double *gbuf;         // ghost adjoints [5][gvol]
};

struct AdjStage
{
    int stage;       // 0..3: RK4 stage of the RHS; -1: RHS only
    double dt;
    const double *Y; // pre-recovery state of U_stage (5 comps, interior)
    const double *pY;
    const unsigned char *br;
    const double *A; // recovery adjoint of the step's last stage
    double *acc;     // adjoint of U^n accumulated over the stages
    double *lamk;    // out: adjoint of the previous stage's RHS
    double *out;     // stage 0 / RHS only: adjoint of the RHS input
};

__host__ __device__ inline void cell_of(const BoxDev &b, int64_t g, int c[3])
{
    c[0] = b.glo[0] + (int)(g % b.gn[0]);
    const int64_t r = g / b.gn[0];
    c[1] = b.glo[1] + (int)(r % b.gn[1]);
    c[2] = b.glo[2] + (int)(r / b.gn[1]);
}

__host__ __device__ inline int64_t stride_of(const BoxDev &b, int d)
{
    return d == 0 ? 1 : (d == 1 ? (int64_t)b.gn[0]
                                : (int64_t)b.gn[0] * b.gn[1]);
}


__host__ __device__ inline void load5(const double *P, int64_t pcs, int64_t g,
                                      double q[5])
{
    for (int c = 0; c < 5; ++c)
        q[c] = P[c * pcs + g];
}

__host__ __device__ inline ConsBar lamk_at(const AdjRhs &A, int64_t ri)
{
    ConsBar k;
    k.D = A.lamk[0 * A.b.rcs + ri];
    k.S[0] = A.lamk[1 * A.b.rcs + ri];
    k.S[1] = A.lamk[2 * A.b.rcs + ri];
    k.S[2] = A.lamk[3 * A.b.rcs + ri];
    k.tau = A.lamk[4 * A.b.rcs + ri];
    return k;
}

__host__ __device__ inline Cons load_cons5(const double *s, int64_t cs,
                                           int64_t g)
{
    Cons c;
    c.D = s[kD * cs + g];
    c.S[0] = s[(kS1 + 0) * cs + g];
    c.S[1] = s[(kS1 + 1) * cs + g];
    c.S[2] = s[(kS1 + 2) * cs + g];
    c.tau = s[kTau * cs + g];
    return c;
}

__host__ __device__ inline double radius_of(const Options &o, const int c[3])
{
    double x, y, z;
    cell_xyz(o, c[0], c[1], c[2], x, y, z);
    return sqrt(x * x + y * y + z * z);
}

// ------------------------------------------------------ forward taping

// Limiter branches of ghosted cell g in each direction (0 where a
// neighbour is outside the ghosted box: those slopes are never used).
__host__ __device__ inline void bits_item(const BoxDev &b, const Options &o,
                                          const double *P, unsigned *bits,
                                          int64_t g)
{
    int c[3];
    cell_of(b, g, c);
    unsigned out = 0;
    double q[5];
    load5(P, b.pcs, g, q);
    for (int d = 0; d < 3; ++d)
    {
        if (c[d] <= b.glo[d] || c[d] >= b.ghi[d])
            continue;
        const int64_t sd = stride_of(b, d);
        double l[5], r[5];
        load5(P, b.pcs, g - sd, l);
        load5(P, b.pcs, g + sd, r);
        out |= slope_bits(l, q, r, o.theta) << (10 * d);
    }
    bits[g] = out;
}

// One RK4 stage combination + post-update recovery of interior cell t,
// recording Y, the con2prim pressure and the recovery branch.  The stage
// arithmetic is that of the operator's fused stage (k_stage mode 0).
__host__ __device__ inline void stage_tape_item(
    const BoxDev &b, const Options &o, double M, double a, const double *un,
    const double *kv, double *acc, int stage, double dt, double *out,
    double *Y, double *pY, unsigned char *br, int64_t t)
{
    const int i = b.lo[0] + (int)(t % b.in[0]);
    const int64_t r = t / b.in[0];
    const int j = b.lo[1] + (int)(r % b.in[1]);
    const int k = b.lo[2] + (int)(r / b.in[1]);
    const int64_t g = b.gidx(i, j, k);
    const int comp_of[5] = {kD, kS1, kS1 + 1, kS1 + 2, kTau};
    if (excised(o, i, j, k))
    {
        if (out != un)
            for (int c = 0; c < kStateComps; ++c)
                out[c * b.cs + g] = un[c * b.cs + g];
        for (int c = 0; c < 5; ++c)
            Y[c * b.rcs + t] = un[comp_of[c] * b.cs + g];
        pY[t] = 0.0;
        br[t] = 0;
        return;
    }
    const double cst = (stage == 2) ? dt : 0.5 * dt;
    const double dt6 = dt / 6.0;
    double u[5];
    for (int c = 0; c < 5; ++c)
    {
        const double kk = kv[c * b.rcs + t];
        const double u0 = un[comp_of[c] * b.cs + g];
        double av = (stage == 0) ? kk : acc[c * b.rcs + t];
        if (stage == 1 || stage == 2)
            av = av + 2.0 * kk;
        if (stage < 3)
        {
            acc[c * b.rcs + t] = av;
            u[c] = u0 + cst * kk;
        }
        else
            u[c] = u0 + dt6 * (av + kk);
        Y[c * b.rcs + t] = u[c];
    }
    Cons c;
    c.D = u[0];
    c.S[0] = u[1];
    c.S[1] = u[2];
    c.S[2] = u[3];
    c.tau = u[4];
    double x, y, z;
    cell_xyz(o, i, j, k, x, y, z);
    Geo geo;
    ks_metric<double, false>(M, a, x, y, z, geo, nullptr);
    Prim pr, stored;
    const bool ok = con2prim(o, c, geo.gUU, pr, nullptr, nullptr);
    unsigned char branch;
    if (ok)
    {
        stored = pr;
        floors(o, stored, geo.gLL);
        branch = differs(pr, stored) ? 1 : 0;
        pY[t] = pr.p;
    }
    else
    {
        stored = atmosphere(o);
        branch = 2;
        pY[t] = 0.0;
    }
    br[t] = branch;
    if (branch)
        c = p2c(stored, geo.gLL);
    out[kRho * b.cs + g] = stored.rho;
    out[kEps * b.cs + g] = stored.eps;
    out[kPress * b.cs + g] = stored.p;
    for (int q = 0; q < 3; ++q)
        out[(kV1 + q) * b.cs + g] = stored.v[q];
    out[kD * b.cs + g] = c.D;
    out[(kS1 + 0) * b.cs + g] = c.S[0];
    out[(kS1 + 1) * b.cs + g] = c.S[1];
    out[(kS1 + 2) * b.cs + g] = c.S[2];
    out[kTau * b.cs + g] = c.tau;
}

// -------------------------------------------------------- reverse items

// Face between L (index t in the direction-d face enumeration) and
// R = L + e_d: writes the adjoints of its two reconstructed states into
// fb[d] at L's ghosted index; returns the face's spin adjoint.
__host__ __device__ inline double face_rev_item(const AdjRhs &A, int d,
                                                int64_t t)
{
    const BoxDev &b = A.b;
    const Options &o = A.o;
    int n[3] = {b.in[0], b.in[1], b.in[2]};
    n[d] += 1;
    int L[3];
    L[0] = b.lo[0] + (int)(t % n[0]);
    const int64_t r = t / n[0];
    L[1] = b.lo[1] + (int)(r % n[1]);
    L[2] = b.lo[2] + (int)(r / n[1]);
    L[d] -= 1;
    int R[3] = {L[0], L[1], L[2]};
    R[d] += 1;
    const int64_t gL = b.gidx(L[0], L[1], L[2]);
    const int64_t sd = stride_of(b, d);
    const int64_t gv = b.gvol();
    double *qlb_out = A.fb + (int64_t)(d * 10) * gv + gL;

    const bool inL = L[d] >= b.lo[d] && !excised(o, L[0], L[1], L[2]);
    const bool inR = R[d] <= b.hi[d] && !excised(o, R[0], R[1], R[2]);
    ConsBar Fb = zero_cons_bar();
    if (inR)
    {
        const ConsBar k = lamk_at(A, b.iidx(R[0], R[1], R[2]));
        Fb.D += k.D;
        Fb.tau += k.tau;
        for (int q = 0; q < 3; ++q)
            Fb.S[q] += k.S[q];
    }
    if (inL)
    {
        const ConsBar k = lamk_at(A, b.iidx(L[0], L[1], L[2]));
        Fb.D -= k.D;
        Fb.tau -= k.tau;
        for (int q = 0; q < 3; ++q)
            Fb.S[q] -= k.S[q];
    }
    const double idx = A.inv_dx[d];
    Fb.D *= idx;
    Fb.tau *= idx;
    for (int q = 0; q < 3; ++q)
        Fb.S[q] *= idx;
    // accretion sphere face (mdot_face): +/- sqrt(det gamma_face) F_D dx^2;
    // faces between two interior cells (the sphere lies inside the domain)
    double wacc = 0.0;
    if (A.mu != 0.0 && o.accretion_radius > 0.0 && L[d] >= b.lo[d] &&
        R[d] <= b.hi[d])
    {
        const bool il = radius_of(o, L) < o.accretion_radius;
        const bool ir = radius_of(o, R) < o.accretion_radius;
        if (il != ir)
            wacc = (il ? -1.0 : 1.0) * o.dx * o.dx * A.mu;
    }
    if (wacc == 0.0 && Fb.D == 0.0 && Fb.tau == 0.0 && Fb.S[0] == 0.0 &&
        Fb.S[1] == 0.0 && Fb.S[2] == 0.0)
    {
        for (int c = 0; c < 10; ++c)
            qlb_out[(int64_t)c * gv] = 0.0;
        return 0.0;
    }
    double xl, yl, zl, xr, yr, zr;
    cell_xyz(o, L[0], L[1], L[2], xl, yl, zl);
    cell_xyz(o, R[0], R[1], R[2], xr, yr, zr);
    GeoT<Dual> gl, gr, gf;
    ks_metric_spin<false>(A.M, A.a, xl, yl, zl, gl, nullptr);
    ks_metric_spin<false>(A.M, A.a, xr, yr, zr, gr, nullptr);
    average_geo(gl, gr, gf);
    Geo g;
    values_of(gf, g);
    Dual sdet(0.0);
    if (wacc != 0.0)
    {
        sdet = sqrt_det(gf.gLL);
        Fb.D += wacc * sdet.v;
    }
    double LL[5], Lq[5], Rq[5], RR[5];
    load5(A.P, b.pcs, gL - sd, LL);
    load5(A.P, b.pcs, gL, Lq);
    load5(A.P, b.pcs, gL + sd, Rq);
    load5(A.P, b.pcs, gL + 2 * sd, RR);
    const unsigned bL = (A.bits[gL] >> (10 * d)) & 0x3ffu;
    const unsigned bR = (A.bits[gL + sd] >> (10 * d)) & 0x3ffu;
    double qlb[5], qrb[5];
    GeoBar gb;
    zero(gb);
    const double FD =
        face_flux_rev(o, LL, Lq, Rq, RR, bL, bR, g, d, Fb, qlb, qrb, gb);
    for (int c = 0; c < 5; ++c)
    {
        qlb_out[(int64_t)c * gv] = qlb[c];
        qlb_out[(int64_t)(5 + c) * gv] = qrb[c];
    }
    double spin = contract(gb, gf);
    if (wacc != 0.0)
        spin += wacc * FD * sdet.d;
    return spin;
}

// Adjoint of the primitive cache of cell c gathered from the faces of
// direction d through the replayed limiter slopes.  The faces of direction
// d have their L cell in [lo_d - 1, hi_d] and the other coordinates
// interior; the caller checks the latter.
__host__ __device__ inline void gather_dir(const AdjRhs &A, int d,
                                           const int c[3], int64_t g,
                                           double lp[5])
{
    const BoxDev &b = A.b;
    const int64_t gv = b.gvol();
    const int64_t sd = stride_of(b, d);
    const double *F = A.fb + (int64_t)(d * 10) * gv;
    const int lo = b.lo[d] - 1, hi = b.hi[d];
    // face with L at offset m from c exists?
    bool ex[4];
    for (int m = -2; m <= 1; ++m)
        ex[m + 2] = (c[d] + m >= lo && c[d] + m <= hi);
    auto qlb = [&](int m, int comp) {
        return ex[m + 2] ? F[(int64_t)comp * gv + g + m * sd] : 0.0;
    };
    auto qrb = [&](int m, int comp) {
        return ex[m + 2] ? F[(int64_t)(5 + comp) * gv + g + m * sd] : 0.0;
    };
    unsigned bm = 0, b0 = 0, bp = 0;
    if (A.o.use_recon)
    {
        if (c[d] - 1 >= b.glo[d])
            bm = (A.bits[g - sd] >> (10 * d)) & 0x3ffu;
        b0 = (A.bits[g] >> (10 * d)) & 0x3ffu;
        if (c[d] + 1 <= b.ghi[d])
            bp = (A.bits[g + sd] >> (10 * d)) & 0x3ffu;
    }
    for (int q = 0; q < 5; ++q)
    {
        // direct: c is R of face (c-1) and L of face (c)
        double v = qrb(-1, q) + qlb(0, q);
        if (A.o.use_recon)
        {
            // slope adjoints of cells c-1, c, c+1
            const double sm = 0.5 * qlb(-1, q) - 0.5 * qrb(-2, q);
            const double s0 = 0.5 * qlb(0, q) - 0.5 * qrb(-1, q);
            const double sp = 0.5 * qlb(1, q) - 0.5 * qrb(0, q);
            double wl, wc, wr;
            slope_weights(bits_of(bm, q), A.o.theta, wl, wc, wr);
            v += sm * wr; // c is the right neighbour of c-1
            slope_weights(bits_of(b0, q), A.o.theta, wl, wc, wr);
            v += s0 * wc;
            slope_weights(bits_of(bp, q), A.o.theta, wl, wc, wr);
            v += sp * wl; // c is the left neighbour of c+1
        }
        lp[q] += v;
    }
}

// Physical ghost cell g (outside the interior in exactly one direction):
// the adjoint of its primitive cache, taken back through its floors to the
// con2prim output of its source cell; stored in gbuf.  Returns its spin
// adjoint (the floors' velocity cap uses the ghost's metric).
__host__ __device__ inline double shell_rev_item(const AdjRhs &A, int64_t g)
{
    const BoxDev &b = A.b;
    const int64_t gv = b.gvol();
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
        return 0.0;
    if (out != 1)
    {
        for (int q = 0; q < 5; ++q)
            A.gbuf[q * gv + g] = 0.0;
        return 0.0;
    }
    double lp[5] = {0, 0, 0, 0, 0};
    gather_dir(A, d0, c, g, lp);
    int s[3] = {c[0], c[1], c[2]};
    s[d0] = c[d0] < b.lo[d0] ? b.lo[d0] : b.hi[d0];
    double sq[5];
    load5(A.P, b.pcs, b.gidx(s[0], s[1], s[2]), sq);
    Prim in;
    in.rho = sq[0];
    in.p = sq[1];
    in.eps = 0.0;
    for (int i = 0; i < 3; ++i)
        in.v[i] = sq[2 + i];
    double x, y, z;
    cell_xyz(A.o, c[0], c[1], c[2], x, y, z);
    GeoT<Dual> gd;
    ks_metric_spin<false>(A.M, A.a, x, y, z, gd, nullptr);
    Geo geo;
    values_of(gd, geo);
    PrimBar ob = zero_prim_bar(), ib = zero_prim_bar();
    ob.rho = lp[0];
    ob.p = lp[1];
    for (int i = 0; i < 3; ++i)
        ob.v[i] = lp[2 + i];
    double Gb[6] = {0, 0, 0, 0, 0, 0};
    floors_rev(A.o, in, geo.gLL, ob, ib, Gb);
    A.gbuf[0 * gv + g] = ib.rho;
    A.gbuf[1 * gv + g] = ib.p;
    for (int i = 0; i < 3; ++i)
        A.gbuf[(2 + i) * gv + g] = ib.v[i];
    double spin = 0.0;
    for (int q = 0; q < 6; ++q)
        spin += Gb[q] * gd.gLL[q].d;
    return spin;
}

// Interior cell t: the adjoint of the RHS input state at this cell, then
// the reverse of the stage combination and recovery (see AdjStage).
__host__ __device__ inline double cell_rev_item(const AdjRhs &A,
                                                const AdjStage &S, int64_t t)
{
    const BoxDev &b = A.b;
    const Options &o = A.o;
    const int64_t gv = b.gvol();
    int c[3];
    c[0] = b.lo[0] + (int)(t % b.in[0]);
    const int64_t r = t / b.in[0];
    c[1] = b.lo[1] + (int)(r % b.in[1]);
    c[2] = b.lo[2] + (int)(r / b.in[1]);
    const int64_t g = b.gidx(c[0], c[1], c[2]);
    const int64_t rcs = b.rcs;
    ConsBar Ub = zero_cons_bar();
    double spin = 0.0;
    const bool exc = excised(o, c[0], c[1], c[2]);
    GeoFullT<Dual> fd;
    GeoFullBar fbar;
    zero(fbar);
    if (!exc)
    {
        double lp[5] = {0, 0, 0, 0, 0};
        for (int d = 0; d < 3; ++d)
            gather_dir(A, d, c, g, lp);
        // ghosts this cell fed (physical boundary)
        for (int d = 0; d < 3; ++d)
        {
            const int64_t sd = stride_of(b, d);
            if (c[d] == b.lo[d] && b.lo[d] == b.dlo[d])
                for (int m = 1; m <= 2; ++m)
                    for (int q = 0; q < 5; ++q)
                        lp[q] += A.gbuf[q * gv + g - m * sd];
            if (c[d] == b.hi[d] && b.hi[d] == b.dhi[d])
                for (int m = 1; m <= 2; ++m)
                    for (int q = 0; q < 5; ++q)
                        lp[q] += A.gbuf[q * gv + g + m * sd];
        }
        PrimBar cb = zero_prim_bar();
        cb.rho = lp[0];
        cb.p = lp[1];
        for (int i = 0; i < 3; ++i)
            cb.v[i] = lp[2 + i];
        double x, y, z;
        cell_xyz(o, c[0], c[1], c[2], x, y, z);
        ks_metric_spin<true>(A.M, A.a, x, y, z, fd.g, &fd);
        GeoFull f;
        values_of(fd, f);
        const Cons U = load_cons5(A.U, b.cs, g);
        double q5[5];
        load5(A.P, b.pcs, g, q5);
        Prim pr;
        pr.rho = q5[0];
        pr.p = q5[1];
        pr.eps = pr.p / ((o.G - 1.0) * pr.rho);
        for (int i = 0; i < 3; ++i)
            pr.v[i] = q5[2 + i];
        if (o.use_src)
        {
            Prim fl = pr;
            floors(o, fl, f.g.gLL);
            if (!is_atmo(o, fl, o.src_atmo_factor))
            {
                const ConsBar sb = lamk_at(A, t);
                PrimBar flb = zero_prim_bar();
                static_sources_rev(fl, U, f, sb, flb, Ub, fbar);
                floors_rev(o, pr, f.g.gLL, flb, cb, fbar.g.gLL);
            }
        }
        con2prim_rev(o, U, f.g.gUU, pr.p, cb, Ub, fbar.g.gUU);
    }
    // stage combination and recovery
    if (S.stage >= 1)
    {
        ConsBar B = zero_cons_bar();
        if (!exc)
        {
            Cons Y;
            Y.D = S.Y[0 * rcs + t];
            Y.S[0] = S.Y[1 * rcs + t];
            Y.S[1] = S.Y[2 * rcs + t];
            Y.S[2] = S.Y[3 * rcs + t];
            Y.tau = S.Y[4 * rcs + t];
            Geo g2;
            values_of(fd.g, g2);
            B = recovery_rev(o, Y, S.br[t], S.pY[t], g2, Ub, fbar.g);
        }
        const double Bv[5] = {B.D, B.S[0], B.S[1], B.S[2], B.tau};
        // lambda_k of the previous stage: cA A + cB B
        const double dt = S.dt;
        const double cA = (S.stage == 1) ? dt / 6.0 : dt / 3.0;
        const double cB = (S.stage == 3) ? dt : 0.5 * dt;
        for (int q = 0; q < 5; ++q)
        {
            S.acc[q * rcs + t] += Bv[q];
            S.lamk[q * rcs + t] = cA * S.A[q * rcs + t] + cB * Bv[q];
        }
    }
    else
    {
        const double Uv[5] = {Ub.D, Ub.S[0], Ub.S[1], Ub.S[2], Ub.tau};
        for (int q = 0; q < 5; ++q)
            S.out[q * rcs + t] =
                (S.stage == 0 ? S.acc[q * rcs + t] : 0.0) + Uv[q];
    }
    if (!exc)
        spin += contract(fbar, fd);
    return spin;
}

// Reverse of the step's last recovery (U^{n+1} = R(Y4)): A = acc = its
// adjoint, lambda_k4 = dt/6 A.  Excised cells pass lambda through.
__host__ __device__ inline double proj_rev_item(
    const BoxDev &b, const Options &o, double M, double a, double dt,
    const double *lam, const double *Y, const double *pY,
    const unsigned char *br, double *A, double *acc, double *lamk, int64_t t)
{
    const int64_t rcs = b.rcs;
    const int i = b.lo[0] + (int)(t % b.in[0]);
    const int64_t r = t / b.in[0];
    const int j = b.lo[1] + (int)(r % b.in[1]);
    const int k = b.lo[2] + (int)(r / b.in[1]);
    ConsBar Ub;
    Ub.D = lam[0 * rcs + t];
    Ub.S[0] = lam[1 * rcs + t];
    Ub.S[1] = lam[2 * rcs + t];
    Ub.S[2] = lam[3 * rcs + t];
    Ub.tau = lam[4 * rcs + t];
    if (excised(o, i, j, k))
    {
        const double Uv[5] = {Ub.D, Ub.S[0], Ub.S[1], Ub.S[2], Ub.tau};
        for (int q = 0; q < 5; ++q)
        {
            A[q * rcs + t] = 0.0;
            acc[q * rcs + t] = Uv[q];
            lamk[q * rcs + t] = 0.0;
        }
        return 0.0;
    }
    Cons Yc;
    Yc.D = Y[0 * rcs + t];
    Yc.S[0] = Y[1 * rcs + t];
    Yc.S[1] = Y[2 * rcs + t];
    Yc.S[2] = Y[3 * rcs + t];
    Yc.tau = Y[4 * rcs + t];
    double x, y, z;
    cell_xyz(o, i, j, k, x, y, z);
    GeoT<Dual> gd;
    ks_metric_spin<false>(M, a, x, y, z, gd, nullptr);
    Geo g;
    values_of(gd, g);
    GeoBar gb;
    zero(gb);
    const ConsBar B = recovery_rev(o, Yc, br[t], pY[t], g, Ub, gb);
    const double Bv[5] = {B.D, B.S[0], B.S[1], B.S[2], B.tau};
    for (int q = 0; q < 5; ++q)
    {
        A[q * rcs + t] = Bv[q];
        acc[q * rcs + t] = Bv[q];
        lamk[q * rcs + t] = dt / 6.0 * Bv[q];
    }
    return contract(gb, gd);
}

// Initial data of interior or ghost cell g and, with tangents, the
// contraction of dU0/dtheta_k with lambda0 (interior cells only).
struct TorusArgs
{
    BoxDev b;
    Options o;
    double M;
    TorusThetaT<double> th;
    TorusThetaT<Dual> thd[8]; // one seed per parameter
    double phase[5];
    double r_in, vmax2;
};

__host__ __device__ inline void torus_fill_item(const TorusArgs &T,
                                                double *state, int64_t g)
{
    const BoxDev &b = T.b;
    int c[3];
    cell_of(b, g, c);
    double x, y, z;
    cell_xyz(T.o, c[0], c[1], c[2], x, y, z);
    PrimT<double> pr;
    const Cons u = torus_cell_T<double>(T.o, T.M, T.th, T.phase, T.r_in,
                                        T.vmax2, x, y, z, pr);
    state[kD * b.cs + g] = u.D;
    state[(kS1 + 0) * b.cs + g] = u.S[0];
    state[(kS1 + 1) * b.cs + g] = u.S[1];
    state[(kS1 + 2) * b.cs + g] = u.S[2];
    state[kTau * b.cs + g] = u.tau;
    state[kRho * b.cs + g] = pr.rho;
    state[kEps * b.cs + g] = pr.eps;
    state[kPress * b.cs + g] = pr.p;
    for (int q = 0; q < 3; ++q)
        state[(kV1 + q) * b.cs + g] = pr.v[q];
}

__host__ __device__ inline void torus_tangent_item(const TorusArgs &T,
                                                   const double *lam,
                                                   double *tangent,
                                                   int64_t tcs, int64_t t,
                                                   double acc[8])
{
    const BoxDev &b = T.b;
    const int i = b.lo[0] + (int)(t % b.in[0]);
    const int64_t r = t / b.in[0];
    const int j = b.lo[1] + (int)(r % b.in[1]);
    const int k = b.lo[2] + (int)(r / b.in[1]);
    double x, y, z;
    cell_xyz(T.o, i, j, k, x, y, z);
    for (int p = 0; p < 8; ++p)
    {
        PrimT<Dual> pr;
        const ConsT<Dual> u = torus_cell_T<Dual>(T.o, T.M, T.thd[p], T.phase,
                                                 T.r_in, T.vmax2, x, y, z, pr);
        const double dv[5] = {u.D.d, u.S[0].d, u.S[1].d, u.S[2].d, u.tau.d};
        if (tangent)
            for (int q = 0; q < 5; ++q)
                tangent[((int64_t)p * 5 + q) * tcs + t] = dv[q];
        if (lam)
        {
            double s = 0.0;
            for (int q = 0; q < 5; ++q)
                s += lam[q * b.rcs + t] * dv[q];
            acc[p] += s;
        }
    }
}

} // namespace adj
} // namespace grhd
