// adjoint_host_check.cu -- host-side check of the reverse-mode pointwise
// functions (grhd_adjoint.cuh) against central finite differences of the
// forward functions they reverse (grhd_device.cuh), at random states on a
// Kerr-Schild a = 0.7 background.  Built and run by
// tests/test_adjoint_host.py with nvcc as a host program (no GPU needed).
// Prints one line per check and exits non-zero on a failure.
#include "grhd_adjoint.cuh"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

using namespace grhd;
using namespace grhd::adj;

static int g_fail = 0;
static std::mt19937_64 rng(20261203);

static double U(double a, double b)
{
    return std::uniform_real_distribution<double>(a, b)(rng);
}

static void report(const char *what, double got, double want, double scale,
                   double tol = 2e-6)
{
    const double err = fabs(got - want) / (scale > 0 ? scale : 1.0);
    const bool ok = err <= tol;
    if (!ok)
        ++g_fail;
    if (!ok || getenv("VERBOSE"))
        printf("%-4s %-40s adj % .10e fd % .10e rel %.2e\n", ok ? "ok" : "FAIL",
               what, got, want, err);
}

static Options opts()
{
    Options o{};
    o.G = 5.0 / 3.0;
    o.rho_floor = 1e-10;
    o.p_floor = 1e-12;
    o.atmo_vmax2 = 0.8;
    o.src_atmo_factor = 1.0;
    o.rec_maxit = 80;
    o.rec_tol = 1e-12;
    o.rec_pfloor = 1e-12;
    o.rec_vmax2 = 0.9;
    o.theta = 2.0;
    o.use_recon = 1;
    o.use_src = 1;
    o.use_vol = 0;
    o.excision_radius = 0.0;
    o.accretion_radius = 0.0;
    o.dx = 0.5;
    o.center[0] = o.center[1] = o.center[2] = 0.0;
    return o;
}

static const double kSpin = 0.7;

static Geo geo_at(double x, double y, double z, double a = kSpin)
{
    Geo g;
    ks_metric<double, false>(1.0, a, x, y, z, g, nullptr);
    return g;
}

static Prim rand_prim(double vscale)
{
    Prim p;
    p.rho = U(0.2, 1.0);
    p.p = U(0.02, 0.3);
    for (int i = 0; i < 3; ++i)
        p.v[i] = U(-vscale, vscale);
    p.eps = p.p / ((5.0 / 3.0 - 1.0) * p.rho);
    return p;
}

static double dotc(const ConsBar &b, const Cons &c)
{
    return b.D * c.D + b.tau * c.tau + b.S[0] * c.S[0] + b.S[1] * c.S[1] +
           b.S[2] * c.S[2];
}

static ConsBar rand_cbar()
{
    ConsBar b;
    b.D = U(-1, 1);
    b.tau = U(-1, 1);
    for (int i = 0; i < 3; ++i)
        b.S[i] = U(-1, 1);
    return b;
}

static double pval(const Prim &p, int k)
{
    switch (k)
    {
    case 0: return p.rho;
    case 1: return p.eps;
    case 2: return p.p;
    default: return p.v[k - 3];
    }
}
static double *pfield(Prim &p, int k)
{
    switch (k)
    {
    case 0: return &p.rho;
    case 1: return &p.eps;
    case 2: return &p.p;
    default: return &p.v[k - 3];
    }
}
static double pbfield(const PrimBar &p, int k)
{
    switch (k)
    {
    case 0: return p.rho;
    case 1: return p.eps;
    case 2: return p.p;
    default: return p.v[k - 3];
    }
}

// ------------------------------------------------------------------ p2c
static void check_p2c()
{
    for (int t = 0; t < 20; ++t)
    {
        const Geo g = geo_at(U(-8, 8), U(-8, 8), U(-8, 8));
        Prim p = rand_prim(0.3);
        const ConsBar cb = rand_cbar();
        PrimBar pb = zero_prim_bar();
        double Gb[6] = {0, 0, 0, 0, 0, 0};
        p2c_rev(p, g.gLL, cb, pb, Gb);
        for (int k = 0; k < 6; ++k)
        {
            Prim a = p, b = p;
            const double h = 1e-6 * fmax(1e-3, fabs(pval(p, k)));
            *pfield(a, k) += h;
            *pfield(b, k) -= h;
            const double fd = (dotc(cb, p2c(a, g.gLL)) -
                               dotc(cb, p2c(b, g.gLL))) / (2 * h);
            report("p2c d/dprim", pbfield(pb, k), fd, 1.0 + fabs(fd));
        }
        for (int q = 0; q < 6; ++q)
        {
            double ga[6], gb[6];
            for (int r = 0; r < 6; ++r)
                ga[r] = gb[r] = g.gLL[r];
            const double h = 1e-6;
            ga[q] += h;
            gb[q] -= h;
            const double fd =
                (dotc(cb, p2c(p, ga)) - dotc(cb, p2c(p, gb))) / (2 * h);
            report("p2c d/dgLL", Gb[q], fd, 1.0 + fabs(fd));
        }
    }
}

// --------------------------------------------------------------- floors
static void check_floors()
{
    const Options o = opts();
    for (int t = 0; t < 40; ++t)
    {
        const Geo g = geo_at(U(-8, 8), U(-8, 8), U(-8, 8));
        Prim p = rand_prim(t % 2 ? 1.2 : 0.3); // half capped
        if (t % 4 == 3)
            p.rho = 1e-11; // floored density
        PrimBar ob = zero_prim_bar();
        ob.rho = U(-1, 1);
        ob.eps = U(-1, 1);
        ob.p = U(-1, 1);
        for (int i = 0; i < 3; ++i)
            ob.v[i] = U(-1, 1);
        if (t % 4 == 3)
            ob.eps = 0.0; // eps ~ 1e9 at the floor would swamp the differences
        auto J = [&](Prim q, const double *G) {
            floors(o, q, G);
            return ob.rho * q.rho + ob.eps * q.eps + ob.p * q.p +
                   ob.v[0] * q.v[0] + ob.v[1] * q.v[1] + ob.v[2] * q.v[2];
        };
        PrimBar ib = zero_prim_bar();
        double Gb[6] = {0, 0, 0, 0, 0, 0};
        floors_rev(o, p, g.gLL, ob, ib, Gb);
        const int ks[5] = {0, 2, 3, 4, 5};
        for (int kk = 0; kk < 5; ++kk)
        {
            const int k = ks[kk];
            Prim a = p, b = p;
            const double h = 1e-7 * fmax(1e-9, fabs(pval(p, k)));
            *pfield(a, k) += h;
            *pfield(b, k) -= h;
            const double fd = (J(a, g.gLL) - J(b, g.gLL)) / (2 * h);
            report("floors d/dprim", pbfield(ib, k), fd, 1.0 + fabs(fd), 1e-5);
        }
        for (int q = 0; q < 6; ++q)
        {
            double ga[6], gb[6];
            for (int r = 0; r < 6; ++r)
                ga[r] = gb[r] = g.gLL[r];
            const double h = 1e-7;
            ga[q] += h;
            gb[q] -= h;
            const double fd = (J(p, ga) - J(p, gb)) / (2 * h);
            report("floors d/dgLL", Gb[q], fd, 1.0 + fabs(fd));
        }
    }
}

// --------------------------------------------------------- char speeds
static void check_speeds()
{
    const Options o = opts();
    for (int t = 0; t < 20; ++t)
    {
        const Geo g = geo_at(U(-8, 8), U(-8, 8), U(-8, 8));
        Prim p = rand_prim(0.3);
        const int d = t % 3;
        const double wl = U(-1, 1), wh = U(-1, 1);
        auto J = [&](const Prim &q, const Geo &gg) {
            double lo, hi;
            char_speeds(o, q, gg, d, lo, hi);
            return wl * lo + wh * hi;
        };
        PrimBar pb = zero_prim_bar();
        GeoBar gb;
        zero(gb);
        char_speeds_rev(o, p, g, d, wl, wh, pb, gb);
        for (int k = 0; k < 6; ++k)
        {
            Prim a = p, b = p;
            const double h = 1e-6 * fmax(1e-3, fabs(pval(p, k)));
            *pfield(a, k) += h;
            *pfield(b, k) -= h;
            const double fd = (J(a, g) - J(b, g)) / (2 * h);
            report("speeds d/dprim", pbfield(pb, k), fd, 1.0 + fabs(fd));
        }
        for (int q = 0; q < 16; ++q)
        {
            Geo ga = g, gm = g;
            double *fa, *fm;
            double bar;
            if (q < 6)
            {
                fa = &ga.gLL[q];
                fm = &gm.gLL[q];
                bar = gb.gLL[q];
            }
            else if (q < 12)
            {
                fa = &ga.gUU[q - 6];
                fm = &gm.gUU[q - 6];
                bar = gb.gUU[q - 6];
            }
            else if (q == 12)
            {
                fa = &ga.lapse;
                fm = &gm.lapse;
                bar = gb.lapse;
            }
            else
            {
                fa = &ga.shift[q - 13];
                fm = &gm.shift[q - 13];
                bar = gb.shift[q - 13];
            }
            const double h = 1e-7;
            *fa += h;
            *fm -= h;
            const double fd = (J(p, ga) - J(p, gm)) / (2 * h);
            report("speeds d/dgeo", bar, fd, 1.0 + fabs(fd));
        }
    }
}

// ------------------------------------------------------------ face flux
// The face flux contracted with Fb.  face_flux takes the limiter branches
// from its inputs; the states sampled below keep every branch away from
// its switching point, so the branches stay the recorded ones (bl, br)
// under the finite-difference perturbations.
static double face_J(const Options &o, const double P[4][5], const Geo &g,
                     int d, const ConsBar &Fb)
{
    PVT<double> a, b, c2, e;
    for (int c = 0; c < 5; ++c)
    {
        a.q[c] = P[0][c];
        b.q[c] = P[1][c];
        c2.q[c] = P[2][c];
        e.q[c] = P[3][c];
    }
    return dotc(Fb, face_flux(o, a, b, c2, e, g, d));
}

static void check_face()
{
    Options o = opts();
    int n = 0;
    for (int t = 0; t < 200 && n < 60; ++t)
    {
        const int d = t % 3;
        const double x = U(-8, 8), y = U(-8, 8), z = U(-8, 8);
        double xr = x, yr = y, zr = z;
        (d == 0 ? xr : d == 1 ? yr : zr) += 0.5;
        const Geo gl = geo_at(x, y, z), gr = geo_at(xr, yr, zr);
        Geo g;
        average_geo(gl, gr, g);
        double P[4][5];
        const Prim base = rand_prim(0.3);
        for (int c = 0; c < 4; ++c)
        {
            const Prim q = rand_prim(0.3);
            P[c][0] = base.rho + 0.2 * (q.rho - 0.6);
            P[c][1] = base.p + 0.1 * (q.p - 0.15);
            for (int i = 0; i < 3; ++i)
                P[c][2 + i] = base.v[i] + 0.3 * q.v[i];
        }
        unsigned bl = 0, br = 0;
        {
            double l[5], c[5], r[5], rr[5];
            for (int q = 0; q < 5; ++q)
            {
                l[q] = P[0][q];
                c[q] = P[1][q];
                r[q] = P[2][q];
                rr[q] = P[3][q];
            }
            bl = slope_bits(l, c, r, o.theta);
            br = slope_bits(c, r, rr, o.theta);
        }
        // skip states where a perturbation would flip a limiter branch
        bool near = false;
        for (int q = 0; q < 5 && !near; ++q)
        {
            const double A = P[1][q] - P[0][q], B = P[2][q] - P[1][q],
                         C = P[3][q] - P[2][q];
            if (fabs(A) < 1e-3 || fabs(B) < 1e-3 || fabs(C) < 1e-3 ||
                fabs(2 * A - B) < 1e-3 || fabs(2 * B - A) < 1e-3 ||
                fabs(2 * B - C) < 1e-3 || fabs(2 * C - B) < 1e-3 ||
                fabs(o.theta * A - 0.5 * (A + B)) < 1e-3 ||
                fabs(o.theta * B - 0.5 * (A + B)) < 1e-3 ||
                fabs(o.theta * B - 0.5 * (B + C)) < 1e-3 ||
                fabs(o.theta * C - 0.5 * (B + C)) < 1e-3)
                near = true;
        }
        if (near)
            continue;
        ++n;
        const ConsBar Fb = rand_cbar();
        double qlb[5], qrb[5];
        GeoBar gb;
        zero(gb);
        face_flux_rev(o, P[0], P[1], P[2], P[3], bl, br, g, d, Fb, qlb, qrb,
                      gb);
        // the reconstruction is linear for fixed branches: chain the face
        // state adjoints back to the four cells
        double Pb[4][5] = {};
        for (int c = 0; c < 5; ++c)
        {
            double wl, wc, wr;
            Pb[1][c] += qlb[c];
            Pb[2][c] += qrb[c];
            slope_weights(bits_of(bl, c), o.theta, wl, wc, wr);
            Pb[0][c] += 0.5 * qlb[c] * wl;
            Pb[1][c] += 0.5 * qlb[c] * wc;
            Pb[2][c] += 0.5 * qlb[c] * wr;
            slope_weights(bits_of(br, c), o.theta, wl, wc, wr);
            Pb[1][c] -= 0.5 * qrb[c] * wl;
            Pb[2][c] -= 0.5 * qrb[c] * wc;
            Pb[3][c] -= 0.5 * qrb[c] * wr;
        }
        for (int cell = 0; cell < 4; ++cell)
            for (int c = 0; c < 5; ++c)
            {
                double Pa[4][5], Pm[4][5];
                for (int i = 0; i < 4; ++i)
                    for (int j = 0; j < 5; ++j)
                        Pa[i][j] = Pm[i][j] = P[i][j];
                const double h = 1e-7;
                Pa[cell][c] += h;
                Pm[cell][c] -= h;
                const double fd = (face_J(o, Pa, g, d, Fb) -
                                   face_J(o, Pm, g, d, Fb)) /
                                  (2 * h);
                report("face d/dP", Pb[cell][c], fd, 1.0 + fabs(fd), 5e-6);
            }
        // spin: the face geometry is the mean of the two cells' metrics
        GeoT<Dual> dl, dr, df;
        ks_metric_spin<false>(1.0, kSpin, x, y, z, dl, nullptr);
        ks_metric_spin<false>(1.0, kSpin, xr, yr, zr, dr, nullptr);
        average_geo(dl, dr, df);
        const double got = contract(gb, df);
        const double h = 1e-6;
        Geo ga, gm;
        average_geo(geo_at(x, y, z, kSpin + h), geo_at(xr, yr, zr, kSpin + h),
                    ga);
        average_geo(geo_at(x, y, z, kSpin - h), geo_at(xr, yr, zr, kSpin - h),
                    gm);
        const double fd = (face_J(o, P, ga, d, Fb) -
                           face_J(o, P, gm, d, Fb)) / (2 * h);
        report("face d/dspin", got, fd, 1.0 + fabs(fd), 5e-6);
    }
    if (n < 30)
    {
        printf("FAIL face: only %d usable samples\n", n);
        ++g_fail;
    }
}

// ------------------------------------------------------------- con2prim
static void check_con2prim()
{
    const Options o = opts();
    for (int t = 0; t < 20; ++t)
    {
        const double x = U(-8, 8), y = U(-8, 8), z = U(-8, 8);
        const Geo g = geo_at(x, y, z);
        const Prim p = rand_prim(0.4);
        const Cons c = p2c(p, g.gLL);
        Prim r;
        if (!con2prim(o, c, g.gUU, r, nullptr, nullptr))
        {
            printf("FAIL con2prim did not converge\n");
            ++g_fail;
            continue;
        }
        PrimBar pb = zero_prim_bar();
        pb.rho = U(-1, 1);
        pb.eps = U(-1, 1);
        pb.p = U(-1, 1);
        for (int i = 0; i < 3; ++i)
            pb.v[i] = U(-1, 1);
        auto J = [&](const Cons &cc, const double *gUU) {
            Prim q;
            con2prim(o, cc, gUU, q, nullptr, nullptr);
            return pb.rho * q.rho + pb.eps * q.eps + pb.p * q.p +
                   pb.v[0] * q.v[0] + pb.v[1] * q.v[1] + pb.v[2] * q.v[2];
        };
        ConsBar cb = zero_cons_bar();
        double gUUb[6] = {0, 0, 0, 0, 0, 0};
        con2prim_rev(o, c, g.gUU, r.p, pb, cb, gUUb);
        const double cbv[5] = {cb.D, cb.S[0], cb.S[1], cb.S[2], cb.tau};
        for (int k = 0; k < 5; ++k)
        {
            Cons a = c, m = c;
            double *pa = k == 0 ? &a.D : k == 4 ? &a.tau : &a.S[k - 1];
            double *pm = k == 0 ? &m.D : k == 4 ? &m.tau : &m.S[k - 1];
            const double h = 1e-5 * fmax(1e-2, fabs(*pa));
            *pa += h;
            *pm -= h;
            const double fd = (J(a, g.gUU) - J(m, g.gUU)) / (2 * h);
            report("con2prim d/dcons", cbv[k], fd, 1.0 + fabs(fd), 1e-5);
        }
        for (int q = 0; q < 6; ++q)
        {
            double ga[6], gm[6];
            for (int s = 0; s < 6; ++s)
                ga[s] = gm[s] = g.gUU[s];
            const double h = 1e-6;
            ga[q] += h;
            gm[q] -= h;
            const double fd = (J(c, ga) - J(c, gm)) / (2 * h);
            report("con2prim d/dgUU", gUUb[q], fd, 1.0 + fabs(fd), 1e-5);
        }
        // c2p_at reproduces the solver's primitives at its pressure
        const Prim q = c2p_at(o, c, g.gUU, r.p);
        report("c2p_at rho", q.rho, r.rho, 1.0, 1e-14);
        report("c2p_at v0", q.v[0], r.v[0], 1.0, 1e-14);
    }
}

// -------------------------------------------------------------- sources
static void check_sources()
{
    for (int t = 0; t < 20; ++t)
    {
        const double x = U(-8, 8), y = U(-8, 8), z = U(-8, 8);
        GeoFull f;
        ks_metric<double, true>(1.0, kSpin, x, y, z, f.g, &f);
        const Prim p = rand_prim(0.4);
        const Cons c = p2c(p, f.g.gLL);
        const ConsBar sb = rand_cbar();
        PrimBar pb = zero_prim_bar();
        ConsBar cb = zero_cons_bar();
        GeoFullBar fb;
        zero(fb);
        static_sources_rev(p, c, f, sb, pb, cb, fb);
        auto J = [&](const Prim &q, const Cons &cc, const GeoFull &ff) {
            return dotc(sb, static_sources(q, cc, ff));
        };
        for (int k = 0; k < 6; ++k)
        {
            Prim a = p, m = p;
            const double h = 1e-6 * fmax(1e-3, fabs(pval(p, k)));
            *pfield(a, k) += h;
            *pfield(m, k) -= h;
            const double fd = (J(a, c, f) - J(m, c, f)) / (2 * h);
            report("sources d/dprim", pbfield(pb, k), fd, 1.0 + fabs(fd));
        }
        const double cbv[5] = {cb.D, cb.S[0], cb.S[1], cb.S[2], cb.tau};
        for (int k = 0; k < 5; ++k)
        {
            Cons a = c, m = c;
            double *pa = k == 0 ? &a.D : k == 4 ? &a.tau : &a.S[k - 1];
            double *pm = k == 0 ? &m.D : k == 4 ? &m.tau : &m.S[k - 1];
            const double h = 1e-6 * fmax(1e-2, fabs(*pa));
            *pa += h;
            *pm -= h;
            const double fd = (J(p, a, f) - J(p, m, f)) / (2 * h);
            report("sources d/dcons", cbv[k], fd, 1.0 + fabs(fd));
        }
        GeoFullT<Dual> fd_;
        ks_metric_spin<true>(1.0, kSpin, x, y, z, fd_.g, &fd_);
        const double got = contract(fb, fd_);
        const double h = 1e-6;
        GeoFull fa, fm;
        ks_metric<double, true>(1.0, kSpin + h, x, y, z, fa.g, &fa);
        ks_metric<double, true>(1.0, kSpin - h, x, y, z, fm.g, &fm);
        const double fdv = (J(p, c, fa) - J(p, c, fm)) / (2 * h);
        report("sources d/dspin", got, fdv, 1.0 + fabs(fdv), 5e-6);
        // dual metric values equal the double metric
        GeoFull fv;
        values_of(fd_, fv);
        report("dual metric K01", fv.K[1], f.K[1], 1.0, 1e-13);
        report("dual metric dgamma", fv.dgamma[2][4], f.dgamma[2][4], 1.0,
               1e-13);
    }
}

// ------------------------------------------------- post-update recovery
static Cons recover_fwd(const Options &o, const Cons &Y, const Geo &g, int &br)
{
    Prim pr;
    if (!con2prim(o, Y, g.gUU, pr, nullptr, nullptr))
    {
        br = 2;
        return p2c(atmosphere(o), g.gLL);
    }
    Prim fl = pr;
    floors(o, fl, g.gLL);
    br = differs(pr, fl) ? 1 : 0;
    return br ? p2c(fl, g.gLL) : Y;
}

static void check_recovery()
{
    Options o = opts();
    o.atmo_vmax2 = 0.3; // so that the velocity cap resets some cells
    int n1 = 0;
    for (int t = 0; t < 40; ++t)
    {
        const double x = U(-8, 8), y = U(-8, 8), z = U(-8, 8);
        const Geo g = geo_at(x, y, z);
        const Prim p = rand_prim(0.5);
        const Cons Y = p2c(p, g.gLL);
        int br;
        recover_fwd(o, Y, g, br);
        Prim pr;
        con2prim(o, Y, g.gUU, pr, nullptr, nullptr);
        const ConsBar Ub = rand_cbar();
        GeoBar gb;
        zero(gb);
        const ConsBar Yb = recovery_rev(o, Y, br, pr.p, g, Ub, gb);
        if (br == 1)
            ++n1;
        const double ybv[5] = {Yb.D, Yb.S[0], Yb.S[1], Yb.S[2], Yb.tau};
        for (int k = 0; k < 5; ++k)
        {
            Cons a = Y, m = Y;
            double *pa = k == 0 ? &a.D : k == 4 ? &a.tau : &a.S[k - 1];
            double *pm = k == 0 ? &m.D : k == 4 ? &m.tau : &m.S[k - 1];
            const double h = 1e-6 * fmax(1e-2, fabs(*pa));
            *pa += h;
            *pm -= h;
            int ba, bm;
            const double fd = (dotc(Ub, recover_fwd(o, a, g, ba)) -
                               dotc(Ub, recover_fwd(o, m, g, bm))) / (2 * h);
            if (ba != br || bm != br)
                continue;
            report("recovery d/dY", ybv[k], fd, 1.0 + fabs(fd), 1e-5);
        }
    }
    if (n1 < 5)
    {
        printf("FAIL recovery: only %d reset samples\n", n1);
        ++g_fail;
    }
}

// --------------------------------------------------- torus initial data
static void check_torus()
{
    Options o = opts();
    const double M = 1.0, r_in = 3.0, r_max = 5.0, vmax2 = 0.8;
    const double phase[5] = {0.3, 1.1, 2.0, 4.0, 5.5};
    auto theta_at = [&](const double th[8], TorusThetaT<double> &T,
                        TorusSetup &S) {
        if (!torus_setup(M, th[2], r_in, r_max, vmax2, o.G, S))
            return false;
        T.A = th[0];
        T.K = th[1];
        T.a = th[2];
        for (int m = 0; m < 5; ++m)
            T.eps[m] = th[3 + m];
        T.ell = S.ell;
        T.W_in = S.W_in;
        return true;
    };
    double th0[8] = {1.0, 0.0, 0.7, 0.01, 0.008, 0.006, 0.004, 0.002};
    TorusSetup S0;
    if (!torus_setup(M, th0[2], r_in, r_max, vmax2, o.G, S0))
    {
        printf("FAIL torus setup\n");
        ++g_fail;
        return;
    }
    th0[1] = S0.K_unit;
    int checked = 0;
    for (int t = 0; t < 400 && checked < 40; ++t)
    {
        const double R = U(3.2, 8.0), ph = U(0, 6.283), z = U(-1.0, 1.0);
        const double x = R * cos(ph), y = R * sin(ph);
        TorusThetaT<double> T0;
        TorusSetup S;
        theta_at(th0, T0, S);
        PrimT<double> p0;
        torus_cell_T<double>(o, M, T0, phase, r_in, vmax2, x, y, z, p0);
        if (!(p0.rho > 1e-6))
            continue; // atmosphere: parameter independent
        ++checked;
        const ConsBar w = rand_cbar();
        for (int k = 0; k < 8; ++k)
        {
            TorusThetaT<Dual> TD;
            TD.A = Dual(th0[0], k == 0);
            TD.K = Dual(th0[1], k == 1);
            TD.a = Dual(th0[2], k == 2);
            for (int m = 0; m < 5; ++m)
                TD.eps[m] = Dual(th0[3 + m], k == 3 + m);
            TD.ell = Dual(S0.ell, k == 2 ? S0.dell_da : 0.0);
            TD.W_in = Dual(S0.W_in, k == 2 ? S0.dWin_da : 0.0);
            PrimT<Dual> pd;
            const ConsT<Dual> cd =
                torus_cell_T<Dual>(o, M, TD, phase, r_in, vmax2, x, y, z, pd);
            const double got = w.D * cd.D.d + w.tau * cd.tau.d +
                               w.S[0] * cd.S[0].d + w.S[1] * cd.S[1].d +
                               w.S[2] * cd.S[2].d;
            const double h = 1e-6 * fmax(0.1, fabs(th0[k]));
            double tp[8], tm[8];
            for (int q = 0; q < 8; ++q)
                tp[q] = tm[q] = th0[q];
            tp[k] += h;
            tm[k] -= h;
            TorusThetaT<double> Tp, Tm;
            TorusSetup Sp, Sm;
            theta_at(tp, Tp, Sp);
            theta_at(tm, Tm, Sm);
            PrimT<double> pp, pm;
            const Cons cp =
                torus_cell_T<double>(o, M, Tp, phase, r_in, vmax2, x, y, z, pp);
            const Cons cm =
                torus_cell_T<double>(o, M, Tm, phase, r_in, vmax2, x, y, z, pm);
            const double fd = (dotc(w, cp) - dotc(w, cm)) / (2 * h);
            char lbl[64];
            snprintf(lbl, sizeof lbl, "torus d/dtheta[%d]", k);
            report(lbl, got, fd,
                   1e-3 + fabs(fd), 1e-5);
        }
    }
    if (checked < 20)
    {
        printf("FAIL torus: only %d torus cells sampled\n", checked);
        ++g_fail;
    }
}

int main()
{
    check_p2c();
    check_floors();
    check_speeds();
    check_face();
    check_con2prim();
    check_sources();
    check_recovery();
    check_torus();
    printf("%s: %d failures\n", g_fail ? "FAILED" : "PASSED", g_fail);
    return g_fail ? 1 : 0;
}
