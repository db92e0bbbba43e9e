// adjoint_rhs_check.cu -- host check of the discrete adjoint's work items
// (grhd_adjoint_items.cuh: limiter bits, face / shell / cell reverse, the
// taped RK4 stage and the reverse of the recovery), run in host loops
// exactly as the kernels run them, against central finite differences of
// the CPU oracle (the reference's algorithm): one RHS evaluation with its
// accretion rate, and one RK4 step with its accretion integral, on a small
// Kerr-Schild box with atmosphere, excision, velocity caps and physical
// boundaries.  Built and run by tests/test_adjoint_host.py (no GPU).
#include "grhd_adjoint_items.cuh"
#include "grhd_oracle.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

using namespace grhd;
using namespace grhd::adj;

static std::mt19937_64 rng(7);
static double U01() { return std::uniform_real_distribution<double>(-1, 1)(rng); }

struct Case
{
    BoxDev b;
    Options o;
    orc_params p;
    orc_box ob;
    double inv[3];
};

static Case make_case(int nx, int ny, int nz, double dx, double spin)
{
    Case c;
    const int n[3] = {nx, ny, nz};
    for (int d = 0; d < 3; ++d)
    {
        c.b.lo[d] = 0;
        c.b.hi[d] = n[d] - 1;
        c.b.glo[d] = -2;
        c.b.ghi[d] = n[d] + 1;
        c.b.dlo[d] = 0;
        c.b.dhi[d] = n[d] - 1;
        c.b.gn[d] = n[d] + 4;
        c.b.in[d] = n[d];
        c.ob.lo[d] = 0;
        c.ob.hi[d] = n[d] - 1;
        c.ob.glo[d] = -2;
        c.ob.ghi[d] = n[d] + 1;
        c.ob.dlo[d] = 0;
        c.ob.dhi[d] = n[d] - 1;
        c.inv[d] = 1.0 / dx;
    }
    c.b.cs = c.b.gvol();
    c.b.pcs = c.b.gvol();
    c.b.rcs = c.b.ivol();
    c.ob.comp_stride = c.b.gvol();
    Options &o = c.o;
    std::memset(&o, 0, sizeof(o));
    o.G = 5.0 / 3.0;
    // floors well above the recovery's absolute residual tolerance, so that
    // the converged pressure of an atmosphere cell is its root to rounding
    o.rho_floor = 1e-5;
    o.p_floor = 1e-7;
    o.atmo_vmax2 = 0.8;
    o.src_atmo_factor = 1.0 + 1e-12;
    o.rec_maxit = 80;
    o.rec_tol = 1e-12;
    o.rec_pfloor = 1e-12;
    o.rec_vmax2 = 0.9;
    o.theta = 2.0;
    o.use_recon = 1;
    o.use_src = 1;
    o.use_vol = 0;
    o.excision_radius = 1.2;
    o.accretion_radius = 1.7; // inside the domain
    o.dx = dx;
    for (int d = 0; d < 3; ++d)
        o.center[d] = 0.5 * n[d] * dx + (d == 1 ? 0.13 : 0.0);
    orc_default_params(&c.p);
    orc_params &p = c.p;
    p.background = 0;
    p.ks_mass = 1.0;
    p.ks_spin = spin;
    p.gamma = o.G;
    p.dx = dx;
    for (int d = 0; d < 3; ++d)
        p.center[d] = o.center[d];
    p.atmo_rho_floor = o.rho_floor;
    p.atmo_pressure_floor = o.p_floor;
    p.atmo_max_velocity_squared = o.atmo_vmax2;
    p.atmo_metric_source_atmosphere_factor = o.src_atmo_factor;
    p.rec_max_iterations = o.rec_maxit;
    p.rec_tolerance = o.rec_tol;
    p.rec_pressure_floor = o.rec_pfloor;
    p.rec_max_velocity_squared = o.rec_vmax2;
    p.limiter_theta = o.theta;
    p.use_reconstruction = 1;
    p.use_static_metric_sources = 1;
    p.use_metric_volume_time_sources = 0;
    p.excision_radius = o.excision_radius;
    p.accretion_radius = o.accretion_radius;
    return c;
}

// A smooth inflowing state with an atmosphere region and a few fast cells.
static std::vector<double> make_state(const Case &c, double spin)
{
    const BoxDev &b = c.b;
    std::vector<double> s((size_t)kStateComps * b.gvol());
    for (int64_t g = 0; g < b.gvol(); ++g)
    {
        int q[3];
        cell_of(b, g, q);
        double x, y, z;
        cell_xyz(c.o, q[0], q[1], q[2], x, y, z);
        const double r = sqrt(x * x + y * y + z * z) + 1e-9;
        Prim pr;
        pr.rho = 0.4 + 0.2 * sin(0.7 * x + 0.3 * y) * cos(0.5 * z) +
                 0.01 * U01();
        pr.p = 0.05 + 0.02 * cos(0.4 * x - 0.6 * y + 0.2 * z) + 0.002 * U01();
        const double vr = -0.35 / sqrt(r);
        pr.v[0] = vr * x / r + 0.15 * sin(y) + 0.02 * U01();
        pr.v[1] = vr * y / r - 0.15 * sin(x) + 0.02 * U01();
        pr.v[2] = vr * z / r + 0.05 * U01();
        if (x > 1.6 * c.o.dx * 3)
        {
            // a low-density layer 1.2-1.8 x the floors: the
            // reconstruction undershoots it, so the face floors act
            // (a state exactly at a floor would sit on the floor's kink)
            pr.rho = 1e-5 * (1.5 + 0.3 * U01());
            pr.p = 1e-7 * (1.5 + 0.3 * U01());
        }
        Geo geo;
        ks_metric<double, false>(1.0, spin, x, y, z, geo, nullptr);
        if (r < c.o.excision_radius)
        {
            // frozen excised cells: a finite state even where the metric
            // is singular (the ring of the spinning hole)
            pr = atmosphere(c.o);
            if (!(geo.gLL[0] == geo.gLL[0] && geo.lapse == geo.lapse))
                for (int q = 0; q < 6; ++q)
                    geo.gLL[q] = (q == 0 || q == 3 || q == 5) ? 1.0 : 0.0;
        }
        floors(c.o, pr, geo.gLL);
        if (q[0] == 3 && q[1] == 4 && r >= c.o.excision_radius)
        {
            // v^2 = 0.85: above the floors' cap 0.8 (faces and sources
            // rescale it), below the recovery's cap 0.9
            const double vv[3] = {1.0, 0.3, 0.1};
            const double s2 = vsq(vv, geo.gLL);
            for (int i = 0; i < 3; ++i)
                pr.v[i] = vv[i] * sqrt(0.85 / s2);
        }
        const Cons u = p2c(pr, geo.gLL);
        const int64_t cs = b.cs;
        s[kD * cs + g] = u.D;
        s[(kS1 + 0) * cs + g] = u.S[0];
        s[(kS1 + 1) * cs + g] = u.S[1];
        s[(kS1 + 2) * cs + g] = u.S[2];
        s[kTau * cs + g] = u.tau;
        s[kRho * cs + g] = pr.rho;
        s[kEps * cs + g] = pr.eps;
        s[kPress * cs + g] = pr.p;
        for (int i = 0; i < 3; ++i)
            s[(kV1 + i) * cs + g] = pr.v[i];
    }
    return s;
}

// The RHS (oracle) with ghosts filled in `s`; returns Mdot.
static double oracle_rhs(const Case &c, std::vector<double> &s,
                         std::vector<double> &rhs)
{
    rhs.assign((size_t)5 * c.b.ivol(), 0.0);
    double mdot = 0.0;
    orc_error err;
    if (orc_compute_rhs_mdot(&c.p, &c.ob, s.data(), rhs.data(), c.b.ivol(),
                             c.inv, 0.0, &mdot, &err) != 0)
    {
        printf("FAIL oracle rhs error %d at %d %d %d\n", err.code, err.cell[0],
               err.cell[1], err.cell[2]);
        exit(1);
    }
    return mdot;
}

// Primitive cache of a ghost-filled state, as the RHS kernels build it.
static std::vector<double> prim_cache(const Case &c, const std::vector<double> &s,
                                      double spin)
{
    const BoxDev &b = c.b;
    std::vector<double> P((size_t)5 * b.gvol());
    for (int64_t g = 0; g < b.gvol(); ++g)
    {
        int q[3];
        cell_of(b, g, q);
        Prim pr;
        const bool interior = q[0] >= b.lo[0] && q[0] <= b.hi[0] &&
                              q[1] >= b.lo[1] && q[1] <= b.hi[1] &&
                              q[2] >= b.lo[2] && q[2] <= b.hi[2];
        if (interior && excised(c.o, q[0], q[1], q[2]))
        {
            pr.rho = s[kRho * b.cs + g];
            pr.p = s[kPress * b.cs + g];
            for (int i = 0; i < 3; ++i)
                pr.v[i] = s[(kV1 + i) * b.cs + g];
        }
        else
        {
            double x, y, z;
            cell_xyz(c.o, q[0], q[1], q[2], x, y, z);
            Geo geo;
            ks_metric<double, false>(1.0, spin, x, y, z, geo, nullptr);
            if (!con2prim(c.o, load_cons5(s.data(), b.cs, g), geo.gUU, pr,
                          nullptr, nullptr))
            {
                pr.rho = pr.p = 1.0;
                pr.v[0] = pr.v[1] = pr.v[2] = 0.0;
            }
        }
        P[0 * b.gvol() + g] = pr.rho;
        P[1 * b.gvol() + g] = pr.p;
        for (int i = 0; i < 3; ++i)
            P[(2 + i) * b.gvol() + g] = pr.v[i];
    }
    return P;
}

struct Tape
{
    std::vector<double> U[4], P[4], Y[4], pY[4];
    std::vector<unsigned> bits[4];
    std::vector<unsigned char> br[4];
    double J = 0.0;
};

// One RK4 step with the oracle RHS and the adjoint's taping stage items.
static std::vector<double> tape_step(const Case &c, const std::vector<double> &s0,
                                     double dt, double spin, Tape &T)
{
    const BoxDev &b = c.b;
    const int64_t iv = b.ivol(), gv = b.gvol();
    std::vector<double> acc((size_t)5 * iv), rhs, next;
    T.U[0] = s0;
    T.J = 0.0;
    for (int st = 0; st < 4; ++st)
    {
        const double mdot = oracle_rhs(c, T.U[st], rhs);
        T.J += dt / 6.0 * stage_weight(st) * mdot;
        T.P[st] = prim_cache(c, T.U[st], spin);
        T.bits[st].assign((size_t)gv, 0u);
        for (int64_t g = 0; g < gv; ++g)
            bits_item(b, c.o, T.P[st].data(), T.bits[st].data(), g);
        T.Y[st].assign((size_t)5 * iv, 0.0);
        T.pY[st].assign((size_t)iv, 0.0);
        T.br[st].assign((size_t)iv, 0);
        std::vector<double> &out = (st < 3) ? T.U[st + 1] : next;
        out = T.U[0];
        for (int64_t t = 0; t < iv; ++t)
            stage_tape_item(b, c.o, 1.0, spin, T.U[0].data(), rhs.data(),
                            acc.data(), st, dt, out.data(), T.Y[st].data(),
                            T.pY[st].data(), T.br[st].data(), t);
    }
    return next;
}

struct Rev
{
    std::vector<double> fb, gbuf, lamk, lam, A, acc;
    double spin = 0.0;
};

static void reverse_rhs(const Case &c, const Tape &T, int st, double mu,
                        const AdjStage &S0, Rev &R, double spin)
{
    const BoxDev &b = c.b;
    AdjRhs A;
    A.b = b;
    A.o = c.o;
    A.M = 1.0;
    A.a = spin;
    for (int d = 0; d < 3; ++d)
        A.inv_dx[d] = c.inv[d];
    A.U = T.U[st].data();
    A.P = T.P[st].data();
    A.bits = T.bits[st].data();
    A.lamk = R.lamk.data();
    A.mu = mu;
    A.fb = R.fb.data();
    A.gbuf = R.gbuf.data();
    for (int d = 0; d < 3; ++d)
    {
        int n[3] = {b.in[0], b.in[1], b.in[2]};
        n[d] += 1;
        const int64_t nf = (int64_t)n[0] * n[1] * n[2];
        for (int64_t t = 0; t < nf; ++t)
            R.spin += face_rev_item(A, d, t);
    }
    for (int64_t g = 0; g < b.gvol(); ++g)
        R.spin += shell_rev_item(A, g);
    for (int64_t t = 0; t < b.ivol(); ++t)
        R.spin += cell_rev_item(A, S0, t);
}

static int g_fail = 0;

// A central difference whose step crosses a switch of the scheme (a
// limiter or HLLE branch, a floor) measures a different one-sided slope;
// the adjoint is the derivative of the branch taken, so it is compared
// with the closest of the differences over a range of steps.
template <typename F>
static double best_fd(double adj, F fd_of, double &h_used)
{
    double best = 0.0, err = INFINITY;
    for (double h : {1e-6, 1e-7, 1e-8})
    {
        const double fd = fd_of(h);
        const double e = fabs(adj - fd);
        if (e < err)
        {
            err = e;
            best = fd;
            h_used = h;
        }
    }
    return best;
}

static void compare(const char *what, double adj, double fd, double tol)
{
    const double err = fabs(adj - fd) / fmax(fabs(fd), 1e-300);
    const bool ok = err <= tol;
    if (!ok)
        ++g_fail;
    printf("%-4s %-34s adj % .12e fd % .12e rel %.2e\n", ok ? "ok" : "FAIL",
           what, adj, fd, err);
}

static void check_rhs(double spin)
{
    Case c = make_case(12, 10, 9, 0.5, spin);
    const BoxDev &b = c.b;
    const int64_t iv = b.ivol(), gv = b.gvol();
    std::vector<double> s = make_state(c, spin), rhs;
    const double mu = 0.37;
    oracle_rhs(c, s, rhs); // fills ghosts
    Tape T;
    T.U[0] = s;
    T.P[0] = prim_cache(c, s, spin);
    T.bits[0].assign((size_t)gv, 0u);
    for (int64_t g = 0; g < gv; ++g)
        bits_item(b, c.o, T.P[0].data(), T.bits[0].data(), g);
    Rev R;
    R.fb.assign((size_t)30 * gv, 0.0);
    R.gbuf.assign((size_t)5 * gv, 0.0);
    R.lamk.resize((size_t)5 * iv);
    R.lam.assign((size_t)5 * iv, 0.0);
    for (auto &v : R.lamk)
        v = U01();
    AdjStage S;
    std::memset(&S, 0, sizeof(S));
    S.stage = -1;
    S.out = R.lam.data();
    reverse_rhs(c, T, 0, mu, S, R, spin);
    // directional derivative along a random interior perturbation
    std::vector<double> dir((size_t)5 * iv);
    for (auto &v : dir)
        v = U01();
    auto J = [&](const std::vector<double> &st, double a) {
        Case cc = c;
        cc.p.ks_spin = a;
        std::vector<double> w = st, r;
        const double m = oracle_rhs(cc, w, r);
        double acc = mu * m;
        for (int64_t i = 0; i < 5 * iv; ++i)
            acc += R.lamk[i] * r[i];
        return acc;
    };
    const int comp_of[5] = {kD, kS1, kS1 + 1, kS1 + 2, kTau};
    double adj = 0.0;
    for (int64_t t = 0; t < iv; ++t)
        for (int q = 0; q < 5; ++q)
            if (R.lam[q * iv + t] != 0.0)
                adj += R.lam[q * iv + t] * dir[q * iv + t] *
                   s[comp_of[q] * b.cs + b.gidx(b.lo[0] + t % b.in[0],
                                               b.lo[1] + (t / b.in[0]) % b.in[1],
                                               b.lo[2] + t / (b.in[0] * b.in[1]))];
    auto perturbed = [&](double h) {
        std::vector<double> w = s;
        for (int64_t t = 0; t < iv; ++t)
        {
            const int i = b.lo[0] + t % b.in[0];
            const int j = b.lo[1] + (t / b.in[0]) % b.in[1];
            const int k = b.lo[2] + t / (b.in[0] * b.in[1]);
            const int64_t g = b.gidx(i, j, k);
            for (int q = 0; q < 5; ++q)
                w[comp_of[q] * b.cs + g] *= 1.0 + h * dir[q * iv + t];
        }
        return w;
    };
    {
        double h;
        const double fd = best_fd(adj, [&](double hh) {
            return (J(perturbed(hh), spin) - J(perturbed(-hh), spin)) /
                   (2 * hh);
        }, h);
        char lbl[64];
        snprintf(lbl, sizeof lbl, "rhs vjp, a=%.2f (h=%.0e)", spin, h);
        compare(lbl, adj, fd, 1e-6);
    }
    if (spin != 0.0)
    {
        double h;
        const double fd = best_fd(R.spin, [&](double hh) {
            return (J(s, spin + hh) - J(s, spin - hh)) / (2 * hh);
        }, h);
        char lbl[64];
        snprintf(lbl, sizeof lbl, "rhs spin, a=%.2f (h=%.0e)", spin, h);
        compare(lbl, R.spin, fd, 1e-6);
    }
}

static void check_step(double spin)
{
    Case c = make_case(12, 10, 9, 0.5, spin);
    const BoxDev &b = c.b;
    const int64_t iv = b.ivol(), gv = b.gvol();
    std::vector<double> s = make_state(c, spin), rhs;
    oracle_rhs(c, s, rhs); // ghost fill, as the previous step would leave it
    double dt;
    {
        orc_error err;
        orc_compute_stable_dt(&c.p, &c.ob, s.data(), c.inv, 0.25, 0.0, &dt,
                              &err);
    }
    Tape T;
    tape_step(c, s, dt, spin, T);
    // the taped step against the oracle's RK4 (same arithmetic)
    {
        std::vector<double> w = s;
        double mi = 0.0;
        orc_diag dg;
        orc_error err;
        orc_advance_rk4_mdot(&c.p, &c.ob, w.data(), c.inv, 0.0, dt, &dg, &err,
                             &mi);
        compare("taped step J vs oracle RK4", T.J, mi, 1e-10);
    }
    const double muJ = 0.61;
    Rev R;
    R.fb.assign((size_t)30 * gv, 0.0);
    R.gbuf.assign((size_t)5 * gv, 0.0);
    R.lamk.assign((size_t)5 * iv, 0.0);
    R.lam.resize((size_t)5 * iv);
    R.A.assign((size_t)5 * iv, 0.0);
    R.acc.assign((size_t)5 * iv, 0.0);
    std::vector<double> lam_next((size_t)5 * iv);
    for (auto &v : lam_next)
        v = U01();
    R.lam = lam_next;
    for (int64_t t = 0; t < iv; ++t)
        R.spin += proj_rev_item(b, c.o, 1.0, spin, dt, R.lam.data(),
                                T.Y[3].data(), T.pY[3].data(), T.br[3].data(),
                                R.A.data(), R.acc.data(), R.lamk.data(), t);
    for (int st = 3; st >= 0; --st)
    {
        AdjStage S;
        S.stage = st;
        S.dt = dt;
        S.Y = st >= 1 ? T.Y[st - 1].data() : nullptr;
        S.pY = st >= 1 ? T.pY[st - 1].data() : nullptr;
        S.br = st >= 1 ? T.br[st - 1].data() : nullptr;
        S.A = R.A.data();
        S.acc = R.acc.data();
        S.lamk = R.lamk.data();
        S.out = R.lam.data();
        reverse_rhs(c, T, st, muJ * dt / 6.0 * stage_weight(st), S, R, spin);
    }
    std::vector<double> dir((size_t)5 * iv);
    for (auto &v : dir)
        v = U01();
    const int comp_of[5] = {kD, kS1, kS1 + 1, kS1 + 2, kTau};
    auto J = [&](const std::vector<double> &st, double a) {
        Case cc = c;
        cc.p.ks_spin = a;
        std::vector<double> w = st;
        double mi = 0.0;
        orc_diag dg;
        orc_error err;
        orc_advance_rk4_mdot(&cc.p, &cc.ob, w.data(), c.inv, 0.0, dt, &dg,
                             &err, &mi);
        double acc = muJ * mi;
        for (int64_t t = 0; t < iv; ++t)
        {
            const int i = b.lo[0] + t % b.in[0];
            const int j = b.lo[1] + (t / b.in[0]) % b.in[1];
            const int k = b.lo[2] + t / (b.in[0] * b.in[1]);
            const int64_t g = b.gidx(i, j, k);
            for (int q = 0; q < 5; ++q)
                acc += lam_next[q * iv + t] * w[comp_of[q] * b.cs + g];
        }
        return acc;
    };
    double adj = 0.0;
    auto perturbed = [&](double h) {
        std::vector<double> w = s;
        for (int64_t t = 0; t < iv; ++t)
        {
            const int i = b.lo[0] + t % b.in[0];
            const int j = b.lo[1] + (t / b.in[0]) % b.in[1];
            const int k = b.lo[2] + t / (b.in[0] * b.in[1]);
            const int64_t g = b.gidx(i, j, k);
            for (int q = 0; q < 5; ++q)
                w[comp_of[q] * b.cs + g] *= 1.0 + h * dir[q * iv + t];
        }
        return w;
    };
    for (int64_t t = 0; t < iv; ++t)
    {
        const int i = b.lo[0] + t % b.in[0];
        const int j = b.lo[1] + (t / b.in[0]) % b.in[1];
        const int k = b.lo[2] + t / (b.in[0] * b.in[1]);
        const int64_t g = b.gidx(i, j, k);
        for (int q = 0; q < 5; ++q)
            if (R.lam[q * iv + t] != 0.0)
                adj += R.lam[q * iv + t] * dir[q * iv + t] *
                       s[comp_of[q] * b.cs + g];
    }
    {
        double h;
        const double fd = best_fd(adj, [&](double hh) {
            return (J(perturbed(hh), spin) - J(perturbed(-hh), spin)) /
                   (2 * hh);
        }, h);
        char lbl[64];
        snprintf(lbl, sizeof lbl, "step vjp, a=%.2f (h=%.0e)", spin, h);
        compare(lbl, adj, fd, 1e-6);
    }
    double h;
    const double fd = best_fd(R.spin, [&](double hh) {
        return (J(s, spin + hh) - J(s, spin - hh)) / (2 * hh);
    }, h);
    char lbl[64];
    snprintf(lbl, sizeof lbl, "step spin, a=%.2f (h=%.0e)", spin, h);
    compare(lbl, R.spin, fd, 1e-6);
}

int main()
{
    check_rhs(0.0);
    check_rhs(0.7);
    check_step(0.7);
    printf("%s: %d failures\n", g_fail ? "FAILED" : "PASSED", g_fail);
    return g_fail ? 1 : 0;
}
