// grhd_dual.cuh -- forward-mode dual numbers (a value and one directional
// derivative) for the spin derivative of the analytic metric and of the
// torus initial data.  The metric and torus functions are templates on
// their arithmetic type; instantiated with Dual and the spin seeded with
// derivative 1 they return each quantity together with d/da.
#pragma once

#include "grhd_device.cuh"

#include <math.h>

namespace grhd {

struct Dual
{
    double v, d;
    GRHD_HD Dual() : v(0.0), d(0.0) {}
    GRHD_HD Dual(double x) : v(x), d(0.0) {}
    GRHD_HD Dual(double x, double dx) : v(x), d(dx) {}
};

GRHD_HD inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
GRHD_HD inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
GRHD_HD inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
GRHD_HD inline Dual operator*(Dual a, Dual b)
{
    return Dual(a.v * b.v, a.d * b.v + a.v * b.d);
}
GRHD_HD inline Dual operator/(Dual a, Dual b)
{
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
GRHD_HD inline Dual operator+(Dual a, double b) { return Dual(a.v + b, a.d); }
GRHD_HD inline Dual operator+(double a, Dual b) { return Dual(a + b.v, b.d); }
GRHD_HD inline Dual operator-(Dual a, double b) { return Dual(a.v - b, a.d); }
GRHD_HD inline Dual operator-(double a, Dual b) { return Dual(a - b.v, -b.d); }
GRHD_HD inline Dual operator*(Dual a, double b) { return Dual(a.v * b, a.d * b); }
GRHD_HD inline Dual operator*(double a, Dual b) { return Dual(a * b.v, a * b.d); }
GRHD_HD inline Dual operator/(Dual a, double b) { return Dual(a.v / b, a.d / b); }
GRHD_HD inline Dual operator/(double a, Dual b)
{
    const double q = a / b.v;
    return Dual(q, -q * b.d / b.v);
}
GRHD_HD inline Dual &operator+=(Dual &a, Dual b)
{
    a = a + b;
    return a;
}
GRHD_HD inline Dual &operator-=(Dual &a, Dual b)
{
    a = a - b;
    return a;
}
GRHD_HD inline Dual &operator*=(Dual &a, Dual b)
{
    a = a * b;
    return a;
}
GRHD_HD inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
GRHD_HD inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
GRHD_HD inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
GRHD_HD inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }

GRHD_HD inline Dual div_(Dual a, Dual b) { return a / b; }
GRHD_HD inline Dual rcp_(Dual a) { return 1.0 / a; }
GRHD_HD inline Dual sqrt_(Dual a)
{
    const double s = sqrt(a.v);
    return Dual(s, a.d / (2.0 * s));
}
GRHD_HD inline Dual rsqrt_(Dual a)
{
    const double r = 1.0 / sqrt(a.v);
    return Dual(r, -0.5 * r * r * r * a.d);
}
GRHD_HD inline Dual lapse_rsqrt(Dual a) { return rsqrt_(a); }
// max/min return the selected operand (derivative included)
GRHD_HD inline Dual max_(Dual a, Dual b) { return (a.v >= b.v) ? a : b; }
GRHD_HD inline Dual min_(Dual a, Dual b) { return (a.v <= b.v) ? a : b; }
GRHD_HD inline Dual abs_(Dual a) { return (a.v < 0.0) ? -a : a; }
GRHD_HD inline Dual exp_(Dual a)
{
    const double e = exp(a.v);
    return Dual(e, e * a.d);
}
GRHD_HD inline Dual log_(Dual a) { return Dual(log(a.v), a.d / a.v); }
GRHD_HD inline Dual cos_(Dual a) { return Dual(cos(a.v), -sin(a.v) * a.d); }
GRHD_HD inline Dual pow_(Dual a, double e)
{
    const double p = pow(a.v, e);
    return Dual(p, e * pow(a.v, e - 1.0) * a.d);
}
GRHD_HD inline double exp_(double a) { return exp(a); }
GRHD_HD inline double log_(double a) { return log(a); }
GRHD_HD inline double cos_(double a) { return cos(a); }
GRHD_HD inline double pow_(double a, double e) { return pow(a, e); }

GRHD_HD inline double val(double a) { return a; }
GRHD_HD inline double val(Dual a) { return a.v; }
GRHD_HD inline double der(double) { return 0.0; }
GRHD_HD inline double der(Dual a) { return a.d; }

} // namespace grhd
