// Oracle test infrastructure (not product code): forward-mode dual numbers
// used to differentiate the lineshape factors with respect to the resonance
// parameters of one amplitude block. Only tests and the CPU baseline use it.
#pragma once

#include <cmath>

namespace oracle {

constexpr int NDUAL = 16;  // max differentiated parameters per block

struct D {
    double v = 0.0;
    double g[NDUAL] = {};
    D() = default;
    D(double x) : v(x) {}  // NOLINT: constants convert implicitly
    static D var(double x, int k)
    {
        D d(x);
        d.g[k] = 1.0;
        return d;
    }
};

inline D operator+(const D& a, const D& b)
{
    D r(a.v + b.v);
    for (int k = 0; k < NDUAL; ++k) r.g[k] = a.g[k] + b.g[k];
    return r;
}
inline D operator-(const D& a, const D& b)
{
    D r(a.v - b.v);
    for (int k = 0; k < NDUAL; ++k) r.g[k] = a.g[k] - b.g[k];
    return r;
}
inline D operator-(const D& a)
{
    D r(-a.v);
    for (int k = 0; k < NDUAL; ++k) r.g[k] = -a.g[k];
    return r;
}
inline D operator*(const D& a, const D& b)
{
    D r(a.v * b.v);
    for (int k = 0; k < NDUAL; ++k) r.g[k] = a.g[k] * b.v + a.v * b.g[k];
    return r;
}
inline D operator/(const D& a, const D& b)
{
    D r(a.v / b.v);
    double ib = 1.0 / b.v;
    for (int k = 0; k < NDUAL; ++k) r.g[k] = (a.g[k] - r.v * b.g[k]) * ib;
    return r;
}
inline D& operator+=(D& a, const D& b) { return a = a + b; }
inline D& operator*=(D& a, const D& b) { return a = a * b; }
inline D chain(const D& a, double f, double df)
{
    D r(f);
    for (int k = 0; k < NDUAL; ++k) r.g[k] = df * a.g[k];
    return r;
}
inline D sqrt(const D& a)
{
    double s = std::sqrt(a.v);
    return chain(a, s, s > 0 ? 0.5 / s : 0.0);
}
inline D log(const D& a) { return chain(a, std::log(a.v), 1.0 / a.v); }
inline D exp(const D& a)
{
    double e = std::exp(a.v);
    return chain(a, e, e);
}
inline D sin(const D& a) { return chain(a, std::sin(a.v), std::cos(a.v)); }
inline D cos(const D& a) { return chain(a, std::cos(a.v), -std::sin(a.v)); }
inline D atan2(const D& y, const D& x)
{
    D r(std::atan2(y.v, x.v));
    double den = x.v * x.v + y.v * y.v;
    for (int k = 0; k < NDUAL; ++k) r.g[k] = den > 0 ? (x.v * y.g[k] - y.v * x.g[k]) / den : 0.0;
    return r;
}
inline D powi(const D& a, int n)
{
    double p = std::pow(a.v, n);
    double dp = n == 0 ? 0.0 : n * std::pow(a.v, n - 1);
    return chain(a, p, dp);
}

// complex dual
struct CD {
    D re, im;
    CD() = default;
    CD(const D& r, const D& i = D(0.0)) : re(r), im(i) {}
};
inline CD operator+(const CD& a, const CD& b) { return {a.re + b.re, a.im + b.im}; }
inline CD operator-(const CD& a, const CD& b) { return {a.re - b.re, a.im - b.im}; }
inline CD operator-(const CD& a) { return {-a.re, -a.im}; }
inline CD operator*(const CD& a, const CD& b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

}  // namespace oracle
