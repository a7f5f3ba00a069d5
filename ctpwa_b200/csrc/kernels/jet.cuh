// Forward-mode jets for lineshape parameter derivatives inside the fused
// likelihood kernel. Jet<N> carries a value and N partial derivatives with
// respect to the fitted parameters of one amplitude block; CJet<N> is the
// complex version. Compiled by NVRTC together with a generated model header,
// so it includes no system headers.
#pragma once

#define CT_HD __device__ __forceinline__

template <int N>
struct Jet {
    double v;
    double d[N > 0 ? N : 1];
};

template <int N>
CT_HD Jet<N> jc(double x)
{
    Jet<N> r;
    r.v = x;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = 0.0;
    return r;
}
template <int N>
CT_HD Jet<N> jvar(double x, int k)
{
    Jet<N> r = jc<N>(x);
    r.d[k] = 1.0;
    return r;
}
template <int N>
CT_HD Jet<N> operator+(const Jet<N>& a, const Jet<N>& b)
{
    Jet<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int N>
CT_HD Jet<N> operator-(const Jet<N>& a, const Jet<N>& b)
{
    Jet<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int N>
CT_HD Jet<N> operator-(const Jet<N>& a)
{
    Jet<N> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int N>
CT_HD Jet<N> operator*(const Jet<N>& a, const Jet<N>& b)
{
    Jet<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int N>
CT_HD Jet<N> operator/(const Jet<N>& a, const Jet<N>& b)
{
    Jet<N> r;
    double ib = 1.0 / b.v;
    r.v = a.v * ib;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
template <int N>
CT_HD Jet<N> operator+(const Jet<N>& a, double b)
{
    Jet<N> r = a;
    r.v += b;
    return r;
}
template <int N>
CT_HD Jet<N> operator+(double b, const Jet<N>& a)
{
    return a + b;
}
template <int N>
CT_HD Jet<N> operator-(const Jet<N>& a, double b)
{
    Jet<N> r = a;
    r.v -= b;
    return r;
}
template <int N>
CT_HD Jet<N> operator-(double b, const Jet<N>& a)
{
    Jet<N> r = -a;
    r.v += b;
    return r;
}
template <int N>
CT_HD Jet<N> operator*(const Jet<N>& a, double b)
{
    Jet<N> r;
    r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b;
    return r;
}
template <int N>
CT_HD Jet<N> operator*(double b, const Jet<N>& a)
{
    return a * b;
}
template <int N>
CT_HD Jet<N> operator/(const Jet<N>& a, double b)
{
    return a * (1.0 / b);
}
template <int N>
CT_HD Jet<N> operator/(double a, const Jet<N>& b)
{
    Jet<N> r;
    double ib = 1.0 / b.v;
    r.v = a * ib;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -r.v * b.d[k] * ib;
    return r;
}
template <int N>
CT_HD Jet<N> jchain(const Jet<N>& a, double f, double df)
{
    Jet<N> r;
    r.v = f;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = df * a.d[k];
    return r;
}
template <int N>
CT_HD Jet<N> jsqrt(const Jet<N>& a)
{
    double s = sqrt(a.v);
    return jchain(a, s, s > 0.0 ? 0.5 / s : 0.0);
}
template <int N>
CT_HD Jet<N> jlog(const Jet<N>& a)
{
    return jchain(a, log(a.v), 1.0 / a.v);
}
template <int N>
CT_HD Jet<N> jexp(const Jet<N>& a)
{
    double e = exp(a.v);
    return jchain(a, e, e);
}
template <int N>
CT_HD Jet<N> jsin(const Jet<N>& a)
{
    double s, c;
    sincos(a.v, &s, &c);
    return jchain(a, s, c);
}
template <int N>
CT_HD Jet<N> jcos(const Jet<N>& a)
{
    double s, c;
    sincos(a.v, &s, &c);
    return jchain(a, c, -s);
}
template <int N>
CT_HD Jet<N> jatan2(const Jet<N>& y, const Jet<N>& x)
{
    Jet<N> r;
    r.v = atan2(y.v, x.v);
    double den = x.v * x.v + y.v * y.v;
    double id = den > 0.0 ? 1.0 / den : 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = (x.v * y.d[k] - y.v * x.d[k]) * id;
    return r;
}
// integer power by repeated multiplication (n >= 0)
template <int N>
CT_HD Jet<N> jpowi(const Jet<N>& a, int n)
{
    Jet<N> r = jc<N>(1.0);
    for (int i = 0; i < n; ++i) r = r * a;
    return r;
}

template <int N>
struct CJet {
    Jet<N> re, im;
};
template <int N>
CT_HD CJet<N> cj(const Jet<N>& re, const Jet<N>& im)
{
    CJet<N> r;
    r.re = re;
    r.im = im;
    return r;
}
template <int N>
CT_HD CJet<N> cjr(const Jet<N>& re)
{
    return cj(re, jc<N>(0.0));
}
template <int N>
CT_HD CJet<N> cjc(double re, double im)
{
    return cj(jc<N>(re), jc<N>(im));
}
template <int N>
CT_HD CJet<N> operator+(const CJet<N>& a, const CJet<N>& b)
{
    return cj(a.re + b.re, a.im + b.im);
}
template <int N>
CT_HD CJet<N> operator-(const CJet<N>& a, const CJet<N>& b)
{
    return cj(a.re - b.re, a.im - b.im);
}
template <int N>
CT_HD CJet<N> operator-(const CJet<N>& a)
{
    return cj(-a.re, -a.im);
}
template <int N>
CT_HD CJet<N> operator*(const CJet<N>& a, const CJet<N>& b)
{
    return cj(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <int N>
CT_HD CJet<N> operator*(const CJet<N>& a, const Jet<N>& b)
{
    return cj(a.re * b, a.im * b);
}
template <int N>
CT_HD CJet<N> cscale(const CJet<N>& a, double b)
{
    return cj(a.re * b, a.im * b);
}
