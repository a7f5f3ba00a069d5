// Resonance lineshapes on jets, for the fused likelihood kernel.
//
// Same mathematics as the reference lineshapes (include/ResModel.cuh:184-223
// Bf/BWR, :398-405 BW, :419-451 Flatte; src/ResModel.cu:376-588 per-call
// BWR x Bf, Flatte x Bf, GS x Bf, ONE; breakup momenta src/AmpGen.cu:2733 and
// include/ResModel.cuh:85-95) written for jets so the kernel gets values and
// exact parameter derivatives in one pass. Custom expressions compile to calls
// of the c* helpers below, with the reference interpreter's conventions
// (src/CustomExpr.cu:999-1221): |b|^2 = 0 in a division uses 1e-30, log|0|
// uses 1e-30, a^b = exp(b log a), sqrt is the principal complex root.
#pragma once

#include "jet.cuh"

// breakup momentum q(m; m1, m2), 0 below threshold
template <int N>
CT_HD Jet<N> ls_breakup(const Jet<N>& m, const Jet<N>& m1, const Jet<N>& m2)
{
    Jet<N> s = m1 + m2, dd = m1 - m2;
    Jet<N> q2 = (m * m - s * s) * (m * m - dd * dd);
    if (q2.v <= 0.0) return jc<N>(0.0);
    return jsqrt(q2) / (2.0 * m);
}

// q0 of the per-call lineshape: sqrt((m0^2-(m1+m2)^2)(m0^2-(m1-m2)^2)/(4 m0^2)), 0 below threshold
template <int N>
CT_HD Jet<N> ls_q0(const Jet<N>& m0, const Jet<N>& m1, const Jet<N>& m2)
{
    Jet<N> s = m1 + m2, dd = m1 - m2, m0s = m0 * m0;
    Jet<N> q2 = (m0s - s * s) * (m0s - dd * dd) / (4.0 * m0s);
    if (q2.v < 0.0) return jc<N>(0.0);
    return jsqrt(q2);
}

// Blatt-Weisskopf normalisation polynomial N_L(z), L <= 6
template <int N>
CT_HD Jet<N> ls_bfpoly(int L, const Jet<N>& z)
{
    Jet<N> z2 = z * z;
    switch (L) {
    case 1: return z2 + 1.0;
    case 2: return (z2 + 3.0) * z2 + 9.0;
    case 3: return ((z2 + 6.0) * z2 + 45.0) * z2 + 225.0;
    case 4: return (((z2 + 10.0) * z2 + 135.0) * z2 + 1575.0) * z2 + 11025.0;
    case 5: return ((((z2 + 15.0) * z2 + 315.0) * z2 + 6300.0) * z2 + 99225.0) * z2 + 893025.0;
    case 6: return (((((z2 + 21.0) * z2 + 630.0) * z2 + 17325.0) * z2 + 363825.0) * z2 + 6185025.0) * z2 + 540326025.0;
    default: return jc<N>(1.0);
    }
}

// Bf(L, q, q0, d) = sqrt(N_L(q0 d) / N_L(q d))
template <int N>
CT_HD Jet<N> ls_bf(int L, const Jet<N>& q, const Jet<N>& q0, double d)
{
    if (L <= 0 || L > 6) return jc<N>(1.0);
    return jsqrt(ls_bfpoly(L, q0 * d) / ls_bfpoly(L, q * d));
}

// Bf^2 without the square root (used inside the BWR running width)
template <int N>
CT_HD Jet<N> ls_bf2(int L, const Jet<N>& q, const Jet<N>& q0, double d)
{
    if (L <= 0 || L > 6) return jc<N>(1.0);
    return ls_bfpoly(L, q0 * d) / ls_bfpoly(L, q * d);
}

// relativistic Breit-Wigner with running width (width uses Lmin):
// 1 / (m0^2 - m^2 - i m0 G(m)), G = G0 (q/q0)^(2L+1) (m0/m) Bf^2
template <int N>
CT_HD CJet<N> ls_bwr(const Jet<N>& m, const Jet<N>& m0, const Jet<N>& g0, int L, const Jet<N>& q, const Jet<N>& q0,
                     double d)
{
    Jet<N> gam = g0 * jpowi(q / q0, 2 * L + 1) * (m0 / m) * ls_bf2(L, q, q0, d);
    Jet<N> x = m0 * m0 - m * m, y = m0 * gam;
    Jet<N> s = x * x + y * y;
    return cj(x / s, y / s);
}

template <int N>
CT_HD CJet<N> ls_bw(const Jet<N>& m, const Jet<N>& m0, const Jet<N>& g0)
{
    Jet<N> x = m0 * m0 - m * m, y = m0 * g0;
    Jet<N> s = x * x + y * y;
    return cj(x / s, y / s);
}

// channel phase-space factor rho (value only): csqrt(1-(ma+mb)^2/s) * sqrt(max(0, 1-(ma-mb)^2/s))
CT_HD void ls_rho(double s, double ma, double mb, double& re, double& im)
{
    double S = (ma + mb) * (ma + mb), Dd = (ma - mb) * (ma - mb);
    double f1 = 1.0 - S / s, f1r, f1i;
    if (f1 >= 0.0) {
        f1r = sqrt(f1);
        f1i = 0.0;
    } else {
        f1r = 0.0;
        f1i = sqrt(-f1);
    }
    double f2s = 1.0 - Dd / s;
    double f2 = f2s > 0.0 ? sqrt(f2s) : 0.0;
    re = f1r * f2;
    im = f1i * f2;
}

// Flatte (FlatteC convention), per-call form: F = (A - iB)/(A^2 + B^2),
// A = m0^2 - s + sum (g m0/2) Im rho, B = -sum (g m0/2) Re rho
template <int N, int NCH>
CT_HD CJet<N> ls_flatte(const Jet<N>& m, const Jet<N>& m0, const Jet<N>* g, const double* ch)
{
    Jet<N> s = m * m;
    Jet<N> A = m0 * m0, B = jc<N>(0.0), half = m0 * 0.5;
#pragma unroll
    for (int i = 0; i < NCH; ++i) {
        double rr, ri;
        ls_rho(s.v, ch[2 * i], ch[2 * i + 1], rr, ri);
        Jet<N> gw = g[i] * half;
        A = A + gw * ri;
        B = B - gw * rr;
    }
    A = A - s;
    Jet<N> den = A * A + B * B;
    return cj(A / den, -(B / den));
}

// Flatte, fixed-parameter form (include/ResModel.cuh:419-451)
template <int N, int NCH>
CT_HD CJet<N> ls_flatte_fixed(const Jet<N>& m, const Jet<N>& m0, const Jet<N>* g, const double* ch)
{
    Jet<N> s = m * m, tr = jc<N>(0.0), ti = jc<N>(0.0);
#pragma unroll
    for (int i = 0; i < NCH; ++i) {
        double rr, ri;
        ls_rho(s.v, ch[2 * i], ch[2 * i + 1], rr, ri);
        Jet<N> gw = (m0 / 2.0) * g[i];
        tr = tr + gw * rr;
        ti = ti + gw * ri;
    }
    Jet<N> dre = m0 * m0 - s + ti, dim = -tr;
    Jet<N> dsq = dre * dre + dim * dim;
    return cj(dre / dsq, -dim / dsq);
}

// Gounaris-Sakurai (rho -> pi pi), per-call form
template <int N>
CT_HD CJet<N> ls_gs(const Jet<N>& m, const Jet<N>& q, const Jet<N>& m0, const Jet<N>& g0, const Jet<N>& q0, double mpi)
{
    const double pi = 3.14159265358979323846;
    Jet<N> hm = (2.0 / pi) * ((q / m) * jlog((m + 2.0 * q) / (2.0 * mpi)));
    Jet<N> q02 = q0 * q0, q03 = q02 * q0;
    double mpi2 = mpi * mpi;
    Jet<N> la = jlog((m0 + 2.0 * q0) / (2.0 * mpi));
    Jet<N> dv = ((3.0 / pi) * (mpi2 / q02)) * la + m0 / ((2.0 * pi) * q0) - (mpi2 * m0) / (pi * q03);
    Jet<N> h0 = (2.0 / pi) * ((q0 / m0) * la);
    Jet<N> dh0 = h0 * (1.0 / (8.0 * q02) - 1.0 / (2.0 * (m0 * m0))) + 1.0 / ((2.0 * pi) * (m0 * m0));
    Jet<N> qr = q / q0;
    Jet<N> gam = (g0 * (qr * qr * qr)) * (m0 / m);
    Jet<N> f = (g0 * ((m0 * m0) / q03)) * ((q * q) * (hm - h0) + ((m0 * m0 - m * m) * q02) * dh0);
    Jet<N> num = 1.0 + (dv * g0) / m0;
    Jet<N> dre = (m0 * m0 - m * m) + f;
    Jet<N> dim = -(m0 * gam);
    Jet<N> dsq = dre * dre + dim * dim;
    return cj((num * dre) / dsq, -((num * dim) / dsq));
}

// Histogram shape (value only): aux = [m_min, m_max, nbins, values...]
CT_HD double ls_hist(double m, const double* aux)
{
    if (!(m >= 0.0)) return 0.0;
    double lo = aux[0], hi = aux[1];
    int n = (int)aux[2];
    const double* v = aux + 3;
    if (n < 2 || hi <= lo) return 0.0;
    if (m <= lo) return v[0];
    if (m >= hi) return v[n - 1];
    double x = (m - lo) / (hi - lo) * n;
    if (x < 0.0) x = 0.0;
    if (x >= (double)(n - 1)) x = (double)(n - 2);
    int i = (int)x;
    double fr = x - i;
    return v[i] * (1.0 - fr) + v[i + 1] * fr;
}

CT_HD double ls_interp1(const double* y, int i, double fr, int method, int N)
{
    if (method == 1) return y[i] + (y[i + 1] - y[i]) * fr;
    if (method == 2) {
        double y0 = (i > 0) ? y[i - 1] : y[i] - (y[i + 1] - y[i]);
        double y1 = y[i], y2 = y[i + 1];
        double y3 = (i + 2 < N) ? y[i + 2] : y[i + 1] + (y[i + 1] - y[i]);
        double f2 = fr * fr, f3 = f2 * fr;
        return 0.5 * ((2 * y1) + (-y0 + y2) * fr + (2 * y0 - 5 * y1 + 4 * y2 - y3) * f2 +
                      (-y0 + 3 * y1 - 3 * y2 + y3) * f3);
    }
    return y[i];
}

// Interpolated table (value only), aux format of the Interp model
CT_HD void ls_interp(const double* t, double x, double& Fr, double& Fi)
{
    int hdr = (int)t[0];
    int method = hdr >= 0 ? hdr : -(hdr + 1);
    int N = (int)t[1];
    int i;
    double fr;
    const double *re, *im;
    if (hdr >= 0) {
        double xmin = t[2], dx = t[3];
        re = t + 4;
        im = t + 4 + N;
        double pos = (x - xmin) / dx;
        i = (int)pos;
        if (i < 0) { i = 0; fr = 0.0; }
        else if (i >= N - 1) { i = N - 2; fr = 1.0; }
        else fr = pos - (double)i;
    } else {
        const double* xv = t + 2;
        re = t + 2 + N;
        im = t + 2 + 2 * N;
        int lo = 0, hi = N - 1;
        while (lo < hi - 1) {
            int mid = (lo + hi) / 2;
            if (x < xv[mid]) hi = mid;
            else lo = mid;
        }
        i = lo;
        if (i < 0) { i = 0; fr = 0.0; }
        else if (i >= N - 1) { i = N - 2; fr = 1.0; }
        else fr = (x - xv[i]) / (xv[i + 1] - xv[i]);
        if (method == 2) method = 0;
    }
    Fr = ls_interp1(re, i, fr, method, N);
    Fi = ls_interp1(im, i, fr, method, N);
}

// ----- complex helpers for custom expressions -----
template <int N>
CT_HD CJet<N> c_div(const CJet<N>& a, const CJet<N>& b)
{
    Jet<N> s = b.re * b.re + b.im * b.im;
    if (s.v == 0.0) s = jc<N>(1e-30);
    return cj((a.re * b.re + a.im * b.im) / s, (a.im * b.re - a.re * b.im) / s);
}
template <int N>
CT_HD CJet<N> c_exp(const CJet<N>& a)
{
    Jet<N> e = jexp(a.re);
    return cj(e * jcos(a.im), e * jsin(a.im));
}
template <int N>
CT_HD CJet<N> c_log(const CJet<N>& a)
{
    Jet<N> r = jsqrt(a.re * a.re + a.im * a.im);
    if (r.v == 0.0) r = jc<N>(1e-30);
    return cj(jlog(r), jatan2(a.im, a.re));
}
template <int N>
CT_HD CJet<N> c_pow(const CJet<N>& b, const CJet<N>& e)
{
    return c_exp(e * c_log(b));
}
template <int N>
CT_HD CJet<N> c_sqrt(const CJet<N>& a)
{
    Jet<N> r = jsqrt(a.re * a.re + a.im * a.im);
    Jet<N> re = jsqrt((r + a.re) * 0.5);
    Jet<N> im = jsqrt((r - a.re) * 0.5);
    if (a.im.v < 0.0) im = -im;
    return cj(re, im);
}
template <int N>
CT_HD CJet<N> c_sin(const CJet<N>& a)
{
    Jet<N> ep = jexp(a.im), em = jexp(-a.im);
    return cj(jsin(a.re) * (ep + em) * 0.5, jcos(a.re) * (ep - em) * 0.5);
}
template <int N>
CT_HD CJet<N> c_cos(const CJet<N>& a)
{
    Jet<N> ep = jexp(a.im), em = jexp(-a.im);
    return cj(jcos(a.re) * (ep + em) * 0.5, -(jsin(a.re) * (ep - em) * 0.5));
}
template <int N>
CT_HD CJet<N> c_abs(const CJet<N>& a)
{
    return cjr(jsqrt(a.re * a.re + a.im * a.im));
}
template <int N>
CT_HD CJet<N> c_re(const CJet<N>& a)
{
    return cjr(a.re);
}
template <int N>
CT_HD CJet<N> c_im(const CJet<N>& a)
{
    return cjr(a.im);
}
template <int N>
CT_HD CJet<N> c_conj(const CJet<N>& a)
{
    return cj(a.re, -a.im);
}
template <int N>
CT_HD CJet<N> c_rho_re(const CJet<N>& s, const CJet<N>& ma, const CJet<N>& mb)
{
    double rr, ri;
    ls_rho(s.re.v, ma.re.v, mb.re.v, rr, ri);
    return cjc<N>(rr, 0.0);
}
template <int N>
CT_HD CJet<N> c_rho_im(const CJet<N>& s, const CJet<N>& ma, const CJet<N>& mb)
{
    double rr, ri;
    ls_rho(s.re.v, ma.re.v, mb.re.v, rr, ri);
    return cjc<N>(ri, 0.0);
}
template <int N>
CT_HD CJet<N> c_q0(const CJet<N>& m0, const CJet<N>& m1, const CJet<N>& m2)
{
    return cjr(ls_q0(m0.re, m1.re, m2.re));
}
template <int N>
CT_HD CJet<N> c_bf(int L, const CJet<N>& q, const CJet<N>& q0, double d)
{
    return cjr(ls_bf(L, q.re, q0.re, d));
}
template <int N>
CT_HD CJet<N> c_bw(const CJet<N>& m, const CJet<N>& m0, const CJet<N>& g0)
{
    return ls_bw(m.re, m0.re, g0.re);
}
template <int N>
CT_HD CJet<N> c_bwr(const CJet<N>& m, const CJet<N>& m0, const CJet<N>& g0, int L, const CJet<N>& q,
                    const CJet<N>& q0, double d)
{
    return ls_bwr(m.re, m0.re, g0.re, L, q.re, q0.re, d);
}
