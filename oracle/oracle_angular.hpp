// Oracle test infrastructure (not product code): a plain FP64 CPU restatement
// of the reference's covariant-tensor two-body amplitude and chain
// contraction, used only as the checker by tests and as the timed CPU baseline.
//
// Follows src/Amplitude.cu (factorial :5-98, ClebschGordan :100-144,
// associated_legendre_poly :146-199, spherical_harmonic :201-234,
// cmf_element :237-270, DFunc :272-317, wignerD_element :319-329,
// MassiveTrans :331-404, MasslessTrans :409-462, multiplyDFuncLeft :466-498,
// pwa_amp :500-644) and include/Amplitude.cuh:8-121 (LorentzVector).
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

namespace oracle {

using cplx = std::complex<double>;

struct LV {
    double E = 0, Px = 0, Py = 0, Pz = 0;
    LV() = default;
    LV(double e, double x, double y, double z) : E(e), Px(x), Py(y), Pz(z) {}
    double P() const { return std::sqrt(Px * Px + Py * Py + Pz * Pz); }
    double M2() const { return E * E - Px * Px - Py * Py - Pz * Pz; }
    double M() const
    {
        if (E * E - Px * Px - Py * Py - Pz * Pz < 0) return 0.0;
        return std::sqrt(E * E - Px * Px - Py * Py - Pz * Pz);
    }
    double Dot(const LV& o) const { return E * o.E - (Px * o.Px + Py * o.Py + Pz * o.Pz); }
    LV operator+(const LV& o) const { return LV(E + o.E, Px + o.Px, Py + o.Py, Pz + o.Pz); }
};

// n! for integer and half-integer n (Gamma(n+1)): exact up to 11.5, the
// Stirling series with two correction terms for integers >= 12, and the
// Lanczos (g = 7, 9 published terms) Gamma approximation otherwise, the
// same scheme as src/Amplitude.cu:5-98.
inline double factorial(float n)
{
    if (n < 0.0 || std::isnan(n)) return 0.0;
    double r = std::round(n);
    bool is_int = std::fabs(n - r) < 1e-10;
    bool is_half = !is_int && std::fabs(n - std::round(2.0 * n) / 2.0) < 1e-10;
    if (n >= 0.0 && n <= 11.5 && (is_int || is_half)) {
        if (is_int) {
            double f = 1.0;
            for (int i = 2; i <= (int)r; ++i) f *= i;
            return f;
        }
        return std::tgamma((double)n + 1.0);  // half-integer: Gamma(n + 1)
    }
    if (is_int && r >= 12) {
        int k = (int)r;
        double st = std::sqrt(2.0 * M_PI * k) * std::pow(k / M_E, k);
        return st * (1.0 + 1.0 / (12.0 * k) + 1.0 / (288.0 * k * k));
    }
    const double g = 7.0;
    const double c[9] = {0.99999999999980993, 676.5203681218851, -1259.1392167224028, 771.32342877765313,
                         -176.61502916214059, 12.507343278686905, -0.13857109526572012, 9.9843695780195716e-6,
                         1.5056327351493116e-7};
    double x = n - 1.0, a = c[0], t = x + g + 0.5;
    for (int i = 1; i < 9; ++i) a += c[i] / (x + i);
    return std::sqrt(2 * M_PI) * std::pow(t, x + 0.5) * std::exp(-t) * a;
}

// <j1 m1 j2 m2 | J M>, Racah formula; dims are 2j+1, m's doubled.
inline double clebsch(int dj1, int m1x2, int dj2, int m2x2, int dJ, int Mx2)
{
    float j1 = (dj1 - 1) / 2.0f, j2 = (dj2 - 1) / 2.0f, J = (dJ - 1) / 2.0f;
    float m1 = m1x2 / 2.0f, m2 = m2x2 / 2.0f, M = Mx2 / 2.0f;
    if (std::fabs(M - (m1 + m2)) > 1e-10) return 0.0;
    if (J < std::fabs(j1 - j2) || J > j1 + j2) return 0.0;
    if (std::fabs(m1) > j1 || std::fabs(m2) > j2 || std::fabs(M) > J) return 0.0;
    double t1 = std::sqrt((2.0 * J + 1.0) * factorial(j1 + j2 - J) * factorial(j1 - j2 + J) *
                          factorial(-j1 + j2 + J) / factorial(j1 + j2 + J + 1.0));
    double t2 = std::sqrt(factorial(J + M) * factorial(J - M) * factorial(j1 - m1) * factorial(j1 + m1) *
                          factorial(j2 - m2) * factorial(j2 + m2));
    int kmin = (int)std::ceil(std::fmax(0.0, std::fmax(j2 - J - m1, j1 - J + m2)));
    int kmax = (int)std::floor(std::fmin(j1 + j2 - J, std::fmin(j1 - m1, j2 + m2)));
    double sum = 0.0;
    for (int k = kmin; k <= kmax; ++k) {
        double den = factorial(k) * factorial(j1 + j2 - J - k) * factorial(j1 - m1 - k) * factorial(j2 + m2 - k) *
                     factorial(J - j2 + m1 + k) * factorial(J - j1 - m2 + k);
        if (std::fabs(den) > 1e-15) sum += ((k % 2 == 0) ? 1.0 : -1.0) / den;
    }
    return t1 * t2 * sum;
}

// P_l^m(x) with the Condon-Shortley phase, m >= 0.
inline double assocLegendre(int l, int m, double x)
{
    if (l < 0 || m < 0 || m > l) return 0.0;
    if (m == 0) {
        if (l == 0) return 1.0;
        if (l == 1) return x;
        if (l == 2) return 0.5 * (3.0 * x * x - 1.0);
        if (l == 3) return 0.5 * (5.0 * x * x * x - 3.0 * x);
        double a = 1.0, b = x, c = 0.0;
        for (int n = 2; n <= l; ++n) {
            c = ((2.0 * n - 1.0) * x * b - (n - 1.0) * a) / n;
            a = b;
            b = c;
        }
        return c;
    }
    double pmm = 1.0;
    for (int i = 1; i <= m; ++i) pmm *= (2 * i - 1) * std::sqrt(1.0 - x * x);
    pmm *= std::pow(-1.0, m);
    if (l == m) return pmm;
    double pm1 = x * (2.0 * m + 1.0) * pmm;
    if (l == m + 1) return pm1;
    double a = pmm, b = pm1, c = 0.0;
    for (int n = m + 2; n <= l; ++n) {
        c = ((2.0 * n - 1.0) * x * b - (n + m - 1.0) * a) / (n - m);
        a = b;
        b = c;
    }
    return c;
}

inline cplx sphericalY(int l, int m, double theta, double phi)
{
    if (l < 0 || std::abs(m) > l) return 0.0;
    if (l == 0 && m == 0) return 0.5 * std::sqrt(1.0 / M_PI);
    double x = std::cos(theta);
    int am = std::abs(m);
    double P = assocLegendre(l, am, x);
    double norm = std::sqrt((2.0 * l + 1.0) * factorial(l - am) / (4.0 * M_PI * factorial(l + am)));
    double phase = (m < 0 && am % 2 != 0) ? -1.0 : 1.0;
    double amp = phase * norm * P;
    return {amp * std::cos(m * phi), amp * std::sin(m * phi)};
}

// Direction and breakup momentum of p1 in the (p1+p2) rest frame.
struct CmfFrame {
    double theta, phi, q;
};
inline CmfFrame cmfFrame(const LV& p1, const LV& p2)
{
    double m1 = p1.M(), m2 = p2.M();
    double m = std::sqrt(m1 * m1 + m2 * m2 + 2 * p1.Dot(p2));
    double lamb = (2 * m * p1.E + m * m + m1 * m1 - m2 * m2) / (2 * m * (m + p1.E + p2.E));
    double qs = std::sqrt(std::pow(m, 4) + std::pow(m1 * m1 - m2 * m2, 2) - 2 * m * m * (m1 * m1 + m2 * m2)) / (2 * m);
    double nx = (p1.Px - lamb * (p1.Px + p2.Px)) / qs;
    double ny = (p1.Py - lamb * (p1.Py + p2.Py)) / qs;
    double nz = (p1.Pz - lamb * (p1.Pz + p2.Pz)) / qs;
    nz = std::fmax(-1.0, std::fmin(1.0, nz));
    return {std::acos(nz), std::atan2(ny, nx), qs};
}

inline double smallD(int dim, int m1x2, int m2x2, double beta)
{
    float j = (dim - 1) / 2.0f, m1 = m1x2 / 2.0f, m2 = m2x2 / 2.0f;
    if (std::fabs(m1) > j || std::fabs(m2) > j) return 0.0;
    double sum = 0.0;
    int kmin = (m1 < m2) ? 0 : (int)(m1 - m2);
    int kmax = (m1 > -m2) ? (int)(j - m2) : (int)(j + m1);
    for (int k = kmin; k <= kmax; ++k) {
        double num = factorial(j + m2) * factorial(j - m2) * factorial(j + m1) * factorial(j - m1);
        double den = factorial(k) * factorial(j - m2 - k) * factorial(j + m1 - k) * factorial(k - m1 + m2);
        double comb = std::sqrt(num) / den;
        double ch = std::cos(beta / 2.0), sh = std::sin(beta / 2.0);
        double ct = std::pow(ch, 2 * j + m1 - m2 - 2 * k);
        double st = std::pow(sh, 2 * k - m1 + m2);
        sum += std::pow(-1.0, k - m1 + m2) * comb * ct * st;
    }
    return sum;
}

inline cplx wignerD(int dim, int m1x2, int m2x2, double a, double b, double g)
{
    double d = smallD(dim, m1x2, m2x2, b);
    float m1 = m1x2 / 2.0f, m2 = m2x2 / 2.0f;
    return std::exp(cplx(0.0, m1 * a)) * d * std::exp(cplx(0.0, m2 * g));
}

// D-matrix [i][j] for m_i = (dim-1-2i)/2.
inline void dmatrix(std::vector<cplx>& out, int dim, double a, double b, double g)
{
    out.assign(dim * dim, 0.0);
    for (int i = 0; i < dim; ++i)
        for (int j = 0; j < dim; ++j) out[i * dim + j] = wignerD(dim, dim - 1 - 2 * i, dim - 1 - 2 * j, a, b, g);
}

inline void matmul(std::vector<cplx>& c, const std::vector<cplx>& a, const std::vector<cplx>& b, int n)
{
    c.assign(n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            cplx s = 0.0;
            for (int k = 0; k < n; ++k) s += a[i * n + k] * b[k * n + j];
            c[i * n + j] = s;
        }
}

// Wigner rotation of a massive particle q seen from P (src/Amplitude.cu:331-404).
inline void massiveTrans(std::vector<cplx>& tr, const LV& p, const LV& q, int dim)
{
    tr.assign(dim * dim, 0.0);
    for (int i = 0; i < dim; ++i) tr[i * dim + i] = 1.0;
    double Pp = p.P(), Pq = q.P();
    double hx = p.Py * q.Pz - p.Pz * q.Py, hy = p.Pz * q.Px - p.Px * q.Pz, hz = p.Px * q.Py - p.Py * q.Px;
    if (std::fabs(hx) < 1e-10 && std::fabs(hy) < 1e-10 && std::fabs(hz) < 1e-10) return;
    double m1 = p.M(), g1 = p.E / m1, m2 = q.M(), g2 = q.E / m2;
    double ca = (p.Px * q.Px + p.Py * q.Py + p.Pz * q.Pz) / (-1.0 * Pp * Pq);
    double sa = std::sqrt(1 - ca * ca);
    double nrm = std::sqrt(hx * hx + hy * hy + hz * hz);
    double th = std::acos(hz / nrm), ph = std::atan2(hy / nrm, hx / nrm);
    double num = sa * std::sqrt((g1 - 1.0) * (g2 - 1.0));
    double den = std::sqrt((g1 + 1.0) * (g2 + 1.0)) + ca * std::sqrt((g1 - 1.0) * (g2 - 1.0));
    double psi = 2.0 * std::atan2(num, den);
    std::vector<cplx> w1, w2;
    dmatrix(w1, dim, -ph, -th, -psi);
    dmatrix(w2, dim, 0.0, th, ph);
    matmul(tr, w1, w2, dim);
}

// Massless-particle transformation (src/Amplitude.cu:409-462).
inline void masslessTrans(std::vector<cplx>& tr, const LV& P, const LV& p, int dim)
{
    tr.assign(dim * dim, 0.0);
    for (int i = 0; i < dim; ++i) tr[i * dim + i] = 1.0;
    double PM = P.P();
    if (PM < 1e-10) return;
    double pm = p.P();
    if (pm < 1e-10) return;
    double n1x = -P.Px / PM, n1y = -P.Py / PM, n1z = -P.Pz / PM;
    double n2x = p.Px / pm, n2y = p.Py / pm, n2z = p.Pz / pm;
    double b1 = PM / P.E, g1 = 1.0 / std::sqrt(1.0 - b1 * b1);
    double sh1 = std::sqrt((g1 - 1.0) / 2.0), ch1 = std::sqrt((g1 + 1.0) / 2.0);
    double dot = n1x * n2x + n1y * n2y + n1z * n2z;
    double cz = n1x * n2y - n1y * n2x;
    double x12 = sh1 * (dot - n1z) + ch1 * (1.0 - n2z), y12 = sh1 * cz;
    double x22 = sh1 * (dot + n1z) + ch1 * (1.0 + n2z), y22 = -y12;
    double tot = -(std::atan2(y12, x12) + std::atan2(y22, x22));
    for (int i = 0; i < dim; ++i) {
        float m2 = (dim - 1 - 2 * i) / 2.0f;
        tr[i * dim + i] = cplx(std::cos(m2 * tot), std::sin(m2 * tot));
    }
}

inline void dLeft(std::vector<cplx>& mat, int dim, double a, double b, double g)
{
    std::vector<cplx> d, t;
    dmatrix(d, dim, a, b, g);
    matmul(t, d, mat, dim);
    mat = t;
}

// Two-body covariant amplitude tensor amp[sigma][sigma1][sigma2] (x10).
inline void pwaAmp(std::vector<cplx>& amp, const LV& p1, int dj1, const LV& p2, int dj2, int dj, int dS, int dL)
{
    int tot = dj * dj1 * dj2, kd = dj1 * dj2;
    std::vector<cplx> a(tot, 0.0);
    for (int s = 0; s < dj; ++s) {
        int sx2 = dj - 1 - 2 * s;
        for (int s1 = 0; s1 < dj1; ++s1) {
            int s1x2 = dj1 - 1 - 2 * s1;
            for (int s2 = 0; s2 < dj2; ++s2) {
                int s2x2 = dj2 - 1 - 2 * s2;
                // cmf_element (src/Amplitude.cu:237-270)
                CmfFrame fr = cmfFrame(p1, p2);
                cplx Y = sphericalY(dL, (sx2 - s1x2 - s2x2) / 2, fr.theta, -1.0 * fr.phi);
                double cg1 = clebsch(dj1, s1x2, dj2, s2x2, dS, s1x2 + s2x2);
                double cg2 = clebsch(dS, s1x2 + s2x2, 2 * dL + 1, sx2 - s1x2 - s2x2, dj, sx2);
                a[s * kd + s1 * dj2 + s2] = (std::pow(fr.q, dL) / std::sqrt((double)dj)) * cg1 * cg2 * Y;
            }
        }
    }
    CmfFrame fr = cmfFrame(p1, p2);
    LV Pt = p1 + p2;
    double m1 = p1.M(), m2 = p2.M();
    std::vector<cplx> t1, t2;
    if (m1 > 1e-10) {
        massiveTrans(t1, Pt, p1, dj1);
    } else {
        masslessTrans(t1, Pt, p1, dj1);
        dLeft(t1, dj1, -fr.phi, -fr.theta, 0.0);
    }
    if (m2 > 1e-10) {
        massiveTrans(t2, Pt, p2, dj2);
    } else {
        masslessTrans(t2, Pt, p2, dj2);
        dLeft(t2, dj2, -(M_PI + fr.phi), -(M_PI - fr.theta), 0.0);
    }
    // amp'[s][n1][n2] = sum_{o1,o2} t1[o1][n1] a[s][o1][o2] t2[o2][n2]
    amp.assign(tot, 0.0);
    std::vector<cplx> mid(kd);
    for (int s = 0; s < dj; ++s) {
        int base = s * kd;
        for (int n1 = 0; n1 < dj1; ++n1)
            for (int o2 = 0; o2 < dj2; ++o2) {
                cplx sum = 0.0;
                for (int o1 = 0; o1 < dj1; ++o1) sum += t1[n1 + dj1 * o1] * a[base + o1 * dj2 + o2];
                mid[n1 * dj2 + o2] = sum;
            }
        for (int n1 = 0; n1 < dj1; ++n1)
            for (int n2 = 0; n2 < dj2; ++n2) {
                cplx sum = 0.0;
                for (int o2 = 0; o2 < dj2; ++o2) sum += mid[n1 * dj2 + o2] * t2[n2 + dj2 * o2];
                amp[base + n1 * dj2 + n2] = sum;
            }
    }
    for (auto& x : amp) x *= 10.0;
}

}  // namespace oracle
