// Likelihood engine (see engine.hpp).
//
// Per analysis (init):
//   1. config -> lowered model (model.cpp); samples read (dataio.cpp) and
//      uploaded; four-momenta transposed to SoA on the device.
//   2. ag_group_kernel: per event and angular group, the spin-orbit amplitude
//      tensors are built and contracted into SoA planes [plane][pol][event]
//      (FP64, plus an FP32 copy for the mixed path), and the per-event
//      kinematics the lineshapes need (invariant masses, breakup momenta) are
//      cached.
//   3. The model-specific fused kernel (kernels/fused_nll.cuh + generated
//      model.cuh) is compiled with NVRTC for sm_100a (cached on disk).
// Per evaluation (stream ordered, no host synchronisation, graph capturable):
//   ct_prepare (couplings) -> fused kernel (one pass over every event of every
//   sample) -> ct_finalize (deterministic reduction, loss/gradient assembly,
//   coupling-gradient transform).
#include "engine.hpp"

#include "angular.cuh"

#include <dlfcn.h>
#include <nvrtc.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <map>
#include <memory>
#include <mutex>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace ctpwa {

#define CT_CUDA(x)                                                                                    \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess)                                                                        \
            throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " + \
                                     __FILE__ + ":" + std::to_string(__LINE__));                      \
    } while (0)

// ============================================================================
// Host tables: Clebsch-Gordan products, Y_lm norms, Wigner small-d sums.
// The factorial uses the same scheme as the reference (exact up to 11.5,
// Stirling with two corrections for integers >= 12, Lanczos otherwise;
// src/Amplitude.cu:5-98) so that high-spin coefficients agree with it.
// ============================================================================
namespace {

double refFactorial(float n)
{
    if (n < 0.0f || std::isnan(n)) return 0.0;
    double r = std::round(n);
    bool is_int = std::fabs(n - r) < 1e-10;
    bool is_half = !is_int && std::fabs(n - std::round(2.0 * n) / 2.0) < 1e-10;
    if (n <= 11.5f && (is_int || is_half)) {
        if (is_int) {
            double f = 1.0;
            for (int i = 2; i <= (int)r; ++i) f *= i;
            return f;
        }
        return std::tgamma((double)n + 1.0);
    }
    if (is_int && r >= 12) {
        int k = (int)r;
        return std::sqrt(2.0 * M_PI * k) * std::pow(k / M_E, k) * (1.0 + 1.0 / (12.0 * k) + 1.0 / (288.0 * k * k));
    }
    // Lanczos approximation (g = 7, 9 published coefficients) of Gamma(n + 1)
    const double g = 7.0;
    const double c[9] = {0.99999999999980993, 676.5203681218851,   -1259.1392167224028,
                         771.32342877765313,  -176.61502916214059, 12.507343278686905,
                         -0.13857109526572012, 9.9843695780195716e-6, 1.5056327351493116e-7};
    double x = n - 1.0, a = c[0], t = x + g + 0.5;
    for (int i = 1; i < 9; ++i) a += c[i] / (x + i);
    return std::sqrt(2 * M_PI) * std::pow(t, x + 0.5) * std::exp(-t) * a;
}

// Racah formula for <j1 m1 j2 m2 | J M> (dims 2j+1, m doubled)
double clebschGordan(int dj1, int m1x2, int dj2, int m2x2, int dJ, int Mx2)
{
    float j1 = (dj1 - 1) / 2.0f, j2 = (dj2 - 1) / 2.0f, J = (dJ - 1) / 2.0f;
    float m1 = m1x2 / 2.0f, m2 = m2x2 / 2.0f, M = Mx2 / 2.0f;
    if (std::fabs(M - (m1 + m2)) > 1e-10) return 0.0;
    if (J < std::fabs(j1 - j2) || J > j1 + j2) return 0.0;
    if (std::fabs(m1) > j1 || std::fabs(m2) > j2 || std::fabs(M) > J) return 0.0;
    double a = std::sqrt((2.0 * J + 1.0) * refFactorial(j1 + j2 - J) * refFactorial(j1 - j2 + J) *
                         refFactorial(-j1 + j2 + J) / refFactorial(j1 + j2 + J + 1.0f));
    double b = std::sqrt(refFactorial(J + M) * refFactorial(J - M) * refFactorial(j1 - m1) * refFactorial(j1 + m1) *
                         refFactorial(j2 - m2) * refFactorial(j2 + m2));
    int kmin = (int)std::ceil(std::fmax(0.0, std::fmax(j2 - J - m1, j1 - J + m2)));
    int kmax = (int)std::floor(std::fmin(j1 + j2 - J, std::fmin(j1 - m1, j2 + m2)));
    double sum = 0.0;
    for (int k = kmin; k <= kmax; ++k) {
        double den = refFactorial((float)k) * refFactorial(j1 + j2 - J - k) * refFactorial(j1 - m1 - k) *
                     refFactorial(j2 + m2 - k) * refFactorial(J - j2 + m1 + k) * refFactorial(J - j1 - m2 + k);
        if (std::fabs(den) > 1e-15) sum += ((k % 2 == 0) ? 1.0 : -1.0) / den;
    }
    return a * b * sum;
}

}  // namespace

// ============================================================================
// Device: angular tensors
// ============================================================================
struct V4 {
    double E, x, y, z;
};

__device__ __forceinline__ V4 v4add(const V4& a, const V4& b) { return {a.E + b.E, a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ double v4mass(const V4& p)
{
    double m2 = p.E * p.E - p.x * p.x - p.y * p.y - p.z * p.z;
    return m2 < 0 ? 0.0 : sqrt(m2);
}
__device__ __forceinline__ double v4p(const V4& p) { return sqrt(p.x * p.x + p.y * p.y + p.z * p.z); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

// polar angles and breakup momentum of p1 in the (p1+p2) rest frame
__device__ void agFrame(const V4& p1, const V4& p2, double& theta, double& phi, double& q)
{
    double m1 = v4mass(p1), m2 = v4mass(p2);
    double dot = p1.E * p2.E - (p1.x * p2.x + p1.y * p2.y + p1.z * p2.z);
    double m = sqrt(m1 * m1 + m2 * m2 + 2 * dot);
    double lamb = (2 * m * p1.E + m * m + m1 * m1 - m2 * m2) / (2 * m * (m + p1.E + p2.E));
    double dm = m1 * m1 - m2 * m2;
    q = sqrt(m * m * m * m + dm * dm - 2 * m * m * (m1 * m1 + m2 * m2)) / (2 * m);
    double nx = (p1.x - lamb * (p1.x + p2.x)) / q;
    double ny = (p1.y - lamb * (p1.y + p2.y)) / q;
    double nz = (p1.z - lamb * (p1.z + p2.z)) / q;
    nz = fmax(-1.0, fmin(1.0, nz));
    theta = acos(nz);
    phi = atan2(ny, nx);
}

// associated Legendre P_l^m(x), m >= 0, Condon-Shortley phase
__device__ double agLegendre(int l, int m, double x)
{
    if (m == 0) {
        if (l == 0) return 1.0;
        if (l == 1) return x;
        if (l == 2) return 0.5 * (3.0 * x * x - 1.0);
        if (l == 3) return 0.5 * (5.0 * x * x * x - 3.0 * x);
        double a = 1.0, b = x, c = 0.0;
        for (int k = 2; k <= l; ++k) {
            c = ((2.0 * k - 1.0) * x * b - (k - 1.0) * a) / k;
            a = b;
            b = c;
        }
        return c;
    }
    double s = sqrt(1.0 - x * x), pmm = 1.0;
    for (int i = 1; i <= m; ++i) pmm *= (2 * i - 1) * s;
    if (m & 1) pmm = -pmm;
    if (l == m) return pmm;
    double pm1 = x * (2.0 * m + 1.0) * pmm;
    if (l == m + 1) return pm1;
    double a = pmm, b = pm1, c = 0.0;
    for (int k = m + 2; k <= l; ++k) {
        c = ((2.0 * k - 1.0) * x * b - (k + m - 1.0) * a) / (k - m);
        a = b;
        b = c;
    }
    return c;
}

__device__ __forceinline__ double ipow(double x, int n)
{
    double r = 1.0;
    for (int i = 0; i < n; ++i) r *= x;
    return r;
}

// d^j_{m1 m2}(beta) from tabulated sum coefficients [count, (c, a, b)...]
__device__ double agSmallD(const AgTables& T, int dim, int i1, int i2, double beta)
{
    const double* t = T.dcoef + T.doff[(dim * AG_MAXD + i1) * AG_MAXD + i2];
    int cnt = (int)t[0];
    double ch = cos(beta / 2.0), sh = sin(beta / 2.0), s = 0.0;
    for (int k = 0; k < cnt; ++k) s += t[1 + 3 * k] * ipow(ch, (int)t[2 + 3 * k]) * ipow(sh, (int)t[3 + 3 * k]);
    return s;
}

// D-matrix element e^{i m1 a} d(b) e^{i m2 g}, m = (dim - 1 - 2 i) / 2
__device__ void agDMatrix(const AgTables& T, int dim, double a, double b, double g, double2* out)
{
    for (int i = 0; i < dim; ++i) {
        double m1 = (dim - 1 - 2 * i) / 2.0;
        for (int j = 0; j < dim; ++j) {
            double m2 = (dim - 1 - 2 * j) / 2.0;
            double d = agSmallD(T, dim, i, j, b);
            double s1, c1, s2, c2;
            sincos(m1 * a, &s1, &c1);
            sincos(m2 * g, &s2, &c2);
            out[i * dim + j] = cmul(make_double2(c1 * d, s1 * d), make_double2(c2, s2));
        }
    }
}

__device__ void agMatMul(const double2* a, const double2* b, double2* c, int n)
{
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double2 s = make_double2(0, 0);
            for (int k = 0; k < n; ++k) s = cadd(s, cmul(a[i * n + k], b[k * n + j]));
            c[i * n + j] = s;
        }
}

// Wigner rotation of a massive particle q as seen from P (reference MassiveTrans)
__device__ __noinline__ void agMassive(const AgTables& T, const V4& P, const V4& q, int dim, double2* tr)
{
    for (int i = 0; i < dim * dim; ++i) tr[i] = make_double2(0, 0);
    for (int i = 0; i < dim; ++i) tr[i * dim + i] = make_double2(1, 0);
    double hx = P.y * q.z - P.z * q.y, hy = P.z * q.x - P.x * q.z, hz = P.x * q.y - P.y * q.x;
    if (fabs(hx) < 1e-10 && fabs(hy) < 1e-10 && fabs(hz) < 1e-10) return;
    double Pp = v4p(P), Pq = v4p(q);
    double g1 = P.E / v4mass(P), g2 = q.E / v4mass(q);
    double ca = (P.x * q.x + P.y * q.y + P.z * q.z) / (-1.0 * Pp * Pq);
    double sa = sqrt(1 - ca * ca);
    double nrm = sqrt(hx * hx + hy * hy + hz * hz);
    double th = acos(hz / nrm), ph = atan2(hy / nrm, hx / nrm);
    double psi = 2.0 * atan2(sa * sqrt((g1 - 1.0) * (g2 - 1.0)),
                             sqrt((g1 + 1.0) * (g2 + 1.0)) + ca * sqrt((g1 - 1.0) * (g2 - 1.0)));
    double2 w1[AG_MAXD * AG_MAXD], w2[AG_MAXD * AG_MAXD];
    agDMatrix(T, dim, -ph, -th, -psi, w1);
    agDMatrix(T, dim, 0.0, th, ph, w2);
    agMatMul(w1, w2, tr, dim);
}

// massless-particle phase rotation (reference MasslessTrans)
__device__ __noinline__ void agMassless(const V4& P, const V4& p, int dim, double2* tr)
{
    for (int i = 0; i < dim * dim; ++i) tr[i] = make_double2(0, 0);
    for (int i = 0; i < dim; ++i) tr[i * dim + i] = make_double2(1, 0);
    double PM = v4p(P);
    if (PM < 1e-10) return;
    double pm = v4p(p);
    if (pm < 1e-10) return;
    double n1x = -P.x / PM, n1y = -P.y / PM, n1z = -P.z / PM;
    double n2x = p.x / pm, n2y = p.y / pm, n2z = p.z / pm;
    double b1 = PM / P.E, g1 = 1.0 / sqrt(1.0 - b1 * b1);
    double sh1 = sqrt((g1 - 1.0) / 2.0), ch1 = sqrt((g1 + 1.0) / 2.0);
    double dot = n1x * n2x + n1y * n2y + n1z * n2z, cz = n1x * n2y - n1y * n2x;
    double x12 = sh1 * (dot - n1z) + ch1 * (1.0 - n2z), y12 = sh1 * cz;
    double x22 = sh1 * (dot + n1z) + ch1 * (1.0 + n2z), y22 = -y12;
    double tot = -(atan2(y12, x12) + atan2(y22, x22));
    for (int i = 0; i < dim; ++i) {
        double m2 = (dim - 1 - 2 * i) / 2.0, s, c;
        sincos(m2 * tot, &s, &c);
        tr[i * dim + i] = make_double2(c, s);
    }
}

__device__ __noinline__ void agDLeft(const AgTables& T, double2* mat, int dim, double a, double b, double g)
{
    double2 d[AG_MAXD * AG_MAXD], t[AG_MAXD * AG_MAXD];
    agDMatrix(T, dim, a, b, g, d);
    agMatMul(d, mat, t, dim);
    for (int i = 0; i < dim * dim; ++i) mat[i] = t[i];
}

// one decay vertex: amp[s][s1][s2] (x10), reference pwa_amp semantics
__device__ __noinline__ void agVertex(const AgTables& T, const AgNodeVar& var, const V4& p1, int dj1, const V4& p2, int dj2, int dj,
                         const double* ylm_norm, double2* amp)
{
    double theta, phi, q;
    agFrame(p1, p2, theta, phi, q);
    const int L = var.L;
    const double ql = ipow(q, L);
    const double x = cos(theta);
    const double* cg = T.cg + var.cg_off;
    const int kd = dj1 * dj2;
    for (int s = 0; s < dj; ++s) {
        int sx2 = dj - 1 - 2 * s;
        for (int s1 = 0; s1 < dj1; ++s1) {
            int s1x2 = dj1 - 1 - 2 * s1;
            for (int s2 = 0; s2 < dj2; ++s2) {
                int s2x2 = dj2 - 1 - 2 * s2;
                double c = cg[s * kd + s1 * dj2 + s2];
                double2 y = make_double2(0, 0);
                int m = (sx2 - s1x2 - s2x2) / 2;
                int am = m < 0 ? -m : m;
                if (c != 0.0 && am <= L) {
                    double P = agLegendre(L, am, x);
                    double a = ylm_norm[L * AG_MAXD + am] * P;
                    if (m < 0 && (am & 1)) a = -a;
                    double sn, cs;
                    sincos(m * (-phi), &sn, &cs);
                    y = make_double2(a * cs, a * sn);
                }
                amp[s * kd + s1 * dj2 + s2] = make_double2(ql * c * y.x, ql * c * y.y);
            }
        }
    }
    // daughters' Wigner rotations
    V4 Pt = v4add(p1, p2);
    double2 t1[AG_MAXD * AG_MAXD], t2[AG_MAXD * AG_MAXD];
    if (v4mass(p1) > 1e-10) agMassive(T, Pt, p1, dj1, t1);
    else {
        agMassless(Pt, p1, dj1, t1);
        agDLeft(T, t1, dj1, -phi, -theta, 0.0);
    }
    if (v4mass(p2) > 1e-10) agMassive(T, Pt, p2, dj2, t2);
    else {
        agMassless(Pt, p2, dj2, t2);
        agDLeft(T, t2, dj2, -(M_PI + phi), -(M_PI - theta), 0.0);
    }
    bool trivial = (dj1 == 1 && dj2 == 1);
    if (!trivial) {
        double2 mid[AG_MAXT];
        for (int s = 0; s < dj; ++s) {
            double2* a = amp + s * kd;
            for (int n1 = 0; n1 < dj1; ++n1)
                for (int o2 = 0; o2 < dj2; ++o2) {
                    double2 sum = make_double2(0, 0);
                    for (int o1 = 0; o1 < dj1; ++o1) sum = cadd(sum, cmul(t1[n1 + dj1 * o1], a[o1 * dj2 + o2]));
                    mid[n1 * dj2 + o2] = sum;
                }
            for (int n1 = 0; n1 < dj1; ++n1)
                for (int n2 = 0; n2 < dj2; ++n2) {
                    double2 sum = make_double2(0, 0);
                    for (int o2 = 0; o2 < dj2; ++o2) sum = cadd(sum, cmul(mid[n1 * dj2 + o2], t2[n2 + dj2 * o2]));
                    a[n1 * dj2 + n2] = sum;
                }
        }
    } else {
        double2 r = cmul(t1[0], t2[0]);
        if (r.x != 1.0 || r.y != 0.0)
            for (int s = 0; s < dj; ++s) amp[s] = cmul(r, amp[s]);
    }
    for (int i = 0; i < dj * kd; ++i) amp[i] = make_double2(amp[i].x * 10.0, amp[i].y * 10.0);
}

__global__ void ag_transpose_kernel(const double* __restrict__ aos, double* __restrict__ soa, long long n, int nfin)
{
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    for (int k = 0; k < nfin * 4; ++k) soa[(long long)k * n + e] = aos[e * nfin * 4 + k];
}

__global__ void __launch_bounds__(128) ag_group_kernel(AgGroup G, AgTables T, const double* __restrict__ p4, long long n,
                                                       long long ld,
                                                       double2* __restrict__ out64, float2* __restrict__ out32,
                                                       double* __restrict__ kin)
{
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    V4 mom[AG_MAXP];
    V4 parent = {0, 0, 0, 0};
    for (int f = 0; f < G.nfin; ++f) {
        V4 pf = {p4[(long long)(4 * f) * n + e], p4[(long long)(4 * f + 1) * n + e], p4[(long long)(4 * f + 2) * n + e],
                 p4[(long long)(4 * f + 3) * n + e]};
        parent = v4add(parent, pf);
    }
    for (int k = 0; k < G.np; ++k) {
        int idx = G.build_order[k];
        int s = G.input_slot[idx];
        if (s >= 0)
            mom[idx] = {p4[(long long)(4 * s) * n + e], p4[(long long)(4 * s + 1) * n + e], p4[(long long)(4 * s + 2) * n + e],
                        p4[(long long)(4 * s + 3) * n + e]};
        else if (s == -1) mom[idx] = parent;
        else mom[idx] = v4add(mom[G.sum_a[idx]], mom[G.sum_b[idx]]);
    }
    // kinematic cache
    for (int k = 0; k < G.nkin; ++k) {
        const int* d = G.kin + 5 * k;
        const V4& a = mom[d[1]];
        double val = 0.0;
        switch (d[0]) {
        case AG_K_MASS: val = v4mass(a); break;
        case AG_K_Q: {
            double m = v4mass(a), m1 = v4mass(mom[d[2]]), m2 = v4mass(mom[d[3]]);
            double q2 = (m * m - (m1 + m2) * (m1 + m2)) * (m * m - (m1 - m2) * (m1 - m2));
            val = q2 <= 0.0 ? 0.0 : sqrt(q2) / (2.0 * m);
            break;
        }
        case AG_K_QRAW: {
            double m = v4mass(a), m1 = v4mass(mom[d[2]]), m2 = v4mass(mom[d[3]]);
            val = sqrt((m * m - (m1 + m2) * (m1 + m2)) * (m * m - (m1 - m2) * (m1 - m2))) / 2 / m;
            break;
        }
        case AG_K_P: val = v4p(a); break;
        case AG_K_E: val = a.E; break;
        case AG_K_CT: {
            double pp = v4p(a);
            val = pp > 0 ? a.z / pp : 0.0;
            break;
        }
        case AG_K_PHI: val = atan2(a.y, a.x); break;
        }
        kin[(long long)d[4] * ld + e] = val;
    }
    // spin-orbit tensors and chain contraction
    double2 cur[AG_MAXT], nxt[AG_MAXT], node[AG_MAXT];
    int shape[AG_MAXN + 2], labels[AG_MAXN + 2];
    for (int s = 0; s < G.nsl; ++s) {
        int rank = 0;
        for (int ni = 0; ni < G.nnodes; ++ni) {
            const AgNode& nd = G.nodes[ni];
            const AgNodeVar& var = T.vars[nd.var_off + G.sl_var[s * G.nnodes + ni]];
            agVertex(T, var, mom[nd.d1], nd.dj1, mom[nd.d2], nd.dj2, nd.dj, T.ylm_norm, ni == 0 ? cur : node);
            if (ni == 0) {
                shape[0] = nd.dj;
                shape[1] = nd.dj1;
                shape[2] = nd.dj2;
                labels[0] = nd.mother;
                labels[1] = nd.d1;
                labels[2] = nd.d2;
                rank = 3;
                continue;
            }
            int c = 0;
            for (int j = 0; j < rank; ++j)
                if (labels[j] == nd.mother) {
                    c = j;
                    break;
                }
            // strides of cur
            int st[AG_MAXN + 2];
            st[rank - 1] = 1;
            for (int j = rank - 2; j >= 0; --j) st[j] = st[j + 1] * shape[j + 1];
            int oshape[AG_MAXN + 2], ro = 0;
            for (int j = 0; j < rank; ++j)
                if (j != c) oshape[ro++] = shape[j];
            oshape[ro++] = nd.dj1;
            oshape[ro++] = nd.dj2;
            int total = 1;
            for (int j = 0; j < ro; ++j) total *= oshape[j];
            for (int idx = 0; idx < total; ++idx) {
                int t = idx, ic[AG_MAXN + 2];
                for (int j = ro - 1; j >= 0; --j) {
                    ic[j] = t % oshape[j];
                    t /= oshape[j];
                }
                int base = 0, pos = 0;
                for (int j = 0; j < rank; ++j)
                    if (j != c) base += ic[pos++] * st[j];
                int e1 = ic[ro - 2], e2 = ic[ro - 1];
                double2 sum = make_double2(0, 0);
                for (int sg = 0; sg < shape[c]; ++sg)
                    sum = cadd(sum, cmul(cur[base + sg * st[c]], node[(sg * nd.dj1 + e1) * nd.dj2 + e2]));
                nxt[idx] = sum;
            }
            for (int i = 0; i < total; ++i) cur[i] = nxt[i];
            for (int j = 0; j < ro; ++j) shape[j] = oshape[j];
            for (int j = c; j < rank - 1; ++j) labels[j] = labels[j + 1];
            labels[rank - 1] = nd.d1;
            labels[rank] = nd.d2;
            rank = ro;
        }
        const long long plane = (long long)(G.plane0 + s) * G.npol;
        for (int p = 0; p < G.npol; ++p) {
            double2 v = G.pol_map ? cur[G.pol_map[p]] : cur[p];
            out64[(plane + p) * ld + e] = v;
            if (out32) out32[(plane + p) * ld + e] = make_float2((float)v.x, (float)v.y);
        }
    }
}

// ============================================================================
// Device: per-evaluation prologue / epilogue
// ============================================================================

// v[a] = ratio[a] * p[chain[a]], params = [Re p (nc), Im p (nc), theta]
// err (may be null): the evaluation's error flag, cleared here because this
// kernel is the first of every evaluation, so a flag raised by one evaluation
// (a staged table copy that did not arrive) does not stick to later ones.
__global__ void ct_prepare_kernel(const double* __restrict__ params, const int* __restrict__ chain,
                                  const double* __restrict__ ratio, int nA, int nc, double* __restrict__ v,
                                  int* __restrict__ err)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a == 0 && err) *err = 0;
    if (a >= nA) return;
    int c = chain[a];
    v[2 * a] = params[c] * ratio[a];
    v[2 * a + 1] = params[nc + c] * ratio[a];
}

// one block per job of a multi-job evaluation: ct_prepare_kernel's work
struct PrepareArgs {
    const double* params;
    const int* chain;
    const double* ratio;
    int nA, nc;
    double* v;
    int* err;
};
__global__ void ct_prepare_multi_kernel(const PrepareArgs* __restrict__ ps)
{
    const PrepareArgs& P = ps[blockIdx.x];
    if (threadIdx.x == 0 && P.err) *P.err = 0;
    for (int a = threadIdx.x; a < P.nA; a += blockDim.x) {
        const int c = P.chain[a];
        P.v[2 * a] = P.params[c] * P.ratio[a];
        P.v[2 * a + 1] = P.params[P.nc + c] * P.ratio[a];
    }
}

struct FinalizeArgs {
    const double* partials;
    int nacc, nA, nc, nT;
    int cta[3][2];  // per sample kind: begin, count
    int has[3];
    double n_phsp, W_data, W_bkg;
    const double* params;
    const double* v;
    const int* chain;
    const int* gauss_idx;
    const double* gauss_ms;
    int ngauss;
    double* out_nll;
    double* out_grad;
    double* out_parts;
    // event-sharded mode: summed per-sample sums [3][nacc] + [n_phsp, W_phsp,
    // W_data, W_bkg] replace the partial rows and the sample totals; the
    // phase-space coupling-gradient sums are then divided by W_phsp here
    const double* sums;
    // set when a fused kernel's staged copy did not arrive: the evaluation is
    // invalid and reported like a non-finite NLL (loss 1e30, zero gradient)
    const int* err;
    // 1 for sums of the mixed form, which evaluates at the couplings rounded
    // to FP32 (v_h): the loss gets the first-order term of v - v_h
    int vshift;
    // cached normalisation: the phase-space row of sums (ct_norm_row)
    // replaces the phase-space CTAs' partial rows
    const double* phsp_row;
};

// Per-sample sums of the partial rows plus the sample totals (event-sharded
// evaluation); the same fixed-order reduction as ct_finalize_kernel (each
// row read by one warp, the warps' sums added in warp order; launched with
// 1024 threads and [32][nacc] doubles of dynamic shared memory), so a
// sharded evaluation on one shard reproduces the unsharded sums bit for bit.
__global__ void __launch_bounds__(1024) ct_rowsum_kernel(const double* __restrict__ partials, int nacc, FinalizeArgs A,
                                                         double W_phsp, double* __restrict__ out)
{
    extern __shared__ double wsum[];  // [nwarp][nacc]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int k = 0; k < 3; ++k) {
        for (int j0 = 0; j0 < nacc; j0 += 32) {
            const int j = j0 + lane;
            if (j >= nacc) continue;
            double s = 0.0;
            if (A.has[k]) {
                const double* rows = partials + (long long)A.cta[k][0] * nacc + j;
#pragma unroll 4
                for (int b = warp; b < A.cta[k][1]; b += nwarp) s += rows[(long long)b * nacc];
            }
            wsum[warp * nacc + j] = s;
        }
        __syncthreads();
        for (int j = threadIdx.x; j < nacc; j += blockDim.x) {
            double s = 0.0;
            for (int w = 0; w < nwarp; ++w) s += wsum[w * nacc + j];
            out[k * nacc + j] = s;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[3 * nacc + 0] = A.n_phsp;
        out[3 * nacc + 1] = W_phsp;
        out[3 * nacc + 2] = A.W_data;
        out[3 * nacc + 3] = A.W_bkg;
    }
}

// One CTA: deterministic column sums of the CTA partials, then loss/gradient
// assembly (src/Analysis.cu:1134-1183) and the coupling-gradient transform
// dL/dp_c = (1/p_c) sum_{a in c} conj(g_a) v_a (src/AmpGen.cu:3581-3637).
__device__ __forceinline__ void ct_finalize_body(const FinalizeArgs& A)
{
    // [3][nacc] sample sums, gv [2 nA] (+ 8 spare), then the inputs of the
    // serial assembly staged by all threads (thread 0 reads no global
    // memory): couplings [2 nA], parameters [2 nc + nT], coupling chain
    // [nA], Gaussian constraints [3 ngauss]; then the per-warp sums of the
    // row reduction [32][nacc] (ct_finalize_shm)
    extern __shared__ double sh[];
    double* sums = sh;
    double* sv = sh + 3 * A.nacc + 2 * A.nA + 8;
    double* sp = sv + 2 * A.nA;
    double* sch = sp + 2 * A.nc + A.nT;
    double* sg = sch + A.nA;
    for (int i = threadIdx.x; i < 2 * A.nA; i += blockDim.x) sv[i] = A.v[i];
    for (int i = threadIdx.x; i < 2 * A.nc + A.nT; i += blockDim.x) sp[i] = A.params[i];
    for (int i = threadIdx.x; i < A.nA; i += blockDim.x) sch[i] = (double)A.chain[i];
    for (int i = threadIdx.x; i < A.ngauss; i += blockDim.x) {
        sg[3 * i] = (double)A.gauss_idx[i];
        sg[3 * i + 1] = A.gauss_ms[2 * i];
        sg[3 * i + 2] = A.gauss_ms[2 * i + 1];
    }
    // one warp per (sample, column): lanes stride over the CTA rows, then a
    // fixed-order shuffle tree, so the sums are bit-reproducible
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    double n_phsp = A.n_phsp, W_data = A.W_data, W_bkg = A.W_bkg, gv_phsp_scale = 1.0;
    if (A.sums) {
        for (int i = threadIdx.x; i < 3 * A.nacc; i += blockDim.x) sums[i] = A.sums[i];
        n_phsp = A.sums[3 * A.nacc + 0];
        const double Wp = A.sums[3 * A.nacc + 1];
        gv_phsp_scale = 1.0 / (Wp > 0 ? Wp : 1.0);
        W_data = A.sums[3 * A.nacc + 2];
        W_bkg = A.sums[3 * A.nacc + 3];
    } else {
        // per sample: warp w sums rows w, w + nwarp, ... of the sample's CTA
        // rows (each row read by one warp, lanes over its columns:
        // coalesced), then one thread per column adds the warps' sums in
        // warp order, so the sums are bit-reproducible
        double* wsum = sg + 3 * A.ngauss;  // [nwarp][nacc]
        for (int k = 0; k < 3; ++k) {
            if (k == 0 && A.phsp_row) {
                for (int j = threadIdx.x; j < A.nacc; j += blockDim.x) sums[j] = A.phsp_row[j];
                continue;
            }
            for (int j0 = 0; j0 < A.nacc; j0 += 32) {
                const int j = j0 + lane;
                if (j >= A.nacc) continue;
                double s = 0.0;
                if (A.has[k]) {
                    const double* rows = A.partials + (long long)A.cta[k][0] * A.nacc + j;
#pragma unroll 4
                    for (int b = warp; b < A.cta[k][1]; b += nwarp) s += rows[(long long)b * A.nacc];
                }
                wsum[warp * A.nacc + j] = s;
            }
            __syncthreads();
            for (int j = threadIdx.x; j < A.nacc; j += blockDim.x) {
                double s = 0.0;
                for (int w = 0; w < nwarp; ++w) s += wsum[w * A.nacc + j];
                sums[k * A.nacc + j] = s;
            }
            __syncthreads();
        }
    }
    __syncthreads();
    // loss and gradient assembly, spread over threads: thread 0 the loss,
    // threads a < nA the coupling sums g_a, then one thread per parameter
    const double* P = sums;               // phase space
    const double* Dd = sums + A.nacc;     // data
    const double* B = sums + 2 * A.nacc;  // background
    double* gv = sums + 3 * A.nacc;
    double* scal = gv + 2 * A.nA;         // pf, W_eff, loss, reset (4 of the 8 spare)
    const double* theta = sp + 2 * A.nc;
    if (threadIdx.x == 0) {
        double pf = n_phsp > 0 ? P[1] / n_phsp : 0.0;
        if (pf <= 1e-30 || isnan(pf) || isinf(pf)) pf = 1e-30;
        const double Weff = W_data - W_bkg;
        double loss = Dd[0] - B[0] + Weff * log(pf);
        if (A.err && *A.err) loss = nan("");
        for (int g = 0; g < A.ngauss; ++g) {
            double dl = theta[(int)sg[3 * g]] - sg[3 * g + 1];
            loss += dl * dl / (2.0 * sg[3 * g + 2] * sg[3 * g + 2]);
        }
        const bool reset = isnan(loss) || isinf(loss);
        scal[0] = pf;
        scal[1] = Weff;
        scal[2] = reset ? 1e30 : loss;
        scal[3] = reset ? 1.0 : 0.0;
    }
    __syncthreads();
    const double pf = scal[0], Weff = scal[1];
    const bool reset = scal[3] != 0.0;
    for (int a = threadIdx.x; a < A.nA; a += blockDim.x) {
        double r = Dd[2 + 2 * a] - B[2 + 2 * a] + (Weff / pf) * (P[2 + 2 * a] * gv_phsp_scale);
        double i = Dd[3 + 2 * a] - B[3 + 2 * a] + (Weff / pf) * (P[3 + 2 * a] * gv_phsp_scale);
        gv[2 * a] = reset ? 0.0 : r;
        gv[2 * a + 1] = reset ? 0.0 : i;
    }
    __syncthreads();
    const int t = threadIdx.x;
    if (t == 0) {
        double loss = scal[2];
        if (A.vshift && !reset) {
            // the mixed form's sums are at v_h = FP32(v): add dL/dRe v . (v - v_h)
            // + dL/dIm v . (v - v_h) with dL/dRe v_a = 2 Re g_a, dL/dIm v_a = 2 Im g_a
            double corr = 0.0;
            for (int a = 0; a < A.nA; ++a) {
                const double vr = sv[2 * a], vi = sv[2 * a + 1];
                corr += 2.0 * (gv[2 * a] * (vr - (double)(float)vr) + gv[2 * a + 1] * (vi - (double)(float)vi));
            }
            loss += corr;
        }
        *A.out_nll = loss;
        if (A.out_parts) {
            A.out_parts[0] = Dd[0];
            A.out_parts[1] = B[0];
            A.out_parts[2] = P[1];
            A.out_parts[3] = W_data;
            A.out_parts[4] = W_bkg;
            A.out_parts[5] = n_phsp;
        }
    }
    // the other warps: one parameter each (couplings, then resonance parameters)
    if (t >= 32)
        for (int u = t - 32; u < A.nc + A.nT; u += (int)blockDim.x - 32) {
            if (u < A.nc) {
                const int c = u;
                double sr = 0.0, si = 0.0;
                for (int a = 0; a < A.nA; ++a) {
                    if ((int)sch[a] != c) continue;
                    double gr = gv[2 * a], gi = gv[2 * a + 1], vr = sv[2 * a], vi = sv[2 * a + 1];
                    sr += gr * vr + gi * vi;
                    si += gr * vi - gi * vr;
                }
                double pr = sp[c], pi = sp[A.nc + c];
                double ps = pr * pr + pi * pi;
                if (ps < 1e-30) ps = 1e-30;
                A.out_grad[c] = 2.0 * (sr * pr + si * pi) / ps;
                A.out_grad[A.nc + c] = -2.0 * (si * pr - sr * pi) / ps;
            } else {
                const int j = u - A.nc;
                double g = Dd[2 + 2 * A.nA + j] - B[2 + 2 * A.nA + j] + (Weff / (pf * n_phsp)) * P[2 + 2 * A.nA + j];
                if (reset) g = 0.0;
                else
                    for (int q = 0; q < A.ngauss; ++q)
                        if ((int)sg[3 * q] == j) g += (theta[j] - sg[3 * q + 1]) / (sg[3 * q + 2] * sg[3 * q + 2]);
                A.out_grad[2 * A.nc + j] = g;
            }
        }
}

__global__ void __launch_bounds__(1024) ct_finalize_kernel(FinalizeArgs A) { ct_finalize_body(A); }

// dynamic shared memory of a finalize launch (layout in ct_finalize_body)
size_t ct_finalize_shm(const FinalizeArgs& f)
{
    return sizeof(double) * (3 * (size_t)f.nacc + 4 * (size_t)f.nA + 8 + 2 * (size_t)f.nc + f.nT + f.nA +
                             3 * (size_t)f.ngauss + 32 * (size_t)f.nacc);
}

// one CTA per job of a multi-job evaluation (all jobs of one model: same shared-memory size)
__global__ void __launch_bounds__(1024) ct_finalize_multi_kernel(const FinalizeArgs* __restrict__ fs)
{
    ct_finalize_body(fs[blockIdx.x]);
}

// ============================================================================
// Host: engine
// ============================================================================
namespace {

std::string readFile(const std::string& p)
{
    std::ifstream f(p, std::ios::binary);
    if (!f) throw std::runtime_error("cannot read " + p);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

// Code generation is a pure function of the model, and the model of the
// configuration text, its chain-filter patterns and its lineshape tables:
// handles built from the same ones (a serving loop creates several per model)
// share one generated model.
GeneratedModel cachedGenerate(const Model& m, const std::string& config_path)
{
    std::string key = readFile(config_path);
    for (const auto& c : m.cfg.chain_filter) key += "\n#chain " + c;
    for (const auto& b : m.blocks)
        for (const auto& r : b.res) {
            key += "\n#aux ";
            key.append((const char*)r.aux.data(), r.aux.size() * sizeof(double));
        }
    static std::mutex mu;
    static std::map<std::string, std::shared_ptr<const GeneratedModel>> cache;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return *it->second;
    }
    auto g = std::make_shared<const GeneratedModel>(generateModel(m));
    std::lock_guard<std::mutex> lk(mu);
    if (cache.size() >= 32) cache.clear();
    cache.emplace(key, g);
    return *g;
}

std::string kernelDir()
{
    const char* e = std::getenv("CTPWA_B200_KERNEL_DIR");
    if (e && *e) return e;
    // next to this library: <pkg>/csrc/kernels
    Dl_info info;
    if (dladdr((void*)&kernelDir, &info) && info.dli_fname) {
        std::filesystem::path p = std::filesystem::path(info.dli_fname).parent_path() / "csrc" / "kernels";
        if (std::filesystem::exists(p)) return p.string();
    }
    return "ctpwa_b200/csrc/kernels";
}

uint64_t fnv1a(const std::string& s)
{
    uint64_t h = 1469598103934665603ULL;
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ULL;
    }
    return h;
}

std::string cacheDir()
{
    const char* e = std::getenv("CTPWA_JIT_CACHE_DIR");
    if (e && *e) return e;
    // next to this library (travels with the package), else the user cache
    Dl_info info;
    if (dladdr((void*)&cacheDir, &info) && info.dli_fname) {
        std::filesystem::path p = std::filesystem::path(info.dli_fname).parent_path() / "_jitcache";
        std::error_code ec;
        std::filesystem::create_directories(p, ec);
        if (!ec && access(p.c_str(), W_OK) == 0) return p.string();
    }
    const char* home = std::getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/ctpwa_b200_jit";
}

}  // namespace

// The library's device-memory pool of one device (created on first use,
// kept for the process): freed blocks stay in the pool for later handles.
cudaMemPool_t enginePool(int device)
{
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool;
    CT_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = ~0ull;
    CT_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pools[device] = pool;
    return pool;
}

void* Engine::devAlloc(size_t bytes)
{
    void* p = nullptr;
    CT_CUDA(cudaMallocFromPoolAsync(&p, std::max<size_t>(bytes, 16), enginePool(opt_.device), mem_stream_));
    // usable on any stream once the allocating stream has reached it
    CT_CUDA(cudaStreamSynchronize(mem_stream_));
    return p;
}

void Engine::devFree(void* p)
{
    if (p) cudaFreeAsync(p, mem_stream_);
}

// Resident 256-thread CTAs per SM of a fused kernel (occupancy query on the
// library kernel handle; from its register count if that query is refused).
int Engine::residentCtas(void* kernel, int block, int dsmem) const
{
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)kernel, block, (size_t)dsmem) == cudaSuccess &&
        nb > 0)
        return nb;
    cudaGetLastError();
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, (const void*)kernel) == cudaSuccess && fa.numRegs > 0) {
        cudaGetLastError();
        int regs = (fa.numRegs + 7) / 8 * 8;
        return std::max(1, std::min(2048 / block, 65536 / (regs * block)));
    }
    cudaGetLastError();
    return 1;
}

// Split `target` CTAs over the samples in proportion to their event counts
// (at least one CTA per non-empty sample, at most one per `block` events);
// no_phsp: over the data and background samples only.
void Engine::layoutCtas(int target, long long tot, int block, CtaLayout& lay, bool no_phsp) const
{
    long long want[3] = {0, 0, 0}, maxc[3] = {0, 0, 0};
    long long sum = 0;
    for (int k = 0; k < 3; ++k) {
        if (samples_[k].n <= 0 || (no_phsp && k == 0)) continue;
        maxc[k] = (samples_[k].n + block - 1) / block;
        want[k] = std::max(1LL, std::min(maxc[k], (long long)std::floor((double)target * samples_[k].n / std::max(1LL, tot))));
        sum += want[k];
    }
    // hand the CTAs lost to rounding to the samples with the most events per CTA
    while (sum < target) {
        int best = -1;
        double most = 0.0;
        for (int k = 0; k < 3; ++k)
            if (want[k] > 0 && want[k] < maxc[k] && (double)samples_[k].n / want[k] > most) {
                most = (double)samples_[k].n / want[k];
                best = k;
            }
        if (best < 0) break;
        ++want[best];
        ++sum;
    }
    int begin = 0;
    for (int k = 0; k < 3; ++k) {
        lay.cta[k][0] = begin;
        lay.cta[k][1] = (int)want[k];
        begin += (int)want[k];
    }
    lay.grid = std::max(1, begin);
}

Engine::Engine(const std::string& config_path, const EngineOptions& opt) : opt_(opt)
{
    // host time of each set-up phase (device work of the phase finished)
    auto t_last = std::chrono::steady_clock::now();
    auto mark = [&](const char* name) {
        if (init_stream_) CT_CUDA(cudaStreamSynchronize(init_stream_));
        const auto t = std::chrono::steady_clock::now();
        setup_ms_.emplace_back(name, std::chrono::duration<double, std::milli>(t - t_last).count());
        t_last = t;
    };
    Config cfg = loadConfig(config_path);
    if (!cfg.valid()) {
        std::string w = cfg.warnings.empty() ? "" : (": " + cfg.warnings.front());
        throw std::runtime_error("analysis not initialized: invalid or missing config file \"" + config_path + "\"" + w);
    }
    model_ = buildModel(cfg, 1);
    if (model_.nAmp() == 0) throw std::runtime_error("the configuration defines no amplitudes");
    for (const auto& b : model_.blocks)
        for (const auto& r : b.res)
            if (r.type == ModelType::Custom) checkCustomExpr(r.options.at("expr"), r.param_names);
    gen_ = cachedGenerate(model_, config_path);
    mark("model");
    int ndev = 0;
    CT_CUDA(cudaGetDeviceCount(&ndev));
    if (ndev == 0) throw std::runtime_error("no CUDA devices available (this engine has no CPU path)");
    CT_CUDA(cudaSetDevice(opt_.device));
    CT_CUDA(cudaStreamCreateWithFlags(&mem_stream_, cudaStreamNonBlocking));
    // the finalize kernels' shared memory grows with the gradient length
    // (per-warp row sums, ct_finalize_shm): allow up to 200 KB
    CT_CUDA(cudaFuncSetAttribute((const void*)ct_finalize_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 200 * 1024));
    CT_CUDA(cudaFuncSetAttribute((const void*)ct_finalize_multi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 200 * 1024));
    CT_CUDA(cudaFuncSetAttribute((const void*)ct_rowsum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 200 * 1024));
    shape_ = fusedShape(gen_);
    // initialisation work goes to a private non-blocking stream, so a handle
    // being created does not serialise with other handles' evaluations
    CT_CUDA(cudaStreamCreateWithFlags(&init_stream_, cudaStreamNonBlocking));
    mark("context");
    compileKernel();
    mark("kernels");
    loadSamples();
    mark("samples");
    buildTables();
    mark("angular_tables");
    {
        // the generated kernels gather the pairing check's maxima as they
        // write the tables (pairPolarisations reads them)
        const int npair = model_.npol / 2, nplane = gen_.nplane;
        bool all = !k_ang_.empty();
        for (void* k : k_ang_) all = all && k;
        if (all && npair > 0 && nplane * npair <= 32) {
            alloc(d_pairmax_, sizeof(unsigned long long) * (2 * nplane * npair + 1));
            CT_CUDA(cudaMemsetAsync(d_pairmax_, 0, sizeof(unsigned long long) * (2 * nplane * npair + 1), init_stream_));
        }
    }
    for (int k = 0; k < 3; ++k)
        if (samples_[k].n > 0 || k < 2) computeAngular(k);
    mark("angular");
    pairPolarisations();
    eventMajorMixedAngular();
    mark("pairing");
    // evaluation buffers
    int nA = model_.nAmp();
    alloc(d_v_, sizeof(double) * 2 * nA);
    alloc(d_consts_, sizeof(double) * std::max(1, gen_.nconst));
    alloc(d_kblock_, k_sym_bytes_);
    std::vector<double> ratio = model_.coupling.ratio;
    alloc(d_amp_chain_, sizeof(int) * nA);
    alloc(d_ratio_, sizeof(double) * nA);
    CT_CUDA(cudaMemcpyAsync(d_amp_chain_, model_.coupling.amp_chain.data(), sizeof(int) * nA, cudaMemcpyHostToDevice, init_stream_));
    CT_CUDA(cudaMemcpyAsync(d_ratio_, ratio.data(), sizeof(double) * nA, cudaMemcpyHostToDevice, init_stream_));
    int ng = (int)model_.gauss.size();
    alloc(d_gauss_idx_, sizeof(int) * std::max(1, ng));
    alloc(d_gauss_ms_, sizeof(double) * 2 * std::max(1, ng));
    if (ng) {
        std::vector<int> gi;
        std::vector<double> gm;
        for (const auto& g : model_.gauss) {
            gi.push_back(g.first);
            gm.push_back(g.second.first);
            gm.push_back(g.second.second);
        }
        CT_CUDA(cudaMemcpyAsync(d_gauss_idx_, gi.data(), sizeof(int) * ng, cudaMemcpyHostToDevice, init_stream_));
        CT_CUDA(cudaMemcpyAsync(d_gauss_ms_, gm.data(), sizeof(double) * 2 * ng, cudaMemcpyHostToDevice, init_stream_));
    }
    // grid: one full wave of resident CTAs of the fused kernel of each
    // precision (SMs x CTAs per SM from the kernel's occupancy), split over
    // the samples in proportion to their sizes, so every CTA gets about the
    // same number of events and no partial second wave is left
    int sms = 148;
    CT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, opt_.device));
    long long tot = 0;
    for (int k = 0; k < 3; ++k) tot += samples_[k].n;
    int maxgrid = 1;
    for (int pr = 0; pr < 2; ++pr) {
        int occ = residentCtas(pr == 0 ? k_f64_ : k_mixed_, shape_.block[pr], shape_.dsmem[pr]);
        layoutCtas(sms * occ, tot, shape_.block[pr], lay_[pr]);
        maxgrid = std::max(maxgrid, lay_[pr].grid);
        layoutCtas(sms * occ, samples_[1].n + samples_[2].n, shape_.block[pr], lay_data_[pr], true);
        maxgrid = std::max(maxgrid, lay_data_[pr].grid);
    }
    grid_max_ = maxgrid;
    int nacc = 2 + 2 * nA + model_.nTheta();
    alloc(d_partials_, sizeof(double) * (size_t)grid_max_ * nacc);
    alloc(d_parts_, sizeof(double) * 8);
    alloc(d_err_, sizeof(int));
    alloc(d_mask_, sizeof(int) * std::max(1, (int)model_.blocks.size()));
    CT_CUDA(cudaMemsetAsync(d_err_, 0, sizeof(int), init_stream_));
    alloc(d_hscratch_, sizeof(double) * (3 * (size_t)std::max(1, model_.nParams()) + 1));
    mark("buffers");
    CT_CUDA(cudaStreamSynchronize(init_stream_));
    cudaStreamDestroy(init_stream_);
    init_stream_ = nullptr;
}

Engine::~Engine()
{
    for (auto& s : samples_) {
        devFree(s.p4);
        devFree(s.slamp64);
        devFree(s.slamp32);
        devFree(s.slamp64p);
        devFree(s.kin);
        devFree(s.ev64);
        devFree(s.evf);
        devFree(s.evd);
        devFree(s.w);
    }
    devFree(d_ag_tables_);
    devFree(d_pairmax_);
    devFree(d_ghpart_);
    devFree(d_ghout_);
    devFree(d_v_);
    devFree(d_consts_);
    devFree(d_kblock_);
    devFree(d_partials_);
    devFree(d_parts_);
    devFree(d_hscratch_);
    devFree(d_err_);
    devFree(d_mask_);
    devFree(d_amp_chain_);
    devFree(d_ratio_);
    devFree(d_gauss_idx_);
    devFree(d_gauss_ms_);
    for (size_t i = 0; i < ev_begin_.size(); ++i) {
        cudaEventDestroy(ev_begin_[i]);
        cudaEventDestroy(ev_end_[i]);
    }
    if (init_stream_) cudaStreamDestroy(init_stream_);
    devFree(d_hdirs_);
    devFree(d_hconsts_);
    devFree(d_hrows_);
    devFree(d_hvsums_);
    devFree(d_htsums_);
    devFree(d_gpart_);
    devFree(d_npart_);
    devFree(d_nmat_);
    devFree(d_ntheta_);
    devFree(d_nrow_);
    if (mem_stream_) {
        cudaStreamSynchronize(mem_stream_);
        cudaStreamDestroy(mem_stream_);
    }
    if (hvp_lib_) cudaLibraryUnload((cudaLibrary_t)hvp_lib_);
    if (gram_lib_) cudaLibraryUnload((cudaLibrary_t)gram_lib_);
    if (gram_hess_lib_) cudaLibraryUnload((cudaLibrary_t)gram_hess_lib_);
    if (norm_lib_) cudaLibraryUnload((cudaLibrary_t)norm_lib_);
    if (lib_) cudaLibraryUnload((cudaLibrary_t)lib_);
}

void Engine::loadSamples()
{
    const char* kinds[3] = {"phsp", "data", "bkg"};
    const char* wkeys[3] = {"phsp_weights", "data_weights", "bkg_weights"};
    int nfin = (int)model_.final_order.size();
    if (opt_.device_samples) {
        // events from the caller's device arrays: transposed straight into
        // the SoA planes, weights copied (and summed on the host)
        for (int k = 0; k < 3; ++k) {
            const long long n = opt_.dev_n[k];
            if (n < 0 || (n > 0 && !opt_.dev_p4[k])) throw std::runtime_error("in-memory sample: bad event array");
            // the arrays must be device memory of this handle's GPU
            for (const void* ptr : {(const void*)opt_.dev_p4[k], (const void*)opt_.dev_w[k]}) {
                if (!ptr || n == 0) continue;
                cudaPointerAttributes at;
                if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
                    at.device != opt_.device) {
                    cudaGetLastError();
                    throw std::runtime_error(std::string("in-memory ") + kinds[k] +
                                             " sample: not device memory of the handle's GPU");
                }
            }
            if (k < 2 && n == 0) throw std::runtime_error(std::string("in-memory samples need a ") + kinds[k] + " sample");
            DeviceSample& d = samples_[k];
            d.n = n;
            d.wsum = (double)n;
            if (k == 2) has_bkg_ = n > 0;
            if (n == 0) continue;
            const size_t bytes = sizeof(double) * (size_t)n * nfin * 4;
            CT_CUDA(cudaMallocFromPoolAsync((void**)&d.p4, bytes, enginePool(opt_.device), init_stream_));
            ag_transpose_kernel<<<(unsigned)((n + 255) / 256), 256, 0, init_stream_>>>(opt_.dev_p4[k], d.p4, n, nfin);
            CT_CUDA(cudaGetLastError());
            device_bytes_ += bytes;
            if (opt_.dev_w[k]) {
                alloc(d.w, sizeof(double) * n);
                CT_CUDA(cudaMemcpyAsync(d.w, opt_.dev_w[k], sizeof(double) * n, cudaMemcpyDeviceToDevice, init_stream_));
                std::vector<double> w((size_t)n);
                CT_CUDA(cudaMemcpyAsync(w.data(), opt_.dev_w[k], sizeof(double) * n, cudaMemcpyDeviceToHost, init_stream_));
                CT_CUDA(cudaStreamSynchronize(init_stream_));
                d.wsum = 0.0;
                for (double x : w) d.wsum += x;
                device_bytes_ += sizeof(double) * n;
            }
            CT_CUDA(cudaStreamSynchronize(init_stream_));
        }
        return;
    }
    for (int k = 0; k < 3; ++k) {
        auto it = model_.cfg.data_files.find(kinds[k]);
        if (it == model_.cfg.data_files.end()) {
            if (k < 2) throw std::runtime_error(std::string("config has no Data.") + kinds[k] + " entry");
            continue;
        }
        Sample s = readSample(it->second, nfin);
        DeviceSample& d = samples_[k];
        if (k == 2) has_bkg_ = true;
        std::vector<double> w;
        auto wi = model_.cfg.data_files.find(wkeys[k]);
        if (wi != model_.cfg.data_files.end() && (k != 2 || has_bkg_)) w = readWeights(wi->second, s.n);
        shardSample(s, w, opt_.shard_rank, opt_.shard_world);
        d.n = s.n;
        d.wsum = 0.0;
        if (w.empty()) d.wsum = (double)s.n;
        else
            for (double x : w) d.wsum += x;
        if (s.n == 0) continue;
        size_t bytes = sizeof(double) * (size_t)s.n * nfin * 4;
        double* tmp = nullptr;
        CT_CUDA(cudaMallocFromPoolAsync((void**)&tmp, bytes, enginePool(opt_.device), init_stream_));
        CT_CUDA(cudaMemcpyAsync(tmp, s.p4.data(), bytes, cudaMemcpyHostToDevice, init_stream_));
        CT_CUDA(cudaMallocFromPoolAsync((void**)&d.p4, bytes, enginePool(opt_.device), init_stream_));
        ag_transpose_kernel<<<(unsigned)((s.n + 255) / 256), 256, 0, init_stream_>>>(tmp, d.p4, s.n, nfin);
        CT_CUDA(cudaGetLastError());
        CT_CUDA(cudaFreeAsync(tmp, init_stream_));
        if (!w.empty()) {
            alloc(d.w, sizeof(double) * s.n);
            CT_CUDA(cudaMemcpyAsync(d.w, w.data(), sizeof(double) * s.n, cudaMemcpyHostToDevice, init_stream_));
        }
        // the host sample is released at the end of this iteration
        CT_CUDA(cudaStreamSynchronize(init_stream_));
        device_bytes_ += bytes + (w.empty() ? 0 : sizeof(double) * s.n);
    }
}

std::string jitAngularCubin(const std::string& src, bool* cache_hit);
bool angularInterpreted();

// Host description of every angular group (AgGroup with its tables: the
// (S, L) variant of each vertex per SL combination, the polarisation map,
// the kinematic slots it fills), appending the vertex variants and their
// Clebsch-Gordan products to vars / cg. Shared by the device tables of
// Engine::buildTables and the generated angular kernels (angularSource),
// so the offsets into cg agree.
struct AgGroupHost {
    AgGroup g;
    std::vector<int> sl_var, pol_map, kin;
};

std::vector<AgGroupHost> angularGroups(const Model& model, const GeneratedModel& gen, std::vector<AgNodeVar>& vars,
                                       std::vector<double>& cg)
{
    std::vector<AgGroupHost> gh(model.groups.size());
    for (size_t gi = 0; gi < model.groups.size(); ++gi) {
        const Group& G = model.groups[gi];
        AgGroupHost& H = gh[gi];
        AgGroup& A = H.g;
        std::memset(&A, 0, sizeof(A));
        if ((int)G.particle_names.size() > AG_MAXP || (int)G.nodes.size() > AG_MAXN)
            throw std::runtime_error("decay chain too large for the angular kernel");
        A.np = (int)G.particle_names.size();
        A.nfin = (int)model.final_order.size();
        A.nnodes = (int)G.nodes.size();
        A.nsl = G.nSL();
        A.npol = model.npol;
        A.tensor_size = G.tensor_size;
        A.plane0 = gen.group_plane0[gi];
        for (int i = 0; i < A.np; ++i) {
            A.input_slot[i] = G.input_slot[i];
            A.sum_a[i] = G.sum_of[i].first;
            A.sum_b[i] = G.sum_of[i].second;
            A.build_order[i] = G.build_order[i];
        }
        for (size_t ni = 0; ni < G.nodes.size(); ++ni) {
            const ModelNode& n = G.nodes[ni];
            if (n.dj > AG_MAXD || n.dj1 > AG_MAXD || n.dj2 > AG_MAXD || n.dj * n.dj1 * n.dj2 > AG_MAXT)
                throw std::runtime_error("spin too large for the angular kernel (2J+1 <= 7, vertex tensor <= 64)");
            AgNode& an = A.nodes[ni];
            an.mother = n.mother;
            an.d1 = n.d1;
            an.d2 = n.d2;
            an.dj = n.dj;
            an.dj1 = n.dj1;
            an.dj2 = n.dj2;
            an.var_off = (int)vars.size();
            an.nvar = (int)n.sls.size();
            for (const auto& sl : n.sls) {
                AgNodeVar v;
                v.S = sl.S;
                v.L = sl.L;
                v.cg_off = (int)cg.size();
                if (sl.L >= AG_MAXD) throw std::runtime_error("orbital angular momentum too large for the angular kernel");
                for (int s = 0; s < n.dj; ++s)
                    for (int s1 = 0; s1 < n.dj1; ++s1)
                        for (int s2 = 0; s2 < n.dj2; ++s2) {
                            int sx2 = n.dj - 1 - 2 * s, s1x2 = n.dj1 - 1 - 2 * s1, s2x2 = n.dj2 - 1 - 2 * s2;
                            double c1 = clebschGordan(n.dj1, s1x2, n.dj2, s2x2, sl.S, s1x2 + s2x2);
                            double c2 = clebschGordan(sl.S, s1x2 + s2x2, 2 * sl.L + 1, sx2 - s1x2 - s2x2, n.dj, sx2);
                            cg.push_back(c1 * c2 / std::sqrt((double)n.dj));
                        }
                vars.push_back(v);
            }
        }
        // contraction size check
        {
            int cur = G.nodes[0].dj * G.nodes[0].dj1 * G.nodes[0].dj2;
            if (cur > AG_MAXT) throw std::runtime_error("amplitude tensor too large for the angular kernel");
            std::vector<int> shape = {G.nodes[0].dj, G.nodes[0].dj1, G.nodes[0].dj2};
            std::vector<int> labels = {G.nodes[0].mother, G.nodes[0].d1, G.nodes[0].d2};
            for (size_t ni = 1; ni < G.nodes.size(); ++ni) {
                const auto& n = G.nodes[ni];
                auto it = std::find(labels.begin(), labels.end(), n.mother);
                size_t c = it - labels.begin();
                shape.erase(shape.begin() + c);
                labels.erase(it);
                shape.push_back(n.dj1);
                shape.push_back(n.dj2);
                labels.push_back(n.d1);
                labels.push_back(n.d2);
                int t = 1;
                for (int x : shape) t *= x;
                if (t > AG_MAXT) throw std::runtime_error("amplitude tensor too large for the angular kernel");
            }
        }
        for (int s = 0; s < G.nSL(); ++s)
            for (size_t ni = 0; ni < G.nodes.size(); ++ni) H.sl_var.push_back(G.sl_combs[s][ni]);
        H.pol_map = model.pol_map;
        for (size_t k = 0; k < gen.slots.size(); ++k) {
            const KinSlot& ks = gen.slots[k];
            if (ks.group != (int)gi) continue;
            H.kin.insert(H.kin.end(), {ks.type, ks.a, ks.b, ks.c, (int)k});
        }
        A.nkin = (int)H.kin.size() / 5;
    }
    return gh;
}

// CUDA source of the generated angular kernels: one kernel ct_ang_<g> per
// angular group, straight-line code over the group's particles, kinematic
// slots, vertices and SL combinations with every tensor shape fixed
// (kernels/angular_gen.cuh), the same values as ag_group_kernel's
// interpretation of the group tables. Each vertex's frame and rotations are
// computed once per event; each SL combination contracts its vertex tensors
// along the chain in the interpreter's order and writes its planes.
std::string angularSource(const std::vector<AgGroupHost>& gh, const std::vector<AgNodeVar>& vars, int nplane)
{
    std::ostringstream o;
    o << "// generated by ctpwa_b200 (Engine angular kernels)\n#include \"angular_gen.cuh\"\n\n";
    for (size_t gi = 0; gi < gh.size(); ++gi) {
        const AgGroup& A = gh[gi].g;
        const int npair = A.npol / 2;
        // pairmax (may be null): maxima over events of
        // |SL_{c,npol-1-q} -+ conj(SL_{c,q})| at [(c npair + q) 2 + 0 / 1] and
        // of |SL| at [2 nplane npair] (the layout of ct_pair_check_kernel),
        // accumulated by one atomic per warp and value
        o << "extern \"C\" __global__ void __launch_bounds__(128) ct_ang_" << gi
          << "(const double* __restrict__ p4, long long n, long long ld, AgTables T, double2* __restrict__ out64,\n"
             "    float2* __restrict__ out32, double* __restrict__ kin, unsigned long long* __restrict__ pairmax)\n{\n"
             "  const long long e = (long long)blockIdx.x * 128 + threadIdx.x;\n";
        if (npair > 0) {
            o << "  double pm[" << std::max(1, 2 * A.nsl * npair) << "] = {}, big = 0.0;\n";
            o << "  if (e < n) {\n";
        } else {
            o << "  if (e >= n) return;\n  {\n";
        }
        for (int f = 0; f < A.nfin; ++f)
            o << "  const V4 f" << f << " = {p4[" << 4 * f << " * n + e], p4[" << 4 * f + 1 << " * n + e], p4[" << 4 * f + 2
              << " * n + e], p4[" << 4 * f + 3 << " * n + e]};\n";
        o << "  V4 parent = {0, 0, 0, 0};\n";
        for (int f = 0; f < A.nfin; ++f) o << "  parent = v4add(parent, f" << f << ");\n";
        for (int k = 0; k < A.np; ++k) {
            const int idx = A.build_order[k], sl = A.input_slot[idx];
            o << "  const V4 m" << idx << " = ";
            if (sl >= 0) o << "f" << sl;
            else if (sl == -1) o << "parent";
            else o << "v4add(m" << A.sum_a[idx] << ", m" << A.sum_b[idx] << ")";
            o << ";\n";
        }
        const auto& K = gh[gi].kin;
        for (size_t k = 0; k + 4 < K.size(); k += 5) {
            const int type = K[k], a = K[k + 1], b = K[k + 2] >= 0 ? K[k + 2] : K[k + 1],
                      c = K[k + 3] >= 0 ? K[k + 3] : K[k + 1];
            o << "  kin[" << K[k + 4] << "LL * ld + e] = agKin<" << type << ">(m" << a << ", m" << b << ", m" << c
              << ");\n";
        }
        for (int ni = 0; ni < A.nnodes; ++ni) {
            const AgNode& nd = A.nodes[ni];
            o << "  AgVertexFrame<" << nd.dj1 << ", " << nd.dj2 << "> F" << ni << ";\n  agVertexFrame<" << nd.dj1 << ", "
              << nd.dj2 << ">(T, m" << nd.d1 << ", m" << nd.d2 << ", F" << ni << ");\n";
        }
        for (int s = 0; s < A.nsl; ++s) {
            o << "  {  // SL combination " << s << "\n";
            std::vector<int> shape, labels;
            for (int ni = 0; ni < A.nnodes; ++ni) {
                const AgNode& nd = A.nodes[ni];
                const AgNodeVar& v = vars[nd.var_off + gh[gi].sl_var[s * A.nnodes + ni]];
                const int size = nd.dj * nd.dj1 * nd.dj2;
                o << "    double2 a" << ni << "[" << size << "];\n    agVertexAmp<" << nd.dj << ", " << nd.dj1 << ", "
                  << nd.dj2 << ", " << v.L << ">(T, F" << ni << ", T.cg + " << v.cg_off << ", a" << ni << ");\n";
                if (ni == 0) {
                    shape = {nd.dj, nd.dj1, nd.dj2};
                    labels = {nd.mother, nd.d1, nd.d2};
                    o << "    const double2* c0 = a0;\n";
                    continue;
                }
                const int rank = (int)shape.size();
                int c = 0;
                for (int j = 0; j < rank; ++j)
                    if (labels[j] == nd.mother) {
                        c = j;
                        break;
                    }
                std::vector<int> st(rank);
                st[rank - 1] = 1;
                for (int j = rank - 2; j >= 0; --j) st[j] = st[j + 1] * shape[j + 1];
                std::vector<int> oshape;
                for (int j = 0; j < rank; ++j)
                    if (j != c) oshape.push_back(shape[j]);
                oshape.push_back(nd.dj1);
                oshape.push_back(nd.dj2);
                int total = 1;
                for (int x : oshape) total *= x;
                o << "    double2 c" << ni << "[" << total << "];\n";
                const int ro = (int)oshape.size();
                for (int idx = 0; idx < total; ++idx) {
                    int t = idx;
                    std::vector<int> ic(ro);
                    for (int j = ro - 1; j >= 0; --j) {
                        ic[j] = t % oshape[j];
                        t /= oshape[j];
                    }
                    int base = 0, pos = 0;
                    for (int j = 0; j < rank; ++j)
                        if (j != c) base += ic[pos++] * st[j];
                    o << "    c" << ni << "[" << idx << "] = agContract<" << shape[c] << ", " << nd.dj1 << ", " << nd.dj2
                      << ">(c" << ni - 1 << ", " << base << ", " << st[c] << ", a" << ni << ", " << ic[ro - 2] << ", "
                      << ic[ro - 1] << ");\n";
                }
                shape = oshape;
                labels.erase(labels.begin() + c);
                labels.push_back(nd.d1);
                labels.push_back(nd.d2);
            }
            const int last = A.nnodes - 1;
            const long long plane = (long long)(A.plane0 + s) * A.npol;
            std::vector<int> srcs(A.npol);
            for (int p = 0; p < A.npol; ++p) {
                const int src = gh[gi].pol_map.empty() ? p : gh[gi].pol_map[p];
                srcs[p] = src;
                o << "    { const double2 v = c" << last << "[" << src << "]; out64[" << plane + p
                  << "LL * ld + e] = v; if (out32) out32[" << plane + p
                  << "LL * ld + e] = make_float2((float)v.x, (float)v.y); }\n";
            }
            if (npair > 0) {
                for (int p = 0; p < A.npol; ++p)
                    o << "    big = fmax(big, agDist(c" << last << "[" << srcs[p] << "].x, c" << last << "[" << srcs[p]
                      << "].y));\n";
                for (int q = 0; q < npair; ++q) {
                    const std::string a = "c" + std::to_string(last) + "[" + std::to_string(srcs[q]) + "]",
                                      b = "c" + std::to_string(last) + "[" + std::to_string(srcs[A.npol - 1 - q]) + "]";
                    const int k = (s * npair + q) * 2;
                    o << "    pm[" << k << "] = fmax(pm[" << k << "], agDist(" << b << ".x - " << a << ".x, " << b << ".y + "
                      << a << ".y));\n";
                    o << "    pm[" << k + 1 << "] = fmax(pm[" << k + 1 << "], agDist(" << b << ".x + " << a << ".x, " << b
                      << ".y - " << a << ".y));\n";
                }
            }
            o << "  }\n";
        }
        o << "  }\n";
        if (npair > 0) {
            o << "  if (pairmax) {\n    const int lane = threadIdx.x & 31;\n";
            for (int s = 0; s < A.nsl; ++s)
                for (int q = 0; q < npair; ++q)
                    for (int w = 0; w < 2; ++w) {
                        const int k = (s * npair + q) * 2 + w;
                        const int out = ((A.plane0 + s) * npair + q) * 2 + w;
                        o << "    { const double v = agWarpMax(pm[" << k << "]); if (lane == 0) atomicMax(pairmax + " << out
                          << ", (unsigned long long)__double_as_longlong(v)); }\n";
                    }
            o << "    { const double v = agWarpMax(big); if (lane == 0) atomicMax(pairmax + " << 2 * nplane * npair
              << ", (unsigned long long)__double_as_longlong(v)); }\n  }\n";
        }
        o << "}\n\n";
    }
    return o.str();
}

void Engine::buildTables()
{
    // Layout of one device allocation: vars | cg | ylm_norm | dcoef | doff | per-group (sl_var, pol_map, kin)
    std::vector<AgNodeVar> vars;
    std::vector<double> cg;
    std::vector<double> ylm(AG_MAXD * AG_MAXD, 0.0);
    for (int l = 0; l < AG_MAXD; ++l)
        for (int am = 0; am <= l; ++am)
            ylm[l * AG_MAXD + am] = (l == 0) ? 0.5 * std::sqrt(1.0 / M_PI)
                                             : std::sqrt((2.0 * l + 1.0) * refFactorial((float)(l - am)) /
                                                         (4.0 * M_PI * refFactorial((float)(l + am))));
    std::vector<double> dcoef;
    std::vector<int> doff((AG_MAXD + 1) * AG_MAXD * AG_MAXD, 0);
    for (int dim = 1; dim <= AG_MAXD; ++dim) {
        float j = (dim - 1) / 2.0f;
        for (int i1 = 0; i1 < dim; ++i1)
            for (int i2 = 0; i2 < dim; ++i2) {
                float m1 = (dim - 1 - 2 * i1) / 2.0f, m2 = (dim - 1 - 2 * i2) / 2.0f;
                doff[(dim * AG_MAXD + i1) * AG_MAXD + i2] = (int)dcoef.size();
                size_t cnt_pos = dcoef.size();
                dcoef.push_back(0.0);
                int kmin = (m1 < m2) ? 0 : (int)(m1 - m2);
                int kmax = (m1 > -m2) ? (int)(j - m2) : (int)(j + m1);
                int cnt = 0;
                for (int k = kmin; k <= kmax; ++k) {
                    double num = refFactorial(j + m2) * refFactorial(j - m2) * refFactorial(j + m1) * refFactorial(j - m1);
                    double den = refFactorial((float)k) * refFactorial(j - m2 - k) * refFactorial(j + m1 - k) *
                                 refFactorial(k - m1 + m2);
                    double c = std::pow(-1.0, k - m1 + m2) * std::sqrt(num) / den;
                    dcoef.push_back(c);
                    dcoef.push_back(2 * j + m1 - m2 - 2 * k);
                    dcoef.push_back(2 * k - m1 + m2);
                    ++cnt;
                }
                dcoef[cnt_pos] = cnt;
            }
    }
    // per-group node variants and CG products
    std::vector<AgGroupHost> gh = angularGroups(model_, gen_, vars, cg);
    if (!angularInterpreted() && !gh.empty()) {
        const std::string src = angularSource(gh, vars, gen_.nplane);
        // the module has no per-handle state (unlike the fused kernels'
        // constant bank): handles of one model share one loaded copy for the
        // life of the process, found by the hash of the generated source, so
        // creating a handle neither compiles, reads nor loads a module
        static std::mutex lib_mu;
        static std::map<uint64_t, cudaLibrary_t> libs;
        cudaLibrary_t lib;
        {
            std::lock_guard<std::mutex> lk(lib_mu);
            const uint64_t key = fnv1a(src);
            auto it = libs.find(key);
            if (it != libs.end()) lib = it->second;
            else {
                bool hit = false;
                const std::string cubin = jitAngularCubin(src, &hit);
                CT_CUDA(cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
                libs.emplace(key, lib);
            }
        }
        k_ang_.assign(gh.size(), nullptr);
        for (size_t g = 0; g < gh.size(); ++g) {
            cudaKernel_t k;
            CT_CUDA(cudaLibraryGetKernel(&k, lib, ("ct_ang_" + std::to_string(g)).c_str()));
            k_ang_[g] = (void*)k;
        }
    }
    // pack everything into one allocation
    auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t off = 0;
    size_t o_vars = off;
    off = align(off + vars.size() * sizeof(AgNodeVar));
    size_t o_cg = off;
    off = align(off + cg.size() * sizeof(double));
    size_t o_ylm = off;
    off = align(off + ylm.size() * sizeof(double));
    size_t o_dc = off;
    off = align(off + dcoef.size() * sizeof(double));
    size_t o_doff = off;
    off = align(off + doff.size() * sizeof(int));
    std::vector<size_t> o_slv(gh.size()), o_pm(gh.size()), o_kin(gh.size());
    for (size_t g = 0; g < gh.size(); ++g) {
        o_slv[g] = off;
        off = align(off + gh[g].sl_var.size() * sizeof(int) + 4);
        o_pm[g] = off;
        off = align(off + gh[g].pol_map.size() * sizeof(int) + 4);
        o_kin[g] = off;
        off = align(off + gh[g].kin.size() * sizeof(int) + 4);
    }
    std::vector<char> img(off, 0);
    std::memcpy(img.data() + o_vars, vars.data(), vars.size() * sizeof(AgNodeVar));
    std::memcpy(img.data() + o_cg, cg.data(), cg.size() * sizeof(double));
    std::memcpy(img.data() + o_ylm, ylm.data(), ylm.size() * sizeof(double));
    std::memcpy(img.data() + o_dc, dcoef.data(), dcoef.size() * sizeof(double));
    std::memcpy(img.data() + o_doff, doff.data(), doff.size() * sizeof(int));
    for (size_t g = 0; g < gh.size(); ++g) {
        std::memcpy(img.data() + o_slv[g], gh[g].sl_var.data(), gh[g].sl_var.size() * sizeof(int));
        std::memcpy(img.data() + o_pm[g], gh[g].pol_map.data(), gh[g].pol_map.size() * sizeof(int));
        std::memcpy(img.data() + o_kin[g], gh[g].kin.data(), gh[g].kin.size() * sizeof(int));
    }
    alloc(d_ag_tables_, off);
    CT_CUDA(cudaMemcpyAsync(d_ag_tables_, img.data(), off, cudaMemcpyHostToDevice, init_stream_));
    CT_CUDA(cudaStreamSynchronize(init_stream_));
    char* base = (char*)d_ag_tables_;
    AgTables T;
    T.vars = (const AgNodeVar*)(base + o_vars);
    T.cg = (const double*)(base + o_cg);
    T.ylm_norm = (const double*)(base + o_ylm);
    T.dcoef = (const double*)(base + o_dc);
    T.doff = (const int*)(base + o_doff);
    ag_host_.assign((char*)&T, (char*)&T + sizeof(T));
    group_desc_.clear();
    for (size_t g = 0; g < gh.size(); ++g) {
        AgGroup A = gh[g].g;
        A.sl_var = (const int*)(base + o_slv[g]);
        A.pol_map = gh[g].pol_map.empty() ? nullptr : (const int*)(base + o_pm[g]);
        A.kin = (const int*)(base + o_kin[g]);
        group_desc_.emplace_back((char*)&A, (char*)&A + sizeof(A));
    }
}

namespace {

__device__ __forceinline__ double ct_warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// a NaN or infinite distance counts as infinitely far
__device__ __forceinline__ double ct_dist(double x, double y)
{
    const double d = hypot(x, y);
    return d == d ? d : (double)INFINITY;
}

// max over events of |SL_{c, npol-1-q} - conj(SL_{c,q})| and of
// |SL_{c, npol-1-q} + conj(SL_{c,q})| per (plane c, pair q), and of |SL|:
// out[(c * npair + q) * 2 + 0 / 1], out[2 * nplane * npair] (doubles >= 0,
// compared through their bit patterns)
//
// Each thread keeps its own maxima over its events, one pair at a time;
// warps combine them by shuffles and lane 0 issues one atomic per warp and
// value (blocks are whole warps).
__global__ void ct_pair_check_kernel(const double2* __restrict__ sl, long long n, long long ld, int nplane, int npol,
                                     unsigned long long* __restrict__ out)
{
    const int npair = npol / 2, lane = threadIdx.x & 31;
    const long long e0 = (long long)blockIdx.x * blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
    for (int c = 0; c < nplane; ++c)
        for (int q = 0; q < npair; ++q) {
            const double2* __restrict__ ra = sl + (long long)(c * npol + q) * ld;
            const double2* __restrict__ rb = sl + (long long)(c * npol + npol - 1 - q) * ld;
            double dp = 0.0, dn = 0.0;
            for (long long e = e0; e < n; e += stride) {
                const double2 a = ra[e], b = rb[e];
                dp = fmax(dp, ct_dist(b.x - a.x, b.y + a.y));
                dn = fmax(dn, ct_dist(b.x + a.x, b.y - a.y));
            }
            dp = ct_warp_max(dp);
            dn = ct_warp_max(dn);
            if (lane == 0) {
                atomicMax(out + (c * npair + q) * 2, (unsigned long long)__double_as_longlong(dp));
                atomicMax(out + (c * npair + q) * 2 + 1, (unsigned long long)__double_as_longlong(dn));
            }
        }
    double big = 0.0;
    for (int r = 0; r < nplane * npol; ++r) {
        const double2* __restrict__ ra = sl + (long long)r * ld;
        for (long long e = e0; e < n; e += stride) big = fmax(big, ct_dist(ra[e].x, ra[e].y));
    }
    big = ct_warp_max(big);
    if (lane == 0) atomicMax(out + 2 * nplane * npair, (unsigned long long)__double_as_longlong(big));
}

}  // namespace

// Decides whether the polarisations pair up as SL_{npol-1-q} = conj(SL_q) on
// every event of the phase-space, data and background samples (to 1e-12 of
// the largest |SL|; e.g. the M = -1 and M = +1 states of a J/psi decaying to
// spin-0 particles), and if so switches the fused kernels to their paired
// variants (ct_fused_*_pc) with compact tables holding polarisations
// 0 .. (npol+1)/2 - 1: the FP32 table is replaced, the plain kernel gets an
// FP64 copy (the other kernels keep the full FP64 table). The check also
// measures the minus-sign relation, which the paired kernels do not use.
// Runs on the constructor's initialisation stream.
// the compact table of paired polarisations, event-major:
// out[e][c ns + q] = rows[c npol + q][e] (q < ns stored polarisations; zeros
// for the padding events past n)
__global__ void ct_compact_event_major_kernel(const double2* __restrict__ rows, long long n, long long ld, int nplane,
                                              int npol, int ns, double2* __restrict__ out)
{
    const int nr = nplane * ns;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ld; e += (long long)gridDim.x * blockDim.x)
        for (int c = 0; c < nplane; ++c)
            for (int q = 0; q < ns; ++q)
                out[e * nr + c * ns + q] = e < n ? rows[(long long)(c * npol + q) * ld + e] : make_double2(0.0, 0.0);
}

void Engine::pairPolarisations()
{
    const int npol = model_.npol, nplane = gen_.nplane, npair = npol / 2;
    const char* off = std::getenv("CTPWA_NO_POL_PAIRING");
    if (!opt_.pair_polarisations || npair == 0 || nplane * npair > 32 || (off && *off && *off != '0')) return;
    const int nout = 2 * nplane * npair + 1;
    std::vector<double> worst(2 * nplane * npair, 0.0);
    double big = 0.0;
    if (d_pairmax_) {
        // gathered by the generated angular kernels over all three samples
        std::vector<unsigned long long> h(nout);
        CT_CUDA(cudaMemcpyAsync(h.data(), d_pairmax_, sizeof(unsigned long long) * nout, cudaMemcpyDeviceToHost,
                                init_stream_));
        CT_CUDA(cudaStreamSynchronize(init_stream_));
        for (int i = 0; i < 2 * nplane * npair; ++i) std::memcpy(&worst[i], &h[i], sizeof(double));
        std::memcpy(&big, &h[2 * nplane * npair], sizeof(double));
    }
    unsigned long long* d_out = nullptr;
    if (!d_pairmax_) alloc(d_out, sizeof(unsigned long long) * nout);
    for (int k = 0; k < 3 && !d_pairmax_; ++k) {
        const DeviceSample& d = samples_[k];
        if (d.n <= 0) continue;
        CT_CUDA(cudaMemsetAsync(d_out, 0, sizeof(unsigned long long) * nout, init_stream_));
        const unsigned grid = (unsigned)std::min<long long>((d.n + 255) / 256, 148LL * 8);
        ct_pair_check_kernel<<<grid, 256, 0, init_stream_>>>(d.slamp64, d.n, d.ld, nplane, npol, d_out);
        CT_CUDA(cudaGetLastError());
        std::vector<unsigned long long> h(nout);
        CT_CUDA(cudaMemcpyAsync(h.data(), d_out, sizeof(unsigned long long) * nout, cudaMemcpyDeviceToHost, init_stream_));
        CT_CUDA(cudaStreamSynchronize(init_stream_));
        for (int i = 0; i < 2 * nplane * npair; ++i) {
            double x;
            std::memcpy(&x, &h[i], sizeof(double));
            worst[i] = std::max(worst[i], x);
        }
        double b;
        std::memcpy(&b, &h[2 * nplane * npair], sizeof(double));
        big = std::max(big, b);
    }
    devFree(d_out);
    const double tol = 1e-12 * big;
    unsigned neg = 0;
    bool ok = big > 0.0;
    for (int c = 0; c < nplane && ok; ++c)
        for (int q = 0; q < npair && ok; ++q) {
            const double dp = worst[(c * npair + q) * 2], dn = worst[(c * npair + q) * 2 + 1];
            if (dp <= tol) continue;
            if (dn <= tol) neg |= 1u << (c * npair + q);
            else ok = false;
        }
    // the paired kernels rebuild conjugates with a plus sign
    if (!ok || neg != 0) return;
    const int ns = (npol + 1) / 2;
    paired_[0] = true;
    paired_[1] = opt_.mixed_tables;
    for (int pr = 0; pr < 2; ++pr)
        if (paired_[pr]) (pr == 0 ? k_f64_ : k_mixed_) = k_pc_[pr];
    for (int k = 0; k < 3; ++k) {
        DeviceSample& d = samples_[k];
        if (!d.slamp64) continue;
        const size_t rows = (size_t)nplane * ns;
        if (paired_[0]) {
            // the compact FP64 table event-major: [ld][plane x stored polarisation]
            alloc(d.slamp64p, sizeof(double2) * rows * d.ld);
            device_bytes_ += sizeof(double2) * rows * d.ld;
            const unsigned grid = (unsigned)std::min<long long>((d.ld + 255) / 256, 148LL * 16);
            ct_compact_event_major_kernel<<<grid, 256, 0, init_stream_>>>(d.slamp64, d.n, d.ld, nplane, npol, ns,
                                                                           d.slamp64p);
            CT_CUDA(cudaGetLastError());
        }
        if (paired_[1] && d.slamp32) {
            float2* compact = nullptr;
            alloc(compact, sizeof(float2) * rows * d.ld);
            for (int c = 0; c < nplane; ++c)
                for (int q = 0; q < ns; ++q)
                    CT_CUDA(cudaMemcpyAsync(compact + (size_t)(c * ns + q) * d.ld, d.slamp32 + (size_t)(c * npol + q) * d.ld,
                                            sizeof(float2) * d.ld, cudaMemcpyDeviceToDevice, init_stream_));
            CT_CUDA(cudaStreamSynchronize(init_stream_));
            devFree(d.slamp32);
            device_bytes_ -= sizeof(float2) * (size_t)(npol - ns) * nplane * d.ld;
            d.slamp32 = compact;
        }
    }
    CT_CUDA(cudaStreamSynchronize(init_stream_));
}

// old [row][ld] FP32 angular rows -> event-major records of sls float2
// (the rows' values, then zeros; zeros for the padding events past n)
__global__ void ct_sl32_event_major_kernel(const float2* __restrict__ rows, long long n, long long ld, int nrow, int sls,
                                           float2* __restrict__ out)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ld; e += (long long)gridDim.x * blockDim.x)
        for (int r = 0; r < sls; ++r)
            out[e * sls + r] = (r < nrow && e < n) ? rows[(long long)r * ld + e] : make_float2(0.0f, 0.0f);
}

// The FP32 angular tables of the evaluated samples event-major: each event's
// values (planes x stored polarisations) in one record of an even number of
// float2 (CT_SL32_STRIDE in kernels/fused_nll.cuh), so the mixed kernels
// read them with 16-byte loads. The FP64 tables stay [row][ld].
void Engine::eventMajorMixedAngular()
{
    const int npol = model_.npol, ns = paired_[1] ? (npol + 1) / 2 : npol;
    const int rows = gen_.nplane * ns, sls = (rows + 1) / 2 * 2;
    for (int k = 0; k < 3; ++k) {
        DeviceSample& d = samples_[k];
        if (!d.slamp32) continue;
        float2* em = nullptr;
        alloc(em, sizeof(float2) * (size_t)sls * d.ld);
        const unsigned grid = (unsigned)std::min<long long>((d.ld + 255) / 256, 148LL * 16);
        ct_sl32_event_major_kernel<<<grid, 256, 0, init_stream_>>>(d.slamp32, d.n, d.ld, rows, sls, em);
        CT_CUDA(cudaGetLastError());
        CT_CUDA(cudaStreamSynchronize(init_stream_));
        devFree(d.slamp32);
        device_bytes_ += sizeof(float2) * (size_t)(sls - rows) * d.ld;
        d.slamp32 = em;
    }
}

void Engine::computeAngular(int kind)
{
    DeviceSample& d = samples_[kind];
    long long n = d.n;
    // table rows padded to a multiple of 256 events: every tile of the fused
    // kernels starts on a 2 KiB boundary and may be copied whole
    d.ld = std::max(256LL, (n + 255) / 256 * 256);
    const long long ld = d.ld;
    int npol = model_.npol;
    size_t nplanes = (size_t)gen_.nplane * npol;
    size_t b64 = sizeof(double2) * nplanes * ld;
    alloc(d.slamp64, b64);
    device_bytes_ += b64;
    if (opt_.mixed_tables) {
        alloc(d.slamp32, b64 / 2);
        device_bytes_ += b64 / 2;
    }
    size_t bk = sizeof(double) * std::max<size_t>(1, gen_.slots.size()) * ld;
    alloc(d.kin, bk);
    device_bytes_ += bk;
    if (n == 0) {
        buildEventCache(kind);
        return;
    }
    AgTables T;
    std::memcpy(&T, ag_host_.data(), sizeof(T));
    for (size_t g = 0; g < group_desc_.size(); ++g) {
        if (g < k_ang_.size() && k_ang_[g]) {
            const double* p4 = d.p4;
            double2* o64 = d.slamp64;
            float2* o32 = d.slamp32;
            double* kin = d.kin;
            long long nn = n, lld = ld;
            unsigned long long* pm = kind < 3 ? d_pairmax_ : nullptr;  // the phase-space truth sample is not checked
            void* args[] = {(void*)&p4, (void*)&nn, (void*)&lld, (void*)&T, (void*)&o64, (void*)&o32, (void*)&kin,
                            (void*)&pm};
            CT_CUDA(cudaLaunchKernel(k_ang_[g], dim3((unsigned)((n + 127) / 128)), dim3(128), args, 0, init_stream_));
            continue;
        }
        AgGroup G;
        std::memcpy(&G, group_desc_[g].data(), sizeof(G));
        ag_group_kernel<<<(unsigned)((n + 127) / 128), 128, 0, init_stream_>>>(G, T, d.p4, n, ld, d.slamp64,
                                                                                 d.slamp32, d.kin);
        CT_CUDA(cudaGetLastError());
    }
    if (!opt_.keep_momenta) {
        CT_CUDA(cudaFreeAsync(d.p4, init_stream_));
        d.p4 = nullptr;
    }
    buildEventCache(kind);
}

// floats per event of the event-major FP32 frontier table (CT_EVF_STRIDE)
int evfStride(const GeneratedModel& gen)
{
    return 4 * (gen.nevf > 0 ? (gen.nevf + 3) / 4 : 1);
}

// The per-event frontier tables (parameter-independent values the per-call
// code reads) from the kinematic cache, once per sample; the kinematic cache
// is released afterwards.
void Engine::buildEventCache(int kind)
{
    DeviceSample& d = samples_[kind];
    const long long ld = d.ld;
    const size_t b64 = sizeof(double) * std::max(1, gen_.nev64) * ld;
    alloc(d.ev64, b64);
    device_bytes_ += b64;
    if (opt_.mixed_tables) {
        // FP32 frontier table event-major, 16-byte records (CT_EVF_STRIDE floats per event)
        const size_t bf = sizeof(float) * evfStride(gen_) * ld, bd = sizeof(double) * std::max(1, gen_.nevd) * ld;
        alloc(d.evf, bf);
        alloc(d.evd, bd);
        device_bytes_ += bf + bd;
    }
    if (d.n > 0) {
        const double* kin = d.kin;
        long long n = d.n;
        double* o64 = d.ev64;
        float* of = d.evf;
        double* od = d.evd;
        void* args[] = {(void*)&kin, (void*)&n, (void*)&ld, (void*)&o64, (void*)&of, (void*)&od};
        const unsigned grid = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 64);
        CT_CUDA(cudaLaunchKernel(k_evc_, dim3(grid), dim3(256), args, 0, init_stream_));
    }
    CT_CUDA(cudaStreamSynchronize(init_stream_));
    devFree(d.kin);
    d.kin = nullptr;
    device_bytes_ -= sizeof(double) * std::max<size_t>(1, gen_.slots.size()) * ld;
}

// Block size and minimum resident CTAs per SM of the plain [0] and mixed [1]
// fused kernels, unless CTPWA_F64_BLOCK / CTPWA_F64_MINB / CTPWA_MX_BLOCK /
// CTPWA_MX_MINB / CTPWA_*_ACC_SMEM override them (tuning). Measured on the
// K+K-pi0 workload with the frontier tables and the constant bank: plain
// 192 x 2 with the gradient sums in shared memory (170 registers, 12 warps
// per SM, no spills) 0.95 ms, against 0.95 ms at 96 x 4, 0.99 ms at 128 x 3,
// 1.15 ms at 256 x 2 (128 registers, spills) and 1.17 ms at 224 x 2; mixed
// (frontier values by asynchronous copies, constants in the constant bank,
// paired polarisations) 256 x 2 with the sums in registers 0.4125 ms,
// against 0.4214 ms in shared memory (0.583 ms with each add a
// shared-memory atomic); later, at 0.399 ms for 256 x 2: 128 x 4 0.416 ms,
// 192 x 2 0.421 ms, 128 x 3 0.450 ms, 224 x 2 0.453 ms, 288 x 2 0.490 ms; before the pairing, with 12 more live registers,
// the shared-memory sums were ahead (0.491 against 0.51 ms), and 3 CTAs per
// SM ran 0.77 ms, 128 x 4 0.55 ms.
FusedShape fusedShape(const GeneratedModel& gen)
{
    FusedShape sh;
    auto get = [](const char* name, int def, int lo, int hi) {
        const char* e = std::getenv(name);
        if (!e || !*e) return def;
        int v = std::atoi(e);
        if (v < lo || v > hi) throw std::runtime_error(std::string(name) + " out of range");
        return v;
    };
    sh.block[0] = get("CTPWA_F64_BLOCK", 192, 32, 1024);
    sh.minb[0] = get("CTPWA_F64_MINB", 2, 1, 16);
    sh.block[1] = get("CTPWA_MX_BLOCK", 256, 32, 1024);
    sh.minb[1] = get("CTPWA_MX_MINB", 2, 1, 16);
    sh.acc[0] = get("CTPWA_F64_ACC_SMEM", 1, 0, 1);
    sh.acc[1] = get("CTPWA_MX_ACC_SMEM", 0, 0, 1);

    for (int i = 0; i < 2; ++i)
        if (sh.block[i] % 32) throw std::runtime_error("fused block sizes must be multiples of 32");
    // Staging of the event tables through shared memory, used when its two
    // buffers fit at the requested residency next to the static shared
    // memory: 1 the frontier rows and 2 the frontier and angular rows, by
    // per-warp bulk copies of 32-event tiles; 3 the frontier values by
    // per-thread asynchronous copies of the next event's values. CTPWA_STAGE
    // sets it for both kernels. Default: 3 for the mixed form (K+K-pi0:
    // 0.52-0.53 ms, against 0.63 ms direct, 0.744 ms with mode 1 and 1.10 ms
    // with mode 2 at 1 CTA per SM), off for the plain path (its gradient-sum
    // slots leave no room for the buffers at 2 CTAs per SM; with the slots
    // in registers instead, mode 3 measured 1.39 ms against 1.15 ms).
    const int st = get("CTPWA_STAGE", -1, 0, 3);
    const int stage_req[2] = {st >= 0 ? st : 0, st >= 0 ? st : 3};
    const long long rowb[2] = {16, 8};  // bytes per complex angular value (FP64, FP32)
    const long long accb[2] = {8, 4};   // bytes per gradient sum (FP64, FP32)
    const long long per_sm = 228LL * 1024, per_cta = 227LL * 1024, reserve = 8LL * 1024;
    auto fits = [&](int i, long long bytes) {
        return bytes + reserve <= per_cta && (long long)sh.minb[i] * (bytes + reserve) <= per_sm;
    };
    for (int i = 0; i < 2; ++i) {
        // dynamic shared memory = [gradient-sum slots][two tile buffers]
        long long acc_bytes = sh.acc[i] ? (gen.ngrad * sh.block[i] * accb[i] + 127) / 128 * 128 : 0;
        if (!fits(i, acc_bytes)) {
            sh.acc[i] = 0;
            acc_bytes = 0;
        }
        long long npl = (long long)std::max(1, gen.nplane) * std::max(1, gen.npol);
        if (i == 1) npl = (npl + 1) / 2 * 2;  // FP32 angular records of an even number of values
        const long long evb = i == 0 ? 8LL * gen.nev64 : 4LL * evfStride(gen) + 8LL * gen.nevd;  // frontier bytes per event
        const int stage_on = stage_req[i];
        long long stage_bytes = 2LL * ((stage_on == 2 ? npl * rowb[i] : 0) + evb) * sh.block[i];
        if (stage_on == 3) {
            // [2][NA][block] values of the table's type (16-byte rounded), then [2][NB][block] FP64
            const long long na = i == 0 ? gen.nev64 : evfStride(gen), nb = i == 0 ? 0 : gen.nevd, sz = i == 0 ? 8 : 4;
            stage_bytes = (2LL * std::max(1LL, na) * sh.block[i] * sz + 15) / 16 * 16 + 2LL * nb * sh.block[i] * 8;
        }
        if (stage_on && fits(i, acc_bytes + stage_bytes)) sh.stage[i] = stage_on;
        sh.dsmem[i] = (int)(acc_bytes + (sh.stage[i] ? stage_bytes : 0));
    }
    return sh;
}

// NVRTC compile of one program (main source + named headers) for sm_100a, with
// a disk cache keyed by the FNV-1a hash of the main source, the header texts,
// the options and the NVRTC version.
std::string nvrtcCubin(const std::string& src, const std::vector<std::pair<std::string, std::string>>& headers,
                       const std::vector<std::string>& optv, const char* what, bool* cache_hit)
{
    std::vector<const char*> optp;
    for (const auto& o : optv) optp.push_back(o.c_str());
    const char* const* opts = optp.data();
    const int nopts = (int)optp.size();
    std::string key_src = src;  // the main source too: the angular module's is the generated code
    for (const auto& h : headers) key_src += h.second;
    for (int i = 0; i < nopts; ++i) key_src += opts[i];
    int nvmaj = 0, nvmin = 0;
    nvrtcVersion(&nvmaj, &nvmin);
    key_src += std::to_string(nvmaj) + "." + std::to_string(nvmin);
    char key[32];
    std::snprintf(key, sizeof key, "%016llx", (unsigned long long)fnv1a(key_src));
    // process-wide copy of the cubins already read or compiled, by the full
    // key text (handles of one model share them)
    static std::mutex mem_mu;
    static std::map<std::string, std::string> mem;
    {
        std::lock_guard<std::mutex> lk(mem_mu);
        auto it = mem.find(key_src);
        if (it != mem.end()) {
            if (cache_hit) *cache_hit = true;
            return it->second;
        }
    }
    auto remember = [&](const std::string& c) {
        std::lock_guard<std::mutex> lk(mem_mu);
        if (mem.size() >= 32) mem.clear();
        mem.emplace(key_src, c);
    };
    std::string cpath = cacheDir() + "/" + key + ".cubin";
    std::string cubin;
    {
        std::ifstream f(cpath, std::ios::binary);
        if (f) {
            std::stringstream ss;
            ss << f.rdbuf();
            cubin = ss.str();
        }
    }
    if (cache_hit) *cache_hit = !cubin.empty();
    if (!cubin.empty()) {
        remember(cubin);
        return cubin;
    }
    std::vector<const char*> hdr_src, hdr_names;
    for (const auto& h : headers) {
        hdr_names.push_back(h.first.c_str());
        hdr_src.push_back(h.second.c_str());
    }
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), "ctpwa_fused.cu", (int)headers.size(), hdr_src.data(), hdr_names.data()) !=
        NVRTC_SUCCESS)
        throw std::runtime_error("NVRTC: program creation failed");
    nvrtcResult r = nvrtcCompileProgram(prog, nopts, opts);
    if (r != NVRTC_SUCCESS) {
        size_t ls2 = 0;
        nvrtcGetProgramLogSize(prog, &ls2);
        std::string log(ls2, '\0');
        nvrtcGetProgramLog(prog, &log[0]);
        nvrtcDestroyProgram(&prog);
        throw std::runtime_error(std::string("NVRTC compile of the ") + what + " failed:\n" + log.substr(0, 4000));
    }
    size_t n = 0;
    nvrtcGetCUBINSize(prog, &n);
    cubin.resize(n);
    nvrtcGetCUBIN(prog, &cubin[0]);
    nvrtcDestroyProgram(&prog);
    std::error_code ec;
    std::filesystem::create_directories(cacheDir(), ec);
    std::string tmpp = cpath + ".tmp" + std::to_string((long long)getpid());
    {
        std::ofstream f(tmpp, std::ios::binary);
        f.write(cubin.data(), (std::streamsize)cubin.size());
    }
    std::filesystem::rename(tmpp, cpath, ec);
    remember(cubin);
    return cubin;
}

const std::vector<std::string> kNvrtcBase = {"--gpu-architecture=sm_100a", "-std=c++17", "-default-device",
                                             "-DCT_BLOCK=256", "--fmad=true", "-lineinfo"};

// The fused likelihood kernels of one generated model.
std::string jitCubin(const GeneratedModel& gen, bool* cache_hit)
{
    std::string dir = kernelDir();
    std::vector<std::string> optv = kNvrtcBase;
    // tuning knobs: block size and minimum resident CTAs per SM of the fused kernels
    const FusedShape sh = fusedShape(gen);
    optv.push_back("-DCT_F64_ACC=" + std::to_string(sh.acc[0]));
    optv.push_back("-DCT_MX_ACC=" + std::to_string(sh.acc[1]));
    optv.push_back("-DCT_F64_STAGE=" + std::to_string(sh.stage[0]));
    optv.push_back("-DCT_MX_STAGE=" + std::to_string(sh.stage[1]));

    optv.push_back("-DCT_F64_BLOCK=" + std::to_string(sh.block[0]));
    optv.push_back("-DCT_F64_MINB=" + std::to_string(sh.minb[0]));
    optv.push_back("-DCT_MX_BLOCK=" + std::to_string(sh.block[1]));
    optv.push_back("-DCT_MX_MINB=" + std::to_string(sh.minb[1]));
    return nvrtcCubin("#include \"fused_nll.cuh\"\n",
                      {{"device_helpers.cuh", readFile(dir + "/device_helpers.cuh")},
                       {"fused_nll.cuh", readFile(dir + "/fused_nll.cuh")},
                       {"model.cuh", gen.header}},
                      optv, "fused kernel", cache_hit);
}

// Block size of the Hessian-vector-product kernel: per-thread tangent sums
// live in shared memory (ngrad + 2 doubles a thread), kept under 96 KiB.
int hvpBlock(const GeneratedModel& gen)
{
    int b = 128;
    while (b > 32 && (long long)(gen.ngrad + 2) * b * 8 > 96LL * 1024) b /= 2;
    return b;
}

// The Hessian-vector-product kernels of one generated model.
std::string jitHvpCubin(const GeneratedModel& gen, bool paired, bool* cache_hit)
{
    std::string dir = kernelDir();
    std::vector<std::string> optv = kNvrtcBase;
    optv.push_back("-DCT_HVP_BLOCK=" + std::to_string(hvpBlock(gen)));
    optv.push_back(std::string("-DCT_HVP_PAIRED=") + (paired ? "1" : "0"));
    return nvrtcCubin("#include \"hessian.cuh\"\n",
                      {{"device_helpers.cuh", readFile(dir + "/device_helpers.cuh")},
                       {"hessian.cuh", readFile(dir + "/hessian.cuh")},
                       {"model.cuh", gen.header},
                       {"model_dual.cuh", gen.dual_header}},
                      optv, "Hessian kernel", cache_hit);
}

// The tensor-core Gram kernels of one generated model (kernels/gram.cuh).
std::string jitGramCubin(const GeneratedModel& gen, bool paired, bool* cache_hit, bool hess = false)
{
    std::string dir = kernelDir();
    std::vector<std::string> optv = kNvrtcBase;
    optv.push_back(std::string("-DCT_GRAM_PAIRED=") + (paired ? "1" : "0"));
    if (hess) optv.push_back("-DCT_GRAM_HESS=1");
    return nvrtcCubin("#include \"gram.cuh\"\n",
                      {{"device_helpers.cuh", readFile(dir + "/device_helpers.cuh")},
                       {"fused_nll.cuh", readFile(dir + "/fused_nll.cuh")},
                       {"gram.cuh", readFile(dir + "/gram.cuh")},
                       {"model.cuh", gen.header}},
                      optv, "Gram kernel", cache_hit);
}

// The normalisation-cache kernels of one model (kernels/norm.cuh).
std::string jitNormCubin(const GeneratedModel& gen, bool* cache_hit)
{
    std::string dir = kernelDir();
    return nvrtcCubin("#include \"norm.cuh\"\n",
                      {{"device_helpers.cuh", readFile(dir + "/device_helpers.cuh")},
                       {"fused_nll.cuh", readFile(dir + "/fused_nll.cuh")},
                       {"norm.cuh", readFile(dir + "/norm.cuh")},
                       {"model.cuh", gen.header}},
                      kNvrtcBase, "normalisation kernel", cache_hit);
}

// The generated angular kernels of one model (angularSource).
std::string jitAngularCubin(const std::string& src, bool* cache_hit)
{
    std::string dir = kernelDir();
    return nvrtcCubin(src, {{"angular_gen.cuh", readFile(dir + "/angular_gen.cuh")}}, kNvrtcBase, "angular kernel",
                      cache_hit);
}

// CTPWA_ANGULAR_INTERP=1: the angular tables from the interpreter
// (ag_group_kernel) instead of the generated kernels
bool angularInterpreted()
{
    const char* e = std::getenv("CTPWA_ANGULAR_INTERP");
    return e && *e && *e != '0';
}

void Engine::compileKernel()
{
    auto t0 = std::chrono::steady_clock::now();
    std::string cubin = jitCubin(gen_, &jit_cache_hit_);
    cudaLibrary_t lib;
    CT_CUDA(cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
    lib_ = (void*)lib;
    cudaKernel_t k64, kmx, kin, kpro;
    CT_CUDA(cudaLibraryGetKernel(&kpro, lib, "ct_prologue"));
    k_pro_ = (void*)kpro;
    cudaKernel_t kevc;
    CT_CUDA(cudaLibraryGetKernel(&kevc, lib, "ct_event_cache"));
    k_evc_ = (void*)kevc;
    CT_CUDA(cudaLibraryGetGlobal(&k_sym_, &k_sym_bytes_, lib, "ct_k"));
    CT_CUDA(cudaLibraryGetKernel(&k64, lib, "ct_fused_f64"));
    CT_CUDA(cudaLibraryGetKernel(&kmx, lib, "ct_fused_mixed"));
    cudaKernel_t k64p, kmxp;
    CT_CUDA(cudaLibraryGetKernel(&k64p, lib, "ct_fused_f64_pc"));
    CT_CUDA(cudaLibraryGetKernel(&kmxp, lib, "ct_fused_mixed_pc"));
    k_pc_[0] = (void*)k64p;
    k_pc_[1] = (void*)kmxp;
    CT_CUDA(cudaLibraryGetKernel(&kin, lib, "ct_intensity_f64"));
    cudaKernel_t kpart, kexp;
    CT_CUDA(cudaLibraryGetKernel(&kpart, lib, "ct_partials_f64"));
    k_part_ = (void*)kpart;
    CT_CUDA(cudaLibraryGetKernel(&kexp, lib, "ct_export_f64"));
    k_exp_ = (void*)kexp;
    k_f64_ = (void*)k64;
    k_mixed_ = (void*)kmx;
    // multi-job variants [precision][paired]
    const char* multi_names[2][2] = {{"ct_fused_f64_multi", "ct_fused_f64_pc_multi"},
                                     {"ct_fused_mixed_multi", "ct_fused_mixed_pc_multi"}};
    for (int pr = 0; pr < 2; ++pr)
        for (int pc = 0; pc < 2; ++pc) {
            cudaKernel_t km;
            CT_CUDA(cudaLibraryGetKernel(&km, lib, multi_names[pr][pc]));
            k_multi_[pr][pc] = (void*)km;
        }
    cudaKernel_t kprom;
    CT_CUDA(cudaLibraryGetKernel(&kprom, lib, "ct_prologue_multi"));
    k_pro_multi_ = (void*)kprom;
    for (int pr = 0; pr < 2; ++pr)
        if (shape_.dsmem[pr] > 0)
            for (void* k : {pr == 0 ? k_f64_ : k_mixed_, k_pc_[pr], k_multi_[pr][0], k_multi_[pr][1]})
                CT_CUDA(cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, shape_.dsmem[pr]));
    k_int_ = (void*)kin;
    {
        std::string key = gen_.header;
        for (int pr = 0; pr < 2; ++pr)
            key += "|" + std::to_string(shape_.block[pr]) + "," + std::to_string(shape_.minb[pr]) + "," +
                   std::to_string(shape_.dsmem[pr]);
        image_key_ = (const void*)(uintptr_t)fnv1a(key);
    }
    jit_seconds_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

double precompileConfig(const std::string& config_path)
{
    auto t0 = std::chrono::steady_clock::now();
    Config cfg = loadConfig(config_path);
    if (!cfg.valid()) throw std::runtime_error("analysis not initialized: invalid or missing config file \"" + config_path + "\"");
    Model m = buildModel(cfg, 1);
    GeneratedModel g = generateModel(m);
    // CTPWA_MODEL_SOURCE_OUT=<file>: also write the generated model header
    // (the CUDA source the kernels include) for inspection
    if (const char* out = std::getenv("CTPWA_MODEL_SOURCE_OUT"); out && *out) {
        std::ofstream f(out);
        f << g.header;
        if (!f) throw std::runtime_error(std::string("cannot write ") + out);
    }
    bool hit = false;
    jitCubin(g, &hit);
    jitHvpCubin(g, false, &hit);
    if (g.nterm + g.nder <= 256 && (size_t)(2 * g.nterm + g.nder) * g.nterm * 16 <= 40000) jitNormCubin(g, &hit);
    {
        std::vector<AgNodeVar> vars;
        std::vector<double> cg;
        const std::vector<AgGroupHost> gh = angularGroups(m, g, vars, cg);
        if (!gh.empty()) {
            const std::string src = angularSource(gh, vars, g.nplane);
            if (const char* out = std::getenv("CTPWA_MODEL_SOURCE_OUT"); out && *out) {
                std::ofstream f(std::string(out) + ".angular.cu");
                f << src;
            }
            jitAngularCubin(src, &hit);
        }
    }
    if (m.npol * 2 * m.nAmp() <= 128) {
        jitGramCubin(g, false, &hit);
        jitGramCubin(g, true, &hit);
    }
    if ((m.npol + 1) * 2 * m.nAmp() <= 128) {
        jitGramCubin(g, false, &hit, true);
        jitGramCubin(g, true, &hit, true);
    }
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// argument block of the fused kernel (must match CtArgs in kernels/fused_nll.cuh)
struct CtSampleH {
    const void* slamp;
    const void* ev;
    const double* evd;
    const double* w;
    long long n;
    long long ld;
    int kind;
    int cta_begin;
    int cta_count;
    int pad;
    double vw_scale;
};
struct CtArgsH {
    CtSampleH s[3];
    int nsamp;
    int pad;
    const double* theta;
    const double* v;
    double* partials;
    double* consts;
    int cta_base;
    int pad2;
    int* err;
    void* kblock;
};

void Engine::nllGrad(const double* d_params, double* d_nll, double* d_grad, int precision, cudaStream_t stream)
{
    const CtaLayout& lay = lay_[precision == kMixed ? 1 : 0];
    const Model& m = model_;
    int nA = m.nAmp(), nc = m.nVector(), nT = m.nTheta();
    ct_prepare_kernel<<<(nA + 127) / 128, 128, 0, stream>>>(d_params, d_amp_chain_, d_ratio_, nA, nc, d_v_, d_err_);
    CT_CUDA(cudaGetLastError());
    CtArgsH a;
    std::memset(&a, 0, sizeof(a));
    int ns = 0;
    for (int k = 0; k < 3; ++k) {
        if (lay.cta[k][1] == 0) continue;
        CtSampleH& s = a.s[ns++];
        const DeviceSample& d = samples_[k];
        s.slamp = precision == kMixed ? (const void*)d.slamp32 : (paired_[0] ? (const void*)d.slamp64p : (const void*)d.slamp64);
        s.ev = precision == kMixed ? (const void*)d.evf : (const void*)d.ev64;
        s.evd = precision == kMixed ? d.evd : nullptr;
        s.w = d.w;
        s.n = d.n;
        s.ld = d.ld;
        s.kind = k;
        s.cta_begin = lay.cta[k][0];
        s.cta_count = lay.cta[k][1];
        s.vw_scale = 1.0 / (samples_[0].wsum > 0 ? samples_[0].wsum : 1.0);
    }
    a.nsamp = ns;
    a.theta = d_params + 2 * nc;
    a.v = d_v_;
    a.partials = d_partials_;
    a.consts = d_consts_;
    a.err = d_err_;
    a.kblock = d_kblock_;
    if (precision == kMixed && !samples_[0].slamp32) throw std::runtime_error("mixed-precision tables were not built");
    void* args[] = {&a};
    CT_CUDA(cudaLaunchKernel(k_pro_, dim3(1), dim3(32), args, 0, stream));
    CT_CUDA(cudaMemcpyAsync(k_sym_, d_kblock_, k_sym_bytes_, cudaMemcpyDeviceToDevice, stream));
    const size_t slot = ev_begin_.empty() ? 0 : (size_t)(ev_count_ % (long long)ev_begin_.size());
    if (!ev_begin_.empty()) CT_CUDA(cudaEventRecord(ev_begin_[slot], stream));
    a.cta_base = 0;
    CT_CUDA(cudaLaunchKernel(precision == kMixed ? k_mixed_ : k_f64_, dim3(lay.grid), dim3(shape_.block[precision == kMixed]),
                             args, (size_t)shape_.dsmem[precision == kMixed], stream));
    if (!ev_begin_.empty()) {
        CT_CUDA(cudaEventRecord(ev_end_[slot], stream));
        ++ev_count_;
    }
    FinalizeArgs f;
    std::memset(&f, 0, sizeof(f));
    f.partials = d_partials_;
    f.nacc = 2 + 2 * nA + nT;
    f.nA = nA;
    f.nc = nc;
    f.nT = nT;
    for (int k = 0; k < 3; ++k) {
        f.cta[k][0] = lay.cta[k][0];
        f.cta[k][1] = lay.cta[k][1];
        f.has[k] = lay.cta[k][1] > 0;
    }
    f.n_phsp = (double)samples_[0].n;
    f.W_data = samples_[1].wsum;
    f.W_bkg = has_bkg_ ? samples_[2].wsum : 0.0;
    f.params = d_params;
    f.v = d_v_;
    f.chain = d_amp_chain_;
    f.gauss_idx = d_gauss_idx_;
    f.gauss_ms = d_gauss_ms_;
    f.ngauss = (int)m.gauss.size();
    f.out_nll = d_nll;
    f.out_grad = d_grad;
    f.out_parts = d_parts_;
    f.err = d_err_;
    f.vshift = precision == kMixed ? 1 : 0;
    size_t shm = ct_finalize_shm(f);
    ct_finalize_kernel<<<1, 1024, shm, stream>>>(f);
    CT_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Several jobs of one model in one evaluation (serving): one prepare, one
// prologue, one fused and one finalize launch for all of them. Each job keeps
// its own grid of CTAs, partial rows and finalize, so its results are those
// of its own nllGrad, bit for bit; only the per-call constants come from the
// job's image in global memory instead of the constant bank.
// ---------------------------------------------------------------------------
MultiScratch::~MultiScratch()
{
    if (host) cudaFreeHost(host);
    if (dev) cudaFreeAsync(dev, 0);
    if (copied) cudaEventDestroy(copied);
}

void Engine::nllGradMulti(const std::vector<Engine*>& es, const std::vector<const double*>& d_params,
                          const std::vector<double*>& d_nll, const std::vector<double*>& d_grad, int precision,
                          MultiScratch& sc, cudaStream_t stream)
{
    const int nj = (int)es.size();
    if (nj == 0) return;
    if (d_params.size() != es.size() || d_nll.size() != es.size() || d_grad.size() != es.size())
        throw std::invalid_argument("multi evaluation: one parameter, NLL and gradient pointer per job");
    Engine* e0 = es[0];
    const int pr = precision == kMixed ? 1 : 0;
    for (Engine* e : es) {
        if (e->opt_.device != e0->opt_.device)
            throw std::invalid_argument("multi evaluation: all jobs must be on one device");
        if (e->kernelImageKey() != e0->kernelImageKey() ||
            e->shape_.block[pr] != e0->shape_.block[pr] || e->shape_.dsmem[pr] != e0->shape_.dsmem[pr])
            throw std::invalid_argument("multi evaluation: all jobs must share one model (generated kernel) and layout");
        if (precision == kMixed && !e->samples_[0].slamp32)
            throw std::runtime_error("mixed-precision tables were not built");
    }
    // staging: [CtArgsH x nj][PrepareArgs x nj][FinalizeArgs x nj][cta_off x (nj + 1)]
    auto up = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t o_args = 0, o_prep = up(sizeof(CtArgsH) * nj), o_fin = o_prep + up(sizeof(PrepareArgs) * nj),
                 o_off = o_fin + up(sizeof(FinalizeArgs) * nj), bytes = o_off + up(sizeof(int) * (nj + 1));
    if (!sc.copied) CT_CUDA(cudaEventCreateWithFlags(&sc.copied, cudaEventDisableTiming));
    CT_CUDA(cudaEventSynchronize(sc.copied));  // the previous call's copy has left the host buffer
    if (bytes > sc.cap) {
        if (sc.host) cudaFreeHost(sc.host);
        if (sc.dev) cudaFreeAsync(sc.dev, stream);
        sc.host = nullptr;
        sc.dev = nullptr;
        CT_CUDA(cudaMallocHost(&sc.host, bytes));
        CT_CUDA(cudaMallocAsync(&sc.dev, bytes, stream));
        sc.cap = bytes;
    }
    unsigned char* hb = (unsigned char*)sc.host;
    unsigned char* db = (unsigned char*)sc.dev;
    CtArgsH* ha = (CtArgsH*)(hb + o_args);
    PrepareArgs* hp = (PrepareArgs*)(hb + o_prep);
    FinalizeArgs* hf = (FinalizeArgs*)(hb + o_fin);
    int* hoff = (int*)(hb + o_off);
    int total = 0, shm_max = 0;
    for (int j = 0; j < nj; ++j) {
        Engine* e = es[j];
        const CtaLayout& lay = e->lay_[pr];
        const Model& m = e->model_;
        const int nA = m.nAmp(), nc = m.nVector(), nT = m.nTheta();
        hoff[j] = total;
        CtArgsH& a = ha[j];
        std::memset(&a, 0, sizeof(a));
        int ns = 0;
        for (int k = 0; k < 3; ++k) {
            if (lay.cta[k][1] == 0) continue;
            CtSampleH& smp = a.s[ns++];
            const DeviceSample& d = e->samples_[k];
            smp.slamp = pr ? (const void*)d.slamp32 : (e->paired_[0] ? (const void*)d.slamp64p : (const void*)d.slamp64);
            smp.ev = pr ? (const void*)d.evf : (const void*)d.ev64;
            smp.evd = pr ? d.evd : nullptr;
            smp.w = d.w;
            smp.n = d.n;
            smp.ld = d.ld;
            smp.kind = k;
            smp.cta_begin = lay.cta[k][0];
            smp.cta_count = lay.cta[k][1];
            smp.vw_scale = 1.0 / (e->samples_[0].wsum > 0 ? e->samples_[0].wsum : 1.0);
        }
        a.nsamp = ns;
        a.theta = d_params[j] + 2 * nc;
        a.v = e->d_v_;
        a.partials = e->d_partials_;
        a.consts = e->d_consts_;
        a.err = e->d_err_;
        a.kblock = e->d_kblock_;
        a.cta_base = -total;
        hp[j] = PrepareArgs{d_params[j], e->d_amp_chain_, e->d_ratio_, nA, nc, e->d_v_, e->d_err_};
        FinalizeArgs& f = hf[j];
        std::memset(&f, 0, sizeof(f));
        f.partials = e->d_partials_;
        f.nacc = 2 + 2 * nA + nT;
        f.nA = nA;
        f.nc = nc;
        f.nT = nT;
        for (int k = 0; k < 3; ++k) {
            f.cta[k][0] = lay.cta[k][0];
            f.cta[k][1] = lay.cta[k][1];
            f.has[k] = lay.cta[k][1] > 0;
        }
        f.n_phsp = (double)e->samples_[0].n;
        f.W_data = e->samples_[1].wsum;
        f.W_bkg = e->has_bkg_ ? e->samples_[2].wsum : 0.0;
        f.params = d_params[j];
        f.v = e->d_v_;
        f.chain = e->d_amp_chain_;
        f.gauss_idx = e->d_gauss_idx_;
        f.gauss_ms = e->d_gauss_ms_;
        f.ngauss = (int)m.gauss.size();
        f.out_nll = d_nll[j];
        f.out_grad = d_grad[j];
        f.out_parts = e->d_parts_;
        f.err = e->d_err_;
        f.vshift = pr;
        shm_max = std::max(shm_max, (int)ct_finalize_shm(f));
        total += lay.grid;
    }
    hoff[nj] = total;
    CT_CUDA(cudaMemcpyAsync(db, hb, bytes, cudaMemcpyHostToDevice, stream));
    CT_CUDA(cudaEventRecord(sc.copied, stream));
    ct_prepare_multi_kernel<<<nj, 128, 0, stream>>>((const PrepareArgs*)(db + o_prep));
    CT_CUDA(cudaGetLastError());
    const CtArgsH* dargs = (const CtArgsH*)(db + o_args);
    void* pargs[] = {&dargs};
    CT_CUDA(cudaLaunchKernel(e0->k_pro_multi_, dim3(nj), dim3(32), pargs, 0, stream));
    const int* doff = (const int*)(db + o_off);
    int njobs = nj;
    void* fargs[] = {&dargs, &doff, &njobs};
    CT_CUDA(cudaLaunchKernel(e0->k_multi_[pr][e0->paired_[pr] ? 1 : 0], dim3(total), dim3(e0->shape_.block[pr]), fargs,
                             (size_t)e0->shape_.dsmem[pr], stream));
    ct_finalize_multi_kernel<<<nj, 1024, shm_max, stream>>>((const FinalizeArgs*)(db + o_fin));
    CT_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Allocation-free evaluation: scratch in a fixed array of this library.
//
// Every GPU that loads the library holds this 2 MiB array until the process
// exits. Host code may not use the symbol's name as a device address (it names
// a host-side stand-in); the address comes from cudaGetSymbolAddress, once per
// device, with that device current, the first time a handle on the device
// calls nllGradStatic. That first call should therefore come before any stream
// capture is begun on the device.
//
// Every call writes all of the scratch it later reads (couplings by
// ct_prepare_kernel, constants by ct_prologue, one full partial row per CTA,
// the parts by ct_finalize_kernel), so nothing has to start at zero. All
// handles on a device share the array and it keeps the last call's contents:
// calls whose GPU work overlaps (different streams, threads or handles
// without ordering between them) race on it.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_ct_static_scratch[Engine::kStaticScratchBytes / sizeof(double)];

namespace {

double* staticScratchAddress(int device)
{
    static std::mutex mu;
    static std::vector<double*> addr;
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0) throw std::runtime_error("static scratch: bad device");
    if ((size_t)device >= addr.size()) addr.resize((size_t)device + 1, nullptr);
    if (addr[device]) return addr[device];
    int prev = -1;
    CT_CUDA(cudaGetDevice(&prev));
    CT_CUDA(cudaSetDevice(device));
    double* p = nullptr;
    cudaError_t rc = cudaGetSymbolAddress((void**)&p, g_ct_static_scratch);
    cudaError_t rc2 = cudaSetDevice(prev);
    if (rc != cudaSuccess)
        throw std::runtime_error(std::string("static scratch: cudaGetSymbolAddress failed: ") + cudaGetErrorString(rc));
    if (rc2 != cudaSuccess)
        throw std::runtime_error(std::string("static scratch: cudaSetDevice failed: ") + cudaGetErrorString(rc2));
    addr[device] = p;
    return p;
}

}  // namespace

void Engine::nllGradStatic(const double* d_params, double* d_nll, double* d_grad, int precision, cudaStream_t stream)
{
    const CtaLayout& lay = lay_[precision == kMixed ? 1 : 0];
    const Model& m = model_;
    const int nA = m.nAmp(), nc = m.nVector(), nT = m.nTheta();
    const int nacc = 2 + 2 * nA + nT;
    // layout in doubles, each part on a 256-byte boundary
    auto up = [](size_t x) { return (x + 31) / 32 * 32; };
    const size_t off_v = 0;
    const size_t off_c = off_v + up((size_t)2 * nA);
    const size_t off_p = off_c + up((size_t)std::max(1, gen_.nconst));
    const size_t off_parts = off_p + up((size_t)lay.grid * nacc);
    const size_t off_err = off_parts + 8;  // one int (copy-timeout flag), cleared by ct_prepare_kernel
    const size_t off_k = up(off_err + 1);  // constant-bank image of this call
    const size_t need = off_k + up((k_sym_bytes_ + 7) / 8);
    const size_t cap = kStaticScratchBytes / sizeof(double);
    if (need > cap)
        throw std::length_error("ctpwa_nll_grad_static: this model needs " + std::to_string(need * sizeof(double)) +
                                " bytes of scratch (" + std::to_string(lay.grid) + " CTA rows of " + std::to_string(nacc) +
                                " sums), more than the fixed " + std::to_string(kStaticScratchBytes) +
                                " bytes; use ctpwa_nll_grad");
    double* base = staticScratchAddress(opt_.device);
    double* s_v = base + off_v;
    double* s_consts = base + off_c;
    double* s_partials = base + off_p;
    double* s_parts = base + off_parts;

    ct_prepare_kernel<<<(nA + 127) / 128, 128, 0, stream>>>(d_params, d_amp_chain_, d_ratio_, nA, nc, s_v, (int*)(base + off_err));
    CT_CUDA(cudaGetLastError());
    CtArgsH a;
    std::memset(&a, 0, sizeof(a));
    int ns = 0;
    for (int k = 0; k < 3; ++k) {
        if (lay.cta[k][1] == 0) continue;
        CtSampleH& sm = a.s[ns++];
        const DeviceSample& d = samples_[k];
        sm.slamp = precision == kMixed ? (const void*)d.slamp32 : (paired_[0] ? (const void*)d.slamp64p : (const void*)d.slamp64);
        sm.ev = precision == kMixed ? (const void*)d.evf : (const void*)d.ev64;
        sm.evd = precision == kMixed ? d.evd : nullptr;
        sm.w = d.w;
        sm.n = d.n;
        sm.ld = d.ld;
        sm.kind = k;
        sm.cta_begin = lay.cta[k][0];
        sm.cta_count = lay.cta[k][1];
        sm.vw_scale = 1.0 / (samples_[0].wsum > 0 ? samples_[0].wsum : 1.0);
    }
    a.nsamp = ns;
    a.theta = d_params + 2 * nc;
    a.v = s_v;
    a.partials = s_partials;
    a.consts = s_consts;
    a.err = (int*)(base + off_err);
    a.kblock = base + off_k;
    if (precision == kMixed && !samples_[0].slamp32) throw std::runtime_error("mixed-precision tables were not built");
    void* args[] = {&a};
    CT_CUDA(cudaLaunchKernel(k_pro_, dim3(1), dim3(32), args, 0, stream));
    CT_CUDA(cudaMemcpyAsync(k_sym_, base + off_k, k_sym_bytes_, cudaMemcpyDeviceToDevice, stream));
    a.cta_base = 0;
    CT_CUDA(cudaLaunchKernel(precision == kMixed ? k_mixed_ : k_f64_, dim3(lay.grid), dim3(shape_.block[precision == kMixed]),
                             args, (size_t)shape_.dsmem[precision == kMixed], stream));
    FinalizeArgs f;
    std::memset(&f, 0, sizeof(f));
    f.partials = s_partials;
    f.nacc = nacc;
    f.nA = nA;
    f.nc = nc;
    f.nT = nT;
    for (int k = 0; k < 3; ++k) {
        f.cta[k][0] = lay.cta[k][0];
        f.cta[k][1] = lay.cta[k][1];
        f.has[k] = lay.cta[k][1] > 0;
    }
    f.n_phsp = (double)samples_[0].n;
    f.W_data = samples_[1].wsum;
    f.W_bkg = has_bkg_ ? samples_[2].wsum : 0.0;
    f.params = d_params;
    f.v = s_v;
    f.chain = d_amp_chain_;
    f.gauss_idx = d_gauss_idx_;
    f.gauss_ms = d_gauss_ms_;
    f.ngauss = (int)m.gauss.size();
    f.out_nll = d_nll;
    f.out_grad = d_grad;
    f.out_parts = s_parts;
    f.err = (const int*)(base + off_err);
    f.vshift = precision == kMixed ? 1 : 0;
    size_t shm = ct_finalize_shm(f);
    ct_finalize_kernel<<<1, 1024, shm, stream>>>(f);
    CT_CUDA(cudaGetLastError());
}

void Engine::shardSums(const double* d_params, int precision, double* d_sums, cudaStream_t stream)
{
    sums_mixed_ = precision == kMixed;
    const CtaLayout& lay = lay_[precision == kMixed ? 1 : 0];
    const Model& m = model_;
    const int nA = m.nAmp(), nc = m.nVector(), nT = m.nTheta();
    const int nacc = 2 + 2 * nA + nT;
    ct_prepare_kernel<<<(nA + 127) / 128, 128, 0, stream>>>(d_params, d_amp_chain_, d_ratio_, nA, nc, d_v_, d_err_);
    CT_CUDA(cudaGetLastError());
    CtArgsH a;
    std::memset(&a, 0, sizeof(a));
    int ns = 0;
    for (int k = 0; k < 3; ++k) {
        if (lay.cta[k][1] == 0) continue;
        CtSampleH& sm = a.s[ns++];
        const DeviceSample& d = samples_[k];
        sm.slamp = precision == kMixed ? (const void*)d.slamp32 : (paired_[0] ? (const void*)d.slamp64p : (const void*)d.slamp64);
        sm.ev = precision == kMixed ? (const void*)d.evf : (const void*)d.ev64;
        sm.evd = precision == kMixed ? d.evd : nullptr;
        sm.w = d.w;
        sm.n = d.n;
        sm.ld = d.ld;
        sm.kind = k;
        sm.cta_begin = lay.cta[k][0];
        sm.cta_count = lay.cta[k][1];
        sm.vw_scale = 1.0;  // the phase-space weight total is global: applied after the sums are combined
    }
    a.nsamp = ns;
    a.theta = d_params + 2 * nc;
    a.v = d_v_;
    a.partials = d_partials_;
    a.consts = d_consts_;
    a.err = d_err_;
    a.kblock = d_kblock_;
    if (precision == kMixed && !samples_[0].slamp32) throw std::runtime_error("mixed-precision tables were not built");
    void* args[] = {&a};
    CT_CUDA(cudaLaunchKernel(k_pro_, dim3(1), dim3(32), args, 0, stream));
    CT_CUDA(cudaMemcpyAsync(k_sym_, d_kblock_, k_sym_bytes_, cudaMemcpyDeviceToDevice, stream));
    a.cta_base = 0;
    CT_CUDA(cudaLaunchKernel(precision == kMixed ? k_mixed_ : k_f64_, dim3(lay.grid), dim3(shape_.block[precision == kMixed]),
                             args, (size_t)shape_.dsmem[precision == kMixed], stream));
    FinalizeArgs f;
    std::memset(&f, 0, sizeof(f));
    for (int k = 0; k < 3; ++k) {
        f.cta[k][0] = lay.cta[k][0];
        f.cta[k][1] = lay.cta[k][1];
        f.has[k] = lay.cta[k][1] > 0;
    }
    f.n_phsp = (double)samples_[0].n;
    f.W_data = samples_[1].wsum;
    f.W_bkg = has_bkg_ ? samples_[2].wsum : 0.0;
    ct_rowsum_kernel<<<1, 1024, sizeof(double) * 32 * (size_t)nacc, stream>>>(d_partials_, nacc, f, samples_[0].wsum,
                                                                               d_sums);
    CT_CUDA(cudaGetLastError());
}

void Engine::finalizeSums(const double* d_params, const double* d_sums, double* d_nll, double* d_grad,
                          cudaStream_t stream)
{
    const Model& m = model_;
    const int nA = m.nAmp(), nc = m.nVector(), nT = m.nTheta();
    ct_prepare_kernel<<<(nA + 127) / 128, 128, 0, stream>>>(d_params, d_amp_chain_, d_ratio_, nA, nc, d_v_, nullptr);
    CT_CUDA(cudaGetLastError());
    FinalizeArgs f;
    std::memset(&f, 0, sizeof(f));
    f.nacc = 2 + 2 * nA + nT;
    f.nA = nA;
    f.nc = nc;
    f.nT = nT;
    f.params = d_params;
    f.v = d_v_;
    f.chain = d_amp_chain_;
    f.gauss_idx = d_gauss_idx_;
    f.gauss_ms = d_gauss_ms_;
    f.ngauss = (int)m.gauss.size();
    f.out_nll = d_nll;
    f.out_grad = d_grad;
    f.out_parts = d_parts_;
    f.sums = d_sums;
    f.vshift = sums_mixed_ ? 1 : 0;
    f.err = d_err_;
    size_t shm = ct_finalize_shm(f);
    ct_finalize_kernel<<<1, 1024, shm, stream>>>(f);
    CT_CUDA(cudaGetLastError());
}

namespace {

__device__ __forceinline__ double ct_hstep(const double* p, int i, double rel)
{
    return rel * fmax(fabs(p[i]), 1e-2);
}

// out = p with p_i shifted by sign * h_i
__global__ void ct_perturb_kernel(const double* __restrict__ p, double* __restrict__ out, int n, int i, double sign,
                                  double rel)
{
    for (int k = threadIdx.x; k < n; k += blockDim.x) out[k] = p[k];
    __syncthreads();
    if (threadIdx.x == 0) out[i] = p[i] + sign * ct_hstep(p, i, rel);
}

// row i of the Hessian from the gradients at p + h_i e_i and p - h_i e_i
__global__ void ct_hess_row_kernel(const double* __restrict__ p, const double* __restrict__ gp,
                                   const double* __restrict__ gm, int n, int i, double rel, double* __restrict__ H)
{
    const double h = ct_hstep(p, i, rel);
    for (int k = threadIdx.x; k < n; k += blockDim.x) H[(size_t)i * n + k] = (gp[k] - gm[k]) / (2.0 * h);
}

__global__ void ct_symmetrize_kernel(double* __restrict__ H, int n)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
        int i = idx / n, k = idx % n;
        if (k <= i) continue;
        double s = 0.5 * (H[(size_t)i * n + k] + H[(size_t)k * n + i]);
        H[(size_t)i * n + k] = s;
        H[(size_t)k * n + i] = s;
    }
}

}  // namespace

void Engine::hessian(const double* d_params, double* d_hess, double rel_step, cudaStream_t stream)
{
    const int n = model_.nParams();
    if (!(rel_step > 0.0)) throw std::runtime_error("hessian: step must be positive");
    double* pp = d_hscratch_;
    double* gp = d_hscratch_ + n;
    double* gm = d_hscratch_ + 2 * n;
    double* nl = d_hscratch_ + 3 * n;
    for (int i = 0; i < n; ++i) {
        ct_perturb_kernel<<<1, 256, 0, stream>>>(d_params, pp, n, i, +1.0, rel_step);
        CT_CUDA(cudaGetLastError());
        nllGrad(pp, nl, gp, kFP64, stream);
        ct_perturb_kernel<<<1, 256, 0, stream>>>(d_params, pp, n, i, -1.0, rel_step);
        CT_CUDA(cudaGetLastError());
        nllGrad(pp, nl, gm, kFP64, stream);
        ct_hess_row_kernel<<<1, 256, 0, stream>>>(d_params, gp, gm, n, i, rel_step, d_hess);
        CT_CUDA(cudaGetLastError());
    }
    ct_symmetrize_kernel<<<std::max(1, (n * n + 255) / 256), 256, 0, stream>>>(d_hess, n);
    CT_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Exact Hessian: forward mode over the adjoint pass (kernels/hessian.cuh)
// ---------------------------------------------------------------------------

// argument block of the Hessian-vector-product kernels (must match CtHvpArgs)
struct CtHvpSampleH {
    const double2* slamp;
    const double* ev;
    const double* w;
    long long n;
    long long ld;
    int kind;
    int cta_begin;
    int cta_count;
    int pad;
};
struct CtHvpArgsH {
    CtHvpSampleH s[3];
    int nsamp;
    int ndir;
    const double* theta;
    const double* v;
    const double* dirs;
    const int* chain;
    const double* ratio;
    int nc;
    int nparam;
    double* consts;
    double* rows;
    int ctas;
    int pad;
};

struct HvpFinalizeArgs {
    const double* vsums;  // [3][nacc] + [n_phsp, W_phsp, W_data, W_bkg]
    const double* tsums;  // [ndir][3][nacc]
    const double* dirs;   // [ndir][nP]
    const double* params;
    const double* v;
    const int* chain;
    const int* gauss_idx;
    const double* gauss_ms;
    int ngauss;
    int nacc, nA, nc, nT, ndir;
    const int* err;
    double* out;  // [ndir][nP]
};

namespace {

// Per-direction, per-sample sums of the tangent rows: one CTA per direction,
// one warp per (sample, column), fixed order.
__global__ void __launch_bounds__(1024) ct_hvp_rowsum_kernel(const double* __restrict__ rows, int ctas, int nacc,
                                                             int c0, int n0, int c1, int n1, int c2, int n2,
                                                             double* __restrict__ out)
{
    const int d = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int beg[3] = {c0, c1, c2}, cnt[3] = {n0, n1, n2};
    for (int i = warp; i < 3 * nacc; i += nwarp) {
        const int k = i / nacc, j = i % nacc;
        double s = 0.0;
        for (int b = lane; b < cnt[k]; b += 32) s += rows[((long long)d * ctas + beg[k] + b) * nacc + j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) out[(long long)d * 3 * nacc + i] = s;
    }
}

// One thread per direction u: the directional derivative of the gradient
// assembly of ct_finalize_kernel (loss terms, phase-space normalisation,
// Gaussian constraints, coupling transform), i.e. the row H u.
__global__ void ct_hvp_finalize_kernel(HvpFinalizeArgs A)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= A.ndir) return;
    const int nacc = A.nacc, nP = 2 * A.nc + A.nT;
    const double* P = A.vsums;
    const double* Dd = A.vsums + nacc;
    const double* B = A.vsums + 2 * nacc;
    const double n_phsp = A.vsums[3 * nacc], Wp = A.vsums[3 * nacc + 1];
    const double W_data = A.vsums[3 * nacc + 2], W_bkg = A.vsums[3 * nacc + 3];
    const double* TP = A.tsums + (long long)d * 3 * nacc;
    const double* TD = TP + nacc;
    const double* TB = TP + 2 * nacc;
    const double* u = A.dirs + (long long)d * nP;
    double* out = A.out + (long long)d * nP;
    const double* theta = A.params + 2 * A.nc;

    const double pf_raw = n_phsp > 0 ? P[1] / n_phsp : 0.0;
    const bool clamped = pf_raw <= 1e-30 || isnan(pf_raw) || isinf(pf_raw);
    const double pf = clamped ? 1e-30 : pf_raw;
    const double pft = clamped ? 0.0 : TP[1] / n_phsp;
    const double Weff = W_data - W_bkg;
    double loss = Dd[0] - B[0] + Weff * log(pf);
    if (A.err && *A.err) loss = nan("");
    for (int g = 0; g < A.ngauss; ++g) {
        const double dl = theta[A.gauss_idx[g]] - A.gauss_ms[2 * g];
        loss += dl * dl / (2.0 * A.gauss_ms[2 * g + 1] * A.gauss_ms[2 * g + 1]);
    }
    if (isnan(loss) || isinf(loss)) {
        for (int k = 0; k < nP; ++k) out[k] = 0.0;
        return;
    }
    const double s = 1.0 / (Wp > 0 ? Wp : 1.0);
    const double pf2 = pf * pf;
    for (int c = 0; c < A.nc; ++c) {
        double sr = 0.0, si = 0.0;
        for (int a = 0; a < A.nA; ++a) {
            if (A.chain[a] != c) continue;
            const double gr = TD[2 + 2 * a] - TB[2 + 2 * a] + Weff * (TP[2 + 2 * a] * s / pf - P[2 + 2 * a] * s * pft / pf2);
            const double gi = TD[3 + 2 * a] - TB[3 + 2 * a] + Weff * (TP[3 + 2 * a] * s / pf - P[3 + 2 * a] * s * pft / pf2);
            const double vr = A.v[2 * a], vi = A.v[2 * a + 1];
            sr += gr * vr + gi * vi;
            si += gr * vi - gi * vr;
        }
        const double pr = A.params[c], pi = A.params[A.nc + c];
        double ps = pr * pr + pi * pi;
        if (ps < 1e-30) ps = 1e-30;
        out[c] = 2.0 * (sr * pr + si * pi) / ps;
        out[A.nc + c] = -2.0 * (si * pr - sr * pi) / ps;
    }
    const int j0 = 2 + 2 * A.nA;
    for (int j = 0; j < A.nT; ++j)
        out[2 * A.nc + j] =
            TD[j0 + j] - TB[j0 + j] + (Weff / n_phsp) * (TP[j0 + j] / pf - P[j0 + j] * pft / pf2);
    for (int g = 0; g < A.ngauss; ++g) {
        const int j = A.gauss_idx[g];
        out[2 * A.nc + j] += u[2 * A.nc + j] / (A.gauss_ms[2 * g + 1] * A.gauss_ms[2 * g + 1]);
    }
}

__global__ void ct_identity_kernel(double* __restrict__ I, int n)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x)
        I[idx] = (idx / n == idx % n) ? 1.0 : 0.0;
}

}  // namespace

void Engine::compileHvp()
{
    if (k_hvp_) return;
    bool hit = false;
    std::string cubin = jitHvpCubin(gen_, paired_[0], &hit);
    cudaLibrary_t lib;
    CT_CUDA(cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
    hvp_lib_ = (void*)lib;
    cudaKernel_t kp, kh;
    CT_CUDA(cudaLibraryGetKernel(&kp, lib, "ct_hvp_prologue"));
    CT_CUDA(cudaLibraryGetKernel(&kh, lib, "ct_hvp_f64"));
    hvp_block_ = hvpBlock(gen_);
    const int nacc = 2 + 2 * model_.nAmp() + model_.nTheta();
    hvp_dsmem_ = nacc * hvp_block_ * (int)sizeof(double);
    if (hvp_dsmem_ > 48 * 1024)
        CT_CUDA(cudaFuncSetAttribute((const void*)kh, cudaFuncAttributeMaxDynamicSharedMemorySize, hvp_dsmem_));
    // CTAs of one direction: one wave of resident CTAs split over the samples
    int sms = 148;
    CT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, opt_.device));
    const int occ = residentCtas((void*)kh, hvp_block_, hvp_dsmem_);
    long long tot = 0;
    for (int k = 0; k < 3; ++k) tot += samples_[k].n;
    layoutCtas(sms * occ, tot, hvp_block_, hlay_);
    const int nP = std::max(1, model_.nParams());
    hvp_cap_ = std::max(nP, 32);
    alloc(d_hdirs_, sizeof(double) * (size_t)nP * nP);
    alloc(d_hconsts_, sizeof(double) * 2 * (size_t)hvp_cap_ * std::max(1, gen_.nconst));
    alloc(d_hrows_, sizeof(double) * (size_t)hvp_cap_ * hlay_.grid * nacc);
    alloc(d_hvsums_, sizeof(double) * (size_t)sumsSize());
    alloc(d_htsums_, sizeof(double) * (size_t)hvp_cap_ * 3 * nacc);
    cudaStream_t st;
    CT_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    ct_identity_kernel<<<std::max(1, std::min(1024, (nP * nP + 255) / 256)), 256, 0, st>>>(d_hdirs_, nP);
    CT_CUDA(cudaGetLastError());
    CT_CUDA(cudaStreamSynchronize(st));
    cudaStreamDestroy(st);
    k_hvp_pro_ = (void*)kp;
    k_hvp_ = (void*)kh;
}

void Engine::hvpSums(const double* d_params, const double* d_dirs, int ndir, double* d_tsums, cudaStream_t stream)
{
    if (ndir <= 0) return;
    compileHvp();
    const Model& m = model_;
    const int nA = m.nAmp(), nc = m.nVector(), nT = m.nTheta(), nP = m.nParams();
    const int nacc = 2 + 2 * nA + nT;
    ct_prepare_kernel<<<(nA + 127) / 128, 128, 0, stream>>>(d_params, d_amp_chain_, d_ratio_, nA, nc, d_v_, nullptr);
    CT_CUDA(cudaGetLastError());
    CtHvpArgsH a;
    std::memset(&a, 0, sizeof(a));
    int ns = 0;
    for (int k = 0; k < 3; ++k) {
        if (hlay_.cta[k][1] == 0) continue;
        CtHvpSampleH& sm = a.s[ns++];
        const DeviceSample& d = samples_[k];
        sm.slamp = paired_[0] ? d.slamp64p : d.slamp64;
        sm.ev = d.ev64;
        sm.w = d.w;
        sm.n = d.n;
        sm.ld = d.ld;
        sm.kind = k;
        sm.cta_begin = hlay_.cta[k][0];
        sm.cta_count = hlay_.cta[k][1];
    }
    a.nsamp = ns;
    a.theta = d_params + 2 * nc;
    a.v = d_v_;
    a.chain = d_amp_chain_;
    a.ratio = d_ratio_;
    a.nc = nc;
    a.nparam = nP;
    a.consts = d_hconsts_;
    a.rows = d_hrows_;
    a.ctas = hlay_.grid;
    for (int d0 = 0; d0 < ndir; d0 += hvp_cap_) {
        const int nd = std::min(hvp_cap_, ndir - d0);
        a.ndir = nd;
        a.dirs = d_dirs + (size_t)d0 * nP;
        void* args[] = {&a};
        CT_CUDA(cudaLaunchKernel(k_hvp_pro_, dim3(nd), dim3(32), args, 0, stream));
        CT_CUDA(cudaLaunchKernel(k_hvp_, dim3(hlay_.grid, nd), dim3(hvp_block_), args, (size_t)hvp_dsmem_, stream));
        ct_hvp_rowsum_kernel<<<nd, 1024, 0, stream>>>(d_hrows_, hlay_.grid, nacc, hlay_.cta[0][0], hlay_.cta[0][1],
                                                      hlay_.cta[1][0], hlay_.cta[1][1], hlay_.cta[2][0], hlay_.cta[2][1],
                                                      d_tsums + (size_t)d0 * 3 * nacc);
        CT_CUDA(cudaGetLastError());
    }
}

void Engine::finalizeHvp(const double* d_params, const double* d_dirs, int ndir, const double* d_vsums,
                         const double* d_tsums, double* d_out, cudaStream_t stream)
{
    if (ndir <= 0) return;
    const Model& m = model_;
    const int nA = m.nAmp(), nc = m.nVector(), nT = m.nTheta();
    ct_prepare_kernel<<<(nA + 127) / 128, 128, 0, stream>>>(d_params, d_amp_chain_, d_ratio_, nA, nc, d_v_, nullptr);
    CT_CUDA(cudaGetLastError());
    HvpFinalizeArgs f;
    std::memset(&f, 0, sizeof(f));
    f.vsums = d_vsums;
    f.tsums = d_tsums;
    f.dirs = d_dirs;
    f.params = d_params;
    f.v = d_v_;
    f.chain = d_amp_chain_;
    f.gauss_idx = d_gauss_idx_;
    f.gauss_ms = d_gauss_ms_;
    f.ngauss = (int)m.gauss.size();
    f.nacc = 2 + 2 * nA + nT;
    f.nA = nA;
    f.nc = nc;
    f.nT = nT;
    f.ndir = ndir;
    f.err = d_err_;
    f.out = d_out;
    ct_hvp_finalize_kernel<<<(ndir + 63) / 64, 64, 0, stream>>>(f);
    CT_CUDA(cudaGetLastError());
}

// argument block of ct_gram (must match CtGramArgs in kernels/gram.cuh)
struct CtGramArgsH {
    const void* slamp;
    const float* evf;
    const double* evd;
    const double* w;
    long long n, ld;
    const void* K;
    double* partials;
    int* err;
    int pad;
};

// Resident CTAs per SM of a Gram kernel from the limits the hardware
// applies: shared memory (dynamic + static + the per-CTA reservation, with
// the whole unified L1 as shared memory), registers, threads. The occupancy
// query on the library kernel handle answered 1 where these give 2 (ncu:
// occupancy limits 2 by shared memory and 2 by registers at 79.9 KB and 127
// registers).
int gramResidentCtas(void* kernel, int block, int dsmem, int device)
{
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, (const void*)kernel) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    int smem_sm = 0, reserved = 0, regs_sm = 65536, thr_sm = 2048;
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, device);
    cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, device);
    cudaGetLastError();
    const long long per_cta_smem = (long long)dsmem + (long long)fa.sharedSizeBytes + reserved;
    const int by_smem = per_cta_smem > 0 ? (int)(smem_sm / per_cta_smem) : 32;
    const int regs = (fa.numRegs + 7) / 8 * 8;  // per-thread allocation granularity
    const int by_regs = regs > 0 ? regs_sm / (regs * block) : 32;
    const int by_thr = thr_sm / block;
    return std::max(1, std::min({by_smem, by_regs, by_thr}));
}

void Engine::compileGram()
{
    if (k_gram_) return;
    const int rows = model_.npol * 2 * model_.nAmp();
    if (rows > 128)
        throw std::length_error("the tensor-core Gram supports npol * 2 * nA <= 128; this model has " +
                                std::to_string(rows));
    if (!samples_[0].slamp32) throw std::runtime_error("the Gram needs the mixed-precision tables");
    bool hit = false;
    std::string cubin = jitGramCubin(gen_, paired_[1], &hit);
    cudaLibrary_t lib;
    CT_CUDA(cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
    gram_lib_ = (void*)lib;
    cudaKernel_t kg, kf;
    CT_CUDA(cudaLibraryGetKernel(&kg, lib, "ct_gram"));
    CT_CUDA(cudaLibraryGetKernel(&kf, lib, "ct_gram_finalize"));
    // operand tile(s) of 128 rows x 256 events (BF16; one when the hi and lo
    // rows fit together) and the FP64 sums [2 nA][128] (kernels/gram.cuh)
    const int r8 = (rows + 7) / 8 * 8;
    gram_dsmem_ = (2 * r8 <= 128 ? 1 : 2) * 128 * 256 * 2 + 128 * 2 * model_.nAmp() * 8;
    CT_CUDA(cudaFuncSetAttribute((const void*)kg, cudaFuncAttributeMaxDynamicSharedMemorySize, gram_dsmem_));
    // the whole unified L1 as shared memory: two CTAs of ~80 KB per SM (the
    // occupancy query answered one with the default carveout)
    CT_CUDA(cudaFuncSetAttribute((const void*)kg, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    int sms = 148;
    CT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, opt_.device));
    // tensor-memory columns per CTA (CT_GRAM_TMEM_COLS): NACC accumulators of N columns
    const int nn = 2 * r8 <= 128 ? 2 * r8 : (rows + 15) / 16 * 16;
    int tcols = 32;
    while (tcols < (nn <= 64 ? 4 : 2) * nn) tcols *= 2;
    gram_resident_ = gramResidentCtas((void*)kg, 256, gram_dsmem_, opt_.device);
    const int occ = std::max(1, std::min({4, 512 / tcols, gram_resident_}));
    const long long ntiles = (samples_[0].n + 255) / 256;
    gram_grid_ = (int)std::max(1LL, std::min<long long>(ntiles, (long long)sms * occ));
    alloc(d_gpart_, sizeof(double) * (size_t)gram_grid_ * rows * 2 * model_.nAmp());
    k_gram_ = (void*)kg;
    k_gram_fin_ = (void*)kf;
}

void Engine::compileGramHess()
{
    if (k_gramh_) return;
    const int nA = model_.nAmp(), rows = (model_.npol + 1) * 2 * nA;
    if (rows > 128)
        throw std::length_error("the Gram-based Hessian supports (npol + 1) * 2 * nA <= 128; this model has " +
                                std::to_string(rows));
    if (!samples_[0].slamp32) throw std::runtime_error("the Gram needs the mixed-precision tables");
    bool hit = false;
    std::string cubin = jitGramCubin(gen_, paired_[1], &hit, true);
    cudaLibrary_t lib;
    CT_CUDA(cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
    gram_hess_lib_ = (void*)lib;
    cudaKernel_t kg, kf;
    CT_CUDA(cudaLibraryGetKernel(&kg, lib, "ct_gram"));
    CT_CUDA(cudaLibraryGetKernel(&kf, lib, "ct_gram_hess_finalize"));
    const int r8 = (rows + 7) / 8 * 8;
    gramh_dsmem_ = (2 * r8 <= 128 ? 1 : 2) * 128 * 256 * 2 + 128 * 2 * nA * 8;
    CT_CUDA(cudaFuncSetAttribute((const void*)kg, cudaFuncAttributeMaxDynamicSharedMemorySize, gramh_dsmem_));
    CT_CUDA(cudaFuncSetAttribute((const void*)kg, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    int sms = 148;
    CT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, opt_.device));
    const int nn = 2 * r8 <= 128 ? 2 * r8 : (rows + 15) / 16 * 16;
    int tcols = 32;
    while (tcols < (nn <= 64 ? 4 : 2) * nn) tcols *= 2;
    gramh_grid_ = sms * std::max(1, std::min({4, 512 / tcols, gramResidentCtas((void*)kg, 256, gramh_dsmem_, opt_.device)}));
    alloc(d_ghpart_, sizeof(double) * (size_t)gramh_grid_ * rows * 2 * nA);
    alloc(d_ghout_, sizeof(double) * 2 * (2 * nA) * (2 * nA));
    k_gramh_ = (void*)kg;
    k_gramh_fin_ = (void*)kf;
}

// Hessian with the coupling block from tensor-core Gram sums (FP32
// amplitudes, split-BF16 products, FP64 assembly): in the real couplings
// z = [Re v; Im v], with per event f = z^T Q_e z, u_e = Q_e z,
//   d2 (sum w log f) = 2 T1 - 4 T2,  T1 = sum (w / f) Q_e,  T2 = sum (w / f^2) u u^T,
// over data (subtracted) and background (added), and for the normalisation
// W_eff log pf with pf = z^T Qbar z (Qbar from the phase-space Gram),
//   W_eff (2 Qbar / pf - 4 (Qbar z)(Qbar z)^T / pf^2);
// mapped to the parameters by the linear coupling map v_a = r_a p_c(a).
// The rows of the resonance parameters come from the exact FP64
// Hessian-vector products along their unit directions. Host-synchronising.
void Engine::hessianGram(const double* d_params, double* d_hess, cudaStream_t stream)
{
    compileGram();
    compileGramHess();
    compileHvp();
    const Model& m = model_;
    const int nA = m.nAmp(), nc = m.nVector(), nT = m.nTheta(), nP = m.nParams(), NA2 = 2 * nA;
    std::vector<double> hp(nP);
    CT_CUDA(cudaMemcpyAsync(hp.data(), d_params, sizeof(double) * nP, cudaMemcpyDeviceToHost, stream));
    // the FP64 evaluation: phase-space factor and sample totals
    nllGrad(d_params, d_hscratch_ + 3 * (size_t)nP, d_hscratch_, kFP64, stream);
    double parts[6];
    lastParts(parts, stream);
    const double n_phsp = parts[5], pf_raw = n_phsp > 0 ? parts[2] / n_phsp : 0.0;
    const double pf = (pf_raw <= 1e-30 || !std::isfinite(pf_raw)) ? 1e-30 : pf_raw;
    const double weff = parts[3] - parts[4];
    // phase-space Gram M = (1/W) sum w A conj(A)^T (complex [nA][nA])
    double* d_M = d_ghout_;  // reused below for the weighted sums
    std::vector<double> M(2 * nA * nA);
    gram(d_params, d_M, stream);
    CT_CUDA(cudaMemcpyAsync(M.data(), d_M, sizeof(double) * 2 * nA * nA, cudaMemcpyDeviceToHost, stream));
    CT_CUDA(cudaStreamSynchronize(stream));
    // weighted sums over data (kind 1) and background (kind 2); the constant
    // block of this call is in place (gram() ran the prologue)
    std::vector<double> S[3];
    for (int kind = 1; kind <= 2; ++kind) {
        const DeviceSample& d = samples_[kind];
        S[kind].assign(2 * NA2 * NA2, 0.0);
        if (d.n <= 0) continue;
        CtGramArgsH g;
        std::memset(&g, 0, sizeof(g));
        g.slamp = d.slamp32;
        g.evf = d.evf;
        g.evd = d.evd;
        g.w = d.w;
        g.n = d.n;
        g.ld = d.ld;
        g.K = d_kblock_;
        g.partials = d_ghpart_;
        g.err = d_err_;
        const int grid = (int)std::max(1LL, std::min<long long>((d.n + 255) / 256, gramh_grid_));
        void* gargs[] = {&g};
        CT_CUDA(cudaLaunchKernel(k_gramh_, dim3(grid), dim3(256), gargs, (size_t)gramh_dsmem_, stream));
        int nb = grid;
        void* fargs[] = {&d_ghpart_, &nb, &d_ghout_};
        CT_CUDA(cudaLaunchKernel(k_gramh_fin_, dim3(1), dim3(256), fargs, 0, stream));
        CT_CUDA(cudaMemcpyAsync(S[kind].data(), d_ghout_, sizeof(double) * 2 * NA2 * NA2, cudaMemcpyDeviceToHost,
                                stream));
        CT_CUDA(cudaStreamSynchronize(stream));
    }
    int herr = 0;
    CT_CUDA(cudaMemcpy(&herr, d_err_, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) throw std::runtime_error("the tensor-core Gram pipeline did not complete");
    // couplings and z
    std::vector<double> z(NA2);
    for (int a = 0; a < nA; ++a) {
        const int c = m.coupling.amp_chain[a];
        const double r = m.coupling.ratio[a];
        z[a] = r * hp[c];
        z[nA + a] = r * hp[nc + c];
    }
    // the real symmetric form Q of a complex Hermitian K: [[Re K, Im K], [-Im K, Re K]]
    auto Qof = [&](const std::vector<double>& reK, const std::vector<double>& imK) {
        std::vector<double> Q(NA2 * NA2);
        for (int a = 0; a < nA; ++a)
            for (int b = 0; b < nA; ++b) {
                Q[a * NA2 + b] = reK[a * nA + b];
                Q[(nA + a) * NA2 + nA + b] = reK[a * nA + b];
                Q[a * NA2 + nA + b] = imK[a * nA + b];
                Q[(nA + a) * NA2 + b] = -imK[a * nA + b];
            }
        return Q;
    };
    std::vector<double> Hz(NA2 * NA2, 0.0);
    for (int kind = 1; kind <= 2; ++kind) {
        if (samples_[kind].n <= 0) continue;
        const double* B = S[kind].data();           // sum of the amplitude blocks [Re; Im][Re; Im]^T
        const double* C = S[kind].data() + NA2 * NA2;  // the c block
        std::vector<double> reK(nA * nA), imK(nA * nA);
        for (int a = 0; a < nA; ++a)
            for (int b = 0; b < nA; ++b) {
                reK[a * nA + b] = B[a * NA2 + b] + B[(nA + a) * NA2 + nA + b];
                imK[a * nA + b] = B[(nA + a) * NA2 + b] - B[a * NA2 + nA + b];
            }
        const std::vector<double> T1 = Qof(reK, imK);
        const double sgn = kind == 1 ? -1.0 : 1.0;  // NLL = -sum_data + sum_bkg
        for (int i = 0; i < NA2; ++i)
            for (int j = 0; j < NA2; ++j) {
                // u u^T with u = [Re c; -Im c] from the [Re c; Im c] sums
                const double flip = ((i < nA) != (j < nA)) ? -1.0 : 1.0;
                const double T2 = flip * C[i * NA2 + j];
                Hz[i * NA2 + j] += sgn * (2.0 * T1[i * NA2 + j] - 4.0 * T2);
            }
    }
    {
        const double wsum = samples_[0].wsum > 0 ? samples_[0].wsum : 1.0, scale = wsum / (n_phsp > 0 ? n_phsp : 1.0);
        std::vector<double> reM(nA * nA), imM(nA * nA);
        for (int i = 0; i < nA * nA; ++i) {
            reM[i] = scale * M[2 * i];
            imM[i] = scale * M[2 * i + 1];
        }
        const std::vector<double> Qb = Qof(reM, imM);
        std::vector<double> qz(NA2, 0.0);
        for (int i = 0; i < NA2; ++i)
            for (int j = 0; j < NA2; ++j) qz[i] += Qb[i * NA2 + j] * z[j];
        for (int i = 0; i < NA2; ++i)
            for (int j = 0; j < NA2; ++j)
                Hz[i * NA2 + j] += weff * (2.0 * Qb[i * NA2 + j] / pf - 4.0 * qz[i] * qz[j] / (pf * pf));
    }
    // symmetrised (the tensor-core sums of (i, j) and (j, i) round apart)
    for (int i = 0; i < NA2; ++i)
        for (int j = 0; j < i; ++j) {
            const double v = 0.5 * (Hz[i * NA2 + j] + Hz[j * NA2 + i]);
            Hz[i * NA2 + j] = Hz[j * NA2 + i] = v;
        }
    // the coupling block in the parameters, then the resonance rows
    std::vector<double> H((size_t)nP * nP, 0.0);
    auto zi = [&](int a, int part) { return part * nA + a; };
    for (int a = 0; a < nA; ++a)
        for (int b = 0; b < nA; ++b)
            for (int pa = 0; pa < 2; ++pa)
                for (int pb = 0; pb < 2; ++pb) {
                    const int i = pa * nc + m.coupling.amp_chain[a], j = pb * nc + m.coupling.amp_chain[b];
                    H[(size_t)i * nP + j] +=
                        m.coupling.ratio[a] * m.coupling.ratio[b] * Hz[zi(a, pa) * NA2 + zi(b, pb)];
                }
    if (nT > 0) {
        std::vector<double> dirs((size_t)nT * nP, 0.0);
        for (int j = 0; j < nT; ++j) dirs[(size_t)j * nP + 2 * nc + j] = 1.0;
        double* d_dirs = nullptr;
        double* d_rows = nullptr;
        CT_CUDA(cudaMallocAsync((void**)&d_dirs, sizeof(double) * dirs.size(), stream));
        CT_CUDA(cudaMallocAsync((void**)&d_rows, sizeof(double) * dirs.size(), stream));
        CT_CUDA(cudaMemcpyAsync(d_dirs, dirs.data(), sizeof(double) * dirs.size(), cudaMemcpyHostToDevice, stream));
        hessianVectorProducts(d_params, d_dirs, nT, d_rows, stream);
        std::vector<double> rows(dirs.size());
        CT_CUDA(cudaMemcpyAsync(rows.data(), d_rows, sizeof(double) * rows.size(), cudaMemcpyDeviceToHost, stream));
        CT_CUDA(cudaFreeAsync(d_dirs, stream));
        CT_CUDA(cudaFreeAsync(d_rows, stream));
        CT_CUDA(cudaStreamSynchronize(stream));
        for (int j = 0; j < nT; ++j)
            for (int i = 0; i < nP; ++i) {
                const double v = rows[(size_t)j * nP + i];
                H[(size_t)(2 * nc + j) * nP + i] = v;
                H[(size_t)i * nP + 2 * nc + j] = v;
            }
    }
    CT_CUDA(cudaMemcpyAsync(d_hess, H.data(), sizeof(double) * H.size(), cudaMemcpyHostToDevice, stream));
    CT_CUDA(cudaStreamSynchronize(stream));
}

// ---------------------------------------------------------------------------
// Normalisation cache (kernels/norm.cuh): the phase-space sums as FP64
// quadratic forms in the couplings at fixed resonance parameters.
// ---------------------------------------------------------------------------
// argument blocks of ct_norm_build and ct_norm_row (must match kernels/norm.cuh)
struct CtNormArgsH {
    const void* slamp;
    const double* ev;
    const double* w;
    long long n, ld;
    const double* consts;
    double* partials;
    int nrows;
    int pad;
};
struct CtNormRowArgsH {
    const double* mat;
    int weighted;
    int use_vh;
    const double* v;
    double vw_scale;
    const double* theta;
    const double* theta_cached;
    int* err;
    int pad;
    double* row;
};

void Engine::compileNorm()
{
    if (k_norm_build_) return;
    const int nt = gen_.nterm, nd = gen_.nder, ng = gen_.nplane * (gen_.nplane + 1) / 2;
    // output rows (terms, derivative entries, weighted terms) x nt columns;
    // phase 2 of ct_norm_build: groups of rb rows, 128 / groups event slices
    norm_rows_ = nt + nd + (samples_[0].w ? nt : 0);
    norm_ne_ = norm_rows_ * nt;
    const int rb = 2, groups = (norm_rows_ + rb - 1) / rb;  // CT_NORM_RB
    if (groups > 128 || nt + nd > 256 || (size_t)(2 * nt + nd) * nt * 16 > 40000)
        throw std::length_error("the normalisation cache supports models with up to 256 lineshape terms and "
                                "derivative entries and (2 terms + entries) x terms <= 2500");
    bool hit = false;
    std::string cubin = jitNormCubin(gen_, &hit);
    cudaLibrary_t lib;
    CT_CUDA(cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
    norm_lib_ = (void*)lib;
    cudaKernel_t kb, kr, kw;
    CT_CUDA(cudaLibraryGetKernel(&kb, lib, "ct_norm_build"));
    CT_CUDA(cudaLibraryGetKernel(&kr, lib, "ct_norm_reduce"));
    CT_CUDA(cudaLibraryGetKernel(&kw, lib, "ct_norm_row"));
    // one record of (terms + derivatives + plane pairs + weight) double2
    // slots per event of a 128-event tile, the record length made odd
    const int rec = (nt + nd + ng + 1) | 1;
    const int slices = 128 / groups;
    norm_dsmem_ = std::max(128 * rec * 16, slices * norm_ne_ * 16);  // records, then the slices' sums
    CT_CUDA(cudaFuncSetAttribute((const void*)kb, cudaFuncAttributeMaxDynamicSharedMemorySize, norm_dsmem_));
    CT_CUDA(cudaFuncSetAttribute((const void*)kb, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    int sms = 148;
    CT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, opt_.device));
    const int occ = gramResidentCtas((void*)kb, 128, norm_dsmem_, opt_.device);
    const long long ntiles = (samples_[0].n + 127) / 128;
    norm_grid_ = (int)std::max(1LL, std::min<long long>(ntiles, (long long)sms * occ));
    alloc(d_npart_, sizeof(double) * 2 * (size_t)norm_grid_ * norm_ne_);
    alloc(d_nmat_, sizeof(double) * 2 * (size_t)norm_ne_);
    alloc(d_ntheta_, sizeof(double) * std::max(1, model_.nTheta()));
    alloc(d_nrow_, sizeof(double) * (2 + 2 * model_.nAmp() + model_.nTheta()));
    k_norm_build_ = (void*)kb;
    k_norm_red_ = (void*)kr;
    k_norm_row_ = (void*)kw;
}

double Engine::normCacheBuild(const double* d_params, cudaStream_t stream)
{
    compileNorm();
    const Model& m = model_;
    const int nA = m.nAmp(), nc = m.nVector(), nT = m.nTheta();
    norm_valid_ = false;
    // the parameter-only subexpressions at this theta
    ct_prepare_kernel<<<(nA + 127) / 128, 128, 0, stream>>>(d_params, d_amp_chain_, d_ratio_, nA, nc, d_v_, nullptr);
    CT_CUDA(cudaGetLastError());
    CtArgsH pa;
    std::memset(&pa, 0, sizeof(pa));
    pa.theta = d_params + 2 * nc;
    pa.v = d_v_;
    pa.consts = d_consts_;
    void* pargs[] = {&pa};
    CT_CUDA(cudaLaunchKernel(k_pro_, dim3(1), dim3(32), pargs, 0, stream));
    const DeviceSample& d = samples_[0];
    CtNormArgsH a;
    std::memset(&a, 0, sizeof(a));
    a.slamp = d.slamp64;
    a.ev = d.ev64;
    a.w = d.w;
    a.n = d.n;
    a.ld = d.ld;
    a.consts = d_consts_;
    a.partials = d_npart_;
    a.nrows = norm_rows_;
    cudaEvent_t e0, e1;
    CT_CUDA(cudaEventCreate(&e0));
    CT_CUDA(cudaEventCreate(&e1));
    CT_CUDA(cudaEventRecord(e0, stream));
    void* args[] = {&a};
    CT_CUDA(cudaLaunchKernel(k_norm_build_, dim3(norm_grid_), dim3(128), args, (size_t)norm_dsmem_, stream));
    CT_CUDA(cudaEventRecord(e1, stream));
    int rows = norm_grid_, ne = norm_ne_;
    double* part = d_npart_;
    double* mat = d_nmat_;
    void* rargs[] = {&part, &rows, &ne, &mat};
    CT_CUDA(cudaLaunchKernel(k_norm_red_, dim3(1), dim3(256), rargs, 0, stream));
    if (nT > 0)
        CT_CUDA(cudaMemcpyAsync(d_ntheta_, d_params + 2 * nc, sizeof(double) * nT, cudaMemcpyDeviceToDevice, stream));
    norm_theta_.assign(nT, 0.0);
    if (nT > 0)
        CT_CUDA(cudaMemcpyAsync(norm_theta_.data(), d_params + 2 * nc, sizeof(double) * nT, cudaMemcpyDeviceToHost,
                                stream));
    CT_CUDA(cudaStreamSynchronize(stream));
    float ms = 0.0f;
    CT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    norm_valid_ = true;
    return (double)ms;
}

bool Engine::normCacheMatches(const double* params) const
{
    if (!norm_valid_) return false;
    const int nT = model_.nTheta(), off = 2 * model_.nVector();
    return nT == 0 || std::memcmp(params + off, norm_theta_.data(), sizeof(double) * nT) == 0;
}

// The evaluation at the cached resonance parameters: the fused pass over the
// data and background samples (their own one-wave layout), the phase-space
// row from the matrices, the usual finalize.
void Engine::nllGradCached(const double* d_params, double* d_nll, double* d_grad, int precision, cudaStream_t stream)
{
    if (!norm_valid_) throw std::runtime_error("no normalisation cache: build it first");
    const CtaLayout& lay = lay_data_[precision == kMixed ? 1 : 0];
    const Model& m = model_;
    const int nA = m.nAmp(), nc = m.nVector(), nT = m.nTheta();
    ct_prepare_kernel<<<(nA + 127) / 128, 128, 0, stream>>>(d_params, d_amp_chain_, d_ratio_, nA, nc, d_v_, d_err_);
    CT_CUDA(cudaGetLastError());
    CtArgsH a;
    std::memset(&a, 0, sizeof(a));
    int ns = 0;
    for (int k = 1; k < 3; ++k) {
        if (lay.cta[k][1] == 0) continue;
        CtSampleH& sm = a.s[ns++];
        const DeviceSample& d = samples_[k];
        sm.slamp = precision == kMixed ? (const void*)d.slamp32 : (paired_[0] ? (const void*)d.slamp64p : (const void*)d.slamp64);
        sm.ev = precision == kMixed ? (const void*)d.evf : (const void*)d.ev64;
        sm.evd = precision == kMixed ? d.evd : nullptr;
        sm.w = d.w;
        sm.n = d.n;
        sm.ld = d.ld;
        sm.kind = k;
        sm.cta_begin = lay.cta[k][0];
        sm.cta_count = lay.cta[k][1];
        sm.vw_scale = 1.0;
    }
    a.nsamp = ns;
    a.theta = d_params + 2 * nc;
    a.v = d_v_;
    a.partials = d_partials_;
    a.consts = d_consts_;
    a.err = d_err_;
    a.kblock = d_kblock_;
    if (precision == kMixed && !samples_[1].slamp32) throw std::runtime_error("mixed-precision tables were not built");
    void* args[] = {&a};
    CT_CUDA(cudaLaunchKernel(k_pro_, dim3(1), dim3(32), args, 0, stream));
    CT_CUDA(cudaMemcpyAsync(k_sym_, d_kblock_, k_sym_bytes_, cudaMemcpyDeviceToDevice, stream));
    a.cta_base = 0;
    if (ns > 0)
        CT_CUDA(cudaLaunchKernel(precision == kMixed ? k_mixed_ : k_f64_, dim3(lay.grid),
                                 dim3(shape_.block[precision == kMixed]), args, (size_t)shape_.dsmem[precision == kMixed],
                                 stream));
    CtNormRowArgsH r;
    std::memset(&r, 0, sizeof(r));
    r.mat = d_nmat_;
    r.weighted = samples_[0].w ? 1 : 0;
    r.use_vh = precision == kMixed ? 1 : 0;
    r.v = d_v_;
    r.vw_scale = 1.0 / (samples_[0].wsum > 0 ? samples_[0].wsum : 1.0);
    r.theta = d_params + 2 * nc;
    r.theta_cached = d_ntheta_;
    r.err = d_err_;
    r.row = d_nrow_;
    void* rargs[] = {&r};
    CT_CUDA(cudaLaunchKernel(k_norm_row_, dim3(1), dim3(256), rargs, 0, stream));  // CT_NORM_ROW_THREADS
    FinalizeArgs f;
    std::memset(&f, 0, sizeof(f));
    f.partials = d_partials_;
    f.nacc = 2 + 2 * nA + nT;
    f.nA = nA;
    f.nc = nc;
    f.nT = nT;
    for (int k = 0; k < 3; ++k) {
        f.cta[k][0] = lay.cta[k][0];
        f.cta[k][1] = lay.cta[k][1];
        f.has[k] = lay.cta[k][1] > 0;
    }
    f.n_phsp = (double)samples_[0].n;
    f.W_data = samples_[1].wsum;
    f.W_bkg = has_bkg_ ? samples_[2].wsum : 0.0;
    f.params = d_params;
    f.v = d_v_;
    f.chain = d_amp_chain_;
    f.gauss_idx = d_gauss_idx_;
    f.gauss_ms = d_gauss_ms_;
    f.ngauss = (int)m.gauss.size();
    f.out_nll = d_nll;
    f.out_grad = d_grad;
    f.out_parts = d_parts_;
    f.err = d_err_;
    f.vshift = precision == kMixed ? 1 : 0;
    f.phsp_row = d_nrow_;
    size_t shm = ct_finalize_shm(f);
    ct_finalize_kernel<<<1, 1024, shm, stream>>>(f);
    CT_CUDA(cudaGetLastError());
}

void Engine::gramShape(int* out4)
{
    compileGram();
    out4[0] = gram_grid_;
    out4[1] = gram_dsmem_;
    out4[2] = gram_resident_;
    out4[3] = 256;
}

void Engine::gram(const double* d_params, double* d_out, cudaStream_t stream)
{
    compileGram();
    const Model& m = model_;
    const int nA = m.nAmp(), nc = m.nVector();
    // this call's couplings and parameter-only constants (the constant-bank image)
    ct_prepare_kernel<<<(nA + 127) / 128, 128, 0, stream>>>(d_params, d_amp_chain_, d_ratio_, nA, nc, d_v_, d_err_);
    CT_CUDA(cudaGetLastError());
    CtArgsH a;
    std::memset(&a, 0, sizeof(a));
    a.theta = d_params + 2 * nc;
    a.v = d_v_;
    a.consts = d_consts_;
    a.err = d_err_;
    a.kblock = d_kblock_;
    void* args[] = {&a};
    CT_CUDA(cudaLaunchKernel(k_pro_, dim3(1), dim3(32), args, 0, stream));
    const DeviceSample& d = samples_[0];
    CtGramArgsH g;
    std::memset(&g, 0, sizeof(g));
    g.slamp = d.slamp32;
    g.evf = d.evf;
    g.evd = d.evd;
    g.w = d.w;
    g.n = d.n;
    g.ld = d.ld;
    g.K = d_kblock_;
    g.partials = d_gpart_;
    g.err = d_err_;
    void* gargs[] = {&g};
    CT_CUDA(cudaLaunchKernel(k_gram_, dim3(gram_grid_), dim3(256), gargs, (size_t)gram_dsmem_, stream));
    int nb = gram_grid_;
    double inv_w = 1.0 / (d.wsum > 0 ? d.wsum : 1.0);
    void* fargs[] = {&d_gpart_, &nb, &inv_w, &d_out};
    CT_CUDA(cudaLaunchKernel(k_gram_fin_, dim3(1), dim3(256), fargs, 0, stream));
}

void Engine::hessianVectorProducts(const double* d_params, const double* d_dirs, int ndir, double* d_out,
                                   cudaStream_t stream)
{
    if (ndir <= 0) return;
    compileHvp();
    shardSums(d_params, kFP64, d_hvsums_, stream);
    for (int d0 = 0; d0 < ndir; d0 += hvp_cap_) {
        const int nd = std::min(hvp_cap_, ndir - d0);
        const size_t off = (size_t)d0 * model_.nParams();
        hvpSums(d_params, d_dirs + off, nd, d_htsums_, stream);
        finalizeHvp(d_params, d_dirs + off, nd, d_hvsums_, d_htsums_, d_out + off, stream);
    }
}

void Engine::hessianExact(const double* d_params, double* d_hess, cudaStream_t stream)
{
    compileHvp();
    const int n = model_.nParams();
    hessianVectorProducts(d_params, d_hdirs_, n, d_hess, stream);
    ct_symmetrize_kernel<<<std::max(1, (n * n + 255) / 256), 256, 0, stream>>>(d_hess, n);
    CT_CUDA(cudaGetLastError());
}

namespace {

// out[j] = sum over rows r of rows[r][j] (fixed order: one warp per column)
__global__ void ct_colsum_kernel(const double* __restrict__ rows, int nrows, int ncols, double* __restrict__ out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int j = warp; j < ncols; j += nwarp) {
        double s = 0.0;
        for (int r = lane; r < nrows; r += 32) s += rows[(long long)r * ncols + j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) out[j] = s;
    }
}

}  // namespace

void Engine::loadTruth()
{
    if (truth_loaded_) return;
    auto it = model_.cfg.data_files.find("phsp_truth");
    if (it == model_.cfg.data_files.end()) throw std::runtime_error("No phsp_truth in config");
    const int nfin = (int)model_.final_order.size();
    Sample s = readSample(it->second, nfin);
    std::vector<double> w;
    shardSample(s, w, opt_.shard_rank, opt_.shard_world);
    DeviceSample& d = samples_[3];
    d.n = s.n;
    d.wsum = (double)s.n;
    CT_CUDA(cudaSetDevice(opt_.device));
    CT_CUDA(cudaStreamCreateWithFlags(&init_stream_, cudaStreamNonBlocking));
    if (s.n > 0) {
        size_t bytes = sizeof(double) * (size_t)s.n * nfin * 4;
        double* tmp = nullptr;
        CT_CUDA(cudaMallocFromPoolAsync((void**)&tmp, bytes, enginePool(opt_.device), init_stream_));
        CT_CUDA(cudaMemcpyAsync(tmp, s.p4.data(), bytes, cudaMemcpyHostToDevice, init_stream_));
        CT_CUDA(cudaMallocFromPoolAsync((void**)&d.p4, bytes, enginePool(opt_.device), init_stream_));
        ag_transpose_kernel<<<(unsigned)((s.n + 255) / 256), 256, 0, init_stream_>>>(tmp, d.p4, s.n, nfin);
        CT_CUDA(cudaGetLastError());
        CT_CUDA(cudaFreeAsync(tmp, init_stream_));
        CT_CUDA(cudaStreamSynchronize(init_stream_));
        device_bytes_ += bytes;
    }
    computeAngular(3);
    cudaStreamDestroy(init_stream_);
    init_stream_ = nullptr;
    truth_loaded_ = true;
}

void Engine::partialIntegrals(const double* d_params, int kind, double* d_out, cudaStream_t stream)
{
    if (kind < 0 || kind > 3) throw std::runtime_error("partial integrals: sample kind must be 0..3");
    if (kind == 3) loadTruth();
    const Model& m = model_;
    const int nA = m.nAmp(), nc = m.nVector(), nb = nBlocks();
    const DeviceSample& d = samples_[kind];
    ct_prepare_kernel<<<(nA + 127) / 128, 128, 0, stream>>>(d_params, d_amp_chain_, d_ratio_, nA, nc, d_v_, nullptr);
    CT_CUDA(cudaGetLastError());
    CtArgsH a;
    std::memset(&a, 0, sizeof(a));
    a.s[0].slamp = d.slamp64;
    a.s[0].ev = d.ev64;
    a.s[0].w = d.w;
    a.s[0].n = d.n;
    a.s[0].ld = d.ld;
    a.s[0].kind = kind;
    a.s[0].cta_count = 1;
    a.nsamp = 1;
    a.theta = d_params + 2 * nc;
    a.v = d_v_;
    a.partials = d_partials_;
    a.consts = d_consts_;
    a.err = d_err_;
    void* pargs[] = {&a};
    CT_CUDA(cudaLaunchKernel(k_pro_, dim3(1), dim3(32), pargs, 0, stream));
    // rows of nb sums in the partials table (nacc >= nA >= nb columns per row available)
    const int nacc = 2 + 2 * nA + m.nTheta();
    const long long cap_rows = (long long)grid_max_ * nacc / std::max(1, nb);
    int grid = (int)std::max(1LL, std::min<long long>((d.n + 255) / 256, std::min<long long>(cap_rows, 148LL * 4)));
    double* rows = d_partials_;
    void* args[] = {&a, &rows};
    CT_CUDA(cudaLaunchKernel(k_part_, dim3(grid), dim3(256), args, 0, stream));
    ct_colsum_kernel<<<1, 256, 0, stream>>>(rows, grid, nb, d_out);
    CT_CUDA(cudaGetLastError());
}

void Engine::exportWeights(const double* d_params, const std::vector<int>& mask, double* d_total, double* d_partial,
                           double* d_interf_ev, double* d_interf, cudaStream_t stream)
{
    const Model& m = model_;
    const int nA = m.nAmp(), nc = m.nVector(), nb = nBlocks();
    const int npair = nb * (nb + 1) / 2;
    if (!mask.empty() && (int)mask.size() != nb) throw std::runtime_error("export: wave mask must have one entry per block");
    const DeviceSample& d = samples_[0];
    ct_prepare_kernel<<<(nA + 127) / 128, 128, 0, stream>>>(d_params, d_amp_chain_, d_ratio_, nA, nc, d_v_, nullptr);
    CT_CUDA(cudaGetLastError());
    CtArgsH a;
    std::memset(&a, 0, sizeof(a));
    a.s[0].slamp = d.slamp64;
    a.s[0].ev = d.ev64;
    a.s[0].w = d.w;
    a.s[0].n = d.n;
    a.s[0].ld = d.ld;
    a.s[0].cta_count = 1;
    a.nsamp = 1;
    a.theta = d_params + 2 * nc;
    a.v = d_v_;
    a.partials = d_partials_;
    a.consts = d_consts_;
    a.err = d_err_;
    void* pargs[] = {&a};
    CT_CUDA(cudaLaunchKernel(k_pro_, dim3(1), dim3(32), pargs, 0, stream));
    const int* dmask = nullptr;
    if (!mask.empty()) {
        CT_CUDA(cudaMemcpyAsync(d_mask_, mask.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, stream));
        dmask = d_mask_;
    }
    const int nacc = 2 + 2 * nA + m.nTheta();
    const long long cap_rows = (long long)grid_max_ * nacc / std::max(1, npair);
    int grid = (int)std::max(1LL, std::min<long long>((d.n + 255) / 256, std::min<long long>(cap_rows, 148LL * 4)));
    double* rows = d_partials_;
    void* args[] = {&a, &d_total, &d_partial, &d_interf_ev, &rows, &dmask};
    CT_CUDA(cudaLaunchKernel(k_exp_, dim3(grid), dim3(256), args, 0, stream));
    ct_colsum_kernel<<<1, 256, 0, stream>>>(rows, grid, npair, d_interf);
    CT_CUDA(cudaGetLastError());
}

void Engine::intensity(const double* d_params, int kind, double* d_out, cudaStream_t stream)
{
    if (kind < 0 || kind > 2 || samples_[kind].n == 0) throw std::runtime_error("intensity: empty or unknown sample");
    const Model& m = model_;
    int nA = m.nAmp(), nc = m.nVector();
    ct_prepare_kernel<<<(nA + 127) / 128, 128, 0, stream>>>(d_params, d_amp_chain_, d_ratio_, nA, nc, d_v_, nullptr);
    CT_CUDA(cudaGetLastError());
    CtArgsH a;
    std::memset(&a, 0, sizeof(a));
    const DeviceSample& d = samples_[kind];
    a.s[0].slamp = d.slamp64;
    a.s[0].ev = d.ev64;
    a.s[0].n = d.n;
    a.s[0].ld = d.ld;
    a.s[0].kind = kind;
    a.s[0].cta_count = 1;
    a.nsamp = 1;
    a.theta = d_params + 2 * nc;
    a.v = d_v_;
    a.partials = d_partials_;
    a.consts = d_consts_;
    a.err = d_err_;
    void* pargs[] = {&a};
    CT_CUDA(cudaLaunchKernel(k_pro_, dim3(1), dim3(32), pargs, 0, stream));
    void* args[] = {&a, &d_out};
    int grid = (int)std::min<long long>((d.n + 255) / 256, 148LL * 16);
    CT_CUDA(cudaLaunchKernel(k_int_, dim3(grid), dim3(256), args, 0, stream));
}

void Engine::setKernelTiming(int slots)
{
    CT_CUDA(cudaSetDevice(opt_.device));
    for (size_t i = 0; i < ev_begin_.size(); ++i) {
        cudaEventSynchronize(ev_end_[i]);
        cudaEventDestroy(ev_begin_[i]);
        cudaEventDestroy(ev_end_[i]);
    }
    ev_begin_.clear();
    ev_end_.clear();
    ev_count_ = 0;
    if (slots < 0 || slots > (1 << 20)) throw std::runtime_error("kernel timing: slots must be in [0, 2^20]");
    ev_begin_.resize(slots);
    ev_end_.resize(slots);
    for (int i = 0; i < slots; ++i) {
        CT_CUDA(cudaEventCreate(&ev_begin_[i]));
        CT_CUDA(cudaEventCreate(&ev_end_[i]));
    }
}

int Engine::kernelTimes(float* ms, int cap)
{
    if (ev_begin_.empty()) return 0;
    const long long ring = (long long)ev_begin_.size();
    const long long avail = std::min<long long>(ev_count_, ring);
    const long long n = std::min<long long>(avail, cap);
    for (long long i = 0; i < n; ++i) {
        const size_t slot = (size_t)((ev_count_ - n + i) % ring);
        CT_CUDA(cudaEventSynchronize(ev_end_[slot]));
        CT_CUDA(cudaEventElapsedTime(&ms[i], ev_begin_[slot], ev_end_[slot]));
    }
    return (int)n;
}

void Engine::lastParts(double* out6, cudaStream_t stream)
{
    CT_CUDA(cudaMemcpyAsync(out6, d_parts_, sizeof(double) * 6, cudaMemcpyDeviceToHost, stream));
    CT_CUDA(cudaStreamSynchronize(stream));
}

}  // namespace ctpwa
