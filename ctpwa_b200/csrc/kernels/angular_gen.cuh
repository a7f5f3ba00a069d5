// Building blocks of the generated angular kernels (one kernel per decay
// group, emitted by Engine::angularSource and compiled with NVRTC).
//
// The same mathematics as the interpreted ag_group_kernel (engine.cu): the
// two-body spin-orbit amplitude of every decay vertex,
//   T[s][s1][s2] = 10 q^L <j1 s1 j2 s2|S s1+s2> <S s1+s2, L m|J s> / sqrt(2J+1) Y_L^m(theta, -phi)
// followed by the daughters' Wigner rotations (the reference's pwa_amp,
// src/Amplitude.cu:237-644), contracted along the chain
// (src/AmpGen.cu:1034-1219). Here the tensor shapes are template arguments,
// so every loop unrolls and the tensors live in registers, and a vertex's
// frame and rotations are computed once per event for all of its (S, L)
// variants. The operations and their order follow the interpreter's, so both
// give the same values.
#pragma once

#define AG_MAXD 7
// pi to double precision (NVRTC compiles without the host math headers)
#define AG_PI 3.141592653589793

struct AgTables {
    const void* vars;
    const double* cg;        // CG products
    const double* ylm_norm;  // [l][|m|]
    const double* dcoef;     // Wigner small-d sum coefficients
    const int* doff;         // [dim][m1][m2] -> offset into dcoef (count first)
};

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
__device__ __forceinline__ void agFrame(const V4& p1, const V4& p2, double& theta, double& phi, double& q)
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
__device__ __forceinline__ double agLegendre(int l, int m, double x)
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

// D-matrix element e^{i m1 a} d(b) e^{i m2 g}, m = (dim - 1 - 2 i) / 2.
// cos(b/2), sin(b/2) and their powers, and the phases of each row and
// column, are formed once per matrix (the interpreter forms them per
// element from the same arguments, by the same products: equal values).
template <int DIM>
__device__ __forceinline__ void agDMatrix(const AgTables& T, double a, double b, double g, double2* out)
{
    const double ch = cos(b / 2.0), sh = sin(b / 2.0);
    double chp[DIM], shp[DIM];  // ch^k, sh^k as 1 * x * x ... (ipow)
    chp[0] = 1.0;
    shp[0] = 1.0;
#pragma unroll
    for (int k = 1; k < DIM; ++k) {
        chp[k] = chp[k - 1] * ch;
        shp[k] = shp[k - 1] * sh;
    }
    double s1[DIM], c1[DIM], s2[DIM], c2[DIM];
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
        const double m = (DIM - 1 - 2 * i) / 2.0;
        sincos(m * a, &s1[i], &c1[i]);
        sincos(m * g, &s2[i], &c2[i]);
    }
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
            const double* t = T.dcoef + T.doff[(DIM * AG_MAXD + i) * AG_MAXD + j];
            const int cnt = (int)t[0];
            double d = 0.0;
            for (int k = 0; k < cnt; ++k) d += t[1 + 3 * k] * chp[(int)t[2 + 3 * k]] * shp[(int)t[3 + 3 * k]];
            out[i * DIM + j] = cmul(make_double2(c1[i] * d, s1[i] * d), make_double2(c2[j], s2[j]));
        }
    }
}

template <int N>
__device__ __forceinline__ void agMatMul(const double2* a, const double2* b, double2* c)
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            double2 s = make_double2(0, 0);
#pragma unroll
            for (int k = 0; k < N; ++k) s = cadd(s, cmul(a[i * N + k], b[k * N + j]));
            c[i * N + j] = s;
        }
}

// Wigner rotation of a massive particle q as seen from P (reference MassiveTrans)
template <int DIM>
__device__ __forceinline__ void agMassive(const AgTables& T, const V4& P, const V4& q, double2* tr)
{
#pragma unroll
    for (int i = 0; i < DIM * DIM; ++i) tr[i] = make_double2(0, 0);
#pragma unroll
    for (int i = 0; i < DIM; ++i) tr[i * DIM + i] = make_double2(1, 0);
    if (DIM == 1) return;
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
    double2 w1[DIM * DIM], w2[DIM * DIM];
    agDMatrix<DIM>(T, -ph, -th, -psi, w1);
    agDMatrix<DIM>(T, 0.0, th, ph, w2);
    agMatMul<DIM>(w1, w2, tr);
}

// massless-particle phase rotation (reference MasslessTrans)
template <int DIM>
__device__ __forceinline__ void agMassless(const V4& P, const V4& p, double2* tr)
{
#pragma unroll
    for (int i = 0; i < DIM * DIM; ++i) tr[i] = make_double2(0, 0);
#pragma unroll
    for (int i = 0; i < DIM; ++i) tr[i * DIM + i] = make_double2(1, 0);
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
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
        double m2 = (DIM - 1 - 2 * i) / 2.0, s, c;
        sincos(m2 * tot, &s, &c);
        tr[i * DIM + i] = make_double2(c, s);
    }
}

template <int DIM>
__device__ __forceinline__ void agDLeft(const AgTables& T, double2* mat, double a, double b, double g)
{
    double2 d[DIM * DIM], t[DIM * DIM];
    agDMatrix<DIM>(T, a, b, g, d);
    agMatMul<DIM>(d, mat, t);
#pragma unroll
    for (int i = 0; i < DIM * DIM; ++i) mat[i] = t[i];
}

// one vertex's frame and its daughters' rotations, shared by its (S, L) variants
template <int DJ1, int DJ2>
struct AgVertexFrame {
    double theta, phi, q, x;
    double2 t1[DJ1 * DJ1], t2[DJ2 * DJ2];
};

template <int DJ1, int DJ2>
__device__ __forceinline__ void agVertexFrame(const AgTables& T, const V4& p1, const V4& p2, AgVertexFrame<DJ1, DJ2>& F)
{
    agFrame(p1, p2, F.theta, F.phi, F.q);
    F.x = cos(F.theta);
    V4 Pt = v4add(p1, p2);
    if (v4mass(p1) > 1e-10) agMassive<DJ1>(T, Pt, p1, F.t1);
    else {
        agMassless<DJ1>(Pt, p1, F.t1);
        agDLeft<DJ1>(T, F.t1, -F.phi, -F.theta, 0.0);
    }
    if (v4mass(p2) > 1e-10) agMassive<DJ2>(T, Pt, p2, F.t2);
    else {
        agMassless<DJ2>(Pt, p2, F.t2);
        agDLeft<DJ2>(T, F.t2, -(AG_PI + F.phi), -(AG_PI - F.theta), 0.0);
    }
}

// the vertex tensor amp[s][s1][s2] of the (S, L) variant whose CG products
// start at cg (dj * dj1 * dj2 doubles), x10
template <int DJ, int DJ1, int DJ2, int L>
__device__ __forceinline__ void agVertexAmp(const AgTables& T, const AgVertexFrame<DJ1, DJ2>& F, const double* cg,
                                            double2* amp)
{
    constexpr int KD = DJ1 * DJ2;
    const double ql = ipow(F.q, L);
    // Y_L^m(theta, -phi) for m = -L .. L, once each
    double2 ylm[2 * L + 1];
#pragma unroll
    for (int m = -L; m <= L; ++m) {
        const int am = m < 0 ? -m : m;
        double P = agLegendre(L, am, F.x);
        double a = T.ylm_norm[L * AG_MAXD + am] * P;
        if (m < 0 && (am & 1)) a = -a;
        double sn, cs;
        sincos(m * (-F.phi), &sn, &cs);
        ylm[m + L] = make_double2(a * cs, a * sn);
    }
#pragma unroll
    for (int s = 0; s < DJ; ++s) {
        const int sx2 = DJ - 1 - 2 * s;
#pragma unroll
        for (int s1 = 0; s1 < DJ1; ++s1) {
            const int s1x2 = DJ1 - 1 - 2 * s1;
#pragma unroll
            for (int s2 = 0; s2 < DJ2; ++s2) {
                const int s2x2 = DJ2 - 1 - 2 * s2;
                const double c = cg[s * KD + s1 * DJ2 + s2];
                double2 y = make_double2(0, 0);
                const int m = (sx2 - s1x2 - s2x2) / 2;
                const int am = m < 0 ? -m : m;
                if (c != 0.0 && am <= L) y = ylm[m + L];
                amp[s * KD + s1 * DJ2 + s2] = make_double2(ql * c * y.x, ql * c * y.y);
            }
        }
    }
    if (DJ1 != 1 || DJ2 != 1) {
        double2 mid[KD];
#pragma unroll
        for (int s = 0; s < DJ; ++s) {
            double2* a = amp + s * KD;
#pragma unroll
            for (int n1 = 0; n1 < DJ1; ++n1)
#pragma unroll
                for (int o2 = 0; o2 < DJ2; ++o2) {
                    double2 sum = make_double2(0, 0);
#pragma unroll
                    for (int o1 = 0; o1 < DJ1; ++o1) sum = cadd(sum, cmul(F.t1[n1 + DJ1 * o1], a[o1 * DJ2 + o2]));
                    mid[n1 * DJ2 + o2] = sum;
                }
#pragma unroll
            for (int n1 = 0; n1 < DJ1; ++n1)
#pragma unroll
                for (int n2 = 0; n2 < DJ2; ++n2) {
                    double2 sum = make_double2(0, 0);
#pragma unroll
                    for (int o2 = 0; o2 < DJ2; ++o2) sum = cadd(sum, cmul(mid[n1 * DJ2 + o2], F.t2[n2 + DJ2 * o2]));
                    a[n1 * DJ2 + n2] = sum;
                }
        }
    } else {
        double2 r = cmul(F.t1[0], F.t2[0]);
        if (r.x != 1.0 || r.y != 0.0)
#pragma unroll
            for (int s = 0; s < DJ; ++s) amp[s] = cmul(r, amp[s]);
    }
#pragma unroll
    for (int i = 0; i < DJ * KD; ++i) amp[i] = make_double2(amp[i].x * 10.0, amp[i].y * 10.0);
}

// one step of the chain contraction, generated as a list of output elements:
// out[i] = sum over sg of cur[ci + sg * cs] * node[(sg * dj1 + e1) * dj2 + e2]
template <int SH, int DJ1, int DJ2>
__device__ __forceinline__ double2 agContract(const double2* cur, int ci, int cs, const double2* node, int e1, int e2)
{
    double2 sum = make_double2(0, 0);
#pragma unroll
    for (int sg = 0; sg < SH; ++sg) sum = cadd(sum, cmul(cur[ci + sg * cs], node[(sg * DJ1 + e1) * DJ2 + e2]));
    return sum;
}

// one kinematic-cache value (type codes of AG_K_* in angular.cuh): particle
// a, and for the breakup momenta its daughters b and c
template <int TYPE>
__device__ __forceinline__ double agKin(const V4& a, const V4& b, const V4& c)
{
    if constexpr (TYPE == 0) {  // mass
        return v4mass(a);
    } else if constexpr (TYPE == 1) {  // breakup momentum, 0 below threshold
        double m = v4mass(a), m1 = v4mass(b), m2 = v4mass(c);
        double q2 = (m * m - (m1 + m2) * (m1 + m2)) * (m * m - (m1 - m2) * (m1 - m2));
        return q2 <= 0.0 ? 0.0 : sqrt(q2) / (2.0 * m);
    } else if constexpr (TYPE == 2) {  // breakup momentum without the clamp
        double m = v4mass(a), m1 = v4mass(b), m2 = v4mass(c);
        return sqrt((m * m - (m1 + m2) * (m1 + m2)) * (m * m - (m1 - m2) * (m1 - m2))) / 2 / m;
    } else if constexpr (TYPE == 3) {  // |p|
        return v4p(a);
    } else if constexpr (TYPE == 4) {  // E
        return a.E;
    } else if constexpr (TYPE == 5) {  // cos(theta) of p
        double pp = v4p(a);
        return pp > 0 ? a.z / pp : 0.0;
    } else {  // phi of p
        return atan2(a.y, a.x);
    }
}

// |x + iy| with a NaN counted as infinitely far (the pairing check's
// distance), and the maximum over a warp (all lanes take part)
__device__ __forceinline__ double agDist(double x, double y)
{
    const double d = hypot(x, y);
    return d == d ? d : __longlong_as_double(0x7ff0000000000000LL);
}
__device__ __forceinline__ double agWarpMax(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
