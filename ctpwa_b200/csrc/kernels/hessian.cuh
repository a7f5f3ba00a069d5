// Hessian-vector products of the likelihood: forward mode over the adjoint.
//
// Compiled by NVRTC for sm_100a on the first Hessian request of a model, in a
// program of its own, with "model.cuh" (the model tables) and "model_dual.cuh"
// (generated: the lineshape products and their theta derivatives in dual
// numbers, model_prologue_dual / model_columns_dual).
//
// Every quantity of the per-event likelihood and adjoint pass (fused_nll.cuh)
// is carried as a dual number (value, derivative along a parameter direction
// u). The derivative part of the per-event gradient terms, summed over the
// events, is the directional derivative of the gradient sums; the host-side
// finalize turns it into H u exactly as the value sums become the gradient.
// With the unit directions this gives the full FP64 Hessian without storing
// any per-parameter table: the lineshapes, amplitudes and coherent sums are
// recomputed for each direction (the reference instead materialises second
// lineshape derivatives and forms the Hessian blocks from Gram matrices,
// src/ComputeHessian.cu:149-1556, src/AmpGen.cu:3020-3540).
//
// Grid: blockIdx.y = direction, blockIdx.x = CTA within the direction; the
// CTAs of a direction split the samples as the fused kernel does. Each CTA
// writes one row of tangent sums
//   [d nll, d sum f (phase space), d gv (re, im) x M_NA, d gt x M_NTH]
// for its sample. Phase-space coupling-gradient terms are not divided by the
// phase-space weight total here (the finalize does it).
#pragma once

#include "device_helpers.cuh"
#include "model.cuh"

// ---- first-order dual numbers ----
struct CtDual {
    double v, t;
    CtDual() = default;
    __device__ __forceinline__ constexpr CtDual(double x) : v(x), t(0.0) {}
    __device__ __forceinline__ constexpr CtDual(double x, double dx) : v(x), t(dx) {}
};
__device__ __forceinline__ CtDual operator+(CtDual a, CtDual b) { return CtDual(a.v + b.v, a.t + b.t); }
__device__ __forceinline__ CtDual operator-(CtDual a, CtDual b) { return CtDual(a.v - b.v, a.t - b.t); }
__device__ __forceinline__ CtDual operator-(CtDual a) { return CtDual(-a.v, -a.t); }
__device__ __forceinline__ CtDual operator*(CtDual a, CtDual b) { return CtDual(a.v * b.v, a.t * b.v + a.v * b.t); }
__device__ __forceinline__ CtDual operator/(CtDual a, CtDual b)
{
    const double q = a.v / b.v;
    return CtDual(q, (a.t - q * b.t) / b.v);
}
__device__ __forceinline__ CtDual operator+(CtDual a, double b) { return CtDual(a.v + b, a.t); }
__device__ __forceinline__ CtDual operator+(double a, CtDual b) { return CtDual(a + b.v, b.t); }
__device__ __forceinline__ CtDual operator-(CtDual a, double b) { return CtDual(a.v - b, a.t); }
__device__ __forceinline__ CtDual operator-(double a, CtDual b) { return CtDual(a - b.v, -b.t); }
__device__ __forceinline__ CtDual operator*(CtDual a, double b) { return CtDual(a.v * b, a.t * b); }
__device__ __forceinline__ CtDual operator*(double a, CtDual b) { return CtDual(a * b.v, a * b.t); }
__device__ __forceinline__ CtDual operator/(CtDual a, double b) { return CtDual(a.v / b, a.t / b); }
__device__ __forceinline__ CtDual operator/(double a, CtDual b)
{
    const double q = a / b.v;
    return CtDual(q, -q * b.t / b.v);
}
__device__ __forceinline__ CtDual& operator+=(CtDual& a, CtDual b)
{
    a.v += b.v;
    a.t += b.t;
    return a;
}
__device__ __forceinline__ bool operator>=(CtDual a, double b) { return a.v >= b; }
__device__ __forceinline__ bool operator>(CtDual a, double b) { return a.v > b; }
__device__ __forceinline__ bool operator<=(CtDual a, double b) { return a.v <= b; }
__device__ __forceinline__ bool operator<(CtDual a, double b) { return a.v < b; }
__device__ __forceinline__ bool operator==(CtDual a, double b) { return a.v == b; }
__device__ __forceinline__ CtDual sqrt(CtDual a)
{
    const double s = sqrt(a.v);
    return CtDual(s, 0.5 * a.t / s);
}
__device__ __forceinline__ CtDual log(CtDual a) { return CtDual(log(a.v), a.t / a.v); }
__device__ __forceinline__ CtDual exp(CtDual a)
{
    const double e = exp(a.v);
    return CtDual(e, e * a.t);
}
__device__ __forceinline__ CtDual sin(CtDual a) { return CtDual(sin(a.v), cos(a.v) * a.t); }
__device__ __forceinline__ CtDual cos(CtDual a) { return CtDual(cos(a.v), -sin(a.v) * a.t); }
__device__ __forceinline__ CtDual atan2(CtDual y, CtDual x)
{
    const double r = x.v * x.v + y.v * y.v;
    return CtDual(atan2(y.v, x.v), (x.v * y.t - y.v * x.t) / r);
}
__device__ __forceinline__ CtDual atan2(CtDual y, double x) { return atan2(y, CtDual(x)); }
__device__ __forceinline__ CtDual atan2(double y, CtDual x) { return atan2(CtDual(y), x); }
template <typename A, typename B>
struct CtSame {
    static constexpr bool value = false;
};
template <typename A>
struct CtSame<A, A> {
    static constexpr bool value = true;
};
__device__ __forceinline__ double ct_value(double x) { return x; }
__device__ __forceinline__ double ct_value(CtDual x) { return x.v; }

#include "model_dual.cuh"

#ifndef CT_HVP_BLOCK
#define CT_HVP_BLOCK 128
#endif
// paired polarisations (SL_{c,NPOL-1-p} = conj(SL_{c,p}) on every event): the
// tables hold polarisations 0 .. (M_NPOL+1)/2 - 1 only, [plane][p][ld]
#ifndef CT_HVP_PAIRED
#define CT_HVP_PAIRED 0
#endif

#define CT_HNACC (2 + 2 * M_NA + M_NTH)
#define CT_HCONST_ALLOC (M_NCONST > 0 ? M_NCONST : 1)

struct CtHvpSample {
    const double2* slamp;  // [M_NPLANE * M_NPOL][ld] angular values; paired: event-major [ld][M_NPLANE * stored]
    const double* ev;      // [M_NEV][ld] FP64 frontier values
    const double* w;       // per-event weights or nullptr
    long long n;
    long long ld;
    int kind;  // 0 = phase space, 1 = data, 2 = background
    int cta_begin;
    int cta_count;
    int pad;
};

struct CtHvpArgs {
    CtHvpSample s[3];
    int nsamp;
    int ndir;
    const double* theta;  // resonance parameters
    const double* v;      // couplings (re, im) x M_NA at the expansion point
    const double* dirs;   // [ndir][nparam] directions in [Re p, Im p, theta]
    const int* chain;     // coupling index of each amplitude column
    const double* ratio;  // its real ratio: v_a = ratio_a p_chain(a)
    int nc;
    int nparam;
    double* consts;       // [ndir][M_NCONST][2] dual parameter-only subexpressions
    double* rows;         // [ndir][ctas][CT_HNACC] tangent sums
    int ctas;             // CTAs per direction
    int pad;
};

// One thread per direction: the parameter-only subexpressions and their
// derivatives along the direction's theta part.
extern "C" __global__ void ct_hvp_prologue(CtHvpArgs A)
{
    const int d = blockIdx.x;
    if (threadIdx.x != 0 || d >= A.ndir) return;
    CtDual th[M_NTH > 0 ? M_NTH : 1];
    const double* u = A.dirs + (long long)d * A.nparam + 2 * A.nc;
#pragma unroll 1
    for (int j = 0; j < M_NTH; ++j) th[j] = CtDual(A.theta[j], u[j]);
    CtDual C[CT_HCONST_ALLOC];
    model_prologue_dual(th, C);
#pragma unroll 1
    for (int k = 0; k < M_NCONST; ++k) {
        A.consts[((long long)d * CT_HCONST_ALLOC + k) * 2] = C[k].v;
        A.consts[((long long)d * CT_HCONST_ALLOC + k) * 2 + 1] = C[k].t;
    }
}

__device__ __forceinline__ CtDual ct_clamp(CtDual x, double k)
{
    const double c = fmin(fmax(x.v, -k), k);
    return CtDual(c, c == x.v ? x.t : 0.0);
}

extern "C" __global__ void __launch_bounds__(CT_HVP_BLOCK) ct_hvp_f64(CtHvpArgs A)
{
    const int d = blockIdx.y, cta = blockIdx.x;
    int si = 0;
#pragma unroll
    for (int k = 1; k < 3; ++k)
        if (k < A.nsamp && cta >= A.s[k].cta_begin) si = k;
    const CtHvpSample& S = A.s[si];
    const int kind = S.kind;
    const double* __restrict__ u = A.dirs + (long long)d * A.nparam;

    // per-thread tangent sums in shared-memory slots (host-sized dynamic shared memory)
    extern __shared__ __align__(16) double ct_hacc[];
    double* acc = ct_hacc + threadIdx.x;
#pragma unroll 1
    for (int i = 0; i < CT_HNACC; ++i) acc[i * CT_HVP_BLOCK] = 0.0;

    __shared__ CtDual sC[CT_HCONST_ALLOC];
    __shared__ double sCv[CT_HCONST_ALLOC];
    for (int i = threadIdx.x; i < M_NCONST; i += CT_HVP_BLOCK) {
        const double* c = A.consts + ((long long)d * CT_HCONST_ALLOC + i) * 2;
        sC[i] = CtDual(c[0], c[1]);
        sCv[i] = c[0];
    }
    // does the direction move any resonance parameter?
    int moves = 0;
    for (int j = threadIdx.x; j < M_NTH; j += CT_HVP_BLOCK) moves |= u[2 * A.nc + j] != 0.0;
    const bool thdir = __syncthreads_or(moves);

    // couplings with their derivatives along the direction
    CtDual vr[M_NA], vi[M_NA];
#pragma unroll
    for (int a = 0; a < M_NA; ++a) {
        const int c = __ldg(A.chain + a);
        const double r = __ldg(A.ratio + a);
        vr[a] = CtDual(__ldg(A.v + 2 * a), r * u[c]);
        vi[a] = CtDual(__ldg(A.v + 2 * a + 1), r * u[A.nc + c]);
    }

    const long long n = S.n, ld = S.ld;
    const long long stride = (long long)S.cta_count * CT_HVP_BLOCK;
    // FT: type of the lineshapes and their derivatives, CtDual when the
    // direction moves a resonance parameter, plain FP64 when it moves only
    // couplings (the lineshapes do not move: no tangent arithmetic on them)
    auto run = [&](auto tag) {
        using FT = decltype(tag);
        for (long long e = (long long)(cta - S.cta_begin) * CT_HVP_BLOCK + threadIdx.x; e < n; e += stride) {
            double ev[M_NEV > 0 ? M_NEV : 1];
#pragma unroll
            for (int k = 0; k < M_NEV; ++k) ev[k] = __ldg(S.ev + (long long)k * ld + e);
            FT Fr[M_NTERM], Fi[M_NTERM], dFr[M_NDER > 0 ? M_NDER : 1], dFi[M_NDER > 0 ? M_NDER : 1];
            if constexpr (CtSame<FT, CtDual>::value) model_columns_dual(ev, sC, Fr, Fi, dFr, dFi);
            else model_columns(ev, sCv, Fr, Fi, dFr, dFi);
            constexpr int NPS = CT_HVP_PAIRED ? (M_NPOL + 1) / 2 : M_NPOL;
            double2 sl[M_NPLANE * NPS];
#pragma unroll
            for (int c = 0; c < M_NPLANE * NPS; ++c)
                sl[c] = CT_HVP_PAIRED ? __ldg(S.slamp + e * (M_NPLANE * NPS) + c)  // compact table: event-major
                                      : __ldg(S.slamp + (long long)c * ld + e);
            CtDual cr[M_NTERM], ci[M_NTERM];
#pragma unroll
            for (int t = 0; t < M_NTERM; ++t) {
                const int a = term_col(t);
                cr[t] = vr[a] * Fr[t] - vi[a] * Fi[t];
                ci[t] = vr[a] * Fi[t] + vi[a] * Fr[t];
            }
            CtDual Sr[M_NPOL], Si[M_NPOL];
#pragma unroll
            for (int p = 0; p < NPS; ++p) {
                const int q = M_NPOL - 1 - p;
                if (CT_HVP_PAIRED && q != p) {
                    // S_p = sum c (x + iy), S_q = sum c (x - iy) from the same products
                    CtDual xr(0.0), yi(0.0), yr(0.0), xi(0.0);
#pragma unroll
                    for (int t = 0; t < M_NTERM; ++t) {
                        const double2 x = sl[term_plane(t) * NPS + p];
                        xr += cr[t] * x.x;
                        yi += ci[t] * x.y;
                        yr += cr[t] * x.y;
                        xi += ci[t] * x.x;
                    }
                    Sr[p] = xr - yi;
                    Si[p] = yr + xi;
                    Sr[q] = xr + yi;
                    Si[q] = xi - yr;
                } else {
                    CtDual sr(0.0), sim(0.0);
#pragma unroll
                    for (int t = 0; t < M_NTERM; ++t) {
                        const double2 x = sl[term_plane(t) * NPS + p];
                        sr += cr[t] * x.x - ci[t] * x.y;
                        sim += cr[t] * x.y + ci[t] * x.x;
                    }
                    Sr[p] = sr;
                    Si[p] = sim;
                }
            }
            CtDual f(0.0);
#pragma unroll
            for (int p = 0; p < M_NPOL; ++p) f += Sr[p] * Sr[p] + Si[p] * Si[p];
            CtDual ur[M_NPOL], ui[M_NPOL];
            double gscale, tscale;
            const double we = S.w ? __ldg(S.w + e) : 1.0;
            if (kind == 0) {
                acc[1 * CT_HVP_BLOCK] += f.t;
#pragma unroll
                for (int p = 0; p < M_NPOL; ++p) {
                    ur[p] = Sr[p];
                    ui[p] = Si[p];
                }
                gscale = we;
                tscale = 2.0;
            } else {
                if (f.v == 0.0) continue;  // constant -w log(1e-10): no derivative
                acc[0] += -we * f.t / f.v;
                const CtDual inv = we / f;
#pragma unroll
                for (int p = 0; p < M_NPOL; ++p) {
                    ur[p] = ct_clamp(Sr[p] * inv, 1e10);
                    ui[p] = ct_clamp(Si[p] * inv, 1e10);
                }
                gscale = -1.0;
                tscale = -2.0;
            }
            // (paired: conj(SL_p) u_p + SL_p u_q = x (u_p + u_q) + iy (u_q - u_p))
            CtDual ar[NPS], br[NPS], ai[NPS], bi[NPS];
#pragma unroll
            for (int p = 0; p < NPS; ++p) {
                const int q = M_NPOL - 1 - p;
                if (CT_HVP_PAIRED && q != p) {
                    ar[p] = ur[p] + ur[q];
                    br[p] = ui[p] - ui[q];
                    ai[p] = ui[p] + ui[q];
                    bi[p] = ur[q] - ur[p];
                } else {
                    ar[p] = ur[p];
                    br[p] = ui[p];
                    ai[p] = ui[p];
                    bi[p] = -ur[p];
                }
            }
            CtDual Tr[M_NPLANE], Ti[M_NPLANE];
#pragma unroll
            for (int c = 0; c < M_NPLANE; ++c) {
                CtDual tr(0.0), ti(0.0);
#pragma unroll
                for (int p = 0; p < NPS; ++p) {
                    const double2 x = sl[c * NPS + p];
                    tr += x.x * ar[p] + x.y * br[p];
                    ti += x.x * ai[p] + x.y * bi[p];
                }
                Tr[c] = tr;
                Ti[c] = ti;
            }
#pragma unroll
            for (int t = 0; t < M_NTERM; ++t) {
                const int a = term_col(t), c = term_plane(t);
                acc[(2 + 2 * a) * CT_HVP_BLOCK] += gscale * (Fr[t] * Tr[c] + Fi[t] * Ti[c]).t;
                acc[(3 + 2 * a) * CT_HVP_BLOCK] += gscale * (Fr[t] * Ti[c] - Fi[t] * Tr[c]).t;
            }
            CtDual Wr[M_NTERM], Wi[M_NTERM];
#pragma unroll
            for (int t = 0; t < M_NTERM; ++t) {
                const int a = term_col(t), c = term_plane(t);
                Wr[t] = tscale * (vr[a] * Tr[c] + vi[a] * Ti[c]);
                Wi[t] = tscale * (vi[a] * Tr[c] - vr[a] * Ti[c]);
            }
#pragma unroll
            for (int k = 0; k < M_NDER; ++k) {
                const int t = der_term(k);
                acc[(2 + 2 * M_NA + der_th(k)) * CT_HVP_BLOCK] += (dFr[k] * Wr[t] - dFi[k] * Wi[t]).t;
            }
        }
    };
    if (thdir) run(CtDual(0.0));
    else run(0.0);
    __syncthreads();
    // CTA sums, one warp per column in a fixed order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* row = A.rows + ((long long)d * A.ctas + cta) * CT_HNACC;
    for (int i = warp; i < CT_HNACC; i += CT_HVP_BLOCK / 32) {
        double s = 0.0;
        for (int j = lane; j < CT_HVP_BLOCK; j += 32) s += ct_hacc[i * CT_HVP_BLOCK + j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) row[i] = s;
    }
}
