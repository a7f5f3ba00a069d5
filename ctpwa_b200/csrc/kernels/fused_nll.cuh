// Fused likelihood + adjoint kernel (one streaming pass per evaluation).
//
// Compiled by NVRTC for sm_100a together with a generated header "model.cuh"
// that supplies, for one physics model:
//   M_NA, M_NPOL, M_NPLANE, M_NKIN, M_NTH, M_NDER     sizes
//   col_plane(a)   angular plane (group, SL combination) of amplitude column a
//   der_col(k), der_th(k)   column / theta index of derivative entry k
//   model_columns(kin, th, Fr, Fi, dFr, dFi)   lineshape products F_a and their
//       theta derivatives for one event (straight-line generated code)
//
// Per event e of a sample (phase space, data or background) the kernel forms
//   A_{a,p} = F_a * SL_{plane(a),p},   S_p = sum_a v_a A_{a,p},   f = sum_p |S_p|^2
// and accumulates, per thread, in FP64:
//   data/bkg: nll += -w log f;  u_p = clamp(w S_p / f);  T_c = sum_p conj(SL_{c,p}) u_p
//             gv_a += -conj(F_a) T_{plane(a)};  gt_j += -2 Re(v_a dF_{a,j} conj(T_{plane(a)}))
//   phsp:     fsum += f;  T_c = sum_p conj(SL_{c,p}) S_p
//             gv_a += (w/W) conj(F_a) T_{plane(a)};  gt_j += 2 Re(v_a dF_{a,j} conj(T_{plane(a)}))
// which are the per-event terms of the reference's NLL and gradients
// (src/ComputeNLL.cu:21-84 and 312-407, src/AmpGen.cu:2762-2822,
// src/Analysis.cu:729-1183). The pass never materialises A, S or w in HBM.
// Each CTA reduces its threads' accumulators with warp shuffles and shared
// memory and writes one row of partial sums; a separate finalize kernel sums
// the rows in a fixed order, so results are bit-reproducible.
//
// R is the arithmetic type of the per-polarisation complex algebra (double for
// the plain path, float for the mixed path); SL2 is the stored angular-table
// element (double2 / float2). Lineshapes, the log and all accumulations are FP64.
// Parameter-only parts of the lineshapes are computed once per call by
// ct_prologue and staged in shared memory by every CTA.
#pragma once

#include "device_helpers.cuh"
#include "model.cuh"

#ifndef CT_BLOCK
#define CT_BLOCK 256
#endif

#define CT_NACC (2 + 2 * M_NA + M_NTH)

struct CtSample {
    const void* slamp;  // [M_NPLANE * M_NPOL planes][n] of SL2
    const double* kin;  // [M_NKIN][n]
    const double* w;    // per-event weights or nullptr (unit weights)
    long long n;
    int kind;           // 0 = phase space, 1 = data, 2 = background
    int cta_begin;
    int cta_count;
    int pad;
    double vw_scale;    // phase space: 1 / sum of weights (v-gradient weighting)
};

struct CtArgs {
    CtSample s[3];
    int nsamp;
    int pad;
    const double* theta;  // fitted resonance parameters
    const double* v;      // couplings, interleaved (re, im) x M_NA
    double* partials;     // [gridDim.x][CT_NACC]
    double* consts;       // [M_NCONST] parameter-only subexpressions of this call
};

// One thread: the parameter-only part of every lineshape (prologue).
extern "C" __global__ void ct_prologue(CtArgs A)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) model_prologue(A.theta, A.consts);
}

#define CT_NCONST_ALLOC (M_NCONST > 0 ? M_NCONST : 1)

__device__ __forceinline__ void ct_stage_consts(const CtArgs& A, double* sC)
{
    for (int i = threadIdx.x; i < M_NCONST; i += blockDim.x) sC[i] = A.consts[i];
    __syncthreads();
}

template <typename T>
struct CtVec2;
template <>
struct CtVec2<double> {
    typedef double2 type;
};
template <>
struct CtVec2<float> {
    typedef float2 type;
};

template <typename R>
__device__ __forceinline__ void ct_block_reduce_store(double* acc, double* out)
{
    __shared__ double red[CT_BLOCK / 32][CT_NACC];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < CT_NACC; ++i) {
        double x = acc[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp][i] = x;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < CT_NACC; i += CT_BLOCK) {
        double x = 0.0;
#pragma unroll
        for (int w = 0; w < CT_BLOCK / 32; ++w) x += red[w][i];
        out[i] = x;
    }
}

template <typename R>
__device__ __forceinline__ void ct_fused_body(const CtArgs& A)
{
    typedef typename CtVec2<R>::type SL2;
    // which sample does this CTA serve?
    int si = 0;
#pragma unroll
    for (int k = 1; k < 3; ++k)
        if (k < A.nsamp && (int)blockIdx.x >= A.s[k].cta_begin) si = k;
    const CtSample& S = A.s[si];
    const int kind = S.kind;
    const long long n = S.n;
    const SL2* __restrict__ slamp = (const SL2*)S.slamp;
    const double* __restrict__ kin = S.kin;
    const double* __restrict__ wts = S.w;

    double acc[CT_NACC];
#pragma unroll
    for (int i = 0; i < CT_NACC; ++i) acc[i] = 0.0;

    __shared__ double sC[CT_NCONST_ALLOC];
    ct_stage_consts(A, sC);
    double vr[M_NA], vi[M_NA];
#pragma unroll
    for (int a = 0; a < M_NA; ++a) {
        vr[a] = __ldg(A.v + 2 * a);
        vi[a] = __ldg(A.v + 2 * a + 1);
    }

    const long long stride = (long long)S.cta_count * CT_BLOCK;
    for (long long e = (long long)(blockIdx.x - S.cta_begin) * CT_BLOCK + threadIdx.x; e < n; e += stride) {
        // ---- lineshapes (FP64, with theta derivatives) ----
        double kv[M_NKIN > 0 ? M_NKIN : 1];
#pragma unroll
        for (int k = 0; k < M_NKIN; ++k) kv[k] = __ldg(kin + (long long)k * n + e);
        double Fr[M_NA], Fi[M_NA], dFr[M_NDER > 0 ? M_NDER : 1], dFi[M_NDER > 0 ? M_NDER : 1];
        model_columns(kv, sC, Fr, Fi, dFr, dFi);

        // ---- coherent sum over amplitudes ----
        SL2 sl[M_NPLANE * M_NPOL];
#pragma unroll
        for (int c = 0; c < M_NPLANE * M_NPOL; ++c) sl[c] = slamp[(long long)c * n + e];
        R cr[M_NA], ci[M_NA];
#pragma unroll
        for (int a = 0; a < M_NA; ++a) {
            cr[a] = (R)(vr[a] * Fr[a] - vi[a] * Fi[a]);
            ci[a] = (R)(vr[a] * Fi[a] + vi[a] * Fr[a]);
        }
        R Sr[M_NPOL], Si[M_NPOL];
        R f = (R)0;
#pragma unroll
        for (int p = 0; p < M_NPOL; ++p) {
            R sr = (R)0, sim = (R)0;
#pragma unroll
            for (int a = 0; a < M_NA; ++a) {
                SL2 x = sl[col_plane(a) * M_NPOL + p];
                sr += cr[a] * x.x - ci[a] * x.y;
                sim += cr[a] * x.y + ci[a] * x.x;
            }
            Sr[p] = sr;
            Si[p] = sim;
            f += sr * sr + sim * sim;
        }

        // ---- per-event weight of the adjoint ----
        const double we = wts ? __ldg(wts + e) : 1.0;
        R ur[M_NPOL], ui[M_NPOL];
        R gscale;  // factor applied to v-gradient contributions
        R tscale;  // factor applied to theta-gradient contributions
        if (kind == 0) {
            acc[1] += (double)f;
#pragma unroll
            for (int p = 0; p < M_NPOL; ++p) {
                ur[p] = Sr[p];
                ui[p] = Si[p];
            }
            gscale = (R)(we * S.vw_scale);
            tscale = (R)2;
        } else {
            if (f == (R)0) {
                acc[0] += -log(1e-10) * we;
                continue;
            }
            acc[0] += -log((double)f) * we;
            const R inv = (R)(we / (double)f);
            const R kmax = (R)1e10;
#pragma unroll
            for (int p = 0; p < M_NPOL; ++p) {
                ur[p] = fmin(fmax(Sr[p] * inv, -kmax), kmax);
                ui[p] = fmin(fmax(Si[p] * inv, -kmax), kmax);
            }
            gscale = (R)-1;
            tscale = (R)-2;
        }
        // T_c = sum_p conj(SL_{c,p}) u_p
        R Tr[M_NPLANE], Ti[M_NPLANE];
#pragma unroll
        for (int c = 0; c < M_NPLANE; ++c) {
            R tr = (R)0, ti = (R)0;
#pragma unroll
            for (int p = 0; p < M_NPOL; ++p) {
                SL2 x = sl[c * M_NPOL + p];
                tr += x.x * ur[p] + x.y * ui[p];
                ti += x.x * ui[p] - x.y * ur[p];
            }
            Tr[c] = tr;
            Ti[c] = ti;
        }
        // v-gradient: conj(F_a) T
#pragma unroll
        for (int a = 0; a < M_NA; ++a) {
            const int c = col_plane(a);
            R fr = (R)Fr[a], fi = (R)Fi[a];
            acc[2 + 2 * a] += (double)(gscale * (fr * Tr[c] + fi * Ti[c]));
            acc[3 + 2 * a] += (double)(gscale * (fr * Ti[c] - fi * Tr[c]));
        }
        // theta-gradient: Re(v_a dF conj(T))
#pragma unroll
        for (int k = 0; k < M_NDER; ++k) {
            const int a = der_col(k), c = col_plane(a);
            double xr = vr[a] * dFr[k] - vi[a] * dFi[k];
            double xi = vr[a] * dFi[k] + vi[a] * dFr[k];
            R re = (R)xr * Tr[c] + (R)xi * Ti[c];
            acc[2 + 2 * M_NA + der_th(k)] += (double)(tscale * re);
        }
    }
    ct_block_reduce_store<R>(acc, A.partials + (long long)blockIdx.x * CT_NACC);
}

extern "C" __global__ void __launch_bounds__(CT_BLOCK) ct_fused_f64(CtArgs a) { ct_fused_body<double>(a); }
extern "C" __global__ void __launch_bounds__(CT_BLOCK) ct_fused_mixed(CtArgs a) { ct_fused_body<float>(a); }

// Per-event intensity f_e = sum_p |S_p|^2 of sample s[0] (FP64), for
// accept-reject toy generation and per-event weights.
extern "C" __global__ void __launch_bounds__(CT_BLOCK) ct_intensity_f64(CtArgs A, double* __restrict__ out)
{
    const CtSample& S = A.s[0];
    const long long n = S.n;
    const double2* __restrict__ slamp = (const double2*)S.slamp;
    __shared__ double sC[CT_NCONST_ALLOC];
    ct_stage_consts(A, sC);
    for (long long e = (long long)blockIdx.x * CT_BLOCK + threadIdx.x; e < n; e += (long long)gridDim.x * CT_BLOCK) {
        double kv[M_NKIN > 0 ? M_NKIN : 1];
#pragma unroll
        for (int k = 0; k < M_NKIN; ++k) kv[k] = __ldg(S.kin + (long long)k * n + e);
        double Fr[M_NA], Fi[M_NA], dFr[M_NDER > 0 ? M_NDER : 1], dFi[M_NDER > 0 ? M_NDER : 1];
        model_columns(kv, sC, Fr, Fi, dFr, dFi);
        double f = 0.0;
#pragma unroll
        for (int p = 0; p < M_NPOL; ++p) {
            double sr = 0.0, si = 0.0;
#pragma unroll
            for (int a = 0; a < M_NA; ++a) {
                double cr = __ldg(A.v + 2 * a) * Fr[a] - __ldg(A.v + 2 * a + 1) * Fi[a];
                double ci = __ldg(A.v + 2 * a) * Fi[a] + __ldg(A.v + 2 * a + 1) * Fr[a];
                double2 x = slamp[(long long)(col_plane(a) * M_NPOL + p) * n + e];
                sr += cr * x.x - ci * x.y;
                si += cr * x.y + ci * x.x;
            }
            f += sr * sr + si * si;
        }
        out[e] = f;
    }
}
