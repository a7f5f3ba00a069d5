// Fused likelihood + adjoint kernel (one streaming pass per evaluation).
//
// Compiled by NVRTC for sm_100a together with a generated header "model.cuh"
// that supplies, for one physics model:
//   M_NA, M_NTERM, M_NPOL, M_NPLANE, M_NKIN, M_NTH, M_NDER     sizes
//   M_NEV, M_NEVF, M_NEVD   rows of the per-event frontier tables (FP64; mixed
//       form FP32 and FP64)
//   term_col(t), term_plane(t)   amplitude column and angular plane (group
//       variant, SL combination) of term t: a column is the sum of its terms
//       (one term, or one per permutation of identical particles)
//   der_term(k), der_th(k)   term / theta index of derivative entry k
//   model_prologue(theta, C)   parameter-only subexpressions, once per call
//   model_event(kin, o), model_event_mx(o, of, od)   the parameter-independent
//       per-event values the per-call code reads (frontier), evaluated once
//       per event by ct_event_cache when a sample is loaded (FP64; the mixed
//       form's FP32 / FP64 rows are those values rounded once)
//   model_columns(ev, C, Fr, Fi, dFr, dFi)   lineshape products F_a and their
//       theta derivatives for one event from its frontier values
//       (straight-line generated code, FP64)
//   model_columns_f32(...)   the same in the mixed form (FP32 except the
//       cancellation-prone polynomial parts such as m0^2 - m^2)
//
// Per event e of a sample (phase space, data or background) the kernel forms
//   A_{a,p} = F_a * SL_{plane(a),p},   S_p = sum_a v_a A_{a,p},   f = sum_p |S_p|^2
// and accumulates, per thread:
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
// Precision. Plain path (ct_fused_f64): everything FP64. Mixed form
// (ct_fused_mixed): FP32 angular tables, FP32 lineshapes (cancellation-prone
// parts FP64, see model_columns_f32), FP32 per-polarisation algebra and
// per-thread gradient sums. The log, the log-likelihood and phase-space
// intensity sums and every cross-thread reduction are FP64 in both forms.
// Parameter-only parts of the lineshapes are computed once per call by
// ct_prologue and, with the couplings, read from the constant bank.
#pragma once

#include "device_helpers.cuh"
#include "model.cuh"

#ifndef CT_BLOCK
#define CT_BLOCK 256
#endif

#define CT_NACC (2 + 2 * M_NA + M_NTH)

// shared-memory staging of the event tables: 0 off; by per-warp bulk copies
// 1 the frontier rows, 2 the frontier and angular rows; 3 the frontier values
// by per-thread asynchronous copies (the host sets it when the two buffers
// fit at the requested residency)
#ifndef CT_F64_STAGE
#define CT_F64_STAGE 0
#endif
#ifndef CT_MX_STAGE
#define CT_MX_STAGE 0
#endif
// per-thread gradient sums in shared memory instead of registers
#ifndef CT_F64_ACC
#define CT_F64_ACC 1
#endif
#ifndef CT_MX_ACC
#define CT_MX_ACC 0
#endif
#ifndef CT_WAIT_LIMIT
#define CT_WAIT_LIMIT (1u << 22)
#endif

struct CtSample {
    const void* slamp;  // full FP64: [M_NPLANE * M_NPOL planes][ld] of SL2; FP32 and paired FP64: event-major records
    const void* ev;     // frontier rows [M_NEV][ld] FP64 (plain), [M_NEVF][ld] FP32 (mixed)
    const double* evd;  // mixed form: FP64 frontier rows [M_NEVD][ld]
    const double* w;    // per-event weights or nullptr (unit weights)
    long long n;
    long long ld;       // row stride of slamp and the frontier rows: n padded to a multiple of 256
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
    double* partials;     // [total CTAs][CT_NACC]
    double* consts;       // [M_NCONST] parameter-only subexpressions of this call
    int cta_base;         // CTA index of this launch's first block (split launches)
    int pad2;
    int* err;             // set to 1 when a staged copy did not arrive in time
    void* kblock;         // CtConsts image of this call (written by ct_prologue) or nullptr
};

#define CT_NCONST_ALLOC (M_NCONST > 0 ? M_NCONST : 1)

// Conjugate-paired polarisations: when every event satisfies
// SL_{plane, npol-1-q} = conj(SL_{plane, q}) (checked on all samples when they
// are loaded), the angular tables of the fused kernels store the first
// CT_NPOL_STORED polarisations only, [plane][q][ld], and the *_pc kernels
// rebuild the others as conjugates (the negation folds into the FMAs).
#define CT_NPOL_STORED ((M_NPOL + 1) / 2)
// The FP32 angular table is event-major: each event's NPL complex values
// (NPL = M_NPLANE x the stored polarisations) in one record of an even
// number of float2, read as float4; the FP64 tables are [row][ld].
#define CT_SL32_STRIDE(NPL) (((NPL) + 1) / 2 * 2)

// Per-call constants of the fused kernels in the constant bank: the
// parameter-only subexpressions (FP64, and FP32 hi + lo pairs) and the
// couplings (FP64, and FP32 hi + lo pairs). ct_prologue writes their image
// into a device buffer, which the host copies to ct_k before each fused
// launch; the fused kernels read them as constant-bank operands, with no load
// instruction or register per use.
struct CtConsts {
    double c[CT_NCONST_ALLOC];
    double v[2 * M_NA];
    float ch[CT_NCONST_ALLOC], cl[CT_NCONST_ALLOC];
    float vh[2 * M_NA];  // the couplings rounded to FP32 (the mixed form's; see ct_fused_body)
};
__constant__ CtConsts ct_k;

// The parameter-only part of every lineshape (prologue, one thread), then
// the constant-bank image of this call (one warp).
__device__ __forceinline__ void ct_prologue_body(const CtArgs& A);
extern "C" __global__ void ct_prologue(CtArgs A)
{
    if (blockIdx.x != 0) return;
    ct_prologue_body(A);
}
// one block per job of a multi-job evaluation
extern "C" __global__ void ct_prologue_multi(const CtArgs* __restrict__ jobs) { ct_prologue_body(jobs[blockIdx.x]); }

__device__ __forceinline__ void ct_prologue_body(const CtArgs& A)
{
    if (threadIdx.x == 0) model_prologue(A.theta, A.consts);
    __syncthreads();
    if (!A.kblock) return;
    CtConsts* K = (CtConsts*)A.kblock;
    for (int i = threadIdx.x; i < M_NCONST; i += blockDim.x) {
        const double c = A.consts[i];
        const float h = (float)c;
        K->c[i] = c;
        K->ch[i] = h;
        K->cl[i] = (float)(c - (double)h);
    }
    for (int i = threadIdx.x; i < 2 * M_NA; i += blockDim.x) {
        const double v = A.v[i];
        const float h = (float)v;
        K->v[i] = v;
        K->vh[i] = h;
    }
}

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

// CTA reduction of the per-thread accumulators: two FP64 sums (log-likelihood
// and phase-space intensity) and the gradient terms (type G), reduced in FP64.
// Per-thread gradient sums: in registers, or (SMEM) in a shared-memory slot
// per thread, which frees registers at the cost of a shared load and store
// per update.
template <typename L, int BLOCK, bool SMEM>
struct CtAccG;
template <typename L, int BLOCK>
struct CtAccG<L, BLOCK, false> {
    L v[CT_NACC - 2];
    __device__ __forceinline__ void init(unsigned char*)
    {
#pragma unroll
        for (int i = 0; i < CT_NACC - 2; ++i) v[i] = (L)0;
    }
    __device__ __forceinline__ void add(int i, L x) { v[i] += x; }
    __device__ __forceinline__ L operator[](int i) const { return v[i]; }
};
template <typename L, int BLOCK>
struct CtAccG<L, BLOCK, true> {
    L* p;
    // slot: the start of the CTA's dynamic shared memory (host-sized)
    __device__ __forceinline__ void init(unsigned char* slot)
    {
        p = (L*)slot + threadIdx.x;
#pragma unroll
        for (int i = 0; i < CT_NACC - 2; ++i) p[i * BLOCK] = (L)0;
    }
    __device__ __forceinline__ void add(int i, L x) { p[i * BLOCK] += x; }
    __device__ __forceinline__ L operator[](int i) const { return p[i * BLOCK]; }
};

// (the v-gradient sums are scaled by vscale and the theta-gradient sums by
// tscale on the way out: the per-event factors common to a CTA's sample)
template <int BLOCK, typename G>
__device__ __forceinline__ void ct_block_reduce_store(const double* accd, const G& accg, double* out, double vscale,
                                                      double tscale)
{
    __shared__ double red[BLOCK / 32][CT_NACC];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < CT_NACC; ++i) {
        double x = i < 2 ? accd[i] : (double)accg[i - 2];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp][i] = x;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < CT_NACC; i += BLOCK) {
        double x = 0.0;
#pragma unroll
        for (int w = 0; w < BLOCK / 32; ++w) x += red[w][i];
        out[i] = i < 2 ? x : (i < 2 + 2 * M_NA ? x * vscale : x * tscale);
    }
}

// One event's frontier values and its lineshape products: FP64 rows (plain
// path) or FP32 + FP64 rows (mixed form).
#define CT_NEV_ALLOC (M_NEV > 0 ? M_NEV : 1)
#define CT_NEVF_ALLOC (M_NEVF > 0 ? M_NEVF : 1)
#define CT_NEVD_ALLOC (M_NEVD > 0 ? M_NEVD : 1)
// The FP32 frontier table is event-major: each event's values in one record
// of CT_EVF_STRIDE floats (padded to 16 bytes), read and copied as float4;
// the FP64 tables are row-major [value][ld].
#define CT_NEVF4 (M_NEVF > 0 ? (M_NEVF + 3) / 4 : 1)
#define CT_EVF_STRIDE (4 * CT_NEVF4)
template <typename L>
struct CtEvent;
template <>
struct CtEvent<double> {
    static constexpr int NA = M_NEV, NB = 0;  // values of the table's type per event, FP64 rows
    static constexpr bool EVMAJ = false;      // table layout [value][ld]
    double v[CT_NEV_ALLOC];
    // this event's first value in the table (consecutive values `ld` apart)
    static __device__ __forceinline__ const double* at(const double* table, long long e) { return table + e; }
    __device__ __forceinline__ void load(const double* a, const double*, long long stride)
    {
#pragma unroll
        for (int k = 0; k < M_NEV; ++k) v[k] = a[(long long)k * stride];
    }
    __device__ __forceinline__ void columns(const double* C, const float*, const float*, double* Fr, double* Fi,
                                            double* dFr, double* dFi) const
    {
        model_columns(v, C, Fr, Fi, dFr, dFi);
    }
};
template <>
struct CtEvent<float> {
    static constexpr int NA = CT_EVF_STRIDE, NB = M_NEVD;  // floats per event record, FP64 rows
    static constexpr bool EVMAJ = true;                    // FP32 table event-major
    float f[CT_NEVF_ALLOC];
    double d[CT_NEVD_ALLOC];
    // this event's record in the table
    static __device__ __forceinline__ const float* at(const float* table, long long e)
    {
        return table + e * CT_EVF_STRIDE;
    }
    // a: the event's 16-byte aligned record; b: its first FP64 value
    // (consecutive values `stride` apart)
    __device__ __forceinline__ void load(const float* a, const double* b, long long stride)
    {
        const float4* r = reinterpret_cast<const float4*>(a);
#pragma unroll
        for (int q = 0; q < CT_NEVF4; ++q) {
            const float4 x = r[q];
            if (4 * q + 0 < M_NEVF) f[4 * q + 0] = x.x;
            if (4 * q + 1 < M_NEVF) f[4 * q + 1] = x.y;
            if (4 * q + 2 < M_NEVF) f[4 * q + 2] = x.z;
            if (4 * q + 3 < M_NEVF) f[4 * q + 3] = x.w;
        }
#pragma unroll
        for (int k = 0; k < M_NEVD; ++k) d[k] = b[(long long)k * stride];
    }
    __device__ __forceinline__ void columns(const double* C, const float* Cfh, const float* Cfl, float* Fr, float* Fi,
                                            float* dFr, float* dFi) const
    {
        model_columns_f32(f, d, C, Cfh, Cfl, Fr, Fi, dFr, dFi);
    }
};

// Once per event when a sample is loaded: the frontier tables from the
// kinematic cache [M_NKIN][ld] (mixed tables only when evf is given).
extern "C" __global__ void __launch_bounds__(CT_BLOCK) ct_event_cache(const double* __restrict__ kin, long long n,
                                                                     long long ld, double* __restrict__ ev64,
                                                                     float* __restrict__ evf, double* __restrict__ evd)
{
    for (long long e = (long long)blockIdx.x * CT_BLOCK + threadIdx.x; e < n; e += (long long)gridDim.x * CT_BLOCK) {
        double kv[M_NKIN > 0 ? M_NKIN : 1];
#pragma unroll
        for (int k = 0; k < M_NKIN; ++k) kv[k] = kin[(long long)k * ld + e];
        double o[CT_NEV_ALLOC];
        model_event(kv, o);
#pragma unroll
        for (int k = 0; k < M_NEV; ++k) ev64[(long long)k * ld + e] = o[k];
        if (evf) {
            float of[CT_NEVF_ALLOC];
            double od[CT_NEVD_ALLOC];
            model_event_mx(o, of, od);
            float* r = evf + (long long)e * CT_EVF_STRIDE;
#pragma unroll
            for (int k = 0; k < CT_EVF_STRIDE; ++k) r[k] = k < M_NEVF ? of[k] : 0.0f;
#pragma unroll
            for (int k = 0; k < M_NEVD; ++k) evd[(long long)k * ld + e] = od[k];
        }
    }
}

// R: type of the per-polarisation complex algebra and of the stored angular
//    table (double: plain path; float: mixed form)
// L: type of the lineshapes, their derivatives and the per-thread gradient
//    sums
// PH_ONLY: the launch serves phase-space events only
// MULTI: one launch over several jobs of this model (ct_fused_*_multi): the
// per-call constants are this job's image in global memory (A.kblock)
// instead of the constant bank.
template <typename R, typename L, bool PH_ONLY, int BLOCK, int STAGE, bool ACC_SMEM, bool PAIRED, bool MULTI = false>
__device__ __forceinline__ void ct_fused_body(const CtArgs& A)
{
    typedef typename CtVec2<R>::type SL2;
    const int cta = (int)blockIdx.x + A.cta_base;
    // which sample does this CTA serve?
    int si = 0;
#pragma unroll
    for (int k = 1; k < 3; ++k)
        if (k < A.nsamp && cta >= A.s[k].cta_begin) si = k;
    const CtSample& S = A.s[si];
    const int kind = PH_ONLY ? 0 : S.kind;
    const long long n = S.n;
    const SL2* __restrict__ slamp = (const SL2*)S.slamp;
    // this event's angular values: its record of the event-major FP32 table,
    // or its first value of the [row][ld] FP64 table
    // (event-major: the FP32 table, and the compact FP64 table of paired
    // polarisations; the full FP64 table is [row][ld])
    constexpr int SL_NPL = M_NPLANE * (PAIRED ? CT_NPOL_STORED : M_NPOL);
    constexpr bool SL_EM = sizeof(R) == 4 || PAIRED;
    constexpr int SL_SLS = sizeof(R) == 4 ? CT_SL32_STRIDE(SL_NPL) : SL_NPL;
    auto slat = [&](long long e) -> const SL2* { return SL_EM ? slamp + e * SL_SLS : slamp + e; };
    const L* __restrict__ eva = (const L*)S.ev;
    const double* __restrict__ evb = S.evd;
    const double* __restrict__ wts = S.w;

    // dynamic shared memory: [gradient-sum slots (ACC_SMEM)][tile buffers (STAGE)]
    extern __shared__ __align__(128) unsigned char ct_dyn[];
    constexpr unsigned ACC_BYTES = ACC_SMEM ? ((CT_NACC - 2) * BLOCK * sizeof(L) + 127) / 128 * 128 : 0;
    double accd[2] = {0.0, 0.0};
    CtAccG<L, BLOCK, ACC_SMEM> accg;
    accg.init(ct_dyn);

    // parameter-only constants and couplings from the constant bank: FP64,
    // and FP32 hi + lo pairs for the FP32 form (a single FP32 rounding would
    // bias every event alike)
    const CtConsts* __restrict__ Kg = MULTI ? (const CtConsts*)A.kblock : nullptr;
    const double* sC = MULTI ? Kg->c : ct_k.c;
    const float* sCfh = MULTI ? Kg->ch : ct_k.ch;
    const float* sCfl = MULTI ? Kg->cl : ct_k.cl;
    auto vr = [&](int a) -> L {
        if constexpr (MULTI) return sizeof(L) == 4 ? (L)__ldg(Kg->vh + 2 * a) : (L)__ldg(Kg->v + 2 * a);
        return sizeof(L) == 4 ? (L)ct_k.vh[2 * a] : (L)ct_k.v[2 * a];
    };
    auto vi = [&](int a) -> L {
        if constexpr (MULTI) return sizeof(L) == 4 ? (L)__ldg(Kg->vh + 2 * a + 1) : (L)__ldg(Kg->v + 2 * a + 1);
        return sizeof(L) == 4 ? (L)ct_k.vh[2 * a + 1] : (L)ct_k.v[2 * a + 1];
    };

    // all per-event work: ap / bp / slp point at this event's frontier values
    // (table type, FP64) and angular values, consecutive values `ks` / `ss`
    // elements apart
    auto event = [&](long long e, const L* __restrict__ ap, const double* __restrict__ bp, long long ks,
                     const SL2* __restrict__ slp, long long ss) {
        // ---- lineshapes with parameter derivatives ----
        CtEvent<L> ev;
        ev.load(ap, bp, ks);
        L Fr[M_NTERM], Fi[M_NTERM], dFr[M_NDER > 0 ? M_NDER : 1], dFi[M_NDER > 0 ? M_NDER : 1];
        ev.columns(sC, sCfh, sCfl, Fr, Fi, dFr, dFi);

        // ---- coherent sum over amplitudes ----
        // (paired tables: SL_{c,NPOL-1-p} = conj(SL_{c,p}), only the first
        // CT_NPOL_STORED polarisations are stored and read)
        constexpr int NPS = PAIRED ? CT_NPOL_STORED : M_NPOL;
        SL2 sl[M_NPLANE * NPS];
        if constexpr (sizeof(R) == 4) {
            // event-major FP32 record (16-byte aligned): two values per load
            const float4* q4 = reinterpret_cast<const float4*>(slp);
#pragma unroll
            for (int c = 0; c < M_NPLANE * NPS; c += 2) {
                const float4 x = q4[c / 2];
                sl[c] = make_float2(x.x, x.y);
                if (c + 1 < M_NPLANE * NPS) sl[c + 1] = make_float2(x.z, x.w);
            }
        } else if constexpr (SL_EM) {
            // event-major FP64 record: consecutive 16-byte values
#pragma unroll
            for (int c = 0; c < M_NPLANE * NPS; ++c) sl[c] = slp[c];
        } else {
#pragma unroll
            for (int c = 0; c < M_NPLANE * NPS; ++c) sl[c] = slp[(long long)c * ss];
        }
        // c_t = v_col(t) F_t per term (one per column, more with identical particles)
        R cr[M_NTERM], ci[M_NTERM];
#pragma unroll
        for (int t = 0; t < M_NTERM; ++t) {
            const int a = term_col(t);
            if constexpr (sizeof(L) == 4) {
                // The mixed form evaluates the NLL at the couplings rounded
                // to FP32, v_h; the finalize step adds the first-order term
                // 2 sum_a Re(conj(g_a) (v_a - v_h,a)) (g = dNLL/d conj(v),
                // which this pass sums), so the result is the NLL at v to
                // second order (~|H| |v - v_h|^2, 1e-12). The products of the
                // per-event values with the fixed v_h are rounded without
                // bias (the per-event factor makes the low bits random).
                cr[t] = fmaf(Fr[t], vr(a), -Fi[t] * vi(a));
                ci[t] = fmaf(Fi[t], vr(a), Fr[t] * vi(a));
            } else {
                cr[t] = (R)(vr(a) * Fr[t] - vi(a) * Fi[t]);
                ci[t] = (R)(vr(a) * Fi[t] + vi(a) * Fr[t]);
            }
        }
        R Sr[M_NPOL], Si[M_NPOL];
#pragma unroll
        for (int p = 0; p < NPS; ++p) {
            const int q = M_NPOL - 1 - p;
            if (PAIRED && q != p) {
                // S_p = sum c (x + iy), S_q = sum c (x - iy) from the same four
                // products per term
                R xr = (R)0, yi = (R)0, yr = (R)0, xi = (R)0;
#pragma unroll
                for (int t = 0; t < M_NTERM; ++t) {
                    SL2 x = sl[term_plane(t) * NPS + p];
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
                R sr = (R)0, sim = (R)0;
#pragma unroll
                for (int t = 0; t < M_NTERM; ++t) {
                    SL2 x = sl[term_plane(t) * NPS + p];
                    sr += cr[t] * x.x - ci[t] * x.y;
                    sim += cr[t] * x.y + ci[t] * x.x;
                }
                Sr[p] = sr;
                Si[p] = sim;
            }
        }
        R f = (R)0;
#pragma unroll
        for (int p = 0; p < M_NPOL; ++p) f += Sr[p] * Sr[p] + Si[p] * Si[p];

        // ---- per-event weight of the adjoint ----
        // (the sample's common factors of the gradient terms, w / W or -1 for
        // the v-gradient and 2 or -2 for the theta-gradient, are applied to
        // the CTA sums; a weighted phase-space event scales its v-gradient
        // terms by its weight here)
        R ur[M_NPOL], ui[M_NPOL];
        L gw = (L)1;
        if (kind == 0) {
            const double we = wts ? __ldg(wts + e) : 1.0;
            accd[1] += (double)f;
#pragma unroll
            for (int p = 0; p < M_NPOL; ++p) {
                ur[p] = Sr[p];
                ui[p] = Si[p];
            }
            gw = (L)we;
        } else {
            const double we = wts ? __ldg(wts + e) : 1.0;
            if (f == (R)0) {
                accd[0] += -log(1e-10) * we;
                return;
            }
            accd[0] += -log((double)f) * we;
            const R inv = (R)(we / (double)f);
            const R kmax = (R)1e10;
#pragma unroll
            for (int p = 0; p < M_NPOL; ++p) {
                ur[p] = fmin(fmax(Sr[p] * inv, -kmax), kmax);
                ui[p] = fmin(fmax(Si[p] * inv, -kmax), kmax);
            }
        }
        // T_c = sum_p conj(SL_{c,p}) u_p
        // (paired: conj(SL_p) u_p + SL_p u_q = x (u_p + u_q) + i y (u_q - u_p))
        R ar[NPS], br[NPS], ai[NPS], bi[NPS];
#pragma unroll
        for (int p = 0; p < NPS; ++p) {
            const int q = M_NPOL - 1 - p;
            if (PAIRED && q != p) {
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
        R Tr[M_NPLANE], Ti[M_NPLANE];
#pragma unroll
        for (int c = 0; c < M_NPLANE; ++c) {
            R tr = (R)0, ti = (R)0;
#pragma unroll
            for (int p = 0; p < NPS; ++p) {
                SL2 x = sl[c * NPS + p];
                tr += x.x * ar[p] + x.y * br[p];
                ti += x.x * ai[p] + x.y * bi[p];
            }
            Tr[c] = tr;
            Ti[c] = ti;
        }
        // v-gradient: sum over the column's terms of conj(F_t) T_plane(t)
        if (kind == 0 && wts) {
#pragma unroll
            for (int t = 0; t < M_NTERM; ++t) {
                const int a = term_col(t), c = term_plane(t);
                const L fr = Fr[t], fi = Fi[t];
                const L tr = (L)Tr[c], ti = (L)Ti[c];
                accg.add(2 * a, gw * (fr * tr + fi * ti));
                accg.add(2 * a + 1, gw * (fr * ti - fi * tr));
            }
        } else {
#pragma unroll
            for (int t = 0; t < M_NTERM; ++t) {
                const int a = term_col(t), c = term_plane(t);
                const L fr = Fr[t], fi = Fi[t];
                const L tr = (L)Tr[c], ti = (L)Ti[c];
                accg.add(2 * a, fr * tr + fi * ti);
                accg.add(2 * a + 1, fr * ti - fi * tr);
            }
        }
        // theta-gradient: Re(v dF_t conj(T)) = Re(dF_t W_t), W_t = v_col(t) conj(T_plane(t))
        L Wr[M_NTERM], Wi[M_NTERM];
#pragma unroll
        for (int t = 0; t < M_NTERM; ++t) {
            const int a = term_col(t), c = term_plane(t);
            const L tr = (L)Tr[c], ti = (L)Ti[c];
            Wr[t] = vr(a) * tr + vi(a) * ti;
            Wi[t] = vi(a) * tr - vr(a) * ti;
        }
#pragma unroll
        for (int k = 0; k < M_NDER; ++k) {
            const int t = der_term(k);
            accg.add(2 * M_NA + der_th(k), dFr[k] * Wr[t] - dFi[k] * Wi[t]);
        }
    };

    if constexpr (STAGE == 3) {
        // Per-thread two-buffer pipeline of the frontier values: each thread
        // copies its next event's frontier values into its own shared-memory
        // slots by cp.async while it computes the current event, and waits
        // only for its own copies; the angular values are loaded directly
        // (they are first needed after the lineshapes).
        constexpr int NA = CtEvent<L>::NA, NB = CtEvent<L>::NB;
        constexpr unsigned ABYTES = (2u * (NA > 0 ? NA : 1) * BLOCK * sizeof(L) + 15) / 16 * 16;
        L* abuf = (L*)(ct_dyn + ACC_BYTES);                  // [2][NA][BLOCK]
        double* bbuf = (double*)(ct_dyn + ACC_BYTES + ABYTES);  // [2][NB][BLOCK]
        const int tid = threadIdx.x;
        auto fetch = [&](long long e, int b) {
            if constexpr (CtEvent<L>::EVMAJ) {
                // the event's record: [2][BLOCK][NA] floats, 16-byte copies
                float4* dst = reinterpret_cast<float4*>(abuf + ((size_t)b * BLOCK + tid) * NA);
                const float4* src = reinterpret_cast<const float4*>(eva + e * NA);
#pragma unroll
                for (int q = 0; q < NA / 4; ++q) ct_cp_async<16>(dst + q, src + q);
            } else {
#pragma unroll
                for (int k = 0; k < NA; ++k)
                    ct_cp_async<sizeof(L)>(abuf + ((size_t)b * NA + k) * BLOCK + tid, eva + (long long)k * S.ld + e);
            }
#pragma unroll
            for (int k = 0; k < NB; ++k)
                ct_cp_async<8>(bbuf + ((size_t)b * NB + k) * BLOCK + tid, evb + (long long)k * S.ld + e);
            ct_cp_async_commit();
        };
        const long long stride = (long long)S.cta_count * BLOCK;
        long long e = (long long)(cta - S.cta_begin) * BLOCK + tid;
        if (e < n) fetch(e, 0);
        for (int it = 0; e < n; e += stride, ++it) {
            const int b = it & 1;
            if (e + stride < n) fetch(e + stride, b ^ 1);
            else ct_cp_async_commit();  // empty group: the wait below covers buffer b alike
            ct_cp_async_wait<1>();
            const L* ap = CtEvent<L>::EVMAJ ? abuf + ((size_t)b * BLOCK + tid) * NA : abuf + (size_t)b * NA * BLOCK + tid;
            event(e, ap, bbuf + (size_t)b * NB * BLOCK + tid, BLOCK, slat(e), S.ld);
        }
        ct_cp_async_wait<0>();
    } else if constexpr (STAGE > 0) {
        // Warp-level two-buffer pipeline. Each warp streams its own 32-event
        // tiles (the same events as the direct loop below); lane 0 copies the
        // next tile's table rows (the frontier values; with STAGE 2 also the
        // angular values) into the warp's other shared-memory buffer by bulk
        // copies that complete on the warp's mbarrier, while the warp computes
        // the current tile. No CTA-wide barrier: warps proceed independently.
        // Rows are padded to multiples of 256 events, so every copy starts on
        // a 128-byte boundary and moves a whole 32-event tile.
        constexpr int NPL = M_NPLANE * (PAIRED ? CT_NPOL_STORED : M_NPOL);  // table rows
        constexpr int W = BLOCK / 32;
        constexpr int NA = CtEvent<L>::NA, NB = CtEvent<L>::NB;
        constexpr unsigned AR = 32 * sizeof(L), BR = 32 * sizeof(double), SR = 32 * sizeof(SL2);
        // angular part of a tile: NPL rows of 32 values (FP64), or 32 records of SL_SLS values (FP32)
        constexpr unsigned SLB = (SL_EM ? SL_SLS : NPL) * SR;
        constexpr unsigned BUF = NA * AR + NB * BR + (STAGE > 1 ? SLB : 0);
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        unsigned char* wbuf = ct_dyn + ACC_BYTES + (size_t)warp * 2 * BUF;
        __shared__ __align__(8) unsigned long long ct_wbar[W][2];
        const long long ntiles = (n + 31) / 32;
        const long long first = (long long)(cta - S.cta_begin) * W + warp, tstep = (long long)S.cta_count * W;
        const long long my = first < ntiles ? (ntiles - 1 - first) / tstep + 1 : 0;
        auto issue = [&](long long k, int b) {
            const long long e0 = (first + k * tstep) * 32;
            unsigned char* buf = wbuf + (size_t)b * BUF;
            unsigned long long* bar = &ct_wbar[warp][b];
            ct_mbar_expect_tx(bar, BUF);
            if constexpr (CtEvent<L>::EVMAJ) {
                // the tile's 32 records in one copy
                ct_bulk_g2s(buf, eva + e0 * NA, NA * AR, bar);
            } else {
#pragma unroll 1
                for (int r = 0; r < NA; ++r) ct_bulk_g2s(buf + (size_t)r * AR, eva + (long long)r * S.ld + e0, AR, bar);
            }
#pragma unroll 1
            for (int r = 0; r < NB; ++r)
                ct_bulk_g2s(buf + (size_t)NA * AR + (size_t)r * BR, evb + (long long)r * S.ld + e0, BR, bar);
            if constexpr (STAGE > 1) {
                if constexpr (SL_EM) {
                    // the tile's 32 records in one copy
                    ct_bulk_g2s(buf + (size_t)NA * AR + (size_t)NB * BR, slamp + e0 * SL_SLS, SLB, bar);
                } else {
#pragma unroll 1
                    for (int c = 0; c < NPL; ++c)
                        ct_bulk_g2s(buf + (size_t)NA * AR + (size_t)NB * BR + (size_t)c * SR,
                                    slamp + (long long)c * S.ld + e0, SR, bar);
                }
            }
        };
        if (lane == 0) {
            ct_mbar_init(&ct_wbar[warp][0], 1);
            ct_mbar_init(&ct_wbar[warp][1], 1);
            ct_fence_mbar_init();
        }
        __syncwarp();
        if (lane == 0) {
            if (my > 0) issue(0, 0);
            if (my > 1) issue(1, 1);
        }
        long long k = 0;
        for (; k < my; ++k) {
            const int b = (int)(k & 1);
            const bool ok = ct_mbar_wait(&ct_wbar[warp][b], (unsigned)((k >> 1) & 1), CT_WAIT_LIMIT);
            if (!__all_sync(0xffffffffu, ok)) break;
            const long long e = (first + k * tstep) * 32 + lane;
            if (e < n) {
                const unsigned char* buf = wbuf + (size_t)b * BUF;
                const L* ap = (const L*)buf + (CtEvent<L>::EVMAJ ? lane * NA : lane);
                const double* bp = (const double*)(buf + (size_t)NA * AR) + lane;
                if constexpr (STAGE > 1)
                    event(e, ap, bp, 32,
                          (const SL2*)(buf + (size_t)NA * AR + (size_t)NB * BR) + (SL_EM ? lane * SL_SLS : lane), 32);
                else
                    event(e, ap, bp, 32, slat(e), S.ld);
            }
            // every lane is done with buffer b before it is refilled
            __syncwarp();
            if (lane == 0 && k + 2 < my) issue(k + 2, b);
        }
        if (k < my) {
            // a copy did not complete in time: flag the evaluation and give
            // the copies still in flight a bounded chance to land before the
            // warp leaves
            if (lane == 0) {
                atomicExch(A.err, 1);
                ct_mbar_wait(&ct_wbar[warp][k & 1], (unsigned)((k >> 1) & 1), CT_WAIT_LIMIT);
                if (k + 1 < my) ct_mbar_wait(&ct_wbar[warp][(k + 1) & 1], (unsigned)(((k + 1) >> 1) & 1), CT_WAIT_LIMIT);
            }
            __syncwarp();
        }
    } else {
        const long long stride = (long long)S.cta_count * BLOCK;
        for (long long e = (long long)(cta - S.cta_begin) * BLOCK + threadIdx.x; e < n; e += stride)
            event(e, CtEvent<L>::at(eva, e), evb ? evb + e : nullptr, S.ld, slat(e), S.ld);
    }
    ct_block_reduce_store<BLOCK>(accd, accg, A.partials + (long long)cta * CT_NACC, kind == 0 ? S.vw_scale : -1.0,
                                 kind == 0 ? 2.0 : -2.0);
}

// block size and minimum resident CTAs per SM of the two fused kernels (the
// host launches with the same block sizes)
#ifndef CT_F64_BLOCK
#define CT_F64_BLOCK 192
#endif
#ifndef CT_F64_MINB
#define CT_F64_MINB 2
#endif
#ifndef CT_MX_BLOCK
#define CT_MX_BLOCK 256
#endif
#ifndef CT_MX_MINB
#define CT_MX_MINB 2
#endif
extern "C" __global__ void __launch_bounds__(CT_F64_BLOCK, CT_F64_MINB) ct_fused_f64(CtArgs a)
{
    ct_fused_body<double, double, false, CT_F64_BLOCK, CT_F64_STAGE, CT_F64_ACC != 0, false>(a);
}
extern "C" __global__ void __launch_bounds__(CT_F64_BLOCK, CT_F64_MINB) ct_fused_f64_pc(CtArgs a)
{
    ct_fused_body<double, double, false, CT_F64_BLOCK, CT_F64_STAGE, CT_F64_ACC != 0, true>(a);
}
// mixed form (FP32 lineshapes and algebra, FP64 logs and sums), all samples
extern "C" __global__ void __launch_bounds__(CT_MX_BLOCK, CT_MX_MINB) ct_fused_mixed(CtArgs a)
{
    ct_fused_body<float, float, false, CT_MX_BLOCK, CT_MX_STAGE, CT_MX_ACC != 0, false>(a);
}
extern "C" __global__ void __launch_bounds__(CT_MX_BLOCK, CT_MX_MINB) ct_fused_mixed_pc(CtArgs a)
{
    ct_fused_body<float, float, false, CT_MX_BLOCK, CT_MX_STAGE, CT_MX_ACC != 0, true>(a);
}

// Several jobs of this model in one launch: the CTAs [cta_off[j],
// cta_off[j+1]) serve job j, whose CtArgs (cta_base = -cta_off[j], kblock =
// its constants image) hold its samples and partial rows; each job's
// partial rows are exactly those of its own launch.
__device__ __forceinline__ int ct_multi_job(const int* __restrict__ cta_off, int njobs)
{
    int j = 0;
    while (j + 1 < njobs && (int)blockIdx.x >= __ldg(cta_off + j + 1)) ++j;
    return j;
}
extern "C" __global__ void __launch_bounds__(CT_F64_BLOCK, CT_F64_MINB)
    ct_fused_f64_multi(const CtArgs* __restrict__ jobs, const int* __restrict__ cta_off, int njobs)
{
    ct_fused_body<double, double, false, CT_F64_BLOCK, CT_F64_STAGE, CT_F64_ACC != 0, false, true>(
        jobs[ct_multi_job(cta_off, njobs)]);
}
extern "C" __global__ void __launch_bounds__(CT_F64_BLOCK, CT_F64_MINB)
    ct_fused_f64_pc_multi(const CtArgs* __restrict__ jobs, const int* __restrict__ cta_off, int njobs)
{
    ct_fused_body<double, double, false, CT_F64_BLOCK, CT_F64_STAGE, CT_F64_ACC != 0, true, true>(
        jobs[ct_multi_job(cta_off, njobs)]);
}
extern "C" __global__ void __launch_bounds__(CT_MX_BLOCK, CT_MX_MINB)
    ct_fused_mixed_multi(const CtArgs* __restrict__ jobs, const int* __restrict__ cta_off, int njobs)
{
    ct_fused_body<float, float, false, CT_MX_BLOCK, CT_MX_STAGE, CT_MX_ACC != 0, false, true>(
        jobs[ct_multi_job(cta_off, njobs)]);
}
extern "C" __global__ void __launch_bounds__(CT_MX_BLOCK, CT_MX_MINB)
    ct_fused_mixed_pc_multi(const CtArgs* __restrict__ jobs, const int* __restrict__ cta_off, int njobs)
{
    ct_fused_body<float, float, false, CT_MX_BLOCK, CT_MX_STAGE, CT_MX_ACC != 0, true, true>(
        jobs[ct_multi_job(cta_off, njobs)]);
}

// Partial-wave integrals of sample s[0] (FP64): per resonance block i,
// sum_e w_e sum_p |sum_{a in block i} v_a A_{a,p}|^2 (the reference's partial
// integrals of its fit fractions, src/ComputeBF.cu:9-60); one row of M_NBLK
// sums per CTA.
extern "C" __global__ void __launch_bounds__(CT_BLOCK) ct_partials_f64(CtArgs A, double* __restrict__ rows)
{
    const CtSample& S = A.s[0];
    const long long n = S.n;
    const double2* __restrict__ slamp = (const double2*)S.slamp;
    __shared__ double sC[CT_NCONST_ALLOC];
    ct_stage_consts(A, sC);
    double acc[M_NBLK];
#pragma unroll
    for (int i = 0; i < M_NBLK; ++i) acc[i] = 0.0;
    for (long long e = (long long)blockIdx.x * CT_BLOCK + threadIdx.x; e < n; e += (long long)gridDim.x * CT_BLOCK) {
        double ev[CT_NEV_ALLOC];
#pragma unroll
        for (int k = 0; k < M_NEV; ++k) ev[k] = __ldg((const double*)S.ev + (long long)k * S.ld + e);
        double Fr[M_NTERM], Fi[M_NTERM], dFr[M_NDER > 0 ? M_NDER : 1], dFi[M_NDER > 0 ? M_NDER : 1];
        model_columns(ev, sC, Fr, Fi, dFr, dFi);
        const double we = S.w ? __ldg(S.w + e) : 1.0;
#pragma unroll
        for (int i = 0; i < M_NBLK; ++i) {
            double blk = 0.0;
#pragma unroll
            for (int p = 0; p < M_NPOL; ++p) {
                double sr = 0.0, si = 0.0;
                for (int t = blk_term0(i); t < blk_term0(i) + blk_nterm(i); ++t) {
                    const int a = term_col(t);
                    const double vr = __ldg(A.v + 2 * a), vi = __ldg(A.v + 2 * a + 1);
                    const double cr = vr * Fr[t] - vi * Fi[t], ci = vr * Fi[t] + vi * Fr[t];
                    const double2 x = slamp[(long long)(term_plane(t) * M_NPOL + p) * S.ld + e];
                    sr += cr * x.x - ci * x.y;
                    si += cr * x.y + ci * x.x;
                }
                blk += sr * sr + si * si;
            }
            acc[i] += we * blk;
        }
    }
    __shared__ double red[CT_BLOCK / 32][M_NBLK];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < M_NBLK; ++i) {
        double x = acc[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp][i] = x;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < M_NBLK; i += CT_BLOCK) {
        double x = 0.0;
#pragma unroll
        for (int w = 0; w < CT_BLOCK / 32; ++w) x += red[w][i];
        rows[(long long)blockIdx.x * M_NBLK + i] = x;
    }
}

// Result export over sample s[0] (FP64): per event, the block amplitudes
// P_i,p = sum_{t in block i} v_col(t) F_t SL_plane(t),p give
//   total[e]      = sum_p |sum_{i in mask} P_i,p|^2 (all blocks when mask is null)
//   partial[i][e] = sum_p |P_i,p|^2
//   interf_ev[k][e] (optional) = sum_p 2 Re(P_i,p conj(P_j,p)) for the k-th pair i < j
// and each CTA adds sum_e sum_p 2 Re(P_i,p conj(P_j,p)) (i <= j) into its row
// of interf_rows (reference computeResults, src/ComputeResults.cu).
extern "C" __global__ void __launch_bounds__(CT_BLOCK) ct_export_f64(CtArgs A, double* __restrict__ total,
                                                                    double* __restrict__ partial,
                                                                    double* __restrict__ interf_ev,
                                                                    double* __restrict__ interf_rows,
                                                                    const int* __restrict__ mask)
{
    constexpr int NPAIR = M_NBLK * (M_NBLK + 1) / 2;
    const CtSample& S = A.s[0];
    const long long n = S.n;
    const double2* __restrict__ slamp = (const double2*)S.slamp;
    __shared__ double sC[CT_NCONST_ALLOC];
    __shared__ double sI[NPAIR];
    for (int i = threadIdx.x; i < NPAIR; i += CT_BLOCK) sI[i] = 0.0;
    ct_stage_consts(A, sC);
    for (long long e = (long long)blockIdx.x * CT_BLOCK + threadIdx.x; e < n; e += (long long)gridDim.x * CT_BLOCK) {
        double ev[CT_NEV_ALLOC];
#pragma unroll
        for (int k = 0; k < M_NEV; ++k) ev[k] = __ldg((const double*)S.ev + (long long)k * S.ld + e);
        double Fr[M_NTERM], Fi[M_NTERM], dFr[M_NDER > 0 ? M_NDER : 1], dFi[M_NDER > 0 ? M_NDER : 1];
        model_columns(ev, sC, Fr, Fi, dFr, dFi);
        double Pr[M_NBLK][M_NPOL], Pi[M_NBLK][M_NPOL];
#pragma unroll
        for (int i = 0; i < M_NBLK; ++i)
#pragma unroll
            for (int p = 0; p < M_NPOL; ++p) {
                double sr = 0.0, si = 0.0;
                for (int t = blk_term0(i); t < blk_term0(i) + blk_nterm(i); ++t) {
                    const int a = term_col(t);
                    const double vr = __ldg(A.v + 2 * a), vi = __ldg(A.v + 2 * a + 1);
                    const double cr = vr * Fr[t] - vi * Fi[t], ci = vr * Fi[t] + vi * Fr[t];
                    const double2 x = slamp[(long long)(term_plane(t) * M_NPOL + p) * S.ld + e];
                    sr += cr * x.x - ci * x.y;
                    si += cr * x.y + ci * x.x;
                }
                Pr[i][p] = sr;
                Pi[i][p] = si;
            }
        double tot = 0.0;
#pragma unroll
        for (int p = 0; p < M_NPOL; ++p) {
            double sr = 0.0, si = 0.0;
#pragma unroll
            for (int i = 0; i < M_NBLK; ++i)
                if (!mask || mask[i]) {
                    sr += Pr[i][p];
                    si += Pi[i][p];
                }
            tot += sr * sr + si * si;
        }
        total[e] = tot;
        int k = 0, kk = 0;
#pragma unroll
        for (int i = 0; i < M_NBLK; ++i) {
            double pi = 0.0;
#pragma unroll
            for (int p = 0; p < M_NPOL; ++p) pi += Pr[i][p] * Pr[i][p] + Pi[i][p] * Pi[i][p];
            partial[(long long)i * S.ld + e] = pi;
#pragma unroll
            for (int j = i; j < M_NBLK; ++j) {
                double x = 0.0;
#pragma unroll
                for (int p = 0; p < M_NPOL; ++p) x += 2.0 * (Pr[i][p] * Pr[j][p] + Pi[i][p] * Pi[j][p]);
                atomicAdd(&sI[k], x);
                if (j > i) {
                    if (interf_ev) interf_ev[(long long)kk * S.ld + e] = x;
                    ++kk;
                }
                ++k;
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < NPAIR; i += CT_BLOCK) interf_rows[(long long)blockIdx.x * NPAIR + i] = sI[i];
}

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
        double ev[CT_NEV_ALLOC];
#pragma unroll
        for (int k = 0; k < M_NEV; ++k) ev[k] = __ldg((const double*)S.ev + (long long)k * S.ld + e);
        double Fr[M_NTERM], Fi[M_NTERM], dFr[M_NDER > 0 ? M_NDER : 1], dFi[M_NDER > 0 ? M_NDER : 1];
        model_columns(ev, sC, Fr, Fi, dFr, dFi);
        double f = 0.0;
#pragma unroll
        for (int p = 0; p < M_NPOL; ++p) {
            double sr = 0.0, si = 0.0;
#pragma unroll
            for (int t = 0; t < M_NTERM; ++t) {
                const int a = term_col(t);
                double cr = __ldg(A.v + 2 * a) * Fr[t] - __ldg(A.v + 2 * a + 1) * Fi[t];
                double ci = __ldg(A.v + 2 * a) * Fi[t] + __ldg(A.v + 2 * a + 1) * Fr[t];
                double2 x = slamp[(long long)(term_plane(t) * M_NPOL + p) * S.ld + e];
                sr += cr * x.x - ci * x.y;
                si += cr * x.y + ci * x.x;
            }
            f += sr * sr + si * si;
        }
        out[e] = f;
    }
}
