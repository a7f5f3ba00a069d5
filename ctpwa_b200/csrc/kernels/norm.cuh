// Normalisation cache: the phase-space part of the likelihood as quadratic
// forms in the couplings, at one set of resonance parameters (FP64).
//
// With c_t = v_col(t) the coupling of term t, X_{t,p} = F_t SL_{plane(t),p}
// its amplitude in polarisation p and the per-event plane products
//   G_{c,d} = sum_p SL_{c,p} conj(SL_{d,p})          (Hermitian in c, d),
// ct_norm_build sums over the phase-space sample
//   Mu[t][s] = sum_e F_t conj(F_s) G_{plane(t),plane(s)}                (t <= s)
//   D[k][s]  = sum_e dF_k conj(F_s) G_{plane(der_term(k)),plane(s)}     (all s)
//   Mw[t][s] = sum_e w_e F_t conj(F_s) G_{plane(t),plane(s)}            (t <= s, weighted samples)
// and ct_norm_row turns them, for any couplings, into the phase-space row of
// partial sums the fused pass would produce (kernels/fused_nll.cuh):
//   sum_e f_e                        = sum_{t,s} c_t conj(c_s) Mu[t][s]
//   sum_e w_e conj(F_t) T_plane(t)   = sum_s c_s conj(Mw[t][s])
//   sum_e Re(dF_k c_t conj(T_plane(t))) = Re(c_t sum_s conj(c_s) D[k][s]),  t = der_term(k)
// (T_c = sum_p conj(SL_{c,p}) S_p, S_p = sum_t c_t X_{t,p}). Mu is the
// reference's phase-space matrix A^H A of its coupling-only evaluations
// (src/Analysis.cu:748-829 with the quadratic form of
// src/ComputeNLL.cu:575-597); D adds the lineshape derivatives, so the
// normalisation and its whole gradient at unchanged resonance parameters
// need the matrices only, not the phase-space sample.
//
// ct_norm_build: a CTA takes tiles of CT_NORM_TILE events. Phase 1: thread i
// evaluates event i's lineshapes and derivatives (model_columns, FP64) and
// plane products and writes them as one record to shared memory. Phase 2:
// thread j owns entries j, j + CT_NORM_BLOCK, ... of the output and adds the
// tile's events to them (three record reads and eight FP64 operations per
// entry and event; the warp's lanes read one record at a time). Per-CTA
// partial sums, reduced in a fixed order by ct_norm_reduce.
#pragma once

#include "fused_nll.cuh"

#define CT_NORM_BLOCK 128
#define CT_NORM_TILE 128  // events per tile (one per thread in phase 1)
#define CT_NORM_NG (M_NPLANE * (M_NPLANE + 1) / 2)
#define CT_NORM_NU (M_NTERM * (M_NTERM + 1) / 2)
// entries: Mu, D, then Mw (weighted samples)
#define CT_NORM_NE_MAX (2 * CT_NORM_NU + M_NDER * M_NTERM)
#define CT_NORM_MAXJ ((CT_NORM_NE_MAX + CT_NORM_BLOCK - 1) / CT_NORM_BLOCK)
// record per event, in double2 slots: F_t, dF_k, G pairs, (w, 0); odd length
// so the phase-1 stores of consecutive threads fall in different banks
#define CT_NORM_REC0 (M_NTERM + M_NDER + CT_NORM_NG + 1)
#define CT_NORM_REC (CT_NORM_REC0 | 1)

struct CtNormArgs {
    const double2* slamp;  // FP64 angular table [M_NPLANE * M_NPOL][ld]
    const double* ev;      // FP64 frontier rows [M_NEV][ld]
    const double* w;       // per-event weights or nullptr
    long long n, ld;
    const double* consts;  // [M_NCONST] parameter-only subexpressions at the cached theta
    double* partials;      // [grid][ne][2]
    int ne;                // entries: CT_NORM_NU + M_NDER M_NTERM (+ CT_NORM_NU when weighted)
    int pad;
};

__device__ __forceinline__ int ct_norm_gpair(int c, int d)  // c <= d
{
    return c * M_NPLANE - c * (c - 1) / 2 + (d - c);
}

// upper-triangle index q -> (t, s), t <= s
__device__ __forceinline__ void ct_norm_tri(int q, int& t, int& s)
{
    t = 0;
    while (q >= M_NTERM - t) {
        q -= M_NTERM - t;
        ++t;
    }
    s = t + q;
}

extern "C" __global__ void __launch_bounds__(CT_NORM_BLOCK) ct_norm_build(CtNormArgs A)
{
    extern __shared__ double2 nrec[];  // [CT_NORM_TILE][CT_NORM_REC]
    __shared__ double sC[CT_NCONST_ALLOC];
    for (int i = threadIdx.x; i < M_NCONST; i += CT_NORM_BLOCK) sC[i] = A.consts[i];

    // this thread's entries: record slots of the two factors and the plane
    // pair, conjugation of the pair, weighting
    short sa[CT_NORM_MAXJ], sb[CT_NORM_MAXJ], sg[CT_NORM_MAXJ];
    bool cj[CT_NORM_MAXJ], wt[CT_NORM_MAXJ];
    double accr[CT_NORM_MAXJ], acci[CT_NORM_MAXJ];
#pragma unroll
    for (int j = 0; j < CT_NORM_MAXJ; ++j) {
        accr[j] = 0.0;
        acci[j] = 0.0;
        int q = threadIdx.x + j * CT_NORM_BLOCK, ra = 0, s = 0, pa = 0;
        bool w = false;
        if (q >= A.ne) q = 0;  // idle slot: computed, never stored
        if (q < CT_NORM_NU) {
            ct_norm_tri(q, ra, s);
            pa = term_plane(ra);
        } else if (q < CT_NORM_NU + M_NDER * M_NTERM) {
            const int k = (q - CT_NORM_NU) / M_NTERM;
            s = (q - CT_NORM_NU) % M_NTERM;
            ra = M_NTERM + k;
            pa = term_plane(der_term(k));
        } else {
            ct_norm_tri(q - CT_NORM_NU - M_NDER * M_NTERM, ra, s);
            pa = term_plane(ra);
            w = true;
        }
        const int pb = term_plane(s);
        sa[j] = (short)ra;
        sb[j] = (short)s;
        sg[j] = (short)(M_NTERM + M_NDER + (pa <= pb ? ct_norm_gpair(pa, pb) : ct_norm_gpair(pb, pa)));
        cj[j] = pa > pb;
        wt[j] = w;
    }
    __syncthreads();

    const long long ntiles = (A.n + CT_NORM_TILE - 1) / CT_NORM_TILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        // ---- phase 1: this thread's event ----
        {
            const long long e = tile * CT_NORM_TILE + threadIdx.x;
            double2* r = nrec + (size_t)threadIdx.x * CT_NORM_REC;
            if (e < A.n) {
                double ev[CT_NEV_ALLOC];
#pragma unroll
                for (int k = 0; k < M_NEV; ++k) ev[k] = __ldg(A.ev + (long long)k * A.ld + e);
                double Fr[M_NTERM], Fi[M_NTERM], dFr[M_NDER > 0 ? M_NDER : 1], dFi[M_NDER > 0 ? M_NDER : 1];
                model_columns(ev, sC, Fr, Fi, dFr, dFi);
#pragma unroll
                for (int t = 0; t < M_NTERM; ++t) r[t] = make_double2(Fr[t], Fi[t]);
#pragma unroll
                for (int k = 0; k < M_NDER; ++k) r[M_NTERM + k] = make_double2(dFr[k], dFi[k]);
                double2 sl[M_NPLANE * M_NPOL];
#pragma unroll
                for (int c = 0; c < M_NPLANE * M_NPOL; ++c) sl[c] = A.slamp[(long long)c * A.ld + e];
#pragma unroll
                for (int c = 0; c < M_NPLANE; ++c)
#pragma unroll
                    for (int d = c; d < M_NPLANE; ++d) {
                        double gr = 0.0, gi = 0.0;
#pragma unroll
                        for (int p = 0; p < M_NPOL; ++p) {
                            const double2 x = sl[c * M_NPOL + p], y = sl[d * M_NPOL + p];
                            gr += x.x * y.x + x.y * y.y;
                            gi += x.y * y.x - x.x * y.y;
                        }
                        r[M_NTERM + M_NDER + ct_norm_gpair(c, d)] = make_double2(gr, gi);
                    }
                r[M_NTERM + M_NDER + CT_NORM_NG] = make_double2(A.w ? __ldg(A.w + e) : 1.0, 0.0);
            } else {
                // past the sample's end: zero factors contribute nothing
#pragma unroll
                for (int t = 0; t < M_NTERM; ++t) r[t] = make_double2(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < M_NDER; ++k) r[M_NTERM + k] = make_double2(0.0, 0.0);
                r[M_NTERM + M_NDER + CT_NORM_NG] = make_double2(0.0, 0.0);
#pragma unroll
                for (int g = 0; g < CT_NORM_NG; ++g) r[M_NTERM + M_NDER + g] = make_double2(0.0, 0.0);
            }
        }
        __syncthreads();
        // ---- phase 2: the tile's events into this thread's entries ----
#pragma unroll 2
        for (int i = 0; i < CT_NORM_TILE; ++i) {
            const double2* r = nrec + (size_t)i * CT_NORM_REC;
            const double we = r[M_NTERM + M_NDER + CT_NORM_NG].x;
#pragma unroll
            for (int j = 0; j < CT_NORM_MAXJ; ++j) {
                const double2 a = r[sa[j]], b = r[sb[j]], g = r[sg[j]];
                // x = a conj(b); accumulate x g (x conj(g) for a transposed plane pair)
                double xr = a.x * b.x + a.y * b.y, xi = a.y * b.x - a.x * b.y;
                if (wt[j]) {
                    xr *= we;
                    xi *= we;
                }
                const double gi = cj[j] ? -g.y : g.y;
                accr[j] = fma(xr, g.x, fma(-xi, gi, accr[j]));
                acci[j] = fma(xr, gi, fma(xi, g.x, acci[j]));
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < CT_NORM_MAXJ; ++j) {
        const int q = threadIdx.x + j * CT_NORM_BLOCK;
        if (q < A.ne) {
            A.partials[((long long)blockIdx.x * A.ne + q) * 2] = accr[j];
            A.partials[((long long)blockIdx.x * A.ne + q) * 2 + 1] = acci[j];
        }
    }
}

// Fixed-order column sums of the per-CTA partials: out[2 ne].
extern "C" __global__ void __launch_bounds__(256) ct_norm_reduce(const double* __restrict__ partials, int rows, int ne,
                                                                 double* __restrict__ out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int i = warp; i < 2 * ne; i += nwarp) {
        double s = 0.0;
        for (int b = lane; b < rows; b += 32) s += partials[(long long)b * 2 * ne + i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) out[i] = s;
    }
}

struct CtNormRowArgs {
    const double* mat;           // [ne][2]: Mu, D, Mw (ct_norm_reduce)
    int weighted;                // Mw present
    int use_vh;                  // mixed form: the couplings rounded to FP32, as its fused pass uses them
    const double* v;             // couplings (re, im) x M_NA
    double vw_scale;             // 1 / sum of the phase-space weights
    const double* theta;         // this evaluation's resonance parameters
    const double* theta_cached;  // those of the matrices
    int* err;                    // set when they differ (the evaluation is then invalid)
    int pad;
    double* row;                 // [CT_NACC] phase-space row of partial sums
};

// The phase-space row of partial sums from the cached matrices (one CTA of
// CT_NORM_ROW_THREADS: the matrices staged in shared memory, one thread per
// term and per derivative entry, then fixed-order sums by thread 0).
#define CT_NORM_ROW_THREADS 256
extern "C" __global__ void __launch_bounds__(CT_NORM_ROW_THREADS) ct_norm_row(CtNormRowArgs A)
{
    constexpr int NE = CT_NORM_NE_MAX;
    __shared__ double sm[2 * NE];
    __shared__ double cr[M_NTERM], ci[M_NTERM];
    __shared__ double tr[M_NTERM], ti[M_NTERM], tf[M_NTERM];  // per term: r_t, Re(c_t u_t)
    __shared__ double dk[M_NDER > 0 ? M_NDER : 1];            // per derivative entry
    const int ne = CT_NORM_NU + M_NDER * M_NTERM + (A.weighted ? CT_NORM_NU : 0);
    for (int i = threadIdx.x; i < 2 * ne; i += blockDim.x) sm[i] = A.mat[i];
    for (int t = threadIdx.x; t < M_NTERM; t += blockDim.x) {
        const int a = term_col(t);
        double re = A.v[2 * a], im = A.v[2 * a + 1];
        if (A.use_vh) {
            re = (double)(float)re;
            im = (double)(float)im;
        }
        cr[t] = re;
        ci[t] = im;
    }
    for (int j = threadIdx.x; j < M_NTH; j += blockDim.x)
        if (__double_as_longlong(A.theta[j]) != __double_as_longlong(A.theta_cached[j])) atomicExch(A.err, 1);
    __syncthreads();
    const double* Mu = sm;
    const double* D = sm + 2 * CT_NORM_NU;
    const double* Mw = A.weighted ? sm + 2 * (CT_NORM_NU + M_NDER * M_NTERM) : Mu;
    // entry (t, s) of a Hermitian matrix stored as its upper triangle
    auto herm = [&](const double* M, int t, int s, double& re, double& im) {
        const int a = t <= s ? t : s, b = t <= s ? s : t;
        const int q = a * M_NTERM - a * (a - 1) / 2 + (b - a);
        re = M[2 * q];
        im = t <= s ? M[2 * q + 1] : -M[2 * q + 1];
    };
    const int i = threadIdx.x;
    if (i < M_NTERM) {
        // r_t = sum_s c_s conj(Mw[t][s]);  u_t = sum_s conj(c_s) Mu[t][s]
        double rr = 0.0, ri = 0.0, ur = 0.0, ui = 0.0;
        for (int s = 0; s < M_NTERM; ++s) {
            double mr, mi, wr, wi;
            herm(Mu, i, s, mr, mi);
            herm(Mw, i, s, wr, wi);
            rr += cr[s] * wr + ci[s] * wi;
            ri += ci[s] * wr - cr[s] * wi;
            ur += cr[s] * mr + ci[s] * mi;
            ui += cr[s] * mi - ci[s] * mr;
        }
        tr[i] = rr;
        ti[i] = ri;
        tf[i] = cr[i] * ur - ci[i] * ui;
    } else if (i - M_NTERM < M_NDER) {
        // 2 Re(c_t sum_s conj(c_s) D[k][s]), t = der_term(k)
        const int k = i - M_NTERM, t = der_term(k);
        double ur = 0.0, ui = 0.0;
        for (int s = 0; s < M_NTERM; ++s) {
            const double dr = D[2 * (k * M_NTERM + s)], di = D[2 * (k * M_NTERM + s) + 1];
            ur += cr[s] * dr + ci[s] * di;
            ui += cr[s] * di - ci[s] * dr;
        }
        dk[k] = 2.0 * (cr[t] * ur - ci[t] * ui);
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double* row = A.row;
    for (int j = 0; j < CT_NACC; ++j) row[j] = 0.0;
    double fs = 0.0;
    for (int t = 0; t < M_NTERM; ++t) {
        fs += tf[t];
        const int a = term_col(t);
        row[2 + 2 * a] += tr[t] * A.vw_scale;
        row[3 + 2 * a] += ti[t] * A.vw_scale;
    }
    row[1] = fs;
    for (int k = 0; k < M_NDER; ++k) row[2 + 2 * M_NA + der_th(k)] += dk[k];
}
