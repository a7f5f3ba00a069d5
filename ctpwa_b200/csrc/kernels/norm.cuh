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
// the output rows (terms, derivative entries, weighted terms), ordered by
// angular plane, are cut into groups of CT_NORM_RB rows; thread (group,
// slice) adds the tile's events slice, slice + slices, ... to its rows x all
// columns, so per event it reads its rows' factors, the column factors and
// the plane products of its rows' planes once and reuses them from
// registers. At the end the slices' sums are added in a fixed order through
// shared memory into one partial row per CTA, reduced over CTAs in a fixed
// order by ct_norm_reduce. Output (complex, full matrices):
//   Mu [M_NTERM][M_NTERM], D [M_NDER][M_NTERM], Mw [M_NTERM][M_NTERM] (weighted).
#pragma once

#include "fused_nll.cuh"

#define CT_NORM_BLOCK 128
#define CT_NORM_TILE 128  // events per tile (one per thread in phase 1)
#define CT_NORM_NG (M_NPLANE * (M_NPLANE + 1) / 2)
// rows per phase-2 thread (rows x M_NTERM complex sums in registers; 4
// spilled on K+K-pi0 next to the FP64 lineshapes of phase 1)
#define CT_NORM_RB 2
// record per event, in double2 slots: F_t, dF_k, G pairs, (w, 0); odd length
// so the phase-1 stores of consecutive threads fall in different banks
#define CT_NORM_REC0 (M_NTERM + M_NDER + CT_NORM_NG + 1)
#define CT_NORM_REC (CT_NORM_REC0 | 1)
#define CT_NORM_WSLOT (M_NTERM + M_NDER + CT_NORM_NG)

struct CtNormArgs {
    const double2* slamp;  // FP64 angular table [M_NPLANE * M_NPOL][ld]
    const double* ev;      // FP64 frontier rows [M_NEV][ld]
    const double* w;       // per-event weights or nullptr
    long long n, ld;
    const double* consts;  // [M_NCONST] parameter-only subexpressions at the cached theta
    double* partials;      // [grid][nrows * M_NTERM][2]
    int nrows;             // output rows: M_NTERM + M_NDER (+ M_NTERM when weighted)
    int pad;
};

__device__ __forceinline__ int ct_norm_gpair(int c, int d)  // c <= d
{
    return c * M_NPLANE - c * (c - 1) / 2 + (d - c);
}

// record slot of the output row's first factor, its plane, weighting
__device__ __forceinline__ void ct_norm_rowinfo(int r, int& slot, int& plane, bool& weighted)
{
    weighted = false;
    if (r < M_NTERM) {
        slot = r;
        plane = term_plane(r);
    } else if (r < M_NTERM + M_NDER) {
        slot = r;
        plane = term_plane(der_term(r - M_NTERM));
    } else {
        slot = r - M_NTERM - M_NDER;
        plane = term_plane(slot);
        weighted = true;
    }
}

extern "C" __global__ void __launch_bounds__(CT_NORM_BLOCK) ct_norm_build(CtNormArgs A)
{
    extern __shared__ double2 nrec[];  // [CT_NORM_TILE][CT_NORM_REC]; at the end [slices][nrows][M_NTERM]
    __shared__ double sC[CT_NCONST_ALLOC];
    for (int i = threadIdx.x; i < M_NCONST; i += CT_NORM_BLOCK) sC[i] = A.consts[i];

    // ---- this thread's rows (plane-sorted order) and event slice ----
    const int nrows = A.nrows;
    const int groups = (nrows + CT_NORM_RB - 1) / CT_NORM_RB;
    const int slices = CT_NORM_BLOCK / groups;  // >= 1 (host check)
    const int grp = threadIdx.x % groups, sl = threadIdx.x / groups;
    const bool active = sl < slices;
    int rid[CT_NORM_RB], aslot[CT_NORM_RB];
    unsigned cjm[CT_NORM_RB];           // bit d: plane pair (row plane, d) stored transposed
    short gsl[CT_NORM_RB][M_NPLANE];    // record slot of G(row plane, d)
    bool wrow[CT_NORM_RB];
    {
        // position grp * RB + j of the rows listed plane by plane
        int pos = 0;
#pragma unroll
        for (int j = 0; j < CT_NORM_RB; ++j) rid[j] = -1;
        for (int c = 0; c < M_NPLANE; ++c)
            for (int r = 0; r < nrows; ++r) {
                int sl_, pl;
                bool wt_;
                ct_norm_rowinfo(r, sl_, pl, wt_);
                if (pl != c) continue;
                const int j = pos - grp * CT_NORM_RB;
#pragma unroll
                for (int q = 0; q < CT_NORM_RB; ++q)
                    if (q == j) rid[q] = r;
                ++pos;
            }
#pragma unroll
        for (int j = 0; j < CT_NORM_RB; ++j) {
            int pl = 0;
            bool wt_ = false;
            aslot[j] = 0;
            if (rid[j] >= 0) ct_norm_rowinfo(rid[j], aslot[j], pl, wt_);
            wrow[j] = wt_;
            cjm[j] = 0u;
#pragma unroll
            for (int d = 0; d < M_NPLANE; ++d) {
                gsl[j][d] = (short)(M_NTERM + M_NDER + (pl <= d ? ct_norm_gpair(pl, d) : ct_norm_gpair(d, pl)));
                if (pl > d) cjm[j] |= 1u << d;
            }
        }
    }
    double accr[CT_NORM_RB][M_NTERM], acci[CT_NORM_RB][M_NTERM];
#pragma unroll
    for (int j = 0; j < CT_NORM_RB; ++j)
#pragma unroll
        for (int s = 0; s < M_NTERM; ++s) {
            accr[j][s] = 0.0;
            acci[j][s] = 0.0;
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
                double2 sl2[M_NPLANE * M_NPOL];
#pragma unroll
                for (int c = 0; c < M_NPLANE * M_NPOL; ++c) sl2[c] = A.slamp[(long long)c * A.ld + e];
#pragma unroll
                for (int c = 0; c < M_NPLANE; ++c)
#pragma unroll
                    for (int d = c; d < M_NPLANE; ++d) {
                        double gr = 0.0, gi = 0.0;
#pragma unroll
                        for (int p = 0; p < M_NPOL; ++p) {
                            const double2 x = sl2[c * M_NPOL + p], y = sl2[d * M_NPOL + p];
                            gr += x.x * y.x + x.y * y.y;
                            gi += x.y * y.x - x.x * y.y;
                        }
                        r[M_NTERM + M_NDER + ct_norm_gpair(c, d)] = make_double2(gr, gi);
                    }
                r[CT_NORM_WSLOT] = make_double2(A.w ? __ldg(A.w + e) : 1.0, 0.0);
            } else {
                // past the sample's end: zero factors contribute nothing
#pragma unroll
                for (int k = 0; k < CT_NORM_REC0; ++k) r[k] = make_double2(0.0, 0.0);
            }
        }
        __syncthreads();
        // ---- phase 2: this slice's events into this thread's rows ----
        if (active)
            for (int i = sl; i < CT_NORM_TILE; i += slices) {
                const double2* r = nrec + (size_t)i * CT_NORM_REC;
                double2 b[M_NTERM];
#pragma unroll
                for (int s = 0; s < M_NTERM; ++s) b[s] = r[s];
                const double we = r[CT_NORM_WSLOT].x;
#pragma unroll
                for (int j = 0; j < CT_NORM_RB; ++j) {
                    double2 a = r[aslot[j]];
                    if (wrow[j]) {
                        a.x *= we;
                        a.y *= we;
                    }
                    double2 g[M_NPLANE];
#pragma unroll
                    for (int d = 0; d < M_NPLANE; ++d) {
                        g[d] = r[gsl[j][d]];
                        if (cjm[j] >> d & 1u) g[d].y = -g[d].y;
                    }
#pragma unroll
                    for (int s = 0; s < M_NTERM; ++s) {
                        // a conj(b_s) G(row plane, plane(s))
                        const double xr = a.x * b[s].x + a.y * b[s].y, xi = a.y * b[s].x - a.x * b[s].y;
                        const double2 gg = g[term_plane(s)];
                        accr[j][s] = fma(xr, gg.x, fma(-xi, gg.y, accr[j][s]));
                        acci[j][s] = fma(xr, gg.y, fma(xi, gg.x, acci[j][s]));
                    }
                }
            }
        __syncthreads();
    }
    // ---- the slices' sums, in slice order, into this CTA's partial row ----
    double2* red = nrec;  // [slices][nrows][M_NTERM]
    if (active)
#pragma unroll
        for (int j = 0; j < CT_NORM_RB; ++j)
            if (rid[j] >= 0)
#pragma unroll
                for (int s = 0; s < M_NTERM; ++s)
                    red[((size_t)sl * nrows + rid[j]) * M_NTERM + s] = make_double2(accr[j][s], acci[j][s]);
    __syncthreads();
    const int ne = nrows * M_NTERM;
    for (int q = threadIdx.x; q < ne; q += CT_NORM_BLOCK) {
        double xr = 0.0, xi = 0.0;
        for (int k = 0; k < slices; ++k) {
            const double2 x = red[(size_t)k * ne + q];
            xr += x.x;
            xi += x.y;
        }
        A.partials[((long long)blockIdx.x * ne + q) * 2] = xr;
        A.partials[((long long)blockIdx.x * ne + q) * 2 + 1] = xi;
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
    const double* mat;           // complex Mu [M_NTERM][M_NTERM], D [M_NDER][M_NTERM], Mw (ct_norm_reduce)
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
    constexpr int NE = (2 * M_NTERM + M_NDER) * M_NTERM;
    __shared__ double sm[2 * NE];
    __shared__ double cr[M_NTERM], ci[M_NTERM];
    __shared__ double tr[M_NTERM], ti[M_NTERM], tf[M_NTERM];  // per term: r_t, Re(c_t u_t)
    __shared__ double dk[M_NDER > 0 ? M_NDER : 1];            // per derivative entry
    const int ne = (M_NTERM + M_NDER + (A.weighted ? M_NTERM : 0)) * M_NTERM;
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
    const double* D = sm + 2 * M_NTERM * M_NTERM;
    const double* Mw = A.weighted ? sm + 2 * (M_NTERM + M_NDER) * M_NTERM : Mu;
    const int i = threadIdx.x;
    if (i < M_NTERM) {
        // r_t = sum_s c_s conj(Mw[t][s]);  u_t = sum_s conj(c_s) Mu[t][s]
        double rr = 0.0, ri = 0.0, ur = 0.0, ui = 0.0;
        for (int s = 0; s < M_NTERM; ++s) {
            const double mr = Mu[2 * (i * M_NTERM + s)], mi = Mu[2 * (i * M_NTERM + s) + 1];
            const double wr = Mw[2 * (i * M_NTERM + s)], wi = Mw[2 * (i * M_NTERM + s) + 1];
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
