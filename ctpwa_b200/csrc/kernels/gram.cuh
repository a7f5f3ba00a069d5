// Phase-space Gram matrix on the tensor cores (tcgen05, sm_100a).
//
//   M_ab = (1/W) sum_e w_e sum_p A_{e,p,a} conj(A_{e,p,b}),
//   A_{e,p,a} = sum_{t in column a} F_t(theta) SL_{plane(t),p}(e)
//
// the reference's normalisation matrix (scalePhspAmpsKernel + CGEMM over the
// amplitude table, src/ComputeHessian.cu:1181-1197, src/Analysis.cu:729-805).
// The amplitudes are formed on the fly from the angular tables and the
// mixed-form (FP32) lineshapes and never written to HBM.
//
// Formulation. A CTA of 256 threads takes tiles of 256 events; thread t
// forms event t's real amplitude vector X (ROWS = npol x 2nA values: Re A
// and Im A of every column for every polarisation, scaled by sqrt(w)) and
// writes it as column t of the operand tile Xt [rows][256 events] in shared
// memory. Each FP32 value x is split into two BF16 numbers, hi = rn(x) and
// lo = rn(x - hi) (residual ~2^-18 |x|). With R8 = ROWS rounded up to 8 and
// 2 R8 <= 128, the hi values fill rows [0, R8) and the lo values rows
// [R8, 2 R8) of one tile, and one MMA chain (kind::f16, BF16 operands, FP32
// accumulator in tensor memory, M = 128, N = 2 R8, K = 16 events per
// instruction) gives all four products hi.hi, hi.lo, lo.hi and lo.lo at
// once; larger models keep hi and lo in two tiles and issue the four
// products as four MMAs (N = ROWS rounded up to 16). The tile's K-steps go to
// NACC accumulators in turn (64 or 128 events each); after every tile they
// are read (tcgen05.ld) and added in FP64 in shared memory, so FP32
// accumulation spans 64 or 128 events only. The npol diagonal blocks of the
// (npol 2nA)^2 product are the Gram of each polarisation; per-CTA FP64
// partials are reduced in a fixed order by ct_gram_finalize.
//
// Shared-memory operand layout: MN-major (the matrix rows contiguous), no
// swizzle: element (row m, event k) at
//   (k / 8) * 128 + (m / 8) * SBO + (k % 8) * 16 + (m % 8) * 2,  SBO = 4096,
// so a thread writes the 8 rows of a core matrix as one 16-byte store and a
// warp's stores are contiguous; the two 8-event groups of one K = 16 step
// are LBO = 128 bytes apart. Tensor-memory layout of D (cta_group::1,
// M = 128): row m in lane m, column n in column n. Several CTAs per SM
// overlap one CTA's MMA chain and read-out with the others' event work.
#pragma once

#include "fused_nll.cuh"

#define CT_GRAM_THREADS 256
#define CT_GRAM_TILE 256  // events per tile (one per thread)
#ifndef CT_GRAM_HESS
#define CT_GRAM_HESS 0
#endif
// CT_GRAM_HESS: the sums of the Hessian's coupling block over a data-like
// sample instead of the normalisation matrix: the npol amplitude row blocks
// scaled by sqrt(w / f_e), and one more block, c_a = sum_p A_pa conj(S_p)
// (S_p = sum_a v_a A_pa, f_e = sum_p |S_p|^2), scaled by sqrt(w) / f_e
#define CT_GRAM_BLOCKS (M_NPOL + CT_GRAM_HESS)
#define CT_GRAM_ROWS (CT_GRAM_BLOCKS * 2 * M_NA)
static_assert(CT_GRAM_ROWS <= 128, "the tensor-core Gram supports (npol + 1 for the Hessian sums) * 2 * nA <= 128");
#define CT_GRAM_R8 ((CT_GRAM_ROWS + 7) / 8 * 8)
#define CT_GRAM_STACK (2 * CT_GRAM_R8 <= 128)                 // hi and lo rows in one tile
// MMA N (a multiple of 16 for M = 128)
#define CT_GRAM_N (CT_GRAM_STACK ? 2 * CT_GRAM_R8 : (CT_GRAM_ROWS + 15) / 16 * 16)
// accumulators per tile, each over 256 / NACC events (the tensor core's FP32
// accumulation rounds toward zero: its bias grows with the accumulation length)
#define CT_GRAM_NACC (CT_GRAM_N <= 64 ? 4 : 2)
#define CT_GRAM_TMEM_COLS \
    (CT_GRAM_NACC * CT_GRAM_N <= 32 ? 32 : CT_GRAM_NACC * CT_GRAM_N <= 64 ? 64 : CT_GRAM_NACC * CT_GRAM_N <= 128 ? 128 : 256)
#define CT_GRAM_SBO 4096
#define CT_GRAM_PART (128 * CT_GRAM_TILE * 2)  // bytes of one BF16 operand tile (128 rows)
#define CT_GRAM_NPART (CT_GRAM_STACK ? 1 : 2)
// dynamic shared memory: operand tile(s), then the FP64 sums [2 nA][128]
#define CT_GRAM_SMEM (CT_GRAM_NPART * CT_GRAM_PART + 128 * 2 * M_NA * 8)
#ifndef CT_GRAM_PAIRED
#define CT_GRAM_PAIRED 0
#endif

struct CtGramArgs {
    const float2* slamp;     // mixed angular table of the phase-space sample (event-major records)
    const float* evf;        // FP32 frontier rows
    const double* evd;       // FP64 frontier rows
    const double* w;         // per-event weights or nullptr
    long long n, ld;
    const CtConsts* K;       // this call's parameter-only constants (written by ct_prologue)
    double* partials;        // [gridDim.x][CT_GRAM_ROWS][2 M_NA]
    int* err;                // set to 2 when the tensor-core pipeline did not complete in time
    int pad;
};

__device__ __forceinline__ unsigned short ct_bf16_rn(float x)
{
    unsigned short r;
    asm("cvt.rn.bf16.f32 %0, %1;" : "=h"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float ct_bf16_to_f32(unsigned short h) { return __uint_as_float((unsigned)h << 16); }

// shared-memory matrix descriptor (tcgen05): start, leading-dimension and
// stride-dimension byte offsets, descriptor version 1, no swizzle
__device__ __forceinline__ unsigned long long ct_umma_desc(unsigned saddr, unsigned lbo, unsigned sbo)
{
    return (unsigned long long)((saddr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: FP32 accumulator, BF16 A and B, both MN-major, N, M
__device__ __forceinline__ unsigned ct_umma_idesc_bf16_mn(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((unsigned)(N >> 3) << 17) |
           ((unsigned)(M >> 4) << 24);
}

__device__ __forceinline__ void ct_tc_mma(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned idesc,
                                          unsigned accumulate)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void ct_tc_commit(unsigned long long* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(ct_smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void ct_tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void ct_tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void ct_fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this warp's 32 tensor-memory lanes (lane = thread)
__device__ __forceinline__ void ct_tmem_ld16(unsigned taddr, float* v)
{
    unsigned r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// two CTAs per SM (<= 128 registers): one CTA's MMA chain, barriers and
// read-out overlap the other's event work
extern "C" __global__ void __launch_bounds__(CT_GRAM_THREADS, 2) ct_gram(CtGramArgs G)
{
    constexpr int NROW = CT_GRAM_ROWS, R8 = CT_GRAM_R8, NN = CT_GRAM_N, NA2 = 2 * M_NA;
    constexpr bool STACK = CT_GRAM_STACK;
    constexpr int NPS = CT_GRAM_PAIRED ? CT_NPOL_STORED : M_NPOL;
    extern __shared__ __align__(1024) unsigned char gsm[];
    double* sacc = (double*)(gsm + CT_GRAM_NPART * CT_GRAM_PART);  // [NA2][128]: a warp's rows are consecutive
    __shared__ __align__(8) unsigned long long bar;
    __shared__ unsigned tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5;

    // zero the operand tile(s) (unused rows stay zero) and the FP64 sums
    for (int i = tid; i < CT_GRAM_SMEM / 16; i += CT_GRAM_THREADS) reinterpret_cast<uint4*>(gsm)[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        ct_mbar_init(&bar, 1);
        ct_fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(ct_smem_addr(&tmem_slot)),
                     "r"((unsigned)CT_GRAM_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    ct_fence_async_smem();
    ct_tc_fence_before();
    __syncthreads();
    ct_tc_fence_after();
    const unsigned tmem = tmem_slot;

    const long long ntiles = (G.n + CT_GRAM_TILE - 1) / CT_GRAM_TILE;
    const unsigned idesc = ct_umma_idesc_bf16_mn(128, NN);
    const unsigned sbase = ct_smem_addr(gsm);
    // this thread's column (event slot) in the operand tile
    const unsigned kofs = (unsigned)(tid >> 3) * 128u + (unsigned)(tid & 7) * 16u;
    // read-out: warps 0-3 read tensor-memory lanes 0-127 (one D row each)
    const int my_row = tid;                       // D row of warps 0-3
    const int my_r = STACK && my_row >= R8 ? my_row - R8 : my_row;  // operand row (hi or lo)
    const int my_blk = my_r < NROW ? my_r / NA2 : 0;
    bool timed_out = false;
    unsigned it = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        // ---- this thread's event -> operand column tid ----
        const long long e = tile * CT_GRAM_TILE + tid;
        float x[CT_GRAM_BLOCKS * NA2];
#pragma unroll
        for (int i = 0; i < CT_GRAM_BLOCKS * NA2; ++i) x[i] = 0.0f;
        if (e < G.n) {
            CtEvent<float> ev;
            ev.load(CtEvent<float>::at(G.evf, e), G.evd + e, G.ld);
            float Fr[M_NTERM], Fi[M_NTERM], dFr[M_NDER > 0 ? M_NDER : 1], dFi[M_NDER > 0 ? M_NDER : 1];
            ev.columns(G.K->c, G.K->ch, G.K->cl, Fr, Fi, dFr, dFi);
            const float sw = (G.w && !CT_GRAM_HESS) ? (float)sqrt(G.w[e]) : 1.0f;
#pragma unroll
            for (int t = 0; t < M_NTERM; ++t) {
                const int a = term_col(t);
                const float fr = Fr[t] * sw, fi = Fi[t] * sw;
#pragma unroll
                for (int p = 0; p < NPS; ++p) {
                    const float2 sl = G.slamp[e * CT_SL32_STRIDE(M_NPLANE * NPS) + term_plane(t) * NPS + p];
                    x[p * NA2 + a] += fr * sl.x - fi * sl.y;
                    x[p * NA2 + M_NA + a] += fr * sl.y + fi * sl.x;
                    const int q = M_NPOL - 1 - p;
                    if (CT_GRAM_PAIRED && q != p) {  // SL_q = conj(SL_p)
                        x[q * NA2 + a] += fr * sl.x + fi * sl.y;
                        x[q * NA2 + M_NA + a] += fi * sl.x - fr * sl.y;
                    }
                }
            }
#if CT_GRAM_HESS
            {
                // S_p = sum_a v_a A_pa, f = sum_p |S_p|^2, c_a = sum_p A_pa conj(S_p)
                float f = 0.0f, cr[M_NA], ci[M_NA];
#pragma unroll
                for (int a = 0; a < M_NA; ++a) cr[a] = ci[a] = 0.0f;
#pragma unroll
                for (int p = 0; p < M_NPOL; ++p) {
                    float sr = 0.0f, si = 0.0f;
#pragma unroll
                    for (int a = 0; a < M_NA; ++a) {
                        const float vr = G.K->vh[2 * a], vi = G.K->vh[2 * a + 1];
                        const float ar = x[p * NA2 + a], ai = x[p * NA2 + M_NA + a];
                        sr += vr * ar - vi * ai;
                        si += vr * ai + vi * ar;
                    }
                    f += sr * sr + si * si;
#pragma unroll
                    for (int a = 0; a < M_NA; ++a) {
                        const float ar = x[p * NA2 + a], ai = x[p * NA2 + M_NA + a];
                        cr[a] += ar * sr + ai * si;
                        ci[a] += ai * sr - ar * si;
                    }
                }
                const double we = G.w ? G.w[e] : 1.0;
                // an event with f = 0 (its log-likelihood is clamped) contributes no curvature
                const float sa = f > 0.0f ? (float)sqrt(we / (double)f) : 0.0f;
                const float sc = f > 0.0f ? (float)(sqrt(we) / (double)f) : 0.0f;
#pragma unroll
                for (int i = 0; i < M_NPOL * NA2; ++i) x[i] *= sa;
#pragma unroll
                for (int a = 0; a < M_NA; ++a) {
                    x[M_NPOL * NA2 + a] = cr[a] * sc;
                    x[M_NPOL * NA2 + M_NA + a] = ci[a] * sc;
                }
            }
#endif
        }
        // hi and lo BF16 values, 8 rows (one core matrix) per 16-byte store
#pragma unroll
        for (int g = 0; g < R8 / 8; ++g) {
            unsigned hw[4], lw[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                unsigned short h2[2], l2[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int r = 8 * g + 2 * q + u;
                    const float v = r < NROW ? x[r] : 0.0f;
                    h2[u] = ct_bf16_rn(v);
                    l2[u] = ct_bf16_rn(v - ct_bf16_to_f32(h2[u]));
                }
                hw[q] = (unsigned)h2[0] | ((unsigned)h2[1] << 16);
                lw[q] = (unsigned)l2[0] | ((unsigned)l2[1] << 16);
            }
            const unsigned hoff = (unsigned)g * CT_GRAM_SBO + kofs;
            const unsigned loff = STACK ? (unsigned)(g + R8 / 8) * CT_GRAM_SBO + kofs : CT_GRAM_PART + hoff;
            *reinterpret_cast<uint4*>(gsm + hoff) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
            *reinterpret_cast<uint4*>(gsm + loff) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        }
        ct_fence_async_smem();
        ct_tc_fence_before();
        __syncthreads();
        // ---- one thread issues the tile's MMA chain: K-steps [h SPA, (h+1) SPA)
        // into accumulator h (tensor-memory columns [h NN, (h+1) NN)) ----
        if (tid == 0) {
            ct_tc_fence_after();
            constexpr int SPA = CT_GRAM_TILE / 16 / CT_GRAM_NACC;
#pragma unroll 1
            for (int s = 0; s < CT_GRAM_TILE / 16; ++s) {
                const unsigned dt = tmem + (unsigned)((s / SPA) * NN);
                const bool first = s % SPA == 0;
                if constexpr (STACK) {
                    const unsigned long long d = ct_umma_desc(sbase + 256u * s, 128u, CT_GRAM_SBO);
                    ct_tc_mma(dt, d, d, idesc, first ? 0u : 1u);
                } else {
#pragma unroll
                    for (int pass = 0; pass < 4; ++pass) {
                        const unsigned pa = (pass < 2 ? 1u : 0u) * CT_GRAM_PART;
                        const unsigned pb = (pass == 0 || pass == 2 ? 1u : 0u) * CT_GRAM_PART;
                        ct_tc_mma(dt, ct_umma_desc(sbase + pa + 256u * s, 128u, CT_GRAM_SBO),
                                  ct_umma_desc(sbase + pb + 256u * s, 128u, CT_GRAM_SBO), idesc,
                                  (first && pass == 0) ? 0u : 1u);
                    }
                }
            }
            ct_tc_commit(&bar);
        }
        // ---- the tile's accumulator -> FP64 sums in shared memory ----
        if (!ct_mbar_wait(&bar, it & 1u, CT_WAIT_LIMIT)) timed_out = true;
        if (__syncthreads_or(timed_out)) break;
        ct_tc_fence_after();
        if (warp < 4) {
            const unsigned lanes = tmem + ((unsigned)(warp * 32) << 16);
#pragma unroll
            for (int c0 = 0; c0 < NN; c0 += 16) {
                double t[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) t[j] = 0.0;
#pragma unroll
                for (int h = 0; h < CT_GRAM_NACC; ++h) {
                    float v[16];
                    ct_tmem_ld16(lanes + (unsigned)(h * NN + c0), v);
#pragma unroll
                    for (int j = 0; j < 16; ++j) t[j] += (double)v[j];
                }
                if (my_r < NROW && (my_row < R8 || (STACK && my_row < 2 * R8))) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        // column c0 + j: a hi column (< R8) or, stacked, a lo column
                        const int c = STACK && c0 + j >= R8 ? c0 + j - R8 : c0 + j;
                        const int col = c - my_blk * NA2;
                        if (col >= 0 && col < NA2 && c0 + j < NN) sacc[col * 128 + my_row] += t[j];
                    }
                }
            }
        }
        ct_tc_fence_before();
        __syncthreads();
    }
    const bool aborted = __syncthreads_or(timed_out);
    if (aborted) {
        if (tid == 0) atomicExch(G.err, 2);
        // the loop left at tile `it`, whose MMA chain may still run: wait for
        // it (bounded) before freeing tensor memory
        ct_mbar_wait(&bar, it & 1u, CT_WAIT_LIMIT);
    }
    ct_tc_fence_before();
    __syncthreads();
    ct_tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((unsigned)CT_GRAM_TMEM_COLS)
                     : "memory");
    // this CTA's FP64 partial rows (hi and lo rows of a stacked tile added)
    double* out = G.partials + (size_t)blockIdx.x * NROW * NA2;
    for (int i = tid; i < NROW * NA2; i += CT_GRAM_THREADS) {
        const int r = i / NA2, j = i % NA2;
        double v = sacc[j * 128 + r];
        if (STACK) v += sacc[j * 128 + R8 + r];
        out[i] = aborted ? 0.0 : v;
    }
}

#if CT_GRAM_HESS
// Fixed-order sum of the CTA partials of the Hessian sums: out[0] = the
// amplitude blocks summed over polarisations, out[1] = the c block, each the
// real [2 nA][2 nA] matrix sum_e X X^T of its scaled rows [Re; Im].
extern "C" __global__ void ct_gram_hess_finalize(const double* __restrict__ partials, int nblocks,
                                                 double* __restrict__ out)
{
    constexpr int NA2 = 2 * M_NA;
    for (int i = threadIdx.x; i < NA2 * NA2; i += blockDim.x) {
        double g1 = 0.0, g2 = 0.0;
        for (int c = 0; c < nblocks; ++c) {
            const double* P = partials + (size_t)c * CT_GRAM_ROWS * NA2;
#pragma unroll 1
            for (int p = 0; p < M_NPOL; ++p) g1 += P[(size_t)p * NA2 * NA2 + i];
            g2 += P[(size_t)M_NPOL * NA2 * NA2 + i];
        }
        out[i] = g1;
        out[NA2 * NA2 + i] = g2;
    }
}
#endif

// Fixed-order sum of the CTA partials into the complex Gram (reference
// orientation M_ab = sum A_a conj(A_b)), scaled by 1/W: out [nA][nA][2].
extern "C" __global__ void ct_gram_finalize(const double* __restrict__ partials, int nblocks, double inv_w,
                                            double* __restrict__ out)
{
    constexpr int NA2 = 2 * M_NA;
    for (int i = threadIdx.x; i < M_NA * M_NA; i += blockDim.x) {
        const int a = i / M_NA, b = i % M_NA;
        double re = 0.0, im = 0.0;
        for (int c = 0; c < nblocks; ++c) {
            const double* P = partials + (size_t)c * CT_GRAM_ROWS * NA2;
#pragma unroll 1
            for (int p = 0; p < M_NPOL; ++p) {
                const double* B = P + (size_t)p * NA2 * NA2;
                re += B[a * NA2 + b] + B[(M_NA + a) * NA2 + (M_NA + b)];
                im += B[(M_NA + a) * NA2 + b] - B[a * NA2 + (M_NA + b)];
            }
        }
        out[2 * i] = re * inv_w;
        out[2 * i + 1] = im * inv_w;
    }
}
