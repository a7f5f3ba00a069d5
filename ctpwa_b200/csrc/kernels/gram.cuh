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
// Formulation. One CTA of 128 threads takes tiles of 128 events; thread t
// forms event t's real amplitude row vector X (NROW = npol x 2nA values:
// Re A and Im A of every column for every polarisation, scaled by sqrt(w))
// and writes it as column t of the operand tile Xt [rows][128 events] in
// shared memory. One MMA chain then accumulates D = Xt Xt^T
// ((npol 2nA)^2, of which the npol diagonal blocks are the Gram of each
// polarisation) in tensor memory: kind::f16 with BF16 operands and FP32
// accumulation, M = 64 (or 128) rows, N = NROW rounded up to 8, K = 16
// events per instruction. Each FP32 value x is split as x = hi + lo (two
// BF16 numbers, hi = rn(x), lo = rn(x - hi)) and the four products
// lo.lo + lo.hi + hi.lo + hi.hi are accumulated, which leaves a residual of
// ~2^-18 |x| per value. Tiles alternate between two FP32 accumulators in
// tensor memory; while one tile's MMAs run, the previous tile's accumulator
// is read out (tcgen05.ld) into per-thread FP64 sums, so FP32 accumulation
// spans one tile (32 MMAs) only. Per-CTA FP64 partials are reduced in a fixed
// order by ct_gram_finalize.
//
// Shared-memory operand layout: K-major, no swizzle ("interleaved" core
// matrices of 8 rows x 16 bytes): element (row m, event k) at
//   (m / 8) * SBO + (k / 8) * 128 + (m % 8) * 16 + (k % 8) * 2,  SBO = 2048,
// so the two core matrices of one K = 16 step are LBO = 128 bytes apart.
// Tensor-memory layout of D (cta_group::1): M = 128, row m in lane m; M = 64,
// row m in lane (m % 16) + 32 (m / 16); column n in column n.
#pragma once

#include "fused_nll.cuh"

#define CT_GRAM_THREADS 128
#define CT_GRAM_TILE 128  // events per tile (one per thread)
#define CT_GRAM_ROWS (M_NPOL * 2 * M_NA)
static_assert(CT_GRAM_ROWS <= 128, "the tensor-core Gram supports npol * 2 * nA <= 128");
#define CT_GRAM_M (CT_GRAM_ROWS <= 64 ? 64 : 128)
#define CT_GRAM_N ((CT_GRAM_ROWS + 7) / 8 * 8)
// two accumulators (tiles alternate), each CT_GRAM_ACC_COLS columns
#define CT_GRAM_ACC_COLS ((CT_GRAM_N + 15) / 16 * 16)
#define CT_GRAM_TMEM_COLS (2 * CT_GRAM_ACC_COLS <= 32 ? 32 : 2 * CT_GRAM_ACC_COLS <= 64 ? 64 : 2 * CT_GRAM_ACC_COLS <= 128 ? 128 : 256)
#define CT_GRAM_SBO 2048
#define CT_GRAM_PART (CT_GRAM_M * CT_GRAM_TILE * 2)  // bytes of one BF16 operand tile
// dynamic shared memory: [2 buffers][hi, lo] operand tiles
#define CT_GRAM_SMEM (4 * CT_GRAM_PART)
#ifndef CT_GRAM_PAIRED
#define CT_GRAM_PAIRED 0
#endif

struct CtGramArgs {
    const float2* slamp;     // mixed angular table of the phase-space sample
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

// shared-memory matrix descriptor (tcgen05): start, leading (K) and stride
// (M/N) byte offsets, descriptor version 1, no swizzle
__device__ __forceinline__ unsigned long long ct_umma_desc(unsigned saddr, unsigned lbo, unsigned sbo)
{
    return (unsigned long long)((saddr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N, M
__device__ __forceinline__ unsigned ct_umma_idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(M >> 4) << 24);
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

extern "C" __global__ void __launch_bounds__(CT_GRAM_THREADS) ct_gram(CtGramArgs G)
{
    constexpr int NROW = CT_GRAM_ROWS, MM = CT_GRAM_M, NN = CT_GRAM_N, NA2 = 2 * M_NA;
    constexpr int NPS = CT_GRAM_PAIRED ? CT_NPOL_STORED : M_NPOL;
    extern __shared__ __align__(1024) unsigned char gsm[];
    __shared__ __align__(8) unsigned long long bar[2];
    __shared__ unsigned tmem_slot;
    __shared__ int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // zero both operand buffers once: rows >= NROW stay zero
    for (int i = tid; i < CT_GRAM_SMEM / 16; i += CT_GRAM_THREADS) reinterpret_cast<uint4*>(gsm)[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        ct_mbar_init(&bar[0], 1);
        ct_mbar_init(&bar[1], 1);
        ct_fence_mbar_init();
        abort_flag = 0;
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

    // this thread's D row in tensor memory (one row per lane; M = 64 uses
    // the first 16 lanes of each warp's quarter)
    const int my_row = MM == 128 ? tid : (lane < 16 ? 16 * warp + lane : NROW);
    const int my_blk = my_row < NROW ? my_row / NA2 : 0;
    double acc[NA2];
#pragma unroll
    for (int j = 0; j < NA2; ++j) acc[j] = 0.0;

    // rows of this warp's tensor-memory lanes -> FP64 sums of this thread's
    // row (columns of its polarisation block)
    auto gram_readout = [&](unsigned tacc) {
        if (MM == 128 || warp * 16 < NROW) {
#pragma unroll
            for (int c0 = 0; c0 < NN; c0 += 16) {
                float v[16];
                ct_tmem_ld16(tacc + ((unsigned)(warp * 32) << 16) + (unsigned)c0, v);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = c0 + j - my_blk * NA2;
                    if (my_row < NROW && col >= 0 && col < NA2) acc[col] += (double)v[j];
                }
            }
        }
    };
    const long long ntiles = (G.n + CT_GRAM_TILE - 1) / CT_GRAM_TILE;
    const unsigned idesc = ct_umma_idesc_bf16(MM, NN);
    const unsigned sbase = ct_smem_addr(gsm);
    unsigned uses[2] = {0u, 0u};  // commits issued per buffer
    int it = 0;
    bool timed_out = false;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const int b = it & 1;
        // the buffer's previous MMAs (two tiles ago) must be done before it is rewritten
        if (uses[b] > 0) {
            if (!ct_mbar_wait(&bar[b], (uses[b] - 1) & 1u, CT_WAIT_LIMIT)) timed_out = true;
            if (__syncthreads_or(timed_out)) break;
        }
        // ---- this thread's event -> operand column tid of buffer b ----
        const long long e = tile * CT_GRAM_TILE + tid;
        float xr[M_NPOL][M_NA], xi[M_NPOL][M_NA];
#pragma unroll
        for (int p = 0; p < M_NPOL; ++p)
#pragma unroll
            for (int a = 0; a < M_NA; ++a) xr[p][a] = xi[p][a] = 0.0f;
        if (e < G.n) {
            CtEvent<float> ev;
            ev.load(G.evf + e, G.evd + e, G.ld);
            float Fr[M_NTERM], Fi[M_NTERM], dFr[M_NDER > 0 ? M_NDER : 1], dFi[M_NDER > 0 ? M_NDER : 1];
            ev.columns(G.K->c, G.K->ch, G.K->cl, Fr, Fi, dFr, dFi);
            const float sw = G.w ? (float)sqrt(G.w[e]) : 1.0f;
#pragma unroll
            for (int t = 0; t < M_NTERM; ++t) {
                const int a = term_col(t);
                const float fr = Fr[t] * sw, fi = Fi[t] * sw;
#pragma unroll
                for (int p = 0; p < NPS; ++p) {
                    const float2 x = G.slamp[(long long)(term_plane(t) * NPS + p) * G.ld + e];
                    xr[p][a] += fr * x.x - fi * x.y;
                    xi[p][a] += fr * x.y + fi * x.x;
                    const int q = M_NPOL - 1 - p;
                    if (CT_GRAM_PAIRED && q != p) {  // SL_q = conj(SL_p)
                        xr[q][a] += fr * x.x + fi * x.y;
                        xi[q][a] += fi * x.x - fr * x.y;
                    }
                }
            }
        }
        unsigned char* hi = gsm + (size_t)b * 2 * CT_GRAM_PART;
        unsigned char* lo = hi + CT_GRAM_PART;
        const unsigned kofs = (unsigned)(tid >> 3) * 128u + (unsigned)(tid & 7) * 2u;
#pragma unroll
        for (int p = 0; p < M_NPOL; ++p)
#pragma unroll
            for (int c = 0; c < NA2; ++c) {
                const int m = p * NA2 + c;
                const float x = c < M_NA ? xr[p][c] : xi[p][c - M_NA];
                const unsigned short h = ct_bf16_rn(x);
                const unsigned short l = ct_bf16_rn(x - ct_bf16_to_f32(h));
                const unsigned off = (unsigned)(m >> 3) * CT_GRAM_SBO + (unsigned)(m & 7) * 16u + kofs;
                *reinterpret_cast<unsigned short*>(hi + off) = h;
                *reinterpret_cast<unsigned short*>(lo + off) = l;
            }
        ct_fence_async_smem();
        ct_tc_fence_before();
        __syncthreads();
        // ---- one thread issues the tile's MMA chain into accumulator b ----
        // (smallest products first: FP32 accumulation rounds relative to the
        // running sum, so the large hi.hi terms come last)
        if (tid == 0) {
            ct_tc_fence_after();
            const unsigned base = sbase + (unsigned)b * 2u * CT_GRAM_PART;
            const unsigned dacc = tmem + (unsigned)(b * CT_GRAM_ACC_COLS);
#pragma unroll
            for (int pass = 0; pass < 4; ++pass) {
                const unsigned pa = (pass < 2 ? 1u : 0u) * CT_GRAM_PART, pb = (pass == 0 || pass == 2 ? 1u : 0u) * CT_GRAM_PART;
#pragma unroll 1
                for (int s = 0; s < CT_GRAM_TILE / 16; ++s) {
                    const unsigned long long da = ct_umma_desc(base + pa + 256u * s, 128u, CT_GRAM_SBO);
                    const unsigned long long db = ct_umma_desc(base + pb + 256u * s, 128u, CT_GRAM_SBO);
                    ct_tc_mma(dacc, da, db, idesc, (s == 0 && pass == 0) ? 0u : 1u);
                }
            }
            ct_tc_commit(&bar[b]);
        }
        ++uses[b];
        // ---- the previous tile's FP32 accumulator -> per-thread FP64 sums ----
        if (it > 0) {
            const int pb = b ^ 1;
            if (!ct_mbar_wait(&bar[pb], (uses[pb] - 1) & 1u, CT_WAIT_LIMIT)) timed_out = true;
            if (__syncthreads_or(timed_out)) break;
            ct_tc_fence_after();
            gram_readout(tmem + (unsigned)(pb * CT_GRAM_ACC_COLS));
        }
    }
    // the last tile's accumulator
    if (!timed_out && it > 0) {
        const int pb = (it - 1) & 1;
        if (!ct_mbar_wait(&bar[pb], (uses[pb] - 1) & 1u, CT_WAIT_LIMIT)) timed_out = true;
        if (!__syncthreads_or(timed_out)) {
            ct_tc_fence_after();
            gram_readout(tmem + (unsigned)(pb * CT_GRAM_ACC_COLS));
        }
    }
    if (__syncthreads_or(timed_out)) {
        if (tid == 0) {
            atomicExch(G.err, 2);
            abort_flag = 1;
        }
        // the MMAs already issued: wait for their completion (bounded) before freeing tensor memory
        for (int bb = 0; bb < 2; ++bb)
            if (uses[bb] > 0) ct_mbar_wait(&bar[bb], (uses[bb] - 1) & 1u, CT_WAIT_LIMIT);
    }
    ct_tc_fence_before();
    __syncthreads();
    ct_tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((unsigned)CT_GRAM_TMEM_COLS)
                     : "memory");
    // this CTA's FP64 partial rows
    double* out = G.partials + (size_t)blockIdx.x * NROW * NA2;
    if (my_row < NROW) {
#pragma unroll
        for (int j = 0; j < NA2; ++j) out[(size_t)my_row * NA2 + j] = abort_flag ? 0.0 : acc[j];
    }
}

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
