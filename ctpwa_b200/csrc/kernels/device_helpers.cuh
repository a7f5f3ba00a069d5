// Value-only helpers called by the generated lineshape code: channel
// phase-space factors of the Flatte lineshape and table lookups (Hist,
// Interp). Same conventions as the reference (include/ResModel.cuh:66-82,
// 248-293, 419-451; src/CustomExpr.cu:1150-1169).
#pragma once

// rho = csqrt(1 - (ma+mb)^2/s) * sqrt(max(0, 1 - (ma-mb)^2/s)); which = 0: Re, 1: Im
__device__ __forceinline__ double ct_rho(double s, double ma, double mb, int which)
{
    double S = (ma + mb) * (ma + mb), Dd = (ma - mb) * (ma - mb);
    double f1 = 1.0 - S / s;
    double f2s = 1.0 - Dd / s;
    double f2 = f2s > 0.0 ? sqrt(f2s) : 0.0;
    if (which == 0) return f1 >= 0.0 ? sqrt(f1) * f2 : 0.0;
    return f1 >= 0.0 ? 0.0 : sqrt(-f1) * f2;
}

// Histogram shape: aux = [m_min, m_max, nbins, values...], linear interpolation
__device__ __forceinline__ double ls_hist(double m, const double* aux)
{
    if (!(m >= 0.0)) return 0.0;
    double lo = aux[0], hi = aux[1];
    int n = (int)aux[2];
    const double* v = aux + 3;
    if (n < 2 || hi <= lo) return 0.0;
    if (m <= lo) return v[0];
    if (m >= hi) return v[n - 1];
    double x = (m - lo) / (hi - lo) * n;
    if (x < 0.0) x = 0.0;
    if (x >= (double)(n - 1)) x = (double)(n - 2);
    int i = (int)x;
    double fr = x - i;
    return v[i] * (1.0 - fr) + v[i + 1] * fr;
}

__device__ __forceinline__ double ls_interp1(const double* y, int i, double fr, int method, int N)
{
    if (method == 1) return y[i] + (y[i + 1] - y[i]) * fr;
    if (method == 2) {
        double y0 = (i > 0) ? y[i - 1] : y[i] - (y[i + 1] - y[i]);
        double y1 = y[i], y2 = y[i + 1];
        double y3 = (i + 2 < N) ? y[i + 2] : y[i + 1] + (y[i + 1] - y[i]);
        double f2 = fr * fr, f3 = f2 * fr;
        return 0.5 * ((2 * y1) + (-y0 + y2) * fr + (2 * y0 - 5 * y1 + 4 * y2 - y3) * f2 +
                      (-y0 + 3 * y1 - 3 * y2 + y3) * f3);
    }
    return y[i];
}

// Interpolated complex table (Interp model aux format)
__device__ __forceinline__ void ls_interp(const double* t, double x, double& Fr, double& Fi)
{
    int hdr = (int)t[0];
    int method = hdr >= 0 ? hdr : -(hdr + 1);
    int N = (int)t[1];
    int i;
    double fr;
    const double *re, *im;
    if (hdr >= 0) {
        double xmin = t[2], dx = t[3];
        re = t + 4;
        im = t + 4 + N;
        double pos = (x - xmin) / dx;
        i = (int)pos;
        if (i < 0) { i = 0; fr = 0.0; }
        else if (i >= N - 1) { i = N - 2; fr = 1.0; }
        else fr = pos - (double)i;
    } else {
        const double* xv = t + 2;
        re = t + 2 + N;
        im = t + 2 + 2 * N;
        int lo = 0, hi = N - 1;
        while (lo < hi - 1) {
            int mid = (lo + hi) / 2;
            if (x < xv[mid]) hi = mid;
            else lo = mid;
        }
        i = lo;
        if (i < 0) { i = 0; fr = 0.0; }
        else if (i >= N - 1) { i = N - 2; fr = 1.0; }
        else fr = (x - xv[i]) / (xv[i + 1] - xv[i]);
        if (method == 2) method = 0;
    }
    Fr = ls_interp1(re, i, fr, method, N);
    Fi = ls_interp1(im, i, fr, method, N);
}

__device__ __forceinline__ double ct_nan() { return __longlong_as_double(0x7ff8000000000000LL); }
__device__ __forceinline__ double ct_inf() { return __longlong_as_double(0x7ff0000000000000LL); }
__device__ __forceinline__ float ct_nanf() { return __int_as_float(0x7fc00000); }
__device__ __forceinline__ float ct_inff() { return __int_as_float(0x7f800000); }

// FP32 reciprocal and square root of the mixed-form lineshapes. The hardware
// approximation (rcp.approx / rsqrt.approx, relative error d of order 2^-23)
// is refined by one Newton-Raphson step whose residual is formed exactly by
// an FMA: the refined value carries a relative error of order d^2 (~1e-14)
// before its final round-to-nearest, so its errors are symmetric and average
// out over a sample instead of biasing the phase-space normalisation (a
// one-sided approximation error would not). Zero and infinite inputs take
// the approximation's own result (the refinement would give NaN there).
__device__ __forceinline__ float ct_rcp_approx(float x)
{
    float r;
    asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float ct_rsqrt_approx(float x)
{
    float r;
    asm("rsqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float ct_rcpf(float x)
{
    const float r0 = ct_rcp_approx(x);
    const float e = fmaf(-x, r0, 1.0f);  // 1 - x r0, exact
    const float r1 = fmaf(r0, e, r0);    // r0 (1 + e) = (1/x)(1 - d^2)
    return (x == 0.0f || fabsf(x) == __int_as_float(0x7f800000)) ? r0 : r1;
}
__device__ __forceinline__ float ct_sqrtf(float x)
{
    const float r = ct_rsqrt_approx(x);
    const float y0 = x * r;
    const float e = fmaf(-y0, y0, x);          // x - y0^2, exact
    const float y1 = fmaf(0.5f * r, e, y0);    // y0 + (x - y0^2) / (2 sqrt x)
    return (x == 0.0f || x == __int_as_float(0x7f800000)) ? x : y1;
}

// t - x and t + x for an FP64 parameter-only t and an FP32 event value x, with
// t entering as hi + lo (the FP32 forms of the mixed lineshapes)
__device__ __forceinline__ float ct_split_sub(double t, float x)
{
    const float hi = (float)t, lo = (float)(t - (double)hi);
    return (hi - x) + lo;
}
__device__ __forceinline__ float ct_split_add(double t, float x)
{
    const float hi = (float)t, lo = (float)(t - (double)hi);
    return (hi + x) + lo;
}

// ---- asynchronous bulk copies global -> shared with mbarrier completion ----
// (cp.async.bulk: the copy engine moves whole contiguous table rows into
// shared memory while the CTA computes on the previous tile)
__device__ __forceinline__ unsigned ct_smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void ct_mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(ct_smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void ct_fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void ct_mbar_expect_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(ct_smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// dst, src and bytes must be multiples of 16 bytes
__device__ __forceinline__ void ct_bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     ct_smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(ct_smem_addr(bar))
                 : "memory");
}
// ---- per-thread asynchronous copies global -> shared (cp.async) ----
// 4-, 8- or 16-byte copies issued by one thread and waited for by the same
// thread (commit groups), no barrier with other threads
template <int BYTES>
__device__ __forceinline__ void ct_cp_async(void* dst, const void* src)
{
    static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async copies 4, 8 or 16 bytes");
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(ct_smem_addr(dst)), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void ct_cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// wait until at most N of this thread's most recent groups are pending
template <int N>
__device__ __forceinline__ void ct_cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Bounded wait for phase `parity` of an mbarrier: gives up after `limit`
// polls (each poll may suspend the thread for a short hardware interval) and
// returns false, so a copy that never completes cannot hang the kernel.
__device__ __forceinline__ bool ct_mbar_wait(unsigned long long* bar, unsigned parity, unsigned limit)
{
    unsigned ok = 0;
    for (unsigned it = 0; it < limit && !ok; ++it)
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(ct_smem_addr(bar)), "r"(parity)
            : "memory");
    return ok != 0;
}
