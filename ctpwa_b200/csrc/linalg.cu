// Dense FP64 linear algebra on the device for fit results: the inverse of a
// symmetric positive definite matrix (Hessian -> covariance), in one CTA.
#include "engine.hpp"

#include <stdexcept>
#include <string>

namespace ctpwa {

namespace {

// In-place Gauss-Jordan inversion without pivoting, which is stable for a
// symmetric positive definite matrix; the k-th pivot is the k-th pivot of its
// LDL^T factorisation, so a pivot <= 0 (or NaN) means the matrix is not
// positive definite: *info = k + 1 and the output is not an inverse.
// The result is symmetrised.
__global__ void ct_spd_inverse_kernel(const double* __restrict__ a, int n, double* __restrict__ out, int* __restrict__ info)
{
    extern __shared__ double col[];  // [n] column k before the update
    __shared__ double piv_s;
    __shared__ int bad;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int idx = tid; idx < n * n; idx += nt) out[idx] = a[idx];
    if (tid == 0) bad = 0;
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (tid == 0) {
            const double p = out[(size_t)k * n + k];
            piv_s = p;
            if (!(p > 0.0)) bad = k + 1;
        }
        __syncthreads();
        if (bad) break;
        const double piv = piv_s;
        for (int i = tid; i < n; i += nt) {
            col[i] = out[(size_t)i * n + k];
            if (i != k) out[(size_t)i * n + k] = 0.0;
        }
        __syncthreads();
        if (tid == 0) out[(size_t)k * n + k] = 1.0;
        __syncthreads();
        for (int j = tid; j < n; j += nt) out[(size_t)k * n + j] /= piv;
        __syncthreads();
        for (int idx = tid; idx < n * n; idx += nt) {
            const int i = idx / n, j = idx % n;
            if (i != k) out[idx] -= col[i] * out[(size_t)k * n + j];
        }
        __syncthreads();
    }
    if (!bad) {
        for (int idx = tid; idx < n * n; idx += nt) {
            const int i = idx / n, j = idx % n;
            if (i < j) {
                const double s = 0.5 * (out[(size_t)i * n + j] + out[(size_t)j * n + i]);
                out[(size_t)i * n + j] = s;
                out[(size_t)j * n + i] = s;
            }
        }
    }
    if (tid == 0) *info = bad;
}

}  // namespace

void spdInverse(const double* d_a, int n, double* d_out, int* d_info, cudaStream_t stream)
{
    if (n <= 0 || n > 4096) throw std::invalid_argument("spd inverse: n must be in 1..4096");
    ct_spd_inverse_kernel<<<1, 256, sizeof(double) * (size_t)n, stream>>>(d_a, n, d_out, d_info);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e));
}

}  // namespace ctpwa
