// Seeded three-body phase-space generator on the device (toy-MC events for
// fit jobs whose samples are generated and kept on the GPU).
//
// One thread per event: the (m12) invariant mass is drawn uniformly and
// accepted with probability q(M; m12, m3) q(m12; m1, m2) / wmax (flat Dalitz
// density), the (12) system and particle 3 recoil back to back in an
// isotropic direction, particles 1 and 2 decay isotropically in the (12)
// rest frame and are boosted to the parent frame. The random numbers come
// from the counter-based Philox-4x32-10 generator (Salmon, Moraes, Dror and
// Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011) keyed by the
// seed with the event index as counter, so every event depends only on
// (seed, index): the sample does not depend on the launch shape.
#include "engine.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>

namespace ctpwa {

namespace {

struct Philox4 {
    unsigned x[4];
};

// Philox-4x32 with 10 rounds: multipliers and Weyl key increments of the
// published algorithm
__device__ __forceinline__ Philox4 philox(unsigned c0, unsigned c1, unsigned c2, unsigned c3, unsigned k0, unsigned k1)
{
    const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const unsigned hi0 = __umulhi(M0, c0), lo0 = M0 * c0;
        const unsigned hi1 = __umulhi(M1, c2), lo1 = M1 * c2;
        const unsigned n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += W0;
        k1 += W1;
    }
    return {{c0, c1, c2, c3}};
}

// uniform in (0, 1) from 32 random bits
__device__ __forceinline__ double ct_unit(unsigned b) { return ((double)b + 0.5) * (1.0 / 4294967296.0); }

__device__ __forceinline__ double ct_breakup(double m, double a, double b)
{
    const double q2 = (m * m - (a + b) * (a + b)) * (m * m - (a - b) * (a - b));
    return q2 > 0.0 ? sqrt(q2) / (2.0 * m) : 0.0;
}

__global__ void ct_phase_space_kernel(double M, double m1, double m2, double m3, double wmax, long long n,
                                      unsigned long long seed, double* __restrict__ out)
{
    const double lo = m1 + m2, hi = M - m3, twopi = 6.283185307179586;
    const unsigned k0 = (unsigned)seed, k1 = (unsigned)(seed >> 32);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned i0 = (unsigned)i, i1 = (unsigned)((unsigned long long)i >> 32);
        double m12 = 0.5 * (lo + hi), u3c = 0.5, u3p = 0.5;
        unsigned att = 0;
        // accept-reject of m12 (acceptance well above 1/2 for three-body decays;
        // after 256 rejections the last candidate is kept)
        for (; att < 256; ++att) {
            const Philox4 r = philox(i0, i1, att, 0u, k0, k1);
            m12 = lo + (hi - lo) * ct_unit(r.x[0]);
            const double w = ct_breakup(M, m12, m3) * ct_breakup(m12, m1, m2);
            u3c = ct_unit(r.x[2]);
            u3p = ct_unit(r.x[3]);
            if (ct_unit(r.x[1]) * wmax < w) break;
        }
        const Philox4 r2 = philox(i0, i1, att, 1u, k0, k1);
        // recoil of particle 3 against the (12) system in the parent frame
        const double q3 = ct_breakup(M, m12, m3);
        const double c3 = 2.0 * u3c - 1.0, s3 = sqrt(fmax(0.0, 1.0 - c3 * c3)), f3 = twopi * u3p;
        const double d3x = s3 * cos(f3), d3y = s3 * sin(f3), d3z = c3;
        // decay of (12) in its rest frame
        const double q12 = ct_breakup(m12, m1, m2);
        const double c1 = 2.0 * ct_unit(r2.x[0]) - 1.0, s1 = sqrt(fmax(0.0, 1.0 - c1 * c1)),
                     f1 = twopi * ct_unit(r2.x[1]);
        const double d1x = s1 * cos(f1), d1y = s1 * sin(f1), d1z = c1;
        const double e12 = sqrt(m12 * m12 + q3 * q3);
        const double bx = q3 * d3x / e12, by = q3 * d3y / e12, bz = q3 * d3z / e12;
        const double b2 = bx * bx + by * by + bz * bz;
        const double gamma = 1.0 / sqrt(1.0 - b2);
        const double coef = b2 > 0.0 ? (gamma - 1.0) / b2 : 0.0;
        double* o = out + i * 12;
        auto boost = [&](double E, double px, double py, double pz, double* p) {
            const double bp = bx * px + by * py + bz * pz;
            const double k = coef * bp + gamma * E;
            p[0] = gamma * (E + bp);
            p[1] = px + k * bx;
            p[2] = py + k * by;
            p[3] = pz + k * bz;
        };
        boost(sqrt(m1 * m1 + q12 * q12), q12 * d1x, q12 * d1y, q12 * d1z, o);
        boost(sqrt(m2 * m2 + q12 * q12), -q12 * d1x, -q12 * d1y, -q12 * d1z, o + 4);
        o[8] = sqrt(m3 * m3 + q3 * q3);
        o[9] = -q3 * d3x;
        o[10] = -q3 * d3y;
        o[11] = -q3 * d3z;
    }
}

double hostBreakup(double m, double a, double b)
{
    const double q2 = (m * m - (a + b) * (a + b)) * (m * m - (a - b) * (a - b));
    return q2 > 0.0 ? std::sqrt(q2) / (2.0 * m) : 0.0;
}

}  // namespace

void phaseSpace(double M, const double* masses, long long n, unsigned long long seed, double* d_out,
                cudaStream_t stream)
{
    const double m1 = masses[0], m2 = masses[1], m3 = masses[2];
    if (!(M > m1 + m2 + m3) || m1 < 0 || m2 < 0 || m3 < 0) throw std::runtime_error("phase space: M <= m1 + m2 + m3");
    if (n < 0) throw std::runtime_error("phase space: n < 0");
    if (n == 0) return;
    // maximum of the weight on a fine grid, with a 5 % margin
    const double lo = m1 + m2, hi = M - m3;
    double wmax = 0.0;
    for (int k = 1; k < 20000; ++k) {
        const double m12 = lo + (hi - lo) * k / 20000.0;
        wmax = std::max(wmax, hostBreakup(M, m12, m3) * hostBreakup(m12, m1, m2));
    }
    wmax *= 1.05;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long blocks = std::min<long long>((n + 255) / 256, (long long)sms * 16);
    ct_phase_space_kernel<<<(unsigned)blocks, 256, 0, stream>>>(M, m1, m2, m3, wmax, n, seed, d_out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e));
}

}  // namespace ctpwa
