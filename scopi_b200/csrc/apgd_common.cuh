// apgd_common.cuh -- pieces shared by the persistent APGD kernels: bounded grid barrier,
// fixed-order block reductions, vector loads and the friction-cone projection.
#pragma once
#include <math.h>

#include "kernels.cuh"

namespace scopi_gpu {
namespace apgdc {

constexpr int kThreadsA = 256;
constexpr unsigned long long kBarrierTimeoutNs = 20ull * 1000ull * 1000ull * 1000ull;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier for a cooperative launch.  bar[0] = arrivals, bar[1] = generation,
// bar[2] = error flag.  A block that waits longer than kBarrierTimeoutNs sets the flag and
// returns false; every waiting block sees the flag and returns false too, so the kernel
// ends with an error status instead of hanging.
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, unsigned int nblocks) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* vgen = bar + 1;
        volatile unsigned int* verr = bar + 2;
        const unsigned int gen = *vgen;
        __threadfence();
        const unsigned int arrived = atomicAdd(bar, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            unsigned int it = 0;
            while (*vgen == gen) {
                if (*verr) break;
                if (((++it) & 1023u) == 0 && global_ns() - t0 > kBarrierTimeoutNs) {
                    atomicExch(bar + 2, 1u);
                    break;
                }
                __nanosleep(20);
            }
        }
        __threadfence();
        s_ok = (*verr == 0u);
    }
    __syncthreads();
    return s_ok != 0;
}

// Fixed-order sum of NP doubles over the block (up to 1024 threads); the result is
// returned in every thread.
template <int NP>
__device__ __forceinline__ void block_sum(double* v) {
    __shared__ double sh[32][NP];
    __shared__ double tot[NP];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[warp][k] = x;
    }
    __syncthreads();
    if (threadIdx.x < NP) {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += sh[w][threadIdx.x];
        tot[threadIdx.x] = s;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NP; ++k) v[k] = tot[k];
    __syncthreads();
}

// Every block sums the per-block partials part[b*stride + k] (b < nb) in the same order.
template <int NP>
__device__ __forceinline__ void grid_sum(const double* part, unsigned int nb, int stride, double* t) {
#pragma unroll
    for (int k = 0; k < NP; ++k) t[k] = 0.0;
    for (unsigned int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NP; ++k) t[k] += __ldcg(part + (size_t)b * stride + k);
    block_sum<NP>(t);
}

// LagrangeMultiplier<Friction>::projection, include/scopi/solvers/lagrange_multiplier.hpp:243-268
template <int DIM>
__device__ __forceinline__ void cone_project(double* l, const double* n, double mu) {
    double ln = 0.0;
    for (int d = 0; d < DIM; ++d) ln += l[d] * n[d];
    double lt[3] = {0, 0, 0};
    for (int d = 0; d < DIM; ++d) lt[d] = l[d] - ln * n[d];
    double nrm = 0.0;
    for (int d = 0; d < DIM; ++d) nrm += lt[d] * lt[d];
    nrm = sqrt(nrm);
    if (nrm > mu * ln) {
        if (ln <= -mu * nrm) {
            for (int d = 0; d < DIM; ++d) l[d] = 0.0;
        } else {
            const double nn = (mu * mu) * (nrm + ln / mu) / (mu * mu + 1);
            const double nln = nn / mu;
            for (int d = 0; d < DIM; ++d) l[d] = nn * (lt[d] / nrm) + nln * n[d];
        }
    }
}

// l+ == y bit for bit: the reference compares F(l+) >= F(y) on identical vectors, doubles
// L (l+ cannot move: -g lies in the normal cone at y) until 0.5*L*0 turns NaN at L = inf,
// then accepts with alpha = 0 (apgd.hpp:172-182).
__device__ __forceinline__ void overflow_cascade(double& lipsch, double& alpha, long long& nbt) {
    while (isfinite(lipsch)) {
        lipsch *= 2;
        ++nbt;
    }
    alpha = 1. / lipsch;
}

}  // namespace apgdc
}  // namespace scopi_gpu
