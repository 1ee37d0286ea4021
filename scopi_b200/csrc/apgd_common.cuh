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

// Barrier words of a persistent launch (the host writes all four before the launch):
// bar[0] = arrivals, bar[1] = generation, bar[2] = error flag, bar[3] = wait limit in
// microseconds (0: kBarrierTimeoutNs).
__device__ __forceinline__ unsigned long long barrier_limit_ns(const unsigned int* bar) {
    const unsigned int us = *(volatile const unsigned int*)(bar + 3);
    return us ? (unsigned long long)us * 1000ull : kBarrierTimeoutNs;
}

// Grid-wide barrier for a cooperative launch.  A block that waits longer than the limit
// sets the error flag and returns false; every waiting block sees the flag and returns
// false too, so the kernel ends with an error status instead of hanging.  withhold: this
// block does not count itself (used once, to test that path: the barrier then never
// completes and every block gives up after the limit).
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, unsigned int nblocks, bool withhold = false) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* vgen = bar + 1;
        volatile unsigned int* verr = bar + 2;
        const unsigned int gen = *vgen;
        __threadfence();
        const unsigned int arrived = withhold ? 0u : atomicAdd(bar, 1u);
        if (!withhold && arrived == nblocks - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const unsigned long long t0 = global_ns(), limit = barrier_limit_ns(bar);
            unsigned int it = 0;
            while (*vgen == gen) {
                if (*verr) break;
                if (((++it) & 1023u) == 0 && global_ns() - t0 > limit) {
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

// Grid barrier taken by ONE thread per block (the caller synchronises its block around
// it).  bar[0] counts arrivals and only grows: it is a multiple of nblocks between
// barriers (the host zeroes it before the launch), so an arrival's target is the next
// multiple.  One atomic per block, then acquire loads.  A thread that waits longer than
// the limit (bar[3]) sets the error flag bar[2]; every waiter sees the flag and returns
// false, so the kernel ends with an error status instead of hanging.  Blocks must not mix
// it with grid_barrier after their first call (grid_barrier resets bar[0]).
__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// Split form: grid_arrive publishes this block's writes and returns the arrival target;
// the block may do independent work before grid_wait.
__device__ __forceinline__ unsigned int atom_add_release_u32(unsigned int* p, unsigned int v) {
    unsigned int old;
    asm volatile("atom.release.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
// The arrival is a release at GPU scope: it orders before it every write this thread has
// observed, which after the block barrier that precedes the call are all the block's
// writes (release is cumulative), so no separate fence is needed.  withhold: compute the
// target without counting this block (the timeout test: the barrier never completes and
// every waiter gives up after the limit).
__device__ __forceinline__ unsigned int grid_arrive(unsigned int* bar, unsigned int nblocks, bool withhold = false) {
    const unsigned int old = withhold ? ld_acquire_u32(bar) : atom_add_release_u32(bar, 1u);
    return (old / nblocks + 1u) * nblocks;
}
__device__ __forceinline__ bool grid_wait(unsigned int* bar, unsigned int target) {
    volatile unsigned int* verr = bar + 2;
    const unsigned long long limit = barrier_limit_ns(bar);
    unsigned int it = 0;
    unsigned long long t0 = 0;
    for (;;) {
        if ((int)(ld_acquire_u32(bar) - target) >= 0) break;
        if (*verr) return false;
        if (((++it) & 1023u) == 0) {
            const unsigned long long t = global_ns();
            if (t0 == 0) {
                t0 = t;
            } else if (t - t0 > limit) {
                atomicExch(bar + 2, 1u);
                return false;
            }
        }
        if (it > 32) __nanosleep(32);
    }
    // the acquire load that saw the target orders the reads after it (the block barrier that
    // follows extends that to the other threads of the block)
    return *verr == 0u;
}
__device__ __forceinline__ bool grid_arrive_wait(unsigned int* bar, unsigned int nblocks) {
    return grid_wait(bar, grid_arrive(bar, nblocks));
}

// Sum over the grid of per-block partials part[b*stride + k] (b < nb), computed by one
// warp: lane l adds blocks l, l+32, ... in order, then a fixed shuffle tree.  Every block
// gets the same bits.  The result is in lane 0.
template <int NP>
__device__ __forceinline__ void warp_grid_sum(const double* part, unsigned int nb, int stride, double* t) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < NP; ++k) t[k] = 0.0;
    for (unsigned int b = lane; b < nb; b += 32)
#pragma unroll
        for (int k = 0; k < NP; ++k) t[k] += __ldcg(part + (size_t)b * stride + k);
#pragma unroll
    for (int k = 0; k < NP; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t[k] += __shfl_down_sync(0xffffffffu, t[k], o);
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

// Block sum whose result only thread 0 needs (it is in thread 0's v[] on return): one
// block barrier.  The caller synchronises the block before the next call, which reuses
// the staging array.  Fixed summation order (deterministic).
template <int NP>
__device__ __forceinline__ void block_reduce_t0(double* v) {
    __shared__ double sh[NP][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[k][warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            double x = lane < nw ? sh[k][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[k] = x;
        }
    }
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

// Backtracking test of apgd.hpp:172-182, F(l+) >= F(y) + g(y).d + L/2 |d|^2 with d = l+ - y.
// FP64 evaluates it as the reference does.  For a quadratic F the test is exactly
// d^T Q d >= L |d|^2; FP32 iterations use that form (dQd = dt^2 sum_p m |u(l+) - u(y)|^2),
// since F(l+) - F(y) in FP32 carries round-off of the size of F itself and fails the
// test spuriously once the steps are small, which collapses alpha and stalls the solve.
template <typename T>
__device__ __forceinline__ bool sufficient_decrease_fails(double F_lp, double Fy, double gd, double dd, double dQd,
                                                          double lipsch) {
    if (sizeof(T) == 4) return dQd >= lipsch * dd;
    return F_lp >= Fy + gd + 0.5 * lipsch * dd;
}

// First projected-gradient direction of a solve at its cold start (lambda = 0, or delta = 0
// for a correction with offset `shift`): d = -g where the bound lets it move.  The
// Rayleigh quotient d^T Q d / |d|^2 then sets the initial step (see the kernels).
template <typename T>
__device__ __forceinline__ T first_descent(T g, const double* shift, long long m) {
    if (shift) return (shift[m] > 0.0 || g < (T)0) ? -g : (T)0;
    return g < (T)0 ? -g : (T)0;
}
// Initial Lipschitz estimate: 1.5 x the curvature along d (d^T Q d = dt^2 sum_p
// w_p . M^-1 w_p with w = B^T d).  The reference starts every solve from the fixed
// alpha = 0.05 (apgd.hpp:120) and grows it by 1/0.97 per accepted iteration; for the
// problems here 1/L is many orders of magnitude larger, so most of its iterations are
// that ramp, and its first step alpha*|g| can fall below the tolerance so that the solve
// stops at once with a resting contact still open by ~ g dt^2.
__device__ __forceinline__ bool initial_lipschitz(double dd, double wmw, double dt2, double& lipsch) {
    if (!(dd > 0.0) || !(wmw > 0.0)) return false;
    const double l = 1.5 * dt2 * wmw / dd;
    if (!isfinite(l) || !(l > 0.0)) return false;
    lipsch = l;
    return true;
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
