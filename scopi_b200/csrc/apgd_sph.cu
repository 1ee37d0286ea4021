// apgd_sph.cu -- persistent APGD for the normal-only problems (NoFriction, Viscous) on
// contacts whose lever arms are parallel to the normal (sphere-sphere, sphere-plane,
// sphere-segment: p_i - x_i = -/+ r_i n), where the rotational terms of the contact
// Jacobian, R^T (r x n), vanish identically.  A contact's row of B is then n^T on the
// two bodies' translational velocities:
//     (B u)_c = n_c . (u_i - u_j),     (B^T l)_p = sum_{c ~ p} +-l_c n_c.
// Same iteration, branch logic and stopping rule as the generic kernel (apgd.cu), i.e.
// apgd::operator() of include/scopi/solvers/apgd.hpp:148-221, with the data cut to
// what this row shape needs:
//   per contact : (ci, cj) int2 + (n, c) packed in one 16/32-byte record, l, l_prev;
//   per incidence of a body: (+-n, contact index) in one record;
//   per body    : u(y) gathered once (u(y_next) = u(l+) + beta (u(l+) - u(l)) is formed in
//                 the particle pass, the restart test being reduced after the first barrier).
#include <algorithm>
#include <cstdio>
#include <mutex>

#include "../../include/scopi_gpu.h"
#include "apgd_common.cuh"

namespace scopi_gpu {

static long long g_sph_launches = 0;
long long apgd_sph_launches() { return g_sph_launches; }

namespace {
using namespace apgdc;

__device__ __forceinline__ float4 ld4(const float4* p) { return *p; }
__device__ __forceinline__ dvec4 ld4(const dvec4* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = q[0], b = q[1];
    return dvec4{a.x, a.y, b.x, b.y};
}
__device__ __forceinline__ float4 ld4cg(const float4* p) { return __ldcg(p); }
__device__ __forceinline__ dvec4 ld4cg(const dvec4* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldcg(q), b = __ldcg(q + 1);
    return dvec4{a.x, a.y, b.x, b.y};
}
__device__ __forceinline__ void st4(float4* p, float x, float y, float z) { *p = make_float4(x, y, z, 0.f); }
__device__ __forceinline__ void st4(dvec4* p, double x, double y, double z) {
    double2* q = reinterpret_cast<double2*>(p);
    q[0] = make_double2(x, y);
    q[1] = make_double2(z, 0.0);
}
__device__ __forceinline__ int idx_of(float w) { return __float_as_int(w); }
__device__ __forceinline__ int idx_of(double w) { return (int)__double_as_longlong(w); }

// ---- asynchronous global -> shared copies (cp.async).  Each thread stages only the
// records it consumes itself, so a stage needs no block barrier: cp.async.wait_group
// makes the thread's own copies visible to it.  src-size 0 zero-fills the slot without
// reading (tails past the end; the source pointer is then the array base).
__device__ __forceinline__ unsigned sm_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp16(void* dst, const void* src, bool on) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sm_addr(dst)), "l"(src), "r"(on ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp8(void* dst, const void* src, bool on) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sm_addr(dst)), "l"(src), "r"(on ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp4(void* dst, const void* src, bool on) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sm_addr(dst)), "l"(src), "r"(on ? 4 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_val(float* d, const float* s, bool on) { cp4(d, s, on); }
__device__ __forceinline__ void cp_val(double* d, const double* s, bool on) { cp8(d, s, on); }
__device__ __forceinline__ void cp_vec(float4* d, const float4* s, bool on) { cp16(d, s, on); }
__device__ __forceinline__ void cp_vec(dvec4* d, const dvec4* s, bool on) {
    cp16(d, s, on);
    cp16(reinterpret_cast<double2*>(d) + 1, reinterpret_cast<const double2*>(s) + 1, on);
}

template <typename T>
struct SphArgs {
    int nin, na;
    const int2* cij;
    const V4<T>* nc;
    const int* slot;
    const double* shift;
    const int* inc_ptr;
    const V4<T>* inc;
    const T* invm;  // 1/m per active body, contiguous
    T* lam0;
    T* lam1;
    T* lam2;
    V4<T>* u0;
    V4<T>* u1;
    V4<T>* u2;
    V4<T>* u3;
    double* partials;
    unsigned int* bar;
    ApgdResult* result;
    const Sizes* sizes;
    double alpha, tol, dt2;
    long long max_ite;
    int dynamic;
    int curvature_start;
    int stall;  // block 0 skips its first barrier arrival (test of the barrier limit)
};

template <typename T>
__device__ __forceinline__ T pick(int k, T a, T b, T c) {
    return k == 0 ? a : (k == 1 ? b : c);
}
template <typename T>
__device__ __forceinline__ T pick4(int k, T a, T b, T c, T d) {
    return k == 0 ? a : (k == 1 ? b : (k == 2 ? c : d));
}

// one multiplier of the contact pass (lm, lpm: its current and previous values)
template <typename T>
__device__ __forceinline__ void mult_update_v(const SphArgs<T>& A, long long m, T qy, T cc, T lm, T lpm, T* lnew,
                                              T beta, bool use_prev, bool bt, double alpha, double* s) {
    const T y = use_prev ? lm + beta * (lm - lpm) : lm;
    const T gm = qy + cc;
    T lp;
    if (A.shift) {
        const double sh = A.shift[m];
        double z = sh + ((double)y - alpha * (double)gm);
        z = z > 0.0 ? z : 0.0;
        lp = (T)(z - sh);
    } else {
        const T z = y - (T)alpha * gm;
        lp = z > (T)0 ? z : (T)0;
    }
    lnew[m] = lp;
    const double dly = (double)lp - (double)y, dll = (double)lp - (double)lm;
    // g.d, c.l+ and F(y) serve the reference's backtracking test (FP64 only; the FP32 test
    // is the curvature form, which reads |d|^2 and the particle pass's d^T Q d)
    if (sizeof(T) == 8) {
        s[0] += (double)gm * dly;
        s[2] += (double)cc * (double)lp;
        if (!bt) s[3] += (double)y * (0.5 * (double)qy + (double)cc);
    }
    s[1] += dly * dly;
    s[4] += dll * dll;
    s[5] += (double)gm * dll;
    s[6] += (double)lp * (double)lp;
}
template <typename T>
__device__ __forceinline__ void mult_update(const SphArgs<T>& A, long long m, T qy, T cc, const T* lam, const T* lprev,
                                            T* lnew, T beta, bool use_prev, bool bt, double alpha, double* s) {
    mult_update_v<T>(A, m, qy, cc, lam[m], use_prev ? lprev[m] : (T)0, lnew, beta, use_prev, bt, alpha, s);
}

// Loop-carried scalars of the iteration (block-uniform) live in shared memory and are
// updated by thread 0, so the registers go to the two passes.
struct SphState {
    double alpha, lipsch, theta, beta, beta_n, theta1, Fy, last_step, lgood;
    double tk[4];  // g.d, |d|^2, c.l+ and |l+|^2 of the candidate (contact pass sums)
    long long ite, nbt, nrs;
    int il, ip, in_, jL, jN, jY, jYN, parity, bt, use_prev, restart, done, conv, err;
};

// One block per SM (SphShape): FP32 768 threads (80 registers, no spills), FP64 512 (128).
// Per-phase globaltimer stamps at 1M spheres (3.0M contacts): FP32 70.6 us per iteration
// (contact pass 30.6, particle pass 31.2, barriers and sums 8.1) against 77.1 with 1024
// threads and the gathers one trip ahead; FP64 110.9 against 117.1.  Shared memory and L1
// share the SM: the particle pass's incidence records live in L1, so deeper stages that
// grow the shared memory slow it down (FP64 with 5 contact stages: 115.1 us).
//
// Both passes stream their per-item records through a cp.async pipeline in dynamic shared
// memory (the passes are separated by grid barriers, so they share it):
//   contact pass, GC stages, per contact : (ci, cj), (n, c), l, l_prev  -- 32 B (FP32), 56 B (FP64)
//   particle pass, GP stages, per body   : inc_ptr[p], inc_ptr[p+1], 1/m, u(l) and (FP32) u(y)
// and the gathers that depend on a staged record (u(y) of the contact's bodies) are issued
// GD trips ahead.  The incidence records stay on plain loads: a body's records share L1
// lines, which an L1-bypassing copy would fetch again from L2 for every record.
// Launch shape per precision: threads per block, contact-pass stages GC (the u(y) gathers
// of trip k + GD are issued during trip k: an L2 round trip is about one trip long),
// particle-pass stages GP.
template <typename T>
struct SphShape;
template <>
struct SphShape<float> {
    static constexpr int threads = 768, GC = 5, GD = 2, GP = 4;
};
template <>
struct SphShape<double> {
    static constexpr int threads = 512, GC = 4, GD = 2, GP = 4;
};
template <typename T>
struct SphOcc {
    static constexpr int threads = SphShape<T>::threads;
    static constexpr int GC = SphShape<T>::GC, GD = SphShape<T>::GD, GP = SphShape<T>::GP;
    static constexpr size_t contact_bytes = (size_t)GC * threads * (sizeof(int2) + sizeof(V4<T>) + 2 * sizeof(T));
    static constexpr size_t particle_bytes =
        (size_t)GP * threads * ((sizeof(T) == 4 ? 2 : 1) * sizeof(V4<T>) + sizeof(T) + 2 * sizeof(int));
    static constexpr size_t smem = contact_bytes > particle_bytes ? contact_bytes : particle_bytes;
};

template <typename T, int DIM, int PROB>
__global__ void __launch_bounds__(SphOcc<T>::threads, 1) k_apgd_sph(SphArgs<T> A) {
    __shared__ SphState S;
    extern __shared__ __align__(32) unsigned char sph_dyn[];
    constexpr int GC = SphOcc<T>::GC, GD = SphOcc<T>::GD, GP = SphOcc<T>::GP;
    static_assert(GD >= 1 && GD <= GC - 2, "the gathered records must be in the prologue's stages");
    const int NT = blockDim.x, tid = threadIdx.x;
    // contact-pass stages [GC][NT] of each field
    V4<T>* s_nc = reinterpret_cast<V4<T>*>(sph_dyn);
    int2* s_ij = reinterpret_cast<int2*>(s_nc + GC * NT);
    T* s_l = reinterpret_cast<T*>(s_ij + GC * NT);
    T* s_lp = s_l + GC * NT;
    // particle-pass stages [GP][NT] (same memory)
    V4<T>* s_ul = reinterpret_cast<V4<T>*>(sph_dyn);
    V4<T>* s_uy = s_ul + GP * NT;  // FP32 only
    T* s_im = reinterpret_cast<T*>(s_ul + (sizeof(T) == 4 ? 2 : 1) * GP * NT);
    int* s_p0 = reinterpret_cast<int*>(s_im + GP * NT);
    int* s_p1 = s_p0 + GP * NT;
    if (threadIdx.x == 0) {
        S.alpha = A.alpha;
        S.lipsch = 1.0 / A.alpha;
        S.lgood = S.lipsch;
        S.theta = 1.0;
        S.beta = 0.0;
        S.beta_n = 0.0;
        S.theta1 = 1.0;
        S.Fy = 0.0;
        S.last_step = 0.0;
        S.ite = S.nbt = S.nrs = 0;
        S.il = 0; S.ip = 1; S.in_ = 2;           // lambda buffers: current, previous, candidate
        S.jL = 0; S.jN = 1; S.jY = 2; S.jYN = 3;  // u buffers: u(l), u(candidate), u(y), u(next y)
        S.parity = 0;
        S.bt = 0;
        S.use_prev = 0;
        S.restart = 0;
        S.done = 0;
        S.conv = 0;
        S.err = 0;
    }
    __syncthreads();
    const int C = A.sizes->C;
    const unsigned int nb = gridDim.x;
    // Trip k of a thread handles item base + k*S (the grid-stride order) in both passes.
    const long long S_ = (long long)gridDim.x * NT, base = (long long)blockIdx.x * NT + tid;
    const long long ntrip_c = ((long long)C - (long long)blockIdx.x * NT + S_ - 1) / S_;
    const long long ntrip_p = ((long long)A.na - (long long)blockIdx.x * NT + S_ - 1) / S_;
    // First stages of each pass are issued before the grid barrier that precedes the pass
    // when they do not depend on it: a contact's geometry (n, c), (ci, cj), and a body's
    // inc_ptr, 1/m, u(l), u(y).  Uncommitted copies join the next commit group.
    auto issue_geom = [&](int k) {
        const int sl = (k % GC) * NT + tid;
        const long long c = base + k * S_;
        const bool on = k < ntrip_c && c < C;
        const long long cc = on ? c : 0;
        cp_vec(s_nc + sl, A.nc + cc, on);
        cp8(s_ij + sl, A.cij + cc, on);
    };
    auto issue_body = [&](long long k, const V4<T>* uL, const V4<T>* uY, bool with_ul) {
        const int sl = (int)(k % GP) * NT + tid;
        const long long p = base + k * S_;
        const bool on = k < ntrip_p && p < A.na;
        const long long pp = on ? p : 0;
        cp4(s_p0 + sl, A.inc_ptr + pp, on);
        cp4(s_p1 + sl, A.inc_ptr + pp + 1, on);
        cp_val(s_im + sl, A.invm + pp, on);
        cp_vec(s_ul + sl, uL + pp, on && with_ul);
        if (sizeof(T) == 4) cp_vec(s_uy + sl, uY + pp, on);
        cp_commit();
    };
    bool geom_issued = false;
    bool withhold = A.stall != 0 && blockIdx.x == 0;
    if (A.curvature_start) {
        // initial step from the curvature along the first descent direction d (stored in
        // the candidate buffer, which the first contact pass overwrites); partial-sum
        // regions 1 and 3 are first reused by the second iteration, after two barriers
        T* dbuf = A.lam2;
        double a2[2] = {0.0, 0.0};
        GRID_STRIDE(c, C) {
            const T cc = ld4(A.nc + c).w;
            const T d = first_descent<T>(cc, A.shift, c);
            dbuf[c] = d;
            a2[0] += (double)d * (double)d;
            if (PROB == kViscous) {
                const int sl = A.slot[c];
                if (sl >= 0) {
                    const T d2 = first_descent<T>(-cc, A.shift, sl);
                    dbuf[sl] = d2;
                    a2[0] += (double)d2 * (double)d2;
                }
            }
        }
        block_sum<2>(a2);
        if (threadIdx.x == 0) A.partials[(size_t)1 * nb * 8 + blockIdx.x * 8] = a2[0];
        bool ok = grid_barrier(A.bar, nb, withhold);
        withhold = false;
        double wm[2] = {0.0, 0.0};
        if (ok) GRID_STRIDE(p, A.na) {
            T w0 = 0, w1 = 0, w2 = 0;
            for (int k = A.inc_ptr[p]; k < A.inc_ptr[p + 1]; ++k) {
                const V4<T> e = ld4(A.inc + k);
                const int ci = idx_of(e.w);
                T mu = __ldcg(dbuf + ci);
                if (PROB == kViscous) {
                    const int sl = A.slot[ci];
                    if (sl >= 0) mu -= __ldcg(dbuf + sl);
                }
                w0 += mu * e.x;
                w1 += mu * e.y;
                if (DIM == 3) w2 += mu * e.z;
            }
            const double im = (double)A.invm[p];
            wm[0] += im * ((double)w0 * w0 + (double)w1 * w1 + (double)w2 * w2);
        }
        block_sum<2>(wm);
        if (threadIdx.x == 0) A.partials[(size_t)3 * nb * 8 + blockIdx.x * 8] = wm[0];
        if (ok) ok = grid_barrier(A.bar, nb);
        double t1[1] = {0.0}, t3[1] = {0.0};
        if (ok) {
            grid_sum<1>(A.partials + (size_t)1 * nb * 8, nb, 8, t1);
            grid_sum<1>(A.partials + (size_t)3 * nb * 8, nb, 8, t3);
        }
        if (threadIdx.x == 0) {
            double l;
            if (ok && initial_lipschitz(t1[0], t3[0], A.dt2, l)) {
                S.lipsch = l;
                S.alpha = 1.0 / l;
                S.lgood = l;
            }
            if (!ok) {
                S.err = 1;
                S.done = 1;
            }
        }
        __syncthreads();
    }
    for (;;) {
        if (S.done) break;
        const double alpha = S.alpha;
        const bool bt = S.bt != 0, use_prev = S.use_prev != 0;
        const T beta = (T)S.beta;
        const T* lam = pick(S.il, A.lam0, A.lam1, A.lam2);
        const T* lprev = pick(S.ip, A.lam0, A.lam1, A.lam2);
        T* lnew = pick(S.in_, A.lam0, A.lam1, A.lam2);
        const V4<T>* uY = pick4(S.jY, A.u0, A.u1, A.u2, A.u3);
        double* part = A.partials + (size_t)S.parity * nb * 8;
        double* part2 = A.partials + (size_t)(2 + S.parity) * nb * 8;
        {
            double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            // ---- contact pass: g = dt^2 n.(u_i(y) - u_j(y)) + c, l+ = P(y - alpha g)
            const int ntrip = (int)ntrip_c;
            auto issue_lam = [&](int k) {
                const int sl = (k % GC) * NT + tid;
                const long long c = base + (long long)k * S_;
                const bool on = k < ntrip && c < C;
                const long long cc = on ? c : 0;
                cp_val(s_l + sl, lam + cc, on);
                cp_val(s_lp + sl, lprev + cc, on && use_prev);
            };
            auto issue = [&](int k) {
                issue_geom(k);
                issue_lam(k);
                cp_commit();
            };
            // u(y) of the contact's two bodies (written by other blocks: L2 loads)
            auto gather = [&](int k, T* g) {
                const int sl = (k % GC) * NT + tid;
                const int2 ij = s_ij[sl];
                const bool on = k < ntrip && base + (long long)k * S_ < C;
                V4<T> ui, uj;
                ui.x = ui.y = ui.z = uj.x = uj.y = uj.z = (T)0;
                if (on && ij.x >= A.nin) ui = ld4cg(uY + (ij.x - A.nin));
                if (on && ij.y >= A.nin) uj = ld4cg(uY + (ij.y - A.nin));
                g[0] = ui.x; g[1] = ui.y; g[2] = ui.z;
                g[3] = uj.x; g[4] = uj.y; g[5] = uj.z;
            };
            // prologue: the geometry of stages 0..GC-2 in one group (issued before the
            // last barrier when geom_issued), then their multipliers one group per stage
            if (!geom_issued)
#pragma unroll 1
                for (int k = 0; k < GC - 1; ++k) issue_geom(k);
            cp_commit();
            geom_issued = false;
#pragma unroll 1
            for (int k = 0; k < GC - 1; ++k) {
                issue_lam(k);
                cp_commit();
            }
            cp_wait<GC - 2>();
            // trip k: commit stage k + GC - 1, wait for stage k + GD, gather trip k + GD's
            // u(y), then compute trip k with the u(y) gathered GD trips ago.  Three register
            // sets in rotation (the loop unrolled by three) so that no gather is forced to
            // complete before its own trip.
            static_assert(GD == 2, "three gather sets in rotation");
            auto trip = [&](int k, const T* g, T* fill) {
                issue(k + GC - 1);
                cp_wait<GC - 1 - GD>();  // stages up to k + GD have landed
                gather(k + GD, fill);
                const long long c = base + (long long)k * S_;
                if (k < ntrip && c < C) {
                    const int sl = (k % GC) * NT + tid;
                    const V4<T> nc = s_nc[sl];
                    // bodies below nin (obstacles) gathered as zeros: same sum as skipping them
                    T qy = 0;
                    qy += nc.x * g[0] + nc.y * g[1] + (DIM == 3 ? nc.z * g[2] : (T)0);
                    qy -= nc.x * g[3] + nc.y * g[4] + (DIM == 3 ? nc.z * g[5] : (T)0);
                    qy *= (T)A.dt2;
                    mult_update_v<T>(A, c, qy, nc.w, s_l[sl], s_lp[sl], lnew, beta, use_prev, bt, alpha, s);
                    if (PROB == kViscous) {
                        const int sv = A.slot[c];
                        if (sv >= 0) mult_update<T>(A, sv, -qy, -nc.w, lam, lprev, lnew, beta, use_prev, bt, alpha, s);
                    }
                }
            };
            T g0[6], g1[6], g2[6];
            gather(0, g0);
            gather(1, g1);
#pragma unroll 1
            for (int k = 0; k < ntrip; k += 3) {
                trip(k, g0, g2);
                trip(k + 1, g1, g0);
                trip(k + 2, g2, g1);
            }
            cp_wait<0>();
            // block partials to thread 0, grid barrier and grid sum in warp 0 only
            // FP32 needs four of the sums (|d|^2, |l+ - l|^2, g.(l+ - l), |l+|^2): they are
            // reduced packed, in the first four slots of the block's record
            constexpr int NS = sizeof(T) == 4 ? 4 : 8;
            double r[NS];
            if (NS == 4) {
                r[0] = s[1];
                r[1 % NS] = s[4];
                r[2 % NS] = s[5];
                r[3 % NS] = s[6];
            } else {
#pragma unroll
                for (int k = 0; k < NS; ++k) r[k] = s[k];
            }
            block_reduce_t0<NS>(r);
            unsigned int target = 0;
            if (tid == 0) {
                for (int k = 0; k < NS; ++k) part[blockIdx.x * 8 + k] = r[k];
                target = grid_arrive(A.bar, nb, withhold);
            }
            withhold = false;
            // every thread is past its contact loop: the particle pass's first stages fill
            // the shared memory while the barrier waits (u(l) copied whatever beta is)
            {
                const V4<T>* uL0 = pick4(S.jL, A.u0, A.u1, A.u2, A.u3);
#pragma unroll 1
                for (int k = 0; k < GP - 1; ++k) issue_body(k, uL0, uY, true);
            }
            if (tid < 32) {
                bool ok = true;
                if (tid == 0) ok = grid_wait(A.bar, target);
                ok = __shfl_sync(0xffffffffu, ok, 0) != 0;
                __syncwarp();  // the lanes' partial loads come after lane 0's acquire
                double t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                {
                    double tt[NS];
                    warp_grid_sum<NS>(part, nb, 8, tt);
                    if (NS == 4) {
                        t[1] = tt[0];
                        t[4] = tt[1 % NS];
                        t[5] = tt[2 % NS];
                        t[6] = tt[3 % NS];
                    } else {
#pragma unroll
                        for (int k = 0; k < NS; ++k) t[k] = tt[k];
                    }
                }
                if (tid == 0) {
                    if (!ok) {
                        S.err = 1;
                        S.done = 1;
                    }
                    // momentum for the next y if this candidate is accepted (apgd.hpp:196-206)
                    const double th = S.theta;
                    S.theta1 = 0.5 * (th * sqrt(4 + th * th) - th * th);
                    S.restart = (A.dynamic && t[5] > 0) ? 1 : 0;
                    S.beta_n = S.restart ? 0.0 : th * (1 - th) / (th * th + S.theta1);
                    if (!bt) S.Fy = t[3];
                    // the scalars the decision needs after the second pass
                    S.last_step = t[4];
                    S.tk[0] = t[0];
                    S.tk[1] = t[1];
                    S.tk[2] = t[2];
                    S.tk[3] = t[6];
                }
            }
        }
        __syncthreads();
        if (S.err) break;
        {
            // ---- particle pass: w = B^T l+, u = M^-1 w, u(next y)
            V4<T>* uL = pick4(S.jL, A.u0, A.u1, A.u2, A.u3);
            V4<T>* uN = pick4(S.jN, A.u0, A.u1, A.u2, A.u3);
            V4<T>* uYN = pick4(S.jYN, A.u0, A.u1, A.u2, A.u3);
            const T bn_ = (T)S.beta_n;
            double sw = 0.0, sq = 0.0;
            // one body per thread; its incidence records, then the l+ gathers they index,
            // are issued in batches so several loads are in flight per thread
            constexpr int KB = 4;
            const long long ntrip = ntrip_p;
            // stages 0..GP-2 were issued before the barrier
#pragma unroll 1
            for (long long kt = 0; kt < ntrip; ++kt) {
                issue_body(kt + GP - 1, uL, uY, bn_ != (T)0);
                cp_wait<GP - 1>();  // stage kt has landed
                const long long p = base + kt * S_;
                if (p >= A.na) continue;
                const int sl = (int)(kt % GP) * NT + tid;
                T w0 = 0, w1 = 0, w2 = 0;
                const int k0 = s_p0[sl], k1 = s_p1[sl];
                for (int kb = k0; kb < k1; kb += KB) {
                    T ex[KB], ey[KB], ez[KB], mu[KB];
                    int ci[KB];
#pragma unroll
                    for (int q = 0; q < KB; ++q) {
                        ex[q] = ey[q] = ez[q] = mu[q] = (T)0;
                        ci[q] = -1;
                        if (kb + q < k1) {
                            const V4<T> e = ld4(A.inc + kb + q);
                            ex[q] = e.x;
                            ey[q] = e.y;
                            ez[q] = e.z;
                            ci[q] = idx_of(e.w);
                        }
                    }
#pragma unroll
                    for (int q = 0; q < KB; ++q)
                        if (ci[q] >= 0) {
                            mu[q] = __ldcg(lnew + ci[q]);
                            if (PROB == kViscous) {
                                const int sv = A.slot[ci[q]];
                                if (sv >= 0) mu[q] -= __ldcg(lnew + sv);
                            }
                        }
#pragma unroll
                    for (int q = 0; q < KB; ++q) {
                        w0 += mu[q] * ex[q];
                        w1 += mu[q] * ey[q];
                        if (DIM == 3) w2 += mu[q] * ez[q];
                    }
                }
                const T im = s_im[sl];
                const T n0 = im * w0, n1 = im * w1, n2 = im * w2;
                st4(uN + p, n0, n1, n2);
                // w.u gives F(l+) for the reference's test (FP64); FP32 tests the curvature
                if (sizeof(T) == 8) sw += (double)w0 * (double)n0 + (double)w1 * (double)n1 + (double)w2 * (double)n2;
                if (sizeof(T) == 4) {
                    // m |u(l+) - u(y)|^2: the curvature d^T Q d / dt^2 along d = l+ - y
                    const V4<T> uy = s_uy[sl];
                    const double d0 = (double)n0 - (double)uy.x, d1 = (double)n1 - (double)uy.y,
                                 d2 = (double)n2 - (double)uy.z;
                    sq += (d0 * d0 + d1 * d1 + d2 * d2) / (double)im;
                }
                if (bn_ != (T)0) {
                    const V4<T> ul = s_ul[sl];
                    st4(uYN + p, n0 + bn_ * (n0 - ul.x), n1 + bn_ * (n1 - ul.y), n2 + bn_ * (n2 - ul.z));
                } else {
                    st4(uYN + p, n0, n1, n2);
                }
            }
            cp_wait<0>();
            // FP64 reduces w.u (slot 0), FP32 the curvature (slot 1)
            constexpr int NQ = sizeof(T) == 4 ? 1 : 2;
            double sw8[2] = {sizeof(T) == 4 ? sq : sw, sq};
            block_reduce_t0<NQ>(sw8);
            unsigned int target2 = 0;
            if (tid == 0) {
                if (NQ == 1) {
                    part2[blockIdx.x * 8 + 1] = sw8[0];
                } else {
                    part2[blockIdx.x * 8] = sw8[0];
                    part2[blockIdx.x * 8 + 1] = sw8[1 % NQ];
                }
                target2 = grid_arrive(A.bar, nb);
            }
            // the next iteration's first contact geometry, while the barrier waits
#pragma unroll 1
            for (int k = 0; k < GC - 1; ++k) issue_geom(k);
            geom_issued = true;
            bool ok = true;
            double t6[2];
            if (tid < 32) {
                if (tid == 0) ok = grid_wait(A.bar, target2);
                ok = __shfl_sync(0xffffffffu, ok, 0) != 0;
                __syncwarp();
                if (NQ == 1) {
                    t6[0] = 0.0;
                    warp_grid_sum<1>(part2 + 1, nb, 8, t6 + 1);
                } else {
                    warp_grid_sum<2>(part2, nb, 8, t6);
                }
            }
            if (tid == 0 && !ok) {
                S.err = 1;
                S.done = 1;
            } else if (tid == 0) {
                const double* tk = S.tk;
                S.parity ^= 1;
                const double F_lp = 0.5 * A.dt2 * t6[0] + tk[2];
                bool accept = true;
                if (A.dynamic && tk[1] == 0.0) {
                    double lip = S.lipsch, al = S.alpha;
                    long long nbt = S.nbt;
                    overflow_cascade(lip, al, nbt);
                    S.lipsch = lip;
                    S.alpha = al;
                    S.nbt = nbt;
                } else if (A.dynamic && sufficient_decrease_fails<T>(F_lp, S.Fy, tk[0], tk[1], A.dt2 * t6[1],
                                                                      S.lipsch)) {
                    S.lipsch *= 2;  // backtracking, apgd.hpp:172-182
                    S.alpha = 1. / S.lipsch;
                    S.bt = 1;
                    ++S.nbt;
                    accept = false;
                }
                if (accept) {
                    ++S.ite;
                    S.bt = 0;
                    if (isfinite(S.lipsch)) S.lgood = S.lipsch;
                    S.last_step = sqrt(S.last_step);
                    double tol = A.tol;
                    if (sizeof(T) == 4) {
                        // FP32 iterations stall at their rounding floor; the FP64 correction recovers the rest
                        const double floor32 = 4.0 * 1.1920929e-7 * sqrt(tk[3]);
                        if (floor32 > tol) tol = floor32;
                    }
                    int tmp = S.ip; S.ip = S.il; S.il = S.in_; S.in_ = tmp;
                    tmp = S.jL; S.jL = S.jN; S.jN = tmp;
                    tmp = S.jY; S.jY = S.jYN; S.jYN = tmp;
                    if (S.last_step < tol) {
                        S.conv = 1;
                        S.done = 1;
                    } else {
                        S.beta = S.beta_n;
                        S.theta = S.restart ? 1.0 : S.theta1;
                        if (S.restart) ++S.nrs;
                        if (A.dynamic) {
                            S.lipsch *= 0.97;
                            S.alpha = 1. / S.lipsch;
                        }
                        S.use_prev = (S.beta != 0.0) ? 1 : 0;
                        if (S.ite >= A.max_ite) S.done = 1;
                    }
                }
            }
            __syncthreads();
            if (S.done) break;
        }
    }
    // copies issued for an iteration that did not run (wait_group does not cover
    // uncommitted copies: commit them first)
    cp_commit();
    cp_wait<0>();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        A.result->iterations = S.ite;
        A.result->backtracks = S.nbt;
        A.result->restarts = S.nrs;
        A.result->converged = S.conv;
        A.result->lam_buf = S.il;
        A.result->u_buf = S.jL;
        A.result->error = S.err;
        A.result->last_step = S.last_step;
        A.result->lipsch = S.lgood;
    }
}

// ------------------------------------------------------------------ packing
__global__ void k_pack_cij(const int* ci, const int* cj, int2* cij, const Sizes* sizes) {
    GRID_STRIDE(c, sizes->C) { cij[c] = make_int2(ci[c], cj[c]); }
}
template <typename T>
__global__ void k_pack_nc(const double* bn, const double* cv, V4<T>* nc, const Sizes* sizes) {
    GRID_STRIDE(c, sizes->C) {
        V4<T> r;
        r.x = (T)bn[3 * c];
        r.y = (T)bn[3 * c + 1];
        r.z = (T)bn[3 * c + 2];
        r.w = (T)cv[c];
        nc[c] = r;
    }
}
template <typename T>
__device__ __forceinline__ T idx_bits(int c);
template <>
__device__ __forceinline__ float idx_bits<float>(int c) { return __int_as_float(c); }
template <>
__device__ __forceinline__ double idx_bits<double>(int c) { return __longlong_as_double((long long)c); }

// cap: the records `inc` holds; a list longer than that is cut (the no-allocation entry
// point rejects such lists before this runs; the engine sizes `inc` for every list)
template <typename T>
__global__ void k_pack_inc(int na, const int* ptr, const int* idx, const double* bn, V4<T>* inc, long long cap) {
    const long long tot = ptr[na] < cap ? (long long)ptr[na] : cap;
    GRID_STRIDE(k, tot) {
        const unsigned e = (unsigned)idx[k];
        const int c = (int)(e & 0x7fffffffu);
        const double sg = (e >> 31) ? -1.0 : 1.0;
        V4<T> r;
        r.x = (T)(sg * bn[3 * (long long)c]);
        r.y = (T)(sg * bn[3 * (long long)c + 1]);
        r.z = (T)(sg * bn[3 * (long long)c + 2]);
        r.w = idx_bits<T>(c);
        inc[k] = r;
    }
}

// ------------------------------------------------------------------ FP64 helpers (mixed form)
template <int DIM, int PROB>
__global__ void k_sph_particle64(int na, const int* ptr, const dvec4* inc, const int* slot, const double* invm,
                                 const double* lam, dvec4* u) {
    GRID_STRIDE(p, na) {
        double w0 = 0, w1 = 0, w2 = 0;
        for (int k = ptr[p]; k < ptr[p + 1]; ++k) {
            const dvec4 e = ld4(inc + k);
            const int c = idx_of(e.w);
            double mu = lam[c];
            if (PROB == kViscous && slot[c] >= 0) mu -= lam[slot[c]];
            w0 += mu * e.x;
            w1 += mu * e.y;
            if (DIM == 3) w2 += mu * e.z;
        }
        const double im = invm[4 * (long long)p];
        st4(u + p, im * w0, im * w1, im * w2);
    }
}

template <int DIM, int PROB>
__global__ void k_sph_residual64(int nin, const int2* cij, const dvec4* nc, const int* slot, double dt2, const dvec4* u,
                                 double* g, unsigned long long* viol_bits, const Sizes* sizes) {
    double vmax = 0.0;
    GRID_STRIDE(c, sizes->C) {
        const int2 ij = cij[c];
        const dvec4 n = ld4(nc + c);
        double q = 0.0;
        if (ij.x >= nin) {
            const dvec4 a = ld4(u + (ij.x - nin));
            q += n.x * a.x + n.y * a.y + (DIM == 3 ? n.z * a.z : 0.0);
        }
        if (ij.y >= nin) {
            const dvec4 b = ld4(u + (ij.y - nin));
            q -= n.x * b.x + n.y * b.y + (DIM == 3 ? n.z * b.z : 0.0);
        }
        const double gg = dt2 * q + n.w;
        g[c] = gg;
        if (PROB == kViscous && slot[c] >= 0) g[slot[c]] = -gg;
        vmax = fmax(vmax, -gg);
    }
    if (vmax > 0.0) atomicMax(viol_bits, (unsigned long long)__double_as_longlong(vmax));
}

int blocks(long long n) {
    long long b = (n + 255) / 256;
    if (b < 1) b = 1;
    return (int)(b < 16 * kSMs ? b : 16 * kSMs);
}

template <typename T, int DIM, int PROB>
void set_sph_smem() {
    static bool done = false;  // per instantiation; the attribute is per function and process
    if (!done) {
        cudaFuncSetAttribute(k_apgd_sph<T, DIM, PROB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)SphOcc<T>::smem);
        done = true;
    }
}

template <typename T, int DIM, int PROB>
int max_blocks_sph() {
    set_sph_smem<T, DIM, PROB>();
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_apgd_sph<T, DIM, PROB>, SphOcc<T>::threads,
                                                  SphOcc<T>::smem);
    int dev = 0, sms = kSMs;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return per_sm * sms;
}

template <typename T, int DIM, int PROB>
cudaError_t launch_t(SphArgs<T>& A, int nblocks, cudaStream_t s) {
    set_sph_smem<T, DIM, PROB>();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(SphOcc<T>::threads);
    cfg.dynamicSmemBytes = SphOcc<T>::smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    g_sph_launches += 1;
    return cudaLaunchKernelEx(&cfg, k_apgd_sph<T, DIM, PROB>, A);
}

}  // namespace

int apgd_sph_threads(bool fp32) { return fp32 ? SphOcc<float>::threads : SphOcc<double>::threads; }

int apgd_sph_max_blocks(int problem, int dim, bool fp32) {
#define MB(T, D, P) \
    if (dim == D && problem == P) return max_blocks_sph<T, D, P>();
    if (fp32) {
        MB(float, 2, 0) MB(float, 2, 2) MB(float, 3, 0) MB(float, 3, 2)
    } else {
        MB(double, 2, 0) MB(double, 2, 2) MB(double, 3, 0) MB(double, 3, 2)
    }
#undef MB
    return 0;
}

template <typename T>
cudaError_t launch_apgd_sph(int nin, int na, int dim, int problem, const ApgdSettings& st, SphSolve<T>& sb,
                            const Sizes* sizes, int nblocks, cudaStream_t s) {
    SphArgs<T> A;
    A.nin = nin;
    A.na = na;
    A.cij = sb.cij;
    A.nc = sb.nc;
    A.slot = sb.slot;
    A.shift = sb.shift;
    A.inc_ptr = sb.inc_ptr;
    A.inc = sb.inc;
    A.invm = sb.invm;
    A.lam0 = sb.lam[0];
    A.lam1 = sb.lam[1];
    A.lam2 = sb.lam[2];
    A.u0 = sb.u[0];
    A.u1 = sb.u[1];
    A.u2 = sb.u[2];
    A.u3 = sb.u[3];
    A.partials = sb.partials;
    A.bar = sb.barrier;
    A.result = sb.result;
    A.sizes = sizes;
    A.alpha = st.alpha;
    A.tol = st.tol;
    A.dt2 = st.dt * st.dt;
    A.max_ite = st.max_ite;
    A.dynamic = st.dynamic;
    A.curvature_start = st.curvature_start;
    A.stall = st.stall;
#define LA(D, P) \
    if (dim == D && problem == P) return launch_t<T, D, P>(A, nblocks, s);
    LA(2, 0) LA(2, 2) LA(3, 0) LA(3, 2)
#undef LA
    return cudaErrorInvalidValue;
}
template cudaError_t launch_apgd_sph<double>(int, int, int, int, const ApgdSettings&, SphSolve<double>&, const Sizes*,
                                             int, cudaStream_t);
template cudaError_t launch_apgd_sph<float>(int, int, int, int, const ApgdSettings&, SphSolve<float>&, const Sizes*,
                                            int, cudaStream_t);

void launch_pack_cij(const int* ci, const int* cj, int2* cij, const Sizes* sizes, long long c_cap, cudaStream_t s) {
    k_pack_cij<<<blocks(c_cap), 256, 0, s>>>(ci, cj, cij, sizes);
    g_sph_launches += 1;
}
template <typename T>
void launch_pack_nc(const double* bn, const double* cvec, V4<T>* nc, const Sizes* sizes, long long c_cap,
                    cudaStream_t s) {
    k_pack_nc<T><<<blocks(c_cap), 256, 0, s>>>(bn, cvec, nc, sizes);
    g_sph_launches += 1;
}
template void launch_pack_nc<double>(const double*, const double*, dvec4*, const Sizes*, long long, cudaStream_t);
template void launch_pack_nc<float>(const double*, const double*, float4*, const Sizes*, long long, cudaStream_t);
template <typename T>
void launch_pack_inc(int na, const int* ptr, const int* idx, const double* bn, V4<T>* inc, long long inc_cap,
                     cudaStream_t s) {
    if (na <= 0) return;
    k_pack_inc<T><<<blocks(inc_cap), 256, 0, s>>>(na, ptr, idx, bn, inc, inc_cap);
    g_sph_launches += 1;
}
template void launch_pack_inc<double>(int, const int*, const int*, const double*, dvec4*, long long, cudaStream_t);
template void launch_pack_inc<float>(int, const int*, const int*, const double*, float4*, long long, cudaStream_t);

void launch_sph_particle64(int na, int dim, int problem, const int* ptr, const dvec4* inc, const int* slot,
                           const double* invm, const double* lam, dvec4* u, cudaStream_t s) {
    if (na <= 0) return;
#define PP(D, P) \
    if (dim == D && problem == P) k_sph_particle64<D, P><<<blocks(na), 256, 0, s>>>(na, ptr, inc, slot, invm, lam, u);
    PP(2, 0) PP(2, 2) PP(3, 0) PP(3, 2)
#undef PP
    g_sph_launches += 1;
}

void launch_sph_residual64(int nin, int dim, int problem, const int2* cij, const dvec4* nc, const int* slot, double dt2,
                           const dvec4* u, double* g, unsigned long long* viol, const Sizes* sizes, long long c_cap,
                           cudaStream_t s) {
#define RR(D, P) \
    if (dim == D && problem == P) \
        k_sph_residual64<D, P><<<blocks(c_cap), 256, 0, s>>>(nin, cij, nc, slot, dt2, u, g, viol, sizes);
    RR(2, 0) RR(2, 2) RR(3, 0) RR(3, 2)
#undef RR
    g_sph_launches += 1;
}

// ------------------------------------------------------------------ entry point without allocation
//
// scopi_gpu_apgd_noalloc runs the FP64 torque-free APGD solve on caller-provided device
// arrays and keeps every intermediate array (packed contact and incidence records, the
// three multiplier buffers, the four per-body velocity buffers, block partials, the grid
// barrier and the result word) in g_noalloc_scratch below instead of cudaMalloc'd memory.
// Some callers cannot allocate device memory while they run the solve: a process whose
// device memory is owned by another allocator (a caching pool that has claimed the
// memory it will hand out), or a latency-critical loop where cudaMalloc / cudaFree would
// synchronise the device and stall the other streams.  They pass inputs and outputs only.
//
// The array is a file-scope __device__ variable, so every GPU that loads this library
// holds it (kNoAllocBytes, about 3.4 MB) until the process exits.  Its host-side name is
// only a stand-in for the device address, so at set-up the device address is fetched once
// per device with cudaGetSymbolAddress (with that device current) and passed to the
// kernels.  All calls share the array and it keeps the last call's contents: each call
// clears what must start at zero, and calls that overlap on the GPU (concurrent streams,
// or several host threads) race on it.
namespace {

constexpr long long kNoAllocMaxContacts = 16384;
constexpr long long kNoAllocMaxBodies = 8192;
constexpr int kNoAllocMaxBlocks = 4 * kSMs;

constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kOffCij = 0;
constexpr size_t kOffNc = align_up(kOffCij + sizeof(int2) * kNoAllocMaxContacts);
constexpr size_t kOffInc = align_up(kOffNc + sizeof(dvec4) * kNoAllocMaxContacts);
constexpr size_t kOffInvm = align_up(kOffInc + sizeof(dvec4) * 2 * kNoAllocMaxContacts);
constexpr size_t kOffLam = align_up(kOffInvm + sizeof(double) * kNoAllocMaxBodies);
constexpr size_t kOffU = align_up(kOffLam + sizeof(double) * 3 * kNoAllocMaxContacts);
constexpr size_t kOffPart = align_up(kOffU + sizeof(dvec4) * 4 * kNoAllocMaxBodies);
constexpr size_t kOffBar = align_up(kOffPart + sizeof(double) * 4 * kNoAllocMaxBlocks * 8);
constexpr size_t kOffRes = align_up(kOffBar + 4 * sizeof(unsigned int));
constexpr size_t kOffSizes = align_up(kOffRes + sizeof(ApgdResult));
constexpr size_t kOffFlag = align_up(kOffSizes + sizeof(Sizes));
constexpr size_t kNoAllocBytes = align_up(kOffFlag + sizeof(unsigned int));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
unsigned char* g_noalloc_dev[kMaxDevices] = {};
std::mutex g_noalloc_mutex;

// Device address of g_noalloc_scratch on the current device (set up on first use).
cudaError_t noalloc_scratch(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_dev[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_dev[dev] = static_cast<unsigned char*>(ptr);
    }
    *out = g_noalloc_dev[dev];
    return cudaSuccess;
}

// The caller's contact list and incidence lists, checked before the solve reads them so that
// no index leaves its array: bit 1 inc_ptr does not start at 0 or decreases, bit 2
// inc_ptr[na] > 2 C (more records than the fixed array holds), bit 4 a record names a
// contact >= C, bit 8 a contact names a body outside [0, nb_inactive + n_active).
constexpr unsigned kBadPtr = 1u, kBadTotal = 2u, kBadRecord = 4u, kBadBody = 8u;
__global__ void k_noalloc_check(int na, int nbody, int C, const int* ci, const int* cj, const int* ptr, const int* idx,
                                unsigned* flag) {
    const int tot = ptr[na];
    const bool tot_ok = tot >= 0 && tot <= 2 * C;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (ptr[0] != 0) atomicOr(flag, kBadPtr);
        if (!tot_ok) atomicOr(flag, kBadTotal);
    }
    GRID_STRIDE(p, na) {
        if (ptr[p] > ptr[p + 1]) atomicOr(flag, kBadPtr);
    }
    if (tot_ok) GRID_STRIDE(k, tot) {
            if ((long long)((unsigned)idx[k] & 0x7fffffffu) >= (long long)C) atomicOr(flag, kBadRecord);
        }
    GRID_STRIDE(c, C) {
        const int a = ci[c], b = cj[c];
        if (a < 0 || a >= nbody || b < 0 || b >= nbody) atomicOr(flag, kBadBody);
    }
}

__global__ void k_noalloc_prepare(Sizes* sizes, int C, int na, const double* inv_mass, double* invm) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sizes->C = C;
        sizes->C_obs = 0;
        sizes->n_extra = 0;
        sizes->overflow = 0;
    }
    GRID_STRIDE(p, na) { invm[p] = inv_mass[p]; }
}

__global__ void k_noalloc_pack_nc(const double* normal, const double* cvec, dvec4* nc, int C) {
    GRID_STRIDE(c, C) { nc[c] = dvec4{normal[3 * c], normal[3 * c + 1], normal[3 * c + 2], cvec[c]}; }
}

// copy the result buffers chosen by the solve (recorded in *res) to the caller's outputs
__global__ void k_noalloc_output(const ApgdResult* res, const double* lam_base, const dvec4* u_base, int C, int na,
                                 double* lambda, double* u) {
    const double* lam = lam_base + (size_t)res->lam_buf * kNoAllocMaxContacts;
    const dvec4* ub = u_base + (size_t)res->u_buf * kNoAllocMaxBodies;
    GRID_STRIDE(k, C) { lambda[k] = lam[k]; }
    if (u)
        GRID_STRIDE(p, na) {
            const dvec4 v = ld4(ub + p);
            u[3 * p] = v.x;
            u[3 * p + 1] = v.y;
            u[3 * p + 2] = v.z;
        }
}

}  // namespace

void set_global_error(const char* msg);
void set_global_error2(const char* a, const char* b);

}  // namespace scopi_gpu

extern "C" int32_t scopi_gpu_apgd_noalloc(int32_t dim, int64_t n_active, int64_t nb_inactive, int64_t n_contacts,
                                          const int32_t* ci, const int32_t* cj, const double* normal,
                                          const double* c, const double* inv_mass, const int32_t* inc_ptr,
                                          const int32_t* inc_idx, double dt, double alpha, double tolerance,
                                          int64_t max_ite, int32_t dynamic_descent, double* lambda, double* u,
                                          int64_t* iterations, void* stream) {
    using namespace scopi_gpu;
    if (dim != 2 && dim != 3) {
        set_global_error("scopi_gpu_apgd_noalloc: dim must be 2 or 3");
        return SCOPI_GPU_EINVAL;
    }
    if (n_contacts < 0 || n_contacts > kNoAllocMaxContacts || n_active < 0 || n_active > kNoAllocMaxBodies ||
        nb_inactive < 0) {
        set_global_error("scopi_gpu_apgd_noalloc: size beyond the no-allocation limits (at most 16384 contacts and "
                         "8192 active bodies)");
        return SCOPI_GPU_EINVAL;
    }
    if (nb_inactive > 0x7fffffffLL - n_active) {
        set_global_error("scopi_gpu_apgd_noalloc: nb_inactive + n_active must fit in a 32-bit index");
        return SCOPI_GPU_EINVAL;
    }
    if (n_contacts > 0 && (!ci || !cj || !normal || !c || !inv_mass || !inc_ptr || !inc_idx || !lambda)) {
        set_global_error("scopi_gpu_apgd_noalloc: null array");
        return SCOPI_GPU_EINVAL;
    }
    if (!(alpha > 0) || max_ite < 1) {
        set_global_error("scopi_gpu_apgd_noalloc: alpha must be > 0 and max_ite >= 1");
        return SCOPI_GPU_EINVAL;
    }
    if (iterations) *iterations = 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (n_contacts == 0) {
        if (u && n_active > 0) {
            cudaError_t e = cudaMemsetAsync(u, 0, 3 * (size_t)n_active * sizeof(double), s);
            if (e != cudaSuccess) {
                set_global_error(cudaGetErrorString(e));
                return SCOPI_GPU_ECUDA;
            }
        }
        return SCOPI_GPU_OK;
    }
    unsigned char* base = nullptr;
    cudaError_t e = noalloc_scratch(&base);
    if (e != cudaSuccess) {
        set_global_error2("scopi_gpu_apgd_noalloc: cudaGetSymbolAddress: ", cudaGetErrorString(e));
        return SCOPI_GPU_ECUDA;
    }
    const int C = (int)n_contacts, na = (int)n_active;
    int2* cij = reinterpret_cast<int2*>(base + kOffCij);
    dvec4* nc = reinterpret_cast<dvec4*>(base + kOffNc);
    dvec4* inc = reinterpret_cast<dvec4*>(base + kOffInc);
    double* invm = reinterpret_cast<double*>(base + kOffInvm);
    double* lam = reinterpret_cast<double*>(base + kOffLam);
    dvec4* ub = reinterpret_cast<dvec4*>(base + kOffU);
    double* part = reinterpret_cast<double*>(base + kOffPart);
    unsigned int* bar = reinterpret_cast<unsigned int*>(base + kOffBar);
    ApgdResult* res = reinterpret_cast<ApgdResult*>(base + kOffRes);
    Sizes* sizes = reinterpret_cast<Sizes*>(base + kOffSizes);
    unsigned* flag = reinterpret_cast<unsigned*>(base + kOffFlag);
    // the caller's lists are checked first (one read-back): nothing below indexes with them
    // before they are known to stay inside their arrays
    e = cudaMemsetAsync(flag, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) {
        set_global_error2("scopi_gpu_apgd_noalloc: cudaMemsetAsync: ", cudaGetErrorString(e));
        return SCOPI_GPU_ECUDA;
    }
    k_noalloc_check<<<blocks(std::max(C, na + 1)), 256, 0, s>>>(na, (int)(nb_inactive + n_active), C, ci, cj,
                                                                inc_ptr, inc_idx, flag);
    unsigned host_flag = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&host_flag, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_global_error2("scopi_gpu_apgd_noalloc: input check: ", cudaGetErrorString(e));
        return SCOPI_GPU_ECUDA;
    }
    if (host_flag) {
        set_global_error((host_flag & kBadTotal)
                             ? "scopi_gpu_apgd_noalloc: inc_ptr[n_active] exceeds 2 * n_contacts"
                             : (host_flag & kBadPtr)
                                   ? "scopi_gpu_apgd_noalloc: inc_ptr must start at 0 and never decrease"
                                   : (host_flag & kBadRecord)
                                         ? "scopi_gpu_apgd_noalloc: inc_idx names a contact >= n_contacts"
                                         : "scopi_gpu_apgd_noalloc: ci/cj must be < nb_inactive + n_active");
        return SCOPI_GPU_EINVAL;
    }
    // the array keeps the previous call's contents: clear what the solve reads before writing
    // (lambda and lambda_prev, u(lambda), u(y), the barrier words, the result)
    struct Clear {
        void* p;
        size_t n;
    } clears[] = {{lam, 2 * sizeof(double) * kNoAllocMaxContacts},
                  {ub, sizeof(dvec4) * kNoAllocMaxBodies},
                  {ub + 2 * kNoAllocMaxBodies, sizeof(dvec4) * kNoAllocMaxBodies},
                  {bar, 4 * sizeof(unsigned int)},
                  {res, sizeof(ApgdResult)}};
    for (const Clear& cl : clears) {
        e = cudaMemsetAsync(cl.p, 0, cl.n, s);
        if (e != cudaSuccess) {
            set_global_error2("scopi_gpu_apgd_noalloc: cudaMemsetAsync: ", cudaGetErrorString(e));
            return SCOPI_GPU_ECUDA;
        }
    }
    k_noalloc_prepare<<<blocks(na), 256, 0, s>>>(sizes, C, na, inv_mass, invm);
    launch_pack_cij(ci, cj, cij, sizes, C, s);
    k_noalloc_pack_nc<<<blocks(C), 256, 0, s>>>(normal, c, nc, C);
    launch_pack_inc<double>(na, inc_ptr, inc_idx, normal, inc, 2 * (long long)C, s);
    SphArgs<double> A;
    A.nin = (int)nb_inactive;
    A.na = na;
    A.cij = cij;
    A.nc = nc;
    A.slot = nullptr;
    A.shift = nullptr;
    A.inc_ptr = inc_ptr;
    A.inc = inc;
    A.invm = invm;
    A.lam0 = lam;
    A.lam1 = lam + kNoAllocMaxContacts;
    A.lam2 = lam + 2 * kNoAllocMaxContacts;
    A.u0 = ub;
    A.u1 = ub + kNoAllocMaxBodies;
    A.u2 = ub + 2 * kNoAllocMaxBodies;
    A.u3 = ub + 3 * kNoAllocMaxBodies;
    A.partials = part;
    A.bar = bar;
    A.result = res;
    A.sizes = sizes;
    A.alpha = alpha;
    A.tol = tolerance;
    A.dt2 = dt * dt;
    A.max_ite = max_ite;
    A.dynamic = dynamic_descent ? 1 : 0;
    A.curvature_start = 0;
    A.stall = 0;
    int maxb = apgd_sph_max_blocks(kNoFriction, dim, false);
    if (maxb > kNoAllocMaxBlocks) maxb = kNoAllocMaxBlocks;
    const int thr = SphOcc<double>::threads;
    long long nb = (std::max<long long>(C, na) + thr - 1) / thr;
    if (nb < 1) nb = 1;
    if (nb > maxb) nb = maxb;
    e = dim == 3 ? launch_t<double, 3, kNoFriction>(A, (int)nb, s) : launch_t<double, 2, kNoFriction>(A, (int)nb, s);
    if (e != cudaSuccess) {
        set_global_error2("scopi_gpu_apgd_noalloc: launch: ", cudaGetErrorString(e));
        return SCOPI_GPU_ECUDA;
    }
    k_noalloc_output<<<blocks(std::max(C, na)), 256, 0, s>>>(res, lam, ub, C, na, lambda, u);
    ApgdResult host_res;
    e = cudaMemcpyAsync(&host_res, res, sizeof(ApgdResult), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_global_error2("scopi_gpu_apgd_noalloc: ", cudaGetErrorString(e));
        return SCOPI_GPU_ECUDA;
    }
    if (iterations) *iterations = host_res.iterations;
    if (host_res.error) {
        set_global_error("scopi_gpu_apgd_noalloc: APGD grid barrier timed out");
        return SCOPI_GPU_ETIMEOUT;
    }
    return host_res.converged ? SCOPI_GPU_OK : SCOPI_GPU_ENOCONV;
}

