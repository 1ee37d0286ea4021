// apgd.cu -- persistent, grid-synchronised APGD (accelerated projected gradient with
// backtracking Lipschitz estimate and gradient restart) on the contact QP
//     min_l  1/2 l^T Q l + c^T l,  Q = dt^2 B M^-1 B^T,  l in K (R+ or the friction cone)
// following apgd::operator() (include/scopi/solvers/apgd.hpp:148-221) step for step:
// same iterate sequence, backtracking inequality, restart test and stopping rule.
//
// One iteration = two sparse passes instead of the reference's six:
//   contact pass : Qy_c = dt^2 B_c (M^-1 B^T y) gathered from the two bodies, g = Qy + c,
//                  l+ = P(y - alpha g), and the partial sums of every scalar the
//                  iteration needs (F(y), g.(l+-y), |l+-y|^2, c.l+, |l+-l|^2, g.(l+-l));
//   particle pass: w = B^T l+ gathered over each body's incidence list, u = M^-1 w,
//                  and w.u, so F(l+) = 1/2 dt^2 w.u + c.l+ needs no second product.
// M^-1 B^T y is never formed: y = l + beta (l - l_prev) so it is the same combination
// of the stored u(l) and u(l_prev).  Reductions are fixed-order (per-block partials,
// reduced identically by every block), so every block takes the same branch and the
// result is bitwise reproducible.  Grid barriers are bounded waits (globaltimer) that
// set an error flag instead of hanging.
#include <math.h>

#include <algorithm>

#include "apgd_common.cuh"

namespace scopi_gpu {

static long long g_apgd_launches = 0;
long long apgd_launches() { return g_apgd_launches; }

namespace {

constexpr int kApgdThreads = 256;
constexpr int kPartials = 9;  // s1..s8 and the FP32 curvature term
// bounded grid barrier with a runtime limit (bar[3]) shared with the torque-free kernel
using apgdc::grid_barrier;

template <typename T>
struct Vec6 {
    T v[6];
};

__device__ __forceinline__ void load6(const double* p, double* o) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = q[0], b = q[1], c = q[2];
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y; o[4] = c.x; o[5] = c.y;
}
__device__ __forceinline__ void load6(const float* p, float* o) {
    const float2* q = reinterpret_cast<const float2*>(p);
    const float2 a = q[0], b = q[1], c = q[2];
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y; o[4] = c.x; o[5] = c.y;
}
__device__ __forceinline__ void load6cg(const double* p, double* o) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldcg(q), b = __ldcg(q + 1), c = __ldcg(q + 2);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y; o[4] = c.x; o[5] = c.y;
}
__device__ __forceinline__ void load6cg(const float* p, float* o) {
    const float2* q = reinterpret_cast<const float2*>(p);
    const float2 a = __ldcg(q), b = __ldcg(q + 1), c = __ldcg(q + 2);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y; o[4] = c.x; o[5] = c.y;
}
__device__ __forceinline__ void store6(double* p, const double* o) {
    double2* q = reinterpret_cast<double2*>(p);
    q[0] = make_double2(o[0], o[1]);
    q[1] = make_double2(o[2], o[3]);
    q[2] = make_double2(o[4], o[5]);
}
__device__ __forceinline__ void store6(float* p, const float* o) {
    float2* q = reinterpret_cast<float2*>(p);
    q[0] = make_float2(o[0], o[1]);
    q[1] = make_float2(o[2], o[3]);
    q[2] = make_float2(o[4], o[5]);
}

// fixed-order block reduction of kPartials doubles; result valid in every thread
__device__ __forceinline__ void block_sum(double* v) {
    __shared__ double sh[kApgdThreads / 32][kPartials];
    __shared__ double tot[kPartials];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kPartials; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[warp][k] = x;
    }
    __syncthreads();
    if (threadIdx.x < kPartials) {
        double s = 0.0;
        for (int w = 0; w < kApgdThreads / 32; ++w) s += sh[w][threadIdx.x];
        tot[threadIdx.x] = s;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kPartials; ++k) v[k] = tot[k];
    __syncthreads();
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

// ViscousFriction: four multiplier slots per contact; the contact's mode (set from gamma at
// assembly, LagrangeMultiplier<ViscousFriction>, lagrange_multiplier.hpp:358-398) says which
// are live: 0 (l) with force l n, 1 (l+, l-) with force (l+ - l-) n, 2 (l0, f) with force
// -l0 n + f.  Unused slots stay 0.
// local2global of one contact's slots (lagrange_multiplier.hpp:428-454)
template <typename T, int DIM>
__device__ __forceinline__ void vf_force(int mode, const T* l, const T* n, T* f) {
    for (int d = 0; d < 3; ++d) {
        if (mode == 0)
            f[d] = l[0] * n[d];
        else if (mode == 1)
            f[d] = (l[0] - l[1]) * n[d];
        else
            f[d] = (-l[0]) * n[d] + ((DIM == 2 && d == 2) ? (T)0 : l[1 + d]);
    }
}
// global2local of a 3-vector x (lagrange_multiplier.hpp:400-426)
template <typename T, int DIM>
__device__ __forceinline__ void vf_local(int mode, const T* x, const T* n, T* o) {
    T xn = 0;
    for (int d = 0; d < DIM; ++d) xn += x[d] * n[d];
    o[0] = mode == 2 ? -xn : xn;
    o[1] = mode == 1 ? -xn : (mode == 2 ? x[0] : (T)0);
    o[2] = mode == 2 ? x[1] : (T)0;
    o[3] = (mode == 2 && DIM == 3) ? x[2] : (T)0;
}
// projection of one contact's slots (lagrange_multiplier.hpp:466-536): R+ per live slot in
// modes 0 and 1; in mode 2 the nearer of (0, P_cone(f)) and (max(l0, 0), 0)
template <int DIM>
__device__ __forceinline__ void vf_project(int mode, double* z, const double* n, double mu) {
    if (mode != 2) {
        z[0] = z[0] > 0.0 ? z[0] : 0.0;
        z[1] = mode == 1 ? (z[1] > 0.0 ? z[1] : 0.0) : 0.0;
        z[2] = 0.0;
        z[3] = 0.0;
        return;
    }
    double fr[4] = {0.0, z[1], z[2], DIM == 3 ? z[3] : 0.0};
    cone_project<DIM>(fr + 1, n, mu);
    const double mo[4] = {z[0] > 0.0 ? z[0] : 0.0, 0.0, 0.0, 0.0};
    double df = 0.0, dm = 0.0;
    for (int k = 0; k < 1 + DIM; ++k) {
        df += (fr[k] - z[k]) * (fr[k] - z[k]);
        dm += (mo[k] - z[k]) * (mo[k] - z[k]);
    }
    const double* pick = sqrt(df) < sqrt(dm) ? fr : mo;
    for (int k = 0; k < 1 + DIM; ++k) z[k] = pick[k];
    if (DIM == 2) z[3] = 0.0;
}

template <typename T>
struct ApgdArgs {
    int nin;
    int na;
    const int* ci;
    const int* cj;
    const int* slot;       // viscous
    const int* mode;       // viscous friction
    const T* bn;
    const T* bai;
    const T* baj;
    const T* bP;
    const T* cvec;
    const double* shift;
    const int* inc_ptr;
    const int* inc_idx;
    const T* inc_coef;
    const T* invm;         // na*4: 1/m, 1/Jx, 1/Jy, 1/Jz (2D: 1/m, 0, 0, 1/Jz)
    T* lam0;
    T* lam1;
    T* lam2;
    T* u0;
    T* u1;
    T* u2;
    T* g;
    double* partials;
    unsigned int* bar;
    ApgdResult* result;
    const Sizes* sizes;
    double alpha, tol, dt2, mu;
    long long max_ite;
    int dynamic;
    int curvature_start;
    int stall;  // block 0 skips its first barrier arrival (test of the barrier limit)
};

template <typename T, int DIM, int PROB>
__device__ __forceinline__ void gather_uy(const ApgdArgs<T>& A, int body, const T* ul, const T* up, T beta, bool use_prev,
                                          T* uy) {
    const int p = body - A.nin;
    T a[6];
    load6cg(ul + 6 * (long long)p, a);
    if (use_prev) {
        T b[6];
        load6cg(up + 6 * (long long)p, b);
#pragma unroll
        for (int k = 0; k < 6; ++k) uy[k] = a[k] + beta * (a[k] - b[k]);
    } else {
#pragma unroll
        for (int k = 0; k < 6; ++k) uy[k] = a[k];
    }
}

// One contact's contribution to the contact pass (normal problems).
template <typename T, int DIM, int PROB>
__device__ __forceinline__ void contact_scalar(const ApgdArgs<T>& A, long long m, T qy, T cc, const T* lam, const T* lprev,
                                               T* lnew, T beta, bool use_prev, bool bt, double alpha, double* s) {
    const T lm = lam[m];
    T y = lm;
    if (use_prev) y = lm + beta * (lm - lprev[m]);
    T gm;
    if (bt) {
        gm = A.g[m];
    } else {
        gm = qy + cc;
        A.g[m] = gm;
    }
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
    s[0] += (double)gm * dly;
    s[1] += dly * dly;
    s[2] += (double)cc * (double)lp;
    if (!bt) s[3] += (double)y * (0.5 * (double)qy + (double)cc);
    s[4] += dll * dll;
    s[5] += (double)gm * dll;
    s[7] += (double)lp * (double)lp;
}

// Contact c's share of the contact pass (its rows of l+ and its terms of the partial sums).
template <typename T, int DIM, int PROB>
__device__ __forceinline__ void contact_one(const ApgdArgs<T>& A, long long c, const T* lam, const T* lprev, T* lnew,
                                            const T* ul, const T* up, T beta, bool use_prev, bool bt, double alpha,
                                            double* s) {
    {
        const int i = A.ci[c], j = A.cj[c];
        if (PROB != kFriction && PROB != kViscousFriction) {
            T qy = 0;
            if (!bt) {
                T n[3];
                n[0] = A.bn[3 * c];
                n[1] = A.bn[3 * c + 1];
                n[2] = DIM == 3 ? A.bn[3 * c + 2] : (T)0;
                if (i >= A.nin) {
                    T uy[6];
                    gather_uy<T, DIM, PROB>(A, i, ul, up, beta, use_prev, uy);
                    if (DIM == 3) {
                        qy += n[0] * uy[0] + n[1] * uy[1] + n[2] * uy[2];
                        qy += A.bai[3 * c] * uy[3] + A.bai[3 * c + 1] * uy[4] + A.bai[3 * c + 2] * uy[5];
                    } else {
                        qy += n[0] * uy[0] + n[1] * uy[1] + A.bai[3 * c + 2] * uy[5];
                    }
                }
                if (j >= A.nin) {
                    T uy[6];
                    gather_uy<T, DIM, PROB>(A, j, ul, up, beta, use_prev, uy);
                    if (DIM == 3) {
                        qy -= n[0] * uy[0] + n[1] * uy[1] + n[2] * uy[2];
                        qy += A.baj[3 * c] * uy[3] + A.baj[3 * c + 1] * uy[4] + A.baj[3 * c + 2] * uy[5];
                    } else {
                        qy -= n[0] * uy[0] + n[1] * uy[1];
                        qy += A.baj[3 * c + 2] * uy[5];
                    }
                }
                qy *= (T)A.dt2;
            }
            const T cc = A.cvec[c];
            contact_scalar<T, DIM, PROB>(A, c, qy, cc, lam, lprev, lnew, beta, use_prev, bt, alpha, s);
            if (PROB == kViscous) {
                const int sl = A.slot[c];
                if (sl >= 0) contact_scalar<T, DIM, PROB>(A, sl, -qy, -cc, lam, lprev, lnew, beta, use_prev, bt, alpha, s);
            }
        } else {
            // friction rows: A_c u = v_i + P_i^T w_i - v_j - P_j^T w_j (three per contact)
            T qy[3] = {0, 0, 0};
            if (!bt) {
                for (int side = 0; side < 2; ++side) {
                    const int b = side == 0 ? i : j;
                    if (b < A.nin) continue;
                    T uy[6];
                    gather_uy<T, DIM, PROB>(A, b, ul, up, beta, use_prev, uy);
                    const T* P = A.bP + 18 * (long long)c + 9 * side;
                    const T sg = side == 0 ? (T)1 : (T)-1;
                    for (int d = 0; d < 3; ++d) {
                        const T pt = P[0 * 3 + d] * uy[3] + P[1 * 3 + d] * uy[4] + P[2 * 3 + d] * uy[5];
                        const T vd = (DIM == 2 && d == 2) ? (T)0 : uy[d];
                        qy[d] += sg * (vd + pt);
                    }
                }
                for (int d = 0; d < 3; ++d) qy[d] *= (T)A.dt2;
            }
            if constexpr (PROB == kViscousFriction) {
                // four slots: g = global2local(Q y) + c, then the mode's projection
                const int md = A.mode[c];
                T nt[3] = {A.bn[3 * c], A.bn[3 * c + 1], A.bn[3 * c + 2]};
                T ql[4];
                vf_local<T, DIM>(md, qy, nt, ql);
                double y[4], gm[4], lm[4], z[4], nd[3];
                for (int k = 0; k < 4; ++k) {
                    const long long m = 4 * c + k;
                    lm[k] = (double)lam[m];
                    y[k] = use_prev ? (double)(lam[m] + beta * (lam[m] - lprev[m])) : lm[k];
                    if (bt) {
                        gm[k] = (double)A.g[m];
                    } else {
                        const T gg = ql[k] + A.cvec[m];
                        A.g[m] = gg;
                        gm[k] = (double)gg;
                    }
                    z[k] = y[k] - alpha * gm[k];
                    if (A.shift) z[k] += A.shift[m];
                }
                for (int d = 0; d < 3; ++d) nd[d] = (double)nt[d];
                vf_project<DIM>(md, z, nd, A.mu);
                for (int k = 0; k < 4; ++k) {
                    const long long m = 4 * c + k;
                    const T lp = (T)(A.shift ? z[k] - A.shift[m] : z[k]);
                    lnew[m] = lp;
                    const double dly = (double)lp - y[k], dll = (double)lp - lm[k];
                    const double cc = (double)A.cvec[m];
                    s[0] += gm[k] * dly;
                    s[1] += dly * dly;
                    s[2] += cc * (double)lp;
                    if (!bt) s[3] += y[k] * (0.5 * (double)ql[k] + cc);
                    s[4] += dll * dll;
                    s[5] += gm[k] * dll;
                    s[7] += (double)lp * (double)lp;
                }
            } else {
                double y[3], gm[3], lm[3];
                for (int d = 0; d < 3; ++d) {
                    const long long m = 3 * c + d;
                    lm[d] = (double)lam[m];
                    y[d] = use_prev ? (double)(lam[m] + beta * (lam[m] - lprev[m])) : lm[d];
                    if (bt) {
                        gm[d] = (double)A.g[m];
                    } else {
                        const T gg = qy[d] + A.cvec[m];
                        A.g[m] = gg;
                        gm[d] = (double)gg;
                    }
                }
                double z[3], n[3];
                for (int d = 0; d < 3; ++d) {
                    n[d] = (double)A.bn[3 * c + d];
                    z[d] = y[d] - alpha * gm[d];
                    if (A.shift) z[d] += A.shift[3 * c + d];
                }
                if (DIM == 2) z[2] = A.shift ? A.shift[3 * c + 2] : 0.0;
                cone_project<DIM>(z, n, A.mu);
                for (int d = 0; d < 3; ++d) {
                    const long long m = 3 * c + d;
                    const T lp = (T)(A.shift ? z[d] - A.shift[m] : z[d]);
                    lnew[m] = lp;
                    const double dly = (double)lp - y[d], dll = (double)lp - lm[d];
                    const double cc = (double)A.cvec[m];
                    s[0] += gm[d] * dly;
                    s[1] += dly * dly;
                    s[2] += cc * (double)lp;
                    if (!bt) s[3] += y[d] * (0.5 * (double)qy[d] + cc);
                    s[4] += dll * dll;
                    s[5] += gm[d] * dll;
                    s[7] += (double)lp * (double)lp;
                }
            }
        }
    }
}

template <typename T, int DIM, int PROB>
__device__ void contact_pass(const ApgdArgs<T>& A, int C, const T* lam, const T* lprev, T* lnew, const T* ul,
                             const T* up, T beta, bool use_prev, bool bt, double alpha, double* s) {
    GRID_STRIDE(c, C) contact_one<T, DIM, PROB>(A, c, lam, lprev, lnew, ul, up, beta, use_prev, bt, alpha, s);
}

// Body p's share of the particle pass.  curv (FP32 iterations): s[8] += (u(l+) - u(y))^T M
// (u(l+) - u(y)), the curvature d^T Q d / dt^2 along d = l+ - y of the curvature-form
// backtracking test.
template <typename T, int DIM, int PROB>
__device__ __forceinline__ void particle_one(const ApgdArgs<T>& A, long long p, const T* lnew, T* unew, const T* ul,
                                             const T* up, T beta, bool use_prev, bool curv, double* s) {
    {
        T w[6] = {0, 0, 0, 0, 0, 0};
        const int k0 = A.inc_ptr[p], k1 = A.inc_ptr[p + 1];
        for (int k = k0; k < k1; ++k) {
            const unsigned e = (unsigned)A.inc_idx[k];
            const long long c = e & 0x7fffffffu;
            if (PROB != kFriction && PROB != kViscousFriction) {
                T mu = __ldcg(lnew + c);
                if (PROB == kViscous) {
                    const int sl = A.slot[c];
                    if (sl >= 0) mu -= __ldcg(lnew + sl);
                }
                T cf[6];
                load6(A.inc_coef + 6 * (long long)k, cf);
#pragma unroll
                for (int d = 0; d < 6; ++d) w[d] += mu * cf[d];
            } else {
                const int side = (int)(e >> 31);
                const T sg = side == 0 ? (T)1 : (T)-1;
                T f[3];
                if (PROB == kViscousFriction) {
                    const T l4[4] = {__ldcg(lnew + 4 * c), __ldcg(lnew + 4 * c + 1), __ldcg(lnew + 4 * c + 2),
                                     __ldcg(lnew + 4 * c + 3)};
                    const T nt[3] = {A.bn[3 * c], A.bn[3 * c + 1], A.bn[3 * c + 2]};
                    vf_force<T, DIM>(A.mode[c], l4, nt, f);
                } else {
                    f[0] = __ldcg(lnew + 3 * c);
                    f[1] = __ldcg(lnew + 3 * c + 1);
                    f[2] = __ldcg(lnew + 3 * c + 2);
                }
                const T* P = A.bP + 18 * c + 9 * side;
                for (int d = 0; d < 3; ++d) {
                    w[d] += sg * f[d];
                    w[3 + d] += sg * (P[3 * d] * f[0] + P[3 * d + 1] * f[1] + P[3 * d + 2] * f[2]);
                }
            }
        }
        const T* im = A.invm + 4 * (long long)p;
        T u[6];
        u[0] = im[0] * w[0];
        u[1] = im[0] * w[1];
        u[2] = DIM == 3 ? im[0] * w[2] : (T)0;
        u[3] = im[1] * w[3];
        u[4] = im[2] * w[4];
        u[5] = im[3] * w[5];
        store6(unew + 6 * (long long)p, u);
        double acc = 0.0;
#pragma unroll
        for (int d = 0; d < 6; ++d) acc += (double)w[d] * (double)u[d];
        s[6] += acc;
        if (curv) {
            T a[6], b[6];
            load6cg(ul + 6 * (long long)p, a);
            if (use_prev) load6cg(up + 6 * (long long)p, b);
            const T m[6] = {im[0], im[0], im[0], im[1], im[2], im[3]};
            double q = 0.0;
#pragma unroll
            for (int d = 0; d < 6; ++d) {
                const T uy = use_prev ? a[d] + beta * (a[d] - b[d]) : a[d];
                const double dd = (double)u[d] - (double)uy;
                if (m[d] > (T)0) q += dd * dd / (double)m[d];
            }
            s[8] += q;
        }
    }
}

template <typename T, int DIM, int PROB>
__device__ void particle_pass(const ApgdArgs<T>& A, const T* lnew, T* unew, const T* ul, const T* up, T beta,
                              bool use_prev, bool curv, double* s) {
    GRID_STRIDE(p, A.na) particle_one<T, DIM, PROB>(A, p, lnew, unew, ul, up, beta, use_prev, curv, s);
}

template <typename T, int DIM, int PROB>
__global__ void __launch_bounds__(kApgdThreads) k_apgd(ApgdArgs<T> A) {
    const int C = A.sizes->C;
    const unsigned int nb = gridDim.x;
    T* lamb[3] = {A.lam0, A.lam1, A.lam2};
    T* ub[3] = {A.u0, A.u1, A.u2};
    int il = 0, ip = 1, in_ = 2;   // lambda (current), previous, candidate
    int jl = 0, jp = 1, jn = 2;    // u of the same three
    double alpha = A.alpha;
    double lipsch = 1.0 / alpha;
    double lgood = lipsch;         // last finite estimate of an accepted iteration
    double theta = 1.0;
    double beta = 0.0;
    bool use_prev = false;         // beta != 0
    bool bt = false;
    double Fy = 0.0;
    long long ite = 0, nbt = 0, nrs = 0;
    int conv = 0, err = 0;
    int parity = 0;
    double last_step = 0.0;
    bool withhold = A.stall != 0 && blockIdx.x == 0;
    if (A.curvature_start) {
        // initial step from the curvature along the first projected-gradient direction d of
        // the cold start (stored in the candidate buffers, which the first iteration
        // overwrites): L = 1.5 dt^2 |B^T d|^2_{M^-1} / |d|^2
        T* dbuf = lamb[in_];
        double s[kPartials] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        GRID_STRIDE(c, C) {
            if (PROB == kViscousFriction) {
                double z[4], n[3];
                for (int d = 0; d < 3; ++d) n[d] = (double)A.bn[3 * c + d];
                for (int k = 0; k < 4; ++k) z[k] = -(double)A.cvec[4 * c + k] + (A.shift ? A.shift[4 * c + k] : 0.0);
                vf_project<DIM>(A.mode[c], z, n, A.mu);
                for (int k = 0; k < 4; ++k) {
                    const T v = (T)(z[k] - (A.shift ? A.shift[4 * c + k] : 0.0));
                    dbuf[4 * c + k] = v;
                    s[1] += (double)v * (double)v;
                }
            } else if (PROB == kFriction) {
                double z[3], n[3];
                for (int d = 0; d < 3; ++d) {
                    n[d] = (double)A.bn[3 * c + d];
                    z[d] = -(double)A.cvec[3 * c + d] + (A.shift ? A.shift[3 * c + d] : 0.0);
                }
                if (DIM == 2) z[2] = A.shift ? A.shift[3 * c + 2] : 0.0;
                cone_project<DIM>(z, n, A.mu);
                for (int d = 0; d < 3; ++d) {
                    const T v = (T)(z[d] - (A.shift ? A.shift[3 * c + d] : 0.0));
                    dbuf[3 * c + d] = v;
                    s[1] += (double)v * (double)v;
                }
            } else {
                const T v = apgdc::first_descent<T>(A.cvec[c], A.shift, c);
                dbuf[c] = v;
                s[1] += (double)v * (double)v;
                if (PROB == kViscous) {
                    const int sl = A.slot[c];
                    if (sl >= 0) {
                        const T v2 = apgdc::first_descent<T>(-A.cvec[c], A.shift, sl);
                        dbuf[sl] = v2;
                        s[1] += (double)v2 * (double)v2;
                    }
                }
            }
        }
        bool ok = grid_barrier(A.bar, nb, withhold);
        withhold = false;
        if (ok) particle_pass<T, DIM, PROB>(A, dbuf, ub[jn], ub[jl], ub[jp], (T)0, false, false, s);
        block_sum(s);
        double* part = A.partials;
        if (threadIdx.x == 0)
            for (int k = 0; k < kPartials; ++k) part[blockIdx.x * kPartials + k] = s[k];
        if (ok) ok = grid_barrier(A.bar, nb);
        double t[kPartials] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (unsigned int b = threadIdx.x; b < nb; b += blockDim.x)
            for (int k = 0; k < kPartials; ++k) t[k] += __ldcg(part + b * kPartials + k);
        block_sum(t);
        // the first iteration writes partials region 1, then region 0 after a barrier
        parity = 1;
        double l;
        if (!ok) {
            err = 1;
        } else if (apgdc::initial_lipschitz(t[1], t[6], A.dt2, l)) {
            lipsch = l;
            alpha = 1.0 / l;
            lgood = l;
        }
    }
    for (;;) {
        if (err) break;
        double s[kPartials] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        contact_pass<T, DIM, PROB>(A, C, lamb[il], lamb[ip], lamb[in_], ub[jl], ub[jp], (T)beta, use_prev, bt, alpha, s);
        const bool wh = withhold;
        withhold = false;
        if (!grid_barrier(A.bar, nb, wh)) { err = 1; break; }
        particle_pass<T, DIM, PROB>(A, lamb[in_], ub[jn], ub[jl], ub[jp], (T)beta, use_prev, sizeof(T) == 4, s);
        block_sum(s);
        double* part = A.partials + (size_t)parity * nb * kPartials;
        if (threadIdx.x == 0)
            for (int k = 0; k < kPartials; ++k) part[blockIdx.x * kPartials + k] = s[k];
        if (!grid_barrier(A.bar, nb)) { err = 1; break; }
        double t[kPartials] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (unsigned int b = threadIdx.x; b < nb; b += blockDim.x)
            for (int k = 0; k < kPartials; ++k) t[k] += __ldcg(part + b * kPartials + k);
        block_sum(t);
        parity ^= 1;
        if (!bt) Fy = t[3];
        const double F_lp = 0.5 * A.dt2 * t[6] + t[2];
        if (A.dynamic && t[1] == 0.0) {
            // l+ == y bit for bit: the reference evaluates F(l+) >= F(y) on identical vectors,
            // keeps doubling L (l+ cannot move: -g is in the normal cone at y) until
            // 0.5*L*0 turns NaN at L = inf, then accepts with alpha = 0.
            while (isfinite(lipsch)) {
                lipsch *= 2;
                ++nbt;
            }
            alpha = 1. / lipsch;
        } else if (A.dynamic && apgdc::sufficient_decrease_fails<T>(F_lp, Fy, t[0], t[1], A.dt2 * t[8], lipsch)) {
            // backtracking, apgd.hpp:172-182 (FP32: its curvature form)
            lipsch *= 2;
            alpha = 1. / lipsch;
            bt = true;
            ++nbt;
            if (nbt > 4000) { err = 2; break; }   // alpha underflow guard
            continue;
        }
        ++ite;
        bt = false;
        if (isfinite(lipsch)) lgood = lipsch;
        last_step = sqrt(t[4]);
        double tol = A.tol;
        if (sizeof(T) == 4) {
            // FP32 iterations stall at their rounding floor; the FP64 correction recovers the rest
            const double floor32 = 4.0 * 1.1920929e-7 * sqrt(t[7]);
            if (floor32 > tol) tol = floor32;
        }
        // lambda <- lambda+, u <- u(lambda+)
        int tmp = ip; ip = il; il = in_; in_ = tmp;
        tmp = jp; jp = jl; jl = jn; jn = tmp;
        if (last_step < tol) { conv = 1; break; }
        const double theta1 = 0.5 * (theta * sqrt(4 + theta * theta) - theta * theta);
        beta = theta * (1 - theta) / (theta * theta + theta1);
        theta = theta1;
        if (A.dynamic) {
            if (t[5] > 0) {  // restart, apgd.hpp:200-206
                beta = 0.0;
                theta = 1.;
                ++nrs;
            }
            lipsch *= 0.97;
            alpha = 1. / lipsch;
        }
        use_prev = (beta != 0.0);
        if (ite >= A.max_ite) break;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        A.result->iterations = ite;
        A.result->backtracks = nbt;
        A.result->restarts = nrs;
        A.result->converged = conv;
        A.result->lam_buf = il;
        A.result->u_buf = jl;
        A.result->error = err;
        A.result->last_step = last_step;
        A.result->lipsch = lgood;
    }
}

// ------------------------------------------------- batched scenes, 6-dof rows (FP64)
// One CTA per scene (scenes taken largest first): the iteration of k_apgd on the scene's
// contacts (its obstacle rows [o0, o1), then its active rows [a0, a1)) and bodies [p0, p1),
// with block barriers and block sums in place of the grid ones, so every scene iterates
// until its own stopping test holds.  At the end the CTA copies its scene's multipliers and
// u = M^-1 B^T l to fixed outputs (which rotating buffer holds them differs per scene) and
// writes the scene's statistics with the violation max(0, -gap) of its final state.
constexpr int kBatch6Threads = 256;

__device__ __forceinline__ double block_max(double v) {
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double m = 0.0;
    for (int w = 0; w < nw; ++w) m = fmax(m, sh[w]);
    __syncthreads();
    return m;
}

template <int DIM, int PROB>
__global__ void __launch_bounds__(kBatch6Threads) k_apgd_batch6(ApgdArgs<double> A, Batch6Scenes S) {
    using T = double;
    constexpr int R = PROB == kFriction ? 3 : 1;  // multipliers per contact
    T* lamb[3] = {A.lam0, A.lam1, A.lam2};
    T* ub[3] = {A.u0, A.u1, A.u2};
    for (int q = blockIdx.x; q < S.n_scenes; q += gridDim.x) {
        const int sc = S.order[q];
        const int o0 = S.sc_o0[sc], n0 = S.sc_o1[sc] - o0, a0 = S.sc_a0[sc];
        const int nc = n0 + (S.sc_a1[sc] - a0);
        const int p0 = S.sc_p0[sc], p1 = S.sc_p1[sc];
        auto contact_at = [&](int k) -> long long { return k < n0 ? (long long)o0 + k : (long long)a0 + (k - n0); };
        int il = 0, ip = 1, in_ = 2, jl = 0, jp = 1, jn = 2;
        double alpha = A.alpha, lipsch = 1.0 / alpha, lgood = lipsch, theta = 1.0, beta = 0.0;
        bool use_prev = false, bt = false;
        double Fy = 0.0, last_step = 0.0;
        long long ite = 0, nbt = 0, nrs = 0;
        int conv = nc == 0 ? 1 : 0, err = 0;
        if (nc > 0 && A.curvature_start) {
            // L = 1.5 dt^2 |B^T d|^2_{M^-1} / |d|^2 along the first projected-gradient direction
            T* dbuf = lamb[in_];
            double s[kPartials] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int k = threadIdx.x; k < nc; k += blockDim.x) {
                const long long c = contact_at(k);
                if (PROB == kFriction) {
                    double z[3], n[3];
                    for (int d = 0; d < 3; ++d) {
                        n[d] = A.bn[3 * c + d];
                        z[d] = -A.cvec[3 * c + d];
                    }
                    if (DIM == 2) z[2] = 0.0;
                    cone_project<DIM>(z, n, A.mu);
                    for (int d = 0; d < 3; ++d) {
                        dbuf[3 * c + d] = z[d];
                        s[1] += z[d] * z[d];
                    }
                } else {
                    const T v = apgdc::first_descent<T>(A.cvec[c], nullptr, c);
                    dbuf[c] = v;
                    s[1] += v * v;
                    if (PROB == kViscous) {
                        const int sl = A.slot[c];
                        if (sl >= 0) {
                            const T v2 = apgdc::first_descent<T>(-A.cvec[c], nullptr, sl);
                            dbuf[sl] = v2;
                            s[1] += v2 * v2;
                        }
                    }
                }
            }
            __syncthreads();
            for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x)
                particle_one<T, DIM, PROB>(A, p, dbuf, ub[jn], ub[jl], ub[jp], (T)0, false, false, s);
            apgdc::block_sum<kPartials>(s);
            double l;
            if (apgdc::initial_lipschitz(s[1], s[6], A.dt2, l)) {
                lipsch = l;
                alpha = 1.0 / l;
                lgood = l;
            }
        }
        while (!conv) {
            double s[kPartials] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int k = threadIdx.x; k < nc; k += blockDim.x)
                contact_one<T, DIM, PROB>(A, contact_at(k), lamb[il], lamb[ip], lamb[in_], ub[jl], ub[jp], (T)beta,
                                          use_prev, bt, alpha, s);
            __syncthreads();
            for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x)
                particle_one<T, DIM, PROB>(A, p, lamb[in_], ub[jn], ub[jl], ub[jp], (T)beta, use_prev, false, s);
            apgdc::block_sum<kPartials>(s);
            const double* t = s;
            if (!bt) Fy = t[3];
            const double F_lp = 0.5 * A.dt2 * t[6] + t[2];
            if (A.dynamic && t[1] == 0.0) {
                while (isfinite(lipsch)) {  // l+ == y bit for bit (as in k_apgd)
                    lipsch *= 2;
                    ++nbt;
                }
                alpha = 1. / lipsch;
            } else if (A.dynamic && apgdc::sufficient_decrease_fails<T>(F_lp, Fy, t[0], t[1], A.dt2 * t[8], lipsch)) {
                lipsch *= 2;
                alpha = 1. / lipsch;
                bt = true;
                ++nbt;
                if (nbt > 4000) {
                    err = 2;
                    break;
                }
                continue;
            }
            ++ite;
            bt = false;
            if (isfinite(lipsch)) lgood = lipsch;
            last_step = sqrt(t[4]);
            int tmp = ip;
            ip = il;
            il = in_;
            in_ = tmp;
            tmp = jp;
            jp = jl;
            jl = jn;
            jn = tmp;
            if (last_step < A.tol) {
                conv = 1;
                break;
            }
            const double theta1 = 0.5 * (theta * sqrt(4 + theta * theta) - theta * theta);
            beta = theta * (1 - theta) / (theta * theta + theta1);
            theta = theta1;
            if (A.dynamic) {
                if (t[5] > 0) {  // restart, apgd.hpp:200-206
                    beta = 0.0;
                    theta = 1.;
                    ++nrs;
                }
                lipsch *= 0.97;
                alpha = 1. / lipsch;
            }
            use_prev = (beta != 0.0);
            if (ite >= A.max_ite) break;
        }
        // the scene's outputs and its violation max(0, -n.(dt^2 A u + C)) over its contacts
        double vmax = 0.0;
        for (int k = threadIdx.x; k < nc; k += blockDim.x) {
            const long long c = contact_at(k);
            for (int r = 0; r < R; ++r) S.lam_out[R * c + r] = lamb[il][R * c + r];
            if (PROB == kViscous) {
                const int sl = A.slot[c];
                if (sl >= 0) S.lam_out[sl] = lamb[il][sl];
            }
            const int bi[2] = {A.ci[c], A.cj[c]};
            double q3[3] = {0, 0, 0};
            for (int side = 0; side < 2; ++side) {
                if (bi[side] < A.nin) continue;
                const T* uu = ub[jl] + 6 * (long long)(bi[side] - A.nin);
                const double sg = side == 0 ? 1.0 : -1.0;
                if (PROB == kFriction) {
                    const T* P = A.bP + 18 * c + 9 * side;
                    for (int d = 0; d < 3; ++d) {
                        const double vd = (DIM == 2 && d == 2) ? 0.0 : uu[d];
                        q3[d] += sg * (vd + P[d] * uu[3] + P[3 + d] * uu[4] + P[6 + d] * uu[5]);
                    }
                } else {
                    const T* a = (side == 0 ? A.bai : A.baj) + 3 * c;
                    for (int d = 0; d < DIM; ++d) q3[0] += sg * A.bn[3 * c + d] * uu[d];
                    q3[0] += DIM == 3 ? a[0] * uu[3] + a[1] * uu[4] + a[2] * uu[5] : a[2] * uu[5];
                }
            }
            double gap = 0.0;
            if (PROB == kFriction) {
                for (int d = 0; d < DIM; ++d) gap += (A.dt2 * q3[d] + A.cvec[3 * c + d]) * A.bn[3 * c + d];
            } else {
                gap = A.dt2 * q3[0] + A.cvec[c];
            }
            vmax = fmax(vmax, -gap);
        }
        for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x)
            for (int d = 0; d < 6; ++d) S.u_out[6 * (long long)p + d] = ub[jl][6 * (long long)p + d];
        vmax = block_max(vmax);
        if (threadIdx.x == 0) {
            BatchSceneStats& st = S.stats[sc];
            st.contacts = nc;
            st.iterations = ite;
            st.fp32_iterations = 0;
            st.backtracks = nbt;
            st.restarts = nrs;
            st.corrections = 0;
            st.converged = conv && !err;
            st.violation = vmax;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- FP64 helpers

template <int DIM, int PROB>
__global__ void k_particle_pass64(int nin, int na, const int* inc_ptr, const int* inc_idx, const double* coef,
                                  const int* slot, const int* mode, const double* bn, const double* bP,
                                  const double* invm, const double* lam, double* u) {
    GRID_STRIDE(p, na) {
        double w[6] = {0, 0, 0, 0, 0, 0};
        for (int k = inc_ptr[p]; k < inc_ptr[p + 1]; ++k) {
            const unsigned e = (unsigned)inc_idx[k];
            const long long c = e & 0x7fffffffu;
            if (PROB != kFriction && PROB != kViscousFriction) {
                double mu = lam[c];
                if (PROB == kViscous && slot[c] >= 0) mu -= lam[slot[c]];
                for (int d = 0; d < 6; ++d) w[d] += mu * coef[6 * (long long)k + d];
            } else {
                const int side = (int)(e >> 31);
                const double sg = side == 0 ? 1.0 : -1.0;
                const double* P = bP + 18 * c + 9 * side;
                double f[3];
                if (PROB == kViscousFriction) {
                    vf_force<double, DIM>(mode[c], lam + 4 * c, bn + 3 * c, f);
                } else {
                    for (int d = 0; d < 3; ++d) f[d] = lam[3 * c + d];
                }
                for (int d = 0; d < 3; ++d) {
                    w[d] += sg * f[d];
                    w[3 + d] += sg * (P[3 * d] * f[0] + P[3 * d + 1] * f[1] + P[3 * d + 2] * f[2]);
                }
            }
        }
        const double* im = invm + 4 * (long long)p;
        u[6 * p + 0] = im[0] * w[0];
        u[6 * p + 1] = im[0] * w[1];
        u[6 * p + 2] = DIM == 3 ? im[0] * w[2] : 0.0;
        u[6 * p + 3] = im[1] * w[3];
        u[6 * p + 4] = im[2] * w[4];
        u[6 * p + 5] = im[3] * w[5];
    }
}

template <int DIM, int PROB>
__global__ void k_residual64(int nin, const int* ci, const int* cj, const int* slot, const int* mode,
                             const double* bn, const double* bai,
                             const double* baj, const double* bP, const double* cvec, double dt2, const double* u,
                             double* g, unsigned long long* viol_bits, const Sizes* sizes) {
    const int C = sizes->C;
    double vmax = 0.0;
    GRID_STRIDE(c, C) {
        const int bi[2] = {ci[c], cj[c]};
        if (PROB != kFriction && PROB != kViscousFriction) {
            double qy = 0.0;
            for (int s = 0; s < 2; ++s) {
                if (bi[s] < nin) continue;
                const double* uu = u + 6 * (long long)(bi[s] - nin);
                const double* a = (s == 0 ? bai : baj) + 3 * c;
                const double sg = s == 0 ? 1.0 : -1.0;
                for (int d = 0; d < DIM; ++d) qy += sg * bn[3 * c + d] * uu[d];
                if (DIM == 3)
                    qy += a[0] * uu[3] + a[1] * uu[4] + a[2] * uu[5];
                else
                    qy += a[2] * uu[5];
            }
            const double gg = dt2 * qy + cvec[c];
            g[c] = gg;
            if (PROB == kViscous && slot[c] >= 0) g[slot[c]] = -gg;
            vmax = fmax(vmax, -gg);
        } else {
            double q3[3] = {0, 0, 0};
            for (int s = 0; s < 2; ++s) {
                if (bi[s] < nin) continue;
                const double* uu = u + 6 * (long long)(bi[s] - nin);
                const double* P = bP + 18 * c + 9 * s;
                const double sg = s == 0 ? 1.0 : -1.0;
                for (int d = 0; d < 3; ++d) {
                    const double vd = (DIM == 2 && d == 2) ? 0.0 : uu[d];
                    q3[d] += sg * (vd + P[d] * uu[3] + P[3 + d] * uu[4] + P[6 + d] * uu[5]);
                }
            }
            if (PROB == kViscousFriction) {
                // local residual global2local(Q l) + c; the gap n.(Q l + C) from the normal slot
                // of c, which the S term does not touch
                const int md = mode[c];
                double qd[3], ql[4];
                for (int d = 0; d < 3; ++d) qd[d] = dt2 * q3[d];
                vf_local<double, DIM>(md, qd, bn + 3 * c, ql);
                for (int k = 0; k < 4; ++k) g[4 * c + k] = ql[k] + cvec[4 * c + k];
                const double qn = md == 2 ? -ql[0] : ql[0];
                const double gap = qn + (md == 2 ? -cvec[4 * c] : cvec[4 * c]);
                vmax = fmax(vmax, -gap);
                continue;
            }
            double gap = 0.0;
            for (int d = 0; d < 3; ++d) {
                const double gg = dt2 * q3[d] + cvec[3 * c + d];
                g[3 * c + d] = gg;
                if (d < DIM) gap += gg * bn[3 * c + d];
            }
            vmax = fmax(vmax, -gap);
        }
    }
    if (vmax > 0.0) atomicMax(viol_bits, (unsigned long long)__double_as_longlong(vmax));
}

template <int DIM, int PROB, typename TD>
__global__ void k_accumulate(const Sizes* sizes, const double* bn, const int* slot, const int* mode, double* lam,
                             const TD* delta, int first, double mu) {
    const int C = sizes->C;
    GRID_STRIDE(c, C) {
        if (PROB == kViscousFriction) {
            double z[4];
            for (int k = 0; k < 4; ++k) z[k] = (first ? 0.0 : lam[4 * c + k]) + (double)delta[4 * c + k];
            vf_project<DIM>(mode[c], z, bn + 3 * c, mu);
            for (int k = 0; k < 4; ++k) lam[4 * c + k] = z[k];
        } else if (PROB != kFriction) {
            const double v = (first ? 0.0 : lam[c]) + (double)delta[c];
            lam[c] = v > 0.0 ? v : 0.0;
            if (PROB == kViscous && slot[c] >= 0) {
                const long long m = slot[c];
                const double v2 = (first ? 0.0 : lam[m]) + (double)delta[m];
                lam[m] = v2 > 0.0 ? v2 : 0.0;
            }
        } else {
            double z[3], n[3];
            for (int d = 0; d < 3; ++d) {
                z[d] = (first ? 0.0 : lam[3 * c + d]) + (double)delta[3 * c + d];
                n[d] = bn[3 * c + d];
            }
            cone_project<DIM>(z, n, mu);
            for (int d = 0; d < 3; ++d) lam[3 * c + d] = z[d];
        }
    }
}

// ---------------------------------------------------------------- FrictionFixedPoint
// Linear term of one fixed-point solve: c + s_c n_c (the S vector of
// LagrangeMultiplier<FrictionFixedPoint>, lagrange_multiplier.hpp:286-292; dim components).
template <int DIM>
__global__ void k_fixed_point_c(const Sizes* sizes, const double* base, const double* bn, const double* sv,
                                double* cvec) {
    GRID_STRIDE(c, sizes->C) {
        for (int d = 0; d < 3; ++d)
            cvec[3 * c + d] = d < DIM ? base[3 * c + d] + sv[c] * bn[3 * c + d] : base[3 * c + d];
    }
}

// ViscousFriction: the S vector of LagrangeMultiplier<ViscousFriction>
// (lagrange_multiplier.hpp:381-384), dt mu s_c n_c on the f slots of the mode-2 contacts
template <int DIM>
__global__ void k_vf_fixed_point_c(const Sizes* sizes, const double* base, const double* bn, const int* mode,
                                   const double* sv, double dtmu, double* cvec) {
    GRID_STRIDE(c, sizes->C) {
        cvec[4 * c] = base[4 * c];
        for (int d = 0; d < 3; ++d) {
            const long long m = 4 * c + 1 + d;
            cvec[m] = (mode[c] == 2 && d < DIM) ? base[m] + dtmu * sv[c] * bn[3 * c + d] : base[m];
        }
    }
}

// ViscousFriction: s_c = 1 on the contacts at gamma_min before the first solve
// (OptimGradient.hpp:96-107); 0 elsewhere (never read)
__global__ void k_vf_fixed_point_init(const Sizes* sizes, const double* gamma, double gamma_min, double* sv) {
    GRID_STRIDE(c, sizes->C) sv[c] = gamma[c] == gamma_min ? 1. : 0.;
}

// s_c = mu dt before the first solve of a step (OptimGradient.hpp:85-94)
__global__ void k_fixed_point_init(const Sizes* sizes, double* sv, double v) {
    GRID_STRIDE(c, sizes->C) sv[c] = v;
}

// After a solve (OptimGradient.hpp:117-176): U = v + dt M^-1 B^T l of the active bodies,
// (A U)_c the contact's relative velocity (active bodies only, AMatrix::mat_mult), s_c =
// scale |(A U)_c - n_c ((A U)_c.n_c)| over dim components; per block the sums of
// (s_new - s_old)^2 and s_new^2 in a fixed order for the stopping test.  FrictionFixedPoint:
// scale = mu dt, every contact; ViscousFriction (:178-250): scale = 1, only the contacts
// whose gamma equals gamma_min (gamma != nullptr).
template <int DIM>
__global__ void __launch_bounds__(kApgdThreads) k_fixed_point_s(const Sizes* sizes, int nin, const int* ci,
                                                                const int* cj, const double* bn, const double* bP,
                                                                const double* v, const double* omega,
                                                                const double* u, double dt, double scale,
                                                                const double* gamma, double gamma_min, double* sv,
                                                                double* part) {
    const int C = sizes->C;
    double s[kPartials] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    GRID_STRIDE(c, C) {
        if (gamma && gamma[c] != gamma_min) continue;
        const int bi[2] = {ci[c], cj[c]};
        double au[3] = {0, 0, 0};
        for (int side = 0; side < 2; ++side) {
            const int b = bi[side];
            if (b < nin) continue;
            const double* uu = u + 6 * (long long)(b - nin);
            double U[6];
            for (int d = 0; d < 3; ++d) {
                U[d] = (DIM == 2 && d == 2) ? 0.0 : v[3 * (long long)b + d] + dt * uu[d];
                U[3 + d] = (DIM == 2 && d < 2) ? 0.0 : omega[3 * (long long)b + d] + dt * uu[3 + d];
            }
            const double* P = bP + 18 * c + 9 * side;
            const double sg = side == 0 ? 1.0 : -1.0;
            for (int d = 0; d < 3; ++d) au[d] += sg * (U[d] + P[d] * U[3] + P[3 + d] * U[4] + P[6 + d] * U[5]);
        }
        double dn = 0.0;
        for (int d = 0; d < DIM; ++d) dn += au[d] * bn[3 * c + d];
        double t2 = 0.0;
        for (int d = 0; d < DIM; ++d) {
            const double t = au[d] - bn[3 * c + d] * dn;
            t2 += t * t;
        }
        const double snew = scale * sqrt(t2);
        const double ds = snew - sv[c];
        s[0] += ds * ds;
        s[1] += snew * snew;
        sv[c] = snew;
    }
    block_sum(s);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = s[0];
        part[2 * blockIdx.x + 1] = s[1];
    }
}

template <typename Src, typename Dst>
__global__ void k_convert(const Src* in, Dst* out, long long n_max, const int* n_dev, int mult) {
    const long long n = n_dev ? (long long)(*n_dev) * mult : n_max;
    GRID_STRIDE(k, n) { out[k] = (Dst)in[k]; }
}

int grid_blocks(long long n) {
    long long b = (n + 255) / 256;
    if (b < 1) b = 1;
    return (int)(b < 16 * kSMs ? b : 16 * kSMs);
}

template <typename T, int DIM, int PROB>
cudaError_t launch_apgd_t(ApgdArgs<T>& A, int nblocks, cudaStream_t s) {
    void* args[] = {&A};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(kApgdThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    (void)args;
    g_apgd_launches += 1;
    return cudaLaunchKernelEx(&cfg, k_apgd<T, DIM, PROB>, A);
}

template <typename T, int DIM, int PROB>
int max_blocks_t() {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_apgd<T, DIM, PROB>, kApgdThreads, 0);
    int dev = 0, sms = kSMs;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return per_sm * sms;
}

}  // namespace

cudaError_t launch_apgd_batch6(const Bodies& b, const StepParams& p, const ApgdSettings& st, const Contacts& c,
                               const Assembly& a, SolveBuffers<double>& sb, const double* invm,
                               const Batch6Scenes& S, cudaStream_t s) {
    ApgdArgs<double> A{};
    A.nin = b.nin;
    A.na = b.n - b.nin;
    A.ci = c.ci;
    A.cj = c.cj;
    A.slot = a.slot;
    A.mode = a.vflag;
    A.bn = sb.bn;
    A.bai = sb.bai;
    A.baj = sb.baj;
    A.bP = sb.bP;
    A.cvec = sb.cvec;
    A.shift = nullptr;
    A.inc_ptr = sb.inc_ptr;
    A.inc_idx = sb.inc_idx;
    A.inc_coef = sb.inc_coef;
    A.invm = invm;
    A.lam0 = sb.lam[0];
    A.lam1 = sb.lam[1];
    A.lam2 = sb.lam[2];
    A.u0 = sb.u[0];
    A.u1 = sb.u[1];
    A.u2 = sb.u[2];
    A.g = sb.g;
    A.alpha = st.alpha;
    A.tol = st.tol;
    A.dt2 = st.dt * st.dt;
    A.mu = st.mu;
    A.curvature_start = st.curvature_start;
    A.max_ite = st.max_ite;
    A.dynamic = st.dynamic;
    const int grid = std::max(1, S.n_scenes);
    if (p.problem == kFriction) {
        if (p.dim == 3)
            k_apgd_batch6<3, kFriction><<<grid, kBatch6Threads, 0, s>>>(A, S);
        else
            k_apgd_batch6<2, kFriction><<<grid, kBatch6Threads, 0, s>>>(A, S);
    } else if (p.problem == kViscous) {
        if (p.dim == 3)
            k_apgd_batch6<3, kViscous><<<grid, kBatch6Threads, 0, s>>>(A, S);
        else
            k_apgd_batch6<2, kViscous><<<grid, kBatch6Threads, 0, s>>>(A, S);
    } else {
        return cudaErrorInvalidValue;
    }
    g_apgd_launches += 1;
    return cudaGetLastError();
}

int apgd_max_blocks(int problem, int dim, bool fp32) {
#define MB(T, D, P) \
    if (dim == D && problem == P) return max_blocks_t<T, D, P>();
    if (fp32) {
        MB(float, 2, 0) MB(float, 2, 1) MB(float, 2, 2) MB(float, 2, 4)
        MB(float, 3, 0) MB(float, 3, 1) MB(float, 3, 2) MB(float, 3, 4)
    } else {
        MB(double, 2, 0) MB(double, 2, 1) MB(double, 2, 2) MB(double, 2, 4)
        MB(double, 3, 0) MB(double, 3, 1) MB(double, 3, 2) MB(double, 3, 4)
    }
#undef MB
    return 0;
}

template <typename T>
cudaError_t launch_apgd_invm(const Bodies& b, const StepParams& p, const ApgdSettings& st, const Contacts& c,
                             const Assembly& a, SolveBuffers<T>& sb, const T* invm, const Sizes* sizes, int nblocks,
                             cudaStream_t s) {
    ApgdArgs<T> A;
    A.nin = b.nin;
    A.na = b.n - b.nin;
    A.ci = c.ci;
    A.cj = c.cj;
    A.slot = a.slot;
    A.mode = a.vflag;
    A.bn = sb.bn;
    A.bai = sb.bai;
    A.baj = sb.baj;
    A.bP = sb.bP;
    A.cvec = sb.cvec;
    A.shift = sb.shift;
    A.inc_ptr = sb.inc_ptr;
    A.inc_idx = sb.inc_idx;
    A.inc_coef = sb.inc_coef;
    A.invm = invm;
    A.lam0 = sb.lam[0];
    A.lam1 = sb.lam[1];
    A.lam2 = sb.lam[2];
    A.u0 = sb.u[0];
    A.u1 = sb.u[1];
    A.u2 = sb.u[2];
    A.g = sb.g;
    A.partials = sb.partials;
    A.bar = sb.barrier;
    A.result = sb.result;
    A.sizes = sizes;
    A.alpha = st.alpha;
    A.tol = st.tol;
    A.dt2 = st.dt * st.dt;
    A.mu = st.mu;
    A.curvature_start = st.curvature_start;
    A.stall = st.stall;
    A.max_ite = st.max_ite;
    A.dynamic = st.dynamic;
#define LA(D, P) \
    if (p.dim == D && p.problem == P) return launch_apgd_t<T, D, P>(A, nblocks, s);
    LA(2, 0) LA(2, 1) LA(2, 2) LA(2, 4) LA(3, 0) LA(3, 1) LA(3, 2) LA(3, 4)
#undef LA
    return cudaErrorInvalidValue;
}

template cudaError_t launch_apgd_invm<double>(const Bodies&, const StepParams&, const ApgdSettings&, const Contacts&,
                                              const Assembly&, SolveBuffers<double>&, const double*, const Sizes*, int,
                                              cudaStream_t);
template cudaError_t launch_apgd_invm<float>(const Bodies&, const StepParams&, const ApgdSettings&, const Contacts&,
                                             const Assembly&, SolveBuffers<float>&, const float*, const Sizes*, int,
                                             cudaStream_t);

void launch_particle_pass64(const Bodies& b, const StepParams& p, const Contacts&, const Assembly& a,
                            const Incidence& inc, const double* invm, const double* lam, double* u, cudaStream_t s) {
    const int na = b.n - b.nin;
    if (na <= 0) return;
#define PP(D, P) \
    if (p.dim == D && p.problem == P) \
        k_particle_pass64<D, P><<<grid_blocks(na), 256, 0, s>>>(b.nin, na, inc.ptr, inc.idx, inc.coef, a.slot, \
                                                                a.vflag, a.bn, a.bP, invm, lam, u);
    PP(2, 0) PP(2, 1) PP(2, 2) PP(2, 4) PP(3, 0) PP(3, 1) PP(3, 2) PP(3, 4)
#undef PP
    g_apgd_launches += 1;
}

void launch_residual64(const Bodies& b, const StepParams& p, const Contacts& c, const Assembly& a, const double* u,
                       double* g, unsigned long long* viol_bits, const Sizes* sizes, long long c_cap, cudaStream_t s) {
    const double dt2 = p.dt * p.dt;
#define RR(D, P) \
    if (p.dim == D && p.problem == P) \
        k_residual64<D, P><<<grid_blocks(c_cap), 256, 0, s>>>(b.nin, c.ci, c.cj, a.slot, a.vflag, a.bn, a.bai, \
                                                              a.baj, a.bP, a.cvec, dt2, u, g, viol_bits, sizes);
    RR(2, 0) RR(2, 1) RR(2, 2) RR(2, 4) RR(3, 0) RR(3, 1) RR(3, 2) RR(3, 4)
#undef RR
    g_apgd_launches += 1;
}

void launch_fixed_point_c(const StepParams& p, const Assembly& a, const double* base, const double* sv,
                          const Sizes* sizes, long long c_cap, cudaStream_t s) {
    if (p.problem == kViscousFriction) {
        const double dtmu = p.dt * p.mu;
        if (p.dim == 3)
            k_vf_fixed_point_c<3><<<grid_blocks(c_cap), 256, 0, s>>>(sizes, base, a.bn, a.vflag, sv, dtmu, a.cvec);
        else
            k_vf_fixed_point_c<2><<<grid_blocks(c_cap), 256, 0, s>>>(sizes, base, a.bn, a.vflag, sv, dtmu, a.cvec);
        g_apgd_launches += 1;
        return;
    }
    if (p.dim == 3)
        k_fixed_point_c<3><<<grid_blocks(c_cap), 256, 0, s>>>(sizes, base, a.bn, sv, a.cvec);
    else
        k_fixed_point_c<2><<<grid_blocks(c_cap), 256, 0, s>>>(sizes, base, a.bn, sv, a.cvec);
    g_apgd_launches += 1;
}
void launch_fixed_point_init(double* sv, double v, const Sizes* sizes, long long c_cap, cudaStream_t s) {
    k_fixed_point_init<<<grid_blocks(c_cap), 256, 0, s>>>(sizes, sv, v);
    g_apgd_launches += 1;
}
void launch_vf_fixed_point_init(double* sv, const double* gamma, double gamma_min, const Sizes* sizes,
                                long long c_cap, cudaStream_t s) {
    k_vf_fixed_point_init<<<grid_blocks(c_cap), 256, 0, s>>>(sizes, gamma, gamma_min, sv);
    g_apgd_launches += 1;
}
int fixed_point_blocks(long long c_cap) {
    const long long b = (c_cap + kApgdThreads - 1) / kApgdThreads;
    return (int)std::max<long long>(1, std::min<long long>(b, kFixedPointMaxBlocks));
}
void launch_fixed_point_s(const Bodies& b, const StepParams& p, const Contacts& c, const Assembly& a, const double* u,
                          double* sv, double* part, const Sizes* sizes, long long c_cap, cudaStream_t s) {
    const int nb = fixed_point_blocks(c_cap);
    const bool vf = p.problem == kViscousFriction;
    const double scale = vf ? 1.0 : p.mu * p.dt;
    const double* gam = vf ? c.gamma : nullptr;
    if (p.dim == 3)
        k_fixed_point_s<3><<<nb, kApgdThreads, 0, s>>>(sizes, b.nin, c.ci, c.cj, a.bn, a.bP, b.v, b.omega, u, p.dt,
                                                       scale, gam, p.gamma_min, sv, part);
    else
        k_fixed_point_s<2><<<nb, kApgdThreads, 0, s>>>(sizes, b.nin, c.ci, c.cj, a.bn, a.bP, b.v, b.omega, u, p.dt,
                                                       scale, gam, p.gamma_min, sv, part);
    g_apgd_launches += 1;
}

template <typename TD>
void launch_accumulate(const StepParams& p, const Contacts&, const Assembly& a, double* lam64, const TD* delta,
                       const Sizes* sizes, long long c_cap, int first, cudaStream_t s) {
#define AC(D, P) \
    if (p.dim == D && p.problem == P) \
        k_accumulate<D, P, TD><<<grid_blocks(c_cap), 256, 0, s>>>(sizes, a.bn, a.slot, a.vflag, lam64, delta, \
                                                                  first, p.mu);
    AC(2, 0) AC(2, 1) AC(2, 2) AC(2, 4) AC(3, 0) AC(3, 1) AC(3, 2) AC(3, 4)
#undef AC
    g_apgd_launches += 1;
}
template void launch_accumulate<float>(const StepParams&, const Contacts&, const Assembly&, double*, const float*,
                                       const Sizes*, long long, int, cudaStream_t);
template void launch_accumulate<double>(const StepParams&, const Contacts&, const Assembly&, double*, const double*,
                                        const Sizes*, long long, int, cudaStream_t);

template <typename Src, typename Dst>
void launch_convert(const Src* in, Dst* out, long long n_max, const int* n_dev, int mult, cudaStream_t s) {
    k_convert<Src, Dst><<<grid_blocks(n_max), 256, 0, s>>>(in, out, n_max, n_dev, mult);
    g_apgd_launches += 1;
}
template void launch_convert<double, float>(const double*, float*, long long, const int*, int, cudaStream_t);
template void launch_convert<float, double>(const float*, double*, long long, const int*, int, cudaStream_t);

}  // namespace scopi_gpu
