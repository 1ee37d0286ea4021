// apgd_batch.cu -- one launch per time step for a batch of independent scenes.
//
// Each CTA solves one scene's contact QP with the same APGD iteration as apgd_sph.cu
// (apgd::operator(), include/scopi/solvers/apgd.hpp:148-221, torque-free rows): the two
// passes are separated by block barriers instead of grid barriers, and every scene
// iterates until its own stopping test holds (per-scene convergence).  Scenes are taken
// largest first so the long solves start early.  The mixed form runs the iterations in
// FP32 and, inside the same CTA, recomputes the scene's residual and violation in FP64
// and reruns the FP32 solve on the correction until the violation target holds.
// The contacts of scene s are two contiguous ranges of the global (i, j)-sorted list:
// the rows of its obstacles and the rows of its active bodies.
#include <cooperative_groups.h>

#include <algorithm>

#include "apgd_common.cuh"

namespace scopi_gpu {

static long long g_batch_launches = 0;
long long apgd_batch_launches() { return g_batch_launches; }

namespace {
using namespace apgdc;

__device__ __forceinline__ float4 bld4(const float4* p) { return *p; }
__device__ __forceinline__ dvec4 bld4(const dvec4* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = q[0], b = q[1];
    return dvec4{a.x, a.y, b.x, b.y};
}
__device__ __forceinline__ void bst4(float4* p, float x, float y, float z) { *p = make_float4(x, y, z, 0.f); }
__device__ __forceinline__ void bst4(dvec4* p, double x, double y, double z) {
    double2* q = reinterpret_cast<double2*>(p);
    q[0] = make_double2(x, y);
    q[1] = make_double2(z, 0.0);
}
__device__ __forceinline__ int bidx(float w) { return __float_as_int(w); }
__device__ __forceinline__ int bidx(double w) { return (int)__double_as_longlong(w); }

template <typename T>
struct BatchArgs {
    int nin;
    int n_scenes;
    int n_big;                        // paired layout: the n_big largest scenes take two CTAs each
    const int* order;                 // scene order (largest first)
    const int* sc_p0;                 // per scene: active bodies [p0, p1) (active index)
    const int* sc_p1;
    const int* sc_o0;                 // per scene: obstacle contacts [o0, o1) and active contacts [a0, a1)
    const int* sc_o1;
    const int* sc_a0;
    const int* sc_a1;
    const int2* cij;
    V4<T>* nc;                        // (n, c) in T; c is replaced by the residual for corrections
    const dvec4* nc64;                // (n, c) in FP64
    const int* inc_ptr;
    const V4<T>* inc;
    const dvec4* inc64;
    const double* invm;               // stride 4, component 0 = 1/m
    T* lam[3];
    V4<T>* u[4];
    double* lam64;                    // FP64 multipliers (output, and the offset of corrections)
    dvec4* ufin;                      // FP64 M^-1 B^T lambda (output)
    BatchSceneStats* stats;
    const Sizes* sizes;
    double alpha, tol, dt2, viol_tol;
    long long max_ite;
    int dynamic;
    int max_corrections;
    int curvature_start;
};

struct BState {
    double alpha, lipsch, theta, beta, beta_n, theta1, Fy, last_step, lgood;
    double tk[4];
    long long ite, nbt, nrs;
    int il, ip, in_, jL, jN, jY, jYN, bt, use_prev, restart, done, conv;
};

template <typename T>
__device__ __forceinline__ T* lam_buf(const BatchArgs<T>& A, int k) {
    return A.lam[k];
}

// contact k of scene (obstacle rows first, then active rows)
__device__ __forceinline__ int scene_contact(int k, int o0, int n0, int a0) { return k < n0 ? o0 + k : a0 + (k - n0); }

// The threads that solve one scene: one CTA (CS = 1), or a cluster of CS CTAs on CS SMs,
// which spreads a large scene's passes over the load/store bandwidth of CS SMs (one SM
// streams the ~1 MB per iteration of a 5000-disk scene at ~60 GB/s).  sync() orders the
// scene's global memory at cluster scope (barrier.cluster arrive.release / wait.acquire);
// reduce<NP>(v, slot) sums v over the scene's threads, the CTAs' partial sums added in rank
// order, into thread 0 of every CTA, so that every CTA takes the same decisions.  `slot`
// alternates between consecutive reductions: a CTA's partials are read through distributed
// shared memory by the others before it can overwrite that slot.
template <int CS>
struct Grp {
    int rank;
    __device__ __forceinline__ int tid() const { return rank * (int)blockDim.x + (int)threadIdx.x; }
    __device__ __forceinline__ int size() const { return CS * (int)blockDim.x; }
    __device__ __forceinline__ void sync() const {
        if (CS == 1)
            __syncthreads();
        else
            asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
    }
    template <int NP>
    __device__ __forceinline__ void reduce(double* v, int slot) const {
        block_reduce_t0<NP>(v);
        if (CS == 1) return;
        __shared__ double part[3][8];
        if (threadIdx.x == 0)
            for (int k = 0; k < NP; ++k) part[slot][k] = v[k];
        sync();
        if (threadIdx.x == 0) {
            cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
            double t[NP];
            for (int k = 0; k < NP; ++k) t[k] = 0.0;
            for (int r = 0; r < CS; ++r) {
                const double* rp = cl.map_shared_rank(&part[slot][0], r);
                for (int k = 0; k < NP; ++k) t[k] += rp[k];
            }
            for (int k = 0; k < NP; ++k) v[k] = t[k];
        }
    }
};

// One APGD solve of the scene on the T data; `shift` (FP64 lambda so far) turns it into the
// correction problem.  Returns in S the iteration counts; the result is lam[S.il], u[S.jL].
// KB independent contacts / incidence records per thread are in flight: the passes are
// bound by the latency of dependent L2 gathers, not by bandwidth.
template <typename T, int DIM, int KB, int CS>
__device__ void solve_scene(const BatchArgs<T>& A, const Grp<CS>& G, BState& S, int o0, int n0, int a0, int nct,
                            int p0, int p1, const double* shift, double alpha0) {
    if (threadIdx.x == 0) {
        S.alpha = alpha0;
        S.lipsch = 1.0 / alpha0;
        S.lgood = S.lipsch;
        S.theta = 1.0;
        S.beta = 0.0;
        S.beta_n = 0.0;
        S.theta1 = 1.0;
        S.Fy = 0.0;
        S.last_step = 0.0;
        S.ite = S.nbt = S.nrs = 0;
        S.il = 0; S.ip = 1; S.in_ = 2;
        S.jL = 0; S.jN = 1; S.jY = 2; S.jYN = 3;
        S.bt = 0;
        S.use_prev = 0;
        S.restart = 0;
        S.done = 0;
        S.conv = 0;
    }
    // cold start: lambda = lambda_prev = 0, u(lambda) = u(y) = 0 (apgd.hpp:152-159)
    const int tid = G.tid(), nt = G.size();
    for (int k = tid; k < nct; k += nt) {
        const int c = scene_contact(k, o0, n0, a0);
        A.lam[0][c] = (T)0;
        A.lam[1][c] = (T)0;
    }
    for (int p = p0 + tid; p < p1; p += nt) {
        bst4(A.u[0] + p, (T)0, (T)0, (T)0);
        bst4(A.u[2] + p, (T)0, (T)0, (T)0);
    }
    G.sync();
    if (A.curvature_start) {
        // initial step from the curvature along the first descent direction d (kept in the
        // candidate buffer, which the first contact pass overwrites)
        T* dbuf = A.lam[2];
        double r2[2] = {0.0, 0.0};
        for (int k = tid; k < nct; k += nt) {
            const int c = scene_contact(k, o0, n0, a0);
            const T d = first_descent<T>(bld4(A.nc + c).w, shift, c);
            dbuf[c] = d;
            r2[0] += (double)d * (double)d;
        }
        G.sync();
        for (int p = p0 + tid; p < p1; p += nt) {
            T w0 = 0, w1 = 0, w2 = 0;
            for (int k = A.inc_ptr[p]; k < A.inc_ptr[p + 1]; ++k) {
                const V4<T> e = bld4(A.inc + k);
                const T mu = dbuf[bidx(e.w)];
                w0 += mu * e.x;
                w1 += mu * e.y;
                if (DIM == 3) w2 += mu * e.z;
            }
            r2[1] += A.invm[4 * (long long)p] * ((double)w0 * w0 + (double)w1 * w1 + (double)w2 * w2);
        }
        G.template reduce<2>(r2, 2);
        if (threadIdx.x == 0) {
            double l;
            if (initial_lipschitz(r2[0], r2[1], A.dt2, l)) {
                S.lipsch = l;
                S.alpha = 1.0 / l;
                S.lgood = l;
            }
        }
        __syncthreads();
    }
    for (;;) {
        const double alpha = S.alpha;
        const bool bt = S.bt != 0, use_prev = S.use_prev != 0;
        const T beta = (T)S.beta;
        const T* lam = A.lam[S.il];
        const T* lprev = A.lam[S.ip];
        T* lnew = A.lam[S.in_];
        const V4<T>* uY = A.u[S.jY];
        double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int kb = tid; kb < nct; kb += KB * nt) {
            int c[KB];
            int2 ij[KB];
            V4<T> n[KB];
            T lm[KB], lq[KB], qy[KB];
#pragma unroll
            for (int q = 0; q < KB; ++q) {
                const int k = kb + q * nt;
                c[q] = k < nct ? scene_contact(k, o0, n0, a0) : -1;
                ij[q] = make_int2(-1, -1);
                if (c[q] >= 0) {
                    ij[q] = A.cij[c[q]];
                    n[q] = bld4(A.nc + c[q]);
                    lm[q] = lam[c[q]];
                    lq[q] = use_prev ? lprev[c[q]] : (T)0;
                }
            }
#pragma unroll
            for (int q = 0; q < KB; ++q) {
                qy[q] = (T)0;
                if (c[q] < 0) continue;
                if (ij[q].x >= A.nin) {
                    const V4<T> ui = bld4(uY + (ij[q].x - A.nin));
                    qy[q] += n[q].x * ui.x + n[q].y * ui.y + (DIM == 3 ? n[q].z * ui.z : (T)0);
                }
                if (ij[q].y >= A.nin) {
                    const V4<T> uj = bld4(uY + (ij[q].y - A.nin));
                    qy[q] -= n[q].x * uj.x + n[q].y * uj.y + (DIM == 3 ? n[q].z * uj.z : (T)0);
                }
            }
#pragma unroll
            for (int q = 0; q < KB; ++q) {
                if (c[q] < 0) continue;
                const T qq = qy[q] * (T)A.dt2;
                const T y = use_prev ? lm[q] + beta * (lm[q] - lq[q]) : lm[q];
                const T gm = qq + n[q].w;
                T lp;
                if (shift) {
                    const double sh = shift[c[q]];
                    double z = sh + ((double)y - alpha * (double)gm);
                    z = z > 0.0 ? z : 0.0;
                    lp = (T)(z - sh);
                } else {
                    const T z = y - (T)alpha * gm;
                    lp = z > (T)0 ? z : (T)0;
                }
                lnew[c[q]] = lp;
                const double dly = (double)lp - (double)y, dll = (double)lp - (double)lm[q];
                s[0] += (double)gm * dly;
                s[1] += dly * dly;
                s[2] += (double)n[q].w * (double)lp;
                if (!bt) s[3] += (double)y * (0.5 * (double)qq + (double)n[q].w);
                s[4] += dll * dll;
                s[5] += (double)gm * dll;
                s[6] += (double)lp * (double)lp;
            }
        }
        G.template reduce<8>(s, 0);
        if (threadIdx.x == 0) {
            const double th = S.theta;
            S.theta1 = 0.5 * (th * sqrt(4 + th * th) - th * th);
            S.restart = (A.dynamic && s[5] > 0) ? 1 : 0;
            S.beta_n = S.restart ? 0.0 : th * (1 - th) / (th * th + S.theta1);
            if (!bt) S.Fy = s[3];
            S.last_step = s[4];
            S.tk[0] = s[0];
            S.tk[1] = s[1];
            S.tk[2] = s[2];
            S.tk[3] = s[6];
        }
        __syncthreads();
        const V4<T>* uL = A.u[S.jL];
        V4<T>* uN = A.u[S.jN];
        V4<T>* uYN = A.u[S.jYN];
        const T bn_ = (T)S.beta_n;
        double sw = 0.0, sq = 0.0;
        for (int p = p0 + tid; p < p1; p += nt) {
            V4<T> ul, uy;
            if (bn_ != (T)0) ul = bld4(uL + p);
            if (sizeof(T) == 4) uy = bld4(uY + p);
            T w0 = 0, w1 = 0, w2 = 0;
            const int k0 = A.inc_ptr[p], k1 = A.inc_ptr[p + 1];
            for (int kb = k0; kb < k1; kb += KB) {
                V4<T> e[KB];
                T mu[KB];
#pragma unroll
                for (int q = 0; q < KB; ++q)
                    if (kb + q < k1) e[q] = bld4(A.inc + kb + q);
#pragma unroll
                for (int q = 0; q < KB; ++q) mu[q] = kb + q < k1 ? lnew[bidx(e[q].w)] : (T)0;
#pragma unroll
                for (int q = 0; q < KB; ++q) {
                    if (kb + q >= k1) continue;
                    w0 += mu[q] * e[q].x;
                    w1 += mu[q] * e[q].y;
                    if (DIM == 3) w2 += mu[q] * e[q].z;
                }
            }
            const T im = (T)A.invm[4 * (long long)p];
            const T v0 = im * w0, v1 = im * w1, v2 = im * w2;
            bst4(uN + p, v0, v1, v2);
            sw += (double)w0 * (double)v0 + (double)w1 * (double)v1 + (double)w2 * (double)v2;
            if (sizeof(T) == 4) {
                // m |u(l+) - u(y)|^2: the curvature d^T Q d / dt^2 along d = l+ - y
                const double d0 = (double)v0 - (double)uy.x, d1 = (double)v1 - (double)uy.y,
                             d2 = (double)v2 - (double)uy.z;
                sq += (d0 * d0 + d1 * d1 + d2 * d2) / (double)im;
            }
            if (bn_ != (T)0) {
                bst4(uYN + p, v0 + bn_ * (v0 - ul.x), v1 + bn_ * (v1 - ul.y), v2 + bn_ * (v2 - ul.z));
            } else {
                bst4(uYN + p, v0, v1, v2);
            }
        }
        double sw1[2] = {sw, sq};
        G.template reduce<2>(sw1, 1);
        if (threadIdx.x == 0) {
            const double F_lp = 0.5 * A.dt2 * sw1[0] + S.tk[2];
            bool accept = true;
            if (A.dynamic && S.tk[1] == 0.0) {
                double lip = S.lipsch, al = S.alpha;
                long long nbt = S.nbt;
                overflow_cascade(lip, al, nbt);
                S.lipsch = lip;
                S.alpha = al;
                S.nbt = nbt;
            } else if (A.dynamic &&
                       sufficient_decrease_fails<T>(F_lp, S.Fy, S.tk[0], S.tk[1], A.dt2 * sw1[1], S.lipsch)) {
                S.lipsch *= 2;
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
                    const double floor32 = 4.0 * 1.1920929e-7 * sqrt(S.tk[3]);
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

// FP64 residual of the scene at lambda64: u = M^-1 B^T lambda (into ufin), g = dt^2 B u + c,
// violation = max(0, -min g).  Writes g into nc[c].w (the next correction's linear term).
template <typename T, int DIM, int CS>
__device__ double residual_scene(const BatchArgs<T>& A, const Grp<CS>& G, int o0, int n0, int a0, int nct, int p0,
                                 int p1, bool write_linear_term) {
    const int tid = G.tid(), nt = G.size();
    for (int p = p0 + tid; p < p1; p += nt) {
        double w0 = 0, w1 = 0, w2 = 0;
        for (int k = A.inc_ptr[p]; k < A.inc_ptr[p + 1]; ++k) {
            const dvec4 e = bld4(A.inc64 + k);
            const double mu = A.lam64[bidx(e.w)];
            w0 += mu * e.x;
            w1 += mu * e.y;
            if (DIM == 3) w2 += mu * e.z;
        }
        const double im = A.invm[4 * (long long)p];
        bst4(A.ufin + p, im * w0, im * w1, im * w2);
    }
    G.sync();
    double vmax[1] = {0.0};
    for (int k = tid; k < nct; k += nt) {
        const int c = scene_contact(k, o0, n0, a0);
        const int2 ij = A.cij[c];
        const dvec4 n = bld4(A.nc64 + c);
        double q = 0.0;
        if (ij.x >= A.nin) {
            const dvec4 ui = bld4(A.ufin + (ij.x - A.nin));
            q += n.x * ui.x + n.y * ui.y + (DIM == 3 ? n.z * ui.z : 0.0);
        }
        if (ij.y >= A.nin) {
            const dvec4 uj = bld4(A.ufin + (ij.y - A.nin));
            q -= n.x * uj.x + n.y * uj.y + (DIM == 3 ? n.z * uj.z : 0.0);
        }
        const double g = A.dt2 * q + n.w;
        vmax[0] = fmax(vmax[0], -g);
        if (write_linear_term) A.nc[c].w = (T)g;
    }
    // block max (fixed order)
    __shared__ double red[32];
    double v = vmax[0];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    __syncthreads();
    if (CS > 1) {
        // the max over the cluster's CTAs, read by every thread through distributed shared memory
        __shared__ double cm;
        if (threadIdx.x == 0) cm = m;
        G.sync();
        cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
        m = 0.0;
        for (int r = 0; r < CS; ++r) m = fmax(m, *cl.map_shared_rank(&cm, r));
        G.sync();  // no CTA overwrites cm before all have read it
    }
    return m;
}

// Two CTAs per SM at 256 and 512 threads (all 256 scenes of the benchmark batch resident
// at once on 148 SMs), one at 1024; loads in flight per thread chosen to fit the registers.
template <int BT>
struct BatchMinBlocks {
    static constexpr int value = BT <= 512 ? 2 : 1;
};

// KB (the tile): independent contacts / incidence records each thread keeps in flight
// One scene's solve (main solve, FP64 residual, corrections) by the group G and its stats.
template <typename T, int DIM, int KB, int CS>
__device__ void batch_scene(const BatchArgs<T>& A, const Grp<CS>& G, BState& S, int scene) {
    const int tid = G.tid(), nt = G.size();
    const int p0 = A.sc_p0[scene], p1 = A.sc_p1[scene];
    const int o0 = A.sc_o0[scene], o1 = A.sc_o1[scene], a0 = A.sc_a0[scene], a1 = A.sc_a1[scene];
    const int n0 = o1 - o0, nct = n0 + (a1 - a0);
    long long iters = 0, f32 = 0, nbt = 0, nrs = 0;
    int corr = 0, conv = 1;
    double viol = 0.0;
    if (nct > 0) {
        solve_scene<T, DIM, KB, CS>(A, G, S, o0, n0, a0, nct, p0, p1, nullptr, A.alpha);
        iters += S.ite;
        nbt += S.nbt;
        nrs += S.nrs;
        conv = conv && S.conv;
        if (sizeof(T) == 4) f32 += S.ite;
        // lambda64 <- lambda (FP32 solves: projected onto R+ in FP64)
        const T* lres = A.lam[S.il];
        for (int k = tid; k < nct; k += nt) {
            const int c = scene_contact(k, o0, n0, a0);
            const double v = (double)lres[c];
            A.lam64[c] = v > 0.0 ? v : 0.0;
        }
        G.sync();
        if (sizeof(T) == 8) {
            viol = residual_scene<T, DIM, CS>(A, G, o0, n0, a0, nct, p0, p1, false);
        } else {
            for (;;) {
                viol = residual_scene<T, DIM, CS>(A, G, o0, n0, a0, nct, p0, p1, true);
                if (viol <= A.viol_tol || corr >= A.max_corrections) break;
                // the correction starts from the step size the previous solve ended with
                const double a_next = 1.0 / S.lgood;
                G.sync();
                solve_scene<T, DIM, KB, CS>(A, G, S, o0, n0, a0, nct, p0, p1, A.lam64, a_next);
                iters += S.ite;
                f32 += S.ite;
                nbt += S.nbt;
                nrs += S.nrs;
                conv = conv && S.conv;
                ++corr;
                const T* dres = A.lam[S.il];
                for (int k = tid; k < nct; k += nt) {
                    const int c = scene_contact(k, o0, n0, a0);
                    const double v = A.lam64[c] + (double)dres[c];
                    A.lam64[c] = v > 0.0 ? v : 0.0;
                }
                G.sync();
            }
            // restore the linear term of the scene's packed records for the next step's reuse
            for (int k = tid; k < nct; k += nt) {
                const int c = scene_contact(k, o0, n0, a0);
                A.nc[c].w = (T)A.nc64[c].w;
            }
        }
    } else {
        for (int p = p0 + tid; p < p1; p += nt) bst4(A.ufin + p, 0.0, 0.0, 0.0);
    }
    if (G.rank == 0 && threadIdx.x == 0) {
        BatchSceneStats& st = A.stats[scene];
        st.contacts = nct;
        st.iterations = iters;
        st.fp32_iterations = f32;
        st.backtracks = nbt;
        st.restarts = nrs;
        st.corrections = corr;
        st.converged = conv;
        st.violation = viol;
    }
}

// one CTA per scene, scenes largest first
template <typename T, int DIM, int BT, int KB>
__global__ void __launch_bounds__(BT, BatchMinBlocks<BT>::value) k_apgd_batch(BatchArgs<T> A) {
    if (A.sizes->overflow) return;  // the step is redone after the buffers grow
    __shared__ BState S;
    Grp<1> G;
    G.rank = 0;
    batch_scene<T, DIM, KB, 1>(A, G, S, A.order[blockIdx.x]);
}

// Paired layout, launched as clusters of two CTAs: cluster q < n_big solves the q-th largest
// scene with both CTAs (its passes on two SMs); every later cluster solves two of the other
// scenes, one per CTA (those never meet a cluster barrier).
template <typename T, int DIM, int BT, int KB>
__global__ void __launch_bounds__(BT, BatchMinBlocks<BT>::value) k_apgd_batch_pairs(BatchArgs<T> A) {
    if (A.sizes->overflow) return;  // all CTAs of a cluster alike
    __shared__ BState S;
    const int rank = (int)cooperative_groups::this_cluster().block_rank();
    const int q = blockIdx.x / 2;
    if (q < A.n_big) {
        Grp<2> G;
        G.rank = rank;
        batch_scene<T, DIM, KB, 2>(A, G, S, A.order[q]);
    } else {
        const int j = A.n_big + 2 * (q - A.n_big) + rank;
        if (j >= A.n_scenes) return;
        Grp<1> G;
        G.rank = 0;
        batch_scene<T, DIM, KB, 1>(A, G, S, A.order[j]);
    }
}

// per scene contact ranges: obstacle rows (contacts of the scene's obstacles) and active rows
__global__ void k_batch_ranges(int n_scenes, int nin, const int* sc_obs0, const int* sc_obs1, const int* sc_p0,
                               const int* sc_p1, const int* obs_off, const int* obs_pos, const int* row_ptr,
                               const Sizes* sizes, int* o0, int* o1, int* a0, int* a1) {
    const int c_obs = sizes->C_obs;
    const int nobs = nin > 0 ? obs_off[nin] : 0;  // obs_pos holds nobs entries
    GRID_STRIDE(s, n_scenes) {
        const int ob0 = sc_obs0[s], ob1 = sc_obs1[s];
        o0[s] = (ob0 < nin && obs_off[ob0] < nobs) ? obs_pos[obs_off[ob0]] : c_obs;
        o1[s] = (ob1 < nin && obs_off[ob1] < nobs) ? obs_pos[obs_off[ob1]] : c_obs;
        if (ob1 <= ob0) o1[s] = o0[s];
        a0[s] = c_obs + row_ptr[sc_p0[s]];
        a1[s] = c_obs + row_ptr[sc_p1[s]];
    }
}

template <typename T, int DIM, int BT, int KB, int CS>
cudaError_t launch_bt(BatchArgs<T>& A, int n_scenes, cudaStream_t s) {
    if (CS == 1) {
        k_apgd_batch<T, DIM, BT, KB><<<n_scenes, BT, 0, s>>>(A);
    } else {
        // the n_big largest scenes on two CTAs each, the rest paired, every cluster two CTAs
        const int clusters = A.n_big + (n_scenes - A.n_big + 1) / 2;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2 * clusters, 1, 1);
        cfg.blockDim = dim3(BT, 1, 1);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 2;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, k_apgd_batch_pairs<T, DIM, BT, KB>, A);
    }
    g_batch_launches += 1;
    return cudaGetLastError();
}

}  // namespace

void launch_batch_ranges(int n_scenes, int nin, const int* sc_obs0, const int* sc_obs1, const int* sc_p0,
                         const int* sc_p1, const int* obs_off, const int* obs_pos, const int* row_ptr,
                         const Sizes* sizes, int* o0, int* o1, int* a0, int* a1, cudaStream_t s) {
    k_batch_ranges<<<(n_scenes + 255) / 256, 256, 0, s>>>(n_scenes, nin, sc_obs0, sc_obs1, sc_p0, sc_p1, obs_off,
                                                          obs_pos, row_ptr, sizes, o0, o1, a0, a1);
    g_batch_launches += 1;
}

// threads per scene: one CTA of 256, 512 or 1024 threads, or 2048 = a cluster of two
// 1024-thread CTAs
bool batch_shape_valid(int block_threads, int tile) {
    return (block_threads == 256 && (tile == 2 || tile == 4)) ||
           ((block_threads == 512 || block_threads == 1024 || block_threads == 2048) && (tile == 1 || tile == 2));
}

template <typename T>
cudaError_t launch_apgd_batch(int dim, int block_threads, int tile, const BatchSolve<T>& b, int n_scenes,
                              cudaStream_t s) {
    BatchArgs<T> A;
    A.nin = b.nin;
    A.n_scenes = n_scenes;
    A.n_big = std::min(std::max(b.n_big, 0), n_scenes);
    A.order = b.order;
    A.sc_p0 = b.sc_p0;
    A.sc_p1 = b.sc_p1;
    A.sc_o0 = b.sc_o0;
    A.sc_o1 = b.sc_o1;
    A.sc_a0 = b.sc_a0;
    A.sc_a1 = b.sc_a1;
    A.cij = b.cij;
    A.nc = b.nc;
    A.nc64 = b.nc64;
    A.inc_ptr = b.inc_ptr;
    A.inc = b.inc;
    A.inc64 = b.inc64;
    A.invm = b.invm;
    for (int k = 0; k < 3; ++k) A.lam[k] = b.lam[k];
    for (int k = 0; k < 4; ++k) A.u[k] = b.u[k];
    A.lam64 = b.lam64;
    A.ufin = b.ufin;
    A.stats = b.stats;
    A.sizes = b.sizes;
    A.alpha = b.alpha;
    A.tol = b.tol;
    A.dt2 = b.dt * b.dt;
    A.viol_tol = b.viol_tol;
    A.max_ite = b.max_ite;
    A.dynamic = b.dynamic;
    A.max_corrections = b.max_corrections;
    A.curvature_start = b.curvature_start;
#define LB(D, B, K, C) \
    if (dim == D && block_threads == B * C && tile == K) return launch_bt<T, D, B, K, C>(A, n_scenes, s);
    LB(2, 256, 4, 1) LB(2, 256, 2, 1) LB(2, 512, 1, 1) LB(2, 512, 2, 1) LB(2, 1024, 1, 1) LB(2, 1024, 2, 1)
    LB(2, 1024, 1, 2) LB(2, 1024, 2, 2)
    LB(3, 256, 4, 1) LB(3, 256, 2, 1) LB(3, 512, 1, 1) LB(3, 512, 2, 1) LB(3, 1024, 1, 1) LB(3, 1024, 2, 1)
    LB(3, 1024, 1, 2) LB(3, 1024, 2, 2)
#undef LB
    return cudaErrorInvalidValue;
}
template cudaError_t launch_apgd_batch<double>(int, int, int, const BatchSolve<double>&, int, cudaStream_t);
template cudaError_t launch_apgd_batch<float>(int, int, int, const BatchSolve<float>&, int, cudaStream_t);

}  // namespace scopi_gpu
