// se.cu -- closest points of pairs of superellipsoids: 3D with one block per pair for the
// start and one thread per pair for the solve, 2D with one thread per pair.
//
// closest_points(superellipsoid<3>, superellipsoid<3>), closest_points.hpp:263-733:
//   start: the angle grids of both bodies (sorted unique binit_xy(6), ainit_yz(6) of
//          superellipsoid.hpp:360-466, ~21 x 21 points each), argmin over all point pairs
//          of |p1 - p2| + 2 (1 + n1.n2), first minimum in row-major order;
//   solve: hybrd1 (minpack.hpp:852-923: Powell's hybrid method, xtol 1e-10, maxfev 1000,
//          unit scaling, factor 100) on F = [ (p2 - p1) x n1 ; n1.n2 + |n1||n2| ] with its
//          analytic Jacobian (n1, n2 unnormalised normals);
//   result: pi = p1(u), pj = p2(u), nij = unit normal of body 2 at pj,
//          dij = sign((pi - pj).nij) |pi - pj|.
// k_se_start (one block per pair) computes the surface samples of both bodies into shared
// memory and finds the first minimum of the start criterion (FP32 screen, FP64 decision);
// k_se_solve (one quad of lanes per pair) runs the hybrid method from it (4 unknowns, bounded
// by maxfev) and writes the closest points.  The rows they take are those k_geometry flags:
// pairs of superellipsoids, and sphere-superellipsoid pairs whose Newton solve it refused,
// solved here with the sphere as the superellipsoid (r, r, r) of squareness 1.  Built with
// -fmad=false like detect.cu.
#include <math.h>

#include <algorithm>

#include "kernels.cuh"
#include "minpack.cuh"
#include "se_geom.cuh"
#include "se_newton.cuh"

namespace scopi_gpu {

static long long g_se_launches = 0;
long long se_launches() { return g_se_launches; }

namespace {
using namespace se;

constexpr int kSeThreads = 256;
constexpr int kSeGrid = 24;       // unique angles per grid axis at most (4 * 6)
constexpr int kSeSamples = kSeGrid * kSeGrid;


// ------------------------------------------------------------- start grids
// binit_xy(num) / ainit_yz(num) (superellipsoid.hpp:360-466): 4 angles per sample of
// [0, pi/2] (num samples: 6 in 3D, 4 in 2D); value k of the list
__device__ double binit_angle(const double* r, double e, int k, int num) {
    const double pi = 3.14159265358979323846;
    const int i = k >> 2, w = k & 3;
    const double t = (0.5 * pi) * i / (num - 1);
    const double x = r[0] * cos(t), y = r[1] * sin(t);
    const double d = pow(pow(r[1] * x, 2.0 / e) + pow(r[0] * y, 2.0 / e), e / 2.0);
    const double ys = y * r[0] * r[1] / d;
    const double sb = fmax(-1.0, fmin(1.0, sqrt(pow(pow(ys / r[1], 2.0), 1.0 / e))));
    const double v = asin(sb);
    const double a = w == 0 ? v : (w == 1 ? v + pi / 2 : (w == 2 ? v - pi : v - pi / 2));
    return fabs(a) < 1.0e-6 ? 0.01 : a;
}
__device__ double init_angle(const Body& s, int k, bool b_axis) {
    const double pi = 3.14159265358979323846;
    const int i = k >> 2, w = k & 3;
    const double t = (0.5 * pi) * i / 5;
    double v;
    if (b_axis) {
        return binit_angle(s.r, s.e, k, 6);
    } else {
        const double y = s.r[1] * cos(t), z = s.r[2] * sin(t);
        const double d = pow(pow(s.r[2] * y, 2.0 / s.n) + pow(s.r[1] * z, 2.0 / s.n), s.n / 2.0);
        const double zs = z * s.r[1] * s.r[2] / d;
        const double sa = fmax(-1.0, fmin(1.0, sqrt(pow(pow(zs / s.r[2], 2.0), 1.0 / s.n))));
        v = asin(sa);
    }
    const double a = w == 0 ? v : (w == 1 ? v + pi / 2 : (w == 2 ? v - pi : v - pi / 2));
    return fabs(a) < 1.0e-6 ? 0.01 : a;
}

// sorted unique of the 24 values in place (one thread); returns the count
__device__ int sort_unique(double* v, int n) {
    for (int i = 1; i < n; ++i) {
        const double x = v[i];
        int j = i - 1;
        while (j >= 0 && v[j] > x) {
            v[j + 1] = v[j];
            --j;
        }
        v[j + 1] = x;
    }
    int m = n > 0 ? 1 : 0;
    for (int i = 1; i < n; ++i)
        if (v[i] != v[m - 1]) v[m++] = v[i];
    return m;
}

struct SeShared {
    double ang[4][kSeGrid];   // a1, b1, a2, b2
    int cnt[4];
    double P[2][kSeSamples][3];
    double Nn[2][kSeSamples][3];
    double best_v[kSeThreads / 32];
    long long best_i[kSeThreads / 32];
};

// |p1 - p2| + 2 (1 + n1.n2) in FP64, the start criterion of closest_points.hpp:654-660
__device__ __forceinline__ double start_value(const double* p1, const double* n1, const double* p2, const double* n2) {
    const double dx = p1[0] - p2[0], dy = p1[1] - p2[1], dz = p1[2] - p2[2];
    return sqrt(dx * dx + dy * dy + dz * dz) + 2 * (1 + (n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2]));
}

// Start of the solve of each superellipsoid row: the first minimum (row-major over
// (sample of body 1, sample of body 2)) of the FP64 start criterion.  Every value is first
// screened in FP32 (samples relative to body 1's centre, error < 1e-6); a value enters the
// exact FP64 comparison when it is within kScreen of the thread's running FP32 minimum, so
// the FP64 minimiser (whose FP32 value is within twice the FP32 error of every running
// minimum) is always compared exactly.
constexpr float kScreen = 1e-5f;
constexpr int kJ = (kSeSamples + kSeThreads - 1) / kSeThreads;  // body-2 samples per thread

__global__ void __launch_bounds__(kSeThreads, 3) k_se_start(Bodies B, Contacts c, const Sizes* sizes, const int* need,
                                                             double* u0) {
    extern __shared__ __align__(16) unsigned char smem[];
    SeShared& S = *reinterpret_cast<SeShared*>(smem);
    const int C = sizes->C, C_obs = sizes->C_obs;
    for (int k = C_obs + blockIdx.x; k < C; k += gridDim.x) {
        if (!need[k]) continue;  // the row's closest points are known (k_geometry)
        const Body s1 = load_any(B, c.ci[k]), s2 = load_any(B, c.cj[k]);
        if (threadIdx.x < 4 * kSeGrid) {
            const int list = threadIdx.x / kSeGrid, m = threadIdx.x % kSeGrid;
            S.ang[list][m] = init_angle(list < 2 ? s1 : s2, m, (list & 1) != 0);
        }
        __syncthreads();
        if (threadIdx.x < 4) S.cnt[threadIdx.x] = sort_unique(S.ang[threadIdx.x], kSeGrid);
        __syncthreads();
        // surface samples: meshgrid(a, b) flattened row-major, index ia * nb + ib
        const int na1 = S.cnt[0], nb1 = S.cnt[1], na2 = S.cnt[2], nb2 = S.cnt[3];
        const int n1 = na1 * nb1, n2 = na2 * nb2;
        for (int t = threadIdx.x; t < n1 + n2; t += blockDim.x) {
            const int w = t < n1 ? 0 : 1;
            const int q = t < n1 ? t : t - n1;
            const int nb = w == 0 ? nb1 : nb2;
            const double a = S.ang[2 * w][q / nb], b = S.ang[2 * w + 1][q % nb];
            const Body& s = w == 0 ? s1 : s2;
            point(s, a, b, S.P[w][q]);
            normal(s, a, b, S.Nn[w][q]);
        }
        __syncthreads();
        // this thread's body-2 samples in registers, FP32, relative to body 1's centre
        float q2[kJ][3], m2[kJ][3];
        int jn = 0;
        for (int jj = 0; jj < kJ; ++jj) {
            const int j = threadIdx.x + jj * kSeThreads;
            if (j < n2) {
                for (int d = 0; d < 3; ++d) {
                    q2[jj][d] = (float)(S.P[1][j][d] - s1.c[d]);
                    m2[jj][d] = (float)S.Nn[1][j][d];
                }
                jn = jj + 1;
            }
        }
        float run32 = INFINITY;
        double bv = INFINITY;
        long long bi = 0x7fffffffffffffffLL;
        for (int a = 0; a < n1; ++a) {
            const float x = (float)(S.P[0][a][0] - s1.c[0]), y = (float)(S.P[0][a][1] - s1.c[1]),
                        z = (float)(S.P[0][a][2] - s1.c[2]);
            const float nx = (float)S.Nn[0][a][0], ny = (float)S.Nn[0][a][1], nz = (float)S.Nn[0][a][2];
            for (int jj = 0; jj < jn; ++jj) {
                const float dx = x - q2[jj][0], dy = y - q2[jj][1], dz = z - q2[jj][2];
                const float v = sqrtf(dx * dx + dy * dy + dz * dz) +
                                2.f * (1.f + (nx * m2[jj][0] + ny * m2[jj][1] + nz * m2[jj][2]));
                if (v <= run32 + kScreen) {
                    const int j = threadIdx.x + jj * kSeThreads;
                    const double v64 = start_value(S.P[0][a], S.Nn[0][a], S.P[1][j], S.Nn[1][j]);
                    const long long idx = (long long)a * n2 + j;
                    if (v64 < bv || (v64 == bv && idx < bi)) {
                        bv = v64;
                        bi = idx;
                    }
                }
                run32 = fminf(run32, v);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, bv, o);
            const long long oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov < bv || (ov == bv && oi < bi)) {
                bv = ov;
                bi = oi;
            }
        }
        if ((threadIdx.x & 31) == 0) {
            S.best_v[threadIdx.x >> 5] = bv;
            S.best_i[threadIdx.x >> 5] = bi;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
                if (S.best_v[w] < bv || (S.best_v[w] == bv && S.best_i[w] < bi)) {
                    bv = S.best_v[w];
                    bi = S.best_i[w];
                }
            if (bi == 0x7fffffffffffffffLL) bi = 0;  // NaN everywhere: start at the first sample
            const int ia = (int)(bi / n2), ib = (int)(bi % n2);
            double* u = u0 + 4 * (long long)k;
            u[0] = S.ang[0][ia / nb1];
            u[1] = S.ang[1][ia % nb1];
            u[2] = S.ang[2][ib / nb2];
            u[3] = S.ang[3][ib % nb2];
        }
        __syncthreads();
    }
}

// --------------------------------------------------------------- F and Jacobian
// One evaluation's point, normal (and derivatives) of both bodies, computed by a quad of four
// lanes that hold the same pair: the sixteen signed powers (8 per body, pw_arg / pw_exp) are
// split four per lane, power m on lane m & 3, and exchanged by shuffles inside the quad, so
// every lane assembles exactly what local() gives.  The lanes of a quad run the same hybrid
// method on the same data, so they reach every shuffle together.
__device__ __forceinline__ void local_pair_quad(const Body& s1, const Body& s2, const double* u, Local& L1, Local& L2,
                                                bool deriv) {
    const int ql = threadIdx.x & 3;
    const unsigned qmask = 0xFu << (threadIdx.x & 28);
    double sa[2], ca[2], sb[2], cb[2];
    sincos(u[0], &sa[0], &ca[0]);
    sincos(u[1], &sb[0], &cb[0]);
    sincos(u[2], &sa[1], &ca[1]);
    sincos(u[3], &sb[1], &cb[1]);
    Pw mine[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int bd = j >> 1, w = ql + 4 * (j & 1);  // power m = ql + 4 j: body m >> 3, index m & 7
        mine[j] = pw(pw_arg(w, sa[bd], ca[bd], sb[bd], cb[bd]), pw_exp(bd ? s2 : s1, w), deriv);
    }
    Pw P[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        P[m].v = __shfl_sync(qmask, mine[m >> 2].v, m & 3, 4);
        P[m].d = deriv ? __shfl_sync(qmask, mine[m >> 2].d, m & 3, 4) : 0.0;
    }
    assemble_local(s1, sa[0], ca[0], sb[0], cb[0], P, L1, deriv);
    assemble_local(s2, sa[1], ca[1], sb[1], cb[1], P + 8, L2, deriv);
}

__device__ void sese_F(const Body& s1, const Body& s2, const double* u, double* F) {
    Local L1, L2;
    local_pair_quad(s1, s2, u, L1, L2, false);
    double p1[3], p2[3], n1[3], n2[3];
    mv(s1.R, L1.p, p1);
    mv(s2.R, L2.p, p2);
    mv(s1.R, L1.N, n1);
    mv(s2.R, L2.N, n2);
    const double d[3] = {p2[0] + s2.c[0] - p1[0] - s1.c[0], p2[1] + s2.c[1] - p1[1] - s1.c[1],
                         p2[2] + s2.c[2] - p1[2] - s1.c[2]};
    cross(d, n1, F);
    F[3] = dot3(n1, n2) + norm3(n1) * norm3(n2);
}

__device__ void sese_J(const Body& s1, const Body& s2, const double* u, double* J) {  // column-major
    Local L1, L2;
    local_pair_quad(s1, s2, u, L1, L2, true);
    double p1[3], p2[3], n1[3], n2[3];
    mv(s1.R, L1.p, p1);
    mv(s2.R, L2.p, p2);
    mv(s1.R, L1.N, n1);
    mv(s2.R, L2.N, n2);
    const double d[3] = {p2[0] + s2.c[0] - p1[0] - s1.c[0], p2[1] + s2.c[1] - p1[1] - s1.c[1],
                         p2[2] + s2.c[2] - p1[2] - s1.c[2]};
    const double l1 = norm3(n1), l2 = norm3(n2);
    for (int k = 0; k < 4; ++k) {
        double dd[3], dn1[3] = {0, 0, 0}, dn2[3] = {0, 0, 0};
        if (k < 2) {
            double t[3];
            mv(s1.R, k == 0 ? L1.pa : L1.pb, t);
            for (int c = 0; c < 3; ++c) dd[c] = -t[c];
            mv(s1.R, k == 0 ? L1.Na : L1.Nb, dn1);
        } else {
            mv(s2.R, k == 2 ? L2.pa : L2.pb, dd);
            mv(s2.R, k == 2 ? L2.Na : L2.Nb, dn2);
        }
        double a[3], b[3];
        cross(dd, n1, a);
        cross(d, dn1, b);
        J[0 + 4 * k] = a[0] + b[0];
        J[1 + 4 * k] = a[1] + b[1];
        J[2 + 4 * k] = a[2] + b[2];
        J[3 + 4 * k] = dot3(dn1, n2) + dot3(n1, dn2) + dot3(n1, dn1) / l1 * l2 + l1 * dot3(n2, dn2) / l2;
    }
}

// The hybrid method from the start and the row's closest points, one row per quad of lanes
// (the evaluations' powers split over the quad: local_pair_quad), rows handed out by a
// counter so that a quad takes the next row when its solve ends.  The evaluations per solve
// vary from a few to maxfev (1000), and the kernel's time is set by the slowest rows while
// the other lanes idle (ncu at 8000 bodies, one lane per row: 2.7 % of the warp slots
// active over a 111 ms launch): the quad shortens those rows.  (One warp per row, with the
// powers spread over 32 lanes, was measured 5x slower: the hybrid method's own scalar work,
// then done 32 times, outweighs the powers.)  Two 128-thread blocks per SM (255 registers):
// the hybrid method's arrays stay in L1.
__global__ void __launch_bounds__(128, 2) k_se_solve(Bodies B, Contacts c, const Sizes* sizes, const int* need,
                                                    const double* u0,
                                                    int* next) {
    const int C = sizes->C, C_obs = sizes->C_obs;
    const int ql = threadIdx.x & 3;
    const unsigned qmask = 0xFu << (threadIdx.x & 28);
    for (;;) {
        int row = 0;
        if (ql == 0) row = atomicAdd(next, 1);
        row = __shfl_sync(qmask, row, 0, 4);
        const int k = C_obs + row;
        if (k >= C) break;
        if (!need[k]) continue;
        const Body s1 = load_any(B, c.ci[k]), s2 = load_any(B, c.cj[k]);
        double u[4];
        for (int q = 0; q < 4; ++q) u[q] = u0[4 * (long long)k + q];
        hybrj<4>([&](const double* x, double* F) { sese_F(s1, s2, x, F); },
              [&](const double* x, double* J) { sese_J(s1, s2, x, J); }, u);
        if (ql != 0) continue;
        double pi_[3], pj_[3], nij[3];
        point(s1, u[0], u[1], pi_);
        point(s2, u[2], u[3], pj_);
        normal(s2, u[2], u[3], nij);
        const double df[3] = {pi_[0] - pj_[0], pi_[1] - pj_[1], pi_[2] - pj_[2]};
        c.dij[k] = sgn(dot3(df, nij)) * norm3(df);
        for (int q = 0; q < 3; ++q) {
            c.pi[3 * (long long)k + q] = pi_[q];
            c.pj[3 * (long long)k + q] = pj_[q];
            c.nij[3 * (long long)k + q] = nij[q];
        }
    }
}


// One thread per row: the start grids (sorted unique binit_xy(4) of both bodies, at most
// 16 angles each), the first minimum of |p1 - p2| + 2 (1 + n1.n2) in row-major order, the
// hybrid method in 2 unknowns and the row's closest points (z = 0).
__global__ void __launch_bounds__(128) k_se2_pairs(Bodies B, Contacts c, const Sizes* sizes, const int* need) {
    constexpr int kNum = 4, kG = 4 * kNum;
    const int C = sizes->C, C_obs = sizes->C_obs;
    for (long long k = C_obs + (long long)blockIdx.x * blockDim.x + threadIdx.x; k < C;
         k += (long long)gridDim.x * blockDim.x) {
        if (!need[k]) continue;
        const Body2 s1 = load_any2(B, c.ci[k]), s2 = load_any2(B, c.cj[k]);
        double g1[kG], g2[kG];
        for (int m = 0; m < kG; ++m) {
            g1[m] = binit_angle(s1.r, s1.e, m, kNum);
            g2[m] = binit_angle(s2.r, s2.e, m, kNum);
        }
        const int n1 = sort_unique(g1, kG), n2 = sort_unique(g2, kG);
        double best = INFINITY, u[2] = {g1[0], g2[0]};
        for (int i = 0; i < n1; ++i) {
            double P1[2], N1[2];
            point2(s1, g1[i], P1);
            normal2(s1, g1[i], N1);
            for (int j = 0; j < n2; ++j) {
                double P2[2], N2[2];
                point2(s2, g2[j], P2);
                normal2(s2, g2[j], N2);
                const double dx = P1[0] - P2[0], dy = P1[1] - P2[1];
                const double v = sqrt(dx * dx + dy * dy) + 2 * (1 + (N1[0] * N2[0] + N1[1] * N2[1]));
                if (v < best) {
                    best = v;
                    u[0] = g1[i];
                    u[1] = g2[j];
                }
            }
        }
        hybrj<2>([&](const double* x, double* F) { se2_F(s1, s2, x, F); },
                 [&](const double* x, double* J) { se2_J(s1, s2, x, J); }, u);
        double pi_[2], pj_[2], nij[2];
        point2(s1, u[0], pi_);
        point2(s2, u[1], pj_);
        normal2(s2, u[1], nij);
        const double dx = pi_[0] - pj_[0], dy = pi_[1] - pj_[1];
        c.dij[k] = sgn(dx * nij[0] + dy * nij[1]) * sqrt(dx * dx + dy * dy);
        for (int q = 0; q < 2; ++q) {
            c.pi[3 * k + q] = pi_[q];
            c.pj[3 * k + q] = pj_[q];
            c.nij[3 * k + q] = nij[q];
        }
        c.pi[3 * k + 2] = c.pj[3 * k + 2] = c.nij[3 * k + 2] = 0.0;
    }
}

// before the solves: drop the candidate rows whose bodies are provably farther apart than
// dmax (gap along the line of centres; obstacle rows kept)
__global__ void k_se_gap_keep(int dim, Bodies B, Contacts c, const Sizes* sizes, double dmax, int* keep) {
    const int C = sizes->C, C_obs = sizes->C_obs;
    GRID_STRIDE(k, C) {
        if (k < C_obs) {
            keep[k] = 1;
            continue;
        }
        const int i = c.ci[k], j = c.cj[k];
        const double gap = dim == 3 ? support_gap3(load_any(B, i), load_any(B, j)) : support_gap2(load_any2(B, i), load_any2(B, j));
        const double lim = B.radius[i] + B.radius[j] + dmax;
        keep[k] = gap > dmax + 1e-9 * lim ? 0 : 1;
    }
}

// keep a row: obstacle rows (already exact) or dij < dmax
__global__ void k_se_keep(Contacts c, const Sizes* sizes, double dmax, int* keep) {
    const int C = sizes->C, C_obs = sizes->C_obs;
    GRID_STRIDE(k, C) keep[k] = (k < C_obs || c.dij[k] < dmax) ? 1 : 0;
}

__global__ void k_se_compact(Contacts src, Contacts dst, const Sizes* sizes, const int* keep, const int* pos) {
    const int C = sizes->C;
    GRID_STRIDE(k, C) {
        if (!keep[k]) continue;
        const int d = pos[k];
        dst.ci[d] = src.ci[k];
        dst.cj[d] = src.cj[k];
        dst.dij[d] = src.dij[k];
        dst.gamma[d] = src.gamma[k];
        for (int q = 0; q < 3; ++q) {
            dst.nij[3 * (long long)d + q] = src.nij[3 * (long long)k + q];
            dst.pi[3 * (long long)d + q] = src.pi[3 * (long long)k + q];
            dst.pj[3 * (long long)d + q] = src.pj[3 * (long long)k + q];
        }
    }
}

__global__ void k_se_sizes(Sizes* sizes, const int* total) {
    if (threadIdx.x == 0 && blockIdx.x == 0) sizes->C = *total;
}

}  // namespace

void launch_se_pairs(int dim, const Bodies& b, Contacts& c, const Sizes* sizes, const int* need, double* u0,
                     int* counter, int grid, cudaStream_t s) {
    if (dim == 2) {
        k_se2_pairs<<<4 * kSMs, 128, 0, s>>>(b, c, sizes, need);
        g_se_launches += 1;
        return;
    }
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_se_start, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SeShared));
        configured = true;
    }
    k_se_start<<<grid, kSeThreads, sizeof(SeShared), s>>>(b, c, sizes, need, u0);
    cudaMemsetAsync(counter, 0, sizeof(int), s);
    k_se_solve<<<4 * kSMs, 128, 0, s>>>(b, c, sizes, need, u0, counter);
    g_se_launches += 2;
}

void launch_se_prefilter(int dim, const Bodies& b, const Contacts& src, Contacts& dst, Sizes* sizes, double dmax,
                         long long c_cap, int* keep, int* pos, int* scan_work, int* total, cudaStream_t s) {
    const int threads = 256;
    const int blocks = (int)std::min<long long>((c_cap + threads - 1) / threads, 4096);
    k_se_gap_keep<<<blocks, threads, 0, s>>>(dim, b, src, sizes, dmax, keep);
    scan_exclusive(keep, pos, &sizes->C, 0, c_cap, total, scan_work, s, &g_se_launches);
    k_se_compact<<<blocks, threads, 0, s>>>(src, dst, sizes, keep, pos);
    k_se_sizes<<<1, 1, 0, s>>>(sizes, total);
    g_se_launches += 3;
}

void launch_se_filter(const Contacts& src, Contacts& dst, Sizes* sizes, double dmax, long long c_cap, int* keep,
                      int* pos, int* scan_work, int* total, cudaStream_t s) {
    const int threads = 256;
    const int blocks = (int)std::min<long long>((c_cap + threads - 1) / threads, 4096);
    k_se_keep<<<blocks, threads, 0, s>>>(src, sizes, dmax, keep);
    scan_exclusive(keep, pos, &sizes->C, 0, c_cap, total, scan_work, s, &g_se_launches);
    k_se_compact<<<blocks, threads, 0, s>>>(src, dst, sizes, keep, pos);
    k_se_sizes<<<1, 1, 0, s>>>(sizes, total);
    g_se_launches += 3;
}

}  // namespace scopi_gpu
