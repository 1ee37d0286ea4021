// se_newton.cuh -- the damped Newton method of the reference on the device (FP64) and its
// caller, the closest points of a sphere and a superellipsoid; the scalar 2D superellipsoid
// system it shares with se.cu.
//
// newton_method (utils.hpp:81-118) in n unknowns: d = solve(J(u), -F(u)); return when
// |d| < xtol (tested before the residual) or |F(u)| < ftol; otherwise a backtracking line
// search t = 1, 0.99, 0.98, ... while |F(u + t d)| > |F(u)| and t > 0.01, then u += t d; at
// most itermax steps (then -1).  The reference solves with LAPACK's dgesv; lu_solve restates
// the published reference-LAPACK algorithm for a small dense matrix: dgetf2 (column pivot =
// the first entry of largest |a| on or below the diagonal, multipliers scaled by the pivot's
// reciprocal when |pivot| >= the safe minimum, rank-1 update of the trailing block) and dgetrs
// (the row interchanges, then the unit lower and the upper triangular solves).  A zero pivot
// (the reference's solve throws there) ends the method with -2.  Norms are sqrt(sum of
// squares).
//
// closest_points(sphere<3>, superellipsoid<3>), closest_points.hpp:944-1282: unknowns
// u = (a1, b1, a2, b2), the superellipsoid's angles then the sphere's;
//   F = [ (p2 - p1) x n1 ; n1.n2 + |n1||n2| ],  n1 = sign(cos a1) N1(a1, b1),  n2 = sign(cos a2) N2(a2, b2)
// (N the unnormalised outward normals of superellipsoid::normal with the sphere as the
// superellipsoid (r, r, r), squareness 1: the reference's expressions carry the factor
// sign(cos a) on both normals, :1013-1037); start (:1262-1274): ten angle pairs per body,
// (ainit(k), binit(k)) with ainit = linspace(-pi/2, pi/2, 10), binit = linspace(-pi, pi, 10),
// the first minimum of |p1 - p2| over the 10 x 10 pairs in row-major order; result
// (:1275-1280): pi on the superellipsoid, pj on the sphere, nij = the sphere's unit normal at
// pj (sphere::normal, sphere.hpp:225-234), dij = (pi - pj).nij.
// 2D (closest_points.hpp:1316-1443): u = (b1, b2), the same F with n2 = the rotated
// r (cos b2, sin b2) and no sign factors (se2_F / se2_J with the sphere as (r, r), e = 1);
// start binit = {-pi, -pi/2, 0.001, pi/2} on both bodies, first minimum of |p1 - p2|.
#pragma once
#include "se_geom.cuh"

namespace scopi_gpu {
namespace se {
namespace {

constexpr double kSafeMin = 2.2250738585072014e-308;  // dlamch('S')

template <int N>
__device__ bool lu_solve(double* A, double* b) {  // A column-major N x N (overwritten), b (in: rhs, out: x)
    int piv[N];
    for (int j = 0; j < N; ++j) {
        int p = j;
        double big = fabs(A[j + N * j]);
        for (int i = j + 1; i < N; ++i)
            if (fabs(A[i + N * j]) > big) {
                big = fabs(A[i + N * j]);
                p = i;
            }
        piv[j] = p;
        if (A[p + N * j] == 0.0) return false;
        if (p != j)
            for (int k = 0; k < N; ++k) {
                const double t = A[j + N * k];
                A[j + N * k] = A[p + N * k];
                A[p + N * k] = t;
            }
        const double pv = A[j + N * j];
        if (fabs(pv) >= kSafeMin) {
            const double r = 1.0 / pv;
            for (int i = j + 1; i < N; ++i) A[i + N * j] *= r;
        } else {
            for (int i = j + 1; i < N; ++i) A[i + N * j] /= pv;
        }
        for (int k = j + 1; k < N; ++k) {
            const double t = -A[j + N * k];
            for (int i = j + 1; i < N; ++i) A[i + N * k] += A[i + N * j] * t;
        }
    }
    for (int j = 0; j < N; ++j)
        if (piv[j] != j) {
            const double t = b[j];
            b[j] = b[piv[j]];
            b[piv[j]] = t;
        }
    for (int k = 0; k < N; ++k)
        if (b[k] != 0.0)
            for (int i = k + 1; i < N; ++i) b[i] -= b[k] * A[i + N * k];
    for (int k = N - 1; k >= 0; --k)
        if (b[k] != 0.0) {
            b[k] /= A[k + N * k];
            for (int i = 0; i < k; ++i) b[i] -= b[k] * A[i + N * k];
        }
    return true;
}

template <int N>
__device__ __forceinline__ double norm_n(const double* x) {
    double s = 0.0;
    for (int k = 0; k < N; ++k) s += x[k] * x[k];
    return sqrt(s);
}

// the iterations taken (>= 0), -1 after itermax steps, -2 on a zero pivot
template <int N, typename Fun, typename Jac>
__device__ int newton(Fun&& fun, Jac&& jac, double* u, int itermax = 200, double ftol = 1.0e-10, double xtol = 1.0e-7) {
    for (int cc = 0; cc < itermax; ++cc) {
        double F[N], J[N * N], d[N];
        fun(u, F);
        jac(u, J);
        for (int k = 0; k < N; ++k) d[k] = -F[k];
        if (!lu_solve<N>(J, d)) return -2;
        if (norm_n<N>(d) < xtol) return cc;
        const double ferr = norm_n<N>(F);
        if (ferr < ftol) return cc;
        double t = 1;
        for (;;) {
            double x[N], Ft[N];
            for (int k = 0; k < N; ++k) x[k] = u[k] + t * d[k];
            fun(x, Ft);
            if (!(norm_n<N>(Ft) > ferr && t > 0.01)) break;
            t -= 0.01;
        }
        for (int k = 0; k < N; ++k) u[k] += t * d[k];
    }
    return -1;
}

// linspace(start, stop, num) with its endpoint (xtensor): start + k (stop - start)/(num - 1),
// the last value stop itself
__device__ __forceinline__ double linspace_at(double start, double stop, int num, int k) {
    if (k == num - 1) return stop;
    return start + k * ((stop - start) / (num - 1));
}

// ------------------------------------------------------------------ 3D system
// F (4) and its Jacobian (column-major 4 x 4) from the parametrisation's derivatives; signs
// = the factors sign(cos a1), sign(cos a2) of the reference's sphere-superellipsoid system
__device__ void sphse_F(const Body& s1, const Body& s2, const double* u, double* F) {
    Local L1, L2;
    local(s1, u[0], u[1], L1, false);
    local(s2, u[2], u[3], L2, false);
    const double k1 = sgn(cos(u[0])), k2 = sgn(cos(u[2]));
    double p1[3], p2[3], n1[3], n2[3];
    mv(s1.R, L1.p, p1);
    mv(s2.R, L2.p, p2);
    mv(s1.R, L1.N, n1);
    mv(s2.R, L2.N, n2);
    for (int c = 0; c < 3; ++c) {
        n1[c] *= k1;
        n2[c] *= k2;
    }
    const double d[3] = {p2[0] + s2.c[0] - p1[0] - s1.c[0], p2[1] + s2.c[1] - p1[1] - s1.c[1],
                         p2[2] + s2.c[2] - p1[2] - s1.c[2]};
    cross(d, n1, F);
    F[3] = dot3(n1, n2) + norm3(n1) * norm3(n2);
}
__device__ void sphse_J(const Body& s1, const Body& s2, const double* u, double* J) {
    Local L1, L2;
    local(s1, u[0], u[1], L1, true);
    local(s2, u[2], u[3], L2, true);
    const double k1 = sgn(cos(u[0])), k2 = sgn(cos(u[2]));
    double p1[3], p2[3], n1[3], n2[3];
    mv(s1.R, L1.p, p1);
    mv(s2.R, L2.p, p2);
    mv(s1.R, L1.N, n1);
    mv(s2.R, L2.N, n2);
    for (int c = 0; c < 3; ++c) {
        n1[c] *= k1;
        n2[c] *= k2;
    }
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
            for (int c = 0; c < 3; ++c) dn1[c] *= k1;
        } else {
            mv(s2.R, k == 2 ? L2.pa : L2.pb, dd);
            mv(s2.R, k == 2 ? L2.Na : L2.Nb, dn2);
            for (int c = 0; c < 3; ++c) dn2[c] *= k2;
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
// sphere::normal(a, b): the rotated (cos a cos b, cos a sin b, sin a), normalised
__device__ __forceinline__ void sphere_normal3(const Body& s, double a, double b, double* w) {
    const double n[3] = {cos(a) * cos(b), cos(a) * sin(b), sin(a)};
    mv(s.R, n, w);
    const double l = norm3(w);
    for (int k = 0; k < 3; ++k) w[k] /= l;
}

// ------------------------------------------------------------------ 2D system
// closest_points(superellipsoid<2>, superellipsoid<2>), closest_points.hpp:65-262, and the 2D
// sphere-superellipsoid system: F = [ (p2 - p1) x n1 ; n1.n2 + |n1||n2| ] in u = (b1, b2),
// n1, n2 unnormalised; J column-major 2 x 2.
__device__ void se2_F(const Body2& s1, const Body2& s2, const double* u, double* F) {
    Local2 L1, L2;
    local2(s1, u[0], L1, false);
    local2(s2, u[1], L2, false);
    double p1[2], p2[2], n1[2], n2[2];
    mv2(s1.R, L1.p, p1);
    mv2(s2.R, L2.p, p2);
    mv2(s1.R, L1.N, n1);
    mv2(s2.R, L2.N, n2);
    const double d[2] = {p2[0] + s2.c[0] - p1[0] - s1.c[0], p2[1] + s2.c[1] - p1[1] - s1.c[1]};
    F[0] = d[0] * n1[1] - d[1] * n1[0];
    F[1] = n1[0] * n2[0] + n1[1] * n2[1] + sqrt(n1[0] * n1[0] + n1[1] * n1[1]) * sqrt(n2[0] * n2[0] + n2[1] * n2[1]);
}
__device__ void se2_J(const Body2& s1, const Body2& s2, const double* u, double* J) {
    Local2 L1, L2;
    local2(s1, u[0], L1);
    local2(s2, u[1], L2);
    double p1[2], p2[2], n1[2], n2[2], pb1[2], pb2[2], nb1[2], nb2[2];
    mv2(s1.R, L1.p, p1);
    mv2(s2.R, L2.p, p2);
    mv2(s1.R, L1.N, n1);
    mv2(s2.R, L2.N, n2);
    mv2(s1.R, L1.pb, pb1);
    mv2(s2.R, L2.pb, pb2);
    mv2(s1.R, L1.Nb, nb1);
    mv2(s2.R, L2.Nb, nb2);
    const double d[2] = {p2[0] + s2.c[0] - p1[0] - s1.c[0], p2[1] + s2.c[1] - p1[1] - s1.c[1]};
    const double l1 = sqrt(n1[0] * n1[0] + n1[1] * n1[1]), l2 = sqrt(n2[0] * n2[0] + n2[1] * n2[1]);
    J[0] = -pb1[0] * n1[1] + pb1[1] * n1[0] + d[0] * nb1[1] - d[1] * nb1[0];
    J[1] = nb1[0] * n2[0] + nb1[1] * n2[1] + (n1[0] * nb1[0] + n1[1] * nb1[1]) / l1 * l2;
    J[2] = pb2[0] * n1[1] - pb2[1] * n1[0];
    J[3] = n1[0] * nb2[0] + n1[1] * nb2[1] + l1 * (n2[0] * nb2[0] + n2[1] * nb2[1]) / l2;
}

// ------------------------------------------------------------------ sphere - superellipsoid
// The reference's solve of (superellipsoid E, sphere S): the result in its convention (pi on
// E, pj on S, nij the sphere's unit normal) and the Newton method's return.  Then the
// engine's acceptance test: F = 0 also holds at pairs that are not the closest points (the
// farther point of the sphere, the far side of E), where the reference's start often leads
// its Newton method, or to no convergence in 200 steps.  For a convex body (squareness in
// (0, 2)) a surface point p whose outward unit normal points at the sphere's centre c is the
// point nearest c, and the sphere's nearest point lies on the segment from c to p: the result
// is accepted when the method converged and both hold to within cos >= 1 - 1e-6.  A pair it
// refuses is solved as the pair of superellipsoids it is (se.cu, the sphere as (r, r, r),
// squareness 1).
struct SphSeOut {
    double pi[3], pj[3], nij[3], dij;
    int status;  // the Newton method's return
    bool valid;
};

__device__ SphSeOut sphere_se3(const Body& E, const Body& S) {
    const double pi_ = 3.14159265358979323846;
    constexpr int num = 10;
    double u[4];
    {
        double best = INFINITY;
        int bi = 0, bj = 0;
        double P1[num][3], P2[num][3];
        for (int k = 0; k < num; ++k) {
            const double a = linspace_at(-pi_ / 2, pi_ / 2, num, k), b = linspace_at(-pi_, pi_, num, k);
            point(E, a, b, P1[k]);
            point(S, a, b, P2[k]);
        }
        for (int i = 0; i < num; ++i)
            for (int j = 0; j < num; ++j) {
                const double df[3] = {P1[i][0] - P2[j][0], P1[i][1] - P2[j][1], P1[i][2] - P2[j][2]};
                const double v = norm3(df);
                if (v < best) {
                    best = v;
                    bi = i;
                    bj = j;
                }
            }
        u[0] = linspace_at(-pi_ / 2, pi_ / 2, num, bi);
        u[1] = linspace_at(-pi_, pi_, num, bi);
        u[2] = linspace_at(-pi_ / 2, pi_ / 2, num, bj);
        u[3] = linspace_at(-pi_, pi_, num, bj);
    }
    SphSeOut o;
    o.status = newton<4>([&](const double* x, double* F) { sphse_F(E, S, x, F); },
                         [&](const double* x, double* J) { sphse_J(E, S, x, J); }, u);
    point(E, u[0], u[1], o.pi);
    point(S, u[2], u[3], o.pj);
    sphere_normal3(S, u[2], u[3], o.nij);
    const double df[3] = {o.pi[0] - o.pj[0], o.pi[1] - o.pj[1], o.pi[2] - o.pj[2]};
    o.dij = dot3(df, o.nij);
    // acceptance
    o.valid = false;
    if (o.status >= 0) {
        const double w[3] = {o.pi[0] - S.c[0], o.pi[1] - S.c[1], o.pi[2] - S.c[2]};
        const double L = norm3(w);
        if (L > 0) {
            const double nu[3] = {w[0] / L, w[1] / L, w[2] / L};
            double N[3];
            normal(E, u[0], u[1], N);
            o.valid = -dot3(N, nu) >= 1.0 - 1e-6 && dot3(o.nij, nu) >= 1.0 - 1e-6;
        }
    }
    return o;
}

__device__ SphSeOut sphere_se2(const Body2& E, const Body2& S) {
    const double pi_ = 3.14159265358979323846;
    const double binit[4] = {-pi_, -pi_ / 2, 0.001, pi_ / 2};
    double u[2] = {binit[0], binit[0]};
    {
        double best = INFINITY;
        double P2[4][2];
        for (int j = 0; j < 4; ++j) point2(S, binit[j], P2[j]);
        for (int i = 0; i < 4; ++i) {
            double P1[2];
            point2(E, binit[i], P1);
            for (int j = 0; j < 4; ++j) {
                const double dx = P1[0] - P2[j][0], dy = P1[1] - P2[j][1];
                const double v = sqrt(dx * dx + dy * dy);
                if (v < best) {
                    best = v;
                    u[0] = binit[i];
                    u[1] = binit[j];
                }
            }
        }
    }
    SphSeOut o;
    o.status = newton<2>([&](const double* x, double* F) { se2_F(E, S, x, F); },
                         [&](const double* x, double* J) { se2_J(E, S, x, J); }, u);
    point2(E, u[0], o.pi);
    point2(S, u[1], o.pj);
    normal2(S, u[1], o.nij);  // sphere::normal(b): the rotated r (cos b, sin b), normalised
    o.pi[2] = o.pj[2] = o.nij[2] = 0.0;
    o.dij = (o.pi[0] - o.pj[0]) * o.nij[0] + (o.pi[1] - o.pj[1]) * o.nij[1];
    o.valid = false;
    if (o.status >= 0) {
        const double w[2] = {o.pi[0] - S.c[0], o.pi[1] - S.c[1]};
        const double L = sqrt(w[0] * w[0] + w[1] * w[1]);
        if (L > 0) {
            const double nu[2] = {w[0] / L, w[1] / L};
            double N[2];
            normal2(E, u[0], N);
            o.valid = -(N[0] * nu[0] + N[1] * nu[1]) >= 1.0 - 1e-6 && o.nij[0] * nu[0] + o.nij[1] * nu[1] >= 1.0 - 1e-6;
        }
    }
    return o;
}

}  // namespace
}  // namespace se
}  // namespace scopi_gpu
