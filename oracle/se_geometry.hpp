// se_geometry.hpp -- superellipsoid closest points for the CPU oracle (test infrastructure:
// only tests/, smoke() and bench.py's CPU legs use the oracle; never the product path).
//
// Restates, for 2D superellipsoids:
//   superellipsoid::point(b) / normal(b)                  superellipsoid.hpp:282-289, 303-312
//   closest_points(superellipsoid<2>, superellipsoid<2>)   closest_points.hpp:65-262
//       (start = argmin over the two binit_xy(4) grids of |p1 - p2| + 2 (1 + n1.n2), then
//        hybrd1 on F = [ (p2 - p1) x n1 ; n1.n2 + |n1||n2| ] (2 unknowns b1, b2))
// and for 3D superellipsoids:
//   superellipsoid::point / normal / binit_xy / ainit_yz
//       include/scopi/objects/types/superellipsoid.hpp:282-325, 360-466
//   closest_points(superellipsoid<3>, superellipsoid<3>)   closest_points.hpp:263-733
//       (start = argmin over the two angle grids of |p1 - p2| + 2 (1 + n1.n2), then
//        hybrd1 on F = [ (p2 - p1) x n1 ; n1.n2 + |n1||n2| ] with the analytic Jacobian)
//   closest_points(superellipsoid<3>, plane<3>)            closest_points.hpp:1479-1768
//       (the solution of its system F = [ (pp - p1) x n1 ; s np.n1 + |np||n1| ], in
//        closed form: see se_plane)
//   hybrd1 / hybrd                                         minpack.hpp:338-923
//       restated from the published MINPACK algorithm (Powell's hybrid method: QR of the
//       Jacobian, dogleg step in a trust region, Broyden rank-1 updates with Givens
//       rotations), mode 2 with unit scaling, factor 100, xtol 1e-10, maxfev 200 (n + 1);
//       the Jacobian is always the analytic one (fdjac_analytic, minpack.hpp:88-125).
// The Jacobians are built by the chain rule from the derivatives of the parametrisation,
// which is the same function as the reference's expanded expressions.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <vector>

namespace orc_se {

using V3 = std::array<double, 3>;
using M3 = std::array<std::array<double, 3>, 3>;

struct SE {
    V3 c;           // centre
    M3 R;           // rotation (body -> world)
    double r[3];    // semi-axes
    double e, n;    // squareness: e for b (xy), n for a
};

inline double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
// sign(t) |t|^k and its derivative w.r.t. the angle for t = cos(x) / sin(x)
inline double cpow(double x, double k) {
    const double c = std::cos(x);
    return sgn(c) * std::pow(std::abs(c), k);
}
inline double spow(double x, double k) {
    const double s = std::sin(x);
    return sgn(s) * std::pow(std::abs(s), k);
}
inline double dcpow(double x, double k) { return -k * std::sin(x) * std::pow(std::abs(std::cos(x)), k - 1); }
inline double dspow(double x, double k) { return k * std::cos(x) * std::pow(std::abs(std::sin(x)), k - 1); }

inline V3 mv(const M3& R, const V3& x) {
    return {R[0][0] * x[0] + R[0][1] * x[1] + R[0][2] * x[2], R[1][0] * x[0] + R[1][1] * x[1] + R[1][2] * x[2],
            R[2][0] * x[0] + R[2][1] * x[1] + R[2][2] * x[2]};
}
inline V3 cross(const V3& a, const V3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
inline double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline double norm(const V3& a) { return std::sqrt(dot(a, a)); }

// body-frame point, unnormalised normal and their angle derivatives
struct Local {
    V3 p, pa, pb;   // point, d/da, d/db
    V3 N, Na, Nb;   // normal (unnormalised), d/da, d/db
};
inline Local local(const SE& s, double a, double b) {
    const double rx = s.r[0], ry = s.r[1], rz = s.r[2];
    const double Ca = cpow(a, s.n), Sa = spow(a, s.n), Cb = cpow(b, s.e), Sb = spow(b, s.e);
    const double dCa = dcpow(a, s.n), dSa = dspow(a, s.n), dCb = dcpow(b, s.e), dSb = dspow(b, s.e);
    const double n2 = 2 - s.n, e2 = 2 - s.e;
    const double Ca2 = cpow(a, n2), Sa2 = spow(a, n2), Cb2 = cpow(b, e2), Sb2 = spow(b, e2);
    const double dCa2 = dcpow(a, n2), dSa2 = dspow(a, n2), dCb2 = dcpow(b, e2), dSb2 = dspow(b, e2);
    Local L;
    L.p = {rx * Ca * Cb, ry * Ca * Sb, rz * Sa};
    L.pa = {rx * dCa * Cb, ry * dCa * Sb, rz * dSa};
    L.pb = {rx * Ca * dCb, ry * Ca * dSb, 0.0};
    L.N = {ry * rz * Ca2 * Cb2, rx * rz * Ca2 * Sb2, rx * ry * Sa2};
    L.Na = {ry * rz * dCa2 * Cb2, rx * rz * dCa2 * Sb2, rx * ry * dSa2};
    L.Nb = {ry * rz * Ca2 * dCb2, rx * rz * Ca2 * dSb2, 0.0};
    return L;
}

// superellipsoid::point(a, b), superellipsoid.hpp:291-300 (world frame)
inline V3 point(const SE& s, double a, double b) {
    const V3 p = {s.r[0] * cpow(a, s.n) * cpow(b, s.e), s.r[1] * cpow(a, s.n) * spow(b, s.e), s.r[2] * spow(a, s.n)};
    const V3 w = mv(s.R, p);
    return {w[0] + s.c[0], w[1] + s.c[1], w[2] + s.c[2]};
}
// superellipsoid::normal(a, b), superellipsoid.hpp:313-325 (unit, world frame)
inline V3 normal(const SE& s, double a, double b) {
    const double n2 = 2 - s.n, e2 = 2 - s.e;
    const V3 N = {s.r[1] * s.r[2] * cpow(a, n2) * cpow(b, e2), s.r[0] * s.r[2] * cpow(a, n2) * spow(b, e2),
                  s.r[0] * s.r[1] * spow(a, n2)};
    V3 w = mv(s.R, N);
    const double l = norm(w);
    for (auto& x : w) x /= l;
    return w;
}

// superellipsoid::binit_xy / ainit_yz, superellipsoid.hpp:360-466
inline std::vector<double> binit_xy(const SE& s, int num) {
    const double pi = 4 * std::atan(1);
    std::vector<double> out;
    for (int i = 0; i < num; ++i) {
        const double t = num > 1 ? (0.5 * pi) * i / (num - 1) : 0.0;
        const double x = s.r[0] * std::cos(t), y = s.r[1] * std::sin(t);
        const double d = std::pow(std::pow(s.r[1] * x, 2.0 / s.e) + std::pow(s.r[0] * y, 2.0 / s.e), s.e / 2.0);
        const double ys = y * s.r[0] * s.r[1] / d;
        const double sb = std::max(-1.0, std::min(1.0, std::sqrt(std::pow(std::pow(ys / s.r[1], 2), 1.0 / s.e))));
        const double b = std::asin(sb);
        out.push_back(b);
        out.push_back(b + pi / 2);
        out.push_back(b - pi);
        out.push_back(b - pi / 2);
    }
    for (auto& b : out)
        if (std::abs(b) < 1.0e-6) b = 0.01;
    return out;
}
inline std::vector<double> ainit_yz(const SE& s, int num) {
    const double pi = 4 * std::atan(1);
    std::vector<double> out;
    for (int i = 0; i < num; ++i) {
        const double t = num > 1 ? (0.5 * pi) * i / (num - 1) : 0.0;
        const double y = s.r[1] * std::cos(t), z = s.r[2] * std::sin(t);
        const double d = std::pow(std::pow(s.r[2] * y, 2.0 / s.n) + std::pow(s.r[1] * z, 2.0 / s.n), s.n / 2.0);
        const double zs = z * s.r[1] * s.r[2] / d;
        const double sa = std::max(-1.0, std::min(1.0, std::sqrt(std::pow(std::pow(zs / s.r[2], 2), 1.0 / s.n))));
        const double a = std::asin(sa);
        out.push_back(a);
        out.push_back(a + pi / 2);
        out.push_back(a - pi);
        out.push_back(a - pi / 2);
    }
    for (auto& a : out)
        if (std::abs(a) < 1.0e-6) a = 0.01;
    return out;
}
inline std::vector<double> sorted_unique(std::vector<double> v) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    return v;
}

// ---------------------------------------------------------------- MINPACK (restated)
constexpr double kEps = 2.220446049250313e-16;    // dpmpar(1)
constexpr double kGiant = std::numeric_limits<double>::max();  // dpmpar(3)

// enorm: Euclidean norm with the three-range accumulation of MINPACK
inline double enorm(int n, const double* x) {
    const double rdwarf = 3.834e-20, rgiant = 1.304e19;
    double s1 = 0, s2 = 0, s3 = 0, x1max = 0, x3max = 0;
    const double agiant = rgiant / n;
    for (int i = 0; i < n; ++i) {
        const double xabs = std::abs(x[i]);
        if (xabs > rdwarf && xabs < agiant) {
            s2 += xabs * xabs;
        } else if (xabs <= rdwarf) {
            if (xabs > x3max) {
                s3 = 1 + s3 * (x3max / xabs) * (x3max / xabs);
                x3max = xabs;
            } else if (xabs != 0) {
                s3 += (xabs / x3max) * (xabs / x3max);
            }
        } else {
            if (xabs > x1max) {
                s1 = 1 + s1 * (x1max / xabs) * (x1max / xabs);
                x1max = xabs;
            } else {
                s1 += (xabs / x1max) * (xabs / x1max);
            }
        }
    }
    if (s1 != 0) return x1max * std::sqrt(s1 + (s2 / x1max) / x1max);
    if (s2 != 0) {
        if (s2 >= x3max) return std::sqrt(s2 * (1 + (x3max / s2) * (x3max * s3)));
        return std::sqrt(x3max * ((s2 / x3max) + (x3max * s3)));
    }
    return x3max * std::sqrt(s3);
}

// Column-major n x n matrices a[i + j*n].  Householder QR without pivoting (qrfac).
inline void qrfac(int n, double* a, double* rdiag, double* acnorm) {
    for (int j = 0; j < n; ++j) {
        acnorm[j] = enorm(n, a + j * n);
        rdiag[j] = acnorm[j];
    }
    for (int j = 0; j < n; ++j) {
        double ajnorm = enorm(n - j, a + j + j * n);
        if (ajnorm != 0) {
            if (a[j + j * n] < 0) ajnorm = -ajnorm;
            for (int i = j; i < n; ++i) a[i + j * n] /= ajnorm;
            a[j + j * n] += 1;
            for (int k = j + 1; k < n; ++k) {
                double sum = 0;
                for (int i = j; i < n; ++i) sum += a[i + j * n] * a[i + k * n];
                const double temp = sum / a[j + j * n];
                for (int i = j; i < n; ++i) a[i + k * n] -= temp * a[i + j * n];
            }
        }
        rdiag[j] = -ajnorm;
    }
}
// orthogonal factor of qrfac accumulated in q (qform)
inline void qform(int n, double* q, double* wa) {
    for (int j = 1; j < n; ++j)
        for (int i = 0; i < j; ++i) q[i + j * n] = 0;
    for (int l = 0; l < n; ++l) {
        const int k = n - 1 - l;
        for (int i = k; i < n; ++i) {
            wa[i] = q[i + k * n];
            q[i + k * n] = 0;
        }
        q[k + k * n] = 1;
        if (wa[k] == 0) continue;
        for (int j = k; j < n; ++j) {
            double sum = 0;
            for (int i = k; i < n; ++i) sum += q[i + j * n] * wa[i];
            const double temp = sum / wa[k];
            for (int i = k; i < n; ++i) q[i + j * n] -= temp * wa[i];
        }
    }
}
// dogleg step in the trust region delta; r = upper triangle packed by rows
inline void dogleg(int n, const double* r, const double* diag, const double* qtb, double delta, double* x, double* wa1,
                   double* wa2) {
    int jj = (n * (n + 1)) / 2;  // one past the last packed element (0-based)
    for (int k = 1; k <= n; ++k) {
        const int j = n - k;
        jj -= k;
        int l = jj + 1;
        double sum = 0;
        for (int i = j + 1; i < n; ++i) sum += r[l++] * x[i];
        double temp = r[jj];
        if (temp == 0) {
            int ll = j;
            for (int i = 0; i <= j; ++i) {
                temp = std::max(temp, std::abs(r[ll]));
                ll += n - i - 1;
            }
            temp = kEps * temp;
            if (temp == 0) temp = kEps;
        }
        x[j] = (qtb[j] - sum) / temp;
    }
    for (int j = 0; j < n; ++j) {
        wa1[j] = 0;
        wa2[j] = diag[j] * x[j];
    }
    const double qnorm = enorm(n, wa2);
    if (qnorm <= delta) return;
    int l = 0;
    for (int j = 0; j < n; ++j) {
        const double temp = qtb[j];
        for (int i = j; i < n; ++i) wa1[i] += r[l++] * temp;
        wa1[j] /= diag[j];
    }
    const double gnorm = enorm(n, wa1);
    double sgnorm = 0, alpha = delta / qnorm;
    if (gnorm != 0) {
        for (int j = 0; j < n; ++j) wa1[j] = (wa1[j] / gnorm) / diag[j];
        l = 0;
        for (int j = 0; j < n; ++j) {
            double sum = 0;
            for (int i = j; i < n; ++i) sum += r[l++] * wa1[i];
            wa2[j] = sum;
        }
        const double temp = enorm(n, wa2);
        sgnorm = (gnorm / temp) / temp;
        alpha = 0;
        if (sgnorm < delta) {
            const double bnorm = enorm(n, qtb);
            double t = (bnorm / gnorm) * (bnorm / qnorm) * (sgnorm / delta);
            t = t - (delta / qnorm) * (sgnorm / delta) * (sgnorm / delta) +
                std::sqrt((t - (delta / qnorm)) * (t - (delta / qnorm)) +
                          (1 - (delta / qnorm) * (delta / qnorm)) * (1 - (sgnorm / delta) * (sgnorm / delta)));
            alpha = ((delta / qnorm) * (1 - (sgnorm / delta) * (sgnorm / delta))) / t;
        }
    }
    const double temp = (1 - alpha) * std::min(sgnorm, delta);
    for (int j = 0; j < n; ++j) x[j] = temp * wa1[j] + alpha * x[j];
}
// rank-1 update of the packed triangle s (m = n) by Givens rotations (r1updt)
inline bool r1updt(int n, double* s, const double* u, double* v, double* w) {
    const int m = n;
    int jj = (n * (2 * m - n + 1)) / 2 - (m - n) - 1;  // 0-based index of s(n, n)
    int l = jj;
    for (int i = n - 1; i < m; ++i) w[i] = s[l++];
    for (int nmj = 1; nmj <= n - 1; ++nmj) {
        const int j = n - 1 - nmj;
        jj -= m - j;
        w[j] = 0;
        if (v[j] != 0) {
            double cs, sn, tau;
            if (std::abs(v[n - 1]) < std::abs(v[j])) {
                const double cotan = v[n - 1] / v[j];
                sn = 0.5 / std::sqrt(0.25 + 0.25 * cotan * cotan);
                cs = sn * cotan;
                tau = 1;
                if (std::abs(cs) * kGiant > 1) tau = 1 / cs;
            } else {
                const double tn = v[j] / v[n - 1];
                cs = 0.5 / std::sqrt(0.25 + 0.25 * tn * tn);
                sn = cs * tn;
                tau = sn;
            }
            v[n - 1] = sn * v[j] + cs * v[n - 1];
            v[j] = tau;
            l = jj;
            for (int i = j; i < m; ++i) {
                const double temp = cs * s[l] - sn * w[i];
                w[i] = sn * s[l] + cs * w[i];
                s[l] = temp;
                ++l;
            }
        }
    }
    for (int i = 0; i < m; ++i) w[i] += v[n - 1] * u[i];
    bool sing = false;
    for (int j = 0; j < n - 1; ++j) {
        if (w[j] != 0) {
            double cs, sn, tau;
            if (std::abs(s[jj]) < std::abs(w[j])) {
                const double cotan = s[jj] / w[j];
                sn = 0.5 / std::sqrt(0.25 + 0.25 * cotan * cotan);
                cs = sn * cotan;
                tau = 1;
                if (std::abs(cs) * kGiant > 1) tau = 1 / cs;
            } else {
                const double tn = w[j] / s[jj];
                cs = 0.5 / std::sqrt(0.25 + 0.25 * tn * tn);
                sn = cs * tn;
                tau = sn;
            }
            l = jj;
            for (int i = j; i < m; ++i) {
                const double temp = cs * s[l] + sn * w[i];
                w[i] = -sn * s[l] + cs * w[i];
                s[l] = temp;
                ++l;
            }
            w[j] = tau;
        }
        if (s[jj] == 0) sing = true;
        jj += m - j;
    }
    l = jj;
    for (int i = n - 1; i < m; ++i) s[l++] = w[i];
    if (s[jj] == 0) sing = true;
    return sing;
}
// apply the stored Givens rotations to the m x n matrix a (r1mpyq), a[i + j*lda]
inline void r1mpyq(int m, int n, double* a, int lda, const double* v, const double* w) {
    for (int nmj = 1; nmj <= n - 1; ++nmj) {
        const int j = n - 1 - nmj;
        double cs, sn;
        if (std::abs(v[j]) > 1) {
            cs = 1 / v[j];
            sn = std::sqrt(1 - cs * cs);
        } else {
            sn = v[j];
            cs = std::sqrt(1 - sn * sn);
        }
        for (int i = 0; i < m; ++i) {
            const double temp = cs * a[i + j * lda] - sn * a[i + (n - 1) * lda];
            a[i + (n - 1) * lda] = sn * a[i + j * lda] + cs * a[i + (n - 1) * lda];
            a[i + j * lda] = temp;
        }
    }
    for (int j = 0; j < n - 1; ++j) {
        double cs, sn;
        if (std::abs(w[j]) > 1) {
            cs = 1 / w[j];
            sn = std::sqrt(1 - cs * cs);
        } else {
            sn = w[j];
            cs = std::sqrt(1 - sn * sn);
        }
        for (int i = 0; i < m; ++i) {
            const double temp = cs * a[i + j * lda] + sn * a[i + (n - 1) * lda];
            a[i + (n - 1) * lda] = -sn * a[i + j * lda] + cs * a[i + (n - 1) * lda];
            a[i + j * lda] = temp;
        }
    }
}

struct HybrResult {
    int info;
    int nfev;
    int njev;
};

// Powell hybrid method with analytic Jacobian (hybrd1 of minpack.hpp:852-923 with
// fdjac_analytic): fun(x, f) evaluates F, jac(x, J) the Jacobian (column-major).
template <int N, typename Fun, typename Jac>
HybrResult hybrj(Fun&& fun, Jac&& jac, double* x, double xtol = 1e-10, int maxfev = 200 * (N + 1),
                 double factor = 100.0) {
    const double p1 = 0.1, p5 = 0.5, p001 = 1e-3, p0001 = 1e-4;
    double fvec[N], fjac[N * N], diag[N], r[(N * (N + 1)) / 2], qtf[N], wa1[N], wa2[N], wa3[N], wa4[N];
    for (int j = 0; j < N; ++j) diag[j] = 1.0;  // mode 2, unit scaling
    HybrResult res{0, 0, 0};
    fun(x, fvec);
    res.nfev = 1;
    double fnorm = enorm(N, fvec);
    int iter = 1, ncsuc = 0, ncfail = 0, nslow1 = 0, nslow2 = 0;
    double delta = 0, xnorm = 0;
    for (;;) {
        bool jeval = true;
        jac(x, fjac);
        ++res.njev;
        qrfac(N, fjac, wa1, wa2);
        if (iter == 1) {
            for (int j = 0; j < N; ++j) wa3[j] = diag[j] * x[j];
            xnorm = enorm(N, wa3);
            delta = factor * xnorm;
            if (delta == 0) delta = factor;
        }
        for (int i = 0; i < N; ++i) qtf[i] = fvec[i];
        for (int j = 0; j < N; ++j) {
            if (fjac[j + j * N] == 0) continue;
            double sum = 0;
            for (int i = j; i < N; ++i) sum += fjac[i + j * N] * qtf[i];
            const double temp = -sum / fjac[j + j * N];
            for (int i = j; i < N; ++i) qtf[i] += fjac[i + j * N] * temp;
        }
        for (int j = 0; j < N; ++j) {
            int l = j;
            for (int i = 0; i < j; ++i) {
                r[l] = fjac[i + j * N];
                l += N - i - 1;
            }
            r[l] = wa1[j];
        }
        qform(N, fjac, wa1);
        for (;;) {
            dogleg(N, r, diag, qtf, delta, wa1, wa2, wa3);
            for (int j = 0; j < N; ++j) {
                wa1[j] = -wa1[j];
                wa2[j] = x[j] + wa1[j];
                wa3[j] = diag[j] * wa1[j];
            }
            const double pnorm = enorm(N, wa3);
            if (iter == 1) delta = std::min(delta, pnorm);
            fun(wa2, wa4);
            ++res.nfev;
            const double fnorm1 = enorm(N, wa4);
            double actred = -1;
            if (fnorm1 < fnorm) actred = 1 - (fnorm1 / fnorm) * (fnorm1 / fnorm);
            int l = 0;
            for (int i = 0; i < N; ++i) {
                double sum = 0;
                for (int j = i; j < N; ++j) sum += r[l++] * wa1[j];
                wa3[i] = qtf[i] + sum;
            }
            const double temp = enorm(N, wa3);
            double prered = 0;
            if (temp < fnorm) prered = 1 - (temp / fnorm) * (temp / fnorm);
            double ratio = 0;
            if (prered > 0) ratio = actred / prered;
            if (ratio < p1) {
                ncsuc = 0;
                ++ncfail;
                delta = p5 * delta;
            } else {
                ncfail = 0;
                ++ncsuc;
                if (ratio >= p5 || ncsuc > 1) delta = std::max(delta, pnorm / p5);
                if (std::abs(ratio - 1) <= p1) delta = pnorm / p5;
            }
            if (ratio >= p0001) {
                for (int j = 0; j < N; ++j) {
                    x[j] = wa2[j];
                    wa2[j] = diag[j] * x[j];
                    fvec[j] = wa4[j];
                }
                xnorm = enorm(N, wa2);
                fnorm = fnorm1;
                ++iter;
            }
            ++nslow1;
            if (actred >= p001) nslow1 = 0;
            if (jeval) ++nslow2;
            if (actred >= p1) nslow2 = 0;
            if (delta <= xtol * xnorm || fnorm == 0) res.info = 1;
            if (res.info != 0) return res;
            if (res.nfev >= maxfev) res.info = 2;
            if (p1 * std::max(p1 * delta, pnorm) <= kEps * xnorm) res.info = 3;
            if (nslow2 == 5) res.info = 4;
            if (nslow1 == 10) res.info = 5;
            if (res.info != 0) return res;
            if (ncfail == 2) break;
            for (int j = 0; j < N; ++j) {
                double sum = 0;
                for (int i = 0; i < N; ++i) sum += fjac[i + j * N] * wa4[i];
                wa2[j] = (sum - wa3[j]) / pnorm;
                wa1[j] = diag[j] * ((diag[j] * wa1[j]) / pnorm);
                if (ratio >= p0001) qtf[j] = sum;
            }
            r1updt(N, r, wa1, wa2, wa3);
            r1mpyq(N, N, fjac, N, wa2, wa3);
            r1mpyq(1, N, qtf, 1, wa2, wa3);
            jeval = false;
        }
    }
}

// ------------------------------------------------------------- SE - SE (3D)
struct PairOut {
    V3 pi, pj, nij;
    double dij;
    int info;
    int nfev = 0;
    double u[4];
};

// F and its Jacobian (column-major 4x4) for u = (a1, b1, a2, b2)
inline void sese_F(const SE& s1, const SE& s2, const double* u, double* F) {
    const Local L1 = local(s1, u[0], u[1]), L2 = local(s2, u[2], u[3]);
    const V3 p1 = mv(s1.R, L1.p), p2 = mv(s2.R, L2.p);
    const V3 d = {p2[0] + s2.c[0] - p1[0] - s1.c[0], p2[1] + s2.c[1] - p1[1] - s1.c[1],
                  p2[2] + s2.c[2] - p1[2] - s1.c[2]};
    const V3 n1 = mv(s1.R, L1.N), n2 = mv(s2.R, L2.N);
    const V3 x = cross(d, n1);
    F[0] = x[0];
    F[1] = x[1];
    F[2] = x[2];
    F[3] = dot(n1, n2) + norm(n1) * norm(n2);
}
inline void sese_J(const SE& s1, const SE& s2, const double* u, double* J) {
    const Local L1 = local(s1, u[0], u[1]), L2 = local(s2, u[2], u[3]);
    const V3 p1 = mv(s1.R, L1.p), p2 = mv(s2.R, L2.p);
    const V3 d = {p2[0] + s2.c[0] - p1[0] - s1.c[0], p2[1] + s2.c[1] - p1[1] - s1.c[1],
                  p2[2] + s2.c[2] - p1[2] - s1.c[2]};
    const V3 n1 = mv(s1.R, L1.N), n2 = mv(s2.R, L2.N);
    const double l1 = norm(n1), l2 = norm(n2);
    V3 dd[4], dn1[4], dn2[4];
    const V3 z = {0, 0, 0};
    const V3 pa1 = mv(s1.R, L1.pa), pb1 = mv(s1.R, L1.pb);
    dd[0] = {-pa1[0], -pa1[1], -pa1[2]};
    dd[1] = {-pb1[0], -pb1[1], -pb1[2]};
    dd[2] = mv(s2.R, L2.pa);
    dd[3] = mv(s2.R, L2.pb);
    dn1[0] = mv(s1.R, L1.Na);
    dn1[1] = mv(s1.R, L1.Nb);
    dn1[2] = dn1[3] = z;
    dn2[0] = dn2[1] = z;
    dn2[2] = mv(s2.R, L2.Na);
    dn2[3] = mv(s2.R, L2.Nb);
    for (int k = 0; k < 4; ++k) {
        const V3 a = cross(dd[k], n1), b = cross(d, dn1[k]);
        J[0 + 4 * k] = a[0] + b[0];
        J[1 + 4 * k] = a[1] + b[1];
        J[2 + 4 * k] = a[2] + b[2];
        J[3 + 4 * k] = dot(dn1[k], n2) + dot(n1, dn2[k]) + dot(n1, dn1[k]) / l1 * l2 + l1 * dot(n2, dn2[k]) / l2;
    }
}

// hybrd1 start: argmin over the (a, b) grids of the two bodies, first minimum in row-major order
inline void sese_start(const SE& s1, const SE& s2, double* u0) {
    const int num = 6;
    const auto b1 = sorted_unique(binit_xy(s1, num)), a1 = sorted_unique(ainit_yz(s1, num));
    const auto b2 = sorted_unique(binit_xy(s2, num)), a2 = sorted_unique(ainit_yz(s2, num));
    // meshgrid(a, b) flattened row-major: index i*nb + j -> (a[i], b[j])
    std::vector<V3> P1, N1, P2, N2;
    std::vector<std::array<double, 2>> U1, U2;
    for (double a : a1)
        for (double b : b1) {
            P1.push_back(point(s1, a, b));
            N1.push_back(normal(s1, a, b));
            U1.push_back({a, b});
        }
    for (double a : a2)
        for (double b : b2) {
            P2.push_back(point(s2, a, b));
            N2.push_back(normal(s2, a, b));
            U2.push_back({a, b});
        }
    double best = INFINITY;
    size_t bi = 0, bj = 0;
    for (size_t i = 0; i < P1.size(); ++i)
        for (size_t j = 0; j < P2.size(); ++j) {
            const V3 df = {P1[i][0] - P2[j][0], P1[i][1] - P2[j][1], P1[i][2] - P2[j][2]};
            const double v = norm(df) + 2 * (1 + dot(N1[i], N2[j]));
            if (v < best) {
                best = v;
                bi = i;
                bj = j;
            }
        }
    u0[0] = U1[bi][0];
    u0[1] = U1[bi][1];
    u0[2] = U2[bj][0];
    u0[3] = U2[bj][1];
}

// closest_points(superellipsoid<3>, superellipsoid<3>), closest_points.hpp:263-733; from a
// given start u0 when it is not null (to compare a solve with another one's from its start)
inline PairOut se_se(const SE& s1, const SE& s2, const double* u0 = nullptr) {
    double u[4];
    if (u0)
        for (int k = 0; k < 4; ++k) u[k] = u0[k];
    else
        sese_start(s1, s2, u);
    const HybrResult h = hybrj<4>([&](const double* x, double* F) { sese_F(s1, s2, x, F); },
                                  [&](const double* x, double* J) { sese_J(s1, s2, x, J); }, u);
    PairOut o;
    o.info = h.info;
    o.nfev = h.nfev;
    for (int k = 0; k < 4; ++k) o.u[k] = u[k];
    o.pi = point(s1, u[0], u[1]);
    o.pj = point(s2, u[2], u[3]);
    o.nij = normal(s2, u[2], u[3]);
    const V3 df = {o.pi[0] - o.pj[0], o.pi[1] - o.pj[1], o.pi[2] - o.pj[2]};
    o.dij = sgn(dot(df, o.nij)) * norm(df);
    return o;
}

// ----------------------------------------------------------- SE - plane (3D)
struct Plane {
    V3 c;
    M3 R;  // normal = column 0, in-plane directions = columns 1 and 2
};
inline V3 plane_normal(const Plane& p) { return {p.R[0][0], p.R[1][0], p.R[2][0]}; }

// u = (a1, b1, a2, b2): body angles and plane coordinates; the normal of the body is taken
// with the factor sign(cos a1) of the reference's expressions
inline void sep_F(const SE& s, const Plane& P, double sg, const double* u, double* F) {
    const Local L = local(s, u[0], u[1]);
    const double k = sgn(std::cos(u[0]));
    const V3 p1 = mv(s.R, L.p);
    const V3 pp = mv(P.R, V3{0.0, u[2], u[3]});
    const V3 d = {pp[0] + P.c[0] - p1[0] - s.c[0], pp[1] + P.c[1] - p1[1] - s.c[1], pp[2] + P.c[2] - p1[2] - s.c[2]};
    V3 n1 = mv(s.R, L.N);
    for (auto& x : n1) x *= k;
    const V3 np = plane_normal(P);
    const V3 x = cross(d, n1);
    F[0] = x[0];
    F[1] = x[1];
    F[2] = x[2];
    F[3] = sg * dot(np, n1) + norm(np) * norm(n1);
}
inline void sep_J(const SE& s, const Plane& P, double sg, const double* u, double* J) {
    const Local L = local(s, u[0], u[1]);
    const double k = sgn(std::cos(u[0]));
    const V3 p1 = mv(s.R, L.p);
    const V3 pp = mv(P.R, V3{0.0, u[2], u[3]});
    const V3 d = {pp[0] + P.c[0] - p1[0] - s.c[0], pp[1] + P.c[1] - p1[1] - s.c[1], pp[2] + P.c[2] - p1[2] - s.c[2]};
    V3 n1 = mv(s.R, L.N);
    for (auto& x : n1) x *= k;
    const V3 np = plane_normal(P);
    const double l1 = norm(n1), lp = norm(np);
    V3 dd[4], dn1[4];
    const V3 pa = mv(s.R, L.pa), pb = mv(s.R, L.pb);
    dd[0] = {-pa[0], -pa[1], -pa[2]};
    dd[1] = {-pb[0], -pb[1], -pb[2]};
    dd[2] = {P.R[0][1], P.R[1][1], P.R[2][1]};
    dd[3] = {P.R[0][2], P.R[1][2], P.R[2][2]};
    dn1[0] = mv(s.R, L.Na);
    dn1[1] = mv(s.R, L.Nb);
    for (int q = 0; q < 2; ++q)
        for (auto& x : dn1[q]) x *= k;
    dn1[2] = dn1[3] = V3{0, 0, 0};
    for (int c = 0; c < 4; ++c) {
        const V3 a = cross(dd[c], n1), b = cross(d, dn1[c]);
        J[0 + 4 * c] = a[0] + b[0];
        J[1 + 4 * c] = a[1] + b[1];
        J[2 + 4 * c] = a[2] + b[2];
        J[3 + 4 * c] = sg * dot(np, dn1[c]) + lp * dot(n1, dn1[c]) / l1;
    }
}

// Angles (a, b) of the body point whose outward normal points along the body-frame
// direction m: from N(a, b) = lambda m (lambda > 0), with cos a >= 0,
//   b = atan2(sign(my) |ry my|^(1/(2-e)), sign(mx) |rx mx|^(1/(2-e))),
//   |tan a|^(2-n) = |mz| |(ry rz C(b,2-e), rx rz S(b,2-e))| / (rx ry |(mx, my)|), sign(a) = sign(mz).
inline void support_angles(const SE& s, const V3& m, double& a, double& b) {
    const double pi = 4 * std::atan(1);
    const double rx = s.r[0], ry = s.r[1], rz = s.r[2];
    const double mxy = std::sqrt(m[0] * m[0] + m[1] * m[1]);
    if (mxy == 0) {
        b = 0;
        a = m[2] >= 0 ? pi / 2 : -pi / 2;
        return;
    }
    const double ke = 1.0 / (2 - s.e), kn = 1.0 / (2 - s.n);
    b = std::atan2(sgn(m[1]) * std::pow(std::abs(ry * m[1]), ke), sgn(m[0]) * std::pow(std::abs(rx * m[0]), ke));
    const double cb = cpow(b, 2 - s.e), sb = spow(b, 2 - s.e);
    const double h = std::sqrt((ry * rz * cb) * (ry * rz * cb) + (rx * rz * sb) * (rx * rz * sb));
    const double t = std::abs(m[2]) * h / (rx * ry * mxy);
    a = sgn(m[2]) * std::atan(std::pow(t, kn));
}

// closest_points(superellipsoid<3>, plane<3>), closest_points.hpp:1479-1759.  The system
// there, F = [ (pp - p1) x n1 ; s np.n1 + |np||n1| ] over the body angles and the plane
// coordinates, has for a convex body one solution: the body point whose outward normal is
// opposite to the plane normal oriented toward the body (s = the body's side), and its
// projection on the plane.  That solution is computed in closed form here.  (The
// reference's Newton does not reach it on bodies of this size: its start takes the plane
// coordinates from the angle grid, in metres, and its residual receives the signed
// centre-plane distance where it needs s; F3 also has a double root.)  pi on the body, pj on
// the plane, nij = s np, dij = (pi - pj).nij.
inline PairOut se_plane(const SE& s, const Plane& P) {
    const V3 np = plane_normal(P);
    const V3 rel = {s.c[0] - P.c[0], s.c[1] - P.c[1], s.c[2] - P.c[2]};
    const double sg = dot(rel, np) < 0 ? -1.0 : 1.0;
    // body-frame direction of the wanted outward normal: -s np
    const V3 m = {-sg * (s.R[0][0] * np[0] + s.R[1][0] * np[1] + s.R[2][0] * np[2]),
                  -sg * (s.R[0][1] * np[0] + s.R[1][1] * np[1] + s.R[2][1] * np[2]),
                  -sg * (s.R[0][2] * np[0] + s.R[1][2] * np[1] + s.R[2][2] * np[2])};
    double a, b;
    support_angles(s, m, a, b);
    PairOut o;
    o.info = 0;
    o.pi = point(s, a, b);
    const V3 d = {o.pi[0] - P.c[0], o.pi[1] - P.c[1], o.pi[2] - P.c[2]};
    const double h = dot(d, np);
    o.pj = {o.pi[0] - h * np[0], o.pi[1] - h * np[1], o.pi[2] - h * np[2]};
    o.nij = {sg * np[0], sg * np[1], sg * np[2]};
    const V3 df = {o.pi[0] - o.pj[0], o.pi[1] - o.pj[1], o.pi[2] - o.pj[2]};
    o.dij = dot(df, o.nij);
    // plane coordinates of pj (columns 1, 2 of the plane's rotation)
    const V3 e = {o.pj[0] - P.c[0], o.pj[1] - P.c[1], o.pj[2] - P.c[2]};
    o.u[0] = a;
    o.u[1] = b;
    o.u[2] = P.R[0][1] * e[0] + P.R[1][1] * e[1] + P.R[2][1] * e[2];
    o.u[3] = P.R[0][2] * e[0] + P.R[1][2] * e[1] + P.R[2][2] * e[2];
    return o;
}

// ------------------------------------------------------------- separation bound
// For convex bodies (squareness in (0, 2)) the distance is at least the gap along any unit
// direction u: (support point of body 2 in -u - support point of body 1 in u).u.  With u
// along the line of centres this bounds the pairs that cannot be in contact.
inline double support_angle2(const SE& s, double m0, double m1) {
    const double ke = 1.0 / (2 - s.e);
    return std::atan2(sgn(m1) * std::pow(std::abs(s.r[1] * m1), ke), sgn(m0) * std::pow(std::abs(s.r[0] * m0), ke));
}
inline V3 point2(const SE& s, double b);
inline double support_gap(const SE& s1, const SE& s2, int dim) {
    V3 d = {s2.c[0] - s1.c[0], s2.c[1] - s1.c[1], dim == 3 ? s2.c[2] - s1.c[2] : 0.0};
    const double l = norm(d);
    if (!(l > 0)) return -INFINITY;
    const V3 u = {d[0] / l, d[1] / l, d[2] / l};
    // body-frame directions R^T u (body 1) and -R^T u (body 2)
    V3 m1 = {0, 0, 0}, m2 = {0, 0, 0};
    for (int k = 0; k < 3; ++k)
        for (int r = 0; r < dim; ++r) {
            m1[k] += s1.R[r][k] * u[r];
            m2[k] -= s2.R[r][k] * u[r];
        }
    V3 p1, p2;
    if (dim == 3) {
        double a, b;
        support_angles(s1, m1, a, b);
        p1 = point(s1, a, b);
        support_angles(s2, m2, a, b);
        p2 = point(s2, a, b);
    } else {
        p1 = point2(s1, support_angle2(s1, m1[0], m1[1]));
        p2 = point2(s2, support_angle2(s2, m2[0], m2[1]));
    }
    return (p2[0] - p1[0]) * u[0] + (p2[1] - p1[1]) * u[1] + (p2[2] - p1[2]) * u[2];
}

// ------------------------------------------------------------- SE - SE (2D)
// A 2D body uses c[0..1], the upper-left 2x2 block of R (a rotation about z), r[0..1], e.
struct Local2 {
    double p[2], N[2], pb[2], Nb[2];  // body-frame point, unnormalised normal, d/db
};
inline Local2 local2(const SE& s, double b) {
    const double cb = std::cos(b), sb = std::sin(b), e = s.e, k = 2 - s.e;
    Local2 L;
    L.p[0] = s.r[0] * sgn(cb) * std::pow(std::abs(cb), e);
    L.p[1] = s.r[1] * sgn(sb) * std::pow(std::abs(sb), e);
    L.N[0] = s.r[1] * sgn(cb) * std::pow(std::abs(cb), k);
    L.N[1] = s.r[0] * sgn(sb) * std::pow(std::abs(sb), k);
    // d/db sign(cos b)|cos b|^m = -m sin b |cos b|^(m-1);  d/db sign(sin b)|sin b|^m = m cos b |sin b|^(m-1)
    L.pb[0] = -s.r[0] * e * sb * std::pow(std::abs(cb), e - 1);
    L.pb[1] = s.r[1] * e * cb * std::pow(std::abs(sb), e - 1);
    L.Nb[0] = -s.r[1] * k * sb * std::pow(std::abs(cb), k - 1);
    L.Nb[1] = s.r[0] * k * cb * std::pow(std::abs(sb), k - 1);
    return L;
}
inline void mv2(const SE& s, const double* x, double* y) {
    y[0] = s.R[0][0] * x[0] + s.R[0][1] * x[1];
    y[1] = s.R[1][0] * x[0] + s.R[1][1] * x[1];
}
inline V3 point2(const SE& s, double b) {
    const Local2 L = local2(s, b);
    double w[2];
    mv2(s, L.p, w);
    return {w[0] + s.c[0], w[1] + s.c[1], 0.0};
}
inline V3 normal2(const SE& s, double b) {
    const Local2 L = local2(s, b);
    double w[2];
    mv2(s, L.N, w);
    const double l = std::sqrt(w[0] * w[0] + w[1] * w[1]);
    return {w[0] / l, w[1] / l, 0.0};
}
// F and its Jacobian (column-major 2x2) for u = (b1, b2)
inline void se2_F(const SE& s1, const SE& s2, const double* u, double* F) {
    const Local2 L1 = local2(s1, u[0]), L2 = local2(s2, u[1]);
    double p1[2], p2[2], n1[2], n2[2];
    mv2(s1, L1.p, p1);
    mv2(s2, L2.p, p2);
    mv2(s1, L1.N, n1);
    mv2(s2, L2.N, n2);
    const double d[2] = {p2[0] + s2.c[0] - p1[0] - s1.c[0], p2[1] + s2.c[1] - p1[1] - s1.c[1]};
    F[0] = d[0] * n1[1] - d[1] * n1[0];
    F[1] = n1[0] * n2[0] + n1[1] * n2[1] + std::sqrt(n1[0] * n1[0] + n1[1] * n1[1]) *
                                               std::sqrt(n2[0] * n2[0] + n2[1] * n2[1]);
}
inline void se2_J(const SE& s1, const SE& s2, const double* u, double* J) {
    const Local2 L1 = local2(s1, u[0]), L2 = local2(s2, u[1]);
    double p1[2], p2[2], n1[2], n2[2], pb1[2], pb2[2], nb1[2], nb2[2];
    mv2(s1, L1.p, p1);
    mv2(s2, L2.p, p2);
    mv2(s1, L1.N, n1);
    mv2(s2, L2.N, n2);
    mv2(s1, L1.pb, pb1);
    mv2(s2, L2.pb, pb2);
    mv2(s1, L1.Nb, nb1);
    mv2(s2, L2.Nb, nb2);
    const double d[2] = {p2[0] + s2.c[0] - p1[0] - s1.c[0], p2[1] + s2.c[1] - p1[1] - s1.c[1]};
    const double l1 = std::sqrt(n1[0] * n1[0] + n1[1] * n1[1]), l2 = std::sqrt(n2[0] * n2[0] + n2[1] * n2[1]);
    // column b1: d' = -p1', n1' = R1 Nb1, n2' = 0
    J[0] = -pb1[0] * n1[1] + pb1[1] * n1[0] + d[0] * nb1[1] - d[1] * nb1[0];
    J[1] = nb1[0] * n2[0] + nb1[1] * n2[1] + (n1[0] * nb1[0] + n1[1] * nb1[1]) / l1 * l2;
    // column b2: d' = p2', n1' = 0, n2' = R2 Nb2
    J[2] = pb2[0] * n1[1] - pb2[1] * n1[0];
    J[3] = n1[0] * nb2[0] + n1[1] * nb2[1] + l1 * (n2[0] * nb2[0] + n2[1] * nb2[1]) / l2;
}
// closest_points(superellipsoid<2>, superellipsoid<2>), closest_points.hpp:65-262
inline PairOut se2_se2(const SE& s1, const SE& s2) {
    const int num = 4;
    const auto g1 = sorted_unique(binit_xy(s1, num)), g2 = sorted_unique(binit_xy(s2, num));
    double best = INFINITY;
    double u[2] = {g1[0], g2[0]};
    for (double b1 : g1) {
        const V3 P1 = point2(s1, b1), N1 = normal2(s1, b1);
        for (double b2 : g2) {
            const V3 P2 = point2(s2, b2), N2 = normal2(s2, b2);
            const double dx = P1[0] - P2[0], dy = P1[1] - P2[1];
            const double v = std::sqrt(dx * dx + dy * dy) + 2 * (1 + (N1[0] * N2[0] + N1[1] * N2[1]));
            if (v < best) {  // first minimum in row-major order
                best = v;
                u[0] = b1;
                u[1] = b2;
            }
        }
    }
    const HybrResult h = hybrj<2>([&](const double* x, double* F) { se2_F(s1, s2, x, F); },
                                  [&](const double* x, double* J) { se2_J(s1, s2, x, J); }, u);
    PairOut o;
    o.info = h.info;
    o.nfev = h.nfev;
    o.u[0] = u[0];
    o.u[1] = u[1];
    o.u[2] = o.u[3] = 0.0;
    o.pi = point2(s1, u[0]);
    o.pj = point2(s2, u[1]);
    o.nij = normal2(s2, u[1]);
    const double dx = o.pi[0] - o.pj[0], dy = o.pi[1] - o.pj[1];
    o.dij = sgn(dx * o.nij[0] + dy * o.nij[1]) * std::sqrt(dx * dx + dy * dy);
    return o;
}

// ------------------------------------------------------------------ damped Newton
// newton_method (utils.hpp:81-118) in n unknowns: d = solve(J(u), -F(u)); return when
// |d| < xtol (tested before the residual) or |F(u)| < ftol; otherwise a backtracking line
// search t = 1, 0.99, 0.98, ... while |F(u + t d)| > |F(u)| and t > 0.01, then u += t d; at
// most itermax steps (then -1).  The reference solves with LAPACK's dgesv (through
// xt::linalg::solve); the solve here restates the published reference-LAPACK algorithm for a
// small dense matrix: dgetf2 (column pivot = the first entry of largest |a| on or below the
// diagonal, multipliers scaled by the pivot's reciprocal when |pivot| >= the safe minimum,
// rank-1 update of the trailing block) and dgetrs (the row interchanges, then the unit lower
// and the upper triangular solves).  An optimised LAPACK orders these operations its own way,
// so the last bits of d are not pinned.  A zero pivot (the reference's solve throws there)
// ends the method with -2.  Norms are sqrt(sum of squares).
constexpr double kSafeMin = 2.2250738585072014e-308;  // dlamch('S')

template <int N>
inline bool lu_solve(double* A, double* b) {  // A column-major N x N (overwritten), b (in: rhs, out: x)
    int piv[N];
    for (int j = 0; j < N; ++j) {
        int p = j;
        double big = std::abs(A[j + N * j]);
        for (int i = j + 1; i < N; ++i)
            if (std::abs(A[i + N * j]) > big) {
                big = std::abs(A[i + N * j]);
                p = i;
            }
        piv[j] = p;
        if (A[p + N * j] == 0.0) return false;
        if (p != j)
            for (int k = 0; k < N; ++k) std::swap(A[j + N * k], A[p + N * k]);
        const double pv = A[j + N * j];
        if (std::abs(pv) >= kSafeMin) {
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
        if (piv[j] != j) std::swap(b[j], b[piv[j]]);
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
inline double norm_n(const double* x) {
    double s = 0.0;
    for (int k = 0; k < N; ++k) s += x[k] * x[k];
    return std::sqrt(s);
}

// returns the iterations taken (>= 0), -1 after itermax steps, -2 on a zero pivot
template <int N, typename Fun, typename Jac>
inline int newton(Fun&& fun, Jac&& jac, double* u, int itermax = 200, double ftol = 1.0e-10, double xtol = 1.0e-7) {
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
inline double linspace_at(double start, double stop, int num, int k) {
    if (k == num - 1) return stop;
    return start + k * ((stop - start) / (num - 1));
}

// ------------------------------------------------------- sphere - superellipsoid
// A sphere of radius r is the superellipsoid with semi-axes (r, r, r) and squareness (1, 1):
// its parametrisation is then exactly sphere::point (sphere.hpp:195-211), since
// sign(t)|t|^1 = t.  Its unit normal is sphere::normal (sphere.hpp:213-234).
inline SE as_se(const V3& c, const M3& R, double r) {
    SE s;
    s.c = c;
    s.R = R;
    s.r[0] = s.r[1] = s.r[2] = r;
    s.e = s.n = 1.0;
    return s;
}
inline V3 sphere_normal(const SE& sph, double a, double b) {  // sphere.hpp:225-234
    const V3 n = {std::cos(a) * std::cos(b), std::cos(a) * std::sin(b), std::sin(a)};
    V3 w = mv(sph.R, n);
    const double l = norm(w);
    for (auto& x : w) x /= l;
    return w;
}

// closest_points(sphere<3>, superellipsoid<3>), closest_points.hpp:944-1282: unknowns
// u = (a1, b1, a2, b2), the superellipsoid's angles then the sphere's;
//   F = [ (p2 - p1) x n1 ; n1.n2 + |n1||n2| ],  n1 = sign(cos a1) N1(a1, b1),  n2 = sign(cos a2) N2(a2, b2)
// with N the unnormalised outward normals of superellipsoid::normal (the reference's
// expressions carry the factor sign(cos a) on both normals, :1013-1037).  The Jacobian is the
// chain rule on the parametrisation's derivatives.
inline void sphse_F(const SE& s1, const SE& s2, const double* u, double* F) {
    const Local L1 = local(s1, u[0], u[1]), L2 = local(s2, u[2], u[3]);
    const double k1 = sgn(std::cos(u[0])), k2 = sgn(std::cos(u[2]));
    const V3 p1 = mv(s1.R, L1.p), p2 = mv(s2.R, L2.p);
    const V3 d = {p2[0] + s2.c[0] - p1[0] - s1.c[0], p2[1] + s2.c[1] - p1[1] - s1.c[1],
                  p2[2] + s2.c[2] - p1[2] - s1.c[2]};
    V3 n1 = mv(s1.R, L1.N), n2 = mv(s2.R, L2.N);
    for (int c = 0; c < 3; ++c) {
        n1[c] *= k1;
        n2[c] *= k2;
    }
    const V3 x = cross(d, n1);
    F[0] = x[0];
    F[1] = x[1];
    F[2] = x[2];
    F[3] = dot(n1, n2) + norm(n1) * norm(n2);
}
inline void sphse_J(const SE& s1, const SE& s2, const double* u, double* J) {  // column-major 4x4
    const Local L1 = local(s1, u[0], u[1]), L2 = local(s2, u[2], u[3]);
    const double k1 = sgn(std::cos(u[0])), k2 = sgn(std::cos(u[2]));
    const V3 p1 = mv(s1.R, L1.p), p2 = mv(s2.R, L2.p);
    const V3 d = {p2[0] + s2.c[0] - p1[0] - s1.c[0], p2[1] + s2.c[1] - p1[1] - s1.c[1],
                  p2[2] + s2.c[2] - p1[2] - s1.c[2]};
    V3 n1 = mv(s1.R, L1.N), n2 = mv(s2.R, L2.N);
    const V3 z = {0, 0, 0};
    V3 dd[4], dn1[4], dn2[4];
    const V3 pa1 = mv(s1.R, L1.pa), pb1 = mv(s1.R, L1.pb);
    dd[0] = {-pa1[0], -pa1[1], -pa1[2]};
    dd[1] = {-pb1[0], -pb1[1], -pb1[2]};
    dd[2] = mv(s2.R, L2.pa);
    dd[3] = mv(s2.R, L2.pb);
    dn1[0] = mv(s1.R, L1.Na);
    dn1[1] = mv(s1.R, L1.Nb);
    dn1[2] = dn1[3] = z;
    dn2[0] = dn2[1] = z;
    dn2[2] = mv(s2.R, L2.Na);
    dn2[3] = mv(s2.R, L2.Nb);
    for (int c = 0; c < 3; ++c) {
        n1[c] *= k1;
        n2[c] *= k2;
        for (int q = 0; q < 4; ++q) {
            dn1[q][c] *= k1;
            dn2[q][c] *= k2;
        }
    }
    const double l1 = norm(n1), l2 = norm(n2);
    for (int q = 0; q < 4; ++q) {
        const V3 a = cross(dd[q], n1), b = cross(d, dn1[q]);
        J[0 + 4 * q] = a[0] + b[0];
        J[1 + 4 * q] = a[1] + b[1];
        J[2 + 4 * q] = a[2] + b[2];
        J[3 + 4 * q] = dot(dn1[q], n2) + dot(n1, dn2[q]) + dot(n1, dn1[q]) / l1 * l2 + l1 * dot(n2, dn2[q]) / l2;
    }
}
// start (closest_points.hpp:1262-1274): ten angle pairs per body, (ainit(k), binit(k)) with
// ainit = linspace(-pi/2, pi/2, 10), binit = linspace(-pi, pi, 10); the first minimum of
// |p1 - p2| over the 10 x 10 pairs in row-major order
inline void sphse_start(const SE& s1, const SE& s2, double* u0) {
    const double pi = 4 * std::atan(1);
    constexpr int num = 10;
    double A[num], Bv[num];
    for (int k = 0; k < num; ++k) {
        A[k] = linspace_at(-pi / 2, pi / 2, num, k);
        Bv[k] = linspace_at(-pi, pi, num, k);
    }
    V3 P1[num], P2[num];
    for (int k = 0; k < num; ++k) {
        P1[k] = point(s1, A[k], Bv[k]);
        P2[k] = point(s2, A[k], Bv[k]);
    }
    double best = INFINITY;
    int bi = 0, bj = 0;
    for (int i = 0; i < num; ++i)
        for (int j = 0; j < num; ++j) {
            const V3 df = {P1[i][0] - P2[j][0], P1[i][1] - P2[j][1], P1[i][2] - P2[j][2]};
            const double v = norm(df);
            if (v < best) {
                best = v;
                bi = i;
                bj = j;
            }
        }
    u0[0] = A[bi];
    u0[1] = Bv[bi];
    u0[2] = A[bj];
    u0[3] = Bv[bj];
}
// 2D start (closest_points.hpp:1425-1436): binit = {-pi, -pi/2, 0.001, pi/2} on both bodies,
// the first minimum of |p1 - p2| over the 4 x 4 pairs in row-major order
inline void sphse2_start(const SE& s1, const SE& s2, double* u0) {
    const double pi = 4 * std::atan(1);
    const double binit[4] = {-pi, -pi / 2, 0.001, pi / 2};
    double best = INFINITY;
    u0[0] = u0[1] = binit[0];
    for (int i = 0; i < 4; ++i) {
        const V3 P1 = point2(s1, binit[i]);
        for (int j = 0; j < 4; ++j) {
            const V3 P2 = point2(s2, binit[j]);
            const double dx = P1[0] - P2[0], dy = P1[1] - P2[1];
            const double v = std::sqrt(dx * dx + dy * dy);
            if (v < best) {
                best = v;
                u0[0] = binit[i];
                u0[1] = binit[j];
            }
        }
    }
}

// closest_points(sphere, superellipsoid) in the reference's result convention
// (closest_points.hpp:1275-1280 in 3D, 1437-1441 in 2D): pi on the superellipsoid, pj on the
// sphere, nij = the sphere's unit normal at pj, dij = (pi - pj).nij; info = the Newton
// method's return.  2D: u = (b1, b2) and F = [ (p2 - p1) x n1 ; n1.n2 + |n1||n2| ] with
// n2 = the rotated r (cos b2, sin b2): se2_F / se2_J with the sphere as the superellipsoid
// (r, r), e = 1 (the 2D expressions carry no sign factors).
inline PairOut sphere_se_newton(const SE& se, const SE& sph, int dim) {
    PairOut o;
    double u[4] = {0, 0, 0, 0};
    if (dim == 3) {
        sphse_start(se, sph, u);
        o.info = newton<4>([&](const double* x, double* F) { sphse_F(se, sph, x, F); },
                           [&](const double* x, double* J) { sphse_J(se, sph, x, J); }, u);
        o.pi = point(se, u[0], u[1]);
        o.pj = point(sph, u[2], u[3]);
        o.nij = sphere_normal(sph, u[2], u[3]);
    } else {
        sphse2_start(se, sph, u);
        o.info = newton<2>([&](const double* x, double* F) { se2_F(se, sph, x, F); },
                           [&](const double* x, double* J) { se2_J(se, sph, x, J); }, u);
        o.pi = point2(se, u[0]);
        o.pj = point2(sph, u[1]);
        o.nij = normal2(sph, u[1]);  // sphere::normal(b): the rotated r (cos b, sin b), normalised
    }
    for (int k = 0; k < 4; ++k) o.u[k] = u[k];
    const V3 df = {o.pi[0] - o.pj[0], o.pi[1] - o.pj[1], o.pi[2] - o.pj[2]};
    o.dij = dot(df, o.nij);
    return o;
}

// The engine's acceptance test.  F = 0 of the reference's system also holds at pairs that are
// not the closest points: the farther point of the sphere (the factors sign(cos a) let the
// two normals be parallel instead of opposite) or the far side of the superellipsoid, and
// its start (ten samples per body along a diagonal of the angle square) often leads the
// Newton method there, or to no convergence in 200 steps (the reference then keeps the last
// iterate; on a singular Jacobian its solve throws).  For a convex body (squareness in
// (0, 2)) a surface point p whose outward unit normal points at the sphere's centre c,
// c - p = t N(p) with t > 0, is the point nearest c, and the sphere's nearest point then lies
// on the segment from c to p.  The Newton result is kept when it converged and both hold to
// within cos >= 1 - 1e-6; otherwise the pair is solved as the pair of superellipsoids it is
// (the sphere with semi-axes (r, r, r) and squareness 1: se_se / se2_se2).
inline bool sphere_se_valid(const SE& se, const SE& sph, int dim, const PairOut& o) {
    if (o.info < 0) return false;
    const double cos_tol = 1.0 - 1e-6;
    const V3 w = {o.pi[0] - sph.c[0], o.pi[1] - sph.c[1], dim == 3 ? o.pi[2] - sph.c[2] : 0.0};
    const double L = norm(w);
    if (!(L > 0)) return false;
    const V3 nu = {w[0] / L, w[1] / L, w[2] / L};
    const V3 N = dim == 3 ? normal(se, o.u[0], o.u[1]) : normal2(se, o.u[0]);
    return -dot(N, nu) >= cos_tol && dot(o.nij, nu) >= cos_tol;
}

// The engine's pair of (body i, body j), one of them a sphere (as_se) and the other a
// superellipsoid, labelled as every other closest_points function labels its pair: pi on
// body i, pj on body j, nij the outward normal of j at pj, pointing toward i (so that
// dij + dt nij.(v_i - v_j) is the first-order gap).  The reference's sphere-superellipsoid
// functions give, for (sphere i, superellipsoid j), the points and normal of the pair (j, i)
// (closest_points.hpp:1275-1280), and for (superellipsoid i, sphere j) that result swapped
// and negated (:1295-1302); with either labelling the contact row would push the bodies
// together.  Here the Newton result R (pi on the superellipsoid, nij the sphere's normal) is
// labelled by body when sphere_se_valid accepts it (info = its iterations); otherwise the
// superellipsoid-pair solve of (i, j) gives the pair (info = 100 + the hybrid method's info).
inline PairOut sphere_se_pair(const SE& bi, const SE& bj, bool i_is_se, int dim) {
    const SE& se = i_is_se ? bi : bj;
    const SE& sph = i_is_se ? bj : bi;
    PairOut o = sphere_se_newton(se, sph, dim);
    if (sphere_se_valid(se, sph, dim, o)) {
        if (!i_is_se) {
            std::swap(o.pi, o.pj);
            for (auto& x : o.nij) x = -x;
        }
        return o;
    }
    o = dim == 3 ? se_se(bi, bj) : se2_se2(bi, bj);
    o.info += 100;
    return o;
}

// closest_points(superellipsoid<2>, plane<2>), closest_points.hpp:1783-1949, in closed form as
// in 3D (se_plane): its system's second equation receives the signed centre-plane distance
// where it needs the side (:1787, :1845), so its Newton has no root to find for bodies nearer
// to the plane than one length unit; the solution of the intended system is the body point
// whose outward normal is opposite to the plane normal oriented toward the body.  The plane
// normal is column 0 of the plane's rotation (plane.hpp:143-147); u[1] = the plane coordinate
// of pj along column 1.
inline PairOut se2_plane(const SE& s, const Plane& P) {
    const double np[2] = {P.R[0][0], P.R[1][0]};
    const double rel[2] = {s.c[0] - P.c[0], s.c[1] - P.c[1]};
    const double sg = rel[0] * np[0] + rel[1] * np[1] < 0 ? -1.0 : 1.0;
    const double m0 = -sg * (s.R[0][0] * np[0] + s.R[1][0] * np[1]);
    const double m1 = -sg * (s.R[0][1] * np[0] + s.R[1][1] * np[1]);
    const double b = support_angle2(s, m0, m1);
    PairOut o;
    o.info = 0;
    o.pi = point2(s, b);
    const double h = (o.pi[0] - P.c[0]) * np[0] + (o.pi[1] - P.c[1]) * np[1];
    o.pj = {o.pi[0] - h * np[0], o.pi[1] - h * np[1], 0.0};
    o.nij = {sg * np[0], sg * np[1], 0.0};
    o.dij = (o.pi[0] - o.pj[0]) * o.nij[0] + (o.pi[1] - o.pj[1]) * o.nij[1];
    o.u[0] = b;
    o.u[1] = P.R[0][1] * (o.pj[0] - P.c[0]) + P.R[1][1] * (o.pj[1] - P.c[1]);
    o.u[2] = o.u[3] = 0.0;
    return o;
}

}  // namespace orc_se
