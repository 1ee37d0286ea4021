// minpack.cuh -- Powell's hybrid method (MINPACK hybrj with the analytic Jacobian) on the
// device, FP64, for n = 2 or 4 unknowns: the superellipsoid closest-point solves of se.cu and
// the fallback of the sphere-superellipsoid Newton method (se_newton.cuh).
//
// Restated from the published MINPACK algorithm that the reference calls as hybrd1
// (minpack.hpp:338-923, src/minpack.cpp:36-667): QR of the Jacobian, dogleg step in a trust
// region, Broyden rank-1 updates with Givens rotations; mode 2 with unit scaling, factor 100,
// xtol 1e-10, maxfev 200 (n + 1).  0-based, templated on n.
#pragma once
#include "common.cuh"

namespace scopi_gpu {
namespace se {
namespace {
// ------------------------------------------------------- MINPACK pieces (n = N: 4 in 3D, 2 in 2D)
constexpr double kEps = 2.220446049250313e-16;
constexpr double kGiant = 1.7976931348623157e308;

__device__ inline double enorm(int n, const double* x) {
    const double rdwarf = 3.834e-20, rgiant = 1.304e19;
    double s1 = 0, s2 = 0, s3 = 0, x1max = 0, x3max = 0;
    const double agiant = rgiant / n;
    for (int i = 0; i < n; ++i) {
        const double xabs = fabs(x[i]);
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
    if (s1 != 0) return x1max * sqrt(s1 + (s2 / x1max) / x1max);
    if (s2 != 0) {
        if (s2 >= x3max) return sqrt(s2 * (1 + (x3max / s2) * (x3max * s3)));
        return sqrt(x3max * ((s2 / x3max) + (x3max * s3)));
    }
    return x3max * sqrt(s3);
}

template <int N>
__device__ void qrfac(double* a, double* rdiag, double* acnorm) {
    for (int j = 0; j < N; ++j) {
        acnorm[j] = enorm(N, a + j * N);
        rdiag[j] = acnorm[j];
    }
    for (int j = 0; j < N; ++j) {
        double ajnorm = enorm(N - j, a + j + j * N);
        if (ajnorm != 0) {
            if (a[j + j * N] < 0) ajnorm = -ajnorm;
            for (int i = j; i < N; ++i) a[i + j * N] /= ajnorm;
            a[j + j * N] += 1;
            for (int k = j + 1; k < N; ++k) {
                double sum = 0;
                for (int i = j; i < N; ++i) sum += a[i + j * N] * a[i + k * N];
                const double temp = sum / a[j + j * N];
                for (int i = j; i < N; ++i) a[i + k * N] -= temp * a[i + j * N];
            }
        }
        rdiag[j] = -ajnorm;
    }
}

template <int N>
__device__ void qform(double* q, double* wa) {
    for (int j = 1; j < N; ++j)
        for (int i = 0; i < j; ++i) q[i + j * N] = 0;
    for (int l = 0; l < N; ++l) {
        const int k = N - 1 - l;
        for (int i = k; i < N; ++i) {
            wa[i] = q[i + k * N];
            q[i + k * N] = 0;
        }
        q[k + k * N] = 1;
        if (wa[k] == 0) continue;
        for (int j = k; j < N; ++j) {
            double sum = 0;
            for (int i = k; i < N; ++i) sum += q[i + j * N] * wa[i];
            const double temp = sum / wa[k];
            for (int i = k; i < N; ++i) q[i + j * N] -= temp * wa[i];
        }
    }
}

template <int N>
__device__ void dogleg(const double* r, const double* diag, const double* qtb, double delta, double* x, double* wa1,
                       double* wa2) {
    int jj = (N * (N + 1)) / 2;
    for (int k = 1; k <= N; ++k) {
        const int j = N - k;
        jj -= k;
        int l = jj + 1;
        double sum = 0;
        for (int i = j + 1; i < N; ++i) sum += r[l++] * x[i];
        double temp = r[jj];
        if (temp == 0) {
            int ll = j;
            for (int i = 0; i <= j; ++i) {
                temp = fmax(temp, fabs(r[ll]));
                ll += N - i - 1;
            }
            temp = kEps * temp;
            if (temp == 0) temp = kEps;
        }
        x[j] = (qtb[j] - sum) / temp;
    }
    for (int j = 0; j < N; ++j) {
        wa1[j] = 0;
        wa2[j] = diag[j] * x[j];
    }
    const double qnorm = enorm(N, wa2);
    if (qnorm <= delta) return;
    int l = 0;
    for (int j = 0; j < N; ++j) {
        const double temp = qtb[j];
        for (int i = j; i < N; ++i) wa1[i] += r[l++] * temp;
        wa1[j] /= diag[j];
    }
    const double gnorm = enorm(N, wa1);
    double sgnorm = 0, alpha = delta / qnorm;
    if (gnorm != 0) {
        for (int j = 0; j < N; ++j) wa1[j] = (wa1[j] / gnorm) / diag[j];
        l = 0;
        for (int j = 0; j < N; ++j) {
            double sum = 0;
            for (int i = j; i < N; ++i) sum += r[l++] * wa1[i];
            wa2[j] = sum;
        }
        const double temp = enorm(N, wa2);
        sgnorm = (gnorm / temp) / temp;
        alpha = 0;
        if (sgnorm < delta) {
            const double bnorm = enorm(N, qtb);
            double t = (bnorm / gnorm) * (bnorm / qnorm) * (sgnorm / delta);
            t = t - (delta / qnorm) * (sgnorm / delta) * (sgnorm / delta) +
                sqrt((t - (delta / qnorm)) * (t - (delta / qnorm)) +
                     (1 - (delta / qnorm) * (delta / qnorm)) * (1 - (sgnorm / delta) * (sgnorm / delta)));
            alpha = ((delta / qnorm) * (1 - (sgnorm / delta) * (sgnorm / delta))) / t;
        }
    }
    const double temp = (1 - alpha) * fmin(sgnorm, delta);
    for (int j = 0; j < N; ++j) x[j] = temp * wa1[j] + alpha * x[j];
}

template <int N>
__device__ void r1updt(double* s, const double* u, double* v, double* w) {
    const int m = N;
    int jj = (N * (2 * m - N + 1)) / 2 - (m - N) - 1;
    int l = jj;
    for (int i = N - 1; i < m; ++i) w[i] = s[l++];
    for (int nmj = 1; nmj <= N - 1; ++nmj) {
        const int j = N - 1 - nmj;
        jj -= m - j;
        w[j] = 0;
        if (v[j] != 0) {
            double cs, sn, tau;
            if (fabs(v[N - 1]) < fabs(v[j])) {
                const double cotan = v[N - 1] / v[j];
                sn = 0.5 / sqrt(0.25 + 0.25 * cotan * cotan);
                cs = sn * cotan;
                tau = 1;
                if (fabs(cs) * kGiant > 1) tau = 1 / cs;
            } else {
                const double tn = v[j] / v[N - 1];
                cs = 0.5 / sqrt(0.25 + 0.25 * tn * tn);
                sn = cs * tn;
                tau = sn;
            }
            v[N - 1] = sn * v[j] + cs * v[N - 1];
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
    for (int i = 0; i < m; ++i) w[i] += v[N - 1] * u[i];
    for (int j = 0; j < N - 1; ++j) {
        if (w[j] != 0) {
            double cs, sn, tau;
            if (fabs(s[jj]) < fabs(w[j])) {
                const double cotan = s[jj] / w[j];
                sn = 0.5 / sqrt(0.25 + 0.25 * cotan * cotan);
                cs = sn * cotan;
                tau = 1;
                if (fabs(cs) * kGiant > 1) tau = 1 / cs;
            } else {
                const double tn = w[j] / s[jj];
                cs = 0.5 / sqrt(0.25 + 0.25 * tn * tn);
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
        jj += m - j;
    }
    l = jj;
    for (int i = N - 1; i < m; ++i) s[l++] = w[i];
}

template <int N>
__device__ void r1mpyq(int m, double* a, int lda, const double* v, const double* w) {
    for (int nmj = 1; nmj <= N - 1; ++nmj) {
        const int j = N - 1 - nmj;
        double cs, sn;
        if (fabs(v[j]) > 1) {
            cs = 1 / v[j];
            sn = sqrt(1 - cs * cs);
        } else {
            sn = v[j];
            cs = sqrt(1 - sn * sn);
        }
        for (int i = 0; i < m; ++i) {
            const double temp = cs * a[i + j * lda] - sn * a[i + (N - 1) * lda];
            a[i + (N - 1) * lda] = sn * a[i + j * lda] + cs * a[i + (N - 1) * lda];
            a[i + j * lda] = temp;
        }
    }
    for (int j = 0; j < N - 1; ++j) {
        double cs, sn;
        if (fabs(w[j]) > 1) {
            cs = 1 / w[j];
            sn = sqrt(1 - cs * cs);
        } else {
            sn = w[j];
            cs = sqrt(1 - sn * sn);
        }
        for (int i = 0; i < m; ++i) {
            const double temp = cs * a[i + j * lda] + sn * a[i + (N - 1) * lda];
            a[i + (N - 1) * lda] = -sn * a[i + j * lda] + cs * a[i + (N - 1) * lda];
            a[i + j * lda] = temp;
        }
    }
}

// hybrd1 with the analytic Jacobian; returns info (1..5); at most maxfev evaluations of F.
// fun(x, F) and jac(x, J) (column-major) evaluate the system.
template <int N, typename Fun, typename Jac>
__device__ int hybrj(Fun&& fun, Jac&& jac, double* x) {
    const double p1 = 0.1, p5 = 0.5, p001 = 1e-3, p0001 = 1e-4, xtol = 1e-10, factor = 100.0;
    const int maxfev = 200 * (N + 1);
    double fvec[N], fjac[N * N], diag[N], r[(N * (N + 1)) / 2], qtf[N], wa1[N], wa2[N], wa3[N], wa4[N];
    for (int j = 0; j < N; ++j) diag[j] = 1.0;
    fun(x, fvec);
    int nfev = 1;
    double fnorm = enorm(N, fvec);
    int iter = 1, ncsuc = 0, ncfail = 0, nslow1 = 0, nslow2 = 0;
    double delta = 0, xnorm = 0;
    for (;;) {
        bool jeval = true;
        jac(x, fjac);
        qrfac<N>(fjac, wa1, wa2);
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
        qform<N>(fjac, wa1);
        for (;;) {
            dogleg<N>(r, diag, qtf, delta, wa1, wa2, wa3);
            for (int j = 0; j < N; ++j) {
                wa1[j] = -wa1[j];
                wa2[j] = x[j] + wa1[j];
                wa3[j] = diag[j] * wa1[j];
            }
            const double pnorm = enorm(N, wa3);
            if (iter == 1) delta = fmin(delta, pnorm);
            fun(wa2, wa4);
            ++nfev;
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
                if (ratio >= p5 || ncsuc > 1) delta = fmax(delta, pnorm / p5);
                if (fabs(ratio - 1) <= p1) delta = pnorm / p5;
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
            if (delta <= xtol * xnorm || fnorm == 0) return 1;
            int info = 0;
            if (nfev >= maxfev) info = 2;
            if (p1 * fmax(p1 * delta, pnorm) <= kEps * xnorm) info = 3;
            if (nslow2 == 5) info = 4;
            if (nslow1 == 10) info = 5;
            if (info != 0) return info;
            if (ncfail == 2) break;
            for (int j = 0; j < N; ++j) {
                double sum = 0;
                for (int i = 0; i < N; ++i) sum += fjac[i + j * N] * wa4[i];
                wa2[j] = (sum - wa3[j]) / pnorm;
                wa1[j] = diag[j] * ((diag[j] * wa1[j]) / pnorm);
                if (ratio >= p0001) qtf[j] = sum;
            }
            r1updt<N>(r, wa1, wa2, wa3);
            r1mpyq<N>(N, fjac, N, wa2, wa3);
            r1mpyq<N>(1, qtf, 1, wa2, wa3);
            jeval = false;
        }
    }
}

}  // namespace
}  // namespace se
}  // namespace scopi_gpu
