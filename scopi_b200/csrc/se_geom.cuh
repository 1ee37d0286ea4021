// se_geom.cuh -- 3D superellipsoid geometry on the device (FP64).
//
// Parametrisation (include/scopi/objects/types/superellipsoid.hpp:291-325), body frame:
//   p(a, b) = (rx C(a,n) C(b,e), ry C(a,n) S(b,e), rz S(a,n)),
//   N(a, b) = (ry rz C(a,2-n) C(b,2-e), rx rz C(a,2-n) S(b,2-e), rx ry S(a,2-n))  (outward, unnormalised)
// with C(t,k) = sign(cos t)|cos t|^k, S(t,k) = sign(sin t)|sin t|^k; world = R(q) p + c.
#pragma once
#include "common.cuh"

namespace scopi_gpu {
namespace se {

struct Body {
    double c[3];
    double R[9];  // row-major rotation (body -> world)
    double r[3];
    double e, n;
};

__device__ __forceinline__ double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
__device__ __forceinline__ double cpow(double x, double k) {
    const double c = cos(x);
    return sgn(c) * pow(fabs(c), k);
}
__device__ __forceinline__ double spow(double x, double k) {
    const double s = sin(x);
    return sgn(s) * pow(fabs(s), k);
}
__device__ __forceinline__ double dcpow(double x, double k) { return -k * sin(x) * pow(fabs(cos(x)), k - 1); }
__device__ __forceinline__ double dspow(double x, double k) { return k * cos(x) * pow(fabs(sin(x)), k - 1); }

// rotation_matrix<3>(q), q = (w, x, y, z) (quaternion.hpp:87-124)
__device__ __forceinline__ void rot(const double* q, double* R) {
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    R[0] = 1 - 2 * z * z - 2 * w * w;
    R[1] = 2 * y * z - 2 * x * w;
    R[2] = 2 * y * w + 2 * x * z;
    R[3] = 2 * y * z + 2 * x * w;
    R[4] = 1 - 2 * y * y - 2 * w * w;
    R[5] = 2 * z * w - 2 * x * y;
    R[6] = 2 * y * w - 2 * x * z;
    R[7] = 2 * z * w + 2 * x * y;
    R[8] = 1 - 2 * y * y - 2 * z * z;
}

__device__ __forceinline__ Body load(const Bodies& B, int b) {
    Body s;
    for (int k = 0; k < 3; ++k) {
        s.c[k] = B.pos[3 * (long long)b + k];
        s.r[k] = B.axes[3 * (long long)b + k];
    }
    s.e = B.sq[2 * (long long)b];
    s.n = B.sq[2 * (long long)b + 1];
    rot(B.q + 4 * (long long)b, s.R);
    return s;
}

// A sphere of radius r is the superellipsoid with semi-axes (r, r, r) and squareness (1, 1):
// its parametrisation is then exactly sphere::point (sphere.hpp:195-211), since
// sign(t)|t|^1 = t.  load_any reads either shape as a Body (shape code 0 = sphere).
__device__ __forceinline__ Body sphere_as_body(const Bodies& B, int b) {
    Body s;
    for (int k = 0; k < 3; ++k) {
        s.c[k] = B.pos[3 * (long long)b + k];
        s.r[k] = B.radius[b];
    }
    s.e = s.n = 1.0;
    rot(B.q + 4 * (long long)b, s.R);
    return s;
}
__device__ __forceinline__ Body load_any(const Bodies& B, int b) {
    return B.shape[b] == 0 ? sphere_as_body(B, b) : load(B, b);
}

__device__ __forceinline__ void mv(const double* R, const double* x, double* y) {
    y[0] = R[0] * x[0] + R[1] * x[1] + R[2] * x[2];
    y[1] = R[3] * x[0] + R[4] * x[1] + R[5] * x[2];
    y[2] = R[6] * x[0] + R[7] * x[1] + R[8] * x[2];
}
__device__ __forceinline__ void cross(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ double norm3(const double* a) { return sqrt(dot3(a, a)); }

// world point and unit world normal at (a, b)
__device__ __forceinline__ void point(const Body& s, double a, double b, double* w) {
    const double ca = cpow(a, s.n);
    const double p[3] = {s.r[0] * ca * cpow(b, s.e), s.r[1] * ca * spow(b, s.e), s.r[2] * spow(a, s.n)};
    mv(s.R, p, w);
    for (int k = 0; k < 3; ++k) w[k] += s.c[k];
}
__device__ __forceinline__ void normal(const Body& s, double a, double b, double* w) {
    const double ca = cpow(a, 2 - s.n);
    const double N[3] = {s.r[1] * s.r[2] * ca * cpow(b, 2 - s.e), s.r[0] * s.r[2] * ca * spow(b, 2 - s.e),
                         s.r[0] * s.r[1] * spow(a, 2 - s.n)};
    mv(s.R, N, w);
    const double l = norm3(w);
    for (int k = 0; k < 3; ++k) w[k] /= l;
}

// body-frame point, unnormalised normal and their angle derivatives
struct Local {
    double p[3], pa[3], pb[3], N[3], Na[3], Nb[3];
};
// sign(t)|t|^k for t = cos or sin (given) and the derivative factors k |t|^(k-1)
struct Pw {
    double v, d;  // sign(t)|t|^k, k |t|^(k-1)
};
__device__ __forceinline__ Pw pw(double t, double k, bool deriv) {
    const double at = fabs(t);
    Pw r;
    r.v = sgn(t) * pow(at, k);
    r.d = deriv ? k * pow(at, k - 1) : 0.0;
    return r;
}
// The eight signed powers of one body at angles (a, b), in the order C(a), S(a), C(b), S(b)
// with exponents n, n, e, e, then the same with 2 - n, 2 - e: power w is the one of
// sin/cos selected by w & 3 (0 cos a, 1 sin a, 2 cos b, 3 sin b) with exponent pw_exp(s, w).
__device__ __forceinline__ double pw_exp(const Body& s, int w) {
    const double n2 = 2 - s.n, e2 = 2 - s.e;
    return (w & 2) ? ((w & 4) ? e2 : s.e) : ((w & 4) ? n2 : s.n);
}
__device__ __forceinline__ double pw_arg(int w, double sa, double ca, double sb, double cb) {
    return (w & 3) == 0 ? ca : ((w & 3) == 1 ? sa : ((w & 3) == 2 ? cb : sb));
}
// point, unnormalised normal and (deriv) their angle derivatives from the eight powers
__device__ __forceinline__ void assemble_local(const Body& s, double sa, double ca, double sb, double cb, const Pw* P,
                                               Local& L, bool deriv) {
    const double rx = s.r[0], ry = s.r[1], rz = s.r[2];
    const Pw &Ca = P[0], &Sa = P[1], &Cb = P[2], &Sb = P[3], &Ca2 = P[4], &Sa2 = P[5], &Cb2 = P[6], &Sb2 = P[7];
    L.p[0] = rx * Ca.v * Cb.v;
    L.p[1] = ry * Ca.v * Sb.v;
    L.p[2] = rz * Sa.v;
    L.N[0] = ry * rz * Ca2.v * Cb2.v;
    L.N[1] = rx * rz * Ca2.v * Sb2.v;
    L.N[2] = rx * ry * Sa2.v;
    if (!deriv) return;
    // d/dx sign(cos x)|cos x|^k = -k sin x |cos x|^(k-1);  d/dx sign(sin x)|sin x|^k = k cos x |sin x|^(k-1)
    const double dCa = -sa * Ca.d, dSa = ca * Sa.d, dCb = -sb * Cb.d, dSb = cb * Sb.d;
    const double dCa2 = -sa * Ca2.d, dSa2 = ca * Sa2.d, dCb2 = -sb * Cb2.d, dSb2 = cb * Sb2.d;
    L.pa[0] = rx * dCa * Cb.v;
    L.pa[1] = ry * dCa * Sb.v;
    L.pa[2] = rz * dSa;
    L.pb[0] = rx * Ca.v * dCb;
    L.pb[1] = ry * Ca.v * dSb;
    L.pb[2] = 0.0;
    L.Na[0] = ry * rz * dCa2 * Cb2.v;
    L.Na[1] = rx * rz * dCa2 * Sb2.v;
    L.Na[2] = rx * ry * dSa2;
    L.Nb[0] = ry * rz * Ca2.v * dCb2;
    L.Nb[1] = rx * rz * Ca2.v * dSb2;
    L.Nb[2] = 0.0;
}
// deriv = false: point and normal only (the residual); true: also their angle derivatives
__device__ __forceinline__ void local(const Body& s, double a, double b, Local& L, bool deriv = true) {
    double sa, ca, sb, cb;
    sincos(a, &sa, &ca);
    sincos(b, &sb, &cb);
    Pw P[8];
#pragma unroll
    for (int w = 0; w < 8; ++w) P[w] = pw(pw_arg(w, sa, ca, sb, cb), pw_exp(s, w), deriv);
    assemble_local(s, sa, ca, sb, cb, P, L, deriv);
}

// ---- 2D superellipsoids (superellipsoid.hpp:282-289, 303-312): p(b) = (rx C(b,e), ry S(b,e)),
// N(b) = (ry C(b,2-e), rx S(b,2-e)); R is the upper-left 2x2 block of R(q) (row-major).
struct Body2 {
    double c[2];
    double R[4];
    double r[2];
    double e;
};
__device__ __forceinline__ Body2 load2(const Bodies& B, int b) {
    double R3[9];
    rot(B.q + 4 * (long long)b, R3);
    Body2 s;
    s.c[0] = B.pos[3 * (long long)b];
    s.c[1] = B.pos[3 * (long long)b + 1];
    s.R[0] = R3[0];
    s.R[1] = R3[1];
    s.R[2] = R3[3];
    s.R[3] = R3[4];
    s.r[0] = B.axes[3 * (long long)b];
    s.r[1] = B.axes[3 * (long long)b + 1];
    s.e = B.sq[2 * (long long)b];
    return s;
}
__device__ __forceinline__ Body2 load_any2(const Bodies& B, int b) {
    Body2 s = load2(B, b);
    if (B.shape[b] == 0) {  // sphere: semi-axes (r, r), squareness 1
        s.r[0] = s.r[1] = B.radius[b];
        s.e = 1.0;
    }
    return s;
}
__device__ __forceinline__ void mv2(const double* R, const double* x, double* y) {
    y[0] = R[0] * x[0] + R[1] * x[1];
    y[1] = R[2] * x[0] + R[3] * x[1];
}
struct Local2 {
    double p[2], N[2], pb[2], Nb[2];
};
__device__ __forceinline__ void local2(const Body2& s, double b, Local2& L, bool deriv = true) {
    double sb, cb;
    sincos(b, &sb, &cb);
    const double k = 2 - s.e;
    const Pw C = pw(cb, s.e, deriv), S = pw(sb, s.e, deriv), C2 = pw(cb, k, deriv), S2 = pw(sb, k, deriv);
    L.p[0] = s.r[0] * C.v;
    L.p[1] = s.r[1] * S.v;
    L.N[0] = s.r[1] * C2.v;
    L.N[1] = s.r[0] * S2.v;
    if (!deriv) return;
    L.pb[0] = s.r[0] * (-sb * C.d);
    L.pb[1] = s.r[1] * (cb * S.d);
    L.Nb[0] = s.r[1] * (-sb * C2.d);
    L.Nb[1] = s.r[0] * (cb * S2.d);
}
__device__ __forceinline__ void point2(const Body2& s, double b, double* w) {
    Local2 L;
    local2(s, b, L, false);
    mv2(s.R, L.p, w);
    w[0] += s.c[0];
    w[1] += s.c[1];
}
__device__ __forceinline__ void normal2(const Body2& s, double b, double* w) {
    Local2 L;
    local2(s, b, L, false);
    mv2(s.R, L.N, w);
    const double l = sqrt(w[0] * w[0] + w[1] * w[1]);
    w[0] /= l;
    w[1] /= l;
}

// Closest points of a superellipsoid and a plane (the solution of the system of
// closest_points.hpp:1479-1759 in closed form): the body point whose outward normal is
// opposite to the plane normal oriented toward the body, and its projection on the plane.
// pi on the body, pj on the plane, nij = the oriented plane normal, dij = (pi - pj).nij.
// Angles (a, b) of the body point whose outward normal points along the body-frame
// direction m: b = atan2(sign(my)|ry my|^(1/(2-e)), sign(mx)|rx mx|^(1/(2-e))),
// |tan a|^(2-n) = |mz| |(ry rz C(b,2-e), rx rz S(b,2-e))| / (rx ry |(mx, my)|), sign(a) = sign(mz).
__device__ __forceinline__ void support_angles(const Body& s, const double* m, double& a, double& b) {
    const double pi_ = 3.14159265358979323846;
    const double rx = s.r[0], ry = s.r[1], rz = s.r[2];
    const double mxy = sqrt(m[0] * m[0] + m[1] * m[1]);
    if (mxy == 0) {
        b = 0;
        a = m[2] >= 0 ? pi_ / 2 : -pi_ / 2;
    } else {
        const double ke = 1.0 / (2 - s.e), kn = 1.0 / (2 - s.n);
        b = atan2(sgn(m[1]) * pow(fabs(ry * m[1]), ke), sgn(m[0]) * pow(fabs(rx * m[0]), ke));
        const double cb = cpow(b, 2 - s.e), sb = spow(b, 2 - s.e);
        const double h = sqrt((ry * rz * cb) * (ry * rz * cb) + (rx * rz * sb) * (rx * rz * sb));
        const double t = fabs(m[2]) * h / (rx * ry * mxy);
        a = sgn(m[2]) * atan(pow(t, kn));
    }
}

__device__ __forceinline__ void body_plane(const Body& s, const double* pc, const double* pq, double* pi, double* pj,
                                           double* nij, double& dij) {
    double P[9];
    rot(pq, P);
    const double np[3] = {P[0], P[3], P[6]};
    const double rel[3] = {s.c[0] - pc[0], s.c[1] - pc[1], s.c[2] - pc[2]};
    const double sg = dot3(rel, np) < 0 ? -1.0 : 1.0;
    // body-frame direction of the wanted outward normal: -sg np (R^T np)
    const double m[3] = {-sg * (s.R[0] * np[0] + s.R[3] * np[1] + s.R[6] * np[2]),
                         -sg * (s.R[1] * np[0] + s.R[4] * np[1] + s.R[7] * np[2]),
                         -sg * (s.R[2] * np[0] + s.R[5] * np[1] + s.R[8] * np[2])};
    double a, b;
    support_angles(s, m, a, b);
    point(s, a, b, pi);
    const double d[3] = {pi[0] - pc[0], pi[1] - pc[1], pi[2] - pc[2]};
    const double h = dot3(d, np);
    for (int k = 0; k < 3; ++k) {
        pj[k] = pi[k] - h * np[k];
        nij[k] = sg * np[k];
    }
    const double df[3] = {pi[0] - pj[0], pi[1] - pj[1], pi[2] - pj[2]};
    dij = dot3(df, nij);
}

// closest_points(superellipsoid<2>, plane<2>) (closest_points.hpp:1783-1949) in closed form, as
// body_plane in 3D: the body point whose outward normal is opposite to the plane normal
// (column 0 of the plane's rotation, plane.hpp:143-147) oriented toward the body, and its
// projection on the plane; pi on the body, pj on the plane, nij = the oriented normal.
__device__ __forceinline__ double support_angle2(const Body2& s, double m0, double m1);
__device__ __forceinline__ void body_plane2(const Body2& s, const double* pc, const double* pq, double* pi, double* pj,
                                            double* nij, double& dij) {
    double P[9];
    rot(pq, P);
    const double np[2] = {P[0], P[3]};
    const double rel[2] = {s.c[0] - pc[0], s.c[1] - pc[1]};
    const double sg = rel[0] * np[0] + rel[1] * np[1] < 0 ? -1.0 : 1.0;
    // body-frame direction of the wanted outward normal: -sg R^T np
    const double m0 = -sg * (s.R[0] * np[0] + s.R[2] * np[1]), m1 = -sg * (s.R[1] * np[0] + s.R[3] * np[1]);
    point2(s, support_angle2(s, m0, m1), pi);
    const double h = (pi[0] - pc[0]) * np[0] + (pi[1] - pc[1]) * np[1];
    pj[0] = pi[0] - h * np[0];
    pj[1] = pi[1] - h * np[1];
    nij[0] = sg * np[0];
    nij[1] = sg * np[1];
    pi[2] = pj[2] = nij[2] = 0.0;
    dij = (pi[0] - pj[0]) * nij[0] + (pi[1] - pj[1]) * nij[1];
}

// ---- separation bound.  For convex bodies (squareness in (0, 2)) the distance is at least
// the gap along any unit direction u: (support point of body 2 in -u - support point of
// body 1 in u).u; u is the line of centres.  -inf for coincident centres.
__device__ __forceinline__ double support_gap3(const Body& s1, const Body& s2) {
    const double d[3] = {s2.c[0] - s1.c[0], s2.c[1] - s1.c[1], s2.c[2] - s1.c[2]};
    const double l = norm3(d);
    if (!(l > 0)) return -INFINITY;
    const double u[3] = {d[0] / l, d[1] / l, d[2] / l};
    double m1[3], m2[3];
    for (int k = 0; k < 3; ++k) {
        m1[k] = s1.R[k] * u[0] + s1.R[3 + k] * u[1] + s1.R[6 + k] * u[2];
        m2[k] = -(s2.R[k] * u[0] + s2.R[3 + k] * u[1] + s2.R[6 + k] * u[2]);
    }
    double a, b, p1[3], p2[3];
    support_angles(s1, m1, a, b);
    point(s1, a, b, p1);
    support_angles(s2, m2, a, b);
    point(s2, a, b, p2);
    return (p2[0] - p1[0]) * u[0] + (p2[1] - p1[1]) * u[1] + (p2[2] - p1[2]) * u[2];
}
__device__ __forceinline__ double support_angle2(const Body2& s, double m0, double m1) {
    const double ke = 1.0 / (2 - s.e);
    return atan2(sgn(m1) * pow(fabs(s.r[1] * m1), ke), sgn(m0) * pow(fabs(s.r[0] * m0), ke));
}
__device__ __forceinline__ double support_gap2(const Body2& s1, const Body2& s2) {
    const double d[2] = {s2.c[0] - s1.c[0], s2.c[1] - s1.c[1]};
    const double l = sqrt(d[0] * d[0] + d[1] * d[1]);
    if (!(l > 0)) return -INFINITY;
    const double u[2] = {d[0] / l, d[1] / l};
    const double m10 = s1.R[0] * u[0] + s1.R[2] * u[1], m11 = s1.R[1] * u[0] + s1.R[3] * u[1];
    const double m20 = -(s2.R[0] * u[0] + s2.R[2] * u[1]), m21 = -(s2.R[1] * u[0] + s2.R[3] * u[1]);
    double p1[2], p2[2];
    point2(s1, support_angle2(s1, m10, m11), p1);
    point2(s2, support_angle2(s2, m20, m21), p2);
    return (p2[0] - p1[0]) * u[0] + (p2[1] - p1[1]) * u[1];
}

}  // namespace se
}  // namespace scopi_gpu
