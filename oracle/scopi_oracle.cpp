// scopi_oracle.cpp -- CPU restatement of the SCoPI time step (TEST INFRASTRUCTURE).
//
// This file is the oracle the CUDA path is checked against; the product never
// links it.  Every function names the reference lines (hpc-maths/scopi v0.1.0)
// whose arithmetic it follows.  Floating-point expressions keep the reference's
// evaluation order (built with -ffp-contract=off) so that the contact set, which
// is decided by the strict test dij < dmax, can be compared bit for bit.
// BLAS nrm2/dot calls of the reference become plain in-order sums here (the
// reference does not pin a BLAS; see tests for the ulp-band handling).

#include "scopi_oracle.h"
#include "se_geometry.hpp"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using V3 = std::array<double, 3>;
using Q4 = std::array<double, 4>;
using M3 = std::array<std::array<double, 3>, 3>;

struct Contact {
    int64_t i, j;
    double dij;
    V3 nij, pi, pj;
    double gamma;
};

double sum_sq(const double* x, int n) {
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += x[k] * x[k];
    return s;
}
double norm_n(const double* x, int n) { return std::sqrt(sum_sq(x, n)); }
double dot_n(const double* a, const double* b, int n) {
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += a[k] * b[k];
    return s;
}
double xsign(double x) { return (x > 0.0) ? 1.0 : ((x < 0.0) ? -1.0 : 0.0); }

// rotation_matrix<3>: include/scopi/quaternion.hpp:87-124 (q = (x, y, z, w) in its naming)
M3 rotation3(const Q4& q) {
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    M3 r;
    r[0] = {1 - 2 * z * z - 2 * w * w, 2 * y * z - 2 * x * w, 2 * y * w + 2 * x * z};
    r[1] = {2 * y * z + 2 * x * w, 1 - 2 * y * y - 2 * w * w, 2 * z * w - 2 * x * y};
    r[2] = {2 * y * w - 2 * x * z, 2 * z * w + 2 * x * y, 1 - 2 * y * y - 2 * z * z};
    return r;
}

// plane::normal / segment::normal = column 0 of rotation_matrix<dim>(q)
// include/scopi/objects/types/plane.hpp:143-147, quaternion.hpp:66-85
V3 body_normal(const Q4& q, int dim) {
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    if (dim == 2) return {1 - 2 * w * w, 2 * x * w, 0.0};
    return {1 - 2 * z * z - 2 * w * w, 2 * y * z + 2 * x * w, 2 * y * w - 2 * x * z};
}

// mult_quaternion, src/quaternion.cpp:92-120
Q4 qmul(const Q4& a, const Q4& b) {
    Q4 r;
    r[0] = a[0] * b[0];
    for (int d = 0; d < 3; ++d) {
        r[0] -= a[d + 1] * b[d + 1];
        r[d + 1] = a[0] * b[d + 1] + b[0] * a[d + 1];
    }
    r[1] += (a[2] * b[3] - a[3] * b[2]);
    r[2] += (a[3] * b[1] - a[1] * b[3]);
    r[3] += (a[1] * b[2] - a[2] * b[1]);
    return r;
}
// normalize, src/quaternion.cpp:6-10
void qnormalize(Q4& q) {
    const double n = norm_n(q.data(), 4);
    for (auto& c : q) c /= n;
}
// q <- normalize(q o exp(w dt / 2)), solver.hpp:335-351 and 449-479
void rotate_body(Q4& q, const V3& w, double normw, double dt) {
    if (normw == 0) normw = 1;
    Q4 e;
    e[0] = std::cos(0.5 * normw * dt);
    const double s = std::sin(0.5 * normw * dt) / normw;
    for (int d = 0; d < 3; ++d) e[d + 1] = s * w[d];
    q = qmul(q, e);
    qnormalize(q);
}

// detail::cross<dim>, include/scopi/matrix/velocities.hpp:26-44
V3 cross_dim(int dim, const V3& x, const V3& y) {
    if (dim == 2) return {x[1] * y[2], -x[0] * y[2], x[0] * y[1] - x[1] * y[0]};
    return {x[1] * y[2] - x[2] * y[1], x[2] * y[0] - x[0] * y[2], x[0] * y[1] - x[1] * y[0]};
}
V3 mat_vec(const M3& a, const V3& x) {
    return {a[0][0] * x[0] + a[0][1] * x[1] + a[0][2] * x[2], a[1][0] * x[0] + a[1][1] * x[1] + a[1][2] * x[2],
            a[2][0] * x[0] + a[2][1] * x[1] + a[2][2] * x[2]};
}
V3 matT_vec(const M3& a, const V3& x) {
    return {a[0][0] * x[0] + a[1][0] * x[1] + a[2][0] * x[2], a[0][1] * x[0] + a[1][1] * x[1] + a[2][1] * x[2],
            a[0][2] * x[0] + a[1][2] * x[1] + a[2][2] * x[2]};
}

}  // namespace

struct orc_solver {
    orc_params p;
    int dim = 3;
    int64_t n = 0, nin = 0;
    std::vector<int32_t> shape;
    std::vector<V3> pos, v, omega, vd, omega_d, f, jm;
    std::vector<Q4> q;
    std::vector<double> m, radius, length;
    std::vector<std::array<double, 5>> se_par;  // superellipsoids: semi-axes, e, n
    std::vector<int32_t> worm;                  // worm index per body, -1 if none
    bool has_worms = false;
    bool periodic_error = false;                // an obstacle would be copied across a periodic bound
    bool periodic_any() const {
        for (int d = 0; d < dim; ++d)
            if (p.periodic[d]) return true;
        return false;
    }
    std::vector<Contact> contacts, old_contacts;
    std::vector<double> lambda;
    orc_stats stats{};
    double dt = 0;
    // FrictionFixedPoint: p.problem holds ORC_FRICTION, this flag the outer loop; sij per contact
    bool fixed_point = false;
    std::vector<double> sij;

    int64_t na() const { return n - nin; }

    // ---------------------------------------------------------------- geometry
    // closest_points(sphere, sphere), closest_points.hpp:36-50
    Contact sphere_sphere(int64_t a, int64_t b) const {
        Contact c{};
        double d[3] = {0, 0, 0};
        for (int k = 0; k < dim; ++k) d[k] = pos[b][k] - pos[a][k];
        const double nrm = norm_n(d, dim);
        double u[3] = {0, 0, 0};
        for (int k = 0; k < dim; ++k) u[k] = d[k] / nrm;
        for (int k = 0; k < dim; ++k) {
            c.pi[k] = pos[a][k] + radius[a] * u[k];
            c.pj[k] = pos[b][k] - radius[b] * u[k];
        }
        double t[3] = {0, 0, 0};
        for (int k = 0; k < dim; ++k) t[k] = c.pj[k] - pos[b][k];
        const double nt = norm_n(t, dim);
        for (int k = 0; k < dim; ++k) c.nij[k] = t[k] / nt;
        double diff[3] = {0, 0, 0};
        for (int k = 0; k < dim; ++k) diff[k] = c.pi[k] - c.pj[k];
        c.dij = dot_n(diff, c.nij.data(), dim);
        return c;
    }
    // closest_points(sphere, plane), closest_points.hpp:768-788
    Contact sphere_plane(int64_t s, int64_t pl) const {
        Contact c{};
        const V3 nrm = body_normal(q[pl], dim);
        double d[3] = {0, 0, 0};
        for (int k = 0; k < dim; ++k) d[k] = pos[s][k] - pos[pl][k];
        const double p2s = dot_n(d, nrm.data(), dim);
        const double sg = xsign(p2s);
        for (int k = 0; k < dim; ++k) {
            c.pi[k] = pos[s][k] - sg * radius[s] * nrm[k];
            c.pj[k] = pos[s][k] - p2s * nrm[k];
            c.nij[k] = sg * nrm[k];
        }
        double diff[3] = {0, 0, 0};
        for (int k = 0; k < dim; ++k) diff[k] = c.pi[k] - c.pj[k];
        c.dij = dot_n(diff, c.nij.data(), dim);
        return c;
    }
    // closest_points(sphere, segment), closest_points.hpp:824-870; segment.hpp:155-181
    Contact sphere_segment(int64_t s, int64_t sg_) const {
        Contact c{};
        const Q4& qq = q[sg_];
        const double x = qq[0], w = qq[3];
        const double r01 = -2 * x * w, r11 = 1 - 2 * w * w;  // column 1 of rotation_matrix<2>
        const double h = 0.5 * length[sg_];
        double e0[2], e1[2];
        // R.(0, -L/2) + pos and R.(0, L/2) + pos; the zero first coordinate adds an exact 0
        e0[0] = (0.0 * (1 - 2 * w * w) + r01 * (-h)) + pos[sg_][0];
        e0[1] = (0.0 * (2 * x * w) + r11 * (-h)) + pos[sg_][1];
        e1[0] = (0.0 * (1 - 2 * w * w) + r01 * h) + pos[sg_][0];
        e1[1] = (0.0 * (2 * x * w) + r11 * h) + pos[sg_][1];
        const V3 nrm = body_normal(qq, 2);
        const double tg[2] = {-nrm[1], nrm[0]};
        const double* sp = pos[s].data();
        double d0[2] = {sp[0] - e0[0], sp[1] - e0[1]};
        double d1[2] = {sp[0] - e1[0], sp[1] - e1[1]};
        auto endpoint = [&](const double* e, const double* de) {
            const double nn = norm_n(de, 2);
            for (int k = 0; k < 2; ++k) {
                c.nij[k] = de[k] / nn;
                c.pi[k] = sp[k] - c.nij[k] * radius[s];
                c.pj[k] = e[k];
            }
        };
        if (dot_n(d0, tg, 2) < 0) {
            endpoint(e0, d0);
        } else if (dot_n(d1, tg, 2) > 0) {
            endpoint(e1, d1);
        } else {
            double d[2] = {sp[0] - pos[sg_][0], sp[1] - pos[sg_][1]};
            const double s2s = dot_n(d, nrm.data(), 2);
            const double sgn = xsign(s2s);
            for (int k = 0; k < 2; ++k) {
                c.pi[k] = sp[k] - sgn * radius[s] * nrm[k];
                c.pj[k] = sp[k] - s2s * nrm[k];
                c.nij[k] = sgn * nrm[k];
            }
        }
        double diff[2] = {c.pi[0] - c.pj[0], c.pi[1] - c.pj[1]};
        c.dij = dot_n(diff, c.nij.data(), 2);
        return c;
    }
    // closest_points_dispatcher for the pairs the hot path meets (obstacle i < active j)
    bool exact(int64_t a, int64_t b, Contact& c) const {
        const int sa = shape[a], sb = shape[b];
        if (sa == ORC_SPHERE && sb == ORC_SPHERE) {
            c = sphere_sphere(a, b);
        } else if (sa == ORC_PLANE && sb == ORC_SPHERE) {  // closest_points.hpp:802-809
            c = sphere_plane(b, a);
            for (auto& x : c.nij) x *= -1.;
            std::swap(c.pi, c.pj);
        } else if (sa == ORC_SPHERE && sb == ORC_PLANE) {
            c = sphere_plane(a, b);
        } else if (sa == ORC_SEGMENT && sb == ORC_SPHERE) {  // closest_points.hpp:874-881
            c = sphere_segment(b, a);
            for (auto& x : c.nij) x *= -1.;
            std::swap(c.pi, c.pj);
        } else if (sa == ORC_SPHERE && sb == ORC_SEGMENT) {
            c = sphere_segment(a, b);
        } else if (dim == 3 && sa == ORC_SUPERELLIPSOID && sb == ORC_SUPERELLIPSOID) {
            // bounding spheres (radius = |semi-axes|) farther apart than dmax: no contact, no
            // solve.  The reference solves every kd-tree candidate; on well-separated pairs
            // its solve can stop at a spurious root with dij < dmax (about 0.1 % of the
            // candidates of the superellipsoid pile), which is not reproduced.
            double s2 = 0.0;
            for (int k = 0; k < 3; ++k) s2 += (pos[a][k] - pos[b][k]) * (pos[a][k] - pos[b][k]);
            const double lim = radius[a] + radius[b] + p.dmax;
            if (!(lim > 0.0) || s2 > lim * lim * (1.0 + 1e-9)) return false;
            // nor when their gap along the line of centres exceeds dmax (convex bodies)
            if (orc_se::support_gap(se_of(a), se_of(b), 3) > p.dmax + 1e-9 * lim) return false;
            c = from_pair(orc_se::se_se(se_of(a), se_of(b)));
        } else if (dim == 2 && sa == ORC_SUPERELLIPSOID && sb == ORC_SUPERELLIPSOID) {
            // same bounding-sphere test as in 3D (radius = |semi-axes|)
            double s2 = 0.0;
            for (int k = 0; k < 2; ++k) s2 += (pos[a][k] - pos[b][k]) * (pos[a][k] - pos[b][k]);
            const double lim = radius[a] + radius[b] + p.dmax;
            if (!(lim > 0.0) || s2 > lim * lim * (1.0 + 1e-9)) return false;
            if (orc_se::support_gap(se_of(a), se_of(b), 2) > p.dmax + 1e-9 * lim) return false;
            c = from_pair(orc_se::se2_se2(se_of(a), se_of(b)));
        } else if ((sa == ORC_SPHERE && sb == ORC_SUPERELLIPSOID) || (sa == ORC_SUPERELLIPSOID && sb == ORC_SPHERE)) {
            // closest_points(sphere, superellipsoid) and its mirror (closest_points.hpp:944-1302,
            // 1316-1463): the same bounding-sphere and line-of-centres bounds as the pairs of
            // two superellipsoids, then the reference's Newton solve, labelled by body
            const int64_t e = sa == ORC_SUPERELLIPSOID ? a : b, sp = sa == ORC_SPHERE ? a : b;
            double s2 = 0.0;
            for (int k = 0; k < dim; ++k) s2 += (pos[a][k] - pos[b][k]) * (pos[a][k] - pos[b][k]);
            const double lim = radius[a] + radius[b] + p.dmax;
            if (!(lim > 0.0) || s2 > lim * lim * (1.0 + 1e-9)) return false;
            const orc_se::SE E = se_of(e), S = sphere_of(sp);
            if (orc_se::support_gap(E, S, dim) > p.dmax + 1e-9 * lim) return false;
            c = from_pair(e == a ? orc_se::sphere_se_pair(E, S, true, dim) : orc_se::sphere_se_pair(S, E, false, dim));
        } else if (dim == 2 && sa == ORC_SUPERELLIPSOID && sb == ORC_PLANE) {
            c = from_pair(orc_se::se2_plane(se_of(a), plane_of(b)));
        } else if (dim == 2 && sa == ORC_PLANE && sb == ORC_SUPERELLIPSOID) {  // closest_points.hpp:1951-1958
            c = from_pair(orc_se::se2_plane(se_of(b), plane_of(a)));
            for (auto& x : c.nij) x *= -1.;
            std::swap(c.pi, c.pj);
        } else if (dim == 3 && sa == ORC_SUPERELLIPSOID && sb == ORC_PLANE) {
            c = from_pair(orc_se::se_plane(se_of(a), plane_of(b)));
        } else if (dim == 3 && sa == ORC_PLANE && sb == ORC_SUPERELLIPSOID) {  // closest_points.hpp:1761-1768
            c = from_pair(orc_se::se_plane(se_of(b), plane_of(a)));
            for (auto& x : c.nij) x *= -1.;
            std::swap(c.pi, c.pj);
        } else {
            return false;  // pairs the reference leaves unimplemented
        }
        c.i = a;
        c.j = b;
        c.gamma = p.gamma;
        return c.dij < p.dmax;  // base.hpp:118
    }

    // --------------------------------------------------------------- contacts
    // contact_brute_force::run_impl / contact_kdtree::run_impl + sort_contacts.
    // The kd-tree's radius search is a candidate filter (squared centre distance
    // < kd_tree_radius, nanoflann L2 metric); any enumeration that visits a
    // superset of the pairs with dij < dmax gives the same set, so large inputs
    // are enumerated with a uniform grid instead of O(N^2) loops.
    void detect() {
        std::vector<Contact> out;
        // add_objects_from_periodicity (utils.hpp:229-257): per periodic axis d, a copy shifted
        // by +L_d of every original body within dmax of the lower bound, appended after the
        // bodies for the search (contact_base::run, base.hpp:71-77)
        const int64_t n0 = n;
        std::vector<std::pair<int64_t, int>> ghosts;
        if (periodic_any()) {
            for (int d = 0; d < dim; ++d) {
                if (!p.periodic[d]) continue;
                for (int64_t b = 0; b < n0; ++b)
                    if (pos[b][d] - p.dmax < p.box_lower[d]) {
                        if (b < nin) {
                            periodic_error = true;
                            continue;
                        }
                        ghosts.push_back({b, d});
                    }
            }
            for (const auto& gd : ghosts) {
                const int64_t b = gd.first;
                V3 x = pos[b];
                x[gd.second] += p.box_upper[gd.second] - p.box_lower[gd.second];
                pos.push_back(x);
                q.push_back(q[b]);
                shape.push_back(shape[b]);
                radius.push_back(radius[b]);
                length.push_back(length[b]);
                se_par.push_back(se_par[b]);
                worm.push_back(-1);
            }
            n = n0 + (int64_t)ghosts.size();
        }
        const int64_t nA = na();
        const bool use_kd = (p.contact_method == ORC_KDTREE);
        auto kd_ok = [&](int64_t a, int64_t b) {
            if (!use_kd) return true;
            double s = 0.0;
            for (int k = 0; k < dim; ++k) {
                const double d = pos[a][k] - pos[b][k];
                s += d * d;
            }
            return s < p.kd_tree_radius;
        };
        std::vector<std::vector<Contact>> per_thread(1);
        if (nA > 1 && nA <= 3000) {
            // literal i<j double loop
            for (int64_t a = nin; a < n - 1; ++a)
                for (int64_t b = a + 1; b < n; ++b) {
                    Contact c;
                    if (kd_ok(a, b) && exact(a, b, c)) out.push_back(c);
                }
        } else if (nA > 1) {
            double rmax = 0;
            double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
            for (int64_t a = nin; a < n; ++a) {
                rmax = std::max(rmax, radius[a]);
                for (int k = 0; k < dim; ++k) {
                    lo[k] = std::min(lo[k], pos[a][k]);
                    hi[k] = std::max(hi[k], pos[a][k]);
                }
            }
            double h = (2 * rmax + p.dmax) * (1 + 1e-6) + 1e-12;
            int64_t nc[3] = {1, 1, 1};
            for (;;) {
                int64_t tot = 1;
                for (int k = 0; k < dim; ++k) {
                    nc[k] = (int64_t)std::floor((hi[k] - lo[k]) / h) + 1;
                    tot *= nc[k];
                }
                if (tot <= (int64_t)1 << 26) break;
                h *= 1.5;
            }
            auto cell_of = [&](int64_t a) {
                int64_t id = 0;
                for (int k = dim - 1; k >= 0; --k) {
                    int64_t c = (int64_t)std::floor((pos[a][k] - lo[k]) / h);
                    c = std::min(std::max<int64_t>(c, 0), nc[k] - 1);
                    id = id * nc[k] + c;
                }
                return id;
            };
            int64_t ncell = 1;
            for (int k = 0; k < dim; ++k) ncell *= nc[k];
            std::vector<int64_t> start(ncell + 1, 0), cellid(nA), order(nA);
            for (int64_t a = 0; a < nA; ++a) {
                cellid[a] = cell_of(nin + a);
                start[cellid[a] + 1]++;
            }
            for (int64_t c = 0; c < ncell; ++c) start[c + 1] += start[c];
            {
                std::vector<int64_t> fill(start.begin(), start.end() - 1);
                for (int64_t a = 0; a < nA; ++a) order[fill[cellid[a]]++] = nin + a;
            }
            int nth = 1;
#ifdef _OPENMP
            nth = omp_get_max_threads();
#endif
            per_thread.assign(nth, {});
#pragma omp parallel for schedule(dynamic, 256)
            for (int64_t a = nin; a < n - 1; ++a) {
                int tid = 0;
#ifdef _OPENMP
                tid = omp_get_thread_num();
#endif
                int64_t ci[3] = {0, 0, 0};
                for (int k = 0; k < dim; ++k) {
                    int64_t c = (int64_t)std::floor((pos[a][k] - lo[k]) / h);
                    ci[k] = std::min(std::max<int64_t>(c, 0), nc[k] - 1);
                }
                const int zr = (dim == 3) ? 1 : 0;
                for (int dz = -zr; dz <= zr; ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx) {
                            int64_t cc[3] = {ci[0] + dx, ci[1] + dy, ci[2] + dz};
                            bool ok = true;
                            for (int k = 0; k < dim; ++k)
                                if (cc[k] < 0 || cc[k] >= nc[k]) ok = false;
                            if (!ok) continue;
                            int64_t id = 0;
                            for (int k = dim - 1; k >= 0; --k) id = id * nc[k] + cc[k];
                            for (int64_t t = start[id]; t < start[id + 1]; ++t) {
                                const int64_t b = order[t];
                                if (b <= a) continue;
                                Contact c;
                                if (kd_ok(a, b) && exact(a, b, c)) per_thread[tid].push_back(c);
                            }
                        }
            }
        }
        for (auto& v_ : per_thread) out.insert(out.end(), v_.begin(), v_.end());
        // obstacles: every (obstacle, active) pair, contact_kdtree.hpp:249-256
        for (int64_t a = 0; a < nin; ++a)
            for (int64_t b = nin; b < n; ++b) {
                Contact c;
                if (exact(a, b, c)) out.push_back(c);
            }
        std::vector<char> via_copy;  // periodic: the pair was found with a copy
        if (!ghosts.empty()) {
            // compute_exact_distance (base.hpp:118-137): pairs of two copies are dropped; a copy's
            // index becomes its original's and its closest point moves back by L_d on every
            // periodic axis d
            std::vector<Contact> kept;
            kept.reserve(out.size());
            for (auto& c : out) {
                if (c.i >= n0 && c.j >= n0) continue;
                via_copy.push_back(c.i >= n0 || c.j >= n0);
                for (int d = 0; d < dim; ++d) {
                    if (!p.periodic[d]) continue;
                    const double L = p.box_upper[d] - p.box_lower[d];
                    if (c.i >= n0) c.pi[d] -= L;
                    if (c.j >= n0) c.pj[d] -= L;
                }
                if (c.i >= n0) c.i = ghosts[c.i - n0].first;
                if (c.j >= n0) c.j = ghosts[c.j - n0].first;
                kept.push_back(c);
            }
            out.swap(kept);
        }
        if (n != n0) {  // reset_periodic
            pos.resize(n0);
            q.resize(n0);
            shape.resize(n0);
            radius.resize(n0);
            length.resize(n0);
            se_par.resize(n0);
            worm.resize(n0);
            n = n0;
        }
        if (!via_copy.empty()) {
            // a body near the lower bound touching an obstacle is paired with it twice (once as
            // itself, once as its copy); the reference's std::sort leaves the order of such equal
            // (i, j) unspecified: here the pair found without a copy comes first
            std::vector<size_t> order(out.size());
            for (size_t k = 0; k < order.size(); ++k) order[k] = k;
            std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
                const Contact &a = out[x], &b = out[y];
                if (a.i != b.i) return a.i < b.i;
                if (a.j != b.j) return a.j < b.j;
                return via_copy[x] < via_copy[y];
            });
            std::vector<Contact> sorted;
            sorted.reserve(out.size());
            for (size_t k : order) sorted.push_back(out[k]);
            contacts.swap(sorted);
            return;
        }
        std::sort(out.begin(), out.end(), [](const Contact& x, const Contact& y) {
            return x.i < y.i || (x.i == y.i && x.j < y.j);
        });
        contacts.swap(out);
    }

    // compute_contacts (solver.hpp:358-367): after the contact method's sorted list, per worm
    // (objects in order) the contacts of its consecutive spheres with normal and distance
    // negated (add_contact_from_object<worm>, add_contact.hpp:11-28), which keep the gap of
    // each link from opening
    void add_worm_contacts() {
        if (!has_worms) return;
        for (int64_t a = nin; a + 1 < n; ++a) {
            if (worm[a] < 0 || worm[a + 1] != worm[a]) continue;
            Contact c = sphere_sphere(a, a + 1);
            for (auto& x : c.nij) x *= -1.;
            c.dij *= -1.;
            c.i = a;
            c.j = a + 1;
            c.gamma = 0.0;
            contacts.push_back(c);
        }
    }

    // transfer(old, new), solver.hpp:241-258
    void transfer() {
        if (old_contacts.empty()) return;
        std::unordered_map<uint64_t, size_t> idx;
        idx.reserve(old_contacts.size() * 2);
        for (size_t k = 0; k < old_contacts.size(); ++k)
            idx[(uint64_t)old_contacts[k].i * 0x9E3779B97F4A7C15ull ^ (uint64_t)old_contacts[k].j] = k;
        for (auto& c : contacts) {
            auto it = idx.find((uint64_t)c.i * 0x9E3779B97F4A7C15ull ^ (uint64_t)c.j);
            if (it != idx.end() && old_contacts[it->second].i == c.i && old_contacts[it->second].j == c.j)
                c.gamma = old_contacts[it->second].gamma;
        }
    }

    // ------------------------------------------------------------ A, A^T, D
    // AMatrix::mat_mult, velocities.hpp:67-144
    void amat(const std::vector<double>& u, std::vector<double>& out) const {
        const int64_t rot = 3 * na();
        out.assign(3 * contacts.size(), 0.0);
        for (size_t c = 0; c < contacts.size(); ++c) {
            const Contact& ct = contacts[c];
            double* row = &out[3 * c];
            for (int side = 0; side < 2; ++side) {
                const int64_t b = side == 0 ? ct.i : ct.j;
                if (b < nin) continue;
                const int64_t st = (b - nin) * 3;
                V3 vb = {u[st], u[st + 1], u[st + 2]};
                V3 wb = {u[st + rot], u[st + rot + 1], u[st + rot + 2]};
                const V3& pt = side == 0 ? ct.pi : ct.pj;
                V3 r = {0, 0, 0};
                for (int k = 0; k < dim; ++k) r[k] = pt[k] - pos[b][k];
                const V3 cr = cross_dim(dim, r, mat_vec(rotation3(q[b]), wb));
                for (int d = 0; d < 3; ++d) {
                    if (side == 0)
                        row[d] += vb[d] - cr[d];
                    else
                        row[d] -= vb[d] - cr[d];
                }
            }
        }
    }
    // ATMatrix::mat_mult, velocities.hpp:167-254
    void atmat(const std::vector<double>& fv, std::vector<double>& out) const {
        const int64_t rot = 3 * na();
        out.assign(6 * na(), 0.0);
        for (size_t c = 0; c < contacts.size(); ++c) {
            const Contact& ct = contacts[c];
            const V3 fc = {fv[3 * c], fv[3 * c + 1], fv[3 * c + 2]};
            for (int side = 0; side < 2; ++side) {
                const int64_t b = side == 0 ? ct.i : ct.j;
                if (b < nin) continue;
                const int64_t st = (b - nin) * 3;
                const V3& pt = side == 0 ? ct.pi : ct.pj;
                V3 r = {0, 0, 0};
                for (int k = 0; k < dim; ++k) r[k] = pt[k] - pos[b][k];
                const V3 res = matT_vec(rotation3(q[b]), cross_dim(dim, r, fc));
                for (int d = 0; d < 3; ++d) {
                    if (side == 0) {
                        out[st + d] += fc[d];
                        out[st + rot + d] += res[d];
                    } else {
                        out[st + d] -= fc[d];
                        out[st + rot + d] -= res[d];
                    }
                }
            }
        }
    }

    // ------------------------------------------------------- the QP (problem)
    struct Problem {
        const orc_solver* s;
        std::vector<double> invM, C;
        std::vector<double> S;          // FrictionFixedPoint: s_c n_c (empty otherwise)
        std::vector<int64_t> neg_slot;  // Viscous: second multiplier slot or -1
        std::vector<int64_t> row;       // ViscousFriction: first local row of each contact
        std::vector<int> mode;          // ViscousFriction: 1, 2 or 4 multipliers (0, 1, 2)
        int64_t size = 0;
        mutable std::vector<double> w1, w2, w3;

        // M_inverse, minimization_problem.hpp:11-31; CVector :34-70
        explicit Problem(const orc_solver* s_) : s(s_) {
            const int64_t nA = s->na(), off = 3 * nA;
            const int dim = s->dim;
            invM.assign(6 * nA, 0.0);
            std::vector<double> U(6 * nA, 0.0);
            for (int64_t i = 0; i < nA; ++i) {
                const int64_t b = s->nin + i;
                for (int d = 0; d < dim; ++d) invM[3 * i + d] = 1. / s->m[b];
                for (int d = 0; d < dim; ++d) U[3 * i + d] = s->v[b][d];
                if (dim == 2) {
                    invM[off + 3 * i + 2] = 1. / s->jm[b][2];
                    U[off + 3 * i + 2] = s->omega[b][2];
                } else {
                    for (int d = 0; d < 3; ++d) {
                        invM[off + 3 * i + d] = 1. / s->jm[b][d];
                        U[off + 3 * i + d] = s->omega[b][d];
                    }
                }
            }
            const size_t nc = s->contacts.size();
            std::vector<double> AU;
            s->amat(U, AU);
            C.assign(3 * nc, 0.0);
            for (size_t c = 0; c < nc; ++c)
                for (int d = 0; d < 3; ++d) {
                    const double dn = d < dim ? s->contacts[c].dij * s->contacts[c].nij[d] : 0.0;  // DMatrix
                    C[3 * c + d] = dn + s->dt * AU[3 * c + d];
                }
            // S vector of LagrangeMultiplier<FrictionFixedPoint> (lagrange_multiplier.hpp:286-292):
            // s_c n_c on the first dim components of the contact's rows
            if (s->fixed_point) {
                S.assign(3 * nc, 0.0);
                for (size_t c = 0; c < nc; ++c)
                    for (int d = 0; d < dim; ++d) S[3 * c + d] = s->sij[c] * s->contacts[c].nij[d];
            }
            // LagrangeMultiplier sizes, lagrange_multiplier.hpp:54-60,125-141,217-236
            if (s->p.problem == ORC_FRICTION) {
                size = 3 * (int64_t)nc;
            } else if (s->p.problem == ORC_VISCOUS_FRICTION) {
                // LagrangeMultiplier<ViscousFriction>, lagrange_multiplier.hpp:358-398: one
                // multiplier while gamma >= -gamma_tol, two (l+, l-) while gamma_min < gamma <
                // -gamma_tol, four (l0, f) at gamma == gamma_min; S = dt mu s_c n_c on f
                row.assign(nc, 0);
                mode.assign(nc, 0);
                int64_t r = 0;
                for (size_t c = 0; c < nc; ++c) {
                    row[c] = r;
                    const double gm = s->contacts[c].gamma;
                    if (gm < -s->p.gamma_tol) {
                        mode[c] = gm != s->p.gamma_min ? 1 : 2;
                        r += gm != s->p.gamma_min ? 2 : 4;
                    } else {
                        r += 1;
                    }
                }
                size = r;
                S.assign(size, 0.0);
                for (size_t c = 0; c < nc; ++c)
                    if (mode[c] == 2)
                        for (int d = 0; d < dim; ++d)
                            S[row[c] + 1 + d] = s->dt * s->p.mu * s->sij[c] * s->contacts[c].nij[d];
            } else if (s->p.problem == ORC_VISCOUS) {
                neg_slot.assign(nc, -1);
                int64_t next = (int64_t)nc;
                for (size_t c = 0; c < nc; ++c)
                    if (s->contacts[c].gamma < -s->p.gamma_tol) neg_slot[c] = next++;
                size = next;
            } else {
                size = (int64_t)nc;
            }
        }
        // local2global
        void l2g(const std::vector<double>& x, std::vector<double>& out) const {
            const size_t nc = s->contacts.size();
            const int dim = s->dim;
            if (s->p.problem == ORC_FRICTION) {
                out = x;
                return;
            }
            out.assign(3 * nc, 0.0);
            if (s->p.problem == ORC_VISCOUS_FRICTION) {  // lagrange_multiplier.hpp:428-454
                for (size_t c = 0; c < nc; ++c) {
                    const double* xr = &x[row[c]];
                    const V3& nn = s->contacts[c].nij;
                    for (int d = 0; d < dim; ++d) {
                        if (mode[c] == 0)
                            out[3 * c + d] = xr[0] * nn[d];
                        else if (mode[c] == 1)
                            out[3 * c + d] = (xr[0] - xr[1]) * nn[d];
                        else
                            out[3 * c + d] = (-xr[0]) * nn[d] + xr[1 + d];
                    }
                }
                return;
            }
            for (size_t c = 0; c < nc; ++c) {
                double lc = x[c];
                if (s->p.problem == ORC_VISCOUS && neg_slot[c] >= 0) lc = x[c] - x[neg_slot[c]];
                for (int d = 0; d < dim; ++d) out[3 * c + d] = lc * s->contacts[c].nij[d];
            }
        }
        // global2local
        void g2l(const std::vector<double>& x, std::vector<double>& out) const {
            const size_t nc = s->contacts.size();
            const int dim = s->dim;
            if (s->p.problem == ORC_FRICTION) {
                out = x;
                return;
            }
            out.assign(size, 0.0);
            if (s->p.problem == ORC_VISCOUS_FRICTION) {  // lagrange_multiplier.hpp:400-426
                for (size_t c = 0; c < nc; ++c) {
                    double acc = 0;
                    for (int d = 0; d < dim; ++d) acc += x[3 * c + d] * s->contacts[c].nij[d];
                    double* o = &out[row[c]];
                    if (mode[c] == 0) {
                        o[0] = acc;
                    } else if (mode[c] == 1) {
                        o[0] = acc;
                        o[1] = -acc;
                    } else {
                        o[0] = -acc;
                        for (int d = 0; d < dim; ++d) o[1 + d] = x[3 * c + d];
                    }
                }
                return;
            }
            for (size_t c = 0; c < nc; ++c) {
                double acc = 0;
                for (int d = 0; d < dim; ++d) acc += x[3 * c + d] * s->contacts[c].nij[d];
                out[c] = acc;
                if (s->p.problem == ORC_VISCOUS && neg_slot[c] >= 0) out[neg_slot[c]] = -acc;
            }
        }
        // QMatrix::operator(), minimization_problem.hpp:85-92
        void Q(const std::vector<double>& lg, std::vector<double>& out) const {
            s->atmat(lg, w1);
            for (size_t k = 0; k < w1.size(); ++k) w1[k] = invM[k] * w1[k];
            s->amat(w1, out);
            const double dt2 = s->dt * s->dt;
            for (auto& x : out) x = dt2 * x;
        }
        // minimization_problem::gradient, :122-128 (S = 0 except for FrictionFixedPoint)
        void gradient(const std::vector<double>& lam, std::vector<double>& out) const {
            l2g(lam, w2);
            Q(w2, w3);
            for (size_t k = 0; k < w3.size(); ++k) w3[k] = w3[k] + C[k];
            g2l(w3, out);
            if (S.empty()) {
                for (auto& x : out) x = x + 0.0;
            } else {
                for (size_t k = 0; k < out.size(); ++k) out[k] = out[k] + S[k];
            }
        }
        // minimization_problem::operator(), :130-134
        double objective(const std::vector<double>& lam) const {
            l2g(lam, w2);
            Q(w2, w3);
            double acc = 0.0;
            for (size_t k = 0; k < w3.size(); ++k) acc += w2[k] * (0.5 * w3[k] + C[k]);
            double accs = 0.0;
            for (size_t k = 0; k < lam.size(); ++k) accs += lam[k] * (S.empty() ? 0.0 : S[k]);
            return acc + accs;
        }
        // projections, lagrange_multiplier.hpp:104-107, 196-200, 243-268
        void projection(std::vector<double>& lam) const {
            if (s->p.problem == ORC_VISCOUS_FRICTION) {
                projection_viscous_friction(lam);
                return;
            }
            if (s->p.problem != ORC_FRICTION) {
                for (auto& x : lam) x = std::max(x, 0.);
                return;
            }
            const int dim = s->dim;
            const double mu = s->p.mu;
            for (size_t c = 0; c < s->contacts.size(); ++c) {
                double* li = &lam[3 * c];
                const V3& nn = s->contacts[c].nij;
                const double ln = dot_n(li, nn.data(), dim);
                double lt[3] = {0, 0, 0};
                for (int d = 0; d < dim; ++d) lt[d] = li[d] - ln * nn[d];
                const double nrm = norm_n(lt, dim);
                if (nrm > mu * ln) {
                    if (ln <= -mu * nrm) {
                        for (int d = 0; d < dim; ++d) li[d] = 0;
                    } else {
                        const double new_norm = (mu * mu) * (nrm + ln / mu) / (mu * mu + 1);
                        const double new_ln = new_norm / mu;
                        for (int d = 0; d < dim; ++d) lt[d] /= nrm;
                        for (int d = 0; d < dim; ++d) li[d] = new_norm * lt[d] + new_ln * nn[d];
                    }
                }
            }
        }
        // LagrangeMultiplier<ViscousFriction>::projection, lagrange_multiplier.hpp:466-536: on the
        // four-multiplier rows, the nearer (Euclidean, over the 1 + dim entries) of (0, P_cone(f))
        // and (max(l0, 0), 0)
        void projection_viscous_friction(std::vector<double>& lam) const {
            const int dim = s->dim;
            const double mu = s->p.mu;
            for (size_t c = 0; c < s->contacts.size(); ++c) {
                double* li = &lam[row[c]];
                if (mode[c] == 0) {
                    li[0] = std::max(li[0], 0.);
                    continue;
                }
                if (mode[c] == 1) {
                    li[0] = std::max(li[0], 0.);
                    li[1] = std::max(li[1], 0.);
                    continue;
                }
                const V3& nn = s->contacts[c].nij;
                const double* lf = li + 1;
                const double ln = dot_n(lf, nn.data(), dim);
                double lt[3] = {0, 0, 0};
                for (int d = 0; d < dim; ++d) lt[d] = lf[d] - ln * nn[d];
                const double nrm = norm_n(lt, dim);
                double fric[4] = {0, 0, 0, 0};
                if (nrm > mu * ln) {
                    if (!(ln <= -mu * nrm)) {
                        const double new_norm = (mu * mu) * (nrm + ln / mu) / (mu * mu + 1);
                        const double new_ln = new_norm / mu;
                        for (int d = 0; d < dim; ++d) fric[1 + d] = new_norm * (lt[d] / nrm) + new_ln * nn[d];
                    }
                } else {
                    for (int d = 0; d < dim; ++d) fric[1 + d] = lf[d];
                }
                double moins[4] = {std::max(li[0], 0.), 0, 0, 0};
                double df = 0.0, dm = 0.0;
                for (int k = 0; k < 1 + dim; ++k) {
                    df += (fric[k] - li[k]) * (fric[k] - li[k]);
                    dm += (moins[k] - li[k]) * (moins[k] - li[k]);
                }
                const double* pick = std::sqrt(df) < std::sqrt(dm) ? fric : moins;
                for (int k = 0; k < 1 + dim; ++k) li[k] = pick[k];
            }
        }
        void velocities(const std::vector<double>& lam, std::vector<double>& out) const {
            l2g(lam, w2);
            s->atmat(w2, out);
            for (size_t k = 0; k < out.size(); ++k) out[k] = invM[k] * out[k];
        }
    };

    static double norm_diff(const std::vector<double>& a, const std::vector<double>& b) {
        double s = 0.0;
        for (size_t k = 0; k < a.size(); ++k) {
            const double d = a[k] - b[k];
            s += d * d;
        }
        return std::sqrt(s);
    }
    static double dot_diff(const std::vector<double>& g, const std::vector<double>& a, const std::vector<double>& b) {
        double s = 0.0;
        for (size_t k = 0; k < g.size(); ++k) s += g[k] * (a[k] - b[k]);
        return s;
    }

    // apgd::operator(), apgd.hpp:148-221
    std::vector<double> apgd(const Problem& pb) {
        const int64_t sz = pb.size;
        std::vector<double> lam(sz, 0.0), lam1(sz, 0.0), y(sz, 0.0), y1(sz, 0.0), dG;
        double theta = 1.0, theta1 = 1.0;
        double alpha = p.alpha;
        double lipsch = 1. / alpha;
        int64_t ite = 0;
        bool conv = false;
        stats.backtracks = 0;
        stats.restarts = 0;
        while (ite < p.max_ite) {
            ++ite;
            pb.gradient(y, dG);
            for (int64_t k = 0; k < sz; ++k) lam1[k] = y[k] - alpha * dG[k];
            pb.projection(lam1);
            if (p.dynamic_descent) {
                for (;;) {
                    const double lhs = pb.objective(lam1);
                    const double nd = norm_diff(lam1, y);
                    const double rhs = pb.objective(y) + dot_diff(dG, lam1, y) + 0.5 * lipsch * (nd * nd);
                    if (!(lhs >= rhs)) break;
                    lipsch *= 2;
                    alpha = 1. / lipsch;
                    for (int64_t k = 0; k < sz; ++k) lam1[k] = y[k] - alpha * dG[k];
                    pb.projection(lam1);
                    stats.backtracks++;
                }
            }
            if (norm_diff(lam1, lam) < p.tolerance) {
                std::swap(lam, lam1);
                conv = true;
                break;
            }
            theta1 = 0.5 * (theta * std::sqrt(4 + theta * theta) - theta * theta);
            const double beta = theta * (1 - theta) / (theta * theta + theta1);
            for (int64_t k = 0; k < sz; ++k) y1[k] = lam1[k] + beta * (lam1[k] - lam[k]);
            if (p.dynamic_descent) {
                if (dot_diff(dG, lam1, lam) > 0) {
                    y1 = lam1;
                    theta1 = 1.;
                    stats.restarts++;
                }
                lipsch *= 0.97;
                alpha = 1. / lipsch;
            }
            std::swap(lam, lam1);
            std::swap(theta, theta1);
            std::swap(y, y1);
        }
        stats.iterations = ite;
        stats.converged = conv ? 1 : 0;
        return lam;
    }

    // -------------------------------------------------------------- one step
    void step() {
        using clk = std::chrono::steady_clock;
        auto t0 = clk::now();
        const int64_t nA = na();
        // displacement_obstacles, solver.hpp:330-355
        for (int64_t i = 0; i < nin; ++i) {
            V3 w = omega_d[i];
            if (dim == 2) w = {0, 0, omega_d[i][2]};
            const double nw = norm_n(w.data(), 3);
            for (int d = 0; d < dim; ++d) pos[i][d] += dt * vd[i][d];
            rotate_body(q[i], w, nw, dt);
        }
        auto t1 = clk::now();
        detect();
        add_worm_contacts();
        transfer();
        auto t2 = clk::now();
        // vap, vap_fixed.hpp:45-55 / vap_fpd.hpp:69-81
        for (int64_t b = nin; b < n; ++b) {
            if (p.vap == ORC_VAP_FIXED) {
                v[b] = vd[b];
                omega[b] = omega_d[b];
            } else {
                for (int d = 0; d < dim; ++d) v[b][d] += dt * f[b][d] / m[b];
                if (dim == 3) {
                    const double o1 = omega[b][0], o2 = omega[b][1], o3 = omega[b][2];
                    const double j1 = jm[b][0], j2 = jm[b][1], j3 = jm[b][2];
                    omega[b][0] += o2 * o3 * (j3 - j2);
                    omega[b][1] += o1 * o3 * (j1 - j3);
                    omega[b][2] += o1 * o2 * (j2 - j1);
                }
            }
        }
        // OptimGradient::run, OptimGradient.hpp:253-306
        std::vector<V3> uad(nA), wad(nA, V3{0, 0, 0});
        stats.contacts = (int64_t)contacts.size();
        stats.iterations = 0;
        stats.converged = 1;
        stats.violation = 0;
        stats.fixed_point_iterations = 0;
        if (!contacts.empty()) {
            // extra_steps_before_solve<FrictionFixedPoint> (OptimGradient.hpp:85-94): s_c = mu dt
            if (fixed_point) sij.assign(contacts.size(), p.mu * dt);
            // extra_steps_before_solve<ViscousFriction> (OptimGradient.hpp:96-107): s_c = 1 on
            // the contacts at gamma_min
            const bool vf = p.problem == ORC_VISCOUS_FRICTION;
            if (vf) {
                sij.assign(contacts.size(), 0.0);
                for (size_t c = 0; c < contacts.size(); ++c)
                    if (contacts[c].gamma == p.gamma_min) sij[c] = 1.;
            }
            Problem pb(this);
            lambda = apgd(pb);
            std::vector<double> vel;
            auto velocities = [&](const Problem& P) {
                P.velocities(lambda, vel);
                for (int64_t i = 0; i < nA; ++i) {
                    for (int d = 0; d < dim; ++d) {
                        uad[i][d] = v[i + nin][d] + dt * vel[i * 3 + d];
                        if (dim == 3) wad[i][d] = omega[i + nin][d] + dt * vel[(i + nA) * 3 + d];
                    }
                    if (dim == 2) wad[i][2] = omega[i + nin][2] + dt * vel[(i + nA) * 3 + 2];
                }
            };
            velocities(pb);
            if (fixed_point || vf) {
                // extra_steps_after_solve<FrictionFixedPoint> (OptimGradient.hpp:117-176), its
                // <ViscousFriction> twin (:178-250: s_c = |(A u)_t| on the contacts at gamma_min,
                // err = |s - s_old| / (1 + |s|)) and the solve loop of ScopiSolver::run
                // (solver.hpp:286-291)
                int64_t iters = stats.iterations, bts = stats.backtracks, rss = stats.restarts, fp = 0;
                const double mudt = p.mu * dt;
                for (;;) {
                    std::vector<double> Uf(6 * nA, 0.0), AUf;
                    for (int64_t i = 0; i < nA; ++i)
                        for (int d = 0; d < 3; ++d) {
                            Uf[3 * i + d] = d < dim ? uad[i][d] : 0.0;
                            Uf[3 * nA + 3 * i + d] = wad[i][d];
                        }
                    amat(Uf, AUf);
                    double dd = 0.0, ss = 0.0;
                    for (size_t c = 0; c < contacts.size(); ++c) {
                        if (vf && contacts[c].gamma != p.gamma_min) continue;
                        const double dn = dot_n(&AUf[3 * c], contacts[c].nij.data(), dim);
                        double t[3] = {0, 0, 0};
                        for (int d = 0; d < dim; ++d) t[d] = AUf[3 * c + d] - contacts[c].nij[d] * dn;
                        const double snew = vf ? norm_n(t, dim) : mudt * norm_n(t, dim);
                        dd += (snew - sij[c]) * (snew - sij[c]);
                        ss += snew * snew;
                        sij[c] = snew;
                    }
                    ++fp;
                    double err;
                    if (vf) {
                        err = std::sqrt(dd) / (1 + std::sqrt(ss));
                    } else {
                        if (!(mudt > 0.0)) break;  // s stays 0: one solve (the reference's 1/(mu dt) is NaN)
                        err = (1 / mudt) * std::sqrt(dd) / (1 + (1 / mudt) * std::sqrt(ss));
                    }
                    if (err < p.fixed_point_tol || fp >= p.fixed_point_max_iter) break;
                    Problem pf(this);
                    lambda = apgd(pf);
                    velocities(pf);
                    iters += stats.iterations;
                    bts += stats.backtracks;
                    rss += stats.restarts;
                }
                stats.iterations = iters;
                stats.backtracks = bts;
                stats.restarts = rss;
                stats.fixed_point_iterations = fp;
            }
            // predicted gap after the step: d + dt n.(A u)
            std::vector<double> Un(6 * nA, 0.0), AU;
            for (int64_t i = 0; i < nA; ++i)
                for (int d = 0; d < 3; ++d) {
                    Un[3 * i + d] = d < dim ? uad[i][d] : 0.0;
                    Un[3 * nA + 3 * i + d] = wad[i][d];
                }
            amat(Un, AU);
            double viol = 0;
            for (size_t c = 0; c < contacts.size(); ++c) {
                double g = contacts[c].dij;
                for (int d = 0; d < dim; ++d) g += dt * contacts[c].nij[d] * AU[3 * c + d];
                viol = std::max(viol, -g);
            }
            stats.violation = viol;
            // update_contact_properties_impl<Viscous>, OptimGradient.hpp:19-35 (<ViscousFriction>
            // :36-52, the same update on its own local-to-global map)
            if (p.problem == ORC_VISCOUS || vf) {
                std::vector<double> lg;
                pb.l2g(lambda, lg);
                for (size_t c = 0; c < contacts.size(); ++c) {
                    const double dl = dot_n(contacts[c].nij.data(), &lg[3 * c], dim);
                    contacts[c].gamma = std::min(std::max(contacts[c].gamma - dt * dl, p.gamma_min), 0.);
                }
            }
        } else {
            lambda.clear();
            for (int64_t i = 0; i < nA; ++i) {
                for (int d = 0; d < dim; ++d) uad[i][d] = v[i + nin][d];
                if (dim == 3) wad[i] = omega[i + nin];
                if (dim == 2) wad[i][2] = omega[i + nin][2];
            }
        }
        auto t3 = clk::now();
        // update_velocity, solver.hpp:528-546
#pragma omp parallel for
        for (int64_t i = 0; i < nA; ++i) {
            for (int d = 0; d < dim; ++d) v[i + nin][d] = uad[i][d];
            if (dim == 2)
                omega[i + nin][2] = wad[i][2];
            else
                omega[i + nin] = wad[i];
        }
        // move_active_particles, solver.hpp:441-480
#pragma omp parallel for
        for (int64_t i = 0; i < nA; ++i) {
            const int64_t b = i + nin;
            V3 w;
            double nw;
            if (dim == 2) {
                w = {0, 0, omega[b][2]};
                nw = std::abs(omega[b][2]);
            } else {
                w = omega[b];
                nw = norm_n(w.data(), 3);
            }
            for (int d = 0; d < dim; ++d) pos[b][d] += dt * v[b][d];
            rotate_body(q[b], w, nw, dt);
        }
        // periodic wrap of every object beyond a periodic bound (solver.hpp:482-522)
        for (int d = 0; d < dim; ++d) {
            if (!p.periodic[d]) continue;
            const double L = p.box_upper[d] - p.box_lower[d];
            for (int64_t b = 0; b < n; ++b) {
                const bool plus = pos[b][d] > p.box_upper[d], minus = pos[b][d] < p.box_lower[d];
                if (plus) pos[b][d] -= L;
                if (minus) pos[b][d] += L;
            }
        }
        auto t4 = clk::now();
        auto sec = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
        stats.seconds_contacts += sec(t1, t2);
        stats.seconds_solve += sec(t2, t3);
        stats.seconds_other += sec(t0, t1) + sec(t3, t4);
        old_contacts = contacts;
    }

    void load(const orc_particles* in) {
        n = in->n;
        nin = in->nb_inactive;
        shape.assign(in->shape, in->shape + n);
        auto v3 = [&](const double* src, std::vector<V3>& dst) {
            dst.resize(n);
            for (int64_t i = 0; i < n; ++i) dst[i] = {src[3 * i], src[3 * i + 1], src[3 * i + 2]};
        };
        v3(in->pos, pos);
        v3(in->v, v);
        v3(in->omega, omega);
        v3(in->vd, vd);
        v3(in->omega_d, omega_d);
        v3(in->f, f);
        v3(in->j, jm);
        q.resize(n);
        for (int64_t i = 0; i < n; ++i) q[i] = {in->q[4 * i], in->q[4 * i + 1], in->q[4 * i + 2], in->q[4 * i + 3]};
        m.assign(in->m, in->m + n);
        radius.assign(in->radius, in->radius + n);
        length.assign(in->length, in->length + n);
        worm.assign(n, -1);
        has_worms = false;
        if (in->worm)
            for (int64_t i = 0; i < n; ++i) {
                worm[i] = in->worm[i];
                if (worm[i] >= 0) has_worms = true;
            }
        se_par.assign(n, {0, 0, 0, 1, 1});
        if (in->axes && in->squareness)
            for (int64_t i = 0; i < n; ++i)
                se_par[i] = {in->axes[3 * i], in->axes[3 * i + 1], in->axes[3 * i + 2], in->squareness[2 * i],
                             in->squareness[2 * i + 1]};
    }
    orc_se::SE se_of(int64_t b) const {
        orc_se::SE s;
        s.c = pos[b];
        s.R = rotation3(q[b]);
        for (int k = 0; k < 3; ++k) s.r[k] = se_par[b][k];
        s.e = se_par[b][3];
        s.n = se_par[b][4];
        return s;
    }
    orc_se::SE sphere_of(int64_t b) const { return orc_se::as_se(pos[b], rotation3(q[b]), radius[b]); }
    orc_se::Plane plane_of(int64_t b) const {
        orc_se::Plane p;
        p.c = pos[b];
        p.R = rotation3(q[b]);
        return p;
    }
    static Contact from_pair(const orc_se::PairOut& o) {
        Contact c{};
        c.pi = o.pi;
        c.pj = o.pj;
        c.nij = o.nij;
        c.dij = o.dij;
        return c;
    }
};

extern "C" {

orc_solver* orc_create(const orc_params* p, const orc_particles* parts) {
    if (!p || !parts || (p->dim != 2 && p->dim != 3)) return nullptr;
    auto* s = new orc_solver();
    s->p = *p;
    if (p->problem == ORC_FRICTION_FIXED_POINT) {
        s->fixed_point = true;
        s->p.problem = ORC_FRICTION;
    }
    s->dim = p->dim;
    s->load(parts);
    if ((s->has_worms && p->problem != ORC_NOFRICTION) || (s->has_worms && s->periodic_any())) {
        delete s;
        return nullptr;
    }
#ifdef _OPENMP
    if (p->num_threads > 0) omp_set_num_threads(p->num_threads);
#endif
    return s;
}

void orc_destroy(orc_solver* s) { delete s; }

int orc_run(orc_solver* s, double dt, int64_t total_it, int64_t initial_iter) {
    if (!s) return -1;
    s->dt = dt;
    for (int64_t it = initial_iter; it < total_it; ++it) {
        s->step();
        if (s->periodic_error) return -2;
    }
    return 0;
}

int orc_set_particles(orc_solver* s, const orc_particles* in) {
    if (!s || !in) return -1;
    s->load(in);
    if (s->has_worms && s->p.problem != ORC_NOFRICTION) return -1;
    return 0;
}

int orc_get_particles(const orc_solver* s, orc_particles* o) {
    if (!s || !o) return -1;
    for (int64_t i = 0; i < s->n; ++i) {
        for (int d = 0; d < 3; ++d) {
            if (o->pos) o->pos[3 * i + d] = s->pos[i][d];
            if (o->v) o->v[3 * i + d] = s->v[i][d];
            if (o->omega) o->omega[3 * i + d] = s->omega[i][d];
        }
        if (o->q)
            for (int d = 0; d < 4; ++d) o->q[4 * i + d] = s->q[i][d];
    }
    return 0;
}

int64_t orc_num_contacts(const orc_solver* s) { return s ? (int64_t)s->contacts.size() : -1; }

int64_t orc_get_contacts(const orc_solver* s, int64_t* ci, int64_t* cj, double* dij, double* nij, double* pi,
                         double* pj, double* gamma, int64_t cap) {
    if (!s) return -1;
    const int64_t nc = std::min<int64_t>(cap, (int64_t)s->contacts.size());
    for (int64_t k = 0; k < nc; ++k) {
        const Contact& c = s->contacts[k];
        if (ci) ci[k] = c.i;
        if (cj) cj[k] = c.j;
        if (dij) dij[k] = c.dij;
        if (gamma) gamma[k] = c.gamma;
        for (int d = 0; d < 3; ++d) {
            if (nij) nij[3 * k + d] = c.nij[d];
            if (pi) pi[3 * k + d] = c.pi[d];
            if (pj) pj[3 * k + d] = c.pj[d];
        }
    }
    return nc;
}

int64_t orc_get_lambda(const orc_solver* s, double* out, int64_t cap) {
    if (!s) return -1;
    const int64_t nl = std::min<int64_t>(cap, (int64_t)s->lambda.size());
    if (out) std::memcpy(out, s->lambda.data(), nl * sizeof(double));
    return (int64_t)s->lambda.size();
}

int orc_get_stats(const orc_solver* s, orc_stats* out) {
    if (!s || !out) return -1;
    *out = s->stats;
    return 0;
}

int64_t orc_detect(orc_solver* s) {
    if (!s) return -1;
    s->detect();
    return (int64_t)s->contacts.size();
}

int orc_amat(const orc_solver* s, const double* u, double* out) {
    if (!s) return -1;
    std::vector<double> uu(u, u + 6 * s->na()), o;
    s->amat(uu, o);
    std::memcpy(out, o.data(), o.size() * sizeof(double));
    return 0;
}

int orc_atmat(const orc_solver* s, const double* fv, double* out) {
    if (!s) return -1;
    std::vector<double> ff(fv, fv + 3 * s->contacts.size()), o;
    s->atmat(ff, o);
    std::memcpy(out, o.data(), o.size() * sizeof(double));
    return 0;
}

namespace {
orc_se::SE se_from(const double* a) {
    orc_se::SE s;
    s.c = {a[0], a[1], a[2]};
    s.R = rotation3({a[3], a[4], a[5], a[6]});
    for (int k = 0; k < 3; ++k) s.r[k] = a[7 + k];
    s.e = a[10];
    s.n = a[11];
    return s;
}
void write_pair(const orc_se::PairOut& o, double* out) {
    for (int k = 0; k < 3; ++k) {
        out[k] = o.pi[k];
        out[3 + k] = o.pj[k];
        out[6 + k] = o.nij[k];
    }
    out[9] = o.dij;
    for (int k = 0; k < 4; ++k) out[10 + k] = o.u[k];
    out[14] = o.nfev;
}
}  // namespace

int orc_se_se(const double* s1, const double* s2, double* out) {
    const orc_se::PairOut o = orc_se::se_se(se_from(s1), se_from(s2));
    write_pair(o, out);
    return o.info;
}

int orc_se_plane(const double* s, const double* plane, double* out) {
    orc_se::Plane p;
    p.c = {plane[0], plane[1], plane[2]};
    p.R = rotation3({plane[3], plane[4], plane[5], plane[6]});
    const orc_se::PairOut o = orc_se::se_plane(se_from(s), p);
    write_pair(o, out);
    return o.info;
}

int orc_se_se_from(const double* s1, const double* s2, const double* u0, double* out) {
    const orc_se::PairOut o = orc_se::se_se(se_from(s1), se_from(s2), u0);
    write_pair(o, out);
    return o.info;
}

double orc_se_se_start_value(const double* s1, const double* s2, const double* u) {
    const orc_se::SE a = se_from(s1), b = se_from(s2);
    const orc_se::V3 p1 = orc_se::point(a, u[0], u[1]), n1 = orc_se::normal(a, u[0], u[1]);
    const orc_se::V3 p2 = orc_se::point(b, u[2], u[3]), n2 = orc_se::normal(b, u[2], u[3]);
    const orc_se::V3 df = {p1[0] - p2[0], p1[1] - p2[1], p1[2] - p2[2]};
    return orc_se::norm(df) + 2 * (1 + orc_se::dot(n1, n2));
}

void orc_se_se_start(const double* s1, const double* s2, double* u0) {
    orc_se::sese_start(se_from(s1), se_from(s2), u0);
}

int orc_se_se_hybrid(const double* s1, const double* s2, double* u, int* nfev) {
    const orc_se::SE a = se_from(s1), b = se_from(s2);
    const orc_se::HybrResult h = orc_se::hybrj<4>([&](const double* x, double* F) { orc_se::sese_F(a, b, x, F); },
                                                  [&](const double* x, double* J) { orc_se::sese_J(a, b, x, J); }, u);
    if (nfev) *nfev = h.nfev;
    return h.info;
}

void orc_se_plane_residual(const double* s, const double* plane, const double* u, double* F) {
    orc_se::Plane p;
    p.c = {plane[0], plane[1], plane[2]};
    p.R = rotation3({plane[3], plane[4], plane[5], plane[6]});
    const orc_se::SE b = se_from(s);
    const orc_se::V3 np = orc_se::plane_normal(p);
    const orc_se::V3 rel = {b.c[0] - p.c[0], b.c[1] - p.c[1], b.c[2] - p.c[2]};
    orc_se::sep_F(b, p, orc_se::dot(rel, np) < 0 ? -1.0 : 1.0, u, F);
}

void orc_se_se_system(const double* s1, const double* s2, const double* u, double* F, double* J) {
    const orc_se::SE a = se_from(s1), b = se_from(s2);
    orc_se::sese_F(a, b, u, F);
    orc_se::sese_J(a, b, u, J);
}

int orc_se2_se2(const double* s1, const double* s2, double* out) {
    const orc_se::PairOut o = orc_se::se2_se2(se_from(s1), se_from(s2));
    write_pair(o, out);
    return o.info;
}

int orc_se2_hybrid(const double* s1, const double* s2, double* u, int* nfev) {
    const orc_se::SE a = se_from(s1), b = se_from(s2);
    const orc_se::HybrResult h = orc_se::hybrj<2>([&](const double* x, double* F) { orc_se::se2_F(a, b, x, F); },
                                                  [&](const double* x, double* J) { orc_se::se2_J(a, b, x, J); }, u);
    if (nfev) *nfev = h.nfev;
    return h.info;
}

void orc_se2_system(const double* s1, const double* s2, const double* u, double* F, double* J) {
    const orc_se::SE a = se_from(s1), b = se_from(s2);
    orc_se::se2_F(a, b, u, F);
    orc_se::se2_J(a, b, u, J);
}

// sph = (centre[3], quaternion[4], radius); out as orc_se_se plus out[15] = the method's return
int orc_sphere_se(int dim, const double* se, const double* sph, int reference_labels, int se_is_i, double* out) {
    const orc_se::SE E = se_from(se);
    const orc_se::SE S = orc_se::as_se({sph[0], sph[1], sph[2]}, rotation3({sph[3], sph[4], sph[5], sph[6]}), sph[7]);
    const orc_se::PairOut o = reference_labels ? orc_se::sphere_se_newton(E, S, dim)
                              : (se_is_i ? orc_se::sphere_se_pair(E, S, true, dim) : orc_se::sphere_se_pair(S, E, false, dim));
    write_pair(o, out);
    out[15] = o.info;
    return o.info;
}

int orc_se2_plane(const double* s, const double* plane, double* out) {
    orc_se::Plane p;
    p.c = {plane[0], plane[1], plane[2]};
    p.R = rotation3({plane[3], plane[4], plane[5], plane[6]});
    const orc_se::PairOut o = orc_se::se2_plane(se_from(s), p);
    write_pair(o, out);
    return o.info;
}

// A x = b for a column-major 4 x 4 A (the Newton method's solve); 0, or -2 on a zero pivot
int orc_lu_solve4(const double* A, const double* b, double* x) {
    double a[16];
    std::memcpy(a, A, sizeof(a));
    std::memcpy(x, b, 4 * sizeof(double));
    return orc_se::lu_solve<4>(a, x) ? 0 : -2;
}

}  // extern "C"
