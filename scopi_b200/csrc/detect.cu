// detect.cu -- obstacle motion, a-priori velocity, cell-list contact detection, closest
// points, contact-Jacobian assembly, particle-major incidence lists, viscous gamma
// update and the velocity/position/quaternion integration.
//
// Built with -fmad=false: the closest-point arithmetic keeps the exact operation
// order of the reference formulas (no contraction into FMA), so the strict test
// dij < dmax (include/scopi/contact/base.hpp:118) selects the same pairs, bit for
// bit, as the CPU restatement of the reference evaluated in the same order.
#include <math.h>

#include "kernels.cuh"
#include "se_geom.cuh"
#include "se_newton.cuh"

namespace scopi_gpu {

static long long g_detect_launches = 0;
long long detect_launches() { return g_detect_launches; }
#define LAUNCHED(k) (g_detect_launches += (k))

namespace {

constexpr int kSphere = 0, kPlane = 1, kSegment = 2, kSuperellipsoid = 3;
constexpr int kBBoxBlocks = 4 * kSMs;

struct PairGeom {
    double dij;
    double nij[3], pi[3], pj[3];
};

__device__ __forceinline__ double xsign(double x) { return (x > 0.0) ? 1.0 : ((x < 0.0) ? -1.0 : 0.0); }

__device__ __forceinline__ double norm_n(const double* x, int n) {
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += x[k] * x[k];
    return sqrt(s);
}
__device__ __forceinline__ double dot_n(const double* a, const double* b, int n) {
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += a[k] * b[k];
    return s;
}

// column 0 of rotation_matrix<dim>(q): plane::normal / segment::normal
// (include/scopi/objects/types/plane.hpp:143-147, include/scopi/quaternion.hpp:66-124)
__device__ __forceinline__ void body_normal(const double* q, int dim, double* nrm) {
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    if (dim == 2) {
        nrm[0] = 1 - 2 * w * w;
        nrm[1] = 2 * x * w;
        nrm[2] = 0.0;
    } else {
        nrm[0] = 1 - 2 * z * z - 2 * w * w;
        nrm[1] = 2 * y * z + 2 * x * w;
        nrm[2] = 2 * y * w - 2 * x * z;
    }
}

// rotation_matrix<3>(q), include/scopi/quaternion.hpp:87-124
__device__ __forceinline__ void rotation3(const double* q, double r[3][3]) {
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    r[0][0] = 1 - 2 * z * z - 2 * w * w;
    r[0][1] = 2 * y * z - 2 * x * w;
    r[0][2] = 2 * y * w + 2 * x * z;
    r[1][0] = 2 * y * z + 2 * x * w;
    r[1][1] = 1 - 2 * y * y - 2 * w * w;
    r[1][2] = 2 * z * w - 2 * x * y;
    r[2][0] = 2 * y * w - 2 * x * z;
    r[2][1] = 2 * z * w + 2 * x * y;
    r[2][2] = 1 - 2 * y * y - 2 * z * z;
}

// detail::cross<dim>, include/scopi/matrix/velocities.hpp:26-44
__device__ __forceinline__ void cross_dim(int dim, const double* x, const double* y, double* o) {
    if (dim == 2) {
        o[0] = x[1] * y[2];
        o[1] = -x[0] * y[2];
        o[2] = x[0] * y[1] - x[1] * y[0];
    } else {
        o[0] = x[1] * y[2] - x[2] * y[1];
        o[1] = x[2] * y[0] - x[0] * y[2];
        o[2] = x[0] * y[1] - x[1] * y[0];
    }
}

// closest_points(sphere, sphere), include/scopi/objects/methods/closest_points.hpp:36-50
__device__ __forceinline__ void sphere_sphere(int dim, const double* xa, double ra, const double* xb, double rb,
                                              PairGeom& g) {
    double d[3] = {0, 0, 0};
    for (int k = 0; k < dim; ++k) d[k] = xb[k] - xa[k];
    const double nrm = norm_n(d, dim);
    double u[3] = {0, 0, 0};
    for (int k = 0; k < dim; ++k) u[k] = d[k] / nrm;
    for (int k = 0; k < 3; ++k) g.pi[k] = g.pj[k] = g.nij[k] = 0.0;
    for (int k = 0; k < dim; ++k) {
        g.pi[k] = xa[k] + ra * u[k];
        g.pj[k] = xb[k] - rb * u[k];
    }
    double t[3] = {0, 0, 0};
    for (int k = 0; k < dim; ++k) t[k] = g.pj[k] - xb[k];
    const double nt = norm_n(t, dim);
    for (int k = 0; k < dim; ++k) g.nij[k] = t[k] / nt;
    double diff[3] = {0, 0, 0};
    for (int k = 0; k < dim; ++k) diff[k] = g.pi[k] - g.pj[k];
    g.dij = dot_n(diff, g.nij, dim);
}

// closest_points(sphere, plane), closest_points.hpp:768-788
__device__ __forceinline__ void sphere_plane(int dim, const double* xs, double rs, const double* xp, const double* qp,
                                             PairGeom& g) {
    double nrm[3];
    body_normal(qp, dim, nrm);
    double d[3] = {0, 0, 0};
    for (int k = 0; k < dim; ++k) d[k] = xs[k] - xp[k];
    const double p2s = dot_n(d, nrm, dim);
    const double sg = xsign(p2s);
    for (int k = 0; k < 3; ++k) g.pi[k] = g.pj[k] = g.nij[k] = 0.0;
    for (int k = 0; k < dim; ++k) {
        g.pi[k] = xs[k] - sg * rs * nrm[k];
        g.pj[k] = xs[k] - p2s * nrm[k];
        g.nij[k] = sg * nrm[k];
    }
    double diff[3] = {0, 0, 0};
    for (int k = 0; k < dim; ++k) diff[k] = g.pi[k] - g.pj[k];
    g.dij = dot_n(diff, g.nij, dim);
}

// closest_points(sphere, segment), closest_points.hpp:824-870; segment.hpp:155-181 (2D)
__device__ __forceinline__ void sphere_segment(const double* sp, double rs, const double* xg, const double* qg,
                                               double len, PairGeom& g) {
    const double x = qg[0], w = qg[3];
    const double r01 = -2 * x * w, r11 = 1 - 2 * w * w;
    const double h = 0.5 * len;
    double e0[2], e1[2];
    e0[0] = (0.0 * (1 - 2 * w * w) + r01 * (-h)) + xg[0];
    e0[1] = (0.0 * (2 * x * w) + r11 * (-h)) + xg[1];
    e1[0] = (0.0 * (1 - 2 * w * w) + r01 * h) + xg[0];
    e1[1] = (0.0 * (2 * x * w) + r11 * h) + xg[1];
    double nrm[3];
    body_normal(qg, 2, nrm);
    const double tg[2] = {-nrm[1], nrm[0]};
    const double d0[2] = {sp[0] - e0[0], sp[1] - e0[1]};
    const double d1[2] = {sp[0] - e1[0], sp[1] - e1[1]};
    for (int k = 0; k < 3; ++k) g.pi[k] = g.pj[k] = g.nij[k] = 0.0;
    if (dot_n(d0, tg, 2) < 0 || dot_n(d1, tg, 2) > 0) {
        const bool first = dot_n(d0, tg, 2) < 0;
        const double* e = first ? e0 : e1;
        const double* de = first ? d0 : d1;
        const double nn = norm_n(de, 2);
        for (int k = 0; k < 2; ++k) {
            g.nij[k] = de[k] / nn;
            g.pi[k] = sp[k] - g.nij[k] * rs;
            g.pj[k] = e[k];
        }
    } else {
        const double d[2] = {sp[0] - xg[0], sp[1] - xg[1]};
        const double s2s = dot_n(d, nrm, 2);
        const double sgn = xsign(s2s);
        for (int k = 0; k < 2; ++k) {
            g.pi[k] = sp[k] - sgn * rs * nrm[k];
            g.pj[k] = sp[k] - s2s * nrm[k];
            g.nij[k] = sgn * nrm[k];
        }
    }
    const double diff[2] = {g.pi[0] - g.pj[0], g.pi[1] - g.pj[1]};
    g.dij = dot_n(diff, g.nij, 2);
}

__device__ __forceinline__ void flip(PairGeom& g) {
    for (int k = 0; k < 3; ++k) {
        g.nij[k] *= -1.;
        const double t = g.pi[k];
        g.pi[k] = g.pj[k];
        g.pj[k] = t;
    }
}

// closest_points_dispatcher restricted to the pairs of the hot path (a < b).  SE = the scene
// holds superellipsoids: their obstacle cases (plane-superellipsoid) compile into those
// instantiations only, so the sphere scenes' kernels carry none of their code.
template <bool SE>
__device__ __forceinline__ bool exact_pair(const Bodies& B, int dim, int a, int b, PairGeom& g) {
    const int sa = B.shape[a], sb = B.shape[b];
    const double* xa = B.pos + 3 * (long long)a;
    const double* xb = B.pos + 3 * (long long)b;
    if (sa == kSphere && sb == kSphere) {
        sphere_sphere(dim, xa, B.radius[a], xb, B.radius[b], g);
    } else if (sa == kPlane && sb == kSphere) {  // closest_points.hpp:802-809
        sphere_plane(dim, xb, B.radius[b], xa, B.q + 4 * (long long)a, g);
        flip(g);
    } else if (sa == kSphere && sb == kPlane) {
        sphere_plane(dim, xa, B.radius[a], xb, B.q + 4 * (long long)b, g);
    } else if (sa == kSegment && sb == kSphere && dim == 2) {  // closest_points.hpp:874-881
        sphere_segment(xb, B.radius[b], xa, B.q + 4 * (long long)a, B.length[a], g);
        flip(g);
    } else if (sa == kSphere && sb == kSegment && dim == 2) {
        sphere_segment(xa, B.radius[a], xb, B.q + 4 * (long long)b, B.length[b], g);
    } else {
        if constexpr (SE) {
            if (sa == kPlane && sb == kSuperellipsoid && dim == 3) {  // closest_points.hpp:1761-1768
                const se::Body s = se::load(B, b);
                se::body_plane(s, xa, B.q + 4 * (long long)a, g.pi, g.pj, g.nij, g.dij);
                flip(g);
                return true;
            }
            if (sa == kSuperellipsoid && sb == kPlane && dim == 3) {
                const se::Body s = se::load(B, a);
                se::body_plane(s, xb, B.q + 4 * (long long)b, g.pi, g.pj, g.nij, g.dij);
                return true;
            }
            if (sa == kPlane && sb == kSuperellipsoid && dim == 2) {  // closest_points.hpp:1951-1958
                const se::Body2 s = se::load2(B, b);
                se::body_plane2(s, xa, B.q + 4 * (long long)a, g.pi, g.pj, g.nij, g.dij);
                flip(g);
                return true;
            }
            if (sa == kSuperellipsoid && sb == kPlane && dim == 2) {
                const se::Body2 s = se::load2(B, a);
                se::body_plane2(s, xb, B.q + 4 * (long long)b, g.pi, g.pj, g.nij, g.dij);
                return true;
            }
        }
        return false;  // superellipsoid pairs: se.cu; sphere-superellipsoid: k_geometry
    }
    return true;
}

// mult_quaternion (src/quaternion.cpp:92-120), normalize (:6-10) and the exp map of
// solver.hpp:335-351 / 449-479.
__device__ __forceinline__ void rotate_body(double* q, const double* w, double normw, double dt) {
    if (normw == 0) normw = 1;
    double e[4];
    e[0] = cos(0.5 * normw * dt);
    const double s = sin(0.5 * normw * dt) / normw;
    for (int d = 0; d < 3; ++d) e[d + 1] = s * w[d];
    double r[4];
    r[0] = q[0] * e[0];
    for (int d = 0; d < 3; ++d) {
        r[0] -= q[d + 1] * e[d + 1];
        r[d + 1] = q[0] * e[d + 1] + e[0] * q[d + 1];
    }
    r[1] += (q[2] * e[3] - q[3] * e[2]);
    r[2] += (q[3] * e[1] - q[1] * e[3]);
    r[3] += (q[1] * e[2] - q[2] * e[1]);
    const double nq = norm_n(r, 4);
    for (int d = 0; d < 4; ++d) q[d] = r[d] / nq;
}

// ------------------------------------------------------------------ kernels

__global__ void k_obstacles_move(Bodies B, double dt, int dim) {
    GRID_STRIDE(i, B.nin) {
        double w[3] = {B.omega_d[3 * i], B.omega_d[3 * i + 1], B.omega_d[3 * i + 2]};
        if (dim == 2) w[0] = w[1] = 0.0;
        const double nw = norm_n(w, 3);
        for (int d = 0; d < dim; ++d) B.pos[3 * i + d] += dt * B.vd[3 * i + d];
        rotate_body(B.q + 4 * i, w, nw, dt);
    }
}

// vap_fixed::set_a_priori_velocity_impl (vap_fixed.hpp:45-55), vap_fpd (vap_fpd.hpp:69-81,
// src/vap/vap_fpd.cpp:6-26)
__global__ void k_vap(Bodies B, StepParams p, const Sizes* sizes) {
    if (sizes && sizes->overflow) return;  // the step is redone after the buffers grow
    GRID_STRIDE(k, B.n - B.nin) {
        const long long b = B.nin + k;
        if (p.vap == 0) {
            for (int d = 0; d < 3; ++d) {
                B.v[3 * b + d] = B.vd[3 * b + d];
                B.omega[3 * b + d] = B.omega_d[3 * b + d];
            }
        } else {
            for (int d = 0; d < p.dim; ++d) B.v[3 * b + d] += p.dt * B.f[3 * b + d] / B.m[b];
            if (p.dim == 3) {
                const double o1 = B.omega[3 * b], o2 = B.omega[3 * b + 1], o3 = B.omega[3 * b + 2];
                const double j1 = B.j[3 * b], j2 = B.j[3 * b + 1], j3 = B.j[3 * b + 2];
                B.omega[3 * b] += o2 * o3 * (j3 - j2);
                B.omega[3 * b + 1] += o1 * o3 * (j1 - j3);
                B.omega[3 * b + 2] += o1 * o2 * (j2 - j1);
            }
        }
    }
}

__global__ void k_bbox_partial(Bodies B, int dim, double* partial) {
    __shared__ double sh[8][kThreads];
    double v[7] = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300, 0.0};
    GRID_STRIDE(k, B.n - B.nin) {
        const long long b = B.nin + k;
        for (int d = 0; d < dim; ++d) {
            const double x = d == 0 ? key_x(B, b, B.pos[3 * b]) : B.pos[3 * b + d];
            v[d] = fmin(v[d], x);
            v[3 + d] = fmax(v[3 + d], x);
        }
        v[6] = fmax(v[6], B.radius[b]);
    }
    for (int k = 0; k < 7; ++k) sh[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] = fmin(sh[k][threadIdx.x], sh[k][threadIdx.x + s]);
            for (int k = 3; k < 7; ++k) sh[k][threadIdx.x] = fmax(sh[k][threadIdx.x], sh[k][threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 7; ++k) partial[blockIdx.x * 8 + k] = sh[k][0];
}

__global__ void k_grid_setup(const double* partial, int nparts, int dim, double dmax, long long cell_cap, int na,
                             Grid* grid) {
    __shared__ double sh[7][32];
    double v[7] = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300, 0.0};
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
        for (int k = 0; k < 3; ++k) {
            v[k] = fmin(v[k], partial[b * 8 + k]);
            v[3 + k] = fmax(v[3 + k], partial[b * 8 + 3 + k]);
        }
        v[6] = fmax(v[6], partial[b * 8 + 6]);
    }
    for (int k = 0; k < 7; ++k) sh[k][threadIdx.x] = v[k];
    __syncthreads();
    if (threadIdx.x != 0) return;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300}, rmax = 0.0;
    for (int t = 0; t < 32; ++t) {
        for (int k = 0; k < 3; ++k) {
            lo[k] = fmin(lo[k], sh[k][t]);
            hi[k] = fmax(hi[k], sh[3 + k][t]);
        }
        rmax = fmax(rmax, sh[6][t]);
    }
    if (na == 0) {
        for (int k = 0; k < 3; ++k) lo[k] = hi[k] = 0.0;
    }
    for (int k = dim; k < 3; ++k) lo[k] = hi[k] = 0.0;
    double h = (2 * rmax + dmax) * (1 + 1e-6) + 1e-12;
    int nc[3] = {1, 1, 1};
    long long tot = 1;
    for (int guard = 0; guard < 200; ++guard) {
        tot = 1;
        for (int k = 0; k < dim; ++k) {
            double c = floor((hi[k] - lo[k]) / h) + 1.0;
            if (!(c >= 1.0)) c = 1.0;  // NaN / inf positions: one cell
            if (c > 2.0e9) c = 2.0e9;
            nc[k] = (int)c;
            tot *= nc[k];
        }
        if (tot <= cell_cap) break;
        h *= 1.5;
    }
    for (int k = 0; k < 3; ++k) {
        grid->lo[k] = lo[k];
        grid->nc[k] = nc[k];
    }
    grid->h = h;
    grid->ncell = (int)tot;
    grid->ncell1 = (int)tot + 1;
    grid->rmax = rmax;
}

__device__ __forceinline__ int cell_coord(double x, double lo, double h, int nc) {
    int c = (int)floor((x - lo) / h);
    return c < 0 ? 0 : (c > nc - 1 ? nc - 1 : c);
}

__global__ void k_cell_assign(Bodies B, int dim, const Grid* grid, int* cell_of, int* cell_count) {
    const Grid g = *grid;
    GRID_STRIDE(k, B.n - B.nin) {
        const long long b = B.nin + k;
        int id = 0;
        for (int d = dim - 1; d >= 0; --d) {
            const double x = d == 0 ? key_x(B, b, B.pos[3 * b]) : B.pos[3 * b + d];
            id = id * g.nc[d] + cell_coord(x, g.lo[d], g.h, g.nc[d]);
        }
        cell_of[k] = id;
        atomicAdd(&cell_count[id], 1);
    }
}

// the first body placed in a cell also appends the cell to the occupied list (the search
// visits only those; its result does not depend on their order: rows are sorted after)
__global__ void k_cell_scatter(Bodies B, const int* cell_of, const int* cell_start, int* cell_fill, int* cell_body,
                               double4* cell_pr, int* occ, int* n_occ) {
    GRID_STRIDE(k, B.n - B.nin) {
        const long long b = B.nin + k;
        const int c = cell_of[k];
        const int slot = atomicAdd(&cell_fill[c], 1);
        if (occ && slot == 0) occ[atomicAdd(n_occ, 1)] = c;
        const int at = cell_start[c] + slot;
        cell_body[at] = (int)b;
        cell_pr[at] = make_double4(B.pos[3 * b], B.pos[3 * b + 1], B.pos[3 * b + 2], B.radius[b]);
    }
}

// Pair test of the contact list: kd-tree candidate filter, sphere bound, then the exact
// closest-point distance < dmax (contact_kdtree.hpp:240-262, base.hpp:104-141).  Always
// evaluated with the lower body index first, as the reference does for its (i < j) pairs,
// so that the decision is bitwise the same whichever body finds the pair.
// DIM is a template argument so that the coordinate loops unroll and the small arrays of
// the geometry stay in registers (a runtime dimension puts them in local memory).
template <int DIM>
__device__ __forceinline__ bool pair_in_contact(const StepParams& p, const double4& L, const double4& H) {
    const double xl[3] = {L.x, L.y, L.z}, xh[3] = {H.x, H.y, H.z};
    double s2 = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        const double dd = xl[d] - xh[d];
        s2 += dd * dd;
    }
    if (p.kd_filter && !(s2 < p.kd_radius)) return false;
    const double lim = L.w + H.w + p.dmax;
    if (!(lim > 0.0) || s2 > lim * lim * (1.0 + 1e-9)) return false;
    // superellipsoids (w = bounding radius): the pairs whose bounding spheres come within
    // dmax go to the exact solve of se.cu, which decides
    if (p.se_mode) return true;
    // clearly inside: |x_i - x_j| < (r_i + r_j + dmax)(1 - 5e-10), a margin far above the
    // rounding of the reference's dij (~1e-16 of the coordinates), so its dij < dmax holds;
    // only the pairs in the thin shell around the threshold need the exact formula
    if (s2 < lim * lim * (1.0 - 1e-9)) return true;
    PairGeom pg;
    sphere_sphere(DIM, xl, L.w, xh, H.w, pg);
    return pg.dij < p.dmax;
}

__device__ __forceinline__ void cell_coords(const Grid& g, int id, int* cc) {
    cc[0] = id % g.nc[0];
    cc[1] = (id / g.nc[0]) % g.nc[1];
    cc[2] = id / (g.nc[0] * g.nc[1]);
}

// Enumerates the (a, b > a) active pairs in contact of body a (position and radius A) over
// the 3^dim neighbour cells of its cell.
template <int DIM, typename F>
__device__ __forceinline__ void for_each_pair_of(const Bodies& B, const StepParams& p, const Grid& g,
                                                 const int* cell_of, const int* cell_start, const int* cell_body,
                                                 const double4* cell_pr, int a, const double4& A, F&& emit) {
    int cc[3];
    cell_coords(g, cell_of[a - B.nin], cc);
    const int zr = DIM == 3 ? 1 : 0;
    for (int dz = -zr; dz <= zr; ++dz) {
        const int z = cc[2] + dz;
        if (z < 0 || z >= g.nc[2]) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int y = cc[1] + dy;
            if (y < 0 || y >= g.nc[1]) continue;
            for (int dx = -1; dx <= 1; ++dx) {
                const int x = cc[0] + dx;
                if (x < 0 || x >= g.nc[0]) continue;
                const int cid = (z * g.nc[1] + y) * g.nc[0] + x;
                const int t1 = cell_start[cid + 1];
                for (int t = cell_start[cid]; t < t1; ++t) {
                    const int b = cell_body[t];
                    if (b <= a) continue;
                    if (B.scene && B.scene[a] != B.scene[b]) continue;
                    if (pair_in_contact<DIM>(p, A, cell_pr[t])) emit(a, b);
                }
            }
        }
    }
}

// Offset o of the half stencil: o = 0 the own cell, then the (dz, dy, dx) > (0, 0, 0) in
// lexicographic order (13 in 3D, 4 in 2D).
template <int DIM>
__device__ __forceinline__ void half_stencil(int o, int& dx, int& dy, int& dz) {
    dx = dy = dz = 0;
    if (o == 0) return;
    const int q = o - 1;
    if (DIM == 3) {
        if (q == 0) {
            dx = 1;
        } else if (q < 4) {
            dy = 1;
            dx = q - 2;
        } else {
            dz = 1;
            dy = (q - 4) / 3 - 1;
            dx = (q - 4) % 3 - 1;
        }
    } else {
        if (q == 0) {
            dx = 1;
        } else {
            dy = 1;
            dx = q - 2;
        }
    }
}

// The pair search of 2D scenes, one thread per body: body k (cell-sorted slot) meets the
// bodies after it in its own cell and those of the 4 neighbour cells of the half stencil.
// With the few bodies per cell of 2D scenes (and the many empty cells of a batch's layout)
// this beats a warp per occupied cell: 0.038 against 0.218 ms per step on the 256 pile
// scenes.  Pairs are tested and emitted as k_pair_search_cells does.
template <int DIM>
__global__ void k_pair_search(Bodies B, StepParams p, const Grid* grid, const int* cell_of, const int* cell_start,
                              const int* cell_body, const double4* cell_pr, int* row_count, int* row_tmp) {
    const Grid g = *grid;
    constexpr int nst = DIM == 3 ? 14 : 5;
    GRID_STRIDE(k, B.n - B.nin) {
        const int a = cell_body[k];
        const double4 A = cell_pr[k];
        int cc[3];
        cell_coords(g, cell_of[a - B.nin], cc);
        for (int o = 0; o < nst; ++o) {
            int dx, dy, dz;
            half_stencil<DIM>(o, dx, dy, dz);
            const int x = cc[0] + dx, y = cc[1] + dy, z = cc[2] + dz;
            if (x < 0 || x >= g.nc[0] || y < 0 || y >= g.nc[1] || z >= g.nc[2]) continue;
            const int cid = (z * g.nc[1] + y) * g.nc[0] + x;
            const int t1 = cell_start[cid + 1];
            for (int t = o == 0 ? (int)k + 1 : cell_start[cid]; t < t1; ++t) {
                const int b = cell_body[t];
                if (B.scene && B.scene[a] != B.scene[b]) continue;
                const double4 Bb = cell_pr[t];
                const bool a_lo = a < b;
                if (!pair_in_contact<DIM>(p, a_lo ? A : Bb, a_lo ? Bb : A)) continue;
                const int lo = a_lo ? a : b, hi = a_lo ? b : a;
                const int r = lo - B.nin;
                const int slot = atomicAdd(&row_count[r], 1);
                if (slot < kRowCap) row_tmp[(long long)r * kRowCap + slot] = hi;
            }
        }
    }
}

// The pair search of 3D scenes over the half stencil, one warp per occupied cell: a body meets
// the bodies after it in its own cell and those of the 13 neighbour cells that follow its cell
// in (z, y, x) order, so every unordered pair of neighbouring cells is visited once.  The
// candidate pairs of the cell with itself (a < b by slot) and with its half-stencil neighbours
// are numbered, and the warp's lanes take them 32 at a time (so the uneven cell counts do not
// idle lanes).  A pair in contact is tested with the lower index first, counted in the row of
// its lower index (atomic slot) and its partner kept in that row's scratch while the row has
// room; the row sort makes the order deterministic.
constexpr int kSearchWarps = 8;
template <int DIM>
__global__ void __launch_bounds__(32 * kSearchWarps, 4) k_pair_search_cells(Bodies B, StepParams p, const Grid* grid,
                                                                        const int* cell_start, const int* cell_body,
                                                                        const double4* cell_pr, const int* occ,
                                                                        const int* n_occ, int* row_count,
                                                                        int* row_tmp) {
    constexpr int nst = DIM == 3 ? 14 : 5;
    __shared__ int s_pref[kSearchWarps][16], s_beg[kSearchWarps][16], s_cnt[kSearchWarps][16];
    __shared__ unsigned s_inv[kSearchWarps][16];  // ceil(2^32 / count) for counts >= 2: l / count = umulhi(l, inv)
    const Grid g = *grid;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long nwarps = (long long)gridDim.x * kSearchWarps;
    const long long nocc = *n_occ;
    for (long long t = (long long)blockIdx.x * kSearchWarps + w; t < nocc; t += nwarps) {
        const int cid = occ[t];
        const int h0 = cell_start[cid], nh = cell_start[cid + 1] - h0;
        if (nh == 0) continue;  // the whole warp
        int cc[3];
        cell_coords(g, (int)cid, cc);
        int cnt = 0, beg = 0, ncb = 0;
        if (lane < nst) {
            if (lane == 0) {
                beg = h0;
                ncb = nh;
                cnt = nh * (nh - 1) / 2;
            } else {
                int dx, dy, dz;
                half_stencil<DIM>(lane, dx, dy, dz);
                const int x = cc[0] + dx, y = cc[1] + dy, z = cc[2] + dz;
                if (x >= 0 && x < g.nc[0] && y >= 0 && y < g.nc[1] && z < g.nc[2]) {
                    const int c2 = (z * g.nc[1] + y) * g.nc[0] + x;
                    beg = cell_start[c2];
                    ncb = cell_start[c2 + 1] - beg;
                    cnt = nh * ncb;
                }
            }
        }
        int incl = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        if (lane < 16) {
            s_pref[w][lane] = incl - cnt;
            s_beg[w][lane] = beg;
            s_cnt[w][lane] = ncb;
            // exact quotient for l < 2^16 and 2 <= counts < 2^16 (l < nh * count here); a count
            // of 1 (whose reciprocal 2^32 does not fit) is taken apart in locate
            s_inv[w][lane] = ncb > 1 ? (unsigned)((0x100000000ULL + (unsigned long long)ncb - 1) / ncb) : 0u;
        }
        __syncwarp();
        // two pairs per lane and round: their loads, tests and row-slot atomics overlap
        // (an atomic's returned slot is a round trip to L2 before the store can go)
        // a lane's pair numbers t only grow: its stencil offset advances with them
        int o_cur = 0;
        auto locate = [&](int t, int& sa, int& sb) {
            while (o_cur < nst - 1 && s_pref[w][o_cur + 1] <= t) ++o_cur;
            int l = t - s_pref[w][o_cur];
            if (o_cur == 0) {
                int i = 0;
                while (l >= nh - 1 - i) {
                    l -= nh - 1 - i;
                    ++i;
                }
                sa = h0 + i;
                sb = h0 + i + 1 + l;
            } else {
                const int n2 = s_cnt[w][o_cur];
                const int ia = n2 == 1 ? l : (int)__umulhi((unsigned)l, s_inv[w][o_cur]);
                sa = h0 + ia;
                sb = s_beg[w][o_cur] + (l - ia * n2);
            }
        };
        for (int t0 = lane; t0 < total; t0 += 64) {
            int row[2] = {-1, -1}, part[2] = {0, 0};
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int t = t0 + 32 * q;
                if (t >= total) continue;
                int sa, sb;
                locate(t, sa, sb);
                const int a = cell_body[sa], b = cell_body[sb];
                if (B.scene && B.scene[a] != B.scene[b]) continue;
                const double4 A = cell_pr[sa], Bb = cell_pr[sb];
                const bool a_lo = a < b;
                if (!pair_in_contact<DIM>(p, a_lo ? A : Bb, a_lo ? Bb : A)) continue;
                row[q] = (a_lo ? a : b) - B.nin;
                part[q] = a_lo ? b : a;
            }
            int slot[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) slot[q] = row[q] >= 0 ? atomicAdd(&row_count[row[q]], 1) : kRowCap;
#pragma unroll
            for (int q = 0; q < 2; ++q)
                if (slot[q] < kRowCap) row_tmp[(long long)row[q] * kRowCap + slot[q]] = part[q];
        }
        __syncwarp();  // the tables are rewritten for the next cell
    }
}

// Rows in place: (ci, cj) of row r at c_obs + row_ptr[r]; a row whose partners did not fit
// its scratch is enumerated again over the full stencil by its thread.
template <int DIM>
__global__ void k_pair_compact(Bodies B, StepParams p, const Grid* grid, const int* cell_of, const int* cell_start,
                               const int* cell_body, const double4* cell_pr, const int* row_count, const int* row_tmp,
                               const int* row_ptr, const Sizes* sizes, long long cap, int* ci, int* cj) {
    const Grid g = *grid;
    const int c_obs = sizes->C_obs;
    GRID_STRIDE(r, B.n - B.nin) {
        const int cnt = row_count[r];
        if (cnt == 0) continue;
        const int a = B.nin + (int)r;
        long long at = (long long)c_obs + row_ptr[r];
        if (at + cnt > cap) continue;  // contact buffers too small: the step is redone
        if (cnt <= kRowCap) {
            for (int q = 0; q < cnt; ++q) {
                ci[at + q] = a;
                cj[at + q] = row_tmp[(long long)r * kRowCap + q];
            }
        } else {
            const double4 A = make_double4(B.pos[3 * (long long)a], B.pos[3 * (long long)a + 1],
                                           B.pos[3 * (long long)a + 2], B.radius[a]);
            const long long end = at + cnt;  // the same test finds the same cnt partners
            for_each_pair_of<DIM>(B, p, g, cell_of, cell_start, cell_body, cell_pr, a, A, [&](int i, int j) {
                if (at < end) {
                    ci[at] = i;
                    cj[at] = j;
                }
                ++at;
            });
        }
    }
}

__global__ void k_row_sort(int na, const int* row_ptr, const Sizes* sizes, long long cap, int* cj) {
    const int c_obs = sizes->C_obs;
    GRID_STRIDE(r, na) {
        const long long s = (long long)c_obs + row_ptr[r], e = (long long)c_obs + row_ptr[r + 1];
        if (e > cap) continue;
        for (long long x = s + 1; x < e; ++x) {
            const int key = cj[x];
            long long y = x - 1;
            while (y >= s && cj[y] > key) {
                cj[y + 1] = cj[y];
                --y;
            }
            cj[y + 1] = key;
        }
    }
}

// (obstacle, active) pair of flag slot k: every active for one scene, the obstacle's own
// scene's actives in a batch (rows stay sorted by (obstacle, active))
__device__ __forceinline__ void obs_pair(const Bodies& B, long long k, int& o, int& b) {
    if (!B.obs_off) {
        // nin * na < 2^31 here (the flag arrays are int-indexed): 32-bit division, not
        // the 64-bit one, which the GPU emulates in software
        const unsigned na = (unsigned)(B.n - B.nin), kk = (unsigned)k;
        o = (int)(kk / na);
        b = B.nin + (int)(kk - (unsigned)o * na);
        return;
    }
    int lo = 0, hi = B.nin;  // last o with obs_off[o] <= k
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (B.obs_off[mid] <= k)
            lo = mid;
        else
            hi = mid;
    }
    o = lo;
    b = B.nin + B.obs_a0[o] + (int)(k - B.obs_off[o]);
}

template <int DIM, bool SE>
__global__ void k_obs_flags(Bodies B, StepParams p, long long nobs, int* flag) {
    GRID_STRIDE(k, nobs) {
        int o, b;
        obs_pair(B, k, o, b);
        PairGeom g;
        flag[k] = (exact_pair<SE>(B, DIM, o, b, g) && g.dij < p.dmax) ? 1 : 0;
    }
}

__global__ void k_obs_fill(Bodies B, long long nobs, const int* flag, const int* pos, long long cap, int* ci, int* cj) {
    GRID_STRIDE(k, nobs) {
        if (!flag[k]) continue;
        const long long at = pos[k];
        if (at < cap) {
            int o, b;
            obs_pair(B, k, o, b);
            ci[at] = o;
            cj[at] = b;
        }
    }
}

__global__ void k_sizes(const int* totals, Sizes* sizes, long long cap) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const long long c = (long long)totals[0] + totals[1];
        sizes->C_obs = totals[0];
        sizes->C = (int)(c < cap ? c : cap);
        if (c > cap) sizes->overflow = 1;
    }
}

__global__ void k_set_cobs(const int* totals, Sizes* sizes) {
    if (threadIdx.x == 0 && blockIdx.x == 0) sizes->C_obs = totals[0];
}

// closest points of the listed pairs; viscous gamma carried over from the previous list
// by (i, j) (transfer, include/scopi/solver.hpp:241-258); the last n_links rows are worm
// links, whose normal and distance are negated (add_contact.hpp:17-18).
// SE (scenes with superellipsoids): a sphere-superellipsoid row takes the reference's Newton
// solve (se_newton.cuh), labelled by body (pi on body i, pj on body j, nij the outward
// normal of j pointing toward i, as every other pair: the reference's own functions give the
// points and normal of the pair (j, i) for (sphere, superellipsoid) and that result swapped
// and negated for (superellipsoid, sphere), closest_points.hpp:1275-1280, 1295-1302, with
// which the contact row would push the bodies together); need_se[k] = 1 leaves the row to
// launch_se_pairs (pairs of superellipsoids, and the sphere rows whose solve was refused).
template <int DIM, bool SE>
__global__ void k_geometry(Bodies B, StepParams p, Contacts c, const Sizes* sizes, Contacts old_c, const int* old_C,
                           int* need_se) {
    const int C = sizes->C;
    const int first_link = C - sizes->n_links;
    const int oC = old_C ? *old_C : 0;
    GRID_STRIDE(k, C) {
        const int a = c.ci[k], b = c.cj[k];
        PairGeom g;
        bool known = exact_pair<SE>(B, DIM, a, b, g);
        if constexpr (SE) {
            const int sa = B.shape[a], sb = B.shape[b];
            int need = 0;
            if (sa == kSuperellipsoid && sb == kSuperellipsoid) {
                need = 1;
            } else if ((sa == kSphere && sb == kSuperellipsoid) || (sa == kSuperellipsoid && sb == kSphere)) {
                const bool i_se = sa == kSuperellipsoid;
                const int e = i_se ? a : b, sph = i_se ? b : a;
                se::SphSeOut o;
                if (DIM == 3)
                    o = se::sphere_se3(se::load(B, e), se::sphere_as_body(B, sph));
                else
                    o = se::sphere_se2(se::load2(B, e), se::load_any2(B, sph));
                if (o.valid) {
                    const double sg = i_se ? 1.0 : -1.0;
                    for (int d = 0; d < 3; ++d) {
                        g.pi[d] = i_se ? o.pi[d] : o.pj[d];
                        g.pj[d] = i_se ? o.pj[d] : o.pi[d];
                        g.nij[d] = sg * o.nij[d];
                    }
                    g.dij = o.dij;
                    known = true;
                } else {
                    need = 1;
                }
            }
            if (need_se) need_se[k] = need;
        }
        if (!known) {
            g.dij = 0.0;
            for (int d = 0; d < 3; ++d) g.nij[d] = g.pi[d] = g.pj[d] = 0.0;
        }
        if (k >= first_link) {
            g.dij *= -1.;
            for (int d = 0; d < 3; ++d) g.nij[d] *= -1.;
        }
        c.dij[k] = g.dij;
        for (int d = 0; d < 3; ++d) {
            c.nij[3 * k + d] = g.nij[d];
            c.pi[3 * k + d] = g.pi[d];
            c.pj[3 * k + d] = g.pj[d];
        }
        double gam = p.gamma0;
        if (oC > 0 && old_c.ci) {
            int lo = 0, hi = oC;  // first index with (ci, cj) >= (a, b)
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                const int mi = old_c.ci[mid], mj = old_c.cj[mid];
                if (mi < a || (mi == a && mj < b))
                    lo = mid + 1;
                else
                    hi = mid;
            }
            if (lo < oC && old_c.ci[lo] == a && old_c.cj[lo] == b) gam = old_c.gamma[lo];
        }
        c.gamma[k] = gam;
    }
}

// Per-contact Jacobian rows.  For the normal problems the contact's row of B = n^T A
// (include/scopi/matrix/velocities.hpp:67-144 projected by global2local) is
//   B_c u = n.v_i + a_i.w_i - n.v_j + a_j.w_j,  a_i = R_i^T (r_i x n),  a_j = -R_j^T (r_j x n),
// and c_c = n.(D n + dt A U)_c (CVector, minimization_problem.hpp:34-70).  For friction
// the three rows of A are kept: P = R^T [r]x so A_c = [I, P_i^T, -I, -P_j^T].
template <int DIM>
__global__ void k_assemble(Bodies B, StepParams p, Contacts c, Assembly a, const Sizes* sizes) {
    const int C = sizes->C;
    GRID_STRIDE(k, C) {
        const int bi[2] = {c.ci[k], c.cj[k]};
        const double* n = c.nij + 3 * k;
        double AU[3] = {0, 0, 0};
        double arow[2][3] = {{0, 0, 0}, {0, 0, 0}};
        double P[2][9];
        for (int s = 0; s < 2; ++s)
            for (int e = 0; e < 9; ++e) P[s][e] = 0.0;
        for (int s = 0; s < 2; ++s) {
            const int b = bi[s];
            if (b < B.nin) continue;
            const double* pt = (s == 0 ? c.pi : c.pj) + 3 * k;
            double r[3] = {0, 0, 0};
            for (int d = 0; d < DIM; ++d) r[d] = pt[d] - B.pos[3 * (long long)b + d];
            double R[3][3];
            rotation3(B.q + 4 * (long long)b, R);
            const double* w = B.omega + 3 * (long long)b;
            const double* v = B.v + 3 * (long long)b;
            double Rw[3], cr[3];
            for (int d = 0; d < 3; ++d) Rw[d] = R[d][0] * w[0] + R[d][1] * w[1] + R[d][2] * w[2];
            cross_dim(DIM, r, Rw, cr);
            const double vz = DIM == 2 ? 0.0 : v[2];
            const double vv[3] = {v[0], v[1], vz};
            for (int d = 0; d < 3; ++d) AU[d] += (s == 0 ? 1.0 : -1.0) * (vv[d] - cr[d]);
            if (p.torque_free) continue;  // no lever-arm rows: the torque-free kernels do not read them
            double rn[3];
            cross_dim(DIM, r, n, rn);
            const double sg = (s == 0) ? 1.0 : -1.0;
            for (int d = 0; d < 3; ++d) arow[s][d] = sg * (R[0][d] * rn[0] + R[1][d] * rn[1] + R[2][d] * rn[2]);
            // P = R^T [r]x : P[k][l] = sum_m R[m][k] X[m][l], X = [[0,-r2,r1],[r2,0,-r0],[-r1,r0,0]]
            const double X[3][3] = {{0.0, -r[2], r[1]}, {r[2], 0.0, -r[0]}, {-r[1], r[0], 0.0}};
            for (int kk = 0; kk < 3; ++kk)
                for (int l = 0; l < 3; ++l)
                    P[s][3 * kk + l] = R[0][kk] * X[0][l] + R[1][kk] * X[1][l] + R[2][kk] * X[2][l];
        }
        double Cv[3];
        for (int d = 0; d < 3; ++d) Cv[d] = (d < DIM ? c.dij[k] * n[d] : 0.0) + p.dt * AU[d];
        if (p.problem == kFriction || p.problem == kViscousFriction) {
            for (int e = 0; e < 9; ++e) {
                a.bP[18 * (long long)k + e] = P[0][e];
                a.bP[18 * (long long)k + 9 + e] = P[1][e];
            }
        }
        if (p.problem == kFriction) {
            for (int d = 0; d < 3; ++d) a.cvec[3 * k + d] = Cv[d];
        } else if (p.problem == kViscousFriction) {
            // mode from gamma and c = global2local(C) on four slots (lagrange_multiplier.hpp:358-426)
            double cn = 0.0;
            for (int d = 0; d < DIM; ++d) cn += Cv[d] * n[d];
            const double gm = c.gamma[k];
            const int md = gm < -p.gamma_tol ? (gm != p.gamma_min ? 1 : 2) : 0;
            a.vflag[k] = md;
            double* cv = a.cvec + 4 * (long long)k;
            cv[0] = md == 2 ? -cn : cn;
            cv[1] = md == 1 ? -cn : (md == 2 ? Cv[0] : 0.0);
            cv[2] = md == 2 ? Cv[1] : 0.0;
            cv[3] = (md == 2 && DIM == 3) ? Cv[2] : 0.0;
        } else {
            double cc = 0.0;
            for (int d = 0; d < DIM; ++d) cc += Cv[d] * n[d];
            a.cvec[k] = cc;
        }
        for (int d = 0; d < 3; ++d) a.bn[3 * (long long)k + d] = n[d];
        if (!p.torque_free)
            for (int d = 0; d < 3; ++d) {
                a.bai[3 * (long long)k + d] = arow[0][d];
                a.baj[3 * (long long)k + d] = arow[1][d];
            }
        if (p.problem == kViscous) a.vflag[k] = (c.gamma[k] < -p.gamma_tol) ? 1 : 0;
    }
}

__global__ void k_viscous_slots(const Sizes* sizes, const int* scanned, const int* flag_src, int* slot) {
    const int C = sizes->C;
    GRID_STRIDE(k, C) { slot[k] = flag_src[k] ? C + scanned[k] : -1; }
}

__global__ void k_set_extra(const int* total, Sizes* sizes) {
    if (threadIdx.x == 0 && blockIdx.x == 0) sizes->n_extra = *total;
}

__global__ void k_inc_count(int nin, Contacts c, const Sizes* sizes, int* count) {
    const int C = sizes->C;
    GRID_STRIDE(k, C) {
        const int a = c.ci[k], b = c.cj[k];
        if (a >= nin) atomicAdd(&count[a - nin], 1);
        if (b >= nin) atomicAdd(&count[b - nin], 1);
    }
}

__global__ void k_inc_fill(int nin, Contacts c, const Sizes* sizes, const int* ptr, int* fill, int* idx) {
    const int C = sizes->C;
    GRID_STRIDE(k, C) {
        const int a = c.ci[k], b = c.cj[k];
        if (a >= nin) {
            const int s = atomicAdd(&fill[a - nin], 1);
            idx[ptr[a - nin] + s] = (int)k;
        }
        if (b >= nin) {
            const int s = atomicAdd(&fill[b - nin], 1);
            idx[ptr[b - nin] + s] = (int)((unsigned)k | 0x80000000u);
        }
    }
}

// sort each particle's incidences by contact index: a deterministic summation order for B^T x
__global__ void k_inc_sort(int na, const int* ptr, int* idx) {
    GRID_STRIDE(p, na) {
        const int s = ptr[p], e = ptr[p + 1];
        for (int x = s + 1; x < e; ++x) {
            const int key = idx[x];
            const unsigned kk = (unsigned)key & 0x7fffffffu;
            int y = x - 1;
            while (y >= s && ((unsigned)idx[y] & 0x7fffffffu) > kk) {
                idx[y + 1] = idx[y];
                --y;
            }
            idx[y + 1] = key;
        }
    }
}

__global__ void k_inc_coef(int na, const int* ptr, const int* idx, Assembly a, double* coef) {
    const int tot = ptr[na];
    GRID_STRIDE(k, tot) {
        const unsigned e = (unsigned)idx[k];
        const long long c = e & 0x7fffffffu;
        const bool jside = (e >> 31) != 0;
        const double sg = jside ? -1.0 : 1.0;
        const double* ar = (jside ? a.baj : a.bai) + 3 * c;
        for (int d = 0; d < 3; ++d) {
            coef[6 * (long long)k + d] = sg * a.bn[3 * c + d];
            coef[6 * (long long)k + 3 + d] = ar[d];
        }
    }
}

// update_contact_properties_impl<Viscous>, include/scopi/solvers/OptimGradient.hpp:19-35
__global__ void k_gamma_update(StepParams p, Contacts c, Assembly a, const double* lam, const Sizes* sizes) {
    const int C = sizes->C;
    GRID_STRIDE(k, C) {
        double mu = lam[k];
        if (a.slot[k] >= 0) mu = lam[k] - lam[a.slot[k]];
        double dl = 0.0;
        for (int d = 0; d < p.dim; ++d) dl += c.nij[3 * k + d] * (mu * c.nij[3 * k + d]);
        c.gamma[k] = fmin(fmax(c.gamma[k] - p.dt * dl, p.gamma_min), 0.);
    }
}

// update_contact_properties_impl<ViscousFriction>, OptimGradient.hpp:36-52: the same update
// with the force of the contact's four slots (mode in vflag: l n, (l+ - l-) n or -l0 n + f)
__global__ void k_append_links(int C, int W, const int* links, Contacts c, Sizes* sizes) {
    GRID_STRIDE(k, W) {
        c.ci[C + k] = links[k];
        c.cj[C + k] = links[k] + 1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sizes->C = C + W;
        sizes->n_links = W;
    }
}

// ---------------------------------------------------------------- periodic box
__global__ void k_ghost_flags(Bodies B, PeriodicBox box, double dmax, int dim, int* flag) {
    const int na = B.n - B.nin;
    GRID_STRIDE(t, (long long)dim * na) {
        const int d = (int)(t / na), a = B.nin + (int)(t - (long long)d * na);
        flag[t] = (box.per[d] && B.pos[3 * (long long)a + d] - dmax < box.lo[d]) ? 1 : 0;
    }
}

__global__ void k_ghost_fill(Bodies B, PeriodicBox box, int dim, GhostBodies g) {
    const int n = B.n, na = B.n - B.nin;
    GRID_STRIDE(k, n) {
        for (int d = 0; d < 3; ++d) g.pos[3 * k + d] = B.pos[3 * k + d];
        for (int d = 0; d < 4; ++d) g.q[4 * k + d] = B.q[4 * k + d];
        g.shape[k] = B.shape[k];
        g.radius[k] = B.radius[k];
        g.length[k] = B.length[k];
    }
    GRID_STRIDE(t, (long long)dim * na) {
        if (!g.flag[t]) continue;
        const int d = (int)(t / na), a = B.nin + (int)(t - (long long)d * na);
        const long long k = n + g.rank[t];
        for (int e = 0; e < 3; ++e) g.pos[3 * k + e] = B.pos[3 * (long long)a + e];
        g.pos[3 * k + d] += box.up[d] - box.lo[d];
        for (int e = 0; e < 4; ++e) g.q[4 * k + e] = B.q[4 * (long long)a + e];
        g.shape[k] = B.shape[a];
        g.radius[k] = B.radius[a];
        g.length[k] = B.length[a];
        g.src[g.rank[t]] = a;
    }
}

__global__ void k_per_classify(const Sizes* sizes, int n, const int* ci, const int* cj, int* fr, int* fg) {
    GRID_STRIDE(k, sizes->C) {
        const bool gi = ci[k] >= n, gj = cj[k] >= n;
        fr[k] = (!gi && !gj) ? 1 : 0;
        fg[k] = (!gi && gj) ? 1 : 0;
    }
}

__global__ void k_per_gather(const Sizes* sizes, int n, const int* ci, const int* cj, PeriodicScratch w,
                             const int* src) {
    GRID_STRIDE(k, sizes->C) {
        if (w.fr[k]) {
            w.r_ci[w.pr[k]] = ci[k];
            w.r_cj[w.pr[k]] = cj[k];
        }
        if (w.fg[k]) {
            w.g_ci[w.pg[k]] = ci[k];
            w.g_cj[w.pg[k]] = src[cj[k] - n];
            w.g_k[w.pg[k]] = (int)k;
        }
    }
}

__device__ __forceinline__ bool key_less(int ai, int aj, int bi, int bj) { return ai < bi || (ai == bi && aj < bj); }

// rank of each copy's pair among the copies' pairs: they come sorted by i, so its segment
// of equal i is found by binary search and ordered by (j, position) by counting
__global__ void k_per_rank(const int* totals, PeriodicScratch w) {
    const int G = totals[1];
    GRID_STRIDE(g, G) {
        const int i = w.g_ci[g], j = w.g_cj[g];
        int lo = 0, hi = (int)g;  // first index with g_ci == i
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (w.g_ci[mid] < i)
                lo = mid + 1;
            else
                hi = mid;
        }
        int r = lo;
        for (int h = lo; h < G && w.g_ci[h] == i; ++h)
            if (w.g_cj[h] < j || (w.g_cj[h] == j && h < g)) ++r;
        w.g_rank[g] = r;
        w.s_ci[r] = i;
        w.s_cj[r] = j;
    }
}

// number of keys of the sorted list (ki, kj)[0, m) below (i, j) (or not above, when `le`)
__device__ __forceinline__ int count_below(const int* ki, const int* kj, int m, int i, int j, bool le) {
    int lo = 0, hi = m;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const bool below = le ? !key_less(i, j, ki[mid], kj[mid]) : key_less(ki[mid], kj[mid], i, j);
        if (below)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void k_per_scatter(const Sizes* sizes, const int* totals, int dim, PeriodicBox box, Contacts ext,
                              Contacts out, PeriodicScratch w) {
    const int R = totals[0], G = totals[1];
    GRID_STRIDE(k, sizes->C) {
        const bool r = w.fr[k], g = w.fg[k];
        if (!r && !g) continue;
        const int i = ext.ci[k];
        int j, at;
        if (r) {
            j = ext.cj[k];
            at = w.pr[k] + count_below(w.s_ci, w.s_cj, G, i, j, false);
        } else {
            const int pg = w.pg[k];
            j = w.g_cj[pg];
            at = w.g_rank[pg] + count_below(w.r_ci, w.r_cj, R, i, j, true);
        }
        out.ci[at] = i;
        out.cj[at] = j;
        out.dij[at] = ext.dij[k];
        for (int d = 0; d < 3; ++d) {
            out.nij[3 * (long long)at + d] = ext.nij[3 * k + d];
            out.pi[3 * (long long)at + d] = ext.pi[3 * k + d];
            double pj = ext.pj[3 * k + d];
            if (g && d < dim && box.per[d]) pj -= box.up[d] - box.lo[d];
            out.pj[3 * (long long)at + d] = pj;
        }
    }
}

__global__ void k_per_size(const int* totals, Sizes* sizes) {
    if (threadIdx.x == 0 && blockIdx.x == 0) sizes->C = totals[0] + totals[1];
}

__global__ void k_transfer(StepParams p, Contacts c, const Sizes* sizes, Contacts old_c, const int* old_C) {
    const int C = sizes->C;
    const int oC = old_C ? *old_C : 0;
    GRID_STRIDE(k, C) {
        const int a = c.ci[k], b = c.cj[k];
        double gam = p.gamma0;
        if (oC > 0) {
            int lo = 0, hi = oC;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (key_less(old_c.ci[mid], old_c.cj[mid], a, b))
                    lo = mid + 1;
                else
                    hi = mid;
            }
            if (lo < oC && old_c.ci[lo] == a && old_c.cj[lo] == b) gam = old_c.gamma[lo];
        }
        c.gamma[k] = gam;
    }
}

__global__ void k_periodic_wrap(Bodies B, PeriodicBox box, int dim) {
    GRID_STRIDE(k, B.n) {
        for (int d = 0; d < dim; ++d) {
            if (!box.per[d]) continue;
            double& x = B.pos[3 * k + d];
            const bool plus = x > box.up[d], minus = x < box.lo[d];
            if (plus) x -= box.up[d] - box.lo[d];
            if (minus) x += box.up[d] - box.lo[d];
        }
    }
}

__global__ void k_gamma_update_vf(StepParams p, Contacts c, Assembly a, const double* lam, const Sizes* sizes) {
    const int C = sizes->C;
    GRID_STRIDE(k, C) {
        const double* l = lam + 4 * k;
        const int md = a.vflag[k];
        double dl = 0.0;
        for (int d = 0; d < p.dim; ++d) {
            const double nd = c.nij[3 * k + d];
            const double f = md == 0 ? l[0] * nd : (md == 1 ? (l[0] - l[1]) * nd : (-l[0]) * nd + l[1 + d]);
            dl += nd * f;
        }
        c.gamma[k] = fmin(fmax(c.gamma[k] - p.dt * dl, p.gamma_min), 0.);
    }
}

// OptimGradient::run velocity recovery (OptimGradient.hpp:265-284), update_velocity
// (solver.hpp:528-546) and move_active_particles (solver.hpp:441-480).
__global__ void k_update(Bodies B, StepParams p, const double* u, int ustride, int urot, const Sizes* sizes) {
    if (sizes && sizes->overflow) return;  // the step is redone after the buffers grow
    const bool has = (u != nullptr) && (sizes == nullptr || sizes->C > 0);
    GRID_STRIDE(k, B.n - B.nin) {
        const long long b = B.nin + k;
        double* v = B.v + 3 * b;
        double* w = B.omega + 3 * b;
        if (has) {
            const double* uk = u + (long long)ustride * k;
            for (int d = 0; d < p.dim; ++d) v[d] = v[d] + p.dt * uk[d];
            if (urot) {
                if (p.dim == 3) {
                    for (int d = 0; d < 3; ++d) w[d] = w[d] + p.dt * uk[3 + d];
                } else {
                    w[2] = w[2] + p.dt * uk[5];
                }
            }
        }
        double ww[3];
        double nw;
        if (p.dim == 2) {
            ww[0] = 0.0;
            ww[1] = 0.0;
            ww[2] = w[2];
            nw = fabs(w[2]);
        } else {
            ww[0] = w[0];
            ww[1] = w[1];
            ww[2] = w[2];
            nw = norm_n(ww, 3);
        }
        for (int d = 0; d < p.dim; ++d) B.pos[3 * b + d] += p.dt * v[d];
        rotate_body(B.q + 4 * b, ww, nw, p.dt);
    }
}

// AMatrix::mat_mult (velocities.hpp:67-144) in the reference's 6N layout (test API)
__global__ void k_amat(Bodies B, StepParams p, Contacts c, const Sizes* sizes, const double* u, double* out) {
    const int C = sizes->C;
    const long long na = B.n - B.nin, rot = 3 * na;
    GRID_STRIDE(k, C) {
        double row[3] = {0, 0, 0};
        for (int s = 0; s < 2; ++s) {
            const int b = s == 0 ? c.ci[k] : c.cj[k];
            if (b < B.nin) continue;
            const long long st = 3 * (long long)(b - B.nin);
            const double vb[3] = {u[st], u[st + 1], u[st + 2]};
            const double wb[3] = {u[st + rot], u[st + rot + 1], u[st + rot + 2]};
            const double* pt = (s == 0 ? c.pi : c.pj) + 3 * k;
            double r[3] = {0, 0, 0};
            for (int d = 0; d < p.dim; ++d) r[d] = pt[d] - B.pos[3 * (long long)b + d];
            double R[3][3];
            rotation3(B.q + 4 * (long long)b, R);
            double Rw[3], cr[3];
            for (int d = 0; d < 3; ++d) Rw[d] = R[d][0] * wb[0] + R[d][1] * wb[1] + R[d][2] * wb[2];
            cross_dim(p.dim, r, Rw, cr);
            for (int d = 0; d < 3; ++d) {
                if (s == 0)
                    row[d] += vb[d] - cr[d];
                else
                    row[d] -= vb[d] - cr[d];
            }
        }
        for (int d = 0; d < 3; ++d) out[3 * k + d] = row[d];
    }
}

// ATMatrix::mat_mult (velocities.hpp:167-254) in the reference's 6N layout (test API)
__global__ void k_atmat(Bodies B, StepParams p, Contacts c, const Sizes* sizes, const double* f, double* out) {
    const int C = sizes->C;
    const long long na = B.n - B.nin, rot = 3 * na;
    GRID_STRIDE(k, C) {
        const double fc[3] = {f[3 * k], f[3 * k + 1], f[3 * k + 2]};
        for (int s = 0; s < 2; ++s) {
            const int b = s == 0 ? c.ci[k] : c.cj[k];
            if (b < B.nin) continue;
            const long long st = 3 * (long long)(b - B.nin);
            const double* pt = (s == 0 ? c.pi : c.pj) + 3 * k;
            double r[3] = {0, 0, 0};
            for (int d = 0; d < p.dim; ++d) r[d] = pt[d] - B.pos[3 * (long long)b + d];
            double R[3][3];
            rotation3(B.q + 4 * (long long)b, R);
            double cr[3];
            cross_dim(p.dim, r, fc, cr);
            const double sg = s == 0 ? 1.0 : -1.0;
            for (int d = 0; d < 3; ++d) {
                const double res = R[0][d] * cr[0] + R[1][d] * cr[1] + R[2][d] * cr[2];
                atomicAdd(&out[st + d], sg * fc[d]);
                atomicAdd(&out[st + rot + d], sg * res);
            }
        }
    }
}

int blocks_for(long long n, int per = kThreads) {
    long long b = (n + per - 1) / per;
    if (b < 1) b = 1;
    const long long cap = 16LL * kSMs;
    return (int)(b < cap ? b : cap);
}

}  // namespace

void launch_obstacles_move(const Bodies& b, double dt, int dim, cudaStream_t s) {
    if (b.nin <= 0) return;
    k_obstacles_move<<<blocks_for(b.nin), kThreads, 0, s>>>(b, dt, dim);
    LAUNCHED(1);
}

void launch_vap(const Bodies& b, const StepParams& p, cudaStream_t s, const Sizes* sizes) {
    if (b.n - b.nin <= 0) return;
    k_vap<<<blocks_for(b.n - b.nin), kThreads, 0, s>>>(b, p, sizes);
    LAUNCHED(1);
}

void launch_detect(const Bodies& b, const StepParams& p, DetectWork& w, Contacts& out, Sizes* sizes, long long c_cap,
                   cudaStream_t s) {
    const int na = b.n - b.nin;
    cudaMemsetAsync(w.tmp_total, 0, 4 * sizeof(int), s);
    // uniform grid over the active particles
    k_bbox_partial<<<kBBoxBlocks, kThreads, 0, s>>>(b, p.dim, w.bbox_partial);
    k_grid_setup<<<1, 32, 0, s>>>(w.bbox_partial, kBBoxBlocks, p.dim, p.dmax, w.cell_cap, na, w.grid);
    cudaMemsetAsync(w.cell_count, 0, (w.cell_cap + 1) * sizeof(int), s);
    cudaMemsetAsync(w.cell_fill, 0, w.cell_cap * sizeof(int), s);
    LAUNCHED(2);
    if (na > 0) {
        k_cell_assign<<<blocks_for(na), kThreads, 0, s>>>(b, p.dim, w.grid, w.cell_of, w.cell_count);
        scan_exclusive(w.cell_count, w.cell_start, &w.grid->ncell1, 0, w.cell_cap + 1, w.tmp_total + 3, w.scan_work, s,
                       &g_detect_launches);
        const bool by_cell = p.dim == 3;  // 3D: a warp per occupied cell; 2D: a thread per body
        cudaMemsetAsync(w.n_occ, 0, sizeof(int), s);
        k_cell_scatter<<<blocks_for(na), kThreads, 0, s>>>(b, w.cell_of, w.cell_start, w.cell_fill, w.cell_body,
                                                           w.cell_pr, by_cell ? w.occ : nullptr, w.n_occ);
        cudaMemsetAsync(w.row_count, 0, (na + 1) * sizeof(int), s);
        if (by_cell)
            k_pair_search_cells<3><<<blocks_for(na, kSearchWarps), 32 * kSearchWarps, 0, s>>>(
                b, p, w.grid, w.cell_start, w.cell_body, w.cell_pr, w.occ, w.n_occ, w.row_count, w.row_tmp);
        else
            k_pair_search<2><<<blocks_for(na), kThreads, 0, s>>>(b, p, w.grid, w.cell_of, w.cell_start, w.cell_body,
                                                                w.cell_pr, w.row_count, w.row_tmp);
        LAUNCHED(3);
    }
    // obstacle rows come first in (i, j) order
    const long long nobs = w.obs_cap;  // nin * na, or the sum of the per-obstacle ranges of a batch
    if (nobs > 0) {
        const bool se = b.axes != nullptr;
        if (p.dim == 3) {
            if (se)
                k_obs_flags<3, true><<<blocks_for(nobs), kThreads, 0, s>>>(b, p, nobs, w.obs_flag);
            else
                k_obs_flags<3, false><<<blocks_for(nobs), kThreads, 0, s>>>(b, p, nobs, w.obs_flag);
        } else {
            if (se)
                k_obs_flags<2, true><<<blocks_for(nobs), kThreads, 0, s>>>(b, p, nobs, w.obs_flag);
            else
                k_obs_flags<2, false><<<blocks_for(nobs), kThreads, 0, s>>>(b, p, nobs, w.obs_flag);
        }
        scan_exclusive(w.obs_flag, w.obs_pos, nullptr, (int)nobs, nobs, w.tmp_total + 0, w.scan_work, s,
                       &g_detect_launches);
        LAUNCHED(1);
    }
    k_set_cobs<<<1, 1, 0, s>>>(w.tmp_total, sizes);
    LAUNCHED(1);
    if (na > 0) {
        scan_exclusive(w.row_count, w.row_ptr, nullptr, na + 1, na + 1, w.tmp_total + 1, w.scan_work, s,
                       &g_detect_launches);
    }
    k_sizes<<<1, 1, 0, s>>>(w.tmp_total, sizes, c_cap);
    LAUNCHED(1);
    if (nobs > 0) {
        k_obs_fill<<<blocks_for(nobs), kThreads, 0, s>>>(b, nobs, w.obs_flag, w.obs_pos, c_cap, out.ci, out.cj);
        LAUNCHED(1);
    }
    if (na > 0) {
        if (p.dim == 3)
            k_pair_compact<3><<<blocks_for(na), kThreads, 0, s>>>(b, p, w.grid, w.cell_of, w.cell_start, w.cell_body,
                                                                  w.cell_pr, w.row_count, w.row_tmp, w.row_ptr, sizes,
                                                                  c_cap, out.ci, out.cj);
        else
            k_pair_compact<2><<<blocks_for(na), kThreads, 0, s>>>(b, p, w.grid, w.cell_of, w.cell_start, w.cell_body,
                                                                  w.cell_pr, w.row_count, w.row_tmp, w.row_ptr, sizes,
                                                                  c_cap, out.ci, out.cj);
        k_row_sort<<<blocks_for(na), kThreads, 0, s>>>(na, w.row_ptr, sizes, c_cap, out.cj);
        LAUNCHED(2);
    }
}

void launch_geometry(const Bodies& b, const StepParams& p, Contacts& c, const Sizes* sizes, long long c_cap,
                     const Contacts* old_c, const int* old_C, long long, cudaStream_t s, int* need_se) {
    Contacts oc{};
    if (old_c) oc = *old_c;
    const int* oC = old_c ? old_C : nullptr;
    const int blocks = blocks_for(c_cap);
    if (b.axes) {
        if (p.dim == 3)
            k_geometry<3, true><<<blocks, kThreads, 0, s>>>(b, p, c, sizes, oc, oC, need_se);
        else
            k_geometry<2, true><<<blocks, kThreads, 0, s>>>(b, p, c, sizes, oc, oC, need_se);
    } else {
        if (p.dim == 3)
            k_geometry<3, false><<<blocks, kThreads, 0, s>>>(b, p, c, sizes, oc, oC, nullptr);
        else
            k_geometry<2, false><<<blocks, kThreads, 0, s>>>(b, p, c, sizes, oc, oC, nullptr);
    }
    LAUNCHED(1);
}

void launch_assemble(const Bodies& b, const StepParams& p, const Contacts& c, Assembly& a, Sizes* sizes,
                     long long c_cap, int* scan_work, int* tmp_total, cudaStream_t s) {
    if (p.dim == 3)
        k_assemble<3><<<blocks_for(c_cap), kThreads, 0, s>>>(b, p, c, a, sizes);
    else
        k_assemble<2><<<blocks_for(c_cap), kThreads, 0, s>>>(b, p, c, a, sizes);
    LAUNCHED(1);
    if (p.problem == kViscous) {
        scan_exclusive(a.vflag, a.slot, &sizes->C, 0, c_cap, tmp_total, scan_work, s, &g_detect_launches);
        // slot holds the exclusive scan; turn it into C + rank (flagged) or -1
        k_viscous_slots<<<blocks_for(c_cap), kThreads, 0, s>>>(sizes, a.slot, a.vflag, a.slot);
        k_set_extra<<<1, 1, 0, s>>>(tmp_total, sizes);
        LAUNCHED(2);
    }
}

void launch_incidence(const Bodies& b, const StepParams& p, const Contacts& c, const Assembly& a, Incidence& inc,
                      const Sizes* sizes, long long c_cap, int* scan_work, int* tmp_total, cudaStream_t s,
                      bool with_coef) {
    const int na = b.n - b.nin;
    if (na <= 0) return;
    cudaMemsetAsync(inc.count, 0, (na + 1) * sizeof(int), s);
    cudaMemsetAsync(inc.jcount, 0, (na + 1) * sizeof(int), s);
    k_inc_count<<<blocks_for(c_cap), kThreads, 0, s>>>(b.nin, c, sizes, inc.count);
    scan_exclusive(inc.count, inc.ptr, nullptr, na + 1, na + 1, tmp_total, scan_work, s, &g_detect_launches);
    k_inc_fill<<<blocks_for(c_cap), kThreads, 0, s>>>(b.nin, c, sizes, inc.ptr, inc.jcount, inc.idx);
    k_inc_sort<<<blocks_for(na), kThreads, 0, s>>>(na, inc.ptr, inc.idx);
    LAUNCHED(3);
    if (with_coef && p.problem != kFriction && p.problem != kViscousFriction) {
        k_inc_coef<<<blocks_for(2 * c_cap), kThreads, 0, s>>>(na, inc.ptr, inc.idx, a, inc.coef);
        LAUNCHED(1);
    }
}

void launch_append_links(int C, int W, const int* links, Contacts& c, Sizes* sizes, cudaStream_t s) {
    k_append_links<<<blocks_for(W), kThreads, 0, s>>>(C, W, links, c, sizes);
    LAUNCHED(1);
}

void launch_ghost_flags(const Bodies& b, const PeriodicBox& box, double dmax, int dim, GhostBodies& g, int* total,
                        int* scan_work, cudaStream_t s) {
    const long long m = (long long)dim * (b.n - b.nin);
    cudaMemsetAsync(total, 0, sizeof(int), s);  // an empty scan (no active body) leaves it alone
    k_ghost_flags<<<blocks_for(m + 1), kThreads, 0, s>>>(b, box, dmax, dim, g.flag);
    LAUNCHED(1);
    scan_exclusive(g.flag, g.rank, nullptr, (int)m, m, total, scan_work, s, &g_detect_launches);
}

Bodies launch_ghost_fill(const Bodies& b, const PeriodicBox& box, int dim, int n_ghosts, GhostBodies& g,
                         cudaStream_t s) {
    const long long m = std::max<long long>((long long)dim * (b.n - b.nin), b.n);
    k_ghost_fill<<<blocks_for(m), kThreads, 0, s>>>(b, box, dim, g);
    LAUNCHED(1);
    Bodies e = b;
    e.n = b.n + n_ghosts;
    e.pos = g.pos;
    e.q = g.q;
    e.shape = g.shape;
    e.radius = g.radius;
    e.length = g.length;
    return e;
}

void launch_periodic_remap(int n, int dim, const PeriodicBox& box, const GhostBodies& g, const Contacts& ext,
                           Contacts& out, PeriodicScratch& w, Sizes* sizes, long long c_cap, int* totals,
                           int* scan_work, cudaStream_t s) {
    k_per_classify<<<blocks_for(c_cap), kThreads, 0, s>>>(sizes, n, ext.ci, ext.cj, w.fr, w.fg);
    scan_exclusive(w.fr, w.pr, &sizes->C, 0, c_cap, totals + 0, scan_work, s, &g_detect_launches);
    scan_exclusive(w.fg, w.pg, &sizes->C, 0, c_cap, totals + 1, scan_work, s, &g_detect_launches);
    k_per_gather<<<blocks_for(c_cap), kThreads, 0, s>>>(sizes, n, ext.ci, ext.cj, w, g.src);
    k_per_rank<<<blocks_for(c_cap), kThreads, 0, s>>>(totals, w);
    k_per_scatter<<<blocks_for(c_cap), kThreads, 0, s>>>(sizes, totals, dim, box, ext, out, w);
    k_per_size<<<1, 1, 0, s>>>(totals, sizes);
    LAUNCHED(5);
}

void launch_transfer(const StepParams& p, Contacts& c, const Sizes* sizes, const Contacts& old, const int* old_C,
                     long long c_cap, cudaStream_t s) {
    k_transfer<<<blocks_for(c_cap), kThreads, 0, s>>>(p, c, sizes, old, old_C);
    LAUNCHED(1);
}

void launch_periodic_wrap(const Bodies& b, const PeriodicBox& box, int dim, cudaStream_t s) {
    k_periodic_wrap<<<blocks_for(b.n), kThreads, 0, s>>>(b, box, dim);
    LAUNCHED(1);
}

void launch_gamma_update(const StepParams& p, Contacts& c, const Assembly& a, const double* lambda, const Sizes* sizes,
                         long long c_cap, cudaStream_t s) {
    if (p.problem == kViscousFriction)
        k_gamma_update_vf<<<blocks_for(c_cap), kThreads, 0, s>>>(p, c, a, lambda, sizes);
    else
        k_gamma_update<<<blocks_for(c_cap), kThreads, 0, s>>>(p, c, a, lambda, sizes);
    LAUNCHED(1);
}

void launch_update(const Bodies& b, const StepParams& p, const double* u, int ustride, int urot, const Sizes* sizes,
                   cudaStream_t s) {
    if (b.n - b.nin <= 0) return;
    k_update<<<blocks_for(b.n - b.nin), kThreads, 0, s>>>(b, p, u, ustride, urot, sizes);
    LAUNCHED(1);
}

void launch_amat(const Bodies& b, const StepParams& p, const Contacts& c, const Sizes* sizes, long long c_cap,
                 const double* u, double* out, cudaStream_t s) {
    k_amat<<<blocks_for(c_cap), kThreads, 0, s>>>(b, p, c, sizes, u, out);
    LAUNCHED(1);
}

void launch_atmat(const Bodies& b, const StepParams& p, const Contacts& c, const Sizes* sizes, long long c_cap,
                  const double* f, double* out, cudaStream_t s) {
    cudaMemsetAsync(out, 0, 6 * (size_t)(b.n - b.nin) * sizeof(double), s);
    k_atmat<<<blocks_for(c_cap), kThreads, 0, s>>>(b, p, c, sizes, f, out);
    LAUNCHED(1);
}

}  // namespace scopi_gpu
