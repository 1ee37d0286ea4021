/*
 * scopi_oracle.h -- CPU restatement of the SCoPI per-time-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the CUDA path is
 * compared against (tests/, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py).  Nothing in the product (scopi_b200/) links, loads or calls it.
 *
 * It restates, in plain C++17 without xtensor/nanoflann/BLAS, the reference
 * hpc-maths/scopi v0.1.0 algorithm for one time step:
 *   ScopiSolver::run loop body           include/scopi/solver.hpp:274-302
 *   displacement_obstacles               include/scopi/solver.hpp:330-355
 *   contact_brute_force / contact_kdtree include/scopi/contact/contact_brute_force.hpp:104-136,
 *                                        include/scopi/contact/contact_kdtree.hpp:202-268
 *   compute_exact_distance, sort         include/scopi/contact/base.hpp:104-175
 *   closest points sphere/plane/segment  include/scopi/objects/methods/closest_points.hpp:36-50,768-881
 *   A, A^T, D, M^-1, c, Q                include/scopi/matrix/velocities.hpp:67-296,
 *                                        include/scopi/solvers/minimization_problem.hpp:11-161
 *   Lagrange multipliers / projections   include/scopi/solvers/lagrange_multiplier.hpp:44-273
 *   apgd (dynamic_descent)               include/scopi/solvers/apgd.hpp:148-221
 *   OptimGradient::run, viscous gamma    include/scopi/solvers/OptimGradient.hpp:19-35,253-306
 *   vap_fixed / vap_fpd                  include/scopi/vap/vap_fixed.hpp:45-55, vap_fpd.hpp:69-81,
 *                                        src/vap/vap_fpd.cpp:6-26
 *   update_velocity / move_active        include/scopi/solver.hpp:441-546
 *   quaternion helpers                   src/quaternion.cpp:6-120, include/scopi/quaternion.hpp:66-124
 *
 * Pinned against the reference's own golden files and known-answer tests
 * (tests/golden/, tests/test_oracle_golden.py).
 *
 * Conventions (shared with the CUDA C-ABI, include/scopi_gpu.h):
 *   every vector quantity has 3 slots; in 2D the z slot of pos/v/vd/f is 0 and
 *   the scalar rotation quantities (omega, desired omega, moment of inertia)
 *   live in the z slot of their 3-vectors.  Obstacles (inactive bodies) come
 *   first.  Quaternions are (w, x, y, z) as in the reference.
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_SPHERE = 0, ORC_PLANE = 1, ORC_SEGMENT = 2, ORC_SUPERELLIPSOID = 3 };
enum { ORC_NOFRICTION = 0, ORC_FRICTION = 1, ORC_VISCOUS = 2, ORC_FRICTION_FIXED_POINT = 3,
       ORC_VISCOUS_FRICTION = 4 };
enum { ORC_VAP_FIXED = 0, ORC_VAP_FPD = 1 };
enum { ORC_BRUTE_FORCE = 0, ORC_KDTREE = 1 };

typedef struct {
    int32_t dim;
    int32_t problem;          /* ORC_NOFRICTION / FRICTION / VISCOUS / FRICTION_FIXED_POINT / VISCOUS_FRICTION */
    int32_t vap;              /* ORC_VAP_FIXED / ORC_VAP_FPD */
    int32_t contact_method;   /* ORC_BRUTE_FORCE / ORC_KDTREE */
    double dmax;              /* ContactsParams::dmax (default 2) */
    double kd_tree_radius;    /* squared candidate radius (default 17) */
    double alpha;             /* apgd_params (0.05, 10000, 1e-7, true) */
    int64_t max_ite;
    double tolerance;
    int32_t dynamic_descent;
    double mu;                /* contact_property<Friction>::mu (0.1) */
    double gamma;             /* contact_property<Viscous> (0, -2, 1e-6) */
    double gamma_min;
    double gamma_tol;
    int32_t num_threads;      /* OpenMP threads for the loops the reference parallelises (0 = default) */
    double fixed_point_tol;   /* contact_property<FixedPoint> (1e-6, 1000): FrictionFixedPoint, ViscousFriction */
    int64_t fixed_point_max_iter;
    double box_lower[3];      /* BoxDomain<dim> (box.hpp): corners, and the periodic axes (none: */
    double box_upper[3];      /* no box); an obstacle within dmax of a periodic lower bound makes */
    int32_t periodic[3];      /* orc_run fail (the reference pairs it with its own ghost) */
} orc_params;

typedef struct {
    int64_t n;                /* number of bodies */
    int64_t nb_inactive;      /* obstacles first */
    int32_t* shape;           /* n */
    double* pos;              /* n*3 */
    double* q;                /* n*4 */
    double* v;                /* n*3 */
    double* omega;            /* n*3 */
    double* vd;               /* n*3 */
    double* omega_d;          /* n*3 */
    double* f;                /* n*3 */
    double* m;                /* n   */
    double* j;                /* n*3 */
    double* radius;           /* n   (sphere radius; bounding radius of a superellipsoid) */
    double* length;           /* n   (segment length) */
    double* axes;             /* n*3 superellipsoid semi-axes (may be NULL without superellipsoids) */
    double* squareness;       /* n*2 superellipsoid squareness (e, n) */
    int32_t* worm;            /* n: index of the worm a sphere belongs to, -1 if none (may be NULL);
                                 worms need the NoFriction problem */
} orc_particles;

typedef struct {
    int64_t contacts;
    int64_t iterations;       /* APGD iterations of the last solve */
    int64_t backtracks;
    int64_t restarts;
    int32_t converged;
    double violation;         /* max_c max(0, -(d_c + dt n_c.(A u)_c)) after the solve */
    double seconds_contacts, seconds_solve, seconds_other;
    int64_t fixed_point_iterations; /* FrictionFixedPoint, ViscousFriction: solves of the last step */
} orc_stats;

typedef struct orc_solver orc_solver;

orc_solver* orc_create(const orc_params* p, const orc_particles* parts);
void orc_destroy(orc_solver* s);
/* ScopiSolver::run(dt, total_it, initial_iter) with output disabled. */
int orc_run(orc_solver* s, double dt, int64_t total_it, int64_t initial_iter);
int orc_get_particles(const orc_solver* s, orc_particles* out);
int orc_set_particles(orc_solver* s, const orc_particles* in);
/* Contacts of the last step, sorted by (i, j): i, j, dij, nij(3), pi(3), pj(3), gamma. */
int64_t orc_num_contacts(const orc_solver* s);
int64_t orc_get_contacts(const orc_solver* s, int64_t* ci, int64_t* cj, double* dij, double* nij,
                         double* pi, double* pj, double* gamma, int64_t cap);
/* Lagrange multiplier of the last solve, in the reference's local layout. */
int64_t orc_get_lambda(const orc_solver* s, double* out, int64_t cap);
int orc_get_stats(const orc_solver* s, orc_stats* out);
/* Contact detection alone on the current particle state (sorted). */
int64_t orc_detect(orc_solver* s);
/* Closest points of two 3D superellipsoids / a superellipsoid and a plane, as the contact
   list would record them (closest_points.hpp:263-733, 1479-1768).  A body is
   {c[3], q[4] (w, x, y, z), r[3], e, n}; a plane {c[3], q[4]}.  out = pi[3], pj[3], nij[3],
   dij, u[4] (the solver's unknowns), function evaluations; returns the solver's info (0 for
   the closed-form superellipsoid-plane case). */
int orc_se_se(const double* s1, const double* s2, double* out);
int orc_se_plane(const double* s, const double* plane, double* out);
/* The hybrid method alone from the start u (in/out); returns info, *nfev its function count. */
int orc_se_se_hybrid(const double* s1, const double* s2, double* u, int* nfev);
/* start of the SE-SE solve: the grid argmin of closest_points.hpp:604-668 (angles a1, b1, a2, b2) */
void orc_se_se_start(const double* s1, const double* s2, double* u0);
/* the start criterion |p1 - p2| + 2 (1 + n1.n2) at angles u (closest_points.hpp:654-660) */
double orc_se_se_start_value(const double* s1, const double* s2, const double* u);
/* the SE-SE closest points with the solve started from u0 instead of the grid argmin */
int orc_se_se_from(const double* s1, const double* s2, const double* u0, double* out);
/* F and the analytic Jacobian (column-major) of the SE-SE system at u, for cross-checks;
   the SE-plane residual (with the body's side as its sign) at u = (a, b, plane coords). */
void orc_se_plane_residual(const double* s, const double* plane, const double* u, double* F);
void orc_se_se_system(const double* s1, const double* s2, const double* u, double* F, double* J);
/* 2D: closest_points(superellipsoid<2>, superellipsoid<2>) on the same body records (c[0..1],
   rotation about z, r[0..1], e); u = (b1, b2); F (2), J (2x2 column-major). */
int orc_se2_se2(const double* s1, const double* s2, double* out);
int orc_se2_hybrid(const double* s1, const double* s2, double* u, int* nfev);
void orc_se2_system(const double* s1, const double* s2, const double* u, double* F, double* J);
// closest_points(sphere, superellipsoid) (closest_points.hpp:944-1302, 1316-1463): sph =
// (centre[3], quaternion[4], radius); reference_labels = 1 gives the reference's own result
// (pi on the superellipsoid, nij the sphere's normal, the Newton method alone), 0 the engine's
// pair (the Newton method, the hybrid method where it fails) labelled by body with the
// superellipsoid as body i when se_is_i; out as orc_se_se, out[15] = the solve's status (the
// Newton method's iterations, -1 at its cap, -2 singular; 100 + the hybrid method's info)
int orc_sphere_se(int dim, const double* se, const double* sph, int reference_labels, int se_is_i, double* out);
// closest_points(superellipsoid<2>, plane<2>) in closed form; out as orc_se_se
int orc_se2_plane(const double* s, const double* plane, double* out);
// the Newton method's linear solve (dgesv restated) for a column-major 4 x 4 system
int orc_lu_solve4(const double* A, const double* b, double* x);
/* A.u and A^T.f on the current contact list (3C and 6*na long vectors). */
int orc_amat(const orc_solver* s, const double* u, double* out);
int orc_atmat(const orc_solver* s, const double* f, double* out);

#ifdef __cplusplus
}
#endif
