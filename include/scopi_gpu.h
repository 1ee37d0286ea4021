/*
 * scopi_gpu.h -- C ABI of the B200 (sm_100a) SCoPI time-step engine.
 *
 * One handle = one ScopiSolver<dim, problem, OptimGradient<apgd>, contact, vap>
 * (include/scopi/solver.hpp:91-206 of hpc-maths/scopi v0.1.0) whose particles
 * live in GPU memory.  A step runs, on the device: obstacle motion, contact
 * detection (uniform-grid cell list, contact set identical to the reference's
 * kd-tree / brute force), closest points and contact-Jacobian assembly, the
 * APGD solve (FP64, or FP32 iterations with an FP64 outer correction), the
 * velocity update and the position/quaternion integration.
 *
 * Conventions: plain C types only, no exceptions across the ABI; every function
 * returns 0 on success or a negative SCOPI_GPU_E* code, and scopi_gpu_last_error()
 * gives a message.  The caller owns host buffers; the handle owns device memory
 * and one CUDA stream.  One host thread per handle.
 *
 * Particle layout (host and device): every vector has 3 slots per body.  In 2D the
 * z slot of pos/v/vd/f is 0 and the scalar rotation quantities (omega, desired
 * omega, moment of inertia) live in the z slot.  Quaternions are (w, x, y, z).
 * Obstacles (inactive bodies) come first, as scopi_container requires
 * (include/scopi/container.hpp:365-373).
 */
#ifndef SCOPI_GPU_H
#define SCOPI_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* error codes */
#define SCOPI_GPU_OK 0
#define SCOPI_GPU_EINVAL -1      /* bad argument */
#define SCOPI_GPU_ECUDA -2       /* CUDA runtime error (message in last_error) */
#define SCOPI_GPU_ENOMEM -3      /* device allocation failed */
#define SCOPI_GPU_EUNSUPPORTED -4 /* shape pair / option the reference does not implement */
#define SCOPI_GPU_ETIMEOUT -5    /* a device-side bounded wait gave up (grid barrier) */
#define SCOPI_GPU_ENOCONV 1      /* positive: APGD reached max_ite ("APGD didn't converge.") */

/* problem_t (include/scopi/contact/property.hpp:14-36) */
#define SCOPI_GPU_NOFRICTION 0
#define SCOPI_GPU_FRICTION 1
#define SCOPI_GPU_VISCOUS 2
/* FrictionFixedPoint (property.hpp:26, OptimGradient.hpp:85-176): the Friction problem with
   the linear term c + s_c n_c, s_c = mu dt |tangential relative velocity| updated after
   each solve until the fixed point (fixed_point_tol, fixed_point_max_iter) */
#define SCOPI_GPU_FRICTION_FIXED_POINT 3
/* ViscousFriction (property.hpp:34, lagrange_multiplier.hpp:347-541, OptimGradient.hpp:36-52,
   96-107, 178-250): per contact 1, 2 or 4 multipliers by its adhesion potential gamma
   (gamma >= -gamma_tol: normal; gamma_min < gamma < -gamma_tol: the viscous pair; gamma ==
   gamma_min: a normal multiplier and a friction-cone force, projected onto the nearer of the
   two), the linear term dt mu s_c n_c on the friction force, s_c = |tangential relative
   velocity| updated after each solve until the fixed point (fixed_point_tol,
   fixed_point_max_iter); gamma updated after the step */
#define SCOPI_GPU_VISCOUS_FRICTION 4
/* vap policies (include/scopi/vap/vap_fixed.hpp, vap_fpd.hpp) */
#define SCOPI_GPU_VAP_FIXED 0
#define SCOPI_GPU_VAP_FPD 1
/* contact policies (contact/contact_brute_force.hpp, contact/contact_kdtree.hpp) */
#define SCOPI_GPU_BRUTE_FORCE 0
#define SCOPI_GPU_KDTREE 1
/* precision of the APGD iterations */
#define SCOPI_GPU_FP64 0
#define SCOPI_GPU_MIXED 1
/* shapes */
#define SCOPI_GPU_SPHERE 0
#define SCOPI_GPU_PLANE 1
#define SCOPI_GPU_SEGMENT 2
#define SCOPI_GPU_SUPERELLIPSOID 3  /* superellipsoid<dim> (superellipsoid.hpp:59-70); 2D scenes
                                       of superellipsoids take no obstacles */

typedef struct scopi_gpu_params {
    int32_t dim;              /* 2 or 3 */
    int32_t problem;          /* SCOPI_GPU_NOFRICTION / FRICTION / VISCOUS / FRICTION_FIXED_POINT /
                                 VISCOUS_FRICTION */
    int32_t vap;              /* SCOPI_GPU_VAP_FIXED / VAP_FPD */
    int32_t contact_method;   /* SCOPI_GPU_BRUTE_FORCE / KDTREE */
    int32_t precision;        /* SCOPI_GPU_FP64 / SCOPI_GPU_MIXED */
    int32_t dynamic_descent;  /* apgd_params::dynamic_descent (apgd.hpp:123) */
    int64_t max_ite;          /* apgd_params::max_ite (apgd.hpp:121) */
    double dmax;              /* ContactsParams::dmax (contact_kdtree.hpp:229) */
    double kd_tree_radius;    /* ContactsParams::kd_tree_radius, squared (contact_kdtree.hpp:237) */
    double alpha;             /* apgd_params::alpha (apgd.hpp:120) */
    double tolerance;         /* apgd_params::tolerance (apgd.hpp:122) */
    double mu;                /* contact_property<Friction>::mu (property.hpp:72) */
    double gamma;             /* contact_property<Viscous> (property.hpp:125-127) */
    double gamma_min;
    double gamma_tol;
    double mixed_violation_tol;   /* MIXED: FP64 constraint violation the outer correction must reach */
    int32_t mixed_max_corrections;/* MIXED: FP32 correction solves after the first one */
    int32_t device;               /* CUDA device ordinal */
    int32_t initial_step;         /* SCOPI_GPU_STEP_AUTO / _REFERENCE / _CURVATURE (below) */
    double fixed_point_tol;       /* contact_property<FixedPoint> (property.hpp:93-94): 1e-6 */
    int64_t fixed_point_max_iter; /* and 1000 solves at most per step */
    double box_lower[3];          /* BoxDomain<dim> (box.hpp): corners and periodic axes (0/1); */
    double box_upper[3];          /* with no periodic axis there is no box.  Each step the active */
    int32_t periodic[3];          /* spheres within dmax of a periodic lower bound are copied shifted
                                     by upper - lower into the contact search; a contact with a copy
                                     takes its body's index and its closest point moved back by
                                     upper - lower on every periodic axis; after the move a body
                                     beyond a bound is wrapped (utils.hpp:229-257, base.hpp:118-137,
                                     solver.hpp:482-522).  Scenes of spheres (planes and segments as
                                     static obstacles away from the periodic lower bounds) */
    int32_t barrier_timeout_us;   /* limit of every wait on a grid barrier inside a persistent APGD
                                     launch, in microseconds (0: 20 s).  A block that waits longer
                                     sets an error word and every block returns; the step then
                                     fails with SCOPI_GPU_ETIMEOUT and the handle stays usable.
                                     Infrastructure of this library: the reference solves on the
                                     host and has no device waits. */
} scopi_gpu_params;

/* First APGD step of every solve.  REFERENCE: alpha as given (apgd.hpp:120, the
   reference's fixed 0.05), grown by 1/0.97 per accepted iteration.  CURVATURE: 1/L with
   L = 1.5 x the Rayleigh quotient d^T Q d / |d|^2 along the first projected-gradient
   direction d (one extra particle pass per solve).  AUTO: REFERENCE for FP64 (the drop-in,
   same iterates as the reference), CURVATURE for MIXED. */
#define SCOPI_GPU_STEP_AUTO (-1)
#define SCOPI_GPU_STEP_REFERENCE 0
#define SCOPI_GPU_STEP_CURVATURE 1

typedef struct scopi_gpu_particles {
    int64_t n;           /* bodies */
    int64_t nb_inactive; /* obstacles first */
    int32_t* shape;      /* n: SCOPI_GPU_SPHERE / PLANE / SEGMENT / SUPERELLIPSOID */
    double* pos;         /* n*3 */
    double* q;           /* n*4 */
    double* v;           /* n*3 */
    double* omega;       /* n*3 */
    double* vd;          /* n*3 */
    double* omega_d;     /* n*3 */
    double* f;           /* n*3 */
    double* m;           /* n */
    double* j;           /* n*3 */
    double* radius;      /* n (sphere radius; superellipsoid: bounding radius |semi-axes|) */
    double* length;      /* n (segment length) */
    double* axes;        /* n*3 superellipsoid semi-axes (rx, ry, rz); 2D: (rx, ry, unused);
                            NULL when there are none */
    double* squareness;  /* n*2 superellipsoid squareness (e, n); 2D: (e, unused); NULL when
                            there are none */
    int32_t* worm;       /* n: index of the worm<dim> (objects/types/worm.hpp) an active sphere
                            belongs to, -1 if none; NULL when there are none.  A worm is a run of
                            consecutive bodies with the same index; each step appends, after the
                            sorted contacts, the contacts of its consecutive spheres with normal
                            and distance negated (add_contact.hpp:11-28).  NoFriction only. */
} scopi_gpu_particles;

typedef struct scopi_gpu_stats {
    int64_t contacts;        /* contacts of the last step */
    int64_t iterations;      /* APGD iterations of the last step (all solves) */
    int64_t backtracks;      /* Lipschitz doublings */
    int64_t restarts;        /* gradient restarts */
    int64_t fp32_iterations; /* MIXED: iterations run in FP32 */
    int64_t corrections;     /* MIXED: FP32 correction solves */
    int32_t converged;       /* 1 if the stopping test was met */
    int32_t status;          /* SCOPI_GPU_OK / ENOCONV / ETIMEOUT of the last step */
    double violation;        /* max_c max(0, -(d_c + dt n_c.(A u)_c)) after the solve (FP64) */
    double ms_step;          /* device time of the last step (CUDA events) */
    double ms_solve;         /* device time of the APGD part of the last step */
    double ms_apgd_kernel;   /* device time of the persistent APGD launches of the last step */
    int64_t steps;           /* steps run by this handle */
    int64_t fixed_point_iterations; /* FRICTION_FIXED_POINT, VISCOUS_FRICTION: solves of the last step */
} scopi_gpu_stats;

typedef struct scopi_gpu_handle scopi_gpu_handle;

/* Reference defaults: apgd (0.05, 10000, 1e-7, true), dmax 2, kd radius 17, mu 0.1,
   gamma (0, -2, 1e-6), NoFriction, vap_fixed, kd-tree, FP64. */
void scopi_gpu_default_params(scopi_gpu_params* p, int32_t dim);

/* ScopiSolver(particles) constructor, solver.hpp:117-126, with the policies' params
   (apgd.hpp:105-124, contact_kdtree.hpp:203-238, property.hpp:41-128). */
int32_t scopi_gpu_create(const scopi_gpu_params* p, scopi_gpu_handle** out);
int32_t scopi_gpu_destroy(scopi_gpu_handle* h);

/* Upload / download the whole container (scopi_container::push_back, container.hpp:339-384,
   and the pos()/q()/v()/omega() accessors).  set_particles keeps the previous contacts
   (and their viscous gamma) so a run can continue after changing forces. */
int32_t scopi_gpu_set_particles(scopi_gpu_handle* h, const scopi_gpu_particles* parts);
int32_t scopi_gpu_get_particles(scopi_gpu_handle* h, scopi_gpu_particles* out);

/* Write the fields a time step updates back into the container already on the device: the
   writable pos()/q()/v()/omega() accessors of scopi_container (container.hpp:129,138,174,183)
   used between two ScopiSolver::run calls.  parts->n and parts->nb_inactive must equal the
   last set_particles' counts; pos, q, v and omega are copied where non-NULL, every other
   field of parts is ignored (shapes, masses, forces and desired velocities stay those of the
   last set_particles; change them with set_particles).  The previous contacts are kept, as
   with set_particles.  The copies are enqueued on the handle's stream and the call returns
   after they complete.  Batch handles and handles without particles return SCOPI_GPU_EINVAL. */
int32_t scopi_gpu_set_state(scopi_gpu_handle* h, const scopi_gpu_particles* parts);

/* ScopiSolver::run(dt, total_it, initial_iter), solver.hpp:267-303 (output disabled). */
int32_t scopi_gpu_run(scopi_gpu_handle* h, double dt, int64_t total_it, int64_t initial_iter);

/* contact_base::run (contact/base.hpp:71-77) on the current state; returns the count in *n. */
int32_t scopi_gpu_detect(scopi_gpu_handle* h, int64_t* n);

/* ScopiSolver::current_contacts (solver.hpp:314-317): the last step's contacts, sorted by (i, j).
   Any pointer may be NULL. nij/pi/pj are cap*3. */
int32_t scopi_gpu_get_contacts(scopi_gpu_handle* h, int64_t cap, int64_t* n, int64_t* ci, int64_t* cj,
                               double* dij, double* nij, double* pi, double* pj, double* gamma);

/* OptimGradient::lagrange_multiplier (OptimGradient.hpp:323-326), reference local layout. */
int32_t scopi_gpu_get_lambda(scopi_gpu_handle* h, int64_t cap, int64_t* n, double* lambda);

int32_t scopi_gpu_get_stats(scopi_gpu_handle* h, scopi_gpu_stats* out);

/* AMatrix::mat_mult / ATMatrix::mat_mult (matrix/velocities.hpp:67-144, 167-254) on the
   current contact list: u is 6*nb_active, f is 3*contacts. */
int32_t scopi_gpu_amat(scopi_gpu_handle* h, const double* u, double* out);
int32_t scopi_gpu_atmat(scopi_gpu_handle* h, const double* f, double* out);

/* Start angles (a1, b1, a2, b2) of the 3D superellipsoid-superellipsoid closest-point solves
   of the last detection (closest_points.hpp:604-668), 4 per row of the candidate list: the
   pairs that passed the bounding-sphere and support-gap tests, in (i, j) order, before the
   dij < dmax filter; *n = the rows of that list.  Obstacle rows (first, solved in closed
   form) hold no start.  For checking each pair's solve against another implementation from
   the same start; no counterpart in the reference. */
int32_t scopi_gpu_get_se_starts(scopi_gpu_handle* h, int64_t cap, int64_t* n, double* u);

/* The contact list AMatrix / ATMatrix are built on (AMatrix(contacts, particles),
   matrix/velocities.hpp:54-66): replaces the handle's current contact list (the one
   scopi_gpu_get_contacts returns and scopi_gpu_amat / scopi_gpu_atmat use) with n records;
   nij/pi/pj are n*3.  Indices must be < the container's size (else SCOPI_GPU_EINVAL).
   Single-scene handles; the next step detects its own contacts again. */
int32_t scopi_gpu_set_contacts(scopi_gpu_handle* h, int64_t n, const int64_t* ci, const int64_t* cj,
                               const double* dij, const double* nij, const double* pi, const double* pj);

/* Message of the last failing call on this handle (or of the last failing create). */
const char* scopi_gpu_last_error(scopi_gpu_handle* h);

/* Number of kernels this library launched on the handle's stream so far. */
int64_t scopi_gpu_kernel_launches(scopi_gpu_handle* h);

/* ---- batches of independent scenes (one ScopiSolver per scene in the reference) ----
   scopi_gpu_batch_create concatenates n_scenes containers (each obstacles first) into one
   handle; scopi_gpu_run(h, dt, k, 0) then advances every scene k steps, one CUDA graph
   replay per step: contact detection keeps scenes apart, and one persistent launch solves
   all scenes (one CTA per scene, each iterating until its own stopping test holds; the
   mixed precision form corrects each scene in FP64 inside the same launch).  The launch
   shape (threads per scene and tile) is chosen on the first step with a non-trivial solve
   by timing each shape on that step's problem.
   NoFriction (FP64 or MIXED), Friction and ViscousWithoutFriction (FP64: the 6-dof rows, 256
   threads per scene, no autotuning; Viscous scenes carry gamma from step to step); the
   other problems return SCOPI_GPU_EUNSUPPORTED.  scopi_gpu_get_stats reports
   the worst scene (iterations, violation). */
typedef struct scopi_gpu_scene_stats {
    int64_t contacts;
    int64_t iterations;
    int64_t fp32_iterations;
    int64_t backtracks;
    int64_t restarts;
    int32_t corrections;
    int32_t converged;
    double violation;
} scopi_gpu_scene_stats;

int32_t scopi_gpu_batch_create(const scopi_gpu_params* p, int32_t n_scenes, const scopi_gpu_particles* scenes,
                               scopi_gpu_handle** out);
/* pos/q/v/omega of one scene, in that scene's own body order (obstacles first). */
int32_t scopi_gpu_batch_get_scene(scopi_gpu_handle* h, int32_t scene, scopi_gpu_particles* out);
/* statistics of one scene for the last step */
int32_t scopi_gpu_batch_get_scene_stats(scopi_gpu_handle* h, int32_t scene, scopi_gpu_scene_stats* out);
/* block size chosen by the autotuner (0 before the first step) */
int32_t scopi_gpu_batch_block_threads(scopi_gpu_handle* h);
/* pin the threads per scene (256, 512 or 1024: one CTA per scene; 2048: the scenes with at
   least half the largest scene's bodies take a cluster of two 1024-thread CTAs, the others
   one each) instead of autotuning it on the first step; 0 restores autotuning.  Only before
   the first step (else SCOPI_GPU_EINVAL). */
int32_t scopi_gpu_batch_set_block_threads(scopi_gpu_handle* h, int32_t threads);
/* the tile of the batched solve (contacts / incidence records each thread keeps in flight),
   autotuned with the threads per scene: 256 x 4 or 2, 512, 1024 and 2048 x 1 or 2 */
int32_t scopi_gpu_batch_tile(scopi_gpu_handle* h);
/* pin both (0, 0 restores autotuning); only before the first step */
int32_t scopi_gpu_batch_set_shape(scopi_gpu_handle* h, int32_t threads, int32_t tile);

/* APGD solve of one normal-contact QP (NoFriction, FP64, torque-free rows: sphere, plane
   and segment contacts) on caller-provided DEVICE arrays, allocating no device memory.
   No counterpart in the reference (it solves on the host inside OptimGradient::run).
   For callers that cannot allocate while they solve: a process whose device memory is
   owned by another allocator, or a latency-critical loop where cudaMalloc/cudaFree would
   synchronise the device.  Intermediate arrays live in a fixed device array inside this
   library (about 3.4 MB, held by every GPU that loads the library until exit), so:
     - limits: at most 16384 contacts and 8192 active bodies; larger sizes return
       SCOPI_GPU_EINVAL with a message in scopi_gpu_last_error(NULL);
     - the first call on a device looks up that array's device address;
     - all calls share the array: calls that overlap on the GPU (other streams or host
       threads) race; run them one after another.
   Inputs: ci, cj (n_contacts body indices, obstacles < nb_inactive), normal (n_contacts*3,
   outer normal of j, as scopi_gpu_get_contacts returns it), c (n_contacts linear term
   n.(d n + dt A U)), inv_mass (n_active, 1/m), inc_ptr/inc_idx (per active body, its
   contacts sorted by index, entry = contact | (1u<<31) when the body is the contact's j).
   Outputs: lambda (n_contacts), u (n_active*3, M^-1 B^T lambda; may be NULL).
   The lists are checked on the device before the solve reads them (one read-back):
   inc_ptr must start at 0, never decrease and end at most at 2 * n_contacts, every
   inc_idx entry must name a contact < n_contacts and ci/cj must be < nb_inactive +
   n_active; otherwise SCOPI_GPU_EINVAL with the reason in scopi_gpu_last_error(NULL).
   Returns SCOPI_GPU_OK, SCOPI_GPU_ENOCONV (max_ite reached) or an error; the call
   synchronises `stream` (a cudaStream_t, NULL = legacy default stream) before it returns. */
int32_t scopi_gpu_apgd_noalloc(int32_t dim, int64_t n_active, int64_t nb_inactive, int64_t n_contacts,
                               const int32_t* ci, const int32_t* cj, const double* normal, const double* c,
                               const double* inv_mass, const int32_t* inc_ptr, const int32_t* inc_idx, double dt,
                               double alpha, double tolerance, int64_t max_ite, int32_t dynamic_descent,
                               double* lambda, double* u, int64_t* iterations, void* stream);

/* Test of the barrier limit (no counterpart in the reference): block 0 of the next persistent
   APGD launch of this handle does not count its first grid-barrier arrival, so that barrier
   never completes; every block gives up after barrier_timeout_us and the step returns
   SCOPI_GPU_ETIMEOUT.  One shot: later launches are not affected.  Single-scene handles
   only (a batch's launch has no grid barrier: SCOPI_GPU_EINVAL). */
int32_t scopi_gpu_test_barrier_stall(scopi_gpu_handle* h);

/* The handle's CUDA stream (a cudaStream_t), so callers can order their own work and
   time the engine with CUDA events recorded on the stream its kernels run on.
   Infrastructure of this library; the reference has no device streams. */
void* scopi_gpu_get_stream(scopi_gpu_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* SCOPI_GPU_H */
