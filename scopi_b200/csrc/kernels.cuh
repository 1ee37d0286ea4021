// kernels.cuh -- host-side launchers of the SCoPI B200 kernels (one translation unit each).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace scopi_gpu {

// ---------------------------------------------------------------- scan.cu
size_t scan_work_ints(long long n_max);
// out[k] = sum_{i<k} in[i] for k < n with n = *n_dev (or n_host when n_dev is null); *total_dev = sum.
void scan_exclusive(const int* in, int* out, const int* n_dev, int n_host, long long n_max, int* total_dev, int* work,
                    cudaStream_t s, long long* launches);

// -------------------------------------------------------------- detect.cu
struct StepParams {
    int dim;
    int problem;
    int vap;
    int kd_filter;        // contact_kdtree: candidate needs |xi-xj|^2 < kd_tree_radius
    int se_mode;          // superellipsoids: the search keeps the bounding-sphere candidates (se.cu decides)
    double dmax;
    double kd_radius;
    double dt;
    double gamma0, gamma_min, gamma_tol, mu;
    int torque_free;      // every row is normal-only with lever arms along n: the assembly
                          // writes no lever-arm rows (only the 6-dof kernels read them)
};

// partners per contact row kept by the one-pass pair search; a row with more is
// re-enumerated by its compaction thread
constexpr int kRowCap = 24;

struct DetectWork {
    Grid* grid;               // device
    double* bbox_partial;     // kBBoxBlocks * 8
    int* cell_count;          // cell_cap + 1
    int* cell_start;          // cell_cap + 1
    int* cell_fill;           // cell_cap
    int* cell_of;             // na
    int* cell_body;           // na (body index, sorted by cell)
    double4* cell_pr;         // na (x, y, z, r) sorted by cell
    int* occ;                 // na: the occupied cells, in the order their first body was placed
    int* n_occ;               // 1: their count
    int* row_count;           // na + 1
    int* row_ptr;             // na + 1
    int* row_tmp;             // na * kRowCap: partners found by the search pass, unordered
    int* obs_flag;            // nin * na
    int* obs_pos;             // nin * na
    int* tmp_total;           // 4 ints
    int* scan_work;
    long long cell_cap;
    long long obs_cap;        // nin * na
};

struct Assembly {             // FP64 Jacobian rows, K = 1 (normal) problems
    double* bn;               // C*3  n
    double* bai;              // C*3  R_i^T (r_i x n)
    double* baj;              // C*3  -R_j^T (r_j x n)
    double* bP;               // C*18 friction: P_i = R_i^T [r_i]x, P_j = R_j^T [r_j]x
    double* cvec;             // C (K=1), 3C (friction) or 4C (viscous friction, local slots)
    int* vflag;               // C viscous flag, then scanned -> slot; viscous friction: mode 0/1/2
    int* slot;                // C viscous second multiplier (-1 = none)
};

struct Incidence {            // particle-major transpose of the contact list
    int* count;               // na
    int* jcount;              // na (j-side incidences)
    int* ptr;                 // na + 1
    int* idx;                 // 2C: contact | side<<31
    double* coef;             // 2C*6 (K=1: sign*n, a_side)
};

long long detect_launches();
void launch_obstacles_move(const Bodies& b, double dt, int dim, cudaStream_t s);
void launch_vap(const Bodies& b, const StepParams& p, cudaStream_t s, const Sizes* sizes = nullptr);
// Full detection: leaves a sorted (ci, cj) list in `out` and the count in sizes->C.
void launch_detect(const Bodies& b, const StepParams& p, DetectWork& w, Contacts& out, Sizes* sizes, long long c_cap,
                   cudaStream_t s);
// Closest points of the listed pairs + viscous gamma transfer from the previous list.
// Scenes with superellipsoids (b.axes set) also solve the sphere-superellipsoid rows and set
// need_se[k] = 1 on the rows left to launch_se_pairs (pairs of superellipsoids and the
// sphere-superellipsoid rows whose Newton solve was refused), 0 on the others.
void launch_geometry(const Bodies& b, const StepParams& p, Contacts& c, const Sizes* sizes, long long c_cap,
                     const Contacts* old_c, const int* old_C, long long old_cap, cudaStream_t s,
                     int* need_se = nullptr);
void launch_assemble(const Bodies& b, const StepParams& p, const Contacts& c, Assembly& a, Sizes* sizes,
                     long long c_cap, int* scan_work, int* tmp_total, cudaStream_t s);
// with_coef: also the 6 FP64 coefficients per incidence (inc.coef) that the 6-dof
// normal-row kernels read; the torque-free kernels pack their own records instead
void launch_incidence(const Bodies& b, const StepParams& p, const Contacts& c, const Assembly& a, Incidence& inc,
                      const Sizes* sizes, long long c_cap, int* scan_work, int* tmp_total, cudaStream_t s,
                      bool with_coef);
// Worm links (compute_contacts, solver.hpp:358-367): contacts (links[k], links[k] + 1) appended
// at C..C+W-1 after the sorted list (C on the host, the list's count), sizes->C = C + W and
// sizes->n_links = W; k_geometry negates their normal and distance.
void launch_append_links(int C, int W, const int* links, Contacts& c, Sizes* sizes, cudaStream_t s);

// Periodic BoxDomain (box.hpp, utils.hpp:229-257, base.hpp:71-77,118-137, solver.hpp:482-522).
struct PeriodicBox {
    double lo[3], up[3];
    int per[3];
};
// Body arrays of the search: the n bodies, then per periodic axis d the copies shifted by
// up[d] - lo[d] of the active bodies within dmax of lo[d] (t = d * na + a order).
struct GhostBodies {
    double* pos;   // (n + ghosts) * 3
    double* q;     // * 4
    int* shape;
    double* radius;
    double* length;
    int* src;      // ghost -> its body
    int* flag;     // dim * na + 1
    int* rank;     // dim * na + 1
};
// flags and ranks of the copies; the count lands in *total (device)
void launch_ghost_flags(const Bodies& b, const PeriodicBox& box, double dmax, int dim, GhostBodies& g, int* total,
                        int* scan_work, cudaStream_t s);
// fills the search arrays with the bodies and the copies; returns the search's Bodies view
Bodies launch_ghost_fill(const Bodies& b, const PeriodicBox& box, int dim, int n_ghosts, GhostBodies& g,
                         cudaStream_t s);
// Scratch of the remap: per contact two flags and two ranks, the real pairs' keys and the
// copies' entries (cap each).
struct PeriodicScratch {
    int *fr, *fg, *pr, *pg;
    int *r_ci, *r_cj, *g_ci, *g_cj, *g_k, *g_rank, *s_ci, *s_cj;
};
// The search's list (over bodies and copies, sorted, geometry from the copies' positions) ->
// `out`: pairs of two copies dropped, a copy's index replaced by its body's and its closest
// point moved back by up[d] - lo[d] on every periodic axis, the list sorted again by (i, j)
// (a real pair before a copy's pair of the same (i, j)); sizes->C updated.
void launch_periodic_remap(int n, int dim, const PeriodicBox& box, const GhostBodies& g, const Contacts& ext,
                           Contacts& out, PeriodicScratch& w, Sizes* sizes, long long c_cap, int* totals,
                           int* scan_work, cudaStream_t s);
// viscous gamma carried over from the previous list by (i, j) (transfer, solver.hpp:241-258)
void launch_transfer(const StepParams& p, Contacts& c, const Sizes* sizes, const Contacts& old, const int* old_C,
                     long long c_cap, cudaStream_t s);
// wrap of the bodies beyond a periodic bound after the move (solver.hpp:482-522)
void launch_periodic_wrap(const Bodies& b, const PeriodicBox& box, int dim, cudaStream_t s);
void launch_gamma_update(const StepParams& p, Contacts& c, const Assembly& a, const double* lambda, const Sizes* sizes,
                         long long c_cap, cudaStream_t s);
// v += dt*u_v, omega += dt*u_w, then pos/q integration (u = M^-1 B^T lambda, may be null).
// u holds `ustride` doubles per active body: translational part first, then (when
// urot != 0) the rotational part at offset 3.
void launch_update(const Bodies& b, const StepParams& p, const double* u, int ustride, int urot, const Sizes* sizes,
                   cudaStream_t s);
void launch_amat(const Bodies& b, const StepParams& p, const Contacts& c, const Sizes* sizes, long long c_cap,
                 const double* u, double* out, cudaStream_t s);
void launch_atmat(const Bodies& b, const StepParams& p, const Contacts& c, const Sizes* sizes, long long c_cap,
                  const double* f, double* out, cudaStream_t s);

// ----------------------------------------------------------------- se.cu
long long se_launches();
// closest points of the rows k in [C_obs, C) of c with need[k] set (launch_geometry); u0: 4
// doubles per row (scratch)
void launch_se_pairs(int dim, const Bodies& b, Contacts& c, const Sizes* sizes, const int* need, double* u0,
                     int* counter, int grid, cudaStream_t s);
// candidate rows of src whose bodies are not provably farther apart than dmax (obstacle
// rows all kept), compacted into dst
void launch_se_prefilter(int dim, const Bodies& b, const Contacts& src, Contacts& dst, Sizes* sizes, double dmax,
                         long long c_cap, int* keep, int* pos, int* scan_work, int* total, cudaStream_t s);
// rows of src with dij < dmax (obstacle rows all kept) into dst, (i, j) order kept; sizes->C updated
void launch_se_filter(const Contacts& src, Contacts& dst, Sizes* sizes, double dmax, long long c_cap, int* keep,
                      int* pos, int* scan_work, int* total, cudaStream_t s);

// --------------------------------------------------------------- apgd.cu
struct ApgdSettings {
    double alpha;
    double tol;
    long long max_ite;
    int dynamic;
    double dt;
    double mu;
    int curvature_start;      // first step from the curvature estimate instead of alpha
    int stall;                // test of the barrier limit: block 0 skips its first arrival
};

struct ApgdResult {           // written by block 0 of the persistent kernel
    long long iterations;
    long long backtracks;
    long long restarts;
    int converged;
    int lam_buf;              // which of the three lambda buffers holds the result
    int u_buf;                // which u buffer holds M^-1 B^T lambda of the result
    int error;                // barrier timeout
    double last_step;
    double lipsch;            // Lipschitz estimate of the last accepted iteration (finite)
};

template <typename T>
struct SolveBuffers {
    const T* bn;
    const T* bai;
    const T* baj;
    const T* bP;
    const T* cvec;            // linear term (per multiplier)
    const double* shift;      // correction solves: solution offset lambda0 (null = none)
    const int* inc_ptr;
    const int* inc_idx;
    const T* inc_coef;
    T* lam[3];
    T* u[3];                  // per active particle: 6 values
    T* g;
    double* partials;         // 2 * max_blocks * kPartials
    unsigned int* barrier;    // 4 uints (zeroed)
    ApgdResult* result;
};

int apgd_max_blocks(int problem, int dim, bool fp32);
long long apgd_launches();
// Persistent APGD solve; contacts / multipliers counts come from `sizes`.
template <typename T>
cudaError_t launch_apgd_invm(const Bodies& b, const StepParams& p, const ApgdSettings& st, const Contacts& c,
                             const Assembly& a, SolveBuffers<T>& sb, const T* invm, const Sizes* sizes, int nblocks,
                             cudaStream_t s);
// FP64 helpers of the mixed form.
template <typename Src, typename Dst>
void launch_convert(const Src* in, Dst* out, long long n_max, const int* n_dev, int mult, cudaStream_t s);
void launch_particle_pass64(const Bodies& b, const StepParams& p, const Contacts& c, const Assembly& a,
                            const Incidence& inc, const double* invm, const double* lam, double* u, cudaStream_t s);
// g = dt^2 B u + c and the violation max(0, -min gap) (bits of a non-negative double in *viol_bits).
void launch_residual64(const Bodies& b, const StepParams& p, const Contacts& c, const Assembly& a, const double* u,
                       double* g, unsigned long long* viol_bits, const Sizes* sizes, long long c_cap, cudaStream_t s);
// FrictionFixedPoint: cvec = base + s n (dim components), and the s update after a solve
// (u = M^-1 B^T l of the active bodies) with per-block partial sums (2 per block,
// fixed_point_blocks(c_cap) blocks, at most kFixedPointMaxBlocks) of (s_new - s_old)^2, s_new^2.
// ViscousFriction (p.problem == kViscousFriction): cvec = base + dt mu s n on the f slots of
// the mode-2 contacts, s = 1 there before the first solve, s = |(A U)_t| after each.
constexpr int kFixedPointMaxBlocks = 1024;
int fixed_point_blocks(long long c_cap);
void launch_fixed_point_init(double* sv, double v, const Sizes* sizes, long long c_cap, cudaStream_t s);
void launch_vf_fixed_point_init(double* sv, const double* gamma, double gamma_min, const Sizes* sizes,
                                long long c_cap, cudaStream_t s);
void launch_fixed_point_c(const StepParams& p, const Assembly& a, const double* base, const double* sv,
                          const Sizes* sizes, long long c_cap, cudaStream_t s);
void launch_fixed_point_s(const Bodies& b, const StepParams& p, const Contacts& c, const Assembly& a, const double* u,
                          double* sv, double* part, const Sizes* sizes, long long c_cap, cudaStream_t s);
// lambda64 += delta (FP32 or FP64) then projection onto the cone / orthant in FP64.
template <typename TD>
void launch_accumulate(const StepParams& p, const Contacts& c, const Assembly& a, double* lam64, const TD* delta,
                       const Sizes* sizes, long long c_cap, int first, cudaStream_t s);

// ----------------------------------------------------------- apgd_sph.cu
// Normal-only problems on torque-free contacts (every pair type of the hot path): one
// record per contact (n, c) and per incidence (+-n, contact index), translational u only.
struct alignas(32) dvec4 {
    double x, y, z, w;
};
template <typename T>
struct V4_of;
template <>
struct V4_of<float> {
    using type = float4;
};
template <>
struct V4_of<double> {
    using type = dvec4;
};
template <typename T>
using V4 = typename V4_of<T>::type;

template <typename T>
struct SphSolve {
    const int2* cij;
    const V4<T>* nc;
    const int* slot;
    const double* shift;
    const int* inc_ptr;
    const V4<T>* inc;
    const T* invm;            // 1/m per active body, contiguous
    T* lam[3];
    V4<T>* u[4];
    double* partials;         // 4 * max_blocks * 8
    unsigned int* barrier;
    ApgdResult* result;
};

long long apgd_sph_launches();
int apgd_sph_max_blocks(int problem, int dim, bool fp32);
int apgd_sph_threads(bool fp32);  // threads per block of the torque-free kernel
template <typename T>
cudaError_t launch_apgd_sph(int nin, int na, int dim, int problem, const ApgdSettings& st, SphSolve<T>& sb,
                            const Sizes* sizes, int nblocks, cudaStream_t s);
void launch_pack_cij(const int* ci, const int* cj, int2* cij, const Sizes* sizes, long long c_cap, cudaStream_t s);
template <typename T>
void launch_pack_nc(const double* bn, const double* cvec, V4<T>* nc, const Sizes* sizes, long long c_cap,
                    cudaStream_t s);
template <typename T>
void launch_pack_inc(int na, const int* ptr, const int* idx, const double* bn, V4<T>* inc, long long inc_cap,
                     cudaStream_t s);
void launch_sph_particle64(int na, int dim, int problem, const int* ptr, const dvec4* inc, const int* slot,
                           const double* invm, const double* lam, dvec4* u, cudaStream_t s);
void launch_sph_residual64(int nin, int dim, int problem, const int2* cij, const dvec4* nc, const int* slot, double dt2,
                           const dvec4* u, double* g, unsigned long long* viol, const Sizes* sizes, long long c_cap,
                           cudaStream_t s);

// --------------------------------------------------------- apgd_batch.cu
struct BatchSceneStats {
    long long contacts;
    long long iterations;
    long long fp32_iterations;
    long long backtracks;
    long long restarts;
    int corrections;
    int converged;
    double violation;
};

template <typename T>
struct BatchSolve {
    int nin;
    int n_big;  // 2048-thread shape: the scenes (largest first) that take two CTAs each
    const int* order;
    const int *sc_p0, *sc_p1, *sc_o0, *sc_o1, *sc_a0, *sc_a1;
    const int2* cij;
    V4<T>* nc;
    const dvec4* nc64;
    const int* inc_ptr;
    const V4<T>* inc;
    const dvec4* inc64;
    const double* invm;
    T* lam[3];
    V4<T>* u[4];
    double* lam64;
    dvec4* ufin;
    BatchSceneStats* stats;
    const Sizes* sizes;
    double alpha, tol, dt, viol_tol;
    long long max_ite;
    int dynamic;
    int max_corrections;
    int curvature_start;
};

// Batched scenes of a 6-dof problem (Friction), FP64: one CTA per scene over the scene
// ranges of launch_batch_ranges; the multipliers (3 per contact) and u (6 per active body)
// of every scene end in lam_out / u_out, its statistics in stats[scene].
struct Batch6Scenes {
    int n_scenes;
    const int* order;
    const int *sc_p0, *sc_p1, *sc_o0, *sc_o1, *sc_a0, *sc_a1;
    BatchSceneStats* stats;
    double* lam_out;
    double* u_out;
};
cudaError_t launch_apgd_batch6(const Bodies& b, const StepParams& p, const ApgdSettings& st, const Contacts& c,
                               const Assembly& a, SolveBuffers<double>& sb, const double* invm,
                               const Batch6Scenes& S, cudaStream_t s);

long long apgd_batch_launches();
void launch_batch_ranges(int n_scenes, int nin, const int* sc_obs0, const int* sc_obs1, const int* sc_p0,
                         const int* sc_p1, const int* obs_off, const int* obs_pos, const int* row_ptr,
                         const Sizes* sizes, int* o0, int* o1, int* a0, int* a1, cudaStream_t s);
// one CTA per scene: block_threads 256 (tile 2 or 4), 512 or 1024 (tile 1 or 2); the tile is
// the number of independent contacts / incidence records a thread keeps in flight
bool batch_shape_valid(int block_threads, int tile);
template <typename T>
cudaError_t launch_apgd_batch(int dim, int block_threads, int tile, const BatchSolve<T>& b, int n_scenes,
                              cudaStream_t s);

}  // namespace scopi_gpu
