// scopi_gpu.cu -- C ABI (include/scopi_gpu.h): handle, device memory, and the per-step
// sequence of ScopiSolver::run (include/scopi/solver.hpp:274-302) on one B200.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/scopi_gpu.h"
#include "kernels.cuh"

using namespace scopi_gpu;

namespace {

// message of the last failing call that has no handle (fixed buffer: setting it allocates nothing)
thread_local char g_global_error[512] = "";

// batched scenes: threads per scene until the autotuner has run, and the longest scene
// solve (APGD iterations) of the step whose problem it is tuned on
constexpr int kBatchDefaultThreads = 512;
// the tile a block size runs with unless the autotuner chose both
inline int batch_default_tile(int threads) { return threads <= 256 ? 4 : 1; }
constexpr long long kBatchTuneIterations = 64;
// launch shapes the autotuner times (threads per scene x tile; 2048 = a cluster of two CTAs)
constexpr int kBatchShapes = 8;

struct DevMem {
    std::vector<void*> ptrs;
    ~DevMem() { release(); }
    void release() {
        for (void* p : ptrs) cudaFree(p);
        ptrs.clear();
    }
};

}  // namespace

namespace scopi_gpu {
// Message returned by scopi_gpu_last_error(NULL) for calls that have no handle.
void set_global_error(const char* msg) { std::snprintf(g_global_error, sizeof(g_global_error), "%s", msg ? msg : ""); }
void set_global_error2(const char* a, const char* b) {
    std::snprintf(g_global_error, sizeof(g_global_error), "%s%s", a ? a : "", b ? b : "");
}
}  // namespace scopi_gpu

struct scopi_gpu_handle {
    scopi_gpu_params P{};
    int dev = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    long long launches0 = 0;

    // bodies
    int n = 0, nin = 0, na = 0;
    DevMem body_mem;
    int* d_shape = nullptr;
    double *d_pos = nullptr, *d_q = nullptr, *d_v = nullptr, *d_omega = nullptr, *d_vd = nullptr, *d_omega_d = nullptr,
           *d_f = nullptr, *d_m = nullptr, *d_j = nullptr, *d_radius = nullptr, *d_length = nullptr;
    double *d_axes = nullptr, *d_sq = nullptr;  // superellipsoids
    int* d_links = nullptr;  // worm links: first body of each (n entries at most)
    int n_links = 0;
    int *d_se_keep = nullptr, *d_se_pos = nullptr;  // contact filter of superellipsoid candidates
    double* d_se_u = nullptr;                       // start of each superellipsoid solve
    bool has_se = false;                        // some active body is a superellipsoid
    double* d_invm64 = nullptr;
    float* d_invm32 = nullptr;
    double* d_imt64 = nullptr;  // 1/m per active body, contiguous (torque-free kernel)
    float* d_imt32 = nullptr;
    // per-particle solve buffers
    double* d_u64[3] = {nullptr, nullptr, nullptr};
    double* d_ufin = nullptr;
    float* d_u32[3] = {nullptr, nullptr, nullptr};
    DetectWork dw{};

    // contact-capacity buffers
    long long c_cap = 0;
    DevMem cap_mem;
    Contacts cur{}, old{};
    // periodic BoxDomain: the search runs over the bodies and their copies into `ext`
    bool periodic = false;
    PeriodicBox box{};
    GhostBodies gb{};
    PeriodicScratch pw{};
    Contacts ext{};
    int* d_gcount = nullptr;  // 1 + 2: copies, remap totals
    int* h_gcount = nullptr;  // pinned
    Sizes* d_sizes_cur = nullptr;
    Sizes* d_sizes_old = nullptr;
    bool has_old = false;
    Assembly as{};
    Incidence inc{};
    double* d_lam64[3] = {nullptr, nullptr, nullptr};
    double* d_g64 = nullptr;
    double* d_res64 = nullptr;
    double* d_lamacc = nullptr;
    float *d_bn32 = nullptr, *d_bai32 = nullptr, *d_baj32 = nullptr, *d_bP32 = nullptr, *d_cvec32 = nullptr,
          *d_coef32 = nullptr;
    float* d_lam32[3] = {nullptr, nullptr, nullptr};
    float* d_g32 = nullptr;
    // packed records of the torque-free (sphere) kernels
    int2* d_cij = nullptr;
    dvec4* d_nc64 = nullptr;
    float4* d_nc32 = nullptr;
    dvec4* d_incv64 = nullptr;
    float4* d_incv32 = nullptr;
    dvec4* d_us64[4] = {nullptr, nullptr, nullptr, nullptr};
    float4* d_us32[4] = {nullptr, nullptr, nullptr, nullptr};
    dvec4* d_usfin = nullptr;

    // fixed small buffers
    DevMem fixed_mem;
    double* d_partials = nullptr;
    unsigned int* d_barrier = nullptr;
    ApgdResult* d_result = nullptr;
    unsigned long long* d_viol = nullptr;
    Sizes* h_sizes = nullptr;          // pinned
    ApgdResult* h_result = nullptr;    // pinned
    unsigned long long* h_viol = nullptr;
    unsigned int* h_bar = nullptr;     // pinned: the four barrier words written before a launch
    int* h_se_cand = nullptr;          // pinned: superellipsoid candidate pairs of the last detection
    int* d_census = nullptr;           // shape census of an upload (k_shape_census)
    int* h_census = nullptr;           // pinned copy
    bool stall_next = false;           // scopi_gpu_test_barrier_stall: withhold one arrival once
    int max_blocks64 = 0, max_blocks32 = 0, max_sph64 = 0, max_sph32 = 0;
    // FrictionFixedPoint: P.problem holds FRICTION (the kernels' problem), this flag the loop
    // (ViscousFriction keeps its own problem code and runs the same loop)
    bool fixed_point = false;
    double* d_cvec_base = nullptr;  // 3C (4C): the linear term of the step without the s term
    double* d_fp_s = nullptr;       // C: s_c
    double* d_fp_part = nullptr;    // 2 per block of the s update
    double* h_fp_part = nullptr;    // pinned copy

    // results of the last step
    const double* last_lambda = nullptr;
    long long last_M = 0;
    scopi_gpu_stats stats{};
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t ev_a[2] = {nullptr, nullptr};  // around the APGD launches

    int fail(int code, const std::string& msg) {
        err = msg;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* where) {
        err = std::string(where) + ": " + cudaGetErrorString(e);
        return SCOPI_GPU_ECUDA;
    }
    int mult_per_contact() const {
        return P.problem == SCOPI_GPU_VISCOUS_FRICTION ? 4
                                                       : (friction_rows() ? 3 : (P.problem == SCOPI_GPU_VISCOUS ? 2 : 1));
    }
    // multipliers in c (and the Jacobian kept as the three rows of A) per contact
    int cvec_per() const { return P.problem == SCOPI_GPU_VISCOUS_FRICTION ? 4 : (friction_rows() ? 3 : 1); }
    bool friction_rows() const { return P.problem == SCOPI_GPU_FRICTION || P.problem == SCOPI_GPU_VISCOUS_FRICTION; }
    bool viscous_friction() const { return P.problem == SCOPI_GPU_VISCOUS_FRICTION; }
    bool fp_loop() const { return fixed_point || viscous_friction(); }
    // the viscous problems carry each contact's gamma from the previous list by (i, j)
    // (transfer, solver.hpp:241-258); the others never read it (it stays at its default)
    bool carries_gamma() const { return P.problem == SCOPI_GPU_VISCOUS || viscous_friction(); }
    bool mixed() const { return P.precision == SCOPI_GPU_MIXED; }
    // Normal-only problems: every pair type of the hot path (sphere-sphere, sphere-plane,
    // sphere-segment) has its lever arm along the normal, so the rotational Jacobian terms
    // vanish and the translational kernels apply.
    // torque-free rows: every contact's lever arms are parallel to its normal (spheres,
    // planes, segments); superellipsoid contacts need the 6-dof rows
    // torque-free rows and the kernels for them (not for batches of Viscous scenes, which are
    // solved with the 6-dof batched kernel)
    bool sphere_mode() const { return !friction_rows() && !has_se && !batch_six(); }
    // batches solved per scene by k_apgd_batch6 (FP64): Friction and Viscous scenes
    bool batch_six() const { return batch && (friction_rows() || P.problem == SCOPI_GPU_VISCOUS); }

    Bodies bodies() const {
        Bodies b;
        b.n = n;
        b.nin = nin;
        b.shape = d_shape;
        b.pos = d_pos;
        b.q = d_q;
        b.v = d_v;
        b.omega = d_omega;
        b.vd = d_vd;
        b.omega_d = d_omega_d;
        b.f = d_f;
        b.m = d_m;
        b.j = d_j;
        b.radius = d_radius;
        b.length = d_length;
        if (has_se) {
            b.axes = d_axes;
            b.sq = d_sq;
        }
        if (batch) {
            b.scene = d_scene;
            b.scene_shift = d_shift;
            b.obs_a0 = d_obs_a0;
            b.obs_off = d_obs_off;
        }
        return b;
    }

    // ---- batch of independent scenes (scopi_gpu_batch_create): all obstacles first (scene
    // by scene), then the active bodies of scene 0, 1, ...
    bool batch = false;
    int n_scenes = 0;
    std::vector<int> sc_n, sc_nin;                     // bodies / obstacles per scene
    std::vector<long long> sc_obs_start, sc_act_start;  // global index of its first obstacle / active
    DevMem batch_mem;
    int* d_scene = nullptr;
    double* d_shift = nullptr;
    int* d_obs_a0 = nullptr;
    int* d_obs_off = nullptr;
    int *d_sc_obs0 = nullptr, *d_sc_obs1 = nullptr, *d_sc_p0 = nullptr, *d_sc_p1 = nullptr, *d_order = nullptr;
    int *d_sc_o0 = nullptr, *d_sc_o1 = nullptr, *d_sc_a0 = nullptr, *d_sc_a1 = nullptr;
    BatchSceneStats* d_bstats = nullptr;
    std::vector<BatchSceneStats> h_bstats;
    double* d_obs_snap = nullptr;  // obstacle pos (3) and q (4) before the step, restored on overflow
    int batch_threads = 0;         // block size chosen by the autotuner or pinned (0 = not yet)
    int batch_tile = 0;            // contacts in flight per thread chosen with it
    int batch_bt_used = 0;         // block size of the last step
    int batch_tile_used = 0;
    float batch_tune_ms[kBatchShapes] = {};
    int batch_n_big = 0;  // 2048-thread shape: scenes with at least half the largest scene's bodies
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    double graph_dt = 0.0;
    long long graph_cap = -1;
    int graph_bt = 0, graph_tile = 0;
    long long graph_kernels = 0;   // kernels one replay of `graph_exec` launches
    long long replayed = 0;        // kernels launched by graph replays so far
    long long cell_cap_hint = 0;   // cell-list capacity wanted by the batch layout

    void drop_graph() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        graph_exec = nullptr;
        graph = nullptr;
    }

    // Every kernel of one batch step, enqueued on `stream` with no host synchronisation
    // (captured once into a CUDA graph and replayed every step).
    void enqueue_batch_step(double dt, int bt, int tile) {
        Bodies b = bodies();
        StepParams sp = step_params(dt);
        if (nin > 0) {
            cudaMemcpyAsync(d_obs_snap, d_pos, 3 * (size_t)nin * sizeof(double), cudaMemcpyDeviceToDevice, stream);
            cudaMemcpyAsync(d_obs_snap + 3 * (size_t)nin, d_q, 4 * (size_t)nin * sizeof(double),
                            cudaMemcpyDeviceToDevice, stream);
        }
        launch_obstacles_move(b, dt, P.dim, stream);
        cudaMemsetAsync(d_sizes_cur, 0, sizeof(Sizes), stream);
        launch_detect(b, sp, dw, cur, d_sizes_cur, c_cap, stream);
        launch_vap(b, sp, stream, d_sizes_cur);
        // Viscous scenes carry gamma from the previous step's list by (i, j) (solver.hpp:241-258)
        const bool visc = P.problem == SCOPI_GPU_VISCOUS;
        launch_geometry(b, sp, cur, d_sizes_cur, c_cap, visc ? &old : nullptr, visc ? &d_sizes_old->C : nullptr, c_cap,
                        stream);
        launch_assemble(b, sp, cur, as, d_sizes_cur, c_cap, dw.scan_work, dw.tmp_total + 2, stream);
        launch_incidence(b, sp, cur, as, inc, d_sizes_cur, c_cap, dw.scan_work, dw.tmp_total + 2, stream,
                         batch_six());
        if (batch_six()) {
            // Friction (three multipliers per contact) and Viscous scenes (a second multiplier on
            // the contacts with gamma < 0): the 6-dof rows solved per scene in FP64
            launch_batch_ranges(n_scenes, nin, d_sc_obs0, d_sc_obs1, d_sc_p0, d_sc_p1, d_obs_off, dw.obs_pos,
                                dw.row_ptr, d_sizes_cur, d_sc_o0, d_sc_o1, d_sc_a0, d_sc_a1, stream);
            enqueue_batch_solve6(dt);
            if (visc) {
                launch_gamma_update(sp, cur, as, d_lamacc, d_sizes_cur, c_cap, stream);
                // this step's list (pairs and gamma) is the next step's previous list
                cudaMemcpyAsync(old.ci, cur.ci, c_cap * sizeof(int), cudaMemcpyDeviceToDevice, stream);
                cudaMemcpyAsync(old.cj, cur.cj, c_cap * sizeof(int), cudaMemcpyDeviceToDevice, stream);
                cudaMemcpyAsync(old.gamma, cur.gamma, c_cap * sizeof(double), cudaMemcpyDeviceToDevice, stream);
                cudaMemcpyAsync(d_sizes_old, d_sizes_cur, sizeof(Sizes), cudaMemcpyDeviceToDevice, stream);
            }
            launch_update(b, sp, d_ufin, 6, 1, d_sizes_cur, stream);
            return;
        }
        launch_pack_cij(cur.ci, cur.cj, d_cij, d_sizes_cur, c_cap, stream);
        launch_pack_nc<double>(as.bn, as.cvec, d_nc64, d_sizes_cur, c_cap, stream);
        launch_pack_inc<double>(na, inc.ptr, inc.idx, as.bn, d_incv64, 2 * c_cap, stream);
        if (mixed()) {
            launch_pack_nc<float>(as.bn, as.cvec, d_nc32, d_sizes_cur, c_cap, stream);
            launch_pack_inc<float>(na, inc.ptr, inc.idx, as.bn, d_incv32, 2 * c_cap, stream);
        }
        launch_batch_ranges(n_scenes, nin, d_sc_obs0, d_sc_obs1, d_sc_p0, d_sc_p1, d_obs_off, dw.obs_pos, dw.row_ptr,
                            d_sizes_cur, d_sc_o0, d_sc_o1, d_sc_a0, d_sc_a1, stream);
        enqueue_batch_solve(dt, bt, tile);
        launch_update(b, sp, reinterpret_cast<const double*>(d_usfin), 4, 0, d_sizes_cur, stream);
    }

    void enqueue_batch_solve6(double dt) {
        Bodies b = bodies();
        StepParams sp = step_params(dt);
        ApgdSettings st{};
        st.alpha = P.alpha;
        st.tol = P.tolerance;
        st.max_ite = P.max_ite;
        st.dynamic = P.dynamic_descent;
        st.dt = dt;
        st.mu = P.mu;
        st.curvature_start = curvature_start();
        const long long M = (long long)mult_per_contact() * c_cap;
        cudaMemsetAsync(d_lam64[0], 0, M * sizeof(double), stream);
        cudaMemsetAsync(d_lam64[1], 0, M * sizeof(double), stream);
        cudaMemsetAsync(d_u64[0], 0, 6 * (size_t)na * sizeof(double), stream);
        cudaMemsetAsync(d_u64[1], 0, 6 * (size_t)na * sizeof(double), stream);
        SolveBuffers<double> sb{};
        sb.bn = as.bn;
        sb.bai = as.bai;
        sb.baj = as.baj;
        sb.bP = as.bP;
        sb.cvec = as.cvec;
        sb.inc_ptr = inc.ptr;
        sb.inc_idx = inc.idx;
        sb.inc_coef = inc.coef;
        for (int k = 0; k < 3; ++k) {
            sb.lam[k] = d_lam64[k];
            sb.u[k] = d_u64[k];
        }
        sb.g = d_g64;
        Batch6Scenes S{};
        S.n_scenes = n_scenes;
        S.order = d_order;
        S.sc_p0 = d_sc_p0;
        S.sc_p1 = d_sc_p1;
        S.sc_o0 = d_sc_o0;
        S.sc_o1 = d_sc_o1;
        S.sc_a0 = d_sc_a0;
        S.sc_a1 = d_sc_a1;
        S.stats = d_bstats;
        S.lam_out = d_lamacc;
        S.u_out = d_ufin;
        launch_apgd_batch6(b, sp, st, cur, as, sb, d_invm64, S, stream);
    }

    void enqueue_batch_solve(double dt, int bt, int tile) {
        auto fill = [&](auto& bs) {
            bs.nin = nin;
            bs.n_big = batch_n_big;
            bs.order = d_order;
            bs.sc_p0 = d_sc_p0;
            bs.sc_p1 = d_sc_p1;
            bs.sc_o0 = d_sc_o0;
            bs.sc_o1 = d_sc_o1;
            bs.sc_a0 = d_sc_a0;
            bs.sc_a1 = d_sc_a1;
            bs.cij = d_cij;
            bs.nc64 = d_nc64;
            bs.inc_ptr = inc.ptr;
            bs.inc64 = d_incv64;
            bs.invm = d_invm64;
            bs.lam64 = d_lamacc;
            bs.ufin = d_usfin;
            bs.stats = d_bstats;
            bs.sizes = d_sizes_cur;
            bs.alpha = P.alpha;
            bs.tol = P.tolerance;
            bs.dt = dt;
            bs.viol_tol = P.mixed_violation_tol;
            bs.max_ite = P.max_ite;
            bs.dynamic = P.dynamic_descent;
            bs.max_corrections = P.mixed_max_corrections;
            bs.curvature_start = curvature_start();
        };
        if (mixed()) {
            BatchSolve<float> bs{};
            fill(bs);
            bs.nc = d_nc32;
            bs.inc = d_incv32;
            for (int k = 0; k < 3; ++k) bs.lam[k] = d_lam32[k];
            for (int k = 0; k < 4; ++k) bs.u[k] = d_us32[k];
            launch_apgd_batch<float>(P.dim, bt, tile, bs, n_scenes, stream);
        } else {
            BatchSolve<double> bs{};
            fill(bs);
            bs.nc = d_nc64;
            bs.inc = d_incv64;
            for (int k = 0; k < 3; ++k) bs.lam[k] = d_lam64[k];
            for (int k = 0; k < 4; ++k) bs.u[k] = d_us64[k];
            launch_apgd_batch<double>(P.dim, bt, tile, bs, n_scenes, stream);
        }
    }

    int read_batch_sizes() {
        cudaMemcpyAsync(h_sizes, d_sizes_cur, sizeof(Sizes), cudaMemcpyDeviceToHost, stream);
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "batch step");
        return 0;
    }

    // undo the obstacle motion of a step that overflowed and grow the contact buffers
    int batch_overflow_recover() {
        if (nin > 0) {
            cudaMemcpyAsync(d_pos, d_obs_snap, 3 * (size_t)nin * sizeof(double), cudaMemcpyDeviceToDevice, stream);
            cudaMemcpyAsync(d_q, d_obs_snap + 3 * (size_t)nin, 4 * (size_t)nin * sizeof(double),
                            cudaMemcpyDeviceToDevice, stream);
        }
        int tot[2] = {0, 0};
        cudaMemcpy(tot, dw.tmp_total, 2 * sizeof(int), cudaMemcpyDeviceToHost);
        const long long need = (long long)(1.3 * ((double)tot[0] + tot[1])) + 4096;
        drop_graph();
        int rc = alloc_contacts(std::max(need, 2 * c_cap));
        has_old = false;
        return rc;
    }

    void collect_batch_stats() {
        h_bstats.resize(n_scenes);
        cudaMemcpy(h_bstats.data(), d_bstats, n_scenes * sizeof(BatchSceneStats), cudaMemcpyDeviceToHost);
        stats.contacts = 0;
        stats.iterations = stats.fp32_iterations = stats.backtracks = stats.restarts = stats.corrections = 0;
        stats.converged = 1;
        stats.violation = 0.0;
        for (const auto& s : h_bstats) {
            stats.contacts += s.contacts;
            stats.iterations = std::max<int64_t>(stats.iterations, s.iterations);  // the longest scene
            stats.fp32_iterations = std::max<int64_t>(stats.fp32_iterations, s.fp32_iterations);
            stats.backtracks += s.backtracks;
            stats.restarts += s.restarts;
            stats.corrections += s.corrections;
            stats.converged = stats.converged && s.converged;
            stats.violation = std::max(stats.violation, s.violation);
        }
        stats.status = stats.converged ? 0 : SCOPI_GPU_ENOCONV;
    }

    // One time step of every scene: one CUDA graph replay (captured on the first step and
    // again whenever dt, the contact capacity or the launch shape changes).  Autotuning: the
    // steps run with 512 threads per scene until the first step whose longest scene solve
    // takes >= 64 iterations (the first steps of a falling pile converge in one); that
    // step's contact problem is then re-solved with each shape (threads per scene x the tile,
    // the contacts each thread keeps in flight: 256 x 4 / 2, 512, 1024 and 2048 x 1 / 2; 2048
    // puts each of the largest scenes on a cluster of two CTAs) and the
    // fastest is kept for the rest of the run.
    int step_batch(double dt) {
        for (int attempt = 0; attempt < 4; ++attempt) {
            const int bt = batch_threads ? batch_threads : kBatchDefaultThreads;
            const int tile = batch_tile ? batch_tile : batch_default_tile(bt);
            cudaEventRecord(ev[0], stream);
            if (!graph_exec || graph_dt != dt || graph_cap != c_cap || graph_bt != bt || graph_tile != tile) {
                drop_graph();
                cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
                if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
                const long long l0 = launches();
                enqueue_batch_step(dt, bt, tile);
                graph_kernels = launches() - l0;
                replayed -= graph_kernels;  // the capture itself launched nothing
                e = cudaStreamEndCapture(stream, &graph);
                if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
                e = cudaGraphInstantiate(&graph_exec, graph, 0);
                if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
                graph_dt = dt;
                graph_cap = c_cap;
                graph_bt = bt;
                graph_tile = tile;
                cudaEventRecord(ev[0], stream);
            }
            cudaError_t e = cudaGraphLaunch(graph_exec, stream);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
            replayed += graph_kernels;
            int rc = read_batch_sizes();
            if (rc) return rc;
            if (h_sizes->overflow) {
                // nothing after detection ran (overflow guards): restore, grow, redo
                rc = batch_overflow_recover();
                if (rc) return rc;
                continue;
            }
            cudaEventRecord(ev[3], stream);
            collect_batch_stats();
            finish_batch_step_timing();
            batch_bt_used = bt;
            batch_tile_used = tile;
            if (!batch_threads && !batch_six() && stats.iterations >= kBatchTuneIterations)
                return autotune_batch(dt);
            return 0;
        }
        return fail(SCOPI_GPU_ENOMEM, "contact capacity could not be grown");
    }

    // timing only: re-solve the last step's contact problem (its packed records are still in
    // place; the update already used the step's own solve) with each block size
    int autotune_batch(double dt) {
        const int cand[kBatchShapes][2] = {{256, 4},  {256, 2},  {512, 1},  {512, 2},
                                           {1024, 1}, {1024, 2}, {2048, 1}, {2048, 2}};
        float best = 1e30f;
        int best_bt = kBatchDefaultThreads, best_tile = batch_default_tile(kBatchDefaultThreads);
        for (int k = 0; k < kBatchShapes; ++k) {
            cudaEventRecord(ev_a[0], stream);
            enqueue_batch_solve(dt, cand[k][0], cand[k][1]);
            cudaEventRecord(ev_a[1], stream);
            cudaError_t e = cudaEventSynchronize(ev_a[1]);
            if (e != cudaSuccess) return cuda_fail(e, "batch autotune");
            float ms = 0;
            cudaEventElapsedTime(&ms, ev_a[0], ev_a[1]);
            batch_tune_ms[k] = ms;
            if (ms < best) {
                best = ms;
                best_bt = cand[k][0];
                best_tile = cand[k][1];
            }
        }
        batch_threads = best_bt;
        batch_tile = best_tile;
        return 0;
    }

    void finish_batch_step_timing() {
        cudaEventSynchronize(ev[3]);
        float t = 0;
        cudaEventElapsedTime(&t, ev[0], ev[3]);
        stats.ms_step = t;
        stats.ms_solve = t;
        stats.ms_apgd_kernel = 0;
        stats.steps += 1;
    }
    StepParams step_params(double dt) const {
        StepParams s;
        s.dim = P.dim;
        s.problem = P.problem;
        s.vap = P.vap;
        s.kd_filter = P.contact_method == SCOPI_GPU_KDTREE ? 1 : 0;
        s.se_mode = has_se ? 1 : 0;
        s.dmax = P.dmax;
        s.kd_radius = P.kd_tree_radius;
        s.dt = dt;
        s.gamma0 = P.gamma;
        s.gamma_min = P.gamma_min;
        s.gamma_tol = P.gamma_tol;
        s.mu = P.mu;
        s.torque_free = sphere_mode() ? 1 : 0;
        return s;
    }

    template <typename T>
    cudaError_t alloc(DevMem& m, T*& p, size_t count) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) return e;
        m.ptrs.push_back(q);
        p = static_cast<T*>(q);
        return cudaSuccess;
    }

    int alloc_fixed() {
        cudaError_t e;
        max_blocks64 = apgd_max_blocks(P.problem, P.dim, false);
        max_blocks32 = apgd_max_blocks(P.problem, P.dim, true);
        if (sphere_mode()) {
            max_sph64 = apgd_sph_max_blocks(P.problem, P.dim, false);
            max_sph32 = apgd_sph_max_blocks(P.problem, P.dim, true);
        }
        const int mb = std::max({max_blocks64, max_blocks32, max_sph64, max_sph32, 1});
        if ((e = alloc(fixed_mem, d_partials, 4 * (size_t)mb * 8)) != cudaSuccess) return cuda_fail(e, "alloc");
        if ((e = alloc(fixed_mem, d_barrier, 4)) != cudaSuccess) return cuda_fail(e, "alloc");
        if ((e = alloc(fixed_mem, d_result, 1)) != cudaSuccess) return cuda_fail(e, "alloc");
        if ((e = alloc(fixed_mem, d_viol, 1)) != cudaSuccess) return cuda_fail(e, "alloc");
        if ((e = alloc(fixed_mem, d_sizes_cur, 1)) != cudaSuccess) return cuda_fail(e, "alloc");
        if ((e = alloc(fixed_mem, d_sizes_old, 1)) != cudaSuccess) return cuda_fail(e, "alloc");
        cudaMemset(d_sizes_cur, 0, sizeof(Sizes));
        cudaMemset(d_sizes_old, 0, sizeof(Sizes));
        cudaMemset(d_barrier, 0, 4 * sizeof(unsigned int));
        if ((e = cudaMallocHost(&h_bar, 4 * sizeof(unsigned int))) != cudaSuccess)
            return cuda_fail(e, "cudaMallocHost");
        if ((e = alloc(fixed_mem, d_census, 4)) != cudaSuccess) return cuda_fail(e, "alloc");
        if ((e = cudaMallocHost(&h_se_cand, sizeof(int))) != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
        *h_se_cand = 0;
        if ((e = cudaMallocHost(&h_census, 4 * sizeof(int))) != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
        h_bar[0] = h_bar[1] = h_bar[2] = 0u;
        h_bar[3] = P.barrier_timeout_us > 0 ? (unsigned int)P.barrier_timeout_us : 0u;
        if ((e = cudaMallocHost(&h_sizes, sizeof(Sizes))) != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
        if ((e = cudaMallocHost(&h_result, sizeof(ApgdResult))) != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
        if ((e = cudaMallocHost(&h_viol, sizeof(unsigned long long))) != cudaSuccess)
            return cuda_fail(e, "cudaMallocHost");
        if (periodic) {
            if ((e = alloc(fixed_mem, d_gcount, 3)) != cudaSuccess) return cuda_fail(e, "alloc");
            if ((e = cudaMallocHost(&h_gcount, sizeof(int))) != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
        }
        if (fp_loop()) {
            if ((e = alloc(fixed_mem, d_fp_part, 2 * (size_t)kFixedPointMaxBlocks)) != cudaSuccess)
                return cuda_fail(e, "alloc");
            if ((e = cudaMallocHost(&h_fp_part, 2 * sizeof(double) * kFixedPointMaxBlocks)) != cudaSuccess)
                return cuda_fail(e, "cudaMallocHost");
        }
        for (auto& x : ev)
            if ((e = cudaEventCreate(&x)) != cudaSuccess) return cuda_fail(e, "cudaEventCreate");
        for (auto& x : ev_a)
            if ((e = cudaEventCreate(&x)) != cudaSuccess) return cuda_fail(e, "cudaEventCreate");
        return 0;
    }

    // Buffers whose size follows the number of bodies.
    int alloc_bodies(int n_, int nin_, long long obs_cap = -1) {
        body_mem.release();
        n = n_;
        nin = nin_;
        na = n - nin;
        cudaError_t e;
#define A(p, c) \
    if ((e = alloc(body_mem, p, (c))) != cudaSuccess) return cuda_fail(e, "cudaMalloc(bodies)");
        A(d_shape, n) A(d_pos, 3 * (size_t)n) A(d_q, 4 * (size_t)n) A(d_v, 3 * (size_t)n) A(d_omega, 3 * (size_t)n)
        A(d_vd, 3 * (size_t)n) A(d_omega_d, 3 * (size_t)n) A(d_f, 3 * (size_t)n) A(d_m, n) A(d_j, 3 * (size_t)n)
        A(d_radius, n) A(d_length, n) A(d_axes, 3 * (size_t)n) A(d_sq, 2 * (size_t)n) A(d_invm64, 4 * (size_t)na + 4) A(d_invm32, 4 * (size_t)na + 4)
        A(d_links, n)
        A(d_imt64, (size_t)na + 1) A(d_imt32, (size_t)na + 1)
        A(d_ufin, 6 * (size_t)na + 6)
        A(d_usfin, (size_t)na + 1)
        for (int k = 0; k < 4; ++k) {
            A(d_us64[k], (size_t)na + 1)
            A(d_us32[k], (size_t)na + 1)
        }
        for (int k = 0; k < 3; ++k) {
            A(d_u64[k], 6 * (size_t)na + 6)
            A(d_u32[k], 6 * (size_t)na + 6)
        }
        // the search of a periodic box also holds the copies: up to dim per active body
        const long long naw = periodic ? (long long)na * (1 + P.dim) : na;
        dw.cell_cap = std::max<long long>({4LL * naw, 4096LL, cell_cap_hint});
        dw.obs_cap = obs_cap >= 0 ? obs_cap : (long long)nin * naw;
        A(dw.grid, 1) A(dw.bbox_partial, 8 * 4 * kSMs) A(dw.cell_count, dw.cell_cap + 1) A(dw.cell_start, dw.cell_cap + 1)
        A(dw.cell_fill, dw.cell_cap) A(dw.cell_of, naw + 1) A(dw.cell_body, naw + 1) A(dw.cell_pr, naw + 1)
        A(dw.occ, naw + 1) A(dw.n_occ, 1)
        A(dw.row_count, naw + 1) A(dw.row_ptr, naw + 1) A(dw.row_tmp, (size_t)naw * kRowCap + 1) A(dw.obs_flag, dw.obs_cap + 1) A(dw.obs_pos, dw.obs_cap + 1)
        A(dw.tmp_total, 4)
        if (periodic) {
            const long long ne = n + (naw - na), m = (long long)P.dim * na + 1;
            A(gb.pos, 3 * ne) A(gb.q, 4 * ne) A(gb.shape, ne) A(gb.radius, ne) A(gb.length, ne) A(gb.src, m)
            A(gb.flag, m) A(gb.rank, m)
        }
        const long long scan_max =
            std::max<long long>(std::max<long long>(dw.cell_cap + 1, dw.obs_cap + 1), std::max<long long>(naw, 1) * 3 + 1);
        A(dw.scan_work, scan_work_ints(std::max<long long>(scan_max, 1LL << 26)))
        A(inc.count, na + 1) A(inc.jcount, na + 1) A(inc.ptr, na + 1)
#undef A
        return 0;
    }

    // Buffers whose size follows the contact capacity.
    int alloc_contacts(long long cap) {
        cap_mem.release();
        c_cap = cap;
        has_old = false;
        const long long M = cap * mult_per_contact();
        cudaError_t e;
#define A(p, c) \
    if ((e = alloc(cap_mem, p, (c))) != cudaSuccess) return cuda_fail(e, "cudaMalloc(contacts)");
        for (Contacts* c : {&cur, &old}) {
            A(c->ci, cap) A(c->cj, cap) A(c->dij, cap) A(c->nij, 3 * cap) A(c->pi, 3 * cap) A(c->pj, 3 * cap)
            A(c->gamma, cap)
        }
        if (periodic) {
            A(ext.ci, cap) A(ext.cj, cap) A(ext.dij, cap) A(ext.nij, 3 * cap) A(ext.pi, 3 * cap) A(ext.pj, 3 * cap)
            A(ext.gamma, cap)
            for (int** q : {&pw.fr, &pw.fg, &pw.pr, &pw.pg, &pw.r_ci, &pw.r_cj, &pw.g_ci, &pw.g_cj, &pw.g_k, &pw.g_rank,
                            &pw.s_ci, &pw.s_cj})
                A(*q, cap + 1)
        }
        A(as.bn, 3 * cap) A(as.bai, 3 * cap) A(as.baj, 3 * cap)
        if (friction_rows()) A(as.bP, 18 * cap)
        A(as.cvec, cvec_per() * cap) A(as.vflag, cap) A(as.slot, cap)
        if (fp_loop()) {
            A(d_cvec_base, cvec_per() * cap) A(d_fp_s, cap)
        }
        A(inc.idx, 2 * cap) A(inc.coef, 12 * cap)
        for (int k = 0; k < 3; ++k) A(d_lam64[k], M)
        A(d_g64, M) A(d_res64, M) A(d_lamacc, M)
        if (mixed()) {
            A(d_bn32, 3 * cap) A(d_bai32, 3 * cap) A(d_baj32, 3 * cap)
            if (friction_rows()) A(d_bP32, 18 * cap)
            A(d_cvec32, cvec_per() * cap) A(d_coef32, 12 * cap)
            for (int k = 0; k < 3; ++k) A(d_lam32[k], M)
            A(d_g32, M)
        }
        A(d_cij, cap) A(d_nc64, cap) A(d_incv64, 2 * cap) A(d_se_keep, cap + 1) A(d_se_pos, cap + 1) A(d_se_u, 4 * cap + 4)
        if (mixed()) {
            A(d_nc32, cap) A(d_incv32, 2 * cap)
        }
#undef A
        cudaMemsetAsync(d_sizes_cur, 0, sizeof(Sizes), stream);
        cudaMemsetAsync(d_sizes_old, 0, sizeof(Sizes), stream);
        return 0;
    }

    // first APGD step: the reference's alpha, or the curvature estimate (AUTO: MIXED only)
    int curvature_start() const {
        if (P.initial_step == SCOPI_GPU_STEP_AUTO) return mixed() ? 1 : 0;
        return P.initial_step == SCOPI_GPU_STEP_CURVATURE ? 1 : 0;
    }

    long long launches() const {
        return detect_launches() + apgd_launches() + apgd_sph_launches() + apgd_batch_launches() + se_launches() +
               replayed;
    }

    // contact detection + closest points + assembly + incidence lists into `cur`
    // Detection in a periodic box: copies of the active bodies near the lower bounds join the
    // search (contact_base::run, base.hpp:71-77), the list is mapped back to the bodies and
    // sorted again (compute_exact_distance, base.hpp:118-137), then gamma is carried over.
    int detect_periodic(double dt, bool assemble) {
        Bodies b = bodies();
        StepParams sp = step_params(dt);
        launch_ghost_flags(b, box, P.dmax, P.dim, gb, d_gcount, dw.scan_work, stream);
        cudaMemcpyAsync(h_gcount, d_gcount, sizeof(int), cudaMemcpyDeviceToHost, stream);
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "periodic copies");
        const Bodies eb = launch_ghost_fill(b, box, P.dim, *h_gcount, gb, stream);
        dw.obs_cap = (long long)nin * (eb.n - eb.nin);
        for (int attempt = 0; attempt < 4; ++attempt) {
            cudaMemsetAsync(d_sizes_cur, 0, sizeof(Sizes), stream);
            launch_detect(eb, sp, dw, ext, d_sizes_cur, c_cap, stream);
            cudaMemcpyAsync(h_sizes, d_sizes_cur, sizeof(Sizes), cudaMemcpyDeviceToHost, stream);
            e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) return cuda_fail(e, "detect");
            if (!h_sizes->overflow) break;
            int tot[2] = {0, 0};
            cudaMemcpy(tot, dw.tmp_total, 2 * sizeof(int), cudaMemcpyDeviceToHost);
            const long long total = (long long)tot[0] + tot[1];
            const long long need = (long long)std::ceil(1.3 * ((double)h_sizes->C + 1.0)) + 1024;
            int rc = regrow(std::max(need, (long long)(1.3 * total) + 1024));
            if (rc) return rc;
            if (attempt == 3) return fail(SCOPI_GPU_ENOMEM, "contact capacity could not be grown");
        }
        launch_geometry(eb, sp, ext, d_sizes_cur, c_cap, nullptr, nullptr, c_cap, stream);
        launch_periodic_remap(n, P.dim, box, gb, ext, cur, pw, d_sizes_cur, c_cap, d_gcount + 1, dw.scan_work, stream);
        launch_transfer(sp, cur, d_sizes_cur, old, (has_old && carries_gamma()) ? &d_sizes_old->C : nullptr, c_cap,
                        stream);
        if (assemble) {
            launch_assemble(b, sp, cur, as, d_sizes_cur, c_cap, dw.scan_work, dw.tmp_total + 2, stream);
            launch_incidence(b, sp, cur, as, inc, d_sizes_cur, c_cap, dw.scan_work, dw.tmp_total + 2, stream,
                             !sphere_mode());
        }
        cudaMemcpyAsync(h_sizes, d_sizes_cur, sizeof(Sizes), cudaMemcpyDeviceToHost, stream);
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "assemble");
        return 0;
    }

    int detect_and_assemble(double dt, bool assemble) {
        if (periodic) return detect_periodic(dt, assemble);
        Bodies b = bodies();
        StepParams sp = step_params(dt);
        for (int attempt = 0; attempt < 4; ++attempt) {
            cudaMemsetAsync(d_sizes_cur, 0, sizeof(Sizes), stream);
            launch_detect(b, sp, dw, cur, d_sizes_cur, c_cap, stream);
            cudaMemcpyAsync(h_sizes, d_sizes_cur, sizeof(Sizes), cudaMemcpyDeviceToHost, stream);
            cudaError_t e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) return cuda_fail(e, "detect");
            const int links = assemble ? n_links : 0;
            if (!h_sizes->overflow && (long long)h_sizes->C + links <= c_cap) break;
            // grow: keep the previous contacts (viscous gamma transfer) across the reallocation
            const long long need = (long long)std::ceil(1.3 * ((double)h_sizes->C + links + 1.0)) + 1024;
            long long total = 0;
            {
                // the true count is C_obs + active rows; recompute it from the scan totals
                int tot[2] = {0, 0};
                cudaMemcpy(tot, dw.tmp_total, 2 * sizeof(int), cudaMemcpyDeviceToHost);
                total = (long long)tot[0] + tot[1];
            }
            const long long newcap = std::max(need, (long long)(1.3 * total) + 1024);
            int rc = regrow(newcap);
            if (rc) return rc;
            if (attempt == 3) return fail(SCOPI_GPU_ENOMEM, "contact capacity could not be grown");
        }
        // the step's list is the contact method's plus the worm links (compute_contacts,
        // solver.hpp:358-367); detection alone (assemble == false) is the contact method's
        if (assemble && n_links > 0) launch_append_links(h_sizes->C, n_links, d_links, cur, d_sizes_cur, stream);
        const bool tr = has_old && carries_gamma();
        if (!has_se) {
            launch_geometry(b, sp, cur, d_sizes_cur, c_cap, tr ? &old : nullptr, tr ? &d_sizes_old->C : nullptr,
                            c_cap, stream);
        } else {
            // the search kept bounding-sphere candidates: the pairs that can touch (gap along
            // the line of centres <= dmax), the closest points of the spheres' rows, those of
            // the rows flagged in d_se_keep (pairs of superellipsoids, sphere rows whose Newton
            // solve was refused), then the rows with dij < dmax (no viscous gamma to carry
            // here); each filter compacts into the other list, which becomes the current one
            launch_se_prefilter(P.dim, b, cur, old, d_sizes_cur, P.dmax, c_cap, d_se_keep, d_se_pos, dw.scan_work,
                                dw.tmp_total + 2, stream);
            std::swap(cur, old);
            launch_geometry(b, sp, cur, d_sizes_cur, c_cap, nullptr, nullptr, c_cap, stream, d_se_keep);
            launch_se_pairs(P.dim, b, cur, d_sizes_cur, d_se_keep, d_se_u, dw.tmp_total + 3, 3 * kSMs, stream);
            cudaMemcpyAsync(h_se_cand, &d_sizes_cur->C, sizeof(int), cudaMemcpyDeviceToHost, stream);
            launch_se_filter(cur, old, d_sizes_cur, P.dmax, c_cap, d_se_keep, d_se_pos, dw.scan_work,
                             dw.tmp_total + 2, stream);
            std::swap(cur, old);
        }
        if (!assemble) return 0;
        launch_assemble(b, sp, cur, as, d_sizes_cur, c_cap, dw.scan_work, dw.tmp_total + 2, stream);
        launch_incidence(b, sp, cur, as, inc, d_sizes_cur, c_cap, dw.scan_work, dw.tmp_total + 2, stream,
                         !sphere_mode());
        cudaMemcpyAsync(h_sizes, d_sizes_cur, sizeof(Sizes), cudaMemcpyDeviceToHost, stream);
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "assemble");
        return 0;
    }

    int regrow(long long newcap) {
        // copy the previous contact list (ci, cj, gamma) so the transfer still works
        std::vector<int> oci, ocj;
        std::vector<double> ogam;
        Sizes osz{};
        if (has_old) {
            cudaMemcpy(&osz, d_sizes_old, sizeof(Sizes), cudaMemcpyDeviceToHost);
            oci.resize(osz.C);
            ocj.resize(osz.C);
            ogam.resize(osz.C);
            if (osz.C > 0) {
                cudaMemcpy(oci.data(), old.ci, osz.C * sizeof(int), cudaMemcpyDeviceToHost);
                cudaMemcpy(ocj.data(), old.cj, osz.C * sizeof(int), cudaMemcpyDeviceToHost);
                cudaMemcpy(ogam.data(), old.gamma, osz.C * sizeof(double), cudaMemcpyDeviceToHost);
            }
        }
        const bool had = has_old;
        int rc = alloc_contacts(newcap);
        if (rc) return rc;
        if (had) {
            if (osz.C > 0) {
                cudaMemcpy(old.ci, oci.data(), osz.C * sizeof(int), cudaMemcpyHostToDevice);
                cudaMemcpy(old.cj, ocj.data(), osz.C * sizeof(int), cudaMemcpyHostToDevice);
                cudaMemcpy(old.gamma, ogam.data(), osz.C * sizeof(double), cudaMemcpyHostToDevice);
            }
            Sizes s{};
            s.C = osz.C;
            cudaMemcpy(d_sizes_old, &s, sizeof(Sizes), cudaMemcpyHostToDevice);
            has_old = true;
        }
        return 0;
    }

    int nblocks_for(int maxb, long long work, int threads = 256) const {
        long long b = (work + threads - 1) / threads;
        b = std::max<long long>(b, 1);
        return (int)std::min<long long>(b, maxb);
    }

    // The barrier words of the next persistent launch: arrivals, generation and error flag
    // zero, the wait limit (us, 0 = the default); and the one-shot stall of the timeout test.
    cudaError_t reset_barrier(ApgdSettings& st) {
        st.stall = stall_next ? 1 : 0;
        stall_next = false;
        return cudaMemcpyAsync(d_barrier, h_bar, 4 * sizeof(unsigned int), cudaMemcpyHostToDevice, stream);
    }

    template <typename T>
    int run_apgd(SolveBuffers<T>& sb, const T* invm, int maxb, double dt, double tol, long long max_ite, long long M,
                 double alpha0 = 0.0) {
        Bodies b = bodies();
        StepParams sp = step_params(dt);
        ApgdSettings st{};
        st.alpha = alpha0 > 0.0 ? alpha0 : P.alpha;
        st.tol = tol;
        st.max_ite = max_ite;
        st.dynamic = P.dynamic_descent;
        st.dt = dt;
        st.mu = P.mu;
        // a correction solve starts from the step size of the solve before it
        st.curvature_start = alpha0 > 0.0 ? 0 : curvature_start();
        cudaMemsetAsync(sb.lam[0], 0, M * sizeof(T), stream);
        cudaMemsetAsync(sb.lam[1], 0, M * sizeof(T), stream);
        cudaMemsetAsync(sb.u[0], 0, 6 * (size_t)na * sizeof(T), stream);
        cudaMemsetAsync(sb.u[1], 0, 6 * (size_t)na * sizeof(T), stream);
        cudaError_t e = reset_barrier(st);
        if (e != cudaSuccess) return cuda_fail(e, "APGD barrier words");
        const int nb = nblocks_for(maxb, std::max<long long>(h_sizes->C, na));
        e = launch_apgd_invm<T>(b, sp, st, cur, as, sb, invm, d_sizes_cur, nb, stream);
        if (e != cudaSuccess) return cuda_fail(e, "APGD launch");
        cudaMemcpyAsync(h_result, d_result, sizeof(ApgdResult), cudaMemcpyDeviceToHost, stream);
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "APGD");
        if (h_result->error == 1) return fail(SCOPI_GPU_ETIMEOUT, "APGD grid barrier timed out");
        return 0;
    }

    template <typename T>
    int run_apgd_sph(SphSolve<T>& sb, int maxb, double dt, double tol, long long max_ite, long long M,
                     double alpha0 = 0.0) {
        ApgdSettings st{};
        st.alpha = alpha0 > 0.0 ? alpha0 : P.alpha;
        st.tol = tol;
        st.max_ite = max_ite;
        st.dynamic = P.dynamic_descent;
        st.dt = dt;
        st.mu = P.mu;
        st.curvature_start = curvature_start();
        // lambda = lambda_prev = 0 and u(lambda) = u(y) = 0 (cold start, apgd.hpp:152-159)
        cudaMemsetAsync(sb.lam[0], 0, M * sizeof(T), stream);
        cudaMemsetAsync(sb.lam[1], 0, M * sizeof(T), stream);
        cudaMemsetAsync(sb.u[0], 0, (size_t)na * sizeof(V4<T>), stream);
        cudaMemsetAsync(sb.u[2], 0, (size_t)na * sizeof(V4<T>), stream);
        cudaError_t e = reset_barrier(st);
        if (e != cudaSuccess) return cuda_fail(e, "APGD barrier words");
        const int nb = nblocks_for(maxb, std::max<long long>(h_sizes->C, na), apgd_sph_threads(sizeof(T) == 4));
        e = launch_apgd_sph<T>(nin, na, P.dim, P.problem, st, sb, d_sizes_cur, nb, stream);
        if (e != cudaSuccess) return cuda_fail(e, "APGD launch");
        cudaMemcpyAsync(h_result, d_result, sizeof(ApgdResult), cudaMemcpyDeviceToHost, stream);
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "APGD");
        if (h_result->error == 1) return fail(SCOPI_GPU_ETIMEOUT, "APGD grid barrier timed out");
        return 0;
    }

    template <typename T>
    SphSolve<T> sph_buffers(const V4<T>* nc, const V4<T>* incv, const T* imt, T* const* lam, V4<T>* const* u) const {
        SphSolve<T> sb{};
        sb.cij = d_cij;
        sb.nc = nc;
        sb.slot = as.slot;
        sb.shift = nullptr;
        sb.inc_ptr = inc.ptr;
        sb.inc = incv;
        sb.invm = imt;
        for (int k = 0; k < 3; ++k) sb.lam[k] = lam[k];
        for (int k = 0; k < 4; ++k) sb.u[k] = u[k];
        sb.partials = d_partials;
        sb.barrier = d_barrier;
        sb.result = d_result;
        return sb;
    }

    int step(double dt) {
        Bodies b = bodies();
        StepParams sp = step_params(dt);
        cudaEventRecord(ev[0], stream);
        launch_obstacles_move(b, dt, P.dim, stream);
        // vap does not read the contacts (vap_fixed.hpp:45-55, vap_fpd.hpp:69-81): run it first
        launch_vap(b, sp, stream);
        int rc = detect_and_assemble(dt, true);
        if (rc) return rc;
        const int C = h_sizes->C;
        const long long M = friction_rows() ? (long long)mult_per_contact() * C : (long long)C + h_sizes->n_extra;
        cudaEventRecord(ev[1], stream);
        const double* ufin = nullptr;
        int ustride = 6, urot = 1;
        stats.iterations = stats.backtracks = stats.restarts = stats.fp32_iterations = stats.corrections = 0;
        stats.fixed_point_iterations = 0;
        stats.converged = 1;
        stats.status = 0;
        stats.violation = 0.0;
        float ms_apgd = 0.0f;
        if (C > 0) {
            if (sphere_mode()) {
                launch_pack_cij(cur.ci, cur.cj, d_cij, d_sizes_cur, c_cap, stream);
                launch_pack_nc<double>(as.bn, as.cvec, d_nc64, d_sizes_cur, c_cap, stream);
                launch_pack_inc<double>(na, inc.ptr, inc.idx, as.bn, d_incv64, 2 * c_cap, stream);
                ustride = 4;
                urot = 0;
            }
            auto solve = [&]() -> int {
            if (!mixed()) {
                float ms = 0.0f;
                cudaEventRecord(ev_a[0], stream);
                if (sphere_mode()) {
                    SphSolve<double> sb = sph_buffers<double>(d_nc64, d_incv64, d_imt64, d_lam64, d_us64);
                    rc = run_apgd_sph<double>(sb, max_sph64, dt, P.tolerance, P.max_ite, M);
                    if (rc) return rc;
                    ufin = reinterpret_cast<const double*>(d_us64[h_result->u_buf]);
                } else {
                    SolveBuffers<double> sb{};
                    sb.bn = as.bn;
                    sb.bai = as.bai;
                    sb.baj = as.baj;
                    sb.bP = as.bP;
                    sb.cvec = as.cvec;
                    sb.shift = nullptr;
                    sb.inc_ptr = inc.ptr;
                    sb.inc_idx = inc.idx;
                    sb.inc_coef = inc.coef;
                    for (int k = 0; k < 3; ++k) {
                        sb.lam[k] = d_lam64[k];
                        sb.u[k] = d_u64[k];
                    }
                    sb.g = d_g64;
                    sb.partials = d_partials;
                    sb.barrier = d_barrier;
                    sb.result = d_result;
                    rc = run_apgd<double>(sb, d_invm64, max_blocks64, dt, P.tolerance, P.max_ite, M);
                    if (rc) return rc;
                    ufin = d_u64[h_result->u_buf];
                }
                cudaEventRecord(ev_a[1], stream);
                cudaEventSynchronize(ev_a[1]);
                cudaEventElapsedTime(&ms, ev_a[0], ev_a[1]);
                ms_apgd += ms;
                accumulate_stats(false);
                last_lambda = d_lam64[h_result->lam_buf];
            } else {
                float ms = 0.0f;
                rc = mixed_solve(dt, M, ms);
                if (rc) return rc;
                ms_apgd += ms;
                last_lambda = d_lamacc;
                ufin = sphere_mode() ? reinterpret_cast<const double*>(d_usfin) : d_ufin;
            }
            return 0;
            };
            if (fp_loop()) {
                // FrictionFixedPoint (OptimGradient.hpp:85-176, solver.hpp:286-291): s_c = mu dt,
                // then solve with the linear term c + s n, update s from the tangential relative
                // velocity, until the relative change of s is below fixed_point_tol.
                // ViscousFriction (OptimGradient.hpp:96-107, 178-250): s_c = 1 on the contacts at
                // gamma_min, linear term c + dt mu s n on their friction slots, s = |(A u)_t|, the
                // change measured without the 1/(mu dt) scale.
                const bool vf = viscous_friction();
                cudaMemcpyAsync(d_cvec_base, as.cvec, (size_t)cvec_per() * C * sizeof(double),
                                cudaMemcpyDeviceToDevice, stream);
                const double mudt = P.mu * dt;
                if (vf)
                    launch_vf_fixed_point_init(d_fp_s, cur.gamma, P.gamma_min, d_sizes_cur, c_cap, stream);
                else
                    launch_fixed_point_init(d_fp_s, mudt, d_sizes_cur, c_cap, stream);
                const int nbk = fixed_point_blocks(c_cap);
                long long it = 0;
                for (;;) {
                    launch_fixed_point_c(sp, as, d_cvec_base, d_fp_s, d_sizes_cur, c_cap, stream);
                    rc = solve();
                    if (rc) return rc;
                    launch_fixed_point_s(b, sp, cur, as, ufin, d_fp_s, d_fp_part, d_sizes_cur, c_cap, stream);
                    cudaMemcpyAsync(h_fp_part, d_fp_part, 2 * sizeof(double) * nbk, cudaMemcpyDeviceToHost, stream);
                    cudaError_t e = cudaStreamSynchronize(stream);
                    if (e != cudaSuccess) return cuda_fail(e, "fixed point");
                    double dd = 0.0, ss = 0.0;
                    for (int k = 0; k < nbk; ++k) {
                        dd += h_fp_part[2 * k];
                        ss += h_fp_part[2 * k + 1];
                    }
                    ++it;
                    double err;
                    if (vf) {
                        err = std::sqrt(dd) / (1.0 + std::sqrt(ss));
                    } else {
                        // mu dt = 0: s stays 0 and one solve is the answer (the reference's
                        // normalisation by 1/(mu dt) would give NaN and run fixed_point_max_iter solves)
                        if (!(mudt > 0.0)) break;
                        err = (std::sqrt(dd) / mudt) / (1.0 + std::sqrt(ss) / mudt);
                    }
                    if (err < P.fixed_point_tol || it >= P.fixed_point_max_iter) break;
                }
                stats.fixed_point_iterations = it;
            } else {
                rc = solve();
                if (rc) return rc;
            }
            // violation of the returned multipliers (FP64 residual); the mixed form's last
            // action was that same residual of its final multipliers, already in h_viol
            if (!(mixed() && !fp_loop())) {
                cudaMemsetAsync(d_viol, 0, sizeof(unsigned long long), stream);
                if (sphere_mode())
                    launch_sph_residual64(nin, P.dim, P.problem, d_cij, d_nc64, as.slot, dt * dt,
                                          reinterpret_cast<const dvec4*>(ufin), d_res64, d_viol, d_sizes_cur, c_cap,
                                          stream);
                else
                    launch_residual64(b, sp, cur, as, ufin, d_res64, d_viol, d_sizes_cur, c_cap, stream);
                cudaMemcpyAsync(h_viol, d_viol, sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream);
            }
            if (P.problem == SCOPI_GPU_VISCOUS || viscous_friction())
                launch_gamma_update(sp, cur, as, last_lambda, d_sizes_cur, c_cap, stream);
        } else {
            last_lambda = nullptr;
            *h_viol = 0;
        }
        last_M = M;
        cudaEventRecord(ev[2], stream);
        launch_update(b, sp, ufin, ustride, urot, d_sizes_cur, stream);
        if (periodic) launch_periodic_wrap(b, box, P.dim, stream);
        cudaEventRecord(ev[3], stream);
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "step");
        double viol;
        std::memcpy(&viol, h_viol, sizeof(double));
        stats.violation = viol;
        stats.contacts = C;
        float t_step = 0, t_solve = 0;
        cudaEventElapsedTime(&t_step, ev[0], ev[3]);
        cudaEventElapsedTime(&t_solve, ev[1], ev[2]);
        stats.ms_step = t_step;
        stats.ms_solve = t_solve;
        stats.ms_apgd_kernel = ms_apgd;
        stats.steps += 1;
        // the contacts of this step become the previous ones (std::swap, solver.hpp:301)
        std::swap(cur, old);
        std::swap(d_sizes_cur, d_sizes_old);
        has_old = true;
        if (!stats.converged) stats.status = SCOPI_GPU_ENOCONV;
        return 0;
    }

    void accumulate_stats(bool fp32) {
        stats.iterations += h_result->iterations;
        stats.backtracks += h_result->backtracks;
        stats.restarts += h_result->restarts;
        if (fp32) stats.fp32_iterations += h_result->iterations;
        stats.converged = stats.converged && h_result->converged;
    }

    // FP32 APGD iterations with an FP64 outer correction: after each FP32 solve the
    // residual g = Q lambda + c and the violation are recomputed in FP64, and APGD is
    // rerun in FP32 on the correction delta (linear term g, constraint lambda + delta in K),
    // up to mixed_max_corrections times; if the violation is still above the target, one
    // last correction runs in FP64.
    int mixed_solve(double dt, long long M, float& ms_apgd) {
        Bodies b = bodies();
        StepParams sp = step_params(dt);
        const int per = cvec_per();
        SphSolve<float> sbs{};
        SolveBuffers<float> sb{};
        if (sphere_mode()) {
            launch_pack_nc<float>(as.bn, as.cvec, d_nc32, d_sizes_cur, c_cap, stream);
            launch_pack_inc<float>(na, inc.ptr, inc.idx, as.bn, d_incv32, 2 * c_cap, stream);
            sbs = sph_buffers<float>(d_nc32, d_incv32, d_imt32, d_lam32, d_us32);
        } else {
            launch_convert<double, float>(as.bn, d_bn32, 3 * c_cap, &d_sizes_cur->C, 3, stream);
            launch_convert<double, float>(as.bai, d_bai32, 3 * c_cap, &d_sizes_cur->C, 3, stream);
            launch_convert<double, float>(as.baj, d_baj32, 3 * c_cap, &d_sizes_cur->C, 3, stream);
            if (friction_rows())
                launch_convert<double, float>(as.bP, d_bP32, 18 * c_cap, &d_sizes_cur->C, 18, stream);
            else
                launch_convert<double, float>(inc.coef, d_coef32, 12 * c_cap, &d_sizes_cur->C, 12, stream);
            launch_convert<double, float>(as.cvec, d_cvec32, per * c_cap, &d_sizes_cur->C, per, stream);
            sb.bn = d_bn32;
            sb.bai = d_bai32;
            sb.baj = d_baj32;
            sb.bP = d_bP32;
            sb.cvec = d_cvec32;
            sb.shift = nullptr;
            sb.inc_ptr = inc.ptr;
            sb.inc_idx = inc.idx;
            sb.inc_coef = d_coef32;
            for (int k = 0; k < 3; ++k) {
                sb.lam[k] = d_lam32[k];
                sb.u[k] = d_u32[k];
            }
            sb.g = d_g32;
            sb.partials = d_partials;
            sb.barrier = d_barrier;
            sb.result = d_result;
        }
        float total = 0.0f;
        // correction solves start from the step size the previous solve ended with (same Q):
        // from the default alpha their first steps alpha * g can be below the tolerance and
        // the solve stops at once, leaving the violation where it was
        double alpha0 = 0.0;
        auto solve32 = [&]() -> int {
            cudaEventRecord(ev_a[0], stream);
            int r = sphere_mode() ? run_apgd_sph<float>(sbs, max_sph32, dt, P.tolerance, P.max_ite, M, alpha0)
                                  : run_apgd<float>(sb, d_invm32, max_blocks32, dt, P.tolerance, P.max_ite, M, alpha0);
            cudaEventRecord(ev_a[1], stream);
            if (r) return r;
            if (std::isfinite(h_result->lipsch) && h_result->lipsch > 0.0) alpha0 = 1.0 / h_result->lipsch;
            cudaEventSynchronize(ev_a[1]);
            float ms = 0;
            cudaEventElapsedTime(&ms, ev_a[0], ev_a[1]);
            total += ms;
            accumulate_stats(true);
            return 0;
        };
        // FP64 correction, when the FP32 corrections end above the target: FP32 steps cannot
        // resolve a correction below their rounding floor (4 eps |lambda|)
        auto solve64 = [&]() -> int {
            cudaEventRecord(ev_a[0], stream);
            int r;
            if (sphere_mode()) {
                launch_pack_nc<double>(as.bn, d_res64, d_nc64, d_sizes_cur, c_cap, stream);
                SphSolve<double> s64 = sph_buffers<double>(d_nc64, d_incv64, d_imt64, d_lam64, d_us64);
                s64.shift = d_lamacc;
                r = run_apgd_sph<double>(s64, max_sph64, dt, P.tolerance, P.max_ite, M, alpha0);
                // the FP64 residual reads (n, c) from the same records
                launch_pack_nc<double>(as.bn, as.cvec, d_nc64, d_sizes_cur, c_cap, stream);
            } else {
                SolveBuffers<double> s64{};
                s64.bn = as.bn;
                s64.bai = as.bai;
                s64.baj = as.baj;
                s64.bP = as.bP;
                s64.cvec = d_res64;
                s64.shift = d_lamacc;
                s64.inc_ptr = inc.ptr;
                s64.inc_idx = inc.idx;
                s64.inc_coef = inc.coef;
                for (int k = 0; k < 3; ++k) {
                    s64.lam[k] = d_lam64[k];
                    s64.u[k] = d_u64[k];
                }
                s64.g = d_g64;
                s64.partials = d_partials;
                s64.barrier = d_barrier;
                s64.result = d_result;
                r = run_apgd<double>(s64, d_invm64, max_blocks64, dt, P.tolerance, P.max_ite, M, alpha0);
            }
            cudaEventRecord(ev_a[1], stream);
            if (r) return r;
            cudaEventSynchronize(ev_a[1]);
            float ms = 0;
            cudaEventElapsedTime(&ms, ev_a[0], ev_a[1]);
            total += ms;
            accumulate_stats(false);
            stats.corrections += 1;
            launch_accumulate(sp, cur, as, d_lamacc, d_lam64[h_result->lam_buf], d_sizes_cur, c_cap, 0, stream);
            return 0;
        };
        int rc = solve32();
        if (rc) return rc;
        launch_accumulate(sp, cur, as, d_lamacc, d_lam32[h_result->lam_buf], d_sizes_cur, c_cap, 1, stream);
        bool fp64_done = false;
        for (int k = 0;; ++k) {
            cudaMemsetAsync(d_viol, 0, sizeof(unsigned long long), stream);
            if (sphere_mode()) {
                launch_sph_particle64(na, P.dim, P.problem, inc.ptr, d_incv64, as.slot, d_invm64, d_lamacc, d_usfin,
                                      stream);
                launch_sph_residual64(nin, P.dim, P.problem, d_cij, d_nc64, as.slot, dt * dt, d_usfin, d_res64, d_viol,
                                      d_sizes_cur, c_cap, stream);
            } else {
                launch_particle_pass64(b, sp, cur, as, inc, d_invm64, d_lamacc, d_ufin, stream);
                launch_residual64(b, sp, cur, as, d_ufin, d_res64, d_viol, d_sizes_cur, c_cap, stream);
            }
            cudaMemcpyAsync(h_viol, d_viol, sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream);
            cudaError_t e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) return cuda_fail(e, "mixed residual");
            double viol;
            std::memcpy(&viol, h_viol, sizeof(double));
            if (viol <= P.mixed_violation_tol || fp64_done) break;
            if (k >= P.mixed_max_corrections) {
                rc = solve64();
                if (rc) return rc;
                fp64_done = true;
                continue;
            }
            // correction solve: linear term = FP64 residual, solution offset = lambda so far
            if (sphere_mode()) {
                launch_pack_nc<float>(as.bn, d_res64, d_nc32, d_sizes_cur, c_cap, stream);
                sbs.shift = d_lamacc;
            } else {
                launch_convert<double, float>(d_res64, d_cvec32, per * c_cap, &d_sizes_cur->C, per, stream);
                sb.shift = d_lamacc;
            }
            rc = solve32();
            if (rc) return rc;
            stats.corrections += 1;
            launch_accumulate(sp, cur, as, d_lamacc, d_lam32[h_result->lam_buf], d_sizes_cur, c_cap, 0, stream);
        }
        ms_apgd = total;
        return 0;
    }
};

extern "C" {

void scopi_gpu_default_params(scopi_gpu_params* p, int32_t dim) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->dim = dim;
    p->problem = SCOPI_GPU_NOFRICTION;
    p->vap = SCOPI_GPU_VAP_FIXED;
    p->contact_method = SCOPI_GPU_KDTREE;
    p->precision = SCOPI_GPU_FP64;
    p->dynamic_descent = 1;
    p->max_ite = 10000;
    p->dmax = 2.0;
    p->kd_tree_radius = 17.0;
    p->alpha = 0.05;
    p->tolerance = 1e-7;
    p->mu = 0.1;
    p->gamma = 0.0;
    p->gamma_min = -2.0;
    p->gamma_tol = 1e-6;
    p->mixed_violation_tol = 1e-6;
    p->mixed_max_corrections = 3;
    p->device = 0;
    p->initial_step = SCOPI_GPU_STEP_AUTO;
    p->fixed_point_tol = 1e-6;
    p->fixed_point_max_iter = 1000;
}

int32_t scopi_gpu_create(const scopi_gpu_params* p, scopi_gpu_handle** out) {
    if (!p || !out) {
        scopi_gpu::set_global_error("null argument");
        return SCOPI_GPU_EINVAL;
    }
    *out = nullptr;
    if (p->dim != 2 && p->dim != 3) {
        scopi_gpu::set_global_error("dim must be 2 or 3");
        return SCOPI_GPU_EINVAL;
    }
    const bool loop = p->problem == SCOPI_GPU_FRICTION_FIXED_POINT || p->problem == SCOPI_GPU_VISCOUS_FRICTION;
    if (p->problem < 0 || p->problem > 4 || p->vap < 0 || p->vap > 1 || p->contact_method < 0 ||
        p->contact_method > 1 || p->precision < 0 || p->precision > 1 || p->alpha <= 0 || p->max_ite < 1 ||
        (loop && (!(p->fixed_point_tol >= 0) || p->fixed_point_max_iter < 1))) {
        scopi_gpu::set_global_error("invalid parameter");
        return SCOPI_GPU_EINVAL;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= p->device) {
        scopi_gpu::set_global_error2("no CUDA device: ", cudaGetErrorString(e));
        return SCOPI_GPU_ECUDA;
    }
    auto* h = new scopi_gpu_handle();
    h->P = *p;
    if (p->problem == SCOPI_GPU_FRICTION_FIXED_POINT) {
        h->fixed_point = true;
        h->P.problem = SCOPI_GPU_FRICTION;  // the Friction problem plus the s term and the loop
    }
    for (int d = 0; d < p->dim; ++d)
        if (p->periodic[d]) {
            if (!(p->box_upper[d] > p->box_lower[d])) {
                delete h;
                scopi_gpu::set_global_error("periodic box: upper bound must exceed the lower bound");
                return SCOPI_GPU_EINVAL;
            }
            h->periodic = true;
        }
    for (int d = 0; d < 3; ++d) {
        h->box.lo[d] = p->box_lower[d];
        h->box.up[d] = p->box_upper[d];
        h->box.per[d] = (d < p->dim && p->periodic[d]) ? 1 : 0;
    }
    h->dev = p->device;
    cudaSetDevice(h->dev);
    if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess) {
        scopi_gpu::set_global_error2("cudaStreamCreate: ", cudaGetErrorString(e));
        delete h;
        return SCOPI_GPU_ECUDA;
    }
    int rc = h->alloc_fixed();
    if (rc) {
        scopi_gpu::set_global_error(h->err.c_str());
        scopi_gpu_destroy(h);
        return rc;
    }
    h->launches0 = h->launches();
    *out = h;
    return 0;
}

int32_t scopi_gpu_destroy(scopi_gpu_handle* h) {
    if (!h) return SCOPI_GPU_EINVAL;
    cudaSetDevice(h->dev);
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->drop_graph();
    h->batch_mem.release();
    h->body_mem.release();
    h->cap_mem.release();
    h->fixed_mem.release();
    if (h->h_sizes) cudaFreeHost(h->h_sizes);
    if (h->h_result) cudaFreeHost(h->h_result);
    if (h->h_viol) cudaFreeHost(h->h_viol);
    if (h->h_bar) cudaFreeHost(h->h_bar);
    if (h->h_census) cudaFreeHost(h->h_census);
    if (h->h_se_cand) cudaFreeHost(h->h_se_cand);
    if (h->h_fp_part) cudaFreeHost(h->h_fp_part);
    if (h->h_gcount) cudaFreeHost(h->h_gcount);
    for (auto& x : h->ev)
        if (x) cudaEventDestroy(x);
    for (auto& x : h->ev_a)
        if (x) cudaEventDestroy(x);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return 0;
}

static int32_t upload_particles(scopi_gpu_handle* h, const scopi_gpu_particles* p, long long obs_cap);

int32_t scopi_gpu_set_particles(scopi_gpu_handle* h, const scopi_gpu_particles* p) {
    if (h && h->batch) return h->fail(SCOPI_GPU_EINVAL, "batch handles take their scenes at creation");
    return upload_particles(h, p, -1);
}

// M^-1 of the active bodies (minimization_problem.hpp:11-31): per body 4 slots, 1/m then
// 1/J (3D: x, y, z; 2D: z in the last slot), in FP64 and rounded to FP32, and 1/m alone
// contiguous for the torque-free kernel.
__global__ void k_inverse_mass(int n, int nin, int dim, const double* m, const double* j, double* im64, float* im32,
                               double* imt64, float* imt32) {
    GRID_STRIDE(i, n - nin) {
        const long long b = i + nin;
        double v[4] = {1. / m[b], 0.0, 0.0, 0.0};
        if (dim == 3) {
            for (int d = 0; d < 3; ++d) v[1 + d] = 1. / j[3 * b + d];
        } else {
            v[3] = 1. / j[3 * b + 2];
        }
        for (int d = 0; d < 4; ++d) {
            im64[4 * i + d] = v[d];
            im32[4 * i + d] = (float)v[d];
        }
        imt64[i] = v[0];
        imt32[i] = (float)v[0];
    }
}
static void launch_inverse_mass(int n, int nin, int dim, const double* m, const double* j, double* im64, float* im32,
                                double* imt64, float* imt32, cudaStream_t s) {
    const long long na = (long long)n - nin;
    // the padding slots past the last body stay zero
    cudaMemsetAsync(im64 + 4 * na, 0, 4 * sizeof(double), s);
    cudaMemsetAsync(im32 + 4 * na, 0, 4 * sizeof(float), s);
    cudaMemsetAsync(imt64 + na, 0, sizeof(double), s);
    cudaMemsetAsync(imt32 + na, 0, sizeof(float), s);
    if (na <= 0) return;
    const int blocks = (int)std::min<long long>((na + 255) / 256, 16LL * kSMs);
    k_inverse_mass<<<blocks, 256, 0, s>>>(n, nin, dim, m, j, im64, im32, imt64, imt32);
}

// Census of an uploaded container, on the device (the host would spend ~3 ns per body on it):
// out[0] active superellipsoids, out[1] active spheres, out[2] bodies with a worm index, and
// out[3] the container's rule violations: bit 1 unknown shape, bit 2 an active body that is
// neither a sphere nor a superellipsoid, bit 4 a superellipsoid obstacle, bit 8 a segment in 3D,
// bit 16 an obstacle that is not a plane (refused with superellipsoids only).
__global__ void k_shape_census(const int* shape, const int* worm, int n, int nin, int dim, int* out) {
    int se = 0, sph = 0, wm = 0, bad = 0;
    GRID_STRIDE(i, n) {
        const int sh = shape[i];
        if (sh < 0 || sh > 3) {
            bad |= 1;
        } else {
            if (i >= nin && sh != SCOPI_GPU_SPHERE && sh != SCOPI_GPU_SUPERELLIPSOID) bad |= 2;
            if (i < nin && sh == SCOPI_GPU_SUPERELLIPSOID) bad |= 4;
            if (sh == SCOPI_GPU_SEGMENT && dim != 2) bad |= 8;
            if (i < nin && sh != SCOPI_GPU_PLANE) bad |= 16;
        }
        if (i >= nin) {
            if (sh == SCOPI_GPU_SUPERELLIPSOID) ++se;
            else if (sh == SCOPI_GPU_SPHERE) ++sph;
        }
        if (worm && worm[i] >= 0) ++wm;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        se += __shfl_down_sync(0xffffffffu, se, o);
        sph += __shfl_down_sync(0xffffffffu, sph, o);
        wm += __shfl_down_sync(0xffffffffu, wm, o);
        bad |= __shfl_down_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (se) atomicAdd(out, se);
        if (sph) atomicAdd(out + 1, sph);
        if (wm) atomicAdd(out + 2, wm);
        if (bad) atomicOr(out + 3, bad);
    }
}

static int32_t upload_particles(scopi_gpu_handle* h, const scopi_gpu_particles* p, long long obs_cap) {
    if (!h || !p || p->n < 0 || p->nb_inactive < 0 || p->nb_inactive > p->n || p->n >= (1LL << 30))
        return h ? h->fail(SCOPI_GPU_EINVAL, "invalid particle container") : SCOPI_GPU_EINVAL;
    if (!p->shape || !p->pos || !p->q || !p->v || !p->omega || !p->vd || !p->omega_d || !p->f || !p->m || !p->j ||
        !p->radius || !p->length)
        return h->fail(SCOPI_GPU_EINVAL, "null particle array");
    const int n = (int)p->n, nin = (int)p->nb_inactive;
    if ((long long)nin * (n - nin) >= (1LL << 31) && obs_cap < 0)
        return h->fail(SCOPI_GPU_EUNSUPPORTED, "obstacles x active bodies must stay below 2^31");
    if (h->periodic) {
        if (h->batch) return h->fail(SCOPI_GPU_EUNSUPPORTED, "periodic box: single scenes of spheres, no worms");
        if ((long long)nin * (n - nin) * (1 + h->P.dim) >= (1LL << 31))
            return h->fail(SCOPI_GPU_EUNSUPPORTED, "obstacles x active bodies and copies must stay below 2^31");
        for (int i = 0; i < nin; ++i) {
            for (int d = 0; d < 3; ++d)
                if (p->vd[3 * (size_t)i + d] != 0.0 || p->omega_d[3 * (size_t)i + d] != 0.0)
                    return h->fail(SCOPI_GPU_EUNSUPPORTED, "periodic box: obstacles must be static");
            // the reference copies such an obstacle too and pairs it with its original through
            // the plane-plane case its dispatcher leaves unimplemented (an empty contact)
            for (int d = 0; d < h->P.dim; ++d)
                if (h->box.per[d] && p->pos[3 * (size_t)i + d] - h->P.dmax < h->box.lo[d])
                    return h->fail(SCOPI_GPU_EUNSUPPORTED,
                                   "periodic box: an obstacle lies within dmax of a periodic lower bound");
        }
    }
    cudaSetDevice(h->dev);
    if (n != h->n || nin != h->nin || h->batch) {
        cudaStreamSynchronize(h->stream);  // the buffers in use are released
        int rc = h->alloc_bodies(n, nin, obs_cap);
        if (rc) return rc;
        if (h->c_cap == 0) {
            rc = h->alloc_contacts(std::max<long long>(8192, 6LL * (n - nin) + 2LL * nin * 64));
            if (rc) return rc;
        } else {
            h->has_old = false;
        }
    }
    cudaStream_t s = h->stream;
    auto up = [&](void* dst, const void* src, size_t bytes) { cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s); };
    // shapes (and worm indices, staged in the link buffer) first, then their census on the
    // device while the other fields copy; a container the census refuses leaves the handle
    // without particles until the next valid upload
    up(h->d_shape, p->shape, n * sizeof(int));
    if (p->worm) up(h->d_links, p->worm, n * sizeof(int));
    cudaMemsetAsync(h->d_census, 0, 4 * sizeof(int), s);
    if (n > 0)
        k_shape_census<<<(int)std::min<long long>((n + 255) / 256, 8LL * kSMs), 256, 0, s>>>(
            h->d_shape, p->worm ? h->d_links : nullptr, n, nin, h->P.dim, h->d_census);
    cudaMemcpyAsync(h->h_census, h->d_census, 4 * sizeof(int), cudaMemcpyDeviceToHost, s);
    up(h->d_pos, p->pos, 3 * (size_t)n * sizeof(double));
    up(h->d_q, p->q, 4 * (size_t)n * sizeof(double));
    up(h->d_v, p->v, 3 * (size_t)n * sizeof(double));
    up(h->d_omega, p->omega, 3 * (size_t)n * sizeof(double));
    up(h->d_vd, p->vd, 3 * (size_t)n * sizeof(double));
    up(h->d_omega_d, p->omega_d, 3 * (size_t)n * sizeof(double));
    up(h->d_f, p->f, 3 * (size_t)n * sizeof(double));
    up(h->d_m, p->m, (size_t)n * sizeof(double));
    up(h->d_j, p->j, 3 * (size_t)n * sizeof(double));
    up(h->d_radius, p->radius, (size_t)n * sizeof(double));
    up(h->d_length, p->length, (size_t)n * sizeof(double));
    launch_inverse_mass(n, nin, h->P.dim, h->d_m, h->d_j, h->d_invm64, h->d_invm32, h->d_imt64, h->d_imt32, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return h->cuda_fail(e, "set_particles");
    const int n_se = h->h_census[0], n_worm = h->h_census[2], bad = h->h_census[3];
    auto refuse = [&](int code, const char* msg) {
        h->n = h->nin = h->na = 0;  // the device holds a container that was not accepted
        return h->fail(code, msg);
    };
    if (bad & 1) return refuse(SCOPI_GPU_EINVAL, "unknown shape");
    if (bad & 2) return refuse(SCOPI_GPU_EUNSUPPORTED, "active bodies must be spheres or superellipsoids");
    if (bad & 4) return refuse(SCOPI_GPU_EUNSUPPORTED, "superellipsoid obstacles are not supported");
    if (bad & 8) return refuse(SCOPI_GPU_EUNSUPPORTED, "segments are 2D only");
    if (n_se > 0) {
        // obstacles of superellipsoid scenes are planes: the reference leaves
        // superellipsoid-segment pairs unimplemented (closest_points.hpp:919-931)
        if (bad & 16) return refuse(SCOPI_GPU_EUNSUPPORTED, "superellipsoid scenes: plane obstacles only");
        if (n_worm > 0) return refuse(SCOPI_GPU_EUNSUPPORTED, "worms: scenes of spheres");
        if (!p->axes || !p->squareness) return refuse(SCOPI_GPU_EINVAL, "superellipsoid axes / squareness missing");
        if (h->P.problem == SCOPI_GPU_VISCOUS || h->P.problem == SCOPI_GPU_VISCOUS_FRICTION)
            return refuse(SCOPI_GPU_EUNSUPPORTED, "superellipsoids: NoFriction and Friction problems");
        if (h->batch) return refuse(SCOPI_GPU_EUNSUPPORTED, "batches hold sphere scenes");
        if (h->periodic) return refuse(SCOPI_GPU_EUNSUPPORTED, "periodic box: single scenes of spheres, no worms");
        const bool d3 = h->P.dim == 3;  // 2D: (rx, ry) and e
        for (int i = nin; i < n; ++i) {
            if (p->shape[i] != SCOPI_GPU_SUPERELLIPSOID) continue;
            const double* r = p->axes + 3 * (size_t)i;
            const double* q = p->squareness + 2 * (size_t)i;
            if (!(r[0] > 0 && r[1] > 0 && (!d3 || r[2] > 0)) || !(q[0] > 0 && q[0] < 2 && (!d3 || (q[1] > 0 && q[1] < 2))))
                return refuse(SCOPI_GPU_EINVAL, "superellipsoid: semi-axes > 0 and squareness in (0, 2)");
        }
        // semi-axes and squareness are read for superellipsoid scenes only
        up(h->d_axes, p->axes, 3 * (size_t)n * sizeof(double));
        up(h->d_sq, p->squareness, 2 * (size_t)n * sizeof(double));
    }
    // worms: a link per pair of consecutive active spheres with the same worm index
    std::vector<int> links;
    if (n_worm > 0) {
        for (int i = 0; i < n; ++i) {
            if (p->worm[i] < 0) continue;
            if (i < nin || p->shape[i] != SCOPI_GPU_SPHERE) return refuse(SCOPI_GPU_EINVAL, "worms are runs of active spheres");
            if (i + 1 < n && p->worm[i + 1] == p->worm[i]) links.push_back(i);
        }
        if (!links.empty() && (h->batch || h->P.problem != SCOPI_GPU_NOFRICTION))
            return refuse(SCOPI_GPU_EUNSUPPORTED, "worms: single scenes with the NoFriction problem");
        if (!links.empty() && h->periodic)
            return refuse(SCOPI_GPU_EUNSUPPORTED, "periodic box: single scenes of spheres, no worms");
    }
    h->has_se = n_se > 0;
    h->n_links = (int)links.size();
    if (!links.empty()) up(h->d_links, links.data(), links.size() * sizeof(int));
    if (n_se > 0 || !links.empty()) {
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return h->cuda_fail(e, "set_particles");
    }
    return 0;
}

int32_t scopi_gpu_set_state(scopi_gpu_handle* h, const scopi_gpu_particles* p) {
    if (!h || !p) return h ? h->fail(SCOPI_GPU_EINVAL, "set_state: null container") : SCOPI_GPU_EINVAL;
    if (h->batch) return h->fail(SCOPI_GPU_EINVAL, "batch handles take their scenes at creation");
    if (h->n == 0) return h->fail(SCOPI_GPU_EINVAL, "set_state: no particles (call set_particles first)");
    if (p->n != h->n || p->nb_inactive != h->nin)
        return h->fail(SCOPI_GPU_EINVAL, "set_state: n and nb_inactive must match the container on the device");
    cudaSetDevice(h->dev);
    cudaStream_t s = h->stream;
    const size_t n = (size_t)h->n;
    cudaError_t e = cudaSuccess;
    auto up = [&](void* dst, const double* src, size_t count) {
        if (src && e == cudaSuccess) e = cudaMemcpyAsync(dst, src, count * n * sizeof(double), cudaMemcpyHostToDevice, s);
    };
    up(h->d_pos, p->pos, 3);
    up(h->d_q, p->q, 4);
    up(h->d_v, p->v, 3);
    up(h->d_omega, p->omega, 3);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return h->cuda_fail(e, "set_state");
    return 0;
}

int32_t scopi_gpu_get_particles(scopi_gpu_handle* h, scopi_gpu_particles* o) {
    if (!h || !o) return SCOPI_GPU_EINVAL;
    cudaSetDevice(h->dev);
    cudaStream_t s = h->stream;
    const size_t n = (size_t)h->n;
    if (o->pos) cudaMemcpyAsync(o->pos, h->d_pos, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (o->q) cudaMemcpyAsync(o->q, h->d_q, 4 * n * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (o->v) cudaMemcpyAsync(o->v, h->d_v, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (o->omega) cudaMemcpyAsync(o->omega, h->d_omega, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return h->cuda_fail(e, "get_particles");
    return 0;
}

int32_t scopi_gpu_run(scopi_gpu_handle* h, double dt, int64_t total_it, int64_t initial_iter) {
    if (!h) return SCOPI_GPU_EINVAL;
    if (h->n == 0) return h->fail(SCOPI_GPU_EINVAL, "no particles");
    cudaSetDevice(h->dev);
    int status = 0;
    for (int64_t it = initial_iter; it < total_it; ++it) {
        int rc = h->batch ? h->step_batch(dt) : h->step(dt);
        if (rc < 0) return rc;
        if (h->stats.status == SCOPI_GPU_ENOCONV) status = SCOPI_GPU_ENOCONV;
    }
    return status;
}

int32_t scopi_gpu_detect(scopi_gpu_handle* h, int64_t* nout) {
    if (!h) return SCOPI_GPU_EINVAL;
    if (h->n == 0) return h->fail(SCOPI_GPU_EINVAL, "no particles");
    cudaSetDevice(h->dev);
    int rc = h->detect_and_assemble(0.0, false);
    if (rc) return rc;
    cudaMemcpyAsync(h->h_sizes, h->d_sizes_cur, sizeof(Sizes), cudaMemcpyDeviceToHost, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->cuda_fail(e, "detect");
    std::swap(h->cur, h->old);
    std::swap(h->d_sizes_cur, h->d_sizes_old);
    h->has_old = true;
    if (nout) *nout = h->h_sizes->C;
    return 0;
}

int32_t scopi_gpu_get_contacts(scopi_gpu_handle* h, int64_t cap, int64_t* nout, int64_t* ci, int64_t* cj, double* dij,
                               double* nij, double* pi, double* pj, double* gamma) {
    if (!h) return SCOPI_GPU_EINVAL;
    cudaSetDevice(h->dev);
    Sizes sz{};
    if (h->has_old) cudaMemcpy(&sz, h->d_sizes_old, sizeof(Sizes), cudaMemcpyDeviceToHost);
    const long long C = sz.C;
    if (nout) *nout = C;
    const long long k = std::min<long long>(C, cap);
    if (k <= 0) return 0;
    std::vector<int> tmp(k);
    if (ci) {
        cudaMemcpy(tmp.data(), h->old.ci, k * sizeof(int), cudaMemcpyDeviceToHost);
        for (long long x = 0; x < k; ++x) ci[x] = tmp[x];
    }
    if (cj) {
        cudaMemcpy(tmp.data(), h->old.cj, k * sizeof(int), cudaMemcpyDeviceToHost);
        for (long long x = 0; x < k; ++x) cj[x] = tmp[x];
    }
    if (dij) cudaMemcpy(dij, h->old.dij, k * sizeof(double), cudaMemcpyDeviceToHost);
    if (nij) cudaMemcpy(nij, h->old.nij, 3 * k * sizeof(double), cudaMemcpyDeviceToHost);
    if (pi) cudaMemcpy(pi, h->old.pi, 3 * k * sizeof(double), cudaMemcpyDeviceToHost);
    if (pj) cudaMemcpy(pj, h->old.pj, 3 * k * sizeof(double), cudaMemcpyDeviceToHost);
    if (gamma) cudaMemcpy(gamma, h->old.gamma, k * sizeof(double), cudaMemcpyDeviceToHost);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return h->cuda_fail(e, "get_contacts");
    return 0;
}

int32_t scopi_gpu_get_lambda(scopi_gpu_handle* h, int64_t cap, int64_t* nout, double* lambda) {
    if (!h) return SCOPI_GPU_EINVAL;
    cudaSetDevice(h->dev);
    const long long M = h->last_lambda ? h->last_M : 0;
    if (h->viscous_friction() && M > 0) {
        // four slots per contact on the device; the reference's rows are 1, 2 or 4 per contact
        // by mode (lagrange_multiplier.hpp:358-379), in contact order
        const long long C = M / 4;
        std::vector<double> l4(M);
        std::vector<int> md(C);
        cudaError_t e = cudaMemcpy(l4.data(), h->last_lambda, M * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(md.data(), h->as.vflag, C * sizeof(int), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return h->cuda_fail(e, "get_lambda");
        std::vector<double> rows;
        rows.reserve(M);
        for (long long c = 0; c < C; ++c) {
            const int k = md[c] == 2 ? 4 : (md[c] == 1 ? 2 : 1);
            for (int r = 0; r < k; ++r) rows.push_back(l4[4 * c + r]);
        }
        if (nout) *nout = (int64_t)rows.size();
        if (lambda) std::copy(rows.begin(), rows.begin() + std::min<long long>((long long)rows.size(), cap), lambda);
        return 0;
    }
    if (nout) *nout = M;
    const long long k = std::min<long long>(M, cap);
    if (k > 0 && lambda) {
        cudaError_t e = cudaMemcpy(lambda, h->last_lambda, k * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return h->cuda_fail(e, "get_lambda");
    }
    return 0;
}

int32_t scopi_gpu_get_stats(scopi_gpu_handle* h, scopi_gpu_stats* out) {
    if (!h || !out) return SCOPI_GPU_EINVAL;
    *out = h->stats;
    return 0;
}

int32_t scopi_gpu_amat(scopi_gpu_handle* h, const double* u, double* out) {
    if (!h || !u || !out) return SCOPI_GPU_EINVAL;
    cudaSetDevice(h->dev);
    Sizes sz{};
    cudaMemcpy(&sz, h->d_sizes_old, sizeof(Sizes), cudaMemcpyDeviceToHost);
    double *du = nullptr, *dout = nullptr;
    cudaMalloc(&du, 6 * (size_t)std::max(h->na, 1) * sizeof(double));
    cudaMalloc(&dout, 3 * (size_t)std::max(sz.C, 1) * sizeof(double));
    cudaMemcpy(du, u, 6 * (size_t)h->na * sizeof(double), cudaMemcpyHostToDevice);
    launch_amat(h->bodies(), h->step_params(0.0), h->old, h->d_sizes_old, h->c_cap, du, dout, h->stream);
    cudaStreamSynchronize(h->stream);
    cudaMemcpy(out, dout, 3 * (size_t)sz.C * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(du);
    cudaFree(dout);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return h->cuda_fail(e, "amat");
    return 0;
}

int32_t scopi_gpu_get_se_starts(scopi_gpu_handle* h, int64_t cap, int64_t* n, double* u) {
    if (!h) return SCOPI_GPU_EINVAL;
    cudaSetDevice(h->dev);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->cuda_fail(e, "get_se_starts");
    const long long cand = h->has_se ? *h->h_se_cand : 0;
    if (n) *n = cand;
    const long long k = std::min<long long>(cand, cap);
    if (k > 0 && u) {
        e = cudaMemcpy(u, h->d_se_u, 4 * k * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return h->cuda_fail(e, "get_se_starts");
    }
    return 0;
}

int32_t scopi_gpu_set_contacts(scopi_gpu_handle* h, int64_t n, const int64_t* ci, const int64_t* cj,
                               const double* dij, const double* nij, const double* pi, const double* pj) {
    if (!h) return SCOPI_GPU_EINVAL;
    if (h->batch) return h->fail(SCOPI_GPU_EINVAL, "set_contacts: single-scene handles only");
    if (h->n == 0) return h->fail(SCOPI_GPU_EINVAL, "set_contacts: no particles");
    if (n < 0 || n > 0x7fffffffLL || (n > 0 && (!ci || !cj || !dij || !nij || !pi || !pj)))
        return h->fail(SCOPI_GPU_EINVAL, "set_contacts: null array or count out of range");
    std::vector<int> i32(n), j32(n);
    for (int64_t k = 0; k < n; ++k) {
        if (ci[k] < 0 || ci[k] >= h->n || cj[k] < 0 || cj[k] >= h->n)
            return h->fail(SCOPI_GPU_EINVAL, "set_contacts: body index out of range");
        i32[k] = (int)ci[k];
        j32[k] = (int)cj[k];
    }
    cudaSetDevice(h->dev);
    if (n > h->c_cap) {
        int rc = h->alloc_contacts(std::max<long long>((long long)(1.3 * (double)n) + 1024, 2 * h->c_cap));
        if (rc) return rc;
    }
    cudaError_t e = cudaSuccess;
    if (n > 0) {
        e = cudaMemcpy(h->old.ci, i32.data(), n * sizeof(int), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(h->old.cj, j32.data(), n * sizeof(int), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(h->old.dij, dij, n * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(h->old.nij, nij, 3 * n * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(h->old.pi, pi, 3 * n * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(h->old.pj, pj, 3 * n * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(h->old.gamma, 0, n * sizeof(double));
    }
    Sizes s{};
    s.C = (int)n;
    if (e == cudaSuccess) e = cudaMemcpy(h->d_sizes_old, &s, sizeof(Sizes), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return h->cuda_fail(e, "set_contacts");
    h->has_old = true;
    h->last_lambda = nullptr;
    return 0;
}

int32_t scopi_gpu_atmat(scopi_gpu_handle* h, const double* f, double* out) {
    if (!h || !f || !out) return SCOPI_GPU_EINVAL;
    cudaSetDevice(h->dev);
    Sizes sz{};
    cudaMemcpy(&sz, h->d_sizes_old, sizeof(Sizes), cudaMemcpyDeviceToHost);
    double *df = nullptr, *dout = nullptr;
    cudaMalloc(&df, 3 * (size_t)std::max(sz.C, 1) * sizeof(double));
    cudaMalloc(&dout, 6 * (size_t)std::max(h->na, 1) * sizeof(double));
    cudaMemcpy(df, f, 3 * (size_t)sz.C * sizeof(double), cudaMemcpyHostToDevice);
    launch_atmat(h->bodies(), h->step_params(0.0), h->old, h->d_sizes_old, h->c_cap, df, dout, h->stream);
    cudaStreamSynchronize(h->stream);
    cudaMemcpy(out, dout, 6 * (size_t)h->na * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(df);
    cudaFree(dout);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return h->cuda_fail(e, "atmat");
    return 0;
}

const char* scopi_gpu_last_error(scopi_gpu_handle* h) { return h ? h->err.c_str() : g_global_error; }

int64_t scopi_gpu_kernel_launches(scopi_gpu_handle* h) { return h ? h->launches() - h->launches0 : 0; }

void* scopi_gpu_get_stream(scopi_gpu_handle* h) { return h ? (void*)h->stream : nullptr; }

int32_t scopi_gpu_batch_create(const scopi_gpu_params* p, int32_t n_scenes, const scopi_gpu_particles* scenes,
                               scopi_gpu_handle** out) {
    if (!p || !scenes || !out || n_scenes <= 0) {
        scopi_gpu::set_global_error("scopi_gpu_batch_create: invalid argument");
        return SCOPI_GPU_EINVAL;
    }
    *out = nullptr;
    if (p->problem != SCOPI_GPU_NOFRICTION && p->problem != SCOPI_GPU_FRICTION && p->problem != SCOPI_GPU_VISCOUS) {
        scopi_gpu::set_global_error("scopi_gpu_batch_create: batches solve NoFriction, Friction and Viscous scenes");
        return SCOPI_GPU_EUNSUPPORTED;
    }
    if (p->problem != SCOPI_GPU_NOFRICTION && p->precision != SCOPI_GPU_FP64) {
        scopi_gpu::set_global_error("scopi_gpu_batch_create: Friction and Viscous batches run in FP64");
        return SCOPI_GPU_EUNSUPPORTED;
    }
    long long ntot = 0, nin_tot = 0;
    for (int s = 0; s < n_scenes; ++s) {
        const scopi_gpu_particles& sc = scenes[s];
        if (sc.n < 0 || sc.nb_inactive < 0 || sc.nb_inactive > sc.n || !sc.shape || !sc.pos || !sc.q || !sc.v ||
            !sc.omega || !sc.vd || !sc.omega_d || !sc.f || !sc.m || !sc.j || !sc.radius || !sc.length) {
            scopi_gpu::set_global_error("scopi_gpu_batch_create: invalid scene container");
            return SCOPI_GPU_EINVAL;
        }
        if (sc.worm)
            for (long long i = 0; i < sc.n; ++i)
                if (sc.worm[i] >= 0) {
                    scopi_gpu::set_global_error("scopi_gpu_batch_create: worms: single scenes only");
                    return SCOPI_GPU_EUNSUPPORTED;
                }
        ntot += sc.n;
        nin_tot += sc.nb_inactive;
    }
    if (ntot >= (1LL << 30)) {
        scopi_gpu::set_global_error("scopi_gpu_batch_create: too many bodies");
        return SCOPI_GPU_EINVAL;
    }
    int rc = scopi_gpu_create(p, out);
    if (rc) return rc;
    scopi_gpu_handle* h = *out;
    h->batch = true;
    h->n_scenes = n_scenes;
    h->sc_n.resize(n_scenes);
    h->sc_nin.resize(n_scenes);
    h->sc_obs_start.resize(n_scenes);
    h->sc_act_start.resize(n_scenes);
    // concatenation: every scene's obstacles first, then every scene's active bodies
    std::vector<int32_t> shape(ntot), scene_of(ntot);
    std::vector<double> pos(3 * ntot), q(4 * ntot), v(3 * ntot), om(3 * ntot), vd(3 * ntot), od(3 * ntot), f(3 * ntot),
        m(ntot), jj(3 * ntot), rad(ntot), len(ntot);
    auto copy_body = [&](const scopi_gpu_particles& sc, long long src, long long dst, int s) {
        shape[dst] = sc.shape[src];
        scene_of[dst] = s;
        for (int d = 0; d < 3; ++d) {
            pos[3 * dst + d] = sc.pos[3 * src + d];
            v[3 * dst + d] = sc.v[3 * src + d];
            om[3 * dst + d] = sc.omega[3 * src + d];
            vd[3 * dst + d] = sc.vd[3 * src + d];
            od[3 * dst + d] = sc.omega_d[3 * src + d];
            f[3 * dst + d] = sc.f[3 * src + d];
            jj[3 * dst + d] = sc.j[3 * src + d];
        }
        for (int d = 0; d < 4; ++d) q[4 * dst + d] = sc.q[4 * src + d];
        m[dst] = sc.m[src];
        rad[dst] = sc.radius[src];
        len[dst] = sc.length[src];
    };
    long long ob = 0, ac = nin_tot;
    std::vector<int> obs_a0(nin_tot + 1), obs_off(nin_tot + 1, 0), sc_obs0(n_scenes), sc_obs1(n_scenes),
        sc_p0(n_scenes), sc_p1(n_scenes);
    for (int s = 0; s < n_scenes; ++s) {
        const scopi_gpu_particles& sc = scenes[s];
        h->sc_n[s] = (int)sc.n;
        h->sc_nin[s] = (int)sc.nb_inactive;
        h->sc_obs_start[s] = ob;
        h->sc_act_start[s] = ac;
        sc_obs0[s] = (int)ob;
        sc_p0[s] = (int)(ac - nin_tot);
        for (long long k = 0; k < sc.nb_inactive; ++k) {
            obs_a0[ob] = (int)(ac - nin_tot);
            obs_off[ob + 1] = obs_off[ob] + (int)(sc.n - sc.nb_inactive);
            copy_body(sc, k, ob++, s);
        }
        for (long long k = sc.nb_inactive; k < sc.n; ++k) copy_body(sc, k, ac++, s);
        sc_obs1[s] = (int)ob;
        sc_p1[s] = (int)(ac - nin_tot);
    }
    // cell-key shift: scene s is moved to x = s * pitch so the scenes occupy disjoint cells
    double wmax = 0.0, rmax = 0.0;
    std::vector<double> xmin(n_scenes, 1e300);
    for (long long b = 0; b < ntot; ++b) {
        const int s = scene_of[b];
        xmin[s] = std::min(xmin[s], pos[3 * b] - len[b] - rad[b]);
        rmax = std::max(rmax, rad[b]);
    }
    for (long long b = 0; b < ntot; ++b) {
        const int s = scene_of[b];
        wmax = std::max(wmax, pos[3 * b] + len[b] + rad[b] - xmin[s]);
    }
    // pairs of different scenes are rejected explicitly, so the gap between scenes only
    // keeps them out of each other's cells (efficiency, not correctness)
    const double hcell = 2.0 * rmax + p->dmax;
    const double pitch = wmax + 2.0 * hcell + 1e-9;
    std::vector<double> shift(n_scenes);
    for (int s = 0; s < n_scenes; ++s) shift[s] = s * pitch - (xmin[s] < 1e299 ? xmin[s] : 0.0);
    // cell-list capacity for the shifted layout at the initial extent in y (z), twice over
    // for bodies that spread while falling; coarser cells are used past this capacity
    {
        double cells = std::ceil(n_scenes * pitch / std::max(hcell, 1e-12)) + 1.0;
        for (int d = 1; d < p->dim; ++d) {
            double lo = 1e300, hi = -1e300;
            for (long long b = nin_tot; b < ntot; ++b) {
                lo = std::min(lo, pos[3 * b + d]);
                hi = std::max(hi, pos[3 * b + d]);
            }
            cells *= (hi >= lo ? std::ceil((hi - lo) / std::max(hcell, 1e-12)) : 0.0) + 1.0;
        }
        h->cell_cap_hint = (long long)std::min(2.0 * cells, 64.0e6);
    }
    std::vector<int> order(n_scenes);
    for (int s = 0; s < n_scenes; ++s) order[s] = s;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return (sc_p1[a] - sc_p0[a]) > (sc_p1[b] - sc_p0[b]); });
    {
        const int largest = n_scenes > 0 ? sc_p1[order[0]] - sc_p0[order[0]] : 0;
        int nb = 0;
        while (nb < n_scenes && 2 * (sc_p1[order[nb]] - sc_p0[order[nb]]) >= largest) ++nb;
        h->batch_n_big = nb;
    }
    scopi_gpu_particles cat{ntot, nin_tot, shape.data(), pos.data(), q.data(), v.data(), om.data(), vd.data(),
                            od.data(), f.data(), m.data(), jj.data(), rad.data(), len.data()};
    rc = upload_particles(h, &cat, obs_off[nin_tot]);
    if (rc) {
        scopi_gpu::set_global_error(h->err.c_str());
        scopi_gpu_destroy(h);
        *out = nullptr;
        return rc;
    }
    cudaError_t e;
#define BA(ptr, cnt) \
    if ((e = h->alloc(h->batch_mem, ptr, (cnt))) != cudaSuccess) return h->cuda_fail(e, "cudaMalloc(batch)");
    BA(h->d_scene, ntot) BA(h->d_shift, n_scenes) BA(h->d_obs_a0, nin_tot + 1) BA(h->d_obs_off, nin_tot + 1)
    BA(h->d_sc_obs0, n_scenes) BA(h->d_sc_obs1, n_scenes) BA(h->d_sc_p0, n_scenes) BA(h->d_sc_p1, n_scenes)
    BA(h->d_order, n_scenes) BA(h->d_sc_o0, n_scenes) BA(h->d_sc_o1, n_scenes) BA(h->d_sc_a0, n_scenes)
    BA(h->d_sc_a1, n_scenes) BA(h->d_bstats, n_scenes) BA(h->d_obs_snap, 7 * nin_tot + 7)
#undef BA
    cudaMemcpy(h->d_scene, scene_of.data(), ntot * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_shift, shift.data(), n_scenes * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_obs_a0, obs_a0.data(), (nin_tot + 1) * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_obs_off, obs_off.data(), (nin_tot + 1) * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_sc_obs0, sc_obs0.data(), n_scenes * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_sc_obs1, sc_obs1.data(), n_scenes * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_sc_p0, sc_p0.data(), n_scenes * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_sc_p1, sc_p1.data(), n_scenes * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_order, order.data(), n_scenes * sizeof(int), cudaMemcpyHostToDevice);
    e = cudaMemset(h->d_bstats, 0, n_scenes * sizeof(BatchSceneStats));
    if (e != cudaSuccess) return h->cuda_fail(e, "batch set-up");
    return 0;
}

int32_t scopi_gpu_batch_get_scene(scopi_gpu_handle* h, int32_t scene, scopi_gpu_particles* o) {
    if (!h || !o || !h->batch || scene < 0 || scene >= h->n_scenes) return SCOPI_GPU_EINVAL;
    cudaSetDevice(h->dev);
    const long long nin_s = h->sc_nin[scene], na_s = h->sc_n[scene] - nin_s;
    struct Seg {
        long long src, dst, cnt;
    } segs[2] = {{h->sc_obs_start[scene], 0, nin_s}, {h->sc_act_start[scene], nin_s, na_s}};
    for (const Seg& g : segs) {
        if (g.cnt <= 0) continue;
        if (o->pos)
            cudaMemcpy(o->pos + 3 * g.dst, h->d_pos + 3 * g.src, 3 * g.cnt * sizeof(double), cudaMemcpyDeviceToHost);
        if (o->q) cudaMemcpy(o->q + 4 * g.dst, h->d_q + 4 * g.src, 4 * g.cnt * sizeof(double), cudaMemcpyDeviceToHost);
        if (o->v) cudaMemcpy(o->v + 3 * g.dst, h->d_v + 3 * g.src, 3 * g.cnt * sizeof(double), cudaMemcpyDeviceToHost);
        if (o->omega)
            cudaMemcpy(o->omega + 3 * g.dst, h->d_omega + 3 * g.src, 3 * g.cnt * sizeof(double),
                       cudaMemcpyDeviceToHost);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return h->cuda_fail(e, "batch_get_scene");
    return 0;
}

int32_t scopi_gpu_batch_get_scene_stats(scopi_gpu_handle* h, int32_t scene, scopi_gpu_scene_stats* out) {
    if (!h || !out || !h->batch || scene < 0 || scene >= h->n_scenes) return SCOPI_GPU_EINVAL;
    if ((int)h->h_bstats.size() != h->n_scenes) {
        std::memset(out, 0, sizeof(*out));
        return 0;
    }
    const BatchSceneStats& s = h->h_bstats[scene];
    out->contacts = s.contacts;
    out->iterations = s.iterations;
    out->fp32_iterations = s.fp32_iterations;
    out->backtracks = s.backtracks;
    out->restarts = s.restarts;
    out->corrections = s.corrections;
    out->converged = s.converged;
    out->violation = s.violation;
    return 0;
}

int32_t scopi_gpu_batch_block_threads(scopi_gpu_handle* h) {
    if (!h) return 0;
    return h->batch_threads ? h->batch_threads : h->batch_bt_used;
}

int32_t scopi_gpu_batch_tile(scopi_gpu_handle* h) {
    if (!h) return 0;
    return h->batch_tile ? h->batch_tile : h->batch_tile_used;
}

int32_t scopi_gpu_batch_set_shape(scopi_gpu_handle* h, int32_t threads, int32_t tile) {
    if (!h || !h->batch) return SCOPI_GPU_EINVAL;
    if (h->stats.steps > 0) return h->fail(SCOPI_GPU_EINVAL, "the launch shape is fixed once the batch has stepped");
    if (!(threads == 0 && tile == 0) && !scopi_gpu::batch_shape_valid(threads, tile))
        return h->fail(SCOPI_GPU_EINVAL, "launch shape must be 256 x 2|4, 512 x 1|2, 1024 x 1|2 or 2048 x 1|2 (0, 0 = autotune)");
    h->batch_threads = threads;
    h->batch_tile = tile;
    return 0;
}

int32_t scopi_gpu_test_barrier_stall(scopi_gpu_handle* h) {
    if (!h) return SCOPI_GPU_EINVAL;
    if (h->batch) return h->fail(SCOPI_GPU_EINVAL, "a batch's APGD launch has no grid barrier");
    h->stall_next = true;
    return 0;
}

int32_t scopi_gpu_batch_set_block_threads(scopi_gpu_handle* h, int32_t threads) {
    if (!h || !h->batch) return SCOPI_GPU_EINVAL;
    if (h->stats.steps > 0) return h->fail(SCOPI_GPU_EINVAL, "the block size is fixed once the batch has stepped");
    if (threads != 0 && !scopi_gpu::batch_shape_valid(threads, batch_default_tile(threads)))
        return h->fail(SCOPI_GPU_EINVAL, "threads per scene must be 256, 512, 1024 or 2048 (0 = autotune)");
    h->batch_threads = threads;
    return 0;
}

}  // extern "C"
