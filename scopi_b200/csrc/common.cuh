// common.cuh -- shared device-side types and helpers of the SCoPI B200 engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace scopi_gpu {

constexpr int kSMs = 148;          // B200: 2 dies x 74 SMs
constexpr int kThreads = 256;

// Bodies in device memory (AoS float64, 3 slots per vector, obstacles first).
struct Bodies {
    int n;
    int nin;            // obstacles
    const int* shape;
    double* pos;        // n*3
    double* q;          // n*4
    double* v;          // n*3
    double* omega;      // n*3
    const double* vd;
    const double* omega_d;
    const double* f;
    const double* m;
    const double* j;    // n*3
    const double* radius;
    const double* length;
    const double* axes = nullptr;      // n*3 superellipsoid semi-axes
    const double* sq = nullptr;        // n*2 superellipsoid squareness (e, n)
    // Batches of independent scenes (null for one scene): scene of each body, an x shift
    // per scene applied to the cell keys only (scenes occupy disjoint cell ranges), and
    // per obstacle the active range it can touch (obs_a0: first active index, obs_off:
    // prefix offsets of the per-obstacle ranges, nin + 1 entries).
    const int* scene = nullptr;
    const double* scene_shift = nullptr;
    const int* obs_a0 = nullptr;
    const int* obs_off = nullptr;
};

__host__ __device__ inline double key_x(const Bodies& B, long long b, double x) {
    return B.scene_shift ? x + B.scene_shift[B.scene[b]] : x;
}

// Device-resident sizes written by the detection kernels (graph friendly: no host sizes).
struct Sizes {
    int C;              // contacts
    int C_obs;          // obstacle contacts (rows of bodies < nin come first)
    int n_extra;        // Viscous: second multipliers
    int overflow;       // capacity exceeded somewhere (host grows and redoes the step)
    int ncell;          // cells of the uniform grid
    int n_links;        // worm links: the last n_links contacts (normal and distance negated)
    int pad[2];
};

struct Grid {
    double lo[3];
    double h;           // cell edge
    int nc[3];
    int ncell;
    int ncell1;         // ncell + 1 (length of the cell-start scan)
    double rmax;
};

// Contact list (sorted by (i, j)) and the per-contact Jacobian rows.
struct Contacts {
    int* ci;
    int* cj;
    double* dij;
    double* nij;     // C*3
    double* pi;      // C*3
    double* pj;      // C*3
    double* gamma;   // Viscous / ViscousFriction property
};

// kernel problem codes; FrictionFixedPoint (3) runs the kFriction kernels inside its loop
enum Problem { kNoFriction = 0, kFriction = 1, kViscous = 2, kViscousFriction = 4 };

__host__ __device__ inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// grid-stride helper
#define GRID_STRIDE(i, n) for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)(n); \
                               i += (long long)gridDim.x * blockDim.x)

}  // namespace scopi_gpu
