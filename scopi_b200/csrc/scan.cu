// scan.cu -- device-wide exclusive prefix sum over int32 with a device-resident length.
//
// Three launches (tile scan, scan of tile totals, tile offsets), grids sized from
// the capacity so the sequence can be captured in a CUDA graph while the actual
// length lives in device memory.  Deterministic (integer).
#include "kernels.cuh"

namespace scopi_gpu {

namespace {
constexpr int kScanThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kScanThreads * kItems;

__device__ int block_exclusive_scan(int x, int* smem_warp, int& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int v = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) smem_warp[warp] = v;
    __syncthreads();
    const int nw = blockDim.x >> 5;
    if (warp == 0) {
        int w = lane < nw ? smem_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < nw) smem_warp[lane] = w;
    }
    __syncthreads();
    const int warp_off = warp > 0 ? smem_warp[warp - 1] : 0;
    total = smem_warp[nw - 1];
    __syncthreads();
    return warp_off + v - x;
}

__global__ void k_scan_tiles(const int* __restrict__ in, int* __restrict__ out, const int* __restrict__ n_dev, int n_host,
                             int* __restrict__ tile_sum) {
    __shared__ int sw[32];
    const int n = n_dev ? *n_dev : n_host;
    const long long base = (long long)blockIdx.x * kTile;
    if (base >= n) {
        if (threadIdx.x == 0) tile_sum[blockIdx.x] = 0;
        return;
    }
    int vals[kItems];
    int acc = 0;
    const long long my = base + (long long)threadIdx.x * kItems;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const long long idx = my + k;
        vals[k] = idx < n ? in[idx] : 0;
        acc += vals[k];
    }
    int total;
    int off = block_exclusive_scan(acc, sw, total);
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const long long idx = my + k;
        if (idx < n) out[idx] = off;
        off += vals[k];
    }
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

__global__ void k_scan_tile_sums(int* __restrict__ tile_sum, const int* __restrict__ n_dev, int n_host,
                                 int* __restrict__ total_out) {
    __shared__ int sw[32];
    const int n = n_dev ? *n_dev : n_host;
    const int ntiles = (n + kTile - 1) / kTile;
    int carry = 0;
    for (int base = 0; base < ntiles; base += blockDim.x) {
        const int idx = base + threadIdx.x;
        const int x = idx < ntiles ? tile_sum[idx] : 0;
        int tot;
        const int ex = block_exclusive_scan(x, sw, tot);
        if (idx < ntiles) tile_sum[idx] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && total_out) *total_out = carry;
}

__global__ void k_scan_add(int* __restrict__ out, const int* __restrict__ n_dev, int n_host,
                           const int* __restrict__ tile_sum) {
    const int n = n_dev ? *n_dev : n_host;
    const long long base = (long long)blockIdx.x * kTile;
    if (base >= n || blockIdx.x == 0) return;
    const int add = tile_sum[blockIdx.x];
    for (int k = threadIdx.x; k < kTile; k += blockDim.x) {
        const long long idx = base + k;
        if (idx < n) out[idx] += add;
    }
}
}  // namespace

size_t scan_work_ints(long long n_max) { return (size_t)((n_max + kTile - 1) / kTile) + 1; }

void scan_exclusive(const int* in, int* out, const int* n_dev, int n_host, long long n_max, int* total_dev, int* work,
                    cudaStream_t s, long long* launches) {
    const int tiles = (int)((n_max + kTile - 1) / kTile);
    if (tiles <= 0) {
        return;
    }
    k_scan_tiles<<<tiles, kScanThreads, 0, s>>>(in, out, n_dev, n_host, work);
    k_scan_tile_sums<<<1, 1024, 0, s>>>(work, n_dev, n_host, total_dev);
    k_scan_add<<<tiles, kScanThreads, 0, s>>>(out, n_dev, n_host, work);
    if (launches) *launches += 3;
}

}  // namespace scopi_gpu
