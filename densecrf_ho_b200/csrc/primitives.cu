// Deterministic device-wide integer primitives (no float atomics anywhere).
#include "primitives.cuh"

namespace dcrf {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr unsigned kFull = 0xffffffffu;

// Exclusive scan of one int per thread across a 256-thread block; also
// returns the block total.
__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_tot, int* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < kScanThreads / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(kFull, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kScanThreads / 32) warp_tot[lane] = s;
    }
    __syncthreads();
    int prefix = w ? warp_tot[w - 1] : 0;
    *total = warp_tot[kScanThreads / 32 - 1];
    return prefix + x - v;
}

__global__ void scan_reduce_kernel(const int* __restrict__ in, int n, int* __restrict__ bsum) {
    __shared__ int wt[kScanThreads / 32];
    long base = (long)blockIdx.x * kScanTile;
    int s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        long idx = base + (long)threadIdx.x * kScanItems + i;
        if (idx < n) s += in[idx];
    }
    int tot;
    block_exclusive_scan(s, wt, &tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

// Single block: in-place exclusive scan of the per-tile sums.
__global__ void scan_top_kernel(int* __restrict__ bsum, int nb, int* __restrict__ d_total) {
    __shared__ int wt[kScanThreads / 32];
    int carry = 0;
    for (int base = 0; base < nb; base += kScanTile) {
        int v[kScanItems];
        int s = 0;
#pragma unroll
        for (int i = 0; i < kScanItems; i++) {
            int idx = base + threadIdx.x * kScanItems + i;
            v[i] = idx < nb ? bsum[idx] : 0;
            s += v[i];
        }
        int tot;
        int ex = block_exclusive_scan(s, wt, &tot);
        int run = carry + ex;
#pragma unroll
        for (int i = 0; i < kScanItems; i++) {
            int idx = base + threadIdx.x * kScanItems + i;
            if (idx < nb) bsum[idx] = run;
            run += v[i];
        }
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0 && d_total) *d_total = carry;
}

__global__ void scan_apply_kernel(const int* in, int* out, int n, const int* __restrict__ bsum) {
    __shared__ int wt[kScanThreads / 32];
    long base = (long)blockIdx.x * kScanTile + (long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        long idx = base + i;
        v[i] = idx < n ? in[idx] : 0;
        s += v[i];
    }
    int tot;
    int run = bsum[blockIdx.x] + block_exclusive_scan(s, wt, &tot);
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        long idx = base + i;
        if (idx < n) out[idx] = run;
        run += v[i];
    }
}

// ---------------------------------------------------------------- sort --
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadix = 256;

__global__ void radix_hist_kernel(const int* __restrict__ keys, int n, int shift, int ntiles,
                                  int* __restrict__ hist) {
    __shared__ int h[kRadix];
    for (int i = threadIdx.x; i < kRadix; i += blockDim.x) h[i] = 0;
    __syncthreads();
    long base = (long)blockIdx.x * kSortTile;
    for (int i = threadIdx.x; i < kSortTile; i += kSortThreads) {
        long idx = base + i;
        if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & (kRadix - 1)], 1);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kRadix; i += blockDim.x) hist[(long)i * ntiles + blockIdx.x] = h[i];
}

// Stable scatter: within a tile, elements are ranked among equal digits in
// index order (warp match + per-warp counts), then placed after the tiles
// before it (digit-major scanned histogram).
__global__ void radix_scatter_kernel(const int* __restrict__ keys_in, const int* __restrict__ vals_in,
                                     int n, int shift, int ntiles, const int* __restrict__ offs,
                                     int* __restrict__ keys_out, int* __restrict__ vals_out) {
    __shared__ int running[kRadix];
    __shared__ int wcnt[kSortThreads / 32][kRadix];
    for (int i = threadIdx.x; i < kRadix; i += blockDim.x) {
        running[i] = 0;
        for (int w = 0; w < kSortThreads / 32; w++) wcnt[w][i] = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    long base = (long)blockIdx.x * kSortTile;
    for (int it = 0; it < kSortItems; it++) {
        long idx = base + (long)it * kSortThreads + threadIdx.x;
        bool valid = idx < n;
        int key = valid ? keys_in[idx] : 0;
        int val = valid ? vals_in[idx] : 0;
        int dig = valid ? ((key >> shift) & (kRadix - 1)) : kRadix;
        unsigned peers = __match_any_sync(kFull, dig);
        int rank = __popc(peers & lt_mask);
        bool leader = (__ffs(peers) - 1) == lane;
        int cnt = __popc(peers);
        if (valid && leader) wcnt[w][dig] = cnt;
        __syncthreads();
        if (valid) {
            int pos = running[dig] + rank;
            for (int ww = 0; ww < w; ww++) pos += wcnt[ww][dig];
            long o = (long)offs[(long)dig * ntiles + blockIdx.x] + pos;
            keys_out[o] = key;
            vals_out[o] = val;
        }
        __syncthreads();
        if (valid && leader) {
            atomicAdd(&running[dig], cnt);
            wcnt[w][dig] = 0;
        }
        __syncthreads();
    }
}

}  // namespace

void exclusive_scan(const int* in, int* out, int n, int* d_total, ScanScratch& s, cudaStream_t st) {
    if (n <= 0) {
        if (d_total) DCRF_CUDA(cudaMemsetAsync(d_total, 0, sizeof(int), st));
        return;
    }
    int nb = ceil_div(n, kScanTile);
    int* bs = s.block_sums.ensure(nb);
    launch(scan_reduce_kernel, nb, kScanThreads, 0, st, in, n, bs);
    launch(scan_top_kernel, 1, kScanThreads, 0, st, bs, nb, d_total);
    launch(scan_apply_kernel, nb, kScanThreads, 0, st, in, out, n, bs);
    DCRF_LAUNCH_CHECK();
}

void radix_sort_pairs(int* keys, int* vals, int n, int key_bits, SortScratch& s, cudaStream_t st) {
    if (n <= 1 || key_bits <= 0) return;
    int ntiles = ceil_div(n, kSortTile);
    int* ka = s.keys_alt.ensure(n);
    int* va = s.vals_alt.ensure(n);
    int* hist = s.hist.ensure((size_t)kRadix * ntiles);
    int *kin = keys, *vin = vals, *kout = ka, *vout = va;
    int passes = 0;
    for (int shift = 0; shift < key_bits; shift += 8, passes++) {
        launch(radix_hist_kernel, ntiles, kSortThreads, 0, st, kin, n, shift, ntiles, hist);
        exclusive_scan(hist, hist, kRadix * ntiles, nullptr, s.scan, st);
        launch(radix_scatter_kernel, ntiles, kSortThreads, 0, st, kin, vin, n, shift, ntiles, hist, kout,
                                                             vout);
        DCRF_LAUNCH_CHECK();
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    if (kin != keys) {
        DCRF_CUDA(cudaMemcpyAsync(keys, kin, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
        DCRF_CUDA(cudaMemcpyAsync(vals, vin, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
    }
}

}  // namespace dcrf
