// Device-wide integer primitives used to build the lattice deterministically:
// an exclusive prefix sum and a stable LSD radix sort of (key, value) pairs.
#pragma once
#include "common.cuh"

namespace dcrf {

// Scratch owned by the caller so repeated builds do not reallocate.
struct ScanScratch {
    DevBuf<int> block_sums;
};

// out[i] = sum_{j<i} in[i]; in may alias out.  If d_total is non-null the
// grand total is written there (device pointer).  n < 2^31.
void exclusive_scan(const int* in, int* out, int n, int* d_total, ScanScratch& s,
                    cudaStream_t st);

struct SortScratch {
    DevBuf<int> keys_alt, vals_alt, hist;
    ScanScratch scan;
};

// Stable sort of keys[0..n) (0 <= key < 2^key_bits) carrying vals; the
// result is left in keys/vals.  Equal keys keep their input order, so a
// sort of (vertex id, entry index) pairs yields per-vertex entry lists in
// increasing entry order.
void radix_sort_pairs(int* keys, int* vals, int n, int key_bits, SortScratch& s, cudaStream_t st);

}  // namespace dcrf
