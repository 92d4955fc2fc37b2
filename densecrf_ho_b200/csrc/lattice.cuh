// Device-resident permutohedral lattice: construction and filtering.
//
// Layout in HBM (all arrays are owned by the Lattice):
//   offset[N*(d+1)], bary[N*(d+1)], rank[N*(d+1)]  pixel-major, as the
//       reference's offset_ / barycentric_ / rank_ (src/permutohedral.cpp:166-170)
//   vkeys[M*d]      int16 key of each vertex, vertex ids = first-occurrence order
//   nbr[(d+1)*M]    int2 (n1+1, n2+1): blur neighbours of each vertex per axis,
//                   shifted by one so that row 0 of a value buffer is the zero
//                   row standing in for "absent" (src/permutohedral.cpp:490-516)
//   seg_start[M+1], seg_pix[E], seg_w[E]   splat lists: for each vertex the
//                   (pixel, weight) pairs that touch it, in increasing
//                   (pixel, remainder) order, E = N*(d+1).  Splatting then
//                   gathers in exactly the order in which the reference's
//                   scatter accumulates, without float atomics.
//   value buffers   [(M+1)][L] floats (ordered filter: [(M+1)][L][20]).
#pragma once
#include "common.cuh"
#include "primitives.cuh"

#include <vector>

namespace dcrf {

// What the slice kernel does with the filtered value v of (pixel i, label k).
struct SliceEpilogue {
    const float* norm = nullptr;  // multiply by norm[i] (symmetric normalisation)
    float scale = 1.0f;           // then by this (Potts: -w); exactly 1 = skip
    bool potts = false;           // apply norm / scale at all
    const float* scale_vec = nullptr;  // per-label scale instead of `scale` (DiagonalCompatibility)
    const float* base = nullptr;  // then out = base[...] + coef * v
    float coef = 1.0f;
    bool zero_base = false;       // out = 0.0f + coef * v  (Eigen fill(0); +=)
};

// LP dual-gap sums folded into an ordered slice (see ord_slice_kernel).
struct GapFusion {
    const float* alpha = nullptr;
    const float* u = nullptr;
    const float* Q = nullptr;
    double* partials = nullptr;  // [2][slice_grid(N*L)]
    const float* su = nullptr;   // clique conditional gradient (lp_sp), or none
};

// Packed ordered-filter bin indices of rescale(Q) (min / max at qminmax[0..1]).
void rescaled_bins(float2* bins, const float* Q, long n, const float* qminmax, cudaStream_t st);
// Blocks of the element-wise slice kernels for n elements.
int slice_grid(long n);
// Capacity, in floats, of the fixed scratch array of compute_noalloc.
size_t noalloc_scratch_floats();
// Bounded device waits (bulk-copy splat) that ran out on the current device.
unsigned long long bulk_wait_timeouts();

// The units a filter launch covers.  Without `n`, every unit of the
// launch's range.  With it (a batched solve), only the units of the images
// still running: image i owns units [base[i], base[i+1]) of the launch's
// domain (list positions, vertex ids or slice tiles), and the live images'
// units are numbered consecutively, pre[r] being the number of units of the
// live images before the r-th (n + 1 entries, written on the device each
// iteration).  Work for finished images is then never launched, and the
// kernels loop over the live units with grids sized for the device, not for
// the batch.
struct Live {
    const int* n = nullptr;     // number of live images (device), or nullptr
    const int* img = nullptr;   // their ids, ascending (device)
    const long* base = nullptr; // the domain: B + 1 ascending unit offsets
    const long* pre = nullptr;  // live prefix: n + 1 entries
    int images = 0;             // images of the domain (B), when known: all live -> no search
};

#ifdef __CUDACC__
// Units of a launch over `count` units, or over its live images' units.
__device__ __forceinline__ long live_total(const Live& lv, long count) { return lv.n ? lv.pre[*lv.n] : count; }
// Live unit u -> its image and its unit within that image.
__device__ __forceinline__ int live_locate(const Live& lv, long u, long& local) {
    int lo = 0, hi = *lv.n;  // pre[lo] <= u < pre[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (lv.pre[mid] <= u) lo = mid;
        else hi = mid;
    }
    local = u - lv.pre[lo];
    return lv.img[lo];
}
// Live unit u -> its unit in the domain (the identity without live images).
// With every image live the live units are the domain's units in order, so
// no search is needed.
__device__ __forceinline__ long live_unit(const Live& lv, long u) {
    if (!lv.n) return u;
    if (*lv.n == lv.images) return lv.base[0] + u;
    long local;
    const int img = live_locate(lv, u, local);
    return lv.base[img] + local;
}
#endif

// Launch shapes of the plain filter for L = 21 (Lattice::splat_blur /
// slice).  Every shape computes the same arithmetic; only the speed
// differs.  Lattice::tune_shape picks them by timing, once per device and
// problem class (L, d, size), and caches the choice for the process.
struct FilterShape {
    // Splat of the lists up to the huge-list threshold (L = 21):
    // 0 = staged splat_kernel for the long lists, one thread per (vertex,
    //     label) for the short ones;
    // 1 = warp splat for the long lists, the thread form for the short ones;
    // 2 = warp splat for every list;
    // 3 = tiled splat (splat_tile21_kernel) for every list;
    // 4 = staged splat_kernel for the long lists, the tiled splat for the
    //     short ones;
    // 5 = bulk-copy splat (splat_bulk21_kernel) for every list.
    int splat_kind = 0;
    int splat_warps = 4;     // vertices (warps) per block of the warp splat: 2, 4 or 8
    int blur_threads = 256;  // threads per block of the float4 blur: 128, 256 or 512
    int slice_tile = 128;    // pixels per block of the tiled slice: 64, 128 or 256
};

struct Lattice {
    int N = 0, d = 0, M = 0;
    FilterShape shape;      // launch shapes in use
    int shape_L = 0;        // the label count they were tuned for (0: defaults)
    int n_long = 0;  // vertices whose splat list exceeds the staging threshold
    int n_huge = 0;  // ... and the (leading) ones whose list is very long
    cudaStream_t stream = nullptr;  // borrowed
    // side stream (highest priority) for splat work that overlaps the rest
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;

    DevBuf<int> offset, rank, seg_start, seg_pix;
    DevBuf<int> vorder, vorder_keys;  // splat visiting order: longest lists first
    DevBuf<float> bary, seg_w;
    DevBuf<int16_t> vkeys;
    DevBuf<int2> nbr;
    DevBuf<float> va, vb;    // filter value buffers
    DevBuf<float2> obins;    // ordered filter: (c_lower, c_upper) per (pixel, label)
    size_t va_floats = 0;    // rows (M+1) * width currently zero-headed

    // build scratch
    DevBuf<int4> ekeys;
    DevBuf<int> table, entry_slot, flags, slot_vid, sort_keys, sort_vals, counts, total;
    DevBuf<float> fscale;
    ScanScratch scan;
    SortScratch sort;

    bool concatenated = false;  // built by concat(): no vertex keys
    DevBuf<int> vimg;           // concat(): image of each vertex
    // concat(): per-image work domains, kDomains rows of (images + 1) longs:
    // the positions in vorder of each image's huge, long and short lists,
    // its vertex ids, its slice tiles (tiles of dom_tile pixels, none
    // crossing an image) and its pixels.
    enum { kDomHuge, kDomLong, kDomShort, kDomVert, kDomTile, kDomPix, kDomains };
    int images = 0;
    std::vector<long> img_pixels;  // host: pixels of each image
    DevBuf<long> dom_base;
    int dom_tile = 0;
    // A batched solve's live images (set around its loop, null otherwise) and
    // this lattice's live prefixes: kDomains rows of (images + 1) longs.
    const int* live_n = nullptr;
    const int* live_img = nullptr;
    const long* live_pre = nullptr;
    // The Live of domain `dom` (no compaction when no live set is attached).
    Live live_of(int dom) const {
        if (!live_n) return Live{};
        return Live{live_n, live_img, dom_base.get() + (long)dom * (images + 1),
                    live_pre + (long)dom * (images + 1), images};
    }
    // Tile size of the L = 21 / L > 2 plain slice for label count L.
    int slice_tile_for(int L) const;
    // Sets the slice-tile domain for label count L (host work, a small copy).
    void prepare_live(int L);

    // features: device [N][d]
    void build(const float* d_features, int d_, int N_);
    // Several images' lattices as one (see Lattice::concat in lattice.cu).
    void concat(const std::vector<const Lattice*>& parts);
    // out/in: device [N][L]; out may alias in.
    void compute(float* out, const float* in, int L, bool reverse, const SliceEpilogue& ep,
                 const float* pre_norm = nullptr);
    // The same in two phases: splat + blur (the vertex values stay in
    // plain_vals), then the slice.  Other work may run between them.
    void splat_blur(const float* in, int L, bool reverse, const float* pre_norm = nullptr);
    void slice(float* out, int L, const SliceEpilogue& ep);
    const float* plain_vals = nullptr;
    int plain_L = 0;
    // The plain filter with its value buffers in a fixed device array instead
    // of memory from cudaMalloc (see dcrf_lattice_compute_noalloc).
    void compute_noalloc(float* out, const float* in, int L, bool reverse);
    // Ordered (upper minus lower, 10-bin) filter of Q in [0,1]; out = epilogue(v).
    void compute_ord(float* out, const float* Q, int L, const SliceEpilogue& ep);
    // The same from precomputed packed bins (lower | upper << 8 per element).
    void compute_ord_bins(float* out, const float2* bins, int L, const SliceEpilogue& ep, const GapFusion* gap);
    // The same in two phases: splat + blur (leaves the vertex values in
    // ord_vals), then the slice.  Other work may run between them.
    void ord_splat_blur(const float2* bins, int L);
    void ord_slice(float* out, const float2* bins, int L, const SliceEpilogue& ep, const GapFusion* gap);
    // Both slices of a two-term sum in one pass: out = eb(b's slice) on top of
    // ea(a's slice), the arithmetic of ord_slice(a, ea with zero_base) then
    // ord_slice(b, eb with base = out); a and b share N and the bins, and each
    // has had its ord_splat_blur.  Runs on a's stream.
    static void ord_slice_pair(float* out, const float2* bins, int L, const Lattice& a, const SliceEpilogue& ea,
                               const Lattice& b, const SliceEpilogue& eb, const GapFusion* gap);
    const float* ord_vals = nullptr;

    // compute_upper_minus_lower_ord_restricted: the ordered filter at the nP
    // pixels pI (device array, strictly ascending) with values rQ [nP][L] ->
    // rout [nP][L]; the other pixels splat their values Q [N][L] (store), or
    // the splat stored by the last store call is reused with the vertex set
    // of that call (store = false).
    void compute_ord_restricted(float* rout, const float* rQ, const int* pI, int nP, const float* Q, int L,
                                bool store, const SliceEpilogue& ep);
    DevBuf<float> r_stored, r_a, r_b;  // [(M + 1)][20][L]: the stored splat, the blur's two buffers
    DevBuf<unsigned char> r_active;    // vertices the pI pixels reach (store call)
    DevBuf<int> r_pos;                 // pixel -> index in pI, or -1
    DevBuf<float2> r_bins, r_ebins;    // bins of rQ and of Q
    int r_L = 0;                       // label count of the stored splat (0: none)

    // Permutohedral::gradient: df [N][d] = d(a^T K b)/d(features); a, b [N][L].
    void gradient(float* df, const float* a, const float* b, int L);

    void ensure_values(size_t row_width);
    void ensure_aux();
    // Times the candidate shapes on this lattice with the input `in` (the
    // first large call) unless the process has tuned this problem class
    // already; outputs are not touched.
    void tune_shape(const float* in, int L, const float* pre_norm);
    // Splat of every list after the first n_huge (whose splat runs on the
    // side stream) into vals, in the form `fs` names; with live images the
    // short lists' launch goes on st_short when one is given.
    void splat_rest(const FilterShape& fs, const float* in, int L, const float* pre_norm, float* vals,
                    bool live, cudaStream_t st, cudaStream_t st_short);
    // Forks the side stream and splats the very long lists there (see
    // lattice.cu); true when it forked (the caller joins ev_join).
    bool splat_huge_fork(const float* in, int L, const float* pre_norm, float* vals, bool fork_anyway);

    Lattice() = default;
    Lattice(const Lattice&) = delete;
    Lattice& operator=(const Lattice&) = delete;
    ~Lattice();
};

}  // namespace dcrf
