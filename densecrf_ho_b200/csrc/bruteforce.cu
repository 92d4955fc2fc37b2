// The exact (brute-force) and divide-and-conquer filters of PairwisePotential
// (src/pairwise.cpp:241-380, src/permutohedral.cpp:902-997, 1065-1070):
//
//   apply_bf                          out(l, c) = sum_b k(c, b) Q(l, b)
//   apply_upper_minus_lower_bf        sorted by ind(l, .): sum_{b>c} k - sum_{b<c} k
//   apply_upper_minus_lower_bf_ord    the same with the order taken from Q
//   apply_upper_minus_lower_dc        the sorted sum by recursive halving, the
//                                     cross terms of each halving by a lattice
//                                     filter restricted to the half's vertices
//
// k(c, b) = exp(-|f_c - f_b|^2) on the features the term was added with
// (DenseKernel::features(), unchanged by setKernelParameters), each followed
// by the term's label compatibility.  None of these is on a solver path: the
// reference keeps them for its BRUTE_FORCE energy check.  Every sum is
// carried in the reference's order and precision: k in double (the
// unqualified exp(float) of those files resolves to the double overload),
// accumulated into a float one term at a time; |f_c - f_b|^2 in Eigen 3.2's
// SSE2 order (sqdist below).
#include <atomic>
#include <cmath>
#include <exception>
#include <memory>
#include <mutex>
#include <thread>
#include <type_traits>
#include <vector>

#include "model.cuh"
#include "primitives.cuh"

namespace dcrf {
namespace {

constexpr int kMaxD = 16;   // feature dimensions (as the lattice)
constexpr int kBfTile = 128;  // pixels b per shared-memory tile
constexpr int kBfLabels = 8;  // labels per thread in apply_bf (one exp serves them all)
// apply_bf's grid below this many threads has one label per thread instead:
// on small images filling the SMs matters more than sharing the exp
constexpr long kBfFillThreads = 148L * 1024;
constexpr int kDcLeaf = 30;   // SMALLEST_BLOCK (include/pairwise.h:31)
constexpr int kDcMaxDepth = 64;

// VectorXf::squaredNorm() of featDiff = f_a - f_b as Eigen 3.2 evaluates it
// with SSE2 (Eigen/src/Core/Redux.h, LinearVectorizedTraversal, aligned
// start): the squares in float; with fewer than 4 of them a left-to-right
// sum; otherwise 4-lane packet sums (a second packet accumulator from 8 on,
// pairs of packets per step, the two added lane-wise, then one more packet if
// a whole one is left), the packet reduced as (p0 + p2) + (p1 + p3)
// (predux, SSE/PacketMath.h), then the remaining squares left to right.
// D > 0 fixes the dimension at compile time (the predicates below fold
// away); D = 0 takes it from d.
template <int D>
__device__ __forceinline__ float sqdist(const float* a, const float* b, int d_rt) {
    const int d = D > 0 ? D : d_rt;
    float s[kMaxD];
#pragma unroll
    for (int i = 0; i < kMaxD; i++) {
        float x = i < d ? fsub(a[i], b[i]) : 0.0f;
        s[i] = fmul(x, x);
    }
    const int al = d & ~3;
    float r;
    if (al == 0) {
        r = s[0];
#pragma unroll
        for (int i = 1; i < 4; i++)
            if (i < d) r = fadd(r, s[i]);
        return r;
    }
    float p0 = s[0], p1 = s[1], p2 = s[2], p3 = s[3];
    if (al > 4) {
        float q0 = s[4], q1 = s[5], q2 = s[6], q3 = s[7];
        const int al2 = d & ~7;
        if (al2 > 8) {  // d = 16: one more pair of packets
            p0 = fadd(p0, s[8]);
            p1 = fadd(p1, s[9]);
            p2 = fadd(p2, s[10]);
            p3 = fadd(p3, s[11]);
            q0 = fadd(q0, s[12]);
            q1 = fadd(q1, s[13]);
            q2 = fadd(q2, s[14]);
            q3 = fadd(q3, s[15]);
        }
        p0 = fadd(p0, q0);
        p1 = fadd(p1, q1);
        p2 = fadd(p2, q2);
        p3 = fadd(p3, q3);
        if (al > al2) {  // d in [12, 15]: the packet at 8
            p0 = fadd(p0, s[8]);
            p1 = fadd(p1, s[9]);
            p2 = fadd(p2, s[10]);
            p3 = fadd(p3, s[11]);
        }
    }
    r = fadd(fadd(p0, p2), fadd(p1, p3));
#pragma unroll
    for (int i = 4; i < kMaxD; i++)
        if (i >= al && i < d) r = fadd(r, s[i]);
    return r;
}

// exp(-|f_a - f_b|^2) as the reference forms it: the float norm negated,
// then the double exp.
template <int D>
__device__ __forceinline__ double kval(const float* a, const float* b, int d) {
    return exp((double)(-sqdist<D>(a, b, d)));
}

// out = (float)((double)out + t)
__device__ __forceinline__ float acc_add(float out, double t) { return __double2float_rn(__dadd_rn((double)out, t)); }
__device__ __forceinline__ float acc_sub(float out, double t) { return __double2float_rn(__dsub_rn((double)out, t)); }

// apply_bf (src/pairwise.cpp:368-380): thread per (pixel c, LC labels); the
// pixels b in order, staged through shared memory a tile at a time.
template <int D, int LC>
__global__ void __launch_bounds__(kBfTile) bf_apply_kernel(int N, int L, int d_rt, const float* __restrict__ feat,
                                                           const float* __restrict__ Q, float* __restrict__ out) {
    const int d = D > 0 ? D : d_rt;
    __shared__ float sf[kBfTile * kMaxD];
    __shared__ float sq[kBfTile * LC];
    const int c = blockIdx.x * kBfTile + threadIdx.x;
    const int l0 = blockIdx.y * LC;
    const int nl = min(LC, L - l0);
    float fc[kMaxD];
#pragma unroll
    for (int i = 0; i < kMaxD; i++) fc[i] = (c < N && i < d) ? feat[(long)c * d + i] : 0.0f;
    float acc[LC];
#pragma unroll
    for (int l = 0; l < LC; l++) acc[l] = 0.0f;
    for (int b0 = 0; b0 < N; b0 += kBfTile) {
        const int nb = min(kBfTile, N - b0);
        __syncthreads();
        for (int t = threadIdx.x; t < nb * d; t += kBfTile) sf[t] = feat[(long)b0 * d + t];
        for (int t = threadIdx.x; t < nb * nl; t += kBfTile) {
            const int bi = t / nl, l = t - bi * nl;
            sq[bi * LC + l] = Q[(long)(b0 + bi) * L + l0 + l];
        }
        __syncthreads();
        if (c < N)
            for (int bi = 0; bi < nb; bi++) {
                const double k = kval<D>(fc, sf + bi * d, d);
#pragma unroll
                for (int l = 0; l < LC; l++)
                    if (l < nl) acc[l] = acc_add(acc[l], __dmul_rn(k, (double)sq[bi * LC + l]));
            }
    }
    if (c < N)
        for (int l = 0; l < nl; l++) out[(long)c * L + l0 + l] = acc[l];
}

// apply_upper_minus_lower_bf (src/pairwise.cpp:301-332) and, with ORD,
// apply_upper_minus_lower_bf_ord (:333-367).  Thread per (sorted position c,
// label l = blockIdx.y); f_s = features of ind(l, s).  Plain: + k over b > c,
// then - k over b < c.  ORD: + k over every b with Q(l, ind(l, b)) <=
// Q(l, ind(l, c)), then - k over every b with Q(l, ind(l, b)) >= that.
// Each sweep walks the tiles in order, so every thread meets its b in order.
template <bool ORD, int D>
__global__ void __launch_bounds__(kBfTile) bf_sorted_kernel(int N, int L, int d_rt, const float* __restrict__ feat,
                                                            const int* __restrict__ ind, const float* __restrict__ Q,
                                                            float* __restrict__ out) {
    const int d = D > 0 ? D : d_rt;
    __shared__ float sf[kBfTile * kMaxD];
    __shared__ float sqv[kBfTile];
    const int c = blockIdx.x * kBfTile + threadIdx.x;
    const int l = blockIdx.y;
    float fc[kMaxD];
    float qc = 0.0f;
    if (c < N) {
        const int pc = ind[(long)c * L + l];
#pragma unroll
        for (int i = 0; i < kMaxD; i++) fc[i] = i < d ? feat[(long)pc * d + i] : 0.0f;
        if (ORD) qc = Q[(long)pc * L + l];
    } else {
#pragma unroll
        for (int i = 0; i < kMaxD; i++) fc[i] = 0.0f;
    }
    float acc = 0.0f;
    const int blo = blockIdx.x * kBfTile, bhi = min(N, blo + kBfTile);
    for (int sweep = 0; sweep < 2; sweep++) {
        // plain: upper over tiles [blo, N), lower over [0, bhi)
        const int t0 = ORD || sweep == 1 ? 0 : blo;
        const int t1 = ORD || sweep == 0 ? N : bhi;
        for (int b0 = t0; b0 < t1; b0 += kBfTile) {
            const int nb = min(kBfTile, t1 - b0);
            __syncthreads();
            for (int t = threadIdx.x; t < nb * d; t += kBfTile) {
                const int bi = t / d, i = t - bi * d;
                sf[t] = feat[(long)ind[(long)(b0 + bi) * L + l] * d + i];
            }
            if (ORD)
                for (int t = threadIdx.x; t < nb; t += kBfTile) sqv[t] = Q[(long)ind[(long)(b0 + t) * L + l] * L + l];
            __syncthreads();
            if (c >= N) continue;
            for (int bi = 0; bi < nb; bi++) {
                const int b = b0 + bi;
                bool take;
                if (ORD) take = sweep == 0 ? !(sqv[bi] > qc) : !(sqv[bi] < qc);
                else take = sweep == 0 ? b > c : b < c;
                if (!take) continue;
                const double k = kval<D>(fc, sf + bi * d, d);
                acc = sweep == 0 ? acc_add(acc, k) : acc_sub(acc, k);
            }
        }
    }
    if (c < N) out[(long)c * L + l] = acc;
}

// ------------------------------------------------- divide and conquer ------
//
// apply_upper_minus_lower_sorted_slice(out, min, max) (src/pairwise.cpp:
// 262-300) recurses on the sorted positions: a range of at most 30 is done
// pair by pair (leaf); a larger one is split at middle_low = min + size/2
// (middle_high = middle_low + 1 when size is odd, else equal), recursing on
// [min, middle_high) and [middle_low, max) and then running the lattice
// cross term dc(min, middle_low, middle_high, max) on a lattice of the
// sorted features (src/permutohedral.cpp:902-997).  The tree depends on N
// only and is built on the host.
//
// The cross term of node X = (lo, ml, mh, hi) splats the barycentric
// weights of the pixels in [mh, hi) ("upper") and, separately, of those in
// [lo, ml) ("lower") on the set S_X of vertices reached by either range,
// blurs both over S_X (the other vertices stay 0), and slices: + upper into
// [lo, ml), - lower into [mh, hi).  On the device every node's S_X is a run
// of (node, vertex) items: the items (X, pixel, j) are numbered node by node,
// pixel by pixel, j by j, stably sorted by vertex and then by node, so each
// run lists its splat entries in the reference's pixel order.  The splat,
// the d + 1 blur passes and the neighbour lookups (binary search within the
// node's runs) cover every node at once.  The slice then walks each pixel's
// nodes in the order the recursion visits them (dc_walk_kernel), which also
// fixes the order of the float additions into out.

struct DcNode {
    int lo, hi, ml, mh;  // leaves: ml = mh = -1
    int left, right;     // children, -1 for leaves
    long base;           // first item of an internal node
};

int build_dc_tree(std::vector<DcNode>& nodes, int lo, int hi, int depth, long& items, int d1) {
    require(depth < kDcMaxDepth, DCRF_E_ARG, "divide-and-conquer filter: recursion too deep");
    const int id = (int)nodes.size();
    nodes.push_back(DcNode{lo, hi, -1, -1, -1, -1, 0});
    const int size = hi - lo;
    if (size <= kDcLeaf) return id;
    const int ml = lo + size / 2;
    const int mh = (size % 2 == 0) ? ml : ml + 1;
    nodes[id].ml = ml;
    nodes[id].mh = mh;
    nodes[id].base = items;
    items += (long)((ml - lo) + (hi - mh)) * d1;
    const int l = build_dc_tree(nodes, lo, mh, depth + 1, items, d1);
    const int r = build_dc_tree(nodes, ml, hi, depth + 1, items, d1);
    nodes[id].left = l;
    nodes[id].right = r;
    return id;
}

// Internal nodes by item base, for the item -> node lookup.
__device__ __forceinline__ int item_node(long g, const long* __restrict__ ibase, const int* __restrict__ iid, int ni) {
    int lo = 0, hi = ni - 1;
    while (lo < hi) {  // last internal node with base <= g
        const int mid = (lo + hi + 1) >> 1;
        if (ibase[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return iid[lo];
}

// The pixel and simplex corner of item g of node x.
__device__ __forceinline__ void item_pixel(long g, const DcNode& x, int d1, int& i, int& j) {
    const long local = g - x.base;
    const int k = (int)(local / d1);
    j = (int)(local - (long)k * d1);
    i = x.lo + k;
    if (i >= x.ml) i += x.mh - x.ml;
}

__global__ void dc_gather_features_kernel(int N, int L, int l, int d, const float* __restrict__ feat,
                                          const int* __restrict__ ind, float* __restrict__ sfeat) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)N * d) return;
    const long c = t / d;
    sfeat[t] = feat[(long)ind[c * L + l] * d + (t - c * d)];
}

// Items: node id and vertex (the sort keys), item number (the value).
__global__ void dc_items_kernel(long T, int d1, const DcNode* __restrict__ nodes, const long* __restrict__ ibase,
                                const int* __restrict__ iid, int ni, const int* __restrict__ offset,
                                int* __restrict__ vkey, int* __restrict__ nkey, int* __restrict__ val) {
    const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= T) return;
    const int x = item_node(g, ibase, iid, ni);
    int i, j;
    item_pixel(g, nodes[x], d1, i, j);
    vkey[g] = offset[(long)i * d1 + j];
    nkey[g] = x;
    val[g] = (int)g;
}

__global__ void dc_gather_keys_kernel(long T, const int* __restrict__ val, const int* __restrict__ nkey_by_item,
                                      int* __restrict__ nkey) {
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < T) nkey[p] = nkey_by_item[val[p]];
}

// Vertex of each sorted item, then the run starts of the (node, vertex) order.
__global__ void dc_vert_kernel(long T, int d1, const DcNode* __restrict__ nodes, const int* __restrict__ nkey,
                               const int* __restrict__ val, const int* __restrict__ offset, int* __restrict__ vert) {
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= T) return;
    int i, j;
    item_pixel(val[p], nodes[nkey[p]], d1, i, j);
    vert[p] = offset[(long)i * d1 + j];
}

__global__ void dc_flags_kernel(long T, const int* __restrict__ nkey, const int* __restrict__ vert,
                                int* __restrict__ flag) {
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= T) return;
    flag[p] = (p == 0 || nkey[p] != nkey[p - 1] || vert[p] != vert[p - 1]) ? 1 : 0;
}

// run(p) = (exclusive scan of the flags) + flag - 1; per run its first item,
// node and vertex; per item its run.
__global__ void dc_runs_kernel(long T, const int* __restrict__ flag, const int* __restrict__ scan,
                               const int* __restrict__ nkey, const int* __restrict__ vert, const int* __restrict__ val,
                               int* __restrict__ run_start, int* __restrict__ run_node, int* __restrict__ run_vert,
                               int* __restrict__ run_of_item) {
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= T) return;
    const int r = scan[p] + flag[p] - 1;
    if (flag[p]) {
        run_start[r] = (int)p;
        run_node[r] = nkey[p];
        run_vert[r] = vert[p];
    }
    run_of_item[val[p]] = r;
}

// Per node its runs [node_run[2x], node_run[2x + 1]).
__global__ void dc_node_runs_kernel(int R, const int* __restrict__ run_node, int* __restrict__ node_run) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    const int x = run_node[r];
    if (r == 0 || run_node[r - 1] != x) node_run[2 * x] = r;
    if (r == R - 1 || run_node[r + 1] != x) node_run[2 * x + 1] = r + 1;
}

// The splat: per run, the upper and lower sums of its items' weights in item
// order (= pixel order); values row 0 is the zero row.
__global__ void dc_splat_kernel(int R, long T, int d1, const DcNode* __restrict__ nodes,
                                const int* __restrict__ run_start, const int* __restrict__ run_node,
                                const int* __restrict__ val, const float* __restrict__ bary, float2* __restrict__ va,
                                float2* __restrict__ vb) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r == 0) {
        va[0] = make_float2(0.0f, 0.0f);
        vb[0] = make_float2(0.0f, 0.0f);
    }
    if (r >= R) return;
    const DcNode x = nodes[run_node[r]];
    const long p1 = r + 1 < R ? run_start[r + 1] : T;
    float up = 0.0f, lo = 0.0f;
    for (long p = run_start[r]; p < p1; p++) {
        int i, j;
        item_pixel(val[p], x, d1, i, j);
        const float w = bary[(long)i * d1 + j];
        if (i >= x.mh) up = fadd(up, w);
        else lo = fadd(lo, w);
    }
    va[r + 1] = make_float2(up, lo);
}

// Blur neighbours of each run along each axis, as value rows (0 = absent).
__global__ void dc_neighbours_kernel(int R, int M, int d1, const int* __restrict__ run_node,
                                     const int* __restrict__ run_vert, const int* __restrict__ node_run,
                                     const int2* __restrict__ nbr, int2* __restrict__ rnb) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)R * d1) return;
    const int j = (int)(t / R), r = (int)(t - (long)j * R);
    const int x = run_node[r];
    const int r0 = node_run[2 * x], r1 = node_run[2 * x + 1];
    const int2 nb = nbr[(long)j * M + run_vert[r]];  // vertex ids + 1, 0 = absent
    int out[2];
    const int want[2] = {nb.x - 1, nb.y - 1};
    for (int s = 0; s < 2; s++) {
        out[s] = 0;
        if (want[s] < 0) continue;
        int lo = r0, hi = r1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (run_vert[mid] < want[s]) lo = mid + 1;
            else hi = mid;
        }
        if (lo < r1 && run_vert[lo] == want[s]) out[s] = lo + 1;
    }
    rnb[t] = make_int2(out[0], out[1]);
}

// One blur pass: new = v + 0.5 (v_n1 + v_n2) for both sums
// (src/permutohedral.cpp:941-948, 972-979).
__global__ void dc_blur_kernel(int R, const int2* __restrict__ rnb, const float2* __restrict__ src,
                               float2* __restrict__ dst) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    const int2 nb = rnb[r];
    const float2 a = src[r + 1], x = src[nb.x], y = src[nb.y];
    dst[r + 1] = make_float2(fadd(a.x, fmul(0.5f, fadd(x.x, y.x))), fadd(a.y, fmul(0.5f, fadd(x.y, y.y))));
}

// The contributions of one node to sorted position c.
template <int D>
__device__ __forceinline__ float dc_leaf(float acc, int c, const DcNode& x, int d_rt, const float* __restrict__ sfeat) {
    const int d = D > 0 ? D : d_rt;
    const double alpha = 1.0 / 0.6;  // src/pairwise.cpp:268
    float fc[kMaxD];
#pragma unroll
    for (int i = 0; i < kMaxD; i++) fc[i] = i < d ? sfeat[(long)c * d + i] : 0.0f;
    float fb[kMaxD];
    // lower: out(c) -= k(c, b) alpha for b in [lo, c), then upper: += for b in (c, hi)
    for (int b = x.lo; b < x.hi; b++) {
        if (b == c) continue;
#pragma unroll
        for (int i = 0; i < kMaxD; i++) fb[i] = i < d ? sfeat[(long)b * d + i] : 0.0f;
        const double t = __dmul_rn(kval<D>(fc, fb, d), alpha);
        acc = b < c ? acc_sub(acc, t) : acc_add(acc, t);
    }
    return acc;
}

__device__ __forceinline__ float dc_cross(float acc, int c, const DcNode& x, int d1, const float* __restrict__ bary,
                                          const int* __restrict__ run_of_item, const float2* __restrict__ vals,
                                          float alpha) {
    if (c < x.ml) {  // upper slice: out += w v alpha
        const long g0 = x.base + (long)(c - x.lo) * d1;
        for (int j = 0; j < d1; j++) {
            const float w = bary[(long)c * d1 + j];
            acc = fadd(acc, fmul(fmul(w, vals[run_of_item[g0 + j] + 1].x), alpha));
        }
    } else if (c >= x.mh) {  // lower slice: out -= w v alpha
        const long g0 = x.base + (long)((x.ml - x.lo) + (c - x.mh)) * d1;
        for (int j = 0; j < d1; j++) {
            const float w = bary[(long)c * d1 + j];
            acc = fsub(acc, fmul(fmul(w, vals[run_of_item[g0 + j] + 1].y), alpha));
        }
    }
    return acc;
}

// The path from node `from` down to the leaf holding c, never forking
// (position c is the middle of at most one node, and of none below it).
__device__ __forceinline__ int dc_descend(int from, int c, const DcNode* __restrict__ nodes, int* path) {
    int n = 0, x = from;
    while (nodes[x].left >= 0 && n < kDcMaxDepth) {
        path[n++] = x;
        x = c < nodes[x].mh ? nodes[x].left : nodes[x].right;
    }
    path[n] = x;  // the leaf
    return n;
}

// Sorted position c's value in the order of the recursion: the leaf, then
// its ancestors from the deepest up.  Where c is the middle pixel of an odd
// node P (in both halves), the left half's chain (leaf up to P's left child)
// runs first, then the right half's, then P (which adds nothing to c) and
// its ancestors.
template <int D>
__global__ void dc_walk_kernel(int N, int L, int l, int d, const DcNode* __restrict__ nodes,
                               const float* __restrict__ sfeat, const float* __restrict__ bary,
                               const int* __restrict__ run_of_item, const float2* __restrict__ vals, float alpha,
                               float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const int d1 = d + 1;
    int top[kDcMaxDepth + 1], sub[kDcMaxDepth + 1];
    // path from the root down to the leaf or to the node whose middle c is
    int nt = 0, x = 0, fork = -1;
    while (nodes[x].left >= 0 && nt < kDcMaxDepth) {
        const DcNode& n = nodes[x];
        top[nt++] = x;
        const bool in_left = c < n.mh, in_right = c >= n.ml;
        if (in_left && in_right) {
            fork = x;
            break;
        }
        x = in_left ? n.left : n.right;
    }
    float acc = 0.0f;
    if (fork < 0) {
        acc = dc_leaf<D>(acc, c, nodes[x], d, sfeat);
    } else {
        for (int side = 0; side < 2; side++) {
            const int ns = dc_descend(side == 0 ? nodes[fork].left : nodes[fork].right, c, nodes, sub);
            acc = dc_leaf<D>(acc, c, nodes[sub[ns]], d, sfeat);
            for (int k = ns - 1; k >= 0; k--) acc = dc_cross(acc, c, nodes[sub[k]], d1, bary, run_of_item, vals, alpha);
        }
    }
    for (int k = nt - 1; k >= 0; k--) acc = dc_cross(acc, c, nodes[top[k]], d1, bary, run_of_item, vals, alpha);
    out[(long)c * L + l] = acc;
}

// Calls f with std::integral_constant<int, D>: D = d for the feature
// dimensions of the Gaussian (2), bilateral (5) and three-dimensional
// features, 0 (runtime d) otherwise.
template <typename F>
void with_dim(int d, F&& f) {
    switch (d) {
        case 2: f(std::integral_constant<int, 2>{}); break;
        case 3: f(std::integral_constant<int, 3>{}); break;
        case 5: f(std::integral_constant<int, 5>{}); break;
        default: f(std::integral_constant<int, 0>{}); break;
    }
}

}  // namespace

void Model::apply_bf(int k, bool nonorm, float* out, const float* Q) {
    Term& t = *terms.at(k);
    float* raw = buf(8);
    const bool share = (long)N * ceil_div(L, kBfLabels) >= kBfFillThreads;
    with_dim(t.d, [&](auto dc) {
        constexpr int D = decltype(dc)::value;
        if (share)
            launch(bf_apply_kernel<D, kBfLabels>, dim3(ceil_div(N, kBfTile), ceil_div(L, kBfLabels)), kBfTile, 0,
                   stream, N, L, t.d, (const float*)t.feat.get(), Q, raw);
        else
            launch(bf_apply_kernel<D, 1>, dim3(ceil_div(N, kBfTile), L), kBfTile, 0, stream, N, L, t.d,
                   (const float*)t.feat.get(), Q, raw);
    });
    DCRF_LAUNCH_CHECK();
    apply_compat(k, nonorm, out, raw);
}

void Model::apply_upper_minus_lower_bf(int k, bool nonorm, float* out, const int* ind, const float* Q) {
    Term& t = *terms.at(k);
    float* raw = buf(8);
    const dim3 grid(ceil_div(N, kBfTile), L);
    with_dim(t.d, [&](auto dc) {
        constexpr int D = decltype(dc)::value;
        if (Q)
            launch(bf_sorted_kernel<true, D>, grid, kBfTile, 0, stream, N, L, t.d, (const float*)t.feat.get(), ind, Q,
                   raw);
        else
            launch(bf_sorted_kernel<false, D>, grid, kBfTile, 0, stream, N, L, t.d, (const float*)t.feat.get(), ind,
                   (const float*)nullptr, raw);
    });
    DCRF_LAUNCH_CHECK();
    apply_compat(k, nonorm, out, raw);
}

namespace {

// One host thread's share of the divide-and-conquer filter: its stream, a
// lattice rebuilt for every label it takes, and the work buffers, all kept
// for the whole call so that no buffer is freed (which waits for the
// device) while the other threads' labels run.
struct DcWorker {
    cudaStream_t st = nullptr;
    Lattice lat;
    DevBuf<float> sfeat;
    DevBuf<int> vkey, nkey, nkey_item, val, vert, flag, scan, run_start, run_node, run_vert, run_of_item, node_run,
        total;
    DevBuf<int2> rnb;
    DevBuf<float2> va, vb;
    SortScratch sort;
    ScanScratch sc;
    int* h_total = nullptr;  // pinned
    DcWorker() {
        DCRF_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        DCRF_CUDA(cudaMallocHost(&h_total, sizeof(int)));
        lat.stream = st;
    }
    ~DcWorker() {
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        if (h_total) cudaFreeHost(h_total);
    }
};

struct DcPlan {
    int N, L, d, nn, ni;
    long T;
    const DcNode* nodes;
    const long* ibase;
    const int* iid;
    const float* feat;
    const int* ind;
    float alpha;
    float* raw;
};

// Label l of the divide-and-conquer filter on the worker's stream: the
// lattice of the sorted features, the (node, vertex) runs, the splat and
// blur of every node, then the walk into column l of raw.
void dc_label(DcWorker& w, const DcPlan& p, int l) {
    const int N = p.N, d = p.d, d1 = d + 1, g256 = 256;
    const long T = p.T;
    cudaStream_t st = w.st;
    float* sf = w.sfeat.ensure((size_t)N * d);
    launch(dc_gather_features_kernel, ceil_div((long)N * d, g256), g256, 0, st, N, p.L, l, d, p.feat, p.ind, sf);
    w.lat.build(sf, d, N);
    const float2* vals = nullptr;
    int* roi = w.run_of_item.ensure(std::max<long>(T, 1));
    if (p.ni) {
        int* vk = w.vkey.ensure(T);
        int* nk = w.nkey.ensure(T);
        int* nki = w.nkey_item.ensure(T);
        int* vl = w.val.ensure(T);
        const int gT = ceil_div(T, g256);
        launch(dc_items_kernel, gT, g256, 0, st, T, d1, p.nodes, p.ibase, p.iid, p.ni, (const int*)w.lat.offset.get(),
               vk, nki, vl);
        int vbits = 1, nbits = 1;
        while ((1L << vbits) < w.lat.M) vbits++;
        while ((1L << nbits) < p.nn) nbits++;
        radix_sort_pairs(vk, vl, (int)T, vbits, w.sort, st);
        launch(dc_gather_keys_kernel, gT, g256, 0, st, T, (const int*)vl, (const int*)nki, nk);
        radix_sort_pairs(nk, vl, (int)T, nbits, w.sort, st);
        int* vt = w.vert.ensure(T);
        int* fl = w.flag.ensure(T);
        int* sn = w.scan.ensure(T);
        launch(dc_vert_kernel, gT, g256, 0, st, T, d1, p.nodes, (const int*)nk, (const int*)vl,
               (const int*)w.lat.offset.get(), vt);
        launch(dc_flags_kernel, gT, g256, 0, st, T, (const int*)nk, (const int*)vt, fl);
        int* tot = w.total.ensure(1);
        exclusive_scan(fl, sn, (int)T, tot, w.sc, st);
        DCRF_CUDA(cudaMemcpyAsync(w.h_total, tot, sizeof(int), cudaMemcpyDeviceToHost, st));
        DCRF_CUDA(cudaStreamSynchronize(st));
        const int R = *w.h_total;
        int* rs = w.run_start.ensure(R);
        int* rn = w.run_node.ensure(R);
        int* rv = w.run_vert.ensure(R);
        int* nr = w.node_run.ensure((size_t)2 * p.nn);
        launch(dc_runs_kernel, gT, g256, 0, st, T, (const int*)fl, (const int*)sn, (const int*)nk, (const int*)vt,
               (const int*)vl, rs, rn, rv, roi);
        launch(dc_node_runs_kernel, ceil_div(R, g256), g256, 0, st, R, (const int*)rn, nr);
        float2* a = w.va.ensure((size_t)R + 1);
        float2* b = w.vb.ensure((size_t)R + 1);
        launch(dc_splat_kernel, ceil_div(R, g256), g256, 0, st, R, T, d1, p.nodes, (const int*)rs, (const int*)rn,
               (const int*)vl, (const float*)w.lat.bary.get(), a, b);
        int2* nb = w.rnb.ensure((size_t)R * d1);
        launch(dc_neighbours_kernel, ceil_div((long)R * d1, g256), g256, 0, st, R, w.lat.M, d1, (const int*)rn,
               (const int*)rv, (const int*)nr, (const int2*)w.lat.nbr.get(), nb);
        for (int j = 0; j < d1; j++) {
            launch(dc_blur_kernel, ceil_div(R, g256), g256, 0, st, R, (const int2*)(nb + (long)j * R),
                   (const float2*)a, b);
            std::swap(a, b);
        }
        vals = a;
    }
    with_dim(d, [&](auto dc) {
        launch(dc_walk_kernel<decltype(dc)::value>, ceil_div(N, 128), 128, 0, st, N, p.L, l, d, p.nodes,
               (const float*)sf, (const float*)w.lat.bary.get(), (const int*)roi, vals, p.alpha, p.raw);
    });
    DCRF_LAUNCH_CHECK();
    // the next label rebuilds the lattice and reuses the buffers: finish this one
    DCRF_CUDA(cudaStreamSynchronize(st));
}

constexpr int kDcThreads = 8;
// Items (node, pixel, corner) the concurrent labels hold at most between
// them (about 50 bytes of buffers each): small images run up to kDcThreads
// labels at once, large ones one at a time (measured on 320x240, bilateral:
// 46 ms one at a time, 1.3 s with eight workers' buffers churning through
// the allocator).
constexpr long kDcConcurrentItems = 4L << 20;

}  // namespace

// The labels are independent: on small images up to kDcThreads host threads
// take them one at a time, each on its own stream, so that one label's host
// waits (the lattice build reads its vertex count, the runs their count)
// overlap the others' kernels.
void Model::apply_upper_minus_lower_dc(int k, bool nonorm, float* out, const int* ind) {
    Term& t = *terms.at(k);
    const int d = t.d, d1 = d + 1;
    std::vector<DcNode> h_nodes;
    long T = 0;
    build_dc_tree(h_nodes, 0, N, 0, T, d1);
    require(T < (1L << 31) - 1, DCRF_E_ARG, "divide-and-conquer filter: image too large");
    std::vector<long> h_ibase;
    std::vector<int> h_iid;
    for (int x = 0; x < (int)h_nodes.size(); x++)
        if (h_nodes[x].left >= 0) {
            h_ibase.push_back(h_nodes[x].base);
            h_iid.push_back(x);
        }
    const int nn = (int)h_nodes.size(), ni = (int)h_iid.size();
    DevBuf<DcNode> nodes;
    DevBuf<long> ibase;
    DevBuf<int> iid;
    DCRF_CUDA(cudaMemcpyAsync(nodes.ensure(nn), h_nodes.data(), sizeof(DcNode) * nn, cudaMemcpyHostToDevice, stream));
    if (ni) {
        DCRF_CUDA(cudaMemcpyAsync(ibase.ensure(ni), h_ibase.data(), sizeof(long) * ni, cudaMemcpyHostToDevice, stream));
        DCRF_CUDA(cudaMemcpyAsync(iid.ensure(ni), h_iid.data(), sizeof(int) * ni, cudaMemcpyHostToDevice, stream));
    }
    float* raw = buf(8);
    // the inputs (ind, the features) and the tables above come in on the model's stream
    DCRF_CUDA(cudaStreamSynchronize(stream));
    const DcPlan plan{N, L, d, nn, ni, T, nodes.get(), ibase.get(), iid.get(), t.feat.get(), ind,
                      1.0f / (1.0f + std::pow(2.0f, (float)-d)),  // src/permutohedral.cpp:950
                      raw};
    const int nth = (int)std::max(1L, std::min<long>(std::min(L, kDcThreads), kDcConcurrentItems / std::max(T, 1L)));
    std::vector<std::unique_ptr<DcWorker>> workers;
    for (int i = 0; i < nth; i++) workers.push_back(std::make_unique<DcWorker>());
    std::atomic<int> next{0};
    std::exception_ptr err = nullptr;
    std::mutex emu;
    auto run = [&](int i) {
        cudaSetDevice(device);
        for (;;) {
            const int l = next.fetch_add(1);
            if (l >= L) break;
            try {
                dc_label(*workers[i], plan, l);
            } catch (...) {
                std::lock_guard<std::mutex> lk(emu);
                if (!err) err = std::current_exception();
                next.store(L);
            }
        }
    };
    std::vector<std::thread> pool;
    try {
        for (int i = 1; i < nth; i++) pool.emplace_back(run, i);
    } catch (...) {  // fewer threads than asked for: the ones running take the labels
    }
    run(0);
    for (auto& th : pool) th.join();
    for (auto& w : workers) DCRF_CUDA(cudaStreamSynchronize(w->st));
    if (err) std::rethrow_exception(err);
    apply_compat(k, nonorm, out, raw);
}

}  // namespace dcrf
