// Permutohedral lattice construction and filtering on sm_100a.
//
// Construction reproduces Permutohedral::init's SSE path
// (src/permutohedral.cpp:152-333) bit for bit:
//   K1 elevate   one thread per pixel: elevation, rounding to the nearest
//                0-coloured vertex (round-to-nearest-even, as _mm_cvtps_epi32
//                does), rank, barycentric weights and the d+1 vertex keys;
//                the pixel count is padded to a multiple of 4 with zero
//                features, like the reference's last SSE block.
//   K2 insert    open-addressing hash insert of every (pixel, remainder)
//                entry; each slot ends up holding the SMALLEST entry index
//                with its key (atomicMin), i.e. the key's first occurrence.
//   K3 compact   vertex id = rank of the first occurrence among all first
//                occurrences (flag + exclusive scan) -- exactly the
//                insertion order HashTable::find produces (:100-128).
//   K4 neighbours  per (axis, vertex) lookup of key -1/+d and key +1/-d
//                (:316-330).
//   K5 splat lists  stable radix sort of entries by vertex id.
// Filtering reproduces sseCompute (L > 2) / seqCompute (L <= 2)
// (src/permutohedral.cpp:998-1058 / 488-540) and the 10-bin ordered filter
// (:548-701) with the same per-element operation order, so results are
// identical to the reference, with no float atomics.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "lattice.cuh"

namespace dcrf {

namespace {

constexpr int kEmpty = -1;
constexpr int kRes = 10;       // RESOLUTION (include/permutohedral.h:41)
constexpr int kOrdW = 2 * kRes;  // lower + upper bins per (vertex, label)
constexpr int kStageWarps = 2;   // warps (splat lists) per splat block
constexpr int kStages = 3;       // shared-memory ring depth, in chunks
constexpr int kChunk = 32;       // entries per chunk (13 KB of ring per warp: 16 warps / SM)
constexpr int kMaxOrderKey = (1 << 24) - 1;
constexpr int kLongList = 64;    // lists longer than this use the staged warp kernels
constexpr int kHugeList = 1024;  // lists longer than this get the finest ordered-splat split
constexpr int kHugeLabels = 12;  // labels per block for those lists (120 threads)
constexpr int kTB = 256;         // threads per block of the element-wise kernels

template <int KW>
struct Key {
    int4 w[KW];
};

template <int KW>
__device__ __forceinline__ Key<KW> load_key(const int4* __restrict__ k, long e) {
    Key<KW> r;
#pragma unroll
    for (int i = 0; i < KW; i++) r.w[i] = __ldg(k + e * KW + i);
    return r;
}

template <int KW>
__device__ __forceinline__ bool key_eq(const Key<KW>& a, const Key<KW>& b) {
    bool eq = true;
#pragma unroll
    for (int i = 0; i < KW; i++)
        eq &= (a.w[i].x == b.w[i].x) & (a.w[i].y == b.w[i].y) & (a.w[i].z == b.w[i].z) &
              (a.w[i].w == b.w[i].w);
    return eq;
}

__device__ __forceinline__ uint32_t mix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

template <int KW>
__device__ __forceinline__ uint32_t key_hash(const Key<KW>& k) {
    uint32_t h = 0x9e3779b9u;
#pragma unroll
    for (int i = 0; i < KW; i++) {
        h = mix32(h ^ (uint32_t)k.w[i].x);
        h = mix32(h ^ (uint32_t)k.w[i].y);
        h = mix32(h ^ (uint32_t)k.w[i].z);
        h = mix32(h ^ (uint32_t)k.w[i].w);
    }
    return h;
}

template <int KW>
__device__ __forceinline__ void key_set(Key<KW>& k, int c, int16_t v) {
    int* words = reinterpret_cast<int*>(k.w);
    int wi = c >> 1;
    uint32_t u = (uint32_t)words[wi];
    if (c & 1) u = (u & 0x0000ffffu) | ((uint32_t)(uint16_t)v << 16);
    else u = (u & 0xffff0000u) | (uint32_t)(uint16_t)v;
    words[wi] = (int)u;
}

template <int KW>
__device__ __forceinline__ int16_t key_get(const Key<KW>& k, int c) {
    const int* words = reinterpret_cast<const int*>(k.w);
    uint32_t u = (uint32_t)words[c >> 1];
    return (int16_t)(uint16_t)((c & 1) ? (u >> 16) : (u & 0xffffu));
}

template <int KW>
__device__ __forceinline__ void key_zero(Key<KW>& k) {
#pragma unroll
    for (int i = 0; i < KW; i++) k.w[i] = make_int4(0, 0, 0, 0);
}

// _mm_cvtps_epi32 (round to nearest even; out-of-range -> INT_MIN) and back.
__device__ __forceinline__ float cvt_rne(float v) {
    if (!(fabsf(v) < 2147483648.0f)) return -2147483648.0f;
    return (float)__float2int_rn(v);
}

// K1: one thread per (padded) pixel.
template <int DM>
__global__ void elevate_kernel(const float* __restrict__ feat, int N, int Np, int d,
                               const float* __restrict__ scale, int4* __restrict__ ekeys,
                               int* __restrict__ rank_out, float* __restrict__ bary_out) {
    constexpr int KW = (DM + 7) / 8;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Np) return;
    const int d1 = d + 1;
    const float invdp1 = 1.0f / (float)d1, dp1 = (float)d1;
    float f[DM], el[DM + 1], rem0[DM + 1], rk[DM + 1], b[DM + 2];
    for (int j = 0; j < d; j++) f[j] = k < N ? feat[(long)k * d + j] : 0.0f;
    // Elevation (:213-219): sm accumulates from the last coordinate down.
    float sm = 0.0f;
    for (int j = d; j > 0; j--) {
        float cf = fmul(f[j - 1], scale[j - 1]);
        el[j] = fsub(sm, fmul((float)j, cf));
        sm = fadd(sm, cf);
    }
    el[0] = sm;
    // Closest 0-coloured simplex (:222-232).
    float sum = 0.0f;
    for (int i = 0; i <= d; i++) {
        float v = cvt_rne(fmul(invdp1, el[i]));
        rem0[i] = fmul(v, dp1);
        sum = fadd(sum, v);
    }
    // Rank (:235-245).
    for (int i = 0; i <= d; i++) rk[i] = 0.0f;
    for (int i = 0; i < d; i++) {
        float di = fsub(el[i], rem0[i]);
        for (int j = i + 1; j <= d; j++) {
            float dj = fsub(el[j], rem0[j]);
            float c = (di < dj) ? 1.0f : 0.0f;
            rk[i] = fadd(rk[i], c);
            rk[j] = fadd(rk[j], fsub(1.0f, c));
        }
    }
    // Back onto the plane (:248-254).
    for (int i = 0; i <= d; i++) {
        rk[i] = fadd(rk[i], sum);
        float add = rk[i] < 0.0f ? dp1 : 0.0f;
        float sub = rk[i] >= dp1 ? dp1 : 0.0f;
        float t = fsub(add, sub);
        rk[i] = fadd(rk[i], t);
        rem0[i] = fadd(rem0[i], t);
    }
    // Barycentric coordinates (:257-275).
    for (int i = 0; i < d + 2; i++) b[i] = 0.0f;
    for (int i = 0; i <= d; i++) {
        float v = fmul(fsub(el[i], rem0[i]), invdp1);
        int p = (int)fsub((float)d, rk[i]);
        p = min(max(p, 0), d);  // in range for finite features; guards NaN input
        b[p] = fadd(b[p], v);
        b[p + 1] = fsub(b[p + 1], v);
    }
    b[0] = fadd(b[0], fadd(1.0f, b[d + 1]));
    // Keys of the d+1 vertices (:280-287); canonical simplex (:183-188).
    for (int r = 0; r <= d; r++) {
        Key<KW> key;
        key_zero(key);
        for (int i = 0; i < d; i++) {
            int ri = (int)rk[i];
            int canon = (ri <= d - r) ? r : r - d1;
            key_set(key, i, (int16_t)(int)fadd(rem0[i], (float)canon));
        }
        long e = (long)k * d1 + r;
#pragma unroll
        for (int w = 0; w < KW; w++) ekeys[e * KW + w] = key.w[w];
        if (k < N) {
            rank_out[e] = (int)rk[r];
            bary_out[e] = b[r];
        }
    }
}

// K2: insert every entry; slots keep the smallest entry index of their key.
template <int KW>
__global__ void insert_kernel(const int4* __restrict__ ekeys, int E, int* table, unsigned mask,
                              int* __restrict__ entry_slot) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const Key<KW> key = load_key<KW>(ekeys, e);
    unsigned h = key_hash(key) & mask;
    for (unsigned probe = 0; probe <= mask; probe++) {  // bounded: table is never full
        int cur = *(volatile int*)(table + h);
        if (cur == kEmpty) {
            int old = atomicCAS(table + h, kEmpty, e);
            if (old == kEmpty) {
                entry_slot[e] = (int)h;
                return;
            }
            cur = old;
        }
        if (key_eq(load_key<KW>(ekeys, cur), key)) {
            atomicMin(table + h, e);
            entry_slot[e] = (int)h;
            return;
        }
        h = (h + 1) & mask;
    }
}

__global__ void first_flag_kernel(int E, const int* __restrict__ entry_slot,
                                  const int* __restrict__ table, int* __restrict__ flag) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    flag[e] = table[entry_slot[e]] == e ? 1 : 0;
}

// K3: vertex ids and vertex keys.
template <int KW>
__global__ void finalize_kernel(int E, int Ereal, int d, const int* __restrict__ entry_slot,
                                const int* __restrict__ table, const int* __restrict__ first_rank,
                                const int4* __restrict__ ekeys, int* __restrict__ offset,
                                int16_t* __restrict__ vkeys, int* __restrict__ slot_vid) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const int s = entry_slot[e];
    const int f = table[s];
    const int vid = first_rank[f];
    if (e < Ereal) offset[e] = vid;
    if (f == e) {
        slot_vid[s] = vid;
        const Key<KW> key = load_key<KW>(ekeys, e);
        for (int c = 0; c < d; c++) vkeys[(long)vid * d + c] = key_get(key, c);
    }
}

template <int KW>
__device__ __forceinline__ int lookup(const Key<KW>& key, const int* __restrict__ table,
                                      unsigned mask, const int4* __restrict__ ekeys,
                                      const int* __restrict__ slot_vid) {
    unsigned h = key_hash(key) & mask;
    for (unsigned probe = 0; probe <= mask; probe++) {
        int cur = table[h];
        if (cur == kEmpty) return -1;
        if (key_eq(load_key<KW>(ekeys, cur), key)) return slot_vid[h];
        h = (h + 1) & mask;
    }
    return -1;
}

// K4: blur neighbours, stored shifted by one (0 = absent).
template <int KW>
__global__ void neighbor_kernel(int M, int d, const int16_t* __restrict__ vkeys,
                                const int* __restrict__ table, unsigned mask,
                                const int4* __restrict__ ekeys, const int* __restrict__ slot_vid,
                                int2* __restrict__ nbr) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)(d + 1) * M) return;
    const int j = (int)(t / M), v = (int)(t - (long)j * M);
    Key<KW> n1, n2;
    key_zero(n1);
    key_zero(n2);
    for (int c = 0; c < d; c++) {
        int kc = vkeys[(long)v * d + c];
        int a = c == j ? kc + d : kc - 1;
        int bb = c == j ? kc - d : kc + 1;
        key_set(n1, c, (int16_t)a);
        key_set(n2, c, (int16_t)bb);
    }
    int i1 = lookup(n1, table, mask, ekeys, slot_vid);
    int i2 = lookup(n2, table, mask, ekeys, slot_vid);
    nbr[t] = make_int2(i1 + 1, i2 + 1);
}

__global__ void count_kernel(int E, const int* __restrict__ offset, int* __restrict__ counts) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < E) atomicAdd(counts + offset[e], 1);
}

__global__ void iota_copy_kernel(int E, const int* __restrict__ offset, int* __restrict__ keys,
                                 int* __restrict__ vals) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    keys[e] = offset[e];
    vals[e] = e;
}

__global__ void seg_fill_kernel(int E, int d1, const int* __restrict__ sorted_entries,
                                const float* __restrict__ bary, int* __restrict__ seg_pix,
                                float* __restrict__ seg_w) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= E) return;
    const int e = sorted_entries[s];
    seg_pix[s] = e / d1;
    seg_w[s] = bary[e];
}

// ------------------------------------------------------------- filter --

// Splat as a gather: value(v, k) = sum over v's entries, in entry order, of
// w * in[p][k] (times the symmetric normalisation when pre_norm is given,
// which DenseKernel::filter applies before the lattice, src/pairwise.cpp:61).
//
// One warp per vertex, lanes = labels (in chunks of 32).  The sum must stay
// sequential in entry order to reproduce the reference's scatter, so each
// lane's float adds form one dependent chain; everything else is kept off
// that chain.  The list is streamed in chunks of 32 entries through a ring
// of kStages shared-memory buffers with cp.async: while chunk c is summed,
// chunks c+1 .. c+kStages-1 (up to 96 entries x L values, plus their weights
// and normalisation factors) are in flight, so a single long list is not
// serialised on L2 latency.  Vertices are visited longest list first
// (`order`) so the few very long lists of a coarse lattice start early.
// The filter kernels loop over their units (list positions, vertices,
// pixels or tiles) with a grid-stride loop: one pass with a full grid, or,
// in a batched solve, the units of the images still running (Live) with a
// grid sized for the device.

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Streams the list [s0, s1) of one vertex through the per-warp ring:
// `vals_of(slot, e)` is this lane's staged word for entry e, and
// consume(slot, n) is called once per chunk, in order.
template <typename T, bool NORM, typename Consume>
__device__ __forceinline__ void stream_list(int s0, int s1, int L, int k, bool act, int lane,
                                            const int* __restrict__ seg_pix, const float* __restrict__ seg_w,
                                            const T* __restrict__ src, const float* __restrict__ norm,
                                            T (*ring)[kChunk][32], float (*mw)[kChunk], float (*mn)[kChunk],
                                            Consume&& consume) {
    const int nch = (s1 - s0 + kChunk - 1) / kChunk;
    auto pix_of = [&](int c) {
        const int base = s0 + c * kChunk;
        return (c < nch && lane < s1 - base) ? seg_pix[base + lane] : 0;
    };
    auto issue = [&](int c, int pc) {
        const int slot = c % kStages, base = s0 + c * kChunk, n = min(kChunk, s1 - base);
        if (lane < n) {
            cp_async4(&mw[slot][lane], seg_w + base + lane);
            if (NORM) cp_async4(&mn[slot][lane], norm + pc);
        }
        for (int e = 0; e < n; e++) {
            const int p = __shfl_sync(0xffffffffu, pc, e);
            if (act) cp_async4(&ring[slot][e][lane], src + (long)p * L + k);
        }
    };
    int pcur = pix_of(0);
#pragma unroll
    for (int c = 0; c < kStages - 1; c++) {
        const int pn = pix_of(c + 1);
        if (c < nch) issue(c, pcur);
        cp_async_commit();
        pcur = pn;
    }
    for (int c = 0; c < nch; c++) {
        const int ci = c + kStages - 1;
        const int pn = pix_of(ci + 1);
        if (ci < nch) issue(ci, pcur);
        cp_async_commit();
        pcur = pn;
        cp_async_wait<kStages - 1>();  // chunk c has landed (this lane's copies)
        __syncwarp();                  // ... and every other lane's
        consume(c % kStages, min(kChunk, s1 - (s0 + c * kChunk)));
        __syncwarp();                  // the slot is refilled kStages-1 chunks later
    }
    cp_async_wait<0>();
    __syncwarp();
}

template <bool PRE_NORM, int LC = 0>
__global__ void __launch_bounds__(32 * kStageWarps)
    splat_kernel(int M, int Lrt, const int* __restrict__ order, const int* __restrict__ seg_start,
                 const int* __restrict__ seg_pix, const float* __restrict__ seg_w, const float* __restrict__ in,
                 const float* __restrict__ norm, float* __restrict__ vals, Live lv, int Lrow) {
    const int L = LC ? LC : Lrt;
    __shared__ float ring[kStageWarps][kStages][kChunk][32];
    __shared__ float mw[kStageWarps][kStages][kChunk];
    __shared__ float mn[kStageWarps][kStages][kChunk];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long total = live_total(lv, M);
    // warp-uniform loop; the kernel has no block-wide barrier
    for (long unit = (long)blockIdx.x * kStageWarps + wib; unit < total; unit += (long)gridDim.x * kStageWarps) {
        const int v = order[live_unit(lv, unit)];
        const int s0 = seg_start[v], s1 = seg_start[v + 1];
        for (int kb = 0; kb < L; kb += 32) {
            const int k = kb + lane;
            const bool act = k < L;
            float acc = 0.0f;
            stream_list<float, PRE_NORM>(s0, s1, L, k, act, lane, seg_pix, seg_w, in, norm, ring[wib], mw[wib],
                                         mn[wib], [&](int slot, int n) {
#pragma unroll 4
                                             for (int e = 0; e < n; e++) {
                                                 float x = ring[wib][slot][e][lane];
                                                 if (PRE_NORM) x = fmul(x, mn[wib][slot][e]);
                                                 acc = fadd(acc, fmul(mw[wib][slot][e], x));
                                             }
                                         });
            if (act) vals[(long)(v + 1) * Lrow + k] = acc;
        }
        for (int k = L + lane; k < Lrow; k += 32) vals[(long)(v + 1) * Lrow + k] = 0.0f;  // row padding
    }
}

// The longest lists with L = 21: the cp.async ring of splat_kernel, kStages chunks
// of 32 entries deep, but each lane copies its own entry's 21 values into a
// [label][entry] ring (no shuffles, 21 copies per chunk instead of 32), and
// lane k < 21 sums its label in entry order with float4 reads of four
// entries' values, weights (and norms) at a time.
constexpr int kRS = 36;  // ring row stride: float4-aligned, 4 banks apart per label
template <bool PRE_NORM>
__global__ void __launch_bounds__(32 * kStageWarps)
    splat_ring21_kernel(int M, const int* __restrict__ order, const int* __restrict__ seg_start,
                        const int* __restrict__ seg_pix, const float* __restrict__ seg_w,
                        const float* __restrict__ in, const float* __restrict__ norm, float* __restrict__ vals,
                        Live lv, int Lrow) {
    constexpr int L = 21;
    __shared__ __align__(16) float X[kStageWarps][kStages][L][kRS];
    __shared__ __align__(16) float Wr[kStageWarps][kStages][kChunk];
    __shared__ __align__(16) float Nr[kStageWarps][kStages][kChunk];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long total = live_total(lv, M);
    // warp-uniform loop; no block-wide barrier inside
    for (long unit = (long)blockIdx.x * kStageWarps + wib; unit < total; unit += (long)gridDim.x * kStageWarps) {
        const int v = order[live_unit(lv, unit)];
        const int s0 = seg_start[v], s1 = seg_start[v + 1];
        const int nch = (s1 - s0 + kChunk - 1) / kChunk;
        auto pix_of = [&](int c) {
            const int e = s0 + c * kChunk + lane;
            return (c < nch && e < s1) ? seg_pix[e] : -1;
        };
        auto issue = [&](int c, int p) {
            if (p < 0) return;  // past the end of the list: never summed
            const int slot = c % kStages, e = s0 + c * kChunk + lane;
            const float* row = in + (long)p * L;
#pragma unroll
            for (int k = 0; k < L; k++) cp_async4(&X[wib][slot][k][lane], row + k);
            cp_async4(&Wr[wib][slot][lane], seg_w + e);
            if (PRE_NORM) cp_async4(&Nr[wib][slot][lane], norm + p);
        };
        float acc = 0.0f;
        int pcur = pix_of(0);
#pragma unroll
        for (int c = 0; c < kStages - 1; c++) {
            const int pn = pix_of(c + 1);
            issue(c, pcur);
            cp_async_commit();
            pcur = pn;
        }
        for (int c = 0; c < nch; c++) {
            const int ci = c + kStages - 1;
            const int pn = pix_of(ci + 1);
            issue(ci, pcur);
            cp_async_commit();
            pcur = pn;
            cp_async_wait<kStages - 1>();  // chunk c has landed (this lane's copies)
            __syncwarp();                  // ... and every other lane's
            const int slot = c % kStages, n = min(kChunk, s1 - (s0 + c * kChunk));
            if (lane < L) {
                const float4* xs = reinterpret_cast<const float4*>(&X[wib][slot][lane][0]);
                const float4* ws = reinterpret_cast<const float4*>(&Wr[wib][slot][0]);
                const float4* ns = reinterpret_cast<const float4*>(&Nr[wib][slot][0]);
                const int n4 = n >> 2;
                for (int q = 0; q < n4; q++) {
                    float4 x = xs[q];
                    const float4 w = ws[q];
                    if (PRE_NORM) {
                        const float4 nv = ns[q];
                        x.x = fmul(x.x, nv.x);
                        x.y = fmul(x.y, nv.y);
                        x.z = fmul(x.z, nv.z);
                        x.w = fmul(x.w, nv.w);
                    }
                    acc = fadd(acc, fmul(w.x, x.x));
                    acc = fadd(acc, fmul(w.y, x.y));
                    acc = fadd(acc, fmul(w.z, x.z));
                    acc = fadd(acc, fmul(w.w, x.w));
                }
                for (int e = n4 << 2; e < n; e++) {
                    float x = X[wib][slot][lane][e];
                    if (PRE_NORM) x = fmul(x, Nr[wib][slot][e]);
                    acc = fadd(acc, fmul(Wr[wib][slot][e], x));
                }
            }
            __syncwarp();  // the slot is refilled kStages-1 chunks later
        }
        cp_async_wait<0>();
        __syncwarp();
        if (lane < L) vals[(long)(v + 1) * Lrow + lane] = acc;
        else if (lane < Lrow) vals[(long)(v + 1) * Lrow + lane] = 0.0f;  // row padding
    }
}

// Lists of at most kHugeList entries: one warp per vertex, lane = label (in
// chunks of 32 labels).  The list streams in chunks of 32 entries: each
// lane loads one entry's pixel, weight and normalisation factor (coalesced,
// the next chunk's while the current one is summed) and stores them as one
// 16-byte record in shared memory; then every entry costs one broadcast
// record read and one coalesced read of the pixel's L input values.  The
// sum is the same in-order chain per (vertex, label) as splat_kernel's.
template <bool PRE_NORM, int LC, int WARPS>
__global__ void __launch_bounds__(32 * WARPS)
    splat_warp_kernel(int n, int Lrt, const int* __restrict__ order, const int* __restrict__ seg_start,
                      const int* __restrict__ seg_pix, const float* __restrict__ seg_w,
                      const float* __restrict__ in, const float* __restrict__ norm, float* __restrict__ vals,
                      Live lv, int Lrow) {
    const int L = LC ? LC : Lrt;
    __shared__ float4 rec[WARPS][32];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long total = live_total(lv, n);
    // warp-uniform loop; no block-wide barrier inside
    for (long unit = (long)blockIdx.x * WARPS + wib; unit < total; unit += (long)gridDim.x * WARPS) {
        const int v = order[live_unit(lv, unit)];
        const int s0 = seg_start[v], s1 = seg_start[v + 1];
        float4* r = rec[wib];
        for (int kb = 0; kb < L; kb += 32) {
            const int k = kb + lane;
            const bool act = k < L;
            float acc = 0.0f;
            int p = 0;
            float w = 0.0f, nn = 1.0f;
            auto fetch = [&](int base) {
                const int e = base + lane;
                if (e < s1) {
                    p = seg_pix[e];
                    w = seg_w[e];
                    if (PRE_NORM) nn = norm[p];
                }
            };
            fetch(s0);
            for (int c0 = s0; c0 < s1; c0 += 32) {
                r[lane] = make_float4(__int_as_float(p), w, nn, 0.0f);
                fetch(c0 + 32);  // in flight while this chunk is summed
                __syncwarp();
                const int cnt = min(32, s1 - c0);
                if (act) {
#pragma unroll 8
                    for (int e = 0; e < cnt; e++) {
                        const float4 q = r[e];
                        float x = in[(long)__float_as_int(q.x) * L + k];
                        if (PRE_NORM) x = fmul(x, q.z);
                        acc = fadd(acc, fmul(q.y, x));
                    }
                }
                __syncwarp();  // the records are rewritten next chunk
            }
            if (act) vals[(long)(v + 1) * Lrow + k] = acc;
        }
        for (int k = L + lane; k < Lrow; k += 32) vals[(long)(v + 1) * Lrow + k] = 0.0f;  // row padding
    }
}

// Short lists (at most kLongList entries; the tail of `order`): one thread
// per (vertex, label), the same in-order sum without staging.
template <bool PRE_NORM, int LC = 0>
__global__ void splat_short_kernel(int n_short, int Lrt, const int* __restrict__ order,
                                   const int* __restrict__ seg_start, const int* __restrict__ seg_pix,
                                   const float* __restrict__ seg_w, const float* __restrict__ in,
                                   const float* __restrict__ norm, float* __restrict__ vals, Live lv, int Lrow) {
    const int L = LC ? LC : Lrt;
    const long total = live_total(lv, n_short) * Lrow;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const long u = t / Lrow;
        const int k = (int)(t - u * Lrow);
        const int v = order[live_unit(lv, u)];
        if (k >= L) {  // row padding
            vals[(long)(v + 1) * Lrow + k] = 0.0f;
            continue;
        }
        const int s0 = seg_start[v], s1 = seg_start[v + 1];
        float acc = 0.0f;
#pragma unroll 4
        for (int s = s0; s < s1; s++) {
            const int p = seg_pix[s];
            float x = in[(long)p * L + k];
            if (PRE_NORM) x = fmul(x, norm[p]);
            acc = fadd(acc, fmul(seg_w[s], x));
        }
        vals[(long)(v + 1) * Lrow + k] = acc;
    }
}

// Block-tiled splat for L = 21.  A block takes kTV consecutive lists of the
// visiting order at a time (a tile) and stages their entries through shared
// memory in slabs of kSL entries per list, so that hundreds of input rows
// are in flight per block instead of a few per warp:
//   1. the slab's (pixel, weight) pairs of the kTV lists (coalesced) and the
//      next tile's list ranges are loaded one step ahead into registers and
//      published to shared memory at the start of the step;
//   2. thread (list g, label k) copies label k of every entry of list g with
//      cp.async into a [list][entry][label] buffer: the 21 threads of a list
//      read one entry's 84 contiguous bytes, and the list stride (693
//      floats, 21 mod 32) makes one warp's writes and reads conflict-free;
//      the record owners copy the entries' norms beside them;
//   3. thread (g, k) adds the slab to its running sum in entry order.
// The per-(vertex, label) chain is the same sequence of float operations as
// in every other splat form, so the values are bit-identical.  Lists longer
// than one slab take several slabs with the sum carried in a register; the
// visiting order puts lists of similar length next to each other.
constexpr int kTV = 12;           // lists per tile (12 x 21 = 252 worker threads)
constexpr int kSL = 32;           // entries per list per slab
constexpr int kTE = kTV * kSL;    // entry slots per slab
constexpr int kXV = kSL * 21 + 21;  // floats per list in the row buffer (21 mod 32)
constexpr int kRV = kSL + 1;      // per-list stride of the weight / norm arrays
constexpr int kTileThreads = 256;
constexpr int kTileBlocksPerSM = 5;
template <bool PRE_NORM>
__global__ void __launch_bounds__(kTileThreads)
    splat_tile21_kernel(int count, const int* __restrict__ order, const int* __restrict__ seg_start,
                        const int* __restrict__ seg_pix, const float* __restrict__ seg_w,
                        const float* __restrict__ in, const float* __restrict__ norm, float* __restrict__ vals,
                        Live lv, int Lrow) {
    constexpr int L = 21;
    __shared__ __align__(16) float X[kTV * kXV];
    __shared__ float Ws[kTV * kRV], Ns[kTV * kRV];
    __shared__ int Ps[kTV * kRV];
    __shared__ int tv[2][kTV], ts0[2][kTV], tn[2][kTV];
    const int t = threadIdx.x;
    const int g = t / L, k = t - g * L;  // worker role (t < kTV * L)
    const bool worker = t < kTV * L;
    const long total = live_total(lv, count);
    const long ntiles = (total + kTV - 1) / kTV;
    // list range (v, s0, n) of slot t < kTV of a tile
    auto load_meta = [&](long tile, int& v, int& s0, int& n) {
        v = -1;
        s0 = n = 0;
        const long u = tile * kTV + t;
        if (tile < ntiles && u < total) {
            v = order[live_unit(lv, u)];
            s0 = seg_start[v];
            n = seg_start[v + 1] - s0;
        }
    };
    // (pixel, weight) of this thread's record slots j = t, t + 256 of slab s
    // of the tile whose ranges are in buffer b
    int rp[2] = {0, 0};
    float rw[2] = {0.0f, 0.0f};
    auto fetch = [&](int b, int s) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int j = t + h * kTileThreads;
            rp[h] = -1;
            if (j < kTE) {
                const int li = j / kSL, e = s * kSL + (j - li * kSL);
                if (e < tn[b][li]) {
                    rp[h] = seg_pix[ts0[b][li] + e];
                    rw[h] = seg_w[ts0[b][li] + e];
                }
            }
        }
    };
    long tile = blockIdx.x;
    if (tile >= ntiles) return;  // block-uniform
    int mv = -1, ms0 = 0, mn = 0;
    if (t < kTV) {
        load_meta(tile, mv, ms0, mn);
        tv[0][t] = mv;
        ts0[0][t] = ms0;
        tn[0][t] = mn;
        load_meta(tile + gridDim.x, mv, ms0, mn);  // in flight during the first tile
    }
    __syncthreads();
    fetch(0, 0);
    for (int it = 0; tile < ntiles; it++, tile += gridDim.x) {  // block-uniform
        const int b = it & 1;
        int nmax = 0;
#pragma unroll
        for (int i = 0; i < kTV; i++) nmax = max(nmax, tn[b][i]);
        const int nslab = (nmax + kSL - 1) / kSL;
        float acc = 0.0f;
        for (int s = 0; s < nslab; s++) {
            const bool last = s + 1 == nslab;
            __syncthreads();  // the previous step's readers of Ps / Ws / Ns / X are done
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int j = t + h * kTileThreads;
                if (j < kTE && rp[h] >= 0) {
                    const int li = j / kSL, r = li * kRV + (j - li * kSL);
                    Ps[r] = rp[h];
                    Ws[r] = rw[h];
                    if (PRE_NORM) cp_async4(&Ns[r], norm + rp[h]);
                }
            }
            if (last && t < kTV) {  // the next tile's ranges, loaded during this one
                tv[b ^ 1][t] = mv;
                ts0[b ^ 1][t] = ms0;
                tn[b ^ 1][t] = mn;
            }
            __syncthreads();
            const int n = worker ? min(kSL, tn[b][g] - s * kSL) : 0;
            if (n > 0) {
                const float* src = in + k;
                float* dst = &X[g * kXV + k];
                const int* pp = &Ps[g * kRV];
#pragma unroll 4
                for (int e = 0; e < n; e++) cp_async4(dst + e * L, src + (long)pp[e] * L);
            }
            cp_async_commit();
            // next step's records (and, after this tile, the following tile's
            // ranges) in flight while this slab lands and is summed
            if (!last) {
                fetch(b, s + 1);
            } else {
                fetch(b ^ 1, 0);
                if (t < kTV) load_meta(tile + 2L * gridDim.x, mv, ms0, mn);
            }
            cp_async_wait<0>();
            __syncthreads();
            if (n > 0) {
                const float* xs = &X[g * kXV + k];
                const float* ws = &Ws[g * kRV];
                const float* ns = &Ns[g * kRV];
#pragma unroll 4
                for (int e = 0; e < n; e++) {
                    float x = xs[e * L];
                    if (PRE_NORM) x = fmul(x, ns[e]);
                    acc = fadd(acc, fmul(ws[e], x));
                }
            }
        }
        if (worker && tv[b][g] >= 0) vals[(long)(tv[b][g] + 1) * Lrow + k] = acc;
        for (int q = t; q < kTV * (Lrow - L); q += kTileThreads) {  // row padding
            const int li = q / (Lrow - L);
            if (tv[b][li] >= 0) vals[(long)(tv[b][li] + 1) * Lrow + L + (q - li * (Lrow - L))] = 0.0f;
        }
    }
}

// ------------------------------------------------- bulk-copy (TMA) splat --
// 1-D bulk copies (cp.async.bulk, the TMA engine; this GPU's own memory, no
// multicast) complete on a shared-memory mbarrier.  Waits are bounded: a
// wait that runs out counts itself in g_bulk_wait_timeouts and the filter's
// output rows of that tile are written as NaN, so a result never silently
// uses unfinished copies.
__device__ unsigned long long g_bulk_wait_timeouts = 0;
constexpr long kBulkWaitLimit = 1L << 24;  // try_wait polls (each suspends briefly): seconds

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase with the given parity; false if the wait ran out.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
    for (long it = 0; it < kBulkWaitLimit; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void bulk_g2s(void* sdst, const void* gsrc, unsigned bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_addr(sdst)),
        "l"(gsrc), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// Splat for L = 21 whose input rows arrive by bulk copy.  The structure is
// splat_tile21_kernel's (tiles of kTV lists, slabs of kSL entries, the next
// tile's ranges and records prefetched), but the rows of a slab are fetched
// per run of consecutive pixels in a list: one cp.async.bulk of the run's
// 16-byte-aligned byte span (at most 96 bytes per entry) into a packed
// shared-memory buffer, issued by the run's first entry.  The rows then
// never pass through the L1 load pipeline, which bounds the other forms.
// Each entry records where its row starts in the buffer.  A run whose
// aligned span would end past the input (the last pixel, when 84 N is not a
// multiple of 16) is copied with plain loads instead.  `in` must be 16-byte
// aligned (the host checks it and uses another form otherwise).
constexpr int kBulkFloats = kTE * 24;  // 96 bytes per entry slot at most
constexpr int kBulkBlocksPerSM = 4;
template <bool PRE_NORM>
__global__ void __launch_bounds__(kTileThreads, kBulkBlocksPerSM)
    splat_bulk21_kernel(int count, const int* __restrict__ order, const int* __restrict__ seg_start,
                        const int* __restrict__ seg_pix, const float* __restrict__ seg_w,
                        const float* __restrict__ in, int N, const float* __restrict__ norm,
                        float* __restrict__ vals, Live lv, int Lrow) {
    constexpr int L = 21;
    __shared__ __align__(128) float X[kBulkFloats];
    __shared__ float Ws[kTV * kRV], Ns[kTV * kRV];
    __shared__ int Ps[kTV * kRV], Os[kTV * kRV];
    __shared__ int tv[2][kTV], ts0[2][kTV], tn[2][kTV];
    __shared__ unsigned s_space, s_tx;
    __shared__ int s_timeout;
    __shared__ __align__(8) unsigned long long bar;
    const int t = threadIdx.x;
    const int g = t / L, k = t - g * L;  // worker role (t < kTV * L)
    const bool worker = t < kTV * L;
    const long total = live_total(lv, count);
    const long ntiles = (total + kTV - 1) / kTV;
    const char* in_b = reinterpret_cast<const char*>(in);
    const char* in_end = in_b + (size_t)N * L * sizeof(float);
    auto load_meta = [&](long tile, int& v, int& s0, int& n) {
        v = -1;
        s0 = n = 0;
        const long u = tile * kTV + t;
        if (tile < ntiles && u < total) {
            v = order[live_unit(lv, u)];
            s0 = seg_start[v];
            n = seg_start[v + 1] - s0;
        }
    };
    int rp[2] = {0, 0};
    float rw[2] = {0.0f, 0.0f};
    auto fetch = [&](int b, int s) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int j = t + h * kTileThreads;
            rp[h] = -1;
            if (j < kTE) {
                const int li = j / kSL, e = s * kSL + (j - li * kSL);
                if (e < tn[b][li]) {
                    rp[h] = seg_pix[ts0[b][li] + e];
                    rw[h] = seg_w[ts0[b][li] + e];
                }
            }
        }
    };
    long tile = blockIdx.x;
    if (tile >= ntiles) return;  // block-uniform
    if (t == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    int mv = -1, ms0 = 0, mn = 0;
    if (t < kTV) {
        load_meta(tile, mv, ms0, mn);
        tv[0][t] = mv;
        ts0[0][t] = ms0;
        tn[0][t] = mn;
        load_meta(tile + gridDim.x, mv, ms0, mn);
    }
    __syncthreads();
    fetch(0, 0);
    unsigned phase = 0;
    for (int it = 0; tile < ntiles; it++, tile += gridDim.x) {  // block-uniform
        const int b = it & 1;
        int nmax = 0;
#pragma unroll
        for (int i = 0; i < kTV; i++) nmax = max(nmax, tn[b][i]);
        const int nslab = (nmax + kSL - 1) / kSL;
        float acc = 0.0f;
        bool bad = false;
        for (int s = 0; s < nslab; s++) {
            const bool last = s + 1 == nslab;
            __syncthreads();  // the previous step's readers of the shared arrays are done
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int j = t + h * kTileThreads;
                if (j < kTE && rp[h] >= 0) {
                    const int li = j / kSL, r = li * kRV + (j - li * kSL);
                    Ps[r] = rp[h];
                    Ws[r] = rw[h];
                    if (PRE_NORM) cp_async4(&Ns[r], norm + rp[h]);
                }
            }
            if (last && t < kTV) {
                tv[b ^ 1][t] = mv;
                ts0[b ^ 1][t] = ms0;
                tn[b ^ 1][t] = mn;
            }
            if (t == 0) {
                s_space = 0;
                s_tx = 0;
                s_timeout = 0;
            }
            __syncthreads();
            // runs of consecutive pixels: the first entry of each places the
            // run in the buffer and records every entry's row start
            const char* rsrc[2] = {nullptr, nullptr};
            unsigned rdst[2] = {0, 0}, rbytes[2] = {0, 0};
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int j = t + h * kTileThreads;
                if (j >= kTE || rp[h] < 0) continue;
                const int li = j / kSL, el = j - li * kSL, base = li * kRV;
                const int n = min(kSL, tn[b][li] - s * kSL);
                const int p = Ps[base + el];
                if (el > 0 && Ps[base + el - 1] == p - 1) continue;  // not a run start
                int len = 1;
                while (el + len < n && Ps[base + el + len] == p + len) len++;
                const char* b0 = in_b + (size_t)p * (L * sizeof(float));
                const char* b1 = b0 + (size_t)len * (L * sizeof(float));
                const char* a0 = reinterpret_cast<const char*>(reinterpret_cast<uintptr_t>(b0) & ~(uintptr_t)15);
                const char* a1 =
                    reinterpret_cast<const char*>((reinterpret_cast<uintptr_t>(b1) + 15) & ~(uintptr_t)15);
                const unsigned bytes = (unsigned)(a1 - a0);
                const unsigned off = atomicAdd(&s_space, bytes);  // bytes and offsets: multiples of 16
                const int row0 = (int)((off + (unsigned)(b0 - a0)) / sizeof(float));
                for (int i = 0; i < len; i++) Os[base + el + i] = row0 + i * L;
                if (a1 <= in_end) {
                    atomicAdd(&s_tx, bytes);
                    rsrc[h] = a0;
                    rdst[h] = off;
                    rbytes[h] = bytes;
                } else {  // the span would pass the end of the input: plain loads
                    for (int i = 0; i < len * L; i++) X[row0 + i] = in[(size_t)p * L + i];
                }
            }
            fence_proxy_async_smem();  // this thread's generic writes of X before any async copy
            __syncthreads();
            // the phase's byte count before any copy can complete against it
            if (t == 0) mbar_expect_tx(&bar, s_tx);
            __syncthreads();
#pragma unroll
            for (int h = 0; h < 2; h++)
                if (rbytes[h]) bulk_g2s(reinterpret_cast<char*>(X) + rdst[h], rsrc[h], rbytes[h], &bar);
            cp_async_commit();
            if (!last) {
                fetch(b, s + 1);
            } else {
                fetch(b ^ 1, 0);
                if (t < kTV) load_meta(tile + 2L * gridDim.x, mv, ms0, mn);
            }
            cp_async_wait<0>();
            if (!mbar_wait_bounded(&bar, phase)) s_timeout = 1;
            phase ^= 1;
            __syncthreads();
            if (s_timeout) bad = true;
            const int n = worker ? min(kSL, tn[b][g] - s * kSL) : 0;
            if (n > 0) {
                const int* os = &Os[g * kRV];
                const float* ws = &Ws[g * kRV];
                const float* ns = &Ns[g * kRV];
#pragma unroll 4
                for (int e = 0; e < n; e++) {
                    float x = X[os[e] + k];
                    if (PRE_NORM) x = fmul(x, ns[e]);
                    acc = fadd(acc, fmul(ws[e], x));
                }
            }
        }
        if (bad && t == 0) atomicAdd(&g_bulk_wait_timeouts, 1ull);
        if (worker && tv[b][g] >= 0) vals[(long)(tv[b][g] + 1) * Lrow + k] = bad ? __int_as_float(0x7fc00000) : acc;
        for (int q = t; q < kTV * (Lrow - L); q += kTileThreads) {  // row padding
            const int li = q / (Lrow - L);
            if (tv[b][li] >= 0) vals[(long)(tv[b][li] + 1) * Lrow + L + (q - li * (Lrow - L))] = 0.0f;
        }
    }
}

__global__ void count_long_kernel(int M, const int* __restrict__ counts, int threshold, int* __restrict__ n) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const bool is_long = v < M && counts[v] > threshold;
    const unsigned b = __ballot_sync(0xffffffffu, is_long);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(n, __popc(b));
}

// Class of a splat list by its length: 0 huge, 1 long, 2 short.
__device__ __forceinline__ int list_class(int c) { return c > kHugeList ? 0 : c > kLongList ? 1 : 2; }

// Concatenated lattices: the key (class, image) of each position of the
// length-sorted visiting order, for a second stable sort that groups each
// class's lists by image (longest first within an image), and the number of
// lists per (class, image).
__global__ void class_image_key_kernel(int M, const int* __restrict__ order, const int* __restrict__ counts,
                                       const int* __restrict__ vimg, int images, int* __restrict__ keys,
                                       int* __restrict__ per_class_image) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= M) return;
    const int v = order[p];
    const int key = list_class(counts[v]) * images + vimg[v];
    keys[p] = key;
    atomicAdd(&per_class_image[key], 1);
}

// Sort key of the splat visiting order (stable radix sort ascending): the
// long lists first, longest first, so that their chains start early; the
// short lists after them in vertex-id order.  Ids follow the pixels' scan
// order (first occurrence), so consecutive short lists gather rows of nearby
// pixels and each input row is fetched from DRAM about once although d + 1
// lists read it (sorting the short lists by length too scattered them over
// the whole image).
__global__ void order_key_kernel(int M, const int* __restrict__ counts, int* __restrict__ keys,
                                 int* __restrict__ vals) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= M) return;
    const int c = counts[v];
    keys[v] = c > kLongList ? kMaxOrderKey - min(c, kMaxOrderKey) : kMaxOrderKey;
    vals[v] = v;
}

// One blur pass along one lattice axis: new = old + 1/2 (n1 + n2).  seqCompute
// evaluates it in double (0.5 is a double literal there, :518).
template <bool SEQ, int LC = 0>
__global__ void blur_kernel(int M, int Lrt, const int2* __restrict__ nbr,
                            const float* __restrict__ src, float* __restrict__ dst, Live lv) {
    const int L = LC ? LC : Lrt;
    const long total = live_total(lv, M) * L;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const long u = t / L;
        const int k = (int)(t - u * L);
        const int v = (int)live_unit(lv, u);
        const int2 nb = nbr[v];
        const float a = src[(long)(v + 1) * L + k];
        const float s = fadd(src[(long)nb.x * L + k], src[(long)nb.y * L + k]);
        float r;
        if (SEQ) r = (float)dadd((double)a, dmul(0.5, (double)s));
        else r = fadd(a, fmul(0.5f, s));
        dst[(long)(v + 1) * L + k] = r;
    }
}

// The blur pass over rows padded to Lp = 4 Q floats (sseCompute, L > 2):
// one thread per (vertex, four labels), float4 loads of the vertex's row and
// of its two neighbours' rows.  The same operations per element as
// blur_kernel; the padding lanes hold zeros and stay zero.
template <int Q>
__global__ void blur4_kernel(int M, int Qrt, const int2* __restrict__ nbr, const float* __restrict__ src,
                             float* __restrict__ dst, Live lv) {
    const int Qn = Q ? Q : Qrt;
    const long lp = 4L * Qn;
    const long total = live_total(lv, M) * Qn;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const long u = t / Qn;
        const int q = (int)(t - u * Qn);
        const int v = (int)live_unit(lv, u);
        const int2 nb = nbr[v];
        const float4 a = *reinterpret_cast<const float4*>(src + (long)(v + 1) * lp + 4 * q);
        const float4 x = *reinterpret_cast<const float4*>(src + (long)nb.x * lp + 4 * q);
        const float4 y = *reinterpret_cast<const float4*>(src + (long)nb.y * lp + 4 * q);
        float4 r;
        r.x = fadd(a.x, fmul(0.5f, fadd(x.x, y.x)));
        r.y = fadd(a.y, fmul(0.5f, fadd(x.y, y.y)));
        r.z = fadd(a.z, fmul(0.5f, fadd(x.z, y.z)));
        r.w = fadd(a.w, fmul(0.5f, fadd(x.w, y.w)));
        *reinterpret_cast<float4*>(dst + (long)(v + 1) * lp + 4 * q) = r;
    }
}

__device__ __forceinline__ float apply_epilogue(float v, long t, int i, int k, const SliceEpilogue& ep) {
    if (ep.potts) {
        if (ep.norm) v = fmul(v, ep.norm[i]);
        v = ep.scale_vec ? fmul(ep.scale_vec[k], v) : fmul(ep.scale, v);
    }
    if (ep.base) v = fadd(ep.base[t], fmul(ep.coef, v));
    else if (ep.zero_base) v = fadd(0.0f, fmul(ep.coef, v));
    return v;
}

// Slice: out(i, k) = sum_j (bary_ij * alpha) * value(o_ij, k) (sseCompute,
// :1046-1051) or sum_j (bary_ij * value) * alpha (seqCompute, :529-534).
template <bool SEQ, int DC, int LC>
__global__ void slice_kernel(int N, int Lrt, int drt, const int* __restrict__ offset,
                             const float* __restrict__ bary, const float* __restrict__ vals,
                             float alpha, float* out, SliceEpilogue ep, Live lv) {
    const int L = LC ? LC : Lrt, d = DC ? DC : drt;
    const int d1 = d + 1;
    const long total = live_total(lv, N) * L;
    for (long tl = (long)blockIdx.x * blockDim.x + threadIdx.x; tl < total; tl += (long)gridDim.x * blockDim.x) {
        const long u = tl / L;
        const int k = (int)(tl - u * L);
        const int i = (int)live_unit(lv, u);  // the pixel
        const long t = (long)i * L + k;
        float acc = 0.0f;
#pragma unroll
        for (int j = 0; j <= d; j++) {
            const int o = offset[(long)i * d1 + j];
            const float w = bary[(long)i * d1 + j];
            const float v = vals[(long)(o + 1) * L + k];
            if (SEQ) acc = fadd(acc, fmul(fmul(w, v), alpha));
            else acc = fadd(acc, fmul(fmul(w, alpha), v));
        }
        out[t] = apply_epilogue(acc, t, i, k, ep);
    }
}

// Slice over rows padded to Lp = 4 Q floats (sseCompute, L > 2), a tile of
// `tile` pixels per block (kSliceTile, fewer for very wide rows): the
// tile's offsets, (barycentric * alpha) weights and normalisation factors
// are staged once in shared memory (coalesced: they are contiguous), every
// (pixel, four labels) item gathers the d+1 vertex rows with float4 loads
// and applies the per-pixel part of the epilogue (norm, compatibility
// scale), and the tile's L outputs per pixel -- contiguous in `out` --
// leave through shared memory, coalesced, with the accumulation part
// (base + coef * v).  Per element the arithmetic is slice_kernel's and
// apply_epilogue's: acc = sum over j in order of (bary_j * alpha) *
// value_j, from +0.
constexpr int kSliceTile = 128;
constexpr int kSliceThreads = 256;
template <int DC, int Q, int LC>
__global__ void __launch_bounds__(kSliceThreads)
    slice4_kernel(int N, int Lrt, int Qrt, int drt, int tile, const int* __restrict__ offset,
                  const float* __restrict__ bary, const float* __restrict__ vals, float alpha, float* out,
                  SliceEpilogue ep, Live lv, const long* __restrict__ pix_base) {
    extern __shared__ __align__(16) unsigned char slice_smem[];
    const int d1 = (DC ? DC : drt) + 1, Qn = Q ? Q : Qrt, L = LC ? LC : Lrt;
    const long lp = 4L * Qn;
    int* s_off = reinterpret_cast<int*>(slice_smem);
    float* s_wa = reinterpret_cast<float*>(s_off + tile * d1);
    float* s_nrm = s_wa + tile * d1;
    float* s_out = s_nrm + tile;
    const bool use_norm = ep.potts && ep.norm;
    // Tiles: of the whole pixel range, or (live images) of each live image's
    // pixels, image by image (pix_base: its pixel offsets).
    const long total = live_total(lv, ((long)N + tile - 1) / tile);
    for (long u = blockIdx.x; u < total; u += gridDim.x) {  // block-uniform
        long p0, pend = N;
        if (lv.n) {
            long local;
            const int img = live_locate(lv, u, local);
            p0 = pix_base[img] + local * tile;
            pend = pix_base[img + 1];
        } else {
            p0 = u * tile;
        }
        const int np = (int)min((long)tile, pend - p0);
        for (int e = threadIdx.x; e < np * d1; e += blockDim.x) {
            s_off[e] = offset[p0 * d1 + e];
            s_wa[e] = fmul(bary[p0 * d1 + e], alpha);
        }
        if (use_norm)
            for (int e = threadIdx.x; e < np; e += blockDim.x) s_nrm[e] = ep.norm[p0 + e];
        __syncthreads();
        for (int it = threadIdx.x; it < np * Qn; it += blockDim.x) {
            const int pl = it / Qn, q = it - pl * Qn;
            float a[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int j = 0; j < (DC ? DC + 1 : 17); j++) {
                if (!DC && j >= d1) break;
                const int o = s_off[pl * d1 + j];
                const float wa = s_wa[pl * d1 + j];
                const float4 v = *reinterpret_cast<const float4*>(vals + (long)(o + 1) * lp + 4 * q);
                a[0] = fadd(a[0], fmul(wa, v.x));
                a[1] = fadd(a[1], fmul(wa, v.y));
                a[2] = fadd(a[2], fmul(wa, v.z));
                a[3] = fadd(a[3], fmul(wa, v.w));
            }
            const int k0 = 4 * q;
            float* so = s_out + pl * L + k0;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                if (k0 + c >= L) break;
                float v = a[c];
                if (ep.potts) {
                    if (use_norm) v = fmul(v, s_nrm[pl]);
                    v = ep.scale_vec ? fmul(ep.scale_vec[k0 + c], v) : fmul(ep.scale, v);
                }
                so[c] = v;
            }
        }
        __syncthreads();
        const long t0 = p0 * L;
        const int ne = np * L;
        if (ep.base) {
            for (int e = threadIdx.x; e < ne; e += blockDim.x)
                out[t0 + e] = fadd(ep.base[t0 + e], fmul(ep.coef, s_out[e]));
        } else if (ep.zero_base) {
            for (int e = threadIdx.x; e < ne; e += blockDim.x) out[t0 + e] = fadd(0.0f, fmul(ep.coef, s_out[e]));
        } else {
            for (int e = threadIdx.x; e < ne; e += blockDim.x) out[t0 + e] = s_out[e];
        }
        __syncthreads();  // the next tile restages the shared arrays
    }
}

// addSplitArray / sliceSplitArray bins (:548-589): the lower pass rounds
// q*10 in float, the upper pass (q - 1e-9)*10 in double.
// For q in [0, 1] these are the reference's indices; other values (which the
// reference rejects with an assert) are clamped to a valid bin so no access
// can leave the bin array.
__device__ __forceinline__ int bin_lower(float q) {
    int c = (int)floorf(fmul(q, (float)kRes));
    c = c < kRes - 1 ? c : kRes - 1;
    return c > 0 ? c : 0;
}
__device__ __forceinline__ int bin_upper(float q) {
    int c = (int)floor(dmul(__dsub_rn((double)q, 1e-9), (double)kRes));
    c = c > 0 ? c : 0;
    return c < kRes - 1 ? c : kRes - 1;
}

// Ordered bins of every (pixel, label), computed once per ordered filter
// (each pixel appears in d+1 splat lists and in the slice): the lower and
// upper bin indices, held as floats (exact small integers) because the splat
// compares them with float bin numbers.
__device__ __forceinline__ float2 ord_bin_pair(float q) {
    return make_float2((float)bin_lower(q), (float)bin_upper(q));
}
__device__ __forceinline__ int ord_lower_of(float2 b) { return (int)b.x; }
__device__ __forceinline__ int ord_upper_of(float2 b) { return (int)b.y; }

__global__ void ord_bins_kernel(long n, const float* __restrict__ Q, float2* __restrict__ bins) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    bins[t] = ord_bin_pair(Q[t]);
}

// The same, four elements per thread with 16-byte loads and stores (Q and
// bins 16-byte aligned; n4 = n / 4 quads, the tail by ord_bins_kernel).
__global__ void ord_bins4_kernel(long n4, const float4* __restrict__ Q, float4* __restrict__ bins) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n4) return;
    const float4 q = Q[t];
    const float2 a = ord_bin_pair(q.x), b = ord_bin_pair(q.y), c = ord_bin_pair(q.z), d = ord_bin_pair(q.w);
    bins[2 * t] = make_float4(a.x, a.y, b.x, b.y);
    bins[2 * t + 1] = make_float4(c.x, c.y, d.x, d.y);
}

// Each of the 10 bins accumulates, in entry order, the weights of the entries
// that reach it: bins 0..c (lower pass) or c..9 (upper pass), addSplitArray
// (:548-569).  Branch-free and bit-identical: the mask m = [c_lower >= b]
// (lower) or [b >= c_upper] (upper) is exactly 1.0 or 0.0 (one PTX `set`,
// NaN giving 0), so fma(m, w, acc) rounds acc + w once when the entry reaches
// the bin and otherwise returns acc (acc + (+-0) = acc: the accumulator
// starts at +0 and is never -0).
__device__ __forceinline__ float step_ge(float a, float b) {  // a >= b ? 1 : 0
    float r;
    asm("set.ge.f32.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}

// One entry into the bin-b pair (lower, upper) of packed accumulators:
// acc = fma({[cl >= b], [b >= cu]}, w2, acc) with one f32x2 FMA, which rounds
// each half exactly as fma.rn.f32 does.  w2 holds (w, w).  The bins are
// small integers, so the masks are saturated sums: cl + (1 - b) and
// (b + 1) - cu are exact integers, clamped to [0, 1] they are exactly the
// comparisons (and a NaN would clamp to +0).  One `add.sat` per mask.
__device__ __forceinline__ void ord_step2(unsigned long long& acc, float cl, float cu, float b,
                                          unsigned long long w2) {
    const float lo_c = 1.0f - b, up_c = b + 1.0f;  // exact; hoisted out of the entry loops
    asm("{\n\t.reg .f32 ml, mu;\n\t.reg .b64 m;\n\t"
        "add.rn.sat.f32 ml, %1, %3;\n\t"
        "sub.rn.sat.f32 mu, %4, %2;\n\t"
        "mov.b64 m, {ml, mu};\n\t"
        "fma.rn.f32x2 %0, m, %5, %0;\n\t}"
        : "+l"(acc)
        : "f"(cl), "f"(cu), "f"(lo_c), "f"(up_c), "l"(w2));
}
// The single masks of ord_step2: [cl >= b] and [b >= cu] as 0.0 / 1.0.
__device__ __forceinline__ float ord_mask_lower(float cl, int b) {
    float m;
    asm("add.rn.sat.f32 %0, %1, %2;" : "=f"(m) : "f"(cl), "f"(1.0f - (float)b));
    return m;
}
__device__ __forceinline__ float ord_mask_upper(float cu, int b) {
    float m;
    asm("sub.rn.sat.f32 %0, %1, %2;" : "=f"(m) : "f"((float)b + 1.0f), "f"(cu));
    return m;
}
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float2 unpack2(unsigned long long v) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
}

template <bool UPPER>
__device__ __forceinline__ void ord_accumulate(float (&acc)[kRes], float c, float w) {
#pragma unroll
    for (int b = 0; b < kRes; b++) {
        const float m = UPPER ? step_ge((float)b, c) : step_ge(c, (float)b);
        acc[b] = __fmaf_rn(m, w, acc[b]);
    }
}

template <bool UPPER>
__device__ __forceinline__ void ord_consume(float (&acc)[kRes], const float (*ring)[32], const float* mw, int lane,
                                            int n) {
#pragma unroll 2
    for (int e = 0; e < n; e++) ord_accumulate<UPPER>(acc, ring[e][lane], mw[e]);
}

// Ordered splat, general L: one warp per (vertex, pass), streaming the
// vertex's list as splat_kernel does.  A vertex row holds 20 bins x L
// labels, bin-major ([v][bin][label]; bins [0,10) lower, [10,20) upper) so
// that the slice's per-label bin reads coalesce.
__global__ void __launch_bounds__(32 * kStageWarps)
    ord_splat_kernel(int M, int L, const int* __restrict__ order, const int* __restrict__ seg_start,
                     const int* __restrict__ seg_pix, const float* __restrict__ seg_w,
                     const float2* __restrict__ bins, float* __restrict__ vals) {
    __shared__ float ring[kStageWarps][kStages][kChunk][32];
    __shared__ float mw[kStageWarps][kStages][kChunk];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int unit = blockIdx.x * kStageWarps + wib;
    if (unit >= 2 * M) return;  // warp-uniform
    const int v = order[unit >> 1];
    const bool upper = unit & 1;
    const int s0 = seg_start[v], s1 = seg_start[v + 1];
    const float* bf = reinterpret_cast<const float*>(bins);  // [pixel][label][lower, upper]
    for (int kb = 0; kb < L; kb += 32) {
        const int k = kb + lane;
        const bool act = k < L;
        float acc[kRes];
#pragma unroll
        for (int b = 0; b < kRes; b++) acc[b] = 0.0f;
        stream_list<float, false>(s0, s1, 2 * L, 2 * k + (upper ? 1 : 0), act, lane, seg_pix, seg_w, bf, nullptr,
                                  ring[wib], mw[wib], nullptr, [&](int slot, int n) {
                                      if (upper) ord_consume<true>(acc, ring[wib][slot], mw[wib][slot], lane, n);
                                      else ord_consume<false>(acc, ring[wib][slot], mw[wib][slot], lane, n);
                                  });
        if (act) {
            float* row = vals + ((long)(v + 1) * kOrdW + (upper ? kRes : 0)) * L + k;
#pragma unroll
            for (int b = 0; b < kRes; b++) row[(long)b * L] = acc[b];
        }
    }
}

// Ordered splat of the long lists by blocks.  The 20 x L bin sums of a
// vertex are 20 L independent in-order chains; thread (k, g) carries the
// chains of label k, bins g*NB .. g*NB+NB-1, both passes, so a block shares
// a long list's work and the longest lists no longer set the kernel's
// length.
//
// The list streams through shared memory in chunks of kOE entries: the
// pixel ids and weights of chunk c + 2 kODX and the (c_lower, c_upper) bins
// of chunk c + kODX are copied with cp.async while chunk c is summed, one
// block barrier per chunk.  Ring rows are label-major ([k][entry][lower,
// upper], padded to an odd number of 16-byte units) so a thread reads two
// entries per 16-byte load and eight consecutive labels hit distinct banks.
// Weights are staged as (w, w) pairs; entries past the end of the list get
// weight 0, which leaves every accumulator unchanged (the masks are 0 or 1
// for any stale bin value).
constexpr int kOE = 32;                 // entries per chunk
constexpr int kODX = 4;                 // bins are copied kODX chunks ahead of use, pixel ids 2 kODX
constexpr int kOXS = kODX + 1;          // bin ring slots (chunks c .. c+kODX)
constexpr int kOPS = 2 * kODX + 1;      // pixel / weight ring slots (chunks c .. c+2 kODX)
constexpr int kORow = 2 * kOE + 4;      // floats per ring row: 17 x 16 bytes
constexpr int kOrdBlockMaxL = 160;      // larger L use ord_splat_kernel (shared-memory ring size)
constexpr int kGroupChoices[] = {1, 2, 3, 5, 10};

// Bin split with the fewest warp instructions per list entry: warps x (three
// instructions per bin slot -- two masks and one f32x2 FMA -- + about two
// for the shared-memory loads).
int ord_groups_cheapest(int L) {
    int best = 1;
    long best_cost = -1;
    for (int G : kGroupChoices) {
        if (L * G > 1024) break;
        const long warps = (L * G + 31) / 32, nb = (kRes + G - 1) / G;
        const long cost = warps * (3 * nb + 2);
        if (best_cost < 0 || cost <= best_cost) {
            best = G;
            best_cost = cost;
        }
    }
    return best;
}

size_t ord_block_smem(int kb) {
    return sizeof(float) * ((size_t)kOXS * kb * kORow + (size_t)kOPS * kOE * 2) + sizeof(int) * kOPS * kOE;
}

// G bin groups per label, NB = ceil(10 / G) bin slots per thread; slots past
// bin 9 (when G does not divide 10) run on a dummy bin that is not stored.
// Block b covers labels [k0, k0 + nk) of vertex order[b / kblocks], k0 =
// (b % kblocks) * kb: a very long list can be shared by several blocks.
// Compute threads are label-major (t = k * G + g), so the G threads reading
// one label's bins sit in one warp and their shared-memory loads broadcast;
// staging threads are entry-major (t = g * nk + k) so one warp's copies read
// consecutive labels of one pixel.
template <int G>
__global__ void __launch_bounds__(kOrdBlockMaxL * G < 1024 ? kOrdBlockMaxL * G : 1024)
    ord_splat_block_kernel(int L, int kb, int kblocks, const int* __restrict__ order,
                           const int* __restrict__ seg_start, const int* __restrict__ seg_pix,
                           const float* __restrict__ seg_w, const float2* __restrict__ bins,
                           float* __restrict__ vals) {
    extern __shared__ __align__(16) float osm[];
    float* xr = osm;                            // [kOXS][kb][kORow]
    float* wr = xr + (size_t)kOXS * kb * kORow;  // [kOPS][kOE][2]
    int* pr = reinterpret_cast<int*>(wr + kOPS * kOE * 2);  // [kOPS][kOE]
    constexpr int NB = (kRes + G - 1) / G;
    const int t = threadIdx.x;
    const int v = order[blockIdx.x / kblocks];
    const int k0 = (blockIdx.x % kblocks) * kb, nk = min(kb, L - k0);
    const int s0 = seg_start[v], s1 = seg_start[v + 1];
    const int nch = (s1 - s0 + kOE - 1) / kOE;
    const bool worker = t < nk * G;
    const int k = t / G, g = t - k * G;      // compute role
    const int sk = t % nk, sg = t / nk;      // staging role (sg < G for workers)

    auto stage_pw = [&](int c) {  // pixel ids and weights of chunk c
        if (c < nch && t < kOE) {
            const int slot = c % kOPS, e = s0 + c * kOE + t;
            if (e < s1) {
                cp_async4(&pr[slot * kOE + t], seg_pix + e);
                cp_async4(&wr[(slot * kOE + t) * 2], seg_w + e);
                cp_async4(&wr[(slot * kOE + t) * 2 + 1], seg_w + e);
            } else {
                pr[slot * kOE + t] = 0;
                wr[(slot * kOE + t) * 2] = 0.0f;
                wr[(slot * kOE + t) * 2 + 1] = 0.0f;
            }
        }
    };
    // (c_lower, c_upper) of chunk c; needs chunk c's pixel ids in place.
    // Staging thread (sk, sg) copies label k0 + sk of entries sg, sg + G, ...
    // All pixel ids are read before the first copy is issued (the copies'
    // memory clobber would otherwise order each read after the last copy).
    auto stage_x = [&](int c) {
        if (c >= nch || !worker) return;
        constexpr int MX = (kOE + G - 1) / G;
        const int slot = c % kOXS, ps = c % kOPS;
        const int n = min(kOE, s1 - (s0 + c * kOE));
        float* dst = &xr[((size_t)slot * kb + sk) * kORow];
        const float2* src = bins + k0 + sk;
        int pix[MX];
#pragma unroll
        for (int i = 0; i < MX; i++) {
            const int e = sg + i * G;
            pix[i] = e < n ? pr[ps * kOE + e] : 0;
        }
#pragma unroll
        for (int i = 0; i < MX; i++) {
            const int e = sg + i * G;
            if (e < n) cp_async8(dst + 2 * e, src + (long)pix[i] * L);
        }
    };

    // Group j (committed at iteration j; j < 0 in the prologue) holds the
    // bins of chunk j + kODX and the pixel ids / weights of chunk j + 2 kODX.
#pragma unroll
    for (int c = 0; c < kODX; c++) stage_pw(c);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
#pragma unroll
    for (int c = 0; c < kODX; c++) {
        stage_x(c);
        stage_pw(c + kODX);
        cp_async_commit();
    }

    // Bin g*NB + i's (lower, upper) sums as one packed pair: ord_step2 adds
    // an entry to both with one f32x2 FMA (each half rounded as fma.rn.f32).
    unsigned long long acc[NB];
    float bf[NB];
#pragma unroll
    for (int i = 0; i < NB; i++) {
        acc[i] = 0ull;
        bf[i] = (float)(g * NB + i);
    }
    for (int c = 0; c < nch; c++) {
        cp_async_wait<kODX - 1>();  // group c - kODX: bins of chunk c, pixel ids of chunk c + kODX
        __syncthreads();            // ... everyone's copies; and chunk c-1's slots are free
        stage_x(c + kODX);
        stage_pw(c + 2 * kODX);
        cp_async_commit();
        if (worker) {
            const float4* xs = reinterpret_cast<const float4*>(&xr[((size_t)(c % kOXS) * kb + k) * kORow]);
            const ulonglong2* ws = reinterpret_cast<const ulonglong2*>(&wr[(c % kOPS) * kOE * 2]);
            const int n2 = (min(kOE, s1 - (s0 + c * kOE)) + 1) >> 1;
            // Batches of eight entries, the next batch's loads issued before
            // this batch is summed.  A batch may run past n2 into the chunk's
            // zero-weight tail (the ring rows hold kOE entries).
            float4 x[4];      // (c_lower, c_upper) of entries 2 j, 2 j + 1
            ulonglong2 w[4];  // ((w, w), (w, w)) of the same entries
#pragma unroll
            for (int j = 0; j < 4; j++) {
                x[j] = xs[j];
                w[j] = ws[j];
            }
            for (int b0 = 0; b0 < n2; b0 += 4) {
                float4 xn[4];
                ulonglong2 wn[4];
                const int nb0 = b0 + 4 < kOE / 2 ? b0 + 4 : b0;  // stays inside the ring row
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    xn[j] = xs[nb0 + j];
                    wn[j] = ws[nb0 + j];
                }
#pragma unroll
                for (int j = 0; j < 4; j++) {
#pragma unroll
                    for (int i = 0; i < NB; i++) ord_step2(acc[i], x[j].x, x[j].y, bf[i], w[j].x);
#pragma unroll
                    for (int i = 0; i < NB; i++) ord_step2(acc[i], x[j].z, x[j].w, bf[i], w[j].y);
                }
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    x[j] = xn[j];
                    w[j] = wn[j];
                }
            }
        }
    }
    cp_async_wait<0>();
    if (worker) {
        float* row = vals + (long)(v + 1) * kOrdW * L + k0 + k;
#pragma unroll
        for (int i = 0; i < NB; i++) {
            if (g * NB + i >= kRes) break;
            const float2 r = unpack2(acc[i]);
            row[(long)(g * NB + i) * L] = r.x;
            row[(long)(kRes + g * NB + i) * L] = r.y;
        }
    }
}

// Ordered splat of the short lists: one thread per (vertex, label), both
// passes, without staging.
template <int LC = 0>
__global__ void ord_splat_short_kernel(int n_short, int Lrt, const int* __restrict__ order,
                                       const int* __restrict__ seg_start, const int* __restrict__ seg_pix,
                                       const float* __restrict__ seg_w, const float2* __restrict__ bins,
                                       float* __restrict__ vals) {
    const int L = LC ? LC : Lrt;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)n_short * L) return;
    const int u = (int)(t / L), k = (int)(t - (long)u * L);
    const int v = order[u];
    const int s0 = seg_start[v], s1 = seg_start[v + 1];
    // Scalar chains: every entry reaches lower bin 0 (c_lower >= 0) and upper
    // bin 9 (c_upper <= 9), plain adds there; the other 18 bins take a
    // saturated-sum mask (exactly 0 or 1) and an FMA, fma(1, w, acc) being
    // acc + w rounded once.
    float lo[kRes], up[kRes];
#pragma unroll
    for (int b = 0; b < kRes; b++) lo[b] = up[b] = 0.0f;
#pragma unroll 2
    for (int s = s0; s < s1; s++) {
        const float2 x = bins[(long)seg_pix[s] * L + k];
        const float w = seg_w[s];
        lo[0] = fadd(lo[0], w);
#pragma unroll
        for (int b = 1; b < kRes; b++) lo[b] = __fmaf_rn(ord_mask_lower(x.x, b), w, lo[b]);
#pragma unroll
        for (int b = 0; b < kRes - 1; b++) up[b] = __fmaf_rn(ord_mask_upper(x.y, b), w, up[b]);
        up[kRes - 1] = fadd(up[kRes - 1], w);
    }
    float* row = vals + (long)(v + 1) * kOrdW * L + k;
#pragma unroll
    for (int b = 0; b < kRes; b++) {
        row[(long)b * L] = lo[b];
        row[(long)(kRes + b) * L] = up[b];
    }
}

// Ordered blur: every bin independently, weightedAddSplitArray (:570-578).
template <int R4>  // row width in float4 as a compile-time constant (0 = run-time row4r)
__global__ void ord_blur_kernel(int M, int row4r, const int2* __restrict__ nbr,
                                const float4* __restrict__ src, float4* __restrict__ dst) {
    const int row4 = R4 ? R4 : row4r;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)M * row4) return;
    const int v = (int)(t / row4), c = (int)(t - (long)v * row4);
    const int2 nb = nbr[v];
    const float4 a = src[(long)(v + 1) * row4 + c];
    const float4 p = src[(long)nb.x * row4 + c];
    const float4 q = src[(long)nb.y * row4 + c];
    float4 r;
    r.x = fadd(a.x, fmul(0.5f, fadd(p.x, q.x)));
    r.y = fadd(a.y, fmul(0.5f, fadd(p.y, q.y)));
    r.z = fadd(a.z, fmul(0.5f, fadd(p.z, q.z)));
    r.w = fadd(a.w, fmul(0.5f, fadd(p.w, q.w)));
    dst[(long)(v + 1) * row4 + c] = r;
}

// Ordered slice: lower pass with weight -w*alpha, then upper with w*alpha
// (:639-650, :687-696), accumulated into one value.  With GAP the LP's dual
// gap terms are folded in: tmp = (alpha + u) - (v + su) for the final slice
// value v, the clique term su (0 without cliques), and per-block sums of
// tmp.Q and tmp.tmp (src/densecrf.cpp:725-729).
// DC / LC: d and L as compile-time constants (0 = run-time drt / Lrt).
template <bool GAP, int DC, int LC>
__global__ void __launch_bounds__(kTB, 8) ord_slice_kernel(int N, int Lrt, int drt, const int* __restrict__ offset,
                                 const float* __restrict__ bary, const float* __restrict__ vals,
                                 const float2* __restrict__ bins, float alpha, float* out, SliceEpilogue ep,
                                 GapFusion gf) {
    const int L = LC ? LC : Lrt, d = DC ? DC : drt;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double g0 = 0.0, g1 = 0.0;
    if (t < (long)N * L) {
        const int i = (int)(t / L), k = (int)(t - (long)i * L);
        const int d1 = d + 1;
        const float2 bp = bins[t];
        const int cl = ord_lower_of(bp), cu = ord_upper_of(bp);
        float acc = 0.0f;
#pragma unroll
        for (int j = 0; j <= d; j++) {
            const int o = offset[(long)i * d1 + j];
            const float w = bary[(long)i * d1 + j];
            acc = fadd(acc, fmul(vals[((long)(o + 1) * kOrdW + cl) * L + k], fmul(-w, alpha)));
        }
#pragma unroll
        for (int j = 0; j <= d; j++) {
            const int o = offset[(long)i * d1 + j];
            const float w = bary[(long)i * d1 + j];
            acc = fadd(acc, fmul(vals[((long)(o + 1) * kOrdW + kRes + cu) * L + k], fmul(w, alpha)));
        }
        const float v = apply_epilogue(acc, t, i, k, ep);
        out[t] = v;
        if (GAP) {
            const float tmp = fsub(fadd(gf.alpha[t], gf.u[t]), fadd(v, gf.su ? gf.su[t] : 0.0f));
            g0 = (double)tmp * (double)gf.Q[t];
            g1 = (double)tmp * (double)tmp;
        }
    }
    if (GAP) {
        __shared__ double s0[kTB / 32], s1[kTB / 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            g0 += __shfl_down_sync(0xffffffffu, g0, o);
            g1 += __shfl_down_sync(0xffffffffu, g1, o);
        }
        if ((threadIdx.x & 31) == 0) {
            s0[threadIdx.x >> 5] = g0;
            s1[threadIdx.x >> 5] = g1;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0, b = 0.0;
            for (int w = 0; w < kTB / 32; w++) {
                a += s0[w];
                b += s1[w];
            }
            gf.partials[blockIdx.x] = a;
            gf.partials[gridDim.x + blockIdx.x] = b;
        }
    }
}

// One term of a fused two-term ordered slice.
struct OrdSliceTerm {
    const int* offset;
    const float* bary;
    const float* vals;
    int d;
    float alpha;
    SliceEpilogue ep;
};

template <int DC>
__device__ __forceinline__ float ord_slice_acc(const OrdSliceTerm& s, int i, int k, int L, int cl, int cu) {
    const int d = DC ? DC : s.d, d1 = d + 1;
    const int* __restrict__ off = s.offset + (long)i * d1;
    const float* __restrict__ by = s.bary + (long)i * d1;
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j <= d; j++)
        acc = fadd(acc, fmul(s.vals[((long)(off[j] + 1) * kOrdW + cl) * L + k], fmul(-by[j], s.alpha)));
#pragma unroll
    for (int j = 0; j <= d; j++)
        acc = fadd(acc, fmul(s.vals[((long)(off[j] + 1) * kOrdW + kRes + cu) * L + k], fmul(by[j], s.alpha)));
    return acc;
}

// sa = t1's slice on top of t0's (Model::apply_ord_sum with two terms): v0 =
// epilogue_0(slice_0) exactly as ord_slice_kernel writes it, then v0 +
// coef_1 * scaled(slice_1) as ord_slice_kernel computes it from base = v0.
// The value v0 never leaves the register; GAP as in ord_slice_kernel.
template <bool GAP, int D0, int D1, int LC>
__global__ void __launch_bounds__(kTB, 8) ord_slice_pair_kernel(int N, int Lrt, OrdSliceTerm t0, OrdSliceTerm t1,
                                      const float2* __restrict__ bins, float* out, GapFusion gf) {
    const int L = LC ? LC : Lrt;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double g0 = 0.0, g1 = 0.0;
    if (t < (long)N * L) {
        const int i = (int)(t / L), k = (int)(t - (long)i * L);
        const float2 bp = bins[t];
        const int cl = ord_lower_of(bp), cu = ord_upper_of(bp);
        const float a0 = ord_slice_acc<D0>(t0, i, k, L, cl, cu);
        const float a1 = ord_slice_acc<D1>(t1, i, k, L, cl, cu);
        const float v0 = apply_epilogue(a0, t, i, k, t0.ep);
        float s1 = a1;
        if (t1.ep.potts) {
            if (t1.ep.norm) s1 = fmul(s1, t1.ep.norm[i]);
            s1 = t1.ep.scale_vec ? fmul(t1.ep.scale_vec[k], s1) : fmul(t1.ep.scale, s1);
        }
        const float v = fadd(v0, fmul(t1.ep.coef, s1));
        out[t] = v;
        if (GAP) {
            const float tmp = fsub(fadd(gf.alpha[t], gf.u[t]), fadd(v, gf.su ? gf.su[t] : 0.0f));
            g0 = (double)tmp * (double)gf.Q[t];
            g1 = (double)tmp * (double)tmp;
        }
    }
    if (GAP) {
        __shared__ double s0[kTB / 32], s1[kTB / 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            g0 += __shfl_down_sync(0xffffffffu, g0, o);
            g1 += __shfl_down_sync(0xffffffffu, g1, o);
        }
        if ((threadIdx.x & 31) == 0) {
            s0[threadIdx.x >> 5] = g0;
            s1[threadIdx.x >> 5] = g1;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0, b = 0.0;
            for (int w = 0; w < kTB / 32; w++) {
                a += s0[w];
                b += s1[w];
            }
            gf.partials[blockIdx.x] = a;
            gf.partials[gridDim.x + blockIdx.x] = b;
        }
    }
}

// ord_slice_pair_kernel for the LP's common case (L = 21, a d = 2 and a
// d = 5 term) with the per-pixel data staged: a block covers the same 256
// elements (at most 14 pixels), and its pixels' offsets, alpha-scaled
// barycentric weights and normalisation factors are loaded once, coalesced,
// into shared memory instead of by each label's thread.  Element, block and
// dual-gap partial sums are those of ord_slice_pair_kernel, so the values
// are too: the lower pass's fmul(-w, alpha) is the exact negation of
// fmul(w, alpha).
template <bool GAP>
__global__ void __launch_bounds__(kTB, 8) ord_slice_pair_staged(int N, OrdSliceTerm t0, OrdSliceTerm t1,
                                                               const float2* __restrict__ bins, float* out,
                                                               GapFusion gf) {
    constexpr int L = 21, D0 = 3, D1 = 6, P = kTB / L + 2;  // pixels a block touches at most
    __shared__ int so0[P * D0], so1[P * D1];
    __shared__ float sw0[P * D0], sw1[P * D1], sn0[P], sn1[P];
    const long NL = (long)N * L;
    const long tb = (long)blockIdx.x * blockDim.x;
    const long t = tb + threadIdx.x;
    const int pf = (int)(tb / L);
    const int np = (int)min((long)P, (long)N - pf);
    for (int e = threadIdx.x; e < np * D0; e += blockDim.x) {
        so0[e] = t0.offset[(long)pf * D0 + e];
        sw0[e] = fmul(t0.bary[(long)pf * D0 + e], t0.alpha);
    }
    for (int e = threadIdx.x; e < np * D1; e += blockDim.x) {
        so1[e] = t1.offset[(long)pf * D1 + e];
        sw1[e] = fmul(t1.bary[(long)pf * D1 + e], t1.alpha);
    }
    if (threadIdx.x < np) {
        if (t0.ep.norm) sn0[threadIdx.x] = t0.ep.norm[pf + threadIdx.x];
        if (t1.ep.norm) sn1[threadIdx.x] = t1.ep.norm[pf + threadIdx.x];
    }
    __syncthreads();
    double g0 = 0.0, g1 = 0.0;
    if (t < NL) {
        const int i = (int)(t / L), k = (int)(t - (long)i * L), li = i - pf;
        const float2 bp = bins[t];
        const int cl = ord_lower_of(bp), cu = ord_upper_of(bp);
        float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
        for (int j = 0; j < D0; j++)
            a0 = fadd(a0, fmul(t0.vals[((long)(so0[li * D0 + j] + 1) * kOrdW + cl) * L + k], -sw0[li * D0 + j]));
#pragma unroll
        for (int j = 0; j < D0; j++)
            a0 = fadd(a0, fmul(t0.vals[((long)(so0[li * D0 + j] + 1) * kOrdW + kRes + cu) * L + k], sw0[li * D0 + j]));
#pragma unroll
        for (int j = 0; j < D1; j++)
            a1 = fadd(a1, fmul(t1.vals[((long)(so1[li * D1 + j] + 1) * kOrdW + cl) * L + k], -sw1[li * D1 + j]));
#pragma unroll
        for (int j = 0; j < D1; j++)
            a1 = fadd(a1, fmul(t1.vals[((long)(so1[li * D1 + j] + 1) * kOrdW + kRes + cu) * L + k], sw1[li * D1 + j]));
        float v0 = a0;
        if (t0.ep.potts) {
            if (t0.ep.norm) v0 = fmul(v0, sn0[li]);
            v0 = t0.ep.scale_vec ? fmul(t0.ep.scale_vec[k], v0) : fmul(t0.ep.scale, v0);
        }
        if (t0.ep.base) v0 = fadd(t0.ep.base[t], fmul(t0.ep.coef, v0));
        else if (t0.ep.zero_base) v0 = fadd(0.0f, fmul(t0.ep.coef, v0));
        float s1 = a1;
        if (t1.ep.potts) {
            if (t1.ep.norm) s1 = fmul(s1, sn1[li]);
            s1 = t1.ep.scale_vec ? fmul(t1.ep.scale_vec[k], s1) : fmul(t1.ep.scale, s1);
        }
        const float v = fadd(v0, fmul(t1.ep.coef, s1));
        out[t] = v;
        if (GAP) {
            const float tmp = fsub(fadd(gf.alpha[t], gf.u[t]), fadd(v, gf.su ? gf.su[t] : 0.0f));
            g0 = (double)tmp * (double)gf.Q[t];
            g1 = (double)tmp * (double)tmp;
        }
    }
    if (GAP) {
        __shared__ double s0[kTB / 32], s1[kTB / 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            g0 += __shfl_down_sync(0xffffffffu, g0, o);
            g1 += __shfl_down_sync(0xffffffffu, g1, o);
        }
        if ((threadIdx.x & 31) == 0) {
            s0[threadIdx.x >> 5] = g0;
            s1[threadIdx.x >> 5] = g1;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0, b = 0.0;
            for (int w = 0; w < kTB / 32; w++) {
                a += s0[w];
                b += s1[w];
            }
            gf.partials[blockIdx.x] = a;
            gf.partials[gridDim.x + blockIdx.x] = b;
        }
    }
}

// Bins of rescale(Q) (src/eigen_utils.cpp:120-141) without materialising it:
// rq = (Q - min) / (max - min), with min / max at qmm[0], qmm[1].
__global__ void rescaled_bins_kernel(long n, const float* __restrict__ Q, const float* __restrict__ qmm,
                                     float2* __restrict__ bins) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float mn = qmm[0], range = fsub(qmm[1], qmm[0]);
    float rq = fsub(Q[t], mn);
    if (range > 0.0f) rq = rq / range;
    bins[t] = ord_bin_pair(rq);
}

// The same, four elements per thread (as ord_bins4_kernel).
__global__ void rescaled_bins4_kernel(long n4, const float4* __restrict__ Q, const float* __restrict__ qmm,
                                      float4* __restrict__ bins) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n4) return;
    const float mn = qmm[0], range = fsub(qmm[1], qmm[0]);
    const float4 q = Q[t];
    float r[4] = {fsub(q.x, mn), fsub(q.y, mn), fsub(q.z, mn), fsub(q.w, mn)};
    if (range > 0.0f)
#pragma unroll
        for (int i = 0; i < 4; i++) r[i] = r[i] / range;
    const float2 a = ord_bin_pair(r[0]), b = ord_bin_pair(r[1]), c = ord_bin_pair(r[2]), d = ord_bin_pair(r[3]);
    bins[2 * t] = make_float4(a.x, a.y, b.x, b.y);
    bins[2 * t + 1] = make_float4(c.x, c.y, d.x, d.y);
}

bool aligned16(const void* p) { return reinterpret_cast<uintptr_t>(p) % 16 == 0; }

// Ordered-filter bins of Q [n]: four per thread where the pointers allow.
void ord_bins(float2* bins, const float* Q, long n, cudaStream_t st) {
    if (aligned16(Q) && aligned16(bins)) {
        const long n4 = n / 4;
        if (n4) launch(ord_bins4_kernel, ceil_div(n4, kTB), kTB, 0, st, n4, reinterpret_cast<const float4*>(Q),
                       reinterpret_cast<float4*>(bins));
        if (n > 4 * n4) launch(ord_bins_kernel, 1, kTB, 0, st, n - 4 * n4, Q + 4 * n4, bins + 4 * n4);
    } else {
        launch(ord_bins_kernel, ceil_div(n, kTB), kTB, 0, st, n, Q, bins);
    }
}

int bits_for(int n) {  // bits needed to hold values 0..n-1
    int b = 0;
    while ((1LL << b) < (long long)n) b++;
    return b;
}

template <int DM>
void build_impl(Lattice& L, const float* d_features) {
    constexpr int KW = (DM + 7) / 8;
    cudaStream_t st = L.stream;
    const int N = L.N, d = L.d, d1 = d + 1;
    const int Np = (N + 3) & ~3;
    const long E = (long)Np * d1, Ereal = (long)N * d1;
    require(E < (1L << 30), DCRF_E_ARG, "lattice too large (N*(d+1) >= 2^30)");

    // scale_factor (:190-194): computed in double, rounded to float.
    std::vector<float> scale(d);
    const float inv_std_dev = (float)(std::sqrt(2.0 / 3.0) * (d + 1));
    for (int i = 0; i < d; i++) scale[i] = (float)(1.0 / std::sqrt((double)((i + 2) * (i + 1))) * inv_std_dev);
    float* dscale = L.fscale.ensure(d);
    DCRF_CUDA(cudaMemcpyAsync(dscale, scale.data(), sizeof(float) * d, cudaMemcpyHostToDevice, st));

    int4* ekeys = L.ekeys.ensure((size_t)E * KW);
    int* rank = L.rank.ensure(Ereal);
    float* bary = L.bary.ensure(Ereal);
    launch(elevate_kernel<DM>, ceil_div(Np, kTB), kTB, 0, st, d_features, N, Np, d, dscale, ekeys, rank, bary);
    DCRF_LAUNCH_CHECK();

    unsigned cap = 1;
    while ((long)cap < 2 * E) cap <<= 1;
    int* table = L.table.ensure(cap);
    DCRF_CUDA(cudaMemsetAsync(table, 0xff, sizeof(int) * cap, st));
    int* eslot = L.entry_slot.ensure(E);
    launch(insert_kernel<KW>, ceil_div(E, kTB), kTB, 0, st, ekeys, (int)E, table, cap - 1, eslot);
    int* flags = L.flags.ensure(E);
    launch(first_flag_kernel, ceil_div(E, kTB), kTB, 0, st, (int)E, eslot, table, flags);
    DCRF_LAUNCH_CHECK();
    int* dtotal = L.total.ensure(1);
    exclusive_scan(flags, flags, (int)E, dtotal, L.scan, st);
    int M = 0;
    DCRF_CUDA(cudaMemcpyAsync(&M, dtotal, sizeof(int), cudaMemcpyDeviceToHost, st));
    DCRF_CUDA(cudaStreamSynchronize(st));
    L.M = M;

    int* offset = L.offset.ensure(Ereal);
    int16_t* vkeys = L.vkeys.ensure((size_t)M * d);
    int* slot_vid = L.slot_vid.ensure(cap);
    launch(finalize_kernel<KW>, ceil_div(E, kTB), kTB, 0, st, (int)E, (int)Ereal, d, eslot, table, flags,
                                                         ekeys, offset, vkeys, slot_vid);
    int2* nbr = L.nbr.ensure((size_t)d1 * M);
    launch(neighbor_kernel<KW>, ceil_div((long)d1 * M, kTB), kTB, 0, st, M, d, vkeys, table, cap - 1,
                                                                     ekeys, slot_vid, nbr);
    DCRF_LAUNCH_CHECK();

    // Splat lists: per-vertex counts -> starts; stable sort of entries by vertex.
    int* counts = L.counts.ensure((size_t)M + 1);
    DCRF_CUDA(cudaMemsetAsync(counts, 0, sizeof(int) * ((size_t)M + 1), st));
    launch(count_kernel, ceil_div(Ereal, kTB), kTB, 0, st, (int)Ereal, offset, counts);
    int* seg_start = L.seg_start.ensure((size_t)M + 1);
    exclusive_scan(counts, seg_start, M + 1, nullptr, L.scan, st);
    int* skeys = L.sort_keys.ensure(Ereal);
    int* svals = L.sort_vals.ensure(Ereal);
    launch(iota_copy_kernel, ceil_div(Ereal, kTB), kTB, 0, st, (int)Ereal, offset, skeys, svals);
    DCRF_LAUNCH_CHECK();
    radix_sort_pairs(skeys, svals, (int)Ereal, bits_for(M), L.sort, st);
    int* seg_pix = L.seg_pix.ensure(Ereal);
    float* seg_w = L.seg_w.ensure(Ereal);
    launch(seg_fill_kernel, ceil_div(Ereal, kTB), kTB, 0, st, (int)Ereal, d1, svals, bary, seg_pix, seg_w);
    // Splat visiting order: longest lists first.
    int* vorder = L.vorder.ensure(M);
    int* okeys = L.vorder_keys.ensure(M);
    launch(order_key_kernel, ceil_div(M, kTB), kTB, 0, st, M, counts, okeys, vorder);
    radix_sort_pairs(okeys, vorder, M, 24, L.sort, st);
    int* dlong = L.total.ensure(2);
    DCRF_CUDA(cudaMemsetAsync(dlong, 0, 2 * sizeof(int), st));
    launch(count_long_kernel, ceil_div(M, kTB), kTB, 0, st, M, counts, kLongList, dlong);
    launch(count_long_kernel, ceil_div(M, kTB), kTB, 0, st, M, counts, kHugeList, dlong + 1);
    DCRF_LAUNCH_CHECK();
    int nl[2];
    DCRF_CUDA(cudaMemcpyAsync(nl, dlong, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    DCRF_CUDA(cudaStreamSynchronize(st));
    L.n_long = nl[0];
    L.n_huge = nl[1];
    L.va_floats = 0;
}

}  // namespace

namespace {

// ----------------------------------------------------- feature gradient --
// Permutohedral::gradient (src/permutohedral.cpp:1095-1178): df [N][d] of
// a^T K b with respect to the (scaled) features.  For each direction the
// host splats one side, blurs with the double-evaluated 1/2 weights in axis
// order (reversed for the second direction), and this kernel forms the
// slice-side derivative per pixel in the reference's float order: for each
// label k, r_j = (0 + alpha v(o0_j)) - alpha v(o1_j) with o0/o1 from the
// pixel's ranks, then for j = 1..d, grad_j += x_k * sf_{j-1} (s - j r_j),
// s += r_j, s starting at r_0; finally df += grad.
struct GradScale {
    float s[16];
};

template <int DM>
__global__ void grad_slice_kernel(int N, int L, int d, const int* __restrict__ offset, const int* __restrict__ rank,
                                  const float* __restrict__ vals, const float* __restrict__ x, float alpha,
                                  GradScale sf, float* __restrict__ df) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int d1 = d + 1;
    int o0[DM + 1], o1[DM + 1];
#pragma unroll
    for (int j = 0; j <= DM; j++)
        if (j <= d) {
            const int r0 = d - rank[(long)i * d1 + j];
            const int r1 = r0 + 1 > d ? 0 : r0 + 1;
            o0[j] = offset[(long)i * d1 + r0] + 1;
            o1[j] = offset[(long)i * d1 + r1] + 1;
        }
    float grad[DM];
#pragma unroll
    for (int j = 0; j < DM; j++) grad[j] = 0.0f;
    for (int k = 0; k < L; k++) {
        float ra[DM + 1];
#pragma unroll
        for (int j = 0; j <= DM; j++)
            if (j <= d)
                ra[j] = fsub(fadd(0.0f, fmul(alpha, vals[(long)o0[j] * L + k])), fmul(alpha, vals[(long)o1[j] * L + k]));
        const float xk = x[(long)i * L + k];
        float sm = ra[0];
#pragma unroll
        for (int j = 1; j <= DM; j++)
            if (j <= d) {
                const float v = fmul(sf.s[j - 1], fsub(sm, fmul((float)j, ra[j])));
                grad[j - 1] = fadd(grad[j - 1], fmul(xk, v));
                sm = fadd(sm, ra[j]);
            }
    }
#pragma unroll
    for (int j = 0; j < DM; j++)
        if (j < d) df[(long)i * d + j] = fadd(df[(long)i * d + j], grad[j]);
}

template <int DM>
void gradient_impl(Lattice& lat, float* df, const float* a, const float* b, int L) {
    cudaStream_t st = lat.stream;
    const int N = lat.N, d = lat.d, M = lat.M;
    lat.ensure_values((size_t)L);
    DCRF_CUDA(cudaMemsetAsync(df, 0, sizeof(float) * (size_t)N * d, st));
    // scale_factor and alpha as the reference computes them (:1104-1111)
    GradScale sf{};
    const float inv_std_dev = std::sqrt(2.0 / 3.0) * (d + 1);
    for (int i = 0; i < d; i++) sf.s[i] = 1.0 / std::sqrt(double((i + 2) * (i + 1))) * inv_std_dev;
    const float alpha = 1.0f / (1 + std::pow(2.0f, (float)-d)) / (d + 1);
    const int n_short = M - lat.n_long;
    const long ML = (long)M * L, SL = (long)n_short * L;
    for (int dir = 0; dir < 2; dir++) {
        const float* in = dir ? b : a;
        float *src = lat.va.get(), *dst = lat.vb.get();
        if (lat.n_long)
            launch(splat_kernel<false>, ceil_div(lat.n_long, kStageWarps), 32 * kStageWarps, 0, st, lat.n_long, L,
                   lat.vorder.get(), lat.seg_start.get(), lat.seg_pix.get(), lat.seg_w.get(), in, nullptr, src,
                   Live{}, L);
        if (n_short)
            launch(splat_short_kernel<false>, ceil_div(SL, kTB), kTB, 0, st, n_short, L,
                   lat.vorder.get() + lat.n_long, lat.seg_start.get(), lat.seg_pix.get(), lat.seg_w.get(), in,
                   nullptr, src, Live{}, L);
        for (int jj = 0; jj <= d; jj++) {
            const int j = dir ? d - jj : jj;
            launch(blur_kernel<true>, ceil_div(ML, kTB), kTB, 0, st, M, L, lat.nbr.get() + (long)j * M, src, dst,
                   Live{});
            std::swap(src, dst);
        }
        launch(grad_slice_kernel<DM>, ceil_div(N, 128), 128, 0, st, N, L, d, lat.offset.get(), lat.rank.get(), src,
               dir ? a : b, alpha, sf, df);
    }
    DCRF_LAUNCH_CHECK();
}

}  // namespace

void Lattice::gradient(float* df, const float* a, const float* b, int L) {
    require(L >= 1, DCRF_E_ARG, "gradient: L must be >= 1");
    require(!concatenated, DCRF_E_STATE, "gradient: not available on a concatenated lattice");
    if (d <= 2) gradient_impl<2>(*this, df, a, b, L);
    else if (d <= 5) gradient_impl<5>(*this, df, a, b, L);
    else if (d <= 8) gradient_impl<8>(*this, df, a, b, L);
    else gradient_impl<16>(*this, df, a, b, L);
}

// ------------------------------------------------------ concatenation --
// Several images' lattices as one: vertex, pixel and entry ids of part i are
// shifted by the parts before it, so one filter launch sequence runs every
// image at once and each image's values are those of its own lattice (no
// list, neighbour or slice crosses an image).
namespace {

__global__ void add_offset_kernel(long n, const int* __restrict__ src, int add, int* __restrict__ dst) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) dst[t] = src[t] + add;
}

// Neighbour rows are vertex + 1, with 0 for "absent".
__global__ void nbr_offset_kernel(long n, const int2* __restrict__ src, int add, int2* __restrict__ dst) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int2 a = src[t];
    dst[t] = make_int2(a.x > 0 ? a.x + add : 0, a.y > 0 ? a.y + add : 0);
}

__global__ void fill_int_kernel(long n, int v, int* __restrict__ x) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) x[t] = v;
}

__global__ void seg_count_kernel(int M, const int* __restrict__ seg_start, int* __restrict__ counts) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < M) counts[v] = seg_start[v + 1] - seg_start[v];
}

}  // namespace

void Lattice::concat(const std::vector<const Lattice*>& parts) {
    require(!parts.empty(), DCRF_E_ARG, "lattice concat: no parts");
    cudaStream_t st = stream;
    d = parts[0]->d;
    const int d1 = d + 1;
    long Nt = 0, Mt = 0;
    for (const Lattice* p : parts) {
        require(p->d == d, DCRF_E_ARG, "lattice concat: parts differ in feature dimension");
        Nt += p->N;
        Mt += p->M;
    }
    require(Nt * d1 < (1L << 30) && Mt < (1L << 30), DCRF_E_ARG, "lattice concat: too large");
    N = (int)Nt;
    M = (int)Mt;
    const long E = Nt * d1;
    int* off = offset.ensure(E);
    int* rk = rank.ensure(E);
    float* by = bary.ensure(E);
    int* ss = seg_start.ensure(M + 1);
    int* sp = seg_pix.ensure(E);
    float* sw = seg_w.ensure(E);
    int2* nb = nbr.ensure((size_t)d1 * M);
    int* vi = vimg.ensure(std::max(M, 1));
    long pb = 0, vb_ = 0;
    int part = 0;
    for (const Lattice* p : parts) {
        const long e = (long)p->N * d1, eb = pb * d1;
        DCRF_CUDA(cudaStreamSynchronize(p->stream));  // the part was built on its own stream
        launch(add_offset_kernel, ceil_div(e, kTB), kTB, 0, st, e, p->offset.get(), (int)vb_, off + eb);
        DCRF_CUDA(cudaMemcpyAsync(rk + eb, p->rank.get(), sizeof(int) * e, cudaMemcpyDeviceToDevice, st));
        DCRF_CUDA(cudaMemcpyAsync(by + eb, p->bary.get(), sizeof(float) * e, cudaMemcpyDeviceToDevice, st));
        if (p->M) {
            launch(add_offset_kernel, ceil_div(p->M, kTB), kTB, 0, st, (long)p->M, p->seg_start.get(), (int)eb,
                   ss + vb_);
            for (int j = 0; j < d1; j++)
                launch(nbr_offset_kernel, ceil_div(p->M, kTB), kTB, 0, st, (long)p->M,
                       p->nbr.get() + (long)j * p->M, (int)vb_, nb + (long)j * M + vb_);
        }
        launch(add_offset_kernel, ceil_div(e, kTB), kTB, 0, st, e, p->seg_pix.get(), (int)pb, sp + eb);
        DCRF_CUDA(cudaMemcpyAsync(sw + eb, p->seg_w.get(), sizeof(float) * e, cudaMemcpyDeviceToDevice, st));
        if (p->M) launch(fill_int_kernel, ceil_div(p->M, kTB), kTB, 0, st, (long)p->M, part, vi + vb_);
        pb += p->N;
        vb_ += p->M;
        part++;
    }
    const int Ei = (int)E;
    DCRF_CUDA(cudaMemcpyAsync(ss + M, &Ei, sizeof(int), cudaMemcpyHostToDevice, st));
    // Longest lists first, over all images.
    int* cnt = counts.ensure(std::max(M, 1));
    launch(seg_count_kernel, ceil_div(M, kTB), kTB, 0, st, M, ss, cnt);
    int* vo = vorder.ensure(M);
    int* ok = vorder_keys.ensure(M);
    launch(order_key_kernel, ceil_div(M, kTB), kTB, 0, st, M, cnt, ok, vo);
    radix_sort_pairs(ok, vo, M, 24, sort, st);
    // Then, stably, by (class, image): each class (huge, long, short lists)
    // holds its lists image by image, longest first within an image, so
    // that an image's lists of a class are one contiguous range of the order
    // (the live-image domains of a batched solve).
    const int B = (int)parts.size();
    DevBuf<int> pci;
    int* per_ci = pci.ensure((size_t)3 * B);
    DCRF_CUDA(cudaMemsetAsync(per_ci, 0, sizeof(int) * 3 * B, st));
    launch(class_image_key_kernel, ceil_div(M, kTB), kTB, 0, st, M, (const int*)vo, (const int*)cnt,
           (const int*)vi, B, ok, per_ci);
    int kbits = 1;
    while ((1L << kbits) < 3L * B) kbits++;
    radix_sort_pairs(ok, vo, M, kbits, sort, st);
    int* dl = total.ensure(2);
    DCRF_CUDA(cudaMemsetAsync(dl, 0, 2 * sizeof(int), st));
    launch(count_long_kernel, ceil_div(M, kTB), kTB, 0, st, M, cnt, kLongList, dl);
    launch(count_long_kernel, ceil_div(M, kTB), kTB, 0, st, M, cnt, kHugeList, dl + 1);
    DCRF_LAUNCH_CHECK();
    int nl[2];
    std::vector<int> hci((size_t)3 * B);
    DCRF_CUDA(cudaMemcpyAsync(nl, dl, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    DCRF_CUDA(cudaMemcpyAsync(hci.data(), per_ci, sizeof(int) * 3 * B, cudaMemcpyDeviceToHost, st));
    DCRF_CUDA(cudaStreamSynchronize(st));  // also keeps &Ei alive until its copy ran
    n_long = nl[0];
    n_huge = nl[1];
    // Per-image domains: list positions per class, vertex ids, pixels.
    images = B;
    img_pixels.assign(B, 0);
    std::vector<long> hb((size_t)kDomains * (B + 1), 0);
    auto row = [&](int dom) { return hb.data() + (long)dom * (B + 1); };
    long pos = 0;
    for (int c = 0; c < 3; c++) {
        long* r = row(kDomHuge + c);
        for (int i = 0; i < B; i++) {
            r[i] = pos;
            pos += hci[(size_t)c * B + i];
        }
        r[B] = pos;
    }
    for (int i = 0; i < B; i++) {
        img_pixels[i] = parts[i]->N;
        row(kDomVert)[i + 1] = row(kDomVert)[i] + parts[i]->M;
        row(kDomPix)[i + 1] = row(kDomPix)[i] + parts[i]->N;
    }
    long* db = dom_base.ensure(hb.size());
    DCRF_CUDA(cudaMemcpyAsync(db, hb.data(), sizeof(long) * hb.size(), cudaMemcpyHostToDevice, st));
    DCRF_CUDA(cudaStreamSynchronize(st));  // hb is the copy's source
    dom_tile = 0;
    va_floats = 0;
    concatenated = true;
}

void Lattice::prepare_live(int L) {
    require(concatenated && images > 0, DCRF_E_STATE, "live images: not a concatenated lattice");
    if (L <= 2) return;  // the element-wise slice needs no tile domain
    const int tile = slice_tile_for(L);
    if (tile == dom_tile) return;
    std::vector<long> r(images + 1, 0);
    for (int i = 0; i < images; i++) r[i + 1] = r[i] + (img_pixels[i] + tile - 1) / tile;
    DCRF_CUDA(cudaMemcpyAsync(dom_base.get() + (long)kDomTile * (images + 1), r.data(), sizeof(long) * r.size(),
                              cudaMemcpyHostToDevice, stream));
    DCRF_CUDA(cudaStreamSynchronize(stream));  // r is the copy's source
    dom_tile = tile;
}

void Lattice::build(const float* d_features, int d_, int N_) {
    require(N_ > 0, DCRF_E_ARG, "lattice: N must be positive");
    require(d_ >= 1 && d_ <= 16, DCRF_E_ARG, "lattice: feature dimension must be in [1, 16]");
    N = N_;
    d = d_;
    if (d <= 2) build_impl<2>(*this, d_features);
    else if (d <= 5) build_impl<5>(*this, d_features);
    else if (d <= 8) build_impl<8>(*this, d_features);
    else build_impl<16>(*this, d_features);
}

void Lattice::ensure_aux() {
    if (aux) return;
    int lo = 0, hi = 0;
    DCRF_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    DCRF_CUDA(cudaStreamCreateWithPriority(&aux, cudaStreamNonBlocking, hi));
    DCRF_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    DCRF_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
}

Lattice::~Lattice() {
    if (aux) {
        cudaStreamSynchronize(aux);
        cudaEventDestroy(ev_fork);
        cudaEventDestroy(ev_join);
        cudaStreamDestroy(aux);
    }
}

void Lattice::ensure_values(size_t row_width) {
    size_t need = (size_t)(M + 1) * row_width;
    if (need > va_floats) {
        va.ensure(need);
        vb.ensure(need);
        va_floats = need;
    }
    // Row 0 is the zero row that absent neighbours read.
    DCRF_CUDA(cudaMemsetAsync(va.get(), 0, sizeof(float) * row_width, stream));
    DCRF_CUDA(cudaMemsetAsync(vb.get(), 0, sizeof(float) * row_width, stream));
}

// ---------------------------------------------------------------------------
// Allocation-free filtering (dcrf_lattice_compute_noalloc).
//
// Some callers cannot let a library allocate device memory during a call:
// hosts that hand out all GPU memory from their own pool, or that run under a
// fixed memory budget in a latency-critical loop where a driver allocation
// would stall or fail.  For them the filter's two value buffers, normally
// grown on demand with cudaMalloc, come from this fixed array instead.  Every
// GPU that loads the library keeps it for the life of the process.
constexpr size_t kNoAllocScratchFloats = size_t(8) << 20;  // 8 Mi floats = 32 MiB
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
float* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// once per device with that device current and cached.
float* noalloc_scratch() {
    int dev = 0;
    DCRF_CUDA(cudaGetDevice(&dev));
    require(dev >= 0 && dev < kMaxDevices, DCRF_E_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            throw Error(DCRF_E_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_noalloc_ptr[dev] = static_cast<float*>(p);
    }
    return g_noalloc_ptr[dev];
}
}  // namespace

size_t noalloc_scratch_floats() { return kNoAllocScratchFloats; }

void Lattice::compute_noalloc(float* out, const float* in, int L, bool reverse) {
    require(N > 0, DCRF_E_STATE, "lattice not initialised");
    require(L >= 1, DCRF_E_ARG, "compute: L must be >= 1");
    const size_t need = 2 * (size_t)(M + 1) * (size_t)L;
    require(need <= kNoAllocScratchFloats, DCRF_E_ARG,
            "compute_noalloc: 2 x (M + 1) x L = " + std::to_string(need) + " floats exceeds the fixed scratch of " +
                std::to_string(kNoAllocScratchFloats) + " floats (32 MiB); use dcrf_lattice_compute_dev");
    float* base = noalloc_scratch();
    float *src = base, *dst = base + (size_t)(M + 1) * L;
    cudaStream_t st = stream;
    // The array keeps the previous call's contents: only the zero rows that
    // absent neighbours read must be cleared; every other row read below is
    // written first.
    DCRF_CUDA(cudaMemsetAsync(src, 0, sizeof(float) * L, st));
    DCRF_CUDA(cudaMemsetAsync(dst, 0, sizeof(float) * L, st));
    const long ML = (long)M * L, NL = (long)N * L;
    const int n_short = M - n_long;
    if (n_long)
        launch(splat_kernel<false>, ceil_div(n_long, kStageWarps), 32 * kStageWarps, 0, st, n_long, L,
               vorder.get(), seg_start.get(), seg_pix.get(), seg_w.get(), in, nullptr, src, Live{}, L);
    if (n_short)
        launch(splat_short_kernel<false>, ceil_div((long)n_short * L, kTB), kTB, 0, st, n_short, L,
               vorder.get() + n_long, seg_start.get(), seg_pix.get(), seg_w.get(), in, nullptr, src, Live{}, L);
    const bool seq = L <= 2;
    for (int jj = 0; jj <= d; jj++) {
        const int j = reverse ? d - jj : jj;
        if (seq)
            launch(blur_kernel<true>, ceil_div(ML, kTB), kTB, 0, st, M, L, nbr.get() + (long)j * M, src, dst, Live{});
        else
            launch(blur_kernel<false>, ceil_div(ML, kTB), kTB, 0, st, M, L, nbr.get() + (long)j * M, src, dst, Live{});
        std::swap(src, dst);
    }
    const float alpha = 1.0f / (1.0f + std::pow(2.0f, (float)-d));
    const SliceEpilogue ep;
    if (seq)
        launch(slice_kernel<true, 0, 0>, ceil_div(NL, kTB), kTB, 0, st, N, L, d, offset.get(), bary.get(), src, alpha,
               out, ep, Live{});
    else
        launch(slice_kernel<false, 0, 0>, ceil_div(NL, kTB), kTB, 0, st, N, L, d, offset.get(), bary.get(), src, alpha,
               out, ep, Live{});
    DCRF_LAUNCH_CHECK();
}

void Lattice::compute(float* out, const float* in, int L, bool reverse, const SliceEpilogue& ep,
                      const float* pre_norm) {
    splat_blur(in, L, reverse, pre_norm);
    slice(out, L, ep);
}

// Row stride of the plain filter's value buffers: L padded to a multiple of
// four (float4 rows) on the sseCompute path (L > 2); seqCompute (L <= 2)
// keeps L.
static int value_row(int L) { return L > 2 ? (L + 3) & ~3 : L; }

// Blocks of a launch over `units` work items, `per_block` per block of
// `threads` threads: all of them at once, or -- with live images, whose
// units are counted on the device -- twice as many blocks as the SMs hold
// at full occupancy, looping over them.
static int unit_grid(long units, int per_block, bool live, int threads) {
    const long g = std::max(1L, (units + per_block - 1) / per_block);
    return live ? (int)std::min(g, (long)sm_count() * 2 * (2048 / threads)) : (int)g;
}

// The warp splat (L = 21) over order[first, first + count) with `warps`
// vertices per block; with live images, over domain `dom`'s live lists.
static void splat_warp_range(const Lattice& lat, int warps, int dom, int first, int count, int L, int Lp,
                             const float* in, const float* pre_norm, float* vals, cudaStream_t st) {
    if (count <= 0) return;
    const Live lv = lat.live_of(dom);
    const int* order = lat.vorder.get() + (lv.n ? 0 : first);
    auto go = [&](auto kern, int w) {
        launch(kern, unit_grid(count, w, lv.n != nullptr, 32 * w), 32 * w, 0, st, count, L, order, lat.seg_start.get(),
               lat.seg_pix.get(), lat.seg_w.get(), in, pre_norm, vals, lv, Lp);
    };
    if (pre_norm) {
        if (warps == 2) go(splat_warp_kernel<true, 21, 2>, 2);
        else if (warps == 8) go(splat_warp_kernel<true, 21, 8>, 8);
        else go(splat_warp_kernel<true, 21, 4>, 4);
    } else {
        if (warps == 2) go(splat_warp_kernel<false, 21, 2>, 2);
        else if (warps == 8) go(splat_warp_kernel<false, 21, 8>, 8);
        else go(splat_warp_kernel<false, 21, 4>, 4);
    }
}

// The tiled splat (L = 21) over order[first, first + count); with live
// images, over domain `dom`'s live lists.
static void splat_tile_range(const Lattice& lat, int dom, int first, int count, const float* in,
                             const float* pre_norm, float* vals, int Lp, cudaStream_t st) {
    if (count <= 0) return;
    // 38 KB of static shared memory per block: ask for the largest carveout
    // so that kTileBlocksPerSM blocks fit on an SM.
    static const bool carveout = [] {
        DCRF_CUDA(cudaFuncSetAttribute(splat_tile21_kernel<true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
        DCRF_CUDA(cudaFuncSetAttribute(splat_tile21_kernel<false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
        return true;
    }();
    (void)carveout;
    const Live lv = lat.live_of(dom);
    const bool live = lv.n != nullptr;
    const int* order = lat.vorder.get() + (live ? 0 : first);
    // persistent blocks: each walks its tiles with the next tile's ranges and
    // records prefetched
    const int grid = (int)std::min<long>((count + kTV - 1) / kTV, (long)sm_count() * kTileBlocksPerSM);
    launch(pre_norm ? splat_tile21_kernel<true> : splat_tile21_kernel<false>,
           grid, kTileThreads, 0, st, count, order, lat.seg_start.get(),
           lat.seg_pix.get(), lat.seg_w.get(), in, pre_norm, vals, lv, Lp);
}

// Bounded waits of the bulk-copy splat that ran out, since the library
// loaded (read from the current device).
unsigned long long bulk_wait_timeouts() {
    unsigned long long v = 0;
    DCRF_CUDA(cudaMemcpyFromSymbol(&v, g_bulk_wait_timeouts, sizeof(v)));
    return v;
}

// The bulk-copy splat (L = 21) over order[first, first + count) (or domain
// `dom`'s live lists); inputs that are not 16-byte aligned take the tiled
// splat, which computes the same values.
static void splat_bulk_range(const Lattice& lat, int dom, int first, int count, const float* in,
                             const float* pre_norm, float* vals, int Lp, cudaStream_t st) {
    if (count <= 0) return;
    if (reinterpret_cast<uintptr_t>(in) % 16 != 0) {
        splat_tile_range(lat, dom, first, count, in, pre_norm, vals, Lp, st);
        return;
    }
    static const bool carveout = [] {
        DCRF_CUDA(cudaFuncSetAttribute(splat_bulk21_kernel<true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
        DCRF_CUDA(cudaFuncSetAttribute(splat_bulk21_kernel<false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
        return true;
    }();
    (void)carveout;
    const Live lv = lat.live_of(dom);
    const bool live = lv.n != nullptr;
    const int* order = lat.vorder.get() + (live ? 0 : first);
    const int grid = (int)std::min<long>((count + kTV - 1) / kTV, (long)sm_count() * kBulkBlocksPerSM);
    launch(pre_norm ? splat_bulk21_kernel<true> : splat_bulk21_kernel<false>, grid, kTileThreads, 0, st, count,
           order, lat.seg_start.get(), lat.seg_pix.get(), lat.seg_w.get(), in, lat.N, pre_norm, vals, lv, Lp);
}

namespace {
constexpr int kTuneMinPixels = 1 << 18;  // smaller lattices keep the default shapes
std::mutex g_tune_mu;
std::vector<std::pair<std::vector<long>, FilterShape>>& tune_cache() {
    static auto* c = new std::vector<std::pair<std::vector<long>, FilterShape>>();  // never destroyed
    return *c;
}
bool autotune_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("DCRF_AUTOTUNE");
        return !(v && v[0] == '0');
    }();
    return on;
}
}  // namespace

void Lattice::tune_shape(const float* in, int L, const float* pre_norm) {
    shape_L = L;  // also when the defaults stay
    if (N < kTuneMinPixels || !autotune_enabled()) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    DCRF_CUDA(cudaStreamIsCapturing(stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) {  // no timing inside a capture: defaults, tuned next time
        shape_L = 0;
        return;
    }
    int dev = 0;
    DCRF_CUDA(cudaGetDevice(&dev));
    int lg = 0;
    while ((1L << (lg + 1)) <= (long)N) lg++;
    const std::vector<long> key = {dev, L, d, lg, M / std::max(N / 64, 1)};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        for (const auto& e : tune_cache())
            if (e.first == key) {
                shape = e.second;
                return;
            }
    }
    const int Lp = value_row(L);
    cudaStream_t st = stream;
    cudaEvent_t e0, e1;
    DCRF_CUDA(cudaEventCreate(&e0));
    DCRF_CUDA(cudaEventCreate(&e1));
    auto timed = [&](auto&& fn) {
        fn();  // warm
        DCRF_CUDA(cudaEventRecord(e0, st));
        for (int r = 0; r < 3; r++) fn();
        DCRF_CUDA(cudaEventRecord(e1, st));
        DCRF_CUDA(cudaEventSynchronize(e1));
        float ms = 0.0f;
        DCRF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms;
    };
    FilterShape best;
    float* src = va.get();
    float* dst = vb.get();
    float tbest = 1e30f;
    for (int kind = 0; kind < 6; kind++) {
        for (int w : {2, 4, 8}) {
            if ((kind == 0 || kind >= 3) && w != 4) continue;  // no warp splat in these forms
            FilterShape fs = best;
            fs.splat_kind = kind;
            fs.splat_warps = w;
            // as splat_blur runs it: beside the very long lists' splat on the side stream
            const float t = timed([&] {
                const bool fork = splat_huge_fork(in, L, pre_norm, src, false);
                splat_rest(fs, in, L, pre_norm, src, false, st, nullptr);
                if (fork) {
                    DCRF_CUDA(cudaEventRecord(ev_join, aux));
                    DCRF_CUDA(cudaStreamWaitEvent(st, ev_join, 0));
                }
            });
            if (t < tbest) {
                tbest = t;
                best.splat_kind = kind;
                best.splat_warps = w;
            }
        }
    }
    const int Q = Lp / 4;
    const long MQ = (long)M * Q;
    tbest = 1e30f;
    for (int bt : {128, 256, 512}) {
        const float t = timed([&] {
            launch(blur4_kernel<6>, ceil_div(MQ, bt), bt, 0, st, M, Q, nbr.get(), (const float*)src, dst, Live{});
        });
        if (t < tbest) tbest = t, best.blur_threads = bt;
    }
    {
        DevBuf<float> probe;  // the slice candidates write here, not to the caller's output
        float* o = probe.ensure((size_t)N * L);
        const float alpha = 1.0f / (1.0f + std::pow(2.0f, (float)-d));
        const SliceEpilogue ep;
        const int per_px = (d + 1) * 8 + 4 + L * 4;
        tbest = 1e30f;
        for (int tile : {64, 128, 256}) {
            const int tl = std::max(1, std::min(tile, (40 << 10) / per_px));
            const float t = timed([&] {
                auto sl = [&](auto kern) {
                    launch(kern, ceil_div(N, tl), kSliceThreads, (size_t)tl * per_px, st, N, L, Q, d, tl,
                           offset.get(), bary.get(), (const float*)src, alpha, o, ep, Live{},
                           (const long*)nullptr);
                };
                if (d == 5) sl(slice4_kernel<5, 6, 21>);
                else if (d == 2) sl(slice4_kernel<2, 6, 21>);
                else sl(slice4_kernel<0, 0, 0>);
            });
            if (t < tbest) tbest = t, best.slice_tile = tile;
        }
        DCRF_CUDA(cudaStreamSynchronize(st));  // before the probe buffer goes back
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    DCRF_LAUNCH_CHECK();
    shape = best;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_cache().push_back({key, best});
}

void Lattice::splat_rest(const FilterShape& fs, const float* in, int L, const float* pre_norm, float* vals,
                         bool live, cudaStream_t st, cudaStream_t st_short) {
    const int Lp = value_row(L);
    // live images: the short lists are their own domain, splatted on
    // st_short (concurrent with the long lists) when the caller gives one
    cudaStream_t sts = live && st_short ? st_short : st;
    const int nh = n_huge, n_short = M - n_long;
    const int kind = L == 21 ? fs.splat_kind : 0;
    if (kind == 2 && !live) {
        splat_warp_range(*this, fs.splat_warps, kDomLong, nh, M - nh, L, Lp, in, pre_norm, vals, st);
        return;
    }
    if (kind == 3) {  // the tiled splat for every list up to the huge ones
        if (!live) {
            splat_tile_range(*this, kDomLong, nh, M - nh, in, pre_norm, vals, Lp, st);
        } else {
            splat_tile_range(*this, kDomLong, nh, n_long - nh, in, pre_norm, vals, Lp, st);
            splat_tile_range(*this, kDomShort, n_long, n_short, in, pre_norm, vals, Lp, sts);
        }
        return;
    }
    if (kind == 5) {  // the bulk-copy splat for every list up to the huge ones
        if (!live) {
            splat_bulk_range(*this, kDomLong, nh, M - nh, in, pre_norm, vals, Lp, st);
        } else {
            splat_bulk_range(*this, kDomLong, nh, n_long - nh, in, pre_norm, vals, Lp, st);
            splat_bulk_range(*this, kDomShort, n_long, n_short, in, pre_norm, vals, Lp, sts);
        }
        return;
    }
    if (kind == 4) {  // the staged warp splat for the long lists, the tiled splat for the short ones
        if (n_long > nh) {
            const Live lv = live ? live_of(kDomLong) : Live{};
            launch(pre_norm ? splat_kernel<true, 21> : splat_kernel<false, 21>,
                   unit_grid(n_long - nh, kStageWarps, live, 32 * kStageWarps), 32 * kStageWarps, 0, st, n_long - nh,
                   L, vorder.get() + (live ? 0 : nh), seg_start.get(), seg_pix.get(), seg_w.get(), in, pre_norm, vals,
                   lv, Lp);
        }
        splat_tile_range(*this, kDomShort, n_long, n_short, in, pre_norm, vals, Lp, sts);
        return;
    }
    if (n_long > nh) {
        if (kind >= 1) {
            splat_warp_range(*this, fs.splat_warps, kDomLong, nh, n_long - nh, L, Lp, in, pre_norm, vals, st);
        } else {
            const Live lv = live ? live_of(kDomLong) : Live{};
            launch(L == 21 ? (pre_norm ? splat_kernel<true, 21> : splat_kernel<false, 21>)
                           : (pre_norm ? splat_kernel<true> : splat_kernel<false>),
                   unit_grid(n_long - nh, kStageWarps, live, 32 * kStageWarps), 32 * kStageWarps, 0, st, n_long - nh, L,
                   vorder.get() + (live ? 0 : nh), seg_start.get(), seg_pix.get(), seg_w.get(), in, pre_norm, vals,
                   lv, Lp);
        }
    }
    if (n_short) {
        if (kind == 2) {  // live: the short lists are their own domain
            splat_warp_range(*this, fs.splat_warps, kDomShort, n_long, n_short, L, Lp, in, pre_norm, vals, sts);
        } else {
            const Live lv = live ? live_of(kDomShort) : Live{};
            launch(L == 21 ? (pre_norm ? splat_short_kernel<true, 21> : splat_short_kernel<false, 21>)
                           : (pre_norm ? splat_short_kernel<true> : splat_short_kernel<false>),
                   unit_grid((long)n_short * Lp, kTB, live, kTB), kTB, 0, sts, n_short, L, vorder.get() + (live ? 0 : n_long),
                   seg_start.get(), seg_pix.get(), seg_w.get(), in, pre_norm, vals, lv, Lp);
        }
    }
}

// The lists longer than kHugeList (the first n_huge of the order) run on the
// high-priority side stream while the others are splatted: with L = 21 by
// the transposing ring (one warp's chain sets their time, and its three
// chunks of copies in flight hide the load latency a lone warp cannot hide
// otherwise), else by splat_kernel.  Forks the side stream from `stream`
// when there are such lists or `fork_anyway`; the caller joins it.
bool Lattice::splat_huge_fork(const float* in, int L, const float* pre_norm, float* vals, bool fork_anyway) {
    const int nh = n_huge;
    if (nh == 0 && !fork_anyway) return false;
    const int Lp = value_row(L);
    const bool live = live_n != nullptr;
    ensure_aux();
    DCRF_CUDA(cudaEventRecord(ev_fork, stream));
    DCRF_CUDA(cudaStreamWaitEvent(aux, ev_fork, 0));
    if (nh > 0) {
        const Live lv = live_of(kDomHuge);
        const int g = unit_grid(nh, kStageWarps, live, 32 * kStageWarps);
        if (L == 21)
            launch(pre_norm ? splat_ring21_kernel<true> : splat_ring21_kernel<false>, g, 32 * kStageWarps, 0, aux,
                   nh, vorder.get(), seg_start.get(), seg_pix.get(), seg_w.get(), in, pre_norm, vals, lv, Lp);
        else
            launch(pre_norm ? splat_kernel<true> : splat_kernel<false>, g, 32 * kStageWarps, 0, aux, nh, L,
                   vorder.get(), seg_start.get(), seg_pix.get(), seg_w.get(), in, pre_norm, vals, lv, Lp);
    }
    return true;
}

void Lattice::splat_blur(const float* in, int L, bool reverse, const float* pre_norm) {
    require(L >= 1, DCRF_E_ARG, "compute: L must be >= 1");
    const int Lp = value_row(L);
    ensure_values((size_t)Lp);
    if (L == 21 && shape_L != L) tune_shape(in, L, pre_norm);
    cudaStream_t st = stream;
    const long ML = (long)M * L;
    float *src = va.get(), *dst = vb.get();
    // A batched solve's live images: only their lists, vertices and pixels.
    const bool live = live_n != nullptr;
    // As in the ordered filter, the very long lists run on the side stream
    // (splat_huge_fork).  With live images the short lists are a separate launch: it runs on the
    // side stream too (after the very long lists), beside the long lists'.
    const bool fork_short = live && M - n_long > 0 && n_long > n_huge;
    const bool forked = splat_huge_fork(in, L, pre_norm, src, fork_short);
    splat_rest(shape, in, L, pre_norm, src, live, st, fork_short ? aux : nullptr);
    if (forked) {
        DCRF_CUDA(cudaEventRecord(ev_join, aux));
        DCRF_CUDA(cudaStreamWaitEvent(st, ev_join, 0));
    }
    const bool seq = L <= 2;
    const int Q = Lp / 4;
    const long MQ = (long)M * Q;
    const Live lvv = live_of(kDomVert);
    for (int jj = 0; jj <= d; jj++) {
        const int j = reverse ? d - jj : jj;
        const int2* nb = nbr.get() + (long)j * M;
        if (seq) {
            launch(blur_kernel<true>, unit_grid(ML, kTB, live, kTB), kTB, 0, st, M, L, nb, src, dst, lvv);
        } else if (Q == 6) {
            const int bt = shape.blur_threads;
            launch(blur4_kernel<6>, unit_grid(MQ, bt, live, bt), bt, 0, st, M, Q, nb, src, dst, lvv);
        } else {
            launch(blur4_kernel<0>, unit_grid(MQ, kTB, live, kTB), kTB, 0, st, M, Q, nb, src, dst, lvv);
        }
        std::swap(src, dst);
    }
    plain_vals = src;
    plain_L = L;
}

int Lattice::slice_tile_for(int L) const {
    // pixels per tile: kSliceTile (the tuned size for L = 21), fewer for very
    // wide rows (40 KB of shared memory at most)
    const int per_px = (d + 1) * 8 + 4 + L * 4;
    return std::max(1, std::min(L == 21 ? shape.slice_tile : kSliceTile, (40 << 10) / per_px));
}

void Lattice::slice(float* out, int L, const SliceEpilogue& ep) {
    require(plain_vals && plain_L == L, DCRF_E_STATE, "slice: no splat_blur for this label count before it");
    cudaStream_t st = stream;
    const long NL = (long)N * L;
    const float* src = plain_vals;
    const float alpha = 1.0f / (1.0f + std::pow(2.0f, (float)-d));
    const bool live = live_n != nullptr;
    if (L <= 2) {
        launch(slice_kernel<true, 0, 0>, unit_grid(NL, kTB, live, kTB), kTB, 0, st, N, L, d, offset.get(), bary.get(),
               src, alpha, out, ep, live_of(kDomPix));
    } else {
        const int Q = value_row(L) / 4;
        const int per_px = (d + 1) * 8 + 4 + L * 4;
        // live images: tiles of each image's pixels, the size prepare_live fixed
        const int tile = live ? dom_tile : slice_tile_for(L);
        require(tile > 0, DCRF_E_STATE, "slice: live images without prepare_live");
        const size_t smem = (size_t)tile * per_px;
        const long* pix_base = live ? dom_base.get() + (long)kDomPix * (images + 1) : nullptr;
        auto sl = [&](auto kern) {
            launch(kern, unit_grid(N, tile, live, kSliceThreads), kSliceThreads, smem, st, N, L, Q, d, tile, offset.get(),
                   bary.get(), src, alpha, out, ep, live_of(kDomTile), pix_base);
        };
        if (d == 5 && L == 21) sl(slice4_kernel<5, 6, 21>);
        else if (d == 2 && L == 21) sl(slice4_kernel<2, 6, 21>);
        else sl(slice4_kernel<0, 0, 0>);
    }
    DCRF_LAUNCH_CHECK();
}

void Lattice::compute_ord(float* out, const float* Q, int L, const SliceEpilogue& ep) {
    require(L >= 1, DCRF_E_ARG, "compute_ord: L must be >= 1");
    const long NL = (long)N * L;
    float2* bins = obins.ensure((size_t)NL);
    ord_bins(bins, Q, NL, stream);
    compute_ord_bins(out, bins, L, ep, nullptr);
}

void rescaled_bins(float2* bins, const float* Q, long n, const float* qminmax, cudaStream_t st) {
    if (aligned16(Q) && aligned16(bins)) {
        const long n4 = n / 4;
        if (n4) launch(rescaled_bins4_kernel, ceil_div(n4, kTB), kTB, 0, st, n4, reinterpret_cast<const float4*>(Q),
                       qminmax, reinterpret_cast<float4*>(bins));
        if (n > 4 * n4)
            launch(rescaled_bins_kernel, 1, kTB, 0, st, n - 4 * n4, Q + 4 * n4, qminmax, bins + 4 * n4);
    } else {
        launch(rescaled_bins_kernel, ceil_div(n, kTB), kTB, 0, st, n, Q, qminmax, bins);
    }
    DCRF_LAUNCH_CHECK();
}

int slice_grid(long n) { return ceil_div(n, kTB); }

void Lattice::compute_ord_bins(float* out, const float2* bins, int L, const SliceEpilogue& ep,
                               const GapFusion* gap) {
    ord_splat_blur(bins, L);
    ord_slice(out, bins, L, ep, gap);
}

void Lattice::ord_splat_blur(const float2* bins, int L) {
    require(L >= 1, DCRF_E_ARG, "compute_ord: L must be >= 1");
    const size_t row = (size_t)L * kOrdW;
    ensure_values(row);
    cudaStream_t st = stream;
    float *src = va.get(), *dst = vb.get();
    const int n_short = M - n_long;
    if (n_long && L <= kOrdBlockMaxL) {
        // Lists longer than kHugeList (the first n_huge of the order) are
        // shared by blocks of kHugeLabels labels x 10 bins, so that they
        // finish early; the rest take one block per list with the bin split
        // that issues the fewest instructions per entry.
        auto run = [&](int G, int kb, int first, int count, cudaStream_t rs) {
            if (count <= 0) return;
            const int kblocks = (L + kb - 1) / kb;
            const int threads = ((kb * G + 31) / 32) * 32;
            const size_t smem = ord_block_smem(kb);
            auto kern = G == 10 ? ord_splat_block_kernel<10>
                      : G == 5  ? ord_splat_block_kernel<5>
                      : G == 3  ? ord_splat_block_kernel<3>
                      : G == 2  ? ord_splat_block_kernel<2>
                                : ord_splat_block_kernel<1>;
            if (smem > 48 * 1024)  // opt-in size: a per-device function attribute, set on every such call
                DCRF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            launch(kern, count * kblocks, threads, smem, rs, L, kb, kblocks, vorder.get() + first,
                   seg_start.get(), seg_pix.get(), seg_w.get(), bins, src);
        };
        // The very long lists set the length of their kernel while leaving
        // most SMs idle; they run on a high-priority side stream, forked
        // after the value buffers are ready and joined before the blur, so
        // the other splats (disjoint vertex rows) fill those SMs meanwhile.
        if (n_huge > 0) {
            ensure_aux();
            DCRF_CUDA(cudaEventRecord(ev_fork, st));
            DCRF_CUDA(cudaStreamWaitEvent(aux, ev_fork, 0));
            run(10, kHugeLabels, 0, n_huge, aux);
            DCRF_CUDA(cudaEventRecord(ev_join, aux));
        }
        run(ord_groups_cheapest(L), L, n_huge, n_long - n_huge, st);
    } else if (n_long) {
        launch(ord_splat_kernel, ceil_div(2L * n_long, kStageWarps), 32 * kStageWarps, 0, st, n_long, L,
               vorder.get(), seg_start.get(), seg_pix.get(), seg_w.get(), bins, src);
    }
    if (n_short)
        launch(ord_splat_short_kernel<0>, ceil_div((long)n_short * L, kTB), kTB, 0, st, n_short, L,
               vorder.get() + n_long, seg_start.get(), seg_pix.get(), seg_w.get(), bins, src);
    if (n_long && L <= kOrdBlockMaxL && n_huge > 0) DCRF_CUDA(cudaStreamWaitEvent(st, ev_join, 0));
    const int row4 = (int)(row / 4);
    for (int j = 0; j <= d; j++) {
        auto kern = row4 == 105 ? ord_blur_kernel<105> : ord_blur_kernel<0>;  // 105 = 20 bins x 21 labels / 4
        launch(kern, ceil_div((long)M * row4, kTB), kTB, 0, st, M, row4, nbr.get() + (long)j * M,
               reinterpret_cast<const float4*>(src), reinterpret_cast<float4*>(dst));
        std::swap(src, dst);
    }
    ord_vals = src;
}

void Lattice::ord_slice_pair(float* out, const float2* bins, int L, const Lattice& a, const SliceEpilogue& ea,
                             const Lattice& b, const SliceEpilogue& eb, const GapFusion* gap) {
    require(a.ord_vals && b.ord_vals, DCRF_E_STATE, "ord_slice_pair: no ord_splat_blur before it");
    require(a.N == b.N, DCRF_E_ARG, "ord_slice_pair: lattices over different pixel counts");
    const long NL = (long)a.N * L;
    const OrdSliceTerm t0{a.offset.get(), a.bary.get(), a.ord_vals, a.d, 1.0f / (1.0f + std::pow(2.0f, (float)-a.d)),
                          ea};
    const OrdSliceTerm t1{b.offset.get(), b.bary.get(), b.ord_vals, b.d, 1.0f / (1.0f + std::pow(2.0f, (float)-b.d)),
                          eb};
    const GapFusion gf = gap ? *gap : GapFusion{};
    auto sl = [&](auto kern) {
        launch(kern, ceil_div(NL, kTB), kTB, 0, a.stream, a.N, L, t0, t1, bins, out, gf);
    };
    if (L == 21 && a.d == 2 && b.d == 5) {
        launch(gap ? ord_slice_pair_staged<true> : ord_slice_pair_staged<false>, ceil_div(NL, kTB), kTB, 0,
               a.stream, a.N, t0, t1, bins, out, gf);
    } else if (gap) {
        sl(ord_slice_pair_kernel<true, 0, 0, 0>);
    } else {
        sl(ord_slice_pair_kernel<false, 0, 0, 0>);
    }
    DCRF_LAUNCH_CHECK();
}

void Lattice::ord_slice(float* out, const float2* bins, int L, const SliceEpilogue& ep, const GapFusion* gap) {
    require(ord_vals, DCRF_E_STATE, "ord_slice: no ord_splat_blur before it");
    cudaStream_t st = stream;
    const long NL = (long)N * L;
    const float* src = ord_vals;
    const float alpha = 1.0f / (1.0f + std::pow(2.0f, (float)-d));
    const GapFusion gf = gap ? *gap : GapFusion{};
    auto sl = [&](auto kern) {
        launch(kern, ceil_div(NL, kTB), kTB, 0, st, N, L, d, offset.get(), bary.get(), src, bins, alpha, out, ep, gf);
    };
    if (gap) {
        if (L == 21 && d == 5) sl(ord_slice_kernel<true, 5, 21>);
        else if (L == 21 && d == 2) sl(ord_slice_kernel<true, 2, 21>);
        else sl(ord_slice_kernel<true, 0, 0>);
    } else {
        if (L == 21 && d == 5) sl(ord_slice_kernel<false, 5, 21>);
        else if (L == 21 && d == 2) sl(ord_slice_kernel<false, 2, 21>);
        else sl(ord_slice_kernel<false, 0, 0>);
    }
    DCRF_LAUNCH_CHECK();
}


// ---------------------------------------------------------------------------
// The restricted ordered filter (seqCompute_upper_minus_lower_ord_restricted,
// src/permutohedral.cpp:702-900).
//
// Splat, per (vertex, label) and both passes: the vertex's list in pixel
// order, first the pixels outside pI with their Q values (only in a store
// call; the sums are then kept), then the pixels of pI with their rQ values.
// That is the reference's order per bin: its outside-pI loop runs over all
// pixels before its pI loop.
__global__ void ord_splat_restricted_kernel(int M, int L, const int* __restrict__ seg_start,
                                            const int* __restrict__ seg_pix, const float* __restrict__ seg_w,
                                            const int* __restrict__ pos, const float2* __restrict__ ebins,
                                            const float2* __restrict__ rbins, float* __restrict__ stored,
                                            float* __restrict__ vals, unsigned char* __restrict__ active, int store) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)M * L) return;
    const int v = (int)(t / L), k = (int)(t - (long)v * L);
    const int s0 = seg_start[v], s1 = seg_start[v + 1];
    const long rowoff = (long)(v + 1) * kOrdW * L + k;
    unsigned long long acc[kRes];  // (lower, upper) sums of bin b
    if (store) {
#pragma unroll
        for (int b = 0; b < kRes; b++) acc[b] = 0ull;
        bool any = false;
        for (int s = s0; s < s1; s++) {
            const int p = seg_pix[s];
            if (pos[p] >= 0) {
                any = true;
                continue;
            }
            const float2 x = ebins[(long)p * L + k];
            const float w = seg_w[s];
            const unsigned long long w2 = pack2(w, w);
#pragma unroll
            for (int b = 0; b < kRes; b++) ord_step2(acc[b], x.x, x.y, (float)b, w2);
        }
#pragma unroll
        for (int b = 0; b < kRes; b++) {
            const float2 r = unpack2(acc[b]);
            stored[rowoff + (long)b * L] = r.x;
            stored[rowoff + (long)(kRes + b) * L] = r.y;
        }
        if (k == 0) active[v] = any ? 1 : 0;
    } else {
#pragma unroll
        for (int b = 0; b < kRes; b++)
            acc[b] = pack2(stored[rowoff + (long)b * L], stored[rowoff + (long)(kRes + b) * L]);
    }
    for (int s = s0; s < s1; s++) {
        const int ii = pos[seg_pix[s]];
        if (ii < 0) continue;
        const float2 x = rbins[(long)ii * L + k];
        const float w = seg_w[s];
        const unsigned long long w2 = pack2(w, w);
#pragma unroll
        for (int b = 0; b < kRes; b++) ord_step2(acc[b], x.x, x.y, (float)b, w2);
    }
#pragma unroll
    for (int b = 0; b < kRes; b++) {
        const float2 r = unpack2(acc[b]);
        vals[rowoff + (long)b * L] = r.x;
        vals[rowoff + (long)(kRes + b) * L] = r.y;
    }
}

// Blur of the active vertices only; the others keep whatever their row of dst
// holds (:773-789: the reference's two buffers swap after every axis, so an
// inactive vertex reads as 0 after odd axes and as its splat after even ones).
__global__ void ord_blur_active_kernel(int M, int row4, const int2* __restrict__ nbr,
                                       const unsigned char* __restrict__ active, const float4* __restrict__ src,
                                       float4* __restrict__ dst) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)M * row4) return;
    const int v = (int)(t / row4), c = (int)(t - (long)v * row4);
    if (!active[v]) return;
    const int2 nb = nbr[v];
    const float4 a = src[(long)(v + 1) * row4 + c];
    const float4 p = src[(long)nb.x * row4 + c];
    const float4 q = src[(long)nb.y * row4 + c];
    float4 r;
    r.x = fadd(a.x, fmul(0.5f, fadd(p.x, q.x)));
    r.y = fadd(a.y, fmul(0.5f, fadd(p.y, q.y)));
    r.z = fadd(a.z, fmul(0.5f, fadd(p.z, q.z)));
    r.w = fadd(a.w, fmul(0.5f, fadd(p.w, q.w)));
    dst[(long)(v + 1) * row4 + c] = r;
}

// Slice at the pI pixels (:791-802, :885-896), as ord_slice_kernel does for
// every pixel; out [nP][L] starts from 0.
__global__ void ord_slice_restricted_kernel(int nP, int L, int d, const int* __restrict__ pI,
                                            const int* __restrict__ offset, const float* __restrict__ bary,
                                            const float* __restrict__ vals, const float2* __restrict__ rbins,
                                            float alpha, float* out, SliceEpilogue ep) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)nP * L) return;
    const int ii = (int)(t / L), k = (int)(t - (long)ii * L);
    const int i = pI[ii], d1 = d + 1;
    const float2 bp = rbins[t];
    const int cl = ord_lower_of(bp), cu = ord_upper_of(bp);
    float acc = 0.0f;
    for (int j = 0; j <= d; j++) {
        const int o = offset[(long)i * d1 + j];
        const float w = bary[(long)i * d1 + j];
        acc = fadd(acc, fmul(vals[((long)(o + 1) * kOrdW + cl) * L + k], fmul(-w, alpha)));
    }
    for (int j = 0; j <= d; j++) {
        const int o = offset[(long)i * d1 + j];
        const float w = bary[(long)i * d1 + j];
        acc = fadd(acc, fmul(vals[((long)(o + 1) * kOrdW + kRes + cu) * L + k], fmul(w, alpha)));
    }
    out[t] = apply_epilogue(acc, t, i, k, ep);
}

__global__ void scatter_pos_kernel(int nP, const int* __restrict__ pI, int* __restrict__ pos) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nP) pos[pI[t]] = t;
}

void Lattice::compute_ord_restricted(float* rout, const float* rQ, const int* pI, int nP, const float* Q, int L,
                                     bool store, const SliceEpilogue& ep) {
    require(L >= 1, DCRF_E_ARG, "compute_ord_restricted: L must be >= 1");
    require(nP >= 0 && nP <= N, DCRF_E_ARG, "compute_ord_restricted: pI larger than the lattice");
    require(store || r_L == L, DCRF_E_STATE,
            "compute_ord_restricted: no stored splat for this label count (call with store first)");
    require(!store || Q, DCRF_E_ARG, "compute_ord_restricted: store needs Q");
    cudaStream_t st = stream;
    const long row = (long)L * kOrdW, cells = (long)(M + 1) * row;
    float* stored = r_stored.ensure((size_t)cells);
    float* a = r_a.ensure((size_t)cells);
    float* b = r_b.ensure((size_t)cells);
    unsigned char* active = r_active.ensure((size_t)std::max(M, 1));
    int* pos = r_pos.ensure((size_t)N);
    float2* rb = r_bins.ensure((size_t)std::max<long>((long)nP * L, 1));
    launch(fill_int_kernel, ceil_div(N, kTB), kTB, 0, st, (long)N, -1, pos);
    if (nP) {
        launch(scatter_pos_kernel, ceil_div(nP, kTB), kTB, 0, st, nP, pI, pos);
        ord_bins(rb, rQ, (long)nP * L, st);
    }
    const float2* eb = nullptr;
    if (store) {
        float2* e = r_ebins.ensure((size_t)N * L);
        ord_bins(e, Q, (long)N * L, st);
        eb = e;
        r_L = 0;  // until this call has stored its splat
    }
    DCRF_CUDA(cudaMemsetAsync(a, 0, sizeof(float) * row, st));      // row 0: the absent neighbour
    DCRF_CUDA(cudaMemsetAsync(b, 0, sizeof(float) * cells, st));    // new_values_ starts zeroed
    if (M)
        launch(ord_splat_restricted_kernel, ceil_div((long)M * L, kTB), kTB, 0, st, M, L, seg_start.get(),
               seg_pix.get(), seg_w.get(), (const int*)pos, eb, (const float2*)rb, stored, a, active, (int)store);
    float *src = a, *dst = b;
    const int row4 = (int)(row / 4);
    for (int j = 0; j <= d; j++) {
        if (M)
            launch(ord_blur_active_kernel, ceil_div((long)M * row4, kTB), kTB, 0, st, M, row4,
                   nbr.get() + (long)j * M, (const unsigned char*)active, reinterpret_cast<const float4*>(src),
                   reinterpret_cast<float4*>(dst));
        std::swap(src, dst);
    }
    const float alpha = 1.0f / (1.0f + std::pow(2.0f, (float)-d));
    if (nP)
        launch(ord_slice_restricted_kernel, ceil_div((long)nP * L, kTB), kTB, 0, st, nP, L, d, pI, offset.get(),
               bary.get(), (const float*)src, (const float2*)rb, alpha, rout, ep);
    DCRF_LAUNCH_CHECK();
    if (store) r_L = L;
}

}  // namespace dcrf
