// Per-pixel and reduction kernels shared by model.cu and solvers.cu.
#pragma once
#include <type_traits>

#include "reduce.cuh"

namespace dcrf {

constexpr int kLMax = 64;  // largest label count of the run-time-L kernels

// Runs f(std::integral_constant<int, LC>) with LC = L for the label counts
// that have a fully unrolled register instantiation, else LC = 0 (run-time L).
template <typename F>
void with_lc(int L, F&& f) {
    require(L >= 1 && L <= kLMax, DCRF_E_ARG, "label count must be in [1, 64]");
    if (L == 21) f(std::integral_constant<int, 21>{});
    else f(std::integral_constant<int, 0>{});
}

template <int LC>
struct PixVec {
    static constexpr int S = LC > 0 ? LC : kLMax;
};

// ---------------------------------------------------------------------------
// Row tiles: the [32][LC] rows of 32 consecutive pixels are contiguous in
// global memory; a warp moves them through shared memory so that its global
// loads and stores coalesce, while each lane works on one pixel's row
// (stride LC; odd LC is bank-conflict free).  Rows of lanes >= npix hold
// stale data and are never written back.
constexpr int kTileWarps = 4;

template <int LC>
__device__ __forceinline__ void tile_in(float* buf, const float* __restrict__ g, long pix0, int npix, int lane) {
    const float* src = g + pix0 * LC;
    const int n = npix * LC;
#pragma unroll
    for (int j = 0; j < LC; j++) {
        const int idx = j * 32 + lane;
        if (idx < n) buf[idx] = src[idx];
    }
}

template <int LC>
__device__ __forceinline__ void tile_out(const float* buf, float* __restrict__ g, long pix0, int npix, int lane) {
    float* dst = g + pix0 * LC;
    const int n = npix * LC;
#pragma unroll
    for (int j = 0; j < LC; j++) {
        const int idx = j * 32 + lane;
        if (idx < n) dst[idx] = buf[idx];
    }
}

// Sum of one double per thread over a block of any size (multiple of 32);
// the result is valid in thread 0.  Fixed order: deterministic.
__device__ __forceinline__ double block_sum_any(double v, double* s32) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) s32[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s32[w];
    return t;
}

namespace {

// One warp per value: sums nblk partials in a fixed order.
__global__ void finalize_sums_kernel(const double* __restrict__ partials, int nblk, int nv, int dst,
                                     SolverScalars* sc) {
    const int j = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (j >= nv) return;
    double s = 0.0;
    const double* p = partials + (long)j * nblk;
    int b = lane;
    for (; b + 7 * 32 < nblk; b += 8 * 32) {  // loads batched, sums in order
        double x[8];
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = p[b + i * 32];
#pragma unroll
        for (int i = 0; i < 8; i++) s += x[i];
    }
    for (; b < nblk; b += 32) s += p[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(kFullMask, s, o);
    if (lane == 0) sc->sums[dst + j] = s;
}

// One 1024-thread block per value, for large partial counts: fixed order.
__global__ void finalize_large_kernel(const double* __restrict__ partials, int nblk, int dst, SolverScalars* sc) {
    __shared__ double s[32];
    const int j = blockIdx.x;
    double v = 0.0;
    const double* p = partials + (long)j * nblk;
    const int bd = blockDim.x;
    int b = threadIdx.x;
    // eight loads in flight, then their sums in the same order as one at a time
    for (; b + 7 * bd < nblk; b += 8 * bd) {
        double x[8];
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = p[b + i * bd];
#pragma unroll
        for (int i = 0; i < 8; i++) v += x[i];
    }
    for (; b < nblk; b += bd) v += p[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFullMask, v, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s[w];
        sc->sums[dst + j] = t;
    }
}

__global__ void dot_kernel(long n, const float* __restrict__ a, const float* __restrict__ b,
                           double* __restrict__ partials) {
    double v[1] = {0.0};
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
        v[0] += (double)a[t] * (double)b[t];
    block_sum_store<1>(v, partials);
}

// min / max that carry a NaN through (fminf / fmaxf drop it): equal to
// fminf / fmaxf on numbers, NaN as soon as either side is NaN, so a NaN
// anywhere in the data reaches the result.
__device__ __forceinline__ float nan_min(float a, float b) { return a != a ? a : (b != b ? b : fminf(a, b)); }
__device__ __forceinline__ float nan_max(float a, float b) { return a != a ? a : (b != b ? b : fmaxf(a, b)); }

// min / max of x (exact, so order-free): per-block partials stored as
// doubles, then minmax_finish_kernel combines them into sc->qmin / sc->qmax.
__global__ void minmax_partial_kernel(long n, const float* __restrict__ x, double* __restrict__ partials) {
    __shared__ float smin[kRedThreads / 32], smax[kRedThreads / 32];
    float mn = INFINITY, mx = -INFINITY;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        const float v = x[t];
        mn = nan_min(mn, v);
        mx = nan_max(mx, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = nan_min(mn, __shfl_down_sync(kFullMask, mn, o));
        mx = nan_max(mx, __shfl_down_sync(kFullMask, mx, o));
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        smin[w] = mn;
        smax[w] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < kRedThreads / 32; i++) {
            mn = nan_min(mn, smin[i]);
            mx = nan_max(mx, smax[i]);
        }
        partials[blockIdx.x] = mn;
        partials[gridDim.x + blockIdx.x] = mx;
    }
}

// Launched with one block of any multiple of 32 threads (<= 1024).  Also
// records in sc->numeric a NaN or infinity among the values (bit 2) and
// rescale's "Maxval < 0" condition, max(x - min x) < 0 (bit 4,
// src/eigen_utils.cpp:136-138).
__global__ void minmax_finish_kernel(const double* __restrict__ partials, int nblk, SolverScalars* sc) {
    __shared__ float smn[32], smx[32];
    float mn = INFINITY, mx = -INFINITY;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
        mn = nan_min(mn, (float)partials[b]);
        mx = nan_max(mx, (float)partials[nblk + b]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = nan_min(mn, __shfl_down_sync(kFullMask, mn, o));
        mx = nan_max(mx, __shfl_down_sync(kFullMask, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        smn[threadIdx.x >> 5] = mn;
        smx[threadIdx.x >> 5] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
            mn = nan_min(mn, smn[w]);
            mx = nan_max(mx, smx[w]);
        }
        sc->qmin = mn;
        sc->qmax = mx;
        if (!(isfinite(mn) && isfinite(mx))) sc->numeric |= 2;
        else if (fsub(mx, mn) < 0.0f) sc->numeric |= 4;
    }
}

// A NaN or infinity in a solver's inputs (the initial Q, the unaries):
// sc->numeric |= 1, one atomicOr per block that saw one.  float4 loads when
// both arrays are 16-byte aligned (the tail and unaligned arrays by floats);
// nonfinite_grid(n) blocks of 256 threads keep enough loads in flight for
// HBM rate.
__device__ __forceinline__ bool nonfinite4(float4 v) {
    return !isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z) || !isfinite(v.w);
}
__global__ void nonfinite_kernel(long n, const float* __restrict__ a, const float* __restrict__ b,
                                 SolverScalars* sc) {
    bool bad = false;
    const long t0 = (long)blockIdx.x * blockDim.x + threadIdx.x, stride = (long)gridDim.x * blockDim.x;
    long head = 0;
    if (((reinterpret_cast<unsigned long long>(a) | reinterpret_cast<unsigned long long>(b)) & 15) == 0) {
        const long n4 = n / 4;
        const float4* a4 = reinterpret_cast<const float4*>(a);
        const float4* b4 = reinterpret_cast<const float4*>(b);
        for (long t = t0; t < n4; t += stride) bad |= nonfinite4(a4[t]) || nonfinite4(b4[t]);
        head = n4 * 4;
    }
    for (long t = head + t0; t < n; t += stride) bad |= !isfinite(a[t]) || !isfinite(b[t]);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&sc->numeric, 1);
}
inline int nonfinite_grid(long n) {
    const long g = (n / 4 + 255) / 256;
    return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

// rescale (src/eigen_utils.cpp:120-141): out = (Q - min) / (max - min);
// max(Q - min) equals fl(max Q - min) because rounding is monotone.
__global__ void rescale_kernel(long n, const float* __restrict__ Q, const SolverScalars* __restrict__ sc,
                               float* __restrict__ out) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float mn = sc->qmin, mx = fsub(sc->qmax, sc->qmin);
    float v = fsub(Q[t], mn);
    if (mx > 0.0f) v = v / mx;
    out[t] = v;
}

// Eigen 3.2's pexp<Packet4f> (Core/arch/SSE/MathFunctions.h:107-170) as
// the reference's SSE2 build evaluates it, one lane: the Cephes
// single-precision exp -- clamp to +-88.376, n = floor(x log2(e) + 1/2) by
// truncation and correction, x - n C1 - n C2, the degree-5 polynomial by
// Horner steps (pmadd is a separate multiply and add there, so each rounds),
// times 2^n built in the exponent bits, then the max with the input.
__device__ __forceinline__ float eigen_pexp(float x0) {
    float x = x0 < 88.3762626647950f ? x0 : 88.3762626647950f;
    x = x > -88.3762626647949f ? x : -88.3762626647949f;
    float fx = fadd(fmul(x, 1.44269504088896341f), 0.5f);
    float t = (float)(int)fx;
    if (t > fx) t = fsub(t, 1.0f);
    fx = t;
    x = fsub(x, fmul(fx, 0.693359375f));
    x = fsub(x, fmul(fx, -2.12194440e-4f));
    const float z = fmul(x, x);
    float y = 1.9875691500E-4f;
    y = fadd(fmul(y, x), 1.3981999507E-3f);
    y = fadd(fmul(y, x), 8.3334519073E-3f);
    y = fadd(fmul(y, x), 4.1665795894E-2f);
    y = fadd(fmul(y, x), 1.6666665459E-1f);
    y = fadd(fmul(y, x), 5.0000001201E-1f);
    y = fadd(fmul(y, z), x);
    y = fadd(y, 1.0f);
    const float r = fmul(y, __int_as_float(((int)fx + 0x7f) << 23));
    return r > x0 ? r : x0;
}

// expAndNormalize(-U) (src/densecrf.cpp:321-336): Eigen evaluates
// b.array().exp() with its packet exp over the aligned packets of four and
// std::exp (libm expf, within 0.502 ulp) over the tail; the tail here is the
// double-precision exp rounded once to float, which is the nearest float and
// equals libm's except where the exact value lies within 0.002 ulp of a
// rounding boundary.  The sum is Eigen's packet redux, then one division.
template <int LC>
__global__ void unary_init_kernel(int N, int Lrt, const float* __restrict__ U, float* __restrict__ Q) {
    const int L = LC ? LC : Lrt;
    const int L4 = L & ~3;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float b[PixVec<LC>::S];
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) b[k] = -U[(long)i * L + k];
    float mx = b[0];
#pragma unroll
    for (int k = 1; k < PixVec<LC>::S; k++)
        if (k < L && b[k] > mx) mx = b[k];
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) {
            const float v = fsub(b[k], mx);
            b[k] = k < L4 ? eigen_pexp(v) : (float)exp((double)v);
        }
    const float s = vec_sum<LC>(b, L);
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) Q[(long)i * L + k] = b[k] / s;
}

// currentMap (src/densecrf.cpp:929-938): first arg-max.
template <int LC>
__global__ void current_map_kernel(int N, int Lrt, const float* __restrict__ Q, int16_t* __restrict__ lab) {
    const int L = LC ? LC : Lrt;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float* q = Q + (long)i * L;
    float best = q[0];
    int bi = 0;
#pragma unroll
    for (int k = 1; k < PixVec<LC>::S; k++)
        if (k < L) {
            float v = q[k];
            if (v > best) {
                best = v;
                bi = k;
            }
        }
    lab[i] = (int16_t)bi;
}

// Q(j, i) = (l[i] == j) ? 0 : 1 (src/densecrf.cpp:915-917).
__global__ void onehot_complement_kernel(int N, int L, const int16_t* __restrict__ lab, float* __restrict__ Q) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)N * L) return;
    const int i = (int)(t / L), j = (int)(t - (long)i * L);
    Q[t] = lab[i] == j ? 0.0f : 1.0f;
}

// r[i] += -Q(l[i], i) (src/densecrf.cpp:920-925, 908-910).
__global__ void pairwise_pick_kernel(int N, int L, const int16_t* __restrict__ lab, const float* __restrict__ o,
                                     float* __restrict__ pw, bool first) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int l = lab[i];
    const float r = (0 <= l && l < L) ? -o[(long)i * L + l] : 0.0f;
    pw[i] = fadd(first ? 0.0f : pw[i], r);
}

// sum_i (unary(l_i, i) + pairwise_i) in double (src/densecrf.cpp:877-884).
__global__ void energy_sum_kernel(int N, int L, const int16_t* __restrict__ lab, const float* __restrict__ U,
                                  const float* __restrict__ pw, double* __restrict__ partials) {
    double v[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int l = lab[i];
        const float u = (0 <= l && l < L) ? U[(long)i * L + l] : 0.0f;
        v[0] += (double)fadd(u, pw[i]);
    }
    block_sum_store<1>(v, partials);
}

// Clique r "changes label" when l[p] != l[idx[0]] for some clique-local
// index p (the reference compares l[pix] with pix the loop index,
// src/densecrf.cpp:859-864).
__global__ void clique_label_change_kernel(const int* __restrict__ off, const int* __restrict__ idx,
                                           const int16_t* __restrict__ lab, int* __restrict__ flags) {
    const int r = blockIdx.x;
    const int s0 = off[r], sz = off[r + 1] - s0;
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    if (sz > 0) {
        const int16_t prev = lab[idx[s0]];
        int mine = 0;
        for (int p = threadIdx.x; p < sz; p += blockDim.x) mine |= lab[p] != prev;
        if (mine) any = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) flags[r] = any;
}

__global__ void energy_ho_finish_kernel(int R, const int* __restrict__ flags, const float* __restrict__ ew,
                                        SolverScalars* sc) {
    double e = sc->sums[0], ho = 0.0;
    for (int r = 0; r < R; r++) {
        if (flags[r]) e += (double)ew[r];
        ho += (double)fmul((float)(R - 1), ew[r]);
    }
    sc->sums[0] = e + ho;
}

// Per clique: max over labels of (max - min of Q over the clique's pixels)
// (src/densecrf.cpp:1020-1034).  The per-label max / min do not depend on
// the order of the pixels, so they are taken per chunk of kCliqueChunk
// pixels (one block per chunk, coalesced reads of the pixels' rows, all SMs
// busy however uneven the clique sizes) and then over each clique's chunks;
// the max over labels runs in label order as Eigen's maxCoeff does.
__global__ void __launch_bounds__(256)
    clique_maxdiff_chunk_kernel(const int2* __restrict__ chunks, const int* __restrict__ off,
                                const int* __restrict__ idx, const int* __restrict__ ubase, int L,
                                const float* __restrict__ Q, float2* __restrict__ part) {
    __shared__ float smx[256], smn[256];
    const int2 rc = chunks[blockIdx.x];
    const int r = rc.x, c = rc.y, t = threadIdx.x;
    const int s0 = off[r], sz = off[r + 1] - s0, nch = (sz + kCliqueChunk - 1) / kCliqueChunk;
    const int j0 = c * kCliqueChunk, n = min(kCliqueChunk, sz - j0);
    const int G = blockDim.x / L;  // pixel groups; thread (g, lab) keeps one label
    const int g = t / L, lab = t - g * L;
    float mx = -INFINITY, mn = INFINITY;
    if (g < G)
        for (int j = g; j < n; j += G) {
            const float q = Q[(long)idx[s0 + j0 + j] * L + lab];
            mx = fmaxf(mx, q);
            mn = fminf(mn, q);
        }
    smx[t] = mx;
    smn[t] = mn;
    __syncthreads();
    if (t < L) {
        for (int gg = 1; gg < G; gg++) {
            mx = fmaxf(mx, smx[gg * L + t]);
            mn = fminf(mn, smn[gg * L + t]);
        }
        part[ubase[r] + t * nch + c] = make_float2(mx, mn);
    }
}

__global__ void clique_maxdiff_finish_kernel(const int* __restrict__ off, const int* __restrict__ ubase, int L,
                                             const float2* __restrict__ part, float* __restrict__ diffs) {
    __shared__ float sd[kLMax];
    const int r = blockIdx.x, t = threadIdx.x;
    const int sz = off[r + 1] - off[r], nch = (sz + kCliqueChunk - 1) / kCliqueChunk;
    if (t < L) {
        float mx = -INFINITY, mn = INFINITY;
        for (int c = 0; c < nch; c++) {
            const float2 v = part[ubase[r] + t * nch + c];
            mx = fmaxf(mx, v.x);
            mn = fminf(mn, v.y);
        }
        sd[t] = fsub(mx, mn);
    }
    __syncthreads();
    if (t == 0) {
        float best = 0.0f;
        for (int lab = 0; lab < L; lab++)
            if (lab == 0 || sd[lab] > best) best = sd[lab];
        diffs[r] = best;
    }
}

__global__ void energy_lp_finish_kernel(int nterms, int R, const float* __restrict__ diffs,
                                        const float* __restrict__ ew, SolverScalars* sc) {
    double e = sc->sums[0];
    for (int k = 0; k < nterms; k++) e -= sc->sums[1 + k];
    for (int r = 0; r < R; r++) e += (double)fmul(ew[r], diffs[r]);
    sc->energy = e;
}

// compute_LR_QP_value(Q, 0): U.Q - 0.Q + sum_k Q.(A_k Q) + Q.(0 o Q).
// compute_LR_QP_value's sum (src/densecrf.cpp:940-957) from sums[0] (U.Q),
// sums[1..nterms] (Q.A_k Q) and, with diag_dom, sums[nterms + 1] (D.Q) and
// sums[nterms + 2] (Q.(D o Q)).
__global__ void lr_finish_kernel(int nterms, SolverScalars* sc, int has_dd) {
    double e = 0.0;
    e += sc->sums[0];
    e -= has_dd ? sc->sums[nterms + 1] : 0.0;
    for (int k = 0; k < nterms; k++) e += sc->sums[1 + k];
    e += has_dd ? sc->sums[nterms + 2] : 0.0;
    sc->energy = e;
}

// sum (double) a o float(b o c) (dotProduct(Q, D.cwiseProduct(Q))).
__global__ void dot3_kernel(long n, const float* __restrict__ a, const float* __restrict__ b,
                            const float* __restrict__ c, double* __restrict__ partials) {
    double v[1] = {0.0};
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
        v[0] += (double)a[t] * (double)fmul(b[t], c[t]);
    block_sum_store<1>(v, partials);
}

// unaryEnergy(l) (src/densecrf.cpp:887-900): r_i = U(l_i, i), 0 off the label range.
__global__ void unary_pick_kernel(int N, int L, const int16_t* __restrict__ lab, const float* __restrict__ U,
                                  float* __restrict__ r) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int l = lab[i];
    r[i] = (0 <= l && l < L) ? U[(long)i * L + l] : 0.0f;
}

}  // namespace
}  // namespace dcrf
