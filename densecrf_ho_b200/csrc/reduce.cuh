// Deterministic reductions and the Eigen 3.2 SSE2 summation order.
#pragma once
#include "model.cuh"

namespace dcrf {

constexpr unsigned kFullMask = 0xffffffffu;

// Block-sum NV doubles and store one partial per block at
// partials[j * gridDim.x + blockIdx.x].  Fixed shuffle tree: deterministic.
template <int NV>
__device__ __forceinline__ void block_sum_store(double (&v)[NV], double* partials) {
    __shared__ double sm[NV][kRedThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; j++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_down_sync(kFullMask, v[j], o);
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < NV; j++) sm[j][w] = v[j];
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        for (int ww = 0; ww < kRedThreads / 32; ww++) s += sm[threadIdx.x][ww];
        partials[(long)threadIdx.x * gridDim.x + blockIdx.x] = s;
    }
}

// Float sum of x[0..N) in the order of Eigen 3.2's LinearVectorizedTraversal
// with Packet4f (Core/Redux.h): two packet accumulators over pairs of aligned
// packets, one trailing packet, predux = (a0+a2)+(a1+a3) (SSE2, no SSE3),
// then the unaligned head [0, AS) and the tail.  AS is the index of the
// first 16-byte aligned element (0 for a VectorXf).  Fully unrolled so x can
// live in registers.
template <int N, int AS>
__device__ __forceinline__ float eig_sum_ct(const float* x) {
    constexpr int as = AS < N ? AS : N;
    constexpr int asz = ((N - as) / 4) * 4, asz2 = ((N - as) / 8) * 8;
    constexpr int end = as + asz, end2 = as + asz2;
    float r;
    if constexpr (asz > 0) {
        float p0[4], p1[4];
#pragma unroll
        for (int l = 0; l < 4; l++) p0[l] = x[as + l];
        if constexpr (asz > 4) {
#pragma unroll
            for (int l = 0; l < 4; l++) p1[l] = x[as + 4 + l];
#pragma unroll
            for (int i = as + 8; i < end2; i += 8)
#pragma unroll
                for (int l = 0; l < 4; l++) {
                    p0[l] = fadd(p0[l], x[i + l]);
                    p1[l] = fadd(p1[l], x[i + 4 + l]);
                }
#pragma unroll
            for (int l = 0; l < 4; l++) p0[l] = fadd(p0[l], p1[l]);
            if constexpr (end > end2)
#pragma unroll
                for (int l = 0; l < 4; l++) p0[l] = fadd(p0[l], x[end2 + l]);
        }
        r = fadd(fadd(p0[0], p0[2]), fadd(p0[1], p0[3]));
#pragma unroll
        for (int i = 0; i < as; i++) r = fadd(r, x[i]);
#pragma unroll
        for (int i = end; i < N; i++) r = fadd(r, x[i]);
    } else {
        r = x[0];
#pragma unroll
        for (int i = 1; i < N; i++) r = fadd(r, x[i]);
    }
    return r;
}

// Same order with run-time n and as (local-memory arrays).
__device__ __forceinline__ float eig_sum_rt(const float* x, int n, int as) {
    if (n <= 0) return 0.0f;
    if (as > n) as = n;
    const int asz = ((n - as) / 4) * 4, asz2 = ((n - as) / 8) * 8;
    const int end = as + asz, end2 = as + asz2;
    float r;
    if (asz) {
        float p0[4], p1[4];
        for (int l = 0; l < 4; l++) p0[l] = x[as + l];
        if (asz > 4) {
            for (int l = 0; l < 4; l++) p1[l] = x[as + 4 + l];
            for (int i = as + 8; i < end2; i += 8)
                for (int l = 0; l < 4; l++) {
                    p0[l] = fadd(p0[l], x[i + l]);
                    p1[l] = fadd(p1[l], x[i + 4 + l]);
                }
            for (int l = 0; l < 4; l++) p0[l] = fadd(p0[l], p1[l]);
            if (end > end2)
                for (int l = 0; l < 4; l++) p0[l] = fadd(p0[l], x[end2 + l]);
        }
        r = fadd(fadd(p0[0], p0[2]), fadd(p0[1], p0[3]));
        for (int i = 0; i < as; i++) r = fadd(r, x[i]);
        for (int i = end; i < n; i++) r = fadd(r, x[i]);
    } else {
        r = x[0];
        for (int i = 1; i < n; i++) r = fadd(r, x[i]);
    }
    return r;
}

// VectorXf sum (aligned start) of a per-thread array of LC (compile-time) or
// n (LC == 0) elements.
template <int LC>
__device__ __forceinline__ float vec_sum(const float* x, int n) {
    if constexpr (LC > 0) return eig_sum_ct<LC, 0>(x);
    else return eig_sum_rt(x, n, 0);
}

// Sum of column `col` of a column-major MatrixXf whose storage is 16-byte
// aligned: the first aligned element is (4 - (col*L) % 4) % 4.
template <int LC>
__device__ __forceinline__ float col_sum(const float* x, int n, long col) {
    const int as = (int)((4 - ((col * (long)n) & 3)) & 3);
    if constexpr (LC > 0) {
        switch (as) {
            case 0: return eig_sum_ct<LC, 0>(x);
            case 1: return eig_sum_ct<LC, 1>(x);
            case 2: return eig_sum_ct<LC, 2>(x);
            default: return eig_sum_ct<LC, 3>(x);
        }
    } else {
        return eig_sum_rt(x, n, as);
    }
}

}  // namespace dcrf
