// QP (Frank-Wolfe, src/densecrf.cpp:340-442) and proximal LP
// (src/densecrf.cpp:444-830) solvers on the device, with the superpixel
// clique terms of qp_sp / lp_sp.
//
// Every per-pixel / per-element update restates the reference's float
// operation order exactly.  Global reductions are deterministic FP64 trees:
//   - the QP line-search dots and the LP dual gap (reference: FP64 Eigen sums);
//   - the LP gamma objective sum (reference: an FP32 Eigen sum) -- summed in
//     FP64 and rounded to float for its stop test;
//   - the QP clique products multiplySuperPixels(p1, p2) -> float
//     (reference: a long sequential FP32 sum) -- evaluated in FP64.
// These can differ from the reference only in their last bits; all other
// clique algebra (prefix chains, running int min/max) is exact.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "model_kernels.cuh"

namespace dcrf {

namespace {

// ------------------------------------------------------------------ QP --

// cond_grad_y = one-hot(first arg-min of grad_y) (src/qp.cpp:5-15);
// sx_y = cond_grad_y - Q; partial sum of unary . sx_y.
template <int LC>
__global__ void qp_direction_kernel(int N, int Lrt, const float* __restrict__ grad, const float* __restrict__ Q,
                                    const float* __restrict__ U, float* __restrict__ sx,
                                    double* __restrict__ partials) {
    const int L = LC ? LC : Lrt;
    double v[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float* g = grad + (long)i * L;
        float best = g[0];
        int bi = 0;
#pragma unroll
        for (int k = 1; k < PixVec<LC>::S; k++)
            if (k < L) {
                float x = g[k];
                if (x < best) {
                    best = x;
                    bi = k;
                }
            }
#pragma unroll
        for (int k = 0; k < PixVec<LC>::S; k++)
            if (k < L) {
                const long e = (long)i * L + k;
                const float s = fsub(k == bi ? 1.0f : 0.0f, Q[e]);
                sx[e] = s;
                v[0] += (double)U[e] * (double)s;
            }
    }
    block_sum_store<1>(v, partials);
}

__global__ void dots2_kernel(long n, const float* __restrict__ a, const float* __restrict__ b,
                             const float* __restrict__ c, double* __restrict__ partials) {
    // partial sums of a.c and b.c
    double v[2] = {0.0, 0.0};
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        const double cc = c[t];
        v[0] += (double)a[t] * cc;
        v[1] += (double)b[t] * cc;
    }
    block_sum_store<2>(v, partials);
}

// Line search (src/densecrf.cpp:412-421).  sums: 0 U.sx, 1 Q.psi, 2 sx.psi,
// 3 a, 4 b, 5 sum(sx_z), 6 clique term of the denominator.
__global__ void qp_step_kernel(SolverScalars* sc) {
    sc->old_energy = sc->energy;
    const double num = sc->sums[0] + 2 * sc->sums[1] + sc->sums[3] + sc->sums[4] + sc->sums[5];
    const double denom = sc->sums[2] + sc->sums[6];
    double step = -num / (2 * denom);
    if (denom == 0 || num == 0) {
        sc->zero_step = 1;
        sc->stop = 1;
        return;
    }
    if (denom < 0) step = 1;
    sc->fstep = (float)step;
    sc->f2step = (float)(2 * step);
    sc->steps++;
}

// Q += step sx_y; grad_y += 2 step psisx + step ho (src/densecrf.cpp:424-431);
// partial sum of Q . (grad_y + unary) (:434).
__global__ void qp_update_kernel(long n, const float* __restrict__ sx, const float* __restrict__ psi,
                                 const float* __restrict__ ho, const float* __restrict__ U, float* __restrict__ Q,
                                 float* __restrict__ grad, const SolverScalars* __restrict__ sc,
                                 double* __restrict__ partials) {
    if (sc->zero_step) return;
    const float fs = sc->fstep, f2s = sc->f2step;
    double v[1] = {0.0};
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        const float q = fadd(Q[t], fmul(fs, sx[t]));
        const float h = ho ? ho[t] : 0.0f;
        const float g = fadd(grad[t], fadd(fmul(f2s, psi[t]), fmul(fs, h)));
        Q[t] = q;
        grad[t] = g;
        v[0] += (double)q * (double)fadd(g, U[t]);
    }
    block_sum_store<1>(v, partials);
}

// energy = sums[7] + (float) clique term sums[8]; stop rule (:390).
__global__ void qp_energy_kernel(SolverScalars* sc, int max_iter) {
    if (sc->zero_step) return;
    const double e = sc->sums[7] + sc->sums[8];
    sc->energy = e;
    if (max_iter > 0) sc->stop = sc->steps >= max_iter;
    else sc->stop = !((sc->old_energy - e) > 100.0);
}

// Loop condition of the QP graph: go on while the stop rule has not fired,
// for at most `cap` iterations per graph launch.
__global__ void qp_cond_kernel(SolverScalars* sc, int cap, cudaGraphConditionalHandle h) {
    const int c = ++sc->chunk;
    cudaGraphSetConditional(h, (!sc->stop && c < cap) ? 1u : 0u);
}

__global__ void qp_init_energy_kernel(SolverScalars* sc, int nterms, int max_iter) {
    // compute_LR_QP_value(Q, 0) + clique term (src/densecrf.cpp:386-387)
    double e = 0.0;
    e += sc->sums[0];
    e -= 0.0;
    for (int k = 0; k < nterms; k++) e += sc->sums[1 + k];
    e += 0.0;
    e += sc->sums[8];
    sc->energy = e;
    sc->old_energy = DBL_MAX;
    sc->zero_step = 0;
    sc->steps = 0;
    // loop entry test of :390 (fixed-iteration mode always enters)
    sc->stop = max_iter > 0 ? 0 : !((DBL_MAX - e) > 100.0);
}

// ------------------------------------------------------ QP clique terms --
// Arrays over (label, clique) are stored [r*L + lab].  The clique list
// buffer holds [R+1 offsets][R cliques by size][their sizes].

struct CliqueView {
    const int* off;
    const int* order;
    const int* sizes;
    const int* idx;
    const float* ew;  // exp_of_superpixels_
    const float* cst; // constants_
    int R, max_size;
    const int* bstart;  // [max_size + 2]: cliques (in size order) of size < s start at bstart[s]
};

// The clique-local prefix chains below walk q = 0 .. max_size-1 with one
// thread per label; the rows p[q][*] they read are staged through shared
// memory kHoChunk at a time by the whole block, the next chunk's copies in
// flight while the current one is summed.
constexpr int kHoChunk = 128;  // rows per staged chunk (two buffers of kHoChunk x L floats, dynamic)
constexpr int kHoThreads = 256;

__device__ __forceinline__ void cp_async4_ca(void* sdst, const void* gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(sdst)),
                 "l"(gsrc)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// The clique-local prefix chains of multiplySuperPixels: pre(lab, s) =
// sum_{q < s} p(lab, q) with p = Q - 1 (or p as given), one sequential chain
// per label in float, as the reference sums it, recorded at every clique
// size: out32[ptr * L + lab] = pre(lab, size of the ptr-th clique in size
// order).  (The FP64 prefixes the clique products use come from
// ho_prefix64's parallel segments.)
// The chain thread only adds and compares: the next record point is the
// size of the next clique in size order, so the loads of the staged rows
// run ahead of the dependent adds.
__global__ void __launch_bounds__(kHoThreads)
    ho_prefix_kernel(CliqueView cv, int L, const float* __restrict__ p, int minus_one, float* __restrict__ out32,
                     const SolverScalars* __restrict__ sc, int skip_on_zero_step) {
    if (sc && skip_on_zero_step && sc->zero_step) return;
    extern __shared__ __align__(16) float ho_rows[];  // [2][kHoChunk][L]
    const int lab = threadIdx.x;
    const bool chain = lab < L;
    int ptr = cv.bstart[1];  // cliques of size 0 come first in size order
    if (chain)
        for (int r = 0; r < ptr; r++) {
            out32[(long)r * L + lab] = 0.0f;
        }
    int next = ptr < cv.R ? cv.sizes[ptr] : INT_MAX;
    const int nchunks = (cv.max_size + kHoChunk - 1) / kHoChunk;
    auto stage = [&](int c) {
        const int q0 = c * kHoChunk, n = min(kHoChunk, cv.max_size - q0) * L;
        float* dst = ho_rows + (size_t)(c & 1) * kHoChunk * L;
        const float* src = p + (long)q0 * L;
        for (int e = threadIdx.x; e < n; e += blockDim.x) cp_async4_ca(dst + e, src + e);
    };
    stage(0);
    cp_async_commit_group();
    float s32 = 0.0f;
    for (int c = 0; c < nchunks; c++) {
        if (c + 1 < nchunks) stage(c + 1);
        cp_async_commit_group();
        cp_async_wait_group<1>();  // chunk c has landed (this thread's copies)
        __syncthreads();           // ... and everyone's
        if (chain) {
            const float* r = ho_rows + (size_t)(c & 1) * kHoChunk * L + lab;
            const int q0 = c * kHoChunk, nq = min(kHoChunk, cv.max_size - q0);
            // one element: add, then record at every clique whose size is
            // the prefix length reached
            auto step = [&](float x, int len) {
                if (minus_one) x = fsub(x, 1.0f);
                s32 = fadd(s32, x);
                while (len == next) {
                    out32[(long)ptr * L + lab] = s32;
                    ptr++;
                    next = ptr < cv.R ? cv.sizes[ptr] : INT_MAX;
                }
            };
            int qq = 0;
            if (nq == kHoChunk && q0 + kHoChunk < next) {
                // a whole chunk before the next record: all its loads first,
                // then one straight chain of adds
                float x[kHoChunk];
#pragma unroll
                for (int i = 0; i < kHoChunk; i++) x[i] = r[i * L];
#pragma unroll
                for (int i = 0; i < kHoChunk; i++) {
                    float xi = x[i];
                    if (minus_one) xi = fsub(xi, 1.0f);
                    s32 = fadd(s32, xi);
                }
                qq = kHoChunk;
            }
            // batches of eight: the eight loads first, then the chain; no
            // record check inside a batch that ends before the next record
            for (; qq + 8 <= nq; qq += 8) {
                float x[8];
#pragma unroll
                for (int i = 0; i < 8; i++) x[i] = r[(qq + i) * L];
                if (q0 + qq + 8 < next) {
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        float xi = x[i];
                        if (minus_one) xi = fsub(xi, 1.0f);
                        s32 = fadd(s32, xi);
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 8; i++) step(x[i], q0 + qq + i + 1);
                }
            }
            for (; qq < nq; qq++) step(r[qq * L], q0 + qq + 1);
        }
        __syncthreads();  // rows[c & 1] is restaged for chunk c + 2
    }
    cp_async_wait_group<0>();
}

// The FP64 prefix chains in segments of kHoSeg rows, so that they run in
// parallel instead of one thread per label over every row.  The FP64 chains
// are this engine's own choice (the reference sums in float; see
// ho_scalar_kernel), so their order is free: segment 0 is summed from 0.0
// exactly as the sequential chain (every clique of at most kHoSeg pixels gets
// the sequential chain's value), a later segment starts from the sum of the
// segments before it.  ho_seg_total_kernel: per (segment, label) the FP64
// sum of the segment's rows; ho_seg_prefix_kernel: per (segment, label) the
// carry-in from the totals, then the segment's prefix with the records of
// the cliques whose size ends in it.
constexpr int kHoSeg = 256;

__global__ void ho_seg_total_kernel(CliqueView cv, int L, const float* __restrict__ p, int minus_one,
                                    double* __restrict__ tot, const SolverScalars* __restrict__ sc, int skip_on_zero_step) {
    if (sc && skip_on_zero_step && sc->zero_step) return;
    const int seg = blockIdx.x, lab = threadIdx.x;
    if (lab >= L) return;
    const int q0 = seg * kHoSeg, q1 = min(cv.max_size, q0 + kHoSeg);
    double s = 0.0;
    int q = q0;
    for (; q + 8 <= q1; q += 8) {
        float x[8];
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = p[(long)(q + i) * L + lab];
#pragma unroll
        for (int i = 0; i < 8; i++) s += (double)(minus_one ? fsub(x[i], 1.0f) : x[i]);
    }
    for (; q < q1; q++) {
        const float x = p[(long)q * L + lab];
        s += (double)(minus_one ? fsub(x, 1.0f) : x);
    }
    tot[(long)seg * L + lab] = s;
}

__global__ void ho_seg_prefix_kernel(CliqueView cv, int L, const float* __restrict__ p, int minus_one,
                                     const double* __restrict__ tot, double* __restrict__ out64,
                                     const SolverScalars* __restrict__ sc, int skip_on_zero_step) {
    if (sc && skip_on_zero_step && sc->zero_step) return;
    const int seg = blockIdx.x, lab = threadIdx.x;
    if (lab >= L) return;
    const int q0 = seg * kHoSeg, q1 = min(cv.max_size, q0 + kHoSeg);
    if (seg == 0)
        for (int r = 0; r < cv.bstart[1]; r++) out64[(long)r * L + lab] = 0.0;  // empty cliques
    double s = 0.0;
    for (int g = 0; g < seg; g++) s += tot[(long)g * L + lab];
    int ptr = cv.bstart[q0 + 1];  // the first clique of size > q0
    int next = ptr < cv.R ? cv.sizes[ptr] : INT_MAX;
    auto step = [&](float x, int len) {
        s += (double)(minus_one ? fsub(x, 1.0f) : x);
        while (len == next) {
            out64[(long)ptr * L + lab] = s;
            ptr++;
            next = ptr < cv.R ? cv.sizes[ptr] : INT_MAX;
        }
    };
    int q = q0;
    for (; q + 8 <= q1; q += 8) {  // eight loads ahead of the eight dependent adds
        float x[8];
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = p[(long)(q + i) * L + lab];
#pragma unroll
        for (int i = 0; i < 8; i++) step(x[i], q + i + 1);
    }
    for (; q < q1; q++) step(p[(long)q * L + lab], q + 1);
}

// The float clique prefix chain of p (minus one when asked) into out32.
static void ho_prefix32(cudaStream_t stream, int L, const CliqueView& cv, const float* p, int minus_one, float* out32,
                        const SolverScalars* sc, int skip_on_zero_step) {
    static const bool attr = [] {  // two 128-row buffers: up to 64 KB for L = 64
        DCRF_CUDA(cudaFuncSetAttribute(ho_prefix_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(sizeof(float) * 2 * kHoChunk * kLMax)));
        return true;
    }();
    (void)attr;
    launch(ho_prefix_kernel, 1, kHoThreads, sizeof(float) * 2 * kHoChunk * L, stream, cv, L, p, minus_one, out32, sc,
           skip_on_zero_step);
}

// FP64 clique prefixes of p (minus one when asked) into out64 [R][L]:
// segment totals, then the segments' prefixes with their carries.
static void ho_prefix64(cudaStream_t stream, DevBuf<double>& seg_buf, int clique_max, int L, const CliqueView& cv,
                        const float* p, int minus_one, double* out64, const SolverScalars* sc, int skip_on_zero_step) {
    const int nseg = (clique_max + kHoSeg - 1) / kHoSeg;
    if (nseg == 0) {  // only empty cliques: their zeros
        launch(ho_seg_prefix_kernel, 1, 64, 0, stream, cv, L, p, minus_one, (const double*)nullptr, out64, sc,
               skip_on_zero_step);
        return;
    }
    double* tot = seg_buf.ensure((size_t)nseg * L);
    launch(ho_seg_total_kernel, nseg, 64, 0, stream, cv, L, p, minus_one, tot, sc, skip_on_zero_step);
    launch(ho_seg_prefix_kernel, nseg, 64, 0, stream, cv, L, p, minus_one, (const double*)tot, out64, sc,
           skip_on_zero_step);
}

// multiplySuperPixels(p [L x N]) with p = Q - 1 (src/densecrf.cpp:81-88): the
// reference sums p(lab, 0..size_r-1) -- the clique-LOCAL index -- so every
// clique's value is a prefix of one chain per label (ho_prefix_kernel).  Then
//   mode 0: grad_z = (1 + res) o c           (:373-374)
//   mode 1: grad_z = 1 o c + res o c         (:432)
__global__ void ho_regions_kernel(CliqueView cv, int L, const float* __restrict__ pre, float* __restrict__ gz,
                                  int mode, const SolverScalars* __restrict__ sc) {
    if (sc && sc->zero_step) return;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)cv.R * L) return;
    const int ptr = (int)(t / L), lab = (int)(t - (long)ptr * L);
    const int r = cv.order[ptr];
    const float c = cv.ew[r], val = pre[t];
    gz[(long)r * L + lab] = mode == 0 ? fmul(fadd(1.0f, val), c) : fadd(fmul(1.0f, c), fmul(val, c));
}

// Small (label, clique) algebra of one Frank-Wolfe iteration.  One thread
// per element, then thread 0 sums sx_z in Eigen order.
//   cz = [gz < 0] (src/qp.cpp:17-25); sxz = cz - z; t1 = sxz o c;
//   t2 = (cz - 1) o c.
__global__ void ho_direction_kernel(CliqueView cv, int L, const float* __restrict__ gz, const float* __restrict__ z,
                                    float* __restrict__ sxz, float* __restrict__ t1, float* __restrict__ t2,
                                    float* __restrict__ cz, SolverScalars* sc) {
    const int n = L * cv.R;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const float c = cv.ew[e / L];
        const float czv = gz[e] >= 0.0f ? 0.0f : 1.0f;
        const float sv = fsub(czv, z[e]);
        cz[e] = czv;
        sxz[e] = sv;
        t1[e] = fmul(sv, c);
        t2[e] = fmul(fsub(czv, 1.0f), c);
    }
}

// float multiplySuperPixels(p1 [L x R], p2 [L x N]) (src/densecrf.cpp:58-72):
// sum_r sum_{q < size_r} sum_lab p1(lab, r) p2(lab, q), clique-local q again.
// Evaluated in FP64 as sum_lab sum_r p1(lab, r) * prefix_lab(size_r), the r
// in size order, then rounded to float; the FP64 prefixes come from
// ho_prefix64.  One thread per label; its loads do not depend on
// its sum, so they run ahead of it.
__global__ void ho_scalar_kernel(CliqueView cv, int L, const float* __restrict__ p1, const double* __restrict__ pre,
                                 int slot, SolverScalars* sc, int add_to_slot) {
    if (sc->zero_step && slot != 8) return;
    __shared__ double part[kLMax];
    const int lab = threadIdx.x;
    double acc = 0.0;
    if (lab < L) {
#pragma unroll 4
        for (int ptr = cv.bstart[1]; ptr < cv.R; ptr++)
            acc += (double)p1[(long)cv.order[ptr] * L + lab] * pre[(long)ptr * L + lab];
    }
    if (threadIdx.x < kLMax) part[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < L; k++) t += part[k];
        const float f = (float)t;
        if (add_to_slot) sc->sums[slot] = (double)fadd((float)sc->sums[slot], f);
        else sc->sums[slot] = (double)f;
    }
}

// multiplySuperPixels(p [L x R]) -> [L x N] (src/densecrf.cpp:90-97):
// out(lab, q) = sum over cliques r (in order) with size_r > q of p(lab, r).
// p = (z - 1) o c is formed on the fly.  Rows q >= max_size stay zero.
__global__ void ho_pixels_kernel(CliqueView cv, int L, const float* __restrict__ z, float* __restrict__ out,
                                 const SolverScalars* __restrict__ sc) {
    if (sc && sc->zero_step) return;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)cv.max_size * L) return;
    const int q = (int)(t / L), lab = (int)(t - (long)q * L);
    float s = 0.0f;
    for (int r = 0; r < cv.R; r++)
        if (cv.off[r + 1] - cv.off[r] > q) s = fadd(s, fmul(fsub(z[(long)r * L + lab], 1.0f), cv.ew[r]));
    out[t] = s;
}

// z += step sx_z (src/densecrf.cpp:425).
__global__ void ho_z_update_kernel(int n, float* __restrict__ z, const float* __restrict__ sxz,
                                   const SolverScalars* __restrict__ sc) {
    if (sc->zero_step) return;
    for (int e = threadIdx.x; e < n; e += blockDim.x) z[e] = fadd(z[e], fmul(sc->fstep, sxz[e]));
}

// z o c sum (Eigen order) and (1 - z) o c, for the energy's clique term.
__global__ void ho_zterm_prep_kernel(CliqueView cv, int L, const float* __restrict__ z, float* __restrict__ zc,
                                     float* __restrict__ omz, SolverScalars* sc) {
    if (sc->zero_step && sc->steps > 0) return;
    const int n = L * cv.R;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const float c = cv.ew[e / L];
        zc[e] = fmul(z[e], c);
        omz[e] = fmul(fsub(1.0f, z[e]), c);
    }
}

// sc->sums[slot] = VectorXf sum of x[0..n) in Eigen's order (eig_sum_rt with
// an aligned start): the eight packet lanes are eight independent chains,
// run here by eight threads over shared-memory chunks of the vector, and
// combined in the reference's order.  skip: the QP step's zero_step rule of
// the kernel that produced x.
__global__ void __launch_bounds__(kHoThreads)
    eig_sum_kernel(const float* __restrict__ x, int n, int slot, SolverScalars* sc, int skip) {
    if ((skip == 1 && sc->zero_step) || (skip == 2 && sc->zero_step && sc->steps > 0)) return;
    constexpr int kC = 2048;  // chunk, a multiple of 8
    __shared__ float buf[kC];
    __shared__ float lanes[8];
    const int asz = (n / 4) * 4, asz2 = (n / 8) * 8;
    if (asz <= 4) {  // no paired-packet loop: the sequential routine
        if (threadIdx.x == 0) sc->sums[slot] = (double)eig_sum_rt(x, n, 0);
        return;
    }
    const int l = threadIdx.x;
    float acc = 0.0f;
    for (int c0 = 0; c0 < asz2; c0 += kC) {
        const int m = min(kC, asz2 - c0);
        __syncthreads();
        for (int e = threadIdx.x; e < m; e += blockDim.x) buf[e] = x[c0 + e];
        __syncthreads();
        if (l < 8) {
            int i = l;
            if (c0 == 0) {
                acc = buf[l];  // p0 = x[0..3], p1 = x[4..7]
                i += 8;
            }
            for (; i < m; i += 8) acc = fadd(acc, buf[i]);
        }
    }
    if (l < 8) lanes[l] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float p0[4];
        for (int k = 0; k < 4; k++) p0[k] = fadd(lanes[k], lanes[4 + k]);
        if (asz > asz2)
            for (int k = 0; k < 4; k++) p0[k] = fadd(p0[k], x[asz2 + k]);
        float r = fadd(fadd(p0[0], p0[2]), fadd(p0[1], p0[3]));
        for (int i = asz; i < n; i++) r = fadd(r, x[i]);
        sc->sums[slot] = (double)r;
    }
}

__global__ void fill_float_kernel(long n, float v, float* x) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) x[t] = v;
}

__global__ void add_inplace_kernel(long n, float* __restrict__ a, const float* __restrict__ b) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) a[t] = fadd(a[t], b[t]);
}

// a += coef * b  (grad_y += 2 * tmp, src/densecrf.cpp:380)
__global__ void add_scaled_kernel(long n, float* __restrict__ a, const float* __restrict__ b, float coef) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) a[t] = fadd(a[t], fmul(coef, b[t]));
}

// ------------------------------------------------------------------ LP --

// Y = multiplyC((alpha + u) - unary) + cur_Q (src/densecrf.cpp:627-635, 517-523).
// With `pending`, the previous Frank-Wolfe iteration's update
// alpha += delta (sa - alpha), u += delta (su - u) (:737-738) is applied here
// first (and stored), saving a pass; su == nullptr means no cliques (su = 0).
template <int LC>
__global__ void lp_y_kernel(int N, int Lrt, float lambda, float cm, float* __restrict__ alpha,
                            float* __restrict__ u, const float* __restrict__ U,
                            const float* __restrict__ curQ, float* __restrict__ Y, bool pending,
                            const float* __restrict__ sa, const float* __restrict__ su,
                            const SolverScalars* __restrict__ sc) {
    const int L = LC ? LC : Lrt;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float x[PixVec<LC>::S];
    const float dl = pending ? sc->delta : 0.0f;
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) {
            const long e = (long)i * L + k;
            float a = alpha[e], uu = u[e];
            if (pending) {
                a = fadd(a, fmul(dl, fsub(sa[e], a)));
                uu = fadd(uu, fmul(dl, fsub(su ? su[e] : 0.0f, uu)));
                alpha[e] = a;
                u[e] = uu;
            }
            x[k] = fsub(fadd(a, uu), U[e]);
        }
    const float s = vec_sum<LC>(x, L);
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) {
            const long e = (long)i * L + k;
            Y[e] = fadd(fmul(fadd(fmul(cm, s), x[k]), lambda), curQ[e]);
        }
}

struct GammaConsts {
    float lambda, delta, c0, c1, c2, cm;
};

// One qp-gamma iteration for every pixel (qp_gamma_step, :495-514, and the
// objective of :665-667); partial sums of the per-pixel objective.
template <int LC>
__global__ void lp_gamma_kernel(int N, int Lrt, GammaConsts gc, const float* __restrict__ Y, float* __restrict__ gamma,
                                const SolverScalars* __restrict__ sc, double* __restrict__ partials) {
    if (sc->stop) return;
    const int L = LC ? LC : Lrt;
    double v[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        float g[PixVec<LC>::S], y[PixVec<LC>::S], t[PixVec<LC>::S];
#pragma unroll
        for (int k = 0; k < PixVec<LC>::S; k++)
            if (k < L) {
                g[k] = gamma[(long)i * L + k];
                y[k] = Y[(long)i * L + k];
            }
        const float s = vec_sum<LC>(g, L);
#pragma unroll
        for (int k = 0; k < PixVec<LC>::S; k++)
            if (k < L) {
                const float ph = (-y[k] < 0.0f) ? 0.0f : -y[k];  // std::max(-Y, 0)
                const float nh = (y[k] < 0.0f) ? 0.0f : y[k];    // std::max(Y, 0)
                float st = fadd(fmul(fsub(s, g[k]), gc.c0), ph);
                st = fadd(st, gc.delta);
                float tt = fmul(fadd(fmul(gc.c1, s), fmul(gc.c2, g[k])), gc.lambda);
                tt = fadd(tt, nh);
                tt = fadd(tt, gc.delta);
                g[k] = fmul(g[k], st / tt);
                gamma[(long)i * L + k] = g[k];
            }
        const float s2 = vec_sum<LC>(g, L);
#pragma unroll
        for (int k = 0; k < PixVec<LC>::S; k++)
            if (k < L) t[k] = fmul(g[k], fmul(fadd(fmul(gc.cm, s2), g[k]), gc.lambda));
        const float d1 = vec_sum<LC>(t, L);
#pragma unroll
        for (int k = 0; k < PixVec<LC>::S; k++)
            if (k < L) t[k] = fmul(g[k], y[k]);
        const float d2 = vec_sum<LC>(t, L);
        const float qv = (float)dadd(dmul(0.5, (double)d1), (double)d2);
        v[0] += (double)qv;
    }
    block_sum_store<1>(v, partials);
}

// |qp_value - qp_value1| < qp_tol test (:670-674).
// Launched with one block of any multiple of 32 threads.
__global__ void lp_gamma_check_kernel(const double* __restrict__ partials, int nblk, float qp_tol,
                                      SolverScalars* sc) {
    if (sc->stop) return;
    __shared__ double s32[32];
    double s = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += partials[b];
    s = block_sum_any(s, s32);
    if (threadIdx.x == 0) {
        const float qv1 = (float)s;
        sc->steps++;
        sc->gamma_sum++;
        if (fabsf(fsub(sc->qp_value, qv1)) < qp_tol) sc->stop = 1;
        else sc->qp_value = qv1;
    }
}

// The same test as the exit condition of a graph's `while` node: the loop
// goes on while the iterate has not converged and fewer than max_iter
// iterations have run (the body always runs at least once).
__global__ void lp_gamma_check_cond_kernel(const double* __restrict__ partials, int nblk, float qp_tol,
                                           SolverScalars* sc, int max_iter, cudaGraphConditionalHandle h) {
    __shared__ double s32[32];
    double s = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += partials[b];
    s = block_sum_any(s, s32);
    if (threadIdx.x == 0) {
        if (!sc->stop) {
            const float qv1 = (float)s;
            sc->steps++;
            sc->gamma_sum++;
            if (fabsf(fsub(sc->qp_value, qv1)) < qp_tol) sc->stop = 1;
            else sc->qp_value = qv1;
        }
        cudaGraphSetConditional(h, (!sc->stop && sc->steps < max_iter) ? 1u : 0u);
    }
}

__global__ void lp_gamma_reset_kernel(SolverScalars* sc) {
    sc->stop = 0;
    sc->steps = 0;
    sc->qp_value = FLT_MAX;
}

// beta = -colsum(alpha + u + gamma - unary) / L (:684-691);
// Q = lambda (alpha + beta + u + gamma - unary) + cur_Q (:697).
// Also writes per-block min / max of Q (the first half of rescale) to
// partials[b] and partials[gridDim.x + b].
template <int LC>
__global__ void lp_q_kernel(int N, int Lrt, float lambda, const float* __restrict__ alpha, const float* __restrict__ u,
                            const float* __restrict__ gamma, const float* __restrict__ U,
                            const float* __restrict__ curQ, float* __restrict__ Q, double* __restrict__ partials) {
    const int L = LC ? LC : Lrt;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float mn = INFINITY, mx = -INFINITY;
    if (i < N) {
        float bm[PixVec<LC>::S];
#pragma unroll
        for (int k = 0; k < PixVec<LC>::S; k++)
            if (k < L) {
                const long e = (long)i * L + k;
                bm[k] = fsub(fadd(fadd(alpha[e], u[e]), gamma[e]), U[e]);
            }
        const float beta = (-col_sum<LC>(bm, L, i)) / (float)L;
#pragma unroll
        for (int k = 0; k < PixVec<LC>::S; k++)
            if (k < L) {
                const long e = (long)i * L + k;
                const float x = fsub(fadd(fadd(fadd(alpha[e], beta), u[e]), gamma[e]), U[e]);
                const float q = fadd(fmul(x, lambda), curQ[e]);
                Q[e] = q;
                mn = nan_min(mn, q);
                mx = nan_max(mx, q);
            }
    }
    __shared__ float smn[32], smx[32];
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
        partials[blockIdx.x] = mn;
        partials[gridDim.x + blockIdx.x] = mx;
    }
}

// --------------------------------------------- row-tiled variants (L = LC) --
// Same arithmetic as lp_y_kernel / lp_q_kernel / lp_gamma_kernel /
// qp_direction_kernel, one warp per 32 pixels, rows staged in shared memory.

template <int LC>
__global__ void __launch_bounds__(32 * kTileWarps)
    lp_y_tiled(int N, float lambda, float cm, float* __restrict__ alpha, float* __restrict__ u,
               const float* __restrict__ U, const float* __restrict__ curQ, float* __restrict__ Y, bool pending,
               const float* __restrict__ sa, const float* __restrict__ su, const SolverScalars* __restrict__ sc) {
    __shared__ float sm[kTileWarps][2][32 * LC];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long pix0 = ((long)blockIdx.x * kTileWarps + wib) * 32;
    if (pix0 >= N) return;
    const int npix = (int)min(32L, (long)N - pix0);
    float* A = sm[wib][0];
    float* B = sm[wib][1];
    float* ra = A + lane * LC;
    float* rb = B + lane * LC;
    const float dl = pending ? sc->delta : 0.0f;
    float x[LC];
    // alpha (+ pending update)
    tile_in<LC>(A, alpha, pix0, npix, lane);
    if (pending) tile_in<LC>(B, sa, pix0, npix, lane);
    __syncwarp();
#pragma unroll
    for (int k = 0; k < LC; k++) {
        float a = ra[k];
        if (pending) {
            a = fadd(a, fmul(dl, fsub(rb[k], a)));
            ra[k] = a;
        }
        x[k] = a;
    }
    __syncwarp();
    if (pending) tile_out<LC>(A, alpha, pix0, npix, lane);
    __syncwarp();
    // u (+ pending update)
    tile_in<LC>(A, u, pix0, npix, lane);
    if (pending && su) tile_in<LC>(B, su, pix0, npix, lane);
    __syncwarp();
#pragma unroll
    for (int k = 0; k < LC; k++) {
        float uu = ra[k];
        if (pending) {
            uu = fadd(uu, fmul(dl, fsub(su ? rb[k] : 0.0f, uu)));
            ra[k] = uu;
        }
        x[k] = fadd(x[k], uu);
    }
    __syncwarp();
    if (pending) tile_out<LC>(A, u, pix0, npix, lane);
    __syncwarp();
    // x = (alpha + u) - unary;  Y = multiplyC(x) + cur_Q
    tile_in<LC>(A, U, pix0, npix, lane);
    tile_in<LC>(B, curQ, pix0, npix, lane);
    __syncwarp();
#pragma unroll
    for (int k = 0; k < LC; k++) x[k] = fsub(x[k], ra[k]);
    const float s = eig_sum_ct<LC, 0>(x);
#pragma unroll
    for (int k = 0; k < LC; k++) rb[k] = fadd(fmul(fadd(fmul(cm, s), x[k]), lambda), rb[k]);
    __syncwarp();
    tile_out<LC>(B, Y, pix0, npix, lane);
}

template <int LC>
__global__ void __launch_bounds__(32 * kTileWarps)
    lp_q_tiled(int N, float lambda, const float* __restrict__ alpha, const float* __restrict__ u,
               const float* __restrict__ gamma, const float* __restrict__ U, const float* __restrict__ curQ,
               float* __restrict__ Q, double* __restrict__ partials) {
    __shared__ float sm[kTileWarps][4][32 * LC];
    __shared__ float smn[kTileWarps], smx[kTileWarps];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long pix0 = ((long)blockIdx.x * kTileWarps + wib) * 32;
    float mn = INFINITY, mx = -INFINITY;
    if (pix0 < N) {
        const int npix = (int)min(32L, (long)N - pix0);
        float* T[4] = {sm[wib][0], sm[wib][1], sm[wib][2], sm[wib][3]};
        tile_in<LC>(T[0], alpha, pix0, npix, lane);
        tile_in<LC>(T[1], u, pix0, npix, lane);
        tile_in<LC>(T[2], gamma, pix0, npix, lane);
        tile_in<LC>(T[3], U, pix0, npix, lane);
        __syncwarp();
        const float *ra = T[0] + lane * LC, *ru = T[1] + lane * LC, *rg = T[2] + lane * LC, *rU = T[3] + lane * LC;
        float t[LC];
#pragma unroll
        for (int k = 0; k < LC; k++) t[k] = fsub(fadd(fadd(ra[k], ru[k]), rg[k]), rU[k]);
        const float beta = (-col_sum<LC>(t, LC, pix0 + lane)) / (float)LC;
#pragma unroll
        for (int k = 0; k < LC; k++) t[k] = fsub(fadd(fadd(fadd(ra[k], beta), ru[k]), rg[k]), rU[k]);
        __syncwarp();
        tile_in<LC>(T[0], curQ, pix0, npix, lane);
        __syncwarp();
        float* rq = T[0] + lane * LC;
        const bool act = lane < npix;
#pragma unroll
        for (int k = 0; k < LC; k++) {
            const float q = fadd(fmul(t[k], lambda), rq[k]);
            rq[k] = q;
            if (act) {
                mn = nan_min(mn, q);
                mx = nan_max(mx, q);
            }
        }
        __syncwarp();
        tile_out<LC>(T[0], Q, pix0, npix, lane);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = nan_min(mn, __shfl_down_sync(kFullMask, mn, o));
        mx = nan_max(mx, __shfl_down_sync(kFullMask, mx, o));
    }
    if (lane == 0) {
        smn[wib] = mn;
        smx[wib] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kTileWarps; w++) {
            mn = nan_min(mn, smn[w]);
            mx = nan_max(mx, smx[w]);
        }
        partials[blockIdx.x] = mn;
        partials[gridDim.x + blockIdx.x] = mx;
    }
}

template <int LC>
__global__ void __launch_bounds__(32 * kTileWarps)
    lp_gamma_tiled(int N, GammaConsts gc, const float* __restrict__ Y, float* __restrict__ gamma,
                   const SolverScalars* __restrict__ sc, double* __restrict__ partials) {
    if (sc->stop) return;  // uniform across the grid
    __shared__ float sm[kTileWarps][2][32 * LC];
    __shared__ double s32[32];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long pix0 = ((long)blockIdx.x * kTileWarps + wib) * 32;
    double acc = 0.0;
    if (pix0 < N) {
        const int npix = (int)min(32L, (long)N - pix0);
        float* G = sm[wib][0];
        float* Yt = sm[wib][1];
        tile_in<LC>(G, gamma, pix0, npix, lane);
        tile_in<LC>(Yt, Y, pix0, npix, lane);
        __syncwarp();
        float* rg = G + lane * LC;
        const float* ry = Yt + lane * LC;
        float g[LC], t[LC];
#pragma unroll
        for (int k = 0; k < LC; k++) g[k] = rg[k];
        const float s = eig_sum_ct<LC, 0>(g);
#pragma unroll
        for (int k = 0; k < LC; k++) {
            const float y = ry[k];
            const float ph = (-y < 0.0f) ? 0.0f : -y;  // std::max(-Y, 0)
            const float nh = (y < 0.0f) ? 0.0f : y;    // std::max(Y, 0)
            float st = fadd(fmul(fsub(s, g[k]), gc.c0), ph);
            st = fadd(st, gc.delta);
            float tt = fmul(fadd(fmul(gc.c1, s), fmul(gc.c2, g[k])), gc.lambda);
            tt = fadd(tt, nh);
            tt = fadd(tt, gc.delta);
            g[k] = fmul(g[k], st / tt);
            rg[k] = g[k];
        }
        const float s2 = eig_sum_ct<LC, 0>(g);
#pragma unroll
        for (int k = 0; k < LC; k++) t[k] = fmul(g[k], fmul(fadd(fmul(gc.cm, s2), g[k]), gc.lambda));
        const float d1 = eig_sum_ct<LC, 0>(t);
#pragma unroll
        for (int k = 0; k < LC; k++) t[k] = fmul(g[k], ry[k]);
        const float d2 = eig_sum_ct<LC, 0>(t);
        if (lane < npix) acc = (double)(float)dadd(dmul(0.5, (double)d1), (double)d2);
        __syncwarp();
        tile_out<LC>(G, gamma, pix0, npix, lane);
    }
    const double tot = block_sum_any(acc, s32);
    if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

template <int LC>
__global__ void __launch_bounds__(32 * kTileWarps)
    qp_direction_tiled(int N, const float* __restrict__ grad, const float* __restrict__ Q,
                       const float* __restrict__ U, float* __restrict__ sx, double* __restrict__ partials) {
    __shared__ float sm[kTileWarps][3][32 * LC];
    __shared__ double s32[32];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long pix0 = ((long)blockIdx.x * kTileWarps + wib) * 32;
    double acc = 0.0;
    if (pix0 < N) {
        const int npix = (int)min(32L, (long)N - pix0);
        float *Gt = sm[wib][0], *Qt = sm[wib][1], *Ut = sm[wib][2];
        tile_in<LC>(Gt, grad, pix0, npix, lane);
        tile_in<LC>(Qt, Q, pix0, npix, lane);
        tile_in<LC>(Ut, U, pix0, npix, lane);
        __syncwarp();
        const float* rg = Gt + lane * LC;
        float* rq = Qt + lane * LC;
        const float* ru = Ut + lane * LC;
        float best = rg[0];
        int bi = 0;
#pragma unroll
        for (int k = 1; k < LC; k++)
            if (rg[k] < best) {
                best = rg[k];
                bi = k;
            }
        const bool act = lane < npix;
#pragma unroll
        for (int k = 0; k < LC; k++) {
            const float s = fsub(k == bi ? 1.0f : 0.0f, rq[k]);
            rq[k] = s;
            if (act) acc += (double)ru[k] * (double)s;
        }
        __syncwarp();
        tile_out<LC>(Qt, sx, pix0, npix, lane);
    }
    const double tot = block_sum_any(acc, s32);
    if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

// Partial sums of tmp.Q and tmp.tmp, tmp = (alpha + u) - (sa + su) (:725-729).
__global__ void lp_gap_kernel(long n, const float* __restrict__ alpha, const float* __restrict__ u,
                              const float* __restrict__ sa, const float* __restrict__ su,
                              const float* __restrict__ Q, double* __restrict__ partials) {
    double v[2] = {0.0, 0.0};
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        const float tmp = fsub(fadd(alpha[t], u[t]), fadd(sa[t], su ? su[t] : 0.0f));
        v[0] += (double)tmp * (double)Q[t];
        v[1] += (double)tmp * (double)tmp;
    }
    block_sum_store<2>(v, partials);
}

__global__ void lp_delta_kernel(SolverScalars* sc, float lambda) {
    float delta = (float)(sc->sums[0] / ((double)lambda * sc->sums[1]));
    delta = (delta < 0.0f) ? 0.0f : delta;  // std::max(delta, 0)
    delta = (1.0f < delta) ? 1.0f : delta;  // std::min(delta, 1)
    sc->delta = delta;
}

template <int LC>
__device__ __forceinline__ void sort_desc(float* s, int L) {
    // insertion sort (values only: ties cannot change feasible_Q's result)
#pragma unroll
    for (int a = 1; a < PixVec<LC>::S; a++)
        if (a < L) {
            const float x = s[a];
            int b = a - 1;
            while (b >= 0 && s[b] < x) {
                s[b + 1] = s[b];
                b--;
            }
            s[b + 1] = x;
        }
}

// renormalize (src/densecrf.cpp:444-455) of one pixel held in registers.
template <int LC>
__device__ __forceinline__ void renorm_pixel(float* t, int L, long i) {
    const double s = (double)col_sum<LC>(t, L, i);
    if (s == 0 || s != s) {
        const float uni = (float)(1.0 / L);
#pragma unroll
        for (int k = 0; k < PixVec<LC>::S; k++)
            if (k < L) t[k] = uni;
    } else {
        const float fs = (float)s;
#pragma unroll
        for (int k = 0; k < PixVec<LC>::S; k++)
            if (k < L) t[k] = t[k] / fs;
    }
}

// feasible_Q (:470-492) + renormalize + currentMap, one thread per pixel.
template <int LC>
__global__ void lp_project_kernel(int N, int Lrt, float* __restrict__ Q, int16_t* __restrict__ lab) {
    const int L = LC ? LC : Lrt;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float q[PixVec<LC>::S], s[PixVec<LC>::S];
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) q[k] = s[k] = Q[(long)i * L + k];
    sort_desc<LC>(s, L);
    double sum = (double)fsub(col_sum<LC>(q, L, i), 1.0f);
    int K = -1;
    for (int k = L; k > 0; --k) {
        const double uk = (double)s[k - 1];
        if (sum / k < uk) {
            K = k;
            break;
        }
        sum -= uk;
    }
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) {
            double v = (double)q[k] - sum / K;
            v = (v < 0.0) ? 0.0 : v;
            v = (1.0 < v) ? 1.0 : v;
            q[k] = (float)v;
        }
    renorm_pixel<LC>(q, L, i);
    float best = q[0];
    int bi = 0;
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) {
            Q[(long)i * L + k] = q[k];
            if (k > 0 && q[k] > best) {
                best = q[k];
                bi = k;
            }
        }
    if (lab) lab[i] = (int16_t)bi;
}

template <int LC>
__global__ void renormalize_kernel(int N, int Lrt, float* __restrict__ Q) {
    const int L = LC ? LC : Lrt;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float q[PixVec<LC>::S];
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) q[k] = Q[(long)i * L + k];
    renorm_pixel<LC>(q, L, i);
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) Q[(long)i * L + k] = q[k];
}

// max_rounding (:832-840).
template <int LC>
__global__ void max_rounding_kernel(int N, int Lrt, float* __restrict__ Q) {
    const int L = LC ? LC : Lrt;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float best = Q[(long)i * L];
    int bi = 0;
    for (int k = 1; k < L; k++)
        if (Q[(long)i * L + k] > best) {
            best = Q[(long)i * L + k];
            bi = k;
        }
    for (int k = 0; k < L; k++) Q[(long)i * L + k] = k == bi ? 1.0f : 0.0f;
}

// less_confident_pixels count (:458-464).
__global__ void less_confident_kernel(int N, int L, const float* __restrict__ Q, float tol, double* partials) {
    double v[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        float mx = Q[(long)i * L];
        for (int k = 1; k < L; k++) mx = fmaxf(mx, Q[(long)i * L + k]);
        if (mx <= tol) v[0] += 1.0;
    }
    block_sum_store<1>(v, partials);
}

// --------------------------------------------------------- LP cliques --

// float -> int as x86 cvttss2si (C++ truncation; NaN / out of range -> INT_MIN).
__device__ __forceinline__ int trunc_x86(float q) {
    return fabsf(q) < 2147483648.0f ? (int)q : INT_MIN;
}

// computeUCondGrad (src/densecrf.cpp:803-830): the positions it selects.
// The reference keeps its running min / max in an int, so position p (in
// label-major, clique order: p = lab * size + j) updates the min iff
// Q_p < (float)s, where s is the running min of trunc(Q) over the positions
// before p (it starts at INT_MAX); the LAST such p is selected.  Same for the
// max.  A min / max over the positions before p does not depend on their
// order, so the scan splits into units (clique r, label lab, chunk c of
// kUcChunk pixels), ordered by (lab, c) within a clique:
//   ucond_minmax_kernel   per (r, c): the min / max of trunc(Q) of each
//                         label's unit (coalesced reads of the pixels' rows);
//   ucond_carry_kernel    per clique: exclusive scan of the units -> carry-in;
//   ucond_select_kernel   per (r, c), a warp per label: its lanes replay runs
//                         of the unit from the carry (a warp scan gives each
//                         run its own) exactly as the reference's loop, and
//                         the unit's last selected positions are kept;
//   ucond_pos_kernel      per clique: the last over its units.
// Work is spread over all SMs however uneven the clique sizes are.
constexpr int kUcChunk = kCliqueChunk;  // pixels per unit (4 per lane of a warp)

__global__ void __launch_bounds__(256)
    ucond_minmax_kernel(const int2* __restrict__ chunks, const int* __restrict__ off, const int* __restrict__ idx,
                        const int* __restrict__ ubase, int L, const float* __restrict__ Q, int2* __restrict__ part) {
    __shared__ int smn[kLMax], smx[kLMax];
    const int2 rc = chunks[blockIdx.x];
    const int r = rc.x, c = rc.y, t = threadIdx.x;
    const int s0 = off[r], sz = off[r + 1] - s0, nch = (sz + kUcChunk - 1) / kUcChunk;
    const int j0 = c * kUcChunk, n = min(kUcChunk, sz - j0);
    if (t < L) {
        smn[t] = INT_MAX;
        smx[t] = INT_MIN;
    }
    __syncthreads();
    const int G = blockDim.x / L;  // pixel groups; thread (g, lab) keeps one label
    const int g = t / L, lab = t - g * L;
    if (g < G) {
        int mn = INT_MAX, mx = INT_MIN;
        for (int j = g; j < n; j += G) {
            const int v = trunc_x86(Q[(long)idx[s0 + j0 + j] * L + lab]);
            mn = min(mn, v);
            mx = max(mx, v);
        }
        atomicMin(&smn[lab], mn);
        atomicMax(&smx[lab], mx);
    }
    __syncthreads();
    if (t < L) part[ubase[r] + t * nch + c] = make_int2(smn[t], smx[t]);
}

__global__ void __launch_bounds__(1024)
    ucond_carry_kernel(const int* __restrict__ off, const int* __restrict__ ubase, int L,
                       const int2* __restrict__ part, int2* __restrict__ carry) {
    __shared__ int wmn[32], wmx[32];
    __shared__ int tmn, tmx;
    const int r = blockIdx.x, t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int sz = off[r + 1] - off[r], units = L * ((sz + kUcChunk - 1) / kUcChunk), base = ubase[r];
    if (t == 0) {
        tmn = INT_MAX;
        tmx = INT_MIN;
    }
    for (int u0 = 0; u0 < units; u0 += blockDim.x) {  // block-uniform
        __syncthreads();
        const int u = u0 + t;
        const int2 v = u < units ? part[base + u] : make_int2(INT_MAX, INT_MIN);
        int xmn = v.x, xmx = v.y;  // inclusive warp scan
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int ymn = __shfl_up_sync(kFullMask, xmn, o), ymx = __shfl_up_sync(kFullMask, xmx, o);
            if (lane >= o) {
                xmn = min(xmn, ymn);
                xmx = max(xmx, ymx);
            }
        }
        if (lane == 31) {
            wmn[w] = xmn;
            wmx[w] = xmx;
        }
        __syncthreads();
        int emn = tmn, emx = tmx;  // carry of the tiles before, then of the warps before
        for (int ww = 0; ww < w; ww++) {
            emn = min(emn, wmn[ww]);
            emx = max(emx, wmx[ww]);
        }
        int pmn = __shfl_up_sync(kFullMask, xmn, 1), pmx = __shfl_up_sync(kFullMask, xmx, 1);
        if (lane > 0) {
            emn = min(emn, pmn);
            emx = max(emx, pmx);
        }
        if (u < units) carry[base + u] = make_int2(emn, emx);
        __syncthreads();
        if (t == blockDim.x - 1) {  // the tile's total joins the running carry
            tmn = min(emn, xmn);
            tmx = max(emx, xmx);
        }
    }
}

__global__ void __launch_bounds__(256)
    ucond_select_kernel(const int2* __restrict__ chunks, const int* __restrict__ off, const int* __restrict__ idx,
                        const int* __restrict__ ubase, int L, const float* __restrict__ Q,
                        const int2* __restrict__ carry, int2* __restrict__ cand) {
    constexpr int kRun = kUcChunk / 32;
    const int2 rc = chunks[blockIdx.x];
    const int r = rc.x, c = rc.y, lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int s0 = off[r], sz = off[r + 1] - s0, nch = (sz + kUcChunk - 1) / kUcChunk;
    const int j0 = c * kUcChunk, n = min(kUcChunk, sz - j0);
    const int a = min(lane * kRun, n), b = min(a + kRun, n);  // this lane's run of the unit
    for (int lab = w; lab < L; lab += nw) {  // warp-uniform
        float q[kRun];
        int mn = INT_MAX, mx = INT_MIN;
#pragma unroll
        for (int i = 0; i < kRun; i++) {
            q[i] = a + i < b ? Q[(long)idx[s0 + j0 + a + i] * L + lab] : 0.0f;
            if (a + i < b) {
                const int v = trunc_x86(q[i]);
                mn = min(mn, v);
                mx = max(mx, v);
            }
        }
        int xmn = mn, xmx = mx;  // inclusive warp scan of the runs
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int ymn = __shfl_up_sync(kFullMask, xmn, o), ymx = __shfl_up_sync(kFullMask, xmx, o);
            if (lane >= o) {
                xmn = min(xmn, ymn);
                xmx = max(xmx, ymx);
            }
        }
        const int2 cin = carry[ubase[r] + lab * nch + c];
        int emn = cin.x, emx = cin.y;
        const int pmn = __shfl_up_sync(kFullMask, xmn, 1), pmx = __shfl_up_sync(kFullMask, xmx, 1);
        if (lane > 0) {
            emn = min(emn, pmn);
            emx = max(emx, pmx);
        }
        int cmn = -1, cmx = -1;
#pragma unroll
        for (int i = 0; i < kRun; i++) {
            if (a + i < b) {
                const int p = lab * sz + j0 + a + i;
                if (q[i] < (float)emn) cmn = p;
                if (q[i] > (float)emx) cmx = p;
                const int v = trunc_x86(q[i]);
                emn = min(emn, v);
                emx = max(emx, v);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            cmn = max(cmn, __shfl_down_sync(kFullMask, cmn, o));
            cmx = max(cmx, __shfl_down_sync(kFullMask, cmx, o));
        }
        if (lane == 0) cand[ubase[r] + lab * nch + c] = make_int2(cmn, cmx);
    }
}

__global__ void __launch_bounds__(256)
    ucond_pos_kernel(const int* __restrict__ off, const int* __restrict__ idx, const int* __restrict__ ubase, int L,
                     const int2* __restrict__ cand, int* __restrict__ pos) {
    __shared__ int smn[8], smx[8];
    const int r = blockIdx.x, t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int s0 = off[r], sz = off[r + 1] - s0, units = L * ((sz + kUcChunk - 1) / kUcChunk), base = ubase[r];
    int cmn = -1, cmx = -1;
    for (int u = t; u < units; u += blockDim.x) {
        const int2 v = cand[base + u];
        cmn = max(cmn, v.x);
        cmx = max(cmx, v.y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cmn = max(cmn, __shfl_down_sync(kFullMask, cmn, o));
        cmx = max(cmx, __shfl_down_sync(kFullMask, cmx, o));
    }
    if (lane == 0) {
        smn[w] = cmn;
        smx[w] = cmx;
    }
    __syncthreads();
    if (t == 0) {
        int lmn = -1, lmx = -1;
        for (int ww = 0; ww < (int)(blockDim.x >> 5); ww++) {
            lmn = max(lmn, smn[ww]);
            lmx = max(lmx, smx[ww]);
        }
        // element index pixel*L + label, or -1 when nothing was selected
        pos[2 * r] = lmn < 0 ? -1 : idx[s0 + lmn % sz] * L + lmn / sz;
        pos[2 * r + 1] = lmx < 0 ? -1 : idx[s0 + lmx % sz] * L + lmx / sz;
    }
}

// The reference then writes, clique after clique, Us[min] = c_r w_r and
// Us[max] = -c_r w_r, where an unselected side keeps the previous clique's
// position (both start at element 0), and later writes overwrite earlier
// ones.  Write 2r targets the min position of clique r, write 2r+1 its max.
// ucond_targets resolves every write's target (a running "last selected"
// scan over r); ucond_claim keeps, per target, the latest write (atomicMax
// into win[], which is -1 everywhere between calls); ucond_write lets that
// write store its value and resets win[].
__global__ void __launch_bounds__(1024) ucond_targets_kernel(int R, const int* __restrict__ pos,
                                                             int* __restrict__ tgt) {
    __shared__ int sl[2][32];
    __shared__ int carry[2];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (t < 2) carry[t] = -1;
    __syncthreads();
    for (int base = 0; base < R; base += 1024) {
        const int r = base + t;
        int last[2];
#pragma unroll
        for (int side = 0; side < 2; side++) {
            int x = (r < R && pos[2 * r + side] >= 0) ? r : -1;  // inclusive running max of selected r
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(kFullMask, x, o);
                if (lane >= o) x = max(x, y);
            }
            if (lane == 31) sl[side][w] = x;
            last[side] = x;
        }
        __syncthreads();
#pragma unroll
        for (int side = 0; side < 2; side++) {
            int x = max(last[side], carry[side]);
            for (int ww = 0; ww < w; ww++) x = max(x, sl[side][ww]);
            last[side] = x;
        }
        __syncthreads();
        if (r < R)
#pragma unroll
            for (int side = 0; side < 2; side++)
                tgt[2 * r + side] = last[side] < 0 ? 0 : pos[2 * last[side] + side];
        if (t == 1023 || r == R - 1) {
            carry[0] = last[0];
            carry[1] = last[1];
        }
        __syncthreads();
    }
}

__global__ void ucond_claim_kernel(int W, const int* __restrict__ tgt, int* __restrict__ win) {
    const int wi = blockIdx.x * blockDim.x + threadIdx.x;
    if (wi < W) atomicMax(win + tgt[wi], wi);
}

__global__ void ucond_write_kernel(int W, const int* __restrict__ tgt, const float* __restrict__ cst,
                                   const float* __restrict__ ew, int* __restrict__ win, float* __restrict__ Us) {
    const int wi = blockIdx.x * blockDim.x + threadIdx.x;
    if (wi >= W) return;
    const int e = tgt[wi], r = wi >> 1;
    if (win[e] == wi) Us[e] = (wi & 1) ? fmul(-cst[r], ew[r]) : fmul(cst[r], ew[r]);
}

__global__ void ucond_reset_kernel(int W, const int* __restrict__ tgt, int* __restrict__ win) {
    const int wi = blockIdx.x * blockDim.x + threadIdx.x;
    if (wi < W) win[tgt[wi]] = -1;
}

constexpr int kPix = 128;

}  // namespace

__global__ void ho_energy_finish_kernel(int nterms, SolverScalars* sc, int has_ho) {
    double e = 0.0;
    e += sc->sums[0];
    for (int k = 0; k < nterms; k++) e += sc->sums[1 + k];
    e += has_ho ? sc->sums[8] : 0.0;
    sc->energy = e;
}

__global__ void clear_step_flags_kernel(SolverScalars* sc) {
    sc->zero_step = 0;
    sc->steps = 0;
}

// compute_energy_higher_order(Q): U.Q + sum_k Q.A_k Q + the clique term
// (z o c).sum() + multiplySuperPixels((1 - z) o c, Q - 1) in float, with z
// the clique variables the last QP left (src/densecrf.cpp:960-980, 439).
double Model::energy_qp_ho(const float* Q) {
    require(has_unary, DCRF_E_STATE, "energy: no unary energy set");
    require(R == 0 || has_z_last, DCRF_E_STATE,
            "compute_energy_higher_order: no QP has run since the cliques were set");
    const int nt = (int)terms.size();
    require(nt + 1 <= 8, DCRF_E_ARG, "energy: too many pairwise terms");
    const long NL = (long)N * L;
    SolverScalars* sc = scal.get();
    double* part = partials.get();
    float* o = buf(11);
    launch(dot_kernel, kRedBlocks, kRedThreads, 0, stream, NL, unary.get(), Q, part);
    launch(finalize_sums_kernel, 1, 32, 0, stream, part, kRedBlocks, 1, 0, sc);
    for (int k = 0; k < nt; k++) {
        apply(k, false, o, Q);
        launch(dot_kernel, kRedBlocks, kRedThreads, 0, stream, NL, Q, o, part);
        launch(finalize_sums_kernel, 1, 32, 0, stream, part, kRedBlocks, 1, 1 + k, sc);
    }
    if (R > 0) {
        const int LR = L * R;
        const int* base = cl_off.get();
        const CliqueView cv{base, base + R + 1, base + 2 * R + 1, cl_idx.get(), cl_exp.get(), cl_const.get(), R,
                            clique_max, cl_bstart.get()};
        float* small = b[14].ensure((size_t)8 * LR);
        float *zc = small + 6 * LR, *omz = small + 7 * LR;
        double* preQ = ho_pre.ensure((size_t)2 * LR);
        launch(clear_step_flags_kernel, 1, 1, 0, stream, sc);
        launch(ho_zterm_prep_kernel, 1, 256, 0, stream, cv, L, (const float*)z_last.get(), zc, omz, sc);
        launch(eig_sum_kernel, 1, kHoThreads, 0, stream, (const float*)zc, LR, 8, sc, 2);
        ho_prefix64(stream, ho_seg, clique_max, L, cv, Q, 1, preQ, nullptr, 0);
        launch(ho_scalar_kernel, 1, kLMax, 0, stream, cv, L, (const float*)omz, (const double*)preQ, 8, sc, 1);
    }
    launch(ho_energy_finish_kernel, 1, 1, 0, stream, nt, sc, (int)(R > 0));
    DCRF_LAUNCH_CHECK();
    fetch_scalars();
    return h_scal->energy;
}

// max_rounding (src/densecrf.cpp:832-840): a one-hot column at the first
// maximum of each pixel.
void Model::max_rounding(const float* Q, float* out) {
    const long NL = (long)N * L;
    if (out != Q) DCRF_CUDA(cudaMemcpyAsync(out, Q, sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
    with_lc(L, [&](auto lc) {
        constexpr int LC = decltype(lc)::value;
        launch(max_rounding_kernel<LC>, ceil_div(N, kPix), kPix, 0, stream, N, L, out);
    });
    DCRF_LAUNCH_CHECK();
}

// ---------------------------------------------------------------- QP host --
// Everything a captured QP iteration holds by address or by value that can
// change between solves.
std::vector<const void*> Model::qp_graph_key(const float* Q, int max_iter) {
    std::vector<const void*> k = {Q, (const void*)(intptr_t)max_iter, (const void*)(uintptr_t)gen, unary.get(),
                                  scal.get(), partials.get(), ipart.get(), ho_pre.get(), cl_off.get(), cl_idx.get()};
    for (int i = 0; i < 16; i++) k.push_back(b[i].get());
    for (const auto& t : terms) {
        k.push_back(t->lat->va.get());
        k.push_back(t->lat->vb.get());
        k.push_back(t->norm.get());
        k.push_back(t->cw.get());
    }
    k.push_back(compat_tmp.get());
    return k;
}

void Model::drop_qp_graph() {
    if (qp_graph) cudaGraphExecDestroy(qp_graph);
    qp_graph = nullptr;
    qp_key.clear();
}

template <typename F>
void Model::build_qp_graph(F&& qp_iter) {
    std::lock_guard<std::recursive_mutex> cap(capture_mutex());
    drop_qp_graph();
    SolverScalars* sc = scal.get();
    cudaGraph_t g = nullptr;
    DCRF_CUDA(cudaGraphCreate(&g, 0));
    bool capturing = false;
    try {
        cudaGraphConditionalHandle h;
        DCRF_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
        cudaMemsetParams mp = {};
        mp.dst = &sc->chunk;
        mp.value = 0;
        mp.elementSize = sizeof(int);
        mp.width = 1;
        mp.height = 1;
        cudaGraphNode_t mn, wn;
        DCRF_CUDA(cudaGraphAddMemsetNode(&mn, g, nullptr, 0, &mp));
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        DCRF_CUDA(cudaGraphAddNode(&wn, g, &mn, 1, &np));
        const unsigned long long k0 = g_kernel_launches.load();
        DCRF_CUDA(cudaStreamBeginCaptureToGraph(stream, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                cudaStreamCaptureModeRelaxed));
        capturing = true;
        qp_iter();
        launch(qp_cond_kernel, 1, 1, 0, stream, sc, kQpChunk, h);
        cudaGraph_t bo = nullptr;
        capturing = false;
        DCRF_CUDA(cudaStreamEndCapture(stream, &bo));
        const unsigned long long captured = g_kernel_launches.load() - k0;
        g_kernel_launches.fetch_sub(captured);  // counted per iteration when the graph runs
        require(captured >= 2, DCRF_E_STATE, "qp: unexpected loop body");
        qp_graph_kernels = captured;
        DCRF_CUDA(cudaGraphInstantiate(&qp_graph, g, 0));
        cudaGraphDestroy(g);
    } catch (...) {
        cudaGraph_t junk = nullptr;
        if (capturing) cudaStreamEndCapture(stream, &junk);
        cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
    }
}

int Model::qp(const float* init, float* out, int max_iter, double* energy_out) {
    require(has_unary, DCRF_E_STATE, "qp: no unary energy set");
    const long NL = (long)N * L;
    float* Q = out;  // iterate in place in the output buffer
    float* grad = buf(0);
    float* sx = buf(1);
    float* psi = buf(2);
    float* tmp = buf(3);
    float* ho = nullptr;
    if (Q != init) DCRF_CUDA(cudaMemcpyAsync(Q, init, sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
    DCRF_CUDA(cudaMemcpyAsync(grad, unary.get(), sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
    DCRF_CUDA(cudaMemsetAsync(scal.get(), 0, sizeof(SolverScalars), stream));
    SolverScalars* sc = scal.get();
    double* part = partials.get();
    const int nt = (int)terms.size();
    const int tgrid = ceil_div(ceil_div(N, 32), kTileWarps);  // row-tiled kernels

    CliqueView cv{};
    float* pre32 = nullptr;                   // float prefixes of Q - 1 at the clique sizes
    double *preQ = nullptr, *preS = nullptr;  // FP64 prefixes of Q - 1 and of sx
    float *gz = nullptr, *z = nullptr, *sxz = nullptr, *t1 = nullptr, *t2 = nullptr, *cz = nullptr, *zc = nullptr,
          *omz = nullptr;
    const int LR = L * R;
    if (R > 0) {
        const int* base = cl_off.get();
        cv = CliqueView{base, base + R + 1, base + 2 * R + 1, cl_idx.get(), cl_exp.get(), cl_const.get(), R, clique_max,
                        cl_bstart.get()};
        float* small = b[14].ensure((size_t)8 * LR);
        pre32 = b[15].ensure((size_t)LR);
        double* dpre = ho_pre.ensure((size_t)2 * LR);
        preQ = dpre;
        preS = dpre + LR;
        gz = small;
        z = small + LR;
        sxz = small + 2 * LR;
        t1 = small + 3 * LR;
        t2 = small + 4 * LR;
        cz = small + 5 * LR;
        zc = small + 6 * LR;
        omz = small + 7 * LR;
        launch(fill_float_kernel, ceil_div(LR, 256), 256, 0, stream, LR, 1.0f, z);
        ho = buf(4);
        DCRF_CUDA(cudaMemsetAsync(ho, 0, sizeof(float) * NL, stream));
        // the float chain of Q - 1 (sequential, as the reference sums it) and its FP64 prefixes
        ho_prefix32(stream, L, cv, Q, 1, pre32, nullptr, 0);
        ho_prefix64(stream, ho_seg, clique_max, L, cv, Q, 1, preQ, nullptr, 0);
        launch(ho_regions_kernel, ceil_div(LR, 256), 256, 0, stream, cv, L, pre32, gz, 0, nullptr);
    }
    // grad_y = unary + sum_k 2 A_k Q; energy terms Q . A_k Q (same applies).
    for (int k = 0; k < nt; k++) {
        apply(k, false, tmp, Q);
        launch(add_scaled_kernel, ceil_div(NL, 256), 256, 0, stream, NL, grad, tmp, 2.0f);
        launch(dot_kernel, kRedBlocks, kRedThreads, 0, stream, NL, Q, tmp, part);
        launch(finalize_sums_kernel, 1, 32, 0, stream, part, kRedBlocks, 1, 1 + k, sc);
    }
    if (R > 0) {
        launch(ho_pixels_kernel, ceil_div((long)clique_max * L, 256), 256, 0, stream, cv, L, z, ho, nullptr);
        launch(add_inplace_kernel, ceil_div(NL, 256), 256, 0, stream, NL, grad, ho);
        launch(ho_zterm_prep_kernel, 1, 256, 0, stream, cv, L, z, zc, omz, sc);
        launch(eig_sum_kernel, 1, kHoThreads, 0, stream, zc, LR, 8, sc, 2);
        launch(ho_scalar_kernel, 1, kLMax, 0, stream, cv, L, omz, preQ, 8, sc, 1);
    }
    launch(dot_kernel, kRedBlocks, kRedThreads, 0, stream, NL, unary.get(), Q, part);
    launch(finalize_sums_kernel, 1, 32, 0, stream, part, kRedBlocks, 1, 0, sc);
    launch(qp_init_energy_kernel, 1, 1, 0, stream, sc, nt, max_iter);
    launch(nonfinite_kernel, nonfinite_grid(NL), 256, 0, stream, NL, (const float*)Q, unary.get(), sc);
    DCRF_LAUNCH_CHECK();
    fetch_scalars();
    if (h_scal->numeric & 1)
        throw Error(DCRF_E_NUMERIC, "qp: the initial Q or the unary energy holds a NaN or an infinity");
    // One Frank-Wolfe iteration (src/densecrf.cpp:389-436) and its stop test.
    auto qp_iter = [&]() {
        with_lc(L, [&](auto lc) {
            constexpr int LC = decltype(lc)::value;
            if constexpr (LC > 0) {
                launch(qp_direction_tiled<LC>, tgrid, 32 * kTileWarps, 0, stream, N, grad, Q, unary.get(), sx, part);
                launch(finalize_large_kernel, 1, 1024, 0, stream, part, tgrid, 0, sc);
            } else {
                launch(qp_direction_kernel<LC>, kRedBlocks, kRedThreads, 0, stream, N, L, grad, Q, unary.get(), sx,
                       part);
                launch(finalize_sums_kernel, 1, 32, 0, stream, part, kRedBlocks, 1, 0, sc);
            }
        });
        if (R > 0) {
            launch(ho_direction_kernel, 1, 256, 0, stream, cv, L, gz, z, sxz, t1, t2, cz, sc);
            launch(eig_sum_kernel, 1, kHoThreads, 0, stream, sxz, LR, 5, sc, 0);
            ho_prefix64(stream, ho_seg, clique_max, L, cv, sx, 0, preS, sc, 0);
            launch(ho_scalar_kernel, 1, kLMax, 0, stream, cv, L, t1, preQ, 3, sc, 0);    // a
            launch(ho_scalar_kernel, 1, kLMax, 0, stream, cv, L, t2, preS, 4, sc, 0);   // b
            launch(ho_scalar_kernel, 1, kLMax, 0, stream, cv, L, t1, preS, 6, sc, 0);   // denom term
        }
        apply_sum(psi, sx);
        launch(dots2_kernel, kRedBlocks, kRedThreads, 0, stream, NL, Q, sx, psi, part);
        launch(finalize_sums_kernel, 1, 64, 0, stream, part, kRedBlocks, 2, 1, sc);
        launch(qp_step_kernel, 1, 1, 0, stream, sc);
        if (R > 0) {
            launch(ho_z_update_kernel, 1, 256, 0, stream, LR, z, sxz, sc);
            launch(ho_pixels_kernel, ceil_div((long)clique_max * L, 256), 256, 0, stream, cv, L, z, ho, sc);
        }
        launch(qp_update_kernel, kRedBlocks, kRedThreads, 0, stream, NL, sx, psi, ho, unary.get(), Q, grad, sc, part);
        launch(finalize_sums_kernel, 1, 32, 0, stream, part, kRedBlocks, 1, 7, sc);
        if (R > 0) {
            // the prefixes of the updated Q - 1 (after a zero step Q is
            // unchanged, and so is the float chain)
            ho_prefix32(stream, L, cv, Q, 1, pre32, sc, 1);
            ho_prefix64(stream, ho_seg, clique_max, L, cv, Q, 1, preQ, nullptr, 0);
            launch(ho_regions_kernel, ceil_div(LR, 256), 256, 0, stream, cv, L, pre32, gz, 1, sc);
            launch(ho_zterm_prep_kernel, 1, 256, 0, stream, cv, L, z, zc, omz, sc);
            launch(eig_sum_kernel, 1, kHoThreads, 0, stream, zc, LR, 8, sc, 2);
            launch(ho_scalar_kernel, 1, kLMax, 0, stream, cv, L, omz, preQ, 8, sc, 1);
        }
        launch(qp_energy_kernel, 1, 1, 0, stream, sc, max_iter);
        DCRF_LAUNCH_CHECK();
    };
    // After the first iteration (eager: it sizes every buffer) the loop runs
    // as a CUDA graph: a `while` node whose body is one iteration and whose
    // condition qp_cond_kernel sets -- until the stop rule fires, or kQpChunk
    // iterations per launch, after which the host looks at the stop flag and
    // launches it again.  The graph is kept for later solves with the same
    // buffers and model.
    const std::vector<const void*> key = qp_graph_key(Q, max_iter);
    int guard = 0;
    while (!h_scal->stop) {
        require(++guard < (1 << 26), DCRF_E_TIMEOUT, "qp: iteration cap reached");
        if (qp_graph && key == qp_key) {
            DCRF_CUDA(cudaGraphLaunch(qp_graph, stream));
            fetch_scalars();
            g_kernel_launches.fetch_add(qp_graph_kernels * (unsigned long long)h_scal->chunk);
            continue;
        }
        qp_iter();
        fetch_scalars();
        if (!h_scal->stop && !qp_graph_failed && graphs_enabled()) {
            try {
                build_qp_graph(qp_iter);
                qp_key = key;
            } catch (const Error&) {
                drop_qp_graph();
                qp_graph_failed = true;  // this device or driver cannot run it: stay eager
            }
        }
    }
    if (R > 0) {  // z_labels_ = z (src/densecrf.cpp:439)
        DCRF_CUDA(cudaMemcpyAsync(z_last.ensure((size_t)LR), z, sizeof(float) * LR, cudaMemcpyDeviceToDevice,
                                  stream));
        sync();
    }
    has_z_last = true;
    if (energy_out) *energy_out = h_scal->energy;
    return h_scal->steps;
}

// ---------------------------------------------------------------- LP host --
int Model::lp(const float* init, float* out, const dcrf_lp_params& p, dcrf_solve_stats* stats) {
    require(has_unary, DCRF_E_STATE, "lp: no unary energy set");
    const long NL = (long)N * L;
    float* Q = buf(0);
    float* bestQ = out;
    float* alpha = buf(1);
    float* u = buf(2);
    float* sa = buf(3);
    float* su = R > 0 ? buf(4) : nullptr;
    float* gamma = buf(5);
    float* curQ = buf(6);
    float2* bins = lp_bins.ensure(NL);
    float* Y = buf(8);
    int16_t* lab = labels.ensure(N);
    SolverScalars* sc = scal.get();
    double* part = partials.get();
    const int nt = (int)terms.size();
    const int pg = ceil_div(N, kPix);
    const int tgrid = ceil_div(ceil_div(N, 32), kTileWarps);  // row-tiled kernels

    DCRF_CUDA(cudaMemcpyAsync(Q, init, sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
    DCRF_CUDA(cudaMemsetAsync(&sc->numeric, 0, sizeof(int), stream));
    launch(nonfinite_kernel, nonfinite_grid(NL), 256, 0, stream, NL, (const float*)Q, unary.get(), sc);
    with_lc(L, [&](auto lc) {
        constexpr int LC = decltype(lc)::value;
        launch(renormalize_kernel<LC>, pg, kPix, 0, stream, N, L, Q);
    });
    DCRF_CUDA(cudaMemcpyAsync(bestQ, Q, sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
    current_map(Q, lab);
    double int_energy = energy_true(lab, true);  // reads the scalars back
    if (h_scal->numeric & 1)
        throw Error(DCRF_E_NUMERIC, "lp: the initial Q or the unary energy holds a NaN or an infinity");
    double energy = energy_lp(Q);
    if (energy > int_energy) {
        with_lc(L, [&](auto lc) {
            constexpr int LC = decltype(lc)::value;
            launch(max_rounding_kernel<LC>, pg, kPix, 0, stream, N, L, Q);
        });
        energy = energy_lp(Q);
    }
    double best_energy = energy, best_int_energy = int_energy;

    const float lambda = p.prox_reg_const;
    GammaConsts gc;
    gc.lambda = lambda;
    gc.delta = p.qp_const;
    gc.c0 = 2 * lambda / float(L);
    gc.c1 = (float)(1.0 / float(L));
    gc.c2 = (float)(1 - 2.0 / float(L));
    gc.cm = (float)(-1.0 / float(L));
    CliqueView cv{};
    int* upos = nullptr;
    if (R > 0) {
        const int* base = cl_off.get();
        cv = CliqueView{base, base + R + 1, base + 2 * R + 1, cl_idx.get(), cl_exp.get(), cl_const.get(), R, clique_max,
                        cl_bstart.get()};
        upos = ipart.ensure(4 * (size_t)R);  // [2R] selected positions, [2R] write targets
        if (!lp_win.get()) {
            int* w = lp_win.ensure((size_t)N * L);
            DCRF_CUDA(cudaMemsetAsync(w, 0xff, sizeof(int) * (size_t)N * L, stream));  // -1: no claim
        }
    }

    int it = 0, count = 0, fw_total = 0;
    DCRF_CUDA(cudaMemsetAsync(&sc->gamma_sum, 0, sizeof(int), stream));

    // One Frank-Wolfe iteration in three parts: lp_y and the qp-gamma reset
    // (s1), the qp-gamma iterations, and Q, the bins, the clique and ordered
    // subgradients and the dual-gap step (s2).
    auto s1 = [&](bool pending) {
        // alpha / u of the previous iteration are updated inside lp_y (the
        // update after the last iteration is never read: both are reset
        // before the next proximal step).
        with_lc(L, [&](auto lc) {
            constexpr int LC = decltype(lc)::value;
            if constexpr (LC > 0)
                launch(lp_y_tiled<LC>, tgrid, 32 * kTileWarps, 0, stream, N, lambda, gc.cm, alpha, u, unary.get(),
                       curQ, Y, pending, sa, su, sc);
            else
                launch(lp_y_kernel<LC>, pg, kPix, 0, stream, N, L, lambda, gc.cm, alpha, u, unary.get(), curQ, Y,
                       pending, sa, su, sc);
        });
        launch(lp_gamma_reset_kernel, 1, 1, 0, stream, sc);
    };
    // One qp-gamma iteration on stream st; with a graph handle its test also
    // sets the graph's loop condition.
    auto gamma_step = [&](cudaStream_t st, const cudaGraphConditionalHandle* h) {
        with_lc(L, [&](auto lc) {
            constexpr int LC = decltype(lc)::value;
            const int nblk = LC > 0 ? tgrid : kRedBlocks;
            if constexpr (LC > 0)
                launch(lp_gamma_tiled<LC>, tgrid, 32 * kTileWarps, 0, st, N, gc, Y, gamma, sc, part);
            else
                launch(lp_gamma_kernel<LC>, kRedBlocks, kRedThreads, 0, st, N, L, gc, Y, gamma, sc, part);
            if (h)
                launch(lp_gamma_check_cond_kernel, 1, 1024, 0, st, part, nblk, p.qp_tol, sc, p.qp_max_iter, *h);
            else
                launch(lp_gamma_check_kernel, 1, 1024, 0, st, part, nblk, p.qp_tol, sc);
        });
    };
    auto s2 = [&]() {
        // Q, with the min / max of rescale folded in; then the bins of
        // rescale(Q) once for all pairwise terms.
        with_lc(L, [&](auto lc) {
            constexpr int LC = decltype(lc)::value;
            if constexpr (LC > 0) {
                launch(lp_q_tiled<LC>, tgrid, 32 * kTileWarps, 0, stream, N, lambda, alpha, u, gamma, unary.get(),
                       curQ, Q, part);
                launch(minmax_finish_kernel, 1, 1024, 0, stream, part, tgrid, sc);
            } else {
                launch(lp_q_kernel<LC>, pg, kPix, 0, stream, N, L, lambda, alpha, u, gamma, unary.get(), curQ, Q,
                       part);
                launch(minmax_finish_kernel, 1, 1024, 0, stream, part, pg, sc);
            }
        });
        rescaled_bins(bins, Q, NL, &sc->qmin, stream);
        // Clique conditional gradient su (computeUCondGrad), before the
        // ordered filters so that the dual-gap sums can ride along the
        // last term's slice with su included.
        if (R > 0) {
            const int nw = 2 * R;
            int* tgt = upos + 2 * R;
            DCRF_CUDA(cudaMemsetAsync(su, 0, sizeof(float) * NL, stream));
            int2* ucp = uc_scan.ensure(std::max<size_t>(3 * (size_t)uc_units, 1));
            if (uc_nchunks > 0) {
                launch(ucond_minmax_kernel, uc_nchunks, 256, 0, stream, uc_chunks.get(), cl_off.get(), cl_idx.get(),
                       uc_base.get(), L, Q, ucp);
                launch(ucond_carry_kernel, R, 1024, 0, stream, cl_off.get(), uc_base.get(), L, (const int2*)ucp,
                       ucp + uc_units);
                launch(ucond_select_kernel, uc_nchunks, 256, 0, stream, uc_chunks.get(), cl_off.get(), cl_idx.get(),
                       uc_base.get(), L, Q, (const int2*)(ucp + uc_units), ucp + 2 * (size_t)uc_units);
            }
            launch(ucond_pos_kernel, R, 256, 0, stream, cl_off.get(), cl_idx.get(), uc_base.get(), L,
                   (const int2*)(ucp + 2 * (size_t)uc_units), upos);
            launch(ucond_targets_kernel, 1, 1024, 0, stream, R, upos, tgt);
            launch(ucond_claim_kernel, ceil_div(nw, 256), 256, 0, stream, nw, tgt, lp_win.get());
            launch(ucond_write_kernel, ceil_div(nw, 256), 256, 0, stream, nw, tgt, cl_const.get(), cl_exp.get(),
                   lp_win.get(), su);
            launch(ucond_reset_kernel, ceil_div(nw, 256), 256, 0, stream, nw, tgt, lp_win.get());
        }
        // Ordered subgradient sa = sum_k apply_upper_minus_lower_ord_k; the
        // dual-gap sums ride along the last term's slice.
        const bool fuse_gap = nt > 0 && terms[nt - 1]->compat != kMatrix;
        GapFusion gf{alpha, u, Q, part, R > 0 ? su : nullptr};
        apply_ord_sum(sa, bins, fuse_gap ? &gf : nullptr);
        if (nt == 0) DCRF_CUDA(cudaMemsetAsync(sa, 0, sizeof(float) * NL, stream));
        if (fuse_gap) {
            launch(finalize_large_kernel, 2, 1024, 0, stream, part, slice_grid(NL), 0, sc);
        } else {
            launch(lp_gap_kernel, kRedBlocks, kRedThreads, 0, stream, NL, alpha, u, sa, su, Q, part);
            launch(finalize_sums_kernel, 1, 64, 0, stream, part, kRedBlocks, 2, 0, sc);
        }
        launch(lp_delta_kernel, 1, 1, 0, stream, sc, lambda);
        DCRF_LAUNCH_CHECK();
    };
    // The whole iteration as one CUDA graph: s1, a `while` node whose body is
    // one qp-gamma iteration and whose condition its test kernel sets, s2.
    // Built after the first iteration has run eagerly (it sizes every buffer
    // the iteration touches) and used for the rest of the solve: no host
    // round trip per iteration.  Kernel launch counts: the graph's own
    // kernels per launch plus two per qp-gamma iteration inside it.
    struct FwGraphs {  // released on every exit from the solve
        cudaGraphExec_t g[2] = {nullptr, nullptr};  // pending = false / true
        void drop() {
            for (auto& x : g)
                if (x) {
                    cudaGraphExecDestroy(x);
                    x = nullptr;
                }
        }
        ~FwGraphs() { drop(); }
    } fwg;
    cudaGraphExec_t* fw_graph = fwg.g;
    unsigned long long fw_graph_kernels = 0;
    bool graphs_ok = graphs_enabled();
    int eager_gamma = 0;
    auto drop_graphs = [&]() { fwg.drop(); };
    auto build_graph = [&](bool pending) -> cudaGraphExec_t {
        std::lock_guard<std::recursive_mutex> cap(capture_mutex());
        if (!gstream) DCRF_CUDA(cudaStreamCreateWithFlags(&gstream, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        DCRF_CUDA(cudaGraphCreate(&g, 0));
        bool main_cap = false, body_cap = false;
        try {
            cudaGraphConditionalHandle h;
            DCRF_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
            const unsigned long long k0 = g_kernel_launches.load();
            DCRF_CUDA(cudaStreamBeginCaptureToGraph(stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
            main_cap = true;
            s1(pending);
            cudaStreamCaptureStatus cs;
            cudaGraph_t cg = nullptr;
            const cudaGraphNode_t* deps = nullptr;
            size_t nd = 0;
            DCRF_CUDA(cudaStreamGetCaptureInfo(stream, &cs, nullptr, &cg, &deps, &nd));
            cudaGraphNodeParams np = {};
            np.type = cudaGraphNodeTypeConditional;
            np.conditional.handle = h;
            np.conditional.type = cudaGraphCondTypeWhile;
            np.conditional.size = 1;
            cudaGraphNode_t wn;
            DCRF_CUDA(cudaGraphAddNode(&wn, cg, deps, nd, &np));
            DCRF_CUDA(cudaStreamUpdateCaptureDependencies(stream, &wn, 1, cudaStreamSetCaptureDependencies));
            const unsigned long long kb = g_kernel_launches.load();
            DCRF_CUDA(cudaStreamBeginCaptureToGraph(gstream, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                    cudaStreamCaptureModeRelaxed));
            body_cap = true;
            gamma_step(gstream, &h);
            cudaGraph_t bo = nullptr;
            body_cap = false;
            DCRF_CUDA(cudaStreamEndCapture(gstream, &bo));
            const unsigned long long body_kernels = g_kernel_launches.load() - kb;
            // The loop ends only through its test kernel: a body without it
            // would never stop, so anything but the two kernels is refused.
            size_t body_nodes = 0;
            DCRF_CUDA(cudaGraphGetNodes(np.conditional.phGraph_out[0], nullptr, &body_nodes));
            require(body_nodes == 2 && body_kernels == 2, DCRF_E_STATE, "lp: unexpected qp-gamma loop body");
            s2();
            cudaGraph_t out = nullptr;
            main_cap = false;
            DCRF_CUDA(cudaStreamEndCapture(stream, &out));
            const unsigned long long captured = g_kernel_launches.load() - k0;
            g_kernel_launches.fetch_sub(captured);  // counted when the graph runs
            fw_graph_kernels = captured - body_kernels;
            cudaGraphExec_t ex = nullptr;
            DCRF_CUDA(cudaGraphInstantiate(&ex, g, 0));
            cudaGraphDestroy(g);
            return ex;
        } catch (...) {
            cudaGraph_t junk = nullptr;
            if (body_cap) cudaStreamEndCapture(gstream, &junk);
            if (main_cap) cudaStreamEndCapture(stream, &junk);
            cudaGraphDestroy(g);
            cudaGetLastError();
            throw;
        }
    };

    do {
        ++it;
        launch(fill_float_kernel, ceil_div(NL, 256), 256, 0, stream, NL, 1.0f, gamma);
        DCRF_CUDA(cudaMemcpyAsync(curQ, Q, sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
        DCRF_CUDA(cudaMemsetAsync(alpha, 0, sizeof(float) * NL, stream));
        DCRF_CUDA(cudaMemsetAsync(u, 0, sizeof(float) * NL, stream));
        int pit = 0;
        do {
            ++pit;
            const bool pending = pit > 1;
            if (graphs_ok && fw_graph[pending]) {
                DCRF_CUDA(cudaGraphLaunch(fw_graph[pending], stream));
                g_kernel_launches.fetch_add(fw_graph_kernels);
                continue;
            }
            s1(pending);
            // qp-gamma iterations; the reference needs at least two (its first
            // test compares against FLT_MAX), so launch in pairs and look at
            // the stop flag after each pair.
            int launched = 0;
            for (;;) {
                const int batch = std::min(2, p.qp_max_iter - launched);
                for (int bi = 0; bi < batch; bi++) gamma_step(stream, nullptr);
                launched += batch;
                DCRF_LAUNCH_CHECK();
                fetch_scalars();
                if (h_scal->stop || launched >= p.qp_max_iter || batch <= 0) break;
            }
            eager_gamma += h_scal->steps;
            s2();
            if (graphs_ok && !fw_graph[0]) {
                try {
                    fw_graph[0] = build_graph(false);
                    fw_graph[1] = build_graph(true);
                } catch (const Error&) {
                    drop_graphs();
                    graphs_ok = false;  // this device or driver cannot run them: stay eager
                }
            }
        } while (pit < p.fw_max_iter);
        fw_total += pit;
        with_lc(L, [&](auto lc) {
            constexpr int LC = decltype(lc)::value;
            launch(lp_project_kernel<LC>, pg, kPix, 0, stream, N, L, Q, lab);
        });
        const double prev_int_energy = int_energy;
        int_energy = energy_true(lab, true);  // reads the scalars back
        // rescale() of an iterate: the reference throws (src/eigen_utils.cpp:138)
        // and the LP rethrows it (src/densecrf.cpp:698-703); a NaN or infinity,
        // which the reference would carry on with, ends the solve too.
        if (h_scal->numeric & 4) throw Error(DCRF_E_NUMERIC, "Maxval < 0, skipping");
        if (h_scal->numeric & 2) throw Error(DCRF_E_NUMERIC, "lp: an iterate holds a NaN or an infinity");
        if (p.best_int) {
            if (std::abs(int_energy - prev_int_energy) < p.prox_energy_tol) ++count;
            else count = 0;
            if (count >= 5) break;
            if (int_energy < best_int_energy) {
                DCRF_CUDA(cudaMemcpyAsync(bestQ, Q, sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
                best_int_energy = int_energy;
            }
        } else {
            const double prev_energy = energy;
            energy = energy_lp(Q);
            if (std::abs(energy - prev_energy) < p.prox_energy_tol) ++count;
            else count = 0;
            if (count >= 5) break;
            if (energy < best_energy) {
                DCRF_CUDA(cudaMemcpyAsync(bestQ, Q, sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
                best_energy = energy;
            }
        }
        if (p.less_confident_percent > 0) {
            launch(less_confident_kernel, kRedBlocks, kRedThreads, 0, stream, N, L, bestQ, p.confidence_tol, part);
            launch(finalize_sums_kernel, 1, 32, 0, stream, part, kRedBlocks, 1, 0, sc);
            fetch_scalars();
            const double percent = h_scal->sums[0] / (double)N * 100;
            if (percent > p.less_confident_percent) break;
        }
    } while (it < p.prox_max_iter);
    fetch_scalars();
    // the two kernels of each qp-gamma iteration that ran inside a graph
    g_kernel_launches.fetch_add(2ull * (unsigned long long)std::max(0, h_scal->gamma_sum - eager_gamma));
    if (stats) {
        stats->iterations = it;
        stats->inner_iters = fw_total;
        stats->gamma_iters = h_scal->gamma_sum;
        stats->energy = p.best_int ? best_int_energy : best_energy;
    }
    return it;
}

}  // namespace dcrf
