// Batched Frank-Wolfe QP over images of different sizes (see batch.cuh).
//
// Each image keeps its own SolverScalars.  Every reduction is partitioned
// per image exactly as Model::qp partitions a single image (the same block
// grid over the image's elements, the same partial layout, the same
// finalisation order), so a batched image's trajectory, output and energy
// are bit-identical to its single-image solve (src/densecrf.cpp:340-442).
#include <algorithm>
#include <cfloat>

#include "batch.cuh"

#include <mutex>
#include "model_kernels.cuh"

namespace dcrf {

namespace {

__global__ void bfill_kernel(long n, float v, float* x) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) x[t] = v;
}

__global__ void bnorm_kernel(long N, float* x) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) x[i] = (float)(1.0 / sqrt(dadd((double)x[i], 1e-20)));
}

// ---- mean-field ---------------------------------------------------------

// expAndNormalize (src/densecrf.cpp:328-336) of the logits a: per pixel
// exp(a - max) / sum, the sum in Eigen's packet order.
template <int LC>
__global__ void softmax_kernel(long N, int Lrt, const float* __restrict__ a, float* __restrict__ Q) {
    const int L = LC ? LC : Lrt;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float b[PixVec<LC>::S];
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) b[k] = a[i * L + k];
    float mx = b[0];
#pragma unroll
    for (int k = 1; k < PixVec<LC>::S; k++)
        if (k < L && b[k] > mx) mx = b[k];
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) b[k] = expf(fsub(b[k], mx));
    const float sm = vec_sum<LC>(b, L);
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) Q[i * L + k] = b[k] / sm;
}

// Softmax adjoint: ga = Q o (g - <g, Q>) per pixel; dU = (first ? 0 : dU) - ga
// (the logits are -U + messages).
template <int LC>
__global__ void softmax_bwd_kernel(long N, int Lrt, const float* __restrict__ Q, const float* __restrict__ g,
                                   float* __restrict__ ga, float* __restrict__ dU, int first) {
    const int L = LC ? LC : Lrt;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) s += (double)g[i * L + k] * (double)Q[i * L + k];
    // g - <g, Q> cancels where g is nearly constant over the labels: formed
    // in FP64, rounded once.
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) {
            const long e = i * L + k;
            const float v = (float)((double)Q[e] * ((double)g[e] - s));
            ga[e] = v;
            dU[e] = (first ? 0.0f : dU[e]) - v;
        }
}

__global__ void negate_kernel(long n, const float* __restrict__ x, float* __restrict__ y) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) y[t] = -x[t];
}

// acc[j] += sum of the nblk partials (one warp, fixed order).
__global__ void accumulate_total_kernel(const double* __restrict__ partials, int nblk, double* acc) {
    const int lane = threadIdx.x;
    double s = 0.0;
    for (int b = lane; b < nblk; b += 32) s += partials[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(kFullMask, s, o);
    if (lane == 0) *acc += s;
}

// ---- lockstep QP ---------------------------------------------------------
// Every image's reductions use the block decomposition Model::qp gives a
// single image of that size (kRedBlocks virtual blocks striding over the
// image's elements, or its row tiles), and every image keeps its own
// SolverScalars, so each image's trajectory, output and energy are those of
// its own solve.  Each iteration starts by compacting the images still
// running (live_build_kernel); every kernel of the iteration, the filters
// included (Lattice::live_n), then loops over the live images' work only,
// with grids sized for the device rather than for the batch.
constexpr int kBPart = 2 * kRedBlocks;  // partial slots per image (two values at most)

struct BImages {
    const long* pix_off;            // B + 1 pixel offsets
    const int* live_n = nullptr;    // live images (device), or nullptr: every image
    const int* live_img = nullptr;
    int B;
    int L;
};

// Virtual blocks (image, vb) of every image or of the live images, numbered
// image after image; the kernels loop over them block-uniformly.
__device__ __forceinline__ long vblocks_total(const BImages& bi) {
    return (long)(bi.live_n ? *bi.live_n : bi.B) * kRedBlocks;
}
__device__ __forceinline__ void vblock_at(const BImages& bi, long u, int& img, int& vb, long& base, long& n) {
    const int r = (int)(u / kRedBlocks);
    vb = (int)(u - (long)r * kRedBlocks);
    img = bi.live_n ? bi.live_img[r] : r;
    base = bi.pix_off[img] * bi.L;
    n = (bi.pix_off[img + 1] - bi.pix_off[img]) * bi.L;
}

// block_sum_store for virtual block vb of an image: partials[j kRedBlocks + vb].
template <int NV>
__device__ __forceinline__ void vblock_store(double (&v)[NV], double* partials, int vb) {
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
        double t = 0.0;
        for (int ww = 0; ww < kRedThreads / 32; ww++) t += sm[threadIdx.x][ww];
        partials[(long)threadIdx.x * kRedBlocks + vb] = t;
    }
}

// dot_kernel per image: partials of a . b.
__global__ void bdot_kernel(BImages bi, const float* __restrict__ a, const float* __restrict__ b,
                            double* __restrict__ part) {
    for (long u = blockIdx.x; u < vblocks_total(bi); u += gridDim.x) {
        int img, vb;
        long base, n;
        vblock_at(bi, u, img, vb, base, n);
        double v[1] = {0.0};
        for (long t = (long)vb * blockDim.x + threadIdx.x; t < n; t += (long)kRedBlocks * blockDim.x)
            v[0] += (double)a[base + t] * (double)b[base + t];
        vblock_store<1>(v, part + (long)img * kBPart, vb);
        __syncthreads();  // vblock_store's shared sums are rewritten next
    }
}

// dots2_kernel per image: partials of a . c and b . c.
__global__ void bdots2_kernel(BImages bi, const float* __restrict__ a, const float* __restrict__ b,
                              const float* __restrict__ c, double* __restrict__ part) {
    for (long u = blockIdx.x; u < vblocks_total(bi); u += gridDim.x) {
        int img, vb;
        long base, n;
        vblock_at(bi, u, img, vb, base, n);
        double v[2] = {0.0, 0.0};
        for (long t = (long)vb * blockDim.x + threadIdx.x; t < n; t += (long)kRedBlocks * blockDim.x) {
            const double cc = c[base + t];
            v[0] += (double)a[base + t] * cc;
            v[1] += (double)b[base + t] * cc;
        }
        vblock_store<2>(v, part + (long)img * kBPart, vb);
        __syncthreads();
    }
}

// qp_update_kernel per image.
__global__ void bqp_update_kernel(BImages bi, const float* __restrict__ sx, const float* __restrict__ psi,
                                  const float* __restrict__ U, float* __restrict__ Q, float* __restrict__ grad,
                                  const SolverScalars* __restrict__ sc, double* __restrict__ part) {
    for (long u = blockIdx.x; u < vblocks_total(bi); u += gridDim.x) {
        int img, vb;
        long base, n;
        vblock_at(bi, u, img, vb, base, n);
        if (sc[img].zero_step) continue;  // block-uniform
        const float fs = sc[img].fstep, f2s = sc[img].f2step;
        double v[1] = {0.0};
        for (long t = (long)vb * blockDim.x + threadIdx.x; t < n; t += (long)kRedBlocks * blockDim.x) {
            const long e = base + t;
            const float q = fadd(Q[e], fmul(fs, sx[e]));
            const float g = fadd(grad[e], fadd(fmul(f2s, psi[e]), fmul(fs, 0.0f)));
            Q[e] = q;
            grad[e] = g;
            v[0] += (double)q * (double)fadd(g, U[e]);
        }
        vblock_store<1>(v, part + (long)img * kBPart, vb);
        __syncthreads();
    }
}

// qp_direction_kernel per image (run-time L): one-hot of the first arg-min
// of grad minus Q, and partials of U . sx.
__global__ void bqp_direction_kernel(BImages bi, const float* __restrict__ grad, const float* __restrict__ Q,
                                     const float* __restrict__ U, float* __restrict__ sx, double* __restrict__ part) {
    const int L = bi.L;
    for (long u = blockIdx.x; u < vblocks_total(bi); u += gridDim.x) {
        int img, vb;
        long base, n;
        vblock_at(bi, u, img, vb, base, n);
        const long p0 = bi.pix_off[img], np = bi.pix_off[img + 1] - p0;
        double v[1] = {0.0};
        for (long i = (long)vb * blockDim.x + threadIdx.x; i < np; i += (long)kRedBlocks * blockDim.x) {
            const float* g = grad + (p0 + i) * L;
            float best = g[0];
            int bk = 0;
            for (int k = 1; k < L; k++)
                if (g[k] < best) {
                    best = g[k];
                    bk = k;
                }
            for (int k = 0; k < L; k++) {
                const long e = (p0 + i) * L + k;
                const float s = fsub(k == bk ? 1.0f : 0.0f, Q[e]);
                sx[e] = s;
                v[0] += (double)U[e] * (double)s;
            }
        }
        vblock_store<1>(v, part + (long)img * kBPart, vb);
        __syncthreads();
    }
}

// qp_direction_tiled per image (L = 21): the image's row tiles of 32 pixels
// per warp, its blocks numbered image after image (the domain lt: tile_off
// as the base), one partial per block; the kernel loops over the live
// images' blocks.
template <int LC>
__global__ void __launch_bounds__(32 * kTileWarps)
    bqp_direction_tiled(Live lt, BImages bi, const float* __restrict__ grad, const float* __restrict__ Q,
                        const float* __restrict__ U, float* __restrict__ sx, double* __restrict__ part) {
    __shared__ float sm[kTileWarps][3][32 * LC];
    __shared__ double s32[32];
    const long total = live_total(lt, 0);
    for (long u = blockIdx.x; u < total; u += gridDim.x) {  // block-uniform
        long lb;
        const int img = live_locate(lt, u, lb);
        const long off = bi.pix_off[img], N = bi.pix_off[img + 1] - off;
        const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const long pix0 = (lb * kTileWarps + wib) * 32;
        double acc = 0.0;
        if (pix0 < N) {
            const int npix = (int)min(32L, N - pix0);
            float *Gt = sm[wib][0], *Qt = sm[wib][1], *Ut = sm[wib][2];
            tile_in<LC>(Gt, grad, off + pix0, npix, lane);
            tile_in<LC>(Qt, Q, off + pix0, npix, lane);
            tile_in<LC>(Ut, U, off + pix0, npix, lane);
            __syncwarp();
            const float* rg = Gt + lane * LC;
            float* rq = Qt + lane * LC;
            const float* ru = Ut + lane * LC;
            float best = rg[0];
            int bk = 0;
#pragma unroll
            for (int k = 1; k < LC; k++)
                if (rg[k] < best) {
                    best = rg[k];
                    bk = k;
                }
            const bool act = lane < npix;
#pragma unroll
            for (int k = 0; k < LC; k++) {
                const float s = fsub(k == bk ? 1.0f : 0.0f, rq[k]);
                rq[k] = s;
                if (act) acc += (double)ru[k] * (double)s;
            }
            __syncwarp();
            tile_out<LC>(Qt, sx, off + pix0, npix, lane);
        }
        const double tot = block_sum_any(acc, s32);
        if (threadIdx.x == 0) part[lt.base[img] + lb] = tot;
        __syncthreads();  // the tiles and s32 are rewritten next
    }
}

// finalize_sums_kernel per image (one block per image, one warp per value).
__global__ void bfinalize_sums_kernel(const double* __restrict__ part, int nv, int dst, const int* __restrict__ done,
                                      SolverScalars* sc) {
    const int img = blockIdx.x, j = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (done[img] || j >= nv) return;
    const double* p = part + (long)img * kBPart + (long)j * kRedBlocks;
    double s = 0.0;
    int b = lane;
    for (; b + 7 * 32 < kRedBlocks; b += 8 * 32) {
        double x[8];
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = p[b + i * 32];
#pragma unroll
        for (int i = 0; i < 8; i++) s += x[i];
    }
    for (; b < kRedBlocks; b += 32) s += p[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(kFullMask, s, o);
    if (lane == 0) sc[img].sums[dst + j] = s;
}

// finalize_large_kernel per image over its tile partials (1024 threads).
__global__ void bfinalize_large_kernel(const double* __restrict__ part, const int* __restrict__ tile_off, int dst,
                                       const int* __restrict__ done, SolverScalars* sc) {
    __shared__ double s[32];
    const int img = blockIdx.x;
    if (done[img]) return;  // block-uniform
    const double* p = part + tile_off[img];
    const int nblk = tile_off[img + 1] - tile_off[img];
    const int bd = blockDim.x;
    double v = 0.0;
    int b = threadIdx.x;
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
        sc[img].sums[dst] = t;
    }
}

// The single-thread QP scalar steps, one thread per image.
__global__ void bqp_init_energy_kernel(int B, SolverScalars* sc, int nterms, int max_iter) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    SolverScalars* s = sc + i;
    double e = 0.0;
    e += s->sums[0];
    e -= 0.0;
    for (int k = 0; k < nterms; k++) e += s->sums[1 + k];
    e += 0.0;
    e += s->sums[8];
    s->energy = e;
    s->old_energy = DBL_MAX;
    s->zero_step = 0;
    s->steps = 0;
    s->stop = max_iter > 0 ? 0 : !((s->old_energy - s->energy) > 100.0);
}

__global__ void bqp_step_kernel(int B, const int* __restrict__ done, SolverScalars* sc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B || done[i]) return;
    SolverScalars* s = sc + i;
    s->old_energy = s->energy;
    const double num = s->sums[0] + 2 * s->sums[1] + s->sums[3] + s->sums[4] + s->sums[5];
    const double denom = s->sums[2] + s->sums[6];
    double step = -num / (2 * denom);
    if (denom == 0 || num == 0) {
        s->zero_step = 1;
        s->stop = 1;
        return;
    }
    if (denom < 0) step = 1;
    s->fstep = (float)step;
    s->f2step = (float)(2 * step);
    s->steps++;
}

__global__ void bqp_energy_kernel(int B, const int* __restrict__ done, SolverScalars* sc, int max_iter) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B || done[i]) return;
    SolverScalars* s = sc + i;
    if (s->zero_step) return;
    const double e = s->sums[7] + s->sums[8];
    s->energy = e;
    if (max_iter > 0) s->stop = s->steps >= max_iter;
    else s->stop = !((s->old_energy - e) > 100.0);
}

// End of an iteration: images whose stop rule fired are done from now on;
// the loop goes on while any image runs, at most `cap` iterations per
// launch (the count kept in *chunk).  With a graph handle it sets the
// loop's condition, otherwise *running for the host.
__global__ void bqp_cond_kernel(int B, const SolverScalars* __restrict__ sc, int* __restrict__ done, int* chunk,
                                int cap, int* running, cudaGraphConditionalHandle h, int use_handle) {
    int any = 0;
    for (int i = threadIdx.x; i < B; i += blockDim.x) {
        const int st = sc[i].stop;
        done[i] = st;
        any |= !st;
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        const int c = ++*chunk;
        *running = any;
        if (use_handle) cudaGraphSetConditional(h, (any && c < cap) ? 1u : 0u);
    }
}

// a += coef * b over the whole batch (grad_y += 2 tmp, src/densecrf.cpp:380).
__global__ void badd_scaled_kernel(long n, float* __restrict__ a, const float* __restrict__ b, float coef) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) a[t] = fadd(a[t], fmul(coef, b[t]));
}

// The per-image work domains whose live prefixes an iteration needs.
constexpr int kMaxLiveDoms = 64;
struct LiveDoms {
    const long* base[kMaxLiveDoms];  // B + 1 unit offsets per image
    long* pre[kMaxLiveDoms];         // out: live prefix, live count + 1 entries
    int n;
};

// Exclusive block-wide scan of one long per thread (blockDim.x a multiple of
// 32, at most 1024); returns the thread's prefix, *total the block's sum.
__device__ __forceinline__ long block_excl_scan(long x, long* s32, long& total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    long v = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long y = __shfl_up_sync(kFullMask, v, o);
        if (lane >= o) v += y;
    }
    if (lane == 31) s32[w] = v;
    __syncthreads();
    if (w == 0) {
        long t = lane < nw ? s32[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long y = __shfl_up_sync(kFullMask, t, o);
            if (lane >= o) t += y;
        }
        if (lane < nw) s32[lane] = t;  // inclusive warp totals
    }
    __syncthreads();
    total = s32[nw - 1];
    const long r = v - x + (w > 0 ? s32[w - 1] : 0);
    __syncthreads();  // s32 is reused by the next scan
    return r;
}

// Start of a lockstep iteration, one block: the images still running, in
// ascending order (live_img, *live_n), and each domain's live prefix.
__global__ void live_build_kernel(int B, const int* __restrict__ done, int* __restrict__ live_n,
                                  int* __restrict__ live_img, LiveDoms doms) {
    __shared__ long s32[32];
    long carry = 0;
    for (int c0 = 0; c0 < B; c0 += blockDim.x) {
        const int i = c0 + threadIdx.x;
        const long f = (i < B && !done[i]) ? 1 : 0;
        long tot;
        const long pos = carry + block_excl_scan(f, s32, tot);
        if (f) live_img[pos] = i;
        carry += tot;
    }
    const int n = (int)carry;
    if (threadIdx.x == 0) *live_n = n;
    __syncthreads();  // live_img complete
    for (int d = 0; d < doms.n; d++) {
        const long* base = doms.base[d];
        long* pre = doms.pre[d];
        long acc = 0;
        for (int r0 = 0; r0 < n; r0 += blockDim.x) {
            const int r = r0 + threadIdx.x;
            long cnt = 0;
            if (r < n) {
                const int img = live_img[r];
                cnt = base[img + 1] - base[img];
            }
            long tot;
            const long p = acc + block_excl_scan(cnt, s32, tot);
            if (r < n) pre[r] = p;
            acc += tot;
        }
        if (threadIdx.x == 0) pre[n] = acc;
    }
}

}  // namespace

Batch::Batch(int n, const int* widths, const int* heights, int L_) : B(n), L(L_) {
    require(n >= 1 && n <= 4096, DCRF_E_ARG, "batch: image count must be in [1, 4096]");
    require(L_ >= 1 && L_ <= kLMax, DCRF_E_ARG, "batch: label count must be in [1, 64]");
    W.assign(widths, widths + n);
    H.assign(heights, heights + n);
    pix_off.assign(n + 1, 0);
    for (int i = 0; i < n; i++) {
        require(W[i] > 0 && H[i] > 0, DCRF_E_ARG, "batch: image sizes must be positive");
        pix_off[i + 1] = pix_off[i] + (long)W[i] * H[i];
    }
    Ntot = pix_off[n];
    require(Ntot * (long)L < (1L << 31), DCRF_E_ARG, "batch: too many pixel-labels");
    DCRF_CUDA(cudaGetDevice(&device));
    DCRF_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    long* po = d_pix_off.ensure(n + 1);
    DCRF_CUDA(cudaMemcpyAsync(po, pix_off.data(), sizeof(long) * (n + 1), cudaMemcpyHostToDevice, stream));
    partials.ensure((size_t)kRedBlocks * 2);
    DCRF_CUDA(cudaStreamSynchronize(stream));
}

Batch::~Batch() {
    if (stream) cudaStreamSynchronize(stream);
    if (bqp_graph) cudaGraphExecDestroy(bqp_graph);
    terms.clear();
    if (stream) cudaStreamDestroy(stream);
}

// Term t's lattice over all images: every image's own lattice, built from
// the term's features, concatenated (Lattice::concat).
void Batch::build_lattice(Term& t) {
    t.lat = std::make_unique<Lattice>();
    t.lat->stream = stream;
    std::vector<std::unique_ptr<Lattice>> parts;
    std::vector<const Lattice*> views;
    for (int i = 0; i < B; i++) {
        auto p = std::make_unique<Lattice>();
        p->stream = stream;
        p->build(t.feat.get() + pix_off[i] * t.d, t.d, W[i] * H[i]);
        views.push_back(p.get());
        parts.push_back(std::move(p));
    }
    t.lat->concat(views);
}  // the per-image lattices are released here

void Batch::ensure_lattices() {
    for (auto& t : terms)
        if (!t->lat) build_lattice(*t);
}

void Batch::add_term(const float* d_features, int d, float w) {
    weights_gen++;
    ensure_lattices();
    auto t = std::make_unique<Term>();
    DCRF_CUDA(cudaMemcpyAsync(t->feat.ensure((size_t)Ntot * d), d_features, sizeof(float) * Ntot * d,
                              cudaMemcpyDeviceToDevice, stream));
    t->d = d;
    build_lattice(*t);
    t->w = w;
    float* nrm = t->norm.ensure(Ntot);
    launch(bfill_kernel, ceil_div(Ntot, 256), 256, 0, stream, Ntot, 1.0f, nrm);
    SliceEpilogue ep;
    t->lat->compute(nrm, nrm, 1, false, ep);
    launch(bnorm_kernel, ceil_div(Ntot, 256), 256, 0, stream, Ntot, nrm);
    DCRF_LAUNCH_CHECK();
    terms.push_back(std::move(t));
}

void Batch::apply(int k, float* out, const float* in, const float* base, float coef, bool zero_base) {
    ensure_lattices();
    Term& t = *terms[k];
    SliceEpilogue ep;
    ep.potts = true;
    ep.norm = t.norm.get();
    ep.scale = -t.w;
    ep.base = base;
    ep.coef = coef;
    ep.zero_base = zero_base;
    t.lat->compute(out, in, L, false, ep, t.norm.get());
}

void Batch::unary_init(float* Q) {
    require(has_unary, DCRF_E_STATE, "unary_init: no unary energy set");
    with_lc(L, [&](auto lc) {
        constexpr int LC = decltype(lc)::value;
        launch(unary_init_kernel<LC>, ceil_div(Ntot, 128), 128, 0, stream, (int)Ntot, L, unary.get(), Q);
    });
    DCRF_LAUNCH_CHECK();
}

// Batched QP in lockstep: every Frank-Wolfe iteration of every image that
// is still running, one launch per step over all images -- the filters over
// the terms' concatenated lattices, the per-pixel and per-image scalar steps
// over the concatenated arrays -- with the loop on the device: a CUDA graph
// whose `while` node repeats the iteration until no image runs (or kQpChunk
// iterations, after which the host relaunches it).  Each image's reductions
// use its own single-image decomposition and scalars, so its output, step
// count and energy are those of its own solve (src/densecrf.cpp:340-442).
int Batch::qp(const float* init, float* out, int max_iter, int* steps, double* energies) {
    require(has_unary, DCRF_E_STATE, "qp: no unary energy set");
    ensure_lattices();
    const long NL = Ntot * L;
    float* Q = out;  // iterated in place
    float* grad = buf(0);
    float* sx = buf(1);
    float* psi = buf(2);
    float* tmp = buf(3);
    const int nt = (int)terms.size();
    SolverScalars* sc = bsc.ensure(B);
    int* done = bdone.ensure(B);
    int* flags = bflags.ensure(2);  // [0] iterations of the current launch, [1] some image runs
    double* part = bpart.ensure((size_t)B * kBPart);
    const bool tiled = L == 21;
    if (tiled && btiles == 0) {  // row-tile blocks of the direction kernel, image after image
        std::vector<int> toff(B + 1, 0);
        std::vector<long> tbase(B + 1, 0);
        for (int i = 0; i < B; i++) {
            const int tg = ceil_div(ceil_div((int)(pix_off[i + 1] - pix_off[i]), 32), kTileWarps);
            toff[i + 1] = toff[i] + tg;
            tbase[i + 1] = toff[i + 1];
        }
        btiles = toff[B];
        DCRF_CUDA(cudaMemcpyAsync(btile_off.ensure(B + 1), toff.data(), sizeof(int) * (B + 1), cudaMemcpyHostToDevice,
                                  stream));
        DCRF_CUDA(cudaMemcpyAsync(btile_base.ensure(B + 1), tbase.data(), sizeof(long) * (B + 1),
                                  cudaMemcpyHostToDevice, stream));
        DCRF_CUDA(cudaStreamSynchronize(stream));  // the host vectors are the copies' sources
    }
    double* part_dir = tiled ? bpart_dir.ensure(btiles) : nullptr;
    // The live images and each domain's live prefix, rebuilt at the start of
    // every iteration: kDomains domains per term (its lattice's lists,
    // vertices, slice tiles and pixels), then the direction kernel's tiles.
    const int nt_l = (int)terms.size();
    require(nt_l * Lattice::kDomains + 1 <= kMaxLiveDoms, DCRF_E_ARG, "batch qp: too many pairwise terms");
    int* live_buf = blive.ensure(B + 1);
    const int* live_n = live_buf;
    const int* live_img = live_buf + 1;
    long* lpre = blive_pre.ensure((size_t)(nt_l * Lattice::kDomains + 1) * (B + 1));
    LiveDoms doms{};
    for (int k = 0; k < nt_l; k++) {
        Lattice& lat = *terms[k]->lat;
        lat.prepare_live(L);
        for (int dm = 0; dm < Lattice::kDomains; dm++) {
            doms.base[doms.n] = lat.dom_base.get() + (long)dm * (B + 1);
            doms.pre[doms.n++] = lpre + (long)(k * Lattice::kDomains + dm) * (B + 1);
        }
    }
    long* tile_pre = lpre + (long)nt_l * Lattice::kDomains * (B + 1);
    if (tiled) {
        doms.base[doms.n] = btile_base.get();
        doms.pre[doms.n++] = tile_pre;
    }
    const BImages all{d_pix_off.get(), nullptr, nullptr, B, L};
    const BImages live{d_pix_off.get(), live_n, live_img, B, L};
    const Live ltiles{live_n, live_img, tiled ? btile_base.get() : nullptr, tile_pre};
    // Grids of the live loops: a few waves of the device, not the batch.
    const int vgrid = std::min(B, 16) * kRedBlocks;
    const int tgrid = std::max(1, std::min(btiles, sm_count() * 2 * (2048 / (32 * kTileWarps))));
    const int sb = ceil_div(B, 128);

    if (Q != init) DCRF_CUDA(cudaMemcpyAsync(Q, init, sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
    DCRF_CUDA(cudaMemcpyAsync(grad, unary.get(), sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
    DCRF_CUDA(cudaMemsetAsync(sc, 0, sizeof(SolverScalars) * B, stream));
    DCRF_CUDA(cudaMemsetAsync(done, 0, sizeof(int) * B, stream));
    // grad_y = unary + sum_k 2 A_k Q; the energy terms Q . A_k Q (the same applies)
    for (int k = 0; k < nt; k++) {
        apply(k, tmp, Q);
        launch(badd_scaled_kernel, ceil_div(NL, 256), 256, 0, stream, NL, grad, tmp, 2.0f);
        launch(bdot_kernel, B * kRedBlocks, kRedThreads, 0, stream, all, Q, tmp, part);
        launch(bfinalize_sums_kernel, B, 32, 0, stream, part, 1, 1 + k, done, sc);
    }
    launch(bdot_kernel, B * kRedBlocks, kRedThreads, 0, stream, all, unary.get(), Q, part);
    launch(bfinalize_sums_kernel, B, 32, 0, stream, part, 1, 0, done, sc);
    launch(bqp_init_energy_kernel, sb, 128, 0, stream, B, sc, nt, max_iter);
    // a NaN or infinity in Q or the unaries
    DCRF_CUDA(cudaMemsetAsync(&sc[0].numeric, 0, sizeof(int), stream));
    launch(nonfinite_kernel, nonfinite_grid(NL), 256, 0, stream, NL, (const float*)Q, (const float*)unary.get(), sc);
    launch(bqp_cond_kernel, 1, 256, 0, stream, B, (const SolverScalars*)sc, done, flags, 1 << 30, flags + 1,
           cudaGraphConditionalHandle{}, 0);
    DCRF_LAUNCH_CHECK();
    int hf[2] = {0, 0};
    int numeric = 0;
    DCRF_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, stream));
    DCRF_CUDA(cudaMemcpyAsync(&numeric, &sc[0].numeric, sizeof(int), cudaMemcpyDeviceToHost, stream));
    DCRF_CUDA(cudaStreamSynchronize(stream));
    if (numeric & 1) throw Error(DCRF_E_NUMERIC, "qp: the initial Q or the unary energy holds a NaN or an infinity");

    // One Frank-Wolfe iteration of every running image (src/densecrf.cpp:389-436)
    // and the loop test.
    for (auto& t : terms) {  // finished images: no filter work
        Lattice& lat = *t->lat;
        lat.live_n = live_n;
        lat.live_img = live_img;
    }
    for (int k = 0; k < nt_l; k++) terms[k]->lat->live_pre = lpre + (long)k * Lattice::kDomains * (B + 1);
    auto iteration = [&](bool graph, cudaGraphConditionalHandle h) {
        launch(live_build_kernel, 1, 256, 0, stream, B, (const int*)done, live_buf, live_buf + 1, doms);
        if (tiled) {
            launch(bqp_direction_tiled<21>, tgrid, 32 * kTileWarps, 0, stream, ltiles, live, (const float*)grad,
                   (const float*)Q, (const float*)unary.get(), sx, part_dir);
            launch(bfinalize_large_kernel, B, 1024, 0, stream, (const double*)part_dir, (const int*)btile_off.get(), 0,
                   (const int*)done, sc);
        } else {
            launch(bqp_direction_kernel, vgrid, kRedThreads, 0, stream, live, (const float*)grad,
                   (const float*)Q, (const float*)unary.get(), sx, part);
            launch(bfinalize_sums_kernel, B, 32, 0, stream, (const double*)part, 1, 0, (const int*)done, sc);
        }
        for (int k = 0; k < nt; k++) apply(k, psi, sx, k == 0 ? nullptr : psi, 1.0f, k == 0);
        if (nt == 0) DCRF_CUDA(cudaMemsetAsync(psi, 0, sizeof(float) * NL, stream));
        launch(bdots2_kernel, vgrid, kRedThreads, 0, stream, live, (const float*)Q, (const float*)sx,
               (const float*)psi, part);
        launch(bfinalize_sums_kernel, B, 64, 0, stream, (const double*)part, 2, 1, (const int*)done, sc);
        launch(bqp_step_kernel, sb, 128, 0, stream, B, (const int*)done, sc);
        launch(bqp_update_kernel, vgrid, kRedThreads, 0, stream, live, (const float*)sx, (const float*)psi,
               (const float*)unary.get(), Q, grad, (const SolverScalars*)sc, part);
        launch(bfinalize_sums_kernel, B, 32, 0, stream, (const double*)part, 1, 7, (const int*)done, sc);
        launch(bqp_energy_kernel, sb, 128, 0, stream, B, (const int*)done, sc, max_iter);
        launch(bqp_cond_kernel, 1, 256, 0, stream, B, (const SolverScalars*)sc, done, flags, kQpChunk, flags + 1, h,
               graph ? 1 : 0);
    };
    std::vector<const void*> key = {Q, grad, sx, psi, unary.get(), sc, done, part, part_dir,
                                    (const void*)(uintptr_t)max_iter, (const void*)(uintptr_t)weights_gen};
    key.push_back(live_buf);
    key.push_back(lpre);
    for (auto& t : terms) {
        key.push_back(t->lat->va.get());
        key.push_back(t->lat->vb.get());
        key.push_back(t->lat.get());
        key.push_back((const void*)(uintptr_t)t->lat->dom_tile);
    }
    auto detach = [&] {
        for (auto& t : terms) {
            t->lat->live_n = nullptr;
            t->lat->live_img = nullptr;
            t->lat->live_pre = nullptr;
        }
    };
    int guard = 0;
    try {
        while (hf[1]) {
            require(++guard < (1 << 26), DCRF_E_TIMEOUT, "batch qp: iteration cap reached");
            if (bqp_graph && key == bqp_key) {
                DCRF_CUDA(cudaMemsetAsync(flags, 0, sizeof(int), stream));
                DCRF_CUDA(cudaGraphLaunch(bqp_graph, stream));
            } else {
                iteration(false, cudaGraphConditionalHandle{});
                DCRF_LAUNCH_CHECK();
            }
            DCRF_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, stream));
            DCRF_CUDA(cudaStreamSynchronize(stream));
            if (hf[1] && !(bqp_graph && key == bqp_key) && !bqp_graph_failed && graphs_enabled()) {
                try {
                    build_bqp_graph(iteration, flags);
                    bqp_key = key;
                } catch (const Error&) {
                    if (bqp_graph) cudaGraphExecDestroy(bqp_graph);
                    bqp_graph = nullptr;
                    bqp_graph_failed = true;  // this device or driver cannot run it: stay eager
                }
            }
        }
    } catch (...) {
        detach();
        throw;
    }
    detach();
    std::vector<SolverScalars> hs(B);
    DCRF_CUDA(cudaMemcpyAsync(hs.data(), sc, sizeof(SolverScalars) * B, cudaMemcpyDeviceToHost, stream));
    DCRF_CUDA(cudaStreamSynchronize(stream));
    int most = 0;
    for (int i = 0; i < B; i++) {
        if (steps) steps[i] = hs[i].steps;
        if (energies) energies[i] = hs[i].energy;
        most = std::max(most, hs[i].steps);
    }
    return most;
}

// The lockstep iteration as a graph: a `while` node whose body is one
// iteration, its condition set by bqp_cond_kernel (some image runs and fewer
// than kQpChunk iterations ran in this launch).  The body is checked to end
// in that kernel, so the loop cannot run on without its test.
template <typename F>
void Batch::build_bqp_graph(F&& iteration, int* flags) {
    std::lock_guard<std::recursive_mutex> cap(capture_mutex());
    if (bqp_graph) cudaGraphExecDestroy(bqp_graph);
    bqp_graph = nullptr;
    cudaGraph_t g = nullptr;
    DCRF_CUDA(cudaGraphCreate(&g, 0));
    bool capturing = false;
    try {
        cudaGraphConditionalHandle h;
        DCRF_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t wn;
        DCRF_CUDA(cudaGraphAddNode(&wn, g, nullptr, 0, &np));
        const unsigned long long k0 = g_kernel_launches.load();
        DCRF_CUDA(cudaStreamBeginCaptureToGraph(stream, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                cudaStreamCaptureModeRelaxed));
        capturing = true;
        iteration(true, h);
        cudaGraph_t bo = nullptr;
        capturing = false;
        DCRF_CUDA(cudaStreamEndCapture(stream, &bo));
        const unsigned long long captured = g_kernel_launches.load() - k0;
        g_kernel_launches.fetch_sub(captured);
        require(captured >= 2, DCRF_E_STATE, "batch qp: unexpected loop body");
        bqp_graph_kernels = captured;
        DCRF_CUDA(cudaGraphInstantiate(&bqp_graph, g, 0));
        cudaGraphDestroy(g);
    } catch (...) {
        cudaGraph_t junk = nullptr;
        if (capturing) cudaStreamEndCapture(stream, &junk);
        cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
    }
    (void)flags;
}

void Batch::set_weight(int k, float w) {
    require(k >= 0 && k < (int)terms.size(), DCRF_E_ARG, "pairwise term index out of range");
    terms[k]->w = w;
    weights_gen++;
}

// out = base + scale * n o K(n o in), K transposed (blur axes reversed) when
// `transpose`.  The blur of one axis is symmetric, so K^T is the filter with
// the axes in reverse order.
static void normalised_filter(Term& t, int L, float* out, const float* in, float scale, const float* base,
                              bool transpose) {
    SliceEpilogue ep;
    ep.potts = true;
    ep.norm = t.norm.get();
    ep.scale = scale;
    ep.base = base;
    ep.coef = 1.0f;
    t.lat->compute(out, in, L, transpose, ep, t.norm.get());
}

void Batch::set_checkpointing(int every, bool recompute_lat) {
    require(every >= 1 && every <= 1000, DCRF_E_ARG, "checkpointing: interval must be in [1, 1000]");
    ck_every = every;
    recompute_lattice = recompute_lat;
    mf_T = -1;  // the checkpoints of an earlier forward pass are laid out differently
}

size_t Batch::meanfield_state_bytes(int T) const {
    const size_t arr = sizeof(float) * (size_t)Ntot * L;
    const size_t slots = (size_t)(T / ck_every + 1 + (T % ck_every ? 1 : 0));
    const size_t seg = ck_every > 1 ? (size_t)std::min(ck_every - 1, std::max(T - 1, 0)) : 0;
    return (slots + seg) * arr;
}

// Q_{t+1} = softmax(-U + sum_k w_k K~_k Q_t) from q into qn.
void Batch::mf_iteration(const float* q, float* qn, const float* negU, float* logits) {
    const long NL = Ntot * L;
    const int nt = (int)terms.size();
    if (nt == 0) DCRF_CUDA(cudaMemcpyAsync(logits, negU, sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
    for (int k = 0; k < nt; k++)  // logits = -U + sum_k w_k K~_k Q
        normalised_filter(*terms[k], L, logits, q, terms[k]->w, k == 0 ? negU : logits, false);
    with_lc(L, [&](auto lc) {
        constexpr int LC = decltype(lc)::value;
        launch(softmax_kernel<LC>, ceil_div(Ntot, 128), 128, 0, stream, Ntot, L, logits, qn);
    });
}

// Forward pass.  Q_t is kept for t % ck_every == 0 and for t = T (the
// backward pass recomputes the others); with ck_every = 1 every iterate is
// kept.  In the recompute_lattice mode the lattices are released at the end
// and rebuilt by the backward pass.
void Batch::meanfield(int iterations, float* Q) {
    require(has_unary, DCRF_E_STATE, "meanfield: no unary energy set");
    require(iterations >= 0 && iterations <= 1000, DCRF_E_ARG, "meanfield: iterations must be in [0, 1000]");
    ensure_lattices();
    const long NL = Ntot * L;
    mf_T = iterations;
    const int slots = iterations / ck_every + 1 + (iterations % ck_every ? 1 : 0);
    float* ck = mf_ck.ensure((size_t)slots * NL);
    float* negU = buf(4);
    float* logits = buf(5);
    float* x[2] = {mf_x0.ensure(ck_every > 1 ? NL : 1), mf_x1.ensure(ck_every > 1 ? NL : 1)};
    launch(negate_kernel, ceil_div(NL, 256), 256, 0, stream, NL, unary.get(), negU);
    unary_init(ck);  // Q_0 = softmax(-U)
    const float* q = ck;
    for (int it = 0; it < iterations; it++) {
        float* qn = ck_stored(it + 1) ? ck + (size_t)ck_slot(it + 1) * NL : x[it & 1];
        mf_iteration(q, qn, negU, logits);
        q = qn;
    }
    DCRF_LAUNCH_CHECK();
    if (Q) DCRF_CUDA(cudaMemcpyAsync(Q, ck + (size_t)ck_slot(iterations) * NL, sizeof(float) * NL,
                                     cudaMemcpyDeviceToDevice, stream));
    if (recompute_lattice) {
        DCRF_CUDA(cudaStreamSynchronize(stream));
        for (auto& t : terms) t->lat.reset();
    }
}

void Batch::meanfield_backward(const float* grad_Q, float* grad_U, double* grad_w) {
    require(mf_T >= 0, DCRF_E_STATE, "meanfield_backward: no meanfield() to differentiate");
    ensure_lattices();  // rebuilt here in the recompute_lattice mode
    const long NL = Ntot * L;
    const int nt = (int)terms.size();
    const float* ck = mf_ck.get();
    float* g = mf_g0.ensure(NL);
    float* gn = mf_g1.ensure(NL);
    float* ga = mf_ga.ensure(NL);
    float* m = mf_m.ensure(NL);
    float* seg = ck_every > 1 ? mf_seg.ensure((size_t)(ck_every - 1) * NL) : nullptr;
    float* negU = buf(4);
    float* logits = buf(5);
    double* dw = mf_dw.ensure(std::max(nt, 1));
    double* part = partials.get();
    if (ck_every > 1) launch(negate_kernel, ceil_div(NL, 256), 256, 0, stream, NL, unary.get(), negU);
    DCRF_CUDA(cudaMemcpyAsync(g, grad_Q, sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
    if (nt) DCRF_CUDA(cudaMemsetAsync(dw, 0, sizeof(double) * nt, stream));
    auto softmax_bwd = [&](const float* q, int first) {
        with_lc(L, [&](auto lc) {
            constexpr int LC = decltype(lc)::value;
            launch(softmax_bwd_kernel<LC>, ceil_div(Ntot, 128), 128, 0, stream, Ntot, L, q, g, ga, grad_U, first);
        });
    };
    // Q_t: a checkpoint, or an iterate of the current segment recomputed
    // from the checkpoint at its start.
    int seg_s = -1;
    auto iterate = [&](int t) -> const float* {
        if (ck_stored(t)) return ck + (size_t)ck_slot(t) * NL;
        return seg + (size_t)(t - seg_s - 1) * NL;
    };
    for (int it = mf_T - 1; it >= 0; it--) {
        const int s = (it / ck_every) * ck_every;
        if (ck_every > 1 && s != seg_s) {  // recompute Q_{s+1} .. Q_{e-1} of this segment
            seg_s = s;
            const int e = std::min(s + ck_every, mf_T);
            for (int t = s; t + 1 < e; t++)
                mf_iteration(iterate(t), seg + (size_t)(t - s) * NL, negU, logits);
        }
        const float* q0 = iterate(it);
        const float* q1 = iterate(it + 1);
        softmax_bwd(q1, it == mf_T - 1);  // ga = dL/dlogits_t; grad_U -= ga
        for (int k = 0; k < nt; k++) {
            // dL/dw_k += <ga, K~_k Q_t>, the message recomputed from the iterate
            normalised_filter(*terms[k], L, m, q0, 1.0f, nullptr, false);
            launch(dot_kernel, kRedBlocks, kRedThreads, 0, stream, NL, ga, m, part);
            launch(accumulate_total_kernel, 1, 32, 0, stream, part, kRedBlocks, dw + k);
            // dL/dQ_t = sum_k w_k K~_k^T ga
            normalised_filter(*terms[k], L, gn, ga, terms[k]->w, k == 0 ? nullptr : gn, true);
        }
        if (nt == 0) DCRF_CUDA(cudaMemsetAsync(gn, 0, sizeof(float) * NL, stream));
        std::swap(g, gn);
    }
    softmax_bwd(ck, mf_T == 0);  // Q_0 = softmax(-U)
    DCRF_LAUNCH_CHECK();
    if (nt) DCRF_CUDA(cudaMemcpyAsync(grad_w, dw, sizeof(double) * nt, cudaMemcpyDeviceToHost, stream));
    DCRF_CUDA(cudaStreamSynchronize(stream));
    if (recompute_lattice)
        for (auto& t : terms) t->lat.reset();
}

}  // namespace dcrf
