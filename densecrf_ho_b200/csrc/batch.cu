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
#include "model_kernels.cuh"

namespace dcrf {

namespace {

__device__ __forceinline__ long img_begin(const long* pix_off, int img) { return pix_off[img]; }
// Row-tile blocks of an image of n pixels (32 pixels per warp, kTileWarps warps).
__host__ __device__ __forceinline__ int tile_blocks(int n) { return ((n + 31) / 32 + kTileWarps - 1) / kTileWarps; }
__device__ __forceinline__ int img_pixels(const long* pix_off, int img) {
    return (int)(pix_off[img + 1] - pix_off[img]);
}

// Start of an iteration: images that stopped are frozen for all of it.
// The filters read the same flags from done_flags (Lattice::skip_done).
__global__ void bqp_begin_kernel(int B, SolverScalars* sc, int* __restrict__ done_flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < B) done_flags[i] = sc[i].done = sc[i].stop;
}

// Number of images still iterating, for the host's loop test.
// Loop condition of the batched QP graph: some image still running, at most
// `cap` iterations per launch (counted in active[1]).
__global__ void bqp_cond_kernel(int* active, int cap, cudaGraphConditionalHandle h) {
    const int c = ++active[1];
    cudaGraphSetConditional(h, (active[0] > 0 && c < cap) ? 1u : 0u);
}

__global__ void bqp_count_kernel(int B, const SolverScalars* __restrict__ sc, int* __restrict__ active) {
    __shared__ int s;
    if (threadIdx.x == 0) s = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < B; i += blockDim.x)
        if (!sc[i].stop) atomicAdd(&s, 1);
    __syncthreads();
    if (threadIdx.x == 0) *active = s;
}

// Per-image finalisation in the order of finalize_sums_kernel (one warp per
// value over nblk partials) and finalize_large_kernel (one 1024-thread block).
__global__ void bfinalize_sums_kernel(const double* __restrict__ partials, int nblk, int nv, int dst,
                                      SolverScalars* sc) {
    const int img = blockIdx.x;
    if (sc[img].done) return;
    const int j = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (j >= nv) return;
    const double* p = partials + (long)img * nv * nblk;
    double s = 0.0;
    for (int b = lane; b < nblk; b += 32) s += p[(long)j * nblk + b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(kFullMask, s, o);
    if (lane == 0) sc[img].sums[dst + j] = s;
}

__global__ void bfinalize_tiles_kernel(const double* __restrict__ partials, int max_tiles,
                                       const long* __restrict__ pix_off, int dst, SolverScalars* sc) {
    __shared__ double s[32];
    const int img = blockIdx.x;
    if (sc[img].done) return;
    const int nblk = tile_blocks(img_pixels(pix_off, img));
    const double* p = partials + (long)img * max_tiles;
    double v = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) v += p[b];
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

// a . b over each image (dot_kernel per image): grid (kRedBlocks, B).
__global__ void bdot_kernel(const long* __restrict__ pix_off, int L, const float* __restrict__ a,
                            const float* __restrict__ b, const SolverScalars* __restrict__ sc,
                            double* __restrict__ partials) {
    const int img = blockIdx.y;
    if (sc[img].done) return;
    const long e0 = img_begin(pix_off, img) * L, n = (long)img_pixels(pix_off, img) * L;
    double v[1] = {0.0};
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
        v[0] += (double)a[e0 + t] * (double)b[e0 + t];
    block_sum_store<1>(v, partials + (long)img * gridDim.x);
}

// Q . psi and sx . psi per image (dots2_kernel).
__global__ void bdots2_kernel(const long* __restrict__ pix_off, int L, const float* __restrict__ a,
                              const float* __restrict__ b, const float* __restrict__ c,
                              const SolverScalars* __restrict__ sc, double* __restrict__ partials) {
    const int img = blockIdx.y;
    if (sc[img].done) return;
    const long e0 = img_begin(pix_off, img) * L, n = (long)img_pixels(pix_off, img) * L;
    double v[2] = {0.0, 0.0};
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        const double cc = c[e0 + t];
        v[0] += (double)a[e0 + t] * cc;
        v[1] += (double)b[e0 + t] * cc;
    }
    block_sum_store<2>(v, partials + (long)img * 2 * gridDim.x);
}

// Conditional gradient (qp_direction_tiled / qp_direction_kernel per image).
template <int LC>
__global__ void __launch_bounds__(32 * kTileWarps)
    bqp_direction_tiled(const long* __restrict__ pix_off, int max_tiles, const float* __restrict__ grad,
                        const float* __restrict__ Q, const float* __restrict__ U, float* __restrict__ sx,
                        const SolverScalars* __restrict__ sc, double* __restrict__ partials) {
    __shared__ float sm[kTileWarps][3][32 * LC];
    __shared__ double s32[32];
    const int img = blockIdx.y;
    const int N = img_pixels(pix_off, img);
    if (sc[img].done || (int)blockIdx.x >= tile_blocks(N)) return;  // block-uniform
    const long base = img_begin(pix_off, img) * LC;
    grad += base;
    Q += base;
    U += base;
    sx += base;
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
    if (threadIdx.x == 0) partials[(long)img * max_tiles + blockIdx.x] = tot;
}

template <int LC>
__global__ void bqp_direction_kernel(const long* __restrict__ pix_off, int Lrt, const float* __restrict__ grad,
                                     const float* __restrict__ Q, const float* __restrict__ U,
                                     float* __restrict__ sx, const SolverScalars* __restrict__ sc,
                                     double* __restrict__ partials) {
    const int L = LC ? LC : Lrt;
    const int img = blockIdx.y;
    if (sc[img].done) return;
    const int N = img_pixels(pix_off, img);
    const long base = img_begin(pix_off, img) * L;
    double v[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float* g = grad + base + (long)i * L;
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
                const long e = base + (long)i * L + k;
                const float s = fsub(k == bi ? 1.0f : 0.0f, Q[e]);
                sx[e] = s;
                v[0] += (double)U[e] * (double)s;
            }
    }
    block_sum_store<1>(v, partials + (long)img * gridDim.x);
}

// Line search per image (qp_step_kernel).
__global__ void bqp_step_kernel(int B, SolverScalars* scs) {
    const int img = blockIdx.x * blockDim.x + threadIdx.x;
    if (img >= B) return;
    SolverScalars* sc = scs + img;
    if (sc->done) return;
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

// Q += step sx; grad += 2 step psi; partial sums of Q . (grad + U) (qp_update_kernel).
__global__ void bqp_update_kernel(const long* __restrict__ pix_off, int L, const float* __restrict__ sx,
                                  const float* __restrict__ psi, const float* __restrict__ U, float* __restrict__ Q,
                                  float* __restrict__ grad, const SolverScalars* __restrict__ scs,
                                  double* __restrict__ partials) {
    const int img = blockIdx.y;
    const SolverScalars* sc = scs + img;
    if (sc->done || sc->zero_step) return;
    const long e0 = img_begin(pix_off, img) * L, n = (long)img_pixels(pix_off, img) * L;
    const float fs = sc->fstep, f2s = sc->f2step;
    double v[1] = {0.0};
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        const long e = e0 + t;
        const float q = fadd(Q[e], fmul(fs, sx[e]));
        const float g = fadd(grad[e], fadd(fmul(f2s, psi[e]), fmul(fs, 0.0f)));
        Q[e] = q;
        grad[e] = g;
        v[0] += (double)q * (double)fadd(g, U[e]);
    }
    block_sum_store<1>(v, partials + (long)img * gridDim.x);
}

// Energy and stop rule per image (qp_energy_kernel).
__global__ void bqp_energy_kernel(int B, SolverScalars* scs, int max_iter) {
    const int img = blockIdx.x * blockDim.x + threadIdx.x;
    if (img >= B) return;
    SolverScalars* sc = scs + img;
    if (sc->done || sc->zero_step) return;
    const double e = sc->sums[7] + sc->sums[8];
    sc->energy = e;
    if (max_iter > 0) sc->stop = sc->steps >= max_iter;
    else sc->stop = !((sc->old_energy - e) > 100.0);
}

__global__ void bqp_init_energy_kernel(int B, SolverScalars* scs, int nterms, int max_iter) {
    const int img = blockIdx.x * blockDim.x + threadIdx.x;
    if (img >= B) return;
    SolverScalars* sc = scs + img;
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
    sc->done = 0;
    sc->stop = max_iter > 0 ? 0 : !((DBL_MAX - e) > 100.0);
}

__global__ void badd_scaled_kernel(long n, float* __restrict__ a, const float* __restrict__ b, float coef) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) a[t] = fadd(a[t], fmul(coef, b[t]));
}

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
    const float sf = (float)s;
#pragma unroll
    for (int k = 0; k < PixVec<LC>::S; k++)
        if (k < L) {
            const long e = i * L + k;
            const float v = Q[e] * (g[e] - sf);
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
        max_tiles = std::max(max_tiles, ceil_div(ceil_div(W[i] * H[i], 32), kTileWarps));
    }
    Ntot = pix_off[n];
    require(Ntot * (long)L < (1L << 31), DCRF_E_ARG, "batch: too many pixel-labels");
    DCRF_CUDA(cudaGetDevice(&device));
    DCRF_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    DCRF_CUDA(cudaMallocHost(&h_scal, sizeof(SolverScalars) * B));
    DCRF_CUDA(cudaMallocHost(&h_active, 2 * sizeof(int)));
    scal.ensure(B);
    d_active.ensure(2);
    DCRF_CUDA(cudaMemsetAsync(d_done.ensure(B), 0, sizeof(int) * B, stream));
    long* po = d_pix_off.ensure(n + 1);
    DCRF_CUDA(cudaMemcpyAsync(po, pix_off.data(), sizeof(long) * (n + 1), cudaMemcpyHostToDevice, stream));
    partials.ensure((size_t)B * std::max<long>((long)kRedBlocks * 2, max_tiles));
    DCRF_CUDA(cudaStreamSynchronize(stream));
}

Batch::~Batch() {
    if (stream) cudaStreamSynchronize(stream);
    drop_graph();
    terms.clear();
    if (h_scal) cudaFreeHost(h_scal);
    if (h_active) cudaFreeHost(h_active);
    if (stream) cudaStreamDestroy(stream);
}

void Batch::drop_graph() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    graph_q = nullptr;
    graph_max_iter = -1;
}

void Batch::add_term(const float* d_features, int d, float w) {
    drop_graph();
    auto t = std::make_unique<Term>();
    t->lat = std::make_unique<Lattice>();
    t->lat->stream = stream;
    {
        std::vector<std::unique_ptr<Lattice>> parts;
        std::vector<const Lattice*> views;
        for (int i = 0; i < B; i++) {
            auto p = std::make_unique<Lattice>();
            p->stream = stream;
            p->build(d_features + pix_off[i] * d, d, W[i] * H[i]);
            views.push_back(p.get());
            parts.push_back(std::move(p));
        }
        t->lat->concat(views);
    }  // the per-image lattices are released here
    t->lat->skip_done = d_done.get();  // all zero outside qp()
    t->w = w;
    t->d = d;
    float* nrm = t->norm.ensure(Ntot);
    launch(bfill_kernel, ceil_div(Ntot, 256), 256, 0, stream, Ntot, 1.0f, nrm);
    SliceEpilogue ep;
    t->lat->compute(nrm, nrm, 1, false, ep);
    launch(bnorm_kernel, ceil_div(Ntot, 256), 256, 0, stream, Ntot, nrm);
    DCRF_LAUNCH_CHECK();
    terms.push_back(std::move(t));
}

void Batch::apply(int k, float* out, const float* in, const float* base, float coef, bool zero_base) {
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

// One Frank-Wolfe iteration for every image that has not stopped, then the
// count of images still running, copied to pinned host memory.
void Batch::qp_iteration(float* Q, int max_iter, bool copy_active) {
    float* grad = buf(0);
    float* sx = buf(1);
    float* psi = buf(2);
    SolverScalars* sc = scal.get();
    double* part = partials.get();
    const long* po = d_pix_off.get();
    const int nt = (int)terms.size();
    const int sgrid = ceil_div(B, 256);
    launch(bqp_begin_kernel, sgrid, 256, 0, stream, B, sc, d_done.get());
    with_lc(L, [&](auto lc) {
        constexpr int LC = decltype(lc)::value;
        if constexpr (LC > 0) {
            launch(bqp_direction_tiled<LC>, dim3(max_tiles, B), 32 * kTileWarps, 0, stream, po, max_tiles, grad, Q,
                   unary.get(), sx, sc, part);
            launch(bfinalize_tiles_kernel, B, 1024, 0, stream, part, max_tiles, po, 0, sc);
        } else {
            launch(bqp_direction_kernel<LC>, dim3(kRedBlocks, B), kRedThreads, 0, stream, po, L, grad, Q,
                   unary.get(), sx, sc, part);
            launch(bfinalize_sums_kernel, B, 32, 0, stream, part, kRedBlocks, 1, 0, sc);
        }
    });
    for (int k = 0; k < nt; k++) {
        if (k == 0) apply(k, psi, sx, nullptr, 1.0f, true);
        else apply(k, psi, sx, psi, 1.0f, false);
    }
    launch(bdots2_kernel, dim3(kRedBlocks, B), kRedThreads, 0, stream, po, L, Q, sx, psi, sc, part);
    launch(bfinalize_sums_kernel, B, 64, 0, stream, part, kRedBlocks, 2, 1, sc);
    launch(bqp_step_kernel, sgrid, 256, 0, stream, B, sc);
    launch(bqp_update_kernel, dim3(kRedBlocks, B), kRedThreads, 0, stream, po, L, sx, psi, unary.get(), Q, grad,
           sc, part);
    launch(bfinalize_sums_kernel, B, 32, 0, stream, part, kRedBlocks, 1, 7, sc);
    launch(bqp_energy_kernel, sgrid, 256, 0, stream, B, sc, max_iter);
    launch(bqp_count_kernel, 1, 256, 0, stream, B, sc, d_active.get());
    if (copy_active)
        DCRF_CUDA(cudaMemcpyAsync(h_active, d_active.get(), sizeof(int), cudaMemcpyDeviceToHost, stream));
}

int Batch::qp(const float* init, float* out, int max_iter, int* steps, double* energies) {
    require(has_unary, DCRF_E_STATE, "qp: no unary energy set");
    const long NL = Ntot * L;
    float* Q = out;
    float* grad = buf(0);
    float* tmp = buf(3);
    buf(1);
    buf(2);
    if (Q != init) DCRF_CUDA(cudaMemcpyAsync(Q, init, sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
    DCRF_CUDA(cudaMemcpyAsync(grad, unary.get(), sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
    DCRF_CUDA(cudaMemsetAsync(scal.get(), 0, sizeof(SolverScalars) * B, stream));
    DCRF_CUDA(cudaMemsetAsync(d_done.get(), 0, sizeof(int) * B, stream));
    SolverScalars* sc = scal.get();
    double* part = partials.get();
    const long* po = d_pix_off.get();
    const int nt = (int)terms.size();
    for (int k = 0; k < nt; k++) {
        apply(k, tmp, Q);
        launch(badd_scaled_kernel, ceil_div(NL, 256), 256, 0, stream, NL, grad, tmp, 2.0f);
        launch(bdot_kernel, dim3(kRedBlocks, B), kRedThreads, 0, stream, po, L, Q, tmp, sc, part);
        launch(bfinalize_sums_kernel, B, 32, 0, stream, part, kRedBlocks, 1, 1 + k, sc);
    }
    launch(bdot_kernel, dim3(kRedBlocks, B), kRedThreads, 0, stream, po, L, unary.get(), Q, sc, part);
    launch(bfinalize_sums_kernel, B, 32, 0, stream, part, kRedBlocks, 1, 0, sc);
    launch(bqp_init_energy_kernel, ceil_div(B, 256), 256, 0, stream, B, sc, nt, max_iter);
    launch(bqp_count_kernel, 1, 256, 0, stream, B, sc, d_active.get());
    DCRF_CUDA(cudaMemcpyAsync(h_active, d_active.get(), sizeof(int), cudaMemcpyDeviceToHost, stream));
    DCRF_LAUNCH_CHECK();
    DCRF_CUDA(cudaStreamSynchronize(stream));
    int guard = 0;
    bool eager = false;
    while (*h_active > 0) {
        require(++guard < (1 << 26), DCRF_E_TIMEOUT, "qp: iteration cap reached");
        if (graph && graph_q == Q && graph_max_iter == max_iter) {
            DCRF_CUDA(cudaGraphLaunch(graph, stream));
            DCRF_CUDA(cudaMemcpyAsync(h_active, d_active.get(), 2 * sizeof(int), cudaMemcpyDeviceToHost, stream));
            DCRF_CUDA(cudaStreamSynchronize(stream));
            g_kernel_launches.fetch_add(graph_kernels * (unsigned long long)h_active[1]);
            continue;
        }
        if (!eager || !graphs_enabled()) {
            // The first iteration runs eagerly: it sizes every buffer that an
            // iteration touches, so none is allocated during the capture.
            qp_iteration(Q, max_iter);
            DCRF_LAUNCH_CHECK();
            DCRF_CUDA(cudaStreamSynchronize(stream));
            eager = true;
            continue;
        }
        // Capture the loop: [iteration counter = 0] -> while (running) { iteration }.
        drop_graph();
        cudaGraph_t g = nullptr;
        DCRF_CUDA(cudaGraphCreate(&g, 0));
        bool capturing = false;
        try {
            cudaGraphConditionalHandle h;
            DCRF_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
            cudaMemsetParams mp = {};
            mp.dst = d_active.get() + 1;
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
            qp_iteration(Q, max_iter, false);
            launch(bqp_cond_kernel, 1, 1, 0, stream, d_active.get(), kQpChunk, h);
            cudaGraph_t bo = nullptr;
            capturing = false;
            DCRF_CUDA(cudaStreamEndCapture(stream, &bo));
            graph_kernels = g_kernel_launches.load() - k0;
            g_kernel_launches.fetch_sub(graph_kernels);  // counted per iteration when the graph runs
            require(graph_kernels >= 2, DCRF_E_STATE, "qp: unexpected loop body");
            DCRF_CUDA(cudaGraphInstantiate(&graph, g, 0));
            cudaGraphDestroy(g);
        } catch (...) {
            cudaGraph_t junk = nullptr;
            if (capturing) cudaStreamEndCapture(stream, &junk);
            cudaGraphDestroy(g);
            graph = nullptr;
            throw;
        }
        graph_q = Q;
        graph_max_iter = max_iter;
    }
    DCRF_CUDA(cudaMemcpyAsync(h_scal, scal.get(), sizeof(SolverScalars) * B, cudaMemcpyDeviceToHost, stream));
    DCRF_CUDA(cudaMemsetAsync(d_done.get(), 0, sizeof(int) * B, stream));
    DCRF_CUDA(cudaStreamSynchronize(stream));
    int most = 0;
    for (int i = 0; i < B; i++) {
        if (steps) steps[i] = h_scal[i].steps;
        if (energies) energies[i] = h_scal[i].energy;
        most = std::max(most, h_scal[i].steps);
    }
    return most;
}

// ---- mean-field and its adjoint --------------------------------------------

void Batch::set_weight(int k, float w) {
    require(k >= 0 && k < (int)terms.size(), DCRF_E_ARG, "pairwise term index out of range");
    terms[k]->w = w;
    drop_graph();  // the captured QP iteration holds the old weight
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

void Batch::meanfield(int iterations, float* Q) {
    require(has_unary, DCRF_E_STATE, "meanfield: no unary energy set");
    require(iterations >= 0 && iterations <= 1000, DCRF_E_ARG, "meanfield: iterations must be in [0, 1000]");
    const long NL = Ntot * L;
    float* ck = mf_ck.ensure((size_t)(iterations + 1) * NL);
    float* negU = buf(4);
    float* logits = buf(5);
    launch(negate_kernel, ceil_div(NL, 256), 256, 0, stream, NL, unary.get(), negU);
    unary_init(ck);  // Q_0 = softmax(-U)
    const int nt = (int)terms.size();
    for (int it = 0; it < iterations; it++) {
        const float* q = ck + (size_t)it * NL;
        if (nt == 0)
            DCRF_CUDA(cudaMemcpyAsync(logits, negU, sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
        for (int k = 0; k < nt; k++)  // logits = -U + sum_k w_k K~_k Q
            normalised_filter(*terms[k], L, logits, q, terms[k]->w, k == 0 ? negU : logits, false);
        with_lc(L, [&](auto lc) {
            constexpr int LC = decltype(lc)::value;
            launch(softmax_kernel<LC>, ceil_div(Ntot, 128), 128, 0, stream, Ntot, L, logits,
                   ck + (size_t)(it + 1) * NL);
        });
    }
    DCRF_LAUNCH_CHECK();
    if (Q) DCRF_CUDA(cudaMemcpyAsync(Q, ck + (size_t)iterations * NL, sizeof(float) * NL,
                                     cudaMemcpyDeviceToDevice, stream));
    mf_T = iterations;
}

void Batch::meanfield_backward(const float* grad_Q, float* grad_U, double* grad_w) {
    require(mf_T >= 0, DCRF_E_STATE, "meanfield_backward: no meanfield() to differentiate");
    const long NL = Ntot * L;
    const int nt = (int)terms.size();
    const float* ck = mf_ck.get();
    float* g = mf_g0.ensure(NL);
    float* gn = mf_g1.ensure(NL);
    float* ga = mf_ga.ensure(NL);
    float* m = mf_m.ensure(NL);
    double* dw = mf_dw.ensure(std::max(nt, 1));
    double* part = partials.get();
    DCRF_CUDA(cudaMemcpyAsync(g, grad_Q, sizeof(float) * NL, cudaMemcpyDeviceToDevice, stream));
    if (nt) DCRF_CUDA(cudaMemsetAsync(dw, 0, sizeof(double) * nt, stream));
    auto softmax_bwd = [&](const float* q, int first) {
        with_lc(L, [&](auto lc) {
            constexpr int LC = decltype(lc)::value;
            launch(softmax_bwd_kernel<LC>, ceil_div(Ntot, 128), 128, 0, stream, Ntot, L, q, g, ga, grad_U, first);
        });
    };
    for (int it = mf_T - 1; it >= 0; it--) {
        const float* q0 = ck + (size_t)it * NL;
        const float* q1 = ck + (size_t)(it + 1) * NL;
        softmax_bwd(q1, it == mf_T - 1);  // ga = dL/dlogits_t; grad_U -= ga
        for (int k = 0; k < nt; k++) {
            // dL/dw_k += <ga, K~_k Q_t>, the message recomputed from the checkpoint
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
}

}  // namespace dcrf
