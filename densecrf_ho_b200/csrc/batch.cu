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

#include <atomic>
#include <exception>
#include <mutex>
#include <thread>
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
    img.clear();
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
    img.clear();  // rebuilt with the new term at the next QP
    qp_warm = false;
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

// One Frank-Wolfe iteration for every image that has not stopped, then the
// count of images still running, copied to pinned host memory.
// Batch QP: every image's own single-image solve (Model::qp, whose
// Frank-Wolfe loop is a device-side graph loop), from up to kQpThreads host
// threads so that the images' solves overlap on their own streams; a solve
// of one image alone leaves SMs idle (one-block reductions and step kernels,
// the longest splat lists' chains), which the other images' kernels fill.
// Each image's output, step count and energy are those of its single-image
// solve, bit for bit.  The per-image models are built at the first solve
// from the features each term was added with, and kept.
void Batch::ensure_image_models() {
    if ((int)img.size() == B) return;
    img.clear();
    DCRF_CUDA(cudaStreamSynchronize(stream));  // the terms' features were copied on this stream
    for (int i = 0; i < B; i++) {
        auto m = std::make_unique<Model>(W[i], H[i], L);
        for (const auto& t : terms) {
            m->add_term(t->feat.get() + pix_off[i] * t->d, t->d, t->w);
            m->sync();
        }
        img.push_back(std::move(m));
    }
    img_unary_gen = ~0ull;
}

int Batch::qp(const float* init, float* out, int max_iter, int* steps, double* energies) {
    require(has_unary, DCRF_E_STATE, "qp: no unary energy set");
    ensure_image_models();
    if (img_unary_gen != unary_gen) {  // each image's slice of the unaries
        for (int i = 0; i < B; i++) {
            Model& m = *img[i];
            const size_t n = (size_t)(pix_off[i + 1] - pix_off[i]) * L;
            DCRF_CUDA(cudaMemcpyAsync(m.unary.ensure(n), unary.get() + pix_off[i] * L, sizeof(float) * n,
                                      cudaMemcpyDeviceToDevice, stream));
            m.has_unary = true;
            m.logit_F = 0;
            m.gen++;
        }
        img_unary_gen = unary_gen;
        qp_warm = false;  // the models changed: their graphs are captured again
    }
    // the images' streams start after the batch stream's work (the unaries, init)
    DCRF_CUDA(cudaStreamSynchronize(stream));
    std::vector<int> st(B, 0);
    std::vector<double> en(B, 0.0);
    // A solve that sizes buffers or captures its graph (the first one for an
    // output buffer, max_iter and model state) runs on this thread, image
    // after image: allocation and capture stay out of the concurrent phase.
    if (!(qp_warm && out == warm_out && max_iter == warm_max_iter)) {
        for (int i = 0; i < B; i++)
            st[i] = img[i]->qp(init + pix_off[i] * L, out + pix_off[i] * L, max_iter, &en[i]);
        qp_warm = true;
        warm_out = out;
        warm_max_iter = max_iter;
        int most = 0;
        for (int i = 0; i < B; i++) {
            if (steps) steps[i] = st[i];
            if (energies) energies[i] = en[i];
            most = std::max(most, st[i]);
        }
        return most;
    }
    std::atomic<int> next{0};
    std::exception_ptr err = nullptr;
    std::mutex emu;
    auto worker = [&]() {
        cudaSetDevice(device);
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= B) break;
            try {
                st[i] = img[i]->qp(init + pix_off[i] * L, out + pix_off[i] * L, max_iter, &en[i]);
            } catch (...) {
                std::lock_guard<std::mutex> lk(emu);
                if (!err) err = std::current_exception();
                next.store(B);
            }
        }
    };
    const int nth = std::min(B, kQpThreads);
    std::vector<std::thread> pool;
    try {
        for (int t = 1; t < nth; t++) pool.emplace_back(worker);
    } catch (...) {  // fewer threads than asked for: the ones running finish the images
    }
    worker();
    for (auto& th : pool) th.join();
    if (err) std::rethrow_exception(err);
    int most = 0;
    for (int i = 0; i < B; i++) {
        if (steps) steps[i] = st[i];
        if (energies) energies[i] = en[i];
        most = std::max(most, st[i]);
    }
    return most;
}

void Batch::set_weight(int k, float w) {
    require(k >= 0 && k < (int)terms.size(), DCRF_E_ARG, "pairwise term index out of range");
    terms[k]->w = w;
    for (auto& m : img) m->set_compat(k, kPotts, &w);  // the per-image models' QP graphs are rebuilt
    qp_warm = false;
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
