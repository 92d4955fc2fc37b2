// DenseCRF2D on the device: model set-up, pairwise application, energies.
//
// Per-pixel arithmetic follows the reference's operation order (Eigen 3.2
// expression evaluation, SSE2, no FMA) so per-pixel results are identical;
// global FP64 sums are deterministic fixed-order trees whose order differs
// from Eigen's sequential packet sums (differences are O(1e-16) relative).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "reduce.cuh"
#include "model_kernels.cuh"

namespace dcrf {

int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

namespace {

__global__ void fill_kernel(long n, float v, float* x) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) x[t] = v;
}

// norm = 1 / sqrt(K 1 + 1e-20) (symmetric) or 1 / (K 1 + 1e-20), in double
// like src/pairwise.cpp:44-56.
__global__ void norm_kernel(int N, float* x, int symmetric) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double s = dadd((double)x[i], 1e-20);
    x[i] = (float)(symmetric ? 1.0 / sqrt(s) : 1.0 / s);
}

// f'(i, :) = diag(p) f(i, :) (DIAG_KERNEL) or P f(i, :) with P d x d
// column-major, summed over the inner index in order (FULL_KERNEL).
__global__ void scale_features_kernel(int N, int d, const float* __restrict__ f, const float* __restrict__ p,
                                      int full, float* __restrict__ out) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)N * d) return;
    const long i = t / d;
    const int r = (int)(t - i * d);
    if (!full) {
        out[t] = fmul(p[r], f[t]);
        return;
    }
    float acc = fmul(p[r], f[i * d]);
    for (int c = 1; c < d; c++) acc = fadd(acc, fmul(p[r + (long)c * d], f[i * d + c]));
    out[t] = acc;
}

// ---- kernel-parameter gradient (src/pairwise.cpp:90-122, 170-181, 402-407) --

// out(i, l) = in(i, l) * s(i)  (Eigen: M * v.asDiagonal()); s == null: out = c * in.
__global__ void scale_cols_kernel(long n, int L, const float* __restrict__ in, const float* __restrict__ s, float c,
                                  float* __restrict__ out) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    out[t] = s ? fmul(in[t], s[t / L]) : fmul(c, in[t]);
}

// X = (0.5 (a o fb + fa o b)) * n^3 per column (featureGradient, symmetric).
__global__ void sym_grad_input_kernel(long n, int L, const float* __restrict__ a, const float* __restrict__ fb,
                                      const float* __restrict__ fa, const float* __restrict__ b,
                                      const float* __restrict__ nrm, float* __restrict__ X) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float ni = nrm[t / L];
    const float n3 = fmul(fmul(ni, ni), ni);
    X[t] = fmul(fmul(fadd(fmul(a[t], fb[t]), fmul(fa[t], b[t])), 0.5f), n3);
}

// X = (x o y) n^2 per column (featureGradient, NORMALIZE_AFTER with x = a,
// y = K(b); NORMALIZE_BEFORE with x = K^T(a), y = b).
__global__ void one_sided_grad_input_kernel(long n, int L, const float* __restrict__ x, const float* __restrict__ y,
                                            const float* __restrict__ nrm, float* __restrict__ X) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float ni = nrm[t / L];
    X[t] = fmul(fmul(x[t], y[t]), fmul(ni, ni));
}

// DenseKernel::gradient's sums over pixels in FP64 (block partials, then a
// fixed-order finish), fg = -r + g (fg = g without r):
// DIAG (full = 0): output j = sum_i f(i, j) fg(i, j);
// FULL (full = 1): output j + k d = sum_i fg(i, j) f(i, k)  (fg f^T).
__global__ void feature_grad_partial_kernel(int N, int d, int full, const float* __restrict__ f,
                                            const float* __restrict__ r, const float* __restrict__ g,
                                            double* __restrict__ part) {
    __shared__ double sm[256];
    const int o = blockIdx.y;
    const int j = full ? o % d : o, kf = full ? o / d : o;
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const long e = (long)i * d;
        const float fg = r ? fadd(-r[e + j], g[e + j]) : g[e + j];
        acc += (double)fmul(f[e + kf], fg);
    }
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sm[threadIdx.x] += sm[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(long)o * gridDim.x + blockIdx.x] = sm[0];
}

// -(b o x).sum() in FP64 partials (PottsCompatibility::gradient).
__global__ void neg_dot_partial_kernel(long n, const float* __restrict__ b, const float* __restrict__ x,
                                       double* __restrict__ part) {
    __shared__ double sm[256];
    double acc = 0.0;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
        acc += (double)fmul(b[t], x[t]);
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = -sm[0];
}

// MatrixCompatibility::apply (src/labelcompatibility.cpp:102-104): out(:, i)
// = W raw(:, i), W column-major L x L, the product summed over m in order;
// then the epilogue's base: out = base + coef * (W raw).
__global__ void matrix_compat_kernel(long n, int L, const float* __restrict__ W, const float* __restrict__ raw,
                                     const float* __restrict__ base, float coef, int zero_base, float* out) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const long i = t / L;
    const int l = (int)(t - i * L);
    const float* x = raw + i * L;
    float r = fmul(W[l], x[0]);
    for (int m = 1; m < L; m++) r = fadd(r, fmul(W[l + (long)m * L], x[m]));
    if (base) r = fadd(base[t], fmul(coef, r));
    else if (zero_base) r = fadd(0.0f, fmul(coef, r));
    out[t] = r;
}

// DiagonalCompatibility::apply: out(l, i) = w_l in(l, i).
__global__ void scale_labels_kernel(long n, int L, const float* __restrict__ in, const float* __restrict__ w,
                                    float* __restrict__ out) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = fmul(w[t % L], in[t]);
}

// part[p * gridDim.x + blk]: this block's share of sum_i b(r, i) x(c, i) for
// pair p = c * L + r (r = c = p when diag_only).
__global__ void label_outer_partial_kernel(int N, int L, const float* __restrict__ b, const float* __restrict__ x,
                                           int diag_only, double* __restrict__ part) {
    __shared__ double sm[256];
    const int p = blockIdx.y;
    const int c = diag_only ? p : p / L, r = diag_only ? p : p - (p / L) * L;
    double acc = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
        acc += (double)fmul(b[i * L + r], x[i * L + c]);
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(long)p * gridDim.x + blockIdx.x] = sm[0];
}

// LogisticUnaryEnergy::get: U(l, i) = sum_f W(l, f) F(f, i), summed over f in
// order (Eigen's GEMM blocks the sum differently: float tolerance).
__global__ void logistic_unary_kernel(long n, int L, int F, const float* __restrict__ W,
                                      const float* __restrict__ feat, float* __restrict__ out) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const long i = t / L;
    const int l = (int)(t - i * L);
    const float* f = feat + i * F;
    float r = fmul(W[l], f[0]);
    for (int c = 1; c < F; c++) r = fadd(r, fmul(W[l + (long)c * L], f[c]));
    out[t] = r;
}

// part[p * gridDim.x + blk]: this block's share of sum_i b(l, i) F(c, i) for
// p = c * L + l (LogisticUnaryEnergy::gradient, b F^T).
__global__ void logistic_grad_partial_kernel(int N, int L, int F, const float* __restrict__ b,
                                             const float* __restrict__ feat, double* __restrict__ part) {
    __shared__ double sm[256];
    const int p = blockIdx.y;
    const int c = p / L, l = p - c * L;
    double acc = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
        acc += (double)fmul(b[i * L + l], feat[i * F + c]);
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(long)p * gridDim.x + blockIdx.x] = sm[0];
}

__global__ void fill_ones_kernel(long n, float* x) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) x[t] = 1.0f;
}

}  // namespace

Model::Model(int W_, int H_, int L_) : W(W_), H(H_), N(W_ * H_), L(L_) {
    DCRF_CUDA(cudaGetDevice(&device));
    DCRF_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    DCRF_CUDA(cudaMallocHost(&h_scal, sizeof(SolverScalars)));
    scal.ensure(1);
    // per-block partials: fixed-grid reductions, and the per-pixel / per-element
    // kernels that fold a reduction in (two values per block)
    partials.ensure(std::max<size_t>((size_t)kRedBlocks * 16, 2 * (size_t)slice_grid((long)N * L) + 64));
}

Model::~Model() {
    if (stream) cudaStreamSynchronize(stream);
    if (side) {
        cudaStreamSynchronize(side);
        cudaEventDestroy(ev_side_fork);
        cudaEventDestroy(ev_side_join);
        cudaStreamDestroy(side);
    }
    drop_qp_graph();
    if (gstream) cudaStreamDestroy(gstream);
    terms.clear();
    if (h_scal) cudaFreeHost(h_scal);
    if (stream) cudaStreamDestroy(stream);
}

void Model::fetch_scalars() {
    DCRF_CUDA(cudaMemcpyAsync(h_scal, scal.get(), sizeof(SolverScalars), cudaMemcpyDeviceToHost, stream));
    sync();
}

void Model::add_term(const float* d_features, int d, float w) {
    gen++;  // a captured QP graph may hold what this changes
    auto t = std::make_unique<Term>();
    t->lat = std::make_unique<Lattice>();
    t->lat->stream = stream;
    t->lat->build(d_features, d, N);
    t->w = w;
    t->d = d;
    float* tf = t->feat.ensure((size_t)N * d);
    DCRF_CUDA(cudaMemcpyAsync(tf, d_features, sizeof(float) * (size_t)N * d, cudaMemcpyDeviceToDevice, stream));
    t->kparams.assign(d, 1.0f);
    compute_norm(*t);
    terms.push_back(std::move(t));
}

// DenseKernel::initLattice's normalisation (src/pairwise.cpp:40-57): K 1 on
// the term's lattice, then per NormalizationType.
void Model::compute_norm(Term& t) {
    if (t.ntype == kNoNorm) return;
    float* nrm = t.norm.ensure(N);
    launch(fill_kernel, ceil_div(N, 256), 256, 0, stream, N, 1.0f, nrm);
    SliceEpilogue ep;  // plain output
    t.lat->compute(nrm, nrm, 1, false, ep);
    launch(norm_kernel, ceil_div(N, 256), 256, 0, stream, N, nrm, (int)(t.ntype == kNormSymmetric));
    DCRF_LAUNCH_CHECK();
}

void Model::set_kernel(int k, int ktype, int ntype) {
    gen++;  // a captured QP graph may hold what this changes
    require(k >= 0 && k < (int)terms.size(), DCRF_E_ARG, "pairwise term index out of range");
    require(ktype >= kConstKernel && ktype <= kFullKernel, DCRF_E_ARG, "unknown kernel type");
    require(ntype >= kNoNorm && ntype <= kNormSymmetric, DCRF_E_ARG, "unknown normalization type");
    Term& t = *terms[k];
    t.ktype = ktype;
    if (ktype == kDiagKernel) t.kparams.assign(t.d, 1.0f);
    else if (ktype == kFullKernel) {
        t.kparams.assign((size_t)t.d * t.d, 0.0f);
        for (int j = 0; j < t.d; j++) t.kparams[(size_t)j * t.d + j] = 1.0f;
    } else t.kparams.clear();
    if (ntype != t.ntype) {
        t.ntype = ntype;
        compute_norm(t);
    }
    sync();
}

int Model::kernel_parameters(int k, float* out) const {
    require(k >= 0 && k < (int)terms.size(), DCRF_E_ARG, "pairwise term index out of range");
    const Term& t = *terms[k];
    if (out) std::copy(t.kparams.begin(), t.kparams.end(), out);
    return (int)t.kparams.size();
}

// DenseKernel::setParameters (src/pairwise.cpp:157-168): the lattice is
// rebuilt on diag(p) f or P f; the unnormalised twin keeps the lattice of the
// features the term was added with, as the reference's no_norm_pairwise_
// does.  CONST_KERNEL has no parameters (no-op).
void Model::set_kernel_parameters(int k, const float* p) {
    gen++;
    require(k >= 0 && k < (int)terms.size(), DCRF_E_ARG, "pairwise term index out of range");
    Term& t = *terms[k];
    if (t.ktype == kConstKernel) return;
    const bool full = t.ktype == kFullKernel;
    const size_t np = full ? (size_t)t.d * t.d : (size_t)t.d;
    t.kparams.assign(p, p + np);
    DevBuf<float> dp, sf;
    DCRF_CUDA(cudaMemcpyAsync(dp.ensure(np), p, sizeof(float) * np, cudaMemcpyHostToDevice, stream));
    float* scaled = sf.ensure((size_t)N * t.d);
    launch(scale_features_kernel, ceil_div((long)N * t.d, 256), 256, 0, stream, N, t.d, (const float*)t.feat.get(),
           (const float*)dp.get(), (int)full, scaled);
    DCRF_LAUNCH_CHECK();
    auto lat = std::make_unique<Lattice>();
    lat->stream = stream;
    lat->build(scaled, t.d, N);
    if (!t.twin) t.twin = std::move(t.lat);
    t.lat = std::move(lat);
    compute_norm(t);
    sync();
}

// pairwise_[k]->kernelGradient(b, Q) (src/pairwise.cpp:402-407, 95-122,
// 170-181): lbl = compatibility(Q), then DenseKernel::featureGradient(a = b,
// lbl) with G = the lattice's gradient and n the term's norm:
//   NO_NORMALIZATION  fg = G(a, lbl)
//   SYMMETRIC         fg = -G(X, 1) + G(a n, lbl n), X = 0.5 (a o K(lbl n) + K^T(a n) o lbl) n^3
//   AFTER             fg = -G(X, 1) + G(a n, lbl),   X = (a o K(lbl)) n^2
//   BEFORE            fg = -G(X, 1) + G(a, lbl n),   X = (K^T(a) o lbl) n^2
// and DenseKernel::gradient: DIAG_KERNEL sum_i f(i, j) fg(i, j) per
// dimension j, FULL_KERNEL fg f^T (d x d, column-major), both over the
// features the term was added with; FP64 sums over pixels, rounded to float
// (the reference sums in float).
int Model::kernel_gradient(int k, const float* b, const float* Q, float* out) {
    Term& t = *terms[k];
    if (t.ktype == kConstKernel) return 0;  // DenseKernel::gradient: no parameters
    Lattice& lat = *t.lat;
    const long NL = (long)N * L;
    const int d = t.d, g = ceil_div(NL, 256);
    float *lbl = buf(8), *bn = buf(9), *ln = buf(10), *fa = buf(11), *fb = buf(12), *X = buf(13);
    float* ones = this->b[7].ensure((size_t)NL);
    float* r = this->b[14].ensure((size_t)N * d);
    float* gg = this->b[15].ensure((size_t)N * d);
    const float* nrm = t.norm.get();
    if (t.compat == kPotts)
        launch(scale_cols_kernel, g, 256, 0, stream, NL, L, Q, (const float*)nullptr, -t.w, lbl);
    else if (t.compat == kDiagonal)
        launch(scale_labels_kernel, g, 256, 0, stream, NL, L, Q, (const float*)t.cw.get(), lbl);
    else
        launch(matrix_compat_kernel, g, 256, 0, stream, NL, L, (const float*)t.cw.get(), Q, (const float*)nullptr,
               1.0f, 0, lbl);
    SliceEpilogue plain;
    const bool has_r = t.ntype != kNoNorm;
    if (t.ntype == kNoNorm) {
        lat.gradient(gg, b, lbl, L);
    } else {
        if (t.ntype == kNormSymmetric) {
            launch(scale_cols_kernel, g, 256, 0, stream, NL, L, b, nrm, 1.0f, bn);
            launch(scale_cols_kernel, g, 256, 0, stream, NL, L, lbl, nrm, 1.0f, ln);
            lat.compute(fa, bn, L, true, plain);
            lat.compute(fb, ln, L, false, plain);
            launch(sym_grad_input_kernel, g, 256, 0, stream, NL, L, b, fb, fa, lbl, nrm, X);
        } else if (t.ntype == kNormAfter) {
            lat.compute(fb, lbl, L, false, plain);
            launch(one_sided_grad_input_kernel, g, 256, 0, stream, NL, L, b, (const float*)fb, nrm, X);
        } else {  // kNormBefore
            lat.compute(fa, b, L, true, plain);
            launch(one_sided_grad_input_kernel, g, 256, 0, stream, NL, L, (const float*)fa, lbl, nrm, X);
        }
        launch(fill_ones_kernel, g, 256, 0, stream, NL, ones);
        lat.gradient(r, X, ones, L);
        if (t.ntype == kNormSymmetric) {
            lat.gradient(gg, bn, ln, L);
        } else if (t.ntype == kNormAfter) {
            launch(scale_cols_kernel, g, 256, 0, stream, NL, L, b, nrm, 1.0f, bn);
            lat.gradient(gg, bn, lbl, L);
        } else {
            launch(scale_cols_kernel, g, 256, 0, stream, NL, L, lbl, nrm, 1.0f, ln);
            lat.gradient(gg, b, ln, L);
        }
    }
    const int nb = 64, nout = t.ktype == kDiagKernel ? d : d * d;
    double* part = partials.ensure((size_t)nb * nout);
    launch(feature_grad_partial_kernel, dim3(nb, nout), 256, 0, stream, N, d, (int)(t.ktype == kFullKernel),
           (const float*)t.feat.get(), has_r ? (const float*)r : nullptr, (const float*)gg, part);
    DCRF_LAUNCH_CHECK();
    std::vector<double> h((size_t)nb * nout);
    DCRF_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream));
    sync();
    for (int j = 0; j < nout; j++) {
        double s = 0.0;
        for (int i = 0; i < nb; i++) s += h[(size_t)j * nb + i];
        out[j] = (float)s;
    }
    return nout;
}

// pairwise_[k]->gradient(b, Q) (src/pairwise.cpp:390-395): the
// compatibility's gradient at fq = n K(n Q) (src/labelcompatibility.cpp):
// Potts -(b o fq).sum() (:72-76), Diagonal (b o fq).rowwise().sum() (:94-96),
// Matrix g = b fq^T folded to its upper triangle, g(i,j) + g(j,i) off the
// diagonal (:123-129).  FP64 sums over pixels, rounded to float.
int Model::compat_gradient(int k, const float* b, const float* Q, float* out) {
    require(k >= 0 && k < (int)terms.size(), DCRF_E_ARG, "pairwise term index out of range");
    Term& t = *terms[k];
    const long NL = (long)N * L;
    float* fq = buf(8);
    SliceEpilogue ep;
    ep.potts = true;
    ep.norm = t.post_norm();
    ep.scale = 1.0f;
    t.lat->compute(fq, Q, L, false, ep, t.pre_norm());
    double* part = partials.get();
    if (t.compat == kPotts) {
        const int nb = 128;
        launch(neg_dot_partial_kernel, nb, 256, 0, stream, NL, b, (const float*)fq, part);
        DCRF_LAUNCH_CHECK();
        std::vector<double> h(nb);
        DCRF_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double) * nb, cudaMemcpyDeviceToHost, stream));
        sync();
        double s = 0.0;
        for (int i = 0; i < nb; i++) s += h[i];
        out[0] = (float)s;
        return 1;
    }
    const bool diag = t.compat == kDiagonal;
    const int pairs = diag ? L : L * L;
    const int nb = 32;
    part = partials.ensure((size_t)nb * pairs);
    launch(label_outer_partial_kernel, dim3(nb, pairs), 256, 0, stream, N, L, b, (const float*)fq, (int)diag, part);
    DCRF_LAUNCH_CHECK();
    std::vector<double> h((size_t)nb * pairs);
    DCRF_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream));
    sync();
    std::vector<double> g(pairs, 0.0);
    for (int p = 0; p < pairs; p++)
        for (int i = 0; i < nb; i++) g[p] += h[(size_t)p * nb + i];
    if (diag) {
        for (int l = 0; l < L; l++) out[l] = (float)g[l];
        return L;
    }
    int n = 0;  // g(r, c) at r * L + c: sum_p b(r, p) fq(c, p)
    for (int c = 0; c < L; c++)
        for (int r = c; r < L; r++, n++) out[n] = (float)(g[(size_t)c * L + r] + (r != c ? g[(size_t)r * L + c] : 0.0));
    return n;
}

// setUnaryEnergy(new LogisticUnaryEnergy(lw, lf)) (src/unary.cpp:47-52).
void Model::set_unary_logistic(const float* lw, const float* lf, int F) {
    require(F >= 1, DCRF_E_ARG, "logistic unary: F must be >= 1");
    logit_F = F;
    DCRF_CUDA(cudaMemcpyAsync(logit_f.ensure((size_t)F * N), lf, sizeof(float) * F * N, cudaMemcpyHostToDevice,
                              stream));
    set_unary_parameters(lw);
}

// LogisticUnaryEnergy::setParameters (:58-63); the unary is recomputed, as
// get() recomputes it at every use.
void Model::set_unary_parameters(const float* lw) {
    gen++;  // a captured QP graph may hold what this changes
    if (logit_F == 0) return;  // UnaryEnergy::setParameters is a no-op
    const size_t nw = (size_t)L * logit_F;
    h_logit_w.assign(lw, lw + nw);
    DCRF_CUDA(cudaMemcpyAsync(logit_w.ensure(nw), h_logit_w.data(), sizeof(float) * nw, cudaMemcpyHostToDevice,
                              stream));
    const long NL = (long)N * L;
    launch(logistic_unary_kernel, ceil_div(NL, 256), 256, 0, stream, NL, L, logit_F, (const float*)logit_w.get(),
           (const float*)logit_f.get(), unary.ensure((size_t)NL));
    DCRF_LAUNCH_CHECK();
    has_unary = true;
    sync();
}

// LogisticUnaryEnergy::gradient(b) = b f^T (:64-68); FP64 sums over pixels.
int Model::unary_gradient(const float* b, float* out) {
    if (logit_F == 0) return 0;  // UnaryEnergy::gradient: empty
    const int F = logit_F, pairs = L * F, nb = 32;
    double* part = partials.ensure((size_t)nb * pairs);
    launch(logistic_grad_partial_kernel, dim3(nb, pairs), 256, 0, stream, N, L, F, b, (const float*)logit_f.get(),
           part);
    DCRF_LAUNCH_CHECK();
    std::vector<double> h((size_t)nb * pairs);
    DCRF_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream));
    sync();
    for (int p = 0; p < pairs; p++) {
        double s = 0.0;
        for (int i = 0; i < nb; i++) s += h[(size_t)p * nb + i];
        out[p] = (float)s;
    }
    return pairs;
}

int Model::n_parameters(int k) const {
    require(k >= 0 && k < (int)terms.size(), DCRF_E_ARG, "pairwise term index out of range");
    const int c = terms[k]->compat;
    return c == kPotts ? 1 : c == kDiagonal ? L : L * (L + 1) / 2;
}

// parameters() (src/labelcompatibility.cpp:64-68, 88-90, 109-115).
int Model::parameters(int k, float* out) const {
    const int n = n_parameters(k);
    const Term& t = *terms[k];
    if (t.compat == kPotts) {
        out[0] = t.w;
    } else if (t.compat == kDiagonal) {
        for (int l = 0; l < L; l++) out[l] = t.hcw[l];
    } else {
        int q = 0;
        for (int c = 0; c < L; c++)
            for (int r = c; r < L; r++) out[q++] = t.hcw[(size_t)c * L + r];
    }
    return n;
}

// setParameters(v) (src/labelcompatibility.cpp:69-71, 91-93, 116-122).
void Model::set_parameters(int k, const float* v) {
    const int kind = terms.at(k)->compat;
    if (kind != kMatrix) {
        set_compat(k, kind, v);
        return;
    }
    std::vector<float> m((size_t)L * L);
    for (int c = 0, q = 0; c < L; c++)
        for (int r = c; r < L; r++, q++) m[(size_t)c * L + r] = m[(size_t)r * L + c] = v[q];
    set_compat(k, kMatrix, m.data());  // already symmetric: the symmetrisation is exact
}

void Model::set_cliques(int R_, const int* off, const int* idx, const float* expw, const float* cst) {
    gen++;  // a captured QP graph may hold what this changes
    has_z_last = false;
    R = R_;
    h_cl_off.assign(off, off + R + 1);
    clique_total = off[R];
    h_cl_idx.assign(idx, idx + clique_total);
    h_cl_exp.assign(expw, expw + R);
    h_cl_const.assign(cst, cst + R);
    clique_max = 0;
    for (int r = 0; r < R; r++) clique_max = std::max(clique_max, off[r + 1] - off[r]);
    // by-size order used by the prefix-chain clique kernels
    std::vector<int> order(R), sorted_sizes(R);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b2) { return off[a + 1] - off[a] < off[b2 + 1] - off[b2]; });
    std::vector<int> packed(2 * (size_t)R + 1 + (size_t)(R + 1));
    // layout: [R+1 offsets][R order][R sorted sizes]
    std::memcpy(packed.data(), off, sizeof(int) * (R + 1));
    for (int r = 0; r < R; r++) {
        packed[R + 1 + r] = order[r];
        packed[2 * R + 1 + r] = off[order[r] + 1] - off[order[r]];
    }
    // bucket starts over the by-size order: cliques of size s are [bs[s], bs[s+1])
    std::vector<int> bs((size_t)clique_max + 2, 0);
    for (int r = 0; r < R; r++) bs[packed[2 * R + 1 + r] + 1]++;
    for (size_t s = 1; s < bs.size(); s++) bs[s] += bs[s - 1];
    int* dbs = cl_bstart.ensure(bs.size());
    DCRF_CUDA(cudaMemcpyAsync(dbs, bs.data(), sizeof(int) * bs.size(), cudaMemcpyHostToDevice, stream));
    int* doff = cl_off.ensure(packed.size());
    DCRF_CUDA(cudaMemcpyAsync(doff, packed.data(), sizeof(int) * packed.size(), cudaMemcpyHostToDevice, stream));
    int* didx = cl_idx.ensure(std::max(clique_total, 1));
    if (clique_total)
        DCRF_CUDA(cudaMemcpyAsync(didx, idx, sizeof(int) * clique_total, cudaMemcpyHostToDevice, stream));
    // the chunked clique kernels' units: chunks of kCliqueChunk pixels per clique, L units each
    {
        std::vector<int2> ch;
        std::vector<int> ub((size_t)R + 1, 0);
        for (int r = 0; r < R; r++) {
            const int nch = (off[r + 1] - off[r] + kCliqueChunk - 1) / kCliqueChunk;
            for (int c = 0; c < nch; c++) ch.push_back(make_int2(r, c));
            ub[r + 1] = ub[r] + L * nch;
        }
        uc_nchunks = (int)ch.size();
        uc_units = ub[R];
        int2* dch = uc_chunks.ensure(std::max<size_t>(ch.size(), 1));
        if (!ch.empty())
            DCRF_CUDA(cudaMemcpyAsync(dch, ch.data(), sizeof(int2) * ch.size(), cudaMemcpyHostToDevice, stream));
        int* dub = uc_base.ensure(ub.size());
        DCRF_CUDA(cudaMemcpyAsync(dub, ub.data(), sizeof(int) * ub.size(), cudaMemcpyHostToDevice, stream));
    }
    float* de = cl_exp.ensure(std::max(R, 1));
    float* dc = cl_const.ensure(std::max(R, 1));
    if (R) {
        DCRF_CUDA(cudaMemcpyAsync(de, expw, sizeof(float) * R, cudaMemcpyHostToDevice, stream));
        DCRF_CUDA(cudaMemcpyAsync(dc, cst, sizeof(float) * R, cudaMemcpyHostToDevice, stream));
    }
    sync();  // host vectors above are the caller's; finish the copies
}

// The term's compatibility as a slice epilogue.  Potts: -w v; Diagonal:
// w_l v (both folded into the slice, with the base accumulation).  Matrix:
// the slice writes the filtered values to a scratch buffer and `finish` runs
// the L x L product with the base accumulation; the caller's epilogue fields
// are returned through `ep` and `*dst` redirected.
namespace {
struct CompatRoute {
    float* slice_out;   // where the slice writes
    bool matrix;        // a matrix pass follows
};
}  // namespace

static CompatRoute route_compat(Model& m, const Term& t, SliceEpilogue& ep, float* out, const float* base,
                                float coef, bool zero_base, bool potts_only = false) {
    ep.potts = true;
    const int kind = potts_only ? (int)kPotts : t.compat;
    if (kind == kMatrix) {
        ep.scale = 1.0f;
        return {m.compat_tmp.ensure((size_t)m.N * m.L), true};
    }
    if (kind == kDiagonal) {
        ep.scale = 1.0f;
        ep.scale_vec = t.cw.get();
    } else {
        ep.scale = -t.w;
    }
    ep.base = base;
    ep.coef = coef;
    ep.zero_base = zero_base;
    return {out, false};
}

static void finish_compat(Model& m, const Term& t, const CompatRoute& r, float* out, const float* base, float coef,
                          bool zero_base) {
    if (!r.matrix) return;
    const long NL = (long)m.N * m.L;
    launch(matrix_compat_kernel, ceil_div(NL, 256), 256, 0, m.stream, NL, m.L, t.cw.get(),
           (const float*)r.slice_out, base, coef, (int)zero_base, out);
    DCRF_LAUNCH_CHECK();
}

void Model::apply_compat(int k, bool nonorm, float* out, const float* in) {
    const Term& t = *terms.at(k);
    const long NL = (long)N * L;
    const int g = ceil_div(NL, 256), kind = nonorm ? (int)kPotts : t.compat;
    if (kind == kPotts)  // out = -w Q (src/labelcompatibility.cpp:49-52)
        launch(scale_cols_kernel, g, 256, 0, stream, NL, L, in, (const float*)nullptr, -t.w, out);
    else if (kind == kDiagonal)
        launch(scale_labels_kernel, g, 256, 0, stream, NL, L, in, (const float*)t.cw.get(), out);
    else
        launch(matrix_compat_kernel, g, 256, 0, stream, NL, L, (const float*)t.cw.get(), in, (const float*)nullptr,
               1.0f, 0, out);
    DCRF_LAUNCH_CHECK();
}

void Model::set_compat(int k, int kind, const float* params) {
    gen++;  // a captured QP graph may hold what this changes
    require(k >= 0 && k < (int)terms.size(), DCRF_E_ARG, "pairwise term index out of range");
    Term& t = *terms[k];
    // Every compatibility's parameters()(0) is also the weight of the term's
    // unnormalised Potts twin (no_norm_pairwise_, src/densecrf.cpp:161-168):
    // Potts w, Diagonal w_0, Matrix w_(0,0).
    t.w = params[0];
    if (kind == kPotts) {
        t.compat = kPotts;
        return;
    }
    require(kind == kDiagonal || kind == kMatrix, DCRF_E_ARG, "unknown label compatibility");
    std::vector<float> h;
    if (kind == kDiagonal) {
        h.assign(params, params + L);
    } else {  // MatrixCompatibility(m): w_ = 0.5 (m + m^T) (src/labelcompatibility.cpp:99-101)
        h.resize((size_t)L * L);
        for (int c = 0; c < L; c++)
            for (int r = 0; r < L; r++) h[(size_t)c * L + r] = (params[(size_t)c * L + r] + params[(size_t)r * L + c]) * 0.5f;
    }
    t.hcw = h;
    float* d = t.cw.ensure(h.size());
    DCRF_CUDA(cudaMemcpyAsync(d, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice, stream));
    sync();
    t.compat = kind;
}

void Model::apply(int k, bool nonorm, float* out, const float* in, const float* base, float coef,
                  bool zero_base) {
    Term& t = *terms[k];
    SliceEpilogue ep;
    ep.norm = nonorm ? nullptr : t.post_norm();
    // nonorm: the unnormalised Potts twin of the term, whatever its
    // compatibility, on the lattice of the features the term was added with
    const CompatRoute r = route_compat(*this, t, ep, out, base, coef, zero_base, nonorm);
    Lattice& lat = nonorm ? t.twin_lat() : *t.lat;
    lat.compute(r.slice_out, in, L, false, ep, nonorm ? nullptr : t.pre_norm());
    finish_compat(*this, t, r, out, base, coef, zero_base);
}

void Model::apply_ord(int k, float* out, const float* rq, const float* base, bool zero_base) {
    Term& t = *terms[k];
    SliceEpilogue ep;
    const CompatRoute r = route_compat(*this, t, ep, out, base, 1.0f, zero_base);
    t.lat->compute_ord(r.slice_out, rq, L, ep);
    finish_compat(*this, t, r, out, base, 1.0f, zero_base);
}

// out = sum_k apply_k(in) in term order (out = 0 + t_0, then out += t_k), as
// the QP's pairwise sums are formed (src/densecrf.cpp:411-420): the splat and
// blur of terms 1.. run on the side stream while term 0's run on the model's
// stream, then the slices carry the sum in term order.  Images above
// kSplitMaxPixels and Matrix terms (their product runs after the slice) take
// the plain path, one term after the other.
void Model::apply_sum(float* out, const float* in) {
    const int nt = (int)terms.size();
    // Concurrency pays on images that do not fill the GPU alone (measured:
    // 320x240 QP 1123 -> 1190 solves/s); on larger ones the two filters
    // compete for L2 and the sum is slower (240-500 px sides: -15 %).
    bool split = nt >= 2 && N <= kSplitMaxPixels;
    for (const auto& t : terms) split = split && t->compat != kMatrix;
    if (!split) {
        for (int k = 0; k < nt; k++) apply(k, false, out, in, k == 0 ? nullptr : out, 1.0f, k == 0);
        return;
    }
    if (!side) {
        DCRF_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        DCRF_CUDA(cudaEventCreateWithFlags(&ev_side_fork, cudaEventDisableTiming));
        DCRF_CUDA(cudaEventCreateWithFlags(&ev_side_join, cudaEventDisableTiming));
    }
    DCRF_CUDA(cudaEventRecord(ev_side_fork, stream));
    DCRF_CUDA(cudaStreamWaitEvent(side, ev_side_fork, 0));
    for (int k = 1; k < nt; k++) {
        Term& t = *terms[k];
        t.lat->stream = side;
        try {
            t.lat->splat_blur(in, L, false, t.pre_norm());
        } catch (...) {
            t.lat->stream = stream;
            throw;
        }
        t.lat->stream = stream;
    }
    DCRF_CUDA(cudaEventRecord(ev_side_join, side));
    terms[0]->lat->splat_blur(in, L, false, terms[0]->pre_norm());
    DCRF_CUDA(cudaStreamWaitEvent(stream, ev_side_join, 0));
    for (int k = 0; k < nt; k++) {
        const Term& t = *terms[k];
        SliceEpilogue ep;
        ep.norm = t.post_norm();
        route_compat(*this, t, ep, out, k == 0 ? nullptr : out, 1.0f, k == 0);
        t.lat->slice(out, L, ep);
    }
}

// sa = sum_k apply_upper_minus_lower_ord_k(rescale(Q)) from shared bins, the
// sum in term order (sa = 0 + t_0, then sa += t_k) as the reference adds it
// (src/densecrf.cpp:705-716).  The splat and blur phases of terms 1.. run on
// a side stream while term 0's run on the model's stream; the slices, which
// carry the accumulation, then run in term order.  `gap`: the dual-gap sums
// folded into the last slice.
void Model::apply_ord_sum(float* sa, const float2* bins, const GapFusion* gap) {
    const int nt = (int)terms.size();
    if (nt >= 2) {
        if (!side) {
            DCRF_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
            DCRF_CUDA(cudaEventCreateWithFlags(&ev_side_fork, cudaEventDisableTiming));
            DCRF_CUDA(cudaEventCreateWithFlags(&ev_side_join, cudaEventDisableTiming));
        }
        DCRF_CUDA(cudaEventRecord(ev_side_fork, stream));
        DCRF_CUDA(cudaStreamWaitEvent(side, ev_side_fork, 0));
        for (int k = 1; k < nt; k++) {
            Lattice& lat = *terms[k]->lat;
            lat.stream = side;
            try {
                lat.ord_splat_blur(bins, L);
            } catch (...) {
                lat.stream = stream;
                throw;
            }
            lat.stream = stream;
        }
        DCRF_CUDA(cudaEventRecord(ev_side_join, side));
    }
    if (nt >= 1) terms[0]->lat->ord_splat_blur(bins, L);
    if (nt >= 2) DCRF_CUDA(cudaStreamWaitEvent(stream, ev_side_join, 0));
    if (nt == 2 && terms[0]->compat != kMatrix && terms[1]->compat != kMatrix) {
        // the two slices in one pass (the sum in term order, bit for bit)
        SliceEpilogue e0, e1;
        route_compat(*this, *terms[0], e0, sa, nullptr, 1.0f, true);
        route_compat(*this, *terms[1], e1, sa, sa, 1.0f, false);
        Lattice::ord_slice_pair(sa, bins, L, *terms[0]->lat, e0, *terms[1]->lat, e1, gap);
        return;
    }
    for (int k = 0; k < nt; k++) {
        SliceEpilogue ep;
        const Term& t = *terms[k];
        const float* base = k == 0 ? nullptr : sa;
        const CompatRoute r = route_compat(*this, t, ep, sa, base, 1.0f, k == 0);
        terms[k]->lat->ord_slice(r.slice_out, bins, L, ep, k == nt - 1 && !r.matrix ? gap : nullptr);
        finish_compat(*this, t, r, sa, base, 1.0f, k == 0);
    }
}

void Model::apply_ord_restricted(int k, float* rout, const float* rQ, const int* pI, int nP, const float* Q,
                                 bool store) {
    Term& t = *terms[k];
    SliceEpilogue ep;
    const CompatRoute r = route_compat(*this, t, ep, rout, nullptr, 1.0f, false);
    t.lat->compute_ord_restricted(r.slice_out, rQ, pI, nP, Q, L, store, ep);
    if (r.matrix && nP) {
        const long n = (long)nP * L;
        launch(matrix_compat_kernel, ceil_div(n, 256), 256, 0, stream, n, L, t.cw.get(), (const float*)r.slice_out,
               (const float*)nullptr, 1.0f, 0, rout);
        DCRF_LAUNCH_CHECK();
    }
}

void Model::apply_ord_bins(int k, float* out, const float2* bins, const float* base, bool zero_base,
                           const GapFusion* gap) {
    Term& t = *terms[k];
    SliceEpilogue ep;
    const CompatRoute r = route_compat(*this, t, ep, out, base, 1.0f, zero_base);
    t.lat->compute_ord_bins(r.slice_out, bins, L, ep, r.matrix ? nullptr : gap);
    finish_compat(*this, t, r, out, base, 1.0f, zero_base);
}

void Model::check_unit_range(const float* Q) {
    launch(minmax_partial_kernel, kRedBlocks, kRedThreads, 0, stream, (long)N * L, Q, partials.get());
    launch(minmax_finish_kernel, 1, 32, 0, stream, partials.get(), kRedBlocks, scal.get());
    DCRF_LAUNCH_CHECK();
    fetch_scalars();
    if (h_scal->qmax > 1.0f || h_scal->qmin < 0.0f) throw Error(DCRF_E_RANGE, "Value out of bounds");
}

void Model::rescale(float* out, const float* Q) {
    launch(minmax_partial_kernel, kRedBlocks, kRedThreads, 0, stream, (long)N * L, Q, partials.get());
    launch(minmax_finish_kernel, 1, 32, 0, stream, partials.get(), kRedBlocks, scal.get());
    launch(rescale_kernel, ceil_div((long)N * L, 256), 256, 0, stream, (long)N * L, Q, scal.get(), out);
    DCRF_LAUNCH_CHECK();
}

void Model::unary_init(float* Q) {
    require(has_unary, DCRF_E_STATE, "unary_init: no unary energy set");
    with_lc(L, [&](auto lc) {
        constexpr int LC = decltype(lc)::value;
        launch(unary_init_kernel<LC>, ceil_div(N, 128), 128, 0, stream, N, L, unary.get(), Q);
    });
    DCRF_LAUNCH_CHECK();
}

void Model::current_map(const float* Q, int16_t* lab) {
    with_lc(L, [&](auto lc) {
        constexpr int LC = decltype(lc)::value;
        launch(current_map_kernel<LC>, ceil_div(N, 128), 128, 0, stream, N, L, Q, lab);
    });
    DCRF_LAUNCH_CHECK();
}

// assignment_energy_true / assignment_energy_higher_order
// (src/densecrf.cpp:873-885, 844-870, 887-927).
double Model::energy_true(const int16_t* d_lab, bool ho) {
    require(has_unary, DCRF_E_STATE, "energy: no unary energy set");
    float* qc = buf(10);
    float* o = buf(11);
    float* pw = b[12].ensure(N);
    launch(onehot_complement_kernel, ceil_div((long)N * L, 256), 256, 0, stream, N, L, d_lab, qc);
    for (size_t k = 0; k < terms.size(); k++) {
        apply((int)k, true, o, qc);
        launch(pairwise_pick_kernel, ceil_div(N, 256), 256, 0, stream, N, L, d_lab, o, pw, k == 0);
    }
    if (terms.empty()) launch(fill_kernel, ceil_div(N, 256), 256, 0, stream, N, 0.0f, pw);
    launch(energy_sum_kernel, kRedBlocks, kRedThreads, 0, stream, N, L, d_lab, unary.get(), pw, partials.get());
    launch(finalize_sums_kernel, 1, 32, 0, stream, partials.get(), kRedBlocks, 1, 0, scal.get());
    if (ho && R > 0) {
        int* flags = ipart.ensure(std::max(R, 1));
        launch(clique_label_change_kernel, R, 256, 0, stream, cl_off.get(), cl_idx.get(), d_lab, flags);
        launch(energy_ho_finish_kernel, 1, 1, 0, stream, R, flags, cl_exp.get(), scal.get());
    }
    DCRF_LAUNCH_CHECK();
    fetch_scalars();
    return h_scal->sums[0];
}

// compute_energy_LP_higher_order (src/densecrf.cpp:982-1037).
double Model::energy_lp(const float* Q) {
    require(has_unary, DCRF_E_STATE, "energy: no unary energy set");
    float* rq = buf(10);
    float* o = buf(11);
    rescale(rq, Q);
    launch(dot_kernel, kRedBlocks, kRedThreads, 0, stream, (long)N * L, unary.get(), Q, partials.get());
    launch(finalize_sums_kernel, 1, 32, 0, stream, partials.get(), kRedBlocks, 1, 0, scal.get());
    for (size_t k = 0; k < terms.size(); k++) {
        apply_ord((int)k, o, rq);
        launch(dot_kernel, kRedBlocks, kRedThreads, 0, stream, (long)N * L, Q, o, partials.get());
        launch(finalize_sums_kernel, 1, 32, 0, stream, partials.get(), kRedBlocks, 1, 1 + (int)k, scal.get());
    }
    if (R > 0) {
        float* diffs = b[13].ensure(std::max(R, 1));
        float2* part = reinterpret_cast<float2*>(uc_scan.ensure(std::max<size_t>(3 * (size_t)uc_units, 1)));
        if (uc_nchunks > 0)
            launch(clique_maxdiff_chunk_kernel, uc_nchunks, 256, 0, stream, uc_chunks.get(), cl_off.get(),
                   cl_idx.get(), uc_base.get(), L, Q, part);
        launch(clique_maxdiff_finish_kernel, R, 64, 0, stream, cl_off.get(), uc_base.get(), L, (const float2*)part,
               diffs);
    }
    launch(energy_lp_finish_kernel, 1, 1, 0, stream, (int)terms.size(), R, b[13].get(), cl_exp.get(), scal.get());
    DCRF_LAUNCH_CHECK();
    fetch_scalars();
    return h_scal->energy;
}

// compute_LR_QP_value(Q, diag_dom) (src/densecrf.cpp:940-957); diag_dom
// null stands for 0.
double Model::lr_qp_value(const float* Q, const float* dd) {
    require(has_unary, DCRF_E_STATE, "energy: no unary energy set");
    const int nt = (int)terms.size();
    require(nt + 3 <= 16, DCRF_E_ARG, "energy: too many pairwise terms");
    const long NL = (long)N * L;
    float* o = buf(11);
    launch(dot_kernel, kRedBlocks, kRedThreads, 0, stream, NL, unary.get(), Q, partials.get());
    launch(finalize_sums_kernel, 1, 32, 0, stream, partials.get(), kRedBlocks, 1, 0, scal.get());
    if (dd) {
        launch(dot_kernel, kRedBlocks, kRedThreads, 0, stream, NL, dd, Q, partials.get());
        launch(finalize_sums_kernel, 1, 32, 0, stream, partials.get(), kRedBlocks, 1, nt + 1, scal.get());
        launch(dot3_kernel, kRedBlocks, kRedThreads, 0, stream, NL, Q, dd, Q, partials.get());
        launch(finalize_sums_kernel, 1, 32, 0, stream, partials.get(), kRedBlocks, 1, nt + 2, scal.get());
    }
    for (int k = 0; k < nt; k++) {
        apply(k, false, o, Q);
        launch(dot_kernel, kRedBlocks, kRedThreads, 0, stream, NL, Q, o, partials.get());
        launch(finalize_sums_kernel, 1, 32, 0, stream, partials.get(), kRedBlocks, 1, 1 + k, scal.get());
    }
    launch(lr_finish_kernel, 1, 1, 0, stream, nt, scal.get(), (int)(dd != nullptr));
    DCRF_LAUNCH_CHECK();
    fetch_scalars();
    return h_scal->energy;
}

void Model::unary_energy(const int16_t* d_lab, float* out) {
    if (!has_unary) {  // no unary energy: zeros, as the reference's r.fill(0)
        launch(fill_kernel, ceil_div(N, 256), 256, 0, stream, N, 0.0f, out);
    } else {
        launch(unary_pick_kernel, ceil_div(N, 256), 256, 0, stream, N, L, d_lab, (const float*)unary.get(), out);
    }
    DCRF_LAUNCH_CHECK();
}

// pairwise_energy_true: the unnormalised twin applied to the one-hot
// complement of l, r_i = -(.)(l_i, i); term -1: r = 0 + r_0 + r_1 + ...
void Model::pairwise_energy(const int16_t* d_lab, int term, float* out) {
    const int nt = (int)terms.size();
    require(term >= -1 && term < nt, DCRF_E_ARG, "pairwise term index out of range");
    float* qc = buf(10);
    float* o = buf(11);
    launch(onehot_complement_kernel, ceil_div((long)N * L, 256), 256, 0, stream, N, L, d_lab, qc);
    const int k0 = term < 0 ? 0 : term, k1 = term < 0 ? nt : term + 1;
    if (k0 == k1) launch(fill_kernel, ceil_div(N, 256), 256, 0, stream, N, 0.0f, out);
    for (int k = k0; k < k1; k++) {
        apply(k, true, o, qc);
        launch(pairwise_pick_kernel, ceil_div(N, 256), 256, 0, stream, N, L, d_lab, (const float*)o, out, k == k0);
    }
    DCRF_LAUNCH_CHECK();
}

}  // namespace dcrf
