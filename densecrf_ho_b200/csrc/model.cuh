// DenseCRF2D state on the device: unaries, Potts pairwise terms (each with
// its lattice and symmetric normalisation), superpixel cliques, and the
// solver work buffers.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "lattice.cuh"

namespace dcrf {

// Label compatibility of a pairwise term (include/labelcompatibility.h).
enum CompatKind { kPotts = 0, kDiagonal = 1, kMatrix = 2 };

// DenseKernel's KernelType and NormalizationType (include/pairwise.h).
enum KernelKind { kConstKernel = 0, kDiagKernel = 1, kFullKernel = 2 };
enum NormKind { kNoNorm = 0, kNormBefore = 1, kNormAfter = 2, kNormSymmetric = 3 };

struct Term {
    std::unique_ptr<Lattice> lat;
    // The unnormalised twin's lattice (no_norm_pairwise_, built on the
    // features the term was added with) once setKernelParameters has rebuilt
    // lat on scaled features; until then the twin shares lat.
    std::unique_ptr<Lattice> twin;
    int ktype = kDiagKernel, ntype = kNormSymmetric;
    std::vector<float> kparams;  // DenseKernel::parameters_: DIAG d scales, FULL d x d (column-major)
    int compat = kPotts;  // Potts: mu = -w [a == b]; Diagonal: cw[L]; Matrix: cw[L x L], symmetrised
    DevBuf<float> cw;
    std::vector<float> hcw;  // host copy of cw
    DevBuf<float> norm;  // 1/sqrt(K 1 + 1e-20) (symmetric) or 1/(K 1 + 1e-20) (src/pairwise.cpp:44-56)
    const float* pre_norm() const {  // scale before the filter (DenseKernel::filter, not transposed)
        return (ntype == kNormSymmetric || ntype == kNormBefore) ? norm.get() : nullptr;
    }
    const float* post_norm() const {  // scale after it
        return (ntype == kNormSymmetric || ntype == kNormAfter) ? norm.get() : nullptr;
    }
    Lattice& twin_lat() { return twin ? *twin : *lat; }
    DevBuf<float> feat;  // the features [N][d] (DenseKernel::f_), for the kernel gradient
    float w = 0.0f;      // Potts weight
    int d = 0;
};

// Fixed-size deterministic FP64 reduction: every reduction kernel runs this
// many blocks and writes one partial per block; a one-warp kernel sums the
// partials in a fixed order.
constexpr int kRedBlocks = 296;
constexpr int kRedThreads = 256;

// Device-side scalars of the solvers (one struct, updated by 1-thread kernels).
struct SolverScalars {
    double sums[16];     // finalised reductions
    double energy, old_energy;
    float fstep, f2step;  // QP step as float and 2*step as float
    float delta;          // LP Frank-Wolfe step
    float qp_value;       // LP gamma objective (previous iterate)
    float qmin, qmax;     // rescale bounds
    int stop;             // loop-exit flag (QP: stop rule / zero step; LP: gamma converged)
    int zero_step;        // QP: num == 0 or denom == 0
    int steps;
    int err;              // DCRF_E_* raised by a device check
    int done;             // batched QP: the image had stopped before this iteration
    int gamma_sum;        // LP: qp-gamma iterations of the whole solve
    int chunk;            // QP graph: iterations in the current launch
    int numeric;          // bits: 1 a NaN / inf in a solver's input, 2 in a rescaled
                          // iterate, 4 rescale's maxval < 0 (src/eigen_utils.cpp:138)
};

constexpr int kQpChunk = 64;  // QP iterations per graph launch at most
constexpr int kSplitMaxPixels = 1 << 17;  // apply_sum runs the terms' filters concurrently up to this size

// Pixels per chunk of the chunked clique kernels (computeUCondGrad, the LP
// clique energy): a clique of n pixels has ceil(n / kCliqueChunk) chunks.
constexpr int kCliqueChunk = 128;

struct Model {
    int W = 0, H = 0, N = 0, L = 0, device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;  // second stream for the other terms' filter work
    cudaStream_t gstream = nullptr;  // captures the body of the LP's qp-gamma loop
    // The QP loop as a graph (see Model::qp), its key and its kernels per
    // iteration; gen counts the changes to the model that a graph may hold.
    cudaGraphExec_t qp_graph = nullptr;
    std::vector<const void*> qp_key;
    unsigned long long qp_graph_kernels = 0;
    bool qp_graph_failed = false;
    unsigned long long gen = 0;
    std::vector<const void*> qp_graph_key(const float* Q, int max_iter);
    void drop_qp_graph();
    template <typename F>
    void build_qp_graph(F&& qp_iter);
    cudaEvent_t ev_side_fork = nullptr, ev_side_join = nullptr;
    bool has_unary = false;
    DevBuf<float> unary;
    // LogisticUnaryEnergy (src/unary.cpp:47-70): unary = lw * lf, lw L x F and
    // lf F x N, both column-major; logit_F = 0 for a constant unary.
    int logit_F = 0;
    DevBuf<float> logit_w, logit_f;
    std::vector<float> h_logit_w;
    std::vector<std::unique_ptr<Term>> terms;

    // cliques (super_pixel_container_, exp_of_superpixels_, constants_)
    int R = 0, clique_total = 0, clique_max = 0;
    std::vector<int> h_cl_off, h_cl_idx;
    std::vector<float> h_cl_exp, h_cl_const;
    DevBuf<int> cl_off, cl_idx;
    DevBuf<int> cl_bstart;  // [max + 2]: in by-size order, the first clique of size >= s
    DevBuf<float> cl_exp, cl_const;

    // work buffers
    DevBuf<float> b[16];
    DevBuf<double> partials;
    DevBuf<SolverScalars> scal;
    DevBuf<int16_t> labels;
    DevBuf<float2> lp_bins;  // ordered-filter bins of rescale(Q), shared by all terms
    DevBuf<int> ipart;
    DevBuf<double> ho_pre;  // qp_sp: FP64 clique prefixes [2][R][L]
    DevBuf<double> ho_seg;  // qp_sp: FP64 per-segment totals of a clique prefix chain
    DevBuf<float> z_last;   // the clique variables z [R][L] at the end of the last QP (z_labels_)
    bool has_z_last = false;
    // compute_energy_higher_order(Q) (src/densecrf.cpp:960-980), with the z of
    // the last QP (DCRF_E_STATE with cliques and no QP since they were set).
    double energy_qp_ho(const float* Q);
    DevBuf<int> lp_win;  // lp_sp: per element, the latest clique write claiming it (-1 between calls)
    // lp_sp: computeUCondGrad's units (clique r, label, chunk c of kCliqueChunk pixels):
    // the (r, c) of every chunk, each clique's first unit, and per unit the
    // (min, max) partials, carries and selected positions
    DevBuf<int2> uc_chunks;
    DevBuf<int> uc_base;
    DevBuf<int2> uc_scan;  // [3][uc_units]
    int uc_nchunks = 0, uc_units = 0;
    SolverScalars* h_scal = nullptr;  // pinned mirror

    Model(int W_, int H_, int L_);
    ~Model();

    float* buf(int i) { return b[i].ensure((size_t)N * L); }
    void add_term(const float* d_features, int d, float w);
    void set_cliques(int R, const int* off, const int* idx, const float* expw, const float* cst);

    // PairwisePotential::apply / no_norm_pairwise_ apply, with epilogue
    // out = base + coef * (-w K~ in)  (see SliceEpilogue).
    void apply(int k, bool nonorm, float* out, const float* in, const float* base = nullptr,
               float coef = 1.0f, bool zero_base = false);
    void apply_ord_sum(float* sa, const float2* bins, const GapFusion* gap);
    // Replaces term k's Potts compatibility: kDiagonal (params: L weights)
    // or kMatrix (params: L x L column-major, used as 0.5 (m + m^T)).
    void set_compat(int k, int kind, const float* params);
    DevBuf<float> compat_tmp;
    // pairwise_[k]->kernelGradient(b, Q) (d floats: the diagonal kernel's
    // feature-scale gradient) and ->gradient(b, Q) (the Potts weight's);
    // b, Q device [N][L], results to host.
    int kernel_gradient(int k, const float* b, const float* Q, float* out);  // returns the count
    // addPairwiseEnergy's KernelType / NormalizationType for term k, and
    // DenseKernel::parameters / setParameters (src/pairwise.cpp:123-168).
    void set_kernel(int k, int ktype, int ntype);
    int kernel_parameters(int k, float* out) const;
    void set_kernel_parameters(int k, const float* p);
    void compute_norm(Term& t);
    // LabelCompatibility::parameters / setParameters / gradient of term k:
    // 1 (Potts), L (Diagonal) or L (L + 1) / 2 (Matrix, upper triangle by
    // column) values; each returns that count.
    // PairwisePotential::apply_upper_minus_lower_ord_restricted
    // (src/pairwise.cpp:229-240): the term's restricted ordered filter and
    // compatibility; rout, rQ [nP][L], pI (device) strictly ascending.
    void apply_ord_restricted(int k, float* rout, const float* rQ, const int* pI, int nP, const float* Q,
                              bool store);
    // The exact filters and the divide-and-conquer ordered filter of
    // PairwisePotential (src/pairwise.cpp:241-380): apply_bf(out, Q),
    // apply_upper_minus_lower_bf(out, ind) (Q = nullptr) /
    // apply_upper_minus_lower_bf_ord(out, ind, Q) and
    // apply_upper_minus_lower_dc(out, ind); device [N][L] buffers, ind [N][L]
    // (ind(l, c) at c L + l); nonorm applies the Potts compatibility of
    // no_norm_pairwise_[k] instead of the term's.
    void apply_bf(int k, bool nonorm, float* out, const float* Q);
    void apply_upper_minus_lower_bf(int k, bool nonorm, float* out, const int* ind, const float* Q);
    void apply_upper_minus_lower_dc(int k, bool nonorm, float* out, const int* ind);
    // out = compatibility_->apply(in) of term k (nonorm: its Potts twin's);
    // out must not alias in.
    void apply_compat(int k, bool nonorm, float* out, const float* in);
    void set_unary_logistic(const float* lw, const float* lf, int F);  // host arrays
    void set_unary_parameters(const float* lw);
    int unary_gradient(const float* b, float* out);  // b f^T, L x F column-major; returns L F
    int n_parameters(int k) const;
    int parameters(int k, float* out) const;
    void set_parameters(int k, const float* v);
    int compat_gradient(int k, const float* b, const float* Q, float* out);
    void apply_ord_bins(int k, float* out, const float2* bins, const float* base, bool zero_base,
                        const GapFusion* gap);
    void apply_ord(int k, float* out, const float* rq, const float* base = nullptr,
                   bool zero_base = false);
    // out = sum_k apply_k(in), terms in order, their splats and blurs concurrent.
    void apply_sum(float* out, const float* in);
    // Checks Q in [0,1] like apply_upper_minus_lower_ord (throws DCRF_E_RANGE).
    void check_unit_range(const float* Q);

    void unary_init(float* Q);
    void current_map(const float* Q, int16_t* lab);
    double energy_true(const int16_t* d_lab, bool ho);
    double energy_lp(const float* Q);
    double lr_qp_value(const float* Q, const float* diag_dom = nullptr);
    // unaryEnergy(l) / pairwise_energy_true(l, term) (src/densecrf.cpp:887-927): per-pixel
    // energies into out[N] (device); term -1 sums every term in order.
    void unary_energy(const int16_t* d_lab, float* out);
    void pairwise_energy(const int16_t* d_lab, int term, float* out);
    void max_rounding(const float* Q, float* out);  // max_rounding (:832-840)
    void rescale(float* out, const float* Q);  // rescale (src/eigen_utils.cpp:120-141)

    int qp(const float* init, float* out, int max_iter, double* energy);
    int lp(const float* init, float* out, const dcrf_lp_params& p, dcrf_solve_stats* stats);

    void sync() { DCRF_CUDA(cudaStreamSynchronize(stream)); }
    void fetch_scalars();  // D2H of the scalars (synchronises)
};

}  // namespace dcrf
