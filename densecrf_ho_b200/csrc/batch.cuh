// Many images of different sizes behind one handle: their pixels are
// concatenated ([sum N_i][L]).  The mean-field iterations and their adjoint
// run over all images at once on each Potts term's concatenated lattice
// (Lattice::concat).  The Frank-Wolfe QP runs every image's own model
// (Model::qp, its loop a device-side graph loop) from several host threads,
// so the images' solves overlap; each image's result is that of its own
// single-image solve, bit for bit.
#pragma once
#include <memory>
#include <vector>

#include "model.cuh"

namespace dcrf {

struct Batch {
    int B = 0, L = 0, device = 0;
    long Ntot = 0;
    std::vector<int> W, H;
    std::vector<long> pix_off;  // B + 1 pixel offsets
    cudaStream_t stream = nullptr;
    bool has_unary = false;
    DevBuf<float> unary;
    std::vector<std::unique_ptr<Term>> terms;

    DevBuf<long> d_pix_off;
    DevBuf<float> b[6];
    DevBuf<double> partials;
    unsigned long long unary_gen = 0;  // bumped by every unary change

    // The QP runs each image's own model (built at the first solve from the
    // terms' features, kept until a term is added).
    std::vector<std::unique_ptr<Model>> img;
    unsigned long long img_unary_gen = ~0ull;
    // The last QP ran (or captured) every image's graph for this output
    // buffer and max_iter: the next such QP may run the images concurrently.
    bool qp_warm = false;
    const float* warm_out = nullptr;
    int warm_max_iter = -1;

    // mean-field checkpoints Q_0 .. Q_mf_T, [mf_T + 1][Ntot][L]
    DevBuf<float> mf_ck, mf_g0, mf_g1, mf_ga, mf_m;
    DevBuf<double> mf_dw;
    int mf_T = -1;


    Batch(int n, const int* widths, const int* heights, int L_);
    ~Batch();

    float* buf(int i) { return b[i].ensure((size_t)Ntot * L); }
    // d_features: device [Ntot][d], image after image
    void add_term(const float* d_features, int d, float w);
    void apply(int k, float* out, const float* in, const float* base = nullptr, float coef = 1.0f,
               bool zero_base = false);
    void unary_init(float* Q);
    // Returns the largest per-image step count; per-image counts / energies
    // go to steps / energies when given (host arrays of B).
    int qp(const float* init, float* out, int max_iter, int* steps, double* energies);

    // Mean-field iterations Q_0 = softmax(-U), Q_{t+1} = softmax(-U + sum_k
    // w_k K~_k Q_t) (K~ = the normalised Gaussian / bilateral filter), with
    // Q_0 .. Q_T kept as checkpoints for meanfield_backward.
    void meanfield(int iterations, float* Q);
    // Gradients of a loss through the last meanfield(): grad_Q = dL/dQ_T in,
    // dL/dU and dL/dw_k (summed over all images, FP64) out.
    void meanfield_backward(const float* grad_Q, float* grad_U, double* grad_w);
    void set_weight(int k, float w);

  private:
    void ensure_image_models();
};

constexpr int kQpThreads = 8;  // host threads of a batch QP

}  // namespace dcrf
