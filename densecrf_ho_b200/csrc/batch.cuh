// Many images of different sizes solved together: their pixels are
// concatenated ([sum N_i][L]), each Potts term's lattices are concatenated
// into one (Lattice::concat), and the Frank-Wolfe QP keeps one set of
// solver scalars per image, so every image follows exactly the trajectory of
// its own single-image solve while each filter, direction and update runs as
// one launch over all images; the filters skip the lattice vertices and
// pixels of images that have already stopped.  After a first eager
// iteration the loop is captured once as a CUDA graph -- a `while` node whose
// body is one iteration and whose condition is "some image still running"
// (at most kQpChunk iterations per launch) -- and replayed.
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
    DevBuf<SolverScalars> scal;  // one per image
    DevBuf<int> d_active;        // [0] images still running, [1] iterations in the current graph launch
    DevBuf<int> d_done;          // per image: stopped before the current iteration (filters skip it)
    int* h_active = nullptr;     // pinned, [2]: copy of d_active
    SolverScalars* h_scal = nullptr;  // pinned, B
    int max_tiles = 0;           // row-tile blocks of the largest image

    // mean-field checkpoints Q_0 .. Q_mf_T, [mf_T + 1][Ntot][L]
    DevBuf<float> mf_ck, mf_g0, mf_g1, mf_ga, mf_m;
    DevBuf<double> mf_dw;
    int mf_T = -1;

    // the captured QP iteration (valid while the output buffer and max_iter are the same)
    cudaGraphExec_t graph = nullptr;
    const float* graph_q = nullptr;
    int graph_max_iter = -1;
    unsigned long long graph_kernels = 0;

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
    void qp_iteration(float* Q, int max_iter, bool copy_active = true);
    void drop_graph();
};

}  // namespace dcrf
