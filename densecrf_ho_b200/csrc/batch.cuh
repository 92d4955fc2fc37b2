// Many images of different sizes behind one handle: their pixels are
// concatenated ([sum N_i][L]) and each Potts term's lattices are
// concatenated too (Lattice::concat).  The mean-field iterations and their
// adjoint, and the Frank-Wolfe QP, run over all images at once: the QP in
// lockstep, one launch per step for every image still running (its loop a
// device-side graph loop), each image's result that of its own single-image
// solve, bit for bit.
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

    // mean-field checkpoints: Q_t for t % ck_every == 0 and Q_T, [slots][Ntot][L];
    // the other iterates are recomputed segment by segment in the backward
    // pass into mf_seg ([ck_every - 1][Ntot][L]).
    DevBuf<float> mf_ck, mf_seg, mf_g0, mf_g1, mf_ga, mf_m, mf_x0, mf_x1;
    DevBuf<double> mf_dw;
    int mf_T = -1;
    int ck_every = 1;              // keep every ck_every-th iterate (1 = all)
    bool recompute_lattice = false;  // release the lattices between the passes, rebuild them


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

    // Lockstep QP state: per-image scalars and loop flags, per-image partial
    // sums, the row-tile table of the direction kernel, the loop as a graph.
    DevBuf<SolverScalars> bsc;
    DevBuf<int> bdone, bflags, btile_off;
    DevBuf<long> btile_base;  // btile_off as the direction kernel's domain
    DevBuf<int> blive;        // [0] live image count, [1 .. B] their ids
    DevBuf<long> blive_pre;   // live prefixes: kDomains per term, then the direction tiles
    DevBuf<double> bpart, bpart_dir;
    int btiles = 0;
    cudaGraphExec_t bqp_graph = nullptr;
    std::vector<const void*> bqp_key;
    unsigned long long bqp_graph_kernels = 0;
    bool bqp_graph_failed = false;
    unsigned long long weights_gen = 0;  // bumped by set_weight and add_term (captured scales)

    // Mean-field iterations Q_0 = softmax(-U), Q_{t+1} = softmax(-U + sum_k
    // w_k K~_k Q_t) (K~ = the normalised Gaussian / bilateral filter), with
    // Q_0 .. Q_T kept as checkpoints for meanfield_backward.
    void meanfield(int iterations, float* Q);
    // Gradients of a loss through the last meanfield(): grad_Q = dL/dQ_T in,
    // dL/dU and dL/dw_k (summed over all images, FP64) out.
    void meanfield_backward(const float* grad_Q, float* grad_U, double* grad_w);
    void set_weight(int k, float w);
    void set_checkpointing(int every, bool recompute_lat);
    // Builds every term's concatenated lattice that is not there (released
    // by the recompute_lattice mode), from the term's features.
    void ensure_lattices();
    // Device bytes the mean-field checkpoints and recompute buffers take for
    // T iterations under the current checkpointing.
    size_t meanfield_state_bytes(int T) const;

  private:
    template <typename F>
    void build_bqp_graph(F&& iteration, int* flags);
    void build_lattice(Term& t);
    int ck_slot(int t) const { return t == mf_T && t % ck_every ? mf_T / ck_every + 1 : t / ck_every; }
    bool ck_stored(int t) const { return t % ck_every == 0 || t == mf_T; }
    void mf_iteration(const float* q, float* qn, const float* negU, float* logits);
};


}  // namespace dcrf
