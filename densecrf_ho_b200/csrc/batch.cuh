// Many images of different sizes solved together: their pixels are
// concatenated ([sum N_i][L]), each Potts term's lattices are concatenated
// into one (Lattice::concat), and the Frank-Wolfe QP keeps one set of
// solver scalars per image, so every image follows exactly the trajectory of
// its own single-image solve while each filter, direction and update runs as
// one launch over all images; the filters skip the lattice vertices and
// pixels of images that have already stopped.  After a first eager
// iteration, an iteration is captured once as a CUDA graph and replayed.
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
    DevBuf<int> d_active;
    DevBuf<int> d_done;          // per image: stopped before the current iteration (filters skip it)
    int* h_active = nullptr;     // pinned
    SolverScalars* h_scal = nullptr;  // pinned, B
    int max_tiles = 0;           // row-tile blocks of the largest image

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

  private:
    void qp_iteration(float* Q, int max_iter);
    void drop_graph();
};

}  // namespace dcrf
