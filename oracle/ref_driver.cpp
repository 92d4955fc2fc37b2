// Test-infrastructure C driver over the UNMODIFIED densecrf_ho reference.
//
// This file is linked against the reference's own sources (compiled in place
// by oracle/Makefile into oracle/_ref/libdcrf_ref.so).  It exists so that the
// test suite, the golden-fixture generator and bench.py's CPU baseline can call
// the reference from Python through ctypes.  Nothing in the product links it.
//
// Reference classes are reached through small subclasses that expose their
// protected members (Permutohedral::offset_ etc., DenseCRF::pairwise_ etc.);
// no reference code is modified or copied.
//
// Layouts: every matrix crosses this boundary as the reference's Eigen
// column-major L x N storage, i.e. a flat float array indexed [pixel*L + label].
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>
#include <limits>

#include "densecrf.h"
#include "probimage.h"
#include "msImageProcessor.h"

#include <cmath>
#include <netinet/in.h>
#include "eigen_utils.hpp"
#include "permutohedral.h"
#include "qp.hpp"

namespace {

struct LatticeProbe : public Permutohedral {
    int N() const { return N_; }
    int M() const { return M_; }
    int d() const { return d_; }
    const std::vector<int>& offsets() const { return offset_; }
    const std::vector<int>& ranks() const { return rank_; }
    const std::vector<float>& barys() const { return barycentric_; }
    void neighbours(int* out) const {
        for (size_t i = 0; i < blur_neighbors_.size(); i++) {
            out[2 * i] = blur_neighbors_[i].n1;
            out[2 * i + 1] = blur_neighbors_[i].n2;
        }
    }
};

// Exposes DenseCRF's protected state so cliques can be injected directly and
// so a fixed-iteration QP can be run from the reference's own building blocks.
struct RefModel : public DenseCRF2D {
    RefModel(int W, int H, int L) : DenseCRF2D(W, H, L) {}
    // pairwise_[k]->kernelGradient(b, Q) and ->gradient(b, Q) (src/pairwise.cpp:390-407)
    VectorXf kernel_gradient(int k, const MatrixXf& b, const MatrixXf& Q) const {
        return pairwise_[k]->kernelGradient(b, Q);
    }
    VectorXf weight_gradient(int k, const MatrixXf& b, const MatrixXf& Q) const {
        return pairwise_[k]->gradient(b, Q);
    }
    VectorXf parameters(int k) const { return pairwise_[k]->parameters(); }
    VectorXf kernel_parameters(int k) const { return pairwise_[k]->kernelParameters(); }
    void set_kernel_parameters(int k, const VectorXf& v) { pairwise_[k]->setKernelParameters(v); }
    VectorXf unary_gradient(const MatrixXf& b) const { return unary_->gradient(b); }
    MatrixXf unary_get() const { return unary_->get(); }
    int N() const { return N_; }
    int L() const { return M_; }
    int R() const { return R_; }
    PairwisePotential* pw(int k) const { return pairwise_[k]; }
    PairwisePotential* pw_nonorm(int k) const { return no_norm_pairwise_[k]; }
    int num_pairwise() const { return (int)pairwise_.size(); }

    void set_cliques(int R, const int* offsets, const int* idx, const float* expw,
                     const float* constants) {
        super_pixel_container_.clear();
        constants_.clear();
        exp_of_superpixels_.resize(R);
        mean_of_superpixels_ = VectorXf::Zero(R);
        for (int r = 0; r < R; r++) {
            std::vector<double> px;
            for (int p = offsets[r]; p < offsets[r + 1]; p++) px.push_back((double)idx[p]);
            super_pixel_container_.push_back(px);
            exp_of_superpixels_[r] = expw[r];
            constants_.push_back(constants[r]);
        }
        R_ = R;
    }
    int clique_total() const {
        int t = 0;
        for (auto& c : super_pixel_container_) t += (int)c.size();
        return t;
    }
    void get_cliques(int* offsets, int* idx, float* expw, float* constants) const {
        int t = 0;
        for (int r = 0; r < R_; r++) {
            offsets[r] = t;
            for (double p : super_pixel_container_[r]) idx[t++] = (int)p;
            expw[r] = exp_of_superpixels_[r];
            constants[r] = constants_[r];
        }
        offsets[R_] = t;
    }

    // The QP loop of DenseCRF::qp_inference_super_pixels_non_convex
    // (src/densecrf.cpp:353-441) with its energy-decrease stop rule replaced by
    // a fixed iteration count; every operation is the reference's own
    // (PairwisePotential::apply, descent_direction, dotProduct,
    // multiplySuperPixels).  Returns the number of iterations run.
    int qp_fixed(const MatrixXf& init, MatrixXf& Qout, int iters, double* energies) {
        MatrixXf Q(M_, N_), unary(M_, N_), tmp(M_, N_), grad_y(M_, N_), cond_grad_y(M_, N_),
            grad_z(M_, R_), cond_grad_z(M_, R_), sx_z(M_, R_), sx_y(M_, N_), psisx(M_, N_),
            z_labels(M_, R_);
        MatrixP temp_dot(M_, N_);
        MatrixXf constant = exp_of_superpixels_.replicate(1, grad_z.rows()).transpose();
        grad_z.fill(0);
        cond_grad_z.fill(0);
        z_labels.fill(1);
        double optimal_step_size = 0;
        unary.fill(0);
        if (unary_) unary = unary_->get();
        Q = init;
        grad_z = (MatrixXf::Ones(M_, R_) + multiplySuperPixels((Q - MatrixXf::Ones(M_, N_))));
        grad_z = grad_z.cwiseProduct(constant);
        descent_direction_z(cond_grad_z, grad_z);
        grad_y = unary;
        for (unsigned int i = 0; i < pairwise_.size(); i++) {
            pairwise_[i]->apply(tmp, Q);
            grad_y += 2 * tmp;
        }
        grad_y += multiplySuperPixels((z_labels - MatrixXf::Ones(M_, R_)).cwiseProduct(constant));
        double energy = compute_LR_QP_value(Q, 0 * MatrixXf::Ones(M_, N_));
        energy += (z_labels.cwiseProduct(constant).sum() +
                   multiplySuperPixels((MatrixXf::Ones(M_, R_) - z_labels).cwiseProduct(constant),
                                       (Q - MatrixXf::Ones(M_, N_))));
        int it = 0;
        for (; it < iters; it++) {
            descent_direction(cond_grad_y, grad_y);
            descent_direction_z(cond_grad_z, grad_z);
            sx_y = cond_grad_y - Q;
            sx_z = cond_grad_z - z_labels;
            psisx.fill(0);
            for (unsigned int i = 0; i < pairwise_.size(); i++) {
                pairwise_[i]->apply(tmp, sx_y);
                psisx += tmp;
            }
            double a = multiplySuperPixels(sx_z.cwiseProduct(constant), (Q - MatrixXf::Ones(M_, N_)));
            double b = multiplySuperPixels((cond_grad_z - MatrixXf::Ones(M_, R_)).cwiseProduct(constant), sx_y);
            double num = dotProduct(unary, sx_y, temp_dot) + 2 * dotProduct(Q, psisx, temp_dot) + a + b + sx_z.sum();
            double denom = dotProduct(sx_y, psisx, temp_dot) + multiplySuperPixels(sx_z.cwiseProduct(constant), sx_y);
            optimal_step_size = -num / (2 * denom);
            if (denom == 0 || num == 0) break;
            if (denom < 0) optimal_step_size = 1;
            Q += optimal_step_size * sx_y;
            z_labels += optimal_step_size * sx_z;
            grad_y += 2 * optimal_step_size * psisx +
                      optimal_step_size * multiplySuperPixels((z_labels - MatrixXf::Ones(M_, R_)).cwiseProduct(constant));
            grad_z = MatrixXf::Ones(M_, R_).cwiseProduct(constant) +
                     (multiplySuperPixels(Q - MatrixXf::Ones(M_, N_))).cwiseProduct(constant);
            energy = dotProduct(Q, grad_y + unary, temp_dot);
            energy += (z_labels.cwiseProduct(constant).sum() +
                       multiplySuperPixels((MatrixXf::Ones(M_, R_) - z_labels).cwiseProduct(constant),
                                           (Q - MatrixXf::Ones(M_, N_))));
            if (energies) energies[it] = energy;
        }
        z_labels_ = z_labels;
        Qout = Q;
        return it;
    }
};

thread_local char g_err[512] = {0};

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err; }

// ---------------------------------------------------------------- lattice --
void* refl_new(const float* f, int d, int N) {
    MatrixXf F = Map<const MatrixXf>(f, d, N);
    LatticeProbe* p = new LatticeProbe();
    p->init(F);
    return p;
}
void refl_free(void* h) { delete (LatticeProbe*)h; }
int refl_M(void* h) { return ((LatticeProbe*)h)->M(); }
// offsets/ranks/barys: (d+1)*N entries of the first N pixels (pixel-major).
// nbr: (d+1)*M pairs (n1, n2), axis-major, raw reference ids (-1 = absent).
void refl_export(void* h, int* offset, int* rank, float* bary, int* nbr) {
    LatticeProbe* p = (LatticeProbe*)h;
    size_t E = (size_t)(p->d() + 1) * p->N();
    if (offset) std::memcpy(offset, p->offsets().data(), E * sizeof(int));
    if (rank) std::memcpy(rank, p->ranks().data(), E * sizeof(int));
    if (bary) std::memcpy(bary, p->barys().data(), E * sizeof(float));
    if (nbr) p->neighbours(nbr);
}
void refl_compute(void* h, float* out, const float* in, int L, int reverse) {
    LatticeProbe* p = (LatticeProbe*)h;
    MatrixXf I = Map<const MatrixXf>(in, L, p->N());
    MatrixXf O;
    p->compute(O, I, reverse != 0);
    std::memcpy(out, O.data(), sizeof(float) * (size_t)L * p->N());
}
// Permutohedral::gradient (src/permutohedral.cpp:1095-1178): df [N][d] of
// a^T K b with respect to the features; a, b [N][L].
void refl_gradient(void* h, float* df, const float* a, const float* b, int L) {
    LatticeProbe* p = (LatticeProbe*)h;
    p->gradient(df, a, b, L);
}
void refl_compute_ord(void* h, float* out, const float* in, int L) {
    LatticeProbe* p = (LatticeProbe*)h;
    MatrixXf I = Map<const MatrixXf>(in, L, p->N());
    MatrixXf O = MatrixXf::Zero(L, p->N());
    p->compute_upper_minus_lower_ord(O, I);
    std::memcpy(out, O.data(), sizeof(float) * (size_t)L * p->N());
}
// pI as the reference takes it, with one sentinel -1 in reserved storage
// right after its last element: the reference reads pI[pI.size()] once it
// has passed the last pI pixel (src/permutohedral.cpp:727-731), and the
// sentinel keeps that read defined and equal to "not in pI".
static std::vector<int> restricted_set(const int* pI, int nP) {
    std::vector<int> v;
    v.reserve((size_t)nP + 1);
    v.assign(pI, pI + nP);
    v.data()[nP] = -1;
    return v;
}
void refl_compute_ord_restricted(void* h, float* rout, const float* rQ, const int* pI, int nP, const float* Q, int L,
                                 int store) {
    LatticeProbe* p = (LatticeProbe*)h;
    std::vector<int> idx = restricted_set(pI, nP);
    MatrixXf RQ = Map<const MatrixXf>(rQ, L, nP);
    MatrixXf QQ = Q ? MatrixXf(Map<const MatrixXf>(Q, L, p->N())) : MatrixXf::Zero(L, p->N());
    MatrixXf O = MatrixXf::Zero(L, nP);
    p->compute_upper_minus_lower_ord_restricted(O, RQ, idx, QQ, store != 0);
    if (nP) std::memcpy(rout, O.data(), sizeof(float) * (size_t)L * nP);
}

// ------------------------------------------------------------------ model --
void* refm_new(int W, int H, int L, const float* unary) {
    RefModel* m = new RefModel(W, H, L);
    MatrixXf U = Map<const MatrixXf>(unary, L, W * H);
    m->setUnaryEnergy(U);
    return m;
}
void refm_free(void* h) { delete (RefModel*)h; }
void refm_add_gaussian(void* h, float sx, float sy, float w) {
    ((RefModel*)h)->addPairwiseGaussian(sx, sy, new PottsCompatibility(w));
}
void refm_add_bilateral(void* h, float sx, float sy, float sr, float sg, float sb,
                        const unsigned char* rgb, float w) {
    ((RefModel*)h)->addPairwiseBilateral(sx, sy, sr, sg, sb, rgb, new PottsCompatibility(w));
}
void refm_add_features(void* h, const float* f, int d, float w) {
    RefModel* m = (RefModel*)h;
    MatrixXf F = Map<const MatrixXf>(f, d, m->N());
    m->addPairwiseEnergy(F, new PottsCompatibility(w));
}
// addPairwiseEnergy(F, Potts(w), KernelType ktype, NormalizationType ntype).
void refm_add_features_kernel(void* h, const float* f, int d, float w, int ktype, int ntype) {
    RefModel* m = (RefModel*)h;
    MatrixXf F = Map<const MatrixXf>(f, d, m->N());
    m->addPairwiseEnergy(F, new PottsCompatibility(w), (KernelType)ktype, (NormalizationType)ntype);
}
int refm_kernel_parameters(void* h, int k, float* out) {
    VectorXf p = ((RefModel*)h)->kernel_parameters(k);
    if (p.size()) std::memcpy(out, p.data(), sizeof(float) * p.size());
    return (int)p.size();
}
void refm_set_kernel_parameters(void* h, int k, const float* p, int n) {
    ((RefModel*)h)->set_kernel_parameters(k, Map<const VectorXf>(p, n));
}
// Gaussian / bilateral term with a Diagonal (kind 1, params[L]) or Matrix
// (kind 2, params[L*L] column-major) compatibility.
static LabelCompatibility* make_compat(int kind, const float* params, int L) {
    if (kind == 1) return new DiagonalCompatibility(Map<const VectorXf>(params, L));
    if (kind == 2) return new MatrixCompatibility(Map<const MatrixXf>(params, L, L));
    return new PottsCompatibility(params[0]);
}
void refm_add_gaussian_compat(void* h, float sx, float sy, int kind, const float* params) {
    RefModel* m = (RefModel*)h;
    m->addPairwiseGaussian(sx, sy, make_compat(kind, params, m->L()));
}
void refm_add_bilateral_compat(void* h, float sx, float sy, float sr, float sg, float sb, const unsigned char* rgb,
                               int kind, const float* params) {
    RefModel* m = (RefModel*)h;
    m->addPairwiseBilateral(sx, sy, sr, sg, sb, rgb, make_compat(kind, params, m->L()));
}
int refm_add_superpixel(void* h, unsigned char* rgb, int sr, int rr, int minreg, float c, float nrm) {
    RefModel* m = (RefModel*)h;
    int before = m->R();
    m->addSuperPixel(rgb, sr, rr, minreg, c, nrm);
    return m->R() - before;
}
int refm_num_cliques(void* h) { return ((RefModel*)h)->R(); }
int refm_clique_total(void* h) { return ((RefModel*)h)->clique_total(); }
void refm_get_cliques(void* h, int* offsets, int* idx, float* expw, float* constants) {
    ((RefModel*)h)->get_cliques(offsets, idx, expw, constants);
}
void refm_set_cliques(void* h, int R, const int* offsets, const int* idx, const float* expw,
                      const float* constants) {
    ((RefModel*)h)->set_cliques(R, offsets, idx, expw, constants);
}
void refm_unary_init(void* h, float* Q) {
    MatrixXf q = ((RefModel*)h)->unary_init();
    std::memcpy(Q, q.data(), sizeof(float) * q.size());
}
void refm_apply(void* h, int k, int nonorm, float* out, const float* in) {
    RefModel* m = (RefModel*)h;
    MatrixXf I = Map<const MatrixXf>(in, m->L(), m->N());
    MatrixXf O;
    (nonorm ? m->pw_nonorm(k) : m->pw(k))->apply(O, I);
    std::memcpy(out, O.data(), sizeof(float) * O.size());
}
void refm_apply_ord_restricted(void* h, int k, float* rout, const float* rQ, const int* pI, int nP, const float* Q,
                               int store) {
    RefModel* m = (RefModel*)h;
    std::vector<int> idx = restricted_set(pI, nP);
    MatrixXf RQ = Map<const MatrixXf>(rQ, m->L(), nP);
    MatrixXf QQ = Q ? MatrixXf(Map<const MatrixXf>(Q, m->L(), m->N())) : MatrixXf::Zero(m->L(), m->N());
    MatrixXf O(m->L(), nP);
    m->pw(k)->apply_upper_minus_lower_ord_restricted(O, RQ, idx, QQ, store != 0);
    if (nP) std::memcpy(rout, O.data(), sizeof(float) * (size_t)m->L() * nP);
}
// PairwisePotential's exact and divide-and-conquer filters
// (src/pairwise.cpp:241-380) on pairwise_[k] or no_norm_pairwise_[k]; ind
// [N][L] (MatrixXi L x N), out [N][L].
void refm_apply_bf(void* h, int k, int nonorm, float* out, const float* Q) {
    RefModel* m = (RefModel*)h;
    MatrixXf I = Map<const MatrixXf>(Q, m->L(), m->N());
    MatrixXf O;
    (nonorm ? m->pw_nonorm(k) : m->pw(k))->apply_bf(O, I);
    std::memcpy(out, O.data(), sizeof(float) * O.size());
}
void refm_apply_sorted(void* h, int k, int nonorm, int kind, float* out, const int* ind, const float* Q) {
    RefModel* m = (RefModel*)h;
    MatrixXi I = Map<const MatrixXi>(ind, m->L(), m->N());
    MatrixXf O(m->L(), m->N());
    PairwisePotential* p = nonorm ? m->pw_nonorm(k) : m->pw(k);
    if (kind == 0) p->apply_upper_minus_lower_bf(O, I);
    else if (kind == 1) p->apply_upper_minus_lower_bf_ord(O, I, Map<const MatrixXf>(Q, m->L(), m->N()));
    else p->apply_upper_minus_lower_dc(O, I);
    std::memcpy(out, O.data(), sizeof(float) * O.size());
}
int refm_apply_ord(void* h, int k, float* out, const float* in) {
    RefModel* m = (RefModel*)h;
    MatrixXf I = Map<const MatrixXf>(in, m->L(), m->N());
    MatrixXf O(m->L(), m->N());
    try {
        m->pw(k)->apply_upper_minus_lower_ord(O, I);
    } catch (std::exception& e) {
        std::snprintf(g_err, sizeof(g_err), "%s", e.what());
        return -1;
    }
    std::memcpy(out, O.data(), sizeof(float) * O.size());
    return 0;
}
void refm_qp(void* h, const float* init, float* out) {
    RefModel* m = (RefModel*)h;
    MatrixXf I = Map<const MatrixXf>(init, m->L(), m->N());
    MatrixXf O = m->qp_inference_super_pixels_non_convex(I);
    std::memcpy(out, O.data(), sizeof(float) * O.size());
}
int refm_qp_fixed(void* h, const float* init, float* out, int iters, double* energies) {
    RefModel* m = (RefModel*)h;
    MatrixXf I = Map<const MatrixXf>(init, m->L(), m->N());
    MatrixXf O;
    int it = m->qp_fixed(I, O, iters, energies);
    std::memcpy(out, O.data(), sizeof(float) * O.size());
    return it;
}
int refm_lp(void* h, const float* init, float* out, float prox_reg_const, float dual_gap_tol,
            float prox_energy_tol, int prox_max_iter, int fw_max_iter, int qp_max_iter,
            float qp_tol, float qp_const, int best_int, int accel_prox, int work_set_size,
            int approx_fw_iter, float less_confident_percent, float confidence_tol) {
    RefModel* m = (RefModel*)h;
    LP_inf_params p(prox_reg_const, dual_gap_tol, prox_energy_tol, prox_max_iter, fw_max_iter,
                    qp_max_iter, qp_tol, qp_const, best_int != 0, accel_prox != 0, work_set_size,
                    approx_fw_iter, less_confident_percent, confidence_tol);
    MatrixXf I = Map<const MatrixXf>(init, m->L(), m->N());
    try {
        MatrixXf O = m->lp_inference_prox_super_pixels(I, p);
        std::memcpy(out, O.data(), sizeof(float) * O.size());
    } catch (std::exception& e) {
        std::snprintf(g_err, sizeof(g_err), "%s", e.what());
        return -1;
    }
    return 0;
}
void refm_current_map(void* h, const float* Q, short* labels) {
    RefModel* m = (RefModel*)h;
    MatrixXf I = Map<const MatrixXf>(Q, m->L(), m->N());
    VectorXs l = m->currentMap(I);
    std::memcpy(labels, l.data(), sizeof(short) * l.size());
}
double refm_energy_true(void* h, const short* labels) {
    RefModel* m = (RefModel*)h;
    VectorXs l = Map<const VectorXs>(labels, m->N());
    return m->assignment_energy_true(l);
}
// Kernel-parameter (feature scale) and Potts-weight gradients of term k;
// b, Q [N][L]; out receives d (kernel) or 1 (weight) floats.
int refm_kernel_gradient(void* h, int k, const float* b, const float* Q, float* out) {
    RefModel* m = (RefModel*)h;
    MatrixXf B = Map<const MatrixXf>(b, m->L(), m->N()), QQ = Map<const MatrixXf>(Q, m->L(), m->N());
    VectorXf g = m->kernel_gradient(k, B, QQ);
    std::memcpy(out, g.data(), sizeof(float) * g.size());
    return (int)g.size();
}
int refm_weight_gradient(void* h, int k, const float* b, const float* Q, float* out) {
    RefModel* m = (RefModel*)h;
    MatrixXf B = Map<const MatrixXf>(b, m->L(), m->N()), QQ = Map<const MatrixXf>(Q, m->L(), m->N());
    VectorXf g = m->weight_gradient(k, B, QQ);
    std::memcpy(out, g.data(), sizeof(float) * g.size());
    return (int)g.size();
}
// setUnaryEnergy(new LogisticUnaryEnergy(W (L x F), f (F x N))).
void refm_set_unary_logistic(void* h, const float* w, const float* f, int F) {
    RefModel* m = (RefModel*)h;
    m->setUnaryEnergy(new LogisticUnaryEnergy(Map<const MatrixXf>(w, m->L(), F), Map<const MatrixXf>(f, F, m->N())));
}
int refm_unary_get(void* h, float* out) {
    MatrixXf u = ((RefModel*)h)->unary_get();
    std::memcpy(out, u.data(), sizeof(float) * u.size());
    return (int)u.size();
}
int refm_unary_gradient(void* h, const float* b, float* out) {
    RefModel* m = (RefModel*)h;
    VectorXf g = m->unary_gradient(Map<const MatrixXf>(b, m->L(), m->N()));
    std::memcpy(out, g.data(), sizeof(float) * g.size());
    return (int)g.size();
}
// The reference's debugging energies and max_rounding (src/densecrf.cpp:832-957).
void refm_unary_energy(void* h, const short* labels, float* out) {
    RefModel* m = (RefModel*)h;
    VectorXf r = m->unaryEnergy(Map<const VectorXs>(labels, m->N()));
    std::memcpy(out, r.data(), sizeof(float) * r.size());
}
void refm_pairwise_energy(void* h, const short* labels, int term, float* out) {
    RefModel* m = (RefModel*)h;
    VectorXf r = m->pairwise_energy_true(Map<const VectorXs>(labels, m->N()), term);
    std::memcpy(out, r.data(), sizeof(float) * r.size());
}
void refm_max_rounding(void* h, const float* Q, float* out) {
    RefModel* m = (RefModel*)h;
    MatrixXf r = m->max_rounding(Map<const MatrixXf>(Q, m->L(), m->N()));
    std::memcpy(out, r.data(), sizeof(float) * r.size());
}
double refm_energy_qp_ho(void* h, const float* Q) {
    RefModel* m = (RefModel*)h;
    return m->compute_energy_higher_order(Map<const MatrixXf>(Q, m->L(), m->N()));
}
double refm_lr_qp_diag(void* h, const float* Q, const float* dd) {
    RefModel* m = (RefModel*)h;
    return m->compute_LR_QP_value(Map<const MatrixXf>(Q, m->L(), m->N()), Map<const MatrixXf>(dd, m->L(), m->N()));
}
int refm_parameters(void* h, int k, float* out) {
    VectorXf p = ((RefModel*)h)->parameters(k);
    std::memcpy(out, p.data(), sizeof(float) * p.size());
    return (int)p.size();
}
double refm_energy_ho(void* h, const short* labels) {
    RefModel* m = (RefModel*)h;
    VectorXs l = Map<const VectorXs>(labels, m->N());
    return m->assignment_energy_higher_order(l);
}
double refm_energy_lp(void* h, const float* Q) {
    RefModel* m = (RefModel*)h;
    MatrixXf I = Map<const MatrixXf>(Q, m->L(), m->N());
    return m->compute_energy_LP_higher_order(I);
}
double refm_lr_qp_value(void* h, const float* Q) {
    RefModel* m = (RefModel*)h;
    MatrixXf I = Map<const MatrixXf>(Q, m->L(), m->N());
    return m->compute_LR_QP_value(I, MatrixXf::Zero(m->L(), m->N()));
}

// ---- ProbImage (.c_unary) codec ------------------------------------------
// ref_probimage_compress: ProbImage::compress of a [H][W][D] float image
// (external/ProbImage/probimage.cpp:87-139).
int ref_probimage_compress(int W, int H, int D, const float* data, float eps, const char* path) {
    ProbImage p;
    FILE* fp = fopen(path, "wb");  // the codec only writes via its own save path: stage through a raw file
    if (!fp) return 1;
    uint32_t hdr[3] = {htonl((uint32_t)W), htonl((uint32_t)H), htonl((uint32_t)D)};
    fwrite(hdr, 4, 3, fp);
    std::vector<uint32_t> buf((size_t)W * H * D);
    for (size_t i = 0; i < buf.size(); i++) {
        uint32_t u;
        std::memcpy(&u, data + i, 4);
        buf[i] = htonl(u);
    }
    fwrite(buf.data(), 4, buf.size(), fp);
    fclose(fp);
    p.load(path);
    p.compress(path, eps);
    return 0;
}
// The unaries load_unary derives from a .c_unary file (src/file_storage.cpp:
// 261-285): decompress, boostToProb, then -log per (pixel, label); out is
// [N][D] (pixel = y * W + x).  Returns W, H, D through the pointers; out may
// be NULL to query the size.
int ref_load_unary(const char* path, float* out, int* W, int* H, int* D) {
    ProbImage t;
    t.decompress(path);
    t.boostToProb();
    *W = t.width();
    *H = t.height();
    *D = t.depth();
    if (out)
        for (int i = 0; i < t.height(); i++)
            for (int j = 0; j < t.width(); j++)
                for (int k = 0; k < t.depth(); k++)
                    out[((size_t)i * t.width() + j) * t.depth() + k] = -log(t(j, i, k));
    return 0;
}

// EDISON's mean shift as addSuperPixel drives it (src/densecrf.cpp:206-210):
// the filtered L*u*v* image of Filter(spatial, range, NO_SPEEDUP), and the
// region labels of Segment(spatial, range, min_region, NO_SPEEDUP).
void refms_filter(unsigned char* rgb, int W, int H, int sr, float rr, float* out) {
    msImageProcessor p;
    p.DefineImage(rgb, COLOR, H, W);
    p.Filter(sr, rr, NO_SPEEDUP);
    p.GetRawData(out);
}
int refms_segment(unsigned char* rgb, int W, int H, int sr, float rr, int minreg, int* labels) {
    msImageProcessor p;
    p.DefineImage(rgb, COLOR, H, W);
    p.Segment(sr, rr, minreg, NO_SPEEDUP);
    std::vector<int> lab;
    const int n = p.GetRegions(lab);
    std::memcpy(labels, lab.data(), sizeof(int) * lab.size());
    return n;
}

}  // extern "C"
