// densecrf.h -- drop-in C++ API of densecrf_ho, running on the B200 engine.
//
// The classes and signatures below are those of the reference's public
// headers (include/densecrf.h:43-194, include/pairwise.h:33-95,
// include/permutohedral.h:50-88, include/labelcompatibility.h,
// include/unary.h); a caller switches by putting this directory first on its
// include path and linking libdcrf_cuda.so.  Every method forwards to the C
// ABI of include/dcrf.h; errors the reference reports with exceptions
// ("Value out of bounds", "Maxval < 0, skipping") are thrown as
// std::runtime_error with the same text, every other failure too.
//
// Scope (the B200 path): Potts, Diagonal and Matrix compatibilities, every
// KernelType and NormalizationType (and the NO_NORMALIZATION copy), constant unaries, the
// qp / lp / qp_sp / lp_sp solvers.  addSuperPixel keeps the reference's
// signature: the engine runs EDISON's mean-shift segmentation itself (the
// mode search on the GPU) and derives the clique weights as
// src/densecrf.cpp:212-247 does; an overload also takes a caller's region map.
//
// Header-only; needs Eigen (the reference vendors 3.2.7) and include/dcrf.h.
#pragma once
#include <Eigen/Core>

#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "dcrf.h"

using namespace Eigen;

typedef Matrix<short, Dynamic, 1> VectorXs;

namespace dcrf_shim {
inline void check(dcrf_status s) {
    if (s != DCRF_OK) throw std::runtime_error(dcrf_last_error());
}
}  // namespace dcrf_shim

// ---------------------------------------------------------------- pairwise.h --
enum NormalizationType { NO_NORMALIZATION, NORMALIZE_BEFORE, NORMALIZE_AFTER, NORMALIZE_SYMMETRIC };
enum KernelType { CONST_KERNEL, DIAG_KERNEL, FULL_KERNEL };

// ------------------------------------------------------ labelcompatibility.h --
// The compatibilities hold their parameters on the host; the model gets them
// through dcrf_model_set_compat when the term is added.
class LabelCompatibility {
public:
    virtual ~LabelCompatibility() {}
    virtual MatrixXf matrixForm(int nb_labels) const = 0;
    virtual VectorXf parameters() const = 0;
    virtual void setParameters(const VectorXf& v) = 0;
    // DCRF_COMPAT_* kind and its dcrf_model_set_compat parameters.
    virtual int kind() const = 0;
    virtual std::vector<float> abi_params() const = 0;
};

class PottsCompatibility : public LabelCompatibility {
protected:
    float w_;
public:
    PottsCompatibility(float weight = 1.0) : w_(weight) {}
    MatrixXf matrixForm(int nb_labels) const override {
        return MatrixXf(-w_ * MatrixXf::Identity(nb_labels, nb_labels));
    }
    VectorXf parameters() const override {
        VectorXf r(1);
        r[0] = w_;
        return r;
    }
    void setParameters(const VectorXf& v) override { w_ = v[0]; }
    int kind() const override { return DCRF_COMPAT_POTTS; }
    std::vector<float> abi_params() const override { return {w_}; }
};

class DiagonalCompatibility : public LabelCompatibility {
protected:
    VectorXf w_;
public:
    DiagonalCompatibility(const VectorXf& v) : w_(v) {}
    MatrixXf matrixForm(int) const override { return MatrixXf(w_.asDiagonal()); }
    VectorXf parameters() const override { return w_; }
    void setParameters(const VectorXf& v) override { w_ = v; }
    int kind() const override { return DCRF_COMPAT_DIAGONAL; }
    std::vector<float> abi_params() const override { return std::vector<float>(w_.data(), w_.data() + w_.size()); }
};

class MatrixCompatibility : public LabelCompatibility {
protected:
    MatrixXf w_;
public:
    MatrixCompatibility(const MatrixXf& m) : w_(0.5 * (m + m.transpose())) {}
    MatrixXf matrixForm(int) const override { return w_; }
    VectorXf parameters() const override {
        VectorXf r(w_.cols() * (w_.rows() + 1) / 2);
        for (int i = 0, k = 0; i < w_.cols(); i++)
            for (int j = i; j < w_.rows(); j++, k++) r[k] = w_(i, j);
        return r;
    }
    void setParameters(const VectorXf& v) override {
        for (int i = 0, k = 0; i < w_.cols(); i++)
            for (int j = i; j < w_.rows(); j++, k++) w_(j, i) = w_(i, j) = v[k];
    }
    int kind() const override { return DCRF_COMPAT_MATRIX; }
    // already symmetric, so the model's symmetrisation leaves it as it is
    std::vector<float> abi_params() const override { return std::vector<float>(w_.data(), w_.data() + w_.size()); }
};

namespace dcrf_shim {
// A term's compatibility as the C ABI takes it; owns f, as the reference does.
struct Compat {
    int kind = DCRF_COMPAT_POTTS;
    std::vector<float> p;  // p[0] is parameters()(0) for every kind
};
inline Compat take_compat(LabelCompatibility* f) {
    std::unique_ptr<LabelCompatibility> own(f);
    if (!f) throw std::runtime_error("a pairwise term needs a LabelCompatibility");
    Compat c;
    c.kind = f->kind();
    c.p = f->abi_params();
    return c;
}
// Gives term k of model m, added with weight c.p[0], compatibility c.
inline void set_compat(dcrf_model m, int k, const Compat& c) {
    if (c.kind != DCRF_COMPAT_POTTS && dcrf_model_set_compat(m, k, c.kind, c.p.data()) != DCRF_OK)
        throw std::runtime_error(dcrf_last_error());
}
// Gives term k of model m the kernel and normalisation types (the model's
// terms start as DIAG_KERNEL, NORMALIZE_SYMMETRIC).
inline void check_types(KernelType kt, NormalizationType nt) {  // before a term is added
    if ((int)kt < CONST_KERNEL || (int)kt > FULL_KERNEL) throw std::runtime_error("unknown kernel type");
    if ((int)nt < NO_NORMALIZATION || (int)nt > NORMALIZE_SYMMETRIC)
        throw std::runtime_error("unknown normalization type");
}
inline void set_kernel(dcrf_model m, int k, KernelType kt, NormalizationType nt) {
    if (kt == DIAG_KERNEL && nt == NORMALIZE_SYMMETRIC) return;
    if (dcrf_model_set_kernel(m, k, (int)kt, (int)nt) != DCRF_OK) throw std::runtime_error(dcrf_last_error());
}
}  // namespace dcrf_shim

// -------------------------------------------------------------------- unary.h --
class UnaryEnergy {
public:
    virtual ~UnaryEnergy() {}
    virtual MatrixXf get() const = 0;
};

class ConstUnaryEnergy : public UnaryEnergy {
protected:
    MatrixXf unary_;
public:
    ConstUnaryEnergy(const MatrixXf& unary) : unary_(unary) {}
    MatrixXf get() const override { return unary_; }
};

// ------------------------------------------------------------ permutohedral.h --
class Permutohedral {
    dcrf_lattice h_ = nullptr;
    int N_ = 0, M_ = 0, d_ = 0;
    Permutohedral(const Permutohedral&) = delete;
    Permutohedral& operator=(const Permutohedral&) = delete;
public:
    Permutohedral() { dcrf_shim::check(dcrf_lattice_create(&h_)); }
    ~Permutohedral() {
        if (h_) dcrf_lattice_destroy(h_);
    }
    // Permutohedral::init (src/permutohedral.cpp:152): features d x N.
    void init(const MatrixXf& features) {
        d_ = (int)features.rows();
        N_ = (int)features.cols();
        dcrf_shim::check(dcrf_lattice_init(h_, features.data(), d_, N_));
        dcrf_shim::check(dcrf_lattice_info(h_, &M_, nullptr, nullptr));
    }
    MatrixXf compute(const MatrixXf& v, bool reverse = false) const {
        MatrixXf r;
        compute(r, v, reverse);
        return r;
    }
    // Permutohedral::compute (src/permutohedral.cpp:1079): in L x N.
    void compute(MatrixXf& out, const MatrixXf& in, bool reverse = false) const {
        MatrixXf src = in;  // out may alias in
        out.resize(in.rows(), in.cols());
        dcrf_shim::check(dcrf_lattice_compute(h_, out.data(), src.data(), (int)in.rows(), reverse ? 1 : 0));
    }
    // Permutohedral::compute_upper_minus_lower_ord (src/permutohedral.cpp:1071).
    void compute_upper_minus_lower_ord(MatrixXf& out, const MatrixXf& Q) {
        out.resize(Q.rows(), Q.cols());
        dcrf_shim::check(dcrf_lattice_compute_ord(h_, out.data(), Q.data(), (int)Q.rows()));
    }
    int size() const { return M_; }
};

// ---------------------------------------------------------------- densecrf.h --
class LP_inf_params {
public:
    float prox_reg_const, dual_gap_tol, prox_energy_tol;
    int prox_max_iter, fw_max_iter, qp_max_iter;
    float qp_tol, qp_const;
    bool best_int, accel_prox;
    int work_set_size, approx_fw_iter;
    float less_confident_percent, confidence_tol;
    LP_inf_params(float prox_reg_const, float dual_gap_tol, float prox_energy_tol, int prox_max_iter,
                  int fw_max_iter, int qp_max_iter, float qp_tol, float qp_const, bool best_int, bool accel_prox,
                  int work_set_size, int approx_fw_iter, float less_confident_percent, float confident_tol)
        : prox_reg_const(prox_reg_const), dual_gap_tol(dual_gap_tol), prox_energy_tol(prox_energy_tol),
          prox_max_iter(prox_max_iter), fw_max_iter(fw_max_iter), qp_max_iter(qp_max_iter), qp_tol(qp_tol),
          qp_const(qp_const), best_int(best_int), accel_prox(accel_prox), work_set_size(work_set_size),
          approx_fw_iter(approx_fw_iter), less_confident_percent(less_confident_percent),
          confidence_tol(confident_tol) {}
    // LP_inf_params() (src/densecrf.cpp:287-302)
    LP_inf_params() {
        dcrf_lp_params p;
        dcrf_lp_params_default(&p);
        *this = from(p);
    }
    dcrf_lp_params to_c() const {
        dcrf_lp_params p;
        p.prox_reg_const = prox_reg_const;
        p.dual_gap_tol = dual_gap_tol;
        p.prox_energy_tol = prox_energy_tol;
        p.prox_max_iter = prox_max_iter;
        p.fw_max_iter = fw_max_iter;
        p.qp_max_iter = qp_max_iter;
        p.qp_tol = qp_tol;
        p.qp_const = qp_const;
        p.best_int = best_int;
        p.accel_prox = accel_prox;
        p.work_set_size = work_set_size;
        p.approx_fw_iter = approx_fw_iter;
        p.less_confident_percent = less_confident_percent;
        p.confidence_tol = confidence_tol;
        return p;
    }
private:
    static LP_inf_params from(const dcrf_lp_params& p) {
        return LP_inf_params(p.prox_reg_const, p.dual_gap_tol, p.prox_energy_tol, p.prox_max_iter, p.fw_max_iter,
                             p.qp_max_iter, p.qp_tol, p.qp_const, p.best_int != 0, p.accel_prox != 0,
                             p.work_set_size, p.approx_fw_iter, p.less_confident_percent, p.confidence_tol);
    }
};

// A standalone PairwisePotential (include/pairwise.h:63-95): its lattice lives
// in a one-term model over N = features.cols() pixels, created for the label
// count of the first apply.
class PairwisePotential {
    MatrixXf f_;
    dcrf_shim::Compat c_;
    KernelType kt_;
    NormalizationType nt_;
    int L_ = 0;
    dcrf_model m_ = nullptr;
    PairwisePotential(const PairwisePotential&) = delete;
    void ensure(int L) {
        if (m_ && L == L_) return;
        if (m_) dcrf_model_destroy(m_);
        m_ = nullptr;
        dcrf_shim::check(dcrf_model_create(&m_, (int)f_.cols(), 1, L));
        dcrf_shim::check(dcrf_model_add_pairwise(m_, f_.data(), (int)f_.rows(), c_.p.at(0)));
        dcrf_shim::set_compat(m_, 0, c_);
        dcrf_shim::set_kernel(m_, 0, kt_, nt_);
        L_ = L;
    }
    void sorted(MatrixXf& out, const MatrixXi& ind, const MatrixXf* Q, int kind) const {
        auto* self = const_cast<PairwisePotential*>(this);
        self->ensure((int)ind.rows());
        Eigen::Matrix<int32_t, Eigen::Dynamic, Eigen::Dynamic> idx = ind.cast<int32_t>();
        out.resize(ind.rows(), ind.cols());
        if (kind == 0)
            dcrf_shim::check(dcrf_model_pairwise_apply_upper_minus_lower_bf(m_, 0, 0, out.data(), idx.data()));
        else if (kind == 1) {
            MatrixXf src = *Q;
            dcrf_shim::check(
                dcrf_model_pairwise_apply_upper_minus_lower_bf_ord(m_, 0, 0, out.data(), idx.data(), src.data()));
        } else
            dcrf_shim::check(dcrf_model_pairwise_apply_upper_minus_lower_dc(m_, 0, 0, out.data(), idx.data()));
    }
public:
    PairwisePotential(const MatrixXf& features, LabelCompatibility* compatibility, KernelType ktype = CONST_KERNEL,
                      NormalizationType ntype = NORMALIZE_SYMMETRIC)
        : f_(features), c_(dcrf_shim::take_compat(compatibility)), kt_(ktype), nt_(ntype) {
        dcrf_shim::check_types(ktype, ntype);
    }
    ~PairwisePotential() {
        if (m_) dcrf_model_destroy(m_);
    }
    // PairwisePotential::apply (src/pairwise.cpp:203-208)
    void apply(MatrixXf& out, const MatrixXf& Q) const {
        auto* self = const_cast<PairwisePotential*>(this);
        self->ensure((int)Q.rows());
        MatrixXf src = Q;
        out.resize(Q.rows(), Q.cols());
        dcrf_shim::check(dcrf_model_pairwise_apply(m_, 0, 0, out.data(), src.data()));
    }
    // PairwisePotential::apply_upper_minus_lower_ord (src/pairwise.cpp:214-228)
    void apply_upper_minus_lower_ord(MatrixXf& out, const MatrixXf& Q) {
        ensure((int)Q.rows());
        MatrixXf src = Q;
        out.resize(Q.rows(), Q.cols());
        dcrf_shim::check(dcrf_model_pairwise_apply_ord(m_, 0, out.data(), src.data()));
    }
    // The exact filters and the divide-and-conquer filter
    // (src/pairwise.cpp:241-380); ind is L x N (sortRows), out L x N in
    // sorted positions for the sorted variants.
    void apply_bf(MatrixXf& out, const MatrixXf& Q) const {
        auto* self = const_cast<PairwisePotential*>(this);
        self->ensure((int)Q.rows());
        MatrixXf src = Q;
        out.resize(Q.rows(), Q.cols());
        dcrf_shim::check(dcrf_model_pairwise_apply_bf(m_, 0, 0, out.data(), src.data()));
    }
    void apply_upper_minus_lower_dc(MatrixXf& out, const MatrixXi& ind) const {
        sorted(out, ind, nullptr, 2);
    }
    void apply_upper_minus_lower_bf(MatrixXf& out, const MatrixXi& ind) const { sorted(out, ind, nullptr, 0); }
    void apply_upper_minus_lower_bf_ord(MatrixXf& out, const MatrixXi& ind, const MatrixXf& Q) const {
        sorted(out, ind, &Q, 1);
    }
    VectorXf parameters() const {
        if (c_.kind == DCRF_COMPAT_MATRIX) {  // the upper triangle by column
            const int L = (int)std::lround(std::sqrt((double)c_.p.size()));
            VectorXf r(L * (L + 1) / 2);
            for (int i = 0, k = 0; i < L; i++)
                for (int j = i; j < L; j++, k++) r[k] = c_.p[(size_t)j * L + i];
            return r;
        }
        return Map<const VectorXf>(c_.p.data(), (long)c_.p.size());
    }
    MatrixXf features() const { return f_; }
};

class DenseCRF {
protected:
    int N_, M_, R_ = 0;
    dcrf_model m_ = nullptr;
    int n_terms_ = 0;
    std::unique_ptr<UnaryEnergy> unary_snapshot_;
    // cliques (super_pixel_container_, exp_of_superpixels_, constants_)
    std::vector<int> cl_off_{0}, cl_idx_;
    std::vector<float> cl_exp_, cl_const_;
    DenseCRF(DenseCRF&) = delete;
    // The model's cliques back into the host copies (after the engine
    // appended some).
    void pull_cliques() {
        int R = 0, total = 0;
        dcrf_shim::check(dcrf_model_clique_info(m_, &R, &total));
        cl_off_.assign(R + 1, 0);
        cl_idx_.assign(total, 0);
        cl_exp_.assign(R, 0.0f);
        cl_const_.assign(R, 0.0f);
        dcrf_shim::check(dcrf_model_get_cliques(m_, cl_off_.data(), cl_idx_.data(), cl_exp_.data(),
                                                cl_const_.data()));
        R_ = R;
    }
    void push_cliques() {
        dcrf_shim::check(dcrf_model_set_cliques(m_, R_, cl_off_.data(), cl_idx_.empty() ? nullptr : cl_idx_.data(),
                                                cl_exp_.data(), cl_const_.data()));
    }
    DenseCRF(int W, int H, int M) : N_(W * H), M_(M) { dcrf_shim::check(dcrf_model_create(&m_, W, H, M)); }

public:
    virtual ~DenseCRF() {
        if (m_) dcrf_model_destroy(m_);
    }
    // DenseCRF::addPairwiseEnergy (src/densecrf.cpp:157-169)
    virtual void addPairwiseEnergy(const MatrixXf& features, LabelCompatibility* function,
                                   KernelType kernel_type = DIAG_KERNEL,
                                   NormalizationType normalization_type = NORMALIZE_SYMMETRIC) {
        const dcrf_shim::Compat c = dcrf_shim::take_compat(function);
        dcrf_shim::check_types(kernel_type, normalization_type);
        dcrf_shim::check(dcrf_model_add_pairwise(m_, features.data(), (int)features.rows(), c.p.at(0)));
        const int k = n_terms_++;
        dcrf_shim::set_compat(m_, k, c);
        dcrf_shim::set_kernel(m_, k, kernel_type, normalization_type);
    }
    void setUnaryEnergy(const MatrixXf& unary) { dcrf_shim::check(dcrf_model_set_unary(m_, unary.data())); }
    void setUnaryEnergy(UnaryEnergy* unary) {
        std::unique_ptr<UnaryEnergy> own(unary);
        setUnaryEnergy(unary->get());
    }
    // unary_init (src/densecrf.cpp:321-325)
    MatrixXf unary_init() const {
        MatrixXf Q(M_, N_);
        dcrf_shim::check(dcrf_model_unary_init(m_, Q.data()));
        return Q;
    }
    // qp_inference_super_pixels_non_convex (src/densecrf.cpp:340-442)
    const MatrixXf qp_inference_super_pixels_non_convex(const MatrixXf& init) {
        MatrixXf out(M_, N_);
        dcrf_shim::check(dcrf_model_qp(m_, init.data(), out.data(), nullptr, nullptr));
        return out;
    }
    // lp_inference_prox_super_pixels (src/densecrf.cpp:526-799)
    const MatrixXf lp_inference_prox_super_pixels(const MatrixXf& init, const LP_inf_params& params) const {
        MatrixXf out(M_, N_);
        const dcrf_lp_params p = params.to_c();
        dcrf_shim::check(dcrf_model_lp(m_, init.data(), out.data(), &p, nullptr));
        return out;
    }
    // max_rounding (src/densecrf.cpp:832-840)
    MatrixXf max_rounding(const MatrixXf& estimates) const {
        MatrixXf r(estimates.rows(), estimates.cols());
        dcrf_shim::check(dcrf_model_max_rounding(m_, estimates.data(), r.data()));
        return r;
    }
    // unaryEnergy / pairwise_energy_true (src/densecrf.cpp:887-927)
    VectorXf unaryEnergy(const VectorXs& l) const {
        VectorXf r(N_);
        dcrf_shim::check(dcrf_model_unary_energy(m_, l.data(), r.data()));
        return r;
    }
    VectorXf pairwise_energy_true(const VectorXs& l, int term = -1) const {
        VectorXf r(N_);
        dcrf_shim::check(dcrf_model_pairwise_energy(m_, l.data(), term, r.data()));
        return r;
    }
    // compute_energy_higher_order (src/densecrf.cpp:960-980)
    double compute_energy_higher_order(const MatrixXf& Q) const {
        double e = 0;
        dcrf_shim::check(dcrf_model_energy_higher_order(m_, Q.data(), &e));
        return e;
    }
    // getUnaryEnergy (src/densecrf.cpp:268-270): a snapshot of the unary in
    // use, owned by the model like the reference's pointer.
    UnaryEnergy* getUnaryEnergy() {
        MatrixXf u(M_, N_);
        dcrf_shim::check(dcrf_model_get_unary(m_, u.data()));
        unary_snapshot_.reset(new ConstUnaryEnergy(u));
        return unary_snapshot_.get();
    }
    // setUnaryEnergy(L, f): LogisticUnaryEnergy (src/densecrf.cpp:264-267)
    void setUnaryEnergy(const MatrixXf& L, const MatrixXf& f) {
        dcrf_shim::check(dcrf_model_set_unary_logistic(m_, L.data(), f.data(), (int)f.rows()));
    }
    VectorXs currentMap(const MatrixXf& Q) const {
        VectorXs l(Q.cols());
        dcrf_shim::check(dcrf_model_current_map(m_, Q.data(), l.data()));
        return l;
    }
    double assignment_energy_higher_order(const VectorXs& l) const {
        double e = 0;
        dcrf_shim::check(dcrf_model_energy_ho(m_, l.data(), &e));
        return e;
    }
    double assignment_energy_true(const VectorXs& l) const {
        double e = 0;
        dcrf_shim::check(dcrf_model_energy_true(m_, l.data(), &e));
        return e;
    }
    double compute_energy_LP_higher_order(const MatrixXf& Q) const {
        double e = 0;
        dcrf_shim::check(dcrf_model_energy_lp(m_, Q.data(), &e));
        return e;
    }
    double compute_LR_QP_value(const MatrixXf& Q, const MatrixXf& diag_dom) const {
        double e = 0;
        dcrf_shim::check(dcrf_model_lr_qp_value_diag(m_, Q.data(), diag_dom.size() ? diag_dom.data() : nullptr, &e));
        return e;
    }
    // addSuperPixel (include/densecrf.h:190, src/densecrf.cpp:193-251):
    // mean-shift regions of img at the given radii, each appended as a clique.
    void addSuperPixel(unsigned char* img, int spatial_radius, int range_radius, int min_region_count,
                       float constant, float normaliser) {
        int reg = 0;
        dcrf_shim::check(dcrf_model_add_superpixel(m_, img, spatial_radius, range_radius, min_region_count,
                                                   constant, normaliser, &reg));
        pull_cliques();
    }
    // The clique state addSuperPixel leaves behind (src/densecrf.cpp:212-247),
    // from a segmentation computed by the caller: region_of_pixel[i] in
    // [0, n_regions).  Means and grey-level deviations follow the reference,
    // including its img[i], img[i+1], img[i+2] reads (:222-233).
    void addSuperPixel(const std::vector<int>& region_of_pixel, int n_regions, const unsigned char* img,
                       float constant, float normaliser) {
        std::vector<std::vector<int>> members(n_regions);
        VectorXf count = VectorXf::Zero(n_regions), mean = VectorXf::Zero(n_regions),
                 sd = VectorXf::Zero(n_regions);
        for (int i = 0; i < N_; i++) {
            const int r = region_of_pixel[i];
            members[r].push_back(i);
            mean(r) += 0.2989 * (double)img[i];
            mean(r) += 0.5870 * (double)img[i + 1];
            mean(r) += 0.1140 * (double)img[i + 2];
            count(r) += 1;
        }
        mean = mean.cwiseQuotient(count);
        for (int i = 0; i < N_; i++) {
            const int r = region_of_pixel[i];
            const double g = 0.2989 * (double)img[i] + 0.5870 * (double)img[i + 1] + 0.1140 * (double)img[i + 2];
            sd(r) += (mean(r) - g) * (mean(r) - g);
        }
        sd = sd.cwiseQuotient(normaliser * count);
        const VectorXf ex = constant * (-1 * sd.array()).exp();
        for (int r = 0; r < n_regions; r++) {
            cl_idx_.insert(cl_idx_.end(), members[r].begin(), members[r].end());
            cl_off_.push_back((int)cl_idx_.size());
            cl_exp_.push_back(ex[r]);
            cl_const_.push_back(constant);
        }
        R_ += n_regions;
        push_cliques();
    }
};

class DenseCRF2D : public DenseCRF {
protected:
    int W_, H_;
public:
    DenseCRF2D(int W, int H, int M) : DenseCRF(W, H, M), W_(W), H_(H) {}
    // addPairwiseGaussian (src/densecrf.cpp:170-178)
    void addPairwiseGaussian(float sx, float sy, LabelCompatibility* function = NULL,
                             KernelType kernel_type = DIAG_KERNEL,
                             NormalizationType normalization_type = NORMALIZE_SYMMETRIC) {
        const dcrf_shim::Compat c = dcrf_shim::take_compat(function);
        dcrf_shim::check_types(kernel_type, normalization_type);
        dcrf_shim::check(dcrf_model_add_gaussian(m_, sx, sy, c.p.at(0)));
        const int k = n_terms_++;
        dcrf_shim::set_compat(m_, k, c);
        dcrf_shim::set_kernel(m_, k, kernel_type, normalization_type);
    }
    // addPairwiseBilateral (src/densecrf.cpp:179-190)
    void addPairwiseBilateral(float sx, float sy, float sr, float sg, float sb, const unsigned char* im,
                              LabelCompatibility* function = NULL, KernelType kernel_type = DIAG_KERNEL,
                              NormalizationType normalization_type = NORMALIZE_SYMMETRIC) {
        const dcrf_shim::Compat c = dcrf_shim::take_compat(function);
        dcrf_shim::check_types(kernel_type, normalization_type);
        dcrf_shim::check(dcrf_model_add_bilateral(m_, sx, sy, sr, sg, sb, im, c.p.at(0)));
        const int k = n_terms_++;
        dcrf_shim::set_compat(m_, k, c);
        dcrf_shim::set_kernel(m_, k, kernel_type, normalization_type);
    }
    using DenseCRF::setUnaryEnergy;
};
