/* dcrf.h -- C ABI of the B200 dense-CRF engine (libdcrf_cuda.so).
 *
 * A drop-in for the hot path of densecrf_ho: the permutohedral lattice, the
 * Potts pairwise potentials, and the qp / lp / qp_sp / lp_sp solvers.  The
 * reference has no FFI; its boundary is its C++ class API, and every entry
 * point below names the reference member function it replaces (file:line in
 * the densecrf_ho tree).  A C++ shim with the reference's own class names and
 * signatures is layered on top of this ABI (densecrf_ho_b200/cpp/).
 *
 * Conventions
 *  - Every call returns a dcrf_status; dcrf_last_error() gives the message of
 *    the last failure on the calling thread.
 *  - Label matrices are float32 in the reference's Eigen column-major L x N
 *    storage: element (label k, pixel i) at [i*L + k].
 *  - Feature matrices are float32 [i*d + c] (Eigen d x N column-major).
 *  - Functions without a suffix take HOST pointers and copy through pinned
 *    staging buffers; *_dev variants take device pointers, run on the
 *    handle's stream and return without synchronising.
 *  - A handle owns one CUDA stream and its device buffers; handles are
 *    independent, a handle is not re-entrant (like the reference objects).
 *  - All compute runs on the device that was current when the handle was
 *    created.  There is no CPU fallback: without a usable GPU every call
 *    fails with DCRF_E_CUDA.
 */
#ifndef DCRF_H
#define DCRF_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    DCRF_OK = 0,
    DCRF_E_ARG = 1,     /* invalid argument / size                               */
    DCRF_E_CUDA = 2,    /* CUDA runtime or launch failure                        */
    DCRF_E_RANGE = 3,   /* "Value out of bounds" (src/pairwise.cpp:218-219)      */
    DCRF_E_STATE = 4,   /* call order (e.g. solve before set_unary)              */
    DCRF_E_NOMEM = 5,   /* device allocation failed                              */
    DCRF_E_NUMERIC = 6, /* "Maxval < 0, skipping" (src/eigen_utils.cpp:138), or a
                           NaN / infinity in a solver's input or iterate        */
    DCRF_E_TIMEOUT = 7  /* a bounded device loop hit its iteration cap           */
} dcrf_status;

typedef struct dcrf_lattice_s* dcrf_lattice;
typedef struct dcrf_model_s* dcrf_model;

/* Device memory freed by a destroyed model, lattice or batch stays cached in
 * the process for the next one (up to DCRF_CACHE_MB MiB from the
 * environment; by default a quarter of the device's memory, at least 2048
 * MiB); this hands every cached block back to the driver.  No
 * counterpart in the reference, which allocates on the host. */
dcrf_status dcrf_release_cached_memory(void);
/* A budget on the device memory the library holds for live models, lattices
 * and batches (bytes; 0 = none, the default).  A request beyond it fails with
 * DCRF_E_NOMEM before any device call.  No counterpart in the reference. */
dcrf_status dcrf_set_device_memory_limit(uint64_t bytes);
/* Bytes held by live models / lattices / batches, bytes kept in the cache,
 * and the number of cudaMalloc calls the library has made (any may be NULL).
 * No counterpart in the reference. */
dcrf_status dcrf_device_memory_stats(uint64_t* in_use, uint64_t* cached, uint64_t* mallocs);

const char* dcrf_last_error(void);
/* Library version string. */
const char* dcrf_version(void);
/* Number of CUDA kernels this process has launched through the library
 * (diagnostics; no counterpart in the reference). */
unsigned long long dcrf_kernel_launches(void);

/* ------------------------------------------------------------------------
 * Permutohedral lattice -- class Permutohedral (include/permutohedral.h:50-88)
 * ---------------------------------------------------------------------- */

/* Permutohedral::Permutohedral() (src/permutohedral.cpp:139). */
dcrf_status dcrf_lattice_create(dcrf_lattice* out);
/* Permutohedral::~Permutohedral() (src/permutohedral.cpp:142). */
dcrf_status dcrf_lattice_destroy(dcrf_lattice lat);
/* Permutohedral::init(const MatrixXf& features) (src/permutohedral.cpp:152):
 * features [N][d], 1 <= d <= 16. */
dcrf_status dcrf_lattice_init(dcrf_lattice lat, const float* features, int d, int N);
dcrf_status dcrf_lattice_init_dev(dcrf_lattice lat, const float* d_features, int d, int N);
/* M_ (number of lattice vertices), N_ and d_. */
dcrf_status dcrf_lattice_info(dcrf_lattice lat, int* M, int* N, int* d);
/* Permutohedral::compute(MatrixXf& out, const MatrixXf& in, bool reverse)
 * (src/permutohedral.cpp:1079-1087): out = alpha S^T B S in, in/out [N][L]. */
dcrf_status dcrf_lattice_compute(dcrf_lattice lat, float* out, const float* in, int L, int reverse);
dcrf_status dcrf_lattice_compute_dev(dcrf_lattice lat, float* d_out, const float* d_in, int L,
                                     int reverse);
/* The filter of dcrf_lattice_compute_dev without any device allocation (no
 * counterpart in the reference).  For callers that may not allocate device
 * memory during a call -- hosts that give out all GPU memory from their own
 * pool, or that run under a fixed memory budget in a latency-critical loop --
 * the filter's scratch (two value buffers of (M + 1) x L floats) comes from a
 * fixed 32 MiB device array that every GPU loading the library holds until
 * exit.  Limit: 2 x (M + 1) x L <= 8 Mi floats, otherwise DCRF_E_ARG.
 * d_in / d_out are caller-owned device buffers [N][L]; the work is queued on
 * the lattice's stream, with the lattice's device current.  The first call on
 * a device looks up the array's device address (cudaGetSymbolAddress); make
 * that first call before any stream capture.  All calls share the one array
 * and it keeps the last call's contents: calls that overlap on the GPU (other
 * lattices or streams) race and must be serialised by the caller. */
dcrf_status dcrf_lattice_compute_noalloc(dcrf_lattice lat, float* d_out, const float* d_in, int L,
                                         int reverse);
/* Permutohedral::compute_upper_minus_lower_ord(MatrixXf& out, const MatrixXf& Q)
 * (src/permutohedral.cpp:1071-1073, 590-701): the 10-bin ordered filter. */
dcrf_status dcrf_lattice_compute_ord(dcrf_lattice lat, float* out, const float* Q, int L);
/* Permutohedral::compute_upper_minus_lower_ord_restricted(rout, rQ, pI, Q,
 * store) (include/permutohedral.h:83-84, src/permutohedral.cpp:702-900,
 * 1074-1078): the ordered filter evaluated at the nP pixels pI (strictly
 * ascending), whose values are rQ [nP][L]; rout [nP][L].  The other pixels
 * enter the splat with their values in Q [N][L]: a call with store != 0
 * splats them and keeps that splat and the set of vertices the pI pixels
 * reach; a call with store = 0 ignores Q and reuses both (DCRF_E_STATE
 * without an earlier store call for this L).  The blur runs over that vertex
 * set only, with the reference's alternating buffers.  rQ and, when read, Q
 * must lie in [0, 1] (DCRF_E_RANGE).  The reference reads pI[nP] past its
 * end after the last pI pixel; here the pixels after it are outside pI. */
dcrf_status dcrf_lattice_compute_ord_restricted(dcrf_lattice lat, float* rout, const float* rQ, const int32_t* pI,
                                                int nP, const float* Q, int L, int store);
dcrf_status dcrf_lattice_compute_ord_dev(dcrf_lattice lat, float* d_out, const float* d_Q, int L);
/* gradient(df, a, b, value_size) (include/permutohedral.h:86-87,
 * src/permutohedral.cpp:1095-1178): df [N][d] = d(a^T K b)/d(features) for
 * a, b [N][L], bit-identical to the reference's float evaluation. */
dcrf_status dcrf_lattice_gradient(dcrf_lattice lat, float* df, const float* a, const float* b, int L);
dcrf_status dcrf_lattice_gradient_dev(dcrf_lattice lat, float* d_df, const float* d_a, const float* d_b,
                                      int L);
/* Read back the lattice tables for parity checks (host buffers, any may be
 * NULL): offset/rank/bary [N*(d+1)] (offset_, rank_, barycentric_), keys
 * [M*d] int16 in vertex-id order, nbr [(d+1)*M*2] = blur_neighbors_ (n1, n2),
 * -1 where the neighbour is absent. */
dcrf_status dcrf_lattice_export(dcrf_lattice lat, int32_t* offset, int32_t* rank, float* bary,
                                int16_t* keys, int32_t* nbr);
/* The stream the lattice's work is queued on (a cudaStream_t). */
dcrf_status dcrf_lattice_stream(dcrf_lattice lat, void** stream);
/* Launch shapes of the 21-label plain filter (shape[4]: splat warps per
 * block in {2,4,8}, blur threads per block in {128,256,512}, slice pixels
 * per tile in {64,128,256}, splat form 0..5 as dcrf_batch_filter_shape
 * lists them).  The autotuner sets them on the first 21-label filter call of
 * a lattice of 2^18 pixels or more; set_filter_shape pins a shape instead
 * (that lattice is then never tuned).  Every shape computes bit-identical
 * values.  No counterpart in the reference. */
dcrf_status dcrf_lattice_filter_shape(dcrf_lattice lat, int* shape);
/* Number of bounded device waits that ran out on the current device since
 * the library was loaded (the bulk-copy splat waits for its copies with a
 * poll limit; a tile whose wait ran out writes NaN rows and counts here).
 * 0 in normal operation.  No counterpart in the reference. */
dcrf_status dcrf_device_wait_timeouts(unsigned long long* count);
dcrf_status dcrf_lattice_set_filter_shape(dcrf_lattice lat, const int* shape);

/* ------------------------------------------------------------------------
 * Dense CRF model -- class DenseCRF / DenseCRF2D (include/densecrf.h:73-194)
 * ---------------------------------------------------------------------- */

/* LP_inf_params (include/densecrf.h:43-69); dcrf_lp_params_default() gives
 * the reference defaults of LP_inf_params() (src/densecrf.cpp:287-302). */
typedef struct {
    float prox_reg_const;
    float dual_gap_tol;
    float prox_energy_tol;
    int prox_max_iter;
    int fw_max_iter;
    int qp_max_iter;
    float qp_tol;
    float qp_const;
    int best_int;
    int accel_prox;
    int work_set_size;
    int approx_fw_iter;
    float less_confident_percent;
    float confidence_tol;
} dcrf_lp_params;
void dcrf_lp_params_default(dcrf_lp_params* p);

typedef struct {
    /* 0: the reference stop rule, iterate while the energy decreases by more
     * than 100 (src/densecrf.cpp:390, DIFF_ENG).  n > 0: at most n
     * Frank-Wolfe steps (the loop still ends when the step numerator or
     * denominator is exactly zero, src/densecrf.cpp:419). */
    int max_iter;
} dcrf_qp_params;

typedef struct {
    int iterations;   /* QP: Frank-Wolfe steps taken; LP: proximal iterations */
    int inner_iters;  /* LP: total Frank-Wolfe (dual) iterations              */
    int gamma_iters;  /* LP: total qp-gamma iterations                        */
    double energy;    /* QP: last relaxed energy; LP: best integer energy     */
} dcrf_solve_stats;

/* DenseCRF2D(int W, int H, int M) (src/densecrf.cpp:149). */
dcrf_status dcrf_model_create(dcrf_model* out, int W, int H, int L);
/* ~DenseCRF (src/densecrf.cpp:141-148). */
dcrf_status dcrf_model_destroy(dcrf_model m);
/* setUnaryEnergy(const MatrixXf& unary) (src/densecrf.cpp:261): U [N][L]. */
dcrf_status dcrf_model_set_unary(dcrf_model m, const float* unary);
dcrf_status dcrf_model_set_unary_dev(dcrf_model m, const float* d_unary);
/* setUnaryEnergy(new LogisticUnaryEnergy(W, f)) (include/unary.h:48-57,
 * src/unary.cpp:47-70): weights W, L x F column-major; features f, F x N
 * column-major ([N][F]); the unary is W f.  parameters() is W (L F values,
 * column-major; *n = 0 for a constant unary), setParameters(v) replaces W and
 * recomputes the unary, gradient(b) = b f^T (L F values, column-major; b
 * [N][L]; *n = L F, 0 for a constant unary, whose gradient is empty; grad
 * may be NULL to query the count). */
dcrf_status dcrf_model_set_unary_logistic(dcrf_model m, const float* weights, const float* features, int F);
/* getUnaryEnergy()->get() (src/densecrf.cpp:268-270, src/unary.cpp:44-53):
 * the unary [N][L] in use (the constant one, or W f). */
dcrf_status dcrf_model_get_unary(dcrf_model m, float* unary);
dcrf_status dcrf_model_unary_parameters(dcrf_model m, float* params, int* n);
dcrf_status dcrf_model_unary_set_parameters(dcrf_model m, const float* params);
dcrf_status dcrf_model_unary_gradient(dcrf_model m, const float* b, float* grad, int* n);
/* addPairwiseGaussian(sx, sy, new PottsCompatibility(w)) (src/densecrf.cpp:170). */
dcrf_status dcrf_model_add_gaussian(dcrf_model m, float sx, float sy, float w_potts);
/* addPairwiseBilateral(sx, sy, sr, sg, sb, im, new PottsCompatibility(w))
 * (src/densecrf.cpp:179); rgb is the uint8 [H][W][3] image. */
dcrf_status dcrf_model_add_bilateral(dcrf_model m, float sx, float sy, float sr, float sg,
                                     float sb, const uint8_t* rgb, float w_potts);
/* addPairwiseEnergy(features, new PottsCompatibility(w), DIAG_KERNEL,
 * NORMALIZE_SYMMETRIC) (src/densecrf.cpp:157-169); features [N][d]. */
dcrf_status dcrf_model_add_pairwise(dcrf_model m, const float* features, int d, float w_potts);
/* The label compatibility of pairwise term k (the LabelCompatibility passed to
 * addPairwise*, include/labelcompatibility.h): kind 0 PottsCompatibility
 * (params[0] = w), 1 DiagonalCompatibility (params[0..L): w_l), 2
 * MatrixCompatibility (params: L x L column-major m, used as 0.5 (m + m^T),
 * src/labelcompatibility.cpp:79-129).  A term starts as the Potts weight it
 * was added with. */
/* The KernelType and NormalizationType of term k (addPairwiseEnergy's last
 * two arguments, include/pairwise.h:33-40, src/pairwise.cpp:32-168).  A term
 * starts as DIAG_KERNEL, NORMALIZE_SYMMETRIC (the reference's defaults).  The
 * kernel type changes only the parameters (CONST none, DIAG d feature scales
 * starting at 1, FULL a d x d column-major matrix starting at the identity);
 * the normalisation changes the filter: out = n o K(n o in) (symmetric,
 * n = 1/sqrt(K1 + 1e-20)), n o K(in) (after) or K(n o in) (before) with
 * n = 1/(K1 + 1e-20), K(in) (none). */
#define DCRF_KERNEL_CONST 0
#define DCRF_KERNEL_DIAG 1
#define DCRF_KERNEL_FULL 2
#define DCRF_NORM_NONE 0
#define DCRF_NORM_BEFORE 1
#define DCRF_NORM_AFTER 2
#define DCRF_NORM_SYMMETRIC 3
dcrf_status dcrf_model_set_kernel(dcrf_model m, int k, int ktype, int ntype);
/* pairwise_[k]->kernelParameters() / setKernelParameters(p)
 * (src/pairwise.cpp:396-401, 146-168): *n receives the count (0 for
 * CONST_KERNEL); params may be NULL to query it.  Setting them rebuilds the
 * term's lattice on diag(p) f (DIAG) or P f (FULL, the product summed in
 * order: float tolerance against Eigen's) from the features it was added
 * with; the term's unnormalised twin (assignment energies) keeps the lattice
 * of the original features, as the reference's no_norm_pairwise_ does. */
dcrf_status dcrf_model_pairwise_kernel_parameters(dcrf_model m, int k, float* params, int* n);
dcrf_status dcrf_model_pairwise_set_kernel_parameters(dcrf_model m, int k, const float* params);
#define DCRF_COMPAT_POTTS 0
#define DCRF_COMPAT_DIAGONAL 1
#define DCRF_COMPAT_MATRIX 2
dcrf_status dcrf_model_set_compat(dcrf_model m, int k, int kind, const float* params);
/* DenseCRF2D::addSuperPixel(img, spatial_radius, range_radius,
 * min_region_count, constant, normaliser) (include/densecrf.h:190,
 * src/densecrf.cpp:193-251): mean-shift segmentation of the model's W x H
 * image rgb (host, pixel-major RGB bytes) as EDISON's Segment(spatial_radius,
 * range_radius, min_region_count, NO_SPEEDUP) computes it
 * (src/mean-shift/msImageProcessor.cpp:714), then one clique per region with
 * the reference's weight constant * exp(-sd / (normaliser * count)), appended
 * after the cliques already set.  n_regions (may be NULL): the regions
 * added. */
dcrf_status dcrf_model_add_superpixel(dcrf_model m, const uint8_t* rgb, int spatial_radius, int range_radius,
                                      int min_region_count, float constant, float normaliser, int* n_regions);
/* The segmentation step alone (msImageProcessor::DefineImage(rgb, COLOR, H,
 * W); Segment(...); GetRegions, src/mean-shift/msImageProcessor.cpp:158,
 * 714, 1122): labels (host, W*H) receives every pixel's region, numbered from
 * 0 in EDISON's order; n_regions the count. */
dcrf_status dcrf_meanshift_segment(const uint8_t* rgb, int W, int H, int spatial_radius, float range_radius,
                                   int min_region_count, int32_t* labels, int* n_regions);
/* Its two halves: the mean-shift filtered L*u*v* colour of every pixel
 * (filtered, host W*H*3 floats: EDISON's msRawData after Filter, :353; the
 * mode search runs on the GPU), and the region steps on the host from such
 * a filtered image (Connect, TransitiveClosure as Segment repeats it, Prune:
 * :1166, :1600, :1985), which need no GPU. */
dcrf_status dcrf_meanshift_filter(const uint8_t* rgb, int W, int H, int spatial_radius, float range_radius,
                                  float* filtered);
dcrf_status dcrf_meanshift_regions(const float* filtered, int W, int H, float range_radius,
                                   int min_region_count, int32_t* labels, int* n_regions);
/* The clique state the model holds (the reference's super_pixel_container_,
 * exp_of_superpixels_ and constants_, include/densecrf.h:78-94): first the
 * count R and total pixel entries, then the arrays (offsets R+1, idx total,
 * exp_weight R, constants R; any may be NULL). */
dcrf_status dcrf_model_clique_info(dcrf_model m, int* R, int* total);
dcrf_status dcrf_model_get_cliques(dcrf_model m, int32_t* offsets, int32_t* idx, float* exp_weight,
                                   float* constants);
/* The clique state that addSuperPixel (src/densecrf.cpp:193-251) leaves in
 * super_pixel_container_, exp_of_superpixels_ and constants_, supplied
 * directly: R cliques, pixel ids idx[offsets[r] .. offsets[r+1]), their
 * weights exp_weight[r] and LP constants[r].  Replaces any earlier cliques. */
dcrf_status dcrf_model_set_cliques(dcrf_model m, int R, const int32_t* offsets,
                                   const int32_t* idx, const float* exp_weight,
                                   const float* constants);
/* unary_init() (src/densecrf.cpp:321-336): softmax of -U, [N][L]. */
dcrf_status dcrf_model_unary_init(dcrf_model m, float* Q);
/* pairwise_[k]->apply(out, in) (src/pairwise.cpp:203-208); nonorm selects the
 * NO_NORMALIZATION copy no_norm_pairwise_[k] (src/densecrf.cpp:161-169). */
dcrf_status dcrf_model_pairwise_apply(dcrf_model m, int k, int nonorm, float* out, const float* in);
dcrf_status dcrf_model_pairwise_apply_dev(dcrf_model m, int k, int nonorm, float* d_out,
                                          const float* d_in);
/* pairwise_[k]->apply_upper_minus_lower_ord(out, Q) (src/pairwise.cpp:214-228);
 * fails with DCRF_E_RANGE when Q leaves [0, 1]. */
dcrf_status dcrf_model_pairwise_apply_ord(dcrf_model m, int k, float* out, const float* Q);
/* PairwisePotential::apply_upper_minus_lower_ord_restricted(rout, rQ, pI, Q,
 * store) (src/pairwise.cpp:229-240, include/pairwise.h:78-79): the term's
 * restricted ordered filter (dcrf_lattice_compute_ord_restricted) followed by
 * its label compatibility; rout, rQ [nP][L], Q [N][L]. */
dcrf_status dcrf_model_pairwise_apply_ord_restricted(dcrf_model m, int k, float* rout, const float* rQ,
                                                     const int32_t* pI, int nP, const float* Q, int store);
/* The exact filters of PairwisePotential (src/pairwise.cpp:301-380,
 * include/pairwise.h:73-77) with k(c, b) = exp(-|f_c - f_b|^2) on the
 * features the term was added with, each followed by the term's label
 * compatibility (nonorm: the Potts compatibility of no_norm_pairwise_[k]).
 * O(N^2) work per label; the reference keeps them for its BRUTE_FORCE
 * energy check.  out, Q [N][L]; ind [N][L] with ind(l, c) at c L + l, the
 * pixel at sorted position c for label l (sortRows, src/eigen_utils.cpp:
 * 76-94), entries in [0, N) (DCRF_E_ARG otherwise); the sorted variants
 * write out in sorted positions.
 *   apply_bf(out, Q):                  out(l, c) = sum_b k(c, b) Q(l, b)
 *   apply_upper_minus_lower_bf(out, ind): sum_{b>c} k - sum_{b<c} k
 *   apply_upper_minus_lower_bf_ord(out, ind, Q): + k over b with
 *       Q(l, ind(l, b)) <= Q(l, ind(l, c)), - k over b with >= */
dcrf_status dcrf_model_pairwise_apply_bf(dcrf_model m, int k, int nonorm, float* out, const float* Q);
dcrf_status dcrf_model_pairwise_apply_upper_minus_lower_bf(dcrf_model m, int k, int nonorm, float* out,
                                                         const int32_t* ind);
dcrf_status dcrf_model_pairwise_apply_upper_minus_lower_bf_ord(dcrf_model m, int k, int nonorm, float* out,
                                                             const int32_t* ind, const float* Q);
/* PairwisePotential::apply_upper_minus_lower_dc(out, ind) (src/pairwise.cpp:
 * 241-300, src/permutohedral.cpp:902-997): the sorted upper-minus-lower sum
 * by recursive halving of the sorted positions, pairs within blocks of at
 * most 30 positions exactly (times 1 / 0.6), the cross terms of each
 * halving by a lattice filter on a lattice of the sorted features, over the
 * vertices of the halves only; then the compatibility.  Arguments as
 * dcrf_model_pairwise_apply_upper_minus_lower_bf. */
dcrf_status dcrf_model_pairwise_apply_upper_minus_lower_dc(dcrf_model m, int k, int nonorm, float* out,
                                                         const int32_t* ind);
/* qp_inference_super_pixels_non_convex(init) (src/densecrf.cpp:340-442);
 * runs qp or, when cliques are set, qp_sp.  params/stats may be NULL. */
dcrf_status dcrf_model_qp(dcrf_model m, const float* init, float* out,
                          const dcrf_qp_params* params, dcrf_solve_stats* stats);
dcrf_status dcrf_model_qp_dev(dcrf_model m, const float* d_init, float* d_out,
                              const dcrf_qp_params* params, dcrf_solve_stats* stats);
/* lp_inference_prox_super_pixels(init, params) (src/densecrf.cpp:526-799);
 * lp or, when cliques are set, lp_sp.  params NULL = reference defaults. */
dcrf_status dcrf_model_lp(dcrf_model m, const float* init, float* out,
                          const dcrf_lp_params* params, dcrf_solve_stats* stats);
dcrf_status dcrf_model_lp_dev(dcrf_model m, const float* d_init, float* d_out,
                              const dcrf_lp_params* params, dcrf_solve_stats* stats);
/* currentMap(Q) (src/densecrf.cpp:929-938): first arg-max per pixel. */
dcrf_status dcrf_model_current_map(dcrf_model m, const float* Q, int16_t* labels);
/* assignment_energy_true(l) (src/densecrf.cpp:873-885). */
dcrf_status dcrf_model_energy_true(dcrf_model m, const int16_t* labels, double* energy);
/* assignment_energy_higher_order(l) (src/densecrf.cpp:844-870). */
dcrf_status dcrf_model_energy_ho(dcrf_model m, const int16_t* labels, double* energy);
/* compute_energy_LP_higher_order(Q) (src/densecrf.cpp:982-1037). */
dcrf_status dcrf_model_energy_lp(dcrf_model m, const float* Q, double* energy);
/* compute_LR_QP_value(Q, 0) (src/densecrf.cpp:940-957). */
dcrf_status dcrf_model_lr_qp_value(dcrf_model m, const float* Q, double* energy);
/* compute_LR_QP_value(Q, diag_dom) (src/densecrf.cpp:940-957) with a
 * diag_dom [N][L] (NULL: 0, as dcrf_model_lr_qp_value). */
dcrf_status dcrf_model_lr_qp_value_diag(dcrf_model m, const float* Q, const float* diag_dom, double* energy);
/* compute_energy_higher_order(Q) (src/densecrf.cpp:960-980): U.Q + the
 * pairwise Q.A_k Q + the clique term with the clique variables the last QP
 * left (z_labels_, :439); DCRF_E_STATE when cliques are set and no QP has
 * run since. */
dcrf_status dcrf_model_energy_higher_order(dcrf_model m, const float* Q, double* energy);
/* The per-pixel energies of a labelling (src/densecrf.cpp:887-927):
 * unaryEnergy(l) -> out[N], and pairwise_energy_true(l, term) -> out[N]
 * (term -1: all terms summed in order). */
dcrf_status dcrf_model_unary_energy(dcrf_model m, const int16_t* labels, float* out);
dcrf_status dcrf_model_pairwise_energy(dcrf_model m, const int16_t* labels, int term, float* out);
/* max_rounding(Q) (src/densecrf.cpp:832-840): out [N][L], a one-hot row at
 * each pixel's first maximum. */
dcrf_status dcrf_model_max_rounding(dcrf_model m, const float* Q, float* out);
/* pairwise_[k]->kernelGradient(b, Q) (src/pairwise.cpp:402-407, 95-122,
 * 170-181): the gradient of the kernel's parameters for every
 * NormalizationType -- DIAG_KERNEL d floats (the feature scales; d = 2
 * Gaussian, 5 bilateral), FULL_KERNEL d x d (column-major), CONST_KERNEL
 * none; the count is returned in *d when d is not NULL, and grad = NULL only
 * queries it -- and pairwise_[k]->gradient(b, Q) (:390-395): the
 * compatibility's gradient, as many floats as its parameters.  b, Q [N][L]. */
dcrf_status dcrf_model_pairwise_kernel_gradient(dcrf_model m, int k, const float* b, const float* Q,
                                                float* grad, int* d);
dcrf_status dcrf_model_pairwise_gradient(dcrf_model m, int k, const float* b, const float* Q, float* grad);
/* pairwise_[k]->parameters() / setParameters(v) (src/pairwise.cpp:384-389,
 * src/labelcompatibility.cpp:64-71, 88-93, 109-122): Potts 1 value, Diagonal
 * L, Matrix L (L + 1) / 2 (w_(i, j), j >= i, by column i).  *n receives the
 * count when not NULL; params may be NULL to query it. */
dcrf_status dcrf_model_pairwise_parameters(dcrf_model m, int k, float* params, int* n);
dcrf_status dcrf_model_pairwise_set_parameters(dcrf_model m, int k, const float* params);
/* Number of pairwise terms, and vertex count of term k's lattice. */
dcrf_status dcrf_model_info(dcrf_model m, int* n_terms, int* N, int* L);
dcrf_status dcrf_model_lattice_size(dcrf_model m, int k, int* M);
dcrf_status dcrf_model_stream(dcrf_model m, void** stream);

/* ---- Batches: many images of different sizes in one solve ----------------
 * No counterpart in the reference, which solves one DenseCRF2D at a time
 * (src/example_inference.cpp:39-63); a batch holds n images that share the
 * label count and the pairwise parameters.  Pixel arrays are the images'
 * arrays one after another: unaries / Q [sum W_i H_i][L], rgb
 * [sum W_i H_i][3].  Each image's QP result equals the single-image
 * dcrf_model_qp of that image. */
typedef struct dcrf_batch_s* dcrf_batch;

dcrf_status dcrf_batch_create(dcrf_batch* out, int n_images, const int* widths,
                              const int* heights, int L);
dcrf_status dcrf_batch_destroy(dcrf_batch b);
/* Total pixel count and pixel offset of each image (offsets: n_images + 1
 * entries, may be NULL). */
dcrf_status dcrf_batch_info(dcrf_batch b, int64_t* n_pixels, int64_t* offsets);
/* setUnaryEnergy for every image (src/densecrf.cpp:151-156). */
dcrf_status dcrf_batch_set_unary(dcrf_batch b, const float* unary);
dcrf_status dcrf_batch_set_unary_dev(dcrf_batch b, const float* d_unary);
/* addPairwiseGaussian / addPairwiseBilateral with Potts weights for every
 * image (src/densecrf.cpp:170-190). */
dcrf_status dcrf_batch_add_gaussian(dcrf_batch b, float sx, float sy, float w_potts);
dcrf_status dcrf_batch_add_bilateral(dcrf_batch b, float sx, float sy, float sr, float sg,
                                     float sb, const uint8_t* rgb, float w_potts);
/* unary_init of every image. */
dcrf_status dcrf_batch_unary_init(dcrf_batch b, float* Q);
/* qp_inference_super_pixels_non_convex of every image (plain QP, no
 * cliques).  stats: NULL or an array of n_images. */
dcrf_status dcrf_batch_qp(dcrf_batch b, const float* init, float* out,
                          const dcrf_qp_params* params, dcrf_solve_stats* stats);
dcrf_status dcrf_batch_qp_dev(dcrf_batch b, const float* d_init, float* d_out,
                              const dcrf_qp_params* params, dcrf_solve_stats* stats);
dcrf_status dcrf_batch_stream(dcrf_batch b, void** stream);
/* PairwisePotential::apply (src/pairwise.cpp:203-208) of pairwise term k on
 * every image at once, over the term's concatenated lattice:
 * out = -w_k n o K(n o in), device arrays [sum N_i][L] on the batch's stream.
 * Each image's rows equal its single-image dcrf_model_pairwise_apply, bit for
 * bit (no splat list, blur neighbour or slice crosses an image). */
dcrf_status dcrf_batch_pairwise_apply(dcrf_batch b, int k, float* out, const float* in);
dcrf_status dcrf_batch_pairwise_apply_dev(dcrf_batch b, int k, float* d_out, const float* d_in);
/* The launch shapes the filter of term k uses, as the autotuner chose them
 * (shape[0] warp-splat vertices per block, [1] blur threads per block, [2]
 * slice pixels per block, [3] splat form: 0 staged long lists + thread-per-
 * label short lists, 1 warp splat for the long lists, 2 warp splat for
 * every list, 3 tiled splat for every list, 4 staged long lists + tiled
 * short lists, 5 bulk-copy splat for every list); the defaults until a
 * filter call of 2^18 pixels or more has
 * tuned them.  shape holds 4 ints.  No counterpart in the reference. */
dcrf_status dcrf_batch_filter_shape(dcrf_batch b, int k, int* shape);
/* Pins term k's launch shapes (as dcrf_lattice_set_filter_shape). */
dcrf_status dcrf_batch_set_filter_shape(dcrf_batch b, int k, const int* shape);
/* Vertex count of term k's concatenated lattice (the sum of the images' M). */
dcrf_status dcrf_batch_lattice_size(dcrf_batch b, int k, int64_t* M);

/* ---- Differentiation: unrolled mean-field and its adjoint ----------------
 * No counterpart in the reference, whose solvers are not differentiable
 * (the QP's conditional gradient is an arg-min).  These run Krahenbuhl's
 * mean-field iterations on every image of the batch,
 *   Q_0 = softmax(-U),  Q_{t+1} = softmax(-U + sum_k w_k K~_k Q_t),
 * K~_k = the k-th term's normalised filter n o K(n o .) (src/pairwise.cpp:
 * 54-75), and back-propagate a loss gradient through them with the adjoint
 * filter (blur axes in reverse order, src/permutohedral.cpp:1079-1093).
 * meanfield keeps Q_0 .. Q_T on the device; meanfield_backward recomputes
 * the messages K~_k Q_t from them. */
/* Q (may be NULL): the final iterate [N][L]. */
dcrf_status dcrf_batch_meanfield(dcrf_batch b, int iterations, float* Q);
dcrf_status dcrf_batch_meanfield_dev(dcrf_batch b, int iterations, float* d_Q);
/* grad_Q = dL/dQ_T [N][L] in; dL/dU [N][L] and dL/dw_k (n_terms doubles,
 * summed over all images) out. */
dcrf_status dcrf_batch_meanfield_backward(dcrf_batch b, const float* grad_Q, float* grad_U,
                                          double* grad_w);
dcrf_status dcrf_batch_meanfield_backward_dev(dcrf_batch b, const float* d_grad_Q, float* d_grad_U,
                                              double* grad_w);
/* Potts weight of pairwise term k (the PottsCompatibility parameter,
 * src/labelcompatibility.cpp:68-70), and the number of terms. */
dcrf_status dcrf_batch_set_weight(dcrf_batch b, int k, float w_potts);
/* Checkpointing of meanfield / meanfield_backward: the forward pass keeps
 * Q_t for t a multiple of checkpoint_every and Q_T (1 = every iterate, the
 * default); the backward pass recomputes the others segment by segment from
 * the checkpoint before them.  recompute_lattice != 0: the terms' lattices
 * are released at the end of each pass and rebuilt from the features by the
 * next (the backward pass rebuilds them before its first filter).  Results
 * do not depend on either setting: every recomputed value is computed by the
 * same kernels from the same inputs. */
dcrf_status dcrf_batch_set_checkpointing(dcrf_batch b, int checkpoint_every, int recompute_lattice);
/* Device bytes the checkpoints and recompute buffers take for T iterations. */
dcrf_status dcrf_batch_meanfield_state_bytes(dcrf_batch b, int T, uint64_t* bytes);
dcrf_status dcrf_batch_terms(dcrf_batch b, int* n_terms);

#ifdef __cplusplus
}
#endif
#endif /* DCRF_H */
