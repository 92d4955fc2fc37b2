/* CPU restatement of the densecrf_ho hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as
 * the checker; the product (libdcrf_cuda.so) never links or calls it.
 *
 * Parity is pinned: tests/test_oracle_pins.py checks every function below
 * against the unmodified reference compiled by oracle/Makefile
 * (oracle/_ref/libdcrf_ref.so) and against the committed golden vectors in
 * tests/golden/ that the reference produced.
 *
 * Matrices use the reference's Eigen column-major L x N storage: a flat array
 * indexed [pixel*L + label].  Lattice features are [pixel*d + dim].
 */
#ifndef DCRF_ORACLE_H
#define DCRF_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_lattice orc_lattice;
typedef struct orc_model orc_model;

typedef struct {
    float prox_reg_const, dual_gap_tol, prox_energy_tol;
    int prox_max_iter, fw_max_iter, qp_max_iter;
    float qp_tol, qp_const;
    int best_int, accel_prox, work_set_size, approx_fw_iter;
    float less_confident_percent, confidence_tol;
} orc_lp_params;

/* Permutohedral lattice (src/permutohedral.cpp). */
orc_lattice* orc_lattice_new(const float* f, int d, int N);
void orc_lattice_free(orc_lattice* l);
int orc_lattice_M(const orc_lattice* l);
void orc_lattice_export(const orc_lattice* l, int* offset, int* rank, float* bary, short* keys,
                        int* nbr);
void orc_lattice_compute(const orc_lattice* l, float* out, const float* in, int L, int reverse);
void orc_lattice_compute_f64(const orc_lattice* l, double* out, const double* in, int L,
                             int reverse);
void orc_lattice_compute_ord(const orc_lattice* l, float* out, const float* in, int L);
/* Permutohedral::gradient (src/permutohedral.cpp:1095-1178): df [N][d] =
 * d(a^T K b) / d(features), a and b [N][L]. */
void orc_lattice_gradient(const orc_lattice* l, float* df, const float* a, const float* b, int L);

/* DenseCRF2D model with Potts terms and optional cliques (src/densecrf.cpp). */
orc_model* orc_model_new(int W, int H, int L, const float* unary);
void orc_model_free(orc_model* m);
int orc_model_add_features(orc_model* m, const float* f, int d, float w);
int orc_model_add_gaussian(orc_model* m, float sx, float sy, float w);
int orc_model_add_bilateral(orc_model* m, float sx, float sy, float sr, float sg, float sb,
                            const unsigned char* rgb, float w);
void orc_model_set_cliques(orc_model* m, int R, const int* offsets, const int* idx,
                           const float* expw, const float* constants);
int orc_model_lattice_M(const orc_model* m, int k);
void orc_unary_init(const orc_model* m, float* Q);
void orc_apply(const orc_model* m, int k, int nonorm, float* out, const float* in);
int orc_apply_ord(const orc_model* m, int k, float* out, const float* in);
/* fixed_iters <= 0: the reference stop rule (energy decrease > 100).
 * Returns the number of completed Frank-Wolfe steps; energies[s] is the
 * energy after step s. */
int orc_qp(const orc_model* m, const float* init, float* out, int fixed_iters, double* energies);
int orc_lp(const orc_model* m, const float* init, float* out, const orc_lp_params* p,
           int* prox_iters_run);
void orc_current_map(const orc_model* m, const float* Q, short* labels);
double orc_energy_true(const orc_model* m, const short* labels);
double orc_energy_ho(const orc_model* m, const short* labels);
double orc_energy_lp(const orc_model* m, const float* Q);
double orc_lr_qp_value(const orc_model* m, const float* Q);
const char* orc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
