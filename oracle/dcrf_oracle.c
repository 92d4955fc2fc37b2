/* CPU restatement of the densecrf_ho hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This is the checker for the CUDA product, not part of it: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 *
 * It restates, in plain C with our own data structures, the arithmetic of the
 * reference as compiled by its own build (g++ -O2, x86-64 SSE2, no FMA):
 *   - the SSE lattice build   src/permutohedral.cpp:152-333 (incl. the zero
 *     feature inserted for the padding lanes of the last 4-pixel block);
 *   - sseCompute (L > 2)      src/permutohedral.cpp:998-1058 and
 *     seqCompute (L <= 2)     src/permutohedral.cpp:488-540;
 *   - the 10-bin ordered filter src/permutohedral.cpp:548-701;
 *   - DenseKernel / PairwisePotential / Potts  src/pairwise.cpp:40-75,203-228,
 *     src/labelcompatibility.cpp:49-52;
 *   - the QP   src/densecrf.cpp:340-442, src/qp.cpp:5-25;
 *   - the LP   src/densecrf.cpp:444-830, src/eigen_utils.cpp:96-141;
 *   - energies src/densecrf.cpp:844-957, 982-1037.
 * Eigen 3.2 reductions are restated with their SSE2 packet order
 * (Core/Redux.h LinearVectorizedTraversal, Packet4f / Packet2d) so results
 * are bit-identical to the reference, unary_init included (Eigen's packet
 * exp restated, eigen_pexp).
 *
 * Compiled with -ffp-contract=off so no multiply-add is fused.
 */
#include "dcrf_oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static char g_err[256];
const char* orc_last_error(void) { return g_err; }

/* ------------------------------------------------------------------------ */
/* Eigen 3.2 SSE2 reduction orders                                          */
/* ------------------------------------------------------------------------ */

/* Float sum of x[0..n) in the order of Eigen's LinearVectorizedTraversal with
 * Packet4f; `as` is the index of the first 16-byte aligned element (0 for a
 * plain VectorXf, (4 - (col*L) % 4) % 4 for column `col` of a MatrixXf).
 * Redux.h: two packet accumulators over aligned pairs of packets, one more
 * packet, predux = (a0+a2)+(a1+a3), then the unaligned head, then the tail. */
static float eig_sum_f(const float* x, long n, long as) {
    if (n <= 0) return 0.0f;
    if (as > n) as = n;
    long asz = ((n - as) / 4) * 4, asz2 = ((n - as) / 8) * 8;
    long end = as + asz, end2 = as + asz2;
    float r;
    if (asz) {
        float p0[4], p1[4];
        for (int l = 0; l < 4; l++) p0[l] = x[as + l];
        if (asz > 4) {
            for (int l = 0; l < 4; l++) p1[l] = x[as + 4 + l];
            for (long i = as + 8; i < end2; i += 8)
                for (int l = 0; l < 4; l++) {
                    p0[l] += x[i + l];
                    p1[l] += x[i + 4 + l];
                }
            for (int l = 0; l < 4; l++) p0[l] += p1[l];
            if (end > end2)
                for (int l = 0; l < 4; l++) p0[l] += x[end2 + l];
        }
        r = (p0[0] + p0[2]) + (p0[1] + p0[3]);
        for (long i = 0; i < as; i++) r += x[i];
        for (long i = end; i < n; i++) r += x[i];
    } else {
        r = x[0];
        for (long i = 1; i < n; i++) r += x[i];
    }
    return r;
}

/* Column `col` (length L) of a 16-byte aligned column-major MatrixXf. */
static float col_sum_f(const float* M, int L, long col) {
    long as = (4 - ((col * (long)L) & 3)) & 3;
    return eig_sum_f(M + col * (long)L, L, as);
}

/* VectorXf::dot: float products, then the aligned packet redux. */
static float dot_f(const float* a, const float* b, int n) {
    float t[64];
    float* p = n <= 64 ? t : (float*)malloc(sizeof(float) * n);
    for (int i = 0; i < n; i++) p[i] = a[i] * b[i];
    float r = eig_sum_f(p, n, 0);
    if (p != t) free(p);
    return r;
}

/* dotProduct (src/eigen_utils.cpp:68-74): exact double products summed in the
 * Packet2d order of MatrixXd::sum(). */
static double dot_d(const float* a, const float* b, long n) {
#define XD(i) ((double)a[i] * (double)b[i])
    if (n <= 0) return 0.0;
    long asz = (n / 2) * 2, asz2 = (n / 4) * 4;
    double r;
    if (asz) {
        double p0a = XD(0), p0b = XD(1);
        if (asz > 2) {
            double p1a = XD(2), p1b = XD(3);
            for (long i = 4; i < asz2; i += 4) {
                p0a += XD(i);
                p0b += XD(i + 1);
                p1a += XD(i + 2);
                p1b += XD(i + 3);
            }
            p0a += p1a;
            p0b += p1b;
            if (asz > asz2) {
                p0a += XD(asz2);
                p0b += XD(asz2 + 1);
            }
        }
        r = p0a + p0b;
        for (long i = asz; i < n; i++) r += XD(i);
    } else {
        r = XD(0);
    }
    return r;
#undef XD
}

/* ------------------------------------------------------------------------ */
/* Permutohedral lattice                                                    */
/* ------------------------------------------------------------------------ */

struct orc_lattice {
    int N, d, M;
    int* offset; /* (d+1)*N vertex ids */
    int* rank;   /* (d+1)*N */
    float* bary; /* (d+1)*N */
    short* keys; /* M*d */
    int* nbr;    /* (d+1)*M*2 : n1, n2 ids, -1 = absent, axis-major */
};

typedef struct {
    int d, cap, n, keycap;
    int* table;
    short* keys;
} khash;

static uint64_t key_hash(const short* k, int d) {
    uint64_t h = 1469598103934665603ull;
    for (int i = 0; i < d; i++) h = (h ^ (uint16_t)k[i]) * 1099511628211ull;
    return h;
}

static int kh_find(khash* h, const short* k, int create) {
    uint64_t s = key_hash(k, h->d) & (uint64_t)(h->cap - 1);
    for (;;) {
        int e = h->table[s];
        if (e < 0) {
            if (!create) return -1;
            if (h->n == h->keycap) {
                h->keycap *= 2;
                h->keys = (short*)realloc(h->keys, sizeof(short) * (size_t)h->keycap * h->d);
            }
            memcpy(h->keys + (size_t)h->n * h->d, k, sizeof(short) * h->d);
            h->table[s] = h->n;
            return h->n++;
        }
        if (memcmp(h->keys + (size_t)e * h->d, k, sizeof(short) * h->d) == 0) return e;
        s = (s + 1) & (uint64_t)(h->cap - 1);
    }
}

/* _mm_cvtps_epi32 under round-to-nearest-even, then back to float. */
static float cvt_rne(float v) {
    if (!(fabsf(v) < 2147483648.0f)) return -2147483648.0f;
    return nearbyintf(v);
}

orc_lattice* orc_lattice_new(const float* f, int d, int N) {
    orc_lattice* l = (orc_lattice*)calloc(1, sizeof(orc_lattice));
    l->N = N;
    l->d = d;
    int d1 = d + 1;
    int Np = (N + 3) & ~3; /* 4-pixel SSE blocks; padded lanes see a zero feature */
    l->offset = (int*)malloc(sizeof(int) * (size_t)d1 * N);
    l->rank = (int*)malloc(sizeof(int) * (size_t)d1 * N);
    l->bary = (float*)malloc(sizeof(float) * (size_t)d1 * N);

    khash h;
    h.d = d > 0 ? d : 1;
    h.cap = 1;
    while (h.cap < 2 * Np * d1 + 16) h.cap <<= 1;
    h.table = (int*)malloc(sizeof(int) * h.cap);
    memset(h.table, 0xff, sizeof(int) * h.cap);
    h.n = 0;
    h.keycap = 1024;
    h.keys = (short*)malloc(sizeof(short) * (size_t)h.keycap * h.d);

    float inv_std_dev = (float)(sqrt(2.0 / 3.0) * (d + 1));
    float* scale = (float*)malloc(sizeof(float) * (d > 0 ? d : 1));
    for (int i = 0; i < d; i++) scale[i] = (float)(1.0 / sqrt((double)((i + 2) * (i + 1))) * inv_std_dev);
    const float invdp1 = 1.0f / (float)d1, dp1 = (float)d1;
    short* canonical = (short*)malloc(sizeof(short) * d1 * d1);
    for (int i = 0; i <= d; i++) {
        for (int j = 0; j <= d - i; j++) canonical[i * d1 + j] = (short)i;
        for (int j = d - i + 1; j <= d; j++) canonical[i * d1 + j] = (short)(i - d1);
    }
    float *fv = (float*)malloc(sizeof(float) * (d + 1)), *el = (float*)malloc(sizeof(float) * d1),
          *rem0 = (float*)malloc(sizeof(float) * d1), *rk = (float*)malloc(sizeof(float) * d1),
          *b = (float*)malloc(sizeof(float) * (d + 2));
    short* key = (short*)malloc(sizeof(short) * d1);

    for (int k = 0; k < Np; k++) {
        for (int j = 0; j < d; j++) fv[j] = k < N ? f[(size_t)k * d + j] : 0.0f;
        float sm = 0.0f;
        for (int j = d; j > 0; j--) {
            float cf = fv[j - 1] * scale[j - 1];
            el[j] = sm - (float)j * cf;
            sm += cf;
        }
        el[0] = sm;
        float sum = 0.0f;
        for (int i = 0; i <= d; i++) {
            float v = cvt_rne(invdp1 * el[i]);
            rem0[i] = v * dp1;
            sum += v;
        }
        for (int i = 0; i <= d; i++) rk[i] = 0.0f;
        for (int i = 0; i < d; i++) {
            float di = el[i] - rem0[i];
            for (int j = i + 1; j <= d; j++) {
                float dj = el[j] - rem0[j];
                float c = (di < dj) ? 1.0f : 0.0f;
                rk[i] += c;
                rk[j] += 1.0f - c;
            }
        }
        for (int i = 0; i <= d; i++) {
            rk[i] += sum;
            float add = rk[i] < 0.0f ? dp1 : 0.0f;
            float sub = rk[i] >= dp1 ? dp1 : 0.0f;
            rk[i] += add - sub;
            rem0[i] += add - sub;
        }
        for (int i = 0; i < d + 2; i++) b[i] = 0.0f;
        for (int i = 0; i <= d; i++) {
            float v = (el[i] - rem0[i]) * invdp1;
            int p = (int)((float)d - rk[i]);
            b[p] += v;
            b[p + 1] -= v;
        }
        b[0] += 1.0f + b[d + 1];
        for (int r = 0; r <= d; r++) {
            for (int i = 0; i < d; i++) key[i] = (short)(rem0[i] + (float)canonical[r * d1 + (int)rk[i]]);
            int id = kh_find(&h, key, 1);
            if (k < N) {
                l->offset[(size_t)k * d1 + r] = id;
                l->rank[(size_t)k * d1 + r] = (int)rk[r];
                l->bary[(size_t)k * d1 + r] = b[r];
            }
        }
    }
    l->M = h.n;
    l->keys = (short*)malloc(sizeof(short) * (size_t)(l->M > 0 ? l->M : 1) * h.d);
    memcpy(l->keys, h.keys, sizeof(short) * (size_t)l->M * h.d);
    l->nbr = (int*)malloc(sizeof(int) * 2 * (size_t)d1 * (l->M > 0 ? l->M : 1));
    short *n1 = (short*)malloc(sizeof(short) * d1), *n2 = (short*)malloc(sizeof(short) * d1);
    for (int j = 0; j <= d; j++)
        for (int i = 0; i < l->M; i++) {
            const short* kk = l->keys + (size_t)i * d;
            for (int c = 0; c < d; c++) {
                n1[c] = (short)(kk[c] - 1);
                n2[c] = (short)(kk[c] + 1);
            }
            if (j < d) {
                n1[j] = (short)(kk[j] + d);
                n2[j] = (short)(kk[j] - d);
            }
            l->nbr[2 * ((size_t)j * l->M + i)] = kh_find(&h, n1, 0);
            l->nbr[2 * ((size_t)j * l->M + i) + 1] = kh_find(&h, n2, 0);
        }
    free(n1); free(n2); free(scale); free(canonical); free(fv); free(el); free(rem0); free(rk);
    free(b); free(key); free(h.table); free(h.keys);
    return l;
}

void orc_lattice_free(orc_lattice* l) {
    if (!l) return;
    free(l->offset); free(l->rank); free(l->bary); free(l->keys); free(l->nbr); free(l);
}
int orc_lattice_M(const orc_lattice* l) { return l->M; }

void orc_lattice_export(const orc_lattice* l, int* offset, int* rank, float* bary, short* keys,
                        int* nbr) {
    size_t E = (size_t)(l->d + 1) * l->N;
    if (offset) memcpy(offset, l->offset, E * sizeof(int));
    if (rank) memcpy(rank, l->rank, E * sizeof(int));
    if (bary) memcpy(bary, l->bary, E * sizeof(float));
    if (keys) memcpy(keys, l->keys, (size_t)l->M * l->d * sizeof(short));
    if (nbr) memcpy(nbr, l->nbr, 2 * (size_t)(l->d + 1) * l->M * sizeof(int));
}

/* Permutohedral::compute: sseCompute when L > 2, seqCompute otherwise. */
void orc_lattice_compute(const orc_lattice* l, float* out, const float* in, int L, int reverse) {
    const int N = l->N, M = l->M, d = l->d, d1 = d + 1, seq = L <= 2;
    float* v = (float*)calloc((size_t)(M + 2) * L, sizeof(float));
    float* nv = (float*)calloc((size_t)(M + 2) * L, sizeof(float));
    for (int i = 0; i < N; i++)
        for (int j = 0; j <= d; j++) {
            int o = l->offset[(size_t)i * d1 + j] + 1;
            float w = l->bary[(size_t)i * d1 + j];
            for (int k = 0; k < L; k++) v[(size_t)o * L + k] += w * in[(size_t)i * L + k];
        }
    for (int jj = 0; jj <= d; jj++) {
        int j = reverse ? d - jj : jj;
        for (int i = 0; i < M; i++) {
            int n1 = l->nbr[2 * ((size_t)j * M + i)] + 1, n2 = l->nbr[2 * ((size_t)j * M + i) + 1] + 1;
            const float *a = v + (size_t)(i + 1) * L, *p = v + (size_t)n1 * L, *q = v + (size_t)n2 * L;
            float* o = nv + (size_t)(i + 1) * L;
            for (int k = 0; k < L; k++) {
                if (seq) o[k] = (float)((double)a[k] + 0.5 * (double)(p[k] + q[k]));
                else o[k] = a[k] + 0.5f * (p[k] + q[k]);
            }
        }
        float* t = v; v = nv; nv = t;
    }
    const float alpha = 1.0f / (1.0f + powf(2.0f, (float)-d));
    for (int i = 0; i < N; i++)
        for (int k = 0; k < L; k++) {
            float acc = 0.0f;
            for (int j = 0; j <= d; j++) {
                int o = l->offset[(size_t)i * d1 + j] + 1;
                float w = l->bary[(size_t)i * d1 + j];
                if (seq) acc += w * v[(size_t)o * L + k] * alpha;
                else acc += (w * alpha) * v[(size_t)o * L + k];
            }
            out[(size_t)i * L + k] = acc;
        }
    free(v); free(nv);
}

/* The same filter carried out in double precision (the FP64 oracle). */
void orc_lattice_compute_f64(const orc_lattice* l, double* out, const double* in, int L,
                             int reverse) {
    const int N = l->N, M = l->M, d = l->d, d1 = d + 1;
    double* v = (double*)calloc((size_t)(M + 2) * L, sizeof(double));
    double* nv = (double*)calloc((size_t)(M + 2) * L, sizeof(double));
    for (int i = 0; i < N; i++)
        for (int j = 0; j <= d; j++) {
            int o = l->offset[(size_t)i * d1 + j] + 1;
            double w = l->bary[(size_t)i * d1 + j];
            for (int k = 0; k < L; k++) v[(size_t)o * L + k] += w * in[(size_t)i * L + k];
        }
    for (int jj = 0; jj <= d; jj++) {
        int j = reverse ? d - jj : jj;
        for (int i = 0; i < M; i++) {
            int n1 = l->nbr[2 * ((size_t)j * M + i)] + 1, n2 = l->nbr[2 * ((size_t)j * M + i) + 1] + 1;
            for (int k = 0; k < L; k++)
                nv[(size_t)(i + 1) * L + k] = v[(size_t)(i + 1) * L + k] +
                                              0.5 * (v[(size_t)n1 * L + k] + v[(size_t)n2 * L + k]);
        }
        double* t = v; v = nv; nv = t;
    }
    const double alpha = 1.0 / (1.0 + pow(2.0, -d));
    for (int i = 0; i < N; i++)
        for (int k = 0; k < L; k++) {
            double acc = 0.0;
            for (int j = 0; j <= d; j++)
                acc += (double)l->bary[(size_t)i * d1 + j] * alpha *
                       v[(size_t)(l->offset[(size_t)i * d1 + j] + 1) * L + k];
            out[(size_t)i * L + k] = acc;
        }
    free(v); free(nv);
}

#define RES 10
/* addSplitArray / sliceSplitArray bin indices (src/permutohedral.cpp:548-589):
 * the lower pass rounds q*10 in float, the upper pass (q - 1e-9)*10 in double. */
static int bin_lower(float q) {
    int c = (int)floorf(q * (float)RES);
    return c < RES - 1 ? c : RES - 1;
}
static int bin_upper(float q) {
    int c = (int)floor(((double)q - 1e-9) * RES);
    return c > 0 ? c : 0;
}

/* seqCompute_upper_minus_lower_ord (src/permutohedral.cpp:590-701). */
/* Permutohedral::gradient (src/permutohedral.cpp:1095-1178).  For each of
 * the two sides (dir 0: splat a, blur axes 0..d, contract with b; dir 1:
 * splat b, blur axes d..0, contract with a) the side is splatted, blurred
 * with the double-evaluated 1/2 weights (:1134), and per pixel the
 * differences r_j of the values at the simplex corners of ranks d - rank_j
 * and the next one (scaled by alpha / (d+1)) are elevated: sm starts at r_0,
 * then for j = 1..d the gradient of feature j-1 gathers
 * other(k) * s_{j-1} (sm(k) - j r_j(k)) over k and sm += r_j -- all in float
 * in the reference's order. */
void orc_lattice_gradient(const orc_lattice* l, float* df, const float* a, const float* b, int L) {
    const int N = l->N, M = l->M, d = l->d, d1 = d + 1;
    const size_t vn = (size_t)(M + 2) * L;
    float* v = (float*)malloc(vn * sizeof(float));
    float* nv = (float*)malloc(vn * sizeof(float));
    float* sf = (float*)malloc((size_t)d * sizeof(float));
    float* ra = (float*)malloc((size_t)d1 * L * sizeof(float));
    float* sm = (float*)malloc((size_t)L * sizeof(float));
    memset(df, 0, (size_t)N * d * sizeof(float));
    const float inv_std_dev = (float)(sqrt(2.0 / 3.0) * (d + 1));
    for (int i = 0; i < d; i++) sf[i] = (float)(1.0 / sqrt((double)((i + 2) * (i + 1))) * (double)inv_std_dev);
    const float alpha = 1.0f / (1.0f + powf(2.0f, (float)-d)) / (float)(d + 1);
    for (int dir = 0; dir < 2; dir++) {
        const float* in = dir ? b : a;
        const float* other = dir ? a : b;
        for (size_t t = 0; t < vn; t++) v[t] = nv[t] = 0.0f;
        for (int i = 0; i < N; i++)
            for (int j = 0; j <= d; j++) {
                const int o = l->offset[(size_t)i * d1 + j] + 1;
                const float w = l->bary[(size_t)i * d1 + j];
                for (int k = 0; k < L; k++) v[(size_t)o * L + k] += w * in[(size_t)i * L + k];
            }
        for (int jj = 0; jj <= d; jj++) {
            const int j = dir ? d - jj : jj;
            for (int i = 0; i < M; i++) {
                const int n1 = l->nbr[2 * ((size_t)j * M + i)] + 1, n2 = l->nbr[2 * ((size_t)j * M + i) + 1] + 1;
                const float *o = v + (size_t)(i + 1) * L, *p = v + (size_t)n1 * L, *q = v + (size_t)n2 * L;
                float* nw = nv + (size_t)(i + 1) * L;
                for (int k = 0; k < L; k++) nw[k] = (float)((double)o[k] + 0.5 * (double)(p[k] + q[k]));
            }
            float* t = v; v = nv; nv = t;
        }
        for (int i = 0; i < N; i++) {
            for (size_t t = 0; t < (size_t)d1 * L; t++) ra[t] = 0.0f;
            for (int j = 0; j <= d; j++) {
                const int r0 = d - l->rank[(size_t)i * d1 + j];
                const int r1 = r0 + 1 > d ? 0 : r0 + 1;
                const int o0 = l->offset[(size_t)i * d1 + r0] + 1, o1 = l->offset[(size_t)i * d1 + r1] + 1;
                for (int k = 0; k < L; k++) {
                    ra[(size_t)j * L + k] += alpha * v[(size_t)o0 * L + k];
                    ra[(size_t)j * L + k] -= alpha * v[(size_t)o1 * L + k];
                }
            }
            for (int k = 0; k < L; k++) sm[k] = ra[k];
            for (int j = 1; j <= d; j++) {
                float grad = 0.0f;
                for (int k = 0; k < L; k++) {
                    const float e = sf[j - 1] * (sm[k] - (float)j * ra[(size_t)j * L + k]);
                    grad += other[(size_t)i * L + k] * e;
                    sm[k] += ra[(size_t)j * L + k];
                }
                df[(size_t)i * d + j - 1] += grad;
            }
        }
    }
    free(v); free(nv); free(sf); free(ra); free(sm);
}

void orc_lattice_compute_ord(const orc_lattice* l, float* out, const float* in, int L) {
    const int N = l->N, M = l->M, d = l->d, d1 = d + 1;
    const size_t rows = (size_t)(M + 2) * L;
    float* v = (float*)malloc(rows * RES * sizeof(float));
    float* nv = (float*)malloc(rows * RES * sizeof(float));
    const float alpha = 1.0f / (1.0f + powf(2.0f, (float)-d));
    for (int pass = 0; pass < 2; pass++) { /* 0: lower, 1: upper */
        memset(v, 0, rows * RES * sizeof(float));
        memset(nv, 0, rows * RES * sizeof(float));
        for (int i = 0; i < N; i++)
            for (int j = 0; j <= d; j++) {
                int o = l->offset[(size_t)i * d1 + j] + 1;
                float w = l->bary[(size_t)i * d1 + j];
                for (int k = 0; k < L; k++) {
                    float q = in[(size_t)i * L + k];
                    float* bins = v + ((size_t)o * L + k) * RES;
                    if (pass == 0) {
                        int c = bin_lower(q);
                        for (int b = 0; b <= c; b++) bins[b] += w;
                    } else {
                        int c = bin_upper(q);
                        for (int b = c; b < RES; b++) bins[b] += w;
                    }
                }
            }
        for (int j = 0; j <= d; j++) {
            for (int i = 0; i < M; i++) {
                int n1 = l->nbr[2 * ((size_t)j * M + i)] + 1, n2 = l->nbr[2 * ((size_t)j * M + i) + 1] + 1;
                for (int k = 0; k < L; k++) {
                    const float* a = v + ((size_t)(i + 1) * L + k) * RES;
                    const float* p = v + ((size_t)n1 * L + k) * RES;
                    const float* q = v + ((size_t)n2 * L + k) * RES;
                    float* o = nv + ((size_t)(i + 1) * L + k) * RES;
                    for (int b = 0; b < RES; b++) o[b] = a[b] + 0.5f * (p[b] + q[b]);
                }
            }
            float* t = v; v = nv; nv = t;
        }
        for (int i = 0; i < N; i++) {
            if (pass == 0)
                for (int k = 0; k < L; k++) out[(size_t)i * L + k] = 0.0f;
            for (int j = 0; j <= d; j++) {
                int o = l->offset[(size_t)i * d1 + j] + 1;
                float w = l->bary[(size_t)i * d1 + j];
                float a = pass == 0 ? (-w) * alpha : w * alpha;
                for (int k = 0; k < L; k++) {
                    float q = in[(size_t)i * L + k];
                    int c = pass == 0 ? bin_lower(q) : bin_upper(q);
                    out[(size_t)i * L + k] += v[((size_t)o * L + k) * RES + c] * a;
                }
            }
        }
    }
    free(v); free(nv);
}

/* ------------------------------------------------------------------------ */
/* Model                                                                    */
/* ------------------------------------------------------------------------ */

#define MAXTERMS 16
typedef struct {
    orc_lattice* lat;
    float* norm; /* 1/sqrt(K 1 + 1e-20) */
    float w;
} orc_term;

struct orc_model {
    int W, H, N, L, nterms, R;
    float* unary;
    orc_term terms[MAXTERMS];
    int* cl_off;
    int* cl_idx;
    float* cl_exp;
    float* cl_const;
};

orc_model* orc_model_new(int W, int H, int L, const float* unary) {
    orc_model* m = (orc_model*)calloc(1, sizeof(orc_model));
    m->W = W; m->H = H; m->N = W * H; m->L = L;
    m->unary = (float*)malloc(sizeof(float) * (size_t)m->N * L);
    memcpy(m->unary, unary, sizeof(float) * (size_t)m->N * L);
    return m;
}

void orc_model_free(orc_model* m) {
    if (!m) return;
    for (int t = 0; t < m->nterms; t++) {
        orc_lattice_free(m->terms[t].lat);
        free(m->terms[t].norm);
    }
    free(m->unary); free(m->cl_off); free(m->cl_idx); free(m->cl_exp); free(m->cl_const); free(m);
}

int orc_model_add_features(orc_model* m, const float* f, int d, float w) {
    if (m->nterms >= MAXTERMS) return -1;
    orc_term* t = &m->terms[m->nterms++];
    t->lat = orc_lattice_new(f, d, m->N);
    t->w = w;
    t->norm = (float*)malloc(sizeof(float) * m->N);
    float* ones = (float*)malloc(sizeof(float) * m->N);
    for (int i = 0; i < m->N; i++) ones[i] = 1.0f;
    orc_lattice_compute(t->lat, t->norm, ones, 1, 0);
    for (int i = 0; i < m->N; i++) t->norm[i] = (float)(1.0 / sqrt((double)t->norm[i] + 1e-20));
    free(ones);
    return m->nterms - 1;
}

int orc_model_add_gaussian(orc_model* m, float sx, float sy, float w) {
    float* f = (float*)malloc(sizeof(float) * 2 * m->N);
    for (int j = 0; j < m->H; j++)
        for (int i = 0; i < m->W; i++) {
            f[2 * (j * m->W + i)] = (float)i / sx;
            f[2 * (j * m->W + i) + 1] = (float)j / sy;
        }
    int r = orc_model_add_features(m, f, 2, w);
    free(f);
    return r;
}

int orc_model_add_bilateral(orc_model* m, float sx, float sy, float sr, float sg, float sb,
                            const unsigned char* im, float w) {
    float* f = (float*)malloc(sizeof(float) * 5 * m->N);
    for (int j = 0; j < m->H; j++)
        for (int i = 0; i < m->W; i++) {
            size_t p = (size_t)(j * m->W + i);
            f[5 * p] = (float)i / sx;
            f[5 * p + 1] = (float)j / sy;
            f[5 * p + 2] = (float)im[p * 3 + 0] / sr;
            f[5 * p + 3] = (float)im[p * 3 + 1] / sg;
            f[5 * p + 4] = (float)im[p * 3 + 2] / sb;
        }
    int r = orc_model_add_features(m, f, 5, w);
    free(f);
    return r;
}

void orc_model_set_cliques(orc_model* m, int R, const int* offsets, const int* idx,
                           const float* expw, const float* constants) {
    free(m->cl_off); free(m->cl_idx); free(m->cl_exp); free(m->cl_const);
    m->R = R;
    m->cl_off = (int*)malloc(sizeof(int) * (R + 1));
    memcpy(m->cl_off, offsets, sizeof(int) * (R + 1));
    int T = offsets[R];
    m->cl_idx = (int*)malloc(sizeof(int) * (T > 0 ? T : 1));
    memcpy(m->cl_idx, idx, sizeof(int) * T);
    m->cl_exp = (float*)malloc(sizeof(float) * (R > 0 ? R : 1));
    m->cl_const = (float*)malloc(sizeof(float) * (R > 0 ? R : 1));
    memcpy(m->cl_exp, expw, sizeof(float) * R);
    memcpy(m->cl_const, constants, sizeof(float) * R);
}

int orc_model_lattice_M(const orc_model* m, int k) { return m->terms[k].lat->M; }

/* Eigen 3.2's pexp<Packet4f> (include/Eigen/src/Core/arch/SSE/MathFunctions.h:
 * 107-170) as the reference's x86-64 SSE2 build evaluates it, one lane: the
 * Cephes single-precision exp -- clamp to +-88.376, n = floor(x log2(e) +
 * 1/2) by truncation and correction, x - n C1 - n C2, the degree-5
 * polynomial by Horner steps, times 2^n assembled in the exponent bits, and
 * the max with the input.  pmadd is a separate multiply and add on SSE2, so
 * every product and sum rounds on its own (this file is compiled without
 * contraction); _mm_min_ps / _mm_max_ps return their second operand when the
 * comparison fails. */
static float eigen_pexp(float x0) {
    float x = x0 < 88.3762626647950f ? x0 : 88.3762626647950f;
    x = x > -88.3762626647949f ? x : -88.3762626647949f;
    float fx = x * 1.44269504088896341f;
    fx = fx + 0.5f;
    float t = (float)(int)fx;
    if (t > fx) t = t - 1.0f;
    fx = t;
    const float a = fx * 0.693359375f, c = fx * -2.12194440e-4f;
    x = x - a;
    x = x - c;
    const float z = x * x;
    float y = 1.9875691500E-4f;
    y = y * x + 1.3981999507E-3f;
    y = y * x + 8.3334519073E-3f;
    y = y * x + 4.1665795894E-2f;
    y = y * x + 1.6666665459E-1f;
    y = y * x + 5.0000001201E-1f;
    y = y * z + x;
    y = y + 1.0f;
    const int bits = ((int)fx + 0x7f) << 23;
    float p2;
    memcpy(&p2, &bits, sizeof p2);
    const float r = y * p2;
    return r > x0 ? r : x0;
}

/* expAndNormalize(-U) (src/densecrf.cpp:321-336).  b.array().exp() on a
 * VectorXf runs Eigen's packet exp over the aligned packets of four and
 * std::exp (libm expf) over the remaining tail; the sum is Eigen's packet
 * redux. */
void orc_unary_init(const orc_model* m, float* Q) {
    const int L = m->L, L4 = L & ~3;
    float* b = (float*)malloc(sizeof(float) * L);
    for (int i = 0; i < m->N; i++) {
        float mx = -FLT_MAX;
        for (int k = 0; k < L; k++) {
            b[k] = -m->unary[(size_t)i * L + k];
            if (k == 0 || b[k] > mx) mx = b[k];
        }
        for (int k = 0; k < L; k++) b[k] = k < L4 ? eigen_pexp(b[k] - mx) : expf(b[k] - mx);
        float s = eig_sum_f(b, L, 0);
        for (int k = 0; k < L; k++) Q[(size_t)i * L + k] = b[k] / s;
    }
    free(b);
}

/* PairwisePotential::apply with DenseKernel NORMALIZE_SYMMETRIC (or the
 * NO_NORMALIZATION copy) and Potts: out = -w * n.K(n.in). */
void orc_apply(const orc_model* m, int k, int nonorm, float* out, const float* in) {
    const orc_term* t = &m->terms[k];
    const size_t NL = (size_t)m->N * m->L;
    float* tmp = (float*)malloc(sizeof(float) * NL);
    for (size_t e = 0; e < NL; e++) tmp[e] = nonorm ? in[e] : in[e] * t->norm[e / m->L];
    orc_lattice_compute(t->lat, out, tmp, m->L, 0);
    for (size_t e = 0; e < NL; e++) {
        float x = nonorm ? out[e] : out[e] * t->norm[e / m->L];
        out[e] = (-t->w) * x;
    }
    free(tmp);
}

/* PairwisePotential::apply_upper_minus_lower_ord (src/pairwise.cpp:214-228). */
int orc_apply_ord(const orc_model* m, int k, float* out, const float* in) {
    const size_t NL = (size_t)m->N * m->L;
    float mx = in[0], mn = in[0];
    for (size_t e = 1; e < NL; e++) {
        if (in[e] > mx) mx = in[e];
        if (in[e] < mn) mn = in[e];
    }
    if (mx > 1 || mn < 0) {
        snprintf(g_err, sizeof(g_err), "Value out of bounds");
        return -1;
    }
    orc_lattice_compute_ord(m->terms[k].lat, out, in, m->L);
    for (size_t e = 0; e < NL; e++) out[e] = (-m->terms[k].w) * out[e];
    return 0;
}

void orc_current_map(const orc_model* m, const float* Q, short* lab) {
    for (int i = 0; i < m->N; i++) {
        const float* q = Q + (size_t)i * m->L;
        int best = 0;
        for (int k = 1; k < m->L; k++)
            if (q[k] > q[best]) best = k;
        lab[i] = (short)best;
    }
}

/* Per-pixel float energy vector unary(l) + pairwise_energy_true(l)
 * (src/densecrf.cpp:887-927). */
static void energy_vector(const orc_model* m, const short* l, float* tot) {
    const int N = m->N, L = m->L;
    const size_t NL = (size_t)N * L;
    float* Q = (float*)malloc(sizeof(float) * NL);
    float* o = (float*)malloc(sizeof(float) * NL);
    float* pw = (float*)calloc(N, sizeof(float));
    for (int t = 0; t < m->nterms; t++) {
        for (int i = 0; i < N; i++)
            for (int j = 0; j < L; j++) Q[(size_t)i * L + j] = (l[i] == j) ? 0.0f : 1.0f;
        orc_apply(m, t, 1, o, Q);
        for (int i = 0; i < N; i++) {
            float r = (0 <= l[i] && l[i] < L) ? -o[(size_t)i * L + l[i]] : 0.0f;
            pw[i] = pw[i] + r;
        }
    }
    for (int i = 0; i < N; i++) {
        float u = (0 <= l[i] && l[i] < L) ? m->unary[(size_t)i * L + l[i]] : 0.0f;
        tot[i] = u + pw[i];
    }
    free(Q); free(o); free(pw);
}

double orc_energy_true(const orc_model* m, const short* l) {
    float* tot = (float*)malloc(sizeof(float) * m->N);
    energy_vector(m, l, tot);
    double e = 0;
    for (int i = 0; i < m->N; i++) e += tot[i];
    free(tot);
    return e;
}

/* assignment_energy_higher_order (src/densecrf.cpp:844-870), including its
 * comparison of l[pix] at the clique-local index. */
double orc_energy_ho(const orc_model* m, const short* l) {
    double e = orc_energy_true(m, l), ho = 0.0;
    for (int r = 0; r < m->R; r++) {
        int sz = m->cl_off[r + 1] - m->cl_off[r];
        short prev = l[m->cl_idx[m->cl_off[r]]];
        for (int p = 0; p < sz; p++)
            if (prev != l[p]) {
                e += m->cl_exp[r];
                break;
            }
        ho += (float)(m->R - 1) * m->cl_exp[r];
    }
    return e + ho;
}

double orc_lr_qp_value(const orc_model* m, const float* Q) {
    const size_t NL = (size_t)m->N * m->L;
    float* tmp = (float*)malloc(sizeof(float) * NL);
    float* zero = (float*)calloc(NL, sizeof(float));
    double e = 0;
    e += dot_d(m->unary, Q, NL);
    e -= dot_d(zero, Q, NL);
    for (int k = 0; k < m->nterms; k++) {
        orc_apply(m, k, 0, tmp, Q);
        e += dot_d(Q, tmp, NL);
    }
    for (size_t i = 0; i < NL; i++) tmp[i] = zero[i] * Q[i];
    e += dot_d(Q, tmp, NL);
    free(tmp); free(zero);
    return e;
}

/* rescale (src/eigen_utils.cpp:120-141). */
static int rescale(float* out, const float* Q, size_t n) {
    float mn = Q[0];
    for (size_t i = 1; i < n; i++)
        if (Q[i] < mn) mn = Q[i];
    for (size_t i = 0; i < n; i++) out[i] = Q[i] - mn;
    float mx = out[0];
    for (size_t i = 1; i < n; i++)
        if (out[i] > mx) mx = out[i];
    if (mx < 0) {
        snprintf(g_err, sizeof(g_err), "Maxval < 0, skipping");
        return -1;
    }
    if (mx > 0)
        for (size_t i = 0; i < n; i++) out[i] /= mx;
    return 0;
}

double orc_energy_lp(const orc_model* m, const float* Q) {
    const int N = m->N, L = m->L;
    const size_t NL = (size_t)N * L;
    double e = dot_d(m->unary, Q, NL);
    float* rq = (float*)malloc(sizeof(float) * NL);
    float* tmp = (float*)malloc(sizeof(float) * NL);
    rescale(rq, Q, NL);
    for (int k = 0; k < m->nterms; k++) {
        orc_apply_ord(m, k, tmp, rq);
        e -= dot_d(Q, tmp, NL);
    }
    for (int r = 0; r < m->R; r++) {
        float best = 0.0f;
        for (int lab = 0; lab < L; lab++) {
            float mx = 0, mn = 0;
            for (int p = m->cl_off[r]; p < m->cl_off[r + 1]; p++) {
                float q = Q[(size_t)m->cl_idx[p] * L + lab];
                if (p == m->cl_off[r] || q > mx) mx = q;
                if (p == m->cl_off[r] || q < mn) mn = q;
            }
            float diff = mx - mn;
            if (lab == 0 || diff > best) best = diff;
        }
        e += m->cl_exp[r] * best;
    }
    free(rq); free(tmp);
    return e;
}

/* ------------------------------------------------------------------------ */
/* Clique algebra of the QP (src/densecrf.cpp:58-102), restated with the    */
/* reference's use of the clique-local index as the pixel index.            */
/* ------------------------------------------------------------------------ */

/* float multiplySuperPixels(p1 [L x R], p2 [L x N]) */
static float ms_scalar(const orc_model* m, const float* p1, const float* p2) {
    float res = 0.0f;
    for (int r = 0; r < m->R; r++) {
        int sz = m->cl_off[r + 1] - m->cl_off[r];
        for (int p = 0; p < sz; p++)
            for (int lab = 0; lab < m->L; lab++)
                res += p1[(size_t)r * m->L + lab] * p2[(size_t)p * m->L + lab];
    }
    return res;
}

/* multiplySuperPixels(p [L x N]) -> [L x R] */
static void ms_to_regions(const orc_model* m, const float* p, float* res) {
    for (int r = 0; r < m->R; r++) {
        int sz = m->cl_off[r + 1] - m->cl_off[r];
        for (int lab = 0; lab < m->L; lab++) {
            float s = 0.0f;
            for (int q = 0; q < sz; q++) s += p[(size_t)q * m->L + lab];
            res[(size_t)r * m->L + lab] = s;
        }
    }
}

/* multiplySuperPixels(p [L x R]) -> [L x N] */
static void ms_to_pixels(const orc_model* m, const float* p, float* res) {
    memset(res, 0, sizeof(float) * (size_t)m->N * m->L);
    for (int r = 0; r < m->R; r++) {
        int sz = m->cl_off[r + 1] - m->cl_off[r];
        for (int lab = 0; lab < m->L; lab++)
            for (int q = 0; q < sz; q++) res[(size_t)q * m->L + lab] += p[(size_t)r * m->L + lab];
    }
}

/* ------------------------------------------------------------------------ */
/* QP: qp_inference_super_pixels_non_convex                                 */
/* ------------------------------------------------------------------------ */
int orc_qp(const orc_model* m, const float* init, float* out, int fixed_iters, double* energies) {
    const int N = m->N, L = m->L, R = m->R;
    const size_t NL = (size_t)N * L, LR = (size_t)L * R;
    float* Q = (float*)malloc(sizeof(float) * NL);
    float* tmp = (float*)malloc(sizeof(float) * NL);
    float* gy = (float*)malloc(sizeof(float) * NL);
    float* sxy = (float*)malloc(sizeof(float) * NL);
    float* psisx = (float*)malloc(sizeof(float) * NL);
    float* hop = (float*)malloc(sizeof(float) * NL);
    float* Qm1 = (float*)malloc(sizeof(float) * NL);
    size_t lr = LR > 0 ? LR : 1;
    float *gz = (float*)malloc(sizeof(float) * lr), *cz = (float*)malloc(sizeof(float) * lr),
          *sxz = (float*)malloc(sizeof(float) * lr), *z = (float*)malloc(sizeof(float) * lr),
          *cst = (float*)malloc(sizeof(float) * lr), *t1 = (float*)malloc(sizeof(float) * lr),
          *t2 = (float*)malloc(sizeof(float) * lr);
    for (int r = 0; r < R; r++)
        for (int lab = 0; lab < L; lab++) {
            cst[(size_t)r * L + lab] = m->cl_exp[r];
            z[(size_t)r * L + lab] = 1.0f;
        }
    memcpy(Q, init, sizeof(float) * NL);
#define ZTERM()                                                                   \
    do {                                                                          \
        for (size_t e = 0; e < NL; e++) Qm1[e] = Q[e] - 1.0f;                     \
        for (size_t e = 0; e < LR; e++) { t1[e] = z[e] * cst[e]; t2[e] = (1.0f - z[e]) * cst[e]; } \
        zt = eig_sum_f(t1, (long)LR, 0) + ms_scalar(m, t2, Qm1);                  \
    } while (0)
    float zt;
    /* grad_z, cond_grad_z */
    for (size_t e = 0; e < NL; e++) Qm1[e] = Q[e] - 1.0f;
    ms_to_regions(m, Qm1, t1);
    for (size_t e = 0; e < LR; e++) gz[e] = (1.0f + t1[e]) * cst[e];
    for (size_t e = 0; e < LR; e++) cz[e] = gz[e] >= 0 ? 0.0f : 1.0f;
    memcpy(gy, m->unary, sizeof(float) * NL);
    for (int k = 0; k < m->nterms; k++) {
        orc_apply(m, k, 0, tmp, Q);
        for (size_t e = 0; e < NL; e++) gy[e] += 2.0f * tmp[e];
    }
    for (size_t e = 0; e < LR; e++) t1[e] = (z[e] - 1.0f) * cst[e];
    ms_to_pixels(m, t1, hop);
    for (size_t e = 0; e < NL; e++) gy[e] += hop[e];
    double old_energy = DBL_MAX;
    double energy = orc_lr_qp_value(m, Q);
    ZTERM();
    energy += zt;
    int it = 0;
    for (;;) {
        if (fixed_iters > 0) {
            if (it >= fixed_iters) break;
        } else if (!((old_energy - energy) > 100)) {
            break;
        }
        old_energy = energy;
        for (int i = 0; i < N; i++) {
            const float* g = gy + (size_t)i * L;
            int best = 0;
            for (int k = 1; k < L; k++)
                if (g[k] < g[best]) best = k;
            for (int k = 0; k < L; k++)
                sxy[(size_t)i * L + k] = (k == best ? 1.0f : 0.0f) - Q[(size_t)i * L + k];
        }
        for (size_t e = 0; e < LR; e++) cz[e] = gz[e] >= 0 ? 0.0f : 1.0f;
        for (size_t e = 0; e < LR; e++) sxz[e] = cz[e] - z[e];
        memset(psisx, 0, sizeof(float) * NL);
        for (int k = 0; k < m->nterms; k++) {
            orc_apply(m, k, 0, tmp, sxy);
            for (size_t e = 0; e < NL; e++) psisx[e] += tmp[e];
        }
        for (size_t e = 0; e < NL; e++) Qm1[e] = Q[e] - 1.0f;
        for (size_t e = 0; e < LR; e++) t1[e] = sxz[e] * cst[e];
        double a = ms_scalar(m, t1, Qm1);
        for (size_t e = 0; e < LR; e++) t2[e] = (cz[e] - 1.0f) * cst[e];
        double b = ms_scalar(m, t2, sxy);
        double num = dot_d(m->unary, sxy, NL) + 2 * dot_d(Q, psisx, NL) + a + b +
                     (double)eig_sum_f(sxz, (long)LR, 0);
        double denom = dot_d(sxy, psisx, NL) + (double)ms_scalar(m, t1, sxy);
        double step = -num / (2 * denom);
        if (denom == 0 || num == 0) break;
        if (denom < 0) step = 1;
        it++; /* completed Frank-Wolfe steps */
        const float fs = (float)step, f2s = (float)(2 * step);
        for (size_t e = 0; e < NL; e++) Q[e] += fs * sxy[e];
        for (size_t e = 0; e < LR; e++) z[e] += fs * sxz[e];
        for (size_t e = 0; e < LR; e++) t1[e] = (z[e] - 1.0f) * cst[e];
        ms_to_pixels(m, t1, hop);
        for (size_t e = 0; e < NL; e++) gy[e] += f2s * psisx[e] + fs * hop[e];
        for (size_t e = 0; e < NL; e++) Qm1[e] = Q[e] - 1.0f;
        ms_to_regions(m, Qm1, t1);
        for (size_t e = 0; e < LR; e++) gz[e] = 1.0f * cst[e] + t1[e] * cst[e];
        for (size_t e = 0; e < NL; e++) tmp[e] = gy[e] + m->unary[e];
        energy = dot_d(Q, tmp, NL);
        ZTERM();
        energy += zt;
        if (energies) energies[it - 1] = energy;
    }
#undef ZTERM
    memcpy(out, Q, sizeof(float) * NL);
    free(Q); free(tmp); free(gy); free(sxy); free(psisx); free(hop); free(Qm1);
    free(gz); free(cz); free(sxz); free(z); free(cst); free(t1); free(t2);
    return it;
}

/* ------------------------------------------------------------------------ */
/* LP: lp_inference_prox_super_pixels                                       */
/* ------------------------------------------------------------------------ */

/* qp_gamma_multiplyC (src/densecrf.cpp:517-523) on one pixel. */
static void gamma_mulC(float* o, const float* in, int L, float lambda) {
    float s = eig_sum_f(in, L, 0);
    const float c = (float)(-1.0 / (float)L);
    for (int k = 0; k < L; k++) o[k] = (c * s + in[k]) * lambda;
}

/* qp_gamma_step (src/densecrf.cpp:495-514) on one pixel. */
static void gamma_step(float* g, const float* ph, const float* nh, float delta, int L, float lambda) {
    float s = eig_sum_f(g, L, 0);
    const float c0 = 2 * lambda / (float)L;
    const float c1 = (float)(1.0 / (float)L), c2 = (float)(1 - 2.0 / (float)L);
    for (int k = 0; k < L; k++) {
        float st = (s - g[k]) * c0 + ph[k];
        st = st + delta;
        float t = (c1 * s + c2 * g[k]) * lambda;
        t = t + nh[k];
        t = t + delta;
        g[k] = g[k] * (st / t);
    }
}

/* computeUCondGrad (src/densecrf.cpp:803-830): running min / max held in int. */
static void ucond_grad(const orc_model* m, float* Us, const float* Q) {
    const int L = m->L;
    memset(Us, 0, sizeof(float) * (size_t)m->N * L);
    int mn, mx, min_lab = 0, max_lab = 0, min_ind = 0, max_ind = 0;
    for (int r = 0; r < m->R; r++) {
        mn = INT_MAX;
        mx = INT_MIN;
        for (int lab = 0; lab < L; lab++)
            for (int p = m->cl_off[r]; p < m->cl_off[r + 1]; p++) {
                int it = m->cl_idx[p];
                float q = Q[(size_t)it * L + lab];
                if ((float)mn > q) { min_ind = it; min_lab = lab; mn = (int)q; }
                if ((float)mx < q) { max_ind = it; max_lab = lab; mx = (int)q; }
            }
        Us[(size_t)min_ind * L + min_lab] = m->cl_const[r] * m->cl_exp[r];
        Us[(size_t)max_ind * L + max_lab] = -m->cl_const[r] * m->cl_exp[r];
    }
}

static void renormalize(float* Q, int N, int L) {
    const double uniform = 1.0 / L;
    for (int i = 0; i < N; i++) {
        double s = col_sum_f(Q, L, i);
        if (s == 0 || s != s) {
            for (int k = 0; k < L; k++) Q[(size_t)i * L + k] = (float)uniform;
        } else {
            float fs = (float)s;
            for (int k = 0; k < L; k++) Q[(size_t)i * L + k] /= fs;
        }
    }
}

static int cmp_desc(const void* a, const void* b) {
    float x = *(const float*)a, y = *(const float*)b;
    return (x < y) - (x > y);
}

/* feasible_Q (src/densecrf.cpp:470-492). Ties in the sort order cannot change
 * the result: only the sorted values are used. */
static void feasible_Q(float* out, const float* Q, int N, int L) {
    float* s = (float*)malloc(sizeof(float) * L);
    for (int i = 0; i < N; i++) {
        const float* q = Q + (size_t)i * L;
        memcpy(s, q, sizeof(float) * L);
        qsort(s, L, sizeof(float), cmp_desc);
        double sum = (double)(col_sum_f(Q, L, i) - 1);
        int K = -1;
        for (int k = L; k > 0; --k) {
            double uk = s[k - 1];
            if (sum / k < uk) {
                K = k;
                break;
            }
            sum -= uk;
        }
        for (int k = 0; k < L; k++) {
            double v = (double)q[k] - sum / K;
            v = (v < 0.0) ? 0.0 : v;
            v = (1.0 < v) ? 1.0 : v;
            out[(size_t)i * L + k] = (float)v;
        }
    }
    free(s);
}

int orc_lp(const orc_model* m, const float* init, float* out, const orc_lp_params* p,
           int* prox_iters_run) {
    const int N = m->N, L = m->L;
    const size_t NL = (size_t)N * L;
    int rc = 0;
    float *Q = (float*)malloc(4 * NL), *bestQ = (float*)malloc(4 * NL), *tmp = (float*)malloc(4 * NL),
          *alpha = (float*)malloc(4 * NL), *u = (float*)malloc(4 * NL), *sa = (float*)malloc(4 * NL),
          *su = (float*)malloc(4 * NL), *gam = (float*)malloc(4 * NL), *curQ = (float*)malloc(4 * NL),
          *rQ = (float*)malloc(4 * NL), *Y = (float*)malloc(4 * NL), *negH = (float*)malloc(4 * NL),
          *posH = (float*)malloc(4 * NL), *bmat = (float*)malloc(4 * NL), *beta = (float*)malloc(4 * (size_t)N),
          *qpv = (float*)malloc(4 * (size_t)N), *vt = (float*)malloc(4 * (size_t)L), *vy = (float*)malloc(4 * (size_t)L);
    short* lab = (short*)malloc(sizeof(short) * N);
    memcpy(Q, init, 4 * NL);
    renormalize(Q, N, L);
    memcpy(bestQ, Q, 4 * NL);
    orc_current_map(m, Q, lab);
    double int_energy = orc_energy_ho(m, lab);
    double energy = orc_energy_lp(m, Q);
    if (energy > int_energy) {
        for (int i = 0; i < N; i++) {
            int best = 0;
            for (int k = 1; k < L; k++)
                if (Q[(size_t)i * L + k] > Q[(size_t)i * L + best]) best = k;
            for (int k = 0; k < L; k++) Q[(size_t)i * L + k] = k == best ? 1.0f : 0.0f;
        }
        energy = orc_energy_lp(m, Q);
    }
    double best_energy = energy, best_int_energy = int_energy;
    const float prox_tol = p->prox_energy_tol, lambda = p->prox_reg_const, qp_delta = p->qp_const,
                qp_tol = p->qp_tol;
    int it = 0, count = 0;
    do {
        ++it;
        memset(bmat, 0, 4 * NL);
        for (size_t e = 0; e < NL; e++) gam[e] = 1.0f;
        memcpy(curQ, Q, 4 * NL);
        memset(alpha, 0, 4 * NL);
        memset(u, 0, 4 * NL);
        int pit = 0;
        do {
            ++pit;
            for (size_t e = 0; e < NL; e++) tmp[e] = (alpha[e] + u[e]) - m->unary[e];
            for (int i = 0; i < N; i++) gamma_mulC(Y + (size_t)i * L, tmp + (size_t)i * L, L, lambda);
            for (size_t e = 0; e < NL; e++) Y[e] += curQ[e];
            for (size_t e = 0; e < NL; e++) {
                /* std::max(a, b) == (a < b) ? b : a */
                posH[e] = (-Y[e] < 0.0f) ? 0.0f : -Y[e];
                negH[e] = (Y[e] < 0.0f) ? 0.0f : Y[e];
            }
            int qpit = 0;
            float qp_value = FLT_MAX;
            do {
                for (int i = 0; i < N; i++) {
                    float* g = gam + (size_t)i * L;
                    gamma_step(g, posH + (size_t)i * L, negH + (size_t)i * L, qp_delta, L, lambda);
                    gamma_mulC(vt, g, L, lambda);
                    memcpy(vy, Y + (size_t)i * L, 4 * (size_t)L);
                    qpv[i] = (float)(0.5 * (double)dot_f(g, vt, L) + (double)dot_f(g, vy, L));
                }
                float qp_value1 = eig_sum_f(qpv, N, 0);
                ++qpit;
                if (fabsf(qp_value - qp_value1) < qp_tol) break;
                qp_value = qp_value1;
            } while (qpit < p->qp_max_iter);
            for (size_t e = 0; e < NL; e++) bmat[e] = ((alpha[e] + u[e]) + gam[e]) - m->unary[e];
            for (int i = 0; i < N; i++) beta[i] = -col_sum_f(bmat, L, i);
            for (int i = 0; i < N; i++) beta[i] /= (float)L;
            for (int i = 0; i < N; i++)
                for (int k = 0; k < L; k++) bmat[(size_t)i * L + k] = beta[i];
            for (size_t e = 0; e < NL; e++)
                Q[e] = ((((alpha[e] + bmat[e]) + u[e]) + gam[e]) - m->unary[e]) * lambda + curQ[e];
            if (rescale(rQ, Q, NL) != 0) { rc = -1; goto done; }
            memset(sa, 0, 4 * NL);
            for (int k = 0; k < m->nterms; k++) {
                if (orc_apply_ord(m, k, tmp, rQ) != 0) { rc = -1; goto done; }
                for (size_t e = 0; e < NL; e++) sa[e] += tmp[e];
            }
            ucond_grad(m, su, Q);
            for (size_t e = 0; e < NL; e++) tmp[e] = (alpha[e] + u[e]) - (sa[e] + su[e]);
            double dual_gap = dot_d(tmp, Q, NL);
            float delta = (float)(dual_gap / ((double)lambda * dot_d(tmp, tmp, NL)));
            delta = (delta < 0.0f) ? 0.0f : delta; /* std::max then std::min */
            delta = (1.0f < delta) ? 1.0f : delta;
            for (size_t e = 0; e < NL; e++) alpha[e] = alpha[e] + delta * (sa[e] - alpha[e]);
            for (size_t e = 0; e < NL; e++) u[e] = u[e] + delta * (su[e] - u[e]);
        } while (pit < p->fw_max_iter);
        feasible_Q(tmp, Q, N, L);
        memcpy(Q, tmp, 4 * NL);
        renormalize(Q, N, L);
        double prev_int_energy = int_energy;
        orc_current_map(m, Q, lab);
        int_energy = orc_energy_ho(m, lab);
        if (p->best_int) {
            if (fabs(int_energy - prev_int_energy) < prox_tol) ++count;
            else count = 0;
            if (count >= 5) break;
            if (int_energy < best_int_energy) {
                memcpy(bestQ, Q, 4 * NL);
                best_int_energy = int_energy;
            }
        } else {
            double prev_energy = energy;
            energy = orc_energy_lp(m, Q);
            if (fabs(energy - prev_energy) < prox_tol) ++count;
            else count = 0;
            if (count >= 5) break;
            if (energy < best_energy) {
                memcpy(bestQ, Q, 4 * NL);
                best_energy = energy;
            }
        }
        if (p->less_confident_percent > 0) {
            int cnt = 0;
            for (int i = 0; i < N; i++) {
                float mx = bestQ[(size_t)i * L];
                for (int k = 1; k < L; k++)
                    if (bestQ[(size_t)i * L + k] > mx) mx = bestQ[(size_t)i * L + k];
                if (mx <= p->confidence_tol) cnt++;
            }
            double percent = (double)cnt / (double)N * 100;
            if (percent > p->less_confident_percent) break;
        }
    } while (it < p->prox_max_iter);
    memcpy(out, bestQ, 4 * NL);
done:
    if (prox_iters_run) *prox_iters_run = it;
    free(Q); free(bestQ); free(tmp); free(alpha); free(u); free(sa); free(su); free(gam); free(curQ);
    free(rQ); free(Y); free(negH); free(posH); free(bmat); free(beta); free(qpv); free(vt); free(vy);
    free(lab);
    return rc;
}
