// extern "C" boundary of libdcrf_cuda.so (declared in include/dcrf.h).
// Converts exceptions to dcrf_status codes; host-pointer entry points stage
// through device buffers owned by the handle and synchronise before return.
#include <cstring>
#include <string>

#include "batch.cuh"
#include "meanshift.cuh"
#include "model.cuh"

using dcrf::DevBuf;
using dcrf::Error;

std::atomic<unsigned long long> dcrf::g_kernel_launches{0};

struct dcrf_lattice_s {
    dcrf::Lattice lat;
    cudaStream_t stream = nullptr;
    DevBuf<float> feat, in, out;
    DevBuf<int> ipi;
};

struct dcrf_batch_s {
    dcrf::Batch* b = nullptr;
    DevBuf<float> io0, io1, feat;
};

struct dcrf_model_s {
    dcrf::Model* m = nullptr;
    DevBuf<float> io0, io1, io2, feat;
    DevBuf<int> ipi;
    DevBuf<uint8_t> img;
    DevBuf<int16_t> lab;
};

namespace {

thread_local std::string g_err;

template <typename F>
dcrf_status guard(F&& f) {
    try {
        f();
        return DCRF_OK;
    } catch (const Error& e) {
        g_err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_err = "host allocation failed";
        return DCRF_E_NOMEM;
    } catch (const std::exception& e) {
        g_err = e.what();
        return DCRF_E_CUDA;
    }
}

void check_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        throw Error(DCRF_E_CUDA, std::string("no usable CUDA device: ") + cudaGetErrorString(e));
}

template <typename T>
T* upload(DevBuf<T>& b, const T* h, size_t n, cudaStream_t st) {
    T* d = b.ensure(n);
    DCRF_CUDA(cudaMemcpyAsync(d, h, sizeof(T) * n, cudaMemcpyHostToDevice, st));
    return d;
}

template <typename T>
void download(T* h, const T* d, size_t n, cudaStream_t st) {
    DCRF_CUDA(cudaMemcpyAsync(h, d, sizeof(T) * n, cudaMemcpyDeviceToHost, st));
    DCRF_CUDA(cudaStreamSynchronize(st));
}

void need(const void* p, const char* what) {
    if (!p) throw Error(DCRF_E_ARG, std::string(what) + " is NULL");
}

dcrf::Model& M(dcrf_model h) {
    if (!h || !h->m) throw Error(DCRF_E_ARG, "invalid model handle");
    return *h->m;
}

void check_term(dcrf::Model& m, int k) {
    if (k < 0 || k >= (int)m.terms.size()) throw Error(DCRF_E_ARG, "pairwise term index out of range");
}

}  // namespace

extern "C" {

const char* dcrf_last_error(void) { return g_err.c_str(); }
const char* dcrf_version(void) { return "dcrf-b200 0.1 (sm_100a)"; }
unsigned long long dcrf_kernel_launches(void) { return dcrf::g_kernel_launches.load(); }

void dcrf_lp_params_default(dcrf_lp_params* p) {
    if (!p) return;
    p->prox_reg_const = 1e-2f;
    p->dual_gap_tol = 1e3f;
    p->prox_energy_tol = 1e3f;
    p->prox_max_iter = 10;
    p->fw_max_iter = 10;
    p->qp_max_iter = 1000;
    p->qp_tol = 1e3f;
    p->qp_const = 1e-16f;
    p->best_int = 1;
    p->accel_prox = 1;
    p->work_set_size = 10;
    p->approx_fw_iter = 10;
    p->less_confident_percent = 0.0f;
    p->confidence_tol = 0.95f;
}

// ------------------------------------------------------------- lattice --
dcrf_status dcrf_lattice_create(dcrf_lattice* out) {
    return guard([&] {
        need(out, "out");
        check_device();
        auto* h = new dcrf_lattice_s();
        cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete h;
            throw Error(DCRF_E_CUDA, cudaGetErrorString(e));
        }
        h->lat.stream = h->stream;
        *out = h;
    });
}

dcrf_status dcrf_lattice_destroy(dcrf_lattice h) {
    return guard([&] {
        if (!h) return;
        cudaStreamSynchronize(h->stream);
        cudaStream_t st = h->stream;
        delete h;
        cudaStreamDestroy(st);
    });
}

dcrf_status dcrf_lattice_init_dev(dcrf_lattice h, const float* d_features, int d, int N) {
    return guard([&] {
        need(h, "lattice");
        need(d_features, "features");
        h->lat.build(d_features, d, N);
    });
}

dcrf_status dcrf_lattice_init(dcrf_lattice h, const float* features, int d, int N) {
    return guard([&] {
        need(h, "lattice");
        need(features, "features");
        if (d < 1 || N < 1) throw Error(DCRF_E_ARG, "invalid feature shape");
        const float* df = upload(h->feat, features, (size_t)d * N, h->stream);
        h->lat.build(df, d, N);
        DCRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

dcrf_status dcrf_lattice_info(dcrf_lattice h, int* M, int* N, int* d) {
    return guard([&] {
        need(h, "lattice");
        if (M) *M = h->lat.M;
        if (N) *N = h->lat.N;
        if (d) *d = h->lat.d;
    });
}

dcrf_status dcrf_lattice_compute_dev(dcrf_lattice h, float* d_out, const float* d_in, int L, int reverse) {
    return guard([&] {
        need(h, "lattice");
        need(d_out, "out");
        need(d_in, "in");
        if (h->lat.N == 0) throw Error(DCRF_E_STATE, "lattice not initialised");
        dcrf::SliceEpilogue ep;
        h->lat.compute(d_out, d_in, L, reverse != 0, ep);
    });
}

dcrf_status dcrf_lattice_compute_noalloc(dcrf_lattice h, float* d_out, const float* d_in, int L, int reverse) {
    return guard([&] {
        need(h, "lattice");
        need(d_out, "out");
        need(d_in, "in");
        if (h->lat.N == 0) throw Error(DCRF_E_STATE, "lattice not initialised");
        h->lat.compute_noalloc(d_out, d_in, L, reverse != 0);
    });
}

dcrf_status dcrf_lattice_compute(dcrf_lattice h, float* out, const float* in, int L, int reverse) {
    return guard([&] {
        need(h, "lattice");
        need(out, "out");
        need(in, "in");
        if (h->lat.N == 0) throw Error(DCRF_E_STATE, "lattice not initialised");
        if (L < 1) throw Error(DCRF_E_ARG, "L must be >= 1");
        const size_t n = (size_t)L * h->lat.N;
        float* di = upload(h->in, in, n, h->stream);
        float* dout = h->out.ensure(n);
        dcrf::SliceEpilogue ep;
        h->lat.compute(dout, di, L, reverse != 0, ep);
        download(out, dout, n, h->stream);
    });
}

dcrf_status dcrf_lattice_gradient_dev(dcrf_lattice h, float* d_df, const float* d_a, const float* d_b, int L) {
    return guard([&] {
        need(h, "lattice");
        need(d_df, "df");
        need(d_a, "a");
        need(d_b, "b");
        if (h->lat.N == 0) throw Error(DCRF_E_STATE, "lattice not initialised");
        h->lat.gradient(d_df, d_a, d_b, L);
    });
}

dcrf_status dcrf_lattice_gradient(dcrf_lattice h, float* df, const float* a, const float* b, int L) {
    return guard([&] {
        need(h, "lattice");
        need(df, "df");
        need(a, "a");
        need(b, "b");
        if (h->lat.N == 0) throw Error(DCRF_E_STATE, "lattice not initialised");
        if (L < 1) throw Error(DCRF_E_ARG, "L must be >= 1");
        const size_t n = (size_t)L * h->lat.N;
        float* da = upload(h->in, a, n, h->stream);
        float* db = upload(h->feat, b, n, h->stream);
        float* ddf = h->out.ensure((size_t)h->lat.N * h->lat.d);
        h->lat.gradient(ddf, da, db, L);
        download(df, ddf, (size_t)h->lat.N * h->lat.d, h->stream);
    });
}

dcrf_status dcrf_lattice_compute_ord_dev(dcrf_lattice h, float* d_out, const float* d_Q, int L) {
    return guard([&] {
        need(h, "lattice");
        need(d_out, "out");
        need(d_Q, "Q");
        if (h->lat.N == 0) throw Error(DCRF_E_STATE, "lattice not initialised");
        dcrf::SliceEpilogue ep;
        h->lat.compute_ord(d_out, d_Q, L, ep);
    });
}

dcrf_status dcrf_lattice_compute_ord(dcrf_lattice h, float* out, const float* Q, int L) {
    return guard([&] {
        need(h, "lattice");
        need(out, "out");
        need(Q, "Q");
        if (h->lat.N == 0) throw Error(DCRF_E_STATE, "lattice not initialised");
        if (L < 1) throw Error(DCRF_E_ARG, "L must be >= 1");
        const size_t n = (size_t)L * h->lat.N;
        for (size_t i = 0; i < n; i++)  // the reference asserts 0 <= Q <= 1 here
            if (!(Q[i] >= 0.0f && Q[i] <= 1.0f)) throw Error(DCRF_E_RANGE, "Value out of bounds");
        float* dq = upload(h->in, Q, n, h->stream);
        float* dout = h->out.ensure(n);
        dcrf::SliceEpilogue ep;
        h->lat.compute_ord(dout, dq, L, ep);
        download(out, dout, n, h->stream);
    });
}

namespace {
// pI: 0 <= pI[i] < N, strictly ascending (the reference walks it in step with
// the pixel loop); rQ (and Q for a store call) in [0, 1].
void check_restricted(int N, int L, const int32_t* pI, int nP, const float* rQ, const float* Q, int store) {
    if (nP < 0 || nP > N) throw Error(DCRF_E_ARG, "pI larger than the lattice");
    if (nP) need(pI, "pI");
    for (int i = 0; i < nP; i++)
        if (pI[i] < 0 || pI[i] >= N || (i && pI[i] <= pI[i - 1]))
            throw Error(DCRF_E_ARG, "pI must be strictly ascending pixel indices");
    if (nP) need(rQ, "rQ");
    for (size_t i = 0; i < (size_t)nP * L; i++)
        if (!(rQ[i] >= 0.0f && rQ[i] <= 1.0f)) throw Error(DCRF_E_RANGE, "Value out of bounds");
    if (store) {
        need(Q, "Q");
        for (size_t i = 0; i < (size_t)N * L; i++)
            if (!(Q[i] >= 0.0f && Q[i] <= 1.0f)) throw Error(DCRF_E_RANGE, "Value out of bounds");
    }
}
}  // namespace

dcrf_status dcrf_lattice_compute_ord_restricted(dcrf_lattice h, float* rout, const float* rQ, const int32_t* pI,
                                                int nP, const float* Q, int L, int store) {
    return guard([&] {
        need(h, "lattice");
        if (h->lat.N == 0) throw Error(DCRF_E_STATE, "lattice not initialised");
        if (L < 1) throw Error(DCRF_E_ARG, "L must be >= 1");
        check_restricted(h->lat.N, L, pI, nP, rQ, Q, store);
        if (nP) need(rout, "rout");
        const size_t n = (size_t)nP * L;
        const float* drq = n ? upload(h->in, rQ, n, h->stream) : nullptr;
        const float* dq = store ? upload(h->feat, Q, (size_t)h->lat.N * L, h->stream) : nullptr;
        const int* dpi = nP ? upload(h->ipi, pI, (size_t)nP, h->stream) : nullptr;
        float* dout = h->out.ensure(std::max<size_t>(n, 1));
        dcrf::SliceEpilogue ep;
        h->lat.compute_ord_restricted(dout, drq, dpi, nP, dq, L, store != 0, ep);
        if (n) download(rout, dout, n, h->stream);
        else DCRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

dcrf_status dcrf_lattice_export(dcrf_lattice h, int32_t* offset, int32_t* rank, float* bary, int16_t* keys,
                                int32_t* nbr) {
    return guard([&] {
        need(h, "lattice");
        dcrf::Lattice& L = h->lat;
        if (L.N == 0) throw Error(DCRF_E_STATE, "lattice not initialised");
        const size_t E = (size_t)L.N * (L.d + 1);
        cudaStream_t st = h->stream;
        if (offset) download(offset, L.offset.get(), E, st);
        if (rank) download(rank, L.rank.get(), E, st);
        if (bary) download(bary, L.bary.get(), E, st);
        if (keys && L.M) download(keys, L.vkeys.get(), (size_t)L.M * L.d, st);
        if (nbr && L.M) {
            const size_t n = (size_t)(L.d + 1) * L.M;
            download(reinterpret_cast<int2*>(nbr), L.nbr.get(), n, st);
            for (size_t i = 0; i < 2 * n; i++) nbr[i] -= 1;  // stored shifted by one
        }
    });
}

namespace {
// shape[4] = {splat warps per block, blur threads, slice pixels per tile,
// splat form} (FilterShape), validated against the tuner's candidates.
dcrf::FilterShape shape_from(const int* shape) {
    need(shape, "shape");
    const int w = shape[0], bt = shape[1], tile = shape[2], kind = shape[3];
    dcrf::require((w == 2 || w == 4 || w == 8) && (bt == 128 || bt == 256 || bt == 512) &&
                      (tile == 64 || tile == 128 || tile == 256) && kind >= 0 && kind <= 5,
                  DCRF_E_ARG, "filter shape: warps in {2,4,8}, blur threads in {128,256,512}, "
                              "slice tile in {64,128,256}, splat form in 0..5");
    dcrf::FilterShape f;
    f.splat_warps = w;
    f.blur_threads = bt;
    f.slice_tile = tile;
    f.splat_kind = kind;
    return f;
}
void shape_to(const dcrf::FilterShape& f, int* shape) {
    need(shape, "shape");
    shape[0] = f.splat_warps;
    shape[1] = f.blur_threads;
    shape[2] = f.slice_tile;
    shape[3] = f.splat_kind;
}
}  // namespace

dcrf_status dcrf_device_wait_timeouts(unsigned long long* count) {
    return guard([&] {
        need(count, "count");
        *count = dcrf::bulk_wait_timeouts();
    });
}

dcrf_status dcrf_lattice_filter_shape(dcrf_lattice h, int* shape) {
    return guard([&] {
        need(h, "lattice");
        shape_to(h->lat.shape, shape);
    });
}

dcrf_status dcrf_lattice_set_filter_shape(dcrf_lattice h, const int* shape) {
    return guard([&] {
        need(h, "lattice");
        h->lat.shape = shape_from(shape);
        h->lat.shape_L = 21;  // pinned: no tuning for this lattice
    });
}

dcrf_status dcrf_lattice_stream(dcrf_lattice h, void** stream) {
    return guard([&] {
        need(h, "lattice");
        need(stream, "stream");
        *stream = (void*)h->stream;
    });
}

// --------------------------------------------------------------- model --
dcrf_status dcrf_model_create(dcrf_model* out, int W, int H, int L) {
    return guard([&] {
        need(out, "out");
        if (W < 1 || H < 1 || L < 1 || L > 64 || (long long)W * H * L >= (1LL << 31))
            throw Error(DCRF_E_ARG, "invalid model size (W, H >= 1; 1 <= L <= 64; W*H*L < 2^31)");
        check_device();
        auto* h = new dcrf_model_s();
        try {
            h->m = new dcrf::Model(W, H, L);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

dcrf_status dcrf_release_cached_memory(void) {
    return guard([&] { dcrf::dev_trim(true); });
}

dcrf_status dcrf_set_device_memory_limit(uint64_t bytes) {
    return guard([&] { dcrf::set_device_memory_limit((size_t)bytes); });
}

dcrf_status dcrf_device_memory_stats(uint64_t* in_use, uint64_t* cached, uint64_t* mallocs) {
    return guard([&] {
        size_t l = 0, c = 0;
        unsigned long long m = 0;
        dcrf::device_memory_stats(&l, &c, &m);
        if (in_use) *in_use = l;
        if (cached) *cached = c;
        if (mallocs) *mallocs = m;
    });
}

dcrf_status dcrf_model_destroy(dcrf_model h) {
    return guard([&] {
        if (!h) return;
        delete h->m;
        delete h;
    });
}

dcrf_status dcrf_model_set_unary_dev(dcrf_model h, const float* d_unary) {
    return guard([&] {
        auto& m = M(h);
        need(d_unary, "unary");
        float* u = m.unary.ensure((size_t)m.N * m.L);
        DCRF_CUDA(cudaMemcpyAsync(u, d_unary, sizeof(float) * m.N * m.L, cudaMemcpyDeviceToDevice, m.stream));
        m.has_unary = true;
        m.logit_F = 0;  // a constant unary replaces the unary energy
        m.gen++;
    });
}

dcrf_status dcrf_model_set_unary(dcrf_model h, const float* unary) {
    return guard([&] {
        auto& m = M(h);
        need(unary, "unary");
        upload(m.unary, unary, (size_t)m.N * m.L, m.stream);
        m.has_unary = true;
        m.logit_F = 0;  // a constant unary replaces the unary energy
        m.gen++;
        m.sync();
    });
}

dcrf_status dcrf_model_get_unary(dcrf_model h, float* unary) {
    return guard([&] {
        auto& m = M(h);
        need(unary, "unary");
        if (!m.has_unary) throw Error(DCRF_E_STATE, "no unary energy set");
        download(unary, m.unary.get(), (size_t)m.N * m.L, m.stream);
    });
}

dcrf_status dcrf_model_set_unary_logistic(dcrf_model h, const float* weights, const float* features, int F) {
    return guard([&] {
        auto& m = M(h);
        need(weights, "weights");
        need(features, "features");
        m.set_unary_logistic(weights, features, F);
    });
}

dcrf_status dcrf_model_unary_parameters(dcrf_model h, float* params, int* n) {
    return guard([&] {
        auto& m = M(h);
        if (n) *n = m.logit_F > 0 ? (int)m.h_logit_w.size() : 0;
        if (params && m.logit_F > 0) std::copy(m.h_logit_w.begin(), m.h_logit_w.end(), params);
    });
}

dcrf_status dcrf_model_unary_set_parameters(dcrf_model h, const float* params) {
    return guard([&] {
        auto& m = M(h);
        if (m.logit_F == 0) return;
        need(params, "params");
        m.set_unary_parameters(params);
    });
}

dcrf_status dcrf_model_unary_gradient(dcrf_model h, const float* b, float* grad, int* n) {
    return guard([&] {
        auto& m = M(h);
        need(b, "b");
        if (n) *n = m.L * m.logit_F;
        if (m.logit_F == 0 || !grad) return;  // grad NULL: query the count
        const float* db = upload(h->io0, b, (size_t)m.N * m.L, m.stream);
        m.unary_gradient(db, grad);
    });
}

dcrf_status dcrf_model_add_pairwise(dcrf_model h, const float* features, int d, float w_potts) {
    return guard([&] {
        auto& m = M(h);
        need(features, "features");
        if (d < 1 || d > 16) throw Error(DCRF_E_ARG, "feature dimension must be in [1, 16]");
        const float* df = upload(h->feat, features, (size_t)d * m.N, m.stream);
        m.add_term(df, d, w_potts);
        m.sync();
    });
}

dcrf_status dcrf_model_add_gaussian(dcrf_model h, float sx, float sy, float w_potts) {
    return guard([&] {
        auto& m = M(h);
        std::vector<float> f((size_t)2 * m.N);
        for (int j = 0; j < m.H; j++)
            for (int i = 0; i < m.W; i++) {
                f[2 * ((size_t)j * m.W + i)] = i / sx;
                f[2 * ((size_t)j * m.W + i) + 1] = j / sy;
            }
        const float* df = upload(h->feat, f.data(), f.size(), m.stream);
        m.add_term(df, 2, w_potts);
        m.sync();
    });
}

dcrf_status dcrf_model_add_bilateral(dcrf_model h, float sx, float sy, float sr, float sg, float sb,
                                     const uint8_t* rgb, float w_potts) {
    return guard([&] {
        auto& m = M(h);
        need(rgb, "rgb");
        std::vector<float> f((size_t)5 * m.N);
        for (int j = 0; j < m.H; j++)
            for (int i = 0; i < m.W; i++) {
                const size_t p = (size_t)j * m.W + i;
                f[5 * p] = i / sx;
                f[5 * p + 1] = j / sy;
                f[5 * p + 2] = rgb[3 * p] / sr;
                f[5 * p + 3] = rgb[3 * p + 1] / sg;
                f[5 * p + 4] = rgb[3 * p + 2] / sb;
            }
        const float* df = upload(h->feat, f.data(), f.size(), m.stream);
        m.add_term(df, 5, w_potts);
        m.sync();
    });
}

dcrf_status dcrf_model_set_kernel(dcrf_model h, int k, int ktype, int ntype) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        m.set_kernel(k, ktype, ntype);
    });
}

dcrf_status dcrf_model_pairwise_kernel_parameters(dcrf_model h, int k, float* params, int* n) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        const int c = m.kernel_parameters(k, params);
        if (n) *n = c;
    });
}

dcrf_status dcrf_model_pairwise_set_kernel_parameters(dcrf_model h, int k, const float* params) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        if (m.kernel_parameters(k, nullptr) == 0) return;
        need(params, "params");
        m.set_kernel_parameters(k, params);
    });
}

dcrf_status dcrf_model_set_compat(dcrf_model h, int k, int kind, const float* params) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        need(params, "params");
        m.set_compat(k, kind, params);
    });
}

dcrf_status dcrf_model_set_cliques(dcrf_model h, int R, const int32_t* offsets, const int32_t* idx,
                                   const float* exp_weight, const float* constants) {
    return guard([&] {
        auto& m = M(h);
        if (R < 0) throw Error(DCRF_E_ARG, "R must be >= 0");
        if (R > 0) {
            need(offsets, "offsets");
            need(exp_weight, "exp_weight");
            need(constants, "constants");
            if (offsets[0] != 0) throw Error(DCRF_E_ARG, "offsets[0] must be 0");
            for (int r = 0; r < R; r++) {
                const int sz = offsets[r + 1] - offsets[r];
                if (sz < 1) throw Error(DCRF_E_ARG, "every clique needs at least one pixel");
                if (sz > m.N) throw Error(DCRF_E_ARG, "clique larger than the image");
            }
            if (offsets[R] > 0) need(idx, "idx");
            for (int p = 0; p < offsets[R]; p++)
                if (idx[p] < 0 || idx[p] >= m.N) throw Error(DCRF_E_ARG, "clique pixel index out of range");
        }
        static const int zero = 0;
        m.set_cliques(R, R > 0 ? offsets : &zero, idx, exp_weight, constants);
    });
}

dcrf_status dcrf_model_add_superpixel(dcrf_model h, const uint8_t* rgb, int spatial_radius, int range_radius,
                                      int min_region_count, float constant, float normaliser, int* n_regions) {
    return guard([&] {
        auto& m = M(h);
        need(rgb, "rgb");
        std::vector<int> labels(m.N);
        const int reg = dcrf::meanshift_segment(rgb, m.W, m.H, spatial_radius, (float)range_radius,
                                                min_region_count, labels.data(), m.stream);
        std::vector<int> off, idx;
        std::vector<float> ew, cs;
        dcrf::superpixel_cliques(rgb, labels.data(), m.N, reg, m.R, constant, normaliser, off, idx, ew, cs);
        // appended after the cliques the model holds, as the reference's R_,
        // super_pixel_container_ and weight vectors grow
        std::vector<int> all_off(m.h_cl_off.empty() ? std::vector<int>{0} : m.h_cl_off);
        std::vector<int> all_idx(m.h_cl_idx);
        std::vector<float> all_ew(m.h_cl_exp), all_cs(m.h_cl_const);
        const int base = all_off.back();
        for (int r = 0; r < reg; r++) all_off.push_back(base + off[r + 1]);
        all_idx.insert(all_idx.end(), idx.begin(), idx.end());
        all_ew.insert(all_ew.end(), ew.begin(), ew.end());
        all_cs.insert(all_cs.end(), cs.begin(), cs.end());
        m.set_cliques(m.R + reg, all_off.data(), all_idx.data(), all_ew.data(), all_cs.data());
        if (n_regions) *n_regions = reg;
    });
}

dcrf_status dcrf_model_clique_info(dcrf_model h, int* R, int* total) {
    return guard([&] {
        auto& m = M(h);
        if (R) *R = m.R;
        if (total) *total = m.R ? m.h_cl_off[m.R] : 0;
    });
}

dcrf_status dcrf_model_get_cliques(dcrf_model h, int32_t* offsets, int32_t* idx, float* exp_weight,
                                   float* constants) {
    return guard([&] {
        auto& m = M(h);
        if (offsets) {
            if (m.R) std::memcpy(offsets, m.h_cl_off.data(), sizeof(int) * (m.R + 1));
            else offsets[0] = 0;
        }
        if (m.R == 0) return;
        if (idx) std::memcpy(idx, m.h_cl_idx.data(), sizeof(int) * m.h_cl_off[m.R]);
        if (exp_weight) std::memcpy(exp_weight, m.h_cl_exp.data(), sizeof(float) * m.R);
        if (constants) std::memcpy(constants, m.h_cl_const.data(), sizeof(float) * m.R);
    });
}

namespace {
// A stream for the model-less mean-shift calls, destroyed on every path.
struct OwnStream {
    cudaStream_t s = nullptr;
    OwnStream() { DCRF_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~OwnStream() {
        if (s) cudaStreamDestroy(s);
    }
};
}  // namespace

dcrf_status dcrf_meanshift_filter(const uint8_t* rgb, int W, int H, int spatial_radius, float range_radius,
                                  float* filtered) {
    return guard([&] {
        need(rgb, "rgb");
        need(filtered, "filtered");
        check_device();
        OwnStream st;
        dcrf::meanshift_filter(rgb, W, H, spatial_radius, range_radius, filtered, st.s);
    });
}

dcrf_status dcrf_meanshift_regions(const float* filtered, int W, int H, float range_radius, int min_region_count,
                                   int32_t* labels, int* n_regions) {
    return guard([&] {
        need(filtered, "filtered");
        need(labels, "labels");
        const int reg = dcrf::meanshift_regions(filtered, W, H, range_radius, min_region_count, labels);
        if (n_regions) *n_regions = reg;
    });
}

dcrf_status dcrf_meanshift_segment(const uint8_t* rgb, int W, int H, int spatial_radius, float range_radius,
                                   int min_region_count, int32_t* labels, int* n_regions) {
    return guard([&] {
        need(rgb, "rgb");
        need(labels, "labels");
        check_device();
        OwnStream st;
        const int reg = dcrf::meanshift_segment(rgb, W, H, spatial_radius, range_radius, min_region_count, labels,
                                                st.s);
        if (n_regions) *n_regions = reg;
    });
}

dcrf_status dcrf_model_unary_init(dcrf_model h, float* Q) {
    return guard([&] {
        auto& m = M(h);
        need(Q, "Q");
        const size_t n = (size_t)m.N * m.L;
        float* d = h->io0.ensure(n);
        m.unary_init(d);
        download(Q, d, n, m.stream);
    });
}

dcrf_status dcrf_model_pairwise_apply_dev(dcrf_model h, int k, int nonorm, float* d_out, const float* d_in) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        need(d_out, "out");
        need(d_in, "in");
        m.apply(k, nonorm != 0, d_out, d_in);
    });
}

dcrf_status dcrf_model_pairwise_apply(dcrf_model h, int k, int nonorm, float* out, const float* in) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        need(out, "out");
        need(in, "in");
        const size_t n = (size_t)m.N * m.L;
        float* di = upload(h->io0, in, n, m.stream);
        float* dout = h->io1.ensure(n);
        m.apply(k, nonorm != 0, dout, di);
        download(out, dout, n, m.stream);
    });
}

dcrf_status dcrf_model_pairwise_apply_ord(dcrf_model h, int k, float* out, const float* Q) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        need(out, "out");
        need(Q, "Q");
        const size_t n = (size_t)m.N * m.L;
        float* dq = upload(h->io0, Q, n, m.stream);
        m.check_unit_range(dq);
        float* dout = h->io1.ensure(n);
        m.apply_ord(k, dout, dq);
        download(out, dout, n, m.stream);
    });
}

dcrf_status dcrf_model_pairwise_apply_ord_restricted(dcrf_model h, int k, float* rout, const float* rQ,
                                                     const int32_t* pI, int nP, const float* Q, int store) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        check_restricted(m.N, m.L, pI, nP, rQ, Q, store);
        if (nP) need(rout, "rout");
        const size_t n = (size_t)nP * m.L;
        const float* drq = n ? upload(h->io0, rQ, n, m.stream) : nullptr;
        const float* dq = store ? upload(h->io2, Q, (size_t)m.N * m.L, m.stream) : nullptr;
        const int* dpi = nP ? upload(h->ipi, pI, (size_t)nP, m.stream) : nullptr;
        float* dout = h->io1.ensure(std::max<size_t>(n, 1));
        m.apply_ord_restricted(k, dout, drq, dpi, nP, dq, store != 0);
        if (n) download(rout, dout, n, m.stream);
        else DCRF_CUDA(cudaStreamSynchronize(m.stream));
    });
}

namespace {
// ind(l, c) of apply_upper_minus_lower_{bf,bf_ord,dc}: [N][L], each in [0, N).
void check_ind(const dcrf::Model& m, const int32_t* ind) {
    need(ind, "ind");
    const size_t n = (size_t)m.N * m.L;
    for (size_t t = 0; t < n; t++)
        if (ind[t] < 0 || ind[t] >= m.N) throw Error(DCRF_E_ARG, "ind: entries must lie in [0, N)");
}
}  // namespace

dcrf_status dcrf_model_pairwise_apply_bf(dcrf_model h, int k, int nonorm, float* out, const float* Q) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        need(out, "out");
        need(Q, "Q");
        const size_t n = (size_t)m.N * m.L;
        const float* dq = upload(h->io0, Q, n, m.stream);
        float* dout = h->io1.ensure(n);
        m.apply_bf(k, nonorm != 0, dout, dq);
        download(out, dout, n, m.stream);
    });
}

dcrf_status dcrf_model_pairwise_apply_upper_minus_lower_bf(dcrf_model h, int k, int nonorm, float* out,
                                                         const int32_t* ind) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        need(out, "out");
        check_ind(m, ind);
        const size_t n = (size_t)m.N * m.L;
        const int* di = upload(h->ipi, ind, n, m.stream);
        float* dout = h->io1.ensure(n);
        m.apply_upper_minus_lower_bf(k, nonorm != 0, dout, di, nullptr);
        download(out, dout, n, m.stream);
    });
}

dcrf_status dcrf_model_pairwise_apply_upper_minus_lower_bf_ord(dcrf_model h, int k, int nonorm, float* out,
                                                             const int32_t* ind, const float* Q) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        need(out, "out");
        need(Q, "Q");
        check_ind(m, ind);
        const size_t n = (size_t)m.N * m.L;
        const int* di = upload(h->ipi, ind, n, m.stream);
        const float* dq = upload(h->io0, Q, n, m.stream);
        float* dout = h->io1.ensure(n);
        m.apply_upper_minus_lower_bf(k, nonorm != 0, dout, di, dq);
        download(out, dout, n, m.stream);
    });
}

dcrf_status dcrf_model_pairwise_apply_upper_minus_lower_dc(dcrf_model h, int k, int nonorm, float* out,
                                                         const int32_t* ind) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        need(out, "out");
        check_ind(m, ind);
        const size_t n = (size_t)m.N * m.L;
        const int* di = upload(h->ipi, ind, n, m.stream);
        float* dout = h->io1.ensure(n);
        m.apply_upper_minus_lower_dc(k, nonorm != 0, dout, di);
        download(out, dout, n, m.stream);
    });
}

dcrf_status dcrf_model_qp_dev(dcrf_model h, const float* d_init, float* d_out, const dcrf_qp_params* params,
                              dcrf_solve_stats* stats) {
    return guard([&] {
        auto& m = M(h);
        need(d_init, "init");
        need(d_out, "out");
        const int max_iter = params ? params->max_iter : 0;
        if (max_iter < 0) throw Error(DCRF_E_ARG, "max_iter must be >= 0");
        double e = 0.0;
        int it = m.qp(d_init, d_out, max_iter, &e);
        if (stats) {
            std::memset(stats, 0, sizeof(*stats));
            stats->iterations = it;
            stats->energy = e;
        }
    });
}

dcrf_status dcrf_model_qp(dcrf_model h, const float* init, float* out, const dcrf_qp_params* params,
                          dcrf_solve_stats* stats) {
    return guard([&] {
        auto& m = M(h);
        need(init, "init");
        need(out, "out");
        const size_t n = (size_t)m.N * m.L;
        float* di = upload(h->io0, init, n, m.stream);
        float* dout = h->io1.ensure(n);
        const int max_iter = params ? params->max_iter : 0;
        if (max_iter < 0) throw Error(DCRF_E_ARG, "max_iter must be >= 0");
        double e = 0.0;
        int it = m.qp(di, dout, max_iter, &e);
        download(out, dout, n, m.stream);
        if (stats) {
            std::memset(stats, 0, sizeof(*stats));
            stats->iterations = it;
            stats->energy = e;
        }
    });
}

static void check_lp_params(const dcrf_lp_params& p) {
    if (p.prox_max_iter < 1 || p.fw_max_iter < 1 || p.qp_max_iter < 1)
        throw Error(DCRF_E_ARG, "LP iteration counts must be >= 1");
}

dcrf_status dcrf_model_lp_dev(dcrf_model h, const float* d_init, float* d_out, const dcrf_lp_params* params,
                              dcrf_solve_stats* stats) {
    return guard([&] {
        auto& m = M(h);
        need(d_init, "init");
        need(d_out, "out");
        dcrf_lp_params p;
        if (params) p = *params;
        else dcrf_lp_params_default(&p);
        check_lp_params(p);
        dcrf_solve_stats s{};
        m.lp(d_init, d_out, p, &s);
        if (stats) *stats = s;
    });
}

dcrf_status dcrf_model_lp(dcrf_model h, const float* init, float* out, const dcrf_lp_params* params,
                          dcrf_solve_stats* stats) {
    return guard([&] {
        auto& m = M(h);
        need(init, "init");
        need(out, "out");
        dcrf_lp_params p;
        if (params) p = *params;
        else dcrf_lp_params_default(&p);
        check_lp_params(p);
        const size_t n = (size_t)m.N * m.L;
        float* di = upload(h->io0, init, n, m.stream);
        float* dout = h->io1.ensure(n);
        dcrf_solve_stats s{};
        m.lp(di, dout, p, &s);
        download(out, dout, n, m.stream);
        if (stats) *stats = s;
    });
}

dcrf_status dcrf_model_current_map(dcrf_model h, const float* Q, int16_t* labels) {
    return guard([&] {
        auto& m = M(h);
        need(Q, "Q");
        need(labels, "labels");
        float* dq = upload(h->io0, Q, (size_t)m.N * m.L, m.stream);
        int16_t* dl = h->lab.ensure(m.N);
        m.current_map(dq, dl);
        download(labels, dl, m.N, m.stream);
    });
}

dcrf_status dcrf_model_energy_true(dcrf_model h, const int16_t* labels, double* energy) {
    return guard([&] {
        auto& m = M(h);
        need(labels, "labels");
        need(energy, "energy");
        int16_t* dl = upload(h->lab, labels, m.N, m.stream);
        *energy = m.energy_true(dl, false);
    });
}

dcrf_status dcrf_model_energy_ho(dcrf_model h, const int16_t* labels, double* energy) {
    return guard([&] {
        auto& m = M(h);
        need(labels, "labels");
        need(energy, "energy");
        int16_t* dl = upload(h->lab, labels, m.N, m.stream);
        *energy = m.energy_true(dl, true);
    });
}

dcrf_status dcrf_model_energy_lp(dcrf_model h, const float* Q, double* energy) {
    return guard([&] {
        auto& m = M(h);
        need(Q, "Q");
        need(energy, "energy");
        float* dq = upload(h->io0, Q, (size_t)m.N * m.L, m.stream);
        *energy = m.energy_lp(dq);
    });
}

dcrf_status dcrf_model_lr_qp_value(dcrf_model h, const float* Q, double* energy) {
    return guard([&] {
        auto& m = M(h);
        need(Q, "Q");
        need(energy, "energy");
        float* dq = upload(h->io0, Q, (size_t)m.N * m.L, m.stream);
        *energy = m.lr_qp_value(dq);
    });
}

dcrf_status dcrf_model_lr_qp_value_diag(dcrf_model h, const float* Q, const float* diag_dom, double* energy) {
    return guard([&] {
        auto& m = M(h);
        need(Q, "Q");
        need(energy, "energy");
        const size_t n = (size_t)m.N * m.L;
        float* dq = upload(h->io0, Q, n, m.stream);
        const float* dd = diag_dom ? upload(h->io1, diag_dom, n, m.stream) : nullptr;
        *energy = m.lr_qp_value(dq, dd);
    });
}

dcrf_status dcrf_model_energy_higher_order(dcrf_model h, const float* Q, double* energy) {
    return guard([&] {
        auto& m = M(h);
        need(Q, "Q");
        need(energy, "energy");
        float* dq = upload(h->io0, Q, (size_t)m.N * m.L, m.stream);
        *energy = m.energy_qp_ho(dq);
    });
}

dcrf_status dcrf_model_unary_energy(dcrf_model h, const int16_t* labels, float* out) {
    return guard([&] {
        auto& m = M(h);
        need(labels, "labels");
        need(out, "out");
        int16_t* dl = upload(h->lab, labels, m.N, m.stream);
        float* dout = h->io1.ensure((size_t)m.N);
        m.unary_energy(dl, dout);
        download(out, dout, (size_t)m.N, m.stream);
    });
}

dcrf_status dcrf_model_pairwise_energy(dcrf_model h, const int16_t* labels, int term, float* out) {
    return guard([&] {
        auto& m = M(h);
        need(labels, "labels");
        need(out, "out");
        int16_t* dl = upload(h->lab, labels, m.N, m.stream);
        float* dout = h->io2.ensure((size_t)m.N);
        m.pairwise_energy(dl, term, dout);
        download(out, dout, (size_t)m.N, m.stream);
    });
}

dcrf_status dcrf_model_max_rounding(dcrf_model h, const float* Q, float* out) {
    return guard([&] {
        auto& m = M(h);
        need(Q, "Q");
        need(out, "out");
        const size_t n = (size_t)m.N * m.L;
        float* dq = upload(h->io0, Q, n, m.stream);
        m.max_rounding(dq, dq);
        download(out, dq, n, m.stream);
    });
}

dcrf_status dcrf_model_info(dcrf_model h, int* n_terms, int* N, int* L) {
    return guard([&] {
        auto& m = M(h);
        if (n_terms) *n_terms = (int)m.terms.size();
        if (N) *N = m.N;
        if (L) *L = m.L;
    });
}

dcrf_status dcrf_model_lattice_size(dcrf_model h, int k, int* Mv) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        need(Mv, "M");
        *Mv = m.terms[k]->lat->M;
    });
}

dcrf_status dcrf_model_pairwise_kernel_gradient(dcrf_model h, int k, const float* b, const float* Q, float* grad,
                                                int* d) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        const auto& t = *m.terms[k];
        const int count = t.ktype == dcrf::kConstKernel ? 0 : t.ktype == dcrf::kDiagKernel ? t.d : t.d * t.d;
        if (d) *d = count;
        if (!grad) return;  // query of the count
        need(b, "b");
        need(Q, "Q");
        const size_t n = (size_t)m.N * m.L;
        const float* db = upload(h->io0, b, n, m.stream);
        const float* dq = upload(h->io1, Q, n, m.stream);
        m.kernel_gradient(k, db, dq, grad);
    });
}

dcrf_status dcrf_model_pairwise_gradient(dcrf_model h, int k, const float* b, const float* Q, float* grad) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        need(b, "b");
        need(Q, "Q");
        need(grad, "grad");
        const size_t n = (size_t)m.N * m.L;
        const float* db = upload(h->io0, b, n, m.stream);
        const float* dq = upload(h->io1, Q, n, m.stream);
        m.compat_gradient(k, db, dq, grad);
    });
}

dcrf_status dcrf_model_pairwise_parameters(dcrf_model h, int k, float* params, int* n) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        if (n) *n = m.n_parameters(k);
        if (params) m.parameters(k, params);
    });
}

dcrf_status dcrf_model_pairwise_set_parameters(dcrf_model h, int k, const float* params) {
    return guard([&] {
        auto& m = M(h);
        check_term(m, k);
        need(params, "params");
        m.set_parameters(k, params);
    });
}

dcrf_status dcrf_model_stream(dcrf_model h, void** stream) {
    return guard([&] {
        auto& m = M(h);
        need(stream, "stream");
        *stream = (void*)m.stream;
    });
}

// ------------------------------------------------------------- batches --

static dcrf::Batch& BT(dcrf_batch h) {
    if (!h || !h->b) throw Error(DCRF_E_ARG, "invalid batch handle");
    return *h->b;
}

dcrf_status dcrf_batch_create(dcrf_batch* out, int n_images, const int* widths, const int* heights, int L) {
    return guard([&] {
        need(out, "out");
        need(widths, "widths");
        need(heights, "heights");
        check_device();
        auto* h = new dcrf_batch_s();
        try {
            h->b = new dcrf::Batch(n_images, widths, heights, L);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

dcrf_status dcrf_batch_destroy(dcrf_batch h) {
    return guard([&] {
        if (!h) return;
        delete h->b;
        delete h;
    });
}

dcrf_status dcrf_batch_info(dcrf_batch h, int64_t* n_pixels, int64_t* offsets) {
    return guard([&] {
        auto& b = BT(h);
        if (n_pixels) *n_pixels = b.Ntot;
        if (offsets)
            for (int i = 0; i <= b.B; i++) offsets[i] = b.pix_off[i];
    });
}

dcrf_status dcrf_batch_set_unary_dev(dcrf_batch h, const float* d_unary) {
    return guard([&] {
        auto& b = BT(h);
        need(d_unary, "unary");
        float* u = b.unary.ensure((size_t)b.Ntot * b.L);
        b.unary_gen++;
        DCRF_CUDA(cudaMemcpyAsync(u, d_unary, sizeof(float) * b.Ntot * b.L, cudaMemcpyDeviceToDevice, b.stream));
        b.has_unary = true;
    });
}

dcrf_status dcrf_batch_set_unary(dcrf_batch h, const float* unary) {
    return guard([&] {
        auto& b = BT(h);
        need(unary, "unary");
        upload(b.unary, unary, (size_t)b.Ntot * b.L, b.stream);
        b.unary_gen++;
        DCRF_CUDA(cudaStreamSynchronize(b.stream));
        b.has_unary = true;
    });
}

dcrf_status dcrf_batch_add_gaussian(dcrf_batch h, float sx, float sy, float w_potts) {
    return guard([&] {
        auto& b = BT(h);
        std::vector<float> f((size_t)2 * b.Ntot);
        for (int n = 0; n < b.B; n++)
            for (int j = 0; j < b.H[n]; j++)
                for (int i = 0; i < b.W[n]; i++) {
                    const size_t p = (size_t)b.pix_off[n] + (size_t)j * b.W[n] + i;
                    f[2 * p] = i / sx;
                    f[2 * p + 1] = j / sy;
                }
        const float* df = upload(h->feat, f.data(), f.size(), b.stream);
        b.add_term(df, 2, w_potts);
        DCRF_CUDA(cudaStreamSynchronize(b.stream));
    });
}

dcrf_status dcrf_batch_add_bilateral(dcrf_batch h, float sx, float sy, float sr, float sg, float sb,
                                     const uint8_t* rgb, float w_potts) {
    return guard([&] {
        auto& b = BT(h);
        need(rgb, "rgb");
        std::vector<float> f((size_t)5 * b.Ntot);
        for (int n = 0; n < b.B; n++)
            for (int j = 0; j < b.H[n]; j++)
                for (int i = 0; i < b.W[n]; i++) {
                    const size_t p = (size_t)b.pix_off[n] + (size_t)j * b.W[n] + i;
                    f[5 * p] = i / sx;
                    f[5 * p + 1] = j / sy;
                    f[5 * p + 2] = rgb[3 * p] / sr;
                    f[5 * p + 3] = rgb[3 * p + 1] / sg;
                    f[5 * p + 4] = rgb[3 * p + 2] / sb;
                }
        const float* df = upload(h->feat, f.data(), f.size(), b.stream);
        b.add_term(df, 5, w_potts);
        DCRF_CUDA(cudaStreamSynchronize(b.stream));
    });
}

dcrf_status dcrf_batch_unary_init(dcrf_batch h, float* Q) {
    return guard([&] {
        auto& b = BT(h);
        need(Q, "Q");
        const size_t n = (size_t)b.Ntot * b.L;
        float* d = h->io0.ensure(n);
        b.unary_init(d);
        download(Q, d, n, b.stream);
    });
}

static void batch_qp(dcrf::Batch& b, const float* d_init, float* d_out, const dcrf_qp_params* params,
                     dcrf_solve_stats* stats) {
    const int max_iter = params ? params->max_iter : 0;
    if (max_iter < 0) throw Error(DCRF_E_ARG, "max_iter must be >= 0");
    std::vector<int> steps(b.B);
    std::vector<double> en(b.B);
    b.qp(d_init, d_out, max_iter, steps.data(), en.data());
    if (stats)
        for (int i = 0; i < b.B; i++) {
            std::memset(stats + i, 0, sizeof(*stats));
            stats[i].iterations = steps[i];
            stats[i].energy = en[i];
        }
}

dcrf_status dcrf_batch_qp_dev(dcrf_batch h, const float* d_init, float* d_out, const dcrf_qp_params* params,
                              dcrf_solve_stats* stats) {
    return guard([&] {
        auto& b = BT(h);
        need(d_init, "init");
        need(d_out, "out");
        batch_qp(b, d_init, d_out, params, stats);
    });
}

dcrf_status dcrf_batch_qp(dcrf_batch h, const float* init, float* out, const dcrf_qp_params* params,
                          dcrf_solve_stats* stats) {
    return guard([&] {
        auto& b = BT(h);
        need(init, "init");
        need(out, "out");
        const size_t n = (size_t)b.Ntot * b.L;
        float* di = upload(h->io0, init, n, b.stream);
        float* dout = h->io1.ensure(n);
        batch_qp(b, di, dout, params, stats);
        download(out, dout, n, b.stream);
    });
}

dcrf_status dcrf_batch_meanfield_dev(dcrf_batch h, int iterations, float* d_Q) {
    return guard([&] { BT(h).meanfield(iterations, d_Q); });
}

dcrf_status dcrf_batch_meanfield(dcrf_batch h, int iterations, float* Q) {
    return guard([&] {
        auto& b = BT(h);
        const size_t n = (size_t)b.Ntot * b.L;
        float* d = Q ? h->io1.ensure(n) : nullptr;
        b.meanfield(iterations, d);
        if (Q) download(Q, d, n, b.stream);
        DCRF_CUDA(cudaStreamSynchronize(b.stream));
    });
}

dcrf_status dcrf_batch_meanfield_backward_dev(dcrf_batch h, const float* d_grad_Q, float* d_grad_U,
                                              double* grad_w) {
    return guard([&] {
        auto& b = BT(h);
        need(d_grad_Q, "grad_Q");
        need(d_grad_U, "grad_U");
        if (!b.terms.empty()) need(grad_w, "grad_w");
        b.meanfield_backward(d_grad_Q, d_grad_U, grad_w);
    });
}

dcrf_status dcrf_batch_meanfield_backward(dcrf_batch h, const float* grad_Q, float* grad_U, double* grad_w) {
    return guard([&] {
        auto& b = BT(h);
        need(grad_Q, "grad_Q");
        need(grad_U, "grad_U");
        if (!b.terms.empty()) need(grad_w, "grad_w");
        const size_t n = (size_t)b.Ntot * b.L;
        const float* dg = upload(h->io0, grad_Q, n, b.stream);
        float* du = h->io1.ensure(n);
        b.meanfield_backward(dg, du, grad_w);
        download(grad_U, du, n, b.stream);
    });
}

dcrf_status dcrf_batch_set_weight(dcrf_batch h, int k, float w_potts) {
    return guard([&] { BT(h).set_weight(k, w_potts); });
}

dcrf_status dcrf_batch_set_checkpointing(dcrf_batch h, int checkpoint_every, int recompute_lattice) {
    return guard([&] { BT(h).set_checkpointing(checkpoint_every, recompute_lattice != 0); });
}

dcrf_status dcrf_batch_meanfield_state_bytes(dcrf_batch h, int T, uint64_t* bytes) {
    return guard([&] {
        need(bytes, "bytes");
        dcrf::require(T >= 0 && T <= 1000, DCRF_E_ARG, "iterations must be in [0, 1000]");
        *bytes = BT(h).meanfield_state_bytes(T);
    });
}

dcrf_status dcrf_batch_terms(dcrf_batch h, int* n_terms) {
    return guard([&] {
        need(n_terms, "n_terms");
        *n_terms = (int)BT(h).terms.size();
    });
}

dcrf_status dcrf_batch_pairwise_apply_dev(dcrf_batch h, int k, float* d_out, const float* d_in) {
    return guard([&] {
        auto& b = BT(h);
        need(d_out, "out");
        need(d_in, "in");
        dcrf::require(k >= 0 && k < (int)b.terms.size(), DCRF_E_ARG, "pairwise term index out of range");
        b.apply(k, d_out, d_in);
    });
}

dcrf_status dcrf_batch_pairwise_apply(dcrf_batch h, int k, float* out, const float* in) {
    return guard([&] {
        auto& b = BT(h);
        need(out, "out");
        need(in, "in");
        dcrf::require(k >= 0 && k < (int)b.terms.size(), DCRF_E_ARG, "pairwise term index out of range");
        const size_t n = (size_t)b.Ntot * b.L;
        upload(h->io0, in, n, b.stream);
        float* d = h->io1.ensure(n);
        b.apply(k, d, h->io0.get());
        download(out, d, n, b.stream);
        DCRF_CUDA(cudaStreamSynchronize(b.stream));
    });
}

dcrf_status dcrf_batch_filter_shape(dcrf_batch h, int k, int* shape) {
    return guard([&] {
        auto& b = BT(h);
        need(shape, "shape");
        dcrf::require(k >= 0 && k < (int)b.terms.size(), DCRF_E_ARG, "pairwise term index out of range");
        b.ensure_lattices();
        shape_to(b.terms[k]->lat->shape, shape);
    });
}

dcrf_status dcrf_batch_set_filter_shape(dcrf_batch h, int k, const int* shape) {
    return guard([&] {
        auto& b = BT(h);
        dcrf::require(k >= 0 && k < (int)b.terms.size(), DCRF_E_ARG, "pairwise term index out of range");
        const dcrf::FilterShape f = shape_from(shape);
        b.ensure_lattices();
        b.terms[k]->lat->shape = f;
        b.terms[k]->lat->shape_L = 21;  // pinned: no tuning for this lattice
    });
}

dcrf_status dcrf_batch_lattice_size(dcrf_batch h, int k, int64_t* M) {
    return guard([&] {
        auto& b = BT(h);
        need(M, "M");
        dcrf::require(k >= 0 && k < (int)b.terms.size(), DCRF_E_ARG, "pairwise term index out of range");
        *M = b.terms[k]->lat->M;
    });
}

dcrf_status dcrf_batch_stream(dcrf_batch h, void** stream) {
    return guard([&] {
        auto& b = BT(h);
        need(stream, "stream");
        *stream = (void*)b.stream;
    });
}

}  // extern "C"
