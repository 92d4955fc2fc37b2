// Mean-shift superpixels for DenseCRF2D::addSuperPixel (src/densecrf.cpp:
// 193-251), which segments the image with EDISON's msImageProcessor
// (DefineImage(img, COLOR, H, W); Segment(spatial, range, min_region,
// NO_SPEEDUP); GetRegions) and turns every region into a clique.
//
// The segmentation is the published mean-shift procedure of Comaniciu and
// Meer with EDISON's choices, which decide the regions and are kept as they
// are:
//   1. CIE L*u*v* of every pixel (msImageProcessor::RGBtoLUV, :846-890);
//   2. per pixel, mean-shift mode seeking with the uniform kernel in the
//      joint domain (x, y) / sigmaS, (L, u, v) / sigmaR, the neighbours found
//      through a grid of unit buckets over (x, y, L), sums in double
//      precision (NewNonOptimizedFilter, :3555-3907) -- the data-parallel
//      step, one GPU thread per pixel (ms_filter_kernel);
//   3. 8-connected labelling of the filtered image, colours closer than 0.1
//      in every channel joining (Connect / Fill, :1166-1330);
//   4. transitive closure over the region adjacency graph, joining adjacent
//      regions whose modes lie within sigmaR / 2 (TransitiveClosure,
//      :1600-1812, repeated as Segment does, :750-765);
//   5. pruning of regions smaller than min_region into their nearest
//      adjacent region (Prune, :1985-2232).
// Steps 3-5 are sequential graph work on a few hundred thousand labels and
// run on the host.  Every float / double operation follows EDISON's order,
// so the regions are the reference's own.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "meanshift.cuh"

namespace dcrf {

namespace {

// The filter's working point of one pixel: x / sigmaS, y / sigmaS and the
// three L*u*v* channels / sigmaR, each a float quotient held in double
// (EDISON builds them from int and float operands).
constexpr int kMsDim = 5;
constexpr double kMsEpsilon = 0.01;    // squared shift length at which a window has converged
constexpr int kMsLimit = 100;          // iterations per pixel at most
constexpr float kLuvThreshold = 0.1f;  // Fill: channels closer than this join a region

struct MsGrid {
    int N = 0;
    int nb1 = 0, nb2 = 0, nb3 = 0;
    double smin = 0.0;  // smallest L / sigmaR
    double hi_l = 0.0;  // 80 / sigmaR: above it the L distance counts four-fold
    float sigma_s = 0.0f, sigma_r = 0.0f;
};

// One window shift at yk: Mh = mean of the points within the unit window
// minus yk (zero when the window is empty).  The 27 buckets around yk's are
// visited x-offset outermost, L-offset innermost, and each bucket's points
// in decreasing pixel order -- the order EDISON's prepended bucket lists
// walk -- so the double sums are the reference's.
__device__ void ms_shift(const MsGrid& g, const double* __restrict__ cand, const int* __restrict__ bstart,
                         const double (&yk)[kMsDim], double (&Mh)[kMsDim]) {
#pragma unroll
    for (int j = 0; j < kMsDim; j++) Mh[j] = 0.0;
    double wsum = 0.0;
    const int c1 = (int)yk[0] + 1, c2 = (int)yk[1] + 1, c3 = (int)__dsub_rn(yk[2], g.smin) + 1;
    const int nb = g.nb1 * g.nb2 * g.nb3;
    const int cb = c1 + g.nb1 * (c2 + g.nb2 * c3);
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++)
            for (int c = -1; c <= 1; c++) {
                const int bk = cb + a + g.nb1 * (b + g.nb2 * c);
                if (bk < 0 || bk >= nb) continue;  // a window inside the data never leaves the grid
                const int e1 = bstart[bk + 1];
                for (int k = bstart[bk]; k < e1; k++) {
                    const double* s = cand + (long)k * kMsDim;
                    double el = __dsub_rn(s[0], yk[0]);
                    double diff = __dmul_rn(el, el);
                    el = __dsub_rn(s[1], yk[1]);
                    diff = __dadd_rn(diff, __dmul_rn(el, el));
                    if (diff < 1.0) {
                        el = __dsub_rn(s[2], yk[2]);
                        diff = yk[2] > g.hi_l ? __dmul_rn(__dmul_rn(4.0, el), el) : __dmul_rn(el, el);
                        el = __dsub_rn(s[3], yk[3]);
                        diff = __dadd_rn(diff, __dmul_rn(el, el));
                        el = __dsub_rn(s[4], yk[4]);
                        diff = __dadd_rn(diff, __dmul_rn(el, el));
                        if (diff < 1.0) {  // uniform kernel, weight 1
#pragma unroll
                            for (int j = 0; j < kMsDim; j++) Mh[j] = __dadd_rn(Mh[j], s[j]);
                            wsum = __dadd_rn(wsum, 1.0);
                        }
                    }
                }
            }
    if (wsum > 0.0) {
#pragma unroll
        for (int j = 0; j < kMsDim; j++) Mh[j] = __dsub_rn(__ddiv_rn(Mh[j], wsum), yk[j]);
    } else {
#pragma unroll
        for (int j = 0; j < kMsDim; j++) Mh[j] = 0.0;
    }
}

// Mode seeking from every pixel: shift until the squared shift (the first
// one unscaled, later ones rescaled to pixel and colour units) drops below
// kMsEpsilon or kMsLimit iterations ran; out = the mode's colour times
// sigmaR, rounded to float.
__global__ void ms_filter_kernel(MsGrid g, const double* __restrict__ pts, const double* __restrict__ cand,
                                 const int* __restrict__ bstart, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    double yk[kMsDim], Mh[kMsDim];
#pragma unroll
    for (int j = 0; j < kMsDim; j++) yk[j] = pts[(long)i * kMsDim + j];
    ms_shift(g, cand, bstart, yk, Mh);
    double mv = 0.0;
#pragma unroll
    for (int j = 0; j < kMsDim; j++) mv = __dadd_rn(mv, __dmul_rn(Mh[j], Mh[j]));
    const double ss = g.sigma_s, sr = g.sigma_r;
    int it = 1;
    while (mv >= kMsEpsilon && it < kMsLimit) {
#pragma unroll
        for (int j = 0; j < kMsDim; j++) yk[j] = __dadd_rn(yk[j], Mh[j]);
        ms_shift(g, cand, bstart, yk, Mh);
        mv = __dmul_rn(__dmul_rn(__dadd_rn(__dmul_rn(Mh[0], Mh[0]), __dmul_rn(Mh[1], Mh[1])), ss), ss);
        const double cr =
            __dadd_rn(__dadd_rn(__dmul_rn(Mh[2], Mh[2]), __dmul_rn(Mh[3], Mh[3])), __dmul_rn(Mh[4], Mh[4]));
        mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(cr, sr), sr));
        it++;
    }
#pragma unroll
    for (int j = 0; j < kMsDim; j++) yk[j] = __dadd_rn(yk[j], Mh[j]);
#pragma unroll
    for (int j = 0; j < 3; j++) out[(long)i * 3 + j] = (float)__dmul_rn(yk[j + 2], sr);
}

// ---------------------------------------------------------------- host --

// RGB -> CIE L*u*v* with EDISON's D65 constants (msImageProcessor.h:62-75)
// and its arithmetic: XYZ by the 3x3 matrix in double, L* by the cube root
// above the linear segment, u* / v* from the chromaticities (4, 9/15 for
// black), each channel rounded to float where EDISON stores it.
void rgb_to_luv(const uint8_t* c, float* luv) {
    static const double M[3][3] = {{0.4125, 0.3576, 0.1804}, {0.2125, 0.7154, 0.0721}, {0.0193, 0.1192, 0.9502}};
    const double Yn = 1.0, Un = 0.19784977571475, Vn = 0.46834507665248, Lt = 0.008856;
    const double x = M[0][0] * c[0] + M[0][1] * c[1] + M[0][2] * c[2];
    const double y = M[1][0] * c[0] + M[1][1] * c[1] + M[1][2] * c[2];
    const double z = M[2][0] * c[0] + M[2][1] * c[1] + M[2][2] * c[2];
    const double l0 = y / (255.0 * Yn);
    luv[0] = l0 > Lt ? (float)(116.0 * std::pow(l0, 1.0 / 3.0) - 16.0) : (float)(903.3 * l0);
    const double den = x + 15 * y + 3 * z;
    double up = 4.0, vp = 9.0 / 15.0;
    if (den != 0) {
        up = (4 * x) / den;
        vp = (9 * y) / den;
    }
    luv[1] = (float)(13 * luv[0] * (up - Un));
    luv[2] = (float)(13 * luv[0] * (vp - Vn));
}

// The region state EDISON's classification keeps: a label per pixel, and
// per region its mode colour and its pixel count.
struct RegionState {
    int W = 0, H = 0, count = 0;
    float sigma_r = 0.0f;
    std::vector<int> labels, npix;
    std::vector<float> modes;           // [count][3]
    std::vector<std::vector<int>> adj;  // ascending adjacent labels (the region adjacency lists)
    std::vector<int> parent;            // canonical-element links

    // Region adjacency from the labelling: a pixel and its right and lower
    // neighbours with different labels are adjacent (BuildRAM, :1336-1565).
    void build_adjacency() {
        adj.assign(count, {});
        parent.resize(count);
        for (int r = 0; r < count; r++) parent[r] = r;
        auto link = [&](int a, int b) {
            if (a == b) return;
            adj[a].push_back(b);
            adj[b].push_back(a);
        };
        for (int i = 0; i < H; i++)
            for (int j = 0; j < W; j++) {
                const int c = labels[i * W + j];
                if (j + 1 < W) link(c, labels[i * W + j + 1]);
                if (i + 1 < H) link(c, labels[(i + 1) * W + j]);
            }
        for (auto& a : adj) {
            std::sort(a.begin(), a.end());
            a.erase(std::unique(a.begin(), a.end()), a.end());
        }
    }
    int canonical(int r) const {
        while (parent[r] != r) r = parent[r];
        return r;
    }
    // Joins the trees of a and b under the smaller canonical element, with
    // EDISON's two link updates.
    void join(int a, int b) {
        const int ca = canonical(a), cb = canonical(b);
        if (ca < cb) {
            parent[cb] = ca;
        } else {
            parent[parent[ca]] = cb;
            parent[ca] = cb;
        }
    }
    // Relabels by the joined trees: the new label order is the order in which
    // canonical elements first appear, modes are the pixel-count-weighted
    // means of the joined modes (float), counts are summed.
    void relabel() {
        for (int r = 0; r < count; r++) parent[r] = canonical(r);
        std::vector<float> mb((size_t)3 * count, 0.0f);
        std::vector<int> nb(count, 0), lb(count, -1);
        for (int r = 0; r < count; r++) {
            const int c = parent[r], m = npix[r];
            for (int k = 0; k < 3; k++) mb[3 * c + k] += (float)m * modes[3 * r + k];
            nb[c] += m;
        }
        int label = -1;
        for (int r = 0; r < count; r++) {
            const int c = parent[r];
            if (lb[c] < 0) {
                lb[c] = ++label;
                for (int k = 0; k < 3; k++) modes[3 * label + k] = mb[3 * c + k] / (float)nb[c];
                npix[label] = nb[c];
            }
        }
        count = label + 1;
        for (auto& l : labels) l = lb[parent[l]];
    }
    // Modes within sigmaR / 2 of each other, the L distance counting four-fold
    // when the first mode's L exceeds 80 (InWindow, :2408-2440).
    bool in_window(int a, int b) const {
        double d = 0.0;
        for (int p = 0; p < 3; p++) {
            const double el = (modes[3 * a + p] - modes[3 * b + p]) / (sigma_r * 1.0f);
            d += (p == 0 && modes[3 * a] > 80) ? 4 * el * el : el * el;
        }
        return d < 0.25;
    }
    // Normalised squared colour distance in float (SqDistance, :2447-2470).
    float sq_distance(int a, int b) const {
        float d = 0.0f;
        for (int p = 0; p < 3; p++) {
            const float el = (modes[3 * a + p] - modes[3 * b + p]) / (sigma_r * 1.0f);
            d += el * el;
        }
        return d;
    }
};

// 8-connected labelling of the filtered colours (Connect / Fill): regions
// are grown from every unlabelled pixel in scan order with EDISON's
// explicit stack, neighbours taken by index offset (so the left and right
// neighbours of a row's ends are the adjacent rows' pixels, as there).
void connect(RegionState& st, const float* luv) {
    const int W = st.W, n = st.W * st.H;
    const int neigh[8] = {1, 1 - W, -W, -(1 + W), -1, W - 1, W, W + 1};
    st.labels.assign(n, -1);
    st.npix.assign(n, 0);
    st.modes.assign((size_t)3 * n, 0.0f);
    std::vector<int> stack(n);
    int label = -1;
    for (int i = 0; i < n; i++) {
        if (st.labels[i] >= 0) continue;
        st.labels[i] = ++label;
        for (int k = 0; k < 3; k++) st.modes[3 * label + k] = luv[3 * i + k];
        int loc = i, top = 0;
        stack[0] = loc;
        st.npix[label]++;
        for (;;) {
            bool found = false;
            for (int q = 0; q < 8; q++) {
                const int nl = loc + neigh[q];
                if (nl < 0 || nl >= n || st.labels[nl] >= 0) continue;
                int k = 0;
                while (k < 3 && std::fabs(luv[loc * 3 + k] - luv[nl * 3 + k]) < kLuvThreshold) k++;
                if (k == 3) {
                    st.labels[nl] = label;
                    st.npix[label]++;
                    stack[++top] = nl;
                    found = true;
                }
            }
            if (found) loc = stack[top];
            else if (top > 1) loc = stack[--top];
            else break;
        }
    }
    st.count = label + 1;
}

// One transitive-closure pass: every region joins each adjacent region
// whose mode is within the window (TransitiveClosure).
void transitive_closure(RegionState& st) {
    st.build_adjacency();
    for (int r = 0; r < st.count; r++)
        for (int nbr : st.adj[r])
            if (st.in_window(r, nbr)) st.join(r, nbr);
    st.relabel();
}

// Regions under min_region pixels join their nearest adjacent region in
// colour, pass after pass until none is left (Prune).
void prune(RegionState& st, int min_region) {
    for (;;) {
        int small = 0;
        st.build_adjacency();
        for (int r = 0; r < st.count; r++) {
            if (st.npix[r] >= min_region) continue;
            small++;
            if (st.adj[r].empty()) continue;  // the whole image is one region
            int best = st.adj[r][0];
            double dmin = st.sq_distance(r, best);
            for (size_t q = 1; q < st.adj[r].size(); q++) {
                const double dd = st.sq_distance(r, st.adj[r][q]);
                if (dd < dmin) {
                    dmin = dd;
                    best = st.adj[r][q];
                }
            }
            st.join(r, best);
        }
        st.relabel();
        if (small == 0 || st.count <= 1) break;
    }
}

// Eigen 3.2's pexp<Packet4f> (Core/arch/SSE/MathFunctions.h:107-170) for the
// reference's SSE2 build, one lane, on the host: the Cephes single-precision
// exp, every product and sum rounded on its own (the host compiler emits
// them without contraction), n = floor(x log2(e) + 1/2) by truncation and
// correction, 2^n built in the exponent bits, then the max with the input.
float eigen_pexp_host(float x0) {
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
    std::memcpy(&p2, &bits, sizeof p2);
    const float r = y * p2;
    return r > x0 ? r : x0;
}

}  // namespace

void superpixel_cliques(const uint8_t* img, const int* labels, int N, int reg, int existing, float constant,
                        float normaliser, std::vector<int>& offsets, std::vector<int>& idx,
                        std::vector<float>& exp_weight, std::vector<float>& constants) {
    // Float accumulators updated with double terms, as addSuperPixel's
    // VectorXf members are (the grey level reads bytes i, i+1, i+2 of
    // pixel i: the reference's indexing, kept).
    std::vector<float> mean(reg, 0.0f), cnt(reg, 0.0f), sd(reg, 0.0f);
    std::vector<int> size(reg, 0);
    for (int i = 0; i < N; i++) {
        const int r = labels[i];
        mean[r] = (float)((double)mean[r] + 0.2989 * (double)img[i]);
        mean[r] = (float)((double)mean[r] + 0.5870 * (double)img[i + 1]);
        mean[r] = (float)((double)mean[r] + 0.1140 * (double)img[i + 2]);
        cnt[r] += 1.0f;
        size[r]++;
    }
    for (int r = 0; r < reg; r++) mean[r] = mean[r] / cnt[r];
    for (int i = 0; i < N; i++) {
        const int r = labels[i];
        const double grey = 0.2989 * (double)img[i] + 0.5870 * (double)img[i + 1] + 0.1140 * (double)img[i + 2];
        const double dv = (double)mean[r] - grey;
        sd[r] = (float)((double)sd[r] + dv * dv);
    }
    for (int r = 0; r < reg; r++) sd[r] = sd[r] / (normaliser * cnt[r]);
    // constant * exp(-sd) is written into exp_of_superpixels_.tail(reg):
    // Eigen runs its packet exp over the elements whose destination is
    // 16-byte aligned in whole packets of four and std::exp over the rest,
    // so which is which depends on the `existing` entries before them.
    const int head = std::min((4 - existing % 4) % 4, reg);
    const int body_end = head + ((reg - head) / 4) * 4;
    exp_weight.resize(reg);
    for (int r = 0; r < reg; r++) {
        const float v = -sd[r];
        exp_weight[r] = constant * ((r >= head && r < body_end) ? eigen_pexp_host(v) : std::exp(v));
    }
    constants.assign(reg, constant);
    offsets.assign(reg + 1, 0);
    for (int r = 0; r < reg; r++) offsets[r + 1] = offsets[r] + size[r];
    idx.resize(N);
    std::vector<int> pos(offsets.begin(), offsets.end() - 1);
    for (int i = 0; i < N; i++) idx[pos[labels[i]]++] = i;
}

void meanshift_filter(const uint8_t* rgb, int W, int H, int spatial_radius, float range_radius, float* filtered,
                      cudaStream_t stream) {
    require(W > 0 && H > 0, DCRF_E_ARG, "mean shift: image size must be positive");
    require(spatial_radius > 0 && range_radius > 0.0f, DCRF_E_ARG,
            "mean shift: spatial and range radius must be positive");
    require((long)W * H < (1L << 28), DCRF_E_ARG, "mean shift: image too large");
    const int N = W * H;
    const float ss = (float)spatial_radius, sr = range_radius;
    std::vector<float> luv((size_t)3 * N);
    for (int i = 0; i < N; i++) rgb_to_luv(rgb + 3 * i, &luv[(size_t)3 * i]);

    // the filter's points and EDISON's bucket grid over (x, y, L)
    std::vector<double> pts((size_t)kMsDim * N);
    for (int i = 0; i < N; i++) {
        double* p = &pts[(size_t)kMsDim * i];
        p[0] = (float)(i % W) / ss;
        p[1] = (float)(i / W) / ss;
        for (int k = 0; k < 3; k++) p[2 + k] = luv[(size_t)3 * i + k] / sr;
    }
    MsGrid g;
    g.N = N;
    g.sigma_s = ss;
    g.sigma_r = sr;
    double smax2 = pts[2];
    g.smin = pts[2];
    for (int i = 0; i < N; i++) {
        const double v = pts[(size_t)kMsDim * i + 2];
        if (v < g.smin) g.smin = v;
        else if (v > smax2) smax2 = v;
    }
    g.nb1 = (int)((double)((float)W / ss) + 3);
    g.nb2 = (int)((double)((float)H / ss) + 3);
    g.nb3 = (int)(smax2 - g.smin + 3);
    g.hi_l = 80.0 / sr;
    const long nb = (long)g.nb1 * g.nb2 * g.nb3;
    require(nb < (1L << 30), DCRF_E_ARG, "mean shift: bucket grid too large");
    std::vector<int> bucket(N), bstart(nb + 1, 0);
    for (int i = 0; i < N; i++) {
        const double* p = &pts[(size_t)kMsDim * i];
        const int c1 = (int)p[0] + 1, c2 = (int)p[1] + 1, c3 = (int)(p[2] - g.smin) + 1;
        bucket[i] = c1 + g.nb1 * (c2 + g.nb2 * c3);
        bstart[bucket[i] + 1]++;
    }
    for (long b = 0; b < nb; b++) bstart[b + 1] += bstart[b];
    // within a bucket, decreasing pixel order (EDISON prepends to its lists)
    std::vector<int> fill(bstart.begin(), bstart.end() - 1);
    std::vector<double> cand((size_t)kMsDim * N);
    for (int i = N - 1; i >= 0; i--) {
        const int slot = fill[bucket[i]]++;
        std::memcpy(&cand[(size_t)kMsDim * slot], &pts[(size_t)kMsDim * i], sizeof(double) * kMsDim);
    }

    DevBuf<double> d_pts, d_cand;
    DevBuf<int> d_bstart;
    DevBuf<float> d_out;
    DCRF_CUDA(cudaMemcpyAsync(d_pts.ensure(pts.size()), pts.data(), sizeof(double) * pts.size(),
                              cudaMemcpyHostToDevice, stream));
    DCRF_CUDA(cudaMemcpyAsync(d_cand.ensure(cand.size()), cand.data(), sizeof(double) * cand.size(),
                              cudaMemcpyHostToDevice, stream));
    DCRF_CUDA(cudaMemcpyAsync(d_bstart.ensure(bstart.size()), bstart.data(), sizeof(int) * bstart.size(),
                              cudaMemcpyHostToDevice, stream));
    float* out = d_out.ensure((size_t)3 * N);
    launch(ms_filter_kernel, ceil_div(N, 128), 128, 0, stream, g, (const double*)d_pts.get(),
           (const double*)d_cand.get(), (const int*)d_bstart.get(), out);
    DCRF_LAUNCH_CHECK();
    DCRF_CUDA(cudaMemcpyAsync(filtered, out, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost, stream));
    DCRF_CUDA(cudaStreamSynchronize(stream));  // the host vectors above are the copies' sources
}

int meanshift_regions(const float* filtered, int W, int H, float range_radius, int min_region, int* labels) {
    require(W > 0 && H > 0, DCRF_E_ARG, "mean shift: image size must be positive");
    require(range_radius > 0.0f, DCRF_E_ARG, "mean shift: range radius must be positive");
    RegionState st;
    st.W = W;
    st.H = H;
    st.sigma_r = range_radius;
    connect(st, filtered);
    transitive_closure(st);
    int old = st.count;
    for (int pass = 0; pass < 10; pass++) {  // Segment's loop: until a pass removes regions, 10 at most
        transitive_closure(st);
        const int delta = old - st.count;
        old = st.count;
        if (delta > 0) break;
    }
    prune(st, min_region);
    std::memcpy(labels, st.labels.data(), sizeof(int) * (size_t)W * H);
    return st.count;
}

int meanshift_segment(const uint8_t* rgb, int W, int H, int spatial_radius, float range_radius, int min_region,
                      int* labels, cudaStream_t stream) {
    std::vector<float> filtered((size_t)3 * W * H);
    meanshift_filter(rgb, W, H, spatial_radius, range_radius, filtered.data(), stream);
    return meanshift_regions(filtered.data(), W, H, range_radius, min_region, labels);
}

}  // namespace dcrf
