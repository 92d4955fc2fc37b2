// Self-test of the drop-in C++ API (densecrf.h) on the B200 engine.
// Usage: shim_selftest W H L rgb.u8 unary.f32 out_prefix
// Builds the example's Gaussian + bilateral Potts model through the
// reference-named classes, runs unary_init, the QP and a short LP, a
// standalone Permutohedral filter and PairwisePotential, and a QP of a model
// with Diagonal and Matrix compatibilities; writes the results as raw float32
// files <out_prefix>.{init,qp,lp,filt,pw,qpc}; energies and the error-path
// checks go to stdout.
#include <cstdio>
#include <algorithm>
#include <fstream>
#include <iostream>
#include <vector>

#include "densecrf.h"

template <typename T>
static std::vector<T> read_raw(const char* path, size_t n) {
    std::vector<T> v(n);
    std::ifstream f(path, std::ios::binary);
    f.read(reinterpret_cast<char*>(v.data()), sizeof(T) * n);
    if (!f) throw std::runtime_error(std::string("cannot read ") + path);
    return v;
}

static void write_raw(const std::string& path, const MatrixXf& m) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(m.data()), sizeof(float) * m.size());
}

int main(int argc, char** argv) {
    if (argc != 7) {
        std::cerr << "usage: shim_selftest W H L rgb.u8 unary.f32 out_prefix\n";
        return 2;
    }
    const int W = std::atoi(argv[1]), H = std::atoi(argv[2]), L = std::atoi(argv[3]), N = W * H;
    const std::string out = argv[6];
    try {
        std::vector<unsigned char> rgb = read_raw<unsigned char>(argv[4], (size_t)N * 3);
        std::vector<float> u = read_raw<float>(argv[5], (size_t)N * L);
        MatrixXf U = Map<MatrixXf>(u.data(), L, N);

        DenseCRF2D crf(W, H, L);
        crf.setUnaryEnergy(U);
        crf.addPairwiseGaussian(3, 3, new PottsCompatibility(3));
        crf.addPairwiseBilateral(50, 50, 15, 15, 15, rgb.data(), new PottsCompatibility(5));
        MatrixXf Q = crf.unary_init();
        MatrixXf qp = crf.qp_inference_super_pixels_non_convex(Q);
        LP_inf_params p;
        p.prox_energy_tol = p.dual_gap_tol;
        p.prox_max_iter = 3;
        p.fw_max_iter = 3;
        MatrixXf lp = crf.lp_inference_prox_super_pixels(Q, p);
        printf("qp_energy %.10f\n", crf.assignment_energy_true(crf.currentMap(qp)));
        printf("lp_energy %.10f\n", crf.assignment_energy_true(crf.currentMap(lp)));

        MatrixXf F(2, N);
        for (int j = 0; j < H; j++)
            for (int i = 0; i < W; i++) {
                F(0, j * W + i) = i / 3.0f;
                F(1, j * W + i) = j / 3.0f;
            }
        Permutohedral lat;
        lat.init(F);
        MatrixXf filt = lat.compute(Q);
        printf("lattice_M %d\n", lat.size());
        PairwisePotential pw(F, new PottsCompatibility(3));
        MatrixXf pwo;
        pw.apply(pwo, Q);
        // the divide-and-conquer filter on the positions sorted by decreasing Q
        Eigen::MatrixXi ind(L, N);
        for (int l = 0; l < L; l++) {
            std::vector<int> o(N);
            for (int c = 0; c < N; c++) o[c] = c;
            std::stable_sort(o.begin(), o.end(), [&](int a, int b) { return Q(l, a) > Q(l, b); });
            for (int c = 0; c < N; c++) ind(l, c) = o[c];
        }
        MatrixXf dco;
        pw.apply_upper_minus_lower_dc(dco, ind);

        MatrixXf bad = Q;
        bad(0, 0) = 2.0f;  // out of [0, 1]
        try {
            MatrixXf o;
            pw.apply_upper_minus_lower_ord(o, bad);
            printf("range_error missing\n");
        } catch (const std::runtime_error& e) {
            printf("range_error %s\n", e.what());
        }
        try {
            crf.addPairwiseGaussian(3, 3, new PottsCompatibility(1), DIAG_KERNEL, (NormalizationType)7);
            printf("kernel_error missing\n");
        } catch (const std::runtime_error& e) {
            printf("kernel_error ok\n");
        }

        // Diagonal on the Gaussian term, Matrix on the bilateral one.
        VectorXf dg(L);
        MatrixXf mt(L, L);
        for (int a = 0; a < L; a++) {
            dg[a] = -(2.0f + 0.1f * a);
            for (int b = 0; b < L; b++) mt(a, b) = a == b ? -5.0f : 0.1f * (a + 2 * b) / L;
        }
        DenseCRF2D crf2(W, H, L);
        crf2.setUnaryEnergy(U);
        crf2.addPairwiseGaussian(3, 3, new DiagonalCompatibility(dg));
        crf2.addPairwiseBilateral(50, 50, 15, 15, 15, rgb.data(), new MatrixCompatibility(mt));
        MatrixXf qpc = crf2.qp_inference_super_pixels_non_convex(crf2.unary_init());
        printf("compat_energy %.10f\n", crf2.assignment_energy_true(crf2.currentMap(qpc)));
        write_raw(out + ".qpc", qpc);
        write_raw(out + ".init", Q);
        write_raw(out + ".qp", qp);
        write_raw(out + ".lp", lp);
        write_raw(out + ".filt", filt);
        write_raw(out + ".pw", pwo);
        write_raw(out + ".dc", dco);
    } catch (const std::exception& e) {
        fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
