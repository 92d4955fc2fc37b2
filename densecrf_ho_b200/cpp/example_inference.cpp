// Headless example_inference on the B200 engine: the argument grammar,
// defaults and output lines of src/example_inference.cpp:88-134, through the
// drop-in C++ API (densecrf.h) and the OpenCV-free readers of file_io.h.
//
//   example_inference method [spc_std spc_potts bil_spcstd bil_colstd bil_potts [const_1 norm_1]]
//
// method: qp, qp_sp, lp, lp_sp or unary.  Input and output paths are the
// reference's (../data/img.bmp, ../data/img.c_unary) unless DCRF_IMAGE /
// DCRF_UNARY / DCRF_OUTPUT name others; the labelling is written as a PGM
// (../data/seg.pgm by default).
//
// qp_sp / lp_sp add superpixel cliques as the reference does:
// addSuperPixel(img, 8, 4, 100, const_1, norm_1), the engine's own EDISON
// mean-shift segmentation (spatial radius 8, range 4, minimum region 100).
//
// Extra modes, no GPU needed: example_inference --dump-unary in.c_unary
// out.f32 writes the decoded unaries [N][D] as raw float32, and
// --dump-image in.bmp out.u8 the decoded RGB [H][W][3].
#include <chrono>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "densecrf.h"
#include "file_io.h"

namespace {

struct sp_params {
    float const_1;
    float norm_1;
};

std::string env_or(const char* name, const char* dflt) {
    const char* v = std::getenv(name);
    return v && *v ? std::string(v) : std::string(dflt);
}

void image_inference(const std::string& method, const std::string& path_to_results, const std::string& path_to_image,
                     const std::string& path_to_unaries, float spc_std, float spc_potts, float bil_spcstd,
                     float bil_colstd, float bil_potts, LP_inf_params& lp_params, sp_params params) {
    int W = 0, H = 0, D = 0, Wi = 0, Hi = 0;
    std::vector<float> u = dcrf_io::load_unary(path_to_unaries, W, H, D);
    std::vector<unsigned char> img = dcrf_io::load_bmp(path_to_image, Wi, Hi);
    if (Wi != W || Hi != H) throw std::runtime_error("image and unaries differ in size");
    MatrixXf unaries = Map<MatrixXf>(u.data(), D, (long)W * H);

    DenseCRF2D crf(W, H, D);
    crf.setUnaryEnergy(unaries);
    crf.addPairwiseGaussian(spc_std, spc_std, new PottsCompatibility(spc_potts));
    crf.addPairwiseBilateral(bil_spcstd, bil_spcstd, bil_colstd, bil_colstd, bil_colstd, img.data(),
                             new PottsCompatibility(bil_potts));
    MatrixXf Q = crf.unary_init();

    auto add_superpixels = [&]() { crf.addSuperPixel(img.data(), 8, 4, 100, params.const_1, params.norm_1); };
    if (method == "lp_sp") {
        std::cout << "---Running tests on proximal LP with higher order potentials\r\n";
        add_superpixels();
        try {
            Q = crf.lp_inference_prox_super_pixels(Q, lp_params);
        } catch (std::runtime_error& e) {
            std::cout << "Runtime Error!: " << e.what() << std::endl;
        }
    } else if (method == "lp") {
        std::cout << "---Running tests on proximal LP\r\n";
        Q = crf.lp_inference_prox_super_pixels(Q, lp_params);
    } else if (method == "qp") {
        std::cout << "---Running tests on QP with non convex energy\r\n";
        Q = crf.qp_inference_super_pixels_non_convex(Q);
    } else if (method == "qp_sp") {
        std::cout << "---Running tests on QP with non convex energy with higher order potentials\r\n";
        add_superpixels();
        Q = crf.qp_inference_super_pixels_non_convex(Q);
    } else if (method == "unary") {
        (void)0;
    } else {
        std::cout << "Unrecognised method.\n Proper error handling would do something but I won't." << '\n';
    }

    // The reference reports the higher-order energy for qp_sp only (its
    // second test names "prox_lp_sp", which no method is called).
    const VectorXs map = crf.currentMap(Q);
    const double discretized_energy =
        method == "qp_sp" ? crf.assignment_energy_higher_order(map) : crf.assignment_energy_true(map);
    dcrf_io::save_labels(path_to_results, std::vector<short>(map.data(), map.data() + map.size()), W, H);
    std::cout << "# method: " << method << '\t' << discretized_energy << std::endl;
}

}  // namespace

int main(int argc, char* argv[]) {
    if (argc == 4 && std::string(argv[1]) == "--dump-unary") {
        try {
            int W, H, D;
            std::vector<float> u = dcrf_io::load_unary(argv[2], W, H, D);
            FILE* fp = fopen(argv[3], "wb");
            if (!fp) throw std::runtime_error(std::string("cannot write ") + argv[3]);
            fwrite(u.data(), sizeof(float), u.size(), fp);
            fclose(fp);
            std::cout << W << " " << H << " " << D << std::endl;
            return 0;
        } catch (const std::exception& e) {
            std::cerr << "error: " << e.what() << std::endl;
            return 1;
        }
    }
    if (argc == 4 && std::string(argv[1]) == "--dump-image") {
        try {
            int W, H;
            std::vector<unsigned char> rgb = dcrf_io::load_bmp(argv[2], W, H);
            FILE* fp = fopen(argv[3], "wb");
            if (!fp) throw std::runtime_error(std::string("cannot write ") + argv[3]);
            fwrite(rgb.data(), 1, rgb.size(), fp);
            fclose(fp);
            std::cout << W << " " << H << std::endl;
            return 0;
        } catch (const std::exception& e) {
            std::cerr << "error: " << e.what() << std::endl;
            return 1;
        }
    }
    if (argc < 2) {
        std::cout << "Usage: ./example_inference method spc_std spc_potts bil_spcstd bil_colstd bil_potts [const_1 "
                     "const_2 const_3 norm_1 norm_2 norm_3]"
                  << '\n';
        std::cout << "Example: ./example_inference qp_sp [3 5 30 5 10 [10 1000]]" << '\n';
        return 1;
    }
    const std::string method = argv[1];
    const std::string image = env_or("DCRF_IMAGE", "../data/img.bmp");
    const std::string unaries = env_or("DCRF_UNARY", "../data/img.c_unary");
    const std::string output = env_or("DCRF_OUTPUT", "../data/seg.pgm");

    float spc_std = 2.0, spc_potts = 3.0, bil_potts = 2.0, bil_spcstd = 30.0, bil_colstd = 8.0;
    if (argc == 7) {
        spc_std = std::stof(argv[2]);
        spc_potts = std::stof(argv[3]);
        bil_spcstd = std::stof(argv[4]);
        bil_colstd = std::stof(argv[5]);
        bil_potts = std::stof(argv[6]);
    }
    sp_params params = {50, 1000};
    if (argc == 9) params = sp_params{std::stof(argv[7]), std::stof(argv[8])};

    LP_inf_params lp_params;
    lp_params.prox_energy_tol = lp_params.dual_gap_tol;
    try {
        image_inference(method, output, image, unaries, spc_std, spc_potts, bil_spcstd, bil_colstd, bil_potts,
                        lp_params, params);
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
