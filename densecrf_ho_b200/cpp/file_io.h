// Headless image / unary readers and a label-map writer for the example
// program, without OpenCV.
//
//  load_bmp      uncompressed 24- or 32-bit BMP (bottom-up or top-down rows,
//                BGR(A) pixels) -> uint8 RGB [H][W][3], the buffer
//                load_image builds from cv::imread (src/file_storage.cpp:
//                197-222).
//  load_unary    a ProbImage .c_unary file (the big-endian header W, H, D,
//                M, eps; M x D int32 keys; W x H key ids; values = key * eps,
//                external/ProbImage/probimage.cpp:140-165), then
//                boostToProb (:64-78) and -log per (pixel, label), as
//                load_unary does (src/file_storage.cpp:261-285); [N][D],
//                pixel = y * W + x.
//  save_labels   the arg-max labelling as a binary PGM (one byte per pixel,
//                the label index) -- the reference colours an image with a
//                dataset legend through OpenCV instead.
#pragma once
#include <arpa/inet.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace dcrf_io {

inline std::vector<unsigned char> read_file(const std::string& path) {
    FILE* fp = fopen(path.c_str(), "rb");
    if (!fp) throw std::runtime_error("cannot open " + path);
    std::vector<unsigned char> b;
    unsigned char buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), fp)) > 0) b.insert(b.end(), buf, buf + n);
    fclose(fp);
    return b;
}

inline uint32_t le32(const unsigned char* p) { return p[0] | (p[1] << 8) | (p[2] << 16) | ((uint32_t)p[3] << 24); }
inline uint16_t le16(const unsigned char* p) { return (uint16_t)(p[0] | (p[1] << 8)); }

inline std::vector<unsigned char> load_bmp(const std::string& path, int& W, int& H) {
    const std::vector<unsigned char> b = read_file(path);
    if (b.size() < 54 || b[0] != 'B' || b[1] != 'M') throw std::runtime_error(path + ": not a BMP file");
    const uint32_t data_off = le32(&b[10]);
    const int32_t w = (int32_t)le32(&b[18]), h = (int32_t)le32(&b[22]);
    const int bpp = le16(&b[28]);
    const uint32_t comp = le32(&b[30]);
    if ((bpp != 24 && bpp != 32) || (comp != 0 && comp != 3)) throw std::runtime_error(path + ": only 24/32-bit BMP");
    if (w <= 0 || h == 0) throw std::runtime_error(path + ": bad BMP size");
    W = w;
    H = h < 0 ? -h : h;
    const size_t row = ((size_t)w * (bpp / 8) + 3) & ~(size_t)3;
    if (data_off + row * H > b.size()) throw std::runtime_error(path + ": truncated BMP");
    std::vector<unsigned char> rgb((size_t)W * H * 3);
    for (int j = 0; j < H; j++) {
        const int src_row = h > 0 ? H - 1 - j : j;  // positive height: bottom-up rows
        const unsigned char* s = &b[data_off + row * src_row];
        for (int i = 0; i < W; i++) {
            const unsigned char* px = s + (size_t)i * (bpp / 8);
            unsigned char* d = &rgb[((size_t)j * W + i) * 3];
            d[0] = px[2];
            d[1] = px[1];
            d[2] = px[0];
        }
    }
    return rgb;
}

inline std::vector<float> load_unary(const std::string& path, int& W, int& H, int& D) {
    const std::vector<unsigned char> b = read_file(path);
    if (b.size() < 20) throw std::runtime_error(path + ": truncated .c_unary");
    auto be = [&](size_t i) {
        uint32_t v;
        std::memcpy(&v, &b[4 * i], 4);
        return ntohl(v);
    };
    W = (int)be(0);
    H = (int)be(1);
    D = (int)be(2);
    const uint32_t M = be(3), eps_bits = be(4);
    float eps;
    std::memcpy(&eps, &eps_bits, 4);
    const size_t N = (size_t)W * H;
    if (W <= 0 || H <= 0 || D <= 0 || b.size() < 4 * (5 + (size_t)M * D + N))
        throw std::runtime_error(path + ": truncated .c_unary");
    std::vector<float> data(N * D);
    for (size_t i = 0; i < N; i++) {
        const uint32_t id = be(5 + (size_t)M * D + i);
        if (id >= M) throw std::runtime_error(path + ": key id out of range");
        for (int j = 0; j < D; j++) data[i * D + j] = (int32_t)be(5 + (size_t)id * D + j) * eps;
    }
    for (size_t i = 0; i < N; i++) {  // boostToProb
        float* dp = &data[i * D];
        float mx = dp[0];
        for (int j = 1; j < D; j++)
            if (mx < dp[j]) mx = dp[j];
        float nm = 0;
        for (int j = 0; j < D; j++) nm += (dp[j] = exp((dp[j] - mx)));
        nm = 1.0 / nm;
        for (int j = 0; j < D; j++) dp[j] *= nm;
    }
    for (size_t i = 0; i < N * D; i++) data[i] = -log(data[i]);
    return data;
}

inline void save_labels(const std::string& path, const std::vector<short>& lab, int W, int H) {
    FILE* fp = fopen(path.c_str(), "wb");
    if (!fp) throw std::runtime_error("cannot write " + path);
    fprintf(fp, "P5\n%d %d\n255\n", W, H);
    std::vector<unsigned char> px(lab.size());
    for (size_t i = 0; i < lab.size(); i++) px[i] = (unsigned char)lab[i];
    fwrite(px.data(), 1, px.size(), fp);
    fclose(fp);
}

}  // namespace dcrf_io
