// Mean-shift superpixels (addSuperPixel's segmentation); see meanshift.cu.
#pragma once
#include <vector>

#include "common.cuh"

namespace dcrf {

// Step 2 alone: the mean-shift filtered L*u*v* colour of every pixel of the
// W x H image rgb (host, pixel-major RGB bytes) into filtered (host, W*H*3
// floats), EDISON's msRawData after Filter(spatial, range, NO_SPEEDUP).  The
// mode search runs on the current device on `stream`.
void meanshift_filter(const uint8_t* rgb, int W, int H, int spatial_radius, float range_radius, float* filtered,
                      cudaStream_t stream);
// Steps 3-5 on the host from a filtered image: the labels (host, W*H) and
// the region count.
int meanshift_regions(const float* filtered, int W, int H, float range_radius, int min_region, int* labels);
// Both: EDISON's Segment(spatial_radius, range_radius, min_region,
// NO_SPEEDUP) then GetRegions.
int meanshift_segment(const uint8_t* rgb, int W, int H, int spatial_radius, float range_radius, int min_region,
                      int* labels, cudaStream_t stream);

// The clique state addSuperPixel derives from a segmentation
// (src/densecrf.cpp:212-247) for regions numbered after `existing` earlier
// ones: per region its pixels in increasing order (offsets / idx), its
// weight constant * exp(-sd / (normaliser * count)) and `constant`.
void superpixel_cliques(const uint8_t* rgb, const int* labels, int N, int regions, int existing, float constant,
                        float normaliser, std::vector<int>& offsets, std::vector<int>& idx,
                        std::vector<float>& exp_weight, std::vector<float>& constants);

}  // namespace dcrf
