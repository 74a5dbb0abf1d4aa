/* Stand-in: cv::distanceTransform with the L1 metric, the one form the reference's depth-noise model
 * calls (staticDepthNoiseModeling.cpp:112): each pixel's exact L1 (4-step) distance to the nearest
 * zero pixel of an 8-bit mask, by a forward and a backward raster pass (with unit steps the
 * two-pass chamfer is exact for L1).  Pixels with no zero pixel in the image get a large value. */
#pragma once
#include <algorithm>
#include <opencv2/core/core.hpp>
#define CV_DIST_L1 1
#define CV_DIST_MASK_PRECISE 0
namespace cv {
inline void distanceTransform(const Mat_<uint8_t>& src, Mat& dst, int, int)
{
    const int H = src.rows, W = src.cols;
    const float big = 1e9f;
    dst.rows = H;
    dst.cols = W;
    dst.f.assign((std::size_t)H * W, big);
    auto at = [&](int i, int j) -> float& { return dst.f[(std::size_t)i * W + j]; };
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            float d = src(i, j) == 0 ? 0.f : big;
            if (i > 0) d = std::min(d, at(i - 1, j) + 1);
            if (j > 0) d = std::min(d, at(i, j - 1) + 1);
            at(i, j) = d;
        }
    for (int i = H - 1; i >= 0; i--)
        for (int j = W - 1; j >= 0; j--) {
            float d = at(i, j);
            if (i < H - 1) d = std::min(d, at(i + 1, j) + 1);
            if (j < W - 1) d = std::min(d, at(i, j + 1) + 1);
            at(i, j) = d;
        }
}
}  // namespace cv
