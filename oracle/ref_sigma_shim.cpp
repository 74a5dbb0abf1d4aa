/*
 * ref_sigma_shim.cpp — C entry point over the reference's OWN depth-noise model
 * (computeDepthMapStdevsPointwise + increaseStdevsNearDepthBoundaries,
 * src/staticDepthNoiseModeling.cpp:85-137, 225-258), compiled from its sources in place with its
 * thread pool (see oracle/Makefile).  TEST INFRASTRUCTURE ONLY: pins the oracle's depth_sigma, never
 * linked into the product.  The L1 distance transform the reference takes from OpenCV is the
 * stand-in of ref_stubs_sigma/opencv2/imgproc/imgproc.hpp; everything else is the reference's code.
 * The glue below only moves buffers in and out, as setUpSceneFlowParams does
 * (src/runFlowTwoFrames.cpp:90-98).
 */
#include <cstdint>
#include <cstring>

#include "rgbd_frame_common/staticDepthNoiseModeling.h"

extern "C" void ref_depth_sigma(const float* depth, int W, int H, int max_dist, float* out)
{
    cv::Mat_<float> d(H, W);
    std::memcpy(d.d.data(), depth, sizeof(float) * (size_t)W * H);
    boost::multi_array<float, 2> stdevs;
    computeDepthMapStdevsPointwise(d, stdevs, (uint32_t)max_dist, false);
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) out[(size_t)i * W + j] = stdevs[i][j];
}
