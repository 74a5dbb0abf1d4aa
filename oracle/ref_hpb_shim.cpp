/*
 * ref_hpb_shim.cpp — C entry point over the reference's OWN code for the depth pyramid its HPB
 * regularisation reads, compiled from its sources in place (see oracle/Makefile).  TEST
 * INFRASTRUCTURE ONLY: pins the oracle's depth_map_pyramid, never linked into the product.
 *
 * Reference code exercised (paths inside eherbst/rgbd-flow):
 *   DepthMapPyramid::ConstructPyramid       src/depthMapPyramid.cpp:15-91
 *   primesensor::stereoError / ErrorRatio   src/primesensorUtils.cpp:51-64
 * The glue below only moves buffers in and out of DImage.
 */
#include <cstring>

#include "celiu_flow/Image.h"
#include "celiu_flow/depthMapPyramid.h"

extern "C" int ref_depth_map_pyramid(const double* depth, int W, int H, double ratio, int minWidth, double* out,
                                     int* dims)
{
    DImage d(W, H, 1);
    std::memcpy(d.data(), depth, sizeof(double) * (size_t)W * H);
    DepthMapPyramid pyr;
    pyr.ConstructPyramid(d, ratio, minWidth);
    size_t off = 0;
    for (int i = 0; i < pyr.numLevels(); i++) {
        DImage& l = pyr.image(i);
        if (dims) { dims[2 * i] = l.width(); dims[2 * i + 1] = l.height(); }
        const size_t n = (size_t)l.width() * l.height();
        if (out) std::memcpy(out + off, l.data(), sizeof(double) * n);
        off += n;
    }
    return pyr.numLevels();
}
