/*
 * ref_rmf_shim.cpp — C entry point over the reference's OWN recursive median hole fill
 * (rgbd::recursiveMedianFilter -> recursiveMedianFilterAux, src/recursiveMedianFiltering.cpp:35-120),
 * compiled from its sources in place (see oracle/Makefile).  TEST INFRASTRUCTURE ONLY: pins the
 * oracle's median_fill, never linked into the product.  The glue only forwards the buffer.
 */
#include <cstdint>

namespace rgbd {
void recursiveMedianFilter(const uint32_t width, const uint32_t height, double* const data, const int32_t windowHalfwidth);
}

extern "C" void ref_median_fill(double* depth, int W, int H)
{
    rgbd::recursiveMedianFilter((uint32_t)W, (uint32_t)H, depth, 1);
}
