/*
 * ref_flow2d_shim.cpp — C entry point over the reference's OWN 2-D optical-flow code (Ce Liu's
 * coarse-to-fine solver, the demo's flow type 1), compiled from its sources in place (see
 * oracle/Makefile).  TEST INFRASTRUCTURE ONLY: used to pin the oracle's 2-D restatement
 * (oracle/flow2d.cpp), never linked into the product.
 *
 * Reference code exercised (paths inside eherbst/rgbd-flow):
 *   OpticalFlow::Coarse2FineFlow          src/opticalFlowMultiscale.cpp (included below)
 *   OpticalFlow::SmoothFlowSOR            src/SmoothFlowSOR.cpp (included below)
 *   OpticalFlow::SmoothFlowSORNonrobust   src/SmoothFlowSORNonrobust.cpp (included below)
 *   getDxs, Laplacian, warpFL, estLaplacianNoise   src/opticalFlowUtils.cpp (compiled beside)
 *   GaussianPyramid, Image, ImageProcessing        src/GaussianPyramid.cpp, include/celiu_flow/
 * src/OpticalFlow.cpp, which holds im2feature and OpticalFlow's static members, cannot be
 * compiled here: it includes the scene-flow sources, which need Eigen, PCL and OpenCV.  The glue
 * below stands in for the parts of it this path uses:
 *   - the static members, with the values OpticalFlow.cpp:22-26 gives them, except IsDisplay
 *     (progress printing only) which is off;
 *   - im2feature for a 3-channel image and RGB_WITH_GRADIENT, calling the reference's own
 *     Image methods in the order OpticalFlow.cpp:189-214 calls them (as ref_im2feature in
 *     ref_cpu_shim.cpp does); every other case raises, as the reference's ASSERT_ALWAYS(false)
 *     does;
 *   - im2featureWithDepth and recursiveMedianFilter, reached only when depth maps are given
 *     (never on this path), raise.
 */
#include <cstring>
#include <iostream>
#include <sstream>
#include <stdexcept>

#include "celiu_flow/GaussianPyramid.h"
#include "celiu_flow/Image.h"
#include "celiu_flow/ImageProcessing.h"
#include "celiu_flow/OpticalFlow.h"
#include "celiu_flow/opticalFlowUtils.h"
#include "celiu_flow/recursiveMedianFiltering.h"
#include "rgbd_util/assert.h"

using std::cout;
using std::endl;
using namespace scene_flow;  // as src/OpticalFlow.cpp:16 does for the sources it includes

bool OpticalFlow::IsDisplay = false;
OpticalFlow::InterpolationMethod OpticalFlow::interpolation = OpticalFlow::Bilinear;
OpticalFlow::NoiseModel OpticalFlow::noiseModel = OpticalFlow::Lap;
GaussianMixture OpticalFlow::GMPara;
Vector<double> OpticalFlow::LapPara;

void OpticalFlow::im2feature(DImage& imfeature, const DImage& im, const constancyType c)
{
    const int W = im.width(), H = im.height();
    if (im.nchannels() != 3 || c != constancyType::RGB_WITH_GRADIENT)
        throw std::runtime_error("im2feature: only the 3-channel RGB_WITH_GRADIENT form is on this path");
    DImage gray;
    im.desaturate(gray);
    imfeature.allocate(W, H, 5);
    DImage imdx(W, H), imdy(W, H);
    gray.dx(imdx, true);
    gray.dy(imdy, true);
    double* f = imfeature.data();
    for (int o = 0; o < W * H; o++) {
        f[o * 5 + 0] = gray.data()[o];
        f[o * 5 + 1] = imdx.data()[o];
        f[o * 5 + 2] = imdy.data()[o];
        f[o * 5 + 3] = im.data()[o * 3 + 1] - im.data()[o * 3];
        f[o * 5 + 4] = im.data()[o * 3 + 1] - im.data()[o * 3 + 2];
    }
}

void OpticalFlow::im2featureWithDepth(DImage&, const DImage&, const DImage&)
{
    throw std::runtime_error("im2featureWithDepth is not on this path");
}

void recursiveMedianFilter(DImage&, const int32_t)
{
    throw std::runtime_error("recursiveMedianFilter is not on this path");
}

#include "SmoothFlowSOR.cpp"
#include "SmoothFlowSORNonrobust.cpp"
#include "opticalFlowMultiscale.cpp"

extern "C" {

/* Coarse2FineFlow on two BGR images in [0, 1] (interleaved doubles, as cv2liuBGR makes them,
 * src/ceLiuOpticalFlow.cpp:19-37) with the given parameters; u, v: W*H doubles each.  The
 * solver's per-iteration progress lines (SmoothFlowSOR.cpp:222) go to a discarded stream.
 * Returns 0, or -1 with the reference's message in err when it raises. */
int ref_coarse2fine_flow(const double* bgr1, const double* bgr2, int W, int H, int variant, double alpha,
                         double ratio, int min_width, int n_outer, int n_inner, int n_sor, double* u, double* v,
                         char* err, int err_len)
{
    std::ostringstream sink;
    std::streambuf* old = std::cout.rdbuf(sink.rdbuf());
    try {
        DImage Im1(W, H, 3), Im2(W, H, 3), vx, vy, warpI2;
        std::memcpy(Im1.data(), bgr1, sizeof(double) * (size_t)W * H * 3);
        std::memcpy(Im2.data(), bgr2, sizeof(double) * (size_t)W * H * 3);
        OpticalFlow::opticalFlowParams p;
        p.variant = variant ? OpticalFlow::opticalFlowVariant::CELIU_NONROBUST : OpticalFlow::opticalFlowVariant::CELIU;
        p.alpha = alpha;
        p.pyramidRatio = ratio;
        p.minWidth = min_width;
        p.nOuterFPIterations = n_outer;
        p.nInnerFPIterations = n_inner;
        p.nSORIterations = n_sor;
        OpticalFlow::Coarse2FineFlow(vx, vy, warpI2, Im1, Im2, p);
        std::memcpy(u, vx.data(), sizeof(double) * (size_t)W * H);
        std::memcpy(v, vy.data(), sizeof(double) * (size_t)W * H);
    } catch (const std::exception& e) {
        std::cout.rdbuf(old);
        if (err && err_len > 0) {
            std::strncpy(err, e.what(), err_len - 1);
            err[err_len - 1] = 0;
        }
        return -1;
    }
    std::cout.rdbuf(old);
    return 0;
}

}  // extern "C"
