/*
 * ref_cuda_shim.cu — C entry point over the reference's OWN CUDA solver
 * (src/sceneFlowSingleScaleJacobiCUDA.cu:660-969, compiled unmodified for sm_100a from its
 * sources in place; see oracle/Makefile).  TEST INFRASTRUCTURE ONLY: it pins the oracle's
 * restatement of the solver on a GPU host and is never linked into the product.
 * The glue only wraps raw planes in DImages and calls sceneFlowSingleScale
 * (include/celiu_flow/OpticalFlow.h:17-22) with the argument order of sceneFlowMultiscale.cpp:177-182.
 */
#include <cstring>
#include "rgbd_util/CameraParams.h"
#include "celiu_flow/Image.h"

void sceneFlowSingleScale(const rgbd::CameraParams& camParams, const DImage& Im1, const DImage& dm1, const DImage& Im2,
                          const DImage& dm2, DImage& warpIm2, DImage& warpDm2, DImage& u, DImage& v, DImage& w,
                          const double colorDataTermWeight, const DImage& depthDataTermWeights, const double alpha,
                          const DImage& depthSmoothnessTermWeights, const double gamma, const DImage& depthMagTermWeights,
                          const DImage& regularizationWeights, int nOuterFPIterations, int nInnerFPIterations,
                          int nSORIterations, const bool allowEarlyTermination);

static DImage make(const double* p, int W, int H, int C)
{
    DImage im(W, H, C);
    std::memcpy(im.data(), p, sizeof(double) * (size_t)W * H * C);
    return im;
}

extern "C" int ref_single_scale(float f_level, const double* Im1, const double* dm1, const double* Im2, const double* dm2,
                                double* warpIm2, double* warpDm2, double* u, double* v, double* w, int W, int H, int C,
                                double colorW, const double* ddw, double alpha, const double* dsw, double gamma,
                                const double* mag, const double* regw, int nOuter, int nInner, int nSOR, int allowEarly)
{
    rgbd::CameraParams cam;
    std::memset(&cam, 0, sizeof(cam));
    cam.xRes = W; cam.yRes = H; cam.focalLength = f_level;
    DImage i1 = make(Im1, W, H, C), d1 = make(dm1, W, H, 1), i2 = make(Im2, W, H, C), d2 = make(dm2, W, H, 1);
    DImage wi = make(warpIm2, W, H, C), wd = make(warpDm2, W, H, 1);
    DImage uu = make(u, W, H, 1), vv = make(v, W, H, 1), ww = make(w, W, H, 1);
    DImage a = make(ddw, W, H, 1), b = make(dsw, W, H, 1), c = make(mag, W, H, 1), r = make(regw, W, H, 2);
    sceneFlowSingleScale(cam, i1, d1, i2, d2, wi, wd, uu, vv, ww, colorW, a, alpha, b, gamma, c, r, nOuter, nInner, nSOR,
                         allowEarly != 0);
    std::memcpy(u, uu.data(), sizeof(double) * W * H);
    std::memcpy(v, vv.data(), sizeof(double) * W * H);
    std::memcpy(w, ww.data(), sizeof(double) * W * H);
    return (int)cudaDeviceSynchronize();
}
