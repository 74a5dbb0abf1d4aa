/*
 * ref_cpu_shim.cpp — C entry points over the reference's OWN CPU image code, compiled from its
 * sources in place (see oracle/Makefile).  TEST INFRASTRUCTURE ONLY: used to pin the CPU
 * restatement in sforacle.cpp, never linked into the product.
 *
 * Reference code exercised (paths inside eherbst/rgbd-flow):
 *   GaussianPyramid::ConstructPyramid   src/GaussianPyramid.cpp:20-63
 *   Image::GaussianSmoothing            include/celiu_flow/Image.h:1179-1199
 *   Image::imresize(int,int)            include/celiu_flow/Image.h:764-770
 *   Image::desaturate, dx, dy           include/celiu_flow/Image.h:1438-1469, 955-1019
 *   ImageProcessing::warpImage          include/celiu_flow/ImageProcessing.h:472-491
 * The glue below only moves buffers in and out of DImage and sequences the calls exactly as
 * OpticalFlow::im2feature (src/OpticalFlow.cpp:189-214) and warpBy3DFlow
 * (src/opticalFlowUtils.cpp:76-89) do.
 */
#include <cstring>
#include "celiu_flow/Image.h"
#include "celiu_flow/ImageProcessing.h"
#include "celiu_flow/GaussianPyramid.h"

static DImage make(const double* p, int W, int H, int C)
{
    DImage im(W, H, C);
    std::memcpy(im.data(), p, sizeof(double) * (size_t)W * H * C);
    return im;
}

extern "C" {

int ref_build_pyramid(const double* img, int W, int H, int C, double ratio, int minWidth, double* out, int* dims)
{
    DImage base = make(img, W, H, C);
    GaussianPyramid pyr;
    pyr.ConstructPyramid(base, ratio, minWidth);
    size_t off = 0;
    for (int i = 0; i < pyr.numLevels(); i++) {
        DImage& l = pyr.image(i);
        if (dims) { dims[2 * i] = l.width(); dims[2 * i + 1] = l.height(); }
        const size_t n = (size_t)l.width() * l.height() * l.nchannels();
        if (out) std::memcpy(out + off, l.data(), sizeof(double) * n);
        off += n;
    }
    return pyr.numLevels();
}

void ref_gaussian_smooth(const double* img, int W, int H, int C, double sigma, int fsize, double* out)
{
    DImage a = make(img, W, H, C), b;
    a.GaussianSmoothing(b, sigma, fsize);
    std::memcpy(out, b.data(), sizeof(double) * (size_t)W * H * C);
}

void ref_resize_dims(const double* img, int W, int H, int C, int DW, int DH, double* out)
{
    DImage a = make(img, W, H, C);
    a.imresize(DW, DH);
    std::memcpy(out, a.data(), sizeof(double) * (size_t)DW * DH * C);
}

void ref_im2feature(const double* bgr01, int W, int H, double* feat5)
{
    DImage im = make(bgr01, W, H, 3), gray;
    im.desaturate(gray);
    DImage imdx(W, H), imdy(W, H);
    gray.dx(imdx, true);
    gray.dy(imdy, true);
    for (int o = 0; o < W * H; o++) {
        feat5[o * 5 + 0] = gray.data()[o];
        feat5[o * 5 + 1] = imdx.data()[o];
        feat5[o * 5 + 2] = imdy.data()[o];
        feat5[o * 5 + 3] = im.data()[o * 3 + 1] - im.data()[o * 3];
        feat5[o * 5 + 4] = im.data()[o * 3 + 1] - im.data()[o * 3 + 2];
    }
}

void ref_warp(const double* feat1, const double* d1, const double* feat2, const double* d2, int W, int H, int C,
              const double* u, const double* v, const double* w, double* wI2, double* wD2)
{
    ImageProcessing::warpImage(wI2, feat1, feat2, u, v, W, H, C);
    ImageProcessing::warpImage(wD2, d1, d2, u, v, W, H, 1);
    for (int l = 0; l < W * H; l++) wD2[l] -= w[l];
}

} // extern "C"
