/*
 * sforacle.cpp — CPU restatement of rgbd-flow's coarse-to-fine RGB-D scene-flow solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the smoke check
 * and the CPU-baseline leg of the benchmark call it; the product library never links it.
 *
 * Two arithmetic variants share one code path (template parameter FP64):
 *   FP64 = false  "faithful": the reference's own mix of FP64 images/flow and FP32 weights,
 *                 system matrix, increments and squares (sqrCU takes and returns float), with
 *                 the same red-black order, relaxation, step clamp and convergence schedule.
 *   FP64 = true   every FP32 quantity of the reference widened to FP64 (the EPE reference).
 *
 * The reference has no CPU version of its 3-D solver (it exists only as CUDA in
 * src/sceneFlowSingleScaleJacobiCUDA.cu), so the solver below restates that CUDA's arithmetic
 * on the CPU; everything around it restates the reference's own CPU code.  Citations are
 * paths inside eherbst/rgbd-flow.
 *
 * Parity pins: the pyramid / resize / filter / feature / warp restatements are compared with
 * the reference's own header code compiled from its sources (oracle/_ref, see Makefile), and
 * the single-scale solver with the reference's CUDA solver run on the device.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <set>
#include <string>
#include <unordered_set>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/rgbdflow.h"
#include "sforacle.h"

namespace sfo {

static inline double sqr(double x) { return x * x; }

/* A Ce Liu DImage: interleaved FP64, zero-initialised (include/celiu_flow/Image.h:505-520). */
struct Img {
    int w = 0, h = 0, c = 0;
    std::vector<double> d;
    void alloc(int W, int H, int C) { w = W; h = H; c = C; d.assign((size_t)W * H * C, 0.0); }
    double* data() { return d.data(); }
    const double* data() const { return d.data(); }
    size_t n() const { return d.size(); }
};

/* ImageProcessing::EnforceRange (include/celiu_flow/ImageProcessing.h:25) */
static inline int enforce_range(int x, int n) { return std::min(std::max(x, 0), n - 1); }

/* ImageProcessing::BilinearInterpolate, multi-channel accumulate form (ImageProcessing.h:128-148).
 * xx = (int)x truncates toward zero; the fractional part is clamped to [0,1]. */
static void bilinear_acc(const double* img, int W, int H, int C, double x, double y, double* out)
{
    const int xx = (int)x, yy = (int)y;
    double dx = x - xx; if (dx > 1) dx = 1; if (dx < 0) dx = 0;
    double dy = y - yy; if (dy > 1) dy = 1; if (dy < 0) dy = 0;
    for (int m = 0; m <= 1; m++)
        for (int n = 0; n <= 1; n++) {
            const int u = enforce_range(xx + m, W);
            const int v = enforce_range(yy + n, H);
            const size_t off = ((size_t)v * W + u) * C;
            const double s = std::fabs(1 - m - dx) * std::fabs(1 - n - dy);
            for (int l = 0; l < C; l++) out[l] += img[off + l] * s;
        }
}

/* ImageProcessing::hfiltering / vfiltering, clamp-to-edge (ImageProcessing.h:247-269, 339-358). */
static void hfilter(const Img& in, Img& out, const double* f, int fs)
{
    out.alloc(in.w, in.h, in.c);
    const int W = in.w, C = in.c;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < in.h; i++)
        for (int j = 0; j < W; j++) {
            double* o = out.data() + ((size_t)i * W + j) * C;
            for (int l = -fs; l <= fs; l++) {
                const double wgt = f[l + fs];
                const int jj = enforce_range(j + l, W);
                const double* s = in.data() + ((size_t)i * W + jj) * C;
                for (int k = 0; k < C; k++) o[k] += s[k] * wgt;
            }
        }
}
static void vfilter(const Img& in, Img& out, const double* f, int fs)
{
    out.alloc(in.w, in.h, in.c);
    const int W = in.w, H = in.h, C = in.c;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            double* o = out.data() + ((size_t)i * W + j) * C;
            for (int l = -fs; l <= fs; l++) {
                const double wgt = f[l + fs];
                const int ii = enforce_range(i + l, H);
                const double* s = in.data() + ((size_t)ii * W + j) * C;
                for (int k = 0; k < C; k++) o[k] += s[k] * wgt;
            }
        }
}

/* Image::GaussianSmoothing (Image.h:1179-1199): normalised exp(-i^2 / 2 sigma^2), separable. */
void gaussian_smooth(const Img& in, Img& out, double sigma, int fsize)
{
    std::vector<double> g(2 * fsize + 1);
    double sum = 0;
    const double s2 = sigma * sigma * 2;
    for (int i = -fsize; i <= fsize; i++) {
        g[i + fsize] = std::exp(-(double)(i * i) / s2);
        sum += g[i + fsize];
    }
    for (int i = 0; i < 2 * fsize + 1; i++) g[i] /= sum;
    Img tmp;
    hfilter(in, tmp, g.data(), fsize);
    vfilter(tmp, out, g.data(), fsize);
}

/* ImageProcessing::ResizeImage by ratio (ImageProcessing.h:203-222; Image.h:739-751). */
void resize_ratio(const Img& in, Img& out, double ratio)
{
    const int DW = (int)((double)in.w * ratio), DH = (int)((double)in.h * ratio);
    out.alloc(DW, DH, in.c);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < DH; i++)
        for (int j = 0; j < DW; j++) {
            const double x = (double)(j + 1) / ratio - 1;
            const double y = (double)(i + 1) / ratio - 1;
            bilinear_acc(in.data(), in.w, in.h, in.c, x, y, out.data() + ((size_t)i * DW + j) * in.c);
        }
}

/* ImageProcessing::ResizeImage to explicit dims (ImageProcessing.h:225-242; Image.h:764-770). */
void resize_dims(const Img& in, Img& out, int DW, int DH)
{
    const double xr = (double)DW / in.w, yr = (double)DH / in.h;
    Img o; o.alloc(DW, DH, in.c);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < DH; i++)
        for (int j = 0; j < DW; j++) {
            const double x = (double)(j + 1) / xr - 1;
            const double y = (double)(i + 1) / yr - 1;
            bilinear_acc(in.data(), in.w, in.h, in.c, x, y, o.data() + ((size_t)i * DW + j) * in.c);
        }
    out = std::move(o);
}

/* GaussianPyramid::ConstructPyramid level count (GaussianPyramid.cpp:22-32). */
int pyramid_levels(int width, double ratio, int min_width)
{
    if (min_width < 0) min_width = std::max(1, width / -min_width);  // API convention: W / d per pair
    if (min_width == 0) throw std::runtime_error("min_width 0: the level count never ends");
    if (ratio > 0.98 || ratio < 0.4) ratio = 0.75;
    double w = width * ratio;
    int n = 1;
    while (w >= min_width) { n++; w *= ratio; }
    return n;
}

/* GaussianPyramid::ConstructPyramid (GaussianPyramid.cpp:20-63). */
void build_pyramid(const Img& image, double ratio, int min_width, std::vector<Img>& lev)
{
    if (min_width < 0) min_width = std::max(1, image.w / -min_width);
    if (ratio > 0.98 || ratio < 0.4) ratio = 0.75;
    const int nLevels = pyramid_levels(image.w, ratio, min_width);
    lev.assign(nLevels, Img());
    lev[0] = image;
    const double baseSigma = (1 / ratio - 1);
    const int n = (int)(std::log(0.25) / std::log(ratio));
    const double nSigma = baseSigma * n;
    for (int i = 1; i < nLevels; i++) {
        Img foo;
        if (i <= n) {
            const double sigma = baseSigma * i;
            gaussian_smooth(image, foo, sigma, (int)(sigma * 3));
            resize_ratio(foo, lev[i], std::pow(ratio, i));
        } else {
            gaussian_smooth(lev[i - n], foo, nSigma, (int)(nSigma * 3));
            const double rate = (double)std::pow(ratio, i) * image.w / foo.w;
            resize_ratio(foo, lev[i], rate);
        }
    }
}

/* OpticalFlow::im2feature RGB_WITH_GRADIENT (OpticalFlow.cpp:189-214) with Image::desaturate
 * (Image.h:1438-1469) and the 5-tap {1,-8,0,8,-1}/12 Image::dx/dy (Image.h:955-1019). */
void im2feature(const Img& im, Img& feat)
{
    const int W = im.w, H = im.h;
    Img gray; gray.alloc(W, H, 1);
    for (size_t i = 0; i < (size_t)W * H; i++) {
        const size_t o = i * 3;
        gray.d[i] = (double)im.d[o] * .114 + im.d[o + 1] * .587 + im.d[o + 2] * .299;
    }
    double f[5] = {1, -8, 0, 8, -1};
    for (int i = 0; i < 5; i++) f[i] /= 12;
    Img gx, gy;
    hfilter(gray, gx, f, 2);
    vfilter(gray, gy, f, 2);
    feat.alloc(W, H, 5);
    for (size_t o = 0; o < (size_t)W * H; o++) {
        feat.d[o * 5 + 0] = gray.d[o];
        feat.d[o * 5 + 1] = gx.d[o];
        feat.d[o * 5 + 2] = gy.d[o];
        feat.d[o * 5 + 3] = im.d[o * 3 + 1] - im.d[o * 3];
        feat.d[o * 5 + 4] = im.d[o * 3 + 1] - im.d[o * 3 + 2];
    }
}

/* rgbd::recursiveMedianFilterAux (src/recursiveMedianFiltering.cpp:35-99), window half-width 1.
 * Reproduces the reference's order exactly: the same std::unordered_set<uint32_t> insert /
 * erase sequence, so libstdc++ iteration order picks the same next point among equals. */
void median_fill(double* data, int width, int height, int hw)
{
    const int win = (2 * hw + 1) * (2 * hw + 1);
    std::vector<std::unordered_set<uint32_t>> byCount(win);
    std::vector<int32_t> cnt((size_t)width * height, -1);
    uint32_t left = 0;
    for (int32_t i = 0, l = 0; i < height; i++)
        for (int32_t j = 0; j < width; j++, l++)
            if (data[l] <= 0) {
                uint32_t k = 0;
                for (int32_t ii = std::max(0, i - hw); ii <= std::min(height - 1, i + hw); ii++)
                    for (int32_t jj = std::max(0, j - hw); jj <= std::min(width - 1, j + hw); jj++)
                        if (data[ii * width + jj] > 0) k++;
                byCount[k].insert(l);
                cnt[l] = k;
                left++;
            }
    std::vector<float> vals(win);
    while (left > 0) {
        int32_t mx = (int32_t)byCount.size() - 1;
        while (mx >= 0 && byCount[mx].empty()) mx--;
        if (mx <= 0) throw std::runtime_error("median_fill: a hole has no valid neighbour");
        const uint32_t l = *byCount[mx].begin();
        const int32_t i = l / width, j = l % width;
        byCount[mx].erase(l);
        cnt[l] = -1;
        uint32_t idx = 0;
        for (int32_t ii = std::max(0, i - hw); ii <= std::min(height - 1, i + hw); ii++)
            for (int32_t jj = std::max(0, j - hw); jj <= std::min(width - 1, j + hw); jj++) {
                const int32_t ll = ii * width + jj;
                if (data[ll] > 0) {
                    vals[idx++] = (float)data[ll];
                } else if (cnt[ll] >= 0) {
                    byCount[cnt[ll]].erase(ll);
                    cnt[ll]++;
                    byCount[cnt[ll]].insert(ll);
                }
            }
        std::sort(vals.begin(), vals.begin() + idx);
        data[l] = vals[(int)std::floor(idx / 2)];
        left--;
    }
}

/* The same fill in the device's order (window half-width 1): rounds r = 1, 2, ...  In round r every
 * hole whose count of known 8-neighbours (valid, or filled in an earlier round) is > 0 and is not
 * smaller than the count of any unfilled 8-neighbour takes the median of its known neighbours, read
 * as they were at the start of the round.  Each value still is the median of the 3x3 known values
 * (recursiveMedianFiltering.cpp:67-94); only the order, among holes that touch, differs from the
 * reference's hash-set order.  Isolated holes get the reference's value.  This restates the
 * library's schedule so that the parity tests can separate the fill order (measured on its own)
 * from the arithmetic of the rest of the solve.  Returns the number of rounds. */
int median_fill_rounds(double* data, int width, int height)
{
    const size_t N = (size_t)width * height;
    std::vector<int> stamp(N);  // 0 valid, -1 unfilled, r filled in round r
    size_t left = 0;
    for (size_t l = 0; l < N; l++) {
        stamp[l] = data[l] > 0 ? 0 : -1;
        if (stamp[l] < 0) left++;
    }
    int r = 0;
    std::vector<int> fill_l;
    std::vector<double> fill_v;
    while (left > 0) {
        r++;
        auto known = [&](int i, int j) {
            return i >= 0 && j >= 0 && i < height && j < width && stamp[(size_t)i * width + j] >= 0 &&
                   stamp[(size_t)i * width + j] < r;
        };
        auto count = [&](int i, int j) {
            int k = 0;
            for (int a = -1; a <= 1; a++)
                for (int b = -1; b <= 1; b++)
                    if ((a | b) && known(i + a, j + b)) k++;
            return k;
        };
        fill_l.clear();
        fill_v.clear();
        for (int i = 0; i < height; i++)
            for (int j = 0; j < width; j++) {
                if (stamp[(size_t)i * width + j] != -1) continue;
                const int c = count(i, j);
                bool fill = c > 0;
                for (int a = -1; a <= 1 && fill; a++)
                    for (int b = -1; b <= 1 && fill; b++) {
                        const int ii = i + a, jj = j + b;
                        if (!(a | b) || ii < 0 || jj < 0 || ii >= height || jj >= width) continue;
                        if (stamp[(size_t)ii * width + jj] == -1 && count(ii, jj) > c) fill = false;
                    }
                if (!fill) continue;
                float vals[8];
                int n = 0;
                for (int a = -1; a <= 1; a++)
                    for (int b = -1; b <= 1; b++)
                        if ((a | b) && known(i + a, j + b)) {
                            const float x = (float)data[(size_t)(i + a) * width + (j + b)];
                            int k = n++;
                            while (k > 0 && vals[k - 1] > x) { vals[k] = vals[k - 1]; k--; }
                            vals[k] = x;
                        }
                fill_l.push_back(i * width + j);
                fill_v.push_back(vals[n / 2]);
            }
        if (fill_l.empty()) throw std::runtime_error("median_fill_rounds: a hole region has no valid neighbour");
        for (size_t q = 0; q < fill_l.size(); q++) {
            data[fill_l[q]] = fill_v[q];
            stamp[fill_l[q]] = r;
        }
        left -= fill_l.size();
    }
    return r;
}

/* Fill order of the scene-flow solve's hole fill: 0 the reference's (median_fill), 1 the device's
 * rounds (median_fill_rounds).  Set by sfo_set_fill_order. */
static int g_fill_order = 0;
static void fill_depth(double* data, int width, int height)
{
    if (g_fill_order == 1) median_fill_rounds(data, width, height);
    else median_fill(data, width, height, 1);
}

/* primesensor::stereoError / stereoErrorRatio (src/primesensorUtils.cpp:53-64). */
double stereo_error(double z) { return sqr(z) / (1 / .00285 + z); }
double stereo_error_ratio(double z) { return stereo_error(z) / stereo_error(1); }

/* computeDepthMapStdevsPointwise + increaseStdevsNearDepthBoundaries
 * (src/staticDepthNoiseModeling.cpp:232-258, 85-137).  cv::distanceTransform(CV_DIST_L1) is the
 * exact L1 distance to the nearest boundary-mask zero; only distances <= maxDist matter, so the
 * diamond of radius maxDist is searched directly. */
void depth_sigma(const float* depth, int W, int H, int maxDist, float* sig)
{
    const float sigmaAt1m = (float)stereo_error(1);
    for (int l = 0; l < W * H; l++) {
        const float z = depth[l];
        sig[l] = (z > 0) ? (float)std::max(1e-4, (double)sigmaAt1m * stereo_error_ratio(z)) : 1.0f;
    }
    if (maxDist <= 0) return;
    std::vector<uint8_t> boundary((size_t)W * H, 0);
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            const float z = depth[i * W + j];
            bool b = false;
            if (i < H - 1 && depth[(i + 1) * W + j] > 0 &&
                std::fabs((double)(z - depth[(i + 1) * W + j])) > .02 * stereo_error_ratio(std::min(z, depth[(i + 1) * W + j])))
                b = true;
            else if (j < W - 1 && depth[i * W + j + 1] > 0 &&
                     std::fabs((double)(z - depth[i * W + j + 1])) > .02 * stereo_error_ratio(std::min(z, depth[i * W + j + 1])))
                b = true;
            boundary[i * W + j] = b;
        }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            int best = maxDist + 1;
            for (int di = -maxDist; di <= maxDist && best > 0; di++) {
                const int ii = i + di;
                if (ii < 0 || ii >= H) continue;
                const int rem = maxDist - std::abs(di);
                for (int dj = -rem; dj <= rem; dj++) {
                    const int jj = j + dj;
                    if (jj < 0 || jj >= W) continue;
                    if (boundary[ii * W + jj]) {
                        const int d = std::abs(di) + std::abs(dj);
                        if (d < best) best = d;
                    }
                }
            }
            if (best <= maxDist) {
                const float a = (float)best / (float)maxDist;
                const float s = sig[i * W + j];
                sig[i * W + j] = (float)std::exp((1 - a) * std::log((double)(10 * s)) + a * std::log((double)s));
            }
        }
}

/* ImageProcessing::warpImage + the depth correction of warpBy3DFlow
 * (src/opticalFlowUtils.cpp:76-99; ImageProcessing.h:472-491). */
void warp_cpu(const Img& Im1, const Img& dm1, const Img& Im2, const Img& dm2, Img& wI2, Img& wD2,
              const double* vx, const double* vy, const double* vz)
{
    const int W = Im2.w, H = Im2.h, C = Im2.c;
    wI2.alloc(W, H, C);
    wD2.alloc(W, H, 1);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            const int o = i * W + j;
            const double y = i + vy[o], x = j + vx[o];
            if (x < 0 || x > W - 1 || y < 0 || y > H - 1) {
                for (int k = 0; k < C; k++) wI2.d[(size_t)o * C + k] = Im1.d[(size_t)o * C + k];
                wD2.d[o] = dm1.d[o];
            } else {
                bilinear_acc(Im2.data(), W, H, C, x, y, wI2.data() + (size_t)o * C);
                bilinear_acc(dm2.data(), W, H, 1, x, y, wD2.data() + o);
            }
            wD2.d[o] -= vz[o];
        }
}

/* getResizedCamParams / getDownsizedCamParams (runFlowTwoFrames.cpp:14-24, sceneFlowMultiscale.cpp:16-27). */
rgbdflow_camera_params resize_cam(rgbdflow_camera_params c, int width)
{
    const double f = (double)width / c.xRes;
    c.xRes = (unsigned)std::rint(c.xRes * f);
    c.yRes = (unsigned)std::rint(c.yRes * f);
    c.centerX = (float)std::rint(c.centerX * f);
    c.centerY = (float)std::rint(c.centerY * f);
    c.focalLength = (float)(c.focalLength * f);
    return c;
}

/* ------------------------------------------------------------------------------------------ */
/* single-scale solver: restates sceneFlowSingleScale (src/sceneFlowSingleScaleJacobiCUDA.cu:660-969) */

template <bool FP64> struct P;
template <> struct P<false> { typedef float F; };
template <> struct P<true> { typedef double F; };

/* sqrCU (.cu:44-47): takes and returns float in the reference. */
template <bool FP64> static inline typename P<FP64>::F sqc(double x)
{
    typedef typename P<FP64>::F F;
    const F f = (F)x;
    return f * f;
}

struct SolverIn {
    int W, H, C;
    float f_level;                         /* level focal length (float, as CameraParams) */
    const double *Im1, *dm1, *Im2, *dm2;  /* W*H*C, W*H */
    double colorW, alpha, gamma;
    const double *ddw, *dsw, *mag, *regw; /* W*H, W*H, W*H, W*H*2 */
    int nOuter, nInner, nSOR, allowEarly;
};

template <bool FP64>
static void sor_sweep(int W, int H, const std::vector<typename P<FP64>::F>& A, std::vector<typename P<FP64>::F>& x,
                      int color, typename P<FP64>::F omega, typename P<FP64>::F step)
{
    typedef typename P<FP64>::F F;
    const size_t nz = (size_t)W * H * 3;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < H; i++)
        for (int j = (i + color) & 1; j < W; j += 2) {
            const size_t l = (size_t)i * W + j;
            const F xp[3] = {x[l * 3 + 0], x[l * 3 + 1], x[l * 3 + 2]};
            F nv[3];
            for (int k = 0; k < 3; k++) {
                const size_t p = l * 3 + k;
                F v = 0;
                if (j > 0) v -= A[0 * nz + p] * x[(l - 1) * 3 + k];
                if (i > 0) v -= A[1 * nz + p] * x[(l - W) * 3 + k];
                if (j < W - 1) v -= A[2 * nz + p] * x[(l + 1) * 3 + k];
                if (i < H - 1) v -= A[3 * nz + p] * x[(l + W) * 3 + k];
                v += A[7 * nz + p];
                switch (k) {
                case 0: v -= A[5 * nz + p] * xp[1]; v -= A[6 * nz + p] * xp[2]; v /= A[4 * nz + p]; break;
                case 1: v -= A[4 * nz + p] * xp[0]; v -= A[6 * nz + p] * xp[2]; v /= A[5 * nz + p]; break;
                default: v -= A[4 * nz + p] * xp[0]; v -= A[5 * nz + p] * xp[1]; v /= A[6 * nz + p]; break;
                }
                F r = omega * v + ((F)1 - omega) * xp[k];
                if (r < xp[k] - step) r = xp[k] - step;
                else if (r > xp[k] + step) r = xp[k] + step;
                nv[k] = r;
            }
            x[l * 3 + 0] = nv[0];
            x[l * 3 + 1] = nv[1];
            x[l * 3 + 2] = nv[2];
        }
}

/* Builds the 8-plane system of fillSystemMtxKernel (.cu:477-575) from the current state.
 * Exposed separately so tests can compare one linearisation coefficient by coefficient. */
template <bool FP64>
static void linearize(const SolverIn& in, const rgbdflow_params& p, const std::vector<double>& u3,
                      const std::vector<typename P<FP64>::F>& du, const Img& wI2, const Img& wD2,
                      const std::vector<typename P<FP64>::F>& q,
                      const std::vector<typename P<FP64>::F>& ddwF, const std::vector<typename P<FP64>::F>& dswF,
                      const std::vector<typename P<FP64>::F>& magF, const std::vector<typename P<FP64>::F>& regF,
                      const std::vector<double>& imdx, const std::vector<double>& imdy, const std::vector<double>& imdt,
                      const std::vector<double>& dmdx, const std::vector<double>& dmdy, const std::vector<double>& dmdt,
                      std::vector<typename P<FP64>::F>& A)
{
    typedef typename P<FP64>::F F;
    const int W = in.W, H = in.H, C = in.C;
    const size_t N = (size_t)W * H, nz = N * 3;
    std::vector<double> ux(N), uy(N), vx(N), vy(N), wx(N), wy(N);
    /* flowDerivativesKernel (.cu:156-182): forward differences of u + du */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            const size_t l = (size_t)i * W + j;
            double* ox[3] = {&ux[l], &vx[l], &wx[l]};
            double* oy[3] = {&uy[l], &vy[l], &wy[l]};
            for (int c = 0; c < 3; c++) {
                const size_t p3 = l * 3 + c;
                *oy[c] = (i == H - 1) ? 0 : u3[p3 + W * 3] + du[p3 + W * 3] - u3[p3] - du[p3];
                *ox[c] = (j == W - 1) ? 0 : u3[p3 + 3] + du[p3 + 3] - u3[p3] - du[p3];
            }
        }
    /* penaltyDerivativesKernel (.cu:340-371) */
    std::vector<double> phi(N), pi(N), psi(N * C);
#pragma omp parallel for schedule(static)
    for (int l = 0; l < (int)N; l++) {
        const F t = sqc<FP64>(ux[l]) + sqc<FP64>(uy[l]) + sqc<FP64>(vx[l]) + sqc<FP64>(vy[l]) +
                    dswF[l] * (sqc<FP64>(wx[l]) + sqc<FP64>(wy[l]));
        phi[l] = 0.5 / std::sqrt((double)t + p.eps_s);
        for (int k = 0; k < C; k++) {
            const size_t o = (size_t)l * C + k;
            const double t1 = (imdt[o] + imdx[o] * du[l * 3 + 0] + imdy[o] * du[l * 3 + 1]) * q[l];
            psi[o] = .5 / std::sqrt((double)sqc<FP64>(t1) + p.eps_d) * in.colorW;
        }
        const double t2 = dmdt[l] + dmdx[l] * du[l * 3 + 0] + dmdy[l] * du[l * 3 + 1] - du[l * 3 + 2];
        pi[l] = .5 / std::sqrt((double)sqc<FP64>(t2) + p.eps_z) * ddwF[l];
    }
    /* product kernels (.cu:189-230), Laplacians (.cu:240-333), fillSystemMtxKernel (.cu:477-575) */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            const size_t l = (size_t)i * W + j;
            double sxy = 0, sx2 = 0, sy2 = 0, stx = 0, sty = 0;
            for (int k = 0; k < C; k++) {
                const size_t o = l * C + k;
                sxy += psi[o] * imdx[o] * imdy[o];
                sx2 += psi[o] * imdx[o] * imdx[o];
                sy2 += psi[o] * imdy[o] * imdy[o];
                stx += psi[o] * imdx[o] * imdt[o];
                sty += psi[o] * imdy[o] * imdt[o];
            }
            const double ixy = sxy / C, ix2 = sx2 / C, iy2 = sy2 / C;
            const double itx = stx * q[l] * q[l] / C, ity = sty * q[l] * q[l] / C;
            const double dxy = pi[l] * dmdx[l] * dmdy[l], dx2 = pi[l] * dmdx[l] * dmdx[l], dy2 = pi[l] * dmdy[l] * dmdy[l];
            const double dtx = pi[l] * dmdx[l] * dmdt[l], dty = pi[l] * dmdy[l] * dmdt[l];
            /* normalised weighted Laplacians of u, v and (times s) w */
            double lap[3];
            for (int c = 0; c < 3; c++) {
                double lv = 0;
                if (j < W - 1) lv -= (u3[(l + 1) * 3 + c] - u3[l * 3 + c]) * phi[l] * regF[l * 2 + 0];
                if (j > 0) lv += (u3[l * 3 + c] - u3[(l - 1) * 3 + c]) * phi[l - 1] * regF[(l - 1) * 2 + 0];
                if (i < H - 1) lv -= (u3[(l + W) * 3 + c] - u3[l * 3 + c]) * phi[l] * regF[l * 2 + 1];
                if (i > 0) lv += (u3[l * 3 + c] - u3[(l - W) * 3 + c]) * phi[l - W] * regF[(l - W) * 2 + 1];
                double nrm = 0;
                int cnt = 0;
                if (j < W - 1) { nrm += regF[l * 2 + 0]; cnt++; }
                if (j > 0) { nrm += regF[(l - 1) * 2 + 0]; cnt++; }
                if (i < H - 1) { nrm += regF[l * 2 + 1]; cnt++; }
                if (i > 0) { nrm += regF[(l - W) * 2 + 1]; cnt++; }
                if (std::fabs(nrm) < 1e-5) lv = 0;
                else lv /= (nrm / cnt);
                lap[c] = lv;
            }
            const double uL = lap[0], vL = lap[1], wL = dswF[l] * lap[2];
            double sumXY = 0, sumZ = 0;
            const double al = in.alpha, ga = in.gamma;
            if (j > 0) {
                const size_t o2 = l - 1;
                const double wxy = phi[o2] * regF[o2 * 2 + 0], wz = wxy * dswF[o2];
                A[0 * nz + l * 3 + 0] = (F)(al * wxy); A[0 * nz + l * 3 + 1] = (F)(al * wxy); A[0 * nz + l * 3 + 2] = (F)(al * wz);
                sumXY += wxy; sumZ += wz;
            }
            if (i > 0) {
                const size_t o2 = l - W;
                const double wxy = phi[o2] * regF[o2 * 2 + 1], wz = wxy * dswF[o2];
                A[1 * nz + l * 3 + 0] = (F)(al * wxy); A[1 * nz + l * 3 + 1] = (F)(al * wxy); A[1 * nz + l * 3 + 2] = (F)(al * wz);
                sumXY += wxy; sumZ += wz;
            }
            if (j < W - 1) {
                const double wxy = phi[l] * regF[l * 2 + 0], wz = wxy * dswF[l];
                A[2 * nz + l * 3 + 0] = (F)(al * wxy); A[2 * nz + l * 3 + 1] = (F)(al * wxy); A[2 * nz + l * 3 + 2] = (F)(al * wz);
                sumXY += wxy; sumZ += wz;
            }
            if (i < H - 1) {
                const double wxy = phi[l] * regF[l * 2 + 1], wz = wxy * dswF[l];
                A[3 * nz + l * 3 + 0] = (F)(al * wxy); A[3 * nz + l * 3 + 1] = (F)(al * wxy); A[3 * nz + l * 3 + 2] = (F)(al * wz);
                sumXY += wxy; sumZ += wz;
            }
            const size_t pu = l * 3, pv = l * 3 + 1, pw = l * 3 + 2;
            A[4 * nz + pu] = (F)(-(ix2 + dx2 + al * sumXY));
            A[5 * nz + pu] = (F)(-ixy - dxy);
            A[6 * nz + pu] = (F)(pi[l] * dmdx[l]);
            A[7 * nz + pu] = (F)(-(-itx - dtx + al * -uL));
            A[4 * nz + pu] = (F)((double)A[4 * nz + pu] + -(ga));
            A[7 * nz + pu] = (F)((double)A[7 * nz + pu] + -(-ga * u3[pu]));

            A[4 * nz + pv] = (F)(-ixy - dxy);
            A[5 * nz + pv] = (F)(-(iy2 + dy2 + al * sumXY));
            A[6 * nz + pv] = (F)(pi[l] * dmdy[l]);
            A[7 * nz + pv] = (F)(-(-ity - dty + al * -vL));
            A[5 * nz + pv] = (F)((double)A[5 * nz + pv] + -(ga));
            A[7 * nz + pv] = (F)((double)A[7 * nz + pv] + -(-ga * u3[pv]));

            A[4 * nz + pw] = (F)(pi[l] * dmdx[l]);
            A[5 * nz + pw] = (F)(pi[l] * dmdy[l]);
            A[6 * nz + pw] = (F)(-(pi[l] + al * sumZ));
            A[7 * nz + pw] = (F)(-(pi[l] * dmdt[l] + al * -wL));
            A[6 * nz + pw] = (F)((double)A[6 * nz + pw] + -(ga * magF[l]));
            A[7 * nz + pw] = (F)((double)A[7 * nz + pw] + -(-ga * magF[l] * u3[pw]));
        }
}

/* imgDerivativesKernel / imgDerivativesKernelWithClamp (.cu:84-147). */
static void img_derivs(int W, int H, int C, const double* I1, const double* I2w, double maxv, bool clampv,
                       std::vector<double>& dx, std::vector<double>& dy, std::vector<double>& dt)
{
    static const double g[5] = {1, -8, 0, 8, -1};
    dx.assign((size_t)W * H * C, 0); dy.assign((size_t)W * H * C, 0); dt.assign((size_t)W * H * C, 0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++)
            for (int k = 0; k < C; k++) {
                const size_t idx = ((size_t)i * W + j) * C + k;
                double sx = 0, sy = 0;
                for (int c = j - 2, m = 0; c <= j + 2; c++, m++) {
                    const int cc = std::max(0, std::min(W - 1, c));
                    sx += g[m] * (.4 * I1[((size_t)i * W + cc) * C + k] + .6 * I2w[((size_t)i * W + cc) * C + k]);
                }
                for (int r = i - 2, m = 0; r <= i + 2; r++, m++) {
                    const int rr = std::max(0, std::min(H - 1, r));
                    sy += g[m] * (.4 * I1[((size_t)rr * W + j) * C + k] + .6 * I2w[((size_t)rr * W + j) * C + k]);
                }
                if (clampv) {
                    dx[idx] = std::min(std::max(sx / 12, -maxv), maxv);
                    dy[idx] = std::min(std::max(sy / 12, -maxv), maxv);
                    dt[idx] = std::min(std::max(I2w[idx] - I1[idx], -maxv), maxv);
                } else {
                    dx[idx] = sx / 12;
                    dy[idx] = sy / 12;
                    dt[idx] = I2w[idx] - I1[idx];
                }
            }
}

/* warpColorImgWithSceneFlowKernel / warpDepthImgWithSceneFlowKernel (.cu:579-635): the device
 * warp the reference uses inside a level (FP32 bilinear weights, floor + clamp). */
template <bool FP64>
static void warp_dev(int W, int H, int C, const double* I1, const double* I2, const double* d1, const double* d2,
                     const std::vector<double>& u3, double* wI2, double* wD2)
{
    typedef typename P<FP64>::F F;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            const size_t l = (size_t)i * W + j;
            const double x = j + u3[l * 3 + 0], y = i + u3[l * 3 + 1];
            if (x < 0 || x > W - 1 || y < 0 || y > H - 1) {
                for (int k = 0; k < C; k++) wI2[l * C + k] = I1[l * C + k];
                wD2[l] = d1[l] - u3[l * 3 + 2];
            } else {
                const int x0 = std::max(0, std::min(W - 1, (int)std::floor(x)));
                const int y0 = std::max(0, std::min(H - 1, (int)std::floor(y)));
                const int x1 = std::min(W - 1, x0 + 1), y1 = std::min(H - 1, y0 + 1);
                const F ax = (F)(x - x0), ay = (F)(y - y0);
                const F w00 = (1 - ax) * (1 - ay), w01 = (1 - ax) * ay, w10 = ax * (1 - ay), w11 = ax * ay;
                for (int k = 0; k < C; k++)
                    wI2[l * C + k] = w00 * I2[((size_t)y0 * W + x0) * C + k] + w01 * I2[((size_t)y1 * W + x0) * C + k] +
                                     w10 * I2[((size_t)y0 * W + x1) * C + k] + w11 * I2[((size_t)y1 * W + x1) * C + k];
                wD2[l] = w00 * d2[(size_t)y0 * W + x0] + w01 * d2[(size_t)y1 * W + x0] + w10 * d2[(size_t)y0 * W + x1] +
                         w11 * d2[(size_t)y1 * W + x1] - u3[l * 3 + 2];
            }
        }
}

/* One level: restates the host loop of sceneFlowSingleScale (.cu:660-969). */
template <bool FP64>
void single_scale(const SolverIn& in, const rgbdflow_params& p, int fixed, Img& wI2, Img& wD2,
                  double* u, double* v, double* w, LevelTrace* tr)
{
    typedef typename P<FP64>::F F;
    const int W = in.W, H = in.H, C = in.C;
    const size_t N = (size_t)W * H;
    std::vector<F> ddwF(N), dswF(N), magF(N), regF(N * 2), conv(N * 3);
    for (size_t l = 0; l < N; l++) {
        ddwF[l] = (F)in.ddw[l]; dswF[l] = (F)in.dsw[l]; magF[l] = (F)in.mag[l];
        regF[l * 2] = (F)in.regw[l * 2]; regF[l * 2 + 1] = (F)in.regw[l * 2 + 1];
        conv[l * 3 + 0] = 1; conv[l * 3 + 1] = 1;
        conv[l * 3 + 2] = (F)((FP64 ? (double)in.f_level : (double)(float)in.f_level) / in.dm1[l]);
    }
    std::vector<double> u3(N * 3);
    for (size_t l = 0; l < N; l++) { u3[l * 3] = u[l]; u3[l * 3 + 1] = v[l]; u3[l * 3 + 2] = w[l]; }
    std::vector<F> du(N * 3, (F)0), q(N), A(N * 3 * 8, (F)0), prev;
    std::vector<double> imdx, imdy, imdt, dmdx, dmdy, dmdt;
    const F omega = (F)p.omega, step = (F)p.max_flow_step;
    const int period = p.sor_check_period > 0 ? p.sor_check_period : 25;
    if (tr) { tr->outer = 0; }
    for (int count = 0; count < in.nOuter; count++) {
        img_derivs(W, H, C, in.Im1, wI2.data(), 0, false, imdx, imdy, imdt);
        img_derivs(W, H, 1, in.dm1, wD2.data(), p.max_depth_grad, true, dmdx, dmdy, dmdt);
        std::fill(du.begin(), du.end(), (F)0);
        /* fillOcclusionPenaltyKernel (.cu:640-648): uses the unwarped dm2 */
        for (size_t l = 0; l < N; l++)
            q[l] = (in.dm1[l] + u3[l * 3 + 2] < in.dm2[l] + p.occ_margin * (double)sqc<FP64>(in.dm1[l])) ? (F)1 : (F)p.occ_penalty;
        int sorDone = 0;
        float lastDiff = -1;
        for (int hh = 0; hh < in.nInner; hh++) {
            linearize<FP64>(in, p, u3, du, wI2, wD2, q, ddwF, dswF, magF, regF, imdx, imdy, imdt, dmdx, dmdy, dmdt, A);
            for (int it = 0; it < in.nSOR; it++) {
                const bool check = !fixed && (it % period == period - 1);
                if (check) prev = du;
                sor_sweep<FP64>(W, H, A, du, 0, omega, step);
                sor_sweep<FP64>(W, H, A, du, 1, omega, step);
                sorDone = it + 1;
                if (check) {
                    F md = 0;
                    for (size_t z = 0; z < N * 3; z++) md = std::max(md, (F)std::fabs(du[z] - prev[z]));
                    lastDiff = (float)md;
                    if ((double)md < p.sor_tol) break;
                    if (md >= step) break;
                }
            }
        }
        for (size_t z = 0; z < N * 3; z++) u3[z] += du[z];
        warp_dev<FP64>(W, H, C, in.Im1, in.Im2, in.dm1, in.dm2, u3, wI2.data(), wD2.data());
        float stat = -1;
        bool stop = false;
        if (in.allowEarly && !fixed) {
            /* thrust::transform_reduce of sqrCU(du) * wt (.cu:948): a fixed-order FP64 sum here */
            std::vector<double> rows(H, 0.0);
#pragma omp parallel for schedule(static)
            for (int i = 0; i < H; i++) {
                double s = 0;
                for (size_t z = (size_t)i * W * 3; z < (size_t)(i + 1) * W * 3; z++) s += (double)(F)(sqc<FP64>(du[z]) * conv[z]);
                rows[i] = s;
            }
            double s = 0;
            for (int i = 0; i < H; i++) s += rows[i];
            const double st = s / (double)(W * H * 3);
            stat = (float)st;
            stop = st < p.outer_tol;
        }
        if (tr && count < RGBDFLOW_MAX_OUTER) {
            tr->sor[count] = sorDone;
            tr->maxdiff[count] = lastDiff;
            tr->stat[count] = stat;
        }
        if (tr) tr->outer = count + 1;
        if (stop) break;
    }
    for (size_t l = 0; l < N; l++) { u[l] = u3[l * 3]; v[l] = u3[l * 3 + 1]; w[l] = u3[l * 3 + 2]; }
}

/* OpticalFlow::calculateDepthMagnitudeTermWeights (OpticalFlow.cpp:104-111).  The reference
 * allocates the full-resolution size but indexes the level's depth with the level's own width;
 * the solver then uses only the first W_k*H_k entries (.cu:686).  Entry l therefore reads
 * Depth_k[(l / xRes) * W_k + l % xRes]; that index never exceeds l. */
void depth_mag_weights(const Img& depthk, const rgbdflow_camera_params& camFull, std::vector<double>& mag)
{
    const size_t N = (size_t)depthk.w * depthk.h;
    mag.assign(N, 0);
    const double f = camFull.focalLength;
    for (size_t l = 0; l < N; l++) {
        const size_t src = (l / camFull.xRes) * depthk.w + (l % camFull.xRes);
        const double z = depthk.d[src];
        mag[l] = (z > 0) ? sqr(f / z) : sqr(f / 2);
    }
}

/* OpticalFlow::calculateRegularizationWeights (OpticalFlow.cpp:113-141); HPB is not restated. */
void reg_weights(int W, int H, const double* depth, int type, std::vector<double>& rw)
{
    rw.assign((size_t)W * H * 2, 0);
    for (int i = 0, l = 0; i < H; i++)
        for (int j = 0; j < W; j++, l++) {
            if (j < W - 1) rw[l * 2 + 0] = (type == RGBDFLOW_REG_LETOUZEY) ? std::exp(-sqr((depth[l] - depth[l + 1]) / .02)) : 1.0;
            if (i < H - 1) rw[l * 2 + 1] = (type == RGBDFLOW_REG_LETOUZEY) ? std::exp(-sqr((depth[l] - depth[l + W]) / .02)) : 1.0;
        }
}

}  // namespace sfo
// HPB pieces, defined below
void heuristic_pb(const double* img, const double* depthd, int W, int H, float* out);
void depth_map_pyramid(const sfo::Img& image, double ratio, int min_width, std::vector<sfo::Img>& lev);
void fill_small_regions_color(sfo::Img& depth, const sfo::Img& col, unsigned maxRegion);
namespace sfo {

/* calculateRegularizationWeights, HPB form (OpticalFlow.cpp:126-131): 1 - .99 hpb for the right and
 * lower neighbours. */
static void hpb_reg_weights(const Img& colour, const Img& rawDepth, std::vector<double>& rw)
{
    const int W = colour.w, H = colour.h;
    std::vector<float> hpb((size_t)W * H * 2);
    heuristic_pb(colour.data(), rawDepth.data(), W, H, hpb.data());
    rw.assign((size_t)W * H * 2, 0);
    for (int i = 0, l = 0; i < H; i++)
        for (int j = 0; j < W; j++, l++) {
            if (j < W - 1) rw[l * 2 + 0] = (1 - hpb[(size_t)l * 2 + 0] * .99);
            if (i < H - 1) rw[l * 2 + 1] = (1 - hpb[(size_t)l * 2 + 1] * .99);
        }
}

/* An external per-level solver with the argument list of sceneFlowSingleScale over raw planes
 * (the reference's own CUDA solver, oracle/ref_cuda_shim.cu): when set, the faithful variant's
 * levels are solved by it, everything around them by this file (the reference's own split between
 * host and device).  Set by sfo_set_level_solver; used to time the reference's GPU path. */
typedef int (*LevelSolverFn)(float f_level, const double* Im1, const double* dm1, const double* Im2, const double* dm2,
                             double* warpIm2, double* warpDm2, double* u, double* v, double* w, int W, int H, int C,
                             double colorW, const double* ddw, double alpha, const double* dsw, double gamma,
                             const double* mag, const double* regw, int nOuter, int nInner, int nSOR, int allowEarly);
static LevelSolverFn g_level_solver = nullptr;

template <bool FP64>
static void run_level(const rgbdflow_camera_params& camFull, const rgbdflow_params& p, int fixed,
                      const Img& feat1, const Img& d1, const Img& feat2, const Img& d2, Img& wI2, Img& wD2,
                      const double* ddw, const double* dsw, Img& u, Img& v, Img& w, int allowEarly, LevelTrace* tr,
                      const Img* hpbColour = nullptr, const Img* hpbDepth = nullptr)
{
    const int W = feat1.w, H = feat1.h;
    const rgbdflow_camera_params ck = resize_cam(camFull, W);
    std::vector<double> mag, rw;
    depth_mag_weights(d1, camFull, mag);
    if (p.regularization == RGBDFLOW_REG_HPB) hpb_reg_weights(*hpbColour, *hpbDepth, rw);
    else reg_weights(W, H, d1.data(), p.regularization, rw);
    SolverIn in;
    in.W = W; in.H = H; in.C = feat1.c; in.f_level = ck.focalLength;
    in.Im1 = feat1.data(); in.dm1 = d1.data(); in.Im2 = feat2.data(); in.dm2 = d2.data();
    in.colorW = p.color_data_weight; in.alpha = p.alpha; in.gamma = p.gamma;
    in.ddw = ddw; in.dsw = dsw; in.mag = mag.data(); in.regw = rw.data();
    in.nOuter = p.n_outer; in.nInner = p.n_inner; in.nSOR = p.n_sor; in.allowEarly = allowEarly;
    if (g_level_solver && !FP64) {
        const int rc = g_level_solver(in.f_level, in.Im1, in.dm1, in.Im2, in.dm2, wI2.data(), wD2.data(), u.data(),
                                      v.data(), w.data(), W, H, in.C, in.colorW, ddw, in.alpha, dsw, in.gamma, in.mag,
                                      in.regw, in.nOuter, in.nInner, in.nSOR, allowEarly);
        if (rc != 0) throw std::runtime_error("external level solver failed: " + std::to_string(rc));
        return;
    }
    single_scale<FP64>(in, p, fixed, wI2, wD2, u.data(), v.data(), w.data(), tr);
}

/* OpticalFlow::sceneFlowMultiscale (src/sceneFlowMultiscale.cpp:30-201) and
 * OpticalFlow::sceneFlowWithInit (src/sceneFlowWithInit.cpp:7-81); cam is the image-size camera. */
template <bool FP64>
void multiscale(const rgbdflow_camera_params& cam, const rgbdflow_params& p, const Img& Im1, const Img& dm1,
                const Img& Im2, const Img& dm2, const float* sigma1, const double* est, Img& u, Img& v, Img& w,
                Trace* trace)
{
    const int fixed = p.fixed_schedule;
    /* calculateDepthDataTermWeights / calculateDepthSmoothnessTermWeights (OpticalFlow.cpp:71-97) */
    Img ddw; ddw.alloc(cam.xRes, cam.yRes, 1);
    Img dsw; dsw.alloc(cam.xRes, cam.yRes, 1);
    for (size_t l = 0; l < ddw.n(); l++) {
        if (!(sigma1[l] > 0)) throw std::runtime_error("depth sigma must be > 0");
        ddw.d[l] = stereo_error(1) / sigma1[l] * p.depth_vs_color_data_weight;
        dsw.d[l] = sqr(cam.focalLength);
    }
    Img d1 = dm1, d2 = dm2;
    if (p.fill_holes) {
        fill_depth(d1.data(), d1.w, d1.h);
        fill_depth(d2.data(), d2.w, d2.h);
    }
    if (est) {
        const int W = Im1.w, H = Im1.h;
        u.alloc(W, H, 1); v.alloc(W, H, 1); w.alloc(W, H, 1);
        for (int l = 0; l < W * H; l++) { u.d[l] = est[l * 3]; v.d[l] = est[l * 3 + 1]; w.d[l] = est[l * 3 + 2]; }
        Img f1, f2, wI2, wD2;
        im2feature(Im1, f1);
        im2feature(Im2, f2);
        warp_cpu(f1, d1, f2, d2, wI2, wD2, u.data(), v.data(), w.data());
        if (trace) { trace->n_levels = 1; trace->w[0] = W; trace->h[0] = H; }
        // sceneFlowWithInit.cpp:48: HPB of the full-size colour and the raw depth
        run_level<FP64>(cam, p, fixed, f1, d1, f2, d2, wI2, wD2, ddw.data(), dsw.data(), u, v, w, 0,
                        trace ? &trace->lev[0] : nullptr, &Im1, &dm1);
        return;
    }
    // the raw-depth pyramid of HPB (sceneFlowMultiscale.cpp:79-83): small invalid regions of the
    // raw depth filled guided by colour, then DepthMapPyramid
    std::vector<Img> rawPyr;
    if (p.regularization == RGBDFLOW_REG_HPB) {
        Img filtered = dm1;
        fill_small_regions_color(filtered, Im1, 60);
        const int mw = p.min_width < 0 ? std::max(1, Im1.w / -p.min_width) : p.min_width;
        depth_map_pyramid(filtered, p.pyramid_ratio, mw, rawPyr);
    }
    std::vector<Img> pI1, pI2, pD1, pD2, pDDW, pDSW;
    build_pyramid(Im1, p.pyramid_ratio, p.min_width, pI1);
    build_pyramid(Im2, p.pyramid_ratio, p.min_width, pI2);
    build_pyramid(d1, p.pyramid_ratio, p.min_width, pD1);
    build_pyramid(d2, p.pyramid_ratio, p.min_width, pD2);
    build_pyramid(ddw, p.pyramid_ratio, p.min_width, pDDW);
    build_pyramid(dsw, p.pyramid_ratio, p.min_width, pDSW);
    const int L = (int)pI1.size();
    if (trace) trace->n_levels = L;
    Img wI2, wD2;
    for (int k = L - 1; k >= 0; k--) {
        Img f1, f2;
        im2feature(pI1[k], f1);
        im2feature(pI2[k], f2);
        const int W = f1.w, H = f1.h;
        if (trace) { trace->w[k] = W; trace->h[k] = H; }
        if (k == L - 1) {
            u.alloc(W, H, 1); v.alloc(W, H, 1); w.alloc(W, H, 1);
            wI2 = f2;
            wD2 = pD2[k];
        } else {
            resize_dims(u, u, W, H);
            resize_dims(v, v, W, H);
            resize_dims(w, w, W, H);
            for (auto& x : u.d) x *= 1 / p.pyramid_ratio;
            for (auto& x : v.d) x *= 1 / p.pyramid_ratio;
            warp_cpu(f1, pD1[k], f2, pD2[k], wI2, wD2, u.data(), v.data(), w.data());
        }
        run_level<FP64>(cam, p, fixed, f1, pD1[k], f2, pD2[k], wI2, wD2, pDDW[k].data(), pDSW[k].data(), u, v, w,
                        k < L - 1, trace ? &trace->lev[k] : nullptr, &pI1[k], rawPyr.empty() ? nullptr : &rawPyr[k]);
    }
}

} // namespace sfo

/* =========================================================================================== */
/* C entry points used by the tests (ctypes) and the CPU baseline.                              */

using namespace sfo;

/* DepthMapPyramid::ConstructPyramid (src/depthMapPyramid.cpp:15-91), the raw-depth pyramid the
 * HPB regularisation reads (sceneFlowMultiscale.cpp:82): values <= 0 are invalid and stay -1;
 * a valid pixel averages, in float, the depths of its 2x2 neighbourhood that lie within
 * .005 * stereoErrorRatio of its own (or of the diagonally opposite pixel's, when its own group
 * is alone).  Both sampling factors are the ratio of the heights, as in the reference. */
void depth_map_pyramid(const Img& image, double ratio, int min_width, std::vector<Img>& lev)
{
    if (min_width < 0) min_width = std::max(1, image.w / -min_width);  // API convention: W / d per pair
    if (min_width == 0) throw std::runtime_error("min_width 0: the level count never ends");
    if (ratio > 0.98 || ratio < 0.4) ratio = 0.75;
    double w = image.w * ratio;
    int nLevels = 1;
    while (w >= min_width) { nLevels++; w *= ratio; }
    lev.assign(nLevels, Img());
    lev[0] = image;
    for (int m = 1; m < nLevels; m++) {
        const Img& L = lev[m - 1];
        const int LW = L.w, LH = L.h;
        const double levelRatio = std::pow(ratio, m);
        Img foo;
        foo.alloc((int)(image.w * levelRatio), (int)(image.h * levelRatio), 1);
        auto at = [&](int y, int x) { return L.d[(size_t)y * LW + x]; };
        const float factor = (float)LH / foo.h;
        const float maxDZ = .005f;
        for (int i = 0; i < foo.h; i++)
            for (int j = 0; j < foo.w; j++) {
                const int x = std::max(0, std::min(LW - 1, (int)std::rint(factor * j)));
                const int y = std::max(0, std::min(LH - 1, (int)std::rint(factor * i)));
                double& out = foo.d[(size_t)i * foo.w + j];
                if (!(at(y, x) > 0)) { out = -1; continue; }
                const int xs[2] = {std::max(0, std::min(LW - 1, (int)std::floor(factor * j))), 0};
                const int ys[2] = {std::max(0, std::min(LH - 1, (int)std::floor(factor * i))), 0};
                const int xs1 = std::min(LW - 1, xs[0] + 1), ys1 = std::min(LH - 1, ys[0] + 1);
                const int X[2] = {xs[0], xs1}, Y[2] = {ys[0], ys1};
                const int xi = (x == X[0]) ? 0 : 1, yi = (y == Y[0]) ? 0 : 1;
                const double z = at(y, x);
                const double tol = maxDZ * stereo_error_ratio(z);
                std::vector<float> comp;
                comp.push_back((float)z);
                if (std::fabs(at(Y[yi], X[!xi]) - z) < tol) comp.push_back((float)at(Y[yi], X[!xi]));
                if (std::fabs(at(Y[!yi], X[xi]) - z) < tol) comp.push_back((float)at(Y[!yi], X[xi]));
                if (std::fabs(at(Y[!yi], X[!xi]) - z) < tol) comp.push_back((float)at(Y[!yi], X[!xi]));
                if (comp.size() > 1) {
                    float avg = 0;
                    for (float v : comp) avg += v;
                    out = avg / comp.size();
                } else {
                    const double zo = at(Y[!yi], X[!xi]);
                    const double tolo = maxDZ * stereo_error_ratio(zo);
                    std::vector<float> other;
                    other.push_back((float)zo);
                    if (std::fabs(at(Y[yi], X[!xi]) - zo) < tolo) other.push_back((float)at(Y[yi], X[!xi]));
                    if (std::fabs(at(Y[!yi], X[xi]) - zo) < tolo) other.push_back((float)at(Y[!yi], X[xi]));
                    if (other.size() > 1) {
                        float avg = 0;
                        for (float v : other) avg += v;
                        out = avg / other.size();
                    } else {
                        out = z;
                    }
                }
            }
        lev[m] = std::move(foo);
    }
}

/* recursiveMedianFilterSmallInvalidRegionsUsingColor (src/recursiveMedianFiltering.cpp:127-222):
 * each 4-connected region of invalid depth (<= 0) of at most maxRegion pixels is filled, the pixel
 * with the most valid 3x3 neighbours first, each with the average of its valid neighbours weighted
 * by exp(-|colour difference|^2 / .6) (float sums, as the reference).  Order: the reference takes
 * regions in the iteration order of a boost::unordered_map and, among pixels with equally many
 * valid neighbours, the first of a std::unordered_set, both hashed by boost::hash, whose mixing
 * depends on the unpinned Boost version.  Here regions go in the raster order of their first
 * pixel and ties by raster order; values differ from the reference's only where that order
 * matters (pixels with equal counts, regions that touch diagonally). */
void fill_small_regions_color(Img& depth, const Img& col, unsigned maxRegion)
{
    const int W = depth.w, H = depth.h;
    const size_t N = (size_t)W * H;
    auto dz = [&](int i, int j) -> double& { return depth.d[(size_t)i * W + j]; };
    std::vector<int> comp(N, -1);
    std::vector<std::vector<int>> comps;
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            if (!(dz(i, j) <= 0) || comp[(size_t)i * W + j] >= 0) continue;
            const int id = (int)comps.size();
            comps.emplace_back();
            std::vector<int> stack{i * W + j};
            comp[(size_t)i * W + j] = id;
            while (!stack.empty()) {
                const int q = stack.back();
                stack.pop_back();
                comps[id].push_back(q);
                const int qi = q / W, qj = q % W;
                const int ni[4] = {qi - 1, qi + 1, qi, qi}, nj[4] = {qj, qj, qj - 1, qj + 1};
                for (int t = 0; t < 4; t++) {
                    if (ni[t] < 0 || ni[t] >= H || nj[t] < 0 || nj[t] >= W) continue;
                    const size_t o = (size_t)ni[t] * W + nj[t];
                    if (comp[o] < 0 && dz(ni[t], nj[t]) <= 0) { comp[o] = id; stack.push_back((int)o); }
                }
            }
        }
    std::vector<int> count(N, -1);  // valid 3x3 neighbours of the region's unfilled pixels; -1 otherwise
    for (auto& c : comps) {
        if (c.size() > maxRegion) continue;
        std::sort(c.begin(), c.end());
        std::vector<std::set<int>> bucket(9);
        for (int q : c) {
            const int i = q / W, j = q % W;
            int n = 0;
            for (int ii = std::max(0, i - 1); ii <= std::min(H - 1, i + 1); ii++)
                for (int jj = std::max(0, j - 1); jj <= std::min(W - 1, j + 1); jj++)
                    if (dz(ii, jj) > 0) n++;
            count[q] = n;
            bucket[n].insert(q);
        }
        for (size_t left = c.size(); left > 0; left--) {
            int m = 8;
            while (m >= 0 && bucket[m].empty()) m--;
            if (m <= 0) throw std::runtime_error("colour-guided fill: a region without valid neighbours");
            const int q = *bucket[m].begin();
            bucket[m].erase(bucket[m].begin());
            count[q] = -1;
            const int i = q / W, j = q % W;
            float zSum = 0, weightSum = 0;
            for (int ii = std::max(0, i - 1); ii <= std::min(H - 1, i + 1); ii++)
                for (int jj = std::max(0, j - 1); jj <= std::min(W - 1, j + 1); jj++) {
                    const size_t o2 = (size_t)ii * W + jj;
                    if (dz(ii, jj) > 0) {
                        const size_t a = (size_t)q * 3, b = o2 * 3;
                        const float w = (float)std::exp(-(sqr(col.d[a] - col.d[b]) + sqr(col.d[a + 1] - col.d[b + 1]) +
                                                          sqr(col.d[a + 2] - col.d[b + 2])) / .6);
                        zSum = (float)(zSum + dz(ii, jj) * w);  // float += double, as the reference
                        weightSum += w;
                    } else if (count[o2] >= 0) {
                        bucket[count[o2]].erase((int)o2);
                        count[o2]++;
                        bucket[count[o2]].insert((int)o2);
                    }
                }
            dz(i, j) = zSum / weightSum;
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* HPB: the heuristic boundary probability the reference's default regularisation weights are
 * made of (computeHeuristicPb, src/heuristicProbBoundary.cpp:21-41 and
 * src/heuristicBoundaries.cpp:40-358).  Restated with the reference's float / double mix, except
 * where its arithmetic is fixed by unpinned library versions:
 *   - normals: the reference takes them from PCL's NormalEstimation (not vendored, version not
 *     pinned): the eigenvector of the smallest eigenvalue of the neighbourhood's covariance,
 *     turned towards the camera.  Here: mean and covariance in double, a cyclic Jacobi
 *     eigen-solve in double, the normal rounded to float.
 *   - exp of a float: the overload the reference's headers select is not pinned; double here.
 *   - normalising a zero vector (Eigen version dependent) leaves it zero here; it only happens
 *     where the normal cue is discarded anyway (fewer than 3 valid normals). */

/* 3x3 symmetric eigen-solve, cyclic Jacobi rotations in double: the eigenvector of the smallest
 * eigenvalue, unit length. */
static void smallest_eigvec(double a[3][3], double n[3])
{
    double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int sweep = 0; sweep < 64; sweep++) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        if (off < 1e-300) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                if (a[p][q] == 0) continue;
                const double theta = (a[q][q] - a[p][p]) / (2 * a[p][q]);
                const double t = (theta >= 0 ? 1 : -1) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                const double c = 1 / std::sqrt(t * t + 1), sn = t * c;
                for (int k = 0; k < 3; k++) {
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - sn * akq;
                    a[k][q] = sn * akp + c * akq;
                }
                for (int k = 0; k < 3; k++) {
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - sn * aqk;
                    a[q][k] = sn * apk + c * aqk;
                }
                for (int k = 0; k < 3; k++) {
                    const double vkp = v[k][p], vkq = v[k][q];
                    v[k][p] = c * vkp - sn * vkq;
                    v[k][q] = sn * vkp + c * vkq;
                }
            }
    }
    int m = 0;
    for (int k = 1; k < 3; k++)
        if (a[k][k] < a[m][m]) m = k;
    const double len = std::sqrt(v[0][m] * v[0][m] + v[1][m] * v[1][m] + v[2][m] * v[2][m]);
    for (int k = 0; k < 3; k++) n[k] = v[k][m] / len;
}

struct Cloud {
    int W = 0, H = 0;
    std::vector<float> x, y, z;       // depth_to_cloud (depth_to_cloud_lib.ipp:13-60)
    std::vector<float> nx, ny, nz;    // normals; 0 where invalid (markNormalInvalid, cloudNormals.ipp:116-120)
};

/* depth_to_cloud with every pixel kept (depth_to_cloud_lib.ipp:35-50) and setOrganizedNormals
 * (cloudNormals.ipp:395-506) with a 9x9 window (k = 4), no downsampling, neighbours whose depth is
 * within .05 * stereoErrorRatio of the centre's, at least max(6, 81 / 3) of them
 * (computeOrganizedPointCloudNormalsThreadMain, cloudNormals.ipp:131-205). */
static void organized_cloud_normals(const float* depth, int W, int H, float cx, float cy, float f, Cloud& cl)
{
    const size_t N = (size_t)W * H;
    cl.W = W; cl.H = H;
    cl.x.assign(N, 0); cl.y.assign(N, 0); cl.z.assign(N, 0);
    cl.nx.assign(N, 0); cl.ny.assign(N, 0); cl.nz.assign(N, 0);
    for (int r = 0; r < H; r++)
        for (int c = 0; c < W; c++) {
            const size_t o = (size_t)r * W + c;
            const float d = depth[o];
            cl.x[o] = (((float)c - cx) * d / f);
            cl.y[o] = (((float)r - cy) * d / f);
            cl.z[o] = d;
        }
    const int k = 4;
    const unsigned minPts = std::max(6u, (unsigned)((2 * k + 1) * (2 * k + 1) / 3));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            const size_t o = (size_t)i * W + j;
            if (!(cl.z[o] > 0)) continue;
            std::vector<size_t> nn;
            for (int yy = std::max(0, i - k); yy <= std::min(H - 1, i + k); yy++)
                for (int xx = std::max(0, j - k); xx <= std::min(W - 1, j + k); xx++) {
                    const size_t o2 = (size_t)yy * W + xx;
                    // setOrganizedNormals takes the .05 as a float, then passes it on as a double
                    if (std::fabs(cl.z[o] - cl.z[o2]) < (double).05f * stereo_error_ratio(cl.z[o])) nn.push_back(o2);
                }
            if (nn.size() < minPts) continue;
            double m[3] = {0, 0, 0};
            for (size_t q : nn) { m[0] += cl.x[q]; m[1] += cl.y[q]; m[2] += cl.z[q]; }
            for (double& t : m) t /= (double)nn.size();
            double a[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (size_t q : nn) {
                const double d[3] = {cl.x[q] - m[0], cl.y[q] - m[1], cl.z[q] - m[2]};
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++) a[r][c] += d[r] * d[c];
            }
            for (auto& row : a)
                for (double& t : row) t /= (double)nn.size();
            double n[3];
            smallest_eigvec(a, n);
            if (!(std::isfinite(n[0]) && std::isfinite(n[1]) && std::isfinite(n[2]))) continue;
            // flipNormalTowardsViewpoint with the viewpoint at the origin
            const double cosv = -(cl.x[o] * n[0] + cl.y[o] * n[1] + cl.z[o] * n[2]);
            if (cosv < 0) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
            cl.nx[o] = (float)n[0]; cl.ny[o] = (float)n[1]; cl.nz[o] = (float)n[2];
        }
}

/* computeIntegralImage (include/image_features/halfDiskFeatures.ipp:102-154): one more row and
 * column of zeros at index -1 (here 0), float (or uint32) sums in the reference's order. */
template <typename T>
static void integral_image(const std::vector<T>& img, int W, int H, int C, std::vector<T>& ii)
{
    const int W1 = W + 1;
    ii.assign((size_t)(H + 1) * W1 * C, 0);
    for (int j = 0; j < W; j++)
        for (int l = 0; l < C; l++)
            ii[((size_t)1 * W1 + j + 1) * C + l] = ii[((size_t)1 * W1 + j) * C + l] + img[((size_t)j) * C + l];
    for (int i = 1; i < H; i++) {
        std::vector<T> rowSum(C, 0);
        for (int j = 0; j < W; j++)
            for (int l = 0; l < C; l++) {
                const T v = img[((size_t)i * W + j) * C + l];
                ii[((size_t)(i + 1) * W1 + j + 1) * C + l] = ii[((size_t)i * W1 + j + 1) * C + l] + rowSum[l] + v;
                rowSum[l] += v;
            }
    }
}

/* computeHeuristicPb on one pyramid level (heuristicProbBoundary.cpp:21-41 wrapping
 * heuristicBoundaries.cpp:40-358): img = the level's colour image (3 channels in [0, 1], BGR),
 * depth = the level of the raw-depth pyramid (<= 0 invalid).  out: W*H*2 floats, (right, down)
 * boundary probability of each pixel. */
void heuristic_pb(const double* img, const double* depthd, int W, int H, float* out)
{
    const size_t N = (size_t)W * H;
    // the wrapper's camera: Kinect intrinsics scaled to the level
    const unsigned xRes = (unsigned)W, yRes = (unsigned)H;
    const float cx = (float)(xRes / 2), cy = (float)(yRes / 2);
    const float f = (float)(525.0 * xRes / 640);
    // the wrapper's 8-bit image: channels reversed, 255 * value truncated; then / 255.0 as float
    std::vector<float> cols(N * 3);
    std::vector<float> depth(N);
    for (size_t l = 0; l < N; l++) {
        const unsigned char px[3] = {(unsigned char)(255 * img[l * 3 + 2]), (unsigned char)(255 * img[l * 3 + 1]),
                                     (unsigned char)(255 * img[l * 3 + 0])};
        for (int k = 0; k < 3; k++) cols[l * 3 + k] = (float)(px[k] / 255.0);
        depth[l] = (float)depthd[l];
    }
    Cloud cl;
    organized_cloud_normals(depth.data(), W, H, cx, cy, f, cl);
    std::vector<float> normals(N * 3);
    std::vector<uint32_t> nvalid(N, 0);
    for (size_t l = 0; l < N; l++) {
        const float n0 = cl.nx[l], n1 = cl.ny[l], n2 = cl.nz[l];
        normals[l * 3] = n0; normals[l * 3 + 1] = n1; normals[l * 3 + 2] = n2;
        const float sq = n0 * n0 + n1 * n1 + n2 * n2;
        if (!std::isfinite(n0) || !std::isfinite(n1) || !std::isfinite(n2) || std::fabs(sq - 1) < 1e-4) nvalid[l] = 1;
    }
    // half-disk radius per pixel: 2 cm at the pixel's depth, 1..5 pixels (heuristicBoundaries.cpp:101-109)
    std::vector<int> radii(N);
    for (size_t l = 0; l < N; l++)
        radii[l] = depth[l] > 0 ? std::max(1, std::min(5, (int)std::rint(f * .02f / depth[l]))) : 5;
    std::vector<float> ciI, niI;
    std::vector<uint32_t> viI;
    integral_image(cols, W, H, 3, ciI);
    integral_image(normals, W, H, 3, niI);
    integral_image(nvalid, W, H, 1, viI);
    const int W1 = W + 1;
    auto II = [&](const auto& v, int C, int y, int x, int k) { return v[((size_t)(y + 1) * W1 + (x + 1)) * C + k]; };
    std::vector<float> colH(N, 0), colV(N, 0), norH(N, 0), norV(N, 0);
    auto normalize3 = [](float v[3]) {
        const float n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        if (n > 0) for (int k = 0; k < 3; k++) v[k] /= n;
    };
#pragma omp parallel for schedule(static)
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            const size_t o = (size_t)i * W + j;
            const int hw = radii[o];
            const int xmin = std::max(0, j - hw), xmax = std::min(W - 1, j + hw - 1);
            const int ymin = std::max(0, i - hw), ymax = std::min(H - 1, i + hw - 1);
            const float hsize0 = (float)((j - xmin) * (ymax - ymin + 1)), hsize1 = (float)((xmax - j + 1) * (ymax - ymin + 1));
            const float vsize0 = (float)((xmax - xmin + 1) * (i - ymin)), vsize1 = (float)((xmax - xmin + 1) * (ymax - i + 1));
            auto H1 = [&](const auto& v, int C, int k) { return II(v, C, ymax, xmax, k) - II(v, C, ymax, j - 1, k) - II(v, C, ymin - 1, xmax, k) + II(v, C, ymin - 1, j - 1, k); };
            auto H0 = [&](const auto& v, int C, int k) { return II(v, C, ymax, j - 1, k) - II(v, C, ymin - 1, j - 1, k) - II(v, C, ymax, xmin - 1, k) + II(v, C, ymin - 1, xmin - 1, k); };
            auto V1 = [&](const auto& v, int C, int k) { return II(v, C, ymax, xmax, k) - II(v, C, i - 1, xmax, k) - II(v, C, ymax, xmin - 1, k) + II(v, C, i - 1, xmin - 1, k); };
            auto V0 = [&](const auto& v, int C, int k) { return II(v, C, i - 1, xmax, k) - II(v, C, i - 1, xmin - 1, k) - II(v, C, ymin - 1, xmax, k) + II(v, C, ymin - 1, xmin - 1, k); };
            auto dot = [](const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
            if (j > 0) {
                float acc = 0;
                for (int k = 0; k < 3; k++) { const float d = H1(ciI, 3, k) / hsize1 - H0(ciI, 3, k) / hsize0; acc += d * d; }
                colH[o] = std::sqrt(acc);
                float n0[3], n1[3];
                for (int k = 0; k < 3; k++) { n0[k] = H0(niI, 3, k); n1[k] = H1(niI, 3, k); }
                normalize3(n0); normalize3(n1);
                const uint32_t v0 = H0(viI, 1, 0), v1 = H1(viI, 1, 0);
                norH[o] = (std::min(v0, v1) < 3) ? 0 : (float)(.5 * (1 - dot(n0, n1)));
                if (std::min(v0, v1) > 3) {
                    const size_t oa = (size_t)i * W + (j - 1);
                    float dx[3] = {cl.x[oa] - cl.x[o], cl.y[oa] - cl.y[o], cl.z[oa] - cl.z[o]};
                    normalize3(dx);
                    const float mdx[3] = {-dx[0], -dx[1], -dx[2]};
                    const double convexity = (dot(n0, dx) + dot(n1, mdx)) / 4 + .5;
                    norH[o] = (float)(norH[o] * (1 - convexity));
                }
            }
            if (i > 0) {
                float acc = 0;
                for (int k = 0; k < 3; k++) { const float d = V1(ciI, 3, k) / vsize1 - V0(ciI, 3, k) / vsize0; acc += d * d; }
                colV[o] = std::sqrt(acc);
                float n0[3], n1[3];
                for (int k = 0; k < 3; k++) { n0[k] = V0(niI, 3, k); n1[k] = V1(niI, 3, k); }
                normalize3(n0); normalize3(n1);
                const uint32_t v0 = V0(viI, 1, 0), v1 = V1(viI, 1, 0);
                norV[o] = (std::min(v0, v1) < 3) ? 0 : (float)(.5 * (1 - dot(n0, n1)));
                if (std::min(v0, v1) > 3) {
                    const size_t oa = (size_t)(i - 1) * W + j;
                    float dx[3] = {cl.x[oa] - cl.x[o], cl.y[oa] - cl.y[o], cl.z[oa] - cl.z[o]};
                    normalize3(dx);
                    const float mdx[3] = {-dx[0], -dx[1], -dx[2]};
                    const double convexity = (dot(n0, dx) + dot(n1, mdx)) / 4 + .5;
                    norV[o] = (float)(norV[o] * (1 - convexity));
                }
            }
        }
    // the probabilities (heuristicBoundaries.cpp:223-293)
    const float depthSigma = .02f, colSigma = .7f, normSigma = .4f;
    std::vector<float> bp(N * 2, 0);
    auto sqrf = [](float v) { return v * v; };
    auto calc = [&](int i, int j, int k, float z1, float z2, float dcol, float dnorm) {
        float colProb, depthProb;
        if (std::max(z1, z2) <= 0) {
            depthProb = 0;
            colProb = (float)(1 - std::exp((double)-sqrf(dcol / colSigma)));
        } else if (std::min(z1, z2) <= 0) {
            const int di[4] = {0, -1, 0, 1}, dj[4] = {-1, 0, 1, 0};
            const int dir = (z1 <= 0) ? (k + 2) % 4 : k;
            int i0 = (z1 <= 0) ? i : i + di[k], j0 = (z1 <= 0) ? j : j + dj[k];
            unsigned size = 0;
            while (j0 >= 0 && j0 < W && i0 >= 0 && i0 < H && depth[(size_t)i0 * W + j0] <= 0) {
                size++;
                i0 += di[dir];
                j0 += dj[dir];
            }
            const bool oob = (j0 < 0 || j0 >= W || i0 < 0 || i0 >= H);
            if (oob) depthProb = 0;
            else {
                const double a = std::min(1.0f, (float)size / 30);
                depthProb = (float)((1 - a) * .2 + a * 1);
            }
            colProb = (float)(1 - std::exp((double)-sqrf(dcol / colSigma)));
        } else {
            const float dz = (float)(std::fabs(z1 - z2) / stereo_error_ratio(std::min(z1, z2)));
            depthProb = (float)(1 - std::exp((double)-sqrf(dz / depthSigma)));
            colProb = 0;
        }
        const float normProb = (float)(1 - std::exp((double)-sqrf(dnorm / normSigma)));
        float v = std::max(depthProb, std::max(colProb, std::max(0.0f, normProb)));
        if (((i == 0 || i == H - 2) && k == 1) || ((j == 0 || j == W - 2) && k == 0)) v = 0;
        bp[((size_t)i * W + j) * 2 + k] = v;
    };
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            const size_t o = (size_t)i * W + j;
            if (j < W - 1) calc(i, j, 0, depth[o], depth[o + 1], colH[o + 1], norH[o + 1]);
            if (i < H - 1) calc(i, j, 1, depth[o], depth[o + W], colV[o + W], norV[o + W]);
        }
    // non-maximum suppression along each direction within the pixel's radius (:298-340)
    std::vector<float> bp2 = bp;
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            const int hw = radii[(size_t)i * W + j];
            int mi = -1;
            for (int k = std::max(0, i - hw); k <= std::min(H - 1, i + hw); k++)
                if (mi < 0 || bp[((size_t)k * W + j) * 2 + 1] > bp[((size_t)mi * W + j) * 2 + 1]) mi = k;
            if (mi != i) bp2[((size_t)i * W + j) * 2 + 1] = 0;
            mi = -1;
            for (int k = std::max(0, j - hw); k <= std::min(W - 1, j + hw); k++)
                if (mi < 0 || bp[((size_t)i * W + k) * 2] > bp[((size_t)i * W + mi) * 2]) mi = k;
            if (mi != j) bp2[((size_t)i * W + j) * 2] = 0;
        }
    std::memcpy(out, bp2.data(), sizeof(float) * N * 2);
}

/* ------------------------------------------------------------------------------------------ */
/* 2-D optical flow: Ce Liu's coarse-to-fine solver, the demo's flow type 1
 * (OpticalFlow::Coarse2FineFlow, src/opticalFlowMultiscale.cpp:4-146, CELIU variant:
 * OpticalFlow::SmoothFlowSOR, src/SmoothFlowSOR.cpp:8-247).  All FP64, like the reference, with
 * its lexicographic SOR order, so the result equals the reference's bit for bit. */

/* Image::dx / Image::dy without the advanced filter (Image.h:955-1019): forward differences;
 * the last column (dx) or row (dy) is 0. */
static void fwd_dx(const std::vector<double>& in, int W, int H, std::vector<double>& out)
{
    out.assign((size_t)W * H, 0.0);
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W - 1; j++) out[(size_t)i * W + j] = in[(size_t)i * W + j + 1] - in[(size_t)i * W + j];
}
static void fwd_dy(const std::vector<double>& in, int W, int H, std::vector<double>& out)
{
    out.assign((size_t)W * H, 0.0);
    for (int i = 0; i < H - 1; i++)
        for (int j = 0; j < W; j++) out[(size_t)i * W + j] = in[(size_t)(i + 1) * W + j] - in[(size_t)i * W + j];
}

/* getDxs (src/opticalFlowUtils.cpp:18-53): spatial derivatives of 0.4 im1 + 0.6 im2 with the
 * 5-tap {1,-8,0,8,-1}/12 filter (Image::dx/dy advanced), temporal derivative im2 - im1. */
static void get_dxs(const Img& im1, const Img& im2, Img& dx, Img& dy, Img& dt)
{
    Img m = im1;
    for (size_t z = 0; z < m.n(); z++) m.d[z] *= 0.4;
    for (size_t z = 0; z < m.n(); z++) m.d[z] += im2.d[z] * 0.6;
    double f[5] = {1, -8, 0, 8, -1};
    for (int i = 0; i < 5; i++) f[i] /= 12;
    hfilter(m, dx, f, 2);
    vfilter(m, dy, f, 2);
    dt.alloc(im1.w, im1.h, im1.c);
    for (size_t z = 0; z < dt.n(); z++) dt.d[z] = im2.d[z] - im1.d[z];
}

/* warpFL, bilinear (src/opticalFlowUtils.cpp:62-67; ImageProcessing::warpImage,
 * ImageProcessing.h:472-491): Im2 at (j + u, i + v), Im1 where that falls outside the image. */
static void warp_fl(const Img& Im1, const Img& Im2, const std::vector<double>& u, const std::vector<double>& v, Img& out)
{
    const int W = Im2.w, H = Im2.h, C = Im2.c;
    out.alloc(W, H, C);
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            const int o = i * W + j;
            const double x = j + u[o], y = i + v[o];
            if (x < 0 || x > W - 1 || y < 0 || y > H - 1)
                for (int k = 0; k < C; k++) out.d[(size_t)o * C + k] = Im1.d[(size_t)o * C + k];
            else
                bilinear_acc(Im2.data(), W, H, C, x, y, out.data() + (size_t)o * C);
        }
}

/* Laplacian with normalising weights (src/opticalFlowUtils.cpp:252-313) as SmoothFlowSOR calls
 * it (SmoothFlowSOR.cpp:144): with the 1-channel phi as the 2-channel weight image.  Channel k of
 * pixel (i, j) of a 1-channel image is element i * W + j + k (Image::operator(), Image.h:76), so
 * the "down" weight of (i, j) is phi at (i, j + 1). */
static void laplacian_phi(const std::vector<double>& in, const std::vector<double>& phi, int W, int H,
                          std::vector<double>& out)
{
    auto nw = [&](int i, int j, int k) { return phi[(size_t)i * W + j + k]; };
    out.assign((size_t)W * H, 0.0);
    std::vector<double> foo((size_t)W * H, 0.0);
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W - 1; j++) {
            const size_t o = (size_t)i * W + j;
            foo[o] = (in[o + 1] - in[o]) * nw(i, j, 0);
        }
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            const size_t o = (size_t)i * W + j;
            if (j < W - 1) out[o] -= foo[o];
            if (j > 0) out[o] += foo[o - 1];
        }
    std::fill(foo.begin(), foo.end(), 0.0);
    for (int i = 0; i < H - 1; i++)
        for (int j = 0; j < W; j++) {
            const size_t o = (size_t)i * W + j;
            foo[o] = (in[o + W] - in[o]) * nw(i, j, 1);
        }
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            const size_t o = (size_t)i * W + j;
            if (i < H - 1) out[o] -= foo[o];
            if (i > 0) out[o] += foo[o - W];
        }
    for (int i = 0; i < H; i++)
        for (int j = 0; j < W; j++) {
            const size_t o = (size_t)i * W + j;
            double norm = 0;
            int count = 0;
            if (j < W - 1) { norm += nw(i, j, 0); count++; }
            if (j > 0) { norm += nw(i, j - 1, 0); count++; }
            if (i < H - 1) { norm += nw(i, j, 1); count++; }
            if (i > 0) { norm += nw(i - 1, j, 1); count++; }
            if (std::fabs(norm) < 1e-5) out[o] = 0;
            else out[o] /= (norm / count);
        }
}

/* estLaplacianNoise (src/opticalFlowUtils.cpp:155-190): per channel, the mean of the absolute
 * differences in (0, 1e6), 0.001 when there are none.  The solve reads it only to reject a
 * value below 1e-20 (SmoothFlowSOR.cpp:113-117). */
static void est_laplacian_noise(const Img& a, const Img& b, std::vector<double>& para)
{
    const int C = a.c;
    para.assign(C, 0.0);
    std::vector<double> total(C, 0.0);
    for (size_t i = 0; i < (size_t)a.w * a.h; i++)
        for (int k = 0; k < C; k++) {
            const double t = std::fabs(a.d[i * C + k] - b.d[i * C + k]);
            if (t > 0 && t < 1000000) { para[k] += t; total[k]++; }
        }
    for (int k = 0; k < C; k++) para[k] = total[k] == 0 ? 0.001 : para[k] / total[k];
}

/* One SOR update of pixel (i, j) (SmoothFlowSOR.cpp:166-215): new values of the left and upper
 * neighbours come from (nu, nv), old values of the right and lower ones and of the pixel itself
 * from (ou, ov); writes (wu, wv)[o] and returns max(|du change|, |dv change|). */
struct Sor2dSys {
    int W, H;
    double alpha;
    const double *phi, *dxy, *dx2, *dy2, *dtdx, *dtdy;
};
static inline double sor2d_update(const Sor2dSys& q, int i, int j, const double* nu, const double* nv, const double* ou,
                                  const double* ov, double* wu, double* wv)
{
    const int W = q.W, H = q.H;
    const size_t o = (size_t)i * W + j;
    const double omega = 1.8;
    double sigmaU = 0, sigmaV = 0, weightSum = 0, w;
    if (j > 0) { w = q.phi[o - 1]; sigmaU += w * nu[o - 1]; sigmaV += w * nv[o - 1]; weightSum += w; }
    if (j < W - 1) { w = q.phi[o]; sigmaU += w * ou[o + 1]; sigmaV += w * ov[o + 1]; weightSum += w; }
    if (i > 0) { w = q.phi[o - W]; sigmaU += w * nu[o - W]; sigmaV += w * nv[o - W]; weightSum += w; }
    if (i < H - 1) { w = q.phi[o]; sigmaU += w * ou[o + W]; sigmaV += w * ov[o + W]; weightSum += w; }
    sigmaU *= -q.alpha;
    sigmaV *= -q.alpha;
    weightSum *= q.alpha;
    const double prevDU = ou[o], prevDV = ov[o];
    sigmaU += q.dxy[o] * prevDV;
    const double nDU = (1 - omega) * prevDU + omega / (q.dx2[o] + weightSum) * (q.dtdx[o] - sigmaU);
    sigmaV += q.dxy[o] * nDU;
    const double nDV = (1 - omega) * prevDV + omega / (q.dy2[o] + weightSum) * (q.dtdy[o] - sigmaV);
    wu[o] = nDU;
    wv[o] = nDV;
    return std::max(std::fabs(nDU - prevDU), std::fabs(nDV - prevDV));
}

/* The same SOR iterations in the order a device runs them, for checking that order on the CPU.
 * Each sweep walks the anti-diagonals d = i + j in turn: every pixel of one diagonal depends only
 * on the diagonal before it in this sweep and the one after it in the previous sweep, exactly as
 * in the lexicographic order.  Consecutive sweeps overlap, each starting two steps after the
 * previous one.  Sweep s writes ring slot s % D and reads the previous sweep's values from slot
 * (s - 1) % D; a sweep starts only after sweep s - D has finished without converging, so the slot
 * of the sweep that converges is never overwritten.  Returns the slot of the last sweep (the
 * first that converged, or sweep nSOR - 1). */
static int sor2d_wavefront(const Sor2dSys& q, int nSOR, int D, std::vector<std::vector<double>>& ru,
                           std::vector<std::vector<double>>& rv)
{
    const int W = q.W, H = q.H, ndiag = W + H - 1, lag = 2;
    const size_t N = (size_t)W * H;
    ru.assign(D, std::vector<double>(N, 0.0));
    rv.assign(D, std::vector<double>(N, 0.0));
    std::vector<long> start(nSOR, -1);
    std::vector<double> maxd(nSOR, 0.0);
    int done = -1;  // last sweep that finished
    int stop = -1;  // sweep that converged
    int next = 0;   // next sweep to start
    for (long t = 0; stop < 0 && done < nSOR - 1; t++) {
        if (next < nSOR && (next == 0 || t >= start[next - 1] + lag) && (next < D || done >= next - D)) {
            start[next] = t;
            next++;
        }
        for (int s = done + 1; s < next; s++) {
            const long d = t - start[s];
            if (d < 0 || d >= ndiag) continue;
            const int cur = s % D, prv = (s + D - 1) % D;
            for (long i = std::max(0L, d - (W - 1)); i <= std::min((long)H - 1, d); i++) {
                const double m = sor2d_update(q, (int)i, (int)(d - i), ru[cur].data(), rv[cur].data(), ru[prv].data(),
                                              rv[prv].data(), ru[cur].data(), rv[cur].data());
                maxd[s] = std::max(maxd[s], m);
            }
        }
        // the sweeps that finished at this step, in order: the first converged one ends the iterations
        while (done + 1 < next && t - start[done + 1] == ndiag - 1) {
            done++;
            if (maxd[done] < 1e-5) { stop = done; break; }
        }
    }
    return (stop >= 0 ? stop : nSOR - 1) % D;
}

/* OpticalFlow::SmoothFlowSOR (src/SmoothFlowSOR.cpp:8-247), Laplacian noise model, bilinear warps.
 * ring > 0 runs the SOR iterations in the device order of sor2d_wavefront with a ring of that
 * many slots; 0 runs them in the reference's lexicographic order. */
static void smooth_flow_sor(const Img& Im1, const Img& Im2, Img& warpIm2, std::vector<double>& u,
                            std::vector<double>& v, double alpha, int nOuter, int nInner, int nSOR,
                            std::vector<double>& lap, int ring = 0)
{
    const int W = Im1.w, H = Im1.h, C = Im1.c;
    const size_t N = (size_t)W * H;
    const double eps_phi = std::pow(0.001, 2), eps_psi = std::pow(0.001, 2);
    Img imdx, imdy, imdt;
    std::vector<double> du(N), dv(N), uu, vv, ux, uy, vx, vy, phi(N), psi(N * C);
    std::vector<double> dxy(N), dx2(N), dy2(N), dtdx(N), dtdy(N), foo1, foo2;
    for (int count = 0; count < nOuter; count++) {
        get_dxs(Im1, warpIm2, imdx, imdy, imdt);
        std::fill(du.begin(), du.end(), 0.0);
        std::fill(dv.begin(), dv.end(), 0.0);
        for (int hh = 0; hh < nInner; hh++) {
            uu = u;
            vv = v;
            if (hh > 0)
                for (size_t i = 0; i < N; i++) { uu[i] = u[i] + du[i]; vv[i] = v[i] + dv[i]; }
            fwd_dx(uu, W, H, ux);
            fwd_dy(uu, W, H, uy);
            fwd_dx(vv, W, H, vx);
            fwd_dy(vv, W, H, vy);
            for (size_t i = 0; i < N; i++) {
                const double t = ux[i] * ux[i] + uy[i] * uy[i] + vx[i] * vx[i] + vy[i] * vy[i];
                phi[i] = 0.5 / std::sqrt(t + eps_phi);
            }
            for (size_t i = 0; i < N; i++)
                for (int k = 0; k < C; k++) {
                    const size_t o = i * C + k;
                    double t = imdt.d[o] + imdx.d[o] * du[i] + imdy.d[o] * dv[i];
                    t *= t;
                    if (lap[k] < 1E-20) throw std::runtime_error("bad lap para");
                    psi[o] = 1 / (2 * std::sqrt(t + eps_psi));
                }
            // Image::Multiply (Image.h:1697-1710) then Image::collapse, channel mean (Image.h:1480-1516)
            for (size_t i = 0; i < N; i++) {
                double sxy = 0, sx2 = 0, sy2 = 0, stx = 0, sty = 0;
                for (int k = 0; k < C; k++) {
                    const size_t o = i * C + k;
                    const double a = imdx.d[o], b = imdy.d[o], c = imdt.d[o];
                    if (C > 1) {
                        sxy += psi[o] * a * b; sx2 += psi[o] * a * a; sy2 += psi[o] * b * b;
                        stx += psi[o] * a * c; sty += psi[o] * b * c;
                    } else {
                        sxy = psi[o] * a * b; sx2 = psi[o] * a * a; sy2 = psi[o] * b * b;
                        stx = psi[o] * a * c; sty = psi[o] * b * c;
                    }
                }
                if (C > 1) { sxy /= C; sx2 /= C; sy2 /= C; stx /= C; sty /= C; }
                dxy[i] = sxy; dx2[i] = sx2; dy2[i] = sy2; dtdx[i] = stx; dtdy[i] = sty;
            }
            laplacian_phi(u, phi, W, H, foo1);
            laplacian_phi(v, phi, W, H, foo2);
            for (size_t i = 0; i < N; i++) {
                dtdx[i] = -dtdx[i] - alpha * foo1[i];
                dtdy[i] = -dtdy[i] - alpha * foo2[i];
            }
            std::fill(du.begin(), du.end(), 0.0);
            std::fill(dv.begin(), dv.end(), 0.0);
            if (ring > 0) {
                const Sor2dSys q{W, H, alpha, phi.data(), dxy.data(), dx2.data(), dy2.data(), dtdx.data(), dtdy.data()};
                std::vector<std::vector<double>> ru, rv;
                const int slot = sor2d_wavefront(q, nSOR, ring, ru, rv);
                du = ru[slot];
                dv = rv[slot];
                continue;
            }
            const double omega = 1.8;
            bool converged = false;
            for (int k = 0; k < nSOR && !converged; k++) {
                double maxDiff = 0;
                for (int i = 0; i < H; i++)
                    for (int j = 0; j < W; j++) {
                        const size_t o = (size_t)i * W + j;
                        double sigmaU = 0, sigmaV = 0, weightSum = 0, w;
                        if (j > 0) { w = phi[o - 1]; sigmaU += w * du[o - 1]; sigmaV += w * dv[o - 1]; weightSum += w; }
                        if (j < W - 1) { w = phi[o]; sigmaU += w * du[o + 1]; sigmaV += w * dv[o + 1]; weightSum += w; }
                        if (i > 0) { w = phi[o - W]; sigmaU += w * du[o - W]; sigmaV += w * dv[o - W]; weightSum += w; }
                        if (i < H - 1) { w = phi[o]; sigmaU += w * du[o + W]; sigmaV += w * dv[o + W]; weightSum += w; }
                        sigmaU *= -alpha;
                        sigmaV *= -alpha;
                        weightSum *= alpha;
                        const double prevDU = du[o], prevDV = dv[o];
                        sigmaU += dxy[o] * dv[o];
                        du[o] = (1 - omega) * du[o] + omega / (dx2[o] + weightSum) * (dtdx[o] - sigmaU);
                        sigmaV += dxy[o] * du[o];
                        dv[o] = (1 - omega) * dv[o] + omega / (dy2[o] + weightSum) * (dtdy[o] - sigmaV);
                        maxDiff = std::max(maxDiff, std::max(std::fabs(du[o] - prevDU), std::fabs(dv[o] - prevDV)));
                    }
                converged = maxDiff < 1e-5;
            }
        }
        for (size_t i = 0; i < N; i++) { u[i] += du[i]; v[i] += dv[i]; }
        warp_fl(Im1, Im2, u, v, warpIm2);
        est_laplacian_noise(Im1, warpIm2, lap);
    }
}

/* OpticalFlow::Coarse2FineFlow (src/opticalFlowMultiscale.cpp:4-146) on two 3-channel images,
 * CELIU variant, no depth maps: per level, coarsest first, the 5-channel features, the flow
 * resized from the coarser level and scaled by 1 / ratio, the warp, SmoothFlowSOR with
 * nOuter + k outer and nSOR + 3 k SOR iterations at level k. */
void coarse2fine_flow(const Img& im1, const Img& im2, double alpha, double ratio, int min_width, int nOuter, int nInner,
                      int nSOR, std::vector<double>& u, std::vector<double>& v, int ring = 0)
{
    std::vector<Img> p1, p2;
    build_pyramid(im1, ratio, min_width, p1);
    build_pyramid(im2, ratio, min_width, p2);
    std::vector<double> lap(im1.c + 2, 0.02);
    Img warp;
    const int L = (int)p1.size();
    for (int k = L - 1; k >= 0; k--) {
        Img f1, f2;
        im2feature(p1[k], f1);
        im2feature(p2[k], f2);
        const int W = p1[k].w, H = p1[k].h;
        if (k == L - 1) {
            u.assign((size_t)W * H, 0.0);
            v.assign((size_t)W * H, 0.0);
            warp = f2;
        } else {
            Img uin, vin, uo, vo;
            uin.w = vin.w = p1[k + 1].w; uin.h = vin.h = p1[k + 1].h; uin.c = vin.c = 1;
            uin.d = u; vin.d = v;
            resize_dims(uin, uo, W, H);
            resize_dims(vin, vo, W, H);
            const double s = 1 / ratio;
            u = uo.d; v = vo.d;
            for (auto& x : u) x *= s;
            for (auto& x : v) x *= s;
            warp_fl(f1, f2, u, v, warp);
        }
        smooth_flow_sor(f1, f2, warp, u, v, alpha, nOuter + k, nInner, nSOR + k * 3, lap, ring);
    }
}

static thread_local std::string g_err;

extern "C" {

const char* sfo_last_error(void) { return g_err.c_str(); }

int sfo_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int sfo_pyramid_levels(int width, double ratio, int min_width)
{
    try { return pyramid_levels(width, ratio, min_width); }
    catch (const std::exception& e) { g_err = e.what(); return -1; }
}

/* All levels of GaussianPyramid::ConstructPyramid, concatenated (level 0 first).
 * dims (2 * nLevels ints) receives the level sizes; returns the level count. */
int sfo_build_pyramid(const double* img, int W, int H, int C, double ratio, int min_width, double* out, int* dims)
{
    Img b; b.alloc(W, H, C);
    std::memcpy(b.data(), img, sizeof(double) * b.n());
    std::vector<Img> lev;
    try { build_pyramid(b, ratio, min_width, lev); }
    catch (const std::exception& e) { g_err = e.what(); return -1; }
    size_t off = 0;
    for (size_t i = 0; i < lev.size(); i++) {
        if (dims) { dims[2 * i] = lev[i].w; dims[2 * i + 1] = lev[i].h; }
        if (out) std::memcpy(out + off, lev[i].data(), sizeof(double) * lev[i].n());
        off += lev[i].n();
    }
    return (int)lev.size();
}

void sfo_gaussian_smooth(const double* img, int W, int H, int C, double sigma, int fsize, double* out)
{
    Img b; b.alloc(W, H, C);
    std::memcpy(b.data(), img, sizeof(double) * b.n());
    Img o;
    gaussian_smooth(b, o, sigma, fsize);
    std::memcpy(out, o.data(), sizeof(double) * o.n());
}

void sfo_resize_dims(const double* img, int W, int H, int C, int DW, int DH, double* out)
{
    Img b; b.alloc(W, H, C);
    std::memcpy(b.data(), img, sizeof(double) * b.n());
    Img o;
    resize_dims(b, o, DW, DH);
    std::memcpy(out, o.data(), sizeof(double) * o.n());
}

void sfo_im2feature(const double* bgr01, int W, int H, double* feat5)
{
    Img b; b.alloc(W, H, 3);
    std::memcpy(b.data(), bgr01, sizeof(double) * b.n());
    Img f;
    im2feature(b, f);
    std::memcpy(feat5, f.data(), sizeof(double) * f.n());
}

void sfo_set_level_solver(void* fn) { g_level_solver = (LevelSolverFn)fn; }

int sfo_set_fill_order(int order)
{
    const int old = g_fill_order;
    g_fill_order = order;
    return old;
}

int sfo_median_fill_rounds(double* depth, int W, int H, int* rounds)
{
    try { *rounds = median_fill_rounds(depth, W, H); return 0; }
    catch (const std::exception& e) { g_err = e.what(); return -1; }
}

int sfo_median_fill(double* depth, int W, int H)
{
    try { median_fill(depth, W, H, 1); return 0; }
    catch (const std::exception& e) { g_err = e.what(); return -1; }
}

void sfo_depth_sigma(const float* depth, int W, int H, int max_dist, float* sigma) { depth_sigma(depth, W, H, max_dist, sigma); }

void sfo_warp_cpu(const double* feat1, const double* d1, const double* feat2, const double* d2, int W, int H, int C,
                  const double* u, const double* v, const double* w, double* wI2, double* wD2)
{
    Img f1, f2, a, b, oI, oD;
    f1.alloc(W, H, C); f2.alloc(W, H, C); a.alloc(W, H, 1); b.alloc(W, H, 1);
    std::memcpy(f1.data(), feat1, sizeof(double) * f1.n());
    std::memcpy(f2.data(), feat2, sizeof(double) * f2.n());
    std::memcpy(a.data(), d1, sizeof(double) * a.n());
    std::memcpy(b.data(), d2, sizeof(double) * b.n());
    warp_cpu(f1, a, f2, b, oI, oD, u, v, w);
    std::memcpy(wI2, oI.data(), sizeof(double) * oI.n());
    std::memcpy(wD2, oD.data(), sizeof(double) * oD.n());
}

void sfo_depth_mag_weights(const double* depthk, int Wk, int Hk, const rgbdflow_camera_params* camFull, double* out)
{
    Img d; d.alloc(Wk, Hk, 1);
    std::memcpy(d.data(), depthk, sizeof(double) * d.n());
    std::vector<double> m;
    depth_mag_weights(d, *camFull, m);
    std::memcpy(out, m.data(), sizeof(double) * m.size());
}

void sfo_reg_weights(const double* depth, int W, int H, int type, double* out)
{
    std::vector<double> r;
    reg_weights(W, H, depth, type, r);
    std::memcpy(out, r.data(), sizeof(double) * r.size());
}

/* One linearisation from a given state, as the 8 SoA planes of the reference's A (.cu:543):
 * A[(plane * W*H + pixel) * 3 + var] -> out[plane][pixel*3 + var], doubles. */
int sfo_linearize(int fp64, const double* Im1, const double* dm1, const double* Im2, const double* dm2,
                  const double* wI2, const double* wD2, const double* u3, const double* du3,
                  int W, int H, int C, double colorW, const double* ddw, double alpha, const double* dsw,
                  double gamma, const double* mag, const double* regw, const rgbdflow_params* prm, double* Aout)
{
    rgbdflow_params p;
    if (prm) p = *prm; else rgbdflow_params_default_oracle(&p);
    SolverIn in;
    in.W = W; in.H = H; in.C = C; in.f_level = 1;
    in.Im1 = Im1; in.dm1 = dm1; in.Im2 = Im2; in.dm2 = dm2;
    in.colorW = colorW; in.alpha = alpha; in.gamma = gamma;
    in.ddw = ddw; in.dsw = dsw; in.mag = mag; in.regw = regw;
    const size_t N = (size_t)W * H;
    Img a, b; a.alloc(W, H, C); b.alloc(W, H, 1);
    std::memcpy(a.data(), wI2, sizeof(double) * a.n());
    std::memcpy(b.data(), wD2, sizeof(double) * b.n());
    std::vector<double> u(u3, u3 + N * 3), imdx, imdy, imdt, dmdx, dmdy, dmdt;
    img_derivs(W, H, C, Im1, wI2, 0, false, imdx, imdy, imdt);
    img_derivs(W, H, 1, dm1, wD2, p.max_depth_grad, true, dmdx, dmdy, dmdt);
    auto go = [&](auto tag) {
        constexpr bool D = decltype(tag)::value;
        typedef typename P<D>::F F;
        std::vector<F> du(N * 3), q(N), ddwF(N), dswF(N), magF(N), regF(N * 2), A(N * 24, (F)0);
        for (size_t z = 0; z < N * 3; z++) du[z] = (F)du3[z];
        for (size_t l = 0; l < N; l++) {
            ddwF[l] = (F)ddw[l]; dswF[l] = (F)dsw[l]; magF[l] = (F)mag[l];
            regF[2 * l] = (F)regw[2 * l]; regF[2 * l + 1] = (F)regw[2 * l + 1];
            q[l] = (dm1[l] + u[l * 3 + 2] < dm2[l] + p.occ_margin * (double)sqc<D>(dm1[l])) ? (F)1 : (F)p.occ_penalty;
        }
        linearize<D>(in, p, u, du, a, b, q, ddwF, dswF, magF, regF, imdx, imdy, imdt, dmdx, dmdy, dmdt, A);
        for (size_t z = 0; z < N * 24; z++) Aout[z] = (double)A[z];
    };
    if (fp64) go(std::true_type()); else go(std::false_type());
    return 0;
}

/* nIter red-black SOR iterations on a given system (8 SoA planes, doubles rounded to the
 * variant's type), starting from x (in/out, W*H*3). */
void sfo_sor(int fp64, const double* A, double* x, int W, int H, int nIter, double omega, double step)
{
    const size_t n = (size_t)W * H * 3;
    auto go = [&](auto tag) {
        constexpr bool D = decltype(tag)::value;
        typedef typename P<D>::F F;
        std::vector<F> a(n * 8), xx(n);
        for (size_t z = 0; z < n * 8; z++) a[z] = (F)A[z];
        for (size_t z = 0; z < n; z++) xx[z] = (F)x[z];
        for (int it = 0; it < nIter; it++) {
            sor_sweep<D>(W, H, a, xx, 0, (F)omega, (F)step);
            sor_sweep<D>(W, H, a, xx, 1, (F)omega, (F)step);
        }
        for (size_t z = 0; z < n; z++) x[z] = (double)xx[z];
    };
    if (fp64) go(std::true_type()); else go(std::false_type());
}

static void trace_to_stats(const Trace& t, rgbdflow_stats* s)
{
    if (!s) return;
    std::memset(s, 0, sizeof(*s));
    s->n_levels = t.n_levels;
    for (int k = 0; k < t.n_levels && k < RGBDFLOW_MAX_LEVELS; k++) {
        s->level_w[k] = t.w[k]; s->level_h[k] = t.h[k];
        s->outer_iters[k] = t.lev[k].outer;
        for (int o = 0; o < RGBDFLOW_MAX_OUTER; o++) {
            s->sor_iters[k][o] = t.lev[k].sor[o];
            s->outer_stat[k][o] = t.lev[k].stat[o];
            s->sor_maxdiff[k][o] = t.lev[k].maxdiff[o];
        }
    }
}

/* The per-level seam sceneFlowSingleScale (OpticalFlow.h:17-22) on raw DImage planes. */
int sfo_single_scale(int fp64, float f_level, const double* Im1, const double* dm1, const double* Im2, const double* dm2,
                     double* warpIm2, double* warpDm2, double* u, double* v, double* w, int W, int H, int C,
                     double colorW, const double* ddw, double alpha, const double* dsw, double gamma,
                     const double* mag, const double* regw, int nOuter, int nInner, int nSOR, int allowEarly,
                     const rgbdflow_params* prm, rgbdflow_stats* stats)
{
    try {
        rgbdflow_params p;
        if (prm) p = *prm; else rgbdflow_params_default_oracle(&p);
        SolverIn in;
        in.W = W; in.H = H; in.C = C; in.f_level = f_level;
        in.Im1 = Im1; in.dm1 = dm1; in.Im2 = Im2; in.dm2 = dm2;
        in.colorW = colorW; in.alpha = alpha; in.gamma = gamma;
        in.ddw = ddw; in.dsw = dsw; in.mag = mag; in.regw = regw;
        in.nOuter = nOuter; in.nInner = nInner; in.nSOR = nSOR; in.allowEarly = allowEarly;
        Img a, b; a.alloc(W, H, C); b.alloc(W, H, 1);
        std::memcpy(a.data(), warpIm2, sizeof(double) * a.n());
        std::memcpy(b.data(), warpDm2, sizeof(double) * b.n());
        Trace t; t.n_levels = 1; t.w[0] = W; t.h[0] = H;
        if (fp64) single_scale<true>(in, p, p.fixed_schedule, a, b, u, v, w, &t.lev[0]);
        else single_scale<false>(in, p, p.fixed_schedule, a, b, u, v, w, &t.lev[0]);
        std::memcpy(warpIm2, a.data(), sizeof(double) * a.n());
        std::memcpy(warpDm2, b.data(), sizeof(double) * b.n());
        trace_to_stats(t, stats);
        return 0;
    } catch (const std::exception& e) { g_err = e.what(); return -1; }
}

/* runFlowTwoFramesSceneFlowExperiments (runFlowTwoFrames.cpp:109-121) -> ceLiuSceneFlow
 * (ceLiuOpticalFlow.cpp:190-215), raw buffers: BGR8 and float metres in, (u,v,w) float out. */
int sfo_scene_flow_two_frames(int fp64, const rgbdflow_camera_params* camFull, const uint8_t* bgr1, const float* depth1,
                              const uint8_t* bgr2, const float* depth2, int W, int H, const rgbdflow_params* prm,
                              const float* est_flow, float* flow_out, rgbdflow_stats* stats)
{
    try {
        const rgbdflow_camera_params cam = resize_cam(*camFull, W);
        std::vector<float> s1((size_t)W * H);
        depth_sigma(depth1, W, H, prm->depth_boundary_dist, s1.data());
        Img I1, I2, D1, D2;
        I1.alloc(W, H, 3); I2.alloc(W, H, 3); D1.alloc(W, H, 1); D2.alloc(W, H, 1);
        for (size_t z = 0; z < (size_t)W * H * 3; z++) { I1.d[z] = bgr1[z] / 255.0; I2.d[z] = bgr2[z] / 255.0; }
        for (size_t z = 0; z < (size_t)W * H; z++) { D1.d[z] = depth1[z]; D2.d[z] = depth2[z]; }
        std::vector<double> est;
        if (est_flow) est.assign(est_flow, est_flow + (size_t)W * H * 3);
        Img u, v, w;
        Trace t;
        if (fp64) multiscale<true>(cam, *prm, I1, D1, I2, D2, s1.data(), est_flow ? est.data() : nullptr, u, v, w, &t);
        else multiscale<false>(cam, *prm, I1, D1, I2, D2, s1.data(), est_flow ? est.data() : nullptr, u, v, w, &t);
        for (size_t l = 0; l < (size_t)W * H; l++) {
            flow_out[l * 3] = (float)u.d[l]; flow_out[l * 3 + 1] = (float)v.d[l]; flow_out[l * 3 + 2] = (float)w.d[l];
        }
        trace_to_stats(t, stats);
        return 0;
    } catch (const std::exception& e) { g_err = e.what(); return -1; }
}

/* recursiveMedianFilterSmallInvalidRegionsUsingColor in place on a W x H depth map, guided by
 * the W*H*3 colour image (doubles in [0, 1]). */
int sfo_fill_small_regions_color(double* depth, const double* col, int W, int H, int max_region)
{
    try {
        Img d, c;
        d.alloc(W, H, 1);
        c.alloc(W, H, 3);
        std::memcpy(d.data(), depth, sizeof(double) * (size_t)W * H);
        std::memcpy(c.data(), col, sizeof(double) * (size_t)W * H * 3);
        fill_small_regions_color(d, c, (unsigned)max_region);
        std::memcpy(depth, d.data(), sizeof(double) * (size_t)W * H);
        return 0;
    } catch (const std::exception& e) { g_err = e.what(); return -1; }
}

/* computeHeuristicPb of one level: img W*H*3 doubles in [0, 1] (BGR), depth W*H doubles;
 * out: W*H*2 floats. */
void sfo_heuristic_pb(const double* img, const double* depth, int W, int H, float* out)
{
    heuristic_pb(img, depth, W, H, out);
}

/* DepthMapPyramid of a W x H depth map (doubles); out: the levels concatenated (NULL: sizes
 * only), dims: 2 ints per level.  Returns the level count. */
int sfo_depth_map_pyramid(const double* depth, int W, int H, double ratio, int min_width, double* out, int* dims)
{
    Img d;
    d.alloc(W, H, 1);
    std::memcpy(d.data(), depth, sizeof(double) * (size_t)W * H);
    std::vector<Img> lev;
    try { depth_map_pyramid(d, ratio, min_width, lev); }
    catch (const std::exception& e) { g_err = e.what(); return -1; }
    size_t off = 0;
    for (size_t i = 0; i < lev.size(); i++) {
        if (dims) { dims[2 * i] = lev[i].w; dims[2 * i + 1] = lev[i].h; }
        if (out) std::memcpy(out + off, lev[i].data(), sizeof(double) * lev[i].n());
        off += lev[i].n();
    }
    return (int)lev.size();
}

/* 2-D optical flow of two BGR8 images (the demo's flow type 1, runFlowTwoFramesCeLiu,
 * src/runFlowTwoFrames.cpp:30-45): colour / 255 as cv2liuBGR (src/ceLiuOpticalFlow.cpp:19-37),
 * then Coarse2FineFlow with the given parameters.  u, v: W*H doubles. */
int sfo_optical_flow_2d_ring(const uint8_t* bgr1, const uint8_t* bgr2, int W, int H, double alpha, double ratio,
                             int min_width, int n_outer, int n_inner, int n_sor, int ring, double* u, double* v);
int sfo_optical_flow_2d(const uint8_t* bgr1, const uint8_t* bgr2, int W, int H, double alpha, double ratio,
                        int min_width, int n_outer, int n_inner, int n_sor, double* u, double* v)
{
    return sfo_optical_flow_2d_ring(bgr1, bgr2, W, H, alpha, ratio, min_width, n_outer, n_inner, n_sor, 0, u, v);
}

/* sfo_optical_flow_2d with the SOR iterations in the device order of sor2d_wavefront (ring > 0
 * slots), or the reference's lexicographic order (ring 0). */
int sfo_optical_flow_2d_ring(const uint8_t* bgr1, const uint8_t* bgr2, int W, int H, double alpha, double ratio,
                             int min_width, int n_outer, int n_inner, int n_sor, int ring, double* u, double* v)
{
    try {
        Img I1, I2;
        I1.alloc(W, H, 3);
        I2.alloc(W, H, 3);
        for (size_t z = 0; z < (size_t)W * H * 3; z++) { I1.d[z] = bgr1[z] / 255.0; I2.d[z] = bgr2[z] / 255.0; }
        std::vector<double> uu, vv;
        coarse2fine_flow(I1, I2, alpha, ratio, min_width, n_outer, n_inner, n_sor, uu, vv, ring);
        std::memcpy(u, uu.data(), sizeof(double) * uu.size());
        std::memcpy(v, vv.data(), sizeof(double) * vv.size());
        return 0;
    } catch (const std::exception& e) { g_err = e.what(); return -1; }
}

} // extern "C"
