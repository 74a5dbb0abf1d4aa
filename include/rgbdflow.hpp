/*
 * rgbdflow.hpp — C++ adapter over the C ABI (rgbdflow.h) with the reference's call shapes.
 *
 * A caller of eherbst/rgbd-flow keeps its code: the functions below take the same arguments as
 *   OpticalFlow::sceneFlowMultiscale   include/celiu_flow/OpticalFlow.h:133
 *   OpticalFlow::sceneFlowWithInit     include/celiu_flow/OpticalFlow.h:145
 *   sceneFlowSingleScale               include/celiu_flow/OpticalFlow.h:17-22
 *   runFlowTwoFramesSceneFlowExperiments  include/rgbd_flow/runFlowTwoFrames.h:49-51
 * with three substitutions: a Context comes first (the device, its workspaces and graphs);
 * cv::Mat arguments become pointer + size (OpenCV is not a dependency); the optional output
 * directory is dropped (the solve writes no debug images).  Images are any type with the Ce Liu
 * Image<T> accessors (width(), height(), nchannels(), data(), allocate(w, h, c);
 * include/celiu_flow/Image.h:45,85-89), so the reference's own DImage passes straight through.
 *
 * Errors are exceptions, as in the reference (ASSERT_ALWAYS throws std::runtime_error,
 * include/rgbd_util/assert.h:57,106): rgbdflow::Error derives from std::runtime_error and
 * carries the C status code.
 */
#ifndef RGBDFLOW_HPP
#define RGBDFLOW_HPP

#include <stdexcept>
#include <string>
#include <vector>

#include "rgbdflow.h"

namespace rgbdflow {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

inline const char* status_name(int s)
{
    switch (s) {
    case RGBDFLOW_OK: return "OK";
    case RGBDFLOW_ERR_INVALID_ARG: return "INVALID_ARG";
    case RGBDFLOW_ERR_UNSUPPORTED: return "UNSUPPORTED";
    case RGBDFLOW_ERR_CUDA: return "CUDA";
    case RGBDFLOW_ERR_BUDGET: return "BUDGET";
    case RGBDFLOW_ERR_TIMEOUT: return "TIMEOUT";
    case RGBDFLOW_ERR_NO_DEVICE: return "NO_DEVICE";
    case RGBDFLOW_ERR_BUSY: return "BUSY";
    default: return "INTERNAL";
    }
}

/* The regularisation types of OpticalFlow::sceneFlowRegularizationType (OpticalFlow.h:99-104). */
enum class sceneFlowRegularizationType { ISOTROPIC = RGBDFLOW_REG_ISOTROPIC, LETOUZEY = RGBDFLOW_REG_LETOUZEY, HPB = RGBDFLOW_REG_HPB };

/* OpticalFlow::sceneFlowParams (OpticalFlow.h:105-129), field names kept.  The constructor sets
 * the reference's defaults (OpticalFlow.h:107-109).  depthSigma1 replaces the cv::Mat_<float>
 * of the same name: W*H standard deviations of frame 1's depth, owned by the caller. */
struct sceneFlowParams {
    sceneFlowRegularizationType regularizationType = sceneFlowRegularizationType::HPB;
    rgbdflow_camera_params camParams{};
    double colorDataWeight = 1;
    double depthVsColorDataWeight = 1;
    double alpha = 0;
    double gamma = 0;
    const float* depthSigma1 = nullptr;
    double pyramidRatio = .75;
    int minWidth = 20;
    int nOuterFPIterations = 7, nInnerFPIterations = 1, nSORIterations = 30;
    /* everything else of rgbdflow_params (solver constants, storage type, schedule mode) */
    rgbdflow_params extra = defaults();

    static rgbdflow_params defaults()
    {
        rgbdflow_params p;
        rgbdflow_params_default(&p);
        return p;
    }
    /* The C parameter block these fields describe. */
    rgbdflow_params to_c() const
    {
        rgbdflow_params p = extra;
        p.regularization = (int)regularizationType;
        p.color_data_weight = colorDataWeight;
        p.depth_vs_color_data_weight = depthVsColorDataWeight;
        p.alpha = alpha;
        p.gamma = gamma;
        p.pyramid_ratio = pyramidRatio;
        p.min_width = minWidth;
        p.n_outer = nOuterFPIterations;
        p.n_inner = nInnerFPIterations;
        p.n_sor = nSORIterations;
        return p;
    }
};

/* Owns one rgbdflow_ctx.  One per host thread, as the C context. */
class Context {
public:
    explicit Context(int device = 0, size_t hbm_budget_bytes = 0)
    {
        const int s = rgbdflow_ctx_create(device, hbm_budget_bytes, &c_);
        if (s != RGBDFLOW_OK) throw Error(s, std::string("rgbdflow_ctx_create: ") + status_name(s));
    }
    ~Context() { if (c_) rgbdflow_ctx_destroy(c_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    rgbdflow_ctx* get() const { return c_; }
    void check(int s, const char* what) const
    {
        if (s != RGBDFLOW_OK) throw Error(s, std::string(what) + ": " + status_name(s) + ": " + rgbdflow_last_error(c_));
    }

private:
    rgbdflow_ctx* c_ = nullptr;
};

namespace detail {
template <class Image> void require(bool ok, const char* what)
{
    if (!ok) throw Error(RGBDFLOW_ERR_INVALID_ARG, what);
}
template <class Image> void check_pair(const Image& Im1, const Image& dm1, const Image& Im2, const Image& dm2)
{
    const int W = Im1.width(), H = Im1.height();
    require<Image>(Im1.nchannels() == 3 && Im2.nchannels() == 3, "colour images must have 3 channels");
    require<Image>(Im2.width() == W && Im2.height() == H, "image sizes differ");
    require<Image>(dm1.width() == W && dm1.height() == H && dm1.nchannels() == 1, "depth 1 size");
    require<Image>(dm2.width() == W && dm2.height() == H && dm2.nchannels() == 1, "depth 2 size");
}
}  // namespace detail

/* OpticalFlow::sceneFlowMultiscale (src/sceneFlowMultiscale.cpp:30-201): Im1/Im2 3-channel in
 * [0,1] (the reference keeps BGR), dm1/dm2 metres.  u, v, w are (re)allocated to W x H. */
template <class Image>
void sceneFlowMultiscale(Context& ctx, const Image& Im1, const Image& dm1, const Image& Im2, const Image& dm2,
                         const sceneFlowParams& params, Image& u, Image& v, Image& w, rgbdflow_stats* stats = nullptr)
{
    detail::check_pair(Im1, dm1, Im2, dm2);
    const int W = Im1.width(), H = Im1.height();
    u.allocate(W, H, 1); v.allocate(W, H, 1); w.allocate(W, H, 1);
    const rgbdflow_params p = params.to_c();
    ctx.check(rgbdflow_scene_flow_multiscale(ctx.get(), &params.camParams, Im1.data(), dm1.data(), Im2.data(),
                                             dm2.data(), params.depthSigma1, W, H, &p, u.data(), v.data(), w.data(),
                                             stats),
              "sceneFlowMultiscale");
}

/* OpticalFlow::sceneFlowWithInit (src/sceneFlowWithInit.cpp:7-81): estFlow is 3-channel
 * (u px, v px, w m); one full-resolution level. */
template <class Image>
void sceneFlowWithInit(Context& ctx, const Image& Im1, const Image& dm1, const Image& Im2, const Image& dm2,
                       const sceneFlowParams& params, const Image& estFlow, Image& u, Image& v, Image& w,
                       rgbdflow_stats* stats = nullptr)
{
    detail::check_pair(Im1, dm1, Im2, dm2);
    const int W = Im1.width(), H = Im1.height();
    detail::require<Image>(estFlow.width() == W && estFlow.height() == H && estFlow.nchannels() == 3,
                           "estFlow must be W x H x 3");
    u.allocate(W, H, 1); v.allocate(W, H, 1); w.allocate(W, H, 1);
    const size_t N = (size_t)W * H;
    for (size_t i = 0; i < N; i++) {
        u.data()[i] = estFlow.data()[3 * i];
        v.data()[i] = estFlow.data()[3 * i + 1];
        w.data()[i] = estFlow.data()[3 * i + 2];
    }
    const rgbdflow_params p = params.to_c();
    ctx.check(rgbdflow_scene_flow_with_init(ctx.get(), &params.camParams, Im1.data(), dm1.data(), Im2.data(),
                                            dm2.data(), params.depthSigma1, W, H, &p, u.data(), v.data(), w.data(),
                                            stats),
              "sceneFlowWithInit");
}

/* sceneFlowSingleScale (src/sceneFlowSingleScaleJacobiCUDA.cu:660-969): the per-level seam.
 * Im1/Im2/warpIm2 carry the level's features (5 channels for RGB_WITH_GRADIENT); warpIm2,
 * warpDm2, u, v, w are in/out; regularizationWeights has 2 channels (right, down). */
template <class Image>
void sceneFlowSingleScale(Context& ctx, const rgbdflow_camera_params& camParams, const Image& Im1, const Image& dm1,
                          const Image& Im2, const Image& dm2, Image& warpIm2, Image& warpDm2, Image& u, Image& v,
                          Image& w, const double colorDataTermWeight, const Image& depthDataTermWeights,
                          const double alpha, const Image& depthSmoothnessTermWeights, const double gamma,
                          const Image& depthMagTermWeights, const Image& regularizationWeights, int nOuterFPIterations,
                          int nInnerFPIterations, int nSORIterations, const bool allowEarlyTermination,
                          const rgbdflow_params* constants = nullptr, rgbdflow_stats* stats = nullptr)
{
    const int W = Im1.width(), H = Im1.height(), C = Im1.nchannels();
    detail::require<Image>(Im2.width() == W && Im2.height() == H && Im2.nchannels() == C, "Im2 size");
    detail::require<Image>(warpIm2.width() == W && warpIm2.height() == H && warpIm2.nchannels() == C, "warpIm2 size");
    detail::require<Image>(regularizationWeights.nchannels() == 2, "regularizationWeights must have 2 channels");
    ctx.check(rgbdflow_scene_flow_single_scale(
                  ctx.get(), &camParams, Im1.data(), dm1.data(), Im2.data(), dm2.data(), warpIm2.data(), warpDm2.data(),
                  u.data(), v.data(), w.data(), W, H, C, colorDataTermWeight, depthDataTermWeights.data(), alpha,
                  depthSmoothnessTermWeights.data(), gamma, depthMagTermWeights.data(), regularizationWeights.data(),
                  nOuterFPIterations, nInnerFPIterations, nSORIterations, allowEarlyTermination ? 1 : 0, constants, stats),
              "sceneFlowSingleScale");
}

/* runFlowTwoFramesSceneFlowExperiments (src/runFlowTwoFrames.cpp:109-121) with cv::Mat replaced
 * by buffers: prevImg/curImg W*H*3 BGR8, prevDepth/curDepth W*H metres (0 = invalid), estFlow
 * NULL or W*H*3, the result W*H*3 floats (u px, v px, w m: the cv::Mat_<cv::Vec3f> layout).
 * smoothnessWeight is alpha; maxIters is nSORIterations, as in the reference. */
inline std::vector<float> runFlowTwoFramesSceneFlowExperiments(
    Context& ctx, const rgbdflow_camera_params& fullSizeCamParams, const uint8_t* prevImg, const float* prevDepth,
    const uint8_t* curImg, const float* curDepth, int W, int H, double smoothnessWeight, double depthVsColorDataWeight,
    sceneFlowRegularizationType regularizationType, uint32_t maxIters, const float* estFlow = nullptr,
    const rgbdflow_params* base = nullptr, rgbdflow_stats* stats = nullptr)
{
    rgbdflow_params p;
    if (base) p = *base;
    else rgbdflow_params_default(&p);
    p.alpha = smoothnessWeight;
    p.depth_vs_color_data_weight = depthVsColorDataWeight;
    p.regularization = (int)regularizationType;
    p.n_sor = (int)maxIters;
    std::vector<float> flow((size_t)W * H * 3);
    ctx.check(rgbdflow_scene_flow_two_frames(ctx.get(), &fullSizeCamParams, prevImg, prevDepth, curImg, curDepth, W, H,
                                             &p, estFlow, flow.data(), stats),
              "runFlowTwoFramesSceneFlowExperiments");
    return flow;
}

}  // namespace rgbdflow

#endif /* RGBDFLOW_HPP */
