// adapter_check.cpp — drives include/rgbdflow.hpp the way a caller of the reference would.
//
//   adapter_check cpu         checks without a device: parameter mapping, error behaviour
//   adapter_check gpu DIR     solves the pair stored in DIR (written by the Python test) through
//                             runFlowTwoFramesSceneFlowExperiments, sceneFlowMultiscale and
//                             sceneFlowWithInit, and writes the flows back to DIR
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rgbdflow.hpp"

// The accessors of the Ce Liu Image<T> (include/celiu_flow/Image.h:45,85-89) over a vector.
class DImage {
public:
    DImage() = default;
    DImage(int w, int h, int c) { allocate(w, h, c); }
    void allocate(int w, int h, int c = 1)
    {
        w_ = w; h_ = h; c_ = c;
        buf_.assign((size_t)w * h * c, 0.0);
        p_ = buf_.data();
    }
    double*& data() { return p_; }
    const double* data() const { return p_; }
    int width() const { return w_; }
    int height() const { return h_; }
    int nchannels() const { return c_; }

private:
    std::vector<double> buf_;
    double* p_ = nullptr;
    int w_ = 0, h_ = 0, c_ = 0;
};

static int fails = 0;
#define CHECK(c)                                                        \
    do {                                                                \
        if (!(c)) { std::fprintf(stderr, "FAILED: %s (line %d)\n", #c, __LINE__); fails++; } \
    } while (0)

template <class T> static std::vector<T> read_file(const std::string& path, size_t n)
{
    std::vector<T> v(n);
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f || std::fread(v.data(), sizeof(T), n, f) != n) { std::fprintf(stderr, "cannot read %s\n", path.c_str()); std::exit(2); }
    std::fclose(f);
    return v;
}
template <class T> static void write_file(const std::string& path, const T* p, size_t n)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f || std::fwrite(p, sizeof(T), n, f) != n) { std::fprintf(stderr, "cannot write %s\n", path.c_str()); std::exit(2); }
    std::fclose(f);
}

static int run_cpu()
{
    // the reference defaults of sceneFlowParams (OpticalFlow.h:107-109) and their C mapping
    rgbdflow::sceneFlowParams p;
    CHECK(p.pyramidRatio == 0.75 && p.minWidth == 20 && p.nOuterFPIterations == 7 && p.nSORIterations == 30);
    p.regularizationType = rgbdflow::sceneFlowRegularizationType::LETOUZEY;
    p.alpha = 0.02; p.gamma = 1e-5; p.pyramidRatio = 0.5; p.minWidth = -16;
    p.nOuterFPIterations = 10; p.nInnerFPIterations = 2; p.nSORIterations = 30; p.depthVsColorDataWeight = 3;
    const rgbdflow_params c = p.to_c();
    CHECK(c.regularization == RGBDFLOW_REG_LETOUZEY && c.alpha == 0.02 && c.gamma == 1e-5);
    CHECK(c.pyramid_ratio == 0.5 && c.min_width == -16 && c.n_outer == 10 && c.n_inner == 2 && c.n_sor == 30);
    CHECK(c.depth_vs_color_data_weight == 3 && c.omega == 0.7 && c.sor_check_period == 25);
    // errors are exceptions derived from std::runtime_error, with the status code
    bool threw = false;
    try {
        rgbdflow::Context ctx(0);
    } catch (const rgbdflow::Error& e) {
        threw = true;
        CHECK(e.code() == RGBDFLOW_ERR_NO_DEVICE);
        const std::runtime_error* base = &e;
        CHECK(std::string(base->what()).find("NO_DEVICE") != std::string::npos);
    }
    CHECK(threw);
    return fails ? 1 : 0;
}

static int run_gpu(const std::string& dir)
{
    const auto meta = read_file<double>(dir + "/meta.bin", 6);  // W, H, f, cx, cy, pyramid ratio
    const int W = (int)meta[0], H = (int)meta[1];
    const size_t N = (size_t)W * H;
    const auto bgr1 = read_file<uint8_t>(dir + "/bgr1.bin", N * 3), bgr2 = read_file<uint8_t>(dir + "/bgr2.bin", N * 3);
    const auto d1 = read_file<float>(dir + "/depth1.bin", N), d2 = read_file<float>(dir + "/depth2.bin", N);
    const auto sig = read_file<float>(dir + "/sigma1.bin", N);
    const auto est = read_file<float>(dir + "/est.bin", N * 3);
    rgbdflow_camera_params cam{};
    cam.xRes = W; cam.yRes = H; cam.focalLength = (float)meta[2]; cam.centerX = (float)meta[3]; cam.centerY = (float)meta[4];

    rgbdflow::Context ctx(0);
    // the two-frames entry, with the benchmark's pyramid (ratio, minWidth W/16, 10 outer)
    rgbdflow_params base;
    rgbdflow_params_default(&base);
    base.pyramid_ratio = meta[5]; base.min_width = -16; base.n_outer = 10;
    const auto flow = rgbdflow::runFlowTwoFramesSceneFlowExperiments(
        ctx, cam, bgr1.data(), d1.data(), bgr2.data(), d2.data(), W, H, 0.02, 1.0,
        rgbdflow::sceneFlowRegularizationType::ISOTROPIC, 30, nullptr, &base);
    write_file(dir + "/flow_two_frames.bin", flow.data(), flow.size());

    // sceneFlowMultiscale / sceneFlowWithInit over DImages, as ceLiuSceneFlow calls them
    DImage Im1(W, H, 3), Im2(W, H, 3), dm1(W, H, 1), dm2(W, H, 1);
    for (size_t i = 0; i < N * 3; i++) { Im1.data()[i] = bgr1[i] / 255.0; Im2.data()[i] = bgr2[i] / 255.0; }
    for (size_t i = 0; i < N; i++) { dm1.data()[i] = d1[i]; dm2.data()[i] = d2[i]; }
    rgbdflow::sceneFlowParams sp;
    sp.regularizationType = rgbdflow::sceneFlowRegularizationType::ISOTROPIC;
    sp.camParams = cam;
    sp.alpha = 0.02; sp.gamma = 1e-5; sp.pyramidRatio = meta[5]; sp.minWidth = -16;
    sp.nOuterFPIterations = 10; sp.nInnerFPIterations = 1; sp.nSORIterations = 30;
    sp.depthSigma1 = sig.data();
    DImage u, v, w;
    rgbdflow::sceneFlowMultiscale(ctx, Im1, dm1, Im2, dm2, sp, u, v, w);
    std::vector<double> uvw(N * 3);
    for (size_t i = 0; i < N; i++) { uvw[3 * i] = u.data()[i]; uvw[3 * i + 1] = v.data()[i]; uvw[3 * i + 2] = w.data()[i]; }
    write_file(dir + "/flow_multiscale.bin", uvw.data(), uvw.size());

    DImage e(W, H, 3);
    for (size_t i = 0; i < N * 3; i++) e.data()[i] = est[i];
    rgbdflow::sceneFlowWithInit(ctx, Im1, dm1, Im2, dm2, sp, e, u, v, w);
    for (size_t i = 0; i < N; i++) { uvw[3 * i] = u.data()[i]; uvw[3 * i + 1] = v.data()[i]; uvw[3 * i + 2] = w.data()[i]; }
    write_file(dir + "/flow_with_init.bin", uvw.data(), uvw.size());

    // a bad argument surfaces as an exception with the C status
    bool threw = false;
    try {
        DImage bad(W, H, 1);
        rgbdflow::sceneFlowMultiscale(ctx, bad, dm1, Im2, dm2, sp, u, v, w);
    } catch (const rgbdflow::Error& er) {
        threw = er.code() == RGBDFLOW_ERR_INVALID_ARG;
    }
    CHECK(threw);
    return fails ? 1 : 0;
}

int main(int argc, char** argv)
{
    if (argc >= 2 && std::string(argv[1]) == "cpu") return run_cpu();
    if (argc >= 3 && std::string(argv[1]) == "gpu") return run_gpu(argv[2]);
    std::fprintf(stderr, "usage: adapter_check cpu | gpu DIR\n");
    return 2;
}
