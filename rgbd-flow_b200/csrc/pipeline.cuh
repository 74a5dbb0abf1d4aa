// pipeline.cuh — host-side planning and enqueueing of a (batched) coarse-to-fine solve.
//
// A Plan lays every pair's device state out in one arena, builds the work lists the kernels
// walk (LevelItem / Tile / PyrJob / PrepItem) and enqueues the whole solve on one stream:
// preprocessing, hole fill, pyramids, then per pyramid level the level set-up and the
// outer / inner / SOR schedule.  Levels of different pairs run in the same launches: step s
// serves level Lmax-1-s of every pair that has it, so pairs of different sizes pack together.
// The enqueue is pure stream work with no host synchronisation, so it is captured once into a
// CUDA graph per batch shape and replayed.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "kernels.cuh"
#include "hpb.cuh"

namespace rgbdflow {

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const std::string& where)
        : std::runtime_error(where + ": " + cudaGetErrorString(c)), code(c) {}
};
#define RF_CUDA(x)                                                                   \
    do {                                                                             \
        cudaError_t e_ = (x);                                                        \
        if (e_ != cudaSuccess) throw CudaError(e_, std::string(#x) + " @" + __FILE__ + ":" + std::to_string(__LINE__)); \
    } while (0)

struct ArgError : std::runtime_error {
    int code;
    ArgError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// GaussianPyramid::ConstructPyramid level sizes (GaussianPyramid.cpp:22-62).
struct PyrShape {
    double ratio;      // ratio after the reference's clamp to [0.4, 0.98]
    int n;             // levels built from the base image (log(0.25)/log(ratio))
    double baseSigma;
    std::vector<int> w, h;
    std::vector<int> src;       // source level of each level (0 for i <= n, else i - n)
    std::vector<double> rate;   // resize ratio of each level
    std::vector<double> sigma;
};

static inline PyrShape pyramid_shape(int W, int H, double ratio, int min_width, int max_levels)
{
    PyrShape s;
    if (min_width < 0) min_width = std::max(1, W / -min_width);  // per-pair W / d
    if (ratio > 0.98 || ratio < 0.4) ratio = 0.75;
    s.ratio = ratio;
    double w = W * ratio;
    int L = 1;
    while (w >= min_width) { L++; w *= ratio; }
    if (max_levels > 0 && L > max_levels) L = max_levels;
    s.baseSigma = 1 / ratio - 1;
    s.n = (int)(std::log(0.25) / std::log(ratio));
    s.w.push_back(W); s.h.push_back(H); s.src.push_back(0); s.rate.push_back(1); s.sigma.push_back(0);
    for (int i = 1; i < L; i++) {
        if (i <= s.n) {
            const double r = std::pow(ratio, i);
            s.w.push_back((int)((double)W * r)); s.h.push_back((int)((double)H * r));
            s.src.push_back(0); s.rate.push_back(r); s.sigma.push_back(s.baseSigma * i);
        } else {
            const int sl = i - s.n;
            const double r = (double)std::pow(ratio, i) * W / s.w[sl];
            s.w.push_back((int)((double)s.w[sl] * r)); s.h.push_back((int)((double)s.h[sl] * r));
            s.src.push_back(sl); s.rate.push_back(r); s.sigma.push_back(s.baseSigma * s.n);
        }
    }
    return s;
}

// What one pair of a batch asks for.  kind selects the caller-facing entry point:
//   0  runFlowTwoFramesSceneFlowExperiments: BGR8 colour, float depth (m), optional float est
//   1  sceneFlowMultiscale / sceneFlowWithInit: FP64 [0,1] colour, FP64 depth, float depth sigma,
//      optional FP64 planar (u, v, w) estimate
//   2  sceneFlowSingleScale: FP64 5-channel features, depths, weights and flow of one level
struct PairSpec {
    int kind = 0;
    int W = 0, H = 0;
    float f_full = 0;         // camera focal length resized to W (getResizedCamParams)
    unsigned xres_full = 0;   // camera xRes resized to W
    const uint8_t* bgr1 = nullptr; const float* depth1 = nullptr;
    const uint8_t* bgr2 = nullptr; const float* depth2 = nullptr;
    const float* est = nullptr;                 // kind 0 warm start (W*H*3 interleaved)
    const double* im1 = nullptr; const double* im2 = nullptr;
    const double* dm1 = nullptr; const double* dm2 = nullptr;
    const float* sigma1 = nullptr;
    const double* est_d = nullptr;              // kind 1 warm start (3 planes)
    // kind 2
    const double* feat1 = nullptr; const double* feat2 = nullptr;
    const double* uvw = nullptr;                // 3 planes
    const double* ddw = nullptr; const double* dsw = nullptr; const double* mag = nullptr;
    const double* regw = nullptr;               // W*H*2
    float f_level = 0;
    int allow_early = 0;        // kind 2; and for kinds 0/1 warm starts when warm_early is set
    int warm_early = 0;         // warm-started pair may stop its outer iterations early
    // outputs
    float* out = nullptr;                       // kind 0: W*H*3 interleaved float
    double* out_u = nullptr; double* out_v = nullptr; double* out_w = nullptr;  // kinds 1, 2
    double* out_warpI = nullptr; double* out_warpD = nullptr;                     // kind 2

    bool warm() const { return est || est_d; }
    // input block: list of (host pointer, bytes) in upload order
    std::vector<std::pair<const void*, size_t>> inputs() const
    {
        const size_t N = (size_t)W * H;
        std::vector<std::pair<const void*, size_t>> v;
        if (kind == 0) {
            v = {{bgr1, N * 3}, {bgr2, N * 3}, {depth1, N * 4}, {depth2, N * 4}};
            if (est) v.push_back({est, N * 12});
        } else if (kind == 1) {
            v = {{im1, N * 24}, {im2, N * 24}, {dm1, N * 8}, {dm2, N * 8}, {sigma1, N * 4}};
            if (est_d) v.push_back({est_d, N * 24});
        } else {
            v = {{feat1, N * 40}, {feat2, N * 40}, {dm1, N * 8}, {dm2, N * 8}, {uvw, N * 24},
                 {ddw, N * 8}, {dsw, N * 8}, {mag, N * 8}, {regw, N * 16}};
        }
        return v;
    }
};

struct HostParams {
    int regularization;
    double color_w, dvc, alpha, gamma, ratio;
    int min_width, n_outer, n_inner, n_sor, max_dist, fill_holes, fixed;
    double omega, step, eps_d, eps_z, eps_s, sor_tol, outer_tol, occ_margin, occ_penalty, max_grad;
    int period, K, fill_rounds;
    int sor_ilp, sor_nbuf;  // 0 = automatic
    int sor_strip;          // strip SOR for large FP32 levels (0: tiles everywhere)
    int strip_min_w, strip_min_h, strip_seg;  // strip eligibility and band height (0: automatic)
    long strip_min_px;                        // strips only for steps with this many eligible pixels
    int strip_balanced;                       // untuned strip steps take the balancing model's bands
    int sor_level;                            // whole-level SOR for levels that fit one CTA (0: off)
    int level_cluster;                        // > 1: such levels run on a cluster of this many CTAs instead
    int level_reg;                            // FP32 whole-level SOR with the system in registers (0: off)
};

// Row pitch of the u planes, and the checkerboard half-row length of the x / sys planes (16-byte
// aligned half-rows for the SOR's cp.async loads).
static inline int pitch_of(int W) { return (W + 3) & ~3; }
static inline int hwp_of(int W) { return (((W + 1) / 2) + 3) & ~3; }

// A SOR kernel configuration: K sweeps per launch, NBUF region buffers, ILP the lane mapping of
// a half-sweep (1: one pixel per thread, rows packed; 2: a half-warp per row, two adjacent
// same-colour pixels per lane with 2-wide shared accesses).
struct SorConfig {
    int K = 2, nbuf = 1, ilp = 1;
};

template <class T> static inline bool sor_cfg_fits(const SorConfig& c);

// Configuration of the SOR launches of one level: explicit parameters win; otherwise the setting
// measured best on every level of the 640x480 benchmark (K = 5, one buffer, pair lanes), shrunk
// where the shared memory does not hold it (FP64).  level_px (pixels of the level over the batch)
// is kept for size-dependent choices.
template <class T>
static inline SorConfig choose_sor_config(const HostParams& hp, long level_px)
{
    (void)level_px;
    SorConfig c;
    c.K = hp.K > 0 ? hp.K : 5;  // measured best on every level (25 = 5 x 5 meets the SOR check)
    c.nbuf = hp.sor_nbuf > 0 ? hp.sor_nbuf : 1;
    c.ilp = hp.sor_ilp > 0 ? hp.sor_ilp : 2;  // 2: pair lanes (2-wide shared accesses), measured faster
    while (c.K > 1 && !sor_cfg_fits<T>(c)) {
        if (c.nbuf == 2) c.nbuf = 1;
        else c.K--;
    }
    return c;
}

// The SOR configuration chosen for one level step by the autotuner (rgbdflow.cu, tune_sor): kernel
// (tile or strip), sweeps per launch, lane mapping, strip band height.  The choice changes speed
// only: every configuration gives the same flow bit for bit.
// Strip SOR band layouts by strip height: the band heights of a strip, top to bottom.
using BandMap = std::vector<std::pair<int, std::vector<int>>>;
struct SorChoice {
    int strip = 0;   // strip kernel for the step's strip-eligible items
    int K = 5;       // sweeps per launch
    int ilp = 2;     // tile kernel lane mapping
    int seg = 0;     // strip band height (0: automatic)
    BandMap bands;   // explicit band layouts (strip_balanced_bands); strips of other heights use seg
    double us_per_it = 0;  // measured time per SOR iteration of the step
};
struct TuneTable {
    std::map<std::string, SorChoice> m;  // by step key (sor_step_key)
};

// A level step's tuning key: the arithmetic type and the sorted sizes of its items.
template <class T, class X>
static std::string sor_step_key(const std::vector<X>& items)
{
    std::vector<std::pair<int, int>> sz;
    for (const auto& x : items) sz.push_back({x.W, x.H});
    std::sort(sz.begin(), sz.end());
    std::string k = sizeof(T) == 8 ? "d" : "f";
    for (size_t i = 0; i < sz.size();) {
        size_t j = i;
        while (j < sz.size() && sz[j] == sz[i]) j++;
        k += std::to_string(sz[i].first) + "x" + std::to_string(sz[i].second) + "*" + std::to_string(j - i) + ",";
        i = j;
    }
    return k;
}

// Whether the SOR configuration may be tuned: no explicit sweeps per launch and no measurement
// overrides.
static inline bool sor_tunable(const HostParams& hp)
{
    return hp.K == 0 && hp.sor_ilp == 0 && hp.sor_nbuf == 0 && hp.sor_strip == 1 && hp.strip_min_w == 0 &&
           hp.strip_min_h == 0 && hp.strip_seg == 0 && hp.strip_min_px == 0 && hp.strip_balanced == 0 &&
           hp.level_cluster == 0;
}

// Items the autotuner may put on the strip kernel (FP32, at least two strips wide and two bands high).
template <class T>
static inline bool strip_ok(const HostParams& hp, int W, int H)
{
    return sizeof(T) == 4 && hp.sor_strip && W >= 2 * kStripW && H >= 64;
}

// Whether an item's level may run on the strip SOR: FP32 planes, at most 5 sweeps per launch, and
// a level large enough that its strips carry many rows (the pipeline fill costs about 6 nit rows).
// Measured on the 640x480 benchmark: strips beat tiles on the 640-wide level of a 16-pair batch,
// tie at 320 and lose at 160; with a single pair the 640-wide level has too few strip units to
// fill the SMs, so a step only uses strips when its eligible items add up to enough pixels.
template <class T>
static inline bool use_strip(const HostParams& hp, int W, int H)
{
    if (sizeof(T) != 4 || !hp.sor_strip || hp.K > kStripMaxNit) return false;
    return W >= (hp.strip_min_w > 0 ? hp.strip_min_w : 400) && H >= (hp.strip_min_h > 0 ? hp.strip_min_h : 96);
}

// Work units of the strip SOR: every item's strips of 64 columns, cut into bands of rows (a
// multiple of 32 high; the last band of a strip takes the remainder).  The band height aims at
// about four units per SM over the step, so units of pairs that finish early leave no SM idle
// for long, and at no fewer than 64 rows, so the pipeline fill stays a small share.  Units are
// ordered band-major, then strip, then item: consecutive tickets spread over the pairs.
// Bands of seg rows from the top; the rest of the strip (or, when seg divides it, its last band) in
// smaller bands, 2^k x 32 rows largest first, the last one reaching the bottom.  The units are
// handed out largest first, so the small bands fill the last wave: the SMs finish closer together
// than with equal bands.  Returns the band heights, top to bottom.
static std::vector<int> strip_default_bands(int H, int seg)
{
    std::vector<int> bl;
    int n = H / seg, rem = H - n * seg;
    if (rem == 0 && n >= 2) { n--; rem = seg; }
    for (int b = 0; b < n; b++) bl.push_back(seg);
    while (rem > 0) {
        int piece = rem;
        if (rem >= 64) {
            int p2 = 32;
            while (p2 * 2 <= rem) p2 *= 2;
            if (rem - p2 >= 32) piece = p2;
        }
        bl.push_back(piece);
        rem -= piece;
    }
    return bl;
}

template <class X>
static std::vector<StripUnit> strip_units(const std::vector<X>& items, const std::vector<int>& which,
                                          const HostParams& hp, int sms, const BandMap* layouts = nullptr)
{
    std::vector<StripUnit> v;
    if (which.empty()) return v;
    long rows = 0;
    for (int i : which) rows += (long)((items[i].W + kStripW - 1) / kStripW) * items[i].H;
    int seg = hp.strip_seg;
    if (seg <= 0) {
        const double want = (double)rows / (4.0 * sms);
        seg = (int)((want + 16) / 32) * 32;
        seg = std::max(64, std::min(seg, 512));
    }
    seg = std::max(32, seg & ~31);
    // the explicit layout of the strip height where one is given, else the default bands
    auto bands_of = [&](int H) {
        std::vector<int> hs = strip_default_bands(H, seg);
        if (layouts)
            for (const auto& e : *layouts)
                if (e.first == H) hs = e.second;
        std::vector<std::pair<int, int>> bl;
        int y = 0;
        for (int h : hs) { bl.push_back({y, y + h}); y += h; }
        return bl;
    };
    struct Cand { int h, band, sx, ord; StripUnit u; };
    std::vector<Cand> c;
    for (size_t o = 0; o < which.size(); o++) {
        const int i = which[o];
        const int W = items[i].W, H = items[i].H;
        const auto bl = bands_of(H);
        for (size_t b = 0; b < bl.size(); b++)
            for (int sx = 0; sx * kStripW < W; sx++)
                c.push_back(Cand{bl[b].second - bl[b].first, (int)b, sx, (int)o,
                                 StripUnit{i, sx * kStripW, bl[b].first, bl[b].second}});
    }
    std::stable_sort(c.begin(), c.end(), [](const Cand& a, const Cand& b) {
        if (a.h != b.h) return a.h > b.h;
        if (a.band != b.band) return a.band < b.band;
        if (a.sx != b.sx) return a.sx < b.sx;
        return a.ord < b.ord;
    });
    for (const auto& x : c) v.push_back(x.u);
    return v;
}

// Band layouts for the strip SOR of one step, chosen on a model of the kernel: a unit of R rows
// takes about R + 20 pipeline steps (the fill and drain of the 2 nit stages two rows apart, and the
// prefetch, at nit = 5), and the persistent CTAs take the units largest first as they free up.  A
// layout's cost is the time at which the last CTA finishes, averaged over the step with all its
// items active and with 3 in 4, 2 in 4 and 1 in 4 of them (items whose index mod 4 is below 3, 2,
// 1: pairs that converge early leave the schedule, and every size of a mixed step keeps its share).
// Each strip height of the step in turn gets the layout of at most 3 cuts (at rows that are
// multiples of 32, bands of at most 256 rows: a tall band left for last keeps one SM busy alone)
// that minimises the cost with the other heights' layouts held; a height with too many cut choices
// for the model's budget keeps the default layout of seg rows.  The layout changes speed only:
// every band layout gives the same flow bit for bit.
template <class X>
static BandMap strip_balanced_bands(const std::vector<X>& items, const std::vector<int>& which, int seg, int sms)
{
    constexpr int kOver = 20;
    BandMap lay;
    if (which.empty()) return lay;
    auto find = [&](int H) -> std::vector<int>& {
        for (auto& e : lay)
            if (e.first == H) return e.second;
        lay.push_back({H, strip_default_bands(H, seg)});
        return lay.back().second;
    };
    for (int i : which) find(items[i].H);
    long units_all = 0;
    for (int i : which) units_all += (long)((items[i].W + kStripW - 1) / kStripW) * (long)find(items[i].H).size();
    std::vector<long> heap;
    std::vector<int> costs;
    auto cost = [&]() {
        double acc = 0;
        const int n = (int)which.size();
        for (int q = 4; q >= 1; q--) {  // the items a with a mod 4 < q (item 0 always)
            costs.clear();
            for (int a = 0; a < n; a++) {
                if (a % 4 >= q) continue;
                const int i = which[a];
                const int nsx = (items[i].W + kStripW - 1) / kStripW;
                for (int h : find(items[i].H))
                    for (int sx = 0; sx < nsx; sx++) costs.push_back(h + kOver);
            }
            std::sort(costs.begin(), costs.end(), std::greater<int>());
            const int g = std::min(sms, (int)costs.size());
            heap.assign(g, 0);
            long mk = 0;
            for (int c : costs) {  // list scheduling: the next unit to the CTA that frees up first
                std::pop_heap(heap.begin(), heap.end(), std::greater<long>());
                heap.back() += c;
                mk = std::max(mk, heap.back());
                std::push_heap(heap.begin(), heap.end(), std::greater<long>());
            }
            acc += (double)mk;
        }
        return acc;
    };
    for (auto& e : lay) {
        const int H = e.first;
        std::vector<int> pos;
        for (int y = 32; y < H; y += 32) pos.push_back(y);
        const long P = (long)pos.size();
        const long n_lay = 1 + P + P * (P - 1) / 2 + P * (P - 1) * (P - 2) / 6;
        if (n_lay * std::max(units_all, 1L) > 4000000L) continue;
        std::vector<int> best = e.second;
        double best_c = cost();
        auto trial = [&](const std::vector<int>& cuts) {
            std::vector<int> hs;
            int y = 0;
            for (int c : cuts) { hs.push_back(c - y); y = c; }
            hs.push_back(H - y);
            for (int h : hs)
                if (h > 256) return;
            e.second = hs;
            const double c = cost();
            if (c < best_c - 1e-9) { best_c = c; best = hs; }
        };
        trial({});
        for (long a = 0; a < P; a++) {
            trial({pos[a]});
            for (long b = a + 1; b < P; b++) {
                trial({pos[a], pos[b]});
                for (long d = b + 1; d < P; d++) trial({pos[a], pos[b], pos[d]});
            }
        }
        e.second = best;
    }
    return lay;
}

// Whether an item's level runs on the whole-level SOR: the level's 15 planes fit one CTA's shared
// memory (the coarsest levels, e.g. 40 x 30).
constexpr size_t kLevelSmemMax = 200 * 1024;
template <class T>
static inline bool use_level(const HostParams& hp, int W, int H, int hwp)
{
    (void)W;
    return hp.sor_level && level_smem_bytes<T>(H, hwp) <= kLevelSmemMax;
}

// The cluster size for the whole-level SOR over a thread-block cluster: the fewest CTAs (up to 8)
// whose row bands' 15 planes fit shared memory, every band holding at least one row; 0 when 8 do
// not suffice.
template <class T>
static inline int level_cluster_size(const HostParams& hp, int H, int hwp)
{
    if (!hp.sor_level) return 0;
    for (int C = std::max(2, std::min(hp.level_cluster, 8)); C <= 8; C++)
        if (level_cluster_smem_bytes<T>((H + C - 1) / C, hwp) <= kLevelSmemMax && (H + C - 1) / C * (C - 1) < H) return C;
    return 0;
}

// The cluster size and positions per thread of the register variant of the cluster whole-level
// SOR (FP32): the fewest CTAs (2..8) whose row bands hold at most KP x its thread limit positions
// each, KP = 1 first, then 2, every band holding at least one row; {0, 0} when none fits.
static inline std::pair<int, int> level_cluster_reg_shape(const HostParams& hp, int H, int hwp)
{
    if (!hp.sor_level || !hp.level_reg) return {0, 0};
    for (int KP = 1; KP <= 2; KP++)
        for (int C = std::max(2, std::min(hp.level_cluster, 8)); C <= 8; C++) {
            const int B = (H + C - 1) / C;
            if (B * (C - 1) < H && B * hwp <= KP * (KP == 1 ? clus_reg_threads_max<1>() : clus_reg_threads_max<2>()) &&
                level_cluster_reg_smem_bytes<float>(B, hwp) <= 64 * 1024)
                return {C, KP};
        }
    return {0, 0};
}

// Bump allocator over a byte range.
struct Bump {
    size_t off = 0;
    size_t take(size_t n) { const size_t o = off; off = align_up(off + n, 256); return o; }
};

template <class T, class S>
struct Plan {
    // ---- shape
    int n = 0, Lmax = 0;
    int sms = 148;                // multiprocessors of the device (persistent SOR grid)
    std::vector<SorConfig> sor_cfg;  // SOR kernel configuration per step
    std::vector<PyrShape> shapes;
    std::vector<int> L;           // levels per pair
    HostParams hp;
    // ---- device layout (offsets into the arena)
    size_t arena_bytes = 0;
    size_t in_off = 0, in_bytes = 0;    // inputs uploaded each call (bgr, depth, est)
    size_t out_off = 0, out_bytes = 0;  // flows read back
    size_t ctl_off = 0;                 // PairCtl[n]
    size_t ctr_off = 0;                 // int[16]: strip SOR ticket counter per step (zeroed with ctl)
    size_t desc_off = 0, desc_bytes = 0;
    int kind = 0;
    std::vector<std::vector<size_t>> in_seg;  // per pair: arena offset of each input segment
    std::vector<size_t> out_pair_off;   // per pair: flow (3N T interleaved) [+ warps 5N + N T for kind 2]
    size_t est_src_off = 0, seam_src_off = 0;
    bool any_warm = false;
    // ---- host descriptors (uploaded as one block at desc_off)
    std::vector<unsigned char> desc;
    struct StepDesc {
        long level_px;  // pixels of this level summed over the step's pairs
        size_t items_off; int n_items;
        size_t lin_tiles_off; int n_lin;
        size_t sor_tiles_off; int n_sor;      // tile SOR work list (items not on the strip kernel)
        size_t strip_units_off; int n_units;  // strip SOR work list
        int strip_grid;
        size_t level_items_off; int n_level;  // whole-level SOR: items (one CTA each)
        size_t level_smem;
        int level_threads;
        int level_reg;  // the whole-level items run on k_sor_level_reg
        size_t clus_items_off; int n_clus;    // whole-level SOR over a cluster of clus_c CTAs per item
        int clus_c, clus_threads;
        size_t clus_smem;
        int clus_kp;  // > 0: the cluster items run on k_sor_level_cluster_reg with this many positions a thread
    };
    std::vector<StepDesc> steps;
    struct PyrLevelDesc { size_t jobs_off; int n_jobs; size_t src_tiles_off; int n_src; size_t dst_tiles_off; int n_dst; size_t g_off; };
    std::vector<PyrLevelDesc> pyr;
    size_t prep_items_off = 0, prep_tiles_off = 0; int n_prep_tiles = 0;
    size_t out_ptrs_off = 0;
    size_t unfilled_off = 0;            // int[256]: hole pixels left after each fill round, then the
                                        // fill's GridSync (zeroed together)
    size_t tleft_off = 0;               // int[prep tiles]: the tile still holds a hole
    std::vector<std::vector<std::vector<SorLaunch>>> sor_sched;  // [step][inner iteration]
    std::vector<std::string> step_keys;                         // autotuner key per step
    std::vector<int> step_tuned;                                // the step's SOR configuration came from the tuner
    std::string tune_desc;                                      // the tuned choices in use (part of the graph key)
    std::vector<std::vector<int>> n_checks;                     // [step][inner iteration]
    std::vector<std::vector<size_t>> u_off;         // per pair per level: offset of u[0] (for warm-start upload)
    std::vector<int> est_flag;
    // HPB regularisation weights (regularization == HPB, kinds 0 and 1)
    bool hpb = false;
    int* status = nullptr;              // the context's device status word (bounded waits that gave up)
    size_t hpb_ctr_off = 0;             // int[2n] region / pixel counts, then the fill's GridSync (zeroed each solve)
    size_t hpb_fill_off = 0;            // HpbFill[n] (descriptor offset)
    struct HpbDepthLevel { size_t jobs_off; int n_jobs; size_t tiles_off; int n_tiles; };
    std::vector<HpbDepthLevel> hpb_dpyr;  // raw-depth pyramid, level index 1..Lmax-1
    struct HpbStep { size_t items_off; int n_items; size_t row_first_off, col_first_off; int row_threads, col_threads; };
    std::vector<HpbStep> hpb_step;      // per step (as steps)

    template <class X> size_t put(const std::vector<X>& v)
    {
        const size_t o = align_up(desc.size(), 256);
        desc.resize(o + sizeof(X) * v.size());
        if (!v.empty()) std::memcpy(desc.data() + o, v.data(), sizeof(X) * v.size());
        return o;
    }
};

// SOR launch schedule of one inner iteration: launches of at most K iterations, split so every
// convergence check (it % period == period - 1, .cu:905-921) ends a launch.
static inline std::vector<SorLaunch> sor_schedule(int nSOR, int K, int period, int fixed, int first_inner,
                                                  int last_inner, int& cur, int& n_checks)
{
    std::vector<SorLaunch> v;
    int start = 0;
    int prev_check = 0, prev_idx = 0;
    n_checks = 0;
    while (start < nSOR) {
        int end = std::min(start + K, nSOR);
        if (!fixed)
            for (int it = start; it < end - 1; it++)
                if (it % period == period - 1) { end = it + 1; break; }
        SorLaunch L{};
        L.it0 = start; L.nit = end - start;
        L.xin = cur;
        L.xin_zero = (start == 0 && first_inner);
        L.check = (!fixed && ((end - 1) % period == period - 1));
        L.check_idx = L.check ? std::min((end - 1) / period, kMaxChecks - 1) : 0;
        if (L.check) n_checks = L.check_idx + 1;
        L.prev_check = prev_check; L.prev_check_idx = prev_idx;
        prev_check = L.check; prev_idx = L.check_idx;
        v.push_back(L);
        cur ^= 1;
        start = end;
    }
    if (v.empty()) {
        SorLaunch L{};
        L.xin = cur; L.xin_zero = first_inner;
        v.push_back(L);
        cur ^= 1;
    }
    // the last launch folds (last inner) or keeps x (earlier inner iterations)
    SorLaunch& last = v.back();
    if (last_inner) { last.final_fold = 1; cur ^= 1; }
    else last.final_keep = 1;
    return v;
}

template <class T, class S>
static Plan<T, S> make_plan(const std::vector<PairSpec>& pairs, const HostParams& hp, const TuneTable* tune = nullptr)
{
    if (!sor_tunable(hp)) tune = nullptr;
    Plan<T, S> P;
    P.hp = hp;
    P.n = (int)pairs.size();
    P.kind = pairs.empty() ? 0 : pairs[0].kind;
    for (const auto& p : pairs) {
        if (p.kind != P.kind) throw ArgError(-1, "mixed entry-point kinds in one batch");
        const bool one = p.warm() || p.kind == 2;
        P.shapes.push_back(pyramid_shape(p.W, p.H, hp.ratio, hp.min_width, one ? 1 : 0));
        P.L.push_back((int)P.shapes.back().w.size());
        P.est_flag.push_back(one);
        P.any_warm = P.any_warm || p.warm();
        P.Lmax = std::max(P.Lmax, P.L.back());
    }
    if (P.Lmax > 16) throw ArgError(-2, "more than 16 pyramid levels");
    for (auto& s : P.shapes)
        for (size_t i = 1; i < s.w.size(); i++) {
            if (s.w[i] < 1 || s.h[i] < 1) throw ArgError(-1, "pyramid level collapses to zero size; raise min_width");
            if ((int)(s.sigma[i] * 3) > (kMaxTaps - 1) / 2) throw ArgError(-2, "pyramid filter too wide");
        }
    Bump A;
    P.ctl_off = A.take(sizeof(PairCtl) * P.n);
    P.ctr_off = A.take(sizeof(int) * 16);
    P.unfilled_off = A.take(sizeof(int) * 256 + sizeof(GridSync));
    {
        size_t nt = 0;
        for (const auto& p : pairs) nt += (size_t)((p.W + LTW - 1) / LTW) * ((p.H + LTH - 1) / LTH);
        P.tleft_off = A.take(sizeof(int) * std::max<size_t>(nt, 1));
    }
    const size_t in0 = A.off;
    for (int p = 0; p < P.n; p++) {
        std::vector<size_t> seg;
        for (const auto& x : pairs[p].inputs()) seg.push_back(A.take(x.second));
        P.in_seg.push_back(seg);
    }
    P.in_off = in0; P.in_bytes = A.off - in0;
    const size_t out0 = A.off;
    for (int p = 0; p < P.n; p++) {
        const size_t N = (size_t)pairs[p].W * pairs[p].H;
        P.out_pair_off.push_back(A.take(sizeof(T) * N * (P.kind == 2 ? 9 : 3)));
    }
    P.out_off = out0; P.out_bytes = A.off - out0;

    // per pair per level planes
    struct LevelMem { size_t pyr[10], I1[5], I2[5], D1, D2, mag, rh, rv, u[3], x[2][3], sys[12], stat, hz; int nsor; };
    std::vector<std::vector<LevelMem>> mem(P.n);
    struct L0Mem { size_t stamp[2], bmask, tmp; };
    std::vector<L0Mem> l0(P.n);
    for (int p = 0; p < P.n; p++) {
        const auto& s = P.shapes[p];
        const size_t N0 = (size_t)s.w[0] * s.h[0];
        l0[p].stamp[0] = A.take(N0); l0[p].stamp[1] = A.take(N0); l0[p].bmask = A.take(N0);
        l0[p].tmp = A.take(sizeof(T) * N0 * 10);
        mem[p].resize(P.L[p]);
        for (int k = 0; k < P.L[p]; k++) {
            const size_t N = (size_t)s.w[k] * s.h[k];
            LevelMem& m = mem[p][k];
            for (int c = 0; c < 10; c++) m.pyr[c] = A.take(sizeof(T) * N);
            for (int c = 0; c < 5; c++) { m.I1[c] = A.take(sizeof(S) * N); m.I2[c] = A.take(sizeof(S) * N); }
            m.D1 = A.take(sizeof(S) * N); m.D2 = A.take(sizeof(S) * N);
            m.mag = A.take(sizeof(T) * N); m.rh = A.take(sizeof(T) * N); m.rv = A.take(sizeof(T) * N);
            const size_t NP = (size_t)pitch_of(s.w[k]) * s.h[k];
            const size_t NC = (size_t)2 * hwp_of(s.w[k]) * s.h[k];
            for (int c = 0; c < 3; c++) m.u[c] = A.take(sizeof(T) * NP);
            for (int b = 0; b < 2; b++) for (int c = 0; c < 3; c++) m.x[b][c] = A.take(sizeof(T) * NC);
            for (int c = 0; c < 12; c++) m.sys[c] = A.take(sizeof(T) * NC);
            m.nsor = ((s.w[k] + kSorTW - 1) / kSorTW) * ((s.h[k] + kSorTH - 1) / kSorTH);
            m.stat = A.take(sizeof(T) * m.nsor);
            m.hz = 0;
        }
    }
    // HPB: the raw-depth pyramid per level and, per pair, scratch for one level at a time
    P.hpb = hp.regularization == 2 && P.kind != 2;
    struct HpbMem { size_t label, par, csz, done, regions, px, nrm[3], nval, rad, pre[6], pre_v, ii[6], ii_v, feat[4], bp[2]; };
    std::vector<HpbMem> hm(P.n);
    if (P.hpb) {
        P.hpb_ctr_off = A.take(sizeof(int) * 2 * P.n + sizeof(GridSync));
        for (int p = 0; p < P.n; p++) {
            const auto& s = P.shapes[p];
            // DepthMapPyramid's level sizes must be the colour pyramid's: the reference reads one
            // with the other's size (heuristicProbBoundary.cpp:31-38)
            for (int k = 1; k < P.L[p]; k++) {
                const double r = std::pow(s.ratio, k);
                if ((int)(s.w[0] * r) != s.w[k] || (int)(s.h[0] * r) != s.h[k])
                    throw ArgError(-2, "HPB: the raw-depth pyramid's level size differs from the colour pyramid's");
            }
            for (int k = 0; k < P.L[p]; k++) mem[p][k].hz = A.take(sizeof(T) * (size_t)s.w[k] * s.h[k]);
            const size_t N0 = (size_t)s.w[0] * s.h[0], NI = (size_t)(s.w[0] + 1) * (s.h[0] + 1);
            HpbMem& h = hm[p];
            h.label = A.take(sizeof(int) * N0); h.par = A.take(sizeof(int) * N0); h.csz = A.take(sizeof(int) * N0);
            h.done = A.take(N0);
            // at most ceil(N0 / 2) 4-connected regions (a checkerboard)
            h.regions = A.take(sizeof(int2) * (N0 / 2 + 2)); h.px = A.take(sizeof(int) * N0);
            for (int c = 0; c < 3; c++) h.nrm[c] = A.take(sizeof(float) * N0);
            h.nval = A.take(sizeof(unsigned) * N0); h.rad = A.take(sizeof(int) * N0);
            for (int c = 0; c < 6; c++) h.pre[c] = A.take(sizeof(float) * N0);
            h.pre_v = A.take(sizeof(unsigned) * N0);
            for (int c = 0; c < 6; c++) h.ii[c] = A.take(sizeof(float) * NI);
            h.ii_v = A.take(sizeof(unsigned) * NI);
            for (int c = 0; c < 4; c++) h.feat[c] = A.take(sizeof(float) * N0);
            for (int c = 0; c < 2; c++) h.bp[c] = A.take(sizeof(float) * N0);
        }
    }
    P.arena_bytes = A.off;  // descriptors are appended after planning (desc_off)
    P.u_off.resize(P.n);
    for (int p = 0; p < P.n; p++)
        for (int k = 0; k < P.L[p]; k++) P.u_off[p].push_back(mem[p][k].u[0]);

    // Descriptor pointer fields hold arena OFFSETS here; bind_plan() rebases them to device
    // addresses once the arena exists.

    // prep items
    std::vector<PrepItem<T>> prep(P.n);
    std::vector<Tile> prep_tiles;
    for (int p = 0; p < P.n; p++) {
        const auto& s = P.shapes[p];
        const size_t N0 = (size_t)s.w[0] * s.h[0];
        PrepItem<T>& it = prep[p];
        std::memset(&it, 0, sizeof(it));
        it.W = s.w[0]; it.H = s.h[0];
        const std::vector<size_t>& sg = P.in_seg[p];
        it.kind = pairs[p].kind;
        if (it.kind == 0) {
            it.bgr[0] = (const uint8_t*)sg[0]; it.bgr[1] = (const uint8_t*)sg[1];
            it.depth[0] = (const float*)sg[2]; it.depth[1] = (const float*)sg[3];
        } else if (it.kind == 1) {
            it.im_d[0] = (const double*)sg[0]; it.im_d[1] = (const double*)sg[1];
            it.dep_d[0] = (const double*)sg[2]; it.dep_d[1] = (const double*)sg[3];
            it.sigma_in = (const float*)sg[4];
        }
        for (int c = 0; c < 3; c++) { it.col[0][c] = (T*)mem[p][0].pyr[c]; it.col[1][c] = (T*)mem[p][0].pyr[3 + c]; }
        it.dep[0] = (T*)mem[p][0].pyr[6]; it.dep[1] = (T*)mem[p][0].pyr[7];
        it.stamp[0] = (uint8_t*)l0[p].stamp[0]; it.stamp[1] = (uint8_t*)l0[p].stamp[1];
        it.bmask = (uint8_t*)l0[p].bmask;
        it.ddw = (T*)mem[p][0].pyr[8]; it.dsw = (T*)mem[p][0].pyr[9];
        it.f2 = (T)((double)pairs[p].f_full * (double)pairs[p].f_full);
        it.dvc = (T)hp.dvc;
        it.max_dist = hp.max_dist;
        it.tiles_x = (s.w[0] + LTW - 1) / LTW;
        it.tile0 = (int)prep_tiles.size();
        const int ty = (s.h[0] + LTH - 1) / LTH;
        for (int y = 0; y < ty; y++)
            for (int x = 0; x < it.tiles_x; x++) prep_tiles.push_back(Tile{p, x, y, y * it.tiles_x + x});
    }
    if (P.kind == 2) prep_tiles.clear();  // the seam takes ready-made level inputs
    P.prep_items_off = P.put(prep);
    P.prep_tiles_off = P.put(prep_tiles);
    P.n_prep_tiles = (int)prep_tiles.size();

    // pyramid jobs per level index i >= 1
    for (int i = 1; i < P.Lmax; i++) {
        std::vector<PyrJob<T>> jobs;
        std::vector<Tile> st, dt;
        std::vector<T> g;
        for (int p = 0; p < P.n; p++) {
            if (i >= P.L[p]) continue;
            const auto& s = P.shapes[p];
            PyrJob<T> jb;
            std::memset(&jb, 0, sizeof(jb));
            const int sl = s.src[i];
            jb.sW = s.w[sl]; jb.sH = s.h[sl]; jb.dW = s.w[i]; jb.dH = s.h[i];
            jb.nplanes = 10;
            jb.fs = (int)(s.sigma[i] * 3);
            jb.rate = s.rate[i];
            for (int c = 0; c < 10; c++) {
                jb.src[c] = (const T*)mem[p][sl].pyr[c];
                jb.tmp[c] = (T*)(l0[p].tmp + sizeof(T) * (size_t)s.w[0] * s.h[0] * c);
                jb.dst[c] = (T*)mem[p][i].pyr[c];
            }
            const int jid = (int)jobs.size();
            // columns the resample reads with a nonzero weight: when every sample falls on a source
            // column of one progression hoff + hstep j (rate 1/2: x = 2j + 1; rate 1/4: x = 4j + 3;
            // weight 1 there, 0 on the next column), only those columns are filtered, stored side by
            // side (tmp rows of dW values); otherwise every column (tmp rows of sW values)
            jb.hstep = 1;
            jb.hoff = 0;
            {
                const double x0 = 1.0 / jb.rate - 1, x1 = 2.0 / jb.rate - 1;
                const int a = (int)x0, d = (int)x1 - (int)x0;
                bool prog = jb.dW >= 2 && x0 == (double)a && x1 == (double)(int)x1 && d >= 2 && a >= 0;
                for (int jj = 0; jj < jb.dW && prog; jj++) {
                    const double x = (double)(jj + 1) / jb.rate - 1;
                    prog = x == (double)(a + d * jj) && a + d * jj < jb.sW;
                }
                if (prog) { jb.hstep = d; jb.hoff = a; }
            }
            jb.tW = jb.hstep > 1 ? jb.dW : jb.sW;
            jb.tiles_x_src = (jb.tW + LTW - 1) / LTW;
            jb.tile0_src = (int)st.size();
            for (int y = 0; y < (jb.sH + LTH - 1) / LTH; y++)
                for (int x = 0; x < jb.tiles_x_src; x++) st.push_back(Tile{jid, x, y, 0});
            jb.tiles_x_dst = (jb.dW + LTW - 1) / LTW;
            jb.tile0_dst = (int)dt.size();
            for (int y = 0; y < (jb.dH + LTH - 1) / LTH; y++)
                for (int x = 0; x < jb.tiles_x_dst; x++) dt.push_back(Tile{jid, x, y, 0});
            jobs.push_back(jb);
            // Image::GaussianSmoothing filter (Image.h:1184-1193), computed in FP64
            std::vector<double> gd(2 * jb.fs + 1);
            double sum = 0;
            const double s2 = s.sigma[i] * s.sigma[i] * 2;
            for (int l = -jb.fs; l <= jb.fs; l++) { gd[l + jb.fs] = std::exp(-(double)(l * l) / s2); sum += gd[l + jb.fs]; }
            for (int l = 0; l < kMaxTaps; l++) g.push_back(l < 2 * jb.fs + 1 ? (T)(gd[l] / sum) : (T)0);
        }
        typename Plan<T, S>::PyrLevelDesc d;
        d.jobs_off = P.put(jobs); d.n_jobs = (int)jobs.size();
        d.src_tiles_off = P.put(st); d.n_src = (int)st.size();
        d.dst_tiles_off = P.put(dt); d.n_dst = (int)dt.size();
        d.g_off = P.put(g);
        P.pyr.push_back(d);
    }

    if (P.hpb) {
        // the colour-guided fill of frame 1's raw depth (level 0), read through the pair's PrepItem
        std::vector<HpbFill<T>> fills(P.n);
        for (int p = 0; p < P.n; p++) {
            HpbFill<T>& f = fills[p];
            std::memset(&f, 0, sizeof(f));
            f.W = P.shapes[p].w[0]; f.H = P.shapes[p].h[0];
            f.src = (const PrepItem<T>*)(P.prep_items_off + sizeof(PrepItem<T>) * p);  // descriptor-relative
            f.fill = P.est_flag[p] ? 0 : 1;  // the warm start reads the raw depth (sceneFlowWithInit.cpp:48)
            f.out = (T*)mem[p][0].hz;
            f.label = (int*)hm[p].label; f.par = (int*)hm[p].par; f.csz = (int*)hm[p].csz;
            f.done = (uint8_t*)hm[p].done; f.regions = (int2*)hm[p].regions; f.px = (int*)hm[p].px;
            f.counts = (int*)(P.hpb_ctr_off + sizeof(int) * 2 * p);
        }
        P.hpb_fill_off = P.put(fills);
        // DepthMapPyramid levels (depthMapPyramid.cpp:15-91)
        for (int i = 1; i < P.Lmax; i++) {
            std::vector<DepthPyrJob<T>> jobs;
            std::vector<Tile> tl;
            for (int p = 0; p < P.n; p++) {
                if (i >= P.L[p]) continue;
                const auto& s = P.shapes[p];
                DepthPyrJob<T> jb;
                jb.sW = s.w[i - 1]; jb.sH = s.h[i - 1]; jb.dW = s.w[i]; jb.dH = s.h[i];
                jb.src = (const T*)mem[p][i - 1].hz;
                jb.dst = (T*)mem[p][i].hz;
                const int jid = (int)jobs.size();
                for (int y = 0; y < (jb.dH + LTH - 1) / LTH; y++)
                    for (int x = 0; x < (jb.dW + LTW - 1) / LTW; x++) tl.push_back(Tile{jid, x, y, 0});
                jobs.push_back(jb);
            }
            typename Plan<T, S>::HpbDepthLevel d;
            d.jobs_off = P.put(jobs); d.n_jobs = (int)jobs.size();
            d.tiles_off = P.put(tl); d.n_tiles = (int)tl.size();
            P.hpb_dpyr.push_back(d);
        }
        // computeHeuristicPb per level, items in the order of the level step's items
        for (int sidx = 0; sidx < P.Lmax; sidx++) {
            const int k = P.Lmax - 1 - sidx;
            std::vector<HpbItem<T>> its;
            std::vector<int> rf{0}, cf{0};
            for (int p = 0; p < P.n; p++) {
                if (k >= P.L[p]) continue;
                const int W = P.shapes[p].w[k], H = P.shapes[p].h[k];
                HpbItem<T> it;
                std::memset(&it, 0, sizeof(it));
                it.W = W; it.H = H;
                // the wrapper's camera (heuristicProbBoundary.cpp:24-29)
                it.f = (float)(525.0 * (unsigned)W / 640);
                it.cx = (float)((unsigned)W / 2);
                it.cy = (float)((unsigned)H / 2);
                for (int c = 0; c < 3; c++) it.col[c] = (const T*)mem[p][k].pyr[c];
                it.z = (const T*)mem[p][k].hz;
                it.rh = (T*)mem[p][k].rh; it.rv = (T*)mem[p][k].rv;
                const HpbMem& h = hm[p];
                for (int c = 0; c < 3; c++) it.nrm[c] = (float*)h.nrm[c];
                it.nval = (unsigned*)h.nval; it.rad = (int*)h.rad;
                for (int c = 0; c < 6; c++) { it.pre[c] = (float*)h.pre[c]; it.ii[c] = (float*)h.ii[c]; }
                it.pre_v = (unsigned*)h.pre_v; it.ii_v = (unsigned*)h.ii_v;
                for (int c = 0; c < 4; c++) it.feat[c] = (float*)h.feat[c];
                for (int c = 0; c < 2; c++) it.bp[c] = (float*)h.bp[c];
                its.push_back(it);
                rf.push_back(rf.back() + 7 * H);
                cf.push_back(cf.back() + 7 * (W + 1));
            }
            typename Plan<T, S>::HpbStep d;
            d.items_off = P.put(its); d.n_items = (int)its.size();
            d.row_first_off = P.put(rf); d.col_first_off = P.put(cf);
            d.row_threads = rf.back(); d.col_threads = cf.back();
            P.hpb_step.push_back(d);
        }
    }

    // level steps
    for (int sidx = 0; sidx < P.Lmax; sidx++) {
        const int k = P.Lmax - 1 - sidx;
        std::vector<LevelItem<T, S>> items;
        std::vector<Tile> lt, stt;
        for (int p = 0; p < P.n; p++) {
            if (k >= P.L[p]) continue;
            const auto& s = P.shapes[p];
            const LevelMem& m = mem[p][k];
            LevelItem<T, S> it;
            std::memset(&it, 0, sizeof(it));
            it.W = s.w[k]; it.H = s.h[k];
            it.level = k;
            it.allow_early = (k < P.L[p] - 1) ? 1 : 0;
            it.est_init = P.est_flag[p];
            // getDownsizedCamParams (sceneFlowMultiscale.cpp:16-27): f *= W_k / xRes, in float
            const double sf = (double)s.w[k] / pairs[p].xres_full;
            it.f_level = (T)(float)(pairs[p].f_full * sf);
            if (P.kind == 2) { it.allow_early = pairs[p].allow_early; it.f_level = (T)pairs[p].f_level; }
            else if (pairs[p].warm() && pairs[p].warm_early) it.allow_early = 1;
            it.ctl = (PairCtl*)(P.ctl_off + sizeof(PairCtl) * p);
            for (int c = 0; c < 10; c++) it.pyr[c] = (T*)m.pyr[c];
            for (int c = 0; c < 5; c++) { it.I1[c] = (S*)m.I1[c]; it.I2[c] = (S*)m.I2[c]; }
            it.D1 = (S*)m.D1; it.D2 = (S*)m.D2;
            it.mag = (T*)m.mag; it.rh = (T*)m.rh; it.rv = (T*)m.rv;
            for (int c = 0; c < 3; c++) it.u[c] = (T*)m.u[c];
            for (int b = 0; b < 2; b++) for (int c = 0; c < 3; c++) it.x[b][c] = (T*)m.x[b][c];
            for (int c = 0; c < 12; c++) it.sys[c] = (T*)m.sys[c];
            it.stat_part = (T*)m.stat;
            it.pitch = pitch_of(s.w[k]);
            it.hwp = hwp_of(s.w[k]);
            if (k + 1 < P.L[p] && !P.est_flag[p]) {
                for (int c = 0; c < 3; c++) it.uc[c] = (const T*)mem[p][k + 1].u[c];
                it.Wc = s.w[k + 1]; it.Hc = s.h[k + 1]; it.pitch_c = pitch_of(s.w[k + 1]);
            }
            it.inv_ratio = (T)(1 / hp.ratio);
            it.xres_full = (int)pairs[p].xres_full;
            it.f_full = (T)pairs[p].f_full;
            const int iid = (int)items.size();
            it.lin_tiles_x = (it.W + LTW - 1) / LTW;
            it.lin_tile0 = (int)lt.size();
            const int lty = (it.H + LTH - 1) / LTH;
            for (int y = 0; y < lty; y++)
                for (int x = 0; x < it.lin_tiles_x; x++) lt.push_back(Tile{iid, x, y, y * it.lin_tiles_x + x});
            items.push_back(it);
        }
        std::vector<int> strip_items, level_items, clus_items;
        size_t level_smem = 0, clus_smem = 0, level_reg_smem = 0;
        int level_thr = 64, clus_c = 0, clus_thr = 64;
        bool level_reg = sizeof(T) == 4 && hp.level_reg != 0;
        long strip_px = 0;
        for (const auto& x : items)
            if (use_strip<T>(hp, x.W, x.H)) strip_px += (long)x.W * x.H;
        // the tuned choice for this step's sizes, where the tuner has measured one
        const std::string skey = sor_step_key<T>(items);
        const SorChoice* ch = nullptr;
        if (tune) {
            const auto f = tune->m.find(skey);
            if (f != tune->m.end()) ch = &f->second;
        }
        P.step_keys.push_back(skey);
        P.step_tuned.push_back(ch != nullptr);
        const bool strips = ch ? ch->strip != 0 : strip_px >= (hp.strip_min_px > 0 ? hp.strip_min_px : 2000000L);
        for (auto& x : items) {
            const int sx = (x.W + kSorTW - 1) / kSorTW, sy = (x.H + kSorTH - 1) / kSorTH;
            x.n_sor_tiles = sx * sy;
            if (use_level<T>(hp, x.W, x.H, x.hwp) && !(hp.level_cluster > 1 && x.H >= 2 * hp.level_cluster)) {
                level_items.push_back((int)(&x - items.data()));
                level_smem = std::max(level_smem, level_smem_bytes<T>(x.H, x.hwp));
                level_reg_smem = std::max(level_reg_smem, level_reg_smem_bytes<T>(x.H, x.hwp));
                level_thr = std::max(level_thr, level_threads(x.H, x.hwp));
                level_reg = level_reg && x.H * x.hwp <= kLevelRegMax && level_reg_smem_bytes<T>(x.H, x.hwp) <= 64 * 1024;
                continue;
            }
            if (level_cluster_size<T>(hp, x.H, x.hwp) > 0 && !(ch && ch->strip)) {
                clus_items.push_back((int)(&x - items.data()));
                clus_c = std::max(clus_c, level_cluster_size<T>(hp, x.H, x.hwp));
                continue;
            }
            if (strips && (ch ? strip_ok<T>(hp, x.W, x.H) : use_strip<T>(hp, x.W, x.H))) {
                strip_items.push_back((int)(&x - items.data()));
                continue;
            }
            for (int y = 0; y < sy; y++)
                for (int xx = 0; xx < sx; xx++) stt.push_back(Tile{(int)(&x - items.data()), xx, y, y * sx + xx});
        }
        HostParams hs = hp;
        if (ch) hs.strip_seg = ch->seg;
        BandMap bal;
        if (!ch && hp.strip_balanced && !strip_items.empty())
            bal = strip_balanced_bands(items, strip_items, hp.strip_seg > 0 ? hp.strip_seg : 128, P.sms > 0 ? P.sms : 148);
        const std::vector<StripUnit> units = strip_units(items, strip_items, hs, P.sms, ch ? &ch->bands : &bal);
        if (ch) {
            P.tune_desc += skey + (ch->strip ? "s" + std::to_string(ch->seg) : "t") + std::to_string(ch->K) +
                           std::to_string(ch->ilp);
            for (const auto& e : ch->bands) {
                P.tune_desc += "b" + std::to_string(e.first);
                for (int h : e.second) P.tune_desc += "." + std::to_string(h);
            }
            P.tune_desc += ";";
        }
        typename Plan<T, S>::StepDesc d;
        d.level_px = 0;
        for (const auto& x : items) d.level_px += (long)x.W * x.H;
        d.items_off = P.put(items); d.n_items = (int)items.size();
        d.lin_tiles_off = P.put(lt); d.n_lin = (int)lt.size();
        d.sor_tiles_off = P.put(stt); d.n_sor = (int)stt.size();
        d.strip_units_off = P.put(units); d.n_units = (int)units.size();
        d.strip_grid = std::min(P.sms, d.n_units);
        d.level_items_off = P.put(level_items); d.n_level = (int)level_items.size();
        d.level_reg = level_reg && !level_items.empty();
        d.level_smem = d.level_reg ? level_reg_smem : level_smem;
        d.level_threads = level_thr;
        // the register variant when every cluster item fits it (FP32)
        int reg_c = 0, reg_kp = 0;
        bool clus_reg = sizeof(T) == 4 && !clus_items.empty();
        for (int i : clus_items) {
            const auto sh = level_cluster_reg_shape(hp, items[i].H, items[i].hwp);
            clus_reg = clus_reg && sh.first > 0;
            reg_c = std::max(reg_c, sh.first);
            reg_kp = std::max(reg_kp, sh.second);
        }
        if (clus_reg) clus_c = reg_c;
        for (int i : clus_items) {
            const int B = (items[i].H + clus_c - 1) / clus_c;
            if (clus_reg) {
                clus_smem = std::max(clus_smem, level_cluster_reg_smem_bytes<T>(B, items[i].hwp));
                clus_thr = std::max(clus_thr, ((B * items[i].hwp + reg_kp - 1) / reg_kp + 31) / 32 * 32);
            } else {
                clus_smem = std::max(clus_smem, level_cluster_smem_bytes<T>(B, items[i].hwp));
                clus_thr = std::max(clus_thr, std::min(1024, (B * items[i].hwp + 31) / 32 * 32));
            }
        }
        d.clus_items_off = P.put(clus_items); d.n_clus = (int)clus_items.size();
        d.clus_c = clus_c; d.clus_smem = clus_smem; d.clus_threads = clus_thr;
        d.clus_kp = clus_reg ? reg_kp : 0;
        P.steps.push_back(d);
    }
    // output pointers (one per pair, in the order of the finest step's items = pair order)
    std::vector<T*> outs;
    for (int p = 0; p < P.n; p++) outs.push_back((T*)P.out_pair_off[p]);
    P.out_ptrs_off = P.put(outs);
    std::vector<EstSrc> est(P.n);
    std::vector<SeamSrc> seam(P.n);
    for (int p = 0; p < P.n; p++) {
        const std::vector<size_t>& sg = P.in_seg[p];
        est[p].f = nullptr; est[p].d = nullptr;
        if (P.kind == 0 && pairs[p].est) est[p].f = (const float*)sg[4];
        if (P.kind == 1 && pairs[p].est_d) est[p].d = (const double*)sg[5];
        std::memset(&seam[p], 0, sizeof(SeamSrc));
        if (P.kind == 2) {
            seam[p].im1 = (const double*)sg[0]; seam[p].im2 = (const double*)sg[1];
            seam[p].dm1 = (const double*)sg[2]; seam[p].dm2 = (const double*)sg[3];
            seam[p].uvw = (const double*)sg[4];
            seam[p].ddw = (const double*)sg[5]; seam[p].dsw = (const double*)sg[6]; seam[p].mag = (const double*)sg[7];
            seam[p].regw = (const double*)sg[8];
        }
    }
    P.est_src_off = P.put(est);
    P.seam_src_off = P.put(seam);

    // SOR configuration and launch schedule per step (level) and inner iteration
    for (int sidx = 0; sidx < P.Lmax; sidx++) {
        SorConfig c = choose_sor_config<T>(hp, P.steps[sidx].level_px);
        if (P.step_tuned[sidx]) {
            const SorChoice& ch = tune->m.find(P.step_keys[sidx])->second;
            c.K = ch.K;
            c.ilp = ch.ilp;
            c.nbuf = 1;
            while (c.K > 1 && !sor_cfg_fits<T>(c)) c.K--;
        }
        P.sor_cfg.push_back(c);
        int cur = 0;
        std::vector<std::vector<SorLaunch>> sch;
        std::vector<int> ncs;
        for (int hh = 0; hh < hp.n_inner; hh++) {
            int nc = 0;
            sch.push_back(sor_schedule(hp.n_sor, c.K, hp.period, hp.fixed, hh == 0, hh == hp.n_inner - 1, cur, nc));
            ncs.push_back(nc);
        }
        P.sor_sched.push_back(sch);
        P.n_checks.push_back(ncs);
    }
    P.desc_off = align_up(P.arena_bytes, 256);
    P.desc_bytes = P.desc.size();
    P.arena_bytes = P.desc_off + P.desc_bytes;
    return P;
}

// Rebase every pointer field of the descriptors from an arena offset to base + offset.
template <class X> static inline void rebase(X*& p, char* base) { p = (X*)(base + (size_t)p); }
template <class X> static inline void rebase_nz(X*& p, char* base) { if (p) p = (X*)(base + (size_t)p); }

template <class T, class S>
static void bind_plan(Plan<T, S>& P, char* base)
{
    unsigned char* d = P.desc.data();
    {
        PrepItem<T>* it = (PrepItem<T>*)(d + P.prep_items_off);
        for (int p = 0; p < P.n; p++) {
            for (int f = 0; f < 2; f++) {
                rebase_nz(it[p].bgr[f], base); rebase_nz(it[p].depth[f], base);
                rebase_nz(it[p].im_d[f], base); rebase_nz(it[p].dep_d[f], base);
                for (int c = 0; c < 3; c++) rebase(it[p].col[f][c], base);
                rebase(it[p].dep[f], base); rebase(it[p].stamp[f], base);
            }
            rebase_nz(it[p].sigma_in, base);
            rebase(it[p].bmask, base); rebase(it[p].ddw, base); rebase(it[p].dsw, base);
        }
    }
    for (auto& lv : P.pyr) {
        PyrJob<T>* jb = (PyrJob<T>*)(d + lv.jobs_off);
        for (int j = 0; j < lv.n_jobs; j++)
            for (int c = 0; c < 10; c++) { rebase(jb[j].src[c], base); rebase(jb[j].tmp[c], base); rebase(jb[j].dst[c], base); }
    }
    for (auto& st : P.steps) {
        LevelItem<T, S>* it = (LevelItem<T, S>*)(d + st.items_off);
        for (int i = 0; i < st.n_items; i++) {
            LevelItem<T, S>& x = it[i];
            rebase(x.ctl, base);
            for (int c = 0; c < 10; c++) rebase(x.pyr[c], base);
            for (int c = 0; c < 5; c++) { rebase(x.I1[c], base); rebase(x.I2[c], base); }
            rebase(x.D1, base); rebase(x.D2, base);
            rebase(x.mag, base); rebase(x.rh, base); rebase(x.rv, base);
            for (int c = 0; c < 3; c++) rebase(x.u[c], base);
            for (int b = 0; b < 2; b++) for (int c = 0; c < 3; c++) rebase(x.x[b][c], base);
            for (int c = 0; c < 12; c++) rebase(x.sys[c], base);
            rebase(x.stat_part, base);
            for (int c = 0; c < 3; c++) rebase_nz(x.uc[c], base);
        }
    }
    if (P.hpb) {
        HpbFill<T>* fl = (HpbFill<T>*)(d + P.hpb_fill_off);
        for (int p = 0; p < P.n; p++) {
            rebase(fl[p].src, base + P.desc_off);
            rebase(fl[p].out, base); rebase(fl[p].label, base); rebase(fl[p].done, base);
            rebase(fl[p].par, base); rebase(fl[p].csz, base); rebase(fl[p].regions, base);
            rebase(fl[p].px, base); rebase(fl[p].counts, base);
        }
        for (auto& lv : P.hpb_dpyr) {
            DepthPyrJob<T>* jb = (DepthPyrJob<T>*)(d + lv.jobs_off);
            for (int j = 0; j < lv.n_jobs; j++) { rebase(jb[j].src, base); rebase(jb[j].dst, base); }
        }
        for (auto& st : P.hpb_step) {
            HpbItem<T>* it = (HpbItem<T>*)(d + st.items_off);
            for (int i = 0; i < st.n_items; i++) {
                HpbItem<T>& x = it[i];
                for (int c = 0; c < 3; c++) { rebase(x.col[c], base); rebase(x.nrm[c], base); }
                rebase(x.z, base); rebase(x.rh, base); rebase(x.rv, base);
                rebase(x.nval, base); rebase(x.rad, base); rebase(x.pre_v, base); rebase(x.ii_v, base);
                for (int c = 0; c < 6; c++) { rebase(x.pre[c], base); rebase(x.ii[c], base); }
                for (int c = 0; c < 4; c++) rebase(x.feat[c], base);
                for (int c = 0; c < 2; c++) rebase(x.bp[c], base);
            }
        }
    }
    T** outs = (T**)(d + P.out_ptrs_off);
    for (int p = 0; p < P.n; p++) rebase(outs[p], base);
    EstSrc* est = (EstSrc*)(d + P.est_src_off);
    SeamSrc* seam = (SeamSrc*)(d + P.seam_src_off);
    for (int p = 0; p < P.n; p++) {
        rebase_nz(est[p].f, base); rebase_nz(est[p].d, base);
        rebase_nz(seam[p].im1, base); rebase_nz(seam[p].im2, base); rebase_nz(seam[p].dm1, base);
        rebase_nz(seam[p].dm2, base); rebase_nz(seam[p].uvw, base); rebase_nz(seam[p].ddw, base);
        rebase_nz(seam[p].dsw, base); rebase_nz(seam[p].mag, base); rebase_nz(seam[p].regw, base);
    }
}

template <class T>
static SolveConst<T> solve_const(const HostParams& hp)
{
    SolveConst<T> k;
    k.alpha = (T)hp.alpha; k.gamma = (T)hp.gamma; k.color_w = (T)hp.color_w;
    k.eps_d = (T)hp.eps_d; k.eps_z = (T)hp.eps_z; k.eps_s = (T)hp.eps_s;
    k.omega = (T)hp.omega; k.step = (T)hp.step;
    k.occ_margin = (T)hp.occ_margin; k.occ_penalty = (T)hp.occ_penalty; k.max_grad = (T)hp.max_grad;
    k.sor_tol = hp.sor_tol; k.outer_tol = hp.outer_tol;
    k.fixed = hp.fixed; k.n_sor = hp.n_sor; k.period = hp.period;
    return k;
}

// ------------------------------------------------------------------------------------------
// Optional kernel timing: CUDA events around every launch, aggregated per kernel class.

enum KClass { KC_PREP, KC_SIGMA, KC_FILL, KC_PYR_H, KC_PYR_V, KC_SETUP, KC_LIN, KC_SOR, KC_CTL, KC_OUT, KC_MISC, KC_HPB, KC_N };
constexpr int KC_SOR_LEVEL0 = KC_N;           // per-level SOR classes: KC_SOR_LEVEL0 + level
constexpr int KC_TOTAL = KC_N + 16;
static const char* const kClassNames[KC_N] = {"prep", "depth_sigma", "hole_fill", "pyr_hfilter", "pyr_vresize",
                                              "level_setup", "linearize", "sor", "control", "output", "misc", "hpb"};

struct Prof {
    std::vector<cudaEvent_t> pool;
    std::vector<int> cls;
    size_t used = 0;
    void begin(int c, cudaStream_t st)
    {
        if (used + 2 > pool.size()) {
            for (int i = 0; i < 256; i++) {
                cudaEvent_t e;
                RF_CUDA(cudaEventCreate(&e));
                pool.push_back(e);
            }
        }
        cls.push_back(c);
        RF_CUDA(cudaEventRecord(pool[used++], st));
    }
    void end(cudaStream_t st) { RF_CUDA(cudaEventRecord(pool[used++], st)); }
    // after the stream synchronised: add per-class time
    void collect(double* ms, int* n)
    {
        for (size_t i = 0; i < cls.size(); i++) {
            float t = 0;
            RF_CUDA(cudaEventElapsedTime(&t, pool[2 * i], pool[2 * i + 1]));
            ms[cls[i]] += t;
            n[cls[i]]++;
        }
        cls.clear();
        used = 0;
    }
    ~Prof() { for (auto e : pool) cudaEventDestroy(e); }
};
#define RF_PROF_B(pf, c, st) do { if (pf) (pf)->begin((c), (st)); } while (0)
#define RF_PROF_E(pf, st) do { if (pf) (pf)->end(st); } while (0)

// ------------------------------------------------------------------------------------------
// kernel launch helpers

// SOR configurations.  A configuration is (K sweeps per launch, NBUF region buffers, ILP lane
// mapping); MINB = 2 CTAs per SM where the shared memory allows it.
static inline int sor_cfg_id(const SorConfig& c) { return (c.K - 1) * 4 + (c.nbuf - 1) * 2 + (c.ilp - 1); }

template <class T, int K, int NB> constexpr bool sor_fits() { return SorGeom<T, K, NB>::smem <= 227 * 1024; }
template <class T, int K, int NB> constexpr int sor_minb() { return SorGeom<T, K, NB>::smem * 2 + 2048 <= 228 * 1024 ? 2 : 1; }

template <class T, class S, int K, int NB, int ILP>
static void launch_sor_k(const LevelItem<T, S>* items, const Tile* tiles, int n, int sms, const SolveConst<T>& k,
                         const SorLaunch& L, cudaStream_t st)
{
    if constexpr (sor_fits<T, K, NB>()) {
        constexpr int MB = sor_minb<T, K, NB>();
        typedef SorGeom<T, K, NB> G;
        k_sor<T, S, K, NB, ILP, MB><<<std::min(n, sms * MB), G::NT, G::smem, st>>>(items, tiles, n, k, L);
    } else {
        throw ArgError(-2, "SOR configuration does not fit shared memory");
    }
}

template <class T, class S, int K>
static void launch_sor_kk(const SorConfig& c, const LevelItem<T, S>* items, const Tile* tiles, int n, int sms,
                          const SolveConst<T>& k, const SorLaunch& L, cudaStream_t st)
{
    if (c.nbuf == 2) {
        if (c.ilp == 2) launch_sor_k<T, S, K, 2, 2>(items, tiles, n, sms, k, L, st);
        else launch_sor_k<T, S, K, 2, 1>(items, tiles, n, sms, k, L, st);
    } else {
        if (c.ilp == 2) launch_sor_k<T, S, K, 1, 2>(items, tiles, n, sms, k, L, st);
        else launch_sor_k<T, S, K, 1, 1>(items, tiles, n, sms, k, L, st);
    }
}

template <class T, class S>
static void launch_sor(const SorConfig& c, const LevelItem<T, S>* items, const Tile* tiles, int n, int sms,
                       const SolveConst<T>& k, const SorLaunch& L, cudaStream_t st)
{
    switch (c.K) {
    case 1: launch_sor_kk<T, S, 1>(c, items, tiles, n, sms, k, L, st); break;
    case 2: launch_sor_kk<T, S, 2>(c, items, tiles, n, sms, k, L, st); break;
    case 3: launch_sor_kk<T, S, 3>(c, items, tiles, n, sms, k, L, st); break;
    case 4: launch_sor_kk<T, S, 4>(c, items, tiles, n, sms, k, L, st); break;
    case 5: launch_sor_kk<T, S, 5>(c, items, tiles, n, sms, k, L, st); break;
    default: launch_sor_kk<T, S, 6>(c, items, tiles, n, sms, k, L, st); break;
    }
}

template <class T, class S>
static void launch_sor_strip(const LevelItem<T, S>* items, const StripUnit* units, int n_units, int grid, int* ticket,
                             const SolveConst<T>& k, const SorLaunch& L, cudaStream_t st)
{
    if constexpr (sizeof(T) == 4) {
        k_sor_strip<T, S><<<grid, kStripNT, strip_smem_bytes<T>(), st>>>(items, units, n_units, ticket, k, L);
    } else {
        throw ArgError(-2, "the strip SOR holds FP32 planes only");
    }
}

template <class T, class S, int K, int NB, int ILP>
static void sor_attr1()
{
    if constexpr (sor_fits<T, K, NB>()) {
        constexpr int MB = sor_minb<T, K, NB>();
        RF_CUDA(cudaFuncSetAttribute(k_sor<T, S, K, NB, ILP, MB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)SorGeom<T, K, NB>::smem));
    }
}
template <class T, class S, int K>
static void sor_attr()
{
    sor_attr1<T, S, K, 1, 1>();
    sor_attr1<T, S, K, 1, 2>();
    sor_attr1<T, S, K, 2, 1>();
    sor_attr1<T, S, K, 2, 2>();
}

template <class T, class S>
static void set_kernel_attrs()
{
    RF_CUDA(cudaFuncSetAttribute(k_linearize<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lin_smem_bytes<T>()));
    sor_attr<T, S, 1>();
    sor_attr<T, S, 2>();
    sor_attr<T, S, 3>();
    sor_attr<T, S, 4>();
    sor_attr<T, S, 5>();
    sor_attr<T, S, 6>();
    if constexpr (sizeof(T) == 4)
        RF_CUDA(cudaFuncSetAttribute(k_sor_strip<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)strip_smem_bytes<T>()));
    RF_CUDA(cudaFuncSetAttribute(k_sor_level<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLevelSmemMax));
    RF_CUDA(cudaFuncSetAttribute(k_sor_level_cluster<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLevelSmemMax));
    if constexpr (sizeof(T) == 4) {
        RF_CUDA(cudaFuncSetAttribute(k_sor_level_reg<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
        RF_CUDA(cudaFuncSetAttribute(k_sor_level_cluster_reg<T, S, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
        RF_CUDA(cudaFuncSetAttribute(k_sor_level_cluster_reg<T, S, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    }
}

// Whether configuration c fits shared memory for type T.
template <class T> static inline bool sor_cfg_fits(const SorConfig& c)
{
    size_t sm = 0;
    switch (c.K) {
    case 1: sm = c.nbuf == 2 ? SorGeom<T, 1, 2>::smem : SorGeom<T, 1, 1>::smem; break;
    case 2: sm = c.nbuf == 2 ? SorGeom<T, 2, 2>::smem : SorGeom<T, 2, 1>::smem; break;
    case 3: sm = c.nbuf == 2 ? SorGeom<T, 3, 2>::smem : SorGeom<T, 3, 1>::smem; break;
    case 4: sm = c.nbuf == 2 ? SorGeom<T, 4, 2>::smem : SorGeom<T, 4, 1>::smem; break;
    case 5: sm = c.nbuf == 2 ? SorGeom<T, 5, 2>::smem : SorGeom<T, 5, 1>::smem; break;
    default: sm = c.nbuf == 2 ? SorGeom<T, 6, 2>::smem : SorGeom<T, 6, 1>::smem; break;
    }
    return sm <= 227 * 1024;
}

// The level loop of one step (sceneFlowSingleScale's outer / inner / SOR structure, .cu:755-954).
template <class T, class S>
static int enqueue_level(const Plan<T, S>& P, char* base, int sidx, cudaStream_t st, int setup, Prof* pf)
{
    const auto& d = P.steps[sidx];
    if (d.n_items == 0) return 0;
    int launches = 0;
    const LevelItem<T, S>* items = (const LevelItem<T, S>*)(base + P.desc_off + d.items_off);
    const Tile* lt = (const Tile*)(base + P.desc_off + d.lin_tiles_off);
    const Tile* stt = (const Tile*)(base + P.desc_off + d.sor_tiles_off);
    const StripUnit* units = (const StripUnit*)(base + P.desc_off + d.strip_units_off);
    const int* level_items = (const int*)(base + P.desc_off + d.level_items_off);
    int* ticket = (int*)(base + P.ctr_off) + sidx;
    int seq = 0;
    const SolveConst<T> k = solve_const<T>(P.hp);
    if (setup) {
        RF_PROF_B(pf, KC_SETUP, st);
        k_level_setup<T, S><<<d.n_lin, LTW * LTH, 0, st>>>(items, lt, P.hp.regularization);
        RF_PROF_E(pf, st);
        launches++;
    }
    // a step whose items are all on the whole-level kernels runs the control in those kernels
    const bool fold_control = !d.n_sor && !d.n_units && (d.n_level || d.n_clus);
    for (int outer = 0; outer < P.hp.n_outer; outer++) {
        for (int hh = 0; hh < P.hp.n_inner; hh++) {
            const auto& sched = P.sor_sched[sidx][hh];
            // inner iterations after the first read the running increment (x of the previous SOR)
            const int xsel = sched.front().xin;
            RF_PROF_B(pf, KC_LIN, st);
            k_linearize<T, S><<<d.n_lin, LTW * LTH, lin_smem_bytes<T>(), st>>>(items, lt, k, hh > 0, xsel);
            RF_PROF_E(pf, st);
            launches++;
            const int lvl = P.Lmax - 1 - sidx;
            if (d.n_level) {
                // the whole-level items: every SOR iteration of this inner iteration in one launch
                SorLaunch L{};
                L.it0 = 0; L.nit = P.hp.n_sor; L.outer = outer;
                L.xin = sched.front().xin;
                L.xin_zero = (hh == 0);
                L.final_fold = (hh == P.hp.n_inner - 1);
                L.xout = L.final_fold ? 0 : P.sor_sched[sidx][hh + 1].front().xin;
                L.control = fold_control && L.final_fold;
                L.n_checks = P.n_checks[sidx].back();
                RF_PROF_B(pf, KC_SOR_LEVEL0 + lvl, st);
                if constexpr (sizeof(T) == 4) {
                    if (d.level_reg)
                        k_sor_level_reg<T, S><<<d.n_level, d.level_threads, d.level_smem, st>>>(items, level_items, k, L);
                    else
                        k_sor_level<T, S><<<d.n_level, d.level_threads, d.level_smem, st>>>(items, level_items, k, L);
                } else {
                    k_sor_level<T, S><<<d.n_level, d.level_threads, d.level_smem, st>>>(items, level_items, k, L);
                }
                RF_PROF_E(pf, st);
                launches++;
            }
            if (d.n_clus) {
                // the same, each item over a cluster of row bands
                SorLaunch L{};
                L.it0 = 0; L.nit = P.hp.n_sor; L.outer = outer;
                L.xin = sched.front().xin;
                L.xin_zero = (hh == 0);
                L.final_fold = (hh == P.hp.n_inner - 1);
                L.xout = L.final_fold ? 0 : P.sor_sched[sidx][hh + 1].front().xin;
                L.control = fold_control && L.final_fold;
                L.n_checks = P.n_checks[sidx].back();
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3(d.n_clus * d.clus_c);
                cfg.blockDim = dim3(d.clus_threads);
                cfg.dynamicSmemBytes = d.clus_smem;
                cfg.stream = st;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeClusterDimension;
                at[0].val.clusterDim.x = d.clus_c;
                at[0].val.clusterDim.y = 1;
                at[0].val.clusterDim.z = 1;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                RF_PROF_B(pf, KC_SOR_LEVEL0 + lvl, st);
                const int* ci = (const int*)(base + P.desc_off + d.clus_items_off);
                if constexpr (sizeof(T) == 4) {
                    if (d.clus_kp == 1)
                        RF_CUDA(cudaLaunchKernelEx(&cfg, k_sor_level_cluster_reg<T, S, 1>, items, ci, k, L));
                    else if (d.clus_kp == 2)
                        RF_CUDA(cudaLaunchKernelEx(&cfg, k_sor_level_cluster_reg<T, S, 2>, items, ci, k, L));
                    else
                        RF_CUDA(cudaLaunchKernelEx(&cfg, k_sor_level_cluster<T, S>, items, ci, k, L));
                } else {
                    RF_CUDA(cudaLaunchKernelEx(&cfg, k_sor_level_cluster<T, S>, items, ci, k, L));
                }
                RF_PROF_E(pf, st);
                launches++;
            }
            for (SorLaunch L : sched) {
                L.outer = outer;
                L.seq = seq++;
                if (!d.n_sor && !d.n_units) continue;
                RF_PROF_B(pf, KC_SOR_LEVEL0 + lvl, st);
                if (d.n_sor) {
                    launch_sor<T, S>(P.sor_cfg[sidx], items, stt, d.n_sor, P.sms, k, L, st);
                    launches++;
                }
                if (d.n_units) {
                    launch_sor_strip<T, S>(items, units, d.n_units, d.strip_grid, ticket, k, L, st);
                    launches++;
                }
                RF_PROF_E(pf, st);
            }
        }
        if (!fold_control) {
            const int wpb = 4;
            RF_PROF_B(pf, KC_CTL, st);
            k_control<T, S><<<(d.n_items + wpb - 1) / wpb, 32 * wpb, 0, st>>>(items, d.n_items, k, outer,
                                                                              P.n_checks[sidx].back());
            RF_PROF_E(pf, st);
            launches++;
        }
    }
    return launches;
}

// Launches a cooperative kernel (every block resident: its blocks meet at grid barriers).
template <class K, class... A>
static void launch_cooperative(K kernel, int grid, int block, cudaStream_t st, A... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    RF_CUDA(cudaLaunchKernelEx(&cfg, kernel, args...));
}

// The HPB regularisation weights of every level (sceneFlowMultiscale.cpp:79-83, 114-116): the
// colour-guided fill of frame 1's raw depth, its DepthMapPyramid, then computeHeuristicPb per
// level into the levels' regularisation weights.
template <class T, class S>
static int enqueue_hpb(const Plan<T, S>& P, char* base, cudaStream_t st, Prof* pf)
{
    int launches = 0;
    char* db = base + P.desc_off;
    const HpbFill<T>* fills = (const HpbFill<T>*)(db + P.hpb_fill_off);
    RF_PROF_B(pf, KC_HPB, st);
    {
        static int per_sm = 0;
        if (!per_sm) RF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hpb_fill<T>, 128, 0));
        const int grid = std::max(1, std::min(per_sm, 4) * P.sms);
        GridSync* gs = (GridSync*)(base + P.hpb_ctr_off + sizeof(int) * 2 * P.n);
        launch_cooperative(k_hpb_fill<T>, grid, 128, st, fills, P.n, gs, 4096, P.status);
        launches++;
    }
    for (const auto& lv : P.hpb_dpyr) {
        if (!lv.n_tiles) continue;
        k_depth_pyr<T><<<lv.n_tiles, LTW * LTH, 0, st>>>((const DepthPyrJob<T>*)(db + lv.jobs_off),
                                                        (const Tile*)(db + lv.tiles_off));
        launches++;
    }
    for (int sidx = 0; sidx < P.Lmax; sidx++) {
        const auto& d = P.steps[sidx];
        const auto& h = P.hpb_step[sidx];
        if (!h.n_items) continue;
        const HpbItem<T>* items = (const HpbItem<T>*)(db + h.items_off);
        const Tile* lt = (const Tile*)(db + d.lin_tiles_off);
        k_hpb_normals<T><<<d.n_lin, LTW * LTH, 0, st>>>(items, lt);
        k_hpb_rowsum<T><<<(h.row_threads + 127) / 128, 128, 0, st>>>(items, (const int*)(db + h.row_first_off), h.n_items);
        k_hpb_colsum<T><<<(h.col_threads + 127) / 128, 128, 0, st>>>(items, (const int*)(db + h.col_first_off), h.n_items);
        k_hpb_halfdisk<T><<<d.n_lin, LTW * LTH, 0, st>>>(items, lt);
        k_hpb_prob<T><<<d.n_lin, LTW * LTH, 0, st>>>(items, lt);
        k_hpb_nms<T><<<d.n_lin, LTW * LTH, 0, st>>>(items, lt);
        launches += 6;
    }
    RF_PROF_E(pf, st);
    return launches;
}

// Whole solve after the inputs are resident: preprocessing, hole fill, pyramids, levels, output.
// outs: the output-pointer array the final kernels write through (device memory).
template <class T, class S>
static int enqueue_solve(const Plan<T, S>& P, char* base, cudaStream_t st, Prof* pf = nullptr)
{
    int launches = 0;
    char* db = base + P.desc_off;
    RF_CUDA(cudaMemsetAsync(base + P.ctl_off, 0, P.ctr_off + sizeof(int) * 16 - P.ctl_off, st));  // ctl + tickets
    const auto& fin = P.steps.back();
    const LevelItem<T, S>* fin_items = (const LevelItem<T, S>*)(db + fin.items_off);
    const Tile* fin_tiles = (const Tile*)(db + fin.lin_tiles_off);
    if (P.kind == 2) {
        RF_PROF_B(pf, KC_SETUP, st);
        k_seam_load<T, S><<<fin.n_lin, LTW * LTH, 0, st>>>(fin_items, fin_tiles, (const SeamSrc*)(db + P.seam_src_off));
        RF_PROF_E(pf, st);
        launches++;
        launches += enqueue_level(P, base, P.Lmax - 1, st, 0, pf);
        RF_PROF_B(pf, KC_OUT, st);
        k_warp_out<T, S><<<fin.n_lin, LTW * LTH, 0, st>>>(fin_items, fin_tiles, (T* const*)(db + P.out_ptrs_off));
        RF_PROF_E(pf, st);
        launches++;
    } else {
        RF_CUDA(cudaMemsetAsync(base + P.unfilled_off, 0, sizeof(int) * 256 + sizeof(GridSync), st));
        if (P.hpb) RF_CUDA(cudaMemsetAsync(base + P.hpb_ctr_off, 0, sizeof(int) * 2 * P.n + sizeof(GridSync), st));
        const PrepItem<T>* prep = (const PrepItem<T>*)(db + P.prep_items_off);
        const Tile* pt = (const Tile*)(db + P.prep_tiles_off);
        RF_PROF_B(pf, KC_PREP, st);
        k_prep<T><<<P.n_prep_tiles, LTW * LTH, 0, st>>>(prep, pt);
        RF_PROF_E(pf, st);
        RF_PROF_B(pf, KC_SIGMA, st);
        k_sigma<T><<<P.n_prep_tiles, LTW * LTH, 0, st>>>(prep, pt);
        RF_PROF_E(pf, st);
        launches += 2;
        if (P.hp.fill_holes) {
            // one cooperative launch runs every round (grid barriers between rounds)
            static int per_sm[2] = {0, 0};
            int& occ = per_sm[sizeof(T) == 8];
            if (!occ) RF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fill<T>, LTW * LTH, 0));
            const int grid = std::max(1, std::min(P.n_prep_tiles, std::min(occ, 8) * P.sms));
            int* left = (int*)(base + P.unfilled_off);
            GridSync* gs = (GridSync*)(left + 256);
            int* tleft = (int*)(base + P.tleft_off);
            RF_PROF_B(pf, KC_FILL, st);
            launch_cooperative(k_fill<T>, grid, LTW * LTH, st, prep, pt, P.n_prep_tiles, left, tleft, gs, P.hp.fill_rounds,
                               P.status);
            RF_PROF_E(pf, st);
            launches++;
        }
        for (const auto& lv : P.pyr) {
            const PyrJob<T>* jobs = (const PyrJob<T>*)(db + lv.jobs_off);
            const T* g = (const T*)(db + lv.g_off);
            RF_PROF_B(pf, KC_PYR_H, st);
            k_hfilter<T><<<dim3(lv.n_src, 10), LTW * LTH, 0, st>>>(jobs, (const Tile*)(db + lv.src_tiles_off), g);
            RF_PROF_E(pf, st);
            RF_PROF_B(pf, KC_PYR_V, st);
            k_vresize<T><<<dim3(lv.n_dst, (10 + kVresizePlanes - 1) / kVresizePlanes), LTW * LTH, 0, st>>>(jobs, (const Tile*)(db + lv.dst_tiles_off), g);
            RF_PROF_E(pf, st);
            launches += 2;
        }
        if (P.hpb) launches += enqueue_hpb(P, base, st, pf);
        if (P.any_warm) {
            RF_PROF_B(pf, KC_MISC, st);
            k_load_est<T, S><<<fin.n_lin, LTW * LTH, 0, st>>>(fin_items, fin_tiles, (const EstSrc*)(db + P.est_src_off));
            RF_PROF_E(pf, st);
            launches++;
        }
        for (int s = 0; s < P.Lmax; s++) launches += enqueue_level(P, base, s, st, 1, pf);
    }
    RF_PROF_B(pf, KC_OUT, st);
    k_output<T, S><<<fin.n_lin, LTW * LTH, 0, st>>>(fin_items, fin_tiles, (T* const*)(db + P.out_ptrs_off));
    RF_PROF_E(pf, st);
    launches++;
    RF_CUDA(cudaGetLastError());
    return launches;
}

// Algorithmic bytes of the work a solve actually executed (early exits included), per class:
//   SOR: per level pixel and executed iteration, the 12-float system (48 B) read plus the
//        3-float increment read and written (24 B) = 72 B; plus, once per outer iteration, the
//        fold u += x (u read and written, 24 B).
//   linearisation: per level pixel and execution, 20 input values (5 + 5 features, 2 depths,
//        3 flow, 5 weights; the 12 feature/depth values in the storage type) plus the 12-float
//        system written.
template <class T, class S>
static void executed_bytes(const Plan<T, S>& P, const PairCtl* ctl, double* sor_bytes, double* lin_bytes,
                           double* sor_level = nullptr)
{
    *sor_bytes = 0;
    *lin_bytes = 0;
    if (sor_level)
        for (int k = 0; k < 16; k++) sor_level[k] = 0;
    const double lin_px = 12.0 * sizeof(S) + 8.0 * sizeof(T) + 12.0 * sizeof(T);
    for (int p = 0; p < P.n; p++)
        for (int k = 0; k < P.L[p]; k++) {
            const double N = (double)P.shapes[p].w[k] * P.shapes[p].h[k];
            const int O = std::min(ctl[p].outer_exec[k], 64);
            for (int o = 0; o < O; o++) {
                const double b = N * (ctl[p].sor_exec[k][o] * 72.0 * sizeof(T) / 4.0 + 24.0 * sizeof(T) / 4.0);
                *sor_bytes += b;
                if (sor_level) sor_level[k] += b;
                *lin_bytes += N * lin_px * P.hp.n_inner;
            }
        }
}

}  // namespace rgbdflow
