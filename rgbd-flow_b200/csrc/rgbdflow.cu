// rgbdflow.cu — C ABI (include/rgbdflow.h) over the sm_100a scene-flow pipeline.
//
// Host orchestration is C++; every arithmetic step of the solve runs in the kernels of
// kernels.cuh.  There is no CPU fallback: without a CUDA device every entry point that computes
// returns RGBDFLOW_ERR_NO_DEVICE.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <set>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include <type_traits>

#include "../../include/rgbdflow.h"
#include "pipeline.cuh"
#include "server.cuh"
#include "flo3.h"
#include "flow2d.cuh"

using namespace rgbdflow;

struct GraphEntry {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int launches = 0;
    std::string topo;       // its launch topology (executables of one topology can be updated in place)
    uint64_t last_use = 0;  // for least-recently-used eviction
};
constexpr size_t kGraphCache = 48;  // executable graphs kept per context

// Where the last solve's planes live, per pair and level (rgbdflow_debug_read_plane).
struct DbgLevel {
    int W = 0, H = 0, pitch = 0, hwp = 0;
    const void* pyr[10];
    const void* I1[5];
    const void* I2[5];
    const void* D[2];
    const void* mag;
    const void* reg[2];
    const void* u[3];
    const void* sys[12];
    const void* hz;  // HPB raw-depth pyramid level (null without HPB)
};
struct DbgPair {
    std::vector<DbgLevel> lev;
    const void* stamp[2] = {nullptr, nullptr};
};

struct rgbdflow_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    size_t budget = 0;
    std::string err;
    char* arena = nullptr;
    size_t arena_cap = 0;
    char* pin = nullptr;
    size_t pin_cap = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::map<std::string, GraphEntry> graphs;  // by exact batch (sizes, cameras, parameters)
    uint64_t graph_clock = 0;
    uint64_t n_graph_builds = 0, n_arena_grows = 0;  // captures and arena reallocations, for counters
    double max_build_ms = 0;                            // longest capture + instantiation, for counters
    bool attrs[4] = {false, false, false, false};
    int last_launches = 0;
    int sms = 148;
    bool use_graphs = true;
    // ordering of work that reuses the arena / pinned staging across calls and streams
    cudaEvent_t done = nullptr;       // end of the last enqueued solve
    cudaEvent_t desc_up = nullptr;    // last upload out of the pinned staging
    bool pending = false;
    // bounded device waits that gave up: a sticky device word (the kernels OR into it; [4..] is the
    // wait self-test's barrier) and its page-locked copy, read once a solve has finished
    int* dev_status = nullptr;
    int* pin_status = nullptr;
    // kernel profiling
    std::unique_ptr<Prof> prof;
    double prof_ms[KC_TOTAL] = {0};
    int prof_n[KC_TOTAL] = {0};
    double prof_bytes[KC_TOTAL] = {0};
    // the last solve's layout (stage read-back)
    std::vector<DbgPair> dbg;
    int dbg_tsize = 4;  // bytes of the arithmetic type T
    int dbg_store = 0;  // storage type of the features / depths: 0 FP32, 1 FP16, 2 BF16, 3 FP64
};

namespace {

void drop_graphs(rgbdflow_ctx* c)
{
    for (auto& kv : c->graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    c->graphs.clear();
}

// page-locked (cudaMallocHost / cudaHostRegister) host memory can be copied by DMA directly
bool is_pinned(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return a.type == cudaMemoryTypeHost;
}

void wait_idle(rgbdflow_ctx* c)
{
    if (c->pending) RF_CUDA(cudaEventSynchronize(c->done));
    RF_CUDA(cudaStreamSynchronize(c->stream));
    c->pending = false;
}

// The status finished solves left in the page-locked copy: a bounded device wait that gave up
// makes the call fail with RGBDFLOW_ERR_TIMEOUT, once; the device word is cleared for the next.
void check_status(rgbdflow_ctx* c)
{
    if (!*c->pin_status) return;
    *c->pin_status = 0;
    RF_CUDA(cudaMemsetAsync(c->dev_status, 0, sizeof(int), c->stream));
    RF_CUDA(cudaStreamSynchronize(c->stream));
    throw ArgError(RGBDFLOW_ERR_TIMEOUT, "a bounded device wait (grid barrier) gave up: the solve's results are not valid");
}

void ensure_arena(rgbdflow_ctx* c, size_t need)
{
    if (c->arena_cap >= need) return;
    if (c->budget && need > c->budget)
        throw ArgError(RGBDFLOW_ERR_BUDGET, "request needs " + std::to_string(need) + " device bytes, budget is " +
                                                std::to_string(c->budget));
    wait_idle(c);
    drop_graphs(c);  // graphs hold arena addresses
    if (c->arena) RF_CUDA(cudaFree(c->arena));
    c->arena = nullptr;
    c->arena_cap = 0;
    // grow at least 2x: a server's batches grow step by step, and every reallocation waits for the
    // device and drops the cached graphs
    const size_t cap = align_up(std::max(need + need / 8, 2 * c->arena_cap), 1 << 20);
    const size_t want = (c->budget && cap > c->budget) ? need : cap;
    RF_CUDA(cudaMalloc(&c->arena, want));
    c->n_arena_grows++;
    c->arena_cap = want;
}

void ensure_pin(rgbdflow_ctx* c, size_t need)
{
    if (c->pin_cap >= need) return;
    wait_idle(c);
    if (c->pin) RF_CUDA(cudaFreeHost(c->pin));
    c->pin = nullptr;
    const size_t cap = align_up(need + need / 8, 1 << 20);
    RF_CUDA(cudaMallocHost(&c->pin, cap));
    c->pin_cap = cap;
}

HostParams host_params(const rgbdflow_params& p)
{
    HostParams h;
    h.regularization = p.regularization;
    h.color_w = p.color_data_weight; h.dvc = p.depth_vs_color_data_weight;
    h.alpha = p.alpha; h.gamma = p.gamma; h.ratio = p.pyramid_ratio;
    h.min_width = p.min_width; h.n_outer = p.n_outer; h.n_inner = p.n_inner; h.n_sor = p.n_sor;
    h.max_dist = p.depth_boundary_dist; h.fill_holes = p.fill_holes; h.fixed = p.fixed_schedule;
    h.omega = p.omega; h.step = p.max_flow_step; h.eps_d = p.eps_d; h.eps_z = p.eps_z; h.eps_s = p.eps_s;
    h.sor_tol = p.sor_tol; h.outer_tol = p.outer_tol; h.occ_margin = p.occ_margin; h.occ_penalty = p.occ_penalty;
    h.max_grad = p.max_depth_grad;
    h.period = p.sor_check_period > 0 ? p.sor_check_period : 25;
    h.K = p.sweeps_per_launch > 0 ? std::min(p.sweeps_per_launch, 6) : 0;  // 0: chosen per level
    const char* e = std::getenv("RGBDFLOW_SOR_ILP");
    h.sor_ilp = e ? std::atoi(e) : 0;
    e = std::getenv("RGBDFLOW_SOR_NBUF");
    h.sor_nbuf = e ? std::atoi(e) : 0;
    e = std::getenv("RGBDFLOW_SOR_STRIP");
    h.sor_strip = e ? std::atoi(e) : 1;
    e = std::getenv("RGBDFLOW_STRIP_MIN_W");
    h.strip_min_w = e ? std::atoi(e) : 0;
    e = std::getenv("RGBDFLOW_STRIP_MIN_H");
    h.strip_min_h = e ? std::atoi(e) : 0;
    e = std::getenv("RGBDFLOW_STRIP_SEG");
    h.strip_seg = e ? std::atoi(e) : 0;
    e = std::getenv("RGBDFLOW_STRIP_MIN_PX");
    h.strip_min_px = e ? std::atol(e) : 0;
    e = std::getenv("RGBDFLOW_STRIP_BALANCED");
    h.strip_balanced = e ? std::atoi(e) : 0;
    e = std::getenv("RGBDFLOW_SOR_LEVEL");
    h.sor_level = e ? std::atoi(e) : 1;
    e = std::getenv("RGBDFLOW_LEVEL_CLUSTER");
    h.level_cluster = e ? std::atoi(e) : 0;
    e = std::getenv("RGBDFLOW_LEVEL_REG");
    h.level_reg = e ? std::atoi(e) : 1;
    h.fill_rounds = 253;  // round stamps are bytes: 0 valid, 1..253 rounds, 254 outside, 255 unfilled
    return h;
}

void validate(const rgbdflow_params* p)
{
    if (!p) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "params is NULL");
    if (p->regularization != RGBDFLOW_REG_ISOTROPIC && p->regularization != RGBDFLOW_REG_LETOUZEY &&
        p->regularization != RGBDFLOW_REG_HPB)
        throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "unknown regularisation type");
    if (p->n_outer < 0 || p->n_inner < 1 || p->n_sor < 0) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "bad iteration counts");
    if (p->n_outer > 64) throw ArgError(RGBDFLOW_ERR_UNSUPPORTED, "n_outer > 64");
    const int period = p->sor_check_period > 0 ? p->sor_check_period : 25;
    if (!p->fixed_schedule && p->n_sor / period > kMaxChecks)
        throw ArgError(RGBDFLOW_ERR_UNSUPPORTED, "more than 512 SOR convergence checks per inner iteration");
    if (p->storage < 0 || p->storage > 2) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "bad storage type");
    if (p->compute == RGBDFLOW_COMPUTE_FP64 && p->storage != RGBDFLOW_STORE_FP32)
        throw ArgError(RGBDFLOW_ERR_UNSUPPORTED, "the FP64 device solve stores its pyramids in FP64");
    if (p->min_width == 0) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "min_width == 0");
}

// getResizedCamParams (runFlowTwoFrames.cpp:14-24)
void resized_cam(const rgbdflow_camera_params& c, int W, float& f, unsigned& xres)
{
    const double sf = (double)W / c.xRes;
    xres = (unsigned)std::rint(c.xRes * sf);
    f = (float)(c.focalLength * sf);
}

std::string plan_key(const std::vector<PairSpec>& ps, const HostParams& hp, int tag)
{
    std::string k = std::to_string(tag) + ":";
    // cameras are left out: they reach the kernels only through the item descriptors, which every
    // call uploads, so batches that differ only in their cameras share one graph
    for (const auto& p : ps)
        k += std::to_string(p.kind) + "k" + std::to_string(p.W) + "x" + std::to_string(p.H) + (p.warm() ? (p.warm_early ? "E" : "e") : "") +
             (p.kind == 2 ? "a" + std::to_string(p.allow_early) : std::string()) + ",";
    char buf[512];
    std::snprintf(buf, sizeof buf, "|%d %.17g %.17g %.17g %.17g %.17g %d %d %d %d %d %d %d %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %d %d %d",
                  hp.regularization, hp.color_w, hp.dvc, hp.alpha, hp.gamma, hp.ratio, hp.min_width, hp.n_outer, hp.n_inner,
                  hp.n_sor, hp.max_dist, hp.fill_holes, hp.fixed, hp.omega, hp.step, hp.eps_d, hp.eps_z, hp.eps_s,
                  hp.sor_tol, hp.outer_tol, hp.occ_margin, hp.occ_penalty, hp.max_grad, hp.period, hp.K * 100 + hp.sor_ilp * 10 + hp.sor_nbuf, hp.fill_rounds);
    k += buf;
    std::snprintf(buf, sizeof buf, " strip %d %d %d %d %ld %d level %d %d %d", hp.sor_strip, hp.strip_min_w, hp.strip_min_h,
                  hp.strip_seg, hp.strip_min_px, hp.strip_balanced, hp.sor_level, hp.level_cluster, hp.level_reg);
    return k + buf;
}

// What decides the sequence of launches (and so the shape of a captured graph), without the
// pair sizes: the kind of solve, level count, which steps have pairs, hole fill, warm starts,
// the SOR configuration per step and every parameter of the schedule.
template <class T, class S>
std::string topo_key(const Plan<T, S>& P, const HostParams& hp, int tag, bool dev)
{
    std::string k = std::to_string(tag) + (dev ? "d" : "h") + std::to_string(P.kind) + "L" + std::to_string(P.Lmax) +
                    "p" + std::to_string(P.pyr.size()) + "w" + std::to_string((int)P.any_warm) + "s";
    for (size_t i = 0; i < P.steps.size(); i++)
        k += std::to_string(P.steps[i].n_items > 0) + std::to_string(P.sor_cfg[i].K) + std::to_string(P.sor_cfg[i].nbuf) +
             std::to_string(P.sor_cfg[i].ilp) + (P.steps[i].n_sor > 0 ? "t" : "") + (P.steps[i].n_units > 0 ? "s" : "") +
             (P.steps[i].n_level > 0 ? "l" : "") + (P.steps[i].n_clus > 0 ? "c" + std::to_string(P.steps[i].clus_c) + "r" + std::to_string(P.steps[i].clus_kp) : "") + ".";
    const std::vector<PairSpec> none;
    return k + plan_key(none, hp, tag);
}

void fill_stats(const PairCtl& c, int L, const PyrShape& s, double ms, rgbdflow_stats* st)
{
    std::memset(st, 0, sizeof(*st));
    st->n_levels = L;
    for (int k = 0; k < L && k < RGBDFLOW_MAX_LEVELS; k++) {
        st->level_w[k] = s.w[k];
        st->level_h[k] = s.h[k];
        st->outer_iters[k] = c.outer_exec[k];
        for (int o = 0; o < RGBDFLOW_MAX_OUTER; o++) {
            const bool ran = o < c.outer_exec[k];
            st->sor_iters[k][o] = ran ? c.sor_exec[k][o] : 0;
            st->outer_stat[k][o] = ran ? c.stat[k][o] : -1.0f;
            st->sor_maxdiff[k][o] = ran ? c.sor_maxdiff[k][o] : -1.0f;
        }
    }
    st->device_ms = ms;
}

// Records where plan P (bound to the arena) keeps every plane, for rgbdflow_debug_read_plane.
template <class T, class S>
void record_layout(rgbdflow_ctx* c, const Plan<T, S>& P)
{
    c->dbg.assign(P.n, DbgPair());
    c->dbg_tsize = (int)sizeof(T);
    c->dbg_store = sizeof(S) == 8 ? 3 : (sizeof(S) == 4 ? 0 : (std::is_same<S, __half>::value ? 1 : 2));
    const unsigned char* d = P.desc.data();
    const PrepItem<T>* prep = (const PrepItem<T>*)(d + P.prep_items_off);
    for (int p = 0; p < P.n; p++) {
        c->dbg[p].lev.resize(P.L[p]);
        c->dbg[p].stamp[0] = prep[p].stamp[0];
        c->dbg[p].stamp[1] = prep[p].stamp[1];
    }
    for (int sidx = 0; sidx < P.Lmax; sidx++) {
        const int k = P.Lmax - 1 - sidx;
        const LevelItem<T, S>* it = (const LevelItem<T, S>*)(d + P.steps[sidx].items_off);
        int q = 0;  // items of a step are its pairs in batch order
        for (int p = 0; p < P.n; p++) {
            if (k >= P.L[p]) continue;
            const LevelItem<T, S>& x = it[q++];
            DbgLevel& L = c->dbg[p].lev[k];
            L.W = x.W; L.H = x.H; L.pitch = x.pitch; L.hwp = x.hwp;
            for (int z = 0; z < 10; z++) L.pyr[z] = x.pyr[z];
            for (int z = 0; z < 5; z++) { L.I1[z] = x.I1[z]; L.I2[z] = x.I2[z]; }
            L.D[0] = x.D1; L.D[1] = x.D2;
            L.mag = x.mag; L.reg[0] = x.rh; L.reg[1] = x.rv;
            for (int z = 0; z < 3; z++) L.u[z] = x.u[z];
            for (int z = 0; z < 12; z++) L.sys[z] = x.sys[z];
            L.hz = nullptr;
        }
    }
    if (P.hpb) {
        for (int sidx = 0; sidx < P.Lmax; sidx++) {
            const int k = P.Lmax - 1 - sidx;
            const HpbItem<T>* hi = (const HpbItem<T>*)(d + P.hpb_step[sidx].items_off);
            int q = 0;
            for (int p = 0; p < P.n; p++)
                if (k < P.L[p]) c->dbg[p].lev[k].hz = hi[q++].z;
        }
    }
}

template <class T, class S>
void ensure_attrs(rgbdflow_ctx* c, int slot)
{
    if (c->attrs[slot]) return;
    set_kernel_attrs<T, S>();
    c->attrs[slot] = true;
}

// Key of a batch's executable graph: the exact batch (sizes, kinds, warm starts, parameters), the
// storage slot and the input form.
std::string graph_key(const std::vector<PairSpec>& pairs, const HostParams& hp, int slot, bool dev,
                      const std::string& tune_desc)
{
    return plan_key(pairs, hp, slot) + (dev ? "|dev" : "") + "|" + tune_desc;
}

// The executable graph of plan P (bound to the context's arena) for `pairs`: from the cache, or
// captured on the context's stream now, without running it.  One executable graph per exact
// batch, least recently used evicted beyond kGraphCache: recurring batch mixes (a server's)
// launch without any capture.  When the cache is full a new batch is written into an evicted
// executable of the same launch topology (cudaGraphExecUpdate: new grids and arguments, no
// re-instantiation) where one exists.
template <class T, class S>
GraphEntry& graph_for(rgbdflow_ctx* c, const Plan<T, S>& P, const std::vector<PairSpec>& pairs, const HostParams& hp,
                      int slot, bool dev)
{
    const std::string exact = graph_key(pairs, hp, slot, dev, P.tune_desc);
    auto it = c->graphs.find(exact);
    if (it == c->graphs.end()) {
        MaxTimer timer(&c->max_build_ms);
        const std::string topo = topo_key(P, hp, slot, dev);
        cudaGraph_t graph = nullptr;
        RF_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        int launches = 0;
        try {
            launches = enqueue_solve(P, c->arena, c->stream);
        } catch (...) {
            cudaGraph_t tmp = nullptr;
            cudaStreamEndCapture(c->stream, &tmp);
            if (tmp) cudaGraphDestroy(tmp);
            throw;
        }
        RF_CUDA(cudaStreamEndCapture(c->stream, &graph));
        c->n_graph_builds++;
        GraphEntry g;
        g.graph = graph;
        g.topo = topo;
        g.launches = launches;
        bool updated = false;
        if (c->graphs.size() >= kGraphCache) {
            // the victim: the least recently used executable of this topology, else of any
            auto victim = c->graphs.end();
            for (auto j = c->graphs.begin(); j != c->graphs.end(); ++j) {
                const bool same = j->second.topo == topo;
                if (victim == c->graphs.end() || (same && victim->second.topo != topo) ||
                    (same == (victim->second.topo == topo) && j->second.last_use < victim->second.last_use))
                    victim = j;
            }
            GraphEntry old = victim->second;
            c->graphs.erase(victim);
            cudaGraphExecUpdateResultInfo info;
            if (old.topo == topo && cudaGraphExecUpdate(old.exec, graph, &info) == cudaSuccess) {
                g.exec = old.exec;
                updated = true;
            } else {
                cudaGetLastError();
                cudaGraphExecDestroy(old.exec);
            }
            cudaGraphDestroy(old.graph);
        }
        if (!updated) RF_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
        it = c->graphs.emplace(exact, g).first;
    }
    return it->second;
}

// ------------------------------------------------------------------------------------------
// SOR autotuner.  The first time a level step with given item sizes is planned, every candidate
// SOR configuration of that step (tile kernel with K = 2..6 sweeps per launch and either lane
// mapping; strip kernel with K = 5, bands of 64, 96 and 128 rows and the layout of the balancing
// model strip_balanced_bands, where the items allow strips) runs a few launches on the context's
// stream over the step's real descriptors, timed with CUDA events, and the fastest per SOR
// iteration is kept.  Every configuration computes the same flow bit for bit, so the choice
// changes speed only.  Convergence checks are off during timing; each candidate is timed with
// every pair active, with every other pair's SOR stopped and with every other pair done with the
// level (the pairs that converge early in a real solve), and the mean counts.  The planes the
// timing launches overwrite (the increment ping-pong, control blocks, tickets) are reset by the
// next solve.  The table is kept per device for the life of the process.  RGBDFLOW_AUTOTUNE=0
// turns it off (the measured defaults of choose_sor_config / use_strip are used).

struct TuneState {
    std::mutex mu;
    TuneTable table[64];                  // per device
    std::set<std::string> complete[64];   // per device: batches (plan_key) whose every step is tuned
};
TuneState& tune_state()
{
    static TuneState s;
    return s;
}
bool autotune_enabled()
{
    static const bool on = [] {
        const char* e = std::getenv("RGBDFLOW_AUTOTUNE");
        return !(e && std::atoi(e) == 0);
    }();
    return on;
}

template <class T, class S>
std::vector<SorChoice> sor_candidates(const Plan<T, S>& P, int sidx)
{
    std::vector<SorChoice> v;
    for (int K = 2; K <= 6; K++)
        for (int ilp = 1; ilp <= 2; ilp++) {
            SorConfig c;
            c.K = K; c.ilp = ilp; c.nbuf = 1;
            if (!sor_cfg_fits<T>(c)) continue;
            SorChoice ch;
            ch.strip = 0; ch.K = K; ch.ilp = ilp;
            v.push_back(ch);
        }
    const LevelItem<T, S>* it = (const LevelItem<T, S>*)(P.desc.data() + P.steps[sidx].items_off);
    std::vector<LevelItem<T, S>> items(it, it + P.steps[sidx].n_items);
    std::vector<int> which;
    for (int i = 0; i < (int)items.size(); i++)
        if (strip_ok<T>(P.hp, items[i].W, items[i].H)) which.push_back(i);
    if (!which.empty() && sizeof(T) == 4) {
        // bands of 64, 96 and 128 rows (larger bands time faster with every pair active but balance
        // the SMs worse once pairs stop early: measured on 16 x 640x480, 128 rows 14.8 ms of level-0
        // SOR a solve, 192 rows 15.2, 64 rows 15.7), and the layout of the balancing model
        for (int seg : {64, 96, 128}) {
            SorChoice ch;
            ch.strip = 1; ch.K = kStripMaxNit; ch.ilp = 2; ch.seg = seg;
            v.push_back(ch);
        }
        SorChoice ch;
        ch.strip = 1; ch.K = kStripMaxNit; ch.ilp = 2; ch.seg = 128;
        ch.bands = strip_balanced_bands(items, which, 128, P.sms > 0 ? P.sms : 148);
        bool differs = false;
        for (const auto& e : ch.bands) differs = differs || e.second != strip_default_bands(e.first, 128);
        if (differs) v.push_back(ch);
    }
    return v;
}

// Tunes every untuned step of the batch's plan (synchronous on the context's stream).
template <class T, class S>
void tune_sor(rgbdflow_ctx* c, const std::vector<PairSpec>& pairs, const HostParams& hp)
{
    if (!autotune_enabled() || !sor_tunable(hp) || !c->use_graphs) return;
    TuneState& ts = tune_state();
    std::lock_guard<std::mutex> lk(ts.mu);
    TuneTable& tt = ts.table[c->device & 63];
    const std::string bkey = plan_key(pairs, hp, (int)sizeof(T) * 10 + (int)sizeof(S));
    if (ts.complete[c->device & 63].count(bkey)) return;
    const Plan<T, S> P0 = make_plan<T, S>(pairs, hp, &tt);
    std::vector<int> todo;
    for (int sidx = 0; sidx < P0.Lmax; sidx++)
        if (!P0.step_tuned[sidx] && (P0.steps[sidx].n_sor || P0.steps[sidx].n_units)) todo.push_back(sidx);
    if (todo.empty()) {
        ts.complete[c->device & 63].insert(bkey);
        return;
    }
    wait_idle(c);
    ensure_attrs<T, S>(c, sizeof(T) == 8 ? 1 : (std::is_same<S, __half>::value ? 2 : (std::is_same<S, float>::value ? 0 : 3)));
    const SolveConst<T> k = solve_const<T>(hp);
    cudaEvent_t ea, eb;
    RF_CUDA(cudaEventCreate(&ea));
    RF_CUDA(cudaEventCreate(&eb));
    for (int sidx : todo) {
        SorChoice best;
        double best_us = 1e30;
        for (SorChoice cand : sor_candidates(P0, sidx)) {
            TuneTable one = tt;
            one.m[P0.step_keys[sidx]] = cand;
            Plan<T, S> Pc = make_plan<T, S>(pairs, hp, &one);
            Pc.sms = c->sms;
            ensure_arena(c, Pc.arena_bytes);
            bind_plan(Pc, c->arena);
            RF_CUDA(cudaMemcpy(c->arena + Pc.desc_off, Pc.desc.data(), Pc.desc_bytes, cudaMemcpyHostToDevice));
            const auto& d = Pc.steps[sidx];
            char* db = c->arena + Pc.desc_off;
            const LevelItem<T, S>* items = (const LevelItem<T, S>*)(db + d.items_off);
            int* ticket = (int*)(c->arena + Pc.ctr_off) + sidx;
            // three activity patterns, each timed: every pair active; (with two or more pairs) every
            // other pair's SOR stopped, so that it only carries its increment through, as a converged
            // pair does; and every other pair done with the level (its work units are skipped, as
            // after an early outer termination).  The mean of the patterns is the candidate's time.
            const int reps = 3, pats = Pc.n > 1 ? 3 : 1;
            double ms_sum = 0;
            for (int pat = 0; pat < pats; pat++) {
                RF_CUDA(cudaMemsetAsync(c->arena + Pc.ctl_off, 0, Pc.ctr_off + sizeof(int) * 16 - Pc.ctl_off, c->stream));
                if (pat > 0)
                    for (int p = 1; p < Pc.n; p += 2)
                        RF_CUDA(cudaMemsetAsync(c->arena + Pc.ctl_off + sizeof(PairCtl) * p +
                                                    (pat == 1 ? offsetof(PairCtl, sor_stop) : offsetof(PairCtl, level_done)),
                                                1, 1, c->stream));
                for (int r = 0; r <= reps; r++) {
                    if (r == 1) RF_CUDA(cudaEventRecord(ea, c->stream));
                    SorLaunch L{};
                    L.it0 = 0; L.nit = Pc.sor_cfg[sidx].K; L.xin = r & 1; L.final_keep = 1; L.seq = r;
                    if (d.n_sor)
                        launch_sor<T, S>(Pc.sor_cfg[sidx], items, (const Tile*)(db + d.sor_tiles_off), d.n_sor, Pc.sms, k, L,
                                         c->stream);
                    if (d.n_units)
                        launch_sor_strip<T, S>(items, (const StripUnit*)(db + d.strip_units_off), d.n_units, d.strip_grid,
                                               ticket, k, L, c->stream);
                }
                RF_CUDA(cudaEventRecord(eb, c->stream));
                RF_CUDA(cudaEventSynchronize(eb));
                float ms = 0;
                RF_CUDA(cudaEventElapsedTime(&ms, ea, eb));
                ms_sum += ms;
            }
            const double us = 1e3 * ms_sum / (pats * reps * Pc.sor_cfg[sidx].K);
            // the balancing model's layout (timed last) has to win by 1 %: on 16 x 640x480 it timed
            // even with 128-row bands but ran the level-0 SOR of a real solve 3 % slower
            if (us < best_us * (cand.bands.empty() ? 1.0 : 0.99)) { best_us = us; best = cand; best.K = Pc.sor_cfg[sidx].K; }
        }
        best.us_per_it = best_us;
        tt.m[P0.step_keys[sidx]] = best;
    }
    ts.complete[c->device & 63].insert(bkey);
    cudaEventDestroy(ea);
    cudaEventDestroy(eb);
    RF_CUDA(cudaGetLastError());
}

// The plan of a batch with the device's tuned SOR choices (tuning first where a step has none).
template <class T, class S>
Plan<T, S> plan_for(rgbdflow_ctx* c, const std::vector<PairSpec>& pairs, const HostParams& hp)
{
    tune_sor<T, S>(c, pairs, hp);
    TuneState& ts = tune_state();
    std::lock_guard<std::mutex> lk(ts.mu);
    return make_plan<T, S>(pairs, hp, autotune_enabled() ? &ts.table[c->device & 63] : nullptr);
}

// Runs a batch through one graph launch.
//   user_stream == nullptr: host buffers, synchronous (pinned staging, H2D, solve, D2H).
//   user_stream != nullptr: every PairSpec pointer is device memory; the solve is enqueued on
//                           user_stream and the call returns without waiting.
template <class T, class S>
void run_batch(rgbdflow_ctx* c, const std::vector<PairSpec>& pairs, const HostParams& hp, rgbdflow_stats* stats, int slot,
               cudaStream_t user_stream = nullptr, bool host_async = false)
{
    ensure_attrs<T, S>(c, slot);
    const bool dev = user_stream != nullptr;
    Plan<T, S> P = plan_for<T, S>(c, pairs, hp);
    P.sms = c->sms;
    P.status = c->dev_status;
    ensure_arena(c, P.arena_bytes);
    bind_plan(P, c->arena);
    record_layout(c, P);
    if (dev) {
        // point the work lists at the caller's device buffers
        unsigned char* d = P.desc.data();
        PrepItem<T>* prep = (PrepItem<T>*)(d + P.prep_items_off);
        T** outs = (T**)(d + P.out_ptrs_off);
        EstSrc* est = (EstSrc*)(d + P.est_src_off);
        for (int p = 0; p < P.n; p++) {
            prep[p].bgr[0] = pairs[p].bgr1; prep[p].bgr[1] = pairs[p].bgr2;
            prep[p].depth[0] = pairs[p].depth1; prep[p].depth[1] = pairs[p].depth2;
            outs[p] = (T*)pairs[p].out;
            est[p].f = pairs[p].est;
        }
    }
    const size_t ctl_bytes = sizeof(PairCtl) * P.n;
    const size_t in_b = dev ? 0 : align_up(P.in_bytes, 256);
    const size_t out_b = dev ? 0 : align_up(P.out_bytes, 256);
    const size_t pin_need = in_b + align_up(P.desc_bytes, 256) + out_b + ctl_bytes;
    ensure_pin(c, pin_need);
    // the pinned staging may still feed the previous call's uploads
    RF_CUDA(cudaEventSynchronize(c->desc_up));
    char* pin_in = c->pin;
    char* pin_desc = pin_in + in_b;
    char* pin_out = pin_desc + align_up(P.desc_bytes, 256);
    char* pin_ctl = pin_out + out_b;
    // host inputs: page-locked caller buffers are copied by DMA directly, others through staging
    std::vector<std::pair<const void*, std::pair<size_t, size_t>>> direct;  // (src, (arena off, bytes))
    if (!dev)
        for (int p = 0; p < P.n; p++) {
            const auto segs = pairs[p].inputs();
            for (size_t q = 0; q < segs.size(); q++) {
                if (!segs[q].first) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "pair " + std::to_string(p) + ": null input buffer");
                if (is_pinned(segs[q].first)) direct.push_back({segs[q].first, {P.in_seg[p][q], segs[q].second}});
                else std::memcpy(pin_in + (P.in_seg[p][q] - P.in_off), segs[q].first, segs[q].second);
            }
        }
    std::memcpy(pin_desc, P.desc.data(), P.desc_bytes);
    cudaStream_t st = dev ? user_stream : c->stream;
    if (c->pending) RF_CUDA(cudaStreamWaitEvent(st, c->done, 0));  // arena reuse across streams
    if (!dev) {
        if (direct.empty()) {
            RF_CUDA(cudaMemcpyAsync(c->arena + P.in_off, pin_in, P.in_bytes, cudaMemcpyHostToDevice, st));
        } else {
            for (int p = 0; p < P.n; p++) {
                const auto segs = pairs[p].inputs();
                for (size_t q = 0; q < segs.size(); q++)
                    if (!is_pinned(segs[q].first))
                        RF_CUDA(cudaMemcpyAsync(c->arena + P.in_seg[p][q], pin_in + (P.in_seg[p][q] - P.in_off),
                                                segs[q].second, cudaMemcpyHostToDevice, st));
            }
            for (const auto& d : direct)
                RF_CUDA(cudaMemcpyAsync(c->arena + d.second.first, d.first, d.second.second, cudaMemcpyHostToDevice, st));
        }
    }
    RF_CUDA(cudaMemcpyAsync(c->arena + P.desc_off, pin_desc, P.desc_bytes, cudaMemcpyHostToDevice, st));
    RF_CUDA(cudaEventRecord(c->desc_up, st));
    RF_CUDA(cudaEventRecord(c->e0, st));
    const bool graphs = c->use_graphs && !c->prof;
    if (graphs) {
        GraphEntry& g = graph_for(c, P, pairs, hp, slot, dev);
        g.last_use = ++c->graph_clock;
        RF_CUDA(cudaGraphLaunch(g.exec, st));
        c->last_launches = g.launches;
    } else {
        c->last_launches = enqueue_solve(P, c->arena, st, c->prof.get());
    }
    RF_CUDA(cudaEventRecord(c->e1, st));
    // outputs: FP32 flows into page-locked caller buffers by DMA directly, the rest through staging
    std::vector<char> out_direct(P.n, 0);
    if (!dev) {
        bool all_direct = true;
        for (int p = 0; p < P.n; p++) {
            out_direct[p] = (sizeof(T) == 4 && pairs[p].out && !pairs[p].out_u && is_pinned(pairs[p].out)) ? 1 : 0;
            all_direct = all_direct && out_direct[p];
        }
        for (int p = 0; p < P.n; p++)
            if (out_direct[p])
                RF_CUDA(cudaMemcpyAsync(pairs[p].out, c->arena + P.out_pair_off[p], (size_t)pairs[p].W * pairs[p].H * 12,
                                        cudaMemcpyDeviceToHost, st));
        if (!all_direct) RF_CUDA(cudaMemcpyAsync(pin_out, c->arena + P.out_off, P.out_bytes, cudaMemcpyDeviceToHost, st));
    }
    const bool want_ctl = stats || c->prof;
    if (want_ctl) RF_CUDA(cudaMemcpyAsync(pin_ctl, c->arena + P.ctl_off, ctl_bytes, cudaMemcpyDeviceToHost, st));
    // the status word is sticky, so a later copy also carries an earlier solve's failure
    if (!dev || want_ctl) RF_CUDA(cudaMemcpyAsync(c->pin_status, c->dev_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    RF_CUDA(cudaEventRecord(c->done, st));
    c->pending = true;
    if (host_async) {
        for (int p = 0; p < P.n; p++)
            if (!out_direct[p]) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "submitted pair " + std::to_string(p) +
                                                                        ": flow_out must be page-locked host memory");
        return;
    }
    if (dev && !want_ctl) return;
    RF_CUDA(cudaEventSynchronize(c->done));
    c->pending = false;
    check_status(c);
    float ms = 0;
    RF_CUDA(cudaEventElapsedTime(&ms, c->e0, c->e1));
    if (c->prof) {
        c->prof->collect(c->prof_ms, c->prof_n);
        double sb, lb, sl[16];
        executed_bytes(P, (const PairCtl*)pin_ctl, &sb, &lb, sl);
        c->prof_bytes[KC_SOR] += sb;
        c->prof_bytes[KC_LIN] += lb;
        for (int k = 0; k < 16; k++) c->prof_bytes[KC_SOR_LEVEL0 + k] += sl[k];
    }
    if (!dev)
        for (int p = 0; p < P.n; p++) {
            const size_t N = (size_t)pairs[p].W * pairs[p].H;
            const T* o = (const T*)(pin_out + (P.out_pair_off[p] - P.out_off));
            const PairSpec& q = pairs[p];
            if (q.out && !out_direct[p])
                for (size_t z = 0; z < N * 3; z++) q.out[z] = (float)o[z];
            if (q.out_u)
                for (size_t z = 0; z < N; z++) { q.out_u[z] = (double)o[z * 3]; q.out_v[z] = (double)o[z * 3 + 1]; q.out_w[z] = (double)o[z * 3 + 2]; }
            if (q.out_warpI)
                for (size_t z = 0; z < N * 5; z++) q.out_warpI[z] = (double)o[N * 3 + z];
            if (q.out_warpD)
                for (size_t z = 0; z < N; z++) q.out_warpD[z] = (double)o[N * 8 + z];
        }
    if (stats)
        for (int p = 0; p < P.n; p++) fill_stats(((PairCtl*)pin_ctl)[p], P.L[p], P.shapes[p], ms, &stats[p]);
}

}  // namespace


static void dispatch(rgbdflow_ctx* c, const std::vector<PairSpec>& ps, const rgbdflow_params& p, rgbdflow_stats* stats,
                     cudaStream_t user_stream = nullptr, bool host_async = false)
{
    const HostParams hp = host_params(p);
    if (host_async) {
        if (p.compute == RGBDFLOW_COMPUTE_FP64)
            throw ArgError(RGBDFLOW_ERR_UNSUPPORTED, "the FP64 device solve has no submitted form");
        if (p.storage == RGBDFLOW_STORE_FP16) run_batch<float, __half>(c, ps, hp, nullptr, 2, nullptr, true);
        else if (p.storage == RGBDFLOW_STORE_BF16) run_batch<float, __nv_bfloat16>(c, ps, hp, nullptr, 3, nullptr, true);
        else run_batch<float, float>(c, ps, hp, nullptr, 0, nullptr, true);
        return;
    }
    if (p.compute == RGBDFLOW_COMPUTE_FP64) {
        if (user_stream) throw ArgError(RGBDFLOW_ERR_UNSUPPORTED, "the FP64 device solve has no device-pointer form");
        run_batch<double, double>(c, ps, hp, stats, 1);
    } else if (p.storage == RGBDFLOW_STORE_FP16) run_batch<float, __half>(c, ps, hp, stats, 2, user_stream);
    else if (p.storage == RGBDFLOW_STORE_BF16) run_batch<float, __nv_bfloat16>(c, ps, hp, stats, 3, user_stream);
    else run_batch<float, float>(c, ps, hp, stats, 0, user_stream);
}

// Captures the graph of a batch of device-pointer pairs (the served form) ahead of its first
// launch; nothing runs.  Returns false, capturing nothing, when the batch would need more solve
// memory than the context holds: its first launch reallocates, which drops the cached graphs.
template <class T, class S>
static bool prepare_batch(rgbdflow_ctx* c, const std::vector<PairSpec>& pairs, const HostParams& hp, int slot)
{
    if (!c->use_graphs || c->prof) return false;
    ensure_attrs<T, S>(c, slot);
    Plan<T, S> P = plan_for<T, S>(c, pairs, hp);
    if (c->graphs.count(graph_key(pairs, hp, slot, true, P.tune_desc))) return true;
    P.sms = c->sms;
    if (!c->arena || P.arena_bytes > c->arena_cap) return false;
    bind_plan(P, c->arena);
    graph_for(c, P, pairs, hp, slot, true);
    return true;
}

// prepare_batch with dispatch's choice of types (the FP32 solve: serving has no FP64 form).
static bool prepare_dispatch(rgbdflow_ctx* c, const std::vector<PairSpec>& ps, const rgbdflow_params& p)
{
    const HostParams hp = host_params(p);
    if (p.storage == RGBDFLOW_STORE_FP16) return prepare_batch<float, __half>(c, ps, hp, 2);
    if (p.storage == RGBDFLOW_STORE_BF16) return prepare_batch<float, __nv_bfloat16>(c, ps, hp, 3);
    return prepare_batch<float, float>(c, ps, hp, 0);
}

// Taps of Image::GaussianSmoothing (Image.h:1179-1199): exp(-i^2 / 2 sigma^2), normalised.
static std::vector<double> gauss_taps(double sigma, int fsize)
{
    std::vector<double> g(2 * fsize + 1);
    double sum = 0;
    const double s2 = sigma * sigma * 2;
    for (int i = -fsize; i <= fsize; i++) {
        g[i + fsize] = std::exp(-(double)(i * i) / s2);
        sum += g[i + fsize];
    }
    for (auto& x : g) x /= sum;
    return g;
}

// The 2-D optical flow of one pair (Coarse2FineFlow, src/opticalFlowMultiscale.cpp:4-146, CELIU
// variant, no depth maps) on the context's stream; synchronous.
static void run_flow2d(rgbdflow_ctx* c, const uint8_t* bgr1, const uint8_t* bgr2, int W, int H,
                       const rgbdflow_flow2d_params& prm, float* flow_out)
{
    using namespace rgbdflow::f2d;
    if (!bgr1 || !bgr2 || !flow_out || W < 2 || H < 2) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "bad frame");
    if (!(prm.alpha >= 0)) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "alpha must be >= 0");
    if (prm.n_outer < 0 || prm.n_inner < 1 || prm.n_sor < 1 || prm.sor_ring < 2 || prm.sor_ring > kMaxRing)
        throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "n_inner and n_sor must be >= 1, sor_ring in 2..16");
    // the level count loop below ends only for min_width >= 1 (the reference's never ends for <= 0),
    // and the flow is scaled by 1 / pyramid_ratio between levels
    if (prm.min_width < 1) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "min_width must be >= 1");
    if (!(prm.pyramid_ratio > 0) || !std::isfinite(prm.pyramid_ratio))
        throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "pyramid_ratio must be a finite number > 0");
    // pyramid geometry (GaussianPyramid::ConstructPyramid, GaussianPyramid.cpp:20-63)
    double ratio = prm.pyramid_ratio;
    if (ratio > 0.98 || ratio < 0.4) ratio = 0.75;
    int L = 1;
    for (double w = W * ratio; w >= prm.min_width; w *= ratio) L++;
    const double baseSigma = (1 / ratio - 1);
    const int nsm = (int)(std::log(0.25) / std::log(ratio));
    const double nSigma = baseSigma * nsm;
    struct Lev {
        int w, h, src, fs;
        double sigma, rate;
        size_t taps_off;
    };
    std::vector<Lev> lev(L);
    std::vector<double> taps = {1, -8, 0, 8, -1};
    for (auto& t : taps) t /= 12;
    lev[0] = {W, H, -1, 0, 0, 1, 0};
    for (int i = 1; i < L; i++) {
        Lev& l = lev[i];
        if (i <= nsm) {
            l.sigma = baseSigma * i;
            l.src = 0;
            l.rate = std::pow(ratio, i);
            l.w = (int)((double)W * l.rate);
            l.h = (int)((double)H * l.rate);
        } else {
            l.sigma = nSigma;
            l.src = i - nsm;
            l.rate = (double)std::pow(ratio, i) * W / lev[l.src].w;
            l.w = (int)((double)lev[l.src].w * l.rate);
            l.h = (int)((double)lev[l.src].h * l.rate);
        }
        l.fs = (int)(l.sigma * 3);
        if (2 * l.fs + 1 > rgbdflow::f2d::kMaxTaps) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "pyramid filter too wide");
        l.taps_off = taps.size();
        const std::vector<double> g = gauss_taps(l.sigma, l.fs);
        taps.insert(taps.end(), g.begin(), g.end());
        if (l.w < 1 || l.h < 1) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "pyramid level below one pixel");
    }
    // one stream-ordered allocation, carved
    const size_t N0 = (size_t)W * H;
    size_t total = 0;
    auto reserve = [&](size_t bytes) { const size_t o = total; total += align_up(bytes, 256); return o; };
    const size_t o_bgr = reserve(N0 * 6);
    const size_t o_taps = reserve(taps.size() * sizeof(double));
    const size_t o_ctl = reserve(2 * sizeof(int));
    std::vector<size_t> o_img[2], o_feat[2], o_u(L), o_v(L);
    for (int f = 0; f < 2; f++)
        for (int i = 0; i < L; i++) {
            o_img[f].push_back(reserve((size_t)lev[i].w * lev[i].h * 3 * sizeof(double)));
            o_feat[f].push_back(reserve((size_t)lev[i].w * lev[i].h * 5 * sizeof(double)));
        }
    for (int i = 0; i < L; i++) {
        o_u[i] = reserve((size_t)lev[i].w * lev[i].h * sizeof(double));
        o_v[i] = reserve((size_t)lev[i].w * lev[i].h * sizeof(double));
    }
    const size_t o_tmpA = reserve(N0 * 3 * sizeof(double)), o_tmpB = reserve(N0 * 3 * sizeof(double));
    const size_t o_warp = reserve(N0 * 5 * sizeof(double));
    size_t o_plane[8];
    for (auto& o : o_plane) o = reserve(N0 * sizeof(double));
    // levels of at least this many pixels run their SOR over a cluster of CTAs with more sweeps in
    // flight (the flow does not depend on it)
    const char* ce = std::getenv("RGBDFLOW_FLOW2D_CLUSTER_MIN_PX");
    const long clus_min_px = ce ? std::atol(ce) : 4096L;
    constexpr int kClusterRing = 64;
    // the cluster: 16 CTAs where the device can co-schedule them (a non-portable size), else 8
    static int clus_ctas = 0;
    if (!clus_ctas) {
        const char* cc = std::getenv("RGBDFLOW_FLOW2D_CLUSTER_CTAS");
        int want = cc ? std::atoi(cc) : 16;
        want = want >= 16 ? 16 : 8;
        if (want == 16) {
            RF_CUDA(cudaFuncSetAttribute(k_sor_wavefront_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            cudaLaunchConfig_t q = {};
            q.gridDim = dim3(16);
            q.blockDim = dim3(kSorThreads);
            cudaLaunchAttribute qa[1];
            qa[0].id = cudaLaunchAttributeClusterDimension;
            qa[0].val.clusterDim.x = 16;
            qa[0].val.clusterDim.y = 1;
            qa[0].val.clusterDim.z = 1;
            q.attrs = qa;
            q.numAttrs = 1;
            int nc = 0;
            if (cudaOccupancyMaxActiveClusters(&nc, k_sor_wavefront_cluster, &q) != cudaSuccess || nc < 1) {
                cudaGetLastError();
                want = 8;
            }
        }
        clus_ctas = want;
    }
    const int kClusterCtas = clus_ctas;
    const int ring_slots = std::max(prm.sor_ring, (long)N0 >= clus_min_px ? kClusterRing : 0);
    const size_t o_ring = reserve((size_t)ring_slots * N0 * sizeof(double2));  // (du, dv) pairs per sweep slot
    const size_t o_coef = reserve(N0 * 8 * sizeof(double));
    if (c->budget && total > c->budget) throw ArgError(RGBDFLOW_ERR_BUDGET, "2-D flow needs " + std::to_string(total) + " device bytes");
    RF_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    if (c->pending) RF_CUDA(cudaStreamWaitEvent(st, c->done, 0));
    char* base = nullptr;
    RF_CUDA(cudaMallocAsync((void**)&base, total, st));
    struct Free {
        char* p;
        cudaStream_t s;
        ~Free() { if (p) { cudaFreeAsync(p, s); cudaStreamSynchronize(s); } }
    } release{base, st};
    auto D = [&](size_t o) { return (double*)(base + o); };
    int* ctl = (int*)(base + o_ctl);
    uint8_t* dbgr = (uint8_t*)(base + o_bgr);
    RF_CUDA(cudaMemcpyAsync(dbgr, bgr1, N0 * 3, cudaMemcpyHostToDevice, st));
    RF_CUDA(cudaMemcpyAsync(dbgr + N0 * 3, bgr2, N0 * 3, cudaMemcpyHostToDevice, st));
    RF_CUDA(cudaMemcpyAsync(D(o_taps), taps.data(), taps.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    RF_CUDA(cudaMemsetAsync(ctl, 0, 2 * sizeof(int), st));
    const double* d5 = D(o_taps);
    int launches = 0;
    auto grid = [&](size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + kThreads - 1) / kThreads, (size_t)c->sms * 8)); };
    for (int f = 0; f < 2; f++) {
        k_unpack<<<grid(N0 * 3), kThreads, 0, st>>>(dbgr + f * N0 * 3, D(o_img[f][0]), N0 * 3);
        launches++;
        for (int i = 1; i < L; i++) {
            const Lev& l = lev[i];
            const int sw = lev[l.src].w, sh = lev[l.src].h;
            const size_t sn = (size_t)sw * sh;
            k_hfilter<<<grid(sn), kThreads, 0, st>>>(D(o_img[f][l.src]), D(o_tmpA), sw, sh, 3, D(o_taps) + l.taps_off, l.fs);
            k_vfilter<<<grid(sn), kThreads, 0, st>>>(D(o_tmpA), D(o_tmpB), sw, sh, 3, D(o_taps) + l.taps_off, l.fs);
            k_resize<<<grid((size_t)l.w * l.h), kThreads, 0, st>>>(D(o_tmpB), sw, sh, 3, D(o_img[f][i]), l.w, l.h, l.rate, l.rate);
            launches += 3;
        }
        for (int i = 0; i < L; i++) {
            k_features<<<grid((size_t)lev[i].w * lev[i].h), kThreads, 0, st>>>(D(o_img[f][i]), D(o_feat[f][i]), lev[i].w, lev[i].h, d5);
            launches++;
        }
    }
    const double eps = std::pow(0.001, 2);
    for (int k = L - 1; k >= 0; k--) {
        const int w = lev[k].w, h = lev[k].h;
        const size_t n = (size_t)w * h;
        LevelBufs b;
        b.f1 = D(o_feat[0][k]);
        b.f2 = D(o_feat[1][k]);
        b.warp = D(o_warp);
        b.u = D(o_u[k]);
        b.v = D(o_v[k]);
        b.du = D(o_plane[0]);
        b.dv = D(o_plane[1]);
        b.phi = D(o_plane[2]);
        b.dxy = D(o_plane[3]);
        b.dx2 = D(o_plane[4]);
        b.dy2 = D(o_plane[5]);
        b.dtdx = D(o_plane[6]);
        b.dtdy = D(o_plane[7]);
        b.coef = D(o_coef);
        b.W = w;
        b.H = h;
        if (k == L - 1) {
            RF_CUDA(cudaMemsetAsync(b.u, 0, n * sizeof(double), st));
            RF_CUDA(cudaMemsetAsync(b.v, 0, n * sizeof(double), st));
            RF_CUDA(cudaMemcpyAsync(b.warp, b.f2, n * 5 * sizeof(double), cudaMemcpyDeviceToDevice, st));
        } else {
            // the coarser flow resized (Image::imresize(w, h)) and scaled by 1 / ratio, then the warp
            const int pw = lev[k + 1].w, ph = lev[k + 1].h;
            const double xr = (double)w / pw, yr = (double)h / ph;
            k_resize<<<grid(n), kThreads, 0, st>>>(D(o_u[k + 1]), pw, ph, 1, b.u, w, h, xr, yr);
            k_resize<<<grid(n), kThreads, 0, st>>>(D(o_v[k + 1]), pw, ph, 1, b.v, w, h, xr, yr);
            const double s = 1 / prm.pyramid_ratio;
            k_scale<<<grid(n), kThreads, 0, st>>>(b.u, n, s);
            k_scale<<<grid(n), kThreads, 0, st>>>(b.v, n, s);
            k_warp<<<grid(n), kThreads, 0, st>>>(b.f1, b.f2, b.u, b.v, b.warp, w, h);
            launches += 5;
        }
        const int nOuter = prm.n_outer + k, nSOR = prm.n_sor + k * 3;
        for (int count = 0; count < nOuter; count++) {
            for (int hh = 0; hh < prm.n_inner; hh++) {
                k_phi_psi<<<grid(n), kThreads, 0, st>>>(b, d5, hh == 0 ? 1 : 0, eps);
                k_rhs<<<grid(n), kThreads, 0, st>>>(b, prm.alpha);
                if ((long)n >= clus_min_px) {
                    cudaLaunchConfig_t cfg = {};
                    cfg.gridDim = dim3(kClusterCtas);
                    cfg.blockDim = dim3(kSorThreads);
                    cfg.stream = st;
                    cudaLaunchAttribute at[1];
                    at[0].id = cudaLaunchAttributeClusterDimension;
                    at[0].val.clusterDim.x = kClusterCtas;
                    at[0].val.clusterDim.y = 1;
                    at[0].val.clusterDim.z = 1;
                    cfg.attrs = at;
                    cfg.numAttrs = 1;
                    RF_CUDA(cudaLaunchKernelEx(&cfg, k_sor_wavefront_cluster, b, prm.alpha, nSOR, kClusterRing,
                                               (double2*)(base + o_ring), ctl + 1, ctl));
                } else {
                    k_sor_wavefront<<<1, kSorThreads, 0, st>>>(b, prm.alpha, nSOR, prm.sor_ring, (double2*)(base + o_ring),
                                                               ctl + 1, ctl);
                }
                launches += 3;
            }
            k_update<<<grid(n), kThreads, 0, st>>>(b);
            k_warp<<<grid(n), kThreads, 0, st>>>(b.f1, b.f2, b.u, b.v, b.warp, w, h);
            launches += 2;
        }
    }
    RF_CUDA(cudaGetLastError());
    std::vector<double> u(N0), v(N0);
    int hctl[2] = {0, 0};
    RF_CUDA(cudaMemcpyAsync(u.data(), D(o_u[0]), N0 * sizeof(double), cudaMemcpyDeviceToHost, st));
    RF_CUDA(cudaMemcpyAsync(v.data(), D(o_v[0]), N0 * sizeof(double), cudaMemcpyDeviceToHost, st));
    RF_CUDA(cudaMemcpyAsync(hctl, ctl, sizeof(hctl), cudaMemcpyDeviceToHost, st));
    RF_CUDA(cudaStreamSynchronize(st));
    c->last_launches = launches;
    if (hctl[0]) throw ArgError(RGBDFLOW_ERR_INTERNAL, "2-D SOR ran out of its step bound");
    for (size_t z = 0; z < N0; z++) {
        flow_out[z * 2] = (float)u[z];
        flow_out[z * 2 + 1] = (float)v[z];
    }
}

static int fail(rgbdflow_ctx* c, int code, const std::string& m)
{
    if (c) c->err = m;
    return code;
}

#define API_BEGIN try {
#define API_END(ctx)                                                                        \
    }                                                                                        \
    catch (const ArgError& e) { return fail(ctx, e.code, e.what()); }                        \
    catch (const CudaError& e) { return fail(ctx, RGBDFLOW_ERR_CUDA, e.what()); }            \
    catch (const std::bad_alloc&) { return fail(ctx, RGBDFLOW_ERR_INTERNAL, "host out of memory"); } \
    catch (const std::exception& e) { return fail(ctx, RGBDFLOW_ERR_INTERNAL, e.what()); }   \
    catch (...) { return fail(ctx, RGBDFLOW_ERR_INTERNAL, "unknown error"); }

extern "C" {

void rgbdflow_params_default(rgbdflow_params* p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->regularization = RGBDFLOW_REG_HPB;
    p->color_data_weight = 1;
    p->depth_vs_color_data_weight = 1;
    p->alpha = 0.02;
    p->gamma = 1e-5;
    p->pyramid_ratio = 0.75;
    p->min_width = 60;
    p->n_outer = 50;
    p->n_inner = 1;
    p->n_sor = 10000;
    p->depth_boundary_dist = 4;
    p->fill_holes = 1;
    p->fixed_schedule = 0;
    p->storage = RGBDFLOW_STORE_FP32;
    p->compute = RGBDFLOW_COMPUTE_FP32;
    p->omega = 0.7;
    p->max_flow_step = 0.3;
    p->eps_d = 1e-6;
    p->eps_z = 1e-10;
    p->eps_s = 1e-6;
    p->sor_tol = 1e-5;
    p->sor_check_period = 25;
    p->outer_tol = 4e-4;
    p->occ_margin = 0.02;
    p->occ_penalty = 0.01;
    p->max_depth_grad = 0.04;
    p->sweeps_per_launch = 0;
}

int rgbdflow_abi_version(void) { return RGBDFLOW_ABI_VERSION; }

int rgbdflow_pyramid_levels(int W, int H, double ratio, int min_width, int* w, int* h)
{
    if (W < 1 || H < 1 || min_width == 0) return RGBDFLOW_ERR_INVALID_ARG;
    try {
        const PyrShape s = pyramid_shape(W, H, ratio, min_width, 0);
        const int L = (int)s.w.size();
        if (L > RGBDFLOW_MAX_LEVELS) return RGBDFLOW_ERR_UNSUPPORTED;
        for (int i = 0; i < L; i++) {
            if (w) w[i] = s.w[i];
            if (h) h[i] = s.h[i];
        }
        return L;
    } catch (...) {
        return RGBDFLOW_ERR_INTERNAL;
    }
}

int rgbdflow_batch_device_bytes(const int* Ws, const int* Hs, const int* warm, int n, const rgbdflow_params* params,
                                size_t* bytes)
{
    if (!Ws || !Hs || n <= 0 || !params || !bytes) return RGBDFLOW_ERR_INVALID_ARG;
    try {
        validate(params);
        std::vector<PairSpec> ps(n);
        static const float dummy = 1;
        for (int i = 0; i < n; i++) {
            ps[i].kind = 0; ps[i].W = Ws[i]; ps[i].H = Hs[i]; ps[i].f_full = 1; ps[i].xres_full = (unsigned)Ws[i];
            if (warm && warm[i]) ps[i].est = &dummy;
        }
        const HostParams hp = host_params(*params);
        if (params->compute == RGBDFLOW_COMPUTE_FP64) *bytes = make_plan<double, double>(ps, hp).arena_bytes;
        else if (params->storage == RGBDFLOW_STORE_FP16) *bytes = make_plan<float, __half>(ps, hp).arena_bytes;
        else if (params->storage == RGBDFLOW_STORE_BF16) *bytes = make_plan<float, __nv_bfloat16>(ps, hp).arena_bytes;
        else *bytes = make_plan<float, float>(ps, hp).arena_bytes;
        return RGBDFLOW_OK;
    } catch (const ArgError& e) {
        return e.code;
    } catch (...) {
        return RGBDFLOW_ERR_INTERNAL;
    }
}

int rgbdflow_ctx_create(int device, size_t hbm_budget_bytes, rgbdflow_ctx** out)
{
    if (!out) return RGBDFLOW_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); return RGBDFLOW_ERR_NO_DEVICE; }
    if (device < 0 || device >= n) return RGBDFLOW_ERR_INVALID_ARG;
    std::unique_ptr<rgbdflow_ctx> c(new rgbdflow_ctx());
    c->device = device;
    c->budget = hbm_budget_bytes;
    if (cudaSetDevice(device) != cudaSuccess) return RGBDFLOW_ERR_CUDA;
    if (cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return RGBDFLOW_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return RGBDFLOW_ERR_CUDA;
    if (cudaEventCreate(&c->e0) != cudaSuccess || cudaEventCreate(&c->e1) != cudaSuccess) return RGBDFLOW_ERR_CUDA;
    if (cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->desc_up, cudaEventDisableTiming) != cudaSuccess)
        return RGBDFLOW_ERR_CUDA;
    if (cudaMalloc(&c->dev_status, 64) != cudaSuccess || cudaMemset(c->dev_status, 0, 64) != cudaSuccess ||
        cudaMallocHost(&c->pin_status, sizeof(int)) != cudaSuccess)
        return RGBDFLOW_ERR_CUDA;
    *c->pin_status = 0;
    const char* g = std::getenv("RGBDFLOW_NO_GRAPHS");
    c->use_graphs = !(g && g[0] == '1');
    *out = c.release();
    return RGBDFLOW_OK;
}

int rgbdflow_ctx_destroy(rgbdflow_ctx* c)
{
    if (!c) return RGBDFLOW_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    if (c->pending) cudaEventSynchronize(c->done);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graphs(c);
    c->prof.reset();
    if (c->done) cudaEventDestroy(c->done);
    if (c->desc_up) cudaEventDestroy(c->desc_up);
    if (c->arena) cudaFree(c->arena);
    if (c->pin) cudaFreeHost(c->pin);
    if (c->dev_status) cudaFree(c->dev_status);
    if (c->pin_status) cudaFreeHost(c->pin_status);
    if (c->e0) cudaEventDestroy(c->e0);
    if (c->e1) cudaEventDestroy(c->e1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return RGBDFLOW_OK;
}

const char* rgbdflow_last_error(const rgbdflow_ctx* c) { return c ? c->err.c_str() : "no context"; }

size_t rgbdflow_ctx_device_bytes(const rgbdflow_ctx* c) { return c ? c->arena_cap : 0; }

int rgbdflow_scene_flow_batch(rgbdflow_ctx* c, const rgbdflow_pair* pairs, int n, const rgbdflow_params* params,
                              rgbdflow_stats* stats)
{
    if (!c) return RGBDFLOW_ERR_INVALID_ARG;
    API_BEGIN
    validate(params);
    if (!pairs || n <= 0) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "no pairs");
    RF_CUDA(cudaSetDevice(c->device));
    std::vector<PairSpec> ps;
    for (int i = 0; i < n; i++) {
        const rgbdflow_pair& q = pairs[i];
        if (q.W < 2 || q.H < 2 || !q.bgr1 || !q.bgr2 || !q.depth1_m || !q.depth2_m || !q.flow_out)
            throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "pair " + std::to_string(i) + ": bad size or null buffer");
        if (q.cam.xRes == 0 || !(q.cam.focalLength > 0))
            throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "pair " + std::to_string(i) + ": bad camera");
        PairSpec s;
        s.W = q.W; s.H = q.H;
        resized_cam(q.cam, q.W, s.f_full, s.xres_full);
        s.bgr1 = q.bgr1; s.depth1 = q.depth1_m; s.bgr2 = q.bgr2; s.depth2 = q.depth2_m;
        s.est = q.est_flow; s.out = q.flow_out;
        ps.push_back(s);
    }
    dispatch(c, ps, *params, stats);
    return RGBDFLOW_OK;
    API_END(c)
}

int rgbdflow_scene_flow_two_frames(rgbdflow_ctx* c, const rgbdflow_camera_params* cam, const uint8_t* bgr1,
                                   const float* depth1_m, const uint8_t* bgr2, const float* depth2_m, int W, int H,
                                   const rgbdflow_params* params, const float* est_flow, float* flow_out,
                                   rgbdflow_stats* stats)
{
    if (!c) return RGBDFLOW_ERR_INVALID_ARG;
    if (!cam) return fail(c, RGBDFLOW_ERR_INVALID_ARG, "cam is NULL");
    rgbdflow_pair p;
    p.W = W; p.H = H; p.cam = *cam;
    p.bgr1 = bgr1; p.depth1_m = depth1_m; p.bgr2 = bgr2; p.depth2_m = depth2_m;
    p.est_flow = est_flow; p.flow_out = flow_out;
    return rgbdflow_scene_flow_batch(c, &p, 1, params, stats);
}

int rgbdflow_scene_flow_multiscale(rgbdflow_ctx* c, const rgbdflow_camera_params* cam, const double* Im1,
                                   const double* dm1, const double* Im2, const double* dm2, const float* depth_sigma1,
                                   int W, int H, const rgbdflow_params* params, double* u, double* v, double* w,
                                   rgbdflow_stats* stats)
{
    if (!c) return RGBDFLOW_ERR_INVALID_ARG;
    API_BEGIN
    validate(params);
    if (!cam || !Im1 || !dm1 || !Im2 || !dm2 || !depth_sigma1 || !u || !v || !w || W < 2 || H < 2)
        throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "null buffer or bad size");
    RF_CUDA(cudaSetDevice(c->device));
    PairSpec s;
    s.kind = 1; s.W = W; s.H = H;
    resized_cam(*cam, W, s.f_full, s.xres_full);
    s.im1 = Im1; s.im2 = Im2; s.dm1 = dm1; s.dm2 = dm2; s.sigma1 = depth_sigma1;
    s.out_u = u; s.out_v = v; s.out_w = w;
    dispatch(c, {s}, *params, stats);
    return RGBDFLOW_OK;
    API_END(c)
}

int rgbdflow_scene_flow_with_init(rgbdflow_ctx* c, const rgbdflow_camera_params* cam, const double* Im1,
                                  const double* dm1, const double* Im2, const double* dm2, const float* depth_sigma1,
                                  int W, int H, const rgbdflow_params* params, double* u, double* v, double* w,
                                  rgbdflow_stats* stats)
{
    if (!c) return RGBDFLOW_ERR_INVALID_ARG;
    API_BEGIN
    validate(params);
    if (!cam || !Im1 || !dm1 || !Im2 || !dm2 || !depth_sigma1 || !u || !v || !w || W < 2 || H < 2)
        throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "null buffer or bad size");
    RF_CUDA(cudaSetDevice(c->device));
    const size_t N = (size_t)W * H;
    std::vector<double> est(N * 3);
    std::memcpy(est.data(), u, N * 8);
    std::memcpy(est.data() + N, v, N * 8);
    std::memcpy(est.data() + 2 * N, w, N * 8);
    PairSpec s;
    s.kind = 1; s.W = W; s.H = H;
    resized_cam(*cam, W, s.f_full, s.xres_full);
    s.im1 = Im1; s.im2 = Im2; s.dm1 = dm1; s.dm2 = dm2; s.sigma1 = depth_sigma1;
    s.est_d = est.data();
    s.out_u = u; s.out_v = v; s.out_w = w;
    dispatch(c, {s}, *params, stats);
    return RGBDFLOW_OK;
    API_END(c)
}

int rgbdflow_scene_flow_single_scale(rgbdflow_ctx* c, const rgbdflow_camera_params* cam, const double* Im1,
                                     const double* dm1, const double* Im2, const double* dm2, double* warpIm2,
                                     double* warpDm2, double* u, double* v, double* w, int W, int H, int nCh,
                                     double colorDataTermWeight, const double* depthDataTermWeights, double alpha,
                                     const double* depthSmoothnessTermWeights, double gamma,
                                     const double* depthMagTermWeights, const double* regularizationWeights,
                                     int nOuterFPIterations, int nInnerFPIterations, int nSORIterations,
                                     int allowEarlyTermination, const rgbdflow_params* params, rgbdflow_stats* stats)
{
    if (!c) return RGBDFLOW_ERR_INVALID_ARG;
    API_BEGIN
    if (nCh != 5) throw ArgError(RGBDFLOW_ERR_UNSUPPORTED, "the device solve takes the 5-channel RGB_WITH_GRADIENT features");
    if (!cam || !Im1 || !dm1 || !Im2 || !dm2 || !u || !v || !w || !depthDataTermWeights || !depthSmoothnessTermWeights ||
        !depthMagTermWeights || !regularizationWeights || W < 2 || H < 2)
        throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "null buffer or bad size");
    rgbdflow_params p;
    if (params) p = *params; else rgbdflow_params_default(&p);
    p.regularization = RGBDFLOW_REG_ISOTROPIC;  // weights are given explicitly
    p.color_data_weight = colorDataTermWeight;
    p.alpha = alpha;
    p.gamma = gamma;
    p.n_outer = nOuterFPIterations;
    p.n_inner = nInnerFPIterations;
    p.n_sor = nSORIterations;
    validate(&p);
    RF_CUDA(cudaSetDevice(c->device));
    const size_t N = (size_t)W * H;
    std::vector<double> uvw(N * 3);
    std::memcpy(uvw.data(), u, N * 8);
    std::memcpy(uvw.data() + N, v, N * 8);
    std::memcpy(uvw.data() + 2 * N, w, N * 8);
    PairSpec s;
    s.kind = 2; s.W = W; s.H = H;
    s.f_full = cam->focalLength; s.xres_full = (unsigned)W;
    s.f_level = cam->focalLength;
    s.allow_early = allowEarlyTermination ? 1 : 0;
    s.feat1 = Im1; s.feat2 = Im2; s.dm1 = dm1; s.dm2 = dm2; s.uvw = uvw.data();
    s.ddw = depthDataTermWeights; s.dsw = depthSmoothnessTermWeights; s.mag = depthMagTermWeights;
    s.regw = regularizationWeights;
    s.out_u = u; s.out_v = v; s.out_w = w;
    s.out_warpI = warpIm2; s.out_warpD = warpDm2;
    dispatch(c, {s}, p, stats);
    return RGBDFLOW_OK;
    API_END(c)
}

int rgbdflow_scene_flow_batch_submit(rgbdflow_ctx* c, const rgbdflow_pair* pairs, int n, const rgbdflow_params* params)
{
    if (!c) return RGBDFLOW_ERR_INVALID_ARG;
    API_BEGIN
    validate(params);
    if (!pairs || n <= 0) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "no pairs");
    RF_CUDA(cudaSetDevice(c->device));
    std::vector<PairSpec> ps;
    for (int i = 0; i < n; i++) {
        const rgbdflow_pair& q = pairs[i];
        if (q.W < 2 || q.H < 2 || !q.bgr1 || !q.bgr2 || !q.depth1_m || !q.depth2_m || !q.flow_out)
            throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "pair " + std::to_string(i) + ": bad size or null buffer");
        if (q.cam.xRes == 0 || !(q.cam.focalLength > 0))
            throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "pair " + std::to_string(i) + ": bad camera");
        if (!is_pinned(q.flow_out))
            throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "pair " + std::to_string(i) + ": flow_out must be page-locked host memory");
        PairSpec s;
        s.W = q.W; s.H = q.H;
        resized_cam(q.cam, q.W, s.f_full, s.xres_full);
        s.bgr1 = q.bgr1; s.depth1 = q.depth1_m; s.bgr2 = q.bgr2; s.depth2 = q.depth2_m;
        s.est = q.est_flow; s.out = q.flow_out;
        ps.push_back(s);
    }
    dispatch(c, ps, *params, nullptr, nullptr, true);
    return RGBDFLOW_OK;
    API_END(c)
}

int rgbdflow_scene_flow_batch_async(rgbdflow_ctx* c, const rgbdflow_pair* pairs, int n, const rgbdflow_params* params,
                                    void* stream)
{
    if (!c) return RGBDFLOW_ERR_INVALID_ARG;
    API_BEGIN
    validate(params);
    if (!pairs || n <= 0) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "no pairs");
    RF_CUDA(cudaSetDevice(c->device));
    std::vector<PairSpec> ps;
    for (int i = 0; i < n; i++) {
        const rgbdflow_pair& q = pairs[i];
        if (q.W < 2 || q.H < 2 || !q.bgr1 || !q.bgr2 || !q.depth1_m || !q.depth2_m || !q.flow_out)
            throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "pair " + std::to_string(i) + ": bad size or null buffer");
        if (q.cam.xRes == 0 || !(q.cam.focalLength > 0))
            throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "pair " + std::to_string(i) + ": bad camera");
        PairSpec s;
        s.W = q.W; s.H = q.H;
        resized_cam(q.cam, q.W, s.f_full, s.xres_full);
        s.bgr1 = q.bgr1; s.depth1 = q.depth1_m; s.bgr2 = q.bgr2; s.depth2 = q.depth2_m;
        s.est = q.est_flow; s.out = q.flow_out;
        ps.push_back(s);
    }
    dispatch(c, ps, *params, nullptr, stream ? (cudaStream_t)stream : c->stream);
    return RGBDFLOW_OK;
    API_END(c)
}

int rgbdflow_ctx_synchronize(rgbdflow_ctx* c)
{
    if (!c) return RGBDFLOW_ERR_INVALID_ARG;
    API_BEGIN
    wait_idle(c);
    // device-pointer solves leave no copy of the status behind: read it here
    RF_CUDA(cudaMemcpy(c->pin_status, c->dev_status, sizeof(int), cudaMemcpyDeviceToHost));
    check_status(c);
    return RGBDFLOW_OK;
    API_END(c)
}

int rgbdflow_debug_wait_timeout(rgbdflow_ctx* c, double* seconds)
{
    if (!c) return RGBDFLOW_ERR_INVALID_ARG;
    API_BEGIN
    RF_CUDA(cudaSetDevice(c->device));
    wait_idle(c);
    GridSync* gs = (GridSync*)(c->dev_status + 4);
    RF_CUDA(cudaMemsetAsync(gs, 0, sizeof(GridSync), c->stream));
    RF_CUDA(cudaStreamSynchronize(c->stream));
    const auto t0 = std::chrono::steady_clock::now();
    k_wait_probe<<<1, 32, 0, c->stream>>>(gs, c->dev_status);
    RF_CUDA(cudaGetLastError());
    RF_CUDA(cudaMemcpyAsync(c->pin_status, c->dev_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    RF_CUDA(cudaStreamSynchronize(c->stream));
    if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    check_status(c);
    return RGBDFLOW_OK;
    API_END(c)
}

int rgbdflow_ctx_last_launch_count(const rgbdflow_ctx* c) { return c ? c->last_launches : 0; }

void rgbdflow_flow2d_params_default(rgbdflow_flow2d_params* p)
{
    if (!p) return;
    // runFlowTwoFramesCeLiu (src/runFlowTwoFrames.cpp:36-41) with the demo's smoothness weight
    // (main.cpp:57) and opticalFlowParams' pyramid (OpticalFlow.h:54)
    p->alpha = 0.02;
    p->pyramid_ratio = 0.75;
    p->min_width = 20;
    p->n_outer = 10;
    p->n_inner = 1;
    p->n_sor = 400;
    p->sor_ring = 8;
}

int rgbdflow_optical_flow_2d(rgbdflow_ctx* c, const uint8_t* bgr1, const uint8_t* bgr2, int W, int H,
                             const rgbdflow_flow2d_params* params, float* flow_out)
{
    if (!c || !params) return RGBDFLOW_ERR_INVALID_ARG;
    API_BEGIN
    run_flow2d(c, bgr1, bgr2, W, H, *params, flow_out);
    return RGBDFLOW_OK;
    API_END(c)
}

int rgbdflow_autotune_describe(int device, char* buf, size_t len)
{
    if (device < 0 || device >= 64) return RGBDFLOW_ERR_INVALID_ARG;
    std::string out;
    {
        TuneState& ts = tune_state();
        std::lock_guard<std::mutex> lk(ts.mu);
        for (const auto& kv : ts.table[device].m) {
            const SorChoice& ch = kv.second;
            char b[512];
            std::string lay;
            for (const auto& e : ch.bands) {
                lay += " H" + std::to_string(e.first) + ":";
                for (size_t q = 0; q < e.second.size(); q++) lay += (q ? "/" : "") + std::to_string(e.second[q]);
            }
            if (ch.strip && !ch.bands.empty())
                std::snprintf(b, sizeof b, "%s strip bands%s K %d %.2f us/it; ", kv.first.c_str(), lay.c_str(), ch.K, ch.us_per_it);
            else if (ch.strip) std::snprintf(b, sizeof b, "%s strip band %d K %d %.2f us/it; ", kv.first.c_str(), ch.seg, ch.K, ch.us_per_it);
            else std::snprintf(b, sizeof b, "%s tile K %d ilp %d %.2f us/it; ", kv.first.c_str(), ch.K, ch.ilp, ch.us_per_it);
            out += b;
        }
    }
    if (buf && len) {
        const size_t n = std::min(out.size(), len - 1);
        std::memcpy(buf, out.data(), n);
        buf[n] = 0;
    }
    return (int)out.size();
}

int rgbdflow_debug_read_plane(rgbdflow_ctx* c, int pair, int level, int kind, int index, double* dst, size_t n, int* W,
                              int* H)
{
    if (!c) return RGBDFLOW_ERR_INVALID_ARG;
    try {
        if (pair < 0 || pair >= (int)c->dbg.size()) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "no such pair in the last solve");
        const DbgPair& dp = c->dbg[pair];
        if (level < 0 || level >= (int)dp.lev.size()) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "no such level");
        if (kind == RGBDFLOW_PLANE_FILL_ROUND && level != 0) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "fill rounds exist at level 0 only");
        const DbgLevel& L = dp.lev[level];
        const int w = L.W, h = L.H;
        if (W) *W = w;
        if (H) *H = h;
        const size_t N = (size_t)w * h;
        if (!dst) return RGBDFLOW_OK;
        if (n < N) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "destination too small");
        static const int counts[10] = {10, 5, 5, 2, 1, 2, 3, 12, 2, 1};
        if (kind < 0 || kind > 9 || index < 0 || index >= counts[kind]) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "bad plane kind or index");
        if (kind == RGBDFLOW_PLANE_HPB_DEPTH && !L.hz) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "the last solve did not use HPB");
        const void* src = nullptr;
        int esize = c->dbg_tsize, etype = c->dbg_tsize == 8 ? 3 : 0;  // 0 FP32, 1 FP16, 2 BF16, 3 FP64, 4 u8
        int layout = 0;                                                // 0 raster, 1 pitched u, 2 checkerboard
        switch (kind) {
        case RGBDFLOW_PLANE_PYRAMID: src = L.pyr[index]; break;
        case RGBDFLOW_PLANE_FEATURES1: src = L.I1[index]; etype = c->dbg_store; break;
        case RGBDFLOW_PLANE_FEATURES2: src = L.I2[index]; etype = c->dbg_store; break;
        case RGBDFLOW_PLANE_DEPTH: src = L.D[index]; etype = c->dbg_store; break;
        case RGBDFLOW_PLANE_DEPTH_MAG: src = L.mag; break;
        case RGBDFLOW_PLANE_REG: src = L.reg[index]; break;
        case RGBDFLOW_PLANE_FLOW: src = L.u[index]; layout = 1; break;
        case RGBDFLOW_PLANE_SYSTEM: src = L.sys[index]; layout = 2; break;
        case RGBDFLOW_PLANE_HPB_DEPTH: src = L.hz; break;
        default: src = dp.stamp[index]; etype = 4; break;
        }
        if (etype == 1 || etype == 2) esize = 2;
        if (etype == 4) esize = 1;
        const size_t elems = layout == 0 ? N : (layout == 1 ? (size_t)L.pitch * h : (size_t)2 * L.hwp * h);
        wait_idle(c);
        std::vector<unsigned char> buf(elems * esize);
        RF_CUDA(cudaMemcpy(buf.data(), src, buf.size(), cudaMemcpyDeviceToHost));
        auto at = [&](size_t e) -> double {
            const unsigned char* b = buf.data() + e * esize;
            switch (etype) {
            case 0: { float f; std::memcpy(&f, b, 4); return f; }
            case 1: { __half x; std::memcpy(&x, b, 2); return (double)__half2float(x); }
            case 2: { __nv_bfloat16 x; std::memcpy(&x, b, 2); return (double)__bfloat162float(x); }
            case 3: { double f; std::memcpy(&f, b, 8); return f; }
            default: return (double)b[0];
            }
        };
        for (int i = 0; i < h; i++)
            for (int j = 0; j < w; j++) {
                const size_t e = layout == 0 ? (size_t)i * w + j
                                             : (layout == 1 ? (size_t)i * L.pitch + j : (size_t)cs_idx(i, j, L.hwp));
                dst[(size_t)i * w + j] = at(e);
            }
        return RGBDFLOW_OK;
    } catch (const ArgError& e) {
        return fail(c, e.code, e.what());
    } catch (const CudaError& e) {
        return fail(c, RGBDFLOW_ERR_CUDA, e.what());
    } catch (const std::exception& e) {
        return fail(c, RGBDFLOW_ERR_INTERNAL, e.what());
    }
}

int rgbdflow_profile(rgbdflow_ctx* c, int enable)
{
    if (!c) return RGBDFLOW_ERR_INVALID_ARG;
    API_BEGIN
    wait_idle(c);
    if (enable) {
        c->prof.reset(new Prof());
        for (int i = 0; i < KC_TOTAL; i++) { c->prof_ms[i] = 0; c->prof_n[i] = 0; c->prof_bytes[i] = 0; }
    } else {
        c->prof.reset();
    }
    return RGBDFLOW_OK;
    API_END(c)
}

int rgbdflow_profile_read(rgbdflow_ctx* c, rgbdflow_kernel_stat* out, int max)
{
    if (!c || (!out && max > 0)) return RGBDFLOW_ERR_INVALID_ARG;
    // the SOR total is the sum of its per-level classes
    c->prof_ms[KC_SOR] = 0;
    c->prof_n[KC_SOR] = 0;
    for (int l = 0; l < 16; l++) { c->prof_ms[KC_SOR] += c->prof_ms[KC_SOR_LEVEL0 + l]; c->prof_n[KC_SOR] += c->prof_n[KC_SOR_LEVEL0 + l]; }
    int k = 0;
    for (int i = 0; i < KC_TOTAL; i++) {
        if (!c->prof_n[i]) continue;
        if (k < max) {
            std::memset(&out[k], 0, sizeof(out[k]));
            if (i < KC_N) std::snprintf(out[k].name, sizeof(out[k].name), "%s", kClassNames[i]);
            else std::snprintf(out[k].name, sizeof(out[k].name), "sor_level%d", i - KC_SOR_LEVEL0);
            out[k].launches = c->prof_n[i];
            out[k].ms = c->prof_ms[i];
            out[k].bytes = c->prof_bytes[i];
        }
        k++;
    }
    return k;
}

int rgbdflow_server_create(rgbdflow_ctx* c, const rgbdflow_server_config* cfg, rgbdflow_server** out)
{
    if (!c || !cfg || !out) return RGBDFLOW_ERR_INVALID_ARG;
    *out = nullptr;
    API_BEGIN
    validate(&cfg->params);
    if (cfg->params.compute == RGBDFLOW_COMPUTE_FP64) throw ArgError(RGBDFLOW_ERR_UNSUPPORTED, "serving runs the FP32 solve");
    if (cfg->max_streams <= 0 || cfg->max_batch <= 0) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "max_streams and max_batch must be > 0");
    RF_CUDA(cudaSetDevice(c->device));
    std::unique_ptr<rgbdflow_server> s(new rgbdflow_server());
    s->ctx = c;
    s->cfg = *cfg;
    RF_CUDA(cudaStreamCreateWithFlags(&s->upload, cudaStreamNonBlocking));
    {
        const char* e = std::getenv("RGBDFLOW_SERVER_SLOTS");
        s->slots.resize(e ? std::max(1, std::min(4, std::atoi(e))) : 4);
    }
    for (auto& sl : s->slots) {
        const int rc = rgbdflow_ctx_create(c->device, 0, &sl.ctx);
        if (rc != RGBDFLOW_OK) throw ArgError(rc, "slot context creation failed");
        sl.st = sl.ctx->stream;
        RF_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
    }
    *out = s.release();
    return RGBDFLOW_OK;
    API_END(c)
}

int rgbdflow_server_destroy(rgbdflow_server* s)
{
    if (!s) return RGBDFLOW_ERR_INVALID_ARG;
    for (auto& sl : s->slots) {
        if (sl.busy) cudaEventSynchronize(sl.done);
        sl.reqs.clear();
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.pin_out) cudaFreeHost(sl.pin_out);
        if (sl.ctx) rgbdflow_ctx_destroy(sl.ctx);
    }
    if (s->upload) cudaStreamSynchronize(s->upload);
    s->queue.clear();
    for (auto& kv : s->streams) {
        kv.second.prev.reset();
        if (kv.second.flow) cudaFree(kv.second.flow);
    }
    s->pool.release_all();
    if (s->upload) cudaStreamDestroy(s->upload);
    delete s;
    return RGBDFLOW_OK;
}

namespace {
void server_prepare(rgbdflow_server* s);
void server_prepare_slot(rgbdflow_server* s, ServerSlot& sl);
// Device arena bytes the other solve slots hold (for the HBM budget of one slot's growth).
size_t other_slot_arenas(const rgbdflow_server* s, const ServerSlot& sl)
{
    size_t n = 0;
    for (const auto& o : s->slots)
        if (&o != &sl) n += o.ctx->arena_cap;
    return n;
}
constexpr int kServerFramesPerStream = 8;  // frame buffer sets stocked per stream (a backlog of ~6 pairs)
constexpr int kServerPrecapture = 40;      // batch graphs captured ahead per slot (within kGraphCache)
}

int rgbdflow_server_submit(rgbdflow_server* s, int stream_id, uint64_t request_id, const rgbdflow_camera_params* cam,
                           const uint8_t* bgr, const float* depth_m, int W, int H, float* flow_out)
{
    if (!s) return RGBDFLOW_ERR_INVALID_ARG;
    rgbdflow_ctx* c = s->ctx;
    API_BEGIN
    MaxTimer timer(&s->counters.max_submit_ms);
    if (!cam || !bgr || !depth_m || W < 2 || H < 2) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "bad frame");
    if (cam->xRes == 0 || !(cam->focalLength > 0)) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "bad camera");
    auto it = s->streams.find(stream_id);
    if (it == s->streams.end()) {
        if ((int)s->streams.size() >= s->cfg.max_streams) throw ArgError(RGBDFLOW_ERR_BUSY, "too many streams");
        it = s->streams.emplace(stream_id, StreamState()).first;
    }
    StreamState& ss = it->second;
    const size_t N = (size_t)W * H;
    const size_t fbytes = N * 3 + N * 4;
    if (s->cfg.hbm_budget_bytes && s->resident_bytes + fbytes + N * 12 > s->cfg.hbm_budget_bytes)
        throw ArgError(RGBDFLOW_ERR_BUDGET, "frame does not fit the HBM budget");
    s->pool.resident = &s->resident_bytes;
    if (!ss.flow || ss.W != W || ss.H != H) {
        // a new stream (or size): stock its frame buffers while the budget allows
        const size_t fb = align_up(N * 3, 256) + N * 4;
        int stock = kServerFramesPerStream;
        while (stock > 0 && s->cfg.hbm_budget_bytes &&
               s->resident_bytes + stock * fb + N * 12 > s->cfg.hbm_budget_bytes / 2)
            stock--;
        RF_CUDA(cudaSetDevice(c->device));
        s->pool.reserve(N, stock);
    }
    RF_CUDA(cudaSetDevice(c->device));
    auto f = std::make_shared<DevFrame>();
    f->W = W; f->H = H; f->cam = *cam;
    f->bufs = s->pool.get(N);
    f->pool = &s->pool;
    f->bgr = f->bufs.dev;
    f->depth = (float*)(f->bufs.dev + align_up(N * 3, 256));
    f->ready = f->bufs.ready;
    // the pinned staging may still feed this buffer set's previous upload
    RF_CUDA(cudaEventSynchronize(f->ready));
    std::memcpy(f->bufs.pin, bgr, N * 3);
    std::memcpy(f->bufs.pin + N * 3, depth_m, N * 4);
    RF_CUDA(cudaMemcpyAsync(f->bgr, f->bufs.pin, N * 3, cudaMemcpyHostToDevice, s->upload));
    RF_CUDA(cudaMemcpyAsync(f->depth, f->bufs.pin + N * 3, N * 4, cudaMemcpyHostToDevice, s->upload));
    RF_CUDA(cudaEventRecord(f->ready, s->upload));
    if (ss.prev && (ss.W != W || ss.H != H)) {  // a resolution change restarts the stream
        ss.has_flow = false;
        ss.prev.reset();
    }
    const bool resized = !ss.flow || ss.W != W || ss.H != H;
    if (resized) {
        if (ss.flow) { RF_CUDA(cudaFree(ss.flow)); s->resident_bytes -= (size_t)ss.W * ss.H * 12; }
        RF_CUDA(cudaMalloc(&ss.flow, N * 12));
        s->resident_bytes += N * 12;
        ss.has_flow = false;
    }
    ss.W = W; ss.H = H;
    if (resized) server_prepare(s);
    if (ss.prev) {
        ServerReq r;
        r.stream = stream_id; r.id = request_id; r.W = W; r.H = H;
        r.f1 = ss.prev; r.f2 = f; r.out_host = flow_out; r.t_submit = mono_now();
        s->queue.push_back(r);
    }
    ss.prev = f;
    return RGBDFLOW_OK;
    API_END(c)
}

namespace {

void server_retire(rgbdflow_server* s, ServerSlot& sl)
{
    MaxTimer timer(&s->counters.max_retire_ms);
    const double now = mono_now();
    // a bounded device wait that gave up fails every pair of the batch (and is cleared)
    const bool failed = *sl.ctx->pin_status != 0;
    if (failed) {
        *sl.ctx->pin_status = 0;
        RF_CUDA(cudaMemsetAsync(sl.ctx->dev_status, 0, sizeof(int), sl.st));
    }
    for (size_t i = 0; i < sl.reqs.size(); i++) {
        ServerReq& r = sl.reqs[i];
        const size_t N = (size_t)r.W * r.H;
        if (r.out_host) std::memcpy(r.out_host, sl.pin_out + sl.out_off[i], N * 12);
        rgbdflow_result res;
        res.stream_id = r.stream; res.request_id = r.id; res.W = r.W; res.H = r.H; res.flow = r.out_host;
        res.submit_time_s = r.t_submit; res.done_time_s = now; res.status = failed ? RGBDFLOW_ERR_TIMEOUT : RGBDFLOW_OK;
        s->ready.push_back(res);
        StreamState& ss = s->streams[r.stream];
        ss.in_flight = false;
        ss.has_flow = true;
        // frames no longer referenced by any pair or stream return to the pool
        r.f1.reset();
        r.f2.reset();
    }
    sl.reqs.clear();
    sl.busy = false;
}

// Device arena and pinned descriptor staging of a slot's batch.
struct SlotNeed {
    size_t arena = 0, pin = 0;
};
SlotNeed slot_need(const std::vector<PairSpec>& ps, const HostParams& hp, int storage)
{
    // the storage type changes plane sizes only, not the descriptor count
    size_t arena = 0, desc = 0;
    if (storage == RGBDFLOW_STORE_FP16) {
        const auto P = make_plan<float, __half>(ps, hp);
        arena = P.arena_bytes; desc = P.desc_bytes;
    } else if (storage == RGBDFLOW_STORE_BF16) {
        const auto P = make_plan<float, __nv_bfloat16>(ps, hp);
        arena = P.arena_bytes; desc = P.desc_bytes;
    } else {
        const auto P = make_plan<float, float>(ps, hp);
        arena = P.arena_bytes; desc = P.desc_bytes;
    }
    return SlotNeed{arena, align_up(desc, 256) + sizeof(PairCtl) * ps.size()};
}
size_t slot_arena_need(const std::vector<PairSpec>& ps, const HostParams& hp, int storage)
{
    return slot_need(ps, hp, storage).arena;
}

// Arena bytes of a batch for admission: the sum of its pairs' single-pair arenas (an upper bound:
// each single-pair plan carries its own control blocks and alignment), cached per pair shape.
size_t admit_need(rgbdflow_server* s, const std::vector<PairSpec>& ps, const HostParams& hp)
{
    static thread_local std::map<std::string, size_t> cache;
    size_t tot = 0;
    for (const auto& q : ps) {
        const std::string key = std::to_string(q.W) + "x" + std::to_string(q.H) + (q.warm() ? "w" : "c") +
                                std::to_string(s->cfg.params.storage) + plan_key({}, hp, 0);
        auto it = cache.find(key);
        if (it == cache.end()) it = cache.emplace(key, slot_arena_need({q}, hp, s->cfg.params.storage)).first;
        tot += it->second;
    }
    return tot;
}

// Sizes a slot's solve memory once for a full batch (max_batch cold pairs of the largest
// registered size) as far as the HBM budget allows, so that serving never regrows an arena
// (which waits for the device and drops the slot's graphs).
void server_presize_slot(rgbdflow_server* s, ServerSlot& sl)
{
    int W = 0, H = 0;
    for (const auto& kv : s->streams)
        if ((long)kv.second.W * kv.second.H > (long)W * H) { W = kv.second.W; H = kv.second.H; }
    if (W < 2 || H < 2) return;
    PairSpec q;
    q.W = W; q.H = H;
    q.f_full = 0.8f * W;
    q.xres_full = (unsigned)W;
    const int nb = std::max(1, std::min(s->cfg.max_batch, s->cfg.max_streams));
    std::vector<PairSpec> ps(nb, q);
    const SlotNeed need = slot_need(ps, host_params(s->cfg.params), s->cfg.params.storage);
    const size_t other = other_slot_arenas(s, sl);
    if (sl.ctx->arena_cap < need.arena &&
        !(s->cfg.hbm_budget_bytes && s->resident_bytes + other + need.arena > s->cfg.hbm_budget_bytes))
        ensure_arena(sl.ctx, need.arena);
    // pinned staging: the slot's descriptors and its results (cudaFreeHost / cudaMallocHost on
    // growth would synchronise the device mid-serving)
    ensure_pin(sl.ctx, need.pin);
    const size_t out = (size_t)nb * align_up((size_t)W * H * 12, 256);
    if (sl.pin_cap < out) {
        if (sl.pin_out) RF_CUDA(cudaFreeHost(sl.pin_out));
        RF_CUDA(cudaMallocHost(&sl.pin_out, out));
        sl.pin_cap = out;
    }
}

// The batches the registered streams can form in the steady state: per frame size any count from
// 0 to the number of streams of that size, max_batch pairs at most, all warm-started when the
// server warm-starts (the cold first pairs of new streams are captured when they come), pairs in
// server_launch's canonical order (larger frames first).  Empty when there are more than
// kServerPrecapture.
std::vector<std::vector<PairSpec>> server_batches(const rgbdflow_server* s)
{
    std::map<std::pair<int, int>, int> count;  // (W, H) -> registered streams
    for (const auto& kv : s->streams)
        if (kv.second.W >= 2 && kv.second.H >= 2) count[{kv.second.W, kv.second.H}]++;
    std::vector<std::pair<std::pair<int, int>, int>> sizes(count.begin(), count.end());
    std::stable_sort(sizes.begin(), sizes.end(), [](const auto& a, const auto& b) {
        return (long)a.first.first * a.first.second > (long)b.first.first * b.first.second;
    });
    static const float kNoFlow = 0;  // marks a pair warm-started; never read (nothing runs)
    std::vector<std::vector<PairSpec>> batches;
    std::vector<int> n(sizes.size(), 0);
    for (;;) {  // an odometer over the per-size counts
        size_t i = 0;
        while (i < n.size() && ++n[i] > sizes[i].second) n[i++] = 0;
        if (i == n.size()) break;
        int pairs = 0;
        for (int v : n) pairs += v;
        if (pairs > s->cfg.max_batch) continue;
        if ((int)batches.size() == kServerPrecapture) return {};
        std::vector<PairSpec> ps;
        for (size_t k = 0; k < sizes.size(); k++)
            for (int j = 0; j < n[k]; j++) {
                PairSpec q;
                q.W = sizes[k].first.first;
                q.H = sizes[k].first.second;
                q.f_full = 0.8f * q.W;
                q.xres_full = (unsigned)q.W;
                q.est = s->cfg.warm_start ? &kNoFlow : nullptr;
                q.warm_early = s->cfg.warm_early_termination;
                ps.push_back(q);
            }
        batches.push_back(std::move(ps));
    }
    return batches;
}

// Readies a slot for the registered streams: its solve memory (server_presize_slot), then the graph
// of every batch of server_batches, captured without running.
void server_prepare_slot(rgbdflow_server* s, ServerSlot& sl)
{
    sl.prepare = false;
    server_presize_slot(s, sl);
    for (const auto& ps : server_batches(s)) prepare_dispatch(sl.ctx, ps, s->cfg.params);
}

// When a stream registers or changes size: ready each idle slot now; a busy slot is readied before
// its next launch (server_step), so the request path neither reallocates nor captures.
void server_prepare(rgbdflow_server* s)
{
    for (auto& sl : s->slots) {
        if (sl.busy) sl.prepare = true;
        else server_prepare_slot(s, sl);
    }
}

void server_launch(rgbdflow_server* s, ServerSlot& sl)
{
    // admit queued requests in arrival order: one pair per stream in flight, max_batch per slot,
    // the slot's solve memory inside the HBM budget
    MaxTimer timer(&s->counters.max_launch_ms);
    const HostParams hp = host_params(s->cfg.params);
    std::vector<ServerReq> take;
    std::vector<PairSpec> specs;
    const size_t other = other_slot_arenas(s, sl);
    for (auto it = s->queue.begin(); it != s->queue.end() && (int)take.size() < s->cfg.max_batch;) {
        StreamState& ss = s->streams[it->stream];
        bool dup = false;
        for (const auto& t : take) dup = dup || t.stream == it->stream;
        if (ss.in_flight || dup) { ++it; continue; }
        PairSpec q;
        q.W = it->W; q.H = it->H;
        resized_cam(it->f1->cam, it->W, q.f_full, q.xres_full);
        q.bgr1 = it->f1->bgr; q.depth1 = it->f1->depth; q.bgr2 = it->f2->bgr; q.depth2 = it->f2->depth;
        q.est = (s->cfg.warm_start && ss.has_flow) ? ss.flow : nullptr;
        q.warm_early = s->cfg.warm_early_termination;
        q.out = ss.flow;
        specs.push_back(q);
        if (s->cfg.hbm_budget_bytes && s->resident_bytes + other + admit_need(s, specs, hp) > s->cfg.hbm_budget_bytes) {
            specs.pop_back();
            break;  // the budget is full: later requests wait for memory
        }
        take.push_back(*it);
        it = s->queue.erase(it);
    }
    if (take.empty()) return;
    // canonical order (largest first) so recurring size mixes reuse one cached graph
    std::vector<size_t> order(take.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        return (long)specs[a].W * specs[a].H > (long)specs[b].W * specs[b].H ||
               ((long)specs[a].W * specs[a].H == (long)specs[b].W * specs[b].H && (specs[a].est != nullptr) < (specs[b].est != nullptr));
    });
    std::vector<PairSpec> ps;
    sl.reqs.clear();
    for (size_t i : order) { ps.push_back(specs[i]); sl.reqs.push_back(take[i]); }
    for (const auto& r : sl.reqs) {
        s->streams[r.stream].in_flight = true;
        RF_CUDA(cudaStreamWaitEvent(sl.st, r.f1->ready, 0));
        RF_CUDA(cudaStreamWaitEvent(sl.st, r.f2->ready, 0));
    }
    size_t total = 0;
    sl.out_off.clear();
    for (const auto& r : sl.reqs) { sl.out_off.push_back(total); total += align_up((size_t)r.W * r.H * 12, 256); }
    if (sl.pin_cap < total) {
        if (sl.pin_out) RF_CUDA(cudaFreeHost(sl.pin_out));
        RF_CUDA(cudaMallocHost(&sl.pin_out, total));
        sl.pin_cap = total;
    }
    dispatch(sl.ctx, ps, s->cfg.params, nullptr, sl.st);
    for (size_t i = 0; i < sl.reqs.size(); i++)
        RF_CUDA(cudaMemcpyAsync(sl.pin_out + sl.out_off[i], ps[i].out, (size_t)ps[i].W * ps[i].H * 12,
                                cudaMemcpyDeviceToHost, sl.st));
    RF_CUDA(cudaMemcpyAsync(sl.ctx->pin_status, sl.ctx->dev_status, sizeof(int), cudaMemcpyDeviceToHost, sl.st));
    RF_CUDA(cudaEventRecord(sl.done, sl.st));
    sl.busy = true;
    s->counters.launches++;
}

}  // namespace

int rgbdflow_server_step(rgbdflow_server* s, int wait, rgbdflow_result* out, int max, int* n_out)
{
    if (!s || !n_out) return RGBDFLOW_ERR_INVALID_ARG;
    *n_out = 0;
    rgbdflow_ctx* c = s->ctx;
    API_BEGIN
    RF_CUDA(cudaSetDevice(c->device));
    // retire finished slots; with `wait`, block on the oldest busy slot if nothing finished
    bool any = false;
    for (auto& sl : s->slots)
        if (sl.busy && cudaEventQuery(sl.done) == cudaSuccess) { server_retire(s, sl); any = true; }
    cudaGetLastError();
    if (wait && !any) {
        ServerSlot* oldest = nullptr;
        for (auto& sl : s->slots)
            if (sl.busy) { oldest = &sl; break; }
        if (oldest) {
            RF_CUDA(cudaEventSynchronize(oldest->done));
            server_retire(s, *oldest);
        }
    }
    // launch into free slots (after readying them for streams registered while they ran)
    for (auto& sl : s->slots) {
        if (!sl.busy && sl.prepare) server_prepare_slot(s, sl);
        if (!sl.busy && !s->queue.empty()) server_launch(s, sl);
    }
    int n = 0;
    while (!s->ready.empty() && n < max) {
        out[n++] = s->ready.front();
        s->ready.pop_front();
    }
    *n_out = n;
    return RGBDFLOW_OK;
    API_END(c)
}

int rgbdflow_server_pending(const rgbdflow_server* s)
{
    if (!s) return 0;
    int n = (int)s->queue.size() + (int)s->ready.size();
    for (const auto& sl : s->slots) n += (int)sl.reqs.size();
    return n;
}

int rgbdflow_server_counters_read(rgbdflow_server* s, int reset, rgbdflow_server_counters* out)
{
    if (!s || !out) return RGBDFLOW_ERR_INVALID_ARG;
    uint64_t graphs = 0, grows = 0;
    for (const auto& sl : s->slots) {
        graphs += sl.ctx->n_graph_builds;
        grows += sl.ctx->n_arena_grows;
    }
    rgbdflow_server_counters k = s->counters;
    for (const auto& sl : s->slots) k.max_graph_build_ms = std::max(k.max_graph_build_ms, sl.ctx->max_build_ms);
    k.frames_allocated = s->pool.misses - s->base_frames;
    k.graphs_built = graphs - s->base_graphs;
    k.arena_grows = grows - s->base_grows;
    *out = k;
    if (reset) {
        s->counters = rgbdflow_server_counters{};
        for (auto& sl : s->slots) sl.ctx->max_build_ms = 0;
        s->base_frames = s->pool.misses;
        s->base_graphs = graphs;
        s->base_grows = grows;
    }
    return RGBDFLOW_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Allocation-free solve: the workspace of one pair lives in this file's static device array.
// The plan is the one rgbdflow_scene_flow_batch_async builds for a batch of one, bound to the
// array instead of a context's arena, and its launches go straight onto the caller's stream.
// ------------------------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(40) << 20;  // one 320 x 240 pair at pyramid ratio <= 0.75
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocDevice {
    char* scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int sms = 0;
};
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];

// Once per device, with that device current: the workspace address and the kernel attributes.
const NoAllocDevice& noalloc_setup(int dev)
{
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc_dev[dev];
    if (d.scratch) return d;
    void* p = nullptr;
    RF_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    int sms = 0;
    RF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    set_kernel_attrs<float, float>();
    d.sms = sms;
    d.scratch = (char*)p;
    return d;
}

// The plan's descriptors reach the workspace as kernel parameters, a chunk per launch: nothing the
// call enqueues reads host memory after the call returns.
constexpr int kDescChunk = 3968;  // with the other parameters, under the 4 KB parameter limit
struct DescChunk {
    unsigned char b[kDescChunk];
};
__global__ void k_put_desc(unsigned char* dst, const DescChunk c, int n)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = c.b[i];
}

int noalloc_fail(char* err, size_t err_len, int code, const std::string& m)
{
    if (err && err_len) {
        const size_t n = std::min(m.size(), err_len - 1);
        std::memcpy(err, m.data(), n);
        err[n] = 0;
    }
    return code;
}

}  // namespace

extern "C" int rgbdflow_scene_flow_noalloc(const rgbdflow_pair* pair, const rgbdflow_params* params, void* stream,
                                           char* err, size_t err_len)
{
    try {
        if (err && err_len) err[0] = 0;
        validate(params);
        if (params->storage != RGBDFLOW_STORE_FP32 || params->compute != RGBDFLOW_COMPUTE_FP32)
            throw ArgError(RGBDFLOW_ERR_UNSUPPORTED, "the allocation-free solve stores and computes in FP32 only");
        if (!pair) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "no pair");
        const rgbdflow_pair& q = *pair;
        if (q.W < 2 || q.H < 2 || !q.bgr1 || !q.bgr2 || !q.depth1_m || !q.depth2_m || !q.flow_out)
            throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "bad size or null buffer");
        if (q.cam.xRes == 0 || !(q.cam.focalLength > 0)) throw ArgError(RGBDFLOW_ERR_INVALID_ARG, "bad camera");
        PairSpec s;
        s.W = q.W; s.H = q.H;
        resized_cam(q.cam, q.W, s.f_full, s.xres_full);
        s.bgr1 = q.bgr1; s.depth1 = q.depth1_m; s.bgr2 = q.bgr2; s.depth2 = q.depth2_m;
        s.est = q.est_flow; s.out = q.flow_out;
        const std::vector<PairSpec> ps(1, s);
        const HostParams hp = host_params(*params);
        Plan<float, float> P = make_plan<float, float>(ps, hp);
        if (P.arena_bytes > kNoAllocScratchBytes)
            throw ArgError(RGBDFLOW_ERR_BUDGET, "a " + std::to_string(q.W) + "x" + std::to_string(q.H) + " pair needs " +
                                                    std::to_string(P.arena_bytes) + " workspace bytes; the static workspace holds " +
                                                    std::to_string(kNoAllocScratchBytes) + " (one 320x240 pair)");
        int dev = 0;
        const cudaError_t ge = cudaGetDevice(&dev);
        if (ge != cudaSuccess) { cudaGetLastError(); throw ArgError(RGBDFLOW_ERR_NO_DEVICE, "no CUDA device"); }
        if (dev < 0 || dev >= kNoAllocMaxDevices) throw ArgError(RGBDFLOW_ERR_UNSUPPORTED, "device index above 63");
        const NoAllocDevice& d = noalloc_setup(dev);
        P.sms = d.sms;
        bind_plan(P, d.scratch);
        unsigned char* db = P.desc.data();
        PrepItem<float>* prep = (PrepItem<float>*)(db + P.prep_items_off);
        prep[0].bgr[0] = q.bgr1; prep[0].bgr[1] = q.bgr2;
        prep[0].depth[0] = q.depth1_m; prep[0].depth[1] = q.depth2_m;
        ((float**)(db + P.out_ptrs_off))[0] = q.flow_out;
        ((EstSrc*)(db + P.est_src_off))[0].f = q.est_flow;
        const cudaStream_t st = (cudaStream_t)stream;
        for (size_t o = 0; o < P.desc_bytes; o += kDescChunk) {
            DescChunk ch;
            const int n = (int)std::min<size_t>(kDescChunk, P.desc_bytes - o);
            std::memcpy(ch.b, P.desc.data() + o, n);
            k_put_desc<<<1, 256, 0, st>>>((unsigned char*)d.scratch + P.desc_off + o, ch, n);
        }
        RF_CUDA(cudaGetLastError());
        enqueue_solve(P, d.scratch, st);
        return RGBDFLOW_OK;
    } catch (const ArgError& e) {
        return noalloc_fail(err, err_len, e.code, e.what());
    } catch (const CudaError& e) {
        return noalloc_fail(err, err_len, RGBDFLOW_ERR_CUDA, e.what());
    } catch (const std::exception& e) {
        return noalloc_fail(err, err_len, RGBDFLOW_ERR_INTERNAL, e.what());
    } catch (...) {
        return noalloc_fail(err, err_len, RGBDFLOW_ERR_INTERNAL, "unknown error");
    }
}

// ------------------------------------------------------------------------------------------
// .flo3 files (host-only)
// ------------------------------------------------------------------------------------------
extern "C" int rgbdflow_flo3_write(const char* path, const float* flow, int W, int H, char* err, size_t err_len)
{
    if (err && err_len) err[0] = 0;
    try {
        flo3_write(path, flow, W, H);
        return RGBDFLOW_OK;
    } catch (const Flo3Error& e) {
        return noalloc_fail(err, err_len, e.code, e.msg);
    } catch (...) {
        return noalloc_fail(err, err_len, RGBDFLOW_ERR_INTERNAL, "unknown error");
    }
}

extern "C" int rgbdflow_flo3_read(const char* path, float* flow, size_t n_floats, int* W, int* H, char* err,
                                  size_t err_len)
{
    if (err && err_len) err[0] = 0;
    try {
        flo3_read(path, flow, n_floats, W, H);
        return RGBDFLOW_OK;
    } catch (const Flo3Error& e) {
        return noalloc_fail(err, err_len, e.code, e.msg);
    } catch (...) {
        return noalloc_fail(err, err_len, RGBDFLOW_ERR_INTERNAL, "unknown error");
    }
}

extern "C" int rgbdflow_flo_write(const char* path, const float* flow, int W, int H, char* err, size_t err_len)
{
    if (err && err_len) err[0] = 0;
    try {
        flo_write(path, flow, W, H);
        return RGBDFLOW_OK;
    } catch (const Flo3Error& e) {
        return noalloc_fail(err, err_len, e.code, e.msg);
    } catch (...) {
        return noalloc_fail(err, err_len, RGBDFLOW_ERR_INTERNAL, "unknown error");
    }
}

extern "C" int rgbdflow_flo_read(const char* path, float* flow, size_t n_floats, int* W, int* H, char* err,
                                 size_t err_len)
{
    if (err && err_len) err[0] = 0;
    try {
        flo_read(path, flow, n_floats, W, H);
        return RGBDFLOW_OK;
    } catch (const Flo3Error& e) {
        return noalloc_fail(err, err_len, e.code, e.msg);
    } catch (...) {
        return noalloc_fail(err, err_len, RGBDFLOW_ERR_INTERNAL, "unknown error");
    }
}
