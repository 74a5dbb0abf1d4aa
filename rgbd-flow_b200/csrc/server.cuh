// server.cuh — the served form: continuous batching of frame pairs from camera streams.
//
// Frames are uploaded once, when submitted, into device buffers that two consecutive pairs of a
// stream share (the frame is frame 2 of one pair and frame 1 of the next).  Each stream keeps its
// last flow on the device; with warm starts a pair is initialised from it and solved at full
// resolution only (sceneFlowWithInit semantics, src/sceneFlowWithInit.cpp:7-81).  Four solve
// slots, each with its own context (arena, stream, graphs), keep the device busy: while some
// slots' batches run, requests that arrive are admitted into a free slot's batch as soon as the
// HBM budget allows, so their uploads and solves overlap the running batches.  Measured on camera
// streams at 30 fps (5 x 640x480 + 3 x 320x240 replayed): with two slots the most served at p99
// under 33 ms was 315 pairs/s (cold); with four, 407.
#pragma once
#include <time.h>

#include <deque>
#include <memory>
#include <unordered_map>

namespace rgbdflow {

static inline double mono_now()
{
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

// Keeps in *slot the longest duration (milliseconds) of the scopes it times.
struct MaxTimer {
    double* slot;
    double t0;
    explicit MaxTimer(double* s) : slot(s), t0(mono_now()) {}
    ~MaxTimer()
    {
        const double ms = 1e3 * (mono_now() - t0);
        if (ms > *slot) *slot = ms;
    }
};

// Device + pinned buffers of one uploaded frame.  They come from, and go back to, the server's
// pool (no allocation, hence no implicit device synchronisation, in the steady state).
struct FrameBufs {
    uint8_t* dev = nullptr;   // bgr (W*H*3, 256-aligned) then depth (W*H float)
    char* pin = nullptr;
    cudaEvent_t ready = nullptr;
    size_t bytes = 0;
};

struct FramePool {
    std::unordered_map<size_t, std::vector<FrameBufs>> free_;
    size_t* resident = nullptr;
    uint64_t misses = 0;  // buffer sets allocated because the stock of their size was empty
    static FrameBufs make(size_t n_px, size_t* resident)
    {
        FrameBufs b;
        b.bytes = align_up(n_px * 3, 256) + n_px * 4;
        RF_CUDA(cudaMalloc(&b.dev, b.bytes));
        RF_CUDA(cudaMallocHost(&b.pin, n_px * 7));
        RF_CUDA(cudaEventCreateWithFlags(&b.ready, cudaEventDisableTiming));
        *resident += b.bytes;
        return b;
    }
    // Stock `count` more buffer sets of this size up front: allocating them while serving (device
    // and page-locked memory) stalls the request loop for milliseconds to a hundred and more,
    // exactly when a burst of arrivals keeps more frames alive.
    void reserve(size_t n_px, int count)
    {
        auto& v = free_[n_px];
        for (int i = 0; i < count; i++) v.push_back(make(n_px, resident));
    }
    FrameBufs get(size_t n_px)
    {
        auto& v = free_[n_px];
        if (!v.empty()) {
            FrameBufs b = v.back();
            v.pop_back();
            return b;
        }
        misses++;
        return make(n_px, resident);
    }
    void put(size_t n_px, const FrameBufs& b) { free_[n_px].push_back(b); }
    void release_all()
    {
        for (auto& kv : free_)
            for (auto& b : kv.second) {
                cudaFree(b.dev);
                cudaFreeHost(b.pin);
                cudaEventDestroy(b.ready);
            }
        free_.clear();
    }
};

struct DevFrame {
    int W = 0, H = 0;
    rgbdflow_camera_params cam{};
    uint8_t* bgr = nullptr;   // device, W*H*3
    float* depth = nullptr;   // device, W*H
    cudaEvent_t ready = nullptr;
    FrameBufs bufs;
    FramePool* pool = nullptr;
    ~DevFrame()
    {
        if (pool) pool->put((size_t)W * H, bufs);
    }
};

struct ServerReq {
    int stream = 0;
    uint64_t id = 0;
    int W = 0, H = 0;
    std::shared_ptr<DevFrame> f1, f2;
    float* out_host = nullptr;
    double t_submit = 0;
};

struct StreamState {
    std::shared_ptr<DevFrame> prev;
    float* flow = nullptr;    // device W*H*3: the last solved flow (warm-start source)
    int W = 0, H = 0;
    bool has_flow = false;
    bool in_flight = false;
};

struct ServerSlot {
    rgbdflow_ctx* ctx = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<ServerReq> reqs;
    bool busy = false;
    bool prepare = false;  // streams registered while busy: size memory and capture graphs when idle
    char* pin_out = nullptr;
    size_t pin_cap = 0;
    std::vector<size_t> out_off;
};

}  // namespace rgbdflow

struct rgbdflow_server {
    rgbdflow_ctx* ctx = nullptr;  // the owning context (device, last error)
    rgbdflow_server_config cfg{};
    cudaStream_t upload = nullptr;
    std::unordered_map<int, rgbdflow::StreamState> streams;
    std::deque<rgbdflow::ServerReq> queue;
    std::vector<rgbdflow::ServerSlot> slots;  // solve slots (4; RGBDFLOW_SERVER_SLOTS: 1..4)
    size_t resident_bytes = 0;    // frame pool + stream flows held on the device
    rgbdflow::FramePool pool;
    std::deque<rgbdflow_result> ready;
    // rgbdflow_server_counters_read: running maxima and step count, and the totals of the last reset
    rgbdflow_server_counters counters{};
    uint64_t base_frames = 0, base_graphs = 0, base_grows = 0;
};
