/*
 * rgbdflow.h — C ABI of the B200-native coarse-to-fine RGB-D scene-flow solver.
 *
 * Every entry point has C linkage, takes plain pointers and sizes, returns an
 * int status (RGBDFLOW_OK == 0, negative on error) and never lets a C++
 * exception cross the boundary.  The message of the last failure on a context
 * is available from rgbdflow_last_error().
 *
 * Reference interfaces replaced (paths inside eherbst/rgbd-flow):
 *   rgbdflow_camera_params           rgbd::CameraParams              include/rgbd_util/CameraParams.h:17-28
 *   rgbdflow_params                  OpticalFlow::sceneFlowParams    include/celiu_flow/OpticalFlow.h:105-129
 *                                    + setUpSceneFlowParams()        src/runFlowTwoFrames.cpp:66-100
 *                                    + solver constants              src/sceneFlowSingleScaleJacobiCUDA.cu:375,461,691,749,768,905,920
 *   rgbdflow_scene_flow_two_frames   runFlowTwoFramesSceneFlowExperiments()  include/rgbd_flow/runFlowTwoFrames.h:49-51
 *                                    (-> ceLiuSceneFlow -> OpticalFlow::sceneFlowMultiscale, or
 *                                        OpticalFlow::sceneFlowWithInit when est_flow != NULL;
 *                                        src/ceLiuOpticalFlow.cpp:190-215)
 *   rgbdflow_scene_flow_multiscale   OpticalFlow::sceneFlowMultiscale()      include/celiu_flow/OpticalFlow.h:133
 *   rgbdflow_scene_flow_with_init    OpticalFlow::sceneFlowWithInit()        include/celiu_flow/OpticalFlow.h:145
 *   rgbdflow_scene_flow_single_scale sceneFlowSingleScale()                  include/celiu_flow/OpticalFlow.h:17-22
 *   rgbdflow_batch_*, rgbdflow_server_*: no counterpart in the reference (batched and
 *                                    served forms of the same solve).
 */
#ifndef RGBDFLOW_H
#define RGBDFLOW_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RGBDFLOW_ABI_VERSION 1

/* status codes */
#define RGBDFLOW_OK                0
#define RGBDFLOW_ERR_INVALID_ARG  (-1)
#define RGBDFLOW_ERR_UNSUPPORTED  (-2)
#define RGBDFLOW_ERR_CUDA         (-3)
#define RGBDFLOW_ERR_BUDGET       (-4) /* request does not fit the context's HBM budget */
#define RGBDFLOW_ERR_TIMEOUT      (-5) /* a bounded device or host wait expired: the solve's results are
                                         not valid; the context stays usable */
#define RGBDFLOW_ERR_NO_DEVICE    (-6)
#define RGBDFLOW_ERR_BUSY         (-7) /* no free slot; retry later */
#define RGBDFLOW_ERR_INTERNAL     (-8)
#define RGBDFLOW_ERR_IO           (-9)  /* a file could not be opened, read or written in full */
#define RGBDFLOW_ERR_FORMAT       (-10) /* a file is not in the expected format */

/* regularisation types (OpticalFlow::sceneFlowRegularizationType, OpticalFlow.h:99-104) */
#define RGBDFLOW_REG_ISOTROPIC 0
#define RGBDFLOW_REG_LETOUZEY  1
#define RGBDFLOW_REG_HPB       2 /* heuristic probability of boundary (the reference's default): 1 - .99 hpb,
                                    hpb from computeHeuristicPb per level (heuristicBoundaries.cpp:40-358) */

/* storage type of the image / depth / gradient pyramids on the device.
 * The flow, the linear system and every Jacobi accumulation stay FP32. */
#define RGBDFLOW_STORE_FP32 0
#define RGBDFLOW_STORE_FP16 1
#define RGBDFLOW_STORE_BF16 2

/* arithmetic of the device solve */
#define RGBDFLOW_COMPUTE_FP32 0
#define RGBDFLOW_COMPUTE_FP64 1 /* FP64 device oracle of the same schedule (EPE reference only) */

/* Mirrors rgbd::CameraParams (include/rgbd_util/CameraParams.h:17-28), field for field. */
typedef struct rgbdflow_camera_params {
    unsigned int xRes;      /* pixels */
    unsigned int yRes;      /* pixels */
    float centerX;          /* pixels */
    float centerY;          /* pixels */
    float focalLength;      /* pixels */
    float stereoBaseline;   /* metres */
    float fovX, fovY;       /* radians */
} rgbdflow_camera_params;

/* OpticalFlow::sceneFlowParams (OpticalFlow.h:105-129) plus every constant the
 * reference hard-codes in its solver.  Fill with rgbdflow_params_default(). */
typedef struct rgbdflow_params {
    int    regularization;             /* RGBDFLOW_REG_* */
    double color_data_weight;          /* colorDataWeight (1) */
    double depth_vs_color_data_weight; /* depthVsColorDataWeight (CLI -v, 1) */
    double alpha;                      /* smoothness weight (CLI -s, 0.02) */
    double gamma;                      /* zero-flow prior (1e-5) */
    double pyramid_ratio;              /* (0.75; values outside [0.4, 0.98] become 0.75 as in GaussianPyramid.cpp:23-24) */
    int    min_width;                  /* (60); a negative value -d means W / d for each pair (W/16 for -16) */
    int    n_outer;                    /* nOuterFPIterations (50) */
    int    n_inner;                    /* nInnerFPIterations (1) */
    int    n_sor;                      /* nSORIterations (maxIters, 10000 from main.cpp:100) */
    int    depth_boundary_dist;        /* depth-sigma increase radius near depth boundaries (4) */
    int    fill_holes;                 /* 1: recursive-median fill of zero depths before the pyramid (reference behaviour) */
    int    fixed_schedule;             /* 1: run every outer and SOR iteration (no convergence breaks) */
    int    storage;                    /* RGBDFLOW_STORE_* */
    int    compute;                    /* RGBDFLOW_COMPUTE_* */
    /* solver constants (sceneFlowSingleScaleJacobiCUDA.cu) */
    double omega;                      /* SOR relaxation (0.7, :461) */
    double max_flow_step;              /* per-sweep step clamp (0.3, :375) */
    double eps_d, eps_z, eps_s;        /* Charbonnier epsilons (1e-6, 1e-10, 1e-6, :749) */
    double sor_tol;                    /* SOR convergence threshold on max |dx| (1e-5, :920) */
    int    sor_check_period;           /* SOR convergence check period (25, :905) */
    double outer_tol;                  /* outer early-termination threshold (4e-4, :691) */
    double occ_margin;                 /* occlusion test margin factor (0.02, :646) */
    double occ_penalty;                /* colour-term weight of occluded pixels (0.01, :646) */
    double max_depth_grad;             /* clamp of depth derivatives (0.04, :768) */
    /* kernel tuning; 0 selects the autotuned value */
    int    sweeps_per_launch;
} rgbdflow_params;

#define RGBDFLOW_MAX_LEVELS 16
#define RGBDFLOW_MAX_OUTER  64

/* What the solve actually executed (early exits are data dependent). */
typedef struct rgbdflow_stats {
    int   n_levels;
    int   level_w[RGBDFLOW_MAX_LEVELS], level_h[RGBDFLOW_MAX_LEVELS];   /* index 0 = finest */
    int   outer_iters[RGBDFLOW_MAX_LEVELS];                           /* outer iterations executed */
    int   sor_iters[RGBDFLOW_MAX_LEVELS][RGBDFLOW_MAX_OUTER];         /* SOR iterations executed per outer */
    float outer_stat[RGBDFLOW_MAX_LEVELS][RGBDFLOW_MAX_OUTER];        /* early-termination statistic (-1 if not evaluated) */
    float sor_maxdiff[RGBDFLOW_MAX_LEVELS][RGBDFLOW_MAX_OUTER];       /* last SOR convergence statistic (-1 if not evaluated) */
    double device_ms;                                                 /* device time of the solve, CUDA events */
} rgbdflow_stats;

/* Reference defaults: sceneFlowParams() + setUpSceneFlowParams(maxIters = 10000) with the
 * demo's CLI defaults (alpha 0.02, depthVsColorDataWeight 1, HPB regularisation). */
void rgbdflow_params_default(rgbdflow_params* p);

/* Version of this ABI (RGBDFLOW_ABI_VERSION). */
int rgbdflow_abi_version(void);

/* Pyramid level sizes a W x H pair is solved at, finest first (GaussianPyramid::ConstructPyramid,
 * src/GaussianPyramid.cpp:22-62).  Host-only: needs no device.  w, h: arrays of at least
 * RGBDFLOW_MAX_LEVELS ints (either may be NULL).  Returns the level count or a negative status. */
int rgbdflow_pyramid_levels(int W, int H, double ratio, int min_width, int* w, int* h);

/* Device bytes a batch of the given pair sizes needs (the context's HBM budget is checked
 * against this).  Host-only.  Ws/Hs: n sizes; warm: NULL or n flags (warm-started pairs are
 * solved at one level).  Returns 0 on success. */
int rgbdflow_batch_device_bytes(const int* Ws, const int* Hs, const int* warm, int n,
                                const rgbdflow_params* params, size_t* bytes);

/* ---------------------------------------------------------------------------------------------
 * Context: owns a CUDA stream, device workspaces (sized lazily, bounded by hbm_budget_bytes),
 * cached CUDA graphs and the last-error string.  One context per host thread; contexts are
 * independent.  hbm_budget_bytes == 0 means "no limit beyond the device's free memory".
 * ------------------------------------------------------------------------------------------- */
typedef struct rgbdflow_ctx rgbdflow_ctx;

int rgbdflow_ctx_create(int device, size_t hbm_budget_bytes, rgbdflow_ctx** out);
int rgbdflow_ctx_destroy(rgbdflow_ctx* ctx);
const char* rgbdflow_last_error(const rgbdflow_ctx* ctx);
/* bytes of device memory the context currently holds */
size_t rgbdflow_ctx_device_bytes(const rgbdflow_ctx* ctx);

/* ---------------------------------------------------------------------------------------------
 * Drop-in for runFlowTwoFramesSceneFlowExperiments (runFlowTwoFrames.cpp:109-121).
 *   bgr1/bgr2: W*H*3 uint8, BGR order (cv::Mat CV_8UC3), row-major
 *   depth1_m/depth2_m: W*H float metres, 0 = invalid
 *   cam: full-size camera; resized to W as in getResizedCamParams (runFlowTwoFrames.cpp:14-24)
 *   est_flow: NULL (coarse-to-fine, sceneFlowMultiscale) or W*H*3 float (u px, v px, w m)
 *             initial estimate (single full-resolution level, sceneFlowWithInit)
 *   flow_out: W*H*3 float (u px, v px, w m), the cv::Mat_<cv::Vec3f> layout
 * Host buffers; the call is synchronous.  stats may be NULL.
 * ------------------------------------------------------------------------------------------- */
int rgbdflow_scene_flow_two_frames(rgbdflow_ctx* ctx, const rgbdflow_camera_params* cam,
                                   const uint8_t* bgr1, const float* depth1_m,
                                   const uint8_t* bgr2, const float* depth2_m,
                                   int W, int H, const rgbdflow_params* params,
                                   const float* est_flow, float* flow_out, rgbdflow_stats* stats);

/* ---------------------------------------------------------------------------------------------
 * OpticalFlow::sceneFlowMultiscale / sceneFlowWithInit over Ce Liu DImage buffers:
 *   Im1/Im2: W*H*3 double in [0,1], channel order as given (the reference keeps BGR)
 *   dm1/dm2: W*H double metres (0 = invalid; filled here when params->fill_holes)
 *   depth_sigma1: W*H float depth standard deviations (params.depthSigma1), must be > 0
 *   u, v, w: W*H double outputs (and inputs for _with_init: the estimate's planes)
 * ------------------------------------------------------------------------------------------- */
int rgbdflow_scene_flow_multiscale(rgbdflow_ctx* ctx, const rgbdflow_camera_params* cam,
                                   const double* Im1, const double* dm1,
                                   const double* Im2, const double* dm2,
                                   const float* depth_sigma1, int W, int H,
                                   const rgbdflow_params* params,
                                   double* u, double* v, double* w, rgbdflow_stats* stats);

int rgbdflow_scene_flow_with_init(rgbdflow_ctx* ctx, const rgbdflow_camera_params* cam,
                                  const double* Im1, const double* dm1,
                                  const double* Im2, const double* dm2,
                                  const float* depth_sigma1, int W, int H,
                                  const rgbdflow_params* params,
                                  double* u, double* v, double* w, rgbdflow_stats* stats);

/* ---------------------------------------------------------------------------------------------
 * The per-level seam sceneFlowSingleScale (OpticalFlow.h:17-22), DImage planes as raw doubles:
 *   Im1, Im2, warpIm2: W*H*nCh interleaved; dm1, dm2, warpDm2: W*H
 *   u, v, w: W*H in/out; warpIm2/warpDm2 in/out (re-warped with the final flow)
 *   depthDataTermWeights, depthSmoothnessTermWeights, depthMagTermWeights: W*H
 *   regularizationWeights: W*H*2 (right, down)
 * params supplies the solver constants (NULL = defaults); its iteration counts are ignored in
 * favour of the explicit arguments, as in the reference signature.
 * ------------------------------------------------------------------------------------------- */
int rgbdflow_scene_flow_single_scale(rgbdflow_ctx* ctx, const rgbdflow_camera_params* cam,
                                     const double* Im1, const double* dm1,
                                     const double* Im2, const double* dm2,
                                     double* warpIm2, double* warpDm2,
                                     double* u, double* v, double* w,
                                     int W, int H, int nCh,
                                     double colorDataTermWeight, const double* depthDataTermWeights,
                                     double alpha, const double* depthSmoothnessTermWeights,
                                     double gamma, const double* depthMagTermWeights,
                                     const double* regularizationWeights,
                                     int nOuterFPIterations, int nInnerFPIterations, int nSORIterations,
                                     int allowEarlyTermination,
                                     const rgbdflow_params* params, rgbdflow_stats* stats);

/* ---------------------------------------------------------------------------------------------
 * Batched form (no reference counterpart): n independent pairs of possibly different sizes
 * solved together, one persistent launch per pyramid level over all pairs' tiles, the level
 * sequence replayed from a cached CUDA graph.  Each pair's result equals its solo result.
 * ------------------------------------------------------------------------------------------- */
typedef struct rgbdflow_pair {
    int W, H;
    rgbdflow_camera_params cam;  /* full-size camera, resized to W like the two-frames call */
    const uint8_t* bgr1;         /* W*H*3 */
    const float*   depth1_m;     /* W*H */
    const uint8_t* bgr2;
    const float*   depth2_m;
    const float*   est_flow;     /* NULL or W*H*3: warm start (single full-resolution level) */
    float*         flow_out;     /* W*H*3 */
} rgbdflow_pair;

/* Host buffers, synchronous.  stats: NULL or an array of n. */
int rgbdflow_scene_flow_batch(rgbdflow_ctx* ctx, const rgbdflow_pair* pairs, int n,
                              const rgbdflow_params* params, rgbdflow_stats* stats);

/* Same, but every pointer in pairs[] is DEVICE memory and the work is enqueued on `stream`
 * (a cudaStream_t passed as void*; NULL = the context's own stream).  Returns after enqueue. */
int rgbdflow_scene_flow_batch_async(rgbdflow_ctx* ctx, const rgbdflow_pair* pairs, int n,
                                    const rgbdflow_params* params, void* stream);

/* Same as rgbdflow_scene_flow_batch (HOST buffers), but returns once the work is enqueued on the
 * context's stream: the inputs' upload, the solve and the flows' download run while the caller
 * goes on, and rgbdflow_ctx_synchronize(ctx) waits for them.  No reference counterpart: a caller
 * that alternates two contexts overlaps one batch's PCIe transfers with the other's solve.
 *   flow_out must be page-locked host memory (cudaMallocHost / cudaHostRegister): the flows are
 *   DMA'd straight into it; RGBDFLOW_ERR_INVALID_ARG otherwise.  Inputs may be pageable (they are
 *   staged before the call returns) or page-locked (DMA'd directly; keep them unchanged until the
 *   context is synchronised).  FP32 compute only (RGBDFLOW_ERR_UNSUPPORTED for FP64).  The flows
 *   of a submitted batch equal rgbdflow_scene_flow_batch's bit for bit. */
int rgbdflow_scene_flow_batch_submit(rgbdflow_ctx* ctx, const rgbdflow_pair* pairs, int n,
                                     const rgbdflow_params* params);

/* Wait for every solve this context enqueued (on any stream).  The device's bounded waits (the
 * grid barriers of the cooperative hole-fill kernels) record a wait that gave up in a status word
 * of the context: synchronous calls return RGBDFLOW_ERR_TIMEOUT for it, and for submitted or
 * device-pointer solves this call does (once; the word is then cleared). */
int rgbdflow_ctx_synchronize(rgbdflow_ctx* ctx);

/* Kernel launches of the last solve enqueued on this context. */
int rgbdflow_ctx_last_launch_count(const rgbdflow_ctx* ctx);

/* ---------------------------------------------------------------------------------------------
 * Kernel timing (no reference counterpart; the reference prints wall-clock phase timers,
 * include/rgbd_util/timer.h:29-56).  While enabled, solves launch their kernels directly (no
 * graph) with CUDA events around every launch; times, launch counts and the algorithmic bytes of
 * the executed work accumulate per kernel class until profiling is disabled.
 * ------------------------------------------------------------------------------------------- */
typedef struct rgbdflow_kernel_stat {
    char   name[32];
    int    launches;
    double ms;      /* summed device time */
    double bytes;   /* algorithmic bytes of the executed work (0 where not counted) */
} rgbdflow_kernel_stat;

int rgbdflow_profile(rgbdflow_ctx* ctx, int enable);

/* SOR autotuner (no reference counterpart; the reference has one SOR kernel configuration).  The
 * first time a pyramid level with given pair sizes is solved on a device, each SOR configuration
 * (tile or strip kernel, sweeps per launch, lane mapping, strip band height) is timed on that
 * level with CUDA events and the fastest is kept for the life of the process; every configuration
 * gives the same flow bit for bit.  RGBDFLOW_AUTOTUNE=0 in the environment turns it off.  Writes
 * the choices made on `device` ("sizes kernel K ... us per SOR iteration; ...") into buf (len bytes,
 * NUL-terminated; either may be 0) and returns the full length. */
int rgbdflow_autotune_describe(int device, char* buf, size_t len);
/* Fills up to max entries; returns the number of kernel classes with launches. */
int rgbdflow_profile_read(rgbdflow_ctx* ctx, rgbdflow_kernel_stat* out, int max);

/* ---------------------------------------------------------------------------------------------
 * Stage read-back (no reference counterpart; diagnostics and per-stage parity tests).  After a
 * solve on ctx, any plane of its device state can be read back: the pyramids, the level inputs
 * the linearisation reads, the flow of each level and the last linear system built at each level.
 * The reference keeps the same quantities as DImage / device buffers inside sceneFlowMultiscale
 * (src/sceneFlowMultiscale.cpp:85-177) and sceneFlowSingleScale (.cu:676-870).
 * ------------------------------------------------------------------------------------------- */
#define RGBDFLOW_PLANE_PYRAMID     0 /* index 0..9: colour 1 (B, G, R in [0, 1]), colour 2 (B, G, R),
                                        filled depth 1, filled depth 2 (m), depth-data weight,
                                        depth-smoothness weight (GaussianPyramid levels) */
#define RGBDFLOW_PLANE_FEATURES1   1 /* index 0..4: im2feature of colour 1 (gray, dx, dy, G-B, G-R) */
#define RGBDFLOW_PLANE_FEATURES2   2 /* index 0..4: the same of colour 2 */
#define RGBDFLOW_PLANE_DEPTH       3 /* index 0, 1: depth 1 / 2 in the storage type */
#define RGBDFLOW_PLANE_DEPTH_MAG   4 /* index 0: depth-magnitude weight */
#define RGBDFLOW_PLANE_REG         5 /* index 0, 1: regularisation weight to the right / lower neighbour */
#define RGBDFLOW_PLANE_FLOW        6 /* index 0..2: u, v (px), w (m) of the level */
#define RGBDFLOW_PLANE_SYSTEM      7 /* index 0..11: the last linearisation's compact system: 1 / diagonal
                                        (u, v, w), couplings uv, uw, vw, right-hand sides (u, v, w),
                                        alpha * phi * right weight, alpha * phi * down weight, depth-
                                        smoothness weight (fillSystemMtxKernel, .cu:477-575) */
#define RGBDFLOW_PLANE_FILL_ROUND  8 /* level 0, index 0, 1: the hole-fill round that filled each pixel of
                                        depth 1 / 2 (0: valid input, 255: never filled) */
#define RGBDFLOW_PLANE_HPB_DEPTH   9 /* index 0: HPB regularisation only: the level of the raw-depth pyramid
                                        (DepthMapPyramid of frame 1's raw depth after the colour-guided
                                        fill of small invalid regions; -1 invalid) */
/* Copies plane (kind, index) of pair `pair` (batch order), pyramid level `level` (0 = finest) of
 * the context's last solve into dst (n doubles, W * H needed, raster order); W and H (either may
 * be NULL) receive the level's size.  Waits for the solve to finish. */
int rgbdflow_debug_read_plane(rgbdflow_ctx* ctx, int pair, int level, int kind, int index, double* dst, size_t n,
                              int* W, int* H);

/* Self-test of the bounded device waits: runs one grid barrier that no other block reaches, which
 * gives up after its spin limit and records it in the context's status word.  Returns
 * RGBDFLOW_ERR_TIMEOUT (the expected outcome) and the wait's duration in *seconds (may be NULL);
 * the context stays usable. */
int rgbdflow_debug_wait_timeout(rgbdflow_ctx* ctx, double* seconds);

/* ---------------------------------------------------------------------------------------------
 * Served form (no reference counterpart): continuous batching over camera streams.  A frame
 * submitted on a stream forms a pair with that stream's previous frame; the stream's previous
 * frame pyramid and previous flow stay resident on the device for warm starts.  Requests are
 * admitted while the HBM budget and the slot count allow (four solve slots, each a batch of up to
 * max_batch pairs on its own stream); newly admitted pairs join the next device step while
 * earlier ones are still in flight.
 * ------------------------------------------------------------------------------------------- */
typedef struct rgbdflow_server rgbdflow_server;

typedef struct rgbdflow_server_config {
    int    max_streams;        /* distinct camera streams */
    int    max_batch;          /* pairs solved per device step */
    size_t hbm_budget_bytes;   /* admission budget for resident state + in-flight pairs */
    int    warm_start;         /* 1: initialise each pair from the stream's previous flow and solve it at
                                  full resolution only (sceneFlowWithInit, src/sceneFlowWithInit.cpp:7-81) */
    int    warm_early_termination; /* 1: warm-started pairs may stop their outer iterations early (the
                                  reference's with-init path never does, sceneFlowWithInit.cpp:74) */
    rgbdflow_params params;
} rgbdflow_server_config;

typedef struct rgbdflow_result {
    int      stream_id;
    uint64_t request_id;
    int      W, H;
    float*   flow;             /* caller buffer given at submit, W*H*3, filled */
    double   submit_time_s;    /* host clock (CLOCK_MONOTONIC) */
    double   done_time_s;
    int      status;           /* RGBDFLOW_OK or an error code */
} rgbdflow_result;

int rgbdflow_server_create(rgbdflow_ctx* ctx, const rgbdflow_server_config* cfg, rgbdflow_server** out);
int rgbdflow_server_destroy(rgbdflow_server* srv);
/* Queue one frame of a stream.  The first frame of a stream only primes it (no result).
 * flow_out (W*H*3 float) receives the flow from the stream's previous frame to this one. */
int rgbdflow_server_submit(rgbdflow_server* srv, int stream_id, uint64_t request_id,
                           const rgbdflow_camera_params* cam, const uint8_t* bgr, const float* depth_m,
                           int W, int H, float* flow_out);
/* Advance the device: admit queued requests, launch a step, retire finished pairs.
 * Non-blocking unless `wait` is set.  Completed results are appended to out (up to max). */
int rgbdflow_server_step(rgbdflow_server* srv, int wait, rgbdflow_result* out, int max, int* n_out);
/* Requests queued or in flight. */
int rgbdflow_server_pending(const rgbdflow_server* srv);

/* Where a served request's latency can go besides the device solve.  Counts and maxima since the
 * server was created or last read with reset = 1.  The server captures the graphs of the batches
 * its registered streams can form when a stream registers (up to 40 per solve slot), so in the
 * steady state graphs_built, arena_grows and frames_allocated stay 0. */
typedef struct rgbdflow_server_counters {
    uint64_t frames_allocated;  /* frame buffer sets allocated after the streams' stock ran out */
    uint64_t graphs_built;      /* solve graphs captured (first sight of a batch composition) */
    uint64_t arena_grows;       /* slot solve-memory reallocations (each waits for the device) */
    uint64_t launches;          /* device steps launched */
    double   max_submit_ms;     /* longest host time inside one submit call */
    double   max_launch_ms;     /* longest host time to admit and enqueue one device step */
    double   max_retire_ms;     /* longest host time to hand one finished step's flows back */
    double   max_graph_build_ms; /* longest capture + instantiation of one solve graph */
} rgbdflow_server_counters;
int rgbdflow_server_counters_read(rgbdflow_server* srv, int reset, rgbdflow_server_counters* out);

/* ---------------------------------------------------------------------------------------------
 * Allocation-free solve (no counterpart in the reference).  For callers that must not allocate
 * once they run: a real-time loop with a fixed memory footprint, a process whose device memory
 * belongs to another allocator, or code that cannot take the implicit device synchronisation of
 * cudaMalloc / cudaFree.  This call allocates no device and no page-locked host memory (its host
 * bookkeeping is ordinary heap memory) and needs no context: its workspace is a 40 MiB array in
 * the library's static device memory, present on every device the library is loaded on.
 *   Limit: one pair whose workspace fits in 40 MiB, i.e. up to 320 x 240 pixels at pyramid ratio
 *   0.75 or below, FP32 storage and compute.  A larger pair is rejected with
 *   RGBDFLOW_ERR_BUDGET, other storage or compute types with RGBDFLOW_ERR_UNSUPPORTED, and
 *   nothing is enqueued then.
 *   pair: DEVICE pointers, with the meaning of rgbdflow_scene_flow_batch_async (same solve, same
 *   result; est_flow NULL or a warm start).  stream: a cudaStream_t as void*, NULL = the legacy
 *   default stream.  Runs on the current device and returns after enqueue.
 *   Set-up: the first call on each device looks up the workspace address and sets kernel
 *   attributes.  The set-up is kept for the life of the process: after cudaDeviceReset on a
 *   device this call is not supported there.
 *   Host memory: the call's descriptors travel to the workspace as kernel parameters, so nothing
 *   it enqueues reads host memory after it returns.
 *   Footprint: the 40 MiB array belongs to the library's device code, so every process that loads
 *   the library holds it on each device where that code is loaded (at the latest when any of the
 *   library's kernels first runs there), whether or not it calls this function.
 *   Zeroing: nothing in the workspace has to start at zero; every call clears, on the stream, the
 *   counters it relies on.
 *   Overlap: all calls on a device share the one workspace.  Two calls whose work overlaps on
 *   the device (different streams, or threads without ordering) race and corrupt each other's
 *   results; keep them on one stream, or order them with events.
 *   err / err_len: NULL or a buffer that receives the error message.
 * ------------------------------------------------------------------------------------------- */
int rgbdflow_scene_flow_noalloc(const rgbdflow_pair* pair, const rgbdflow_params* params, void* stream,
                                char* err, size_t err_len);

/* ---------------------------------------------------------------------------------------------
 * 2-D optical flow: the reference demo's flow type 1, Ce Liu's coarse-to-fine solver
 * (runFlowTwoFramesCeLiu, src/runFlowTwoFrames.cpp:30-45 -> OpticalFlow::Coarse2FineFlow,
 * src/opticalFlowMultiscale.cpp, with SmoothFlowSOR, src/SmoothFlowSOR.cpp).  The device solve
 * keeps the reference's FP64 arithmetic, operation order and lexicographic SOR order, so its flow
 * equals the reference's.  Its SOR runs as overlapping anti-diagonal sweeps in one thread block
 * per inner iteration, with sor_ring sweeps in flight.
 * ------------------------------------------------------------------------------------------- */
typedef struct rgbdflow_flow2d_params {
    double alpha;          /* smoothness weight (the demo's -s, 0.02) */
    double pyramid_ratio;  /* (0.75) */
    int    min_width;      /* (20) */
    int    n_outer;        /* outer fixed-point iterations at the finest level, + k at level k (10) */
    int    n_inner;        /* (1) */
    int    n_sor;          /* SOR iterations at the finest level, + 3 k at level k (400) */
    int    sor_ring;       /* SOR sweeps in flight, 2..16 (8); the result does not depend on it */
} rgbdflow_flow2d_params;

/* The demo's values for flow type 1 (runFlowTwoFramesCeLiu, opticalFlowParams). */
void rgbdflow_flow2d_params_default(rgbdflow_flow2d_params* p);
/* Host buffers (BGR8, W*H*3 each), synchronous.  flow_out: W*H*2 floats (u, v in pixels), the
 * reference's cv::Vec2f result (liu2cvFlow2d).  RGBDFLOW_ERR_INVALID_ARG for alpha < 0 (the
 * reference asserts alpha >= 0), min_width < 1 (the reference's level count never ends), a
 * pyramid_ratio that is not a finite number > 0, n_inner or n_sor < 1, sor_ring outside 2..16. */
int rgbdflow_optical_flow_2d(rgbdflow_ctx* ctx, const uint8_t* bgr1, const uint8_t* bgr2, int W, int H,
                             const rgbdflow_flow2d_params* params, float* flow_out);

/* ---------------------------------------------------------------------------------------------
 * .flo3 scene-flow files: readSceneFlow / writeSceneFlow (src/sceneFlowIO.cpp:18-61), the format
 * the reference's demo writes its result in (src/main.cpp:126).  Layout: the 8 bytes
 * 237 159 43 26 202 94 218 68, int32 width, int32 height, then width*height (u, v, w) float32
 * triples, rows top to bottom; numbers little-endian (the reference writes host order, which is
 * little-endian on its platforms).  Host-only: no device, no context.
 * err / err_len: NULL or a buffer that receives the message of a failure.
 * ------------------------------------------------------------------------------------------- */
/* Writes W*H*3 floats.  A file that cannot be opened or written in full: RGBDFLOW_ERR_IO. */
int rgbdflow_flo3_write(const char* path, const float* flow, int W, int H, char* err, size_t err_len);
/* Reads the size into *W, *H and, with flow != NULL, the W*H*3 values (n_floats >= W*H*3, else
 * RGBDFLOW_ERR_INVALID_ARG).  A file that cannot be opened or ends early: RGBDFLOW_ERR_IO; another
 * magic number or a size below 1: RGBDFLOW_ERR_FORMAT.  Bytes after the last value are ignored. */
int rgbdflow_flo3_read(const char* path, float* flow, size_t n_floats, int* W, int* H, char* err, size_t err_len);

/* Middlebury .flo 2-D flow files: readFlow / writeFlow (src/middleburyFlowIO.cpp:15-65), the
 * format the reference's demo writes 2-D flows in (src/main.cpp:125).  Layout: the 4 bytes "PIEH"
 * (the float 202021.25), int32 width, int32 height, then width*height (u, v) float32 pairs, rows
 * top to bottom, little-endian.  Host-only; arguments, sizes and failures as the .flo3 calls, with
 * W*H*2 values. */
int rgbdflow_flo_write(const char* path, const float* flow, int W, int H, char* err, size_t err_len);
int rgbdflow_flo_read(const char* path, float* flow, size_t n_floats, int* W, int* H, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif /* RGBDFLOW_H */
