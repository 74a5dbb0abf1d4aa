// kernels.cuh — sm_100a device code of the RGB-D scene-flow solve.
//
// Every kernel walks a device-resident work list (LevelItem descriptors + tile lists), so one
// launch serves one pair or a ragged batch of pairs of different sizes alike.  T is the
// arithmetic type (float for the product, double for the FP64 device oracle); S is the storage
// type of the feature / depth planes the linearisation reads (float, __half or __nv_bfloat16).
// All steps are bandwidth- or latency-bound stencils: no step is a dense contraction, so no
// tensor-core path exists here.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cooperative_groups.h>
#include <stdint.h>

namespace rgbdflow {

constexpr int kMaxChecks = 512;  // SOR convergence checks per inner iteration (nSOR / period)

// Linearisation / elementwise tiling.
constexpr int LTW = 32, LTH = 8;  // 256 threads, one interior pixel each

// ------------------------------------------------------------------------------------------
// descriptors

// Per (pair) control block, device resident; written only by the kernels named beside each field.
struct PairCtl {
    int level_done;               // k_control sets it when the outer early-termination test passes
    int sor_stop;                 // k_sor (the CTA of tile 0) sets it once a convergence check breaks
    int sor_stop_iter;            // iterations executed when the break happened
    int pad0;
    unsigned maxdiff[kMaxChecks]; // k_sor: max |dx| of the checked iteration (float bits), per check
    // history (finest level = 0)
    int outer_exec[16];
    int sor_exec[16][64];
    float stat[16][64];
    float sor_maxdiff[16][64];
};

template <class T, class S>
struct LevelItem {
    int W, H;
    int level;                  // 0 = finest
    int allow_early;            // outer early termination permitted at this level
    int est_init;               // flow initialised by the caller (warm start): no upsample
    T f_level;                  // focal length of this level (convergence weights f / depth)
    PairCtl* ctl;
    // pyramid planes of this level (T): colour 1 (3), colour 2 (3), depth 1, depth 2,
    // depth-data weight, depth-smoothness weight
    T* pyr[10];
    // solver inputs (S): features 1 (5), features 2 (5), depth 1, depth 2
    S* I1[5];
    S* I2[5];
    S* D1;
    S* D2;
    T* mag;                     // depth-magnitude weight
    T* rh;                      // regularisation weight to the right neighbour
    T* rv;                      // regularisation weight to the lower neighbour
    int pitch;                  // row pitch (elements) of the u planes: W rounded up to 4
    int hwp;                    // checkerboard half-row length of the x and sys planes (see cs_idx)
    T* u[3];                    // flow (u px, v px, w m)
    T* x[2][3];                 // SOR increment, ping-pong pair
    T* sys[12];                 // compact linear system (see k_linearize)
    T* stat_part;               // per SOR tile partial of the early-termination statistic
    int lin_tiles_x, lin_tile0; // linearisation / elementwise tiles: index base in the step's list
    int n_sor_tiles;            // SOR tiles (32 x 32 interior) of this item
    // coarser level (for the flow upsample); null at the coarsest level
    const T* uc[3];
    int Wc, Hc, pitch_c;
    T inv_ratio;                // 1 / pyramid ratio (u, v scale on upsample)
    // full-resolution info for the depth-magnitude quirk
    int xres_full;
    T f_full;
};

struct Tile {
    int item;  // index into the step's LevelItem array
    int tx, ty;
    int idx;   // tile index within its item
};

// Constants of the solve (sceneFlowSingleScaleJacobiCUDA.cu:375,461,646,691,749,768,905,920).
template <class T>
struct SolveConst {
    T alpha, gamma, color_w;
    T eps_d, eps_z, eps_s;
    T omega, step;
    T occ_margin, occ_penalty, max_grad;
    double sor_tol;
    double outer_tol;
    int fixed;
    int n_sor;
    int period;         // SOR convergence check period (iterations)
};

// One SOR launch of the host schedule.
struct SorLaunch {
    int it0, nit;      // first iteration (within the inner loop) and iteration count
    int xin;           // ping-pong buffer read (0/1); the other one is written
    int xin_zero;      // first launch of an outer iteration: the increment starts at 0
    int final_fold;    // last launch of the outer iteration: u += x and the statistic partials
    int final_keep;    // last launch of a non-final inner iteration: write x
    int check;         // the last iteration of this launch is a convergence check
    int check_idx;     // its slot in PairCtl::maxdiff
    int prev_check;    // the previous launch ended with a check: decide here whether to stop
    int prev_check_idx;
    int outer;         // outer iteration index (stats)
    int seq;           // index of this launch among the level's SOR launches (strip kernel tickets)
    int xout;          // whole-level kernel: ping-pong buffer that receives x (non-final inner iterations)
    int control;       // whole-level kernels: run the outer iteration's control after the fold (k_control's work)
    int n_checks;      // its convergence-check count
};

template <class T, class S>
__device__ __forceinline__ void control_item(const LevelItem<T, S>& it, const SolveConst<T>& k, int outer, int n_checks,
                                             int lane);

// ------------------------------------------------------------------------------------------
// small helpers

template <class S> __device__ __forceinline__ float tof(S v);
template <> __device__ __forceinline__ float tof<float>(float v) { return v; }
template <> __device__ __forceinline__ float tof<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float tof<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <class T, class S> __device__ __forceinline__ T ldS(const S* p) { return (T)tof<S>(p[0]); }
template <> __device__ __forceinline__ double ldS<double, double>(const double* p) { return p[0]; }

template <class S> __device__ __forceinline__ S fromT(float v);
template <> __device__ __forceinline__ float fromT<float>(float v) { return v; }
template <> __device__ __forceinline__ __half fromT<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 fromT<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <class S, class T> __device__ __forceinline__ S stS(T v) { return fromT<S>((float)v); }
template <> __device__ __forceinline__ double stS<double, double>(double v) { return v; }

// Typed math: explicit float / double entry points so FP32 code never widens to FP64.
__device__ __forceinline__ float minT(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double minT(double a, double b) { return ::fmin(a, b); }
__device__ __forceinline__ float maxT(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double maxT(double a, double b) { return ::fmax(a, b); }
__device__ __forceinline__ float absT(float a) { return fabsf(a); }
__device__ __forceinline__ double absT(double a) { return ::fabs(a); }
__device__ __forceinline__ float expT(float a) { return expf(a); }
__device__ __forceinline__ double expT(double a) { return ::exp(a); }

template <class T> __device__ __forceinline__ T rsqrtT(T v);
template <> __device__ __forceinline__ float rsqrtT<float>(float v) { return 1.0f / sqrtf(v); }
template <> __device__ __forceinline__ double rsqrtT<double>(double v) { return 1.0 / sqrt(v); }

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Explicitly rounded arithmetic: the SOR update and the early-termination statistic are written
// with these so that no contraction choice of the compiler can make two kernels that share them
// (the tile and the strip SOR) round differently.
__device__ __forceinline__ float fmaR(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaR(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mulR(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mulR(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float addR(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double addR(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float subR(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double subR(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float divR(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double divR(double a, double b) { return __ddiv_rn(a, b); }

// One pixel's term of the outer early-termination statistic: du^2 + dv^2 + dw^2 * f / depth1
// (sceneFlowSingleScaleJacobiCUDA.cu:943-951).
template <class T>
__device__ __forceinline__ T stat_px(T a, T b, T c, T fl, T dep)
{
    return addR(addR(mulR(a, a), mulR(b, b)), mulR(mulR(c, c), divR(fl, dep)));
}

// Checkerboard ("colour-split") layout of the SOR's planes (system and increment): every row
// holds its (i + j) even pixels first, then its odd ones, each half hwp long, so one colour's
// pixels -- and their other-colour neighbours -- are contiguous.
__host__ __device__ __forceinline__ int cs_idx(int i, int j, int hwp) { return i * 2 * hwp + ((i + j) & 1) * hwp + (j >> 1); }

// ------------------------------------------------------------------------------------------
// Preprocessing at full resolution.

// BGR8 -> [0,1] planes (cv2liuBGR keeps BGR order: ceLiuOpticalFlow.cpp:19-34); depth copies.
template <class T>
struct PrepItem {
    int W, H;
    int kind;                   // 0: BGR8 + float depth; 1: [0,1] FP64 colour + FP64 depth + given sigma
    const uint8_t* bgr[2];
    const float* depth[2];
    const double* im_d[2];      // kind 1: W*H*3 interleaved
    const double* dep_d[2];     // kind 1: W*H
    const float* sigma_in;      // kind 1: depth sigma of frame 1 (params.depthSigma1)
    T* col[2][3];       // level-0 colour planes
    T* dep[2];          // level-0 depth planes (filled in place by the hole fill)
    uint8_t* stamp[2];  // hole-fill round stamps: 0 valid, 255 unfilled, r filled in round r
    uint8_t* bmask;     // depth-boundary mask of frame 1
    T* ddw;             // level-0 depth-data weight
    T* dsw;             // level-0 depth-smoothness weight
    T f2;               // focal length squared (calculateDepthSmoothnessTermWeights)
    T dvc;              // depthVsColorDataWeight
    int max_dist;       // depth-sigma boundary radius
    int tiles_x, tile0;
};

template <class T>
__global__ void k_prep(const PrepItem<T>* items, const Tile* tiles)
{
    const Tile t = tiles[blockIdx.x];
    const PrepItem<T>& it = items[t.item];
    const int j = t.tx * LTW + (threadIdx.x % LTW), i = t.ty * LTH + (threadIdx.x / LTW);
    if (i >= it.H || j >= it.W) return;
    const int l = i * it.W + j;
    for (int f = 0; f < 2; f++) {
        if (it.kind == 0) {
            const uint8_t* b = it.bgr[f] + (size_t)l * 3;
            for (int c = 0; c < 3; c++) it.col[f][c][l] = (T)b[c] / (T)255.0;
            const float z = it.depth[f][l];
            it.dep[f][l] = (T)z;
            it.stamp[f][l] = (z > 0) ? 0 : 255;
        } else {
            const double* b = it.im_d[f] + (size_t)l * 3;
            for (int c = 0; c < 3; c++) it.col[f][c][l] = (T)b[c];
            const double z = it.dep_d[f][l];
            it.dep[f][l] = (T)z;
            it.stamp[f][l] = (z > 0) ? 0 : 255;
        }
    }
    if (it.kind != 0) return;  // sigma supplied by the caller
    // boundary mask (staticDepthNoiseModeling.cpp:92-98); stereoErrorRatio(min z) scales 0.02
    const float* d = it.depth[0];
    const double z = d[l];
    bool bnd = false;
    auto ser = [](double zz) { const double e1 = 1.0 / (1.0 / .00285 + 1.0); return (zz * zz / (1.0 / .00285 + zz)) / e1; };
    if (i < it.H - 1 && d[l + it.W] > 0 && fabs((double)(d[l] - d[l + it.W])) > .02 * ser(fmin((double)d[l], (double)d[l + it.W])))
        bnd = true;
    else if (j < it.W - 1 && d[l + 1] > 0 && fabs((double)(d[l] - d[l + 1])) > .02 * ser(fmin((double)d[l], (double)d[l + 1])))
        bnd = true;
    (void)z;
    it.bmask[l] = bnd;
}

// Depth sigma with the boundary increase (staticDepthNoiseModeling.cpp:232-258, 85-137): the L1
// distance to the nearest boundary pixel is searched over the diamond of radius max_dist (the
// exact cv::distanceTransform L1 value wherever it is <= max_dist).  Writes the level-0
// depth-data and depth-smoothness weights (OpticalFlow.cpp:71-97).
template <class T>
__global__ void k_sigma(const PrepItem<T>* items, const Tile* tiles)
{
    const Tile t = tiles[blockIdx.x];
    const PrepItem<T>& it = items[t.item];
    const int j = t.tx * LTW + (threadIdx.x % LTW), i = t.ty * LTH + (threadIdx.x / LTW);
    if (i >= it.H || j >= it.W) return;
    const int W = it.W, H = it.H, l = i * W + j;
    const double e1 = 1.0 / (1.0 / .00285 + 1.0);
    if (it.kind != 0) {
        it.ddw[l] = (T)(e1 / (double)it.sigma_in[l] * (double)it.dvc);
        it.dsw[l] = it.f2;
        return;
    }
    const float z = it.depth[0][l];
    float s;
    if (z > 0) {
        const float sig1 = (float)e1;
        const double r = ((double)z * z / (1.0 / .00285 + z)) / e1;
        s = (float)fmax(1e-4, (double)sig1 * r);
    } else {
        s = 1.0f;
    }
    const int md = it.max_dist;
    if (md > 0) {
        int best = md + 1;
        for (int di = -md; di <= md && best > 0; di++) {
            const int ii = i + di;
            if (ii < 0 || ii >= H) continue;
            const int rem = md - abs(di);
            for (int dj = -rem; dj <= rem; dj++) {
                const int jj = j + dj;
                if (jj < 0 || jj >= W) continue;
                if (it.bmask[ii * W + jj]) {
                    const int dd = abs(di) + abs(dj);
                    if (dd < best) best = dd;
                }
            }
        }
        if (best <= md) {
            const float a = (float)best / (float)md;
            s = (float)exp((1 - a) * log((double)(10 * s)) + a * log((double)s));
        }
    }
    it.ddw[l] = (T)(e1 / (double)s * (double)it.dvc);
    it.dsw[l] = it.f2;
}

// The parallel recursive-median hole fill.  The reference fills holes one at a time,
// most-known-neighbours first, each from the median of its valid 3x3 neighbours
// (recursiveMedianFiltering.cpp:35-99).  Here the fill runs in rounds: in round r every unfilled
// pixel whose known-neighbour count is >= that of every unfilled pixel in its 3x3 neighbourhood is
// filled, from the pixels valid before the round (round stamps make the rounds deterministic).
// Isolated holes get exactly the reference's value; inside larger holes the order (and so the
// value) can differ from the reference's hash-set order.

// Grid-wide barrier of a cooperative launch (every block resident), bounded: a block that waits
// longer than ~0.3 s sets err and leaves; every later barrier then fails at once.
struct GridSync {
    unsigned count;  // blocks arrived at the current barrier
    unsigned gen;    // barriers completed
    int err;         // a wait gave up
    int pad;
};

__device__ __forceinline__ bool grid_barrier(GridSync* g, unsigned nblocks)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = *(volatile int*)&g->err == 0;
        const unsigned gen0 = *(volatile unsigned*)&g->gen;  // read before arriving
        __threadfence();
        if (atomicAdd(&g->count, 1u) == nblocks - 1) {
            atomicExch(&g->count, 0u);
            __threadfence();
            atomicAdd(&g->gen, 1u);
        } else {
            unsigned spins = 0;
            while (*(volatile unsigned*)&g->gen == gen0) {
                if (++spins > (1u << 22) || *(volatile int*)&g->err) {
                    atomicExch(&g->err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// A bounded wait that gave up leaves the solve's results invalid: recorded in the context's status
// word, which the host reads once the solve has finished (null: the caller has none).
__device__ __forceinline__ void report_wait_failure(int* status)
{
    if (status && threadIdx.x == 0) atomicOr(status, 1);
}

// A grid barrier that no other block reaches: gives up after its bounded wait and reports it (the
// device side of the wait-timeout self-test).
__global__ void k_wait_probe(GridSync* gs, int* status)
{
    if (!grid_barrier(gs, gridDim.x + 1)) report_wait_failure(status);
}

// One round over the tiles of block `blk` of `nblk`.  left[r]: hole pixels (all pairs, both frames)
// still unfilled after round r; tleft[ti]: nonzero while tile ti holds one.  A block takes the tiles
// blk + k nblk; after round 1 it gathers, 32 at a time, only those that still hold holes.
template <class T>
__device__ __forceinline__ void fill_round(const PrepItem<T>* items, const Tile* tiles, int n_tiles, int* left,
                                           int* tleft, int round, int blk, int nblk)
{
    constexpr int FH = LTH + 4, FW = LTW + 4;
    __shared__ int s_list[32];
    __shared__ int s_n;
    __shared__ uint8_t s_st[2][FH][FW];
    const int per = (n_tiles - blk + nblk - 1) / nblk;
    for (int k0 = 0; k0 < per; k0 += 32) {
        if (threadIdx.x < 32) {
            const int k = k0 + threadIdx.x;
            const int ti = blk + k * nblk;
            const bool has = k < per && (round == 1 || tleft[ti] != 0);
            const unsigned m = __ballot_sync(0xffffffffu, has);
            if (has) s_list[__popc(m & ((1u << threadIdx.x) - 1))] = ti;
            if (threadIdx.x == 0) s_n = __popc(m);
        }
        __syncthreads();
        const int n = s_n;
        for (int q = 0; q < n; q++) {
            const int ti = s_list[q];
            const Tile t = tiles[ti];
            const PrepItem<T>& it = items[t.item];
            const int W = it.W, H = it.H;
            const int i0 = t.ty * LTH, j0 = t.tx * LTW;
            // the tile's stamps with a 2-pixel halo, both frames (254: outside the image).  Every
            // decision of a round reads the state at the round's start: a stamp another block
            // sets to `round` meanwhile reads like 255 (neither is known, both are candidates).
            for (int e = threadIdx.x; e < 2 * FH * FW; e += LTW * LTH) {
                const int f = e / (FH * FW), rr = (e / FW) % FH, cc = e % FW;
                const int gi = i0 - 2 + rr, gj = j0 - 2 + cc;
                s_st[f][rr][cc] = (gi >= 0 && gi < H && gj >= 0 && gj < W) ? it.stamp[f][gi * W + gj] : (uint8_t)254;
            }
            __syncthreads();
            const int tx = threadIdx.x % LTW, ty = threadIdx.x / LTW;
            const int j = j0 + tx, i = i0 + ty;
            int nleft = 0;
            for (int f = 0; f < 2 && i < H && j < W; f++) {
                if (s_st[f][ty + 2][tx + 2] != 255) continue;  // valid or already filled
                auto known = [&](int r, int c) { return s_st[f][r][c] < round; };
                auto count = [&](int r, int c) {
                    int kn = 0;
                    for (int a = -1; a <= 1; a++)
                        for (int b = -1; b <= 1; b++)
                            if ((a | b) && known(r + a, c + b)) kn++;
                    return kn;
                };
                const int c = count(ty + 2, tx + 2);
                bool fill = c > 0;
                for (int a = -1; a <= 1 && fill; a++)
                    for (int b = -1; b <= 1; b++) {
                        if (!(a | b)) continue;
                        const int sn = s_st[f][ty + 2 + a][tx + 2 + b];
                        if (sn >= round && sn != 254 && count(ty + 2 + a, tx + 2 + b) > c) { fill = false; break; }
                    }
                if (!fill) { nleft++; continue; }
                float v[8];
                int nv = 0;
                for (int a = -1; a <= 1; a++)
                    for (int b = -1; b <= 1; b++)
                        if ((a | b) && known(ty + 2 + a, tx + 2 + b)) {  // row-major neighbour order
                            const float x = (float)it.dep[f][(i + a) * W + (j + b)];
                            int kk = nv++;
                            while (kk > 0 && v[kk - 1] > x) { v[kk] = v[kk - 1]; kk--; }
                            v[kk] = x;
                        }
                it.dep[f][i * W + j] = (T)v[nv / 2];
                it.stamp[f][i * W + j] = (uint8_t)round;
            }
            // pixels still unfilled after this round: all pairs (end of the rounds) and per tile
            // (later rounds skip the tile when none is left)
            const int any = __syncthreads_count(nleft > 0);
            const unsigned m = __ballot_sync(0xffffffffu, nleft > 0);
            int tot = nleft;
            for (int o = 16; o > 0; o >>= 1) tot += __shfl_down_sync(0xffffffffu, tot, o);
            if ((threadIdx.x & 31) == 0 && m) atomicAdd(&left[round], tot);
            if (threadIdx.x == 0) tleft[ti] = any;
        }
        __syncthreads();  // s_list is refilled
    }
}

// Every round of the fill in one cooperative launch: a grid barrier between rounds, done once no
// hole is left (or after max_rounds, or when a barrier wait gives up).
template <class T>
__global__ void __launch_bounds__(LTW * LTH)
k_fill(const PrepItem<T>* items, const Tile* tiles, int n_tiles, int* left, int* tleft, GridSync* gs, int max_rounds,
       int* status)
{
    for (int round = 1; round <= max_rounds; round++) {
        if (round > 1 && *(volatile int*)&left[round - 1] == 0) break;  // the same value in every block
        fill_round<T>(items, tiles, n_tiles, left, tleft, round, blockIdx.x, gridDim.x);
        if (!grid_barrier(gs, gridDim.x)) {
            report_wait_failure(status);
            break;
        }
    }
}

// ------------------------------------------------------------------------------------------
// Gaussian pyramid (GaussianPyramid.cpp:20-63; Image::GaussianSmoothing Image.h:1179-1199,
// ResizeImage ImageProcessing.h:203-222).  A job smooths up to 10 planes of one source level
// and bilinearly resamples them to the destination level.

template <class T>
struct PyrJob {
    int sW, sH, dW, dH;
    int nplanes;
    int fs;                // filter half-width
    double rate;           // resize ratio
    const T* src[10];
    T* tmp[10];
    T* dst[10];
    int tiles_x_src, tile0_src;  // tiles over the computed source columns (horizontal pass)
    int tiles_x_dst, tile0_dst;  // tiles over the destination
    int hstep, hoff;             // horizontal pass computes columns hoff + hstep * k only: the ones the
                                 // resample reads with a nonzero weight (columns 2k + 1 at rate 1/2,
                                 // 4k + 3 at rate 1/4)
    int tW;                      // row length of tmp: the computed columns side by side
};

constexpr int kMaxTaps = 33;

// One thread per (plane, computed column, row): plane blockIdx.y.
template <class T>
__global__ void k_hfilter(const PyrJob<T>* jobs, const Tile* tiles, const T* __restrict__ gall)
{
    const Tile t = tiles[blockIdx.x];
    const PyrJob<T>& jb = jobs[t.item];
    const int p = blockIdx.y;
    const int kc = t.tx * LTW + (threadIdx.x % LTW), i = t.ty * LTH + (threadIdx.x / LTW);
    const int j = jb.hoff + jb.hstep * kc;
    if (p >= jb.nplanes || i >= jb.sH || kc >= jb.tW || j >= jb.sW) return;
    const T* g = gall + t.item * kMaxTaps;
    const int fs = jb.fs, W = jb.sW;
    const T* s = jb.src[p] + (size_t)i * W;
    T acc = 0;
    for (int l = -fs; l <= fs; l++) acc += s[clampi(j + l, 0, W - 1)] * g[l + fs];
    jb.tmp[p][(size_t)i * jb.tW + kc] = acc;
}

template <class T>
__device__ __forceinline__ T vtap(const T* tp, int W, int H, int x, int y, const T* g, int fs)
{
    T acc = 0;
    for (int l = -fs; l <= fs; l++) acc += tp[(size_t)clampi(y + l, 0, H - 1) * W + x] * g[l + fs];
    return acc;
}

// One thread per (pair of planes, destination pixel): planes 2 blockIdx.y and 2 blockIdx.y + 1.
// tmp holds the computed columns side by side: source column u is tmp column (u - hoff) / hstep
// (corners off the progression have weight 0 and are skipped).
constexpr int kVresizePlanes = 2;
template <class T>
__global__ void k_vresize(const PyrJob<T>* jobs, const Tile* tiles, const T* __restrict__ gall)
{
    const Tile t = tiles[blockIdx.x];
    const PyrJob<T>& jb = jobs[t.item];
    const int j = t.tx * LTW + (threadIdx.x % LTW), i = t.ty * LTH + (threadIdx.x / LTW);
    if (i >= jb.dH || j >= jb.dW) return;
    const T* g = gall + t.item * kMaxTaps;
    const double x = (double)(j + 1) / jb.rate - 1, y = (double)(i + 1) / jb.rate - 1;
    const int xx = (int)x, yy = (int)y;
    double dx = x - xx, dy = y - yy;
    dx = dx > 1 ? 1 : (dx < 0 ? 0 : dx);
    dy = dy > 1 ? 1 : (dy < 0 ? 0 : dy);
    const int u0 = clampi(xx, 0, jb.sW - 1), u1 = clampi(xx + 1, 0, jb.sW - 1);
    const int v0 = clampi(yy, 0, jb.sH - 1), v1 = clampi(yy + 1, 0, jb.sH - 1);
    const T s00 = (T)(fabs(1 - dx) * fabs(1 - dy)), s01 = (T)(fabs(1 - dx) * fabs(dy));
    const T s10 = (T)(fabs(dx) * fabs(1 - dy)), s11 = (T)(fabs(dx) * fabs(dy));
    // a corner of weight 0 adds exactly 0 (every pyramid value is finite): it is skipped, which at
    // rates 1/2 and 1/4 (samples on source pixels) leaves one corner of four
    const int c0 = (u0 - jb.hoff) / jb.hstep, c1 = (u1 - jb.hoff) / jb.hstep;
    const int p1 = min(jb.nplanes, (int)(blockIdx.y + 1) * kVresizePlanes);
    for (int p = blockIdx.y * kVresizePlanes; p < p1; p++) {
        const T* tp = jb.tmp[p];
        T acc = 0;
        acc += vtap(tp, jb.tW, jb.sH, c0, v0, g, jb.fs) * s00;
        if (s01 != (T)0) acc += vtap(tp, jb.tW, jb.sH, c0, v1, g, jb.fs) * s01;
        if (s10 != (T)0) acc += vtap(tp, jb.tW, jb.sH, c1, v0, g, jb.fs) * s10;
        if (s11 != (T)0) acc += vtap(tp, jb.tW, jb.sH, c1, v1, g, jb.fs) * s11;
        jb.dst[p][(size_t)i * jb.dW + j] = acc;
    }
}

// ------------------------------------------------------------------------------------------
// Level set-up: features (OpticalFlow::im2feature RGB_WITH_GRADIENT, OpticalFlow.cpp:189-214),
// depth copies in storage type, depth-magnitude weight (OpticalFlow.cpp:104-111, including the
// reference's full-resolution indexing), regularisation weights (OpticalFlow.cpp:113-141) and
// the initial flow (zero at the coarsest level, else the coarser flow resized with
// ResizeImage(dims) and u, v scaled by 1/ratio: sceneFlowMultiscale.cpp:120-134).

template <class T>
__device__ __forceinline__ T gray_at(const T* const* c, int l)
{
    return c[0][l] * (T).114 + c[1][l] * (T).587 + c[2][l] * (T).299;
}

template <class T, class S>
__global__ void k_level_setup(const LevelItem<T, S>* items, const Tile* tiles, int regtype)
{
    const Tile t = tiles[blockIdx.x];
    const LevelItem<T, S>& it = items[t.item];
    const int j = t.tx * LTW + (threadIdx.x % LTW), i = t.ty * LTH + (threadIdx.x / LTW);
    if (t.idx == 0 && threadIdx.x == 0) it.ctl->level_done = 0;
    if (i >= it.H || j >= it.W) return;
    const int W = it.W, H = it.H, l = i * W + j;
    const T gf[5] = {(T)1 / 12, (T)-8 / 12, (T)0, (T)8 / 12, (T)-1 / 12};
    for (int f = 0; f < 2; f++) {
        const T* const* c = (const T* const*)(it.pyr + 3 * f);
        T gx = 0, gy = 0;
        for (int m = -2; m <= 2; m++) gx += gray_at(c, i * W + clampi(j + m, 0, W - 1)) * gf[m + 2];
        for (int m = -2; m <= 2; m++) gy += gray_at(c, clampi(i + m, 0, H - 1) * W + j) * gf[m + 2];
        S* const* o = f ? it.I2 : it.I1;
        o[0][l] = stS<S>(gray_at(c, l));
        o[1][l] = stS<S>(gx);
        o[2][l] = stS<S>(gy);
        o[3][l] = stS<S>(c[1][l] - c[0][l]);
        o[4][l] = stS<S>(c[1][l] - c[2][l]);
    }
    const T z1 = it.pyr[6][l];
    it.D1[l] = stS<S>(z1);
    it.D2[l] = stS<S>(it.pyr[7][l]);
    {
        const int src = (l / it.xres_full) * W + (l % it.xres_full);
        const T z = it.pyr[6][src];
        const T q = (z > 0) ? it.f_full / z : it.f_full / 2;
        it.mag[l] = q * q;
    }
    if (regtype != 2) {  // HPB weights are written by the HPB kernels (hpb.cuh)
        T rh = 0, rv = 0;
        if (regtype == 1) {
            if (j < W - 1) { const T d = (z1 - it.pyr[6][l + 1]) / (T).02; rh = expT(-(d * d)); }
            if (i < H - 1) { const T d = (z1 - it.pyr[6][l + W]) / (T).02; rv = expT(-(d * d)); }
        } else {
            rh = (j < W - 1) ? (T)1 : (T)0;
            rv = (i < H - 1) ? (T)1 : (T)0;
        }
        it.rh[l] = rh;
        it.rv[l] = rv;
    }
    if (it.est_init) return;  // flow supplied by the caller
    const int lp = i * it.pitch + j;
    if (it.uc[0] == nullptr) {
        it.u[0][lp] = 0; it.u[1][lp] = 0; it.u[2][lp] = 0;
    } else {
        const double xr = (double)W / it.Wc, yr = (double)H / it.Hc;
        const double x = (double)(j + 1) / xr - 1, y = (double)(i + 1) / yr - 1;
        const int xx = (int)x, yy = (int)y;
        double dx = x - xx, dy = y - yy;
        dx = dx > 1 ? 1 : (dx < 0 ? 0 : dx);
        dy = dy > 1 ? 1 : (dy < 0 ? 0 : dy);
        const int u0 = clampi(xx, 0, it.Wc - 1), u1 = clampi(xx + 1, 0, it.Wc - 1);
        const int v0 = clampi(yy, 0, it.Hc - 1), v1 = clampi(yy + 1, 0, it.Hc - 1);
        const T s00 = (T)(fabs(1 - dx) * fabs(1 - dy)), s01 = (T)(fabs(1 - dx) * fabs(dy));
        const T s10 = (T)(fabs(dx) * fabs(1 - dy)), s11 = (T)(fabs(dx) * fabs(dy));
        for (int c = 0; c < 3; c++) {
            const T* s = it.uc[c];
            const int pc = it.pitch_c;
            T acc = 0;
            acc += s[v0 * pc + u0] * s00;
            acc += s[v1 * pc + u0] * s01;
            acc += s[v0 * pc + u1] * s10;
            acc += s[v1 * pc + u1] * s11;
            it.u[c][lp] = (c < 2) ? acc * it.inv_ratio : acc;
        }
    }
}

// ------------------------------------------------------------------------------------------
// Linearisation: one fused kernel per inner iteration.  Per interior pixel it warps frame 2 by
// the current flow (warpColorImgWithSceneFlowKernel / warpDepthImgWithSceneFlowKernel,
// .cu:579-635), takes the 5-tap derivatives of 0.4*I1 + 0.6*warped I2 (.cu:84-147), the
// occlusion weight (.cu:640-648), the robust weights phi / psi / pi (.cu:340-371), the weighted
// products (.cu:189-230), the normalised weighted Laplacians (.cu:240-333) and writes the
// compact form of the system of fillSystemMtxKernel (.cu:477-575):
//   sys[0..2]  reciprocal of the diagonal (u, v, w rows)
//   sys[3..5]  symmetric couplings uv, uw, vw
//   sys[6..8]  right-hand sides
//   sys[9]     alpha * phi * (right regularisation weight)   (0 on the last column)
//   sys[10]    alpha * phi * (down regularisation weight)    (0 on the last row)
//   sys[11]    depth-smoothness weight s (w-row neighbour coefficients are edge * s of the
//              edge's left / upper pixel)
// The neighbour coefficient of the u/v rows toward the left (upper) pixel is sys[9] (sys[10])
// of that pixel, so the 8-plane matrix of the reference is implied without being stored.

constexpr int LRW = LTW + 4, LRH = LTH + 4;  // warped region (halo 2)
template <class T> constexpr size_t lin_smem_bytes() { return sizeof(T) * 19 * LRW * LRH; }

template <class T, class S>
__global__ void __launch_bounds__(LTW * LTH)
k_linearize(const LevelItem<T, S>* items, const Tile* tiles, SolveConst<T> k, int use_du, int xsel)
{
    const Tile t = tiles[blockIdx.x];
    const LevelItem<T, S>& it = items[t.item];
    PairCtl* ctl = it.ctl;
    if (ctl->level_done) return;
    if (t.idx == 0) {
        if (threadIdx.x == 0) { ctl->sor_stop = 0; ctl->sor_stop_iter = -1; }
        for (int c = threadIdx.x; c < kMaxChecks; c += blockDim.x) ctl->maxdiff[c] = 0;
    }
    const int W = it.W, H = it.H;
    const int x0 = t.tx * LTW, y0 = t.ty * LTH;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    typedef T Plane[LRH][LRW];
    Plane* sB = reinterpret_cast<Plane*>(smem_raw);  // [6] 0.4*I1 + 0.6*warped I2 (5 features + depth)
    Plane* sDT = sB + 6;                              // [6] warped I2 - I1
    Plane* sU = sDT + 6;                              // [3] flow u
    Plane* sUD = sU + 3;                              // [3] u + du
    Plane& sPhi = *(sUD + 3);                         // robust smoothness weight
    const int tid = threadIdx.x;
    for (int r = tid; r < LRW * LRH; r += blockDim.x) {
        const int ry = r / LRW, rx = r % LRW;
        const int gi = y0 - 2 + ry, gj = x0 - 2 + rx;
        if (gi < 0 || gj < 0 || gi >= H || gj >= W) continue;
        const int l = gi * W + gj, lp = gi * it.pitch + gj;
        T U[3], D[3];
        for (int c = 0; c < 3; c++) {
            U[c] = it.u[c][lp];
            D[c] = use_du ? it.x[xsel][c][cs_idx(gi, gj, it.hwp)] : (T)0;
            sU[c][ry][rx] = U[c];
            sUD[c][ry][rx] = U[c] + D[c];
        }
        const T x = (T)gj + U[0], y = (T)gi + U[1];
        T wI[6], I1v[6];
        for (int c = 0; c < 5; c++) I1v[c] = ldS<T, S>(it.I1[c] + l);
        I1v[5] = ldS<T, S>(it.D1 + l);
        if (x < 0 || x > (T)(W - 1) || y < 0 || y > (T)(H - 1)) {
            for (int c = 0; c < 5; c++) wI[c] = I1v[c];
            wI[5] = I1v[5] - U[2];
        } else {
            const int xa = clampi((int)floor(x), 0, W - 1), ya = clampi((int)floor(y), 0, H - 1);
            const int xb = min(W - 1, xa + 1), yb = min(H - 1, ya + 1);
            const T ax = x - (T)xa, ay = y - (T)ya;
            const T w00 = (1 - ax) * (1 - ay), w01 = (1 - ax) * ay, w10 = ax * (1 - ay), w11 = ax * ay;
            const int p00 = ya * W + xa, p01 = yb * W + xa, p10 = ya * W + xb, p11 = yb * W + xb;
            for (int c = 0; c < 5; c++) {
                const S* s = it.I2[c];
                wI[c] = w00 * ldS<T, S>(s + p00) + w01 * ldS<T, S>(s + p01) + w10 * ldS<T, S>(s + p10) +
                        w11 * ldS<T, S>(s + p11);
            }
            const S* s = it.D2;
            wI[5] = w00 * ldS<T, S>(s + p00) + w01 * ldS<T, S>(s + p01) + w10 * ldS<T, S>(s + p10) +
                    w11 * ldS<T, S>(s + p11) - U[2];
        }
        for (int c = 0; c < 6; c++) {
            sB[c][ry][rx] = (T).4 * I1v[c] + (T).6 * wI[c];
            sDT[c][ry][rx] = wI[c] - I1v[c];
        }
    }
    __syncthreads();
    // robust smoothness weight phi on the interior plus the column to its left and the row above
    for (int r = tid; r < (LTW + 1) * (LTH + 1); r += blockDim.x) {
        const int ry = 1 + r / (LTW + 1), rx = 1 + r % (LTW + 1);
        const int gi = y0 - 2 + ry, gj = x0 - 2 + rx;
        if (gi < 0 || gj < 0 || gi >= H || gj >= W) continue;
        T d[6];
        for (int c = 0; c < 3; c++) {
            d[2 * c] = (gj == W - 1) ? (T)0 : sUD[c][ry][rx + 1] - sUD[c][ry][rx];
            d[2 * c + 1] = (gi == H - 1) ? (T)0 : sUD[c][ry + 1][rx] - sUD[c][ry][rx];
        }
        const T s = it.pyr[9][gi * W + gj];
        const T q = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + d[3] * d[3] + s * (d[4] * d[4] + d[5] * d[5]);
        sPhi[ry][rx] = (T)0.5 * rsqrtT<T>(q + k.eps_s);
    }
    __syncthreads();
    const int lx = tid % LTW, ly = tid / LTW;
    const int gi = y0 + ly, gj = x0 + lx;
    if (gi >= H || gj >= W) return;
    const int l = gi * W + gj;
    const int ry = ly + 2, rx = lx + 2;
    const T gfl[5] = {1, -8, 0, 8, -1};
    T Ix[6], Iy[6], It[6];
    for (int c = 0; c < 6; c++) {
        T sx = 0, sy = 0;
        for (int m = 0; m < 5; m++) {
            const int cc = clampi(gj - 2 + m, 0, W - 1) - (x0 - 2);
            const int rr = clampi(gi - 2 + m, 0, H - 1) - (y0 - 2);
            sx += gfl[m] * sB[c][ry][cc];
            sy += gfl[m] * sB[c][rr][rx];
        }
        Ix[c] = sx / (T)12;
        Iy[c] = sy / (T)12;
        It[c] = sDT[c][ry][rx];
    }
    Ix[5] = minT(maxT(Ix[5], -k.max_grad), k.max_grad);
    Iy[5] = minT(maxT(Iy[5], -k.max_grad), k.max_grad);
    It[5] = minT(maxT(It[5], -k.max_grad), k.max_grad);
    const T U0 = sU[0][ry][rx], U1 = sU[1][ry][rx], U2 = sU[2][ry][rx];
    const T du0 = sUD[0][ry][rx] - U0, du1 = sUD[1][ry][rx] - U1, du2 = sUD[2][ry][rx] - U2;
    const T z1 = ldS<T, S>(it.D1 + l);
    const T q = (z1 + U2 < ldS<T, S>(it.D2 + l) + k.occ_margin * (z1 * z1)) ? (T)1 : k.occ_penalty;
    T sxy = 0, sx2 = 0, sy2 = 0, stx = 0, sty = 0;
    for (int c = 0; c < 5; c++) {
        const T e = (It[c] + Ix[c] * du0 + Iy[c] * du1) * q;
        const T psi = (T)0.5 * rsqrtT<T>(e * e + k.eps_d) * k.color_w;
        sxy += psi * Ix[c] * Iy[c];
        sx2 += psi * Ix[c] * Ix[c];
        sy2 += psi * Iy[c] * Iy[c];
        stx += psi * Ix[c] * It[c];
        sty += psi * Iy[c] * It[c];
    }
    const T ixy = sxy / (T)5, ix2 = sx2 / (T)5, iy2 = sy2 / (T)5;
    const T itx = stx * q * q / (T)5, ity = sty * q * q / (T)5;
    const T e2 = It[5] + Ix[5] * du0 + Iy[5] * du1 - du2;
    const T pi = (T)0.5 * rsqrtT<T>(e2 * e2 + k.eps_z) * it.pyr[8][l];
    const T dxy = pi * Ix[5] * Iy[5], dx2 = pi * Ix[5] * Ix[5], dy2 = pi * Iy[5] * Iy[5];
    const T dtx = pi * Ix[5] * It[5], dty = pi * Iy[5] * It[5];
    // weighted Laplacians of u (not u + du) and edge weights
    const bool hasR = gj < W - 1, hasL = gj > 0, hasD = gi < H - 1, hasU = gi > 0;
    const T rhl = it.rh[l], rvl = it.rv[l];
    const T rhL = hasL ? it.rh[l - 1] : (T)0, rvU = hasU ? it.rv[l - W] : (T)0;
    const T phi = sPhi[ry][rx];
    const T phiL = hasL ? sPhi[ry][rx - 1] : (T)0, phiU = hasU ? sPhi[ry - 1][rx] : (T)0;
    T nrm = 0;
    int cnt = 0;
    if (hasR) { nrm += rhl; cnt++; }
    if (hasL) { nrm += rhL; cnt++; }
    if (hasD) { nrm += rvl; cnt++; }
    if (hasU) { nrm += rvU; cnt++; }
    T lap[3];
    for (int c = 0; c < 3; c++) {
        T lv = 0;
        const T uc = sU[c][ry][rx];
        if (hasR) lv -= (sU[c][ry][rx + 1] - uc) * phi * rhl;
        if (hasL) lv += (uc - sU[c][ry][rx - 1]) * phiL * rhL;
        if (hasD) lv -= (sU[c][ry + 1][rx] - uc) * phi * rvl;
        if (hasU) lv += (uc - sU[c][ry - 1][rx]) * phiU * rvU;
        lap[c] = (absT(nrm) < (T)1e-5) ? (T)0 : lv / (nrm / (T)cnt);
    }
    const T s = it.pyr[9][l];
    const T sL = hasL ? it.pyr[9][l - 1] : (T)0, sU_ = hasU ? it.pyr[9][l - W] : (T)0;
    T sumXY = 0, sumZ = 0;
    if (hasL) { const T e = phiL * rhL; sumXY += e; sumZ += e * sL; }
    if (hasU) { const T e = phiU * rvU; sumXY += e; sumZ += e * sU_; }
    if (hasR) { const T e = phi * rhl; sumXY += e; sumZ += e * s; }
    if (hasD) { const T e = phi * rvl; sumXY += e; sumZ += e * s; }
    const T al = k.alpha, ga = k.gamma, mg = it.mag[l];
    T* const* o = it.sys;
    const int lp = cs_idx(gi, gj, it.hwp);
    // reciprocals of the diagonal: the SOR multiplies instead of dividing
    o[0][lp] = (T)1 / (-(ix2 + dx2 + al * sumXY) - ga);
    o[1][lp] = (T)1 / (-(iy2 + dy2 + al * sumXY) - ga);
    o[2][lp] = (T)1 / (-(pi + al * sumZ) - ga * mg);
    o[3][lp] = -ixy - dxy;
    o[4][lp] = pi * Ix[5];
    o[5][lp] = pi * Iy[5];
    o[6][lp] = -(-itx - dtx + al * -lap[0]) + ga * U0;
    o[7][lp] = -(-ity - dty + al * -lap[1]) + ga * U1;
    o[8][lp] = -(pi * It[5] + al * -(s * lap[2])) + ga * mg * U2;
    o[9][lp] = hasR ? al * (phi * rhl) : (T)0;
    o[10][lp] = hasD ? al * (phi * rvl) : (T)0;
    o[11][lp] = s;
}

// ------------------------------------------------------------------------------------------
// Red-black SOR, K iterations per launch (temporal blocking), persistent CTAs.
//
// The work unit is a fixed 32 x 32 interior tile.  A CTA loads the tile plus a halo of 2K pixels
// (12 system planes + 3 increment planes) into shared memory with cp.async, runs the red and
// black half-sweeps of K iterations over the whole region (errors from the unknown outside of the
// halo creep inward one pixel per half-sweep and never reach the interior), and writes back the
// interior.  With NBUF = 2 the next tile's region streams in while the current one is solved.
// x ping-pongs between two global buffers, so no CTA reads a neighbour's already-updated values.
// Same-colour updates are independent, so the interior equals a whole-image sweep colour by
// colour (sceneFlowSingleScaleJacobiKernel, .cu:382-470): each unknown of a pixel is updated from
// the pre-sweep values of the other two (pointwise Jacobi inside red-black Gauss-Seidel), relaxed
// with omega and clamped to +-max_flow_step around its old value; the result does not depend on
// K or on the tiling.

constexpr int kSorTW = 32, kSorTH = 32;  // interior tile (fixed: per-tile reductions stay identical)

template <class T, int K, int NBUF> struct SorGeom {
    static constexpr int RW = (kSorTW + 4 * K + 8 + 7) & ~7;  // region width incl. alignment slack; HRW % 4 == 0
    static constexpr int HRW = RW / 2;                // checkerboard half-row length
    static constexpr int RH = kSorTH + 4 * K;
    static constexpr int NPL = 15;                    // planes: 12 system + 3 increment
    static constexpr int NT = 512;
    static constexpr size_t buf_elems = (size_t)NPL * RH * RW;
    static constexpr size_t smem = sizeof(T) * (NBUF * buf_elems + 64);
};
template <class T, int K, int NBUF> constexpr size_t sor_smem_bytes() { return SorGeom<T, K, NBUF>::smem; }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <class T>
__device__ __forceinline__ void sor_point(const T* c, T aL, T aU, T aR, T aD, T sL, T sU, T s,
                                          const T* xl, const T* xu, const T* xr, const T* xd, const T* xp,
                                          T omega, T step, T* out)
{
    // Each row: v = (rhs - sum of neighbour terms - the other two unknowns' terms) / diag, relaxed
    // and clamped; every product-subtract is one fused multiply-add, in the reference's order.
    const T omc = (T)1 - omega;
    // u row
    T v = -mulR(aL, xl[0]);
    v = fmaR(-aU, xu[0], v); v = fmaR(-aR, xr[0], v); v = fmaR(-aD, xd[0], v);
    v = addR(v, c[6]);
    v = fmaR(-c[3], xp[1], v); v = fmaR(-c[4], xp[2], v);
    v = mulR(v, c[0]);
    T r = fmaR(omega, v, mulR(omc, xp[0]));
    out[0] = minT(maxT(r, subR(xp[0], step)), addR(xp[0], step));
    // v row
    v = -mulR(aL, xl[1]);
    v = fmaR(-aU, xu[1], v); v = fmaR(-aR, xr[1], v); v = fmaR(-aD, xd[1], v);
    v = addR(v, c[7]);
    v = fmaR(-c[3], xp[0], v); v = fmaR(-c[5], xp[2], v);
    v = mulR(v, c[1]);
    r = fmaR(omega, v, mulR(omc, xp[1]));
    out[1] = minT(maxT(r, subR(xp[1], step)), addR(xp[1], step));
    // w row: neighbour coefficients carry the depth-smoothness weight of the edge's source pixel
    v = -mulR(mulR(aL, sL), xl[2]);
    v = fmaR(-mulR(aU, sU), xu[2], v); v = fmaR(-mulR(aR, s), xr[2], v); v = fmaR(-mulR(aD, s), xd[2], v);
    v = addR(v, c[8]);
    v = fmaR(-c[4], xp[0], v); v = fmaR(-c[5], xp[1], v);
    v = mulR(v, c[2]);
    r = fmaR(omega, v, mulR(omc, xp[2]));
    out[2] = minT(maxT(r, subR(xp[2], step)), addR(xp[2], step));
}

// Two same-colour neighbours of one row as one aligned vector access (even index).
template <class T> struct Vec2;
template <> struct Vec2<float> { typedef float2 t; };
template <> struct Vec2<double> { typedef double2 t; };
template <class T> __device__ __forceinline__ typename Vec2<T>::t ld2(const T* p)
{
    return *reinterpret_cast<const typename Vec2<T>::t*>(p);
}
template <class T> __device__ __forceinline__ void st2(T* p, T a, T b)
{
    typename Vec2<T>::t v;
    v.x = a;
    v.y = b;
    *reinterpret_cast<typename Vec2<T>::t*>(p) = v;
}

// One pair of same-colour pixels (half-row positions m, m + 1; m even) of region row rw: loads
// with 2-wide shared accesses, both updates, 2-wide stores.  b = column parity of the colour in
// this row: the left neighbour of position m is other-colour position m - 1 + b, the right one
// m + b.  Returns the largest |x_new - x_old| over the pair's interior pixels (imask bit 0 / 1).
// The offsets name the pair's own half-row position (own), the other colour's half-row of the
// same row at the same position (oth), and the other colour's half-rows of the rows above (ou)
// and below (od); planes are PL elements apart.
template <class T, int PL>
__device__ __forceinline__ T sor_pair_at(T* buf, int own, int oth, int ou, int od, int b, T omega, T step, int imask)
{
    // left / right neighbours of the two pixels from one 2-wide and one scalar access
    T l0[5], l1[5], r0[5], r1[5];
    const int pls[5] = {9, 11, 12, 13, 14};
#pragma unroll
    for (int z = 0; z < 5; z++) {
        const T* pb = buf + pls[z] * PL;
        const typename Vec2<T>::t v = ld2<T>(pb + oth);
        if (b) {
            const T e = pb[oth + 2];
            l0[z] = v.x; l1[z] = v.y; r0[z] = v.y; r1[z] = e;
        } else {
            const T e = pb[oth - 1];
            l0[z] = e; l1[z] = v.x; r0[z] = v.x; r1[z] = v.y;
        }
    }
    T c0[9], c1[9];
#pragma unroll
    for (int z = 0; z < 9; z++) {
        const typename Vec2<T>::t v = ld2<T>(buf + z * PL + own);
        c0[z] = v.x; c1[z] = v.y;
    }
    const typename Vec2<T>::t aR = ld2<T>(buf + 9 * PL + own), aD = ld2<T>(buf + 10 * PL + own);
    const typename Vec2<T>::t sO = ld2<T>(buf + 11 * PL + own);
    const typename Vec2<T>::t aU = ld2<T>(buf + 10 * PL + ou), sU = ld2<T>(buf + 11 * PL + ou);
    T xu0[3], xu1[3], xd0[3], xd1[3], xp0[3], xp1[3], n0[3], n1[3];
#pragma unroll
    for (int v = 0; v < 3; v++) {
        const T* xv = buf + (12 + v) * PL;
        const typename Vec2<T>::t u = ld2<T>(xv + ou), d = ld2<T>(xv + od), q = ld2<T>(xv + own);
        xu0[v] = u.x; xu1[v] = u.y; xd0[v] = d.x; xd1[v] = d.y; xp0[v] = q.x; xp1[v] = q.y;
    }
    sor_point<T>(c0, l0[0], aU.x, aR.x, aD.x, l0[1], sU.x, sO.x, l0 + 2, xu0, r0 + 2, xd0, xp0, omega, step, n0);
    sor_point<T>(c1, l1[0], aU.y, aR.y, aD.y, l1[1], sU.y, sO.y, l1 + 2, xu1, r1 + 2, xd1, xp1, omega, step, n1);
#pragma unroll
    for (int v = 0; v < 3; v++) st2<T>(buf + (12 + v) * PL + own, n0[v], n1[v]);
    T md = 0;
    if (imask & 1)
        for (int v = 0; v < 3; v++) md = maxT(md, absT(n0[v] - xp0[v]));
    if (imask & 2)
        for (int v = 0; v < 3; v++) md = maxT(md, absT(n1[v] - xp1[v]));
    return md;
}

template <class T, int PL, int HRW>
__device__ __forceinline__ T sor_pair(T* buf, int rw, int color, int m, int b, T omega, T step, int imask)
{
    const int own = (rw * 2 + color) * HRW + m;
    const int oth = (rw * 2 + (color ^ 1)) * HRW + m;
    return sor_pair_at<T, PL>(buf, own, oth, oth - 2 * HRW, oth + 2 * HRW, b, omega, step, imask);
}

// Region of a tile: global columns [ws, ws + RW), rows [y0, y0 + RH); ws a multiple of 8 so
// each checkerboard half-row segment starts 16-byte aligned.  Shared layout per plane:
// [RH rows][2 colours][HRW], colour = parity of (global row + column).
template <class T, int K>
__device__ __forceinline__ int sor_ws(int tx) { return (tx * kSorTW - 2 * K) & ~7; }

template <class T, class S, int K, int NBUF>
__device__ __forceinline__ void sor_load(const LevelItem<T, S>& it, const Tile& t, const SorLaunch& L, T* buf)
{
    typedef SorGeom<T, K, NBUF> G;
    constexpr int CH = 16 / sizeof(T), NCH = G::HRW / CH;
    if (it.ctl->level_done) return;  // the pair finished this level: its tiles are skipped unread
    const int W = it.W, H = it.H, hw = it.hwp;
    const int m0 = sor_ws<T, K>(t.tx) / 2;
    const int y0 = t.ty * kSorTH - 2 * K;
    const T* base[G::NPL];
#pragma unroll
    for (int pl = 0; pl < 12; pl++) base[pl] = it.sys[pl];
#pragma unroll
    for (int v = 0; v < 3; v++) base[12 + v] = it.x[L.xin][v];
    const int npl = L.xin_zero ? 12 : G::NPL;  // a zero increment is not read
    // one 16-byte chunk position per pass; all planes of that position in a row
    for (int q = threadIdx.x; q < G::RH * 2 * NCH; q += G::NT) {
        const int ch = q % NCH, c = (q / NCH) & 1, rr = q / (2 * NCH);
        const int gi = y0 + rr, m = m0 + ch * CH;
        // pixels of colour c in row gi: columns (c ^ (gi & 1)) + 2m', m' < count
        const int cnt = (W + 1 - (c ^ (gi & 1))) >> 1;
        int nb = 0;
        size_t off = 0;
        if (gi >= 0 && gi < H && m >= 0 && m < cnt) {
            nb = min(CH, cnt - m) * (int)sizeof(T);
            off = (size_t)gi * 2 * hw + c * hw + m;
        }
        T* dst = buf + ((size_t)rr * 2 + c) * G::HRW + ch * CH;
#pragma unroll
        for (int pl = 0; pl < G::NPL; pl++) {
            const bool rd = nb > 0 && pl < npl;
            cp_async16(dst + (size_t)pl * G::RH * G::RW, rd ? base[pl] + off : base[0], rd ? nb : 0);
        }
    }
}

template <class T, class S, int K, int NBUF, int ILP, int MINB>
__global__ void __launch_bounds__(512, MINB)
k_sor(const LevelItem<T, S>* items, const Tile* tiles, int ntiles, SolveConst<T> k, SorLaunch L)
{
    typedef SorGeom<T, K, NBUF> G;
    constexpr int RW = G::RW, RH = G::RH, PL = RH * RW, HRW = G::HRW;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* bufs = reinterpret_cast<T*>(smem_raw);
    T* red = bufs + NBUF * G::buf_elems;  // [64] reduction scratch
    int cur = 0;
    int tid = blockIdx.x;
    if (tid < ntiles) sor_load<T, S, K, NBUF>(items[tiles[tid].item], tiles[tid], L, bufs);
    cp_async_commit();
    for (; tid < ntiles; tid += gridDim.x) {
        const Tile t = tiles[tid];
        const LevelItem<T, S>& it = items[t.item];
        T* buf = bufs + cur * G::buf_elems;
        const int nxt = tid + gridDim.x;
        if (NBUF == 2) {
            if (nxt < ntiles) sor_load<T, S, K, NBUF>(items[tiles[nxt].item], tiles[nxt], L, bufs + (cur ^ 1) * G::buf_elems);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        PairCtl* ctl = it.ctl;
        const bool done = ctl->level_done != 0;
        int nit = L.nit;
        bool stopped = ctl->sor_stop != 0;
        if (!stopped && L.prev_check) {
            const float md = __uint_as_float(ctl->maxdiff[L.prev_check_idx]);
            if ((double)md < k.sor_tol || (T)md >= k.step) {
                stopped = true;
                if (t.idx == 0 && threadIdx.x == 0) { ctl->sor_stop = 1; ctl->sor_stop_iter = L.it0; }
            }
        }
        if (stopped) nit = 0;
        const int W = it.W, H = it.H;
        const int ws = sor_ws<T, K>(t.tx);
        const int y0 = t.ty * kSorTH - 2 * K;
        const int ix0 = t.tx * kSorTW, iy0 = t.ty * kSorTH;  // interior origin
        T md = 0;
        if (!done) {
            for (int hs = 0; hs < 2 * nit; hs++) {
                const int color = hs & 1;
                const bool chk = L.check && hs >= 2 * nit - 2;
                // half-sweep hs only has to be right within h = 2 nit - 1 - hs of the interior: later
                // half-sweeps read it there and nowhere else, so the window shrinks to the interior
                // and never touches the region's outermost ring (no index clamping needed)
                const int h = 2 * nit - 1 - hs;
                const int r0 = max(iy0 - h, 0), r1 = min(iy0 + kSorTH + h, H);
                const int cl = max(ix0 - h, 0), chh = min(ix0 + kSorTW + h, W);
                if constexpr (ILP == 2) {
                    // pair lanes: a half-warp per row, each lane two adjacent same-colour pixels; the
                    // two rows of a warp have one parity (no divergence on b).  A pixel of a pair that
                    // falls outside the window is updated too, which is harmless: the window already
                    // tolerates stale values outside it, errors travel one pixel per half-sweep, and
                    // every access stays inside the shared buffer (window rows are >= 1 row inside
                    // the region; positions m - 1 and m + 2 fall in the neighbouring half-rows).
                    const int mlo = (cl - ws) >> 1, mhi = (chh - ws + 1) >> 1;
                    const int plo = mlo & ~1;
                    const int np = min((mhi - plo + 1) >> 1, (HRW - plo) >> 1);
                    const int l16 = threadIdx.x & 15, hw = threadIdx.x >> 4, wq = hw >> 1;
                    const int kofs = ((wq >> 1) << 2) + (wq & 1) + 2 * (hw & 1);
                    if (l16 < np)
                        for (int kk = kofs; kk < r1 - r0; kk += G::NT / 16) {
                            const int gi = r0 + kk;
                            const int b = color ^ (gi & 1);
                            const int m = plo + 2 * l16;
                            int imask = 0;
                            if (chk && gi >= iy0 && gi < iy0 + kSorTH) {
                                const int gj = ws + 2 * m + b;
                                imask = (gj >= ix0 && gj < ix0 + kSorTW ? 1 : 0) | (gj + 2 >= ix0 && gj + 2 < ix0 + kSorTW ? 2 : 0);
                            }
                            const T d = sor_pair<T, PL, HRW>(buf, gi - y0, color, m, b, k.omega, k.step, imask);
                            md = maxT(md, d);
                        }
                    __syncthreads();
                    continue;
                }
                const int NM = (chh - cl + 2) >> 1;                 // colour pixels per row (upper bound)
                const int nq = (r1 - r0) * NM;
                const unsigned magic = ((1u << 20) + NM - 1) / NM;  // q / NM = (q * magic) >> 20, exact here
                for (int q = threadIdx.x; q < nq; q += G::NT) {
                    const int ro = (int)__umulhi((unsigned)q << 12, magic);
                    const int mo = q - ro * NM;
                    const int gi = r0 + ro;
                    const int b = color ^ (gi & 1);                 // column parity of this colour in row gi
                    const int m = ((cl - ws - b + 1) >> 1) + mo;
                    if (m >= ((chh - ws - b + 1) >> 1)) continue;   // past this row's last pixel
                    const int rw = gi - y0;
                    const int own = (rw * 2 + color) * HRW + m;
                    const int oth = (rw * 2 + (color ^ 1)) * HRW + m;
                    const int ol = oth - 1 + b, orr = oth + b, ou = oth - 2 * HRW, od = oth + 2 * HRW;
                    T c[9], xl[3], xu[3], xr[3], xd[3], xp[3], nv[3];
#pragma unroll
                    for (int z = 0; z < 9; z++) c[z] = buf[z * PL + own];
#pragma unroll
                    for (int v = 0; v < 3; v++) {
                        const T* xv = buf + (12 + v) * PL;
                        xl[v] = xv[ol]; xr[v] = xv[orr]; xu[v] = xv[ou]; xd[v] = xv[od]; xp[v] = xv[own];
                    }
                    sor_point<T>(c, buf[9 * PL + ol], buf[10 * PL + ou], buf[9 * PL + own], buf[10 * PL + own],
                                 buf[11 * PL + ol], buf[11 * PL + ou], buf[11 * PL + own], xl, xu, xr, xd, xp,
                                 k.omega, k.step, nv);
#pragma unroll
                    for (int v = 0; v < 3; v++) buf[(12 + v) * PL + own] = nv[v];
                    if (chk) {
                        const int gj = ws + 2 * m + b;
                        if (gi >= iy0 && gi < iy0 + kSorTH && gj >= ix0 && gj < ix0 + kSorTW)
                            for (int v = 0; v < 3; v++) md = maxT(md, absT(nv[v] - xp[v]));
                    }
                }
                __syncthreads();
            }
            // interior out: x to the other buffer, or the fold u += x with the statistic partial
            T part = 0;
            T* const o0 = L.final_fold ? it.u[0] : it.x[L.xin ^ 1][0];
            T* const o1 = L.final_fold ? it.u[1] : it.x[L.xin ^ 1][1];
            T* const o2 = L.final_fold ? it.u[2] : it.x[L.xin ^ 1][2];
            const T* const dep = it.pyr[6];
            const int pitch = it.pitch, hwp = it.hwp;
            const T fl = it.f_level;
            for (int q = threadIdx.x; q < kSorTW * kSorTH; q += G::NT) {
                const int gi = iy0 + q / kSorTW, gj = ix0 + q % kSorTW;
                if (gi >= H || gj >= W) continue;
                const int cl = (gi + gj) & 1;
                const int o = ((gi - y0) * 2 + cl) * HRW + ((gj - ws) >> 1);
                const T a = buf[12 * PL + o], bq = buf[13 * PL + o], cz = buf[14 * PL + o];
                if (L.final_fold) {
                    const size_t lp = (size_t)gi * pitch + gj;
                    o0[lp] = addR(o0[lp], a); o1[lp] = addR(o1[lp], bq); o2[lp] = addR(o2[lp], cz);
                    part = addR(part, stat_px<T>(a, bq, cz, fl, dep[(size_t)gi * W + gj]));
                } else {
                    const int lc = cs_idx(gi, gj, hwp);
                    o0[lc] = a; o1[lc] = bq; o2[lc] = cz;
                }
            }
            if (L.check && nit > 0) {
                float mm = (float)md;
                for (int off = 16; off > 0; off >>= 1) mm = fmaxf(mm, __shfl_xor_sync(0xffffffffu, mm, off));
                if ((threadIdx.x & 31) == 0 && mm > 0) atomicMax(&ctl->maxdiff[L.check_idx], __float_as_uint(mm));
            }
            if (L.final_fold) {
                // deterministic per-tile sum: warp trees, then warps in order
                for (int off = 16; off > 0; off >>= 1) part += __shfl_down_sync(0xffffffffu, part, off);
                if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
                __syncthreads();
                if (threadIdx.x == 0) {
                    T tot = 0;
                    for (int w = 0; w < G::NT / 32; w++) tot += red[w];
                    it.stat_part[t.idx] = tot;
                }
            }
        }
        __syncthreads();  // buffer `cur` is free for the load after next
        if (NBUF == 1) {
            if (nxt < ntiles) sor_load<T, S, K, NBUF>(items[tiles[nxt].item], tiles[nxt], L, bufs);
            cp_async_commit();
        }
        cur ^= (NBUF - 1);
    }
    cp_async_wait<0>();
}

// ------------------------------------------------------------------------------------------
// Red-black SOR over column strips, the rows streamed through a shared-memory ring (wavefront
// temporal blocking).
//
// A work unit is one item's strip of 64 interior columns [x0, x0 + 64) over a band of rows
// [ya, yb) (ya a multiple of 32; yb a multiple of 32 or H).  Shared memory holds the strip plus
// 16 columns each side (the 2K-pixel halo of K <= 5 iterations, widened to whole 16-byte chunks)
// for a ring of 32 rows, all 15 planes, in the checkerboard layout.  The 2 nit half-sweeps of
// the launch run as a pipeline of stages: at step t, stage s (colour s & 1) updates row t - 2s.
// The lag of two rows per stage makes the in-place update exact: when stage s writes row r,
// stage s - 1 has finished every row <= r + 1 in earlier steps and stage s + 1 has not yet read
// any row >= r - 1, so each update sees exactly the values of a whole-image red-black sweep.  As
// in the tile kernel, stage s only has to be right within h = 2 nit - 1 - s pixels of the unit's
// interior, so its window is the interior widened by h (clipped to the image).
//
// Every step: each thread issues one cp.async of the row 2 + P steps ahead (P = 8 rows in
// flight; only the threads that own a load position issue them); threads 0..479 run the stages
// (48 lanes a stage, one pixel a lane); threads 480..511 write the row that left the pipeline (x
// to the other ping-pong buffer, or the fold u += x with the statistic); one barrier.  Units come from a ticket counter, so a pair that has finished its
// level costs nothing and the SMs stay balanced.  Results equal the tile kernel's bit for bit:
// the same pixel update, and the same statistic partial per 32 x 32 tile summed in the same order
// (rows r and r + 16 paired, a warp tree over the 32 columns, then the 16 row pairs in order).
constexpr int kStripW = 64, kStripRW = 96, kStripHRW = 48, kStripNR = 32, kStripNU = 16, kStripP = 8;
constexpr int kStripNT = 512, kStripLanes = 48, kStripOutT = 480, kStripMaxNit = 5;
constexpr int kStripPL = kStripNR * kStripRW;  // ring plane stride (elements)
constexpr int kStripUPL = kStripNU * kStripW;  // fold ring plane stride: u (3 planes) and depth 1
template <class T> constexpr size_t strip_smem_bytes()
{
    return sizeof(T) * ((size_t)15 * kStripPL + 4 * kStripUPL + 2 * 16 * 32);
}
static_assert(4 * kStripMaxNit + 1 + kStripP < kStripNR, "ring too short for the pipeline depth");
static_assert(kStripNU > kStripP + 1, "fold ring too short for the prefetch depth");
static_assert(2 * kStripMaxNit * kStripLanes <= kStripOutT && kStripOutT + 32 == kStripNT,
              "stage lanes and the output warp exceed the block");
static_assert(kStripLanes >= (kStripW + 2 * (2 * kStripMaxNit - 1)) / 2 + 1, "too few lanes for a stage row");
static_assert(15 * 2 * (kStripHRW / 4) + 3 * (kStripW / 4) + kStripW <= kStripNT, "one load per thread per row");

struct StripUnit {
    int item;
    int x0;      // first interior column (a multiple of 64)
    int ya, yb;  // interior rows
};

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, int src_bytes)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes) : "memory");
}

template <class T, class S>
__global__ void __launch_bounds__(kStripNT, 1)
k_sor_strip(const LevelItem<T, S>* items, const StripUnit* units, int n_units, int* ticket, SolveConst<T> k,
            SorLaunch L)
{
    static_assert(sizeof(T) == 4, "the strip SOR holds FP32 planes (16-byte chunks of 4 values)");
    constexpr int RW = kStripRW, HRW = kStripHRW, PL = kStripPL, UPL = kStripUPL, NRM = kStripNR - 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* const ring = reinterpret_cast<T*>(smem_raw);
    T* const uring = ring + 15 * PL;
    T* const sacc = uring + 4 * UPL;  // [2 tile columns][16 rows][32 lanes]
    __shared__ int s_unit, s_nit;
    const int tid = threadIdx.x, lane = tid & 31;
    const int tbase = L.seq * (n_units + (int)gridDim.x);  // the tickets of this launch
    const int s = tid / kStripLanes, j = tid % kStripLanes;  // stage and lane (threads < 480)
    const bool outw = tid >= kStripOutT;
    for (;;) {
        if (tid == 0) {
            const int u = atomicAdd(ticket, 1) - tbase;
            int nit = -1;  // -1: nothing to do for this unit
            if (u < n_units) {
                const StripUnit su = units[u];
                PairCtl* ctl = items[su.item].ctl;
                if (!ctl->level_done) {
                    nit = L.nit;
                    bool stopped = ctl->sor_stop != 0;
                    if (!stopped && L.prev_check) {
                        const float md = __uint_as_float(ctl->maxdiff[L.prev_check_idx]);
                        if ((double)md < k.sor_tol || (T)md >= k.step) {
                            stopped = true;
                            if (su.x0 == 0 && su.ya == 0) { ctl->sor_stop = 1; ctl->sor_stop_iter = L.it0; }
                        }
                    }
                    if (stopped) nit = 0;
                }
            }
            s_unit = u;
            s_nit = nit;
        }
        __syncthreads();
        const int u = s_unit, nit = s_nit;
        __syncthreads();  // s_unit and s_nit are rewritten only after every thread has read them
        if (u >= n_units) break;
        if (nit < 0) continue;

        const StripUnit su = units[u];
        const LevelItem<T, S>& it = items[su.item];
        const int W = it.W, H = it.H, hw = it.hwp, pitch = it.pitch;
        const int x0 = su.x0, ya = su.ya, yb = su.yb;
        const int wsh = x0 / 2 - 8;  // the region's first half-row position (column x0 - 16)
        const int S2 = 2 * nit;
        const int t0 = nit > 0 ? max(0, ya - S2 + 1) : ya - 1;
        const int t1 = yb + 4 * nit - 1;           // the last step outputs row yb - 1
        const int rhi_load = min(yb + S2 - 1, H);  // rows read by the stages: [t0 - 1, rhi_load]
        const bool fold = L.final_fold != 0;

        // ---- this thread's load of every row, a fixed position: kind 1 a system / increment
        // chunk, 2 a u chunk (fold), 3 a depth element (fold), 0 none.  Rows are loaded in order
        // t0 - 1, t0, t0 + 1, ...; the row R of the next load, its source and its ring address
        // advance by one row per load.
        int lkind = 0, nb0 = 0, nb1 = 0;  // valid bytes of the chunk in even / odd rows
        const T* lbase = nullptr;         // a valid address for zero-filled copies
        const T* lsrc = nullptr;          // source of row lR (meaningful only where it is in range)
        size_t lstride = 0;
        unsigned ldst = 0, lwrap = 0, lring = 0;  // shared address of row lR's slot; ring span
        int lR = t0 - 1, lU = 0;
        if (tid < 360) {
            const int pl = tid / 24, rem = tid % 24, ch = rem % 12, lc = rem / 12;
            const int lm = wsh + 4 * ch;
            lbase = pl < 12 ? it.sys[pl] : it.x[L.xin][pl - 12];
            lkind = 1;
            if (!(pl >= 12 && L.xin_zero) && lm >= 0) {
                const int cnt0 = (W + 1 - lc) >> 1, cnt1 = (W + 1 - (lc ^ 1)) >> 1;
                nb0 = lm < cnt0 ? min(4, cnt0 - lm) * (int)sizeof(T) : 0;
                nb1 = lm < cnt1 ? min(4, cnt1 - lm) * (int)sizeof(T) : 0;
            }
            lstride = (size_t)2 * hw;
            lsrc = lbase + lc * hw + lm + (ptrdiff_t)lR * (ptrdiff_t)lstride;
            const unsigned a0 = (unsigned)__cvta_generic_to_shared(ring + pl * PL + lc * HRW + 4 * ch);
            lring = kStripNR * RW * sizeof(T);
            lwrap = a0 + lring;
            ldst = a0 + (unsigned)((lR & NRM) * RW * sizeof(T));
        } else if (fold && tid < 472) {
            const bool dep = tid >= 408;
            const int col = dep ? x0 + (tid - 408) : x0 + 4 * ((tid - 360) % 16);
            const int pl = dep ? 0 : (tid - 360) / 16;
            nb0 = dep ? (col < W ? (int)sizeof(T) : 0) : max(0, min(4, W - col)) * (int)sizeof(T);
            lbase = dep ? it.pyr[6] : it.u[pl];
            lstride = dep ? (size_t)W : (size_t)pitch;
            lU = lR - 4 * nit;
            lsrc = lbase + col + (ptrdiff_t)lU * (ptrdiff_t)lstride;
            const unsigned a0 = (unsigned)__cvta_generic_to_shared(uring + (dep ? 3 : pl) * UPL + (col - x0));
            lring = kStripNU * kStripW * sizeof(T);
            lwrap = a0 + lring;
            ldst = a0 + (unsigned)((lU & (kStripNU - 1)) * kStripW * sizeof(T));
            lkind = dep ? 3 : 2;
        }
        auto load_next = [&]() {
            if (lkind == 1) {
                if (lR <= rhi_load) {
                    const int nb = (lR >= 0 && lR < H) ? ((lR & 1) ? nb1 : nb0) : 0;
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(ldst), "l"(nb ? lsrc : lbase),
                                 "r"(nb) : "memory");
                }
            } else if (lkind) {
                // the fold row written when row lR enters the ring
                if (lU >= ya && lU < yb) {
                    const T* sp = nb0 ? lsrc : lbase;
                    if (lkind == 2)
                        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(ldst), "l"(sp), "r"(nb0) : "memory");
                    else
                        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(ldst), "l"(sp), "r"(nb0) : "memory");
                }
                lU++;
            }
            lR++;
            lsrc += lstride;
            ldst += (unsigned)(lkind == 1 ? RW * sizeof(T) : kStripW * sizeof(T));
            if (ldst >= lwrap) ldst -= lring;
        };

        // ---- this thread's stage: window, and per b (the column parity of this colour in a row)
        // its pixel's half-row position, whether it is in the window, whether it is interior
        const bool stage = tid < 2 * kStripMaxNit * kStripLanes && s < S2;
        const int colour = s & 1, h = S2 - 1 - s;
        const int cl = max(x0 - h, 0), chh = min(x0 + kStripW + h, W);
        const int rlo = max(ya - h, 0), rhi = min(yb + h, H);
        const bool chk = L.check && s >= S2 - 2;
        const int m0 = ((cl + 1) >> 1) + j, m1 = (cl >> 1) + j;
        const bool pv0 = 2 * m0 < chh, pv1 = 2 * m1 + 1 < chh;
        const int pp0 = m0 - wsh, pp1 = m1 - wsh;
        const bool in0 = 2 * m0 >= x0 && 2 * m0 < x0 + kStripW, in1 = 2 * m1 + 1 >= x0 && 2 * m1 + 1 < x0 + kStripW;
        // output pointers in registers: the asm memory clobbers of cp.async would otherwise make
        // every step reload them from the item descriptor
        T* const xo0 = fold ? it.u[0] : it.x[L.xin ^ 1][0];
        T* const xo1 = fold ? it.u[1] : it.x[L.xin ^ 1][1];
        T* const xo2 = fold ? it.u[2] : it.x[L.xin ^ 1][2];
        T* const statp = it.stat_part;
        const T fl = it.f_level;
        const int sx = (W + kSorTW - 1) / kSorTW;
        T md = 0, tot0 = 0, tot1 = 0;

        if (lkind) {
            load_next();  // rows t0 - 1, t0, t0 + 1: the first group
            load_next();
            load_next();
            cp_async_commit();
#pragma unroll 1
            for (int i = 2; i <= kStripP + 1; i++) {
                load_next();  // row t0 + i
                cp_async_commit();
            }
            cp_async_wait<kStripP>();
        }
        __syncthreads();
#pragma unroll 1
        for (int t = t0; t < t1; t++) {
            if (lkind) {
                load_next();  // row t + 2 + P
                cp_async_commit();
            }
            if (stage) {
                const int r = t - 2 * s;
                const int b = colour ^ (r & 1);  // column parity of this colour in row r
                if (r >= rlo && r < rhi && (b ? pv1 : pv0)) {
                    const int p = b ? pp1 : pp0;
                    const int oc = (colour ^ 1) * HRW + p;
                    const int rs = (r & NRM) * RW;
                    const int own = rs + colour * HRW + p, oth = rs + oc;
                    const int ol = oth - 1 + b, orr = oth + b;
                    const int ou = ((r - 1) & NRM) * RW + oc, od = ((r + 1) & NRM) * RW + oc;
                    T c[9], xl[3], xu[3], xr[3], xd[3], xp[3], nv[3];
#pragma unroll
                    for (int z = 0; z < 9; z++) c[z] = ring[z * PL + own];
#pragma unroll
                    for (int v = 0; v < 3; v++) {
                        const T* xv = ring + (12 + v) * PL;
                        xl[v] = xv[ol]; xr[v] = xv[orr]; xu[v] = xv[ou]; xd[v] = xv[od]; xp[v] = xv[own];
                    }
                    sor_point<T>(c, ring[9 * PL + ol], ring[10 * PL + ou], ring[9 * PL + own], ring[10 * PL + own],
                                 ring[11 * PL + ol], ring[11 * PL + ou], ring[11 * PL + own], xl, xu, xr, xd, xp,
                                 k.omega, k.step, nv);
#pragma unroll
                    for (int v = 0; v < 3; v++) ring[(12 + v) * PL + own] = nv[v];
                    if (chk && r >= ya && r < yb && (b ? in1 : in0))
                        for (int v = 0; v < 3; v++) md = maxT(md, absT(nv[v] - xp[v]));
                }
            } else if (outw) {
                const int ro = t - 4 * nit + 1;  // the row the last stage finished in the previous step
                if (ro >= ya && ro < yb) {
                    const int rs = (ro & NRM) * RW;
                    T val[2];
#pragma unroll
                    for (int kk = 0; kk < 2; kk++) {
                        const int gj = x0 + lane + 32 * kk;
                        val[kk] = 0;
                        if (gj < W) {
                            const int o = rs + ((ro + gj) & 1) * HRW + ((gj >> 1) - wsh);
                            const T a = ring[12 * PL + o], bq = ring[13 * PL + o], cz = ring[14 * PL + o];
                            if (fold) {
                                const int ui = (ro & (kStripNU - 1)) * kStripW + lane + 32 * kk;
                                const size_t lp = (size_t)ro * pitch + gj;
                                xo0[lp] = addR(uring[ui], a);
                                xo1[lp] = addR(uring[UPL + ui], bq);
                                xo2[lp] = addR(uring[2 * UPL + ui], cz);
                                val[kk] = stat_px<T>(a, bq, cz, fl, uring[3 * UPL + ui]);
                            } else {
                                const int lcx = cs_idx(ro, gj, hw);
                                xo0[lcx] = a; xo1[lcx] = bq; xo2[lcx] = cz;
                            }
                        }
                    }
                    if (fold) {
                        // statistic partials of the (up to) two 32 x 32 tiles this row crosses
                        const int rl = ro & 31;
                        if (rl < 16) {
                            sacc[rl * 32 + lane] = val[0];
                            sacc[(16 + rl) * 32 + lane] = val[1];
                        } else {
                            T p0 = addR(sacc[(rl - 16) * 32 + lane], val[0]);
                            T p1 = addR(sacc[rl * 32 + lane], val[1]);
                            for (int off = 16; off > 0; off >>= 1) {
                                p0 = addR(p0, __shfl_down_sync(0xffffffffu, p0, off));
                                p1 = addR(p1, __shfl_down_sync(0xffffffffu, p1, off));
                            }
                            tot0 = addR(tot0, p0);
                            tot1 = addR(tot1, p1);
                        }
                        if (rl == 31 || ro == yb - 1) {
                            const int nrows = rl + 1;  // rows r2 whose row r2 + 16 does not exist
                            for (int r2 = max(0, nrows - 16); r2 < min(16, nrows); r2++) {
                                T p0 = sacc[r2 * 32 + lane], p1 = sacc[(16 + r2) * 32 + lane];
                                for (int off = 16; off > 0; off >>= 1) {
                                    p0 = addR(p0, __shfl_down_sync(0xffffffffu, p0, off));
                                    p1 = addR(p1, __shfl_down_sync(0xffffffffu, p1, off));
                                }
                                tot0 = addR(tot0, p0);
                                tot1 = addR(tot1, p1);
                            }
                            if (lane == 0) {
                                const int tb = (ro >> 5) * sx + (x0 >> 5);
                                statp[tb] = tot0;
                                if (x0 + 32 < W) statp[tb + 1] = tot1;
                            }
                            tot0 = 0;
                            tot1 = 0;
                        }
                    }
                }
            }
            if (lkind) cp_async_wait<kStripP>();
            __syncthreads();
        }
        cp_async_wait<0>();
        if (L.check && nit > 0) {
            float mm = (float)md;
            for (int off = 16; off > 0; off >>= 1) mm = fmaxf(mm, __shfl_xor_sync(0xffffffffu, mm, off));
            if (lane == 0 && mm > 0) atomicMax(&items[su.item].ctl->maxdiff[L.check_idx], __float_as_uint(mm));
        }
        __syncthreads();  // the ring is refilled by the next unit
    }
}

// ------------------------------------------------------------------------------------------
// Whole-level SOR for levels that fit one CTA's shared memory (the coarsest, e.g. 40 x 30): one
// CTA per pair stages the level's system and increment once and runs every SOR iteration of the
// inner iteration in one launch.  The convergence check (iteration it with it % period ==
// period - 1, .cu:905-921) is a block reduction and the stop decision is taken in the kernel
// with the tile kernels' rule, so the executed schedule and the result equal theirs: the same
// pixel update (sor_point), whole-image red-black half-sweeps, the same statistic partial per
// 32 x 32 tile summed in the same order.  Replaces the tile kernel's six latency-bound launches
// per inner iteration at these levels.
//
// Shared layout: 15 planes of [H + 2 rows][2 colours][hwp + 2 positions] (checkerboard, one
// zero row / position of padding on every side, so neighbours never need a bounds test).
template <class T> __host__ __device__ constexpr size_t level_smem_bytes(int H, int hwp)
{
    return sizeof(T) * ((size_t)15 * (H + 2) * 2 * (hwp + 2) + 64);
}
__host__ __device__ constexpr int level_threads(int H, int hwp)
{
    return (H * hwp + 31) / 32 * 32 > 1024 ? 1024 : ((H * hwp + 31) / 32 * 32 < 64 ? 64 : (H * hwp + 31) / 32 * 32);
}

template <class T, class S>
__global__ void __launch_bounds__(1024)
k_sor_level(const LevelItem<T, S>* items, const int* which, SolveConst<T> k, SorLaunch L)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* const buf = reinterpret_cast<T*>(smem_raw);
    __shared__ int s_stop;
    const LevelItem<T, S>& it = items[which[blockIdx.x]];
    PairCtl* ctl = it.ctl;
    if (ctl->level_done) return;
    const int W = it.W, H = it.H, hw = it.hwp, RP = hw + 2;
    const int PLS = (H + 2) * 2 * RP;
    T* const red = buf + 15 * PLS;
    const int tid = threadIdx.x, NT = blockDim.x;
    // stage: valid pixels from global, zero everywhere else (padding, positions past a row's count);
    // a thread's position is decoded once and its 15 planes' loads are all in flight together
    for (int e = tid; e < PLS; e += NT) {
        const int rr = e / (2 * RP) - 1, c = (e / RP) & 1, p = e % RP - 1;
        const bool valid = rr >= 0 && rr < H && p >= 0 && p < ((W + 1 - (c ^ (rr & 1))) >> 1);
        const size_t g = valid ? (size_t)rr * 2 * hw + c * hw + p : 0;
        T v[15];
#pragma unroll
        for (int z = 0; z < 12; z++) v[z] = valid ? it.sys[z][g] : (T)0;
#pragma unroll
        for (int z = 12; z < 15; z++) v[z] = (valid && !L.xin_zero) ? it.x[L.xin][z - 12][g] : (T)0;
#pragma unroll
        for (int z = 0; z < 15; z++) buf[z * PLS + e] = v[z];
    }
    if (tid == 0) s_stop = 0;
    __syncthreads();
    int executed = k.n_sor;
    // the block is launched with about one thread per position (H x hwp); a thread's positions and
    // their rows are fixed across the half-sweeps
    const int q0 = tid, q1 = tid + NT;
    const int i0 = q0 / hw, m0 = q0 % hw, i1 = q1 / hw, m1 = q1 % hw;
    for (int itn = 0; itn < k.n_sor; itn++) {
        const bool chk = !k.fixed && (itn % k.period == k.period - 1);
        T md = 0;
        for (int color = 0; color < 2; color++) {
            for (int r = 0, q = q0; q < H * hw; r++, q += NT) {
                const int i = r == 0 ? i0 : (r == 1 ? i1 : q / hw), m = r == 0 ? m0 : (r == 1 ? m1 : q % hw);
                const int b = color ^ (i & 1);
                if (m >= ((W + 1 - b) >> 1)) continue;
                const int own = ((i + 1) * 2 + color) * RP + m + 1;
                const int oth = ((i + 1) * 2 + (color ^ 1)) * RP + m + 1;
                const int ol = oth - 1 + b, orr = oth + b, ou = oth - 2 * RP, od = oth + 2 * RP;
                T c[9], xl[3], xu[3], xr[3], xd[3], xp[3], nv[3];
#pragma unroll
                for (int z = 0; z < 9; z++) c[z] = buf[z * PLS + own];
#pragma unroll
                for (int v = 0; v < 3; v++) {
                    const T* xv = buf + (12 + v) * PLS;
                    xl[v] = xv[ol]; xr[v] = xv[orr]; xu[v] = xv[ou]; xd[v] = xv[od]; xp[v] = xv[own];
                }
                sor_point<T>(c, buf[9 * PLS + ol], buf[10 * PLS + ou], buf[9 * PLS + own], buf[10 * PLS + own],
                             buf[11 * PLS + ol], buf[11 * PLS + ou], buf[11 * PLS + own], xl, xu, xr, xd, xp,
                             k.omega, k.step, nv);
#pragma unroll
                for (int v = 0; v < 3; v++) buf[(12 + v) * PLS + own] = nv[v];
                if (chk)
                    for (int v = 0; v < 3; v++) md = maxT(md, absT(nv[v] - xp[v]));
            }
            __syncthreads();
        }
        if (chk) {
            // the check: max |dx| of this iteration over the level (float bits, as the tile kernels)
            float mm = (float)md;
            for (int off = 16; off > 0; off >>= 1) mm = fmaxf(mm, __shfl_xor_sync(0xffffffffu, mm, off));
            if ((tid & 31) == 0) red[tid >> 5] = (T)mm;
            __syncthreads();
            if (tid == 0) {
                float g = 0;
                for (int w = 0; w < NT / 32; w++) g = fmaxf(g, (float)red[w]);
                const int ci = min(itn / k.period, kMaxChecks - 1);
                if (g > 0) ctl->maxdiff[ci] = __float_as_uint(g);
                if ((double)g < k.sor_tol || (T)g >= k.step) {
                    s_stop = 1;
                    ctl->sor_stop = 1;
                    ctl->sor_stop_iter = itn + 1;
                }
            }
            __syncthreads();
            if (s_stop) { executed = itn + 1; break; }
        }
    }
    (void)executed;
    // out: the fold u += x with the statistic partial per 32 x 32 tile (the tile kernels' order),
    // or x into the ping-pong buffer the next inner iteration reads
    const int sx = (W + kSorTW - 1) / kSorTW, sy = (H + kSorTH - 1) / kSorTH;
    if (L.final_fold) {
        const int pitch = it.pitch;
        const T fl = it.f_level;
        // the partials are summed exactly as a 512-thread tile CTA sums them: "virtual thread" vt
        // (0..511) takes pixels vt and vt + 512 of the tile, a warp tree per virtual warp, then
        // the 16 virtual warps in order; a real warp takes virtual warps w, w + NT / 32, ...
        const int lane = tid & 31;
        for (int ti = 0; ti < sx * sy; ti++) {
            const int ix0 = (ti % sx) * kSorTW, iy0 = (ti / sx) * kSorTH;
            for (int vw = tid >> 5; vw < 16; vw += NT >> 5) {
                T part = 0;
                for (int q = vw * 32 + lane; q < kSorTW * kSorTH; q += 512) {
                    const int gi = iy0 + q / kSorTW, gj = ix0 + q % kSorTW;
                    if (gi >= H || gj >= W) continue;
                    const int o = ((gi + 1) * 2 + ((gi + gj) & 1)) * RP + (gj >> 1) + 1;
                    const T a = buf[12 * PLS + o], bq = buf[13 * PLS + o], cz = buf[14 * PLS + o];
                    const size_t lp = (size_t)gi * pitch + gj;
                    it.u[0][lp] = addR(it.u[0][lp], a); it.u[1][lp] = addR(it.u[1][lp], bq);
                    it.u[2][lp] = addR(it.u[2][lp], cz);
                    part = addR(part, stat_px<T>(a, bq, cz, fl, it.pyr[6][(size_t)gi * W + gj]));
                }
                for (int off = 16; off > 0; off >>= 1) part += __shfl_down_sync(0xffffffffu, part, off);
                if (lane == 0) red[vw] = part;
            }
            __syncthreads();
            if (tid == 0) {
                T tot = 0;
                for (int w = 0; w < 16; w++) tot += red[w];
                it.stat_part[ti] = tot;
            }
            __syncthreads();
        }
        if (L.control && tid < 32) control_item(it, k, L.outer, L.n_checks, tid);
    } else {
        for (int q = tid; q < H * W; q += NT) {
            const int gi = q / W, gj = q % W;
            const int o = ((gi + 1) * 2 + ((gi + gj) & 1)) * RP + (gj >> 1) + 1;
            const int lc = cs_idx(gi, gj, hw);
            for (int v = 0; v < 3; v++) it.x[L.xout][v][lc] = buf[(12 + v) * PLS + o];
        }
    }
}


// ------------------------------------------------------------------------------------------
// Whole-level SOR with the system held in registers (FP32; levels of at most kLevelRegMax
// positions of the checkerboard layout, e.g. 40 x 30).  The same launch and results as
// k_sor_level, but a thread owns one position (row i, half-row index m): one pixel of each
// colour, whose 12 coefficients and the 4 neighbour coefficients its update needs (the left
// pixel's horizontal weight and s, the upper pixel's vertical weight and s) stay in registers for
// the whole launch, as do its own unknowns.  Shared memory holds only the three increment planes,
// so a pixel update reads its 4 neighbours' unknowns (12 values) and writes 3, instead of reading
// 31 values.
constexpr int kLevelRegMax = 768;  // positions (= threads) of a level on this kernel
// Row pitch (positions) of a half-row in the shared planes of the register whole-level kernels: at
// least hwp + 2 (a zero position each side) and with 2 RP = hwp (mod 32), so that the 32 threads of
// a warp, which span consecutive rows of one colour when hwp < 32, touch 32 consecutive banks (with
// hwp + 2, 20-position rows put 8 threads of a warp on the banks of 8 others).
__host__ __device__ constexpr int level_reg_rp(int hwp)
{
    int rp = hwp + 2;
    while (((2 * rp - hwp) & 31) != 0) rp++;
    return rp;
}
template <class T> __host__ __device__ constexpr size_t level_reg_smem_bytes(int H, int hwp)
{
    return sizeof(T) * ((size_t)3 * (H + 2) * 2 * level_reg_rp(hwp) + 64);
}

template <class T, class S>
__global__ void __launch_bounds__(kLevelRegMax, 1)
k_sor_level_reg(const LevelItem<T, S>* items, const int* which, SolveConst<T> k, SorLaunch L)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* const xb = reinterpret_cast<T*>(smem_raw);
    __shared__ int s_stop;
    __shared__ T red[32];
    const LevelItem<T, S>& it = items[which[blockIdx.x]];
    PairCtl* ctl = it.ctl;
    if (ctl->level_done) return;
    const int W = it.W, H = it.H, hw = it.hwp, RP = level_reg_rp(hw);
    const int PLS = (H + 2) * 2 * RP;
    const int tid = threadIdx.x, NT = blockDim.x;
    // the unknowns: valid pixels from global, zero everywhere else (padding, positions past a
    // row's count)
    for (int e = tid; e < 3 * PLS; e += NT) {
        const int v = e / PLS, f = e % PLS;
        const int rr = f / (2 * RP) - 1, c = (f / RP) & 1, p = f % RP - 1;
        const bool valid = !L.xin_zero && rr >= 0 && rr < H && p >= 0 && p < ((W + 1 - (c ^ (rr & 1))) >> 1);
        xb[e] = valid ? it.x[L.xin][v][(size_t)rr * 2 * hw + c * hw + p] : (T)0;
    }
    // this thread's position and, per colour, its pixel's system in registers
    const int i = tid / hw, m = tid % hw;
    const bool inpos = tid < H * hw;
    T cf[2][9], aL[2], aU[2], aR[2], aD[2], sL[2], sU[2], sw[2], xp[2][3];
    bool valid[2];
    int own[2], oth[2];
#pragma unroll
    for (int color = 0; color < 2; color++) {
        const int b = color ^ (i & 1);
        valid[color] = inpos && m < ((W + 1 - b) >> 1);
        own[color] = ((i + 1) * 2 + color) * RP + m + 1;
        oth[color] = ((i + 1) * 2 + (color ^ 1)) * RP + m + 1;
        const size_t g = (size_t)i * 2 * hw + color * hw + m;
        // the left neighbour is the other colour's position m - 1 + b of the row, the upper one its
        // position m of the row above; outside the level they are zero, as in the staged planes
        const int ml = m - 1 + b;
        const bool lok = valid[color] && ml >= 0 && ml < ((W + 1 - (b ^ 1)) >> 1);
        const bool uok = valid[color] && i >= 1;
        const size_t gl = (size_t)i * 2 * hw + (color ^ 1) * hw + ml;
        const size_t gu = (size_t)(i - 1) * 2 * hw + (color ^ 1) * hw + m;
#pragma unroll
        for (int z = 0; z < 9; z++) cf[color][z] = valid[color] ? it.sys[z][g] : (T)0;
        aR[color] = valid[color] ? it.sys[9][g] : (T)0;
        aD[color] = valid[color] ? it.sys[10][g] : (T)0;
        sw[color] = valid[color] ? it.sys[11][g] : (T)0;
        aL[color] = lok ? it.sys[9][gl] : (T)0;
        sL[color] = lok ? it.sys[11][gl] : (T)0;
        aU[color] = uok ? it.sys[10][gu] : (T)0;
        sU[color] = uok ? it.sys[11][gu] : (T)0;
    }
    if (tid == 0) s_stop = 0;
    __syncthreads();
    // own unknowns of the valid pixels (a thread past the level's positions reads nothing)
#pragma unroll
    for (int color = 0; color < 2; color++)
#pragma unroll
        for (int v = 0; v < 3; v++) xp[color][v] = valid[color] ? xb[v * PLS + own[color]] : (T)0;
    for (int itn = 0; itn < k.n_sor; itn++) {
        const bool chk = !k.fixed && (itn % k.period == k.period - 1);
        T md = 0;
#pragma unroll
        for (int color = 0; color < 2; color++) {
            if (valid[color]) {
                const int b = color ^ (i & 1);
                const int ol = oth[color] - 1 + b, orr = oth[color] + b, ou = oth[color] - 2 * RP, od = oth[color] + 2 * RP;
                T xl[3], xu[3], xr[3], xd[3], nv[3];
#pragma unroll
                for (int v = 0; v < 3; v++) {
                    const T* xv = xb + v * PLS;
                    xl[v] = xv[ol]; xr[v] = xv[orr]; xu[v] = xv[ou]; xd[v] = xv[od];
                }
                sor_point<T>(cf[color], aL[color], aU[color], aR[color], aD[color], sL[color], sU[color], sw[color],
                             xl, xu, xr, xd, xp[color], k.omega, k.step, nv);
#pragma unroll
                for (int v = 0; v < 3; v++) {
                    xb[v * PLS + own[color]] = nv[v];
                    if (chk) md = maxT(md, absT(nv[v] - xp[color][v]));
                    xp[color][v] = nv[v];
                }
            }
            __syncthreads();
        }
        if (chk) {
            // the check: max |dx| of this iteration over the level (float bits, as the tile kernels)
            float mm = (float)md;
            for (int off = 16; off > 0; off >>= 1) mm = fmaxf(mm, __shfl_xor_sync(0xffffffffu, mm, off));
            if ((tid & 31) == 0) red[tid >> 5] = (T)mm;
            __syncthreads();
            if (tid == 0) {
                float g = 0;
                for (int w = 0; w < NT / 32; w++) g = fmaxf(g, (float)red[w]);
                const int ci = min(itn / k.period, kMaxChecks - 1);
                if (g > 0) ctl->maxdiff[ci] = __float_as_uint(g);
                if ((double)g < k.sor_tol || (T)g >= k.step) {
                    s_stop = 1;
                    ctl->sor_stop = 1;
                    ctl->sor_stop_iter = itn + 1;
                }
            }
            __syncthreads();
            if (s_stop) break;
        }
    }
    // out: the fold u += x with the statistic partial per 32 x 32 tile (the tile kernels' order),
    // or x into the ping-pong buffer the next inner iteration reads
    const int sx = (W + kSorTW - 1) / kSorTW, sy = (H + kSorTH - 1) / kSorTH;
    if (L.final_fold) {
        const int pitch = it.pitch;
        const T fl = it.f_level;
        // the partials are summed exactly as a 512-thread tile CTA sums them: "virtual thread" vt
        // (0..511) takes pixels vt and vt + 512 of the tile, a warp tree per virtual warp, then
        // the 16 virtual warps in order; a real warp takes virtual warps w, w + NT / 32, ...
        const int lane = tid & 31;
        for (int ti = 0; ti < sx * sy; ti++) {
            const int ix0 = (ti % sx) * kSorTW, iy0 = (ti / sx) * kSorTH;
            for (int vw = tid >> 5; vw < 16; vw += NT >> 5) {
                T part = 0;
                for (int q = vw * 32 + lane; q < kSorTW * kSorTH; q += 512) {
                    const int gi = iy0 + q / kSorTW, gj = ix0 + q % kSorTW;
                    if (gi >= H || gj >= W) continue;
                    const int o = ((gi + 1) * 2 + ((gi + gj) & 1)) * RP + (gj >> 1) + 1;
                    const T a = xb[o], bq = xb[PLS + o], cz = xb[2 * PLS + o];
                    const size_t lp = (size_t)gi * pitch + gj;
                    it.u[0][lp] = addR(it.u[0][lp], a); it.u[1][lp] = addR(it.u[1][lp], bq);
                    it.u[2][lp] = addR(it.u[2][lp], cz);
                    part = addR(part, stat_px<T>(a, bq, cz, fl, it.pyr[6][(size_t)gi * W + gj]));
                }
                for (int off = 16; off > 0; off >>= 1) part += __shfl_down_sync(0xffffffffu, part, off);
                if (lane == 0) red[vw] = part;
            }
            __syncthreads();
            if (tid == 0) {
                T tot = 0;
                for (int w = 0; w < 16; w++) tot += red[w];
                it.stat_part[ti] = tot;
            }
            __syncthreads();
        }
        if (L.control && tid < 32) control_item(it, k, L.outer, L.n_checks, tid);
    } else {
        for (int q = tid; q < H * W; q += NT) {
            const int gi = q / W, gj = q % W;
            const int o = ((gi + 1) * 2 + ((gi + gj) & 1)) * RP + (gj >> 1) + 1;
            const int lc = cs_idx(gi, gj, hw);
            for (int v = 0; v < 3; v++) it.x[L.xout][v][lc] = xb[v * PLS + o];
        }
    }
}

// ------------------------------------------------------------------------------------------
// Whole-level SOR over a thread-block cluster, for levels whose 15 planes need up to 8 SMs' shared
// memory (the 80 x 60 and 160 x 120 levels).  One cluster per pair: CTA r of C holds rows
// [r B, r B + B) (B = ceil(H / C)) with one halo row above and below, runs every SOR iteration of
// the inner iteration, and after each half-sweep takes the neighbour CTAs' freshly updated boundary
// row of that colour from their shared memory (distributed shared memory, one cluster barrier per
// half-sweep).  The convergence check combines the CTAs' maxima through distributed shared memory,
// so every CTA takes the same decision.  At the end x goes to global memory and, for the fold, each
// 32 x 32 tile's u += x and statistic partial is taken by one CTA in the tile kernels' order, so
// results equal the tile kernel's bit for bit, as the one-CTA whole-level kernel's do.
// Shared layout: 15 planes of [B + 2 rows][2 colours][hwp + 2 positions], padding zero.
template <class T> __host__ __device__ constexpr size_t level_cluster_smem_bytes(int B, int hwp)
{
    return sizeof(T) * ((size_t)15 * (B + 2) * 2 * (hwp + 2) + 64);
}

template <class T, class S>
__global__ void __launch_bounds__(1024)
k_sor_level_cluster(const LevelItem<T, S>* items, const int* which, SolveConst<T> k, SorLaunch L)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* const buf = reinterpret_cast<T*>(smem_raw);
    __shared__ int s_stop;
    __shared__ float s_max;
    const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const LevelItem<T, S>& it = items[which[blockIdx.x / C]];
    PairCtl* ctl = it.ctl;
    if (ctl->level_done) return;  // the same for every CTA of the cluster: none reaches a barrier
    const int W = it.W, H = it.H, hw = it.hwp, RP = hw + 2;
    const int B = (H + C - 1) / C, r0 = rank * B, nr = max(0, min(H, r0 + B) - r0);
    const int PLS = (B + 2) * 2 * RP;
    T* const red = buf + 15 * PLS;
    const int tid = threadIdx.x, NT = blockDim.x;
    // stage rows r0 - 1 .. r0 + nr (local rows 0 .. nr + 1): valid pixels from global, zero elsewhere
    for (int e = tid; e < PLS; e += NT) {
        const int lr = e / (2 * RP), c = (e / RP) & 1, p = e % RP - 1;
        const int rr = r0 - 1 + lr;
        const bool valid = lr <= nr + 1 && rr >= 0 && rr < H && p >= 0 && p < ((W + 1 - (c ^ (rr & 1))) >> 1);
        const size_t g = valid ? (size_t)rr * 2 * hw + c * hw + p : 0;
        T v[15];
#pragma unroll
        for (int z = 0; z < 12; z++) v[z] = valid ? it.sys[z][g] : (T)0;
#pragma unroll
        for (int z = 12; z < 15; z++) v[z] = (valid && !L.xin_zero) ? it.x[L.xin][z - 12][g] : (T)0;
#pragma unroll
        for (int z = 0; z < 15; z++) buf[z * PLS + e] = v[z];
    }
    if (tid == 0) s_stop = 0;
    cl.sync();  // every CTA of the cluster has started and staged (its shared memory may be read)
    T* const up_buf = rank > 0 ? cl.map_shared_rank(buf, rank - 1) : nullptr;
    T* const dn_buf = rank < C - 1 ? cl.map_shared_rank(buf, rank + 1) : nullptr;
    for (int itn = 0; itn < k.n_sor; itn++) {
        const bool chk = !k.fixed && (itn % k.period == k.period - 1);
        T md = 0;
        for (int color = 0; color < 2; color++) {
            for (int q = tid; q < nr * hw; q += NT) {
                const int li = q / hw, m = q % hw, i = r0 + li;
                const int b = color ^ (i & 1);
                if (m >= ((W + 1 - b) >> 1)) continue;
                const int own = ((li + 1) * 2 + color) * RP + m + 1;
                const int oth = ((li + 1) * 2 + (color ^ 1)) * RP + m + 1;
                const int ol = oth - 1 + b, orr = oth + b, ou = oth - 2 * RP, od = oth + 2 * RP;
                T c[9], xl[3], xu[3], xr[3], xd[3], xp[3], nv[3];
#pragma unroll
                for (int z = 0; z < 9; z++) c[z] = buf[z * PLS + own];
#pragma unroll
                for (int v = 0; v < 3; v++) {
                    const T* xv = buf + (12 + v) * PLS;
                    xl[v] = xv[ol]; xr[v] = xv[orr]; xu[v] = xv[ou]; xd[v] = xv[od]; xp[v] = xv[own];
                }
                sor_point<T>(c, buf[9 * PLS + ol], buf[10 * PLS + ou], buf[9 * PLS + own], buf[10 * PLS + own],
                             buf[11 * PLS + ol], buf[11 * PLS + ou], buf[11 * PLS + own], xl, xu, xr, xd, xp,
                             k.omega, k.step, nv);
#pragma unroll
                for (int v = 0; v < 3; v++) buf[(12 + v) * PLS + own] = nv[v];
                if (chk)
                    for (int v = 0; v < 3; v++) md = maxT(md, absT(nv[v] - xp[v]));
            }
            cl.sync();  // this half-sweep is done in every CTA
            // the neighbours' boundary rows of this colour into the halo rows (x planes); the
            // neighbours write the other colour meanwhile, and reach this colour again only after
            // the next cluster barrier
            for (int e = tid; e < 2 * 3 * RP; e += NT) {
                const int side = e / (3 * RP), v = (e / RP) % 3, p = e % RP;
                const T* src = side == 0 ? up_buf : dn_buf;
                if (!src) continue;
                const int srow = side == 0 ? B : 1;  // the neighbour's last / first own row
                const int drow = side == 0 ? 0 : nr + 1;
                buf[(12 + v) * PLS + (drow * 2 + color) * RP + p] = src[(12 + v) * PLS + (srow * 2 + color) * RP + p];
            }
            __syncthreads();
        }
        if (chk) {
            float mm = (float)md;
            for (int off = 16; off > 0; off >>= 1) mm = fmaxf(mm, __shfl_xor_sync(0xffffffffu, mm, off));
            if ((tid & 31) == 0) red[tid >> 5] = (T)mm;
            __syncthreads();
            if (tid == 0) {
                float g = 0;
                for (int w = 0; w < NT / 32; w++) g = fmaxf(g, (float)red[w]);
                s_max = g;
            }
            cl.sync();  // every CTA's maximum is in place
            if (tid == 0) {
                float g = 0;
                for (int r = 0; r < C; r++) g = fmaxf(g, *cl.map_shared_rank(&s_max, r));
                if (rank == 0) {
                    const int ci = min(itn / k.period, kMaxChecks - 1);
                    if (g > 0) ctl->maxdiff[ci] = __float_as_uint(g);
                }
                if ((double)g < k.sor_tol || (T)g >= k.step) {
                    s_stop = 1;
                    if (rank == 0) { ctl->sor_stop = 1; ctl->sor_stop_iter = itn + 1; }
                }
            }
            cl.sync();  // every CTA has read the maxima (s_max may be rewritten) and decided
            if (s_stop) break;
        }
    }
    // no CTA may leave while a neighbour still copies from its shared memory (the last half-sweep's
    // halo rows)
    cl.sync();
    // x of the own rows to global: the next inner iteration's buffer, or (fold) scratch that the CTA
    // folding each tile reads (the fold's next use of x starts from zero)
    T* const* xo = it.x[L.final_fold ? 0 : L.xout];
    for (int q = tid; q < nr * W; q += NT) {
        const int li = q / W, gj = q % W, gi = r0 + li;
        const int o = ((li + 1) * 2 + ((gi + gj) & 1)) * RP + (gj >> 1) + 1;
        const int lc = cs_idx(gi, gj, hw);
        for (int v = 0; v < 3; v++) xo[v][lc] = buf[(12 + v) * PLS + o];
    }
    if (!L.final_fold) return;
    __threadfence();
    cl.sync();  // every CTA's x is in global memory
    const int sx = (W + kSorTW - 1) / kSorTW, sy = (H + kSorTH - 1) / kSorTH;
    const int pitch = it.pitch;
    const T fl = it.f_level;
    const int lane = tid & 31;
    for (int ti = rank; ti < sx * sy; ti += C) {
        const int ix0 = (ti % sx) * kSorTW, iy0 = (ti / sx) * kSorTH;
        // the tile kernels' order: virtual thread vt (0..511) takes pixels vt and vt + 512 of the
        // tile, a warp tree per virtual warp, then the 16 virtual warps in order
        for (int vw = tid >> 5; vw < 16; vw += NT >> 5) {
            T part = 0;
            for (int q = vw * 32 + lane; q < kSorTW * kSorTH; q += 512) {
                const int gi = iy0 + q / kSorTW, gj = ix0 + q % kSorTW;
                if (gi >= H || gj >= W) continue;
                const int lc = cs_idx(gi, gj, hw);
                const T a = __ldcg(xo[0] + lc), bq = __ldcg(xo[1] + lc), cz = __ldcg(xo[2] + lc);
                const size_t lp = (size_t)gi * pitch + gj;
                it.u[0][lp] = addR(it.u[0][lp], a); it.u[1][lp] = addR(it.u[1][lp], bq);
                it.u[2][lp] = addR(it.u[2][lp], cz);
                part = addR(part, stat_px<T>(a, bq, cz, fl, it.pyr[6][(size_t)gi * W + gj]));
            }
            for (int off = 16; off > 0; off >>= 1) part += __shfl_down_sync(0xffffffffu, part, off);
            if (lane == 0) red[vw] = part;
        }
        __syncthreads();
        if (tid == 0) {
            T tot = 0;
            for (int w = 0; w < 16; w++) tot += red[w];
            it.stat_part[ti] = tot;
        }
        __syncthreads();
    }
    if (L.control) {
        __threadfence();
        cl.sync();  // every tile's statistic partial is written
        if (rank == 0 && tid < 32) control_item(it, k, L.outer, L.n_checks, tid);
    }
}

// ------------------------------------------------------------------------------------------
// Whole-level SOR over a thread-block cluster with the system in registers (FP32): the schedule,
// halo exchange and results of k_sor_level_cluster, but a thread owns KP positions of its CTA's
// row band (one pixel of each colour per position) whose coefficients, the 4 neighbour
// coefficients their updates need and their own unknowns stay in registers for the whole launch.
// Shared memory holds only the three increment planes of the band plus a halo row above and
// below, so a pixel update reads 12 values from shared memory instead of 31.
template <int KP> __host__ __device__ constexpr int clus_reg_threads_max() { return KP == 1 ? 768 : 640; }
template <class T> __host__ __device__ constexpr size_t level_cluster_reg_smem_bytes(int B, int hwp)
{
    return sizeof(T) * ((size_t)3 * (B + 2) * 2 * level_reg_rp(hwp) + 64);
}

template <class T, class S, int KP>
__global__ void __launch_bounds__(clus_reg_threads_max<KP>(), 1)
k_sor_level_cluster_reg(const LevelItem<T, S>* items, const int* which, SolveConst<T> k, SorLaunch L)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* const xb = reinterpret_cast<T*>(smem_raw);
    __shared__ int s_stop;
    __shared__ float s_max;
    __shared__ T red[32];
    const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const LevelItem<T, S>& it = items[which[blockIdx.x / C]];
    PairCtl* ctl = it.ctl;
    if (ctl->level_done) return;  // the same for every CTA of the cluster: none reaches a barrier
    const int W = it.W, H = it.H, hw = it.hwp, RP = level_reg_rp(hw);
    const int B = (H + C - 1) / C, r0 = rank * B, nr = max(0, min(H, r0 + B) - r0);
    const int PLS = (B + 2) * 2 * RP;
    const int tid = threadIdx.x, NT = blockDim.x;
    // the unknowns of rows r0 - 1 .. r0 + nr (local rows 0 .. nr + 1): valid pixels from global,
    // zero elsewhere
    for (int e = tid; e < 3 * PLS; e += NT) {
        const int v = e / PLS, f = e % PLS;
        const int lr = f / (2 * RP), c = (f / RP) & 1, p = f % RP - 1;
        const int rr = r0 - 1 + lr;
        const bool valid = !L.xin_zero && lr <= nr + 1 && rr >= 0 && rr < H && p >= 0 &&
                           p < ((W + 1 - (c ^ (rr & 1))) >> 1);
        xb[e] = valid ? it.x[L.xin][v][(size_t)rr * 2 * hw + c * hw + p] : (T)0;
    }
    // this thread's positions (local row li, half-row index m) and their pixels' systems
    T cf[KP][2][9], aL[KP][2], aU[KP][2], aR[KP][2], aD[KP][2], sL[KP][2], sU[KP][2], sw[KP][2], xp[KP][2][3];
    int li[KP], mm[KP];
    bool valid[KP][2];
#pragma unroll
    for (int kp = 0; kp < KP; kp++) {
        const int q = tid + kp * NT;
        li[kp] = q / hw;
        mm[kp] = q % hw;
        const int i = r0 + li[kp], m = mm[kp];
        const bool inpos = q < nr * hw;
#pragma unroll
        for (int color = 0; color < 2; color++) {
            const int b = color ^ (i & 1);
            const bool vd = inpos && m < ((W + 1 - b) >> 1);
            valid[kp][color] = vd;
            const size_t g = (size_t)i * 2 * hw + color * hw + m;
            // the left neighbour is the other colour's position m - 1 + b of the row, the upper one
            // its position m of the row above; outside the level they are zero
            const int ml = m - 1 + b;
            const bool lok = vd && ml >= 0 && ml < ((W + 1 - (b ^ 1)) >> 1);
            const bool uok = vd && i >= 1;
            const size_t gl = (size_t)i * 2 * hw + (color ^ 1) * hw + ml;
            const size_t gu = (size_t)(i - 1) * 2 * hw + (color ^ 1) * hw + m;
#pragma unroll
            for (int z = 0; z < 9; z++) cf[kp][color][z] = vd ? it.sys[z][g] : (T)0;
            aR[kp][color] = vd ? it.sys[9][g] : (T)0;
            aD[kp][color] = vd ? it.sys[10][g] : (T)0;
            sw[kp][color] = vd ? it.sys[11][g] : (T)0;
            aL[kp][color] = lok ? it.sys[9][gl] : (T)0;
            sL[kp][color] = lok ? it.sys[11][gl] : (T)0;
            aU[kp][color] = uok ? it.sys[10][gu] : (T)0;
            sU[kp][color] = uok ? it.sys[11][gu] : (T)0;
        }
    }
    if (tid == 0) s_stop = 0;
    cl.sync();  // every CTA of the cluster has started and staged (its shared memory may be read)
    // own unknowns of the valid pixels (a thread past the band's positions reads nothing)
#pragma unroll
    for (int kp = 0; kp < KP; kp++)
#pragma unroll
        for (int color = 0; color < 2; color++)
#pragma unroll
            for (int v = 0; v < 3; v++)
                xp[kp][color][v] = valid[kp][color] ? xb[v * PLS + ((li[kp] + 1) * 2 + color) * RP + mm[kp] + 1] : (T)0;
    T* const up_buf = rank > 0 ? cl.map_shared_rank(xb, rank - 1) : nullptr;
    T* const dn_buf = rank < C - 1 ? cl.map_shared_rank(xb, rank + 1) : nullptr;
    for (int itn = 0; itn < k.n_sor; itn++) {
        const bool chk = !k.fixed && (itn % k.period == k.period - 1);
        T md = 0;
#pragma unroll
        for (int color = 0; color < 2; color++) {
#pragma unroll
            for (int kp = 0; kp < KP; kp++) {
                if (valid[kp][color]) {
                    const int b = color ^ ((r0 + li[kp]) & 1);
                    const int own = ((li[kp] + 1) * 2 + color) * RP + mm[kp] + 1;
                    const int oth = ((li[kp] + 1) * 2 + (color ^ 1)) * RP + mm[kp] + 1;
                    const int ol = oth - 1 + b, orr = oth + b, ou = oth - 2 * RP, od = oth + 2 * RP;
                    T xl[3], xu[3], xr[3], xd[3], nv[3];
#pragma unroll
                    for (int v = 0; v < 3; v++) {
                        const T* xv = xb + v * PLS;
                        xl[v] = xv[ol]; xr[v] = xv[orr]; xu[v] = xv[ou]; xd[v] = xv[od];
                    }
                    sor_point<T>(cf[kp][color], aL[kp][color], aU[kp][color], aR[kp][color], aD[kp][color],
                                 sL[kp][color], sU[kp][color], sw[kp][color], xl, xu, xr, xd, xp[kp][color], k.omega,
                                 k.step, nv);
#pragma unroll
                    for (int v = 0; v < 3; v++) {
                        xb[v * PLS + own] = nv[v];
                        if (chk) md = maxT(md, absT(nv[v] - xp[kp][color][v]));
                        xp[kp][color][v] = nv[v];
                    }
                }
            }
            cl.sync();  // this half-sweep is done in every CTA
            // the neighbours' boundary rows of this colour into the halo rows; the neighbours write
            // the other colour meanwhile, and reach this colour again only after the next cluster
            // barrier
            for (int e = tid; e < 2 * 3 * RP; e += NT) {
                const int side = e / (3 * RP), v = (e / RP) % 3, p = e % RP;
                const T* src = side == 0 ? up_buf : dn_buf;
                if (!src) continue;
                const int srow = side == 0 ? B : 1;  // the neighbour's last / first own row
                const int drow = side == 0 ? 0 : nr + 1;
                xb[v * PLS + (drow * 2 + color) * RP + p] = src[v * PLS + (srow * 2 + color) * RP + p];
            }
            __syncthreads();
        }
        if (chk) {
            float mx = (float)md;
            for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
            if ((tid & 31) == 0) red[tid >> 5] = (T)mx;
            __syncthreads();
            if (tid == 0) {
                float g = 0;
                for (int w = 0; w < NT / 32; w++) g = fmaxf(g, (float)red[w]);
                s_max = g;
            }
            cl.sync();  // every CTA's maximum is in place
            if (tid == 0) {
                float g = 0;
                for (int r = 0; r < C; r++) g = fmaxf(g, *cl.map_shared_rank(&s_max, r));
                if (rank == 0) {
                    const int ci = min(itn / k.period, kMaxChecks - 1);
                    if (g > 0) ctl->maxdiff[ci] = __float_as_uint(g);
                }
                if ((double)g < k.sor_tol || (T)g >= k.step) {
                    s_stop = 1;
                    if (rank == 0) { ctl->sor_stop = 1; ctl->sor_stop_iter = itn + 1; }
                }
            }
            cl.sync();  // every CTA has read the maxima (s_max may be rewritten) and decided
            if (s_stop) break;
        }
    }
    // no CTA may leave while a neighbour still copies from its shared memory (the last half-sweep's
    // halo rows)
    cl.sync();
    // x of the own rows to global: the next inner iteration's buffer, or (fold) scratch that the CTA
    // folding each tile reads (the fold's next use of x starts from zero)
    T* const* xo = it.x[L.final_fold ? 0 : L.xout];
    for (int q = tid; q < nr * W; q += NT) {
        const int lr = q / W, gj = q % W, gi = r0 + lr;
        const int o = ((lr + 1) * 2 + ((gi + gj) & 1)) * RP + (gj >> 1) + 1;
        const int lc = cs_idx(gi, gj, hw);
        for (int v = 0; v < 3; v++) xo[v][lc] = xb[v * PLS + o];
    }
    if (!L.final_fold) return;
    __threadfence();
    cl.sync();  // every CTA's x is in global memory
    const int sx = (W + kSorTW - 1) / kSorTW, sy = (H + kSorTH - 1) / kSorTH;
    const int pitch = it.pitch;
    const T fl = it.f_level;
    const int lane = tid & 31;
    for (int ti = rank; ti < sx * sy; ti += C) {
        const int ix0 = (ti % sx) * kSorTW, iy0 = (ti / sx) * kSorTH;
        // the tile kernels' order: virtual thread vt (0..511) takes pixels vt and vt + 512 of the
        // tile, a warp tree per virtual warp, then the 16 virtual warps in order
        for (int vw = tid >> 5; vw < 16; vw += NT >> 5) {
            T part = 0;
            for (int q = vw * 32 + lane; q < kSorTW * kSorTH; q += 512) {
                const int gi = iy0 + q / kSorTW, gj = ix0 + q % kSorTW;
                if (gi >= H || gj >= W) continue;
                const int lc = cs_idx(gi, gj, hw);
                const T a = __ldcg(xo[0] + lc), bq = __ldcg(xo[1] + lc), cz = __ldcg(xo[2] + lc);
                const size_t lp = (size_t)gi * pitch + gj;
                it.u[0][lp] = addR(it.u[0][lp], a); it.u[1][lp] = addR(it.u[1][lp], bq);
                it.u[2][lp] = addR(it.u[2][lp], cz);
                part = addR(part, stat_px<T>(a, bq, cz, fl, it.pyr[6][(size_t)gi * W + gj]));
            }
            for (int off = 16; off > 0; off >>= 1) part += __shfl_down_sync(0xffffffffu, part, off);
            if (lane == 0) red[vw] = part;
        }
        __syncthreads();
        if (tid == 0) {
            T tot = 0;
            for (int w = 0; w < 16; w++) tot += red[w];
            it.stat_part[ti] = tot;
        }
        __syncthreads();
    }
    if (L.control) {
        __threadfence();
        cl.sync();  // every tile's statistic partial is written
        if (rank == 0 && tid < 32) control_item(it, k, L.outer, L.n_checks, tid);
    }
}

// After each outer iteration: the early-termination statistic of the pair (mean over 3N of
// sqr(du) * (1, 1, f / depth1), .cu:943-951), the stop decision and the executed-schedule record.
// One warp per item (lane = the thread's lane); the statistic partials are read from L2 (the
// whole-level cluster kernel calls this after other CTAs wrote them).
template <class T, class S>
__device__ __forceinline__ void control_item(const LevelItem<T, S>& it, const SolveConst<T>& k, int outer, int n_checks,
                                             int lane)
{
    PairCtl* ctl = it.ctl;
    if (ctl->level_done) return;
    T s = 0;
    for (int i = lane; i < it.n_sor_tiles; i += 32) s += __ldcg(it.stat_part + i);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) {
        const double st = (double)s / ((double)it.W * it.H * 3);
        const int lv = it.level;
        if (outer < 64) {
            ctl->sor_exec[lv][outer] = ctl->sor_stop ? ctl->sor_stop_iter : k.n_sor;
            ctl->stat[lv][outer] = (it.allow_early && !k.fixed) ? (float)st : -1.0f;
            float md = -1.0f;  // the last convergence check evaluated in this outer iteration
            for (int c = min(n_checks, kMaxChecks) - 1; c >= 0; c--) {
                const unsigned b = ctl->maxdiff[c];
                if (b) { md = __uint_as_float(b); break; }
            }
            ctl->sor_maxdiff[lv][outer] = md;
        }
        ctl->outer_exec[lv] = outer + 1;
        if (it.allow_early && !k.fixed && st < k.outer_tol) ctl->level_done = 1;
    }
}

template <class T, class S>
__global__ void k_control(const LevelItem<T, S>* items, int n_items, SolveConst<T> k, int outer, int n_checks)
{
    const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (w >= n_items) return;
    control_item(items[w], k, outer, n_checks, threadIdx.x & 31);
}

// Final flow (level 0) to the caller's interleaved (u, v, w) float layout.
template <class T, class S>
__global__ void k_output(const LevelItem<T, S>* items, const Tile* tiles, T* const* outs)
{
    const Tile t = tiles[blockIdx.x];
    const LevelItem<T, S>& it = items[t.item];
    const int j = t.tx * LTW + (threadIdx.x % LTW), i = t.ty * LTH + (threadIdx.x / LTW);
    if (i >= it.H || j >= it.W) return;
    const int l = i * it.W + j;
    T* o = outs[t.item];
    const int lp = i * it.pitch + j;
    o[(size_t)l * 3 + 0] = it.u[0][lp];
    o[(size_t)l * 3 + 1] = it.u[1][lp];
    o[(size_t)l * 3 + 2] = it.u[2][lp];
}

// Device warp of the final flow (for the single-scale seam's warpIm2 / warpDm2 outputs).
// Output block of a pair: flow (3N interleaved), then warped features (5N interleaved), then the
// warped depth (N).
template <class T, class S>
__global__ void k_warp_out(const LevelItem<T, S>* items, const Tile* tiles, T* const* outs)
{
    const Tile t = tiles[blockIdx.x];
    const LevelItem<T, S>& it = items[t.item];
    const int j = t.tx * LTW + (threadIdx.x % LTW), i = t.ty * LTH + (threadIdx.x / LTW);
    if (i >= it.H || j >= it.W) return;
    const int W = it.W, H = it.H, l = i * W + j;
    T* wI = outs[t.item] + (size_t)3 * W * H;
    T* wD = outs[t.item] + (size_t)8 * W * H;
    const int lp = i * it.pitch + j;
    const T U0 = it.u[0][lp], U1 = it.u[1][lp], U2 = it.u[2][lp];
    const T x = (T)j + U0, y = (T)i + U1;
    if (x < 0 || x > (T)(W - 1) || y < 0 || y > (T)(H - 1)) {
        for (int c = 0; c < 5; c++) wI[(size_t)l * 5 + c] = ldS<T, S>(it.I1[c] + l);
        wD[l] = ldS<T, S>(it.D1 + l) - U2;
        return;
    }
    const int xa = clampi((int)floor(x), 0, W - 1), ya = clampi((int)floor(y), 0, H - 1);
    const int xb = min(W - 1, xa + 1), yb = min(H - 1, ya + 1);
    const T ax = x - (T)xa, ay = y - (T)ya;
    const T w00 = (1 - ax) * (1 - ay), w01 = (1 - ax) * ay, w10 = ax * (1 - ay), w11 = ax * ay;
    const int p00 = ya * W + xa, p01 = yb * W + xa, p10 = ya * W + xb, p11 = yb * W + xb;
    for (int c = 0; c < 5; c++) {
        const S* s = it.I2[c];
        wI[(size_t)l * 5 + c] = w00 * ldS<T, S>(s + p00) + w01 * ldS<T, S>(s + p01) + w10 * ldS<T, S>(s + p10) +
                                w11 * ldS<T, S>(s + p11);
    }
    const S* s = it.D2;
    wD[l] = w00 * ldS<T, S>(s + p00) + w01 * ldS<T, S>(s + p01) + w10 * ldS<T, S>(s + p10) + w11 * ldS<T, S>(s + p11) - U2;
}

// Warm start (sceneFlowWithInit.cpp:11-20): the caller's flow estimate becomes the finest level's u.
struct EstSrc {
    const float* f;   // interleaved (u, v, w) floats, or null
    const double* d;  // planar u, v, w doubles, or null
};

template <class T, class S>
__global__ void k_load_est(const LevelItem<T, S>* items, const Tile* tiles, const EstSrc* est)
{
    const Tile t = tiles[blockIdx.x];
    const LevelItem<T, S>& it = items[t.item];
    if (!it.est_init) return;
    const EstSrc e = est[t.item];
    const int j = t.tx * LTW + (threadIdx.x % LTW), i = t.ty * LTH + (threadIdx.x / LTW);
    if (i >= it.H || j >= it.W) return;
    const int l = i * it.W + j;
    const size_t N = (size_t)it.W * it.H;
    const int lp = i * it.pitch + j;
    for (int c = 0; c < 3; c++) it.u[c][lp] = e.f ? (T)e.f[(size_t)l * 3 + c] : (T)e.d[c * N + l];
}

// Per-level seam (sceneFlowSingleScale's own inputs): features, depths, weights and flow come
// from the caller as FP64 planes; this kernel only converts them into the level's planes.
struct SeamSrc {
    const double* im1; const double* im2;   // W*H*5 interleaved features
    const double* dm1; const double* dm2;   // W*H
    const double* uvw;                      // 3 planes
    const double* ddw; const double* dsw; const double* mag;
    const double* regw;                     // W*H*2 interleaved (right, down)
};

template <class T, class S>
__global__ void k_seam_load(const LevelItem<T, S>* items, const Tile* tiles, const SeamSrc* src)
{
    const Tile t = tiles[blockIdx.x];
    const LevelItem<T, S>& it = items[t.item];
    const SeamSrc q = src[t.item];
    if (t.idx == 0 && threadIdx.x == 0) it.ctl->level_done = 0;
    const int j = t.tx * LTW + (threadIdx.x % LTW), i = t.ty * LTH + (threadIdx.x / LTW);
    if (i >= it.H || j >= it.W) return;
    const int W = it.W, H = it.H, l = i * W + j;
    const size_t N = (size_t)W * H;
    for (int c = 0; c < 5; c++) {
        it.I1[c][l] = stS<S>((T)q.im1[(size_t)l * 5 + c]);
        it.I2[c][l] = stS<S>((T)q.im2[(size_t)l * 5 + c]);
    }
    it.D1[l] = stS<S>((T)q.dm1[l]);
    it.D2[l] = stS<S>((T)q.dm2[l]);
    it.pyr[6][l] = (T)q.dm1[l];
    it.pyr[7][l] = (T)q.dm2[l];
    it.pyr[8][l] = (T)q.ddw[l];
    it.pyr[9][l] = (T)q.dsw[l];
    it.mag[l] = (T)q.mag[l];
    // weights of edges that leave the image are never used by the reference; keep them 0
    it.rh[l] = (j < W - 1) ? (T)q.regw[(size_t)l * 2 + 0] : (T)0;
    it.rv[l] = (i < H - 1) ? (T)q.regw[(size_t)l * 2 + 1] : (T)0;
    const int lp = i * it.pitch + j;
    for (int c = 0; c < 3; c++) it.u[c][lp] = (T)q.uvw[c * N + l];
}

}  // namespace rgbdflow
