// flow2d.cuh — 2-D optical flow on the device: Ce Liu's coarse-to-fine solver, the reference
// demo's flow type 1 (OpticalFlow::Coarse2FineFlow, src/opticalFlowMultiscale.cpp:4-146, with
// OpticalFlow::SmoothFlowSOR, src/SmoothFlowSOR.cpp:8-247).
//
// The reference's solver is numerically fragile (lexicographic SOR with omega 1.8): reordering
// its sweep changes the result by pixels on ordinary scenes.  So this solve keeps the
// reference's arithmetic exactly: FP64, every operation rounded on its own (explicit __d*_rn
// intrinsics, no fused multiply-adds), the reference's operation order, and its lexicographic
// SOR order.  The SOR runs as anti-diagonal wavefronts: pixel (i, j) needs new values only from
// diagonal i + j - 1 of its own sweep and old values from diagonal i + j + 1 of the previous
// one, so one diagonal is a parallel step.  Consecutive sweeps overlap, each starting two steps
// after the previous one; sweep s writes ring slot s % D and reads the previous sweep from slot
// (s - 1) % D, and starts only after sweep s - D has finished without converging, so the slot of
// the sweep that converges is never overwritten.
//
// Data: planar FP64 per level; colour pyramids 3 channels interleaved (as DImage), features 5
// channels interleaved.
#pragma once
#include <cuda_runtime.h>
#include <cooperative_groups.h>

#include <cmath>
#include <vector>

namespace rgbdflow {
namespace f2d {

constexpr int kThreads = 256;
constexpr int kSorThreads = 1024;
constexpr int kMaxRing = 16;
constexpr int kMaxTaps = 64;

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ int clampi(int x, int n) { return min(max(x, 0), n - 1); }
// std::max(a, b) of the C++ library: (a < b) ? b : a (a NaN b is dropped, a NaN a is kept)
__device__ __forceinline__ double cmax(double a, double b) { return (a < b) ? b : a; }

// ImageProcessing::BilinearInterpolate, accumulating form (ImageProcessing.h:128-148)
__device__ __forceinline__ void bilinear_acc(const double* img, int W, int H, int C, double x, double y, double* out)
{
    const int xx = (int)x, yy = (int)y;
    double dx = dsub(x, (double)xx);
    if (dx > 1) dx = 1;
    if (dx < 0) dx = 0;
    double dy = dsub(y, (double)yy);
    if (dy > 1) dy = 1;
    if (dy < 0) dy = 0;
    for (int m = 0; m <= 1; m++)
        for (int n = 0; n <= 1; n++) {
            const int u = clampi(xx + m, W), v = clampi(yy + n, H);
            const size_t off = ((size_t)v * W + u) * C;
            const double s = dmul(fabs(dsub((double)(1 - m), dx)), fabs(dsub((double)(1 - n), dy)));
            for (int l = 0; l < C; l++) out[l] = dadd(out[l], dmul(img[off + l], s));
        }
}

// colour / 255 (cv2liuBGR, src/ceLiuOpticalFlow.cpp:19-37)
__global__ void k_unpack(const uint8_t* __restrict__ bgr, double* __restrict__ out, size_t n)
{
    for (size_t z = blockIdx.x * (size_t)blockDim.x + threadIdx.x; z < n; z += (size_t)gridDim.x * blockDim.x)
        out[z] = ddiv((double)bgr[z], 255.0);
}

// ImageProcessing::hfiltering / vfiltering with clamp-to-edge (ImageProcessing.h:247-269, 339-358)
__global__ void k_hfilter(const double* __restrict__ in, double* __restrict__ out, int W, int H, int C,
                          const double* __restrict__ taps, int fs)
{
    const size_t n = (size_t)W * H;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(p / W), j = (int)(p % W);
        for (int k = 0; k < C; k++) {
            double acc = 0;
            for (int l = -fs; l <= fs; l++)
                acc = dadd(acc, dmul(in[((size_t)i * W + clampi(j + l, W)) * C + k], taps[l + fs]));
            out[p * C + k] = acc;
        }
    }
}
__global__ void k_vfilter(const double* __restrict__ in, double* __restrict__ out, int W, int H, int C,
                          const double* __restrict__ taps, int fs)
{
    const size_t n = (size_t)W * H;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(p / W), j = (int)(p % W);
        for (int k = 0; k < C; k++) {
            double acc = 0;
            for (int l = -fs; l <= fs; l++)
                acc = dadd(acc, dmul(in[((size_t)clampi(i + l, H) * W + j) * C + k], taps[l + fs]));
            out[p * C + k] = acc;
        }
    }
}

// ImageProcessing::ResizeImage (ImageProcessing.h:203-242): dst (j, i) samples src at
// ((j + 1) / xr - 1, (i + 1) / yr - 1)
__global__ void k_resize(const double* __restrict__ in, int W, int H, int C, double* __restrict__ out, int DW, int DH,
                         double xr, double yr)
{
    const size_t n = (size_t)DW * DH;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(p / DW), j = (int)(p % DW);
        double acc[5] = {0, 0, 0, 0, 0};
        const double x = dsub(ddiv((double)(j + 1), xr), 1.0), y = dsub(ddiv((double)(i + 1), yr), 1.0);
        bilinear_acc(in, W, H, C, x, y, acc);
        for (int k = 0; k < C; k++) out[p * C + k] = acc[k];
    }
}

// Image::desaturate (Image.h:1438-1469): .114 B + .587 G + .299 R, channels in BGR order
__device__ __forceinline__ double gray_at(const double* im, size_t p)
{
    return dadd(dadd(dmul(im[p * 3], .114), dmul(im[p * 3 + 1], .587)), dmul(im[p * 3 + 2], .299));
}

// OpticalFlow::im2feature RGB_WITH_GRADIENT (OpticalFlow.cpp:189-214): gray, its 5-tap dx, dy,
// G - B, G - R
__global__ void k_features(const double* __restrict__ im, double* __restrict__ feat, int W, int H,
                           const double* __restrict__ d5)
{
    const size_t n = (size_t)W * H;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(p / W), j = (int)(p % W);
        double gx = 0, gy = 0;
        for (int l = -2; l <= 2; l++) gx = dadd(gx, dmul(gray_at(im, (size_t)i * W + clampi(j + l, W)), d5[l + 2]));
        for (int l = -2; l <= 2; l++) gy = dadd(gy, dmul(gray_at(im, (size_t)clampi(i + l, H) * W + j), d5[l + 2]));
        feat[p * 5 + 0] = gray_at(im, p);
        feat[p * 5 + 1] = gx;
        feat[p * 5 + 2] = gy;
        feat[p * 5 + 3] = dsub(im[p * 3 + 1], im[p * 3]);
        feat[p * 5 + 4] = dsub(im[p * 3 + 1], im[p * 3 + 2]);
    }
}

// x *= s (Image::Multiplywith, Image.h:1778-1782)
__global__ void k_scale(double* __restrict__ x, size_t n, double s)
{
    for (size_t z = blockIdx.x * (size_t)blockDim.x + threadIdx.x; z < n; z += (size_t)gridDim.x * blockDim.x)
        x[z] = dmul(x[z], s);
}

// warpFL, bilinear (src/opticalFlowUtils.cpp:62-67; ImageProcessing::warpImage,
// ImageProcessing.h:472-491): Im2 at (j + u, i + v), Im1 where that falls outside
__global__ void k_warp(const double* __restrict__ f1, const double* __restrict__ f2, const double* __restrict__ u,
                       const double* __restrict__ v, double* __restrict__ out, int W, int H)
{
    const size_t n = (size_t)W * H;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(p / W), j = (int)(p % W);
        const double x = dadd((double)j, u[p]), y = dadd((double)i, v[p]);
        double acc[5] = {0, 0, 0, 0, 0};
        if (x < 0 || x > W - 1 || y < 0 || y > H - 1) {
            for (int k = 0; k < 5; k++) acc[k] = f1[p * 5 + k];
        } else {
            bilinear_acc(f2, W, H, 5, x, y, acc);
        }
        for (int k = 0; k < 5; k++) out[p * 5 + k] = acc[k];
    }
}

// One level's per-iteration state.
struct LevelBufs {
    const double *f1, *f2;  // features of frames 1 and 2 (5 channels)
    double* warp;           // frame 2 features warped by the flow (5 channels)
    double *u, *v, *du, *dv, *phi;
    double *dxy, *dx2, *dy2, *dtdx, *dtdy;
    double* coef;  // the SOR's per-pixel coefficients packed, 8 doubles a pixel: dxy, dx2, dy2,
                   // dtdx, dtdy, phi (written by k_rhs; read-only during the SOR)
    int W, H;
};

// 0.4 Im1 + 0.6 warp at pixel p, channel k (getDxs, src/opticalFlowUtils.cpp:33-37)
__device__ __forceinline__ double mix_at(const LevelBufs& b, size_t p, int k)
{
    return dadd(dmul(b.f1[p * 5 + k], 0.4), dmul(b.warp[p * 5 + k], 0.6));
}

// SmoothFlowSOR.cpp:52-139 for one inner iteration: the flow gradient weight phi of u + du
// (forward differences, Image::dx/dy, Image.h:955-1019), and the robust data weights psi of the
// derivatives of getDxs (5-tap dx, dy of 0.4 Im1 + 0.6 warp, dt = warp - Im1), multiplied out
// and averaged over the channels (Image::Multiply, Image::collapse).  first: the inner
// iteration's uu is u itself.
// eps: pow(0.001, 2) as the host's pow computes it (SmoothFlowSOR.cpp:30-31).
__global__ void k_phi_psi(LevelBufs b, const double* __restrict__ d5, int first, double eps)
{
    const int W = b.W, H = b.H;
    const size_t n = (size_t)W * H;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(p / W), j = (int)(p % W);
        auto uu = [&](size_t q) { return first ? b.u[q] : dadd(b.u[q], b.du[q]); };
        auto vv = [&](size_t q) { return first ? b.v[q] : dadd(b.v[q], b.dv[q]); };
        const double ux = (j < W - 1) ? dsub(uu(p + 1), uu(p)) : 0.0;
        const double uy = (i < H - 1) ? dsub(uu(p + W), uu(p)) : 0.0;
        const double vx = (j < W - 1) ? dsub(vv(p + 1), vv(p)) : 0.0;
        const double vy = (i < H - 1) ? dsub(vv(p + W), vv(p)) : 0.0;
        const double t = dadd(dadd(dadd(dmul(ux, ux), dmul(uy, uy)), dmul(vx, vx)), dmul(vy, vy));
        b.phi[p] = ddiv(0.5, __dsqrt_rn(dadd(t, eps)));
        const double du = first ? 0.0 : b.du[p], dv = first ? 0.0 : b.dv[p];
        double sxy = 0, sx2 = 0, sy2 = 0, stx = 0, sty = 0;
        for (int k = 0; k < 5; k++) {
            double ix = 0, iy = 0;
            for (int l = -2; l <= 2; l++) ix = dadd(ix, dmul(mix_at(b, (size_t)i * W + clampi(j + l, W), k), d5[l + 2]));
            for (int l = -2; l <= 2; l++) iy = dadd(iy, dmul(mix_at(b, (size_t)clampi(i + l, H) * W + j, k), d5[l + 2]));
            const double it = dsub(b.warp[p * 5 + k], b.f1[p * 5 + k]);
            double r = dadd(dadd(it, dmul(ix, du)), dmul(iy, dv));
            r = dmul(r, r);
            const double psi = ddiv(1.0, dmul(2.0, __dsqrt_rn(dadd(r, eps))));
            sxy = dadd(sxy, dmul(dmul(psi, ix), iy));
            sx2 = dadd(sx2, dmul(dmul(psi, ix), ix));
            sy2 = dadd(sy2, dmul(dmul(psi, iy), iy));
            stx = dadd(stx, dmul(dmul(psi, ix), it));
            sty = dadd(sty, dmul(dmul(psi, iy), it));
        }
        b.dxy[p] = ddiv(sxy, 5.0);
        b.dx2[p] = ddiv(sx2, 5.0);
        b.dy2[p] = ddiv(sy2, 5.0);
        b.dtdx[p] = ddiv(stx, 5.0);
        b.dtdy[p] = ddiv(sty, 5.0);
    }
}

// Laplacian with normalising weights (src/opticalFlowUtils.cpp:252-313) of x at pixel (i, j),
// weighted by the 1-channel phi read as a 2-channel image, as SmoothFlowSOR.cpp:144 calls it:
// channel k of (i, j) is element i * W + j + k (Image::operator(), Image.h:76).
__device__ __forceinline__ double laplacian_phi(const double* x, const double* phi, int W, int H, int i, int j)
{
    const size_t o = (size_t)i * W + j;
    double out = 0;
    if (j < W - 1) out = dsub(out, dmul(dsub(x[o + 1], x[o]), phi[o]));
    if (j > 0) out = dadd(out, dmul(dsub(x[o], x[o - 1]), phi[o - 1]));
    if (i < H - 1) out = dsub(out, dmul(dsub(x[o + W], x[o]), phi[o + 1]));
    if (i > 0) out = dadd(out, dmul(dsub(x[o], x[o - W]), phi[o - W + 1]));
    double norm = 0;
    int count = 0;
    if (j < W - 1) { norm = dadd(norm, phi[o]); count++; }
    if (j > 0) { norm = dadd(norm, phi[o - 1]); count++; }
    if (i < H - 1) { norm = dadd(norm, phi[o + 1]); count++; }
    if (i > 0) { norm = dadd(norm, phi[o - W + 1]); count++; }
    if (fabs(norm) < 1e-5) return 0;
    return ddiv(out, ddiv(norm, (double)count));
}

// The right-hand sides (SmoothFlowSOR.cpp:144-151): -Itx - alpha * Lap(u), -Ity - alpha * Lap(v)
__global__ void k_rhs(LevelBufs b, double alpha)
{
    const int W = b.W, H = b.H;
    const size_t n = (size_t)W * H;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(p / W), j = (int)(p % W);
        const double tx = dsub(-b.dtdx[p], dmul(alpha, laplacian_phi(b.u, b.phi, W, H, i, j)));
        const double ty = dsub(-b.dtdy[p], dmul(alpha, laplacian_phi(b.v, b.phi, W, H, i, j)));
        b.dtdx[p] = tx;
        b.dtdy[p] = ty;
        double4* c = reinterpret_cast<double4*>(b.coef + p * 8);
        c[0] = make_double4(b.dxy[p], b.dx2[p], b.dy2[p], tx);
        c[1] = make_double4(ty, b.phi[p], 0.0, 0.0);
    }
}

// One SOR update (SmoothFlowSOR.cpp:166-215) of pixel (i, j): left / upper neighbours new (this
// sweep's ring slot nw), right / lower neighbours and the pixel itself old (the previous sweep's
// slot ow); a slot holds (du, dv) pairs.  Writes the new pair to nw and returns the change.
template <bool CG = false>
__device__ __forceinline__ double sor_update(const LevelBufs& b, double alpha, int i, int j, double2* nw,
                                             const double2* ow)
{
    // CG: the ring is written by other CTAs of a cluster; its values are read from L2
    auto R = [](const double2* p) { return CG ? __ldcg(p) : *p; };
    const int W = b.W, H = b.H;
    const size_t o = (size_t)i * W + j;
    const double omega = 1.8;
    const double4 c0 = *reinterpret_cast<const double4*>(b.coef + o * 8);            // dxy, dx2, dy2, dtdx
    const double2 c1 = __ldg(reinterpret_cast<const double2*>(b.coef + o * 8 + 4));  // dtdy, phi
    const double phi = c1.y;
    double sigmaU = 0, sigmaV = 0, weightSum = 0, w;
    if (j > 0) {
        w = __ldg(b.coef + (o - 1) * 8 + 5);
        const double2 x = R(nw + o - 1);
        sigmaU = dadd(sigmaU, dmul(w, x.x)); sigmaV = dadd(sigmaV, dmul(w, x.y)); weightSum = dadd(weightSum, w);
    }
    if (j < W - 1) {
        w = phi;
        const double2 x = R(ow + o + 1);
        sigmaU = dadd(sigmaU, dmul(w, x.x)); sigmaV = dadd(sigmaV, dmul(w, x.y)); weightSum = dadd(weightSum, w);
    }
    if (i > 0) {
        w = __ldg(b.coef + (o - W) * 8 + 5);
        const double2 x = R(nw + o - W);
        sigmaU = dadd(sigmaU, dmul(w, x.x)); sigmaV = dadd(sigmaV, dmul(w, x.y)); weightSum = dadd(weightSum, w);
    }
    if (i < H - 1) {
        w = phi;
        const double2 x = R(ow + o + W);
        sigmaU = dadd(sigmaU, dmul(w, x.x)); sigmaV = dadd(sigmaV, dmul(w, x.y)); weightSum = dadd(weightSum, w);
    }
    sigmaU = dmul(sigmaU, -alpha);
    sigmaV = dmul(sigmaV, -alpha);
    weightSum = dmul(weightSum, alpha);
    const double2 prev = R(ow + o);
    const double prevDU = prev.x, prevDV = prev.y;
    sigmaU = dadd(sigmaU, dmul(c0.x, prevDV));
    const double nDU = dadd(dmul(1 - omega, prevDU), dmul(ddiv(omega, dadd(c0.y, weightSum)), dsub(c0.w, sigmaU)));
    sigmaV = dadd(sigmaV, dmul(c0.x, nDU));
    const double nDV = dadd(dmul(1 - omega, prevDV), dmul(ddiv(omega, dadd(c0.z, weightSum)), dsub(c1.x, sigmaV)));
    nw[o] = make_double2(nDU, nDV);
    return cmax(fabs(dsub(nDU, prevDU)), fabs(dsub(nDV, prevDV)));
}

// The step's work table, built by warp 0: for each sweep in flight (done + 1 .. next - 1, at most
// 64), its diagonal and first row, and the prefix count of the step's items up to it (pre[0] = 0,
// pre[n] = the step's items).  A sweep not on a diagonal of the level this step has no items.
__device__ __forceinline__ void sor_table(int W, int H, long long t, int done, int next, const long long* start, int D,
                                          int ndiag, int* pre, int* dd, int* ii0)
{
    const int lane = threadIdx.x & 31;
    const int n = next - (done + 1);
    int run = 0;
    for (int h = 0; h < 2; h++) {
        const int l = lane + 32 * h;
        int cnt = 0, d = 0, i0 = 0;
        if (l < n) {
            const long long dl = t - start[(done + 1 + l) % D];
            if (dl >= 0 && dl < ndiag) {
                d = (int)dl;
                i0 = max(0, d - (W - 1));
                cnt = min(H - 1, d) - i0 + 1;
            }
        }
        int x = cnt;  // inclusive scan over the warp
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (l < n) {
            pre[l + 1] = run + x;
            dd[l] = d;
            ii0[l] = i0;
        }
        run += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) pre[0] = 0;
}

// One step of the overlapping sweeps: for every sweep in flight, the pixels of its current
// diagonal.  The step's updates are flattened into one list spread over the G threads (thread g
// takes items g, g + G, ...), so the memory latency of the sweeps' updates overlaps across threads
// instead of adding up sweep after sweep; an item finds its sweep in the step's table by binary
// search.  Every update reads only values no other update of the step writes (the diagonal
// structure), so the order within the step is free.
template <bool CG>
__device__ __forceinline__ void sor_step(const LevelBufs& b, double alpha, int done, int next, const int* pre,
                                         const int* dd, const int* ii0, int D, size_t N, double2* ring,
                                         unsigned long long* maxd, int g, int G)
{
    const int n = next - (done + 1);
    const int total = n > 0 ? pre[n] : 0;
    // whole warps iterate together (item k = kb + lane), so the sweeps' maxima can be combined
    // per warp before the shared atomics
    const int lane = threadIdx.x & 31;
    for (int kb = g - lane; kb < total; kb += G) {
        const int k = kb + lane;
        int slot = -1;
        unsigned long long bits = 0;
        if (k < total) {
            int lo = 0, hi = n - 1;  // the sweep l with pre[l] <= k < pre[l + 1]
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (pre[mid + 1] > k) hi = mid;
                else lo = mid + 1;
            }
            const int s = done + 1 + lo;
            const int i = ii0[lo] + (k - pre[lo]);
            const int cur = s % D, prv = (s + D - 1) % D;
            const double m = sor_update<CG>(b, alpha, i, dd[lo] - i, ring + (size_t)cur * N, ring + (size_t)prv * N);
            if (m == m) {  // NaN is skipped, as std::max skips it
                slot = cur;
                bits = (unsigned long long)__double_as_longlong(m);  // ordered as the value (m >= 0)
            }
        }
        // the largest change of each sweep among the warp's items (exact: the maximum of the
        // 64-bit patterns, high word first), then one shared atomic per sweep and warp
        const unsigned peers = __match_any_sync(0xffffffffu, slot);
        const unsigned hi = __reduce_max_sync(peers, (unsigned)(bits >> 32));
        const unsigned lo = __reduce_max_sync(peers, (unsigned)(bits >> 32) == hi ? (unsigned)bits : 0u);
        if (slot >= 0 && lane == __ffs(peers) - 1) atomicMax(&maxd[slot], ((unsigned long long)hi << 32) | lo);
    }
}

// The SOR iterations of one inner iteration (SmoothFlowSOR.cpp:156-226) as overlapping
// anti-diagonal sweeps, one CTA.  ring: D slots of (u, v) increments, each N doubles.  Leaves the
// last sweep's increments (the first that converged, max change < 1e-5, or sweep nSOR - 1) in
// (du, dv) and the number of sweeps run in *sweeps.  status: 0, or 1 when the step bound ran out.
__global__ void __launch_bounds__(kSorThreads) k_sor_wavefront(LevelBufs b, double alpha, int nSOR, int D,
                                                               double2* ring, int* sweeps, int* status)
{
    const int W = b.W, H = b.H, ndiag = W + H - 1, lag = 2;
    const size_t N = (size_t)W * H;
    __shared__ long long start[kMaxRing];
    __shared__ unsigned long long maxd[kMaxRing];
    __shared__ int s_done, s_stop, s_next;
    __shared__ int pre[kMaxRing + 1], dd[kMaxRing], ii0[kMaxRing];
    for (size_t p = threadIdx.x; p < N; p += blockDim.x) {
        ring[(size_t)(D - 1) * N + p] = make_double2(0.0, 0.0);
    }
    if (threadIdx.x == 0) { s_done = -1; s_stop = -1; s_next = 0; }
    __syncthreads();
    // every sweep takes ndiag steps and starts within ndiag + lag steps of the previous one
    const long long t_max = (long long)nSOR * (ndiag + lag) + ndiag + 8;
    long long t = 0;
    for (; t < t_max; t++) {
        if (threadIdx.x < 32) {
            // warp 0: the step's new sweep (lane 0), then the step's table
            if (threadIdx.x == 0) {
                const int nx = s_next;
                if (nx < nSOR && (nx == 0 || t >= start[(nx - 1) % D] + lag) && (nx < D || s_done >= nx - D)) {
                    start[nx % D] = t;
                    maxd[nx % D] = 0ull;
                    s_next = nx + 1;
                }
            }
            __syncwarp();
            sor_table(W, H, t, s_done, s_next, start, D, ndiag, pre, dd, ii0);
        }
        __syncthreads();
        const int done = s_done, next = s_next;
        if (s_stop >= 0 || done >= nSOR - 1) break;
        sor_step<false>(b, alpha, done, next, pre, dd, ii0, D, N, ring, maxd, threadIdx.x, blockDim.x);
        __syncthreads();
        if (threadIdx.x == 0) {
            while (s_done + 1 < s_next && t - start[(s_done + 1) % D] == ndiag - 1) {
                s_done++;
                if (__longlong_as_double((long long)maxd[s_done % D]) < 1e-5) {
                    s_stop = s_done;
                    break;
                }
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *sweeps = s_done + 1;
        if (t >= t_max) *status = 1;
    }
    const int last = (s_stop >= 0 ? s_stop : nSOR - 1) % D;
    for (size_t p = threadIdx.x; p < N; p += blockDim.x) {
        const double2 x = ring[(size_t)last * N + p];
        b.du[p] = x.x;
        b.dv[p] = x.y;
    }
}

// The same SOR over a thread-block cluster of C CTAs, for the larger levels: every CTA keeps the
// same sweep schedule (start steps, completed sweeps, the stop), decided by each CTA's thread 0
// from the same inputs; the pixels of each step's diagonals are spread over all the cluster's
// threads; a sweep's maximum change is the largest of the CTAs' partial maxima, read through
// distributed shared memory.  One cluster barrier a step, after the updates (the ring's new values
// are visible to the next step); a ring slot, with its partial-maximum slot, is reused only a step
// after its sweep completed, so no CTA resets a partial maximum another CTA may still be reading.  The order of the updates is the single-CTA kernel's, so the
// flow is the same bit for bit; with more sweeps in flight (D up to kMaxRingC) a step carries more
// independent work.
constexpr int kMaxRingC = 64;

__global__ void __launch_bounds__(kSorThreads) k_sor_wavefront_cluster(LevelBufs b, double alpha, int nSOR, int D,
                                                                       double2* ring, int* sweeps,
                                                                       int* status)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const int W = b.W, H = b.H, ndiag = W + H - 1, lag = 2;
    const size_t N = (size_t)W * H;
    const int G = C * blockDim.x, g = rank * blockDim.x + threadIdx.x;
    __shared__ long long start[kMaxRingC];
    __shared__ long long fin[kMaxRingC];  // the step at which the sweep in each slot completed
    __shared__ unsigned long long maxd[kMaxRingC];
    __shared__ int s_done, s_stop, s_next;
    __shared__ int pre[kMaxRingC + 1], dd[kMaxRingC], ii0[kMaxRingC];
    if (threadIdx.x < kMaxRingC) fin[threadIdx.x] = -1;
    for (size_t p = g; p < N; p += G) {
        ring[(size_t)(D - 1) * N + p] = make_double2(0.0, 0.0);
    }
    if (threadIdx.x == 0) { s_done = -1; s_stop = -1; s_next = 0; }
    __threadfence();
    cl.sync();
    const long long t_max = (long long)nSOR * (ndiag + lag) + ndiag + 8;
    long long t = 0;
    for (; t < t_max; t++) {
        if (threadIdx.x < 32) {
            // warp 0: the step's new sweep (lane 0), then the step's table.  A slot is reused one
            // step after its sweep completed: other CTAs may read its partial maximum during the
            // completion step, up to their next cluster barrier
            if (threadIdx.x == 0) {
                const int nx = s_next;
                if (nx < nSOR && (nx == 0 || t >= start[(nx - 1) % D] + lag) &&
                    (nx < D || (s_done >= nx - D && fin[nx % D] < t - 1))) {
                    start[nx % D] = t;
                    maxd[nx % D] = 0ull;
                    s_next = nx + 1;
                }
            }
            __syncwarp();
            sor_table(W, H, t, s_done, s_next, start, D, ndiag, pre, dd, ii0);
        }
        __syncthreads();
        const int done = s_done, next = s_next;
        if (s_stop >= 0 || done >= nSOR - 1) break;  // the same in every CTA
        sor_step<true>(b, alpha, done, next, pre, dd, ii0, D, N, ring, maxd, g, G);
        cl.sync();  // this step's updates are done and visible in every CTA (release / acquire at cluster scope)
        if (threadIdx.x == 0) {
            while (s_done + 1 < s_next && t - start[(s_done + 1) % D] == ndiag - 1) {
                s_done++;
                fin[s_done % D] = t;
                double mx = 0;
                for (int r = 0; r < C; r++)
                    mx = cmax(mx, __longlong_as_double((long long)*cl.map_shared_rank(&maxd[s_done % D], r)));
                if (mx < 1e-5) {
                    s_stop = s_done;
                    break;
                }
            }
        }
    }
    cl.sync();  // no CTA leaves while another may still read its partial maxima
    if (rank == 0 && threadIdx.x == 0) {
        *sweeps = s_done + 1;
        if (t >= t_max) *status = 1;
    }
    const int last = (s_stop >= 0 ? s_stop : nSOR - 1) % D;
    for (size_t p = g; p < N; p += G) {
        const double2 x = __ldcg(ring + (size_t)last * N + p);
        b.du[p] = x.x;
        b.dv[p] = x.y;
    }
}

// u += du, v += dv (Image::Add, SmoothFlowSOR.cpp:227-228)
__global__ void k_update(LevelBufs b)
{
    const size_t n = (size_t)b.W * b.H;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        b.u[p] = dadd(b.u[p], b.du[p]);
        b.v[p] = dadd(b.v[p], b.dv[p]);
    }
}

}  // namespace f2d
}  // namespace rgbdflow
