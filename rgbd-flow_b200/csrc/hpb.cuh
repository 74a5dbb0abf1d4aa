// hpb.cuh — the HPB regularisation weights (the reference's default, -z 2) on the device.
//
// The reference builds them per pyramid level from the level's colour image and its raw-depth
// pyramid (sceneFlowMultiscale.cpp:79-83, 114-116; sceneFlowWithInit.cpp:48): computeHeuristicPb
// (heuristicProbBoundary.cpp:21-41 -> heuristicBoundaries.cpp:40-358) gives a boundary
// probability to the right and lower neighbour of every pixel, and the weights are 1 - .99 hpb
// (OpticalFlow.cpp:126-131).  The raw-depth pyramid is DepthMapPyramid (depthMapPyramid.cpp:15-91)
// of frame 1's raw depth after recursiveMedianFilterSmallInvalidRegionsUsingColor
// (recursiveMedianFiltering.cpp:127-222).
//
// Every step follows the reference's arithmetic in its own precision (float or double), with each
// operation rounded on its own (__fmul_rn, __dadd_rn, ...: no fused multiply-add the reference's
// x86 build would not make), so that the weights are reproducible against a CPU restatement.
// Three choices stand where the reference's result depends on unpinned library versions (PCL's
// normal estimation, the boost::hash order of the colour-guided fill, exp of a float): normals by
// double-precision PCA with cyclic Jacobi rotations, hole regions filled in the raster order of
// their first pixel (pixels by most valid neighbours, ties in raster order), exp in double.
#pragma once
#include "kernels.cuh"

namespace rgbdflow {

// float / double operations rounded on their own
__device__ __forceinline__ float fmu(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fad(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsb(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double dmu(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dad(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsb(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddv(double a, double b) { return __ddiv_rn(a, b); }

// primesensor::stereoError / stereoErrorRatio (primesensorUtils.cpp:53-64), in double
__device__ __forceinline__ double stereo_err(double z) { return ddv(dmu(z, z), dad(1 / .00285, z)); }
__device__ __forceinline__ double stereo_err_ratio(double z) { return ddv(stereo_err(z), stereo_err(1.0)); }

// ------------------------------------------------------------------------------------------
// Colour-guided fill of small invalid regions of frame 1's raw depth (level 0).
//
// One cooperative launch does it all: the invalid pixels' 4-connected regions by union-find
// (parents always point to a smaller raster index, so a region's root is its first pixel), their
// sizes and pixel lists, then the fill in passes, one warp per region.

// One pair's fill.
template <class T>
struct HpbFill {
    int W, H;
    const PrepItem<T>* src;   // the pair's inputs: colour 1 and raw depth 1 (BGR8 + float, or FP64)
    int fill;                 // 0: no colour-guided fill (the warm start reads the raw depth)
    T* out;                   // level 0 of the raw-depth pyramid (the filled raw depth)
    int* label;               // per pixel: -1 valid, -2 in a region of more than 60 pixels, else the
                              // raster index of its region's first pixel
    int* par;                 // union-find parent of an invalid pixel; at a region's first pixel, then
                              // the cursor of its pixel list
    int* csz;                 // region size, at its first pixel
    uint8_t* done;            // set at a region's first pixel once the region is filled
    int2* regions;            // per region of at most 60 pixels: {first pixel, list start << 6 | size}
    int* px;                  // the regions' pixels, region by region
    int* counts;              // [0] regions listed, [1] pixels listed
};

constexpr int kHpbMaxRegion = 60;  // largest invalid region the fill takes (sceneFlowMultiscale.cpp:81)

// The pair's colour, read as the reference's fill reads it: BGR8 scaled to [0,1], or FP64.
struct HpbColour {
    int kind;
    const uint8_t* bgr;
    const double* im;
    __device__ __forceinline__ double operator()(size_t l, int c) const
    {
        return kind == 0 ? (double)__ldg(bgr + l * 3 + c) / 255.0 : __ldg(im + l * 3 + c);
    }
};

template <class T>
__device__ __forceinline__ double hpb_raw(const PrepItem<T>& s, size_t l)
{
    return s.kind == 0 ? (double)s.depth[0][l] : s.dep_d[0][l];
}

// Root of x: parents strictly decrease, so the walk ends.
__device__ __forceinline__ int uf_find(const int* par, int x)
{
    int p = __ldcg(par + x);
    while (p != x) {
        x = p;
        p = __ldcg(par + x);
    }
    return x;
}

// Joins the regions of a and b: the larger root is hooked under the smaller one.  When another
// thread moved the root first, the join is retried from the root's new parent (which keeps every
// earlier link's region connected).  Bounded: gives up, flagging err, after 2^20 retries.
__device__ __forceinline__ void uf_union(int* par, int a, int b, int* err)
{
    for (int k = 0; k < (1 << 20); k++) {
        a = uf_find(par, a);
        b = uf_find(par, b);
        if (a == b) return;
        if (a < b) { const int t = a; a = b; b = t; }
        const int old = atomicMin(par + a, b);
        if (old == a) return;
        a = old;
    }
    atomicExch(err, 1);
}

// Fills one region (recursiveMedianFilterSmallInvalidRegionsUsingColor's loop over its points):
// repeatedly the pixel with the most valid 3x3 neighbours (ties: smallest raster index) takes the
// average of its valid neighbours weighted by exp(-|colour difference|^2 / .6), in float sums.
// One warp: lane k holds the region's pixels k and k + 32 (q0, q1; -1 past the end) with their
// valid-neighbour counts; lane k < 9 reads the k-th 3x3 neighbour of the pixel being filled, and
// the sums run over them in the reference's row-major order.
template <class T>
__device__ void hpb_fill_region_warp(const HpbFill<T>& f, const HpbColour& col, int q0, int q1, int n)
{
    const int W = f.W, H = f.H, lane = threadIdx.x & 31;
    // depths are read past L1: regions filled by other blocks before this one became ready
    auto dz = [&](int o) { return (double)__ldcg(f.out + o); };
    auto valid_count = [&](int p) {
        const int i = p / W, j = p % W;
        int c = 0;
        for (int ii = max(0, i - 1); ii <= min(H - 1, i + 1); ii++)
            for (int jj = max(0, j - 1); jj <= min(W - 1, j + 1); jj++)
                if (dz(ii * W + jj) > 0) c++;
        return c;
    };
    int c0 = q0 >= 0 ? valid_count(q0) : -1, c1 = q1 >= 0 ? valid_count(q1) : -1;
    for (int step = 0; step < n; step++) {
        // the unfilled pixel with the most valid neighbours, ties to the smaller raster index
        unsigned long long key = 0;
        if (c0 >= 0) key = max(key, ((unsigned long long)(c0 + 1) << 32) | (unsigned)~q0);
        if (c1 >= 0) key = max(key, ((unsigned long long)(c1 + 1) << 32) | (unsigned)~q1);
        for (int o = 16; o; o >>= 1) key = max(key, __shfl_xor_sync(~0u, key, o));
        const int p = (int)~(unsigned)key;
        if (q0 == p) c0 = -1;
        if (q1 == p) c1 = -1;
        const int i = p / W, j = p % W;
        const int i0 = max(0, i - 1), i1 = min(H - 1, i + 1), j0 = max(0, j - 1), j1 = min(W - 1, j + 1);
        const int cols = j1 - j0 + 1, m = (i1 - i0 + 1) * cols;
        int o2 = -1;
        bool v = false;
        float w = 0;
        double term = 0;
        if (lane < m) {
            o2 = (i0 + lane / cols) * W + j0 + lane % cols;
            const double z = dz(o2);
            v = z > 0;
            if (v) {
                double s = 0;
                for (int c = 0; c < 3; c++) {
                    const double d = dsb(col(p, c), col(o2, c));
                    s = dad(s, dmu(d, d));
                }
                w = (float)exp(ddv(-s, .6));
                term = dmu(z, (double)w);
            }
        }
        const unsigned vm = __ballot_sync(~0u, v);
        float zSum = 0, weightSum = 0;
        for (int k = 0; k < m; k++) {
            const double tk = __shfl_sync(~0u, term, k);
            const float wk = __shfl_sync(~0u, w, k);
            if (vm >> k & 1) {
                zSum = (float)dad((double)zSum, tk);
                weightSum = fad(weightSum, wk);
            }
        }
        // each unfilled pixel of the region among the invalid neighbours gains a valid neighbour
        unsigned im = __ballot_sync(~0u, lane < m && !v);
        while (im) {
            const int k = __ffs(im) - 1;
            im &= im - 1;
            const int ok = __shfl_sync(~0u, o2, k);
            if (q0 == ok && c0 >= 0) c0++;
            if (q1 == ok && c1 >= 0) c1++;
        }
        if (lane == 0) f.out[p] = (T)fdv(zSum, weightSum);
        __syncwarp();
    }
}

// The whole fill in one cooperative launch, phases split by grid barriers:
//   1. level 0 of the raw-depth pyramid is the raw depth; each invalid pixel its own region;
//   2. joins with the left and upper invalid neighbours (4-connectivity);
//   3. every invalid pixel's region (its first pixel) and the regions' sizes;
//   4. regions of more than 60 pixels are marked and left unfilled; the others get a list slot;
//   5. the regions' pixel lists;
//   6. passes, one warp per region: a region is filled once every region with a smaller first
//      pixel that touches it (a pixel within one step, diagonals included) is filled, which is
//      the raster order's result.  Bounded by max_passes.
template <class T>
__global__ void __launch_bounds__(128)
k_hpb_fill(const HpbFill<T>* items, int n_items, GridSync* gs, int max_passes, int* status)
{
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gn = gridDim.x * blockDim.x;
    for (int it = 0; it < n_items; it++) {
        const HpbFill<T>& f = items[it];
        const PrepItem<T>& s = *f.src;
        for (int l = gt; l < f.W * f.H; l += gn) {
            const double z = hpb_raw(s, l);
            f.out[l] = (T)z;
            f.done[l] = 0;
            f.csz[l] = 0;
            f.par[l] = (f.fill && !(z > 0)) ? l : -1;
        }
    }
    if (!grid_barrier(gs, gridDim.x)) { report_wait_failure(status); return; }
    for (int it = 0; it < n_items; it++) {
        const HpbFill<T>& f = items[it];
        for (int l = gt; l < f.W * f.H; l += gn) {
            if (__ldcg(f.par + l) < 0) continue;
            if (l % f.W > 0 && __ldcg(f.par + l - 1) >= 0) uf_union(f.par, l, l - 1, &gs->err);
            if (l >= f.W && __ldcg(f.par + l - f.W) >= 0) uf_union(f.par, l, l - f.W, &gs->err);
        }
    }
    if (!grid_barrier(gs, gridDim.x)) { report_wait_failure(status); return; }
    for (int it = 0; it < n_items; it++) {
        const HpbFill<T>& f = items[it];
        for (int l = gt; l < f.W * f.H; l += gn) {
            if (__ldcg(f.par + l) < 0) { f.label[l] = -1; continue; }
            const int r = uf_find(f.par, l);
            f.label[l] = r;
            atomicAdd(f.csz + r, 1);
        }
    }
    if (!grid_barrier(gs, gridDim.x)) { report_wait_failure(status); return; }
    for (int it = 0; it < n_items; it++) {
        const HpbFill<T>& f = items[it];
        for (int l = gt; l < f.W * f.H; l += gn) {
            const int r = __ldcg(f.label + l);
            if (r < 0) continue;
            const int sz = __ldcg(f.csz + r);
            if (sz > kHpbMaxRegion) {
                f.label[l] = -2;
            } else if (r == l) {
                const int slot = atomicAdd(f.counts, 1), start = atomicAdd(f.counts + 1, sz);
                f.regions[slot] = make_int2(l, start << 6 | sz);
                f.par[l] = start;  // the list cursor from here on
            }
        }
    }
    if (!grid_barrier(gs, gridDim.x)) { report_wait_failure(status); return; }
    for (int it = 0; it < n_items; it++) {
        const HpbFill<T>& f = items[it];
        for (int l = gt; l < f.W * f.H; l += gn) {
            const int r = __ldcg(f.label + l);
            if (r >= 0) f.px[atomicAdd(f.par + r, 1)] = l;
        }
    }
    if (!grid_barrier(gs, gridDim.x)) { report_wait_failure(status); return; }

    const int lane = threadIdx.x & 31, gw = gt >> 5, nw = gn >> 5;
    __shared__ int s_left;
    for (int pass = 0; pass < max_passes; pass++) {
        if (threadIdx.x == 0) s_left = 0;
        __syncthreads();
        int pending = 0;
        for (int it = 0; it < n_items; it++) {
            const HpbFill<T>& f = items[it];
            const PrepItem<T>& s = *f.src;
            const HpbColour col{s.kind, s.bgr[0], s.im_d[0]};
            const int nr = __ldcg(f.counts);
            for (int r = gw; r < nr; r += nw) {
                const int2 g = __ldcg(f.regions + r);
                const int rep = g.x, n = g.y & 63, start = g.y >> 6;
                int dn = lane == 0 ? *(volatile uint8_t*)&f.done[rep] : 0;
                if (__shfl_sync(~0u, dn, 0)) continue;
                const int q0 = lane < n ? __ldcg(f.px + start + lane) : -1;
                const int q1 = lane + 32 < n ? __ldcg(f.px + start + lane + 32) : -1;
                bool blocked = false;
                for (int h = 0; h < 2; h++) {
                    const int q = h ? q1 : q0;
                    if (q < 0) continue;
                    const int i = q / f.W, j = q % f.W;
                    for (int ii = max(0, i - 1); ii <= min(f.H - 1, i + 1); ii++)
                        for (int jj = max(0, j - 1); jj <= min(f.W - 1, j + 1); jj++) {
                            const int lb = __ldcg(f.label + ii * f.W + jj);
                            if (lb >= 0 && lb < rep && !*(volatile uint8_t*)&f.done[lb]) blocked = true;
                        }
                }
                if (__any_sync(~0u, blocked)) { pending++; continue; }
                __threadfence();  // the touching regions' depths are read after their done flags
                hpb_fill_region_warp(f, col, q0, q1, n);
                if (lane == 0) {
                    __threadfence();
                    *(volatile uint8_t*)&f.done[rep] = 1;
                }
            }
        }
        if (lane == 0 && pending) atomicAdd(&s_left, pending);
        __syncthreads();
        const int mine = s_left;
        // the number of pending regions over the grid: accumulated in the barrier's pad word
        if (threadIdx.x == 0 && mine) atomicAdd(&gs->pad, mine);
        if (!grid_barrier(gs, gridDim.x)) break;
        const int total = *(volatile int*)&gs->pad;
        if (!grid_barrier(gs, gridDim.x)) break;  // every block has read the total
        if (total == 0) return;
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(&gs->pad, 0);
        if (!grid_barrier(gs, gridDim.x)) break;
    }
    report_wait_failure(status);  // a wait gave up, or regions were left after max_passes
}

// ------------------------------------------------------------------------------------------
// DepthMapPyramid::ConstructPyramid, one level from the previous (depthMapPyramid.cpp:15-91).

template <class T>
struct DepthPyrJob {
    int sW, sH, dW, dH;
    const T* src;
    T* dst;
};

template <class T>
__global__ void k_depth_pyr(const DepthPyrJob<T>* jobs, const Tile* tiles)
{
    const Tile t = tiles[blockIdx.x];
    const DepthPyrJob<T>& jb = jobs[t.item];
    const int j = t.tx * LTW + (threadIdx.x % LTW), i = t.ty * LTH + (threadIdx.x / LTW);
    if (i >= jb.dH || j >= jb.dW) return;
    const int LW = jb.sW, LH = jb.sH;
    auto at = [&](int y, int x) { return (double)jb.src[(size_t)y * LW + x]; };
    // both sampling factors are the ratio of the heights, as in the reference
    const float factor = fdv((float)LH, (float)jb.dH);
    const float maxDZ = .005f;
    T* out = jb.dst + (size_t)i * jb.dW + j;
    const int x = min(LW - 1, max(0, (int)rintf(fmu(factor, (float)j))));
    const int y = min(LH - 1, max(0, (int)rintf(fmu(factor, (float)i))));
    if (!(at(y, x) > 0)) { *out = (T)-1; return; }
    const int X0 = max(0, min(LW - 1, (int)floorf(fmu(factor, (float)j)))), Y0 = max(0, min(LH - 1, (int)floorf(fmu(factor, (float)i))));
    const int X[2] = {X0, min(LW - 1, X0 + 1)}, Y[2] = {Y0, min(LH - 1, Y0 + 1)};
    const int xi = (x == X[0]) ? 0 : 1, yi = (y == Y[0]) ? 0 : 1;
    const double z = at(y, x);
    const double tol = dmu((double)maxDZ, stereo_err_ratio(z));
    float avg = (float)z;
    int n = 1;
    const double c1 = at(Y[yi], X[!xi]), c2 = at(Y[!yi], X[xi]), c3 = at(Y[!yi], X[!xi]);
    if (fabs(dsb(c1, z)) < tol) { avg = fad(avg, (float)c1); n++; }
    if (fabs(dsb(c2, z)) < tol) { avg = fad(avg, (float)c2); n++; }
    if (fabs(dsb(c3, z)) < tol) { avg = fad(avg, (float)c3); n++; }
    if (n > 1) { *out = (T)fdv(avg, (float)n); return; }
    const double zo = c3;
    const double tolo = dmu((double)maxDZ, stereo_err_ratio(zo));
    float avo = (float)zo;
    int m = 1;
    if (fabs(dsb(c1, zo)) < tolo) { avo = fad(avo, (float)c1); m++; }
    if (fabs(dsb(c2, zo)) < tolo) { avo = fad(avo, (float)c2); m++; }
    *out = (m > 1) ? (T)fdv(avo, (float)m) : (T)z;
}

// ------------------------------------------------------------------------------------------
// computeHeuristicPb on one level.

template <class T>
struct HpbItem {
    int W, H;
    float f, cx, cy;       // the wrapper's camera: Kinect intrinsics scaled to the level (heuristicProbBoundary.cpp:24-29)
    const T* col[3];       // the level's colour planes (B, G, R in [0, 1])
    const T* z;            // the level of the raw-depth pyramid (<= 0 invalid)
    T* rh;                 // out: 1 - .99 hpb to the right neighbour (0 on the last column)
    T* rv;                 // out: to the lower neighbour (0 on the last row)
    // scratch, W x H unless noted
    float* nrm[3];         // normals (0 where invalid)
    unsigned* nval;        // the normal counts as valid (finite, or unit length)
    int* rad;              // half-disk radius
    float* pre[6];         // per row: the sum of the channel before each pixel (colour R, G, B, normal x, y, z)
    unsigned* pre_v;       // the same of nval
    float* ii[6];          // integral images, (W + 1) x (H + 1)
    unsigned* ii_v;
    float* feat[4];        // colour / normal contrast across the left (H) and upper (V) edge: colH, colV, norH, norV
    float* bp[2];          // boundary probability to the right / lower neighbour before suppression
};

// the wrapper's 8-bit colour: channels reversed, 255 * value truncated, then / 255 (channel 0 = R)
template <class T>
__device__ __forceinline__ float hpb_colour(const HpbItem<T>& it, size_t l, int k)
{
    const unsigned char px = (unsigned char)(255.0 * (double)it.col[2 - k][l]);
    return (float)((double)px / 255.0);
}

// depth_to_cloud (depth_to_cloud_lib.ipp:35-50) of one pixel
__device__ __forceinline__ void hpb_point(float d, int r, int c, float cx, float cy, float f, float* p)
{
    p[0] = fdv(fmu(fsb((float)c, cx), d), f);
    p[1] = fdv(fmu(fsb((float)r, cy), d), f);
    p[2] = d;
}

// 3x3 symmetric eigen-solve by cyclic Jacobi rotations in double: the unit eigenvector of the
// smallest eigenvalue.
__device__ void hpb_smallest_eigvec(double a[3][3], double n[3])
{
    double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int sweep = 0; sweep < 64; sweep++) {
        const double off = dad(dad(dmu(a[0][1], a[0][1]), dmu(a[0][2], a[0][2])), dmu(a[1][2], a[1][2]));
        if (off < 1e-300) break;
#pragma unroll
        for (int pq = 0; pq < 3; pq++) {
            const int p = pq < 2 ? 0 : 1, q = pq == 0 ? 1 : 2;
            if (a[p][q] == 0) continue;
            const double theta = ddv(dsb(a[q][q], a[p][p]), dmu(2.0, a[p][q]));
            const double t = ddv(theta >= 0 ? 1.0 : -1.0, dad(fabs(theta), __dsqrt_rn(dad(dmu(theta, theta), 1.0))));
            const double c = ddv(1.0, __dsqrt_rn(dad(dmu(t, t), 1.0))), sn = dmu(t, c);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const double akp = a[k][p], akq = a[k][q];
                a[k][p] = dsb(dmu(c, akp), dmu(sn, akq));
                a[k][q] = dad(dmu(sn, akp), dmu(c, akq));
            }
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const double apk = a[p][k], aqk = a[q][k];
                a[p][k] = dsb(dmu(c, apk), dmu(sn, aqk));
                a[q][k] = dad(dmu(sn, apk), dmu(c, aqk));
            }
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const double vkp = v[k][p], vkq = v[k][q];
                v[k][p] = dsb(dmu(c, vkp), dmu(sn, vkq));
                v[k][q] = dad(dmu(sn, vkp), dmu(c, vkq));
            }
        }
    }
    int m = 0;
    if (a[1][1] < a[m][m]) m = 1;
    if (a[2][2] < a[m][m]) m = 2;
    const double len = __dsqrt_rn(dad(dad(dmu(v[0][m], v[0][m]), dmu(v[1][m], v[1][m])), dmu(v[2][m], v[2][m])));
    for (int k = 0; k < 3; k++) n[k] = ddv(v[k][m], len);
}

// Organised normals with a 9 x 9 window (setOrganizedNormals, cloudNormals.ipp:131-207 and
// 395-506): neighbours whose depth is within .05 * stereoErrorRatio of the centre's, at least 27
// of them; turned towards the camera.  Also the normal's validity and the half-disk radius.
constexpr int kHpbK = 4;
template <class T>
__global__ void __launch_bounds__(LTW * LTH)
k_hpb_normals(const HpbItem<T>* items, const Tile* tiles)
{
    constexpr int RH = LTH + 2 * kHpbK, RW = LTW + 2 * kHpbK;
    __shared__ float sz[RH][RW];
    const Tile t = tiles[blockIdx.x];
    const HpbItem<T>& it = items[t.item];
    const int W = it.W, H = it.H;
    const int i0 = t.ty * LTH, j0 = t.tx * LTW;
    for (int e = threadIdx.x; e < RH * RW; e += LTW * LTH) {
        const int r = e / RW, c = e % RW, gi = i0 - kHpbK + r, gj = j0 - kHpbK + c;
        sz[r][c] = (gi >= 0 && gi < H && gj >= 0 && gj < W) ? (float)it.z[(size_t)gi * W + gj] : 0.f;
    }
    __syncthreads();
    const int tx = threadIdx.x % LTW, ty = threadIdx.x / LTW, i = i0 + ty, j = j0 + tx;
    if (i >= H || j >= W) return;
    const size_t o = (size_t)i * W + j;
    const float zc = sz[ty + kHpbK][tx + kHpbK];
    float n3[3] = {0, 0, 0};
    if (zc > 0) {
        const double tol = dmu((double).05f, stereo_err_ratio((double)zc));
        const int y0 = max(0, i - kHpbK), y1 = min(H - 1, i + kHpbK), x0 = max(0, j - kHpbK), x1 = min(W - 1, j + kHpbK);
        int cnt = 0;
        double m[3] = {0, 0, 0};
        for (int yy = y0; yy <= y1; yy++)
            for (int xx = x0; xx <= x1; xx++) {
                const float z2 = sz[yy - i0 + kHpbK][xx - j0 + kHpbK];
                if (!((double)fabsf(fsb(zc, z2)) < tol)) continue;
                float p[3];
                hpb_point(z2, yy, xx, it.cx, it.cy, it.f, p);
                m[0] = dad(m[0], (double)p[0]); m[1] = dad(m[1], (double)p[1]); m[2] = dad(m[2], (double)p[2]);
                cnt++;
            }
        if (cnt >= 27) {  // max(6, 81 / 3)
            for (int k = 0; k < 3; k++) m[k] = ddv(m[k], (double)cnt);
            double a[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (int yy = y0; yy <= y1; yy++)
                for (int xx = x0; xx <= x1; xx++) {
                    const float z2 = sz[yy - i0 + kHpbK][xx - j0 + kHpbK];
                    if (!((double)fabsf(fsb(zc, z2)) < tol)) continue;
                    float p[3];
                    hpb_point(z2, yy, xx, it.cx, it.cy, it.f, p);
                    const double d[3] = {dsb((double)p[0], m[0]), dsb((double)p[1], m[1]), dsb((double)p[2], m[2])};
#pragma unroll
                    for (int r = 0; r < 3; r++)
#pragma unroll
                        for (int c = 0; c < 3; c++) a[r][c] = dad(a[r][c], dmu(d[r], d[c]));
                }
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) a[r][c] = ddv(a[r][c], (double)cnt);
            double n[3];
            hpb_smallest_eigvec(a, n);
            if (isfinite(n[0]) && isfinite(n[1]) && isfinite(n[2])) {
                float pc[3];
                hpb_point(zc, i, j, it.cx, it.cy, it.f, pc);
                const double cosv = -dad(dad(dmu((double)pc[0], n[0]), dmu((double)pc[1], n[1])), dmu((double)pc[2], n[2]));
                if (cosv < 0) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
                n3[0] = (float)n[0]; n3[1] = (float)n[1]; n3[2] = (float)n[2];
            }
        }
    }
    for (int k = 0; k < 3; k++) it.nrm[k][o] = n3[k];
    const float sq = fad(fad(fmu(n3[0], n3[0]), fmu(n3[1], n3[1])), fmu(n3[2], n3[2]));
    it.nval[o] = (!isfinite(n3[0]) || !isfinite(n3[1]) || !isfinite(n3[2]) || (double)fabsf(sq - 1.f) < 1e-4) ? 1u : 0u;
    it.rad[o] = zc > 0 ? max(1, min(5, (int)rintf(fdv(fmu(it.f, .02f), zc)))) : 5;
}

// Integral images (computeIntegralImage, halfDiskFeatures.ipp:102-154) in the reference's float
// order: ii(i + 1, j + 1) = (ii(i, j + 1) + sum of row i before j) + v(i, j).  Pass 1, one thread
// per (row, channel): the row sums before each pixel.  Pass 2, one thread per (column, channel):
// the recurrence down the column.  Channels 0..2 colour (R, G, B), 3..5 normal, 6 normal validity.
template <class T>
__device__ __forceinline__ float hpb_chan(const HpbItem<T>& it, size_t l, int c)
{
    return c < 3 ? hpb_colour(it, l, c) : it.nrm[c - 3][l];
}

// first[k]: the first global thread of item k (first[n_items]: the total)
template <class T>
__global__ void k_hpb_rowsum(const HpbItem<T>* items, const int* first, int n_items)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= first[n_items]) return;
    int k = 0;
    while (k + 1 < n_items && g >= first[k + 1]) k++;
    const HpbItem<T>& it = items[k];
    const int rel = g - first[k];
    if (rel < 0 || rel >= 7 * it.H) return;
    const int i = rel / 7, c = rel % 7;
    const size_t base = (size_t)i * it.W;
    // the loads of 32 pixels are issued together; the sums stay in the reference's order
    constexpr int B = 32;
    if (c == 6) {
        unsigned s = 0;
        for (int j0 = 0; j0 < it.W; j0 += B) {
            unsigned v[B];
#pragma unroll
            for (int u = 0; u < B; u++) v[u] = j0 + u < it.W ? it.nval[base + j0 + u] : 0u;
#pragma unroll
            for (int u = 0; u < B; u++)
                if (j0 + u < it.W) { it.pre_v[base + j0 + u] = s; s += v[u]; }
        }
    } else {
        float s = 0;
        for (int j0 = 0; j0 < it.W; j0 += B) {
            float v[B];
#pragma unroll
            for (int u = 0; u < B; u++) v[u] = j0 + u < it.W ? hpb_chan(it, base + j0 + u, c) : 0.f;
#pragma unroll
            for (int u = 0; u < B; u++)
                if (j0 + u < it.W) { it.pre[c][base + j0 + u] = s; s = fad(s, v[u]); }
        }
    }
}

template <class T>
__global__ void k_hpb_colsum(const HpbItem<T>* items, const int* first, int n_items)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= first[n_items]) return;
    int k = 0;
    while (k + 1 < n_items && g >= first[k + 1]) k++;
    const HpbItem<T>& it = items[k];
    const int rel = g - first[k];
    if (rel < 0 || rel >= 7 * (it.W + 1)) return;
    const int W1 = it.W + 1;
    const int c = rel / W1, jj = rel % W1;  // a warp: 32 columns of one channel; jj = 0 the zero column
    // the loads of 16 rows are issued together; the sums stay in the reference's order
    constexpr int B = 16;
    if (c == 6) {
        unsigned* ii = it.ii_v;
        ii[jj] = 0;
        unsigned a = 0;
        for (int i0 = 0; i0 < it.H; i0 += B) {
            unsigned p[B], v[B];
#pragma unroll
            for (int u = 0; u < B; u++) {
                const bool in = jj > 0 && i0 + u < it.H;
                const size_t l = in ? (size_t)(i0 + u) * it.W + jj - 1 : 0;
                p[u] = in ? it.pre_v[l] : 0u;
                v[u] = in ? it.nval[l] : 0u;
            }
#pragma unroll
            for (int u = 0; u < B; u++)
                if (i0 + u < it.H) {
                    if (jj > 0) a = (a + p[u]) + v[u];
                    ii[(size_t)(i0 + u + 1) * W1 + jj] = a;
                }
        }
    } else {
        float* ii = it.ii[c];
        ii[jj] = 0;
        float a = 0;
        for (int i0 = 0; i0 < it.H; i0 += B) {
            float p[B], v[B];
#pragma unroll
            for (int u = 0; u < B; u++) {
                const bool in = jj > 0 && i0 + u < it.H;
                const size_t l = in ? (size_t)(i0 + u) * it.W + jj - 1 : 0;
                p[u] = in ? it.pre[c][l] : 0.f;
                v[u] = in ? hpb_chan(it, l, c) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < B; u++)
                if (i0 + u < it.H) {
                    if (jj > 0) a = fad(fad(a, p[u]), v[u]);
                    ii[(size_t)(i0 + u + 1) * W1 + jj] = a;
                }
        }
    }
}

// Half-disk contrasts across each pixel's left and upper edge (heuristicBoundaries.cpp:101-222):
// colour distance of the two half-disk means, normal disagreement of the two half-disk mean normals
// weighted by the convexity of the edge.
template <class T>
__global__ void k_hpb_halfdisk(const HpbItem<T>* items, const Tile* tiles)
{
    const Tile t = tiles[blockIdx.x];
    const HpbItem<T>& it = items[t.item];
    const int j = t.tx * LTW + (threadIdx.x % LTW), i = t.ty * LTH + (threadIdx.x / LTW);
    const int W = it.W, H = it.H;
    if (i >= H || j >= W) return;
    const size_t o = (size_t)i * W + j;
    const int W1 = W + 1;
    const int hw = it.rad[o];
    const int xmin = max(0, j - hw), xmax = min(W - 1, j + hw - 1);
    const int ymin = max(0, i - hw), ymax = min(H - 1, i + hw - 1);
    auto IF = [&](int c, int y, int x) { return it.ii[c][(size_t)(y + 1) * W1 + (x + 1)]; };
    auto IV = [&](int y, int x) { return it.ii_v[(size_t)(y + 1) * W1 + (x + 1)]; };
    // a box sum A - B - C + D, left to right, with the reference's corner order per half-disk
    // (A, B, C, D as (y, x) pairs)
    auto boxf = [&](int c, const int* q) {
        return fad(fsb(fsb(IF(c, q[0], q[1]), IF(c, q[2], q[3])), IF(c, q[4], q[5])), IF(c, q[6], q[7]));
    };
    auto boxv = [&](const int* q) { return IV(q[0], q[1]) - IV(q[2], q[3]) - IV(q[4], q[5]) + IV(q[6], q[7]); };
    auto dot = [](const float* a, const float* b) { return fad(fad(fmu(a[0], b[0]), fmu(a[1], b[1])), fmu(a[2], b[2])); };
    auto normalize3 = [](float* v) {
        const float n = sqrtf(fad(fad(fmu(v[0], v[0]), fmu(v[1], v[1])), fmu(v[2], v[2])));
        if (n > 0)
            for (int k = 0; k < 3; k++) v[k] = fdv(v[k], n);
    };
    const float d0 = (float)it.z[o];
    float pc[3];
    hpb_point(d0, i, j, it.cx, it.cy, it.f, pc);
    float colH = 0, colV = 0, norH = 0, norV = 0;
    for (int dir = 0; dir < 2; dir++) {
        if (dir == 0 ? j == 0 : i == 0) continue;
        // half-disks 0 and 1: dir 0 left [xmin, j - 1] / right [j, xmax] over rows [ymin, ymax];
        // dir 1 upper [ymin, i - 1] / lower [i, ymax] over columns [xmin, xmax]
        // (heuristicBoundaries.cpp's H0 / H1 / V0 / V1 box sums, corners in its order)
        int q0[8], q1[8];
        float s0, s1;
        if (dir == 0) {
            const int a[8] = {ymax, j - 1, ymin - 1, j - 1, ymax, xmin - 1, ymin - 1, xmin - 1};
            const int b[8] = {ymax, xmax, ymax, j - 1, ymin - 1, xmax, ymin - 1, j - 1};
            for (int e = 0; e < 8; e++) { q0[e] = a[e]; q1[e] = b[e]; }
            s0 = (float)((j - xmin) * (ymax - ymin + 1));
            s1 = (float)((xmax - j + 1) * (ymax - ymin + 1));
        } else {
            const int a[8] = {i - 1, xmax, i - 1, xmin - 1, ymin - 1, xmax, ymin - 1, xmin - 1};
            const int b[8] = {ymax, xmax, i - 1, xmax, ymax, xmin - 1, i - 1, xmin - 1};
            for (int e = 0; e < 8; e++) { q0[e] = a[e]; q1[e] = b[e]; }
            s0 = (float)((xmax - xmin + 1) * (i - ymin));
            s1 = (float)((xmax - xmin + 1) * (ymax - i + 1));
        }
        float acc = 0;
        for (int k = 0; k < 3; k++) {
            const float d = fsb(fdv(boxf(k, q1), s1), fdv(boxf(k, q0), s0));
            acc = fad(acc, fmu(d, d));
        }
        const float cd = sqrtf(acc);
        float n0[3], n1[3];
        for (int k = 0; k < 3; k++) { n0[k] = boxf(3 + k, q0); n1[k] = boxf(3 + k, q1); }
        normalize3(n0);
        normalize3(n1);
        const unsigned v0 = boxv(q0), v1 = boxv(q1);
        float nd = (min(v0, v1) < 3u) ? 0.f : (float)(.5 * (double)(1.f - dot(n0, n1)));
        if (min(v0, v1) > 3u) {
            const int ai = dir == 0 ? i : i - 1, aj = dir == 0 ? j - 1 : j;
            float pa[3];
            hpb_point((float)it.z[(size_t)ai * W + aj], ai, aj, it.cx, it.cy, it.f, pa);
            float dx[3] = {fsb(pa[0], pc[0]), fsb(pa[1], pc[1]), fsb(pa[2], pc[2])};
            normalize3(dx);
            const float mdx[3] = {-dx[0], -dx[1], -dx[2]};
            const double convexity = dad((double)fdv(fad(dot(n0, dx), dot(n1, mdx)), 4.f), .5);
            nd = (float)dmu((double)nd, dsb(1.0, convexity));
        }
        if (dir == 0) { colH = cd; norH = nd; } else { colV = cd; norV = nd; }
    }
    it.feat[0][o] = colH;
    it.feat[1][o] = colV;
    it.feat[2][o] = norH;
    it.feat[3][o] = norV;
}

// Boundary probabilities (heuristicBoundaries.cpp:223-293): from the depth step where both depths
// are valid, from the run of invalid depth behind the edge where one is not, from colour where
// either is invalid, and from the normals; the largest wins; edges on the image border's
// second-to-last row / column are cleared (the reference's edge hack).
template <class T>
__global__ void k_hpb_prob(const HpbItem<T>* items, const Tile* tiles)
{
    const Tile t = tiles[blockIdx.x];
    const HpbItem<T>& it = items[t.item];
    const int j = t.tx * LTW + (threadIdx.x % LTW), i = t.ty * LTH + (threadIdx.x / LTW);
    const int W = it.W, H = it.H;
    if (i >= H || j >= W) return;
    const size_t o = (size_t)i * W + j;
    const float depthSigma = .02f, colSigma = .7f, normSigma = .4f;
    auto dep = [&](int y, int x) { return (float)it.z[(size_t)y * W + x]; };
    auto prob1 = [](float v, float sig) {
        const float q = fdv(v, sig);
        return (float)dsb(1.0, exp(-(double)fmu(q, q)));
    };
    for (int k = 0; k < 2; k++) {
        if (k == 0 ? j >= W - 1 : i >= H - 1) { it.bp[k][o] = 0; continue; }
        const size_t o2 = k == 0 ? o + 1 : o + W;
        const float z1 = dep(i, j), z2 = k == 0 ? dep(i, j + 1) : dep(i + 1, j);
        const float dcol = it.feat[k][o2], dnorm = it.feat[2 + k][o2];
        float colProb, depthProb;
        if (fmaxf(z1, z2) <= 0) {
            depthProb = 0;
            colProb = prob1(dcol, colSigma);
        } else if (fminf(z1, z2) <= 0) {
            // the length of the run of invalid depth: the reference indexes its direction table
            // (0 left, 1 up, 2 right, 3 down) with the edge index k, so its walk starts and moves as
            // written here
            const int di[4] = {0, -1, 0, 1}, dj[4] = {-1, 0, 1, 0};
            const int dir = (z1 <= 0) ? (k + 2) % 4 : k;
            int ii = (z1 <= 0) ? i : i + di[k], jj = (z1 <= 0) ? j : j + dj[k];
            unsigned size = 0;
            while (jj >= 0 && jj < W && ii >= 0 && ii < H && dep(ii, jj) <= 0) {
                size++;
                ii += di[dir];
                jj += dj[dir];
            }
            const bool oob = (jj < 0 || jj >= W || ii < 0 || ii >= H);
            if (oob) depthProb = 0;
            else {
                const double a = (double)fminf(1.0f, fdv((float)size, 30.f));
                depthProb = (float)dad(dmu(dsb(1.0, a), .2), dmu(a, 1.0));
            }
            colProb = prob1(dcol, colSigma);
        } else {
            const float dz = (float)ddv((double)fabsf(fsb(z1, z2)), stereo_err_ratio((double)fminf(z1, z2)));
            depthProb = prob1(dz, depthSigma);
            colProb = 0;
        }
        const float normProb = prob1(dnorm, normSigma);
        float v = fmaxf(depthProb, fmaxf(colProb, fmaxf(0.0f, normProb)));
        if (((i == 0 || i == H - 2) && k == 1) || ((j == 0 || j == W - 2) && k == 0)) v = 0;
        it.bp[k][o] = v;
    }
}

// Non-maximum suppression along each edge direction within the pixel's radius
// (heuristicBoundaries.cpp:298-340), then the weights 1 - .99 hpb (OpticalFlow.cpp:126-131).
template <class T>
__global__ void k_hpb_nms(const HpbItem<T>* items, const Tile* tiles)
{
    const Tile t = tiles[blockIdx.x];
    const HpbItem<T>& it = items[t.item];
    const int j = t.tx * LTW + (threadIdx.x % LTW), i = t.ty * LTH + (threadIdx.x / LTW);
    const int W = it.W, H = it.H;
    if (i >= H || j >= W) return;
    const size_t o = (size_t)i * W + j;
    const int hw = it.rad[o];
    int mi = -1;
    for (int k = max(0, i - hw); k <= min(H - 1, i + hw); k++)
        if (mi < 0 || it.bp[1][(size_t)k * W + j] > it.bp[1][(size_t)mi * W + j]) mi = k;
    const float down = mi != i ? 0.f : it.bp[1][o];
    mi = -1;
    for (int k = max(0, j - hw); k <= min(W - 1, j + hw); k++)
        if (mi < 0 || it.bp[0][(size_t)i * W + k] > it.bp[0][(size_t)i * W + mi]) mi = k;
    const float right = mi != j ? 0.f : it.bp[0][o];
    it.rh[o] = j < W - 1 ? (T)dsb(1.0, dmu((double)right, .99)) : (T)0;
    it.rv[o] = i < H - 1 ? (T)dsb(1.0, dmu((double)down, .99)) : (T)0;
}

}  // namespace rgbdflow
