// Correlation lookups of the DROID update operator — drop-in for the
// reference's droid_net_ext (vipe csrc/droid_net_ext/droid.cpp:75-81):
//
//   corr_index_forward / backward   bilinear radius-r lookup in a materialised
//       volume (correlation_kernels.cu:22-158)
//   altcorr_forward / backward      the same lookup computed on the fly from
//       feature maps (altcorr_kernel.cu:26-138, 242-366)
//   altcorr_index_forward           indexed, multi-level on-the-fly lookup
//       (altcorr_kernel.cu:140-240, 394-424)
//   corr_index_coords_backward, altcorr_index_backward
//                                   adjoints the reference does not have: the
//       coordinate gradient of the volume lookup and the map / pyramid /
//       coordinate gradients of the indexed lookup
//
// Conventions kept from the reference: taps at floor(x) - r + i, floor(y) - r
// + j for i, j in [0, 2r+1]; output channel = i * (2r+1) + j (x-offset major);
// bilinear weights from the fractional parts; zeros outside the map; pyramid
// level l looks up at coords / 2^l.  Accumulation is in FP32 (FP64 for double
// inputs) and each output is written once.
//
// On-the-fly kernels: one warp per (pixel, sample), one tap per lane (a window
// of (2r+2)^2 = 64 taps for r = 3 is two taps per lane); each lane computes the
// full C-channel dot product of its tap against the pixel's feature vector
// (staged once in shared memory and reused for every pyramid level), then the
// bilinear combination is done with warp shuffles.  Output tiles of 32 pixels
// are staged in shared memory and written as coalesced rows.

#include "common.cuh"
#include "corr_window.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <climits>
#include <type_traits>

namespace vipe {
namespace corr {

template <typename T>
struct Acc {
    using type = float;
};
template <>
struct Acc<double> {
    using type = double;
};

// ---------------------------------------------------------------- materialised-volume lookup

template <typename T>
__global__ void corr_index_fwd_kernel(const T* __restrict__ vol, const float* __restrict__ coords, T* __restrict__ out,
                                      int B, int h1, int w1, int h2, int w2, int r) {
    using A = typename Acc<T>::type;
    const int64_t HW1 = (int64_t)h1 * w1;
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= B * HW1) return;
    const int n = (int)(idx / HW1);
    const int64_t pix = idx % HW1;
    const float x0 = coords[((int64_t)n * 2 + 0) * HW1 + pix];
    const float y0 = coords[((int64_t)n * 2 + 1) * HW1 + pix];
    const float fx0 = floorf(x0), fy0 = floorf(y0);
    const A dx = (A)(x0 - fx0), dy = (A)(y0 - fy0);
    const int bx = window_origin(fx0, r), by = window_origin(fy0, r);
    const int rd = 2 * r + 1;
    const T* plane = vol + ((int64_t)n * HW1 + pix) * ((int64_t)h2 * w2);
    T* o = out + (int64_t)n * rd * rd * HW1 + pix;
    for (int i = 0; i < rd; i++) {
        for (int j = 0; j < rd; j++) {
            // out[i][j] = bilinear at (bx + i + dx, by + j + dy)
            A v = 0;
            const int xa = bx + i, ya = by + j;
            if (inb(ya, xa, h2, w2)) v += (1 - dx) * (1 - dy) * (A)to_f(plane[(int64_t)ya * w2 + xa]);
            if (inb(ya, xa + 1, h2, w2)) v += dx * (1 - dy) * (A)to_f(plane[(int64_t)ya * w2 + xa + 1]);
            if (inb(ya + 1, xa, h2, w2)) v += (1 - dx) * dy * (A)to_f(plane[(int64_t)(ya + 1) * w2 + xa]);
            if (inb(ya + 1, xa + 1, h2, w2)) v += dx * dy * (A)to_f(plane[(int64_t)(ya + 1) * w2 + xa + 1]);
            o[(int64_t)(i * rd + j) * HW1] = from_f<T>((float)v);
        }
    }
}

template <>
__global__ void corr_index_fwd_kernel<double>(const double* __restrict__ vol, const float* __restrict__ coords,
                                              double* __restrict__ out, int B, int h1, int w1, int h2, int w2, int r) {
    const int64_t HW1 = (int64_t)h1 * w1;
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= B * HW1) return;
    const int n = (int)(idx / HW1);
    const int64_t pix = idx % HW1;
    const float x0 = coords[((int64_t)n * 2 + 0) * HW1 + pix];
    const float y0 = coords[((int64_t)n * 2 + 1) * HW1 + pix];
    const float fx0 = floorf(x0), fy0 = floorf(y0);
    const double dx = (double)(x0 - fx0), dy = (double)(y0 - fy0);
    const int bx = window_origin(fx0, r), by = window_origin(fy0, r);
    const int rd = 2 * r + 1;
    const double* plane = vol + ((int64_t)n * HW1 + pix) * ((int64_t)h2 * w2);
    double* o = out + (int64_t)n * rd * rd * HW1 + pix;
    for (int i = 0; i < rd; i++)
        for (int j = 0; j < rd; j++) {
            double v = 0;
            const int xa = bx + i, ya = by + j;
            if (inb(ya, xa, h2, w2)) v += (1 - dx) * (1 - dy) * plane[(int64_t)ya * w2 + xa];
            if (inb(ya, xa + 1, h2, w2)) v += dx * (1 - dy) * plane[(int64_t)ya * w2 + xa + 1];
            if (inb(ya + 1, xa, h2, w2)) v += (1 - dx) * dy * plane[(int64_t)(ya + 1) * w2 + xa];
            if (inb(ya + 1, xa + 1, h2, w2)) v += dx * dy * plane[(int64_t)(ya + 1) * w2 + xa + 1];
            o[(int64_t)(i * rd + j) * HW1] = v;
        }
}

template <typename T>
__global__ void corr_index_fwd_r3_kernel(const T* __restrict__ vol, const float* __restrict__ coords,
                                         T* __restrict__ out, int B, int h1, int w1, int h2, int w2) {
    const int64_t HW1 = (int64_t)h1 * w1;
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= B * HW1) return;
    const int n = (int)(idx / HW1);
    const int64_t pix = idx % HW1;
    const float x0 = coords[((int64_t)n * 2 + 0) * HW1 + pix];
    const float y0 = coords[((int64_t)n * 2 + 1) * HW1 + pix];
    const float fx0 = floorf(x0), fy0 = floorf(y0);
    // far-away or non-finite coordinates read only zeros (and their weights are zeroed too,
    // so the output is 0 rather than 0 * NaN)
    const bool near = fabsf(x0) < 1e6f && fabsf(y0) < 1e6f;
    const float dx = near ? x0 - fx0 : 0.f, dy = near ? y0 - fy0 : 0.f;
    const int bx = near ? window_origin(fx0, 3) : -64, by = near ? window_origin(fy0, 3) : -64;
    const T* plane = vol + ((int64_t)n * HW1 + pix) * ((int64_t)h2 * w2);
    float t[8][8];  // [y offset][x offset]
#pragma unroll
    for (int j = 0; j < 8; j++) window_row8<T>(plane, h2, w2, by + j, bx, t[j]);
    T* o = out + (int64_t)n * 49 * HW1 + pix;
#pragma unroll
    for (int i = 0; i < 7; i++)
#pragma unroll
        for (int j = 0; j < 7; j++) {
            float v = (1 - dx) * (1 - dy) * t[j][i];
            v += dx * (1 - dy) * t[j][i + 1];
            v += (1 - dx) * dy * t[j + 1][i];
            v += dx * dy * t[j + 1][i + 1];
            o[(int64_t)(i * 7 + j) * HW1] = from_f<T>(v);
        }
}

// volume_grad must be zero on entry; each pixel owns its (h2, w2) plane, so the
// scatter has no conflicts and is deterministic
template <typename T>
__global__ void corr_index_bwd_kernel(const float* __restrict__ coords, const T* __restrict__ g,
                                      T* __restrict__ vgrad, int B, int h1, int w1, int h2, int w2, int r) {
    using A = typename Acc<T>::type;
    const int64_t HW1 = (int64_t)h1 * w1;
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= B * HW1) return;
    const int n = (int)(idx / HW1);
    const int64_t pix = idx % HW1;
    const float x0 = coords[((int64_t)n * 2 + 0) * HW1 + pix];
    const float y0 = coords[((int64_t)n * 2 + 1) * HW1 + pix];
    const float fx0 = floorf(x0), fy0 = floorf(y0);
    const A dx = (A)(x0 - fx0), dy = (A)(y0 - fy0);
    const int bx = window_origin(fx0, r), by = window_origin(fy0, r);
    const int rd = 2 * r + 1;
    T* plane = vgrad + ((int64_t)n * HW1 + pix) * ((int64_t)h2 * w2);
    const T* go = g + (int64_t)n * rd * rd * HW1 + pix;
    for (int i = 0; i <= rd; i++)
        for (int j = 0; j <= rd; j++) {
            const int x1 = bx + i, y1 = by + j;
            if (!inb(y1, x1, h2, w2)) continue;
            A s = 0;
            if (i > 0 && j > 0) s += (A)to_f(go[(int64_t)((i - 1) * rd + (j - 1)) * HW1]) * dx * dy;
            if (i > 0 && j < rd) s += (A)to_f(go[(int64_t)((i - 1) * rd + j) * HW1]) * dx * (1 - dy);
            if (i < rd && j > 0) s += (A)to_f(go[(int64_t)(i * rd + (j - 1)) * HW1]) * (1 - dx) * dy;
            if (i < rd && j < rd) s += (A)to_f(go[(int64_t)(i * rd + j) * HW1]) * (1 - dx) * (1 - dy);
            plane[(int64_t)y1 * w2 + x1] = from_f<T>((float)s);
        }
}

template <>
__global__ void corr_index_bwd_kernel<double>(const float* __restrict__ coords, const double* __restrict__ g,
                                              double* __restrict__ vgrad, int B, int h1, int w1, int h2, int w2,
                                              int r) {
    const int64_t HW1 = (int64_t)h1 * w1;
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= B * HW1) return;
    const int n = (int)(idx / HW1);
    const int64_t pix = idx % HW1;
    const float x0 = coords[((int64_t)n * 2 + 0) * HW1 + pix];
    const float y0 = coords[((int64_t)n * 2 + 1) * HW1 + pix];
    const float fx0 = floorf(x0), fy0 = floorf(y0);
    const double dx = x0 - fx0, dy = y0 - fy0;
    const int bx = window_origin(fx0, r), by = window_origin(fy0, r);
    const int rd = 2 * r + 1;
    double* plane = vgrad + ((int64_t)n * HW1 + pix) * ((int64_t)h2 * w2);
    const double* go = g + (int64_t)n * rd * rd * HW1 + pix;
    for (int i = 0; i <= rd; i++)
        for (int j = 0; j <= rd; j++) {
            const int x1 = bx + i, y1 = by + j;
            if (!inb(y1, x1, h2, w2)) continue;
            double s = 0;
            if (i > 0 && j > 0) s += go[(int64_t)((i - 1) * rd + (j - 1)) * HW1] * dx * dy;
            if (i > 0 && j < rd) s += go[(int64_t)((i - 1) * rd + j) * HW1] * dx * (1 - dy);
            if (i < rd && j > 0) s += go[(int64_t)(i * rd + (j - 1)) * HW1] * (1 - dx) * dy;
            if (i < rd && j < rd) s += go[(int64_t)(i * rd + j) * HW1] * (1 - dx) * (1 - dy);
            plane[(int64_t)y1 * w2 + x1] = s;
        }
}

// Exact coordinate gradient of the lookup (the reference's CorrSampler returns
// none): with taps v00 = V[y, x], v10 = V[y, x+1], v01 = V[y+1, x], v11 = V[y+1, x+1]
// of output (i, j),  d/dx = (1-dy)(v10 - v00) + dy (v11 - v01),
//                    d/dy = (1-dx)(v01 - v00) + dx (v11 - v10),
// contracted with the output gradient over the (2r+1)^2 channels.  The floor is
// piecewise constant, so the derivative is the one-sided one inside each cell.
// One thread per pixel; the (2r+2)^2 window of its plane is read once.
template <typename A, typename T>
__device__ __forceinline__ A load_acc(const T* p) {
    return (A)to_f(*p);
}
template <>
__device__ __forceinline__ double load_acc<double, double>(const double* p) {
    return *p;
}

template <typename T>
__global__ void corr_index_coords_bwd_kernel(const T* __restrict__ vol, const float* __restrict__ coords,
                                             const T* __restrict__ g, float* __restrict__ cgrad, int B, int h1,
                                             int w1, int h2, int w2, int r) {
    using A = typename Acc<T>::type;
    const int64_t HW1 = (int64_t)h1 * w1;
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= B * HW1) return;
    const int n = (int)(idx / HW1);
    const int64_t pix = idx % HW1;
    const float x0 = coords[((int64_t)n * 2 + 0) * HW1 + pix];
    const float y0 = coords[((int64_t)n * 2 + 1) * HW1 + pix];
    const float fx0 = floorf(x0), fy0 = floorf(y0);
    const A dx = (A)(x0 - fx0), dy = (A)(y0 - fy0);
    const int bx = window_origin(fx0, r), by = window_origin(fy0, r);
    const int rd = 2 * r + 1;
    const T* plane = vol + ((int64_t)n * HW1 + pix) * ((int64_t)h2 * w2);
    const T* go = g + (int64_t)n * rd * rd * HW1 + pix;
    auto tap = [&](int x, int y) -> A { return inb(y, x, h2, w2) ? load_acc<A>(plane + (int64_t)y * w2 + x) : (A)0; };
    A gx = 0, gy = 0;
    for (int i = 0; i < rd; i++) {
        // column pair x = bx + i, bx + i + 1 walked down the rows: each row's taps are reused by the next j
        A v00 = tap(bx + i, by), v10 = tap(bx + i + 1, by);
        for (int j = 0; j < rd; j++) {
            const A v01 = tap(bx + i, by + j + 1), v11 = tap(bx + i + 1, by + j + 1);
            const A gij = load_acc<A>(go + (int64_t)(i * rd + j) * HW1);
            gx += gij * ((1 - dy) * (v10 - v00) + dy * (v11 - v01));
            gy += gij * ((1 - dx) * (v01 - v00) + dx * (v11 - v10));
            v00 = v01;
            v10 = v11;
        }
    }
    cgrad[((int64_t)n * 2 + 0) * HW1 + pix] = (float)gx;
    cgrad[((int64_t)n * 2 + 1) * HW1 + pix] = (float)gy;
}

// ---------------------------------------------------------------- on-the-fly lookup (warp per pixel)

constexpr int kWarps = 8;        // warps per CTA
constexpr int kTile = 32;        // pixels per CTA tile (one row segment)
constexpr int kMaxC = 256;       // channels staged per pixel
constexpr int kMaxR = 3;         // radius supported by the warp kernels
constexpr int kMaxOut = (2 * kMaxR + 1) * (2 * kMaxR + 1);

// Dot product of C channels of a tap row (global, dtype T) with f1 (shared, A);
// 16-byte vector loads when C allows.
template <typename T, typename A>
__device__ __forceinline__ A row_dot(const T* __restrict__ f2, const A* f1s, int C) {
    constexpr int V = 16 / (int)sizeof(T);
    A s = 0;
    if (C % V == 0) {
        for (int c = 0; c < C; c += V) {
            const uint4 raw = __ldg(reinterpret_cast<const uint4*>(f2 + c));
            const T* e = reinterpret_cast<const T*>(&raw);
#pragma unroll
            for (int k = 0; k < V; k++) s += f1s[c + k] * (A)to_f(e[k]);
        }
    } else {
        for (int c = 0; c < C; c++) s += f1s[c] * (A)to_f(f2[c]);
    }
    return s;
}

// Dot products of the (2r+2)^2 window taps against f1 (shared memory) for one
// pixel; lane owns taps `lane` and `lane + 32`.  Returns them in t0, t1.
template <typename T, typename A>
__device__ __forceinline__ void window_dots(const T* __restrict__ fmap2, int H2, int W2, int C, const A* f1s, float xc,
                                            float yc, int r, A& t0, A& t1) {
    const int lane = threadIdx.x & 31;
    const int ne = 2 * r + 2;
    const int nt = ne * ne;
    const int bx = window_origin(floorf(xc), r), by = window_origin(floorf(yc), r);
    t0 = 0;
    t1 = 0;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int tap = lane + 32 * h;
        if (tap >= nt) continue;
        const int ix = tap / ne, iy = tap % ne;
        const int x2 = bx + ix, y2 = by + iy;
        A sacc = 0;
        if (inb(y2, x2, H2, W2)) sacc = row_dot<T, A>(fmap2 + ((int64_t)y2 * W2 + x2) * C, f1s, C);
        if (h == 0) t0 = sacc; else t1 = sacc;
    }
}

// value of tap (ix, iy) held by lane (ix*ne+iy) mod 32 in t0/t1
template <typename A>
__device__ __forceinline__ A tap_value(A t0, A t1, int ne, int ix, int iy) {
    const int tap = ix * ne + iy;
    const A a = __shfl_sync(0xffffffffu, t0, tap & 31);
    const A b = __shfl_sync(0xffffffffu, t1, tap & 31);
    return tap < 32 ? a : b;
}

// bilinear combination of the window taps into (2r+1)^2 outputs; lane writes
// outputs lane and lane+32 into out_s[ch * stride]
template <typename A>
__device__ __forceinline__ void combine(A t0, A t1, int r, float xc, float yc, float* out_s, int stride) {
    const int lane = threadIdx.x & 31;
    const int rd = 2 * r + 1, ne = rd + 1;
    const A dx = (A)(xc - floorf(xc)), dy = (A)(yc - floorf(yc));
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int ch = lane + 32 * h;
        // shuffles must be executed by all lanes: compute indices clamped
        const int chc = ch < rd * rd ? ch : 0;
        const int i = chc / rd, j = chc % rd;
        const A a00 = tap_value(t0, t1, ne, i, j);
        const A a10 = tap_value(t0, t1, ne, i + 1, j);
        const A a01 = tap_value(t0, t1, ne, i, j + 1);
        const A a11 = tap_value(t0, t1, ne, i + 1, j + 1);
        const A v = (1 - dx) * (1 - dy) * a00 + dx * (1 - dy) * a10 + (1 - dx) * dy * a01 + dx * dy * a11;
        if (ch < rd * rd) out_s[ch * stride] = (float)v;
    }
}

// altcorr_forward: fmap1 (B,H1,W1,C), fmap2 (B,H2,W2,C), coords (B,S,H1,W1,2)
// -> out (B,S,rd^2,H1,W1).  grid: (ceil(W1/32), H1, B*S)
template <typename T>
__global__ void __launch_bounds__(kWarps * 32)
    altcorr_fwd_kernel(const T* __restrict__ fmap1, const T* __restrict__ fmap2, const float* __restrict__ coords,
                       T* __restrict__ out, int B, int S, int H1, int W1, int H2, int W2, int C, int r) {
    using A = typename Acc<T>::type;
    __shared__ A f1s[kWarps][kMaxC];
    __shared__ float os[kMaxOut][kTile];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bs = blockIdx.z, b = bs / S;
    const int h1 = blockIdx.y, w0 = blockIdx.x * kTile;
    const int rd = 2 * r + 1;
    const int64_t HW1 = (int64_t)H1 * W1;
    for (int pp = warp; pp < kTile; pp += kWarps) {
        const int w1 = w0 + pp;
        if (w1 >= W1) break;
        const T* f1 = fmap1 + (((int64_t)b * H1 + h1) * W1 + w1) * C;
        for (int c = lane; c < C; c += 32) f1s[warp][c] = (A)to_f(f1[c]);
        __syncwarp();
        const float* cp = coords + (((int64_t)bs * H1 + h1) * W1 + w1) * 2;
        const float xc = cp[0], yc = cp[1];
        A t0, t1;
        window_dots<T, A>(fmap2 + (int64_t)b * H2 * W2 * C, H2, W2, C, f1s[warp], xc, yc, r, t0, t1);
        combine<A>(t0, t1, r, xc, yc, &os[0][pp], kTile);
        __syncwarp();
    }
    __syncthreads();
    const int nw = min(kTile, W1 - w0);
    for (int q = threadIdx.x; q < rd * rd * kTile; q += blockDim.x) {
        const int ch = q / kTile, pp = q % kTile;
        if (pp < nw) out[((int64_t)bs * rd * rd + ch) * HW1 + (int64_t)h1 * W1 + w0 + pp] = from_f<T>(os[ch][pp]);
    }
}

// altcorr_index_forward: fmap1 (B,Nf,H,W,C) level 0, levels[l] (B,Nf,H2[l],W2[l],C),
// coords (B,M,H,W,2), ii/jj (M) -> out (B,M,L*rd^2,H,W) f32.  grid (ceil(W/32), H, B*M)
struct LevelPtrs {
    const void* p[8];
    int H2[8];
    int W2[8];
};

constexpr int kMaxL = 4;  // pyramid levels kept in the shared output tile

template <typename T>
__global__ void __launch_bounds__(kWarps * 32)
    altcorr_index_fwd_kernel(const T* __restrict__ fmap1, LevelPtrs lv, int L, const float* __restrict__ coords,
                             const int64_t* __restrict__ ii, const int64_t* __restrict__ jj, float* __restrict__ out,
                             int B, int Nf, int M, int H, int W, int C, int r) {
    using A = typename Acc<T>::type;
    __shared__ A f1s[kWarps][kMaxC];
    __shared__ float os[kMaxL * kMaxOut][kTile];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bm = blockIdx.z, b = bm / M, m = bm % M;
    const int h = blockIdx.y, w0 = blockIdx.x * kTile;
    const int src = (int)ii[m], dst = (int)jj[m];
    const int rd = 2 * r + 1, nch = rd * rd;
    const int64_t HW = (int64_t)H * W;
    const int nw = min(kTile, W - w0);
    for (int pp = warp; pp < nw; pp += kWarps) {
        const int w = w0 + pp;
        const T* f1 = fmap1 + ((((int64_t)b * Nf + src) * H + h) * W + w) * C;
        for (int c = lane; c < C; c += 32) f1s[warp][c] = (A)to_f(f1[c]);
        __syncwarp();
        const float* cp = coords + (((int64_t)bm * H + h) * W + w) * 2;
        for (int l = 0; l < L; l++) {
            // reference: coords / 2^l at level l (droid_net.py:78, altcorr_kernel.cu:182-183)
            const float scale = (float)(1 << l);
            const float xc = cp[0] / scale, yc = cp[1] / scale;
            const int H2 = lv.H2[l], W2 = lv.W2[l];
            const T* f2base = static_cast<const T*>(lv.p[l]) + ((int64_t)b * Nf + dst) * H2 * W2 * C;
            A t0, t1;
            window_dots<T, A>(f2base, H2, W2, C, f1s[warp], xc, yc, r, t0, t1);
            combine<A>(t0, t1, r, xc, yc, &os[l * nch][pp], kTile);
        }
        __syncwarp();
    }
    __syncthreads();
    for (int q = threadIdx.x; q < L * nch * kTile; q += blockDim.x) {
        const int ch = q / kTile, pp = q % kTile;
        if (pp < nw) out[((int64_t)bm * L * nch + ch) * HW + (int64_t)h * W + w0 + pp] = os[ch][pp];
    }
}

// Indexed lookup for 16-bit maps, radius 3, C in {64, 128, 256}, on the tensor
// cores (warp-level mma.sync m16n8k16, FP32 accumulation).  A warp owns 8
// consecutive pixels of one row (the 8 columns of B: each pixel's fmap1 row)
// and, per level, the union box of their 8x8 windows: the box taps are the M
// rows of A (16-row tiles, row r = tap (X0 + r % bw, Y0 + r / bw), rows
// outside the map read as zeros), so D holds the dot product of every box tap
// with every pixel, and each pixel's window is a sub-box of D.  For smooth
// coordinates the windows of neighbouring pixels overlap and the box holds far
// fewer taps than 8 x 64 (about 200 at level 0, 90 at level 3); a box above
// kMaxBox taps falls back to one pass per pixel over its own window.
// Channels are permuted identically in A and B so that one 16-byte load per
// row gives a lane its elements of two consecutive k-steps: k-step s, lane quad
// index q, element e in 0..3 reads channel 32 (s / 2) + 8 q + 4 (s % 2) + e (a
// dot product is invariant to the channel order).  D goes through shared
// memory to the bilinear combination; outputs leave as 32-byte row segments.
template <typename T>
__device__ __forceinline__ void mma_16816(float* d, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                          uint32_t b1) {
    if constexpr (std::is_same<T, __half>::value) {
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
            "{%0, %1, %2, %3};"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
    } else {
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
            "{%0, %1, %2, %3};"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
    }
}

constexpr int kUnionTile = 64;  // pixels per CTA (8 per warp)
constexpr int kMaxBox = 384;    // union taps per warp pass (24 row tiles)
constexpr size_t kUnionSmem = (size_t)kWarps * kMaxBox * 8 * sizeof(float);

template <typename T, int NK>  // NK = C / 32
__global__ void __launch_bounds__(kWarps * 32, 2)
    altcorr_index_fwd_mma_kernel(const T* __restrict__ fmap1, LevelPtrs lv, int L, const float* __restrict__ coords,
                                 const int64_t* __restrict__ ii, const int64_t* __restrict__ jj,
                                 float* __restrict__ out, int B, int Nf, int M, int H, int W) {
    constexpr int C = 32 * NK;
    constexpr unsigned kFull = 0xffffffffu;
    extern __shared__ float dsm_all[];  // [kWarps][kMaxBox][8]: D of the current box pass
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane >> 2, quad = lane & 3;
    float* Dsm = dsm_all + (size_t)warp * kMaxBox * 8;
    const int bm = blockIdx.z, b = bm / M, m = bm % M;
    const int h = blockIdx.y;
    const int wbase = blockIdx.x * kUnionTile + 8 * warp;  // the warp's first pixel
    if (wbase >= W) return;                                // whole warp (no block-level barrier below)
    const int src = (int)ii[m], dst = (int)jj[m];
    const int64_t HW = (int64_t)H * W;
    // B column grp: pixel wbase + grp (zeros past the row end)
    const int pg = wbase + grp;
    const bool gvalid = pg < W;
    uint4 bf[NK];
    const T* f1 = fmap1 + ((((int64_t)b * Nf + src) * H + h) * W + (gvalid ? pg : wbase)) * C + 8 * quad;
#pragma unroll
    for (int t = 0; t < NK; t++)
        bf[t] = gvalid ? __ldg(reinterpret_cast<const uint4*>(f1 + 32 * t)) : make_uint4(0, 0, 0, 0);
    float xc = 0.f, yc = 0.f;
    if (gvalid) {
        const float* cp = coords + (((int64_t)bm * H + h) * W + pg) * 2;
        xc = cp[0];
        yc = cp[1];
    }
    // the pixel this lane writes outputs for (fixed: lane + 32 k has the same low 3 bits)
    const int n = lane & 7;
    const bool nvalid = wbase + n < W;
    for (int l = 0; l < L; l++) {
        // coords / 2^l at level l (droid_net.py:78, altcorr_kernel.cu:182-183)
        const float scale = (float)(1 << l);
        const float xl = xc / scale, yl = yc / scale;
        const int bx = window_origin(floorf(xl), 3), by = window_origin(floorf(yl), 3);
        const int H2 = lv.H2[l], W2 = lv.W2[l];
        const T* f2 = static_cast<const T*>(lv.p[l]) + ((int64_t)b * Nf + dst) * H2 * W2 * C + 8 * quad;
        const int bxn = __shfl_sync(kFull, bx, 4 * n), byn = __shfl_sync(kFull, by, 4 * n);
        const float xln = __shfl_sync(kFull, xl, 4 * n), yln = __shfl_sync(kFull, yl, 4 * n);
        const float dxn = xln - floorf(xln), dyn = yln - floorf(yln);
        const int X0 = __reduce_min_sync(kFull, gvalid ? bx : INT_MAX);
        const int X1 = __reduce_max_sync(kFull, gvalid ? bx : INT_MIN) + 7;
        const int Y0 = __reduce_min_sync(kFull, gvalid ? by : INT_MAX);
        const int Y1 = __reduce_max_sync(kFull, gvalid ? by : INT_MIN) + 7;
        // window origins are clamped to +-2^24, so the extents fit an int and their product an int64
        const bool joint = (int64_t)(X1 - X0 + 1) * (Y1 - Y0 + 1) <= kMaxBox;
        const int npass = joint ? 1 : 8;
        for (int pass = 0; pass < npass; pass++) {
            const int sx = __shfl_sync(kFull, bx, 4 * pass), sy = __shfl_sync(kFull, by, 4 * pass);
            if (!joint && wbase + pass >= W) break;  // warp-uniform
            const int bx0 = joint ? X0 : sx, by0 = joint ? Y0 : sy;
            const int bw = joint ? X1 - X0 + 1 : 8, bh = joint ? Y1 - Y0 + 1 : 8;
            const unsigned mask = joint ? 0xffu : 1u << pass;
            const int nbox = bw * bh;
            const int ntile = (nbox + 15) >> 4;
            for (int mt = 0; mt < ntile; mt += 2) {  // two row tiles per step (rows past nbox are zeros)
                int off[4];
                bool ok[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int r = 16 * (mt + (q >> 1)) + grp + 8 * (q & 1);
                    const int x = bx0 + r % bw, y = by0 + r / bw;
                    ok[q] = r < nbox && inb(y, x, H2, W2);
                    off[q] = ok[q] ? (y * W2 + x) * C : 0;
                }
                float acc[2][4];
#pragma unroll
                for (int tt = 0; tt < 2; tt++)
#pragma unroll
                    for (int e = 0; e < 4; e++) acc[tt][e] = 0.f;
#pragma unroll
                for (int t = 0; t < NK; t++) {
                    uint4 rows[4];
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        rows[q] = ok[q] ? __ldg(reinterpret_cast<const uint4*>(f2 + off[q] + 32 * t))
                                        : make_uint4(0, 0, 0, 0);
#pragma unroll
                    for (int tt = 0; tt < 2; tt++) {
                        const uint4 r0 = rows[2 * tt], r1 = rows[2 * tt + 1];
                        // k-step 2t: elements 0..3 of the chunk; k-step 2t + 1: elements 4..7
                        mma_16816<T>(acc[tt], r0.x, r1.x, r0.y, r1.y, bf[t].x, bf[t].y);
                        mma_16816<T>(acc[tt], r0.z, r1.z, r0.w, r1.w, bf[t].z, bf[t].w);
                    }
                }
#pragma unroll
                for (int tt = 0; tt < 2; tt++) {
                    const int row = 16 * (mt + tt) + grp;
                    *reinterpret_cast<float2*>(Dsm + row * 8 + 2 * quad) = make_float2(acc[tt][0], acc[tt][1]);
                    *reinterpret_cast<float2*>(Dsm + (row + 8) * 8 + 2 * quad) = make_float2(acc[tt][2], acc[tt][3]);
                }
            }
            __syncwarp();
            if (((mask >> n) & 1u) && nvalid) {
                const int px = bxn - bx0, py = byn - by0;  // the pixel's window inside the box
                const float* col = Dsm + n;
                for (int o = lane; o < 49 * 8; o += 32) {
                    const int ch = o >> 3;
                    const int i = ch / 7, j = ch % 7;
                    const int r = (py + j) * bw + px + i;
                    const float v = (1.f - dxn) * (1.f - dyn) * col[r * 8] + dxn * (1.f - dyn) * col[(r + 1) * 8] +
                                    (1.f - dxn) * dyn * col[(r + bw) * 8] + dxn * dyn * col[(r + bw + 1) * 8];
                    out[((int64_t)bm * L * 49 + l * 49 + ch) * HW + (int64_t)h * W + wbase + n] = v;
                }
            }
            __syncwarp();
        }
    }
}

// altcorr_backward (f32): fmap1_grad (B,H1,W1,C) and fmap2_grad (B,H2,W2,C) must
// be zero on entry.  Per (pixel, sample) warp: tap gradients from the bilinear
// adjoint; fmap1_grad gathered per pixel (owned by the warp across samples);
// fmap2_grad scattered with atomic adds (windows of neighbouring pixels overlap),
// as the reference does.  With exact_coords the derivative of the bilinear
// weights is written to coords_grad (B,S,H1,W1,2); otherwise zeros.
__global__ void __launch_bounds__(kWarps * 32)
    altcorr_bwd_kernel(const float* __restrict__ fmap1, const float* __restrict__ fmap2,
                       const float* __restrict__ coords, const float* __restrict__ g, float* __restrict__ g1,
                       float* __restrict__ g2, float* __restrict__ gc, int B, int S, int H1, int W1, int H2, int W2,
                       int C, int r, int exact_coords) {
    __shared__ float f1s[kWarps][kMaxC];
    __shared__ float acc1[kWarps][kMaxC];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.z;
    const int h1 = blockIdx.y;
    const int w1 = blockIdx.x * kWarps + warp;
    if (w1 >= W1) return;
    const int rd = 2 * r + 1, ne = rd + 1, nt = ne * ne;
    const int64_t HW1 = (int64_t)H1 * W1;
    const float* f1 = fmap1 + (((int64_t)b * H1 + h1) * W1 + w1) * C;
    for (int c = lane; c < C; c += 32) {
        f1s[warp][c] = f1[c];
        acc1[warp][c] = 0.f;
    }
    __syncwarp();
    const float* f2base = fmap2 + (int64_t)b * H2 * W2 * C;
    float* g2base = g2 + (int64_t)b * H2 * W2 * C;
    for (int s = 0; s < S; s++) {
        const int64_t bs = (int64_t)b * S + s;
        const float* cp = coords + ((bs * H1 + h1) * W1 + w1) * 2;
        const float xc = cp[0], yc = cp[1];
        const float dx = xc - floorf(xc), dy = yc - floorf(yc);
        const int bx = window_origin(floorf(xc), r), by = window_origin(floorf(yc), r);
        const float* gp = g + bs * rd * rd * HW1 + (int64_t)h1 * W1 + w1;
        float gt[2];
#pragma unroll
        for (int hh = 0; hh < 2; hh++) {
            const int tap = lane + 32 * hh;
            float v = 0.f;
            if (tap < nt) {
                const int i = tap / ne, j = tap % ne;
                if (i > 0 && j > 0) v += gp[(int64_t)((i - 1) * rd + (j - 1)) * HW1] * dx * dy;
                if (i > 0 && j < rd) v += gp[(int64_t)((i - 1) * rd + j) * HW1] * dx * (1.f - dy);
                if (i < rd && j > 0) v += gp[(int64_t)(i * rd + (j - 1)) * HW1] * (1.f - dx) * dy;
                if (i < rd && j < rd) v += gp[(int64_t)(i * rd + j) * HW1] * (1.f - dx) * (1.f - dy);
            }
            gt[hh] = v;
        }
        float t0 = 0.f, t1 = 0.f;
        if (exact_coords) window_dots<float, float>(f2base, H2, W2, C, f1s[warp], xc, yc, r, t0, t1);
        // taps: fmap1 grad gather (lanes over channels) and fmap2 grad scatter
        for (int tap = 0; tap < nt; tap++) {
            const float gv = __shfl_sync(0xffffffffu, gt[tap >> 5], tap & 31);
            const int ix = tap / ne, iy = tap % ne;
            const int x2 = bx + ix, y2 = by + iy;
            if (gv == 0.f || !inb(y2, x2, H2, W2)) continue;
            const float* f2 = f2base + ((int64_t)y2 * W2 + x2) * C;
            float* q2 = g2base + ((int64_t)y2 * W2 + x2) * C;
            for (int c = lane; c < C; c += 32) {
                acc1[warp][c] += gv * f2[c];
                atomicAdd(q2 + c, gv * f1s[warp][c]);
            }
        }
        if (gc) {
            float cx = 0.f, cy = 0.f;
            if (exact_coords) {
                // d out[i][j] / d dx = (1-dy)(a10 - a00) + dy (a11 - a01), similarly for dy
#pragma unroll
                for (int hh = 0; hh < 2; hh++) {
                    const int ch = lane + 32 * hh;
                    const int chc = ch < rd * rd ? ch : 0;
                    const int i = chc / rd, j = chc % rd;
                    const float a00 = tap_value(t0, t1, ne, i, j);
                    const float a10 = tap_value(t0, t1, ne, i + 1, j);
                    const float a01 = tap_value(t0, t1, ne, i, j + 1);
                    const float a11 = tap_value(t0, t1, ne, i + 1, j + 1);
                    if (ch < rd * rd) {
                        const float go = gp[(int64_t)ch * HW1];
                        cx += go * ((1.f - dy) * (a10 - a00) + dy * (a11 - a01));
                        cy += go * ((1.f - dx) * (a01 - a00) + dx * (a11 - a10));
                    }
                }
                cx = warp_sum(cx);
                cy = warp_sum(cy);
            }
            if (lane == 0) {
                float* o = gc + ((bs * H1 + h1) * W1 + w1) * 2;
                o[0] = cx;
                o[1] = cy;
            }
        }
    }
    __syncwarp();
    float* q1 = g1 + (((int64_t)b * H1 + h1) * W1 + w1) * C;
    for (int c = lane; c < C; c += 32) q1[c] = acc1[warp][c];
}

// four consecutive channels as floats (16-bit types: one 8-byte load, f32: one 16-byte load)
template <typename T>
__device__ __forceinline__ void load4(const T* p, float* v) {
    const uint2 raw = __ldg(reinterpret_cast<const uint2*>(p));
    const T* e = reinterpret_cast<const T*>(&raw);
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = to_f(e[k]);
}
template <>
__device__ __forceinline__ void load4<float>(const float* p, float* v) {
    const float4 raw = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = raw.x;
    v[1] = raw.y;
    v[2] = raw.z;
    v[3] = raw.w;
}

struct LevelGrads {
    float* p[8];
};

// Adjoint of altcorr_index_forward (the reference has none): gradients to the
// level-0 map fmap1 (B,Nf,H,W,C), to every pyramid level (B,Nf,H2[l],W2[l],C)
// and, with exact_coords, to coords (B,M,H,W,2) (sum over levels of 2^-l times
// the derivative of the bilinear weights at level l; zeros otherwise).  All
// gradients are f32; the map gradients must be zero on entry.  One warp per
// (pixel, edge): tap gradients from the bilinear adjoint per level; the
// fmap1 gradient is gathered in registers over all levels' taps and added once
// (edges sharing a source frame add into the same row); the level gradients
// are scattered into the window rows (windows of neighbouring pixels and of
// edges sharing a target overlap).  Both use 16-byte vector atomics when
// `vec` (C % 4 == 0 and aligned rows), one lane per 4 channels.
// grid (ceil(W / kWarps), H, B * M)
template <typename T>
__global__ void __launch_bounds__(kWarps * 32)
    altcorr_index_bwd_kernel(const T* __restrict__ fmap1, LevelPtrs lv, LevelGrads lg, int L,
                             const float* __restrict__ coords, const int64_t* __restrict__ ii,
                             const int64_t* __restrict__ jj, const float* __restrict__ g, float* __restrict__ g1,
                             float* __restrict__ gc, int B, int Nf, int M, int H, int W, int C, int r,
                             int exact_coords, int vec) {
    __shared__ float f1s[kWarps][kMaxC];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bm = blockIdx.z, b = bm / M, m = bm % M;
    const int h = blockIdx.y, w = blockIdx.x * kWarps + warp;
    if (w >= W) return;
    const int src = (int)ii[m], dst = (int)jj[m];
    const int rd = 2 * r + 1, nch = rd * rd, ne = rd + 1, nt = ne * ne;
    const int64_t HW = (int64_t)H * W;
    const T* f1 = fmap1 + ((((int64_t)b * Nf + src) * H + h) * W + w) * C;
    for (int c = lane; c < C; c += 32) f1s[warp][c] = to_f(f1[c]);
    __syncwarp();
    // this lane's channels of the fmap1 gradient: vector path c = 4 lane + 128 k, scalar path c = lane + 32 k
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float* cp = coords + (((int64_t)bm * H + h) * W + w) * 2;
    float gcx = 0.f, gcy = 0.f;
    for (int l = 0; l < L; l++) {
        const float scale = (float)(1 << l);
        const float xc = cp[0] / scale, yc = cp[1] / scale;
        const float dx = xc - floorf(xc), dy = yc - floorf(yc);
        const int bx = window_origin(floorf(xc), r), by = window_origin(floorf(yc), r);
        const int H2 = lv.H2[l], W2 = lv.W2[l];
        const int64_t plane = ((int64_t)b * Nf + dst) * H2 * W2;
        const T* f2base = static_cast<const T*>(lv.p[l]) + plane * C;
        float* g2base = lg.p[l] + plane * C;
        const float* gp = g + ((int64_t)bm * L * nch + (int64_t)l * nch) * HW + (int64_t)h * W + w;
        float gt[2];
#pragma unroll
        for (int hh = 0; hh < 2; hh++) {
            const int tap = lane + 32 * hh;
            float v = 0.f;
            if (tap < nt) {
                const int i = tap / ne, j = tap % ne;
                if (i > 0 && j > 0) v += gp[(int64_t)((i - 1) * rd + (j - 1)) * HW] * dx * dy;
                if (i > 0 && j < rd) v += gp[(int64_t)((i - 1) * rd + j) * HW] * dx * (1.f - dy);
                if (i < rd && j > 0) v += gp[(int64_t)(i * rd + (j - 1)) * HW] * (1.f - dx) * dy;
                if (i < rd && j < rd) v += gp[(int64_t)(i * rd + j) * HW] * (1.f - dx) * (1.f - dy);
            }
            gt[hh] = v;
        }
        if (exact_coords) {
            float t0, t1;
            window_dots<T, float>(f2base, H2, W2, C, f1s[warp], xc, yc, r, t0, t1);
            float cx = 0.f, cy = 0.f;
#pragma unroll
            for (int hh = 0; hh < 2; hh++) {
                const int ch = lane + 32 * hh;
                const int chc = ch < nch ? ch : 0;
                const int i = chc / rd, j = chc % rd;
                const float a00 = tap_value(t0, t1, ne, i, j);
                const float a10 = tap_value(t0, t1, ne, i + 1, j);
                const float a01 = tap_value(t0, t1, ne, i, j + 1);
                const float a11 = tap_value(t0, t1, ne, i + 1, j + 1);
                if (ch < nch) {
                    const float go = gp[(int64_t)ch * HW];
                    cx += go * ((1.f - dy) * (a10 - a00) + dy * (a11 - a01));
                    cy += go * ((1.f - dx) * (a01 - a00) + dx * (a11 - a10));
                }
            }
            gcx += warp_sum(cx) / scale;
            gcy += warp_sum(cy) / scale;
        }
        for (int tap = 0; tap < nt; tap++) {
            const float gv = __shfl_sync(0xffffffffu, gt[tap >> 5], tap & 31);
            const int ix = tap / ne, iy = tap % ne;
            const int x2 = bx + ix, y2 = by + iy;
            if (gv == 0.f || !inb(y2, x2, H2, W2)) continue;  // warp-uniform
            const int64_t row = ((int64_t)y2 * W2 + x2) * C;
            if (vec) {
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    const int c = 4 * lane + 128 * k;
                    if (c >= C) break;
                    float f2v[4];
                    load4<T>(f2base + row + c, f2v);
                    float4 add;
                    add.x = gv * f1s[warp][c];
                    add.y = gv * f1s[warp][c + 1];
                    add.z = gv * f1s[warp][c + 2];
                    add.w = gv * f1s[warp][c + 3];
#pragma unroll
                    for (int q = 0; q < 4; q++) acc[4 * k + q] += gv * f2v[q];
                    atomicAdd(reinterpret_cast<float4*>(g2base + row + c), add);
                }
            } else {
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int c = lane + 32 * k;
                    if (c >= C) break;
                    acc[k] += gv * to_f(f2base[row + c]);
                    atomicAdd(g2base + row + c, gv * f1s[warp][c]);
                }
            }
        }
    }
    float* q1 = g1 + ((((int64_t)b * Nf + src) * H + h) * W + w) * C;
    if (vec) {
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int c = 4 * lane + 128 * k;
            if (c >= C) break;
            atomicAdd(reinterpret_cast<float4*>(q1 + c), make_float4(acc[4 * k], acc[4 * k + 1], acc[4 * k + 2],
                                                                     acc[4 * k + 3]));
        }
    } else {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int c = lane + 32 * k;
            if (c >= C) break;
            atomicAdd(q1 + c, acc[k]);
        }
    }
    if (gc && lane == 0) {
        float* o = gc + (((int64_t)bm * H + h) * W + w) * 2;
        o[0] = gcx;
        o[1] = gcy;
    }
}

template <typename F>
int dispatch(int dtype, F&& f) {
    switch (dtype) {
        case VIPE_F32: return f(float());
        case VIPE_F64: return f(double());
        case VIPE_F16: return f(__half());
        case VIPE_BF16: return f(__nv_bfloat16());
        default: return VIPE_ERR_DTYPE;
    }
}

// f32 / f16 / bf16 only
template <typename F>
int dispatch_no_f64(int dtype, F&& f) {
    switch (dtype) {
        case VIPE_F32: return f(float());
        case VIPE_F16: return f(__half());
        case VIPE_BF16: return f(__nv_bfloat16());
        default: return VIPE_ERR_DTYPE;
    }
}

}  // namespace corr
}  // namespace vipe

using namespace vipe;
using namespace vipe::corr;

extern "C" int vipe_corr_index_forward(int dtype, const void* volume, const float* coords, int B, int h1, int w1,
                                       int h2, int w2, int radius, void* corr_out, void* stream) {
    if (B < 0 || h1 < 0 || w1 < 0 || h2 <= 0 || w2 <= 0 || radius < 0) return VIPE_ERR_ARG;
    const int64_t n = (int64_t)B * h1 * w1;
    if (n == 0) return VIPE_OK;
    cudaStream_t st = as_stream(stream);
    return dispatch(dtype, [&](auto tag) {
        using T = decltype(tag);
        VIPE_PROF("corr_index_fwd", st);
        if constexpr (!std::is_same<T, double>::value) {
            if (radius == 3 && ((size_t)w2 * sizeof(T)) % 16 == 0 && (uintptr_t)volume % 16 == 0) {
                corr_index_fwd_r3_kernel<T><<<ceil_div(n, 256), 256, 0, st>>>(
                    static_cast<const T*>(volume), coords, static_cast<T*>(corr_out), B, h1, w1, h2, w2);
                VIPE_LAUNCH_CHECK();
                return (int)VIPE_OK;
            }
        }
        corr_index_fwd_kernel<T><<<ceil_div(n, 256), 256, 0, st>>>(static_cast<const T*>(volume), coords,
                                                                   static_cast<T*>(corr_out), B, h1, w1, h2, w2,
                                                                   radius);
        VIPE_LAUNCH_CHECK();
        return (int)VIPE_OK;
    });
}

extern "C" int vipe_corr_index_backward(int dtype, const float* coords, const void* corr_grad, int B, int h1, int w1,
                                        int h2, int w2, int radius, void* volume_grad_out, void* stream) {
    if (B < 0 || h1 < 0 || w1 < 0 || h2 <= 0 || w2 <= 0 || radius < 0) return VIPE_ERR_ARG;
    const int64_t n = (int64_t)B * h1 * w1;
    cudaStream_t st = as_stream(stream);
    return dispatch(dtype, [&](auto tag) {
        using T = decltype(tag);
        VIPE_CUDA_TRY(cudaMemsetAsync(volume_grad_out, 0, (size_t)n * h2 * w2 * sizeof(T), st));
        if (n == 0) return (int)VIPE_OK;
        VIPE_PROF("corr_index_bwd", st);
        corr_index_bwd_kernel<T><<<ceil_div(n, 256), 256, 0, st>>>(coords, static_cast<const T*>(corr_grad),
                                                                   static_cast<T*>(volume_grad_out), B, h1, w1, h2,
                                                                   w2, radius);
        VIPE_LAUNCH_CHECK();
        return (int)VIPE_OK;
    });
}

extern "C" int vipe_corr_index_coords_backward(int dtype, const void* volume, const float* coords,
                                               const void* corr_grad, int B, int h1, int w1, int h2, int w2,
                                               int radius, float* coords_grad_out, void* stream) {
    if (B < 0 || h1 < 0 || w1 < 0 || h2 <= 0 || w2 <= 0 || radius < 0) return VIPE_ERR_ARG;
    const int64_t n = (int64_t)B * h1 * w1;
    if (n == 0) return VIPE_OK;
    cudaStream_t st = as_stream(stream);
    return dispatch(dtype, [&](auto tag) {
        using T = decltype(tag);
        VIPE_PROF("corr_index_coords_bwd", st);
        corr_index_coords_bwd_kernel<T><<<ceil_div(n, 256), 256, 0, st>>>(
            static_cast<const T*>(volume), coords, static_cast<const T*>(corr_grad), coords_grad_out, B, h1, w1, h2,
            w2, radius);
        VIPE_LAUNCH_CHECK();
        return (int)VIPE_OK;
    });
}

extern "C" int vipe_altcorr_forward(int dtype, const void* fmap1, const void* fmap2, const float* coords, int B, int S,
                                    int H1, int W1, int H2, int W2, int C, int radius, void* corr_out, void* stream) {
    if (B < 0 || S < 0 || H1 < 0 || W1 < 0 || H2 <= 0 || W2 <= 0 || C <= 0) return VIPE_ERR_ARG;
    if (C > kMaxC || radius < 0 || radius > kMaxR) return VIPE_ERR_CAPACITY;
    if ((int64_t)B * S * H1 * W1 == 0) return VIPE_OK;
    if (B * S > 65535 || H1 > 65535) return VIPE_ERR_CAPACITY;
    cudaStream_t st = as_stream(stream);
    dim3 grid(ceil_div(W1, kTile), H1, B * S);
    return dispatch(dtype, [&](auto tag) {
        using T = decltype(tag);
        VIPE_PROF("altcorr_fwd", st);
        altcorr_fwd_kernel<T><<<grid, kWarps * 32, 0, st>>>(static_cast<const T*>(fmap1),
                                                             static_cast<const T*>(fmap2), coords,
                                                             static_cast<T*>(corr_out), B, S, H1, W1, H2, W2, C,
                                                             radius);
        VIPE_LAUNCH_CHECK();
        return (int)VIPE_OK;
    });
}

extern "C" int vipe_altcorr_backward(const float* fmap1, const float* fmap2, const float* coords,
                                     const float* corr_grad, int B, int S, int H1, int W1, int H2, int W2, int C,
                                     int radius, int exact_coords_grad, float* fmap1_grad_out, float* fmap2_grad_out,
                                     float* coords_grad_out, void* stream) {
    if (B < 0 || S < 0 || H1 < 0 || W1 < 0 || H2 <= 0 || W2 <= 0 || C <= 0) return VIPE_ERR_ARG;
    if (C > kMaxC || radius < 0 || radius > kMaxR) return VIPE_ERR_CAPACITY;
    cudaStream_t st = as_stream(stream);
    VIPE_CUDA_TRY(cudaMemsetAsync(fmap1_grad_out, 0, (size_t)B * H1 * W1 * C * sizeof(float), st));
    VIPE_CUDA_TRY(cudaMemsetAsync(fmap2_grad_out, 0, (size_t)B * H2 * W2 * C * sizeof(float), st));
    if (coords_grad_out)
        VIPE_CUDA_TRY(cudaMemsetAsync(coords_grad_out, 0, (size_t)B * S * H1 * W1 * 2 * sizeof(float), st));
    if ((int64_t)B * H1 * W1 == 0 || S == 0) return VIPE_OK;
    if (B > 65535 || H1 > 65535) return VIPE_ERR_CAPACITY;
    dim3 grid(ceil_div(W1, kWarps), H1, B);
    VIPE_PROF("altcorr_bwd", st);
    altcorr_bwd_kernel<<<grid, kWarps * 32, 0, st>>>(fmap1, fmap2, coords, corr_grad, fmap1_grad_out, fmap2_grad_out,
                                                     coords_grad_out, B, S, H1, W1, H2, W2, C, radius,
                                                     exact_coords_grad);
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}

extern "C" int vipe_altcorr_index_forward(int dtype, const void* fmap1, const void* const* fmap2_levels,
                                          const int* H2, const int* W2, int num_levels, const float* coords,
                                          const int64_t* ii, const int64_t* jj, int B, int Nf, int M, int H, int W,
                                          int C, int radius, float* corr_out, void* stream) {
    if (B < 0 || Nf <= 0 || M < 0 || H < 0 || W < 0 || C <= 0 || num_levels <= 0) return VIPE_ERR_ARG;
    if (num_levels > kMaxL || C > kMaxC || radius < 0 || radius > kMaxR) return VIPE_ERR_CAPACITY;
    if ((int64_t)B * M * H * W == 0) return VIPE_OK;
    if (B * M > 65535 || H > 65535) return VIPE_ERR_CAPACITY;
    LevelPtrs lv;
    for (int l = 0; l < num_levels; l++) {
        if (H2[l] <= 0 || W2[l] <= 0 || !fmap2_levels[l]) return VIPE_ERR_ARG;
        lv.p[l] = fmap2_levels[l];
        lv.H2[l] = H2[l];
        lv.W2[l] = W2[l];
    }
    cudaStream_t st = as_stream(stream);
    dim3 grid(ceil_div(W, kTile), H, B * M);
    bool aligned16 = (uintptr_t)fmap1 % 16 == 0;
    for (int l = 0; l < num_levels; l++) aligned16 = aligned16 && (uintptr_t)fmap2_levels[l] % 16 == 0;
    return dispatch(dtype, [&](auto tag) {
        using T = decltype(tag);
        VIPE_PROF("altcorr_index_fwd", st);
        if constexpr (sizeof(T) == 2) {
            if (radius == 3 && (C == 64 || C == 128 || C == 256) && aligned16) {
                const T* f1 = static_cast<const T*>(fmap1);
                const dim3 ug(ceil_div(W, kUnionTile), H, B * M);
                auto go = [&](auto kern) -> int {
                    VIPE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)kUnionSmem));
                    kern<<<ug, kWarps * 32, kUnionSmem, st>>>(f1, lv, num_levels, coords, ii, jj, corr_out, B, Nf, M,
                                                             H, W);
                    VIPE_LAUNCH_CHECK();
                    return (int)VIPE_OK;
                };
                if (C == 64) return go(altcorr_index_fwd_mma_kernel<T, 2>);
                if (C == 128) return go(altcorr_index_fwd_mma_kernel<T, 4>);
                return go(altcorr_index_fwd_mma_kernel<T, 8>);
            }
        }
        altcorr_index_fwd_kernel<T><<<grid, kWarps * 32, 0, st>>>(static_cast<const T*>(fmap1), lv, num_levels,
                                                                   coords, ii, jj, corr_out, B, Nf, M, H, W, C,
                                                                   radius);
        VIPE_LAUNCH_CHECK();
        return (int)VIPE_OK;
    });
}

extern "C" int vipe_altcorr_index_backward(int dtype, const void* fmap1, const void* const* fmap2_levels,
                                           const int* H2, const int* W2, int num_levels, const float* coords,
                                           const int64_t* ii, const int64_t* jj, const float* corr_grad, int B,
                                           int Nf, int M, int H, int W, int C, int radius, int exact_coords_grad,
                                           float* fmap1_grad_out, float* const* level_grads_out,
                                           float* coords_grad_out, void* stream) {
    if (B < 0 || Nf <= 0 || M < 0 || H < 0 || W < 0 || C <= 0 || num_levels <= 0) return VIPE_ERR_ARG;
    if (num_levels > kMaxL || C > kMaxC || radius < 0 || radius > kMaxR) return VIPE_ERR_CAPACITY;
    if (!fmap1_grad_out || !level_grads_out) return VIPE_ERR_ARG;
    cudaStream_t st = as_stream(stream);
    const size_t esz = dtype == VIPE_F32 ? 4 : 2;
    LevelPtrs lv;
    LevelGrads lg;
    bool aligned = C % 4 == 0 && (uintptr_t)fmap1 % 16 == 0 && (uintptr_t)fmap1_grad_out % 16 == 0;
    for (int l = 0; l < num_levels; l++) {
        if (H2[l] <= 0 || W2[l] <= 0 || !fmap2_levels[l] || !level_grads_out[l]) return VIPE_ERR_ARG;
        lv.p[l] = fmap2_levels[l];
        lv.H2[l] = H2[l];
        lv.W2[l] = W2[l];
        lg.p[l] = level_grads_out[l];
        aligned = aligned && (uintptr_t)fmap2_levels[l] % (4 * esz) == 0 && (uintptr_t)level_grads_out[l] % 16 == 0;
        VIPE_CUDA_TRY(cudaMemsetAsync(level_grads_out[l], 0, (size_t)B * Nf * H2[l] * W2[l] * C * sizeof(float), st));
    }
    VIPE_CUDA_TRY(cudaMemsetAsync(fmap1_grad_out, 0, (size_t)B * Nf * H * W * C * sizeof(float), st));
    if ((int64_t)B * M * H * W == 0) return VIPE_OK;
    if (B * M > 65535 || H > 65535) return VIPE_ERR_CAPACITY;
    dim3 grid(ceil_div(W, kWarps), H, B * M);
    return dispatch_no_f64(dtype, [&](auto tag) {
        using T = decltype(tag);
        VIPE_PROF("altcorr_index_bwd", st);
        altcorr_index_bwd_kernel<T><<<grid, kWarps * 32, 0, st>>>(
            static_cast<const T*>(fmap1), lv, lg, num_levels, coords, ii, jj, corr_grad, fmap1_grad_out,
            coords_grad_out, B, Nf, M, H, W, C, radius, exact_coords_grad, aligned ? 1 : 0);
        VIPE_LAUNCH_CHECK();
        return (int)VIPE_OK;
    });
}
