// gt_internal.cuh — shared device-side definitions of the B200 locate/link engine.
//
// Numerics contract (identical to the CPU oracle, which checks every kernel
// bit for bit): WGSL statements `acc += a * b;` are one fused multiply-add
// (__fmaf_rn); every other float operation is a separately rounded IEEE
// binary32 operation (the library is compiled with --fmad=false so nvcc
// never contracts on its own); division and sqrt are IEEE round-to-nearest;
// transcendental values (Gaussian taps, sin/cos of 2*atan2) come from tables
// the host computes with its libm.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gpu_tracking_b200.h"

namespace gt {

constexpr int kMaxTaps = 129;        // smoothing_size up to 129 (radius 64)
constexpr int kMaxLogTaps = 257;     // LoG: rint = int(4 sigma + 0.5) up to 128
constexpr int kLocateTH = 32;        // locate tile: rows
constexpr int kLocateTW = 64;        // locate tile: columns
constexpr int kLocateThreads = 256;
constexpr int kFinalizeThreads = 1024;
constexpr int kFinalizeSmemSort = 8192;  // per-frame detections sorted in shared memory

// Error flags raised by kernels (bitmask in a device word).
enum : uint32_t {
    kFlagCandOverflow = 1u,
    kFlagFeatOverflow = 2u,
    kFlagTooDense = 4u,
    kFlagSubnetBudget = 8u,
    kFlagScratch = 16u,
    kFlagListOverflow = 32u,   // windowed linking: a neighbour list buffer is full
    kFlagEdgeOverflow = 64u,   // windowed linking: a frame has more edges than the scratch holds
    kFlagTensorTimeout = 128u,  // a tensor-core kernel gave up waiting for its UMMAs
    kFlagLocalWalk = 256u,      // a learned seed did not finish its walk in the rounds allowed
};
// Linker flags after which the remaining frames of a video are not linked.
constexpr uint32_t kLinkStopFlags = 4u | 8u | 16u | 32u | 64u;

// Derived parameters of the trackpy locate pipeline
// (gpuparams_from_tracking_params, src/gpu_setup.rs:528-580).
struct LocateConsts {
    int32_t H, W;
    int32_t R;            // smoothing_size / 2
    float kk;             // (float)(smoothing_size^2)
    float gnorm;          // sequential sum of the taps
    int32_t truncate;
    int32_t kd, o;        // dilation size and its left offset int(kd/2 - 0.5)
    int32_t margin;
    float thr;            // pic_std * snr * rough_snr_factor
    // walk / characterize
    int32_t circle;       // circle_dims (diameter)
    uint32_t max_iter;
    float shift_thr;
    float minmass;
    float minmass_snr;
    float image_std;
    float rough;
    int32_t characterize;
    // Division by the call's constant divisors gnorm and kk as
    // fma(x, zh, x*zl) with zh + zl a two-float reciprocal; set only when
    // that equals IEEE x/d for every mantissa (checked on the device) and
    // every dividend the pipeline can produce lies in the exponent range
    // where the check carries over (integer pixel types).
    int32_t fast_div;
    float zh_g, zl_g, zh_k, zl_k;
    // Candidates at a processed value of exactly 0 may be left out: with
    // truncation every processed value is 0 or >= 1/255, so such a pixel's
    // whole dilation window is 0; when that window covers the walk circle the
    // walk ends where it started with mass 0 (0/0 centroid moves nothing),
    // and minmass > 0 rejects it (walk_keep, walk.wgsl).
    int32_t skip_zero;
    // snr / minmass_snr: per-frame std of the current chunk (nullptr when the
    // reference computes none); the candidate threshold is std * snr * rough
    // and the walk's minmass minmass_snr * count * std * rough
    const float* frame_std;
    float snr;
    float taps[kMaxTaps];
};

// A detection as the walk and characterize kernels produce it
// (ResultRow, src/execute_gpu.rs:48-61) plus its canonical sort key.
struct Feature {
    uint32_t key_hi;      // radius index (LoG) or 0
    uint32_t key_lo;      // candidate pixel index u*W+v, or input order
    float x, y, mass, r, max_i, Rg, raw, signal, ecc, count;
    float d_raw, d_bg, d_corr;
    int32_t ridx;         // radius index for doughnut tables (LoG)
};
static_assert(sizeof(Feature) == 64, "Feature is one 64-byte record");

// Orderable 32-bit key of a float (NaN sorts last).
__device__ __forceinline__ uint32_t float_order_key(float f) {
    uint32_t u = __float_as_uint(f);
    if (f != f) return 0xFFFFFFFFu;
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float float_from_order_key(uint32_t k) {
    uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
    return __uint_as_float(u);
}

// WGSL max(a, b): b if a < b else a.
__device__ __forceinline__ float wgsl_max(float a, float b) { return (a < b) ? b : a; }

// Row and column of element idx = r * w + c of a tile whose width w is a
// runtime value, stepped `step` elements at a time: two divisions when the
// stepping starts instead of one per element.
struct TileRowCol {
    int r, c, dq, dr, w;
    __device__ __forceinline__ TileRowCol(int idx, int step, int w_) : w(w_) {
        r = idx / w;
        c = idx - r * w;
        dq = step / w;
        dr = step - dq * w;
    }
    __device__ __forceinline__ void advance() {
        r += dq;
        c += dr;
        if (c >= w) {
            c -= w;
            r++;
        }
    }
};

// Rust `f32 as i32` (saturating, NaN -> 0) and WGSL i32(f32) for finite values.
__device__ __forceinline__ int32_t sat_f2i(float f) {
    if (f != f) return 0;
    if (f >= 2147483647.0f) return INT32_MAX;
    if (f <= -2147483648.0f) return INT32_MIN;
    return (int32_t)f;
}

// within_radius_rd2 (src/linking.rs:211-247): box prefilter per axis, then
// 0 + dx^2 + dy^2 (item - query) with strict `< r^2`.  Separate roundings.
__device__ __forceinline__ bool within_rd2(float ix, float iy, float qx, float qy, float radius, float* dist) {
    if (ix < __fsub_rn(qx, radius) || ix > __fadd_rn(qx, radius)) return false;
    if (iy < __fsub_rn(qy, radius) || iy > __fadd_rn(qy, radius)) return false;
    float r2 = __fmul_rn(radius, radius);
    float dx = __fsub_rn(ix, qx);
    float dy = __fsub_rn(iy, qy);
    float s = __fadd_rn(0.0f, __fmul_rn(dx, dx));
    s = __fadd_rn(s, __fmul_rn(dy, dy));
    *dist = s;
    return s < r2;
}

template <typename T>
__device__ __forceinline__ float load_px(const T* p, size_t i) {
    return (float)p[i];
}
template <>
__device__ __forceinline__ float load_px<float>(const float* p, size_t i) {
    return __ldg(p + i);
}
template <>
__device__ __forceinline__ float load_px<uint16_t>(const uint16_t* p, size_t i) {
    return (float)__ldg(p + i);
}
template <>
__device__ __forceinline__ float load_px<uint8_t>(const uint8_t* p, size_t i) {
    return (float)__ldg(p + i);
}

// Block-wide bitonic sort of n 64-bit keys (ascending); pads to a power of two.
__device__ __forceinline__ void block_sort_u64(uint64_t* keys, int n_pow2) {
    for (int k = 2; k <= n_pow2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < n_pow2; i += blockDim.x) {
                int ixj = i ^ j;
                if (ixj > i) {
                    uint64_t a = keys[i], b = keys[ixj];
                    bool up = ((i & k) == 0);
                    if ((a > b) == up) {
                        keys[i] = b;
                        keys[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Block-wide exclusive scan of one int per thread (blockDim <= 1024).
__device__ __forceinline__ int block_excl_scan(int v, int* total, int* wsum) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int incl = v;
    for (int d = 1; d < 32; d <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += t;
    }
    __syncthreads();
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int x = (lane < nw) ? wsum[lane] : 0;
        int s = x;
        for (int d = 1; d < 32; d <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= d) s += t;
        }
        if (lane < nw) wsum[lane] = s - x;
        if (lane == 31) wsum[32] = s;
    }
    __syncthreads();
    *total = wsum[32];
    return wsum[wid] + incl - v;
}

// Block-wide exclusive scan of one 64-bit value per thread (blockDim <= 1024).
__device__ __forceinline__ long long block_excl_scan64(long long v, long long* total, long long* wsum) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    long long incl = v;
    for (int d = 1; d < 32; d <<= 1) {
        long long t = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += t;
    }
    __syncthreads();
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        long long x = (lane < nw) ? wsum[lane] : 0;
        long long s = x;
        for (int d = 1; d < 32; d <<= 1) {
            long long t = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= d) s += t;
        }
        if (lane < nw) wsum[lane] = s - x;
        if (lane == 31) wsum[32] = s;
    }
    __syncthreads();
    *total = wsum[32];
    return wsum[wid] + incl - v;
}

}  // namespace gt
