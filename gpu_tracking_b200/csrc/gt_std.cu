// gt_std.cu — per-frame std (snr / minmass_snr) and the adaptive background
// filter, for a chunk of frames at a time.
//
// The std is the reference's StdArray (src/utils.rs:297-640) as a fixed tree
// of sums, reproduced level by level so every sum has the same operands in
// the same order:
//   mean:     s = N/8 outputs, each the sequential sum of 8 pixels s apart
//             (sum_image_outplace.wgsl; masked pixels left out), then levels
//             of 8 values L/8 apart while L > 24 (sum_image_inplace.wgsl),
//             then the sequential sum of the rest / divisor (last_reduction);
//   variance: the same tree over (x - mean)^2 (0 where masked, std_image.wgsl),
//             starting from N, then / (divisor - 1) and sqrt.
// Only pixel counts whose levels all divide by 8 are accepted by the host
// (the reference's in-place levels read stale buffer contents otherwise).
//
// Adaptive filter (adaptive_filter.wgsl, src/execute_gpu.rs:289-366): one
// thread per walked row tests mass against minmass (minmass_snr * count *
// std when minmass is not positive) and max_intensity against snr * std; an
// accepted row masks its circle in a per-frame byte mask and takes its count
// off the frame's divisor.  The std of the masked frame is recomputed before
// every pass but the first.  Accepted rows are then compacted in place.
#include <math.h>

#include "gt_internal.cuh"
#include "gt_kernels.h"

namespace gt {

template <typename T>
__device__ __forceinline__ bool pixel_masked(const T* img, const uint8_t* mask, int64_t i, float v) {
    (void)img;
    bool m = mask != nullptr && mask[i] != 0;
    // the reference marks masked pixels by the bit pattern 0xFFFFFFFF in its
    // f32 frame; an f32 input pixel with that pattern counts as masked too
    if (std::is_same<T, float>::value) m = m || (__float_as_uint(v) == 0xFFFFFFFFu);
    return m;
}

template <typename T>
__global__ void std_mean0_kernel(const T* __restrict__ frames, int64_t frame_stride, const uint8_t* __restrict__ mask,
                                 int64_t N, int64_t s, float* __restrict__ out) {
    const int f = blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s) return;
    const T* img = frames + (size_t)f * frame_stride;
    const uint8_t* mk = mask ? mask + (size_t)f * N : nullptr;
    float sum = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int64_t idx = i + k * s;
        const float v = load_px<T>(img, (size_t)idx);
        if (!pixel_masked<T>(img, mk, idx, v)) sum = __fadd_rn(sum, v);
    }
    out[(size_t)f * s + i] = sum;
}

template <typename T>
__global__ void std_var0_kernel(const T* __restrict__ frames, int64_t frame_stride, const uint8_t* __restrict__ mask,
                                int64_t N, int64_t t, const float* __restrict__ mean, float* __restrict__ out) {
    const int f = blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t) return;
    const T* img = frames + (size_t)f * frame_stride;
    const uint8_t* mk = mask ? mask + (size_t)f * N : nullptr;
    const float m = mean[f];
    float sum = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int64_t idx = i + k * t;
        const float v = load_px<T>(img, (size_t)idx);
        float sq = 0.0f;
        if (!pixel_masked<T>(img, mk, idx, v)) {
            const float diff = __fsub_rn(v, m);
            sq = __fmul_rn(diff, diff);
        }
        sum = __fadd_rn(sum, sq);
    }
    out[(size_t)f * t + i] = sum;
}

// one level: out[f][i] = sum_k in[f][i + k t], i < t (input length 8t)
__global__ void std_level_kernel(const float* __restrict__ in, int64_t in_len, float* __restrict__ out, int64_t t) {
    const int f = blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t) return;
    const float* a = in + (size_t)f * in_len;
    float sum = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; k++) sum = __fadd_rn(sum, a[i + k * t]);
    out[(size_t)f * t + i] = sum;
}

// last_reduction.wgsl: sequential sum of L values, / divisor (mean) or
// / (divisor - 1) then sqrt (std); one thread per frame
__global__ void std_final_kernel(const float* __restrict__ in, int64_t in_len, int64_t L,
                                 const uint32_t* __restrict__ divisors, uint32_t divisor, int variance,
                                 float* __restrict__ out, int nframes) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nframes) return;
    const float* a = in + (size_t)f * in_len;
    float acc = 0.0f;
    for (int64_t i = 0; i < L; i++) acc = __fadd_rn(acc, a[i]);
    const uint32_t d = divisors ? divisors[f] : divisor;
    if (variance) {
        acc = __fdiv_rn(acc, (float)(d - 1u));
        acc = __fsqrt_rn(acc);
    } else {
        acc = __fdiv_rn(acc, (float)d);
    }
    out[f] = acc;
}

bool std_reduction_exact(int64_t N) {
    if (N <= 0 || N % 8) return false;
    for (int64_t L : {N / 8, N}) {
        while (L > 24) {
            if (L % 8) return false;
            L /= 8;
        }
    }
    return true;
}

size_t std_scratch_floats(int64_t N, int nframes) {
    // two ping-pong level buffers: N/8 and N/64 values per frame, plus the means
    return (size_t)nframes * ((size_t)(N / 8) + (size_t)(N / 64) + 1) + 64;
}

template <typename T>
cudaError_t launch_frame_std(const T* frames, int64_t frame_stride, int nframes, int64_t N, const uint8_t* mask,
                             const uint32_t* divisors, float* out_std, float* scratch, cudaStream_t st) {
    if (nframes <= 0) return cudaSuccess;
    const int64_t s = N / 8;
    float* bufA = scratch;                                  // nframes * N/8
    float* bufB = bufA + (size_t)nframes * s;               // nframes * N/64
    float* mean = bufB + (size_t)nframes * (N / 64);        // nframes
    const uint32_t uN = (uint32_t)N;
    auto levels = [&](int64_t L) -> const float* {
        // the level outputs alternate between bufA (length L) and bufB
        const float* in = bufA;
        float* outp = bufB;
        while (L > 24) {
            const int64_t t = L / 8;
            dim3 grid((unsigned)((t + 255) / 256), nframes);
            std_level_kernel<<<grid, 256, 0, st>>>(in, L, outp, t);
            L = t;
            const float* nin = outp;
            outp = (outp == bufB) ? bufA : bufB;
            in = nin;
        }
        return in;
    };
    auto tail_len = [](int64_t L) {
        while (L > 24) L /= 8;
        return L;
    };
    {
        dim3 grid((unsigned)((s + 255) / 256), nframes);
        std_mean0_kernel<T><<<grid, 256, 0, st>>>(frames, frame_stride, mask, N, s, bufA);
        // the last level holds L values per frame, at a per-frame stride of L
        const float* r = levels(s);
        const int64_t L = tail_len(s);
        std_final_kernel<<<(nframes + 127) / 128, 128, 0, st>>>(r, L, L, divisors, uN, 0, mean, nframes);
    }
    {
        const int64_t t = N / 8;
        dim3 grid((unsigned)((t + 255) / 256), nframes);
        std_var0_kernel<T><<<grid, 256, 0, st>>>(frames, frame_stride, mask, N, t, mean, bufA);
        const float* r = levels(t);
        const int64_t L = tail_len(t);
        std_final_kernel<<<(nframes + 127) / 128, 128, 0, st>>>(r, L, L, divisors, uN, 1, out_std, nframes);
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------ adaptive filter
__global__ void adaptive_init_kernel(uint32_t* counters, uint32_t N, uint8_t* status, size_t n_status, int nframes) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < (size_t)nframes) counters[i] = N;
    if (i < n_status) status[i] = 0;
}

__global__ void adaptive_pass_kernel(const Feature* __restrict__ feats, const uint32_t* __restrict__ count,
                                     uint32_t feat_cap, uint8_t* __restrict__ status,
                                     const float* __restrict__ frame_std, float minmass, float minmass_snr, float snr,
                                     uint8_t* __restrict__ mask, uint32_t* __restrict__ counters, int32_t H,
                                     int32_t W, int32_t circle) {
    const int f = blockIdx.y;
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= min(count[f], feat_cap)) return;
    uint8_t& st = status[(size_t)f * feat_cap + j];
    if (st) return;
    const Feature& r = feats[(size_t)f * feat_cap + j];
    const float sd = frame_std[f];
    float mm;
    if (minmass > 0.0f) mm = minmass;
    else mm = __fmul_rn(__fmul_rn(minmass_snr, r.count), sd);
    if ((r.mass < mm) || (r.max_i < __fmul_rn(snr, sd))) return;  // stays for the next pass
    st = 1;
    // set_nan: the row's circle (radius ceil(r), or (diameter - 1) / 2)
    const int rint = (r.r > 0.0f) ? sat_f2i(ceilf(r.r)) : (circle - 1) / 2;
    const int u = sat_f2i(rintf(r.x)), v = sat_f2i(rintf(r.y));
    const float rf = (float)rint;
    const float r2 = __fmul_rn(rf, rf);
    uint8_t* mk = mask + (size_t)f * H * W;
    for (int i = -rint; i <= rint; i++) {
        const float x = (float)i;
        const float x2 = __fmul_rn(x, x);
        for (int jj = -rint; jj <= rint; jj++) {
            const float y = (float)jj;
            if (__fadd_rn(x2, __fmul_rn(y, y)) > r2) continue;
            const int pu = u + i, pv = v + jj;
            if (pu < 0 || pu >= H || pv < 0 || pv >= W) continue;
            mk[(size_t)pu * W + pv] = 1;
        }
    }
    const float c = r.count;
    const uint32_t cu = (c > 0.0f) ? ((c >= 4294967295.0f) ? 0xFFFFFFFFu : (uint32_t)c) : 0u;
    atomicSub(counters + f, cu);
}

// stable in-place compaction of the accepted rows; one CTA per frame
__global__ void adaptive_compact_kernel(Feature* __restrict__ feats, uint32_t* __restrict__ count, uint32_t feat_cap,
                                        const uint8_t* __restrict__ status) {
    __shared__ int wsum[33];
    const int f = blockIdx.x;
    const int n = (int)min(count[f], feat_cap);
    Feature* F = feats + (size_t)f * feat_cap;
    const uint8_t* S = status + (size_t)f * feat_cap;
    int total = 0;
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int keep = (i < n && S[i]) ? 1 : 0;
        Feature ft;
        if (keep) ft = F[i];
        int tot;
        const int pos = block_excl_scan(keep, &tot, wsum);
        // every read of this round happened before the scan's barriers; the
        // writes go to positions <= their sources, none of a later round
        if (keep) F[total + pos] = ft;
        total += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) count[f] = (uint32_t)total;
}

cudaError_t launch_adaptive_init(uint32_t* counters, uint32_t N, uint8_t* status, size_t n_status, int nframes,
                                 cudaStream_t st) {
    const size_t n = std::max<size_t>(n_status, (size_t)nframes);
    if (n == 0) return cudaSuccess;
    adaptive_init_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(counters, N, status, n_status, nframes);
    return cudaGetLastError();
}

cudaError_t launch_adaptive_pass(const Feature* feats, const uint32_t* count, uint32_t feat_cap, uint8_t* status,
                                 const float* frame_std, float minmass, float minmass_snr, float snr, uint8_t* mask,
                                 uint32_t* counters, int32_t H, int32_t W, int32_t circle, int nframes,
                                 cudaStream_t st) {
    if (nframes <= 0) return cudaSuccess;
    dim3 grid((feat_cap + 255) / 256, nframes);
    adaptive_pass_kernel<<<grid, 256, 0, st>>>(feats, count, feat_cap, status, frame_std, minmass, minmass_snr, snr,
                                               mask, counters, H, W, circle);
    return cudaGetLastError();
}

cudaError_t launch_adaptive_compact(Feature* feats, uint32_t* count, uint32_t feat_cap, const uint8_t* status,
                                    int nframes, cudaStream_t st) {
    if (nframes <= 0) return cudaSuccess;
    adaptive_compact_kernel<<<nframes, 1024, 0, st>>>(feats, count, feat_cap, status);
    return cudaGetLastError();
}

#define GT_STD_INST(T)                                                                                           \
    template cudaError_t launch_frame_std<T>(const T*, int64_t, int, int64_t, const uint8_t*, const uint32_t*, \
                                             float*, float*, cudaStream_t);
GT_STD_INST(uint16_t)
GT_STD_INST(float)
GT_STD_INST(uint8_t)
#undef GT_STD_INST

// --------------------------------------------------- illumination correction
// smooth_mean_frame.wgsl, one pass (dim 0: along the rows' direction, u =
// row; dim 1: along the columns): out = sum_i g_i * in / sum_i g_i over the
// in-frame taps, the products accumulated by fused multiply-adds.  n_frames
// is 1 in every call of the reference, so dim 0's norm is the tap sum.
template <typename TIn>
__global__ void illum_smooth_kernel(const TIn* __restrict__ in, int64_t in_stride, float* __restrict__ out, int H,
                                    int W, int dim, const float* __restrict__ g, int rint) {
    const int f = blockIdx.z;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (c >= W || r >= H) return;
    const TIn* src = in + (size_t)f * in_stride;
    const int u = dim == 0 ? r : c;
    const int bound = dim == 0 ? H : W;
    float gsum = 0.0f, nsum = 0.0f;
    for (int i = -rint; i <= rint; i++) {
        const int pu = u + i;
        if (pu < 0 || pu >= bound) continue;
        const size_t idx = dim == 0 ? (size_t)pu * W + c : (size_t)r * W + pu;
        const float gv = __ldg(g + i + rint);
        gsum = __fmaf_rn(gv, load_px<TIn>(src, idx), gsum);
        nsum = __fadd_rn(nsum, gv);
    }
    out[(size_t)f * H * W + (size_t)r * W + c] = __fdiv_rn(gsum, nsum);
}

// correct_illumination.wgsl: frame / profile, per pixel
template <typename T>
__global__ void illum_divide_kernel(const T* __restrict__ frames, int64_t frame_stride, const float* __restrict__ prof,
                                    int64_t prof_stride, float* __restrict__ out, int64_t out_stride, int64_t N) {
    const int f = blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    out[(size_t)f * out_stride + i] =
        __fdiv_rn(load_px<T>(frames + (size_t)f * frame_stride, (size_t)i), prof[(size_t)f * prof_stride + i]);
}

template <typename TIn>
cudaError_t launch_illum_smooth(const TIn* in, int64_t in_stride, float* out, int H, int W, int dim, const float* g,
                                int rint, int nframes, cudaStream_t st) {
    if (nframes <= 0) return cudaSuccess;
    dim3 grid((W + 127) / 128, H, nframes);
    illum_smooth_kernel<TIn><<<grid, 128, 0, st>>>(in, in_stride, out, H, W, dim, g, rint);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_illum_divide(const T* frames, int64_t frame_stride, const float* prof, int64_t prof_stride,
                                float* out, int64_t out_stride, int nframes, cudaStream_t st) {
    if (nframes <= 0) return cudaSuccess;
    dim3 grid((unsigned)((out_stride + 255) / 256), nframes);
    illum_divide_kernel<T><<<grid, 256, 0, st>>>(frames, frame_stride, prof, prof_stride, out, out_stride, out_stride);
    return cudaGetLastError();
}

#define GT_ILLUM_INST(T)                                                                                      \
    template cudaError_t launch_illum_smooth<T>(const T*, int64_t, float*, int, int, int, const float*, int, int, \
                                                cudaStream_t);                                               \
    template cudaError_t launch_illum_divide<T>(const T*, int64_t, const float*, int64_t, float*, int64_t, int, \
                                                cudaStream_t);
GT_ILLUM_INST(uint16_t)
GT_ILLUM_INST(float)
GT_ILLUM_INST(uint8_t)
#undef GT_ILLUM_INST

}  // namespace gt
