// gt_log.cu — multi-scale Laplacian-of-Gaussian kernels for sm_100a.
//
//   laplace_kernel       separable_log.wgsl driven by Laplace<2>
//                        (src/utils.rs:252-296): for one radius, the four
//                        separable passes of -(d2/du2 + d2/dv2) G_sigma fused in
//                        one tile kernel; the column-pass intermediates stay in
//                        shared memory.
//   logspace_max_kernel  logspace_max.wgsl: strict maximum against the 8 in-plane
//                        neighbours and the 8 neighbours (centre excluded) of the
//                        adjacent scales, positive response, processed >= threshold.
//   mean_frame_kernel    mean_from_iter (src/execute_gpu.rs:819-847).
#include <math.h>

#include "gt_kernels.h"

namespace gt {

constexpr int kLapTH = 32, kLapTW = 64, kLapThreads = 256;

size_t laplace_smem_bytes(int rint) {
    const int RH = kLapTH + 2 * rint, RW = kLapTW + 2 * rint;
    return ((size_t)RH * RW + 2 * (size_t)kLapTH * RW) * sizeof(float);
}

// One plane tile for one (frame, radius).  The order of floating-point
// operations per pixel is the reference's:
//   a = (sum_i d_i f[u+i,v]) * nd ; ra = (sum_j g_j a[u,v+j]) * ng ; L = 0 - ra
//   b = (sum_i g_i f[u+i,v]) * ng ; rb = (sum_j d_j b[u,v+j]) * nd ; L = L - rb
template <typename T>
__global__ void __launch_bounds__(kLapThreads)
laplace_kernel(const T* __restrict__ frames, int64_t frame_stride, float* __restrict__ planes, const LogConsts lc,
               const float* __restrict__ taps_g, const float* __restrict__ taps_d, const int32_t* __restrict__ tap_off,
               const int32_t* __restrict__ rints, const float* __restrict__ norm_g, const float* __restrict__ norm_d) {
    extern __shared__ float sm[];
    const int H = lc.H, W = lc.W;
    const int f = blockIdx.z / lc.n_radii, k = blockIdx.z % lc.n_radii;
    const int rint = rints[k];
    const float* tg = taps_g + tap_off[k];
    const float* td = taps_d + tap_off[k];
    const float ng = norm_g[k], nd = norm_d[k];
    const int r0 = blockIdx.y * kLapTH, c0 = blockIdx.x * kLapTW;
    const int RH = kLapTH + 2 * rint, RW = kLapTW + 2 * rint;
    float* sraw = sm;
    float* sa = sraw + RH * RW;
    float* sb = sa + kLapTH * RW;
    const T* img = frames + (size_t)f * frame_stride;
    for (int idx = threadIdx.x; idx < RH * RW; idx += blockDim.x) {
        int rr = idx / RW, cc = idx - rr * RW;
        int gr = r0 - rint + rr, gc = c0 - rint + cc;
        sraw[idx] = (gr >= 0 && gr < H && gc >= 0 && gc < W) ? load_px<T>(img, (size_t)gr * W + gc) : 0.0f;
    }
    __syncthreads();
    // dim 0 (along rows): derivative taps -> a, Gaussian taps -> b
    for (int idx = threadIdx.x; idx < kLapTH * RW; idx += blockDim.x) {
        int rr = idx / RW, cc = idx - rr * RW;
        int gr = r0 + rr;
        float sa_ = 0.0f, sb_ = 0.0f;
        for (int i = 0; i <= 2 * rint; i++) {
            int pu = gr + i - rint;
            if (pu < 0 || pu >= H) continue;
            float x = sraw[(rr + i) * RW + cc];
            sa_ = __fmaf_rn(td[i], x, sa_);
            sb_ = __fmaf_rn(tg[i], x, sb_);
        }
        sa[idx] = __fmul_rn(sa_, nd);
        sb[idx] = __fmul_rn(sb_, ng);
    }
    __syncthreads();
    // dim 1 (along columns) and the two subtractions
    float* out = planes + ((size_t)f * lc.n_radii + k) * H * W;
    for (int idx = threadIdx.x; idx < kLapTH * kLapTW; idx += blockDim.x) {
        int rr = idx / kLapTW, cc = idx - rr * kLapTW;
        int gr = r0 + rr, gc = c0 + cc;
        if (gr >= H || gc >= W) continue;
        float ra = 0.0f, rb = 0.0f;
        for (int j = 0; j <= 2 * rint; j++) {
            int pv = gc + j - rint;
            if (pv < 0 || pv >= W) continue;
            ra = __fmaf_rn(tg[j], sa[rr * RW + cc + j], ra);
            rb = __fmaf_rn(td[j], sb[rr * RW + cc + j], rb);
        }
        float L = __fsub_rn(0.0f, __fmul_rn(ra, ng));
        L = __fsub_rn(L, __fmul_rn(rb, nd));
        out[(size_t)gr * W + gc] = L;
    }
}

__device__ __forceinline__ bool max_in_plane(const float* __restrict__ pl, int H, int W, int i, int j, float center) {
    for (int li = -1; li < 2; li++) {
        for (int lj = -1; lj < 2; lj++) {
            if (li == 0 && lj == 0) continue;
            int x = i + li, y = j + lj;
            if (x < 0 || x >= H || y < 0 || y >= W) return false;
            if (__ldg(pl + (size_t)x * W + y) >= center) return false;
        }
    }
    return true;
}

__global__ void __launch_bounds__(256)
logspace_max_kernel(const float* __restrict__ planes, const float* __restrict__ processed, const LogConsts lc,
                    uint32_t* __restrict__ cand_count, uint32_t* __restrict__ cand_keys, uint32_t cand_cap,
                    uint32_t* __restrict__ flags) {
    __shared__ int wsum[33];
    __shared__ uint32_t s_base;
    const int H = lc.H, W = lc.W, n = lc.n_radii;
    const int f = blockIdx.y / n, k = blockIdx.y % n;
    const size_t npx = (size_t)H * W;
    const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    const float* mid = planes + ((size_t)f * n + k) * npx;
    const float* proc = processed + (size_t)f * npx;
    int is = 0;
    if (pix < npx) {
        int i = pix / W, j = pix - i * W;
        float center = __ldg(mid + pix);
        // logspace_max.wgsl:122: std_pic * snr * rough_snr_factor
        const float thr = lc.frame_std ? __fmul_rn(__fmul_rn(lc.frame_std[f], lc.snr), lc.rough) : lc.thr;
        if (!(__ldg(proc + pix) < thr) && !(center <= 0.0f) && max_in_plane(mid, H, W, i, j, center)) {
            bool ok = true;
            if (k > 0) ok = max_in_plane(mid - npx, H, W, i, j, center);
            if (ok && k < n - 1) ok = max_in_plane(mid + npx, H, W, i, j, center);
            is = ok ? 1 : 0;
        }
    }
    int tot;
    int pos = block_excl_scan(is, &tot, wsum);
    if (threadIdx.x == 0) s_base = tot > 0 ? atomicAdd(cand_count + blockIdx.y, (uint32_t)tot) : 0u;
    __syncthreads();
    if (is) {
        uint32_t q = s_base + pos;
        if (q < cand_cap) cand_keys[(size_t)blockIdx.y * cand_cap + q] = pix;
        else atomicOr(flags, kFlagCandOverflow);
    }
}

template <typename T>
__global__ void mean_frame_kernel(const T* __restrict__ frames, int64_t T_, int64_t npix, float* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    float acc = 0.0f;
    for (int64_t t = 0; t < T_; t++) acc = __fadd_rn(acc, load_px<T>(frames, (size_t)t * npix + i));
    out[i] = __fdiv_rn(acc, (float)T_);
}

template <typename T>
cudaError_t launch_laplace(const T* frames, int64_t frame_stride, float* planes, const LogConsts& lc,
                           const float* taps_g, const float* taps_d, const int32_t* tap_off, const int32_t* rints,
                           const float* norm_g, const float* norm_d, int max_rint, int nframes, cudaStream_t st) {
    dim3 grid((lc.W + kLapTW - 1) / kLapTW, (lc.H + kLapTH - 1) / kLapTH, nframes * lc.n_radii);
    size_t smem = laplace_smem_bytes(max_rint);
    cudaFuncSetAttribute(laplace_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    laplace_kernel<T><<<grid, kLapThreads, smem, st>>>(frames, frame_stride, planes, lc, taps_g, taps_d, tap_off,
                                                       rints, norm_g, norm_d);
    return cudaGetLastError();
}

cudaError_t launch_logspace_max(const float* planes, const float* processed, const LogConsts& lc, int nframes,
                                uint32_t* cand_count, uint32_t* cand_keys, uint32_t cand_cap, uint32_t* flags,
                                cudaStream_t st) {
    const size_t npx = (size_t)lc.H * lc.W;
    dim3 grid((unsigned)((npx + 255) / 256), nframes * lc.n_radii);
    logspace_max_kernel<<<grid, 256, 0, st>>>(planes, processed, lc, cand_count, cand_keys, cand_cap, flags);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_mean_frame(const T* frames, int64_t T_, int64_t npix, float* out, cudaStream_t st) {
    mean_frame_kernel<T><<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(frames, T_, npix, out);
    return cudaGetLastError();
}

#define GT_LOG_INST(T)                                                                                        \
    template cudaError_t launch_laplace<T>(const T*, int64_t, float*, const LogConsts&, const float*,          \
                                           const float*, const int32_t*, const int32_t*, const float*,         \
                                           const float*, int, int, cudaStream_t);                               \
    template cudaError_t launch_mean_frame<T>(const T*, int64_t, int64_t, float*, cudaStream_t);
GT_LOG_INST(uint16_t)
GT_LOG_INST(float)
GT_LOG_INST(uint8_t)

}  // namespace gt
