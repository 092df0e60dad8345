// gt_logss.cu — fused multi-scale LoG scale space for sm_100a.
//
// One CTA owns a 16 x 128 output tile of one frame and computes, radius by
// radius, the Laplacian-of-Gaussian plane of every scale (separable_log.wgsl
// as driven by Laplace<2>, src/utils.rs:252-296) and the 3x3x3 scale-space
// maximum test (logspace_max.wgsl:97-154) without writing a plane to memory:
//
//   raw tile   the frame's pixels around the tile, staged once for all radii
//              (halo of the largest radius + 1), zero outside the frame;
//   pass A     vertical taps of one radius: a = (sum_i d_i f[u+i, v]) * nd and
//              b = (sum_i g_i f[u+i, v]) * ng, for the tile rows +- 1 and the
//              tile columns +- (1 + rint);
//   pass B     horizontal taps: L = (0 - (sum_j g_j a[u, v+j]) * ng)
//                                   - (sum_j d_j b[u, v+j]) * nd
//              for the tile +- 1, into a ring of three planes;
//   maxima     once plane k is in the ring, plane k-1's pixels are tested
//              against their 8 neighbours in planes k-1 and (without the
//              centre) k-2 and k, strict, and appended to the candidate list
//              of (frame, radius k-1).
//
// Every sum is the reference's sequential fused multiply-add chain in tap
// order, so the planes equal the reference's wherever the reference's result
// is not a zero: taps that fall outside the frame read the zero padding
// instead of being skipped, which can only turn a -0 into a +0, and the
// maximum test (> 0, >= comparisons) does not tell the two apart.  Tap counts
// are compile-time (one specialisation per rint = 1..kLogSSMaxR), and the taps
// are applied in chunks whose windows sit in registers.
#include <math.h>

#include "gt_internal.cuh"
#include "gt_kernels.h"

namespace gt {

namespace {

constexpr int kSSTH = 16, kSSTW = 128, kSSThreads = 256;
constexpr int kSSCB = 10;                // pass B columns per task ((TW + 2) = 13 * 10: one round of 234 tasks)
constexpr int kSSBatch = 8;              // raw-tile loads a thread keeps in flight
static_assert((kSSTW + 2) % kSSCB == 0, "pass B column blocks");
constexpr int kSSPW = kSSTW + 2;         // plane tile width (tile +- 1)
constexpr int kSSPH = kSSTH + 2;
// row stride of the raw tile and the pass A planes: fixed for every largest
// radius, so the vertical pass's tap loads are constant offsets
constexpr int kSSRW = kSSPW + 2 * kLogSSMaxR;

// Tap weights of every compile-time radius R (= rint) at offset R * R (radii
// 0 .. R-1 take sum(2r + 1) = R^2 slots), passed as a kernel parameter: a tap
// chain then reads its weights as constant-bank operands instead of one
// shared-memory load per tap.  Usable when the radii of a call have distinct
// rints (the host falls back to shared-memory taps otherwise).
constexpr int kSSParamTaps = (kLogSSMaxR + 1) * (kLogSSMaxR + 1);
struct SSTaps {
    float g[kSSParamTaps];
    float d[kSSParamTaps];
};

struct SSGeom {
    int RMAX, RH, RW;   // raw tile: RH rows of RW used columns (row stride kSSRW, as the pass A planes)
    size_t off_a, off_b, off_ring, off_taps, floats;
};

__host__ __device__ inline SSGeom ss_geom(int rmax, int ntaps_total) {
    SSGeom g;
    g.RMAX = rmax;
    g.RH = kSSPH + 2 * rmax;
    g.RW = kSSPW + 2 * rmax;
    g.off_a = (size_t)g.RH * kSSRW;
    g.off_b = g.off_a + (size_t)kSSPH * kSSRW;
    g.off_ring = g.off_b + (size_t)kSSPH * kSSRW;
    g.off_taps = g.off_ring + 3 * (size_t)kSSPH * kSSPW;
    g.floats = g.off_taps + 2 * (size_t)ntaps_total;
    return g;
}

// The taps of a chain are applied in chunks: a chunk needs a window of
// chunk + outputs - 1 values, so registers stay bounded for the largest radii
// while every chain keeps its sequential tap order.
template <int R>
struct SSChunk {
    static constexpr int value = R > 23 ? 4 : (R > 20 ? 8 : 16);
};

// Rows per pass A task for radius R: the plane's kSSPH rows of each of its
// kSSPW + 2R columns are split into tasks of RG rows; RG (a divisor of
// kSSPH) minimises the thread rounds ceil(tasks / threads) * RG, the larger
// RG on a tie (a longer register window per loaded value).
template <int R>
struct SSRows {
    static constexpr int C = kSSPW + 2 * R;
    static constexpr int rounds(int rg) { return ((kSSPH / rg) * C + kSSThreads - 1) / kSSThreads * rg; }
    static constexpr int pick() {
        int best = 9;
        for (int rg : {6, 3, 2})
            if (rounds(rg) < rounds(best)) best = rg;
        return best;
    }
    static constexpr int value = pick();
    static_assert(kSSPH % value == 0, "row groups tile the plane rows");
};

// pass A of one radius: column `col` of the pass A planes, rows grp*RG ..
template <int R>
__device__ __forceinline__ void ss_pass_a(const float* __restrict__ raw, const SSGeom& g, float* __restrict__ sa,
                                          float* __restrict__ sb, const float* __restrict__ tg,
                                          const float* __restrict__ td, float ng, float nd) {
    constexpr int NT = 2 * R + 1;
    constexpr int kSSChunk = SSChunk<R>::value;
    constexpr int kSSRG = SSRows<R>::value, NGRP = kSSPH / kSSRG;
    const int ncols = kSSPW + 2 * R;
    for (int task = threadIdx.x; task < NGRP * ncols; task += kSSThreads) {
        const int grp = task / ncols;
        const int col = task - grp * ncols;
        const int u0 = grp * kSSRG;
        // plane row u0 + k, column col <-> raw row u0 + k + RMAX - R + i, raw column col + RMAX - R
        const float* src = raw + (size_t)(u0 + g.RMAX - R) * kSSRW + (col + g.RMAX - R);
        float aa[kSSRG], bb[kSSRG];
#pragma unroll
        for (int k = 0; k < kSSRG; k++) aa[k] = bb[k] = 0.0f;
#pragma unroll
        for (int i0 = 0; i0 < NT; i0 += kSSChunk) {
            constexpr int NXC = kSSChunk + kSSRG - 1;
            float x[NXC];
#pragma unroll
            for (int m = 0; m < NXC; m++)
                if (i0 + m < NT + kSSRG - 1) x[m] = src[(i0 + m) * kSSRW];
#pragma unroll
            for (int ii = 0; ii < kSSChunk; ii++) {
                if (i0 + ii < NT) {
                    const float d = td[i0 + ii], gg = tg[i0 + ii];
#pragma unroll
                    for (int k = 0; k < kSSRG; k++) {
                        aa[k] = __fmaf_rn(d, x[k + ii], aa[k]);
                        bb[k] = __fmaf_rn(gg, x[k + ii], bb[k]);
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < kSSRG; k++) {
            sa[(u0 + k) * kSSRW + col] = __fmul_rn(aa[k], nd);
            sb[(u0 + k) * kSSRW + col] = __fmul_rn(bb[k], ng);
        }
    }
}

// one horizontal chain block: acc[c] = sum_j t_j p[c + j], j = 0 .. NT-1 in order
template <int R>
__device__ __forceinline__ void ss_hchain(const float* __restrict__ p, const float* __restrict__ t, float* acc) {
    constexpr int NT = 2 * R + 1;
    constexpr int kSSChunk = SSChunk<R>::value;
#pragma unroll
    for (int c = 0; c < kSSCB; c++) acc[c] = 0.0f;
#pragma unroll
    for (int j0 = 0; j0 < NT; j0 += kSSChunk) {
        // the window is read in 8-byte pairs (p + j0 is 8-byte aligned: even
        // row stride, even task column, even chunk); a pair's second value
        // past the window is a loaded but unused float of the same tile row
        // or the next one
        constexpr int NXC = kSSChunk + kSSCB - 1;
        float x[NXC + 1];
#pragma unroll
        for (int m = 0; m < NXC; m += 2)
            if (j0 + m < NT + kSSCB - 1) {
                const float2 v2 = *reinterpret_cast<const float2*>(p + j0 + m);
                x[m] = v2.x;
                x[m + 1] = v2.y;
            }
#pragma unroll
        for (int jj = 0; jj < kSSChunk; jj++) {
            if (j0 + jj < NT) {
                const float tv = t[j0 + jj];
#pragma unroll
                for (int c = 0; c < kSSCB; c++) acc[c] = __fmaf_rn(tv, x[c + jj], acc[c]);
            }
        }
    }
}

// pass B of one radius: row u, columns cb*CB .. of the plane tile
template <int R>
__device__ __forceinline__ void ss_pass_b(const float* __restrict__ sa, const float* __restrict__ sb,
                                          const SSGeom& g, float* __restrict__ plane, const float* __restrict__ tg,
                                          const float* __restrict__ td, float ng, float nd) {
    constexpr int NB = kSSPW / kSSCB;
    for (int task = threadIdx.x; task < kSSPH * NB; task += kSSThreads) {
        const int u = task / NB;
        const int v0 = (task - u * NB) * kSSCB;
        // plane column v, tap j <-> pass A column v + j
        float ra[kSSCB], rb[kSSCB];
        ss_hchain<R>(sa + (size_t)u * kSSRW + v0, tg, ra);
        ss_hchain<R>(sb + (size_t)u * kSSRW + v0, td, rb);
#pragma unroll
        for (int c = 0; c < kSSCB; c++) {
            float L = __fsub_rn(0.0f, __fmul_rn(ra[c], ng));
            L = __fsub_rn(L, __fmul_rn(rb[c], nd));
            plane[u * kSSPW + v0 + c] = L;
        }
    }
}

template <int R>
__device__ void ss_radius(const float* raw, const SSGeom& g, float* sa, float* sb, float* plane, const float* tg,
                          const float* td, float ng, float nd) {
    ss_pass_a<R>(raw, g, sa, sb, tg, td, ng, nd);
    __syncthreads();
    ss_pass_b<R>(sa, sb, g, plane, tg, td, ng, nd);
}

#define GT_SS_CASES(X)                                                                                    \
    X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17) X(18) \
    X(19) X(20) X(21) X(22) X(23) X(24) X(25) X(26) X(27) X(28) X(29) X(30) X(31) X(32)

// strict maximum of `center` against the 8 neighbours of (u, v) in a plane tile
__device__ __forceinline__ bool ss_max_in_plane(const float* __restrict__ p, int u, int v, float center) {
#pragma unroll
    for (int du = -1; du <= 1; du++)
#pragma unroll
        for (int dv = -1; dv <= 1; dv++) {
            if (du == 0 && dv == 0) continue;
            if (p[(u + du) * kSSPW + v + dv] >= center) return false;
        }
    return true;
}

// logspace_max for radius slot km of the tile (planes in the ring)
__device__ void ss_maxima(const float* __restrict__ ring, int km, int n, int f, int r0, int c0, const LogConsts& lc,
                          const float* __restrict__ proc, uint32_t* __restrict__ cand_count,
                          uint32_t* __restrict__ cand_keys, uint32_t cand_cap, uint32_t* __restrict__ flags) {
    const int H = lc.H, W = lc.W;
    const float* mid = ring + (size_t)(km % 3) * kSSPH * kSSPW;
    const float* bot = km > 0 ? ring + (size_t)((km + 2) % 3) * kSSPH * kSSPW : nullptr;
    const float* top = km < n - 1 ? ring + (size_t)((km + 1) % 3) * kSSPH * kSSPW : nullptr;
    // logspace_max.wgsl:122: std_pic * snr * rough_snr_factor
    const float thr = lc.frame_std ? __fmul_rn(__fmul_rn(lc.frame_std[f], lc.snr), lc.rough) : lc.thr;
    const size_t slot = (size_t)f * n + km;
    uint32_t* keys = cand_keys + slot * cand_cap;
    for (int e0 = 0; e0 < kSSTH * kSSTW; e0 += kSSThreads) {
        const int e = e0 + threadIdx.x;
        const int u = e / kSSTW + 1, v = e % kSSTW + 1;
        const int gi = r0 + u - 1, gj = c0 + v - 1;
        bool is = false;
        if (gi > 0 && gi < H - 1 && gj > 0 && gj < W - 1) {
            const float center = mid[u * kSSPW + v];
            if (center > 0.0f && ss_max_in_plane(mid, u, v, center) && (!bot || ss_max_in_plane(bot, u, v, center)) &&
                (!top || ss_max_in_plane(top, u, v, center)))
                is = !(__ldg(proc + (size_t)gi * W + gj) < thr);
        }
        const unsigned ball = __ballot_sync(0xffffffffu, is);
        if (ball) {
            const int lane = threadIdx.x & 31;
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(cand_count + slot, (uint32_t)__popc(ball));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (is) {
                const uint32_t q = base + __popc(ball & ((1u << lane) - 1u));
                if (q < cand_cap) keys[q] = (uint32_t)gi * (uint32_t)W + (uint32_t)gj;
                else atomicOr(flags, kFlagCandOverflow);
            }
        }
    }
}

template <typename T, bool kPT>
__global__ void __launch_bounds__(kSSThreads, 2)
log_scale_space_kernel(const T* __restrict__ frames, int64_t frame_stride, const float* __restrict__ processed,
                       const LogConsts lc, const float* __restrict__ taps_g, const float* __restrict__ taps_d,
                       const int32_t* __restrict__ tap_off, const int32_t* __restrict__ rints,
                       const float* __restrict__ norm_g, const float* __restrict__ norm_d, int rmax, int ntaps_total,
                       uint32_t* __restrict__ cand_count, uint32_t* __restrict__ cand_keys, uint32_t cand_cap,
                       uint32_t* __restrict__ flags, const __grid_constant__ SSTaps tp) {
    extern __shared__ float4 ss_sm4[];
    float* sm = (float*)ss_sm4;
    const SSGeom g = ss_geom(rmax, ntaps_total);
    float* raw = sm;
    float* sa = sm + g.off_a;
    float* sb = sm + g.off_b;
    float* ring = sm + g.off_ring;
    float* stg = sm + g.off_taps;              // Gaussian taps of every radius
    float* std_ = stg + ntaps_total;           // second-derivative taps
    const int H = lc.H, W = lc.W, n = lc.n_radii;
    const int f = blockIdx.z;
    const int r0 = blockIdx.y * kSSTH, c0 = blockIdx.x * kSSTW;
    const T* img = frames + (size_t)f * frame_stride;
    const float* proc = processed + (size_t)f * H * W;
    if (!kPT)
        for (int i = threadIdx.x; i < ntaps_total; i += kSSThreads) {
            stg[i] = taps_g[i];
            std_[i] = taps_d[i];
        }
    // raw tile: rows r0 - 1 - RMAX .., columns c0 - 1 - RMAX .., zero outside
    // the frame; kSSBatch independent loads per thread are in flight before
    // their shared-memory stores
    // each thread's elements (row, column) stepped without a division per element
    const int gr0 = r0 - 1 - rmax, gc0 = c0 - 1 - rmax;
    TileRowCol rc(threadIdx.x, kSSThreads, g.RW);
    while (rc.r < g.RH) {
        float v[kSSBatch];
        int at[kSSBatch];
#pragma unroll
        for (int b = 0; b < kSSBatch; b++) {
            const int rr = rc.r, cc = rc.c;
            const int gr = gr0 + rr, gc = gc0 + cc;
            const bool in_tile = rr < g.RH;
            at[b] = in_tile ? rr * kSSRW + cc : -1;
            v[b] = (in_tile && gr >= 0 && gr < H && gc >= 0 && gc < W) ? load_px<T>(img, (size_t)gr * W + gc) : 0.0f;
            rc.advance();
        }
#pragma unroll
        for (int b = 0; b < kSSBatch; b++)
            if (at[b] >= 0) raw[at[b]] = v[b];
    }
    __syncthreads();
    for (int k = 0; k < n; k++) {
        const int R = rints[k];
        const float* tg = stg + tap_off[k];
        const float* td = std_ + tap_off[k];
        float* plane = ring + (size_t)(k % 3) * kSSPH * kSSPW;
        switch (R) {
#define GT_SS_CASE(RR)                                                                                 \
    case RR:                                                                                           \
        if (kPT)                                                                                       \
            ss_radius<RR>(raw, g, sa, sb, plane, tp.g + RR * RR, tp.d + RR * RR, norm_g[k], norm_d[k]); \
        else                                                                                           \
            ss_radius<RR>(raw, g, sa, sb, plane, tg, td, norm_g[k], norm_d[k]);                        \
        break;
            GT_SS_CASES(GT_SS_CASE)
#undef GT_SS_CASE
            default:
                break;
        }
        __syncthreads();
        if (k >= 1) ss_maxima(ring, k - 1, n, f, r0, c0, lc, proc, cand_count, cand_keys, cand_cap, flags);
    }
    ss_maxima(ring, n - 1, n, f, r0, c0, lc, proc, cand_count, cand_keys, cand_cap, flags);
}

}  // namespace

size_t log_scale_space_smem_bytes(int max_rint, int ntaps_total) {
    return ss_geom(max_rint, ntaps_total).floats * sizeof(float);
}

bool log_scale_space_supported(int max_rint, int ntaps_total) {
    return max_rint >= 0 && max_rint <= kLogSSMaxR && log_scale_space_smem_bytes(max_rint, ntaps_total) <= 227 * 1024;
}

template <typename T>
cudaError_t launch_log_scale_space(const T* frames, int64_t frame_stride, const float* processed, const LogConsts& lc,
                                   const float* taps_g, const float* taps_d, const int32_t* tap_off,
                                   const int32_t* rints, const float* norm_g, const float* norm_d, int max_rint,
                                   int ntaps_total, int nframes, uint32_t* cand_count, uint32_t* cand_keys,
                                   uint32_t cand_cap, uint32_t* flags, const float* h_taps_g, const float* h_taps_d,
                                   const int32_t* h_tap_off, const int32_t* h_rints, cudaStream_t st) {
    dim3 grid((lc.W + kSSTW - 1) / kSSTW, (lc.H + kSSTH - 1) / kSSTH, nframes);
    const size_t smem = log_scale_space_smem_bytes(max_rint, ntaps_total);
    // taps as a kernel parameter when every radius has its own rint
    static_assert(sizeof(SSTaps) + 512 <= 32764, "kernel parameters stay within the launch limit");
    SSTaps tp;
    bool param_taps = h_taps_g && h_taps_d && h_tap_off && h_rints;
    uint64_t seen[(kLogSSMaxR + 64) / 64] = {};
    for (int k = 0; param_taps && k < lc.n_radii; k++) {
        const int R = h_rints[k];
        if (R < 0 || R > kLogSSMaxR || (seen[R / 64] >> (R % 64) & 1u)) {
            param_taps = false;
            break;
        }
        seen[R / 64] |= 1ull << (R % 64);
        for (int i = 0; i < 2 * R + 1; i++) {
            tp.g[R * R + i] = h_taps_g[h_tap_off[k] + i];
            tp.d[R * R + i] = h_taps_d[h_tap_off[k] + i];
        }
    }
    if (param_taps) {
        cudaFuncSetAttribute(log_scale_space_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        log_scale_space_kernel<T, true><<<grid, kSSThreads, smem, st>>>(
            frames, frame_stride, processed, lc, taps_g, taps_d, tap_off, rints, norm_g, norm_d, max_rint, ntaps_total,
            cand_count, cand_keys, cand_cap, flags, tp);
    } else {
        cudaFuncSetAttribute(log_scale_space_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        log_scale_space_kernel<T, false><<<grid, kSSThreads, smem, st>>>(
            frames, frame_stride, processed, lc, taps_g, taps_d, tap_off, rints, norm_g, norm_d, max_rint, ntaps_total,
            cand_count, cand_keys, cand_cap, flags, tp);
    }
    return cudaGetLastError();
}

#define GT_SS_INST(T)                                                                                          \
    template cudaError_t launch_log_scale_space<T>(const T*, int64_t, const float*, const LogConsts&, const float*, \
                                                   const float*, const int32_t*, const int32_t*, const float*,       \
                                                   const float*, int, int, int, uint32_t*, uint32_t*, uint32_t,      \
                                                   uint32_t*, const float*, const float*, const int32_t*,            \
                                                   const int32_t*, cudaStream_t);
GT_SS_INST(uint16_t)
GT_SS_INST(float)
GT_SS_INST(uint8_t)

}  // namespace gt
