// gt_cnn.cu — the learned proposal network: a 4-layer 3x3 convolutional net
// over the frame at stride 4 (each 4x4 pixel block is one 16-channel cell),
// BF16 weights and activations with FP32 accumulation on the tcgen05 tensor
// cores, and the kernels that train it (loss, weight gradients, Adam).
//
// Network (per cell of the 4x4 grid):
//   x   = (pixel - mean) * scale, 16 channels (pixel (dy, dx) of the block at 4*dy + dx)
//   a1  = relu(conv3x3(x, 16 -> 32) + b1)
//   a2  = relu(conv3x3(a1, 32 -> 32) + b2)
//   a3  = relu(conv3x3(a2, 32 -> 32) + b3)
//   out = conv3x3(a3, 32 -> 3) + b4: score logit, row offset, column offset
// The offsets are in pixels from the cell centre (4*cy + 1.5, 4*cx + 1.5).
// Convolutions pad with zeros ("same").  The parameter vector (fp32 master
// copy) stores each layer as W[co][ci][ky*3 + kx] followed by b[co].
//
// Activations are BF16 in planes of 8 channels: [image][C/8][Hc][Wc][8].
// Convolution as an implicit GEMM on the tensor cores: a CTA owns tiles of
// 16 rows x 8 cells (M = 128 rows of D), the output channels are N and K runs
// over the 9 taps x input channels.  One TMA box per tile (8 channels x 10
// cells x 18 rows x C/8 planes, the tile and its halo) lands in shared memory
// as [plane][row][10 cells][8 channels]: 8 consecutive cells of a row are one
// 128-byte K-major core matrix, so the operand of a tap (dy, dx) is a plain
// descriptor at row dy, cell dx (rows 160 bytes apart, planes one plane
// apart) and one UMMA of K = 16 covers a tap and 16 input channels.
// The CTA is warp-specialised and persistent over its tiles: warp 0 issues
// the TMA loads into a ring of staging buffers, one thread of warp 1 issues
// the UMMAs into a ring of TMEM accumulators (32 columns each), and warps
// 2-5 drain the accumulators (tcgen05.ld, bias, ReLU or the ReLU mask of the
// backward pass, BF16 planes out).  The roles hand buffers to each other
// through mbarriers only (full / empty per staging buffer, full / empty per
// accumulator), so loads, UMMAs and epilogues of different tiles overlap.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <mutex>

#include "gt_internal.cuh"
#include "gt_kernels.h"
#include "gt_tc.cuh"

namespace gt {

namespace {

constexpr int kConvRows = 16;     // tile rows (one core-matrix row of M each)
constexpr int kConvCols = 8;      // tile cells per row
constexpr uint32_t kConvPolls = 1u << 22;

template <int KS, int N>
struct ConvGeom {
    static constexpr int PLANES = 2 * KS;                 // 8-channel input planes
    static constexpr int RS = (kConvCols + 2) * 16;       // staged row: 10 cells x 16 bytes
    static constexpr int PLANE = (kConvRows + 2) * RS;    // one plane: 18 rows
    static constexpr int STAGE = ((PLANES * PLANE + 127) / 128) * 128;
    static constexpr int NSTAGE = 6;
    static constexpr int NACC = 4;                        // TMEM accumulators of 32 columns
    static constexpr int B_BYTES = 9 * KS * (N / 8) * 256;
    static constexpr int SMEM = 128 + NSTAGE * STAGE + B_BYTES + 128 + 8 * (2 * NSTAGE + 2 * NACC) + 16;
};
constexpr int kConvWsThreads = 320;  // warp 0 loads, warp 1 issues, warps 2-5 and 6-9 drain alternate tiles

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

// bf16 > 0: sign bit clear and not +0
__device__ __forceinline__ bool bf16_pos(uint32_t h) { return h != 0u && !(h & 0x8000u); }

// MODE 0: relu(acc + bias) -> bf16 planes (32 channels)
// MODE 1: acc + bias      -> float4 [cell] (score, row offset, column offset, 0), N = 16
// MODE 2: acc * (mask > 0) -> bf16 planes (backward through the ReLU of the layer below)
template <int KS, int N, int MODE>
__global__ void __launch_bounds__(kConvWsThreads)
conv3x3_kernel(const __grid_constant__ CUtensorMap tin, int nimg, int Hc, int Wc, const uint8_t* __restrict__ wpk,
               const float* __restrict__ bias, const __nv_bfloat16* __restrict__ mask, void* __restrict__ out,
               uint32_t* __restrict__ flags) {
    using G = ConvGeom<KS, N>;
    constexpr int NS = G::NSTAGE, NA = G::NACC;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* S0 = (uint8_t*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint8_t* B = S0 + NS * G::STAGE;
    float* sbias = (float*)(B + G::B_BYTES);  // [32]
    uint64_t* full = (uint64_t*)(sbias + 32);  // [NS] staging buffer loaded
    uint64_t* empty = full + NS;               // [NS] staging buffer consumed by its UMMAs
    uint64_t* accf = empty + NS;               // [NA] accumulator written
    uint64_t* acce = accf + NA;                // [NA] accumulator read by the 4 epilogue warps
    uint32_t* tslot = (uint32_t*)(acce + NA);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    for (int i = tid; i < G::B_BYTES / 16; i += kConvWsThreads) ((uint4*)B)[i] = __ldg((const uint4*)wpk + i);
    if (tid < 32) sbias[tid] = (bias && tid < (MODE == 1 ? 3 : 32)) ? bias[tid] : 0.0f;
    if (tid == 0) {
        for (int i = 0; i < 2 * NS + NA; i++) tc::mbar_init(full + i, 1);
        for (int i = 0; i < NA; i++) tc::mbar_init(acce + i, 4);
    }
    if (warp == 0) tc::tmem_alloc(tslot, 32 * NA);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;

    // tile counts fit in 32 bits (conv_launch checks)
    const int ntx = (Wc + kConvCols - 1) / kConvCols, nty = (Hc + kConvRows - 1) / kConvRows;
    const int per_img = nty * ntx;
    const int ntiles = nimg * per_img;
    const int t0 = blockIdx.x, stride = gridDim.x;
    // this CTA's tiles are t0 + k * stride, k = 0 .. nmine - 1
    const int nmine = t0 < ntiles ? (ntiles - 1 - t0) / stride + 1 : 0;
    auto tile_pos = [&](int k, int& img, int& y0, int& x0) {
        const int tile = t0 + k * stride;
        img = tile / per_img;
        const int rem = tile - img * per_img;
        const int ty = rem / ntx;
        y0 = ty * kConvRows;
        x0 = (rem - ty * ntx) * kConvCols;
    };

    if (warp == 0) {
        if (lane == 0) {
            // producer: stage k % NS is free again once tile k - NS's UMMAs completed
            int k = 0;
            for (; k < nmine; k++) {
                const int st = k % NS;
                if (k >= NS && !tc::mbar_wait_bounded(empty + st, (uint32_t)((k / NS - 1) & 1), kConvPolls)) {
                    atomicOr(flags, kFlagTensorTimeout);
                    break;
                }
                int img, y0, x0;
                tile_pos(k, img, y0, x0);
                tc::mbar_arrive_expect_tx(full + st, G::PLANES * G::PLANE);
                // innermost coordinate: element (x0 - 1) * 8 of the flattened row, 16-byte aligned
                tc::tma_load_3d(S0 + st * G::STAGE, &tin, (x0 - 1) * 8, y0 - 1, img * G::PLANES, full + st);
            }
            // no load may still be landing when the CTA leaves
            for (int j = max(0, k - NS); j < k; j++)
                tc::mbar_wait_bounded(full + j % NS, (uint32_t)((j / NS) & 1), kConvPolls);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_bf16_f32(128, N);
            // descriptors of stage 0 and of the weights; a stage or a tap is a
            // start-address offset (the low 14 bits, in 16-byte units)
            const uint64_t a_desc0 = tc::desc_kmajor(tc::smem_addr(S0), G::PLANE, G::RS);
            uint64_t b_desc[9 * KS];
#pragma unroll
            for (int j = 0; j < 9 * KS; j++) b_desc[j] = tc::desc_kmajor(tc::smem_addr(B) + j * (N / 8) * 256, 128, 256);
            int k = 0;
            for (; k < nmine; k++) {
                const int st = k % NS, ab = k % NA;
                if (!tc::mbar_wait_bounded(full + st, (uint32_t)((k / NS) & 1), kConvPolls) ||
                    (k >= NA && !tc::mbar_wait_bounded(acce + ab, (uint32_t)((k / NA - 1) & 1), kConvPolls))) {
                    atomicOr(flags, kFlagTensorTimeout);
                    break;
                }
                tc::fence_after_sync();
                const uint64_t a_desc = a_desc0 + (uint64_t)((st * G::STAGE) >> 4);
                uint32_t acc = 0;
#pragma unroll
                for (int t = 0; t < 9; t++) {
                    const int dy = t / 3, dx = t % 3;
#pragma unroll
                    for (int kk = 0; kk < KS; kk++) {
                        const uint64_t ad = a_desc + (uint64_t)((2 * kk * G::PLANE + dy * G::RS + dx * 16) >> 4);
                        tc::mma_bf16(tmem + 32 * ab, ad, b_desc[t * KS + kk], idesc, acc);
                        acc = 1;
                    }
                }
                tc::mma_commit(empty + st);
                tc::mma_commit(accf + ab);
            }
            // the accumulators of the issued tiles must be complete before TMEM is freed
            for (int j = max(0, k - NA); j < k; j++)
                tc::mbar_wait_bounded(accf + j % NA, (uint32_t)((j / NA) & 1), kConvPolls);
        }
    } else {
        // epilogue: warp w reads TMEM lanes 32 * (w % 4) .. + 31 = tile rows 4 * (w % 4) .. + 3;
        // warps 2-5 take the even tiles, warps 6-9 the odd ones
        const int sub = warp & 3, grp = (warp - 2) >> 2;
        for (int k = grp; k < nmine; k += 2) {
            const int ab = k % NA;
            const bool ready = tc::mbar_wait_bounded(accf + ab, (uint32_t)((k / NA) & 1), kConvPolls);
            if (!__all_sync(0xffffffffu, ready)) {
                if (lane == 0) atomicOr(flags, kFlagTensorTimeout);
                break;
            }
            tc::fence_after_sync();
            int img, y0, x0;
            tile_pos(k, img, y0, x0);
            const int gy = y0 + 4 * sub + (lane >> 3), gx = x0 + (lane & 7);
            const bool in_frame = gy < Hc && gx < Wc;
            const uint32_t taddr = tmem + 32 * ab + ((uint32_t)(32 * sub) << 16);
            if (MODE == 1) {
                uint32_t r[16];
                tc::tmem_ld16(taddr, r);
                tc::tmem_ld_wait();
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(acce + ab);
                if (in_frame) {
                    float4 o;
                    o.x = __fadd_rn(__uint_as_float(r[0]), sbias[0]);
                    o.y = __fadd_rn(__uint_as_float(r[1]), sbias[1]);
                    o.z = __fadd_rn(__uint_as_float(r[2]), sbias[2]);
                    o.w = 0.0f;
                    ((float4*)out)[((size_t)img * Hc + gy) * Wc + gx] = o;
                }
            } else {
                uint32_t r[32];
                tc::tmem_ld32(taddr, r);
                tc::tmem_ld_wait();
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(acce + ab);
                if (in_frame) {
                    float v[32];
#pragma unroll
                    for (int n = 0; n < 32; n++) v[n] = __uint_as_float(r[n]);
                    if (MODE == 0) {
#pragma unroll
                        for (int n = 0; n < 32; n++) v[n] = fmaxf(__fadd_rn(v[n], sbias[n]), 0.0f);
                    } else {
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            const uint4 m4 =
                                __ldg((const uint4*)(mask + ((((size_t)img * 4 + q) * Hc + gy) * Wc + gx) * 8));
                            const uint32_t mw[4] = {m4.x, m4.y, m4.z, m4.w};
#pragma unroll
                            for (int h = 0; h < 4; h++) {
                                if (!bf16_pos(mw[h] & 0xFFFFu)) v[8 * q + 2 * h] = 0.0f;
                                if (!bf16_pos(mw[h] >> 16)) v[8 * q + 2 * h + 1] = 0.0f;
                            }
                        }
                    }
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        *(uint4*)((__nv_bfloat16*)out + ((((size_t)img * 4 + q) * Hc + gy) * Wc + gx) * 8) =
                            make_uint4(pack_bf16x2(v[8 * q], v[8 * q + 1]), pack_bf16x2(v[8 * q + 2], v[8 * q + 3]),
                                       pack_bf16x2(v[8 * q + 4], v[8 * q + 5]),
                                       pack_bf16x2(v[8 * q + 6], v[8 * q + 7]));
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem, 32 * NA);
}

// The tensor map of a BF16 plane tensor [planes_total][Hc][Wc][8] seen as
// [planes_total][Hc][Wc * 8] (a plane row's cells and channels are one
// contiguous run): the box is one tile with its halo, 10 cells x 8 channels
// = 160 bytes per row, x 18 rows x planes_per_img planes.
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        else
            cudaGetLastError();
    });
    return fn;
}

cudaError_t plane_map(CUtensorMap* m, const void* base, int nimg, int planes_per_img, int Hc, int Wc) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn) return cudaErrorNotSupported;
    if (((uintptr_t)base & 15u) != 0u) return cudaErrorMisalignedAddress;
    const cuuint64_t dims[3] = {(cuuint64_t)Wc * 8, (cuuint64_t)Hc, (cuuint64_t)nimg * planes_per_img};
    const cuuint64_t strides[2] = {(cuuint64_t)Wc * 16, (cuuint64_t)Hc * Wc * 16};
    const cuuint32_t box[3] = {(cuuint32_t)(kConvCols + 2) * 8, (cuuint32_t)(kConvRows + 2), (cuuint32_t)planes_per_img};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int KS, int N, int MODE>
cudaError_t conv_launch(const __nv_bfloat16* in, int nimg, int Hc, int Wc, const uint8_t* wpk, const float* bias,
                        const __nv_bfloat16* mask, void* out, uint32_t* flags, int num_sms, cudaStream_t st) {
    using G = ConvGeom<KS, N>;
    const int64_t ntiles =
        (int64_t)nimg * ((Hc + kConvRows - 1) / kConvRows) * ((Wc + kConvCols - 1) / kConvCols);
    if (ntiles == 0) return cudaSuccess;
    if (ntiles > INT32_MAX) return cudaErrorInvalidValue;
    CUtensorMap tm;
    cudaError_t e = plane_map(&tm, in, nimg, G::PLANES, Hc, Wc);
    if (e != cudaSuccess) return e;
    // once per instantiation and device
    static std::atomic<uint64_t> attr_set{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = 1ull << (dev & 63);
    if (!(attr_set.load() & bit)) {
        e = cudaFuncSetAttribute(conv3x3_kernel<KS, N, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);
        if (e != cudaSuccess) return e;
        attr_set.fetch_or(bit);
    }
    // persistent: at most 2 CTAs per SM, 2 x 128 of the 512 TMEM columns
    static_assert(2 * G::SMEM <= 227 * 1024, "two CTAs per SM");
    const int64_t grid = std::min<int64_t>(ntiles, (int64_t)num_sms * 2);
    conv3x3_kernel<KS, N, MODE><<<(unsigned)grid, kConvWsThreads, G::SMEM, st>>>(tm, nimg, Hc, Wc, wpk, bias, mask,
                                                                                 out, flags);
    return cudaGetLastError();
}

// -------------------------------------------------------------- packing
// Packed B operand of one convolution: for tap t, K step k (16 input
// channels), N group g (8 output channels), K chunk c (8 input channels),
// row r, element e:  byte ((t*KS + k)*(N/8) + g)*256 + c*128 + r*16 + e*2.
// mode 0 (forward):  B[n][ci] = W[n][ci][t]
// mode 1 (backward): B[n][ci] = W[ci][n][8 - t] (input gradient: the
//                    transposed kernel, flipped), zero beyond the channels.
__global__ void cnn_pack_kernel(const float* __restrict__ W, int cin, int cout, int KS, int N, int mode,
                                __nv_bfloat16* __restrict__ dst) {
    const int total = 9 * KS * N * 16;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int e = idx & 7, r = (idx >> 3) & 7, c = (idx >> 6) & 1;
    const int rest = idx >> 7;              // (t*KS + k)*(N/8) + g
    const int g = rest % (N / 8), tk = rest / (N / 8);
    const int k = tk % KS, t = tk / KS;
    const int n = 8 * g + r, ci = 16 * k + 8 * c + e;
    float v = 0.0f;
    if (mode == 0) {
        if (n < cout && ci < cin) v = W[((size_t)n * cin + ci) * 9 + t];
    } else {
        // forward layer (cin, cout): here n runs over its cin, ci over its cout
        if (n < cin && ci < cout) v = W[((size_t)ci * cin + n) * 9 + (8 - t)];
    }
    dst[idx] = __float2bfloat16_rn(v);
}

// ------------------------------------------------- input (space to depth)
// Cell (cy, cx) of image i holds the 4x4 pixels from (oy + 4cy, ox + 4cx) of
// frame fi, channel 4*dy + dx, as (pixel - mean) * scale in BF16; pixels
// outside the frame read as the mean (0).  Without a crop table image i is
// frame i at offset (0, 0).  A crop (fi, oy, ox, aug) of a square Hc x Wc
// cell window is seen through one of the 8 symmetries of the square: pixel
// (a, b) of the crop reads source pixel aug_map(a, b) (swap the axes if bit 2,
// then mirror the rows if bit 0 and the columns if bit 1).
__device__ __forceinline__ void aug_map(int aug, int n, int& a, int& b) {
    if (aug & 4) {
        const int t = a;
        a = b;
        b = t;
    }
    if (aug & 1) a = n - 1 - a;
    if (aug & 2) b = n - 1 - b;
}
template <typename T>
__global__ void cnn_input_kernel(const T* __restrict__ frames, int64_t frame_stride, int H, int W,
                                 const int4* __restrict__ crops, int nimg, int Hc, int Wc, float mean, float scale,
                                 __nv_bfloat16* __restrict__ out) {
    const int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= (int64_t)nimg * Hc * Wc) return;
    const int img = (int)(cell / ((int64_t)Hc * Wc));
    const int rem = (int)(cell - (int64_t)img * Hc * Wc);
    const int cy = rem / Wc, cx = rem % Wc;
    int fi = img, oy = 0, ox = 0, aug = 0;
    if (crops) {
        const int4 cr = crops[img];
        fi = cr.x;
        oy = cr.y;
        ox = cr.z;
        aug = cr.w;
    }
    const T* f = frames + (size_t)fi * frame_stride;
    float v[16];
    const int yb = oy + 4 * cy, xb = ox + 4 * cx;
    if (!aug && yb + 3 < H && xb + 3 < W && (W & 3) == 0 && (frame_stride & 3) == 0) {
        // whole block inside the frame, rows of 4 pixels aligned to 4: one load per row
#pragma unroll
        for (int dy = 0; dy < 4; dy++) {
            const T* row = f + (size_t)(yb + dy) * W + xb;
            float q[4];
            if (sizeof(T) == 2) {
                const uint2 w = __ldg((const uint2*)row);
                q[0] = (float)(w.x & 0xFFFFu);
                q[1] = (float)(w.x >> 16);
                q[2] = (float)(w.y & 0xFFFFu);
                q[3] = (float)(w.y >> 16);
            } else if (sizeof(T) == 1) {
                const uint32_t w = __ldg((const uint32_t*)row);
                q[0] = (float)(w & 0xFFu);
                q[1] = (float)((w >> 8) & 0xFFu);
                q[2] = (float)((w >> 16) & 0xFFu);
                q[3] = (float)(w >> 24);
            } else {
                const float4 w = __ldg((const float4*)row);
                q[0] = w.x;
                q[1] = w.y;
                q[2] = w.z;
                q[3] = w.w;
            }
#pragma unroll
            for (int dx = 0; dx < 4; dx++) v[4 * dy + dx] = __fmul_rn(__fsub_rn(q[dx], mean), scale);
        }
    } else {
#pragma unroll
        for (int dy = 0; dy < 4; dy++)
#pragma unroll
            for (int dx = 0; dx < 4; dx++) {
                int a = 4 * cy + dy, b = 4 * cx + dx;
                if (aug) aug_map(aug, 4 * Hc, a, b);
                const int y = oy + a, x = ox + b;
                float p = 0.0f;
                if (y < H && x < W) p = __fmul_rn(__fsub_rn(load_px<T>(f, (size_t)y * W + x), mean), scale);
                v[4 * dy + dx] = p;
            }
    }
    // two planes of 8 channels
    const size_t plane = (size_t)Hc * Wc;
    uint4* o0 = (uint4*)(out + ((size_t)img * 2 * plane + rem) * 8);
    uint4* o1 = (uint4*)(out + (((size_t)img * 2 + 1) * plane + rem) * 8);
    *o0 = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                     pack_bf16x2(v[6], v[7]));
    *o1 = make_uint4(pack_bf16x2(v[8], v[9]), pack_bf16x2(v[10], v[11]), pack_bf16x2(v[12], v[13]),
                     pack_bf16x2(v[14], v[15]));
}

// ---------------------------------------------------------------- labels
constexpr int32_t kLabelFree = 0x7F7F7F7F;  // byte-fill value of an unclaimed cell
// Target map of each frame: the lowest-index label whose pixel lies in a
// cell owns it; (1, row offset, column offset) from the cell centre.
__global__ void cnn_label_claim_kernel(const int32_t* __restrict__ lf, const float* __restrict__ ly,
                                       const float* __restrict__ lx, int64_t n, int Hc, int Wc,
                                       int32_t* __restrict__ owner) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float y = ly[i], x = lx[i];
    if (!(y >= 0.0f) || !(x >= 0.0f)) return;
    const int cy = (int)(y * 0.25f), cx = (int)(x * 0.25f);
    if (cy >= Hc || cx >= Wc) return;
    atomicMin(owner + ((size_t)lf[i] * Hc + cy) * Wc + cx, (int32_t)i);
}
__global__ void cnn_label_write_kernel(const float* __restrict__ ly, const float* __restrict__ lx,
                                       const int32_t* __restrict__ owner, int64_t ncells, int Hc, int Wc,
                                       float4* __restrict__ tmap) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    const int32_t o = owner[c];
    float4 t = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (o != kLabelFree) {
        const int rem = (int)(c % ((int64_t)Hc * Wc));
        const int cy = rem / Wc, cx = rem % Wc;
        t.x = 1.0f;
        t.y = ly[o] - (4.0f * cy + 1.5f);
        t.z = lx[o] - (4.0f * cx + 1.5f);
    }
    tmap[c] = t;
}

// Random crops of CH x CW cells, cell-aligned, inside their frame: a hash of
// (seed, step, crop) picks the frame, the offset and (for square crops) one
// of the 8 symmetries of the square.
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
__global__ void cnn_crop_kernel(uint32_t seed, uint32_t step, int nimg, int T, int Hc, int Wc, int CH, int CW,
                                int augment, int4* __restrict__ crops) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nimg) return;
    const uint32_t h0 = mix32(seed ^ mix32(step * 0x9E3779B9u + (uint32_t)i * 0x85EBCA6Bu));
    const uint32_t h1 = mix32(h0 + 0x632BE5ABu), h2 = mix32(h1 + 0x2545F491u), h3 = mix32(h2 + 0x1B873593u);
    const int f = (int)(h0 % (uint32_t)T);
    const int cy = (int)(h1 % (uint32_t)(Hc - CH + 1)), cx = (int)(h2 % (uint32_t)(Wc - CW + 1));
    crops[i] = make_int4(f, 4 * cy, 4 * cx, augment ? (int)(h3 & 7u) : 0);
}

// ------------------------------------------------------------------ loss
// Per cell: pos_weight * y * softplus(-s) + (1 - y) * softplus(s) for the
// score, lambda * y * |offset - target|^2 for the offsets, averaged over the
// cells; gradients into a 16-channel BF16 cell (channels 3..15 zero).
__global__ void cnn_loss_kernel(const float4* __restrict__ head, const float4* __restrict__ tmap,
                                const int4* __restrict__ crops, int nimg, int CH, int CW, int Hc_f, int Wc_f,
                                float pos_weight, float lambda, __nv_bfloat16* __restrict__ grad,
                                float* __restrict__ partial) {
    __shared__ float red[2][8];
    const int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t ncell = (int64_t)nimg * CH * CW;
    float ls = 0.0f, lo = 0.0f;
    if (cell < ncell) {
        const int img = (int)(cell / (CH * CW));
        const int rem = (int)(cell - (int64_t)img * CH * CW);
        const int cy = rem / CW, cx = rem % CW;
        const int4 cr = crops[img];
        int sy = cy, sx = cx;
        if (cr.w) aug_map(cr.w, CH, sy, sx);
        float4 t = tmap[((size_t)cr.x * Hc_f + cr.y / 4 + sy) * Wc_f + cr.z / 4 + sx];
        // the offset vector seen through the symmetry: mirrors negate, the swap exchanges
        if (cr.w & 1) t.y = -t.y;
        if (cr.w & 2) t.z = -t.z;
        if (cr.w & 4) {
            const float q = t.y;
            t.y = t.z;
            t.z = q;
        }
        const float4 o = head[cell];
        const float s = o.x, y = t.x;
        const float sp_pos = fmaxf(-s, 0.0f) + log1pf(expf(-fabsf(s)));  // softplus(-s)
        const float sp_neg = fmaxf(s, 0.0f) + log1pf(expf(-fabsf(s)));   // softplus(s)
        const float sig = 1.0f / (1.0f + expf(-s));
        const float inv = 1.0f / (float)ncell;
        ls = pos_weight * y * sp_pos + (1.0f - y) * sp_neg;
        const float gs = (pos_weight * y * (sig - 1.0f) + (1.0f - y) * sig) * inv;
        const float ey = o.y - t.y, ex = o.z - t.z;
        lo = lambda * y * (ey * ey + ex * ex);
        const float gy = 2.0f * lambda * y * ey * inv, gx = 2.0f * lambda * y * ex * inv;
        // two planes of 8 channels: the three gradients, then zeros
        const size_t plane = (size_t)CH * CW;
        *(uint4*)(grad + ((size_t)img * 2 * plane + rem) * 8) =
            make_uint4(pack_bf16x2(gs, gy), pack_bf16x2(gx, 0.0f), 0u, 0u);
        *(uint4*)(grad + (((size_t)img * 2 + 1) * plane + rem) * 8) = make_uint4(0u, 0u, 0u, 0u);
    }
#pragma unroll
    for (int d = 16; d; d >>= 1) {
        ls += __shfl_xor_sync(0xffffffffu, ls, d);
        lo += __shfl_xor_sync(0xffffffffu, lo, d);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = ls;
        red[1][threadIdx.x >> 5] = lo;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float a = 0.0f, b = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            a += red[0][w];
            b += red[1][w];
        }
        partial[2 * blockIdx.x] = a;
        partial[2 * blockIdx.x + 1] = b;
    }
}

// -------------------------------------------------------- weight gradient
// dW[co][ci][t] = sum over cells of G[cell][co] * X[cell + tap t][ci] (both
// in 8-channel planes; G has GSTRIDE channels of which COUT are used), and
// db[co] = sum of G[cell][co]: one thread per (t, ci) (plus one for the
// bias) accumulating all output channels in registers over the tiles its
// CTA owns; per-CTA partial sums go to `partial` and are added in CTA order.
constexpr int kWgTH = 4, kWgTW = 32;
template <int CIN, int COUT, int GSTRIDE>
__global__ void __launch_bounds__(((9 * CIN + 1 + 31) / 32) * 32)
cnn_wgrad_kernel(const __nv_bfloat16* __restrict__ X, const __nv_bfloat16* __restrict__ Gd, int nimg, int Hc,
                 int Wc, float* __restrict__ partial) {
    __shared__ float xs[(kWgTH + 2) * (kWgTW + 2) * CIN];
    __shared__ float gs[kWgTH * kWgTW * COUT];
    const int tid = threadIdx.x;
    const int tap = tid / CIN, ci = tid % CIN;
    const bool is_w = tid < 9 * CIN, is_b = tid == 9 * CIN;
    const int dy = tap / 3, dx = tap % 3;
    float acc[COUT];
#pragma unroll
    for (int o = 0; o < COUT; o++) acc[o] = 0.0f;
    const int ntx = (Wc + kWgTW - 1) / kWgTW, nty = (Hc + kWgTH - 1) / kWgTH;
    const int64_t ntiles = (int64_t)nimg * nty * ntx;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int img = (int)(tile / ((int64_t)nty * ntx));
        const int rem = (int)(tile - (int64_t)img * nty * ntx);
        const int y0 = (rem / ntx) * kWgTH, x0 = (rem % ntx) * kWgTW;
        __syncthreads();
        for (int i = tid; i < (kWgTH + 2) * (kWgTW + 2) * CIN; i += blockDim.x) {
            const int c = i % CIN, rest = i / CIN;
            const int j = rest % (kWgTW + 2), r = rest / (kWgTW + 2);
            const int gy = y0 - 1 + r, gx = x0 - 1 + j;
            float v = 0.0f;
            if (gy >= 0 && gy < Hc && gx >= 0 && gx < Wc)
                v = __bfloat162float(X[((((size_t)img * (CIN / 8) + c / 8) * Hc + gy) * Wc + gx) * 8 + (c & 7)]);
            xs[i] = v;
        }
        for (int i = tid; i < kWgTH * kWgTW * COUT; i += blockDim.x) {
            const int o = i % COUT, rest = i / COUT;
            const int j = rest % kWgTW, r = rest / kWgTW;
            const int gy = y0 + r, gx = x0 + j;
            float v = 0.0f;
            if (gy < Hc && gx < Wc)
                v = __bfloat162float(Gd[((((size_t)img * (GSTRIDE / 8) + o / 8) * Hc + gy) * Wc + gx) * 8 + (o & 7)]);
            gs[i] = v;
        }
        __syncthreads();
        if (is_w || is_b) {
            for (int p = 0; p < kWgTH * kWgTW; p++) {
                const int r = p / kWgTW, j = p % kWgTW;
                const float x = is_w ? xs[((r + dy) * (kWgTW + 2) + j + dx) * CIN + ci] : 1.0f;
#pragma unroll
                for (int o = 0; o < COUT; o++) acc[o] = __fmaf_rn(gs[p * COUT + o], x, acc[o]);
            }
        }
    }
    constexpr int NP = COUT * CIN * 9 + COUT;
    float* dst = partial + (size_t)blockIdx.x * NP;
    if (is_w) {
#pragma unroll
        for (int o = 0; o < COUT; o++) dst[((size_t)o * CIN + ci) * 9 + tap] = acc[o];
    } else if (is_b) {
#pragma unroll
        for (int o = 0; o < COUT; o++) dst[COUT * CIN * 9 + o] = acc[o];
    }
}

// grad[i] = sum over blocks b (in order) of partial[b][i]
__global__ void cnn_reduce_kernel(const float* __restrict__ partial, int nblocks, int np, float* __restrict__ grad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    float s = 0.0f;
    for (int b = 0; b < nblocks; b++) s += partial[(size_t)b * np + i];
    grad[i] = s;
}

// Adam on the fp32 master parameters (bias-corrected step size lr_t).
__global__ void cnn_adam_kernel(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                                const float* __restrict__ g, int n, float lr_t, float b1, float b2, float eps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr_t * mi / (sqrtf(vi) + eps);
}

// ------------------------------------------------------------ proposals
// A cell proposes a walk seed when its score logit exceeds the threshold: the
// pixel nearest to the cell centre plus the predicted offset, clamped inside
// the candidate margin.  Of two cells in one 3x3 window whose seeds lie
// within one pixel of each other only the higher-scoring one proposes (ties
// go to the earlier cell in raster order): their walks would end together.
__device__ __forceinline__ void cell_seed(const float4& o, int cy, int cx, int lo_y, int hi_y, int lo_x, int hi_x,
                                          int& u, int& v) {
    u = (o.y == o.y) ? (int)rintf(4.0f * cy + 1.5f + o.y) : 4 * cy + 1;
    v = (o.z == o.z) ? (int)rintf(4.0f * cx + 1.5f + o.z) : 4 * cx + 1;
    u = min(max(u, lo_y), hi_y);
    v = min(max(v, lo_x), hi_x);
}

__global__ void cnn_proposal_kernel(const float4* __restrict__ head, int Hc, int Wc, int H, int W, int margin,
                                    float thr, uint32_t* __restrict__ cand_count, uint32_t* __restrict__ cand_keys,
                                    uint32_t cand_cap, uint32_t* __restrict__ flags) {
    const int f = blockIdx.y;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const float4* hf = head + (size_t)f * Hc * Wc;
    const int lo_y = margin, hi_y = H - 1 - margin, lo_x = margin, hi_x = W - 1 - margin;
    bool keep = false;
    uint32_t key = 0;
    if (c < Hc * Wc && hi_y >= lo_y && hi_x >= lo_x) {
        const int cy = c / Wc, cx = c % Wc;
        const float4 o = hf[c];
        const float s = o.x;
        keep = s > thr;
        int u = 0, v = 0;
        if (keep) cell_seed(o, cy, cx, lo_y, hi_y, lo_x, hi_x, u, v);
        for (int dy = -1; dy <= 1 && keep; dy++)
            for (int dx = -1; dx <= 1 && keep; dx++) {
                if (dy == 0 && dx == 0) continue;
                const int ny = cy + dy, nx = cx + dx;
                if (ny < 0 || ny >= Hc || nx < 0 || nx >= Wc) continue;
                const float4 on = hf[ny * Wc + nx];
                if (!(on.x > s || (on.x == s && (dy < 0 || (dy == 0 && dx < 0))))) continue;
                int nu, nv;
                cell_seed(on, ny, nx, lo_y, hi_y, lo_x, hi_x, nu, nv);
                if (abs(nu - u) <= 1 && abs(nv - v) <= 1) keep = false;
            }
        key = (uint32_t)u * (uint32_t)W + (uint32_t)v;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (!bal) return;
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(cand_count + f, (uint32_t)__popc(bal));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (keep) {
        const uint32_t pos = base + __popc(bal & ((1u << lane) - 1u));
        if (pos < cand_cap) cand_keys[(size_t)f * cand_cap + pos] = key;
        else atomicOr(flags, kFlagCandOverflow);
    }
}

}  // namespace

// ============================================================ launchers
cudaError_t cnn_pack(const float* W, int layer, bool backward, __nv_bfloat16* dst, cudaStream_t st) {
    const int cin = kCnnCin[layer], cout = kCnnCout[layer];
    int KS, N;
    if (!backward) {
        KS = cin / 16;
        N = layer == 3 ? 16 : 32;
    } else {
        KS = layer == 3 ? 1 : cout / 16;  // the head's 3 gradient channels sit in a 16-channel cell
        N = cin;
    }
    const int total = 9 * KS * N * 16;
    cnn_pack_kernel<<<(total + 255) / 256, 256, 0, st>>>(W, cin, cout, KS, N, backward ? 1 : 0, dst);
    return cudaGetLastError();
}

size_t cnn_packed_bytes(int layer, bool backward) {
    const int cin = kCnnCin[layer], cout = kCnnCout[layer];
    if (!backward) return (size_t)9 * (cin / 16) * (layer == 3 ? 16 : 32) * 32;
    return (size_t)9 * (layer == 3 ? 1 : cout / 16) * cin * 32;
}

template <typename T>
cudaError_t cnn_input(const T* frames, int64_t frame_stride, int H, int W, const int4* crops, int nimg, int Hc,
                      int Wc, float mean, float scale, __nv_bfloat16* out, cudaStream_t st) {
    const int64_t n = (int64_t)nimg * Hc * Wc;
    if (n == 0) return cudaSuccess;
    cnn_input_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(frames, frame_stride, H, W, crops, nimg, Hc,
                                                                      Wc, mean, scale, out);
    return cudaGetLastError();
}
template cudaError_t cnn_input<uint16_t>(const uint16_t*, int64_t, int, int, const int4*, int, int, int, float, float,
                                         __nv_bfloat16*, cudaStream_t);
template cudaError_t cnn_input<float>(const float*, int64_t, int, int, const int4*, int, int, int, float, float,
                                      __nv_bfloat16*, cudaStream_t);
template cudaError_t cnn_input<uint8_t>(const uint8_t*, int64_t, int, int, const int4*, int, int, int, float, float,
                                        __nv_bfloat16*, cudaStream_t);

cudaError_t cnn_forward(const CnnNet& net, const __nv_bfloat16* x, int nimg, int Hc, int Wc, __nv_bfloat16* a1,
                        __nv_bfloat16* a2, __nv_bfloat16* a3, float4* head, uint32_t* flags, int num_sms,
                        cudaStream_t st) {
    cudaError_t e;
    e = conv_launch<1, 32, 0>(x, nimg, Hc, Wc, net.wf[0], net.bias[0], nullptr, a1, flags, num_sms, st);
    if (e != cudaSuccess) return e;
    e = conv_launch<2, 32, 0>(a1, nimg, Hc, Wc, net.wf[1], net.bias[1], nullptr, a2, flags, num_sms, st);
    if (e != cudaSuccess) return e;
    e = conv_launch<2, 32, 0>(a2, nimg, Hc, Wc, net.wf[2], net.bias[2], nullptr, a3, flags, num_sms, st);
    if (e != cudaSuccess) return e;
    return conv_launch<2, 16, 1>(a3, nimg, Hc, Wc, net.wf[3], net.bias[3], nullptr, head, flags, num_sms, st);
}

cudaError_t cnn_backward_input(const CnnNet& net, int layer, const __nv_bfloat16* gout, const __nv_bfloat16* act_below,
                               int nimg, int Hc, int Wc, __nv_bfloat16* gin, uint32_t* flags, int num_sms,
                               cudaStream_t st) {
    if (layer == 3)
        return conv_launch<1, 32, 2>(gout, nimg, Hc, Wc, net.wd[3], nullptr, act_below, gin, flags, num_sms, st);
    return conv_launch<2, 32, 2>(gout, nimg, Hc, Wc, net.wd[layer], nullptr, act_below, gin, flags, num_sms, st);
}

cudaError_t cnn_wgrad(int layer, const __nv_bfloat16* X, const __nv_bfloat16* G, int nimg, int Hc, int Wc,
                      float* partial, int nblocks, float* grad, cudaStream_t st) {
    const int cin = kCnnCin[layer], cout = kCnnCout[layer];
    const int np = cout * cin * 9 + cout;
    switch (layer) {
        case 0:
            cnn_wgrad_kernel<16, 32, 32><<<nblocks, ((9 * 16 + 1 + 31) / 32) * 32, 0, st>>>(X, G, nimg, Hc, Wc,
                                                                                             partial);
            break;
        case 1:
        case 2:
            cnn_wgrad_kernel<32, 32, 32><<<nblocks, ((9 * 32 + 1 + 31) / 32) * 32, 0, st>>>(X, G, nimg, Hc, Wc,
                                                                                             partial);
            break;
        default:
            cnn_wgrad_kernel<32, 3, 16><<<nblocks, ((9 * 32 + 1 + 31) / 32) * 32, 0, st>>>(X, G, nimg, Hc, Wc,
                                                                                            partial);
            break;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cnn_reduce_kernel<<<(np + 255) / 256, 256, 0, st>>>(partial, nblocks, np, grad);
    return cudaGetLastError();
}

size_t cnn_wgrad_partial_floats(int nblocks) {
    size_t mx = 0;
    for (int l = 0; l < 4; l++) mx = std::max(mx, (size_t)kCnnCout[l] * kCnnCin[l] * 9 + kCnnCout[l]);
    return mx * nblocks;
}

cudaError_t cnn_labels(const int32_t* lf, const float* ly, const float* lx, int64_t n, int T, int Hc, int Wc,
                       int32_t* owner, float4* tmap, cudaStream_t st) {
    const int64_t ncells = (int64_t)T * Hc * Wc;
    if (n >= kLabelFree) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(owner, 0x7F, (size_t)ncells * 4, st);  // kLabelFree, above every index
    if (e != cudaSuccess) return e;
    if (n > 0)
        cnn_label_claim_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(lf, ly, lx, n, Hc, Wc, owner);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cnn_label_write_kernel<<<(unsigned)((ncells + 255) / 256), 256, 0, st>>>(ly, lx, owner, ncells, Hc, Wc, tmap);
    return cudaGetLastError();
}

cudaError_t cnn_crops(uint32_t seed, uint32_t step, int nimg, int T, int Hc, int Wc, int CH, int CW, int4* crops,
                      cudaStream_t st) {
    cnn_crop_kernel<<<(nimg + 127) / 128, 128, 0, st>>>(seed, step, nimg, T, Hc, Wc, CH, CW, CH == CW ? 1 : 0, crops);
    return cudaGetLastError();
}

cudaError_t cnn_loss(const float4* head, const float4* tmap, const int4* crops, int nimg, int CH, int CW, int Hc_f,
                     int Wc_f, float pos_weight, float lambda, __nv_bfloat16* grad, float* partial, int* nblocks,
                     cudaStream_t st) {
    const int64_t n = (int64_t)nimg * CH * CW;
    *nblocks = (int)((n + 255) / 256);
    cnn_loss_kernel<<<*nblocks, 256, 0, st>>>(head, tmap, crops, nimg, CH, CW, Hc_f, Wc_f, pos_weight, lambda, grad,
                                              partial);
    return cudaGetLastError();
}

// out[0..1] = the loss partial sums of the step (fixed order), times `inv`
__global__ void cnn_loss_sum_kernel(const float* __restrict__ partial, int nblocks, float inv, float* __restrict__ out) {
    __shared__ float red[2][256];
    float a = 0.0f, b = 0.0f;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
        a += partial[2 * i];
        b += partial[2 * i + 1];
    }
    red[0][threadIdx.x] = a;
    red[1][threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s; s >>= 1) {
        if ((int)threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = red[0][0] * inv;
        out[1] = red[1][0] * inv;
    }
}

cudaError_t cnn_loss_sum(const float* partial, int nblocks, float inv, float* out, cudaStream_t st) {
    cnn_loss_sum_kernel<<<1, 256, 0, st>>>(partial, nblocks, inv, out);
    return cudaGetLastError();
}

cudaError_t cnn_adam(float* p, float* m, float* v, const float* g, int n, float lr_t, float b1, float b2, float eps,
                     cudaStream_t st) {
    cnn_adam_kernel<<<(n + 255) / 256, 256, 0, st>>>(p, m, v, g, n, lr_t, b1, b2, eps);
    return cudaGetLastError();
}

cudaError_t cnn_proposals(const float4* head, int nimg, int Hc, int Wc, int H, int W, int margin, float thr,
                          uint32_t* cand_count, uint32_t* cand_keys, uint32_t cand_cap, uint32_t* flags,
                          cudaStream_t st) {
    dim3 grid((unsigned)((Hc * Wc + 255) / 256), (unsigned)nimg);
    if (Hc * Wc == 0 || nimg == 0) return cudaSuccess;
    cnn_proposal_kernel<<<grid, 256, 0, st>>>(head, Hc, Wc, H, W, margin, thr, cand_count, cand_keys, cand_cap,
                                              flags);
    return cudaGetLastError();
}

}  // namespace gt
