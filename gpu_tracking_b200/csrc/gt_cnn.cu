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
// Convolution as an implicit GEMM on the tensor cores: a CTA owns a tile of
// 4 x 32 cells (M = 128 rows of D), the output channels are N and K runs over
// the 9 taps x input channels.  The input tile (6 x 34 cells with the halo)
// is staged three times in shared memory, shifted by -1, 0 and +1 cells, in
// the K-major "interleave" layout (8 cells x 8 channels = one 128-byte core
// matrix): a tap (dy, dx) is then the copy of dx read from row dy, a plain
// descriptor offset, and one UMMA of K = 16 per tap and 16 input channels.
// D lives in TMEM (32 columns); the epilogue reads it with tcgen05.ld, adds
// the bias, applies the ReLU (or the ReLU mask of the backward pass) and
// writes BF16 cells.
#include <cuda_bf16.h>

#include "gt_internal.cuh"
#include "gt_kernels.h"
#include "gt_tc.cuh"

namespace gt {

namespace {

constexpr int kConvTW = 32;       // tile width in cells (4 core-matrix groups)
constexpr int kConvTH = 4;        // tile rows: M = 128
constexpr int kConvThreads = 128;  // 4 warps: warp w reads TMEM lanes 32w..32w+31 = tile row w
constexpr uint32_t kConvPolls = 1u << 22;

template <int KS, int N>
struct ConvGeom {
    static constexpr int CIN = 16 * KS;
    static constexpr int GROUP = KS * 2 * 128;          // bytes of 8 cells x CIN channels
    static constexpr int ROW = (kConvTW / 8) * GROUP;   // one row of the tile
    static constexpr int COPY = (kConvTH + 2) * ROW;    // one dx-shifted copy (with the row halo)
    static constexpr int A_BYTES = 3 * COPY;
    static constexpr int B_BYTES = 9 * KS * (N / 8) * 256;
    static constexpr int SMEM = 128 + 2 * A_BYTES + B_BYTES + 16;  // two staging buffers
};

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

// Stage the input cells (y0 - 1 + r, x0 - 1 + j) of a tile into the three
// shifted copies at A: every load of the tile is issued before the first
// shared-memory store, so the tile costs one round trip to L2.
template <int KS>
__device__ __forceinline__ void conv_fill(uint8_t* A, const __nv_bfloat16* __restrict__ src, int Hc, int Wc, int y0,
                                          int x0, int tid) {
    using G = ConvGeom<KS, 32>;
    constexpr int NQ = 2 * KS, NJ = kConvTW + 2;
    constexpr int TOTAL = (kConvTH + 2) * NQ * NJ;
    constexpr int NIT = (TOTAL + kConvThreads - 1) / kConvThreads;
    uint4 v[NIT];
#pragma unroll
    for (int k = 0; k < NIT; k++) {
        const int it = tid + k * kConvThreads;
        v[k] = make_uint4(0u, 0u, 0u, 0u);
        if (it < TOTAL) {
            const int j = it % NJ, rest = it / NJ;
            const int q = rest % NQ, r = rest / NQ;
            const int gy = y0 - 1 + r, gx = x0 - 1 + j;
            if (gy >= 0 && gy < Hc && gx >= 0 && gx < Wc)
                v[k] = __ldg((const uint4*)(src + ((size_t)gy * Wc + gx) * G::CIN) + q);
        }
    }
#pragma unroll
    for (int k = 0; k < NIT; k++) {
        const int it = tid + k * kConvThreads;
        if (it < TOTAL) {
            const int j = it % NJ, rest = it / NJ;
            const int q = rest % NQ, r = rest / NQ;
#pragma unroll
            for (int dx = 0; dx < 3; dx++) {
                const int c = j - dx;
                if (c >= 0 && c < kConvTW)
                    *(uint4*)(A + dx * G::COPY + r * G::ROW + (c >> 3) * G::GROUP + q * 128 + (c & 7) * 16) = v[k];
            }
        }
    }
}

// MODE 0: relu(acc + bias) -> bf16 [cell][32]
// MODE 1: acc + bias      -> float4 [cell] (score, row offset, column offset, 0), N = 16
// MODE 2: acc * (mask > 0) -> bf16 [cell][32] (backward through the ReLU of the layer below)
// A CTA walks its tiles with two staging buffers: the next tile is staged
// while the tensor cores work on the current one.
template <int KS, int N, int MODE>
__global__ void __launch_bounds__(kConvThreads)
conv3x3_kernel(const __nv_bfloat16* __restrict__ in, int nimg, int Hc, int Wc, const uint8_t* __restrict__ wpk,
               const float* __restrict__ bias, const __nv_bfloat16* __restrict__ mask, void* __restrict__ out,
               uint32_t* __restrict__ flags) {
    using G = ConvGeom<KS, N>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* A0 = (uint8_t*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint8_t* B = A0 + 2 * G::A_BYTES;
    uint64_t* mbar = (uint64_t*)(B + G::B_BYTES);
    uint32_t* tslot = (uint32_t*)(mbar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    for (int i = tid; i < G::B_BYTES / 16; i += kConvThreads) ((uint4*)B)[i] = __ldg((const uint4*)wpk + i);
    if (tid == 0) tc::mbar_init(mbar, 1);
    if (warp == 0) tc::tmem_alloc(tslot, 32);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t idesc = tc::idesc_bf16_f32(128, N);
    const uint32_t b_base = tc::smem_addr(B);

    const int ntx = (Wc + kConvTW - 1) / kConvTW, nty = (Hc + kConvTH - 1) / kConvTH;
    const int64_t per_img = (int64_t)nty * ntx;
    const int64_t ntiles = (int64_t)nimg * per_img;
    auto tile_pos = [&](int64_t tile, int& img, int& y0, int& x0) {
        img = (int)(tile / per_img);
        const int rem = (int)(tile - (int64_t)img * per_img);
        y0 = (rem / ntx) * kConvTH;
        x0 = (rem % ntx) * kConvTW;
    };
    auto issue = [&](const uint8_t* A) {
        const uint32_t a_base = tc::smem_addr(A);
        uint32_t acc = 0;
#pragma unroll
        for (int t = 0; t < 9; t++) {
            const int dy = t / 3, dx = t % 3;
#pragma unroll
            for (int k = 0; k < KS; k++) {
                const uint64_t ad = tc::desc_kmajor(a_base + dx * G::COPY + dy * G::ROW + k * 256, 128, G::GROUP);
                const uint64_t bd = tc::desc_kmajor(b_base + (t * KS + k) * (N / 8) * 256, 128, 256);
                tc::mma_bf16(tmem, ad, bd, idesc, acc);
                acc = 1;
            }
        }
        tc::mma_commit(mbar);
    };

    uint32_t phase = 0;
    bool ok = true, pending = false;
    int64_t tile = blockIdx.x;
    if (tile < ntiles) {
        int img, y0, x0;
        tile_pos(tile, img, y0, x0);
        conv_fill<KS>(A0, in + (size_t)img * Hc * Wc * G::CIN, Hc, Wc, y0, x0, tid);
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) issue(A0);
        pending = true;
    }
    for (int k = 0; tile < ntiles; k++, tile += gridDim.x) {
        const int64_t next = tile + gridDim.x;
        uint8_t* An = A0 + ((k + 1) & 1) * G::A_BYTES;
        if (next < ntiles) {
            int img, y0, x0;
            tile_pos(next, img, y0, x0);
            conv_fill<KS>(An, in + (size_t)img * Hc * Wc * G::CIN, Hc, Wc, y0, x0, tid);
        }
        const bool done = __syncthreads_and(tc::mbar_wait_bounded(mbar, phase, kConvPolls) ? 1 : 0) != 0;
        if (!done) {
            if (tid == 0) atomicOr(flags, kFlagTensorTimeout);
            ok = false;
            break;
        }
        pending = false;
        phase ^= 1u;
        tc::fence_after_sync();
        int img, y0, x0;
        tile_pos(tile, img, y0, x0);
        const int gy = y0 + warp, gx = x0 + lane;
        const bool in_frame = gy < Hc && gx < Wc;
        const size_t cell = ((size_t)img * Hc + gy) * Wc + gx;
        if (MODE == 1) {
            uint32_t r[16];
            tc::tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16), r);
            tc::tmem_ld_wait();
            if (in_frame) {
                float4 o;
                o.x = __fadd_rn(__uint_as_float(r[0]), bias[0]);
                o.y = __fadd_rn(__uint_as_float(r[1]), bias[1]);
                o.z = __fadd_rn(__uint_as_float(r[2]), bias[2]);
                o.w = 0.0f;
                ((float4*)out)[cell] = o;
            }
        } else {
            uint32_t r[32];
            tc::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16), r);
            tc::tmem_ld_wait();
            if (in_frame) {
                float v[32];
#pragma unroll
                for (int n = 0; n < 32; n++) v[n] = __uint_as_float(r[n]);
                if (MODE == 0) {
#pragma unroll
                    for (int n = 0; n < 32; n++) v[n] = fmaxf(__fadd_rn(v[n], bias[n]), 0.0f);
                } else {
                    const uint4* mk = (const uint4*)(mask + cell * 32);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        uint4 m4 = __ldg(mk + q);
                        const uint32_t mw[4] = {m4.x, m4.y, m4.z, m4.w};
#pragma unroll
                        for (int h = 0; h < 4; h++) {
                            // bf16 > 0: sign bit clear and not +0
                            const uint32_t lo = mw[h] & 0xFFFFu, hi = mw[h] >> 16;
                            if (!(lo != 0u && !(lo & 0x8000u))) v[8 * q + 2 * h] = 0.0f;
                            if (!(hi != 0u && !(hi & 0x8000u))) v[8 * q + 2 * h + 1] = 0.0f;
                        }
                    }
                }
                uint4* o = (uint4*)((__nv_bfloat16*)out + cell * 32);
#pragma unroll
                for (int q = 0; q < 4; q++)
                    o[q] = make_uint4(pack_bf16x2(v[8 * q], v[8 * q + 1]), pack_bf16x2(v[8 * q + 2], v[8 * q + 3]),
                                      pack_bf16x2(v[8 * q + 4], v[8 * q + 5]),
                                      pack_bf16x2(v[8 * q + 6], v[8 * q + 7]));
            }
        }
        // the staged next tile becomes visible to the tensor cores and TMEM
        // is free again once every warp has read it
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (next < ntiles) {
            if (tid == 0) issue(An);
            pending = true;
        }
    }
    if (!ok && pending) tc::mbar_wait_bounded(mbar, phase, kConvPolls);  // let issued UMMAs drain before the free
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem, 32);
}

template <int KS, int N, int MODE>
cudaError_t conv_launch(const __nv_bfloat16* in, int nimg, int Hc, int Wc, const uint8_t* wpk, const float* bias,
                        const __nv_bfloat16* mask, void* out, uint32_t* flags, int num_sms, cudaStream_t st) {
    using G = ConvGeom<KS, N>;
    cudaError_t e = cudaFuncSetAttribute(conv3x3_kernel<KS, N, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         G::SMEM);
    if (e != cudaSuccess) return e;
    const int64_t ntiles = (int64_t)nimg * ((Hc + kConvTH - 1) / kConvTH) * ((Wc + kConvTW - 1) / kConvTW);
    if (ntiles == 0) return cudaSuccess;
    // 2 CTAs per SM (shared memory) hold 2 x 32 of the 512 TMEM columns
    const int64_t grid = std::min<int64_t>(ntiles, (int64_t)num_sms * 2);
    conv3x3_kernel<KS, N, MODE><<<(unsigned)grid, kConvThreads, G::SMEM, st>>>(in, nimg, Hc, Wc, wpk, bias, mask,
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
    uint4* o = (uint4*)(out + cell * 16);
    o[0] = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                      pack_bf16x2(v[6], v[7]));
    o[1] = make_uint4(pack_bf16x2(v[8], v[9]), pack_bf16x2(v[10], v[11]), pack_bf16x2(v[12], v[13]),
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
        uint4* g = (uint4*)(grad + cell * 16);
        g[0] = make_uint4(pack_bf16x2(gs, gy), pack_bf16x2(gx, 0.0f), 0u, 0u);
        g[1] = make_uint4(0u, 0u, 0u, 0u);
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
// dW[co][ci][t] = sum over cells of G[cell][co] * X[cell + tap t][ci], and
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
                v = __bfloat162float(X[(((size_t)img * Hc + gy) * Wc + gx) * CIN + c]);
            xs[i] = v;
        }
        for (int i = tid; i < kWgTH * kWgTW * COUT; i += blockDim.x) {
            const int o = i % COUT, rest = i / COUT;
            const int j = rest % kWgTW, r = rest / kWgTW;
            const int gy = y0 + r, gx = x0 + j;
            float v = 0.0f;
            if (gy < Hc && gx < Wc) v = __bfloat162float(Gd[(((size_t)img * Hc + gy) * Wc + gx) * GSTRIDE + o]);
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
