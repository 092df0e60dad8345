// gt_strip.cu — streaming bandpass + grey-dilation local-max kernel (sm_100a).
//
// Same results as bandpass_kernel<T, true> (preprocess_rows.wgsl,
// preprocess_cols.wgsl, max_rows.wgsl, extract_max.wgsl), organised for
// instruction throughput.  A CTA owns a strip of 128 output columns and walks
// down a segment of rows eight rows per step:
//   A  the step's raw rows are staged in shared memory (4 pixels per load,
//      converted exactly to float), the next step's are prefetched;
//   B  row pass: each thread makes 4 adjacent columns from float4 loads;
//   C  column pass: each thread makes the step's 8 rows of one column;
//   D  vertical dilation maximum, 8 rows of one column per thread;
//   E  horizontal dilation maximum, the candidate test and the store of the
//      segment's processed rows, 4 columns per thread; candidates gather in a
//      shared-memory buffer of the tile (one shared atomic per warp) and go
//      to the frame's list with one global reservation per tile.
// Two ring layouts hold the row-pass rows and the processed rows:
//   integer pixels (ring_tile): single-copy rings of RING rows, RING a
//      multiple of the 8-row step, so step s writes ring rows
//      8*(s % (RING/8)) .. +7 without wrapping; the column pass and the
//      vertical maxima are compiled once per ring phase s % (RING/8) and
//      picked by a uniform branch, so every ring row they touch is a
//      compile-time offset.  Rows above and below the frame hold a Gaussian
//      row sum of +0 instead of being skipped: integer pixels make every row
//      sum >= +0, and fma(w, +0, acc) == acc for acc >= +0, so the column
//      pass needs no per-row bounds test.  The smaller rings let 4 CTAs share
//      an SM where the shared memory allows it;
//   float pixels (strip_tile): rings that hold every row twice (at r and
//      r + ring), so any window of consecutive rows is contiguous, with
//      per-tap bounds tests at the frame's top and bottom (a float row sum
//      may be -0, which the skipped term keeps and +0 would not).
// The tap loops are unrolled for the compile-time radius.
// The floating-point operation sequence of every output is the oracle's:
// sequential fused multiply-adds over the taps, sequential boxcar sums (for
// integer inputs a pairwise window sum and sliding differences instead: every
// partial sum is an exactly representable integer, so any order gives the
// same value), and division by the constants gnorm and kk either
// as IEEE division or, where proven equal to it (LocateConsts::fast_div), as
// fma(x, zh, x*zl).
#include <math.h>

#include <map>
#include <mutex>
#include <tuple>

#include "gt_internal.cuh"
#include "gt_kernels.h"

namespace gt {

constexpr int kStripTW = 128;
constexpr int kStripThreads = 288;
constexpr int kStepRows = 8;
constexpr int kCandBuf = 768;   // candidate keys a tile buffers in shared memory

template <int R, int KD>
struct StripGeom {
    static constexpr int O = (int)((float)KD / 2.0f - 0.5f);
    static constexpr int E = KD - 1 - O;
    static constexpr int PW = kStripTW + KD - 1;          // processed columns a strip needs
    // raw column origin rc0 = c0 - O - R is rounded down to a multiple of 4
    // (c0 is a multiple of 128): the row-pass columns start SH4 early
    static constexpr int SH4 = (4 - (O + R) % 4) % 4;
    static constexpr int NG = (PW + SH4 + 3) / 4;         // 4-column groups of the row pass
    static constexpr int PWp = 4 * NG;                    // row stride of row-pass / processed rows
    static constexpr int NX4 = (4 + 2 * R + 3) / 4;       // float4 loads per row-pass group
    static constexpr int RWp = PWp + 4 * (NX4 - 1);       // staged raw columns (>= PWp + 2R)
    static constexpr int RW4 = RWp / 4;
    static constexpr int XR = kStepRows + 2 * R;          // row-pass ring rows
    static constexpr int PR = kStepRows + KD - 1;         // processed ring rows
    static constexpr int NV4 = (KD + 3 + 3) / 4;          // float4 loads per dilation group
    static constexpr int RAWV = kStepRows * RW4;          // 4-pixel loads per step
    static constexpr int RAWVPT = (RAWV + kStripThreads - 1) / kStripThreads;
    static constexpr int RAWN = kStepRows * RWp;
    static constexpr int RAWPT = (RAWN + kStripThreads - 1) / kStripThreads;
    // the vertical maxima (stages D-E) reuse the staged raw rows (stages A-B)
    static constexpr size_t smem_floats = (size_t)kStepRows * RWp + 2 * (size_t)(2 * XR) * PWp +
                                          (size_t)(2 * PR) * PWp + 4 + kCandBuf;
    static constexpr int min_blocks = (smem_floats * 4 + 1024) * 3 <= 227 * 1024 ? 3 : 2;
    static_assert(RWp % 4 == 0 && RWp >= PWp + 2 * R, "staged raw row");
    static_assert(RWp >= PWp, "vertical maxima fit in the staging rows");
    static_assert(4 * 31 + 4 * NV4 <= PWp, "dilation row reads stay in the row");
    static_assert(4 * 31 + KD + 2 <= PW - 1 && SH4 + O + kStripTW <= PWp, "dilation windows inside the row");
    static_assert(KD >= kStepRows && kStepRows == 8, "vertical maxima: 8 rows share the window rows 7 .. KD-1");
    static_assert(PWp <= kStripThreads, "one thread per column in the column pass and vertical maxima");
};

template <typename T>
struct IsIntPix {
    static constexpr bool value = !std::is_same<T, float>::value;
};

// Four raw pixels of one aligned load, exactly as floats (u8/u16 through the
// 2^23 bias: the integer's bits under the exponent of 2^23, minus 2^23).
__device__ __forceinline__ float bias_to_f32(uint32_t bits) { return __fsub_rn(__uint_as_float(bits), 8388608.0f); }

template <typename T>
struct Quad;
template <>
struct Quad<uint16_t> {
    using V = uint2;
    __device__ static V load(const uint16_t* p) { return __ldg((const uint2*)p); }
    __device__ static float4 cvt(V v) {
        return make_float4(bias_to_f32(__byte_perm(v.x, 0x4B00u, 0x5410)), bias_to_f32(__byte_perm(v.x, 0x4B00u, 0x5432)),
                           bias_to_f32(__byte_perm(v.y, 0x4B00u, 0x5410)), bias_to_f32(__byte_perm(v.y, 0x4B00u, 0x5432)));
    }
};
template <>
struct Quad<uint8_t> {
    using V = uint32_t;
    __device__ static V load(const uint8_t* p) { return __ldg((const uint32_t*)p); }
    __device__ static float4 cvt(V v) {
        return make_float4(bias_to_f32(__byte_perm(v, 0x4B000000u, 0x7440)),
                           bias_to_f32(__byte_perm(v, 0x4B000000u, 0x7441)),
                           bias_to_f32(__byte_perm(v, 0x4B000000u, 0x7442)),
                           bias_to_f32(__byte_perm(v, 0x4B000000u, 0x7443)));
    }
};
template <>
struct Quad<float> {
    using V = float4;
    __device__ static V load(const float* p) { return __ldg((const float4*)p); }
    __device__ static float4 cvt(V v) { return v; }
};

// Pairwise reductions with a short dependency chain.  Both are exact in any
// order here: the maximum always, the sum because it only adds integer pixel
// values (or integer row sums) whose partial sums stay below 2^24.
template <int N>
struct Tree {
    __device__ __forceinline__ static float max(const float* a) {
        return fmaxf(Tree<N / 2>::max(a), Tree<N - N / 2>::max(a + N / 2));
    }
    __device__ __forceinline__ static float sum(const float* a) {
        return __fadd_rn(Tree<N / 2>::sum(a), Tree<N - N / 2>::sum(a + N / 2));
    }
};
template <>
struct Tree<1> {
    __device__ __forceinline__ static float max(const float* a) { return a[0]; }
    __device__ __forceinline__ static float sum(const float* a) { return a[0]; }
};

template <bool FAST>
__device__ __forceinline__ float div_gnorm(float x, const LocateConsts& c) {
    return FAST ? __fmaf_rn(x, c.zh_g, __fmul_rn(x, c.zl_g)) : __fdiv_rn(x, c.gnorm);
}
template <bool FAST>
__device__ __forceinline__ float div_kk(float x, const LocateConsts& c) {
    return FAST ? __fmaf_rn(x, c.zh_k, __fmul_rn(x, c.zl_k)) : __fdiv_rn(x, c.kk);
}

// Appends the candidates a thread found among its 4 columns (bits of cmask,
// cnt of them) at row cd, columns ccol..ccol+3: warp-aggregated slots in the
// tile's shared buffer (one shared atomic per warp); a full buffer sends the
// warp's candidates straight to the frame's list.
__device__ __forceinline__ void append_cands(const int tid, const int cnt, const uint32_t cmask, const int cd,
                                             const int ccol, const int W, uint32_t* cbuf_n, uint32_t* cbuf,
                                             uint32_t* __restrict__ cand_slot, uint32_t* __restrict__ cout,
                                             const uint32_t cand_cap, uint32_t* __restrict__ flags) {
    if (!__any_sync(0xffffffffu, cnt != 0)) return;
    const int lane = tid & 31;
    int incl = cnt;
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, dd);
        if (lane >= dd) incl += v;
    }
    const int wtot = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t base = 0;
    if (lane == 31) base = atomicAdd(cbuf_n, (uint32_t)wtot);
    base = __shfl_sync(0xffffffffu, base, 31);
    uint32_t pos = base + (uint32_t)(incl - cnt);
    if (base + (uint32_t)wtot <= (uint32_t)kCandBuf) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!(cmask & (1u << k))) continue;
            cbuf[pos++] = (uint32_t)cd * (uint32_t)W + (uint32_t)(ccol + k);
        }
    } else {
        uint32_t gb = 0;
        if (lane == 31) gb = atomicAdd(cand_slot, (uint32_t)wtot);
        gb = __shfl_sync(0xffffffffu, gb, 31);
        pos = gb + (uint32_t)(incl - cnt);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!(cmask & (1u << k))) continue;
            if (pos < cand_cap) cout[pos] = (uint32_t)cd * (uint32_t)W + (uint32_t)(ccol + k);
            else atomicOr(flags, kFlagCandOverflow);
            pos++;
        }
    }
}

// The tile's buffered candidates go to the frame's list in one reservation
// (after a barrier that ends the tile's last step).
__device__ __forceinline__ void flush_tile_cands(const int tid, uint32_t* cbuf_n, const uint32_t* cbuf,
                                                 uint32_t* __restrict__ cand_slot, uint32_t* __restrict__ cout,
                                                 const uint32_t cand_cap, uint32_t* __restrict__ flags) {
    const uint32_t n = min(*cbuf_n, (uint32_t)kCandBuf);
    if (tid == 0) cbuf_n[1] = n ? atomicAdd(cand_slot, n) : 0u;
    __syncthreads();
    const uint32_t gb = cbuf_n[1];
    for (uint32_t i = tid; i < n; i += kStripThreads) {
        if (gb + i < cand_cap) cout[gb + i] = cbuf[i];
        else atomicOr(flags, kFlagCandOverflow);
    }
    __syncthreads();
}

// Raw rows of one 8-row step of a tile: loaded into registers (4 pixels per
// aligned load, or one clamped pixel each at the frame's edges) while the
// previous step is being filtered, then stored to the staging rows as exact
// floats.  Rows and columns outside the frame read the nearest edge pixel.
template <typename T, int R, int KD>
struct RawRows {
    using G = StripGeom<R, KD>;
    typename Quad<T>::V pv[G::RAWVPT];
    float px[G::RAWPT];

    __device__ __forceinline__ void load(const T* __restrict__ img, const int H, const int W, const int x0,
                                         const int xa, const bool vec, const int s) {
        const int tid = threadIdx.x;
        const int rbase = x0 + kStepRows * s;
        if (vec) {
#pragma unroll
            for (int q = 0; q < G::RAWVPT; q++) {
                const int v = tid + q * kStripThreads;
                if (v < G::RAWV) {
                    const int j = v / G::RW4, k4 = v - j * G::RW4;
                    const int gr = min(max(rbase + j, 0), H - 1);
                    pv[q] = Quad<T>::load(img + (size_t)gr * W + xa + 4 * k4);
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < G::RAWPT; q++) {
                const int idx = tid + q * kStripThreads;
                float v = 0.0f;
                if (idx < G::RAWN) {
                    const int j = idx / G::RWp, k = idx - j * G::RWp;
                    const int gr = min(max(rbase + j, 0), H - 1);
                    const int gc = min(max(xa + k, 0), W - 1);
                    v = load_px<T>(img, (size_t)gr * W + gc);
                }
                px[q] = v;
            }
        }
    }

    __device__ __forceinline__ void store(float* __restrict__ stage, const bool vec) const {
        const int tid = threadIdx.x;
        if (vec) {
#pragma unroll
            for (int q = 0; q < G::RAWVPT; q++) {
                const int v = tid + q * kStripThreads;
                if (v < G::RAWV) {
                    const int j = v / G::RW4, k4 = v - j * G::RW4;
                    *(float4*)(stage + j * G::RWp + 4 * k4) = Quad<T>::cvt(pv[q]);
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < G::RAWPT; q++) {
                const int idx = tid + q * kStripThreads;
                if (idx < G::RAWN) stage[idx] = px[q];
            }
        }
    }
};

// Stage E of one step (extract_max.wgsl): for the step's 8 dilation rows
// d = dbase + jj, 4 columns per thread, the horizontal maximum of the
// vertical maxima vb, the candidate test of every column without branches
// (columns and rows inside the margin need no bounds test) and the store of
// the processed row to HBM; center_row(jj) is the shared-memory row that
// holds processed row dbase + jj.
template <int R, int KD, typename CenterRow>
__device__ __forceinline__ void extract_step(const int tid, const float* vb, CenterRow center_row, const int dbase,
                                             const int R0, const int R1, const int c0, const int H, const int W,
                                             const LocateConsts& c, const float thr, const bool st4,
                                             float* __restrict__ proc, uint32_t* cbuf_n, uint32_t* cbuf,
                                             uint32_t* __restrict__ cand_slot, uint32_t* __restrict__ cout,
                                             const uint32_t cand_cap, uint32_t* __restrict__ flags) {
    using G = StripGeom<R, KD>;
    constexpr int O = G::O, PWp = G::PWp, SH4 = G::SH4;
    int cnt = 0;
    uint32_t cmask = 0;
    int cd = 0, ccol = 0;
    if (tid < kStepRows * (kStripTW / 4)) {
        const int jj = tid / (kStripTW / 4), cg = tid - jj * (kStripTW / 4);
        const int d = dbase + jj;
        const int cc = 4 * cg;  // interior column offset; processed column = cc + O (pc0-relative)
        if (d >= R0 && d < R1) {
            const float4* src = (const float4*)(vb + jj * PWp + cc);
            float a[4 * G::NV4];
#pragma unroll
            for (int i = 0; i < G::NV4; i++) {
                const float4 v = src[i];
                a[4 * i] = v.x;
                a[4 * i + 1] = v.y;
                a[4 * i + 2] = v.z;
                a[4 * i + 3] = v.w;
            }
            const float mid = Tree<KD - 3>::max(a + 3);
            float s2 = a[2], s1 = fmaxf(a[1], s2), s0 = fmaxf(a[0], s1);
            float p1 = a[KD], p2 = fmaxf(p1, a[KD + 1]), p3 = fmaxf(p2, a[KD + 2]);
            float m[4] = {fmaxf(s0, mid), fmaxf(fmaxf(s1, mid), p1), fmaxf(fmaxf(s2, mid), p2), fmaxf(mid, p3)};
            const float* cen = center_row(jj) + SH4 + O + cc;
            float cv[4];
#pragma unroll
            for (int k = 0; k < 4; k++) cv[k] = cen[k];
            const int gc0 = c0 + cc;
            float* dst = proc + (size_t)d * W + gc0;
            if (st4 && gc0 + 3 < W) {
                *(float4*)dst = make_float4(cv[0], cv[1], cv[2], cv[3]);
            } else {
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (gc0 + k < W) dst[k] = cv[k];
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float center = cv[k];
                bool ok = !(center < thr) && !(m[k] > center);
                if (c.skip_zero) ok = ok && (center != 0.0f);
                cmask |= (uint32_t)ok << k;
            }
            const bool inner = d >= c.margin && d < H - c.margin && gc0 >= c.margin && gc0 + 3 < W - c.margin;
            if (!inner) {
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int gc = gc0 + k;
                    if (gc >= W || d < c.margin || d >= H - c.margin || gc < c.margin || gc >= W - c.margin)
                        cmask &= ~(1u << k);
                }
            }
            cnt = __popc(cmask);
            cd = d;
            ccol = gc0;
        }
    }
    append_cands(tid, cnt, cmask, cd, ccol, W, cbuf_n, cbuf, cand_slot, cout, cand_cap, flags);
}

// One tile: the strip of output columns [c0, c0 + 128) and rows [R0, R1) of
// an H x W frame (img: its pixels, proc: its processed image), candidates
// appended to the list counted by *cand_slot (keys at cout).
template <typename T, int R, int KD, bool FAST>
__device__ __forceinline__ void strip_tile(const T* __restrict__ img, float* __restrict__ proc, const LocateConsts& c,
                                           const int H, const int W, const int c0, const int R0, const int R1,
                                           const int vec_ok, const float thr, uint32_t* __restrict__ cand_slot,
                                           uint32_t* __restrict__ cout, const uint32_t cand_cap,
                                           uint32_t* __restrict__ flags) {
    using G = StripGeom<R, KD>;
    constexpr int O = G::O, E = G::E, PWp = G::PWp, RWp = G::RWp, XR = G::XR, PR = G::PR, SH4 = G::SH4;
    constexpr bool kInt = IsIntPix<T>::value;
    extern __shared__ float4 sm4[];
    float* sm = (float*)sm4;
    float* stage = sm;                          // [8][RWp]      raw columns xa .. xa+RWp
    float* xg = stage + kStepRows * RWp;        // [2XR][PWp]    row pass g / gnorm, rows stored twice
    float* xb = xg + 2 * XR * PWp;              // [2XR][PWp]    row pass boxcar
    float* pr = xb + 2 * XR * PWp;              // [2PR][PWp]    processed rows, stored twice
    float* vb = stage;                          // [8][PWp]      vertical maxima (pc0-relative columns)
    uint32_t* cbuf_n = (uint32_t*)(pr + 2 * PR * PWp);   // [4]   buffered candidates, flush base
    uint32_t* cbuf = cbuf_n + 4;                // [kCandBuf]    candidate keys of the tile

    const int x0 = R0 - O - R;          // first raw / row-pass row
    const int pc0 = c0 - O;             // first processed column of the strip's dilation windows
    const int xa = pc0 - R - SH4;       // first staged raw column (a multiple of 4)
    const int ps = xa + R;              // processed column of row-pass index 0 (= pc0 - SH4)
    const int tid = threadIdx.x;
    const bool edge_cols = (xa < 0) || (xa + RWp > W);
    const bool vec = vec_ok && !edge_cols;
    // 16-byte stores of processed rows: every row start is a multiple of 4 floats
    const bool st4 = (W % 4 == 0) && ((uintptr_t)proc % 16 == 0);
    // steps until the dilation rows reach R1: x0 + 8s - R - E + 8 >= R1
    const int nsteps = (R1 - x0 + R + E + kStepRows - 1) / kStepRows;

    // ---- A: staging of raw rows (registers hold the next step's pixels)
    RawRows<T, R, KD> raw;
    if (tid == 0) *cbuf_n = 0;
    raw.load(img, H, W, x0, xa, vec, 0);
    // The first column-pass groups read row-pass rows above x0 that no step
    // writes.  The outputs that need them are never used, but the sliding
    // boxcar sum of a group carries its first window into the rows after it
    // (cs + new - old cancels exactly only for finite integers), so the rings
    // start as zeros instead of whatever the previous kernel left.
    for (int i = tid; i < 2 * 2 * XR * PWp / 4; i += kStripThreads)
        ((float4*)xg)[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float trunc_thr = 1.0f / 255.0f;

    for (int s = 0; s < nsteps; s++) {
        raw.store(stage, vec);
        __syncthreads();
        if (s + 1 < nsteps) raw.load(img, H, W, x0, xa, vec, s + 1);

        // ---- B: row pass (preprocess_rows.wgsl), 8 rows x PWp columns, 4 per thread
        {
            for (int t = tid; t < kStepRows * G::NG; t += kStripThreads) {
                const int j = t / G::NG, gq = t - j * G::NG;
                const int col = 4 * gq;
                const float4* src = (const float4*)(stage + j * RWp + col);
                float x[4 * G::NX4];
#pragma unroll
                for (int i = 0; i < G::NX4; i++) {
                    const float4 v = src[i];
                    x[4 * i] = v.x;
                    x[4 * i + 1] = v.y;
                    x[4 * i + 2] = v.z;
                    x[4 * i + 3] = v.w;
                }
                float og[4], ob[4];
                float cs = 0.0f;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    float gs = 0.0f;
                    if (!edge_cols) {
#pragma unroll
                        for (int i = 0; i <= 2 * R; i++) gs = __fmaf_rn(c.taps[i], x[k + i], gs);
                    } else {
                        // Gaussian taps outside the frame are skipped
                        const int gcol = ps + col + k;
#pragma unroll
                        for (int i = 0; i <= 2 * R; i++) {
                            const int gc = gcol + i - R;
                            if (gc >= 0 && gc < W) gs = __fmaf_rn(c.taps[i], x[k + i], gs);
                        }
                    }
                    if (kInt) {
                        // exact integers: the window sum, then sliding differences
                        if (k == 0) cs = Tree<2 * R + 1>::sum(x);
                        else cs = __fadd_rn(cs, __fsub_rn(x[k + 2 * R], x[k - 1]));
                    } else {
                        cs = 0.0f;
#pragma unroll
                        for (int i = 0; i <= 2 * R; i++) cs = __fadd_rn(cs, x[k + i]);
                    }
                    og[k] = div_gnorm<FAST>(gs, c);
                    ob[k] = cs;
                }
                const int xrow = (kStepRows * s + j) % XR;
                const float4 g4 = make_float4(og[0], og[1], og[2], og[3]);
                const float4 b4 = make_float4(ob[0], ob[1], ob[2], ob[3]);
                *(float4*)(xg + xrow * PWp + col) = g4;
                *(float4*)(xg + (xrow + XR) * PWp + col) = g4;
                *(float4*)(xb + xrow * PWp + col) = b4;
                *(float4*)(xb + (xrow + XR) * PWp + col) = b4;
            }
        }
        __syncthreads();

        // ---- C: column pass (preprocess_cols.wgsl) for the step's 8 processed
        // rows q = x0 + 8s - R + k, one column per thread
        if (tid < PWp) {
            const int pc = tid;
            const int q0 = x0 + kStepRows * s - R;
            const int gcol = ps + pc;
            // row-pass rows q0 - R .. q0 + 7 + R: relative index 8s - 2R + i
            const int w0 = (kStepRows * s + (XR - 2 * R)) % XR;
            const float* pg = xg + w0 * PWp + pc;
            const float* pb = xb + w0 * PWp + pc;
            float vg[kStepRows + 2 * R], vbx[kStepRows + 2 * R];
#pragma unroll
            for (int i = 0; i < kStepRows + 2 * R; i++) {
                vg[i] = pg[i * PWp];
                vbx[i] = pb[i * PWp];
            }
            const bool col_in = (gcol >= 0 && gcol < W);
            const bool rows_in = (q0 >= R && q0 + kStepRows - 1 < H - R);
            float cs = 0.0f;
            // processed row q has relative index q - (x0 - R) = 8s + k
            const int p0 = (kStepRows * s) % PR;
#pragma unroll
            for (int k = 0; k < kStepRows; k++) {
                const int q = q0 + k;
                float gs = 0.0f;
                if (rows_in) {
#pragma unroll
                    for (int i = 0; i <= 2 * R; i++) gs = __fmaf_rn(c.taps[i], vg[k + i], gs);
                } else {
#pragma unroll
                    for (int i = 0; i <= 2 * R; i++) {
                        const int gr = q + i - R;
                        if (gr >= 0 && gr < H) gs = __fmaf_rn(c.taps[i], vg[k + i], gs);
                    }
                }
                if (kInt) {
                    if (k == 0) cs = Tree<2 * R + 1>::sum(vbx);
                    else cs = __fadd_rn(cs, __fsub_rn(vbx[k + 2 * R], vbx[k - 1]));
                } else {
                    cs = 0.0f;
#pragma unroll
                    for (int i = 0; i <= 2 * R; i++) cs = __fadd_rn(cs, vbx[k + i]);
                }
                float r = __fsub_rn(div_gnorm<FAST>(gs, c), div_kk<FAST>(cs, c));
                if (c.truncate && r < trunc_thr) r = 0.0f;
                const float v = (col_in && q >= 0 && q < H) ? r : -INFINITY;
                int pp = p0 + k;
                if (pp >= PR) pp -= PR;
                pr[pp * PWp + pc] = v;
                pr[(pp + PR) * PWp + pc] = v;
            }
        }
        __syncthreads();

        // ---- D: vertical maximum over KD processed rows for the step's 8
        // dilation rows d = x0 + 8s - R - E + k, one column per thread
        const int dbase = x0 + kStepRows * s - R - E;
        if (tid < PWp - SH4) {
            const int pc = tid + SH4;
            const int vcol = tid;   // pc0-relative column
            // output k: processed rows d + k - O .. d + k + E, relative index
            // 8s - (KD - 1) + k + i
            const int w0 = (kStepRows * s + (2 * PR - (KD - 1))) % PR;
            const float* pp = pr + w0 * PWp + pc;
            float a[KD + kStepRows - 1];
#pragma unroll
            for (int i = 0; i < KD + kStepRows - 1; i++) a[i] = pp[i * PWp];
            // out k = max(a[k..6], mid = a[7..KD-1], a[KD..KD+k-1])
            const float mid = Tree<KD - 7>::max(a + 7);
            float sfx[7], pfx[8];
            sfx[6] = a[6];
#pragma unroll
            for (int k = 5; k >= 0; k--) sfx[k] = fmaxf(a[k], sfx[k + 1]);
            pfx[1] = a[KD];
#pragma unroll
            for (int k = 2; k < 8; k++) pfx[k] = fmaxf(pfx[k - 1], a[KD + k - 1]);
            vb[vcol] = fmaxf(sfx[0], mid);
#pragma unroll
            for (int k = 1; k < 7; k++) vb[k * PWp + vcol] = fmaxf(fmaxf(sfx[k], mid), pfx[k]);
            vb[7 * PWp + vcol] = fmaxf(mid, pfx[7]);
        }
        __syncthreads();

        // ---- E: horizontal maximum, the candidate test and the processed rows
        // (processed row d = dbase + jj is ring row (8s + jj - E) mod PR)
        extract_step<R, KD>(tid, vb, [&](int jj) { return pr + ((kStepRows * s + jj + (PR - E)) % PR) * PWp; },
                            dbase, R0, R1, c0, H, W, c, thr, st4, proc, cbuf_n, cbuf, cand_slot, cout, cand_cap,
                            flags);
        __syncthreads();
    }
    __syncthreads();
    flush_tile_cands(tid, cbuf_n, cbuf, cand_slot, cout, cand_cap, flags);
}


// Calls f(std::integral_constant<int, p>) for the runtime phase p < PER.
template <int PER, typename F>
__device__ __forceinline__ void by_phase(const int p, F&& f) {
    using std::integral_constant;
    static_assert(PER >= 1 && PER <= 4, "ring periods of 1 to 4 steps");
    if constexpr (PER == 1) {
        f(integral_constant<int, 0>{});
    } else if constexpr (PER == 2) {
        if (p == 0) f(integral_constant<int, 0>{});
        else f(integral_constant<int, 1>{});
    } else if constexpr (PER == 3) {
        if (p == 0) f(integral_constant<int, 0>{});
        else if (p == 1) f(integral_constant<int, 1>{});
        else f(integral_constant<int, 2>{});
    } else {
        if (p == 0) f(integral_constant<int, 0>{});
        else if (p == 1) f(integral_constant<int, 1>{});
        else if (p == 2) f(integral_constant<int, 2>{});
        else f(integral_constant<int, 3>{});
    }
}

// Single-copy rings of the integer-pixel tile: RING rows, a multiple of the
// 8-row step that holds both the column pass's window (8 + 2R row-pass rows)
// and the vertical maxima's (KD + 7 processed rows).
template <int R, int KD>
struct RingGeom {
    using G = StripGeom<R, KD>;
    static constexpr int rows = (kStepRows + 2 * R > KD + kStepRows - 1) ? kStepRows + 2 * R : KD + kStepRows - 1;
    static constexpr int RING = (rows + kStepRows - 1) / kStepRows * kStepRows;
    static constexpr int PER = RING / kStepRows;   // steps per ring period
    static constexpr size_t smem_floats =
        (size_t)kStepRows * G::RWp + 3 * (size_t)RING * G::PWp + 4 + kCandBuf;
    // 4 CTAs per SM (56 registers a thread) where the shared memory allows it
    // and the radius keeps the column pass's windows in registers
    static constexpr int min_blocks = (R <= 5 && (smem_floats * 4 + 1024) * 4 <= 227 * 1024) ? 4 : 3;
    static_assert(PER <= 4, "ring period");
    static_assert((smem_floats * 4 + 1024) * min_blocks <= 228 * 1024, "shared memory of the resident CTAs");
};

// The integer-pixel tile (same outputs as strip_tile; layout in the file
// header): strip of output columns [c0, c0 + 128), rows [R0, R1).
template <typename T, int R, int KD>
__device__ __forceinline__ void ring_tile(const T* __restrict__ img, float* __restrict__ proc, const LocateConsts& c,
                                          const int H, const int W, const int c0, const int R0, const int R1,
                                          const int vec_ok, const float thr, uint32_t* __restrict__ cand_slot,
                                          uint32_t* __restrict__ cout, const uint32_t cand_cap,
                                          uint32_t* __restrict__ flags) {
    using G = StripGeom<R, KD>;
    using RG = RingGeom<R, KD>;
    constexpr int O = G::O, E = G::E, PWp = G::PWp, RWp = G::RWp, SH4 = G::SH4;
    constexpr int RING = RG::RING, PER = RG::PER;
    static_assert(IsIntPix<T>::value, "row sums >= +0 need non-negative pixels");
    extern __shared__ float4 sm4[];
    float* sm = (float*)sm4;
    float* stage = sm;                          // [8][RWp]      raw columns xa .. xa+RWp
    float* xg = stage + kStepRows * RWp;        // [RING][PWp]   row pass g / gnorm
    float* xb = xg + RING * PWp;                // [RING][PWp]   row pass boxcar
    float* pr = xb + RING * PWp;                // [RING][PWp]   processed rows
    float* vb = stage;                          // [8][PWp]      vertical maxima (pc0-relative columns)
    uint32_t* cbuf_n = (uint32_t*)(pr + RING * PWp);   // [4]   buffered candidates, flush base
    uint32_t* cbuf = cbuf_n + 4;                // [kCandBuf]    candidate keys of the tile

    const int x0 = R0 - O - R;          // first raw / row-pass row
    const int pc0 = c0 - O;             // first processed column of the strip's dilation windows
    const int xa = pc0 - R - SH4;       // first staged raw column (a multiple of 4)
    const int ps = xa + R;              // processed column of row-pass index 0 (= pc0 - SH4)
    const int tid = threadIdx.x;
    const bool edge_cols = (xa < 0) || (xa + RWp > W);
    const bool vec = vec_ok && !edge_cols;
    const bool st4 = (W % 4 == 0) && ((uintptr_t)proc % 16 == 0);
    const int nsteps = (R1 - x0 + R + E + kStepRows - 1) / kStepRows;

    // ---- A: staging of raw rows (registers hold the next step's pixels)
    RawRows<T, R, KD> raw;
    if (tid == 0) *cbuf_n = 0;
    raw.load(img, H, W, x0, xa, vec, 0);
    // The first column-pass groups read row-pass rows above x0 that no step
    // writes; the sliding boxcar sum carries their values into the rows after
    // them, so the rings start as zeros.
    for (int i = tid; i < 2 * RING * PWp / 4; i += kStripThreads)
        ((float4*)xg)[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float trunc_thr = 1.0f / 255.0f;

    int phase = 0;   // s % PER
    for (int s = 0; s < nsteps; s++) {
        const int P8 = kStepRows * phase;   // first ring row of this step
        raw.store(stage, vec);
        __syncthreads();
        if (s + 1 < nsteps) raw.load(img, H, W, x0, xa, vec, s + 1);

        // ---- B: row pass (preprocess_rows.wgsl), 8 rows x PWp columns, 4 per thread
        for (int t = tid; t < kStepRows * G::NG; t += kStripThreads) {
            const int j = t / G::NG, gq = t - j * G::NG;
            const int col = 4 * gq;
            const float4* src = (const float4*)(stage + j * RWp + col);
            float x[4 * G::NX4];
#pragma unroll
            for (int i = 0; i < G::NX4; i++) {
                const float4 v = src[i];
                x[4 * i] = v.x;
                x[4 * i + 1] = v.y;
                x[4 * i + 2] = v.z;
                x[4 * i + 3] = v.w;
            }
            float og[4], ob[4];
            float cs = 0.0f;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                float gs = 0.0f;
                if (!edge_cols) {
#pragma unroll
                    for (int i = 0; i <= 2 * R; i++) gs = __fmaf_rn(c.taps[i], x[k + i], gs);
                } else {
                    // Gaussian taps outside the frame are skipped
                    const int gcol = ps + col + k;
#pragma unroll
                    for (int i = 0; i <= 2 * R; i++) {
                        const int gc = gcol + i - R;
                        if (gc >= 0 && gc < W) gs = __fmaf_rn(c.taps[i], x[k + i], gs);
                    }
                }
                // exact integers: the window sum, then sliding differences
                if (k == 0) cs = Tree<2 * R + 1>::sum(x);
                else cs = __fadd_rn(cs, __fsub_rn(x[k + 2 * R], x[k - 1]));
                og[k] = div_gnorm<true>(gs, c);
                ob[k] = cs;
            }
            // rows outside the frame: Gaussian row sum +0 (the column pass
            // skips them), boxcar of the clamped row
            const int grow = x0 + kStepRows * s + j;
            if (grow < 0 || grow >= H) og[0] = og[1] = og[2] = og[3] = 0.0f;
            const int xrow = P8 + j;
            *(float4*)(xg + xrow * PWp + col) = make_float4(og[0], og[1], og[2], og[3]);
            *(float4*)(xb + xrow * PWp + col) = make_float4(ob[0], ob[1], ob[2], ob[3]);
        }
        __syncthreads();

        // ---- C: column pass (preprocess_cols.wgsl) for the step's 8 processed
        // rows q = x0 + 8s - R + k, one column per thread
        by_phase<PER>(phase, [&](auto ph) {
            constexpr int P = decltype(ph)::value;
            if (tid < PWp) {
                const int pc = tid;
                const int q0 = x0 + kStepRows * s - R;
                const int gcol = ps + pc;
                // row-pass rows q0 - R .. q0 + 7 + R: ring rows 8P - 2R + i
                float vg[kStepRows + 2 * R], vbx[kStepRows + 2 * R];
#pragma unroll
                for (int i = 0; i < kStepRows + 2 * R; i++) {
                    const int rr = ((kStepRows * P - 2 * R + i) % RING + RING) % RING;
                    vg[i] = xg[rr * PWp + pc];
                    vbx[i] = xb[rr * PWp + pc];
                }
                const bool col_in = (gcol >= 0 && gcol < W);
                float cs = 0.0f;
#pragma unroll
                for (int k = 0; k < kStepRows; k++) {
                    const int q = q0 + k;
                    float gs = 0.0f;
#pragma unroll
                    for (int i = 0; i <= 2 * R; i++) gs = __fmaf_rn(c.taps[i], vg[k + i], gs);
                    if (k == 0) cs = Tree<2 * R + 1>::sum(vbx);
                    else cs = __fadd_rn(cs, __fsub_rn(vbx[k + 2 * R], vbx[k - 1]));
                    float r = __fsub_rn(div_gnorm<true>(gs, c), div_kk<true>(cs, c));
                    if (c.truncate && r < trunc_thr) r = 0.0f;
                    const float v = (col_in && q >= 0 && q < H) ? r : -INFINITY;
                    pr[(kStepRows * P + k) * PWp + pc] = v;
                }
            }
        });
        __syncthreads();

        // ---- D: vertical maximum over KD processed rows for the step's 8
        // dilation rows d = x0 + 8s - R - E + k, one column per thread
        const int dbase = x0 + kStepRows * s - R - E;
        by_phase<PER>(phase, [&](auto ph) {
            constexpr int P = decltype(ph)::value;
            if (tid < PWp - SH4) {
                const int pc = tid + SH4;
                const int vcol = tid;   // pc0-relative column
                // output k: processed rows d + k - O .. d + k + E, ring rows
                // 8P - (KD - 1) + k + i
                float a[KD + kStepRows - 1];
#pragma unroll
                for (int i = 0; i < KD + kStepRows - 1; i++) {
                    const int rr = ((kStepRows * P - (KD - 1) + i) % RING + RING) % RING;
                    a[i] = pr[rr * PWp + pc];
                }
                // out k = max(a[k..6], mid = a[7..KD-1], a[KD..KD+k-1])
                const float mid = Tree<KD - 7>::max(a + 7);
                float sfx[7], pfx[8];
                sfx[6] = a[6];
#pragma unroll
                for (int k = 5; k >= 0; k--) sfx[k] = fmaxf(a[k], sfx[k + 1]);
                pfx[1] = a[KD];
#pragma unroll
                for (int k = 2; k < 8; k++) pfx[k] = fmaxf(pfx[k - 1], a[KD + k - 1]);
                vb[vcol] = fmaxf(sfx[0], mid);
#pragma unroll
                for (int k = 1; k < 7; k++) vb[k * PWp + vcol] = fmaxf(fmaxf(sfx[k], mid), pfx[k]);
                vb[7 * PWp + vcol] = fmaxf(mid, pfx[7]);
            }
        });
        __syncthreads();

        // ---- E: horizontal maximum, the candidate test and the processed rows
        // (processed row d = dbase + jj is ring row 8 * phase + jj - E, mod RING)
        extract_step<R, KD>(tid, vb,
                            [&](int jj) {
                                int prow = P8 + jj - E;
                                if (prow < 0) prow += RING;
                                return pr + prow * PWp;
                            },
                            dbase, R0, R1, c0, H, W, c, thr, st4, proc, cbuf_n, cbuf, cand_slot, cout, cand_cap,
                            flags);
        __syncthreads();
        phase = (phase + 1 == PER) ? 0 : phase + 1;
    }
    __syncthreads();
    flush_tile_cands(tid, cbuf_n, cbuf, cand_slot, cout, cand_cap, flags);
}

// Shared memory and CTAs per SM of the strip kernels for a pixel type.
template <typename T, int R, int KD>
struct StripCfg {
    static constexpr bool ring = IsIntPix<T>::value;
    static constexpr size_t smem_floats = ring ? RingGeom<R, KD>::smem_floats : StripGeom<R, KD>::smem_floats;
    static constexpr int min_blocks = ring ? RingGeom<R, KD>::min_blocks : StripGeom<R, KD>::min_blocks;
};

template <typename T, int R, int KD, bool FAST>
__global__ void __launch_bounds__(kStripThreads, (StripCfg<T, R, KD>::min_blocks))
strip_kernel(const T* __restrict__ frames, int64_t frame_stride, float* __restrict__ processed, const LocateConsts c,
             int SH, int vec_ok, uint32_t* __restrict__ cand_count, uint32_t* __restrict__ cand_keys,
             uint32_t cand_cap, uint32_t* __restrict__ flags) {
    const int H = c.H, W = c.W;
    const int f = blockIdx.z;
    const int R0 = blockIdx.y * SH;
    // extract_max.wgsl:37: pic_std * snr * rough_snr_factor
    const float thr = c.frame_std ? __fmul_rn(__fmul_rn(c.frame_std[f], c.snr), c.rough) : c.thr;
    if constexpr (StripCfg<T, R, KD>::ring)
        ring_tile<T, R, KD>(frames + (size_t)f * frame_stride, processed + (size_t)f * H * W, c, H, W,
                            blockIdx.x * kStripTW, R0, min(R0 + SH, H), vec_ok, thr, cand_count + f,
                            cand_keys + (size_t)f * cand_cap, cand_cap, flags);
    else
        strip_tile<T, R, KD, FAST>(frames + (size_t)f * frame_stride, processed + (size_t)f * H * W, c, H, W,
                                   blockIdx.x * kStripTW, R0, min(R0 + SH, H), vec_ok, thr, cand_count + f,
                                   cand_keys + (size_t)f * cand_cap, cand_cap, flags);
}

// Many frames of different sizes (frames of many videos) in one persistent
// launch: CTAs take tiles from a task list with a fixed stride.  The task and
// frame tables live in device memory, so a captured launch replays for any
// batch whose tables were rewritten.
template <typename T, int R, int KD, bool FAST>
__global__ void __launch_bounds__(kStripThreads, (StripCfg<T, R, KD>::min_blocks))
strip_ragged_kernel(const RaggedFrame* __restrict__ frames, const StripTask* __restrict__ tasks,
                    const int32_t* __restrict__ ntasks, float* __restrict__ processed, const LocateConsts c,
                    uint32_t* __restrict__ cand_count, uint32_t* __restrict__ cand_keys, uint32_t cand_cap,
                    uint32_t* __restrict__ flags) {
    const int n = *ntasks;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const StripTask tk = tasks[t];
        const RaggedFrame d = frames[tk.slot];
        if constexpr (StripCfg<T, R, KD>::ring)
            ring_tile<T, R, KD>((const T*)d.raw, processed + d.proc_off, c, d.H, d.W, tk.c0, tk.r0, tk.r1,
                                d.vec_ok, c.thr, cand_count + tk.slot, cand_keys + (size_t)tk.slot * cand_cap,
                                cand_cap, flags);
        else
            strip_tile<T, R, KD, FAST>((const T*)d.raw, processed + d.proc_off, c, d.H, d.W, tk.c0, tk.r0, tk.r1,
                                       d.vec_ok, c.thr, cand_count + tk.slot, cand_keys + (size_t)tk.slot * cand_cap,
                                       cand_cap, flags);
    }
}

template <typename T, int R, int KD>
size_t strip_smem() {
    return StripCfg<T, R, KD>::smem_floats * sizeof(float);
}

template <typename T, int R, int KD, bool FAST>
cudaError_t strip_launch(const T* frames, int64_t frame_stride, float* processed, const LocateConsts& c, int nframes,
                         uint32_t* cand_count, uint32_t* cand_keys, uint32_t cand_cap, uint32_t* flags,
                         cudaStream_t st) {
    // row segments of at most 512 rows: enough CTAs for whole waves at 1024 rows and up
    const int SH = c.H > 512 ? 512 : c.H;
    dim3 grid((c.W + kStripTW - 1) / kStripTW, (c.H + SH - 1) / SH, nframes);
    const size_t smem = strip_smem<T, R, KD>();
    // 4-pixel loads need every row start (and the frames) aligned to 4 pixels
    const int vec_ok = (c.W % 4 == 0) && (frame_stride % 4 == 0) &&
                       ((uintptr_t)frames % (4 * sizeof(T)) == 0) ? 1 : 0;
    cudaFuncSetAttribute(strip_kernel<T, R, KD, FAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(strip_kernel<T, R, KD, FAST>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    strip_kernel<T, R, KD, FAST><<<grid, kStripThreads, smem, st>>>(frames, frame_stride, processed, c, SH, vec_ok,
                                                                     cand_count, cand_keys, cand_cap, flags);
    return cudaGetLastError();
}

// (smoothing radius, dilation size) pairs with a specialised kernel: the
// default separation = diameter + 1 for diameters 5..15 and the common
// separation = diameter case.
#define GT_STRIP_CASES(X) \
    X(2, 8) X(3, 11) X(4, 12) X(4, 14) X(5, 15) X(5, 16) X(6, 18) X(6, 19) X(7, 21) X(7, 22)

// Integer pixels use the proven constant division (fast_div) and fall back to
// the tile kernel when it is not proven; float pixels use IEEE division.
template <typename T>
bool launch_strip(const T* frames, int64_t frame_stride, float* processed, const LocateConsts& c, int nframes,
                  uint32_t* cand_count, uint32_t* cand_keys, uint32_t cand_cap, uint32_t* flags, cudaStream_t st,
                  cudaError_t* err) {
    constexpr bool kInt = IsIntPix<T>::value;
    if (kInt && !c.fast_div) return false;
#define GT_STRIP_TRY(RR, KK)                                                                              \
    if (c.R == RR && c.kd == KK) {                                                                       \
        *err = strip_launch<T, RR, KK, kInt>(frames, frame_stride, processed, c, nframes, cand_count,     \
                                             cand_keys, cand_cap, flags, st);                             \
        return true;                                                                                     \
    }
    GT_STRIP_CASES(GT_STRIP_TRY)
#undef GT_STRIP_TRY
    return false;
}

template <typename T, int R, int KD, bool FAST>
cudaError_t strip_ragged_launch(const RaggedFrame* frames, const StripTask* tasks, const int32_t* ntasks, int grid,
                                float* processed, const LocateConsts& c, uint32_t* cand_count, uint32_t* cand_keys,
                                uint32_t cand_cap, uint32_t* flags, cudaStream_t st) {
    const size_t smem = strip_smem<T, R, KD>();
    cudaFuncSetAttribute(strip_ragged_kernel<T, R, KD, FAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(strip_ragged_kernel<T, R, KD, FAST>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    strip_ragged_kernel<T, R, KD, FAST><<<grid, kStripThreads, smem, st>>>(frames, tasks, ntasks, processed, c,
                                                                            cand_count, cand_keys, cand_cap, flags);
    return cudaGetLastError();
}

template <typename T>
bool launch_strip_ragged(const RaggedFrame* frames, const StripTask* tasks, const int32_t* ntasks, int grid,
                         float* processed, const LocateConsts& c, uint32_t* cand_count, uint32_t* cand_keys,
                         uint32_t cand_cap, uint32_t* flags, cudaStream_t st, cudaError_t* err) {
    constexpr bool kInt = IsIntPix<T>::value;
    if (kInt && !c.fast_div) return false;
#define GT_STRIP_TRY(RR, KK)                                                                                  \
    if (c.R == RR && c.kd == KK) {                                                                           \
        *err = strip_ragged_launch<T, RR, KK, kInt>(frames, tasks, ntasks, grid, processed, c, cand_count,   \
                                                    cand_keys, cand_cap, flags, st);                         \
        return true;                                                                                         \
    }
    GT_STRIP_CASES(GT_STRIP_TRY)
#undef GT_STRIP_TRY
    return false;
}

template <typename T>
int strip_blocks_per_sm(const LocateConsts& c) {
#define GT_STRIP_TRY(RR, KK)                                                                                  \
    if (c.R == RR && c.kd == KK) return StripCfg<T, RR, KK>::min_blocks;
    GT_STRIP_CASES(GT_STRIP_TRY)
#undef GT_STRIP_TRY
    return 0;
}

template <typename T>
int strip_tile_width(const LocateConsts& c) {
    constexpr bool kInt = IsIntPix<T>::value;
    if (kInt && !c.fast_div) return 0;
#define GT_STRIP_TRY(RR, KK)                                                                                  \
    if (c.R == RR && c.kd == KK) return kStripTW;
    GT_STRIP_CASES(GT_STRIP_TRY)
#undef GT_STRIP_TRY
    return 0;
}

// Processed image only: the dilation width is fixed at 8 (the smallest the
// tile geometry supports; the processed values do not depend on it) and the
// margin covers the whole frame, so the candidate test rejects every pixel
// (NaN and infinite values included) and no candidate list is touched.
#define GT_STRIP_PROC_CASES(X) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)
constexpr int kStripProcKD = 8;

template <typename T>
bool launch_strip_processed(const T* frames, int64_t frame_stride, float* processed, const LocateConsts& c,
                            int nframes, uint32_t* cand_count, uint32_t* cand_keys, uint32_t* flags, cudaStream_t st,
                            cudaError_t* err) {
    constexpr bool kInt = IsIntPix<T>::value;
    if (kInt && !c.fast_div) return false;
    LocateConsts cb = c;
    cb.kd = kStripProcKD;
    cb.o = (int32_t)((float)kStripProcKD / 2.0f - 0.5f);
    cb.margin = c.H > c.W ? c.H : c.W;
    cb.skip_zero = 0;
    cb.frame_std = nullptr;
    cb.thr = 0.0f;
#define GT_STRIP_PROC_TRY(RR)                                                                                  \
    if (c.R == RR) {                                                                                           \
        *err = strip_launch<T, RR, kStripProcKD, kInt>(frames, frame_stride, processed, cb, nframes, cand_count, \
                                                       cand_keys, 0, flags, st);                               \
        return true;                                                                                           \
    }
    GT_STRIP_PROC_CASES(GT_STRIP_PROC_TRY)
#undef GT_STRIP_PROC_TRY
    return false;
}

#define GT_STRIP_RAGGED_INST(T)                                                                                  \
    template bool launch_strip_ragged<T>(const RaggedFrame*, const StripTask*, const int32_t*, int, float*,      \
                                         const LocateConsts&, uint32_t*, uint32_t*, uint32_t, uint32_t*,         \
                                         cudaStream_t, cudaError_t*);                                            \
    template int strip_blocks_per_sm<T>(const LocateConsts&);                                                    \
    template int strip_tile_width<T>(const LocateConsts&);                                                       \
    template bool launch_strip_processed<T>(const T*, int64_t, float*, const LocateConsts&, int, uint32_t*,      \
                                            uint32_t*, uint32_t*, cudaStream_t, cudaError_t*);
GT_STRIP_RAGGED_INST(uint16_t)
GT_STRIP_RAGGED_INST(float)
GT_STRIP_RAGGED_INST(uint8_t)

template bool launch_strip<uint16_t>(const uint16_t*, int64_t, float*, const LocateConsts&, int, uint32_t*,
                                     uint32_t*, uint32_t, uint32_t*, cudaStream_t, cudaError_t*);
template bool launch_strip<float>(const float*, int64_t, float*, const LocateConsts&, int, uint32_t*, uint32_t*,
                                  uint32_t, uint32_t*, cudaStream_t, cudaError_t*);
template bool launch_strip<uint8_t>(const uint8_t*, int64_t, float*, const LocateConsts&, int, uint32_t*, uint32_t*,
                                    uint32_t, uint32_t*, cudaStream_t, cudaError_t*);

// ------------------------------------------------ constant-divisor proof
// Counts the mantissas x in [1, 2) where fma(x, zh, x*zl) != x / d.  Both
// sides scale exactly with x by powers of two while x*zl and the quotient
// stay normal, so zero mismatches prove the identity for every dividend in
// that exponent range (and for zero).
__global__ void const_div_check_kernel(float d, float zh, float zl, unsigned int* bad) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= (1u << 23)) return;
    const float x = __uint_as_float(0x3F800000u | m);
    const float want = __fdiv_rn(x, d);
    const float got = __fmaf_rn(x, zh, __fmul_rn(x, zl));
    const bool ok = __float_as_uint(got) == __float_as_uint(want);
    const unsigned int nbad = __popc(__ballot_sync(0xffffffffu, !ok));
    if (nbad && (threadIdx.x & 31) == 0) atomicAdd(bad, nbad);
}

__device__ unsigned int g_const_div_bad;

bool const_div_proven(float d, float zh, float zl, cudaStream_t st) {
    static std::mutex mu;
    static std::map<std::tuple<uint32_t, uint32_t, uint32_t>, bool> cache;
    uint32_t kd, kh, kl;
    memcpy(&kd, &d, 4);
    memcpy(&kh, &zh, 4);
    memcpy(&kl, &zl, 4);
    const auto key = std::make_tuple(kd, kh, kl);
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    unsigned int* bad = nullptr;
    if (cudaGetSymbolAddress((void**)&bad, g_const_div_bad) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    unsigned int nbad = 1;
    if (cudaMemsetAsync(bad, 0, sizeof(unsigned int), st) != cudaSuccess) return false;
    const_div_check_kernel<<<(1u << 23) / 256, 256, 0, st>>>(d, zh, zl, bad);
    if (cudaMemcpyAsync(&nbad, bad, sizeof(nbad), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const bool ok = (nbad == 0);
    cache[key] = ok;
    return ok;
}

}  // namespace gt
