// gt_strip.cu — streaming bandpass + grey-dilation local-max kernel (sm_100a).
//
// Same results as bandpass_kernel<T, true> (preprocess_rows.wgsl,
// preprocess_cols.wgsl, max_rows.wgsl, extract_max.wgsl), organised for
// throughput: a CTA owns a strip of 128 output columns and walks down a
// segment of rows eight rows per step.  The row-pass results (g/gauss_norm,
// boxcar) and the processed rows live in shared-memory ring buffers, so the
// vertical halo is computed once per strip instead of once per tile; the tap
// loops are unrolled for the compile-time radius (taps come from the constant
// bank); each thread computes four outputs per pass from registers; the
// dilation maximum of a 4-output run is built from one shared middle block
// plus prefix/suffix maxima.  The floating-point operation sequence of every
// output is the oracle's: sequential fused multiply-adds over the taps,
// sequential boxcar sums (a sliding sum for integer inputs, where every
// partial sum is an exactly representable integer), IEEE division.
#include <math.h>

#include "gt_internal.cuh"
#include "gt_kernels.h"

namespace gt {

constexpr int kStripTW = 128;
constexpr int kStripThreads = 288;
constexpr int kStepRows = 8;

template <int R, int KD>
struct StripGeom {
    static constexpr int O = (int)((float)KD / 2.0f - 0.5f);
    static constexpr int E = KD - 1 - O;
    static constexpr int PW = kStripTW + KD - 1;   // processed / row-pass columns
    static constexpr int RW = PW + 2 * R;          // raw columns
    static constexpr int XR = ((kStepRows + 2 * R + 7) / 8) * 8;   // row-pass ring rows
    static constexpr int PR = ((kStepRows + KD - 1 + 7) / 8) * 8;  // processed ring rows
    static constexpr int RAWN = kStepRows * RW;
    static constexpr int RAWPT = (RAWN + kStripThreads - 1) / kStripThreads;
    static constexpr size_t smem_floats = (size_t)kStepRows * RW + 2 * (size_t)XR * PW + (size_t)PR * PW +
                                          (size_t)kStepRows * PW;
};

template <typename T>
struct IsIntPix {
    static constexpr bool value = !std::is_same<T, float>::value;
};

template <typename T, int R, int KD>
__global__ void __launch_bounds__(kStripThreads, 3)
strip_kernel(const T* __restrict__ frames, int64_t frame_stride, float* __restrict__ processed, const LocateConsts c,
             int SH, uint32_t* __restrict__ cand_count, uint32_t* __restrict__ cand_keys, uint32_t cand_cap,
             uint32_t* __restrict__ flags) {
    using G = StripGeom<R, KD>;
    constexpr int O = G::O, E = G::E, PW = G::PW, RW = G::RW, XR = G::XR, PR = G::PR;
    constexpr bool kInt = IsIntPix<T>::value;
    extern __shared__ float sm[];
    float* stage = sm;                          // [8][RW]
    float* xg = stage + kStepRows * RW;         // [XR][PW]
    float* xb = xg + XR * PW;                   // [XR][PW]
    float* pr = xb + XR * PW;                   // [PR][PW]
    float* vb = pr + PR * PW;                   // [8][PW]

    const int H = c.H, W = c.W;
    const int f = blockIdx.z;
    const int c0 = blockIdx.x * kStripTW;
    const int R0 = blockIdx.y * SH;
    const int R1 = min(R0 + SH, H);
    const int x0 = R0 - O - R;          // first raw/row-pass row
    const int pc0 = c0 - O;             // first processed column
    const int rc0 = pc0 - R;            // first raw column
    const T* img = frames + (size_t)f * frame_stride;
    float* proc = processed + (size_t)f * H * W;
    const int tid = threadIdx.x;
    const bool edge_cols = (rc0 < 0) || (rc0 + RW > W);
    // steps until the dilation rows reach R1: x0 + 8s - R - E + 8 >= R1
    const int nsteps = (R1 - x0 + R + E + kStepRows - 1) / kStepRows;

    float pre[G::RAWPT];
    auto load_raw = [&](int s) {
#pragma unroll
        for (int q = 0; q < G::RAWPT; q++) {
            int idx = tid + q * kStripThreads;
            float v = 0.0f;
            if (idx < G::RAWN) {
                int j = idx / RW, k = idx - j * RW;
                int gr = min(max(x0 + kStepRows * s + j, 0), H - 1);
                int gc = min(max(rc0 + k, 0), W - 1);
                v = load_px<T>(img, (size_t)gr * W + gc);
            }
            pre[q] = v;
        }
    };
    load_raw(0);
    const float trunc_thr = 1.0f / 255.0f;
    uint32_t* cout = cand_keys + (size_t)f * cand_cap;

    for (int s = 0; s < nsteps; s++) {
        // ---- A: raw rows of this step into shared memory; prefetch the next step
#pragma unroll
        for (int q = 0; q < G::RAWPT; q++) {
            int idx = tid + q * kStripThreads;
            if (idx < G::RAWN) stage[idx] = pre[q];
        }
        __syncthreads();
        if (s + 1 < nsteps) load_raw(s + 1);

        // ---- B: row pass (preprocess_rows.wgsl) for 8 rows x PW columns, 4 per thread
        {
            constexpr int NG = (PW + 3) / 4;
            for (int t = tid; t < kStepRows * NG; t += kStripThreads) {
                const int j = t / NG, gq = t - j * NG;
                const int col = 4 * gq;
                const float* src = stage + j * RW + col;
                float x[4 + 2 * R];
#pragma unroll
                for (int i = 0; i < 4 + 2 * R; i++) x[i] = (col + i < RW) ? src[i] : 0.0f;
                const int xrow = (kStepRows * s + j) % XR;
                float cs = 0.0f;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    if (col + k >= PW) break;
                    float gs = 0.0f;
                    if (!edge_cols) {
#pragma unroll
                        for (int i = 0; i <= 2 * R; i++) gs = __fmaf_rn(c.taps[i], x[k + i], gs);
                    } else {
                        const int gcol = pc0 + col + k;
#pragma unroll
                        for (int i = 0; i <= 2 * R; i++) {
                            int gc = gcol + i - R;
                            if (gc >= 0 && gc < W) gs = __fmaf_rn(c.taps[i], x[k + i], gs);
                        }
                    }
                    if (kInt) {
                        if (k == 0) {
#pragma unroll
                            for (int i = 0; i <= 2 * R; i++) cs = __fadd_rn(cs, x[i]);
                        } else {
                            cs = __fsub_rn(__fadd_rn(cs, x[k + 2 * R]), x[k - 1]);
                        }
                    } else {
                        cs = 0.0f;
#pragma unroll
                        for (int i = 0; i <= 2 * R; i++) cs = __fadd_rn(cs, x[k + i]);
                    }
                    xg[xrow * PW + col + k] = __fdiv_rn(gs, c.gnorm);
                    xb[xrow * PW + col + k] = cs;
                }
            }
        }
        __syncthreads();

        // ---- C: column pass (preprocess_cols.wgsl) for processed rows q = x0 + 8s - R + jj
        {
            const int qbase = x0 + kStepRows * s - R;
            for (int t = tid; t < 2 * PW; t += kStripThreads) {
                const int h = t / PW, pc = t - h * PW;
                const int q0 = qbase + 4 * h;        // first of 4 processed rows
                const int gcol = pc0 + pc;
                float vg[4 + 2 * R], vbx[4 + 2 * R];
#pragma unroll
                for (int i = 0; i < 4 + 2 * R; i++) {
                    // X row q0 - R + i lives at ring row (q0 - R + i - x0) mod XR
                    int rr = (q0 - R + i - x0 + 8 * XR) % XR;
                    vg[i] = xg[rr * PW + pc];
                    vbx[i] = xb[rr * PW + pc];
                }
                const bool col_in = (gcol >= 0 && gcol < W);
                float cs = 0.0f;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int q = q0 + k;
                    float res;
                    float gs = 0.0f;
                    if (q >= R && q < H - R) {
#pragma unroll
                        for (int i = 0; i <= 2 * R; i++) gs = __fmaf_rn(c.taps[i], vg[k + i], gs);
                    } else {
#pragma unroll
                        for (int i = 0; i <= 2 * R; i++) {
                            int gr = q + i - R;
                            if (gr >= 0 && gr < H) gs = __fmaf_rn(c.taps[i], vg[k + i], gs);
                        }
                    }
                    if (kInt) {
                        if (k == 0) {
#pragma unroll
                            for (int i = 0; i <= 2 * R; i++) cs = __fadd_rn(cs, vbx[i]);
                        } else {
                            cs = __fsub_rn(__fadd_rn(cs, vbx[k + 2 * R]), vbx[k - 1]);
                        }
                    } else {
                        cs = 0.0f;
#pragma unroll
                        for (int i = 0; i <= 2 * R; i++) cs = __fadd_rn(cs, vbx[k + i]);
                    }
                    res = __fsub_rn(__fdiv_rn(gs, c.gnorm), __fdiv_rn(cs, c.kk));
                    if (c.truncate && res < trunc_thr) res = 0.0f;
                    const bool in = col_in && q >= 0 && q < H;
                    const int prow = (q - x0 + R + 8 * PR) % PR;
                    pr[prow * PW + pc] = in ? res : -INFINITY;
                    // the segment's own rows and the strip's own columns go to HBM
                    if (in && q >= R0 && q < R1 && pc >= O && pc < O + kStripTW) proc[(size_t)q * W + gcol] = res;
                }
            }
        }
        __syncthreads();

        // ---- D: vertical maximum over KD processed rows for dilation rows d = x0 + 8s - R - E + jj
        const int dbase = x0 + kStepRows * s - R - E;
        {
            for (int t = tid; t < 2 * PW; t += kStripThreads) {
                const int h = t / PW, pc = t - h * PW;
                const int d0 = dbase + 4 * h;
                // window of output k: rows d0 + k - O .. d0 + k + E
                float a[KD + 3];
#pragma unroll
                for (int i = 0; i < KD + 3; i++) {
                    int rr = (d0 - O + i - x0 + R + 8 * PR) % PR;
                    a[i] = pr[rr * PW + pc];
                }
                float mid = a[3];
#pragma unroll
                for (int i = 4; i < KD; i++) mid = fmaxf(mid, a[i]);
                // out k = max(a[k..2], mid(a[3..KD-1]), a[KD..KD+k-1])
                float s2 = a[2], s1 = fmaxf(a[1], s2), s0 = fmaxf(a[0], s1);
                float p1 = a[KD], p2 = fmaxf(p1, a[KD + 1]), p3 = fmaxf(p2, a[KD + 2]);
                const int vr = 4 * h;
                vb[(vr + 0) * PW + pc] = fmaxf(s0, mid);
                vb[(vr + 1) * PW + pc] = fmaxf(fmaxf(s1, mid), p1);
                vb[(vr + 2) * PW + pc] = fmaxf(fmaxf(s2, mid), p2);
                vb[(vr + 3) * PW + pc] = fmaxf(mid, p3);
            }
        }
        __syncthreads();

        // ---- E: horizontal maximum and the candidate test (extract_max.wgsl)
        {
            const int t = tid;
            int cnt = 0;
            uint32_t cmask = 0;
            int cd = 0, ccol = 0;
            if (t < kStepRows * (kStripTW / 4)) {
                const int jj = t / (kStripTW / 4), cg = t - jj * (kStripTW / 4);
                const int d = dbase + jj;
                const int cc = 4 * cg;  // interior column offset; processed column = cc + O
                if (d >= R0 && d < R1) {
                    float a[KD + 3];
#pragma unroll
                    for (int i = 0; i < KD + 3; i++) a[i] = vb[jj * PW + cc + i];
                    float mid = a[3];
#pragma unroll
                    for (int i = 4; i < KD; i++) mid = fmaxf(mid, a[i]);
                    float s2 = a[2], s1 = fmaxf(a[1], s2), s0 = fmaxf(a[0], s1);
                    float p1 = a[KD], p2 = fmaxf(p1, a[KD + 1]), p3 = fmaxf(p2, a[KD + 2]);
                    float m[4] = {fmaxf(s0, mid), fmaxf(fmaxf(s1, mid), p1), fmaxf(fmaxf(s2, mid), p2),
                                  fmaxf(mid, p3)};
                    const int prow = (d - x0 + R + 8 * PR) % PR;
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const int gc = c0 + cc + k;
                        if (gc >= W) continue;
                        if (d < c.margin || d >= H - c.margin || gc < c.margin || gc >= W - c.margin) continue;
                        const float center = pr[prow * PW + cc + k + O];
                        if (center < c.thr) continue;
                        if (m[k] > center) continue;
                        cmask |= 1u << k;
                        cnt++;
                    }
                    cd = d;
                    ccol = c0 + cc;
                }
            }
            // warp-aggregated reservation of output slots
            const int lane = tid & 31;
            int incl = cnt;
#pragma unroll
            for (int dd = 1; dd < 32; dd <<= 1) {
                int v = __shfl_up_sync(0xffffffffu, incl, dd);
                if (lane >= dd) incl += v;
            }
            const int wtot = __shfl_sync(0xffffffffu, incl, 31);
            uint32_t base = 0;
            if (wtot > 0) {
                if (lane == 31) base = atomicAdd(cand_count + f, (uint32_t)wtot);
                base = __shfl_sync(0xffffffffu, base, 31);
            }
            uint32_t pos = base + (uint32_t)(incl - cnt);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (!(cmask & (1u << k))) continue;
                if (pos < cand_cap) cout[pos] = (uint32_t)cd * (uint32_t)W + (uint32_t)(ccol + k);
                else atomicOr(flags, kFlagCandOverflow);
                pos++;
            }
        }
        __syncthreads();
    }
}

template <int R, int KD>
size_t strip_smem() {
    return StripGeom<R, KD>::smem_floats * sizeof(float);
}

template <typename T, int R, int KD>
cudaError_t strip_launch(const T* frames, int64_t frame_stride, float* processed, const LocateConsts& c, int nframes,
                         uint32_t* cand_count, uint32_t* cand_keys, uint32_t cand_cap, uint32_t* flags,
                         cudaStream_t st) {
    const int SH = c.H > 1024 ? 512 : c.H;
    dim3 grid((c.W + kStripTW - 1) / kStripTW, (c.H + SH - 1) / SH, nframes);
    const size_t smem = strip_smem<R, KD>();
    cudaFuncSetAttribute(strip_kernel<T, R, KD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    strip_kernel<T, R, KD><<<grid, kStripThreads, smem, st>>>(frames, frame_stride, processed, c, SH, cand_count,
                                                               cand_keys, cand_cap, flags);
    return cudaGetLastError();
}

// (smoothing radius, dilation size) pairs with a specialised kernel: the
// default separation = diameter + 1 for diameters 5..15 and the common
// separation = diameter case.
#define GT_STRIP_CASES(X) \
    X(2, 8) X(3, 11) X(4, 12) X(4, 14) X(5, 15) X(5, 16) X(6, 18) X(6, 19) X(7, 21) X(7, 22)

template <typename T>
bool launch_strip(const T* frames, int64_t frame_stride, float* processed, const LocateConsts& c, int nframes,
                  uint32_t* cand_count, uint32_t* cand_keys, uint32_t cand_cap, uint32_t* flags, cudaStream_t st,
                  cudaError_t* err) {
#define GT_STRIP_TRY(RR, KK)                                                                                \
    if (c.R == RR && c.kd == KK) {                                                                         \
        *err = strip_launch<T, RR, KK>(frames, frame_stride, processed, c, nframes, cand_count, cand_keys, \
                                       cand_cap, flags, st);                                               \
        return true;                                                                                       \
    }
    GT_STRIP_CASES(GT_STRIP_TRY)
#undef GT_STRIP_TRY
    return false;
}

template bool launch_strip<uint16_t>(const uint16_t*, int64_t, float*, const LocateConsts&, int, uint32_t*,
                                     uint32_t*, uint32_t, uint32_t*, cudaStream_t, cudaError_t*);
template bool launch_strip<float>(const float*, int64_t, float*, const LocateConsts&, int, uint32_t*, uint32_t*,
                                  uint32_t, uint32_t*, cudaStream_t, cudaError_t*);
template bool launch_strip<uint8_t>(const uint8_t*, int64_t, float*, const LocateConsts&, int, uint32_t*, uint32_t*,
                                    uint32_t, uint32_t*, cudaStream_t, cudaError_t*);

}  // namespace gt
