// gt_locate.cu — Crocker–Grier locate kernels for sm_100a.
//
//   bandpass_kernel   preprocess_rows.wgsl + preprocess_cols.wgsl (+ max_rows.wgsl
//                     and extract_max.wgsl when kCand): one CTA per 32x64 tile of
//                     one frame; the raw tile with its halo, the row-pass result
//                     and the processed tile live in shared memory, only the
//                     processed interior and the candidate pixels reach HBM.
//   walk_kernel       walk.wgsl + characterize.wgsl, one thread per candidate.
//   finalize_kernel   canonical order, filter_close_trackpy / prune_blobs_log and
//                     the doughnut correction (src/execute_gpu.rs:556-790), one CTA
//                     per frame.
//   scatter_kernel    per-frame results into the output table columns.
#include <math.h>

#include "gt_internal.cuh"
#include "gt_kernels.h"

namespace gt {

// ------------------------------------------------------------------ bandpass
template <typename T, bool kCand>
__global__ void __launch_bounds__(kLocateThreads)
bandpass_kernel(const T* __restrict__ frames, int64_t frame_stride, float* __restrict__ processed,
                const LocateConsts c, uint32_t* __restrict__ cand_count, uint32_t* __restrict__ cand_keys,
                uint32_t cand_cap, uint32_t* __restrict__ flags) {
    extern __shared__ float smem[];
    const int H = c.H, W = c.W, R = c.R;
    const int kd = kCand ? c.kd : 1;
    const int o = kCand ? c.o : 0;
    constexpr int TH = kLocateTH, TW = kLocateTW;
    const int r0 = blockIdx.y * TH, c0 = blockIdx.x * TW;
    const int f = blockIdx.z;
    const T* img = frames + (size_t)f * frame_stride;
    float* proc = processed + (size_t)f * H * W;

    const int PH = TH + kd - 1, PW = TW + kd - 1;
    const int pr0 = r0 - o, pc0 = c0 - o;
    const int XH = PH + 2 * R, RW = PW + 2 * R;
    const int xr0 = pr0 - R, rc0 = pc0 - R;
    float* sraw = smem;
    float* sxg = sraw + XH * RW;
    float* sxb = sxg + XH * PW;
    float* sp = sxb + XH * PW;
    float* sv = sp + PH * PW;
    const int tid = threadIdx.x;

    // raw tile with clamp-to-edge addressing (the boxcar's addressing); 8
    // independent loads per thread in flight before their shared-memory stores
    TileRowCol rc(tid, (int)blockDim.x, RW);  // this thread's elements in order
    for (int i0 = 0; i0 < XH * RW; i0 += 8 * (int)blockDim.x) {
        float v[8];
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const int idx = i0 + b * (int)blockDim.x + tid;
            const int gr = min(max(xr0 + rc.r, 0), H - 1);
            const int gc = min(max(rc0 + rc.c, 0), W - 1);
            v[b] = idx < XH * RW ? load_px<T>(img, (size_t)gr * W + gc) : 0.0f;
            rc.advance();
        }
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const int idx = i0 + b * (int)blockDim.x + tid;
            if (idx < XH * RW) sraw[idx] = v[b];
        }
    }
    __syncthreads();
    // a tile whose raw rows and columns all lie inside the frame needs no
    // per-tap bounds tests or clamps (every tap counts, every clamp is the
    // identity: the same operation sequence)
    const bool inside = xr0 >= 0 && xr0 + XH <= H && rc0 >= 0 && rc0 + RW <= W;

    // preprocess_rows.wgsl:30-54 — Gaussian taps skip out-of-frame columns,
    // the boxcar sums clamped columns; temp = (g / gauss_norm, box)
    TileRowCol rp(tid, (int)blockDim.x, PW);
    for (int idx = tid; idx < XH * PW; idx += blockDim.x, rp.advance()) {
        const int rr = rp.r, cc = rp.c;
        const float* rowp = sraw + rr * RW + cc;
        const int gcol = pc0 + cc;
        float gs = 0.0f, cs = 0.0f;
        if (inside) {
            for (int i = 0; i <= 2 * R; i++) {
                const float x = rowp[i];
                gs = __fmaf_rn(c.taps[i], x, gs);
                cs = __fadd_rn(cs, x);
            }
        } else {
            for (int i = 0; i <= 2 * R; i++) {
                float x = rowp[i];
                int gc = gcol + i - R;
                if (gc >= 0 && gc < W) gs = __fmaf_rn(c.taps[i], x, gs);
                cs = __fadd_rn(cs, x);
            }
        }
        sxg[idx] = __fdiv_rn(gs, c.gnorm);
        sxb[idx] = cs;
    }
    __syncthreads();

    // preprocess_cols.wgsl:29-59
    const float trunc_thr = 1.0f / 255.0f;
    TileRowCol cp(tid, (int)blockDim.x, PW);
    for (int idx = tid; idx < PH * PW; idx += blockDim.x, cp.advance()) {
        const int pr = cp.r, pc = cp.c;
        int grow = pr0 + pr, gcol = pc0 + pc;
        if (grow < 0 || grow >= H || gcol < 0 || gcol >= W) {
            sp[idx] = -INFINITY;  // outside the frame: never part of a dilation window
            continue;
        }
        float gs = 0.0f, cs = 0.0f;
        if (inside) {
            // rows grow - R .. grow + R are raw rows pr .. pr + 2R of the tile
            const float* pg = sxg + pr * PW + pc;
            const float* pb = sxb + pr * PW + pc;
            for (int i = 0; i <= 2 * R; i++) {
                gs = __fmaf_rn(c.taps[i], pg[i * PW], gs);
                cs = __fadd_rn(cs, pb[i * PW]);
            }
        } else {
            for (int i = 0; i <= 2 * R; i++) {
                int gr = grow + i - R;
                int xrow = min(max(gr, 0), H - 1) - xr0;
                float xg = sxg[xrow * PW + pc];
                float xb = sxb[xrow * PW + pc];
                if (gr >= 0 && gr < H) gs = __fmaf_rn(c.taps[i], xg, gs);
                cs = __fadd_rn(cs, xb);
            }
        }
        float res = __fsub_rn(__fdiv_rn(gs, c.gnorm), __fdiv_rn(cs, c.kk));
        if (c.truncate && res < trunc_thr) res = 0.0f;
        sp[idx] = res;
    }
    __syncthreads();

    // processed interior to HBM (the walk reads it back)
    for (int idx = tid; idx < TH * TW; idx += blockDim.x) {
        int r = idx / TW, cc = idx - r * TW;
        int gr = r0 + r, gc = c0 + cc;
        if (gr < H && gc < W) proc[(size_t)gr * W + gc] = sp[(r + o) * PW + cc + o];
    }
    if (!kCand) return;

    // max_rows.wgsl + extract_max.wgsl: the pixel is a candidate iff no value in
    // its kd x kd window (out-of-frame cells skipped) exceeds it
    TileRowCol mp(tid, (int)blockDim.x, PW);
    for (int idx = tid; idx < TH * PW; idx += blockDim.x, mp.advance()) {
        const int r = mp.r, cc = mp.c;
        float m = -INFINITY;
        for (int j = 0; j < kd; j++) m = fmaxf(m, sp[(r + j) * PW + cc]);
        sv[idx] = m;
    }
    __syncthreads();

    constexpr int PER = (TH * TW) / kLocateThreads;  // 8 consecutive pixels per thread
    // extract_max.wgsl:37: pic_std * snr * rough_snr_factor
    const float thr = c.frame_std ? __fmul_rn(__fmul_rn(c.frame_std[f], c.snr), c.rough) : c.thr;
    uint32_t mask = 0;
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < PER; k++) {
        int idx = tid * PER + k;
        int r = idx / TW, cc = idx - r * TW;
        int gr = r0 + r, gc = c0 + cc;
        if (gr >= H || gc >= W) continue;
        if (gr < c.margin || gr >= H - c.margin || gc < c.margin || gc >= W - c.margin) continue;
        float center = sp[(r + o) * PW + cc + o];
        if (center < thr) continue;
        if (c.skip_zero && center == 0.0f) continue;
        float m = -INFINITY;
        for (int j = 0; j < kd; j++) m = fmaxf(m, sv[r * PW + cc + j]);
        if (m > center) continue;
        mask |= 1u << k;
        cnt++;
    }
    // block exclusive scan of the per-thread counts (row-major tile order)
    __shared__ int warp_tot[kLocateThreads / 32];
    __shared__ uint32_t s_base;
    const int lane = tid & 31, wid = tid >> 5;
    int incl = cnt;
    for (int d = 1; d < 32; d <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int v = (lane < kLocateThreads / 32) ? warp_tot[lane] : 0;
        int s = v;
        for (int d = 1; d < 32; d <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= d) s += t;
        }
        if (lane < kLocateThreads / 32) warp_tot[lane] = s - v;  // exclusive
        if (lane == kLocateThreads / 32 - 1) {
            s_base = s > 0 ? atomicAdd(cand_count + f, (uint32_t)s) : 0u;
        }
    }
    __syncthreads();
    uint32_t pos = s_base + warp_tot[wid] + (incl - cnt);
    uint32_t* out = cand_keys + (size_t)f * cand_cap;
#pragma unroll
    for (int k = 0; k < PER; k++) {
        if (!(mask & (1u << k))) continue;
        int idx = tid * PER + k;
        int r = idx / TW, cc = idx - r * TW;
        if (pos < cand_cap) out[pos] = (uint32_t)((r0 + r) * W + (c0 + cc));
        else atomicOr(flags, kFlagCandOverflow);
        pos++;
    }
}

// ---------------------------------------------------------------------- walk
struct WalkRes {
    float x, y, mass, max, count;
};

// walk.wgsl:67-102 get_center
__device__ __forceinline__ WalkRes get_center(const float* __restrict__ p, int H, int W, int u, int v, int rint,
                                              float r2) {
    WalkRes res = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    for (int i = -rint; i <= rint; i++) {
        float x = (float)i;
        float x2 = __fmul_rn(x, x);
        int pu = u + i;
        for (int j = -rint; j <= rint; j++) {
            float y = (float)j;
            float mask = __fadd_rn(x2, __fmul_rn(y, y));
            if (mask > r2) continue;
            int pv = v + j;
            if (pu < 0 || pu >= H || pv < 0 || pv >= W) continue;
            float data = __ldg(p + (size_t)pu * W + pv);
            res.x = __fmaf_rn(data, x, res.x);
            res.y = __fmaf_rn(data, y, res.y);
            res.mass = __fadd_rn(res.mass, data);
            res.count = __fadd_rn(res.count, 1.0f);
            res.max = wgsl_max(res.max, data);
        }
    }
    res.x = __fdiv_rn(res.x, res.mass);
    res.y = __fdiv_rn(res.y, res.mass);
    return res;
}

// walk.wgsl:104-169
__device__ __forceinline__ WalkRes walk_one(const float* __restrict__ p, const LocateConsts& c, int u0, int v0,
                                            float r) {
    int pu = u0, pv = v0;
    WalkRes res = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    int rint;
    float r2;
    if (r <= 0.0f) {
        rint = (c.circle - 1) / 2;
        float rr = (float)rint;
        r2 = __fmul_rn(rr, rr);
    } else {
        rint = (int)ceilf(r);
        r2 = __fmul_rn(r, r);
    }
    const int margin = rint;
    const float thr = c.shift_thr;
    for (uint32_t it = 0; it < c.max_iter; it++) {
        res = get_center(p, c.H, c.W, pu, pv, rint, r2);
        bool changed = false;
        if ((res.x > thr) && (pu < c.H - 1 - margin)) { pu += 1; changed = true; }
        else if (res.x < -thr && pu > margin) { pu -= 1; changed = true; }
        if ((res.y > thr) && (pv < c.W - 1 - margin)) { pv += 1; changed = true; }
        else if ((res.y < -thr) && (pv > margin)) { pv -= 1; changed = true; }
        if (!changed) break;
    }
    res.x = __fadd_rn(res.x, (float)pu);
    res.y = __fadd_rn(res.y, (float)pv);
    return res;
}

// characterize.wgsl:61-143; angle table holds (sin 2θ, cos 2θ) for the
// (2 rint + 1)^2 integer offsets of the circle.
template <typename T>
__device__ __forceinline__ void characterize_one(const float* __restrict__ p, const T* __restrict__ raw,
                                                 const LocateConsts& c, Feature& ft, bool char_points,
                                                 const float2* __restrict__ angle_tab,
                                                 const int32_t* __restrict__ angle_off) {
    float r = ft.r;
    int rint;
    if (r <= 0.0f) {
        rint = (c.circle - 1) / 2;
        r = (float)rint;
    } else {
        rint = (int)ceilf(r);
    }
    const float r2 = __fmul_rn(r, r);
    const float2* angles = angle_tab + angle_off[rint];
    const int u = sat_f2i(rintf(ft.x));
    const int v = sat_f2i(rintf(ft.y));
    const int H = c.H, W = c.W;
    if (char_points) {
        float mass = 0.0f;
        for (int i = -rint; i <= rint; i++) {
            float x = (float)i;
            float x2 = __fmul_rn(x, x);
            for (int j = -rint; j <= rint; j++) {
                float y = (float)j;
                float mask = __fadd_rn(x2, __fmul_rn(y, y));
                if (mask > r2) continue;
                int pu = u + i, pv = v + j;
                if (pu < 0 || pu >= H || pv < 0 || pv >= W) continue;
                mass = __fadd_rn(mass, __ldg(p + (size_t)pu * W + pv));
            }
        }
        ft.mass = mass;
    }
    const float mass = ft.mass;
    float middle = 0.0f;
    const int64_t middle_idx = (int64_t)u * W + v;
    if (middle_idx >= 0 && middle_idx < (int64_t)H * W) middle = __ldg(p + middle_idx);
    float Rg = 0.0f, raw_mass = 0.0f, signal = 0.0f, es = 0.0f, ec = 0.0f;
    const int side = 2 * rint + 1;
    for (int i = -rint; i <= rint; i++) {
        float x = (float)i;
        float x2 = __fmul_rn(x, x);
        int pu = u + i;
        for (int j = -rint; j <= rint; j++) {
            float y = (float)j;
            float mask = __fadd_rn(x2, __fmul_rn(y, y));
            if (mask > r2) continue;
            int pv = v + j;
            if (pu < 0 || pu >= H || pv < 0 || pv >= W) continue;
            size_t idx = (size_t)pu * W + pv;
            float data = __ldg(p + idx);
            Rg = __fmaf_rn(data, mask, Rg);
            raw_mass = __fadd_rn(raw_mass, load_px<T>(raw, idx));
            signal = wgsl_max(signal, data);
            if ((i != 0) | (j != 0)) {
                float2 sc = __ldg(angles + (i + rint) * side + (j + rint));
                es = __fmaf_rn(data, sc.x, es);
                ec = __fmaf_rn(data, sc.y, ec);
            } else {
                ec = __fadd_rn(ec, data);
            }
        }
    }
    es = __fmul_rn(es, es);
    ec = __fmul_rn(ec, ec);
    ft.ecc = __fdiv_rn(__fsqrt_rn(__fadd_rn(es, ec)), __fsub_rn(mass, middle));
    ft.Rg = __fsqrt_rn(__fdiv_rn(Rg, mass));
    ft.raw = raw_mass;
    ft.signal = signal;
}

// walk.wgsl:171-229 + characterize over kept rows.  cand_r < 0 selects the
// trackpy circle; LoG passes the candidate's radius (per-radius candidates).
template <typename T>
__global__ void __launch_bounds__(128)
walk_kernel(const float* __restrict__ processed, const T* __restrict__ frames, int64_t frame_stride,
            const LocateConsts c, const uint32_t* __restrict__ cand_count, const uint32_t* __restrict__ cand_keys,
            uint32_t cand_cap, const float* __restrict__ radii, const int32_t* __restrict__ angle_off,
            const float2* __restrict__ angles, Feature* __restrict__ feats, uint32_t* __restrict__ feat_count,
            uint32_t feat_cap, uint32_t* __restrict__ flags, int32_t n_radius_slots) {
    const int f = blockIdx.y;
    const int slot = blockIdx.z;  // radius index for LoG, 0 for trackpy
    const int fs = f * n_radius_slots + slot;
    const uint32_t n = min(cand_count[fs], cand_cap);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t key = cand_keys[(size_t)fs * cand_cap + i];
    const int u = (int)(key / (uint32_t)c.W), v = (int)(key % (uint32_t)c.W);
    const float* p = processed + (size_t)f * c.H * c.W;
    const float r = radii ? radii[slot] : -1.0f;
    WalkRes res = walk_one(p, c, u, v, r);
    float minmass;
    if (c.minmass > 0.0f) minmass = c.minmass;
    else minmass = __fmul_rn(__fmul_rn(__fmul_rn(c.minmass_snr, res.count), c.frame_std ? c.frame_std[f] : c.image_std),
                             c.rough);
    if (!(res.mass >= minmass)) return;
    Feature ft;
    ft.key_hi = (uint32_t)slot;
    ft.key_lo = key;
    ft.x = res.x;
    ft.y = res.y;
    ft.mass = res.mass;
    ft.r = (r > 0.0f) ? r : 0.0f;
    ft.max_i = res.max;
    ft.count = res.count;
    ft.Rg = ft.raw = ft.signal = ft.ecc = 0.0f;
    ft.d_raw = ft.d_bg = ft.d_corr = __int_as_float(0x7fc00000);
    ft.ridx = slot;
    if (c.characterize) {
        const T* raw = frames + (size_t)f * frame_stride;
        characterize_one<T>(p, raw, c, ft, false, angles, angle_off);
    }
    uint32_t pos = atomicAdd(feat_count + f, 1u);
    if (pos < feat_cap) feats[(size_t)f * feat_cap + pos] = ft;
    else atomicOr(flags, kFlagFeatOverflow);
}

// ------------------------------------------------ walk for a fixed radius
// The trackpy circle has integer radius RI = (diameter - 1) / 2: membership
// of an offset (i*i + j*j <= RI*RI, exact in float) is decided at compile
// time, the loops unroll completely so every load is independent, and a
// circle that lies inside the frame skips the bounds tests.  The operation
// sequence per output is the one of get_center / walk / characterize above.
template <int RI, bool CHECK>
__device__ __forceinline__ WalkRes get_center_fixed(const float* __restrict__ p, int H, int W, int u, int v) {
    WalkRes res = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    const float* pc = p + (ptrdiff_t)u * W + v;
#pragma unroll
    for (int i = -RI; i <= RI; i++) {
        const float* prow = pc + (ptrdiff_t)i * W;
        const bool row_in = !CHECK || (u + i >= 0 && u + i < H);
#pragma unroll
        for (int j = -RI; j <= RI; j++) {
            if (i * i + j * j > RI * RI) continue;
            if (CHECK && (!row_in || v + j < 0 || v + j >= W)) continue;
            const float data = __ldg(prow + j);
            res.x = __fmaf_rn(data, (float)i, res.x);
            res.y = __fmaf_rn(data, (float)j, res.y);
            res.mass = __fadd_rn(res.mass, data);
            res.count = __fadd_rn(res.count, 1.0f);
            res.max = wgsl_max(res.max, data);
        }
    }
    res.x = __fdiv_rn(res.x, res.mass);
    res.y = __fdiv_rn(res.y, res.mass);
    return res;
}

template <int RI>
__device__ __forceinline__ WalkRes walk_fixed(const float* __restrict__ p, const LocateConsts& c, const int H,
                                              const int W, int u0, int v0) {
    int pu = u0, pv = v0;
    WalkRes res = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    const float thr = c.shift_thr;
    for (uint32_t it = 0; it < c.max_iter; it++) {
        if (pu >= RI && pu + RI < H && pv >= RI && pv + RI < W)
            res = get_center_fixed<RI, false>(p, H, W, pu, pv);
        else
            res = get_center_fixed<RI, true>(p, H, W, pu, pv);
        bool changed = false;
        if ((res.x > thr) && (pu < H - 1 - RI)) { pu += 1; changed = true; }
        else if (res.x < -thr && pu > RI) { pu -= 1; changed = true; }
        if ((res.y > thr) && (pv < W - 1 - RI)) { pv += 1; changed = true; }
        else if ((res.y < -thr) && (pv > RI)) { pv -= 1; changed = true; }
        if (!changed) break;
    }
    res.x = __fadd_rn(res.x, (float)pu);
    res.y = __fadd_rn(res.y, (float)pv);
    return res;
}

template <typename T, int RI, bool CHECK>
__device__ __forceinline__ void characterize_fixed_at(const float* __restrict__ p, const T* __restrict__ raw, int H,
                                                      int W, int u, int v, const float2* __restrict__ angles,
                                                      float* Rg_, float* raw_mass_, float* signal_, float* es_,
                                                      float* ec_) {
    constexpr int side = 2 * RI + 1;
    float Rg = 0.0f, raw_mass = 0.0f, signal = 0.0f, es = 0.0f, ec = 0.0f;
    const ptrdiff_t cidx = (ptrdiff_t)u * W + v;
#pragma unroll
    for (int i = -RI; i <= RI; i++) {
        const bool row_in = !CHECK || (u + i >= 0 && u + i < H);
#pragma unroll
        for (int j = -RI; j <= RI; j++) {
            if (i * i + j * j > RI * RI) continue;
            if (CHECK && (!row_in || v + j < 0 || v + j >= W)) continue;
            const ptrdiff_t idx = cidx + (ptrdiff_t)i * W + j;
            const float data = __ldg(p + idx);
            Rg = __fmaf_rn(data, (float)(i * i + j * j), Rg);
            raw_mass = __fadd_rn(raw_mass, load_px<T>(raw, (size_t)idx));
            signal = wgsl_max(signal, data);
            if ((i != 0) | (j != 0)) {
                const float2 sc = __ldg(angles + (i + RI) * side + (j + RI));
                es = __fmaf_rn(data, sc.x, es);
                ec = __fmaf_rn(data, sc.y, ec);
            } else {
                ec = __fadd_rn(ec, data);
            }
        }
    }
    *Rg_ = Rg;
    *raw_mass_ = raw_mass;
    *signal_ = signal;
    *es_ = es;
    *ec_ = ec;
}

template <typename T, int RI>
__global__ void __launch_bounds__(128)
walk_kernel_fixed(const float* __restrict__ processed, const T* __restrict__ frames, int64_t frame_stride,
                  const LocateConsts c, const uint32_t* __restrict__ cand_count,
                  const uint32_t* __restrict__ cand_keys, uint32_t cand_cap, const int32_t* __restrict__ angle_off,
                  const float2* __restrict__ angles, Feature* __restrict__ feats, uint32_t* __restrict__ feat_count,
                  uint32_t feat_cap, uint32_t* __restrict__ flags, const RaggedFrame* __restrict__ rf) {
    // frames in reverse order: the strip kernel wrote the last frames' processed
    // images last, so the first blocks find them in L2
    const int f = gridDim.y - 1 - blockIdx.y;
    const uint32_t n = min(cand_count[f], cand_cap);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // a ragged batch gives every frame slot its own size, pixels and processed image
    const int H = rf ? rf[f].H : c.H, W = rf ? rf[f].W : c.W;
    const uint32_t key = cand_keys[(size_t)f * cand_cap + i];
    const int u = (int)(key / (uint32_t)W), v = (int)(key % (uint32_t)W);
    const float* p = rf ? processed + rf[f].proc_off : processed + (size_t)f * H * W;
    const WalkRes res = walk_fixed<RI>(p, c, H, W, u, v);
    float minmass;
    if (c.minmass > 0.0f) minmass = c.minmass;
    else minmass = __fmul_rn(__fmul_rn(__fmul_rn(c.minmass_snr, res.count), c.frame_std ? c.frame_std[f] : c.image_std),
                             c.rough);
    if (!(res.mass >= minmass)) return;
    Feature ft;
    ft.key_hi = 0;
    ft.key_lo = key;
    ft.x = res.x;
    ft.y = res.y;
    ft.mass = res.mass;
    ft.r = 0.0f;
    ft.max_i = res.max;
    ft.count = res.count;
    ft.Rg = ft.raw = ft.signal = ft.ecc = 0.0f;
    ft.d_raw = ft.d_bg = ft.d_corr = __int_as_float(0x7fc00000);
    ft.ridx = 0;
    if (c.characterize) {
        // characterize.wgsl:61-143 at the rounded position, radius RI
        const T* raw = rf ? (const T*)rf[f].raw : frames + (size_t)f * frame_stride;
        const int cu = sat_f2i(rintf(ft.x)), cv = sat_f2i(rintf(ft.y));
        const float2* ang = angles + angle_off[RI];
        float middle = 0.0f;
        const int64_t middle_idx = (int64_t)cu * W + cv;
        if (middle_idx >= 0 && middle_idx < (int64_t)H * W) middle = __ldg(p + middle_idx);
        float Rg, raw_mass, signal, es, ec;
        if (cu >= RI && cu + RI < H && cv >= RI && cv + RI < W)
            characterize_fixed_at<T, RI, false>(p, raw, H, W, cu, cv, ang, &Rg, &raw_mass, &signal, &es, &ec);
        else
            characterize_fixed_at<T, RI, true>(p, raw, H, W, cu, cv, ang, &Rg, &raw_mass, &signal, &es, &ec);
        es = __fmul_rn(es, es);
        ec = __fmul_rn(ec, ec);
        ft.ecc = __fdiv_rn(__fsqrt_rn(__fadd_rn(es, ec)), __fsub_rn(ft.mass, middle));
        ft.Rg = __fsqrt_rn(__fdiv_rn(Rg, ft.mass));
        ft.raw = raw_mass;
        ft.signal = signal;
    }
    uint32_t pos = atomicAdd(feat_count + f, 1u);
    if (pos < feat_cap) feats[(size_t)f * feat_cap + pos] = ft;
    else atomicOr(flags, kFlagFeatOverflow);
}

// ------------------------------------------------ walk from learned seeds
// Seeds proposed by the learned network come without a processed image.
// Each warp takes 32 seeds and builds, for each, a PS x PS patch of processed
// values around it: the bandpass of preprocess_rows.wgsl / preprocess_cols.wgsl
// evaluated with the operation order of bandpass_kernel (clamped raw rows and
// columns, Gaussian taps skipped outside the frame, sequential sums, IEEE
// division), so every value equals the full-frame one bit for bit.  Each lane
// then climbs from its seed to a 3x3 local maximum of the processed image
// (inside the candidate margin; the current pixel wins ties, then row-major
// order; at most kLwClimb steps) -- a bandpass local maximum, the kind of
// pixel the plain method starts its walks from -- and walks and
// characterizes from there with the
// operation sequence of walk_kernel_fixed, reading its patch.  A lane whose
// walk or characterize circle leaves the patch asks for a patch centred
// where it stands and resumes there.
constexpr int kLwWarps = 4;
constexpr int kLwSeeds = 16;  // seeds per warp (lanes 0-15); all 32 lanes build the patches
constexpr int kLwShift = 1;   // walk steps a patch covers around its centre
constexpr int kLwClimb = 4;   // hill-climbing steps of a seed before its walk

__host__ __device__ constexpr int lw_patch(int RI) { return 2 * (RI + kLwShift) + 1; }
__host__ __device__ constexpr int lw_warp_floats(int RI, int R) {
    return kLwSeeds * lw_patch(RI) * lw_patch(RI) + (lw_patch(RI) + 2 * R) * (lw_patch(RI) + 2 * R) +
           2 * (lw_patch(RI) + 2 * R) * lw_patch(RI);
}

// Division by the bandpass constants: the proven two-float reciprocal when
// LocateConsts::fast_div is set (equal to IEEE division for every dividend
// of integer frames), else IEEE division.
__device__ __forceinline__ float lw_div(float x, float d, float zh, float zl, bool fast) {
    return fast ? __fmaf_rn(x, zh, __fmul_rn(x, zl)) : __fdiv_rn(x, d);
}

// The raw pixels of a patch (clamped rows and columns) are gathered into
// registers, lane-strided, so the next patch's loads are in flight while the
// current patch's passes run.
constexpr int kLwMaxR = 7;  // largest smoothing radius of the seed-patch walk
template <int RI>
struct LwRaw {
    static constexpr int RWMAX = lw_patch(RI) + 2 * kLwMaxR;
    static constexpr int NR = (RWMAX * RWMAX + 31) / 32;
    float v[NR];
};

// RC > 0: the smoothing radius as a compile-time constant (= c.R), else c.R.
template <typename T, int RI, int RC>
__device__ __forceinline__ void lw_raw_load(const T* __restrict__ img, const LocateConsts& c, int cu, int cv,
                                            LwRaw<RI>& reg, int lane) {
    constexpr int PS = lw_patch(RI);
    const int R = RC > 0 ? RC : c.R;
    const int H = c.H, W = c.W, RW = PS + 2 * R;
    const int br = cu - RI - kLwShift - R, bc = cv - RI - kLwShift - R;
#pragma unroll
    for (int k = 0; k < LwRaw<RI>::NR; k++) {
        const int idx = lane + 32 * k;
        if (idx < RW * RW) {
            const int rr = idx / RW, cc = idx - rr * RW;
            const int gr = min(max(br + rr, 0), H - 1), gc = min(max(bc + cc, 0), W - 1);
            reg.v[k] = load_px<T>(img, (size_t)gr * W + gc);
        }
    }
}

template <int RI, int RC>
__device__ __forceinline__ void lw_raw_store(const LwRaw<RI>& reg, const LocateConsts& c, float* raw, int lane) {
    const int RW = lw_patch(RI) + 2 * (RC > 0 ? RC : c.R);
#pragma unroll
    for (int k = 0; k < LwRaw<RI>::NR; k++) {
        const int idx = lane + 32 * k;
        if (idx < RW * RW) raw[idx] = reg.v[k];
    }
}

// Row and column passes of a patch centred at (cu, cv) from its raw pixels.
// A patch whose raw window lies inside the frame takes no bounds tests.
template <int RI, int RC>
__device__ void lw_passes(const LocateConsts& c, int cu, int cv, float* patch, const float* raw, float* xg, float* xb,
                          int lane) {
    constexpr int PS = lw_patch(RI);
    const int R = RC > 0 ? RC : c.R;
    const int H = c.H, W = c.W, RW = PS + 2 * R;
    const int r0 = cu - RI - kLwShift, c0 = cv - RI - kLwShift;  // patch origin
    const bool fast = c.fast_div != 0;
    const bool interior = r0 - R >= 0 && r0 + PS - 1 + R < H && c0 - R >= 0 && c0 + PS - 1 + R < W;
    if (interior) {
        for (int idx = lane; idx < RW * PS; idx += 32) {
            const int rr = idx / PS, pc = idx - rr * PS;
            const float* rowp = raw + rr * RW + pc;
            float gs = 0.0f, cs = 0.0f;
#pragma unroll
            for (int i = 0; i <= 2 * R; i++) {
                const float x = rowp[i];
                gs = __fmaf_rn(c.taps[i], x, gs);
                cs = __fadd_rn(cs, x);
            }
            xg[idx] = lw_div(gs, c.gnorm, c.zh_g, c.zl_g, fast);
            xb[idx] = cs;
        }
    } else {
        for (int idx = lane; idx < RW * PS; idx += 32) {
            const int rr = idx / PS, pc = idx - rr * PS;
            const float* rowp = raw + rr * RW + pc;
            const int gcol = c0 + pc;
            float gs = 0.0f, cs = 0.0f;
#pragma unroll
            for (int i = 0; i <= 2 * R; i++) {
                const float x = rowp[i];
                const int gc = gcol + i - R;
                if (gc >= 0 && gc < W) gs = __fmaf_rn(c.taps[i], x, gs);
                cs = __fadd_rn(cs, x);
            }
            xg[idx] = lw_div(gs, c.gnorm, c.zh_g, c.zl_g, fast);
            xb[idx] = cs;
        }
    }
    __syncwarp();
    const float trunc_thr = 1.0f / 255.0f;
    for (int idx = lane; idx < PS * PS; idx += 32) {
        const int pr = idx / PS, pc = idx - pr * PS;
        const int grow = r0 + pr, gcol = c0 + pc;
        float res = 0.0f;
        if (interior || (grow >= 0 && grow < H && gcol >= 0 && gcol < W)) {
            // raw row (pr + i) holds row clamp(grow + i - R): the row pass of a
            // clamped row is the row pass of the edge row
            float gs = 0.0f, cs = 0.0f;
#pragma unroll
            for (int i = 0; i <= 2 * R; i++) {
                const int gr = grow + i - R;
                const int xr = (pr + i) * PS + pc;
                if (interior || (gr >= 0 && gr < H)) gs = __fmaf_rn(c.taps[i], xg[xr], gs);
                cs = __fadd_rn(cs, xb[xr]);
            }
            res = __fsub_rn(lw_div(gs, c.gnorm, c.zh_g, c.zl_g, fast), lw_div(cs, c.kk, c.zh_k, c.zl_k, fast));
            if (c.truncate && res < trunc_thr) res = 0.0f;
        }
        patch[idx] = res;
    }
    __syncwarp();
}

// One processed value computed on its own (the same sequence as the patch).
template <typename T>
__device__ float lw_processed_at(const T* __restrict__ img, const LocateConsts& c, int u, int v) {
    const int H = c.H, W = c.W, R = c.R;
    float gs = 0.0f, cs = 0.0f;
    for (int i = 0; i <= 2 * R; i++) {
        const int gr = u + i - R;
        const int row = min(max(gr, 0), H - 1);
        float rg = 0.0f, rb = 0.0f;
        for (int j = 0; j <= 2 * R; j++) {
            const int gc = v + j - R;
            const float x = load_px<T>(img, (size_t)row * W + min(max(gc, 0), W - 1));
            if (gc >= 0 && gc < W) rg = __fmaf_rn(c.taps[j], x, rg);
            rb = __fadd_rn(rb, x);
        }
        if (gr >= 0 && gr < H) gs = __fmaf_rn(c.taps[i], __fdiv_rn(rg, c.gnorm), gs);
        cs = __fadd_rn(cs, rb);
    }
    float res = __fsub_rn(__fdiv_rn(gs, c.gnorm), __fdiv_rn(cs, c.kk));
    if (c.truncate && res < 1.0f / 255.0f) res = 0.0f;
    return res;
}

// get_center_fixed over a patch: `pc` points at (u, v), rows `stride` apart.
template <int RI, bool CHECK>
__device__ __forceinline__ WalkRes lw_get_center(const float* pc, int stride, int H, int W, int u, int v) {
    WalkRes res = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int i = -RI; i <= RI; i++) {
        const float* prow = pc + i * stride;
        const bool row_in = !CHECK || (u + i >= 0 && u + i < H);
#pragma unroll
        for (int j = -RI; j <= RI; j++) {
            if (i * i + j * j > RI * RI) continue;
            if (CHECK && (!row_in || v + j < 0 || v + j >= W)) continue;
            const float data = prow[j];
            res.x = __fmaf_rn(data, (float)i, res.x);
            res.y = __fmaf_rn(data, (float)j, res.y);
            res.mass = __fadd_rn(res.mass, data);
            res.count = __fadd_rn(res.count, 1.0f);
            res.max = wgsl_max(res.max, data);
        }
    }
    res.x = __fdiv_rn(res.x, res.mass);
    res.y = __fdiv_rn(res.y, res.mass);
    return res;
}

// characterize_fixed_at with the processed values from a patch.
template <typename T, int RI, bool CHECK>
__device__ __forceinline__ void lw_characterize(const float* pc, int stride, const T* __restrict__ raw, int H, int W,
                                                int u, int v, const float2* __restrict__ angles, float* Rg_,
                                                float* raw_mass_, float* signal_, float* es_, float* ec_) {
    constexpr int side = 2 * RI + 1;
    float Rg = 0.0f, raw_mass = 0.0f, signal = 0.0f, es = 0.0f, ec = 0.0f;
#pragma unroll
    for (int i = -RI; i <= RI; i++) {
        const bool row_in = !CHECK || (u + i >= 0 && u + i < H);
#pragma unroll
        for (int j = -RI; j <= RI; j++) {
            if (i * i + j * j > RI * RI) continue;
            if (CHECK && (!row_in || v + j < 0 || v + j >= W)) continue;
            const float data = pc[i * stride + j];
            Rg = __fmaf_rn(data, (float)(i * i + j * j), Rg);
            raw_mass = __fadd_rn(raw_mass, load_px<T>(raw, (size_t)(u + i) * W + (v + j)));
            signal = wgsl_max(signal, data);
            if ((i != 0) | (j != 0)) {
                const float2 sc = __ldg(angles + (i + RI) * side + (j + RI));
                es = __fmaf_rn(data, sc.x, es);
                ec = __fmaf_rn(data, sc.y, ec);
            } else {
                ec = __fadd_rn(ec, data);
            }
        }
    }
    *Rg_ = Rg;
    *raw_mass_ = raw_mass;
    *signal_ = signal;
    *es_ = es;
    *ec_ = ec;
}

template <typename T, int RI, int RC>
__global__ void __launch_bounds__(32 * kLwWarps)
walk_local_kernel(const T* __restrict__ frames, int64_t frame_stride, const LocateConsts c,
                  const uint32_t* __restrict__ cand_count, const uint32_t* __restrict__ cand_keys, uint32_t cand_cap,
                  const int32_t* __restrict__ angle_off, const float2* __restrict__ angles,
                  Feature* __restrict__ feats, uint32_t* __restrict__ feat_count, uint32_t feat_cap,
                  uint32_t* __restrict__ flags) {
    extern __shared__ float lsm[];
    constexpr int PS = lw_patch(RI);
    constexpr int OFF = RI + kLwShift;
    const int R = RC > 0 ? RC : c.R, RW = PS + 2 * R;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int f = blockIdx.y;
    const uint32_t n = min(cand_count[f], cand_cap);
    const uint32_t first = (blockIdx.x * kLwWarps + warp) * (uint32_t)kLwSeeds;
    if (first >= n) return;  // warp-uniform
    float* wbase = lsm + (size_t)warp * lw_warp_floats(RI, R);
    float* patches = wbase;
    float* raw = wbase + kLwSeeds * PS * PS;
    float* xg = raw + RW * RW;
    float* xb = xg + RW * PS;
    float* my = patches + (lane < kLwSeeds ? lane : 0) * PS * PS;
    const int H = c.H, W = c.W;
    const T* img = frames + (size_t)f * frame_stride;
    const uint32_t i = first + lane;
    const bool active = lane < kLwSeeds && i < n;
    const uint32_t key = active ? cand_keys[(size_t)f * cand_cap + i] : 0u;
    int pu = (int)(key / (uint32_t)W), pv = (int)(key % (uint32_t)W);
    int stage = active ? 0 : 2;  // 0 walk, 1 characterize, 2 done
    uint32_t it = 0;
    WalkRes res = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    float fx = 0.0f, fy = 0.0f;
    bool need = active, snapped = false;
    int want_u = pu, want_v = pv, cen_u = pu, cen_v = pv;
    const float thr = c.shift_thr;
    for (int round = 0; round < (int)c.max_iter + 4; round++) {
        const unsigned needmask = __ballot_sync(0xffffffffu, need);
        if (needmask == 0u && !__any_sync(0xffffffffu, stage != 2)) break;
        if (needmask) {
            // patch k's passes run while patch k+1's pixels are loaded
            LwRaw<RI> reg;
            int k = __ffs(needmask) - 1;
            int cu = __shfl_sync(0xffffffffu, want_u, k), cv = __shfl_sync(0xffffffffu, want_v, k);
            lw_raw_load<T, RI, RC>(img, c, cu, cv, reg, lane);
            for (unsigned m = needmask; m;) {
                m &= m - 1u;
                lw_raw_store<RI, RC>(reg, c, raw, lane);
                __syncwarp();
                const int kn = m ? __ffs(m) - 1 : 0;
                const int nu = __shfl_sync(0xffffffffu, want_u, kn), nv = __shfl_sync(0xffffffffu, want_v, kn);
                if (m) lw_raw_load<T, RI, RC>(img, c, nu, nv, reg, lane);
                lw_passes<RI, RC>(c, cu, cv, patches + k * PS * PS, raw, xg, xb, lane);
                k = kn;
                cu = nu;
                cv = nv;
            }
        }
        if (need) {
            cen_u = want_u;
            cen_v = want_v;
            need = false;
        }
        if (stage == 0 && !need && it == 0 && pu == cen_u && pv == cen_v && !snapped) {
            // climb to a 3x3 local maximum of the processed image (at most
            // kLwClimb steps, every 3x3 block inside the patch)
            snapped = true;
            for (int step = 0; step < kLwClimb; step++) {
                const float* pc = my + (pu - cen_u + OFF) * PS + (pv - cen_v + OFF);
                float best = pc[0];
                int bu = 0, bv = 0;
                for (int di = -1; di <= 1; di++)
                    for (int dj = -1; dj <= 1; dj++) {
                        const int u = pu + di, v = pv + dj;
                        if (u < c.margin || u >= H - c.margin || v < c.margin || v >= W - c.margin) continue;
                        const float val = pc[di * PS + dj];
                        if (val > best) {
                            best = val;
                            bu = di;
                            bv = dj;
                        }
                    }
                if (bu == 0 && bv == 0) break;
                if (abs(pu + bu - cen_u) > OFF - 1 || abs(pv + bv - cen_v) > OFF - 1) break;
                pu += bu;
                pv += bv;
            }
        }
        if (stage == 0) {
            bool fin = false;
            for (;;) {
                if (it >= c.max_iter) {
                    fin = true;
                    break;
                }
                if (abs(pu - cen_u) > kLwShift || abs(pv - cen_v) > kLwShift) {
                    need = true;
                    want_u = pu;
                    want_v = pv;
                    break;
                }
                const float* pc = my + (pu - cen_u + OFF) * PS + (pv - cen_v + OFF);
                if (pu >= RI && pu + RI < H && pv >= RI && pv + RI < W)
                    res = lw_get_center<RI, false>(pc, PS, H, W, pu, pv);
                else
                    res = lw_get_center<RI, true>(pc, PS, H, W, pu, pv);
                it++;
                bool changed = false;
                if ((res.x > thr) && (pu < H - 1 - RI)) { pu += 1; changed = true; }
                else if (res.x < -thr && pu > RI) { pu -= 1; changed = true; }
                if ((res.y > thr) && (pv < W - 1 - RI)) { pv += 1; changed = true; }
                else if ((res.y < -thr) && (pv > RI)) { pv -= 1; changed = true; }
                if (!changed) {
                    fin = true;
                    break;
                }
            }
            if (fin) {
                fx = __fadd_rn(res.x, (float)pu);
                fy = __fadd_rn(res.y, (float)pv);
                float minmass;
                if (c.minmass > 0.0f) minmass = c.minmass;
                else minmass = __fmul_rn(__fmul_rn(__fmul_rn(c.minmass_snr, res.count), c.image_std), c.rough);
                // a seed in an empty region (mass 0) proposes nothing
                stage = (res.mass >= minmass && res.mass > 0.0f) ? 1 : 2;
            }
        }
        if (stage == 1 && !need) {
            const int cu = sat_f2i(rintf(fx)), cv = sat_f2i(rintf(fy));
            if (abs(cu - cen_u) > kLwShift || abs(cv - cen_v) > kLwShift) {
                need = true;
                want_u = cu;
                want_v = cv;
            } else {
                Feature ft;
                ft.key_hi = 0;
                ft.key_lo = key;
                ft.x = fx;
                ft.y = fy;
                ft.mass = res.mass;
                ft.r = 0.0f;
                ft.max_i = res.max;
                ft.count = res.count;
                ft.Rg = ft.raw = ft.signal = ft.ecc = 0.0f;
                ft.d_raw = ft.d_bg = ft.d_corr = __int_as_float(0x7fc00000);
                ft.ridx = 0;
                if (c.characterize) {
                    const float2* ang = angles + angle_off[RI];
                    const float* pc = my + (cu - cen_u + OFF) * PS + (cv - cen_v + OFF);
                    float middle = 0.0f;
                    const int64_t middle_idx = (int64_t)cu * W + cv;
                    if (middle_idx >= 0 && middle_idx < (int64_t)H * W) {
                        if (cu >= 0 && cu < H && cv >= 0 && cv < W) middle = *pc;
                        else middle = lw_processed_at<T>(img, c, (int)(middle_idx / W), (int)(middle_idx % W));
                    }
                    float Rg, raw_mass, signal, es, ec;
                    if (cu >= RI && cu + RI < H && cv >= RI && cv + RI < W)
                        lw_characterize<T, RI, false>(pc, PS, img, H, W, cu, cv, ang, &Rg, &raw_mass, &signal, &es,
                                                      &ec);
                    else
                        lw_characterize<T, RI, true>(pc, PS, img, H, W, cu, cv, ang, &Rg, &raw_mass, &signal, &es,
                                                     &ec);
                    es = __fmul_rn(es, es);
                    ec = __fmul_rn(ec, ec);
                    ft.ecc = __fdiv_rn(__fsqrt_rn(__fadd_rn(es, ec)), __fsub_rn(ft.mass, middle));
                    ft.Rg = __fsqrt_rn(__fdiv_rn(Rg, ft.mass));
                    ft.raw = raw_mass;
                    ft.signal = signal;
                }
                const uint32_t pos = atomicAdd(feat_count + f, 1u);
                if (pos < feat_cap) feats[(size_t)f * feat_cap + pos] = ft;
                else atomicOr(flags, kFlagFeatOverflow);
                stage = 2;
            }
        }
    }
    if (stage != 2) atomicOr(flags, kFlagLocalWalk);
}

// characterize_points: characterize.wgsl with _feat_characterize_points (mass
// recomputed at the rounded position); one thread per given point.
template <typename T>
__global__ void __launch_bounds__(128)
characterize_points_kernel(const float* __restrict__ processed, const T* __restrict__ frames, int64_t frame_stride,
                           const LocateConsts c, const float* __restrict__ pts, const int64_t* __restrict__ grp_off,
                           const int32_t* __restrict__ grp_frame, const float2* __restrict__ angle_tab,
                           const int32_t* __restrict__ angle_off, const float* __restrict__ radii_tab,
                           int32_t n_radii_tab, int32_t has_r, Feature* __restrict__ feats, uint32_t* feat_count,
                           uint32_t feat_cap, int32_t g0) {
    const int g = blockIdx.y;  // group within this chunk
    const int64_t a = grp_off[g0 + g], b = grp_off[g0 + g + 1];
    const int64_t i = a + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b) return;
    Feature ft;
    ft.key_hi = 0;
    ft.key_lo = (uint32_t)(i - a);
    ft.x = pts[3 * i + 0];
    ft.y = pts[3 * i + 1];
    ft.r = has_r ? pts[3 * i + 2] : 0.0f;
    ft.mass = 0.0f;
    ft.max_i = 0.0f;
    ft.count = 0.0f;
    ft.d_raw = ft.d_bg = ft.d_corr = __int_as_float(0x7fc00000);
    ft.ridx = 0;
    (void)radii_tab;
    (void)n_radii_tab;
    const float* p = processed + (size_t)g * c.H * c.W;
    const T* raw = frames + (size_t)grp_frame[g0 + g] * frame_stride;
    characterize_one<T>(p, raw, c, ft, true, angle_tab, angle_off);
    uint32_t pos = (uint32_t)(i - a);
    if (pos < feat_cap) feats[(size_t)g * feat_cap + pos] = ft;
    if (threadIdx.x == 0 && blockIdx.x == 0) feat_count[g] = (uint32_t)((b - a) < (int64_t)feat_cap ? (b - a) : (int64_t)feat_cap);
}

// ------------------------------------------------------------------ finalize
// disk_overlap / blob_overlap of prune_blobs_log (src/execute_gpu.rs:599-628);
// Rust arithmetic, separately rounded.  acos is evaluated in double and
// rounded, the oracle does the same.
__device__ float make_acos(float d, float r1, float r1s, float r2s) {
    float num = __fsub_rn(__fadd_rn(__fmul_rn(d, d), r1s), r2s);
    float den = __fmul_rn(__fmul_rn(2.0f, d), r1);
    float ratio = __fdiv_rn(num, den);
    ratio = fminf(fmaxf(ratio, -1.0f), 1.0f);
    return (float)acos((double)ratio);
}
__device__ float disk_overlap(float d, float r1, float r2) {
    float r1s = __fmul_rn(r1, r1);
    float r2s = __fmul_rn(r2, r2);
    float acos1 = make_acos(d, r1, r1s, r2s);
    float acos2 = make_acos(d, r2, r2s, r1s);
    float a = __fadd_rn(__fadd_rn(-d, r2), r1);
    float b = __fadd_rn(__fsub_rn(d, r2), r1);
    float cc = __fsub_rn(__fadd_rn(d, r2), r1);
    float dd = __fadd_rn(__fadd_rn(d, r2), r1);
    float prod = __fmul_rn(__fmul_rn(__fmul_rn(a, b), cc), dd);
    float area = __fsub_rn(__fadd_rn(__fmul_rn(r1s, acos1), __fmul_rn(r2s, acos2)),
                           __fmul_rn(0.5f, __fsqrt_rn(fabsf(prod))));
    const float pi = 3.14159265358979323846f;
    return __fdiv_rn(area, __fmul_rn(pi, fminf(r1s, r2s)));
}
__device__ float blob_overlap(float r1, float r2, float distance) {
    if (distance > __fadd_rn(r1, r2)) return 0.0f;
    else if (distance <= fabsf(__fsub_rn(r1, r2))) return 1.0f;
    else return disk_overlap(distance, r1, r2);
}

// Upper median (sorted[len/2]) of the valid annulus pixels by a warp-wide
// radix select on order keys; exact.
template <typename T>
__device__ float warp_upper_median(const T* __restrict__ raw, int H, int W, int mu, int mv,
                                   const short2* __restrict__ inds, int n_inds, uint32_t* hist, int* n_out) {
    const int lane = threadIdx.x & 31;
    int nvalid = 0;
    for (int b = 0; b < n_inds; b += 32) {
        int k = b + lane;
        bool ok = false;
        if (k < n_inds) {
            short2 d = inds[k];
            int64_t a = (int64_t)mu + d.x, bb = (int64_t)mv + d.y;
            ok = (a >= 0 && a < H && bb >= 0 && bb < W);
        }
        nvalid += __popc(__ballot_sync(0xffffffffu, ok));
    }
    *n_out = nvalid;
    if (nvalid == 0) return 0.0f;
    uint32_t want = (uint32_t)(nvalid / 2);
    uint32_t prefix = 0, pmask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int q = lane; q < 256; q += 32) hist[q] = 0;
        __syncwarp();
        for (int b = lane; b < n_inds; b += 32) {
            short2 d = inds[b];
            int64_t a = (int64_t)mu + d.x, bb = (int64_t)mv + d.y;
            if (a >= 0 && a < H && bb >= 0 && bb < W) {
                uint32_t key = float_order_key(load_px<T>(raw, (size_t)a * W + bb));
                if ((key & pmask) == prefix) atomicAdd(hist + ((key >> shift) & 255u), 1u);
            }
        }
        __syncwarp();
        uint32_t local[8];
        uint32_t s = 0;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            local[q] = hist[lane * 8 + q];
            s += local[q];
        }
        uint32_t incl = s;
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
        }
        uint32_t excl = incl - s;
        int found_bin = -1;
        uint32_t below = 0;
        if (want >= excl && want < incl) {
            uint32_t acc = excl;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                if (found_bin < 0 && want < acc + local[q]) {
                    found_bin = lane * 8 + q;
                    below = acc;
                }
                acc += local[q];
            }
        }
        unsigned bal = __ballot_sync(0xffffffffu, found_bin >= 0);
        int src = __ffs(bal) - 1;
        found_bin = __shfl_sync(0xffffffffu, found_bin, src);
        below = __shfl_sync(0xffffffffu, below, src);
        want -= below;
        prefix |= ((uint32_t)found_bin) << shift;
        pmask |= 255u << shift;
        __syncwarp();
    }
    return float_from_order_key(prefix);
}

// Same upper median with the annulus held in registers (up to 32 *
// kMedianRegs pixels, loaded once): the key of rank len/2 is built bit by
// bit from the top, counting keys below each trial value with one warp
// reduction; bits that every valid key shares are taken as they are.
constexpr int kMedianRegs = 13;
// Median keys: the orderable bits of a float pixel, or an integer pixel's
// own value (the same order, in the fewest bits: the bit-by-bit search only
// visits the bits in which the annulus' values differ).
template <typename T>
struct MedKey {
    __device__ static uint32_t key(const T* raw, size_t i) { return float_order_key(load_px<T>(raw, i)); }
    __device__ static float value(uint32_t k) { return float_from_order_key(k); }
};
template <>
struct MedKey<uint16_t> {
    __device__ static uint32_t key(const uint16_t* raw, size_t i) { return (uint32_t)__ldg(raw + i); }
    __device__ static float value(uint32_t k) { return (float)k; }
};
template <>
struct MedKey<uint8_t> {
    __device__ static uint32_t key(const uint8_t* raw, size_t i) { return (uint32_t)__ldg(raw + i); }
    __device__ static float value(uint32_t k) { return (float)k; }
};

template <typename T>
__device__ __forceinline__ float warp_upper_median_regs(const T* __restrict__ raw, int H, int W, int mu, int mv,
                                        const short2* __restrict__ inds, int n_inds, int* n_out) {
    const int lane = threadIdx.x & 31;
    uint32_t key[kMedianRegs];
    int nv = 0;
    uint32_t kor = 0u, kand = 0xFFFFFFFFu;
#pragma unroll
    for (int q = 0; q < kMedianRegs; q++) {
        const int k = q * 32 + lane;
        key[q] = 0xFFFFFFFFu;  // never below a trial value: left out of every count
        if (k < n_inds) {
            const short2 d = inds[k];
            // 32-bit row / column tests (wrapping unsigned sums: a negative or
            // saturated centre fails them) and index (frames hold < 2^31 pixels)
            const uint32_t a = (uint32_t)mu + (uint32_t)(int32_t)d.x, b = (uint32_t)mv + (uint32_t)(int32_t)d.y;
            if (a < (uint32_t)H && b < (uint32_t)W) {
                key[q] = MedKey<T>::key(raw, a * (uint32_t)W + b);
                kor |= key[q];
                kand &= key[q];
                nv++;
            }
        }
    }
    int nvalid = nv;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nvalid += __shfl_xor_sync(0xffffffffu, nvalid, o);
    *n_out = nvalid;
    if (nvalid == 0) return 0.0f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        kor |= __shfl_xor_sync(0xffffffffu, kor, o);
        kand &= __shfl_xor_sync(0xffffffffu, kand, o);
    }
    const uint32_t diff = kor ^ kand;
    if (diff == 0u) return MedKey<T>::value(kand);
    const uint32_t want = (uint32_t)(nvalid / 2);
    const int hb = 31 - __clz(diff), lb = __ffs(diff) - 1;
    uint32_t prefix = kand & ~((2u << hb) - 1u);      // bits above hb: common to all keys
    if (hb == 31) prefix = 0u;
    for (int bit = hb; bit >= lb; bit--) {
        const uint32_t trial = prefix | (1u << bit);
        int c = 0;
#pragma unroll
        for (int q = 0; q < kMedianRegs; q++) c += (key[q] < trial) ? 1 : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if ((uint32_t)c <= want) prefix = trial;
    }
    prefix |= kand & ((1u << lb) - 1u);                 // bits below lb: common to all keys
    return MedKey<T>::value(prefix);
}

// Doughnut correction of one feature by one warp (src/execute_gpu.rs:717-790).
template <typename T>
__device__ __forceinline__ void doughnut_warp(const T* __restrict__ raw, int H, int W, Feature& ft, const short2* __restrict__ sig,
                              int n_sig, const short2* __restrict__ bg, int n_bg, uint32_t* hist) {
    const int lane = threadIdx.x & 31;
    const int mu = sat_f2i(roundf(ft.x));
    const int mv = sat_f2i(roundf(ft.y));
    // sequential sum in circle_inds order (Iterator::sum); integer pixels
    // make every partial sum an exact integer below 2^24, so a warp
    // reduction gives the same value
    float sum = 0.0f;
    int nsig = 0;
    if (!std::is_same<T, float>::value && n_sig <= 256) {
        uint32_t acc = 0;
        for (int b = 0; b < n_sig; b += 32) {
            const int k = b + lane;
            bool ok = false;
            if (k < n_sig) {
                const short2 d = sig[k];
                const uint32_t a = (uint32_t)mu + (uint32_t)(int32_t)d.x;
                const uint32_t bb = (uint32_t)mv + (uint32_t)(int32_t)d.y;
                ok = a < (uint32_t)H && bb < (uint32_t)W;
                if (ok) acc += (uint32_t)load_px<T>(raw, a * (uint32_t)W + bb);
            }
            nsig += __popc(__ballot_sync(0xffffffffu, ok));
        }
        sum = (float)__reduce_add_sync(0xffffffffu, acc);
    } else
    for (int b = 0; b < n_sig; b += 32) {
        int k = b + lane;
        float val = 0.0f;
        bool ok = false;
        if (k < n_sig) {
            short2 d = sig[k];
            int64_t a = (int64_t)mu + d.x, bb = (int64_t)mv + d.y;
            ok = (a >= 0 && a < H && bb >= 0 && bb < W);
            if (ok) val = load_px<T>(raw, (size_t)a * W + bb);
        }
        unsigned bal = __ballot_sync(0xffffffffu, ok);
        nsig += __popc(bal);
        for (int q = 0; q < 32; q++) {
            float v = __shfl_sync(0xffffffffu, val, q);
            if ((bal >> q) & 1u) sum = __fadd_rn(sum, v);
        }
    }
    int nbg;
    const float med = (n_bg <= 32 * kMedianRegs) ? warp_upper_median_regs<T>(raw, H, W, mu, mv, bg, n_bg, &nbg)
                                                  : warp_upper_median<T>(raw, H, W, mu, mv, bg, n_bg, hist, &nbg);
    ft.d_raw = sum;
    ft.d_bg = med;
    ft.d_corr = __fsub_rn(sum, __fmul_rn(med, (float)nsig));
}

// Shared memory of finalize: sort keys, permutation, order, keep flags and
// a histogram, then the filter_close positions and masses of up to
// kFinalizeFcSmem detections.
constexpr int kFinalizeFcSmem = 4096;
__host__ __device__ constexpr size_t finalize_smem_core_bytes() {
    return (size_t)kFinalizeSmemSort * (8 + 4 + 4 + 1) + 32 * 256 * sizeof(uint32_t);
}

// One CTA per frame: canonical order, filter_close / prune_blobs_log, the
// doughnut correction and compaction of the kept rows in output order.
template <typename T>
__global__ void __launch_bounds__(kFinalizeThreads)
finalize_kernel(const Feature* __restrict__ feats, const uint32_t* __restrict__ feat_count, uint32_t feat_cap,
                Feature* __restrict__ out, uint32_t* __restrict__ kept_count, uint8_t* __restrict__ gscratch,
                const FinalizeConsts fc, const T* __restrict__ frames, int64_t frame_stride,
                const int32_t* __restrict__ frame_index, const short2* __restrict__ dn_inds,
                const int4* __restrict__ dn_meta, uint32_t* __restrict__ flags, const RaggedFrame* __restrict__ rf) {
    extern __shared__ uint64_t fsm[];
    __shared__ int wsum[33];
    const int g = blockIdx.x;
    const int fW = rf ? rf[g].W : fc.W;
    const int og = rf ? rf[g].out_slot : g;   // result slot (ragged batches: the frame's slot of the call)
    const int n = (int)min(feat_count[g], feat_cap);
    const Feature* F = feats + (size_t)g * feat_cap;
    int np2 = 1;
    while (np2 < n) np2 <<= 1;
    // working arrays: keys (u64), perm (i32), order (i32), keep (u8)
    uint64_t* keys;
    int32_t *perm, *order;
    uint8_t* keep;
    uint32_t* hist;
    const size_t need = (size_t)np2 * (8 + 4 + 4 + 1);
    if (np2 <= kFinalizeSmemSort) {
        keys = fsm;
        perm = (int32_t*)(keys + kFinalizeSmemSort);
        order = perm + kFinalizeSmemSort;
        keep = (uint8_t*)(order + kFinalizeSmemSort);
        hist = (uint32_t*)(keep + kFinalizeSmemSort);
    } else {
        if (need > fc.scratch_per_frame) {
            if (threadIdx.x == 0) atomicOr(flags, kFlagFeatOverflow);
            if (threadIdx.x == 0) kept_count[og] = 0;
            return;
        }
        uint8_t* base = gscratch + (size_t)g * fc.scratch_per_frame;
        keys = (uint64_t*)base;
        perm = (int32_t*)(keys + np2);
        order = perm + np2;
        keep = (uint8_t*)(order + np2);
        uint8_t* sm_after = (uint8_t*)fsm;
        hist = (uint32_t*)sm_after;
    }
    // 1. canonical order: (radius index, candidate pixel index), or input order
    for (int i = threadIdx.x; i < np2; i += blockDim.x) {
        if (i < n) {
            const Feature& ft = F[i];
            keys[i] = fc.presorted ? (uint64_t)i
                                   : (((uint64_t)ft.key_hi << 56) | ((uint64_t)ft.key_lo << 24) | (uint64_t)i);
        } else {
            keys[i] = ~0ull;
        }
    }
    __syncthreads();
    if (!fc.presorted) block_sort_u64(keys, np2);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        perm[i] = (int32_t)(keys[i] & 0xFFFFFFull);
        keep[i] = 1;
        order[i] = i;
    }
    __syncthreads();

    if (!fc.log_style) {
        // 2a. filter_close_trackpy (src/execute_gpu.rs:556-590) in canonical order
        if (fc.filter_close) {
            // positions and masses in canonical order, in shared memory when
            // they fit: the neighbour scans then read no global memory
            const bool fc_smem = np2 <= kFinalizeSmemSort && n <= kFinalizeFcSmem;
            float* const fcx = (float*)((uint8_t*)fsm + finalize_smem_core_bytes());
            float* const fcy = fcx + kFinalizeFcSmem;
            float* const fcm = fcy + kFinalizeFcSmem;
            if (fc_smem) {
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    const Feature& ft = F[perm[i]];
                    fcx[i] = ft.x;
                    fcy[i] = ft.y;
                    fcm[i] = ft.mass;
                }
                __syncthreads();
            }
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const Feature& q = F[perm[i]];
                int lo = 0, hi = n;
                if (fc.band >= 0) {
                    // rows of candidates that can hold a neighbour (|x - u| <= reach)
                    int64_t u = (int64_t)q.key_lo / fW;
                    int64_t ulo = u - fc.band, uhi = u + fc.band + 1;
                    uint64_t klo = ulo <= 0 ? 0ull : ((uint64_t)(ulo * fW) << 24);
                    uint64_t khi = ((uint64_t)(uhi * fW) << 24);
                    int a = 0, b = n;
                    while (a < b) { int m = (a + b) >> 1; if (keys[m] < klo) a = m + 1; else b = m; }
                    lo = a;
                    a = lo; b = n;
                    while (a < b) { int m = (a + b) >> 1; if (keys[m] < khi) a = m + 1; else b = m; }
                    hi = a;
                }
                bool kp = true;
                if (fc_smem) {
                    const float qx = fcx[i], qy = fcy[i], qm = fcm[i];
                    for (int j = lo; j < hi && kp; j++) {
                        if (j == i) continue;
                        float dist;
                        if (!within_rd2(fcx[j], fcy[j], qx, qy, fc.separation, &dist)) continue;
                        if (qm < fcm[j]) kp = false;
                        else if (qm == fcm[j] && i > j) kp = false;
                    }
                } else {
                    for (int j = lo; j < hi && kp; j++) {
                        if (j == i) continue;
                        const Feature& nb = F[perm[j]];
                        float dist;
                        if (!within_rd2(nb.x, nb.y, q.x, q.y, fc.separation, &dist)) continue;
                        if (q.mass < nb.mass) kp = false;
                        else if (q.mass == nb.mass && i > j) kp = false;
                    }
                }
                keep[i] = kp ? 1 : 0;
            }
            __syncthreads();
        }
    } else if (fc.prune) {
        // 2b. sort by (r desc, mass desc), stable w.r.t. the canonical order
        for (int i = threadIdx.x; i < np2; i += blockDim.x) {
            if (i < n) {
                const Feature& ft = F[perm[i]];
                uint64_t rk = (uint64_t)fc.radius_rank_desc[ft.ridx];
                uint64_t mk = (uint64_t)(~float_order_key(ft.mass));
                keys[i] = (rk << 56) | (mk << 24) | (uint64_t)i;
            } else {
                keys[i] = ~0ull;
            }
        }
        __syncthreads();
        block_sort_u64(keys, np2);
        for (int i = threadIdx.x; i < n; i += blockDim.x) order[i] = (int32_t)(keys[i] & 0xFFFFFFull);
        __syncthreads();
        // prune_blobs_log (src/execute_gpu.rs:592-669): greedy in priority
        // order, one step per kept blob.  Positions and radii in priority
        // order sit in shared memory when they fit, so a step's scan reads no
        // global memory.
        const bool pr_smem = np2 <= kFinalizeSmemSort && n <= kFinalizeFcSmem;
        if (pr_smem) {
            float* const bx = (float*)((uint8_t*)fsm + finalize_smem_core_bytes());
            float* const by = bx + kFinalizeFcSmem;
            float* const br = by + kFinalizeFcSmem;
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const Feature& ft = F[perm[order[i]]];
                bx[i] = ft.x;
                by[i] = ft.y;
                br[i] = ft.r;
            }
            __syncthreads();
            for (int q = 0; q < n; q++) {
                if (!keep[q]) continue;  // uniform: keep[] only changes between barriers
                const float Qx = bx[q], Qy = by[q], Qr = br[q];
                const float qr = __fmul_rn(Qr, 2.0f);
                for (int j = threadIdx.x; j < n; j += blockDim.x) {
                    if (j == q || !keep[j]) continue;
                    float d2;
                    if (!within_rd2(bx[j], by[j], Qx, Qy, qr, &d2)) continue;
                    float ov = blob_overlap(Qr, br[j], __fsqrt_rn(d2));
                    if (ov > fc.overlap_threshold) keep[j] = 0;
                }
                __syncthreads();
            }
        } else {
            for (int q = 0; q < n; q++) {
                if (!keep[q]) continue;  // uniform: keep[] only changes between barriers
                const Feature& Q = F[perm[order[q]]];
                const float qr = __fmul_rn(Q.r, 2.0f);
                for (int j = threadIdx.x; j < n; j += blockDim.x) {
                    if (j == q || !keep[j]) continue;
                    const Feature& Nb = F[perm[order[j]]];
                    float d2;
                    if (!within_rd2(Nb.x, Nb.y, Q.x, Q.y, qr, &d2)) continue;
                    float ov = blob_overlap(Q.r, Nb.r, __fsqrt_rn(d2));
                    if (ov > fc.overlap_threshold) keep[j] = 0;
                }
                __syncthreads();
            }
        }
    }

    // 3. doughnut correction of the kept rows, one warp per row
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // 4. compaction in output order
    int total = 0;
    for (int base = 0; base < n; base += blockDim.x) {
        int i = base + threadIdx.x;
        int k = (i < n) ? keep[i] : 0;
        int tot;
        int pos = block_excl_scan(k, &tot, wsum);
        if (k) {
            Feature ft = F[perm[order[i]]];
            out[(size_t)og * feat_cap + total + pos] = ft;
        }
        total += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) kept_count[og] = (uint32_t)total;
}

// Doughnut correction of the kept rows (src/execute_gpu.rs:717-790): one warp
// per row, kDoughnutBlocks x 8 warps per frame walking the frame's rows, so the
// per-row latency (gathers, median bits) overlaps across the whole GPU.
constexpr int kDoughnutWarps = 8;
constexpr int kDoughnutBlocks = 16;
template <typename T>
__global__ void __launch_bounds__(32 * kDoughnutWarps)
doughnut_kernel(Feature* __restrict__ out, const uint32_t* __restrict__ kept_count, uint32_t feat_cap,
                const FinalizeConsts fc, const T* __restrict__ frames, int64_t frame_stride,
                const int32_t* __restrict__ frame_index, const short2* __restrict__ dn_inds,
                const int4* __restrict__ dn_meta, const RaggedFrame* __restrict__ rf) {
    __shared__ uint32_t hist[kDoughnutWarps * 256];
    const int g = blockIdx.y;
    const int og = rf ? rf[g].out_slot : g;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int total = (int)kept_count[og];
    const T* raw = rf ? (const T*)rf[g].raw : frames + (size_t)frame_index[g] * frame_stride;
    const int H = rf ? rf[g].H : fc.H, W = rf ? rf[g].W : fc.W;
    uint32_t* myhist = hist + wid * 256;
    for (int q = blockIdx.x * kDoughnutWarps + wid; q < total; q += gridDim.x * kDoughnutWarps) {
        Feature* o = out + (size_t)og * feat_cap + q;
        Feature ft = *o;
        const int4 m = dn_meta[fc.log_style ? ft.ridx : 0];
        doughnut_warp<T>(raw, H, W, ft, dn_inds + m.x, m.y, dn_inds + m.z, m.w, myhist);
        if (lane == 0) {
            o->d_raw = ft.d_raw;
            o->d_bg = ft.d_bg;
            o->d_corr = ft.d_corr;
        }
        __syncwarp();
    }
}

// Per-frame rows -> table columns at the frame's row offset.
__global__ void scatter_kernel(const Feature* __restrict__ feats, uint32_t feat_cap,
                               const uint32_t* __restrict__ kept_count, const int64_t* __restrict__ row_off,
                               const int64_t* __restrict__ frame_number, TableCols tab, int32_t g0) {
    const int g = blockIdx.y;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kept_count[g]) return;
    const Feature& ft = feats[(size_t)g * feat_cap + k];
    const int64_t row = row_off[g0 + g] + k;
    tab.frame[row] = frame_number[g0 + g];
    tab.col[GT_COL_Y][row] = ft.x;
    tab.col[GT_COL_X][row] = ft.y;
    tab.col[GT_COL_MASS][row] = ft.mass;
    tab.col[GT_COL_R][row] = ft.r;
    tab.col[GT_COL_RG][row] = ft.Rg;
    tab.col[GT_COL_RAW][row] = ft.raw;
    tab.col[GT_COL_SIGNAL][row] = ft.signal;
    tab.col[GT_COL_ECC][row] = ft.ecc;
    tab.col[GT_COL_RAW_MASS][row] = ft.d_raw;
    tab.col[GT_COL_RAW_BG_MEDIAN][row] = ft.d_bg;
    tab.col[GT_COL_RAW_MASS_CORRECTED][row] = ft.d_corr;
    tab.col[GT_COL_MAX_INTENSITY][row] = ft.max_i;
    tab.col[GT_COL_COUNT][row] = ft.count;
}

// ------------------------------------------------------------ launch helpers
size_t bandpass_smem_bytes(int R, int kd, bool cand) {
    const int k = cand ? kd : 1;
    const int PH = kLocateTH + k - 1, PW = kLocateTW + k - 1;
    const int XH = PH + 2 * R, RW = PW + 2 * R;
    size_t fl = (size_t)XH * RW + 2 * (size_t)XH * PW + (size_t)PH * PW + (cand ? (size_t)kLocateTH * PW : 0);
    return fl * sizeof(float);
}

size_t finalize_smem_bytes() { return finalize_smem_core_bytes() + (size_t)kFinalizeFcSmem * 3 * sizeof(float); }

template <typename T>
cudaError_t launch_bandpass(const T* frames, int64_t frame_stride, float* processed, const LocateConsts& c,
                            int nframes, bool cand, uint32_t* cand_count, uint32_t* cand_keys, uint32_t cand_cap,
                            uint32_t* flags, cudaStream_t st) {
    dim3 grid((c.W + kLocateTW - 1) / kLocateTW, (c.H + kLocateTH - 1) / kLocateTH, nframes);
    size_t smem = bandpass_smem_bytes(c.R, c.kd, cand);
    if (cand) {
        cudaError_t e = cudaSuccess;
        if (launch_strip<T>(frames, frame_stride, processed, c, nframes, cand_count, cand_keys, cand_cap, flags, st,
                            &e))
            return e;
        cudaFuncSetAttribute(bandpass_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        bandpass_kernel<T, true><<<grid, kLocateThreads, smem, st>>>(frames, frame_stride, processed, c, cand_count,
                                                                    cand_keys, cand_cap, flags);
    } else {
        cudaFuncSetAttribute(bandpass_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        bandpass_kernel<T, false><<<grid, kLocateThreads, smem, st>>>(frames, frame_stride, processed, c, cand_count,
                                                                     cand_keys, cand_cap, flags);
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_walk(const float* processed, const T* frames, int64_t frame_stride, const LocateConsts& c,
                        int nframes, int n_slots, const uint32_t* cand_count, const uint32_t* cand_keys,
                        uint32_t cand_cap, uint32_t max_cands, const float* radii, const int32_t* angle_off,
                        const float2* angles, Feature* feats, uint32_t* feat_count, uint32_t feat_cap,
                        uint32_t* flags, cudaStream_t st, const RaggedFrame* rf) {
    if (max_cands == 0) return cudaSuccess;
    dim3 grid((max_cands + 127) / 128, nframes, n_slots);
    if (rf && (radii || n_slots != 1)) return cudaErrorInvalidValue;   // ragged batches: trackpy style only
    if (!radii && n_slots == 1) {
        const int ri = (c.circle - 1) / 2;
#define GT_WALK_FIXED(RI)                                                                                          \
    if (ri == RI) {                                                                                                \
        walk_kernel_fixed<T, RI><<<grid, 128, 0, st>>>(processed, frames, frame_stride, c, cand_count, cand_keys,  \
                                                       cand_cap, angle_off, angles, feats, feat_count, feat_cap,   \
                                                       flags, rf);                                                 \
        return cudaGetLastError();                                                                                 \
    }
        GT_WALK_FIXED(2) GT_WALK_FIXED(3) GT_WALK_FIXED(4) GT_WALK_FIXED(5) GT_WALK_FIXED(6) GT_WALK_FIXED(7)
#undef GT_WALK_FIXED
    }
    walk_kernel<T><<<grid, 128, 0, st>>>(processed, frames, frame_stride, c, cand_count, cand_keys, cand_cap, radii,
                                         angle_off, angles, feats, feat_count, feat_cap, flags, n_slots);
    return cudaGetLastError();
}

size_t walk_local_smem_bytes(int circle, int R) {
    const int ri = (circle - 1) / 2;
    return (size_t)kLwWarps * lw_warp_floats(ri, R) * sizeof(float);
}

template <typename T>
cudaError_t launch_walk_local(const T* frames, int64_t frame_stride, const LocateConsts& c, int nframes,
                              const uint32_t* cand_count, const uint32_t* cand_keys, uint32_t cand_cap,
                              const int32_t* angle_off, const float2* angles, Feature* feats, uint32_t* feat_count,
                              uint32_t feat_cap, uint32_t* flags, cudaStream_t st) {
    if (cand_cap == 0 || nframes == 0) return cudaSuccess;
    const int ri = (c.circle - 1) / 2;
    const size_t smem = walk_local_smem_bytes(c.circle, c.R);
    dim3 grid((cand_cap + kLwSeeds * kLwWarps - 1) / (kLwSeeds * kLwWarps), nframes);
    // the smoothing radius unrolled where it is the circle radius or one more
    // (smoothing_size = diameter, its default), looped otherwise
#define GT_WALK_LOCAL_RC(RI, RC)                                                                                     \
    {                                                                                                                \
        cudaFuncSetAttribute(walk_local_kernel<T, RI, RC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
        walk_local_kernel<T, RI, RC><<<grid, 32 * kLwWarps, smem, st>>>(frames, frame_stride, c, cand_count,         \
                                                                        cand_keys, cand_cap, angle_off, angles,      \
                                                                        feats, feat_count, feat_cap, flags);          \
        return cudaGetLastError();                                                                                   \
    }
#define GT_WALK_LOCAL(RI)                                \
    if (ri == RI) {                                      \
        if (c.R == RI) GT_WALK_LOCAL_RC(RI, RI)          \
        if (c.R == RI + 1) GT_WALK_LOCAL_RC(RI, RI + 1)  \
        GT_WALK_LOCAL_RC(RI, 0)                          \
    }
    GT_WALK_LOCAL(2) GT_WALK_LOCAL(3) GT_WALK_LOCAL(4) GT_WALK_LOCAL(5) GT_WALK_LOCAL(6) GT_WALK_LOCAL(7)
#undef GT_WALK_LOCAL
#undef GT_WALK_LOCAL_RC
    return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t launch_characterize_points(const float* processed, const T* frames, int64_t frame_stride,
                                       const LocateConsts& c, const float* pts, const int64_t* grp_off,
                                       const int32_t* grp_frame, int32_t g0, int ngroups, int64_t max_pts,
                                       const float2* angles, const int32_t* angle_off, int32_t n_angle_tabs,
                                       int32_t has_r, Feature* feats, uint32_t* feat_count, uint32_t feat_cap,
                                       cudaStream_t st) {
    if (max_pts <= 0) return cudaSuccess;
    dim3 grid((unsigned)((max_pts + 127) / 128), ngroups);
    characterize_points_kernel<T><<<grid, 128, 0, st>>>(processed, frames, frame_stride, c, pts, grp_off, grp_frame,
                                                        angles, angle_off, nullptr, n_angle_tabs, has_r, feats,
                                                        feat_count, feat_cap, g0);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_finalize(const Feature* feats, const uint32_t* feat_count, uint32_t feat_cap, Feature* out,
                            uint32_t* kept_count, uint8_t* gscratch, const FinalizeConsts& fc, const T* frames,
                            int64_t frame_stride, const int32_t* frame_index, const short2* dn_inds,
                            const int4* dn_meta, uint32_t* flags, int ngroups, cudaStream_t st,
                            const RaggedFrame* rf) {
    size_t smem = finalize_smem_bytes();
    cudaFuncSetAttribute(finalize_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    finalize_kernel<T><<<ngroups, kFinalizeThreads, smem, st>>>(feats, feat_count, feat_cap, out, kept_count,
                                                                gscratch, fc, frames, frame_stride, frame_index,
                                                                dn_inds, dn_meta, flags, rf);
    if (fc.doughnut && ngroups > 0) {
        dim3 grid(kDoughnutBlocks, ngroups);
        doughnut_kernel<T><<<grid, 32 * kDoughnutWarps, 0, st>>>(out, kept_count, feat_cap, fc, frames,
                                                                  frame_stride, frame_index, dn_inds, dn_meta, rf);
    }
    return cudaGetLastError();
}

cudaError_t launch_scatter(const Feature* feats, uint32_t feat_cap, const uint32_t* kept_count,
                           uint32_t max_kept, const int64_t* row_off, const int64_t* frame_number,
                           const TableCols& tab, int32_t g0, int ngroups, cudaStream_t st) {
    if (max_kept == 0) return cudaSuccess;
    dim3 grid((max_kept + 255) / 256, ngroups);
    scatter_kernel<<<grid, 256, 0, st>>>(feats, feat_cap, kept_count, row_off, frame_number, tab, g0);
    return cudaGetLastError();
}

#define GT_INSTANTIATE(T)                                                                                       \
    template cudaError_t launch_bandpass<T>(const T*, int64_t, float*, const LocateConsts&, int, bool, uint32_t*, \
                                            uint32_t*, uint32_t, uint32_t*, cudaStream_t);                        \
    template cudaError_t launch_walk<T>(const float*, const T*, int64_t, const LocateConsts&, int, int,          \
                                        const uint32_t*, const uint32_t*, uint32_t, uint32_t, const float*,      \
                                        const int32_t*, const float2*, Feature*, uint32_t*, uint32_t, uint32_t*, \
                                        cudaStream_t, const RaggedFrame*);                                       \
    template cudaError_t launch_walk_local<T>(const T*, int64_t, const LocateConsts&, int, const uint32_t*,     \
                                              const uint32_t*, uint32_t, const int32_t*, const float2*, Feature*, \
                                              uint32_t*, uint32_t, uint32_t*, cudaStream_t);                     \
    template cudaError_t launch_characterize_points<T>(const float*, const T*, int64_t, const LocateConsts&,     \
                                                       const float*, const int64_t*, const int32_t*, int32_t,     \
                                                       int, int64_t, const float2*, const int32_t*, int32_t,      \
                                                       int32_t, Feature*, uint32_t*, uint32_t, cudaStream_t);     \
    template cudaError_t launch_finalize<T>(const Feature*, const uint32_t*, uint32_t, Feature*, uint32_t*,      \
                                            uint8_t*, const FinalizeConsts&, const T*, int64_t, const int32_t*,  \
                                            const short2*, const int4*, uint32_t*, int, cudaStream_t,            \
                                            const RaggedFrame*);

GT_INSTANTIATE(uint16_t)
GT_INSTANTIATE(float)
GT_INSTANTIATE(uint8_t)

}  // namespace gt
