// gt_api.cu — the C ABI (include/gpu_tracking_b200.h): context, the locate
// runtime and the batch calls.  The linking calls are in gt_linkdrv.cu, the
// result tables in gt_table.cu; the internals they share (context, buffers,
// error handling, profiling) in gt_runtime.cuh.
//
// The runtime replaces execute_gpu / submit_work / get_work / post_process
// (src/execute_gpu.rs:95-467, 671-1184) and setup_state (src/gpu_setup.rs:611-1292):
//   * frames are processed in chunks on one compute stream; host frames are
//     staged through two device buffers filled on a copy stream, so the H2D
//     copy of chunk c+1 overlaps the kernels of chunk c;
//   * every per-frame result stays in HBM until the whole video is done
//     (filter, doughnut and linking included), then one table is assembled
//     on the device;
//   * capacities (candidates / detections per frame) grow and the call is
//     replayed when a kernel reports an overflow, so nothing is truncated.
#include <cuda.h>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "gt_kernels.h"
#include "gt_proposal.h"
#include "gt_runtime.cuh"

using namespace gt;
using namespace gt::rt;

namespace {

// ------------------------------------------------------- derived parameters
struct Derived {
    int32_t smoothing, circle, dilation, margin;
};

// gpuparams_from_tracking_params (src/gpu_setup.rs:528-580)
Derived derive(const gt_params& p) {
    Derived d;
    if (p.style == GT_STYLE_TRACKPY) {
        uint32_t smoothing = p.has_smoothing_size ? p.smoothing_size : p.diameter;
        float dil = 2.0f * (float)p.separation / std::sqrt(2.0f);
        uint32_t a = p.diameter / 2, b = p.separation / 2 - 1u, c = smoothing / 2;
        uint32_t m = std::max(a, std::max(b, c));
        d.smoothing = (int32_t)smoothing;
        d.circle = (int32_t)p.diameter;
        d.dilation = (int32_t)(uint32_t)dil;
        d.margin = (int32_t)m;
    } else {
        uint32_t smoothing = p.has_smoothing_size ? p.smoothing_size : ((uint32_t)(p.max_radius + 0.5f)) * 2 + 1;
        d.smoothing = (int32_t)smoothing;
        d.circle = 0;
        d.dilation = 0;
        d.margin = 0;
    }
    return d;
}

gt_status make_locate_consts(gt_ctx* ctx, const gt_params& p, int32_t H, int32_t W, LocateConsts& c) {
    Derived d = derive(p);
    std::memset(&c, 0, sizeof(c));
    c.H = H;
    c.W = W;
    c.R = d.smoothing / 2;
    if (2 * c.R + 1 > kMaxTaps)
        return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "smoothing_size %d exceeds the supported %d", d.smoothing,
                       kMaxTaps);
    // preprocess_rows.wgsl:46-47: exp(-x*x / (2.0 * sigma2)) with sigma2 = noise_size
    float gnorm = 0.0f;
    for (int i = -c.R; i <= c.R; i++) {
        float x = (float)i;
        float g = std::exp(-x * x / (2.0f * p.noise_size));
        c.taps[i + c.R] = g;
        gnorm += g;
    }
    c.gnorm = gnorm;
    c.kk = (float)(d.smoothing * d.smoothing);
    c.truncate = p.truncate_preprocessed ? 1 : 0;
    c.kd = d.dilation;
    c.o = (int32_t)((float)d.dilation / 2.0f - 0.5f);
    c.margin = d.margin;
    c.thr = 0.0f;  // pic_std (0 unless snr/minmass_snr) * snr * rough
    c.circle = d.circle;
    c.max_iter = p.max_iterations;
    c.shift_thr = p.shift_threshold;
    c.minmass = p.minmass;
    c.minmass_snr = p.has_minmass_snr ? p.minmass_snr : 0.0f;
    c.image_std = 0.0f;
    c.rough = p.has_adaptive_background ? 0.5f : 1.0f;
    c.snr = p.has_snr ? p.snr : 0.0f;
    c.frame_std = nullptr;  // set per call when the std pass runs
    c.characterize = p.characterize ? 1 : 0;
    {
        const int rint = std::max(0, (c.circle - 1) / 2);
        c.skip_zero = (p.style == GT_STYLE_TRACKPY && c.truncate && p.minmass > 0.0f && c.o >= rint &&
                       c.kd - 1 - c.o >= rint)
                          ? 1
                          : 0;
    }
    return GT_OK;
}

// Division by gnorm and kk in the strip kernel as fma(x, zh, x*zl), zh + zl
// the two-float reciprocal, when that is IEEE division for every dividend the
// pipeline can produce: integer pixels 0..65535 and positive taps bound the
// row-pass sums, the column-pass sums and the boxcar sums away from zero and
// infinity, and inside those bounds (x*zl and the quotient normal) the
// identity checked for every mantissa of [1, 2) holds at every exponent.
template <typename T>
void set_fast_div(gt_ctx* ctx, LocateConsts& c) {
    c.fast_div = 0;
    if (std::is_same<T, float>::value) return;
    auto split = [](float d, float* zh, float* zl) {
        const double r = 1.0 / (double)d;
        *zh = (float)r;
        *zl = (float)(r - (double)*zh);
    };
    split(c.gnorm, &c.zh_g, &c.zl_g);
    split(c.kk, &c.zh_k, &c.zl_k);
    double tmin = INFINITY, tsum = 0.0;
    for (int i = 0; i <= 2 * c.R; i++) {
        if (!(c.taps[i] > 0.0f)) return;
        tmin = std::min(tmin, (double)c.taps[i]);
        tsum += c.taps[i];
    }
    const double gn = c.gnorm, kk = c.kk;
    const double row_lo = tmin, row_hi = 65535.0 * tsum;
    const double col_lo = tmin * (row_lo / gn), col_hi = tsum * (row_hi / gn);
    const double g_lo = 0.5 * std::min(row_lo, col_lo), g_hi = 2.0 * std::max(row_hi, col_hi);
    const double k_lo = 0.5, k_hi = 2.0 * 65535.0 * kk;
    auto safe = [](double lo, double hi, double d, double zh, double zl) {
        const double tiny = std::ldexp(1.0, -120), big = std::ldexp(1.0, 100);
        if (zl != 0.0 && lo * std::fabs(zl) < tiny) return false;
        if (lo / d < tiny || hi * zh > big || hi / d > big) return false;
        return true;
    };
    if (!safe(g_lo, g_hi, gn, c.zh_g, c.zl_g) || !safe(k_lo, k_hi, kk, c.zh_k, c.zl_k)) return;
    if (!const_div_proven(c.gnorm, c.zh_g, c.zl_g, ctx->st) || !const_div_proven(c.kk, c.zh_k, c.zl_k, ctx->st))
        return;
    c.fast_div = 1;
}

// (sin 2θ, cos 2θ) tables per integer radius 0..max_rint (characterize.wgsl:120-124)
void angle_tables(int max_rint, std::vector<float2>& tab, std::vector<int32_t>& off) {
    tab.clear();
    off.clear();
    for (int r = 0; r <= max_rint; r++) {
        off.push_back((int32_t)tab.size());
        for (int i = -r; i <= r; i++)
            for (int j = -r; j <= r; j++) {
                float x = (float)i, y = (float)j;
                float2 v = make_float2(0.0f, 0.0f);
                if (i != 0 || j != 0) {
                    float theta = std::atan2(y, x);
                    v = make_float2(std::sin(2.0f * theta), std::cos(2.0f * theta));
                }
                tab.push_back(v);
            }
    }
}

// circle_inds / annulus_inds (src/kernels.rs:138-171)
void circle_inds(float radius, std::vector<short2>& v) {
    int rb = (int)std::ceil(radius);
    float r2 = radius * radius;
    for (int i = -rb; i < rb + 1; i++)
        for (int j = -rb; j < rb + 1; j++)
            if ((float)(i * i + j * j) <= r2) v.push_back(make_short2((short)i, (short)j));
}
void annulus_inds(float outer, float inner, std::vector<short2>& v) {
    int b = (int)std::ceil(outer);
    float or2 = outer * outer, ir2 = inner * inner;
    for (int i = -b; i < b + 1; i++)
        for (int j = -b; j < b + 1; j++) {
            float r2 = (float)(i * i + j * j);
            if (r2 <= or2 && r2 >= ir2) v.push_back(make_short2((short)i, (short)j));
        }
}

// Doughnut tables for the given particle radii (one entry per radius index).
void doughnut_tables(const gt_params& p, const std::vector<float>& radii, std::vector<short2>& inds,
                     std::vector<int4>& meta) {
    inds.clear();
    meta.clear();
    for (float radius : radii) {
        int4 m;
        m.x = (int)inds.size();
        circle_inds(radius, inds);
        m.y = (int)inds.size() - m.x;
        float outer = p.has_bg_radius ? p.bg_radius : 2.0f * radius;
        float gap = (p.has_bg_radius && p.has_gap_radius) ? p.gap_radius : 0.0f;
        m.z = (int)inds.size();
        annulus_inds(outer, gap + radius, inds);
        m.w = (int)inds.size() - m.z;
        meta.push_back(m);
    }
}

// LoG radii (src/gpu_setup.rs:958-984)
std::vector<float> log_radii(const gt_params& p) {
    std::vector<float> out;
    size_t n = p.n_radii;
    if (n == 0) return out;
    if (p.log_spacing) {
        float start = std::log(p.min_radius) / std::log(10.0f);
        float end = std::log(p.max_radius) / std::log(10.0f);
        float diff = (end - start) / (float)(n - 1);
        for (size_t i = 0; i + 1 < n; i++) {
            float temp = start;
            start += diff;
            out.push_back(std::pow(10.0f, temp));
        }
        out.push_back(std::pow(10.0f, start));
    } else {
        float start = p.min_radius;
        float end = p.max_radius;
        float diff = (end - start) / (float)(n - 1);
        for (size_t i = 0; i + 1 < n; i++) {
            float temp = start;
            start += diff;
            out.push_back(temp);
        }
        out.push_back(start);
    }
    return out;
}

struct LogTables {
    std::vector<float> radii, taps_g, taps_d, norm_g, norm_d;
    std::vector<int32_t> tap_off, rints;
    int max_rint = 0;
    // the scale space runs as one fused kernel (gt_logss.cu) when its tiles
    // fit; otherwise as a plane per radius plus a maxima pass
    bool fused() const { return log_scale_space_supported(max_rint, (int)taps_g.size()); }
};

// separable_log.wgsl:27-76 tap values, computed per radius with sigma = r / sqrt(2)
LogTables log_tables(const gt_params& p) {
    LogTables t;
    t.radii = log_radii(p);
    const float sqrt2pi = (float)2.5066282746310002;
    for (float r : t.radii) {
        float sigma = r / std::sqrt(2.0f);
        float sigma2 = sigma * sigma;
        int rint = (int)(4.0f * sigma + 0.5f);
        t.tap_off.push_back((int32_t)t.taps_g.size());
        t.rints.push_back(rint);
        t.max_rint = std::max(t.max_rint, rint);
        for (int i = -rint; i <= rint; i++) {
            float x = (float)i;
            float x2 = x * x;
            float g = std::exp(-x2 / (2.0f * sigma2));
            t.taps_g.push_back(g);
            t.taps_d.push_back(g * (x2 - sigma2));
        }
        t.norm_d.push_back(1.0f / (sqrt2pi * sigma * sigma2));
        t.norm_g.push_back(1.0f / (sqrt2pi * sigma));
    }
    return t;
}

// ---------------------------------------------------------------- linking
// acc += sum of min(count[i], cap) over the chunk's frames (walk starts)
__global__ void sum_counts_kernel(const uint32_t* __restrict__ count, int n, uint32_t cap,
                                  unsigned long long* __restrict__ acc) {
    unsigned long long s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += min(count[i], cap);
    for (int d = 16; d; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(acc, s);
}

// Windowed linking inside gt_batch.  Every super-chunk of located frames is
// linked on the link stream while the next super-chunk is being located, so
// the linker's sequential frame loop runs beside the locate kernels instead
// of after them.  The detections are read in place from their per-frame
// slots (feats_out / kept_count, slot stride = feat_cap); each window builds
// the neighbour lists of its frames and of the memory+1 frames before it, and
// the linker's state (memory ring, stamps, id counter) carries over in its
// scratch from one window to the next, so ids and durations are those of the
// whole-video linker.  A window whose list or edge buffers are too small
// stops the video (kFlagListOverflow / kFlagEdgeOverflow); the call then
// links the finished table with the whole-video linker and the buffers grow
// for the next call.
struct PipeLink {
    gt_ctx* ctx = nullptr;
    LinkInput in;
    LinkScratch S;
    LinkOutput out;
    int K = 1;
    int64_t C = 0, list_cap = 0, max_items = 0;
    size_t scan_bytes = 0;
    int64_t nwin = 0;   // windows issued in this call
    float bin_w = 1.0f;  // row-bin width of the neighbour search index

    gt_status setup(gt_ctx* c, int64_t NT, uint32_t feat_cap, int SC, float radius, int memory,
                    const std::vector<uint8_t>& reset, int32_t H) {
        ctx = c;
        C = feat_cap;
        K = memory + 1;
        const int64_t NS = NT * C;
        max_items = (int64_t)(SC + K) * C * K + 1;
        if (ctx->w_list_cap <= 0) ctx->w_list_cap = std::max<int64_t>(max_items, 1 << 20);
        if (ctx->w_edge_cap <= 0) ctx->w_edge_cap = std::max<int64_t>(C * 16, 1 << 16);
        list_cap = ctx->w_list_cap;
        CK(ctx->w_srt.ensure(NS * 4));
        // row bins of at least the search radius over the frame height: a
        // neighbour search reads two bin offsets and scans about three bins
        CK(ctx->w_bins.ensure((size_t)NT * (kLinkRowBins + 1) * 4));
        bin_w = std::max(radius, (float)H / (float)kLinkRowBins);
        if (!(bin_w > 0.0f) || !std::isfinite(bin_w)) bin_w = 1.0f;
        // the previous call's list kernels may still read the buffers
        CK(cudaStreamSynchronize(ctx->ls));
        for (int b = 0; b < 2; b++) {
            CK(ctx->w_fcnt[b].ensure(max_items * 8));
            CK(ctx->w_bcnt[b].ensure(max_items * 8));
            CK(ctx->w_foff[b].ensure(max_items * 8));
            CK(ctx->w_boff[b].ensure(max_items * 8));
            CK(ctx->w_fpts[b].ensure(list_cap * 4));
            CK(ctx->w_bpts[b].ensure(list_cap * 4));
            CK(ctx->w_bdist[b].ensure(list_cap * 4));
        }
        nwin = 0;
        CK(ctx->w_ids.ensure(NS * 8));
        CK(ctx->w_dur.ensure(NS * 8));
        CK(ctx->w_state.ensure(sizeof(LinkState)));
        CK(ctx->w_cnt.ensure(8));
        CK(ctx->w_flags.ensure(4));
        CK(ctx->w_vgrp.ensure(8));
        CK(ctx->w_reset.ensure(std::max<int64_t>(NT, 1)));
        S.max_group = (int32_t)C;
        S.max_edges = ctx->w_edge_cap;
        S.max_points = NS;
        S.bytes_per_video = link_scratch_bytes(S.max_group, S.max_edges, NS, memory);
        CK(ctx->w_scratch.ensure(S.bytes_per_video));
        S.base = ctx->w_scratch.as<uint8_t>();
        scan_bytes = 0;
        CK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, ctx->w_fcnt[0].as<int64_t>(),
                                         ctx->w_foff[0].as<int64_t>(), max_items, ctx->ls));
        CK(ctx->w_scan.ensure(scan_bytes));

        const int32_t vg[2] = {0, (int32_t)NT};
        CK(cudaMemcpyAsync(ctx->w_vgrp.p, vg, sizeof(vg), cudaMemcpyHostToDevice, ctx->lk));
        CK(cudaMemcpyAsync(ctx->w_reset.p, reset.data(), NT, cudaMemcpyHostToDevice, ctx->lk));
        // the per-point linker arrays start cleared: stamps -1, first positions 0
        size_t o_id, o_src, o_first;
        link_scratch_point_arrays(S.max_group, S.max_edges, NS, memory, &o_id, &o_src, &o_first);
        CK(cudaMemsetAsync(S.base + o_id, 0xFF, NS * 4, ctx->lk));
        CK(cudaMemsetAsync(S.base + o_src, 0xFF, NS * 4, ctx->lk));
        CK(cudaMemsetAsync(S.base + o_first, 0, NS * 8, ctx->lk));
        CK(cudaMemsetAsync(ctx->w_flags.p, 0, 4, ctx->lk));
        CK(cudaMemsetAsync(ctx->w_cnt.p, 0, 8, ctx->lk));
        // the host buffers above are read before the call returns
        CK(sync_link_streams(ctx));

        in = LinkInput();
        const float* f = (const float*)ctx->feats_out.p;
        in.px = f + offsetof(Feature, x) / 4;
        in.py = f + offsetof(Feature, y) / 4;
        in.xy_stride = (int32_t)(sizeof(Feature) / 4);
        in.gcount = ctx->kept_count.as<uint32_t>();
        in.slot_stride = C;
        in.vgrp = ctx->w_vgrp.as<int32_t>();
        in.reset = ctx->w_reset.as<uint8_t>();
        in.ngroups = (int32_t)NT;
        in.nvideos = 1;
        in.npoints = NS;
        in.radius = radius;
        in.memory = memory;
        out.ids = ctx->w_ids.as<int64_t>();
        out.counter = ctx->w_cnt.as<int64_t>();
        out.dur = ctx->w_dur.as<int64_t>();
        out.vpoff = nullptr;
        out.flags = ctx->w_flags.as<uint32_t>();
        return GT_OK;
    }

    // frames [s0, s1) have been located on the compute stream.  The window's
    // sort and neighbour lists run on the lists stream into list set b (the
    // set window w - 2 used, once its linker is done with it), so they overlap
    // the linker of window w - 1; the linker of this window waits for them.
    gt_status window(int s0, int s1, bool first, bool last) {
        const int LA = std::max(0, s0 - K);
        const int64_t p0 = (int64_t)LA * C, p1 = (int64_t)s1 * C;
        const int64_t items = (p1 - p0) * K + 1;
        if (items > max_items) return set_err(ctx, GT_ERR_INTERNAL, "link window larger than its buffers");
        const int b = (int)(nwin & 1);
        CK(cudaEventRecord(ctx->located, ctx->st));
        CK(cudaStreamWaitEvent(ctx->ls, ctx->located, 0));
        if (nwin >= 2) CK(cudaStreamWaitEvent(ctx->ls, ctx->w_linked[b], 0));
        nwin++;
        in.groups_ready = s1;
        uint32_t* srt = ctx->w_srt.as<uint32_t>();
        {
            Prof pf(ctx, "link_sort", ctx->ls);
            CK(link_sort_groups_range(in, srt, s0, s1, ctx->w_bins.as<int32_t>(), bin_w, ctx->ls));
        }
        int64_t* fcnt = ctx->w_fcnt[b].as<int64_t>();
        int64_t* bcnt = ctx->w_bcnt[b].as<int64_t>();
        CK(cudaMemsetAsync(fcnt, 0, items * 8, ctx->ls));
        CK(cudaMemsetAsync(bcnt, 0, items * 8, ctx->ls));
        {
            Prof pf(ctx, "link_lists", ctx->ls);
            CK(link_count_lists_range(in, srt, p0, p1, fcnt, bcnt, out.flags, ctx->ls));
        }
        size_t tb = scan_bytes;
        CK(cub::DeviceScan::ExclusiveSum(ctx->w_scan.p, tb, fcnt, ctx->w_foff[b].as<int64_t>(), items, ctx->ls));
        CK(cub::DeviceScan::ExclusiveSum(ctx->w_scan.p, tb, bcnt, ctx->w_boff[b].as<int64_t>(), items, ctx->ls));
        LinkLists L;
        L.f_off = ctx->w_foff[b].as<int64_t>();
        L.b_off = ctx->w_boff[b].as<int64_t>();
        L.f_pts = ctx->w_fpts[b].as<int32_t>();
        L.b_pts = ctx->w_bpts[b].as<int32_t>();
        L.b_dist = ctx->w_bdist[b].as<float>();
        L.srt = srt;
        L.bins = ctx->w_bins.as<int32_t>();
        L.bin_w = bin_w;
        L.pbase = p0;
        L.f_cap = list_cap;
        L.b_cap = list_cap;
        {
            Prof pf(ctx, "link_lists", ctx->ls);
            CK(link_fill_lists_range(in, L, p1, out.flags, ctx->ls));
        }
        CK(cudaEventRecord(ctx->listed[b], ctx->ls));
        CK(cudaStreamWaitEvent(ctx->lk, ctx->listed[b], 0));
        LinkWindow w;
        w.g0 = s0;
        w.g1 = s1;
        w.first = first ? 1 : 0;
        w.last = last ? 1 : 0;
        w.init_points = 0;
        w.state = (LinkState*)ctx->w_state.p;
        {
            Prof pf(ctx, "link_video", ctx->lk);
            CK(link_run_window(in, L, S, out, w, ctx->lk));
        }
        CK(cudaEventRecord(ctx->w_linked[b], ctx->lk));
        return GT_OK;
    }
};

// --------------------------------------------------------------- locate
struct Chunking {
    int F;
};

int pick_chunk(int64_t T, int32_t H, int32_t W, int n_planes) {
    const size_t px = (size_t)H * W;
    size_t per_frame = px * 4 * (1 + n_planes);
    int F = (int)std::max<size_t>(1, (size_t)(1024u << 20) / per_frame);
    F = std::min<int>(F, 64);
    F = (int)std::min<int64_t>(F, T);
    return std::max(F, 1);
}

template <typename T>
__global__ void mean_accumulate_kernel(const T* __restrict__ frames, int nf, int64_t npix, float* __restrict__ acc) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    float a = acc[i];
    for (int t = 0; t < nf; t++) a = __fadd_rn(a, load_px<T>(frames, (size_t)t * npix + i));
    acc[i] = a;
}

__global__ void mean_divide_kernel(float* acc, int64_t npix, float n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < npix) acc[i] = __fdiv_rn(acc[i], n);
}

// mean_from_iter (src/execute_gpu.rs:819-847) into device memory: the
// sequential per-pixel sum over the frames, then / n_frames.
template <typename T>
gt_status mean_device(gt_ctx* ctx, const T* frames, bool on_device, int64_t NT, int32_t H, int32_t W, float* acc) {
    const size_t npx = (size_t)H * W;
    const int F = pick_chunk(NT, H, W, 0);
    CK(cudaMemsetAsync(acc, 0, npx * 4, ctx->st));
    if (!on_device) CK(ctx->stage[0].ensure((size_t)F * npx * sizeof(T)));
    for (int64_t f0 = 0; f0 < NT; f0 += F) {
        if (interrupted(ctx)) return set_err(ctx, GT_ERR_INTERRUPTED, "Keyboard Interrupt, my custom version");
        int nf = (int)std::min<int64_t>(F, NT - f0);
        const T* src = frames + f0 * npx;
        if (!on_device) {
            CK(cudaMemcpyAsync(ctx->stage[0].p, src, (size_t)nf * npx * sizeof(T), cudaMemcpyHostToDevice,
                               ctx->st));
            src = ctx->stage[0].as<T>();
        }
        Prof pf(ctx, "mean_frame");
        mean_accumulate_kernel<T><<<(unsigned)((npx + 255) / 256), 256, 0, ctx->st>>>(src, nf, npx, acc);
        CK(cudaGetLastError());
    }
    {
        Prof pf(ctx, "mean_frame");
        mean_divide_kernel<<<(unsigned)((npx + 255) / 256), 256, 0, ctx->st>>>(acc, npx, (float)NT);
    }
    CK(cudaGetLastError());
    return GT_OK;
}

// Illumination correction set-up (src/execute_gpu.rs:1324-1330, 849-884): the
// smoothing taps exp(-x^2 / (2 sigma^2)), rint = i32(4 sigma + 0.5), and,
// unless the profile is per frame, the smoothed mean frame of the whole call.
template <typename T>
gt_status illumination_setup(gt_ctx* ctx, const gt_params& p, const T* frames, bool on_device, int64_t NT, int32_t H,
                             int32_t W) {
    const float sigma = p.illumination_sigma;
    const float sigma2 = sigma * sigma;
    const float rf = 4.0f * sigma + 0.5f;
    if (!(rf < 65536.0f)) return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "illumination_sigma too large");
    const int32_t rint = (int32_t)rf;
    std::vector<float> taps((size_t)(2 * rint + 1));
    for (int32_t i = -rint; i <= rint; i++) {
        const float x = (float)i;
        const float x2 = x * x;
        taps[(size_t)(i + rint)] = std::exp(-x2 / (2.0f * sigma2));
    }
    CKS(upload(ctx, ctx->illum_taps, taps));
    ctx->illum_rint = rint;
    if (!p.illumination_correction_per_frame) {
        const size_t npx = (size_t)H * W;
        CK(ctx->illum_shared.ensure(npx * 4));
        CK(ctx->illum_prof.ensure(npx * 4));
        float* mean = ctx->illum_shared.as<float>();
        CKS(mean_device<T>(ctx, frames, on_device, NT, H, W, mean));
        float* tmp = ctx->illum_prof.as<float>();
        CK(launch_illum_smooth<float>(mean, (int64_t)npx, tmp, H, W, 0, ctx->illum_taps.as<float>(), rint, 1,
                                      ctx->st));
        CK(launch_illum_smooth<float>(tmp, (int64_t)npx, mean, H, W, 1, ctx->illum_taps.as<float>(), rint, 1,
                                      ctx->st));
    }
    return GT_OK;
}

template <typename T>
gt_status locate_pass(gt_ctx* ctx, const gt_params& p, const T* frames, bool on_device, int64_t NT, int32_t H,
                      int32_t W, const LocateConsts& c_in, const LogTables* lt, int F, uint32_t* out_flags,
                      PipeLink* pl, const std::vector<uint8_t>* reset, const gt_proposal* net) {
    LocateConsts c = c_in;
    const size_t npx = (size_t)H * W;
    const bool log_style = (p.style == GT_STYLE_LOG);
    const int nslots = log_style ? (int)lt->radii.size() : 1;
    const uint32_t cand_cap = ctx->cand_cap, feat_cap = ctx->feat_cap;
    // super-chunks of SC frames: located chunk by chunk (F frames per launch),
    // then finalized together (one CTA per frame fills the GPU)
    const int per_super = std::max(1, (int)std::min<int64_t>(128 / F, (NT + F - 1) / F));
    const int SC = F * per_super;
    const int nsuper = (int)((NT + SC - 1) / SC);
    CK(ctx->processed.ensure((size_t)F * npx * 4));
    if (log_style && !lt->fused()) CK(ctx->planes.ensure((size_t)F * nslots * npx * 4));
    CK(ctx->cand_count.ensure((size_t)F * nslots * 4));
    CK(ctx->cand_keys.ensure((size_t)F * nslots * cand_cap * 4));
    CK(ctx->feats_raw.ensure((size_t)SC * feat_cap * sizeof(Feature)));
    CK(ctx->feat_count.ensure((size_t)SC * 4));
    CK(ctx->feats_out.ensure((size_t)NT * feat_cap * sizeof(Feature)));
    CK(ctx->kept_count.ensure((size_t)NT * 4));
    CK(ctx->flags.ensure(16));
    CK(cudaMemsetAsync(ctx->flags.p, 0, 16, ctx->st));
    CK(ctx->walk_starts.ensure(8));
    CK(cudaMemsetAsync(ctx->walk_starts.p, 0, 8, ctx->st));
    if (pl) CKS(pl->setup(ctx, NT, feat_cap, SC, p.search_range, (int)p.memory, *reset, H));
    // finalize scratch for frames with more detections than shared memory sorts
    size_t fin_per_frame = 0;
    if (feat_cap > (uint32_t)kFinalizeSmemSort) {
        size_t np2 = 1;
        while (np2 < feat_cap) np2 <<= 1;
        fin_per_frame = (np2 * 17 + 255) & ~(size_t)255;
    }
    CK(ctx->fin_scratch.ensure(std::max<size_t>(fin_per_frame * SC, 256)));
    {
        std::vector<int32_t> ident(SC);
        for (int i = 0; i < SC; i++) ident[i] = i;
        CKS(upload(ctx, ctx->ident, ident));
    }
    // constant tables
    std::vector<float2> atab;
    std::vector<int32_t> aoff;
    int max_rint = log_style ? 0 : std::max(0, (c.circle - 1) / 2);
    if (log_style)
        for (float r : lt->radii) max_rint = std::max(max_rint, (int)std::ceil(r));
    angle_tables(max_rint, atab, aoff);
    std::vector<short2> dn;
    std::vector<int4> dmeta;
    std::vector<float> dradii;
    if (log_style) dradii = lt->radii;
    else dradii.push_back((float)p.diameter / 2.0f);
    doughnut_tables(p, dradii, dn, dmeta);
    CKS(upload(ctx, ctx->tabs_f, atab));
    CKS(upload(ctx, ctx->tabs_i, aoff));
    CKS(upload(ctx, ctx->tabs_s, dn));
    CKS(upload(ctx, ctx->tabs_m, dmeta));
    // LoG tables
    DBuf ltg, ltd, loff, lrint, lng, lnd, lrad;
    if (log_style) {
        CKS(upload(ctx, ltg, lt->taps_g));
        CKS(upload(ctx, ltd, lt->taps_d));
        CKS(upload(ctx, loff, lt->tap_off));
        CKS(upload(ctx, lrint, lt->rints));
        CKS(upload(ctx, lng, lt->norm_g));
        CKS(upload(ctx, lnd, lt->norm_d));
        CKS(upload(ctx, lrad, lt->radii));
    }
    FinalizeConsts fc;
    std::memset(&fc, 0, sizeof(fc));
    fc.H = H;
    fc.W = W;
    fc.log_style = log_style ? 1 : 0;
    fc.prune = (log_style && p.overlap_threshold < 1.0f) ? 1 : 0;
    fc.overlap_threshold = p.overlap_threshold;
    fc.filter_close = (!log_style && p.filter_close) ? 1 : 0;
    fc.separation = (float)p.separation;
    {
        // every filter_close neighbour's candidate row lies within this band
        // when the processed image is non-negative (centroid offsets <= rint)
        int rint = std::max(0, (c.circle - 1) / 2);
        long long band = (long long)std::ceil(fc.separation) + 2LL * ((long long)c.max_iter + rint) + 2;
        fc.band = (c.truncate && band < (1LL << 30)) ? (int32_t)band : -1;
    }
    fc.doughnut = p.doughnut_correction ? 1 : 0;
    fc.presorted = 0;
    fc.scratch_per_frame = fin_per_frame;
    if (log_style) {
        for (size_t k = 0; k < lt->radii.size(); k++) {
            int rank = 0;
            for (size_t q = 0; q < lt->radii.size(); q++)
                if (lt->radii[q] > lt->radii[k]) rank++;
            fc.radius_rank_desc[k] = (uint8_t)rank;
        }
    }
    // snr / minmass_snr: the per-frame std of each chunk, computed before its
    // bandpass (src/execute_gpu.rs:183-186); adaptive_background: its passes
    // after the walk (src/execute_gpu.rs:289-366)
    const bool std_pass = p.has_snr || p.has_minmass_snr;
    const bool adaptive = p.has_adaptive_background;
    const bool illum = p.has_illumination_sigma != 0;
    const int32_t illum_rint = ctx->illum_rint;
    if (illum) {
        CK(ctx->illum_corr.ensure((size_t)F * npx * 4));
        if (p.illumination_correction_per_frame) CK(ctx->illum_prof.ensure((size_t)F * npx * 4));
    }
    if (std_pass || adaptive) {
        CK(ctx->fstd.ensure((size_t)F * 4));
        CK(cudaMemsetAsync(ctx->fstd.p, 0, (size_t)F * 4, ctx->st));  // no std pass: the reference's buffer stays 0
        c.frame_std = ctx->fstd.as<float>();
    }
    if (std_pass) CK(ctx->std_scratch.ensure(std_scratch_floats((int64_t)npx, F) * 4));
    if (adaptive) {
        CK(ctx->amask.ensure((size_t)F * npx));
        CK(ctx->astatus.ensure((size_t)F * feat_cap));
        CK(ctx->acount.ensure((size_t)F * 4));
    }
    LogConsts lc;
    lc.H = H;
    lc.W = W;
    lc.n_radii = nslots;
    lc.thr = 0.0f;
    lc.frame_std = c.frame_std;
    lc.snr = c.snr;
    lc.rough = c.rough;

    // learned proposals: the network runs on groups of cnn_g frames (about
    // 160 MB of activations per layer at 64 B per 4x4 cell): long persistent
    // launches, part of each layer's input still in L2 for the next
    const int Hc = (H + 3) / 4, Wc = (W + 3) / 4;
    const size_t cells = (size_t)Hc * Wc;
    const int cnn_g = net ? (int)std::max<size_t>(1, std::min<size_t>((size_t)F, (160u << 20) / (cells * 64))) : 0;
    if (net) {
        CK(ctx->cnn_x.ensure((size_t)cnn_g * cells * 32));
        CK(ctx->cnn_p.ensure((size_t)cnn_g * cells * 64));
        CK(ctx->cnn_q.ensure((size_t)cnn_g * cells * 64));
        CK(ctx->cnn_head.ensure((size_t)cnn_g * cells * 16));
    }
    const size_t super_bytes = (size_t)SC * npx * sizeof(T);
    if (!on_device) {
        CK(ctx->stage[0].ensure(super_bytes));
        CK(ctx->stage[1].ensure(super_bytes));
    }
    auto issue_copy = [&](int sc) -> gt_status {
        int b = sc & 1;
        int64_t f0 = (int64_t)sc * SC;
        int nf = (int)std::min<int64_t>(SC, NT - f0);
        CK(cudaStreamWaitEvent(ctx->cp, ctx->used[b], 0));
        CK(cudaMemcpyAsync(ctx->stage[b].p, frames + f0 * npx, (size_t)nf * npx * sizeof(T), cudaMemcpyHostToDevice,
                           ctx->cp));
        CK(cudaEventRecord(ctx->filled[b], ctx->cp));
        return GT_OK;
    };
    if (!on_device) {
        // both staging buffers start free
        CK(cudaEventRecord(ctx->used[0], ctx->st));
        CK(cudaEventRecord(ctx->used[1], ctx->st));
        CKS(issue_copy(0));
    }
    uint32_t* flags = ctx->flags.as<uint32_t>();
    float* proc = ctx->processed.as<float>();
    for (int sc = 0; sc < nsuper; sc++) {
        if (interrupted(ctx)) {
            cudaStreamSynchronize(ctx->st);
            cudaStreamSynchronize(ctx->cp);
            sync_link_streams(ctx);
            return set_err(ctx, GT_ERR_INTERRUPTED, "Keyboard Interrupt, my custom version");
        }
        const int64_t s0 = (int64_t)sc * SC;
        const int ns = (int)std::min<int64_t>(SC, NT - s0);
        const T* sbase;
        if (on_device) {
            sbase = frames + s0 * npx;
        } else {
            if (sc + 1 < nsuper) CKS(issue_copy(sc + 1));
            CK(cudaStreamWaitEvent(ctx->st, ctx->filled[sc & 1], 0));
            sbase = ctx->stage[sc & 1].as<T>();
        }
        CK(cudaMemsetAsync(ctx->feat_count.p, 0, (size_t)ns * 4, ctx->st));
        for (int64_t c0f = 0; c0f < ns; c0f += F) {
            const int nf = (int)std::min<int64_t>(F, ns - c0f);
            // the locate stages of one chunk, on the input frames or on the
            // illumination-corrected f32 frames
            auto run_chunk = [&](auto* src) -> gt_status {
                using TS = typename std::remove_const<typename std::remove_pointer<decltype(src)>::type>::type;
                if (std_pass) {
                    Prof pf(ctx, "frame_std");
                    CK(launch_frame_std<TS>(src, (int64_t)npx, nf, (int64_t)npx, nullptr, nullptr, ctx->fstd.as<float>(),
                                           ctx->std_scratch.as<float>(), ctx->st));
                }
                CK(cudaMemsetAsync(ctx->cand_count.p, 0, (size_t)nf * nslots * 4, ctx->st));
                if (net) {
                    // seeds from the network, then the walk on per-seed patches
                    {
                        Prof pf(ctx, "proposal_net");
                        const CnnNet nv = net->views();
                        for (int g0 = 0; g0 < nf; g0 += cnn_g) {
                            const int ng = std::min(cnn_g, nf - g0);
                            CK(cnn_input<TS>(src + (size_t)g0 * npx, (int64_t)npx, H, W, nullptr, ng, Hc, Wc,
                                             net->mean, net->scale, ctx->cnn_x.as<__nv_bfloat16>(), ctx->st));
                            CK(cnn_forward(nv, ctx->cnn_x.as<__nv_bfloat16>(), ng, Hc, Wc,
                                           ctx->cnn_p.as<__nv_bfloat16>(), ctx->cnn_q.as<__nv_bfloat16>(),
                                           ctx->cnn_p.as<__nv_bfloat16>(), ctx->cnn_head.as<float4>(), flags,
                                           ctx->num_sms, ctx->st));
                            CK(cnn_proposals(ctx->cnn_head.as<float4>(), ng, Hc, Wc, H, W, c.margin, net->threshold,
                                             ctx->cand_count.as<uint32_t>() + g0,
                                             ctx->cand_keys.as<uint32_t>() + (size_t)g0 * cand_cap, cand_cap, flags,
                                             ctx->st));
                        }
                    }
                    sum_counts_kernel<<<1, 256, 0, ctx->st>>>(ctx->cand_count.as<uint32_t>(), nf, cand_cap,
                                                              ctx->walk_starts.as<unsigned long long>());
                    CK(cudaGetLastError());
                    Prof pf(ctx, "walk_local");
                    CK(launch_walk_local<TS>(src, (int64_t)npx, c, nf, ctx->cand_count.as<uint32_t>(),
                                             ctx->cand_keys.as<uint32_t>(), cand_cap, ctx->tabs_i.as<int32_t>(),
                                             ctx->tabs_f.as<float2>(),
                                             ctx->feats_raw.as<Feature>() + (size_t)c0f * feat_cap,
                                             ctx->feat_count.as<uint32_t>() + c0f, feat_cap, flags, ctx->st));
                    return GT_OK;
                }
                if (!log_style) {
                    Prof pf(ctx, "bandpass_localmax");
                    CK(launch_bandpass<TS>(src, (int64_t)npx, proc, c, nf, true, ctx->cand_count.as<uint32_t>(),
                                          ctx->cand_keys.as<uint32_t>(), cand_cap, flags, ctx->st));
                } else {
                    {
                        Prof pf(ctx, "bandpass");
                        cudaError_t es = cudaSuccess;
                        if (launch_strip_processed<TS>(src, (int64_t)npx, proc, c, nf, ctx->cand_count.as<uint32_t>(),
                                                       ctx->cand_keys.as<uint32_t>(), flags, ctx->st, &es)) {
                            CK(es);
                        } else {
                            CK(launch_bandpass<TS>(src, (int64_t)npx, proc, c, nf, false, nullptr, nullptr, 0, flags,
                                                  ctx->st));
                        }
                    }
                    if (lt->fused()) {
                        Prof pf(ctx, "log_scale_space");
                        CK(launch_log_scale_space<TS>(src, (int64_t)npx, proc, lc, ltg.as<float>(), ltd.as<float>(),
                                                     loff.as<int32_t>(), lrint.as<int32_t>(), lng.as<float>(),
                                                     lnd.as<float>(), lt->max_rint, (int)lt->taps_g.size(), nf,
                                                     ctx->cand_count.as<uint32_t>(), ctx->cand_keys.as<uint32_t>(),
                                                     cand_cap, flags, lt->taps_g.data(), lt->taps_d.data(),
                                                     lt->tap_off.data(), lt->rints.data(), ctx->st));
                    } else {
                        {
                            Prof pf(ctx, "laplace");
                            CK(launch_laplace<TS>(src, (int64_t)npx, ctx->planes.as<float>(), lc, ltg.as<float>(),
                                                 ltd.as<float>(), loff.as<int32_t>(), lrint.as<int32_t>(),
                                                 lng.as<float>(), lnd.as<float>(), lt->max_rint, nf, ctx->st));
                        }
                        {
                            Prof pf(ctx, "logspace_max");
                            CK(launch_logspace_max(ctx->planes.as<float>(), proc, lc, nf,
                                                   ctx->cand_count.as<uint32_t>(), ctx->cand_keys.as<uint32_t>(),
                                                   cand_cap, flags, ctx->st));
                        }
                    }
                }
                sum_counts_kernel<<<1, 256, 0, ctx->st>>>(ctx->cand_count.as<uint32_t>(), nf * nslots, cand_cap,
                                                          ctx->walk_starts.as<unsigned long long>());
                CK(cudaGetLastError());
                {
                    Prof pf(ctx, "walk_characterize");
                    CK(launch_walk<TS>(proc, src, (int64_t)npx, c, nf, nslots, ctx->cand_count.as<uint32_t>(),
                                      ctx->cand_keys.as<uint32_t>(), cand_cap, cand_cap,
                                      log_style ? lrad.as<float>() : nullptr, ctx->tabs_i.as<int32_t>(),
                                      ctx->tabs_f.as<float2>(), ctx->feats_raw.as<Feature>() + (size_t)c0f * feat_cap,
                                      ctx->feat_count.as<uint32_t>() + c0f, feat_cap, flags, ctx->st));
                }
                if (adaptive) {
                    // adaptive_filter passes over the chunk's walked rows; the
                    // masked frame's std is recomputed before every pass but the first
                    Prof pf(ctx, "adaptive");
                    Feature* fr = ctx->feats_raw.as<Feature>() + (size_t)c0f * feat_cap;
                    uint32_t* fcn = ctx->feat_count.as<uint32_t>() + c0f;
                    uint8_t* status = ctx->astatus.as<uint8_t>();
                    uint32_t* counters = ctx->acount.as<uint32_t>();
                    uint8_t* mask = ctx->amask.as<uint8_t>();
                    CK(launch_adaptive_init(counters, (uint32_t)npx, status, (size_t)nf * feat_cap, nf, ctx->st));
                    CK(cudaMemsetAsync(mask, 0, (size_t)nf * npx, ctx->st));
                    for (uint32_t it = 0; it < p.adaptive_background; it++) {
                        if (it > 0)
                            CK(launch_frame_std<TS>(src, (int64_t)npx, nf, (int64_t)npx, mask, counters,
                                                   ctx->fstd.as<float>(), ctx->std_scratch.as<float>(), ctx->st));
                        CK(launch_adaptive_pass(fr, fcn, feat_cap, status, ctx->fstd.as<float>(), c.minmass,
                                                c.minmass_snr, c.snr, mask, counters, H, W, c.circle, nf, ctx->st));
                    }
                    CK(launch_adaptive_compact(fr, fcn, feat_cap, status, nf, ctx->st));
                }

                return GT_OK;
            };
            const T* csrc = sbase + c0f * npx;
            if (illum) {
                Prof pf(ctx, "illumination");
                float* corr = ctx->illum_corr.as<float>();
                if (p.illumination_correction_per_frame) {
                    // the profile of each frame is the frame itself, smoothed
                    float* prof = ctx->illum_prof.as<float>();
                    CK(launch_illum_smooth<T>(csrc, (int64_t)npx, corr, H, W, 0, ctx->illum_taps.as<float>(),
                                              illum_rint, nf, ctx->st));
                    CK(launch_illum_smooth<float>(corr, (int64_t)npx, prof, H, W, 1, ctx->illum_taps.as<float>(),
                                                  illum_rint, nf, ctx->st));
                    CK(launch_illum_divide<T>(csrc, (int64_t)npx, prof, (int64_t)npx, corr, (int64_t)npx, nf,
                                              ctx->st));
                } else {
                    CK(launch_illum_divide<T>(csrc, (int64_t)npx, ctx->illum_shared.as<float>(), 0, corr,
                                              (int64_t)npx, nf, ctx->st));
                }
                CKS(run_chunk((const float*)corr));
            } else {
                CKS(run_chunk(csrc));
            }
        }
        {
            Prof pf(ctx, "finalize");
            CK(launch_finalize<T>(ctx->feats_raw.as<Feature>(), ctx->feat_count.as<uint32_t>(), feat_cap,
                                  ctx->feats_out.as<Feature>() + (size_t)s0 * feat_cap,
                                  ctx->kept_count.as<uint32_t>() + s0, ctx->fin_scratch.as<uint8_t>(), fc, sbase,
                                  (int64_t)npx, ctx->ident.as<int32_t>(), ctx->tabs_s.as<short2>(),
                                  ctx->tabs_m.as<int4>(), flags, ns, ctx->st));
        }
        if (!on_device) CK(cudaEventRecord(ctx->used[sc & 1], ctx->st));
        if (pl) CKS(pl->window((int)s0, (int)(s0 + ns), sc == 0, sc == nsuper - 1));
        ctx->done = s0 + ns;
    }
    CK(cudaMemcpyAsync(out_flags, flags, 4, cudaMemcpyDeviceToHost, ctx->st));
    unsigned long long starts = 0;
    CK(cudaMemcpyAsync(&starts, ctx->walk_starts.p, 8, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->last_walk_starts = (int64_t)starts;
    drain_profile(ctx, false);
    return GT_OK;
}

// Assemble the output table from per-frame results (kept_count, feats_out)
// of the NT frame slots starting at slot0.
gt_status assemble_table(gt_ctx* ctx, int64_t NT, const std::vector<int64_t>& frame_numbers, bool log_style,
                         gt_table* tab, std::vector<int64_t>& row_off, int64_t slot0 = 0) {
    std::vector<uint32_t> kept(NT);
    CK(cudaMemcpyAsync(kept.data(), ctx->kept_count.as<uint32_t>() + slot0, NT * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    row_off.assign(NT + 1, 0);
    uint32_t maxk = 0;
    for (int64_t t = 0; t < NT; t++) {
        row_off[t + 1] = row_off[t] + kept[t];
        maxk = std::max(maxk, kept[t]);
    }
    const int64_t N = row_off[NT];
    tab->n = N;
    const size_t n1 = std::max<int64_t>(N, 1);
    CK(tab->frame.ensure(n1 * 8));
    for (int c = 0; c < GT_NUM_COLUMNS; c++) {
        if (c == GT_COL_FRAME || c == GT_COL_PARTICLE || c == GT_COL_DURATION) continue;
        CK(tab->col[c].ensure(n1 * 4));
        tab->has[c] = true;
    }
    tab->has[GT_COL_FRAME] = true;
    (void)log_style;
    CKS(upload(ctx, ctx->row_off, row_off));
    CKS(upload(ctx, ctx->frame_num, frame_numbers));
    TableCols tc;
    tc.frame = tab->frame.as<int64_t>();
    for (int c = 0; c < GT_NUM_COLUMNS; c++) tc.col[c] = tab->col[c].as<float>();
    tc.particle = nullptr;
    tc.duration = nullptr;
    for (int64_t g0 = 0; g0 < NT; g0 += 65535) {
        int ng = (int)std::min<int64_t>(65535, NT - g0);
        Prof pf(ctx, "scatter");
        CK(launch_scatter(ctx->feats_out.as<Feature>() + (size_t)(slot0 + g0) * ctx->feat_cap, ctx->feat_cap,
                          ctx->kept_count.as<uint32_t>() + slot0 + g0, maxk, ctx->row_off.as<int64_t>(),
                          ctx->frame_num.as<int64_t>(), tc, (int32_t)g0, ng, ctx->st));
    }
    return GT_OK;
}

template <typename T>
gt_status batch_impl(gt_ctx* ctx, const gt_params& p, const T* frames, bool on_device, int64_t NT, int32_t H,
                     int32_t W, const int64_t* frame_numbers, const int64_t* reset_points, int64_t n_reset,
                     gt_table* tab, const gt_proposal* net = nullptr) {
    LocateConsts c;
    CKS(make_locate_consts(ctx, p, H, W, c));
    set_fast_div<T>(ctx, c);
    if (net) {
        const int ri = (c.circle - 1) / 2;
        if (ri < 2 || ri > 7)
            return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "learned proposals need a diameter between 5 and 16");
        if (c.R > 7 || walk_local_smem_bytes(c.circle, c.R) > 227 * 1024)
            return set_err(ctx, GT_ERR_INVALID_ARGUMENT,
                           "learned proposals need a smoothing_size of at most 15 (the seed-patch walk)");
    }
    if (p.has_illumination_sigma) {
        // the locate stages see the corrected f32 frames
        c.fast_div = 0;
        CKS(illumination_setup<T>(ctx, p, frames, on_device, NT, H, W));
    }
    LogTables lt;
    const bool log_style = (p.style == GT_STYLE_LOG);
    if (log_style) {
        lt = log_tables(p);
        if (lt.radii.empty()) return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "n_radii must be >= 1");
        if (lt.radii.size() > (size_t)kMaxRadii) return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "n_radii > 256");
        if (!lt.fused() && laplace_smem_bytes(lt.max_rint) > 227 * 1024)
            return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "max_radius too large for the LoG tile kernel");
    } else {
        if (bandpass_smem_bytes(c.R, c.kd, true) > 227 * 1024)
            return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "separation/smoothing_size too large for the tile kernel");
    }
    if (bandpass_smem_bytes(c.R, 1, false) > 227 * 1024)
        return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "smoothing_size too large for the tile kernel");
    {
        // the reference computes the frame std (snr / minmass_snr) as a tree of
        // 8-way sums; where a level's length is not a multiple of 8 its shaders
        // read what earlier passes left in a shared buffer, so only pixel counts
        // whose levels all divide by 8 have a reproducible result
        const bool std_pass = p.has_snr || p.has_minmass_snr;
        if (std_pass && !std_reduction_exact((int64_t)H * W))
            return set_err(ctx, GT_ERR_INVALID_ARGUMENT,
                           "snr / minmass_snr need a frame of N = H*W pixels with N = 8^k * m, m <= 24 (e.g. "
                           "512x512, 1024x1024, 2048x2048): got %dx%d",
                           H, W);
        if (p.has_adaptive_background && p.adaptive_background == 0)
            return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "adaptive_background must be at least 1");
        if (p.has_adaptive_background && p.adaptive_background >= 2 && !std_pass)
            return set_err(ctx, GT_ERR_INVALID_ARGUMENT,
                           "adaptive_background >= 2 needs snr or minmass_snr (the image std between passes)");
    }
    const int F = pick_chunk(NT, H, W, (log_style && !lt.fused()) ? (int)lt.radii.size() : 0);
    ctx->total = NT;
    ctx->done = 0;
    std::vector<int64_t> fnum(NT);
    for (int64_t t = 0; t < NT; t++) fnum[t] = frame_numbers ? frame_numbers[t] : t;
    std::vector<uint8_t> reset(NT, 0);
    for (int64_t t = 0; t < NT; t++)
        for (int64_t k = 0; k < n_reset; k++)
            if (reset_points[k] == fnum[t]) reset[t] = 1;
    PipeLink pl;
    bool windowed = false;
    for (int attempt = 0;; attempt++) {
        uint32_t fl = 0;
        HostSpan hs(ctx, "host_locate");
        // frames link while later frames are located when every frame's
        // detections sort in shared memory (the group sort's limit)
        windowed = p.has_search_range && ctx->feat_cap <= 4096u;
        gt_status st = locate_pass<T>(ctx, p, frames, on_device, NT, H, W, c, log_style ? &lt : nullptr, F, &fl,
                                      windowed ? &pl : nullptr, &reset, net);
        if (st != GT_OK) {
            sync_link_streams(ctx);
            return st;
        }
        if (fl & (kFlagTensorTimeout | kFlagLocalWalk)) {
            sync_link_streams(ctx);
            return set_err(ctx, GT_ERR_INTERNAL,
                           (fl & kFlagTensorTimeout) ? "a tensor-core kernel timed out waiting for its UMMAs"
                                                     : "a learned seed's walk did not finish");
        }
        if (!(fl & (kFlagCandOverflow | kFlagFeatOverflow))) break;
        CK(sync_link_streams(ctx));
        const uint64_t npx = (uint64_t)H * W;
        if (attempt > 8) return set_err(ctx, GT_ERR_CAPACITY_EXCEEDED, "per-frame capacity exceeded");
        if (fl & kFlagCandOverflow) {
            uint64_t nc = std::min<uint64_t>((uint64_t)ctx->cand_cap * 4, npx + 1);
            if (nc <= ctx->cand_cap)
                return set_err(ctx, GT_ERR_CAPACITY_EXCEEDED, "candidate capacity exceeded");
            ctx->cand_cap = (uint32_t)nc;
        }
        if (fl & kFlagFeatOverflow) {
            uint64_t nf = std::min<uint64_t>((uint64_t)ctx->feat_cap * 4, std::min<uint64_t>(npx + 1, 1u << 24));
            if (nf <= ctx->feat_cap)
                return set_err(ctx, GT_ERR_CAPACITY_EXCEEDED, "per-frame detection capacity exceeded");
            ctx->feat_cap = (uint32_t)nf;
        }
    }
    std::vector<int64_t> row_off;
    {
        HostSpan hs(ctx, "host_assemble");
        gt_status st = assemble_table(ctx, NT, fnum, log_style, tab, row_off);
        if (st != GT_OK) {
            sync_link_streams(ctx);
            return st;
        }
    }
    if (p.has_search_range) {
        HostSpan hs(ctx, "host_link");
        const size_t n1 = std::max<int64_t>(tab->n, 1);
        CK(tab->particle.ensure(n1 * 8));
        CK(tab->duration.ensure(n1 * 8));
        bool whole = !windowed;
        if (windowed) {
            // the table rows take the windowed linker's ids and durations
            CK(cudaEventRecord(ctx->linked, ctx->lk));
            CK(cudaStreamWaitEvent(ctx->st, ctx->linked, 0));
            {
                Prof pf(ctx, "link_rows");
                CK(link_slot_rows(pl.in, pl.out, ctx->row_off.as<int64_t>(), tab->particle.as<int64_t>(),
                                  tab->duration.as<int64_t>(), ctx->st));
            }
            uint32_t lf = 0;
            CK(cudaMemcpyAsync(&lf, pl.out.flags, 4, cudaMemcpyDeviceToHost, ctx->st));
            CK(cudaStreamSynchronize(ctx->st));
            if (lf & kFlagTooDense)
                return set_err(ctx, GT_ERR_TOO_DENSE_TO_LINK,
                               "computational load during linking is abnormally high. try setting a smaller search "
                               "range or track with settings that give fewer detections.");
            if (lf & kFlagSubnetBudget)
                return set_err(ctx, GT_ERR_SUBNET_TOO_EXPENSIVE, "a linking subnet exceeded the device search budget");
            if (lf & (kFlagListOverflow | kFlagEdgeOverflow)) {
                // buffers too small for this video: grow them for the next
                // call and link this one with the whole-video linker
                if (lf & kFlagListOverflow) ctx->w_list_cap *= 4;
                if (lf & kFlagEdgeOverflow) ctx->w_edge_cap *= 4;
                whole = true;
            } else if (lf & kFlagScratch) {
                return set_err(ctx, GT_ERR_INTERNAL,
                               "a particle id has no duration entry after a linker reset (the reference panics here)");
            }
        }
        if (whole) {
            LinkJob job;
            job.goff = row_off;
            job.vgrp = {0, (int32_t)NT};
            job.reset = reset;
            job.radius = p.search_range;
            job.memory = (int32_t)p.memory;
            CK(ctx->l_ids.ensure(n1 * 8));
            CKS(run_link(ctx, job, tab->col[GT_COL_Y].as<float>(), tab->col[GT_COL_X].as<float>(),
                         ctx->l_ids.as<int64_t>(), tab->duration.as<int64_t>(), nullptr, nullptr));
            if (tab->n > 0) {
                Prof pf(ctx, "round_ids");
                CK(launch_round_ids(ctx->l_ids.as<int64_t>(), tab->particle.as<int64_t>(), tab->n, ctx->st));
            }
            CK(cudaGetLastError());
        }
        tab->has[GT_COL_PARTICLE] = true;
        tab->has[GT_COL_DURATION] = true;
    }
    if (!p.doughnut_correction) {
        tab->has[GT_COL_RAW_MASS] = tab->has[GT_COL_RAW_BG_MEDIAN] = tab->has[GT_COL_RAW_MASS_CORRECTED] = false;
    }
    {
        HostSpan hs(ctx, "host_tail_sync");
        CK(cudaStreamSynchronize(ctx->st));
    }
    drain_profile(ctx);
    return GT_OK;
}

gt_status validate(gt_ctx* ctx, const gt_params* p, const void* frames, int32_t dtype, int64_t T, int32_t H,
                   int32_t W) {
    if (!ctx) return GT_ERR_INVALID_ARGUMENT;
    if (!p || !frames) return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "null argument");
    if (T <= 0) return set_err(ctx, GT_ERR_EMPTY_ITERATOR, "the provided video doesn't contain any frames.");
    if (H <= 0 || W <= 0) return set_err(ctx, GT_ERR_DIMENSION_MISMATCH, "frame dimensions must be positive");
    if ((int64_t)H * W >= (1LL << 31)) return set_err(ctx, GT_ERR_DIMENSION_MISMATCH, "frame too large");
    if (dtype != GT_DTYPE_U16 && dtype != GT_DTYPE_F32 && dtype != GT_DTYPE_U8)
        return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "unsupported dtype %d", dtype);
    if (p->style != GT_STYLE_TRACKPY && p->style != GT_STYLE_LOG)
        return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "unknown style %d", p->style);
    if (p->has_illumination_sigma && !(p->illumination_sigma > 0.0f))
        return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "illumination_sigma must be positive");
    if (p->style == GT_STYLE_TRACKPY && p->diameter == 0)
        return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "diameter must be positive");
    CK(cudaSetDevice(ctx->device));
    return GT_OK;
}

// FrameSubsetter grouping of rows sorted by their frame column
// (src/linking.rs:97-196): a group is emitted whenever the frame number
// increases (so a positive first frame yields a leading empty group 0); a
// decreasing frame number is NonSortedCharacterization.

template <typename T>
gt_status mean_impl(gt_ctx* ctx, const T* frames, bool on_device, int64_t NT, int32_t H, int32_t W, float* out) {
    const size_t npx = (size_t)H * W;
    CK(ctx->processed.ensure(npx * 4));
    float* acc = ctx->processed.as<float>();
    CKS(mean_device<T>(ctx, frames, on_device, NT, H, W, acc));
    CK(cudaMemcpyAsync(out, acc, npx * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return GT_OK;
}

// characterize_points (src/execute_gpu.rs:189-229, 1286-1319;
// gpu_tracking_macros/src/lib.rs:641-683)
template <typename T>
gt_status charpoints_impl(gt_ctx* ctx, const gt_params& p0, const T* frames, bool on_device, int64_t NT, int32_t H,
                          int32_t W, const float* points, int64_t n, int32_t has_frames, int32_t has_r,
                          gt_table* tab) {
    gt_params p = p0;
    p.style = GT_STYLE_TRACKPY;
    p.filter_close = 0;
    p.characterize = 1;
    const int ncols = 2 + (has_frames ? 1 : 0) + (has_r ? 1 : 0);
    const int c0 = has_frames ? 1 : 0;
    std::vector<int64_t> goff, gframe;
    if (has_frames) {
        CKS(subset_groups(ctx, points, n, ncols, goff, gframe));
    } else {
        goff.assign(1, 0);
        for (int64_t t = 0; t < NT; t++) {
            goff.push_back(goff.back() + n);
            gframe.push_back(t);
        }
    }
    const int64_t G = (int64_t)gframe.size();
    if (G == 0) return set_err(ctx, GT_ERR_EMPTY_ITERATOR, "the provided video doesn't contain any frames.");
    for (int64_t g = 0; g < G; g++)
        if (gframe[g] >= NT)
            return set_err(ctx, GT_ERR_FRAME_OUT_OF_BOUNDS,
                           "Requested a frame outside the length\n of the video. Video length is %lld, requested "
                           "frame %lld",
                           (long long)NT, (long long)gframe[g]);
    // (y, x, r) per point in group order
    std::vector<float> pts((size_t)goff.back() * 3);
    int64_t maxg = 0;
    float max_r = 0.0f;
    for (int64_t g = 0; g < G; g++) {
        maxg = std::max(maxg, goff[g + 1] - goff[g]);
        for (int64_t i = goff[g]; i < goff[g + 1]; i++) {
            int64_t src = has_frames ? i : (i - goff[g]);
            pts[3 * i + 0] = points[src * ncols + c0];
            pts[3 * i + 1] = points[src * ncols + c0 + 1];
            pts[3 * i + 2] = has_r ? points[src * ncols + c0 + 2] : 0.0f;
            if (has_r && pts[3 * i + 2] > max_r) max_r = pts[3 * i + 2];
        }
    }
    LocateConsts c;
    CKS(make_locate_consts(ctx, p, H, W, c));
    if (bandpass_smem_bytes(c.R, 1, false) > 227 * 1024)
        return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "smoothing_size too large for the tile kernel");
    const size_t npx = (size_t)H * W;
    const int F = pick_chunk(G, H, W, 0);
    const uint32_t feat_cap = (uint32_t)std::max<int64_t>(maxg, 1);
    if (feat_cap >= (1u << 24)) return set_err(ctx, GT_ERR_CAPACITY_EXCEEDED, "too many points in one frame");
    CK(ctx->processed.ensure((size_t)F * npx * 4));
    CK(ctx->stage[0].ensure((size_t)F * npx * sizeof(T)));
    CK(ctx->feats_raw.ensure((size_t)F * feat_cap * sizeof(Feature)));
    CK(ctx->feat_count.ensure((size_t)F * 4));
    CK(ctx->feats_out.ensure((size_t)G * feat_cap * sizeof(Feature)));
    CK(ctx->kept_count.ensure((size_t)G * 4));
    CK(ctx->flags.ensure(16));
    CK(cudaMemsetAsync(ctx->flags.p, 0, 16, ctx->st));
    size_t fin_per_frame = 0;
    if (feat_cap > (uint32_t)kFinalizeSmemSort) {
        size_t np2 = 1;
        while (np2 < feat_cap) np2 <<= 1;
        fin_per_frame = (np2 * 17 + 255) & ~(size_t)255;
    }
    CK(ctx->fin_scratch.ensure(std::max<size_t>(fin_per_frame * F, 256)));
    DBuf dpts, dgoff, dgloc;
    CKS(upload(ctx, dpts, pts));
    CKS(upload(ctx, dgoff, goff));
    std::vector<int32_t> gloc(G);
    for (int64_t g = 0; g < G; g++) gloc[g] = (int32_t)(g % F);
    CKS(upload(ctx, dgloc, gloc));
    std::vector<int32_t> ident(F);
    for (int i = 0; i < F; i++) ident[i] = i;
    CKS(upload(ctx, ctx->ident, ident));
    std::vector<float2> atab;
    std::vector<int32_t> aoff;
    int max_rint = std::max(std::max(0, (c.circle - 1) / 2), (int)std::ceil(max_r));
    angle_tables(max_rint, atab, aoff);
    std::vector<short2> dn;
    std::vector<int4> dmeta;
    doughnut_tables(p, std::vector<float>{(float)p.diameter / 2.0f}, dn, dmeta);
    CKS(upload(ctx, ctx->tabs_f, atab));
    CKS(upload(ctx, ctx->tabs_i, aoff));
    CKS(upload(ctx, ctx->tabs_s, dn));
    CKS(upload(ctx, ctx->tabs_m, dmeta));
    FinalizeConsts fc;
    std::memset(&fc, 0, sizeof(fc));
    fc.H = H;
    fc.W = W;
    fc.doughnut = p.doughnut_correction ? 1 : 0;
    fc.presorted = 1;
    fc.band = -1;
    fc.scratch_per_frame = fin_per_frame;
    ctx->total = G;
    ctx->done = 0;
    for (int64_t g0 = 0; g0 < G; g0 += F) {
        if (interrupted(ctx)) return set_err(ctx, GT_ERR_INTERRUPTED, "Keyboard Interrupt, my custom version");
        const int ng = (int)std::min<int64_t>(F, G - g0);
        T* stage = ctx->stage[0].as<T>();
        for (int g = 0; g < ng; g++)
            CK(cudaMemcpyAsync(stage + (size_t)g * npx, frames + (size_t)gframe[g0 + g] * npx, npx * sizeof(T),
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemsetAsync(ctx->feat_count.p, 0, (size_t)ng * 4, ctx->st));
        Prof pf1(ctx, "bandpass");
        CK(launch_bandpass<T>(stage, (int64_t)npx, ctx->processed.as<float>(), c, ng, false, nullptr, nullptr, 0,
                              ctx->flags.as<uint32_t>(), ctx->st));
        Prof pf2(ctx, "characterize_points");
        CK(launch_characterize_points<T>(ctx->processed.as<float>(), stage, (int64_t)npx, c, dpts.as<float>(),
                                         dgoff.as<int64_t>(), dgloc.as<int32_t>(), (int32_t)g0, ng, maxg,
                                         ctx->tabs_f.as<float2>(), ctx->tabs_i.as<int32_t>(), (int32_t)aoff.size(),
                                         has_r, ctx->feats_raw.as<Feature>(), ctx->feat_count.as<uint32_t>(),
                                         feat_cap, ctx->st));
        Prof pf3(ctx, "finalize");
        CK(launch_finalize<T>(ctx->feats_raw.as<Feature>(), ctx->feat_count.as<uint32_t>(), feat_cap,
                              ctx->feats_out.as<Feature>() + (size_t)g0 * feat_cap,
                              ctx->kept_count.as<uint32_t>() + g0, ctx->fin_scratch.as<uint8_t>(), fc, stage,
                              (int64_t)npx, ctx->ident.as<int32_t>(), ctx->tabs_s.as<short2>(),
                              ctx->tabs_m.as<int4>(), ctx->flags.as<uint32_t>(), ng, ctx->st));
        ctx->done = g0 + ng;
    }
    const uint32_t saved_cap = ctx->feat_cap;
    ctx->feat_cap = feat_cap;
    std::vector<int64_t> row_off;
    gt_status st = assemble_table(ctx, G, gframe, false, tab, row_off);
    ctx->feat_cap = saved_cap;
    CKS(st);
    tab->has[GT_COL_R] = has_r != 0;
    tab->has[GT_COL_MAX_INTENSITY] = tab->has[GT_COL_COUNT] = false;
    if (!p.doughnut_correction)
        tab->has[GT_COL_RAW_MASS] = tab->has[GT_COL_RAW_BG_MEDIAN] = tab->has[GT_COL_RAW_MASS_CORRECTED] = false;
    if (p.has_search_range) {
        LinkJob job;
        job.goff = row_off;
        job.vgrp = {0, (int32_t)G};
        job.reset.assign(G, 0);
        job.radius = p.search_range;
        job.memory = (int32_t)p.memory;
        const size_t n1 = std::max<int64_t>(tab->n, 1);
        CK(ctx->l_ids.ensure(n1 * 8));
        CK(tab->particle.ensure(n1 * 8));
        CK(tab->duration.ensure(n1 * 8));
        CKS(run_link(ctx, job, tab->col[GT_COL_Y].as<float>(), tab->col[GT_COL_X].as<float>(),
                     ctx->l_ids.as<int64_t>(), tab->duration.as<int64_t>(), nullptr, nullptr));
        if (tab->n > 0) {
            Prof pf(ctx, "round_ids");
            CK(launch_round_ids(ctx->l_ids.as<int64_t>(), tab->particle.as<int64_t>(), tab->n, ctx->st));
        }
        CK(cudaGetLastError());
        tab->has[GT_COL_PARTICLE] = true;
        tab->has[GT_COL_DURATION] = true;
    }
    CK(cudaStreamSynchronize(ctx->st));
    return GT_OK;
}

// ------------------------------------------------------------ ragged batches
// Many videos of uneven frame size located together: the frames of all
// videos, in order, are cut into waves of at most kRaggedSlots frames whose
// processed images fit a byte budget.  A wave runs ONE launch per stage over
// all its frames — the persistent strip kernel over the wave's tile list,
// the walk over every frame's candidates, finalize and the doughnut over the
// frame slots — each launch reading the wave's frame and tile tables from
// device memory.  The launch sequence is therefore captured once as a CUDA
// graph and replayed for every wave after the tables are rewritten.  Tile
// height and wave budget come from the autotuner below.  Results equal one
// gt_batch call per video (same kernels per tile and per frame).
constexpr int kRaggedSlots = 512;

struct RaggedShape {
    int32_t seg;       // rows per strip tile
    int64_t budget;    // processed-image bytes per wave
};

// Candidate shapes: tall tiles waste the fewest halo rows, short ones balance
// the persistent CTAs better on small frames; a small wave keeps its
// processed images in L2 for the walk, a large one fills the GPU with tiles
// and gives finalize (one CTA per frame) many frames at once.
const RaggedShape kRaggedShapes[] = {{512, 4LL << 30},   {256, 4LL << 30},   {128, 4LL << 30},
                                     {512, 1LL << 30},   {256, 1LL << 30},   {128, 1LL << 30},
                                     {512, 192LL << 20}, {256, 192LL << 20}, {128, 192LL << 20}};
constexpr int kRaggedNShapes = (int)(sizeof(kRaggedShapes) / sizeof(kRaggedShapes[0]));

template <typename T>
bool ragged_eligible(const gt_params& p, const LocateConsts& c) {
    if (p.style != GT_STYLE_TRACKPY || p.has_snr || p.has_minmass_snr || p.has_adaptive_background ||
        p.has_illumination_sigma)
        return false;
    if (!std::is_same<T, float>::value && !c.fast_div) return false;
    const int ri = (c.circle - 1) / 2;
    return strip_tile_width<T>(c) > 0 && ri >= 2 && ri <= 7;
}

struct RaggedSlot {
    int32_t video;
    int64_t t;
};

template <typename T>
gt_status batch_videos_ragged(gt_ctx* ctx, const gt_params& p, const LocateConsts& c, int32_t nv,
                              const void* const* frames, const bool* on_device, const int64_t* T_, const int32_t* H_,
                              const int32_t* W_, gt_table** tabs, std::vector<std::vector<int64_t>>& row_off) {
    const int TW = strip_tile_width<T>(c);
    // slots of the call: video v's frame t is slot vslot[v] + t
    std::vector<int64_t> vslot((size_t)nv + 1, 0);
    for (int32_t v = 0; v < nv; v++) vslot[(size_t)v + 1] = vslot[(size_t)v] + T_[v];
    const int64_t NT = vslot[(size_t)nv];
    int64_t max_px = 0;
    for (int32_t v = 0; v < nv; v++) max_px = std::max<int64_t>(max_px, (int64_t)H_[v] * W_[v]);
    // a wave never holds more than the call's frames
    int64_t all_px = 0;
    for (int32_t v = 0; v < nv; v++) all_px += T_[v] * (int64_t)H_[v] * W_[v];
    int64_t max_budget = 0;
    for (const auto& s : kRaggedShapes) max_budget = std::max(max_budget, s.budget);
    max_budget = std::min<int64_t>(max_budget, all_px * 4);
    max_budget = std::max<int64_t>(max_budget, max_px * 4);
    ctx->total = NT;
    ctx->done = 0;
    // tuned shape for this workload
    char keybuf[160];
    snprintf(keybuf, sizeof(keybuf), "%d:%d:%d:%d:%d:%lld", (int)sizeof(T), c.R, c.kd, c.circle, p.doughnut_correction,
             (long long)max_px);
    const std::string tkey = keybuf;
    auto tuned = ctx->rg_best.find(tkey);
    // the tables
    int64_t max_tasks = 0;
    for (const auto& s : kRaggedShapes) {
        // a wave's tiles: per frame ceil(W/TW) strips x ceil(H/seg) segments, at most
        int64_t m = 0;
        for (int32_t v = 0; v < nv; v++)
            m = std::max<int64_t>(m, (int64_t)((W_[v] + TW - 1) / TW) * ((H_[v] + s.seg - 1) / s.seg));
        max_tasks = std::max<int64_t>(max_tasks, m * kRaggedSlots);
    }
    const int grid = ctx->num_sms * strip_blocks_per_sm<T>(c);
    // angle and doughnut tables, finalize constants (as locate_pass)
    std::vector<float2> atab;
    std::vector<int32_t> aoff;
    angle_tables(std::max(0, (c.circle - 1) / 2), atab, aoff);
    std::vector<short2> dn;
    std::vector<int4> dmeta;
    doughnut_tables(p, std::vector<float>{(float)p.diameter / 2.0f}, dn, dmeta);
    FinalizeConsts fc;
    std::memset(&fc, 0, sizeof(fc));
    fc.H = (int32_t)0;
    fc.W = (int32_t)0;
    fc.filter_close = p.filter_close ? 1 : 0;
    fc.separation = (float)p.separation;
    {
        int rint = std::max(0, (c.circle - 1) / 2);
        long long band = (long long)std::ceil(fc.separation) + 2LL * ((long long)c.max_iter + rint) + 2;
        fc.band = (c.truncate && band < (1LL << 30)) ? (int32_t)band : -1;
    }
    fc.doughnut = p.doughnut_correction ? 1 : 0;
    for (int attempt = 0;; attempt++) {
        const uint32_t cand_cap = ctx->cand_cap, feat_cap = ctx->feat_cap;
        size_t fin_per_frame = 0;
        if (feat_cap > (uint32_t)kFinalizeSmemSort) {
            size_t np2 = 1;
            while (np2 < feat_cap) np2 <<= 1;
            fin_per_frame = (np2 * 17 + 255) & ~(size_t)255;
        }
        fc.scratch_per_frame = fin_per_frame;
        CK(ctx->processed.ensure((size_t)max_budget));
        CK(ctx->cand_count.ensure((size_t)kRaggedSlots * 4));
        CK(ctx->cand_keys.ensure((size_t)kRaggedSlots * cand_cap * 4));
        CK(ctx->feats_raw.ensure((size_t)kRaggedSlots * feat_cap * sizeof(Feature)));
        CK(ctx->feat_count.ensure((size_t)kRaggedSlots * 4));
        // one more result slot: the padding frames of a short wave write there
        CK(ctx->feats_out.ensure((size_t)(NT + 1) * feat_cap * sizeof(Feature)));
        CK(ctx->kept_count.ensure((size_t)(NT + 1) * 4));
        CK(ctx->flags.ensure(16));
        CK(ctx->walk_starts.ensure(8));
        CK(ctx->fin_scratch.ensure(std::max<size_t>(fin_per_frame * kRaggedSlots, 256)));
        CK(ctx->rg_frames.ensure((size_t)kRaggedSlots * sizeof(RaggedFrame)));
        CK(ctx->rg_tasks.ensure((size_t)std::max<int64_t>(max_tasks, 1) * sizeof(StripTask)));
        CK(ctx->rg_ntasks.ensure(4));
        {
            std::vector<int32_t> ident(kRaggedSlots);
            for (int i = 0; i < kRaggedSlots; i++) ident[i] = i;
            CKS(upload(ctx, ctx->ident, ident));
        }
        CKS(upload(ctx, ctx->tabs_f, atab));
        CKS(upload(ctx, ctx->tabs_i, aoff));
        CKS(upload(ctx, ctx->tabs_s, dn));
        CKS(upload(ctx, ctx->tabs_m, dmeta));
        CK(cudaMemsetAsync(ctx->flags.p, 0, 16, ctx->st));
        CK(cudaMemsetAsync(ctx->walk_starts.p, 0, 8, ctx->st));
        bool any_host = false;
        for (int32_t v = 0; v < nv; v++) any_host |= !on_device[v];
        if (any_host) {
            CK(ctx->stage[0].ensure((size_t)max_budget / 4 * sizeof(T)));
            CK(ctx->stage[1].ensure((size_t)max_budget / 4 * sizeof(T)));
        }
        RaggedFrame* d_frames = ctx->rg_frames.as<RaggedFrame>();
        StripTask* d_tasks = ctx->rg_tasks.as<StripTask>();
        int32_t* d_ntasks = ctx->rg_ntasks.as<int32_t>();
        float* proc = ctx->processed.as<float>();
        uint32_t* flags = ctx->flags.as<uint32_t>();

        // ---- the stage sequence of one wave (captured once, then replayed;
        // a profiled call launches it directly, timing every stage)
        auto stages = [&](cudaStream_t st, bool timed) -> gt_status {
            std::unique_ptr<Prof> pf;
            auto stage = [&](const char* name) {
                pf.reset();
                if (timed) pf.reset(new Prof(ctx, name, st));
            };
            CK(cudaMemsetAsync(ctx->cand_count.p, 0, (size_t)kRaggedSlots * 4, st));
            CK(cudaMemsetAsync(ctx->feat_count.p, 0, (size_t)kRaggedSlots * 4, st));
            cudaError_t e = cudaSuccess;
            stage("bandpass_localmax");
            if (!launch_strip_ragged<T>(d_frames, d_tasks, d_ntasks, grid, proc, c, ctx->cand_count.as<uint32_t>(),
                                        ctx->cand_keys.as<uint32_t>(), cand_cap, flags, st, &e))
                return set_err(ctx, GT_ERR_INTERNAL, "no strip kernel for this parameter set");
            CK(e);
            stage("walk_characterize");
            sum_counts_kernel<<<1, 256, 0, st>>>(ctx->cand_count.as<uint32_t>(), kRaggedSlots, cand_cap,
                                                 ctx->walk_starts.as<unsigned long long>());
            CK(cudaGetLastError());
            CK(launch_walk<T>(proc, (const T*)nullptr, 0, c, kRaggedSlots, 1, ctx->cand_count.as<uint32_t>(),
                              ctx->cand_keys.as<uint32_t>(), cand_cap, cand_cap, nullptr, ctx->tabs_i.as<int32_t>(),
                              ctx->tabs_f.as<float2>(), ctx->feats_raw.as<Feature>(), ctx->feat_count.as<uint32_t>(),
                              feat_cap, flags, st, d_frames));
            stage("finalize");
            CK(launch_finalize<T>(ctx->feats_raw.as<Feature>(), ctx->feat_count.as<uint32_t>(), feat_cap,
                                  ctx->feats_out.as<Feature>(), ctx->kept_count.as<uint32_t>(),
                                  ctx->fin_scratch.as<uint8_t>(), fc, (const T*)nullptr, 0, ctx->ident.as<int32_t>(),
                                  ctx->tabs_s.as<short2>(), ctx->tabs_m.as<int4>(), flags, kRaggedSlots, st,
                                  d_frames));
            return GT_OK;
        };
        // the graph names these buffers and sizes; a call that moved any of
        // them captures a new one
        char gk[512];
        snprintf(gk, sizeof(gk), "%p %p %p %p %p %p %p %p %p %p %p %p %p %p %p %u %u %d %d %d %d %d", (void*)d_frames,
                 (void*)d_tasks, (void*)d_ntasks, (void*)proc, ctx->cand_count.p, ctx->cand_keys.p, ctx->feats_raw.p,
                 ctx->feat_count.p, ctx->feats_out.p, ctx->kept_count.p, ctx->fin_scratch.p, ctx->tabs_f.p,
                 ctx->tabs_s.p, ctx->walk_starts.p, (void*)flags, cand_cap, feat_cap, (int)sizeof(T), c.R, c.kd,
                 c.circle, grid);
        std::string gkey = std::string(gk) + ":" + std::string((const char*)&c, sizeof(c)) +
                           std::string((const char*)&fc, sizeof(fc));
        if (ctx->rg_graph && ctx->rg_graph_key != gkey) {
            cudaGraphExecDestroy(ctx->rg_graph);
            ctx->rg_graph = nullptr;
        }
        if (!ctx->rg_graph) {
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal));
            gt_status sst = stages(ctx->st, false);
            cudaError_t ee = cudaStreamEndCapture(ctx->st, &g);
            if (sst != GT_OK) {
                if (g) cudaGraphDestroy(g);
                return sst;
            }
            CK(ee);
            cudaError_t ei = cudaGraphInstantiate(&ctx->rg_graph, g, 0);
            cudaGraphDestroy(g);
            CK(ei);
            ctx->rg_graph_key = gkey;
        }

        // ---- waves
        int64_t cur = 0;     // next slot of the call
        int shape_i = -1;    // tuning: index of the shape being timed
        std::vector<double> shape_ms(kRaggedNShapes, 0.0), shape_px(kRaggedNShapes, 0.0);
        RaggedShape shape = kRaggedShapes[0];
        if (tuned != ctx->rg_best.end()) shape = RaggedShape{tuned->second.first, tuned->second.second};
        // tune when the call has waves to spare and no shape is known yet
        int64_t tot_px = 0;
        for (int32_t v = 0; v < nv; v++) tot_px += T_[v] * (int64_t)H_[v] * W_[v];
        const bool tune = tuned == ctx->rg_best.end() &&
                          (ctx->rg_force_tune || tot_px * 4 >= 2 * kRaggedNShapes * (1LL << 30));
        if (tune) shape_i = 0;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (tune) {
            CK(cudaEventCreate(&e0));
            CK(cudaEventCreate(&e1));
        }
        std::vector<RaggedSlot> wave;
        std::vector<RaggedFrame> hf(kRaggedSlots);
        std::vector<StripTask> htask;
        int wave_no = 0;
        auto video_of = [&](int64_t slot) -> int32_t {
            return (int32_t)(std::upper_bound(vslot.begin(), vslot.end(), slot) - vslot.begin() - 1);
        };
        while (cur < NT) {
            if (interrupted(ctx)) {
                cudaStreamSynchronize(ctx->st);
                cudaStreamSynchronize(ctx->cp);
                if (e0) cudaEventDestroy(e0);
                if (e1) cudaEventDestroy(e1);
                return set_err(ctx, GT_ERR_INTERRUPTED, "Keyboard Interrupt, my custom version");
            }
            if (shape_i >= 0) shape = kRaggedShapes[shape_i % kRaggedNShapes];
            // the wave: frames in order while the budget and the slots last
            // (the tuning test hook shrinks the budgets, so that small calls
            // run many waves)
            const int64_t budget = ctx->rg_force_tune ? std::max<int64_t>(shape.budget >> 12, 1) : shape.budget;
            wave.clear();
            int64_t used = 0;
            while (cur < NT && (int)wave.size() < kRaggedSlots) {
                const int32_t v = video_of(cur);
                const int64_t px = (int64_t)H_[v] * W_[v];
                if (!wave.empty() && used + px * 4 > budget) break;
                wave.push_back(RaggedSlot{v, cur - vslot[(size_t)v]});
                used += px * 4;
                cur++;
            }
            // host frames of the wave go to a staging buffer
            const int b = wave_no & 1;
            bool staged = false;
            int64_t soff = 0;
            std::vector<const void*> raw(wave.size());
            for (size_t i = 0; i < wave.size(); i++) {
                const int32_t v = wave[i].video;
                const size_t fb = (size_t)H_[v] * W_[v] * sizeof(T);
                const T* src = (const T*)frames[v] + (size_t)wave[i].t * H_[v] * W_[v];
                if (on_device[v]) {
                    raw[i] = src;
                } else {
                    if (!staged) {
                        CK(cudaStreamWaitEvent(ctx->cp, ctx->used[b], 0));
                        staged = true;
                    }
                    // 16-byte aligned frame starts in the staging buffer
                    soff = (soff + 15) & ~(int64_t)15;
                    uint8_t* dst = ctx->stage[b].as<uint8_t>() + soff;
                    CK(cudaMemcpyAsync(dst, src, fb, cudaMemcpyHostToDevice, ctx->cp));
                    raw[i] = dst;
                    soff += (int64_t)fb;
                }
            }
            if (staged) {
                CK(cudaEventRecord(ctx->filled[b], ctx->cp));
                CK(cudaStreamWaitEvent(ctx->st, ctx->filled[b], 0));
            }
            // frame and tile tables (largest tiles first: the persistent
            // CTAs finish together)
            htask.clear();
            int64_t poff = 0;
            for (int i = 0; i < kRaggedSlots; i++) {
                RaggedFrame& f = hf[(size_t)i];
                if (i < (int)wave.size()) {
                    const int32_t v = wave[(size_t)i].video;
                    f.raw = raw[(size_t)i];
                    f.proc_off = poff;
                    f.H = H_[v];
                    f.W = W_[v];
                    f.vec_ok = (W_[v] % 4 == 0 && ((uintptr_t)raw[(size_t)i] % (4 * sizeof(T))) == 0) ? 1 : 0;
                    f.out_slot = (int32_t)(vslot[(size_t)v] + wave[(size_t)i].t);
                    poff += (int64_t)H_[v] * W_[v];
                    for (int32_t r0 = 0; r0 < H_[v]; r0 += shape.seg)
                        for (int32_t c0 = 0; c0 < W_[v]; c0 += TW)
                            htask.push_back(StripTask{i, c0, r0, std::min(r0 + shape.seg, H_[v])});
                } else {
                    f.raw = nullptr;
                    f.proc_off = 0;
                    f.H = f.W = 0;
                    f.vec_ok = 0;
                    f.out_slot = (int32_t)NT;   // the spare result slot
                }
            }
            std::stable_sort(htask.begin(), htask.end(), [](const StripTask& a, const StripTask& b2) {
                return (a.r1 - a.r0) > (b2.r1 - b2.r0);
            });
            const int32_t ntask = (int32_t)htask.size();
            CK(cudaMemcpyAsync(d_frames, hf.data(), hf.size() * sizeof(RaggedFrame), cudaMemcpyHostToDevice, ctx->st));
            if (ntask > 0)
                CK(cudaMemcpyAsync(d_tasks, htask.data(), htask.size() * sizeof(StripTask), cudaMemcpyHostToDevice,
                                   ctx->st));
            CK(cudaMemcpyAsync(d_ntasks, &ntask, 4, cudaMemcpyHostToDevice, ctx->st));
            if (shape_i >= 0) CK(cudaEventRecord(e0, ctx->st));
            if (ctx->profile) {
                CKS(stages(ctx->st, true));
            } else {
                // the graph's kernels: strip, candidate totals, walk, finalize (+ doughnut)
                ctx->launch_count["ragged_wave"] += fc.doughnut ? 5 : 4;
                CK(cudaGraphLaunch(ctx->rg_graph, ctx->st));
            }
            if (staged) CK(cudaEventRecord(ctx->used[b], ctx->st));
            if (shape_i >= 0) {
                CK(cudaEventRecord(e1, ctx->st));
                CK(cudaEventSynchronize(e1));
                float ms = 0.0f;
                CK(cudaEventElapsedTime(&ms, e0, e1));
                // the first round of shapes warms up; the second one counts
                if (shape_i >= kRaggedNShapes) {
                    shape_ms[(size_t)(shape_i % kRaggedNShapes)] += ms;
                    shape_px[(size_t)(shape_i % kRaggedNShapes)] += (double)used / 4.0;
                }
                shape_i++;
                if (shape_i == 2 * kRaggedNShapes) {
                    int best = 0;
                    for (int k = 1; k < kRaggedNShapes; k++)
                        if (shape_ms[(size_t)k] / shape_px[(size_t)k] < shape_ms[(size_t)best] / shape_px[(size_t)best])
                            best = k;
                    ctx->rg_best[tkey] = {kRaggedShapes[best].seg, kRaggedShapes[best].budget};
                    shape = kRaggedShapes[best];
                    shape_i = -1;
                }
            }
            ctx->done = cur;
            wave_no++;
        }
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        uint32_t fl = 0;
        CK(cudaMemcpyAsync(&fl, flags, 4, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if (!(fl & (kFlagCandOverflow | kFlagFeatOverflow))) break;
        if (attempt > 8) return set_err(ctx, GT_ERR_CAPACITY_EXCEEDED, "per-frame capacity exceeded");
        const uint64_t npx = (uint64_t)max_px;
        if (fl & kFlagCandOverflow) {
            uint64_t ncap = std::min<uint64_t>((uint64_t)ctx->cand_cap * 4, npx + 1);
            if (ncap <= ctx->cand_cap) return set_err(ctx, GT_ERR_CAPACITY_EXCEEDED, "candidate capacity exceeded");
            ctx->cand_cap = (uint32_t)ncap;
        }
        if (fl & kFlagFeatOverflow) {
            uint64_t nf = std::min<uint64_t>((uint64_t)ctx->feat_cap * 4, std::min<uint64_t>(npx + 1, 1u << 24));
            if (nf <= ctx->feat_cap)
                return set_err(ctx, GT_ERR_CAPACITY_EXCEEDED, "per-frame detection capacity exceeded");
            ctx->feat_cap = (uint32_t)nf;
        }
    }
    // ---- per-video tables
    for (int32_t v = 0; v < nv; v++) {
        std::vector<int64_t> fnum((size_t)T_[v]);
        for (int64_t t = 0; t < T_[v]; t++) fnum[(size_t)t] = t;
        HostSpan hs(ctx, "host_assemble");
        CKS(assemble_table(ctx, T_[v], fnum, false, tabs[v], row_off[(size_t)v], vslot[(size_t)v]));
        if (!p.doughnut_correction)
            tabs[v]->has[GT_COL_RAW_MASS] = tabs[v]->has[GT_COL_RAW_BG_MEDIAN] =
                tabs[v]->has[GT_COL_RAW_MASS_CORRECTED] = false;
    }
    CK(cudaStreamSynchronize(ctx->st));
    drain_profile(ctx, false);
    return GT_OK;
}

// Many videos in one call: the videos are located together in ragged waves
// (batch_videos_ragged) where the parameter set allows it, otherwise each
// into its own table as gt_batch would; then every video is linked in ONE
// launch of the whole-video linker (one CTA per video), so the videos'
// sequential frame scans run side by side.  Results equal separate gt_batch
// calls.
template <typename T>
gt_status batch_videos_impl(gt_ctx* ctx, const gt_params& p, int32_t n_videos, const void* const* frames,
                            const int64_t* T_, const int32_t* H_, const int32_t* W_, gt_table** tabs) {
    gt_params pl = p;
    pl.has_search_range = 0;
    std::vector<std::vector<int64_t>> row_off((size_t)n_videos);
    std::unique_ptr<bool[]> on_dev(new bool[(size_t)std::max(n_videos, 1)]);
    for (int32_t v = 0; v < n_videos; v++) {
        on_dev[(size_t)v] = false;
        CKS(check_frames_ptr(ctx, frames[v], (size_t)T_[v] * H_[v] * W_[v] * sizeof(T), &on_dev[(size_t)v]));
    }
    bool ragged = n_videos > 0 && !ctx->no_ragged;
    LocateConsts c;
    if (ragged) {
        int32_t Hm = 0, Wm = 0;
        for (int32_t v = 0; v < n_videos; v++) {
            Hm = std::max(Hm, H_[v]);
            Wm = std::max(Wm, W_[v]);
        }
        CKS(make_locate_consts(ctx, p, Hm, Wm, c));
        set_fast_div<T>(ctx, c);
        ragged = ragged_eligible<T>(p, c);
    }
    if (ragged) {
        HostSpan hs(ctx, "host_locate");
        CKS(batch_videos_ragged<T>(ctx, p, c, n_videos, frames, on_dev.get(), T_, H_, W_, tabs, row_off));
    }
    for (int32_t v = 0; v < n_videos && !ragged; v++) {
        const bool on_device = on_dev[(size_t)v];
        const int64_t NT = T_[v];
        gt_status st = batch_impl<T>(ctx, pl, (const T*)frames[v], on_device, NT, H_[v], W_[v], nullptr, nullptr, 0,
                                     tabs[v]);
        if (st != GT_OK) return st;
        // rows of frame t are [row_off[t], row_off[t+1]) (batch_impl's kept counts)
        std::vector<uint32_t> kept((size_t)NT);
        CK(cudaMemcpyAsync(kept.data(), ctx->kept_count.p, (size_t)NT * 4, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        auto& ro = row_off[(size_t)v];
        ro.assign((size_t)NT + 1, 0);
        for (int64_t t = 0; t < NT; t++) ro[(size_t)t + 1] = ro[(size_t)t] + kept[(size_t)t];
        if (ro.back() != tabs[v]->n) return set_err(ctx, GT_ERR_INTERNAL, "row count mismatch");
    }
    if (!p.has_search_range) return GT_OK;
    LinkJob job;
    job.vgrp.push_back(0);
    job.goff.push_back(0);
    int64_t N = 0;
    for (int32_t v = 0; v < n_videos; v++) {
        const auto& ro = row_off[(size_t)v];
        for (size_t t = 1; t < ro.size(); t++) job.goff.push_back(N + ro[t]);
        N += ro.back();
        job.vgrp.push_back((int32_t)(job.goff.size() - 1));
    }
    job.reset.assign(job.goff.size() - 1, 0);
    job.radius = p.search_range;
    job.memory = (int32_t)p.memory;
    const size_t n1 = (size_t)std::max<int64_t>(N, 1);
    CK(ctx->l_px.ensure(n1 * 4));
    CK(ctx->l_py.ensure(n1 * 4));
    CK(ctx->l_ids.ensure(n1 * 8));
    CK(ctx->l_rowdur.ensure(n1 * 8));
    float* px = ctx->l_px.as<float>();
    float* py = ctx->l_py.as<float>();
    int64_t base = 0;
    for (int32_t v = 0; v < n_videos; v++) {
        const int64_t n = tabs[v]->n;
        if (n > 0) {
            CK(cudaMemcpyAsync(px + base, tabs[v]->col[GT_COL_Y].p, (size_t)n * 4, cudaMemcpyDeviceToDevice, ctx->st));
            CK(cudaMemcpyAsync(py + base, tabs[v]->col[GT_COL_X].p, (size_t)n * 4, cudaMemcpyDeviceToDevice, ctx->st));
        }
        base += n;
    }
    {
        HostSpan hs(ctx, "host_link");
        CKS(run_link(ctx, job, px, py, ctx->l_ids.as<int64_t>(), ctx->l_rowdur.as<int64_t>(), nullptr, nullptr));
    }
    base = 0;
    for (int32_t v = 0; v < n_videos; v++) {
        gt_table* tab = tabs[v];
        const int64_t n = tab->n;
        const size_t m = (size_t)std::max<int64_t>(n, 1);
        CK(tab->particle.ensure(m * 8));
        CK(tab->duration.ensure(m * 8));
        if (n > 0) {
            CK(launch_round_ids(ctx->l_ids.as<int64_t>() + base, tab->particle.as<int64_t>(), n, ctx->st));
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(tab->duration.p, ctx->l_rowdur.as<int64_t>() + base, (size_t)n * 8,
                               cudaMemcpyDeviceToDevice, ctx->st));
        }
        tab->has[GT_COL_PARTICLE] = true;
        tab->has[GT_COL_DURATION] = true;
        base += n;
    }
    CK(cudaStreamSynchronize(ctx->st));
    return GT_OK;
}

// Fills the shared memory of every resident CTA slot with hashed non-zero
// words: what a kernel finds in shared memory it has not written depends on
// the kernels that ran before it, and this makes that content adversarial.
__global__ void scribble_shared_kernel(uint32_t seed, int nwords) {
    extern __shared__ uint32_t sw[];
    for (int i = threadIdx.x; i < nwords; i += blockDim.x)
        sw[i] = (seed ^ ((uint32_t)i * 2654435761u) ^ (blockIdx.x * 40503u)) | 0x00800000u;
}

}  // namespace

// =================================================================== C ABI
extern "C" {

// internal accessors for the other translation units (not exported)
int gt__ctx_device(const gt_ctx* ctx) { return ctx->device; }
// GT_OK when `bytes` bytes from device pointer p lie inside the allocation
// that holds p (cuMemGetAddressRange), or when the driver cannot tell;
// GT_ERR_INVALID_ARGUMENT, with the context's message set, when they run past it.
gt_status gt__device_span_check(gt_ctx* ctx, const void* p, size_t bytes, const char* what) {
    CUdeviceptr base = 0;
    size_t size = 0;
    AddressRangeFn fn = address_range_fn();
    if (!fn || fn(&base, &size, (CUdeviceptr)p) != CUDA_SUCCESS) {
        cudaGetLastError();
        return GT_OK;
    }
    const uint64_t off = (uint64_t)(uintptr_t)p - (uint64_t)base;
    if (off > size || bytes > size - off)
        return set_err(ctx, GT_ERR_INVALID_ARGUMENT,
                       "%s: %zu bytes from the pointer run past the end of its allocation (%zu bytes left)", what,
                       bytes, (size_t)(size - std::min<uint64_t>(off, size)));
    return GT_OK;
}
cudaStream_t gt__ctx_stream(const gt_ctx* ctx) { return ctx->st; }
void gt__ctx_set_error(gt_ctx* ctx, const char* msg) { ctx->err = msg; }

// Test hook (exported, not part of the public header): the entries of each
// windowed-linking neighbour-list buffer and the backward edges per frame its
// scratch holds; values <= 0 restore the defaults.  Small values make gt_batch
// take its fallback to the whole-video linker.
GT_API gt_status gt__set_link_window_caps(gt_ctx* ctx, int64_t list_entries, int64_t edges_per_frame) {
    if (!ctx) return GT_ERR_INVALID_ARGUMENT;
    ctx->w_list_cap = list_entries;
    ctx->w_edge_cap = edges_per_frame;
    return GT_OK;
}

// Test hook (exported, not part of the public header): the per-frame
// candidate and detection capacities the next gt_batch starts from (values
// <= 0 keep the current ones).  Small values make the kernels report overflow
// and the call replay with grown capacities, the path that replaces the
// reference's silent truncation (src/gpu_setup.rs:246-253).
GT_API gt_status gt__set_capacities(gt_ctx* ctx, int64_t cand_cap, int64_t feat_cap) {
    if (!ctx) return GT_ERR_INVALID_ARGUMENT;
    if (cand_cap > 0) ctx->cand_cap = (uint32_t)std::min<int64_t>(cand_cap, 1LL << 30);
    if (feat_cap > 0) ctx->feat_cap = (uint32_t)std::min<int64_t>(feat_cap, 1LL << 24);
    return GT_OK;
}

// Test hook: gt_batch_videos locates video by video (ragged = 0) or in
// ragged waves where the parameters allow (ragged = 1, the default; 2: the
// autotuner runs on every call, however small).  The tuned wave shapes are
// forgotten, so the next call tunes again.
GT_API gt_status gt__set_ragged(gt_ctx* ctx, int32_t ragged) {
    if (!ctx) return GT_ERR_INVALID_ARGUMENT;
    ctx->no_ragged = ragged == 0;
    ctx->rg_force_tune = ragged == 2;
    ctx->rg_best.clear();
    return GT_OK;
}

// Test hook: the wave shape the autotuner chose for the last ragged call
// (0, 0 when none was tuned).
GT_API gt_status gt__ragged_shape(const gt_ctx* ctx, int32_t* seg, int64_t* budget) {
    if (!ctx) return GT_ERR_INVALID_ARGUMENT;
    *seg = 0;
    *budget = 0;
    for (const auto& kv : ctx->rg_best) {
        *seg = kv.second.first;
        *budget = kv.second.second;
    }
    return GT_OK;
}

// Test hook: the capacities the last call ended with.
GT_API gt_status gt__get_capacities(const gt_ctx* ctx, int64_t* cand_cap, int64_t* feat_cap) {
    if (!ctx) return GT_ERR_INVALID_ARGUMENT;
    if (cand_cap) *cand_cap = ctx->cand_cap;
    if (feat_cap) *feat_cap = ctx->feat_cap;
    return GT_OK;
}

// Test hook (exported, not part of the public header): overwrite the shared
// memory of every SM with non-zero words on the context's stream, so that a
// following call shows any dependence on shared memory it did not write.
GT_API gt_status gt__scribble_shared_memory(gt_ctx* ctx, uint32_t seed) {
    if (!ctx) return GT_ERR_INVALID_ARGUMENT;
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, ctx->device));
    const int bytes = (int)prop.sharedMemPerBlockOptin;
    CK(cudaFuncSetAttribute(scribble_shared_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    scribble_shared_kernel<<<prop.multiProcessorCount * 4, 1024, bytes, ctx->st>>>(seed, bytes / 4);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    return GT_OK;
}

const char* gt_version(void) { return "gpu_tracking_b200 0.1 (sm_100a)"; }

void gt_params_default(gt_params* p) {
    std::memset(p, 0, sizeof(*p));
    // TrackingParams::default() (src/gpu_setup.rs:61-97)
    p->style = GT_STYLE_TRACKPY;
    p->diameter = 9;
    p->separation = 10;
    p->filter_close = 1;
    p->max_iterations = 10;
    p->minmass = 0.0f;
    p->characterize = 0;
    p->doughnut_correction = 0;
    p->truncate_preprocessed = 1;
    p->shift_threshold = 0.6f;
    p->noise_size = 1.0f;
    p->n_radii = 10;
}

// The linker runs one frame after another in one CTA beside the locate
// kernels; its stream gets the device's highest priority so that its CTAs are
// placed before further locate CTAs whenever an SM frees up.
static int link_stream_priority() {
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return greatest;
}

gt_status gt_create(int32_t device, gt_ctx** out) {
    if (!out) return GT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return GT_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) return GT_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return GT_ERR_NO_DEVICE;
    gt_ctx* ctx = new gt_ctx();
    ctx->device = device;
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->cp, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ctx->lk, cudaStreamNonBlocking, link_stream_priority()) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ctx->ls, cudaStreamNonBlocking, link_stream_priority()) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->located, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->linked, cudaEventDisableTiming) != cudaSuccess) {
        delete ctx;
        return GT_ERR_CUDA;
    }
    for (int i = 0; i < 2; i++) {
        if (cudaEventCreateWithFlags(&ctx->used[i], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ctx->filled[i], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ctx->listed[i], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ctx->w_linked[i], cudaEventDisableTiming) != cudaSuccess) {
            gt_destroy(ctx);
            return GT_ERR_CUDA;
        }
    }
    *out = ctx;
    return GT_OK;
}

void gt_destroy(gt_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->st);
    cudaStreamSynchronize(ctx->cp);
    sync_link_streams(ctx);
    drain_profile(ctx);
    for (auto e : ctx->event_pool) cudaEventDestroy(e);
    for (int i = 0; i < 2; i++) {
        if (ctx->used[i]) cudaEventDestroy(ctx->used[i]);
        if (ctx->filled[i]) cudaEventDestroy(ctx->filled[i]);
        if (ctx->listed[i]) cudaEventDestroy(ctx->listed[i]);
        if (ctx->w_linked[i]) cudaEventDestroy(ctx->w_linked[i]);
    }
    if (ctx->rg_graph) cudaGraphExecDestroy(ctx->rg_graph);
    cudaEventDestroy(ctx->located);
    cudaEventDestroy(ctx->linked);
    cudaStreamDestroy(ctx->st);
    cudaStreamDestroy(ctx->cp);
    cudaStreamDestroy(ctx->lk);
    cudaStreamDestroy(ctx->ls);
    delete ctx;
}

const char* gt_last_error(const gt_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

gt_status gt_set_interrupt(gt_ctx* ctx, const volatile int32_t* flag) {
    if (!ctx) return GT_ERR_INVALID_ARGUMENT;
    ctx->interrupt = flag;
    return GT_OK;
}

gt_status gt_progress(const gt_ctx* ctx, int64_t* done, int64_t* total) {
    if (!ctx) return GT_ERR_INVALID_ARGUMENT;
    if (done) *done = ctx->done.load();
    if (total) *total = ctx->total.load();
    return GT_OK;
}


gt_status gt_batch(gt_ctx* ctx, const gt_params* params, const void* frames, int32_t dtype, int64_t T, int32_t H,
                   int32_t W, const int64_t* frame_numbers, const int64_t* linker_reset_points, int64_t n_reset,
                   gt_table** out) {
    if (!out) return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "null output");
    *out = nullptr;
    CKS(validate(ctx, params, frames, dtype, T, H, W));
    bool on_device = false;
    CKS(check_frames_ptr(ctx, frames, (size_t)T * H * W * dtype_bytes(dtype), &on_device));
    std::unique_ptr<gt_table> tab(new gt_table(ctx->device, ctx->st));
    gt_status st;
    if (dtype == GT_DTYPE_U16)
        st = batch_impl<uint16_t>(ctx, *params, (const uint16_t*)frames, on_device, T, H, W, frame_numbers,
                                  linker_reset_points, n_reset, tab.get());
    else if (dtype == GT_DTYPE_F32)
        st = batch_impl<float>(ctx, *params, (const float*)frames, on_device, T, H, W, frame_numbers,
                               linker_reset_points, n_reset, tab.get());
    else
        st = batch_impl<uint8_t>(ctx, *params, (const uint8_t*)frames, on_device, T, H, W, frame_numbers,
                                 linker_reset_points, n_reset, tab.get());
    if (st != GT_OK) {
        // no kernel may still write the table when its columns go back to the pool
        cudaStreamSynchronize(ctx->st);
        sync_link_streams(ctx);
        return st;
    }
    *out = tab.release();
    return GT_OK;
}

gt_status gt_batch_learned(gt_ctx* ctx, const gt_params* params, const gt_proposal* net, const void* frames,
                           int32_t dtype, int64_t T, int32_t H, int32_t W, const int64_t* frame_numbers,
                           const int64_t* linker_reset_points, int64_t n_reset, gt_table** out) {
    if (!out || !net) return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    CKS(validate(ctx, params, frames, dtype, T, H, W));
    if (net->device != ctx->device)
        return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "the network lives on device %d, the context on %d", net->device,
                       ctx->device);
    if (params->style != GT_STYLE_TRACKPY)
        return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "learned proposals replace the trackpy-style local maxima");
    if (params->has_snr || params->has_minmass_snr || params->has_adaptive_background ||
        params->has_illumination_sigma)
        return set_err(ctx, GT_ERR_INVALID_ARGUMENT,
                       "snr, minmass_snr, adaptive_background and illumination correction are not supported with "
                       "learned proposals");
    bool on_device = false;
    CKS(check_frames_ptr(ctx, frames, (size_t)T * H * W * dtype_bytes(dtype), &on_device));
    std::unique_ptr<gt_table> tab(new gt_table(ctx->device, ctx->st));
    gt_status st;
    if (dtype == GT_DTYPE_U16)
        st = batch_impl<uint16_t>(ctx, *params, (const uint16_t*)frames, on_device, T, H, W, frame_numbers,
                                  linker_reset_points, n_reset, tab.get(), net);
    else if (dtype == GT_DTYPE_F32)
        st = batch_impl<float>(ctx, *params, (const float*)frames, on_device, T, H, W, frame_numbers,
                               linker_reset_points, n_reset, tab.get(), net);
    else
        st = batch_impl<uint8_t>(ctx, *params, (const uint8_t*)frames, on_device, T, H, W, frame_numbers,
                                 linker_reset_points, n_reset, tab.get(), net);
    if (st != GT_OK) {
        cudaStreamSynchronize(ctx->st);
        sync_link_streams(ctx);
        return st;
    }
    *out = tab.release();
    return GT_OK;
}

int64_t gt_last_walk_starts(const gt_ctx* ctx) { return ctx ? ctx->last_walk_starts : 0; }

gt_status gt_batch_videos(gt_ctx* ctx, const gt_params* params, int32_t n_videos, const void* const* frames,
                          int32_t dtype, const int64_t* T, const int32_t* H, const int32_t* W, gt_table** out) {
    if (!out || !frames || !T || !H || !W || n_videos < 0) return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "null argument");
    for (int32_t v = 0; v < n_videos; v++) out[v] = nullptr;
    for (int32_t v = 0; v < n_videos; v++) CKS(validate(ctx, params, frames[v], dtype, T[v], H[v], W[v]));
    std::vector<std::unique_ptr<gt_table>> tabs((size_t)n_videos);
    std::vector<gt_table*> raw((size_t)n_videos);
    for (int32_t v = 0; v < n_videos; v++) {
        tabs[(size_t)v].reset(new gt_table(ctx->device, ctx->st));
        raw[(size_t)v] = tabs[(size_t)v].get();
    }
    gt_status st;
    if (dtype == GT_DTYPE_U16)
        st = batch_videos_impl<uint16_t>(ctx, *params, n_videos, frames, T, H, W, raw.data());
    else if (dtype == GT_DTYPE_F32)
        st = batch_videos_impl<float>(ctx, *params, n_videos, frames, T, H, W, raw.data());
    else
        st = batch_videos_impl<uint8_t>(ctx, *params, n_videos, frames, T, H, W, raw.data());
    if (st != GT_OK) {
        cudaStreamSynchronize(ctx->st);
        sync_link_streams(ctx);
        return st;
    }
    for (int32_t v = 0; v < n_videos; v++) out[v] = tabs[(size_t)v].release();
    return GT_OK;
}

gt_status gt_characterize_points(gt_ctx* ctx, const gt_params* params, const void* frames, int32_t dtype, int64_t T,
                                 int32_t H, int32_t W, const float* points, int64_t n_points, int32_t has_frames,
                                 int32_t has_r, gt_table** out) {
    if (!out) return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "null output");
    *out = nullptr;
    CKS(validate(ctx, params, frames, dtype, T, H, W));
    if (n_points > 0 && !points) return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "null points");
    bool on_device = false;
    CKS(check_frames_ptr(ctx, frames, (size_t)T * H * W * dtype_bytes(dtype), &on_device));
    std::unique_ptr<gt_table> tab(new gt_table(ctx->device, ctx->st));
    gt_status st;
    if (dtype == GT_DTYPE_U16)
        st = charpoints_impl<uint16_t>(ctx, *params, (const uint16_t*)frames, on_device, T, H, W, points, n_points,
                                       has_frames, has_r, tab.get());
    else if (dtype == GT_DTYPE_F32)
        st = charpoints_impl<float>(ctx, *params, (const float*)frames, on_device, T, H, W, points, n_points,
                                    has_frames, has_r, tab.get());
    else
        st = charpoints_impl<uint8_t>(ctx, *params, (const uint8_t*)frames, on_device, T, H, W, points, n_points,
                                      has_frames, has_r, tab.get());
    if (st != GT_OK) {
        // no kernel may still write the table when its columns go back to the pool
        cudaStreamSynchronize(ctx->st);
        sync_link_streams(ctx);
        return st;
    }
    *out = tab.release();
    return GT_OK;
}

gt_status gt_mean_frame(gt_ctx* ctx, const void* frames, int32_t dtype, int64_t T, int32_t H, int32_t W,
                        float* out) {
    gt_params p;
    gt_params_default(&p);
    CKS(validate(ctx, &p, frames, dtype, T, H, W));
    if (!out) return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "null output");
    bool on_device = false;
    CKS(check_frames_ptr(ctx, frames, (size_t)T * H * W * dtype_bytes(dtype), &on_device));
    if (dtype == GT_DTYPE_U16) return mean_impl<uint16_t>(ctx, (const uint16_t*)frames, on_device, T, H, W, out);
    if (dtype == GT_DTYPE_F32) return mean_impl<float>(ctx, (const float*)frames, on_device, T, H, W, out);
    return mean_impl<uint8_t>(ctx, (const uint8_t*)frames, on_device, T, H, W, out);
}

// Per-kernel CUDA-event timing on the compute stream (diagnostics; no
// counterpart in the reference).  name_out receives a comma-separated list.
gt_status gt_profile_enable(gt_ctx* ctx, int32_t enable) {
    if (!ctx) return GT_ERR_INVALID_ARGUMENT;
    ctx->profile = enable != 0;
    ctx->stats.clear();
    ctx->launch_count.clear();
    return GT_OK;
}

gt_status gt_profile_read(gt_ctx* ctx, const char* name, int64_t* launches, double* total_ms) {
    if (!ctx || !name) return GT_ERR_INVALID_ARGUMENT;
    drain_profile(ctx);
    auto it = ctx->stats.find(name);
    if (it == ctx->stats.end()) {
        if (launches) *launches = 0;
        if (total_ms) *total_ms = 0.0;
        return GT_OK;
    }
    if (launches) *launches = it->second.launches;
    if (total_ms) *total_ms = it->second.ms;
    return GT_OK;
}

int64_t gt_launch_count(gt_ctx* ctx) {
    if (!ctx) return 0;
    int64_t n = 0;
    for (auto& kv : ctx->launch_count) n += kv.second;
    return n;
}

}  // extern "C"
