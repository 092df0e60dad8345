// gt_linkdrv.cu — the linking calls of the C ABI and the whole-video link
// driver they share with gt_batch: gt_link (link_rust -> linker_all,
// src/linking.rs:818-831) and gt_connect (connect_rust -> connect_all,
// src/linking.rs:960-1020) group their rows by frame on the host
// (FrameSubsetter, src/linking.rs:97-196) and run the device linker
// (gt_link.cu) once over all groups.
#include <cub/device/device_scan.cuh>

#include <memory>

#include "gt_runtime.cuh"

using namespace gt;
using namespace gt::rt;

namespace gt {
namespace rt {

// pgroup[i] = g for the points i of group g (goff: group offsets)
__global__ void fill_pgroup_kernel(const int64_t* __restrict__ goff, int ngroups, int32_t* __restrict__ pgroup) {
    for (int g = blockIdx.x; g < ngroups; g += gridDim.x)
        for (int64_t i = goff[g] + threadIdx.x; i < goff[g + 1]; i += blockDim.x) pgroup[i] = g;
}

// out[g] = boff[goff[g] * K], g = 0..ngroups: where each group's backward lists start
__global__ void group_list_starts_kernel(const int64_t* __restrict__ boff, const int64_t* __restrict__ goff, int K,
                                         int ngroups, int64_t* __restrict__ out) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g <= ngroups) out[g] = boff[goff[g] * K];
}

// Runs the linker over px/py (device, npoints) and writes ids (device) and,
// when row_dur is given, per-row durations and f32-rounded particle ids.
gt_status run_link(gt_ctx* ctx, const LinkJob& job, const float* px, const float* py, int64_t* ids_out,
                   int64_t* row_dur, int64_t* row_particle, std::vector<int64_t>* counters) {
    const int ngroups = (int)job.goff.size() - 1;
    const int nvideos = (int)job.vgrp.size() - 1;
    const int64_t N = job.goff.back();
    const int K = job.memory + 1;
    std::unique_ptr<HostSpan> hs(new HostSpan(ctx, "host_link_prep"));
    int max_group = 0;
    for (int g = 0; g < ngroups; g++) max_group = std::max<int64_t>(max_group, job.goff[g + 1] - job.goff[g]);
    CKS(upload(ctx, ctx->l_goff, job.goff));
    CK(ctx->l_pgroup.ensure((size_t)std::max<int64_t>(N, 1) * 4));
    if (N > 0 && ngroups > 0) {
        fill_pgroup_kernel<<<std::min(ngroups, 4 * ctx->num_sms), 256, 0, ctx->st>>>(
            ctx->l_goff.as<int64_t>(), ngroups, ctx->l_pgroup.as<int32_t>());
        CK(cudaGetLastError());
    }
    CKS(upload(ctx, ctx->l_vgrp, job.vgrp));
    CKS(upload(ctx, ctx->l_reset, job.reset));
    LinkInput in;
    in.px = px;
    in.py = py;
    in.goff = ctx->l_goff.as<int64_t>();
    in.pgroup = ctx->l_pgroup.as<int32_t>();
    in.vgrp = ctx->l_vgrp.as<int32_t>();
    in.reset = ctx->l_reset.as<uint8_t>();
    in.ngroups = ngroups;
    in.nvideos = nvideos;
    in.npoints = N;
    in.radius = job.radius;
    in.memory = job.memory;

    int np2 = 1;
    while (np2 < max_group) np2 <<= 1;
    size_t per_group = (np2 > 4096) ? (size_t)np2 * 8 : 0;
    CK(ctx->l_srt.ensure(std::max<int64_t>(N, 1) * 4));
    CK(ctx->l_sortscr.ensure(std::max<size_t>(per_group * ngroups, 8)));
    {
        Prof pf(ctx, "link_sort");
        CK(link_sort_groups(in, ctx->l_srt.as<uint32_t>(), ctx->l_sortscr.as<uint8_t>(), per_group, max_group,
                            ctx->st));
    }
    const size_t NK = (size_t)N * K;
    CK(ctx->l_fcnt.ensure((NK + 1) * 8));
    CK(ctx->l_bcnt.ensure((NK + 1) * 8));
    CK(ctx->l_foff.ensure((NK + 1) * 8));
    CK(ctx->l_boff.ensure((NK + 1) * 8));
    CK(cudaMemsetAsync(ctx->l_fcnt.p, 0, (NK + 1) * 8, ctx->st));
    CK(cudaMemsetAsync(ctx->l_bcnt.p, 0, (NK + 1) * 8, ctx->st));
    {
        Prof pf(ctx, "link_lists");
        CK(link_count_lists(in, ctx->l_srt.as<uint32_t>(), ctx->l_fcnt.as<int64_t>(), ctx->l_bcnt.as<int64_t>(),
                            ctx->st));
    }
    size_t tmp_bytes = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, ctx->l_fcnt.as<int64_t>(), ctx->l_foff.as<int64_t>(),
                                     (int64_t)NK + 1, ctx->st));
    CK(ctx->l_scan.ensure(tmp_bytes));
    CK(cub::DeviceScan::ExclusiveSum(ctx->l_scan.p, tmp_bytes, ctx->l_fcnt.as<int64_t>(), ctx->l_foff.as<int64_t>(),
                                     (int64_t)NK + 1, ctx->st));
    CK(cub::DeviceScan::ExclusiveSum(ctx->l_scan.p, tmp_bytes, ctx->l_bcnt.as<int64_t>(), ctx->l_boff.as<int64_t>(),
                                     (int64_t)NK + 1, ctx->st));
    hs.reset(new HostSpan(ctx, "host_link_counts"));
    int64_t ftot = 0, btot = 0;
    CK(cudaMemcpyAsync(&ftot, ctx->l_foff.as<int64_t>() + NK, 8, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(&btot, ctx->l_boff.as<int64_t>() + NK, 8, cudaMemcpyDeviceToHost, ctx->st));
    // per-group backward-edge totals bound the per-frame edge list
    std::vector<int64_t> boff_at(ngroups + 1);
    CK(ctx->l_ge.ensure((size_t)(ngroups + 1) * 8));
    group_list_starts_kernel<<<(ngroups + 256) / 256, 256, 0, ctx->st>>>(
        ctx->l_boff.as<int64_t>(), ctx->l_goff.as<int64_t>(), K, ngroups, ctx->l_ge.as<int64_t>());
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(boff_at.data(), ctx->l_ge.p, (size_t)(ngroups + 1) * 8, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    hs.reset(new HostSpan(ctx, "host_link_run"));
    int64_t max_edges = 1;
    for (int g = 0; g < ngroups; g++) max_edges = std::max(max_edges, boff_at[g + 1] - boff_at[g]);
    CK(ctx->l_fpts.ensure(std::max<int64_t>(ftot, 1) * 4));
    CK(ctx->l_bpts.ensure(std::max<int64_t>(btot, 1) * 4));
    CK(ctx->l_bdist.ensure(std::max<int64_t>(btot, 1) * 4));
    LinkLists L;
    L.f_off = ctx->l_foff.as<int64_t>();
    L.b_off = ctx->l_boff.as<int64_t>();
    L.f_pts = ctx->l_fpts.as<int32_t>();
    L.b_pts = ctx->l_bpts.as<int32_t>();
    L.b_dist = ctx->l_bdist.as<float>();
    L.srt = ctx->l_srt.as<uint32_t>();
    L.f_entries = ftot;
    {
        Prof pf(ctx, "link_lists");
        CK(link_fill_lists(in, L, ctx->st));
    }
    // scratch per video
    int64_t max_np = 1;
    for (int v = 0; v < nvideos; v++) max_np = std::max(max_np, job.goff[job.vgrp[v + 1]] - job.goff[job.vgrp[v]]);
    LinkScratch S;
    S.max_group = std::max(max_group, 1);
    S.max_edges = max_edges;
    S.bytes_per_video = link_scratch_bytes(S.max_group, S.max_edges, max_np, job.memory);
    S.max_points = max_np;
    CK(ctx->l_scratch.ensure(S.bytes_per_video * nvideos));
    S.base = ctx->l_scratch.as<uint8_t>();
    LinkOutput out;
    CK(ctx->l_cnt.ensure(nvideos * 8));
    CK(ctx->l_dur.ensure(std::max<int64_t>(N, 1) * 8));
    CK(ctx->l_flags.ensure(nvideos * 4));
    CK(cudaMemsetAsync(ctx->l_flags.p, 0, nvideos * 4, ctx->st));
    out.ids = ids_out;
    out.counter = ctx->l_cnt.as<int64_t>();
    out.dur = ctx->l_dur.as<int64_t>();
    out.vpoff = nullptr;
    out.flags = ctx->l_flags.as<uint32_t>();
    {
        Prof pf(ctx, "link_video");
        CK(link_run(in, L, S, out, ctx->st));
    }
    std::vector<uint32_t> flags(nvideos);
    CK(cudaMemcpyAsync(flags.data(), out.flags, nvideos * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    uint32_t all = 0;
    for (auto f : flags) all |= f;
    if (all & kFlagTooDense)
        return set_err(ctx, GT_ERR_TOO_DENSE_TO_LINK,
                       "computational load during linking is abnormally high. try setting a smaller search range "
                       "or track with settings that give fewer detections.");
    if (all & kFlagSubnetBudget)
        return set_err(ctx, GT_ERR_SUBNET_TOO_EXPENSIVE, "a linking subnet exceeded the device search budget");
    if (all & kFlagScratch) return set_err(ctx, GT_ERR_INTERNAL, "linker scratch overflow");
    if (counters) {
        counters->resize(nvideos);
        CK(cudaMemcpy(counters->data(), out.counter, nvideos * 8, cudaMemcpyDeviceToHost));
    }
    hs.reset(new HostSpan(ctx, "host_link_durations"));
    if (row_dur) {
        {
            Prof pf(ctx, "link_durations");
            CK(link_durations(in, out, row_dur, ctx->st));
        }
        CK(cudaMemcpyAsync(flags.data(), out.flags, nvideos * 4, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        for (auto f : flags)
            if (f & kFlagScratch)
                return set_err(ctx, GT_ERR_INTERNAL,
                               "a particle id has no duration entry after a linker reset (the reference panics here)");
    }
    (void)row_particle;
    return GT_OK;
}


__global__ void f32_round_ids_kernel(const int64_t* ids, int64_t* out, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (int64_t)(float)ids[i];
}

cudaError_t launch_round_ids(const int64_t* ids, int64_t* out, int64_t n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    f32_round_ids_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(ids, out, n);
    return cudaGetLastError();
}

}  // namespace rt
}  // namespace gt

extern "C" {

gt_status gt_link(gt_ctx* ctx, const float* frame_y_x, int64_t n, float search_range, uint32_t memory,
                  int64_t* particle_out) {
    if (!ctx) return GT_ERR_INVALID_ARGUMENT;
    if (n == 0) return GT_OK;
    if (!frame_y_x || !particle_out) return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "null argument");
    CK(cudaSetDevice(ctx->device));
    LinkJob job;
    std::vector<int64_t> gframe;
    CKS(subset_groups(ctx, frame_y_x, n, 3, job.goff, gframe));
    const int64_t N = job.goff.back();
    job.vgrp = {0, (int32_t)gframe.size()};
    job.reset.assign(gframe.size(), 0);
    job.radius = search_range;
    job.memory = (int32_t)memory;
    std::vector<float> px(N), py(N);
    for (int64_t i = 0; i < N; i++) {
        px[i] = frame_y_x[3 * i + 1];
        py[i] = frame_y_x[3 * i + 2];
    }
    CKS(upload(ctx, ctx->l_px, px));
    CKS(upload(ctx, ctx->l_py, py));
    CK(ctx->l_ids.ensure(std::max<int64_t>(N, 1) * 8));
    CKS(run_link(ctx, job, ctx->l_px.as<float>(), ctx->l_py.as<float>(), ctx->l_ids.as<int64_t>(), nullptr, nullptr,
                 nullptr));
    CK(cudaMemcpyAsync(particle_out, ctx->l_ids.p, N * 8, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return GT_OK;
}

// connect_all (src/linking.rs:960-1020): the frame bookkeeping runs on the
// host exactly as the reference's iterators do; every connected frame pair is
// an independent two-frame linking job, all of them solved in one launch.
gt_status gt_connect(gt_ctx* ctx, const float* a1, int64_t n1, const float* a2, int64_t n2, float search_range,
                     int64_t* out1, int64_t* out2) {
    if (!ctx) return GT_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(ctx->device));
    std::vector<int64_t> g1, f1, g2, f2;
    CKS(subset_groups(ctx, a1, n1, 3, g1, f1));
    CKS(subset_groups(ctx, a2, n2, 3, g2, f2));
    // operations in the reference's order
    struct Op {
        int kind;  // 0 fill side 1, 1 fill side 2, 2 connect
        int64_t i1, i2;
    };
    std::vector<Op> ops;
    size_t p1 = 0, p2 = 0;
    auto next1 = [&](int64_t* g) { if (p1 < f1.size()) { *g = (int64_t)p1++; return true; } return false; };
    auto next2 = [&](int64_t* g) { if (p2 < f2.size()) { *g = (int64_t)p2++; return true; } return false; };
    while (true) {
        int64_t a, b;
        bool h1 = next1(&a), h2 = next2(&b);
        if (h1 && h2) {
            if (f1[a] == f2[b]) {
                ops.push_back({2, a, b});
                continue;
            }
            // sync_iterators (src/linking.rs:914-958)
            bool left = f1[a] > f2[b];
            int64_t hit = left ? a : b;
            if (left) ops.push_back({1, -1, b}); else ops.push_back({0, a, -1});
            while (true) {
                int64_t nx;
                bool got = left ? next2(&nx) : next1(&nx);
                if (!got) {
                    if (left) ops.push_back({0, hit, -1}); else ops.push_back({1, -1, hit});
                    break;
                }
                int64_t fh = left ? f1[hit] : f2[hit];
                int64_t fn = left ? f2[nx] : f1[nx];
                if (fh > fn) {
                    if (left) ops.push_back({1, -1, nx}); else ops.push_back({0, nx, -1});
                } else if (fh == fn) {
                    if (left) ops.push_back({2, hit, nx}); else ops.push_back({2, nx, hit});
                    break;
                } else {
                    if (left) ops.push_back({1, -1, nx}); else ops.push_back({0, nx, -1});
                    if (left) ops.push_back({0, hit, -1}); else ops.push_back({1, -1, hit});
                    hit = nx;
                    left = !left;
                }
            }
        } else if (h1) {
            ops.push_back({0, a, -1});
        } else if (h2) {
            ops.push_back({1, -1, b});
        } else {
            break;
        }
    }
    // linking jobs for the connect operations
    LinkJob job;
    job.goff.assign(1, 0);
    job.vgrp.assign(1, 0);
    job.radius = search_range;
    job.memory = 0;
    std::vector<float> px, py;
    std::vector<int64_t> op_video(ops.size(), -1);
    for (size_t k = 0; k < ops.size(); k++) {
        if (ops[k].kind != 2) continue;
        op_video[k] = (int64_t)job.vgrp.size() - 1;
        for (int side = 0; side < 2; side++) {
            const float* arr = side ? a2 : a1;
            const std::vector<int64_t>& go = side ? g2 : g1;
            int64_t gi = side ? ops[k].i2 : ops[k].i1;
            for (int64_t i = go[gi]; i < go[gi + 1]; i++) {
                px.push_back(arr[3 * i + 1]);
                py.push_back(arr[3 * i + 2]);
            }
            job.goff.push_back((int64_t)px.size());
            job.reset.push_back(0);
        }
        job.vgrp.push_back((int32_t)job.goff.size() - 1);
    }
    std::vector<int64_t> local((size_t)px.size());
    std::vector<int64_t> counters;
    if (!px.empty()) {
        CKS(upload(ctx, ctx->l_px, px));
        CKS(upload(ctx, ctx->l_py, py));
        CK(ctx->l_ids.ensure(px.size() * 8));
        CKS(run_link(ctx, job, ctx->l_px.as<float>(), ctx->l_py.as<float>(), ctx->l_ids.as<int64_t>(), nullptr,
                     nullptr, &counters));
        CK(cudaMemcpy(local.data(), ctx->l_ids.p, px.size() * 8, cudaMemcpyDeviceToHost));
    }
    std::vector<int64_t> r1, r2;
    int64_t part = 0;
    for (size_t k = 0; k < ops.size(); k++) {
        const Op& o = ops[k];
        if (o.kind == 0) {
            for (int64_t i = g1[o.i1]; i < g1[o.i1 + 1]; i++) r1.push_back(part++);
        } else if (o.kind == 1) {
            for (int64_t i = g2[o.i2]; i < g2[o.i2 + 1]; i++) r2.push_back(part++);
        } else {
            int64_t v = op_video[k];
            int64_t b0 = job.goff[job.vgrp[v]], b1 = job.goff[job.vgrp[v] + 1], b2 = job.goff[job.vgrp[v] + 2];
            for (int64_t i = b0; i < b1; i++) r1.push_back(part + local[i]);
            for (int64_t i = b1; i < b2; i++) r2.push_back(part + local[i]);
            part += counters[v];
        }
    }
    if ((int64_t)r1.size() != n1 || (int64_t)r2.size() != n2)
        return set_err(ctx, GT_ERR_INVALID_ARGUMENT,
                       "connect produced %lld/%lld ids for %lld/%lld rows (frame interleaving the reference "
                       "double-counts)",
                       (long long)r1.size(), (long long)r2.size(), (long long)n1, (long long)n2);
    if (n1) std::memcpy(out1, r1.data(), n1 * 8);
    if (n2) std::memcpy(out2, r2.data(), n2 * 8);
    return GT_OK;
}

}  // extern "C"
