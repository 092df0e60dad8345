// gt_runtime.cuh — host runtime internals shared by the units of the C ABI
// (gt_api.cu: context, locating and batch calls; gt_linkdrv.cu: the linking
// calls; gt_table.cu: result tables and their export).  Not installed: the
// public interface is include/gpu_tracking_b200.h.
#pragma once

#include <nvtx3/nvToolsExt.h>
#include <cuda.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "gt_kernels.h"

namespace gt {
namespace rt {

struct DBuf {
    void* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t ensure(size_t bytes) {
        if (bytes <= n && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) n = want;
        return e;
    }
    template <class T>
    T* as() const {
        return (T*)p;
    }
};

// Result tables come and go with every call: their columns are stream-ordered
// allocations from one pool per device that keeps its memory, so a call
// neither maps fresh device memory nor synchronises the device to free it.
inline cudaMemPool_t table_pool(int device) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[device] = pool;
    return pool;
}

struct TBuf {
    void* p = nullptr;
    size_t n = 0;
    int device = 0;
    cudaStream_t stream = nullptr;   // the call's compute stream
    TBuf() = default;
    TBuf(const TBuf&) = delete;
    TBuf& operator=(const TBuf&) = delete;
    // a table is freed only when no work on it is pending
    ~TBuf() {
        if (p) cudaFreeAsync(p, cudaStreamPerThread);
    }
    cudaError_t ensure(size_t bytes) {
        if (bytes <= n && p) return cudaSuccess;
        if (p) cudaFreeAsync(p, stream);
        p = nullptr;
        n = 0;
        const size_t want = std::max<size_t>(bytes, 256);
        cudaMemPool_t pool = table_pool(device);
        if (!pool) return cudaErrorMemoryAllocation;
        cudaError_t e = cudaMallocFromPoolAsync(&p, want, pool, stream);
        if (e == cudaSuccess) n = want;
        return e;
    }
    template <class T>
    T* as() const {
        return (T*)p;
    }
};

struct KernelStat {
    int64_t launches = 0;
    double ms = 0.0;
};


}  // namespace rt
}  // namespace gt

using gt::rt::DBuf;
using gt::rt::KernelStat;
using gt::rt::TBuf;

struct gt_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t st = nullptr;   // compute
    cudaStream_t cp = nullptr;   // host -> device copies
    cudaStream_t lk = nullptr;   // linking of located frames, overlapped with locating
    cudaStream_t ls = nullptr;   // neighbour lists of the next link window, beside the linker
    cudaEvent_t located = nullptr, linked = nullptr;
    cudaEvent_t listed[2] = {nullptr, nullptr};    // list set b holds its window's lists
    cudaEvent_t w_linked[2] = {nullptr, nullptr};  // the linker finished with list set b
    cudaEvent_t used[2] = {nullptr, nullptr};    // compute finished with staging buffer b
    cudaEvent_t filled[2] = {nullptr, nullptr};  // staging buffer b holds its chunk
    std::string err;
    const volatile int32_t* interrupt = nullptr;
    std::atomic<int64_t> done{0}, total{0};
    // profiling of the main kernels (CUDA events on the compute stream)
    bool profile = false;
    std::map<std::string, KernelStat> stats;
    std::map<std::string, int64_t> launch_count;
    std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
    std::vector<cudaEvent_t> event_pool;
    // device buffers, grown on demand and kept for the next call
    DBuf stage[2], processed, planes, cand_count, cand_keys, feats_raw, feat_count, feats_out, kept_count,
        fin_scratch, flags, ident, tabs_f, tabs_i, tabs_s, tabs_m, row_off, frame_num;
    DBuf l_srt, l_sortscr, l_fcnt, l_bcnt, l_foff, l_boff, l_fpts, l_bpts, l_bdist, l_scan, l_scratch, l_ids, l_cnt,
        l_dur, l_flags, l_goff, l_pgroup, l_vgrp, l_reset, l_vpoff, l_px, l_py, l_ge, l_rowdur, l_part;
    // windowed linking inside gt_batch (slot mode)
    DBuf fstd, std_scratch, amask, astatus, acount;   // snr / minmass_snr / adaptive_background
    DBuf illum_taps, illum_shared, illum_prof, illum_corr;  // illumination correction
    DBuf cnn_x, cnn_p, cnn_q, cnn_head;   // learned proposals: network input, activations, outputs
    DBuf walk_starts;                     // walk starts of the current call (u64)
    DBuf vd_src, vd_dec, vd_blk, vd_bad;  // video files decoded on the device: streams, bytes, blocks, flag
    int64_t last_walk_starts = 0;
    int32_t illum_rint = 0;
    DBuf w_srt, w_bins, w_scan, w_scratch, w_ids, w_dur, w_state, w_cnt, w_flags, w_vgrp, w_reset;
    // two sets of window neighbour lists: the lists of window w + 1 are built
    // while the linker reads those of window w
    DBuf w_fcnt[2], w_bcnt[2], w_foff[2], w_boff[2], w_fpts[2], w_bpts[2], w_bdist[2];
    // ragged batches (gt_batch_videos): frame / task tables of the current
    // wave, the captured stage graph (valid while the buffers it names stay
    // where they are: rg_graph_key) and the tuned wave shape per workload
    DBuf rg_frames, rg_tasks, rg_ntasks;
    cudaGraphExec_t rg_graph = nullptr;
    std::string rg_graph_key;
    std::map<std::string, std::pair<int32_t, int64_t>> rg_best;
    bool no_ragged = false;   // test hook: gt_batch_videos locates video by video
    bool rg_force_tune = false;   // test hook: tune on every ragged call
    int64_t w_list_cap = 0;   // entries of each window neighbour-list buffer (0 = not sized yet)
    int64_t w_edge_cap = 0;   // backward edges per frame the window scratch holds
    uint32_t cand_cap = 16384;
    uint32_t feat_cap = 4096;
};

struct gt_table {
    int device = 0;
    int64_t n = 0;
    TBuf frame, particle, duration;
    TBuf col[GT_NUM_COLUMNS];
    bool has[GT_NUM_COLUMNS] = {};
    gt_table(int dev, cudaStream_t st) : device(dev) {
        for (TBuf* b : {&frame, &particle, &duration}) {
            b->device = dev;
            b->stream = st;
        }
        for (auto& b : col) {
            b.device = dev;
            b.stream = st;
        }
    }
};

namespace gt {
namespace rt {

// Waits for the link-side streams (neighbour lists and linker) to finish.
inline cudaError_t sync_link_streams(gt_ctx* ctx) {
    const cudaError_t a = cudaStreamSynchronize(ctx->ls);
    const cudaError_t b = cudaStreamSynchronize(ctx->lk);
    return a != cudaSuccess ? a : b;
}

inline gt_status set_err(gt_ctx* ctx, gt_status st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf;
    return st;
}

#define CK(expr)                                                                                             \
    do {                                                                                                     \
        cudaError_t e_ = (expr);                                                                             \
        if (e_ != cudaSuccess)                                                                               \
            return set_err(ctx, GT_ERR_CUDA, "CUDA error %s at %s:%d (%s)", cudaGetErrorString(e_), __FILE__, \
                           __LINE__, #expr);                                                                 \
    } while (0)

#define CKS(expr)                        \
    do {                                 \
        gt_status s_ = (expr);           \
        if (s_ != GT_OK) return s_;      \
    } while (0)

// --------------------------------------------------------------- profiling
// Counts every kernel launch of the engine; with profiling enabled also
// brackets it with CUDA events on the compute stream.
// Every Prof and HostSpan is also an NVTX range under its name (header-only
// NVTX v3: the ranges cost a branch unless a profiler such as Nsight Systems
// is attached, which then shows each stage's launches and host phases).
struct Prof {
    gt_ctx* ctx;
    const char* name;
    cudaStream_t stream;
    cudaEvent_t a = nullptr, b = nullptr;
    Prof(gt_ctx* c, const char* n, cudaStream_t s = nullptr) : ctx(c), name(n), stream(s ? s : c->st) {
        nvtxRangePushA(name);
        ctx->launch_count[name]++;
        if (!ctx->profile) return;
        a = take();
        b = take();
        cudaEventRecord(a, stream);
    }
    cudaEvent_t take() {
        if (!ctx->event_pool.empty()) {
            cudaEvent_t e = ctx->event_pool.back();
            ctx->event_pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    ~Prof() {
        nvtxRangePop();
        if (!ctx->profile) return;
        cudaEventRecord(b, stream);
        ctx->pending.push_back({name, {a, b}});
    }
};

// Host wall-clock of one phase of a call, accumulated under `name` next to
// the kernels' device times when profiling is on (gaps between kernels are
// host work: allocation, uploads, read-backs).
struct HostSpan {
    gt_ctx* ctx;
    const char* name;
    std::chrono::steady_clock::time_point t0;
    HostSpan(gt_ctx* c, const char* n) : ctx(c), name(n), t0(std::chrono::steady_clock::now()) {
        nvtxRangePushA(name);
    }
    ~HostSpan() {
        nvtxRangePop();
        if (!ctx->profile) return;
        auto& s = ctx->stats[name];
        s.launches++;
        s.ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

// Folds finished launches into the statistics; with block, waits for all.
inline void drain_profile(gt_ctx* ctx, bool block = true) {
    size_t keep = 0;
    for (size_t i = 0; i < ctx->pending.size(); i++) {
        auto& p = ctx->pending[i];
        if (block) {
            cudaEventSynchronize(p.second.second);
        } else if (cudaEventQuery(p.second.second) != cudaSuccess) {
            cudaGetLastError();
            ctx->pending[keep++] = p;
            continue;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, p.second.first, p.second.second);
        auto& s = ctx->stats[p.first];
        s.launches++;
        s.ms += ms;
        ctx->event_pool.push_back(p.second.first);
        ctx->event_pool.push_back(p.second.second);
    }
    ctx->pending.resize(keep);
}

inline size_t dtype_bytes(int32_t dtype) { return dtype == GT_DTYPE_F32 ? 4 : (dtype == GT_DTYPE_U16 ? 2 : 1); }

// cuMemGetAddressRange through the runtime's driver entry point (no link
// against libcuda); null when the driver does not offer it.
typedef CUresult (*AddressRangeFn)(CUdeviceptr*, size_t*, CUdeviceptr);
inline AddressRangeFn address_range_fn() {
    static AddressRangeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* q = nullptr;
        cudaDriverEntryPointQueryResult r;
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &q, cudaEnableDefault, &r) == cudaSuccess &&
            r == cudaDriverEntryPointSuccess)
            fn = (AddressRangeFn)q;
        else
            cudaGetLastError();
    });
    return fn;
}

// Host or device frames; device frames must live on the context's device and
// the `bytes` the call reads must lie inside the allocation that holds them
// (a wrong dtype or shape for a device tensor is an error, not a read past
// the end of its memory).
inline gt_status check_frames_ptr(gt_ctx* ctx, const void* frames, size_t bytes, bool* on_device) {
    cudaPointerAttributes at;
    cudaError_t e = cudaPointerGetAttributes(&at, frames);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *on_device = false;
        return GT_OK;
    }
    if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) {
        if (at.device != ctx->device)
            return set_err(ctx, GT_ERR_INVALID_ARGUMENT, "frames live on device %d, context is on device %d",
                           at.device, ctx->device);
        *on_device = true;
        CUdeviceptr base = 0;
        size_t size = 0;
        AddressRangeFn fn = address_range_fn();
        if (at.type == cudaMemoryTypeDevice && fn && fn(&base, &size, (CUdeviceptr)frames) == CUDA_SUCCESS) {
            const uint64_t off = (uint64_t)(uintptr_t)frames - (uint64_t)base;
            if (off > size || bytes > size - off)
                return set_err(ctx, GT_ERR_INVALID_ARGUMENT,
                               "the device frames (%zu bytes from their pointer) run past the end of their "
                               "allocation (%zu bytes left): check the dtype and shape",
                               bytes, (size_t)(size - std::min<uint64_t>(off, size)));
        }
    } else {
        *on_device = false;
    }
    return GT_OK;
}

inline bool interrupted(gt_ctx* ctx) { return ctx->interrupt && *ctx->interrupt != 0; }

template <class T>
inline gt_status upload(gt_ctx* ctx, DBuf& b, const std::vector<T>& v) {
    CK(b.ensure(std::max<size_t>(1, v.size()) * sizeof(T)));
    if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->st));
    return GT_OK;
}

inline gt_status subset_groups(gt_ctx* ctx, const float* rows, int64_t n, int ncols, std::vector<int64_t>& goff,
                        std::vector<int64_t>& gframe) {
    goff.assign(1, 0);
    gframe.clear();
    float cur = 0.0f;
    int64_t idx = 0;
    while (true) {
        if (idx < n) {
            float f = rows[idx * ncols];
            if (f > cur) {
                goff.push_back(idx);
                gframe.push_back((int64_t)cur);
                cur = f;
                continue;
            }
            if (f < cur)
                return set_err(ctx, GT_ERR_NON_SORTED_CHARACTERIZATION,
                               "the points provided for characterization aren't sorted in ascending frame number.");
            idx++;
        } else {
            if (idx > goff.back()) {
                goff.push_back(idx);
                gframe.push_back((int64_t)cur);
            }
            break;
        }
    }
    return GT_OK;
}

// ---------------------------------------------------------------- linking
// host description of the groups (frames) and videos to link
struct LinkJob {
    std::vector<int64_t> goff;   // ngroups + 1, row offsets into px/py
    std::vector<int32_t> vgrp;   // nvideos + 1
    std::vector<uint8_t> reset;  // per group
    float radius = 0;
    int32_t memory = 0;
};

// Runs the linker over px/py (device, npoints) and writes ids (device) and,
// when row_dur is given, per-row durations (gt_linkdrv.cu).
gt_status run_link(gt_ctx* ctx, const LinkJob& job, const float* px, const float* py, int64_t* ids_out,
                   int64_t* row_dur, int64_t* row_particle, std::vector<int64_t>* counters);
// out[i] = (int64)(float)ids[i]: particle ids as the reference stores them (float32)
cudaError_t launch_round_ids(const int64_t* ids, int64_t* out, int64_t n, cudaStream_t st);

}  // namespace rt
}  // namespace gt
