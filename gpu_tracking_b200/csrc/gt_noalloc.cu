// gt_noalloc.cu — linking without any device allocation.
//
// gt_link_noalloc links detections that already sit in device memory and
// writes the particle ids to device memory the caller provides.  Every
// intermediate buffer (frame groups, neighbour lists, the linker's working
// set) is carved out of one file-scope __device__ array, so the call performs
// no cudaMalloc / cudaFree and calls no allocating library routine.  This is
// for callers that cannot allocate device memory while they run: a live
// acquisition loop that links each batch of detections as frames arrive
// (cudaMalloc and cudaFree synchronise the whole device and would stall the
// camera pipeline), or a host process whose device memory is owned by
// another allocator (a framework's caching allocator, a fixed memory budget)
// and must not be grown behind its back.
//
// Limits (kNoAlloc*): at most 32768 detections per call, at most 4096 in one
// frame, memory <= 3, at most 16 neighbour-list entries per detection on
// average in each direction.  Larger inputs get GT_ERR_CAPACITY_EXCEEDED.
// The array (kNoAllocBytes) is held by every GPU that loads the library until
// the process exits; all calls share it and it keeps the last call's
// contents, so calls whose GPU work overlaps in time race on it (run them on
// one stream or serialise them).  Everything a call needs zeroed is cleared
// by the call itself.
//
// The device address of the array is looked up with cudaGetSymbolAddress
// once per device, on the first call made with that device current; make
// that first call before any stream capture begins.  The address stays valid
// for the life of the process's CUDA context on that device: a
// cudaDeviceReset (which also ends this library's contexts) is not supported
// while the library is in use.  Every call reads sizes back to the host and
// synchronises the context's stream before it returns.  The caller's current
// device is restored on return.
#include <mutex>

#include "gt_kernels.h"

namespace gt {

constexpr int64_t kNoAllocMaxPoints = 32768;
constexpr int32_t kNoAllocMaxGroup = 4096;   // sorted in shared memory by sort_groups_kernel
constexpr int32_t kNoAllocMaxMemory = 3;
constexpr int64_t kNoAllocMaxEdges = 16 * kNoAllocMaxPoints;
constexpr size_t kNoAllocBytes = (size_t)20 << 20;

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocBytes];

namespace {

inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

struct NoAllocLayout {
    size_t px, py, goff, pgroup, vgrp, reset, srt, fcnt, bcnt, foff, boff, fpts, bpts, bdist, scal, counter, dur,
        flags, lay, total;
};

NoAllocLayout noalloc_layout() {
    const int64_t N = kNoAllocMaxPoints, K = kNoAllocMaxMemory + 1, E = kNoAllocMaxEdges;
    NoAllocLayout l;
    size_t o = 0;
    l.px = o; o = al256(o + 4 * N);
    l.py = o; o = al256(o + 4 * N);
    l.goff = o; o = al256(o + 8 * (N + 2));
    l.pgroup = o; o = al256(o + 4 * N);
    l.vgrp = o; o = al256(o + 8);
    l.reset = o; o = al256(o + N + 1);
    l.srt = o; o = al256(o + 4 * N);
    l.fcnt = o; o = al256(o + 8 * (N * K + 1));
    l.bcnt = o; o = al256(o + 8 * (N * K + 1));
    l.foff = o; o = al256(o + 8 * (N * K + 1));
    l.boff = o; o = al256(o + 8 * (N * K + 1));
    l.fpts = o; o = al256(o + 4 * E);
    l.bpts = o; o = al256(o + 4 * E);
    l.bdist = o; o = al256(o + 4 * E);
    l.scal = o; o = al256(o + 8 * 8);
    l.counter = o; o = al256(o + 8);
    l.dur = o; o = al256(o + 8 * N);
    l.flags = o; o = al256(o + 4);
    l.lay = o; o = al256(o + link_scratch_bytes(kNoAllocMaxGroup, E, N, kNoAllocMaxMemory));
    l.total = o;
    return l;
}

// Block-wide inclusive max scan of one float per thread.
__device__ float block_incl_max(float v, float* wsm) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int d = 1; d < 32; d <<= 1) {
        float t = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v = fmaxf(v, t);
    }
    __syncthreads();
    if (lane == 31) wsm[wid] = v;
    __syncthreads();
    if (wid == 0) {
        float x = (lane < nw) ? wsm[lane] : -INFINITY;
        for (int d = 1; d < 32; d <<= 1) {
            float t = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x = fmaxf(x, t);
        }
        if (lane < nw) wsm[lane] = x;
    }
    __syncthreads();
    if (wid > 0) v = fmaxf(v, wsm[wid - 1]);
    return v;
}

// FrameSubsetter grouping on the device (src/linking.rs:97-196): the current
// frame value starts at 0 and only rises; a row whose frame exceeds it starts a
// group (a positive first frame leaves an empty group 0 in front), a row
// below it is NonSortedCharacterization.  One CTA.
__global__ void __launch_bounds__(1024)
noalloc_groups_kernel(const float* __restrict__ fyx, int64_t n, float* px, float* py, int64_t* goff,
                      int32_t* pgroup, int32_t* vgrp, uint8_t* reset, int64_t* scal) {
    __shared__ float wsm[32];
    __shared__ int wsum[33];
    __shared__ float s_cur;
    __shared__ int s_groups;
    if (threadIdx.x == 0) {
        s_cur = 0.0f;
        s_groups = 0;
        scal[0] = 0;
        scal[1] = 0;
        scal[2] = 0;
        goff[0] = 0;
    }
    __syncthreads();
    for (int64_t b = 0; b < n; b += blockDim.x) {
        const int64_t i = b + threadIdx.x;
        float f = (i < n) ? fyx[3 * i] : NAN;
        if (i < n) {
            px[i] = fyx[3 * i + 1];
            py[i] = fyx[3 * i + 2];
        }
        // current value before row i: max of 0 and every earlier non-NaN frame
        float fv = (f == f) ? f : -INFINITY;
        float incl = block_incl_max(fv, wsm);
        float excl = __shfl_up_sync(0xffffffffu, incl, 1);
        if ((threadIdx.x & 31) == 0) excl = (threadIdx.x == 0) ? -INFINITY : wsm[(threadIdx.x >> 5) - 1];
        const float cur = fmaxf(s_cur, excl);
        const int start = (i < n && f > cur) ? 1 : 0;
        if (i < n && f < cur) atomicOr((unsigned long long*)&scal[2], 1ull);
        int tot;
        int pos = block_excl_scan(start, &tot, wsum);
        const int g0 = s_groups;
        if (start) goff[g0 + pos + 1] = i;
        if (i < n) pgroup[i] = g0 + pos + start;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) {
            s_cur = fmaxf(s_cur, incl);
            s_groups = g0 + tot;
        }
        __syncthreads();
    }
    const int ng = s_groups + 1;
    if (threadIdx.x == 0) {
        goff[ng] = n;
        vgrp[0] = 0;
        vgrp[1] = ng;
        scal[0] = ng;
    }
    __syncthreads();
    for (int g = threadIdx.x; g < ng; g += blockDim.x) {
        reset[g] = 0;
        atomicMax((unsigned long long*)&scal[1], (unsigned long long)(goff[g + 1] - goff[g]));
    }
}

// Exclusive prefix sum of n int64 values in one CTA (chunks of 1024).
__global__ void __launch_bounds__(1024) noalloc_scan_kernel(const int64_t* __restrict__ in, int64_t* out,
                                                            int64_t n) {
    __shared__ long long wsum[33];
    __shared__ long long s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int64_t b = 0; b < n; b += blockDim.x) {
        const int64_t i = b + threadIdx.x;
        long long v = (i < n) ? in[i] : 0;
        long long incl = v;
        for (int d = 1; d < 32; d <<= 1) {
            long long t = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += t;
        }
        if (lane == 31) wsum[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            long long x = (lane < nw) ? wsum[lane] : 0;
            long long sum = x;
            for (int d = 1; d < 32; d <<= 1) {
                long long t = __shfl_up_sync(0xffffffffu, sum, d);
                if (lane >= d) sum += t;
            }
            if (lane < nw) wsum[lane] = sum - x;
            if (lane == 31) wsum[32] = sum;
        }
        __syncthreads();
        if (i < n) out[i] = s_carry + wsum[wid] + incl - v;
        __syncthreads();
        if (threadIdx.x == 0) s_carry += wsum[32];
        __syncthreads();
    }
}

std::mutex g_setup_mu;
uint8_t* g_base[64] = {};

}  // namespace
}  // namespace gt

using namespace gt;

// gt_ctx is opaque here; the entry point needs its device and stream only.
extern "C" int gt__ctx_device(const gt_ctx* ctx);
extern "C" cudaStream_t gt__ctx_stream(const gt_ctx* ctx);
extern "C" void gt__ctx_set_error(gt_ctx* ctx, const char* msg);
extern "C" gt_status gt__device_span_check(gt_ctx* ctx, const void* p, size_t bytes, const char* what);

namespace {
// Restores the calling thread's current device when the call returns.
struct DeviceGuard {
    int prev = -1;
    DeviceGuard() {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            cudaGetLastError();
            prev = -1;
        }
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};
}  // namespace

static gt_status noalloc_fail(gt_ctx* ctx, gt_status st, const char* msg) {
    gt__ctx_set_error(ctx, msg);
    return st;
}

#define NA_CK(expr)                                                                \
    do {                                                                           \
        cudaError_t e_ = (expr);                                                   \
        if (e_ != cudaSuccess) return noalloc_fail(ctx, GT_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)

extern "C" gt_status gt_link_noalloc(gt_ctx* ctx, const float* d_fyx, int64_t n, float search_range,
                                     uint32_t memory, int64_t* d_out) {
    if (!ctx) return GT_ERR_INVALID_ARGUMENT;
    if (n < 0) return noalloc_fail(ctx, GT_ERR_INVALID_ARGUMENT, "negative row count");
    if (n == 0) return GT_OK;
    if (!d_fyx || !d_out) return noalloc_fail(ctx, GT_ERR_INVALID_ARGUMENT, "null argument");
    const int dev = gt__ctx_device(ctx);
    cudaStream_t st = gt__ctx_stream(ctx);
    DeviceGuard restore_device;
    NA_CK(cudaSetDevice(dev));
    for (const void* ptr : {(const void*)d_fyx, (const void*)d_out}) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess ||
            !(at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) || at.device != dev) {
            cudaGetLastError();
            return noalloc_fail(ctx, GT_ERR_INVALID_ARGUMENT, "gt_link_noalloc takes device pointers of the context's device");
        }
    }
    // the n rows read and the n ids written must lie inside their allocations
    {
        gt_status s = gt__device_span_check(ctx, d_fyx, (size_t)n * 12, "gt_link_noalloc rows (n x 3 float32)");
        if (s != GT_OK) return s;
        s = gt__device_span_check(ctx, d_out, (size_t)n * 8, "gt_link_noalloc ids (n int64)");
        if (s != GT_OK) return s;
    }
    if (n > kNoAllocMaxPoints)
        return noalloc_fail(ctx, GT_ERR_CAPACITY_EXCEEDED, "gt_link_noalloc links at most 32768 detections");
    if (memory > (uint32_t)kNoAllocMaxMemory)
        return noalloc_fail(ctx, GT_ERR_CAPACITY_EXCEEDED, "gt_link_noalloc supports memory <= 3");
    const NoAllocLayout L = noalloc_layout();
    if (L.total > kNoAllocBytes) return noalloc_fail(ctx, GT_ERR_INTERNAL, "static scratch layout too large");
    uint8_t* base;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (dev < 0 || dev >= 64) return noalloc_fail(ctx, GT_ERR_INVALID_ARGUMENT, "device index");
        if (!g_base[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) return noalloc_fail(ctx, GT_ERR_CUDA, "cudaGetSymbolAddress failed");
            g_base[dev] = (uint8_t*)p;
        }
        base = g_base[dev];
    }
    const int K = (int)memory + 1;
    float* px = (float*)(base + L.px);
    float* py = (float*)(base + L.py);
    int64_t* goff = (int64_t*)(base + L.goff);
    int32_t* pgroup = (int32_t*)(base + L.pgroup);
    int32_t* vgrp = (int32_t*)(base + L.vgrp);
    uint8_t* reset = base + L.reset;
    uint32_t* srt = (uint32_t*)(base + L.srt);
    int64_t* fcnt = (int64_t*)(base + L.fcnt);
    int64_t* bcnt = (int64_t*)(base + L.bcnt);
    int64_t* foff = (int64_t*)(base + L.foff);
    int64_t* boff = (int64_t*)(base + L.boff);
    int64_t* scal = (int64_t*)(base + L.scal);
    uint32_t* flags = (uint32_t*)(base + L.flags);

    noalloc_groups_kernel<<<1, 1024, 0, st>>>(d_fyx, n, px, py, goff, pgroup, vgrp, reset, scal);
    NA_CK(cudaGetLastError());
    int64_t hs[3] = {0, 0, 0};
    NA_CK(cudaMemcpyAsync(hs, scal, sizeof(hs), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    if (hs[2]) return noalloc_fail(ctx, GT_ERR_NON_SORTED_CHARACTERIZATION,
                                   "the points provided for characterization aren't sorted in ascending frame number.");
    const int ngroups = (int)hs[0];
    const int64_t maxg = hs[1];
    if (maxg > kNoAllocMaxGroup)
        return noalloc_fail(ctx, GT_ERR_CAPACITY_EXCEEDED, "gt_link_noalloc links at most 4096 detections per frame");

    LinkInput in;
    in.px = px;
    in.py = py;
    in.goff = goff;
    in.pgroup = pgroup;
    in.vgrp = vgrp;
    in.reset = reset;
    in.ngroups = ngroups;
    in.nvideos = 1;
    in.npoints = n;
    in.radius = search_range;
    in.memory = (int32_t)memory;
    NA_CK(link_sort_groups(in, srt, nullptr, 0, (int)maxg, st));
    const int64_t NK = n * K;
    NA_CK(cudaMemsetAsync(fcnt + NK, 0, 8, st));
    NA_CK(cudaMemsetAsync(bcnt + NK, 0, 8, st));
    NA_CK(link_count_lists(in, srt, fcnt, bcnt, st));
    noalloc_scan_kernel<<<1, 1024, 0, st>>>(fcnt, foff, NK + 1);
    noalloc_scan_kernel<<<1, 1024, 0, st>>>(bcnt, boff, NK + 1);
    NA_CK(cudaGetLastError());
    int64_t tots[2] = {0, 0};
    NA_CK(cudaMemcpyAsync(&tots[0], foff + NK, 8, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaMemcpyAsync(&tots[1], boff + NK, 8, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    if (tots[0] > kNoAllocMaxEdges || tots[1] > kNoAllocMaxEdges)
        return noalloc_fail(ctx, GT_ERR_CAPACITY_EXCEEDED, "too many neighbour pairs for gt_link_noalloc's scratch");
    LinkLists LL;
    LL.f_off = foff;
    LL.b_off = boff;
    LL.f_pts = (int32_t*)(base + L.fpts);
    LL.b_pts = (int32_t*)(base + L.bpts);
    LL.b_dist = (float*)(base + L.bdist);
    LL.srt = srt;
    // the list sizes select the linker variant with 32-bit list offsets when
    // they fit, as gt_link does (a larger shared-memory working set per frame)
    LL.f_entries = tots[0];
    NA_CK(link_fill_lists(in, LL, st));
    LinkScratch S;
    S.base = base + L.lay;
    S.max_group = kNoAllocMaxGroup;
    S.max_edges = kNoAllocMaxEdges;
    S.bytes_per_video = link_scratch_bytes(S.max_group, S.max_edges, n, (int32_t)memory);
    S.max_points = n;
    LinkOutput out;
    out.ids = d_out;
    out.counter = (int64_t*)(base + L.counter);
    out.dur = (int64_t*)(base + L.dur);
    out.vpoff = nullptr;
    out.flags = flags;
    NA_CK(cudaMemsetAsync(flags, 0, 4, st));
    NA_CK(link_run(in, LL, S, out, st));
    uint32_t hf = 0;
    NA_CK(cudaMemcpyAsync(&hf, flags, 4, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    if (hf & kFlagTooDense)
        return noalloc_fail(ctx, GT_ERR_TOO_DENSE_TO_LINK,
                            "computational load during linking is abnormally high. try setting a smaller search range "
                            "or track with settings that give fewer detections.");
    if (hf & kFlagSubnetBudget)
        return noalloc_fail(ctx, GT_ERR_SUBNET_TOO_EXPENSIVE, "a linking subnet exceeded the device search budget");
    if (hf) return noalloc_fail(ctx, GT_ERR_INTERNAL, "linker scratch overflow");
    return GT_OK;
}
