// gt_table.cu — result tables of the C ABI: row counts, single columns and
// gt_table_export, which copies several columns at once through per-device
// pools of pinned staging lanes and widens them to the dtypes of the
// reference's DataFrame (gpu_tracking_macros/src/lib.rs:138-147) on host
// threads.
#include <memory>
#include <thread>

#include "gt_runtime.cuh"

using namespace gt;
using namespace gt::rt;

extern "C" {

int64_t gt_table_nrows(const gt_table* t) { return t ? t->n : 0; }

int32_t gt_table_has_column(const gt_table* t, int32_t column) {
    if (!t || column < 0 || column >= GT_NUM_COLUMNS) return 0;
    return t->has[column] ? 1 : 0;
}

gt_status gt_table_column_f32(const gt_table* t, int32_t column, float* dst) {
    if (!t || !dst || column < 0 || column >= GT_NUM_COLUMNS) return GT_ERR_INVALID_ARGUMENT;
    if (!t->has[column]) return GT_ERR_INVALID_ARGUMENT;
    if (t->n == 0) return GT_OK;
    cudaSetDevice(t->device);
    if (column == GT_COL_FRAME || column == GT_COL_PARTICLE || column == GT_COL_DURATION) {
        std::vector<int64_t> v(t->n);
        const TBuf& b = column == GT_COL_FRAME ? t->frame : (column == GT_COL_PARTICLE ? t->particle : t->duration);
        if (cudaMemcpy(v.data(), b.p, t->n * 8, cudaMemcpyDeviceToHost) != cudaSuccess) return GT_ERR_CUDA;
        for (int64_t i = 0; i < t->n; i++) dst[i] = (float)v[i];
        return GT_OK;
    }
    if (cudaMemcpy(dst, t->col[column].p, t->n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return GT_ERR_CUDA;
    return GT_OK;
}

gt_status gt_table_column_i64(const gt_table* t, int32_t column, int64_t* dst) {
    if (!t || !dst) return GT_ERR_INVALID_ARGUMENT;
    if (column != GT_COL_FRAME && column != GT_COL_PARTICLE && column != GT_COL_DURATION)
        return GT_ERR_INVALID_ARGUMENT;
    if (!t->has[column]) return GT_ERR_INVALID_ARGUMENT;
    if (t->n == 0) return GT_OK;
    cudaSetDevice(t->device);
    const TBuf& b = column == GT_COL_FRAME ? t->frame : (column == GT_COL_PARTICLE ? t->particle : t->duration);
    if (cudaMemcpy(dst, b.p, t->n * 8, cudaMemcpyDeviceToHost) != cudaSuccess) return GT_ERR_CUDA;
    return GT_OK;
}

namespace {

// Table export: each lane (one host thread) owns two pinned slots and a
// stream; it copies its share of the rows chunk by chunk into one slot while
// it widens the previous chunk from the other into the destination.
constexpr int kExportLanes = 8;
constexpr size_t kExportSlot = (size_t)1 << 20;
constexpr int kExportMaxDevices = 64;

struct ExportLane {
    char* slot[2] = {nullptr, nullptr};
    cudaStream_t st = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
};

struct ExportPool {
    std::mutex mu;
    bool ready = false;
    ExportLane lane[kExportLanes];
};

// One pool per device for the life of the process (never destroyed: no CUDA
// call runs from a static destructor after the runtime has shut down).
ExportPool* export_pool(int device) {
    static ExportPool* pools = new ExportPool[kExportMaxDevices];
    return device >= 0 && device < kExportMaxDevices ? &pools[device] : nullptr;
}

// All or nothing: on a failure everything created so far is released and the
// next call tries again.
cudaError_t export_pool_init(ExportPool& p) {
    if (p.ready) return cudaSuccess;
    char* block = nullptr;
    cudaError_t e = cudaHostAlloc((void**)&block, 2 * kExportLanes * kExportSlot, cudaHostAllocDefault);
    if (e != cudaSuccess) return e;
    for (int l = 0; l < kExportLanes && e == cudaSuccess; l++) {
        ExportLane& L = p.lane[l];
        L.slot[0] = block + (2 * l) * kExportSlot;
        L.slot[1] = block + (2 * l + 1) * kExportSlot;
        e = cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking);
        for (int s = 0; s < 2 && e == cudaSuccess; s++) e = cudaEventCreateWithFlags(&L.ev[s], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        for (ExportLane& L : p.lane) {
            for (cudaEvent_t& ev : L.ev)
                if (ev) cudaEventDestroy(ev), ev = nullptr;
            if (L.st) cudaStreamDestroy(L.st), L.st = nullptr;
            L.slot[0] = L.slot[1] = nullptr;
        }
        cudaFreeHost(block);
        return e;
    }
    p.ready = true;
    return cudaSuccess;
}

struct ExportItem {
    const char* src;   // device rows
    char* dst;         // host rows
    int64_t rows;
    bool widen;        // float32 -> double; otherwise int64 copied as is
};

cudaError_t export_lane(int device, ExportLane& L, const std::vector<ExportItem>& items) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return e;
    auto issue = [&](size_t i) {
        const ExportItem& it = items[i];
        const size_t bytes = (size_t)it.rows * (it.widen ? 4 : 8);
        cudaError_t r = cudaMemcpyAsync(L.slot[i & 1], it.src, bytes, cudaMemcpyDeviceToHost, L.st);
        return r != cudaSuccess ? r : cudaEventRecord(L.ev[i & 1], L.st);
    };
    if (items.empty()) return cudaSuccess;
    if ((e = issue(0)) != cudaSuccess) return e;
    for (size_t i = 0; i < items.size(); i++) {
        // slot (i + 1) & 1 held item i - 1, already widened by this thread
        if (i + 1 < items.size() && (e = issue(i + 1)) != cudaSuccess) break;
        if ((e = cudaEventSynchronize(L.ev[i & 1])) != cudaSuccess) break;
        const ExportItem& it = items[i];
        if (it.widen) {
            const float* s = (const float*)L.slot[i & 1];
            double* d = (double*)it.dst;
            for (int64_t j = 0; j < it.rows; j++) d[j] = (double)s[j];
        } else {
            memcpy(it.dst, L.slot[i & 1], (size_t)it.rows * 8);
        }
    }
    // nothing may still land in the slots once the pool is handed on
    cudaError_t e2 = cudaStreamSynchronize(L.st);
    return e != cudaSuccess ? e : e2;
}

}  // namespace

namespace {

gt_status table_export_impl(const gt_table* t, const int32_t* columns, int32_t ncolumns, void* const* dst) {
    if (!t || ncolumns < 0 || (ncolumns > 0 && (!columns || !dst))) return GT_ERR_INVALID_ARGUMENT;
    for (int32_t k = 0; k < ncolumns; k++) {
        const int32_t c = columns[k];
        if (c < 0 || c >= GT_NUM_COLUMNS || !t->has[c] || !dst[k]) return GT_ERR_INVALID_ARGUMENT;
    }
    const int64_t N = t->n;
    if (N == 0 || ncolumns == 0) return GT_OK;
    ExportPool* pool = export_pool(t->device);
    if (!pool) return GT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(pool->mu);
    if (cudaSetDevice(t->device) != cudaSuccess || export_pool_init(*pool) != cudaSuccess) return GT_ERR_CUDA;
    // lanes: one per 256k rows, at most kExportLanes and half the host threads
    const int hw = std::max(1, (int)std::thread::hardware_concurrency() / 2);
    const int lanes = (int)std::max<int64_t>(1, std::min<int64_t>({kExportLanes, hw, (N + (1 << 18) - 1) >> 18}));
    std::vector<std::vector<ExportItem>> work(lanes);
    for (int l = 0; l < lanes; l++) {
        const int64_t r0 = N * l / lanes, r1 = N * (l + 1) / lanes;
        for (int32_t k = 0; k < ncolumns; k++) {
            const int32_t c = columns[k];
            const bool integer = c == GT_COL_FRAME || c == GT_COL_PARTICLE || c == GT_COL_DURATION;
            const TBuf& b = c == GT_COL_FRAME ? t->frame
                                              : (c == GT_COL_PARTICLE ? t->particle
                                                                      : (c == GT_COL_DURATION ? t->duration : t->col[c]));
            const int64_t chunk = (int64_t)(kExportSlot / (integer ? 8 : 4));
            for (int64_t r = r0; r < r1; r += chunk) {
                ExportItem it;
                it.rows = std::min(chunk, r1 - r);
                it.src = (const char*)b.p + (size_t)r * (integer ? 8 : 4);
                it.dst = (char*)dst[k] + (size_t)r * 8;
                it.widen = !integer;
                work[l].push_back(it);
            }
        }
    }
    std::vector<cudaError_t> err(lanes, cudaSuccess);
    std::vector<std::thread> th;
    // lanes whose thread cannot be started run on the calling thread
    for (int l = 1; l < lanes; l++) {
        try {
            th.emplace_back([&, l] { err[l] = export_lane(t->device, pool->lane[l], work[l]); });
        } catch (...) {
            err[l] = export_lane(t->device, pool->lane[l], work[l]);
        }
    }
    err[0] = export_lane(t->device, pool->lane[0], work[0]);
    for (auto& x : th) x.join();
    for (cudaError_t e : err)
        if (e != cudaSuccess) return GT_ERR_CUDA;
    return GT_OK;
}

}  // namespace

gt_status gt_table_export(const gt_table* t, const int32_t* columns, int32_t ncolumns, void* const* dst) {
    try {
        return table_export_impl(t, columns, ncolumns, dst);
    } catch (...) {
        return GT_ERR_INTERNAL;   // no C++ exception crosses the C ABI
    }
}

void gt_table_free(gt_table* t) {
    if (!t) return;
    cudaSetDevice(t->device);
    delete t;
}

}  // extern "C"
