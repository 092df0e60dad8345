// gt_proposal.cu — the learned proposal network behind the C ABI: creation
// (seeded He-normal weights), parameter access, training on the GPU with the
// network's own forward and backward kernels (gt_cnn.cu), and the per-cell
// output maps.  Inference inside a tracking call lives in gt_api.cu
// (gt_batch_learned); this file owns the network object.
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "gpu_tracking_b200.h"
#include "gt_proposal.h"

extern "C" int gt__ctx_device(const gt_ctx* ctx);
extern "C" cudaStream_t gt__ctx_stream(const gt_ctx* ctx);
extern "C" void gt__ctx_set_error(gt_ctx* ctx, const char* msg);

namespace gt {

cudaError_t proposal_repack(const gt_proposal* p, cudaStream_t st) {
    for (int l = 0; l < kCnnLayers; l++) {
        cudaError_t e = cnn_pack(p->params + cnn_layer_offset(l), l, false, (__nv_bfloat16*)(p->packed + p->off_f[l]),
                                 st);
        if (e != cudaSuccess) return e;
        if (l > 0) {
            e = cnn_pack(p->params + cnn_layer_offset(l), l, true, (__nv_bfloat16*)(p->packed + p->off_d[l]), st);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

namespace {

gt_status fail(gt_ctx* ctx, gt_status st, const std::string& msg) {
    if (ctx) gt__ctx_set_error(ctx, msg.c_str());
    return st;
}

#define PK(expr)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (expr);                                                                          \
        if (e_ != cudaSuccess)                                                                            \
            return fail(ctx, GT_ERR_CUDA, std::string("CUDA error ") + cudaGetErrorString(e_) + " at " #expr); \
    } while (0)

// Device buffers of one call, freed on every exit path.
struct Scratch {
    std::vector<void*> ptrs;
    cudaError_t get(void** p, size_t bytes) {
        *p = nullptr;
        cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 256));
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
    template <class T>
    cudaError_t get(T** p, size_t bytes) {
        return get((void**)p, bytes);
    }
    ~Scratch() {
        for (void* p : ptrs) cudaFree(p);
    }
};

int num_sms(int device) {
    int n = 148;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
    return n;
}

bool on_device_ptr(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

size_t dtype_size(int32_t dtype) { return dtype == GT_DTYPE_U16 ? 2 : dtype == GT_DTYPE_F32 ? 4 : 1; }

cudaError_t input_any(int32_t dtype, const void* frames, int64_t stride, int H, int W, const int4* crops, int nimg,
                      int Hc, int Wc, float mean, float scale, __nv_bfloat16* out, cudaStream_t st) {
    if (dtype == GT_DTYPE_U16)
        return cnn_input<uint16_t>((const uint16_t*)frames, stride, H, W, crops, nimg, Hc, Wc, mean, scale, out, st);
    if (dtype == GT_DTYPE_F32)
        return cnn_input<float>((const float*)frames, stride, H, W, crops, nimg, Hc, Wc, mean, scale, out, st);
    return cnn_input<uint8_t>((const uint8_t*)frames, stride, H, W, crops, nimg, Hc, Wc, mean, scale, out, st);
}

// One training step's buffers for `B` crops of CH x CW cells.
struct StepBufs {
    int4* crops = nullptr;
    __nv_bfloat16 *x = nullptr, *a1 = nullptr, *a2 = nullptr, *a3 = nullptr, *gout = nullptr, *g3 = nullptr,
                  *g2 = nullptr, *g1 = nullptr;
    float4* head = nullptr;
    float *wpart = nullptr, *lpart = nullptr;
    int wblocks = 0;
    cudaError_t alloc(Scratch& s, int B, int CH, int CW, int sms) {
        const size_t nc = (size_t)B * CH * CW;
        wblocks = 2 * sms;
        cudaError_t e;
        if ((e = s.get(&crops, (size_t)B * sizeof(int4))) != cudaSuccess) return e;
        if ((e = s.get(&x, nc * 16 * 2)) != cudaSuccess) return e;
        for (__nv_bfloat16** b : {&a1, &a2, &a3, &g3, &g2, &g1})
            if ((e = s.get(b, nc * 32 * 2)) != cudaSuccess) return e;
        if ((e = s.get(&gout, nc * 16 * 2)) != cudaSuccess) return e;
        if ((e = s.get(&head, nc * sizeof(float4))) != cudaSuccess) return e;
        if ((e = s.get(&wpart, cnn_wgrad_partial_floats(wblocks) * 4)) != cudaSuccess) return e;
        if ((e = s.get(&lpart, ((nc + 255) / 256) * 2 * 4)) != cudaSuccess) return e;
        return cudaSuccess;
    }
};

// Forward, loss and all gradients of one batch (crops already in sb.crops).
cudaError_t train_step_grads(const gt_proposal* p, int32_t dtype, const void* frames, int64_t stride, int H, int W,
                             const float4* tmap, int Hc, int Wc, int B, int CH, int CW, float pos_weight,
                             float lambda, StepBufs& sb, float* loss2, uint32_t* flags, int sms, cudaStream_t st) {
    const CnnNet net = p->views();
    cudaError_t e;
    if ((e = input_any(dtype, frames, stride, H, W, sb.crops, B, CH, CW, p->mean, p->scale, sb.x, st)) != cudaSuccess)
        return e;
    if ((e = cnn_forward(net, sb.x, B, CH, CW, sb.a1, sb.a2, sb.a3, sb.head, flags, sms, st)) != cudaSuccess) return e;
    int nlb = 0;
    if ((e = cnn_loss(sb.head, tmap, sb.crops, B, CH, CW, Hc, Wc, pos_weight, lambda, sb.gout, sb.lpart, &nlb, st)) !=
        cudaSuccess)
        return e;
    if ((e = cnn_loss_sum(sb.lpart, nlb, 1.0f / (float)((size_t)B * CH * CW), loss2, st)) != cudaSuccess) return e;
    float* g = p->grad;
    if ((e = cnn_wgrad(3, sb.a3, sb.gout, B, CH, CW, sb.wpart, sb.wblocks, g + cnn_layer_offset(3), st)) != cudaSuccess)
        return e;
    if ((e = cnn_backward_input(net, 3, sb.gout, sb.a3, B, CH, CW, sb.g3, flags, sms, st)) != cudaSuccess) return e;
    if ((e = cnn_wgrad(2, sb.a2, sb.g3, B, CH, CW, sb.wpart, sb.wblocks, g + cnn_layer_offset(2), st)) != cudaSuccess)
        return e;
    if ((e = cnn_backward_input(net, 2, sb.g3, sb.a2, B, CH, CW, sb.g2, flags, sms, st)) != cudaSuccess) return e;
    if ((e = cnn_wgrad(1, sb.a1, sb.g2, B, CH, CW, sb.wpart, sb.wblocks, g + cnn_layer_offset(1), st)) != cudaSuccess)
        return e;
    if ((e = cnn_backward_input(net, 1, sb.g2, sb.a1, B, CH, CW, sb.g1, flags, sms, st)) != cudaSuccess) return e;
    return cnn_wgrad(0, sb.x, sb.g1, B, CH, CW, sb.wpart, sb.wblocks, g + cnn_layer_offset(0), st);
}

// Labels -> per-cell targets of every frame.
gt_status build_targets(gt_ctx* ctx, Scratch& s, int64_t T, int Hc, int Wc, const int64_t* label_frame,
                        const float* label_y, const float* label_x, int64_t n, float4** tmap, cudaStream_t st) {
    std::vector<int32_t> lf;
    std::vector<float> ly, lx;
    lf.reserve(n);
    for (int64_t i = 0; i < n; i++) {
        if (label_frame[i] < 0 || label_frame[i] >= T) continue;
        lf.push_back((int32_t)label_frame[i]);
        ly.push_back(label_y[i]);
        lx.push_back(label_x[i]);
    }
    const int64_t m = (int64_t)lf.size();
    int32_t *dlf, *owner;
    float *dly, *dlx;
    PK(s.get(&dlf, m * 4));
    PK(s.get(&dly, m * 4));
    PK(s.get(&dlx, m * 4));
    PK(s.get(&owner, (size_t)T * Hc * Wc * 4));
    PK(s.get(tmap, (size_t)T * Hc * Wc * sizeof(float4)));
    if (m > 0) {
        PK(cudaMemcpyAsync(dlf, lf.data(), m * 4, cudaMemcpyHostToDevice, st));
        PK(cudaMemcpyAsync(dly, ly.data(), m * 4, cudaMemcpyHostToDevice, st));
        PK(cudaMemcpyAsync(dlx, lx.data(), m * 4, cudaMemcpyHostToDevice, st));
    }
    PK(cnn_labels(dlf, dly, dlx, m, (int)T, Hc, Wc, owner, *tmap, st));
    PK(cudaStreamSynchronize(st));  // the host label vectors go out of scope
    return GT_OK;
}

// Frames in device memory for the call (a copy when they are on the host).
gt_status device_frames(gt_ctx* ctx, Scratch& s, const void* frames, int32_t dtype, int64_t T, int H, int W,
                        const void** dev, cudaStream_t st) {
    if (on_device_ptr(frames)) {
        *dev = frames;
        return GT_OK;
    }
    void* d;
    const size_t bytes = (size_t)T * H * W * dtype_size(dtype);
    PK(s.get(&d, bytes));
    PK(cudaMemcpyAsync(d, frames, bytes, cudaMemcpyHostToDevice, st));
    *dev = d;
    return GT_OK;
}

gt_status check_dims(gt_ctx* ctx, int32_t dtype, int64_t T, int32_t H, int32_t W) {
    if (dtype != GT_DTYPE_U16 && dtype != GT_DTYPE_F32 && dtype != GT_DTYPE_U8)
        return fail(ctx, GT_ERR_INVALID_ARGUMENT, "dtype must be u16, f32 or u8");
    if (T <= 0 || H <= 0 || W <= 0) return fail(ctx, GT_ERR_EMPTY_ITERATOR, "no frames");
    return GT_OK;
}

}  // namespace
}  // namespace gt

using namespace gt;

extern "C" {

GT_API void gt_train_opts_default(gt_train_opts* o) {
    o->steps = 800;
    o->batch = 256;
    o->crop = 128;
    o->lr = 3e-3f;
    o->pos_weight = 8.0f;
    o->offset_weight = 1.0f;
    o->seed = 1;
}

GT_API int64_t gt_proposal_num_params(void) { return kCnnParams; }

GT_API gt_status gt_proposal_create(gt_ctx* ctx, uint64_t seed, gt_proposal** out) {
    if (!ctx || !out) return GT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    std::unique_ptr<gt_proposal> p(new gt_proposal());
    p->device = gt__ctx_device(ctx);
    cudaStream_t st = gt__ctx_stream(ctx);
    size_t off = 0;
    for (int l = 0; l < kCnnLayers; l++) {
        p->off_f[l] = off;
        off += (cnn_packed_bytes(l, false) + 255) & ~(size_t)255;
        if (l > 0) {
            p->off_d[l] = off;
            off += (cnn_packed_bytes(l, true) + 255) & ~(size_t)255;
        }
    }
    p->packed_bytes = off;
    PK(cudaMalloc(&p->params, kCnnParams * 4));
    PK(cudaMalloc(&p->packed, p->packed_bytes));
    // He-normal convolution weights, zero biases; the score bias starts at a
    // 1% prior and the head weights small
    std::vector<float> h(kCnnParams, 0.0f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < kCnnLayers; l++) {
        const int cin = kCnnCin[l], cout = kCnnCout[l];
        const float sd = l == 3 ? 0.1f * std::sqrt(1.0f / (9.0f * cin)) : std::sqrt(2.0f / (9.0f * cin));
        std::normal_distribution<float> nd(0.0f, sd);
        float* w = h.data() + cnn_layer_offset(l);
        for (int i = 0; i < cout * cin * 9; i++) w[i] = nd(rng);
    }
    h[cnn_layer_offset(3) + 3 * 32 * 9] = -4.6f;
    PK(cudaMemcpyAsync(p->params, h.data(), kCnnParams * 4, cudaMemcpyHostToDevice, st));
    PK(proposal_repack(p.get(), st));
    PK(cudaStreamSynchronize(st));
    *out = p.release();
    return GT_OK;
}

GT_API void gt_proposal_destroy(gt_proposal* p) {
    if (!p) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(p->device);
    for (void* q : {(void*)p->params, (void*)p->adam_m, (void*)p->adam_v, (void*)p->grad, (void*)p->packed})
        if (q) cudaFree(q);
    cudaSetDevice(cur);
    delete p;
}

GT_API gt_status gt_proposal_set(gt_ctx* ctx, gt_proposal* p, const float* params, float mean, float scale,
                                 float threshold) {
    if (!ctx || !p) return GT_ERR_INVALID_ARGUMENT;
    if (!(scale > 0.0f) || !std::isfinite(mean) || !std::isfinite(scale) || std::isnan(threshold))
        return fail(ctx, GT_ERR_INVALID_ARGUMENT, "mean and scale must be finite, scale > 0, threshold not NaN");
    cudaStream_t st = gt__ctx_stream(ctx);
    p->mean = mean;
    p->scale = scale;
    p->threshold = threshold;
    if (params) {
        PK(cudaMemcpyAsync(p->params, params, kCnnParams * 4, cudaMemcpyHostToDevice, st));
        PK(proposal_repack(p, st));
        PK(cudaStreamSynchronize(st));
    }
    return GT_OK;
}

GT_API gt_status gt_proposal_get(gt_ctx* ctx, const gt_proposal* p, float* params, float* mean, float* scale,
                                 float* threshold) {
    if (!ctx || !p) return GT_ERR_INVALID_ARGUMENT;
    if (params) {
        cudaStream_t st = gt__ctx_stream(ctx);
        PK(cudaMemcpyAsync(params, p->params, kCnnParams * 4, cudaMemcpyDeviceToHost, st));
        PK(cudaStreamSynchronize(st));
    }
    if (mean) *mean = p->mean;
    if (scale) *scale = p->scale;
    if (threshold) *threshold = p->threshold;
    return GT_OK;
}

GT_API gt_status gt_proposal_train(gt_ctx* ctx, gt_proposal* p, const void* frames, int32_t dtype, int64_t T,
                                   int32_t H, int32_t W, const int64_t* label_frame, const float* label_y,
                                   const float* label_x, int64_t n_labels, const gt_train_opts* opts,
                                   float* loss_out) {
    if (!ctx || !p || !frames || !opts) return GT_ERR_INVALID_ARGUMENT;
    if (n_labels > 0 && (!label_frame || !label_y || !label_x))
        return fail(ctx, GT_ERR_INVALID_ARGUMENT, "null label arrays");
    {
        gt_status s0 = check_dims(ctx, dtype, T, H, W);
        if (s0 != GT_OK) return s0;
    }
    const gt_train_opts o = *opts;
    if (o.steps < 0 || o.batch <= 0 || o.crop <= 0 || o.crop % 4 != 0 || o.crop > H || o.crop > W ||
        !(o.lr > 0.0f) || !(o.pos_weight > 0.0f) || !(o.offset_weight >= 0.0f))
        return fail(ctx, GT_ERR_INVALID_ARGUMENT,
                    "train options: steps >= 0, batch > 0, crop a positive multiple of 4 within the frame, lr > 0, "
                    "pos_weight > 0, offset_weight >= 0");
    if (n_labels >= 0x7F7F7F7F) return fail(ctx, GT_ERR_CAPACITY_EXCEEDED, "too many labels");
    cudaStream_t st = gt__ctx_stream(ctx);
    const int sms = num_sms(p->device);
    const int Hc = (H + 3) / 4, Wc = (W + 3) / 4, CH = o.crop / 4, CW = o.crop / 4;
    Scratch s;
    const void* dframes = nullptr;
    {
        gt_status r = device_frames(ctx, s, frames, dtype, T, H, W, &dframes, st);
        if (r != GT_OK) return r;
    }
    float4* tmap = nullptr;
    {
        gt_status r = build_targets(ctx, s, T, Hc, Wc, label_frame, label_y, label_x, n_labels, &tmap, st);
        if (r != GT_OK) return r;
    }
    if (!p->adam_m) {
        PK(cudaMalloc(&p->adam_m, kCnnParams * 4));
        PK(cudaMalloc(&p->adam_v, kCnnParams * 4));
        PK(cudaMemsetAsync(p->adam_m, 0, kCnnParams * 4, st));
        PK(cudaMemsetAsync(p->adam_v, 0, kCnnParams * 4, st));
    }
    if (!p->grad) PK(cudaMalloc(&p->grad, kCnnParams * 4));
    StepBufs sb;
    PK(sb.alloc(s, o.batch, CH, CW, sms));
    float* loss_dev = nullptr;
    uint32_t* flags = nullptr;
    PK(s.get(&loss_dev, (size_t)std::max(o.steps, 1) * 2 * 4));
    PK(s.get(&flags, 16));
    PK(cudaMemsetAsync(flags, 0, 16, st));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int stp = 0; stp < o.steps; stp++) {
        PK(cnn_crops(o.seed, (uint32_t)stp, o.batch, (int)T, Hc, Wc, CH, CW, sb.crops, st));
        PK(train_step_grads(p, dtype, dframes, (int64_t)H * W, H, W, tmap, Hc, Wc, o.batch, CH, CW, o.pos_weight,
                            o.offset_weight, sb, loss_dev + 2 * stp, flags, sms, st));
        p->adam_t++;
        const double frac = o.steps > 1 ? (double)stp / (double)(o.steps - 1) : 0.0;
        const double lr = o.lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(M_PI * frac)));
        const double corr = std::sqrt(1.0 - std::pow((double)b2, (double)p->adam_t)) /
                            (1.0 - std::pow((double)b1, (double)p->adam_t));
        PK(cnn_adam(p->params, p->adam_m, p->adam_v, p->grad, kCnnParams, (float)(lr * corr), b1, b2, eps, st));
        PK(proposal_repack(p, st));
    }
    uint32_t fl = 0;
    PK(cudaMemcpyAsync(&fl, flags, 4, cudaMemcpyDeviceToHost, st));
    if (loss_out && o.steps > 0)
        PK(cudaMemcpyAsync(loss_out, loss_dev, (size_t)o.steps * 2 * 4, cudaMemcpyDeviceToHost, st));
    PK(cudaStreamSynchronize(st));
    if (fl & kFlagTensorTimeout) return fail(ctx, GT_ERR_INTERNAL, "a tensor-core kernel timed out");
    return GT_OK;
}

GT_API gt_status gt_proposal_maps(gt_ctx* ctx, const gt_proposal* p, const void* frames, int32_t dtype, int64_t T,
                                  int32_t H, int32_t W, float* maps) {
    if (!ctx || !p || !frames || !maps) return GT_ERR_INVALID_ARGUMENT;
    {
        gt_status s0 = check_dims(ctx, dtype, T, H, W);
        if (s0 != GT_OK) return s0;
    }
    cudaStream_t st = gt__ctx_stream(ctx);
    const int sms = num_sms(p->device);
    const int Hc = (H + 3) / 4, Wc = (W + 3) / 4;
    const size_t cells = (size_t)Hc * Wc;
    const int G = (int)std::max<int64_t>(1, std::min<int64_t>(T, (int64_t)((256u << 20) / (cells * 64 + 1))));
    Scratch s;
    const void* dframes = nullptr;
    {
        gt_status r = device_frames(ctx, s, frames, dtype, T, H, W, &dframes, st);
        if (r != GT_OK) return r;
    }
    __nv_bfloat16 *x, *pa, *pb;
    float4* head;
    uint32_t* flags;
    PK(s.get(&x, (size_t)G * cells * 32));
    PK(s.get(&pa, (size_t)G * cells * 64));
    PK(s.get(&pb, (size_t)G * cells * 64));
    PK(s.get(&head, (size_t)G * cells * 16));
    PK(s.get(&flags, 16));
    PK(cudaMemsetAsync(flags, 0, 16, st));
    const CnnNet net = p->views();
    const size_t px = (size_t)H * W * dtype_size(dtype);
    for (int64_t t0 = 0; t0 < T; t0 += G) {
        const int ng = (int)std::min<int64_t>(G, T - t0);
        PK(input_any(dtype, (const uint8_t*)dframes + (size_t)t0 * px, (int64_t)H * W, H, W, nullptr, ng, Hc, Wc,
                     p->mean, p->scale, x, st));
        PK(cnn_forward(net, x, ng, Hc, Wc, pa, pb, pa, head, flags, sms, st));
        PK(cudaMemcpyAsync(maps + (size_t)t0 * cells * 4, head, (size_t)ng * cells * 16, cudaMemcpyDeviceToHost, st));
    }
    uint32_t fl = 0;
    PK(cudaMemcpyAsync(&fl, flags, 4, cudaMemcpyDeviceToHost, st));
    PK(cudaStreamSynchronize(st));
    if (fl & kFlagTensorTimeout) return fail(ctx, GT_ERR_INTERNAL, "a tensor-core kernel timed out");
    return GT_OK;
}

// Test hook (exported, not part of the public header): loss and gradient of
// one batch of given crops (int32 triples frame, row, column in pixels,
// multiples of 4) without an update.  grad_out: kCnnParams floats, loss_out:
// the score and offset losses.
GT_API gt_status gt__proposal_loss_grad(gt_ctx* ctx, gt_proposal* p, const void* frames, int32_t dtype, int64_t T,
                                        int32_t H, int32_t W, const int64_t* label_frame, const float* label_y,
                                        const float* label_x, int64_t n_labels, const int32_t* crops, int32_t B,
                                        int32_t crop, float pos_weight, float offset_weight, float* grad_out,
                                        float* loss_out) {
    if (!ctx || !p || !frames || !crops || !grad_out || !loss_out || B <= 0 || crop <= 0 || crop % 4)
        return GT_ERR_INVALID_ARGUMENT;
    {
        gt_status s0 = check_dims(ctx, dtype, T, H, W);
        if (s0 != GT_OK) return s0;
    }
    for (int32_t b = 0; b < B; b++) {
        const int32_t f = crops[3 * b], y = crops[3 * b + 1], x = crops[3 * b + 2];
        if (f < 0 || f >= T || y < 0 || x < 0 || y % 4 || x % 4 || y + crop > H || x + crop > W)
            return fail(ctx, GT_ERR_INVALID_ARGUMENT, "crop outside its frame or not cell-aligned");
    }
    cudaStream_t st = gt__ctx_stream(ctx);
    const int sms = num_sms(p->device);
    const int Hc = (H + 3) / 4, Wc = (W + 3) / 4, CH = crop / 4, CW = crop / 4;
    Scratch s;
    const void* dframes = nullptr;
    {
        gt_status r = device_frames(ctx, s, frames, dtype, T, H, W, &dframes, st);
        if (r != GT_OK) return r;
    }
    float4* tmap = nullptr;
    {
        gt_status r = build_targets(ctx, s, T, Hc, Wc, label_frame, label_y, label_x, n_labels, &tmap, st);
        if (r != GT_OK) return r;
    }
    if (!p->grad) PK(cudaMalloc(&p->grad, kCnnParams * 4));
    StepBufs sb;
    PK(sb.alloc(s, B, CH, CW, sms));
    std::vector<int4> hc(B);
    for (int32_t b = 0; b < B; b++) hc[b] = make_int4(crops[3 * b], crops[3 * b + 1], crops[3 * b + 2], 0);
    PK(cudaMemcpyAsync(sb.crops, hc.data(), B * sizeof(int4), cudaMemcpyHostToDevice, st));
    float* loss_dev;
    uint32_t* flags;
    PK(s.get(&loss_dev, 16));
    PK(s.get(&flags, 16));
    PK(cudaMemsetAsync(flags, 0, 16, st));
    PK(train_step_grads(p, dtype, dframes, (int64_t)H * W, H, W, tmap, Hc, Wc, B, CH, CW, pos_weight, offset_weight,
                        sb, loss_dev, flags, sms, st));
    uint32_t fl = 0;
    PK(cudaMemcpyAsync(grad_out, p->grad, kCnnParams * 4, cudaMemcpyDeviceToHost, st));
    PK(cudaMemcpyAsync(loss_out, loss_dev, 8, cudaMemcpyDeviceToHost, st));
    PK(cudaMemcpyAsync(&fl, flags, 4, cudaMemcpyDeviceToHost, st));
    PK(cudaStreamSynchronize(st));
    if (fl & kFlagTensorTimeout) return fail(ctx, GT_ERR_INTERNAL, "a tensor-core kernel timed out");
    return GT_OK;
}

}  // extern "C"
