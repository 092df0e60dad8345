// gt_kernels.h — host-visible launch interface of the engine's kernels.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "gt_internal.cuh"

namespace gt {

constexpr int kMaxRadii = 256;
constexpr int kLinkRowBins = 512;   // row bins per group of the windowed linker's neighbour search

struct FinalizeConsts {
    int32_t H, W;
    int32_t log_style;
    int32_t prune;              // LoG: overlap_threshold < 1
    float overlap_threshold;
    int32_t filter_close;
    float separation;
    int32_t band;               // candidate-row band holding every filter_close neighbour, -1 = all
    int32_t doughnut;
    int32_t presorted;          // characterize_points: rows stay in input order
    uint64_t scratch_per_frame; // bytes of global sort scratch per frame (0 = shared memory only)
    uint8_t radius_rank_desc[kMaxRadii];
};

// One frame of a ragged batch (frames of many videos and sizes in one launch
// per stage): its pixels, where its processed image starts in the batch's
// buffer, its size, whether 4-pixel loads of its rows are aligned, and the
// slot of the call's per-frame results (detections, kept count) it fills.
struct RaggedFrame {
    const void* raw;
    int64_t proc_off;
    int32_t H, W;
    int32_t vec_ok;
    int32_t out_slot;
};
// One bandpass tile of a ragged batch: frame slot, first output column, rows [r0, r1).
struct StripTask {
    int32_t slot, c0, r0, r1;
};

struct TableCols {
    int64_t* frame;
    float* col[GT_NUM_COLUMNS];
    int64_t* particle;
    int64_t* duration;
};

// LoG per-radius tap tables live in global memory: taps_g/taps_d of radius k
// start at tap_off[k] and have 2*rint[k]+1 entries.
struct LogConsts {
    int32_t H, W, n_radii;
    float thr;  // pic_std * snr * rough_snr_factor when no per-frame std is given
    const float* frame_std;  // per-frame std of the chunk (nullptr: use thr)
    float snr, rough;
};

// ---- learned proposal network (gt_cnn.cu): 4 layers of 3x3 convolutions
// over 4x4-pixel cells; layer l maps kCnnCin[l] to kCnnCout[l] channels.
constexpr int kCnnLayers = 4;
constexpr int kCnnCin[kCnnLayers] = {16, 32, 32, 32};
constexpr int kCnnCout[kCnnLayers] = {32, 32, 32, 3};
constexpr int kCnnParams = 32 * 16 * 9 + 32 + 2 * (32 * 32 * 9 + 32) + 3 * 32 * 9 + 3;
constexpr int cnn_layer_offset(int l) {
    return l == 0 ? 0 : cnn_layer_offset(l - 1) + kCnnCout[l - 1] * kCnnCin[l - 1] * 9 + kCnnCout[l - 1];
}
// Device views of one network: packed BF16 UMMA operands of the forward
// convolutions (wf) and of the input-gradient convolutions (wd, layers 1-3),
// fp32 biases.
struct CnnNet {
    const uint8_t* wf[kCnnLayers];
    const uint8_t* wd[kCnnLayers];
    const float* bias[kCnnLayers];
};
size_t cnn_packed_bytes(int layer, bool backward);
cudaError_t cnn_pack(const float* W, int layer, bool backward, __nv_bfloat16* dst, cudaStream_t st);
template <typename T>
cudaError_t cnn_input(const T* frames, int64_t frame_stride, int H, int W, const int4* crops, int nimg, int Hc,
                      int Wc, float mean, float scale, __nv_bfloat16* out, cudaStream_t st);
cudaError_t cnn_forward(const CnnNet& net, const __nv_bfloat16* x, int nimg, int Hc, int Wc, __nv_bfloat16* a1,
                        __nv_bfloat16* a2, __nv_bfloat16* a3, float4* head, uint32_t* flags, int num_sms,
                        cudaStream_t st);
cudaError_t cnn_backward_input(const CnnNet& net, int layer, const __nv_bfloat16* gout, const __nv_bfloat16* act_below,
                               int nimg, int Hc, int Wc, __nv_bfloat16* gin, uint32_t* flags, int num_sms,
                               cudaStream_t st);
size_t cnn_wgrad_partial_floats(int nblocks);
cudaError_t cnn_wgrad(int layer, const __nv_bfloat16* X, const __nv_bfloat16* G, int nimg, int Hc, int Wc,
                      float* partial, int nblocks, float* grad, cudaStream_t st);
cudaError_t cnn_labels(const int32_t* lf, const float* ly, const float* lx, int64_t n, int T, int Hc, int Wc,
                       int32_t* owner, float4* tmap, cudaStream_t st);
cudaError_t cnn_crops(uint32_t seed, uint32_t step, int nimg, int T, int Hc, int Wc, int CH, int CW, int4* crops,
                      cudaStream_t st);
cudaError_t cnn_loss(const float4* head, const float4* tmap, const int4* crops, int nimg, int CH, int CW, int Hc_f,
                     int Wc_f, float pos_weight, float lambda, __nv_bfloat16* grad, float* partial, int* nblocks,
                     cudaStream_t st);
cudaError_t cnn_adam(float* p, float* m, float* v, const float* g, int n, float lr_t, float b1, float b2, float eps,
                     cudaStream_t st);
cudaError_t cnn_loss_sum(const float* partial, int nblocks, float inv, float* out, cudaStream_t st);
cudaError_t cnn_proposals(const float4* head, int nimg, int Hc, int Wc, int H, int W, int margin, float thr,
                          uint32_t* cand_count, uint32_t* cand_keys, uint32_t cand_cap, uint32_t* flags,
                          cudaStream_t st);
// walk + characterize from seeds with the processed image built per seed
size_t walk_local_smem_bytes(int circle, int R);
template <typename T>
cudaError_t launch_walk_local(const T* frames, int64_t frame_stride, const LocateConsts& c, int nframes,
                              const uint32_t* cand_count, const uint32_t* cand_keys, uint32_t cand_cap,
                              const int32_t* angle_off, const float2* angles, Feature* feats, uint32_t* feat_count,
                              uint32_t feat_cap, uint32_t* flags, cudaStream_t st);

// Per-frame std (snr / minmass_snr), the reference's reduction tree.
bool std_reduction_exact(int64_t N);
size_t std_scratch_floats(int64_t N, int nframes);
template <typename T>
cudaError_t launch_frame_std(const T* frames, int64_t frame_stride, int nframes, int64_t N, const uint8_t* mask,
                             const uint32_t* divisors, float* out_std, float* scratch, cudaStream_t st);
// adaptive_background passes over the walked rows of a chunk
cudaError_t launch_adaptive_init(uint32_t* counters, uint32_t N, uint8_t* status, size_t n_status, int nframes,
                                 cudaStream_t st);
cudaError_t launch_adaptive_pass(const Feature* feats, const uint32_t* count, uint32_t feat_cap, uint8_t* status,
                                 const float* frame_std, float minmass, float minmass_snr, float snr, uint8_t* mask,
                                 uint32_t* counters, int32_t H, int32_t W, int32_t circle, int nframes,
                                 cudaStream_t st);
cudaError_t launch_adaptive_compact(Feature* feats, uint32_t* count, uint32_t feat_cap, const uint8_t* status,
                                    int nframes, cudaStream_t st);
// illumination correction: one separable smoothing pass of nframes profiles
// (stride H*W in the output) and frame / profile (prof_stride 0: one profile)
template <typename TIn>
cudaError_t launch_illum_smooth(const TIn* in, int64_t in_stride, float* out, int H, int W, int dim, const float* g,
                                int rint, int nframes, cudaStream_t st);
template <typename T>
cudaError_t launch_illum_divide(const T* frames, int64_t frame_stride, const float* prof, int64_t prof_stride,
                                float* out, int64_t out_stride, int nframes, cudaStream_t st);

size_t bandpass_smem_bytes(int R, int kd, bool cand);
size_t finalize_smem_bytes();
size_t laplace_smem_bytes(int rint);

template <typename T>
cudaError_t launch_bandpass(const T* frames, int64_t frame_stride, float* processed, const LocateConsts& c,
                            int nframes, bool cand, uint32_t* cand_count, uint32_t* cand_keys, uint32_t cand_cap,
                            uint32_t* flags, cudaStream_t st);

// Streaming strip kernel for the specialised (radius, dilation) pairs; returns
// false when the pair has no specialisation (the tile kernel is used then).
// The strip kernel over a ragged batch: persistent CTAs (grid of them) take
// the tiles of `tasks` (*ntasks of them, in device memory) in turn; candidate
// lists per frame slot.  False when no specialisation exists (as launch_strip).
template <typename T>
bool launch_strip_ragged(const RaggedFrame* frames, const StripTask* tasks, const int32_t* ntasks, int grid,
                         float* processed, const LocateConsts& c, uint32_t* cand_count, uint32_t* cand_keys,
                         uint32_t cand_cap, uint32_t* flags, cudaStream_t st, cudaError_t* err);
// CTAs of the strip kernel resident per SM for these parameters (0: no specialisation)
template <typename T>
int strip_blocks_per_sm(const LocateConsts& c);
// Output columns of one strip tile for these parameters (0: no specialisation)
template <typename T>
int strip_tile_width(const LocateConsts& c);
template <typename T>
bool launch_strip(const T* frames, int64_t frame_stride, float* processed, const LocateConsts& c, int nframes,
                  uint32_t* cand_count, uint32_t* cand_keys, uint32_t cand_cap, uint32_t* flags, cudaStream_t st,
                  cudaError_t* err);
// The processed image alone through the strip kernel, for smoothing radii
// 3..10 (the LoG style's bandpass, which takes no local-maximum candidates):
// the same processed values as bandpass_kernel<T, false>.  False when the
// radius has no specialisation or integer pixels lack the proven division;
// cand_count / cand_keys are never written.
template <typename T>
bool launch_strip_processed(const T* frames, int64_t frame_stride, float* processed, const LocateConsts& c,
                            int nframes, uint32_t* cand_count, uint32_t* cand_keys, uint32_t* flags, cudaStream_t st,
                            cudaError_t* err);

// True when fma(x, zh, x*zl) equals IEEE x/d for every x in [1, 2) (checked
// on the device once per (d, zh, zl) and remembered).
bool const_div_proven(float d, float zh, float zl, cudaStream_t st);

template <typename T>
cudaError_t launch_walk(const float* processed, const T* frames, int64_t frame_stride, const LocateConsts& c,
                        int nframes, int n_slots, const uint32_t* cand_count, const uint32_t* cand_keys,
                        uint32_t cand_cap, uint32_t max_cands, const float* radii, const int32_t* angle_off,
                        const float2* angles, Feature* feats, uint32_t* feat_count, uint32_t feat_cap,
                        uint32_t* flags, cudaStream_t st, const RaggedFrame* rf = nullptr);

template <typename T>
cudaError_t launch_characterize_points(const float* processed, const T* frames, int64_t frame_stride,
                                       const LocateConsts& c, const float* pts, const int64_t* grp_off,
                                       const int32_t* grp_frame, int32_t g0, int ngroups, int64_t max_pts,
                                       const float2* angles, const int32_t* angle_off, int32_t n_angle_tabs,
                                       int32_t has_r, Feature* feats, uint32_t* feat_count, uint32_t feat_cap,
                                       cudaStream_t st);

// rf (optional): per-slot frames of a ragged batch (pixels and size replace
// frames / frame_index / fc.H, fc.W)
template <typename T>
cudaError_t launch_finalize(const Feature* feats, const uint32_t* feat_count, uint32_t feat_cap, Feature* out,
                            uint32_t* kept_count, uint8_t* gscratch, const FinalizeConsts& fc, const T* frames,
                            int64_t frame_stride, const int32_t* frame_index, const short2* dn_inds,
                            const int4* dn_meta, uint32_t* flags, int ngroups, cudaStream_t st,
                            const RaggedFrame* rf = nullptr);

cudaError_t launch_scatter(const Feature* feats, uint32_t feat_cap, const uint32_t* kept_count, uint32_t max_kept,
                           const int64_t* row_off, const int64_t* frame_number, const TableCols& tab, int32_t g0,
                           int ngroups, cudaStream_t st);

// LoG
template <typename T>
cudaError_t launch_laplace(const T* frames, int64_t frame_stride, float* planes, const LogConsts& lc,
                           const float* taps_g, const float* taps_d, const int32_t* tap_off, const int32_t* rints,
                           const float* norm_g, const float* norm_d, int max_rint, int nframes, cudaStream_t st);

cudaError_t launch_logspace_max(const float* planes, const float* processed, const LogConsts& lc, int nframes,
                                uint32_t* cand_count, uint32_t* cand_keys, uint32_t cand_cap, uint32_t* flags,
                                cudaStream_t st);

// fused scale space (gt_logss.cu): the LoG planes of every radius and their
// 3x3x3 maxima in one pass over the frame, for rint <= kLogSSMaxR
constexpr int kLogSSMaxR = 32;
size_t log_scale_space_smem_bytes(int max_rint, int ntaps_total);
bool log_scale_space_supported(int max_rint, int ntaps_total);
template <typename T>
cudaError_t launch_log_scale_space(const T* frames, int64_t frame_stride, const float* processed, const LogConsts& lc,
                                   const float* taps_g, const float* taps_d, const int32_t* tap_off,
                                   const int32_t* rints, const float* norm_g, const float* norm_d, int max_rint,
                                   int ntaps_total, int nframes, uint32_t* cand_count, uint32_t* cand_keys,
                                   uint32_t cand_cap, uint32_t* flags, const float* h_taps_g, const float* h_taps_d,
                                   const int32_t* h_tap_off, const int32_t* h_rints, cudaStream_t st);

// mean frame (src/execute_gpu.rs:819-847)
template <typename T>
cudaError_t launch_mean_frame(const T* frames, int64_t T_, int64_t npix, float* out, cudaStream_t st);

// Linking --------------------------------------------------------------
// Points are addressed in one of two ways:
//   compact   point p of group g is p in [goff[g], goff[g+1]) and its
//             coordinates are px[p], py[p] (table columns);
//   slot      point j of group g is p = g*slot_stride + j, j < gcount[g], and
//             its coordinates are px[p*xy_stride] (per-frame result slots,
//             read in place while later frames are still being located).
struct LinkInput {
    const float* px = nullptr;          // row coordinate of every point ("y" column)
    const float* py = nullptr;          // column coordinate ("x" column)
    int32_t xy_stride = 1;              // floats between consecutive points
    const int64_t* goff = nullptr;      // compact: group offsets, ngroups+1
    const int32_t* pgroup = nullptr;    // compact: group of every point
    const uint32_t* gcount = nullptr;   // slot: points per group
    int64_t slot_stride = 0;            // slot: slots per group (0 = compact)
    const int32_t* vgrp = nullptr;      // group range of every video, nvideos+1
    const uint8_t* reset = nullptr;     // reset flag per group (linker_reset_points)
    int32_t ngroups = 0, nvideos = 0;
    int32_t groups_ready = 0;           // groups whose points exist (forward lists stop there)
    int64_t npoints = 0;                // compact: points; slot: ngroups*slot_stride
    float radius = 0.0f;
    int32_t memory = 0;
};

struct LinkLists {
    // per point p and k in 1..K: forward (dests in group+k) and backward
    // (sources in group-k) neighbour lists, ascending point index; the
    // offsets of (p, k) are at [(p - pbase)*K + k - 1] and the next entry
    int64_t* f_off = nullptr;
    int64_t* b_off = nullptr;
    int32_t* f_pts = nullptr;
    int32_t* b_pts = nullptr;
    float* b_dist = nullptr;      // squared distances of the backward lists
    uint32_t* srt = nullptr;      // per group: points sorted by row key
    int64_t pbase = 0;            // first point the offset arrays cover
    int64_t f_cap = -1, b_cap = -1;  // entries f_pts / b_pts hold (-1: sized exactly)
    int64_t f_entries = -1;          // forward entries of lists sized exactly (-1: not known)
    // optional row-bin index of the sorted groups: for group g, entry
    // g * (kLinkRowBins + 1) + b is the first sorted position whose row falls
    // in bin b or later (bin = clamp(floor(row / bin_w), 0, kLinkRowBins - 1),
    // rows that are NaN after every bin); nullptr = bisect the rows instead
    const int32_t* bins = nullptr;
    float bin_w = 0.0f;
};

struct LinkScratch {
    uint8_t* base;
    size_t bytes_per_video;
    int32_t max_group;
    int64_t max_edges;   // max over groups of the per-step backward-edge total
    int64_t max_points;  // per-video point space (compact: points of the video)
};

// Linker state carried from one window of frames to the next (slot mode).
struct LinkState {
    long long counter, frame;
    int32_t prevg, head;
};

// Frames [g0, g1) of video 0 linked by one launch; g0 < 0 = every video whole.
struct LinkWindow {
    int32_t g0 = -1, g1 = -1;
    int32_t first = 1, last = 1;   // initialise state / run Linker::finish
    int32_t init_points = 1;       // clear the per-point arrays in the kernel
    LinkState* state = nullptr;
};

struct LinkOutput {
    int64_t* ids;        // per point
    int64_t* counter;    // per video: ids used by the last segment
    int64_t* dur;        // per video region of npoints_video: durations by id
    int64_t* vpoff;      // per video: first point index (nvideos+1)
    uint32_t* flags;     // per video error flags
};

cudaError_t link_sort_groups(const LinkInput& in, uint32_t* srt, uint8_t* scratch, size_t scratch_per_group,
                             int max_group, cudaStream_t st);
// groups [g0, g1) only
// groups [g0, g1) only; with bins, also their row-bin index (LinkLists::bins)
cudaError_t link_sort_groups_range(const LinkInput& in, uint32_t* srt, int g0, int g1, int32_t* bins, float bin_w,
                                   cudaStream_t st);
cudaError_t link_count_lists(const LinkInput& in, const uint32_t* srt, int64_t* f_cnt, int64_t* b_cnt,
                             cudaStream_t st);
cudaError_t link_fill_lists(const LinkInput& in, const LinkLists& L, cudaStream_t st);
// points [p0, p1) only; f_cnt/b_cnt and L's offsets are relative to p0 (L.pbase == p0)
cudaError_t link_count_lists_range(const LinkInput& in, const uint32_t* srt, int64_t p0, int64_t p1,
                                   int64_t* f_cnt, int64_t* b_cnt, uint32_t* flags, cudaStream_t st);
cudaError_t link_fill_lists_range(const LinkInput& in, const LinkLists& L, int64_t p1, uint32_t* flags,
                                  cudaStream_t st);
size_t link_scratch_bytes(int32_t max_group, int64_t max_edges, int64_t npoints_video, int32_t memory);
// byte offsets of the per-point arrays the host may clear itself (LinkWindow::init_points == 0):
// idstamp and srcstamp to 0xFF bytes, firstpos to zero
void link_scratch_point_arrays(int32_t max_group, int64_t max_edges, int64_t npoints_video, int32_t memory,
                               size_t* idstamp, size_t* srcstamp, size_t* firstpos);
cudaError_t link_run(const LinkInput& in, const LinkLists& L, const LinkScratch& S, const LinkOutput& out,
                     cudaStream_t st);
cudaError_t link_run_window(const LinkInput& in, const LinkLists& L, const LinkScratch& S, const LinkOutput& out,
                            const LinkWindow& w, cudaStream_t st);
cudaError_t link_durations(const LinkInput& in, const LinkOutput& out, int64_t* row_dur, cudaStream_t st);
// slot mode: particle ids (through the f32 round trip) and durations of every
// point written to table rows row_off[g] + j
cudaError_t link_slot_rows(const LinkInput& in, const LinkOutput& out, const int64_t* row_off, int64_t* particle,
                           int64_t* row_dur, cudaStream_t st);

}  // namespace gt
