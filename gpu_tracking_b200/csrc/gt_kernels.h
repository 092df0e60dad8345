// gt_kernels.h — host-visible launch interface of the engine's kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gt_internal.cuh"

namespace gt {

constexpr int kMaxRadii = 256;

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
    float thr;  // pic_std * snr * rough_snr_factor
};

size_t bandpass_smem_bytes(int R, int kd, bool cand);
size_t finalize_smem_bytes();
size_t laplace_smem_bytes(int rint);

template <typename T>
cudaError_t launch_bandpass(const T* frames, int64_t frame_stride, float* processed, const LocateConsts& c,
                            int nframes, bool cand, uint32_t* cand_count, uint32_t* cand_keys, uint32_t cand_cap,
                            uint32_t* flags, cudaStream_t st);

// Streaming strip kernel for the specialised (radius, dilation) pairs; returns
// false when the pair has no specialisation (the tile kernel is used then).
template <typename T>
bool launch_strip(const T* frames, int64_t frame_stride, float* processed, const LocateConsts& c, int nframes,
                  uint32_t* cand_count, uint32_t* cand_keys, uint32_t cand_cap, uint32_t* flags, cudaStream_t st,
                  cudaError_t* err);

template <typename T>
cudaError_t launch_walk(const float* processed, const T* frames, int64_t frame_stride, const LocateConsts& c,
                        int nframes, int n_slots, const uint32_t* cand_count, const uint32_t* cand_keys,
                        uint32_t cand_cap, uint32_t max_cands, const float* radii, const int32_t* angle_off,
                        const float2* angles, Feature* feats, uint32_t* feat_count, uint32_t feat_cap,
                        uint32_t* flags, cudaStream_t st);

template <typename T>
cudaError_t launch_characterize_points(const float* processed, const T* frames, int64_t frame_stride,
                                       const LocateConsts& c, const float* pts, const int64_t* grp_off,
                                       const int32_t* grp_frame, int32_t g0, int ngroups, int64_t max_pts,
                                       const float2* angles, const int32_t* angle_off, int32_t n_angle_tabs,
                                       int32_t has_r, Feature* feats, uint32_t* feat_count, uint32_t feat_cap,
                                       cudaStream_t st);

template <typename T>
cudaError_t launch_finalize(const Feature* feats, const uint32_t* feat_count, uint32_t feat_cap, Feature* out,
                            uint32_t* kept_count, uint8_t* gscratch, const FinalizeConsts& fc, const T* frames,
                            int64_t frame_stride, const int32_t* frame_index, const short2* dn_inds,
                            const int4* dn_meta, uint32_t* flags, int ngroups, cudaStream_t st);

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

// mean frame (src/execute_gpu.rs:819-847)
template <typename T>
cudaError_t launch_mean_frame(const T* frames, int64_t T_, int64_t npix, float* out, cudaStream_t st);

// Linking --------------------------------------------------------------
struct LinkInput {
    const float* px;          // row coordinate of every point ("y" column)
    const float* py;          // column coordinate ("x" column)
    const int64_t* goff;      // group offsets, ngroups+1
    const int32_t* pgroup;    // group of every point
    const int32_t* vgrp;      // group range of every video, nvideos+1
    const uint8_t* reset;     // reset flag per group (linker_reset_points)
    int32_t ngroups, nvideos;
    int64_t npoints;
    float radius;
    int32_t memory;
};

struct LinkLists {
    // per point and k in 1..K: forward (dests in group+k) and backward
    // (sources in group-k) neighbour lists, ascending point index
    int64_t* f_off;   // npoints*K + 1
    int64_t* b_off;   // npoints*K + 1
    int32_t* f_pts;
    int32_t* b_pts;
    float* b_dist;    // squared distances of the backward lists
    uint32_t* srt;    // per group: points sorted by row key
};

struct LinkScratch {
    uint8_t* base;
    size_t bytes_per_video;
    int32_t max_group;
    int64_t max_edges;   // max over groups of the per-step backward-edge total
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
cudaError_t link_count_lists(const LinkInput& in, const uint32_t* srt, int64_t* f_cnt, int64_t* b_cnt,
                             cudaStream_t st);
cudaError_t link_fill_lists(const LinkInput& in, const LinkLists& L, cudaStream_t st);
size_t link_scratch_bytes(int32_t max_group, int64_t max_edges, int64_t npoints_video, int32_t memory);
cudaError_t link_run(const LinkInput& in, const LinkLists& L, const LinkScratch& S, const LinkOutput& out,
                     cudaStream_t st);
cudaError_t link_durations(const LinkInput& in, const LinkOutput& out, int64_t* row_dur, cudaStream_t st);

}  // namespace gt
