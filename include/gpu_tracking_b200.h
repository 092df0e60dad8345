/*
 * gpu_tracking_b200 — C ABI of the B200 particle locating + linking engine.
 *
 * This is the drop-in boundary for the hot path of amfaber/gpu_tracking
 * (Crocker–Grier / LoG locate -> characterize -> filter_close -> doughnut ->
 * trackpy-style subnet linking).  Every entry point takes plain pointers and
 * sizes; no CUDA or torch types cross it.  Each declaration names the
 * reference interface it replaces (file:line within the reference project).
 *
 * Conventions
 *   - Frames are C-contiguous (T, H, W) arrays, row index first ("y" in the
 *     output table is the row coordinate, "x" the column coordinate, exactly
 *     as src/execute_gpu.rs:482-519 names them).
 *   - A frame pointer may be host memory or device memory of the context's
 *     device; the library detects which (cudaPointerGetAttributes).
 *   - Status codes mirror the reference's error enum (src/error.rs:5-94) plus
 *     GT_ERR_CAPACITY_EXCEEDED / GT_ERR_CUDA for conditions the reference
 *     either truncates silently or panics on.
 *   - Result tables are library-allocated; free them with gt_table_free.
 *   - One context per host thread.  Calls are synchronous at the ABI.
 */
#ifndef GPU_TRACKING_B200_H
#define GPU_TRACKING_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define GT_API __attribute__((visibility("default")))
#else
#define GT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef enum gt_status {
    GT_OK = 0,
    GT_ERR_INVALID_ARGUMENT = 1,          /* Error::WrongBuilder and bad parameters   (src/error.rs:92)  */
    GT_ERR_DIMENSION_MISMATCH = 2,        /* Error::DimensionMismatch                 (src/error.rs:20)  */
    GT_ERR_EMPTY_ITERATOR = 3,            /* Error::EmptyIterator                     (src/error.rs:27)  */
    GT_ERR_NON_SORTED_CHARACTERIZATION = 4, /* Error::NonSortedCharacterization       (src/error.rs:30)  */
    GT_ERR_FRAME_OUT_OF_BOUNDS = 5,       /* Error::FrameOutOfBounds                  (src/error.rs:33)  */
    GT_ERR_NON_STANDARD_ARRAY_LAYOUT = 6, /* Error::NonStandardArrayLayout            (src/error.rs:49)  */
    GT_ERR_ARRAY_DIMENSIONS = 7,          /* Error::ArrayDimensionsError              (src/error.rs:58)  */
    GT_ERR_TOO_DENSE_TO_LINK = 8,         /* Error::TooDenseToLink                    (src/error.rs:77)  */
    GT_ERR_INTERRUPTED = 9,               /* Error::Interrupted                       (src/error.rs:83)  */
    GT_ERR_CAPACITY_EXCEEDED = 10,        /* reference truncates silently (src/gpu_setup.rs:246-253)      */
    GT_ERR_CUDA = 11,                     /* ~ Error::GpuDeviceError                  (src/error.rs:11)  */
    GT_ERR_NO_DEVICE = 12,                /* ~ Error::GpuAdapterError                 (src/error.rs:8)   */
    GT_ERR_SUBNET_TOO_EXPENSIVE = 13,     /* device subnet search exceeded its step budget (no ref analogue) */
    GT_ERR_INTERNAL = 14,
    GT_ERR_FILE_NOT_FOUND = 15,           /* Error::FileNotFound / InvalidFileName    (src/error.rs)      */
    GT_ERR_READ = 16                      /* Error::ReadError / CastError / UnsupportedFileformat         */
} gt_status;

/* ------------------------------------------------------------- parameters */
typedef enum gt_style { GT_STYLE_TRACKPY = 0, GT_STYLE_LOG = 1 } gt_style;

typedef enum gt_dtype { GT_DTYPE_U16 = 0, GT_DTYPE_F32 = 1, GT_DTYPE_U8 = 2 } gt_dtype;

/*
 * Mirror of the reference's TrackingParams + ParamStyle
 * (src/gpu_setup.rs:10-59).  Option<T> fields carry an explicit has_* flag.
 * Trackpy-only fields that the reference accepts and ignores (maxsize,
 * threshold, invert, percentile, topn, preprocess) are not represented.
 */
typedef struct gt_params {
    int32_t style;                 /* gt_style                                                */
    /* ParamStyle::Trackpy */
    uint32_t diameter;
    uint32_t separation;
    int32_t filter_close;
    /* ParamStyle::Log */
    float min_radius;
    float max_radius;
    uint32_t n_radii;
    int32_t log_spacing;
    float overlap_threshold;
    /* common */
    float minmass;
    uint32_t max_iterations;
    int32_t characterize;
    int32_t has_search_range;  float search_range;
    uint32_t memory;                                   /* memory.unwrap_or(0)                 */
    int32_t doughnut_correction;
    int32_t has_bg_radius;     float bg_radius;
    int32_t has_gap_radius;    float gap_radius;
    int32_t has_snr;           float snr;
    int32_t has_minmass_snr;   float minmass_snr;
    int32_t truncate_preprocessed;
    int32_t has_illumination_sigma; float illumination_sigma;
    int32_t illumination_correction_per_frame;
    int32_t has_adaptive_background; uint32_t adaptive_background;
    int32_t include_r_in_output;
    float shift_threshold;
    float noise_size;
    int32_t has_smoothing_size; uint32_t smoothing_size;
} gt_params;

/* TrackingParams::default() (src/gpu_setup.rs:61-97). */
GT_API void gt_params_default(gt_params* p);

/* ------------------------------------------------------------- context */
typedef struct gt_ctx gt_ctx;

/* new_adapter + new_device_queue (src/gpu_setup.rs:582-609): binds a device. */
GT_API gt_status gt_create(int32_t device, gt_ctx** out);
GT_API void gt_destroy(gt_ctx* ctx);
/* Human-readable message of the last failing call on this context. */
GT_API const char* gt_last_error(const gt_ctx* ctx);
/* Cooperative interrupt (the reference's Arc<AtomicBool>, src/execute_gpu.rs:1094-1099):
 * a non-zero *flag makes the running call return GT_ERR_INTERRUPTED between
 * frame chunks.  Pass NULL to clear. */
GT_API gt_status gt_set_interrupt(gt_ctx* ctx, const volatile int32_t* flag);
/* Progress of the running/last call: (frames done, frames total), the
 * reference's Arc<Mutex<(usize, Option<usize>)>> (src/execute_gpu.rs:972-975). */
GT_API gt_status gt_progress(const gt_ctx* ctx, int64_t* done, int64_t* total);

/* ------------------------------------------------------------ result table */
typedef struct gt_table gt_table;

/* Superset of the reference's output columns (src/execute_gpu.rs:482-519)
 * plus two diagnostics the reference computes but does not emit. */
typedef enum gt_column {
    GT_COL_FRAME = 0, GT_COL_Y, GT_COL_X, GT_COL_MASS, GT_COL_R,
    GT_COL_RG, GT_COL_RAW, GT_COL_SIGNAL, GT_COL_ECC,
    GT_COL_RAW_MASS, GT_COL_RAW_BG_MEDIAN, GT_COL_RAW_MASS_CORRECTED,
    GT_COL_PARTICLE, GT_COL_DURATION,
    GT_COL_MAX_INTENSITY, GT_COL_COUNT,
    GT_NUM_COLUMNS
} gt_column;

GT_API int64_t gt_table_nrows(const gt_table* t);
/* Copy one column to host memory as float32 (all value columns, and the
 * integer columns converted the way the reference stores them). */
GT_API gt_status gt_table_column_f32(const gt_table* t, int32_t column, float* dst);
/* Copy an integer column (frame / particle / duration) as int64. */
GT_API gt_status gt_table_column_i64(const gt_table* t, int32_t column, int64_t* dst);
/* Copy several columns at once in the dtypes of the reference's DataFrame
 * (the `astype` of the column types after `pandas.DataFrame(array)`,
 * gpu_tracking_macros/src/lib.rs:138-147: "int" -> int64, "float" ->
 * float64).  dst[k] receives column columns[k]: int64_t values for
 * GT_COL_FRAME / GT_COL_PARTICLE / GT_COL_DURATION, double for every other
 * column (the float32 value widened exactly).  The rows cross PCIe through
 * pinned staging buffers and are widened on several host threads, so the
 * destinations may be ordinary pageable memory.  Returns
 * GT_ERR_INVALID_ARGUMENT for a column the table does not have. */
GT_API gt_status gt_table_export(const gt_table* t, const int32_t* columns, int32_t ncolumns, void* const* dst);
/* 1 if the column was computed for this table (e.g. GT_COL_PARTICLE only
 * when linking ran). */
GT_API int32_t gt_table_has_column(const gt_table* t, int32_t column);
GT_API void gt_table_free(gt_table* t);

/* ---------------------------------------------------------------- entry points */
/*
 * Locate + characterize + filter_close + doughnut + link over a video.
 * Replaces execute_ndarray / execute_provider / execute_gpu
 * (src/execute_gpu.rs:1378-1403, 1272-1352, 886-1184), i.e. the pyo3
 * functions batch_rust and LoG_rust (gpu_tracking_macros/src/lib.rs:57-156).
 * style selects Crocker–Grier (batch) or LoG.
 * frames may live in host memory or in device memory of the context's
 * device; device frames must be complete when the call is made (the
 * engine's streams do not wait for the caller's).
 * frame_numbers (nullable, length T) gives the frame index written to the
 * "frame" column and used for linker_reset_points; NULL means 0..T-1 (the
 * reference's `frames`/keys selection, src/execute_gpu.rs:1041-1077).
 * linker_reset_points (nullable, length n_reset) mirrors
 * TrackingParams::linker_reset_points (src/execute_gpu.rs:792-798).
 */
GT_API gt_status gt_batch(gt_ctx* ctx, const gt_params* params,
                   const void* frames, int32_t dtype, int64_t T, int32_t H, int32_t W,
                   const int64_t* frame_numbers,
                   const int64_t* linker_reset_points, int64_t n_reset,
                   gt_table** out);

/*
 * gt_batch over many videos of any sizes in one call: out[v] receives video
 * v's table, equal to what gt_batch(frames[v], T[v], H[v], W[v]) returns
 * (frame numbers 0..T[v]-1, no linker resets).  The videos share params and
 * dtype; linking runs for all videos in one launch.  Replaces a loop of
 * execute_ndarray calls (src/execute_gpu.rs:1378-1403), one per video; the
 * reference has no multi-video entry point.
 */
GT_API gt_status gt_batch_videos(gt_ctx* ctx, const gt_params* params, int32_t n_videos,
                          const void* const* frames, int32_t dtype,
                          const int64_t* T, const int32_t* H, const int32_t* W,
                          gt_table** out);

/*
 * Characterize given points instead of detected ones.  Replaces
 * characterize_points_rust (gpu_tracking_macros/src/lib.rs:641-683) and the
 * FrameSubsetter characterization path (src/execute_gpu.rs:189-229,
 * src/linking.rs:97-196).  points is row-major (n_points, ncols) float32 with
 * columns [frame,] y, x [, r] according to has_frames / has_r.
 */
GT_API gt_status gt_characterize_points(gt_ctx* ctx, const gt_params* params,
                                 const void* frames, int32_t dtype, int64_t T, int32_t H, int32_t W,
                                 const float* points, int64_t n_points,
                                 int32_t has_frames, int32_t has_r,
                                 gt_table** out);

/*
 * Link detections.  Replaces link_rust (gpu_tracking_python/src/python_bindings.rs:275-291)
 * -> linker_all (src/linking.rs:818-831).  frame_y_x is row-major (n, 3)
 * float32, sorted by frame.  particle_out receives one id per row.
 */
GT_API gt_status gt_link(gt_ctx* ctx, const float* frame_y_x, int64_t n,
                  float search_range, uint32_t memory, int64_t* particle_out);

/*
 * Connect two detection sets frame by frame.  Replaces connect_rust
 * (gpu_tracking_python/src/python_bindings.rs:293-312) -> connect_all
 * (src/linking.rs:960-1020).
 */
GT_API gt_status gt_connect(gt_ctx* ctx, const float* frame_y_x1, int64_t n1,
                     const float* frame_y_x2, int64_t n2, float search_range,
                     int64_t* out1, int64_t* out2);

/*
 * Mean frame of a video (src/execute_gpu.rs:819-847, mean_from_file_rust
 * gpu_tracking_python/src/python_bindings.rs:361-371), out is (H, W) float32.
 */
GT_API gt_status gt_mean_frame(gt_ctx* ctx, const void* frames, int32_t dtype,
                        int64_t T, int32_t H, int32_t W, float* out);

/*
 * Link detections that are already in device memory without allocating any
 * device memory.  No counterpart in the reference: it exists for callers that
 * cannot allocate while they run — a live acquisition loop linking each batch
 * of detections as frames arrive (cudaMalloc/cudaFree synchronise the device
 * and would stall it), or a process whose device memory belongs to another
 * allocator.  d_frame_y_x is (n, 3) float32 [frame, y, x] rows sorted by frame
 * on the context's device; d_particle_out receives n int64 ids on that device;
 * the ids equal gt_link's.  Working memory is one static device array shared
 * by all calls (limits: n <= 32768, <= 4096 detections per frame, memory <= 3;
 * larger inputs return GT_ERR_CAPACITY_EXCEEDED), so calls whose GPU work
 * overlaps race on it.  The first call on a device looks up the array's
 * address (cudaGetSymbolAddress); make it before any stream capture.
 */
GT_API gt_status gt_link_noalloc(gt_ctx* ctx, const float* d_frame_y_x, int64_t n, float search_range,
                                 uint32_t memory, int64_t* d_particle_out);

/* ------------------------------------------------- learned proposals
 * No counterpart in the reference.  A small BF16 network (4 layers of 3x3
 * convolutions, 32 channels, over 4x4-pixel cells) proposes walk seeds in
 * place of the bandpass local maxima; the walk, characterization,
 * filter_close, doughnut correction and linking are the plain method's.  It
 * is trained on the plain method's own detections.
 */
typedef struct gt_proposal gt_proposal;

typedef struct gt_train_opts {
    int32_t steps;        /* optimizer steps */
    int32_t batch;        /* crops per step */
    int32_t crop;         /* crop side in pixels, a multiple of 4 */
    float lr;             /* Adam step size, cosine-decayed to lr / 20 over the steps */
    float pos_weight;     /* weight of the labelled cells in the score loss */
    float offset_weight;  /* weight of the squared offset error at labelled cells */
    uint32_t seed;        /* crop sampling */
} gt_train_opts;

GT_API void gt_train_opts_default(gt_train_opts* o);
/* Number of fp32 parameters (layer by layer: W[co][ci][ky*3+kx], then b[co]). */
GT_API int64_t gt_proposal_num_params(void);
/* A network with seeded He-normal weights. */
GT_API gt_status gt_proposal_create(gt_ctx* ctx, uint64_t seed, gt_proposal** out);
GT_API void gt_proposal_destroy(gt_proposal* p);
/* Set (params may be NULL to keep them) or read the parameters, the input
 * normalisation (pixel - mean) * scale and the score-logit threshold. */
GT_API gt_status gt_proposal_set(gt_ctx* ctx, gt_proposal* p, const float* params, float mean, float scale,
                                 float threshold);
GT_API gt_status gt_proposal_get(gt_ctx* ctx, const gt_proposal* p, float* params, float* mean, float* scale,
                                 float* threshold);
/* Train on crops of the frames (host or device memory) labelled by the
 * detections (label_frame indexes 0..T-1, label_y / label_x in pixels).
 * loss_out (nullable, 2 * steps floats) receives the score and offset loss
 * of every step. */
GT_API gt_status gt_proposal_train(gt_ctx* ctx, gt_proposal* p, const void* frames, int32_t dtype, int64_t T,
                                   int32_t H, int32_t W, const int64_t* label_frame, const float* label_y,
                                   const float* label_x, int64_t n_labels, const gt_train_opts* opts,
                                   float* loss_out);
/* Network outputs of every cell: maps is (T, ceil(H/4), ceil(W/4), 4) float32
 * holding (score logit, row offset, column offset, 0). */
GT_API gt_status gt_proposal_maps(gt_ctx* ctx, const gt_proposal* p, const void* frames, int32_t dtype, int64_t T,
                                  int32_t H, int32_t W, float* maps);
/* gt_batch with the network's seeds instead of the bandpass local maxima
 * (trackpy style; snr, minmass_snr, adaptive_background and illumination
 * correction are not supported here). */
GT_API gt_status gt_batch_learned(gt_ctx* ctx, const gt_params* params, const gt_proposal* p,
                                  const void* frames, int32_t dtype, int64_t T, int32_t H, int32_t W,
                                  const int64_t* frame_numbers, const int64_t* linker_reset_points,
                                  int64_t n_reset, gt_table** out);
/* Walk starts (bandpass candidates or learned seeds) of the last gt_batch /
 * gt_batch_learned call on this context, summed over its frames. */
GT_API int64_t gt_last_walk_starts(const gt_ctx* ctx);

/* ------------------------------------------------------------ video files
 * Frame providers of path_to_iter (src/execute_gpu.rs:1186-1270,
 * src/decoderiter.rs:64-481): .tif/.tiff stacks (every image in IFD order;
 * classic or BigTIFF, strips or tiles, one sample per pixel, 8/16-bit
 * integers or 32-bit floats, uncompressed / PackBits / LZW / Deflate, with or
 * without horizontal differencing), Olympus .ets (one channel's frames) and
 * .vsi (the .ets at _<stem>_/stack1/frame_t_0.ets beside it), decoded on
 * the host (gt_video_read, no device needed) or on a GPU
 * (gt_video_read_device).  u8 and u16 files keep their dtype; other
 * sample types decode to f32.
 */
typedef struct gt_video gt_video;
GT_API gt_status gt_video_open(const char* path, int32_t channel, gt_video** out);
GT_API gt_status gt_video_info(const gt_video* v, int64_t* T, int32_t* H, int32_t* W, int32_t* dtype);
/* Decode frames (frame indices, or the first n when frames is NULL) into dst,
 * (n, H, W) of `dtype` (the video's own dtype or GT_DTYPE_F32). */
GT_API gt_status gt_video_read(gt_video* v, const int64_t* frames, int64_t n, int32_t dtype, void* dst);
/* The same frames decoded on the context's GPU into device memory `dst`
 * (n x H x W of `dtype`): the file's strips, tiles or ETS frames are read on
 * the host, copied to the device and decompressed there (LZW, PackBits;
 * Deflate is inflated on the host), with the predictor and the sample
 * conversion on the device.  Same values as gt_video_read.  Replaces the
 * decode half of the frame providers (src/decoderiter.rs:64-481). */
GT_API gt_status gt_video_read_device(gt_ctx* ctx, gt_video* v, const int64_t* frames, int64_t n, int32_t dtype,
                                      void* dst);
GT_API void gt_video_close(gt_video* v);
/* Message of the last failing gt_video_* call of this thread. */
GT_API const char* gt_video_last_error(void);

/* Library version string. */
GT_API const char* gt_version(void);

/* ------------------------------------------------------------ diagnostics */
/* Per-kernel timing with CUDA events on the engine's compute stream (no
 * counterpart in the reference): enable, run calls, then read the launch
 * count and summed milliseconds of a kernel class ("bandpass_localmax",
 * "walk_characterize", "finalize", "bandpass", "log_scale_space", "laplace", "logspace_max",
 * "link_sort", "link_lists", "link_video"). */
GT_API gt_status gt_profile_enable(gt_ctx* ctx, int32_t enable);
GT_API gt_status gt_profile_read(gt_ctx* ctx, const char* name, int64_t* launches, double* total_ms);
/* Number of engine kernel launches since the last gt_profile_enable. */
GT_API int64_t gt_launch_count(gt_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* GPU_TRACKING_B200_H */
