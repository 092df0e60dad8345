// ref_driver.cpp — runs the reference's own WGSL shaders on the CPU.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle).  The shader bodies are
// included from oracle/_ref/gen_*.inc, which oracle/wgsl2cpp.py generates
// from the reference checkout at build time; this file only provides the
// WGSL builtins and dispatches the shaders in the reference's pass order
// (src/gpu_setup.rs:872-895, src/execute_gpu.rs:231-286 and 368-375,
// src/utils.rs:114-296 for Laplace<2>), one invocation at a time in
// row-major order (the canonical order for the reference's atomics).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct vec2f {
    float v[2];
    vec2f() : v{0.0f, 0.0f} {}
    vec2f(float a, float b) : v{a, b} {}
    float& operator[](int i) { return v[i]; }
    float operator[](int i) const { return v[i]; }
};
struct ivec2 {
    int32_t v[2];
    ivec2() : v{0, 0} {}
    ivec2(int32_t a, int32_t b) : v{a, b} {}
    int32_t& operator[](int i) { return v[i]; }
    int32_t operator[](int i) const { return v[i]; }
};
struct uvec3 {
    uint32_t x, y, z;
    uint32_t operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

// WGSL storage array with robust buffer access.
template <class T>
struct RobustArray {
    T* p = nullptr;
    int64_t n = 0;
    T dummy{};
    RobustArray() = default;
    RobustArray& operator=(T* q) {
        p = q;
        return *this;
    }
    T& operator[](int64_t i) {
        if (i < 0 || i >= n) {
            dummy = T{};
            return dummy;
        }
        return p[i];
    }
};

template <class T>
void bind(RobustArray<T>& a, T* p, int64_t n) {
    a.p = p;
    a.n = n;
}

inline float wgsl_f32(float x) { return x; }
inline float wgsl_f32(int32_t x) { return (float)x; }
inline float wgsl_f32(uint32_t x) { return (float)x; }
inline int32_t wgsl_i32(int32_t x) { return x; }
inline int32_t wgsl_i32(uint32_t x) { return (int32_t)x; }
inline int32_t wgsl_i32(float x) {
    if (std::isnan(x)) return 0;
    if (x >= 2147483647.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}
inline uint32_t wgsl_u32(uint32_t x) { return x; }
inline uint32_t wgsl_u32(int32_t x) { return (uint32_t)x; }
inline uint32_t wgsl_u32(float x) { return x <= 0.0f ? 0u : (uint32_t)x; }
inline float wgsl_exp(float x) { return std::exp(x); }
inline float wgsl_sqrt(float x) { return std::sqrt(x); }
inline float wgsl_atan2(float y, float x) { return std::atan2(y, x); }
inline float wgsl_sin(float x) { return std::sin(x); }
inline float wgsl_cos(float x) { return std::cos(x); }
inline float wgsl_ceil(float x) { return std::ceil(x); }
inline float wgsl_round(float x) { return std::rint(x); }  // WGSL: round half to even
inline float wgsl_max(float a, float b) { return (a < b) ? b : a; }
inline int32_t wgsl_max(int32_t a, int32_t b) { return (a < b) ? b : a; }
inline float wgsl_fma(float a, float b, float c) { return std::fmaf(a, b, c); }
inline uint32_t wgsl_atomicAdd(uint32_t* p, uint32_t v) {
    uint32_t o = *p;
    *p += v;
    return o;
}
inline uint32_t wgsl_atomicSub(uint32_t* p, uint32_t v) {
    uint32_t o = *p;
    *p -= v;
    return o;
}
inline uint32_t wgsl_bitcast_u32(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    return u;
}
inline float wgsl_bitcast_f32(uint32_t u) {
    float x;
    std::memcpy(&x, &u, 4);
    return x;
}

#include "_ref/gen_preprocess_rows.inc"
#include "_ref/gen_preprocess_cols_trunc.inc"
#include "_ref/gen_preprocess_cols_notrunc.inc"
#include "_ref/gen_max_rows.inc"
#include "_ref/gen_extract_max.inc"
#include "_ref/gen_walk.inc"
#include "_ref/gen_characterize.inc"
#include "_ref/gen_characterize_points.inc"
#include "_ref/gen_separable_log.inc"
#include "_ref/gen_logspace_max.inc"
#include "_ref/gen_sum_image_outplace.inc"
#include "_ref/gen_sum_image_inplace.inc"
#include "_ref/gen_last_reduction.inc"
#include "_ref/gen_std_image.inc"
#include "_ref/gen_adaptive_filter.inc"
#include "_ref/gen_smooth_mean_frame.inc"
#include "_ref/gen_correct_illumination.inc"

// Flat copy of the WGSL Params uniform (params.wgsl:1-20).
struct RefParams {
    int32_t pic_nrows, pic_ncols, preprocess_nrows, preprocess_ncols;
    float sigma2;
    int32_t circle_nrows, circle_ncols, dilation_nrows, dilation_ncols;
    uint32_t max_iterations;
    float threshold, minmass;
    int32_t margin;
    float snr, minmass_snr, rough_snr_factor;
};

template <class P>
void set_params(P& dst, const RefParams* src) {
    static_assert(sizeof(P) == sizeof(RefParams), "Params layout");
    std::memcpy(&dst, src, sizeof(RefParams));
}

template <class F>
void dispatch2d(int32_t H, int32_t W, F&& f) {
    for (int32_t x = 0; x < H; x++)
        for (int32_t y = 0; y < W; y++) f(uvec3{(uint32_t)x, (uint32_t)y, 0u});
}

}  // namespace

extern "C" {

int ref_preprocess(const RefParams* p, int32_t truncate, const float* frame, float* processed) {
    const int32_t H = p->pic_nrows, W = p->pic_ncols;
    std::vector<vec2f> temp((size_t)H * W);
    set_params(sh_preprocess_rows::params, p);
    bind(sh_preprocess_rows::picture, const_cast<float*>(frame), (int64_t)H * W);
    bind(sh_preprocess_rows::temp, temp.data(), (int64_t)H * W);
    dispatch2d(H, W, [](uvec3 g) { sh_preprocess_rows::main_(g); });
    if (truncate) {
        set_params(sh_preprocess_cols_trunc::params, p);
        bind(sh_preprocess_cols_trunc::temp, temp.data(), (int64_t)H * W);
        bind(sh_preprocess_cols_trunc::processed_buffer, processed, (int64_t)H * W);
        dispatch2d(H, W, [](uvec3 g) { sh_preprocess_cols_trunc::main_(g); });
    } else {
        set_params(sh_preprocess_cols_notrunc::params, p);
        bind(sh_preprocess_cols_notrunc::temp, temp.data(), (int64_t)H * W);
        bind(sh_preprocess_cols_notrunc::processed_buffer, processed, (int64_t)H * W);
        dispatch2d(H, W, [](uvec3 g) { sh_preprocess_cols_notrunc::main_(g); });
    }
    return 0;
}

int64_t ref_candidates(const RefParams* p, const float* processed, float pic_std, int32_t* uv, int64_t cap) {
    const int32_t H = p->pic_nrows, W = p->pic_ncols;
    std::vector<float> mr((size_t)H * W);
    set_params(sh_max_rows::params, p);
    bind(sh_max_rows::processed_buffer, const_cast<float*>(processed), (int64_t)H * W);
    bind(sh_max_rows::max_rows, mr.data(), (int64_t)H * W);
    dispatch2d(H, W, [](uvec3 g) { sh_max_rows::main_(g); });
    // every pixel may be a candidate; the reference's own buffer holds H*W/4
    // entries and drops the rest, which the callers treat as an error case
    std::vector<sh_extract_max::ParticleLocation> pts((size_t)H * W + 1);
    set_params(sh_extract_max::params, p);
    bind(sh_extract_max::processed_buffer, const_cast<float*>(processed), (int64_t)H * W);
    bind(sh_extract_max::max_rows, mr.data(), (int64_t)H * W);
    sh_extract_max::n_particles = 0;
    bind(sh_extract_max::max_points, pts.data(), (int64_t)pts.size());
    sh_extract_max::pic_std = pic_std;
    sh_extract_max::wg_size = {};
    dispatch2d(H, W, [](uvec3 g) { sh_extract_max::main_(g); });
    int64_t n = sh_extract_max::n_particles;
    for (int64_t i = 0; i < n && i < cap; i++) {
        uv[2 * i] = pts[i].x;
        uv[2 * i + 1] = pts[i].y;
    }
    return n;
}

// walk over candidates (with radius r, -1 for trackpy), then characterize the
// kept rows when characterize != 0.  rows_out: 10 floats per kept row.
int64_t ref_walk(const RefParams* p, const float* processed, const float* raw, const int32_t* uv, int64_t n,
                 float r, float pic_std, int32_t characterize, float* rows_out) {
    std::vector<sh_walk::ParticleLocation> parts((size_t)n + 1);
    for (int64_t i = 0; i < n; i++) parts[i] = {uv[2 * i], uv[2 * i + 1], r, -1.0f};
    std::vector<sh_walk::ResultRow> res((size_t)n + 1);
    set_params(sh_walk::params, p);
    bind(sh_walk::processed_buffer, const_cast<float*>(processed), (int64_t)p->pic_nrows * p->pic_ncols);
    bind(sh_walk::particles, parts.data(), (int64_t)parts.size());
    sh_walk::n_particles = (uint32_t)n;
    sh_walk::n_particles_filtered = 0;
    bind(sh_walk::results, res.data(), (int64_t)res.size());
    bind(sh_walk::raw_frame, const_cast<float*>(raw), (int64_t)p->pic_nrows * p->pic_ncols);
    sh_walk::image_std = pic_std;
    sh_walk::next_dispatch = {};
    for (int64_t i = 0; i < n; i++) sh_walk::main_(uvec3{(uint32_t)i, 0u, 0u});
    int64_t nk = sh_walk::n_particles_filtered;
    if (characterize) {
        static_assert(sizeof(sh_walk::ResultRow) == sizeof(sh_characterize::ResultRow), "row");
        std::vector<sh_characterize::ResultRow> cr((size_t)nk + 1);
        std::memcpy(cr.data(), res.data(), (size_t)nk * sizeof(sh_walk::ResultRow));
        set_params(sh_characterize::params, p);
        bind(sh_characterize::processed_buffer, const_cast<float*>(processed), (int64_t)p->pic_nrows * p->pic_ncols);
        bind(sh_characterize::raw_frame, const_cast<float*>(raw), (int64_t)p->pic_nrows * p->pic_ncols);
        sh_characterize::n_particles = (uint32_t)nk;
        bind(sh_characterize::results, cr.data(), (int64_t)cr.size());
        for (int64_t i = 0; i < nk; i++) sh_characterize::main_(uvec3{(uint32_t)i, 0u, 0u});
        std::memcpy(res.data(), cr.data(), (size_t)nk * sizeof(sh_walk::ResultRow));
    }
    std::memcpy(rows_out, res.data(), (size_t)nk * 10 * sizeof(float));
    return nk;
}

// characterize_points: rows_inout holds 10-float ResultRows with x, y, r set.
int ref_characterize_points(const RefParams* p, const float* processed, const float* raw, float* rows_inout,
                            int64_t n) {
    std::vector<sh_characterize_points::ResultRow> cr((size_t)n + 1);
    std::memcpy(cr.data(), rows_inout, (size_t)n * 10 * sizeof(float));
    set_params(sh_characterize_points::params, p);
    bind(sh_characterize_points::processed_buffer, const_cast<float*>(processed), (int64_t)p->pic_nrows * p->pic_ncols);
    bind(sh_characterize_points::raw_frame, const_cast<float*>(raw), (int64_t)p->pic_nrows * p->pic_ncols);
    sh_characterize_points::n_particles = (uint32_t)n;
    bind(sh_characterize_points::results, cr.data(), (int64_t)cr.size());
    for (int64_t i = 0; i < n; i++) sh_characterize_points::main_(uvec3{(uint32_t)i, 0u, 0u});
    std::memcpy(rows_inout, cr.data(), (size_t)n * 10 * sizeof(float));
    return 0;
}

// Laplace<2>::execute with SeparableConvolution<2> buffers: input = frame,
// temp2 = first output, final = log-space plane (src/utils.rs:114-296).
int ref_laplace(const RefParams* p, const float* frame, float sigma, float* final_out) {
    const int32_t H = p->pic_nrows, W = p->pic_ncols;
    std::vector<float> temp2((size_t)H * W), temp1((size_t)H * W);
    set_params(sh_separable_log::params, p);
    bind(sh_separable_log::final_output, final_out, (int64_t)H * W);
    for (uint32_t diff_dim = 0; diff_dim < 2; diff_dim++) {
        sh_separable_log::pc = {0u, diff_dim, sigma};
        bind(sh_separable_log::input, const_cast<float*>(frame), (int64_t)H * W);
        bind(sh_separable_log::output, temp2.data(), (int64_t)H * W);
        dispatch2d(H, W, [](uvec3 g) { sh_separable_log::main_(g); });
        sh_separable_log::pc = {1u, diff_dim, sigma};
        bind(sh_separable_log::input, temp2.data(), (int64_t)H * W);
        bind(sh_separable_log::output, temp1.data(), (int64_t)H * W);
        dispatch2d(H, W, [](uvec3 g) { sh_separable_log::main_(g); });
    }
    return 0;
}

int64_t ref_logspace_max(const RefParams* p, const float* bottom, const float* middle, const float* top,
                         const float* processed, float pic_std, int32_t edge, float radius, int32_t* uv,
                         int64_t cap) {
    const int32_t H = p->pic_nrows, W = p->pic_ncols;
    std::vector<sh_logspace_max::ParticleLocation> pts((size_t)H * W + 1);
    set_params(sh_logspace_max::params, p);
    bind(sh_logspace_max::bottom, const_cast<float*>(bottom), (int64_t)H * W);
    bind(sh_logspace_max::middle, const_cast<float*>(middle), (int64_t)H * W);
    bind(sh_logspace_max::top, const_cast<float*>(top), (int64_t)H * W);
    sh_logspace_max::n_particles = 0;
    bind(sh_logspace_max::particles, pts.data(), (int64_t)pts.size());
    sh_logspace_max::wg_size = {};
    sh_logspace_max::std_pic = pic_std;
    bind(sh_logspace_max::processed, const_cast<float*>(processed), (int64_t)H * W);
    sh_logspace_max::pc = {edge, radius};
    dispatch2d(H, W, [](uvec3 g) { sh_logspace_max::main_(g); });
    int64_t n = sh_logspace_max::n_particles;
    for (int64_t i = 0; i < n && i < cap; i++) {
        uv[2 * i] = pts[i].x;
        uv[2 * i + 1] = pts[i].y;
    }
    return n;
}


// StdArray::execute (src/utils.rs:614-640): MeanArrayOutplace over the frame,
// std_image, MeanArray with the square root.  `temp` is the reference's shared
// temp buffer (2N floats); it keeps its contents between calls like the
// reference's does.  Returns the value left in std_buffer.
float ref_frame_std(const float* frame, int64_t N, uint32_t divisor, float* temp) {
    auto meanarray = [&](uint32_t size, uint32_t sqrt_mean) -> float {
        // MeanArray::execute (src/utils.rs:417-440)
        uint32_t to_start = size;
        while (to_start > 24) {
            to_start += 7;
            to_start /= 8;
            sh_sum_image_inplace::pc.stride = to_start;
            bind(sh_sum_image_inplace::arr, temp, 2 * N);
            for (uint32_t x = 0; x < to_start; x++) sh_sum_image_inplace::main_(uvec3{x, 0u, 0u});
        }
        sh_last_reduction::pc.n_elements = to_start;
        sh_last_reduction::pc.doing_variance = sqrt_mean;
        bind(sh_last_reduction::input, temp, 2 * N);
        sh_last_reduction::mean_divisor = divisor;
        sh_last_reduction::main_(uvec3{0u, 0u, 0u});
        return sh_last_reduction::output;
    };
    // MeanArrayOutplace::execute (src/utils.rs:514-531)
    const uint32_t s = (uint32_t)((N + 7) / 8);
    sh_sum_image_outplace::pc.stride = s;
    bind(sh_sum_image_outplace::input, const_cast<float*>(frame), N);
    bind(sh_sum_image_outplace::output, temp, 2 * N);
    for (uint32_t x = 0; x < s; x++) sh_sum_image_outplace::main_(uvec3{x, 0u, 0u});
    const float mean = meanarray(s, 0u);
    // std_pass over the frame, then MeanArray(size N, sqrt)
    sh_std_image::pc.total_elements = (uint32_t)N;
    bind(sh_std_image::input, const_cast<float*>(frame), N);
    bind(sh_std_image::output, temp, 2 * N);
    sh_std_image::mean = mean;
    for (uint32_t x = 0; x < (uint32_t)N; x++) sh_std_image::main_(uvec3{x, 0u, 0u});
    return meanarray((uint32_t)N, 1u);
}

// The adaptive_background loop of submit_work (src/execute_gpu.rs:289-366):
// n_iter passes of adaptive_filter.wgsl ping-ponging between the two particle
// buffers, the frame std recomputed (on the masked frame, divided by the
// decremented counter) before every pass but the first.  rows_in: walked
// ResultRows (10 floats); rows_out receives the accepted rows in the order
// the serial dispatch accepts them.  `frame` is masked in place.
int64_t ref_adaptive(const RefParams* p, float* frame, const float* rows_in, int64_t n_in, uint32_t n_iter,
                     float std0, int32_t recompute_std, float* temp, float* rows_out) {
    const int64_t N = (int64_t)p->pic_nrows * p->pic_ncols;
    using Row = sh_adaptive_filter::ResultRow;
    std::vector<Row> a((size_t)n_in + 1), b((size_t)n_in + 1), res((size_t)n_in + 1);
    std::memcpy(a.data(), rows_in, (size_t)n_in * sizeof(Row));
    uint32_t count_a = (uint32_t)n_in, count_b = 0;
    uint32_t result_n = 0;
    uint32_t counter = (uint32_t)N;
    float std_buffer = std0;
    set_params(sh_adaptive_filter::params, p);
    bind(sh_adaptive_filter::frame, frame, N);
    for (uint32_t it = 0; it < n_iter; it++) {
        const bool even = (it % 2) == 0;
        if (it > 0 && recompute_std) std_buffer = ref_frame_std(frame, N, counter, temp);
        uint32_t& cur = even ? count_a : count_b;
        uint32_t& nxt = even ? count_b : count_a;
        nxt = 0;
        bind(sh_adaptive_filter::input, even ? a.data() : b.data(), n_in + 1);
        bind(sh_adaptive_filter::output, even ? b.data() : a.data(), n_in + 1);
        bind(sh_adaptive_filter::results, res.data(), n_in + 1);
        sh_adaptive_filter::image_std = std_buffer;
        sh_adaptive_filter::current_n = cur;
        sh_adaptive_filter::new_n = 0;
        sh_adaptive_filter::result_n = result_n;
        sh_adaptive_filter::counter = counter;
        sh_adaptive_filter::dispatcher = {};
        sh_adaptive_filter::dispatcher_results = {};
        for (uint32_t x = 0; x < cur; x++) sh_adaptive_filter::main_(uvec3{x, 0u, 0u});
        nxt = sh_adaptive_filter::new_n;
        result_n = sh_adaptive_filter::result_n;
        counter = sh_adaptive_filter::counter;
    }
    std::memcpy(rows_out, res.data(), (size_t)result_n * sizeof(Row));
    return result_n;
}

// SeparableConvolution<2>::execute with smooth_mean_frame.wgsl on the
// illumination buffer (input = output = the buffer, temp = the shared temp
// buffer; push constants dim, sigma, n_frames = 1), then correct_illumination
// over `frame` (frame /= profile).  profile_out receives the smoothed buffer.
int ref_illumination(const RefParams* p, const float* profile_in, float sigma, float* frame_inout,
                     float* profile_out) {
    const int32_t H = p->pic_nrows, W = p->pic_ncols;
    const int64_t N = (int64_t)H * W;
    std::vector<float> buf(profile_in, profile_in + N), temp((size_t)(2 * N));
    set_params(sh_smooth_mean_frame::params, p);
    sh_smooth_mean_frame::pc = {0u, sigma, 1.0f};
    bind(sh_smooth_mean_frame::input, buf.data(), N);
    bind(sh_smooth_mean_frame::output, temp.data(), 2 * N);
    dispatch2d(H, W, [](uvec3 g) { sh_smooth_mean_frame::main_(g); });
    sh_smooth_mean_frame::pc = {1u, sigma, 1.0f};
    bind(sh_smooth_mean_frame::input, temp.data(), 2 * N);
    bind(sh_smooth_mean_frame::output, buf.data(), N);
    dispatch2d(H, W, [](uvec3 g) { sh_smooth_mean_frame::main_(g); });
    std::memcpy(profile_out, buf.data(), (size_t)N * 4);
    sh_correct_illumination::pc.arraylen = (uint32_t)N;
    bind(sh_correct_illumination::frame, buf.data(), N);
    bind(sh_correct_illumination::acc, frame_inout, N);
    for (uint32_t x = 0; x < (uint32_t)N; x++) sh_correct_illumination::main_(uvec3{x, 0u, 0u});
    return 0;
}

}  // extern "C"