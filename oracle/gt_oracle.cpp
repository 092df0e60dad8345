// gt_oracle.cpp — CPU oracle for the gpu_tracking locate + link hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: it restates, on the
// CPU, the algorithm of the reference's WGSL shaders (src/shaders/*.wgsl)
// and of its Rust post-processing and linker (src/execute_gpu.rs,
// src/linking.rs, src/kernels.rs, src/gpu_setup.rs).  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.  The
// product (gpu_tracking_b200/) never links or calls it.
//
// Pinning.  The shader stages restated here (preprocess, extract_max, walk,
// characterize, separable LoG, logspace_max) are pinned bit-for-bit against
// the reference's own WGSL source executed on the CPU: oracle/wgsl2cpp.py
// translates the reference checkout's src/shaders/*.wgsl into C++ at build time
// (output only under oracle/_ref/, never committed) and tests compare both.
// The Rust post-processing (filter_close_trackpy, prune_blobs_log, the
// doughnut block of post_process, the column layout and durations) and the
// linker (Linker, link, linker_all, connect_all) are pinned the same way:
// oracle/rust2py.py translates the reference's own Rust source into Python at
// build time (oracle/_ref/rust_ref.py, run by oracle/ref_post.py with Rust's
// binary32 and integer semantics), and tests/test_golden_post.py compares this
// file with it on randomized inputs and against the committed fixture
// tests/golden/postprocess_ref.npz.  The one piece not taken from the
// reference is the neighbour order of the kd-tree crate (kd-tree 0.5.1,
// not vendored): neighbour lists are in index order here and in the
// translation's shim; the order decides only exact score ties in the
// subnet search.  tests/test_oracle_linking.py keeps its hand-derived
// known-answer cases.
//
// Floating-point conventions (shared with the CUDA kernels, which are
// bit-exact against this file):
//   * WGSL statements of the form `acc += a * b;` are evaluated as one fused
//     multiply-add fmaf(a, b, acc) (what a contracting shader compiler emits);
//     every other operation is a separately rounded IEEE binary32 operation.
//   * Division and sqrt are IEEE round-to-nearest.
//   * exp/atan2/sin/cos/log/pow use the host libm in binary32 (expf, ...).
//   * WGSL round() is round-half-to-even (rintf); Rust f32::round is
//     round-half-away-from-zero (roundf).
//   * Rust code is never contracted (separate mul and add).
//   * Result order is canonical: candidates in row-major pixel order (the
//     reference's atomicAdd order is nondeterministic), LoG results in radius
//     order then row-major.  kd-tree neighbour lists are taken in index order.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off -shared -pthread).

#include "../include/gpu_tracking_b200.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <functional>
#include <limits>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include <atomic>
#include <thread>

namespace oracle {

// ----------------------------------------------------------------- params
// GpuParams derived from TrackingParams: gpuparams_from_tracking_params
// (src/gpu_setup.rs:528-580).
struct Derived {
    int32_t H = 0, W = 0;
    int32_t smoothing = 0;   // composite_dims (preprocess_nrows/ncols)
    float sigma2 = 1.0f;     // GpuParams.sigma = noise_size; WGSL names it sigma2 (params.wgsl:6)
    int32_t circle = 0;      // circle_dims
    int32_t dilation = 0;    // dilation_dims
    uint32_t max_iterations = 10;
    float threshold = 0.6f;  // shift_threshold
    float minmass = 0.0f;
    int32_t margin = 0;
    float snr = 0.0f;
    float minmass_snr = 0.0f;
    float rough = 1.0f;
};

static Derived derive(const gt_params& p, int32_t H, int32_t W) {
    Derived d;
    d.H = H;
    d.W = W;
    if (p.style == GT_STYLE_TRACKPY) {
        uint32_t smoothing = p.has_smoothing_size ? p.smoothing_size : p.diameter;
        uint32_t circle = p.diameter;
        // (2. * separation as f32 / (2 as f32).sqrt()) as u32
        float dil = 2.0f * (float)p.separation / std::sqrt(2.0f);
        uint32_t dilation = (uint32_t)dil;
        // vec![diameter / 2, separation / 2 - 1, smoothing_size / 2].max() as i32 (u32 arithmetic)
        uint32_t a = p.diameter / 2, b = p.separation / 2 - 1u, c = smoothing / 2;
        uint32_t m = std::max(a, std::max(b, c));
        d.smoothing = (int32_t)smoothing;
        d.circle = (int32_t)circle;
        d.dilation = (int32_t)dilation;
        d.margin = (int32_t)m;
    } else {
        uint32_t smoothing;
        if (p.has_smoothing_size) {
            smoothing = p.smoothing_size;
        } else {
            uint32_t radius = (uint32_t)(p.max_radius + 0.5f);
            smoothing = radius * 2 + 1;
        }
        d.smoothing = (int32_t)smoothing;
        d.circle = 0;
        d.dilation = 0;
        d.margin = 0;
    }
    d.sigma2 = p.noise_size;
    d.max_iterations = p.max_iterations;
    d.threshold = p.shift_threshold;
    d.minmass = p.minmass;
    d.snr = p.has_snr ? p.snr : 0.0f;
    d.minmass_snr = p.has_minmass_snr ? p.minmass_snr : 0.0f;
    d.rough = p.has_adaptive_background ? 0.5f : 1.0f;
    return d;
}

// LoG radii (src/gpu_setup.rs:958-984).  Rust f32::log(base) = ln(x)/ln(base).
static std::vector<float> log_radii(const gt_params& p) {
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

static inline float wgsl_max(float a, float b) { return (a < b) ? b : a; }

// ----------------------------------------------------------------- rows
// ResultRow (src/execute_gpu.rs:48-61) plus post-processing outputs.
struct Row {
    float x = 0, y = 0, mass = 0, r = 0, max_intensity = 0;
    float Rg = 0, raw_mass = 0, signal = 0, ecc = 0, count = 0;
    // doughnut (src/execute_gpu.rs:717-790)
    float d_raw_mass = NAN, d_bg_median = NAN, d_corrected = NAN;
    int64_t particle = -1, duration = -1;
    int64_t key = 0;  // position in the canonical (candidate) order of its frame
};

// ------------------------------------------------------------ preprocess
// preprocess_rows.wgsl:14-55 followed by preprocess_cols.wgsl:11-60.
static void preprocess(const Derived& d, bool truncate, const float* img, std::vector<float>& tg,
                       std::vector<float>& tb, float* out) {
    const int32_t H = d.H, W = d.W;
    const int32_t k = d.smoothing;
    const int32_t R = k / 2;
    std::vector<float> taps(2 * R + 1);
    float gnorm = 0.0f;
    for (int32_t i = -R; i <= R; i++) {
        float x = (float)i;
        float g = std::exp(-x * x / (2.0f * d.sigma2));
        taps[i + R] = g;
        gnorm += g;
    }
    tg.resize((size_t)H * W);
    tb.resize((size_t)H * W);
    for (int32_t u = 0; u < H; u++) {
        for (int32_t v = 0; v < W; v++) {
            float gs = 0.0f, cs = 0.0f;
            for (int32_t i = -R; i <= R; i++) {
                int32_t pv = v + i;
                bool do_g = true;
                if (pv < 0) { pv = 0; do_g = false; }
                else if (pv >= W) { pv = W - 1; do_g = false; }
                float px = img[(size_t)u * W + pv];
                if (do_g) gs = std::fmaf(taps[i + R], px, gs);
                cs = cs + px;
            }
            tg[(size_t)u * W + v] = gs / gnorm;
            tb[(size_t)u * W + v] = cs;
        }
    }
    const float kk = (float)(k * k);
    const float trunc_thr = 1.0f / 255.0f;
    for (int32_t u = 0; u < H; u++) {
        for (int32_t v = 0; v < W; v++) {
            float gs = 0.0f, cs = 0.0f;
            for (int32_t i = -R; i <= R; i++) {
                int32_t pu = u + i;
                bool do_g = true;
                if (pu < 0) { pu = 0; do_g = false; }
                else if (pu >= H) { pu = H - 1; do_g = false; }
                size_t idx = (size_t)pu * W + v;
                if (do_g) gs = std::fmaf(taps[i + R], tg[idx], gs);
                cs = cs + tb[idx];
            }
            float result = gs / gnorm - cs / kk;
            if (truncate && result < trunc_thr) result = 0.0f;
            out[(size_t)u * W + v] = result;
        }
    }
}

// ---------------------------------------------------- max_rows + extract_max
// max_rows.wgsl:10-32 and extract_max.wgsl:35-78.  Candidates in row-major order.
static void extract_max(const Derived& d, const float* p, float pic_std, std::vector<float>& mr,
                        std::vector<std::pair<int32_t, int32_t>>& cands) {
    const int32_t H = d.H, W = d.W;
    const int32_t kd = d.dilation;
    const int32_t o = (int32_t)((float)kd / 2.0f - 0.5f);
    mr.resize((size_t)H * W);
    for (int32_t u = 0; u < H; u++) {
        for (int32_t v = 0; v < W; v++) {
            float center = p[(size_t)u * W + v];
            float m = center;
            int32_t pv = v - o;
            for (int32_t j = 0; j < kd; j++) {
                if (pv >= 0 && pv < W) m = wgsl_max(m, p[(size_t)u * W + pv]);
                pv += 1;
            }
            mr[(size_t)u * W + v] = m;
        }
    }
    const float thr = pic_std * d.snr * d.rough;
    cands.clear();
    for (int32_t u = 0; u < H; u++) {
        for (int32_t v = 0; v < W; v++) {
            if (u < d.margin || u >= H - d.margin || v < d.margin || v >= W - d.margin) continue;
            float center = p[(size_t)u * W + v];
            if (center < thr) continue;
            bool ok = true;
            int32_t pu = u - o;
            for (int32_t i = 0; i < kd; i++) {
                if (pu >= 0 && pu < H) {
                    if (mr[(size_t)pu * W + v] > center) { ok = false; break; }
                }
                pu += 1;
            }
            if (ok) cands.push_back({u, v});
        }
    }
}

// ------------------------------------------------------------------- walk
// walk.wgsl:67-229.
struct WalkResult { float x = 0, y = 0, mass = 0, max = 0, count = 0; };

static WalkResult get_center(const Derived& d, const float* p, int32_t u, int32_t v, int32_t rint, float r2) {
    WalkResult res;
    for (int32_t i = -rint; i <= rint; i++) {
        float x = (float)i;
        float x2 = x * x;
        for (int32_t j = -rint; j <= rint; j++) {
            float y = (float)j;
            float y2 = y * y;
            float mask = x2 + y2;
            if (mask > r2) continue;
            int32_t pu = u + i, pv = v + j;
            if (pu < 0 || pu >= d.H || pv < 0 || pv >= d.W) continue;
            float data = p[(size_t)pu * d.W + pv];
            res.x = std::fmaf(data, x, res.x);
            res.y = std::fmaf(data, y, res.y);
            res.mass = res.mass + data;
            res.count = res.count + 1.0f;
            res.max = wgsl_max(res.max, data);
        }
    }
    res.x /= res.mass;
    res.y /= res.mass;
    return res;
}

static WalkResult walk(const Derived& d, const float* p, int32_t u0, int32_t v0, float r) {
    int32_t pu = u0, pv = v0;
    WalkResult res;
    int32_t rint;
    float r2;
    if (r <= 0.0f) {
        rint = (d.circle - 1) / 2;
        float rr = (float)rint;
        r2 = rr * rr;
    } else {
        rint = (int32_t)std::ceil(r);
        r2 = r * r;
    }
    const int32_t margin = rint;
    for (uint32_t it = 0; it < d.max_iterations; it++) {
        res = get_center(d, p, pu, pv, rint, r2);
        bool changed = false;
        if ((res.x > d.threshold) && (pu < d.H - 1 - margin)) { pu += 1; changed = true; }
        else if (res.x < -d.threshold && pu > margin) { pu -= 1; changed = true; }
        if ((res.y > d.threshold) && (pv < d.W - 1 - margin)) { pv += 1; changed = true; }
        else if ((res.y < -d.threshold) && (pv > margin)) { pv -= 1; changed = true; }
        if (!changed) break;
    }
    res.x += (float)pu;
    res.y += (float)pv;
    return res;
}

// walk.wgsl:171-229 (main): minmass filter and ResultRow construction.
static bool walk_keep(const Derived& d, const float* p, int32_t u, int32_t v, float r, float image_std, Row& row) {
    WalkResult res = walk(d, p, u, v, r);
    float minmass;
    if (d.minmass > 0.0f) minmass = d.minmass;
    else minmass = d.minmass_snr * res.count * image_std * d.rough;
    if (res.mass >= minmass) {
        row = Row();
        row.x = res.x;
        row.y = res.y;
        row.mass = res.mass;
        row.count = res.count;
        row.max_intensity = res.max;
        if (r > 0.0f) row.r = r;
        return true;
    }
    return false;
}

// ----------------------------------------------------------- characterize
// characterize.wgsl:30-155.
static float get_mass(const Derived& d, const float* p, int32_t u, int32_t v, int32_t rint, float r2) {
    float mass = 0.0f;
    for (int32_t i = -rint; i <= rint; i++) {
        float x = (float)i;
        float x2 = x * x;
        for (int32_t j = -rint; j <= rint; j++) {
            float y = (float)j;
            float y2 = y * y;
            float mask = x2 + y2;
            if (mask > r2) continue;
            int32_t pu = u + i, pv = v + j;
            if (pu < 0 || pu >= d.H || pv < 0 || pv >= d.W) continue;
            mass += p[(size_t)pu * d.W + pv];
        }
    }
    return mass;
}

static inline int32_t wgsl_i32(float f) {
    // WGSL i32(f32) for the values that occur here (in-range, finite); NaN -> 0.
    if (std::isnan(f)) return 0;
    if (f >= 2147483647.0f) return INT32_MAX;
    if (f <= -2147483648.0f) return INT32_MIN;
    return (int32_t)f;
}
// WGSL u32(f32) for the in-range values that occur here (counts).
static inline uint32_t wgsl_u32(float f) {
    if (!(f > 0.0f)) return 0u;
    if (f >= 4294967295.0f) return UINT32_MAX;
    return (uint32_t)f;
}

static void characterize(const Derived& d, const float* p, const float* raw, Row& row, bool char_points) {
    const int32_t kr = d.circle;
    float r = row.r;
    int32_t rint;
    if (r <= 0.0f) {
        rint = (kr - 1) / 2;
        r = (float)rint;
    } else {
        rint = (int32_t)std::ceil(r);
    }
    const float r2 = r * r;
    const int32_t u = wgsl_i32(std::rint(row.x));
    const int32_t v = wgsl_i32(std::rint(row.y));
    if (char_points) row.mass = get_mass(d, p, u, v, rint, r2);
    const float mass = row.mass;
    // processed_buffer[u * ncols + v] is read unchecked as a flat index
    // (characterize.wgsl:79,131); a flat index outside the buffer reads 0
    // (robust buffer access).
    float middle = 0.0f;
    const int64_t middle_idx = (int64_t)u * d.W + v;
    if (middle_idx >= 0 && middle_idx < (int64_t)d.H * d.W) middle = p[middle_idx];
    float Rg = 0.0f, raw_mass = 0.0f, signal = 0.0f, es = 0.0f, ec = 0.0f;
    for (int32_t i = -rint; i <= rint; i++) {
        float x = (float)i;
        float x2 = x * x;
        for (int32_t j = -rint; j <= rint; j++) {
            float y = (float)j;
            float y2 = y * y;
            float mask = x2 + y2;
            if (mask > r2) continue;
            int32_t pu = u + i, pv = v + j;
            if (pu < 0 || pu >= d.H || pv < 0 || pv >= d.W) continue;
            size_t idx = (size_t)pu * d.W + pv;
            float data = p[idx];
            Rg = std::fmaf(data, mask, Rg);
            raw_mass = raw_mass + raw[idx];
            signal = wgsl_max(signal, data);
            if ((x != 0.0f) | (y != 0.0f)) {
                float theta = std::atan2(y, x);
                es = std::fmaf(data, std::sin(2.0f * theta), es);
                ec = std::fmaf(data, std::cos(2.0f * theta), ec);
            } else {
                ec = ec + data;
            }
        }
    }
    es = es * es;
    ec = ec * ec;
    float ecc = std::sqrt(es + ec) / (mass - middle);
    Rg = std::sqrt(Rg / mass);
    row.Rg = Rg;
    row.raw_mass = raw_mass;
    row.signal = signal;
    row.ecc = ecc;
}

// ------------------------------------------------------------------ LoG
// separable_log.wgsl:22-89 driven by Laplace<2>/SeparableConvolution<2>
// (src/utils.rs:114-296): for diff_dim in {0,1}: dim 0 (along rows) from
// the frame into temp, dim 1 (along columns) from temp into final -= result.
static void log_pass(const Derived& d, const float* in, float* out, int dim, bool deriv, float sigma) {
    const int32_t H = d.H, W = d.W;
    const float sigma2 = sigma * sigma;
    const int32_t rint = (int32_t)(4.0f * sigma + 0.5f);
    const float sqrt2pi = (float)2.5066282746310002;
    float norm = deriv ? 1.0f / (sqrt2pi * sigma * sigma2) : 1.0f / (sqrt2pi * sigma);
    std::vector<float> taps(2 * rint + 1);
    for (int32_t i = -rint; i <= rint; i++) {
        float x = (float)i;
        float x2 = x * x;
        float g = std::exp(-x2 / (2.0f * sigma2));
        taps[i + rint] = deriv ? g * (x2 - sigma2) : g;
    }
    for (int32_t a = 0; a < H; a++) {
        for (int32_t b = 0; b < W; b++) {
            int32_t u, ubound;
            size_t stride;
            if (dim == 0) { u = a; ubound = H; stride = (size_t)W; }
            else { u = b; ubound = W; stride = 1; }
            size_t base = (size_t)a * W + b;
            float s = 0.0f;
            for (int32_t i = -rint; i <= rint; i++) {
                int32_t pu = u + i;
                if (pu < 0 || pu >= ubound) continue;
                s = std::fmaf(taps[i + rint], in[(size_t)((int64_t)base + (int64_t)i * (int64_t)stride)], s);
            }
            out[base] = s * norm;
        }
    }
}

static void laplace(const Derived& d, const float* frame, float sigma, std::vector<float>& temp, float* final_out) {
    const size_t n = (size_t)d.H * d.W;
    temp.resize(n);
    std::vector<float> r(n);
    // diff_dim 0
    log_pass(d, frame, temp.data(), 0, true, sigma);
    log_pass(d, temp.data(), r.data(), 1, false, sigma);
    for (size_t i = 0; i < n; i++) final_out[i] = 0.0f - r[i];
    // diff_dim 1
    log_pass(d, frame, temp.data(), 0, false, sigma);
    log_pass(d, temp.data(), r.data(), 1, true, sigma);
    for (size_t i = 0; i < n; i++) final_out[i] = final_out[i] - r[i];
}

// logspace_max.wgsl:151-243.
static bool is_max_in_plane(const Derived& d, const float* plane, int32_t i, int32_t j, float center) {
    for (int32_t li = -1; li < 2; li++) {
        for (int32_t lj = -1; lj < 2; lj++) {
            if (li == 0 && lj == 0) continue;
            int32_t x = i + li, y = j + lj;
            if (x < 0 || x >= d.H || y < 0 || y >= d.W) return false;
            float nb = plane[(size_t)x * d.W + y];
            if (nb >= center) return false;
        }
    }
    return true;
}

static void logspace_max(const Derived& d, const float* bottom, const float* middle, const float* top,
                         const float* processed, float pic_std, int edge,
                         std::vector<std::pair<int32_t, int32_t>>& cands) {
    cands.clear();
    const float thr = pic_std * d.snr * d.rough;
    for (int32_t i = 0; i < d.H; i++) {
        for (int32_t j = 0; j < d.W; j++) {
            size_t idx = (size_t)i * d.W + j;
            float center = middle[idx];
            if (processed[idx] < thr) continue;
            if (center <= 0.0f) continue;
            if (!is_max_in_plane(d, middle, i, j, center)) continue;
            if (edge != -1 && !is_max_in_plane(d, bottom, i, j, center)) continue;
            if (edge != 1 && !is_max_in_plane(d, top, i, j, center)) continue;
            cands.push_back({i, j});
        }
    }
}

// --------------------------------------------------------- per-frame locate
// ---------------------------------------------------------------- frame std
// StdArray::execute (src/utils.rs:614-640): sum_image_outplace.wgsl (each of
// N/8 outputs sums 8 values N/8 apart, skipping the 0xFFFFFFFF pattern that
// marks masked pixels), sum_image_inplace.wgsl levels (8 values L/8 apart)
// while the length exceeds 24, last_reduction.wgsl (sequential sum / divisor);
// std_image.wgsl ((x - mean)^2, 0 where masked), the same levels from N, then
// sum / (divisor - 1) and sqrt.  Exact only when every level's length is a
// multiple of 8 (std_clean); otherwise the shaders read leftovers of earlier
// passes beyond the valid length.
static inline uint32_t f32_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
static inline float bits_f32(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
static constexpr uint32_t kMaskedPixel = 0xFFFFFFFFu;

static bool std_clean(int64_t N) {
    if (N <= 0 || N % 8) return false;
    for (int64_t L : {N / 8, N}) {
        while (L > 24) {
            if (L % 8) return false;
            L /= 8;
        }
    }
    return true;
}

static float frame_std(const float* f, int64_t N, uint32_t divisor, std::vector<float>& tmp) {
    tmp.resize((size_t)N);
    auto levels = [&](int64_t L) {
        while (L > 24) {
            const int64_t t = L / 8;
            for (int64_t i = 0; i < t; i++) {
                float sum = 0.0f;
                for (int k = 0; k < 8; k++) sum += tmp[(size_t)(i + k * t)];
                tmp[(size_t)i] = sum;
            }
            L = t;
        }
        return L;
    };
    const int64_t s = N / 8;
    for (int64_t i = 0; i < s; i++) {
        float sum = 0.0f;
        for (int k = 0; k < 8; k++) {
            const float v = f[i + k * s];
            if (f32_bits(v) != kMaskedPixel) sum += v;
        }
        tmp[(size_t)i] = sum;
    }
    int64_t L = levels(s);
    float mean = 0.0f;
    for (int64_t i = 0; i < L; i++) mean += tmp[(size_t)i];
    mean /= (float)divisor;
    for (int64_t i = 0; i < N; i++) {
        const float v = f[i];
        if (f32_bits(v) != kMaskedPixel) {
            const float diff = v - mean;
            tmp[(size_t)i] = diff * diff;
        } else {
            tmp[(size_t)i] = 0.0f;
        }
    }
    L = levels(N);
    float var = 0.0f;
    for (int64_t i = 0; i < L; i++) var += tmp[(size_t)i];
    var /= (float)(divisor - 1u);
    return std::sqrt(var);
}

// adaptive_filter.wgsl set_nan: the row's circle marked as masked.
static void mask_circle(const Derived& d, const Row& row, float* frame) {
    const int32_t rint = (row.r > 0.0f) ? wgsl_i32(std::ceil(row.r)) : (d.circle - 1) / 2;
    const int32_t u = wgsl_i32(std::rint(row.x)), v = wgsl_i32(std::rint(row.y));
    const float r = (float)rint;
    const float r2 = r * r;
    for (int32_t i = -rint; i <= rint; i++) {
        const float x = (float)i;
        const float x2 = x * x;
        for (int32_t j = -rint; j <= rint; j++) {
            const float y = (float)j;
            const float y2 = y * y;
            if (x2 + y2 > r2) continue;
            const int32_t pu = u + i, pv = v + j;
            if (pu < 0 || pu >= d.H || pv < 0 || pv >= d.W) continue;
            frame[(size_t)pu * d.W + pv] = bits_f32(kMaskedPixel);
        }
    }
}

// The adaptive_background loop (src/execute_gpu.rs:289-366 with
// adaptive_filter.wgsl): n_iter passes over the rows not yet accepted; a row
// is accepted unless mass < minmass (minmass_snr * count * std when minmass
// is not positive) or max_intensity < snr * std; an accepted row masks its
// circle and takes its count off the divisor; before every pass but the
// first the std is recomputed on the masked frame.  The accepted rows keep
// their canonical order (the reference appends them with atomics).
static void adaptive_filter(const Derived& d, uint32_t n_iter, bool recompute, const float* img, float std0,
                            std::vector<Row>& rows, std::vector<float>& frame, std::vector<float>& tmp) {
    const int64_t N = (int64_t)d.H * d.W;
    frame.assign(img, img + N);
    uint32_t counter = (uint32_t)N;
    float sd = std0;
    std::vector<Row> pending = rows, accepted, next;
    for (uint32_t it = 0; it < n_iter; it++) {
        if (it > 0 && recompute) sd = frame_std(frame.data(), N, counter, tmp);
        next.clear();
        for (const Row& row : pending) {
            float minmass;
            if (d.minmass > 0.0f) minmass = d.minmass;
            else minmass = d.minmass_snr * row.count * sd;
            if ((row.mass < minmass) || (row.max_intensity < d.snr * sd)) {
                next.push_back(row);
            } else {
                mask_circle(d, row, frame.data());
                counter -= wgsl_u32(row.count);
                accepted.push_back(row);
            }
        }
        pending.swap(next);
    }
    std::stable_sort(accepted.begin(), accepted.end(), [](const Row& a, const Row& b) { return a.key < b.key; });
    rows.swap(accepted);
}

struct FrameScratch {
    std::vector<float> tg, tb, processed, mr, temp, masked, stdtmp;
    std::vector<std::vector<float>> planes;
    std::vector<std::pair<int32_t, int32_t>> cands;
};

// ------------------------------------------------------ illumination profile
// smooth_mean_frame.wgsl through SeparableConvolution<2> (src/utils.rs:120-245,
// src/gpu_setup.rs:317-340): pass 0 along the rows' direction (u = row), then
// pass 1 along the columns, each result = sum_i gauss_i * x / sum_i gauss_i
// over the in-frame taps i in [-rint, rint], rint = i32(4 sigma + 0.5),
// gauss_i = exp(-x^2 / (2 sigma^2)); the accumulation of gauss * x is a fused
// multiply-add (`gauss_sum += gauss * input[...]`).  n_frames = 1 in every
// call the reference makes, so pass 0's norm is unchanged.
static void smooth_profile(const float* in, int32_t H, int32_t W, float sigma, float* out, std::vector<float>& tmp) {
    const float sigma2 = sigma * sigma;
    const int32_t rint = wgsl_i32(4.0f * sigma + 0.5f);
    std::vector<float> g((size_t)(2 * rint + 1));
    for (int32_t i = -rint; i <= rint; i++) {
        const float x = (float)i;
        const float x2 = x * x;
        g[(size_t)(i + rint)] = std::exp(-x2 / (2.0f * sigma2));
    }
    tmp.resize((size_t)H * W);
    for (int pass = 0; pass < 2; pass++) {
        const float* src = pass == 0 ? in : tmp.data();
        float* dst = pass == 0 ? tmp.data() : out;
        for (int32_t r = 0; r < H; r++) {
            for (int32_t c = 0; c < W; c++) {
                const int32_t u = pass == 0 ? r : c;
                const int32_t bound = pass == 0 ? H : W;
                float gsum = 0.0f, nsum = 0.0f;
                for (int32_t i = -rint; i <= rint; i++) {
                    const int32_t pu = u + i;
                    if (pu < 0 || pu >= bound) continue;
                    const size_t idx = pass == 0 ? (size_t)pu * W + c : (size_t)r * W + pu;
                    const float gv = g[(size_t)(i + rint)];
                    gsum = std::fmaf(gv, src[idx], gsum);
                    nsum += gv;
                }
                float norm = nsum;
                if (pass == 0) norm *= 1.0f;
                dst[(size_t)r * W + c] = gsum / norm;
            }
        }
    }
}

// The illumination-corrected frames (src/execute_gpu.rs:138-166, 819-884):
// the profile is the smoothed mean frame (mean_from_iter: sequential sum over
// the frames, / n_frames) or, per frame, the smoothed frame itself; every
// pixel is divided by it (correct_illumination.wgsl: acc /= frame).
static void illumination_correct(const gt_params& p, const float* frames, int64_t T, int32_t H, int32_t W,
                                 std::vector<float>& out) {
    const size_t npix = (size_t)H * W;
    out.resize((size_t)T * npix);
    std::vector<float> prof(npix), tmp;
    if (!p.illumination_correction_per_frame) {
        std::vector<float> mean(npix, 0.0f);
        for (int64_t t = 0; t < T; t++)
            for (size_t i = 0; i < npix; i++) mean[i] += frames[(size_t)t * npix + i];
        const float nf = (float)T;
        for (size_t i = 0; i < npix; i++) mean[i] /= nf;
        smooth_profile(mean.data(), H, W, p.illumination_sigma, prof.data(), tmp);
    }
    for (int64_t t = 0; t < T; t++) {
        const float* f = frames + (size_t)t * npix;
        if (p.illumination_correction_per_frame) smooth_profile(f, H, W, p.illumination_sigma, prof.data(), tmp);
        for (size_t i = 0; i < npix; i++) out[(size_t)t * npix + i] = f[i] / prof[i];
    }
}

// snr / minmass_snr / adaptive_background combinations this restatement
// reproduces (the library accepts the same ones):
//  * the frame std needs a pixel count whose reduction levels are all
//    multiples of 8 (std_clean);
//  * adaptive_background = 0 and adaptive_background >= 2 without snr or
//    minmass_snr make the reference panic (an empty pass iterator, a missing
//    std pass: src/execute_gpu.rs:297-310).
static int check_std_params(const gt_params& p, int64_t N) {
    const bool std_pass = p.has_snr || p.has_minmass_snr;
    if (std_pass && !std_clean(N)) return GT_ERR_INVALID_ARGUMENT;
    if (p.has_adaptive_background) {
        if (p.adaptive_background == 0) return GT_ERR_INVALID_ARGUMENT;
        if (p.adaptive_background >= 2 && !std_pass) return GT_ERR_INVALID_ARGUMENT;
    }
    return GT_OK;
}

// One frame through the shader passes in the reference's order
// (src/gpu_setup.rs:872-895 and src/execute_gpu.rs:231-286, 368-375).
static void locate_frame(const gt_params& p, const Derived& d, const std::vector<float>& radii, const float* img,
                         FrameScratch& s, std::vector<Row>& rows) {
    const size_t n = (size_t)d.H * d.W;
    s.processed.resize(n);
    preprocess(d, p.truncate_preprocessed != 0, img, s.tg, s.tb, s.processed.data());
    // the std buffer is written only when snr or minmass_snr is set (src/gpu_setup.rs:990)
    const bool std_pass = p.has_snr || p.has_minmass_snr;
    const float pic_std = std_pass ? frame_std(img, (int64_t)n, (uint32_t)n, s.stdtmp) : 0.0f;
    rows.clear();
    if (p.style == GT_STYLE_TRACKPY) {
        extract_max(d, s.processed.data(), pic_std, s.mr, s.cands);
        for (auto& c : s.cands) {
            Row row;
            if (walk_keep(d, s.processed.data(), c.first, c.second, -1.0f, pic_std, row)) { row.key = (int64_t)rows.size(); rows.push_back(row); }
        }
    } else {
        const size_t nr = radii.size();
        s.planes.assign(3, std::vector<float>(n, 0.0f));
        auto sig = [&](size_t i) { return radii[i] / std::sqrt(2.0f); };
        if (nr == 0) return;
        laplace(d, img, sig(0), s.temp, s.planes[0].data());
        int edge = -1;
        for (size_t i = 1; i < nr; i++) {
            laplace(d, img, sig(i), s.temp, s.planes[i % 3].data());
            size_t mid = (i - 1) % 3;
            const float* bottom = s.planes[(mid + 2) % 3].data();
            const float* top = s.planes[(mid + 1) % 3].data();
            logspace_max(d, bottom, s.planes[mid].data(), top, s.processed.data(), pic_std, edge, s.cands);
            for (auto& c : s.cands) {
                Row row;
                if (walk_keep(d, s.processed.data(), c.first, c.second, radii[i - 1], pic_std, row))
                    { row.key = (int64_t)rows.size(); rows.push_back(row); }
            }
            edge = 0;
        }
        edge = 1;
        size_t mid = (nr - 1) % 3;
        const float* bottom = s.planes[(mid + 2) % 3].data();
        const float* top = s.planes[(mid + 1) % 3].data();
        logspace_max(d, bottom, s.planes[mid].data(), top, s.processed.data(), pic_std, edge, s.cands);
        for (auto& c : s.cands) {
            Row row;
            if (walk_keep(d, s.processed.data(), c.first, c.second, radii[nr - 1], pic_std, row)) { row.key = (int64_t)rows.size(); rows.push_back(row); }
        }
    }
    if (p.has_adaptive_background)
        adaptive_filter(d, p.adaptive_background, std_pass, img, pic_std, rows, s.masked, s.stdtmp);
    // characterize reads the unmasked frame (raw_frame, src/gpu_setup.rs:194-205)
    if (p.characterize) {
        for (auto& row : rows) characterize(d, s.processed.data(), img, row, false);
    }
}

// --------------------------------------------------------- neighbour query
// within_radius_rd2 (src/linking.rs:211-247): box prefilter on each axis,
// then squared distance accumulated as 0 + dx^2 + dy^2 (item - query),
// strict `< r^2`.  Results in index order (the kd-tree's order is not
// reproducible without the crate; it only matters on exact cost ties).
static inline bool within(float ix, float iy, float qx, float qy, float radius, float& dist) {
    if (ix < qx - radius || ix > qx + radius) return false;
    if (iy < qy - radius || iy > qy + radius) return false;
    float r2 = radius * radius;
    float dx = ix - qx;
    float dy = iy - qy;
    float s = 0.0f;
    s += dx * dx;
    s += dy * dy;
    dist = s;
    return s < r2;
}

// filter_close_trackpy (src/execute_gpu.rs:556-590).
static std::vector<Row> filter_close(const std::vector<Row>& rows, float separation) {
    std::vector<Row> out;
    for (size_t idx = 0; idx < rows.size(); idx++) {
        const Row& q = rows[idx];
        bool keep = true;
        for (size_t n = 0; n < rows.size() && keep; n++) {
            if (n == idx) continue;
            float dist;
            if (!within(rows[n].x, rows[n].y, q.x, q.y, separation, dist)) continue;
            float nm = rows[n].mass;
            if (q.mass < nm) keep = false;
            else if (q.mass == nm && idx > n) keep = false;
        }
        if (keep) out.push_back(q);
    }
    return out;
}

// prune_blobs_log (src/execute_gpu.rs:592-669), input presorted.
static float disk_overlap(float d, float r1, float r2) {
    auto make_acos = [](float d, float r1, float r1s, float r2s) {
        float ratio = (d * d + r1s - r2s) / (2.0f * d * r1);
        ratio = std::min(std::max(ratio, -1.0f), 1.0f);
        return std::acos(ratio);
    };
    float r1s = r1 * r1;
    float r2s = r2 * r2;
    float acos1 = make_acos(d, r1, r1s, r2s);
    float acos2 = make_acos(d, r2, r2s, r1s);
    float a = -d + r2 + r1;
    float b = d - r2 + r1;
    float c = d + r2 - r1;
    float dd = d + r2 + r1;
    float area = r1s * acos1 + r2s * acos2 - 0.5f * std::sqrt(std::fabs(a * b * c * dd));
    return area / ((float)M_PI * std::min(r1s, r2s));
}

static float blob_overlap(const Row& b1, const Row& b2, float distance) {
    if (distance > b1.r + b2.r) return 0.0f;
    else if (distance <= std::fabs(b1.r - b2.r)) return 1.0f;
    else return disk_overlap(distance, b1.r, b2.r);
}

static std::vector<Row> prune_blobs_log(const std::vector<Row>& rows, float overlap_threshold) {
    std::vector<char> keep(rows.size(), 1);
    for (size_t idx = 0; idx < rows.size(); idx++) {
        if (!keep[idx]) continue;
        const Row& q = rows[idx];
        float qr = q.r * 2.0f;
        for (size_t n = 0; n < rows.size(); n++) {
            if (n == idx) continue;
            float d2;
            if (!within(rows[n].x, rows[n].y, q.x, q.y, qr, d2)) continue;
            if (!keep[n]) continue;
            float ov = blob_overlap(q, rows[n], std::sqrt(d2));
            if (ov > overlap_threshold) keep[n] = 0;
        }
    }
    std::vector<Row> out;
    for (size_t i = 0; i < rows.size(); i++)
        if (keep[i]) out.push_back(rows[i]);
    return out;
}

// circle_inds / annulus_inds (src/kernels.rs:138-171).
static std::vector<std::array<int32_t, 2>> circle_inds(float radius) {
    int32_t rb = (int32_t)std::ceil(radius);
    std::vector<std::array<int32_t, 2>> inds;
    float r2 = radius * radius;
    for (int32_t i = -rb; i < rb + 1; i++)
        for (int32_t j = -rb; j < rb + 1; j++)
            if ((float)(i * i + j * j) <= r2) inds.push_back({i, j});
    return inds;
}

static std::vector<std::array<int32_t, 2>> annulus_inds(float outer, float inner) {
    int32_t b = (int32_t)std::ceil(outer);
    std::vector<std::array<int32_t, 2>> inds;
    float or2 = outer * outer, ir2 = inner * inner;
    for (int32_t i = -b; i < b + 1; i++)
        for (int32_t j = -b; j < b + 1; j++) {
            float r2 = (float)(i * i + j * j);
            if (r2 <= or2 && r2 >= ir2) inds.push_back({i, j});
        }
    return inds;
}

static inline int32_t rust_f32_to_i32(float f) {
    if (std::isnan(f)) return 0;
    if (f >= 2147483647.0f) return INT32_MAX;
    if (f <= -2147483648.0f) return INT32_MIN;
    return (int32_t)f;
}

// Doughnut block of post_process (src/execute_gpu.rs:717-790).
static void doughnut(const gt_params& p, const Derived& d, const float* frame, std::vector<Row>& rows) {
    std::vector<float> sig, bg;
    for (auto& row : rows) {
        float radius = (p.style == GT_STYLE_TRACKPY) ? (float)p.diameter / 2.0f : row.r;
        auto sig_inds = circle_inds(radius);
        float outer = p.has_bg_radius ? p.bg_radius : 2.0f * radius;
        float gap = (p.has_bg_radius && p.has_gap_radius) ? p.gap_radius : 0.0f;
        auto bg_inds = annulus_inds(outer, gap + radius);
        int32_t mu = rust_f32_to_i32(std::round(row.x));
        int32_t mv = rust_f32_to_i32(std::round(row.y));
        sig.clear();
        bg.clear();
        for (auto& ind : sig_inds) {
            int64_t a = (int64_t)mu + ind[0], b = (int64_t)mv + ind[1];
            if (a >= 0 && a < d.H && b >= 0 && b < d.W) sig.push_back(frame[(size_t)a * d.W + b]);
        }
        for (auto& ind : bg_inds) {
            int64_t a = (int64_t)mu + ind[0], b = (int64_t)mv + ind[1];
            if (a >= 0 && a < d.H && b >= 0 && b < d.W) bg.push_back(frame[(size_t)a * d.W + b]);
        }
        float sum = 0.0f;
        for (float s : sig) sum = sum + s;
        std::sort(bg.begin(), bg.end());
        float med = bg.empty() ? 0.0f : bg[bg.size() / 2];
        float corrected = sum - med * (float)sig.size();
        row.d_raw_mass = sum;
        row.d_bg_median = med;
        row.d_corrected = corrected;
    }
}

// ------------------------------------------------------------------ linker
// Linker / link (src/linking.rs:345-816).
struct Dur { size_t start; size_t duration; };
using Pos = std::array<float, 2>;
using Src = std::pair<Pos, size_t>;

struct TooDense : std::exception {};

static std::vector<size_t> link_frame(const std::vector<Src>& src, const std::vector<Pos>& dest, bool has_mem_start,
                                      size_t memory_start_idx, float radius, size_t& counter,
                                      std::vector<Src>& unused_out) {
    const size_t S = src.size(), D = dest.size();
    std::vector<std::vector<std::pair<size_t, float>>> s2d(S), d2s(D);
    for (size_t s = 0; s < S; s++) {
        for (size_t dd = 0; dd < D; dd++) {
            float dist;
            if (within(dest[dd][0], dest[dd][1], src[s].first[0], src[s].first[1], radius, dist)) {
                s2d[s].push_back({dd, dist});
                d2s[dd].push_back({s, dist});
            }
        }
    }
    std::vector<char> vis0(S, 0), vis1(D, 0);
    std::vector<std::array<std::vector<size_t>, 2>> paths;
    size_t load = 0;
    std::vector<int64_t> output(D, -1);
    std::function<void(size_t, int, std::array<std::vector<size_t>, 2>&)> recurse =
        [&](size_t node, int side, std::array<std::vector<size_t>, 2>& path) {
            if (side == 0) {
                if (vis0[node]) return;
                vis0[node] = 1;
                path[0].push_back(node);
                for (auto& e : s2d[node]) recurse(e.first, 1, path);
            } else {
                if (vis1[node]) return;
                vis1[node] = 1;
                path[1].push_back(node);
                for (auto& e : d2s[node]) recurse(e.first, 0, path);
            }
        };
    for (size_t i = 0; i < D; i++) {
        std::array<std::vector<size_t>, 2> path;
        recurse(i, 1, path);
        if (path[1].size() == 1) {
            if (path[0].size() == 0) {
            } else if (path[0].size() == 1) {
                output[i] = (int64_t)src[path[0][0]].second;
            } else {
                paths.push_back(path);
            }
        } else if (path[1].size() > 0) {
            load += path[0].size() * path[1].size();
            paths.push_back(path);
        }
    }
    if (load > 5000) throw TooDense();

    const float default_score = radius * radius;
    for (auto& path : paths) {
        std::unordered_map<size_t, size_t> used;   // src ident -> dest
        std::unordered_set<size_t> nulls;
        float score = 0.0f;
        float best = std::numeric_limits<float>::infinity();
        std::function<void(size_t)> recurse2 = [&](size_t progress) {
            size_t cur = path[1][progress];
            size_t nopt = d2s[cur].size() + 1;
            for (size_t o = 0; o < nopt; o++) {
                bool is_null = (o == d2s[cur].size());
                size_t ident = is_null ? 0 : src[d2s[cur][o].first].second;
                float c = is_null ? default_score : d2s[cur][o].second;
                if (score > best) return;
                score += c;
                if (!is_null) {
                    if (used.count(ident)) { score -= c; continue; }
                    used[ident] = cur;
                } else {
                    nulls.insert(cur);
                }
                if (progress == path[1].size() - 1) {
                    if (score < best) {
                        best = score;
                        for (auto& kv : used) output[kv.second] = (int64_t)kv.first;
                        for (auto& nl : nulls) output[nl] = -1;
                    }
                } else {
                    recurse2(progress + 1);
                }
                if (!is_null) used.erase(ident);
                else nulls.erase(cur);
                score -= c;
            }
        };
        recurse2(0);
    }
    std::vector<size_t> out(D);
    for (size_t i = 0; i < D; i++) {
        if (output[i] >= 0) out[i] = (size_t)output[i];
        else out[i] = counter++;
    }
    std::unordered_set<size_t> used_sources(out.begin(), out.end());
    unused_out.clear();
    size_t lim = has_mem_start ? std::min(memory_start_idx, S) : S;
    for (size_t i = 0; i < lim; i++)
        if (!used_sources.count(src[i].second)) unused_out.push_back(src[i]);
    return out;
}

struct Linker {
    float search_range;
    size_t memory;
    std::vector<Src> prev;
    size_t prev_N = 0;
    bool has_mem;
    std::deque<std::vector<Src>> memvec;
    size_t frame_idx = 0, part_idx = 0;
    std::vector<Dur> starting_frame;

    Linker(float sr, size_t mem) : search_range(sr), memory(mem), has_mem(mem > 0) {
        if (has_mem)
            for (size_t i = 0; i < mem; i++) memvec.push_back({});
    }
    void reset() { *this = Linker(search_range, memory); }

    // Linker::advance (src/linking.rs:435-503)
    std::vector<size_t> advance(const std::vector<Pos>& frame) {
        size_t N = frame.size();
        bool has_start = false;
        size_t mstart = 0;
        if (has_mem) {
            std::unordered_set<size_t> memset;
            for (auto& e : prev) memset.insert(e.second);
            for (auto& vec : memvec)
                for (auto& e : vec)
                    if (!memset.count(e.second)) {
                        prev.push_back(e);
                        memset.insert(e.second);
                    }
            has_start = true;
            mstart = prev_N;
        }
        size_t prev_part = part_idx;
        std::vector<Src> unused;
        std::vector<size_t> result = link_frame(prev, frame, has_start, mstart, search_range, part_idx, unused);
        for (size_t i = 0; i < part_idx - prev_part; i++) starting_frame.push_back({frame_idx, 0});
        prev.clear();
        for (size_t i = 0; i < N; i++) prev.push_back({frame[i], result[i]});
        if (has_mem) {
            memvec.push_back(unused);
            std::vector<Src> leaving = memvec.front();
            memvec.pop_front();
            for (auto& e : leaving) {
                Dur& sf = starting_frame.at(e.second);
                sf.duration = (frame_idx - sf.start) - memvec.size();
            }
        } else {
            for (auto& e : unused) {
                Dur& sf = starting_frame.at(e.second);
                sf.duration = frame_idx - sf.start;
            }
        }
        prev_N = N;
        frame_idx += 1;
        return result;
    }

    // Linker::finish (src/linking.rs:505-520)
    std::vector<Dur> finish() {
        if (has_mem) {
            size_t i = 0;
            for (auto& vec : memvec) {
                for (auto& e : vec) {
                    Dur& sf = starting_frame.at(e.second);
                    sf.duration = (frame_idx - sf.start) - (memvec.size() - i);
                }
                i++;
            }
        }
        for (auto& e : prev) {
            Dur& sf = starting_frame.at(e.second);
            sf.duration = frame_idx - sf.start;
        }
        return starting_frame;
    }

    // Linker::connect (src/linking.rs:405-433)
    std::pair<std::vector<size_t>, std::vector<size_t>> connect(const std::vector<Pos>& f1, const std::vector<Pos>& f2) {
        std::vector<Src> pv;
        for (auto& e : f1) pv.push_back({e, part_idx++});
        std::vector<Src> unused;
        std::vector<size_t> result = link_frame(pv, f2, false, 0, search_range, part_idx, unused);
        std::vector<size_t> first;
        for (auto& e : pv) first.push_back(e.second);
        return {first, result};
    }
};

// FrameSubsetter over an (n, 3) [frame, y, x] array (src/linking.rs:97-196),
// linking flavour; includes the reference's leading empty frame 0 when the
// first frame number is positive.
struct Subsetter {
    const float* arr;
    int64_t n;
    int64_t idx = 0;
    float cur = 0.0f;
    bool done = false;
    // returns 1 = item, 0 = end, -1 = error (NonSorted)
    int next(size_t& frame_out, std::vector<Pos>& out) {
        out.clear();
        while (true) {
            if (idx < n) {
                float f = arr[idx * 3 + 0];
                if (f > cur) {
                    frame_out = (size_t)cur;
                    cur = f;
                    return 1;
                }
                if (f < cur) return -1;
            } else {
                if (!out.empty()) {
                    frame_out = (size_t)cur;
                    idx = n + 1;
                    return 1;
                }
                return 0;
            }
            out.push_back({arr[idx * 3 + 1], arr[idx * 3 + 2]});
            idx++;
        }
    }
};

}  // namespace oracle

// ====================================================================== C API
using namespace oracle;

struct OracleTable {
    std::vector<double> data;  // nrows x GT_NUM_COLUMNS, NaN where absent
    int64_t nrows = 0;
};

static void put_row(OracleTable& t, int64_t frame, const Row& r, bool has_doughnut) {
    double v[GT_NUM_COLUMNS];
    for (int c = 0; c < GT_NUM_COLUMNS; c++) v[c] = NAN;
    v[GT_COL_FRAME] = (double)frame;
    v[GT_COL_Y] = r.x;
    v[GT_COL_X] = r.y;
    v[GT_COL_MASS] = r.mass;
    v[GT_COL_R] = r.r;
    v[GT_COL_RG] = r.Rg;
    v[GT_COL_RAW] = r.raw_mass;
    v[GT_COL_SIGNAL] = r.signal;
    v[GT_COL_ECC] = r.ecc;
    if (has_doughnut) {
        v[GT_COL_RAW_MASS] = r.d_raw_mass;
        v[GT_COL_RAW_BG_MEDIAN] = r.d_bg_median;
        v[GT_COL_RAW_MASS_CORRECTED] = r.d_corrected;
    }
    v[GT_COL_PARTICLE] = (double)r.particle;
    v[GT_COL_DURATION] = (double)r.duration;
    v[GT_COL_MAX_INTENSITY] = r.max_intensity;
    v[GT_COL_COUNT] = r.count;
    t.data.insert(t.data.end(), v, v + GT_NUM_COLUMNS);
    t.nrows++;
}

// Post-processing over frames in order (src/execute_gpu.rs:671-817, 1165-1181).
static int post_process_all(const gt_params& p, const Derived& d, const float* frames,
                            std::vector<std::vector<Row>>& per_frame, const int64_t* frame_numbers,
                            const int64_t* reset, int64_t n_reset, OracleTable& table) {
    const size_t T = per_frame.size();
    const size_t npix = (size_t)d.H * d.W;
    bool link = p.has_search_range != 0;
    Linker linker(p.search_range, p.memory);
    std::vector<std::vector<Row>> kept(T);
    for (size_t t = 0; t < T; t++) {
        std::vector<Row> rel;
        if (p.style == GT_STYLE_TRACKPY) {
            if (p.filter_close) rel = filter_close(per_frame[t], (float)p.separation);
            else rel = per_frame[t];
        } else {
            rel = per_frame[t];
            if (p.overlap_threshold < 1.0f) {
                std::stable_sort(rel.begin(), rel.end(), [](const Row& a, const Row& b) {
                    if (a.r != b.r) return b.r < a.r;
                    return b.mass < a.mass;
                });
                rel = prune_blobs_log(rel, p.overlap_threshold);
            }
        }
        if (p.doughnut_correction) doughnut(p, d, frames + t * npix, rel);
        int64_t fnum = frame_numbers ? frame_numbers[t] : (int64_t)t;
        if (link) {
            for (int64_t k = 0; k < n_reset; k++)
                if (reset[k] == fnum) { linker.reset(); break; }
            std::vector<Pos> pos;
            for (auto& r : rel) pos.push_back({r.x, r.y});
            try {
                auto ids = linker.advance(pos);
                for (size_t i = 0; i < rel.size(); i++) rel[i].particle = (int64_t)ids[i];
            } catch (TooDense&) {
                return GT_ERR_TOO_DENSE_TO_LINK;
            }
        }
        kept[t] = std::move(rel);
    }
    std::vector<Dur> durs;
    if (link) durs = linker.finish();
    for (size_t t = 0; t < T; t++) {
        int64_t fnum = frame_numbers ? frame_numbers[t] : (int64_t)t;
        for (auto& r : kept[t]) {
            Row rr = r;
            if (link) {
                // ids travel through f32 in the reference's output matrix
                // (src/execute_gpu.rs:812-815, 1165-1181)
                size_t pid = (size_t)(float)rr.particle;
                if (pid >= durs.size()) return GT_ERR_INTERNAL;
                rr.particle = (int64_t)pid;
                rr.duration = (int64_t)durs[pid].duration;
            }
            put_row(table, fnum, rr, p.doughnut_correction != 0);
        }
    }
    return GT_OK;
}

extern "C" {

// The WGSL Params uniform (params.wgsl:1-20) as gpuparams_from_tracking_params
// fills it (src/gpu_setup.rs:528-580): 16 four-byte fields in order.
int oracle_gpu_params(const gt_params* p, int32_t H, int32_t W, void* out16) {
    Derived d = derive(*p, H, W);
    int32_t* o = (int32_t*)out16;
    float* f = (float*)out16;
    o[0] = H; o[1] = W; o[2] = d.smoothing; o[3] = d.smoothing;
    f[4] = d.sigma2;
    o[5] = d.circle; o[6] = d.circle; o[7] = d.dilation; o[8] = d.dilation;
    ((uint32_t*)out16)[9] = d.max_iterations;
    f[10] = d.threshold; f[11] = d.minmass;
    o[12] = d.margin;
    f[13] = d.snr; f[14] = d.minmass_snr; f[15] = d.rough;
    return GT_OK;
}

int32_t oracle_params_sizeof(void) { return (int32_t)sizeof(gt_params); }

int oracle_log_radii(const gt_params* p, float* out) {
    auto r = log_radii(*p);
    for (size_t i = 0; i < r.size(); i++) out[i] = r[i];
    return (int)r.size();
}

int oracle_preprocess(const gt_params* p, const float* frame, int32_t H, int32_t W, float* out) {
    Derived d = derive(*p, H, W);
    std::vector<float> tg, tb;
    preprocess(d, p->truncate_preprocessed != 0, frame, tg, tb, out);
    return GT_OK;
}

// The smoothed illumination profile of one frame (SeparableConvolution<2>
// with smooth_mean_frame.wgsl).
int oracle_smooth_profile(const float* in, int32_t H, int32_t W, float sigma, float* out) {
    std::vector<float> tmp;
    smooth_profile(in, H, W, sigma, out, tmp);
    return GT_OK;
}

// Frame std as the reference computes it (StdArray::execute); frame may
// hold the 0xFFFFFFFF masked-pixel pattern.  Returns an error for pixel
// counts whose reduction is not exact (see std_clean).
int oracle_frame_std(const float* frame, int64_t N, uint32_t divisor, float* out) {
    if (!std_clean(N)) return GT_ERR_INVALID_ARGUMENT;
    std::vector<float> tmp;
    *out = frame_std(frame, N, divisor, tmp);
    return GT_OK;
}

// The adaptive_background passes over walked rows (10 floats each, ResultRow
// order); rows_out gets the accepted rows in canonical (input) order.
int64_t oracle_adaptive(const gt_params* p, const float* frame, int32_t H, int32_t W, const float* rows_in, int64_t n,
                        uint32_t n_iter, float std0, int32_t recompute, float* rows_out) {
    Derived d = derive(*p, H, W);
    std::vector<Row> rows((size_t)n);
    for (int64_t i = 0; i < n; i++) {
        const float* r = rows_in + 10 * i;
        Row& w = rows[(size_t)i];
        w.x = r[0]; w.y = r[1]; w.mass = r[2]; w.r = r[3]; w.max_intensity = r[4];
        w.Rg = r[5]; w.raw_mass = r[6]; w.signal = r[7]; w.ecc = r[8]; w.count = r[9];
        w.key = i;
    }
    std::vector<float> masked, tmp;
    adaptive_filter(d, n_iter, recompute != 0, frame, std0, rows, masked, tmp);
    for (size_t i = 0; i < rows.size(); i++) {
        const Row& w = rows[i];
        float* r = rows_out + 10 * i;
        r[0] = w.x; r[1] = w.y; r[2] = w.mass; r[3] = w.r; r[4] = w.max_intensity;
        r[5] = w.Rg; r[6] = w.raw_mass; r[7] = w.signal; r[8] = w.ecc; r[9] = w.count;
    }
    return (int64_t)rows.size();
}

int64_t oracle_candidates(const gt_params* p, const float* processed, int32_t H, int32_t W, float pic_std,
                          int32_t* uv_out, int64_t cap) {
    Derived d = derive(*p, H, W);
    std::vector<float> mr;
    std::vector<std::pair<int32_t, int32_t>> c;
    extract_max(d, processed, pic_std, mr, c);
    for (int64_t i = 0; i < (int64_t)c.size() && i < cap; i++) {
        uv_out[2 * i] = c[i].first;
        uv_out[2 * i + 1] = c[i].second;
    }
    return (int64_t)c.size();
}

// Walk + (optional) characterize for the given candidates on a processed
// frame; writes one 10-float ResultRow per candidate and keep flags.
int oracle_walk(const gt_params* p, const float* processed, const float* raw, int32_t H, int32_t W,
                const int32_t* uv, int64_t n, float r, float pic_std, float* rows_out, int32_t* keep_out) {
    Derived d = derive(*p, H, W);
    for (int64_t i = 0; i < n; i++) {
        Row row;
        bool k = walk_keep(d, processed, uv[2 * i], uv[2 * i + 1], r, pic_std, row);
        if (!k) {
            WalkResult w = walk(d, processed, uv[2 * i], uv[2 * i + 1], r);
            row.x = w.x; row.y = w.y; row.mass = w.mass; row.count = w.count; row.max_intensity = w.max;
        }
        if (k && p->characterize) characterize(d, processed, raw, row, false);
        float* o = rows_out + 10 * i;
        o[0] = row.x; o[1] = row.y; o[2] = row.mass; o[3] = row.r; o[4] = row.max_intensity;
        o[5] = row.Rg; o[6] = row.raw_mass; o[7] = row.signal; o[8] = row.ecc; o[9] = row.count;
        keep_out[i] = k ? 1 : 0;
    }
    return GT_OK;
}

// n_radii LoG planes (radius order) and the radii.
int oracle_log_planes(const gt_params* p, const float* frame, int32_t H, int32_t W, float* planes, float* radii_out) {
    Derived d = derive(*p, H, W);
    auto radii = log_radii(*p);
    std::vector<float> temp;
    for (size_t i = 0; i < radii.size(); i++) {
        radii_out[i] = radii[i];
        laplace(d, frame, radii[i] / std::sqrt(2.0f), temp, planes + i * (size_t)H * W);
    }
    return GT_OK;
}

int oracle_batch(const gt_params* p, const float* frames, int64_t T, int32_t H, int32_t W,
                 const int64_t* frame_numbers, const int64_t* reset, int64_t n_reset, int32_t nthreads,
                 void** out_table) {
    if (T <= 0) return GT_ERR_EMPTY_ITERATOR;
    {
        const int st = check_std_params(*p, (int64_t)H * W);
        if (st != GT_OK) return st;
    }
    Derived d = derive(*p, H, W);
    auto radii = log_radii(*p);
    std::vector<std::vector<Row>> per_frame((size_t)T);
    const size_t npix = (size_t)H * W;
    // with illumination correction every stage but the doughnut sees the
    // corrected frames (the doughnut reads the host frames)
    std::vector<float> corrected;
    if (p->has_illumination_sigma) illumination_correct(*p, frames, T, H, W, corrected);
    const float* located = p->has_illumination_sigma ? corrected.data() : frames;
    // frames are independent: locate them on nthreads host threads
    if (nthreads <= 0) nthreads = (int32_t)std::max(1u, std::thread::hardware_concurrency());
    nthreads = (int32_t)std::min<int64_t>(nthreads, T);
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        FrameScratch s;
        for (int64_t t = next++; t < T; t = next++)
            locate_frame(*p, d, radii, located + (size_t)t * npix, s, per_frame[(size_t)t]);
    };
    std::vector<std::thread> pool;
    for (int32_t i = 1; i < nthreads; i++) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    OracleTable* table = new OracleTable();
    int st = post_process_all(*p, d, frames, per_frame, frame_numbers, reset, n_reset, *table);
    if (st != GT_OK) {
        delete table;
        return st;
    }
    *out_table = table;
    return GT_OK;
}

// characterize_points (src/execute_gpu.rs:189-229, 1286-1319; macros lib.rs:641-683).
// points: (n, ncols) with [frame,] y, x [, r].
int oracle_characterize_points(const gt_params* p, const float* frames, int64_t T, int32_t H, int32_t W,
                               const float* points, int64_t n, int32_t has_frames, int32_t has_r,
                               int32_t nthreads, void** out_table) {
    (void)nthreads;
    if (T <= 0) return GT_ERR_EMPTY_ITERATOR;
    Derived d = derive(*p, H, W);
    const size_t npix = (size_t)H * W;
    const int ncols = 2 + (has_frames ? 1 : 0) + (has_r ? 1 : 0);
    const int c0 = has_frames ? 1 : 0;
    // group points per frame exactly as FrameSubsetter does
    std::vector<std::pair<size_t, std::vector<Row>>> groups;
    auto mkrow = [&](int64_t i) {
        Row r;
        r.x = points[i * ncols + c0];
        r.y = points[i * ncols + c0 + 1];
        r.r = has_r ? points[i * ncols + c0 + 2] : 0.0f;
        return r;
    };
    if (has_frames) {
        float cur = 0.0f;
        std::vector<Row> out;
        int64_t idx = 0;
        while (true) {
            if (idx < n) {
                float f = points[idx * ncols];
                if (f > cur) {
                    groups.push_back({(size_t)cur, out});
                    out.clear();
                    cur = f;
                    continue;
                }
                if (f < cur) return GT_ERR_NON_SORTED_CHARACTERIZATION;
                out.push_back(mkrow(idx));
                idx++;
            } else {
                if (!out.empty()) groups.push_back({(size_t)cur, out});
                break;
            }
        }
    } else {
        std::vector<Row> all;
        for (int64_t i = 0; i < n; i++) all.push_back(mkrow(i));
        for (int64_t t = 0; t < T; t++) groups.push_back({(size_t)t, all});
    }
    if (groups.empty()) return GT_ERR_EMPTY_ITERATOR;
    std::vector<std::vector<Row>> per_frame(groups.size());
    std::vector<int64_t> fnums(groups.size());
    std::vector<float> frames_sel(groups.size() * npix);
    for (size_t g = 0; g < groups.size(); g++) {
        size_t f = groups[g].first;
        if ((int64_t)f >= T) return GT_ERR_FRAME_OUT_OF_BOUNDS;
        fnums[g] = (int64_t)f;
        std::memcpy(frames_sel.data() + g * npix, frames + f * npix, npix * sizeof(float));
        std::vector<float> tg, tb, proc(npix);
        preprocess(d, p->truncate_preprocessed != 0, frames + f * npix, tg, tb, proc.data());
        per_frame[g] = groups[g].second;
        for (auto& row : per_frame[g]) characterize(d, proc.data(), frames + f * npix, row, true);
    }
    gt_params q = *p;
    q.filter_close = 0;
    q.characterize = 1;
    OracleTable* table = new OracleTable();
    int st = post_process_all(q, d, frames_sel.data(), per_frame, fnums.data(), nullptr, 0, *table);
    if (st != GT_OK) {
        delete table;
        return st;
    }
    *out_table = table;
    return GT_OK;
}

int64_t oracle_table_nrows(void* t) { return ((OracleTable*)t)->nrows; }
void oracle_table_get(void* t, double* dst) {
    auto* tb = (OracleTable*)t;
    std::memcpy(dst, tb->data.data(), tb->data.size() * sizeof(double));
}
void oracle_table_free(void* t) { delete (OracleTable*)t; }

// link_rust -> linker_all (src/linking.rs:818-831).
int oracle_link(const float* fyx, int64_t n, float search_range, uint32_t memory, int64_t* out) {
    Subsetter sub{fyx, n};
    Linker linker(search_range, memory);
    std::vector<Pos> pts;
    size_t frame;
    int64_t o = 0;
    while (true) {
        int r = sub.next(frame, pts);
        if (r == 0) break;
        if (r < 0) return GT_ERR_NON_SORTED_CHARACTERIZATION;
        try {
            auto ids = linker.advance(pts);
            for (auto id : ids) out[o++] = (int64_t)id;
        } catch (TooDense&) {
            return GT_ERR_TOO_DENSE_TO_LINK;
        }
    }
    return GT_OK;
}

// connect_all (src/linking.rs:960-1020) with sync_iterators (:914-958).
int oracle_connect(const float* a1, int64_t n1, const float* a2, int64_t n2, float search_range, int64_t* out1,
                   int64_t* out2) {
    Subsetter it1{a1, n1}, it2{a2, n2};
    Linker linker(search_range, 0);
    std::vector<int64_t> r1, r2;
    struct Item { size_t frame; std::vector<Pos> pts; };
    auto fill = [&](const Item& it, std::vector<int64_t>& res) {
        for (size_t i = 0; i < it.pts.size(); i++) res.push_back((int64_t)linker.part_idx++);
    };
    auto nextof = [](Subsetter& s, Item& it) { return s.next(it.frame, it.pts); };
    try {
        while (true) {
            Item f1, f2;
            int s1 = nextof(it1, f1);
            int s2 = nextof(it2, f2);
            if (s1 < 0 || s2 < 0) return GT_ERR_NON_SORTED_CHARACTERIZATION;
            if (s1 == 1 && s2 == 1) {
                bool have_both = false;
                Item b1, b2;
                if (f1.frame == f2.frame) {
                    have_both = true; b1 = f1; b2 = f2;
                } else {
                    // sync_iterators, iteratively
                    bool left = f1.frame > f2.frame;   // to_hit side
                    Item to_hit = left ? f1 : f2;
                    if (left) fill(f2, r2); else fill(f1, r1);
                    while (true) {
                        Item nx;
                        int sn = left ? nextof(it2, nx) : nextof(it1, nx);
                        if (sn < 0) return GT_ERR_NON_SORTED_CHARACTERIZATION;
                        if (sn == 0) {
                            if (left) fill(to_hit, r1); else fill(to_hit, r2);
                            break;
                        }
                        if (to_hit.frame > nx.frame) {
                            if (left) fill(nx, r2); else fill(nx, r1);
                            continue;
                        } else if (to_hit.frame == nx.frame) {
                            have_both = true;
                            if (left) { b1 = to_hit; b2 = nx; } else { b1 = nx; b2 = to_hit; }
                            break;
                        } else {
                            if (left) fill(nx, r2); else fill(nx, r1);
                            if (left) fill(to_hit, r1); else fill(to_hit, r2);
                            to_hit = nx;
                            left = !left;
                            continue;
                        }
                    }
                }
                if (have_both) {
                    auto res = linker.connect(b1.pts, b2.pts);
                    for (auto v : res.first) r1.push_back((int64_t)v);
                    for (auto v : res.second) r2.push_back((int64_t)v);
                }
            } else if (s1 == 1 && s2 == 0) {
                fill(f1, r1);
            } else if (s1 == 0 && s2 == 1) {
                fill(f2, r2);
            } else {
                break;
            }
        }
    } catch (TooDense&) {
        return GT_ERR_TOO_DENSE_TO_LINK;
    }
    if ((int64_t)r1.size() != n1 || (int64_t)r2.size() != n2) return GT_ERR_INTERNAL;
    std::memcpy(out1, r1.data(), n1 * sizeof(int64_t));
    std::memcpy(out2, r2.data(), n2 * sizeof(int64_t));
    return GT_OK;
}

}  // extern "C"
