// gt_link.cu — trackpy-style optimal subnet linking on the GPU.
//
// Replaces Linker / link / recurse / recurse2 (src/linking.rs:345-816) and
// the kd-tree neighbour search (within_radius_rd2, src/linking.rs:211-247).
//
//   sort_groups_kernel   points of every frame group sorted by row (the
//                        grid-free neighbour index: a binary search on rows
//                        plus the exact within_radius_rd2 predicate).
//   count/fill_lists     for every point and every lag k = 1..memory+1, the
//                        forward (dests in group+k) and backward (sources in
//                        group-k) neighbour lists in ascending point order; all
//                        frame pairs in parallel.
//   link_video_kernel    one CTA per video walks its frames in order (the
//                        linker's only true sequential dependency) doing each
//                        frame's work in parallel: memory merge, subnet
//                        detection by union-find, the reference's DFS order
//                        per subnet, the exact branch-and-bound per subnet
//                        (one thread each, same float operation sequence),
//                        new ids in destination order, memory ring and
//                        duration bookkeeping.
#include "gt_kernels.h"

namespace gt {

constexpr int kLinkThreads = 1024;
constexpr int kSortSmem = 4096;
constexpr long long kSubnetBudget = 1ll << 28;
constexpr int kLagRegs = 4;     // backward-list offsets of up to 4 lags held in registers
constexpr int kEdgeRegs = 2;    // backward edges per lag gathered in registers before they are written
constexpr int kRingSmem = 64;   // memory ring bookkeeping in shared memory up to memory = 64
// A frame with at most LinkSmem<SF>::D detections and LinkSmem<SF>::S sources
// keeps its per-destination and per-source working arrays in shared memory;
// larger frames use the same arrays in the global scratch.  SF is the type of
// the per-source forward-list offsets: int32 when every offset of the lists
// fits (a larger working set in the same shared memory), int64 otherwise.
template <typename SF>
struct LinkSmem;
template <>
struct LinkSmem<int64_t> {
    static constexpr int D = 2048, S = 2560;
};
template <>
struct LinkSmem<int32_t> {
    static constexpr int D = 3840, S = 4608;
};
template <typename SF>
constexpr size_t link_smem_bytes() {
    return (size_t)(LinkSmem<SF>::D + 1) * 4 * 10 + (size_t)LinkSmem<SF>::S * (2 * sizeof(SF) + 4 + 1);
}
static_assert(((LinkSmem<int64_t>::D + 1) * 4 * 10) % 8 == 0, "source block stays 8-byte aligned");
static_assert(link_smem_bytes<int32_t>() + 4096 <= 227 * 1024, "the int32 working set fits with the static arrays");

// ------------------------------------------------------- point addressing
__device__ __forceinline__ int64_t gbase(const LinkInput& in, int g) {
    return in.slot_stride ? (int64_t)g * in.slot_stride : in.goff[g];
}
__device__ __forceinline__ int64_t gsize(const LinkInput& in, int g) {
    return in.slot_stride ? (int64_t)in.gcount[g] : in.goff[g + 1] - in.goff[g];
}
__device__ __forceinline__ int ggroup(const LinkInput& in, int64_t p) {
    return in.slot_stride ? (int)(p / in.slot_stride) : in.pgroup[p];
}
__device__ __forceinline__ float prow(const LinkInput& in, int64_t p) { return in.px[p * in.xy_stride]; }
__device__ __forceinline__ float pcol(const LinkInput& in, int64_t p) { return in.py[p * in.xy_stride]; }
// offset-array index of (point p, lag slot k) in 0..K
__device__ __forceinline__ int64_t lix(const LinkLists& L, int64_t p, int K, int k) {
    return (p - L.pbase) * K + k;
}

// ------------------------------------------------------------ group sorting
// Row bin of a row key (monotone in the row; NaN after every bin).
__device__ __forceinline__ int row_bin(float row, float bin_w) {
    if (row != row) return kLinkRowBins;
    const float t = floorf(__fdiv_rn(row, bin_w));
    if (!(t >= 0.0f)) return 0;
    if (t >= (float)(kLinkRowBins - 1)) return kLinkRowBins - 1;
    return (int)t;
}

__global__ void __launch_bounds__(kLinkThreads)
sort_groups_kernel(LinkInput in, uint32_t* __restrict__ srt, uint64_t* __restrict__ scratch, size_t per_group,
                   int g0, int32_t* __restrict__ bins, float bin_w) {
    __shared__ uint64_t sk[kSortSmem];
    const int g = g0 + blockIdx.x;
    const int64_t a = gbase(in, g), n = gsize(in, g);
    int32_t* const off = bins ? bins + (size_t)g * (kLinkRowBins + 1) : nullptr;
    if (n == 0) {
        if (off)
            for (int b = threadIdx.x; b <= kLinkRowBins; b += blockDim.x) off[b] = 0;
        return;
    }
    int np2 = 1;
    while (np2 < n) np2 <<= 1;
    uint64_t* keys = (np2 <= kSortSmem) ? sk : scratch + (size_t)blockIdx.x * per_group;
    for (int i = threadIdx.x; i < np2; i += blockDim.x)
        keys[i] = (i < n) ? (((uint64_t)float_order_key(prow(in, a + i)) << 32) | (uint64_t)i) : ~0ull;
    __syncthreads();
    block_sort_u64(keys, np2);
    for (int i = threadIdx.x; i < n; i += blockDim.x) srt[a + i] = (uint32_t)(keys[i] & 0xFFFFFFFFull);
    if (off) {
        // off[b] = first sorted position whose bin is >= b: position i writes
        // the bins in (bin(i - 1), bin(i)], position n those up to the end
        auto bin_at = [&](int64_t i) -> int {
            if (i >= n) return kLinkRowBins;
            return row_bin(float_from_order_key((uint32_t)(keys[i] >> 32)), bin_w);
        };
        for (int64_t i = threadIdx.x; i <= n; i += blockDim.x) {
            const int prev = i == 0 ? -1 : bin_at(i - 1), cur = bin_at(i);
            for (int b = prev + 1; b <= cur; b++) off[b] = (int32_t)i;
        }
    }
}

// Sorted positions [p0, p1) of group t that hold every row in [lo, hi]: the
// first position whose row key is >= klo and the first > khi, or, with the
// row-bin index, the positions of the bins that lo and hi fall in (a few
// more rows, which the exact distance test rejects).
__device__ __forceinline__ void row_range(const LinkInput& in, const LinkLists& L, int t, float lo, float hi,
                                          int64_t* p0, int64_t* p1) {
    if (L.bins) {
        const int32_t* off = L.bins + (size_t)t * (kLinkRowBins + 1);
        *p0 = off[row_bin(lo, L.bin_w)];
        *p1 = off[row_bin(hi, L.bin_w) + 1];
        return;
    }
    const uint32_t* srt = L.srt;
    const int64_t a = gbase(in, t), n = gsize(in, t);
    const uint32_t klo = float_order_key(lo), khi = float_order_key(hi);
    int64_t x = 0, y = n;
    while (x < y) {
        int64_t m = (x + y) >> 1;
        if (float_order_key(prow(in, a + srt[a + m])) < klo) x = m + 1; else y = m;
    }
    *p0 = x;
    y = n;
    while (x < y) {
        int64_t m = (x + y) >> 1;
        if (float_order_key(prow(in, a + srt[a + m])) <= khi) x = m + 1; else y = m;
    }
    *p1 = x;
}

__device__ __forceinline__ void search_bounds(float q, float R, float* lo, float* hi) {
    // conservative superset of the rows within_rd2 can accept
    float delta = __fmul_rn(fmaxf(fabsf(q), R), 1.0f / 1048576.0f) + 1e-30f;
    *lo = __fsub_rn(__fsub_rn(q, R), delta);
    *hi = __fadd_rn(__fadd_rn(q, R), delta);
}

__device__ __forceinline__ void group_video_range(const LinkInput& in, int h, int* vb, int* ve) {
    int x = 0, y = in.nvideos;  // last video with vgrp[v] <= h
    while (y - x > 1) {
        int m = (x + y) >> 1;
        if (in.vgrp[m] <= h) x = m; else y = m;
    }
    *vb = in.vgrp[x];
    *ve = in.vgrp[x + 1];
}

// mode 0: count, mode 1: fill (and sort ascending); points [p0, p1), offsets
// relative to L.pbase.  A fill whose list would pass the end of its buffer
// (f_cap / b_cap) writes nothing and raises kFlagListOverflow.
template <int kMode>
__global__ void lists_kernel(LinkInput in, LinkLists L, int64_t* f_cnt, int64_t* b_cnt, int64_t p0, int64_t p1,
                             uint32_t* flags) {
    const int64_t p = p0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= p1) return;
    const int K = in.memory + 1;
    const int h = ggroup(in, p);
    if (in.slot_stride && p - gbase(in, h) >= gsize(in, h)) return;  // empty slot
    int vb, ve;
    group_video_range(in, h, &vb, &ve);
    const int ready = in.groups_ready > 0 ? in.groups_ready : in.ngroups;
    const float qx = prow(in, p), qy = pcol(in, p);
    const float R = in.radius;
    float lo, hi;
    search_bounds(qx, R, &lo, &hi);
    const bool qnan = (qx != qx) || (qy != qy);
    for (int k = 1; k <= K; k++) {
        // forward: p is a source, dests in group h + k
        int t = h + k;
        int64_t cnt = 0;
        bool skip = false;
        if (kMode && t < ve && t < ready && L.f_cap >= 0 && L.f_off[lix(L, p, K, k)] > L.f_cap) {
            atomicOr(flags, kFlagListOverflow);
            skip = true;
        }
        if (t < ve && t < ready && !qnan && !skip) {
            int64_t s0, s1;
            row_range(in, L, t, lo, hi, &s0, &s1);
            const int64_t a = gbase(in, t);
            int32_t* out = kMode ? L.f_pts + L.f_off[lix(L, p, K, k - 1)] : nullptr;
            for (int64_t m = s0; m < s1; m++) {
                int64_t d = a + L.srt[a + m];
                float dist;
                if (within_rd2(prow(in, d), pcol(in, d), qx, qy, R, &dist)) {
                    if (kMode) out[cnt] = (int32_t)(d - a);
                    cnt++;
                }
            }
            if (kMode) {  // ascending destination order
                for (int64_t i = 1; i < cnt; i++) {
                    int32_t v = out[i];
                    int64_t j = i - 1;
                    while (j >= 0 && out[j] > v) { out[j + 1] = out[j]; j--; }
                    out[j + 1] = v;
                }
            }
        }
        if (!kMode) f_cnt[lix(L, p, K, k - 1)] = cnt;
        // backward: p is a dest, sources in group h - k
        t = h - k;
        cnt = 0;
        skip = false;
        if (kMode && t >= vb && L.b_cap >= 0 && L.b_off[lix(L, p, K, k)] > L.b_cap) {
            atomicOr(flags, kFlagListOverflow);
            skip = true;
        }
        if (t >= vb && !qnan && !skip) {
            int64_t s0, s1;
            row_range(in, L, t, lo, hi, &s0, &s1);
            const int64_t a = gbase(in, t);
            int32_t* out = kMode ? L.b_pts + L.b_off[lix(L, p, K, k - 1)] : nullptr;
            float* outd = kMode ? L.b_dist + L.b_off[lix(L, p, K, k - 1)] : nullptr;
            for (int64_t m = s0; m < s1; m++) {
                int64_t s = a + L.srt[a + m];
                float dist;
                if (within_rd2(qx, qy, prow(in, s), pcol(in, s), R, &dist)) {
                    if (kMode) {
                        out[cnt] = (int32_t)(s - a);
                        outd[cnt] = dist;
                    }
                    cnt++;
                }
            }
            if (kMode) {  // ascending source order
                for (int64_t i = 1; i < cnt; i++) {
                    int32_t v = out[i];
                    float vd = outd[i];
                    int64_t j = i - 1;
                    while (j >= 0 && out[j] > v) { out[j + 1] = out[j]; outd[j + 1] = outd[j]; j--; }
                    out[j + 1] = v;
                    outd[j + 1] = vd;
                }
            }
        }
        if (!kMode) b_cnt[lix(L, p, K, k - 1)] = cnt;
    }
}

// ---------------------------------------------------------- scratch layout
// dblk: 10 per-destination int32 arrays of G + 1 entries (d_off, d_end,
// out_src, parent, comp_nd, comp_ns, comp_off, comp_soff, roots, tmp);
// sblk: per-source sf0, sf1 (int64), src_pt (int32), srcUsed (u8), Smax each.
struct Lay {
    size_t start, idstamp, firstpos, srcidx, srcstamp, ring_pt, ring_n, ringpre, dblk, sblk, e_src, e_dist, pathD,
        pathS, srcLocal, vis_d, vis_s, stack, r2a, r2b, r2c, r2used, total;
};

__host__ __device__ inline size_t al(size_t x) { return (x + 15) & ~(size_t)15; }

__host__ __device__ inline Lay make_lay(int64_t G, int64_t E, int64_t NP, int64_t M) {
    Lay l;
    const int64_t Smax = G * (M + 1);
    size_t o = 0;
    l.start = o; o = al(o + 8 * NP);
    l.idstamp = o; o = al(o + 4 * NP);
    l.firstpos = o; o = al(o + 8 * NP);
    l.srcidx = o; o = al(o + 4 * NP);
    l.srcstamp = o; o = al(o + 4 * NP);
    l.ring_pt = o; o = al(o + 4 * (M * G + 1));
    l.ring_n = o; o = al(o + 4 * (M + 1));
    l.ringpre = o; o = al(o + 4 * (M + 2));
    l.dblk = o; o = al(o + 4 * 10 * (G + 1));
    l.sblk = o; o = al(o + (8 + 8 + 4 + 1) * Smax);
    l.e_src = o; o = al(o + 4 * (E + 1));
    l.e_dist = o; o = al(o + 4 * (E + 1));
    l.pathD = o; o = al(o + 4 * G);
    l.pathS = o; o = al(o + 4 * Smax);
    l.srcLocal = o; o = al(o + 4 * Smax);
    l.vis_d = o; o = al(o + 4 * G);
    l.vis_s = o; o = al(o + 4 * Smax);
    l.stack = o; o = al(o + 8 * (G + Smax));
    l.r2a = o; o = al(o + 4 * G);
    l.r2b = o; o = al(o + 4 * G);
    l.r2c = o; o = al(o + 4 * G);
    l.r2used = o; o = al(o + Smax);
    l.total = o;
    return l;
}

size_t link_scratch_bytes(int32_t max_group, int64_t max_edges, int64_t npoints_video, int32_t memory) {
    return make_lay(max_group, max_edges, npoints_video, memory).total;
}

void link_scratch_point_arrays(int32_t max_group, int64_t max_edges, int64_t npoints_video, int32_t memory,
                               size_t* idstamp, size_t* srcstamp, size_t* firstpos) {
    const Lay l = make_lay(max_group, max_edges, npoints_video, memory);
    *idstamp = l.idstamp;
    *srcstamp = l.srcstamp;
    *firstpos = l.firstpos;
}

// union-find over the destinations of one frame; roots are minimal indices
__device__ __forceinline__ int uf_find(volatile int* parent, int x) {
    while (true) {
        int p = parent[x];
        if (p == x) return x;
        int gp = parent[p];
        if (gp != p) parent[x] = gp;
        x = p;
    }
}
__device__ __forceinline__ void uf_union(volatile int* parent, int a, int b) {
    while (true) {
        a = uf_find(parent, a);
        b = uf_find(parent, b);
        if (a == b) return;
        if (a > b) { int t = a; a = b; b = t; }
        int old = atomicCAS((int*)&parent[b], b, a);
        if (old == b) return;
    }
}

template <typename SF>
__global__ void __launch_bounds__(kLinkThreads)
link_video_kernel(LinkInput in, LinkLists L, LinkScratch S, LinkOutput out, LinkWindow W) {
    constexpr int kLinkSmemD = LinkSmem<SF>::D, kLinkSmemS = LinkSmem<SF>::S;
    __shared__ int wsum[33];
    __shared__ long long wsum64[33];
    __shared__ int sh_ring_n[kRingSmem + 1], sh_ringpre[kRingSmem + 2];
    __shared__ long long sh_counter, sh_frame, sh_load;
    __shared__ int sh_prevg, sh_head, sh_nroots, sh_ringtot;
    const int v = blockIdx.x;
    const int gb = in.vgrp[v], ge = in.vgrp[v + 1];
    const int g_lo = (W.g0 < 0) ? gb : W.g0, g_hi = (W.g0 < 0) ? ge : W.g1;
    if (out.flags[v] & kLinkStopFlags) return;  // an earlier window stopped this video
    const int64_t P0 = gbase(in, gb);
    const int64_t NP = in.slot_stride ? (int64_t)(ge - gb) * in.slot_stride : in.goff[ge] - P0;
    const int M = in.memory, K = M + 1;
    const int G = S.max_group;
    const Lay lay = make_lay(G, S.max_edges, S.max_points, M);
    uint8_t* base = S.base + (size_t)v * S.bytes_per_video;
    int64_t* start = (int64_t*)(base + lay.start);
    int32_t* idstamp = (int32_t*)(base + lay.idstamp);
    unsigned long long* firstpos = (unsigned long long*)(base + lay.firstpos);
    int32_t* srcidx = (int32_t*)(base + lay.srcidx);
    int32_t* srcstamp = (int32_t*)(base + lay.srcstamp);
    int32_t* ring_pt = (int32_t*)(base + lay.ring_pt);
    int32_t* ring_n = (int32_t*)(base + lay.ring_n);
    int32_t* ringpre = (int32_t*)(base + lay.ringpre);
    int32_t* const g_dblk = (int32_t*)(base + lay.dblk);
    uint8_t* const g_sblk = base + lay.sblk;
    int32_t* e_src = (int32_t*)(base + lay.e_src);
    float* e_dist = (float*)(base + lay.e_dist);
    int32_t* pathD = (int32_t*)(base + lay.pathD);
    int32_t* pathS = (int32_t*)(base + lay.pathS);
    int32_t* srcLocal = (int32_t*)(base + lay.srcLocal);
    int32_t* vis_d = (int32_t*)(base + lay.vis_d);
    int32_t* vis_s = (int32_t*)(base + lay.vis_s);
    int2* stack = (int2*)(base + lay.stack);
    int32_t* r2opt = (int32_t*)(base + lay.r2a);
    int32_t* r2cho = (int32_t*)(base + lay.r2b);
    int32_t* r2best = (int32_t*)(base + lay.r2c);
    uint8_t* r2used = base + lay.r2used;
    int64_t* dur = out.dur + P0;
    int64_t* ids = out.ids;
    const int Smax = G * K;
    const float R = in.radius;
    const float R2 = __fmul_rn(R, R);
    const int tid = threadIdx.x, nth = blockDim.x;
    // shared-memory copies of the per-frame blocks (same layout as dblk / sblk)
    extern __shared__ int64_t lsm[];
    int32_t* const s_dblk = (int32_t*)lsm;                             // 10 x (kLinkSmemD + 1)
    uint8_t* const s_sblk = (uint8_t*)(s_dblk + 10 * (kLinkSmemD + 1));  // kLinkSmemS sources

    // ring sizes and their prefix live in shared memory for memory <= kRingSmem
    const bool ring_smem = M <= kRingSmem;
    int32_t* ringN = ring_smem ? sh_ring_n : ring_n;
    int32_t* ringP = ring_smem ? sh_ringpre : ringpre;
    if (W.first) {
        if (W.init_points) {
            for (int64_t i = tid; i < NP; i += nth) {
                idstamp[i] = -1;
                srcstamp[i] = -1;
                firstpos[i] = 0ull;
            }
        }
        for (int i = tid; i < Smax; i += nth) vis_s[i] = -1;
        for (int i = tid; i < G; i += nth) vis_d[i] = -1;
        for (int i = tid; i <= M; i += nth) ringN[i] = 0;
        if (tid == 0) {
            sh_counter = 0;
            sh_frame = 0;
            sh_prevg = -1;
            sh_head = 0;
        }
    } else {
        if (ring_smem)
            for (int i = tid; i <= M; i += nth) ringN[i] = ring_n[i];
    }
    if (!W.first && tid == 0) {
        const LinkState st = W.state[v];
        sh_counter = st.counter;
        sh_frame = st.frame;
        sh_prevg = st.prevg;
        sh_head = st.head;
    }
    __syncthreads();

    for (int g = g_lo; g < g_hi; g++) {
        const int step = g - gb;
        if (in.reset[g]) {
            // Linker::reset (src/linking.rs:401-403, src/execute_gpu.rs:792-798)
            if (tid == 0) {
                sh_counter = 0;
                sh_frame = 0;
                sh_prevg = -1;
                sh_head = 0;
            }
            for (int i = tid; i <= M; i += nth) ringN[i] = 0;
            __syncthreads();
        }
        const int64_t a = gbase(in, g);
        const int D = (int)gsize(in, g);
        const int prevg = sh_prevg;
        const int S0 = (prevg == g - 1 && prevg >= gb) ? (int)gsize(in, g - 1) : 0;
        const int64_t pa = (S0 > 0) ? gbase(in, g - 1) : 0;
        // working arrays of this frame: shared memory when they fit
        int ring_all = 0;
        if (ring_smem)
            for (int q = 0; q < M; q++) ring_all += ringN[q];
        const bool fast = ring_smem && D <= kLinkSmemD && S0 + ring_all <= kLinkSmemS;
        const int dstr = fast ? kLinkSmemD + 1 : G + 1;
        const int sstr = fast ? kLinkSmemS : Smax;
        int32_t* const dblk = fast ? s_dblk : g_dblk;
        uint8_t* const sblk = fast ? s_sblk : g_sblk;
        SF* const sf0 = (SF*)sblk;
        SF* const sf1 = sf0 + sstr;
        int32_t* const src_pt = (int32_t*)(sf1 + sstr);
        uint8_t* const srcUsed = (uint8_t*)(src_pt + sstr);
        int32_t* const d_off = dblk;
        int32_t* const d_end = dblk + dstr;
        int32_t* const out_src = dblk + 2 * dstr;
        volatile int* const parent = (volatile int*)(dblk + 3 * dstr);
        int32_t* const comp_nd = dblk + 4 * dstr;
        int32_t* const comp_ns = dblk + 5 * dstr;
        int32_t* const comp_off = dblk + 6 * dstr;
        int32_t* const comp_soff = dblk + 7 * dstr;
        int32_t* const roots = dblk + 8 * dstr;
        int32_t* const tmp = dblk + 9 * dstr;
        // ---- P1: sources = previous frame + memory entries not already present
        for (int i0 = 2 * tid; i0 < S0; i0 += 2 * nth) {
            const int n2 = min(2, S0 - i0);
            int64_t idv[2];
#pragma unroll
            for (int u = 0; u < 2; u++)
                if (u < n2) idv[u] = ids[pa + i0 + u];
#pragma unroll
            for (int u = 0; u < 2; u++) {
                if (u >= n2) break;
                const int i = i0 + u;
                const int64_t lp = pa + i - P0;
                idstamp[idv[u]] = step;
                src_pt[i] = (int32_t)lp;
                srcidx[lp] = i;
                srcstamp[lp] = step;
            }
        }
        if (tid == 0) {
            int tot = 0;
            for (int q = 0; q < M; q++) {
                ringP[q] = tot;
                tot += ringN[(sh_head + q) % M];
            }
            ringP[M] = tot;
            sh_ringtot = tot;
        }
        __syncthreads();
        const int RT = (M > 0) ? sh_ringtot : 0;
        // ring entries in ring order: position r -> (slot q, entry e)
        auto ring_lp = [&](int r) -> int32_t {
            int q = 0;
            while (ringP[q + 1] <= r) q++;
            const int slot = (sh_head + q) % M;
            return ring_pt[slot * G + (r - ringP[q])];
        };
        for (int r = tid; r < RT; r += nth) {
            const int64_t id = ids[P0 + ring_lp(r)];
            if (idstamp[id] != step)
                atomicMax(&firstpos[id], ((unsigned long long)(uint32_t)step << 32) | (0xFFFFFFFFull - (uint32_t)r));
        }
        __syncthreads();
        int kept_tot = 0;
        for (int base0 = 0; base0 < RT; base0 += 2 * nth) {
            int keep[2] = {0, 0};
            int32_t lpv[2] = {0, 0};
#pragma unroll
            for (int u = 0; u < 2; u++) {
                const int r = base0 + 2 * tid + u;
                if (r < RT) {
                    lpv[u] = ring_lp(r);
                    const int64_t id = ids[P0 + lpv[u]];
                    keep[u] = (idstamp[id] != step) &&
                              firstpos[id] ==
                                  (((unsigned long long)(uint32_t)step << 32) | (0xFFFFFFFFull - (uint32_t)r));
                }
            }
            int tot;
            const int pos = block_excl_scan(keep[0] + keep[1], &tot, wsum);
#pragma unroll
            for (int u = 0; u < 2; u++) {
                if (!keep[u]) continue;
                const int si = S0 + kept_tot + pos + (u ? keep[0] : 0);
                src_pt[si] = lpv[u];
                srcidx[lpv[u]] = si;
                srcstamp[lpv[u]] = step;
            }
            kept_tot += tot;
        }
        const int Sn = S0 + kept_tot;
        __syncthreads();
        // ---- P2: destination -> source lists (ascending source index).  The
        // edges of destination j go to its own range of the frame's backward
        // lists, whose size bounds the kept edges: [d_off[j], d_end[j]).
        const int64_t fb = L.b_off[lix(L, a, K, 0)];
        if (L.b_off[lix(L, a + D, K, 0)] - fb > S.max_edges) {
            if (tid == 0) atomicOr(out.flags + v, in.slot_stride ? kFlagEdgeOverflow : kFlagScratch);
            break;
        }
        for (int j = tid; j < D; j += nth) {
            const int64_t pt = a + j;
            const int64_t lb = lix(L, pt, K, 0);
            int64_t bo[kLagRegs + 1];
            const bool regs = K <= kLagRegs;
#pragma unroll
            for (int i = 0; i <= kLagRegs; i++) bo[i] = (regs && i <= K) ? L.b_off[lb + i] : 0;
            const int64_t b0 = regs ? bo[0] : L.b_off[lb];
            int w = (int)(b0 - fb);
            d_off[j] = w;
            // When every lag has at most kEdgeRegs edges, all list reads are
            // issued before any write (the writes could alias them for the
            // compiler), so their latencies overlap: three dependent levels
            // instead of one chain per edge.  Same edges, same order.
            bool fits = regs;
#pragma unroll
            for (int k = 1; k <= kLagRegs; k++)
                if (k <= K && bo[k] - bo[k - 1] > kEdgeRegs) fits = false;
            if (fits) {
                int32_t ep[kLagRegs][kEdgeRegs], es[kLagRegs][kEdgeRegs];
                float ed[kLagRegs][kEdgeRegs];
#pragma unroll
                for (int k = 1; k <= kLagRegs; k++) {
                    const bool lag_on = k <= K && (k == 1 ? S0 > 0 : g - k >= gb);
#pragma unroll
                    for (int u = 0; u < kEdgeRegs; u++) {
                        const int64_t e = bo[k - 1] + u;
                        const bool on = lag_on && e < bo[k];
                        ep[k - 1][u] = on ? L.b_pts[e] : -1;
                        ed[k - 1][u] = on ? L.b_dist[e] : 0.0f;
                    }
                }
                // lags 2..K: the source's index in this step's source list,
                // or -1 when it is not a source of this step
#pragma unroll
                for (int k = 2; k <= kLagRegs; k++) {
                    const int64_t ta = (k <= K && g - k >= gb) ? gbase(in, g - k) - P0 : 0;
#pragma unroll
                    for (int u = 0; u < kEdgeRegs; u++) {
                        es[k - 1][u] = -1;
                        if (ep[k - 1][u] >= 0) {
                            const int64_t lp = ta + ep[k - 1][u];
                            const int32_t stamp = srcstamp[lp], idx = srcidx[lp];
                            es[k - 1][u] = (stamp == step) ? idx : -1;
                        }
                    }
                }
                // lag 1 (index within group g-1 == source index), then lags K..2
#pragma unroll
                for (int u = 0; u < kEdgeRegs; u++)
                    if (ep[0][u] >= 0) {
                        e_src[w] = ep[0][u];
                        e_dist[w] = ed[0][u];
                        w++;
                    }
#pragma unroll
                for (int k = kLagRegs; k >= 2; k--)
#pragma unroll
                    for (int u = 0; u < kEdgeRegs; u++)
                        if (es[k - 1][u] >= 0) {
                            e_src[w] = es[k - 1][u];
                            e_dist[w] = ed[k - 1][u];
                            w++;
                        }
                d_end[j] = w;
                parent[j] = j;
                out_src[j] = -2;
                continue;
            }
            if (S0 > 0) {
                const int64_t o1 = regs ? bo[1] : L.b_off[lb + 1];
                for (int64_t e = b0; e < o1; e++) {
                    e_src[w] = L.b_pts[e];  // index within group g-1 == source index
                    e_dist[w] = L.b_dist[e];
                    w++;
                }
            }
            // lags K..2: only sources that are in this step's source list
            auto lag = [&](int k, int64_t o0, int64_t o1) {
                const int t = g - k;
                if (t < gb) return;
                const int64_t ta = gbase(in, t) - P0;
                for (int64_t e = o0; e < o1; e++) {
                    const int64_t lp = ta + L.b_pts[e];
                    if (srcstamp[lp] == step) {
                        e_src[w] = srcidx[lp];
                        e_dist[w] = L.b_dist[e];
                        w++;
                    }
                }
            };
            if (regs) {
#pragma unroll
                for (int k = kLagRegs; k >= 2; k--)
                    if (k <= K) lag(k, bo[k - 1], bo[k]);
            } else {
                for (int k = K; k >= 2; k--) lag(k, L.b_off[lb + k - 1], L.b_off[lb + k]);
            }
            d_end[j] = w;
            parent[j] = j;
            out_src[j] = -2;
        }
        // ---- P3: trivial links and subnets (connected components)
        // forward range of every source toward this frame, read once
        for (int s = tid; s < Sn; s += nth) {
            const int64_t pt = P0 + src_pt[s];
            const int64_t l = lix(L, pt, K, g - ggroup(in, pt) - 1);
            const int64_t f0 = L.f_off[l], f1 = L.f_off[l + 1];
            sf0[s] = (SF)f0;
            sf1[s] = (SF)f1;
            srcUsed[s] = 0;
        }
        __syncthreads();
        for (int s = tid; s < Sn; s += nth) {
            const int64_t f0 = sf0[s], f1 = sf1[s];
            if (f1 - f0 >= 2) {
                const int j0 = L.f_pts[f0];
                for (int64_t e = f0 + 1; e < f1; e++) uf_union(parent, j0, L.f_pts[e]);
            }
        }
        for (int j = tid; j < D; j += nth) {
            const int e0 = d_off[j], deg = d_end[j] - e0;
            if (deg == 0) {
                out_src[j] = -1;
            } else if (deg == 1) {
                const int s = e_src[e0];
                if (sf1[s] - sf0[s] == 1) out_src[j] = s;
            }
        }
        __syncthreads();
        for (int j = tid; j < D; j += nth) {
            tmp[j] = uf_find(parent, j);
            comp_nd[j] = 0;
            comp_ns[j] = 0;
        }
        __syncthreads();
        for (int j = tid; j < D; j += nth)
            if (out_src[j] == -2) atomicAdd(&comp_nd[tmp[j]], 1);
        for (int s = tid; s < Sn; s += nth) {
            const int64_t f0 = sf0[s];
            if (sf1[s] > f0) {
                const int j0 = L.f_pts[f0];
                if (out_src[j0] == -2) atomicAdd(&comp_ns[tmp[j0]], 1);
            }
        }
        __syncthreads();
        {
            // one 64-bit scan of (roots, destinations) and one of sources, two
            // destinations per thread in destination order
            long long acc_rd = 0;
            int offs = 0;
            for (int base0 = 0; base0 < D; base0 += 2 * nth) {
                int isroot[2], nd[2], ns[2];
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const int j = base0 + 2 * tid + u;
                    isroot[u] = (j < D && out_src[j] == -2 && tmp[j] == j) ? 1 : 0;
                    nd[u] = isroot[u] ? comp_nd[j] : 0;
                    ns[u] = isroot[u] ? comp_ns[j] : 0;
                }
                const long long rd0 = (long long)isroot[0] + ((long long)nd[0] << 32);
                const long long rd1 = (long long)isroot[1] + ((long long)nd[1] << 32);
                long long trd;
                int ts;
                const long long prd = block_excl_scan64(rd0 + rd1, &trd, wsum64);
                const int ps = block_excl_scan(ns[0] + ns[1], &ts, wsum);
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    if (!isroot[u]) continue;
                    const int j = base0 + 2 * tid + u;
                    const long long pr_ = acc_rd + prd + (u ? rd0 : 0);
                    roots[(int)(pr_ & 0xFFFFFFFFll)] = j;
                    comp_off[j] = (int)(pr_ >> 32);
                    comp_soff[j] = offs + ps + (u ? ns[0] : 0);
                }
                acc_rd += trd;
                offs += ts;
            }
            if (tid == 0) {
                sh_nroots = (int)(acc_rd & 0xFFFFFFFFll);
                sh_load = 0;
            }
        }
        __syncthreads();
        const int nroots = sh_nroots;
        // ---- P4: the reference's DFS order per subnet (recurse, linking.rs:595-621)
        for (int q = tid; q < nroots; q += nth) {
            const int r = roots[q];
            const int od = comp_off[r], os = comp_soff[r];
            int2* stk = stack + od + os;
            int nd = 0, ns = 0, sp = 0;
            vis_d[r] = step;
            pathD[od + nd++] = r;
            stk[sp++] = make_int2(r, 0);  // (node, next edge); dests tagged by >= 0 side bit below
            // side encoding: dest nodes stored as node, sources as -(node+1)
            while (sp > 0) {
                int2& top = stk[sp - 1];
                if (top.x >= 0) {  // destination: its sources in list order
                    const int j = top.x;
                    const int e0 = d_off[j], e1 = d_end[j];
                    bool pushed = false;
                    while (e0 + top.y < e1) {
                        int s = e_src[e0 + top.y];
                        top.y++;
                        if (vis_s[s] != step) {
                            vis_s[s] = step;
                            srcLocal[s] = ns;
                            pathS[os + ns++] = s;
                            stk[sp++] = make_int2(-(s + 1), 0);
                            pushed = true;
                            break;
                        }
                    }
                    if (!pushed) sp--;
                } else {  // source: its destinations in list order
                    const int s = -top.x - 1;
                    const int64_t f0 = sf0[s], f1 = sf1[s];
                    bool pushed = false;
                    while (f0 + top.y < f1) {
                        int j = L.f_pts[f0 + top.y];
                        top.y++;
                        if (vis_d[j] != step) {
                            vis_d[j] = step;
                            pathD[od + nd++] = j;
                            stk[sp++] = make_int2(j, 0);
                            pushed = true;
                            break;
                        }
                    }
                    if (!pushed) sp--;
                }
            }
            if (nd > 1) atomicAdd((unsigned long long*)&sh_load, (unsigned long long)((long long)nd * ns));
        }
        __syncthreads();
        if (sh_load > 5000) {
            // TooDenseToLink (src/linking.rs:677-682)
            if (tid == 0) atomicOr(out.flags + v, kFlagTooDense);
            break;
        }
        // ---- P5: branch and bound per subnet (recurse2, linking.rs:687-766)
        for (int q = tid; q < nroots; q += nth) {
            const int r = roots[q];
            const int od = comp_off[r], os = comp_soff[r];
            const int nd = comp_nd[r], ns = comp_ns[r];
            int* opt = r2opt + od;
            int* cho = r2cho + od;
            int* bst = r2best + od;
            uint8_t* used = r2used + os;
            for (int i = 0; i < ns; i++) used[i] = 0;
            float score = 0.0f, best = INFINITY;
            bool has_best = false;
            long long budget = 0;
            int level = 0;
            opt[0] = 0;
            bool over = false;
            while (true) {
                if (++budget > kSubnetBudget) { over = true; break; }
                const int j = pathD[od + level];
                const int e0 = d_off[j];
                const int deg = d_end[j] - e0;
                const int o = opt[level];
                bool ascend = false;
                if (o > deg) {
                    ascend = true;
                } else if (score > best) {
                    ascend = true;
                } else {
                    const bool is_null = (o == deg);
                    const float c = is_null ? R2 : e_dist[e0 + o];
                    score = __fadd_rn(score, c);
                    int ls = -1;
                    if (!is_null) {
                        ls = srcLocal[e_src[e0 + o]];
                        if (used[ls]) {
                            score = __fsub_rn(score, c);
                            opt[level] = o + 1;
                            continue;
                        }
                        used[ls] = 1;
                    }
                    cho[level] = ls;
                    if (level == nd - 1) {
                        if (score < best) {
                            best = score;
                            has_best = true;
                            for (int l = 0; l < nd; l++) bst[l] = cho[l];
                        }
                        if (!is_null) used[ls] = 0;
                        score = __fsub_rn(score, c);
                        opt[level] = o + 1;
                    } else {
                        level++;
                        opt[level] = 0;
                    }
                    continue;
                }
                if (ascend) {
                    level--;
                    if (level < 0) break;
                    const int jp = pathD[od + level];
                    const int ep = d_off[jp];
                    const int degp = d_end[jp] - ep;
                    const int op = opt[level];
                    const bool nullp = (op == degp);
                    const float cp = nullp ? R2 : e_dist[ep + op];
                    if (!nullp) used[cho[level]] = 0;
                    score = __fsub_rn(score, cp);
                    opt[level] = op + 1;
                }
            }
            if (over) atomicOr(out.flags + v, kFlagSubnetBudget);
            for (int l = 0; l < nd; l++) {
                int ch = has_best ? bst[l] : -1;
                out_src[pathD[od + l]] = (ch >= 0) ? pathS[os + ch] : -1;
            }
        }
        __syncthreads();
        if (out.flags[v] & kFlagSubnetBudget) break;
        // ---- P6: ids (new ones in destination order, src/linking.rs:788-798)
        {
            int newtot = 0;
            const long long counter = sh_counter;
            const long long frame = sh_frame;
            for (int base0 = 0; base0 < D; base0 += 2 * nth) {
                int osrc[2], isnew[2];
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const int j = base0 + 2 * tid + u;
                    osrc[u] = (j < D) ? out_src[j] : 0;
                    isnew[u] = (j < D && osrc[u] < 0) ? 1 : 0;
                }
                int tot;
                const int pos = block_excl_scan(isnew[0] + isnew[1], &tot, wsum);
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const int j = base0 + 2 * tid + u;
                    if (j >= D) break;
                    const int64_t pt = a + j;
                    if (isnew[u]) {
                        const long long id = counter + newtot + pos + (u ? isnew[0] : 0);
                        ids[pt] = id;
                        start[id] = frame;
                    } else {
                        const int s = osrc[u];
                        ids[pt] = ids[P0 + src_pt[s]];
                        srcUsed[s] = 1;
                    }
                }
                newtot += tot;
            }
            __syncthreads();
            if (tid == 0) sh_counter = counter + newtot;
        }
        // ---- P7: memory ring and durations (src/linking.rs:481-503)
        {
            const long long frame = sh_frame;
            if (M > 0) {
                const int hs = sh_head;
                const int nleave = ringN[hs];
                for (int e = tid; e < nleave; e += nth) {
                    int64_t id = ids[P0 + ring_pt[hs * G + e]];
                    dur[id] = (frame - start[id]) - M;
                }
                __syncthreads();
                int ut = 0;
                for (int base0 = 0; base0 < S0; base0 += 2 * nth) {
                    int un[2];
#pragma unroll
                    for (int u = 0; u < 2; u++) {
                        const int s = base0 + 2 * tid + u;
                        un[u] = (s < S0 && !srcUsed[s]) ? 1 : 0;
                    }
                    int tot;
                    const int pos = block_excl_scan(un[0] + un[1], &tot, wsum);
#pragma unroll
                    for (int u = 0; u < 2; u++)
                        if (un[u]) ring_pt[hs * G + ut + pos + (u ? un[0] : 0)] = src_pt[base0 + 2 * tid + u];
                    ut += tot;
                }
                if (tid == 0) {
                    ringN[hs] = ut;
                    sh_head = (hs + 1) % M;
                }
            } else {
                for (int s = tid; s < S0; s += nth) {
                    if (!srcUsed[s]) {
                        int64_t id = ids[P0 + src_pt[s]];
                        dur[id] = frame - start[id];
                    }
                }
            }
            __syncthreads();
            if (tid == 0) {
                sh_prevg = g;
                sh_frame = frame + 1;
            }
            __syncthreads();
        }
    }
    __syncthreads();
    if (!W.last) {
        if (ring_smem)
            for (int i = tid; i <= M; i += nth) ring_n[i] = ringN[i];
        if (tid == 0 && !(out.flags[v] & kLinkStopFlags)) {
            LinkState st;
            st.counter = sh_counter;
            st.frame = sh_frame;
            st.prevg = sh_prevg;
            st.head = sh_head;
            W.state[v] = st;
        }
        return;
    }
    // ---- Linker::finish (src/linking.rs:505-520)
    if (!(out.flags[v] & kLinkStopFlags)) {
        const long long frame = sh_frame;
        if (M > 0) {
            for (int q = 0; q < M; q++) {
                int slot = (sh_head + q) % M;
                int n = ringN[slot];
                for (int e = tid; e < n; e += nth) {
                    int64_t id = ids[P0 + ring_pt[slot * G + e]];
                    dur[id] = (frame - start[id]) - (M - q);
                }
                __syncthreads();
            }
        }
        if (sh_prevg >= gb) {
            const int pg = sh_prevg;
            const int64_t pb = gbase(in, pg), pe = pb + gsize(in, pg);
            for (int64_t p = pb + tid; p < pe; p += nth) {
                int64_t id = ids[p];
                dur[id] = frame - start[id];
            }
        }
    }
    if (tid == 0) out.counter[v] = sh_counter;
}

// Per-row durations through the reference's f32 round trip of the particle
// id (src/execute_gpu.rs:812-815, 1165-1181).
__global__ void durations_kernel(LinkInput in, LinkOutput out, int64_t* row_dur) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= in.npoints) return;
    const int h = in.pgroup[p];
    int x = 0, y = in.nvideos;
    while (y - x > 1) {
        int m = (x + y) >> 1;
        if (in.vgrp[m] <= h) x = m; else y = m;
    }
    const int v = x;
    const int64_t P0 = in.goff[in.vgrp[v]];
    const int64_t id = (int64_t)(float)out.ids[p];
    if (id >= out.counter[v]) {
        atomicOr(out.flags + v, kFlagScratch);
        row_dur[p] = -1;
        return;
    }
    row_dur[p] = out.dur[P0 + id];
}

// Slot mode: the table rows of every point (row_off[g] + j) receive the
// particle id after the reference's f32 round trip and its duration
// (src/execute_gpu.rs:812-815, 1165-1181).  One video.
__global__ void slot_rows_kernel(LinkInput in, LinkOutput out, const int64_t* __restrict__ row_off,
                                 int64_t* __restrict__ particle, int64_t* __restrict__ row_dur) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= in.npoints) return;
    const int g = (int)(p / in.slot_stride);
    const int64_t j = p - (int64_t)g * in.slot_stride;
    if (j >= (int64_t)in.gcount[g]) return;
    const int64_t row = row_off[g] + j;
    const int64_t id = (int64_t)(float)out.ids[p];
    particle[row] = id;
    if (id >= out.counter[0]) {
        atomicOr(out.flags, kFlagScratch);
        row_dur[row] = -1;
        return;
    }
    row_dur[row] = out.dur[id];
}

// --------------------------------------------------------------- launchers
cudaError_t link_sort_groups(const LinkInput& in, uint32_t* srt, uint8_t* scratch, size_t scratch_per_group,
                             int max_group, cudaStream_t st) {
    (void)max_group;
    if (in.ngroups == 0) return cudaSuccess;
    sort_groups_kernel<<<in.ngroups, kLinkThreads, 0, st>>>(in, srt, (uint64_t*)scratch, scratch_per_group / 8, 0,
                                                           nullptr, 0.0f);
    return cudaGetLastError();
}

cudaError_t link_sort_groups_range(const LinkInput& in, uint32_t* srt, int g0, int g1, int32_t* bins, float bin_w,
                                   cudaStream_t st) {
    if (g1 <= g0) return cudaSuccess;
    // groups of at most kSortSmem points sort in shared memory; no scratch
    if (in.slot_stride > kSortSmem) return cudaErrorInvalidValue;
    if (bins && !(bin_w > 0.0f)) return cudaErrorInvalidValue;
    sort_groups_kernel<<<g1 - g0, kLinkThreads, 0, st>>>(in, srt, nullptr, 0, g0, bins, bin_w);
    return cudaGetLastError();
}

cudaError_t link_count_lists(const LinkInput& in, const uint32_t* srt, int64_t* f_cnt, int64_t* b_cnt,
                             cudaStream_t st) {
    return link_count_lists_range(in, srt, 0, in.npoints, f_cnt, b_cnt, nullptr, st);
}

cudaError_t link_count_lists_range(const LinkInput& in, const uint32_t* srt, int64_t p0, int64_t p1,
                                   int64_t* f_cnt, int64_t* b_cnt, uint32_t* flags, cudaStream_t st) {
    if (p1 <= p0) return cudaSuccess;
    LinkLists L;
    L.srt = (uint32_t*)srt;
    L.pbase = p0;
    lists_kernel<0><<<(unsigned)((p1 - p0 + 255) / 256), 256, 0, st>>>(in, L, f_cnt, b_cnt, p0, p1, flags);
    return cudaGetLastError();
}

cudaError_t link_fill_lists(const LinkInput& in, const LinkLists& L, cudaStream_t st) {
    return link_fill_lists_range(in, L, in.npoints, nullptr, st);
}

cudaError_t link_fill_lists_range(const LinkInput& in, const LinkLists& L, int64_t p1, uint32_t* flags,
                                  cudaStream_t st) {
    const int64_t p0 = L.pbase;
    if (p1 <= p0) return cudaSuccess;
    if ((L.f_cap >= 0 || L.b_cap >= 0) && !flags) return cudaErrorInvalidValue;
    lists_kernel<1><<<(unsigned)((p1 - p0 + 255) / 256), 256, 0, st>>>(in, L, nullptr, nullptr, p0, p1, flags);
    return cudaGetLastError();
}

cudaError_t link_run(const LinkInput& in, const LinkLists& L, const LinkScratch& S, const LinkOutput& out,
                     cudaStream_t st) {
    return link_run_window(in, L, S, out, LinkWindow(), st);
}

cudaError_t link_run_window(const LinkInput& in, const LinkLists& L, const LinkScratch& S, const LinkOutput& out,
                            const LinkWindow& w, cudaStream_t st) {
    if (in.nvideos == 0) return cudaSuccess;
    if (w.g0 >= 0 && (in.nvideos != 1 || !w.state)) return cudaErrorInvalidValue;
    // narrow offsets when the forward lists hold fewer than 2^31 entries
    const int64_t fmax = L.f_cap >= 0 ? L.f_cap : L.f_entries;
    if (fmax >= 0 && fmax < (int64_t)INT32_MAX) {
        constexpr size_t bytes = link_smem_bytes<int32_t>();
        cudaFuncSetAttribute(link_video_kernel<int32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        link_video_kernel<int32_t><<<in.nvideos, kLinkThreads, bytes, st>>>(in, L, S, out, w);
    } else {
        constexpr size_t bytes = link_smem_bytes<int64_t>();
        cudaFuncSetAttribute(link_video_kernel<int64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        link_video_kernel<int64_t><<<in.nvideos, kLinkThreads, bytes, st>>>(in, L, S, out, w);
    }
    return cudaGetLastError();
}

cudaError_t link_durations(const LinkInput& in, const LinkOutput& out, int64_t* row_dur, cudaStream_t st) {
    if (in.npoints == 0) return cudaSuccess;
    durations_kernel<<<(unsigned)((in.npoints + 255) / 256), 256, 0, st>>>(in, out, row_dur);
    return cudaGetLastError();
}

cudaError_t link_slot_rows(const LinkInput& in, const LinkOutput& out, const int64_t* row_off, int64_t* particle,
                           int64_t* row_dur, cudaStream_t st) {
    if (in.npoints == 0) return cudaSuccess;
    if (!in.slot_stride || in.nvideos != 1) return cudaErrorInvalidValue;
    slot_rows_kernel<<<(unsigned)((in.npoints + 255) / 256), 256, 0, st>>>(in, out, row_off, particle, row_dur);
    return cudaGetLastError();
}

}  // namespace gt
