// Internal declarations shared by the CUDA sources of libvite_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "vite_b200.h"

// ---------------------------------------------------------------------------------
// error handling

struct vg_error : public std::exception {
    vg_status status;
    std::string msg;
    vg_error(vg_status s, std::string m) : status(s), msg(std::move(m)) {}
    const char *what() const noexcept override { return msg.c_str(); }
};

[[noreturn]] void vg_throw(vg_status s, const char *fmt, ...);

#define VG_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t _e = (call);                                                               \
        if (_e != cudaSuccess)                                                                 \
            vg_throw(_e == cudaErrorMemoryAllocation ? VG_ERR_OOM : VG_ERR_CUDA, "%s: %s (%s:%d)", \
                     #call, cudaGetErrorString(_e), __FILE__, __LINE__);                       \
    } while (0)

#define VG_CHECK_LAUNCH() VG_CUDA(cudaGetLastError())

#define VG_REQUIRE(cond, ...)                                                                  \
    do {                                                                                       \
        if (!(cond)) vg_throw(VG_ERR_ARG, __VA_ARGS__);                                        \
    } while (0)

// ---------------------------------------------------------------------------------
// context

struct vg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    size_t budget = 0;        // 0 = unlimited
    size_t in_use = 0;        // bytes held through vg_alloc
    std::string last_error;
    int sm_count = 148;
    // pinned host staging for small read-backs
    void *pinned = nullptr;
    size_t pinned_bytes = 0;
    // kernel instrumentation (events around each launch when enabled)
    bool profile = false;
    double profile_ms = 0.0;
    int64_t profile_launches = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> event_pool;
    // sweep launch tuning (vg_ctx_set_tuning / vg_autotune); all zero = built-in defaults
    vg_tuning tune{};
    // a second stream for kernels that may overlap the main stream's (vg_side_stream),
    // with the events that fork it from and join it back to the main stream
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

// the context's side stream: work enqueued on the stream vg_side_fork returns, up to
// vg_side_join, runs concurrently with the main stream's (both ordered after what the
// main stream held at the fork; the main stream's later work waits for the join)
cudaStream_t vg_side_fork(vg_ctx *ctx);
void vg_side_join(vg_ctx *ctx);

// stream-ordered device allocation accounted against the context budget
void *vg_alloc(vg_ctx *ctx, size_t bytes);
void vg_free(vg_ctx *ctx, void *p, size_t bytes);

template <class T> struct DevBuf {
    vg_ctx *ctx = nullptr;
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(vg_ctx *c, size_t count) { alloc(c, count); }
    void alloc(vg_ctx *c, size_t count) {
        release();
        ctx = c;
        n = count;
        p = count ? (T *)vg_alloc(c, count * sizeof(T)) : nullptr;
    }
    void release() {
        if (p) vg_free(ctx, p, n * sizeof(T));
        p = nullptr;
        n = 0;
    }
    T *detach() {
        T *q = p;
        p = nullptr;
        n = 0;
        return q;
    }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : ctx(o.ctx), p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) { release(); ctx = o.ctx; p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    void swap(DevBuf &o) { std::swap(ctx, o.ctx); std::swap(p, o.p); std::swap(n, o.n); }
};

// pinned scratch for read-backs of a few scalars
void *vg_pinned(vg_ctx *ctx, size_t bytes);
void vg_sync(vg_ctx *ctx);

// launch bracketing for instrumentation
struct LaunchTimer {
    vg_ctx *ctx;
    cudaEvent_t a = nullptr, b = nullptr;
    explicit LaunchTimer(vg_ctx *c);
    ~LaunchTimer();
};
void vg_profile_collect(vg_ctx *ctx);

// ---------------------------------------------------------------------------------
// device graph: Vite's CSR with int32 tails and FP64 weights in separate arrays

struct vg_graph {
    int64_t nv = 0, ne = 0;
    int64_t *rowptr = nullptr; // nv+1
    int32_t *tail = nullptr;   // ne
    double *weight = nullptr;  // ne
    // coloring attached by vg_color / vg_set_colors (int32, -1 uncolored)
    int32_t *colors = nullptr;
    int64_t num_colors = -1;   // reference's nextColor; -1 = none
    // communities of the last phase (int32, positions), kept for vg_rebuild
    int32_t *comm = nullptr;
    // HBM layout: position p holds the vertex with reference id ref[p]; pos is the
    // inverse. Both null when positions are the reference ids.
    int32_t *ref = nullptr;
    int32_t *pos = nullptr;
    // 1: every weight is an integer of magnitude at most 2^20 (and ne < 2^31), so
    // every sum of weights is an exact integer below 2^51 whatever its order;
    // 0: not so; -1: not yet known (vg_weights_integral computes it)
    int8_t integral = -1;
};

// whether g's weights are integral in the sense above (computed once per graph)
bool vg_weights_integral(vg_ctx *ctx, vg_graph *g);

// reference id of the vertex (or community) at position p
__device__ __forceinline__ int32_t vg_rid(const int32_t *__restrict__ ref, int32_t p) {
    return ref ? __ldg(ref + p) : p;
}

// layout helpers (layout.cu)
void vg_bfs_order(vg_ctx *ctx, const vg_graph *g, DevBuf<int32_t> &order);
vg_graph *vg_apply_layout(vg_ctx *ctx, const vg_graph *g, const int32_t *order);
vg_graph *vg_remove_layout(vg_ctx *ctx, const vg_graph *g);
void vg_download_comm_ref(vg_ctx *ctx, const vg_graph *g, const int32_t *comm, int64_t *out);
// graphClustering's -o map (main.cpp:381-425) built on the device: compose level g's
// communities into the level-0 map `all` (n0 int32 entries), then copy it out as int64
void vg_compose_level(vg_ctx *ctx, const vg_graph *g, int32_t *all, int64_t n0, bool first);
void vg_download_map(vg_ctx *ctx, const int32_t *all, int64_t n0, int64_t *out);
void vg_download_vals_ref(vg_ctx *ctx, const vg_graph *g, const int32_t *x, int64_t *out);
void vg_ref_to_pos_inplace(vg_ctx *ctx, const vg_graph *g, int32_t *x, bool are_ids);
// whether the locality layout pays for g (sampled clustering coefficient)
bool vg_local_structure(vg_ctx *ctx, const vg_graph *g);
// layout mode 2 (automatic): graphs of at least 2^18 vertices with local structure
inline bool vg_auto_layout(vg_ctx *ctx, const vg_graph *g, int mode) {
    if (g->ref || mode == 0) return false;
    if (mode == 1) return true;
    return g->nv >= (1 << 18) && vg_local_structure(ctx, g);
}

// stream-ordered check of n1 row offsets (the first one is `base`): sets *bad (device
// memory) when they decrease, a row holds more than INT32_MAX entries, or the last is
// not base + ne
void vg_check_rowptr_async(vg_ctx *ctx, const int64_t *rp, int64_t n1, int64_t base, int64_t ne,
                           int *bad);

void vg_graph_release(vg_ctx *ctx, vg_graph *g);
// the graph takes ownership of the three arrays
vg_graph *vg_graph_wrap(vg_ctx *ctx, int64_t nv, int64_t ne, int64_t *rowptr, int32_t *tail,
                        double *weight);

// ---------------------------------------------------------------------------------
// primitives (primitives.cu)

// exclusive scan in place over n elements; returns the total (one stream sync)
int64_t vg_exclusive_scan_i64(vg_ctx *ctx, int64_t *data, int64_t n);
int64_t vg_exclusive_scan_i32_to_i64(vg_ctx *ctx, const int32_t *in, int64_t *out, int64_t n);
// the same, stream-ordered with no host round trip; the total goes to *dev_total
// (device memory) when dev_total is not null
void vg_scan_i64_async(vg_ctx *ctx, int64_t *data, int64_t n, int64_t *dev_total);
void vg_scan_i32_async(vg_ctx *ctx, const int32_t *in, int64_t *out, int64_t n,
                       int64_t *dev_total);
// stable LSD radix sort of 64-bit keys with 32-bit payloads over the low `bits` bits
void vg_radix_sort_pairs(vg_ctx *ctx, uint64_t *keys, uint32_t *vals, int64_t n, int bits);
// sum of a double array (deterministic)
double vg_sum_f64(vg_ctx *ctx, const double *x, int64_t n);

// CSR from (src, dst, w) triples in their given order: stable sort by (src, dst),
// adjacent duplicates combined by summing their weights in order when `combine`.
// nv rows; the three inputs are consumed (freed). With dst_map the stored tail
// is dst_map[dst] (dst orders the row, dst_map names the position).
vg_graph *vg_csr_from_triples(vg_ctx *ctx, int64_t nv, DevBuf<int32_t> &src,
                              DevBuf<int32_t> &dst, DevBuf<double> &w, int64_t m, bool combine,
                              const int32_t *dst_map = nullptr);

// ---------------------------------------------------------------------------------
// kernels shared across files

// grid of at most per_sm * VG_GRID_SCALE blocks per SM for `work` threads in blocks
// of `block` (grid-stride kernels)
#ifndef VG_GRID_SCALE
#define VG_GRID_SCALE 4
#endif
int vg_grid(vg_ctx *ctx, int64_t work, int block, int per_sm = 8);

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31; }

// A chunk leader's left fold: acc + stage[j] for each lane j of `above` (its peers
// above it) in lane order; stage holds the warp's 32 values, 16-byte aligned. Every
// read is issued before the first add, so the chain waits on the additions only.
__device__ __forceinline__ double vg_fold_above(double acc, const double *stage, unsigned above) {
    const double2 *s2 = reinterpret_cast<const double2 *>(stage);
    double2 x[16];
#pragma unroll
    for (int j = 0; j < 16; j++) x[j] = s2[j];
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if (above & (1u << (2 * j))) acc = __dadd_rn(acc, x[j].x);
        if (above & (2u << (2 * j))) acc = __dadd_rn(acc, x[j].y);
    }
    return acc;
}

// One left fold of n values, get(0) .. get(n - 1) in that order, by a whole warp:
// lane 0 returns s + get(0) + ... + get(n - 1) added one at a time (with first, the
// fold starts from get(0) instead of s + get(0)). The additions are one chain of
// dependent operations, so the warp only keeps that chain fed: all lanes fetch the
// next VG_FOLD_STEP values into registers while lane 0 adds the current ones from
// `stage`, the warp's own 2 x VG_FOLD_STEP doubles of shared memory. A stage is
// rewritten only after the __syncwarp that follows lane 0's reads of it; the final
// __syncwarp lets the caller reuse `stage` at once. n, s and first are warp-uniform.
constexpr int VG_FOLD_STEP = 256;
template <class Get>
__device__ __forceinline__ double vg_warp_ordered_fold(int64_t n, Get get, double *stage,
                                                       double s, bool first) {
    constexpr int PER = VG_FOLD_STEP / 32;
    const int lane = threadIdx.x & 31;
    double x[PER];
#pragma unroll
    for (int t = 0; t < PER; t++) {
        const int64_t j = t * 32 + lane;
        x[t] = j < n ? get(j) : 0.0;
    }
    int b = 0;
    for (int64_t c0 = 0; c0 < n; c0 += VG_FOLD_STEP, b ^= 1) {
        double *st = stage + b * VG_FOLD_STEP;
#pragma unroll
        for (int t = 0; t < PER; t++) st[t * 32 + lane] = x[t];
        __syncwarp();
        const int64_t c1 = c0 + VG_FOLD_STEP;
        if (c1 < n) { // the next step's values, in flight during the additions
#pragma unroll
            for (int t = 0; t < PER; t++) {
                const int64_t j = c1 + t * 32 + lane;
                x[t] = j < n ? get(j) : 0.0;
            }
        }
        if (lane == 0) {
            const int cnt = (int)(n - c0 < VG_FOLD_STEP ? n - c0 : VG_FOLD_STEP);
            int t = 0;
            if (first && c0 == 0) {
                s = st[0];
                t = 1;
            }
            if (t + 8 <= cnt) {
                // groups of eight, alternately in ya and yb: the next group is read
                // before the current one is added, so the chain waits on the
                // additions only
                double ya[8], yb[8];
#pragma unroll
                for (int u = 0; u < 8; u++) ya[u] = st[t + u];
                t += 8;
                for (;;) {
                    if (t + 8 > cnt) {
#pragma unroll
                        for (int u = 0; u < 8; u++) s = __dadd_rn(s, ya[u]);
                        break;
                    }
#pragma unroll
                    for (int u = 0; u < 8; u++) yb[u] = st[t + u];
                    t += 8;
#pragma unroll
                    for (int u = 0; u < 8; u++) s = __dadd_rn(s, ya[u]);
                    if (t + 8 > cnt) {
#pragma unroll
                        for (int u = 0; u < 8; u++) s = __dadd_rn(s, yb[u]);
                        break;
                    }
#pragma unroll
                    for (int u = 0; u < 8; u++) ya[u] = st[t + u];
                    t += 8;
#pragma unroll
                    for (int u = 0; u < 8; u++) s = __dadd_rn(s, yb[u]);
                }
            }
            for (; t < cnt; t++) s = __dadd_rn(s, st[t]);
        }
    }
    __syncwarp();
    return s;
}

// counter-based generator shared with the oracle's restatement
__host__ __device__ __forceinline__ uint64_t vg_sm64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
__host__ __device__ __forceinline__ uint64_t vg_mix(uint64_t seed, uint64_t stream, uint64_t k) {
    return vg_sm64(vg_sm64(seed ^ (stream * 0xD1B54A32D192ED03ULL)) ^ k);
}
__device__ __forceinline__ uint64_t vg_uint_below(uint64_t r, uint64_t n) { return __umul64hi(r, n); }
__device__ __forceinline__ double vg_unit_double(uint64_t r) {
    return __dmul_rn((double)(r >> 11), 1.0 / 9007199254740992.0);
}

// entry-point wrapper: converts exceptions into a status + message
template <class F> vg_status vg_guard(vg_ctx *ctx, F &&f) {
    try {
        f();
        return VG_OK;
    } catch (const vg_error &e) {
        if (ctx) ctx->last_error = e.msg;
        return e.status;
    } catch (const std::exception &e) {
        if (ctx) ctx->last_error = e.what();
        return VG_ERR_CUDA;
    }
}
