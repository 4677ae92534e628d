// Context, device memory accounting, graph upload/download and the vertex degree
// kernel (distSumVertexDegree / distCalcConstantForSecondTerm, louvain.cpp:2161-2218).
#include "vg_internal.cuh"

#include <cstring>

void vg_throw(vg_status s, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    throw vg_error(s, buf);
}

int vg_grid(vg_ctx *ctx, int64_t work, int block, int per_sm) {
    int64_t g = (work + block - 1) / block;
    int64_t cap = (int64_t)ctx->sm_count * per_sm * VG_GRID_SCALE;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

void *vg_alloc(vg_ctx *ctx, size_t bytes) {
    if (bytes == 0) return nullptr;
    if (ctx->budget && ctx->in_use + bytes > ctx->budget)
        vg_throw(VG_ERR_OOM, "device memory budget exceeded: %zu in use + %zu requested > %zu",
                 ctx->in_use, bytes, ctx->budget);
    void *p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, ctx->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        vg_throw(VG_ERR_OOM, "cudaMallocAsync(%zu bytes): %s", bytes, cudaGetErrorString(e));
    }
    ctx->in_use += bytes;
    return p;
}

void vg_free(vg_ctx *ctx, void *p, size_t bytes) {
    if (!p) return;
    cudaFreeAsync(p, ctx->stream);
    ctx->in_use -= bytes;
}

void *vg_pinned(vg_ctx *ctx, size_t bytes) {
    if (ctx->pinned_bytes < bytes) {
        if (ctx->pinned) cudaFreeHost(ctx->pinned);
        ctx->pinned = nullptr;
        size_t b = bytes < 4096 ? 4096 : bytes;
        VG_CUDA(cudaMallocHost(&ctx->pinned, b));
        ctx->pinned_bytes = b;
    }
    return ctx->pinned;
}

void vg_sync(vg_ctx *ctx) {
    VG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->profile) vg_profile_collect(ctx);
}

LaunchTimer::LaunchTimer(vg_ctx *c) : ctx(c) {
    ctx->profile_launches++;
    if (!ctx->profile) return;
    if (!ctx->event_pool.empty()) {
        a = ctx->event_pool.back().first;
        b = ctx->event_pool.back().second;
        ctx->event_pool.pop_back();
    } else {
        VG_CUDA(cudaEventCreate(&a));
        VG_CUDA(cudaEventCreate(&b));
    }
    VG_CUDA(cudaEventRecord(a, ctx->stream));
}

LaunchTimer::~LaunchTimer() {
    if (!a) return;
    cudaEventRecord(b, ctx->stream);
    ctx->pending.emplace_back(a, b);
}

void vg_profile_collect(vg_ctx *ctx) {
    for (auto &pr : ctx->pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) ctx->profile_ms += ms;
        ctx->event_pool.push_back(pr);
    }
    ctx->pending.clear();
}

// ---------------------------------------------------------------------------------

extern "C" vg_status vg_ctx_create(int device, size_t mem_budget_bytes, vg_ctx **out) {
    if (!out) return VG_ERR_ARG;
    *out = nullptr;
    vg_ctx *ctx = new vg_ctx();
    vg_status st = vg_guard(ctx, [&] {
        int n = 0;
        VG_CUDA(cudaGetDeviceCount(&n));
        VG_REQUIRE(device >= 0 && device < n, "device %d not present (%d devices)", device, n);
        VG_CUDA(cudaSetDevice(device));
        ctx->device = device;
        ctx->budget = mem_budget_bytes;
        VG_CUDA(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device));
        VG_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        // the side stream and its fork/join events exist from the start, so that a
        // fork inside a stream capture creates nothing
        VG_CUDA(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
        VG_CUDA(cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming));
        VG_CUDA(cudaEventCreateWithFlags(&ctx->join, cudaEventDisableTiming));
        // keep freed blocks in the stream-ordered pool instead of returning them
        cudaMemPool_t pool;
        VG_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t thr = UINT64_MAX;
        VG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    });
    if (st != VG_OK) {
        fprintf(stderr, "vg_ctx_create: %s\n", ctx->last_error.c_str());
        delete ctx;
        return st;
    }
    *out = ctx;
    return VG_OK;
}

cudaStream_t vg_side_fork(vg_ctx *ctx) {
    VG_CUDA(cudaEventRecord(ctx->fork, ctx->stream));
    VG_CUDA(cudaStreamWaitEvent(ctx->side, ctx->fork, 0));
    return ctx->side;
}

void vg_side_join(vg_ctx *ctx) {
    VG_CUDA(cudaEventRecord(ctx->join, ctx->side));
    VG_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->join, 0));
}

extern "C" vg_status vg_ctx_destroy(vg_ctx *ctx) {
    if (!ctx) return VG_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->side) cudaStreamSynchronize(ctx->side);
    for (auto &pr : ctx->pending) ctx->event_pool.push_back(pr);
    for (auto &pr : ctx->event_pool) {
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->fork) cudaEventDestroy(ctx->fork);
    if (ctx->join) cudaEventDestroy(ctx->join);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return VG_OK;
}

extern "C" vg_status vg_ctx_reserve(vg_ctx *ctx, size_t bytes) {
    if (!ctx) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        void *p = vg_alloc(ctx, bytes);
        vg_free(ctx, p, bytes);
        vg_sync(ctx);
    });
}

extern "C" vg_status vg_ctx_stream(vg_ctx *ctx, void **stream_out) {
    if (!ctx || !stream_out) return VG_ERR_ARG;
    *stream_out = (void *)ctx->stream;
    return VG_OK;
}

extern "C" const char *vg_last_error(const vg_ctx *ctx) {
    return ctx ? ctx->last_error.c_str() : "null context";
}

extern "C" size_t vg_ctx_bytes_in_use(const vg_ctx *ctx) { return ctx ? ctx->in_use : 0; }

extern "C" vg_status vg_ctx_profile(vg_ctx *ctx, int32_t enable, double *kernel_ms_out,
                                    int64_t *launches_out, int32_t reset) {
    if (!ctx) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        vg_sync(ctx);
        if (kernel_ms_out) *kernel_ms_out = ctx->profile_ms;
        if (launches_out) *launches_out = ctx->profile_launches;
        if (reset) {
            ctx->profile_ms = 0.0;
            ctx->profile_launches = 0;
        }
        ctx->profile = enable != 0;
    });
}

// ---------------------------------------------------------------------------------
// graphs

namespace {
__global__ void k_integral(const double *__restrict__ w, int64_t ne, int *__restrict__ bad) {
    int mine = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ne;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double x = w[i];
        if (!(fabs(x) <= 1048576.0) || x != floor(x)) mine = 1;
    }
    if (__any_sync(0xffffffffu, mine) && (threadIdx.x & 31) == 0) atomicOr(bad, 1);
}
} // namespace

bool vg_weights_integral(vg_ctx *ctx, vg_graph *g) {
    if (g->integral >= 0) return g->integral == 1;
    int r = 1;
    if (g->ne >= ((int64_t)1 << 31)) {
        r = 0;
    } else if (g->ne > 0) {
        DevBuf<int> bad(ctx, 1);
        VG_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
        {
            LaunchTimer lt(ctx);
            k_integral<<<vg_grid(ctx, g->ne, 256), 256, 0, ctx->stream>>>(g->weight, g->ne, bad.p);
        }
        VG_CHECK_LAUNCH();
        int *h = (int *)vg_pinned(ctx, sizeof(int));
        VG_CUDA(cudaMemcpyAsync(h, bad.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        vg_sync(ctx);
        r = *h ? 0 : 1;
    }
    g->integral = (int8_t)r;
    return r == 1;
}

vg_graph *vg_graph_wrap(vg_ctx *ctx, int64_t nv, int64_t ne, int64_t *rowptr, int32_t *tail,
                        double *weight) {
    (void)ctx;
    vg_graph *g = new vg_graph();
    g->nv = nv;
    g->ne = ne;
    g->rowptr = rowptr;
    g->tail = tail;
    g->weight = weight;
    return g;
}

void vg_graph_release(vg_ctx *ctx, vg_graph *g) {
    if (!g) return;
    vg_free(ctx, g->rowptr, sizeof(int64_t) * (g->nv + 1));
    vg_free(ctx, g->tail, sizeof(int32_t) * g->ne);
    vg_free(ctx, g->weight, sizeof(double) * g->ne);
    vg_free(ctx, g->colors, sizeof(int32_t) * g->nv);
    vg_free(ctx, g->comm, sizeof(int32_t) * g->nv);
    vg_free(ctx, g->ref, sizeof(int32_t) * g->nv);
    vg_free(ctx, g->pos, sizeof(int32_t) * g->nv);
    g->ref = nullptr;
    g->pos = nullptr;
    g->rowptr = nullptr;
    g->tail = nullptr;
    g->weight = nullptr;
    g->colors = nullptr;
    g->comm = nullptr;
}

namespace {
// flags row offsets (n1 of them, the first taken as base) that decrease, hold a row of
// more than INT32_MAX entries (degrees are 32-bit in the sweep), or do not end at base + ne
__global__ void k_check_rowptr(const int64_t *__restrict__ rp, int64_t n1, int64_t base,
                               int64_t ne, int *__restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n1;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i + 1 < n1) {
            const int64_t len = rp[i + 1] - rp[i];
            if (len < 0 || len > (int64_t)INT32_MAX) *bad = 1;
        }
        if (i == n1 - 1 && rp[i] - base != ne) *bad = 1;
    }
}
} // namespace

void vg_check_rowptr_async(vg_ctx *ctx, const int64_t *rp, int64_t n1, int64_t base, int64_t ne,
                           int *bad) {
    if (n1 <= 0) return;
    {
        LaunchTimer lt(ctx);
        k_check_rowptr<<<vg_grid(ctx, n1, 256), 256, 0, ctx->stream>>>(rp, n1, base, ne, bad);
    }
    VG_CHECK_LAUNCH();
}

// Vite's 16-byte Edge records -> int32 tails + FP64 weights; flags tails out of range
__global__ void k_split_edges(const vg_edge *__restrict__ e, int64_t ne, int64_t nv,
                              int32_t *__restrict__ tail, double *__restrict__ w,
                              int *__restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ne;
         i += (int64_t)gridDim.x * blockDim.x) {
        const longlong2 v = reinterpret_cast<const longlong2 *>(e)[i];
        const int64_t t = v.x;
        if (t < 0 || t >= nv) *bad = 1;
        tail[i] = (int32_t)t;
        w[i] = __longlong_as_double(v.y);
    }
}

__global__ void k_join_edges(const int32_t *__restrict__ tail, const double *__restrict__ w,
                             int64_t ne, vg_edge *__restrict__ e) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ne;
         i += (int64_t)gridDim.x * blockDim.x) {
        longlong2 v;
        v.x = tail[i];
        v.y = __double_as_longlong(w[i]);
        reinterpret_cast<longlong2 *>(e)[i] = v;
    }
}

extern "C" vg_status vg_graph_upload(vg_ctx *ctx, int64_t nv, int64_t ne, const int64_t *rowptr,
                                     const vg_edge *edges, vg_graph **out) {
    if (!ctx || !out) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        *out = nullptr;
        VG_REQUIRE(nv >= 0 && ne >= 0 && rowptr, "bad graph sizes");
        VG_REQUIRE(ne == 0 || edges, "edges missing");
        VG_REQUIRE(nv < (int64_t)INT32_MAX, "graphs must have fewer than 2^31 vertices (nv=%lld)",
                   (long long)nv);
        VG_REQUIRE(rowptr[0] == 0 && rowptr[nv] == ne, "rowptr must start at 0 and end at ne");
        VG_CUDA(cudaSetDevice(ctx->device));
        DevBuf<int64_t> rp(ctx, nv + 1);
        DevBuf<int32_t> tail(ctx, ne);
        DevBuf<double> w(ctx, ne);
        VG_CUDA(cudaMemcpyAsync(rp.p, rowptr, sizeof(int64_t) * (nv + 1), cudaMemcpyHostToDevice,
                                ctx->stream));
        // bad[0]: row offsets, bad[1]: tails; read back together
        DevBuf<int> bad(ctx, 2);
        VG_CUDA(cudaMemsetAsync(bad.p, 0, 2 * sizeof(int), ctx->stream));
        vg_check_rowptr_async(ctx, rp.p, nv + 1, 0, ne, bad.p);
        if (ne) {
            // stage the 16-byte records through two bounded device buffers in chunks:
            // the copies run back to back on the context's stream while the side
            // stream splits the chunk before (a buffer is refilled only after its split)
            const int64_t chunk = ne < (int64_t)(1 << 24) ? ne : (int64_t)(1 << 24);
            DevBuf<vg_edge> stage0(ctx, chunk), stage1(ctx, chunk);
            vg_edge *stage[2] = {stage0.p, stage1.p};
            cudaEvent_t copied[2] = {nullptr, nullptr}, split[2] = {nullptr, nullptr};
            auto destroy = [&] {
                for (int b = 0; b < 2; b++) {
                    if (copied[b]) cudaEventDestroy(copied[b]);
                    if (split[b]) cudaEventDestroy(split[b]);
                }
            };
            try {
                for (int b = 0; b < 2; b++) {
                    VG_CUDA(cudaEventCreateWithFlags(&copied[b], cudaEventDisableTiming));
                    VG_CUDA(cudaEventCreateWithFlags(&split[b], cudaEventDisableTiming));
                }
                const bool two = !ctx->profile; // with profiling every launch stays on one stream
                cudaStream_t ss = two ? ctx->side : ctx->stream;
                int64_t k = 0;
                for (int64_t off = 0; off < ne; off += chunk, k++) {
                    const int b = (int)(k & 1);
                    const int64_t len = (ne - off) < chunk ? (ne - off) : chunk;
                    if (two && k >= 2) VG_CUDA(cudaStreamWaitEvent(ctx->stream, split[b], 0));
                    VG_CUDA(cudaMemcpyAsync(stage[b], edges + off, sizeof(vg_edge) * len,
                                            cudaMemcpyHostToDevice, ctx->stream));
                    if (two) {
                        VG_CUDA(cudaEventRecord(copied[b], ctx->stream));
                        VG_CUDA(cudaStreamWaitEvent(ss, copied[b], 0));
                    }
                    {
                        LaunchTimer lt(ctx);
                        k_split_edges<<<vg_grid(ctx, len, 256), 256, 0, ss>>>(
                            stage[b], len, nv, tail.p + off, w.p + off, bad.p + 1);
                    }
                    VG_CHECK_LAUNCH();
                    if (two) VG_CUDA(cudaEventRecord(split[b], ss));
                }
                if (two) { // the stream waits for the last splits
                    for (int b = 0; b < 2 && b < k; b++)
                        VG_CUDA(cudaStreamWaitEvent(ctx->stream, split[(k - 1 - b) & 1], 0));
                }
            } catch (...) {
                destroy();
                throw;
            }
            destroy();
        }
        int *hb = (int *)vg_pinned(ctx, 2 * sizeof(int));
        VG_CUDA(cudaMemcpyAsync(hb, bad.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        vg_sync(ctx);
        VG_REQUIRE(hb[0] == 0, "rowptr must not decrease, and no row may hold more than 2^31 - 1 "
                               "entries");
        VG_REQUIRE(hb[1] == 0, "edge tail out of range [0, nv)");
        *out = vg_graph_wrap(ctx, nv, ne, rp.detach(), tail.detach(), w.detach());
    });
}

extern "C" vg_status vg_graph_info(const vg_graph *g, int64_t *nv, int64_t *ne) {
    if (!g) return VG_ERR_ARG;
    if (nv) *nv = g->nv;
    if (ne) *ne = g->ne;
    return VG_OK;
}

extern "C" vg_status vg_graph_download(vg_ctx *ctx, const vg_graph *g_in, int64_t *rowptr,
                                       vg_edge *edges) {
    if (!ctx || !g_in) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        // a graph stored in the library's own layout goes out in reference order
        vg_graph *tmp = g_in->ref ? vg_remove_layout(ctx, g_in) : nullptr;
        const vg_graph *g = tmp ? tmp : g_in;
        struct Drop {
            vg_ctx *c;
            vg_graph *t;
            ~Drop() {
                if (t) {
                    vg_graph_release(c, t);
                    delete t;
                }
            }
        } drop{ctx, tmp};
        if (rowptr)
            VG_CUDA(cudaMemcpyAsync(rowptr, g->rowptr, sizeof(int64_t) * (g->nv + 1),
                                    cudaMemcpyDeviceToHost, ctx->stream));
        if (edges && g->ne) {
            const int64_t chunk = g->ne < (int64_t)(1 << 24) ? g->ne : (int64_t)(1 << 24);
            DevBuf<vg_edge> stage(ctx, chunk);
            for (int64_t off = 0; off < g->ne; off += chunk) {
                const int64_t len = (g->ne - off) < chunk ? (g->ne - off) : chunk;
                {
                    LaunchTimer lt(ctx);
                    k_join_edges<<<vg_grid(ctx, len, 256), 256, 0, ctx->stream>>>(
                        g->tail + off, g->weight + off, len, stage.p);
                }
                VG_CHECK_LAUNCH();
                VG_CUDA(cudaMemcpyAsync(edges + off, stage.p, sizeof(vg_edge) * len,
                                        cudaMemcpyDeviceToHost, ctx->stream));
            }
        }
        vg_sync(ctx);
    });
}

extern "C" vg_status vg_graph_free(vg_ctx *ctx, vg_graph *g) {
    if (!ctx || !g) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        vg_graph_release(ctx, g);
        delete g;
    });
}
