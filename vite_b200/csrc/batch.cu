// Batched and served Louvain. Many independent graphs run as one: their CSRs are
// packed into a union (graph j owns the vertex range [voff[j], voff[j+1]) and its
// edges reference only that range), every iteration is one set of launches for
// all graphs with each graph's own 1/(2m), modularity and loop test
// (vg_phase_batch_internal), and one rebuild coarsens all of them at once:
// communities never cross graphs, and first appearance in union order restricted
// to one graph is that graph's own first appearance, so the union's next level is
// the union of the graphs' next levels, packed in the same order.
//
// Each graph follows the level loop of graphClustering (main.cpp:242-513, the
// same steps as vg_louvain_run): phase, rebuild test (main.cpp:378), rebuild
// (:431), caps (:504). Graphs join at round boundaries (one round = one phase
// for every graph in the union, then the rebuild): continuous batching, with
// admission by an estimated device-memory footprint against the batch budget.
#include "vg_internal.cuh"

#include <algorithm>
#include <deque>
#include <map>
#include <memory>

void vg_phase_batch_internal(vg_ctx *ctx, vg_graph *U, int64_t J, const int64_t *h_voff,
                             const int32_t *vjob, const double *h_thresh, const double *h_lower,
                             double *mod_out, int32_t *iters_out, double *sweep_ms);
vg_graph *vg_rebuild_new(vg_ctx *ctx, const vg_graph *g, const int32_t *comm);

namespace {

constexpr int PACK_VCHUNK = 2048;
constexpr int64_t MAX_UNION = INT32_MAX; // vertices and CSR entries of one packed graph
constexpr int PACK_ECHUNK = 8192;

// one source range of a pack: vertices [v_lo, v_lo + nv) with edges
// [e_lo, e_lo + ne) of a graph (a whole graph: v_lo = e_lo = 0, or one graph's
// range inside a union), written at (dst_v, dst_e) of the new union
struct PackSrc {
    const int64_t *rowptr;
    const int32_t *tail;
    const double *weight;
    const int32_t *ref; // null: positions are the graph's own ids
    const int32_t *pos;
    int64_t v_lo, nv, e_lo, ne, dst_v, dst_e;
    int32_t job;
};

__device__ __forceinline__ int64_t table_entry_of(const int64_t *__restrict__ cb, int64_t n,
                                                  int64_t q) {
    int64_t lo = 0, hi = n; // largest j with cb[j] <= q
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (cb[mid] <= q) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void k_pack_vertices(const PackSrc *__restrict__ src, const int64_t *__restrict__ cb,
                                int64_t ns, int64_t nchunks, int64_t *__restrict__ rowptr,
                                int32_t *__restrict__ vjob, int32_t *__restrict__ ref,
                                int32_t *__restrict__ pos) {
    for (int64_t q = blockIdx.x; q < nchunks; q += gridDim.x) {
        const int64_t k = table_entry_of(cb, ns, q);
        const PackSrc s = src[k];
        const int64_t lo = (q - cb[k]) * PACK_VCHUNK;
        const int64_t hi = min(lo + PACK_VCHUNK, s.nv);
        for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const int64_t P = s.dst_v + i;
            rowptr[P] = s.rowptr[s.v_lo + i] - s.e_lo + s.dst_e;
            vjob[P] = s.job;
            if (ref) {
                ref[P] = (int32_t)(s.dst_v + (s.ref ? s.ref[s.v_lo + i] - s.v_lo : i));
                pos[P] = (int32_t)(s.dst_v + (s.pos ? s.pos[s.v_lo + i] - s.v_lo : i));
            }
        }
    }
}

__global__ void k_pack_edges(const PackSrc *__restrict__ src, const int64_t *__restrict__ cb,
                             int64_t ns, int64_t nchunks, int32_t *__restrict__ tail,
                             double *__restrict__ weight) {
    for (int64_t q = blockIdx.x; q < nchunks; q += gridDim.x) {
        const int64_t k = table_entry_of(cb, ns, q);
        const PackSrc s = src[k];
        const int64_t lo = (q - cb[k]) * PACK_ECHUNK;
        const int64_t hi = min(lo + PACK_ECHUNK, s.ne);
        const int64_t shift = s.dst_v - s.v_lo;
        for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            tail[s.dst_e + i] = (int32_t)(s.tail[s.e_lo + i] + shift);
            weight[s.dst_e + i] = s.weight[s.e_lo + i];
        }
    }
}

// communities per graph: used[c] marks the labels in use; every label lies in
// its graph's own range, so its graph is vjob[c]
__global__ void k_mark_used(const int32_t *__restrict__ comm, int64_t n, int32_t *__restrict__ used) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        used[comm[i]] = 1;
}

__global__ void k_count_used(const int32_t *__restrict__ used, const int32_t *__restrict__ vjob,
                             int64_t n, int64_t *__restrict__ count) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        if (used[i]) atomicAdd((unsigned long long *)&count[vjob[i]], 1ULL);
}

__global__ void k_fill_vjob(const int64_t *__restrict__ voff, int64_t J, int64_t n,
                            int32_t *__restrict__ vjob) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        vjob[i] = (int32_t)table_entry_of(voff, J, i);
}

__global__ void k_gather_rowptr(const int64_t *__restrict__ rowptr, const int64_t *__restrict__ at,
                                int64_t n, int64_t *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = rowptr[at[i]];
}

// the level's communities in reference numbering: cvr[ref(p)] = ref(comm[p])
__global__ void k_comm_ref(const int32_t *__restrict__ comm, const int32_t *__restrict__ ref,
                           int64_t n, int32_t *__restrict__ cvr) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = comm[p];
        if (ref) cvr[ref[p]] = ref[c];
        else cvr[p] = c;
    }
}

// main.cpp:381-425 for several graphs at once: each label is renamed by its rank
// among the graph's labels in use (rank = global exclusive scan of `used`, less
// the graph's first entry), then composed into the graph's level-0 map
struct ComposeJob {
    int32_t *all;      // the graph's level-0 map (n entries)
    int64_t n, voff;   // level-0 vertices; the graph's first vertex in the union
    int32_t first;     // level 0: the map is the renamed labels themselves
};

__global__ void k_compose(const ComposeJob *__restrict__ jobs, const int64_t *__restrict__ cb,
                          int64_t nj, int64_t nchunks, const int32_t *__restrict__ cvr,
                          const int64_t *__restrict__ rank) {
    for (int64_t q = blockIdx.x; q < nchunks; q += gridDim.x) {
        const int64_t k = table_entry_of(cb, nj, q);
        const ComposeJob J = jobs[k];
        const int64_t lo = (q - cb[k]) * PACK_VCHUNK;
        const int64_t hi = min(lo + PACK_VCHUNK, J.n);
        const int64_t base = rank[J.voff];
        for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const int64_t x = J.voff + (J.first ? i : J.all[i]);
            J.all[i] = (int32_t)(rank[cvr[x]] - base);
        }
    }
}

template <class T> void upload_vec(vg_ctx *ctx, DevBuf<T> &d, const std::vector<T> &h) {
    d.alloc(ctx, h.size());
    if (!h.empty())
        VG_CUDA(cudaMemcpyAsync(d.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice,
                                ctx->stream));
}

enum JobState { QUEUED = 0, RUNNING = 1, DONE = 2 };

struct BJob {
    int64_t id = 0;
    const vg_graph *src = nullptr; // until packed
    bool take = false;             // the batch frees `src` once packed
    vg_run_params rp{};
    bool want_comm = false;
    int64_t nv0 = 0, ne0 = 0;
    size_t est = 0;
    JobState state = QUEUED;
    bool forgotten = false; // results dropped; erased once out of the packed graph
    // level loop (main.cpp:242-513)
    double prevMod = -1.0;
    int phase = 0, tot_iters = 0;
    std::vector<vg_level_stat> stats;
    DevBuf<int32_t> all; // composed level-0 map (want_comm)
    // current level
    int64_t nv = 0, ne = 0;
};

// one graph's level map: all[i] = rank of the label of level-0 vertex i (or, at
// level 0, of vertex i itself) among the labels in use at this level
__global__ void k_compose_one(int32_t *__restrict__ all, int64_t n0, int32_t first,
                              const int32_t *__restrict__ cvr, const int64_t *__restrict__ rank) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n0;
         i += (int64_t)gridDim.x * blockDim.x)
        all[i] = (int32_t)rank[cvr[first ? i : all[i]]];
}

__global__ void k_widen(const int32_t *__restrict__ x, int64_t n, int64_t *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = x[i];
}

} // namespace

// main.cpp:381-425 for one graph on the device: the level's communities (in
// reference numbering) are renamed by their rank among the labels in use, then
// composed into the level-0 map `all` (n0 entries; at level 0 the renamed
// labels themselves)
void vg_compose_level(vg_ctx *ctx, const vg_graph *g, int32_t *all, int64_t n0, bool first) {
    const int64_t n = g->nv;
    if (!n || !n0) return;
    const int grid = vg_grid(ctx, n, 256);
    DevBuf<int32_t> cvr(ctx, n), used(ctx, n);
    DevBuf<int64_t> rank(ctx, n);
    VG_CUDA(cudaMemsetAsync(used.p, 0, sizeof(int32_t) * n, ctx->stream));
    { LaunchTimer lt(ctx); k_comm_ref<<<grid, 256, 0, ctx->stream>>>(g->comm, g->ref, n, cvr.p); }
    VG_CHECK_LAUNCH();
    { LaunchTimer lt(ctx); k_mark_used<<<grid, 256, 0, ctx->stream>>>(cvr.p, n, used.p); }
    VG_CHECK_LAUNCH();
    vg_scan_i32_async(ctx, used.p, rank.p, n, nullptr);
    { LaunchTimer lt(ctx);
      k_compose_one<<<vg_grid(ctx, n0, 256), 256, 0, ctx->stream>>>(all, n0, first ? 1 : 0, cvr.p,
                                                                    rank.p); }
    VG_CHECK_LAUNCH();
}

// the level-0 map widened to Vite's 64-bit ids and copied to the host buffer
// `out` (pinned memory makes the copy a single DMA at the link's rate)
void vg_download_map(vg_ctx *ctx, const int32_t *all, int64_t n0, int64_t *out) {
    if (!n0) return;
    DevBuf<int64_t> wide(ctx, n0);
    { LaunchTimer lt(ctx);
      k_widen<<<vg_grid(ctx, n0, 256), 256, 0, ctx->stream>>>(all, n0, wide.p); }
    VG_CHECK_LAUNCH();
    VG_CUDA(cudaMemcpyAsync(out, wide.p, sizeof(int64_t) * n0, cudaMemcpyDeviceToHost, ctx->stream));
    vg_sync(ctx);
}

struct vg_batch {
    vg_ctx *ctx = nullptr;
    size_t budget = 0;
    int64_t next_id = 0;
    std::map<int64_t, std::unique_ptr<BJob>> jobs;
    std::deque<int64_t> queue;
    std::vector<int64_t> running; // union order
    std::vector<int64_t> finished;
    size_t running_bytes = 0;
    vg_graph *U = nullptr;
    DevBuf<int32_t> vjob;
    std::vector<int64_t> voff, eoff; // per running job, J + 1
    bool dirty = false;              // membership changed since U was built
    vg_batch_stats st{};
};

namespace {

size_t estimate_bytes(int64_t nv, int64_t ne) {
    // union copy (rowptr, tails, weights, graph id, layout), phase state, and the
    // rebuild's sort and group buffers
    return (size_t)(40 * ne + 200 * nv) + ((size_t)1 << 20);
}

void release_graph(vg_ctx *ctx, vg_graph *&g) {
    if (!g) return;
    vg_graph_release(ctx, g);
    delete g;
    g = nullptr;
}

// Build the union from the running graphs still in U and the newly admitted ones.
void pack(vg_batch *b, const std::vector<int64_t> &keep, const std::vector<int64_t> &admit) {
    vg_ctx *ctx = b->ctx;
    std::vector<PackSrc> srcs;
    std::vector<vg_graph *> laid_raw;
    bool any_ref = b->U && b->U->ref;
    int64_t NV = 0, NE = 0;
    std::vector<int64_t> nvoff(1, 0), neoff(1, 0);
    std::vector<int64_t> order;
    // running graphs keep their place order; their ranges come from U
    std::map<int64_t, size_t> idx;
    for (size_t k = 0; k < b->running.size(); k++) idx[b->running[k]] = k;
    for (int64_t id : keep) {
        const size_t k = idx.at(id);
        PackSrc s{};
        s.rowptr = b->U->rowptr;
        s.tail = b->U->tail;
        s.weight = b->U->weight;
        s.ref = b->U->ref;
        s.pos = b->U->pos;
        s.v_lo = b->voff[k];
        s.nv = b->voff[k + 1] - b->voff[k];
        s.e_lo = b->eoff[k];
        s.ne = b->eoff[k + 1] - b->eoff[k];
        srcs.push_back(s);
        order.push_back(id);
    }
    for (int64_t id : admit) {
        BJob &j = *b->jobs.at(id);
        const vg_graph *g = j.src;
        vg_graph *lg = nullptr;
        if (vg_auto_layout(ctx, g, j.rp.layout)) {
            // the locality layout the plain path gives a graph of this size
            DevBuf<int32_t> ord;
            vg_bfs_order(ctx, g, ord);
            lg = vg_apply_layout(ctx, g, ord.p);
            laid_raw.push_back(lg);
            g = lg;
        }
        if (g->ref) any_ref = true;
        PackSrc s{};
        s.rowptr = g->rowptr;
        s.tail = g->tail;
        s.weight = g->weight;
        s.ref = g->ref;
        s.pos = g->pos;
        s.v_lo = 0;
        s.nv = g->nv;
        s.e_lo = 0;
        s.ne = g->ne;
        srcs.push_back(s);
        order.push_back(id);
    }
    for (size_t k = 0; k < srcs.size(); k++) {
        srcs[k].dst_v = NV;
        srcs[k].dst_e = NE;
        srcs[k].job = (int32_t)k;
        NV += srcs[k].nv;
        NE += srcs[k].ne;
        nvoff.push_back(NV);
        neoff.push_back(NE);
    }
    auto cleanup = [&] {
        for (vg_graph *g : laid_raw) release_graph(ctx, g);
        laid_raw.clear();
    };
    try {
        VG_REQUIRE(NV < INT32_MAX && NE >= 0, "a batch holds fewer than 2^31 vertices (got %lld)",
                   (long long)NV);
        vg_graph *N = new vg_graph();
        N->nv = NV;
        N->ne = NE;
        try {
            N->rowptr = (int64_t *)vg_alloc(ctx, sizeof(int64_t) * (NV + 1));
            N->tail = (int32_t *)vg_alloc(ctx, sizeof(int32_t) * NE);
            N->weight = (double *)vg_alloc(ctx, sizeof(double) * NE);
            if (any_ref) {
                N->ref = (int32_t *)vg_alloc(ctx, sizeof(int32_t) * NV);
                N->pos = (int32_t *)vg_alloc(ctx, sizeof(int32_t) * NV);
            }
            DevBuf<int32_t> vj(ctx, NV);
            std::vector<int64_t> vcb(1, 0), ecb(1, 0);
            for (auto &s : srcs) {
                vcb.push_back(vcb.back() + (s.nv + PACK_VCHUNK - 1) / PACK_VCHUNK);
                ecb.push_back(ecb.back() + (s.ne + PACK_ECHUNK - 1) / PACK_ECHUNK);
            }
            DevBuf<PackSrc> dsrc;
            DevBuf<int64_t> dvcb, decb;
            upload_vec(ctx, dsrc, srcs);
            upload_vec(ctx, dvcb, vcb);
            upload_vec(ctx, decb, ecb);
            const int64_t ns = (int64_t)srcs.size();
            if (vcb.back()) {
                LaunchTimer lt(ctx);
                k_pack_vertices<<<(int)std::min<int64_t>(vcb.back(), 8LL * ctx->sm_count), 256, 0,
                                  ctx->stream>>>(dsrc.p, dvcb.p, ns, vcb.back(), N->rowptr, vj.p,
                                                 N->ref, N->pos);
            }
            VG_CHECK_LAUNCH();
            if (ecb.back()) {
                LaunchTimer lt(ctx);
                k_pack_edges<<<(int)std::min<int64_t>(ecb.back(), 16LL * ctx->sm_count), 256, 0,
                               ctx->stream>>>(dsrc.p, decb.p, ns, ecb.back(), N->tail, N->weight);
            }
            VG_CHECK_LAUNCH();
            VG_CUDA(cudaMemcpyAsync(N->rowptr + NV, &neoff.back(), sizeof(int64_t),
                                    cudaMemcpyHostToDevice, ctx->stream));
            vg_sync(ctx); // the host tables above go out of scope
            release_graph(ctx, b->U);
            b->U = N;
            b->vjob = std::move(vj);
        } catch (...) {
            vg_graph_release(ctx, N);
            delete N;
            throw;
        }
    } catch (...) {
        cleanup();
        throw;
    }
    cleanup();
    for (int64_t id : admit) {
        BJob &j = *b->jobs.at(id);
        if (j.take) {
            vg_graph *g = const_cast<vg_graph *>(j.src);
            release_graph(ctx, g);
        }
        j.src = nullptr;
        j.state = RUNNING;
    }
    b->running = order;
    b->voff = nvoff;
    b->eoff = neoff;
    for (size_t k = 0; k < order.size(); k++) {
        BJob &j = *b->jobs.at(order[k]);
        j.nv = nvoff[k + 1] - nvoff[k];
        j.ne = neoff[k + 1] - neoff[k];
    }
    b->dirty = false;
}

// compose the accepted graphs' level maps (main.cpp:381-425) on the device
void compose_levels(vg_batch *b, const std::vector<size_t> &which) {
    if (which.empty()) return;
    vg_ctx *ctx = b->ctx;
    vg_graph *U = b->U;
    const int64_t n = U->nv;
    const int grid = vg_grid(ctx, n, 256);
    DevBuf<int32_t> cvr(ctx, n), used(ctx, n);
    DevBuf<int64_t> rank(ctx, n);
    VG_CUDA(cudaMemsetAsync(used.p, 0, sizeof(int32_t) * n, ctx->stream));
    { LaunchTimer lt(ctx); k_comm_ref<<<grid, 256, 0, ctx->stream>>>(U->comm, U->ref, n, cvr.p); }
    VG_CHECK_LAUNCH();
    { LaunchTimer lt(ctx); k_mark_used<<<grid, 256, 0, ctx->stream>>>(cvr.p, n, used.p); }
    VG_CHECK_LAUNCH();
    vg_scan_i32_async(ctx, used.p, rank.p, n, nullptr);
    std::vector<ComposeJob> cj;
    std::vector<int64_t> cb(1, 0);
    for (size_t k : which) {
        BJob &j = *b->jobs.at(b->running[k]);
        const bool first = j.phase == 0;
        if (first) j.all.alloc(ctx, j.nv0);
        ComposeJob c{j.all.p, j.nv0, b->voff[k], first ? 1 : 0};
        cj.push_back(c);
        cb.push_back(cb.back() + (j.nv0 + PACK_VCHUNK - 1) / PACK_VCHUNK);
    }
    DevBuf<ComposeJob> dj;
    DevBuf<int64_t> dcb;
    upload_vec(ctx, dj, cj);
    upload_vec(ctx, dcb, cb);
    if (cb.back()) {
        LaunchTimer lt(ctx);
        k_compose<<<(int)std::min<int64_t>(cb.back(), 8LL * ctx->sm_count), 256, 0, ctx->stream>>>(
            dj.p, dcb.p, (int64_t)cj.size(), cb.back(), cvr.p, rank.p);
    }
    VG_CHECK_LAUNCH();
    vg_sync(ctx);
}

// the next level of every graph in U, and where each graph landed in it
void rebuild_union(vg_batch *b) {
    vg_ctx *ctx = b->ctx;
    vg_graph *U = b->U;
    const int64_t J = (int64_t)b->running.size();
    const int64_t n = U->nv;
    const int grid = vg_grid(ctx, n, 256);
    DevBuf<int64_t> cnt(ctx, J);
    {
        DevBuf<int32_t> used(ctx, n);
        VG_CUDA(cudaMemsetAsync(used.p, 0, sizeof(int32_t) * n, ctx->stream));
        VG_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int64_t) * J, ctx->stream));
        { LaunchTimer lt(ctx); k_mark_used<<<grid, 256, 0, ctx->stream>>>(U->comm, n, used.p); }
        VG_CHECK_LAUNCH();
        { LaunchTimer lt(ctx); k_count_used<<<grid, 256, 0, ctx->stream>>>(used.p, b->vjob.p, n, cnt.p); }
        VG_CHECK_LAUNCH();
    }
    std::vector<int64_t> hc(J);
    VG_CUDA(cudaMemcpyAsync(hc.data(), cnt.p, sizeof(int64_t) * J, cudaMemcpyDeviceToHost, ctx->stream));
    vg_sync(ctx);
    vg_graph *N = vg_rebuild_new(ctx, U, U->comm);
    std::vector<int64_t> nvoff(J + 1, 0);
    for (int64_t k = 0; k < J; k++) nvoff[k + 1] = nvoff[k] + hc[k];
    try {
        VG_REQUIRE(nvoff[J] == N->nv, "batch rebuild: %lld communities counted, %lld vertices built",
                   (long long)nvoff[J], (long long)N->nv);
        DevBuf<int64_t> dv, de(ctx, J + 1);
        upload_vec(ctx, dv, nvoff);
        {
            LaunchTimer lt(ctx);
            k_gather_rowptr<<<1, 256, 0, ctx->stream>>>(N->rowptr, dv.p, J + 1, de.p);
        }
        VG_CHECK_LAUNCH();
        std::vector<int64_t> neoff(J + 1);
        VG_CUDA(cudaMemcpyAsync(neoff.data(), de.p, sizeof(int64_t) * (J + 1),
                                cudaMemcpyDeviceToHost, ctx->stream));
        DevBuf<int32_t> vj(ctx, N->nv);
        if (N->nv) {
            LaunchTimer lt(ctx);
            k_fill_vjob<<<vg_grid(ctx, N->nv, 256), 256, 0, ctx->stream>>>(dv.p, J + 1, N->nv, vj.p);
        }
        VG_CHECK_LAUNCH();
        vg_sync(ctx);
        release_graph(ctx, b->U);
        b->U = N;
        b->vjob = std::move(vj);
        b->voff = nvoff;
        b->eoff = neoff;
        for (int64_t k = 0; k < J; k++) {
            BJob &j = *b->jobs.at(b->running[k]);
            j.nv = nvoff[k + 1] - nvoff[k];
            j.ne = neoff[k + 1] - neoff[k];
        }
    } catch (...) {
        release_graph(ctx, N);
        throw;
    }
}

double elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    VG_CUDA(cudaEventSynchronize(b));
    VG_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
}

void check_params(const vg_run_params *rp) {
    VG_REQUIRE(!rp->coloring && !rp->vertex_order,
               "batched runs take the plain phase (no coloring or vertex ordering)");
    VG_REQUIRE(rp->et_type == 0, "batched runs take the plain phase (no early termination)");
    VG_REQUIRE(!rp->threshold_scaling, "batched runs do not take threshold cycling");
    VG_REQUIRE(rp->threshold > 0.0 && rp->threshold < 1.0,
               "batched runs need a threshold in (0, 1) (got %g)", rp->threshold);
    VG_REQUIRE(rp->layout >= 0 && rp->layout <= 2, "layout must be 0, 1 or 2");
}

// erase the forgotten jobs that are no longer part of the packed graph
void sweep_forgotten(vg_batch *b) {
    std::vector<int64_t> gone;
    for (auto &kv : b->jobs)
        if (kv.second->forgotten &&
            std::find(b->running.begin(), b->running.end(), kv.first) == b->running.end())
            gone.push_back(kv.first);
    for (int64_t id : gone) b->jobs.erase(id);
}

// one round: admit, phase, per-graph level bookkeeping, rebuild
void step(vg_batch *b) {
    vg_ctx *ctx = b->ctx;
    std::vector<int64_t> keep;
    int64_t union_nv = 0, union_ne = 0;
    for (int64_t id : b->running) {
        const BJob &j = *b->jobs.at(id);
        if (j.state != RUNNING) continue;
        keep.push_back(id);
        union_nv += j.nv;
        union_ne += j.ne;
    }
    // admission: first come first served while the estimated footprint fits the
    // budget and the union stays within 32-bit vertex and edge indexing
    std::vector<int64_t> admit;
    size_t bytes = b->running_bytes;
    while (!b->queue.empty()) {
        BJob &j = *b->jobs.at(b->queue.front());
        const bool alone = keep.empty() && admit.empty();
        if (b->budget && bytes + j.est > b->budget && !alone) break;
        if (union_nv + j.nv0 > MAX_UNION || union_ne + j.ne0 > MAX_UNION) break;
        bytes += j.est;
        union_nv += j.nv0;
        union_ne += j.ne0;
        admit.push_back(j.id);
        b->queue.pop_front();
    }
    if (keep.empty() && admit.empty()) {
        release_graph(ctx, b->U);
        b->vjob.release();
        b->running.clear();
        b->voff.assign(1, 0);
        b->eoff.assign(1, 0);
        b->dirty = false;
        sweep_forgotten(b);
        return;
    }
    if (!admit.empty() || b->dirty || keep.size() != b->running.size()) {
        try {
            pack(b, keep, admit);
        } catch (...) {
            for (auto it = admit.rbegin(); it != admit.rend(); ++it) b->queue.push_front(*it);
            throw;
        }
        b->running_bytes = bytes;
        b->st.admitted += (int64_t)admit.size();
        sweep_forgotten(b);
    }
    if (b->running.empty()) return;
    const int64_t J = (int64_t)b->running.size();
    std::vector<double> thresh(J), lower(J, -1.0), mod(J);
    std::vector<int32_t> iters(J);
    for (int64_t k = 0; k < J; k++) thresh[k] = b->jobs.at(b->running[k])->rp.threshold;
    cudaEvent_t evs[3] = {nullptr, nullptr, nullptr};
    struct EvGuard {
        cudaEvent_t *e;
        ~EvGuard() {
            for (int i = 0; i < 3; i++)
                if (e[i]) cudaEventDestroy(e[i]);
        }
    } evguard{evs};
    for (auto &e : evs) VG_CUDA(cudaEventCreate(&e));
    cudaEvent_t e0 = evs[0], e1 = evs[1], e2 = evs[2];
    VG_CUDA(cudaEventRecord(e0, ctx->stream));
    double sweep_ms = 0.0;
    vg_phase_batch_internal(ctx, b->U, J, b->voff.data(), b->vjob.p, thresh.data(), lower.data(),
                            mod.data(), iters.data(), &sweep_ms);
    VG_CUDA(cudaEventRecord(e1, ctx->stream));
    const double phase_s = elapsed_ms(e0, e1) * 1e-3;
    std::vector<size_t> compose;
    std::vector<char> cont(J, 0);
    bool any_cont = false;
    for (int64_t k = 0; k < J; k++) {
        BJob &j = *b->jobs.at(b->running[k]);
        vg_level_stat ls{};
        ls.nv = j.nv;
        ls.ne = j.ne;
        ls.iters = iters[k];
        ls.modularity = mod[k];
        ls.seconds_phase = phase_s;
        ls.seconds_sweep = sweep_ms * 1e-3;
        ls.edges_swept = (int64_t)iters[k] * j.ne;
        j.tot_iters += iters[k];
        const bool accepted = (mod[k] - j.prevMod) > j.rp.threshold; // main.cpp:378
        if (accepted && j.want_comm) compose.push_back((size_t)k);
        j.stats.push_back(ls);
        bool go = false;
        if (accepted) {
            // compose first: it reads j.phase to tell level 0
            go = !j.rp.one_phase;
        }
        cont[k] = go;
    }
    compose_levels(b, compose);
    for (int64_t k = 0; k < J; k++) {
        BJob &j = *b->jobs.at(b->running[k]);
        const bool accepted = (mod[k] - j.prevMod) > j.rp.threshold;
        if (accepted) {
            j.prevMod = mod[k];
            j.phase++;
            if (j.phase == 200 /* TERMINATION_PHASE_COUNT */ || j.tot_iters > 10000) cont[k] = 0;
        }
        if (cont[k]) {
            any_cont = true;
        } else {
            j.state = DONE;
            b->finished.push_back(j.id);
            b->running_bytes -= std::min(b->running_bytes, j.est);
            b->st.completed++;
        }
    }
    double rebuild_s = 0.0;
    if (any_cont) {
        VG_CUDA(cudaEventRecord(e1, ctx->stream));
        rebuild_union(b);
        VG_CUDA(cudaEventRecord(e2, ctx->stream));
        rebuild_s = elapsed_ms(e1, e2) * 1e-3;
        for (int64_t k = 0; k < J; k++) {
            BJob &j = *b->jobs.at(b->running[k]);
            if (cont[k]) j.stats.back().seconds_rebuild = rebuild_s;
        }
        b->dirty = false;
        for (int64_t k = 0; k < J; k++)
            if (!cont[k]) b->dirty = true;
    } else {
        release_graph(ctx, b->U);
        b->vjob.release();
        b->running.clear();
        b->voff.assign(1, 0);
        b->eoff.assign(1, 0);
        sweep_forgotten(b);
    }
    b->st.rounds++;
    b->st.seconds_phase += phase_s;
    b->st.seconds_rebuild += rebuild_s;
    vg_sync(ctx);
}

} // namespace

extern "C" vg_status vg_batch_create(vg_ctx *ctx, size_t budget_bytes, vg_batch **out) {
    if (!ctx || !out) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        vg_batch *b = new vg_batch();
        b->ctx = ctx;
        b->budget = budget_bytes;
        b->voff.assign(1, 0);
        b->eoff.assign(1, 0);
        *out = b;
    });
}

extern "C" vg_status vg_batch_destroy(vg_batch *b) {
    if (!b) return VG_ERR_ARG;
    vg_ctx *ctx = b->ctx;
    return vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        for (auto &kv : b->jobs) {
            BJob &j = *kv.second;
            if (j.state == QUEUED && j.take && j.src) {
                vg_graph *g = const_cast<vg_graph *>(j.src);
                release_graph(ctx, g);
            }
        }
        b->jobs.clear();
        release_graph(ctx, b->U);
        b->vjob.release();
        vg_sync(ctx);
        delete b;
    });
}

extern "C" vg_status vg_batch_submit(vg_batch *b, vg_graph *g, const vg_run_params *rp,
                                     int32_t flags, int64_t *job_out) {
    if (!b || !g || !rp || !job_out) return VG_ERR_ARG;
    return vg_guard(b->ctx, [&] {
        check_params(rp);
        VG_REQUIRE(g->nv >= 1 && g->ne >= 1, "a batched graph needs vertices and edges");
        VG_REQUIRE(g->nv <= MAX_UNION && g->ne <= MAX_UNION,
                   "a batched graph has fewer than 2^31 vertices and CSR entries");
        auto j = std::make_unique<BJob>();
        j->id = b->next_id++;
        j->src = g;
        j->take = (flags & VG_BATCH_TAKE) != 0;
        j->want_comm = (flags & VG_BATCH_COMM) != 0;
        j->rp = *rp;
        j->nv0 = g->nv;
        j->ne0 = g->ne;
        j->est = estimate_bytes(g->nv, g->ne);
        VG_REQUIRE(!b->budget || j->est <= b->budget,
                   "graph needs about %zu bytes of device memory, more than the batch budget %zu",
                   j->est, b->budget);
        *job_out = j->id;
        b->queue.push_back(j->id);
        b->jobs.emplace(j->id, std::move(j));
        b->st.submitted++;
    });
}

extern "C" vg_status vg_batch_step(vg_batch *b, int32_t *running_out, int32_t *queued_out) {
    if (!b) return VG_ERR_ARG;
    return vg_guard(b->ctx, [&] {
        VG_CUDA(cudaSetDevice(b->ctx->device));
        step(b);
        int32_t r = 0;
        for (int64_t id : b->running)
            if (b->jobs.at(id)->state == RUNNING) r++;
        if (running_out) *running_out = r;
        if (queued_out) *queued_out = (int32_t)b->queue.size();
    });
}

extern "C" vg_status vg_batch_poll(vg_batch *b, int64_t *ids, int32_t max_ids, int32_t *n_out) {
    if (!b || !n_out || (max_ids > 0 && !ids)) return VG_ERR_ARG;
    return vg_guard(b->ctx, [&] {
        const int32_t n = (int32_t)std::min<size_t>(b->finished.size(), (size_t)std::max(max_ids, 0));
        for (int32_t i = 0; i < n; i++) ids[i] = b->finished[i];
        b->finished.erase(b->finished.begin(), b->finished.begin() + n);
        *n_out = n;
    });
}

extern "C" vg_status vg_batch_result(vg_batch *b, int64_t job, vg_level_stat *levels,
                                     int32_t max_levels, int32_t *nlevels_out, int64_t *comm_out) {
    if (!b) return VG_ERR_ARG;
    return vg_guard(b->ctx, [&] {
        auto it = b->jobs.find(job);
        VG_REQUIRE(it != b->jobs.end() && !it->second->forgotten, "unknown batch job %lld",
                   (long long)job);
        BJob &j = *it->second;
        VG_REQUIRE(j.state == DONE, "batch job %lld has not finished", (long long)job);
        const int32_t n = (int32_t)j.stats.size();
        if (levels)
            for (int32_t i = 0; i < std::min(n, max_levels); i++) levels[i] = j.stats[i];
        if (nlevels_out) *nlevels_out = n;
        if (comm_out) {
            VG_REQUIRE(j.want_comm, "batch job %lld was submitted without VG_BATCH_COMM",
                       (long long)job);
            VG_CUDA(cudaSetDevice(b->ctx->device));
            if (!j.all.p) { // no level accepted: every vertex is its own community
                for (int64_t i = 0; i < j.nv0; i++) comm_out[i] = -1;
            } else {
                std::vector<int32_t> h(j.nv0);
                VG_CUDA(cudaMemcpyAsync(h.data(), j.all.p, sizeof(int32_t) * j.nv0,
                                        cudaMemcpyDeviceToHost, b->ctx->stream));
                vg_sync(b->ctx);
                for (int64_t i = 0; i < j.nv0; i++) comm_out[i] = h[i];
            }
        }
    });
}

extern "C" vg_status vg_batch_forget(vg_batch *b, int64_t job) {
    if (!b) return VG_ERR_ARG;
    return vg_guard(b->ctx, [&] {
        auto it = b->jobs.find(job);
        VG_REQUIRE(it != b->jobs.end() && !it->second->forgotten, "unknown batch job %lld",
                   (long long)job);
        VG_REQUIRE(it->second->state == DONE, "batch job %lld has not finished", (long long)job);
        VG_CUDA(cudaSetDevice(b->ctx->device));
        if (std::find(b->running.begin(), b->running.end(), job) == b->running.end()) {
            b->jobs.erase(it);
        } else { // still a range of the packed graph until the next step repacks it
            it->second->forgotten = true;
            it->second->all.release();
            it->second->stats.clear();
        }
    });
}

extern "C" vg_status vg_batch_get_stats(vg_batch *b, vg_batch_stats *out) {
    if (!b || !out) return VG_ERR_ARG;
    *out = b->st;
    out->running = 0;
    for (int64_t id : b->running)
        if (b->jobs.at(id)->state == RUNNING) out->running++;
    out->queued = (int64_t)b->queue.size();
    out->running_bytes = b->running_bytes;
    return VG_OK;
}
