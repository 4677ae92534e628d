// HBM layout of a level graph.
//
// The reference numbers vertices by its input (for the in-memory RGG: LCG order,
// which is random in space), so the gathers of a sweep (community of every
// neighbour, degree of every candidate community) hit random cache lines. The
// library may therefore store a graph in its own vertex order ("positions"):
// position p holds the vertex whose reference id is ref[p] (pos is the inverse).
// Rows keep the reference's CSR order of their entries, so every sum is the same
// left fold; every comparison of ids (tie-breaks, the singleton rule, the
// early-termination test, coloring hashes, first-appearance numbering in the
// rebuild) is made on reference ids, so results are identical to the
// reference's. Only the addresses change.
//
// The locality order is computed on the device from the graph alone: a
// multi-source breadth-first search from hashed seeds (about one seed per 256
// vertices) labels each vertex with its nearest seed, and vertices are ordered by
// (seed, degree bucket, BFS distance, id), so a cluster occupies a contiguous range
// of positions, most neighbours of a vertex lie in the same few cache lines, and
// 32 consecutive vertices mostly share a degree bucket.
#include "vg_internal.cuh"

#include <algorithm>

namespace {

// one seed per 2^SEED_SHIFT vertices on average. Measured on RGG 2^24 (level-0 sweep
// set / whole run): 2^12 25.4 / 57.9 ms, 2^11 23.8 / 56.0, 2^10 22.7 / 54.9, 2^9 22.2 /
// 54.3, 2^8 22.3 / 54.1, 2^7 22.8 / 54.7, 2^6 23.4 / 55.3; with the current BFS and
// degree buckets 2^10 22.8 / 53.5, 2^9 22.3 / 52.9, 2^8 22.3 / 52.8
#ifndef VG_SEED_SHIFT
#define VG_SEED_SHIFT 8
#endif
constexpr int SEED_SHIFT = VG_SEED_SHIFT;
constexpr int MAX_BFS_STEPS = 255;

__global__ void k_bfs_init(int64_t nv, uint64_t seed, int32_t *__restrict__ label,
                           uint8_t *__restrict__ dist) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv;
         v += (int64_t)gridDim.x * blockDim.x) {
        const bool s = (vg_mix(seed, 41, (uint64_t)v) & ((1ULL << SEED_SHIFT) - 1)) == 0;
        label[v] = s ? (int32_t)v : -1;
        dist[v] = s ? 0 : 255;
    }
}

// one level: vertices at distance step-1 claim their unlabeled neighbours. A warp
// takes 128 consecutive vertices (four per lane, read as one word of distances),
// lists its frontier vertices in shared memory and spreads all their entries over
// its lanes, four per lane per pass (each lane finds its entry's row by a search
// over the rows' running offsets): the tail loads, distance gathers and claims of a
// whole pass are issued together, so a pass costs one chain of dependent memory
// accesses for up to 128 entries.
// unvisited vertices are found through the byte array of distances (255 =
// unvisited), which stays in L2. Frontier vertices that reach the same unvisited
// vertex in one level all write it: its distance is the same either way and its
// label ends up as one of theirs (any of them is a nearest seed), so nothing waits on
// a compare-and-swap (which made the layout 0.5 ms slower at 2^24); the claim count
// can exceed the vertices claimed, and is only tested against zero
constexpr int BFS_WARPS = 8;

// a relaxed (but atomic) 32-bit store: concurrent writers leave one of their values
__device__ __forceinline__ void store_relaxed(int32_t *p, int32_t v) {
    asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__global__ void __launch_bounds__(BFS_WARPS * 32) k_bfs_step(
    const int64_t *__restrict__ rowptr, const int32_t *__restrict__ tail, int64_t nv, int step,
    int32_t *__restrict__ label, uint8_t *__restrict__ dist, unsigned long long *__restrict__ claimed,
    const unsigned long long *__restrict__ prev_claimed) {
    // the level before claimed nothing: the search has ended, so has this level
    if (prev_claimed && *prev_claimed == 0) return;
    __shared__ int32_t fl_all[BFS_WARPS][128];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int32_t *fl = fl_all[threadIdx.x >> 5];
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t prev = (uint32_t)(step - 1);
    unsigned long long mine = 0;
    for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 128; base < nv;
         base += nw * 128) {
        // 1. the frontier among vertices u0 .. u0 + 3 (u0 is a multiple of 4)
        const int64_t u0 = base + 4 * lane;
        unsigned fb = 0;
        if (u0 + 3 < nv) {
            const uint32_t dw = *reinterpret_cast<const uint32_t *>(dist + u0);
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (((dw >> (8 * q)) & 0xffu) == prev) fb |= 1u << q;
        } else {
            for (int q = 0; q < 4; q++)
                if (u0 + q < nv && dist[u0 + q] == prev) fb |= 1u << q;
        }
        const int cnt = __popc(fb);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(full, incl, o);
            if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(full, incl, 31);
        if (total == 0) continue;
        {
            int at = incl - cnt;
            for (int q = 0; q < 4; q++)
                if ((fb >> q) & 1u) fl[at++] = (int32_t)(u0 + q);
        }
        __syncwarp();
        // 2. up to 32 frontier vertices at a time, their entries spread over the lanes
        for (int r0 = 0; r0 < total; r0 += 32) {
            const bool has = r0 + lane < total;
            int64_t e0 = 0, len = 0;
            int32_t lu = 0;
            if (has) {
                const int32_t u = fl[r0 + lane];
                e0 = rowptr[u];
                len = rowptr[u + 1] - e0;
                lu = label[u];
            }
            int64_t ri = len; // inclusive running offsets of the rows
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t y = __shfl_up_sync(full, ri, o);
                if (lane >= o) ri += y;
            }
            const int64_t T = __shfl_sync(full, ri, 31);
            const int64_t rs = has ? ri - len : INT64_MAX; // this lane's row start
            for (int64_t k0 = 0; k0 < T; k0 += 128) {
                int32_t w[4], L[4];
                bool h[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int64_t k = k0 + 32 * q + lane;
                    h[q] = k < T;
                    const int64_t kq = h[q] ? k : 0;
                    // the row holding entry kq: the last lane whose row starts at or before it
                    int j = 0;
#pragma unroll
                    for (int st = 16; st; st >>= 1) {
                        const int64_t r = __shfl_sync(full, rs, j + st);
                        if (r <= kq) j += st;
                    }
                    const int64_t ej = __shfl_sync(full, e0, j) + (kq - __shfl_sync(full, rs, j));
                    L[q] = __shfl_sync(full, lu, j);
                    w[q] = h[q] ? tail[ej] : 0;
                }
                uint8_t dd[4];
#pragma unroll
                for (int q = 0; q < 4; q++) dd[q] = h[q] ? dist[w[q]] : 0;
#pragma unroll
                for (int q = 0; q < 4; q++)
                    if (h[q] && dd[q] == 255) {
                        store_relaxed(&label[w[q]], L[q]);
                        dist[w[q]] = (uint8_t)step;
                        mine++;
                    }
            }
        }
        __syncwarp();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(claimed, mine);
}

// degree bucket of the order key: the sweep's short-row kernels run each warp of
// 32 consecutive vertices (the degree 17..32 kernel: 32 consecutive entries of its
// position-ordered list) with loops as long as its largest row, so vertices of
// similar degree are kept together inside a cluster (RGG 2^24 run: buckets of width 4
// up to 16 and one for 17..32: 53.3 ms; 17..32 split in three: 53.1 ms; widths 2 up to
// 16 as well: 52.6 ms against 52.75)
__device__ __forceinline__ uint32_t degree_bucket(int64_t d) {
    return d <= 6 ? 0u : d <= 8 ? 1u : d <= 10 ? 2u : d <= 12 ? 3u : d <= 14 ? 4u : d <= 16 ? 5u
         : d <= 20 ? 6u : d <= 24 ? 7u : d <= 32 ? 8u : 9u;
}

// (cluster, degree bucket, BFS distance), the distance in dbits bits; unreached
// vertices (components without a seed) keep their own place, in a bucket of their own
__global__ void k_order_keys(int64_t nv, const int64_t *__restrict__ rowptr,
                             const int32_t *__restrict__ label, const uint8_t *__restrict__ dist,
                             int dbits, uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t l = label[v];
        const uint64_t b = degree_bucket(rowptr[v + 1] - rowptr[v]);
        keys[v] = l < 0 ? (((uint64_t)v << (4 + dbits)) | (15ull << dbits))
                        : (((uint64_t)l << (4 + dbits)) | (b << dbits) | dist[v]);
        vals[v] = (uint32_t)v;
    }
}

__global__ void k_inverse(const int32_t *__restrict__ perm, int64_t n, int32_t *__restrict__ inv) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x)
        inv[perm[k]] = (int32_t)k;
}

// k-th row of the moved graph: its degree and where it starts in the source CSR
__global__ void k_gather_deg(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ from,
                             int64_t n, int64_t *__restrict__ deg, int64_t *__restrict__ src_start) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = from[k];
        const int64_t s = rowptr[r];
        deg[k] = rowptr[r + 1] - s;
        src_start[k] = s;
    }
}

// new row k = old row from[k] (starting at src_start[k]), tails renamed through
// `rename`, entry order kept; eight lanes per row (rows are short), two rows per
// group of lanes at a time and two entries of each per lane per step: the four
// tails and weights are loaded before the renames are gathered
__global__ void k_move_rows(const int32_t *__restrict__ tail, const double *__restrict__ w, int64_t n,
                            const int64_t *__restrict__ src_start,
                            const int32_t *__restrict__ rename, const int64_t *__restrict__ rp2,
                            int32_t *__restrict__ tail2, double *__restrict__ w2) {
    const int sub = threadIdx.x & 7;
    const int64_t grp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 3;
    const int64_t ng = ((int64_t)gridDim.x * blockDim.x) >> 3;
    for (int64_t k = grp; k < n; k += 2 * ng) {
        const int64_t kb = k + ng;
        const bool hb = kb < n;
        const int64_t sa = src_start[k], oa = rp2[k], la = rp2[k + 1] - oa;
        const int64_t sb = hb ? src_start[kb] : 0, ob = hb ? rp2[kb] : 0;
        const int64_t lb = hb ? rp2[kb + 1] - ob : 0;
        const int64_t m = la > lb ? la : lb;
        for (int64_t j = sub; j < m; j += 16) {
            int32_t t[4] = {0, 0, 0, 0}, r[4];
            double x[4] = {0.0, 0.0, 0.0, 0.0};
            const bool h[4] = {j < la, j + 8 < la, j < lb, j + 8 < lb};
            const int64_t src[4] = {sa + j, sa + j + 8, sb + j, sb + j + 8};
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (h[q]) {
                    t[q] = tail[src[q]];
                    x[q] = w[src[q]];
                }
#pragma unroll
            for (int q = 0; q < 4; q++) r[q] = h[q] ? rename[t[q]] : 0;
            const int64_t dst[4] = {oa + j, oa + j + 8, ob + j, ob + j + 8};
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (h[q]) {
                    tail2[dst[q]] = r[q];
                    w2[dst[q]] = x[q];
                }
        }
    }
}

__global__ void k_copy_i32(const int32_t *__restrict__ a, int64_t n, int32_t *__restrict__ b) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x)
        b[k] = a[k];
}

// community vector of positions -> reference ids, indexed by reference vertex id
__global__ void k_comm_to_ref(const int32_t *__restrict__ comm, int64_t n,
                              const int32_t *__restrict__ ref, int64_t *__restrict__ out) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x)
        out[ref[p]] = ref[comm[p]];
}

// per-vertex values (colors) in position order -> reference order
__global__ void k_vals_to_ref(const int32_t *__restrict__ x, int64_t n,
                              const int32_t *__restrict__ ref, int64_t *__restrict__ out) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x)
        out[ref[p]] = x[p];
}

// reference-ordered int32 values -> position order; `rename` maps the values too
__global__ void k_ref_to_pos(const int32_t *__restrict__ in, int64_t n,
                             const int32_t *__restrict__ ref, const int32_t *__restrict__ rename,
                             int32_t *__restrict__ out) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int32_t x = in[ref[p]];
        out[p] = (rename && x >= 0) ? rename[x] : x;
    }
}

// Local structure test: for a hashed sample of vertices, pairs of neighbours (u, w)
// are checked for an edge u-w (the clustering coefficient). Geometric graphs have
// a high one (about 0.59 for a 2-D random geometric graph), preferential-attachment
// and uniform random graphs a vanishing one; only the former gain from the
// locality layout. One warp per sampled vertex; u's row is scanned up to SCAN_CAP.
constexpr int CC_SAMPLE = 4096;
constexpr int CC_PAIRS = 8;
constexpr int CC_SCAN_CAP = 256;

__global__ void k_cc_sample(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ tail,
                            int64_t nv, uint64_t seed, unsigned long long *__restrict__ counts) {
    const int lane = threadIdx.x & 31;
    const int64_t wg = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long hits = 0, pairs = 0;
    for (int64_t s = wg; s < CC_SAMPLE; s += nw) {
        const int64_t v = (int64_t)vg_uint_below(vg_mix(seed, 43, (uint64_t)s), (uint64_t)nv);
        const int64_t e0 = rowptr[v], d = rowptr[v + 1] - e0;
        if (d < 2) continue;
        for (int p = 0; p < CC_PAIRS; p++) {
            const uint64_t r = vg_mix(seed, 44, (uint64_t)(s * CC_PAIRS + p));
            const int64_t i = (int64_t)vg_uint_below(r, (uint64_t)d);
            int64_t j = (int64_t)vg_uint_below(r * 0x9E3779B97F4A7C15ULL + 1, (uint64_t)(d - 1));
            if (j >= i) j++;
            const int32_t u = tail[e0 + i], w = tail[e0 + j];
            if (u == w || u == v || w == v) continue;
            const int64_t f0 = rowptr[u], f1 = min(rowptr[u + 1], f0 + CC_SCAN_CAP);
            bool found = false;
            for (int64_t k = f0 + lane; k < f1; k += 32) found |= tail[k] == w;
            found = __any_sync(0xffffffffu, found);
            if (lane == 0) {
                pairs++;
                hits += found ? 1 : 0;
            }
        }
    }
    if (lane == 0 && pairs) {
        atomicAdd(&counts[0], hits);
        atomicAdd(&counts[1], pairs);
    }
}

} // namespace

// whether g has the local structure the locality layout exploits (sampled
// clustering coefficient at least 0.1)
bool vg_local_structure(vg_ctx *ctx, const vg_graph *g) {
    if (g->nv < 3 || g->ne == 0) return false;
    DevBuf<unsigned long long> counts(ctx, 2);
    VG_CUDA(cudaMemsetAsync(counts.p, 0, 2 * sizeof(unsigned long long), ctx->stream));
    {
        LaunchTimer lt(ctx);
        k_cc_sample<<<CC_SAMPLE * 32 / 256, 256, 0, ctx->stream>>>(g->rowptr, g->tail, g->nv,
                                                                 0xcc5eedULL, counts.p);
    }
    VG_CHECK_LAUNCH();
    unsigned long long *h = (unsigned long long *)vg_pinned(ctx, 2 * sizeof(unsigned long long));
    VG_CUDA(cudaMemcpyAsync(h, counts.p, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            ctx->stream));
    vg_sync(ctx);
    return h[1] > 0 && (double)h[0] >= 0.1 * (double)h[1];
}

// graph with rows in `from` order; tails renamed through `rename`
static vg_graph *move_rows(vg_ctx *ctx, const vg_graph *g, const int32_t *from,
                           const int32_t *rename) {
    const int64_t nv = g->nv, ne = g->ne;
    DevBuf<int64_t> rp(ctx, nv + 1), src(ctx, nv);
    VG_CUDA(cudaMemsetAsync(rp.p + nv, 0, sizeof(int64_t), ctx->stream));
    if (nv) {
        LaunchTimer lt(ctx);
        k_gather_deg<<<vg_grid(ctx, nv, 256), 256, 0, ctx->stream>>>(g->rowptr, from, nv, rp.p,
                                                                     src.p);
    }
    VG_CHECK_LAUNCH();
    vg_scan_i64_async(ctx, rp.p, nv + 1, nullptr);
    DevBuf<int32_t> tail(ctx, ne);
    DevBuf<double> w(ctx, ne);
    if (nv) {
        LaunchTimer lt(ctx);
        k_move_rows<<<vg_grid(ctx, nv * 8, 256), 256, 0, ctx->stream>>>(
            g->tail, g->weight, nv, src.p, rename, rp.p, tail.p, w.p);
    }
    VG_CHECK_LAUNCH();
    return vg_graph_wrap(ctx, nv, ne, rp.detach(), tail.detach(), w.detach());
}

void vg_bfs_order(vg_ctx *ctx, const vg_graph *g, DevBuf<int32_t> &order) {
    const int64_t nv = g->nv;
    order.alloc(ctx, nv);
    if (!nv) return;
    DevBuf<int32_t> label(ctx, nv);
    DevBuf<uint8_t> dist(ctx, nv);
    // steps run in groups of BFS_GROUP, each with its own claim counter, and the
    // counters are read back once per group: the search has ended at the first
    // step that claimed nothing (the steps after it see that count and return at once)
    constexpr int BFS_GROUP = 8;
    DevBuf<unsigned long long> claimed(ctx, BFS_GROUP);
    unsigned long long *h =
        (unsigned long long *)vg_pinned(ctx, BFS_GROUP * sizeof(unsigned long long));
    const int grid = vg_grid(ctx, nv, 256);
    const int sgrid = vg_grid(ctx, (nv + 3) / 4, BFS_WARPS * 32); // a lane per four vertices
    { LaunchTimer lt(ctx); k_bfs_init<<<grid, 256, 0, ctx->stream>>>(nv, 0x5eedULL, label.p, dist.p); }
    VG_CHECK_LAUNCH();
    bool done = false;
    int depth = 0; // largest distance any vertex got
    for (int step0 = 1; step0 <= MAX_BFS_STEPS - 1 && !done; step0 += BFS_GROUP) {
        const int ns = std::min(BFS_GROUP, MAX_BFS_STEPS - step0);
        VG_CUDA(cudaMemsetAsync(claimed.p, 0, BFS_GROUP * sizeof(unsigned long long), ctx->stream));
        for (int k = 0; k < ns; k++) {
            LaunchTimer lt(ctx);
            k_bfs_step<<<sgrid, BFS_WARPS * 32, 0, ctx->stream>>>(
                g->rowptr, g->tail, nv, step0 + k, label.p, dist.p, claimed.p + k,
                k > 0 ? claimed.p + k - 1 : nullptr);
            VG_CHECK_LAUNCH();
        }
        VG_CUDA(cudaMemcpyAsync(h, claimed.p, ns * sizeof(*h), cudaMemcpyDeviceToHost, ctx->stream));
        vg_sync(ctx);
        for (int k = 0; k < ns && !done; k++) {
            if (h[k] == 0) done = true;
            else depth = step0 + k;
        }
    }
    int dbits = 1;
    while ((1 << dbits) <= depth) dbits++;
    DevBuf<uint64_t> keys(ctx, nv);
    DevBuf<uint32_t> vals(ctx, nv);
    { LaunchTimer lt(ctx);
      k_order_keys<<<grid, 256, 0, ctx->stream>>>(nv, g->rowptr, label.p, dist.p, dbits, keys.p,
                                                  vals.p); }
    VG_CHECK_LAUNCH();
    int vbits = 1;
    while (vbits < 40 && ((int64_t)1 << vbits) < nv) vbits++;
    vg_radix_sort_pairs(ctx, keys.p, vals.p, nv, vbits + 4 + dbits);
    VG_CUDA(cudaMemcpyAsync(order.p, vals.p, sizeof(int32_t) * nv, cudaMemcpyDeviceToDevice,
                            ctx->stream));
}

// g in reference layout -> the same graph stored in `order` (order[p] = reference id)
vg_graph *vg_apply_layout(vg_ctx *ctx, const vg_graph *g, const int32_t *order) {
    VG_REQUIRE(g->ref == nullptr, "graph already has a layout");
    const int64_t nv = g->nv;
    DevBuf<int32_t> pos(ctx, nv), ref(ctx, nv);
    if (nv) {
        { LaunchTimer lt(ctx); k_inverse<<<vg_grid(ctx, nv, 256), 256, 0, ctx->stream>>>(order, nv, pos.p); }
        VG_CHECK_LAUNCH();
        { LaunchTimer lt(ctx); k_copy_i32<<<vg_grid(ctx, nv, 256), 256, 0, ctx->stream>>>(order, nv, ref.p); }
        VG_CHECK_LAUNCH();
    }
    vg_graph *h = move_rows(ctx, g, order, pos.p);
    h->ref = ref.detach();
    h->pos = pos.detach();
    h->integral = g->integral;
    return h;
}

// the graph back in reference layout (rows by reference id, tails as reference ids)
vg_graph *vg_remove_layout(vg_ctx *ctx, const vg_graph *g) {
    VG_REQUIRE(g->ref != nullptr, "graph has no layout");
    return move_rows(ctx, g, g->pos, g->ref);
}

// device community vector (positions) -> host reference ids indexed by reference id
void vg_download_comm_ref(vg_ctx *ctx, const vg_graph *g, const int32_t *comm, int64_t *out) {
    const int64_t n = g->nv;
    if (!n) return;
    if (!g->ref) {
        void vg_download_comm(vg_ctx *, const int32_t *, int64_t, int64_t *);
        vg_download_comm(ctx, comm, n, out);
        return;
    }
    DevBuf<int64_t> wide(ctx, n);
    { LaunchTimer lt(ctx);
      k_comm_to_ref<<<vg_grid(ctx, n, 256), 256, 0, ctx->stream>>>(comm, n, g->ref, wide.p); }
    VG_CHECK_LAUNCH();
    VG_CUDA(cudaMemcpyAsync(out, wide.p, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
    vg_sync(ctx);
}

void vg_download_vals_ref(vg_ctx *ctx, const vg_graph *g, const int32_t *x, int64_t *out) {
    const int64_t n = g->nv;
    if (!n) return;
    if (!g->ref) {
        void vg_download_comm(vg_ctx *, const int32_t *, int64_t, int64_t *);
        vg_download_comm(ctx, x, n, out);
        return;
    }
    DevBuf<int64_t> wide(ctx, n);
    { LaunchTimer lt(ctx);
      k_vals_to_ref<<<vg_grid(ctx, n, 256), 256, 0, ctx->stream>>>(x, n, g->ref, wide.p); }
    VG_CHECK_LAUNCH();
    VG_CUDA(cudaMemcpyAsync(out, wide.p, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
    vg_sync(ctx);
}

// reference-ordered device int32 values -> position order in place (values
// renamed through pos when `are_ids`)
void vg_ref_to_pos_inplace(vg_ctx *ctx, const vg_graph *g, int32_t *x, bool are_ids) {
    if (!g->ref || !g->nv) return;
    DevBuf<int32_t> tmp(ctx, g->nv);
    { LaunchTimer lt(ctx);
      k_ref_to_pos<<<vg_grid(ctx, g->nv, 256), 256, 0, ctx->stream>>>(x, g->nv, g->ref,
                                                                       are_ids ? g->pos : nullptr, tmp.p); }
    VG_CHECK_LAUNCH();
    VG_CUDA(cudaMemcpyAsync(x, tmp.p, sizeof(int32_t) * g->nv, cudaMemcpyDeviceToDevice, ctx->stream));
}

extern "C" vg_status vg_graph_reorder(vg_ctx *ctx, vg_graph *g, int32_t mode) {
    if (!ctx || !g) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        VG_REQUIRE(mode == 0 || mode == 1, "layout mode must be 0 (reference order) or 1 (locality)");
        vg_graph *h = nullptr;
        if (mode == 1 && !g->ref) {
            DevBuf<int32_t> order;
            vg_bfs_order(ctx, g, order);
            h = vg_apply_layout(ctx, g, order.p);
        } else if (mode == 0 && g->ref) {
            h = vg_remove_layout(ctx, g);
        }
        if (h) {
            vg_graph_release(ctx, g); // communities and colors of the old layout are dropped
            *g = *h;
            delete h;
        }
        vg_sync(ctx);
    });
}
