// distbuildNextLevelGraph for one rank (rebuild.cpp:77-504) and the graph
// generators (distgraph.cpp:391-983 for the RGG; own designs for BA/ER).
//
// Rebuild: communities are renumbered by first appearance in vertex order
// (distReNumber, rebuild.cpp:122-135) with an atomicMin of the first member,
// a flag and an exclusive scan; every CSR entry becomes a triple
// (new(c(src)), new(c(tail)), w) in CSR order; a stable radix sort on the pair
// and an in-order fold of equal pairs give the next CSR with rows sorted by
// neighbour id and weights summed in the reference's (vertex, edge) order
// (fill_newEdgesMap / send_newEdges, rebuild.cpp:294-478).
#include "vg_internal.cuh"

#include <climits>
#include <cmath>
#include <random>

void vg_upload_ids(vg_ctx *ctx, const int64_t *in, int64_t n, int64_t lim, int32_t *out);

namespace {

__global__ void k_fill_first(int32_t *__restrict__ first, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        first[i] = INT_MAX;
}

__global__ void k_first_member(const int32_t *__restrict__ comm, int64_t nv,
                               int32_t *__restrict__ first) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv;
         i += (int64_t)gridDim.x * blockDim.x)
        atomicMin(&first[comm[i]], (int32_t)i);
}

// per community slot c with members (first[c] set): flag its first member, in the
// order the flags are indexed by
__global__ void k_comm_flag(const int32_t *__restrict__ first, int64_t n, int32_t *__restrict__ flag) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t f = first[c];
        if (f != INT_MAX) flag[f] = 1;
    }
}

// per community slot: its new id, the rank of its first member among the flagged
// ones (in place over first[])
__global__ void k_comm_rank(int32_t *__restrict__ first, int64_t n, const int64_t *__restrict__ rank) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t f = first[c];
        if (f != INT_MAX) first[c] = (int32_t)rank[f];
    }
}

// per vertex: the new id of its community
__global__ void k_new_of(const int32_t *__restrict__ comm, int64_t nv, const int32_t *__restrict__ cid,
                         int32_t *__restrict__ newof) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv;
         i += (int64_t)gridDim.x * blockDim.x)
        newof[i] = cid[comm[i]];
}

// one warp per row: triples in CSR order with coalesced writes
__global__ void k_triples(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ tail,
                          const double *__restrict__ w, int64_t nv,
                          const int32_t *__restrict__ map, int32_t *__restrict__ src,
                          int32_t *__restrict__ dst, double *__restrict__ wo) {
    const int lane = threadIdx.x & 31;
    const int64_t wg = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = wg; v < nv; v += nw) {
        const int32_t s = map ? map[v] : (int32_t)v;
        const int64_t e1 = rowptr[v + 1];
        for (int64_t e = rowptr[v] + lane; e < e1; e += 32) {
            src[e] = s;
            dst[e] = map ? map[tail[e]] : tail[e];
            wo[e] = w[e];
        }
    }
}

} // namespace

// Graph in the library's layout: communities are named by positions. The next
// level's reference numbering is the first appearance in REFERENCE vertex order
// (min reference id of the members); its positions follow the first member's
// position, so the coarse graph keeps the locality of the fine one. Triples are
// emitted in reference vertex order, so equal pairs fold in the reference's order.
namespace {

// both first members of each community: smallest reference id and smallest position
__global__ void k_first_both(const int32_t *__restrict__ comm, int64_t nv,
                             const int32_t *__restrict__ ref, int32_t *__restrict__ first_ref,
                             int32_t *__restrict__ first_pos) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nv;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = comm[p];
        atomicMin(&first_ref[c], ref[p]);
        atomicMin(&first_pos[c], (int32_t)p);
    }
}

// per community slot with members: flag_ref at its first reference id, flag_pos at
// its first position
__global__ void k_comm_flags(const int32_t *__restrict__ first_ref, const int32_t *__restrict__ first_pos,
                             int64_t n, int32_t *__restrict__ flag_ref, int32_t *__restrict__ flag_pos) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t fp = first_pos[c];
        if (fp != INT_MAX) {
            flag_ref[first_ref[c]] = 1;
            flag_pos[fp] = 1;
        }
    }
}

// per community slot with members: its next-level reference id nr and position np
// (in place over first_ref / first_pos), and the next level's ref/pos maps
__global__ void k_comm_ids(int32_t *__restrict__ first_ref, int32_t *__restrict__ first_pos, int64_t n,
                           const int64_t *__restrict__ rank_ref, const int64_t *__restrict__ rank_pos,
                           int32_t *__restrict__ next_ref, int32_t *__restrict__ next_pos) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t fp = first_pos[c];
        if (fp != INT_MAX) {
            const int32_t nr = (int32_t)rank_ref[first_ref[c]];
            const int32_t np = (int32_t)rank_pos[fp];
            first_ref[c] = nr;
            first_pos[c] = np;
            next_ref[np] = nr;
            next_pos[nr] = np;
        }
    }
}

// per vertex: its community's next-level reference id and position
__global__ void k_vertex_ids(const int32_t *__restrict__ comm, int64_t nv,
                             const int32_t *__restrict__ cnr, const int32_t *__restrict__ cnp,
                             int32_t *__restrict__ new_ref, int32_t *__restrict__ new_pos) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nv;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = comm[p];
        new_ref[p] = cnr[c];
        new_pos[p] = cnp[c];
    }
}

} // namespace

vg_graph *vg_aggregate_rows(vg_ctx *ctx, const vg_graph *g, const int32_t *pos,
                            const int32_t *new_row, const int32_t *new_key, int64_t nc,
                            const int32_t *key_to_pos);

vg_graph *vg_rebuild_new(vg_ctx *ctx, const vg_graph *g, const int32_t *comm) {
    const int64_t nv = g->nv;
    const int grid = vg_grid(ctx, nv, 256);
    if (!g->ref) {
        // reference layout: first appearance by position is first appearance by id
        DevBuf<int32_t> first(ctx, nv), flag(ctx, nv), newof(ctx, nv);
        DevBuf<int64_t> rank(ctx, nv);
        int64_t nc = 0;
        if (nv) {
            { LaunchTimer lt(ctx); k_fill_first<<<grid, 256, 0, ctx->stream>>>(first.p, nv); }
            VG_CHECK_LAUNCH();
            { LaunchTimer lt(ctx); k_first_member<<<grid, 256, 0, ctx->stream>>>(comm, nv, first.p); }
            VG_CHECK_LAUNCH();
            VG_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int32_t) * nv, ctx->stream));
            { LaunchTimer lt(ctx); k_comm_flag<<<grid, 256, 0, ctx->stream>>>(first.p, nv, flag.p); }
            VG_CHECK_LAUNCH();
            nc = vg_exclusive_scan_i32_to_i64(ctx, flag.p, rank.p, nv);
            { LaunchTimer lt(ctx); k_comm_rank<<<grid, 256, 0, ctx->stream>>>(first.p, nv, rank.p); }
            VG_CHECK_LAUNCH();
            { LaunchTimer lt(ctx); k_new_of<<<grid, 256, 0, ctx->stream>>>(comm, nv, first.p, newof.p); }
            VG_CHECK_LAUNCH();
        }
        first.release();
        flag.release();
        rank.release();
        vg_graph *h = vg_aggregate_rows(ctx, g, nullptr, newof.p, newof.p, nc, nullptr);
        h->integral = g->integral == 1 ? 1 : -1; // sums of the same integers
        return h;
    }
    DevBuf<int32_t> first_ref(ctx, nv), first_pos(ctx, nv), flag_ref(ctx, nv), flag_pos(ctx, nv);
    DevBuf<int64_t> rank_ref(ctx, nv), rank_pos(ctx, nv);
    DevBuf<int32_t> new_ref(ctx, nv), new_pos(ctx, nv), next_ref(ctx, nv), next_pos(ctx, nv);
    int64_t nc = 0;
    if (nv) {
        { LaunchTimer lt(ctx); k_fill_first<<<grid, 256, 0, ctx->stream>>>(first_ref.p, nv); }
        VG_CHECK_LAUNCH();
        { LaunchTimer lt(ctx); k_fill_first<<<grid, 256, 0, ctx->stream>>>(first_pos.p, nv); }
        VG_CHECK_LAUNCH();
        { LaunchTimer lt(ctx);
          k_first_both<<<grid, 256, 0, ctx->stream>>>(comm, nv, g->ref, first_ref.p, first_pos.p); }
        VG_CHECK_LAUNCH();
        VG_CUDA(cudaMemsetAsync(flag_ref.p, 0, sizeof(int32_t) * nv, ctx->stream));
        VG_CUDA(cudaMemsetAsync(flag_pos.p, 0, sizeof(int32_t) * nv, ctx->stream));
        { LaunchTimer lt(ctx);
          k_comm_flags<<<grid, 256, 0, ctx->stream>>>(first_ref.p, first_pos.p, nv, flag_ref.p,
                                                      flag_pos.p); }
        VG_CHECK_LAUNCH();
        vg_scan_i32_async(ctx, flag_pos.p, rank_pos.p, nv, nullptr);
        nc = vg_exclusive_scan_i32_to_i64(ctx, flag_ref.p, rank_ref.p, nv);
        { LaunchTimer lt(ctx);
          k_comm_ids<<<grid, 256, 0, ctx->stream>>>(first_ref.p, first_pos.p, nv, rank_ref.p,
                                                    rank_pos.p, next_ref.p, next_pos.p); }
        VG_CHECK_LAUNCH();
        { LaunchTimer lt(ctx);
          k_vertex_ids<<<grid, 256, 0, ctx->stream>>>(comm, nv, first_ref.p, first_pos.p, new_ref.p,
                                                      new_pos.p); }
        VG_CHECK_LAUNCH();
    }
    flag_ref.release();
    flag_pos.release();
    rank_ref.release();
    rank_pos.release();
    first_ref.release();
    first_pos.release();
    vg_graph *h = vg_aggregate_rows(ctx, g, g->pos, new_pos.p, new_ref.p, nc, next_pos.p);
    // the arrays were sized nv; the next level keeps its first nc entries
    DevBuf<int32_t> r2(ctx, nc), p2(ctx, nc);
    if (nc) {
        VG_CUDA(cudaMemcpyAsync(r2.p, next_ref.p, sizeof(int32_t) * nc, cudaMemcpyDeviceToDevice, ctx->stream));
        VG_CUDA(cudaMemcpyAsync(p2.p, next_pos.p, sizeof(int32_t) * nc, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    h->ref = r2.detach();
    h->pos = p2.detach();
    h->integral = g->integral == 1 ? 1 : -1; // sums of the same integers
    return h;
}

extern "C" vg_status vg_rebuild(vg_ctx *ctx, vg_graph *g, const int64_t *cvect) {
    if (!ctx || !g) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        DevBuf<int32_t> up;
        const int32_t *comm = g->comm;
        if (cvect) {
            up.alloc(ctx, g->nv);
            vg_upload_ids(ctx, cvect, g->nv, g->nv, up.p);
            vg_ref_to_pos_inplace(ctx, g, up.p, true);
            comm = up.p;
        }
        VG_REQUIRE(comm != nullptr || g->nv == 0, "vg_rebuild: no communities (run a phase first)");
        vg_graph *next = vg_rebuild_new(ctx, g, comm);
        up.release();
        vg_graph_release(ctx, g);
        *g = *next;
        delete next;
        vg_sync(ctx);
    });
}

// ---------------------------------------------------------------------------------
// generators

namespace {

constexpr int64_t MLCG = 2147483647LL; // utils.hpp:79
constexpr int64_t ALCG = 16807LL;      // utils.hpp:80

__device__ __forceinline__ int64_t mulmod(int64_t a, int64_t b) { return (a * b) % MLCG; }

// x_k of LCG::generate for one rank (utils.hpp:248-298) by jump-ahead:
// x_0 = reseeder(seed), x_k = x_0 * 16807^k mod (2^31 - 1)
__global__ void k_lcg_points(int64_t count, int64_t x0, double mult, double *__restrict__ X) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < count;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t x;
        if (k == 0) {
            x = x0;
        } else {
            int64_t r = 1, b = ALCG, e = k;
            while (e) {
                if (e & 1) r = mulmod(r, b);
                b = mulmod(b, b);
                e >>= 1;
            }
            x = mulmod(x0 % MLCG, r);
        }
        X[k] = __dmul_rn(fabs((double)x), mult);
    }
}

__global__ void k_minmax(const double *__restrict__ X, int64_t n, double *__restrict__ out) {
    // out: [xmin, xmax, ymin, ymax] partial per block -> final on host
    double xmn = INFINITY, xmx = -INFINITY, ymn = INFINITY, ymx = -INFINITY;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double x = X[i], y = X[n + i];
        xmn = fmin(xmn, x);
        xmx = fmax(xmx, x);
        ymn = fmin(ymn, y);
        ymx = fmax(ymx, y);
    }
    for (int o = 16; o > 0; o >>= 1) {
        xmn = fmin(xmn, __shfl_down_sync(0xffffffffu, xmn, o));
        xmx = fmax(xmx, __shfl_down_sync(0xffffffffu, xmx, o));
        ymn = fmin(ymn, __shfl_down_sync(0xffffffffu, ymn, o));
        ymx = fmax(ymx, __shfl_down_sync(0xffffffffu, ymx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        const int64_t slot = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
        out[4 * slot + 0] = xmn;
        out[4 * slot + 1] = xmx;
        out[4 * slot + 2] = ymn;
        out[4 * slot + 3] = ymx;
    }
}

struct Grid {
    double xmin, ymin, sx, sy;
    int64_t ncx, ncy;
};

__device__ __forceinline__ int64_t cell_of(const Grid &gr, double x, double y, int64_t *cx,
                                           int64_t *cy) {
    int64_t a = (int64_t)(__dmul_rn(__dsub_rn(x, gr.xmin), gr.sx));
    int64_t b = (int64_t)(__dmul_rn(__dsub_rn(y, gr.ymin), gr.sy));
    if (a >= gr.ncx) a = gr.ncx - 1;
    if (b >= gr.ncy) b = gr.ncy - 1;
    *cx = a;
    *cy = b;
    return b * gr.ncx + a;
}

__global__ void k_cells(const double *__restrict__ X, int64_t n, Grid gr, int32_t *__restrict__ cell,
                        int32_t *__restrict__ ccount) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t cx, cy;
        const int64_t c = cell_of(gr, X[i], X[n + i], &cx, &cy);
        cell[i] = (int32_t)c;
        atomicAdd(&ccount[c], 1);
    }
}

__global__ void k_cell_scatter(const int32_t *__restrict__ cell, int64_t n,
                               const int64_t *__restrict__ cstart, int32_t *__restrict__ cfill,
                               int32_t *__restrict__ order) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = cell[i];
        order[cstart[c] + atomicAdd(&cfill[c], 1)] = (int32_t)i;
    }
}

// distance of the pair as the reference computes it for i < j (distgraph.cpp:537-539)
__device__ __forceinline__ double pair_distance(const double *__restrict__ X, int64_t n, int64_t i,
                                                int64_t j) {
    const int64_t a = i < j ? i : j, b = i < j ? j : i;
    const double dx = __dsub_rn(X[a], X[b]);
    const double dy = __dsub_rn(X[n + a], X[n + b]);
    return __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
}

// pass 0 counts the neighbours of every point, pass 1 writes them and sorts the row
template <int PASS>
__global__ void k_rgg_rows(const double *__restrict__ X, int64_t n, Grid gr, double rn,
                           const int64_t *__restrict__ cstart, const int32_t *__restrict__ order,
                           const int32_t *__restrict__ cell, int64_t *__restrict__ deg_or_rowptr,
                           int32_t *__restrict__ tail, double *__restrict__ w) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = cell[i];
        const int64_t cx = c % gr.ncx, cy = c / gr.ncx;
        int64_t cnt = 0;
        const int64_t base = PASS ? deg_or_rowptr[i] : 0;
        for (int64_t ny = cy - 1; ny <= cy + 1; ny++) {
            if (ny < 0 || ny >= gr.ncy) continue;
            for (int64_t nx = cx - 1; nx <= cx + 1; nx++) {
                if (nx < 0 || nx >= gr.ncx) continue;
                const int64_t cc = ny * gr.ncx + nx;
                for (int64_t k = cstart[cc]; k < cstart[cc + 1]; k++) {
                    const int64_t j = order[k];
                    if (j == i) continue;
                    const double ed = pair_distance(X, n, i, j);
                    if (ed <= rn) {
                        if (PASS) {
                            // insertion into the sorted row
                            int64_t p = base + cnt;
                            while (p > base && tail[p - 1] > (int32_t)j) {
                                tail[p] = tail[p - 1];
                                w[p] = w[p - 1];
                                p--;
                            }
                            tail[p] = (int32_t)j;
                            w[p] = ed;
                        }
                        cnt++;
                    }
                }
            }
        }
        if (!PASS) deg_or_rowptr[i] = cnt;
    }
}

__device__ __forceinline__ uint64_t pair_key(int64_t i, int64_t j, int64_t n) {
    const int64_t a = i < j ? i : j, b = i < j ? j : i;
    return (uint64_t)a * (uint64_t)n + (uint64_t)b;
}

__device__ bool row_has(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ tail,
                        int64_t i, int32_t j) {
    int64_t lo = rowptr[i], hi = rowptr[i + 1];
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        const int32_t t = tail[mid];
        if (t == j) return true;
        if (t < j) lo = mid + 1;
        else hi = mid;
    }
    return false;
}

constexpr uint64_t NO_KEY = ~0ULL;

// candidate extra edges (streams 1, 2, 3 of the counter-based generator)
__global__ void k_extra_candidates(int64_t nrande, int64_t n, uint64_t seed,
                                   const int64_t *__restrict__ rowptr,
                                   const int32_t *__restrict__ tail, uint64_t *__restrict__ keys,
                                   uint32_t *__restrict__ vals) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nrande;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = (int64_t)vg_uint_below(vg_mix(seed, 1, (uint64_t)k), (uint64_t)n);
        const int64_t j = (int64_t)vg_uint_below(vg_mix(seed, 2, (uint64_t)k), (uint64_t)n);
        uint64_t key = NO_KEY;
        if (i != j && !row_has(rowptr, tail, i, (int32_t)j)) key = pair_key(i, j, n);
        keys[k] = key;
        vals[k] = (uint32_t)k;
    }
}

// Barabasi-Albert edge targets (own design; hash-resolved Batagelj-Brandes copy model)
__global__ void k_ba_edges(int64_t ecount, int64_t m, int64_t n, uint64_t seed,
                           uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ecount;
         e += (int64_t)gridDim.x * blockDim.x) {
        uint64_t pos = 2 * (uint64_t)e + 1;
        int64_t dst;
        for (;;) {
            const uint64_t r = vg_uint_below(vg_mix(seed, 11, pos), pos);
            if ((r & 1) == 0) {
                dst = (int64_t)((r / 2) / (uint64_t)m);
                break;
            }
            pos = r;
        }
        const int64_t src = e / m;
        keys[e] = src == dst ? NO_KEY : pair_key(src, dst, n);
        vals[e] = (uint32_t)e;
    }
}

// Erdos-Renyi G(n, M) candidates (own design, streams 21/22)
__global__ void k_er_edges(int64_t M, int64_t n, uint64_t seed, uint64_t *__restrict__ keys,
                           uint32_t *__restrict__ vals) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < M;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = (int64_t)vg_uint_below(vg_mix(seed, 21, (uint64_t)c), (uint64_t)n);
        const int64_t j = (int64_t)vg_uint_below(vg_mix(seed, 22, (uint64_t)c), (uint64_t)n);
        keys[c] = i == j ? NO_KEY : pair_key(i, j, n);
        vals[c] = (uint32_t)c;
    }
}

__global__ void k_unique_heads(const uint64_t *__restrict__ keys, int64_t m,
                               int32_t *__restrict__ head) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x)
        head[i] = (keys[i] != NO_KEY && (i == 0 || keys[i] != keys[i - 1])) ? 1 : 0;
}

// both directions of every kept pair, appended after `base` entries
__global__ void k_pairs_to_triples(const uint64_t *__restrict__ keys,
                                   const uint32_t *__restrict__ vals,
                                   const int32_t *__restrict__ head, const int64_t *__restrict__ pos,
                                   int64_t m, int64_t n, int wmode, uint64_t seed, int64_t base,
                                   int32_t *__restrict__ src, int32_t *__restrict__ dst,
                                   double *__restrict__ w) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (!head[i]) continue;
        const uint64_t k = keys[i];
        const int32_t a = (int32_t)(k / (uint64_t)n), b = (int32_t)(k % (uint64_t)n);
        const double wt = wmode == 0 ? 1.0 : vg_unit_double(vg_mix(seed, 3, vals[i]));
        const int64_t o = base + 2 * pos[i];
        src[o] = a;
        dst[o] = b;
        w[o] = wt;
        src[o + 1] = b;
        dst[o + 1] = a;
        w[o + 1] = wt;
    }
}

__global__ void k_reweight(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ tail,
                           double *__restrict__ w, int64_t nv, int mode, uint64_t seed) {
    const int lane = threadIdx.x & 31;
    const int64_t wg = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = wg; v < nv; v += nw) {
        const int64_t e1 = rowptr[v + 1];
        for (int64_t e = rowptr[v] + lane; e < e1; e += 32)
            w[e] = mode == 1 ? 1.0 : vg_unit_double(vg_mix(seed, 31, pair_key(v, tail[e], nv)));
    }
}

// pair keys a*n+b (a<b) are below n*n, and NO_KEY's low bits exceed them all
int key_bits(int64_t n) {
    int b = 1;
    while (b < 63 && ((unsigned long long)1 << b) < (unsigned long long)n * (unsigned long long)n) b++;
    return b;
}

// sort candidate pair keys (stable by candidate index) and emit both directions
// of the first occurrence of every pair after the `base` existing triples
int64_t pairs_to_triples(vg_ctx *ctx, DevBuf<uint64_t> &keys, DevBuf<uint32_t> &vals, int64_t m,
                         int64_t n, int wmode, uint64_t seed, DevBuf<int32_t> &src,
                         DevBuf<int32_t> &dst, DevBuf<double> &w, int64_t base) {
    if (m == 0) return 0;
    vg_radix_sort_pairs(ctx, keys.p, vals.p, m, key_bits(n));
    DevBuf<int32_t> head(ctx, m);
    DevBuf<int64_t> pos(ctx, m);
    { LaunchTimer lt(ctx); k_unique_heads<<<vg_grid(ctx, m, 256), 256, 0, ctx->stream>>>(keys.p, m, head.p); }
    VG_CHECK_LAUNCH();
    const int64_t u = vg_exclusive_scan_i32_to_i64(ctx, head.p, pos.p, m);
    // grow the triple arrays to hold base + 2u entries
    DevBuf<int32_t> s2(ctx, base + 2 * u), d2(ctx, base + 2 * u);
    DevBuf<double> w2(ctx, base + 2 * u);
    if (base) {
        VG_CUDA(cudaMemcpyAsync(s2.p, src.p, sizeof(int32_t) * base, cudaMemcpyDeviceToDevice, ctx->stream));
        VG_CUDA(cudaMemcpyAsync(d2.p, dst.p, sizeof(int32_t) * base, cudaMemcpyDeviceToDevice, ctx->stream));
        VG_CUDA(cudaMemcpyAsync(w2.p, w.p, sizeof(double) * base, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    { LaunchTimer lt(ctx);
      k_pairs_to_triples<<<vg_grid(ctx, m, 256), 256, 0, ctx->stream>>>(
          keys.p, vals.p, head.p, pos.p, m, n, wmode, seed, base, s2.p, d2.p, w2.p); }
    VG_CHECK_LAUNCH();
    src = std::move(s2);
    dst = std::move(d2);
    w = std::move(w2);
    return u;
}

} // namespace

static int64_t lcg_x0(uint32_t seed) {
    // LCG::reseeder (utils.hpp:163-170): the first word of std::seed_seq({seed})
    std::seed_seq seq({seed});
    std::vector<uint32_t> s(1);
    seq.generate(s.begin(), s.end());
    return (int64_t)s[0];
}

static double rgg_radius(int64_t nv) {
    // generateInMemGraph (distgraph.cpp:395-399); PI as distgraph.hpp:65
    const double PI_ = 3.14159;
    double rc = std::sqrt((double)std::log((double)nv) / (double)(PI_ * (double)nv));
    double rt = std::sqrt((double)2.0736 / (double)nv);
    return (rc + rt) / (double)2.0;
}

extern "C" vg_status vg_generate_rgg(vg_ctx *ctx, int64_t n, double extra_percent, uint64_t seed,
                                     vg_graph **out) {
    if (!ctx || !out) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        *out = nullptr;
        VG_REQUIRE(n >= 2 && n < (int64_t)INT32_MAX, "RGG size must be in [2, 2^31)");
        VG_CUDA(cudaSetDevice(ctx->device));
        const double rn = rgg_radius(n);
        VG_REQUIRE(1.0 > rn, "r(n) must be below 1/nprocs (distgraph.cpp:401)");
        const double mult = 1.0 / (double)(1.0 + (double)(MLCG - 1));
        DevBuf<double> X(ctx, 2 * n);
        { LaunchTimer lt(ctx);
          k_lcg_points<<<vg_grid(ctx, 2 * n, 256), 256, 0, ctx->stream>>>(2 * n, lcg_x0(1), mult, X.p); }
        VG_CHECK_LAUNCH();
        // grid: same construction as the restatement (cells wider than r(n))
        const int mblocks = 64;
        DevBuf<double> mm(ctx, 4 * mblocks * 8);
        { LaunchTimer lt(ctx); k_minmax<<<mblocks, 256, 0, ctx->stream>>>(X.p, n, mm.p); }
        VG_CHECK_LAUNCH();
        std::vector<double> hm(4 * mblocks * 8);
        VG_CUDA(cudaMemcpyAsync(hm.data(), mm.p, sizeof(double) * hm.size(), cudaMemcpyDeviceToHost,
                                ctx->stream));
        vg_sync(ctx);
        double xmin = INFINITY, xmax = -INFINITY, ymin = INFINITY, ymax = -INFINITY;
        for (size_t s = 0; s < hm.size() / 4; s++) {
            xmin = std::fmin(xmin, hm[4 * s]);
            xmax = std::fmax(xmax, hm[4 * s + 1]);
            ymin = std::fmin(ymin, hm[4 * s + 2]);
            ymax = std::fmax(ymax, hm[4 * s + 3]);
        }
        const double cwid = rn * (1.0 + 1e-9);
        Grid gr;
        gr.ncx = (int64_t)std::floor((xmax - xmin) / cwid) + 1;
        gr.ncy = (int64_t)std::floor((ymax - ymin) / cwid) + 1;
        if (gr.ncx > 32768) gr.ncx = 32768;
        if (gr.ncy > 32768) gr.ncy = 32768;
        gr.sx = (double)gr.ncx / ((xmax - xmin) + cwid);
        gr.sy = (double)gr.ncy / ((ymax - ymin) + cwid);
        gr.xmin = xmin;
        gr.ymin = ymin;
        const int64_t ncell = gr.ncx * gr.ncy;
        DevBuf<int32_t> cell(ctx, n), ccount(ctx, ncell), order(ctx, n);
        DevBuf<int64_t> cstart(ctx, ncell + 1);
        VG_CUDA(cudaMemsetAsync(ccount.p, 0, sizeof(int32_t) * ncell, ctx->stream));
        const int grid = vg_grid(ctx, n, 256);
        { LaunchTimer lt(ctx); k_cells<<<grid, 256, 0, ctx->stream>>>(X.p, n, gr, cell.p, ccount.p); }
        VG_CHECK_LAUNCH();
        VG_CUDA(cudaMemsetAsync(cstart.p + ncell, 0, sizeof(int64_t), ctx->stream));
        vg_scan_i32_async(ctx, ccount.p, cstart.p, ncell, nullptr);
        {
            // cstart[ncell] = n
            VG_CUDA(cudaMemcpyAsync(cstart.p + ncell, &n, sizeof(int64_t), cudaMemcpyHostToDevice,
                                    ctx->stream));
        }
        VG_CUDA(cudaMemsetAsync(ccount.p, 0, sizeof(int32_t) * ncell, ctx->stream));
        { LaunchTimer lt(ctx);
          k_cell_scatter<<<grid, 256, 0, ctx->stream>>>(cell.p, n, cstart.p, ccount.p, order.p); }
        VG_CHECK_LAUNCH();
        ccount.release();
        DevBuf<int64_t> rowptr(ctx, n + 1);
        VG_CUDA(cudaMemsetAsync(rowptr.p + n, 0, sizeof(int64_t), ctx->stream));
        { LaunchTimer lt(ctx);
          k_rgg_rows<0><<<grid, 256, 0, ctx->stream>>>(X.p, n, gr, rn, cstart.p, order.p, cell.p,
                                                       rowptr.p, nullptr, nullptr); }
        VG_CHECK_LAUNCH();
        const int64_t ne = vg_exclusive_scan_i64(ctx, rowptr.p, n + 1);
        DevBuf<int32_t> tail(ctx, ne);
        DevBuf<double> w(ctx, ne);
        { LaunchTimer lt(ctx);
          k_rgg_rows<1><<<grid, 256, 0, ctx->stream>>>(X.p, n, gr, rn, cstart.p, order.p, cell.p,
                                                       rowptr.p, tail.p, w.p); }
        VG_CHECK_LAUNCH();
        vg_sync(ctx);
        vg_graph *g = vg_graph_wrap(ctx, n, ne, rowptr.detach(), tail.detach(), w.detach());
        if (extra_percent > 0.0) {
            // count as distgraph.cpp:703-706: percent of the undirected edges
            const int64_t nrande = ((int64_t)(extra_percent * (double)(ne / 2))) / 100;
            DevBuf<uint64_t> keys(ctx, nrande);
            DevBuf<uint32_t> vals(ctx, nrande);
            if (nrande) {
                LaunchTimer lt(ctx);
                k_extra_candidates<<<vg_grid(ctx, nrande, 256), 256, 0, ctx->stream>>>(
                    nrande, n, seed, g->rowptr, g->tail, keys.p, vals.p);
            }
            VG_CHECK_LAUNCH();
            DevBuf<int32_t> src(ctx, ne), dst(ctx, ne);
            DevBuf<double> ww(ctx, ne);
            if (ne) {
                LaunchTimer lt(ctx);
                k_triples<<<vg_grid(ctx, n * 32, 256), 256, 0, ctx->stream>>>(
                    g->rowptr, g->tail, g->weight, n, nullptr, src.p, dst.p, ww.p);
            }
            VG_CHECK_LAUNCH();
            const int64_t added = pairs_to_triples(ctx, keys, vals, nrande, n, 1, seed, src, dst, ww, ne);
            keys.release();
            vals.release();
            vg_graph_release(ctx, g);
            delete g;
            g = vg_csr_from_triples(ctx, n, src, dst, ww, ne + 2 * added, false);
        }
        vg_sync(ctx);
        *out = g;
    });
}

static vg_graph *pairs_graph(vg_ctx *ctx, int64_t n, DevBuf<uint64_t> &keys, DevBuf<uint32_t> &vals,
                             int64_t m) {
    DevBuf<int32_t> src, dst;
    DevBuf<double> w;
    const int64_t u = pairs_to_triples(ctx, keys, vals, m, n, 0, 0, src, dst, w, 0);
    keys.release();
    vals.release();
    return vg_csr_from_triples(ctx, n, src, dst, w, 2 * u, false);
}

extern "C" vg_status vg_generate_ba(vg_ctx *ctx, int64_t n, int64_t m, uint64_t seed, vg_graph **out) {
    if (!ctx || !out) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        *out = nullptr;
        VG_REQUIRE(n >= 2 && n < (int64_t)INT32_MAX && m >= 1, "bad BA parameters");
        VG_REQUIRE(n * m < (int64_t)UINT32_MAX, "too many BA edges for one sort");
        VG_CUDA(cudaSetDevice(ctx->device));
        const int64_t ecount = n * m;
        DevBuf<uint64_t> keys(ctx, ecount);
        DevBuf<uint32_t> vals(ctx, ecount);
        { LaunchTimer lt(ctx);
          k_ba_edges<<<vg_grid(ctx, ecount, 256), 256, 0, ctx->stream>>>(ecount, m, n, seed, keys.p, vals.p); }
        VG_CHECK_LAUNCH();
        *out = pairs_graph(ctx, n, keys, vals, ecount);
        vg_sync(ctx);
    });
}

extern "C" vg_status vg_generate_er(vg_ctx *ctx, int64_t n, double avg_degree, uint64_t seed,
                                    vg_graph **out) {
    if (!ctx || !out) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        *out = nullptr;
        VG_REQUIRE(n >= 2 && n < (int64_t)INT32_MAX && avg_degree > 0, "bad ER parameters");
        VG_CUDA(cudaSetDevice(ctx->device));
        const int64_t M = (int64_t)std::llround(avg_degree * (double)n / 2.0);
        VG_REQUIRE(M < (int64_t)UINT32_MAX, "too many ER edges for one sort");
        DevBuf<uint64_t> keys(ctx, M);
        DevBuf<uint32_t> vals(ctx, M);
        { LaunchTimer lt(ctx);
          k_er_edges<<<vg_grid(ctx, M, 256), 256, 0, ctx->stream>>>(M, n, seed, keys.p, vals.p); }
        VG_CHECK_LAUNCH();
        *out = pairs_graph(ctx, n, keys, vals, M);
        vg_sync(ctx);
    });
}

extern "C" vg_status vg_graph_reweight(vg_ctx *ctx, vg_graph *g, int32_t mode, uint64_t seed) {
    if (!ctx || !g) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        VG_REQUIRE(mode == 1 || mode == 2, "reweight mode must be 1 (unit) or 2 (U(0,1))");
        VG_CUDA(cudaSetDevice(ctx->device));
        if (g->ne) {
            LaunchTimer lt(ctx);
            k_reweight<<<vg_grid(ctx, g->nv * 32, 256), 256, 0, ctx->stream>>>(g->rowptr, g->tail,
                                                                               g->weight, g->nv, mode, seed);
        }
        VG_CHECK_LAUNCH();
        g->integral = -1; // the weights changed
        vg_sync(ctx);
    });
}
