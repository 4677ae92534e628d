// distColoringMultiHashMinMax for one rank (coloring.cpp:52-118). Each round of
// distColoringIteration (coloring.cpp:133-247) only compares hashes against
// neighbours that are uncolored or colored in this round, so a round is
// order-independent; here one thread colors one vertex and a round is one launch.
#include "vg_internal.cuh"

namespace {

constexpr int MAX_HASH = 32;

// coloring.cpp:120-131
__host__ __device__ __forceinline__ uint32_t color_hash(uint32_t a, uint32_t seed) {
    a ^= seed;
    a = (a + 0x7ed55d16u) + (a << 12);
    a = (a ^ 0xc761c23cu) + (a >> 19);
    a = (a + 0x165667b1u) + (a << 5);
    a = (a ^ 0xd3a2646cu) + (a << 9);
    a = (a + 0xfd7046c5u) + (a << 3);
    a = (a ^ 0xb55a4f09u) + (a >> 16);
    return a;
}

// one round; colors of this round are >= nextColor, so reading a neighbour
// colored concurrently in this round gives the same decision as reading -1
__global__ void k_color_round(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ tail,
                              int64_t nv, int32_t *__restrict__ color, int nHash, int64_t nextColor,
                              uint32_t seed, unsigned long long *__restrict__ ncolored,
                              const int32_t *__restrict__ ref) {
    unsigned long long mine = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv;
         v += (int64_t)gridDim.x * blockDim.x) {
        if (color[v] != -1) continue;
        // hashes and the color pick use reference ids (v + base of the reference)
        const int64_t rv = vg_rid(ref, (int32_t)v);
        int64_t possible = 2 * (int64_t)nHash;
        uint32_t vHash[MAX_HASH];
        for (int t = 0; t < nHash; t++)
            vHash[t] = color_hash((uint32_t)rv, (uint32_t)((int64_t)seed + 1043 * (int64_t)t));
        uint32_t not_min = 0, not_max = 0;
        bool can_color = true;
        const int64_t e1 = rowptr[v + 1];
        for (int64_t k = rowptr[v]; k < e1; k++) {
            const int32_t u = tail[k];
            if (u == v) continue;
            const int32_t cu = color[u];
            if (cu != -1 && cu < nextColor) continue;
            for (int t = 0; t < nHash; t++) {
                const uint32_t j = color_hash((uint32_t)vg_rid(ref, u),
                                              (uint32_t)((int64_t)seed + 1043 * (int64_t)t));
                if (vHash[t] <= j && !(not_max & (1u << t))) {
                    not_max |= (1u << t);
                    possible--;
                }
                if (vHash[t] >= j && !(not_min & (1u << t))) {
                    not_min |= (1u << t);
                    possible--;
                }
            }
            if (possible == 0) {
                can_color = false;
                break;
            }
        }
        if (can_color) {
            const int64_t col_id = rv % possible;
            int64_t this_col = 0;
            for (int t = 0; t < nHash; t++) {
                if (!(not_min & (1u << t)) && col_id == this_col) {
                    color[v] = (int32_t)(2 * t + nextColor);
                    mine++;
                    break;
                }
                this_col += !(not_min & (1u << t));
                if (!(not_max & (1u << t)) && col_id == this_col) {
                    color[v] = (int32_t)(2 * t + 1 + nextColor);
                    mine++;
                    break;
                }
                this_col += !(not_max & (1u << t));
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(ncolored, mine);
}

__global__ void k_fill_i32(int32_t *__restrict__ x, int64_t n, int32_t val) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        x[i] = val;
}

} // namespace

void vg_download_comm(vg_ctx *ctx, const int32_t *comm, int64_t n, int64_t *out);
void vg_upload_ids(vg_ctx *ctx, const int64_t *in, int64_t n, int64_t lim, int32_t *out);

// returns nextColor; the colors land in g->colors
int64_t vg_color_internal(vg_ctx *ctx, vg_graph *g, int64_t nHash, int32_t target_percent,
                          int32_t single_iteration) {
    VG_REQUIRE(nHash >= 1 && nHash <= MAX_HASH, "number of hash functions must be 1..%d (got %lld)",
               MAX_HASH, (long long)nHash);
    const int64_t nv = g->nv;
    if (!g->colors) g->colors = (int32_t *)vg_alloc(ctx, sizeof(int32_t) * (nv ? nv : 1));
    if (nv) {
        LaunchTimer lt(ctx);
        k_fill_i32<<<vg_grid(ctx, nv, 256), 256, 0, ctx->stream>>>(g->colors, nv, -1);
    }
    VG_CHECK_LAUNCH();
    DevBuf<unsigned long long> cnt(ctx, 1);
    unsigned long long *h = (unsigned long long *)vg_pinned(ctx, sizeof(unsigned long long));
    uint32_t seed = 1012; // coloring.cpp:60
    int64_t nextColor = 0, lastCount = 0, currentCount = 0;
    const int64_t targetCount = (nv * target_percent) / 100;
    bool finished = false;
    while (!finished) {
        VG_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long), ctx->stream));
        if (nv) {
            LaunchTimer lt(ctx);
            k_color_round<<<vg_grid(ctx, nv, 256), 256, 0, ctx->stream>>>(
                g->rowptr, g->tail, nv, g->colors, (int)nHash, nextColor, seed, cnt.p, g->ref);
        }
        VG_CHECK_LAUNCH();
        VG_CUDA(cudaMemcpyAsync(h, cnt.p, sizeof(*h), cudaMemcpyDeviceToHost, ctx->stream));
        vg_sync(ctx);
        currentCount += (int64_t)*h; // countUnassigned (coloring.cpp:468-491)
        finished = single_iteration || currentCount >= targetCount || lastCount == currentCount;
        nextColor += nHash * 2;
        seed = color_hash(seed, 0);
        lastCount = currentCount;
    }
    g->num_colors = nextColor;
    return nextColor;
}

extern "C" vg_status vg_color(vg_ctx *ctx, vg_graph *g, int64_t n_hash, int32_t target_percent,
                              int32_t single_iteration, int64_t *colors_out,
                              int64_t *num_colors_out) {
    if (!ctx || !g) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        const int64_t nc = vg_color_internal(ctx, g, n_hash, target_percent, single_iteration);
        if (num_colors_out) *num_colors_out = nc;
        if (colors_out) vg_download_vals_ref(ctx, g, g->colors, colors_out);
    });
}

extern "C" vg_status vg_set_colors(vg_ctx *ctx, vg_graph *g, const int64_t *colors,
                                   int64_t num_colors) {
    if (!ctx || !g || !colors) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        VG_REQUIRE(num_colors >= 0 && num_colors < INT32_MAX, "bad number of colors");
        if (!g->colors) g->colors = (int32_t *)vg_alloc(ctx, sizeof(int32_t) * (g->nv ? g->nv : 1));
        vg_upload_ids(ctx, colors, g->nv, num_colors + 1, g->colors);
        vg_ref_to_pos_inplace(ctx, g, g->colors, false);
        g->num_colors = num_colors;
    });
}
