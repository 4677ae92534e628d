// Device primitives: exclusive scans, a stable LSD radix sort of (key, payload)
// pairs, a deterministic FP64 sum, and CSR assembly from (src, dst, w) triples.
// All are written for this library (no CUB/Thrust); tiles are 2048 elements so
// every kernel streams HBM with coalesced accesses.
#include "vg_internal.cuh"

namespace {

constexpr int SCAN_BLOCK = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;
constexpr int SCAN_ONE = 1024;                     // threads of the single-CTA scan
constexpr int64_t SCAN_ONE_MAX = 4LL * SCAN_ONE * SCAN_ITEMS; // single-CTA below this

// exclusive block scan of one int64 per thread; returns the block total in *total.
// Ends with a barrier, so a block may call it again in a loop.
template <int NT>
__device__ int64_t block_exclusive_scan(int64_t v, int64_t *total) {
    __shared__ int64_t warp_sums[NT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int64_t s = lane < NT / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < NT / 32) warp_sums[lane] = s;
    }
    __syncthreads();
    const int64_t warp_prefix = warp ? warp_sums[warp - 1] : 0;
    *total = warp_sums[NT / 32 - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

// per-tile sums: part[t] = sum of tile t
template <class TIn>
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_reduce(const TIn *__restrict__ in, int64_t n,
                                                            int64_t *__restrict__ part) {
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    int64_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        const int64_t i = base + (int64_t)k * SCAN_BLOCK + threadIdx.x;
        if (i < n) s += (int64_t)in[i];
    }
    int64_t total;
    block_exclusive_scan<SCAN_BLOCK>(s, &total);
    if (threadIdx.x == 0) part[blockIdx.x] = total;
}

// One CTA scans all n elements in chunks of SCAN_ONE * SCAN_ITEMS, carrying the
// running sum; *total (when not null) gets the sum of all n. in may equal out:
// every thread reads its items before it writes them and owns them alone.
template <class TIn>
__global__ void __launch_bounds__(SCAN_ONE) k_scan_one(const TIn *in, int64_t *out, int64_t n,
                                                      int64_t *total) {
    int64_t carry = 0;
    for (int64_t base = 0; base < n; base += (int64_t)SCAN_ONE * SCAN_ITEMS) {
        const int64_t b = base + (int64_t)threadIdx.x * SCAN_ITEMS;
        int64_t v[SCAN_ITEMS];
        int64_t s = 0;
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; k++) {
            v[k] = b + k < n ? (int64_t)in[b + k] : 0;
            s += v[k];
        }
        int64_t tot;
        int64_t run = block_exclusive_scan<SCAN_ONE>(s, &tot) + carry;
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; k++) {
            if (b + k < n) out[b + k] = run;
            run += v[k];
        }
        carry += tot;
    }
    if (total && threadIdx.x == 0) *total = carry;
}

// down sweep of tile t from its exclusive prefix part[t]; in may equal out (as above)
template <class TIn>
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_down(const TIn *in, int64_t *out, int64_t n,
                                                          const int64_t *__restrict__ part) {
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int64_t v[SCAN_ITEMS];
    int64_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        const int64_t i = base + k;
        v[k] = i < n ? (int64_t)in[i] : 0;
        s += v[k];
    }
    int64_t total;
    int64_t run = block_exclusive_scan<SCAN_BLOCK>(s, &total) + part[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        const int64_t i = base + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
}

// Small inputs: one launch. Larger: tile sums, one CTA scans them (and writes the
// total), then the down sweep: three launches, no host round trip.
template <class TIn>
void scan_async(vg_ctx *ctx, const TIn *in, int64_t *out, int64_t n, int64_t *dev_total) {
    if (n <= SCAN_ONE_MAX) {
        LaunchTimer lt(ctx);
        k_scan_one<TIn><<<1, SCAN_ONE, 0, ctx->stream>>>(in, out, n, dev_total);
        VG_CHECK_LAUNCH();
        return;
    }
    const int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    DevBuf<int64_t> part(ctx, tiles);
    {
        LaunchTimer lt(ctx);
        k_scan_reduce<TIn><<<(unsigned)tiles, SCAN_BLOCK, 0, ctx->stream>>>(in, n, part.p);
    }
    VG_CHECK_LAUNCH();
    {
        LaunchTimer lt(ctx);
        k_scan_one<int64_t><<<1, SCAN_ONE, 0, ctx->stream>>>(part.p, part.p, tiles, dev_total);
    }
    VG_CHECK_LAUNCH();
    {
        LaunchTimer lt(ctx);
        k_scan_down<TIn><<<(unsigned)tiles, SCAN_BLOCK, 0, ctx->stream>>>(in, out, n, part.p);
    }
    VG_CHECK_LAUNCH();
}

template <class TIn>
int64_t scan_total(vg_ctx *ctx, const TIn *in, int64_t *out, int64_t n) {
    if (n <= 0) return 0;
    DevBuf<int64_t> tot(ctx, 1);
    scan_async<TIn>(ctx, in, out, n, tot.p);
    int64_t *h = (int64_t *)vg_pinned(ctx, sizeof(int64_t));
    VG_CUDA(cudaMemcpyAsync(h, tot.p, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    vg_sync(ctx);
    return *h;
}

} // namespace

int64_t vg_exclusive_scan_i64(vg_ctx *ctx, int64_t *data, int64_t n) {
    return scan_total<int64_t>(ctx, data, data, n);
}

int64_t vg_exclusive_scan_i32_to_i64(vg_ctx *ctx, const int32_t *in, int64_t *out, int64_t n) {
    return scan_total<int32_t>(ctx, in, out, n);
}

void vg_scan_i64_async(vg_ctx *ctx, int64_t *data, int64_t n, int64_t *dev_total) {
    if (n > 0) scan_async<int64_t>(ctx, data, data, n, dev_total);
}

void vg_scan_i32_async(vg_ctx *ctx, const int32_t *in, int64_t *out, int64_t n,
                       int64_t *dev_total) {
    if (n > 0) scan_async<int32_t>(ctx, in, out, n, dev_total);
}
// ---------------------------------------------------------------------------------
// stable LSD radix sort, 8-bit digits
//
// One pass = a per-tile digit histogram, a scan of the (digit, tile) counts, and a
// scatter. A tile is RS_TILE consecutive elements; each of its warps ranks its own
// run of 32 * RS_ROUNDS elements in order (32 elements per round, equal digits ranked
// by lane through match_any), so the tile-local order of equal digits is the input
// order and the sort is stable. The scatter first places the tile in digit order in
// shared memory and then writes it out with consecutive threads on consecutive
// elements, so each digit's run leaves the tile as whole coalesced stores instead of
// one partial sector per element.

namespace {

constexpr int RS_BLOCK = 256;
constexpr int RS_WARPS = RS_BLOCK / 32;
constexpr int RS_ROUNDS = 16; // rounds of 32 elements per warp
constexpr int RS_TILE = RS_BLOCK * RS_ROUNDS;

__global__ void k_radix_hist(const uint64_t *__restrict__ keys, int64_t n, int shift,
                             int32_t *__restrict__ counts, int64_t ntiles) {
    __shared__ int32_t hist[256];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * RS_TILE;
#pragma unroll 4
    for (int r = 0; r < RS_ROUNDS; r++) {
        const int64_t i = base + (int64_t)r * RS_BLOCK + threadIdx.x;
        if (i < n) atomicAdd(&hist[(keys[i] >> shift) & 0xff], 1);
    }
    __syncthreads();
    counts[(int64_t)threadIdx.x * ntiles + blockIdx.x] = hist[threadIdx.x];
}

struct RadixSmem {
    uint64_t sk[RS_TILE];
    uint32_t sv[RS_TILE];
    int32_t warp_cnt[RS_WARPS][256]; // per warp: digit counts, then exclusive prefix over warps
    int64_t digit_base[256];         // where the tile's run of each digit starts in the output
    int32_t tile_start[256];         // where it starts inside the tile's sorted order
    int32_t wsum[RS_WARPS];
};

__global__ void __launch_bounds__(RS_BLOCK) k_radix_scatter(
    const uint64_t *__restrict__ kin, const uint32_t *__restrict__ vin, uint64_t *__restrict__ kout,
    uint32_t *__restrict__ vout, int64_t n, int shift, const int64_t *__restrict__ offsets,
    int64_t ntiles) {
    extern __shared__ unsigned char rs_raw[];
    RadixSmem &S = *reinterpret_cast<RadixSmem *>(rs_raw);
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int64_t tile0 = (int64_t)blockIdx.x * RS_TILE;
    const int64_t base = tile0 + (int64_t)warp * (32 * RS_ROUNDS);
    for (int d = lane; d < 256; d += 32) S.warp_cnt[warp][d] = 0;
    S.digit_base[threadIdx.x] = offsets[(int64_t)threadIdx.x * ntiles + blockIdx.x];
    __syncwarp();
    // 1. each warp ranks its run: loc = earlier elements of the run with the same
    // digit; the run goes to shared memory in input order meanwhile
    int loc[RS_ROUNDS];
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; r++) {
        const int64_t i = base + r * 32 + lane;
        const bool valid = i < n;
        const uint64_t k = valid ? kin[i] : 0;
        const int d = valid ? (int)((k >> shift) & 0xff) : 256 + lane;
        const unsigned peers = __match_any_sync(full, d);
        const int before = valid ? S.warp_cnt[warp][d] : 0;
        loc[r] = before + __popc(peers & lt_mask);
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) S.warp_cnt[warp][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // 2. thread t owns digit t: exclusive prefix over the warps, then over the digits
    int32_t run = 0;
    for (int w = 0; w < RS_WARPS; w++) {
        const int32_t c = S.warp_cnt[w][threadIdx.x];
        S.warp_cnt[w][threadIdx.x] = run;
        run += c;
    }
    int32_t incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(full, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) S.wsum[warp] = incl;
    __syncthreads();
    int32_t wpre = 0;
    for (int w = 0; w < warp; w++) wpre += S.wsum[w];
    S.tile_start[threadIdx.x] = wpre + incl - run;
    __syncthreads();
    // 3. the tile in digit order, in shared memory (keys re-read: they are in L1/L2)
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; r++) {
        const int64_t i = base + r * 32 + lane;
        if (i < n) {
            const uint64_t k = kin[i];
            const int d = (int)((k >> shift) & 0xff);
            const int sp = S.tile_start[d] + S.warp_cnt[warp][d] + loc[r];
            S.sk[sp] = k;
            S.sv[sp] = vin[i];
        }
    }
    __syncthreads();
    // 4. out in order: consecutive threads write consecutive elements of a digit's run
    const int cnt = (int)min((int64_t)RS_TILE, n - tile0);
    for (int sp = threadIdx.x; sp < cnt; sp += RS_BLOCK) {
        const uint64_t kk = S.sk[sp];
        const int d = (int)((kk >> shift) & 0xff);
        const int64_t dst = S.digit_base[d] + (sp - S.tile_start[d]);
        kout[dst] = kk;
        vout[dst] = S.sv[sp];
    }
}

} // namespace

void vg_radix_sort_pairs(vg_ctx *ctx, uint64_t *keys, uint32_t *vals, int64_t n, int bits) {
    if (n <= 1 || bits <= 0) return;
    static bool configured = false;
    if (!configured) {
        VG_CUDA(cudaFuncSetAttribute(k_radix_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(RadixSmem)));
        configured = true;
    }
    const int64_t ntiles = (n + RS_TILE - 1) / RS_TILE;
    DevBuf<uint64_t> k2(ctx, n);
    DevBuf<uint32_t> v2(ctx, n);
    DevBuf<int32_t> counts(ctx, 256 * ntiles);
    DevBuf<int64_t> offsets(ctx, 256 * ntiles);
    uint64_t *ka = keys, *kb = k2.p;
    uint32_t *va = vals, *vb = v2.p;
    int passes = 0;
    for (int shift = 0; shift < bits; shift += 8) {
        {
            LaunchTimer lt(ctx);
            k_radix_hist<<<(unsigned)ntiles, RS_BLOCK, 0, ctx->stream>>>(ka, n, shift, counts.p,
                                                                          ntiles);
        }
        VG_CHECK_LAUNCH();
        vg_scan_i32_async(ctx, counts.p, offsets.p, 256 * ntiles, nullptr);
        {
            LaunchTimer lt(ctx);
            k_radix_scatter<<<(unsigned)ntiles, RS_BLOCK, sizeof(RadixSmem), ctx->stream>>>(
                ka, va, kb, vb, n, shift, offsets.p, ntiles);
        }
        VG_CHECK_LAUNCH();
        std::swap(ka, kb);
        std::swap(va, vb);
        passes++;
    }
    if (passes & 1) {
        VG_CUDA(cudaMemcpyAsync(keys, ka, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice,
                                ctx->stream));
        VG_CUDA(cudaMemcpyAsync(vals, va, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice,
                                ctx->stream));
    }
}

// ---------------------------------------------------------------------------------
// deterministic FP64 sum: fixed grid of per-block partials, then one block

namespace {

__device__ double block_sum_f64(double v) {
    __shared__ double ws[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) ws[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (warp == 0) {
        s = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s = __dadd_rn(s, __shfl_down_sync(0xffffffffu, s, o));
    }
    __syncthreads();
    return s;
}

__global__ void k_sum_part(const double *__restrict__ x, int64_t n, double *__restrict__ part) {
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        s = __dadd_rn(s, x[i]);
    s = block_sum_f64(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

} // namespace

double vg_sum_f64(vg_ctx *ctx, const double *x, int64_t n) {
    const int grid = 512;
    DevBuf<double> part(ctx, grid);
    DevBuf<double> tot(ctx, 1);
    {
        LaunchTimer lt(ctx);
        k_sum_part<<<grid, 256, 0, ctx->stream>>>(x, n, part.p);
    }
    VG_CHECK_LAUNCH();
    {
        LaunchTimer lt(ctx);
        k_sum_part<<<1, 512, 0, ctx->stream>>>(part.p, grid, tot.p);
    }
    VG_CHECK_LAUNCH();
    double *h = (double *)vg_pinned(ctx, sizeof(double));
    VG_CUDA(cudaMemcpyAsync(h, tot.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    vg_sync(ctx);
    return *h;
}

// ---------------------------------------------------------------------------------
// CSR from triples

namespace {

__global__ void k_make_keys(const int32_t *__restrict__ src, const int32_t *__restrict__ dst,
                            int64_t m, int b2, uint64_t *__restrict__ keys,
                            uint32_t *__restrict__ vals) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        keys[i] = ((uint64_t)(uint32_t)src[i] << b2) | (uint64_t)(uint32_t)dst[i];
        vals[i] = (uint32_t)i;
    }
}

__global__ void k_run_heads(const uint64_t *__restrict__ keys, int64_t m, bool combine,
                            int32_t *__restrict__ head) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x)
        head[i] = (!combine || i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// one thread per run: fold the run's weights in their (stable) order
__global__ void k_fold_runs(const uint64_t *__restrict__ keys, const uint32_t *__restrict__ order,
                            const double *__restrict__ w, const int32_t *__restrict__ head,
                            const int64_t *__restrict__ pos, int64_t m, int b2,
                            const int32_t *__restrict__ dst_map, int32_t *__restrict__ out_tail,
                            double *__restrict__ out_w, int64_t *__restrict__ rowcount) {
    const uint64_t mask = (b2 >= 64) ? ~0ULL : ((1ULL << b2) - 1ULL);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (!head[i]) continue;
        const uint64_t k = keys[i];
        double s = w[order[i]];
        int64_t j = i + 1;
        while (j < m && !head[j]) {
            s = __dadd_rn(s, w[order[j]]);
            j++;
        }
        const int64_t o = pos[i];
        const int32_t lo = (int32_t)(k & mask);
        out_tail[o] = dst_map ? dst_map[lo] : lo;
        out_w[o] = s;
        atomicAdd((unsigned long long *)&rowcount[k >> b2], 1ULL);
    }
}

} // namespace

static int bits_for(int64_t n) {
    int b = 1;
    while (b < 62 && ((int64_t)1 << b) < n) b++;
    return b;
}

vg_graph *vg_csr_from_triples(vg_ctx *ctx, int64_t nv, DevBuf<int32_t> &src, DevBuf<int32_t> &dst,
                              DevBuf<double> &w, int64_t m, bool combine, const int32_t *dst_map) {
    const int b2 = bits_for(nv > 1 ? nv : 2);
    VG_REQUIRE(2 * b2 <= 64, "graph too large for 64-bit sort keys");
    VG_REQUIRE(m < (int64_t)UINT32_MAX, "too many edges for one sort (%lld)", (long long)m);
    DevBuf<uint64_t> keys(ctx, m);
    DevBuf<uint32_t> order(ctx, m);
    if (m) {
        {
            LaunchTimer lt(ctx);
            k_make_keys<<<vg_grid(ctx, m, 256), 256, 0, ctx->stream>>>(src.p, dst.p, m, b2, keys.p,
                                                                        order.p);
        }
        VG_CHECK_LAUNCH();
        src.release();
        dst.release();
        vg_radix_sort_pairs(ctx, keys.p, order.p, m, 2 * b2);
    }
    DevBuf<int32_t> head(ctx, m);
    DevBuf<int64_t> pos(ctx, m);
    int64_t u = 0;
    if (m) {
        {
            LaunchTimer lt(ctx);
            k_run_heads<<<vg_grid(ctx, m, 256), 256, 0, ctx->stream>>>(keys.p, m, combine, head.p);
        }
        VG_CHECK_LAUNCH();
        u = vg_exclusive_scan_i32_to_i64(ctx, head.p, pos.p, m);
    }
    DevBuf<int64_t> rowptr(ctx, nv + 1);
    DevBuf<int32_t> tail(ctx, u);
    DevBuf<double> weight(ctx, u);
    VG_CUDA(cudaMemsetAsync(rowptr.p, 0, sizeof(int64_t) * (nv + 1), ctx->stream));
    if (m) {
        {
            LaunchTimer lt(ctx);
            k_fold_runs<<<vg_grid(ctx, m, 256), 256, 0, ctx->stream>>>(
                keys.p, order.p, w.p, head.p, pos.p, m, b2, dst_map, tail.p, weight.p, rowptr.p);
        }
        VG_CHECK_LAUNCH();
    }
    w.release();
    vg_scan_i64_async(ctx, rowptr.p, nv + 1, nullptr);
    return vg_graph_wrap(ctx, nv, u, rowptr.detach(), tail.detach(), weight.detach());
}
