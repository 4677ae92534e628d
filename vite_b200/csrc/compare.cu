// Ground-truth comparison (compare_communities and compute_gini_coeff,
// compare.cpp:58-318) on the device.
//
// The reference counts, over every pair of vertices inside each community of C1
// (the truth) and then of C2, whether the pair is together in the other vector
// (O(sum of squared community sizes)). The same counts follow from the
// contingency table: with n(a, b) the vertices labelled a in C1 and b in C2,
//   SameSame = sum over (a, b) of n(a, b) (n(a, b) - 1) / 2,
//   SameDiff = sum over a of |C1 = a| (|C1 = a| - 1) / 2 - SameSame,
//   DiffSame = sum over b of |C2 = b| (|C2 = b| - 1) / 2 - SameSame;
// the table's non-zero cells are the runs of the sorted keys a * nc2 + b. All
// counts are exact integers; precision, recall and the F-score are then the
// reference's double expressions. The Gini coefficient sorts the community sizes
// and takes sum (i + 1) size_i, an exact integer (the reference's double
// accumulation of the same integers is exact below 2^53).
#include "vg_internal.cuh"

#include <algorithm>

namespace {

__global__ void k_labels_in(const int64_t *__restrict__ c, int64_t n, int32_t *__restrict__ out,
                            int *__restrict__ bad, unsigned long long *__restrict__ maxv) {
    unsigned long long m = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = c[i];
        if (x < 0 || x >= INT32_MAX) {
            *bad = 1;
            out[i] = 0;
        } else {
            out[i] = (int32_t)x;
            if ((unsigned long long)x > m) m = (unsigned long long)x;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_down_sync(0xffffffffu, m, o);
        if (y > m) m = y;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(maxv, m);
}

__global__ void k_sizes(const int32_t *__restrict__ c, int64_t n, unsigned long long *__restrict__ size) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&size[c[i]], 1ULL);
}

// sum of size (size - 1) / 2 over an array of counts
__global__ void k_pairs(const unsigned long long *__restrict__ size, int64_t n,
                        unsigned long long *__restrict__ out) {
    unsigned long long s = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long x = size[i];
        s += x * (x - (x ? 1 : 0)) / 2;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

__global__ void k_pair_keys(const int32_t *__restrict__ a, const int32_t *__restrict__ b, int64_t n,
                            uint64_t nb, uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        keys[i] = (uint64_t)a[i] * nb + (uint64_t)b[i];
        vals[i] = (uint32_t)i;
    }
}

// sum over the runs of equal sorted keys of len (len - 1) / 2: each run head
// measures its run
__global__ void k_run_pairs(const uint64_t *__restrict__ k, int64_t n,
                            unsigned long long *__restrict__ out) {
    unsigned long long s = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i > 0 && k[i - 1] == k[i]) continue;
        int64_t j = i + 1;
        while (j < n && k[j] == k[i]) j++;
        const unsigned long long len = (unsigned long long)(j - i);
        s += len * (len - 1) / 2;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

__global__ void k_size_keys(const unsigned long long *__restrict__ size, int64_t n,
                            uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        keys[i] = size[i];
        vals[i] = (uint32_t)i;
    }
}

// sum of (i + 1) * sorted_size[i]
__global__ void k_gini_num(const uint64_t *__restrict__ sorted, int64_t n,
                           unsigned long long *__restrict__ out) {
    unsigned long long s = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        s += (unsigned long long)(i + 1) * sorted[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

int bits_for(uint64_t x) {
    int b = 1;
    while (b < 64 && (x >> b) != 0) b++;
    return b;
}

unsigned long long read_u64(vg_ctx *ctx, const unsigned long long *d) {
    unsigned long long *h = (unsigned long long *)vg_pinned(ctx, sizeof(unsigned long long));
    VG_CUDA(cudaMemcpyAsync(h, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
    vg_sync(ctx);
    return *h;
}

// compute_gini_coeff (compare.cpp:287-318) from exact sums; numColors is the
// reference's int argument
double gini_of(vg_ctx *ctx, const unsigned long long *size, int64_t nc, int64_t n) {
    DevBuf<uint64_t> keys(ctx, nc);
    DevBuf<uint32_t> vals(ctx, nc);
    const int grid = vg_grid(ctx, nc, 256);
    { LaunchTimer lt(ctx); k_size_keys<<<grid, 256, 0, ctx->stream>>>(size, nc, keys.p, vals.p); }
    VG_CHECK_LAUNCH();
    vg_radix_sort_pairs(ctx, keys.p, vals.p, nc, bits_for((uint64_t)n));
    DevBuf<unsigned long long> num(ctx, 1);
    VG_CUDA(cudaMemsetAsync(num.p, 0, sizeof(unsigned long long), ctx->stream));
    { LaunchTimer lt(ctx); k_gini_num<<<grid, 256, 0, ctx->stream>>>(keys.p, nc, num.p); }
    VG_CHECK_LAUNCH();
    const double numFunc = (double)read_u64(ctx, num.p);
    const double denFunc = (double)n;
    const int numColors = (int)nc;
    return ((2 * numFunc) / (numColors * denFunc)) - ((double)(numColors + 1) / (double)numColors);
}

} // namespace

extern "C" vg_status vg_compare_communities(vg_ctx *ctx, int64_t n, const int64_t *c1,
                                            const int64_t *c2, vg_compare_stats *out) {
    if (!ctx || !out || n < 1 || !c1 || !c2) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        VG_REQUIRE(n < ((int64_t)1 << 32), "at most 2^32 - 1 vertices (got %lld)", (long long)n);
        const int grid = vg_grid(ctx, n, 256);
        DevBuf<int64_t> wide(ctx, n);
        DevBuf<int32_t> a(ctx, n), b(ctx, n);
        DevBuf<int> bad(ctx, 1);
        DevBuf<unsigned long long> mx(ctx, 2), cnt(ctx, 3);
        VG_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
        VG_CUDA(cudaMemsetAsync(mx.p, 0, 2 * sizeof(unsigned long long), ctx->stream));
        VG_CUDA(cudaMemsetAsync(cnt.p, 0, 3 * sizeof(unsigned long long), ctx->stream));
        const int64_t *src[2] = {c1, c2};
        int32_t *dst[2] = {a.p, b.p};
        for (int k = 0; k < 2; k++) {
            VG_CUDA(cudaMemcpyAsync(wide.p, src[k], sizeof(int64_t) * n, cudaMemcpyHostToDevice,
                                    ctx->stream));
            { LaunchTimer lt(ctx);
              k_labels_in<<<grid, 256, 0, ctx->stream>>>(wide.p, n, dst[k], bad.p, mx.p + k); }
            VG_CHECK_LAUNCH();
        }
        wide.release();
        int *hb = (int *)vg_pinned(ctx, 32);
        unsigned long long *hm = reinterpret_cast<unsigned long long *>(hb + 2);
        VG_CUDA(cudaMemcpyAsync(hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        VG_CUDA(cudaMemcpyAsync(hm, mx.p, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                ctx->stream));
        vg_sync(ctx);
        VG_REQUIRE(*hb == 0, "community labels must lie in [0, 2^31 - 1)");
        // the number of communities is the largest label + 1 (compare.cpp:74-94)
        const int64_t nc1 = (int64_t)hm[0] + 1, nc2 = (int64_t)hm[1] + 1;
        DevBuf<unsigned long long> s1(ctx, nc1), s2(ctx, nc2);
        VG_CUDA(cudaMemsetAsync(s1.p, 0, sizeof(unsigned long long) * nc1, ctx->stream));
        VG_CUDA(cudaMemsetAsync(s2.p, 0, sizeof(unsigned long long) * nc2, ctx->stream));
        { LaunchTimer lt(ctx); k_sizes<<<grid, 256, 0, ctx->stream>>>(a.p, n, s1.p); }
        VG_CHECK_LAUNCH();
        { LaunchTimer lt(ctx); k_sizes<<<grid, 256, 0, ctx->stream>>>(b.p, n, s2.p); }
        VG_CHECK_LAUNCH();
        { LaunchTimer lt(ctx);
          k_pairs<<<vg_grid(ctx, nc1, 256), 256, 0, ctx->stream>>>(s1.p, nc1, cnt.p + 0); }
        VG_CHECK_LAUNCH();
        { LaunchTimer lt(ctx);
          k_pairs<<<vg_grid(ctx, nc2, 256), 256, 0, ctx->stream>>>(s2.p, nc2, cnt.p + 1); }
        VG_CHECK_LAUNCH();
        {
            DevBuf<uint64_t> keys(ctx, n);
            DevBuf<uint32_t> vals(ctx, n);
            { LaunchTimer lt(ctx);
              k_pair_keys<<<grid, 256, 0, ctx->stream>>>(a.p, b.p, n, (uint64_t)nc2, keys.p, vals.p); }
            VG_CHECK_LAUNCH();
            vg_radix_sort_pairs(ctx, keys.p, vals.p, n, bits_for((uint64_t)nc1 * (uint64_t)nc2));
            { LaunchTimer lt(ctx); k_run_pairs<<<grid, 256, 0, ctx->stream>>>(keys.p, n, cnt.p + 2); }
            VG_CHECK_LAUNCH();
        }
        unsigned long long *hc = (unsigned long long *)vg_pinned(ctx, 3 * sizeof(unsigned long long));
        VG_CUDA(cudaMemcpyAsync(hc, cnt.p, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                ctx->stream));
        vg_sync(ctx);
        const int64_t pairs1 = (int64_t)hc[0], pairs2 = (int64_t)hc[1], ss = (int64_t)hc[2];
        vg_compare_stats r{};
        r.n = n;
        r.nc1 = nc1;
        r.nc2 = nc2;
        r.same_same = ss;
        r.same_diff = pairs1 - ss;
        r.diff_same = pairs2 - ss;
        // compare.cpp:265-271
        r.precision = (double)r.same_same / (double)(r.same_same + r.diff_same);
        r.recall = (double)r.same_same / (double)(r.same_same + r.same_diff);
        r.fscore = 2.0 * ((r.precision * r.recall) / (r.precision + r.recall));
        r.gini1 = gini_of(ctx, s1.p, nc1, n);
        r.gini2 = gini_of(ctx, s2.p, nc2, n);
        *out = r;
    });
}
