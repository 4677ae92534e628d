// Aggregation of the next-level CSR for distbuildNextLevelGraph (rebuild.cpp:294-478).
//
// The reference accumulates newEdgesMap[c1][c2] += w scanning vertices in id order
// and each row in CSR order, and writes every row sorted by c2 (std::map). Here:
//   1. vertices are grouped by their new row c1 with a stable sort of the VERTICES
//      (keys in reference order), so each row's entries can be copied as whole
//      CSR rows, in the reference's (vertex, edge) order, into one segment;
//   2. each segment is reduced by c2 with every sum a left fold in segment order,
//      giving the reference's sums bit for bit: one thread per segment keeps up to
//      16 distinct c2 in registers and sorts them with a network; segments with
//      more distinct neighbours (or longer than 4096 entries) are sorted by c2
//      (stable) -- one warp per segment up to 1024 entries, one CTA up to 8192, a
//      single-CTA radix sort in global scratch above -- and their runs folded;
//   3. the unique entries are compacted into the next CSR.
#include "vg_internal.cuh"

#include <algorithm>
#include <climits>

namespace {

constexpr int U_MAX = 16;     // thread path: distinct neighbours kept in registers
constexpr int L_THREAD = 4096; // thread path: longest segment
constexpr int W_MAX = 1024;   // warp path
constexpr int C_MAX = 8192;   // CTA path
constexpr int AG_WARPS = 8;
constexpr int AG_THREADS = 256;

__device__ __forceinline__ int32_t pos_of(const int32_t *__restrict__ pos, int64_t r) {
    return pos ? pos[r] : (int32_t)r;
}

__global__ void k_vertex_keys(int64_t nv, const int32_t *__restrict__ pos,
                              const int32_t *__restrict__ new_row, uint64_t *__restrict__ keys,
                              uint32_t *__restrict__ vals) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nv;
         r += (int64_t)gridDim.x * blockDim.x) {
        keys[r] = (uint64_t)new_row[pos_of(pos, r)];
        vals[r] = (uint32_t)r;
    }
}

__global__ void k_sorted_deg(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ pos,
                             const uint32_t *__restrict__ order, int64_t nv, int64_t *__restrict__ deg) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nv;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = pos_of(pos, order[k]);
        deg[k] = rowptr[p + 1] - rowptr[p];
    }
}

__global__ void k_row_starts(const uint64_t *__restrict__ keys, const int64_t *__restrict__ off,
                             int64_t nv, int64_t *__restrict__ rstart) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nv;
         k += (int64_t)gridDim.x * blockDim.x)
        if (k == 0 || keys[k] != keys[k - 1]) rstart[keys[k]] = off[k];
}

// one warp per vertex (in grouped order): its row goes to the segment, neighbours
// renamed to their ordering keys
__global__ void k_group_copy(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ tail,
                             const double *__restrict__ w, const int32_t *__restrict__ pos,
                             const uint32_t *__restrict__ order, const int64_t *__restrict__ off,
                             int64_t nv, const int32_t *__restrict__ new_key,
                             int32_t *__restrict__ gk, double *__restrict__ gw) {
    const int lane = threadIdx.x & 31;
    const int64_t wg = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t k = wg; k < nv; k += nw) {
        const int32_t p = pos_of(pos, order[k]);
        const int64_t e0 = rowptr[p], len = rowptr[p + 1] - e0, o = off[k];
        for (int64_t j = lane; j < len; j += 32) {
            gk[o + j] = new_key[tail[e0 + j]];
            gw[o + j] = w[e0 + j];
        }
    }
}

// ascending bitonic sort of n2 (power of two) packed keys, by `nt` threads
template <bool WARP>
__device__ void bitonic(uint64_t *sk, int n2, int t, int nt) {
    for (int k = 2; k <= n2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = t; i < n2; i += nt) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const uint64_t a = sk[i], b = sk[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        sk[i] = b;
                        sk[ixj] = a;
                    }
                }
            }
            if (WARP) __syncwarp();
            else __syncthreads();
        }
}

// fold the run that starts at sorted index i (keys packed key<<32 | index in segment)
__device__ __forceinline__ double fold_run(const uint64_t *sk, int i, int L, const double *__restrict__ seg_w) {
    const uint32_t key = (uint32_t)(sk[i] >> 32);
    double s = seg_w[(uint32_t)sk[i]];
    for (int j = i + 1; j < L && (uint32_t)(sk[j] >> 32) == key; j++) s = __dadd_rn(s, seg_w[(uint32_t)sk[j]]);
    return s;
}

// One thread per segment: entries are scanned in order and each is added to its
// key's accumulator (a list of at most U_MAX keys in registers), so every sum is
// the left fold in segment order; the list is then sorted by key with a
// sorting network. Segments that are longer than L_THREAD or have more distinct
// keys are flagged for the sorting paths below.
__global__ void __launch_bounds__(256) k_rows_thread(
    int64_t nc, const int64_t *__restrict__ rstart, const int32_t *__restrict__ gk,
    const double *__restrict__ gw, int32_t *__restrict__ uk, double *__restrict__ uw,
    int64_t *__restrict__ ucount, int32_t *__restrict__ flag) {
    for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < nc;
         row += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = rstart[row];
        const int64_t L = rstart[row + 1] - b;
        if (L > L_THREAD) {
            flag[row] = 1;
            continue;
        }
        int32_t key[U_MAX];
        double acc[U_MAX];
#pragma unroll
        for (int q = 0; q < U_MAX; q++) {
            key[q] = INT_MAX;
            acc[q] = 0.0;
        }
        int U = 0;
        bool over = false;
        for (int64_t i = 0; i < L; i++) {
            const int32_t k = gk[b + i];
            const double w = gw[b + i];
            bool hit = false;
#pragma unroll
            for (int q = 0; q < U_MAX; q++)
                if (q < U && key[q] == k) {
                    acc[q] = __dadd_rn(acc[q], w);
                    hit = true;
                }
            if (!hit) {
                if (U == U_MAX) {
                    over = true;
                    break;
                }
#pragma unroll
                for (int q = 0; q < U_MAX; q++)
                    if (q == U) {
                        key[q] = k;
                        acc[q] = w;
                    }
                U++;
            }
        }
        if (over) {
            flag[row] = 1;
            continue;
        }
        // bitonic network over the 16 (key, sum) pairs; unused slots hold INT_MAX
#pragma unroll
        for (int k2 = 2; k2 <= U_MAX; k2 <<= 1)
#pragma unroll
            for (int j = k2 >> 1; j > 0; j >>= 1)
#pragma unroll
                for (int i = 0; i < U_MAX; i++) {
                    const int ixj = i ^ j;
                    if (ixj > i) {
                        const bool up = (i & k2) == 0;
                        if ((key[i] > key[ixj]) == up) {
                            const int32_t tk = key[i];
                            key[i] = key[ixj];
                            key[ixj] = tk;
                            const double ta = acc[i];
                            acc[i] = acc[ixj];
                            acc[ixj] = ta;
                        }
                    }
                }
#pragma unroll
        for (int q = 0; q < U_MAX; q++)
            if (q < U) {
                uk[b + q] = key[q];
                uw[b + q] = acc[q];
            }
        ucount[row] = U;
        flag[row] = 0;
    }
}

__global__ void __launch_bounds__(AG_WARPS * 32) k_rows_warp(
    int64_t nc, const int64_t *__restrict__ rstart, const int32_t *__restrict__ gk,
    const double *__restrict__ gw, int32_t *__restrict__ uk, double *__restrict__ uw,
    int64_t *__restrict__ ucount, const int32_t *__restrict__ flag) {
    extern __shared__ uint64_t smem64[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t *sk = smem64 + (size_t)warp * W_MAX;
    const int64_t wg = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (int64_t row = wg; row < nc; row += nw) {
        if (!flag[row]) continue;
        const int64_t b = rstart[row];
        const int L = (int)(rstart[row + 1] - b);
        if (L > W_MAX) continue;
        int n2 = 1;
        while (n2 < L) n2 <<= 1;
        for (int i = lane; i < n2; i += 32)
            sk[i] = i < L ? (((uint64_t)(uint32_t)gk[b + i] << 32) | (uint32_t)i) : ~0ULL;
        __syncwarp();
        bitonic<true>(sk, n2, lane, 32);
        int64_t u = 0;
        for (int base = 0; base < L; base += 32) {
            const int i = base + lane;
            const bool head = i < L && (i == 0 || (sk[i] >> 32) != (sk[i - 1] >> 32));
            const unsigned hm = __ballot_sync(0xffffffffu, head);
            if (head) {
                const int64_t o = b + u + __popc(hm & lt);
                uk[o] = (int32_t)(sk[i] >> 32);
                uw[o] = fold_run(sk, i, L, gw + b);
            }
            u += __popc(hm);
        }
        if (lane == 0) ucount[row] = u;
        __syncwarp();
    }
}

// block-wide exclusive scan of one int per thread (AG_THREADS threads)
__device__ int block_scan_excl(int v, int *total, int *ws) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int w = 0; w < AG_THREADS / 32; w++) {
            const int c = ws[w];
            ws[w] = run;
            run += c;
        }
        ws[AG_THREADS / 32] = run;
    }
    __syncthreads();
    const int r = ws[warp] + x - v;
    *total = ws[AG_THREADS / 32];
    __syncthreads();
    return r;
}

// fold + compaction of a sorted segment by a whole CTA
__device__ void cta_fold(const uint64_t *sk, int L, int64_t b, const double *__restrict__ gw,
                         int32_t *__restrict__ uk, double *__restrict__ uw, int64_t *ucount_row,
                         int *ws) {
    int64_t u = 0;
    for (int base = 0; base < L; base += AG_THREADS) {
        const int i = base + threadIdx.x;
        const bool head = i < L && (i == 0 || (sk[i] >> 32) != (sk[i - 1] >> 32));
        int tot;
        const int rank = block_scan_excl(head ? 1 : 0, &tot, ws);
        if (head) {
            const int64_t o = b + u + rank;
            uk[o] = (int32_t)(sk[i] >> 32);
            uw[o] = fold_run(sk, i, L, gw + b);
        }
        u += tot;
    }
    if (threadIdx.x == 0) *ucount_row = u;
}

__global__ void __launch_bounds__(AG_THREADS) k_rows_cta(
    int64_t nc, const int64_t *__restrict__ rstart, const int32_t *__restrict__ gk,
    const double *__restrict__ gw, int32_t *__restrict__ uk, double *__restrict__ uw,
    int64_t *__restrict__ ucount, const int32_t *__restrict__ flag) {
    extern __shared__ uint64_t smem64[];
    __shared__ int ws[AG_THREADS / 32 + 1];
    for (int64_t row = blockIdx.x; row < nc; row += gridDim.x) {
        if (!flag[row]) continue;
        const int64_t b = rstart[row];
        const int L = (int)(rstart[row + 1] - b);
        if (L <= W_MAX || L > C_MAX) continue;
        int n2 = 1;
        while (n2 < L) n2 <<= 1;
        for (int i = threadIdx.x; i < n2; i += AG_THREADS)
            smem64[i] = i < L ? (((uint64_t)(uint32_t)gk[b + i] << 32) | (uint32_t)i) : ~0ULL;
        __syncthreads();
        bitonic<false>(smem64, n2, threadIdx.x, AG_THREADS);
        cta_fold(smem64, L, b, gw, uk, uw, ucount + row, ws);
        __syncthreads();
    }
}

// segments above C_MAX: a single-CTA stable LSD radix sort in global scratch
// (scratch holds 2*L packed keys per segment, at offset sbase[row])
__global__ void __launch_bounds__(AG_THREADS) k_rows_big(
    int64_t nc, const int64_t *__restrict__ rstart, const int32_t *__restrict__ gk,
    const double *__restrict__ gw, int32_t *__restrict__ uk, double *__restrict__ uw,
    int64_t *__restrict__ ucount, const int64_t *__restrict__ sbase, uint64_t *__restrict__ scratch,
    int key_bits, const int32_t *__restrict__ flag) {
    __shared__ int hist[256];
    __shared__ int64_t dbase[256];
    __shared__ int wcnt[AG_THREADS / 32][256];
    __shared__ int ws[AG_THREADS / 32 + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (int64_t row = blockIdx.x; row < nc; row += gridDim.x) {
        if (!flag[row]) continue;
        const int64_t b = rstart[row];
        const int64_t L = rstart[row + 1] - b;
        if (L <= C_MAX) continue;
        uint64_t *A = scratch + sbase[row], *B = A + L;
        for (int64_t i = threadIdx.x; i < L; i += AG_THREADS)
            A[i] = ((uint64_t)(uint32_t)gk[b + i] << 32) | (uint32_t)i;
        __syncthreads();
        for (int shift = 32; shift < 32 + key_bits; shift += 8) {
            hist[threadIdx.x] = 0;
            __syncthreads();
            for (int64_t i = threadIdx.x; i < L; i += AG_THREADS) atomicAdd(&hist[(A[i] >> shift) & 0xff], 1);
            __syncthreads();
            if (threadIdx.x == 0) {
                int64_t run = 0;
                for (int d = 0; d < 256; d++) {
                    dbase[d] = run;
                    run += hist[d];
                }
            }
            __syncthreads();
            for (int64_t base = 0; base < L; base += AG_THREADS) {
                for (int w = 0; w < AG_THREADS / 32; w++) wcnt[w][threadIdx.x] = 0;
                __syncthreads();
                const int64_t i = base + threadIdx.x;
                const bool valid = i < L;
                const uint64_t x = valid ? A[i] : 0;
                const int d = valid ? (int)((x >> shift) & 0xff) : 256 + lane;
                const unsigned peers = __match_any_sync(0xffffffffu, d);
                const int rk = __popc(peers & lt);
                if (valid && rk == 0) wcnt[warp][d] = __popc(peers);
                __syncthreads();
                int run = 0;
                for (int w = 0; w < AG_THREADS / 32; w++) {
                    const int c = wcnt[w][threadIdx.x];
                    wcnt[w][threadIdx.x] = run;
                    run += c;
                }
                __syncthreads();
                if (valid) B[dbase[d] + wcnt[warp][d] + rk] = x;
                __syncthreads();
                dbase[threadIdx.x] += run;
                __syncthreads();
            }
            uint64_t *t = A;
            A = B;
            B = t;
            __syncthreads();
        }
        // fold from global scratch
        int64_t u = 0;
        for (int64_t base = 0; base < L; base += AG_THREADS) {
            const int64_t i = base + threadIdx.x;
            const bool head = i < L && (i == 0 || (A[i] >> 32) != (A[i - 1] >> 32));
            int tot;
            const int rank = block_scan_excl(head ? 1 : 0, &tot, ws);
            if (head) {
                const uint32_t key = (uint32_t)(A[i] >> 32);
                double s = gw[b + (uint32_t)A[i]];
                for (int64_t j = i + 1; j < L && (uint32_t)(A[j] >> 32) == key; j++)
                    s = __dadd_rn(s, gw[b + (uint32_t)A[j]]);
                uk[b + u + rank] = (int32_t)key;
                uw[b + u + rank] = s;
            }
            u += tot;
        }
        if (threadIdx.x == 0) ucount[row] = u;
        __syncthreads();
    }
}

__global__ void k_big_sizes(int64_t nc, const int64_t *__restrict__ rstart,
                            const int32_t *__restrict__ flag, int64_t *__restrict__ sz) {
    for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < nc;
         row += (int64_t)gridDim.x * blockDim.x) {
        const int64_t L = rstart[row + 1] - rstart[row];
        sz[row] = (flag[row] && L > C_MAX) ? 2 * L : 0;
    }
}

__global__ void k_compact_rows(int64_t nc, const int64_t *__restrict__ rstart,
                               const int64_t *__restrict__ rowptr, const int32_t *__restrict__ uk,
                               const double *__restrict__ uw, const int32_t *__restrict__ key_to_pos,
                               int32_t *__restrict__ tail, double *__restrict__ w) {
    const int lane = threadIdx.x & 31;
    const int64_t wg = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t row = wg; row < nc; row += nw) {
        const int64_t s = rstart[row], o = rowptr[row], len = rowptr[row + 1] - o;
        for (int64_t j = lane; j < len; j += 32) {
            const int32_t k = uk[s + j];
            tail[o + j] = key_to_pos ? key_to_pos[k] : k;
            w[o + j] = uw[s + j];
        }
    }
}

} // namespace

// Next-level CSR with nc rows. new_row[p]: row of position p's community; new_key[p]:
// the ordering key of p's community as a neighbour (the next level's reference
// number); emission in reference order (pos: reference id -> position, or null);
// key_to_pos names the stored tail (null: the key itself).
vg_graph *vg_aggregate_rows(vg_ctx *ctx, const vg_graph *g, const int32_t *pos,
                            const int32_t *new_row, const int32_t *new_key, int64_t nc,
                            const int32_t *key_to_pos) {
    const int64_t nv = g->nv, ne = g->ne;
    static bool configured = false;
    if (!configured) {
        VG_CUDA(cudaFuncSetAttribute(k_rows_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(AG_WARPS * W_MAX * sizeof(uint64_t))));
        VG_CUDA(cudaFuncSetAttribute(k_rows_cta, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(C_MAX * sizeof(uint64_t))));
        configured = true;
    }
    int kbits = 1;
    while (kbits < 31 && ((int64_t)1 << kbits) < nc) kbits++;
    // 1. vertices grouped by new row, reference order inside a row
    DevBuf<uint64_t> vkeys(ctx, nv);
    DevBuf<uint32_t> vorder(ctx, nv);
    const int grid = vg_grid(ctx, nv, 256);
    if (nv) {
        { LaunchTimer lt(ctx);
          k_vertex_keys<<<grid, 256, 0, ctx->stream>>>(nv, pos, new_row, vkeys.p, vorder.p); }
        VG_CHECK_LAUNCH();
        vg_radix_sort_pairs(ctx, vkeys.p, vorder.p, nv, kbits);
    }
    // 2. segment offsets
    DevBuf<int64_t> off(ctx, nv + 1), rstart(ctx, nc + 1);
    VG_CUDA(cudaMemsetAsync(off.p + nv, 0, sizeof(int64_t), ctx->stream));
    if (nv) {
        { LaunchTimer lt(ctx);
          k_sorted_deg<<<grid, 256, 0, ctx->stream>>>(g->rowptr, pos, vorder.p, nv, off.p); }
        VG_CHECK_LAUNCH();
    }
    vg_exclusive_scan_i64(ctx, off.p, nv + 1);
    VG_CUDA(cudaMemcpyAsync(rstart.p + nc, &ne, sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
    if (nv) {
        { LaunchTimer lt(ctx);
          k_row_starts<<<grid, 256, 0, ctx->stream>>>(vkeys.p, off.p, nv, rstart.p); }
        VG_CHECK_LAUNCH();
    }
    vkeys.release();
    // 3. copy rows into segments
    DevBuf<int32_t> gk(ctx, ne);
    DevBuf<double> gw(ctx, ne);
    if (ne) {
        LaunchTimer lt(ctx);
        k_group_copy<<<vg_grid(ctx, nv * 32, 256), 256, 0, ctx->stream>>>(
            g->rowptr, g->tail, g->weight, pos, vorder.p, off.p, nv, new_key, gk.p, gw.p);
    }
    VG_CHECK_LAUNCH();
    vorder.release();
    off.release();
    // 4. sort + fold per segment
    DevBuf<int32_t> uk(ctx, ne);
    DevBuf<double> uw(ctx, ne);
    DevBuf<int64_t> ucount(ctx, nc + 1);
    VG_CUDA(cudaMemsetAsync(ucount.p + nc, 0, sizeof(int64_t), ctx->stream));
    DevBuf<int32_t> flag(ctx, nc);
    if (nc) {
        { LaunchTimer lt(ctx);
          k_rows_thread<<<vg_grid(ctx, nc, 256, 8), 256, 0, ctx->stream>>>(
              nc, rstart.p, gk.p, gw.p, uk.p, uw.p, ucount.p, flag.p); }
        VG_CHECK_LAUNCH();
        { LaunchTimer lt(ctx);
          k_rows_warp<<<vg_grid(ctx, nc * 32, AG_WARPS * 32, 4), AG_WARPS * 32,
                        AG_WARPS * W_MAX * sizeof(uint64_t), ctx->stream>>>(nc, rstart.p, gk.p, gw.p,
                                                                            uk.p, uw.p, ucount.p, flag.p); }
        VG_CHECK_LAUNCH();
        { LaunchTimer lt(ctx);
          k_rows_cta<<<vg_grid(ctx, nc, 1, 2), AG_THREADS, C_MAX * sizeof(uint64_t), ctx->stream>>>(
              nc, rstart.p, gk.p, gw.p, uk.p, uw.p, ucount.p, flag.p); }
        VG_CHECK_LAUNCH();
        // big segments: scratch sized by their total length
        DevBuf<int64_t> sbase(ctx, nc + 1);
        VG_CUDA(cudaMemsetAsync(sbase.p + nc, 0, sizeof(int64_t), ctx->stream));
        { LaunchTimer lt(ctx);
          k_big_sizes<<<vg_grid(ctx, nc, 256), 256, 0, ctx->stream>>>(nc, rstart.p, flag.p, sbase.p); }
        VG_CHECK_LAUNCH();
        const int64_t big = vg_exclusive_scan_i64(ctx, sbase.p, nc + 1);
        if (big > 0) {
            DevBuf<uint64_t> scratch(ctx, big);
            LaunchTimer lt(ctx);
            k_rows_big<<<vg_grid(ctx, nc, 1, 2), AG_THREADS, 0, ctx->stream>>>(
                nc, rstart.p, gk.p, gw.p, uk.p, uw.p, ucount.p, sbase.p, scratch.p, kbits, flag.p);
            VG_CHECK_LAUNCH();
            vg_sync(ctx);
        }
    }
    gk.release();
    gw.release();
    // 5-6. next CSR
    const int64_t m = vg_exclusive_scan_i64(ctx, ucount.p, nc + 1);
    DevBuf<int32_t> tail(ctx, m);
    DevBuf<double> w(ctx, m);
    if (nc) {
        LaunchTimer lt(ctx);
        k_compact_rows<<<vg_grid(ctx, nc * 32, 256), 256, 0, ctx->stream>>>(
            nc, rstart.p, ucount.p, uk.p, uw.p, key_to_pos, tail.p, w.p);
    }
    VG_CHECK_LAUNCH();
    vg_sync(ctx);
    return vg_graph_wrap(ctx, nc, m, ucount.detach(), tail.detach(), w.detach());
}
