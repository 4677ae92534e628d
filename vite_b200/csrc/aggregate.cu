// Aggregation of the next-level CSR for distbuildNextLevelGraph (rebuild.cpp:294-478).
//
// The reference accumulates newEdgesMap[c1][c2] += w scanning vertices in id order
// and each row in CSR order, and writes every row sorted by c2 (std::map). Here:
//   1. vertices are grouped by their new row c1 with a stable sort of the VERTICES
//      (keys in reference order), so each row's entries can be copied as whole
//      CSR rows, in the reference's (vertex, edge) order, into one segment;
//   2. each segment is reduced by c2 with every sum a left fold in segment order,
//      giving the reference's sums bit for bit: one warp per segment folds its
//      entries into a shared-memory hash table in order and sorts the distinct
//      keys; segments with more than 256 distinct keys go through one stable radix
//      sort of all their entries by (segment, c2) and each run is folded in order;
//   3. the unique entries are compacted into the next CSR.
#include "vg_internal.cuh"

#include <algorithm>
#include <climits>

namespace {


__device__ __forceinline__ int32_t pos_of(const int32_t *__restrict__ pos, int64_t r) {
    return pos ? pos[r] : (int32_t)r;
}

// vertices in reference order r, keyed by their new row; the payload is the
// vertex's position, so the stable sort lists each row's vertices in reference
// order by position
__global__ void k_vertex_keys(int64_t nv, const int32_t *__restrict__ pos,
                              const int32_t *__restrict__ new_row, uint64_t *__restrict__ keys,
                              uint32_t *__restrict__ vals) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nv;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = pos_of(pos, r);
        keys[r] = (uint64_t)new_row[p];
        vals[r] = (uint32_t)p;
    }
}

// k-th vertex in grouped order (order[k]: its position): its degree, and where its
// row starts in the CSR
__global__ void k_sorted_deg(const int64_t *__restrict__ rowptr, const uint32_t *__restrict__ order,
                             int64_t nv, int64_t *__restrict__ deg, int64_t *__restrict__ src_start) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nv;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = (int32_t)order[k];
        const int64_t e0 = rowptr[p];
        deg[k] = rowptr[p + 1] - e0;
        src_start[k] = e0;
    }
}

__global__ void k_row_starts(const uint64_t *__restrict__ keys, const int64_t *__restrict__ off,
                             int64_t nv, int64_t *__restrict__ rstart) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nv;
         k += (int64_t)gridDim.x * blockDim.x)
        if (k == 0 || keys[k] != keys[k - 1]) rstart[keys[k]] = off[k];
}

// Rows of at most LONG_ROW entries are copied by eight lanes each; the longer ones
// (hubs, giant communities) are cut into chunks of COPY_CHUNK entries, one block per
// chunk, so one row never serialises a warp.
constexpr int64_t LONG_ROW = 4096;
// a copy takes a warp per row instead of eight lanes when rows average this many
// entries
constexpr int64_t LANES32_ROW = 64;
constexpr int64_t COPY_CHUNK = 4096;

// vertices in grouped order: each one's row goes to its segment, neighbours renamed
// to their ordering keys
// G lanes per row: 8 for rows of a few tens of entries, 32 when the rows are long
// (a coarse level with hundreds of entries per row)
template <int G>
__global__ void k_group_copy(const int32_t *__restrict__ tail, const double *__restrict__ w,
                             const int64_t *__restrict__ src_start, const int64_t *__restrict__ off,
                             int64_t nv, const int32_t *__restrict__ new_key,
                             int32_t *__restrict__ gk, double *__restrict__ gw) {
    const int sub = threadIdx.x & (G - 1);
    const int64_t grp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / G;
    const int64_t ng = ((int64_t)gridDim.x * blockDim.x) / G;
    for (int64_t k = grp; k < nv; k += ng) {
        const int64_t o = off[k], len = off[k + 1] - o;
        if (len > LONG_ROW) continue;
        const int64_t e0 = src_start[k];
        // two entries per lane per step: both tails are loaded before the key gathers
        for (int64_t j = sub; j < len; j += 2 * G) {
            const bool two = j + G < len;
            const int32_t t0 = tail[e0 + j];
            const int32_t t1 = two ? tail[e0 + j + G] : 0;
            const double w0 = w[e0 + j];
            const double w1 = two ? w[e0 + j + G] : 0.0;
            const int32_t k0 = new_key[t0];
            const int32_t k1 = two ? new_key[t1] : 0;
            gk[o + j] = k0;
            gw[o + j] = w0;
            if (two) {
                gk[o + j + G] = k1;
                gw[o + j + G] = w1;
            }
        }
    }
}

// rows [offs[r], offs[r+1]) longer than LONG_ROW, in any order (each chunk writes
// its own entries, so the order changes no result): list[s] = row, chunks[s] = its
// chunk count; cnt[0] counts them. At most cap rows qualify (each has more than
// LONG_ROW of the offs' entries); the guard keeps writes inside the lists anyway.
__global__ void k_long_collect(const int64_t *__restrict__ offs, int64_t n, int64_t cap,
                               int32_t *__restrict__ list, int64_t *__restrict__ chunks,
                               int64_t *__restrict__ cnt) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t len = offs[r + 1] - offs[r];
        if (len > LONG_ROW) {
            const int64_t s = (int64_t)atomicAdd((unsigned long long *)cnt, 1ULL);
            if (s < cap) {
                list[s] = (int32_t)r;
                chunks[s] = (len + COPY_CHUNK - 1) / COPY_CHUNK;
            }
        }
    }
}
__device__ __forceinline__ int64_t chunk_owner(const int64_t *__restrict__ cb, int64_t n, int64_t c) {
    int64_t lo = 0, hi = n; // largest q with cb[q] <= c
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (cb[mid] <= c) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void k_group_copy_long(const int32_t *__restrict__ tail, const double *__restrict__ w,
                                  const int64_t *__restrict__ src_start, const int64_t *__restrict__ off,
                                  const int32_t *__restrict__ list, const int64_t *__restrict__ cb,
                                  const int64_t *__restrict__ cnt, const int32_t *__restrict__ new_key,
                                  int32_t *__restrict__ gk, double *__restrict__ gw) {
    const int64_t nl = cnt[0], nchunks = cnt[1];
    for (int64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const int64_t q = chunk_owner(cb, nl, c);
        const int64_t k = list[q];
        const int64_t o = off[k], len = off[k + 1] - o;
        const int64_t e0 = src_start[k];
        const int64_t j0 = (c - cb[q]) * COPY_CHUNK, j1 = min(j0 + COPY_CHUNK, len);
        for (int64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
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

// One warp per segment. The segment is read in chunks of 32 entries; inside a
// chunk the lanes holding the same key elect the lowest as leader, which adds its
// peers' weights in lane order onto the key's running sum in a shared-memory
// table, so every sum is the left fold in segment order. Only the distinct keys
// are then sorted: in registers across the warp when there are at most 32 of
// them, else in shared memory. The reduction runs in two tiers: first every segment
// with a small table (MAXU_S distinct keys at most, so more warps fit per SM), then
// the segments that overflowed it with a large one (MAXU_L); a segment with more
// than MAXU_L distinct keys is flagged for the sorted path.
#ifndef VG_RH_GRID
#define VG_RH_GRID 3 // CTAs per SM in the grid of the large-table tier
#endif
#ifndef VG_RH_GRID_S
#define VG_RH_GRID_S 5 // CTAs per SM in the grid of the small-table tier
#endif
constexpr int H_MAXU_S = 96, H_CAP_S = 256;  // small tier
constexpr int H_MAXU = 256, H_CAP = 512;     // large tier
// a chunk can add 32 keys to MAXU before the check: a third of the slots stay empty
static_assert(2 * H_CAP >= 3 * (H_MAXU + 32) && 2 * H_CAP_S >= 3 * (H_MAXU_S + 32),
              "a warp table must keep a third of its slots empty");
constexpr int H_WARPS = 8;
constexpr int32_t H_EMPTY = -1;

template <int CAP, int MAXU> struct HashWarpSmem {
    int32_t keys[CAP];
    double vals[CAP];
    uint64_t list[MAXU + 32]; // (key << 32 | slot) of the distinct keys
    alignas(16) double stage[32];
};

// rows: null for every segment 0..nc-1, else the segments rows[0 .. *nrows)
template <int CAP, int MAXU>
__global__ void __launch_bounds__(H_WARPS * 32) k_rows_hash(
    int64_t nc, const int32_t *__restrict__ rows, const int64_t *__restrict__ nrows,
    const int64_t *__restrict__ rstart, const int32_t *__restrict__ gk,
    const double *__restrict__ gw, int32_t *__restrict__ uk, double *__restrict__ uw,
    int64_t *__restrict__ ucount, int32_t *__restrict__ flag) {
    extern __shared__ unsigned char hsm_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    HashWarpSmem<CAP, MAXU> &S = reinterpret_cast<HashWarpSmem<CAP, MAXU> *>(hsm_raw)[warp];
    const unsigned full = 0xffffffffu, lt = (1u << lane) - 1u;
    const int64_t wg = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t n = rows ? *nrows : nc;
    for (int64_t idx = wg; idx < n; idx += nw) {
        const int64_t row = rows ? rows[idx] : idx;
        const int64_t b = rstart[row];
        const int64_t L = rstart[row + 1] - b;
        if (L <= 32) {
            // one chunk: the leader of each key folds its lanes in lane order (the
            // table path's sum for a key first met in this chunk), and the leaders'
            // (key, sum) pairs are sorted across the lanes; no table needed
            const bool has = lane < L;
            const int32_t k = has ? gk[b + lane] : -2 - lane;
            const double w = has ? gw[b + lane] : 0.0;
            S.stage[lane] = w;
            const unsigned peers = __match_any_sync(full, k);
            __syncwarp();
            const bool lead = has && lane == __ffs(peers) - 1;
            double val = w;
            const unsigned above = peers & ~((2u << lane) - 1u);
            if (lead && above) val = vg_fold_above(val, S.stage, above);
            const int U = __popc(__ballot_sync(full, lead));
            int32_t key = lead ? k : INT_MAX;
#pragma unroll
            for (int k2 = 2; k2 <= 32; k2 <<= 1)
#pragma unroll
                for (int j = k2 >> 1; j > 0; j >>= 1) {
                    const int32_t pk = __shfl_xor_sync(full, key, j);
                    const double pv = __shfl_xor_sync(full, val, j);
                    const bool up = (lane & k2) == 0;
                    const bool low = (lane & j) == 0;
                    const bool take = (low == up) ? (pk < key) : (pk > key);
                    if (take) {
                        key = pk;
                        val = pv;
                    }
                }
            if (lane < U) {
                uk[b + lane] = key;
                uw[b + lane] = val;
            }
            if (lane == 0) {
                ucount[row] = U;
                flag[row] = 0;
            }
            __syncwarp();
            continue;
        }
        int logcap = 5;
        while ((1 << logcap) < 2 * L && (1 << logcap) < CAP) logcap++;
        const int cap = 1 << logcap; // > twice the distinct keys held (at most MAXU + 31)
        for (int s = lane; s < cap; s += 32) S.keys[s] = H_EMPTY;
        __syncwarp();
        int U = 0;
        bool over = false;
        // groups of four 32-entry chunks, the group's loads issued together
        for (int64_t base = 0; base < L && !over; base += 4 * 32) {
            int32_t kq[4];
            double wq[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int64_t i = base + j * 32 + lane;
                kq[j] = -2 - lane; // distinct non-keys for idle lanes
                wq[j] = 0.0;
                if (i < L) {
                    kq[j] = gk[b + i];
                    wq[j] = gw[b + i];
                }
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (base + j * 32 >= L) break; // warp-uniform
                const bool has = base + j * 32 + lane < L;
                const int32_t k = kq[j];
                const double w = wq[j];
                S.stage[lane] = w;
                const unsigned peers = __match_any_sync(full, k);
                __syncwarp();
                bool fresh = false;
                int slot = 0;
                if (has && lane == __ffs(peers) - 1) {
                    uint32_t h = ((uint32_t)k * 2654435761u) >> (32 - logcap);
                    for (;;) {
                        const int32_t kk = S.keys[h];
                        if (kk == k) break;
                        if (kk == H_EMPTY) {
                            const int32_t old = atomicCAS(&S.keys[h], H_EMPTY, k);
                            if (old == H_EMPTY) {
                                fresh = true;
                                break;
                            }
                            if (old == k) break;
                        }
                        h = (h + 1) & (uint32_t)(cap - 1);
                    }
                    slot = (int)h;
                    double acc = fresh ? w : __dadd_rn(S.vals[h], w);
                    const unsigned above = peers & ~((2u << lane) - 1u);
                    if (above) acc = vg_fold_above(acc, S.stage, above);
                    S.vals[h] = acc;
                }
                const unsigned fm = __ballot_sync(full, fresh);
                if (fresh) S.list[U + __popc(fm & lt)] = ((uint64_t)(uint32_t)k << 32) | (uint32_t)slot;
                U += __popc(fm);
                __syncwarp();
                if (U > MAXU) { // too many distinct keys for the table: the next tier
                    over = true;
                    break;
                }
            }
        }
        if (over) {
            if (lane == 0) flag[row] = 1;
            __syncwarp();
            continue;
        }
        if (U <= 32) {
            // bitonic network across the lanes on (key, sum)
            int32_t key = INT_MAX;
            double val = 0.0;
            if (lane < U) {
                const uint64_t e = S.list[lane];
                key = (int32_t)(e >> 32);
                val = S.vals[(uint32_t)e];
            }
#pragma unroll
            for (int k2 = 2; k2 <= 32; k2 <<= 1)
#pragma unroll
                for (int j = k2 >> 1; j > 0; j >>= 1) {
                    const int32_t pk = __shfl_xor_sync(full, key, j);
                    const double pv = __shfl_xor_sync(full, val, j);
                    const bool up = (lane & k2) == 0;
                    const bool low = (lane & j) == 0;
                    // the lower lane of an ascending pair keeps the minimum
                    const bool take = (low == up) ? (pk < key) : (pk > key);
                    if (take) {
                        key = pk;
                        val = pv;
                    }
                }
            if (lane < U) {
                uk[b + lane] = key;
                uw[b + lane] = val;
            }
        } else {
            int n2 = 64;
            while (n2 < U) n2 <<= 1;
            for (int i = U + lane; i < n2; i += 32) S.list[i] = ~0ULL;
            __syncwarp();
            bitonic<true>(S.list, n2, lane, 32);
            for (int i = lane; i < U; i += 32) {
                const uint64_t e = S.list[i];
                uk[b + i] = (int32_t)(e >> 32);
                uw[b + i] = S.vals[(uint32_t)e];
            }
        }
        if (lane == 0) {
            ucount[row] = U;
            flag[row] = 0;
        }
        __syncwarp();
    }
}

// the segments a tier flagged, listed in order (pos: exclusive scan of the flags)
__global__ void k_list_flagged(int64_t nc, const int32_t *__restrict__ flag,
                               const int64_t *__restrict__ pos, int32_t *__restrict__ rows) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nc;
         r += (int64_t)gridDim.x * blockDim.x)
        if (flag[r]) rows[pos[r]] = (int32_t)r;
}

// Segments with more than H_MAXU distinct keys, all together: every entry becomes the key
// (segment rank << kbits | neighbour key) with its index in the grouped arrays as
// payload; one stable radix sort over all of them puts each (segment, key) run in
// segment order, and the run is folded left to right.
__global__ void k_big_rowmap(int64_t nc, const int32_t *__restrict__ flag,
                             const int64_t *__restrict__ bigidx, int32_t *__restrict__ big_row) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nc;
         r += (int64_t)gridDim.x * blockDim.x)
        if (flag[r]) big_row[bigidx[r]] = (int32_t)r;
}

constexpr int BIG_CHUNK = 4096;
constexpr int64_t BIG_RUN_LONG = 1024; // integral weights: longer runs are folded by a warp
constexpr int64_t SEQ_RUN = 128;       // real weights: longer runs go to k_big_fold_seq
constexpr int SEQ_WARPS = 4;           // warps per k_big_fold_seq block

// per segment r: its length and chunk count when flagged (more distinct keys than
// the warp table holds), else 0
__global__ void k_big_prep(int64_t nc, const int32_t *__restrict__ flag,
                           const int64_t *__restrict__ rstart, int64_t *__restrict__ len,
                           int64_t *__restrict__ chunks) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nc;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t L = flag[r] ? rstart[r + 1] - rstart[r] : 0;
        len[r] = L;
        chunks[r] = (L + BIG_CHUNK - 1) / BIG_CHUNK;
    }
}

// one block per chunk of BIG_CHUNK entries of a flagged segment; cb: exclusive
// prefix of the chunk counts over all nc segments (unflagged ones hold none, so the
// largest r with cb[r] <= c owns chunk c); q = bigidx[r] is the segment's rank
// among the flagged ones and leads its sort key; the payload is the entry's index
// inside its segment (the folds add the segment's start back), so a level of 2^32
// or more entries still fits the 32-bit payload
__global__ void k_big_keys(int64_t nc, const int64_t *__restrict__ cb, int64_t nchunks,
                           const int64_t *__restrict__ bigidx, const int64_t *__restrict__ rstart,
                           const int64_t *__restrict__ boff, const int32_t *__restrict__ gk,
                           int kbits, uint64_t *__restrict__ K, uint32_t *__restrict__ V) {
    for (int64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        int64_t lo = 0, hi = nc;
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (cb[mid] <= c) lo = mid;
            else hi = mid;
        }
        const int64_t r = lo, q = bigidx[r];
        const int64_t b = rstart[r], L = rstart[r + 1] - b, o = boff[r];
        const int64_t i0 = (c - cb[r]) * BIG_CHUNK, i1 = min(i0 + BIG_CHUNK, L);
        for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
            K[o + i] = ((uint64_t)q << kbits) | (uint64_t)(uint32_t)gk[b + i];
            V[o + i] = (uint32_t)i;
        }
    }
}

__global__ void k_big_heads(const uint64_t *__restrict__ K, int64_t m, int32_t *__restrict__ h) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x)
        h[i] = (i == 0 || K[i] != K[i - 1]) ? 1 : 0;
}

__global__ void k_big_rowfirst(const uint64_t *__restrict__ K, int64_t m, int kbits,
                               const int64_t *__restrict__ hr, int64_t *__restrict__ rowfirst,
                               int64_t *__restrict__ headpos) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = K[i];
        const uint64_t q = k >> kbits;
        if (i == 0 || (K[i - 1] >> kbits) != q) rowfirst[q] = hr[i];
        if (i == 0 || K[i - 1] != k) headpos[hr[i]] = i;
    }
}

// one thread per run: the run's bounds are known, so its weights are fetched
// eight at a time ahead of the strictly ordered additions; runs longer than
// run_long entries are listed for a warp each (k_big_fold_long, k_big_fold_seq)
__global__ void k_big_fold(const uint64_t *__restrict__ K, const uint32_t *__restrict__ V, int64_t m,
                           int kbits, const int64_t *__restrict__ nheads_dev,
                           const int64_t *__restrict__ headpos,
                           const int64_t *__restrict__ rowfirst, const int32_t *__restrict__ big_row,
                           const int64_t *__restrict__ rstart, const double *__restrict__ gw,
                           int32_t *__restrict__ uk, double *__restrict__ uw,
                           int64_t *__restrict__ long_runs, int64_t long_cap, int64_t run_long,
                           unsigned long long *__restrict__ long_count) {
    const uint64_t mask = ((uint64_t)1 << kbits) - 1;
    const int64_t nheads = *nheads_dev;
    for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < nheads;
         h += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i0 = headpos[h], i1 = h + 1 < nheads ? headpos[h + 1] : m;
        if (long_runs && i1 - i0 > run_long) {
            const unsigned long long sl = atomicAdd(long_count, 1ULL);
            if ((int64_t)sl < long_cap) long_runs[sl] = h;
            continue;
        }
        const uint64_t k = K[i0];
        const uint64_t q = k >> kbits;
        const int64_t seg = rstart[big_row[q]];
        const double *__restrict__ sw = gw + seg; // the segment's weights
        double s = sw[V[i0]];
        int64_t j = i0 + 1;
        for (; j + 8 <= i1; j += 8) {
            double x[8];
#pragma unroll
            for (int t = 0; t < 8; t++) x[t] = sw[V[j + t]];
#pragma unroll
            for (int t = 0; t < 8; t++) s = __dadd_rn(s, x[t]);
        }
        for (; j < i1; j++) s = __dadd_rn(s, sw[V[j]]);
        const int64_t o = seg + (h - rowfirst[q]);
        uk[o] = (int32_t)(k & mask);
        uw[o] = s;
    }
}

// integral weights only (every partial sum exact, so any order gives the same bits):
// the listed runs (longer than BIG_RUN_LONG entries), one warp each, eight partial
// sums per lane
__global__ void k_big_fold_long(const uint64_t *__restrict__ K, const uint32_t *__restrict__ V,
                                int64_t m, int kbits, const int64_t *__restrict__ nheads_dev,
                                const int64_t *__restrict__ headpos,
                                const int64_t *__restrict__ rowfirst, const int32_t *__restrict__ big_row,
                                const int64_t *__restrict__ rstart, const double *__restrict__ gw,
                                int32_t *__restrict__ uk, double *__restrict__ uw,
                                const int64_t *__restrict__ long_runs, int64_t long_cap,
                                const unsigned long long *__restrict__ long_count) {
    const uint64_t mask = ((uint64_t)1 << kbits) - 1;
    const int64_t nheads = *nheads_dev;
    const int64_t nl = min((int64_t)*long_count, long_cap);
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < nl; r += nw) {
        const int64_t h = long_runs[r];
        const int64_t i0 = headpos[h], i1 = h + 1 < nheads ? headpos[h + 1] : m;
        const double *__restrict__ sw = gw + rstart[big_row[K[i0] >> kbits]]; // segment's weights
        double ps[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        int64_t j = i0 + lane;
        for (; j + 7 * 32 < i1; j += 8 * 32) {
#pragma unroll
            for (int t = 0; t < 8; t++) ps[t] = __dadd_rn(ps[t], sw[V[j + t * 32]]);
        }
        for (; j < i1; j += 32) ps[0] = __dadd_rn(ps[0], sw[V[j]]);
#pragma unroll
        for (int t = 1; t < 8; t++) ps[0] = __dadd_rn(ps[0], ps[t]);
        double sum = ps[0];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum = __dadd_rn(sum, __shfl_xor_sync(0xffffffffu, sum, o));
        if (lane == 0) {
            const uint64_t k = K[i0];
            const uint64_t q = k >> kbits;
            const int64_t o = rstart[big_row[q]] + (h - rowfirst[q]);
            uk[o] = (int32_t)(k & mask);
            uw[o] = sum;
        }
    }
}

// real weights: the listed runs (longer than SEQ_RUN entries), one warp each; the
// sum stays one left fold in run order (vg_warp_ordered_fold)
__global__ void k_big_fold_seq(
    const uint64_t *__restrict__ K, const uint32_t *__restrict__ V, int64_t m, int kbits,
    const int64_t *__restrict__ nheads_dev, const int64_t *__restrict__ headpos,
    const int64_t *__restrict__ rowfirst, const int32_t *__restrict__ big_row,
    const int64_t *__restrict__ rstart, const double *__restrict__ gw, int32_t *__restrict__ uk,
    double *__restrict__ uw, const int64_t *__restrict__ long_runs, int64_t long_cap,
    const unsigned long long *__restrict__ long_count) {
    __shared__ double stage[SEQ_WARPS][2 * VG_FOLD_STEP];
    const uint64_t mask = ((uint64_t)1 << kbits) - 1;
    const int64_t nheads = *nheads_dev;
    const int64_t nl = min((int64_t)*long_count, long_cap);
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < nl; r += nw) {
        const int64_t h = long_runs[r];
        const int64_t i0 = headpos[h], i1 = h + 1 < nheads ? headpos[h + 1] : m;
        const double *__restrict__ sw = gw + rstart[big_row[K[i0] >> kbits]]; // segment's weights
        const uint32_t *__restrict__ rv = V + i0;
        const double s = vg_warp_ordered_fold(
            i1 - i0, [sw, rv](int64_t j) { return sw[rv[j]]; }, stage[threadIdx.x >> 5], 0.0, true);
        if ((threadIdx.x & 31) == 0) { // the run's key and place read again: fewer live values
            const uint64_t k = K[i0];
            const uint64_t q = k >> kbits;
            const int64_t o = rstart[big_row[q]] + (h - rowfirst[q]);
            uk[o] = (int32_t)(k & mask);
            uw[o] = s;
        }
    }
}

__global__ void k_big_counts(int64_t nbig, const int32_t *__restrict__ big_row,
                             const int64_t *__restrict__ rowfirst,
                             const int64_t *__restrict__ heads_dev, int64_t *__restrict__ ucount) {
    const int64_t heads = *heads_dev;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nbig;
         q += (int64_t)gridDim.x * blockDim.x)
        ucount[big_row[q]] = (q + 1 < nbig ? rowfirst[q + 1] : heads) - rowfirst[q];
}

template <int G> // lanes per row, as k_group_copy
__global__ void k_compact_rows(int64_t nc, const int64_t *__restrict__ rstart,
                               const int64_t *__restrict__ rowptr, const int32_t *__restrict__ uk,
                               const double *__restrict__ uw, const int32_t *__restrict__ key_to_pos,
                               int32_t *__restrict__ tail, double *__restrict__ w) {
    const int sub = threadIdx.x & (G - 1);
    const int64_t grp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / G;
    const int64_t ng = ((int64_t)gridDim.x * blockDim.x) / G;
    for (int64_t row = grp; row < nc; row += ng) {
        const int64_t s = rstart[row], o = rowptr[row], len = rowptr[row + 1] - o;
        if (len > LONG_ROW) continue;
        for (int64_t j = sub; j < len; j += G) {
            const int32_t k = uk[s + j];
            tail[o + j] = key_to_pos ? key_to_pos[k] : k;
            w[o + j] = uw[s + j];
        }
    }
}

__global__ void k_compact_long(const int64_t *__restrict__ rstart, const int64_t *__restrict__ rowptr,
                               const int32_t *__restrict__ list, const int64_t *__restrict__ cb,
                               const int64_t *__restrict__ cnt, const int32_t *__restrict__ uk,
                               const double *__restrict__ uw, const int32_t *__restrict__ key_to_pos,
                               int32_t *__restrict__ tail, double *__restrict__ w) {
    const int64_t nl = cnt[0], nchunks = cnt[1];
    for (int64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const int64_t q = chunk_owner(cb, nl, c);
        const int64_t row = list[q];
        const int64_t s = rstart[row], o = rowptr[row], len = rowptr[row + 1] - o;
        const int64_t j0 = (c - cb[q]) * COPY_CHUNK, j1 = min(j0 + COPY_CHUNK, len);
        for (int64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
            const int32_t k = uk[s + j];
            tail[o + j] = key_to_pos ? key_to_pos[k] : k;
            w[o + j] = uw[s + j];
        }
    }
}

// The rows of offs (n + 1 offsets, total entries) longer than LONG_ROW with the
// exclusive prefix of their chunk counts, all stream-ordered: the counts stay on
// the device (cnt[0] rows, cnt[1] chunks) for the chunk kernels to read. grid: the
// blocks those kernels take (0 when no row can be long).
struct LongRows {
    DevBuf<int32_t> list;
    DevBuf<int64_t> cb, cnt;
    int grid = 0;
};

void long_rows(vg_ctx *ctx, const int64_t *offs, int64_t n, int64_t total, LongRows &L) {
    const int64_t cap = total / (LONG_ROW + 1);
    if (n == 0 || cap == 0) return;
    L.list.alloc(ctx, cap);
    L.cb.alloc(ctx, cap);
    L.cnt.alloc(ctx, 2);
    VG_CUDA(cudaMemsetAsync(L.cnt.p, 0, 2 * sizeof(int64_t), ctx->stream));
    VG_CUDA(cudaMemsetAsync(L.cb.p, 0, cap * sizeof(int64_t), ctx->stream));
    { LaunchTimer lt(ctx);
      k_long_collect<<<vg_grid(ctx, n, 256), 256, 0, ctx->stream>>>(offs, n, cap, L.list.p, L.cb.p,
                                                                     L.cnt.p); }
    VG_CHECK_LAUNCH();
    vg_scan_i64_async(ctx, L.cb.p, cap, L.cnt.p + 1);
    // each long row has more than COPY_CHUNK entries: chunks <= total / COPY_CHUNK + rows
    L.grid = (int)std::min<int64_t>(total / COPY_CHUNK + cap, 16LL * ctx->sm_count);
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
    const int integral = g->integral == 1 ? 1 : 0; // every weight a small integer
    using SmemS = HashWarpSmem<H_CAP_S, H_MAXU_S>;
    using SmemL = HashWarpSmem<H_CAP, H_MAXU>;
    static bool configured = false;
    if (!configured) {
        VG_CUDA(cudaFuncSetAttribute(k_rows_hash<H_CAP_S, H_MAXU_S>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(H_WARPS * sizeof(SmemS))));
        VG_CUDA(cudaFuncSetAttribute(k_rows_hash<H_CAP, H_MAXU>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(H_WARPS * sizeof(SmemL))));
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
    DevBuf<int64_t> off(ctx, nv + 1), rstart(ctx, nc + 1), src_start(ctx, nv);
    VG_CUDA(cudaMemsetAsync(off.p + nv, 0, sizeof(int64_t), ctx->stream));
    if (nv) {
        { LaunchTimer lt(ctx);
          k_sorted_deg<<<grid, 256, 0, ctx->stream>>>(g->rowptr, vorder.p, nv, off.p,
                                                      src_start.p); }
        VG_CHECK_LAUNCH();
    }
    vg_scan_i64_async(ctx, off.p, nv + 1, nullptr);
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
        if (ne >= LANES32_ROW * nv)
            k_group_copy<32><<<vg_grid(ctx, nv * 32, 256), 256, 0, ctx->stream>>>(
                g->tail, g->weight, src_start.p, off.p, nv, new_key, gk.p, gw.p);
        else
            k_group_copy<8><<<vg_grid(ctx, nv * 8, 256), 256, 0, ctx->stream>>>(
                g->tail, g->weight, src_start.p, off.p, nv, new_key, gk.p, gw.p);
    }
    VG_CHECK_LAUNCH();
    {
        LongRows L;
        long_rows(ctx, off.p, nv, ne, L);
        if (L.grid) {
            LaunchTimer lt(ctx);
            k_group_copy_long<<<L.grid, 256, 0, ctx->stream>>>(g->tail, g->weight, src_start.p,
                                                               off.p, L.list.p, L.cb.p, L.cnt.p,
                                                               new_key, gk.p, gw.p);
        }
        VG_CHECK_LAUNCH();
    }
    vorder.release();
    off.release();
    src_start.release();
    // 4. sort + fold per segment
    DevBuf<int32_t> uk(ctx, ne);
    DevBuf<double> uw(ctx, ne);
    DevBuf<int64_t> ucount(ctx, nc + 1);
    VG_CUDA(cudaMemsetAsync(ucount.p + nc, 0, sizeof(int64_t), ctx->stream));
    DevBuf<int32_t> flag(ctx, nc);
    if (nc) {
        { LaunchTimer lt(ctx);
          k_rows_hash<H_CAP_S, H_MAXU_S>
              <<<vg_grid(ctx, nc * 32, H_WARPS * 32, VG_RH_GRID_S), H_WARPS * 32,
                 H_WARPS * sizeof(SmemS), ctx->stream>>>(nc, nullptr, nullptr, rstart.p, gk.p, gw.p,
                                                         uk.p, uw.p, ucount.p, flag.p); }
        VG_CHECK_LAUNCH();
        {
            // the segments that overflowed the small table, with the large one (their
            // count stays on the device; the grid covers every segment's warp)
            DevBuf<int64_t> fpos(ctx, nc), fcount(ctx, 1);
            DevBuf<int32_t> frows(ctx, nc);
            vg_scan_i32_async(ctx, flag.p, fpos.p, nc, fcount.p);
            { LaunchTimer lt(ctx);
              k_list_flagged<<<vg_grid(ctx, nc, 256), 256, 0, ctx->stream>>>(nc, flag.p, fpos.p,
                                                                              frows.p); }
            VG_CHECK_LAUNCH();
            { LaunchTimer lt(ctx);
              k_rows_hash<H_CAP, H_MAXU>
                  <<<vg_grid(ctx, nc * 32, H_WARPS * 32, VG_RH_GRID), H_WARPS * 32,
                     H_WARPS * sizeof(SmemL), ctx->stream>>>(nc, frows.p, fcount.p, rstart.p, gk.p,
                                                             gw.p, uk.p, uw.p, ucount.p, flag.p); }
            VG_CHECK_LAUNCH();
        }
        // segments with more than H_MAXU distinct keys: one global stable sort. Their
        // count, entries and chunks are scanned on the device and read back together.
        DevBuf<int64_t> bigidx(ctx, nc), boff(ctx, nc), cb(ctx, nc), tot(ctx, 4);
        { LaunchTimer lt(ctx);
          k_big_prep<<<vg_grid(ctx, nc, 256), 256, 0, ctx->stream>>>(nc, flag.p, rstart.p, boff.p,
                                                                     cb.p); }
        VG_CHECK_LAUNCH();
        vg_scan_i32_async(ctx, flag.p, bigidx.p, nc, tot.p);
        vg_scan_i64_async(ctx, boff.p, nc, tot.p + 1);
        vg_scan_i64_async(ctx, cb.p, nc, tot.p + 2);
        int64_t *ht = (int64_t *)vg_pinned(ctx, 3 * sizeof(int64_t));
        VG_CUDA(cudaMemcpyAsync(ht, tot.p, 3 * sizeof(int64_t), cudaMemcpyDeviceToHost,
                                ctx->stream));
        vg_sync(ctx);
        const int64_t nbig = ht[0], m = ht[1], nch = ht[2];
        // the sort's payload indexes inside a segment, and no segment outgrows m
        VG_REQUIRE(m <= (int64_t)UINT32_MAX, "aggregation sorts at most 2^32 - 1 entries (got %lld)",
                   (long long)m);
        if (nbig > 0) {
            DevBuf<int32_t> big_row(ctx, nbig);
            { LaunchTimer lt(ctx);
              k_big_rowmap<<<vg_grid(ctx, nc, 256), 256, 0, ctx->stream>>>(nc, flag.p, bigidx.p,
                                                                           big_row.p); }
            VG_CHECK_LAUNCH();
            int qbits = 1;
            while (qbits < 32 && ((int64_t)1 << qbits) < nbig) qbits++;
            VG_REQUIRE(kbits + qbits <= 64, "aggregation keys need %d bits", kbits + qbits);
            DevBuf<uint64_t> K(ctx, m);
            DevBuf<uint32_t> V(ctx, m);
            { LaunchTimer lt(ctx);
              k_big_keys<<<(int)std::min<int64_t>(nch, 16LL * ctx->sm_count), 256, 0,
                           ctx->stream>>>(nc, cb.p, nch, bigidx.p, rstart.p, boff.p, gk.p, kbits,
                                          K.p, V.p); }
            VG_CHECK_LAUNCH();
            cb.release();
            vg_radix_sort_pairs(ctx, K.p, V.p, m, kbits + qbits);
            // runs of equal (segment, key): their count stays on the device (tot[3]);
            // headpos is sized by its bound m
            DevBuf<int32_t> heads(ctx, m);
            DevBuf<int64_t> hr(ctx, m), rowfirst(ctx, nbig), headpos(ctx, m);
            { LaunchTimer lt(ctx);
              k_big_heads<<<vg_grid(ctx, m, 256), 256, 0, ctx->stream>>>(K.p, m, heads.p); }
            VG_CHECK_LAUNCH();
            vg_scan_i32_async(ctx, heads.p, hr.p, m, tot.p + 3);
            heads.release();
            { LaunchTimer lt(ctx);
              k_big_rowfirst<<<vg_grid(ctx, m, 256), 256, 0, ctx->stream>>>(K.p, m, kbits, hr.p,
                                                                            rowfirst.p, headpos.p); }
            VG_CHECK_LAUNCH();
            hr.release();
            // runs longer than run_long entries are listed for a warp each: integral
            // weights sum them in any order (k_big_fold_long), real weights in order
            // (k_big_fold_seq)
            const int64_t run_long = integral ? BIG_RUN_LONG : SEQ_RUN;
            const int64_t lcap = m / (run_long + 1) + 1;
            DevBuf<int64_t> lruns(ctx, lcap);
            DevBuf<unsigned long long> lcount(ctx, 1);
            VG_CUDA(cudaMemsetAsync(lcount.p, 0, sizeof(unsigned long long), ctx->stream));
            { LaunchTimer lt(ctx);
              k_big_fold<<<vg_grid(ctx, m, 128), 128, 0, ctx->stream>>>(
                  K.p, V.p, m, kbits, tot.p + 3, headpos.p, rowfirst.p, big_row.p, rstart.p, gw.p,
                  uk.p, uw.p, lruns.p, lcap, run_long, lcount.p); }
            VG_CHECK_LAUNCH();
            if (integral) {
                LaunchTimer lt(ctx);
                k_big_fold_long<<<vg_grid(ctx, lcap * 32, 256), 256, 0, ctx->stream>>>(
                    K.p, V.p, m, kbits, tot.p + 3, headpos.p, rowfirst.p, big_row.p, rstart.p, gw.p,
                    uk.p, uw.p, lruns.p, lcap, lcount.p);
            } else {
                LaunchTimer lt(ctx);
                k_big_fold_seq<<<vg_grid(ctx, lcap * 32, SEQ_WARPS * 32), SEQ_WARPS * 32, 0,
                                 ctx->stream>>>(K.p, V.p, m, kbits, tot.p + 3, headpos.p,
                                                rowfirst.p, big_row.p, rstart.p, gw.p, uk.p, uw.p,
                                                lruns.p, lcap, lcount.p);
            }
            VG_CHECK_LAUNCH();
            { LaunchTimer lt(ctx);
              k_big_counts<<<vg_grid(ctx, nbig, 256), 256, 0, ctx->stream>>>(
                  nbig, big_row.p, rowfirst.p, tot.p + 3, ucount.p); }
            VG_CHECK_LAUNCH();
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
        if (m >= LANES32_ROW * nc)
            k_compact_rows<32><<<vg_grid(ctx, nc * 32, 256), 256, 0, ctx->stream>>>(
                nc, rstart.p, ucount.p, uk.p, uw.p, key_to_pos, tail.p, w.p);
        else
            k_compact_rows<8><<<vg_grid(ctx, nc * 8, 256), 256, 0, ctx->stream>>>(
                nc, rstart.p, ucount.p, uk.p, uw.p, key_to_pos, tail.p, w.p);
    }
    VG_CHECK_LAUNCH();
    {
        LongRows L;
        long_rows(ctx, ucount.p, nc, m, L);
        if (L.grid) {
            LaunchTimer lt(ctx);
            k_compact_long<<<L.grid, 256, 0, ctx->stream>>>(rstart.p, ucount.p, L.list.p, L.cb.p,
                                                            L.cnt.p, uk.p, uw.p, key_to_pos, tail.p,
                                                            w.p);
        }
        VG_CHECK_LAUNCH();
    }
    return vg_graph_wrap(ctx, nc, m, ucount.detach(), tail.detach(), w.detach());
}
