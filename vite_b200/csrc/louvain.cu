// One Louvain phase on the device: distLouvainMethod and its early-termination,
// coloring and vertex-ordering variants (louvain.cpp:7-1938), for one rank.
//
// Per iteration:
//   sweep      distExecuteLouvainIteration + distBuildLocalMapCounter +
//              distGetMaxIndex (louvain.cpp:2220-2466), one kernel per degree class
//              over precomputed vertex lists; moves go to FP64/int delta arrays
//              with atomics (the localCupdate of louvain.cpp:2351-2410);
//   apply+mod  distUpdateLocalCinfo + distComputeModularity (louvain.cpp:2468-2547)
//              fused: deltas folded into the community info while the two sums
//              of the modularity are reduced deterministically;
//   swap       pointer rotation (plain) or the early-termination swaps.
// Arithmetic follows the reference's expression order with explicit
// round-to-nearest intrinsics, so no multiply-add is ever fused.
#include "vg_internal.cuh"

#include <algorithm>
#include <climits>
#include <cmath>

namespace {

constexpr int NCLS = 6;
// class by degree: 0: <= TMAX (one thread per vertex) 1: <= 32 (one thread per vertex)
// 2: <= WS_MAXDEG (warp, small shared-memory table) 3: <= WT_MAXDEG (warp, large
// table) 4: <= CT_MAXDEG (CTA, shared table) 5: above (hubs, spread over many CTAs)
constexpr int TMAX = 16;
constexpr int TB = 256;
#ifndef VG_WS_MAXDEG
#define VG_WS_MAXDEG 128
#endif
#ifndef VG_WT_MAXDEG
#define VG_WT_MAXDEG 512
#endif
#ifndef VG_CT_MAXDEG
#define VG_CT_MAXDEG 4096
#endif
#ifndef VG_T32
#define VG_T32 1
#endif
#ifndef VG_T32_GRID
#define VG_T32_GRID 12 // CTAs per SM in the grid of the degree-<=32 list kernel
#endif
#ifndef VG_WS_GRID
#define VG_WS_GRID 4 // CTAs per SM in the grids of the warp kernels
#endif
#ifndef VG_CT_GRID_S
#define VG_CT_GRID_S 8 // CTAs per SM in the grid of the CTA kernel's small table
#endif
#ifndef VG_CT_GRID
#define VG_CT_GRID 2 // CTAs per SM in the grid of the CTA kernel
#endif
#ifndef VG_T16_MINB
#define VG_T16_MINB 3 // resident CTAs per SM of the degree-<=16 list kernel (coloured sweeps)
#endif
#ifndef VG_T32_MINB
#define VG_T32_MINB 4 // resident CTAs per SM the degree-<=32 list kernel is sized for
#endif
constexpr int WS_MAXDEG = VG_WS_MAXDEG;
constexpr int WS_CAP = 256;  // > 2 * WS_MAXDEG - 1: load factor at most one half
constexpr int WS_WARPS = 8;
constexpr int WT_MAXDEG = VG_WT_MAXDEG;
constexpr int WT_CAP = 1024;
constexpr int WT_WARPS = 4;
static_assert(2 * WS_MAXDEG <= WS_CAP && 2 * WT_MAXDEG <= WT_CAP, "warp tables too small");
constexpr int CT_MAXDEG = VG_CT_MAXDEG;
constexpr int CT_CAP = 8192;
constexpr int CT_CAP_S = 2048;
constexpr int CT_THREADS = 256;
constexpr int32_t EMPTY = -1;

// the degree bounds of classes 1-4 (the context's vg_tuning, checked against the
// table capacities above)
struct ClassBounds {
    int32_t t32, ws, wt, ct;
};

__host__ __device__ __forceinline__ int degree_class(int64_t d, const ClassBounds &b) {
    if (d <= TMAX) return 0;
    if (b.t32 && d <= 32) return 1;
    if (d <= b.ws) return 2;
    if (d <= b.wt) return 3;
    if (d <= b.ct) return 4;
    return 5;
}

// community update (localCupdate, Comm of graph.hpp:77-82) packed in 16 bytes so
// that the four atomics of a move land on two sectors
struct __align__(16) CommInfo {
    double deg;
    int32_t size;
    int32_t pad;
};

struct SweepArgs {
    const int64_t *__restrict__ rowptr;
    const int32_t *__restrict__ tail;
    const double *__restrict__ weight;
    const int32_t *__restrict__ curr;
    int32_t *__restrict__ target;
    const double *__restrict__ vdeg;
    const double *__restrict__ cdeg;    // community degree at the start of the sweep
    const int32_t *__restrict__ csize;  // community size at the start of the sweep
    CommInfo *__restrict__ cupd;        // moves of this sweep (localCupdate)
    double *__restrict__ cw;
    double *__restrict__ frozen;
    const uint8_t *__restrict__ active; // nullptr when early termination is off
    const int32_t *__restrict__ ref;     // reference id of each position (null: identity)
    // set on the device when some vertex degree or non-empty community's degree is
    // negative or NaN (then candidate pruning is off); null: pruning off
    const int32_t *__restrict__ noprune;
    int64_t ne;                          // CSR entries (bounds of the vector loads)
    // 1 when every vertex is still in its own community (curr[u] == u: a phase's first
    // iteration, launched directly): the tile kernel then runs its instantiation
    // without community gathers
    int32_t ident;
    double constant;
    // batched graphs (null for one graph): the graph of each vertex, each graph's
    // 1/(2m), and the graphs whose phase has ended (their vertices are skipped)
    const int32_t *__restrict__ vjob = nullptr;
    const double *__restrict__ jconst = nullptr;
    const uint8_t *__restrict__ jdone = nullptr;
};

// the constant of v's graph; false when v belongs to a graph whose phase has ended
__device__ __forceinline__ bool vertex_live(const SweepArgs &a, int32_t v, double &cst) {
    cst = a.constant;
    if (!a.vjob) return true;
    const int32_t j = __ldg(a.vjob + v);
    if (__ldg(a.jdone + j)) return false;
    cst = __ldg(a.jconst + j);
    return true;
}

// gain of moving to a community (louvain.cpp:2263), evaluated in the reference's order
__device__ __forceinline__ double gain_of(double eiy, double eix, double vd, double ay, double ax,
                                          double constant) {
    const double first = __dmul_rn(2.0, __dsub_rn(eiy, eix));
    const double second = __dmul_rn(__dmul_rn(__dmul_rn(2.0, vd), __dsub_rn(ay, ax)), constant);
    return __dsub_rn(first, second);
}

// (gain, id) ordering of distGetMaxIndex: larger gain wins, equal gains go to the
// smaller reference id (looked up only on an exact tie)
__device__ __forceinline__ bool better(bool ok_a, double g_a, int32_t c_a, bool ok_b, double g_b,
                                       int32_t c_b, const int32_t *__restrict__ ref) {
    if (!ok_a) return false;
    if (!ok_b) return true;
    return g_a > g_b || (g_a == g_b && vg_rid(ref, c_a) < vg_rid(ref, c_b));
}

// Candidate pruning (exact). With vd >= 0, a finite constant >= 0 and every
// candidate community's degree ay >= 0 (*noprune == 0), gain_of(eiy, eix, vd, 0, ax,
// constant) is an upper bound of the computed gain for every such ay: each rounding
// step of gain_of is monotone, a larger ay gives a larger (ay - ax), a larger second
// term and a smaller difference. A candidate whose bound is below the best gain found
// so far cannot win (nor tie), so its community degree is never read.
__device__ __forceinline__ bool can_prune(const SweepArgs &a, double vd, double cst) {
    return a.noprune && !__ldg(a.noprune) && vd >= 0.0 && isfinite(vd) && cst >= 0.0 &&
           isfinite(cst);
}

// distGetMaxIndex (louvain.cpp:2220-2279) over one row of a one-thread kernel: the
// communities c[j] whose bit is set in `first` (first occurrences in the row, all
// below dmax), their counters at cnt[j * stride]. With pruning, everything in the
// bound but the counter is fixed for the row and the bound is monotone in it, so the
// two largest counters give the two largest bounds: the candidate with the largest
// is evaluated first and the others only when their bound reaches the best gain
// (the second-largest bound tells when none can). Without pruning, or when the two
// largest bounds are equal (integral weights give many equal counters, and every
// tied candidate must be read anyway), every candidate, eight community-degree loads
// at a time.
template <int T>
__device__ __forceinline__ void best_of_row(const SweepArgs &a, const int32_t (&c)[T],
                                            uint32_t first, int32_t cc, const double *cnt,
                                            int stride, double eix, double vd, double ax,
                                            double cst, int dmax, bool &ok, double &bg,
                                            int32_t &bc) {
    ok = false;
    bg = 0.0;
    bc = INT_MAX;
    if (can_prune(a, vd, cst)) {
        double e1 = -INFINITY, e2 = -INFINITY;
        int32_t uc = -1;
#pragma unroll
        for (int j = 0; j < T; j++) {
            if (j >= dmax) break;
            if (((first >> j) & 1u) && c[j] != cc) {
                const double w = cnt[j * stride];
                if (w > e1) {
                    e2 = e1;
                    e1 = w;
                    uc = c[j];
                } else if (w > e2) {
                    e2 = w;
                }
            }
        }
        if (uc < 0) return;
        const double ub = gain_of(e1, eix, vd, 0.0, ax, cst);
        if (!(ub > 0.0)) return; // no candidate has a positive bound: no move
        const double u2 = e2 == -INFINITY ? -INFINITY : gain_of(e2, eix, vd, 0.0, ax, cst);
        if (u2 < ub) {
            const double g = gain_of(e1, eix, vd, __ldg(a.cdeg + uc), ax, cst);
            if (g > 0.0) {
                ok = true;
                bg = g;
                bc = uc;
            }
            if (!(u2 > 0.0 && (!ok || u2 >= bg))) return; // no other candidate can win
#pragma unroll
            for (int j = 0; j < T; j++) {
                if (j >= dmax) break;
                if (((first >> j) & 1u) && c[j] != cc && c[j] != uc) {
                    const double w = cnt[j * stride];
                    const double u = gain_of(w, eix, vd, 0.0, ax, cst);
                    if (u > 0.0 && (!ok || u >= bg)) {
                        const double g2 = gain_of(w, eix, vd, __ldg(a.cdeg + c[j]), ax, cst);
                        if (g2 > 0.0 && better(true, g2, c[j], ok, bg, bc, a.ref)) {
                            bg = g2;
                            bc = c[j];
                            ok = true;
                        }
                    }
                }
            }
            return;
        }
        // a tie at the top: one round over every candidate below
    }
#pragma unroll
    for (int b = 0; b < T; b += 8) {
        if (b >= dmax) break;
        double ay[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int j = b + q;
            ay[q] = 0.0;
            if (j < T && ((first >> j) & 1u) && c[j] != cc) ay[q] = __ldg(a.cdeg + c[j]);
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int j = b + q;
            if (j < T && ((first >> j) & 1u) && c[j] != cc) {
                const double g = gain_of(cnt[j * stride], eix, vd, ay[q], ax, cst);
                if (g > 0.0 && better(true, g, c[j], ok, bg, bc, a.ref)) {
                    bg = g;
                    bc = c[j];
                    ok = true;
                }
            }
        }
    }
}

// distGetMaxIndex over the candidate slots keys/vals[i], i = base + lane + k * step < nk,
// of one warp (all lanes call it); every lane returns the warp's best (ok, gain, cand).
// With pruning (can_prune) the slot of largest bound is evaluated first and the others
// only when their bound reaches the best gain; without, or when the largest bound is
// shared by two slots, every slot, four community-degree loads per lane at a time. The
// (gain, id) order makes the result independent of the visiting order.
__device__ __forceinline__ void warp_best(const SweepArgs &a, const int32_t *keys,
                                          const double *vals, int64_t base, int64_t step,
                                          int64_t nk, double eix, double vd, double ax, double cst,
                                          bool &ok, double &gain, int32_t &cand) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    ok = false;
    gain = 0.0;
    cand = INT_MAX;
    bool scan_all = true;
    if (can_prune(a, vd, cst)) { // vd and cst are the same in every lane
        scan_all = false;
        double ub = 0.0, u2 = 0.0, uw = 0.0;
        int32_t uc = -1;
        for (int64_t i = base + lane; i < nk; i += step) {
            const double w = vals[i];
            const double u = gain_of(w, eix, vd, 0.0, ax, cst);
            if (u > ub) {
                u2 = ub;
                ub = u;
                uc = keys[i];
                uw = w;
            } else if (u > u2) {
                u2 = u;
            }
        }
        double m = ub;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(full, m, o));
        if (m > 0.0) {
            const int wl = __ffs(__ballot_sync(full, uc >= 0 && ub == m)) - 1;
            double sec = lane == wl ? u2 : ub; // the warp's second-largest bound
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sec = fmax(sec, __shfl_xor_sync(full, sec, o));
            if (sec == m) {
                // a tie at the top (integral weights): one round over every slot
                scan_all = true;
                goto full_scan;
            }
            double g = 0.0;
            if (lane == wl) g = gain_of(uw, eix, vd, __ldg(a.cdeg + uc), ax, cst);
            g = __shfl_sync(full, g, wl);
            const int32_t c0 = __shfl_sync(full, uc, wl);
            if (g > 0.0) {
                ok = true;
                gain = g;
                cand = c0;
            }
            if (sec > 0.0 && (!ok || sec >= gain)) {
                for (int64_t i = base + lane; i < nk; i += step) {
                    const int32_t k = keys[i];
                    if (k == c0) continue;
                    const double w = vals[i];
                    const double u = gain_of(w, eix, vd, 0.0, ax, cst);
                    if (u > 0.0 && (!ok || u >= gain)) {
                        const double gg = gain_of(w, eix, vd, __ldg(a.cdeg + k), ax, cst);
                        if (gg > 0.0 && better(true, gg, k, ok, gain, cand, a.ref)) {
                            gain = gg;
                            cand = k;
                            ok = true;
                        }
                    }
                }
                scan_all = false;
            } else {
                return; // every lane holds the warp's result
            }
        } else {
            return; // no candidate has a positive bound: no move
        }
    }
full_scan:
    if (scan_all) {
        for (int64_t i0 = base; i0 < nk; i0 += 4 * step) {
            int32_t kq[4];
            double aq[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int64_t i = i0 + j * step + lane;
                kq[j] = i < nk ? keys[i] : EMPTY;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) aq[j] = kq[j] != EMPTY ? __ldg(a.cdeg + kq[j]) : 0.0;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (kq[j] == EMPTY) continue;
                const double g = gain_of(vals[i0 + j * step + lane], eix, vd, aq[j], ax, cst);
                if (g > 0.0 && better(true, g, kq[j], ok, gain, cand, a.ref)) {
                    gain = g;
                    cand = kq[j];
                    ok = true;
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double og = __shfl_xor_sync(full, gain, o);
        const int32_t oc = __shfl_xor_sync(full, cand, o);
        const bool ook = __shfl_xor_sync(full, (int)ok, o) != 0;
        if (better(ook, og, oc, ok, gain, cand, a.ref)) {
            gain = og;
            cand = oc;
            ok = true;
        }
    }
}

// the community sizes the singleton rule (louvain.cpp:2275-2276) reads: needed only
// when the chosen community's id is larger than the current one's
__device__ __forceinline__ void sizes_for_rule(const SweepArgs &a, bool ok, int32_t cand, int32_t cc,
                                               int32_t &ccSize, int32_t &csz) {
    ccSize = 0;
    csz = 0;
    if (ok && vg_rid(a.ref, cand) > vg_rid(a.ref, cc)) {
        ccSize = __ldg(a.csize + cc);
        csz = __ldg(a.csize + cand);
    }
}

// decision + bookkeeping shared by all kernels (louvain.cpp:2275-2416)
__device__ __forceinline__ void load_comm(const SweepArgs &a, int32_t c, double &deg, int32_t &size) {
    deg = __ldg(a.cdeg + c);
    size = __ldg(a.csize + c);
}

__device__ __forceinline__ void commit_vertex(const SweepArgs &a, int32_t v, int32_t cc,
                                              int32_t ccSize, double vd, bool has_edges,
                                              double counter0, bool ok, int32_t cand, int32_t csz) {
    int32_t tgt = cc;
    if (has_edges) {
        int32_t maxSize = ccSize;
        if (ok) {
            tgt = cand;
            maxSize = csz;
        }
        if (maxSize == 1 && ccSize == 1 && vg_rid(a.ref, tgt) > vg_rid(a.ref, cc)) tgt = cc;
    }
    const double cwv = has_edges ? counter0 : 0.0;
    a.cw[v] = cwv;
    if (a.active) a.frozen[v] = cwv;
    a.target[v] = tgt;
    if (tgt != cc) {
        atomicAdd(&a.cupd[tgt].deg, vd);
        atomicAdd(&a.cupd[tgt].size, 1);
        atomicAdd(&a.cupd[cc].deg, -vd);
        atomicAdd(&a.cupd[cc].size, -1);
    }
}

// Global -> shared copies that bypass the registers: all of a thread's copies are
// in flight together and complete at cp_async_wait_all (visible to the issuing
// thread; a __syncwarp after the wait publishes them to the warp). The 16-byte
// form needs 16-byte aligned addresses on both sides.
__device__ __forceinline__ void cp_async4(void *dst_smem, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst_smem, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst_smem, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// ---------------------------------------------------------------------------------
// classes 0 and 1: one thread per vertex (degree <= T). All edge loads are issued
// up front (streaming hint on the CSR, read-only path on the gathered arrays);
// each community's counter is the reference's left fold in CSR order,
// accumulated in an interleaved shared-memory slot of the community's first
// occurrence. Candidate degrees are gathered eight at a time.

template <bool LIST, int T, int NT>
__global__ void __launch_bounds__(NT, (T <= 16 ? VG_T16_MINB : VG_T32_MINB)) k_sweep_thread(
    SweepArgs a, const int32_t *__restrict__ list, int64_t count) {
    __shared__ double ssum[T][NT];
    const int tid = threadIdx.x;
    for (int64_t idx = blockIdx.x * (int64_t)NT + tid; idx < count; idx += (int64_t)gridDim.x * NT) {
        const int32_t v = LIST ? list[idx] : (int32_t)idx;
        const int64_t e0 = a.rowptr[v];
        const int d = (int)(a.rowptr[v + 1] - e0);
        if (!LIST && d > T) continue; // the list kernels take the larger degrees
        double cst;
        if (!vertex_live(a, v, cst)) continue;
        if (a.active && !a.active[v]) {
            a.cw[v] = a.frozen[v];
            continue;
        }
        const int32_t cc = __ldg(a.curr + v);
        const double vd = a.vdeg[v];
        const double ccDeg = __ldg(a.cdeg + cc);
        // the 32-slot kernel's loops end at the largest degree among the lanes here (at
        // least each lane's own): they take the same vertex class in position order
        const int dmax = T > 16 ? (int)__reduce_max_sync(__activemask(), (unsigned)d) : T;
        int32_t c[T];
        uint32_t selfm = 0; // bit j: edge j is a self loop
        {
            // weights go straight to the thread's shared-memory slots (asynchronous
            // copies); tails are loaded up front, then their communities gathered
            int32_t t[T];
#pragma unroll
            for (int j = 0; j < T; j++) {
                if (j >= dmax) break;
                t[j] = -1;
                if (j < d) {
                    t[j] = __ldcs(a.tail + e0 + j);
                    cp_async8(&ssum[j][tid], a.weight + e0 + j);
                }
            }
#pragma unroll
            for (int j = 0; j < T; j++) {
                if (j >= dmax) break;
                c[j] = -1;
                if (j < d) {
                    c[j] = __ldg(a.curr + t[j]);
                    if (t[j] == v) selfm |= 1u << j;
                }
            }
        }
        cp_async_wait_all();
        double selfLoop = 0.0;
        if (selfm) {
#pragma unroll
            for (int j = 0; j < T; j++) {
                if (j >= dmax) break;
                if ((selfm >> j) & 1u) selfLoop = __dadd_rn(selfLoop, ssum[j][tid]);
            }
        }
        // counters fold in place at the slot of each community's first occurrence,
        // in CSR order (slot j still holds w_j when edge j is folded: only first
        // occurrences receive additions)
        uint32_t first = 0; // bit j: edge j is the first occurrence of its community
        int j0 = -1;        // first occurrence of the current community
#pragma unroll
        for (int j = 0; j < T; j++) {
            if (j >= dmax) break;
            if (j < d) {
                int fj = j;
#pragma unroll
                for (int k = j - 1; k >= 0; k--)
                    if (c[k] == c[j]) fj = k;
                if (fj == j) {
                    first |= 1u << j;
                    if (c[j] == cc) j0 = j;
                } else {
                    ssum[fj][tid] = __dadd_rn(ssum[fj][tid], ssum[j][tid]);
                }
            }
        }
        const double counter0 = j0 >= 0 ? ssum[j0][tid] : 0.0;
        const double eix = __dsub_rn(counter0, selfLoop);
        const double ax = __dsub_rn(ccDeg, vd);
        double bg;
        int32_t bc;
        bool ok;
        best_of_row<T>(a, c, first, cc, &ssum[0][tid], NT, eix, vd, ax, cst, dmax, ok, bg, bc);
        // the singleton rule (louvain.cpp:2275-2276) needs the sizes only when
        // the winner's id is larger than the current community's
        int32_t ccSize = 0, bs = 0;
        if (ok && vg_rid(a.ref, bc) > vg_rid(a.ref, cc)) {
            ccSize = __ldg(a.csize + cc);
            bs = __ldg(a.csize + bc);
        }
        commit_vertex(a, v, cc, ccSize, vd, d > 0, counter0, ok, bc, bs);
    }
}

// one vertex of a tile (degree d <= T): counters fold in place in the staged
// weights of its row, in CSR order, at the slot of each community's first occurrence
template <int T, bool IDENT>
__device__ __forceinline__ void tile_vertex(const SweepArgs &a, int32_t v, int d, int dmax,
                                            double cst, const int32_t *ts, double *ws, int32_t cc,
                                            double vd, double ccDeg) {
    if (a.active && !a.active[v]) {
        a.cw[v] = a.frozen[v];
        return;
    }
    // every loop stops at dmax, the warp's largest degree (the same in every lane)
    int32_t c[T];
    uint32_t selfm = 0; // bit j: edge j is a self loop
#pragma unroll
    for (int j = 0; j < T; j++) {
        if (j >= dmax) break;
        c[j] = -1;
        if (j < d) {
            const int32_t t = ts[j];
            c[j] = IDENT ? t : __ldg(a.curr + t);
            if (t == v) selfm |= 1u << j;
        }
    }
    double selfLoop = 0.0;
    if (selfm) {
#pragma unroll
        for (int j = 0; j < T; j++) {
            if (j >= dmax) break;
            if ((selfm >> j) & 1u) selfLoop = __dadd_rn(selfLoop, ws[j]);
        }
    }
    uint32_t first = 0;
    int j0 = -1; // first occurrence of the current community
#pragma unroll
    for (int j = 0; j < T; j++) {
        if (j >= dmax) break;
        if (j < d) {
            int fj = j;
#pragma unroll
            for (int k = j - 1; k >= 0; k--)
                if (c[k] == c[j]) fj = k;
            if (fj == j) {
                first |= 1u << j;
                if (c[j] == cc) j0 = j;
            } else {
                ws[fj] = __dadd_rn(ws[fj], ws[j]);
            }
        }
    }
    const double counter0 = j0 >= 0 ? ws[j0] : 0.0;
    const double eix = __dsub_rn(counter0, selfLoop);
    const double ax = __dsub_rn(ccDeg, vd);
    double bg;
    int32_t bc;
    bool ok;
    best_of_row<T>(a, c, first, cc, ws, 1, eix, vd, ax, cst, dmax, ok, bg, bc);
    int32_t ccSize = 0, bs = 0;
    if (ok && vg_rid(a.ref, bc) > vg_rid(a.ref, cc)) {
        ccSize = __ldg(a.csize + cc);
        bs = __ldg(a.csize + bc);
    }
    commit_vertex(a, v, cc, ccSize, vd, d > 0, counter0, ok, bc, bs);
}

// ---------------------------------------------------------------------------------
// class 0 in vertex order: a warp takes a tile of 32 consecutive vertices, whose
// rows form one contiguous edge range, and stages that range into shared memory
// with coalesced 128-bit loads; each lane then works on its own vertex from shared
// memory. Counters fold in place, in the staged weights of the lane's row, in
// CSR order (slot of the community's first occurrence). A range longer than the
// staging buffer falls back to per-lane copies of the (short) rows.

constexpr int TILE_CAP = 504;          // staged edges per warp (48 KB of shared memory per CTA)
#ifndef VG_TILE_WARPS
#define VG_TILE_WARPS 8
#endif
#ifndef VG_TILE_MINB
#define VG_TILE_MINB 4 // resident CTAs per SM the register budget is sized for
#endif
#ifndef VG_TILE_GRID
#define VG_TILE_GRID 64 // CTAs per SM in the grid (grid-stride; more CTAs balance the tail)
#endif
constexpr int TILE_WARPS = VG_TILE_WARPS;

template <int T, bool IDENT>
__global__ void __launch_bounds__(TILE_WARPS * 32, VG_TILE_MINB) k_sweep_tile(SweepArgs a, int64_t nv) {
    static_assert(32 * T <= TILE_CAP + 8, "the per-lane fallback layout must fit the buffer");
    __shared__ __align__(16) int32_t st_all[TILE_WARPS][TILE_CAP + 8];
    __shared__ __align__(16) double sw_all[TILE_WARPS][TILE_CAP + 8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t *st = st_all[warp];
    double *sw = sw_all[warp];
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t tile = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile * 32 < nv;
         tile += nwarps) {
        const int64_t v64 = tile * 32 + lane;
        const int32_t v = (int32_t)v64;
        const bool valid = v64 < nv;
        double cst = a.constant;
        const bool live = valid && vertex_live(a, v, cst);
        if (!__any_sync(0xffffffffu, live)) continue;
        int64_t e0 = 0, e1 = 0;
        if (valid) {
            e0 = a.rowptr[v];
            e1 = a.rowptr[v + 1];
        }
        const int d = (int)(e1 - e0);
        const unsigned vm = __ballot_sync(0xffffffffu, valid);
        const int last = 31 - __clz(vm);
        const int64_t E0 = __shfl_sync(0xffffffffu, e0, 0);
        const int64_t E1 = __shfl_sync(0xffffffffu, e1, last);
        const int64_t A0 = E0 & ~3LL, B0 = E0 & ~1LL;
        int off_t, off_w; // where this lane's row starts in st / sw
        if (E1 - A0 <= TILE_CAP) {
            // coalesced 16-byte copies (16-byte aligned starts), all in flight at once
            const int64_t nt = (E1 - A0 + 3) >> 2, nw2 = (E1 - B0 + 1) >> 1;
            for (int64_t k = lane; k < nt; k += 32) {
                const int64_t i = A0 + 4 * k;
                if (i + 4 <= a.ne) {
                    cp_async16(st + 4 * k, a.tail + i);
                } else {
                    for (int q = 0; q < 4 && i + q < a.ne; q++) cp_async4(st + 4 * k + q, a.tail + i + q);
                }
            }
            for (int64_t k = lane; k < nw2; k += 32) {
                const int64_t i = B0 + 2 * k;
                if (i + 2 <= a.ne) {
                    cp_async16(sw + 2 * k, a.weight + i);
                } else if (i < a.ne) {
                    cp_async8(sw + 2 * k, a.weight + i);
                }
            }
            off_t = (int)(e0 - A0);
            off_w = (int)(e0 - B0);
        } else {
            // long range (hub rows inside the tile): each lane copies its own short row
            if (live && d <= T) {
                for (int j = 0; j < d; j++) {
                    cp_async4(st + lane * T + j, a.tail + e0 + j);
                    cp_async8(sw + lane * T + j, a.weight + e0 + j);
                }
            }
            off_t = lane * T;
            off_w = lane * T;
        }
        // the vertex's own community, degree and community degree do not depend on
        // the staged row: their loads overlap the staging copies
        int32_t cc = 0;
        double vd = 0.0, ccDeg = 0.0;
        if (live && d <= T) {
            cc = IDENT ? v : __ldg(a.curr + v);
            vd = a.vdeg[v];
            ccDeg = __ldg(a.cdeg + cc);
        }
        const int dmax = (int)__reduce_max_sync(0xffffffffu, (live && d <= T) ? (unsigned)d : 0u);
        cp_async_wait_all();
        __syncwarp();
        if (live && d <= T)
            tile_vertex<T, IDENT>(a, v, d, dmax, cst, st + off_t, sw + off_w, cc, vd, ccDeg);
        __syncwarp();
    }
}

// open addressing: multiplicative hash, linear probing
__device__ __forceinline__ uint32_t slot_hash(int32_t c, int logcap) {
    return ((uint32_t)c * 2654435761u) >> (32 - logcap);
}

// ---------------------------------------------------------------------------------
// class 4: one warp per vertex, table in shared memory private to the warp.
// Chunks of 32 edges; inside a chunk one leader per community folds its lanes'
// weights in CSR order onto the table value, so each counter is the reference's
// exact left fold.

// shared memory of a k_sweep_warp block: vals[WARPS][CAP], keys[WARPS][CAP], stage[WARPS][32]
template <int CAP, int WARPS> constexpr size_t warp_smem_bytes() {
    return (size_t)WARPS * CAP * (sizeof(double) + sizeof(int32_t)) + (size_t)WARPS * 32 * sizeof(double);
}

template <int CAP, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, CAP <= 256 ? 4 : 1) k_sweep_warp(
    SweepArgs a, const int32_t *__restrict__ list, int64_t count) {
    extern __shared__ unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *vals = reinterpret_cast<double *>(smem_raw) + (size_t)warp * CAP;
    int32_t *keys = reinterpret_cast<int32_t *>(reinterpret_cast<double *>(smem_raw) +
                                                (size_t)WARPS * CAP) +
                    (size_t)warp * CAP;
    double *stage = reinterpret_cast<double *>(reinterpret_cast<int32_t *>(
                        reinterpret_cast<double *>(smem_raw) + (size_t)WARPS * CAP) +
                                               (size_t)WARPS * CAP) +
                    (size_t)warp * 32;
    const unsigned full = 0xffffffffu;
    const int64_t wg = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t idx = wg; idx < count; idx += nw) {
        const int32_t v = list[idx];
        double cst;
        if (!vertex_live(a, v, cst)) continue;
        const int32_t cc = a.curr[v];
        if (a.active && !a.active[v]) {
            if (lane == 0) a.cw[v] = a.frozen[v];
            continue;
        }
        const int64_t e0 = a.rowptr[v];
        const int d = (int)(a.rowptr[v + 1] - e0);
        int logcap = 5;
        while ((1 << logcap) < 2 * d) logcap++;
        const int cap = 1 << logcap;
        for (int s = lane; s < cap; s += 32) keys[s] = EMPTY;
        __syncwarp();
        double selfLoop = 0.0;
        // groups of four 32-edge chunks: the group's tails and weights are loaded
        // together, then their communities, so a group costs two round trips
        for (int g0 = 0; g0 < d; g0 += 4 * 32) {
            int32_t tt[4], cg[4];
            double ww[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int k = g0 + j * 32 + lane;
                tt[j] = k < d ? a.tail[e0 + k] : -1;
                ww[j] = k < d ? a.weight[e0 + k] : 0.0;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) cg[j] = tt[j] >= 0 ? a.curr[tt[j]] : -1;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (g0 + j * 32 >= d) break; // warp-uniform
                const bool has = tt[j] >= 0;
                const int32_t t = tt[j], c = cg[j];
                stage[lane] = ww[j];
                const unsigned peers = __match_any_sync(full, has ? c : (-1 - lane));
                __syncwarp();
                if (has && lane == __ffs(peers) - 1) {
                    uint32_t h = slot_hash(c, logcap);
                    bool fresh = false;
                    for (;;) {
                        const int32_t kk = keys[h];
                        if (kk == c) break;
                        if (kk == EMPTY) {
                            const int32_t old = atomicCAS(&keys[h], EMPTY, c);
                            if (old == EMPTY) {
                                fresh = true;
                                break;
                            }
                            if (old == c) break;
                        }
                        h = (h + 1) & (cap - 1);
                    }
                    const unsigned above = peers & ~((2u << lane) - 1u);
                    double acc = fresh ? stage[lane] : __dadd_rn(vals[h], stage[lane]);
                    if (above) acc = vg_fold_above(acc, stage, above);
                    vals[h] = acc;
                }
                const unsigned selfm = __ballot_sync(full, has && t == v);
                {
                    unsigned m = selfm;
                    while (m) {
                        const int b = __ffs(m) - 1;
                        selfLoop = __dadd_rn(selfLoop, stage[b]);
                        m &= m - 1;
                    }
                }
                __syncwarp();
            }
        }
        // counter[0]: the current community's entry, if any neighbour is in it
        double counter0 = 0.0;
        {
            uint32_t h = slot_hash(cc, logcap);
            for (int probe = 0; probe < cap; probe++) {
                const int32_t kk = keys[h];
                if (kk == cc) {
                    counter0 = vals[h];
                    break;
                }
                if (kk == EMPTY) break;
                h = (h + 1) & (cap - 1);
            }
        }
        // the other communities, compacted to the front of the table: a kept slot
        // moves to the count of kept slots before it, never past a slot not yet read
        int nk = 0;
        for (int base = 0; base < cap; base += 32) {
            const int32_t kk = keys[base + lane];
            const double vv = vals[base + lane];
            const bool keep = kk != EMPTY && kk != cc;
            const unsigned bm = __ballot_sync(full, keep);
            __syncwarp();
            if (keep) {
                const int dst = nk + __popc(bm & ((1u << lane) - 1u));
                keys[dst] = kk;
                vals[dst] = vv;
            }
            nk += __popc(bm);
            __syncwarp();
        }
        const double vd = a.vdeg[v];
        const double ccDeg = __ldg(a.cdeg + cc);
        const double eix = __dsub_rn(counter0, selfLoop);
        const double ax = __dsub_rn(ccDeg, vd);
        double gain;
        int32_t cand;
        bool ok;
        warp_best(a, keys, vals, 0, 32, nk, eix, vd, ax, cst, ok, gain, cand);
        if (lane == 0) {
            int32_t ccSize, csz;
            sizes_for_rule(a, ok, cand, cc, ccSize, csz);
            commit_vertex(a, v, cc, ccSize, vd, d > 0, counter0, ok, cand, csz);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------
// classes 5-6: one CTA per vertex. Warps take 32-edge slices of each 256-edge
// chunk; inside a slice the leader folds its lanes in CSR order, and the slices
// meet in the table through atomics (table in shared memory, or in a global
// scratch region per CTA for the largest degrees).

struct CtaShared {
    double red_g[CT_THREADS / 32];
    int32_t red_c[CT_THREADS / 32];
    int red_ok[CT_THREADS / 32];
    double self_part[CT_THREADS / 32];
    double counter0;
};

// CAP: the table's slots. The class runs as two launches over the same list, a
// table of CT_CAP_S slots for the rows of at most CT_CAP_S / 2 entries (more CTAs fit
// per SM) and one of CT_CAP slots for the longer ones; each skips the other's rows.
template <int CAP>
__global__ void __launch_bounds__(CT_THREADS) k_sweep_cta(SweepArgs a, const int32_t *__restrict__ list,
                                                          int64_t count) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ CtaShared sh;
    __shared__ __align__(16) double stage[CT_THREADS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    double *vals = reinterpret_cast<double *>(smem_raw);
    int32_t *keys = reinterpret_cast<int32_t *>(vals + CAP);
    for (int64_t idx = blockIdx.x; idx < count; idx += gridDim.x) {
        const int32_t v = list[idx];
        const int64_t e0 = a.rowptr[v];
        const int64_t d = a.rowptr[v + 1] - e0;
        if ((CAP == CT_CAP) != (d > CT_CAP_S / 2)) continue; // the other launch's row
        double cst;
        if (!vertex_live(a, v, cst)) continue;
        const int32_t cc = a.curr[v];
        if (a.active && !a.active[v]) {
            if (threadIdx.x == 0) a.cw[v] = a.frozen[v];
            continue;
        }
        int logcap = 5;
        while (((int64_t)1 << logcap) < 2 * d) logcap++;
        const int64_t cap = (int64_t)1 << logcap;
        for (int64_t s = threadIdx.x; s < cap; s += CT_THREADS) {
            keys[s] = EMPTY;
            vals[s] = 0.0;
        }
        double selfLoop = 0.0; // per-warp partial, in CSR order inside the warp's slices
        __syncthreads();
        for (int64_t off = 0; off < d; off += CT_THREADS) {
            const int64_t k = off + threadIdx.x;
            const bool has = k < d;
            int32_t t = -1, c = -1;
            double w = 0.0;
            if (has) {
                t = a.tail[e0 + k];
                w = a.weight[e0 + k];
                c = a.curr[t];
            }
            stage[threadIdx.x] = w;
            const unsigned peers = __match_any_sync(full, has ? c : (-1 - lane));
            __syncwarp();
            if (has && lane == __ffs(peers) - 1) {
                double acc = stage[threadIdx.x];
                const unsigned above = peers & ~((2u << lane) - 1u);
                if (above) acc = vg_fold_above(acc, stage + (threadIdx.x & ~31), above);
                uint32_t h = slot_hash(c, logcap);
                for (;;) {
                    const int32_t kk = keys[h];
                    if (kk == c) break;
                    if (kk == EMPTY) {
                        const int32_t old = atomicCAS(&keys[h], EMPTY, c);
                        if (old == EMPTY || old == c) break;
                    }
                    h = (h + 1) & (uint32_t)(cap - 1);
                }
                atomicAdd(&vals[h], acc);
            }
            const unsigned selfm = __ballot_sync(full, has && t == v);
            {
                unsigned m = selfm;
                while (m) {
                    const int b = __ffs(m) - 1;
                    selfLoop = __dadd_rn(selfLoop, stage[(threadIdx.x & ~31) + b]);
                    m &= m - 1;
                }
            }
            __syncwarp();
        }
        if (lane == 0) sh.self_part[warp] = selfLoop;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int w = 0; w < CT_THREADS / 32; w++) s = __dadd_rn(s, sh.self_part[w]);
            sh.self_part[0] = s;
            double c0 = 0.0;
            uint32_t h = slot_hash(cc, logcap);
            for (int64_t probe = 0; probe < cap; probe++) {
                const int32_t kk = keys[h];
                if (kk == cc) {
                    c0 = vals[h];
                    break;
                }
                if (kk == EMPTY) break;
                h = (h + 1) & (uint32_t)(cap - 1);
            }
            sh.counter0 = c0;
        }
        __syncthreads();
        const double counter0 = sh.counter0;
        selfLoop = sh.self_part[0];
        const double vd = a.vdeg[v];
        const double ccDeg = __ldg(a.cdeg + cc);
        const double eix = __dsub_rn(counter0, selfLoop);
        const double ax = __dsub_rn(ccDeg, vd);
        double gain;
        int32_t cand;
        bool ok;
        // the other communities, compacted to the front of the table in slot order:
        // a kept slot moves to the count of kept slots before it, so no write lands
        // on a slot not yet read (each group's reads end at the barrier before its
        // writes)
        int64_t nk = 0;
        for (int64_t base = 0; base < cap; base += CT_THREADS) {
            const int64_t s = base + threadIdx.x;
            const int32_t kk = s < cap ? keys[s] : EMPTY;
            const double vv = s < cap ? vals[s] : 0.0;
            const bool keep = kk != EMPTY && kk != cc;
            const unsigned bm = __ballot_sync(full, keep);
            if (lane == 0) sh.red_c[warp] = __popc(bm);
            __syncthreads();
            int before = 0, tot = 0;
#pragma unroll
            for (int w = 0; w < CT_THREADS / 32; w++) {
                const int c = sh.red_c[w];
                before += w < warp ? c : 0;
                tot += c;
            }
            if (keep) {
                const int64_t dst = nk + before + __popc(bm & ((1u << lane) - 1u));
                keys[dst] = kk;
                vals[dst] = vv;
            }
            nk += tot;
            __syncthreads();
        }
        // each warp its own slots (warp * 32 + lane + k * CT_THREADS), then the warps' bests
        warp_best(a, keys, vals, warp * 32, CT_THREADS, nk, eix, vd, ax, cst, ok, gain, cand);
        if (lane == 0) {
            sh.red_g[warp] = gain;
            sh.red_c[warp] = cand;
            sh.red_ok[warp] = ok;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < CT_THREADS / 32; w++) {
                if (better(sh.red_ok[w] != 0, sh.red_g[w], sh.red_c[w], ok, gain, cand, a.ref)) {
                    gain = sh.red_g[w];
                    cand = sh.red_c[w];
                    ok = true;
                }
            }
            int32_t ccSize, csz;
            sizes_for_rule(a, ok, cand, cc, ccSize, csz);
            commit_vertex(a, v, cc, ccSize, vd, d > 0, counter0, ok, cand, csz);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------
// class 5 (degree > CT_MAXDEG, the hubs): every hub's row is spread over many CTAs.
// Each hub owns a hash table in global memory (capacity the power of two >= twice its
// degree, so at most half full). k_hub_accum: work items are chunks of HUB_CHUNK
// entries of any hub; inside a warp's 32 entries the leader of each community folds
// its lanes in lane order and the warps meet in the table through atomics (as the
// CTA class does for its slices). k_hub_c0: the current community's counter.
// k_hub_eval: work items are slices of HUB_SLICE table slots; each slice reports
// its best (gain, id) and clears its slots for the next sweep. k_hub_commit: a warp
// per hub picks the best of its slices (the (gain, id) order makes the choice
// independent of the slices' order) and commits the move.

constexpr int HUB_CHUNK = 4096;
constexpr int HUB_SLICE = 4096;
constexpr int HUB_THREADS = 256;

struct HubBest {
    double g;
    int32_t c, sz;
    int32_t ok, pad;
};

// largest q in [q0, q1) with pre[q] <= x (pre nondecreasing, pre[q0] <= x)
__device__ __forceinline__ int64_t hub_owner(const int64_t *__restrict__ pre, int64_t q0, int64_t q1,
                                             int64_t x) {
    int64_t lo = q0, hi = q1;
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (pre[mid] <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ bool hub_swept(const SweepArgs &a, int32_t v, double &cst) {
    return vertex_live(a, v, cst) && !(a.active && !a.active[v]);
}

__global__ void __launch_bounds__(HUB_THREADS) k_hub_accum(
    SweepArgs a, const int32_t *__restrict__ vtx, const int64_t *__restrict__ toff,
    const int64_t *__restrict__ cb, int64_t q0, int64_t q1, int32_t *__restrict__ keys,
    double *__restrict__ vals, double *__restrict__ self) {
    __shared__ __align__(16) double stage[HUB_THREADS];
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    double *st = stage + (threadIdx.x & ~31);
    for (int64_t c = cb[q0] + blockIdx.x; c < cb[q1]; c += gridDim.x) {
        const int64_t q = hub_owner(cb, q0, q1, c);
        const int32_t v = vtx[q];
        double cst;
        if (!hub_swept(a, v, cst)) continue; // uniform over the block
        const int64_t r0 = a.rowptr[v], r1 = a.rowptr[v + 1];
        const int64_t e0 = r0 + (c - cb[q]) * HUB_CHUNK, e1 = min(e0 + HUB_CHUNK, r1);
        const int64_t cap = toff[q + 1] - toff[q];
        int logcap = 0;
        while (((int64_t)1 << logcap) < cap) logcap++;
        int32_t *hk = keys + toff[q];
        double *hv = vals + toff[q];
        double selfsum = 0.0;
        bool anyself = false;
        for (int64_t base = e0; base < e1; base += HUB_THREADS) {
            const int64_t e = base + threadIdx.x;
            const bool has = e < e1;
            int32_t t = -1, cm = -1;
            double w = 0.0;
            if (has) {
                t = a.tail[e];
                w = a.weight[e];
                cm = a.curr[t];
            }
            st[lane] = w;
            const unsigned peers = __match_any_sync(full, has ? cm : (-1 - lane));
            __syncwarp();
            if (has && lane == __ffs(peers) - 1) {
                double acc = w;
                const unsigned above = peers & ~((2u << lane) - 1u);
                if (above) acc = vg_fold_above(acc, st, above);
                uint32_t h = slot_hash(cm, logcap);
                for (;;) {
                    const int32_t kk = hk[h];
                    if (kk == cm) break;
                    if (kk == EMPTY) {
                        const int32_t old = atomicCAS(&hk[h], EMPTY, cm);
                        if (old == EMPTY || old == cm) break;
                    }
                    h = (h + 1) & (uint32_t)(cap - 1);
                }
                atomicAdd(&hv[h], acc);
            }
            unsigned m = __ballot_sync(full, has && t == v);
            anyself |= m != 0;
            while (m) {
                const int b = __ffs(m) - 1;
                selfsum = __dadd_rn(selfsum, st[b]);
                m &= m - 1;
            }
            __syncwarp();
        }
        if (lane == 0 && anyself) atomicAdd(&self[q], selfsum);
    }
}

__global__ void k_hub_c0(SweepArgs a, const int32_t *__restrict__ vtx, const int64_t *__restrict__ toff,
                         int64_t q0, int64_t q1, const int32_t *__restrict__ keys,
                         const double *__restrict__ vals, double *__restrict__ c0) {
    for (int64_t q = q0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < q1;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = vtx[q];
        double cst;
        if (!hub_swept(a, v, cst)) continue;
        const int32_t cc = a.curr[v];
        const int64_t cap = toff[q + 1] - toff[q];
        int logcap = 0;
        while (((int64_t)1 << logcap) < cap) logcap++;
        const int32_t *hk = keys + toff[q];
        double x = 0.0;
        uint32_t h = slot_hash(cc, logcap);
        for (int64_t probe = 0; probe < cap; probe++) {
            const int32_t kk = hk[h];
            if (kk == cc) {
                x = vals[toff[q] + h];
                break;
            }
            if (kk == EMPTY) break;
            h = (h + 1) & (uint32_t)(cap - 1);
        }
        c0[q] = x;
    }
}

__global__ void __launch_bounds__(HUB_THREADS) k_hub_eval(
    SweepArgs a, const int32_t *__restrict__ vtx, const int64_t *__restrict__ toff,
    const int64_t *__restrict__ sb, int64_t q0, int64_t q1, int32_t *__restrict__ keys,
    double *__restrict__ vals, const double *__restrict__ self, const double *__restrict__ c0,
    HubBest *__restrict__ best) {
    __shared__ double red_g[HUB_THREADS / 32];
    __shared__ int32_t red_c[HUB_THREADS / 32], red_s[HUB_THREADS / 32], red_ok[HUB_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned full = 0xffffffffu;
    for (int64_t sl = sb[q0] + blockIdx.x; sl < sb[q1]; sl += gridDim.x) {
        const int64_t q = hub_owner(sb, q0, q1, sl);
        const int32_t v = vtx[q];
        double cst;
        if (!hub_swept(a, v, cst)) continue; // its table was left empty
        const int32_t cc = a.curr[v];
        const double vd = a.vdeg[v];
        const double eix = __dsub_rn(c0[q], self[q]);
        const double ax = __dsub_rn(__ldg(a.cdeg + cc), vd);
        const int64_t s0 = toff[q] + (sl - sb[q]) * HUB_SLICE;
        double gain = 0.0;
        int32_t cand = INT_MAX, csz = 0;
        bool ok = false;
        // four slots per thread per round, their community loads issued together
        for (int64_t r = 0; r < HUB_SLICE; r += 4 * HUB_THREADS) {
            int32_t kq[4], sq[4];
            double vq[4], aq[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int64_t sidx = s0 + r + j * HUB_THREADS + threadIdx.x;
                kq[j] = keys[sidx];
                vq[j] = vals[sidx];
                if (kq[j] != EMPTY) {
                    keys[sidx] = EMPTY; // clean for the next sweep
                    vals[sidx] = 0.0;
                }
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                aq[j] = 0.0;
                sq[j] = 0;
                if (kq[j] != EMPTY && kq[j] != cc) load_comm(a, kq[j], aq[j], sq[j]);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (kq[j] == EMPTY || kq[j] == cc) continue;
                const double g = gain_of(vq[j], eix, vd, aq[j], ax, cst);
                if (g > 0.0 && better(true, g, kq[j], ok, gain, cand, a.ref)) {
                    gain = g;
                    cand = kq[j];
                    csz = sq[j];
                    ok = true;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double og = __shfl_xor_sync(full, gain, o);
            const int32_t oc = __shfl_xor_sync(full, cand, o);
            const int32_t os = __shfl_xor_sync(full, csz, o);
            const bool ook = __shfl_xor_sync(full, (int)ok, o) != 0;
            if (better(ook, og, oc, ok, gain, cand, a.ref)) {
                gain = og;
                cand = oc;
                csz = os;
                ok = true;
            }
        }
        if (lane == 0) {
            red_g[warp] = gain;
            red_c[warp] = cand;
            red_s[warp] = csz;
            red_ok[warp] = ok;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < HUB_THREADS / 32; w++) {
                if (better(red_ok[w] != 0, red_g[w], red_c[w], ok, gain, cand, a.ref)) {
                    gain = red_g[w];
                    cand = red_c[w];
                    csz = red_s[w];
                    ok = true;
                }
            }
            HubBest b;
            b.g = gain;
            b.c = cand;
            b.sz = csz;
            b.ok = ok;
            b.pad = 0;
            best[sl] = b;
        }
        __syncthreads();
    }
}

__global__ void k_hub_commit(SweepArgs a, const int32_t *__restrict__ vtx, const int64_t *__restrict__ sb,
                             int64_t q0, int64_t q1, double *__restrict__ self,
                             const double *__restrict__ c0, const HubBest *__restrict__ best) {
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t q = q0 + ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5); q < q1; q += nw) {
        const int32_t v = vtx[q];
        double cst;
        if (!vertex_live(a, v, cst)) continue;
        if (a.active && !a.active[v]) {
            if (lane == 0) a.cw[v] = a.frozen[v];
            continue;
        }
        double gain = 0.0;
        int32_t cand = INT_MAX, csz = 0;
        bool ok = false;
        for (int64_t sl = sb[q] + lane; sl < sb[q + 1]; sl += 32) {
            const HubBest b = best[sl];
            if (better(b.ok != 0, b.g, b.c, ok, gain, cand, a.ref)) {
                gain = b.g;
                cand = b.c;
                csz = b.sz;
                ok = true;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double og = __shfl_xor_sync(full, gain, o);
            const int32_t oc = __shfl_xor_sync(full, cand, o);
            const int32_t os = __shfl_xor_sync(full, csz, o);
            const bool ook = __shfl_xor_sync(full, (int)ok, o) != 0;
            if (better(ook, og, oc, ok, gain, cand, a.ref)) {
                gain = og;
                cand = oc;
                csz = os;
                ok = true;
            }
        }
        if (lane == 0) {
            const int32_t cc = a.curr[v];
            const int32_t ccSize = __ldg(a.csize + cc);
            commit_vertex(a, v, cc, ccSize, a.vdeg[v], true, c0[q], ok, cand, csz);
            self[q] = 0.0; // for the next sweep
        }
    }
}

// per listed hub: its degree -> table capacity, accumulation chunks, evaluation slices
__global__ void k_hub_plan(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ list,
                           int64_t n, int32_t *__restrict__ vtx, int64_t *__restrict__ cap,
                           int64_t *__restrict__ chunks, int64_t *__restrict__ slices) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = list[q];
        const int64_t d = rowptr[v + 1] - rowptr[v];
        int64_t c = HUB_SLICE;
        while (c < 2 * d) c <<= 1;
        vtx[q] = v;
        cap[q] = c;
        chunks[q] = (d + HUB_CHUNK - 1) / HUB_CHUNK;
        slices[q] = c / HUB_SLICE;
    }
}

// ---------------------------------------------------------------------------------
// init, degree, apply + modularity, swaps

// distSumVertexDegree (louvain.cpp:2161-2186): each row summed in CSR order, one
// row per lane, its loads issued eight at a time ahead of the ordered additions.
// With integral weights every order gives the same exact sum, so a warp adds the
// rows longer than DEG_LONG together as trees (no lane waits on a hub row).
constexpr int DEG_LONG = 64;

__device__ __forceinline__ double row_fold(const double *__restrict__ w, int64_t e0, int64_t e1) {
    double sum = 0.0;
    int64_t k = e0;
    for (; k + 8 <= e1; k += 8) {
        double x[8];
#pragma unroll
        for (int t = 0; t < 8; t++) x[t] = w[k + t];
#pragma unroll
        for (int t = 0; t < 8; t++) sum = __dadd_rn(sum, x[t]);
    }
    for (; k < e1; k++) sum = __dadd_rn(sum, w[k]);
    return sum;
}

// With integral weights, rows longer than DEG_HUGE (the hubs of a coarse level) are
// cut into DEG_CHUNK-entry chunks summed by many blocks (exact partial sums, added
// atomically), so one row does not hold the whole launch on one warp.
constexpr int64_t DEG_HUGE = 16384;
constexpr int64_t DEG_CHUNK = 16384;

// one lane per row for rows of at most DEG_LONG entries; longer rows are listed
// (any order) for k_degree_long, or for the chunked sums when integral and huge
// (their degree starts at zero)
__global__ void k_degree(const int64_t *__restrict__ rowptr, const double *__restrict__ w,
                         int64_t nv, double *__restrict__ vdeg, int32_t *__restrict__ long_rows,
                         int64_t long_cap, unsigned long long *__restrict__ long_count,
                         int32_t *__restrict__ huge_rows, int64_t huge_cap,
                         unsigned long long *__restrict__ huge_count) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e0 = rowptr[v], e1 = rowptr[v + 1];
        if (e1 - e0 <= DEG_LONG) {
            vdeg[v] = row_fold(w, e0, e1);
        } else if (huge_rows && e1 - e0 > DEG_HUGE) {
            vdeg[v] = 0.0;
            const unsigned long long s = atomicAdd(huge_count, 1ULL);
            if ((int64_t)s < huge_cap) huge_rows[s] = (int32_t)v;
        } else {
            const unsigned long long s = atomicAdd(long_count, 1ULL);
            if ((int64_t)s < long_cap) long_rows[s] = (int32_t)v;
        }
    }
}

// exclusive prefix of the listed huge rows' chunk counts (one thread; the list holds
// at most ne / DEG_HUGE rows); cb[n] = all chunks
__global__ void k_degree_huge_plan(const int64_t *__restrict__ rowptr,
                                   const int32_t *__restrict__ huge_rows, int64_t huge_cap,
                                   const unsigned long long *__restrict__ huge_count,
                                   int64_t *__restrict__ cb) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int64_t n = min((int64_t)*huge_count, huge_cap);
    int64_t run = 0;
    for (int64_t q = 0; q < n; q++) {
        cb[q] = run;
        const int32_t v = huge_rows[q];
        run += (rowptr[v + 1] - rowptr[v] + DEG_CHUNK - 1) / DEG_CHUNK;
    }
    cb[n] = run;
}

// one block per chunk of a huge row: eight loads per thread issued before the adds,
// a warp tree, and one atomic per warp (every partial sum an exact integer)
__global__ void k_degree_huge(const int64_t *__restrict__ rowptr, const double *__restrict__ w,
                              double *__restrict__ vdeg, const int32_t *__restrict__ huge_rows,
                              int64_t huge_cap, const unsigned long long *__restrict__ huge_count,
                              const int64_t *__restrict__ cb) {
    const int64_t n = min((int64_t)*huge_count, huge_cap);
    const int64_t nch = cb[n];
    for (int64_t c = blockIdx.x; c < nch; c += gridDim.x) {
        int64_t lo = 0, hi = n; // the largest q with cb[q] <= c
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (cb[mid] <= c) lo = mid;
            else hi = mid;
        }
        const int32_t v = huge_rows[lo];
        const int64_t E1 = rowptr[v + 1];
        const int64_t a0 = rowptr[v] + (c - cb[lo]) * DEG_CHUNK;
        const int64_t a1 = min(a0 + DEG_CHUNK, E1);
        double sum = 0.0;
        for (int64_t k0 = a0 + threadIdx.x; k0 < a1; k0 += 8 * (int64_t)blockDim.x) {
            double x[8];
#pragma unroll
            for (int t = 0; t < 8; t++) {
                const int64_t k = k0 + (int64_t)t * blockDim.x;
                x[t] = k < a1 ? w[k] : 0.0;
            }
#pragma unroll
            for (int t = 0; t < 8; t++) sum = __dadd_rn(sum, x[t]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum = __dadd_rn(sum, __shfl_xor_sync(0xffffffffu, sum, o));
        if ((threadIdx.x & 31) == 0 && sum != 0.0) atomicAdd(&vdeg[v], sum);
    }
}

// one warp per listed row. Integral weights: every partial sum is exact, so lanes
// add strided entries and a shuffle tree combines them. Otherwise the row's left
// fold in CSR order (vg_warp_ordered_fold: the warp fetches the weights ahead of
// lane 0's chain of additions).
constexpr int DEG_LONG_WARPS = 4; // warps per k_degree_long block (one chain per scheduler)
__global__ void __launch_bounds__(DEG_LONG_WARPS * 32)
    k_degree_long(const int64_t *__restrict__ rowptr, const double *__restrict__ w,
                  double *__restrict__ vdeg, const int32_t *__restrict__ long_rows,
                  int64_t long_cap, const unsigned long long *__restrict__ long_count,
                  int integral) {
    __shared__ double stage[DEG_LONG_WARPS][2 * VG_FOLD_STEP];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t n = min((int64_t)*long_count, long_cap);
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t q = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; q < n; q += nw) {
        const int32_t v = long_rows[q];
        const int64_t E0 = rowptr[v], E1 = rowptr[v + 1];
        double sum = 0.0;
        if (integral) {
            // eight independent partial sums per lane (exact in any order), so eight
            // loads are in flight instead of one chain
            double ps[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            int64_t k = E0 + lane;
            for (; k + 7 * 32 < E1; k += 8 * 32) {
#pragma unroll
                for (int t = 0; t < 8; t++) ps[t] = __dadd_rn(ps[t], w[k + t * 32]);
            }
            for (; k < E1; k += 32) ps[0] = __dadd_rn(ps[0], w[k]);
#pragma unroll
            for (int t = 1; t < 8; t++) ps[0] = __dadd_rn(ps[0], ps[t]);
            sum = ps[0];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sum = __dadd_rn(sum, __shfl_xor_sync(full, sum, o));
        } else {
            // real weights: one left fold in CSR order (lane 0's result)
            const double *__restrict__ rw = w + E0;
            sum = vg_warp_ordered_fold(E1 - E0, [rw](int64_t j) { return rw[j]; },
                                       stage[threadIdx.x >> 5], 0.0, false);
        }
        if (lane == 0) vdeg[v] = sum;
    }
}

// distInitLouvain (louvain.cpp:2138-2159) plus the early-termination buffers
__global__ void k_init(int64_t nv, const double *__restrict__ vdeg, double *__restrict__ cdeg,
                       int32_t *__restrict__ csize, CommInfo *__restrict__ cupd,
                       int32_t *__restrict__ past,
                       int32_t *__restrict__ curr, int32_t *__restrict__ target,
                       uint8_t *__restrict__ active, double *__restrict__ pcurr,
                       double *__restrict__ pprev, int32_t *__restrict__ noprune) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (noprune && !(vdeg[i] >= 0.0)) *noprune = 1; // negative or NaN degree
        cdeg[i] = vdeg[i];
        csize[i] = 1;
        CommInfo z;
        z.deg = 0.0;
        z.size = 0;
        z.pad = 0;
        cupd[i] = z;
        past[i] = (int32_t)i;
        curr[i] = (int32_t)i;
        target[i] = (int32_t)i;
        if (active) active[i] = 1;
        if (pcurr) pcurr[i] = 0.0; // value-initialised (louvain.cpp:244-249)
        if (pprev) pprev[i] = 1.0;
    }
}

__device__ double block_sum(double v, double *ws) {
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

// ---------------------------------------------------------------------------------
// Fixed-order segmented sums. A segment (the vertex range of one graph) is cut
// into chunks of SEG_CHUNK entries counted from the segment's start; thread t of
// a chunk's block adds entries t, t + SEG_THREADS, ... in order and the warps
// combine through a fixed shuffle tree; a segment's chunk partials are then
// combined the same way by one block of SEG_FINAL threads. The order depends only
// on the segment's own length, so a graph's 2m and modularity sums are the same
// bits whether it runs alone or packed with other graphs.

constexpr int SEG_CHUNK = 2048;
constexpr int SEG_THREADS = 256;
constexpr int SEG_FINAL = 1024;

// largest j with cb[j] <= q (cb[0] = 0 <= q < cb[J])
__device__ __forceinline__ int64_t seg_of_chunk(const int64_t *__restrict__ cb, int64_t J, int64_t q) {
    int64_t lo = 0, hi = J;
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (cb[mid] <= q) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(SEG_THREADS) k_seg_sum_chunks(
    const double *__restrict__ x, const int64_t *__restrict__ voff, const int64_t *__restrict__ cb,
    int64_t J, int64_t C, double *__restrict__ part) {
    __shared__ double ws[32];
    for (int64_t q = blockIdx.x; q < C; q += gridDim.x) {
        const int64_t j = seg_of_chunk(cb, J, q);
        const int64_t lo = voff[j] + (q - cb[j]) * SEG_CHUNK;
        const int64_t hi = min(lo + SEG_CHUNK, voff[j + 1]);
        double s = 0.0;
        for (int64_t i = lo + threadIdx.x; i < hi; i += SEG_THREADS) s = __dadd_rn(s, x[i]);
        s = block_sum(s, ws);
        if (threadIdx.x == 0) part[q] = s;
    }
}

__global__ void __launch_bounds__(SEG_FINAL) k_seg_sum_final(const double *__restrict__ part,
                                                             const int64_t *__restrict__ cb,
                                                             int64_t J, double *__restrict__ out) {
    __shared__ double ws[32];
    for (int64_t j = blockIdx.x; j < J; j += gridDim.x) {
        double s = 0.0;
        for (int64_t q = cb[j] + threadIdx.x; q < cb[j + 1]; q += SEG_FINAL) s = __dadd_rn(s, part[q]);
        s = block_sum(s, ws);
        if (threadIdx.x == 0) out[j] = s;
    }
}

// distUpdateLocalCinfo (louvain.cpp:2534-2547) fused with the two sums of
// distComputeModularity (louvain.cpp:2496-2504) and the frozen-vertex count,
// per chunk of each segment; segments whose phase has ended are skipped
__global__ void __launch_bounds__(SEG_THREADS) k_apply_seg(
    const int64_t *__restrict__ voff, const int64_t *__restrict__ cb, int64_t J, int64_t C,
    double *__restrict__ cdeg, int32_t *__restrict__ csize, CommInfo *__restrict__ cupd,
    const double *__restrict__ cw, const uint8_t *__restrict__ active,
    const uint8_t *__restrict__ jdone, int do_sums, double *__restrict__ part,
    int32_t *__restrict__ noprune) {
    __shared__ double ws[32];
    for (int64_t q = blockIdx.x; q < C; q += gridDim.x) {
        const int64_t j = seg_of_chunk(cb, J, q);
        if (jdone && jdone[j]) continue;
        const int64_t lo = voff[j] + (q - cb[j]) * SEG_CHUNK;
        const int64_t hi = min(lo + SEG_CHUNK, voff[j + 1]);
        double le = 0.0, la2 = 0.0, frozen = 0.0;
        // a thread's entries i, i + SEG_THREADS, ... in that order (the sums' fixed
        // order), four of them loaded together
        constexpr int U4 = 4;
        for (int64_t i0 = lo + threadIdx.x; i0 < hi; i0 += U4 * SEG_THREADS) {
            CommInfo u[U4];
            double cd0[U4], cwv[U4];
#pragma unroll
            for (int k = 0; k < U4; k++) {
                const int64_t i = i0 + (int64_t)k * SEG_THREADS;
                u[k].deg = 0.0;
                u[k].size = 0;
                cd0[k] = 0.0;
                cwv[k] = 0.0;
                if (i < hi) {
                    u[k] = cupd[i];
                    if (do_sums) {
                        cd0[k] = cdeg[i];
                        cwv[k] = cw[i];
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < U4; k++) {
                const int64_t i = i0 + (int64_t)k * SEG_THREADS;
                if (i >= hi) break;
                double cd = cd0[k];
                if (u[k].size != 0 || u[k].deg != 0.0) {
                    cd = __dadd_rn(do_sums ? cd : cdeg[i], u[k].deg);
                    cdeg[i] = cd;
                    const int32_t ns = csize[i] + u[k].size;
                    csize[i] = ns;
                    // a community with members must keep a degree >= 0 for the pruning
                    // bound (rounding can leave an emptied one at -0.0 or a tiny negative)
                    if (noprune && ns > 0 && !(cd >= 0.0)) *noprune = 1;
                    CommInfo z;
                    z.deg = 0.0;
                    z.size = 0;
                    z.pad = 0;
                    cupd[i] = z;
                }
                if (do_sums) {
                    le = __dadd_rn(le, cwv[k]);
                    la2 = __dadd_rn(la2, __dmul_rn(cd, cd));
                    if (active && !active[i]) frozen += 1.0;
                }
            }
        }
        if (!do_sums) continue;
        le = block_sum(le, ws);
        la2 = block_sum(la2, ws);
        frozen = block_sum(frozen, ws);
        if (threadIdx.x == 0) {
            part[3 * q + 0] = le;
            part[3 * q + 1] = la2;
            part[3 * q + 2] = frozen;
        }
    }
}

// per-graph phase state of a batch: the loop test of distLouvainMethod
// (louvain.cpp:553-563) evaluated for every graph on the device
struct BatchDecide {
    double *prev_mod;      // prevMod, starts at `lower`
    const double *lower;
    const double *thresh;
    int32_t *iters;
    uint8_t *done;
    int8_t *resbuf;        // which of the three community buffers held pastComm at the break
    int32_t *live_count;   // graphs still iterating after this iteration
    int32_t iter;
    int32_t past_idx;
    const int32_t *iter_dev; // when set, the iteration number is read here (graph replays)
};

// iteration counter of a captured batch iteration
__global__ void k_iter_inc(int32_t *__restrict__ it) { *it += 1; }

// final reduction and the ABS_MOD_PER_ITER modularity (louvain.cpp:2518-2524),
// one block per segment. One graph: out = {Q, frozen, le, la2}; a batch: the
// loop test per graph
__global__ void __launch_bounds__(SEG_FINAL) k_mod_seg(const double *__restrict__ part,
                                                       const int64_t *__restrict__ cb, int64_t J,
                                                       double constant,
                                                       const double *__restrict__ jconst,
                                                       double *__restrict__ out, BatchDecide bd) {
    __shared__ double ws[32];
    for (int64_t j = blockIdx.x; j < J; j += gridDim.x) {
        if (bd.done && bd.done[j]) continue;
        double le = 0.0, la2 = 0.0, fr = 0.0;
        for (int64_t q = cb[j] + threadIdx.x; q < cb[j + 1]; q += SEG_FINAL) {
            le = __dadd_rn(le, part[3 * q]);
            la2 = __dadd_rn(la2, part[3 * q + 1]);
            fr += part[3 * q + 2];
        }
        le = block_sum(le, ws);
        la2 = block_sum(la2, ws);
        fr = block_sum(fr, ws);
        if (threadIdx.x == 0) {
            const double c = jconst ? jconst[j] : constant;
            const double m = fabs(__dsub_rn(__dmul_rn(le, c), __dmul_rn(__dmul_rn(la2, c), c)));
            if (!bd.done) {
                out[0] = m;
                out[1] = fr;
                out[2] = le;
                out[3] = la2;
            } else {
                bd.iters[j] = bd.iter_dev ? *bd.iter_dev : bd.iter;
                if (m != m || __dsub_rn(m, bd.prev_mod[j]) < bd.thresh[j]) { // NaN: 2m = 0
                    bd.done[j] = 1;
                    bd.resbuf[j] = (int8_t)bd.past_idx;
                } else {
                    bd.prev_mod[j] = m < bd.lower[j] ? bd.lower[j] : m;
                    atomicAdd(bd.live_count, 1);
                }
            }
        }
    }
}

struct SegTable {
    DevBuf<int64_t> voff, cb; // J + 1 each
    int64_t J = 0, C = 0;
};

void seg_table_build(vg_ctx *ctx, const int64_t *h_voff, int64_t J, SegTable &t) {
    std::vector<int64_t> cb(J + 1, 0);
    for (int64_t j = 0; j < J; j++)
        cb[j + 1] = cb[j] + (h_voff[j + 1] - h_voff[j] + SEG_CHUNK - 1) / SEG_CHUNK;
    t.J = J;
    t.C = cb[J];
    t.voff.alloc(ctx, J + 1);
    t.cb.alloc(ctx, J + 1);
    VG_CUDA(cudaMemcpyAsync(t.voff.p, h_voff, sizeof(int64_t) * (J + 1), cudaMemcpyHostToDevice,
                            ctx->stream));
    VG_CUDA(cudaMemcpyAsync(t.cb.p, cb.data(), sizeof(int64_t) * (J + 1), cudaMemcpyHostToDevice,
                            ctx->stream));
    vg_sync(ctx); // the host vectors go out of scope
}

int seg_grid(vg_ctx *ctx, int64_t chunks) {
    return (int)std::max<int64_t>(1, std::min<int64_t>(chunks, 8LL * ctx->sm_count));
}

// per-segment sums of x into out[J] (device)
void seg_sums(vg_ctx *ctx, const double *x, const SegTable &t, double *out) {
    DevBuf<double> part(ctx, std::max<int64_t>(t.C, 1));
    if (t.C) {
        LaunchTimer lt(ctx);
        k_seg_sum_chunks<<<seg_grid(ctx, t.C), SEG_THREADS, 0, ctx->stream>>>(x, t.voff.p, t.cb.p,
                                                                               t.J, t.C, part.p);
    }
    VG_CHECK_LAUNCH();
    {
        LaunchTimer lt(ctx);
        k_seg_sum_final<<<(int)std::min<int64_t>(std::max<int64_t>(t.J, 1), 65535), SEG_FINAL, 0,
                          ctx->stream>>>(part.p, t.cb.p, t.J, out);
    }
    VG_CHECK_LAUNCH();
}

// 2m of one graph in the segmented order
double twice_m_one(vg_ctx *ctx, const double *vdeg, int64_t nv) {
    const int64_t voff[2] = {0, nv};
    SegTable t;
    seg_table_build(ctx, voff, 1, t);
    DevBuf<double> out(ctx, 1);
    seg_sums(ctx, vdeg, t, out.p);
    double *h = (double *)vg_pinned(ctx, sizeof(double));
    VG_CUDA(cudaMemcpyAsync(h, out.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    vg_sync(ctx);
    return *h;
}

// early termination -t 1/3 (louvain.cpp:172-184): C++'s chained
// `target == curr == past` compares the bool (target == curr) with past
__global__ void k_swap_et13(int64_t nv, int numIters, int32_t *__restrict__ past,
                            int32_t *__restrict__ curr, int32_t *__restrict__ target,
                            uint8_t *__restrict__ active, const int32_t *__restrict__ ref) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = past[i], c = curr[i], t = target[i];
        if (numIters > 2 && ((int32_t)(t == c) == vg_rid(ref, p))) {
            active[i] = 0;
        } else {
            past[i] = c;
            curr[i] = t;
            target[i] = p;
        }
    }
}

// early termination -t 2/4 (louvain.cpp:381-400)
__global__ void k_swap_et24(int64_t nv, int numIters, double one_minus_delta,
                            int32_t *__restrict__ past, int32_t *__restrict__ curr,
                            int32_t *__restrict__ target, uint8_t *__restrict__ active,
                            double *__restrict__ pcurr, const double *__restrict__ pprev) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (!active[i]) continue;
        const int32_t p = past[i], c = curr[i];
        bool act = true;
        if (numIters > 2 && c == p) {
            const double pc = __dmul_rn(pprev[i], one_minus_delta);
            pcurr[i] = pc;
            if (pc <= 0.02) { // P_CUTOFF (louvain.hpp:74)
                act = false;
                active[i] = 0;
            }
        }
        if (act) {
            past[i] = c;
            curr[i] = target[i];
            target[i] = p;
        }
    }
}

__global__ void k_widen(const int32_t *__restrict__ in, int64_t n, int64_t *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[i];
}

__global__ void k_narrow(const int64_t *__restrict__ in, int64_t n, int64_t lim,
                         int32_t *__restrict__ out, int *__restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = in[i];
        if (x < -1 || x >= lim) *bad = 1;
        out[i] = (int32_t)x;
    }
}

// bucket key of a vertex: (color bucket, degree class)
__device__ __forceinline__ int32_t bucket_key(const int64_t *__restrict__ rowptr, int64_t i,
                                              const int32_t *__restrict__ colors, int64_t numColor,
                                              int64_t *d_out, const ClassBounds &bnd) {
    const int64_t d = rowptr[i + 1] - rowptr[i];
    int64_t cb = 0;
    if (colors) cb = colors[i] < 0 ? numColor - 1 : colors[i];
    *d_out = d;
    return (int32_t)(cb * NCLS + degree_class(d, bnd));
}

// Each block histograms a contiguous chunk of vertices in shared memory and
// adds its counts to the global ones (one atomic per bucket per block).
__global__ void k_bucket_count(const int64_t *__restrict__ rowptr, int64_t nv,
                               const int32_t *__restrict__ colors, int64_t numColor, int nb,
                               int64_t chunk, int32_t *__restrict__ counts, ClassBounds bnd) {
    extern __shared__ int32_t sc[];
    for (int k = threadIdx.x; k < nb; k += blockDim.x) sc[k] = 0;
    __syncthreads();
    const int64_t b0 = blockIdx.x * chunk, b1 = min(nv, b0 + chunk);
    for (int64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        int64_t d;
        atomicAdd(&sc[bucket_key(rowptr, i, colors, numColor, &d, bnd)], 1);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nb; k += blockDim.x)
        if (sc[k]) atomicAdd(&counts[k], sc[k]);
}

// Each block reserves a range per bucket with one atomic and places its vertices
// there (order inside a bucket follows the blocks' chunks).
// Order-preserving placement for at most 32 buckets (the uncoloured sweep): a
// block ranks each round of 256 vertices of its chunk with match_any inside a warp
// and per-warp counts across warps, so every list keeps position order within a
// chunk and the list kernels walk adjacent rows.
constexpr int PLACE_THREADS = 256;

__global__ void __launch_bounds__(PLACE_THREADS) k_bucket_place_ordered(
    const int64_t *__restrict__ rowptr, int64_t nv, int nb, int64_t chunk,
    int32_t *__restrict__ fill, int32_t *__restrict__ list, ClassBounds bnd) {
    __shared__ int32_t cnt[PLACE_THREADS / 32][32];
    __shared__ int32_t base[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    // block totals first: one global reservation per bucket and block
    if (threadIdx.x < 32) base[threadIdx.x] = 0;
    __syncthreads();
    const int64_t b0 = blockIdx.x * chunk, b1 = min(nv, b0 + chunk);
    int64_t d;
    for (int64_t i = b0 + threadIdx.x; i < b1; i += PLACE_THREADS)
        atomicAdd(&base[bucket_key(rowptr, i, nullptr, 1, &d, bnd)], 1);
    __syncthreads();
    if (threadIdx.x < nb) base[threadIdx.x] = base[threadIdx.x] ? atomicAdd(&fill[threadIdx.x], base[threadIdx.x]) : 0;
    __syncthreads();
    for (int64_t r0 = b0; r0 < b1; r0 += PLACE_THREADS) {
        const int64_t i = r0 + threadIdx.x;
        const bool valid = i < b1;
        const int k = valid ? bucket_key(rowptr, i, nullptr, 1, &d, bnd) : 32 + lane;
        const unsigned peers = __match_any_sync(0xffffffffu, k);
        if (lane < 32) cnt[warp][lane] = 0;
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) cnt[warp][k] = __popc(peers);
        __syncthreads();
        int off = 0;
        if (valid)
            for (int w = 0; w < warp; w++) off += cnt[w][k];
        if (valid) list[base[k] + off + __popc(peers & lt)] = (int32_t)i;
        __syncthreads();
        if (threadIdx.x < nb) {
            int tot = 0;
            for (int w = 0; w < PLACE_THREADS / 32; w++) tot += cnt[w][threadIdx.x];
            base[threadIdx.x] += tot;
        }
        __syncthreads();
    }
}

__global__ void k_bucket_place(const int64_t *__restrict__ rowptr, int64_t nv,
                               const int32_t *__restrict__ colors, int64_t numColor, int nb,
                               int64_t chunk, int32_t *__restrict__ fill,
                               int32_t *__restrict__ list, ClassBounds bnd) {
    extern __shared__ int32_t sc[]; // [0, nb) counts then local cursors, [nb, 2nb) bases
    int32_t *base = sc + nb;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) sc[k] = 0;
    __syncthreads();
    const int64_t b0 = blockIdx.x * chunk, b1 = min(nv, b0 + chunk);
    int64_t d;
    for (int64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x)
        atomicAdd(&sc[bucket_key(rowptr, i, colors, numColor, &d, bnd)], 1);
    __syncthreads();
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        base[k] = sc[k] ? atomicAdd(&fill[k], sc[k]) : 0;
        sc[k] = 0;
    }
    __syncthreads();
    for (int64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const int32_t k = bucket_key(rowptr, i, colors, numColor, &d, bnd);
        list[base[k] + atomicAdd(&sc[k], 1)] = (int32_t)i;
    }
}

} // namespace

// ---------------------------------------------------------------------------------
// host side

// the context's tuning with unset (zero) fields at the built-in defaults
static vg_tuning effective_tuning(const vg_ctx *ctx) {
    vg_tuning t = ctx->tune;
    if (t.ws_max == 0) {
        t.t32 = VG_T32;
        t.ws_max = WS_MAXDEG;
        t.wt_max = WT_MAXDEG;
        t.ct_max = CT_MAXDEG;
    }
    if (t.tile_grid == 0) t.tile_grid = VG_TILE_GRID;
    return t;
}

static bool tuning_valid(const vg_tuning &t) {
    return (t.t32 == 0 || t.t32 == 1) && t.ws_max >= 32 && t.ws_max <= WS_CAP / 2 &&
           t.wt_max >= t.ws_max && t.wt_max <= WT_CAP / 2 && t.ct_max >= t.wt_max &&
           t.ct_max <= CT_CAP / 2 && t.tile_grid >= 1 && t.tile_grid <= 1024;
}

static ClassBounds class_bounds(const vg_ctx *ctx) {
    const vg_tuning t = effective_tuning(ctx);
    return ClassBounds{t.t32, t.ws_max, t.wt_max, t.ct_max};
}

struct Buckets {
    DevBuf<int32_t> list;
    std::vector<int64_t> start; // (numColor * NCLS) + 1 offsets
    int64_t ncolor = 1;
};

static void build_buckets(vg_ctx *ctx, const vg_graph *g, const int32_t *colors, int64_t numColor,
                          Buckets &b) {
    const int64_t nv = g->nv;
    const int64_t nb = numColor * NCLS;
    const ClassBounds bnd = class_bounds(ctx);
    VG_REQUIRE(nb <= 6000, "too many color buckets (%lld colors)", (long long)numColor);
    b.ncolor = numColor;
    DevBuf<int32_t> counts(ctx, nb);
    VG_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(int32_t) * nb, ctx->stream));
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((nv + 1023) / 1024, 4LL * ctx->sm_count));
    const int64_t chunk = (nv + blocks - 1) / blocks;
    if (nv) {
        LaunchTimer lt(ctx);
        k_bucket_count<<<blocks, 256, sizeof(int32_t) * nb, ctx->stream>>>(
            g->rowptr, nv, colors, numColor, (int)nb, chunk, counts.p, bnd);
    }
    VG_CHECK_LAUNCH();
    std::vector<int32_t> hc(nb);
    VG_CUDA(cudaMemcpyAsync(hc.data(), counts.p, sizeof(int32_t) * nb, cudaMemcpyDeviceToHost,
                            ctx->stream));
    vg_sync(ctx);
    b.start.assign(nb + 1, 0);
    std::vector<int32_t> fill(nb);
    for (int64_t k = 0; k < nb; k++) {
        fill[k] = (int32_t)b.start[k];
        b.start[k + 1] = b.start[k] + hc[k];
    }
    VG_CUDA(cudaMemcpyAsync(counts.p, fill.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice,
                            ctx->stream));
    b.list.alloc(ctx, nv);
    if (nv && !colors && nb <= 32) {
        LaunchTimer lt(ctx);
        k_bucket_place_ordered<<<blocks, PLACE_THREADS, 0, ctx->stream>>>(
            g->rowptr, nv, (int)nb, chunk, counts.p, b.list.p, bnd);
    } else if (nv) {
        LaunchTimer lt(ctx);
        k_bucket_place<<<blocks, 256, 2 * sizeof(int32_t) * nb, ctx->stream>>>(
            g->rowptr, nv, colors, numColor, (int)nb, chunk, counts.p, b.list.p, bnd);
    }
    VG_CHECK_LAUNCH();
    vg_sync(ctx); // keep `fill` alive until the copy is done
}

static size_t cta_smem_bytes(int cap = CT_CAP) { return (size_t)cap * (sizeof(double) + sizeof(int32_t)); }

static void configure_kernels_once() {
    static bool done = false;
    if (done) return;
    VG_CUDA(cudaFuncSetAttribute(k_sweep_warp<WS_CAP, WS_WARPS>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)warp_smem_bytes<WS_CAP, WS_WARPS>()));
    VG_CUDA(cudaFuncSetAttribute(k_sweep_warp<WT_CAP, WT_WARPS>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)warp_smem_bytes<WT_CAP, WT_WARPS>()));
    VG_CUDA(cudaFuncSetAttribute(k_sweep_cta<CT_CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cta_smem_bytes()));
    VG_CUDA(cudaFuncSetAttribute(k_sweep_cta<CT_CAP_S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cta_smem_bytes(CT_CAP_S)));
    done = true;
}

// vdeg[v] = the sum of v's row weights (distCalcVertexDegree, louvain.cpp:2118-2136):
// short rows one per lane, rows longer than DEG_LONG one per warp
static void vertex_degrees(vg_ctx *ctx, const vg_graph *g, double *vdeg, int integral) {
    const int64_t nv = g->nv;
    if (nv == 0) return;
    const int64_t cap = std::min<int64_t>(nv, g->ne / (DEG_LONG + 1) + 1);
    DevBuf<int32_t> list(ctx, cap);
    DevBuf<unsigned long long> cnt(ctx, 2); // long rows, huge rows
    VG_CUDA(cudaMemsetAsync(cnt.p, 0, 2 * sizeof(unsigned long long), ctx->stream));
    const bool chunked = integral && g->ne > DEG_HUGE;
    const int64_t hcap = chunked ? std::min<int64_t>(nv, g->ne / (DEG_HUGE + 1) + 1) : 0;
    DevBuf<int32_t> hlist(ctx, hcap);
    DevBuf<int64_t> hcb(ctx, chunked ? hcap + 1 : 0);
    {
        LaunchTimer lt(ctx);
        k_degree<<<vg_grid(ctx, nv, 256), 256, 0, ctx->stream>>>(g->rowptr, g->weight, nv, vdeg,
                                                                 list.p, cap, cnt.p, hlist.p, hcap,
                                                                 cnt.p + 1);
    }
    VG_CHECK_LAUNCH();
    if (chunked) {
        { LaunchTimer lt(ctx);
          k_degree_huge_plan<<<1, 32, 0, ctx->stream>>>(g->rowptr, hlist.p, hcap, cnt.p + 1, hcb.p); }
        VG_CHECK_LAUNCH();
        { LaunchTimer lt(ctx);
          k_degree_huge<<<(int)std::min<int64_t>(g->ne / DEG_CHUNK + hcap, 16LL * ctx->sm_count), 256,
                          0, ctx->stream>>>(g->rowptr, g->weight, vdeg, hlist.p, hcap, cnt.p + 1,
                                            hcb.p); }
        VG_CHECK_LAUNCH();
    }
    if (g->ne > DEG_LONG) {
        LaunchTimer lt(ctx);
        k_degree_long<<<vg_grid(ctx, cap * 32, DEG_LONG_WARPS * 32, 8), DEG_LONG_WARPS * 32, 0,
                        ctx->stream>>>(
            g->rowptr, g->weight, vdeg, list.p, cap, cnt.p, integral);
    }
    VG_CHECK_LAUNCH();
}

// The hubs (class 5) of every color, planned once per phase: plan index q runs over
// the colors' class-5 lists in color order; color k owns [first[k], first[k+1]).
struct HubPlan {
    int64_t n = 0;
    std::vector<int64_t> first;    // numColor + 1
    std::vector<int64_t> hcb, hsb; // host copies of the chunk and slice prefixes (n + 1)
    DevBuf<int32_t> vtx;
    DevBuf<int64_t> toff, cb, sb;
    DevBuf<int32_t> keys;
    DevBuf<double> vals, self, c0;
    DevBuf<HubBest> best;
};

static void plan_hubs(vg_ctx *ctx, const vg_graph *g, const Buckets &bk, int64_t numColor,
                      HubPlan &hp) {
    hp.first.assign(numColor + 1, 0);
    for (int64_t k = 0; k < numColor; k++)
        hp.first[k + 1] = hp.first[k] + (bk.start[k * NCLS + 6] - bk.start[k * NCLS + 5]);
    hp.n = hp.first[numColor];
    if (hp.n == 0) return;
    const int64_t n = hp.n;
    hp.vtx.alloc(ctx, n);
    hp.toff.alloc(ctx, n + 1);
    hp.cb.alloc(ctx, n + 1);
    hp.sb.alloc(ctx, n + 1);
    VG_CUDA(cudaMemsetAsync(hp.toff.p + n, 0, sizeof(int64_t), ctx->stream));
    VG_CUDA(cudaMemsetAsync(hp.cb.p + n, 0, sizeof(int64_t), ctx->stream));
    VG_CUDA(cudaMemsetAsync(hp.sb.p + n, 0, sizeof(int64_t), ctx->stream));
    for (int64_t k = 0; k < numColor; k++) {
        const int64_t m = hp.first[k + 1] - hp.first[k];
        if (m == 0) continue;
        const int64_t q = hp.first[k];
        LaunchTimer lt(ctx);
        k_hub_plan<<<vg_grid(ctx, m, 256), 256, 0, ctx->stream>>>(
            g->rowptr, bk.list.p + bk.start[k * NCLS + 5], m, hp.vtx.p + q, hp.toff.p + q,
            hp.cb.p + q, hp.sb.p + q);
        VG_CHECK_LAUNCH();
    }
    vg_scan_i64_async(ctx, hp.toff.p, n + 1, nullptr);
    vg_scan_i64_async(ctx, hp.cb.p, n + 1, nullptr);
    vg_scan_i64_async(ctx, hp.sb.p, n + 1, nullptr);
    hp.hcb.resize(n + 1);
    hp.hsb.resize(n + 1);
    int64_t slots = 0;
    VG_CUDA(cudaMemcpyAsync(hp.hcb.data(), hp.cb.p, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost,
                            ctx->stream));
    VG_CUDA(cudaMemcpyAsync(hp.hsb.data(), hp.sb.p, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost,
                            ctx->stream));
    VG_CUDA(cudaMemcpyAsync(&slots, hp.toff.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost,
                            ctx->stream));
    vg_sync(ctx);
    hp.keys.alloc(ctx, slots);
    hp.vals.alloc(ctx, slots);
    hp.self.alloc(ctx, n);
    hp.c0.alloc(ctx, n);
    hp.best.alloc(ctx, hp.hsb[n]);
    VG_CUDA(cudaMemsetAsync(hp.keys.p, 0xff, sizeof(int32_t) * slots, ctx->stream)); // EMPTY
    VG_CUDA(cudaMemsetAsync(hp.vals.p, 0, sizeof(double) * slots, ctx->stream));
    VG_CUDA(cudaMemsetAsync(hp.self.p, 0, sizeof(double) * n, ctx->stream));
}

// one sweep over the hubs of color k
static void sweep_hubs(vg_ctx *ctx, const SweepArgs &a, HubPlan &hp, int64_t k,
                       cudaStream_t st) {
    const int64_t q0 = hp.first[k], q1 = hp.first[k + 1];
    if (q1 == q0) return;
    const int64_t nch = hp.hcb[q1] - hp.hcb[q0], nsl = hp.hsb[q1] - hp.hsb[q0];
    const int64_t cap_blocks = 8LL * ctx->sm_count;
    {
        LaunchTimer lt(ctx);
        k_hub_accum<<<(int)std::min(nch, cap_blocks), HUB_THREADS, 0, st>>>(
            a, hp.vtx.p, hp.toff.p, hp.cb.p, q0, q1, hp.keys.p, hp.vals.p, hp.self.p);
    }
    VG_CHECK_LAUNCH();
    {
        LaunchTimer lt(ctx);
        k_hub_c0<<<vg_grid(ctx, q1 - q0, 256), 256, 0, st>>>(
            a, hp.vtx.p, hp.toff.p, q0, q1, hp.keys.p, hp.vals.p, hp.c0.p);
    }
    VG_CHECK_LAUNCH();
    {
        LaunchTimer lt(ctx);
        k_hub_eval<<<(int)std::min(nsl, cap_blocks), HUB_THREADS, 0, st>>>(
            a, hp.vtx.p, hp.toff.p, hp.sb.p, q0, q1, hp.keys.p, hp.vals.p, hp.self.p, hp.c0.p,
            hp.best.p);
    }
    VG_CHECK_LAUNCH();
    {
        LaunchTimer lt(ctx);
        k_hub_commit<<<vg_grid(ctx, (q1 - q0) * 32, 256), 256, 0, st>>>(
            a, hp.vtx.p, hp.sb.p, q0, q1, hp.self.p, hp.c0.p, hp.best.p);
    }
    VG_CHECK_LAUNCH();
}

// launch the sweep kernels over one color bucket; with `natural` the low-degree
// class runs over all vertices in id order instead of its list. The classes touch
// disjoint vertices (reading the community arrays, which no sweep kernel writes, and
// adding to the deltas with atomics), so when the first class and another one both
// have work, the other classes run on the context's side stream alongside the first
// (their blocks fill the SMs the first one's tail leaves idle); with profiling on,
// every launch stays on the main stream so that each one is timed alone.
static void sweep_color(vg_ctx *ctx, const SweepArgs &a, const Buckets &b, int64_t color,
                        HubPlan &hp, bool natural, int64_t nv) {
    const int32_t *list = b.list.p;
    auto count = [&](int cls) { return b.start[color * NCLS + cls + 1] - b.start[color * NCLS + cls]; };
    const bool first_busy = natural ? nv > 0 : count(0) > 0;
    bool others = false;
    for (int cls = 1; cls < NCLS; cls++) others = others || count(cls) > 0;
    const bool fork = first_busy && others && !ctx->profile;
    cudaStream_t st = fork ? vg_side_fork(ctx) : ctx->stream;
    for (int cls = 1; cls < NCLS; cls++) {
        const int64_t s = b.start[color * NCLS + cls];
        const int64_t n = count(cls);
        if (n == 0) continue;
        if (cls == NCLS - 1) { // the hubs
            sweep_hubs(ctx, a, hp, color, st);
            continue;
        }
        LaunchTimer lt(ctx);
        switch (cls) {
        case 1:
            k_sweep_thread<true, 32, 128><<<vg_grid(ctx, n, 128, VG_T32_GRID), 128, 0, st>>>(a, list + s, n);
            break;
        case 2:
            k_sweep_warp<WS_CAP, WS_WARPS><<<vg_grid(ctx, n * 32, WS_WARPS * 32, VG_WS_GRID), WS_WARPS * 32,
                                             warp_smem_bytes<WS_CAP, WS_WARPS>(), st>>>(
                a, list + s, n);
            break;
        case 3:
            k_sweep_warp<WT_CAP, WT_WARPS><<<vg_grid(ctx, n * 32, WT_WARPS * 32, VG_WS_GRID), WT_WARPS * 32,
                                             warp_smem_bytes<WT_CAP, WT_WARPS>(), st>>>(
                a, list + s, n);
            break;
        case 4:
            k_sweep_cta<CT_CAP_S><<<vg_grid(ctx, n * CT_THREADS, CT_THREADS, VG_CT_GRID_S), CT_THREADS,
                                    cta_smem_bytes(CT_CAP_S), st>>>(a, list + s, n);
            VG_CHECK_LAUNCH();
            if (effective_tuning(ctx).ct_max > CT_CAP_S / 2) {
                LaunchTimer lt2(ctx);
                k_sweep_cta<CT_CAP><<<vg_grid(ctx, n * CT_THREADS, CT_THREADS, VG_CT_GRID), CT_THREADS,
                                      cta_smem_bytes(), st>>>(a, list + s, n);
            }
            break;
        default:
            break;
        }
        VG_CHECK_LAUNCH();
    }
    if (first_busy) {
        LaunchTimer lt(ctx);
        if (natural) {
            const int64_t tiles_blocks = (nv + TILE_WARPS * 32 - 1) / (TILE_WARPS * 32);
            const int tgrid = (int)std::max<int64_t>(
                1, std::min<int64_t>(tiles_blocks,
                                     (int64_t)effective_tuning(ctx).tile_grid * ctx->sm_count));
            if (a.ident)
                k_sweep_tile<TMAX, true><<<tgrid, TILE_WARPS * 32, 0, ctx->stream>>>(a, nv);
            else
                k_sweep_tile<TMAX, false><<<tgrid, TILE_WARPS * 32, 0, ctx->stream>>>(a, nv);
        } else {
            const int64_t n = count(0);
            k_sweep_thread<true, TMAX, TB><<<vg_grid(ctx, n, TB, 8), TB, 0, ctx->stream>>>(
                a, list + b.start[color * NCLS], n);
        }
        VG_CHECK_LAUNCH();
    }
    if (fork) vg_side_join(ctx);
}

struct PhaseTiming {
    double sweep_ms = 0.0;
    int64_t edges = 0;
};

// the phase proper; returns the communities in g->comm
// max_iters > 0 stops after that many iterations (the autotuner's timing runs)
static void run_phase(vg_ctx *ctx, vg_graph *g, const vg_phase_params *p, double *mod_out,
                      int32_t *iters_out, PhaseTiming *timing, int max_iters = 0) {
    configure_kernels_once();
    const int64_t nv = g->nv;
    int ordering = p->ordering;
    int et = p->et_type;
    VG_REQUIRE(et >= 0 && et <= 4, "early-termination type must be 0..4 (got %d)", et);
    VG_REQUIRE(ordering >= 0 && ordering <= 2, "ordering must be 0, 1 or 2 (got %d)", ordering);
    int64_t numColor = 1;
    if (ordering != 0) {
        VG_REQUIRE(g->colors != nullptr && g->num_colors >= 0,
                   "ordering %d needs a coloring (vg_color or vg_set_colors)", ordering);
        numColor = g->num_colors + 1;
        if (numColor == 1) { // louvain.cpp:600-605: plain fallback without early termination
            ordering = 0;
            et = 0;
        }
    }
    const bool use_et = et != 0;
    DevBuf<double> vdeg(ctx, nv), cw(ctx, nv);
    DevBuf<double> cdeg(ctx, nv);
    DevBuf<int32_t> csize(ctx, nv);
    DevBuf<CommInfo> cupd(ctx, nv);
    DevBuf<int32_t> A(ctx, nv), B(ctx, nv), C(ctx, nv);
    DevBuf<double> frozen, pA, pB;
    DevBuf<uint8_t> active;
    if (use_et) {
        frozen.alloc(ctx, nv);
        active.alloc(ctx, nv);
        if (et == 2 || et == 4) {
            pA.alloc(ctx, nv);
            pB.alloc(ctx, nv);
        }
    }
    const int grid = vg_grid(ctx, nv, 256);
    DevBuf<int32_t> noprune(ctx, 1); // see can_prune
    VG_CUDA(cudaMemsetAsync(noprune.p, 0, sizeof(int32_t), ctx->stream));
    if (nv) {
        vertex_degrees(ctx, g, vdeg.p, (int)vg_weights_integral(ctx, g));
    }
    const double twice_m = nv ? twice_m_one(ctx, vdeg.p, nv) : 0.0;
    const double constant = 1.0 / twice_m; // distCalcConstantForSecondTerm (louvain.cpp:2217)
    if (nv) {
        LaunchTimer lt(ctx);
        k_init<<<grid, 256, 0, ctx->stream>>>(nv, vdeg.p, cdeg.p, csize.p, cupd.p, A.p, B.p,
                                              C.p, active.p, pA.p, pB.p, noprune.p);
    }
    VG_CHECK_LAUNCH();
    Buckets bk;
    build_buckets(ctx, g, ordering ? g->colors : nullptr, numColor, bk);
    HubPlan hp;
    plan_hubs(ctx, g, bk, numColor, hp);
    SegTable seg;
    {
        const int64_t voff[2] = {0, nv};
        seg_table_build(ctx, voff, 1, seg);
    }
    DevBuf<double> part(ctx, 3 * std::max<int64_t>(seg.C, 1));
    const int agrid = seg_grid(ctx, seg.C);
    DevBuf<double> modv(ctx, 4);
    double *hmod = (double *)vg_pinned(ctx, 4 * sizeof(double));

    int32_t *past = A.p, *curr = B.p, *target = C.p;
    double *pcurr = pA.p, *pprev = pB.p;
    double prevMod = p->lower, currMod = -1.0;
    const double lower = p->lower;
    int numIters = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (timing) {
        VG_CUDA(cudaEventCreate(&ev0));
        VG_CUDA(cudaEventCreate(&ev1));
    }
    for (;;) {
        numIters++;
        SweepArgs a{};
        a.rowptr = g->rowptr;
        a.tail = g->tail;
        a.weight = g->weight;
        a.curr = curr;
        a.target = target;
        a.vdeg = vdeg.p;
        a.cdeg = cdeg.p;
        a.csize = csize.p;
        a.cupd = cupd.p;
        a.cw = cw.p;
        a.frozen = frozen.p;
        a.active = use_et ? active.p : nullptr;
        a.ref = g->ref;
        a.noprune = noprune.p;
        a.ne = g->ne;
        a.ident = numIters == 1 ? 1 : 0; // k_init put every vertex in its own community
        a.constant = constant;
        if (timing) VG_CUDA(cudaEventRecord(ev0, ctx->stream));
        for (int64_t ci = 0; ci < numColor; ci++) {
            sweep_color(ctx, a, bk, ci, hp, ordering == 0, nv);
            if (ordering == 1 && nv) { // per-color community update (louvain.cpp:724-735)
                LaunchTimer lt(ctx);
                k_apply_seg<<<agrid, SEG_THREADS, 0, ctx->stream>>>(
                    seg.voff.p, seg.cb.p, 1, seg.C, cdeg.p, csize.p, cupd.p, cw.p, a.active,
                    nullptr, 0, part.p, noprune.p);
                VG_CHECK_LAUNCH();
            }
        }
        if (timing) VG_CUDA(cudaEventRecord(ev1, ctx->stream));
        if (nv) {
            {
                LaunchTimer lt(ctx);
                k_apply_seg<<<agrid, SEG_THREADS, 0, ctx->stream>>>(
                    seg.voff.p, seg.cb.p, 1, seg.C, cdeg.p, csize.p, cupd.p, cw.p, a.active,
                    nullptr, 1, part.p, noprune.p);
            }
            VG_CHECK_LAUNCH();
            {
                LaunchTimer lt(ctx);
                k_mod_seg<<<1, SEG_FINAL, 0, ctx->stream>>>(part.p, seg.cb.p, 1, constant, nullptr,
                                                           modv.p, BatchDecide{});
            }
            VG_CHECK_LAUNCH();
            VG_CUDA(cudaMemcpyAsync(hmod, modv.p, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                    ctx->stream));
        } else {
            hmod[0] = NAN;
            hmod[1] = 0.0;
        }
        vg_sync(ctx);
        if (timing) {
            float ms = 0.f;
            VG_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
            timing->sweep_ms += ms;
            timing->edges += g->ne;
        }
        if (max_iters > 0 && numIters >= max_iters) break;
        if (et == 3 || et == 4) { // ETLocalOrRemote == false (louvain.cpp:112-121)
            if ((long)hmod[1] >= 90) { // ET_CUTOFF (louvain.hpp:70)
                currMod = -1;
                break;
            }
        }
        currMod = hmod[0];
        // a NaN modularity (no edges, 2m = 0) would never pass the reference's test
        // (louvain.cpp:553-563); the phase ends there instead of looping
        if (std::isnan(currMod) || (currMod - prevMod) < p->threshold) break;
        prevMod = currMod;
        if (prevMod < lower) prevMod = lower;
        if (et == 0) {
            int32_t *tmp = past; // louvain.cpp:565-570
            past = curr;
            curr = target;
            target = tmp;
        } else if (et == 1 || et == 3) {
            LaunchTimer lt(ctx);
            k_swap_et13<<<grid, 256, 0, ctx->stream>>>(nv, numIters, past, curr, target, active.p,
                                                       g->ref);
            VG_CHECK_LAUNCH();
        } else {
            {
                LaunchTimer lt(ctx);
                k_swap_et24<<<grid, 256, 0, ctx->stream>>>(nv, numIters, 1.0 - p->et_delta, past,
                                                           curr, target, active.p, pcurr, pprev);
            }
            VG_CHECK_LAUNCH();
            std::swap(pcurr, pprev);
        }
    }
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    (void)currMod;
    // cvect = pastComm (louvain.cpp:579): keep it on the device for the rebuild
    vg_free(ctx, g->comm, sizeof(int32_t) * nv);
    g->comm = nullptr;
    if (past == A.p) g->comm = A.detach();
    else if (past == B.p) g->comm = B.detach();
    else g->comm = C.detach();
    *mod_out = prevMod;
    *iters_out = numIters;
}

namespace {

// result of graph j = the buffer that held pastComm when its loop ended
__global__ void k_gather_result(int64_t nv, const int32_t *__restrict__ vjob,
                                const int8_t *__restrict__ resbuf, const int32_t *__restrict__ b0,
                                const int32_t *__restrict__ b1, const int32_t *__restrict__ b2,
                                int32_t *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int r = resbuf[vjob[i]];
        out[i] = r == 0 ? b0[i] : (r == 1 ? b1[i] : b2[i]);
    }
}

} // namespace

// One Louvain phase (plain distLouvainMethod, louvain.cpp:427-591) for each of the
// J graphs packed in U (graph j owns vertices [voff[j], voff[j+1]) and only
// references its own vertices). Every graph keeps its own 1/(2m), modularity,
// loop test and iteration count; a graph whose loop has ended is skipped by all
// later launches. Results: U->comm (each graph's pastComm at its break),
// mod_out[j] (prevMod) and iters_out[j].
void vg_phase_batch_internal(vg_ctx *ctx, vg_graph *U, int64_t J, const int64_t *h_voff,
                             const int32_t *vjob, const double *h_thresh, const double *h_lower,
                             double *mod_out, int32_t *iters_out, double *sweep_ms) {
    configure_kernels_once();
    const int64_t nv = U->nv;
    VG_REQUIRE(J >= 1 && nv >= J, "a batch needs at least one vertex per graph");
    SegTable seg;
    seg_table_build(ctx, h_voff, J, seg);
    DevBuf<double> vdeg(ctx, nv), cw(ctx, nv), cdeg(ctx, nv);
    DevBuf<int32_t> csize(ctx, nv);
    DevBuf<CommInfo> cupd(ctx, nv);
    DevBuf<int32_t> B0(ctx, nv), B1(ctx, nv), B2(ctx, nv);
    const int grid = vg_grid(ctx, nv, 256);
    DevBuf<int32_t> noprune(ctx, 1); // see can_prune
    VG_CUDA(cudaMemsetAsync(noprune.p, 0, sizeof(int32_t), ctx->stream));
    vertex_degrees(ctx, U, vdeg.p, (int)vg_weights_integral(ctx, U));
    // per-graph 2m in each graph's own fixed order, 1/(2m) on the host as in the plain path
    DevBuf<double> jconst(ctx, J);
    {
        DevBuf<double> tm(ctx, J);
        seg_sums(ctx, vdeg.p, seg, tm.p);
        std::vector<double> h(J);
        VG_CUDA(cudaMemcpyAsync(h.data(), tm.p, sizeof(double) * J, cudaMemcpyDeviceToHost,
                                ctx->stream));
        vg_sync(ctx);
        for (auto &x : h) x = 1.0 / x; // distCalcConstantForSecondTerm (louvain.cpp:2217)
        VG_CUDA(cudaMemcpyAsync(jconst.p, h.data(), sizeof(double) * J, cudaMemcpyHostToDevice,
                                ctx->stream));
        vg_sync(ctx);
    }
    {
        LaunchTimer lt(ctx);
        k_init<<<grid, 256, 0, ctx->stream>>>(nv, vdeg.p, cdeg.p, csize.p, cupd.p, B0.p, B1.p, B2.p,
                                              nullptr, nullptr, nullptr, noprune.p);
    }
    VG_CHECK_LAUNCH();
    Buckets bk;
    build_buckets(ctx, U, nullptr, 1, bk);
    HubPlan hp;
    plan_hubs(ctx, U, bk, 1, hp);
    DevBuf<double> part(ctx, 3 * std::max<int64_t>(seg.C, 1));
    const int agrid = seg_grid(ctx, seg.C);
    // per-graph loop state
    DevBuf<double> prev_mod(ctx, J), lower(ctx, J), thresh(ctx, J);
    DevBuf<int32_t> iters(ctx, J), live(ctx, 1);
    DevBuf<uint8_t> done(ctx, J);
    DevBuf<int8_t> resbuf(ctx, J);
    VG_CUDA(cudaMemcpyAsync(prev_mod.p, h_lower, sizeof(double) * J, cudaMemcpyHostToDevice, ctx->stream));
    VG_CUDA(cudaMemcpyAsync(lower.p, h_lower, sizeof(double) * J, cudaMemcpyHostToDevice, ctx->stream));
    VG_CUDA(cudaMemcpyAsync(thresh.p, h_thresh, sizeof(double) * J, cudaMemcpyHostToDevice, ctx->stream));
    VG_CUDA(cudaMemsetAsync(iters.p, 0, sizeof(int32_t) * J, ctx->stream));
    VG_CUDA(cudaMemsetAsync(done.p, 0, J, ctx->stream));
    VG_CUDA(cudaMemsetAsync(resbuf.p, 0, J, ctx->stream));
    int32_t *hlive = (int32_t *)vg_pinned(ctx, sizeof(int32_t));
    int32_t *bufs[3] = {B0.p, B1.p, B2.p};
    DevBuf<int32_t> iter_dev(ctx, 1);
    VG_CUDA(cudaMemsetAsync(iter_dev.p, 0, sizeof(int32_t), ctx->stream));
    // one iteration with bufs[pi] = past, bufs[pi+1] = curr, bufs[pi+2] = target; the
    // iteration number is `it`, or read from iter_dev after k_iter_inc when `graph`
    auto enqueue = [&](int pi, int32_t it, bool graph, cudaEvent_t e0, cudaEvent_t e1) {
        if (graph) k_iter_inc<<<1, 1, 0, ctx->stream>>>(iter_dev.p);
        SweepArgs a{};
        a.rowptr = U->rowptr;
        a.tail = U->tail;
        a.weight = U->weight;
        a.curr = bufs[(pi + 1) % 3];
        a.target = bufs[(pi + 2) % 3];
        a.vdeg = vdeg.p;
        a.cdeg = cdeg.p;
        a.csize = csize.p;
        a.cupd = cupd.p;
        a.cw = cw.p;
        a.ref = U->ref;
        a.noprune = noprune.p;
        a.ne = U->ne;
        a.constant = 0.0;
        a.vjob = vjob;
        a.jconst = jconst.p;
        a.jdone = done.p;
        VG_CUDA(cudaMemsetAsync(live.p, 0, sizeof(int32_t), ctx->stream));
        if (e0) VG_CUDA(cudaEventRecord(e0, ctx->stream));
        sweep_color(ctx, a, bk, 0, hp, true, nv);
        if (e1) VG_CUDA(cudaEventRecord(e1, ctx->stream));
        {
            LaunchTimer lt(ctx);
            k_apply_seg<<<agrid, SEG_THREADS, 0, ctx->stream>>>(seg.voff.p, seg.cb.p, J, seg.C,
                                                                cdeg.p, csize.p, cupd.p, cw.p,
                                                                nullptr, done.p, 1, part.p,
                                                                noprune.p);
        }
        VG_CHECK_LAUNCH();
        BatchDecide bd;
        bd.prev_mod = prev_mod.p;
        bd.lower = lower.p;
        bd.thresh = thresh.p;
        bd.iters = iters.p;
        bd.done = done.p;
        bd.resbuf = resbuf.p;
        bd.live_count = live.p;
        bd.iter = it;
        bd.past_idx = pi;
        bd.iter_dev = graph ? iter_dev.p : nullptr;
        {
            LaunchTimer lt(ctx);
            k_mod_seg<<<(int)std::min<int64_t>(J, 65535), SEG_FINAL, 0, ctx->stream>>>(
                part.p, seg.cb.p, J, 0.0, jconst.p, nullptr, bd);
        }
        VG_CHECK_LAUNCH();
        VG_CUDA(cudaMemcpyAsync(hlive, live.p, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    };
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (sweep_ms) *sweep_ms = 0.0;
    if (!ctx->profile) {
        // captured iterations: three graphs (one per rotation of the community
        // buffers) replayed in turn, one launch and one 4-byte read-back per iteration
        cudaGraphExec_t exec[3] = {nullptr, nullptr, nullptr};
        int64_t per_iter = 0;
        auto destroy = [&] {
            for (auto &e : exec)
                if (e) cudaGraphExecDestroy(e);
        };
        try {
            for (int pi = 0; pi < 3; pi++) {
                const int64_t l0 = ctx->profile_launches;
                cudaGraph_t gr = nullptr;
                VG_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
                try {
                    enqueue(pi, 0, true, nullptr, nullptr);
                } catch (...) {
                    cudaStreamEndCapture(ctx->stream, &gr);
                    if (gr) cudaGraphDestroy(gr);
                    throw;
                }
                VG_CUDA(cudaStreamEndCapture(ctx->stream, &gr));
                const cudaError_t e = cudaGraphInstantiate(&exec[pi], gr, 0);
                cudaGraphDestroy(gr);
                VG_CUDA(e);
                per_iter = ctx->profile_launches - l0 + 1; // + k_iter_inc
                ctx->profile_launches = l0;
            }
            int pi = 0;
            for (;;) {
                VG_CUDA(cudaGraphLaunch(exec[pi], ctx->stream));
                ctx->profile_launches += per_iter;
                pi = (pi + 1) % 3;
                vg_sync(ctx);
                if (*hlive == 0) break;
            }
        } catch (...) {
            destroy();
            throw;
        }
        destroy();
    } else {
        VG_CUDA(cudaEventCreate(&ev0));
        VG_CUDA(cudaEventCreate(&ev1));
        for (int32_t it = 1;; it++) {
            const int pi = (it - 1) % 3; // past <- curr <- target <- past (louvain.cpp:565-570)
            enqueue(pi, it, false, sweep_ms ? ev0 : nullptr, sweep_ms ? ev1 : nullptr);
            vg_sync(ctx);
            if (sweep_ms) {
                float ms = 0.f;
                VG_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
                *sweep_ms += ms;
            }
            if (*hlive == 0) break;
        }
    }
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    vg_free(ctx, U->comm, sizeof(int32_t) * nv);
    U->comm = nullptr;
    DevBuf<int32_t> out(ctx, nv);
    {
        LaunchTimer lt(ctx);
        k_gather_result<<<grid, 256, 0, ctx->stream>>>(nv, vjob, resbuf.p, B0.p, B1.p, B2.p, out.p);
    }
    VG_CHECK_LAUNCH();
    U->comm = out.detach();
    VG_CUDA(cudaMemcpyAsync(mod_out, prev_mod.p, sizeof(double) * J, cudaMemcpyDeviceToHost,
                            ctx->stream));
    VG_CUDA(cudaMemcpyAsync(iters_out, iters.p, sizeof(int32_t) * J, cudaMemcpyDeviceToHost,
                            ctx->stream));
    vg_sync(ctx);
}

void vg_phase_internal(vg_ctx *ctx, vg_graph *g, const vg_phase_params *p, double *mod_out,
                       int32_t *iters_out, double *sweep_ms, int64_t *edges) {
    PhaseTiming t;
    run_phase(ctx, g, p, mod_out, iters_out, sweep_ms ? &t : nullptr);
    if (sweep_ms) *sweep_ms = t.sweep_ms;
    if (edges) *edges = t.edges;
}

void vg_download_comm(vg_ctx *ctx, const int32_t *comm, int64_t n, int64_t *out) {
    if (!n) return;
    DevBuf<int64_t> wide(ctx, n);
    {
        LaunchTimer lt(ctx);
        k_widen<<<vg_grid(ctx, n, 256), 256, 0, ctx->stream>>>(comm, n, wide.p);
    }
    VG_CHECK_LAUNCH();
    VG_CUDA(cudaMemcpyAsync(out, wide.p, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
    vg_sync(ctx);
}

// host int64 ids -> device int32, each in [-1, lim)
void vg_upload_ids(vg_ctx *ctx, const int64_t *in, int64_t n, int64_t lim, int32_t *out) {
    if (!n) return;
    DevBuf<int64_t> wide(ctx, n);
    DevBuf<int> bad(ctx, 1);
    VG_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
    VG_CUDA(cudaMemcpyAsync(wide.p, in, sizeof(int64_t) * n, cudaMemcpyHostToDevice, ctx->stream));
    {
        LaunchTimer lt(ctx);
        k_narrow<<<vg_grid(ctx, n, 256), 256, 0, ctx->stream>>>(wide.p, n, lim, out, bad.p);
    }
    VG_CHECK_LAUNCH();
    int *hb = (int *)vg_pinned(ctx, sizeof(int));
    VG_CUDA(cudaMemcpyAsync(hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    vg_sync(ctx);
    VG_REQUIRE(*hb == 0, "id out of range");
}

extern "C" vg_status vg_louvain_phase(vg_ctx *ctx, vg_graph *g, const vg_phase_params *p,
                                      int64_t *cvect_out, double *mod_out, int32_t *iters_out) {
    if (!ctx || !g || !p || !mod_out || !iters_out) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        run_phase(ctx, g, p, mod_out, iters_out, nullptr);
        if (cvect_out) vg_download_comm_ref(ctx, g, g->comm, cvect_out);
    });
}

extern "C" vg_status vg_ctx_get_tuning(const vg_ctx *ctx, vg_tuning *out) {
    if (!ctx || !out) return VG_ERR_ARG;
    *out = effective_tuning(ctx);
    return VG_OK;
}

extern "C" vg_status vg_ctx_set_tuning(vg_ctx *ctx, const vg_tuning *t) {
    if (!ctx || !t) return VG_ERR_ARG;
    if (!tuning_valid(*t)) {
        ctx->last_error = "vg_ctx_set_tuning: t32 must be 0 or 1, 32 <= ws_max <= wt_max <= ct_max "
                          "with ws_max <= 128, wt_max <= 512, ct_max <= 4096, 1 <= tile_grid <= 1024";
        return VG_ERR_ARG;
    }
    ctx->tune = *t;
    return VG_OK;
}

// Coordinate descent over the tuning fields: each candidate's cost is the summed
// sweep time (CUDA events around the sweep launches) of the first `sweeps`
// iterations of a plain phase on every graph, the faster of two timings. A change
// is kept when it saves more than 1 %.
extern "C" vg_status vg_autotune(vg_ctx *ctx, vg_graph *const *graphs, int32_t n, int32_t sweeps,
                                 vg_tuning *best_out, double *best_ms_out, double *start_ms_out) {
    if (!ctx || !graphs || n < 1 || sweeps < 0 || sweeps > 8) return VG_ERR_ARG;
    for (int32_t i = 0; i < n; i++)
        if (!graphs[i]) return VG_ERR_ARG;
    const vg_tuning start = effective_tuning(ctx);
    return vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        const int its = sweeps == 0 ? 2 : sweeps;
        vg_phase_params pp{};
        pp.lower = -1.0;
        pp.threshold = 1e-6;
        pp.et_type = 0;
        pp.et_delta = 1.0;
        pp.ordering = 0;
        auto one = [&](const vg_tuning &t) {
            ctx->tune = t;
            double total = 0.0;
            for (int32_t i = 0; i < n; i++) {
                vg_graph tmp = *graphs[i]; // shares the CSR; the trial's communities are its own
                tmp.comm = nullptr;
                PhaseTiming pt;
                double mod = 0.0;
                int32_t it = 0;
                try {
                    run_phase(ctx, &tmp, &pp, &mod, &it, &pt, its);
                } catch (...) {
                    if (tmp.comm) vg_free(ctx, tmp.comm, sizeof(int32_t) * tmp.nv);
                    throw;
                }
                if (tmp.comm) vg_free(ctx, tmp.comm, sizeof(int32_t) * tmp.nv);
                graphs[i]->integral = tmp.integral; // the cached weight test
                total += pt.sweep_ms;
            }
            return total;
        };
        auto cost = [&](const vg_tuning &t) { return std::min(one(t), one(t)); };
        vg_tuning best = start;
        double best_ms = 0.0, start_ms = 0.0;
        try {
            start_ms = best_ms = cost(start);
            const int32_t t32s[] = {1, 0};
            const int32_t wss[] = {64, 96, 128};
            const int32_t wts[] = {256, 384, 512};
            const int32_t cts[] = {1024, 2048, 4096};
            const int32_t grids[] = {16, 32, 64, 128};
            auto consider = [&](vg_tuning t) {
                if (!tuning_valid(t)) return;
                if (t.t32 == best.t32 && t.ws_max == best.ws_max && t.wt_max == best.wt_max &&
                    t.ct_max == best.ct_max && t.tile_grid == best.tile_grid)
                    return;
                const double c = cost(t);
                if (c < 0.99 * best_ms) {
                    best = t;
                    best_ms = c;
                }
            };
            for (int32_t v : t32s) { vg_tuning t = best; t.t32 = v; consider(t); }
            for (int32_t v : wss) { vg_tuning t = best; t.ws_max = v; consider(t); }
            for (int32_t v : wts) { vg_tuning t = best; t.wt_max = v; consider(t); }
            for (int32_t v : cts) { vg_tuning t = best; t.ct_max = v; consider(t); }
            for (int32_t v : grids) { vg_tuning t = best; t.tile_grid = v; consider(t); }
        } catch (...) {
            ctx->tune = start;
            throw;
        }
        ctx->tune = best;
        if (best_out) *best_out = best;
        if (best_ms_out) *best_ms_out = best_ms;
        if (start_ms_out) *start_ms_out = start_ms;
    });
}

extern "C" vg_status vg_vertex_degree(vg_ctx *ctx, vg_graph *g, double *vdeg_out,
                                      double *constant_out) {
    if (!ctx || !g) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        DevBuf<double> vdeg(ctx, g->nv);
        if (g->nv) vertex_degrees(ctx, g, vdeg.p, (int)vg_weights_integral(ctx, g));
        const double tm = g->nv ? twice_m_one(ctx, vdeg.p, g->nv) : 0.0;
        if (constant_out) *constant_out = 1.0 / tm;
        if (vdeg_out && g->nv) {
            VG_CUDA(cudaMemcpyAsync(vdeg_out, vdeg.p, sizeof(double) * g->nv, cudaMemcpyDeviceToHost,
                                    ctx->stream));
        }
        vg_sync(ctx);
    });
}
