// Allocation-free variant of the vertex-degree step (distSumVertexDegree +
// distCalcConstantForSecondTerm): the same per-row degree sums as vg_vertex_degree,
// with the reduction's scratch in a file-scope device array instead of memory
// allocated per call. For callers that cannot allocate device memory while they
// run: a serving process that carved its whole memory budget at start-up, a host
// framework whose own allocator owns the device memory, a caller for which an
// allocation failing or stalling mid-run is not acceptable.
//
// Limits and sharing:
//   * at most VG_NOALLOC_MAX_VERTICES vertices (one partial sum per 2048 vertices,
//     65,536 partials = 512 KiB of device memory, held by every GPU that loads the
//     library until the process exits); larger graphs are rejected with an error;
//   * every call shares the one array and overwrites exactly the partials it then
//     reads, so nothing has to start at zero; calls that overlap on the GPU (two
//     streams, two host threads) race on it and must be serialised by the caller;
//   * the first call on a device looks up the array's device address with that
//     device current (cudaGetSymbolAddress). The address is kept for the life of
//     the process: a cudaDeviceReset would leave it stale, so the entry point must
//     not be used on a device after a reset;
//   * the row offsets are not checked (checking them would need memory of its
//     own): the caller passes a valid CSR, offsets non-decreasing and inside the
//     weights array.
#include "vg_internal.cuh"

#include <mutex>

namespace {

constexpr int NA_TILE = 2048;       // vertices per partial sum
constexpr int NA_THREADS = 256;
constexpr int NA_MAX_TILES = 65536; // partials held in the array
constexpr int NA_MAX_DEVICES = 64;

// [0, NA_MAX_TILES): per-tile partial sums of the degrees; [NA_MAX_TILES]: 1/(2m)
static __device__ __align__(256) double g_noalloc_scratch[NA_MAX_TILES + 32];

std::mutex g_noalloc_mutex;
double *g_noalloc_addr[NA_MAX_DEVICES] = {};

__device__ double na_block_sum(double v, double *ws) {
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

// rows longer than this are folded by the whole warp
constexpr int64_t NA_LONG = 64;

// one block per tile: each row summed in CSR order (as distSumVertexDegree), and
// the tile's degrees reduced into its partial. A lane folds its own row when it is
// short; the warp's long rows (hubs) are folded one after another by all its lanes
// (vg_warp_ordered_fold: the lanes fetch the row's weights ahead of lane 0's chain of
// additions, in static shared memory), so a hub costs one addition per entry
__global__ void __launch_bounds__(NA_THREADS) k_na_degree(const int64_t *__restrict__ rowptr,
                                                          const double *__restrict__ w, int64_t nv,
                                                          double *__restrict__ vdeg,
                                                          double *__restrict__ partial) {
    __shared__ double ws[32];
    __shared__ double stage[NA_THREADS / 32][2 * VG_FOLD_STEP];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    const int64_t base = (int64_t)blockIdx.x * NA_TILE;
    for (int k = threadIdx.x; k < NA_TILE; k += NA_THREADS) { // warp-uniform trip count
        const int64_t v = base + k;
        const bool valid = v < nv;
        int64_t e0 = 0, e1 = 0;
        if (valid) {
            e0 = rowptr[v];
            e1 = rowptr[v + 1];
        }
        // w is null only for a CSR without entries (checked on the host)
        const bool lng = valid && w && e1 - e0 > NA_LONG;
        double tw = 0.0;
        if (valid && w && !lng)
            for (int64_t e = e0; e < e1; e++) tw = __dadd_rn(tw, w[e]);
        for (unsigned lm = __ballot_sync(full, lng); lm; lm &= lm - 1) {
            const int src = __ffs(lm) - 1;
            const int64_t E0 = __shfl_sync(full, e0, src), E1 = __shfl_sync(full, e1, src);
            const double *__restrict__ rw = w + E0;
            double acc = vg_warp_ordered_fold(E1 - E0, [rw](int64_t j) { return rw[j]; },
                                              stage[threadIdx.x >> 5], 0.0, false);
            acc = __shfl_sync(full, acc, 0); // lane 0 holds the fold
            if (lane == src) tw = acc;
        }
        if (valid) {
            vdeg[v] = tw;
            s = __dadd_rn(s, tw);
        }
    }
    s = na_block_sum(s, ws);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// one block: the partials in a fixed order, then 1/(2m)
__global__ void __launch_bounds__(NA_THREADS) k_na_constant(const double *__restrict__ partial,
                                                            int ntiles, double *__restrict__ out) {
    __shared__ double ws[32];
    double s = 0.0;
    for (int t = threadIdx.x; t < ntiles; t += NA_THREADS) s = __dadd_rn(s, partial[t]);
    s = na_block_sum(s, ws);
    if (threadIdx.x == 0) out[0] = 1.0 / s;
}

void set_err(char *errbuf, size_t errlen, const char *msg) {
    if (errbuf && errlen) snprintf(errbuf, errlen, "%s", msg);
}

} // namespace

extern "C" vg_status vg_vertex_degree_noalloc(int64_t nv, const int64_t *d_rowptr,
                                              const double *d_weight, double *d_vdeg_out,
                                              double *constant_out, void *stream, char *errbuf,
                                              size_t errlen) {
    char msg[256];
    if (nv < 1 || !d_rowptr || !d_vdeg_out || !constant_out) {
        set_err(errbuf, errlen, "vg_vertex_degree_noalloc: nv must be >= 1 and the pointers non-null");
        return VG_ERR_ARG;
    }
    if (nv > (int64_t)NA_TILE * NA_MAX_TILES) {
        snprintf(msg, sizeof(msg),
                 "vg_vertex_degree_noalloc: nv = %lld exceeds the allocation-free maximum of %lld "
                 "vertices; use vg_vertex_degree",
                 (long long)nv, (long long)NA_TILE * NA_MAX_TILES);
        set_err(errbuf, errlen, msg);
        return VG_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) {
        set_err(errbuf, errlen, "vg_vertex_degree_noalloc: no current CUDA device");
        return VG_ERR_CUDA;
    }
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_addr[dev]) {
            // set-up, once per device, with that device current
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) {
                snprintf(msg, sizeof(msg), "vg_vertex_degree_noalloc: cudaGetSymbolAddress: %s",
                         cudaGetErrorString(e));
                set_err(errbuf, errlen, msg);
                return VG_ERR_CUDA;
            }
            g_noalloc_addr[dev] = static_cast<double *>(p);
        }
        scratch = g_noalloc_addr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!d_weight) {
        // no weights: allowed for a CSR without entries only (rowptr[0] == rowptr[nv]);
        // two 8-byte reads into host stack memory, nothing allocated
        int64_t ends[2] = {0, 0};
        e = cudaMemcpyAsync(&ends[0], d_rowptr, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&ends[1], d_rowptr + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            snprintf(msg, sizeof(msg), "vg_vertex_degree_noalloc: %s", cudaGetErrorString(e));
            set_err(errbuf, errlen, msg);
            return VG_ERR_CUDA;
        }
        if (ends[1] != ends[0]) {
            snprintf(msg, sizeof(msg),
                     "vg_vertex_degree_noalloc: d_weight is NULL but the CSR holds %lld entries",
                     (long long)(ends[1] - ends[0]));
            set_err(errbuf, errlen, msg);
            return VG_ERR_ARG;
        }
    }
    const int ntiles = (int)((nv + NA_TILE - 1) / NA_TILE);
    k_na_degree<<<ntiles, NA_THREADS, 0, s>>>(d_rowptr, d_weight, nv, d_vdeg_out, scratch);
    k_na_constant<<<1, NA_THREADS, 0, s>>>(scratch, ntiles, scratch + NA_MAX_TILES);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(constant_out, scratch + NA_MAX_TILES, sizeof(double),
                            cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        snprintf(msg, sizeof(msg), "vg_vertex_degree_noalloc: %s", cudaGetErrorString(e));
        set_err(errbuf, errlen, msg);
        return VG_ERR_CUDA;
    }
    return VG_OK;
}
