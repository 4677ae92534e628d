// Vite's binary graph file read straight into a device graph, and written from one.
//
// The format (distgraph.cpp:119-253 reads it with MPI-IO, writeGraph and the converters
// write it, converters/convert.cpp:245-278): [nv:i64][ne:i64][rowptr:i64 x (nv+1)]
// [Edge{tail:i64, weight:f64} x ne]. The reader rebases the offsets to start at zero
// (distgraph.cpp:244-247), checks them and every tail, and converts the 16-byte edge
// records to the library's int32 tails and FP64 weights on the device. The edge array
// streams through two pinned host buffers: while chunk k is copied to the device and
// split there, the host reads chunk k+1 from the file, so disk reads, PCIe copies and
// the conversion overlap.
#include "vg_internal.cuh"

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cerrno>
#include <cstring>

namespace {

constexpr size_t IO_CHUNK = 64ull << 20; // most bytes per pinned buffer (a multiple of 16)

// rowptr -= base (after vg_check_rowptr_async has read them all)
__global__ void k_rebase(int64_t *__restrict__ rp, int64_t n1, int64_t base) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n1;
         i += (int64_t)gridDim.x * blockDim.x)
        rp[i] -= base;
}

// Vite edge records -> int32 tails in [0, nv) and FP64 weights
__global__ void k_split_records(const longlong2 *__restrict__ e, int64_t n, int64_t nv,
                                int32_t *__restrict__ tail, double *__restrict__ w,
                                int *__restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const longlong2 v = e[i];
        if (v.x < 0 || v.x >= nv) *bad = 1;
        tail[i] = (int32_t)v.x;
        w[i] = __longlong_as_double(v.y);
    }
}

struct Fd {
    int fd = -1;
    ~Fd() {
        if (fd >= 0) close(fd);
    }
};

struct Pinned {
    void *p = nullptr;
    ~Pinned() {
        if (p) cudaFreeHost(p);
    }
};

void pread_all(int fd, void *buf, size_t len, off_t off, const char *path) {
    char *p = static_cast<char *>(buf);
    while (len) {
        const ssize_t got = pread(fd, p, len, off);
        if (got < 0 && errno == EINTR) continue;
        VG_REQUIRE(got > 0, "short read from %s at byte %lld", path, (long long)off);
        p += got;
        len -= (size_t)got;
        off += got;
    }
}

void pwrite_all(int fd, const void *buf, size_t len, off_t off, const char *path) {
    const char *p = static_cast<const char *>(buf);
    while (len) {
        const ssize_t put = pwrite(fd, p, len, off);
        if (put < 0 && errno == EINTR) continue;
        VG_REQUIRE(put > 0, "write to %s failed at byte %lld: %s", path, (long long)off,
                   strerror(errno));
        p += put;
        len -= (size_t)put;
        off += put;
    }
}

} // namespace

extern "C" vg_status vg_graph_read_vite(vg_ctx *ctx, const char *path, vg_graph **out) {
    if (!ctx || !path || !out) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        *out = nullptr;
        VG_CUDA(cudaSetDevice(ctx->device));
        Fd f;
        f.fd = open(path, O_RDONLY);
        VG_REQUIRE(f.fd >= 0, "cannot open %s: %s", path, strerror(errno));
        struct stat st;
        VG_REQUIRE(fstat(f.fd, &st) == 0, "cannot stat %s", path);
        int64_t hdr[2];
        VG_REQUIRE(st.st_size >= (off_t)sizeof(hdr), "%s is shorter than the 16-byte header", path);
        pread_all(f.fd, hdr, sizeof(hdr), 0, path);
        const int64_t nv = hdr[0], ne = hdr[1];
        VG_REQUIRE(nv >= 0 && ne >= 0 && nv < (int64_t)INT32_MAX && ne < ((int64_t)1 << 40),
                   "%s: bad header (nv=%lld, ne=%lld; vertices must be fewer than 2^31)", path,
                   (long long)nv, (long long)ne);
        const int64_t rp_bytes = 8 * (nv + 1), e_bytes = 16 * ne;
        VG_REQUIRE((int64_t)st.st_size >= 16 + rp_bytes + e_bytes,
                   "%s is truncated: %lld bytes for nv=%lld, ne=%lld (need %lld)", path,
                   (long long)st.st_size, (long long)nv, (long long)ne,
                   (long long)(16 + rp_bytes + e_bytes));
        DevBuf<int64_t> rp(ctx, nv + 1);
        DevBuf<int32_t> tail(ctx, ne);
        DevBuf<double> w(ctx, ne);
        DevBuf<int> bad(ctx, 2);
        VG_CUDA(cudaMemsetAsync(bad.p, 0, 2 * sizeof(int), ctx->stream));
        // pinned buffers sized to the file (a small file needs no 64 MiB buffers), a
        // multiple of 16 bytes so edge records never straddle two chunks
        const size_t chunk = (size_t)std::min<int64_t>(
            (int64_t)IO_CHUNK, (std::max<int64_t>(std::max(rp_bytes, e_bytes), 4096) + 15) & ~15LL);
        Pinned hb[2];
        VG_CUDA(cudaMallocHost(&hb[0].p, chunk));
        VG_CUDA(cudaMallocHost(&hb[1].p, chunk));
        cudaEvent_t done[2] = {nullptr, nullptr};
        VG_CUDA(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming));
        VG_CUDA(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming));
        auto destroy = [&] {
            for (auto &e : done)
                if (e) cudaEventDestroy(e);
        };
        try {
            // reuse of pinned buffer b waits for the copy that last read it
            bool used[2] = {false, false};
            auto take = [&](int b) {
                if (used[b]) VG_CUDA(cudaEventSynchronize(done[b]));
                used[b] = true;
            };
            // row offsets
            int64_t base = 0;
            int k = 0;
            for (int64_t off = 0; off < rp_bytes; off += (int64_t)chunk, k++) {
                const int b = k & 1;
                const size_t len = (size_t)std::min<int64_t>((int64_t)chunk, rp_bytes - off);
                take(b);
                pread_all(f.fd, hb[b].p, len, 16 + off, path);
                if (off == 0) base = *static_cast<int64_t *>(hb[b].p);
                VG_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(rp.p) + off, hb[b].p, len,
                                        cudaMemcpyHostToDevice, ctx->stream));
                VG_CUDA(cudaEventRecord(done[b], ctx->stream));
            }
            vg_check_rowptr_async(ctx, rp.p, nv + 1, base, ne, bad.p);
            if (base != 0) {
                LaunchTimer lt(ctx);
                k_rebase<<<vg_grid(ctx, nv + 1, 256), 256, 0, ctx->stream>>>(rp.p, nv + 1, base);
            }
            VG_CHECK_LAUNCH();
            // edge records, chunk by chunk through two device staging buffers
            if (ne) {
                const int64_t per = (int64_t)(chunk / 16);
                DevBuf<longlong2> stage[2];
                stage[0].alloc(ctx, (size_t)std::min<int64_t>(per, ne));
                stage[1].alloc(ctx, (size_t)std::min<int64_t>(per, ne));
                for (int64_t e0 = 0; e0 < ne; e0 += per, k++) {
                    const int b = k & 1;
                    const int64_t n = std::min<int64_t>(per, ne - e0);
                    take(b);
                    pread_all(f.fd, hb[b].p, (size_t)(16 * n), 16 + rp_bytes + 16 * e0, path);
                    VG_CUDA(cudaMemcpyAsync(stage[b].p, hb[b].p, (size_t)(16 * n),
                                            cudaMemcpyHostToDevice, ctx->stream));
                    VG_CUDA(cudaEventRecord(done[b], ctx->stream));
                    {
                        LaunchTimer lt(ctx);
                        k_split_records<<<vg_grid(ctx, n, 256), 256, 0, ctx->stream>>>(
                            stage[b].p, n, nv, tail.p + e0, w.p + e0, bad.p + 1);
                    }
                    VG_CHECK_LAUNCH();
                }
            }
            int *hbad = (int *)vg_pinned(ctx, 2 * sizeof(int));
            VG_CUDA(cudaMemcpyAsync(hbad, bad.p, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                                    ctx->stream));
            vg_sync(ctx);
            VG_REQUIRE(hbad[0] == 0, "%s: row offsets decrease, hold a row of 2^31 or more entries or "
                                   "do not end at ne=%lld", path,
                       (long long)ne);
            VG_REQUIRE(hbad[1] == 0, "%s: an edge tail is outside [0, nv=%lld)", path,
                       (long long)nv);
        } catch (...) {
            cudaStreamSynchronize(ctx->stream); // no copy may still read the pinned buffers
            destroy();
            throw;
        }
        destroy();
        *out = vg_graph_wrap(ctx, nv, ne, rp.detach(), tail.detach(), w.detach());
    });
}

extern "C" vg_status vg_graph_write_vite(vg_ctx *ctx, const vg_graph *g, const char *path) {
    if (!ctx || !g || !path) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        const int64_t nv = g->nv, ne = g->ne;
        // the graph in Vite's layout and reference vertex order
        std::vector<int64_t> rowptr((size_t)nv + 1);
        std::vector<vg_edge> edges((size_t)ne);
        const vg_status s = vg_graph_download(ctx, g, rowptr.data(), edges.data());
        if (s != VG_OK) vg_throw(s, "%s", ctx->last_error.c_str());
        Fd f;
        f.fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
        VG_REQUIRE(f.fd >= 0, "cannot create %s: %s", path, strerror(errno));
        const int64_t hdr[2] = {nv, ne};
        pwrite_all(f.fd, hdr, sizeof(hdr), 0, path);
        pwrite_all(f.fd, rowptr.data(), sizeof(int64_t) * (size_t)(nv + 1), sizeof(hdr), path);
        if (ne)
            pwrite_all(f.fd, edges.data(), sizeof(vg_edge) * (size_t)ne,
                       (off_t)(sizeof(hdr) + sizeof(int64_t) * (size_t)(nv + 1)), path);
        VG_REQUIRE(close(f.fd) == 0, "closing %s failed: %s", path, strerror(errno));
        f.fd = -1;
    });
}
