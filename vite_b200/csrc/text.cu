// Text edge lists read straight into a device graph: the input formats of Vite's
// fileConvert (converters/convert.cpp:102-281) that the clustering tools are fed
// with -- a plain edge list (-s, converters/simple.cpp:61-160), a SNAP file (-n,
// converters/snap.cpp:65-196) and a Matrix Market coordinate file (-m,
// converters/matrix-market.cpp:65-241) -- with fileConvert's weight options (-w all
// ones, -i the file's weights, -r random weights, default their absolute values) and
// one-based ids (-z, plain lists).
//
// The file is read into pinned memory and copied to the device once. The few header
// lines of SNAP and Matrix Market files are parsed on the host; the rest is cut into
// lines (or, for SNAP, blank-separated tokens) by a flag scan, every line is parsed by
// one thread, and the edges go through the same stable (source, tail) sort that builds
// every other CSR here (vg_csr_from_triples, duplicates kept), so each row lists its
// tails in increasing order and equal pairs in file order. Weights that the exact
// device conversion cannot round correctly (text_parse.cuh) are converted on the host
// with strtod.
//
// What the reference does and this does not, by design:
//   * its SNAP reader sizes the edge list to 2 x numEdges default entries before
//     appending the real ones (snap.cpp:123-124), so processGraphData's assertion
//     (utils.cpp:145) stops every SNAP conversion; this implements what the reader
//     computes otherwise (ids renumbered from 0 in order of first appearance, every
//     edge in both directions, unit or random weights, numVertices from the header);
//   * a line that does not parse in the middle of a plain list or a Matrix Market file
//     leaves variables uninitialised there; here it is an error (VG_ERR_ARG);
//   * std::sort leaves equal (source, tail) pairs in an unspecified order; here they
//     keep the file's order.
// Kept as the reference does: a plain list's text after its last newline is not an
// edge (simple.cpp:100-112 reads one line fewer than it counted) although its ids
// still count towards the number of vertices; ids of Matrix Market files are 1-based;
// a self loop of a symmetric Matrix Market file is stored once, any other entry in
// both directions; a missing or unreadable weight is 0 (C++11 operator>>); -r draws
// the weights of std::default_random_engine through
// std::uniform_real_distribution<double>(0.01, 1.0) (utils.cpp:93-99), one draw per
// edge in file order, restated from the C++ standard's minstd_rand0 and
// generate_canonical so that the weights are the reference's own.
#include "vg_internal.cuh"
#include "text_parse.cuh"

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

namespace {

using namespace vgtext;

// per-line parse status
enum : int8_t { L_SKIP = 0, L_EDGE = 1, L_BAD = 2, L_VERTS = 3 };

// line (or token) heads: i starts one when it is the region's first byte or follows a
// newline (tokens: a non-blank byte after a blank one)
__global__ void k_heads(const char *__restrict__ s, int64_t n, int tokens,
                        int32_t *__restrict__ flag) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int32_t f;
        if (tokens)
            f = !is_space((unsigned char)s[i]) && (i == 0 || is_space((unsigned char)s[i - 1]));
        else
            f = i == 0 || s[i - 1] == '\n';
        flag[i] = f;
    }
}

__global__ void k_scatter_heads(const int32_t *__restrict__ flag, const int64_t *__restrict__ idx,
                                int64_t n, int64_t *__restrict__ starts) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        if (flag[i]) starts[idx[i]] = i;
}

struct ParseOut {
    int64_t *a, *b;      // the two ids
    double *w;           // the weight (as read; the weight mode is applied later)
    int64_t *wtok;       // start of a weight token the host must convert, else -1
    int8_t *st;          // L_*
    int32_t *emit;       // entries this line adds to the edge list
    int32_t *draw;       // 1 when the line takes one random draw (-r)
    unsigned long long *bad_line; // first line that does not parse (atomicMin)
    long long *max_id;   // largest id seen (plain lists: the number of vertices - 1)
    int32_t *n_host;     // weight tokens left to the host
    int32_t *range_bad;  // an id outside [0, nv) (Matrix Market)
};

enum { FMT_SIMPLE = 1, FMT_SNAP = 2, FMT_MM = 3 };

// one thread per line of a plain list (simple.cpp:100-160) or of the data lines of a
// Matrix Market file (matrix-market.cpp:164-236)
// (lines [0, L) of the Lall lines that start in s[0, n))
__global__ void k_parse_lines(const char *__restrict__ s, int64_t n,
                              const int64_t *__restrict__ starts, int64_t L, int64_t Lall,
                              int fmt, int read_weight, int one_based, int symmetric, int64_t nv,
                              int64_t final_piece, ParseOut o) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < L;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = starts[k];
        int64_t e = k + 1 < Lall ? starts[k + 1] : n;
        if (e > b && s[e - 1] == '\n') e--;
        int8_t st = L_EDGE;
        int64_t v0 = 0, v1 = 0, tok = -1;
        double w = fmt == FMT_MM ? 1.0 : 0.0; // pattern entries keep 1.0
        int emit = 0, draw = 0;
        if (fmt == FMT_SIMPLE && b < e && (s[b] == '#' || s[b] == '%')) {
            st = L_SKIP;
        } else {
            int64_t p = b;
            const int r0 = parse_i64(s, &p, e, &v0, false);
            const int r1 = r0 == 1 ? parse_i64(s, &p, e, &v1, false) : 0;
            if (r0 != 1 || r1 != 1) {
                st = L_BAD;
                // a failed read stores 0 (C++11); only the first id is certain then
                if (k == final_piece) v0 = r0 == 1 ? v0 : 0;
            } else if (read_weight) {
                double x = 0.0;
                int64_t ts = -1;
                const int rw = parse_f64(s, &p, e, &x, &ts);
                if (rw == F_OK) w = x;
                else if (rw == F_NONE) w = 0.0;
                else {
                    w = 0.0;
                    tok = ts;
                    atomicAdd(o.n_host, 1);
                }
            }
            if (fmt == FMT_MM || one_based) {
                v0--;
                v1--;
            }
            if (k == final_piece) {
                // text after the last newline: its ids count, it is not an edge
                if (st == L_BAD && fmt == FMT_SIMPLE) v1 = v0;
                if (fmt == FMT_SIMPLE) {
                    atomicMax(o.max_id, (long long)(v0 > v1 ? v0 : v1));
                    st = L_VERTS;
                }
                tok = -1;
            } else if (st == L_EDGE) {
                if (fmt == FMT_SIMPLE) {
                    if (v0 < 0 || v1 < 0) atomicOr(o.range_bad, 1);
                    atomicMax(o.max_id, (long long)(v0 > v1 ? v0 : v1));
                    emit = 2;
                } else {
                    if (v0 < 0 || v0 >= nv || v1 < 0 || v1 >= nv) atomicOr(o.range_bad, 1);
                    emit = (symmetric && v0 != v1) ? 2 : 1;
                }
                draw = 1;
            }
        }
        if (st == L_BAD && k != final_piece)
            atomicMin(o.bad_line, (unsigned long long)k);
        o.a[k] = v0;
        o.b[k] = v1;
        o.w[k] = w;
        o.wtok[k] = tok;
        o.st[k] = st;
        o.emit[k] = emit;
        o.draw[k] = draw;
    }
}

// SNAP: one thread per token of the first 2 x numEdges (snap.cpp:134-143)
__global__ void k_parse_tokens(const char *__restrict__ s, int64_t n,
                               const int64_t *__restrict__ starts, int64_t T,
                               int64_t *__restrict__ val, uint64_t *__restrict__ key,
                               uint32_t *__restrict__ pos, unsigned long long *__restrict__ bad) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < T;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t p = starts[k], v = 0;
        const int64_t e = n;
        const int r = parse_i64(s, &p, e, &v, false);
        // a token must be a whole number (what follows it is a blank or the end)
        if (r != 1 || (p < e && !is_space((unsigned char)s[p]))) atomicMin(bad, (unsigned long long)k);
        val[k] = v;
        key[k] = (uint64_t)v;
        pos[k] = (uint32_t)k;
    }
}

// runs of equal ids after the sort: the run's first position (its first appearance)
// is marked in `first`
__global__ void k_first_appearance(const uint64_t *__restrict__ key,
                                   const uint32_t *__restrict__ pos, int64_t T,
                                   int32_t *__restrict__ first) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < T;
         i += (int64_t)gridDim.x * blockDim.x)
        first[pos[i]] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
}

// every token gets the new id of its run (the rank of the run's first appearance)
__global__ void k_run_ids(const uint64_t *__restrict__ key, const uint32_t *__restrict__ pos,
                          int64_t T, const int64_t *__restrict__ rank, int64_t *__restrict__ id) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < T;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i != 0 && key[i] == key[i - 1]) continue;
        const int64_t r = rank[pos[i]];
        for (int64_t j = i; j < T && key[j] == key[i]; j++) id[pos[j]] = r;
    }
}

// std::default_random_engine (minstd_rand0: x <- 16807 x mod 2^31 - 1, seed 1) and
// generate_canonical<double, 53> over it (two draws: r = 2^31 - 2, 53 bits need
// ceil(53 / 30) words), as std::uniform_real_distribution<double>(0.01, 1.0) uses
// them for genRandom (utils.cpp:93-99); draw j of the stream is x_j = 16807^j mod M
__device__ uint64_t minstd_pow(uint64_t e) {
    const uint64_t M = 2147483647ULL;
    uint64_t r = 1, b = 16807ULL;
    while (e) {
        if (e & 1) r = (r * b) % M;
        b = (b * b) % M;
        e >>= 1;
    }
    return r;
}

__device__ double random_weight(int64_t edge) {
    const uint64_t x1 = minstd_pow(2 * (uint64_t)edge + 1);
    const uint64_t x2 = (x1 * 16807ULL) % 2147483647ULL;
    const double r = 2147483646.0;
    double sum = __dmul_rn((double)(x1 - 1), 1.0);
    const double tmp1 = r;
    sum = __dadd_rn(sum, __dmul_rn((double)(x2 - 1), tmp1));
    const double tmp2 = 4611686009837453316.0; // (double)(r * r), rounded as the loop's long double product is
    double c = __ddiv_rn(sum, tmp2);
    if (c >= 1.0) c = 0.99999999999999989; // nextafter(1.0, 0.0)
    return __dadd_rn(__dmul_rn(c, __dsub_rn(1.0, 0.01)), 0.01);
}

enum { W_ABS = 0, W_ORIG = 1, W_ONE = 2, W_RANDOM = 3 };

// the edge list: each line's entries at its offset, weights after the weight mode
__global__ void k_emit_lines(const ParseOut o, int64_t L, const int64_t *__restrict__ at,
                             const int64_t *__restrict__ ordinal, int wmode, int pattern,
                             int32_t *__restrict__ src, int32_t *__restrict__ dst,
                             double *__restrict__ w) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < L;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int m = o.emit[k];
        if (!m) continue;
        double x = o.w[k];
        if (wmode == W_ABS && !pattern) x = fabs(x);
        if (wmode == W_ONE) x = 1.0;
        if (wmode == W_RANDOM) x = random_weight(ordinal[k]);
        const int64_t p = at[k];
        const int32_t u = (int32_t)o.a[k], v = (int32_t)o.b[k];
        src[p] = u;
        dst[p] = v;
        w[p] = x;
        if (m == 2) {
            src[p + 1] = v;
            dst[p + 1] = u;
            w[p + 1] = x;
        }
    }
}

__global__ void k_emit_snap(const int64_t *__restrict__ id, int64_t M, int wmode,
                            int32_t *__restrict__ src, int32_t *__restrict__ dst,
                            double *__restrict__ w) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < M;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = (int32_t)id[2 * k], v = (int32_t)id[2 * k + 1];
        const double x = wmode == W_RANDOM ? random_weight(k) : 1.0;
        src[2 * k] = u;
        dst[2 * k] = v;
        w[2 * k] = x;
        src[2 * k + 1] = v;
        dst[2 * k + 1] = u;
        w[2 * k + 1] = x;
    }
}

struct Pinned {
    void *p = nullptr;
    ~Pinned() {
        if (p) cudaFreeHost(p);
    }
};

struct Fd {
    int fd = -1;
    ~Fd() {
        if (fd >= 0) close(fd);
    }
};

// whole file into pinned host memory
int64_t read_file(const char *path, Pinned &buf) {
    Fd f;
    f.fd = open(path, O_RDONLY);
    VG_REQUIRE(f.fd >= 0, "cannot open %s: %s", path, strerror(errno));
    struct stat st;
    VG_REQUIRE(fstat(f.fd, &st) == 0, "cannot stat %s", path);
    const int64_t n = st.st_size;
    VG_CUDA(cudaMallocHost(&buf.p, (size_t)n + 1));
    char *p = static_cast<char *>(buf.p);
    int64_t got = 0;
    while (got < n) {
        const ssize_t r = pread(f.fd, p + got, (size_t)(n - got), got);
        if (r < 0 && errno == EINTR) continue;
        VG_REQUIRE(r > 0, "short read from %s at byte %lld", path, (long long)got);
        got += r;
    }
    p[n] = '\0';
    return n;
}

// the host's view of a line: [b, e) without its newline
int64_t line_end(const char *s, int64_t b, int64_t n) {
    const void *q = memchr(s + b, '\n', (size_t)(n - b));
    return q ? (int64_t)(static_cast<const char *>(q) - s) : n;
}

std::string upper(std::string x) {
    for (auto &c : x) c = (char)toupper((unsigned char)c);
    return x;
}

// line or token heads of s[0, n) on the device: returns their count
int64_t heads(vg_ctx *ctx, const char *d_s, int64_t n, bool tokens, DevBuf<int64_t> &starts) {
    if (n == 0) return 0;
    DevBuf<int32_t> flag(ctx, n);
    DevBuf<int64_t> idx(ctx, n);
    { LaunchTimer lt(ctx);
      k_heads<<<vg_grid(ctx, n, 256), 256, 0, ctx->stream>>>(d_s, n, tokens ? 1 : 0, flag.p); }
    VG_CHECK_LAUNCH();
    const int64_t L = vg_exclusive_scan_i32_to_i64(ctx, flag.p, idx.p, n);
    starts.alloc(ctx, std::max<int64_t>(L, 1));
    if (L) {
        LaunchTimer lt(ctx);
        k_scatter_heads<<<vg_grid(ctx, n, 256), 256, 0, ctx->stream>>>(flag.p, idx.p, n, starts.p);
    }
    VG_CHECK_LAUNCH();
    return L;
}

} // namespace

extern "C" vg_status vg_graph_read_text(vg_ctx *ctx, const char *path, const vg_text_params *tp,
                                        vg_graph **out) {
    if (!ctx || !path || !tp || !out) return VG_ERR_ARG;
    return vg_guard(ctx, [&] {
        *out = nullptr;
        VG_CUDA(cudaSetDevice(ctx->device));
        const int fmt = tp->format;
        const int wmode = tp->weights;
        VG_REQUIRE(fmt == VG_TEXT_SIMPLE || fmt == VG_TEXT_SNAP || fmt == VG_TEXT_MATRIX_MARKET,
                   "unknown text format %d", fmt);
        VG_REQUIRE(wmode >= VG_WEIGHTS_ABS && wmode <= VG_WEIGHTS_RANDOM, "unknown weight mode %d",
                   wmode);
        VG_REQUIRE(!tp->one_based || fmt == VG_TEXT_SIMPLE,
                   "one-based ids (-z) apply to plain edge lists only");
        Pinned hb;
        const int64_t n = read_file(path, hb);
        const char *hs = static_cast<const char *>(hb.p);

        // header (host): where the data begin, and the counts the header gives
        int64_t d0 = 0, nv = -1, nedges = -1;
        bool symmetric = false, pattern = false;
        if (fmt == VG_TEXT_SNAP) {
            // leading '#' lines; the one naming "Nodes" gives numVertices and numEdges
            int64_t p = 0;
            while (p < n && hs[p] == '#') {
                const int64_t e = line_end(hs, p, n);
                const std::string line(hs + p, (size_t)(e - p));
                if (line.find("Nodes") != std::string::npos) {
                    int64_t vals[2] = {-1, -1};
                    int c = 0;
                    size_t q = 0;
                    while (c < 2 && (q = line.find(':', q)) != std::string::npos) {
                        q++;
                        char *endp = nullptr;
                        const long long x = strtoll(line.c_str() + q, &endp, 10);
                        if (endp == line.c_str() + q) break;
                        vals[c++] = x;
                    }
                    nv = vals[0];
                    nedges = vals[1];
                }
                p = e < n ? e + 1 : n;
            }
            d0 = p;
            VG_REQUIRE(nv >= 0 && nedges >= 0,
                       "%s: no '# Nodes: <n> Edges: <m>' line in the SNAP header", path);
        } else if (fmt == VG_TEXT_MATRIX_MARKET) {
            int64_t e = line_end(hs, 0, n);
            char f[5][64] = {{0}};
            const std::string first(hs, (size_t)e);
            const int got = sscanf(first.c_str(), "%63s %63s %63s %63s %63s", f[0], f[1], f[2],
                                   f[3], f[4]);
            VG_REQUIRE(got == 5, "%s: cannot parse the Matrix Market banner", path);
            VG_REQUIRE(std::string(f[0]) == "%%MatrixMarket",
                       "%s: the first line must start with %%%%MatrixMarket", path);
            VG_REQUIRE(upper(f[1]) == "MATRIX", "%s: the object type must be matrix", path);
            VG_REQUIRE(upper(f[2]) == "COORDINATE", "%s: the format must be coordinate", path);
            pattern = upper(f[3]) == "PATTERN";
            const std::string sym = upper(f[4]);
            symmetric = sym == "SYMMETRIC";
            VG_REQUIRE(symmetric || sym == "GENERAL",
                       "%s: the symmetry must be SYMMETRIC or GENERAL", path);
            int64_t p = e < n ? e + 1 : n;
            while (p < n && hs[p] == '%') {
                e = line_end(hs, p, n);
                p = e < n ? e + 1 : n;
            }
            e = line_end(hs, p, n);
            long long ns = -1, nt = -1, ne = -1;
            const std::string sz(hs + p, (size_t)(e - p));
            VG_REQUIRE(sscanf(sz.c_str(), "%lld %lld %lld", &ns, &nt, &ne) == 3 && ns >= 0 && ne >= 0,
                       "%s: cannot parse the Matrix Market size line", path);
            nv = ns;
            nedges = ne;
            d0 = e < n ? e + 1 : n;
        }
        VG_REQUIRE(nv < (int64_t)INT32_MAX, "%s: %lld vertices (the device needs fewer than 2^31)",
                   path, (long long)nv);

        const int64_t nd = n - d0; // data region
        DevBuf<char> ds(ctx, std::max<int64_t>(nd, 1));
        if (nd)
            VG_CUDA(cudaMemcpyAsync(ds.p, hs + d0, (size_t)nd, cudaMemcpyHostToDevice, ctx->stream));
        DevBuf<int64_t> starts;
        DevBuf<int32_t> src, dst;
        DevBuf<double> w;
        int64_t m = 0;
        int64_t *hcnt = (int64_t *)vg_pinned(ctx, 4 * sizeof(int64_t));

        if (fmt == VG_TEXT_SNAP) {
            const int64_t T = heads(ctx, ds.p, nd, true, starts);
            VG_REQUIRE(T >= 2 * nedges, "%s: %lld edges announced, %lld ids found", path,
                       (long long)nedges, (long long)T);
            const int64_t t2 = 2 * nedges;
            VG_REQUIRE(t2 < (int64_t)UINT32_MAX, "%s: too many edges", path);
            DevBuf<int64_t> val(ctx, std::max<int64_t>(t2, 1)), id(ctx, std::max<int64_t>(t2, 1));
            DevBuf<uint64_t> key(ctx, std::max<int64_t>(t2, 1));
            DevBuf<uint32_t> pos(ctx, std::max<int64_t>(t2, 1));
            DevBuf<unsigned long long> bad(ctx, 1);
            VG_CUDA(cudaMemsetAsync(bad.p, 0xff, sizeof(unsigned long long), ctx->stream));
            int64_t nuniq = 0;
            if (t2) {
                { LaunchTimer lt(ctx);
                  k_parse_tokens<<<vg_grid(ctx, t2, 256), 256, 0, ctx->stream>>>(
                      ds.p, nd, starts.p, t2, val.p, key.p, pos.p, bad.p); }
                VG_CHECK_LAUNCH();
                VG_CUDA(cudaMemcpyAsync(hcnt, bad.p, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                        ctx->stream));
                vg_sync(ctx);
                VG_REQUIRE(hcnt[0] == -1, "%s: SNAP id %lld of the edge list is not a number", path,
                           (long long)hcnt[0]);
                // ids renumbered from 0 in order of first appearance (snap.cpp:146-168)
                vg_radix_sort_pairs(ctx, key.p, pos.p, t2, 64);
                DevBuf<int32_t> first(ctx, t2);
                DevBuf<int64_t> rank(ctx, t2);
                { LaunchTimer lt(ctx);
                  k_first_appearance<<<vg_grid(ctx, t2, 256), 256, 0, ctx->stream>>>(key.p, pos.p, t2,
                                                                                     first.p); }
                VG_CHECK_LAUNCH();
                nuniq = vg_exclusive_scan_i32_to_i64(ctx, first.p, rank.p, t2);
                { LaunchTimer lt(ctx);
                  k_run_ids<<<vg_grid(ctx, t2, 256), 256, 0, ctx->stream>>>(key.p, pos.p, t2, rank.p,
                                                                            id.p); }
                VG_CHECK_LAUNCH();
            }
            VG_REQUIRE(nuniq <= nv, "%s: %lld distinct ids, but the header gives %lld nodes", path,
                       (long long)nuniq, (long long)nv);
            m = t2;
            src.alloc(ctx, m);
            dst.alloc(ctx, m);
            w.alloc(ctx, m);
            if (nedges) {
                LaunchTimer lt(ctx);
                k_emit_snap<<<vg_grid(ctx, nedges, 256), 256, 0, ctx->stream>>>(
                    id.p, nedges, wmode == VG_WEIGHTS_RANDOM ? W_RANDOM : W_ONE, src.p, dst.p, w.p);
            }
            VG_CHECK_LAUNCH();
        } else {
            const int64_t Lall = heads(ctx, ds.p, nd, false, starts);
            int64_t L = Lall;
            int64_t final_piece = -1;
            if (fmt == VG_TEXT_SIMPLE) {
                // the text after the last newline (simple.cpp:100-112); none when the
                // file ends with one
                if (nd > 0 && hs[n - 1] != '\n') final_piece = L - 1;
            } else {
                VG_REQUIRE(L >= nedges, "%s: %lld entries announced, %lld lines found", path,
                           (long long)nedges, (long long)L);
                L = nedges; // lines after the announced entries are not read
            }
            const int Lb = (int)std::max<int64_t>(L, 1);
            DevBuf<int64_t> a(ctx, Lb), b(ctx, Lb), wtok(ctx, Lb), at(ctx, Lb), ord(ctx, Lb);
            DevBuf<double> wl(ctx, Lb);
            DevBuf<int8_t> st(ctx, Lb);
            DevBuf<int32_t> emit(ctx, Lb), draw(ctx, Lb);
            DevBuf<unsigned long long> bad(ctx, 1);
            DevBuf<long long> maxid(ctx, 1);
            DevBuf<int32_t> flags(ctx, 2);
            VG_CUDA(cudaMemsetAsync(bad.p, 0xff, sizeof(unsigned long long), ctx->stream));
            const long long minus1 = -1;
            VG_CUDA(cudaMemcpyAsync(maxid.p, &minus1, sizeof(long long), cudaMemcpyHostToDevice,
                                    ctx->stream));
            VG_CUDA(cudaMemsetAsync(flags.p, 0, 2 * sizeof(int32_t), ctx->stream));
            ParseOut o{a.p, b.p, wl.p, wtok.p, st.p, emit.p, draw.p, bad.p, maxid.p, flags.p,
                       flags.p + 1};
            const bool read_weight =
                (wmode == VG_WEIGHTS_ABS || wmode == VG_WEIGHTS_ORIGINAL) && !pattern;
            if (L) {
                LaunchTimer lt(ctx);
                k_parse_lines<<<vg_grid(ctx, L, 256), 256, 0, ctx->stream>>>(
                    ds.p, nd, starts.p, L, Lall, fmt == VG_TEXT_SIMPLE ? FMT_SIMPLE : FMT_MM,
                    read_weight ? 1 : 0, tp->one_based ? 1 : 0, symmetric ? 1 : 0, nv,
                    final_piece, o);
            }
            VG_CHECK_LAUNCH();
            VG_CUDA(cudaMemcpyAsync(&hcnt[0], bad.p, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                    ctx->stream));
            VG_CUDA(cudaMemcpyAsync(&hcnt[1], maxid.p, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                    ctx->stream));
            VG_CUDA(cudaMemcpyAsync(&hcnt[2], flags.p, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                    ctx->stream));
            vg_sync(ctx);
            const int32_t n_host = ((int32_t *)&hcnt[2])[0], range_bad = ((int32_t *)&hcnt[2])[1];
            VG_REQUIRE(hcnt[0] == -1, "%s: data line %lld does not hold two ids", path,
                       (long long)hcnt[0] + 1);
            VG_REQUIRE(!range_bad, fmt == VG_TEXT_SIMPLE ? "%s: a negative vertex id"
                                                         : "%s: an entry's row or column is outside [1, %lld]",
                       path, (long long)nv);
            if (fmt == VG_TEXT_SIMPLE) {
                // every piece that is not a comment counts towards the largest id; an
                // empty last piece reads as id 0 (a failed read stores 0)
                int64_t mx = hcnt[1];
                if (nd == 0 || hs[n - 1] == '\n') mx = std::max<int64_t>(mx, tp->one_based ? -1 : 0);
                nv = mx + 1;
                VG_REQUIRE(nv < (int64_t)INT32_MAX, "%s: ids up to %lld (the device needs fewer "
                           "than 2^31 vertices)", path, (long long)mx);
            }
            if (n_host > 0) {
                // weights the device cannot round correctly: strtod on the host
                std::vector<int64_t> ht(L);
                std::vector<double> hw(L);
                VG_CUDA(cudaMemcpyAsync(ht.data(), wtok.p, sizeof(int64_t) * L,
                                        cudaMemcpyDeviceToHost, ctx->stream));
                VG_CUDA(cudaMemcpyAsync(hw.data(), wl.p, sizeof(double) * L,
                                        cudaMemcpyDeviceToHost, ctx->stream));
                vg_sync(ctx);
                for (int64_t k = 0; k < L; k++)
                    if (ht[k] >= 0) hw[k] = strtod(hs + d0 + ht[k], nullptr);
                VG_CUDA(cudaMemcpyAsync(wl.p, hw.data(), sizeof(double) * L,
                                        cudaMemcpyHostToDevice, ctx->stream));
                vg_sync(ctx);
            }
            // output offsets, and each edge line's place in the random stream
            m = L ? vg_exclusive_scan_i32_to_i64(ctx, emit.p, at.p, L) : 0;
            if (L && wmode == VG_WEIGHTS_RANDOM) vg_exclusive_scan_i32_to_i64(ctx, draw.p, ord.p, L);
            src.alloc(ctx, std::max<int64_t>(m, 1));
            dst.alloc(ctx, std::max<int64_t>(m, 1));
            w.alloc(ctx, std::max<int64_t>(m, 1));
            if (L) {
                const int wk = wmode == VG_WEIGHTS_ABS ? W_ABS
                               : wmode == VG_WEIGHTS_ORIGINAL ? W_ORIG
                               : wmode == VG_WEIGHTS_ONE ? W_ONE : W_RANDOM;
                LaunchTimer lt(ctx);
                k_emit_lines<<<vg_grid(ctx, L, 256), 256, 0, ctx->stream>>>(
                    o, L, at.p, ord.p, wk, pattern ? 1 : 0, src.p, dst.p, w.p);
            }
            VG_CHECK_LAUNCH();
        }
        VG_REQUIRE(nv >= 0, "%s: no vertices", path);
        VG_REQUIRE(m < (int64_t)UINT32_MAX, "%s: too many entries", path);
        vg_graph *g = vg_csr_from_triples(ctx, nv, src, dst, w, m, false, nullptr);
        vg_sync(ctx);
        *out = g;
    });
}
