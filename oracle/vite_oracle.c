/*
 * vite_oracle.c -- plain-C, single-threaded restatement of Vite's Louvain path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg are the only users.
 *
 * Every function follows the reference in the order a one-thread run of the
 * reference takes, so every floating-point sum is the same left fold and the
 * results match a one-thread reference run bit for bit. Citations are
 * file:line in the reference (ECP-ExaGraph/vite).
 */
#define _POSIX_C_SOURCE 200809L
#include "vite_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define VO_PI 3.14159            /* distgraph.hpp:65 */
#define VO_MLCG 2147483647LL     /* utils.hpp:79 */
#define VO_ALCG 16807LL          /* utils.hpp:80 */
#define VO_ET_CUTOFF 90          /* louvain.hpp:70 */
#define VO_P_CUTOFF 0.02         /* louvain.hpp:74 */
#define VO_MAX_COVG 70           /* coloring.hpp:69-71 */
#define VO_PHASE_CAP 200         /* utils.hpp:67-69 */

/* ------------------------------------------------------------------------ */
/* graph lifetime                                                            */

int vo_graph_alloc(vo_graph *g, int64_t nv, int64_t ne)
{
    g->nv = nv;
    g->ne = ne;
    g->rowptr = (int64_t *)calloc((size_t)nv + 1, sizeof(int64_t));
    g->tail = (int64_t *)malloc((size_t)(ne > 0 ? ne : 1) * sizeof(int64_t));
    g->weight = (double *)malloc((size_t)(ne > 0 ? ne : 1) * sizeof(double));
    return (g->rowptr && g->tail && g->weight) ? 0 : -1;
}

void vo_graph_free(vo_graph *g)
{
    free(g->rowptr);
    free(g->tail);
    free(g->weight);
    memset(g, 0, sizeof(*g));
}

/* ------------------------------------------------------------------------ */
/* counter-based random numbers shared with the CUDA generators (own design) */

static uint64_t sm64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

uint64_t vo_mix(uint64_t seed, uint64_t stream, uint64_t k)
{
    return sm64(sm64(seed ^ (stream * 0xD1B54A32D192ED03ULL)) ^ k);
}

static uint64_t uint_below(uint64_t r, uint64_t n)
{
    return (uint64_t)(((unsigned __int128)r * (unsigned __int128)n) >> 64);
}

static double unit_double(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

/* ------------------------------------------------------------------------ */
/* LCG and RGG (utils.hpp:135-330, distgraph.cpp:391-983)                    */

static uint32_t seedseq_T(uint32_t x) { return x ^ (x >> 27); }

/* std::seed_seq({seed}).generate(1 word), restated from the C++ standard's
 * [rand.util.seedseq] algorithm (n = 1 output, s = 1 input); used by
 * LCG::reseeder (utils.hpp:163-170). */
uint32_t vo_seed_seq1(uint32_t seed)
{
    const uint32_t n = 1, s = 1;
    uint32_t b[1] = {0x8b8b8b8bu};
    const uint32_t t = 0; /* (n - 1) / 2 for n < 7 */
    const uint32_t p = (n - t) / 2, q = p + t, m = (s + 1 > n) ? s + 1 : n;
    for (uint32_t k = 0; k < m; k++) {
        uint32_t r1 = 1664525u * seedseq_T(b[k % n] ^ b[(k + p) % n] ^ b[(k + n - 1) % n]);
        uint32_t r2 = r1 + (k == 0 ? s : (k <= s ? (k % n) + seed : k % n));
        b[(k + p) % n] += r1;
        b[(k + q) % n] += r2;
        b[k % n] = r2;
    }
    for (uint32_t k = m; k < m + n; k++) {
        uint32_t r3 = 1566083941u * seedseq_T(b[k % n] + b[(k + p) % n] + b[(k + n - 1) % n]);
        uint32_t r4 = r3 - (k % n);
        b[(k + p) % n] ^= r3;
        b[(k + q) % n] ^= r4;
        b[k % n] = r4;
    }
    return b[0];
}

/* LCG constructor + generate() for one rank (utils.hpp:139-158, 248-298):
 * x0 = reseeder(seed); x_i = x_{i-1} * 16807 mod (2^31 - 1);
 * drand_i = |x_i| * (1 / (1 + (M - 1))). */
void vo_lcg_drand(uint32_t seed, int64_t count, double *drand)
{
    const double mult = 1.0 / (double)(1.0 + (double)(VO_MLCG - 1));
    int64_t x = (int64_t)vo_seed_seq1(seed);
    for (int64_t i = 0; i < count; i++) {
        if (i > 0) x = (x * VO_ALCG) % VO_MLCG;
        drand[i] = (double)(fabs((double)x) * mult);
    }
}

/* distgraph.cpp:395-399 */
double vo_rgg_radius(int64_t n)
{
    double rc = sqrt((double)log((double)n) / (double)(VO_PI * (double)n));
    double rt = sqrt((double)2.0736 / (double)n);
    return (rc + rt) / (double)2.0;
}

typedef struct { int64_t src, dst; double w; } vo_trip;
typedef struct { int64_t dst; double w; } vo_half;

static int half_cmp(const void *a, const void *b)
{
    const vo_half *x = (const vo_half *)a, *y = (const vo_half *)b;
    return x->dst < y->dst ? -1 : (x->dst > y->dst ? 1 : 0);
}

/* Sort one row's (tail, weight) pairs by tail: insertion sort for short rows,
 * qsort through a scratch array for long ones. */
static void sort_row(int64_t *tail, double *w, int64_t len, vo_half *scratch)
{
    if (len <= 48) {
        for (int64_t a = 1; a < len; a++) {
            const int64_t t = tail[a];
            const double x = w[a];
            int64_t b = a - 1;
            while (b >= 0 && tail[b] > t) {
                tail[b + 1] = tail[b];
                w[b + 1] = w[b];
                b--;
            }
            tail[b + 1] = t;
            w[b + 1] = x;
        }
        return;
    }
    for (int64_t a = 0; a < len; a++) { scratch[a].dst = tail[a]; scratch[a].w = w[a]; }
    qsort(scratch, (size_t)len, sizeof(vo_half), half_cmp);
    for (int64_t a = 0; a < len; a++) { tail[a] = scratch[a].dst; w[a] = scratch[a].w; }
}

/* CSR sorted by (src, dst) from a triple list (distgraph.cpp:899-952 order):
 * a counting sort by source, then each row sorted by destination. The
 * generators never emit a (src, dst) pair twice, so the order is unique. */
static int csr_from_triples(int64_t n, const vo_trip *t, int64_t m, vo_graph *out)
{
    if (vo_graph_alloc(out, n, m)) return -1;
    for (int64_t k = 0; k < m; k++) out->rowptr[t[k].src + 1]++;
    for (int64_t i = 0; i < n; i++) out->rowptr[i + 1] += out->rowptr[i];
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    if (!fill) return -1;
    memcpy(fill, out->rowptr, sizeof(int64_t) * (size_t)n);
    int64_t maxlen = 0;
    for (int64_t k = 0; k < m; k++) {
        const int64_t p = fill[t[k].src]++;
        out->tail[p] = t[k].dst;
        out->weight[p] = t[k].w;
    }
    free(fill);
    for (int64_t i = 0; i < n; i++) {
        const int64_t len = out->rowptr[i + 1] - out->rowptr[i];
        if (len > maxlen) maxlen = len;
    }
    vo_half *scratch = (vo_half *)malloc(sizeof(vo_half) * (size_t)(maxlen > 0 ? maxlen : 1));
    if (!scratch) return -1;
    for (int64_t i = 0; i < n; i++)
        sort_row(out->tail + out->rowptr[i], out->weight + out->rowptr[i],
                 out->rowptr[i + 1] - out->rowptr[i], scratch);
    free(scratch);
    return 0;
}

/* 1 when row i of a (src, dst)-sorted CSR holds tail j (binary search). */
static int csr_has(const vo_graph *g, int64_t i, int64_t j)
{
    int64_t lo = g->rowptr[i], hi = g->rowptr[i + 1];
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo) / 2;
        if (g->tail[mid] < j) lo = mid + 1;
        else hi = mid;
    }
    return lo < g->rowptr[i + 1] && g->tail[lo] == j;
}

/* generateRGG for one rank (distgraph.cpp:412-983) without extra edges. The
 * reference tests all pairs i<j; this restatement tests the pairs in adjacent
 * cells of a grid whose cells are wider than r(n), with the identical
 * predicate `sqrt(dx*dx + dy*dy) <= rn` and dx = X[i]-X[j] for i<j
 * (distgraph.cpp:533-562), so the edge set and weights are the same. */
int vo_rgg(int64_t n, vo_graph *out)
{
    const double rn = vo_rgg_radius(n);
    double *X = (double *)malloc(sizeof(double) * (size_t)(2 * n));
    double *Y = (double *)malloc(sizeof(double) * (size_t)n);
    vo_lcg_drand(1, 2 * n, X); /* LCG xr(1, X.data(), 2*n) (distgraph.cpp:476) */
    const double lo = 0.0, range = 1.0 / (double)1;
    for (int64_t j = 0; j < n; j++) Y[j] = lo + (double)(range * X[n + j]); /* rescale (utils.hpp:299-321) */

    double xmin = X[0], xmax = X[0], ymin = Y[0], ymax = Y[0];
    for (int64_t i = 1; i < n; i++) {
        if (X[i] < xmin) xmin = X[i];
        if (X[i] > xmax) xmax = X[i];
        if (Y[i] < ymin) ymin = Y[i];
        if (Y[i] > ymax) ymax = Y[i];
    }
    const double cw = rn * (1.0 + 1e-9);
    int64_t ncx = (int64_t)floor((xmax - xmin) / cw) + 1, ncy = (int64_t)floor((ymax - ymin) / cw) + 1;
    if (ncx > 65536) ncx = 65536;
    if (ncy > 65536) ncy = 65536;
    const double sx = (double)ncx / ((xmax - xmin) + cw), sy = (double)ncy / ((ymax - ymin) + cw);
    int64_t *cell = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    int64_t *cstart = (int64_t *)calloc((size_t)(ncx * ncy + 1), sizeof(int64_t));
    int64_t *order = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    for (int64_t i = 0; i < n; i++) {
        int64_t cx = (int64_t)((X[i] - xmin) * sx), cy = (int64_t)((Y[i] - ymin) * sy);
        if (cx >= ncx) cx = ncx - 1;
        if (cy >= ncy) cy = ncy - 1;
        cell[i] = cy * ncx + cx;
        cstart[cell[i] + 1]++;
    }
    for (int64_t c = 0; c < ncx * ncy; c++) cstart[c + 1] += cstart[c];
    {
        int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)(ncx * ncy));
        memcpy(fill, cstart, sizeof(int64_t) * (size_t)(ncx * ncy));
        for (int64_t i = 0; i < n; i++) order[fill[cell[i]]++] = i;
        free(fill);
    }
    int64_t cap = 16 * n + 16, m = 0;
    vo_trip *t = (vo_trip *)malloc(sizeof(vo_trip) * (size_t)cap);
    /* vertices visited cell by cell (neighbouring points stay in cache); the
     * CSR assembly sorts the pairs, so the visiting order leaves it unchanged */
    for (int64_t q = 0; q < n; q++) {
        const int64_t i = order[q];
        const int64_t cx = cell[i] % ncx, cy = cell[i] / ncx;
        for (int64_t ny = cy - 1; ny <= cy + 1; ny++) {
            if (ny < 0 || ny >= ncy) continue;
            for (int64_t nx = cx - 1; nx <= cx + 1; nx++) {
                if (nx < 0 || nx >= ncx) continue;
                const int64_t c = ny * ncx + nx;
                for (int64_t k = cstart[c]; k < cstart[c + 1]; k++) {
                    const int64_t j = order[k];
                    if (j == i) continue;
                    const int64_t a = i < j ? i : j, b = i < j ? j : i;
                    const double dx = X[a] - X[b];
                    const double dy = Y[a] - Y[b];
                    const double ed = sqrt(dx * dx + dy * dy);
                    if (ed <= rn) {
                        if (m == cap) {
                            cap *= 2;
                            t = (vo_trip *)realloc(t, sizeof(vo_trip) * (size_t)cap);
                        }
                        t[m].src = i;
                        t[m].dst = j;
                        t[m].w = ed;
                        m++;
                    }
                }
            }
        }
    }
    int rc = csr_from_triples(n, t, m, out);
    free(t); free(X); free(Y); free(cell); free(cstart); free(order);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* open-addressing set of unordered pairs (generators)                       */

typedef struct { uint64_t *keys; uint64_t mask; } vo_set;

static void set_init(vo_set *s, int64_t expect)
{
    uint64_t cap = 16;
    while (cap < (uint64_t)(2 * expect + 16)) cap <<= 1;
    s->keys = (uint64_t *)malloc(sizeof(uint64_t) * cap);
    memset(s->keys, 0xff, sizeof(uint64_t) * cap);
    s->mask = cap - 1;
}

/* returns 1 if inserted, 0 if present */
static int set_insert(vo_set *s, uint64_t key)
{
    uint64_t h = sm64(key) & s->mask;
    for (;;) {
        if (s->keys[h] == key) return 0;
        if (s->keys[h] == ~0ULL) { s->keys[h] = key; return 1; }
        h = (h + 1) & s->mask;
    }
}

static void set_free(vo_set *s) { free(s->keys); }

static uint64_t pair_key(int64_t i, int64_t j, int64_t n)
{
    int64_t a = i < j ? i : j, b = i < j ? j : i;
    return (uint64_t)a * (uint64_t)n + (uint64_t)b;
}

/* Seeded extra random edges: the count follows distgraph.cpp:703-706
 * (percent of the undirected edges); endpoints and U(0,1) weights come from
 * the counter-based generator (streams 1, 2, 3), self-pairs and pairs that
 * are already edges (either direction, or an earlier candidate) are skipped.
 * The reference's own extra edges are time-seeded (distgraph.cpp:755) and so
 * cannot be reproduced; this is the seeded variant the workload names. */
int64_t vo_add_random_edges(const vo_graph *in, double percent, uint64_t seed, vo_graph *out)
{
    const int64_t n = in->nv, m0 = in->ne / 2;
    const int64_t nrande = ((int64_t)(percent * (double)m0)) / 100;
    /* pairs already in the graph (either direction) are found by binary
     * searches of the two rows, which are sorted by tail; the set holds only
     * the candidates accepted so far */
    vo_set s;
    set_init(&s, nrande);
    int64_t m = in->ne;
    vo_trip *t = (vo_trip *)malloc(sizeof(vo_trip) * (size_t)(in->ne + 2 * nrande + 1));
    for (int64_t i = 0; i < n; i++)
        for (int64_t e = in->rowptr[i]; e < in->rowptr[i + 1]; e++) {
            t[e].src = i; t[e].dst = in->tail[e]; t[e].w = in->weight[e];
        }
    int64_t added = 0;
    for (int64_t k = 0; k < nrande; k++) {
        const int64_t i = (int64_t)uint_below(vo_mix(seed, 1, (uint64_t)k), (uint64_t)n);
        const int64_t j = (int64_t)uint_below(vo_mix(seed, 2, (uint64_t)k), (uint64_t)n);
        if (i == j) continue;
        if (csr_has(in, i, j) || csr_has(in, j, i)) continue;
        if (!set_insert(&s, pair_key(i, j, n))) continue;
        const double w = unit_double(vo_mix(seed, 3, (uint64_t)k));
        t[m].src = i; t[m].dst = j; t[m].w = w; m++;
        t[m].src = j; t[m].dst = i; t[m].w = w; m++;
        added++;
    }
    set_free(&s);
    int rc = csr_from_triples(n, t, m, out);
    free(t);
    return rc ? -1 : added;
}

/* Barabasi-Albert, own design: the Batagelj-Brandes edge list where edge e
 * (source e/m) copies the endpoint at a uniformly drawn earlier position, with
 * each draw a hash of the position (so every edge resolves independently, as in
 * Sanders & Schulz, "Scalable generation of scale-free graphs", 2016). Self
 * loops and repeated pairs are dropped; weights are 1. */
static int64_t ba_target(int64_t e, int64_t m, uint64_t seed)
{
    uint64_t pos = 2 * (uint64_t)e + 1;
    for (;;) {
        uint64_t r = uint_below(vo_mix(seed, 11, pos), pos);
        if ((r & 1) == 0) return (int64_t)((r / 2) / (uint64_t)m);
        pos = r;
    }
}

int vo_ba(int64_t n, int64_t m, uint64_t seed, vo_graph *out)
{
    const int64_t ecount = n * m;
    vo_set s;
    set_init(&s, ecount);
    vo_trip *t = (vo_trip *)malloc(sizeof(vo_trip) * (size_t)(2 * ecount + 1));
    int64_t k = 0;
    for (int64_t e = 0; e < ecount; e++) {
        const int64_t src = e / m, dst = ba_target(e, m, seed);
        if (src == dst) continue;
        if (!set_insert(&s, pair_key(src, dst, n))) continue;
        t[k].src = src; t[k].dst = dst; t[k].w = 1.0; k++;
        t[k].src = dst; t[k].dst = src; t[k].w = 1.0; k++;
    }
    set_free(&s);
    int rc = csr_from_triples(n, t, k, out);
    free(t);
    return rc;
}

/* Erdos-Renyi G(n, M), own design: M = round(avg_degree * n / 2) candidate
 * pairs from streams 21/22, self pairs and repeats dropped, weights 1. */
int vo_er(int64_t n, double avg_degree, uint64_t seed, vo_graph *out)
{
    const int64_t M = (int64_t)llround(avg_degree * (double)n / 2.0);
    vo_set s;
    set_init(&s, M);
    vo_trip *t = (vo_trip *)malloc(sizeof(vo_trip) * (size_t)(2 * M + 1));
    int64_t k = 0;
    for (int64_t c = 0; c < M; c++) {
        const int64_t i = (int64_t)uint_below(vo_mix(seed, 21, (uint64_t)c), (uint64_t)n);
        const int64_t j = (int64_t)uint_below(vo_mix(seed, 22, (uint64_t)c), (uint64_t)n);
        if (i == j) continue;
        if (!set_insert(&s, pair_key(i, j, n))) continue;
        t[k].src = i; t[k].dst = j; t[k].w = 1.0; k++;
        t[k].src = j; t[k].dst = i; t[k].w = 1.0; k++;
    }
    set_free(&s);
    int rc = csr_from_triples(n, t, k, out);
    free(t);
    return rc;
}

void vo_reweight(vo_graph *g, int mode, uint64_t seed)
{
    for (int64_t i = 0; i < g->nv; i++)
        for (int64_t e = g->rowptr[i]; e < g->rowptr[i + 1]; e++) {
            if (mode == 1) g->weight[e] = 1.0;
            else if (mode == 2)
                g->weight[e] = unit_double(vo_mix(seed, 31, pair_key(i, g->tail[e], g->nv)));
        }
}

/* ------------------------------------------------------------------------ */
/* Louvain phase (louvain.cpp)                                               */

/* distSumVertexDegree (louvain.cpp:2161-2186) and
 * distCalcConstantForSecondTerm (louvain.cpp:2188-2218): returns 1/(2m). */
double vo_vertex_degree(const vo_graph *g, double *vdeg)
{
    double total = 0;
    for (int64_t i = 0; i < g->nv; i++) {
        double tw = 0.0;
        for (int64_t k = g->rowptr[i]; k < g->rowptr[i + 1]; k++) tw += g->weight[k];
        vdeg[i] = tw;
    }
    for (int64_t i = 0; i < g->nv; i++) total += vdeg[i];
    return 1.0 / (double)total;
}

typedef struct {
    int64_t nv;
    const vo_graph *g;
    int64_t *past, *curr, *target;
    double *vdeg, *cw, *frozen_cw;
    int64_t *csize, *usize;
    double *cdeg, *udeg;
    /* per-vertex map scratch (ClusterLocalMap + counter, louvain.cpp:2419-2466) */
    int64_t *slot_of; /* community -> slot, -1 when absent */
    int64_t *slot_comm;
    double *counter;
    double constant;
} vo_state;

/* distGetMaxIndex (louvain.cpp:2220-2279) */
static int64_t get_max_index(vo_state *s, int64_t nslots, double selfLoop, double vDegree,
                             int64_t currSize, double currDegree, int64_t currComm)
{
    int64_t maxIndex = currComm;
    double curGain = 0.0, maxGain = 0.0;
    const double eix = s->counter[0] - selfLoop;
    const double ax = currDegree - vDegree;
    int64_t maxSize = currSize;
    for (int64_t k = 0; k < nslots; k++) {
        const int64_t c = s->slot_comm[k];
        if (c == currComm) continue;
        const double ay = s->cdeg[c];
        const int64_t size = s->csize[c];
        const double eiy = s->counter[k];
        curGain = 2.0 * (eiy - eix) - 2.0 * vDegree * (ay - ax) * s->constant;
        if ((curGain > maxGain) || ((curGain == maxGain) && (curGain != 0.0) && (c < maxIndex))) {
            maxGain = curGain;
            maxIndex = c;
            maxSize = size;
        }
    }
    if ((maxSize == 1) && (currSize == 1) && (maxIndex > currComm)) maxIndex = currComm;
    return maxIndex;
}

/* distExecuteLouvainIteration (louvain.cpp:2281-2417) with
 * distBuildLocalMapCounter (louvain.cpp:2419-2466), one rank. */
static void execute_vertex(vo_state *s, int64_t i)
{
    const vo_graph *g = s->g;
    const int64_t cc = s->curr[i];
    const double ccDegree = s->cdeg[cc];
    const int64_t ccSize = s->csize[cc];
    const int64_t e0 = g->rowptr[i], e1 = g->rowptr[i + 1];
    int64_t localTarget;
    if (e0 != e1) {
        int64_t nslots = 1;
        double selfLoop = 0.0;
        s->slot_comm[0] = cc;
        s->counter[0] = 0.0;
        s->slot_of[cc] = 0;
        for (int64_t j = e0; j < e1; j++) {
            const int64_t tail = g->tail[j];
            const double weight = g->weight[j];
            if (tail == i) selfLoop += weight;
            const int64_t tcomm = s->curr[tail];
            const int64_t sl = s->slot_of[tcomm];
            if (sl >= 0)
                s->counter[sl] += weight;
            else {
                s->slot_of[tcomm] = nslots;
                s->slot_comm[nslots] = tcomm;
                s->counter[nslots] = weight;
                nslots++;
            }
        }
        s->cw[i] += s->counter[0];
        localTarget = get_max_index(s, nslots, selfLoop, s->vdeg[i], ccSize, ccDegree, cc);
        for (int64_t k = 0; k < nslots; k++) s->slot_of[s->slot_comm[k]] = -1;
    } else
        localTarget = cc;
    if (localTarget != cc && localTarget != -1) {
        s->udeg[localTarget] += s->vdeg[i];
        s->usize[localTarget]++;
        s->udeg[cc] -= s->vdeg[i];
        s->usize[cc]--;
    }
    s->target[i] = localTarget;
}

/* distUpdateLocalCinfo (louvain.cpp:2534-2547) followed by zeroing the update */
static void apply_updates(vo_state *s)
{
    for (int64_t i = 0; i < s->nv; i++) {
        s->csize[i] += s->usize[i];
        s->cdeg[i] += s->udeg[i];
        s->usize[i] = 0;
        s->udeg[i] = 0;
    }
}

/* distComputeModularity with ABS_MOD_PER_ITER (louvain.cpp:2468-2532) */
static double modularity(vo_state *s)
{
    double le_xx = 0.0, la2_x = 0.0;
    for (int64_t i = 0; i < s->nv; i++) {
        le_xx += s->cw[i];
        la2_x += s->cdeg[i] * s->cdeg[i];
    }
    return fabs((le_xx * s->constant) - (la2_x * s->constant * s->constant));
}

int vo_louvain_phase(const vo_graph *g, const vo_phase_params *p, const int64_t *colors,
                     int64_t *cvect_out, double *mod_out, int *iters_out)
{
    const int64_t nv = g->nv;
    int ordering = p->ordering, et = p->et_type;
    const int64_t numColor = p->num_color;
    /* "if no colors, then fall back to original distLouvain" (louvain.cpp:600-605):
     * the fallback is the plain variant, without early termination */
    if (ordering != 0 && numColor == 1) { ordering = 0; et = 0; }
    vo_state s;
    memset(&s, 0, sizeof(s));
    s.nv = nv;
    s.g = g;
    const size_t n1 = (size_t)(nv > 0 ? nv : 1);
    s.past = (int64_t *)malloc(n1 * sizeof(int64_t));
    s.curr = (int64_t *)malloc(n1 * sizeof(int64_t));
    s.target = (int64_t *)calloc(n1, sizeof(int64_t));
    s.vdeg = (double *)malloc(n1 * sizeof(double));
    s.cw = (double *)calloc(n1, sizeof(double));
    s.frozen_cw = (double *)calloc(n1, sizeof(double));
    s.csize = (int64_t *)malloc(n1 * sizeof(int64_t));
    s.usize = (int64_t *)calloc(n1, sizeof(int64_t));
    s.cdeg = (double *)malloc(n1 * sizeof(double));
    s.udeg = (double *)calloc(n1, sizeof(double));
    s.slot_of = (int64_t *)malloc(n1 * sizeof(int64_t));
    s.slot_comm = (int64_t *)malloc(n1 * sizeof(int64_t));
    s.counter = (double *)malloc(n1 * sizeof(double));
    unsigned char *active = (unsigned char *)malloc(n1);
    double *p_curr = (double *)calloc(n1, sizeof(double)); /* value-initialised (louvain.cpp:244-249) */
    double *p_prev = (double *)malloc(n1 * sizeof(double));
    for (int64_t i = 0; i < nv; i++) {
        s.slot_of[i] = -1;
        active[i] = 1;
        p_prev[i] = 1.0;
    }

    /* distInitLouvain (louvain.cpp:2138-2159) */
    s.constant = vo_vertex_degree(g, s.vdeg);
    for (int64_t i = 0; i < nv; i++) {
        s.cdeg[i] = s.vdeg[i];
        s.csize[i] = 1;
        s.past[i] = i;
        s.curr[i] = i;
    }

    /* color CSR (louvain.cpp:646-677): uncolored vertices go to the last color;
     * with one thread the order inside a color is increasing vertex id */
    int64_t *colorPtr = NULL, *colorIndex = NULL;
    if (ordering != 0) {
        colorPtr = (int64_t *)calloc((size_t)numColor + 1, sizeof(int64_t));
        colorIndex = (int64_t *)malloc(n1 * sizeof(int64_t));
        int64_t *added = (int64_t *)calloc((size_t)numColor, sizeof(int64_t));
        for (int64_t i = 0; i < nv; i++) {
            const int64_t c = colors[i] < 0 ? numColor - 1 : colors[i];
            colorPtr[c + 1]++;
        }
        for (int64_t c = 0; c < numColor; c++) colorPtr[c + 1] += colorPtr[c];
        for (int64_t i = 0; i < nv; i++) {
            const int64_t c = colors[i] < 0 ? numColor - 1 : colors[i];
            colorIndex[colorPtr[c] + added[c]++] = i;
        }
        free(added);
    }

    double prevMod = p->lower, currMod = -1.0;
    const double lower = p->lower;
    int numIters = 0;
    for (;;) {
        numIters++;
        long vc_count = 0;
        for (int64_t i = 0; i < nv; i++) s.cw[i] = 0;
        if (ordering == 0) {
            for (int64_t i = 0; i < nv; i++) {
                if (et && !active[i]) {
                    s.cw[i] = s.frozen_cw[i];
                    vc_count++;
                    continue;
                }
                execute_vertex(&s, i);
                if (et) s.frozen_cw[i] = s.cw[i];
            }
            apply_updates(&s);
        } else {
            for (int64_t ci = 0; ci < numColor; ci++) {
                for (int64_t K = colorPtr[ci]; K < colorPtr[ci + 1]; K++) {
                    const int64_t i = colorIndex[K];
                    if (et && !active[i]) {
                        s.cw[i] = s.frozen_cw[i];
                        vc_count++;
                        continue;
                    }
                    execute_vertex(&s, i);
                    if (et) s.frozen_cw[i] = s.cw[i];
                }
                /* coloring applies the community updates after every color
                 * (louvain.cpp:724-735); vertex ordering after all colors
                 * (louvain.cpp:1405-1417) */
                if (ordering == 1) apply_updates(&s);
            }
            if (ordering == 2) apply_updates(&s);
        }
        if (et == 3 || et == 4) { /* ETLocalOrRemote == false (louvain.cpp:112-121) */
            if (vc_count >= VO_ET_CUTOFF) {
                currMod = -1;
                break;
            }
        }
        currMod = modularity(&s);
        if ((currMod - prevMod) < p->threshold) break;
        prevMod = currMod;
        if (prevMod < lower) prevMod = lower;

        if (et == 0) {
            int64_t *tmp = s.past; /* louvain.cpp:565-570 */
            s.past = s.curr;
            s.curr = s.target;
            s.target = tmp;
        } else if (et == 1 || et == 3) { /* louvain.cpp:172-184 */
            for (int64_t i = 0; i < nv; i++) {
                if (numIters > 2 && ((int64_t)(s.target[i] == s.curr[i]) == s.past[i]))
                    active[i] = 0;
                else {
                    int64_t tmp = s.past[i];
                    s.past[i] = s.curr[i];
                    s.curr[i] = s.target[i];
                    s.target[i] = tmp;
                }
            }
        } else { /* et 2/4: louvain.cpp:381-400 */
            const double one_minus_delta = (1.0 - p->et_delta);
            for (int64_t i = 0; i < nv; i++) {
                if (!active[i]) continue;
                if (numIters > 2 && (s.curr[i] == s.past[i])) {
                    p_curr[i] = p_prev[i] * one_minus_delta;
                    if (p_curr[i] <= VO_P_CUTOFF) active[i] = 0;
                }
                if (active[i]) {
                    int64_t tmp = s.past[i];
                    s.past[i] = s.curr[i];
                    s.curr[i] = s.target[i];
                    s.target[i] = tmp;
                }
            }
            double *t = p_curr;
            p_curr = p_prev;
            p_prev = t;
        }
    }
    memcpy(cvect_out, s.past, sizeof(int64_t) * (size_t)nv);
    *mod_out = prevMod;
    *iters_out = numIters;

    free(s.past); free(s.curr); free(s.target); free(s.vdeg); free(s.cw); free(s.frozen_cw);
    free(s.csize); free(s.usize); free(s.cdeg); free(s.udeg); free(s.slot_of); free(s.slot_comm);
    free(s.counter); free(active); free(p_curr); free(p_prev); free(colorPtr); free(colorIndex);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* coloring (coloring.cpp)                                                   */

/* coloring.cpp:120-131 */
uint32_t vo_color_hash(uint32_t a, uint32_t seed)
{
    a ^= seed;
    a = (a + 0x7ed55d16) + (a << 12);
    a = (a ^ 0xc761c23c) + (a >> 19);
    a = (a + 0x165667b1) + (a << 5);
    a = (a ^ 0xd3a2646c) + (a << 9);
    a = (a + 0xfd7046c5) + (a << 3);
    a = (a ^ 0xb55a4f09) + (a >> 16);
    return a;
}

/* distColoringIteration for one rank (coloring.cpp:133-247) */
static void color_iteration(const vo_graph *g, int64_t *color, int64_t nHash, int64_t nextColor,
                            uint32_t seed)
{
    uint32_t *vHash = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)nHash);
    for (int64_t v = 0; v < g->nv; v++) {
        int64_t possible_colors = 2 * nHash;
        if (color[v] != -1) continue;
        int64_t not_min = 0, not_max = 0;
        int can_color = 1;
        for (int64_t t = 0; t < nHash; t++) vHash[t] = vo_color_hash((uint32_t)v, (uint32_t)(seed + 1043 * t));
        for (int64_t k = g->rowptr[v]; k < g->rowptr[v + 1]; k++) {
            const int64_t tail = g->tail[k];
            if (v == tail) continue;
            if (color[tail] != -1 && color[tail] < nextColor) continue;
            for (int64_t t = 0; t < nHash; t++) {
                const uint32_t jHash = vo_color_hash((uint32_t)tail, (uint32_t)(seed + 1043 * t));
                if (vHash[t] <= jHash && !(not_max & (1LL << t))) {
                    not_max |= (1LL << t);
                    possible_colors--;
                }
                if (vHash[t] >= jHash && !(not_min & (1LL << t))) {
                    not_min |= (1LL << t);
                    possible_colors--;
                }
            }
            if (possible_colors == 0) {
                can_color = 0;
                break;
            }
        }
        if (can_color) {
            const int64_t col_id = v % possible_colors;
            int64_t this_col_id = 0;
            for (int64_t t = 0; t < nHash; t++) {
                if (!(not_min & (1LL << t)) && col_id == this_col_id) {
                    color[v] = 2 * t + nextColor;
                    break;
                }
                this_col_id += !(not_min & (1LL << t));
                if (!(not_max & (1LL << t)) && col_id == this_col_id) {
                    color[v] = 2 * t + 1 + nextColor;
                    break;
                }
                this_col_id += !(not_max & (1LL << t));
            }
        }
    }
    free(vHash);
}

/* distColoringMultiHashMinMax for one rank (coloring.cpp:52-118) */
int64_t vo_color(const vo_graph *g, int64_t nHash, int target_percent, int single_iteration,
                 int64_t *color)
{
    uint32_t seed = 1012;
    int64_t nextColor = 0, lastCount = 0, currentCount = 0;
    const int64_t tnv = g->nv;
    const int64_t targetCount = (tnv * target_percent) / 100;
    int finished = 0;
    for (int64_t i = 0; i < tnv; i++) color[i] = -1;
    while (!finished) {
        color_iteration(g, color, nHash, nextColor, seed);
        int64_t unassigned = 0;
        for (int64_t i = 0; i < tnv; i++) unassigned += (color[i] == -1);
        currentCount = tnv - unassigned;
        finished = single_iteration || currentCount >= targetCount || lastCount == currentCount;
        nextColor += nHash * 2;
        seed = vo_color_hash(seed, 0);
        lastCount = currentCount;
    }
    return nextColor;
}

/* ------------------------------------------------------------------------ */
/* rebuild (rebuild.cpp)                                                     */

typedef struct { int64_t key, pos; double w; } vo_kv;

static int kv_cmp(const void *a, const void *b)
{
    const vo_kv *x = (const vo_kv *)a, *y = (const vo_kv *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return (x->pos < y->pos) ? -1 : (x->pos > y->pos);
}

/* distbuildNextLevelGraph for one rank: distReNumber numbers communities by
 * first appearance in vertex order (rebuild.cpp:122-135); fill_newEdgesMap
 * sums weights per (c1, c2) in (vertex, edge) order (rebuild.cpp:294-329);
 * send_newEdges writes rows sorted by c2, the std::map order (rebuild.cpp:380,
 * 462-477, rebuild.hpp:89). Self loops stay. */
int vo_rebuild(const vo_graph *g, const int64_t *cvect, vo_graph *out)
{
    const int64_t nv = g->nv;
    int64_t *lookup = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nv > 0 ? nv : 1));
    for (int64_t i = 0; i < nv; i++) lookup[i] = -1;
    int64_t lnc = 0;
    for (int64_t i = 0; i < nv; i++)
        if (lookup[cvect[i]] < 0) lookup[cvect[i]] = lnc++;
    /* group the CSR entries by c1, keeping (vertex, edge) order */
    int64_t *start = (int64_t *)calloc((size_t)lnc + 1, sizeof(int64_t));
    for (int64_t i = 0; i < nv; i++) start[lookup[cvect[i]] + 1] += g->rowptr[i + 1] - g->rowptr[i];
    for (int64_t c = 0; c < lnc; c++) start[c + 1] += start[c];
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)(lnc > 0 ? lnc : 1));
    memcpy(fill, start, sizeof(int64_t) * (size_t)lnc);
    vo_kv *kv = (vo_kv *)malloc(sizeof(vo_kv) * (size_t)(g->ne > 0 ? g->ne : 1));
    for (int64_t i = 0; i < nv; i++) {
        const int64_t c1 = lookup[cvect[i]];
        for (int64_t e = g->rowptr[i]; e < g->rowptr[i + 1]; e++) {
            vo_kv *x = &kv[fill[c1]];
            x->key = lookup[cvect[g->tail[e]]];
            x->pos = fill[c1];
            x->w = g->weight[e];
            fill[c1]++;
        }
    }
    /* per row: stable sort by c2, then fold each run in order */
    int64_t m = 0;
    for (int64_t c = 0; c < lnc; c++) {
        const int64_t b = start[c], e = start[c + 1];
        qsort(kv + b, (size_t)(e - b), sizeof(vo_kv), kv_cmp);
        for (int64_t k = b; k < e;) {
            int64_t r = k + 1;
            while (r < e && kv[r].key == kv[k].key) r++;
            m++;
            k = r;
        }
    }
    vo_graph_alloc(out, lnc, m);
    int64_t o = 0;
    for (int64_t c = 0; c < lnc; c++) {
        const int64_t b = start[c], e = start[c + 1];
        out->rowptr[c] = o;
        for (int64_t k = b; k < e;) {
            double w = kv[k].w;
            int64_t r = k + 1;
            while (r < e && kv[r].key == kv[k].key) { w += kv[r].w; r++; }
            out->tail[o] = kv[k].key;
            out->weight[o] = w;
            o++;
            k = r;
        }
    }
    out->rowptr[lnc] = o;
    free(lookup); free(start); free(fill); free(kv);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* phase loop (main.cpp:242-513)                                             */

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int vo_run(const vo_graph *g0, const vo_run_params *rp, int max_levels, int64_t *level_nv,
           int64_t *level_ne, int *level_iters, double *level_mod, int64_t *level_colors,
           double *seconds_out)
{
    vo_graph cur;
    vo_graph_alloc(&cur, g0->nv, g0->ne);
    memcpy(cur.rowptr, g0->rowptr, sizeof(int64_t) * (size_t)(g0->nv + 1));
    memcpy(cur.tail, g0->tail, sizeof(int64_t) * (size_t)g0->ne);
    memcpy(cur.weight, g0->weight, sizeof(double) * (size_t)g0->ne);
    double currMod = -1.0, prevMod = -1.0, threshold;
    int phase = 0, short_phase = 0, tot_iters = 0, nrec = 0;
    double t0 = now_s();
    for (;;) {
        if (rp->threshold_scaling && !rp->one_phase) {
            if (short_phase > 12) short_phase = 0;
            if (short_phase <= 2) threshold = 1.0E-3;
            else if (short_phase <= 6) threshold = 1.0E-4;
            else if (short_phase <= 9) threshold = 1.0E-5;
            else threshold = rp->threshold;
        } else
            threshold = rp->threshold;
        int64_t *cvect = (int64_t *)malloc(sizeof(int64_t) * (size_t)(cur.nv > 0 ? cur.nv : 1));
        vo_phase_params pp;
        memset(&pp, 0, sizeof(pp));
        pp.lower = currMod;
        pp.threshold = threshold;
        pp.et_type = rp->et_type;
        pp.et_delta = rp->et_delta;
        int64_t numColors = 0;
        int64_t *colors = NULL;
        if ((rp->coloring || rp->vertex_order) && phase == 0) {
            colors = (int64_t *)malloc(sizeof(int64_t) * (size_t)(cur.nv > 0 ? cur.nv : 1));
            numColors = vo_color(&cur, rp->max_colors / 2, VO_MAX_COVG, rp->single_color_iter, colors);
            pp.ordering = rp->coloring ? 1 : 2;
            pp.num_color = numColors + 1;
        }
        int iters = 0;
        vo_louvain_phase(&cur, &pp, colors, cvect, &currMod, &iters);
        free(colors);
        tot_iters += iters;
        if (nrec < max_levels) {
            if (level_nv) level_nv[nrec] = cur.nv;
            if (level_ne) level_ne[nrec] = cur.ne;
            if (level_iters) level_iters[nrec] = iters;
            if (level_mod) level_mod[nrec] = currMod;
            if (level_colors) level_colors[nrec] = numColors;
        }
        nrec++;
        if ((currMod - prevMod) > threshold) {
            if (!rp->one_phase) {
                vo_graph next;
                vo_rebuild(&cur, cvect, &next);
                vo_graph_free(&cur);
                cur = next;
            }
        } else {
            if (rp->threshold_scaling && !rp->one_phase && phase < 10) {
                memset(&pp, 0, sizeof(pp));
                pp.lower = currMod;
                pp.threshold = 1.0E-6;
                vo_louvain_phase(&cur, &pp, NULL, cvect, &currMod, &iters);
                if (nrec < max_levels) {
                    if (level_nv) level_nv[nrec] = cur.nv;
                    if (level_ne) level_ne[nrec] = cur.ne;
                    if (level_iters) level_iters[nrec] = iters;
                    if (level_mod) level_mod[nrec] = currMod;
                    if (level_colors) level_colors[nrec] = 0;
                }
                nrec++;
            }
            free(cvect);
            break;
        }
        free(cvect);
        prevMod = currMod;
        currMod = -1.0;
        phase++;
        if (rp->one_phase) break;
        if (rp->threshold_scaling && !rp->one_phase) short_phase++;
        if (phase == VO_PHASE_CAP || tot_iters > 10000) break;
    }
    if (seconds_out) *seconds_out = now_s() - t0;
    vo_graph_free(&cur);
    return nrec;
}

/* ------------------------------------------------------------------------------
 * compare_communities (compare.cpp:58-285) with its per-community pair loops, and
 * compute_gini_coeff (compare.cpp:287-318).
 */
static int vo_cmp_i64(const void *a, const void *b) {
    const int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return x < y ? -1 : x > y;
}

static double vo_gini(int64_t *size, int numColors) {
    qsort(size, (size_t)numColors, sizeof(int64_t), vo_cmp_i64);
    double numFunc = 0.0, denFunc = 0.0;
    for (int64_t i = 0; i < numColors; i++) {
        numFunc = numFunc + (double)((i + 1) * size[i]);
        denFunc = denFunc + (double)size[i];
    }
    return ((2 * numFunc) / (numColors * denFunc)) - ((double)(numColors + 1) / (double)numColors);
}

/* community CSR of labels c: ptr[nc + 1], idx[n] (compare.cpp:97-141), sizes[nc] */
static int vo_comm_csr(int64_t n, const int64_t *c, int64_t nc, int64_t **ptr, int64_t **idx,
                       int64_t **sizes) {
    int64_t *p = calloc((size_t)nc + 1, sizeof(int64_t));
    int64_t *x = malloc(sizeof(int64_t) * (size_t)n);
    int64_t *s = malloc(sizeof(int64_t) * (size_t)nc);
    int64_t *fill = calloc((size_t)nc, sizeof(int64_t));
    if (!p || !x || !s || !fill) {
        free(p); free(x); free(s); free(fill);
        return -1;
    }
    for (int64_t i = 0; i < n; i++) p[c[i] + 1]++;
    for (int64_t k = 0; k < nc; k++) s[k] = p[k + 1];
    for (int64_t k = 0; k < nc; k++) p[k + 1] += p[k];
    for (int64_t i = 0; i < n; i++) x[p[c[i]] + fill[c[i]]++] = i;
    free(fill);
    *ptr = p;
    *idx = x;
    *sizes = s;
    return 0;
}

int vo_compare(int64_t n, const int64_t *c1, const int64_t *c2, vo_compare_stats *out) {
    if (n <= 0) return -1;
    int64_t nc1 = -1, nc2 = -1;
    for (int64_t i = 0; i < n; i++) {
        if (c1[i] < 0 || c2[i] < 0) return -1;
        if (c1[i] > nc1) nc1 = c1[i];
        if (c2[i] > nc2) nc2 = c2[i];
    }
    nc1++;
    nc2++;
    int64_t *p1, *x1, *s1, *p2, *x2, *s2;
    if (vo_comm_csr(n, c1, nc1, &p1, &x1, &s1)) return -1;
    if (vo_comm_csr(n, c2, nc2, &p2, &x2, &s2)) {
        free(p1); free(x1); free(s1);
        return -1;
    }
    int64_t ss = 0, sd = 0, ds = 0, agree = 0;
    for (int64_t ci = 0; ci < nc1; ci++)
        for (int64_t i = p1[ci]; i < p1[ci + 1]; i++)
            for (int64_t j = i + 1; j < p1[ci + 1]; j++) {
                if (c2[x1[i]] == c2[x1[j]]) ss++;
                else sd++;
            }
    for (int64_t ci = 0; ci < nc2; ci++)
        for (int64_t i = p2[ci]; i < p2[ci + 1]; i++)
            for (int64_t j = i + 1; j < p2[ci + 1]; j++) {
                if (c1[x2[i]] == c1[x2[j]]) agree++;
                else ds++;
            }
    out->n = n;
    out->nc1 = nc1;
    out->nc2 = nc2;
    out->same_same = ss;
    out->same_diff = sd;
    out->diff_same = ds;
    out->precision = (double)ss / (double)(ss + ds);
    out->recall = (double)ss / (double)(ss + sd);
    out->fscore = 2.0 * ((out->precision * out->recall) / (out->precision + out->recall));
    out->gini1 = vo_gini(s1, (int)nc1);
    out->gini2 = vo_gini(s2, (int)nc2);
    free(p1); free(x1); free(s1); free(p2); free(x2); free(s2);
    return agree == ss ? 0 : -2;
}
