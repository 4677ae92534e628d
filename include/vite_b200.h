/*
 * vite_b200.h -- C ABI of the B200-native Louvain library (libvite_b200.so).
 *
 * The whole graph lives on one GPU as one rank: Vite's MPI ghost exchange and
 * remote community-info messages become reads of device arrays, so the ABI has
 * no communicator. Ids cross the boundary as int64 and weights as double, the
 * reference's default 64-bit build (edge.hpp:65-69); on the device ids are
 * int32 (every graph must have fewer than 2^31 vertices) and all arithmetic on
 * weights, degrees, gains and modularity stays FP64, evaluated in the
 * reference's order without fused multiply-adds.
 *
 * Every function returns a vg_status; VG_OK is 0. On failure vg_last_error()
 * names the cause. A context is bound to one device and one CUDA stream; calls
 * on one context must not overlap (one host thread per context).
 */
#ifndef VITE_B200_H
#define VITE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum vg_status {
    VG_OK = 0,
    VG_ERR_ARG = 1,      /* invalid argument (the reference asserts or MPI_Aborts, main.cpp:714-768) */
    VG_ERR_OOM = 2,      /* device memory or the context's memory budget is exhausted */
    VG_ERR_CUDA = 3,     /* a CUDA runtime call failed */
    VG_ERR_TIMEOUT = 4,  /* a bounded device-side wait ran out */
    VG_ERR_STATE = 5     /* call made in the wrong state (e.g. rebuild before any phase) */
} vg_status;

typedef struct vg_ctx vg_ctx;
typedef struct vg_graph vg_graph;

/* Vite's Edge for the default 64-bit build (edge.hpp:72-80): 16 bytes. */
typedef struct vg_edge {
    int64_t tail;
    double weight;
} vg_edge;

/* Arguments of one Louvain phase: the trailing arguments of the nine
 * distLouvainMethod* overloads (louvain.hpp:80-137), selected the way main.cpp
 * dispatches them (main.cpp:267-370). */
typedef struct vg_phase_params {
    double lower;       /* `lower`; main passes -1.0 */
    double threshold;   /* `thresh` */
    int32_t et_type;    /* 0 plain; 1..4 early termination as -t 1..4 */
    double et_delta;    /* `ETDelta` (-a), used by types 2 and 4 */
    int32_t ordering;   /* 0 distLouvainMethod, 1 distLouvainMethodWithColoring,
                           2 distLouvainMethodVertexOrder (both need vg_color or vg_set_colors) */
} vg_phase_params;

/* graphClustering's options that shape the phase loop (main.cpp:609-708). */
typedef struct vg_run_params {
    double threshold;          /* -h (default 1e-6, utils.hpp:71-73) */
    int32_t coloring;          /* -c */
    int32_t vertex_order;      /* -d */
    int32_t max_colors;        /* the k of -c/-d (default 8) */
    int32_t single_color_iter; /* the "single" flag of -c/-d */
    int32_t et_type;           /* -t (0 = off) */
    double et_delta;           /* -a */
    int32_t threshold_scaling; /* -i */
    int32_t one_phase;         /* -p */
    int32_t layout;            /* HBM layout of the level-0 graph: 0 as given, 1 locality order
                                  computed on the device (vg_graph_reorder mode 1), 2 locality
                                  order when the graph has at least 2^18 vertices and local
                                  structure (a sampled clustering coefficient of at least 0.1:
                                  geometric graphs yes, preferential-attachment and uniform
                                  random graphs no). Results are the same in every layout. */
} vg_run_params;

/* What graphClustering prints per level (main.cpp:465-474), measured on the device. */
typedef struct vg_level_stat {
    int64_t nv, ne;            /* graph the level ran on */
    int32_t iters;             /* iterations of the phase */
    double modularity;         /* value returned by the phase */
    int64_t num_colors;        /* colors returned by the coloring (0 if none) */
    double seconds_color;      /* device time of the coloring */
    double seconds_phase;      /* device time of the phase, coloring excluded */
    double seconds_sweep;      /* device time of the local-moving sweeps alone */
    double seconds_rebuild;    /* device time of the rebuild after the level (0 if none) */
    int64_t edges_swept;       /* sum over iterations of the edges the sweeps visited */
    double seconds_layout;     /* device time of the level-0 layout step (0 if none) */
} vg_level_stat;

/* --- context ---------------------------------------------------------------- */

/* Create a context on `device` with a device-memory budget in bytes (0 = no
 * budget beyond the device's capacity). Replaces MPI_Init/communicator set-up
 * (main.cpp:112-118). */
vg_status vg_ctx_create(int device, size_t mem_budget_bytes, vg_ctx **out);
vg_status vg_ctx_destroy(vg_ctx *ctx);
const char *vg_last_error(const vg_ctx *ctx);
/* Bytes the context currently holds on the device. */
size_t vg_ctx_bytes_in_use(const vg_ctx *ctx);
/* Kernel launches issued since the last reset (always counted) and, while
 * enabled, the sum of their device times in ms (events around each launch). */
vg_status vg_ctx_profile(vg_ctx *ctx, int32_t enable, double *kernel_ms_out,
                         int64_t *launches_out, int32_t reset);
/* Grow the context's device memory pool to at least `bytes` now (no reference
 * counterpart). Freed memory stays in the pool, so later phases and rebuilds of
 * up to this working set allocate without mapping new memory mid-run. Counted
 * against the budget only while held (it is released back to the pool at once). */
vg_status vg_ctx_reserve(vg_ctx *ctx, size_t bytes);
/* The CUDA stream (cudaStream_t) all of the context's work runs on, so callers
 * can time it with events or order their own work after it. */
vg_status vg_ctx_stream(vg_ctx *ctx, void **stream_out);

/* --- graphs ----------------------------------------------------------------- */

/* Copy a CSR in Vite's layout (Graph::edgeListIndexes / edgeList,
 * graph.hpp:77-106) to the device. Replaces loadDistGraphMPIIO's hand-off of
 * the local graph (distgraph.cpp:119-253) for one rank. */
vg_status vg_graph_upload(vg_ctx *ctx, int64_t nv, int64_t ne, const int64_t *rowptr,
                          const vg_edge *edges, vg_graph **out);
vg_status vg_graph_info(const vg_graph *g, int64_t *nv, int64_t *ne);
/* Copy the device CSR back in Vite's layout (writeGraph's input,
 * distgraph.cpp:986-1064). rowptr has nv+1 entries, edges ne. */
vg_status vg_graph_download(vg_ctx *ctx, const vg_graph *g, int64_t *rowptr, vg_edge *edges);
vg_status vg_graph_free(vg_ctx *ctx, vg_graph *g);

/* Vite's binary graph file ([nv][ne][rowptr x (nv+1)][Edge x ne], all little-endian
 * int64 / f64; read by loadDistGraphMPIIO, distgraph.cpp:119-253, written by writeGraph
 * and the converters, converters/convert.cpp:245-278) straight to and from a device
 * graph. The reader streams the file through pinned host buffers with the copies and
 * the conversion overlapping the reads, rebases the offsets to start at zero
 * (distgraph.cpp:244-247) and rejects a truncated file, offsets that decrease or do
 * not end at ne, and tails outside [0, nv) with VG_ERR_ARG. The writer writes the
 * graph in reference vertex order, as vg_graph_download returns it. */
vg_status vg_graph_read_vite(vg_ctx *ctx, const char *path, vg_graph **out);
vg_status vg_graph_write_vite(vg_ctx *ctx, const vg_graph *g, const char *path);

/* Text edge lists parsed on the device into a graph: fileConvert's input formats and
 * weight options (converters/convert.cpp:102-281, parseCommandLine :286-368), replacing
 * loadSimpleFile (converters/simple.cpp:61), loadSNAPFile (converters/snap.cpp:65) and
 * loadMatrixMarketFile (converters/matrix-market.cpp:65) followed by processGraphData
 * (utils.cpp:101-152). Rows list their tails in increasing order (equal pairs in file
 * order), duplicates kept. A malformed file is VG_ERR_ARG with the line named. */
typedef enum vg_text_format {
    VG_TEXT_SIMPLE = 1,        /* -s: "u v [w]" per line, '#'/'%' comment lines */
    VG_TEXT_SNAP = 2,          /* -n: "# Nodes: N Edges: M" header, ids renumbered */
    VG_TEXT_MATRIX_MARKET = 3  /* -m: coordinate, general or symmetric, 1-based */
} vg_text_format;
typedef enum vg_text_weights {
    VG_WEIGHTS_ABS = 0,        /* default: |w| (pattern files and SNAP: 1) */
    VG_WEIGHTS_ORIGINAL = 1,   /* -i: w as written */
    VG_WEIGHTS_ONE = 2,        /* -w: 1 */
    VG_WEIGHTS_RANDOM = 3      /* -r: the reference's genRandom stream (utils.cpp:93-99) */
} vg_text_weights;
typedef struct vg_text_params {
    int32_t format;            /* vg_text_format */
    int32_t weights;           /* vg_text_weights */
    int32_t one_based;         /* -z: ids start at 1 (VG_TEXT_SIMPLE only) */
} vg_text_params;
vg_status vg_graph_read_text(vg_ctx *ctx, const char *path, const vg_text_params *p,
                             vg_graph **out);

/* Store the graph in another vertex order on the device (no reference
 * counterpart: the reference keeps its input order). mode 1: locality order
 * (multi-source BFS clusters) so that a sweep's gathers stay in few cache
 * lines; mode 0: back to reference order. Ids at the boundary stay the
 * reference's in every layout and every result is unchanged; the communities
 * and colors attached to g are dropped. */
vg_status vg_graph_reorder(vg_ctx *ctx, vg_graph *g, int32_t mode);

/* distSumVertexDegree + distCalcConstantForSecondTerm (louvain.cpp:2161-2218):
 * weighted degree of every vertex (optional copy out) and 1/(2m). */
vg_status vg_vertex_degree(vg_ctx *ctx, vg_graph *g, double *vdeg_out, double *constant_out);

/* Allocation-free variant of vg_vertex_degree (no counterpart in the reference,
 * which allocates with std::vector). For callers that cannot allocate device memory
 * while they run -- a server that reserved its whole memory budget at start-up, a
 * framework whose allocator owns the device memory, code that must not stall or fail
 * on an allocation mid-run. The caller passes device pointers: rowptr int64[nv+1]
 * and weights f64[ne] of a CSR (weights may be NULL only when the CSR holds no
 * entries, else VG_ERR_ARG), and vdeg_out f64[nv] for the degrees; 1/(2m) is
 * written to *constant_out (host). The CSR must be valid: offsets non-decreasing and
 * every offset in [0, ne] of the weights array the caller passes. Unlike
 * vg_graph_upload, this function does not check the offsets (a check would need
 * memory of its own); offsets past the weights array make the kernel read out of
 * bounds. Runs on `stream` (a cudaStream_t, NULL = default stream) of the current
 * device and waits for that stream to finish before it returns. The scratch of the
 * reduction is a file-scope device array of 512 KiB held by every GPU that loads the
 * library: at most VG_NOALLOC_MAX_VERTICES vertices, larger graphs are rejected with
 * VG_ERR_ARG. All calls share that array, so calls that overlap on the GPU race. The
 * first call on a device looks the array's address up with that device current. The
 * address is kept for the life of the process, so do not call this function again on
 * a device after cudaDeviceReset. errbuf (may be
 * NULL) receives a message on failure. Allocates nothing: no cudaMalloc, no
 * cudaFree. */
#define VG_NOALLOC_MAX_VERTICES (2048LL * 65536LL)
vg_status vg_vertex_degree_noalloc(int64_t nv, const int64_t *d_rowptr, const double *d_weight,
                                   double *d_vdeg_out, double *constant_out, void *stream,
                                   char *errbuf, size_t errlen);

/* --- the Louvain path ----------------------------------------------------------- */

/* Launch tuning of the local-moving sweep, held per context. It has no counterpart
 * in the reference (its sweep is one loop per rank); it chooses which kernel
 * handles a vertex of degree d: d <= 16 one thread; d <= 32 one thread when t32 is
 * 1 (else the small warp table); d <= ws_max one warp with a 256-slot table;
 * d <= wt_max one warp with a 1024-slot table; d <= ct_max one CTA with an 8192-slot
 * table; above, the hub path (many CTAs per row). tile_grid is the number of CTAs
 * per SM of the degree <= 16 sweep in vertex order. Every class folds a vertex's
 * counters in CSR order except the two CTA-based ones, whose slices meet through
 * FP64 atomics: with unit or integral weights any setting gives the same bits, with
 * real weights results agree to the last few bits. */
typedef struct vg_tuning {
    int32_t t32;       /* 0 or 1 */
    int32_t ws_max;    /* 32..128 */
    int32_t wt_max;    /* ws_max..512 */
    int32_t ct_max;    /* wt_max..4096 */
    int32_t tile_grid; /* 1..1024 */
} vg_tuning;

/* The context's current tuning (the built-in defaults until set). */
vg_status vg_ctx_get_tuning(const vg_ctx *ctx, vg_tuning *out);
/* Set the tuning; VG_ERR_ARG when a field is outside its range above. */
vg_status vg_ctx_set_tuning(vg_ctx *ctx, const vg_tuning *t);

/* The autotuner (no counterpart in the reference). Starting from the context's
 * tuning, it varies one field at a time over a few candidate values and keeps a
 * change when it lowers the summed sweep time of the first `sweeps` iterations (1..8;
 * 0 means 2) of a plain phase on every graph given, each timed twice, the faster
 * taken. The graphs are left as they were (each trial runs on a shallow copy). The
 * best tuning is set on the context and returned with its summed sweep time and that
 * of the tuning it started from (milliseconds; either pointer may be NULL). */
vg_status vg_autotune(vg_ctx *ctx, vg_graph *const *graphs, int32_t n, int32_t sweeps,
                      vg_tuning *best_out, double *best_ms_out, double *start_ms_out);

/* One Louvain phase: distLouvainMethod / ...WithColoring / ...VertexOrder
 * (louvain.cpp:7-1938). Returns the phase's modularity (`prevMod` of the
 * reference), its iteration count and, if cvect_out is not NULL, the community
 * of every vertex (`cvect`). The communities also stay on the device for
 * vg_rebuild. */
vg_status vg_louvain_phase(vg_ctx *ctx, vg_graph *g, const vg_phase_params *p,
                           int64_t *cvect_out, double *mod_out, int32_t *iters_out);

/* distColoringMultiHashMinMax (coloring.cpp:52-118) for one rank: n_hash hash
 * functions, stop at target_percent coverage or after one round. Returns the
 * reference's return value (`nextColor`, main passes it +1 as numColor) and
 * optionally every vertex's color (-1 = uncolored). The colors stay on the
 * device for phases with ordering 1 or 2. */
vg_status vg_color(vg_ctx *ctx, vg_graph *g, int64_t n_hash, int32_t target_percent,
                   int32_t single_iteration, int64_t *colors_out, int64_t *num_colors_out);
/* Provide a coloring computed elsewhere (the ColorVector argument of the
 * ...WithColoring / ...VertexOrder overloads); num_colors is the reference's
 * numColor - 1. */
vg_status vg_set_colors(vg_ctx *ctx, vg_graph *g, const int64_t *colors, int64_t num_colors);

/* distbuildNextLevelGraph (rebuild.cpp:480-504) for one rank: replace g by the
 * next-level graph. cvect NULL uses the communities of the last phase on g. */
vg_status vg_rebuild(vg_ctx *ctx, vg_graph *g, const int64_t *cvect);

/* The phase loop of graphClustering (main.cpp:242-513) run on the device:
 * coloring at phase 0, phases, rebuilds, threshold cycling and the phase caps.
 * g is not modified. levels receives up to max_levels entries; comm_out (may
 * be NULL) receives the final community of every vertex of g, renumbered by
 * sorted id exactly like graphClustering's -o output (main.cpp:381-425). */
vg_status vg_louvain_run(vg_ctx *ctx, const vg_graph *g, const vg_run_params *p,
                         vg_level_stat *levels, int32_t max_levels, int32_t *nlevels_out,
                         int64_t *comm_out);

/* --- batched and served runs ---------------------------------------------------
 * No counterpart in the reference, which runs one graph per job: many
 * independent graphs run as one packed graph, each with the level loop of
 * vg_louvain_run (plain phase, threshold, one_phase, layout) and the same
 * results as a run of its own. One step = one round: admit queued graphs while
 * their estimated footprint fits the budget, run one phase for every graph in
 * the batch, retire the graphs whose level loop ended, rebuild the rest. */
typedef struct vg_batch vg_batch;

/* the batch frees the submitted graph once it has been packed */
#define VG_BATCH_TAKE 1
/* keep the composed community of every vertex (vg_batch_result comm_out) */
#define VG_BATCH_COMM 2

typedef struct vg_batch_stats {
    int64_t submitted, admitted, completed, rounds;
    int64_t running, queued;
    size_t running_bytes;          /* estimated footprint of the running graphs */
    double seconds_phase, seconds_rebuild;
} vg_batch_stats;

/* budget_bytes = 0: admit every queued graph at the next step */
vg_status vg_batch_create(vg_ctx *ctx, size_t budget_bytes, vg_batch **out);
vg_status vg_batch_destroy(vg_batch *b);
/* Queue a graph; it must stay valid until packed (the next step), or be handed
 * over with VG_BATCH_TAKE. Rejected when p asks for coloring, vertex ordering,
 * early termination or threshold cycling, or when the graph alone exceeds the
 * budget. */
vg_status vg_batch_submit(vg_batch *b, vg_graph *g, const vg_run_params *p, int32_t flags,
                          int64_t *job_out);
vg_status vg_batch_step(vg_batch *b, int32_t *running_out, int32_t *queued_out);
/* ids of the graphs finished since the last poll */
vg_status vg_batch_poll(vg_batch *b, int64_t *ids, int32_t max_ids, int32_t *n_out);
/* per-level statistics (the phase and rebuild times are the shared round's)
 * and, with VG_BATCH_COMM, the communities as vg_louvain_run's comm_out */
vg_status vg_batch_result(vg_batch *b, int64_t job, vg_level_stat *levels, int32_t max_levels,
                          int32_t *nlevels_out, int64_t *comm_out);
/* drop a finished graph's results */
vg_status vg_batch_forget(vg_batch *b, int64_t job);
vg_status vg_batch_get_stats(vg_batch *b, vg_batch_stats *out);

/* --- ground-truth comparison ------------------------------------------------- */

/* compare_communities + compute_gini_coeff (compare.cpp:58-318): c1 is the truth
 * (graphClustering -g), c2 the computed communities, both n labels in
 * [0, 2^31 - 1); the number of communities of each is its largest label + 1.
 * Pair counts over all vertex pairs, precision, recall, F-score and the Gini
 * coefficient of each vector's community sizes, as the reference prints them. */
typedef struct vg_compare_stats {
    int64_t n, nc1, nc2;
    int64_t same_same, same_diff, diff_same; /* true positives, false negatives, false positives */
    double precision, recall, fscore, gini1, gini2;
} vg_compare_stats;
vg_status vg_compare_communities(vg_ctx *ctx, int64_t n, const int64_t *c1, const int64_t *c2,
                                 vg_compare_stats *out);

/* --- generators --------------------------------------------------------------- */

/* generateInMemGraph for one rank (distgraph.cpp:391-407, 412-983): n points
 * from Vite's LCG (seed 1), edge when the distance is at most r(n), weight =
 * distance; bit-identical to the reference. extra_percent > 0 adds that
 * percent of extra edges with U(0,1) weights drawn from `seed` (the
 * reference's own extra edges are time-seeded, distgraph.cpp:755). */
vg_status vg_generate_rgg(vg_ctx *ctx, int64_t n, double extra_percent, uint64_t seed,
                          vg_graph **out);
/* Seeded Barabasi-Albert (m attachments per vertex) and Erdos-Renyi G(n, M)
 * graphs with unit weights, for the workloads the reference feeds through
 * NetworKit (generators/nkit-ba.cpp:66-116, nkit-er.cpp:67); own designs. */
vg_status vg_generate_ba(vg_ctx *ctx, int64_t n, int64_t m, uint64_t seed, vg_graph **out);
vg_status vg_generate_er(vg_ctx *ctx, int64_t n, double avg_degree, uint64_t seed,
                         vg_graph **out);
/* Re-weight every edge: mode 1 = 1.0 (SET_EDGE_WEIGHTS_TO_ONE,
 * distgraph.cpp:249-252), mode 2 = U(0,1) drawn per unordered pair from seed. */
vg_status vg_graph_reweight(vg_ctx *ctx, vg_graph *g, int32_t mode, uint64_t seed);

#ifdef __cplusplus
}
#endif
#endif
