/*
 * vite_oracle: plain-C, single-threaded restatement of Vite's Louvain path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA product
 * path: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it. It follows the reference sequentially (the order a one-thread
 * OpenMP run of the reference takes), so on any weights it reproduces a
 * one-thread reference run bit for bit; the tests pin it against the
 * reference's own outputs (tests/golden/).
 *
 * Ids are int64 and weights double, like the reference's default build
 * (edge.hpp:65-69).
 */
#ifndef VITE_ORACLE_H
#define VITE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vo_graph {
    int64_t nv, ne;
    int64_t *rowptr; /* nv+1 */
    int64_t *tail;   /* ne */
    double *weight;  /* ne */
} vo_graph;

typedef struct vo_phase_params {
    double lower;      /* `lower` of distLouvainMethod (louvain.hpp:80-96); main passes -1 */
    double threshold;  /* `thresh` */
    int et_type;       /* 0: plain; 1..4: main.cpp:349-369 dispatch of -t */
    double et_delta;   /* -a alpha (used by types 2 and 4) */
    int ordering;      /* 0 plain, 1 distLouvainMethodWithColoring, 2 distLouvainMethodVertexOrder */
    int64_t num_color; /* numColor argument = colors returned by the coloring + 1 */
} vo_phase_params;

/* graph lifetime */
int vo_graph_alloc(vo_graph *g, int64_t nv, int64_t ne);
void vo_graph_free(vo_graph *g);

/* std::seed_seq({seed}).generate() first word (utils.hpp:163-170) */
uint32_t vo_seed_seq1(uint32_t seed);
/* LCG(seed, drand, count).generate() for one rank (utils.hpp:135-298) */
void vo_lcg_drand(uint32_t seed, int64_t count, double *drand);
/* r(n) of generateInMemGraph (distgraph.cpp:395-399) */
double vo_rgg_radius(int64_t n);
/* generateRGG for one rank without extra edges (distgraph.cpp:412-983) */
int vo_rgg(int64_t n, vo_graph *out);
/* seeded extra edges with U(0,1) weights (this project's seeded variant of
 * distgraph.cpp:702-892); returns the number of undirected edges added */
int64_t vo_add_random_edges(const vo_graph *in, double percent, uint64_t seed, vo_graph *out);
/* seeded Barabasi-Albert (hash-resolved Batagelj-Brandes copy model) and
 * Erdos-Renyi G(n, M) generators: this project's own designs, no reference code */
int vo_ba(int64_t n, int64_t m, uint64_t seed, vo_graph *out);
int vo_er(int64_t n, double avg_degree, uint64_t seed, vo_graph *out);
/* weights: mode 1 = all 1.0, mode 2 = U(0,1) hashed on the unordered pair */
void vo_reweight(vo_graph *g, int mode, uint64_t seed);
/* the counter-based generator shared with the CUDA generators */
uint64_t vo_mix(uint64_t seed, uint64_t stream, uint64_t k);

/* distSumVertexDegree + distCalcConstantForSecondTerm (louvain.cpp:2161-2218) */
double vo_vertex_degree(const vo_graph *g, double *vdeg);

/* one Louvain phase; returns 0 on success. cvect_out[nv], colors may be NULL
 * when ordering == 0 (louvain.cpp:7-1938) */
int vo_louvain_phase(const vo_graph *g, const vo_phase_params *p, const int64_t *colors,
                     int64_t *cvect_out, double *mod_out, int *iters_out);

/* distColoringMultiHashMinMax for one rank (coloring.cpp:52-118); returns nextColor */
int64_t vo_color(const vo_graph *g, int64_t nHash, int target_percent, int single_iteration,
                 int64_t *colors_out);
uint32_t vo_color_hash(uint32_t a, uint32_t seed);

/* distbuildNextLevelGraph for one rank (rebuild.cpp:77-504) */
int vo_rebuild(const vo_graph *g, const int64_t *cvect, vo_graph *out);

/* main.cpp phase loop (main.cpp:242-513); per-level outputs up to max_levels.
 * Returns the number of levels recorded (accepted and final rejected phase). */
typedef struct vo_run_params {
    double threshold;   /* -h, default 1e-6 */
    int coloring;       /* -c */
    int vertex_order;   /* -d */
    int max_colors;     /* k of -c/-d */
    int single_color_iter;
    int et_type;        /* -t (0 = off) */
    double et_delta;    /* -a */
    int threshold_scaling; /* -i */
    int one_phase;      /* -p */
} vo_run_params;

int vo_run(const vo_graph *g0, const vo_run_params *rp, int max_levels, int64_t *level_nv,
           int64_t *level_ne, int *level_iters, double *level_mod, int64_t *level_colors,
           double *seconds_out);

/* compare_communities + compute_gini_coeff (compare.cpp:58-318): c1 the truth. */
typedef struct vo_compare_stats {
    int64_t n, nc1, nc2, same_same, same_diff, diff_same;
    double precision, recall, fscore, gini1, gini2;
} vo_compare_stats;
int vo_compare(int64_t n, const int64_t *c1, const int64_t *c2, vo_compare_stats *out);

#ifdef __cplusplus
}
#endif
#endif
