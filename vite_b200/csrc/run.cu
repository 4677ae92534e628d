// The phase loop of graphClustering (main.cpp:242-513) with the graph kept on
// the device from level to level: coloring at phase 0, the phase variant that
// main dispatches, the rebuild test (main.cpp:378) and rebuild (:431), the exit
// re-run under threshold cycling (:448-463) and the phase caps (:504-512).
#include "vg_internal.cuh"


void vg_phase_internal(vg_ctx *ctx, vg_graph *g, const vg_phase_params *p, double *mod_out,
                       int32_t *iters_out, double *sweep_ms, int64_t *edges);
int64_t vg_color_internal(vg_ctx *ctx, vg_graph *g, int64_t nHash, int32_t target_percent,
                          int32_t single_iteration);
vg_graph *vg_rebuild_new(vg_ctx *ctx, const vg_graph *g, const int32_t *comm);

namespace {

struct EventTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t s;
    explicit EventTimer(cudaStream_t st) : s(st) {
        VG_CUDA(cudaEventCreate(&a));
        VG_CUDA(cudaEventCreate(&b));
        VG_CUDA(cudaEventRecord(a, s));
    }
    double stop_ms() {
        VG_CUDA(cudaEventRecord(b, s));
        VG_CUDA(cudaEventSynchronize(b));
        float ms = 0.f;
        VG_CUDA(cudaEventElapsedTime(&ms, a, b));
        return ms;
    }
    ~EventTimer() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

} // namespace

extern "C" vg_status vg_louvain_run(vg_ctx *ctx, const vg_graph *g0, const vg_run_params *rp,
                                    vg_level_stat *levels, int32_t max_levels,
                                    int32_t *nlevels_out, int64_t *comm_out) {
    if (!ctx || !g0 || !rp) return VG_ERR_ARG;
    vg_graph *owned = nullptr;
    vg_status st = vg_guard(ctx, [&] {
        VG_CUDA(cudaSetDevice(ctx->device));
        VG_REQUIRE(!(rp->coloring && rp->vertex_order),
                   "Cannot turn on both coloring (-c) and vertex ordering (-d)");
        VG_REQUIRE(!(rp->one_phase && rp->threshold_scaling),
                   "Cannot turn on threshold-cycling (-i) with a single phase run (-p)");
        VG_REQUIRE(rp->et_type >= 0 && rp->et_type <= 4, "early-term-type parameter is between 1-4");
        VG_REQUIRE(!((rp->et_type == 2 || rp->et_type == 4) &&
                     (rp->et_delta > 1.0 || rp->et_delta < 0.0)),
                   "early-term-alpha must be between 0 and 1");
        // whether sums of g0's weights are exact in any order: computed once, cached on g0
        vg_weights_integral(ctx, const_cast<vg_graph *>(g0));
        // level 0 runs on a shallow view of g0 so that its attached state stays untouched
        vg_graph view = *g0;
        view.colors = nullptr;
        view.comm = nullptr;
        view.num_colors = -1;
        vg_graph *cur = &view;
        VG_REQUIRE(rp->layout >= 0 && rp->layout <= 2, "layout must be 0, 1 or 2");
        double layout_s = 0.0;
        if (vg_auto_layout(ctx, g0, rp->layout)) {
            EventTimer tl(ctx->stream);
            DevBuf<int32_t> order;
            vg_bfs_order(ctx, g0, order);
            owned = vg_apply_layout(ctx, g0, order.p);
            cur = owned;
            layout_s = tl.stop_ms() * 1e-3;
        }
        // the -o map lives on the device; it is copied out once at the end
        DevBuf<int32_t> commAll;
        if (comm_out) commAll.alloc(ctx, g0->nv);
        double currMod = -1.0, prevMod = -1.0, threshold = rp->threshold;
        int phase = 0, short_phase = 0, tot_iters = 0, nrec = 0;
        auto cleanup_view = [&] {
            vg_free(ctx, view.colors, sizeof(int32_t) * view.nv);
            vg_free(ctx, view.comm, sizeof(int32_t) * view.nv);
            view.colors = nullptr;
            view.comm = nullptr;
        };
        try {
            for (;;) {
                if (rp->threshold_scaling && !rp->one_phase) {
                    if (short_phase > 12) short_phase = 0;
                    if (short_phase <= 2) threshold = 1.0E-3;
                    else if (short_phase <= 6) threshold = 1.0E-4;
                    else if (short_phase <= 9) threshold = 1.0E-5;
                    else threshold = rp->threshold;
                } else
                    threshold = rp->threshold;
                vg_level_stat ls = {};
                ls.nv = cur->nv;
                ls.ne = cur->ne;
                if (phase == 0) ls.seconds_layout = layout_s;
                vg_phase_params pp = {};
                pp.lower = currMod;
                pp.threshold = threshold;
                pp.et_type = rp->et_type;
                pp.et_delta = rp->et_delta;
                pp.ordering = 0;
                if ((rp->coloring || rp->vertex_order) && phase == 0) {
                    EventTimer tc(ctx->stream);
                    ls.num_colors = vg_color_internal(ctx, cur, rp->max_colors / 2, 70 /* MAX_COVG */,
                                                      rp->single_color_iter);
                    ls.seconds_color = tc.stop_ms() * 1e-3;
                    pp.ordering = rp->coloring ? 1 : 2;
                }
                int32_t iters = 0;
                {
                    EventTimer tp(ctx->stream);
                    double sweep_ms = 0.0;
                    vg_phase_internal(ctx, cur, &pp, &currMod, &iters, &sweep_ms, &ls.edges_swept);
                    ls.seconds_phase = tp.stop_ms() * 1e-3;
                    ls.seconds_sweep = sweep_ms * 1e-3;
                }
                ls.iters = iters;
                ls.modularity = currMod;
                tot_iters += iters;
                const bool accepted = (currMod - prevMod) > threshold;
                if (accepted) {
                    if (comm_out) vg_compose_level(ctx, cur, commAll.p, g0->nv, phase == 0);
                    if (!rp->one_phase) {
                        EventTimer tr(ctx->stream);
                        vg_graph *next = vg_rebuild_new(ctx, cur, cur->comm);
                        if (cur == &view) {
                            cleanup_view();
                        } else {
                            vg_graph_release(ctx, owned);
                            delete owned;
                        }
                        owned = next;
                        cur = owned;
                        ls.seconds_rebuild = tr.stop_ms() * 1e-3;
                    }
                }
                if (levels && nrec < max_levels) levels[nrec] = ls;
                nrec++;
                if (!accepted) {
                    if (rp->threshold_scaling && !rp->one_phase && phase < 10) {
                        vg_level_stat lx = {};
                        lx.nv = cur->nv;
                        lx.ne = cur->ne;
                        vg_phase_params px = {};
                        px.lower = currMod;
                        px.threshold = 1.0E-6;
                        EventTimer tp(ctx->stream);
                        double sweep_ms = 0.0;
                        vg_phase_internal(ctx, cur, &px, &currMod, &iters, &sweep_ms, &lx.edges_swept);
                        lx.seconds_phase = tp.stop_ms() * 1e-3;
                        lx.seconds_sweep = sweep_ms * 1e-3;
                        lx.iters = iters;
                        lx.modularity = currMod;
                        if (levels && nrec < max_levels) levels[nrec] = lx;
                        nrec++;
                    }
                    break;
                }
                prevMod = currMod;
                currMod = -1.0;
                phase++;
                if (rp->one_phase) break;
                if (rp->threshold_scaling && !rp->one_phase) short_phase++;
                if (phase == 200 /* TERMINATION_PHASE_COUNT */ || tot_iters > 10000) break;
            }
        } catch (...) {
            cleanup_view();
            throw;
        }
        cleanup_view();
        if (nlevels_out) *nlevels_out = nrec;
        if (comm_out) vg_download_map(ctx, commAll.p, g0->nv, comm_out);
        vg_sync(ctx);
    });
    if (owned) {
        vg_graph_release(ctx, owned);
        delete owned;
    }
    return st;
}
