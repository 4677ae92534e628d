// Vite's host entry points over the C ABI (see vite_host.hpp).
#include "vite_host.hpp"

#include <fcntl.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <mutex>
#include <sstream>

namespace {

[[noreturn]] void fail(const char *what, vg_status st) {
    std::cerr << "vite-b200: " << what << " failed (status " << (int)st
              << "): " << vg_last_error(vite_ctx()) << std::endl;
    std::exit(EXIT_FAILURE);
}

void check(vg_status st, const char *what) {
    if (st != VG_OK) fail(what, st);
}

void one_rank(int me, int nprocs) {
    if (me != 0 || nprocs != 1) {
        std::cerr << "vite-b200 runs the whole graph on one GPU as one rank (me=0, nprocs=1)"
                  << std::endl;
        std::exit(EXIT_FAILURE);
    }
}

// the exchange set-up of exchangeVertexReqs (louvain.cpp:3251-3397) for one rank:
// nothing to send or receive
void no_ghosts(size_t &ssz, size_t &rsz, std::vector<GraphElem> &ssizes,
               std::vector<GraphElem> &rsizes, std::vector<GraphElem> &svdata,
               std::vector<GraphElem> &rvdata) {
    ssz = rsz = 0;
    ssizes.assign(1, 0);
    rsizes.assign(1, 0);
    svdata.clear();
    rvdata.clear();
}

GraphWeight phase(const DistGraph &dg, int et_type, double et_delta, int ordering,
                  const ColorVector *colors, long numColor, CommunityVector &cvect,
                  GraphWeight lower, GraphWeight thresh, int &iters) {
    DistGraph &g = const_cast<DistGraph &>(dg);
    vg_graph *d = g.device();
    if (ordering) {
        if ((int64_t)colors->size() != g.getTotalNumVertices()) {
            std::cerr << "vertexColor must have one entry per vertex" << std::endl;
            std::exit(EXIT_FAILURE);
        }
        check(vg_set_colors(vite_ctx(), d, colors->data(), numColor - 1), "vg_set_colors");
    }
    vg_phase_params p;
    p.lower = lower;
    p.threshold = thresh;
    p.et_type = et_type;
    p.et_delta = et_delta;
    p.ordering = ordering;
    cvect.resize(g.getTotalNumVertices());
    double mod = 0.0;
    int32_t it = 0;
    check(vg_louvain_phase(vite_ctx(), d, &p, cvect.data(), &mod, &it), "vg_louvain_phase");
    iters = it;
    return mod;
}

} // namespace

vg_ctx *vite_ctx() {
    static vg_ctx *ctx = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        const char *dev = std::getenv("VITE_B200_DEVICE");
        vg_status st = vg_ctx_create(dev ? std::atoi(dev) : 0, 0, &ctx);
        if (st != VG_OK) {
            std::cerr << "vite-b200: no usable CUDA device (status " << (int)st << ")" << std::endl;
            std::exit(EXIT_FAILURE);
        }
    });
    return ctx;
}

// ---------------------------------------------------------------------------------
// DistGraph

DistGraph::~DistGraph() {
    delete localGraph;
    delete parts;
    if (dev) vg_graph_free(vite_ctx(), dev);
}

void DistGraph::createLocalGraph(GraphElem lnv, GraphElem lne, const PartRanges *oparts) {
    delete localGraph;
    localGraph = new Graph(lnv, lne);
    delete parts;
    parts = new PartRanges(*oparts);
}

void DistGraph::syncHost() const {
    if (!hostStale) return;
    int64_t nv = 0, ne = 0;
    check(vg_graph_info(dev, &nv, &ne), "vg_graph_info");
    delete localGraph;
    localGraph = new Graph(nv, ne);
    check(vg_graph_download(vite_ctx(), dev, localGraph->edgeListIndexes.data(),
                            reinterpret_cast<vg_edge *>(localGraph->edgeList.data())),
          "vg_graph_download");
    hostStale = false;
}

Graph &DistGraph::getLocalGraph() {
    syncHost();
    return *localGraph;
}

const Graph &DistGraph::getLocalGraph() const {
    syncHost();
    return *localGraph;
}

vg_graph *DistGraph::device() {
    if (!dev) {
        const Graph &g = *localGraph;
        check(vg_graph_upload(vite_ctx(), g.getNumVertices(), g.getNumEdges(),
                              g.edgeListIndexes.data(),
                              reinterpret_cast<const vg_edge *>(g.edgeList.data()), &dev),
              "vg_graph_upload");
    }
    return dev;
}

void DistGraph::adoptDevice(vg_graph *g) {
    dev = g;
    int64_t nv = 0, ne = 0;
    check(vg_graph_info(dev, &nv, &ne), "vg_graph_info");
    totalNumVertices = nv;
    totalNumEdges = ne;
    delete parts;
    parts = new PartRanges{0, nv};
    hostStale = true;
}

// ---------------------------------------------------------------------------------
// Louvain phases (louvain.hpp:80-137): et_type follows main's dispatch (main.cpp:349-369):
// (bool true) = -t 1, (delta, true) = -t 2, (bool false) = -t 3, (delta, false) = -t 4

#define GHOSTS ssz, rsz, ssizes, rsizes, svdata, rvdata
#define GHOST_PARAMS                                                                             \
    size_t &ssz, size_t &rsz, std::vector<GraphElem> &ssizes, std::vector<GraphElem> &rsizes,      \
        std::vector<GraphElem> &svdata, std::vector<GraphElem> &rvdata

GraphWeight distLouvainMethod(const int me, const int nprocs, const DistGraph &dg, GHOST_PARAMS,
                              CommunityVector &cvect, const GraphWeight lower,
                              const GraphWeight thresh, int &iters) {
    one_rank(me, nprocs);
    no_ghosts(GHOSTS);
    return phase(dg, 0, 1.0, 0, nullptr, 1, cvect, lower, thresh, iters);
}

GraphWeight distLouvainMethod(const int me, const int nprocs, const DistGraph &dg, GHOST_PARAMS,
                              CommunityVector &cvect, const GraphWeight lower,
                              const GraphWeight thresh, int &iters, bool ETLocalOrRemote) {
    one_rank(me, nprocs);
    no_ghosts(GHOSTS);
    return phase(dg, ETLocalOrRemote ? 1 : 3, 1.0, 0, nullptr, 1, cvect, lower, thresh, iters);
}

GraphWeight distLouvainMethod(const int me, const int nprocs, const DistGraph &dg, GHOST_PARAMS,
                              CommunityVector &cvect, const GraphWeight lower,
                              const GraphWeight thresh, int &iters, GraphWeight ETDelta,
                              bool ETLocalOrRemote) {
    one_rank(me, nprocs);
    no_ghosts(GHOSTS);
    return phase(dg, ETLocalOrRemote ? 2 : 4, ETDelta, 0, nullptr, 1, cvect, lower, thresh, iters);
}

GraphWeight distLouvainMethodWithColoring(const int me, const int nprocs, const DistGraph &dg,
                                          const long numColor, const ColorVector &vertexColor,
                                          GHOST_PARAMS, CommunityVector &cvect,
                                          const GraphWeight lower, const GraphWeight thresh,
                                          int &iters) {
    one_rank(me, nprocs);
    no_ghosts(GHOSTS);
    return phase(dg, 0, 1.0, 1, &vertexColor, numColor, cvect, lower, thresh, iters);
}

GraphWeight distLouvainMethodWithColoring(const int me, const int nprocs, const DistGraph &dg,
                                          const long numColor, const ColorVector &vertexColor,
                                          GHOST_PARAMS, CommunityVector &cvect,
                                          const GraphWeight lower, const GraphWeight thresh,
                                          int &iters, bool ETLocalOrRemote) {
    one_rank(me, nprocs);
    no_ghosts(GHOSTS);
    return phase(dg, ETLocalOrRemote ? 1 : 3, 1.0, 1, &vertexColor, numColor, cvect, lower, thresh,
                 iters);
}

GraphWeight distLouvainMethodWithColoring(const int me, const int nprocs, const DistGraph &dg,
                                          const long numColor, const ColorVector &vertexColor,
                                          GHOST_PARAMS, CommunityVector &cvect,
                                          const GraphWeight lower, const GraphWeight thresh,
                                          int &iters, GraphWeight ETDelta, bool ETLocalOrRemote) {
    one_rank(me, nprocs);
    no_ghosts(GHOSTS);
    return phase(dg, ETLocalOrRemote ? 2 : 4, ETDelta, 1, &vertexColor, numColor, cvect, lower,
                 thresh, iters);
}

GraphWeight distLouvainMethodVertexOrder(const int me, const int nprocs, const DistGraph &dg,
                                         const long numColor, const ColorVector &vertexColor,
                                         GHOST_PARAMS, CommunityVector &cvect,
                                         const GraphWeight lower, const GraphWeight thresh,
                                         int &iters) {
    one_rank(me, nprocs);
    no_ghosts(GHOSTS);
    return phase(dg, 0, 1.0, 2, &vertexColor, numColor, cvect, lower, thresh, iters);
}

GraphWeight distLouvainMethodVertexOrder(const int me, const int nprocs, const DistGraph &dg,
                                         const long numColor, const ColorVector &vertexColor,
                                         GHOST_PARAMS, CommunityVector &cvect,
                                         const GraphWeight lower, const GraphWeight thresh,
                                         int &iters, bool ETLocalOrRemote) {
    one_rank(me, nprocs);
    no_ghosts(GHOSTS);
    return phase(dg, ETLocalOrRemote ? 1 : 3, 1.0, 2, &vertexColor, numColor, cvect, lower, thresh,
                 iters);
}

GraphWeight distLouvainMethodVertexOrder(const int me, const int nprocs, const DistGraph &dg,
                                         const long numColor, const ColorVector &vertexColor,
                                         GHOST_PARAMS, CommunityVector &cvect,
                                         const GraphWeight lower, const GraphWeight thresh,
                                         int &iters, GraphWeight ETDelta, bool ETLocalOrRemote) {
    one_rank(me, nprocs);
    no_ghosts(GHOSTS);
    return phase(dg, ETLocalOrRemote ? 2 : 4, ETDelta, 2, &vertexColor, numColor, cvect, lower,
                 thresh, iters);
}

// ---------------------------------------------------------------------------------

ColorElem distColoringMultiHashMinMax(const int me, const int nprocs, const DistGraph &dg,
                                      ColorVector &vertexColor, const ColorElem nHash,
                                      const int target_percent, const bool singleIteration) {
    one_rank(me, nprocs);
    DistGraph &g = const_cast<DistGraph &>(dg);
    vertexColor.resize(g.getTotalNumVertices());
    int64_t nc = 0;
    check(vg_color(vite_ctx(), g.device(), nHash, target_percent, singleIteration ? 1 : 0,
                   vertexColor.data(), &nc),
          "vg_color");
    return nc;
}

void distbuildNextLevelGraph(int nprocs, int me, DistGraph *&dg, const size_t &, const size_t &,
                             const std::vector<GraphElem> &, const std::vector<GraphElem> &,
                             const std::vector<GraphElem> &, const std::vector<GraphElem> &,
                             CommunityVector &cvect) {
    one_rank(me, nprocs);
    vg_graph *d = dg->device();
    check(vg_rebuild(vite_ctx(), d, cvect.data()), "vg_rebuild");
    dg->adoptDevice(d);
}

// ---------------------------------------------------------------------------------
// Vite's binary format: [nv:i64][ne:i64][rowptr:i64 x (nv+1)][Edge x ne]
// (converters/convert.cpp:245-278, distgraph.cpp:1008-1061)

static void read_all(int fd, void *buf, size_t len, off_t off, const std::string &name) {
    char *p = static_cast<char *>(buf);
    while (len) {
        const ssize_t got = pread(fd, p, len, off);
        if (got <= 0) {
            std::cout << " Error opening file! " << std::endl;
            std::cerr << "short read from " << name << std::endl;
            std::exit(EXIT_FAILURE);
        }
        p += got;
        len -= (size_t)got;
        off += got;
    }
}

void loadDistGraphMPIIO(int me, int nprocs, int, DistGraph *&dg, std::string &fileName) {
    one_rank(me, nprocs);
    const int fd = open(fileName.c_str(), O_RDONLY);
    if (fd < 0) {
        std::cout << " Error opening file! " << std::endl;
        std::exit(EXIT_FAILURE);
    }
    GraphElem hdr[2];
    read_all(fd, hdr, sizeof(hdr), 0, fileName);
    const GraphElem nv = hdr[0], ne = hdr[1];
    std::cout << "Reading file of " << nv << " vertices and " << ne << " edges." << std::endl;
    dg = new DistGraph(nv, ne);
    PartRanges parts{0, nv};
    dg->createLocalGraph(nv, ne, &parts);
    Graph &g = dg->getLocalGraph();
    read_all(fd, g.edgeListIndexes.data(), sizeof(GraphElem) * (nv + 1), sizeof(hdr), fileName);
    read_all(fd, g.edgeList.data(), sizeof(Edge) * ne,
             sizeof(hdr) + sizeof(GraphElem) * (nv + 1), fileName);
    close(fd);
    // rebase the offsets (distgraph.cpp:244-247)
    const GraphElem base = g.edgeListIndexes[0];
    for (auto &x : g.edgeListIndexes) x -= base;
}

void loadDistGraphMPIIOBalanced(int me, int nprocs, int ranks_per_node, DistGraph *&dg,
                                std::string &fileName) {
    // one rank: the edge-balanced split is the whole graph (distgraph.cpp:256-387)
    loadDistGraphMPIIO(me, nprocs, ranks_per_node, dg, fileName);
}

void writeGraph(int me, int nprocs, DistGraph *&dg, std::vector<GraphElem> &, std::string &fileName) {
    one_rank(me, nprocs);
    const Graph &g = dg->getLocalGraph();
    FILE *f = std::fopen(fileName.c_str(), "wb");
    if (!f) {
        std::cout << " Error opening output binary file for storing graph data! " << std::endl;
        std::exit(EXIT_FAILURE);
    }
    const GraphElem hdr[2] = {g.getNumVertices(), g.getNumEdges()};
    std::fwrite(hdr, sizeof(hdr), 1, f);
    std::fwrite(g.edgeListIndexes.data(), sizeof(GraphElem), g.edgeListIndexes.size(), f);
    std::fwrite(g.edgeList.data(), sizeof(Edge), g.edgeList.size(), f);
    std::fclose(f);
}

void generateInMemGraph(int rank, int nprocs, DistGraph *&dg, GraphElem nv,
                        GraphWeight randomEdgePercent, std::string fileOut) {
    one_rank(rank, nprocs);
    const char *s = std::getenv("VITE_B200_SEED");
    vg_graph *d = nullptr;
    check(vg_generate_rgg(vite_ctx(), nv, randomEdgePercent, s ? std::strtoull(s, nullptr, 10) : 1,
                          &d),
          "vg_generate_rgg");
    int64_t gnv = 0, gne = 0;
    check(vg_graph_info(d, &gnv, &gne), "vg_graph_info");
    dg = new DistGraph(gnv, gne);
    dg->adoptDevice(d);
    if (!fileOut.empty()) {
        std::vector<GraphElem> unused;
        writeGraph(rank, nprocs, dg, unused, fileOut);
        std::cout << "Written binary file: " << fileOut << std::endl;
    }
}

// ---------------------------------------------------------------------------------------
// ground truth

void loadGroundTruthFile(std::vector<GraphElem> &commGroundTruth,
                         std::string const &groundTruthFileName, bool isGroundTruthZeroBased) {
    std::ifstream ifs(groundTruthFileName.c_str(), std::ifstream::in);
    if (!ifs) {
        std::cerr << "Error opening ground truth file: " << groundTruthFileName << std::endl;
        exit(EXIT_FAILURE);
    }
    std::string line;
    while (std::getline(ifs, line)) {
        GraphElem v = -1, comm_id = -1;
        std::istringstream iss(line);
        iss >> v >> comm_id;
        if (!isGroundTruthZeroBased) comm_id--;
        commGroundTruth.push_back(comm_id);
    }
    std::cout << "Loaded ground-truth file: " << groundTruthFileName
              << ", containing community information for " << commGroundTruth.size()
              << " vertices." << std::endl;
}

void compare_communities(std::vector<GraphElem> const &C1, std::vector<GraphElem> const &C2) {
    if (C1.empty() || C1.size() != C2.size()) {
        std::cerr << "compare_communities: the truth has " << C1.size()
                  << " vertices and the communities " << C2.size() << std::endl;
        exit(EXIT_FAILURE);
    }
    vg_compare_stats st;
    check(vg_compare_communities(vite_ctx(), (int64_t)C1.size(), C1.data(), C2.data(), &st),
          "vg_compare_communities");
    std::cout << "Number of unique communities in C1 = " << st.nc1 << ", and C2 = " << st.nc2
              << std::endl;
    std::cout << "*******************************************" << std::endl;
    std::cout << "Communities comparison statistics:" << std::endl;
    std::cout << "*******************************************" << std::endl;
    std::cout << "|C1| (truth)       : " << st.n << std::endl;
    std::cout << "#communities in C1 : " << st.nc1 << std::endl;
    std::cout << "|C2| (output)      : " << st.n << std::endl;
    std::cout << "#communities in C2 : " << st.nc2 << std::endl;
    std::cout << "-------------------------------------------" << std::endl;
    std::cout << "Same-Same (True positive)  : " << st.same_same << std::endl;
    std::cout << "Same-Diff (False negative) : " << st.same_diff << std::endl;
    std::cout << "Diff-Same (False positive) : " << st.diff_same << std::endl;
    std::cout << "-------------------------------------------" << std::endl;
    std::cout << "Precision :  " << st.precision << " (" << (st.precision * 100) << ")" << std::endl;
    std::cout << "Recall    :  " << st.recall << " (" << (st.recall * 100) << ")" << std::endl;
    std::cout << "F-score   :  " << st.fscore << std::endl;
    std::cout << "-------------------------------------------" << std::endl;
    std::cout << "Gini coefficient, C1  :  " << st.gini1 << std::endl;
    std::cout << "Gini coefficient, C2  :  " << st.gini2 << std::endl;
    std::cout << "*******************************************" << std::endl;
}
