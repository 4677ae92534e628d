// Host C++ interface of vite-b200 with Vite's types and entry points.
//
// The types keep the layout of Vite's default 64-bit build -- Edge{int64 tail,
// double weight} (edge.hpp:65-80), Graph's edgeListIndexes/edgeList CSR
// (graph.hpp:77-106), DistGraph with 1-D `parts` (distgraph.hpp:77-107) -- and
// the functions keep the signatures Vite's main calls (louvain.hpp:80-137,
// coloring.hpp:86, rebuild.hpp:109-112, distgraph.hpp:109-119), so a caller
// written against Vite links against libvite_host.so instead. There is one rank:
// `me` must be 0 and `nprocs` 1; the ghost-exchange buffers (ssz ... rvdata) are
// accepted and left empty. Every call runs on the GPU through include/vite_b200.h;
// a DistGraph keeps its device copy from level to level and fills its host CSR
// only when asked (getLocalGraph()).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "vite_b200.h"

typedef int64_t GraphElem;
typedef double GraphWeight;
typedef int64_t ColorElem;
typedef std::vector<GraphElem> CommunityVector;
typedef std::vector<ColorElem> ColorVector;
typedef std::vector<GraphElem> PartRanges;

#ifndef CONVERGENCE_THRESHOLD
#define CONVERGENCE_THRESHOLD (1.0E-06)
#endif
#ifndef TERMINATION_PHASE_COUNT
#define TERMINATION_PHASE_COUNT (200)
#endif
#ifndef MAX_COVG
#define MAX_COVG (70)
#endif

struct Edge {
    GraphElem tail;
    GraphWeight weight;
    Edge() : tail(-1), weight(0.0) {}
    Edge(GraphElem t, GraphWeight w) : tail(t), weight(w) {}
};
static_assert(sizeof(Edge) == sizeof(vg_edge), "Edge must match vg_edge");

class Graph {
  public:
    std::vector<GraphElem> edgeListIndexes;
    std::vector<Edge> edgeList;

    Graph(GraphElem nv, GraphElem ne) : numVertices(nv), numEdges(ne) {
        edgeListIndexes.assign(nv + 1, 0);
        edgeList.resize(ne);
    }
    GraphElem getNumVertices() const { return numVertices; }
    GraphElem getNumEdges() const { return numEdges; }
    void setNumEdges(GraphElem ne) {
        edgeList.resize(ne);
        numEdges = ne;
    }
    void setEdgeWeightstoOne() {
        for (auto &e : edgeList) e.weight = 1.0;
    }
    void getEdgeRangeForVertex(GraphElem v, GraphElem &e0, GraphElem &e1) const {
        e0 = edgeListIndexes[v];
        e1 = edgeListIndexes[v + 1];
    }
    const Edge &getEdge(GraphElem e) const { return edgeList[e]; }
    Edge &getEdge(GraphElem e) { return edgeList[e]; }

  private:
    GraphElem numVertices, numEdges;
};

class DistGraph {
  public:
    PartRanges *parts = nullptr;

    DistGraph(GraphElem tnv, GraphElem tne) : totalNumVertices(tnv), totalNumEdges(tne) {}
    ~DistGraph();
    DistGraph(const DistGraph &) = delete;
    DistGraph &operator=(const DistGraph &) = delete;

    GraphElem getTotalNumVertices() const { return totalNumVertices; }
    GraphElem getTotalNumEdges() const { return totalNumEdges; }
    void setNumEdges(GraphElem ne) { totalNumEdges = ne; }
    void createLocalGraph(GraphElem lnv, GraphElem lne, const PartRanges *oparts);
    // host CSR; downloaded from the device copy on first use after a device-side change
    Graph &getLocalGraph();
    const Graph &getLocalGraph() const;
    GraphElem getBase(int me) const { return (*parts)[me]; }
    GraphElem getBound(int me) const { return (*parts)[me + 1]; }
    int getOwner(GraphElem) const { return 0; }

    // device copy (uploaded on first use); owned by the graph
    vg_graph *device();
    // the device copy became the truth (after a rebuild); the host CSR is stale
    void adoptDevice(vg_graph *g);

  private:
    GraphElem totalNumVertices, totalNumEdges;
    mutable Graph *localGraph = nullptr;
    mutable bool hostStale = false;
    vg_graph *dev = nullptr;
    void syncHost() const;
};

// the process's GPU context (device from VITE_B200_DEVICE, default 0)
vg_ctx *vite_ctx();

// --- Louvain phase: the nine overloads of louvain.hpp:80-137 -------------------------
GraphWeight distLouvainMethod(const int me, const int nprocs, const DistGraph &dg, size_t &ssz,
                              size_t &rsz, std::vector<GraphElem> &ssizes,
                              std::vector<GraphElem> &rsizes, std::vector<GraphElem> &svdata,
                              std::vector<GraphElem> &rvdata, CommunityVector &cvect,
                              const GraphWeight lower, const GraphWeight thresh, int &iters);
GraphWeight distLouvainMethod(const int me, const int nprocs, const DistGraph &dg, size_t &ssz,
                              size_t &rsz, std::vector<GraphElem> &ssizes,
                              std::vector<GraphElem> &rsizes, std::vector<GraphElem> &svdata,
                              std::vector<GraphElem> &rvdata, CommunityVector &cvect,
                              const GraphWeight lower, const GraphWeight thresh, int &iters,
                              bool ETLocalOrRemote);
GraphWeight distLouvainMethod(const int me, const int nprocs, const DistGraph &dg, size_t &ssz,
                              size_t &rsz, std::vector<GraphElem> &ssizes,
                              std::vector<GraphElem> &rsizes, std::vector<GraphElem> &svdata,
                              std::vector<GraphElem> &rvdata, CommunityVector &cvect,
                              const GraphWeight lower, const GraphWeight thresh, int &iters,
                              GraphWeight ETDelta, bool ETLocalOrRemote);
GraphWeight distLouvainMethodWithColoring(const int me, const int nprocs, const DistGraph &dg,
                                          const long numColor, const ColorVector &vertexColor,
                                          size_t &ssz, size_t &rsz, std::vector<GraphElem> &ssizes,
                                          std::vector<GraphElem> &rsizes,
                                          std::vector<GraphElem> &svdata,
                                          std::vector<GraphElem> &rvdata, CommunityVector &cvect,
                                          const GraphWeight lower, const GraphWeight thresh,
                                          int &iters);
GraphWeight distLouvainMethodWithColoring(const int me, const int nprocs, const DistGraph &dg,
                                          const long numColor, const ColorVector &vertexColor,
                                          size_t &ssz, size_t &rsz, std::vector<GraphElem> &ssizes,
                                          std::vector<GraphElem> &rsizes,
                                          std::vector<GraphElem> &svdata,
                                          std::vector<GraphElem> &rvdata, CommunityVector &cvect,
                                          const GraphWeight lower, const GraphWeight thresh,
                                          int &iters, bool ETLocalOrRemote);
GraphWeight distLouvainMethodWithColoring(const int me, const int nprocs, const DistGraph &dg,
                                          const long numColor, const ColorVector &vertexColor,
                                          size_t &ssz, size_t &rsz, std::vector<GraphElem> &ssizes,
                                          std::vector<GraphElem> &rsizes,
                                          std::vector<GraphElem> &svdata,
                                          std::vector<GraphElem> &rvdata, CommunityVector &cvect,
                                          const GraphWeight lower, const GraphWeight thresh,
                                          int &iters, GraphWeight ETDelta, bool ETLocalOrRemote);
GraphWeight distLouvainMethodVertexOrder(const int me, const int nprocs, const DistGraph &dg,
                                         const long numColor, const ColorVector &vertexColor,
                                         size_t &ssz, size_t &rsz, std::vector<GraphElem> &ssizes,
                                         std::vector<GraphElem> &rsizes,
                                         std::vector<GraphElem> &svdata,
                                         std::vector<GraphElem> &rvdata, CommunityVector &cvect,
                                         const GraphWeight lower, const GraphWeight thresh,
                                         int &iters);
GraphWeight distLouvainMethodVertexOrder(const int me, const int nprocs, const DistGraph &dg,
                                         const long numColor, const ColorVector &vertexColor,
                                         size_t &ssz, size_t &rsz, std::vector<GraphElem> &ssizes,
                                         std::vector<GraphElem> &rsizes,
                                         std::vector<GraphElem> &svdata,
                                         std::vector<GraphElem> &rvdata, CommunityVector &cvect,
                                         const GraphWeight lower, const GraphWeight thresh,
                                         int &iters, bool ETLocalOrRemote);
GraphWeight distLouvainMethodVertexOrder(const int me, const int nprocs, const DistGraph &dg,
                                         const long numColor, const ColorVector &vertexColor,
                                         size_t &ssz, size_t &rsz, std::vector<GraphElem> &ssizes,
                                         std::vector<GraphElem> &rsizes,
                                         std::vector<GraphElem> &svdata,
                                         std::vector<GraphElem> &rvdata, CommunityVector &cvect,
                                         const GraphWeight lower, const GraphWeight thresh,
                                         int &iters, GraphWeight ETDelta, bool ETLocalOrRemote);

// --- coloring (coloring.hpp:86), rebuild (rebuild.hpp:109-112) ----------------------
ColorElem distColoringMultiHashMinMax(const int me, const int nprocs, const DistGraph &dg,
                                      ColorVector &vertexColor, const ColorElem nHash,
                                      const int target_percent, const bool singleIteration);
void distbuildNextLevelGraph(int nprocs, int me, DistGraph *&dg, const size_t &ssz,
                             const size_t &rsz, const std::vector<GraphElem> &ssizes,
                             const std::vector<GraphElem> &rsizes,
                             const std::vector<GraphElem> &svdata,
                             const std::vector<GraphElem> &rvdata, CommunityVector &cvect);

// --- ground truth (louvain.hpp:201, compare.hpp) -------------------------------------
// one "vertex community" pair per line (LFR format); ids shifted down by one unless
// zero-based
void loadGroundTruthFile(std::vector<GraphElem> &commGroundTruth,
                         std::string const &groundTruthFileName, bool isGroundTruthZeroBased);
// pair counts, precision, recall, F-score and Gini coefficients of C2 against the
// truth C1, printed as the reference prints them; computed on the GPU
void compare_communities(std::vector<GraphElem> const &C1, std::vector<GraphElem> const &C2);

// --- graph input/output and generation (distgraph.hpp:109-119) -----------------------
void loadDistGraphMPIIO(int me, int nprocs, int ranks_per_node, DistGraph *&dg,
                        std::string &fileName);
void loadDistGraphMPIIOBalanced(int me, int nprocs, int ranks_per_node, DistGraph *&dg,
                                std::string &fileName);
void generateInMemGraph(int rank, int nprocs, DistGraph *&dg, GraphElem nv,
                        GraphWeight randomEdgePercent, std::string fileOut);
void writeGraph(int me, int nprocs, DistGraph *&dg, std::vector<GraphElem> &edgeCount,
                std::string &fileName);
