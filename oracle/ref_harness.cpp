// Reference harness: TEST INFRASTRUCTURE for the oracle, never part of the product.
//
// Links the UNMODIFIED reference objects (louvain.cpp, rebuild.cpp, coloring.cpp,
// distgraph.cpp, utils.cpp, compare.cpp built against the single-rank MPI shim)
// and drives them with the same phase loop as the reference's `main`
// (main.cpp:242-513): threshold choice (:249-263), coloring / vertex ordering at
// phase 0 only (:267-347), early-termination dispatch (:349-370), the rebuild test
// (:378) and rebuild (:431), the exit re-run under threshold cycling (:448-463)
// and the phase caps (:504-512).  Unlike the reference `main`, it records every
// level's result (community vector, modularity printed with all 17 digits,
// iteration count, colors) and, on request, the CSR each level ran on, in a small
// binary record file that the parity tests and the golden-fixture script read.
// With -r R it runs the whole level loop R times, each run on a copy of the
// loaded graph made before its clock starts, and prints each run's totals
// (clustering + rebuild seconds, as main's "Average time for clustering" and
// "Rebuild Time" lines add up); -B stops before a run that would end past a
// budget of seconds. Only the first run is recorded.
//
// Record file layout (little endian):
//   header  : "VREC" u32 version=1
//   level   : i32 tag=1, i64 level, i64 nv, i64 ne, i32 iters, f64 mod,
//             i64 numColors, f64 seconds_clustering, f64 seconds_rebuild,
//             i64 cvect[nv]
//   graph   : i32 tag=2, i64 level, i64 nv, i64 ne, i64 rowptr[nv+1],
//             i64 tail[ne], f64 weight[ne]
//   colors  : i32 tag=3, i64 nv, i64 color[nv]
//   end     : i32 tag=0
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <omp.h>
#include <mpi.h>

#include "rebuild.hpp"
#include "louvain.hpp"
#include "coloring.hpp"
#include "utils.hpp"

std::ofstream ofs;
std::ofstream ofcks;

struct Opts {
  long long genN = 0;
  double randomEdgePercent = 0.0;
  std::string inFile, saveGraph, recFile;
  bool unitWeights = false;
  bool coloring = false, vertexOrdering = false, singleColorIter = false;
  int maxColors = 8;
  bool earlyTerm = false;
  int etType = 0;
  double etDelta = 1.0;
  bool thresholdScaling = false, runOnePhase = false;
  double threshold = CONVERGENCE_THRESHOLD;
  bool dumpGraphs = false;
  int repeats = 1;          // timed runs of the whole level loop from the loaded graph
  double budget = 0.0;      // seconds; 0 = no limit on the repeats
};

static void usage()
{
  std::fprintf(stderr,
      "vite_ref_harness (-n N [-e pct] [-s save.bin] | -f file) [-u] [-c \"k [single]\"]\n"
      "  [-d \"k [single]\"] [-t type] [-a alpha] [-i] [-p] [-h thresh] [-w out.rec] [-G]\n"
      "  [-r repeats] [-B budget_seconds]\n");
  std::exit(2);
}

static void parseColor(const char *arg, Opts &o)
{
  std::string s(arg);
  size_t sp = s.find(' ');
  o.maxColors = std::atoi(s.substr(0, sp).c_str());
  if (sp != std::string::npos) {
    std::string b = s.substr(sp + 1);
    o.singleColorIter = (b == "true" || b == "1" || b == "TRUE" || b == "True");
  }
}

static FILE *g_rec = nullptr;

template <class T> static void put(const T &v) { std::fwrite(&v, sizeof(T), 1, g_rec); }

static void recordGraph(long long level, const DistGraph &dg)
{
  if (!g_rec) return;
  const Graph &g = dg.getLocalGraph();
  const long long nv = g.getNumVertices(), ne = g.getNumEdges();
  put<int>(2); put(level); put(nv); put(ne);
  std::fwrite(g.edgeListIndexes.data(), sizeof(GraphElem), nv + 1, g_rec);
  std::vector<long long> tails(ne);
  std::vector<double> w(ne);
  for (long long e = 0; e < ne; e++) { tails[e] = g.edgeList[e].tail; w[e] = g.edgeList[e].weight; }
  std::fwrite(tails.data(), sizeof(long long), ne, g_rec);
  std::fwrite(w.data(), sizeof(double), ne, g_rec);
}

struct RunTotals {
  double clustering = 0.0, rebuild = 0.0, finalMod = 0.0;
  int levels = 0, iterations = 0;
};

// One run of main's phase loop (main.cpp:242-513) on dg, which the rebuilds
// replace (rebuild.cpp:334) and which is deleted at the end.
static RunTotals runLevels(int me, int nprocs, DistGraph *dg, const Opts &o)
{
  GraphWeight currMod = -1.0, prevMod = -1.0, threshold = o.threshold;
  int phase = 0, short_phase = 0, iters = 0, tot_iters = 0;
  ColorElem numColors = 0;
  ColorVector colors;
  CommunityVector cvect;
  std::vector<GraphElem> ssizes, rsizes, svdata, rvdata;
  size_t ssz = 0, rsz = 0;
  double totalClustering = 0.0, totalRebuild = 0.0;

  while (true) {
    if (o.thresholdScaling && !o.runOnePhase) {
      if (short_phase > 12) short_phase = 0;
      if (short_phase <= 2) threshold = 1.0E-3;
      else if (short_phase <= 6) threshold = 1.0E-4;
      else if (short_phase <= 9) threshold = 1.0E-5;
      else threshold = o.threshold;
    } else
      threshold = o.threshold;

    if (o.dumpGraphs) recordGraph(phase, *dg);
    const long long lnv = dg->getLocalGraph().getNumVertices();
    const long long lne = dg->getLocalGraph().getNumEdges();
    numColors = 0;
    double t1 = MPI_Wtime();
    const bool et = o.earlyTerm;
    const int ty = o.etType;
    if ((o.coloring || o.vertexOrdering) && phase == 0) {
      numColors = distColoringMultiHashMinMax(me, nprocs, *dg, colors, (o.maxColors / 2),
                                              MAX_COVG, o.singleColorIter);
      if (g_rec) {
        put<int>(3); put((long long)colors.size());
        std::fwrite(colors.data(), sizeof(ColorElem), colors.size(), g_rec);
      }
      if (o.coloring) {
        if (et && ty == 1) currMod = distLouvainMethodWithColoring(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, true);
        else if (et && ty == 2) currMod = distLouvainMethodWithColoring(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, o.etDelta, true);
        else if (et && ty == 3) currMod = distLouvainMethodWithColoring(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, false);
        else if (et && ty == 4) currMod = distLouvainMethodWithColoring(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, o.etDelta, false);
        else currMod = distLouvainMethodWithColoring(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters);
      } else {
        if (et && ty == 1) currMod = distLouvainMethodVertexOrder(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, true);
        else if (et && ty == 2) currMod = distLouvainMethodVertexOrder(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, o.etDelta, true);
        else if (et && ty == 3) currMod = distLouvainMethodVertexOrder(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, false);
        else if (et && ty == 4) currMod = distLouvainMethodVertexOrder(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, o.etDelta, false);
        else currMod = distLouvainMethodVertexOrder(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters);
      }
    } else {
      if (et && ty == 1) currMod = distLouvainMethod(me, nprocs, *dg, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, true);
      else if (et && ty == 2) currMod = distLouvainMethod(me, nprocs, *dg, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, o.etDelta, true);
      else if (et && ty == 3) currMod = distLouvainMethod(me, nprocs, *dg, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, false);
      else if (et && ty == 4) currMod = distLouvainMethod(me, nprocs, *dg, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, o.etDelta, false);
      else currMod = distLouvainMethod(me, nprocs, *dg, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters);
    }
    double t0 = MPI_Wtime();
    tot_iters += iters;
    totalClustering += (t0 - t1);
    double rebuildSec = 0.0;
    const bool accepted = (currMod - prevMod) > threshold;

    if (g_rec) {
      put<int>(1); put((long long)phase); put(lnv); put(lne); put<int>(iters); put((double)currMod);
      put((long long)numColors); put(t0 - t1); put(0.0);
      std::fwrite(cvect.data(), sizeof(GraphElem), cvect.size(), g_rec);
    }
    std::printf("HARNESS level %d nv %lld ne %lld iters %d mod %.17g colors %lld clustering_s %.6f\n",
                phase, lnv, lne, iters, (double)currMod, (long long)numColors, t0 - t1);

    if (accepted) {
      if (!o.runOnePhase) {
        double t3 = MPI_Wtime();
        distbuildNextLevelGraph(nprocs, me, dg, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect);
        double t2 = MPI_Wtime();
        rebuildSec = t2 - t3;
        totalRebuild += rebuildSec;
        std::printf("HARNESS rebuild %d seconds %.6f\n", phase, rebuildSec);
      }
    } else {
      if (o.thresholdScaling && !o.runOnePhase && phase < 10) {
        double tx = MPI_Wtime();
        currMod = distLouvainMethod(me, nprocs, *dg, ssz, rsz, ssizes, rsizes, svdata, rvdata,
                                    cvect, currMod, 1.0E-6, iters);
        totalClustering += MPI_Wtime() - tx;
        std::printf("HARNESS exit_rerun iters %d mod %.17g\n", iters, (double)currMod);
        if (g_rec) {
          put<int>(1); put((long long)-1); put(lnv); put(lne); put<int>(iters); put((double)currMod);
          put((long long)0); put(0.0); put(0.0);
          std::fwrite(cvect.data(), sizeof(GraphElem), cvect.size(), g_rec);
        }
      }
      break;
    }
    prevMod = currMod;
    currMod = -1.0;
    phase++;
    if (o.runOnePhase) break;
    if (o.thresholdScaling && !o.runOnePhase) short_phase++;
    if (phase == TERMINATION_PHASE_COUNT || tot_iters > 10000) break;
  }

  RunTotals t;
  t.clustering = totalClustering;
  t.rebuild = totalRebuild;
  t.levels = phase;
  t.iterations = tot_iters;
  t.finalMod = prevMod;
  delete dg;
  return t;
}

int main(int argc, char **argv)
{
  MPI_Init(&argc, &argv);
  int me = 0, nprocs = 1;
  MPI_Comm_rank(MPI_COMM_WORLD, &me);
  MPI_Comm_size(MPI_COMM_WORLD, &nprocs);

  Opts o;
  for (int i = 1; i < argc; i++) {
    std::string a(argv[i]);
    auto need = [&](void) -> const char * { if (i + 1 >= argc) usage(); return argv[++i]; };
    if (a == "-n") o.genN = std::atoll(need());
    else if (a == "-e") o.randomEdgePercent = std::atof(need());
    else if (a == "-s") o.saveGraph = need();
    else if (a == "-f") o.inFile = need();
    else if (a == "-u") o.unitWeights = true;
    else if (a == "-c") { parseColor(need(), o); o.coloring = true; }
    else if (a == "-d") { parseColor(need(), o); o.vertexOrdering = true; }
    else if (a == "-t") { o.earlyTerm = true; o.etType = std::atoi(need()); }
    else if (a == "-a") o.etDelta = std::atof(need());
    else if (a == "-i") o.thresholdScaling = true;
    else if (a == "-p") o.runOnePhase = true;
    else if (a == "-h") o.threshold = std::atof(need());
    else if (a == "-w") o.recFile = need();
    else if (a == "-G") o.dumpGraphs = true;
    else if (a == "-r") o.repeats = std::atoi(need());
    else if (a == "-B") o.budget = std::atof(need());
    else usage();
  }
  if (o.genN == 0 && o.inFile.empty()) usage();

  createCommunityMPIType();
  createEdgeMPIType();

  DistGraph *dg = nullptr;
  double tg0 = MPI_Wtime();
  if (o.genN > 0)
    generateInMemGraph(me, nprocs, dg, o.genN, o.randomEdgePercent, o.saveGraph);
  else
    loadDistGraphMPIIO(me, nprocs, 1, dg, o.inFile);
  double tg1 = MPI_Wtime();
  if (o.unitWeights) dg->getLocalGraph().setEdgeWeightstoOne();
  std::printf("HARNESS graph_seconds %.6f nv %lld ne %lld threads %d\n", tg1 - tg0,
              (long long)dg->getTotalNumVertices(),
              (long long)dg->getLocalGraph().getNumEdges(), omp_get_max_threads());

  if (!o.recFile.empty()) {
    g_rec = std::fopen(o.recFile.c_str(), "wb");
    if (!g_rec) { std::perror("record file"); return 1; }
    std::fwrite("VREC", 1, 4, g_rec);
    put<unsigned>(1);
  }

  // -r R: R timed runs of the level loop, each from a copy of the loaded graph
  // made before its clock starts (the loaded graph itself runs last); -B stops
  // before a run that would end past the budget, counted from the first run.
  const int repeats = o.repeats > 0 ? o.repeats : 1;
  double tStart = MPI_Wtime(), spent = 0.0;
  for (int r = 0; r < repeats; r++) {
    if (r > 0 && o.budget > 0.0) {
      const double elapsed = MPI_Wtime() - tStart;
      if (elapsed + spent / r > o.budget) {
        std::printf("HARNESS budget_stop after %d runs elapsed_s %.3f\n", r, elapsed);
        break;
      }
    }
    DistGraph *run = (r + 1 < repeats) ? new DistGraph(*dg) : dg;
    RunTotals t = runLevels(me, nprocs, run, o);
    spent += t.clustering + t.rebuild;
    std::printf("HARNESS total_clustering_s %.6f total_rebuild_s %.6f total_s %.6f levels %d iterations %d final_mod %.17g\n",
                t.clustering, t.rebuild, t.clustering + t.rebuild, t.levels, t.iterations,
                t.finalMod);
    std::fflush(stdout);
    if (g_rec) { put<int>(0); std::fclose(g_rec); g_rec = nullptr; }
    if (run == dg) dg = nullptr;  // the last run consumed the loaded graph
  }
  if (dg) delete dg;
  destroyCommunityMPIType();
  destroyEdgeMPIType();
  MPI_Finalize();
  return 0;
}
