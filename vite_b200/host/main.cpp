// graphClustering for vite-b200: the command line of Vite's main (main.cpp:609-770)
// and its phase loop (main.cpp:242-513) over the GPU entry points of vite_host.hpp.
// Same flags, checks, messages and per-level report; one rank, one GPU.
#include <getopt.h>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>

#include "vite_host.hpp"

namespace {

struct Options {
    std::string inputFileName, outputFileName, groundTruthFileName;
    bool coloring = false, vertexOrdering = false, runOnePhase = false, singleColorIter = false;
    int maxColors = 8;
    bool generateGraph = false, justProcessGraph = false;
    GraphElem numVerticesGenGraph = 0;
    GraphWeight randomEdgePercent = 0.0, defaultThreshold = CONVERGENCE_THRESHOLD;
    bool readBalanced = false, outputFiles = false, thresholdScaling = false;
    int ranksPerNode = 1;
    bool earlyTerm = false;
    int ETType = 0;
    GraphWeight ETDelta = 1.0;
    bool compareCommunities = false, isGroundTruthZeroBased = true;
};

[[noreturn]] void abort_run() { std::exit(157); } // the reference's MPI_Abort(-99) exit code

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void parse_color(const char *arg, Options &o) {
    std::stringstream ss(arg);
    std::string s;
    std::vector<std::string> args;
    while (std::getline(ss, s, ' ')) args.push_back(s);
    o.maxColors = std::stol(args[0]);
    if (args.size() > 1) {
        std::string b = args[1];
        std::transform(b.begin(), b.end(), b.begin(), ::tolower);
        o.singleColorIter = (b == "true" || b == "1");
    }
}

Options parse(int argc, char *argv[]) {
    Options o;
    int ret;
    while ((ret = getopt(argc, argv, "f:bc:od:r:t:a:ig:zpn:e:s:jh:")) != -1) {
        switch (ret) {
        case 'f': o.inputFileName.assign(optarg); break;
        case 'b': o.readBalanced = true; break;
        case 'c': parse_color(optarg, o); o.coloring = true; break;
        case 'o': o.outputFiles = true; break;
        case 'd': parse_color(optarg, o); o.vertexOrdering = true; break;
        case 'r': o.ranksPerNode = std::atoi(optarg); break;
        case 't': o.earlyTerm = true; o.ETType = std::atoi(optarg); break;
        case 'a': o.ETDelta = std::atof(optarg); break;
        case 'i': o.thresholdScaling = true; break;
        case 'g': o.groundTruthFileName.assign(optarg); o.compareCommunities = true; break;
        case 'z': o.isGroundTruthZeroBased = false; break;
        case 'p': o.runOnePhase = true; break;
        case 'n': o.generateGraph = true; o.numVerticesGenGraph = std::atol(optarg); break;
        case 'e': o.randomEdgePercent = std::atof(optarg); break;
        case 's': o.outputFileName.assign(optarg); break;
        case 'j': o.justProcessGraph = true; break;
        case 'h': o.defaultThreshold = std::atof(optarg); break;
        default:
            std::cerr << "Unknown option" << std::endl;
            abort_run();
        }
    }
    // the checks of main.cpp:710-768, with the same messages
    if (!o.generateGraph && !o.outputFileName.empty())
        std::cout << "Passing an output file has no effect for real-world graphs." << std::endl;
    if (o.earlyTerm && (o.ETType < 1 || o.ETType > 4)) {
        std::cerr << "early-term-type parameter is between 1-4 : -t 1 OR -t 2 OR -t 3 OR -t 4" << std::endl;
        abort_run();
    }
    if (o.earlyTerm && (o.ETType == 2 || o.ETType == 4) && (o.ETDelta > 1.0 || o.ETDelta < 0.0)) {
        std::cerr << "early-term-alpha must be between 0 and 1: -t 2 -a 0.5" << std::endl;
        abort_run();
    }
    if (!o.generateGraph && o.inputFileName.empty()) {
        std::cerr << "Must specify a binary file name with -f" << std::endl;
        abort_run();
    }
    if (o.compareCommunities && o.groundTruthFileName.empty()) {
        std::cerr << "Must specify a ground-truth file name with -g" << std::endl;
        abort_run();
    }
    if (o.coloring && o.vertexOrdering) {
        std::cerr << "Cannot turn on both coloring (-c) and vertex ordering (-d). Re-run using one of the options." << std::endl;
        abort_run();
    }
    if (o.runOnePhase && o.thresholdScaling) {
        std::cerr << "Cannot turn on threshold-cycling (-i) with a single phase run (-p). Re-run using one of the options." << std::endl;
        abort_run();
    }
    if (!o.generateGraph && o.randomEdgePercent > 0.0) {
        std::cerr << "Must specify -n <...> for graph generation first and then -p <...> to add random edges to it." << std::endl;
        abort_run();
    }
    return o;
}

// renumber by sorted id and compose with earlier levels (main.cpp:381-425)
void compose(std::vector<GraphElem> &commAll, const CommunityVector &cvect, int phase) {
    std::vector<GraphElem> ren(cvect);
    std::sort(ren.begin(), ren.end());
    std::map<GraphElem, GraphElem> kval;
    GraphElem nidx = 0;
    for (GraphElem x : ren)
        if (kval.find(x) == kval.end()) kval.emplace(x, nidx++);
    std::vector<GraphElem> all(cvect.size());
    for (size_t c = 0; c < cvect.size(); c++) all[c] = kval[cvect[c]];
    if (phase == 0)
        std::copy(all.begin(), all.end(), commAll.begin());
    else
        for (auto &p : commAll) p = all[p];
}

} // namespace

int main(int argc, char *argv[]) {
    const Options o = parse(argc, argv);
    const int me = 0, nprocs = 1;
    // the ground truth, in LFR's "vertex community" format (main.cpp:119-138)
    std::vector<GraphElem> commGroundTruth;
    if (o.compareCommunities) {
        const double tg1 = now();
        loadGroundTruthFile(commGroundTruth, o.groundTruthFileName, o.isGroundTruthZeroBased);
        std::cout << "Time taken to load ground truth file (" << o.groundTruthFileName
                  << "): " << (now() - tg1) << std::endl;
    }
    const double td0 = now();
    DistGraph *dg = nullptr;
    if (o.generateGraph)
        generateInMemGraph(me, nprocs, dg, o.numVerticesGenGraph, o.randomEdgePercent, o.outputFileName);
    else {
        std::string f = o.inputFileName;
        if (o.readBalanced) loadDistGraphMPIIOBalanced(me, nprocs, o.ranksPerNode, dg, f);
        else loadDistGraphMPIIO(me, nprocs, o.ranksPerNode, dg, f);
    }
    const double td1 = now();
    std::cout << "Number of vertices: " << dg->getTotalNumVertices() << std::endl;
    std::cout << "Number of edges: " << dg->getTotalNumEdges() << std::endl;
    std::cout << "Time to create distributed graph: " << (td1 - td0) << std::endl;
    if (o.justProcessGraph) {
        std::cout << "Option to just process the graph is turned on, so exiting without invoking community detection." << std::endl;
        delete dg;
        return 0;
    }

    GraphWeight currMod = -1.0, prevMod = -1.0, threshold = o.defaultThreshold;
    double total = td1 - td0, ctime = 0.0;
    int phase = 0, short_phase = 0, iters = 0, tot_iters = 0;
    ColorElem numColors = 0;
    ColorVector colors;
    CommunityVector cvect;
    std::vector<GraphElem> ssizes, rsizes, svdata, rvdata;
    size_t ssz = 0, rsz = 0;
    const GraphElem nv = dg->getTotalNumVertices();
    std::vector<GraphElem> commAll;
    const bool keepComm = o.outputFiles || o.compareCommunities; // main.cpp:236
    if (keepComm) commAll.assign(nv, -1);
    GraphElem teps = 0;
    const bool et = o.earlyTerm;
    const int ty = o.ETType;

    while (true) {
        double ptotal = 0.0;
        if (o.thresholdScaling && !o.runOnePhase) {
            if (short_phase > 12) short_phase = 0;
            if (short_phase <= 2) threshold = 1.0E-3;
            else if (short_phase <= 6) threshold = 1.0E-4;
            else if (short_phase <= 9) threshold = 1.0E-5;
            else threshold = o.defaultThreshold;
        } else
            threshold = o.defaultThreshold;
        double t1 = now();
        if ((o.coloring || o.vertexOrdering) && phase == 0) {
            numColors = distColoringMultiHashMinMax(me, nprocs, *dg, colors, (o.maxColors / 2), MAX_COVG, o.singleColorIter);
            std::cout << "Number of colors (2*nHash): " << numColors << std::endl;
            const double t0c = now();
            std::cout << "Coloring Time: " << t0c - t1 << std::endl;
            if (o.coloring) {
                if (et && ty == 1) currMod = distLouvainMethodWithColoring(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, true);
                else if (et && ty == 2) currMod = distLouvainMethodWithColoring(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, o.ETDelta, true);
                else if (et && ty == 3) currMod = distLouvainMethodWithColoring(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, false);
                else if (et && ty == 4) currMod = distLouvainMethodWithColoring(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, o.ETDelta, false);
                else currMod = distLouvainMethodWithColoring(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters);
            } else {
                if (et && ty == 1) currMod = distLouvainMethodVertexOrder(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, true);
                else if (et && ty == 2) currMod = distLouvainMethodVertexOrder(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, o.ETDelta, true);
                else if (et && ty == 3) currMod = distLouvainMethodVertexOrder(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, false);
                else if (et && ty == 4) currMod = distLouvainMethodVertexOrder(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, o.ETDelta, false);
                else currMod = distLouvainMethodVertexOrder(me, nprocs, *dg, numColors + 1, colors, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters);
            }
        } else {
            if (et && ty == 1) currMod = distLouvainMethod(me, nprocs, *dg, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, true);
            else if (et && ty == 2) currMod = distLouvainMethod(me, nprocs, *dg, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, o.ETDelta, true);
            else if (et && ty == 3) currMod = distLouvainMethod(me, nprocs, *dg, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, false);
            else if (et && ty == 4) currMod = distLouvainMethod(me, nprocs, *dg, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters, o.ETDelta, false);
            else currMod = distLouvainMethod(me, nprocs, *dg, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, threshold, iters);
        }
        const double t0 = now();
        tot_iters += iters;
        ptotal += t0 - t1;
        ctime += t0 - t1;
        if ((currMod - prevMod) > threshold) {
            if (keepComm) compose(commAll, cvect, phase);
            if (!o.runOnePhase) {
                const double t3 = now();
                distbuildNextLevelGraph(nprocs, me, dg, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect);
                const double t2 = now();
                std::cout << "**************************" << std::endl;
                std::cout << "Rebuild Time: " << t2 - t3 << std::endl;
                ptotal += t2 - t3;
            }
        } else {
            if (o.thresholdScaling && !o.runOnePhase && phase < 10) {
                const double tx1 = now();
                currMod = distLouvainMethod(me, nprocs, *dg, ssz, rsz, ssizes, rsizes, svdata, rvdata, cvect, currMod, 1.0E-6, iters);
                ptotal += now() - tx1;
            }
            break;
        }
        // TEPS as the reference counts it: next level's edges x cumulative iterations (main.cpp:466)
        teps += dg->getTotalNumEdges() * tot_iters;
        std::cout.precision(6);
        std::cout << "Level " << phase << ", Modularity: " << currMod << ", Clustering time: " << t0 - t1
                  << ", Iterations: " << tot_iters << std::endl;
        prevMod = currMod;
        currMod = -1.0;
        std::cout << "Phase Total time: " << ptotal << std::endl;
        total += ptotal;
        phase++;
        if (o.runOnePhase) {
            std::cout << "Exiting at the end of first phase." << std::endl;
            break;
        }
        if (o.thresholdScaling && !o.runOnePhase) short_phase++;
        if (phase == TERMINATION_PHASE_COUNT || tot_iters > 10000) {
            std::cout << "Program ran for " << TERMINATION_PHASE_COUNT << " phases or 10K iterations, exiting..." << std::endl;
            break;
        }
    }
    std::cout << "-------------------------------------------------------" << std::endl;
    std::cout << "Average total time (secs.): " << total << std::endl;
    std::cout << "Average time for clustering (secs.): " << ctime << std::endl;
    std::cout << "Convergence threshold (for fixed-threshold workloads): " << threshold << std::endl;
    std::cout << "MODS (final modularity * average clustering time): " << currMod * ctime << std::endl;
    std::cout << "TEPS (traversed edges across clustering iterations): " << (double)teps / ctime << std::endl;
    std::cout << "-------------------------------------------------------" << std::endl;
    if (o.outputFiles) {
        const std::string outFileName = o.inputFileName + ".communities";
        std::ofstream ofs(outFileName);
        if (!ofs) {
            std::cerr << "Error creating community file: " << outFileName << std::endl;
            return EXIT_FAILURE;
        }
        for (GraphElem i = 0; i < nv; i++) ofs << commAll[i] << "\n";
        std::cout << "Saved community information (" << commAll.size() << " vertices)  on file: "
                  << outFileName << std::endl;
    }
    // compare the computed communities with the ground truth (main.cpp:574-581)
    if (o.compareCommunities) compare_communities(commGroundTruth, commAll);
    delete dg;
    return 0;
}
