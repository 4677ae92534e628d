// fileConvert for vite-b200: the command line of Vite's converter
// (converters/convert.cpp:102-281, flags :286-368) over the device text readers
// (vg_graph_read_text) and the device binary writer (vg_graph_write_vite). Same flags,
// same checks; the formats read on the device are plain edge lists (-s), SNAP (-n)
// and Matrix Market (-m), with -w (unit weights), -i (the file's weights), -r (the
// reference's random weights) and -z (one-based ids); the reference's other readers
// (-d DIMACS, -e METIS, -p Pajek, -u, -b, -x shards) are refused with a message.
#include <getopt.h>

#include <chrono>
#include <cstdlib>
#include <iostream>
#include <string>

#include "vite_b200.h"

namespace {

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

[[noreturn]] void fail(const std::string &msg) {
    std::cerr << msg << std::endl;
    std::exit(EXIT_FAILURE);
}

} // namespace

int main(int argc, char *argv[]) {
    std::string in, out, other;
    bool simple = false, snap = false;
    bool one = false, rnd = false, orig = false, oneBased = false;
    int nformats = 0;
    int ret;
    while ((ret = getopt(argc, argv, "f:o:md:upesnrix:zwb:")) != -1) {
        switch (ret) {
        case 'f': in.assign(optarg); break;
        case 'o': out.assign(optarg); break;
        case 'm': nformats++; break; // Matrix Market: the remaining case below
        case 's': simple = true; nformats++; break;
        case 'n': snap = true; nformats++; break;
        case 'p': other = "Pajek (-p)"; nformats++; break;
        case 'd': other = "DIMACS (-d)"; nformats++; break;
        case 'e': other = "METIS (-e)"; nformats++; break;
        case 'u': other = "-u"; nformats++; break;
        case 'b': other = "-b"; nformats++; break;
        case 'x': other = "sharded (-x)"; nformats++; break;
        case 'r': rnd = true; break;
        case 'i': orig = true; break;
        case 'z': oneBased = true; break;
        case 'w': one = true; break;
        default: fail("Unknown option");
        }
    }
    if (nformats == 0) fail("Must select a file format for the input file!");
    if (nformats > 1) fail("Must select a SINGLE file format for the input file!");
    if (in.empty()) fail("Must specify an input file name with -f");
    if (out.empty()) fail("Must specify an output file name with -o");
    if (!other.empty()) fail("The " + other + " format is not read on the device; use -s, -n or -m");

    vg_text_params p{};
    p.format = simple ? VG_TEXT_SIMPLE : snap ? VG_TEXT_SNAP : VG_TEXT_MATRIX_MARKET;
    // the reference's order of precedence (convert.cpp:146-190): -r, then -w, then -i
    p.weights = rnd ? VG_WEIGHTS_RANDOM : one ? VG_WEIGHTS_ONE : orig ? VG_WEIGHTS_ORIGINAL
                                                                 : VG_WEIGHTS_ABS;
    if (snap && p.weights != VG_WEIGHTS_RANDOM) p.weights = VG_WEIGHTS_ONE; // SNAP: 1 unless -r
    p.one_based = (simple && oneBased) ? 1 : 0;

    vg_ctx *ctx = nullptr;
    if (vg_ctx_create(0, 0, &ctx) != VG_OK) fail("cannot create a device context");
    const double t0 = now();
    vg_graph *g = nullptr;
    if (vg_graph_read_text(ctx, in.c_str(), &p, &g) != VG_OK)
        fail(std::string("Error reading ") + in + ": " + vg_last_error(ctx));
    int64_t nv = 0, ne = 0;
    vg_graph_info(g, &nv, &ne);
    std::cout << "Loaded graph from file: " << in << " (" << nv << " vertices, " << ne
              << " edges) in " << (now() - t0) << " s" << std::endl;
    const double t1 = now();
    if (vg_graph_write_vite(ctx, g, out.c_str()) != VG_OK)
        fail(std::string("Error writing ") + out + ": " + vg_last_error(ctx));
    std::cout << "Time writing binary file: " << (now() - t1) << std::endl;
    vg_graph_free(ctx, g);
    vg_ctx_destroy(ctx);
    return 0;
}
