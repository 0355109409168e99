// mtc_harness.cpp -- drives the drop-in C++ classes the way the reference's
// CLI does (bin/match.cpp:363-470): read a METIS or MatrixMarket file, srand,
// per repetition optionally random_shuffle, construct a GPU matcher,
// initialMatching + performMatching, testMatching, getWeight.  Built and run
// by tests/test_mtc_cpp.py.
//
//   mtc_harness dump    <file> <out.bin>                   CSR as read
//   mtc_harness shuffle <file> <seed> <reps> <out.bin>     CSR after srand + reps shuffles
//   mtc_harness match <file> <type> <seed> <shuffle> <reps> <out.bin>
//
// out.bin (match): reps x n int32 match arrays; stdout: one JSON line.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "graph.h"
#include "matchcpu.h"
#include "matchgpu.h"

using namespace mtc;

static bool read_graph(Graph &g, const std::string &path)
{
    std::ifstream f(path.c_str());
    if (!f.good()) return false;
    if (path.find(".mtx") != std::string::npos) g.readMatrixMarket(f);
    else g.readMETIS(f);
    return true;
}

static GraphMatching *make(const Graph &g, int type, unsigned barrier)
{
    if (type == 6) return new GraphMatchingGPURandom(g, 256, barrier);
    if (type == 7) return new GraphMatchingGPURandomMaximal(g, 256, barrier);
    if (type == 8) return new GraphMatchingGPUWeighted(g, 256, barrier);
    if (type == 9) return new GraphMatchingGPUWeightedMaximal(g, 256, barrier);
    return nullptr;
}

int main(int argc, char **argv)
{
    if (argc < 4) return 2;
    const std::string mode = argv[1];
    Graph graph;
    try {
        if (!read_graph(graph, argv[2])) return 3;
    } catch (std::exception &) {
        std::printf("{\"read_error\": true}\n");
        return 4;
    }
    if (mode == "shuffle") {
        if (argc < 6) return 2;
        srand((unsigned)std::strtoul(argv[3], nullptr, 10));
        for (int k = std::atoi(argv[4]); k > 0; --k) graph.random_shuffle();
    }
    if (mode == "dump" || mode == "shuffle") {
        FILE *out = std::fopen(mode == "dump" ? argv[3] : argv[5], "wb");
        const long long nnz = (long long)graph.neighbours.size();
        std::fwrite(&graph.nrVertices, sizeof(int), 1, out);
        std::fwrite(&graph.nrEdges, sizeof(int), 1, out);
        std::fwrite(&nnz, sizeof(long long), 1, out);
        if (graph.nrVertices) std::fwrite(&graph.neighbourRanges[0], sizeof(int2), graph.nrVertices, out);
        if (nnz) {
            std::fwrite(&graph.neighbours[0], sizeof(int), nnz, out);
            std::fwrite(&graph.neighbourWeights[0], sizeof(float), nnz, out);
        }
        std::fclose(out);
        std::printf("{\"n\": %d, \"edges\": %d, \"nnz\": %lld, \"empty\": %s, \"next_rand\": %u}\n", graph.nrVertices,
                    graph.nrEdges, nnz, graph.empty() ? "true" : "false", (unsigned)rand());
        return 0;
    }
    if (mode != "match" || argc < 8) return 2;
    const int type = std::atoi(argv[3]);
    const unsigned seed = (unsigned)std::strtoul(argv[4], nullptr, 10);
    const bool shuffle = std::atoi(argv[5]) != 0;
    const int reps = std::atoi(argv[6]);
    const unsigned barrier = 0x88B81733u;
    FILE *out = std::fopen(argv[7], "wb");
    Graph graph2 = graph;
    srand(seed);
    std::string json = "{\"runs\": [";
    for (int k = 0; k < reps; ++k) {
        if (shuffle) graph2.random_shuffle();
        cudaEvent_t t0, t1, t2, t3;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventCreate(&t2);
        cudaEventCreate(&t3);
        cudaEventRecord(t0, 0);
        cudaEventSynchronize(t0);
        std::vector<int> match;
        try {
            GraphMatching *m = make(graph2, type, barrier);
            match = m->initialMatching();
            m->performMatching(match, t1, t2);
            delete m;
        } catch (std::exception &) {
            std::printf("{\"match_error\": true}\n");
            return 5;
        }
        cudaEventRecord(t3, 0);
        cudaEventSynchronize(t3);
        float total = 0.f, mt = 0.f;
        cudaEventElapsedTime(&total, t0, t3);
        cudaEventElapsedTime(&mt, t1, t2);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        cudaEventDestroy(t2);
        cudaEventDestroy(t3);
        std::streambuf *keep = std::cout.rdbuf(nullptr);  // testMatching prints a summary
        const bool valid = GraphMatching::testMatching(match, graph2);
        std::cout.rdbuf(keep);
        double weight = 0.0;
        long size = 0;
        GraphMatching::getWeight(weight, size, match, graph2);
        if (!match.empty()) std::fwrite(&match[0], sizeof(int), match.size(), out);
        char buf[256];
        std::snprintf(buf, sizeof buf, "%s{\"valid\": %s, \"weight\": %.17g, \"size\": %ld, \"total_ms\": %.4f, \"match_ms\": %.4f}",
                      k ? ", " : "", valid ? "true" : "false", weight, size, total, mt);
        json += buf;
    }
    std::fclose(out);
    char tail[64];
    std::snprintf(tail, sizeof tail, "], \"next_rand\": %u}", (unsigned)rand());
    std::printf("%s%s\n", json.c_str(), tail);
    return 0;
}
