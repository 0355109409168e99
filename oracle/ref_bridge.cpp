/*
 * ref_bridge.cpp -- C entry points around the reference's OWN CPU matchers.
 *
 * TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile together with the
 * unmodified reference sources src/graph.cu, src/matchcpu.cu and
 * src/matchtbb.cu (read where they lie, never copied) into
 * oracle/_ref/libmmref.so.  The same bridge is linked into
 * oracle/_ref/libmmref20.so against ref_tbb20.cpp, the TBB matchers with the
 * round cap at NR_MATCH_ROUNDS, which is the fixed-round loop of the GPU types
 * 6 and 8 (matchgpu.cu:507, 705).
 *
 * Used as (1) the pin for oracle/mm_oracle.c and the golden fixtures and (2)
 * the "reference" CPU baseline that bench.py times on the host cores.
 */
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <cstdio>
#include <string>
#include <vector>

#include "graph.h"
#include "matchcpu.h"
#include "matchtbb.h"
#ifdef _OPENMP
#include <omp.h>
#endif

/* The reference matchers bracket their work with cudaEventRecord /
 * cudaEventSynchronize (matchcpu.cu:266-302, matchtbb.cu:511-553).  The oracle
 * has no GPU, so the two calls resolve to these no-ops (hidden, so they bind
 * only inside this library). */
extern "C" __attribute__((visibility("hidden"))) cudaError_t cudaEventRecord(cudaEvent_t, cudaStream_t)
{
    return cudaSuccess;
}
extern "C" __attribute__((visibility("hidden"))) cudaError_t cudaEventSynchronize(cudaEvent_t)
{
    return cudaSuccess;
}

#define MMREF_API extern "C" __attribute__((visibility("default")))

static void build_graph(mtc::Graph &g, int n, const int *ranges, long long nnz, const int *nbrs,
                        const float *w, bool with_edges)
{
    g.clear();
    g.nrVertices = n;
    g.neighbourRanges.resize(n);
    for (int v = 0; v < n; ++v) g.neighbourRanges[v] = make_int2(ranges[2 * v], ranges[2 * v + 1]);
    g.neighbours.assign(nbrs, nbrs + nnz);
    if (w) g.neighbourWeights.assign(w, w + nnz);
    else g.neighbourWeights.assign((size_t)nnz, 1.0f);
    /* Edge list as readMETIS builds it (graph.cu:485-497): one entry per i > j. */
    if (with_edges) {
        for (int v = 0; v < n; ++v)
            for (int j = ranges[2 * v]; j < ranges[2 * v + 1]; ++j)
                if (v > nbrs[j]) g.edges.push_back(mtc::Edge(v, nbrs[j], g.neighbourWeights[j]));
    }
    g.nrEdges = (int)g.edges.size();
}

/*
 * Run reference matcher `type` (0 CPU random, 4 CPU weighted, 5 CPU weighted
 * edge, 10 TBB random, 11 TBB weighted; bin/match.cpp:136-158) after
 * srand(seed), as bin/match.cpp:382-420 does.  Writes match_out[n], the
 * wall-clock ms of performMatching and the next rand() value (which tells how
 * many values the matcher consumed).  Returns 0 on success.
 */
MMREF_API int mmref_run(int type, int n, const int *ranges, long long nnz, const int *nbrs,
                        const float *w, unsigned barrier, unsigned seed, int nthreads,
                        int *match_out, double *ms_out, unsigned *next_rand_out)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    mtc::Graph g;
    build_graph(g, n, ranges, nnz, nbrs, w, type == 5);
    mtc::GraphMatching *m = nullptr;
    switch (type) {
    case 0: m = new mtc::GraphMatchingCPURandom(g); break;
    case 4: m = new mtc::GraphMatchingCPUWeighted(g); break;
    case 5: m = new mtc::GraphMatchingCPUWeightedEdge(g); break;
    case 10: m = new mtc::GraphMatchingTBBRandom(g, barrier); break;
    case 11: m = new mtc::GraphMatchingTBBWeighted(g, barrier); break;
    default: return 1;
    }
    srand(seed);
    std::vector<int> match = m->initialMatching();
    cudaEvent_t t1 = nullptr, t2 = nullptr;
    const auto a = std::chrono::steady_clock::now();
    m->performMatching(match, t1, t2);
    const auto b = std::chrono::steady_clock::now();
    if (next_rand_out) *next_rand_out = (unsigned)rand();
    if (ms_out) *ms_out = std::chrono::duration<double, std::milli>(b - a).count();
    std::memcpy(match_out, match.data(), sizeof(int) * (size_t)n);
    delete m;
    return 0;
}

/* GraphMatching::getWeight and testMatching of the reference (matchcpu.cu:64-246). */
MMREF_API int mmref_check(int n, const int *ranges, long long nnz, const int *nbrs, const float *w,
                          const int *match, double *weight, long long *size)
{
    mtc::Graph g;
    build_graph(g, n, ranges, nnz, nbrs, w, false);
    std::vector<int> m(match, match + n);
    double wt = 0.0;
    long sz = 0;
    mtc::GraphMatching::getWeight(wt, sz, m, g);
    *weight = wt;
    *size = sz;
    return mtc::GraphMatching::testMatching(m, g) ? 1 : 0;
}

/*
 * testMatching's four counters (matchcpu.cu:239-243), read from the lines it
 * prints: matched to themselves, to more than one vertex, not to a
 * neighbour, can still be matched.  Returns its verdict.
 */
MMREF_API int mmref_check_counts(int n, const int *ranges, long long nnz, const int *nbrs, const float *w,
                                 const int *match, long long counts[4])
{
    mtc::Graph g;
    build_graph(g, n, ranges, nnz, nbrs, w, false);
    std::vector<int> m(match, match + n);
    std::ostringstream text;
    std::streambuf *saved = std::cout.rdbuf(text.rdbuf());
    const bool ok = mtc::GraphMatching::testMatching(m, g);
    std::cout.rdbuf(saved);
    std::istringstream lines(text.str());
    std::string line;
    int k = 0;
    while (std::getline(lines, line) && k < 4) {
        long long v = 0;
        if (line.rfind("    ", 0) == 0 && std::sscanf(line.c_str(), " %lld", &v) == 1) counts[k++] = v;
    }
    return ok ? 1 : 0;
}

/*
 * Read a graph file with the reference's own readers (graph.cu:86-511) and
 * copy its CSR out.  Call with null arrays first to get the sizes.
 */
MMREF_API int mmref_read(const char *path, int is_mtx, int *n, int *edges, long long *nnz, int *ranges, int *nbrs,
                         float *w)
{
    mtc::Graph g;
    std::ifstream f(path);
    if (!f.good()) return 1;
    try {
        if (is_mtx) g.readMatrixMarket(f);
        else g.readMETIS(f);
    } catch (std::exception &) {
        return 2;
    }
    *n = g.nrVertices;
    *edges = g.nrEdges;
    *nnz = (long long)g.neighbours.size();
    if (ranges)
        for (int v = 0; v < g.nrVertices; ++v) {
            ranges[2 * v] = g.neighbourRanges[v].x;
            ranges[2 * v + 1] = g.neighbourRanges[v].y;
        }
    if (nbrs && !g.neighbours.empty()) std::memcpy(nbrs, g.neighbours.data(), sizeof(int) * g.neighbours.size());
    if (w && !g.neighbourWeights.empty())
        std::memcpy(w, g.neighbourWeights.data(), sizeof(float) * g.neighbourWeights.size());
    return 0;
}

/*
 * The reference CLI's per-type loop (bin/match.cpp:380-420) with one of its
 * CPU/TBB matchers: read `path`, srand(seed), then `reps` times: optional
 * Graph::random_shuffle, match.  out receives reps x n match arrays; returns
 * the next rand() value through next_rand.
 */
MMREF_API int mmref_cli(const char *path, int is_mtx, int type, unsigned barrier, unsigned seed, int shuffle, int reps,
                        int *out, unsigned *next_rand)
{
    mtc::Graph g;
    std::ifstream f(path);
    if (!f.good()) return 1;
    try {
        if (is_mtx) g.readMatrixMarket(f);
        else g.readMETIS(f);
    } catch (std::exception &) {
        return 2;
    }
    mtc::Graph g2 = g;
    srand(seed);
    for (int k = 0; k < reps; ++k) {
        if (shuffle) g2.random_shuffle();
        mtc::GraphMatching *m = nullptr;
        switch (type) {
        case 0: m = new mtc::GraphMatchingCPURandom(g2); break;
        case 4: m = new mtc::GraphMatchingCPUWeighted(g2); break;
        case 10: m = new mtc::GraphMatchingTBBRandom(g2, barrier); break;
        case 11: m = new mtc::GraphMatchingTBBWeighted(g2, barrier); break;
        default: return 3;
        }
        std::vector<int> match = m->initialMatching();
        cudaEvent_t t1 = nullptr, t2 = nullptr;
        m->performMatching(match, t1, t2);
        std::memcpy(out + (size_t)k * g.nrVertices, match.data(), sizeof(int) * (size_t)g.nrVertices);
        delete m;
    }
    *next_rand = (unsigned)rand();
    return 0;
}

/*
 * srand(seed), then `reps` calls of the reference's Graph::random_shuffle
 * (graph.cu:513-548) on the graph read from `path`.  ranges_out[2n] and
 * nbrs_out[nnz] receive the final CSR; next_rand the next rand() value.
 */
MMREF_API int mmref_shuffle(const char *path, int is_mtx, unsigned seed, int reps, int *ranges_out, int *nbrs_out,
                            unsigned *next_rand)
{
    mtc::Graph g;
    std::ifstream f(path);
    if (!f.good()) return 1;
    try {
        if (is_mtx) g.readMatrixMarket(f);
        else g.readMETIS(f);
    } catch (std::exception &) {
        return 2;
    }
    srand(seed);
    for (int k = 0; k < reps; ++k) g.random_shuffle();
    for (int v = 0; v < g.nrVertices; ++v) {
        ranges_out[2 * v] = g.neighbourRanges[v].x;
        ranges_out[2 * v + 1] = g.neighbourRanges[v].y;
    }
    if (!g.neighbours.empty()) std::memcpy(nbrs_out, g.neighbours.data(), sizeof(int) * g.neighbours.size());
    *next_rand = (unsigned)rand();
    return 0;
}
