// mtc_gpu.cpp -- the reference's GPU matcher classes (src/matchgpu.h:29-84)
// over the C ABI of include/mm_match.h.
#include <cassert>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <iostream>
#include <vector>

#include "mm_match.h"
#include "mtc/matchcpu.h"
#include "mtc/matchgpu.h"

using namespace std;

namespace {

// Read the next `count` values of the C library's rand() stream without
// consuming them.  glibc keeps rand()'s position inside its state array:
// initstate() parks the current position in the array's header word and
// returns the array, a copy of which continues the same stream under
// setstate(); switching back to the untouched original restores it.
bool peek_rand(uint32_t *out, int count)
{
    alignas(8) static thread_local char parking[128];
    char *orig = initstate(1u, parking, sizeof parking);
    if (!orig) return false;
    int32_t header;
    std::memcpy(&header, orig, sizeof header);
    static const int degree[5] = {0, 7, 15, 31, 63};
    const int type = header % 5;
    if (type < 0 || type > 4) {
        setstate(orig);
        return false;
    }
    const size_t words = (size_t)(degree[type] > 0 ? degree[type] : 1) + 1;
    alignas(8) char copy[4 * 64 + 8];
    std::memcpy(copy, orig, 4 * words);
    setstate(copy);
    for (int i = 0; i < count; ++i) out[i] = (uint32_t)rand();
    setstate(orig);
    return true;
}

uint32_t draw_rand(void *) { return (uint32_t)rand(); }

// MTC_RAND_READ_AHEAD=0 makes the classes take the portable path (seeds drawn
// from rand() one round at a time) even where the read-ahead works.
bool read_ahead_allowed()
{
    const char *e = std::getenv("MTC_RAND_READ_AHEAD");
    return !(e && e[0] == '0');
}

// The reference's MATCH_INTERMEDIATE_COUNT switch (src/matchcpu.h:26, used by
// saturate.sh): its fixed-round GPU matchers print the matching's weight and
// size after every round (src/matchgpu.cu:503-523, 701-712), "round<TAB>weight
// <TAB>size" on standard output, starting with "0<TAB>0<TAB>0".  The same
// switch at compile time, or MTC_MATCH_INTERMEDIATE_COUNT=1 at run time (the
// library is built once), gives the same lines here.
bool intermediate_count()
{
#ifdef MATCH_INTERMEDIATE_COUNT
    return true;
#else
    const char *e = std::getenv("MTC_MATCH_INTERMEDIATE_COUNT");
    return e && e[0] == '1';
#endif
}

// Between rounds of the host-stepped matching (mm_match_drawn calls `draw` as
// each round starts): the rounds done so far, their match values copied back.
struct RoundCounts {
    const mtc::Graph *graph;
    const int *dmatch;
    std::vector<int> *match;
    int done;
};

void print_counts(RoundCounts &rc)
{
    if (cudaDeviceSynchronize() != cudaSuccess ||
        (rc.graph->nrVertices > 0 && cudaMemcpy(&(*rc.match)[0], rc.dmatch, sizeof(int) * (size_t)rc.graph->nrVertices,
                                                cudaMemcpyDeviceToHost) != cudaSuccess)) {
        cerr << "Unable to retrieve data!" << endl;
        throw exception();
    }
    double weight = 0;
    long size = 0;
    mtc::GraphMatching::getWeight(weight, size, *rc.match, *rc.graph);
    cout << rc.done << "\t" << weight << "\t" << size << endl;
}

uint32_t draw_and_count(void *ctx)
{
    RoundCounts &rc = *(RoundCounts *)ctx;
    if (rc.done > 0) print_counts(rc);  // after the previous round
    ++rc.done;
    return (uint32_t)rand();
}

[[noreturn]] void fail(const char *what)
{
    cerr << what << ": " << mm_last_error() << endl;
    throw exception();
}

}  // namespace

namespace mtc {

GraphMatchingGPU::GraphMatchingGPU(const Graph &_graph, const int &_threadsPerBlock, const unsigned int &_selectBarrier)
    : GraphMatchingGPU(_graph, _threadsPerBlock, _selectBarrier, 0)
{
}

GraphMatchingGPU::GraphMatchingGPU(const Graph &_graph, const int &_threadsPerBlock, const unsigned int &_selectBarrier,
                                   int type)
    : GraphMatching(_graph),
      threadsPerBlock(_threadsPerBlock),
      selectBarrier(_selectBarrier),
      dneighbourRanges(nullptr),
      dneighbours(nullptr),
      dgraph(nullptr),
      dmatch(nullptr)
{
    const bool weighted = type == MM_TYPE_WEIGHTED || type == MM_TYPE_WEIGHTED_MAXIMAL ||
                          (type == 0 && graph.neighbourWeights.size() == graph.neighbours.size());
    if (weighted) assert(graph.neighbourWeights.size() == graph.neighbours.size());
    const float *w = weighted && !graph.neighbourWeights.empty() ? graph.neighbourWeights.data() : nullptr;
    if (mm_graph_create(graph.nrVertices, graph.neighbourRanges.empty() ? nullptr : &graph.neighbourRanges[0].x,
                        (long long)graph.neighbours.size(), graph.neighbours.empty() ? nullptr : graph.neighbours.data(),
                        w, -1, &dgraph) != MM_OK) {
        cerr << "Not enough memory on device to store this graph!" << endl;
        fail("mm_graph_create");
    }
    dneighbourRanges = (int2 *)mm_graph_device_ranges(dgraph);
    dneighbours = (int *)mm_graph_device_neighbours(dgraph);
    if (type != 0 && mm_graph_prepare(dgraph, type) != MM_OK) {
        mm_graph_destroy(dgraph);
        fail("Unable to prepare the graph on the device");
    }
    if (cudaMalloc(&dmatch, sizeof(int) * (size_t)(graph.nrVertices > 0 ? graph.nrVertices : 1)) != cudaSuccess) {
        mm_graph_destroy(dgraph);
        cerr << "Not enough memory on device!" << endl;
        throw exception();
    }
}

GraphMatchingGPU::~GraphMatchingGPU()
{
    cudaFree(dmatch);
    mm_graph_destroy(dgraph);
}

void GraphMatchingGPU::runMatching(vector<int> &match, cudaEvent_t &t1, cudaEvent_t &t2, int type) const
{
    assert((int)match.size() == graph.nrVertices);
    const int cap = mm_max_rounds(type);
    if (cap == NR_MATCH_ROUNDS && intermediate_count()) {
        // the rounds one at a time, the counts printed between them (the
        // reference prints inside its timed region too)
        cudaEventRecord(t1, 0);
        cudaEventSynchronize(t1);
        cout << "0\t0\t0" << endl;
        RoundCounts rc{&graph, dmatch, &match, 0};
        int rounds = 0;
        if (mm_match_drawn(dgraph, type, selectBarrier, draw_and_count, &rc, dmatch, &rounds, nullptr) != MM_OK)
            fail("A CUDA error occurred during the matching process");
        print_counts(rc);  // the last round; match now holds the result
        cudaEventRecord(t2, 0);
        cudaEventSynchronize(t2);
        return;
    }
    uint32_t seeds[256];
    if (!read_ahead_allowed() || !peek_rand(seeds, cap)) {
        // rand()'s state could not be read ahead (another C library, say): the
        // rounds run one at a time from the host, each drawing its rand() value
        // as it starts, exactly as the reference's loop does (src/matchgpu.cu:604-615)
        cudaEventRecord(t1, 0);
        cudaEventSynchronize(t1);
        int rounds = 0;
        if (mm_match_drawn(dgraph, type, selectBarrier, draw_rand, nullptr, dmatch, &rounds, nullptr) != MM_OK)
            fail("A CUDA error occurred during the matching process");
        cudaEventRecord(t2, 0);
        cudaEventSynchronize(t2);
        if (graph.nrVertices > 0 &&
            cudaMemcpy(&match[0], dmatch, sizeof(int) * (size_t)graph.nrVertices, cudaMemcpyDeviceToHost) !=
                cudaSuccess) {
            cerr << "Unable to retrieve data!" << endl;
            throw exception();
        }
        return;
    }

    cudaEventRecord(t1, 0);
    cudaEventSynchronize(t1);

    int rounds = 0;
    if (mm_match_device(dgraph, type, selectBarrier, seeds, cap, dmatch, &rounds, nullptr) != MM_OK)
        fail("A CUDA error occurred during the matching process");

    cudaEventRecord(t2, 0);
    cudaEventSynchronize(t2);

    // One rand() per executed round, as the reference's host loop draws them.
    for (int r = 0; r < rounds; ++r) {
        if ((uint32_t)rand() != seeds[r]) {
            cerr << "rand() stream changed while matching!" << endl;
            throw exception();
        }
    }

    if (graph.nrVertices > 0 &&
        cudaMemcpy(&match[0], dmatch, sizeof(int) * (size_t)graph.nrVertices, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cerr << "Unable to retrieve data!" << endl;
        throw exception();
    }
}

GraphMatchingGPURandom::GraphMatchingGPURandom(const Graph &_graph, const int &_nrThreads,
                                               const unsigned int &_selectBarrier)
    : GraphMatchingGPU(_graph, _nrThreads, _selectBarrier, MM_TYPE_RANDOM)
{
}

GraphMatchingGPURandom::~GraphMatchingGPURandom() {}

void GraphMatchingGPURandom::performMatching(vector<int> &match, cudaEvent_t &t1, cudaEvent_t &t2) const
{
    runMatching(match, t1, t2, MM_TYPE_RANDOM);
}

GraphMatchingGPURandomMaximal::GraphMatchingGPURandomMaximal(const Graph &_graph, const int &_nrThreads,
                                                             const unsigned int &_selectBarrier)
    : GraphMatchingGPU(_graph, _nrThreads, _selectBarrier, MM_TYPE_RANDOM_MAXIMAL)
{
}

GraphMatchingGPURandomMaximal::~GraphMatchingGPURandomMaximal() {}

void GraphMatchingGPURandomMaximal::performMatching(vector<int> &match, cudaEvent_t &t1, cudaEvent_t &t2) const
{
    runMatching(match, t1, t2, MM_TYPE_RANDOM_MAXIMAL);
}

GraphMatchingGPUWeighted::GraphMatchingGPUWeighted(const Graph &_graph, const int &_nrThreads,
                                                   const unsigned int &_selectBarrier)
    : GraphMatchingGPU(_graph, _nrThreads, _selectBarrier, MM_TYPE_WEIGHTED),
      dweights((float *)mm_graph_device_weights(dgraph))
{
}

GraphMatchingGPUWeighted::~GraphMatchingGPUWeighted() {}

void GraphMatchingGPUWeighted::performMatching(vector<int> &match, cudaEvent_t &t1, cudaEvent_t &t2) const
{
    runMatching(match, t1, t2, MM_TYPE_WEIGHTED);
}

GraphMatchingGPUWeightedMaximal::GraphMatchingGPUWeightedMaximal(const Graph &_graph, const int &_nrThreads,
                                                                 const unsigned int &_selectBarrier)
    : GraphMatchingGPU(_graph, _nrThreads, _selectBarrier, MM_TYPE_WEIGHTED_MAXIMAL),
      dweights((float *)mm_graph_device_weights(dgraph))
{
}

GraphMatchingGPUWeightedMaximal::~GraphMatchingGPUWeightedMaximal() {}

void GraphMatchingGPUWeightedMaximal::performMatching(vector<int> &match, cudaEvent_t &t1, cudaEvent_t &t2) const
{
    runMatching(match, t1, t2, MM_TYPE_WEIGHTED_MAXIMAL);
}

}  // namespace mtc
