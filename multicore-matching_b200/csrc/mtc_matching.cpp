// mtc_matching.cpp -- the mtc::GraphMatching base of include/mtc/matchcpu.h.
//
// initialMatching, getWeight and testMatching with the reference's semantics
// and output (src/matchcpu.cu:32-246).
#include <algorithm>
#include <cassert>
#include <iostream>
#include <vector>

#include "mtc/matchcpu.h"

using namespace std;

namespace mtc {

GraphMatching::GraphMatching(const Graph &_graph) : graph(_graph) {}

GraphMatching::~GraphMatching() {}

vector<int> GraphMatching::initialMatching() const { return vector<int>(graph.nrVertices, 0); }

// Size = matched vertices whose partner appears in their own list; weight =
// half the sum of the weights of those entries (matchcpu.cu:64-97).
void GraphMatching::getWeight(double &_weight, long &_size, const vector<int> &match, const Graph &graph)
{
    assert((int)match.size() == graph.nrVertices);
    double weight = 0.0;
    long size = 0;
    for (int i = 0; i < graph.nrVertices; ++i) {
        const int m = match[i];
        if (!isMatched(m)) continue;
        const int2 r = graph.neighbourRanges[i];
        for (int j = r.x; j < r.y; ++j) {
            if (match[graph.neighbours[j]] == m) {
                weight += (double)graph.neighbourWeights[j];
                size += 1;
                break;
            }
        }
    }
    _weight = weight / 2.0;
    _size = size;
}

// Validity check with the reference's counting (matchcpu.cu:127-246): vertices
// ordered by match value (unmatched first); each matched value must be held by
// exactly two vertices that are neighbours of each other.  Prints the same
// summary; maximality (unmatched vertices with an unmatched neighbour) is
// reported, not enforced.
bool GraphMatching::testMatching(const vector<int> &match, const Graph &graph)
{
    if ((int)match.size() != graph.nrVertices) {
        cerr << "Incompatible matching size!" << endl;
        return false;
    }
    vector<int> order(graph.nrVertices);
    for (int i = 0; i < graph.nrVertices; ++i) order[i] = i;
    sort(order.begin(), order.end(), [&match](int a, int b) {
        const bool ma = isMatched(match[a]), mb = isMatched(match[b]);
        if (ma != mb) return mb;
        return match[a] < match[b];
    });
    size_t k = 0;
    while (k < order.size() && !isMatched(match[order[k]])) ++k;
    int under = 0, multi = 0, invalid = 0;
    while (k < order.size()) {
        const int i1 = order[k];
        const int m = match[i1];
        ++k;
        if (k == order.size()) {
            ++under;
            continue;
        }
        const int i2 = order[k];
        ++k;
        if (match[i2] != m) {
            ++under;
            continue;
        }
        bool f1 = false, f2 = false;
        const int2 r1 = graph.neighbourRanges[i1], r2 = graph.neighbourRanges[i2];
        for (int j = r1.x; j < r1.y && !f1; ++j) f1 = graph.neighbours[j] == i2;
        for (int j = r2.x; j < r2.y && !f2; ++j) f2 = graph.neighbours[j] == i1;
        if (!f1 || !f2) ++invalid;
        while (k < order.size() && match[order[k]] == m) {
            ++multi;
            ++k;
        }
    }
    int matchable = 0;
    for (int i = 0; i < (int)match.size(); ++i) {
        if (isMatched(match[i])) continue;
        const int2 r = graph.neighbourRanges[i];
        int free_nbrs = 0;
        for (int j = r.x; j < r.y; ++j) {
            const int u = graph.neighbours[j];
            if (u != i && !isMatched(match[u])) ++free_nbrs;
        }
        if (free_nbrs > 0) ++matchable;
    }
    cout << "Verified a matching of " << match.size() << " vertices, of these" << endl;
    cout << "    " << under << " were matched to themselves," << endl;
    cout << "    " << multi << " were matched to more than one vertex," << endl;
    cout << "    " << invalid << " were not matched to a neighbour," << endl;
    cout << "    " << matchable << " can still be matched." << endl;
    return under == 0 && multi == 0 && invalid == 0;
}

}  // namespace mtc
