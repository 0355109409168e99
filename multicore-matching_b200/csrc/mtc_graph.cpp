// mtc_graph.cpp -- mtc::Edge and mtc::Graph of include/mtc/graph.h.
//
// Same observable behaviour as the reference's src/graph.cu: the readers
// produce the same CSR (entry order included), warnings and exceptions, so
// matchings computed on file inputs agree with the reference's.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <exception>
#include <iostream>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "mtc/graph.h"

using namespace std;

namespace mtc {

Edge::Edge() {}

Edge::Edge(const int &_x, const int &_y, const float &_w) : x(_x), y(_y), w(_w) {}

Edge::~Edge() {}

Graph::Graph() : nrVertices(0), nrVertexWeights(0), nrEdges(0) {}

Graph::~Graph() {}

// graph.cu:67-72
bool Graph::empty() const
{
    return nrVertices == 0 || nrEdges == 0 || neighbours.empty() || neighbourRanges.empty() || edges.empty();
}

void Graph::clear()
{
    nrVertices = 0;
    nrVertexWeights = 0;
    nrEdges = 0;
    neighbourRanges.clear();
    vertexWeights.clear();
    neighbours.clear();
    neighbourWeights.clear();
    edges.clear();
}

namespace {

[[noreturn]] void fail(const char *msg)
{
    cerr << msg << endl;
    throw exception();
}

void trim_front(string &line)
{
    size_t k = 0;
    while (k < line.size() && isspace((unsigned char)line[k])) ++k;
    line.erase(0, k);
}

}  // namespace

// MatrixMarket reader (graph.cu:86-349).  Only symmetric layouts are accepted;
// entries strictly below the diagonal become edges with weight |value|; the
// CSR lists each edge twice, in edge order.
istream &Graph::readMatrixMarket(istream &in)
{
    enum { NoStorage, Coordinate, Array } storage = NoStorage;
    enum { NoData, Real, Complex, Integer, Pattern } data = NoData;
    enum { NoLayout, General, Symmetric, Skew, Hermitean } layout = NoLayout;
    bool have_dims = false;
    int cur_row = 1, cur_col = 1, rows = 0, cols = 0, entries = 0;

    clear();

    while (in.good()) {
        string line;
        getline(in, line);
        trim_front(line);
        if (line.length() < 2) continue;
        istringstream sline(line);
        if (line[0] == '%' && line[1] == '%') {
            while (sline.good()) {
                string word;
                sline >> word;
                if (word == "%%MatrixMarket" || word == "matrix") {
                } else if (word == "coordinate") {
                    storage = Coordinate;
                } else if (word == "array") {
                    storage = Array;
                } else if (word == "float" || word == "real" || word == "double") {
                    data = Real;
                } else if (word == "complex") {
                    data = Complex;
                } else if (word == "int" || word == "integer") {
                    data = Integer;
                } else if (word == "pattern") {
                    data = Pattern;
                } else if (word == "general") {
                    layout = General;
                } else if (word == "symmetric") {
                    layout = Symmetric;
                } else if (word == "skew" || word == "skew-symmetric") {
                    layout = Skew;
                } else if (word == "hermitean" || word == "Hermitean") {
                    layout = Hermitean;
                } else {
                    cerr << "Unknown Matrix Market header tag '" << word << "'!" << endl;
                }
            }
            continue;
        }
        if (line[0] == '%') continue;

        if (storage == NoStorage || data == NoData || layout == NoLayout) fail("Incomplete Matrix Market header!");
        if (layout == General) fail("Matrix with unsymmetric nonzero pattern!");
        if (have_dims && (rows == 0 || cols == 0 || entries == 0)) fail("Invalid Matrix Market dimensions!");

        if (!have_dims) {
            sline >> rows;
            sline >> cols;
            if (layout != General && rows != cols) fail("Non-square matrix with symmetry flags!");
            if (storage == Coordinate) sline >> entries;
            else entries = rows * cols;
            if (entries == 0) fail("No Matrix Market data!");
            nrVertices = rows;
            nrVertexWeights = 0;
            nrEdges = 0;
            vertexWeights.clear();
            neighbourRanges.assign(nrVertices, make_int2(0, 0));
            neighbours.clear();
            neighbourWeights.clear();
            edges.clear();
            edges.reserve(entries);
            have_dims = true;
            continue;
        }

        int row, col;
        double re = 0.0, im = 0.0;
        if (storage == Coordinate) {
            sline >> row;
            sline >> col;
            if (row < 1 || row > rows || col < 1 || col > cols) {
                cerr << "Invalid row and/or column index " << row << ", " << col << "!" << endl;
                throw exception();
            }
            --row;
            --col;
            if (data != Pattern) {
                sline >> re;
                if (data == Complex) sline >> im;
                else im = 0.0;
            } else {
                re = 1.0;
                im = 0.0;
            }
        } else {
            // dense column-major walk, with the reference's row wrap (graph.cu:275-279)
            row = cur_row - 1;
            col = cur_col - 1;
            sline >> re;
            if (data == Complex) sline >> im;
            else im = 0.0;
            if (++cur_row >= rows) {
                cur_row = 1;
                cur_col++;
            }
        }
        if (row > col) edges.push_back(Edge(row, col, (float)sqrt(re * re + im * im)));
    }

    // CSR: count, offsets, fill in edge order (graph.cu:293-324)
    neighbours.assign(2 * edges.size(), 0);
    neighbourWeights.assign(2 * edges.size(), 1.0f);
    nrEdges = (int)edges.size();
    if (nrVertices > 0) {
        for (const Edge &e : edges) {
            neighbourRanges[e.x].y++;
            neighbourRanges[e.y].y++;
        }
        for (int i = 1; i < nrVertices; ++i) {
            neighbourRanges[i].x = neighbourRanges[i - 1].x + neighbourRanges[i - 1].y;
            neighbourRanges[i - 1].y = neighbourRanges[i - 1].x;
        }
        neighbourRanges[nrVertices - 1].y = neighbourRanges[nrVertices - 1].x;
        for (const Edge &e : edges) {
            neighbours[neighbourRanges[e.x].y] = e.y;
            neighbourWeights[neighbourRanges[e.x].y] = e.w;
            neighbourRanges[e.x].y++;
            neighbours[neighbourRanges[e.y].y] = e.x;
            neighbourWeights[neighbourRanges[e.y].y] = e.w;
            neighbourRanges[e.y].y++;
        }
    }
    return in;
}

// METIS reader (graph.cu:351-511): 1-based neighbour lists, optional vertex and
// edge weights (fmt digits), self-loops and repeated neighbours skipped with a
// one-time warning; edges are the entries with i > neighbour.
istream &Graph::readMETIS(istream &in)
{
    int flags = 0;
    clear();
    while (in.good()) {
        string line;
        getline(in, line);
        trim_front(line);
        if (line.length() < 2) continue;
        if (line[0] == '%') continue;
        istringstream sline(line);
        if (!(sline >> nrVertices >> nrEdges)) fail("Unable to read METIS header!");
        nrVertexWeights = 0;
        sline >> flags >> nrVertexWeights;
        break;
    }
    const bool weighted_edges = (flags % 10) != 0, weighted_vertices = ((flags / 10) % 10) != 0;
    if (nrVertexWeights != 0 && !weighted_vertices) fail("Invalid vertex weight specification!");
    if (weighted_vertices && nrVertexWeights == 0) nrVertexWeights = 1;

    neighbourRanges.assign(nrVertices, make_int2(0, 0));
    neighbours.reserve(nrEdges);
    neighbourWeights.reserve(nrEdges);
    edges.reserve(nrEdges);
    if (nrVertexWeights > 0) vertexWeights.assign(nrVertexWeights * nrVertices, 0);
    else vertexWeights.clear();

    bool warned_self = false, warned_dup = false;
    for (int i = 0; i < nrVertices; ++i) {
        if (!in.good()) fail("Read error!");
        string line;
        getline(in, line);
        istringstream sline(line);
        if (weighted_vertices)
            for (int j = 0; j < nrVertexWeights; ++j) sline >> vertexWeights[nrVertexWeights * i + j];
        set<int> seen;
        int var;
        neighbourRanges[i].x = (int)neighbours.size();
        while (sline >> var) {
            if (var < 1 || var > nrVertices) fail("Invalid neighbour index!");
            float wgt = 1.0f;
            if (weighted_edges) sline >> wgt;
            if (var - 1 != i) {
                if (seen.insert(var).second) {
                    neighbours.push_back(var - 1);
                    neighbourWeights.push_back(wgt);
                } else if (!warned_dup) {
                    warned_dup = true;
                    cerr << "Warning, duplicate neighbours!" << endl;
                }
            } else if (!warned_self) {
                warned_self = true;
                cerr << "Warning, skipping v--v edges!" << endl;
            }
        }
        neighbourRanges[i].y = (int)neighbours.size();
    }
    for (int i = 0; i < nrVertices; ++i)
        for (int j = neighbourRanges[i].x; j < neighbourRanges[i].y; ++j)
            if (i > neighbours[j]) edges.push_back(Edge(i, neighbours[j], neighbourWeights[j]));
    if (nrEdges != (int)edges.size()) {
        cerr << "Warning: Invalid edge count!" << endl;
        nrEdges = (int)edges.size();
    }
    return in;
}

// Random vertex relabelling (graph.cu:513-548): a permutation drawn with
// std::random_shuffle (so it consumes rand() exactly as the reference does);
// ranges move with their vertices, neighbour lists stay where they are and
// their ids are relabelled.  Returns the permutation (new index -> old vertex).
vector<int> Graph::random_shuffle()
{
    vector<int> perm(nrVertices);
    for (int i = 0; i < nrVertices; ++i) perm[i] = i;
    // deprecated since C++14, but the only shuffle whose draws are rand()'s
#pragma GCC diagnostic push
#pragma GCC diagnostic ignored "-Wdeprecated-declarations"
    std::random_shuffle(perm.begin(), perm.end());
#pragma GCC diagnostic pop
    vector<int2> moved(nrVertices);
    for (int i = 0; i < nrVertices; ++i) moved[i] = neighbourRanges[perm[i]];
    neighbourRanges = moved;
    vector<int> inv(nrVertices);
    for (int i = 0; i < nrVertices; ++i) inv[perm[i]] = i;
    for (int &u : neighbours) u = inv[u];
    for (Edge &e : edges) {
        e.x = inv[e.x];
        e.y = inv[e.y];
    }
    return perm;
}

}  // namespace mtc
