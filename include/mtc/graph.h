/*
 * mtc/graph.h -- drop-in for the reference's src/graph.h (Multicore-Matching).
 *
 * Same classes, members and layout: mtc::Edge {x, y, w} (graph.h:30-39) and
 * mtc::Graph with public CSR members (graph.h:41-60).  neighbourRanges[v] is
 * {begin, end} into neighbours / neighbourWeights; it is not a prefix array,
 * so ranges may be permuted (random_shuffle) and need not be contiguous.
 * Implemented in libmtc.so (multicore-matching_b200/csrc/mtc_graph.cpp).
 */
#ifndef MATCH_GRAPH_H
#define MATCH_GRAPH_H

#include <iostream>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>
#include <vector_types.h>

namespace mtc
{

class Edge
{
	public:
		Edge();
		Edge(const int &, const int &, const float & = 1.0);
		~Edge();

		int x, y;
		float w;
};

class Graph
{
	public:
		Graph();
		~Graph();

		void clear();
		std::istream &readMETIS(std::istream &);
		std::istream &readMatrixMarket(std::istream &);
		std::vector<int> random_shuffle();
		bool empty() const;

	public:
		int nrVertices, nrVertexWeights, nrEdges;
		std::vector<int> vertexWeights;
		std::vector<int2> neighbourRanges;
		std::vector<int> neighbours;
		std::vector<float> neighbourWeights;
		std::vector<Edge> edges;
};

}

#endif
