/*
 * mtc/matchcpu.h -- drop-in for the reference's src/matchcpu.h.
 *
 * mtc::GraphMatching (matchcpu.h:31-48) is implemented in libmtc.so: the
 * match encoding helpers, initialMatching, getWeight and testMatching with
 * the reference's semantics.  The sequential CPU matchers (types 0-5,
 * matchcpu.h:50-102) are declared for source compatibility only; they are
 * not part of this library (link the reference's matchcpu.cu for them; the
 * program's own definitions of the base class then take precedence).
 */
#ifndef MATCH_MATCH_H
#define MATCH_MATCH_H

#include <vector>

#include "graph.h"

#define NR_MATCH_ROUNDS 20
#define NR_MAX_MATCH_ROUNDS 256

namespace mtc
{

class GraphMatching
{
	public:
		GraphMatching(const Graph &);
		virtual ~GraphMatching();

		static void getWeight(double &, long &, const std::vector<int> &, const Graph &);
		static bool testMatching(const std::vector<int> &, const Graph &);

		static inline int matchVal(const int &i, const int &j) {return 4 + (i < j ? i : j);};
		static inline bool isMatched(const int &m) {return m >= 4;};

		std::vector<int> initialMatching() const;
		virtual void performMatching(std::vector<int> &, cudaEvent_t &, cudaEvent_t &) const = 0;

	protected:
		const Graph &graph;
};

class GraphMatchingCPURandom : public GraphMatching
{
	public:
		GraphMatchingCPURandom(const Graph &);
		~GraphMatchingCPURandom();

		void performMatching(std::vector<int> &, cudaEvent_t &, cudaEvent_t &) const;
};

class GraphMatchingCPUMinDeg : public GraphMatching
{
	public:
		GraphMatchingCPUMinDeg(const Graph &);
		~GraphMatchingCPUMinDeg();

		void performMatching(std::vector<int> &, cudaEvent_t &, cudaEvent_t &) const;
};

class GraphMatchingCPUStatMinDeg : public GraphMatching
{
	public:
		GraphMatchingCPUStatMinDeg(const Graph &);
		~GraphMatchingCPUStatMinDeg();

		void performMatching(std::vector<int> &, cudaEvent_t &, cudaEvent_t &) const;
};

class GraphMatchingCPUKarpSipser : public GraphMatching
{
	public:
		GraphMatchingCPUKarpSipser(const Graph &);
		~GraphMatchingCPUKarpSipser();

		void performMatching(std::vector<int> &, cudaEvent_t &, cudaEvent_t &) const;
};

class GraphMatchingCPUWeighted : public GraphMatching
{
	public:
		GraphMatchingCPUWeighted(const Graph &);
		~GraphMatchingCPUWeighted();

		void performMatching(std::vector<int> &, cudaEvent_t &, cudaEvent_t &) const;
};

class GraphMatchingCPUWeightedEdge : public GraphMatching
{
	public:
		GraphMatchingCPUWeightedEdge(const Graph &);
		~GraphMatchingCPUWeightedEdge();

		void performMatching(std::vector<int> &, cudaEvent_t &, cudaEvent_t &) const;
};

};

#endif
