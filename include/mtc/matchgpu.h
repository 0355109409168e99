/*
 * mtc/matchgpu.h -- drop-in for the reference's src/matchgpu.h.
 *
 * Same class names, constructors and performMatching signature as
 * matchgpu.h:29-84; implemented in libmtc.so over the C ABI of
 * include/mm_match.h (libmmatch.so, sm_100a kernels).
 *
 *   GraphMatchingGPU(graph, threadsPerBlock, selectBarrier)
 *       uploads and validates the CSR (matchgpu.cu:39-66); the weighted
 *       subclasses also upload the weights (matchgpu.cu:97-147) and every
 *       subclass builds its device proposal index here, so that cost lands in
 *       the reference's "total time" (t0 -> t3) and not in its match time.
 *       threadsPerBlock is accepted and ignored: launch shapes are chosen per
 *       degree class.  The barrier is per object (the reference keeps one in a
 *       process-global __constant__, matchgpu.cu:37).
 *   performMatching(match, t1, t2)
 *       records t1 / t2 on the legacy default stream around the round loop
 *       exactly where the reference does (matchgpu.cu:500-527), copies the
 *       result into match, and draws exactly one rand() per executed round,
 *       in order, as the reference's host loop does (matchgpu.cu:509, 609,
 *       707, 816).  The whole loop runs on the device: the per-round seeds are
 *       read ahead from the C library's rand() state without consuming it,
 *       and the stream is then advanced by the rounds actually executed.
 *   Errors print to std::cerr and throw std::exception(), as the reference.
 */
#ifndef MATCH_MATCH_GPU_H
#define MATCH_MATCH_GPU_H

#include <vector>
#include <cuda.h>

#include "graph.h"
#include "matchcpu.h"

struct mm_graph;

namespace mtc
{

class GraphMatchingGPU : public GraphMatching
{
	public:
		GraphMatchingGPU(const Graph &, const int &, const unsigned int &);
		virtual ~GraphMatchingGPU();

		virtual void performMatching(std::vector<int> &, cudaEvent_t &, cudaEvent_t &) const = 0;

	protected:
		GraphMatchingGPU(const Graph &, const int &, const unsigned int &, int type);
		void runMatching(std::vector<int> &, cudaEvent_t &, cudaEvent_t &, int type) const;

		const int threadsPerBlock;
		const uint selectBarrier;
		int2 *dneighbourRanges;
		int *dneighbours;
		mm_graph *dgraph;  /* device-resident graph of libmmatch.so */
		int *dmatch;       /* device match[] the round loop writes */
};

class GraphMatchingGPURandom : public GraphMatchingGPU
{
	public:
		GraphMatchingGPURandom(const Graph &, const int &, const unsigned int &);
		~GraphMatchingGPURandom();

		void performMatching(std::vector<int> &, cudaEvent_t &, cudaEvent_t &) const;
};

class GraphMatchingGPURandomMaximal : public GraphMatchingGPU
{
	public:
		GraphMatchingGPURandomMaximal(const Graph &, const int &, const unsigned int &);
		~GraphMatchingGPURandomMaximal();

		void performMatching(std::vector<int> &, cudaEvent_t &, cudaEvent_t &) const;
};

class GraphMatchingGPUWeighted : public GraphMatchingGPU
{
	public:
		GraphMatchingGPUWeighted(const Graph &, const int &, const unsigned int &);
		~GraphMatchingGPUWeighted();

		void performMatching(std::vector<int> &, cudaEvent_t &, cudaEvent_t &) const;

	private:
		float *dweights;
};

class GraphMatchingGPUWeightedMaximal : public GraphMatchingGPU
{
	public:
		GraphMatchingGPUWeightedMaximal(const Graph &, const int &, const unsigned int &);
		~GraphMatchingGPUWeightedMaximal();

		void performMatching(std::vector<int> &, cudaEvent_t &, cudaEvent_t &) const;

	private:
		float *dweights;
};

};

#endif
