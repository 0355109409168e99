/*
 * Minimal stand-in for <tbb/tbb.h>, project-written.  TEST INFRASTRUCTURE:
 * it exists only so that the reference's own matchtbb.cu compiles into
 * oracle/_ref (TBB is not installed here).  It provides exactly what
 * matchtbb.cu uses: tbb::blocked_range<T> (begin/end) and
 * tbb::parallel_for(range, body), run as OpenMP dynamic chunks.
 *
 * The matchers written against it are deterministic for any chunking: each
 * body invocation reads only arrays that no invocation of the same
 * parallel_for writes (matchtbb.cu:121-485).
 */
#ifndef MM_TBB_SHIM_H
#define MM_TBB_SHIM_H

#include <cstddef>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace tbb {

template <typename T>
class blocked_range {
  public:
    blocked_range(T b, T e, std::size_t grain = 1) : lo_(b), hi_(e), grain_(grain) {}
    T begin() const { return lo_; }
    T end() const { return hi_; }
    bool empty() const { return !(lo_ < hi_); }
    std::size_t size() const { return empty() ? 0 : (std::size_t)(hi_ - lo_); }
    std::size_t grainsize() const { return grain_; }

  private:
    T lo_, hi_;
    std::size_t grain_;
};

template <typename T, typename Body>
void parallel_for(const blocked_range<T> &range, const Body &body)
{
    const long long total = (long long)range.size();
    if (total <= 0) return;
#ifdef _OPENMP
    const int threads = omp_get_max_threads();
#else
    const int threads = 1;
#endif
    if (threads <= 1) {
        body(range);
        return;
    }
    /* 16 chunks per thread, as TBB's auto partitioner roughly does. */
    long long chunk = total / ((long long)threads * 16);
    if (chunk < 256) chunk = 256;
    const long long nchunks = (total + chunk - 1) / chunk;
#pragma omp parallel for schedule(dynamic, 1)
    for (long long c = 0; c < nchunks; ++c) {
        const T b = (T)(range.begin() + c * chunk);
        const long long rest = total - c * chunk;
        const T e = (T)(b + (rest < chunk ? rest : chunk));
        body(blocked_range<T>(b, e));
    }
}

}  // namespace tbb

#endif
