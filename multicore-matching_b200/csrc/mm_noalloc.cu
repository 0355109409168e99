// mm_noalloc.cu -- mm_match_noalloc: a matching entry point that allocates nothing.
//
// Who needs it: callers that must not allocate device memory while they run.
// cudaMalloc and cudaFree synchronise the whole device, so a caller that
// shares the GPU with latency-sensitive streams (a serving process, a
// real-time loop) cannot afford them mid-flight, and callers whose device
// memory is owned up front by a framework or pool (a fixed memory budget
// reserved at start-up) are not allowed to allocate at all.  The regular
// entry points allocate: mm_graph_create copies the graph and
// mm_graph_prepare builds a per-slot proposal index.
//
// This entry point takes the graph and the match output as the caller's own
// device arrays and keeps its only scratch -- one request slot per vertex plus
// two status words -- in a fixed file-scope device array.  It runs the
// reference-structured kernel family (select / request / respond / commit,
// one thread per vertex, as src/matchgpu.cu:184-451) with these kernels'
// request array placed in that array.
//
// Limits and rules:
//   * at most kNoAllocMaxVertices vertices; larger graphs get MM_ERR_UNSUPPORTED;
//   * the array takes 4 MiB plus 256 bytes on a device.  The CUDA runtime loads
//     this library's device code lazily, so the array is placed on a device by
//     the first call there (which also loads the kernels and may synchronise the
//     device), then held until the process exits: a caller that must not allocate
//     later makes one call at start-up, for each device and matching type it uses;
//   * the first call on a device also looks up the array's device address (with
//     that device current), kept for the life of the process: make that first call
//     before any stream capture, and do not use this entry point on a device
//     after cudaDeviceReset in the same process;
//   * d_ranges is read as int2 pairs and must be 8-byte aligned (else MM_ERR_ARG);
//   * every call shares the array and leaves its contents behind: calls that
//     overlap on the GPU (two streams, two threads) race and must not be made.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "mm_common.cuh"

#define MM_API extern "C" __attribute__((visibility("default")))

namespace mm {
namespace {

constexpr int kNoAllocMaxVertices = 1 << 20;
constexpr int kCtlWords = 64;  // [0] keep-matching flag, [1] validation flags
constexpr int kBlock = 256;

// Scratch of mm_match_noalloc: kCtlWords status words, then one request slot
// per vertex.  In host code this name is only a handle for
// cudaGetSymbolAddress, never a device address.
static __device__ __align__(256) int g_noalloc_scratch[kCtlWords + kNoAllocMaxVertices];

std::mutex g_lookup_mutex;
int *g_scratch_of_device[256] = {};

// Device address of g_noalloc_scratch on the current device (looked up once per device).
mm_status scratch_address(int **out)
{
    int dev = -1;
    MM_CUDA_TRY(cudaGetDevice(&dev), "mm_match_noalloc: current device");
    if (dev < 0 || dev >= 256) {
        set_error("mm_match_noalloc: device ordinal out of range");
        return MM_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_lookup_mutex);
    if (!g_scratch_of_device[dev]) {
        void *p = nullptr;
        MM_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch), "mm_match_noalloc: scratch address");
        g_scratch_of_device[dev] = (int *)p;
    }
    *out = g_scratch_of_device[dev];
    return MM_OK;
}

__global__ void na_validate(const int2 *ranges, const int *nbrs, int n, long long nnz, int *flags)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int2 r = ranges[v];
        if (r.y <= r.x) continue;
        if (r.x < 0 || (long long)r.y > nnz) {
            atomicOr(flags, 1);
            continue;
        }
        for (int j = r.x; j < r.y; ++j) {
            const int u = nbrs[j];
            if (u < 0 || u >= n) {
                atomicOr(flags, 2);
                break;
            }
        }
    }
}

__global__ void na_select(int *match, int n, uint32_t seed, uint32_t barrier, int *keep)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        if (match[v] >= 2) continue;
        *keep = 1;
        match[v] = colour_of((uint32_t)v, seed, barrier);
    }
}

template <bool kWeighted>
__global__ void na_request(int *req, const int *match, int n, const int2 *ranges, const int *nbrs, const float *w)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        if (match[v] != kBlue) {
            req[v] = n;
            continue;
        }
        const int2 r = ranges[v];
        int dead = 1, chosen = n;
        float best = -1.0f;
        for (int j = r.x; j < r.y; ++j) {
            const int u = nbrs[j];
            const int m = match[u];
            if (m < 4) {
                dead = 0;
                if (m == kRed) {
                    if (!kWeighted) {
                        chosen = u;
                        break;
                    }
                    const float x = w ? w[j] : 1.0f;
                    if (x > best) {
                        best = x;
                        chosen = u;
                    }
                }
            }
        }
        req[v] = chosen + dead;
    }
}

template <bool kWeighted>
__global__ void na_respond(int *req, const int *match, int n, const int2 *ranges, const int *nbrs, const float *w)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        if (match[v] != kRed) continue;
        const int2 r = ranges[v];
        int chosen = n;
        float best = -1.0f;
        for (int j = r.x; j < r.y; ++j) {
            const int u = nbrs[j];
            if (match[u] == kBlue && req[u] == v) {
                if (!kWeighted) {
                    chosen = u;
                    break;
                }
                const float x = w ? w[j] : 1.0f;
                if (x > best) {
                    best = x;
                    chosen = u;
                }
            }
        }
        if (chosen < n) req[v] = chosen;
    }
}

__global__ void na_commit(int *match, const int *req, int n)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int r = req[v];
        if (r == n + 1) match[v] = kDead;
        else if (r < n && req[r] == v) match[v] = 4 + min(v, r);
    }
}

}  // namespace
}  // namespace mm

using namespace mm;

// Declared in include/mm_match.h.  No cudaMalloc / cudaFree and no allocating
// library call anywhere on this path.
MM_API mm_status mm_match_noalloc(int n, const int *d_ranges, long long nnz, const int *d_neighbours,
                                  const float *d_weights, int type, uint32_t barrier, const uint32_t *seeds,
                                  int nseeds, int *d_match_out, int *rounds_out, void *stream)
{
    if (!rounds_out || n < 0 || nnz < 0 || (n > 0 && (!d_ranges || !d_match_out)) || (nnz > 0 && !d_neighbours)) {
        set_error("mm_match_noalloc: null argument or negative size");
        return MM_ERR_ARG;
    }
    if (max_rounds_of(type) < 0) {
        set_error("mm_match_noalloc: type must be 6, 7, 8 or 9");
        return MM_ERR_ARG;
    }
    if (!seeds || nseeds < 1) {
        set_error("mm_match_noalloc: no seeds");
        return MM_ERR_SEEDS;
    }
    if (n > kNoAllocMaxVertices) {
        set_error("mm_match_noalloc: n = " + std::to_string(n) + " exceeds the fixed scratch of " +
                  std::to_string(kNoAllocMaxVertices) + " vertices; use mm_graph_create + mm_match");
        return MM_ERR_UNSUPPORTED;
    }
    if (nnz >= (1ll << 31)) {
        set_error("mm_match_noalloc: nnz must be below 2^31");
        return MM_ERR_UNSUPPORTED;
    }
    if (((uintptr_t)d_ranges & 7u) != 0) {
        set_error("mm_match_noalloc: d_ranges must be 8-byte aligned (it is read as int2 pairs)");
        return MM_ERR_ARG;
    }
    int *scratch = nullptr;
    mm_status s = scratch_address(&scratch);
    if (s != MM_OK) return s;
    int *keep = scratch;
    int *flags = scratch + 1;
    int *req = scratch + kCtlWords;
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = grid_for(n, kBlock, 148 * 16);

    // Validate what the kernels will read (the previous call's flags are stale: clear them).
    MM_CUDA_TRY(cudaMemsetAsync(flags, 0, sizeof(int), st), "mm_match_noalloc: clear flags");
    if (n > 0) na_validate<<<grid, kBlock, 0, st>>>((const int2 *)d_ranges, d_neighbours, n, nnz, flags);
    MM_CUDA_TRY(cudaGetLastError(), "mm_match_noalloc: validate");
    int bad = 0;
    MM_CUDA_TRY(cudaMemcpyAsync(&bad, flags, sizeof(int), cudaMemcpyDeviceToHost, st), "mm_match_noalloc: flags");
    MM_CUDA_TRY(cudaStreamSynchronize(st), "mm_match_noalloc: validate");
    if (bad) {
        set_error((bad & 1) ? "mm_match_noalloc: a neighbour range lies outside [0, nnz)"
                            : "mm_match_noalloc: a neighbour id lies outside [0, n)");
        return MM_ERR_GRAPH;
    }

    const bool weighted = is_weighted(type), maximal = is_maximal(type);
    const int cap = max_rounds_of(type);
    if (n > 0) MM_CUDA_TRY(cudaMemsetAsync(d_match_out, 0, sizeof(int) * (size_t)n, st), "mm_match_noalloc: clear");
    const int2 *ranges = (const int2 *)d_ranges;
    int rounds = 0;
    for (;;) {
        if (rounds >= cap) break;
        if (rounds >= nseeds) {
            set_error("mm_match_noalloc: fewer seeds than rounds");
            return MM_ERR_SEEDS;
        }
        MM_CUDA_TRY(cudaMemsetAsync(keep, 0, sizeof(int), st), "mm_match_noalloc: clear flag");
        if (n > 0) {
            na_select<<<grid, kBlock, 0, st>>>(d_match_out, n, seeds[rounds], barrier, keep);
            if (weighted) {
                na_request<true><<<grid, kBlock, 0, st>>>(req, d_match_out, n, ranges, d_neighbours, d_weights);
                na_respond<true><<<grid, kBlock, 0, st>>>(req, d_match_out, n, ranges, d_neighbours, d_weights);
            } else {
                na_request<false><<<grid, kBlock, 0, st>>>(req, d_match_out, n, ranges, d_neighbours, d_weights);
                na_respond<false><<<grid, kBlock, 0, st>>>(req, d_match_out, n, ranges, d_neighbours, d_weights);
            }
            na_commit<<<grid, kBlock, 0, st>>>(d_match_out, req, n);
        }
        MM_CUDA_TRY(cudaGetLastError(), "mm_match_noalloc: round");
        ++rounds;
        if (maximal) {
            int flag = 0;
            MM_CUDA_TRY(cudaMemcpyAsync(&flag, keep, sizeof(int), cudaMemcpyDeviceToHost, st), "mm_match_noalloc: flag");
            MM_CUDA_TRY(cudaStreamSynchronize(st), "mm_match_noalloc: round");
            if (!flag) break;
        }
    }
    MM_CUDA_TRY(cudaStreamSynchronize(st), "mm_match_noalloc: finish");
    *rounds_out = rounds;
    return MM_OK;
}
