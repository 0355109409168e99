// mm_pull.cu -- reference-structured kernel family ("pull" path).
//
// One kernel per step of the reference's round (src/matchgpu.cu:184-451):
// select (hash colouring), request (blue proposes), respond (red scans its
// list for proposers), commit (mutual pairs matched), one thread per vertex.
// The round loop runs on the host and, in maximal mode, reads the
// keep-matching flag back after every round exactly like the reference
// (src/matchgpu.cu:604-615).  This family is kept as the structural baseline
// the push path is measured against and as a second, independent device
// implementation for cross-checking; it reads every adjacency list of every
// active vertex once per round (blue in request, red in respond).
#include <cuda_runtime.h>

#include "mm_common.cuh"

namespace mm {
namespace {

constexpr int kBlock = 256;

// Sum `value` over the block and add it to *dst with one atomic per block.
__device__ __forceinline__ void block_add(unsigned long long *dst, unsigned long long value)
{
    __shared__ unsigned long long part[kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) value += __shfl_down_sync(0xffffffffu, value, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) part[warp] = value;
    __syncthreads();
    if (warp == 0) {
        value = lane < (kBlock / 32) ? part[lane] : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) value += __shfl_down_sync(0xffffffffu, value, o);
        if (lane == 0 && value) atomicAdd(dst, value);
    }
}

__device__ __forceinline__ int degree_of(int2 r) { return r.y > r.x ? r.y - r.x : 0; }

// gSelect / gaSelect (src/matchgpu.cu:184-258).
template <bool kStats>
__global__ void __launch_bounds__(kBlock) pull_select(int *match, int n, const uint32_t *seeds, int round,
                                                      uint32_t barrier, int *keep,
                                                      unsigned long long *st)
{
    const uint32_t seed = seeds[round];
    unsigned long long active = 0, blue = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        if (match[v] >= 2) continue;
        *keep = 1;
        const int c = colour_of((uint32_t)v, seed, barrier);
        match[v] = c;
        ++active;
        blue += c == kBlue;
    }
    if (kStats) {
        block_add(st + MM_ST_ACTIVE, active);
        block_add(st + MM_ST_BLUE, blue);
        block_add(st + MM_ST_RED, active - blue);
    }
}

// grRequest / gwRequest (src/matchgpu.cu:286-327, 360-409).
template <bool kWeighted, bool kStats>
__global__ void __launch_bounds__(kBlock) pull_request(int *req, const int *match, int n,
                                                       const int2 *ranges, const int *nbrs,
                                                       const float *w, unsigned long long *st)
{
    unsigned long long seen = 0, deg = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        if (match[v] != kBlue) {
            req[v] = n;
            continue;
        }
        const int2 r = ranges[v];
        deg += degree_of(r);
        int dead = 1;
        int chosen = n;
        float best = -1.0f;
        for (int j = r.x; j < r.y; ++j) {
            ++seen;
            const int u = nbrs[j];
            const int m = match[u];
            if (m < 4) {
                dead = 0;
                if (m == kRed) {
                    if (!kWeighted) {
                        chosen = u;
                        break;
                    }
                    const float x = w[j];
                    if (x > best) {
                        best = x;
                        chosen = u;
                    }
                }
            }
        }
        req[v] = chosen + dead;
    }
    if (kStats) {
        block_add(st + MM_ST_REQ_ENTRIES, seen);
        block_add(st + MM_ST_BLUE_DEG, deg);
    }
}

// grRespond / gwRespond (src/matchgpu.cu:329-357, 411-451).
template <bool kWeighted, bool kStats>
__global__ void __launch_bounds__(kBlock) pull_respond(int *req, const int *match, int n,
                                                       const int2 *ranges, const int *nbrs,
                                                       const float *w, unsigned long long *st)
{
    unsigned long long seen = 0, deg = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        if (match[v] != kRed) continue;
        const int2 r = ranges[v];
        deg += degree_of(r);
        int chosen = n;
        float best = -1.0f;
        for (int j = r.x; j < r.y; ++j) {
            ++seen;
            const int u = nbrs[j];
            if (match[u] == kBlue && req[u] == v) {
                if (!kWeighted) {
                    chosen = u;
                    break;
                }
                const float x = w[j];
                if (x > best) {
                    best = x;
                    chosen = u;
                }
            }
        }
        if (chosen < n) req[v] = chosen;
    }
    if (kStats) {
        block_add(st + MM_ST_RESP_ENTRIES, seen);
        block_add(st + MM_ST_RED_DEG, deg);
    }
}

// gMatch (src/matchgpu.cu:260-283).
template <bool kStats>
__global__ void __launch_bounds__(kBlock) pull_commit(int *match, const int *req, int n,
                                                      unsigned long long *st)
{
    unsigned long long matched = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int r = req[v];
        if (r == n + 1) {
            match[v] = kDead;
        } else if (r < n && req[r] == v) {
            match[v] = 4 + min(v, r);
            ++matched;
        }
    }
    if (kStats) block_add(st + MM_ST_MATCHED, matched);
}

template <bool kWeighted, bool kStats>
void launch_round(int *match, int *req, int n, const int2 *ranges, const int *nbrs, const float *w,
                  const uint32_t *d_seeds, int round, uint32_t barrier, int *keep,
                  unsigned long long *st, cudaStream_t s)
{
    const int grid = grid_for(n, kBlock, 148 * 16);
    pull_select<kStats><<<grid, kBlock, 0, s>>>(match, n, d_seeds, round, barrier, keep, st);
    pull_request<kWeighted, kStats><<<grid, kBlock, 0, s>>>(req, match, n, ranges, nbrs, w, st);
    pull_respond<kWeighted, kStats><<<grid, kBlock, 0, s>>>(req, match, n, ranges, nbrs, w, st);
    pull_commit<kStats><<<grid, kBlock, 0, s>>>(match, req, n, st);
}

}  // namespace

mm_status pull_match(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                     int *d_match, int *rounds_out, long long *stats, int stats_rounds,
                     cudaStream_t stream, uint32_t (*draw)(void *), void *draw_ctx)
{
    const int n = g->n;
    const bool weighted = is_weighted(type), maximal = is_maximal(type);
    const int cap = max_rounds_of(type);
    // scratch: req[n] | keep flag | seeds[255] | stats[255 * MM_STATS_COLS]
    const size_t req_bytes = ((size_t)(n > 0 ? n : 1) * sizeof(int) + 255) & ~(size_t)255;
    const size_t seed_off = req_bytes + 256;
    const size_t st_off = seed_off + 1024;
    const size_t total = st_off + sizeof(unsigned long long) * kMaxRounds * MM_STATS_COLS;
    mm_status s = ensure_scratch(g, total);
    if (s != MM_OK) return s;
    char *base = (char *)g->scratch;
    int *req = (int *)base;
    int *keep = (int *)(base + req_bytes);
    uint32_t *d_seeds = (uint32_t *)(base + seed_off);
    unsigned long long *d_st = (unsigned long long *)(base + st_off);
    const int nup = nseeds < cap ? nseeds : cap;
    if (!draw)
        MM_CUDA_TRY(cudaMemcpyAsync(d_seeds, seeds, sizeof(uint32_t) * nup, cudaMemcpyHostToDevice, stream),
                    "seed upload");
    MM_CUDA_TRY(cudaMemsetAsync(d_match, 0, sizeof(int) * (size_t)(n > 0 ? n : 1), stream), "clear match");
    if (stats) MM_CUDA_TRY(cudaMemsetAsync(d_st, 0, sizeof(unsigned long long) * kMaxRounds * MM_STATS_COLS, stream),
                           "clear stats");

    int rounds = 0;
    for (;;) {
        if (rounds >= cap) break;
        if (draw) {
            // the round's seed, drawn as the round starts (src/matchgpu.cu:609): one
            // draw per executed round; a pageable copy is done once it returns
            const uint32_t sd = draw(draw_ctx);
            MM_CUDA_TRY(cudaMemcpyAsync(d_seeds + rounds, &sd, sizeof sd, cudaMemcpyHostToDevice, stream),
                        "seed upload");
            MM_CUDA_TRY(cudaStreamSynchronize(stream), "seed upload");
        } else if (rounds >= nseeds) {
            set_error("mm_match: fewer seeds than rounds");
            return MM_ERR_SEEDS;
        }
        if (maximal) MM_CUDA_TRY(cudaMemsetAsync(keep, 0, sizeof(int), stream), "clear flag");
        unsigned long long *st = d_st + (size_t)rounds * MM_STATS_COLS;
        if (weighted) {
            if (stats) launch_round<true, true>(d_match, req, n, g->d_ranges, g->d_nbrs, g->d_w, d_seeds, rounds, barrier, keep, st, stream);
            else launch_round<true, false>(d_match, req, n, g->d_ranges, g->d_nbrs, g->d_w, d_seeds, rounds, barrier, keep, st, stream);
        } else {
            if (stats) launch_round<false, true>(d_match, req, n, g->d_ranges, g->d_nbrs, g->d_w, d_seeds, rounds, barrier, keep, st, stream);
            else launch_round<false, false>(d_match, req, n, g->d_ranges, g->d_nbrs, g->d_w, d_seeds, rounds, barrier, keep, st, stream);
        }
        MM_CUDA_TRY(cudaGetLastError(), "round launch");
        ++rounds;
        if (maximal) {
            int flag = 0;
            MM_CUDA_TRY(cudaMemcpyAsync(&flag, keep, sizeof(int), cudaMemcpyDeviceToHost, stream), "flag read");
            MM_CUDA_TRY(cudaStreamSynchronize(stream), "flag sync");
            if (!flag) break;
        }
    }
    if (stats && stats_rounds > 0) {
        const int nr = rounds < stats_rounds ? rounds : stats_rounds;
        MM_CUDA_TRY(cudaMemcpyAsync(stats, d_st, sizeof(long long) * MM_STATS_COLS * nr, cudaMemcpyDeviceToHost, stream),
                    "stats read");
        MM_CUDA_TRY(cudaStreamSynchronize(stream), "stats sync");
    }
    *rounds_out = rounds;
    return MM_OK;
}

}  // namespace mm
