// mm_common.cuh -- shared device helpers and the mm_graph object.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "mm_match.h"

namespace mm {

// Round caps of the reference (src/matchcpu.h:24-25): fixed types run
// NR_MATCH_ROUNDS = 20 rounds, maximal types loop while ++count < 256.
constexpr int kFixedRounds = 20;
constexpr int kMaxRounds = 255;

// Per-vertex colour state used by the kernels ("col"): one byte per vertex.
// It carries exactly what a neighbour's request/respond test needs from the
// reference's match value (src/matchgpu.cu:303-316, 380-386, 346, 431):
//   kBlue (match 0), kRed (match 1), kDead (match 2), kMatched (match >= 4).
enum : uint8_t { kBlue = 0, kRed = 1, kDead = 2, kMatched = 3 };

// Colouring hash of src/matchgpu.cu:196-217: 16 MD5-style steps over
// (vertex id, round seed) with the first 16 SHA-256 constants, the MD5
// round-1 rotations and the MD5 initial words.  Returns h0 + h1 + h2 + h3,
// accumulated as one running sum (the four words are only ever added).
__device__ __forceinline__ uint32_t colour_hash(uint32_t v, uint32_t seed)
{
    constexpr uint32_t K[16] = {0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u,
                                0x3956c25bu, 0x59f111f1u, 0x923f82a4u, 0xab1c5ed5u,
                                0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u,
                                0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u};
    constexpr int R[4] = {7, 12, 17, 22};
    uint32_t a = 0x67452301u, b = 0xefcdab89u, c = 0x98badcfeu, d = 0x10325476u;
    uint32_t sum = a + b + c + d;
    uint32_t g = v;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const uint32_t f = (b & c) | (~b & d);
        const uint32_t x = a + f + K[k] + g;
        const uint32_t t = d;
        d = c;
        c = b;
        b = b + __funnelshift_l(x, x, R[k & 3]);
        a = t;
        sum += a + b + c + d;
        g *= seed;
    }
    return sum;
}

// Blue iff the hash is below the select barrier (src/matchgpu.cu:217).
__device__ __forceinline__ uint8_t colour_of(uint32_t v, uint32_t seed, uint32_t barrier)
{
    return colour_hash(v, seed) < barrier ? kBlue : kRed;
}

// Order-preserving map of a float to uint32 for the weighted argmax.  Only
// weights the reference can pick reach it (w > -1, so never NaN); -0.0 is
// folded onto +0.0 because the reference's `nw > maxWeight` treats them as
// equal (src/matchgpu.cu:391, 437).
__device__ __forceinline__ uint32_t weight_order(float w)
{
    uint32_t u = __float_as_uint(w);
    if (u == 0x80000000u) u = 0u;
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

}  // namespace mm

// Device-resident graph plus per-graph scratch.  Everything lives on `device`.
struct mm_graph {
    int device = 0;
    int n = 0;
    long long nnz = 0;
    bool has_weights = false;
    bool contiguous = false;  // ranges tile [0, nnz) in vertex order
    // Set at upload: ranges tile [0, nnz), every list is strictly increasing and
    // the entries (v, u) are those (u, v) transposed -- with the weights too for
    // sym_weights.  Then a red vertex's order of preference over its proposers is
    // (weight, smaller proposer id) and the push path needs no reverse index.
    bool sym_struct = false;
    bool sym_weights = false;
    int2 *d_ranges = nullptr;
    int *d_nbrs = nullptr;
    float *d_w = nullptr;     // unit weights when the graph came without any
    long long max_degree = 0;
    long long sum_degree = 0;
    bool scanned = false;          // degree classes below are valid
    long long short_count = 0;     // vertices with at most 32 neighbour entries
    long long long_count = 0;      // vertices with more
    long long long_entries = 0;    // entries in those longer lists

    // device buffer for host-output calls (mm_match)
    int *d_out = nullptr;

    // scratch shared by the paths, grown on demand
    void *scratch = nullptr;
    size_t scratch_bytes = 0;

    // push path: reverse proposal keys, one per adjacency slot, per weighting
    unsigned long long *d_revkey[2] = {nullptr, nullptr};  // [0] random, [1] weighted
    long long *d_slot_off = nullptr;  // non-contiguous CSR: slot index of vertex v's first entry
    int2 *d_pwin = nullptr;           // weighted types: preference windows {neighbour, position | flag}
    long long *d_pwin_off = nullptr;  // weighted types: first window slot of each vertex; [n] = total
    bool pwin_weights = false;        // d_pwin's second words hold weights (symmetric weighted path)
    int2 *win_build = nullptr;        // windows while being built (d_pwin once complete)
    int *win_big = nullptr;           // while being built: queued lists longer than a window chunk

    // push path: per-call state of the round kernel
    void *push_exec = nullptr;  // internal (mm::PushState *)
    // launch options (mm_graph_tune; 0 = the library's default)
    int opt_fin_div = 0;        // finish phase from the round whose active set is <= 1/opt of round 0's; -1 never
    int opt_blocks_per_sm = 0;  // blocks per SM of the round and finish kernels

    // a batch of independent graphs (mm_graph_set_batch): graph i holds
    // vertices [goff[i], goff[i + 1]); vbase[v] = goff of v's graph; last[v]
    // = last round at whose colouring v was unmatched
    int ngraphs = 0;
    int *d_goff = nullptr;
    int *d_vbase = nullptr;
    uint8_t *d_last = nullptr;
};

namespace mm {

void set_error(const std::string &msg);
mm_status cuda_fail(cudaError_t e, const char *what);
#define MM_CUDA_TRY(expr, what)                              \
    do {                                                     \
        cudaError_t mm_e_ = (expr);                          \
        if (mm_e_ != cudaSuccess) return mm::cuda_fail(mm_e_, what); \
    } while (0)

// Pooled device memory (one stream-ordered pool per device, never trimmed
// unless mm_release_cached_memory asks): allocation and free are ordered on
// `stream`; a buffer used on other streams needs that stream synchronised first.
cudaError_t dev_alloc(void **p, size_t bytes, cudaStream_t stream);
void dev_free(void *p, cudaStream_t stream);
// Small page-locked host blocks, recycled process-wide.
cudaError_t pinned_get(void **p, size_t bytes);
void pinned_put(void *p, size_t bytes);
mm_status release_cached(int device);

// Polls a grid-barrier wait makes before it gives up (the kernel then returns
// an error status instead of waiting on).
constexpr long long kSpinLimitDefault = 1ll << 22;
// Testing hooks (mm_debug): the grid barriers' poll limit and the barrier mark
// at which block 0 does not arrive (-1: none).
long long debug_spin_limit();
int debug_skip_mark();

// Ensure g->scratch holds at least `bytes`; returns MM_OK or an error.
mm_status ensure_scratch(mm_graph *g, size_t bytes);

// Paths.
mm_status pull_match(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                     int *d_match, int *rounds_out, long long *stats, int stats_rounds,
                     cudaStream_t stream, uint32_t (*draw)(void *) = nullptr, void *draw_ctx = nullptr);
mm_status push_prepare(mm_graph *g, int weighted, cudaStream_t stream);
mm_status push_match(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                     int *d_match, int *rounds_out, long long *stats, int stats_rounds,
                     cudaStream_t stream);
mm_status push_profile(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds, int *d_match,
                       int *rounds_out, float *ms_kernels, int cap_rounds, int *launched, cudaStream_t stream);
void push_release(mm_graph *g);
mm_status push_batch_rounds(mm_graph *g, int type, int *rounds_host, cudaStream_t stream);
mm_status push_match_policy(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                            const float *mlp_host, float level, int *d_match, int *rounds_out, float *trace,
                            int trace_rounds, cudaStream_t stream);
// Preference windows of the weighted types, in steps (see mm_push.cu).
mm_status windows_begin(mm_graph *g, cudaStream_t stream);
mm_status windows_range(mm_graph *g, int va, int vb, cudaStream_t stream);
mm_status windows_end(mm_graph *g, cudaStream_t stream);
void windows_discard(mm_graph *g);

inline int max_rounds_of(int type)
{
    if (type == MM_TYPE_RANDOM || type == MM_TYPE_WEIGHTED) return kFixedRounds;
    if (type == MM_TYPE_RANDOM_MAXIMAL || type == MM_TYPE_WEIGHTED_MAXIMAL) return kMaxRounds;
    return -1;
}
inline bool is_weighted(int type) { return type == MM_TYPE_WEIGHTED || type == MM_TYPE_WEIGHTED_MAXIMAL; }
inline bool is_maximal(int type) { return type == MM_TYPE_RANDOM_MAXIMAL || type == MM_TYPE_WEIGHTED_MAXIMAL; }

inline int grid_for(long long items, int block, int cap = 148 * 32)
{
    long long g = (items + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

}  // namespace mm
