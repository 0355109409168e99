/*
 * mm_match.h -- C ABI of the B200 greedy graph matching library (libmmatch.so).
 *
 * The reference (Multicore-Matching) exposes its GPU matcher only as C++
 * classes (src/matchgpu.h:29-84).  This header is the plain-C boundary those
 * classes sit on here (include/mtc/matchgpu.h implements them over it), and
 * what an FFI (ctypes, cgo, JNI, N-API) binds.  No CUDA or C++ types appear
 * in the signatures: graphs are plain arrays, streams are opaque pointers.
 *
 * Graph layout (the reference's mtc::Graph CSR, src/graph.h:41-60):
 *   ranges[2*v], ranges[2*v+1]  begin / end of vertex v's neighbour list
 *                               (std::vector<int2> neighbourRanges); lists
 *                               need not be contiguous, sorted or disjoint;
 *                               an empty or reversed range means degree 0
 *   neighbours[j]               neighbour id, 0 <= id < n, for j in a range
 *   weights[j]                  float edge weight (NULL: unit weights)
 *
 * Match encoding (src/matchgpu.cu:157-164, src/matchcpu.h:40-41): 0 blue,
 * 1 red, 2 unmatchable, >= 4 matched with value 4 + min(v, partner).
 *
 * Matching types (bin/match.cpp:145-148): 6 random, 7 random maximal,
 * 8 weighted, 9 weighted maximal.  The fixed types run exactly 20 rounds
 * (NR_MATCH_ROUNDS, src/matchcpu.h:24); the maximal types run until a round
 * finds no vertex left to colour, at most 255 rounds (src/matchgpu.cu:604).
 * Round r colours with seeds[r], the value the reference draws from the host
 * rand() at the start of that round (src/matchgpu.cu:509, 609, 707, 816).
 *
 * All functions are thread-compatible (one call per graph at a time) and
 * report failures through their status; mm_last_error() gives the message of
 * the calling thread's last failure.  Nothing aborts or traps.
 */
#ifndef MM_MATCH_H
#define MM_MATCH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum mm_status {
    MM_OK = 0,
    MM_ERR_ARG = 1,          /* bad argument: null pointer, unknown type, n < 0 */
    MM_ERR_GRAPH = 2,        /* CSR rejected: a range outside [0, nnz) or a neighbour id outside [0, n) */
    MM_ERR_CUDA = 3,         /* CUDA runtime error; see mm_last_error() */
    MM_ERR_NOMEM = 4,        /* device allocation failed */
    MM_ERR_UNSUPPORTED = 5,  /* size beyond the library's limits */
    MM_ERR_SEEDS = 6,        /* fewer seeds than rounds the matching needs */
    MM_ERR_DEVICE = 7        /* a device-side step reported failure (status word) */
} mm_status;

enum {
    MM_TYPE_RANDOM = 6,
    MM_TYPE_RANDOM_MAXIMAL = 7,
    MM_TYPE_WEIGHTED = 8,
    MM_TYPE_WEIGHTED_MAXIMAL = 9
};

/* Kernel families for mm_match_ex (the default, MM_PATH_AUTO, is the push path). */
enum {
    MM_PATH_AUTO = 0,
    MM_PATH_PULL = 1,  /* reference-structured select/request/respond/commit kernels */
    MM_PATH_PUSH = 2   /* worklists, preference windows and proposals; device-resident round loop */
};

/* Number of int64 counters per round written by mm_match_stats. */
#define MM_STATS_COLS 13
enum {
    MM_ST_ACTIVE = 0,     /* vertices that could still be matched at the round's colouring */
    MM_ST_BLUE = 1,       /* of those, coloured blue */
    MM_ST_RED = 2,        /* of those, coloured red */
    MM_ST_REQ_ENTRIES = 3,  /* adjacency entries the reference's request loop inspects */
    MM_ST_RESP_ENTRIES = 4, /* adjacency entries the reference's respond loop inspects */
    MM_ST_BLUE_DEG = 5,   /* sum of degrees of blue vertices */
    MM_ST_RED_DEG = 6,    /* sum of degrees of red vertices */
    MM_ST_MATCHED = 7,    /* vertices matched in the round */
    MM_ST_STAGED_DEG = 8,   /* push path: entries its fallback (full-list) scan read */
    MM_ST_STAGED_ITEMS = 9, /* push path: list pieces that scan handled */
    MM_ST_WINDOW_ENTRIES = 10, /* push path: preference-window entries the blue scans read */
    MM_ST_FINISH_ITEMS = 11,  /* push path: active vertices its finish phase classified (round it ran in) */
    MM_ST_FINISH_ENTRIES = 12 /* push path: adjacency entries the finish phase's list scans read */
};

typedef struct mm_graph mm_graph;

/*
 * Upload a CSR graph to `device` (-1: the current device) and validate it on
 * the device.  Replaces the GraphMatchingGPU constructor (src/matchgpu.cu:39-66)
 * and the weighted constructors' weight upload (src/matchgpu.cu:97-147).
 * Host arrays are read only during the call.
 */
mm_status mm_graph_create(int n, const int *ranges, long long nnz, const int *neighbours,
                          const float *weights, int device, mm_graph **out);

/* Same, from arrays already in device memory of the current device (copied). */
mm_status mm_graph_create_device(int n, const int *d_ranges, long long nnz, const int *d_neighbours,
                                 const float *d_weights, mm_graph **out);

/*
 * Build the per-type device structures a matching type needs ahead of the
 * first mm_match call (the push path's preference windows for the weighted
 * types, and its reverse proposal keys off the symmetric path, i.e. unless
 * the lists are contiguous and sorted and every entry has a reverse entry of
 * the same weight), so that their cost lands in set-up rather than in the
 * timed round loop.  Optional.
 */
mm_status mm_graph_prepare(mm_graph *g, int type);

/*
 * Free all device memory of g.  Replaces ~GraphMatchingGPU (src/matchgpu.cu:68-73, 117-121).
 * Waits for the device to finish its work first.  The memory goes back to the
 * library's per-device pool, where the next graph reuses it.
 */
void mm_graph_destroy(mm_graph *g);

/*
 * Hand the pool's unused device memory on `device` back to the driver (no
 * counterpart in the reference, whose objects cudaMalloc and cudaFree
 * directly).  Live graphs keep theirs.
 */
mm_status mm_release_cached_memory(int device);

int mm_graph_n(const mm_graph *g);
long long mm_graph_nnz(const mm_graph *g);
int mm_graph_weighted(const mm_graph *g);
/* Device copies of the CSR (the reference's dneighbourRanges / dneighbours / dweights). */
const void *mm_graph_device_ranges(const mm_graph *g);
const int *mm_graph_device_neighbours(const mm_graph *g);
const float *mm_graph_device_weights(const mm_graph *g);

/*
 * Copy g's CSR to host arrays: ranges (2n ints), neighbours (nnz ints) and
 * weights (nnz floats; unit weights if g was created without), each may be
 * NULL to skip it.  For graphs the library made, such as coarse graphs.
 */
mm_status mm_graph_copy_out(const mm_graph *g, int *ranges, int *neighbours, float *weights);

/* Round cap of a type: 20 (types 6, 8) or 255 (types 7, 9); -1 if unknown. */
int mm_max_rounds(int type);

/*
 * Run one matching of `type` and copy match[n] to the HOST array match_out.
 * Replaces GraphMatchingGPU*::performMatching (src/matchgpu.cu:453-851).
 * seeds[0..nseeds) are the per-round colouring seeds; *rounds_out receives the
 * number of rounds executed, which is the number of seeds the reference would
 * have drawn.  stream: a cudaStream_t, or NULL for the legacy default stream.
 * Weighted types on a graph created without weights use unit weights.
 */
mm_status mm_match(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                   int *match_out, int *rounds_out, void *stream);

/* As mm_match, but match_out is a DEVICE array of n ints on g's device. */
mm_status mm_match_device(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds,
                          int nseeds, int *d_match_out, int *rounds_out, void *stream);

/*
 * As mm_match_device, but each round's seed comes from draw(ctx), called once
 * as the round starts -- exactly once per executed round, the final round of
 * a maximal matching included, as the reference draws host rand() values
 * (src/matchgpu.cu:509, 609, 707, 816).  Runs the reference-structured kernels
 * one round at a time from the host (MM_PATH_PULL), since the rounds cannot
 * be known ahead.  For callers whose seed source cannot be read ahead, such
 * as a rand() whose state layout is unknown.  Single graphs only.
 */
mm_status mm_match_drawn(mm_graph *g, int type, uint32_t barrier, uint32_t (*draw)(void *ctx), void *ctx,
                         int *d_match_out, int *rounds_out, void *stream);

/*
 * Launch options of a graph's matchings (no counterpart in the reference),
 * set by the autotuner (multicore-matching_b200/tune.py) or by hand; 0
 * restores the default.  The result never depends on them, only the time.
 *   MM_TUNE_FINISH_DIV     the finish phase (the late rounds played component by
 *                          component) starts at the first round whose active set
 *                          is at most 1/value of round 0's; default 12 (24 for
 *                          mm_match_policy, whose retirement shrinks the active
 *                          set sooner), at least 2, -1 never
 *   MM_TUNE_BLOCKS_PER_SM  blocks of 512 threads per multiprocessor for the round
 *                          and finish kernels; default all that fit (2)
 */
enum { MM_TUNE_FINISH_DIV = 1, MM_TUNE_BLOCKS_PER_SM = 2 };
mm_status mm_graph_tune(mm_graph *g, int key, int value);

/* As mm_match_device with an explicit kernel family (MM_PATH_*). */
mm_status mm_match_ex(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                      int *d_match_out, int *rounds_out, int path, void *stream);

/*
 * As mm_match_ex, additionally filling stats[r * MM_STATS_COLS + c] for the
 * first min(rounds, stats_rounds) rounds (counters of MM_ST_*).  Slower than
 * mm_match_device; meant for instrumentation, not for timing.
 */
mm_status mm_match_stats(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds,
                         int nseeds, int *d_match_out, int *rounds_out, long long *stats,
                         int stats_rounds, int path, void *stream);

/*
 * Measurement entry: the same launches as mm_match_device, with timestamps
 * taken by the kernels as their grid barriers complete (the device's global
 * timer, nanoseconds).
 * ms_per_kernel[r * MM_PROFILE_KERNELS + k] receives, for each round r <
 * cap_rounds that the kernel executed, k = 0 the window scan (blue vertices'
 * preference windows and proposals), k = 1 the fallback scan of lists longer
 * than their window (0 in rounds without one), k = 2 the commit phase
 * (commit, recolour, worklist compaction), k = 3 their sum; rows of rounds
 * not executed are zero; the finish kernel's work is reported in the row of
 * the round it took over at, its scan pass as k = 0 and the rest as k = 1.
 * *launches receives the number of kernels launched: 3 on the symmetric path
 * (contiguous sorted lists, every entry with a reverse entry of the same
 * weight): the round kernel, the finish kernel and the round kernel again,
 * each returning at once when nothing is left for it; else 1.  Same matching
 * result.
 */
#define MM_PROFILE_KERNELS 4
mm_status mm_match_profile(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                           int *d_match_out, int *rounds_out, float *ms_per_kernel, int cap_rounds,
                           int *launches, void *stream);

/*
 * Allocation-free matching.  No counterpart in the reference: it exists for
 * callers that must not allocate device memory while they run -- cudaMalloc and
 * cudaFree synchronise the whole device, which a process sharing the GPU with
 * latency-sensitive streams cannot afford, and a caller whose device memory is
 * reserved up front by a framework or pool is not allowed to allocate at all.
 * The graph (d_ranges as int2 pairs, d_neighbours, d_weights or NULL for unit
 * weights) and d_match_out are the caller's own DEVICE arrays on the current
 * device; seeds are host values.  Same result and round count as mm_match.
 * Scratch lives in a fixed device array inside the library: at most 1048576
 * vertices (larger n returns MM_ERR_UNSUPPORTED).  The array (4 MiB) is placed
 * on a device by the first call there, which also loads the kernels and may
 * synchronise the device, and is held until the process exits: make one call at
 * start-up for each device and type you use.  That first call also looks up the
 * array's address (make it before any stream capture; do not call this after a
 * cudaDeviceReset of that device).  d_ranges must be 8-byte aligned
 * (MM_ERR_ARG).  All calls share the array: calls that overlap on the GPU race.
 * Calls no cudaMalloc / cudaFree.
 */
mm_status mm_match_noalloc(int n, const int *d_ranges, long long nnz, const int *d_neighbours,
                           const float *d_weights, int type, uint32_t barrier, const uint32_t *seeds,
                           int nseeds, int *d_match_out, int *rounds_out, void *stream);

/*
 * Batches of independent graphs, matched in one launch; no counterpart in the
 * reference, whose matcher takes one graph per call.  g holds the disjoint
 * union: graph i owns vertices [offsets[i], offsets[i + 1]) (ngraphs + 1 host
 * ints from 0 to n) and no entry may join two graphs (MM_ERR_GRAPH).  Each
 * graph is coloured and numbered in its own ids (v - offsets[i]), so its
 * slice of the result, and its round count, are exactly what a matching of
 * that graph alone with the same seeds would give.  mm_match_batch writes
 * d_match_out (n ints on the device, values in each graph's own numbering)
 * and rounds_out[i] per graph (host, ngraphs ints).  After set_batch, the
 * other match entries also number per graph and report the largest count.
 */
mm_status mm_graph_set_batch(mm_graph *g, int ngraphs, const int *offsets);
mm_status mm_match_batch(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                         int *d_match_out, int *rounds_out, void *stream);

/*
 * Learned colouring; no counterpart in the reference, whose select kernel
 * colours every vertex blue with the same probability (the barrier).  Here a
 * per-vertex MLP (6 -> 16 -> 1, ReLU, sigmoid) gives each vertex its own blue
 * probability from local features: log2(1 + degree), its role in the previous
 * round (0 red or first round, 0.5 blue without a proposal, 1 blue whose
 * proposal lost), max and mean weight it could pick, min(round, 32) / 32 and
 * level / 16 (the caller's coarsening level).  The probability is clamped to
 * [1/16, 15/16], so the maximal types finish inside the round cap whatever
 * the weights.  On graphs that take the symmetric path, from round 3 on, a
 * red vertex of at most 128 entries whose neighbours are all matched leaves in
 * that round (the reference waits until it is coloured blue); the matching is
 * the same as the one the same colours give without that.  mlp: MM_POLICY_FLOATS host
 * floats, W1[16][6], b1[16], W2[16], b2.  The result is a valid matching
 * (maximal for types 7, 9) but not the reference's: the reference's path is
 * mm_match.  d_trace (device, trace_rounds * n * 8 floats, or NULL) receives
 * for every vertex coloured in round r < trace_rounds, at [(r * n + v) * 8]:
 * its 6 features, its colour (1 blue, 0 red) and 1 if it left the active set
 * in that round (matched, or retired as unmatchable: match value 2); entries
 * of vertices not coloured keep their contents.  On a graph marked as a batch
 * (mm_graph_set_batch) every graph's slice is a valid matching of that graph
 * in its own numbering, and *rounds_out is the rounds of the whole launch.
 */
#define MM_POLICY_FLOATS 129
mm_status mm_match_policy(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                          const float *mlp, float level, int *d_match_out, int *rounds_out, float *d_trace,
                          int trace_rounds, void *stream);

/*
 * Weight and size of a matching, computed on the device exactly as
 * GraphMatching::getWeight does (src/matchcpu.cu:64-97): a matched vertex adds
 * the weight of the first entry of its list whose neighbour carries the same
 * match value, and counts one; weight is half the sum (double), size the
 * count of such vertices.  d_match: n ints on g's device.  The sum is taken in
 * a fixed tree, not the reference's vertex order: it agrees to rounding.
 */
mm_status mm_matching_weight(mm_graph *g, const int *d_match, double *weight, long long *size, void *stream);

/*
 * GraphMatching::testMatching (src/matchcpu.cu:127-246) on the device.
 * counts[0] under-matched (matched to themselves), [1] matched to more than
 * one vertex, [2] not matched to a neighbour, [3] can still be matched,
 * [4] unmatched; *valid = 1 iff counts[0..2] are all 0 (the reference's return
 * value: maximality is reported, not enforced).  The counts follow the
 * reference's walk over the vertices sorted by match value.  Where a value is
 * shared by three or more vertices, the reference's order among them is
 * std::sort's; here it is ascending id.
 */
mm_status mm_matching_check(mm_graph *g, const int *d_match, long long counts[5], int *valid, void *stream);

/*
 * One level of multilevel coarsening; no counterpart in the reference, which
 * stops at the matching.  Contracts each matched pair of d_match (n ints on
 * g's device, values 4 + min(v, partner) as mm_match writes them) into one
 * vertex; unmatched vertices stay.  Coarse vertex ids follow the smaller
 * member's id order.  The coarse lists hold the members' entries mapped to
 * coarse ids, in increasing id, without self-loops.  An edge that several fine
 * entries map to carries their weights' sum, taken in double and rounded once
 * (unit weights when g has none).  *coarse is a new graph on the same device,
 * to be freed with mm_graph_destroy.  d_cmap (n ints on the device, or NULL)
 * receives each vertex's coarse id.  A match array whose value names no
 * partner that names it back gives MM_ERR_ARG.
 */
mm_status mm_graph_contract(mm_graph *g, const int *d_match, mm_graph **coarse, int *d_cmap);

/*
 * Measurement entry, no counterpart in the reference: the device's rate of
 * random one-byte reads (2^27 gathers from a table of table_bytes bytes,
 * indices streamed coalesced), in gathers per second, best of four runs.
 * The round kernel's scans are bound by such reads rather than by streaming
 * bandwidth, so this is the ceiling their rate is reported against.
 */
mm_status mm_probe_gather_rate(int device, long long table_bytes, double *gathers_per_s);

/*
 * Testing hook, no counterpart in the reference: lets tests drive the library's
 * failure handling without any GPU fault.  Process-wide; not for production
 * use.  *out (may be NULL) receives the previous value, or the queried one.
 *   MM_DEBUG_SPIN_LIMIT    polls a grid-barrier wait of the round and finish
 *                          kernels makes before giving up (0: the default,
 *                          2^22); a wait that gives up makes the call return
 *                          MM_ERR_DEVICE
 *   MM_DEBUG_SKIP_BARRIER  mark of a grid barrier at which block 0 does not
 *                          arrive, so every wait on it runs out (-1: none);
 *                          marks: 0 after set-up, 3r + 1 after round r's
 *                          window scan, 3r + 3 after its commit
 *   MM_DEBUG_ALLOC_LIMIT   bytes in use in the device pool above which
 *                          allocations fail as out of memory (-1: none)
 *   MM_DEBUG_POOL_USED     query (value ignored): bytes in use in the current
 *                          device's pool, after synchronising the device
 */
enum {
    MM_DEBUG_SPIN_LIMIT = 1,
    MM_DEBUG_SKIP_BARRIER = 2,
    MM_DEBUG_ALLOC_LIMIT = 3,
    MM_DEBUG_POOL_USED = 4
};
mm_status mm_debug(int key, long long value, long long *out);

/* Message of the calling thread's most recent failure ("" if none). */
const char *mm_last_error(void);

/* Library version string. */
const char *mm_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MM_MATCH_H */
