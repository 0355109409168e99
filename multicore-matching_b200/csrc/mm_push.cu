// mm_push.cu -- the B200 round loop ("push" path).
//
// Same matching as the reference's GPU round (src/matchgpu.cu:184-451), with
// the work re-cut so that each round streams only the adjacency lists of BLUE
// vertices, and the whole loop runs in one cooperative kernel launch.
//
// Reformulation (exact, for any CSR the reference accepts):
//   * Respond (grRespond / gwRespond, matchgpu.cu:329-357, 411-451) lets red r
//     pick, among its blue neighbours u with requests[u] == r, the entry of its
//     own list with the largest weight (strict >, starting from -1), earliest
//     position first; in random mode the earliest position.  That is the
//     maximum over r's list of a 64-bit key (weight order << 32 | ~position),
//     restricted to entries pointing at proposers.  For every adjacency slot
//     (v -> r) the preparation step stores revkey = the best such key among
//     r's entries pointing back at v (0 if none can ever be picked).  A blue
//     proposer then atomicMax-es its revkey into best[r]; the maximum over
//     proposers equals the maximum over r's list.  Red vertices never scan.
//   * Commit (gMatch, matchgpu.cu:260-283): red r is matched iff best[r] is
//     non-zero (its partner is neighbours[~low32(key)]); blue u is matched iff
//     the low 32 bits of best[its target] equal the low 32 bits of its own
//     revkey (positions in r's list are unique).
//   * Select (gaSelect, matchgpu.cu:220-258) of round t+1 is fused into the
//     commit pass of round t: a survivor recolours itself with seed t+1.
//   * Dead marking (requests == n+1) happens as soon as the blue scan finds no
//     unmatched neighbour; readers of that colour byte see "unmatched, not red"
//     either way, so their outcome is unchanged.
//
// Work layout.  Vertices that can still be matched sit in worklists; an item
// carries the vertex, its neighbour range and its window offset, so the scans
// never read neighbourRanges again.
//   windows        a blue vertex's choice is the first red candidate among its
//                  best min(deg, 32) entries in order of preference (weight,
//                  then position; list order for random types), stored at
//                  preparation.  A lane holds one vertex and reads eight
//                  window entries a step, refilled from a prefetched item as
//                  soon as its vertex is decided (scan_window).
//   fallback       a list longer than its window with no red candidate in it
//                  is appended to the round's fallback list; that entry space
//                  is cut into 256-entry segments and a warp walks one segment
//                  in coalesced rows of 32 (scan_long).  A list cut by segment
//                  edges is combined by atomics and its last piece proposes.
//   finish phase   once the active set is small its components are tiny, and
//                  a second cooperative kernel plays the remaining rounds of
//                  each component on its own (k_finish), with no grid barrier.
// A list's best entry is kept as a 64-bit key (weight order << 32 | ~position),
// which orders ties by position exactly as the reference's strict ">" scan in
// list order does.
//
// Loop.  k_rounds is launched cooperatively (all blocks resident) and runs
// set-up, then per round the window scan (A1), the fallback scan (A2, only in
// rounds that have fallback lists) and the commit phase (B: commit + recolour
// + worklist compaction), with bounded grid barriers in between, until it
// hands over to the finish kernel.  Nothing returns to the host until the
// matching is maximal (the reference copies a flag back every round,
// matchgpu.cu:607-614), and no round pays for kernel launches.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cstddef>
#include <cmath>
#include <cstring>
#include <new>

#include "mm_common.cuh"

namespace mm {
namespace {

constexpr int kThreads = 512;            // threads per block of the round kernel
constexpr int kWarps = kThreads / 32;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kWin = 32;                 // preference window: the first min(deg, 32) choices
constexpr int kReqFallback = -3;         // reqi: the item's list went to the fallback scan
constexpr int kSegEntries = 256;         // entries per fallback segment: 8 rows of 32; at most 9
                                         // pieces of lists > 32 entries overlap one segment

// Worklists: blue and red vertices by round parity; the staged list holds the round's
// fallback lists (blue lists longer than the window with no red choice in
// it) with their offsets in the concatenated fallback entry space.
enum : int { kBlue = 0, kRed = 1, kParityLists = 2 };

struct Ctl {
    int *match;            // output array of this call
    uint32_t barrier;
    int cap;               // 20 or 255
    int maximal;
    int nseeds;
    int rounds;            // rounds the reference executes (set at loop exit)
    int status;            // 0 ok, 1 seeds exhausted, 2 a bounded grid-barrier wait gave up
    int cnt[2][kParityLists];      // worklist lengths by round parity
    unsigned long long staged_pack;  // fallback list of the round: (items << 32) | entries
    int retired[2];        // vertices of the round that were unmatchable as soon as coloured
    int fin_abort;         // finish phase: t + 1 if the attempt in round t was called off
    int fin_last;          // finish phase: last round in which any of its vertices was active
    int fin_round;         // finish phase: the round it starts at (set by k_rounds)
    int fin_state;         // finish phase: kFinState*
    long long active0;     // vertices active at round 0 (for a resumed round kernel)
    int iso_last;          // 1 + the last round in which a vertex without neighbours was active (0: none)
};

// Finish-phase hand-over between the launches of one matching.
enum : int { kFinStateNone = 0, kFinStatePending = 1, kFinStateDone = 2, kFinStateResume = 3 };

struct Params {
    int n;
    int contiguous;
    int sym;                        // proposal keys computed from the proposer's entry (no reverse index)
    const int2 *ranges;
    const int *nbrs;
    const float *w;
    const unsigned long long *revkey;
    const long long *slot_off;
    const int2 *pwin;               // weighted: preference windows {neighbour, position | flag or weight}
    int wwin;                       // pwin's second words are weights (symmetric weighted path)
    const long long *pwin_off;      // weighted: first window slot of each vertex (< 2^31)
    uint8_t *col;
    int2 *req;                      // per vertex: proposal of a fallback list (and the finish phase's item map)
    int2 *reqi;                     // per blue item of the round: {target, key low half}, -1 unmatchable,
                                    // -2 no proposal, kReqFallback: look in req
    unsigned long long *best;       // per red vertex: max proposal key this round
    unsigned long long *part_key;   // per cut fallback list: max over finished pieces
    int *part_cnt;                  // per cut fallback list: finished pieces
    int4 *lists[2][kParityLists];   // items {v, begin, end, window offset} by parity and colour
    int4 *staged;                   // fallback items {v, begin, end, entry offset}
    int *seg_first;                 // per fallback segment: item holding its first entry
    const uint32_t *seeds;
    Ctl *ctl;
    unsigned long long *stats;      // [kMaxRounds][MM_STATS_COLS] or null
    unsigned long long *tstamp;     // [3 * kMaxRounds + 1] barrier times (ns) or null
    unsigned *bar;                  // [kBarWords] grid barrier words, zero at launch
    int resume;                     // round kernel: continue from ctl->fin_round (finish called off)
    int zero_parts;                 // set-up clears part_key and part_cnt (not known to be zero)
    int fin_div;                    // finish phase from the round whose active set is <= 1/fin_div of round 0's (0: never)
    // testing hooks (mm_debug): polls before a barrier wait gives up, and the
    // mark of a barrier at which block 0 does not arrive (-1: none)
    long long spin_limit;
    int skip_mark;
    // A batch of independent graphs (a disjoint union, edges never cross): each
    // vertex's graph starts at vbase[v], and the graph's own numbering (v -
    // vbase[v]) drives the colouring and the match values, so every graph gets
    // the matching a call on it alone would give.  last[v] is the last round
    // at whose colouring v was still unmatched.  Both null for one graph.
    const int *vbase;
    uint8_t *last;
    // Learned colouring (k_rounds<..., kPolicy>): blue iff hash < p_v * 2^32 with
    // p_v from a per-vertex MLP over local features.  wfeat[v]: (max, mean)
    // incident weight; trace: per round and vertex, the features, colour and
    // outcome (for training), or null.
    float level;
    const float2 *wfeat;
    float *trace;
    int trace_rounds;
    // The policy's weights travel by value in the launch parameters: every
    // thread reads the same one, so the unrolled MLP takes them straight from
    // the constant bank as operands, with no load instruction per weight.
    float mlp[MM_POLICY_FLOATS];
    // A policy whose output weights are all zero ignores the features: its
    // threshold, computed once on the host, is policy_bar (policy_const = 1).
    int policy_const;
    uint32_t policy_bar;
    // Learned colouring with a constant policy: the finish phase plays the
    // remaining rounds under the policy's threshold and its retirement rule.
    int fin_retire;
};
static_assert(sizeof(Params) <= 4096, "launch parameters stay within the classic 4 KB limit");

template <class P>
__device__ __forceinline__ int base_of(const P &p, int v) { return p.vbase ? __ldg(p.vbase + v) : 0; }

__device__ __forceinline__ int degree_of(int2 r) { return r.y > r.x ? r.y - r.x : 0; }
__device__ __forceinline__ int degree_of(int4 it) { return it.z > it.y ? it.z - it.y : 0; }
__device__ __forceinline__ int win_len(int deg) { return deg < kWin ? deg : kWin; }

__device__ __forceinline__ int warp_incl_scan(int v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += y;
    }
    return v;
}

template <class P>
__device__ __forceinline__ void stat_add(const P &p, int round, int col, unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&p.stats[(size_t)round * MM_STATS_COLS + col], v);
}

// ---- grid barrier ----
//
// The round kernel is launched cooperatively, so all its blocks are resident
// at once and a barrier over them cannot deadlock on scheduling.  Blocks
// arrive in groups of kBarGroup on their group's word, and the last of each
// group arrives on the top word, which every block polls; each word sits in
// its own 128-byte line, so no word sees more than kBarGroup (or group-count)
// atomics per barrier.  Every word uses the same counting: the first member
// adds 2^31 - (members - 1), every other member adds 1, so the top bit flips
// exactly when the last member arrives and the low bits return to where they
// were.  Each wait is still bounded: after kSpinLimitDefault polls (a testing
// hook, mm_debug, can set fewer) the block records
// status 2 and the kernel returns; the other blocks then give up at their next
// barrier.  Thread 0's fences (release before arriving, acquire after the
// wait), with the block barriers around them, make every block's writes of
// the phase visible to every thread of every block afterwards.
constexpr int kBarGroup = 16;
constexpr int kBarStride = 32;   // words per barrier line (128 bytes)
constexpr int kBarMaxGroups = 64;
constexpr int kBarWords = (kBarMaxGroups + 1) * kBarStride;  // group words, then the top word

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __noinline__ bool grid_sync(unsigned *bar, Ctl *ctl, unsigned long long *tstamp, int mark,
                                       long long spin_limit, int skip_mark)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned nb = gridDim.x, b = blockIdx.x;
        const unsigned g = b / kBarGroup, ngroups = (nb + kBarGroup - 1) / kBarGroup;
        const unsigned gsize = min((unsigned)kBarGroup, nb - g * kBarGroup);
        unsigned *gword = bar + g * kBarStride;
        unsigned *top = bar + kBarMaxGroups * kBarStride;
        const unsigned top_before = ld_acquire(top);  // cannot flip before this block arrives
        fence_acq_rel();
        // testing hook: block 0 leaves this barrier out, so every wait on it runs out
        if (!(b == 0 && mark >= 0 && mark == skip_mark)) {
            const unsigned ginc = b % kBarGroup == 0 ? 0x80000000u - (gsize - 1u) : 1u;
            const unsigned gold = atomicAdd(gword, ginc);
            if (((gold + ginc) ^ gold) & 0x80000000u) {  // last of the group
                const unsigned tinc = g == 0 ? 0x80000000u - (ngroups - 1u) : 1u;
                atomicAdd(top, tinc);
            }
        }
        int ok = 1;
        long long it = 0;
        while (((top_before ^ ld_acquire(top)) & 0x80000000u) == 0u) {
            if (++it > spin_limit) {
                ok = 0;
                break;
            }
            if (it > 64) __nanosleep(32);
        }
        fence_acq_rel();
        if (!ok) atomicExch(&ctl->status, 2);
        s_ok = ok;
        if (tstamp && b == 0 && mark >= 0) tstamp[mark] = global_ns();
    }
    __syncthreads();
    return s_ok != 0;
}


// L2 residency: the colour bytes, which every scan reads at random, are loaded
// with an evict-last policy, the streamed worklists and requests with
// evict-first (.cs) loads and stores.
__device__ __forceinline__ unsigned long long pol_keep()
{
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint8_t ld_col(const uint8_t *a)
{
    unsigned short r;
    asm volatile("ld.global.L2::cache_hint.u8 %0, [%1], %2;" : "=h"(r) : "l"(a), "l"(pol_keep()));
    return (uint8_t)r;
}
// At the end of a matching the colour bytes go back to the normal eviction
// priority, so that they do not crowd the L2 of the work that follows.
template <class T>
__device__ __forceinline__ void release_lines(const T *a, long long count)
{
    const uintptr_t lo = (uintptr_t)a & ~(uintptr_t)127, hi = (uintptr_t)(a + count);
    const long long lines = (long long)((hi - lo + 127) / 128);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < lines; i += (long long)gridDim.x * blockDim.x)
        asm volatile("applypriority.global.L2::evict_normal [%0], 128;" ::"l"(lo + (uintptr_t)i * 128) : "memory");
}

// Key under which a blue vertex ranks a red neighbour at position j
// (gwRequest: strict > from -1, earliest j on ties; grRequest: earliest j).
// Every candidate key is >= 2^31, so the value 1 can stand for "an unmatched
// neighbour that is not a candidate" and a single max-reduction carries both
// the choice and the dead flag (0 = nothing unmatched seen).
template <bool kW>
__device__ __forceinline__ unsigned long long cand_key(int j, float w)
{
    if (kW) return w > -1.0f ? (((unsigned long long)weight_order(w) << 32) | (uint32_t)~j) : 1ull;
    return (unsigned long long)(uint32_t)~j;
}

// Scan result of one adjacency entry with neighbour colour c.
template <bool kW>
__device__ __forceinline__ unsigned long long entry_key(uint8_t c, int j, float w)
{
    if (c == kRed) return cand_key<kW>(j, w);
    return c == kMatched ? 0ull : 1ull;
}

// Key of a scan's best entry: weight order and position of its best red
// neighbour (the reference's rule: strict > from -1 in list order), else 1 if
// an unmatched neighbour was seen, else 0.
template <bool kW>
__device__ __forceinline__ unsigned long long strip_key(float bw, int bj, bool alive)
{
    if (bw > -1.0f) return kW ? (((unsigned long long)weight_order(bw) << 32) | (uint32_t)~bj)
                              : (unsigned long long)(uint32_t)~bj;
    return alive ? 1ull : 0ull;
}

// Fold one scanned entry (neighbour colour c, weight w, position j) into a
// lane's running best: strict > from -1 over increasing positions, so ties
// keep the earliest entry; in random mode the first red entry.
template <bool kW>
__device__ __forceinline__ void fold_entry(uint8_t c, float w, int j, float &bw, int &bj, bool &alive)
{
    alive |= c != kMatched;
    if (c == kRed) {
        const float x = kW ? w : 0.0f;
        if (x > bw) {
            bw = x;
            bj = j;
        }
    }
}

// Blue vertex v proposes to `target`, the neighbour at position j of its list
// (begin = first position): the reverse key of that slot goes to best[target].
template <bool kW>
__device__ __forceinline__ void propose_to(const Params &p, int2 *rq, int v, int begin, int j, int target)
{
    unsigned long long rk;
    if (p.sym) {
        // target's entry for v has v's weight, and earlier positions in its
        // strictly increasing list hold smaller ids
        if (kW) {
            const float x = __ldg(p.w + j);
            rk = x > -1.0f ? (((unsigned long long)weight_order(x) << 32) | (uint32_t)~v) : 0ull;
        } else {
            rk = (unsigned long long)(uint32_t)~v;
        }
    } else {
        const long long slot = p.contiguous ? (long long)j : __ldg(p.slot_off + v) + (j - begin);
        rk = __ldg(p.revkey + slot);
    }
    if (rk) atomicMax(&p.best[target], rk);
    __stcs(rq, make_int2(target, (int)(uint32_t)rk));
}

// Symmetric weighted path, windows carrying weights: blue v proposes to
// `target` through an entry of weight w (w > -1); the target's entry for v has
// the same weight, and v's id breaks ties (smaller first).
__device__ __forceinline__ void propose_weight(const Params &p, int2 *rq, int v, float w, int target)
{
    const unsigned long long rk = ((unsigned long long)weight_order(w) << 32) | (uint32_t)~v;
    atomicMax(&p.best[target], rk);
    __stcs(rq, make_int2(target, (int)(uint32_t)rk));
}

// Blue vertex v without a red choice: unmatchable if no neighbour is
// unmatched (requests == n + 1), else no proposal this round.
__device__ __forceinline__ void no_proposal(const Params &p, int2 *rq, int v, bool alive)
{
    if (!alive) {
        p.col[v] = kDead;
        p.ctl->match[v] = 2;
        __stcs(rq, make_int2(-1, 0));
    } else {
        __stcs(rq, make_int2(-2, 0));
    }
}

// Finish blue vertex v after a full scan whose result is `key`.
template <bool kW>
__device__ __forceinline__ void propose(const Params &p, int v, int begin, unsigned long long key)
{
    if (key < 2) {
        no_proposal(p, p.req + v, v, key == 1);
        return;
    }
    const int j = (int)~(uint32_t)key;
    propose_to<kW>(p, p.req + v, v, begin, j, __ldg(p.nbrs + j));
}

// Adjacency entries the reference's request loop inspects for this vertex
// (random mode stops at the first red neighbour, at position j).
template <bool kW>
__device__ __forceinline__ unsigned long long request_seen(int begin, int deg, int j)
{
    if (kW || j < 0) return (unsigned long long)deg;
    return (unsigned long long)(j - begin + 1);
}

template <bool kW, bool kStats>
__device__ __forceinline__ void propose_counted(const Params &p, int4 it, unsigned long long key, int t)
{
    if (kStats) {
        const int j = key >= 2 ? (int)~(uint32_t)key : -1;
        atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_REQ_ENTRIES], request_seen<kW>(it.y, degree_of(it), j));
        atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_BLUE_DEG], (unsigned long long)degree_of(it));
    }
    propose<kW>(p, it.x, it.y, key);
}

constexpr int kRows = 4;    // fallback scan: rows of 32 entries per iteration
constexpr int kStages = 3;  // fallback scan: iterations staged in shared memory (2 loading, 1 in use)

// Fallback-scan staging of one warp: neighbour ids and weights of kStages
// iterations, written by cp.async.
struct LongStage {
    int nb[kStages][kRows * 32];
    float w[kStages][kRows * 32];
};

// Shared memory of the round kernel (dynamic).
struct Smem {
    int delta[kWarps][33];                // fallback scan: global position of segment entry e = e + delta[k]
    int pend[kWarps][33];                 // fallback scan: segment-relative end of each piece
    LongStage stage[kWarps];
    int tile_warp[kWarps][2];             // compaction: per-warp counts, then offsets
    int tile_base[2];                     // compaction: tile bases
    uint32_t seeds[256];                  // the call's colouring seeds (finish phase)
    int wnext;                            // window scan: next item of the block's share
    int iso_n;                            // set-up: queued vertices without neighbours
    int iso_cnt[3];                       // set-up: survivors of a round of the queue (rotating)
    int stage_n;                          // window scan: fallback lists collected by the block
};

// window scan: fallback lists a block collects in its (then unused) staging area
constexpr int kStageCap = (int)(sizeof(LongStage) * kWarps / sizeof(int4));

// ---- learned colouring ----
//
// The policy is a 6 -> 16 -> 1 MLP (ReLU, sigmoid output) evaluated per vertex
// when it is coloured; its weights are a launch parameter, laid out as
// W1[16][6], b1[16], W2[16], b2.  Features: log2(1 + deg), the vertex's role
// in the previous round (0 red or first round, 0.5 blue without a proposal, 1
// blue whose proposal lost), max and mean incident weight, min(round, 32) /
// 32, level / 16.  The blue probability is clamped
// to [1/16, 15/16] and compared with the colouring hash like the select
// barrier: an unmatched edge then splits blue/red in at least 11.7% of the
// rounds, so the maximal types finish well inside the 255-round cap whatever
// the weights (a pair left alone survives 255 rounds with p < 1e-13).
constexpr int kFeat = 6, kHid = 16;
static_assert(kHid * kFeat + kHid + kHid + 1 == MM_POLICY_FLOATS, "policy layout");
constexpr int kTraceCols = 8;  // features, colour (1 blue, 0 red), left the active set in that round
constexpr int kRetireFrom = 3;      // learned colouring: first round in which red vertices retire
constexpr int kRetireMaxDeg = 128;  // learned colouring: longest list a red vertex checks

// Trace: vertex v left the active set in round t (matched, or blue with no
// unmatched neighbour and so retired).
template <bool kPolicy>
__device__ __forceinline__ void trace_left(const Params &p, int t, int v)
{
    if (kPolicy && p.trace && t < p.trace_rounds) p.trace[((size_t)t * p.n + v) * kTraceCols + kFeat + 1] = 1.0f;
}

__device__ __forceinline__ void policy_features(const Params &p, float2 wf, int deg, float role, int t,
                                                float (&x)[kFeat])
{
    x[0] = __log2f(1.0f + (float)deg);
    x[1] = role;
    x[2] = wf.x;
    x[3] = wf.y;
    x[4] = (float)min(t, 32) * (1.0f / 32.0f);
    x[5] = p.level * (1.0f / 16.0f);
}

__device__ __forceinline__ uint32_t policy_barrier(const Params &p, const float (&x)[kFeat])
{
    constexpr int kB1 = kHid * kFeat, kW2 = kB1 + kHid, kB2 = kW2 + kHid;
    float out = p.mlp[kB2];
#pragma unroll
    for (int j = 0; j < kHid; ++j) {
        float a = p.mlp[kB1 + j];
#pragma unroll
        for (int i = 0; i < kFeat; ++i) a = fmaf(p.mlp[j * kFeat + i], x[i], a);
        out = fmaf(p.mlp[kW2 + j], fmaxf(a, 0.0f), out);
    }
    float prob = 1.0f / (1.0f + __expf(-out));
    prob = fminf(fmaxf(prob, 1.0f / 16.0f), 15.0f / 16.0f);
    return (uint32_t)(prob * 4294967296.0f);
}

// Colour of vertex v for round t: the select barrier, or the policy's.
// Whether colouring round t needs the features: a policy that ignores them
// needs them only for the trace.
__device__ __forceinline__ bool policy_needs_features(const Params &p, int t)
{
    return !p.policy_const || (p.trace && t < p.trace_rounds);
}

template <bool kPolicy>
__device__ __forceinline__ bool colour_blue(const Params &p, int v, int deg, float role, float2 wf, int t,
                                            uint32_t seed, uint32_t barrier)
{
    uint32_t bar = barrier;
    if (kPolicy) {
        float x[kFeat];
        if (policy_needs_features(p, t)) policy_features(p, wf, deg, role, t, x);
        bar = p.policy_const ? p.policy_bar : policy_barrier(p, x);
        const bool blue = colour_of((uint32_t)(v - base_of(p, v)), seed, bar) == kBlue;
        if (p.trace && t < p.trace_rounds) {
            float *row = p.trace + ((size_t)t * p.n + v) * kTraceCols;
#pragma unroll
            for (int i = 0; i < kFeat; ++i) row[i] = x[i];
            row[kFeat] = blue ? 1.0f : 0.0f;
            row[kFeat + 1] = 0.0f;
        }
        return blue;
    }
    return colour_of((uint32_t)(v - base_of(p, v)), seed, bar) == kBlue;
}

// ---- worklist compaction for the set-up and commit passes ----
//
// A block handles tiles of kTileItems vertices, kPer per thread.  Each thread
// decides the next list of its vertices; the block counts them per list with
// warp scans, takes one atomic per list and tile, and writes its items.

constexpr int kPer = 4;
constexpr int kTileItems = kThreads * kPer;

// dest[k]: -1 (drop), kBlue or kRed.
__device__ __forceinline__ void compact_tile(const Params &p, Smem &sm, int parity, const int (&dest)[kPer],
                                             const int4 (&item)[kPer])
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int c[2] = {0, 0};
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        c[0] += dest[k] == kBlue;
        c[1] += dest[k] == kRed;
    }
    int ex[2];
#pragma unroll
    for (int l = 0; l < 2; ++l) {
        const int incl = warp_incl_scan(c[l]);
        ex[l] = incl - c[l];
        if (lane == 31) sm.tile_warp[warp][l] = incl;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        const int l = threadIdx.x;
        int run = 0;
        for (int w = 0; w < kWarps; ++w) {
            const int x = sm.tile_warp[w][l];
            sm.tile_warp[w][l] = run;
            run += x;
        }
        sm.tile_base[l] = run ? atomicAdd(&p.ctl->cnt[parity][l], run) : 0;
    }
    __syncthreads();
    int rc[2] = {0, 0};
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const int l = dest[k];
        if (l < 0) continue;
        const int idx = l == kBlue ? sm.tile_base[0] + sm.tile_warp[warp][0] + ex[0] + rc[0]++
                                   : sm.tile_base[1] + sm.tile_warp[warp][1] + ex[1] + rc[1]++;
        __stcs(&p.lists[parity][l][idx], item[k]);
    }
    __syncthreads();  // tile_warp / tile_base are reused by the next tile
}

// Vertices without neighbours on the symmetric path: no list names them, so
// nothing depends on them but their own match value and the round count.  One
// leaves (match value 2) in the first round in which it is blue, or stays red
// to the cap (match value 1).  The set-up queues the ones red in round 0 in
// shared memory and resolves the queue round by round, a hash per queued
// vertex and round (a walk per thread would cost every lane its warp's longest
// walk); a vertex that finds the queue full stays in the rounds, which give it
// the same fate.  iso_last: the last round in which any of them is active (the cap's
// last round if one stays red to it, nseeds if the seeds run out first: the
// reference would draw more, and the round count then exceeds nseeds).
constexpr int kIsoHalf = (int)(sizeof(LongStage) * kWarps / sizeof(int) / 2);  // queue capacity (two halves)

// Called by the whole block once, after the set-up's last tile (whose
// compaction ends with a barrier, after the last append).
// Round r reads the queue half qa and appends its survivors to the other,
// counting them in iso_cnt[r % 3]: that counter is cleared by thread 0 in
// round r - 1, after every thread read it (in round r - 3's closing step) and
// before any thread appends to it, so one barrier a round suffices.
__device__ void resolve_isolated(const Params &p, Smem &sm, int &iso_last)
{
    const Ctl *ctl = p.ctl;
    int *qa = reinterpret_cast<int *>(&sm.stage[0]), *qb = qa + kIsoHalf;
    const int cap = ctl->cap, lim = min(cap, ctl->nseeds);
    const uint32_t barrier = ctl->barrier;
    int nq = min(sm.iso_n, kIsoHalf);
    if (threadIdx.x == 0) sm.iso_cnt[1] = 0;
    __syncthreads();
    for (int r = 1; nq > 0; ++r) {
        int *cnt = &sm.iso_cnt[r % 3];
        if (threadIdx.x == 0) sm.iso_cnt[(r + 1) % 3] = 0;
        for (int i = threadIdx.x; i < nq; i += kThreads) {
            const int v = qa[i];
            if (r >= lim) {
                // red in every round up to the limit
                p.ctl->match[v] = 1;
                if (p.last) p.last[v] = (uint8_t)(cap - 1);
                iso_last = max(iso_last, lim == cap ? cap - 1 : lim);
            } else if (colour_of((uint32_t)(v - base_of(p, v)), p.seeds[r], barrier) == kBlue) {
                p.ctl->match[v] = 2;
                if (p.last) p.last[v] = (uint8_t)r;
                iso_last = max(iso_last, r);
            } else {
                qb[atomicAdd(cnt, 1)] = v;
            }
        }
        __syncthreads();  // the survivors and their count are complete
        nq = r >= lim ? 0 : *cnt;
        int *x = qa;
        qa = qb;
        qb = x;
    }
    __syncthreads();  // every thread has left the loop before the queue is emptied
    if (threadIdx.x == 0) sm.iso_n = 0;
    __syncthreads();
}

// Set-up: colour every vertex with seeds[0] and fill the first worklists.
// best[] starts at 0 and stays 0 for every vertex that is not matched: a red
// vertex that receives a proposal is matched in the same round.  On the
// symmetric path the vertices without neighbours are resolved here, whatever
// their colour (resolve_isolated); the instrumented kernel keeps them in the
// rounds, whose per-round counters count them as the reference does.
template <bool kW, bool kStats, bool kPolicy>
__device__ void init_phase(const Params &p, Smem &sm)
{
    const Ctl *ctl = p.ctl;
    const uint32_t seed = p.seeds[0], barrier = ctl->barrier;
    const int n = p.n;
    int iso_last = -1;
    if (threadIdx.x == 0) sm.iso_n = 0;
    __syncthreads();
    const int ntiles = (n + kTileItems - 1) / kTileItems;
    // each tile's ranges and window offsets are loaded while the tile before
    // it is coloured and compacted
    int2 rr[kPer];
    long long wo[kPer];
    auto fetch = [&](int tile) {
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const int v = tile * kTileItems + k * kThreads + threadIdx.x;
            rr[k] = make_int2(0, 0);
            wo[k] = 0;
            if (tile < ntiles && v < n) {
                rr[k] = __ldg(p.ranges + v);
                if (kW) wo[k] = __ldg(p.pwin_off + v);
            }
        }
    };
    fetch(blockIdx.x);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int dest[kPer];
        int4 item[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) item[k] = make_int4(tile * kTileItems + k * kThreads + threadIdx.x, rr[k].x, rr[k].y, (int)wo[k]);
        fetch(tile + gridDim.x);
        unsigned long long act = 0, blue_n = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const int v = item[k].x;
            dest[k] = -1;
            if (v < n) {
                int slot;
                const int deg = degree_of(item[k]);
                const float2 wf = kPolicy && policy_needs_features(p, 0) ? __ldg(p.wfeat + v) : make_float2(0.0f, 0.0f);
                const bool blue = colour_blue<kPolicy>(p, v, deg, 0.0f, wf, 0, seed, barrier);
                if (p.last) p.last[v] = 0;
                p.best[v] = 0ull;
                // (every completed round leaves them zero: a cut list's last piece clears them)
                if (deg > kWin && p.zero_parts) {
                    p.part_key[v] = 0ull;
                    p.part_cnt[v] = 0;
                }
                ++act;
                blue_n += blue;
                // no neighbours: unmatchable as soon as it is blue (learned
                // colouring on the symmetric path: at once, whatever its colour;
                // elsewhere another list may still name it, and a blue vertex
                // there must keep seeing it red)
                if ((blue || (kPolicy && p.sym)) && deg == 0) {
                    p.col[v] = kDead;
                    p.ctl->match[v] = 2;
                    trace_left<kPolicy>(p, 0, v);
                } else if (!kPolicy && !kStats && p.sym && deg == 0 &&
                           (slot = atomicAdd(&sm.iso_n, 1)) < kIsoHalf) {
                    // red in round 0: queued, resolved with the block's others (a
                    // vertex that finds the queue full stays in the rounds)
                    p.col[v] = kDead;
                    reinterpret_cast<int *>(&sm.stage[0])[slot] = v;
                } else {
                    p.col[v] = blue ? kBlue : kRed;
                    dest[k] = blue ? kBlue : kRed;
                }
            }
        }
        if (kStats) {
            stat_add(p, 0, MM_ST_ACTIVE, act);
            stat_add(p, 0, MM_ST_BLUE, blue_n);
            stat_add(p, 0, MM_ST_RED, act - blue_n);
        }
        compact_tile(p, sm, 0, dest, item);
    }
    if (!kPolicy && !kStats) {
        if (sm.iso_n > 0) resolve_isolated(p, sm, iso_last);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) iso_last = max(iso_last, __shfl_xor_sync(kFull, iso_last, o));
        if ((threadIdx.x & 31) == 0 && iso_last >= 0) atomicMax(&p.ctl->iso_last, iso_last + 1);
    }
}

// ---- phase A1: preference windows ----
//
// A blue vertex picks the entry the reference's request loop would pick
// (gwRequest: the heaviest red neighbour, strict > from -1, earliest position
// on ties; grRequest: the first red neighbour in list order).  Its candidates
// in that order of preference are its window: for weighted types the
// preparation step sorts each list's best min(deg, 32) entries by (weight,
// earlier position) into pwin, with entries whose weight can never be picked
// (<= -1 or NaN) flagged and last; for random types the window is simply the
// first min(deg, 32) entries of the list.  So the first red candidate in the
// window is the reference's choice, and the scan stops there.  A list that
// fits in its window and has no red candidate is decided too (unmatchable iff
// no entry is unmatched).  A longer list with no red candidate in its window
// falls back to a full scan in phase A2: it is appended to the round's
// fallback list.

// Learned colouring, graphs with symmetric structure: a red vertex of at most
// kRetireMaxDeg entries whose neighbours are all matched leaves in phase A of
// this round, while the blue vertices scan (the reference waits until it is
// coloured blue and scans).  Colours do not change during phase A, so the
// check is exact, and no vertex reads the retired one's colour: every vertex
// that lists it is its neighbour, hence matched, and matched vertices do not
// scan.  (Without symmetry an unmatched blue vertex could list it, and its
// choice would depend on the timing of the retirement.)  Red items are taken
// from the top of the thread range down, so on small rounds they run on
// threads that have no blue item.  Each list is read 16 entries at a time,
// each batch's colour loads in flight together, stopping after the first batch
// with an unmatched neighbour (most lists fit the first batch).  A limit of
// 128 entries cut R-MAT rounds further than 32 did; 512 cut no more and cost
// time.  A retired vertex's worklist item is marked with its id complemented,
// so the commit phase sees the retirement in the item it loads anyway.
template <bool kPolicy>
__device__ __forceinline__ void retire_red(const Params &p, int t, int par, int n_red)
{
    int4 *list = p.lists[par][kRed];
    const long long stride = (long long)gridDim.x * kThreads;
    const long long tid = stride - 1 - ((long long)blockIdx.x * kThreads + threadIdx.x);
    for (long long i = tid; i < n_red; i += stride) {
        const int4 it = __ldcg(list + i);
        if (degree_of(it) > kRetireMaxDeg) continue;
        bool gone = true;
        {
            int nb[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) nb[u] = it.y + u < it.z ? __ldg(p.nbrs + it.y + u) : -1;
#pragma unroll
            for (int u = 0; u < 16; ++u)
                if (nb[u] >= 0 && p.col[nb[u]] != kMatched) gone = false;
        }
        for (int j0 = it.y + 16; gone && j0 < it.z; j0 += 16) {
            int nb[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) nb[u] = j0 + u < it.z ? __ldg(p.nbrs + j0 + u) : -1;
#pragma unroll
            for (int u = 0; u < 16; ++u)
                if (nb[u] >= 0 && p.col[nb[u]] != kMatched) gone = false;
        }
        if (gone) {
            p.col[it.x] = kDead;
            p.ctl->match[it.x] = 2;
            list[i].x = ~it.x;
            trace_left<kPolicy>(p, t, it.x);
        }
    }
}

// The end of a blue vertex's window scan: propose to the red candidate found,
// or decide "no proposal" / "unmatchable" for a list that fits its window, or
// stage a longer list with no red candidate in its window for the fallback scan.
template <bool kW, bool kStats>
__device__ __forceinline__ void window_done(const Params &p, Smem &sm, int t, long long i, int4 it, bool found, int cj,
                                            int ct, bool alive, int seen)
{
    Ctl *ctl = p.ctl;
    const int v = it.x, deg = degree_of(it);
    if (kStats) atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_WINDOW_ENTRIES], (unsigned long long)seen);
    if (found || deg <= kWin) {
        if (kStats) {
            atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_REQ_ENTRIES],
                      request_seen<kW>(it.y, deg, found ? cj : -1));
            atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_BLUE_DEG], (unsigned long long)deg);
        }
        if (found) {
            if (kW && p.wwin) propose_weight(p, p.reqi + i, v, __int_as_float(cj), ct);
            else propose_to<kW>(p, p.reqi + i, v, it.y, cj & 0x7fffffff, ct);
        } else {
            no_proposal(p, p.reqi + i, v, alive);
        }
    } else {
        // the fallback scan proposes through req[v]
        p.reqi[i] = make_int2(kReqFallback, 0);
        // fallback: the whole list is scanned in phase A2.  The block collects
        // its fallback lists in shared memory and appends them to the round's
        // list at the end of the phase, with one global atomic; only a list
        // that finds the block's buffer full is appended at once.
        const int slot = atomicAdd(&sm.stage_n, 1);
        if (slot < kStageCap) {
            reinterpret_cast<int4 *>(&sm.stage[0])[slot] = make_int4(v, it.y, it.z, 0);
            return;
        }
        const unsigned long long old = atomicAdd(&ctl->staged_pack, (1ull << 32) | (unsigned long long)(unsigned)deg);
        const int idx = (int)(old >> 32), off = (int)(old & 0xffffffffull);
        p.staged[idx] = make_int4(v, it.y, it.z, off);
        for (int s = (off + kSegEntries - 1) / kSegEntries; s * kSegEntries < off + deg; ++s) p.seg_first[s] = idx;
    }
}

// Window entries q and q + 1 of a blue vertex (item it, window length wl):
// neighbours and second words (weight, position | flag, or position).
template <bool kW>
__device__ __forceinline__ void window_pair(const Params &p, int4 it, int wl, int q, int &n0, int &j0, int &n1, int &j1)
{
    n0 = n1 = 0;
    j0 = j1 = 0;
    if (q >= wl) return;
    if (kW) {
        const int4 x = __ldg(reinterpret_cast<const int4 *>(p.pwin + it.w + q));
        n0 = x.x;
        j0 = x.y;
        n1 = x.z;
        j1 = x.w;
    } else {
        j0 = it.y + q;
        j1 = j0 + 1;
        n0 = __ldg(p.nbrs + j0);
        if (q + 1 < wl) n1 = __ldg(p.nbrs + j1);
    }
}

// Whether a window entry's neighbour colour c and second word j make it the
// vertex's choice (a red candidate): on the symmetric weighted path j is the
// weight; elsewhere for weighted types the position, bit 31 set for a weight
// that can never be picked; random types: the position.
template <bool kW>
__device__ __forceinline__ bool window_choice(const Params &p, uint8_t c, int j)
{
    return c == kRed && (!kW || (p.wwin ? __int_as_float(j) > -1.0f : j >= 0));
}

// Phase A1.  Each block takes an equal share of the round's blue items, in
// chunks of kScanChunk interleaved with the other blocks' (ids, and with them
// degrees, cluster in the worklists: on R-MAT graphs the hubs have small ids),
// and hands them to its warps 32 at a time from a counter in shared memory.  A lane
// holds one vertex at a time and reads its window eight entries a step (four
// 16-byte loads, then the eight colours); as soon as a lane's vertex is decided it
// swaps in the item it prefetched and prefetches the next, so every lane keeps
// an independent chain of loads in flight and no lane waits for the slowest
// vertex of its warp or block.  Block barriers come only before the scan (the
// counter) and after it (the block's fallback lists are appended at once).
constexpr int kScanChunk = 64;

template <bool kW, bool kStats, bool kPolicy>
__device__ void scan_window(const Params &p, Smem &sm, int t, int par)
{
    Ctl *ctl = p.ctl;
    const int n_blue = __ldcg(&ctl->cnt[par][kBlue]);
    const int n_red = kPolicy ? __ldcg(&ctl->cnt[par][kRed]) : 0;  // read with n_blue: one round trip
    const int4 *list = p.lists[par][kBlue];
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    // this block's items: chunk c of its share is chunk c * gridDim.x + blockIdx.x of the list
    const long long span = (long long)gridDim.x * kScanChunk;
    const long long full = n_blue / span, rest = n_blue - full * span;
    const int bhi = (int)(full * kScanChunk + min((long long)kScanChunk, max(0ll, rest - (long long)blockIdx.x * kScanChunk)));
    if (threadIdx.x == 0) {
        sm.wnext = 0;
        sm.stage_n = 0;
    }
    __syncthreads();
    bool dry = bhi == 0;  // warp-uniform: the block's share is handed out
    // Items for the lanes in `mask`: one shared atomic per warp.  Returns this
    // lane's item index in the list, or -1.
    auto grab = [&](unsigned mask) -> long long {
        const int leader = __ffs(mask) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&sm.wnext, __popc(mask));
        base = __shfl_sync(kFull, base, leader);
        dry = base + __popc(mask) >= bhi;
        const int k = base + __popc(mask & below);
        if (!((mask >> lane) & 1u) || k >= bhi) return -1;
        return (long long)(k / kScanChunk) * span + (long long)blockIdx.x * kScanChunk + k % kScanChunk;
    };
    // the lane's vertex and its prefetched next, with their item indices
    int4 cur = make_int4(-1, 0, 0, 0), nxt = make_int4(-1, 0, 0, 0);
    int ci = -1, ni = -1;  // item indices (a list holds at most n < 2^31 items)
    if (!dry) {
        ci = (int)grab(kFull);
        if (ci >= 0) cur = __ldcs(list + ci);
    }
    if (!dry) {
        ni = (int)grab(kFull);
        if (ni >= 0) nxt = __ldcs(list + ni);
    }
    bool has = cur.x >= 0, alive = false;
    int q = 0, wl = has ? win_len(degree_of(cur)) : 0;
    while (__any_sync(kFull, has)) {
        if (has) {
            // eight entries a step (one dependent round trip for each 8: the scan
            // is bound by the latency of its load chains); the first step of
            // round 0, where most vertices stop at their first or second entry,
            // reads four
            const int width = q == 0 && t == 0 ? 4 : 8;
            int nb[8], jv[8];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                nb[2 * h] = nb[2 * h + 1] = jv[2 * h] = jv[2 * h + 1] = 0;
                if (2 * h < width) window_pair<kW>(p, cur, wl, q + 2 * h, nb[2 * h], jv[2 * h], nb[2 * h + 1], jv[2 * h + 1]);
            }
            uint8_t c[8];
#pragma unroll
            for (int x = 0; x < 8; ++x) c[x] = x < width && q + x < wl ? ld_col(p.col + nb[x]) : (uint8_t)kMatched;
            bool found = false;
            int cj = -1, ct = 0, seen = q;
#pragma unroll
            for (int x = 0; x < 8; ++x) {
                if (x >= width || q + x >= wl || found) continue;
                seen = q + x + 1;
                if (window_choice<kW>(p, c[x], jv[x])) {
                    found = true;
                    cj = jv[x];
                    ct = nb[x];
                } else {
                    alive |= c[x] != kMatched;
                }
            }
            q += width;
            if (found || q >= wl) {
                window_done<kW, kStats>(p, sm, t, ci, cur, found, cj, ct, alive, seen);
                has = false;
            }
        }
        // lanes whose vertex is decided take their prefetched item and prefetch the next
        const unsigned need = __ballot_sync(kFull, !has && nxt.x >= 0);
        if (need) {
            if (!has && nxt.x >= 0) {
                cur = nxt;
                ci = ni;
                nxt.x = -1;
                has = true;
                alive = false;
                q = 0;
                wl = win_len(degree_of(cur));
            }
            if (!dry) {
                const int i = (int)grab(need);
                if (i >= 0) {
                    nxt = __ldcs(list + i);
                    ni = i;
                }
            }
        }
    }
    // append the block's fallback lists: one atomic for the block, item
    // offsets by a block-wide prefix sum of their lengths
    __syncthreads();
    const int ns = min(sm.stage_n, kStageCap);
    if (ns > 0) {
        const int4 *buf = reinterpret_cast<const int4 *>(&sm.stage[0]);
        const int warp = threadIdx.x >> 5;
        const int per = (ns + kThreads - 1) / kThreads;
        const int lo = min(ns, (int)threadIdx.x * per), hi = min(ns, lo + per);
        int s = 0;
        for (int i = lo; i < hi; ++i) s += degree_of(buf[i]);
        const int incl = warp_incl_scan(s);
        if (lane == 31) sm.tile_warp[warp][0] = incl;
        __syncthreads();
        if (threadIdx.x == 0) {
            int run = 0;
            for (int w = 0; w < kWarps; ++w) {
                const int x = sm.tile_warp[w][0];
                sm.tile_warp[w][0] = run;
                run += x;
            }
            const unsigned long long old =
                atomicAdd(&ctl->staged_pack, ((unsigned long long)ns << 32) | (unsigned long long)(unsigned)run);
            sm.tile_base[0] = (int)(old >> 32);
            sm.tile_base[1] = (int)(old & 0xffffffffull);
        }
        __syncthreads();
        int off = sm.tile_base[1] + sm.tile_warp[warp][0] + incl - s;
        for (int i = lo; i < hi; ++i) {
            const int4 it = buf[i];
            const int idx = sm.tile_base[0] + i, deg = degree_of(it);
            p.staged[idx] = make_int4(it.x, it.y, it.z, off);
            for (int sg = (off + kSegEntries - 1) / kSegEntries; sg * kSegEntries < off + deg; ++sg) p.seg_first[sg] = idx;
            off += deg;
        }
        __syncthreads();  // the buffer and the tile words are reused
    }
    if (kPolicy && p.sym && t >= kRetireFrom) retire_red<kPolicy>(p, t, par, n_red);
}

// ---- phase A2: fallback lists, entry-balanced segments ----
//
// The round's fallback lists are concatenated (each item's .w is its offset)
// and cut into kSegEntries-entry segments; seg_first[s] is the first item
// overlapping segment s.  Items are numbered in offset order: one 64-bit
// atomic hands out both.  A warp takes a segment: lane l describes the l-th
// list piece in it (at most 9), then the warp walks the segment in rows of
// 32 consecutive entries.  Every piece but the segment's first and last is a
// whole list of more than 32 entries, so a row holds at most one piece
// boundary and the piece being scanned is the same for the whole warp: each
// lane keeps a running best (weight, position, alive) for it, and at the
// boundary the warp max-reduces the lanes' keys with shuffles and the lane
// describing the piece finishes it.  A list inside one segment proposes at
// once; a cut list max-combines its piece into part_key and the piece that
// arrives last proposes.
//
// Loads are pipelined over iterations of kRows rows: the neighbour ids and
// weights of iteration i+2 stream into shared memory (cp.async, kStages
// buffers) and the colour gathers of iteration i+1 are in flight while
// iteration i is folded.
template <bool kW, bool kStats>
__device__ __forceinline__ void finish_piece(const Params &p, int4 it, int pieces, unsigned long long key, int t)
{
    if (pieces == 1) {
        propose_counted<kW, kStats>(p, it, key, t);
        return;
    }
    const int v = it.x;
    if (key) atomicMax(&p.part_key[v], key);
    // acq_rel: this piece's max is visible before its arrival counts, and the
    // last arrival sees every other piece's max
    int done;
    asm volatile("atom.add.acq_rel.gpu.s32 %0, [%1], 1;" : "=r"(done) : "l"(p.part_cnt + v) : "memory");
    if (done == pieces - 1) {
        const unsigned long long all = atomicExch(&p.part_key[v], 0ull);
        atomicExch(&p.part_cnt[v], 0);
        propose_counted<kW, kStats>(p, it, all, t);
    }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async4_s(unsigned saddr, const void *gmem)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(saddr), "l"(gmem) : "memory");
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long k)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync(kFull, k, o);
        k = y > k ? y : k;
    }
    return k;
}

// Finish piece k of the segment table: lane k holds its item.
template <bool kW, bool kStats>
__device__ __forceinline__ void finish_table_piece(const Params &p, int k, int lane, int4 it, int pieces, int lo, int hi,
                                                   unsigned long long key, int t)
{
    if (lane == k) {
        if (kStats) {
            atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_STAGED_DEG], (unsigned long long)(hi - lo));
            atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_STAGED_ITEMS], 1ull);
        }
        finish_piece<kW, kStats>(p, it, pieces, key, t);
    }
}

template <bool kW, bool kStats>
__device__ void scan_long(const Params &p, Smem &sm, int t, int gwarp, int nwarps)
{
    const unsigned long long pack = __ldcg(&p.ctl->staged_pack);
    const int nitems = (int)(pack >> 32);
    const int nentries = (int)(pack & 0xffffffffull);
    const int nseg = (nentries + kSegEntries - 1) / kSegEntries;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int *pend = sm.pend[warp];
    int *delta = sm.delta[warp];
    LongStage &stg = sm.stage[warp];
    // shared addresses of this lane's slots in stage 0 (stage k: + k * kStageBytes)
    constexpr unsigned kStageBytes = kRows * 32 * 4;
    const unsigned nb_slot = (unsigned)__cvta_generic_to_shared(&stg.nb[0][lane]);
    const unsigned w_slot = (unsigned)__cvta_generic_to_shared(&stg.w[0][lane]);
    const int4 *list = p.staged;
    const int *seg_first = p.seg_first;
    // the piece table of segment s + nwarps is loaded while segment s is
    // scanned: seg_first two segments ahead, the items one segment ahead
    int sf_a = gwarp < nseg ? __ldcg(seg_first + gwarp) + lane : nitems;
    int sf_b = gwarp + nwarps < nseg ? __ldcg(seg_first + gwarp + nwarps) + lane : nitems;
    int4 x_a = sf_a < nitems ? __ldcg(list + sf_a) : make_int4(-1, 0, 0, -1);
    for (int s = gwarp; s < nseg; s += nwarps) {
        const int s_lo = s * kSegEntries;
        const int seg_len = min(kSegEntries, nentries - s_lo);
        const int idx = sf_a;
        const int4 x = x_a;
        x_a = sf_b < nitems ? __ldcg(list + sf_b) : make_int4(-1, 0, 0, -1);
        sf_a = sf_b;
        sf_b = s + 2 * nwarps < nseg ? __ldcg(seg_first + s + 2 * nwarps) + lane : nitems;
        int4 it = make_int4(-1, 0, 0, 0);
        int pieces = 1, lo = 0, hi = 0;
        if (idx < nitems) {
            const int deg = degree_of(x);
            if (x.w < s_lo + seg_len && x.w + deg > s_lo) {
                it = x;
                lo = max(x.w, s_lo) - x.w;
                hi = min(x.w + deg, s_lo + seg_len) - x.w;
                pieces = (x.w + deg - 1) / kSegEntries - x.w / kSegEntries + 1;
            }
        }
        pend[lane] = it.x >= 0 ? it.w + hi - s_lo : 0x7fffffff;
        if (lane == 0) pend[32] = 0x7fffffff;
        delta[lane] = it.y - it.w + s_lo;
        if (lane == 0) delta[32] = 0;
        __syncwarp();
        const int nit = (seg_len + 32 * kRows - 1) / (32 * kRows);
        // Load side: piece kl holds the first entry of the row being staged;
        // its end and the position offsets of kl and kl + 1 stay in registers.
        int kl = 0, endl = pend[0], dl0 = delta[0], dl1 = delta[1];
        int stage_in = 0;  // stage that iteration i + 2 is staged into
        auto issue = [&](int i) {
            if (i < nit) {
                const unsigned so = (unsigned)stage_in * kStageBytes;
#pragma unroll
                for (int r = 0; r < kRows; ++r) {
                    const int rb = i * 32 * kRows + r * 32;
                    if (rb < seg_len) {
                        while (endl <= rb) {
                            ++kl;
                            endl = pend[kl];
                            dl0 = dl1;
                            dl1 = delta[kl + 1];
                        }
                        const int e = rb + lane;
                        if (e < seg_len) {
                            const int pos = e + (e >= endl ? dl1 : dl0);
                            cp_async4_s(nb_slot + so + r * 128, p.nbrs + pos);
                            if (kW) cp_async4_s(w_slot + so + r * 128, p.w + pos);
                        }
                    }
                }
            }
            cp_async_commit();
            stage_in = stage_in == kStages - 1 ? 0 : stage_in + 1;
        };
        // colours of iteration i (staged in stage st), one byte per row
        auto gather = [&](int i, int st) -> unsigned {
            unsigned c = 0x03030303u;  // kMatched in every row
            if (i < nit) {
#pragma unroll
                for (int r = 0; r < kRows; ++r) {
                    const int e = i * 32 * kRows + r * 32 + lane;
                    if (e < seg_len) {
                        const unsigned x = ld_col(p.col + stg.nb[st][r * 32 + lane]);
                        c = (c & ~(0xffu << (8 * r))) | (x << (8 * r));
                    }
                }
            }
            return c;
        };
        issue(0);
        issue(1);
        cp_async_wait1();
        unsigned cc = gather(0, 0);
        // Fold side: piece kp, its end and the offsets of kp and kp + 1.
        int kp = 0, endp = pend[0], dp0 = delta[0], dp1 = delta[1];
        int st = 0;  // stage of iteration i
        float bw = -1.0f;
        int bj = 0;
        bool alive = false;
        for (int i = 0; i < nit; ++i) {
            issue(i + 2);
            cp_async_wait1();
            const int st1 = st == kStages - 1 ? 0 : st + 1;
            const unsigned cn = gather(i + 1, st1);
#pragma unroll
            for (int r = 0; r < kRows; ++r) {
                const int rb = i * 32 * kRows + r * 32;
                if (rb >= seg_len) break;
                const int e = rb + lane;
                const bool in = e < seg_len;
                const uint8_t c = (uint8_t)(cc >> (8 * r));
                const float wv = kW ? stg.w[st][r * 32 + lane] : 0.0f;
                if (endp < min(rb + 32, seg_len)) {
                    // piece kp ends inside this row: finish it, then start kp + 1
                    const bool second = e >= endp;
                    if (in && !second) fold_entry<kW>(c, wv, e + dp0, bw, bj, alive);
                    const unsigned long long key = warp_max_u64(strip_key<kW>(bw, bj, alive));
                    finish_table_piece<kW, kStats>(p, kp, lane, it, pieces, lo, hi, key, t);
                    bw = -1.0f;
                    alive = false;
                    ++kp;
                    endp = pend[kp];
                    dp0 = dp1;
                    dp1 = delta[kp + 1];
                    if (in && second) fold_entry<kW>(c, wv, e + dp0, bw, bj, alive);
                } else if (in) {
                    fold_entry<kW>(c, wv, e + dp0, bw, bj, alive);
                }
            }
            cc = cn;
            st = st1;
        }
        {
            const unsigned long long key = warp_max_u64(strip_key<kW>(bw, bj, alive));
            finish_table_piece<kW, kStats>(p, kp, lane, it, pieces, lo, hi, key, t);
        }
        __syncwarp();  // the tables and stages are refilled by the next segment
    }
}

// Phase B: commit proposals, recolour survivors with the next seed, compact
// the worklists of round t+1.
template <bool kW, bool kStats, bool kPolicy>
__device__ void commit_phase(const Params &p, Smem &sm, int t, bool has_next)
{
    Ctl *ctl = p.ctl;
    const int par = t & 1;
    const uint32_t next_seed = has_next ? p.seeds[t + 1] : 0u;
    const uint32_t barrier = ctl->barrier;
    const int c0 = __ldcg(&ctl->cnt[par][kBlue]), c1 = __ldcg(&ctl->cnt[par][kRed]);
    const long long total = (long long)c0 + c1;
    // tiles of at most kTileItems items, as many for every block (the last tile may be short)
    const long long per_block = (total + (long long)gridDim.x * kTileItems - 1) / ((long long)gridDim.x * kTileItems);
    const long long tsize = per_block > 0 ? (total + (long long)gridDim.x * per_block - 1) / ((long long)gridDim.x * per_block) : 1;
    const long long ntiles = (total + tsize - 1) / tsize;
    int *match = ctl->match;
    int retired = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long base = tile * tsize, tend = min(total, base + tsize);
        // items, and with a blue item its request, loaded together
        int4 it[kPer];
        int2 q[kPer];
        bool in[kPer], blue[kPer], gone[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const long long i = base + k * kThreads + threadIdx.x;
            in[k] = i < tend;
            blue[k] = i < c0;
            it[k] = make_int4(0, 0, 0, 0);
            q[k] = make_int2(-1, 0);
            if (in[k]) {
                if (blue[k]) {
                    it[k] = __ldcs(p.lists[par][kBlue] + i);
                } else {
                    it[k] = __ldcs(p.lists[par][kRed] + (i - c0));
                }
            }
            // learned colouring: a red item retired in phase A carries its id complemented
            gone[k] = kPolicy && in[k] && !blue[k] && it[k].x < 0;
            if (gone[k]) it[k].x = ~it[k].x;
        }
        // proposal state: blue -> its request (a fallback list's is in req), red -> the
        // best proposal it received
        unsigned long long key[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            key[k] = 0ull;
            if (in[k]) {
                if (blue[k]) {
                    q[k] = __ldcs(p.reqi + (base + k * kThreads + threadIdx.x));
                    if (q[k].x == kReqFallback) q[k] = __ldcg(p.req + it[k].x);
                } else {
                    key[k] = __ldcg(p.best + it[k].x);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < kPer; ++k)
            if (in[k] && blue[k] && q[k].y != 0) key[k] = __ldcg(p.best + q[k].x);
        int partner[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            partner[k] = -1;
            if (!in[k]) continue;
            if (blue[k]) {
                if (q[k].y != 0 && (uint32_t)key[k] == (uint32_t)q[k].y) partner[k] = q[k].x;
            } else if (key[k]) {
                // the low half of the key names the proposer: its id on the
                // symmetric path, else the position of the red's entry for it
                partner[k] = p.sym ? (int)~(uint32_t)key[k] : __ldg(p.nbrs + (int)~(uint32_t)key[k]);
            }
        }
        int dest[kPer];
        unsigned long long matched = 0, seen = 0, rdeg = 0, act = 0, nblue = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            dest[k] = -1;
            if (!in[k]) continue;
            const int v = it[k].x;
            const int deg = degree_of(it[k]);
            if (kStats && !blue[k]) {
                rdeg += deg;
                // random mode: grRespond stops at its first proposer, whose position
                // is the key's low half (symmetric path: found in the sorted list)
                int first = -1;
                if (!kW && key[k]) {
                    first = (int)~(uint32_t)key[k];
                    if (p.sym) {
                        int lo = it[k].y, hi = it[k].z;
                        while (lo < hi) {
                            const int mid = (int)(((long long)lo + hi) >> 1);
                            if (__ldg(p.nbrs + mid) < first) lo = mid + 1;
                            else hi = mid;
                        }
                        first = lo;
                    }
                }
                seen += first >= 0 ? (unsigned long long)(first - it[k].y + 1) : (unsigned long long)deg;
            }
            if (partner[k] >= 0) {
                trace_left<kPolicy>(p, t, v);
                match[v] = 4 + min(v, partner[k]) - base_of(p, v);
                p.col[v] = kMatched;
                ++matched;
                continue;
            }
            // unmatchable (marked in phase A; learned colouring: red ones too)
            if ((blue[k] && q[k].x == -1) || gone[k]) {
                trace_left<kPolicy>(p, t, v);
                continue;
            }
            // survivor
            if (!has_next) {
                dest[k] = blue[k] ? kBlue : kRed;
                continue;
            }
            const float role = blue[k] ? (q[k].y != 0 ? 1.0f : 0.5f) : 0.0f;
            const float2 wf =
                kPolicy && policy_needs_features(p, t + 1) ? __ldg(p.wfeat + v) : make_float2(0.0f, 0.0f);
            const bool nb = colour_blue<kPolicy>(p, v, deg, role, wf, t + 1, next_seed, barrier);
            if (p.last) p.last[v] = (uint8_t)(t + 1);
            ++act;
            nblue += nb;
            // no neighbours: unmatchable as soon as it is blue
            if (nb && deg == 0) {
                p.col[v] = kDead;
                match[v] = 2;
                ++retired;
                trace_left<kPolicy>(p, t + 1, v);
            } else {
                p.col[v] = nb ? kBlue : kRed;
                dest[k] = nb ? kBlue : kRed;
            }
        }
        if (kStats) {
            stat_add(p, t, MM_ST_MATCHED, matched);
            stat_add(p, t, MM_ST_RESP_ENTRIES, seen);
            stat_add(p, t, MM_ST_RED_DEG, rdeg);
            if (has_next) {
                stat_add(p, t + 1, MM_ST_ACTIVE, act);
                stat_add(p, t + 1, MM_ST_BLUE, nblue);
                stat_add(p, t + 1, MM_ST_RED, act - nblue);
            }
        }
        compact_tile(p, sm, par ^ 1, dest, it);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) retired += __shfl_xor_sync(kFull, retired, o);
    if ((threadIdx.x & 31) == 0 && retired) atomicAdd(&ctl->retired[par ^ 1], retired);
}

// ---- finish phase ----
//
// After the first rounds the vertices that can still be matched form a sparse
// subgraph: on R-MAT 2^23 at round 5, 334 k active vertices share 40 k entries
// that point at another active vertex, and its connected components have at
// most 7 members (grids, random geometric and Erdos-Renyi graphs reach the same
// state by round 3).  A vertex's future depends only on the colours and choices
// of the active vertices it can reach: matched neighbours never change, and on
// the symmetric path no active vertex has an unmatchable neighbour (a vertex
// became unmatchable because every neighbour was matched).  So each component
// can play all its remaining rounds on its own, with the same seeds, and the
// grid needs no further barrier.
//
// The phase runs at the start of round t in two passes over the round's
// worklist items, each ended by a grid barrier:
//   scan   every item scans its own list: no active neighbour (a singleton),
//          an active neighbour with a smaller id (a member: another vertex
//          speaks for its component), or else a root candidate.  It records
//          its first two active neighbours with their preference keys.  A
//          singleton walks its own hash sequence at once: it leaves (match
//          value 2) in the first round it is blue, or keeps red to the cap.
//   roots  each root candidate's lane follows the records breadth first to
//          its component and, if no member has a smaller id, plays it: per
//          round colour, request (the best red neighbour by the same keys as
//          the scans), respond (the largest proposal key), commit.  A
//          component that a lane cannot hold (records incomplete, more than
//          kFinTMembers members) is searched and played by the warp, lane l
//          holding member l (up to kFinMembers members, kFinEntries entries).
// A larger component, a list longer than kFinMaxDeg or an unmatchable
// neighbour calls the attempt off (ctl->fin_abort), and round t runs as
// usual; values already written are the ones the rounds write again.  The
// instrumented kernel checks first and resolves in a third pass, so that its
// counters never include a called-off attempt.
// Every vertex's match value is then final, and the matching executed
// max(last active round) + 2 rounds, the reference's closing round included
// (at most the cap).
constexpr int kFinMembers = 32;    // members of a component played by one warp (one per lane)
constexpr int kFinEntries = 128;   // entries between members of one component
constexpr int kFinShort = 32;      // lists a thread scans on its own; longer ones its warp scans
constexpr int kFinMaxDeg = 2048;   // longest list the finish phase accepts
constexpr int kFinDiv = 12;        // default: first attempt once the active set is at most 1/kFinDiv of round 0's
enum : int { kFinSingle = 1, kFinMember = 2, kFinRootCand = 3 };
enum : int { kFinNotRoot = 0, kFinRoot = 1, kFinTooBig = 2 };

// One warp's component: members' first entry, list start and degree, the
// entries between members (preference key and the target's member slot), the
// members' colours of the round being played and the best proposal each
// received.
struct FinWarp {
    unsigned long long pref[kFinEntries];
    unsigned long long best[kFinMembers];
    int mem[kFinMembers];
    int eoff[kFinMembers + 1];
    int mbeg[kFinMembers];
    int mdeg[kFinMembers];
    uint8_t tgt[kFinEntries];
    uint8_t st[kFinMembers];
};
static_assert(sizeof(FinWarp) * kWarps <= offsetof(Smem, tile_warp),
              "the finish phase reuses the fallback scan's shared memory");

// Item i of round parity `par` (blue list first, then red).
__device__ __forceinline__ int4 item_at(const Params &p, int par, int c0, long long i)
{
    return i < c0 ? __ldcg(p.lists[par][kBlue] + i) : __ldcg(p.lists[par][kRed] + (i - c0));
}

// Own-list scan of vertex v, entries [b, e): active neighbours (blue or red),
// whether one has a smaller id, whether a neighbour is unmatchable, and the
// positions and ids of the first kFinRec active neighbours.
constexpr int kFinRec = 4;  // active neighbours a record holds
__device__ __forceinline__ void fin_scan_thread(const Params &p, int v, int b, int e, int &nint, bool &lower,
                                                bool &bad, int (&jr)[kFinRec], int (&ur)[kFinRec])
{
    for (int j0 = b; j0 < e; j0 += 8) {
        int u[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) u[k] = j0 + k < e ? __ldg(p.nbrs + j0 + k) : -1;
        uint8_t c[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) c[k] = u[k] >= 0 ? p.col[u[k]] : (uint8_t)kMatched;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (c[k] <= kRed) {
#pragma unroll
                for (int q = 0; q < kFinRec; ++q) {
                    if (nint == q) {
                        jr[q] = j0 + k;
                        ur[q] = u[k];
                    }
                }
                ++nint;
                lower |= u[k] < v;
            }
            bad |= c[k] == kDead;
        }
    }
}

// The same scan by a whole warp, rows of 32 entries, for a list longer than
// kFinShort; every lane gets the results (the first kFinRec active
// neighbours in list order too).
__device__ __forceinline__ void fin_scan_warp(const Params &p, int v, int b, int e, int &nint, bool &lower,
                                              bool &bad, int (&jr)[kFinRec], int (&ur)[kFinRec])
{
    const int lane = threadIdx.x & 31;
    int cnt = 0;
    bool lo = false, bd = false;
    for (int r0 = b; r0 < e; r0 += 32 * 4) {
        int u[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) u[k] = r0 + 32 * k + lane < e ? __ldg(p.nbrs + r0 + 32 * k + lane) : -1;
        uint8_t c[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) c[k] = u[k] >= 0 ? p.col[u[k]] : (uint8_t)kMatched;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const bool in = c[k] <= kRed;
            lo |= in && u[k] < v;
            bd |= c[k] == kDead;
            unsigned m = __ballot_sync(kFull, in);
            while (m && cnt < kFinRec) {
                const int sb = __ffs(m) - 1;
                m &= m - 1;
                const int us = __shfl_sync(kFull, u[k], sb);
#pragma unroll
                for (int q = 0; q < kFinRec; ++q) {
                    if (cnt == q) {
                        jr[q] = r0 + 32 * k + sb;
                        ur[q] = us;
                    }
                }
                ++cnt;
            }
            cnt += __popc(m);
        }
    }
    nint = cnt;
    lower = __any_sync(kFull, lo);
    bad = __any_sync(kFull, bd);
}

// Component search for root candidate v by its warp.  Members are numbered in
// discovery order (member 0 is v; lane l's `mem` holds member l); each
// member's entries that point at a member are stored in order, from
// fw.eoff[member].  Returns kFinNotRoot as soon as a member has a smaller id
// than v, kFinTooBig if the component does not fit, else kFinRoot with *k
// members.
template <bool kW>
__device__ __forceinline__ int fin_search(const Params &p, FinWarp &fw, int v, int *mem_out, int *k_out,
                                          unsigned long long *scanned)
{
    const int lane = threadIdx.x & 31;
    int mem = lane == 0 ? v : -1;
    int k = 1, ne = 0;
    unsigned long long seen = 0;
    for (int f = 0; f < k; ++f) {
        const int x = __shfl_sync(kFull, mem, f);
        const int2 r = __ldg(p.ranges + x);
        const int b = r.x, e = r.y > r.x ? r.y : r.x;
        if (e - b > kFinMaxDeg) return kFinTooBig;
        if (lane == 0) {
            fw.eoff[f] = ne;
            fw.mbeg[f] = b;
            fw.mdeg[f] = e - b;
        }
        seen += (unsigned long long)(e - b);
        for (int j0 = b; j0 < e; j0 += 32) {
            const int j = j0 + lane;
            int u = -1;
            float wj = 0.0f;
            uint8_t c = kMatched;
            if (j < e) {
                u = __ldg(p.nbrs + j);
                if (kW) wj = __ldg(p.w + j);  // with the id: no dependent load once the colour is known
                c = p.col[u];
            }
            const bool in = c <= kRed;
            if (__any_sync(kFull, c == kDead)) return kFinTooBig;
            if (__any_sync(kFull, in && u < v)) return kFinNotRoot;
            unsigned m = __ballot_sync(kFull, in);
            unsigned long long pref = 0;
            if (in) pref = kW ? cand_key<true>(j, wj) : (unsigned long long)(uint32_t)~j;
            while (m) {
                const int s = __ffs(m) - 1;
                m &= m - 1;
                const int us = __shfl_sync(kFull, u, s);
                const unsigned hit = __ballot_sync(kFull, lane < k && mem == us);
                int slot;
                if (hit) {
                    slot = __ffs(hit) - 1;
                } else {
                    if (k == kFinMembers) return kFinTooBig;
                    slot = k;
                    if (lane == k) mem = us;
                    ++k;
                }
                if (ne == kFinEntries) return kFinTooBig;
                if (lane == s) {
                    fw.pref[ne] = pref;
                    fw.tgt[ne] = (uint8_t)slot;
                }
                ++ne;
            }
        }
    }
    if (lane == 0) fw.eoff[k] = ne;
    __syncwarp();
    *mem_out = mem;
    *k_out = k;
    if (scanned) *scanned = seen;
    return kFinRoot;
}

// Adjacency entries the reference's respond loop inspects for red vertex v
// (entries [b, b + deg)) whose best proposal key is kb: in random mode it
// stops at its first proposer in list order, here the proposer with the
// smallest id (kb's low half complemented), found in the sorted list.
template <bool kW>
__device__ __forceinline__ unsigned long long respond_seen(const Params &p, int b, int deg, unsigned long long kb)
{
    if (kW || !kb) return (unsigned long long)deg;
    const int first = (int)~(uint32_t)kb;
    int lo = b, hi = b + deg;
    while (lo < hi) {
        const int mid = (int)(((long long)lo + hi) >> 1);
        if (__ldg(p.nbrs + mid) < first) lo = mid + 1;
        else hi = mid;
    }
    return (unsigned long long)(lo - b + 1);
}

// Play a component found by fin_search (k members, lane l = member l) from
// round t0 until none of its members can be matched or the cap is reached;
// writes every member's match value (and batch round marks).  Returns, in
// every lane, the last round in which a member was active.
template <bool kW, bool kStats>
__device__ __forceinline__ int fin_play(const Params &p, FinWarp &fw, const uint32_t *seeds, int t0, int cap, int mem,
                                       int k)
{
    const int lane = threadIdx.x & 31;
    const bool own = lane < k;
    const int g = own ? mem : 0;
    const int base = own ? base_of(p, g) : 0;
    const uint32_t hid = (uint32_t)(g - base);
    const uint32_t bar = p.fin_retire ? p.policy_bar : p.ctl->barrier;
    int eb = 0, ee = 0, deg = 0, beg = 0;
    if (own) {
        eb = fw.eoff[lane];
        ee = fw.eoff[lane + 1];
        deg = fw.mdeg[lane];
        beg = fw.mbeg[lane];
        fw.best[lane] = 0ull;
    }
    // learned colouring: whether a red member may retire (its list is short enough)
    const bool may_retire = p.fin_retire && own && degree_of(__ldg(p.ranges + g)) <= kRetireMaxDeg;
    bool act = own, blue = false;
    int val = 0, lastr = -1;
    __syncwarp();
    for (int t = t0; t < cap && __any_sync(kFull, act); ++t) {
        if (act) {
            blue = colour_of(hid, seeds[t], bar) == kBlue;
            lastr = t;
        }
        if (own) fw.st[lane] = act ? (blue ? kBlue : kRed) : (val == 2 ? kDead : kMatched);
        __syncwarp();
        // learned colouring: from round kRetireFrom a red member whose neighbours
        // are all matched leaves at once (the round kernel's retire_red; its
        // neighbours outside the component are matched)
        bool retired = false;
        if (may_retire && act && !blue && t >= kRetireFrom) {
            bool alive = false;
            for (int e = eb; e < ee; ++e) alive |= fw.st[fw.tgt[e]] != kMatched;
            if (!alive) {
                val = 2;
                retired = true;
            }
        }
        // request: the best red neighbour among the members (matched ones
        // outside the component neither attract nor keep a vertex alive)
        unsigned long long best = 0ull;
        int choice = 0;
        if (act && blue) {
            for (int e = eb; e < ee; ++e) {
                const int tg = fw.tgt[e];
                const uint8_t c = fw.st[tg];
                const unsigned long long key = c == kRed ? fw.pref[e] : (c == kMatched ? 0ull : 1ull);
                if (key > best) {
                    best = key;
                    choice = tg;
                }
            }
        }
        unsigned long long crk = 0ull;
        if (act && blue && best >= 2) {
            // the target's entry for this vertex has the same weight (symmetric path)
            crk = kW ? (((best >> 32) << 32) | (unsigned long long)(uint32_t)~(uint32_t)g)
                     : (unsigned long long)(uint32_t)~(uint32_t)g;
            atomicMax(&fw.best[choice], crk);
        }
        __syncwarp();
        const int gp = __shfl_sync(kFull, g, choice);
        bool matched = false, dead = false;
        unsigned long long kb = 0ull;
        if (act) {
            if (blue) {
                if (best >= 2 && (uint32_t)fw.best[choice] == (uint32_t)crk) {
                    val = 4 + min(g, gp) - base;
                    matched = true;
                } else if (best == 0) {
                    val = 2;
                    dead = true;
                }
            } else {
                kb = fw.best[lane];
                if (kb) {
                    val = 4 + min(g, (int)~(uint32_t)kb) - base;
                    matched = true;
                }
            }
        }
        if (kStats) {
            const bool b = act && blue, r = act && !blue;
            if (t > t0) {  // round t0's colouring was counted by the commit that made it
                stat_add(p, t, MM_ST_ACTIVE, act ? 1ull : 0ull);
                stat_add(p, t, MM_ST_BLUE, b ? 1ull : 0ull);
                stat_add(p, t, MM_ST_RED, r ? 1ull : 0ull);
            }
            stat_add(p, t, MM_ST_BLUE_DEG, b ? (unsigned long long)deg : 0ull);
            stat_add(p, t, MM_ST_RED_DEG, r ? (unsigned long long)deg : 0ull);
            stat_add(p, t, MM_ST_REQ_ENTRIES,
                     b ? request_seen<kW>(beg, deg, best >= 2 ? (int)~(uint32_t)best : -1) : 0ull);
            stat_add(p, t, MM_ST_RESP_ENTRIES, r ? respond_seen<kW>(p, beg, deg, kb) : 0ull);
            stat_add(p, t, MM_ST_MATCHED, matched ? 1ull : 0ull);
        }
        __syncwarp();
        if (own) fw.best[lane] = 0ull;
        if (matched || dead || retired) act = false;
    }
    if (own) {
        // members still unmatched at the cap keep their last colour
        p.ctl->match[g] = act ? (blue ? 0 : 1) : val;
        if (p.last) p.last[g] = (uint8_t)lastr;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lastr = max(lastr, __shfl_xor_sync(kFull, lastr, o));
    return lastr;
}

// Lane-level components.  Most components of the finish round are pairs and
// short paths.  A warp that searched its lanes' roots one after another, each
// rescanning its members' lists, made every warp a chain of dependent loads
// (on RGG 2^20 at round 3, 9 root candidates a tile and 52 us a warp).  So each
// lane searches its own root's component through the records and plays it in
// per-thread storage.
constexpr int kFinTMembers = 16;
constexpr int kFinTEntries = 32;
enum : int { kFinOverflow = 3 };

struct FinComp {
    unsigned long long pref[kFinTEntries];
    int mem[kFinTMembers];
    int mbeg[kFinTMembers];
    int mdeg[kFinTMembers];
    uint8_t tgt[kFinTEntries];
    uint8_t eoff[kFinTMembers + 1];
    int k;
};

// The finish phase's record of item i: four int4 slots, rec[4i .. 4i + 3], in
// the worklist memory of the other parity (2n slots, which the round has not
// written yet; an attempt has at most n / 2 items): {meta, v, 0, 0},
// then the ids, preference-key low halves and high halves of its first
// kFinRec entries that point at an active vertex.  meta = class | count << 8,
// count = its active neighbours, kFinRec + 1 if more than a record holds.
__device__ __forceinline__ int fin_meta_class(int meta) { return meta & 0xff; }
__device__ __forceinline__ int fin_meta_count(int meta) { return (meta >> 8) & 0xff; }

// As fin_search, by one thread for root candidate v (item i), following the
// records instead of the lists: each member costs two loads from L2 (its
// item index, its record).  kFinOverflow when a member's record is incomplete
// or the component does not fit FinComp.  The lists' bounds are read only
// for the instrumented kernel's counters.
template <bool kW, bool kStats>
__device__ __forceinline__ int fin_search_thread(const Params &p, const int4 *rec, int v, long long i, FinComp &cp)
{
    long long ix[kFinTMembers];
    int k = 1, ne = 0;
    cp.mem[0] = v;
    ix[0] = i;
    for (int f = 0; f < k; ++f) {
        const int4 r0 = __ldcg(rec + 4 * ix[f]);
        const int cnt = fin_meta_count(r0.x);
        if (cnt > kFinRec) return kFinOverflow;
        cp.eoff[f] = (uint8_t)ne;
        if (kStats) {
            const int2 r = __ldg(p.ranges + cp.mem[f]);
            cp.mbeg[f] = r.x;
            cp.mdeg[f] = r.y > r.x ? r.y - r.x : 0;
        }
        if (cnt == 0) continue;
        const int4 ru = __ldcg(rec + 4 * ix[f] + 1), rl = __ldcg(rec + 4 * ix[f] + 2), rh = __ldcg(rec + 4 * ix[f] + 3);
        const int uu[kFinRec] = {ru.x, ru.y, ru.z, ru.w};
        const int lo[kFinRec] = {rl.x, rl.y, rl.z, rl.w};
        const int hi[kFinRec] = {rh.x, rh.y, rh.z, rh.w};
#pragma unroll
        for (int q = 0; q < kFinRec; ++q) {
            if (q >= cnt) break;
            const int u = uu[q];
            if (u < v) return kFinNotRoot;
            int slot = -1;
            for (int m = 0; m < k; ++m)
                if (cp.mem[m] == u) slot = m;
            if (slot < 0) {
                if (k == kFinTMembers) return kFinOverflow;
                slot = k;
                cp.mem[k] = u;
                ix[k] = __ldcg(p.req + u).x;  // its item (written by the scan pass)
                ++k;
            }
            if (ne == kFinTEntries) return kFinOverflow;
            cp.pref[ne] = ((unsigned long long)(uint32_t)hi[q] << 32) | (uint32_t)lo[q];
            cp.tgt[ne] = (uint8_t)slot;
            ++ne;
        }
    }
    cp.eoff[k] = (uint8_t)ne;
    cp.k = k;
    return kFinRoot;
}

// Singletons of a tile (mine): each leaves in the first round from t on in
// which it is blue (blue0: its colour in round t), or keeps red to the cap.
template <bool kStats>
__device__ __forceinline__ void fin_singles(const Params &p, const uint32_t *seeds, int t, int cap, bool mine, int v,
                                            int deg, bool blue0, int &last_all)
{
    const uint32_t bar = p.fin_retire ? p.policy_bar : p.ctl->barrier;
    const uint32_t hid = mine ? (uint32_t)(v - base_of(p, v)) : 0u;
    // learned colouring: a short list retires as soon as it is red from round
    // kRetireFrom (a singleton's neighbours are all matched)
    const bool may_retire = p.fin_retire && deg <= kRetireMaxDeg;
    bool act = mine, blue = blue0;
    int lastr = -1;
    for (int r = t; r < cap && __any_sync(kFull, act); ++r) {
        if (act) {
            if (r > t) blue = colour_of(hid, seeds[r], bar) == kBlue;
            lastr = r;
        }
        if (kStats) {
            const bool b = act && blue, rd = act && !blue;
            if (r > t) {  // round t's colouring was counted by the commit that made it
                stat_add(p, r, MM_ST_ACTIVE, act ? 1ull : 0ull);
                stat_add(p, r, MM_ST_BLUE, b ? 1ull : 0ull);
                stat_add(p, r, MM_ST_RED, rd ? 1ull : 0ull);
            }
            stat_add(p, r, MM_ST_BLUE_DEG, b ? (unsigned long long)deg : 0ull);
            stat_add(p, r, MM_ST_RED_DEG, rd ? (unsigned long long)deg : 0ull);
            stat_add(p, r, MM_ST_REQ_ENTRIES, b ? (unsigned long long)deg : 0ull);
            stat_add(p, r, MM_ST_RESP_ENTRIES, rd ? (unsigned long long)deg : 0ull);
        }
        if (act && (blue || (may_retire && r >= kRetireFrom))) act = false;
    }
    if (mine) {
        // still red at the cap: it keeps that colour
        p.ctl->match[v] = act ? 1 : 2;
        if (p.last) p.last[v] = (uint8_t)lastr;
        last_all = max(last_all, lastr);
    }
}

// Finish pass 1 over round t's items: scan each item's own list (a thread
// each, its warp for lists longer than kFinShort), classify it, record its
// first two active neighbours (non-singletons also record their item index
// in req[v].x), and, with kSingles, resolve the singletons at once.  Calls
// the attempt off for a list longer than kFinMaxDeg or an unmatchable
// neighbour.
template <bool kW, bool kStats, bool kSingles>
__device__ __forceinline__ void finish_scan(const Params &p, Smem &sm, int t, int par, int c0, int c1, int cap,
                                            int4 *rec)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long A = (long long)c0 + c1;
    const long long gw = (long long)blockIdx.x * kWarps + warp, nw = (long long)gridDim.x * kWarps;
    bool abort = false;
    int last_all = -1;
    for (long long base = gw * 32; base < A; base += nw * 32) {
        // another warp may have called the attempt off: its remaining work is wasted
        if (__shfl_sync(kFull, lane == 0 ? __ldcg(&p.ctl->fin_abort) : 0, 0) == t + 1) break;
        const long long i = base + lane;
        const int4 it = i < A ? item_at(p, par, c0, i) : make_int4(-1, 0, 0, 0);
        const int deg = it.x >= 0 ? degree_of(it) : 0;
        int nint = 0, jr[kFinRec] = {0, 0, 0, 0}, ur[kFinRec] = {0, 0, 0, 0};
        bool lower = false, bad = false;
        if (it.x >= 0 && deg <= kFinShort) fin_scan_thread(p, it.x, it.y, it.y + deg, nint, lower, bad, jr, ur);
        unsigned longs = __ballot_sync(kFull, it.x >= 0 && deg > kFinShort);
        while (longs) {
            const int s = __ffs(longs) - 1;
            longs &= longs - 1;
            const int vs = __shfl_sync(kFull, it.x, s), bs = __shfl_sync(kFull, it.y, s);
            const int ds = __shfl_sync(kFull, deg, s);
            if (ds > kFinMaxDeg) {
                if (lane == s) bad = true;
                continue;
            }
            int n2, j2[kFinRec], u2[kFinRec];
            bool l2, b2;
            fin_scan_warp(p, vs, bs, bs + ds, n2, l2, b2, j2, u2);
            if (lane == s) {
                nint = n2;
                lower = l2;
                bad = b2;
#pragma unroll
                for (int q = 0; q < kFinRec; ++q) {
                    jr[q] = j2[q];
                    ur[q] = u2[q];
                }
            }
        }
        const int c = it.x < 0 ? 0 : (nint == 0 ? kFinSingle : (lower ? kFinMember : kFinRootCand));
        abort |= bad;
        if (it.x >= 0) {
            const int cnt = min(nint, kFinRec + 1);
            rec[4 * i] = make_int4(c | (cnt << 8), it.x, 0, 0);
            if (nint > 0) {
                p.req[it.x].x = (int)i;
                if (cnt <= kFinRec) {
                    uint32_t lo[kFinRec], hi[kFinRec];
#pragma unroll
                    for (int q = 0; q < kFinRec; ++q) {
                        unsigned long long key = 0ull;
                        if (q < cnt) key = kW ? cand_key<true>(jr[q], __ldg(p.w + jr[q])) : (unsigned long long)(uint32_t)~jr[q];
                        lo[q] = (uint32_t)key;
                        hi[q] = (uint32_t)(key >> 32);
                    }
                    rec[4 * i + 1] = make_int4(ur[0], ur[1], ur[2], ur[3]);
                    rec[4 * i + 2] = make_int4((int)lo[0], (int)lo[1], (int)lo[2], (int)lo[3]);
                    rec[4 * i + 3] = make_int4((int)hi[0], (int)hi[1], (int)hi[2], (int)hi[3]);
                }
            }
        }
        if (kStats) {
            stat_add(p, t, MM_ST_FINISH_ITEMS, it.x >= 0 ? 1ull : 0ull);
            stat_add(p, t, MM_ST_FINISH_ENTRIES, (unsigned long long)deg);
        }
        if (__any_sync(kFull, abort)) {  // the attempt is off: tell the other warps now
            if (lane == 0) atomicExch(&p.ctl->fin_abort, t + 1);
            break;
        }
        if (kSingles) fin_singles<kStats>(p, sm.seeds, t, cap, c == kFinSingle, it.x, deg, i < c0, last_all);
    }
    if (abort && lane == 0) atomicExch(&p.ctl->fin_abort, t + 1);
    if (kSingles) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) last_all = max(last_all, __shfl_xor_sync(kFull, last_all, o));
        if (lane == 0 && last_all >= 0) atomicMax(&p.ctl->fin_last, last_all);
    }
}

// Finish pass 2 over round t's items: each root candidate's lane searches its
// component through the records and, with kPlay, plays it; a component that
// a lane cannot hold goes to the warp (list scans, up to kFinMembers members),
// and one larger than that calls the attempt off.  With kSingles (the
// instrumented kernel's last pass) the singletons are resolved here too.
template <bool kW, bool kStats, bool kPlay, bool kSingles>
__device__ __forceinline__ void finish_roots(const Params &p, Smem &sm, int t, int par, int c0, int c1, int cap,
                                             const int4 *rec)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    FinWarp &fw = reinterpret_cast<FinWarp *>(&sm)[warp];
    const long long A = (long long)c0 + c1;
    const long long gw = (long long)blockIdx.x * kWarps + warp, nw = (long long)gridDim.x * kWarps;
    bool abort = false;
    int last_all = -1;
    for (long long base = gw * 32; base < A; base += nw * 32) {
        if (__shfl_sync(kFull, lane == 0 ? __ldcg(&p.ctl->fin_abort) : 0, 0) == t + 1) break;
        const long long i = base + lane;
        const int4 r0 = i < A ? __ldcg(rec + 4 * i) : make_int4(0, -1, 0, 0);
        const int meta = r0.x;
        const int c = fin_meta_class(meta);
        if (kSingles) {
            const int4 it = c == kFinSingle ? item_at(p, par, c0, i) : make_int4(-1, 0, 0, 0);
            fin_singles<kStats>(p, sm.seeds, t, cap, c == kFinSingle, it.x, c == kFinSingle ? degree_of(it) : 0,
                                i < c0, last_all);
        }
        const int v = c == kFinRootCand ? r0.y : -1;
        int rres = kFinNotRoot;
        FinComp cp;
        if (c == kFinRootCand) rres = fin_search_thread<kW, kStats>(p, rec, v, i, cp);
        // the lanes' components, packed into the warp and played together, a lane
        // per member (a lane playing its component alone would colour its
        // members one after another)
        unsigned pend = __ballot_sync(kFull, kPlay && rres == kFinRoot);
        while (pend) {
            const bool mine = (pend >> lane) & 1u;
            const int km = mine ? cp.k : 0, nem = mine ? (int)cp.eoff[cp.k] : 0;
            int pk = km, pe = nem;  // inclusive prefix sums in lane order
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(kFull, pk, o), z = __shfl_up_sync(kFull, pe, o);
                if (lane >= o) {
                    pk += y;
                    pe += z;
                }
            }
            const bool take = mine && pk <= kFinMembers && pe <= kFinEntries;
            const unsigned batch = __ballot_sync(kFull, take);  // a prefix of pend
            const int lastl = 31 - __clz(batch);
            const int ktot = __shfl_sync(kFull, pk, lastl), etot = __shfl_sync(kFull, pe, lastl);
            if (take) {
                const int mo = pk - km, eo = pe - nem;
                for (int l = 0; l < km; ++l) {
                    fw.mem[mo + l] = cp.mem[l];
                    fw.eoff[mo + l] = eo + cp.eoff[l];
                    fw.mdeg[mo + l] = cp.mdeg[l];
                    fw.mbeg[mo + l] = cp.mbeg[l];
                }
                for (int e = 0; e < nem; ++e) {
                    fw.pref[eo + e] = cp.pref[e];
                    fw.tgt[eo + e] = (uint8_t)(mo + cp.tgt[e]);
                }
            }
            if (lane == 0) fw.eoff[ktot] = etot;
            __syncwarp();
            const int ml = lane < ktot ? fw.mem[lane] : 0;
            last_all = max(last_all, fin_play<kW, kStats>(p, fw, sm.seeds, t, cap, ml, ktot));
            __syncwarp();  // fw is refilled by the next batch
            pend &= ~batch;
        }
        unsigned roots = __ballot_sync(kFull, rres == kFinOverflow);
        while (roots) {
            const int s = __ffs(roots) - 1;
            roots &= roots - 1;
            int mem, k;
            unsigned long long seen = 0;
            const int r = fin_search<kW>(p, fw, __shfl_sync(kFull, v, s), &mem, &k, kStats && !kPlay ? &seen : nullptr);
            if (kStats && !kPlay && lane == 0) atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_FINISH_ENTRIES], seen);
            if (r == kFinTooBig) {
                abort = true;
                break;
            }
            if (kPlay && r == kFinRoot) last_all = max(last_all, fin_play<kW, kStats>(p, fw, sm.seeds, t, cap, mem, k));
            __syncwarp();  // fw is reused by the next root
        }
        if (__any_sync(kFull, abort)) {
            if (lane == 0) atomicExch(&p.ctl->fin_abort, t + 1);
            break;
        }
    }
    if (abort && lane == 0) atomicExch(&p.ctl->fin_abort, t + 1);
    if (kPlay) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) last_all = max(last_all, __shfl_xor_sync(kFull, last_all, o));
        if (lane == 0 && last_all >= 0) atomicMax(&p.ctl->fin_last, last_all);
    }
}

// The whole matching in one cooperative launch: set-up, then per round the
// window scan (A1), the fallback scan (A2, only in rounds that have fallback
// lists) and the commit phase (B), separated by grid barriers.  Every block
// reads the same counters after a barrier, so all blocks take the same
// branches and leave the loop at the same round.  Afterwards, vertices that
// could still be matched keep their last colour as their match value (the
// reference leaves match[v] = 0 / 1 for them).
template <bool kW, bool kStats, bool kPolicy>
__global__ void __launch_bounds__(kThreads, 2) k_rounds(Params p)
{
    extern __shared__ __align__(16) unsigned char dsmem[];
    Smem &sm = *reinterpret_cast<Smem *>(dsmem);
    Ctl *ctl = p.ctl;
    const int cap = ctl->cap;
    const int maximal = ctl->maximal;
    const int nseeds = ctl->nseeds;
    const int gwarp = blockIdx.x * kWarps + (threadIdx.x >> 5);
    const int nwarps = gridDim.x * kWarps;

    long long active0, fin_next;
    int t;
    if (p.resume) {
        // the finish kernel called its attempt off: carry on from its round,
        // without another attempt
        if (ctl->fin_state != kFinStateResume) {
            release_lines(p.col, p.n);
            return;
        }
        t = ctl->fin_round;
        active0 = ctl->active0;
        fin_next = -1;
    } else {
        init_phase<kW, kStats, kPolicy>(p, sm);
        if (!grid_sync(p.bar, p.ctl, p.tstamp, 0, p.spin_limit, p.skip_mark)) return;
        // active vertices at round 0; round 1 clears these counters only after
        // two more grid barriers
        active0 = (long long)__ldcg(&ctl->cnt[0][kBlue]) + __ldcg(&ctl->cnt[0][kRed]);
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->active0 = active0;
        fin_next = active0;  // finish phase: attempt once the active set is this small
        t = 0;
    }
    for (;; ++t) {
        const int par = t & 1;
        // Hand the rest to the finish kernel (the symmetric path of the
        // reference's colouring only).  Every block reads the same counters and
        // leaves here; round t's worklists and colours are complete.
        if ((!kPolicy || p.fin_retire) && p.sym && t > 0) {
            const long long act = (long long)__ldcg(&ctl->cnt[par][kBlue]) + __ldcg(&ctl->cnt[par][kRed]);
            if (p.fin_div > 0 && act > 0 && act * p.fin_div <= active0 && act <= fin_next) {
                if (blockIdx.x == 0 && threadIdx.x == 0) {
                    ctl->fin_round = t;
                    ctl->fin_state = kFinStatePending;
                }
                return;
            }
        }
        // phase A1; the next round's counters were last read in round t - 1
        if (blockIdx.x == 0 && threadIdx.x < kParityLists) {
            ctl->cnt[par ^ 1][threadIdx.x] = 0;
            if (threadIdx.x == 0) ctl->retired[par ^ 1] = 0;
        }
        scan_window<kW, kStats, kPolicy>(p, sm, t, par);
        if (!grid_sync(p.bar, p.ctl, p.tstamp, 3 * t + 1, p.spin_limit, p.skip_mark)) return;
        // phase A2 (all blocks see the same fallback count)
        if (__ldcg(&ctl->staged_pack) != 0ull) {
            scan_long<kW, kStats>(p, sm, t, gwarp, nwarps);
            if (!grid_sync(p.bar, p.ctl, p.tstamp, -1, p.spin_limit, p.skip_mark)) return;
        }
        if (p.tstamp && blockIdx.x == 0 && threadIdx.x == 0) p.tstamp[3 * t + 2] = global_ns();
        // phase B; the fallback list is empty again for the next round
        bool has_next = t + 1 < cap;
        const bool seeds_short = has_next && t + 1 >= nseeds;
        if (seeds_short) has_next = false;
        commit_phase<kW, kStats, kPolicy>(p, sm, t, has_next);
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->staged_pack = 0ull;
        if (!grid_sync(p.bar, p.ctl, p.tstamp, 3 * t + 3, p.spin_limit, p.skip_mark)) return;
        // close the round (every block decides alike)
        const long long next = (long long)__ldcg(&ctl->cnt[par ^ 1][kBlue]) + __ldcg(&ctl->cnt[par ^ 1][kRed]);
        const bool more = has_next && next > 0;
        if (!more) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                if (seeds_short) ctl->status = 1;
                // Vertices retired while being coloured for round t+1 are still
                // active in that round for the reference, so it runs round t+1
                // and only finds nothing left at round t+2.
                const int retired_all = __ldcg(&ctl->retired[par ^ 1]);
                if (!maximal || next > 0) ctl->rounds = cap;
                else ctl->rounds = min(retired_all > 0 ? t + 3 : t + 2, cap);
                // vertices without neighbours resolved at set-up
                const int iso = __ldcg(&ctl->iso_last) - 1;
                if (maximal && iso >= 0) ctl->rounds = max(ctl->rounds, min(iso + 2, cap));
            }
            break;
        }
    }
    // finish: survivors of the last round (lists of parity (t + 1) & 1)
    const int par = (t + 1) & 1;
    const int cb = __ldcg(&ctl->cnt[par][kBlue]), cr = __ldcg(&ctl->cnt[par][kRed]);
    const long long total = (long long)cb + cr;
    int *match = ctl->match;
    for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < total; i += (long long)gridDim.x * kThreads) {
        const int v = i < cb ? __ldcg(p.lists[par][kBlue] + i).x : __ldcg(p.lists[par][kRed] + (i - cb)).x;
        match[v] = __ldcg(p.col + v);
    }
    // the last launch of the matching (a finish kernel and a resumed round
    // kernel follow only a hand-over, which returns above)
    release_lines(p.col, p.n);
}

// The finish phase as its own cooperative launch, after k_rounds has stopped
// at round ctl->fin_round (its code inside the round kernel cost that kernel's
// scan and commit loops registers: its rounds 0-4 ran 7% slower on R-MAT 2^23).
// It returns at once if the round kernel finished the matching itself.  If the
// attempt is called off, the resumed round kernel carries on from that round.
template <bool kW, bool kStats>
__global__ void __launch_bounds__(kThreads, 2) k_finish(Params p)
{
    extern __shared__ __align__(16) unsigned char dsmem[];
    Smem &sm = *reinterpret_cast<Smem *>(dsmem);
    Ctl *ctl = p.ctl;
    if (ctl->fin_state != kFinStatePending) return;
    const int cap = ctl->cap, maximal = ctl->maximal;
    const int t = ctl->fin_round, par = t & 1;
    const int c0 = ctl->cnt[par][kBlue], c1 = ctl->cnt[par][kRed];
    // the seed buffer holds 256 words (only the call's seeds are meaningful)
    for (int i = threadIdx.x; i < 256; i += kThreads) sm.seeds[i] = p.seeds[i];
    __syncthreads();
    // records: the worklist memory of the other parity (2n items, written by
    // round t's commit only, which runs after this kernel if at all)
    int4 *rec = p.lists[par ^ 1][kBlue];
    // profile: the first pass is reported as round t's window scan, the rest
    // as its fallback scan
    bool done;
    if (kStats) {
        // counters must not count a called-off attempt: check, then resolve
        finish_scan<kW, kStats, false>(p, sm, t, par, c0, c1, cap, rec);
        if (!grid_sync(p.bar, p.ctl, p.tstamp, 3 * t + 1, p.spin_limit, p.skip_mark)) return;
        done = __ldcg(&ctl->fin_abort) != t + 1;
        if (done) {
            finish_roots<kW, kStats, false, false>(p, sm, t, par, c0, c1, cap, rec);
            if (!grid_sync(p.bar, p.ctl, p.tstamp, -1, p.spin_limit, p.skip_mark)) return;
            done = __ldcg(&ctl->fin_abort) != t + 1;
        }
        if (done) {
            finish_roots<kW, kStats, true, true>(p, sm, t, par, c0, c1, cap, rec);
            if (!grid_sync(p.bar, p.ctl, p.tstamp, 3 * t + 2, p.spin_limit, p.skip_mark)) return;
        }
    } else {
        // speculative: a called-off attempt leaves only values that the
        // resumed rounds write again
        finish_scan<kW, kStats, true>(p, sm, t, par, c0, c1, cap, rec);
        if (!grid_sync(p.bar, p.ctl, p.tstamp, 3 * t + 1, p.spin_limit, p.skip_mark)) return;
        done = __ldcg(&ctl->fin_abort) != t + 1;
        if (done) {
            finish_roots<kW, kStats, true, false>(p, sm, t, par, c0, c1, cap, rec);
            if (!grid_sync(p.bar, p.ctl, p.tstamp, 3 * t + 2, p.spin_limit, p.skip_mark)) return;
            done = __ldcg(&ctl->fin_abort) != t + 1;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (done) {
            const int last = max(__ldcg(&ctl->fin_last), __ldcg(&ctl->iso_last) - 1);
            ctl->rounds = maximal ? min(last + 2, cap) : cap;
            ctl->fin_state = kFinStateDone;
            if (p.tstamp) p.tstamp[3 * t + 3] = p.tstamp[3 * t + 2];
        } else {
            ctl->fin_state = kFinStateResume;
        }
    }
}

// ---------------------------------------------------------------------------
// Preparation: degree classes and reverse proposal keys.

struct PrepInfo {
    unsigned long long sum_deg;
    unsigned long long max_deg;
    unsigned long long short_count;   // lists of at most kWin entries
    unsigned long long long_count;    // longer lists
    unsigned long long long_entries;  // entries in longer lists
    int noncontig;
    int pad;
};

__global__ void k_scan_ranges(const int2 *ranges, int n, long long nnz, PrepInfo *info, long long *deg_out)
{
    unsigned long long sum = 0, mx = 0, nshort = 0, nlong = 0, elong = 0;
    int nc = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int2 r = ranges[v];
        const int d = degree_of(r);
        sum += d;
        mx = d > (long long)mx ? d : mx;
        if (d > kWin) {
            nlong += 1;
            elong += d;
        } else {
            nshort += 1;
        }
        if (deg_out) deg_out[v] = d;
        if (r.y < r.x) nc = 1;
        if (v == 0 && r.x != 0) nc = 1;
        if (v + 1 < n && ranges[v + 1].x != r.y) nc = 1;
        if (v == n - 1 && (long long)r.y != nnz) nc = 1;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_down_sync(kFull, sum, o);
        const unsigned long long m2 = __shfl_down_sync(kFull, mx, o);
        mx = m2 > mx ? m2 : mx;
        nshort += __shfl_down_sync(kFull, nshort, o);
        nlong += __shfl_down_sync(kFull, nlong, o);
        elong += __shfl_down_sync(kFull, elong, o);
        nc |= __shfl_down_sync(kFull, nc, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (sum) atomicAdd(&info->sum_deg, sum);
        if (mx) atomicMax(&info->max_deg, mx);
        if (nshort) atomicAdd(&info->short_count, nshort);
        if (nlong) atomicAdd(&info->long_count, nlong);
        if (elong) atomicAdd(&info->long_entries, elong);
        if (nc) atomicOr(&info->noncontig, 1);
    }
}

// One item per (owner, slot): key = (min << B | max) << 1 | (owner == max).
__global__ void k_pair_items(const int2 *ranges, const int *nbrs, int n, int bits, int contiguous,
                             const long long *slot_off, unsigned long long *keys, int *vals)
{
    const int lane = threadIdx.x & 31;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long v = warp0; v < n; v += nwarps) {
        const int2 r = ranges[v];
        const long long s0 = contiguous ? (long long)r.x : slot_off[v];
        for (int j = r.x + lane; j < r.y; j += 32) {
            const unsigned long long a = (unsigned long long)v, b = (unsigned long long)nbrs[j];
            const unsigned long long lo = a < b ? a : b, hi = a < b ? b : a;
            const long long slot = s0 + (j - r.x);
            keys[slot] = (((lo << bits) | hi) << 1) | (a > b ? 1ull : 0ull);
            vals[slot] = (int)slot;
        }
    }
}

// Key red `owner` gives the entry at `slot` of its own list (the revkey form:
// 0 for weights the reference can never pick).
template <bool kW>
__device__ __forceinline__ unsigned long long red_key(const int2 *ranges, const float *w, int contiguous,
                                                      const long long *slot_off, long long owner, long long slot)
{
    const long long pos = contiguous ? slot : (long long)ranges[owner].x + (slot - slot_off[owner]);
    if (kW) {
        const float x = w[pos];
        return x > -1.0f ? (((unsigned long long)weight_order(x) << 32) | (uint32_t)~(int)pos) : 0ull;
    }
    return (unsigned long long)(uint32_t)~(int)pos;
}

// For each group of equal unordered pair, give every item the best key of the
// opposite direction.  Groups are walked by their first item.
template <bool kW>
__global__ void k_pair_groups(const unsigned long long *keys, const int *vals, long long count, int bits,
                              const int2 *ranges, const float *w, int contiguous, const long long *slot_off,
                              unsigned long long *revkey)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < count;
         q += (long long)gridDim.x * blockDim.x) {
        const unsigned long long kq = keys[q] >> 1;
        if (q > 0 && (keys[q - 1] >> 1) == kq) continue;
        const long long lo = (long long)(kq >> bits), hi = (long long)(kq & ((1ull << bits) - 1));
        long long end = q + 1;
        while (end < count && (keys[end] >> 1) == kq) ++end;
        if (lo == hi) {  // self-loops never carry a proposal
            for (long long x = q; x < end; ++x) revkey[vals[x]] = 0ull;
            continue;
        }
        unsigned long long best_dir[2] = {0ull, 0ull};
        for (long long x = q; x < end; ++x) {
            const int dir = (int)(keys[x] & 1ull);
            const long long owner = dir ? hi : lo;
            const unsigned long long k = red_key<kW>(ranges, w, contiguous, slot_off, owner, vals[x]);
            best_dir[dir] = k > best_dir[dir] ? k : best_dir[dir];
        }
        for (long long x = q; x < end; ++x) revkey[vals[x]] = best_dir[(keys[x] & 1ull) ^ 1ull];
    }
}

// ---- preference windows (weighted types) ----
//
// pwin holds, for every vertex, its best min(deg, 32) entries in the order in
// which the reference's gwRequest would prefer them: candidates (weight > -1)
// by weight, then earlier position; entries whose weight can never be picked
// after them, flagged by bit 31 of the position.  A vertex's window starts at
// pwin_off[v], an even slot (pairs are read as one 16-byte load).
__device__ __forceinline__ unsigned long long pref_key(float w, int j)
{
    return w > -1.0f ? (((unsigned long long)weight_order(w) << 32) | (uint32_t)~j) : (unsigned long long)(uint32_t)~j;
}

// One compare-exchange step of a bitonic network across the warp: the lower
// lane of each pair keeps the larger key in a descending block.
__device__ __forceinline__ void cas_step(unsigned long long &k, int &nb, int &j, int lane, int stride, bool desc)
{
    const unsigned long long ok = __shfl_xor_sync(kFull, k, stride);
    const int onb = __shfl_xor_sync(kFull, nb, stride);
    const int oj = __shfl_xor_sync(kFull, j, stride);
    const bool lower = (lane & stride) == 0;
    if (lower == desc ? ok > k : ok < k) {
        k = ok;
        nb = onb;
        j = oj;
    }
}

__device__ __forceinline__ void warp_sort_desc(unsigned long long &k, int &nb, int &j, int lane)
{
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1)
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) cas_step(k, nb, j, lane, stride, (lane & size) == 0);
}

__global__ void k_win_sizes(const int2 *ranges, int n, long long *slots)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        slots[v] = (win_len(degree_of(ranges[v])) + 1) & ~1;
}

constexpr int kWinRows = 8;       // rows of 32 entries tested against the window threshold per step
constexpr int kWinChunk = 4096;   // lists longer than this are split into chunks of this many entries

// Merge entries [from, to) of a list into its sorted best 32 (k, nb, j): a row
// can change them only if one of its keys beats the 32nd.
__device__ __forceinline__ void win_merge_range(const int *nbrs, const float *w, int from, int to, int lane,
                                                unsigned long long &k, int &nb, int &j)
{
    for (int base = from; base < to; base += 32 * kWinRows) {
        float wr[kWinRows];
#pragma unroll
        for (int q = 0; q < kWinRows; ++q) {
            const int jj = base + q * 32 + lane;
            wr[q] = jj < to ? __ldg(w + jj) : 0.0f;
        }
#pragma unroll
        for (int q = 0; q < kWinRows; ++q) {
            const int jj = base + q * 32 + lane;
            if (base + q * 32 >= to) break;
            const unsigned long long thr = __shfl_sync(kFull, k, 31);
            unsigned long long k2 = jj < to ? pref_key(wr[q], jj) : 0ull;
            if (!__any_sync(kFull, k2 > thr)) continue;
            int nb2 = jj < to ? __ldg(nbrs + jj) : 0, j2 = jj;
            warp_sort_desc(k2, nb2, j2, lane);
            // the larger of T[l] and R[31 - l] is a bitonic sequence holding
            // the best 32 of both; sort it descending
            const unsigned long long rk = __shfl_sync(kFull, k2, 31 - lane);
            const int rnb = __shfl_sync(kFull, nb2, 31 - lane), rj = __shfl_sync(kFull, j2, 31 - lane);
            if (rk > k) {
                k = rk;
                nb = rnb;
                j = rj;
            }
#pragma unroll
            for (int stride = 16; stride > 0; stride >>= 1) cas_step(k, nb, j, lane, stride, true);
        }
    }
}

// Best 32 entries of [from, to): the first 32 sorted, then the rest merged in.
__device__ __forceinline__ void win_top32(const int *nbrs, const float *w, int from, int to, int lane,
                                          unsigned long long &k, int &nb, int &j)
{
    k = 0ull;
    nb = 0;
    j = 0;
    if (from + lane < to) {
        j = from + lane;
        nb = __ldg(nbrs + j);
        k = pref_key(__ldg(w + j), j);
    }
    warp_sort_desc(k, nb, j, lane);
    if (to - from > 32) win_merge_range(nbrs, w, from + 32, to, lane, k, nb, j);
}

__device__ __forceinline__ void win_store(int2 *pwin, long long off, int deg, int lane, unsigned long long k, int nb, int j)
{
    if (lane < win_len(deg)) pwin[off + lane] = make_int2(nb, k >= (1ull << 32) ? j : (int)((unsigned)j | 0x80000000u));
}

// Windows of lists of at most kWinChunk entries, a warp per list (vertices
// dealt round-robin, so long lists spread over the grid); longer lists are
// queued for the chunked kernels.
__global__ void __launch_bounds__(256) k_win_build(const int2 *ranges, const int *nbrs, const float *w, int va, int vb,
                                                   const long long *pwin_off, int2 *pwin, int *big, int *nbig)
{
    const int lane = threadIdx.x & 31;
    const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long v = va + gwarp; v < vb; v += nwarps) {
        const int2 r = ranges[v];
        const int deg = degree_of(r);
        if (deg == 0) continue;
        if (deg > kWinChunk) {
            if (lane == 0) big[atomicAdd(nbig, 1)] = (int)v;
            continue;
        }
        unsigned long long k;
        int nb, j;
        win_top32(nbrs, w, r.x, r.y, lane, k, nb, j);
        win_store(pwin, pwin_off[v], deg, lane, k, nb, j);
    }
}

// Chunked lists, step 1: the best 32 of every kWinChunk-entry chunk of every
// queued list, a warp per chunk.  cand holds 32 {key, nb, j} per chunk.
struct WinCand {
    unsigned long long k;
    int nb;
    int j;
};

__global__ void __launch_bounds__(256) k_win_chunks(const int2 *ranges, const int *nbrs, const float *w,
                                                    const int *big, int nbig, const long long *chunk_off,
                                                    WinCand *cand)
{
    const int lane = threadIdx.x & 31;
    const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long total = chunk_off[nbig];
    for (long long c = gwarp; c < total; c += nwarps) {
        int lo = 0, hi = nbig - 1;  // the list holding chunk c: largest i with chunk_off[i] <= c
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (chunk_off[mid] <= c) lo = mid;
            else hi = mid - 1;
        }
        const int2 r = ranges[big[lo]];
        const int from = r.x + (int)(c - chunk_off[lo]) * kWinChunk;
        const int to = min(from + kWinChunk, r.y);
        unsigned long long k;
        int nb, j;
        win_top32(nbrs, w, from, to, lane, k, nb, j);
        cand[c * 32 + lane] = WinCand{k, nb, j};
    }
}

__global__ void k_win_chunk_counts(const int2 *ranges, const int *big, int nbig, long long *counts)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nbig; i += gridDim.x * blockDim.x)
        counts[i] = (degree_of(ranges[big[i]]) + kWinChunk - 1) / kWinChunk;
}

// Chunked lists, step 2: a warp per list merges its chunks' sorted best 32s.
__global__ void __launch_bounds__(256) k_win_chunk_merge(const int2 *ranges, const int *big, int nbig,
                                                         const long long *chunk_off, const WinCand *cand,
                                                         const long long *pwin_off, int2 *pwin)
{
    const int lane = threadIdx.x & 31;
    const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long i = gwarp; i < nbig; i += nwarps) {
        const long long c0 = chunk_off[i], c1 = chunk_off[i + 1];
        WinCand x = cand[c0 * 32 + lane];
        unsigned long long k = x.k;
        int nb = x.nb, j = x.j;
        for (long long c = c0 + 1; c < c1; ++c) {
            const WinCand y = cand[c * 32 + (31 - lane)];  // reversed: the pairwise larger is bitonic
            if (y.k > k) {
                k = y.k;
                nb = y.nb;
                j = y.j;
            }
#pragma unroll
            for (int stride = 16; stride > 0; stride >>= 1) cas_step(k, nb, j, lane, stride, true);
        }
        const int v = big[i];
        win_store(pwin, pwin_off[v], degree_of(ranges[v]), lane, k, nb, j);
    }
}

// ---- reverse keys from sorted lists ----------------------------------------
// When every neighbour list is sorted, the entries of u that point back at v
// form one run in u's list, found by binary search.  Of the two entries of a
// pair {v, u} only the one whose partner list is shorter searches (ties by
// id): it finds the run of entries pointing back in the partner's list, stores
// the best of their keys in its own slot (pull) and max-combines its own key
// into the slots of that run (push), which nobody else writes.  Each pair thus
// costs one search in its shorter list; hub lists are never searched by their
// many neighbours.  Slots are cut into chunks of kRevChunk; k_chunk_owner
// finds the vertex owning each chunk's first slot, k_revkey_sorted resolves
// the owner of every slot in shared memory and checks sortedness on the way
// (any descending neighbour pair sets *unsorted and the pair-sort build runs).
// revkey must be zero on entry.
constexpr int kRevChunk = 2048;
constexpr int kRevThreads = 256;

__device__ __forceinline__ long long slot_prefix(const int2 *ranges, int contiguous, const long long *slot_off,
                                                 long long v)
{
    return contiguous ? (long long)ranges[v].x : slot_off[v];
}

// Owner of slot s: the largest v with prefix(v) <= s.
__device__ __forceinline__ int owner_of(const int2 *ranges, int contiguous, const long long *slot_off, int lo, int hi,
                                        long long s)
{
    while (lo < hi) {
        const int mid = (int)(((long long)lo + hi + 1) >> 1);
        if (slot_prefix(ranges, contiguous, slot_off, mid) <= s) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void k_chunk_owner(const int2 *ranges, int n, int contiguous, const long long *slot_off, long long S,
                              int *chunk_v)
{
    const long long chunks = (S + kRevChunk - 1) / kRevChunk;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c <= chunks;
         c += (long long)gridDim.x * blockDim.x) {
        const long long s = c * kRevChunk < S ? c * kRevChunk : S - 1;
        chunk_v[c] = owner_of(ranges, contiguous, slot_off, 0, n - 1, s);
    }
}

// Key red `owner` gives its entry at absolute position q (0: never picked).
template <bool kW>
__device__ __forceinline__ unsigned long long entry_red_key(const float *w, int q)
{
    if (kW) {
        const float x = __ldg(w + q);
        return x > -1.0f ? (((unsigned long long)weight_order(x) << 32) | (uint32_t)~q) : 0ull;
    }
    return (unsigned long long)(uint32_t)~q;
}

template <bool kW>
__global__ void __launch_bounds__(kRevThreads) k_revkey_sorted(const int2 *ranges, const int *nbrs, const float *w,
                                                               int contiguous, const long long *slot_off, long long S,
                                                               const int *chunk_v, unsigned long long *revkey,
                                                               int *unsorted)
{
    constexpr int kCap = kRevChunk + 1;
    __shared__ int pre[kCap];  // prefix(v0 + i) - chunk start
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    const long long chunks = (S + kRevChunk - 1) / kRevChunk;
    for (long long c = blockIdx.x; c < chunks; c += gridDim.x) {
        const long long s0 = c * kRevChunk;
        const int v0 = chunk_v[c], v1 = chunk_v[c + 1];
        const int cnt = v1 - v0 + 1;
        const bool in_smem = cnt <= kCap;
        __syncthreads();
        if (in_smem)
            for (int i = threadIdx.x; i < cnt; i += kRevThreads)
                pre[i] = (int)(slot_prefix(ranges, contiguous, slot_off, v0 + i) - s0);
        __syncthreads();
        for (int k = threadIdx.x; k < kRevChunk; k += kRevThreads) {
            const long long s = s0 + k;
            if (s >= S) break;
            int v;
            if (in_smem) {
                int lo = 0, hi = cnt - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (pre[mid] <= k) lo = mid;
                    else hi = mid - 1;
                }
                v = v0 + lo;
            } else {
                v = owner_of(ranges, contiguous, slot_off, v0, v1, s);
            }
            const int2 rv = ranges[v];
            const int pos = contiguous ? (int)s : (int)(rv.x + (s - slot_off[v]));
            const int u = nbrs[pos];
            if (pos + 1 < rv.y && nbrs[pos + 1] < u) bad = 1;
            if (u == v) continue;  // self-loops never carry a proposal
            const int2 ru = ranges[u];
            const int dv = degree_of(rv), du = degree_of(ru);
            if (du > dv || (du == dv && u > v)) continue;  // u's entries search my list and push here
            int lo = ru.x, hi = ru.x + du;  // first entry >= v in u's list
            while (lo < hi) {
                const int mid = (int)(((long long)lo + hi) >> 1);
                if (__ldg(nbrs + mid) < v) lo = mid + 1;
                else hi = mid;
            }
            const unsigned long long mine = entry_red_key<kW>(w, pos);
            const long long su0 = contiguous ? 0ll : slot_off[u] - ru.x;  // slot of entry q of u: su0 + q
            unsigned long long key = 0ull;
            for (int q = lo; q < ru.x + du && __ldg(nbrs + q) == v; ++q) {
                const unsigned long long kq = entry_red_key<kW>(w, q);
                key = kq > key ? kq : key;
                if (mine) atomicMax(revkey + su0 + q, mine);
            }
            if (key) revkey[s] = key;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && bad) atomicOr(unsorted, 1);
}


int bits_for(long long n)
{
    int b = 1;
    while ((1ll << b) < n) ++b;
    return b;
}

// Weight features of the learned colouring: max and mean of the weights a
// blue vertex could pick (> -1), 0 without any; a warp per vertex.
__global__ void k_wfeat(const int2 *ranges, const float *w, int n, float2 *wfeat)
{
    const int lane = threadIdx.x & 31;
    const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long v = gwarp; v < n; v += nwarps) {
        const int2 r = ranges[v];
        float mx = 0.0f, sum = 0.0f;
        int cnt = 0;
        for (int j = r.x + lane; j < r.y; j += 32) {
            const float x = __ldg(w + j);
            if (x > -1.0f) {
                mx = cnt ? fmaxf(mx, x) : x;
                sum += x;
                ++cnt;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float m2 = __shfl_xor_sync(kFull, mx, o);
            const int c2 = __shfl_xor_sync(kFull, cnt, o);
            mx = c2 && (!cnt || m2 > mx) ? m2 : mx;
            sum += __shfl_xor_sync(kFull, sum, o);
            cnt += c2;
        }
        if (lane == 0) wfeat[v] = make_float2(mx, cnt ? sum / (float)cnt : 0.0f);
    }
}

// Rounds of each graph of a batch: the reference's loop for a graph runs
// until a round finds none of its vertices unmatched at the colouring, so it
// executes its last active round and one more (at most the cap; an empty
// graph runs one round).  A warp per graph takes the max of last[].
__global__ void k_batch_rounds(const uint8_t *last, const int *goff, int ngraphs, int cap, int fixed, int *rounds)
{
    const int lane = threadIdx.x & 31;
    const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long gi = gwarp; gi < ngraphs; gi += nwarps) {
        int mx = -1;
        for (int v = goff[gi] + lane; v < goff[gi + 1]; v += 32) mx = max(mx, (int)last[v]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(kFull, mx, o));
        if (lane == 0) rounds[gi] = fixed ? cap : min(mx + 2, cap);
    }
}

// Control block rounded to 256 bytes so the seeds that follow it stay aligned.
constexpr size_t kCtlBytes = (sizeof(Ctl) + 255) / 256 * 256;
constexpr int kStampCount = 3 * kMaxRounds + 1;

struct PushState {
    uint8_t *col = nullptr;
    int2 *req = nullptr;
    int2 *reqi = nullptr;
    unsigned long long *best = nullptr;
    unsigned long long *part_key = nullptr;
    int *part_cnt = nullptr;
    int4 *list_mem = nullptr;
    int4 *lists[2][kParityLists] = {};
    int4 *staged = nullptr;
    int *seg_first = nullptr;
    uint32_t *seeds = nullptr;        // device: right after ctl in one allocation
    Ctl *ctl = nullptr;
    unsigned char *host_stage = nullptr;  // pinned: control block + seeds, uploaded in one copy
    unsigned char *host_back = nullptr;   // pinned: control block read back
    unsigned long long *stats = nullptr;
    unsigned long long *tstamp = nullptr;
    unsigned *bar = nullptr;
    int grid[2][3] = {{0, 0, 0}, {0, 0, 0}};  // co-resident blocks of k_rounds by weighting and mode
    int fgrid[2][2] = {{0, 0}, {0, 0}};       // co-resident blocks of k_finish by weighting and stats
    int sms = 0;                              // multiprocessors of the device
    // The last call on this state ended with every grid barrier complete (the
    // barrier words are back at rest) and every fallback list combined (part_key
    // and part_cnt all zero); false after a call that gave up or failed.
    bool at_rest = false;
    bool zero_next = true;  // the call being launched resets them (the last one did not end at rest)
    float2 *wfeat = nullptr;              // learned colouring: (max, mean) incident weight per vertex
};

void free_state(PushState *s)
{
    // callers have synchronised the device (graph destroy or a failed set-up)
    dev_free(s->col, 0);
    dev_free(s->req, 0);
    dev_free(s->reqi, 0);
    dev_free(s->best, 0);
    dev_free(s->part_key, 0);
    dev_free(s->part_cnt, 0);
    dev_free(s->list_mem, 0);
    dev_free(s->staged, 0);
    dev_free(s->seg_first, 0);
    dev_free(s->ctl, 0);
    pinned_put(s->host_stage, kCtlBytes + 256 * sizeof(uint32_t));
    pinned_put(s->host_back, kCtlBytes);
    dev_free(s->stats, 0);
    dev_free(s->tstamp, 0);
    dev_free(s->bar, 0);
    dev_free(s->wfeat, 0);
    delete s;
}

template <bool kW, bool kStats>
int coresident_finish_blocks(int sms)
{
    int occ = 0;
    if (cudaFuncSetAttribute(k_finish<kW, kStats>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem)) !=
        cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_finish<kW, kStats>, kThreads, sizeof(Smem)) != cudaSuccess)
        return 0;
    return occ * sms;
}

template <bool kW, bool kStats, bool kPolicy>
int coresident_blocks(int sms)
{
    int occ = 0;
    if (cudaFuncSetAttribute(k_rounds<kW, kStats, kPolicy>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(Smem)) != cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rounds<kW, kStats, kPolicy>, kThreads, sizeof(Smem)) !=
        cudaSuccess)
        return 0;
    return occ * sms;
}

mm_status alloc_state(mm_graph *g, PushState **out)
{
    PushState *s = new (std::nothrow) PushState();
    if (!s) {
        set_error("push: host allocation failed");
        return MM_ERR_NOMEM;
    }
    const size_t n = (size_t)(g->n > 0 ? g->n : 1);
    // list capacities: every vertex is in at most one list per parity; only
    // lists longer than the window can fall back
    const size_t nseg_cap = (size_t)(g->long_entries / kSegEntries) + 2;
    const size_t nstaged = (size_t)(g->long_count > 0 ? g->long_count : 1);
    // pooled on the legacy stream, then synchronised so that any stream may use them
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = dev_alloc((void **)&s->col, n, 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->req, n * sizeof(int2), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->reqi, n * sizeof(int2), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->best, n * sizeof(unsigned long long), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->part_key, n * sizeof(unsigned long long), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->part_cnt, n * sizeof(int), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->list_mem, 4 * n * sizeof(int4), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->staged, nstaged * sizeof(int4), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->seg_first, nseg_cap * sizeof(int), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->ctl, kCtlBytes + 256 * sizeof(uint32_t), 0);
    if (e == cudaSuccess) s->seeds = reinterpret_cast<uint32_t *>(reinterpret_cast<unsigned char *>(s->ctl) + kCtlBytes);
    if (e == cudaSuccess) e = pinned_get((void **)&s->host_stage, kCtlBytes + 256 * sizeof(uint32_t));
    if (e == cudaSuccess) e = pinned_get((void **)&s->host_back, kCtlBytes);
    if (e == cudaSuccess)
        e = dev_alloc((void **)&s->stats, sizeof(unsigned long long) * kMaxRounds * MM_STATS_COLS, 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->tstamp, sizeof(unsigned long long) * kStampCount, 0);
    // two sets of barrier words: the round kernel's and the finish kernel's
    if (e == cudaSuccess) e = dev_alloc((void **)&s->bar, sizeof(unsigned) * 2 * kBarWords, 0);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->bar, 0, sizeof(unsigned) * 2 * kBarWords, 0);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->part_key, 0, n * sizeof(unsigned long long), 0);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->part_cnt, 0, n * sizeof(int), 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        cudaDeviceSynchronize();
        free_state(s);
        cudaGetLastError();
        set_error(std::string("push: device allocation failed: ") + cudaGetErrorString(e));
        return MM_ERR_NOMEM;
    }
    // a parity's two lists are adjacent: the finish phase uses both as one array of 2n
    for (int par = 0; par < 2; ++par)
        for (int l = 0; l < kParityLists; ++l) s->lists[par][l] = s->list_mem + (2 * par + l) * n;
    int sms = 0, dev = 0, coop = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    s->sms = sms;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    s->grid[0][0] = coresident_blocks<false, false, false>(sms);
    s->grid[0][1] = coresident_blocks<false, true, false>(sms);
    s->grid[0][2] = coresident_blocks<false, false, true>(sms);
    s->grid[1][0] = coresident_blocks<true, false, false>(sms);
    s->grid[1][1] = coresident_blocks<true, true, false>(sms);
    s->grid[1][2] = coresident_blocks<true, false, true>(sms);
    s->fgrid[0][0] = coresident_finish_blocks<false, false>(sms);
    s->fgrid[0][1] = coresident_finish_blocks<false, true>(sms);
    s->fgrid[1][0] = coresident_finish_blocks<true, false>(sms);
    s->fgrid[1][1] = coresident_finish_blocks<true, true>(sms);
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
        free_state(s);
        return cuda_fail(le, "push: kernel attributes");
    }
    const int most = kBarMaxGroups * kBarGroup;
    bool over = false, under = false;
    for (int a = 0; a < 2; ++a) {
        for (int b = 0; b < 3; ++b) {
            over |= s->grid[a][b] > most;
            under |= s->grid[a][b] < 1;
        }
        for (int b = 0; b < 2; ++b) {
            over |= s->fgrid[a][b] > most;
            under |= s->fgrid[a][b] < 1;
        }
    }
    if (over) {
        free_state(s);
        set_error("push: more co-resident blocks than the grid barrier supports");
        return MM_ERR_UNSUPPORTED;
    }
    if (!coop || under) {
        free_state(s);
        set_error("push: the device cannot run the cooperative round kernel");
        return MM_ERR_UNSUPPORTED;
    }
    s->at_rest = true;
    *out = s;
    return MM_OK;
}

Params make_params(mm_graph *g, PushState *s, bool weighted, bool stats, bool timing)
{
    Params p;
    p.n = g->n;
    p.contiguous = g->contiguous ? 1 : 0;
    p.sym = (weighted ? g->sym_weights : g->sym_struct) ? 1 : 0;
    p.ranges = g->d_ranges;
    p.nbrs = g->d_nbrs;
    p.w = g->d_w;
    p.revkey = g->d_revkey[weighted ? 1 : 0];
    p.slot_off = g->d_slot_off;
    p.pwin = g->d_pwin;
    p.wwin = weighted && g->pwin_weights ? 1 : 0;
    p.pwin_off = g->d_pwin_off;
    p.col = s->col;
    p.req = s->req;
    p.reqi = s->reqi;
    p.best = s->best;
    p.part_key = s->part_key;
    p.part_cnt = s->part_cnt;
    for (int par = 0; par < 2; ++par)
        for (int l = 0; l < kParityLists; ++l) p.lists[par][l] = s->lists[par][l];
    p.staged = s->staged;
    p.seg_first = s->seg_first;
    p.vbase = g->ngraphs > 0 ? g->d_vbase : nullptr;
    p.last = g->ngraphs > 0 ? g->d_last : nullptr;
    std::memset(p.mlp, 0, sizeof(p.mlp));
    p.policy_const = 0;
    p.policy_bar = 0u;
    p.fin_retire = 0;
    p.level = 0.0f;
    p.wfeat = s->wfeat;
    p.trace = nullptr;
    p.trace_rounds = 0;
    p.seeds = s->seeds;
    p.ctl = s->ctl;
    p.stats = stats ? s->stats : nullptr;
    p.tstamp = timing ? s->tstamp : nullptr;
    p.bar = s->bar;
    p.resume = 0;
    p.zero_parts = s->zero_next ? 1 : 0;
    // at least 2: the finish phase's records take 4 slots an item in 2n
    p.fin_div = g->opt_fin_div < 0 ? 0 : (g->opt_fin_div == 0 ? kFinDiv : max(g->opt_fin_div, 2));
    p.spin_limit = debug_spin_limit();
    p.skip_mark = debug_skip_mark();
    return p;
}

struct PolicyArgs {
    const float *mlp = nullptr;  // host, MM_POLICY_FLOATS
    bool constant = false;       // output weights all zero: the threshold is constant_bar
    uint32_t constant_bar = 0u;
    float level = 0.0f;
    float *trace = nullptr;
    int trace_rounds = 0;
};

template <bool kW, bool kStats, bool kPolicy>
mm_status launch_rounds(mm_graph *g, PushState *s, bool timing, cudaStream_t stream, const PolicyArgs *pol = nullptr)
{
    Params prm = make_params(g, s, kW, kStats, timing);
    if (kPolicy) {
        std::memcpy(prm.mlp, pol->mlp, sizeof(prm.mlp));
        prm.policy_const = pol->constant ? 1 : 0;
        prm.policy_bar = pol->constant_bar;
        prm.level = pol->level;
        prm.trace = pol->trace;
        prm.trace_rounds = pol->trace_rounds;
        // the finish phase knows the policy's threshold, not its features
        prm.fin_retire = pol->constant && !pol->trace ? 1 : 0;
        // Retirement shrinks the active set from round kRetireFrom on, so the
        // default threshold comes a round or two earlier than on the plain
        // path, while components are still too large for the finish phase (on
        // the R-MAT 2^22 hierarchy every level but the first called its attempt
        // off, and the round kernel then played all the remaining rounds): the
        // default divisor is doubled here.
        if (g->opt_fin_div == 0) prm.fin_div = 2 * kFinDiv;
    }
    void *args[] = {&prm};
    const int mode = kPolicy ? 2 : (kStats ? 1 : 0);
    // blocks: all that fit at once, or the tuned number per SM (never more)
    const int bps = g->opt_blocks_per_sm;
    const int grid = bps > 0 ? min(s->grid[kW][mode], bps * s->sms) : s->grid[kW][mode];
    const int fgrid = bps > 0 ? min(s->fgrid[kW][kStats ? 1 : 0], bps * s->sms) : s->fgrid[kW][kStats ? 1 : 0];
    MM_CUDA_TRY(cudaLaunchCooperativeKernel((void *)k_rounds<kW, kStats, kPolicy>, dim3(grid),
                                            dim3(kThreads), args, sizeof(Smem), stream),
                "round kernel launch");
    if ((!kPolicy || prm.fin_retire) && prm.sym) {
        // the finish kernel (its own barrier words), then the round kernel again
        // for the case that the finish phase is called off; each returns at once
        // when there is nothing left for it
        Params fin = prm;
        fin.bar = s->bar + kBarWords;
        void *fargs[] = {&fin};
        MM_CUDA_TRY(cudaLaunchCooperativeKernel((void *)k_finish<kW, kStats>, dim3(fgrid),
                                                dim3(kThreads), fargs, sizeof(Smem), stream),
                    "finish kernel launch");
        Params res = prm;
        res.resume = 1;
        void *rargs[] = {&res};
        MM_CUDA_TRY(cudaLaunchCooperativeKernel((void *)k_rounds<kW, kStats, kPolicy>, dim3(grid),
                                                dim3(kThreads), rargs, sizeof(Smem), stream),
                    "round kernel launch (resumed)");
    }
    return MM_OK;
}

// Shared set-up of one matching call: preparation, state, control block.
mm_status begin_call(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds, int *d_match,
                     cudaStream_t stream, PushState **out)
{
    mm_status st = push_prepare(g, is_weighted(type) ? 1 : 0, stream);
    if (st != MM_OK) return st;
    PushState *s = (PushState *)g->push_exec;
    if (!s) {
        st = alloc_state(g, &s);
        if (st != MM_OK) return st;
        g->push_exec = s;
    }
    // One pinned upload of control block + seeds.  The previous call on this
    // graph synchronised its stream before returning, so the staging buffer is free.
    // the barrier words: reset only after a call that did not end at rest; until
    // this call ends well, the state counts as not at rest
    s->zero_next = !s->at_rest;
    s->at_rest = false;
    if (s->zero_next)
        MM_CUDA_TRY(cudaMemsetAsync(s->bar, 0, sizeof(unsigned) * 2 * kBarWords, stream), "barrier clear");
    Ctl *ctl = reinterpret_cast<Ctl *>(s->host_stage);
    std::memset(ctl, 0, kCtlBytes);
    ctl->match = d_match;
    ctl->barrier = barrier;
    ctl->cap = max_rounds_of(type);
    ctl->maximal = is_maximal(type) ? 1 : 0;
    ctl->nseeds = nseeds < 256 ? nseeds : 256;
    std::memcpy(s->host_stage + kCtlBytes, seeds, sizeof(uint32_t) * ctl->nseeds);
    MM_CUDA_TRY(cudaMemcpyAsync(s->ctl, s->host_stage, kCtlBytes + sizeof(uint32_t) * ctl->nseeds,
                                cudaMemcpyHostToDevice, stream),
                "control block");
    *out = s;
    return MM_OK;
}

mm_status end_call(mm_graph *g, PushState *s, int nseeds, int *rounds_out, long long *stats, int stats_rounds,
                   unsigned long long *stamps, cudaStream_t stream)
{
    MM_CUDA_TRY(cudaMemcpyAsync(s->host_back, s->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream), "control read");
    if (stats && stats_rounds > 0)
        MM_CUDA_TRY(cudaMemcpyAsync(stats, s->stats,
                                    sizeof(long long) * MM_STATS_COLS *
                                        (size_t)(stats_rounds < kMaxRounds ? stats_rounds : kMaxRounds),
                                    cudaMemcpyDeviceToHost, stream),
                    "stats read");
    if (stamps)
        MM_CUDA_TRY(cudaMemcpyAsync(stamps, s->tstamp, sizeof(unsigned long long) * kStampCount,
                                    cudaMemcpyDeviceToHost, stream),
                    "timestamps read");
    MM_CUDA_TRY(cudaStreamSynchronize(stream), "round loop");
    Ctl out;
    std::memcpy(&out, s->host_back, sizeof out);
    // every barrier completed unless one gave up (status 2)
    s->at_rest = out.status != 2;
    if (out.status == 2) {
        set_error("mm_match: a bounded grid-barrier wait in the round kernel gave up");
        return MM_ERR_DEVICE;
    }
    if (out.status == 1 || out.rounds > nseeds) {
        set_error("mm_match: fewer seeds than rounds");
        return MM_ERR_SEEDS;
    }
    *rounds_out = out.rounds;
    return MM_OK;
}

mm_status run_rounds(mm_graph *g, PushState *s, int type, bool stats, bool timing, cudaStream_t stream)
{
    const bool w = is_weighted(type);
    if (stats)
        MM_CUDA_TRY(cudaMemsetAsync(s->stats, 0, sizeof(unsigned long long) * kMaxRounds * MM_STATS_COLS, stream),
                    "stats clear");
    if (w)
        return stats ? launch_rounds<true, true, false>(g, s, timing, stream)
                     : launch_rounds<true, false, false>(g, s, timing, stream);
    return stats ? launch_rounds<false, true, false>(g, s, timing, stream)
                 : launch_rounds<false, false, false>(g, s, timing, stream);
}

}  // namespace


namespace {

// Degrees, classes, contiguity, slot offsets (once per graph).
mm_status scan_graph(mm_graph *g, cudaStream_t stream)
{
    const int n = g->n;
    if (n == 0 || g->scanned) return MM_OK;
    {
        PrepInfo *d_info = nullptr;
        long long *d_deg = nullptr;
        MM_CUDA_TRY(dev_alloc((void **)&d_info, sizeof(PrepInfo), stream), "prep info");
        MM_CUDA_TRY(cudaMemsetAsync(d_info, 0, sizeof(PrepInfo), stream), "prep info clear");
        cudaError_t e = dev_alloc((void **)&d_deg, sizeof(long long) * (size_t)n, stream);
        if (e != cudaSuccess) {
            dev_free(d_info, stream);
            return cuda_fail(e, "prep degrees");
        }
        k_scan_ranges<<<grid_for(n, 256, 148 * 8), 256, 0, stream>>>(g->d_ranges, n, g->nnz, d_info, d_deg);
        PrepInfo info;
        e = cudaMemcpyAsync(&info, d_info, sizeof info, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        dev_free(d_info, stream);
        if (e != cudaSuccess) {
            dev_free(d_deg, stream);
            return cuda_fail(e, "prep scan");
        }
        g->sum_degree = (long long)info.sum_deg;
        g->max_degree = (long long)info.max_deg;
        g->short_count = (long long)info.short_count;
        g->long_count = (long long)info.long_count;
        g->long_entries = (long long)info.long_entries;
        g->contiguous = info.noncontig == 0;
        if (g->sum_degree >= (1ll << 31) - 1) {
            dev_free(d_deg, stream);
            set_error("push: more than 2^31 - 2 adjacency slots are not supported");
            return MM_ERR_UNSUPPORTED;
        }
        if (!g->contiguous) {
            e = dev_alloc((void **)&g->d_slot_off, sizeof(long long) * (size_t)n, stream);
            void *tmp = nullptr;
            size_t tmp_bytes = 0;
            if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_deg, g->d_slot_off, n, stream);
            if (e == cudaSuccess) e = dev_alloc((void **)&tmp, tmp_bytes, stream);
            if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, d_deg, g->d_slot_off, n, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            dev_free(tmp, stream);
            if (e != cudaSuccess) {
                dev_free(d_deg, stream);
                return cuda_fail(e, "slot offsets");
            }
        }
        dev_free(d_deg, stream);
        g->scanned = true;
    }
    return MM_OK;
}

// Reverse proposal keys of one weighting (built once per graph).
mm_status build_revkey(mm_graph *g, int weighted, cudaStream_t stream)
{
    const int wi = weighted ? 1 : 0;
    if (g->d_revkey[wi]) return MM_OK;
    const int n = g->n;
    if (n == 0) return MM_OK;
    const long long S = g->sum_degree;

    unsigned long long *revkey = nullptr;
    cudaError_t e = dev_alloc((void **)&revkey, sizeof(unsigned long long) * (size_t)(S > 0 ? S : 1), stream);
    if (e != cudaSuccess) return cuda_fail(e, "reverse keys");
    if (S == 0) {
        g->d_revkey[wi] = revkey;
        return MM_OK;
    }
    // Sorted lists: binary-search build.
    {
        const long long chunks = (S + kRevChunk - 1) / kRevChunk;
        int *chunk_v = nullptr;
        e = dev_alloc((void **)&chunk_v, sizeof(int) * (size_t)(chunks + 2), stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(chunk_v + chunks + 1, 0, sizeof(int), stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(revkey, 0, sizeof(unsigned long long) * (size_t)S, stream);
        if (e == cudaSuccess) {
            k_chunk_owner<<<grid_for(chunks + 1, 256, 148 * 8), 256, 0, stream>>>(
                g->d_ranges, n, g->contiguous ? 1 : 0, g->d_slot_off, S, chunk_v);
            const int grid = grid_for(chunks, 1, 148 * 8);
            if (weighted)
                k_revkey_sorted<true><<<grid, kRevThreads, 0, stream>>>(g->d_ranges, g->d_nbrs, g->d_w,
                                                                        g->contiguous ? 1 : 0, g->d_slot_off, S,
                                                                        chunk_v, revkey, chunk_v + chunks + 1);
            else
                k_revkey_sorted<false><<<grid, kRevThreads, 0, stream>>>(g->d_ranges, g->d_nbrs, g->d_w,
                                                                         g->contiguous ? 1 : 0, g->d_slot_off, S,
                                                                         chunk_v, revkey, chunk_v + chunks + 1);
            e = cudaGetLastError();
        }
        int unsorted = 1;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&unsorted, chunk_v + chunks + 1, sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        dev_free(chunk_v, stream);
        if (e != cudaSuccess) {
            dev_free(revkey, stream);
            return cuda_fail(e, "reverse key build (sorted lists)");
        }
        if (!unsorted) {
            g->d_revkey[wi] = revkey;
            return MM_OK;
        }
    }

    // General lists: sort the (unordered pair, direction) items.
    const int bits = bits_for(n);
    unsigned long long *k0 = nullptr, *k1 = nullptr;
    int *v0 = nullptr, *v1 = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    e = dev_alloc((void **)&k0, sizeof(unsigned long long) * S, stream);
    if (e == cudaSuccess) e = dev_alloc((void **)&k1, sizeof(unsigned long long) * S, stream);
    if (e == cudaSuccess) e = dev_alloc((void **)&v0, sizeof(int) * S, stream);
    if (e == cudaSuccess) e = dev_alloc((void **)&v1, sizeof(int) * S, stream);
    if (e == cudaSuccess) {
        k_pair_items<<<grid_for(n * 32ll, 256, 148 * 16), 256, 0, stream>>>(
            g->d_ranges, g->d_nbrs, n, bits, g->contiguous ? 1 : 0, g->d_slot_off, k0, v0);
        e = cudaGetLastError();
    }
    cub::DoubleBuffer<unsigned long long> kb(k0, k1);
    cub::DoubleBuffer<int> vb(v0, v1);
    const int end_bit = 2 * bits + 1;
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kb, vb, (int)S, 0, end_bit, stream);
    if (e == cudaSuccess) e = dev_alloc((void **)&tmp, tmp_bytes, stream);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, kb, vb, (int)S, 0, end_bit, stream);
    if (e == cudaSuccess) {
        const int grid = grid_for(S, 256, 148 * 16);
        if (weighted)
            k_pair_groups<true><<<grid, 256, 0, stream>>>(kb.Current(), vb.Current(), S, bits, g->d_ranges, g->d_w,
                                                          g->contiguous ? 1 : 0, g->d_slot_off, revkey);
        else
            k_pair_groups<false><<<grid, 256, 0, stream>>>(kb.Current(), vb.Current(), S, bits, g->d_ranges, g->d_w,
                                                           g->contiguous ? 1 : 0, g->d_slot_off, revkey);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    dev_free(tmp, stream);
    dev_free(k0, stream);
    dev_free(k1, stream);
    dev_free(v0, stream);
    dev_free(v1, stream);
    if (e != cudaSuccess) {
        dev_free(revkey, stream);
        return cuda_fail(e, "reverse key build");
    }
    g->d_revkey[wi] = revkey;
    return MM_OK;
}

}  // namespace

// Preference windows of the weighted types, built once per graph in three
// steps so that the upload can build the windows of the lists that have
// arrived while later chunks are still in transfer: windows_begin sizes and
// allocates them (it needs only the ranges), windows_range builds those of
// vertices [va, vb) and queues lists longer than kWinChunk, windows_end builds
// the queued lists and publishes d_pwin.
mm_status windows_begin(mm_graph *g, cudaStream_t stream)
{
    const int n = g->n;
    long long *slots = nullptr, *off = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    MM_CUDA_TRY(dev_alloc((void **)&slots, sizeof(long long) * ((size_t)n + 1), stream), "window sizes");
    cudaError_t e = dev_alloc((void **)&off, sizeof(long long) * ((size_t)n + 1), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(slots + n, 0, sizeof(long long), stream);
    if (e == cudaSuccess) {
        k_win_sizes<<<grid_for(n, 256, 148 * 8), 256, 0, stream>>>(g->d_ranges, n, slots);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, slots, off, n + 1, stream);
    if (e == cudaSuccess) e = dev_alloc(&tmp, tmp_bytes, stream);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, slots, off, n + 1, stream);
    long long total = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, off + n, sizeof total, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    dev_free(tmp, stream);
    dev_free(slots, stream);
    if (e != cudaSuccess) {
        dev_free(off, stream);
        return cuda_fail(e, "window offsets");
    }
    if (total >= (1ll << 31)) {
        dev_free(off, stream);
        set_error("push: more than 2^31 - 1 preference-window slots are not supported");
        return MM_ERR_UNSUPPORTED;
    }
    int2 *win = nullptr;
    int *big = nullptr;  // [n + 1]: queued long lists, then their count
    e = dev_alloc((void **)&win, sizeof(int2) * (size_t)(total > 0 ? total : 1), stream);
    if (e == cudaSuccess) e = dev_alloc((void **)&big, sizeof(int) * ((size_t)n + 1), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(big + n, 0, sizeof(int), stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        dev_free(win, stream);
        dev_free(big, stream);
        dev_free(off, stream);
        return cuda_fail(e, "window buffers");
    }
    g->win_build = win;
    g->win_big = big;
    g->d_pwin_off = off;
    return MM_OK;
}

mm_status windows_range(mm_graph *g, int va, int vb, cudaStream_t stream)
{
    if (vb <= va) return MM_OK;
    k_win_build<<<grid_for((long long)(vb - va) * 32, 256, 148 * 16), 256, 0, stream>>>(
        g->d_ranges, g->d_nbrs, g->d_w, va, vb, g->d_pwin_off, g->win_build, g->win_big, g->win_big + g->n);
    MM_CUDA_TRY(cudaGetLastError(), "preference windows");
    return MM_OK;
}

mm_status windows_end(mm_graph *g, cudaStream_t stream)
{
    const int n = g->n;
    int *big = g->win_big;
    int2 *win = g->win_build;
    const long long *off = g->d_pwin_off;
    int nbig = 0;
    cudaError_t e = cudaMemcpyAsync(&nbig, big + n, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess && nbig > 0) {
        long long *coff = nullptr, *ccnt = nullptr;
        WinCand *cand = nullptr;
        void *tmp2 = nullptr;
        size_t tmp2_bytes = 0;
        long long nchunks = 0;
        e = dev_alloc((void **)&coff, sizeof(long long) * ((size_t)nbig + 1), stream);
        if (e == cudaSuccess) e = dev_alloc((void **)&ccnt, sizeof(long long) * ((size_t)nbig + 1), stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(ccnt + nbig, 0, sizeof(long long), stream);
        if (e == cudaSuccess) {
            k_win_chunk_counts<<<grid_for(nbig, 256, 148 * 4), 256, 0, stream>>>(g->d_ranges, big, nbig, ccnt);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tmp2_bytes, ccnt, coff, nbig + 1, stream);
        if (e == cudaSuccess) e = dev_alloc(&tmp2, tmp2_bytes, stream);
        if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp2, tmp2_bytes, ccnt, coff, nbig + 1, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&nchunks, coff + nbig, sizeof nchunks, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        dev_free(tmp2, stream);
        if (e == cudaSuccess) e = dev_alloc((void **)&cand, sizeof(WinCand) * 32 * (size_t)(nchunks > 0 ? nchunks : 1), stream);
        if (e == cudaSuccess) {
            k_win_chunks<<<grid_for(nchunks * 32, 256, 148 * 16), 256, 0, stream>>>(g->d_ranges, g->d_nbrs, g->d_w, big,
                                                                                  nbig, coff, cand);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) {
            k_win_chunk_merge<<<grid_for((long long)nbig * 32, 256, 148 * 16), 256, 0, stream>>>(
                g->d_ranges, big, nbig, coff, cand, off, win);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        dev_free(cand, stream);
        dev_free(ccnt, stream);
        dev_free(coff, stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    dev_free(big, stream);
    g->win_big = nullptr;
    if (e != cudaSuccess) {
        windows_discard(g);
        return cuda_fail(e, "preference windows");
    }
    g->d_pwin = win;
    g->pwin_weights = false;
    g->win_build = nullptr;
    return MM_OK;
}

namespace {

// Symmetric weighted path: a window entry's second word becomes the entry's
// weight, so a proposal needs no dependent load of it (the proposal key is the
// weight and the proposer's id).  An entry flagged as never chosen keeps a
// weight that fails the same test (<= -1 or NaN).
__global__ void k_win_weights(const int2 *ranges, const float *w, const long long *pwin_off, int2 *pwin, int n)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int wl = win_len(degree_of(ranges[v]));
        const long long o = pwin_off[v];
        for (int e = 0; e < wl; ++e) {
            int2 x = pwin[o + e];
            x.y = __float_as_int(__ldg(w + (x.y & 0x7fffffff)));
            pwin[o + e] = x;
        }
    }
}

}  // namespace

void windows_discard(mm_graph *g)
{
    dev_free(g->win_build, 0);
    dev_free(g->win_big, 0);
    if (!g->d_pwin) {
        dev_free(g->d_pwin_off, 0);
        g->d_pwin_off = nullptr;
    }
    g->win_build = nullptr;
    g->win_big = nullptr;
}

namespace {

mm_status build_windows(mm_graph *g, cudaStream_t stream)
{
    mm_status st = windows_begin(g, stream);
    if (st == MM_OK) st = windows_range(g, 0, g->n, stream);
    if (st == MM_OK) st = windows_end(g, stream);
    return st;
}

}  // namespace

mm_status push_prepare(mm_graph *g, int weighted, cudaStream_t stream)
{
    // the symmetric path computes each proposal's key: no reverse index
    const bool sym = weighted ? g->sym_weights : g->sym_struct;
    mm_status st = scan_graph(g, stream);
    if (st == MM_OK && !sym) st = build_revkey(g, weighted, stream);
    if (st == MM_OK && weighted && g->n > 0 && !g->d_pwin) st = build_windows(g, stream);
    if (st == MM_OK && weighted && g->d_pwin && g->sym_weights && !g->pwin_weights) {
        k_win_weights<<<grid_for(g->n, 256, 148 * 16), 256, 0, stream>>>(g->d_ranges, g->d_w, g->d_pwin_off, g->d_pwin,
                                                                        g->n);
        MM_CUDA_TRY(cudaGetLastError(), "window weights");
        g->pwin_weights = true;
    }
    return st;
}

mm_status push_match(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds, int *d_match,
                     int *rounds_out, long long *stats, int stats_rounds, cudaStream_t stream)
{
    const bool maximal = is_maximal(type);
    if (g->n == 0) {
        // The reference still runs (and draws a seed for) its first round.
        *rounds_out = maximal ? 1 : max_rounds_of(type);
        if (nseeds < *rounds_out) {
            set_error("mm_match: fewer seeds than rounds");
            return MM_ERR_SEEDS;
        }
        return MM_OK;
    }
    PushState *s = nullptr;
    mm_status st = begin_call(g, type, barrier, seeds, nseeds, d_match, stream, &s);
    if (st != MM_OK) return st;
    st = run_rounds(g, s, type, stats != nullptr, false, stream);
    if (st != MM_OK) return st;
    return end_call(g, s, nseeds, rounds_out, stats, stats_rounds, nullptr, stream);
}

// The round kernel with the learned colouring: each vertex's blue probability
// comes from the policy (MM_POLICY_FLOATS weights, host) instead of the select
// barrier.  trace (device, trace_rounds * n * 8 floats, or null) receives the
// features, colour and outcome of every vertex coloured in those rounds.
mm_status push_match_policy(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                            const float *mlp_host, float level, int *d_match, int *rounds_out, float *trace,
                            int trace_rounds, cudaStream_t stream)
{
    if (g->n == 0) return push_match(g, type, barrier, seeds, nseeds, d_match, rounds_out, nullptr, 0, stream);
    PushState *s = nullptr;
    mm_status st = begin_call(g, type, barrier, seeds, nseeds, d_match, stream, &s);
    if (st != MM_OK) return st;
    if (!s->wfeat) {
        cudaError_t e = dev_alloc((void **)&s->wfeat, sizeof(float2) * (size_t)g->n, stream);
        if (e == cudaSuccess) {
            k_wfeat<<<grid_for((long long)g->n * 32, 256, 148 * 16), 256, 0, stream>>>(g->d_ranges, g->d_w, g->n,
                                                                                    s->wfeat);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) return cuda_fail(e, "policy state");
    }
    PolicyArgs pol;
    pol.mlp = mlp_host;
    // the output layer's weights W2 (after W1 and b1): all zero means every
    // vertex gets sigmoid(b2), the same clamp and scaling as on the device
    {
        constexpr int kW2 = kHid * kFeat + kHid;
        bool zero = true;
        for (int j = 0; j < kHid; ++j) zero = zero && mlp_host[kW2 + j] == 0.0f;
        if (zero) {
            float prob = 1.0f / (1.0f + std::exp(-mlp_host[kW2 + kHid]));
            prob = std::fmin(std::fmax(prob, 1.0f / 16.0f), 15.0f / 16.0f);
            pol.constant = true;
            pol.constant_bar = (uint32_t)((double)prob * 4294967296.0);
        }
    }
    pol.level = level;
    pol.trace = trace;
    pol.trace_rounds = trace ? trace_rounds : 0;
    st = is_weighted(type) ? launch_rounds<true, false, true>(g, s, false, stream, &pol)
                           : launch_rounds<false, false, true>(g, s, false, stream, &pol);
    if (st != MM_OK) return st;
    return end_call(g, s, nseeds, rounds_out, nullptr, 0, nullptr, stream);
}

// Same launch as push_match with barrier timestamps on: block 0 reads the
// global timer as each grid barrier completes, giving every round's window
// scan (A1), fallback scan (A2) and commit (B) durations.
mm_status push_profile(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds, int *d_match,
                       int *rounds_out, float *ms_phases, int cap_rounds, int *launched, cudaStream_t stream)
{
    if (g->n == 0) return push_match(g, type, barrier, seeds, nseeds, d_match, rounds_out, nullptr, 0, stream);
    PushState *s = nullptr;
    mm_status st = begin_call(g, type, barrier, seeds, nseeds, d_match, stream, &s);
    if (st != MM_OK) return st;
    MM_CUDA_TRY(cudaMemsetAsync(s->tstamp, 0, sizeof(unsigned long long) * kStampCount, stream), "timestamps clear");
    st = run_rounds(g, s, type, false, true, stream);
    if (st != MM_OK) return st;
    unsigned long long stamps[kStampCount];
    st = end_call(g, s, nseeds, rounds_out, nullptr, 0, stamps, stream);
    if (st != MM_OK) return st;
    if (ms_phases) {
        const int r_exec = *rounds_out;
        for (int r = 0; r < cap_rounds; ++r) {
            float a = 0.f, b = 0.f, c = 0.f;
            if (r < r_exec && stamps[3 * r] && stamps[3 * r + 1] && stamps[3 * r + 2] && stamps[3 * r + 3]) {
                a = (float)((double)(stamps[3 * r + 1] - stamps[3 * r]) * 1e-6);
                b = (float)((double)(stamps[3 * r + 2] - stamps[3 * r + 1]) * 1e-6);
                c = (float)((double)(stamps[3 * r + 3] - stamps[3 * r + 2]) * 1e-6);
            }
            ms_phases[(size_t)r * MM_PROFILE_KERNELS + 0] = a;
            ms_phases[(size_t)r * MM_PROFILE_KERNELS + 1] = b;
            ms_phases[(size_t)r * MM_PROFILE_KERNELS + 2] = c;
            ms_phases[(size_t)r * MM_PROFILE_KERNELS + 3] = a + b + c;
        }
    }
    if (launched) *launched = (is_weighted(type) ? g->sym_weights : g->sym_struct) ? 3 : 1;
    return MM_OK;
}

// Per-graph round counts of the last matching of a batch (after push_match).
mm_status push_batch_rounds(mm_graph *g, int type, int *rounds_host, cudaStream_t stream)
{
    int *d = nullptr;
    MM_CUDA_TRY(dev_alloc((void **)&d, sizeof(int) * (size_t)g->ngraphs, stream), "batch rounds");
    k_batch_rounds<<<grid_for((long long)g->ngraphs * 32, 256, 148 * 8), 256, 0, stream>>>(
        g->d_last, g->d_goff, g->ngraphs, max_rounds_of(type), is_maximal(type) ? 0 : 1, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(rounds_host, d, sizeof(int) * (size_t)g->ngraphs, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    dev_free(d, stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch rounds");
    return MM_OK;
}

void push_release(mm_graph *g)
{
    PushState *s = (PushState *)g->push_exec;
    if (s) {
        free_state(s);
        g->push_exec = nullptr;
    }
    for (int i = 0; i < 2; ++i) {
        dev_free(g->d_revkey[i], 0);
        g->d_revkey[i] = nullptr;
    }
    dev_free(g->d_slot_off, 0);
    g->d_slot_off = nullptr;
    windows_discard(g);
    dev_free(g->d_pwin, 0);
    g->d_pwin = nullptr;
    g->pwin_weights = false;
    dev_free(g->d_pwin_off, 0);
    g->d_pwin_off = nullptr;
}

}  // namespace mm
