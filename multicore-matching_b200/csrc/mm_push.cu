// mm_push.cu -- the B200 round loop ("push" path).
//
// Same matching as the reference's GPU round (src/matchgpu.cu:184-451), with
// the work re-cut so that each round streams only the adjacency lists of BLUE
// vertices and the loop never returns to the host.
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
//     proposer then atomicMax-es its revkey into slot_best[r]; the maximum over
//     proposers equals the maximum over r's list.  Red vertices never scan.
//   * Commit (gMatch, matchgpu.cu:260-283): red r is matched iff slot_best[r]
//     is non-zero (its partner is neighbours[~low32(key)]); blue u is matched
//     iff the low 32 bits of slot_best[its target] equal the low 32 bits of its
//     own revkey (positions in r's list are unique).
//   * Select (gaSelect, matchgpu.cu:220-258) of round t+1 is fused into the
//     commit pass of round t: a survivor recolours itself with seed t+1.
//   * Dead marking (requests == n+1) happens as soon as the blue scan finds no
//     unmatched neighbour; readers of that colour byte see "unmatched, not red"
//     either way, so their outcome is unchanged.
//
// Round t is two kernels: phase A (blue scan + proposal) and phase B
// (commit + recolour + worklist compaction).  They form the body of a CUDA
// graph WHILE node; the last block of phase B decides whether another round
// runs (cudaGraphSetConditional), so there is no host synchronisation inside
// the loop.  Worklists hold only vertices that can still be matched, split
// by colour and by degree class (long lists are scanned by a whole block).
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cstring>
#include <new>

#include "mm_common.cuh"

namespace mm {
namespace {

constexpr int kBlockA = 256;
constexpr int kBlockB = 256;
constexpr int kWarpsA = kBlockA / 32;
constexpr int kLargeDegree = 1024;  // lists longer than this are scanned by a whole block
constexpr unsigned kFull = 0xffffffffu;

// Worklists: [colour][degree class] -> index 0 blue-short, 1 blue-long,
// 2 red-short, 3 red-long.
constexpr int kLists = 4;

struct Ctl {
    int *match;            // output array of this call
    uint32_t barrier;
    int cap;               // 20 or 255
    int maximal;
    int nseeds;
    int t;                 // 0-based index of the round being executed
    int rounds;            // rounds the reference executes (set at loop exit)
    int status;            // 0 ok, 1 seeds exhausted
    int cont;              // 1 while another round follows (read by the stepped driver)
    unsigned ticket;       // phase-B block arrivals
    int cnt[2][kLists];    // worklist lengths by round parity
};

struct Params {
    int n;
    int contiguous;
    const int2 *ranges;
    const int *nbrs;
    const float *w;
    const unsigned long long *revkey;
    const long long *slot_off;
    uint8_t *col;
    int2 *req;
    unsigned long long *best;  // per red vertex: max proposal key this round
    int *lists;                // [2][kLists][n]
    const uint32_t *seeds;
    Ctl *ctl;
    unsigned long long *stats; // [kMaxRounds][MM_STATS_COLS] or null
    cudaGraphConditionalHandle loop;
};

__device__ __forceinline__ int *list_ptr(const Params &p, int parity, int which)
{
    return p.lists + ((size_t)parity * kLists + which) * (size_t)p.n;
}

__device__ __forceinline__ int degree_of(int2 r) { return r.y > r.x ? r.y - r.x : 0; }

// Append v to worklist `which` of `parity`, one atomic per warp and list.
__device__ __forceinline__ void append(const Params &p, int parity, int which, int v, bool take)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int l = 0; l < kLists; ++l) {
        const unsigned m = __ballot_sync(kFull, take && which == l);
        if (!m) continue;
        const int leader = __ffs(m) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&p.ctl->cnt[parity][l], __popc(m));
        base = __shfl_sync(kFull, base, leader);
        if (take && which == l) list_ptr(p, parity, l)[base + __popc(m & ((1u << lane) - 1))] = v;
    }
}

__device__ __forceinline__ void stat_add(const Params &p, int round, int col, unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&p.stats[(size_t)round * MM_STATS_COLS + col], v);
}

// Key under which a blue vertex ranks a red neighbour at position j
// (gwRequest: strict > from -1, earliest j on ties; grRequest: earliest j).
template <bool kW>
__device__ __forceinline__ unsigned long long cand_key(int j, float w)
{
    if (kW) return w > -1.0f ? (((unsigned long long)weight_order(w) << 32) | (uint32_t)~j) : 0ull;
    return (unsigned long long)(uint32_t)~j;
}

// Finish blue vertex v after its scan: dead, no proposal, or propose.
template <bool kStats>
__device__ __forceinline__ void propose(const Params &p, int v, int2 r, unsigned long long key, int alive,
                                        int t, bool weighted)
{
    if (!alive) {
        p.col[v] = kDead;
        p.ctl->match[v] = 2;
        p.req[v] = make_int2(-1, 0);
        return;
    }
    if (key == 0) {
        p.req[v] = make_int2(-2, 0);
        return;
    }
    const int j = (int)~(uint32_t)key;
    const int target = p.nbrs[j];
    const long long slot = p.contiguous ? (long long)j : p.slot_off[v] + (j - r.x);
    const unsigned long long rk = p.revkey[slot];
    if (rk) atomicMax(&p.best[target], rk);
    p.req[v] = make_int2(target, (int)(uint32_t)rk);
}

// Phase A for one long list: the whole block scans, then thread 0 proposes.
template <bool kW, bool kStats>
__device__ void scan_long(const Params &p, int v, int t)
{
    __shared__ unsigned long long s_key[kWarpsA];
    __shared__ int s_alive[kWarpsA];
    const int2 r = p.ranges[v];
    unsigned long long key = 0;
    int alive = 0;
    for (int base = r.x; base < r.y; base += kBlockA) {
        const int j = base + threadIdx.x;
        if (j < r.y) {
            const uint8_t c = p.col[p.nbrs[j]];
            alive |= c != kMatched;
            if (c == kRed) {
                const unsigned long long k = cand_key<kW>(j, kW ? p.w[j] : 0.0f);
                key = k > key ? k : key;
            }
        }
        // Random mode stops at the first red neighbour (grRequest returns there).
        if (!kW && __syncthreads_or(key != 0)) break;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long k2 = __shfl_down_sync(kFull, key, o);
        key = k2 > key ? k2 : key;
        alive |= __shfl_down_sync(kFull, alive, o);
    }
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        s_key[warp] = key;
        s_alive[warp] = alive;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < kWarpsA; ++i) {
            key = s_key[i] > key ? s_key[i] : key;
            alive |= s_alive[i];
        }
        if (kStats) {
            const int deg = degree_of(r);
            const long long seen = kW ? deg : (key ? (long long)((int)~(uint32_t)key - r.x + 1) : deg);
            atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_REQ_ENTRIES], (unsigned long long)seen);
            atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_BLUE_DEG], (unsigned long long)deg);
        }
        propose<kStats>(p, v, r, key, alive, t, kW);
    }
    __syncthreads();
}

// Phase A for 32 short lists: the warp walks their concatenated entries, 32 at
// a time, and reduces per vertex with a segmented shuffle.
template <bool kW, bool kStats>
__device__ void scan_short_batch(const Params &p, const int *list, int begin, int count, int t)
{
    const int lane = threadIdx.x & 31;
    const int idx = begin + lane;
    int v = -1;
    int2 r = make_int2(0, 0);
    int deg = 0;
    if (idx < count) {
        v = list[idx];
        r = p.ranges[v];
        deg = degree_of(r);
    }
    int incl = deg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    const int excl = incl - deg;
    const int total = __shfl_sync(kFull, incl, 31);
    unsigned long long acc = 0;
    int alive = 0;
    for (int e0 = 0; e0 < total; e0 += 32) {
        const int e = e0 + lane;
        const bool valid = e < total;
        // owner = first lane whose inclusive prefix exceeds e
        int o = 0;
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1) {
            const int probe = __shfl_sync(kFull, incl, o + step - 1);
            if (probe <= e) o += step;
        }
        const int ox = __shfl_sync(kFull, r.x, o);
        const int oexcl = __shfl_sync(kFull, excl, o);
        unsigned long long k = 0;
        int a = 0;
        if (valid) {
            const int j = ox + (e - oexcl);
            const uint8_t c = p.col[p.nbrs[j]];
            a = c != kMatched;
            if (c == kRed) k = cand_key<kW>(j, kW ? p.w[j] : 0.0f);
        }
        const int owner = valid ? o : 32 + lane;
        // segmented suffix max / or over runs of equal owner
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long k2 = __shfl_down_sync(kFull, k, d);
            const int a2 = __shfl_down_sync(kFull, a, d);
            const int o2 = __shfl_down_sync(kFull, owner, d);
            if (lane + d < 32 && o2 == owner) {
                k = k2 > k ? k2 : k;
                a |= a2;
            }
        }
        // each vertex lane pulls the value from the head of its run in this chunk
        const bool hit = deg > 0 && excl < e0 + 32 && incl > e0;
        const int head = excl > e0 ? excl - e0 : 0;
        const unsigned long long hk = __shfl_sync(kFull, k, head & 31);
        const int ha = __shfl_sync(kFull, a, head & 31);
        if (hit) {
            acc = hk > acc ? hk : acc;
            alive |= ha;
        }
    }
    if (v >= 0) {
        if (kStats) {
            const long long seen = kW ? deg : (acc ? (long long)((int)~(uint32_t)acc - r.x + 1) : deg);
            atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_REQ_ENTRIES], (unsigned long long)seen);
            atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_BLUE_DEG], (unsigned long long)deg);
        }
        propose<kStats>(p, v, r, acc, alive, t, kW);
    }
}

// Round set-up: colour every vertex with seeds[0], clear proposal slots, and
// fill the first worklists.
template <bool kStats>
__global__ void __launch_bounds__(kBlockB) k_init(Params p)
{
    const Ctl *ctl = p.ctl;
    const uint32_t seed = p.seeds[0], barrier = ctl->barrier;
    const int n = p.n;
    const int nloop = (n + blockDim.x - 1) / blockDim.x * blockDim.x;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nloop; v += gridDim.x * blockDim.x) {
        const bool in = v < n;
        int which = 0;
        unsigned long long blue = 0;
        if (in) {
            const uint8_t c = colour_of((uint32_t)v, seed, barrier);
            p.col[v] = c;
            p.best[v] = 0ull;
            const bool longl = degree_of(p.ranges[v]) > kLargeDegree;
            which = (c == kRed ? 2 : 0) + (longl ? 1 : 0);
            blue = c == kBlue;
        }
        append(p, 0, which, v, in);
        if (kStats) {
            stat_add(p, 0, MM_ST_ACTIVE, in ? 1ull : 0ull);
            stat_add(p, 0, MM_ST_BLUE, blue);
            stat_add(p, 0, MM_ST_RED, in && !blue ? 1ull : 0ull);
        }
    }
}

// Phase A: every blue vertex scans its list and proposes.
template <bool kW, bool kStats>
__global__ void __launch_bounds__(kBlockA) k_phase_a(Params p)
{
    Ctl *ctl = p.ctl;
    const int t = ctl->t;
    const int par = t & 1;
    const int n_short = ctl->cnt[par][0];
    const int n_long = ctl->cnt[par][1];
    if (blockIdx.x == 0 && threadIdx.x < kLists) ctl->cnt[par ^ 1][threadIdx.x] = 0;
    const int per_block = kBlockA;  // short lists per block unit (32 per warp)
    const long long units = (long long)n_long + (n_short + per_block - 1) / per_block;
    const int *longs = list_ptr(p, par, 1);
    const int *shorts = list_ptr(p, par, 0);
    const int warp = threadIdx.x >> 5;
    for (long long u = blockIdx.x; u < units; u += gridDim.x) {
        if (u < n_long) {
            scan_long<kW, kStats>(p, longs[u], t);
        } else {
            const int b = (int)(u - n_long) * per_block + warp * 32;
            if (b < n_short) scan_short_batch<kW, kStats>(p, shorts, b, n_short, t);
        }
    }
}

// Phase B: commit proposals, recolour survivors with the next seed, compact
// the worklists; the last block closes the round.
template <bool kW, bool kStats>
__global__ void __launch_bounds__(kBlockB) k_phase_b(Params p)
{
    Ctl *ctl = p.ctl;
    const int t = ctl->t;
    const int par = t & 1;
    const int cap = ctl->cap;
    bool has_next = t + 1 < cap;
    bool seeds_short = has_next && t + 1 >= ctl->nseeds;
    if (seeds_short) has_next = false;
    const uint32_t next_seed = has_next ? p.seeds[t + 1] : 0u;
    const uint32_t barrier = ctl->barrier;
    int cnt[kLists];
    long long total = 0;
#pragma unroll
    for (int l = 0; l < kLists; ++l) {
        cnt[l] = ctl->cnt[par][l];
        total += cnt[l];
    }
    int *match = ctl->match;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long loop_end = (total + blockDim.x - 1) / blockDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < loop_end; i += stride) {
        bool in = i < total;
        int which = 0;
        long long k = i;
        if (in) {
            while (which < kLists - 1 && k >= cnt[which]) {
                k -= cnt[which];
                ++which;
            }
        }
        int v = in ? list_ptr(p, par, which)[k] : 0;
        bool survive = false;
        unsigned long long matched = 0, seen = 0, rdeg = 0;
        if (in) {
            if (which < 2) {  // blue
                const int2 q = p.req[v];
                if (q.x != -1) {
                    bool won = false;
                    if (q.y != 0) won = (uint32_t)p.best[q.x] == (uint32_t)q.y;
                    if (won) {
                        match[v] = 4 + min(v, q.x);
                        p.col[v] = kMatched;
                        matched = 1;
                    } else {
                        survive = true;
                    }
                }
            } else {  // red
                const unsigned long long key = p.best[v];
                if (kStats) {
                    const int2 r = p.ranges[v];
                    const int deg = degree_of(r);
                    rdeg = deg;
                    seen = kW ? deg : (key ? (long long)((int)~(uint32_t)key - r.x + 1) : deg);
                }
                if (key) {
                    const int u = p.nbrs[(int)~(uint32_t)key];
                    match[v] = 4 + min(v, u);
                    p.col[v] = kMatched;
                    matched = 1;
                } else {
                    survive = true;
                }
            }
        }
        int next_which = which;
        unsigned long long nb = 0;
        if (survive && has_next) {
            const uint8_t c = colour_of((uint32_t)v, next_seed, barrier);
            p.col[v] = c;
            next_which = (c == kRed ? 2 : 0) + (which & 1);
            nb = c == kBlue;
        }
        append(p, par ^ 1, next_which, v, survive);
        if (kStats) {
            stat_add(p, t, MM_ST_MATCHED, matched);
            stat_add(p, t, MM_ST_RESP_ENTRIES, seen);
            stat_add(p, t, MM_ST_RED_DEG, rdeg);
            if (has_next) {
                stat_add(p, t + 1, MM_ST_ACTIVE, survive ? 1ull : 0ull);
                stat_add(p, t + 1, MM_ST_BLUE, nb);
                stat_add(p, t + 1, MM_ST_RED, survive && !nb ? 1ull : 0ull);
            }
        }
    }
    // Round bookkeeping by the last block to arrive.
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned ticket = atomicAdd(&ctl->ticket, 1u);
        if (ticket == gridDim.x - 1) {
            __threadfence();
            long long next = 0;
#pragma unroll
            for (int l = 0; l < kLists; ++l) next += atomicAdd(&ctl->cnt[par ^ 1][l], 0);
            const bool cont = has_next && next > 0;
            if (!cont) {
                if (seeds_short) ctl->status = 1;
                ctl->rounds = (ctl->maximal && next == 0) ? min(t + 2, cap) : cap;
            }
            ctl->t = t + 1;
            ctl->ticket = 0u;
            ctl->cont = cont ? 1 : 0;
            // Outside a graph (the stepped profiling driver) the host reads ctl->cont instead.
            if (p.loop) cudaGraphSetConditional(p.loop, cont ? 1u : 0u);
        }
    }
}

// After the loop: vertices still able to match keep their last colour as
// their match value (the reference leaves match[v] = 0 / 1 for them).
__global__ void __launch_bounds__(kBlockB) k_finish(Params p)
{
    const Ctl *ctl = p.ctl;
    const int par = ctl->t & 1;
    long long total = 0;
    int cnt[kLists];
#pragma unroll
    for (int l = 0; l < kLists; ++l) {
        cnt[l] = ctl->cnt[par][l];
        total += cnt[l];
    }
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int which = 0;
        long long k = i;
        while (which < kLists - 1 && k >= cnt[which]) {
            k -= cnt[which];
            ++which;
        }
        const int v = list_ptr(p, par, which)[k];
        ctl->match[v] = p.col[v];
    }
}

// ---------------------------------------------------------------------------
// Preparation: reverse proposal keys.

struct PrepInfo {
    unsigned long long sum_deg;
    unsigned long long max_deg;
    int noncontig;
    int bad;
};

__global__ void k_scan_ranges(const int2 *ranges, int n, long long nnz, PrepInfo *info, long long *deg_out)
{
    unsigned long long sum = 0, mx = 0;
    int nc = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int2 r = ranges[v];
        const int d = degree_of(r);
        sum += d;
        mx = d > (long long)mx ? d : mx;
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
        nc |= __shfl_down_sync(kFull, nc, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (sum) atomicAdd(&info->sum_deg, sum);
        if (mx) atomicMax(&info->max_deg, mx);
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

// Key red `owner` gives the entry at `slot` (its own list).
template <bool kW>
__device__ __forceinline__ unsigned long long red_key(const int2 *ranges, const float *w, int contiguous,
                                                      const long long *slot_off, long long owner, long long slot)
{
    const long long pos = contiguous ? slot : (long long)ranges[owner].x + (slot - slot_off[owner]);
    return cand_key<kW>((int)pos, kW ? w[pos] : 0.0f);
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

// Captured round loop of one (graph, type, stats) combination.
struct Plan {
    int type = 0;
    bool stats = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

struct PushState {
    // scratch owned by the push path
    uint8_t *col = nullptr;
    int2 *req = nullptr;
    unsigned long long *best = nullptr;
    int *lists = nullptr;
    uint32_t *seeds = nullptr;
    Ctl *ctl = nullptr;
    unsigned long long *stats = nullptr;
    Plan plans[8];
    int nplans = 0;
    int blocks_a = 0, blocks_b = 0;
};

int bits_for(long long n)
{
    int b = 1;
    while ((1ll << b) < n) ++b;
    return b;
}

mm_status alloc_state(mm_graph *g, PushState **out)
{
    PushState *s = new (std::nothrow) PushState();
    if (!s) {
        set_error("push: host allocation failed");
        return MM_ERR_NOMEM;
    }
    const size_t n = (size_t)(g->n > 0 ? g->n : 1);
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc(&s->col, n);
    if (e == cudaSuccess) e = cudaMalloc(&s->req, n * sizeof(int2));
    if (e == cudaSuccess) e = cudaMalloc(&s->best, n * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&s->lists, n * 2 * kLists * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&s->seeds, 256 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&s->ctl, sizeof(Ctl));
    if (e == cudaSuccess) e = cudaMalloc(&s->stats, sizeof(unsigned long long) * kMaxRounds * MM_STATS_COLS);
    if (e != cudaSuccess) {
        cudaFree(s->col); cudaFree(s->req); cudaFree(s->best); cudaFree(s->lists);
        cudaFree(s->seeds); cudaFree(s->ctl); cudaFree(s->stats);
        delete s;
        cudaGetLastError();
        set_error(std::string("push: device allocation failed: ") + cudaGetErrorString(e));
        return MM_ERR_NOMEM;
    }
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int occ_a = 0, occ_b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a, k_phase_a<true, false>, kBlockA, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, k_phase_b<true, false>, kBlockB, 0);
    s->blocks_a = sms * (occ_a > 0 ? occ_a : 4);
    s->blocks_b = sms * (occ_b > 0 ? occ_b : 4);
    *out = s;
    return MM_OK;
}

Params make_params(mm_graph *g, PushState *s, bool weighted, bool stats, cudaGraphConditionalHandle h)
{
    Params p;
    p.n = g->n;
    p.contiguous = g->contiguous ? 1 : 0;
    p.ranges = g->d_ranges;
    p.nbrs = g->d_nbrs;
    p.w = g->d_w;
    p.revkey = g->d_revkey[weighted ? 1 : 0];
    p.slot_off = g->d_slot_off;
    p.col = s->col;
    p.req = s->req;
    p.best = s->best;
    p.lists = s->lists;
    p.seeds = s->seeds;
    p.ctl = s->ctl;
    p.stats = stats ? s->stats : nullptr;
    p.loop = h;
    return p;
}

template <bool kW, bool kStats>
mm_status build_plan(mm_graph *g, PushState *s, Plan *plan)
{
    cudaGraph_t graph = nullptr;
    MM_CUDA_TRY(cudaGraphCreate(&graph, 0), "graph create");
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_fail(e, "conditional handle");
    }
    Params prm = make_params(g, s, kW, kStats, h);
    void *args[] = {&prm};
    const int blocks_init = grid_for(g->n, kBlockB, s->blocks_b);

    cudaKernelNodeParams kp = {};
    kp.func = (void *)k_init<kStats>;
    kp.gridDim = dim3(blocks_init);
    kp.blockDim = dim3(kBlockB);
    kp.kernelParams = args;
    cudaGraphNode_t n_init, n_loop, n_fin, n_a, n_b;
    e = cudaGraphAddKernelNode(&n_init, graph, nullptr, 0, &kp);

    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    if (e == cudaSuccess) e = cudaGraphAddNode(&n_loop, graph, &n_init, 1, &cp);
    if (e == cudaSuccess) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        cudaKernelNodeParams ka = {};
        ka.func = (void *)k_phase_a<kW, kStats>;
        ka.gridDim = dim3(s->blocks_a);
        ka.blockDim = dim3(kBlockA);
        ka.kernelParams = args;
        e = cudaGraphAddKernelNode(&n_a, body, nullptr, 0, &ka);
        if (e == cudaSuccess) {
            cudaKernelNodeParams kb = {};
            kb.func = (void *)k_phase_b<kW, kStats>;
            kb.gridDim = dim3(s->blocks_b);
            kb.blockDim = dim3(kBlockB);
            kb.kernelParams = args;
            e = cudaGraphAddKernelNode(&n_b, body, &n_a, 1, &kb);
        }
    }
    if (e == cudaSuccess) {
        cudaKernelNodeParams kf = {};
        kf.func = (void *)k_finish;
        kf.gridDim = dim3(grid_for(g->n, kBlockB, s->blocks_b));
        kf.blockDim = dim3(kBlockB);
        kf.kernelParams = args;
        e = cudaGraphAddKernelNode(&n_fin, graph, &n_loop, 1, &kf);
    }
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_fail(e, "round-loop graph");
    }
    plan->graph = graph;
    plan->exec = exec;
    return MM_OK;
}

}  // namespace

mm_status push_prepare(mm_graph *g, int weighted, cudaStream_t stream)
{
    const int wi = weighted ? 1 : 0;
    if (g->d_revkey[wi]) return MM_OK;
    const int n = g->n;
    if (n == 0) return MM_OK;

    // Degrees, contiguity, slot offsets.
    PrepInfo *d_info = nullptr;
    long long *d_deg = nullptr;
    MM_CUDA_TRY(cudaMalloc(&d_info, sizeof(PrepInfo)), "prep info");
    MM_CUDA_TRY(cudaMemsetAsync(d_info, 0, sizeof(PrepInfo), stream), "prep info clear");
    cudaError_t e = cudaMalloc(&d_deg, sizeof(long long) * (size_t)n);
    if (e != cudaSuccess) {
        cudaFree(d_info);
        return cuda_fail(e, "prep degrees");
    }
    k_scan_ranges<<<grid_for(n, 256, 148 * 8), 256, 0, stream>>>(g->d_ranges, n, g->nnz, d_info, d_deg);
    PrepInfo info;
    e = cudaMemcpyAsync(&info, d_info, sizeof info, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d_info);
    if (e != cudaSuccess) {
        cudaFree(d_deg);
        return cuda_fail(e, "prep scan");
    }
    const long long S = (long long)info.sum_deg;
    g->sum_degree = S;
    g->max_degree = (long long)info.max_deg;
    g->contiguous = info.noncontig == 0;
    if (S >= (1ll << 31) - 1) {
        cudaFree(d_deg);
        set_error("push: more than 2^31 - 2 adjacency slots are not supported");
        return MM_ERR_UNSUPPORTED;
    }
    if (!g->contiguous && !g->d_slot_off) {
        e = cudaMalloc(&g->d_slot_off, sizeof(long long) * (size_t)n);
        void *tmp = nullptr;
        size_t tmp_bytes = 0;
        if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_deg, g->d_slot_off, n, stream);
        if (e == cudaSuccess) e = cudaMalloc(&tmp, tmp_bytes);
        if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, d_deg, g->d_slot_off, n, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        cudaFree(tmp);
        if (e != cudaSuccess) {
            cudaFree(d_deg);
            return cuda_fail(e, "slot offsets");
        }
    }
    cudaFree(d_deg);

    unsigned long long *revkey = nullptr;
    e = cudaMalloc(&revkey, sizeof(unsigned long long) * (size_t)(S > 0 ? S : 1));
    if (e != cudaSuccess) return cuda_fail(e, "reverse keys");
    if (S == 0) {
        g->d_revkey[wi] = revkey;
        return MM_OK;
    }
    const int bits = bits_for(n);
    unsigned long long *k0 = nullptr, *k1 = nullptr;
    int *v0 = nullptr, *v1 = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    e = cudaMalloc(&k0, sizeof(unsigned long long) * S);
    if (e == cudaSuccess) e = cudaMalloc(&k1, sizeof(unsigned long long) * S);
    if (e == cudaSuccess) e = cudaMalloc(&v0, sizeof(int) * S);
    if (e == cudaSuccess) e = cudaMalloc(&v1, sizeof(int) * S);
    if (e == cudaSuccess) {
        k_pair_items<<<grid_for(n * 32ll, 256, 148 * 16), 256, 0, stream>>>(
            g->d_ranges, g->d_nbrs, n, bits, g->contiguous ? 1 : 0, g->d_slot_off, k0, v0);
        e = cudaGetLastError();
    }
    cub::DoubleBuffer<unsigned long long> kb(k0, k1);
    cub::DoubleBuffer<int> vb(v0, v1);
    const int end_bit = 2 * bits + 1;
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kb, vb, (int)S, 0, end_bit, stream);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tmp_bytes);
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
    cudaFree(tmp);
    cudaFree(k0);
    cudaFree(k1);
    cudaFree(v0);
    cudaFree(v1);
    if (e != cudaSuccess) {
        cudaFree(revkey);
        return cuda_fail(e, "reverse key build");
    }
    g->d_revkey[wi] = revkey;
    return MM_OK;
}

mm_status push_match(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds, int *d_match,
                     int *rounds_out, long long *stats, int stats_rounds, cudaStream_t stream)
{
    const bool weighted = is_weighted(type), maximal = is_maximal(type);
    const int cap = max_rounds_of(type);
    if (g->n == 0) {
        // The reference still runs (and draws a seed for) its first round.
        *rounds_out = maximal ? 1 : cap;
        if (nseeds < *rounds_out) {
            set_error("mm_match: fewer seeds than rounds");
            return MM_ERR_SEEDS;
        }
        return MM_OK;
    }
    mm_status st = push_prepare(g, weighted, stream);
    if (st != MM_OK) return st;
    PushState *s = (PushState *)g->push_exec;
    if (!s) {
        st = alloc_state(g, &s);
        if (st != MM_OK) return st;
        g->push_exec = s;
    }
    const bool want_stats = stats != nullptr;
    Plan *plan = nullptr;
    for (int i = 0; i < s->nplans; ++i)
        if (s->plans[i].type == type && s->plans[i].stats == want_stats) plan = &s->plans[i];
    if (!plan) {
        if (s->nplans == 8) {
            set_error("push: plan cache full");
            return MM_ERR_UNSUPPORTED;
        }
        plan = &s->plans[s->nplans];
        if (weighted) st = want_stats ? build_plan<true, true>(g, s, plan) : build_plan<true, false>(g, s, plan);
        else st = want_stats ? build_plan<false, true>(g, s, plan) : build_plan<false, false>(g, s, plan);
        if (st != MM_OK) return st;
        plan->type = type;
        plan->stats = want_stats;
        ++s->nplans;
    }
    if (nseeds < 1) {
        set_error("mm_match: no seeds");
        return MM_ERR_SEEDS;
    }
    Ctl ctl;
    std::memset(&ctl, 0, sizeof ctl);
    ctl.match = d_match;
    ctl.barrier = barrier;
    ctl.cap = cap;
    ctl.maximal = maximal ? 1 : 0;
    ctl.nseeds = nseeds < 256 ? nseeds : 256;
    const int nup = ctl.nseeds;
    MM_CUDA_TRY(cudaMemcpyAsync(s->seeds, seeds, sizeof(uint32_t) * nup, cudaMemcpyHostToDevice, stream), "seeds");
    MM_CUDA_TRY(cudaMemcpyAsync(s->ctl, &ctl, sizeof ctl, cudaMemcpyHostToDevice, stream), "control block");
    if (want_stats)
        MM_CUDA_TRY(cudaMemsetAsync(s->stats, 0, sizeof(unsigned long long) * kMaxRounds * MM_STATS_COLS, stream),
                    "stats clear");
    MM_CUDA_TRY(cudaGraphLaunch(plan->exec, stream), "round loop launch");
    Ctl out;
    MM_CUDA_TRY(cudaMemcpyAsync(&out, s->ctl, sizeof out, cudaMemcpyDeviceToHost, stream), "control read");
    if (want_stats && stats_rounds > 0)
        MM_CUDA_TRY(cudaMemcpyAsync(stats, s->stats, sizeof(long long) * MM_STATS_COLS *
                                                         (size_t)(stats_rounds < kMaxRounds ? stats_rounds : kMaxRounds),
                                    cudaMemcpyDeviceToHost, stream),
                    "stats read");
    MM_CUDA_TRY(cudaStreamSynchronize(stream), "round loop");
    if (out.status == 1 || out.rounds > nseeds) {
        set_error("mm_match: fewer seeds than rounds");
        return MM_ERR_SEEDS;
    }
    *rounds_out = out.rounds;
    return MM_OK;
}

namespace {

template <bool kW>
mm_status stepped_rounds(mm_graph *g, PushState *s, int *rounds_done, float *ms_a, float *ms_b, int cap_rounds,
                         cudaStream_t stream)
{
    Params p = make_params(g, s, kW, false, 0);
    const int blocks_init = grid_for(g->n, kBlockB, s->blocks_b);
    cudaEvent_t ev[3];
    for (int i = 0; i < 3; ++i) MM_CUDA_TRY(cudaEventCreate(&ev[i]), "event create");
    mm_status st = MM_OK;
    k_init<false><<<blocks_init, kBlockB, 0, stream>>>(p);
    int r = 0;
    for (;; ++r) {
        cudaEventRecord(ev[0], stream);
        k_phase_a<kW, false><<<s->blocks_a, kBlockA, 0, stream>>>(p);
        cudaEventRecord(ev[1], stream);
        k_phase_b<kW, false><<<s->blocks_b, kBlockB, 0, stream>>>(p);
        cudaEventRecord(ev[2], stream);
        int cont = 0;
        cudaError_t e = cudaMemcpyAsync(&cont, &s->ctl->cont, sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) {
            st = cuda_fail(e, "stepped round");
            break;
        }
        float a = 0.f, b = 0.f;
        cudaEventElapsedTime(&a, ev[0], ev[1]);
        cudaEventElapsedTime(&b, ev[1], ev[2]);
        if (r < cap_rounds) {
            if (ms_a) ms_a[r] = a;
            if (ms_b) ms_b[r] = b;
        }
        if (!cont) {
            ++r;
            break;
        }
    }
    if (st == MM_OK) {
        k_finish<<<grid_for(g->n, kBlockB, s->blocks_b), kBlockB, 0, stream>>>(p);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(e, "finish");
    }
    for (int i = 0; i < 3; ++i) cudaEventDestroy(ev[i]);
    *rounds_done = r;
    return st;
}

}  // namespace

// Same kernels as push_match, launched one by one from the host with CUDA
// events around each phase, so the duration of every phase-A and phase-B
// launch can be read.  For measurement only (it synchronises every round).
mm_status push_profile(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds, int *d_match,
                       int *rounds_out, float *ms_a, float *ms_b, int cap_rounds, int *launched,
                       cudaStream_t stream)
{
    const bool weighted = is_weighted(type), maximal = is_maximal(type);
    if (g->n == 0 || nseeds < 1) return push_match(g, type, barrier, seeds, nseeds, d_match, rounds_out, nullptr, 0, stream);
    mm_status st = push_prepare(g, weighted, stream);
    if (st != MM_OK) return st;
    PushState *s = (PushState *)g->push_exec;
    if (!s) {
        st = alloc_state(g, &s);
        if (st != MM_OK) return st;
        g->push_exec = s;
    }
    Ctl ctl;
    std::memset(&ctl, 0, sizeof ctl);
    ctl.match = d_match;
    ctl.barrier = barrier;
    ctl.cap = max_rounds_of(type);
    ctl.maximal = maximal ? 1 : 0;
    ctl.nseeds = nseeds < 256 ? nseeds : 256;
    MM_CUDA_TRY(cudaMemcpyAsync(s->seeds, seeds, sizeof(uint32_t) * ctl.nseeds, cudaMemcpyHostToDevice, stream), "seeds");
    MM_CUDA_TRY(cudaMemcpyAsync(s->ctl, &ctl, sizeof ctl, cudaMemcpyHostToDevice, stream), "control block");
    int executed = 0;
    st = weighted ? stepped_rounds<true>(g, s, &executed, ms_a, ms_b, cap_rounds, stream)
                  : stepped_rounds<false>(g, s, &executed, ms_a, ms_b, cap_rounds, stream);
    if (st != MM_OK) return st;
    Ctl out;
    MM_CUDA_TRY(cudaMemcpyAsync(&out, s->ctl, sizeof out, cudaMemcpyDeviceToHost, stream), "control read");
    MM_CUDA_TRY(cudaStreamSynchronize(stream), "profile");
    if (out.status == 1 || out.rounds > nseeds) {
        set_error("mm_match: fewer seeds than rounds");
        return MM_ERR_SEEDS;
    }
    *rounds_out = out.rounds;
    if (launched) *launched = 2 + 2 * executed;
    return MM_OK;
}

void push_release(mm_graph *g)
{
    PushState *s = (PushState *)g->push_exec;
    if (s) {
        for (int i = 0; i < s->nplans; ++i) {
            if (s->plans[i].exec) cudaGraphExecDestroy(s->plans[i].exec);
            if (s->plans[i].graph) cudaGraphDestroy(s->plans[i].graph);
        }
        cudaFree(s->col);
        cudaFree(s->req);
        cudaFree(s->best);
        cudaFree(s->lists);
        cudaFree(s->seeds);
        cudaFree(s->ctl);
        cudaFree(s->stats);
        delete s;
        g->push_exec = nullptr;
    }
    for (int i = 0; i < 2; ++i) {
        cudaFree(g->d_revkey[i]);
        g->d_revkey[i] = nullptr;
    }
    cudaFree(g->d_slot_off);
    g->d_slot_off = nullptr;
}

}  // namespace mm
