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
// carries the vertex and its neighbour range, so the scans never read
// neighbourRanges again.
//   short lists (deg <= 32)   a warp takes 32 blue vertices and walks their
//                             concatenated entries row by row, 32 consecutive
//                             entries per load (k_phase_a_short)
//   long lists  (deg  > 32)   blue ones are appended with their offset in the
//                             round's concatenated long-list entry space; that
//                             space is cut into 512-entry segments and a warp
//                             walks one segment row by row (k_phase_a_long).
//                             A list cut by segment edges is combined by
//                             atomics and its last piece proposes.  Every warp
//                             claims equal amounts of work whatever the skew.
// Every load of neighbour ids and weights is a coalesced row of 32 consecutive
// entries; a list's best entry is kept as a 64-bit key (weight order << 32 |
// ~position) max-combined in shared memory, which orders ties by position
// exactly as the reference's strict ">" scan in list order does.
// The two scans run concurrently.
//
// Round t is three kernels: the two phase-A scans (blue scan + proposal) and
// phase B (commit + recolour + worklist compaction).  They form the body of a
// CUDA graph WHILE node; the last block of phase B decides whether another
// round runs (cudaGraphSetConditional), so there is no host synchronisation
// inside the loop.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cstddef>
#include <cstring>
#include <new>

#include "mm_common.cuh"

namespace mm {
namespace {

constexpr int kBlockA = 256;
constexpr int kBlockB = 256;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kSmallMax = 32;       // short lists: degree <= 32
constexpr int kSegEntries = 512;    // entries per long-list segment (at most 16 pieces of lists > 32)

// Worklists.  kStaged holds blue long lists with their entry offsets.
enum : int { kBlueS = 0, kRedS, kRedLong, kStaged, kLists };

struct Ctl {
    int *match;            // output array of this call
    uint32_t barrier;
    int cap;               // 20 or 255
    int maximal;
    int nseeds;
    int t;                 // 0-based index of the round being executed
    int rounds;            // rounds the reference executes (set at loop exit)
    int status;            // 0 ok, 1 seeds exhausted, 2 a bounded device wait gave up
    int cont;              // 1 while another round follows (read by the stepped driver)
    unsigned ticket;       // phase-B block arrivals
    int task_short[2];     // phase-A cursors by round parity: short-list batches
    int task_long[2];      //   and long-list segments
    int cnt[2][kLists];    // worklist lengths by round parity (kStaged unused)
    unsigned long long staged_pack[2];  // kStaged: (items << 32) | entries, by parity
    int retired[2];        // vertices of the round that were unmatchable as soon as coloured
    int tail;              // 1: the remaining rounds run in the single-block tail kernel
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
    unsigned long long *best;       // per red vertex: max proposal key this round
    unsigned long long *part_key;   // per cut long list: max over finished pieces
    int *part_cnt;                  // per cut long list: finished pieces
    int4 *lists[2][kLists];         // items {v, begin, end, offset} by parity and list id
    int *seg_first[2];              // per staged segment: item holding its first entry
    const uint32_t *seeds;
    Ctl *ctl;
    unsigned long long *stats;      // [kMaxRounds][MM_STATS_COLS] or null
    cudaGraphConditionalHandle loop;
};

__device__ __forceinline__ int degree_of(int2 r) { return r.y > r.x ? r.y - r.x : 0; }
__device__ __forceinline__ int degree_of(int4 it) { return it.z > it.y ? it.z - it.y : 0; }

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

__device__ __forceinline__ void stat_add(const Params &p, int round, int col, unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&p.stats[(size_t)round * MM_STATS_COLS + col], v);
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

// Finish blue vertex v after its scan: dead, no proposal, or propose.
__device__ __forceinline__ void propose(const Params &p, int v, int begin, unsigned long long key)
{
    if (key == 0) {  // no unmatched neighbour: unmatchable (requests == n + 1)
        p.col[v] = kDead;
        p.ctl->match[v] = 2;
        p.req[v] = make_int2(-1, 0);
        return;
    }
    if (key == 1) {  // unmatched neighbours but no red one to propose to
        p.req[v] = make_int2(-2, 0);
        return;
    }
    const int j = (int)~(uint32_t)key;
    const int target = p.nbrs[j];
    const long long slot = p.contiguous ? (long long)j : p.slot_off[v] + (j - begin);
    const unsigned long long rk = p.revkey[slot];
    if (rk) atomicMax(&p.best[target], rk);
    p.req[v] = make_int2(target, (int)(uint32_t)rk);
}

// Adjacency entries the reference's request loop inspects for this vertex
// (random mode stops at the first red neighbour).
template <bool kW>
__device__ __forceinline__ unsigned long long request_seen(int begin, int deg, unsigned long long key)
{
    if (kW || key < 2) return (unsigned long long)deg;
    return (unsigned long long)((int)~(uint32_t)key - begin + 1);
}

template <bool kW, bool kStats>
__device__ __forceinline__ void propose_counted(const Params &p, int4 it, unsigned long long key, int t)
{
    if (kStats) {
        atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_REQ_ENTRIES], request_seen<kW>(it.y, degree_of(it), key));
        atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_BLUE_DEG], (unsigned long long)degree_of(it));
    }
    propose(p, it.x, it.y, key);
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

constexpr int kShortStep = 8;  // entries a tail thread loads (and gathers) at once
constexpr int kRows = 4;       // rows of 32 entries a warp keeps in flight in the grid scans

// ---- worklist compaction for the set-up and commit passes ----
//
// A block handles tiles of kTileItems vertices, kPer per thread.  Each thread
// decides the next list of its vertices; the block counts them per list with
// warp scans, takes one atomic per list and tile (the staged list's item and
// entry counts in one 64-bit atomic), and writes its items.

constexpr int kBlockT = 512;
constexpr int kPer = 4;
constexpr int kTileItems = kBlockT * kPer;
constexpr int kWarpsT = kBlockT / 32;

// dest[k]: -1 (drop) or the list id kBlueS, kRedS, kRedLong, kStaged.
__device__ __forceinline__ void compact_tile(const Params &p, int parity, const int (&dest)[kPer],
                                             const int4 (&item)[kPer])
{
    __shared__ int s_warp[kWarpsT][5];  // per-warp counts, then per-warp offsets within the tile
    __shared__ int s_base[5];           // tile bases: 4 list indices, then the staged entry offset
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int c[4] = {0, 0, 0, 0}, ent = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
#pragma unroll
        for (int l = 0; l < 4; ++l) c[l] += dest[k] == l;
        if (dest[k] == kStaged) ent += degree_of(item[k]);
    }
    int ex[5];
#pragma unroll
    for (int l = 0; l < 5; ++l) {
        const int v = l < 4 ? c[l] : ent;
        const int incl = warp_incl_scan(v);
        ex[l] = incl - v;
        if (lane == 31) s_warp[warp][l] = incl;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        const int l = threadIdx.x;
        int run = 0;
        for (int w = 0; w < kWarpsT; ++w) {
            const int x = s_warp[w][l];
            s_warp[w][l] = run;
            run += x;
        }
        if (l < kStaged) {
            s_base[l] = run ? atomicAdd(&p.ctl->cnt[parity][l], run) : 0;
        } else {
            int run_e = 0;
            for (int w = 0; w < kWarpsT; ++w) {
                const int x = s_warp[w][4];
                s_warp[w][4] = run_e;
                run_e += x;
            }
            unsigned long long old = 0;
            if (run) old = atomicAdd(&p.ctl->staged_pack[parity], ((unsigned long long)run << 32) | (unsigned)run_e);
            s_base[3] = (int)(old >> 32);
            s_base[4] = (int)(old & 0xffffffffull);
        }
    }
    __syncthreads();
    int rc[4] = {0, 0, 0, 0}, re = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const int l = dest[k];
        if (l < 0) continue;
        int idx = 0;
#pragma unroll
        for (int m = 0; m < 4; ++m)
            if (l == m) idx = s_base[m] + s_warp[warp][m] + ex[m] + rc[m]++;
        if (l != kStaged) {
            p.lists[parity][l][idx] = item[k];
        } else {
            const int deg = degree_of(item[k]);
            const int off = s_base[4] + s_warp[warp][4] + ex[4] + re;
            re += deg;
            p.lists[parity][kStaged][idx] = make_int4(item[k].x, item[k].y, item[k].z, off);
            for (int s = (off + kSegEntries - 1) / kSegEntries; s * kSegEntries < off + deg; ++s)
                p.seg_first[parity][s] = idx;
        }
    }
    __syncthreads();  // s_warp / s_base are reused by the next tile
}

__device__ __forceinline__ int next_list(bool blue, int deg)
{
    if (deg > kSmallMax) return blue ? kStaged : kRedLong;
    return blue ? kBlueS : kRedS;
}

// Round set-up: colour every vertex with seeds[0], clear proposal slots, and
// fill the first worklists.
template <bool kStats>
__global__ void __launch_bounds__(kBlockT) k_init(Params p)
{
    const Ctl *ctl = p.ctl;
    const uint32_t seed = p.seeds[0], barrier = ctl->barrier;
    const int n = p.n;
    const int ntiles = (n + kTileItems - 1) / kTileItems;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int dest[kPer];
        int4 item[kPer];
        unsigned long long act = 0, blue_n = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const int v = tile * kTileItems + k * kBlockT + threadIdx.x;
            dest[k] = -1;
            item[k] = make_int4(v, 0, 0, 0);
            if (v < n) {
                const int2 r = p.ranges[v];
                item[k].y = r.x;
                item[k].z = r.y;
                const int deg = degree_of(r);
                const bool blue = colour_of((uint32_t)v, seed, barrier) == kBlue;
                p.best[v] = 0ull;
                if (deg > kSmallMax) {
                    p.part_key[v] = 0ull;
                    p.part_cnt[v] = 0;
                }
                ++act;
                blue_n += blue;
                if (blue && deg == 0) {  // no neighbours: unmatchable as soon as it is blue
                    p.col[v] = kDead;
                    p.ctl->match[v] = 2;
                } else {
                    p.col[v] = blue ? kBlue : kRed;
                    dest[k] = next_list(blue, deg);
                }
            }
        }
        if (kStats) {
            stat_add(p, 0, MM_ST_ACTIVE, act);
            stat_add(p, 0, MM_ST_BLUE, blue_n);
            stat_add(p, 0, MM_ST_RED, act - blue_n);
        }
        compact_tile(p, 0, dest, item);
    }
}

// Phase A, short lists: a warp claims 32 blue short-list vertices, lays their
// entries end to end (at most 1024) and walks them in rows of 32: lane l of
// row r takes entry 32r + l, so every load is one coalesced row.  The owner of
// each entry comes from a byte table the lanes fill for their own lists; keys
// are max-combined per list in shared memory.  Block 0 also resets the next
// round's list counters and cursors.
constexpr int kWarpsA = kBlockA / 32;

template <bool kW, bool kStats>
__global__ void __launch_bounds__(kBlockA) k_phase_a_short(Params p)
{
    __shared__ unsigned long long s_acc[kWarpsA][32];
    __shared__ int s_delta[kWarpsA][32];
    __shared__ uint8_t s_owner[kWarpsA][32 * kSmallMax];
    Ctl *ctl = p.ctl;
    const int t = ctl->t;
    const int par = t & 1;
    const int n_short = ctl->cnt[par][kBlueS];
    if (blockIdx.x == 0 && threadIdx.x < kLists) ctl->cnt[par ^ 1][threadIdx.x] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 32) {
        ctl->task_short[par ^ 1] = 0;
        ctl->task_long[par ^ 1] = 0;
        ctl->staged_pack[par ^ 1] = 0ull;
        ctl->retired[par ^ 1] = 0;
    }
    const int units = (n_short + 31) / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long *acc = s_acc[warp];
    int *delta = s_delta[warp];
    uint8_t *owner = s_owner[warp];
    const int4 *list = p.lists[par][kBlueS];
    for (;;) {
        int u = 0;
        if (lane == 0) u = atomicAdd(&ctl->task_short[par], 1);
        u = __shfl_sync(kFull, u, 0);
        if (u >= units) break;
        const int idx = u * 32 + lane;
        const bool valid = idx < n_short;
        const int4 it = valid ? list[idx] : make_int4(-1, 0, 0, 0);
        const int deg = valid ? degree_of(it) : 0;
        const int incl = warp_incl_scan(deg);
        const int start = incl - deg;
        const int total = __shfl_sync(kFull, incl, 31);
        delta[lane] = it.y - start;  // global position of concatenated entry e: e + delta[owner]
        acc[lane] = 0ull;
        for (int k = 0; k < deg; ++k) owner[start + k] = (uint8_t)lane;
        __syncwarp();
        for (int base = 0; base < total; base += 32 * kRows) {
            int own[kRows], pos[kRows], nb[kRows];
            float wv[kRows];
#pragma unroll
            for (int r = 0; r < kRows; ++r) {
                const int e = base + r * 32 + lane;
                const bool in = e < total;
                own[r] = in ? owner[e] : -1;
                pos[r] = in ? e + delta[own[r]] : 0;
                nb[r] = in ? __ldcs(p.nbrs + pos[r]) : 0;
                wv[r] = kW && in ? __ldcs(p.w + pos[r]) : 0.0f;
            }
            uint8_t c[kRows];
#pragma unroll
            for (int r = 0; r < kRows; ++r) c[r] = own[r] >= 0 ? p.col[nb[r]] : (uint8_t)kMatched;
#pragma unroll
            for (int r = 0; r < kRows; ++r) {
                const unsigned long long key = entry_key<kW>(c[r], pos[r], wv[r]);
                if (key) atomicMax(&acc[own[r]], key);
            }
        }
        __syncwarp();
        if (valid) propose_counted<kW, kStats>(p, it, acc[lane], t);
        __syncwarp();  // the tables are refilled by the next batch
    }
}

// ---- long lists: entry-balanced segments ----
//
// The blue long lists of a round are concatenated (each item's .w is its
// offset) and cut into kSegEntries-entry segments; seg_first[s] is the first
// item overlapping segment s.  A warp takes a segment: lane l describes the
// l-th list piece in it (at most 16), then the warp walks the segment in rows
// of 32 consecutive entries.  Each lane keeps a cursor on the piece its entry
// falls in (it moves forward only) and a running key for it, folded into the
// piece's shared slot when the cursor moves on.  A list inside one segment
// proposes at once; a cut list max-combines its piece into part_key and the
// piece that arrives last proposes.

constexpr int kWarpsL = 8;

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
        p.part_cnt[v] = 0;
        propose_counted<kW, kStats>(p, it, all, t);
    }
}

template <bool kW, bool kStats>
__global__ void __launch_bounds__(kWarpsL * 32) k_phase_a_long(Params p)
{
    __shared__ unsigned long long s_acc[kWarpsL][32];
    __shared__ int s_end[kWarpsL][33];    // segment-relative end of each piece; INT_MAX past the last
    __shared__ int s_delta[kWarpsL][32];  // global position of segment entry e: e + delta[piece]
    Ctl *ctl = p.ctl;
    const int t = ctl->t;
    const int par = t & 1;
    const unsigned long long pack = ctl->staged_pack[par];
    const int nitems = (int)(pack >> 32);
    const int nentries = (int)(pack & 0xffffffffull);
    const int nseg = (nentries + kSegEntries - 1) / kSegEntries;
    if (nseg == 0) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long *acc = s_acc[warp];
    int *pend = s_end[warp];
    int *delta = s_delta[warp];
    const int4 *list = p.lists[par][kStaged];
    for (;;) {
        int s = 0;
        if (lane == 0) s = atomicAdd(&ctl->task_long[par], 1);
        s = __shfl_sync(kFull, s, 0);
        if (s >= nseg) break;
        const int s_lo = s * kSegEntries;
        const int seg_len = min(kSegEntries, nentries - s_lo);
        const int idx = p.seg_first[par][s] + lane;
        int4 it = make_int4(-1, 0, 0, 0);
        int pieces = 1, lo = 0, hi = 0;
        if (idx < nitems) {
            const int4 x = list[idx];
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
        acc[lane] = 0ull;
        __syncwarp();
        int cur = 0;
        unsigned long long best = 0ull;
        int fold = 0;  // piece the running key belongs to
        for (int base = 0; base < seg_len; base += 32 * kRows) {
            int own[kRows], pos[kRows], nb[kRows];
            float wv[kRows];
#pragma unroll
            for (int r = 0; r < kRows; ++r) {
                const int e = base + r * 32 + lane;
                const bool in = e < seg_len;
                while (in && e >= pend[cur]) ++cur;
                own[r] = in ? cur : -1;
                pos[r] = e + delta[cur];
                nb[r] = in ? __ldcs(p.nbrs + pos[r]) : 0;
                wv[r] = kW && in ? __ldcs(p.w + pos[r]) : 0.0f;
            }
            uint8_t c[kRows];
#pragma unroll
            for (int r = 0; r < kRows; ++r) c[r] = own[r] >= 0 ? p.col[nb[r]] : (uint8_t)kMatched;
#pragma unroll
            for (int r = 0; r < kRows; ++r) {
                if (own[r] < 0) continue;
                if (own[r] != fold) {
                    if (best) atomicMax(&acc[fold], best);
                    best = 0ull;
                    fold = own[r];
                }
                const unsigned long long key = entry_key<kW>(c[r], pos[r], wv[r]);
                best = key > best ? key : best;
            }
        }
        if (best) atomicMax(&acc[fold], best);
        __syncwarp();
        if (it.x >= 0) {
            if (kStats) {
                atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_STAGED_DEG], (unsigned long long)(hi - lo));
                atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_STAGED_ITEMS], 1ull);
            }
            finish_piece<kW, kStats>(p, it, pieces, acc[lane], t);
        }
        __syncwarp();  // the tables are refilled by the next segment
    }
}

// Rounds small enough for one block run in the tail kernel.
constexpr int kTailThreads = 1024;
constexpr long long kTailItems = 4096;        // vertices that can still be matched
constexpr unsigned kTailEntries = 32768;      // entries of blue long lists

// Close round t (one thread): record the outcome and decide what runs next.
// Returns true if another round runs in the caller's loop.
__device__ __forceinline__ bool close_round(Ctl *ctl, int t, int cap, bool has_next, bool seeds_short, long long next,
                                            unsigned staged_entries, int retired, bool in_tail)
{
    const bool more = has_next && next > 0;
    if (!more) {
        if (seeds_short) ctl->status = 1;
        // Vertices retired while being coloured for round t+1 are still active
        // in that round for the reference, so it runs round t+1 and only finds
        // nothing left at round t+2.
        if (!ctl->maximal || next > 0) ctl->rounds = cap;
        else ctl->rounds = min(retired > 0 ? t + 3 : t + 2, cap);
    }
    ctl->t = t + 1;
    const bool to_tail = more && !in_tail && next <= kTailItems && staged_entries <= kTailEntries;
    if (to_tail) ctl->tail = 1;
    const bool loop = more && !to_tail;
    ctl->cont = loop ? 1 : 0;
    return loop;
}

// Phase B: commit proposals, recolour survivors with the next seed, compact
// the worklists; the last block closes the round.
template <bool kW, bool kStats>
__global__ void __launch_bounds__(kBlockT) k_phase_b(Params p)
{
    Ctl *ctl = p.ctl;
    const int t = ctl->t;
    const int par = t & 1;
    const int cap = ctl->cap;
    bool has_next = t + 1 < cap;
    const bool seeds_short = has_next && t + 1 >= ctl->nseeds;
    if (seeds_short) has_next = false;
    const uint32_t next_seed = has_next ? p.seeds[t + 1] : 0u;
    const uint32_t barrier = ctl->barrier;
    // lists in the order: blue short, blue long (staged), red short, red long
    const int c0 = ctl->cnt[par][kBlueS], c1 = (int)(ctl->staged_pack[par] >> 32), c2 = ctl->cnt[par][kRedS],
              c3 = ctl->cnt[par][kRedLong];
    const long long total = (long long)c0 + c1 + c2 + c3;
    const long long ntiles = (total + kTileItems - 1) / kTileItems;
    int *match = ctl->match;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int4 it[kPer];
        bool in[kPer], blue[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            long long i = tile * kTileItems + k * kBlockT + threadIdx.x;
            in[k] = i < total;
            blue[k] = true;
            it[k] = make_int4(0, 0, 0, 0);
            if (in[k]) {
                if (i < c0) {
                    it[k] = p.lists[par][kBlueS][i];
                } else if ((i -= c0) < c1) {
                    it[k] = p.lists[par][kStaged][i];
                } else if ((i -= c1) < c2) {
                    it[k] = p.lists[par][kRedS][i];
                    blue[k] = false;
                } else {
                    it[k] = p.lists[par][kRedLong][i - c2];
                    blue[k] = false;
                }
            }
        }
        // proposal state: blue -> its request, red -> the best proposal it received
        int2 q[kPer];
        unsigned long long key[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            q[k] = make_int2(-1, 0);
            key[k] = 0ull;
            if (in[k]) {
                if (blue[k]) q[k] = p.req[it[k].x];
                else key[k] = p.best[it[k].x];
            }
        }
#pragma unroll
        for (int k = 0; k < kPer; ++k)
            if (in[k] && blue[k] && q[k].y != 0) key[k] = p.best[q[k].x];
        int partner[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            partner[k] = -1;
            if (!in[k]) continue;
            if (blue[k]) {
                if (q[k].y != 0 && (uint32_t)key[k] == (uint32_t)q[k].y) partner[k] = q[k].x;
            } else if (key[k]) {
                partner[k] = p.nbrs[(int)~(uint32_t)key[k]];
            }
        }
        int dest[kPer];
        unsigned long long matched = 0, seen = 0, rdeg = 0, act = 0, nblue = 0;
        int retired = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            dest[k] = -1;
            if (!in[k]) continue;
            const int v = it[k].x;
            const int deg = degree_of(it[k]);
            if (kStats && !blue[k]) {
                rdeg += deg;
                seen += kW ? deg : (key[k] ? (unsigned long long)((int)~(uint32_t)key[k] - it[k].y + 1) : deg);
            }
            if (partner[k] >= 0) {
                match[v] = 4 + min(v, partner[k]);
                p.col[v] = kMatched;
                ++matched;
                continue;
            }
            if (blue[k] && q[k].x == -1) continue;  // unmatchable (marked in phase A)
            // survivor
            if (!has_next) {
                dest[k] = next_list(blue[k], deg);
                continue;
            }
            const bool nb = colour_of((uint32_t)v, next_seed, barrier) == kBlue;
            ++act;
            nblue += nb;
            if (nb && deg == 0) {  // no neighbours: unmatchable as soon as it is blue
                p.col[v] = kDead;
                match[v] = 2;
                ++retired;
            } else {
                p.col[v] = nb ? kBlue : kRed;
                dest[k] = next_list(nb, deg);
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
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) retired += __shfl_xor_sync(kFull, retired, o);
        if ((threadIdx.x & 31) == 0 && retired) atomicAdd(&ctl->retired[par ^ 1], retired);
        compact_tile(p, par ^ 1, dest, it);
    }
    // Round bookkeeping by the last block to arrive.
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned ticket = atomicAdd(&ctl->ticket, 1u);
        if (ticket == gridDim.x - 1) {
            __threadfence();
            long long next = (long long)(atomicAdd(&ctl->staged_pack[par ^ 1], 0ull) >> 32);
#pragma unroll
            for (int l = 0; l < kStaged; ++l) next += atomicAdd(&ctl->cnt[par ^ 1][l], 0);
            const int retired_all = atomicAdd(&ctl->retired[par ^ 1], 0);
            const unsigned staged_entries =
                (unsigned)(atomicAdd(&ctl->staged_pack[par ^ 1], 0ull) & 0xffffffffull);
            ctl->ticket = 0u;
            const bool cont = close_round(ctl, t, cap, has_next, seeds_short, next, staged_entries, retired_all, false);
            // Outside a graph (the stepped profiling driver) the host reads ctl->cont instead.
            if (p.loop) cudaGraphSetConditional(p.loop, cont ? 1u : 0u);
        }
    }
}

// ---- tail: the last, small rounds in one block ----
//
// Same round as the grid kernels (scan + propose, commit + recolour), with
// block barriers between the phases instead of kernel launches.  Values that
// other threads of the block changed by atomics (best, counters) are read
// from L2 (__ldcg), never from this SM's L1.

// One short list scanned by one thread, kShortStep loads and gathers at a time.
template <bool kW, bool kStats>
__device__ void tail_scan_thread(const Params &p, int4 it, int t)
{
    float bw = -1.0f;
    int bj = 0;
    bool alive = false;
    for (int b = it.y; b < it.z; b += kShortStep) {
        int nb[kShortStep];
        float wv[kShortStep];
#pragma unroll
        for (int k = 0; k < kShortStep; ++k) {
            const bool in = b + k < it.z;
            nb[k] = in ? p.nbrs[b + k] : 0;
            wv[k] = kW && in ? p.w[b + k] : 0.0f;
        }
        uint8_t c[kShortStep];
#pragma unroll
        for (int k = 0; k < kShortStep; ++k) c[k] = __ldcg(p.col + nb[k]);
#pragma unroll
        for (int k = 0; k < kShortStep; ++k) {
            if (b + k >= it.z) break;
            alive |= c[k] != kMatched;
            if (c[k] == kRed && wv[k] > bw) {
                bw = wv[k];
                bj = b + k;
            }
        }
        if (!kW && bw > -1.0f) break;  // grRequest returns at the first red neighbour
    }
    propose_counted<kW, kStats>(p, it, strip_key<kW>(bw, bj, alive), t);
}

// One long list scanned by one warp: 4 entries per lane per step, 32 apart.
template <bool kW, bool kStats>
__device__ void tail_scan_warp(const Params &p, int4 it, int t)
{
    const int lane = threadIdx.x & 31;
    float bw = -1.0f;
    int bj = 0;
    bool alive = false;
    for (int base = it.y; base < it.z; base += 128) {
        int nb[4];
        float wv[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int j = base + k * 32 + lane;
            nb[k] = j < it.z ? p.nbrs[j] : 0;
            wv[k] = kW && j < it.z ? p.w[j] : 0.0f;
        }
        uint8_t c[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) c[k] = __ldcg(p.col + nb[k]);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int j = base + k * 32 + lane;
            if (j >= it.z) break;
            alive |= c[k] != kMatched;
            if (c[k] == kRed && wv[k] > bw) {
                bw = wv[k];
                bj = j;
            }
        }
        if (!kW && __any_sync(kFull, bw > -1.0f)) break;
    }
    unsigned long long key = strip_key<kW>(bw, bj, alive);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long k2 = __shfl_xor_sync(kFull, key, o);
        key = k2 > key ? k2 : key;
    }
    if (lane == 0) propose_counted<kW, kStats>(p, it, key, t);
}

template <bool kW, bool kStats>
__global__ void __launch_bounds__(kTailThreads) k_tail(Params p)
{
    Ctl *ctl = p.ctl;
    if (!__ldcg(&ctl->tail)) return;
    __shared__ int s_t, s_more;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (;;) {
        if (tid == 0) {
            const int t = ctl->t;
            s_t = t;
            const int nx = (t & 1) ^ 1;
            for (int l = 0; l < kLists; ++l) ctl->cnt[nx][l] = 0;
            ctl->staged_pack[nx] = 0ull;
            ctl->retired[nx] = 0;
        }
        __syncthreads();
        const int t = s_t, par = t & 1, nx = par ^ 1;
        const int cap = ctl->cap;
        const int c_bs = __ldcg(&ctl->cnt[par][kBlueS]);
        const int c_st = (int)(__ldcg(&ctl->staged_pack[par]) >> 32);
        const int c_rs = __ldcg(&ctl->cnt[par][kRedS]);
        const int c_rl = __ldcg(&ctl->cnt[par][kRedLong]);
        // scan + propose
        for (int i = tid; i < c_bs; i += kTailThreads) tail_scan_thread<kW, kStats>(p, p.lists[par][kBlueS][i], t);
        for (int i = warp; i < c_st; i += kTailThreads / 32) tail_scan_warp<kW, kStats>(p, p.lists[par][kStaged][i], t);
        __syncthreads();
        // commit + recolour + compact
        bool has_next = t + 1 < cap;
        const bool seeds_short = has_next && t + 1 >= ctl->nseeds;
        if (seeds_short) has_next = false;
        const uint32_t next_seed = has_next ? p.seeds[t + 1] : 0u;
        const uint32_t barrier = ctl->barrier;
        int *match = ctl->match;
        const int total = c_bs + c_st + c_rs + c_rl;
        for (int i = tid; i < total; i += kTailThreads) {
            int4 it;
            bool blue = true;
            if (i < c_bs) it = p.lists[par][kBlueS][i];
            else if (i < c_bs + c_st) it = p.lists[par][kStaged][i - c_bs];
            else if (i < c_bs + c_st + c_rs) { it = p.lists[par][kRedS][i - c_bs - c_st]; blue = false; }
            else { it = p.lists[par][kRedLong][i - c_bs - c_st - c_rs]; blue = false; }
            const int v = it.x;
            const int deg = degree_of(it);
            int partner = -1;
            bool dead = false;
            if (blue) {
                const int2 q = __ldcg(&p.req[v]);
                dead = q.x == -1;
                if (q.y != 0 && (uint32_t)__ldcg(&p.best[q.x]) == (uint32_t)q.y) partner = q.x;
            } else {
                const unsigned long long key = __ldcg(&p.best[v]);
                if (key) partner = p.nbrs[(int)~(uint32_t)key];
                if (kStats) {
                    atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_RED_DEG], (unsigned long long)deg);
                    atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_RESP_ENTRIES],
                              kW ? (unsigned long long)deg
                                 : (key ? (unsigned long long)((int)~(uint32_t)key - it.y + 1) : (unsigned long long)deg));
                }
            }
            if (partner >= 0) {
                match[v] = 4 + min(v, partner);
                p.col[v] = kMatched;
                if (kStats) atomicAdd(&p.stats[(size_t)t * MM_STATS_COLS + MM_ST_MATCHED], 1ull);
                continue;
            }
            if (dead) continue;
            int dest;
            if (!has_next) {
                dest = next_list(blue, deg);
            } else {
                const bool nb = colour_of((uint32_t)v, next_seed, barrier) == kBlue;
                if (kStats) {
                    atomicAdd(&p.stats[(size_t)(t + 1) * MM_STATS_COLS + MM_ST_ACTIVE], 1ull);
                    atomicAdd(&p.stats[(size_t)(t + 1) * MM_STATS_COLS + (nb ? MM_ST_BLUE : MM_ST_RED)], 1ull);
                }
                if (nb && deg == 0) {  // no neighbours: unmatchable as soon as it is blue
                    p.col[v] = kDead;
                    match[v] = 2;
                    atomicAdd(&ctl->retired[nx], 1);
                    continue;
                }
                p.col[v] = nb ? kBlue : kRed;
                dest = next_list(nb, deg);
            }
            if (dest == kStaged) {
                const unsigned long long old =
                    atomicAdd(&ctl->staged_pack[nx], (1ull << 32) | (unsigned long long)(unsigned)deg);
                p.lists[nx][kStaged][(int)(old >> 32)] = make_int4(it.x, it.y, it.z, (int)(old & 0xffffffffull));
            } else {
                p.lists[nx][dest][atomicAdd(&ctl->cnt[nx][dest], 1)] = it;
            }
        }
        __syncthreads();
        if (tid == 0) {
            long long next = (long long)(__ldcg(&ctl->staged_pack[nx]) >> 32);
            for (int l = 0; l < kStaged; ++l) next += __ldcg(&ctl->cnt[nx][l]);
            s_more = close_round(ctl, t, cap, has_next, seeds_short, next, 0u, __ldcg(&ctl->retired[nx]), true);
        }
        __syncthreads();
        if (!s_more) break;
    }
    (void)lane;
}

// After the loop: vertices still able to match keep their last colour as
// their match value (the reference leaves match[v] = 0 / 1 for them).
__global__ void __launch_bounds__(kBlockB) k_finish(Params p)
{
    const Ctl *ctl = p.ctl;
    const int par = ctl->t & 1;
    int cnt[kLists];
    long long total = 0;
#pragma unroll
    for (int l = 0; l < kLists; ++l) {
        cnt[l] = l == kStaged ? (int)(ctl->staged_pack[par] >> 32) : ctl->cnt[par][l];
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
        const int v = p.lists[par][which][k].x;
        ctl->match[v] = p.col[v];
    }
}

// ---------------------------------------------------------------------------
// Preparation: degree classes and reverse proposal keys.

struct PrepInfo {
    unsigned long long sum_deg;
    unsigned long long max_deg;
    unsigned long long short_count;   // lists of at most kSmallMax entries
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
        if (d > kSmallMax) {
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

// Control block rounded to 256 bytes so the seeds that follow it stay aligned.
constexpr size_t kCtlBytes = (sizeof(Ctl) + 255) / 256 * 256;

// Captured round loop of one (graph, type, stats) combination.
struct Plan {
    int type = 0;
    bool stats = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

struct PushState {
    uint8_t *col = nullptr;
    int2 *req = nullptr;
    unsigned long long *best = nullptr;
    unsigned long long *part_key = nullptr;
    int *part_cnt = nullptr;
    int4 *list_mem = nullptr;
    int4 *lists[2][kLists] = {};
    int *seg_mem = nullptr;
    int *seg_first[2] = {};
    uint32_t *seeds = nullptr;        // device: right after ctl in one allocation
    Ctl *ctl = nullptr;
    unsigned char *host_stage = nullptr;  // pinned: control block + seeds, uploaded in one copy
    unsigned char *host_back = nullptr;   // pinned: control block read back
    unsigned long long *stats = nullptr;
    Plan plans[8];
    int nplans = 0;
    int blocks_a = 0, blocks_b = 0, blocks_long = 0;
};

int bits_for(long long n)
{
    int b = 1;
    while ((1ll << b) < n) ++b;
    return b;
}

void free_state(PushState *s)
{
    for (int i = 0; i < s->nplans; ++i) {
        if (s->plans[i].exec) cudaGraphExecDestroy(s->plans[i].exec);
        if (s->plans[i].graph) cudaGraphDestroy(s->plans[i].graph);
    }
    // callers have synchronised the device (graph destroy or a failed set-up)
    dev_free(s->col, 0);
    dev_free(s->req, 0);
    dev_free(s->best, 0);
    dev_free(s->part_key, 0);
    dev_free(s->part_cnt, 0);
    dev_free(s->list_mem, 0);
    dev_free(s->seg_mem, 0);
    dev_free(s->ctl, 0);
    pinned_put(s->host_stage, kCtlBytes + 256 * sizeof(uint32_t));
    pinned_put(s->host_back, kCtlBytes);
    dev_free(s->stats, 0);
    delete s;
}

mm_status alloc_state(mm_graph *g, PushState **out)
{
    PushState *s = new (std::nothrow) PushState();
    if (!s) {
        set_error("push: host allocation failed");
        return MM_ERR_NOMEM;
    }
    const size_t n = (size_t)(g->n > 0 ? g->n : 1);
    // list capacities: every vertex is in at most one list per parity
    const size_t cap[kLists] = {(size_t)g->short_count, (size_t)g->short_count, (size_t)g->long_count,
                                (size_t)g->long_count};
    size_t per_parity = 0;
    for (int l = 0; l < kLists; ++l) per_parity += cap[l];
    const size_t nseg_cap = (size_t)(g->long_entries / kSegEntries) + 2;
    // pooled on the legacy stream, then synchronised so that any stream may use them
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = dev_alloc((void **)&s->col, n, 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->req, n * sizeof(int2), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->best, n * sizeof(unsigned long long), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->part_key, n * sizeof(unsigned long long), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->part_cnt, n * sizeof(int), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->list_mem, (2 * per_parity + 1) * sizeof(int4), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->seg_mem, 2 * nseg_cap * sizeof(int), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&s->ctl, kCtlBytes + 256 * sizeof(uint32_t), 0);
    if (e == cudaSuccess) s->seeds = reinterpret_cast<uint32_t *>(reinterpret_cast<unsigned char *>(s->ctl) + kCtlBytes);
    if (e == cudaSuccess) e = pinned_get((void **)&s->host_stage, kCtlBytes + 256 * sizeof(uint32_t));
    if (e == cudaSuccess) e = pinned_get((void **)&s->host_back, kCtlBytes);
    if (e == cudaSuccess)
        e = dev_alloc((void **)&s->stats, sizeof(unsigned long long) * kMaxRounds * MM_STATS_COLS, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        cudaDeviceSynchronize();
        free_state(s);
        cudaGetLastError();
        set_error(std::string("push: device allocation failed: ") + cudaGetErrorString(e));
        return MM_ERR_NOMEM;
    }
    size_t off = 0;
    for (int par = 0; par < 2; ++par) {
        for (int l = 0; l < kLists; ++l) {
            s->lists[par][l] = s->list_mem + off;
            off += cap[l];
        }
        s->seg_first[par] = s->seg_mem + par * nseg_cap;
    }
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int occ_a = 0, occ_l = 0, occ_b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a, k_phase_a_short<true, false>, kBlockA, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_l, k_phase_a_long<true, false>, kWarpsL * 32, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, k_phase_b<true, false>, kBlockT, 0);
    s->blocks_a = sms * (occ_a > 0 ? occ_a : 4);
    s->blocks_long = sms * (occ_l > 0 ? occ_l : 4);
    s->blocks_b = sms * (occ_b > 0 ? occ_b : 4);
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
        free_state(s);
        return cuda_fail(le, "push: kernel attributes");
    }
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
    p.part_key = s->part_key;
    p.part_cnt = s->part_cnt;
    for (int par = 0; par < 2; ++par) {
        for (int l = 0; l < kLists; ++l) p.lists[par][l] = s->lists[par][l];
        p.seg_first[par] = s->seg_first[par];
    }
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
    const int blocks_init = grid_for(g->n, kTileItems, s->blocks_b);

    cudaKernelNodeParams kp = {};
    kp.func = (void *)k_init<kStats>;
    kp.gridDim = dim3(blocks_init);
    kp.blockDim = dim3(kBlockT);
    kp.kernelParams = args;
    cudaGraphNode_t n_init, n_loop, n_fin, n_a, n_l, n_b;
    e = cudaGraphAddKernelNode(&n_init, graph, nullptr, 0, &kp);

    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    if (e == cudaSuccess) e = cudaGraphAddNode(&n_loop, graph, &n_init, 1, &cp);
    if (e == cudaSuccess) {
        // loop body: the two phase-A scans run side by side, then phase B
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        cudaKernelNodeParams ka = {};
        ka.func = (void *)k_phase_a_short<kW, kStats>;
        ka.gridDim = dim3(s->blocks_a);
        ka.blockDim = dim3(kBlockA);
        ka.kernelParams = args;
        e = cudaGraphAddKernelNode(&n_a, body, nullptr, 0, &ka);
        if (e == cudaSuccess) {
            cudaKernelNodeParams kl = {};
            kl.func = (void *)k_phase_a_long<kW, kStats>;
            kl.gridDim = dim3(s->blocks_long);
            kl.blockDim = dim3(kWarpsL * 32);
            kl.kernelParams = args;
            e = cudaGraphAddKernelNode(&n_l, body, nullptr, 0, &kl);
        }
        if (e == cudaSuccess) {
            cudaKernelNodeParams kb = {};
            kb.func = (void *)k_phase_b<kW, kStats>;
            kb.gridDim = dim3(s->blocks_b);
            kb.blockDim = dim3(kBlockT);
            kb.kernelParams = args;
            const cudaGraphNode_t deps[2] = {n_a, n_l};
            e = cudaGraphAddKernelNode(&n_b, body, deps, 2, &kb);
        }
    }
    cudaGraphNode_t n_tail;
    if (e == cudaSuccess) {
        cudaKernelNodeParams kt = {};
        kt.func = (void *)k_tail<kW, kStats>;
        kt.gridDim = dim3(1);
        kt.blockDim = dim3(kTailThreads);
        kt.kernelParams = args;
        e = cudaGraphAddKernelNode(&n_tail, graph, &n_loop, 1, &kt);
    }
    if (e == cudaSuccess) {
        cudaKernelNodeParams kf = {};
        kf.func = (void *)k_finish;
        kf.gridDim = dim3(grid_for(g->n, kBlockB, s->blocks_b));
        kf.blockDim = dim3(kBlockB);
        kf.kernelParams = args;
        e = cudaGraphAddKernelNode(&n_fin, graph, &n_tail, 1, &kf);
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
                   cudaStream_t stream)
{
    MM_CUDA_TRY(cudaMemcpyAsync(s->host_back, s->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream), "control read");
    if (stats && stats_rounds > 0)
        MM_CUDA_TRY(cudaMemcpyAsync(stats, s->stats,
                                    sizeof(long long) * MM_STATS_COLS *
                                        (size_t)(stats_rounds < kMaxRounds ? stats_rounds : kMaxRounds),
                                    cudaMemcpyDeviceToHost, stream),
                    "stats read");
    MM_CUDA_TRY(cudaStreamSynchronize(stream), "round loop");
    Ctl out;
    std::memcpy(&out, s->host_back, sizeof out);
    if (out.status == 2) {
        set_error("mm_match: a bounded device wait gave up (staged copy did not complete)");
        return MM_ERR_DEVICE;
    }
    if (out.status == 1 || out.rounds > nseeds) {
        set_error("mm_match: fewer seeds than rounds");
        return MM_ERR_SEEDS;
    }
    *rounds_out = out.rounds;
    return MM_OK;
}

template <bool kW>
mm_status stepped_rounds(mm_graph *g, PushState *s, int *rounds_done, float *ms_kernels, int cap_rounds,
                         cudaStream_t stream)
{
    Params p = make_params(g, s, kW, false, 0);
    const int blocks_init = grid_for(g->n, kTileItems, s->blocks_b);
    cudaEvent_t ev[4];
    for (int i = 0; i < 4; ++i) MM_CUDA_TRY(cudaEventCreate(&ev[i]), "event create");
    mm_status st = MM_OK;
    k_init<false><<<blocks_init, kBlockT, 0, stream>>>(p);
    int r = 0;
    for (;; ++r) {
        cudaEventRecord(ev[0], stream);
        k_phase_a_short<kW, false><<<s->blocks_a, kBlockA, 0, stream>>>(p);
        cudaEventRecord(ev[1], stream);
        k_phase_a_long<kW, false><<<s->blocks_long, kWarpsL * 32, 0, stream>>>(p);
        cudaEventRecord(ev[2], stream);
        k_phase_b<kW, false><<<s->blocks_b, kBlockT, 0, stream>>>(p);
        cudaEventRecord(ev[3], stream);
        int cont = 0;
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&cont, &s->ctl->cont, sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) {
            st = cuda_fail(e, "stepped round");
            break;
        }
        if (r < cap_rounds && ms_kernels) {
            for (int k = 0; k < 3; ++k) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
                ms_kernels[(size_t)r * MM_PROFILE_KERNELS + k] = ms;
            }
            ms_kernels[(size_t)r * MM_PROFILE_KERNELS + 3] = 0.f;
        }
        if (!cont) {
            ++r;
            break;
        }
    }
    if (st == MM_OK) {
        cudaEventRecord(ev[0], stream);
        k_tail<kW, false><<<1, kTailThreads, 0, stream>>>(p);
        cudaEventRecord(ev[1], stream);
        k_finish<<<grid_for(g->n, kBlockB, s->blocks_b), kBlockB, 0, stream>>>(p);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[1]);
        if (e != cudaSuccess) {
            st = cuda_fail(e, "tail / finish");
        } else if (r < cap_rounds && ms_kernels) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[0], ev[1]);
            for (int k = 0; k < MM_PROFILE_KERNELS; ++k) ms_kernels[(size_t)r * MM_PROFILE_KERNELS + k] = 0.f;
            ms_kernels[(size_t)r * MM_PROFILE_KERNELS + 3] = ms;
        }
    }
    for (int i = 0; i < 4; ++i) cudaEventDestroy(ev[i]);
    *rounds_done = r;
    return st;
}

}  // namespace

mm_status push_prepare(mm_graph *g, int weighted, cudaStream_t stream)
{
    const int wi = weighted ? 1 : 0;
    if (g->d_revkey[wi]) return MM_OK;
    const int n = g->n;
    if (n == 0) return MM_OK;

    // Degrees, classes, contiguity, slot offsets.
    if (!g->scanned) {
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

mm_status push_match(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds, int *d_match,
                     int *rounds_out, long long *stats, int stats_rounds, cudaStream_t stream)
{
    const bool weighted = is_weighted(type), maximal = is_maximal(type);
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
    if (want_stats)
        MM_CUDA_TRY(cudaMemsetAsync(s->stats, 0, sizeof(unsigned long long) * kMaxRounds * MM_STATS_COLS, stream),
                    "stats clear");
    MM_CUDA_TRY(cudaGraphLaunch(plan->exec, stream), "round loop launch");
    return end_call(g, s, nseeds, rounds_out, stats, stats_rounds, stream);
}

// Same kernels as push_match, launched one by one from the host with CUDA
// events around each phase, so the duration of every phase-A and phase-B
// launch can be read.  For measurement only (it synchronises every round).
mm_status push_profile(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds, int *d_match,
                       int *rounds_out, float *ms_kernels, int cap_rounds, int *launched, cudaStream_t stream)
{
    if (g->n == 0) return push_match(g, type, barrier, seeds, nseeds, d_match, rounds_out, nullptr, 0, stream);
    PushState *s = nullptr;
    mm_status st = begin_call(g, type, barrier, seeds, nseeds, d_match, stream, &s);
    if (st != MM_OK) return st;
    int executed = 0;
    st = is_weighted(type) ? stepped_rounds<true>(g, s, &executed, ms_kernels, cap_rounds, stream)
                           : stepped_rounds<false>(g, s, &executed, ms_kernels, cap_rounds, stream);
    if (st != MM_OK) return st;
    st = end_call(g, s, nseeds, rounds_out, nullptr, 0, stream);
    if (st == MM_OK && launched) *launched = 3 + 3 * executed;  // init, rounds, tail, finish
    return st;
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
}

}  // namespace mm
