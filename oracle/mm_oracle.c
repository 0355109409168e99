/*
 * mm_oracle.c -- CPU restatement of the reference GPU matching round loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it.
 * The product (libmmatch.so) never calls it and has no CPU fallback.
 *
 * What it restates (Multicore-Matching, src/matchgpu.cu):
 *   - gSelect / gaSelect      matchgpu.cu:184-258  hash colouring blue/red
 *   - grRequest / grRespond   matchgpu.cu:286-357  random greedy request/respond
 *   - gwRequest / gwRespond   matchgpu.cu:360-451  weighted request/respond
 *   - gMatch                  matchgpu.cu:260-283  commit mutual requests
 *   - round loops             matchgpu.cu:507-524 (type 6), 604-615 (type 7),
 *                             705-722 (type 8), 811-822 (type 9)
 *   - getWeight               matchcpu.cu:64-97
 *   - testMatching counters   matchcpu.cu:127-246 (plus maximality as a count)
 *
 * Pinning: the maximal types (7, 9) are checked bit-for-bit against the
 * reference's own GraphMatchingTBBRandom / GraphMatchingTBBWeighted
 * (matchtbb.cu:498-623) compiled from the reference sources into oracle/_ref,
 * and the fixed-round types (6, 8) against the same TBB code built with its
 * round cap at NR_MATCH_ROUNDS.  The committed fixtures under tests/golden/
 * were produced by that reference build (tests/golden/make_golden.py).
 *
 * Each phase reads only arrays that no iteration of the same phase writes, so
 * the OpenMP loops give the same result for every thread count.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MMO_FIXED_ROUNDS 20   /* NR_MATCH_ROUNDS, matchcpu.h:24 */
#define MMO_MAX_ROUNDS 256    /* NR_MAX_MATCH_ROUNDS, matchcpu.h:25 */

/* Per-round instrumentation record (one row of int64 per executed round). */
enum {
    MMO_ST_ACTIVE = 0,   /* vertices with match < 2 when the round's select ran */
    MMO_ST_BLUE,         /* of those, coloured blue */
    MMO_ST_RED,          /* of those, coloured red */
    MMO_ST_REQ_ENTRIES,  /* adjacency entries the request loop inspected */
    MMO_ST_RESP_ENTRIES, /* adjacency entries the respond loop inspected */
    MMO_ST_BLUE_DEG,     /* sum of full degrees of blue vertices */
    MMO_ST_RED_DEG,      /* sum of full degrees of red vertices */
    MMO_ST_MATCHED,      /* vertices newly matched in the round */
    MMO_ST_DEAD,         /* vertices newly marked unmatchable in the round */
    MMO_ST_COLS
};

/* First 16 SHA-256 round constants and the MD5 round-1 rotation amounts; the
 * colouring hash of matchgpu.cu:167-182 uses exactly these 16 steps. */
static const uint32_t kMix[16] = {
    0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u,
    0x923f82a4u, 0xab1c5ed5u, 0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u,
    0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u};
static const int kRot[4] = {7, 12, 17, 22};

static inline uint32_t rotl32(uint32_t x, int s) { return (x << s) | (x >> (32 - s)); }

/* Sum h0+h1+h2+h3 of the colouring hash for vertex v and round seed r
 * (matchgpu.cu:196-217). */
uint32_t mmo_colour_hash(uint32_t v, uint32_t r)
{
    uint32_t h0 = 0x67452301u, h1 = 0xefcdab89u, h2 = 0x98badcfeu, h3 = 0x10325476u;
    uint32_t a = h0, b = h1, c = h2, d = h3, g = v;
    for (int k = 0; k < 16; ++k) {
        const uint32_t f = (b & c) | (~b & d);
        const uint32_t t = d;
        d = c;
        c = b;
        b = b + rotl32(a + f + kMix[k] + g, kRot[k & 3]);
        a = t;
        h0 += a; h1 += b; h2 += c; h3 += d;
        g *= r;
    }
    return h0 + h1 + h2 + h3;
}

static inline int span_begin(const int *ranges, int v) { return ranges[2 * v]; }
static inline int span_end(const int *ranges, int v) { return ranges[2 * v + 1]; }

/* Colour every vertex that can still be matched (match < 2).  Returns the number
 * of such vertices (the reference's keep-matching flag is "> 0"). */
static long long select_phase(int n, int *match, uint32_t seed, uint32_t barrier,
                              long long *blue_out)
{
    long long active = 0, blue = 0;
#pragma omp parallel for schedule(static) reduction(+ : active, blue)
    for (int v = 0; v < n; ++v) {
        if (match[v] >= 2) continue;
        ++active;
        const int colour = mmo_colour_hash((uint32_t)v, seed) < barrier ? 0 : 1;
        blue += colour == 0;
        match[v] = colour;
    }
    *blue_out = blue;
    return active;
}

/* Blue vertices propose (grRequest / gwRequest). */
static void request_phase(int n, const int *ranges, const int *nbrs, const float *w,
                          int weighted, const int *match, int *req, long long *inspected,
                          long long *blue_deg)
{
    long long seen = 0, bdeg = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : seen, bdeg)
    for (int v = 0; v < n; ++v) {
        if (match[v] != 0) { req[v] = n; continue; }
        const int b = span_begin(ranges, v), e = span_end(ranges, v);
        if (e > b) bdeg += e - b;
        int dead = 1;
        if (!weighted) {
            int chosen = -1;
            for (int j = b; j < e; ++j) {
                ++seen;
                const int m = match[nbrs[j]];
                if (m < 4) {
                    if (m == 1) { chosen = nbrs[j]; break; }
                    dead = 0;
                }
            }
            req[v] = chosen >= 0 ? chosen : n + dead;
        } else {
            float best = -1.0f;
            int chosen = n;
            for (int j = b; j < e; ++j) {
                ++seen;
                const int u = nbrs[j];
                const int m = match[u];
                if (m < 4) {
                    if (m == 1 && w[j] > best) { best = w[j]; chosen = u; }
                    dead = 0;
                }
            }
            req[v] = chosen + dead;
        }
    }
    *inspected = seen;
    *blue_deg = bdeg;
}

/* Red vertices answer one proposer (grRespond / gwRespond).  Only red entries
 * of req[] are written and only blue entries are read, so the loop is race free. */
static void respond_phase(int n, const int *ranges, const int *nbrs, const float *w,
                          int weighted, const int *match, int *req, long long *inspected,
                          long long *red_deg)
{
    long long seen = 0, rdeg = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : seen, rdeg)
    for (int v = 0; v < n; ++v) {
        if (match[v] != 1) continue;
        const int b = span_begin(ranges, v), e = span_end(ranges, v);
        if (e > b) rdeg += e - b;
        if (!weighted) {
            for (int j = b; j < e; ++j) {
                ++seen;
                const int u = nbrs[j];
                if (match[u] == 0 && req[u] == v) { req[v] = u; break; }
            }
        } else {
            float best = -1.0f;
            int chosen = n;
            for (int j = b; j < e; ++j) {
                ++seen;
                const int u = nbrs[j];
                if (match[u] == 0 && req[u] == v && w[j] > best) { best = w[j]; chosen = u; }
            }
            if (chosen < n) req[v] = chosen;
        }
    }
    *inspected = seen;
    *red_deg = rdeg;
}

/* Commit mutual proposals and retire dead blue vertices (gMatch). */
static void commit_phase(int n, int *match, const int *req, long long *matched, long long *dead)
{
    long long mcount = 0, dcount = 0;
#pragma omp parallel for schedule(static) reduction(+ : mcount, dcount)
    for (int v = 0; v < n; ++v) {
        const int r = req[v];
        if (r == n + 1) { match[v] = 2; ++dcount; }
        else if (r < n && req[r] == v) { match[v] = 4 + (v < r ? v : r); ++mcount; }
    }
    *matched = mcount;
    *dead = dcount;
}

/*
 * Run one GPU-type matching (6 random, 7 random maximal, 8 weighted, 9 weighted
 * maximal) on a CSR given as ranges[2n] = {begin, end} pairs (the int2
 * neighbourRanges of graph.h:56), nbrs[] and optional weights w[].
 *
 * seeds[] holds the values the reference draws from rand() once per executed
 * round (matchgpu.cu:509, 609, 707, 816); nseeds must cover every round that
 * runs (20 for the fixed types, up to 255 for the maximal ones).  match[n] is
 * overwritten.  If stats is non-null it receives MMO_ST_COLS int64 per round for
 * up to stats_cap rounds.  Returns the number of rounds executed (= seeds
 * consumed), or -1 if nseeds ran out.
 */
int mmo_match(int n, const int *ranges, const int *nbrs, const float *w, int type,
              uint32_t barrier, const uint32_t *seeds, int nseeds, int *match,
              long long *stats, int stats_cap, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    const int weighted = (type == 8 || type == 9);
    const int maximal = (type == 7 || type == 9);
    int *req = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (!req) return -1;
    memset(match, 0, sizeof(int) * (size_t)n);
    memset(req, 0, sizeof(int) * (size_t)(n > 0 ? n : 1));

    int rounds = 0;
    for (;;) {
        if (maximal) {
            /* while (keepMatching == 1 && ++count < NR_MAX_MATCH_ROUNDS) */
            if (rounds + 1 >= MMO_MAX_ROUNDS) break;
        } else if (rounds >= MMO_FIXED_ROUNDS) {
            break;
        }
        if (rounds >= nseeds) { free(req); return -1; }
        long long row[MMO_ST_COLS] = {0};
        long long blue = 0;
        const long long active = select_phase(n, match, seeds[rounds], barrier, &blue);
        row[MMO_ST_ACTIVE] = active;
        row[MMO_ST_BLUE] = blue;
        row[MMO_ST_RED] = active - blue;
        request_phase(n, ranges, nbrs, w, weighted, match, req, &row[MMO_ST_REQ_ENTRIES],
                      &row[MMO_ST_BLUE_DEG]);
        respond_phase(n, ranges, nbrs, w, weighted, match, req, &row[MMO_ST_RESP_ENTRIES],
                      &row[MMO_ST_RED_DEG]);
        commit_phase(n, match, req, &row[MMO_ST_MATCHED], &row[MMO_ST_DEAD]);
        if (stats && rounds < stats_cap) memcpy(stats + (size_t)rounds * MMO_ST_COLS, row, sizeof row);
        ++rounds;
        if (maximal && active == 0) break;
    }
    free(req);
    return rounds;
}

/* glibc rand() stream after srand(seed): the values the reference's host loop
 * would draw, in order. */
void mmo_rand_seeds(uint32_t seed, int count, uint32_t *out)
{
    srand(seed);
    for (int i = 0; i < count; ++i) out[i] = (uint32_t)rand();
}

/* GraphMatching::getWeight (matchcpu.cu:64-97): size counts matched vertices
 * that found their partner among their neighbours, weight is half the sum. */
void mmo_weight(int n, const int *ranges, const int *nbrs, const float *w, const int *match,
                double *weight_out, long long *size_out)
{
    double weight = 0.0;
    long long size = 0;
    for (int v = 0; v < n; ++v) {
        const int m = match[v];
        if (m < 4) continue;
        for (int j = span_begin(ranges, v); j < span_end(ranges, v); ++j) {
            if (match[nbrs[j]] == m) {
                weight += w ? (double)w[j] : 1.0;
                ++size;
                break;
            }
        }
    }
    *weight_out = weight / 2.0;
    *size_out = size;
}

/* testMatching (src/matchcpu.cu:127-246): the matched vertices sorted by match
 * value (ties by id here; the reference's std::sort leaves that order open) are
 * walked two at a time.  i1, then i2: if i2's value differs, i1 is
 * under-matched and i2 is consumed with it; else the pair must be in each
 * other's lists (else invalidly matched) and every further vertex of the value
 * is multi-matched.  Then every unmatched vertex with an unmatched neighbour
 * other than itself can still be matched.  out: under, multi, invalid,
 * matchable; returns the verdict (the first three are zero). */
static const int *g_sort_match;
static int by_value_then_id(const void *pa, const void *pb)
{
    const int a = *(const int *)pa, b = *(const int *)pb;
    const int ma = g_sort_match[a], mb = g_sort_match[b];
    if (ma != mb) return ma < mb ? -1 : 1;
    return a < b ? -1 : (a > b);
}

static int in_span(const int *ranges, const int *nbrs, int a, int b)
{
    for (int j = span_begin(ranges, a); j < span_end(ranges, a); ++j)
        if (nbrs[j] == b) return 1;
    return 0;
}

int mmo_check(int n, const int *ranges, const int *nbrs, const int *match, long long out[4])
{
    int *order = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int cnt = 0;
    for (int v = 0; v < n; ++v)
        if (match[v] >= 4) order[cnt++] = v;
    g_sort_match = match;
    qsort(order, (size_t)cnt, sizeof(int), by_value_then_id);
    long long under = 0, multi = 0, invalid = 0, matchable = 0;
    int p = 0;
    while (p < cnt) {
        const int i1 = order[p++];
        const int cur = match[i1];
        if (p == cnt) { ++under; continue; }
        const int i2 = order[p++];
        if (match[i2] != cur) { ++under; continue; }
        if (!in_span(ranges, nbrs, i1, i2) || !in_span(ranges, nbrs, i2, i1)) ++invalid;
        while (p < cnt && match[order[p]] == cur) { ++multi; ++p; }
    }
    for (int v = 0; v < n; ++v) {
        if (match[v] >= 4) continue;
        for (int j = span_begin(ranges, v); j < span_end(ranges, v); ++j) {
            const int u = nbrs[j];
            if (u != v && match[u] < 4) { ++matchable; break; }
        }
    }
    free(order);
    out[0] = under; out[1] = multi; out[2] = invalid; out[3] = matchable;
    return under == 0 && multi == 0 && invalid == 0;
}
