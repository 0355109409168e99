// graphgen.cpp -- deterministic synthetic graphs in the reference's CSR layout.
//
// The reference reads DIMACS / UF Sparse Matrix files (graph.cu:86-511) that
// are not available here.  These generators stand in for them with the shapes
// the benchmark configurations name: 2-D 5-point grids, random geometric
// graphs, R-MAT power-law graphs and Erdos-Renyi graphs.  Every graph is
// symmetric, free of self-loops and duplicates, has each neighbour list
// sorted by neighbour id and stored contiguously (neighbourRanges[v].y ==
// neighbourRanges[v+1].x, as graph.cu:293-324 builds it), and is a pure
// function of its parameters and seed: every random draw is a counter-based
// splitmix64 value, so the OpenMP loops give identical output for any
// thread count.
//
// Edge weights (when not unit) are a hash of the sorted endpoint pair mapped
// to (0, 1] in steps of 2^-24, so both directions of an edge carry the same
// float, as MatrixMarket input does (graph.cu:285-323).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// k-th value of the stream named by (seed, stream).
inline uint64_t draw(uint64_t seed, uint64_t stream, uint64_t k)
{
    return splitmix64(splitmix64(seed ^ (stream * 0xD1B54A32D192ED03ull)) + k * 0x9E3779B97F4A7C15ull);
}

inline float pair_weight(uint32_t u, uint32_t v, uint64_t seed)
{
    const uint64_t lo = u < v ? u : v, hi = u < v ? v : u;
    const uint64_t h = splitmix64(splitmix64(seed + 0x5851F42D4C957F2Dull) ^ ((lo << 32) | hi));
    return (float)((double)((h >> 40) + 1) * (1.0 / 16777216.0));
}

int thread_count()
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// LSD radix sort of keys < 2^bits, 11-bit digits, OpenMP-parallel and stable.
void radix_sort_u64(std::vector<uint64_t> &keys, int bits)
{
    const size_t n = keys.size();
    if (n < 2) return;
    const int D = 11, B = 1 << D;
    std::vector<uint64_t> tmp(n);
    const int T = thread_count();
    std::vector<size_t> hist((size_t)T * B);
    for (int shift = 0; shift < bits; shift += D) {
        std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(T)
        {
#ifdef _OPENMP
            const int t = omp_get_thread_num();
#else
            const int t = 0;
#endif
            const size_t lo = n * t / T, hi = n * (t + 1) / T;
            size_t *h = &hist[(size_t)t * B];
            for (size_t i = lo; i < hi; ++i) ++h[(keys[i] >> shift) & (B - 1)];
#pragma omp barrier
#pragma omp single
            {
                size_t run = 0;
                for (int d = 0; d < B; ++d)
                    for (int tt = 0; tt < T; ++tt) {
                        const size_t c = hist[(size_t)tt * B + d];
                        hist[(size_t)tt * B + d] = run;
                        run += c;
                    }
            }
            for (size_t i = lo; i < hi; ++i) tmp[h[(keys[i] >> shift) & (B - 1)]++] = keys[i];
        }
        keys.swap(tmp);
    }
}

int bits_for(uint64_t n)
{
    int b = 0;
    while ((1ull << b) < n) ++b;
    return b < 1 ? 1 : b;
}

}  // namespace

struct mmg_csr {
    int n = 0;
    long long nnz = 0;
    std::vector<int> ranges;  // 2n: begin, end
    std::vector<int> nbrs;
    std::vector<float> weights;
};

namespace {

// Build a CSR from sorted, unique directed keys (src << bits | dst).
mmg_csr *csr_from_keys(int n, const std::vector<uint64_t> &keys, int bits, bool unit, uint64_t wseed)
{
    if ((long long)keys.size() >= (1ll << 31)) return nullptr;
    mmg_csr *g = new (std::nothrow) mmg_csr();
    if (!g) return nullptr;
    g->n = n;
    g->nnz = (long long)keys.size();
    g->ranges.assign((size_t)2 * n, 0);
    g->nbrs.resize(keys.size());
    g->weights.resize(keys.size());
    const uint64_t mask = (1ull << bits) - 1;
    std::vector<int> deg(n, 0);
    for (size_t i = 0; i < keys.size(); ++i) ++deg[keys[i] >> bits];
    int run = 0;
    for (int v = 0; v < n; ++v) {
        g->ranges[2 * v] = run;
        run += deg[v];
        g->ranges[2 * v + 1] = run;
    }
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)keys.size(); ++i) {
        const uint32_t u = (uint32_t)(keys[i] >> bits), v = (uint32_t)(keys[i] & mask);
        g->nbrs[i] = (int)v;
        g->weights[i] = unit ? 1.0f : pair_weight(u, v, wseed);
    }
    return g;
}

// Symmetrise directed edge list, drop self-loops and duplicates, build CSR.
mmg_csr *from_edge_pairs(int n, const std::vector<uint32_t> &us, const std::vector<uint32_t> &vs,
                         bool unit, uint64_t wseed)
{
    const int bits = bits_for((uint64_t)n);
    const size_t m = us.size();
    std::vector<uint64_t> keys;
    keys.resize(2 * m);
    size_t w = 0;
    for (size_t i = 0; i < m; ++i) {
        if (us[i] == vs[i]) continue;
        keys[w++] = ((uint64_t)us[i] << bits) | vs[i];
        keys[w++] = ((uint64_t)vs[i] << bits) | us[i];
    }
    keys.resize(w);
    radix_sort_u64(keys, 2 * bits);
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    return csr_from_keys(n, keys, bits, unit, wseed);
}

}  // namespace

#define MMG_API extern "C" __attribute__((visibility("default")))

// 2-D W x H grid, 5-point stencil: v = y*W + x, neighbours in ascending order
// (v-W, v-1, v+1, v+W), unit weights.
MMG_API mmg_csr *mmg_grid(int width, int height)
{
    if (width <= 0 || height <= 0 || (long long)width * height >= (1ll << 31)) return nullptr;
    mmg_csr *g = new (std::nothrow) mmg_csr();
    if (!g) return nullptr;
    const int n = width * height;
    g->n = n;
    g->ranges.assign((size_t)2 * n, 0);
    long long run = 0;
    for (int v = 0; v < n; ++v) {
        const int x = v % width, y = v / width;
        g->ranges[2 * v] = (int)run;
        if (y > 0) g->nbrs.push_back(v - width);
        if (x > 0) g->nbrs.push_back(v - 1);
        if (x + 1 < width) g->nbrs.push_back(v + 1);
        if (y + 1 < height) g->nbrs.push_back(v + width);
        run = (long long)g->nbrs.size();
        g->ranges[2 * v + 1] = (int)run;
    }
    g->nnz = run;
    g->weights.assign((size_t)run, 1.0f);
    return g;
}

// Random geometric graph: n points uniform in [0,1)^2, edge iff Euclidean
// distance < radius (radius = sqrt(avg_deg / (pi n))).  Hash weights in (0,1]
// unless unit != 0.
MMG_API mmg_csr *mmg_rgg(int n, double avg_deg, unsigned long long seed, int unit)
{
    if (n <= 0) return nullptr;
    const double r = std::sqrt(avg_deg / (M_PI * (double)n));
    const double r2 = r * r;
    std::vector<double> px(n), py(n);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        px[i] = (double)(draw(seed, 1, 2 * (uint64_t)i) >> 11) * (1.0 / 9007199254740992.0);
        py[i] = (double)(draw(seed, 1, 2 * (uint64_t)i + 1) >> 11) * (1.0 / 9007199254740992.0);
    }
    int G = (int)std::floor(1.0 / r);
    if (G < 1) G = 1;
    if (G > 65536) G = 65536;
    auto cell_of = [&](int i) {
        int cx = (int)(px[i] * G), cy = (int)(py[i] * G);
        cx = cx >= G ? G - 1 : cx;
        cy = cy >= G ? G - 1 : cy;
        return (long long)cy * G + cx;
    };
    const long long ncell = (long long)G * G;
    std::vector<long long> cstart(ncell + 1, 0);
    for (int i = 0; i < n; ++i) ++cstart[cell_of(i) + 1];
    for (long long c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    std::vector<int> order(n);
    {
        std::vector<long long> fill(cstart.begin(), cstart.end() - 1);
        for (int i = 0; i < n; ++i) order[fill[cell_of(i)]++] = i;
    }
    auto visit = [&](int i, auto &&emit) {
        const int cx = std::min((int)(px[i] * G), G - 1), cy = std::min((int)(py[i] * G), G - 1);
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int x = cx + dx, y = cy + dy;
                if (x < 0 || y < 0 || x >= G || y >= G) continue;
                const long long c = (long long)y * G + x;
                for (long long k = cstart[c]; k < cstart[c + 1]; ++k) {
                    const int j = order[k];
                    if (j == i) continue;
                    const double ddx = px[i] - px[j], ddy = py[i] - py[j];
                    if (ddx * ddx + ddy * ddy < r2) emit(j);
                }
            }
    };
    std::vector<int> deg(n, 0);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int i = 0; i < n; ++i) {
        int d = 0;
        visit(i, [&](int) { ++d; });
        deg[i] = d;
    }
    long long total = 0;
    for (int i = 0; i < n; ++i) total += deg[i];
    if (total >= (1ll << 31)) return nullptr;
    mmg_csr *g = new (std::nothrow) mmg_csr();
    if (!g) return nullptr;
    g->n = n;
    g->nnz = total;
    g->ranges.assign((size_t)2 * n, 0);
    g->nbrs.resize((size_t)total);
    g->weights.resize((size_t)total);
    long long run = 0;
    for (int i = 0; i < n; ++i) {
        g->ranges[2 * i] = (int)run;
        run += deg[i];
        g->ranges[2 * i + 1] = (int)run;
    }
#pragma omp parallel for schedule(dynamic, 4096)
    for (int i = 0; i < n; ++i) {
        int *out = &g->nbrs[g->ranges[2 * i]];
        int d = 0;
        visit(i, [&](int j) { out[d++] = j; });
        std::sort(out, out + d);
        for (int k = 0; k < d; ++k)
            g->weights[(size_t)g->ranges[2 * i] + k] = unit ? 1.0f : pair_weight((uint32_t)i, (uint32_t)out[k], seed);
    }
    return g;
}

// R-MAT graph with 2^scale vertices and edge_factor * 2^scale generated edges,
// quadrant probabilities (a, b, c, 1-a-b-c); symmetrised, self-loops and
// duplicates removed.  Each level draws 32 random bits.
MMG_API mmg_csr *mmg_rmat(int scale, int edge_factor, double a, double b, double c,
                          unsigned long long seed, int unit)
{
    if (scale < 1 || scale > 30 || edge_factor < 1) return nullptr;
    const int n = 1 << scale;
    const size_t m = (size_t)edge_factor << scale;
    const double two32 = 4294967296.0;
    const uint64_t ta = (uint64_t)(a * two32), tab = (uint64_t)((a + b) * two32),
                   tabc = (uint64_t)((a + b + c) * two32);
    std::vector<uint32_t> us(m), vs(m);
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < (long long)m; ++k) {
        uint32_t u = 0, v = 0;
        uint64_t bitsrc = 0;
        for (int lvl = 0; lvl < scale; ++lvl) {
            if ((lvl & 1) == 0) bitsrc = draw(seed, 2, (uint64_t)k * (uint64_t)((scale + 1) / 2) + (uint64_t)(lvl / 2));
            const uint64_t r = (lvl & 1) ? (bitsrc >> 32) : (bitsrc & 0xFFFFFFFFull);
            const uint32_t bit = 1u << (scale - 1 - lvl);
            if (r < ta) {
            } else if (r < tab) {
                v |= bit;
            } else if (r < tabc) {
                u |= bit;
            } else {
                u |= bit;
                v |= bit;
            }
        }
        us[k] = u;
        vs[k] = v;
    }
    return from_edge_pairs(n, us, vs, unit != 0, seed);
}

// Erdos-Renyi style graph: n * avg_deg / 2 uniformly random vertex pairs,
// symmetrised, self-loops and duplicates removed.
MMG_API mmg_csr *mmg_er(int n, double avg_deg, unsigned long long seed, int unit)
{
    if (n <= 1) return nullptr;
    const size_t m = (size_t)((double)n * avg_deg / 2.0);
    std::vector<uint32_t> us(m), vs(m);
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < (long long)m; ++k) {
        const uint64_t r = draw(seed, 3, (uint64_t)k);
        us[k] = (uint32_t)(((r & 0xFFFFFFFFull) * (uint64_t)n) >> 32);
        vs[k] = (uint32_t)(((r >> 32) * (uint64_t)n) >> 32);
    }
    return from_edge_pairs(n, us, vs, unit != 0, seed);
}

MMG_API int mmg_n(const mmg_csr *g) { return g ? g->n : 0; }
MMG_API long long mmg_nnz(const mmg_csr *g) { return g ? g->nnz : 0; }
MMG_API const int *mmg_ranges(const mmg_csr *g) { return g ? g->ranges.data() : nullptr; }
MMG_API const int *mmg_nbrs(const mmg_csr *g) { return g ? g->nbrs.data() : nullptr; }
MMG_API const float *mmg_weights(const mmg_csr *g) { return g ? g->weights.data() : nullptr; }
MMG_API void mmg_free(mmg_csr *g) { delete g; }
