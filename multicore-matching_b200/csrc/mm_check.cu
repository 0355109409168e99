// mm_check.cu -- GPU validation and weight of a matching.
//
// Device counterparts of the reference's host-side checks, so that a matching
// of a large graph can be judged without copying it back and sorting it on
// the host:
//   mm_matching_weight  GraphMatching::getWeight   (src/matchcpu.cu:64-97)
//   mm_matching_check   GraphMatching::testMatching (src/matchcpu.cu:127-246)
// Both read the graph's device CSR and a device match array, and report
// through their outputs; nothing is printed.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>

#include "mm_common.cuh"

#define MM_API extern "C" __attribute__((visibility("default")))

namespace mm {
namespace {

__device__ __forceinline__ bool is_matched(int m) { return m >= 4; }  // matchcpu.h:41

// getWeight: a matched vertex i adds the weight of the first entry of its list
// whose neighbour carries the same match value, and counts 1.  contrib[i]
// holds that weight (0 otherwise); size is counted alongside.
__global__ void k_weight(const int2 *ranges, const int *nbrs, const float *w, const int *match, int n,
                         double *contrib, unsigned long long *size)
{
    unsigned long long cnt = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int m = match[i];
        double x = 0.0;
        if (is_matched(m)) {
            const int2 r = ranges[i];
            for (int j = r.x; j < r.y; ++j) {
                if (match[nbrs[j]] == m) {
                    x = (double)w[j];
                    ++cnt;
                    break;
                }
            }
        }
        contrib[i] = x;
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(size, cnt);
}

// Sort keys for testMatching's order: unmatched vertices first, then by match
// value; the sort is stable, so a value's vertices follow in increasing id.
__global__ void k_check_keys(const int *match, int n, unsigned *keys, int *ids)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int m = match[i];
        keys[i] = is_matched(m) ? (unsigned)m : 0u;
        ids[i] = i;
    }
}

// Is b in a's list?  Binary search when the graph's lists are sorted.
__device__ bool in_list(const int2 *ranges, const int *nbrs, int a, int b, bool sorted)
{
    const int2 r = ranges[a];
    if (r.y <= r.x) return false;
    if (sorted) {
        int lo = r.x, hi = r.y;
        while (lo < hi) {
            const int mid = (int)(((long long)lo + hi) >> 1);
            if (nbrs[mid] < b) lo = mid + 1;
            else hi = mid;
        }
        return lo < r.y && nbrs[lo] == b;
    }
    for (int j = r.x; j < r.y; ++j)
        if (nbrs[j] == b) return true;
    return false;
}

// testMatching walks the matched vertices in sorted order two at a time: i1,
// then i2.  A pair of equal values is checked (both must be in each other's
// lists, else "invalidly matched") and further vertices of that value are
// "multi-matched"; if i2's value differs, i1 is "under-matched" and i2 is
// consumed with it, so the walk enters i2's group at its second vertex.
// Per group of equal value (size s), the walk is a map of one bit: whether
// the group's first vertex was already consumed (c).  Entering with c:
//   s - c >= 2   pair (c, c + 1) checked, s - c - 2 multi-matched, leave 0
//   s - c == 1   one under-matched, leave 1 (the next group's first is consumed)
//   s - c == 0   nothing (the group was that consumed vertex), leave 0
// A prefix scan of the composed maps gives each group its c, exactly as the
// sequential walk would.
__global__ void k_group_flags(const unsigned *keys, int n, int *flag)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        flag[p] = keys[p] != 0u && (p == 0 || keys[p - 1] != keys[p]) ? 1 : 0;
}

__global__ void k_group_starts(const int *flag, const int *gidx, int n, int *starts)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        if (flag[p]) starts[gidx[p]] = p;
}

// bit c of a map: the bit it leaves for the next group when entered with c
__global__ void k_group_maps(const int *starts, int ngroups, uint8_t *maps)
{
    for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < ngroups; gi += gridDim.x * blockDim.x) {
        const int s = starts[gi + 1] - starts[gi];
        const int out0 = s == 1 ? 1 : 0, out1 = s == 2 ? 1 : 0;
        maps[gi] = (uint8_t)(out0 | (out1 << 1));
    }
}

struct ComposeMaps {
    // a applies first, then b
    __host__ __device__ uint8_t operator()(uint8_t a, uint8_t b) const
    {
        const int r0 = (b >> (a & 1)) & 1, r1 = (b >> ((a >> 1) & 1)) & 1;
        return (uint8_t)(r0 | (r1 << 1));
    }
};

// counts: [0] under, [1] multi, [2] invalid
__global__ void k_group_eval(const int *starts, const uint8_t *prefix, int ngroups, const int *ids, const int2 *ranges,
                             const int *nbrs, int sorted, unsigned long long *counts)
{
    unsigned long long under = 0, multi = 0, invalid = 0;
    for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < ngroups; gi += gridDim.x * blockDim.x) {
        const int c = prefix[gi] & 1;  // the composed maps of all earlier groups, entered with 0
        const int p = starts[gi], s = starts[gi + 1] - p, r = s - c;
        if (r >= 2) {
            const int i1 = ids[p + c], i2 = ids[p + c + 1];
            if (!in_list(ranges, nbrs, i1, i2, sorted != 0) || !in_list(ranges, nbrs, i2, i1, sorted != 0)) ++invalid;
            multi += (unsigned long long)(r - 2);
        } else if (r == 1) {
            ++under;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        under += __shfl_down_sync(0xffffffffu, under, o);
        multi += __shfl_down_sync(0xffffffffu, multi, o);
        invalid += __shfl_down_sync(0xffffffffu, invalid, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (under) atomicAdd(counts + 0, under);
        if (multi) atomicAdd(counts + 1, multi);
        if (invalid) atomicAdd(counts + 2, invalid);
    }
}

// Vertices that can still be matched: unmatched with an unmatched neighbour
// other than themselves.  counts[3] matchable, counts[4] unmatched.
__global__ void k_check_matchable(const int2 *ranges, const int *nbrs, const int *match, int n,
                                  unsigned long long *counts)
{
    unsigned long long matchable = 0, unmatched = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (is_matched(match[i])) continue;
        ++unmatched;
        const int2 r = ranges[i];
        for (int j = r.x; j < r.y; ++j) {
            const int u = nbrs[j];
            if (u != i && !is_matched(match[u])) {
                ++matchable;
                break;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        matchable += __shfl_down_sync(0xffffffffu, matchable, o);
        unmatched += __shfl_down_sync(0xffffffffu, unmatched, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (matchable) atomicAdd(counts + 3, matchable);
        if (unmatched) atomicAdd(counts + 4, unmatched);
    }
}

struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceScope()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace
}  // namespace mm

using namespace mm;

MM_API mm_status mm_matching_weight(mm_graph *g, const int *d_match, double *weight, long long *size, void *stream)
{
    if (!g || !weight || !size || (!d_match && g->n > 0)) {
        set_error("mm_matching_weight: null argument");
        return MM_ERR_ARG;
    }
    *weight = 0.0;
    *size = 0;
    if (g->n == 0) return MM_OK;
    DeviceScope scope(g->device);
    cudaStream_t st = (cudaStream_t)stream;
    const int n = g->n;
    double *contrib = nullptr, *sum = nullptr;
    unsigned long long *cnt = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    cudaError_t e = dev_alloc((void **)&contrib, sizeof(double) * (size_t)n, st);
    if (e == cudaSuccess) e = dev_alloc((void **)&sum, sizeof(double), st);
    if (e == cudaSuccess) e = dev_alloc((void **)&cnt, sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess) {
        k_weight<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(g->d_ranges, g->d_nbrs, g->d_w, d_match, n, contrib, cnt);
        e = cudaGetLastError();
    }
    // a fixed reduction tree: the same sum on every run
    if (e == cudaSuccess) e = cub::DeviceReduce::Sum(nullptr, tmp_bytes, contrib, sum, n, st);
    if (e == cudaSuccess) e = dev_alloc(&tmp, tmp_bytes, st);
    if (e == cudaSuccess) e = cub::DeviceReduce::Sum(tmp, tmp_bytes, contrib, sum, n, st);
    double total = 0.0;
    unsigned long long count = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, sum, sizeof total, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&count, cnt, sizeof count, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    dev_free(tmp, st);
    dev_free(contrib, st);
    dev_free(sum, st);
    dev_free(cnt, st);
    if (e != cudaSuccess) return cuda_fail(e, "mm_matching_weight");
    *weight = total / 2.0;  // every matched edge is counted from both ends
    *size = (long long)count;
    return MM_OK;
}

MM_API mm_status mm_matching_check(mm_graph *g, const int *d_match, long long *counts, int *valid, void *stream)
{
    if (!g || !counts || !valid || (!d_match && g->n > 0)) {
        set_error("mm_matching_check: null argument");
        return MM_ERR_ARG;
    }
    for (int k = 0; k < 5; ++k) counts[k] = 0;
    *valid = 1;
    if (g->n == 0) return MM_OK;
    DeviceScope scope(g->device);
    cudaStream_t st = (cudaStream_t)stream;
    const int n = g->n;
    unsigned *k0 = nullptr, *k1 = nullptr;
    int *v0 = nullptr, *v1 = nullptr;
    unsigned long long *c = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    cudaError_t e = dev_alloc((void **)&k0, sizeof(unsigned) * (size_t)n, st);
    if (e == cudaSuccess) e = dev_alloc((void **)&k1, sizeof(unsigned) * (size_t)n, st);
    if (e == cudaSuccess) e = dev_alloc((void **)&v0, sizeof(int) * (size_t)n, st);
    if (e == cudaSuccess) e = dev_alloc((void **)&v1, sizeof(int) * (size_t)n, st);
    if (e == cudaSuccess) e = dev_alloc((void **)&c, sizeof(unsigned long long) * 5, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(c, 0, sizeof(unsigned long long) * 5, st);
    if (e == cudaSuccess) {
        k_check_keys<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(d_match, n, k0, v0);
        e = cudaGetLastError();
    }
    cub::DoubleBuffer<unsigned> kb(k0, k1);
    cub::DoubleBuffer<int> vb(v0, v1);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kb, vb, n, 0, 32, st);
    if (e == cudaSuccess) e = dev_alloc(&tmp, tmp_bytes, st);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, kb, vb, n, 0, 32, st);
    // groups of equal value: starts, per-group maps, their prefix composition, counts
    int *flag = nullptr, *gidx = nullptr, *starts = nullptr;
    uint8_t *maps = nullptr, *prefix = nullptr;
    void *tmp2 = nullptr;
    size_t tmp2_bytes = 0;
    int ngroups = 0;
    if (e == cudaSuccess) e = dev_alloc((void **)&flag, sizeof(int) * (size_t)n, st);
    if (e == cudaSuccess) e = dev_alloc((void **)&gidx, sizeof(int) * (size_t)n, st);
    if (e == cudaSuccess) {
        k_group_flags<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(kb.Current(), n, flag);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tmp2_bytes, flag, gidx, n, st);
    if (e == cudaSuccess) e = dev_alloc(&tmp2, tmp2_bytes, st);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp2, tmp2_bytes, flag, gidx, n, st);
    int last[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last[0], gidx + n - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last[1], flag + n - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    dev_free(tmp2, st);
    tmp2 = nullptr;
    if (e == cudaSuccess) ngroups = last[0] + last[1];
    if (e == cudaSuccess && ngroups > 0) {
        e = dev_alloc((void **)&starts, sizeof(int) * ((size_t)ngroups + 1), st);
        if (e == cudaSuccess) e = dev_alloc((void **)&maps, (size_t)ngroups, st);
        if (e == cudaSuccess) e = dev_alloc((void **)&prefix, (size_t)ngroups, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(starts + ngroups, &n, sizeof(int), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            k_group_starts<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(flag, gidx, n, starts);
            k_group_maps<<<grid_for(ngroups, 256, 148 * 8), 256, 0, st>>>(starts, ngroups, maps);
            e = cudaGetLastError();
        }
        tmp2_bytes = 0;
        if (e == cudaSuccess)
            e = cub::DeviceScan::ExclusiveScan(nullptr, tmp2_bytes, maps, prefix, ComposeMaps(), (uint8_t)2, ngroups, st);
        if (e == cudaSuccess) e = dev_alloc(&tmp2, tmp2_bytes, st);
        if (e == cudaSuccess)
            e = cub::DeviceScan::ExclusiveScan(tmp2, tmp2_bytes, maps, prefix, ComposeMaps(), (uint8_t)2, ngroups, st);
        if (e == cudaSuccess) {
            k_group_eval<<<grid_for(ngroups, 256, 148 * 8), 256, 0, st>>>(starts, prefix, ngroups, vb.Current(),
                                                                          g->d_ranges, g->d_nbrs,
                                                                          g->sym_struct ? 1 : 0, c);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // n above is a host value copied asynchronously
    dev_free(tmp2, st);
    dev_free(flag, st);
    dev_free(gidx, st);
    dev_free(starts, st);
    dev_free(maps, st);
    dev_free(prefix, st);
    if (e == cudaSuccess) {
        k_check_matchable<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(g->d_ranges, g->d_nbrs, d_match, n, c);
        e = cudaGetLastError();
    }
    unsigned long long h[5] = {0, 0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, c, sizeof h, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    dev_free(tmp, st);
    dev_free(k0, st);
    dev_free(k1, st);
    dev_free(v0, st);
    dev_free(v1, st);
    dev_free(c, st);
    if (e != cudaSuccess) return cuda_fail(e, "mm_matching_check");
    for (int k = 0; k < 5; ++k) counts[k] = (long long)h[k];
    *valid = (h[0] == 0 && h[1] == 0 && h[2] == 0) ? 1 : 0;
    return MM_OK;
}
