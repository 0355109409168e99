// mm_contract.cu -- contraction of a matched graph (one level of multilevel coarsening).
//
// No counterpart in the reference, which stops at the matching; this is the
// step that multilevel partitioners put after it.  Each matched pair becomes
// one coarse vertex and every unmatched vertex stays one; the coarse lists
// hold the members' entries mapped to coarse ids, in increasing id, without
// self-loops, and an edge that several fine entries map to carries the sum of
// their weights.  The sum is taken in double and rounded once, so it does not
// depend on the order of the entries: the coarse graph of a symmetric graph is
// symmetric again, weights included (exactly so while the weights' sum fits a
// double's mantissa, as for weights on a common 2^-k grid).
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include <climits>

#include "mm_common.cuh"

#define MM_API extern "C" __attribute__((visibility("default")))

namespace mm {
namespace {

__device__ __forceinline__ int degree_of(int2 r) { return r.y > r.x ? r.y - r.x : 0; }

// rep[v]: the smaller vertex of v's pair (the match value minus 4), or v.
// A value naming no vertex, or a vertex that does not name v back, is an
// invalid matching: bad is set and v stays alone.
__global__ void k_reps(const int *match, int n, int *rep, int *flag, int *bad)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int m = match[v];
        int r = v;
        if (m >= 4) {
            const long long a = (long long)m - 4;
            if (a >= n || match[a] != m) atomicOr(bad, 1);
            else r = (int)a;
        }
        rep[v] = r;
        flag[v] = r == v ? 1 : 0;
    }
}

// cmap[v] = coarse id of v's representative; coarse degree bound = sum of the
// members' degrees; a member's entries start after its representative's.
__global__ void k_cmap(const int2 *ranges, const int *rep, const int *cid, int n, int *cmap, long long *cdeg,
                       int *member_off)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int r = rep[v];
        const int c = cid[r];
        cmap[v] = c;
        const int d = degree_of(ranges[v]);
        if (d) atomicAdd((unsigned long long *)&cdeg[c], (unsigned long long)d);
        member_off[v] = r == v ? 0 : degree_of(ranges[r]);
    }
}

// Entries of the members, mapped: key = coarse neighbour (INT_MAX for a
// self-loop, sorted last and dropped), value = weight.
__global__ void k_scatter(const int2 *ranges, const int *nbrs, const float *w, const int *cmap, const int *member_off,
                          const long long *coff, int n, int *key, float *val)
{
    const int lane = threadIdx.x & 31;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long v = warp0; v < n; v += nwarps) {
        const int2 r = ranges[v];
        const int c = cmap[v];
        const long long base = coff[c] + member_off[v];
        for (int j = r.x + lane; j < r.y; j += 32) {
            const int cu = cmap[nbrs[j]];
            key[base + (j - r.x)] = cu == c ? INT_MAX : cu;
            val[base + (j - r.x)] = w[j];
        }
    }
}

// Runs of equal key within a coarse list: a run's first entry is its head.
__global__ void k_heads(const int *key, const long long *coff, const int *seg_of, long long total, int *head)
{
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        const long long s0 = coff[seg_of[k]];
        head[k] = key[k] != INT_MAX && (k == s0 || key[k - 1] != key[k]) ? 1 : 0;
    }
}

__global__ void k_seg_of(const long long *coff, int nc, int *seg_of)
{
    const int lane = threadIdx.x & 31;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long c = warp0; c < nc; c += nwarps)
        for (long long k = coff[c] + lane; k < coff[c + 1]; k += 32) seg_of[k] = (int)c;
}

// A head writes its key and the run's weight sum (double, rounded once).
__global__ void k_merge(const int *key, const float *val, const int *head, const long long *hpos, long long total,
                        int *out_nbr, float *out_w)
{
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        if (!head[k]) continue;
        double s = 0.0;
        long long e = k;
        do {
            s += (double)val[e];
            ++e;
        } while (e < total && !head[e] && key[e] == key[k]);
        out_nbr[hpos[k]] = key[k];
        out_w[hpos[k]] = (float)s;
    }
}

__global__ void k_coarse_ranges(const long long *coff, const long long *hpos_ext, int nc, int2 *ranges)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
        ranges[c] = make_int2((int)hpos_ext[coff[c]], (int)hpos_ext[coff[c + 1]]);
}

struct Scratch {
    static constexpr int kMax = 32;
    void *p[kMax] = {};
    int k = 0;
    cudaStream_t st;
    explicit Scratch(cudaStream_t s) : st(s) {}
    template <class T>
    cudaError_t get(T **out, size_t count)
    {
        if (k == kMax) return cudaErrorMemoryAllocation;
        cudaError_t e = dev_alloc((void **)out, sizeof(T) * (count ? count : 1), st);
        if (e == cudaSuccess) p[k++] = *out;
        return e;
    }
    ~Scratch()
    {
        cudaStreamSynchronize(st);
        for (int i = 0; i < k; ++i) dev_free(p[i], st);
        cudaStreamSynchronize(st);
    }
};

}  // namespace
}  // namespace mm

using namespace mm;

MM_API mm_status mm_graph_contract(mm_graph *g, const int *d_match, mm_graph **coarse, int *d_cmap)
{
    if (!g || !coarse || (!d_match && g->n > 0)) {
        set_error("mm_graph_contract: null argument");
        return MM_ERR_ARG;
    }
    *coarse = nullptr;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != g->device) MM_CUDA_TRY(cudaSetDevice(g->device), "set device");
    const int n = g->n;
    cudaStream_t st = 0;
    mm_status result = MM_OK;
    {
        Scratch sc(st);
        int *rep = nullptr, *flag = nullptr, *cid = nullptr, *cmap = nullptr, *bad = nullptr, *member_off = nullptr;
        long long *cdeg = nullptr, *coff = nullptr;
        cudaError_t e = sc.get(&rep, n);
        if (e == cudaSuccess) e = sc.get(&flag, n + 1);
        if (e == cudaSuccess) e = sc.get(&cid, n + 1);
        if (e == cudaSuccess) e = sc.get(&bad, 1);
        if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int), st);
        if (e == cudaSuccess) e = cudaMemsetAsync(flag + n, 0, sizeof(int), st);
        if (e == cudaSuccess && n > 0) {
            k_reps<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(d_match, n, rep, flag, bad);
            e = cudaGetLastError();
        }
        void *tmp = nullptr;
        size_t tb = 0;
        if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb, flag, cid, n + 1, st);
        if (e == cudaSuccess) e = sc.get((char **)&tmp, tb);
        if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tb, flag, cid, n + 1, st);
        int nc = 0, hbad = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&nc, cid + n, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && hbad) {
            set_error("mm_graph_contract: the match array is not a matching (a value names no partner that names it back)");
            result = MM_ERR_ARG;
        }
        if (e == cudaSuccess && result == MM_OK) {
            cmap = d_cmap;
            if (!cmap) e = sc.get(&cmap, n);
            if (e == cudaSuccess) e = sc.get(&member_off, n);
            if (e == cudaSuccess) e = sc.get(&cdeg, (size_t)nc + 1);
            if (e == cudaSuccess) e = sc.get(&coff, (size_t)nc + 1);
            if (e == cudaSuccess) e = cudaMemsetAsync(cdeg, 0, sizeof(long long) * ((size_t)nc + 1), st);
            if (e == cudaSuccess && n > 0) {
                k_cmap<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(g->d_ranges, rep, cid, n, cmap, cdeg, member_off);
                e = cudaGetLastError();
            }
            tb = 0;
            void *tmp2 = nullptr;
            if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb, cdeg, coff, nc + 1, st);
            if (e == cudaSuccess) e = sc.get((char **)&tmp2, tb);
            if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp2, tb, cdeg, coff, nc + 1, st);
            long long total = 0;
            if (e == cudaSuccess) e = cudaMemcpyAsync(&total, coff + nc, sizeof total, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            int *k0 = nullptr, *k1 = nullptr, *seg_of = nullptr, *head = nullptr, *out_nbr = nullptr;
            float *v0 = nullptr, *v1 = nullptr, *out_w = nullptr;
            long long *hpos = nullptr;
            int2 *cranges = nullptr;
            if (e == cudaSuccess) e = sc.get(&k0, total);
            if (e == cudaSuccess) e = sc.get(&k1, total);
            if (e == cudaSuccess) e = sc.get(&v0, total);
            if (e == cudaSuccess) e = sc.get(&v1, total);
            if (e == cudaSuccess) e = sc.get(&seg_of, total);
            if (e == cudaSuccess) e = sc.get(&head, total + 1);
            if (e == cudaSuccess) e = sc.get(&hpos, total + 1);
            if (e == cudaSuccess) e = cudaMemsetAsync(head + total, 0, sizeof(int), st);
            if (e == cudaSuccess && n > 0) {
                k_scatter<<<grid_for((long long)n * 32, 256, 148 * 16), 256, 0, st>>>(
                    g->d_ranges, g->d_nbrs, g->d_w, cmap, member_off, coff, n, k0, v0);
                e = cudaGetLastError();
            }
            // stable: equal neighbours keep the members' list order
            if (e == cudaSuccess && total > 0) {
                tb = 0;
                void *tmp3 = nullptr;
                e = cub::DeviceSegmentedSort::StableSortPairs(nullptr, tb, k0, k1, v0, v1, total, nc, coff, coff + 1, st);
                if (e == cudaSuccess) e = sc.get((char **)&tmp3, tb);
                if (e == cudaSuccess)
                    e = cub::DeviceSegmentedSort::StableSortPairs(tmp3, tb, k0, k1, v0, v1, total, nc, coff, coff + 1, st);
            }
            if (e == cudaSuccess && nc > 0) {
                k_seg_of<<<grid_for((long long)nc * 32, 256, 148 * 16), 256, 0, st>>>(coff, nc, seg_of);
                k_heads<<<grid_for(total, 256, 148 * 8), 256, 0, st>>>(k1, coff, seg_of, total, head);
                e = cudaGetLastError();
            }
            tb = 0;
            void *tmp4 = nullptr;
            if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb, head, hpos, total + 1, st);
            if (e == cudaSuccess) e = sc.get((char **)&tmp4, tb);
            if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp4, tb, head, hpos, total + 1, st);
            long long ne = 0;
            if (e == cudaSuccess) e = cudaMemcpyAsync(&ne, hpos + total, sizeof ne, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e == cudaSuccess) e = sc.get(&out_nbr, ne);
            if (e == cudaSuccess) e = sc.get(&out_w, ne);
            if (e == cudaSuccess) e = sc.get(&cranges, nc);
            if (e == cudaSuccess && total > 0) {
                k_merge<<<grid_for(total, 256, 148 * 8), 256, 0, st>>>(k1, v1, head, hpos, total, out_nbr, out_w);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess && nc > 0) {
                k_coarse_ranges<<<grid_for(nc, 256, 148 * 8), 256, 0, st>>>(coff, hpos, nc, cranges);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                result = cuda_fail(e, "mm_graph_contract");
            } else {
                // coarse weights are the merged sums even when the fine graph had unit weights
                result = mm_graph_create_device(nc, reinterpret_cast<const int *>(cranges), ne, out_nbr, out_w, coarse);
            }
        } else if (e != cudaSuccess) {
            result = cuda_fail(e, "mm_graph_contract");
        }
    }
    if (prev >= 0 && prev != g->device) cudaSetDevice(prev);
    return result;
}
