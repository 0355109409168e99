// mm_capi.cu -- the C ABI of libmmatch.so (include/mm_match.h).
//
// Graph upload and validation (the reference's GraphMatchingGPU constructors,
// src/matchgpu.cu:39-147), matching dispatch (performMatching,
// src/matchgpu.cu:453-851) and error reporting.  No call aborts: every CUDA
// failure is turned into a status plus a thread-local message.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "mm_common.cuh"

#define MM_API extern "C" __attribute__((visibility("default")))

namespace mm {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

mm_status cuda_fail(cudaError_t e, const char *what)
{
    cudaGetLastError();  // clear a sticky-free error so later calls can proceed
    set_error(std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
    if (e == cudaErrorMemoryAllocation) return MM_ERR_NOMEM;
    return MM_ERR_CUDA;
}

// ---- memory ----------------------------------------------------------------
// Device buffers come from one stream-ordered pool per device whose release
// threshold is unlimited: memory a destroyed graph returns stays mapped in the
// pool and the next graph of similar size reuses it without a new mapping
// (cudaMalloc / cudaFree of gigabytes cost tens to hundreds of milliseconds).
// mm_release_cached_memory hands the unused part back to the driver.

namespace {
std::mutex g_pool_mu;
constexpr int kMaxDevices = 256;
cudaMemPool_t g_pools[kMaxDevices] = {};

struct PinnedBlock {
    void *ptr;
    size_t bytes;
};
std::mutex g_pinned_mu;
std::vector<PinnedBlock> g_pinned_free;
}  // namespace

static cudaError_t device_pool(int device, cudaMemPool_t *out)
{
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pools[device]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        cudaError_t e = cudaMemPoolCreate(&pool, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = ~0ull;
        e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return e;
        }
        g_pools[device] = pool;
    }
    *out = g_pools[device];
    return cudaSuccess;
}

cudaError_t dev_alloc(void **p, size_t bytes, cudaStream_t stream)
{
    *p = nullptr;
    int device = -1;
    cudaError_t e = cudaGetDevice(&device);
    cudaMemPool_t pool = nullptr;
    if (e == cudaSuccess) e = device_pool(device, &pool);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, stream);
    return e;
}

void dev_free(void *p, cudaStream_t stream)
{
    if (p) cudaFreeAsync(p, stream);
}

cudaError_t pinned_get(void **p, size_t bytes)
{
    {
        std::lock_guard<std::mutex> lock(g_pinned_mu);
        for (size_t i = 0; i < g_pinned_free.size(); ++i)
            if (g_pinned_free[i].bytes >= bytes) {
                *p = g_pinned_free[i].ptr;
                g_pinned_free.erase(g_pinned_free.begin() + (long)i);
                return cudaSuccess;
            }
    }
    const size_t rounded = (bytes + 4095) / 4096 * 4096;
    return cudaHostAlloc(p, rounded, cudaHostAllocPortable);
}

void pinned_put(void *p, size_t bytes)
{
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    g_pinned_free.push_back(PinnedBlock{p, (bytes + 4095) / 4096 * 4096});
}

mm_status release_cached(int device)
{
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        if (device >= 0 && device < kMaxDevices) pool = g_pools[device];
    }
    if (!pool) return MM_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    MM_CUDA_TRY(cudaSetDevice(device), "set device");
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemPoolTrimTo(pool, 0);
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) return cuda_fail(e, "release cached memory");
    return MM_OK;
}

mm_status ensure_scratch(mm_graph *g, size_t bytes)
{
    if (g->scratch_bytes >= bytes) return MM_OK;
    if (g->scratch) cudaFree(g->scratch);
    g->scratch = nullptr;
    g->scratch_bytes = 0;
    MM_CUDA_TRY(cudaMalloc(&g->scratch, bytes), "scratch allocation");
    g->scratch_bytes = bytes;
    return MM_OK;
}

namespace {

// Check every range and every neighbour id a kernel will read: a non-empty
// range must lie in [0, nnz) and its ids in [0, n).  Empty or reversed ranges
// are never read (the reference's loops run zero times), so they pass.
__global__ void k_validate(const int2 *ranges, const int *nbrs, int n, long long nnz, int *bad)
{
    const int lane = threadIdx.x & 31;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long v = warp0; v < n; v += nwarps) {
        const int2 r = ranges[v];
        if (r.y <= r.x) continue;
        if (r.x < 0 || (long long)r.y > nnz) {
            if (lane == 0) atomicOr(bad, 1);
            continue;
        }
        int local = 0;
        for (int j = r.x + lane; j < r.y; j += 32) {
            const int u = nbrs[j];
            local |= (u < 0 || u >= n);
        }
        if (__any_sync(0xffffffffu, local) && lane == 0) atomicOr(bad, 2);
    }
}

__global__ void k_fill_one(float *w, long long count)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        w[i] = 1.0f;
}

void free_graph(mm_graph *g)
{
    if (!g) return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(g->device);
    cudaDeviceSynchronize();  // pooled frees are stream-ordered: let every stream finish with the graph
    push_release(g);
    dev_free(g->d_ranges, 0);
    dev_free(g->d_nbrs, 0);
    dev_free(g->d_w, 0);
    cudaFree(g->scratch);
    dev_free(g->d_out, 0);
    cudaStreamSynchronize(0);
    if (prev >= 0) cudaSetDevice(prev);
    delete g;
}

// Shared tail of both create entry points: fill weights if absent, validate.
mm_status finish_create(mm_graph *g, bool have_weights)
{
    const size_t m = (size_t)(g->nnz > 0 ? g->nnz : 1);
    if (!have_weights) {
        k_fill_one<<<grid_for((long long)m, 256, 148 * 8), 256>>>(g->d_w, (long long)m);
        MM_CUDA_TRY(cudaGetLastError(), "unit weights");
    }
    g->has_weights = have_weights;
    int *d_bad = nullptr;
    MM_CUDA_TRY(dev_alloc((void **)&d_bad, sizeof(int), 0), "validation flag");
    cudaError_t e = cudaMemset(d_bad, 0, sizeof(int));
    if (e == cudaSuccess && g->n > 0) {
        k_validate<<<grid_for((long long)g->n * 32, 256, 148 * 16), 256>>>(g->d_ranges, g->d_nbrs, g->n, g->nnz, d_bad);
        e = cudaGetLastError();
    }
    int bad = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost);
    dev_free(d_bad, 0);
    if (e != cudaSuccess) return cuda_fail(e, "graph validation");
    if (bad & 1) {
        set_error("mm_graph_create: a neighbour range lies outside [0, nnz)");
        return MM_ERR_GRAPH;
    }
    if (bad & 2) {
        set_error("mm_graph_create: a neighbour id lies outside [0, n)");
        return MM_ERR_GRAPH;
    }
    return MM_OK;
}

mm_status create_common(int n, const int *ranges, long long nnz, const int *nbrs, const float *w, int device,
                        bool from_device, mm_graph **out)
{
    if (!out) {
        set_error("mm_graph_create: out is null");
        return MM_ERR_ARG;
    }
    *out = nullptr;
    if (n < 0 || nnz < 0 || (n > 0 && !ranges) || (nnz > 0 && !nbrs)) {
        set_error("mm_graph_create: bad sizes or null arrays");
        return MM_ERR_ARG;
    }
    if (nnz >= (1ll << 31)) {
        set_error("mm_graph_create: nnz must fit the reference's int indices (< 2^31)");
        return MM_ERR_UNSUPPORTED;
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (device >= 0) MM_CUDA_TRY(cudaSetDevice(device), "set device");
    mm_graph *g = new (std::nothrow) mm_graph();
    if (!g) {
        set_error("mm_graph_create: host allocation failed");
        return MM_ERR_NOMEM;
    }
    cudaGetDevice(&g->device);
    g->n = n;
    g->nnz = nnz;
    // Neighbour and weight arrays are padded to a multiple of 4 entries plus 4 so
    // that 16-byte vector loads starting at any in-range, 4-aligned slot stay inside.
    const size_t nv = (size_t)(n > 0 ? n : 1), ne = ((size_t)nnz + 3) / 4 * 4 + 4;
    const cudaMemcpyKind kind = from_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    cudaError_t e = dev_alloc((void **)&g->d_ranges, nv * sizeof(int2), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&g->d_nbrs, ne * sizeof(int), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&g->d_w, ne * sizeof(float), 0);
    if (e == cudaSuccess) e = cudaMemset(g->d_nbrs + nnz, 0, (ne - (size_t)nnz) * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(g->d_w + nnz, 0, (ne - (size_t)nnz) * sizeof(float));
    if (e == cudaSuccess && n > 0) e = cudaMemcpy(g->d_ranges, ranges, (size_t)n * sizeof(int2), kind);
    if (e == cudaSuccess && nnz > 0) e = cudaMemcpy(g->d_nbrs, nbrs, (size_t)nnz * sizeof(int), kind);
    if (e == cudaSuccess && nnz > 0 && w) e = cudaMemcpy(g->d_w, w, (size_t)nnz * sizeof(float), kind);
    mm_status s = MM_OK;
    if (e != cudaSuccess) s = cuda_fail(e, "graph upload");
    if (s == MM_OK) s = finish_create(g, w != nullptr);
    if (s != MM_OK) {
        free_graph(g);
        if (prev >= 0) cudaSetDevice(prev);
        return s;
    }
    if (prev >= 0 && device >= 0) cudaSetDevice(prev);
    *out = g;
    return MM_OK;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

mm_status check_match_args(mm_graph *g, int type, const uint32_t *seeds, int nseeds, const void *out,
                           int *rounds_out)
{
    if (!g || !rounds_out || (!out && g->n > 0)) {
        set_error("mm_match: null argument");
        return MM_ERR_ARG;
    }
    if (max_rounds_of(type) < 0) {
        set_error("mm_match: type must be 6, 7, 8 or 9");
        return MM_ERR_ARG;
    }
    if (!seeds || nseeds < 1) {
        set_error("mm_match: no seeds");
        return MM_ERR_SEEDS;
    }
    return MM_OK;
}

}  // namespace
}  // namespace mm

using namespace mm;

MM_API mm_status mm_graph_create(int n, const int *ranges, long long nnz, const int *neighbours,
                                 const float *weights, int device, mm_graph **out)
{
    return create_common(n, ranges, nnz, neighbours, weights, device, false, out);
}

MM_API mm_status mm_graph_create_device(int n, const int *d_ranges, long long nnz, const int *d_neighbours,
                                        const float *d_weights, mm_graph **out)
{
    return create_common(n, d_ranges, nnz, d_neighbours, d_weights, -1, true, out);
}

MM_API mm_status mm_graph_prepare(mm_graph *g, int type)
{
    if (!g || max_rounds_of(type) < 0) {
        set_error("mm_graph_prepare: bad argument");
        return MM_ERR_ARG;
    }
    DeviceGuard guard(g->device);
    return push_prepare(g, is_weighted(type) ? 1 : 0, 0);
}

MM_API void mm_graph_destroy(mm_graph *g) { free_graph(g); }

MM_API mm_status mm_release_cached_memory(int device) { return release_cached(device); }

MM_API int mm_graph_n(const mm_graph *g) { return g ? g->n : 0; }
MM_API long long mm_graph_nnz(const mm_graph *g) { return g ? g->nnz : 0; }
MM_API int mm_graph_weighted(const mm_graph *g) { return g && g->has_weights ? 1 : 0; }
MM_API const void *mm_graph_device_ranges(const mm_graph *g) { return g ? (const void *)g->d_ranges : nullptr; }
MM_API const int *mm_graph_device_neighbours(const mm_graph *g) { return g ? g->d_nbrs : nullptr; }
MM_API const float *mm_graph_device_weights(const mm_graph *g) { return g ? g->d_w : nullptr; }

MM_API int mm_max_rounds(int type) { return max_rounds_of(type); }

MM_API mm_status mm_match_ex(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                             int *d_match_out, int *rounds_out, int path, void *stream)
{
    mm_status s = check_match_args(g, type, seeds, nseeds, d_match_out, rounds_out);
    if (s != MM_OK) return s;
    DeviceGuard guard(g->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (path == MM_PATH_PULL)
        return pull_match(g, type, barrier, seeds, nseeds, d_match_out, rounds_out, nullptr, 0, st);
    if (path == MM_PATH_AUTO || path == MM_PATH_PUSH)
        return push_match(g, type, barrier, seeds, nseeds, d_match_out, rounds_out, nullptr, 0, st);
    set_error("mm_match_ex: unknown path");
    return MM_ERR_ARG;
}

MM_API mm_status mm_match_device(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                                 int *d_match_out, int *rounds_out, void *stream)
{
    return mm_match_ex(g, type, barrier, seeds, nseeds, d_match_out, rounds_out, MM_PATH_AUTO, stream);
}

MM_API mm_status mm_match(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                          int *match_out, int *rounds_out, void *stream)
{
    mm_status s = check_match_args(g, type, seeds, nseeds, match_out, rounds_out);
    if (s != MM_OK) return s;
    DeviceGuard guard(g->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (!g->d_out) {
        MM_CUDA_TRY(dev_alloc((void **)&g->d_out, (size_t)(g->n > 0 ? g->n : 1) * sizeof(int), 0), "match buffer");
        MM_CUDA_TRY(cudaStreamSynchronize(0), "match buffer");
    }
    s = push_match(g, type, barrier, seeds, nseeds, g->d_out, rounds_out, nullptr, 0, st);
    if (s == MM_OK && g->n > 0) {
        cudaError_t e = cudaMemcpyAsync(match_out, g->d_out, (size_t)g->n * sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) s = cuda_fail(e, "match download");
    }
    return s;
}

MM_API mm_status mm_match_stats(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                                int *d_match_out, int *rounds_out, long long *stats, int stats_rounds, int path,
                                void *stream)
{
    mm_status s = check_match_args(g, type, seeds, nseeds, d_match_out, rounds_out);
    if (s != MM_OK) return s;
    if (!stats) {
        set_error("mm_match_stats: stats is null");
        return MM_ERR_ARG;
    }
    DeviceGuard guard(g->device);
    if (path == MM_PATH_PULL)
        return pull_match(g, type, barrier, seeds, nseeds, d_match_out, rounds_out, stats, stats_rounds,
                          (cudaStream_t)stream);
    return push_match(g, type, barrier, seeds, nseeds, d_match_out, rounds_out, stats, stats_rounds,
                      (cudaStream_t)stream);
}

MM_API mm_status mm_match_profile(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                                  int *d_match_out, int *rounds_out, float *ms_per_kernel, int cap_rounds,
                                  int *launches, void *stream)
{
    mm_status s = check_match_args(g, type, seeds, nseeds, d_match_out, rounds_out);
    if (s != MM_OK) return s;
    DeviceGuard guard(g->device);
    return push_profile(g, type, barrier, seeds, nseeds, d_match_out, rounds_out, ms_per_kernel, cap_rounds, launches,
                        (cudaStream_t)stream);
}

MM_API const char *mm_last_error(void) { return g_last_error.c_str(); }

MM_API const char *mm_version(void) { return "mmatch 0.1 (sm_100a)"; }
