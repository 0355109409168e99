// mm_capi.cu -- the C ABI of libmmatch.so (include/mm_match.h).
//
// Graph upload and validation (the reference's GraphMatchingGPU constructors,
// src/matchgpu.cu:39-147), matching dispatch (performMatching,
// src/matchgpu.cu:453-851) and error reporting.  No call aborts: every CUDA
// failure is turned into a status plus a thread-local message.
#include <cuda_runtime.h>

#include <cstdio>
#include <atomic>
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
// testing hooks (mm_debug)
std::atomic<long long> g_dbg_spin_limit{0};   // 0: the kernels' own limit
std::atomic<int> g_dbg_skip_mark{-1};
std::atomic<long long> g_dbg_alloc_limit{-1};  // pool bytes in use above which allocations fail
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
    const long long limit = g_dbg_alloc_limit.load();
    if (e == cudaSuccess && limit >= 0) {
        uint64_t used = 0;
        e = cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
        if (e == cudaSuccess && (long long)(used + bytes) > limit) return cudaErrorMemoryAllocation;
    }
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, stream);
    return e;
}

long long debug_spin_limit()
{
    const long long v = g_dbg_spin_limit.load();
    return v > 0 ? v : kSpinLimitDefault;
}

int debug_skip_mark() { return g_dbg_skip_mark.load(); }

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

// ---- validation ----
//
// Every range and neighbour id a kernel will read is checked: a non-empty
// range must lie in [0, nnz) and its ids in [0, n).  Empty or reversed ranges
// are never read (the reference's loops run zero times), so they pass.  The
// same passes establish the graph properties the push path can use:
//   contiguous   ranges tile [0, nnz) in vertex order;
//   sorted       every list is strictly increasing (no duplicate entries);
//   symmetric    the multiset of entries (v, u) equals that of (u, v), and
//                with weights, of (v, u, w) and (u, v, w).
// Symmetry is tested with two pairs of 64-bit sums of a hash of the ordered
// entry (splitmix64's finalizer): a transposed multiset has equal sums, a
// different one has equal sums only by a 64-bit coincidence.
struct GraphCheck {
    unsigned long long fwd_s, rev_s;  // structure: sum F(v, u), sum F(u, v)
    unsigned long long fwd_w, rev_w;  // with weight bits
    int bad;        // 1: a range outside [0, nnz); 2: an id outside [0, n)
    int noncontig;  // ranges do not tile [0, nnz) in vertex order
    int unsorted;   // some list is not strictly increasing
    int pad;
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ unsigned long long hash_s(unsigned a, unsigned b)
{
    return mix64((((unsigned long long)a << 32) | b) + 0x9E3779B97F4A7C15ull);
}
__device__ __forceinline__ unsigned long long hash_w(unsigned a, unsigned b, unsigned wbits)
{
    return mix64((((unsigned long long)a << 32) | b) ^ mix64((unsigned long long)wbits + 0xD1B54A32D192ED03ull));
}

__global__ void k_check_ranges(const int2 *ranges, int n, long long nnz, GraphCheck *c)
{
    int bad = 0, nc = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int2 r = ranges[v];
        if (r.y > r.x && (r.x < 0 || (long long)r.y > nnz)) bad = 1;
        if (r.y < r.x) nc = 1;
        if (v == 0 && r.x != 0) nc = 1;
        if (v + 1 < n && ranges[v + 1].x != r.y) nc = 1;
        if (v == n - 1 && (long long)r.y != nnz) nc = 1;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&c->bad, 1);
    if (__any_sync(0xffffffffu, nc) && (threadIdx.x & 31) == 0) atomicOr(&c->noncontig, 1);
}

// Contiguous CSR: slots [j0, j1) in chunks of kChk, a block per chunk; the
// owner of each slot comes from a table of the chunk's list starts.
constexpr int kChk = 2048;

__device__ __forceinline__ int first_owner(const int2 *ranges, int n, long long s)
{
    int lo = 0, hi = n - 1;  // largest v with ranges[v].x <= s
    while (lo < hi) {
        const int mid = (int)(((long long)lo + hi + 1) >> 1);
        if ((long long)ranges[mid].x <= s) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <bool kWeights>
__global__ void __launch_bounds__(256) k_check_entries(const int2 *ranges, const int *nbrs, const float *w, int n,
                                                       long long j0, long long j1, GraphCheck *c)
{
    __shared__ int start[kChk + 1];
    __shared__ int s_v0, s_cnt;
    unsigned long long fs = 0, rs = 0, fw = 0, rw = 0;
    int bad = 0, uns = 0;
    const long long chunks = (j1 - j0 + kChk - 1) / kChk;
    for (long long ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
        const long long c0 = j0 + ch * kChk, c1 = min(c0 + kChk, j1);
        __syncthreads();
        if (threadIdx.x == 0) {
            const int v0 = first_owner(ranges, n, c0), v1 = first_owner(ranges, n, c1 - 1);
            s_v0 = v0;
            s_cnt = v1 - v0 + 1;
        }
        __syncthreads();
        const int v0 = s_v0, cnt = s_cnt;
        const bool table = cnt <= kChk + 1;
        if (table)
            for (int i = threadIdx.x; i < cnt; i += blockDim.x) start[i] = ranges[v0 + i].x;
        __syncthreads();
        for (long long j = c0 + threadIdx.x; j < c1; j += blockDim.x) {
            int v;
            if (table) {
                int lo = 0, hi = cnt - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if ((long long)start[mid] <= j) lo = mid;
                    else hi = mid - 1;
                }
                v = v0 + lo;
            } else {
                v = first_owner(ranges, n, j);
            }
            const int u = nbrs[j];
            if (u < 0 || u >= n) {
                bad = 1;
                continue;
            }
            // compared with the entry before (earlier chunks have arrived; later ones may not have)
            if (j > (long long)ranges[v].x && nbrs[j - 1] >= u) uns = 1;
            fs += hash_s((unsigned)v, (unsigned)u);
            rs += hash_s((unsigned)u, (unsigned)v);
            if (kWeights) {
                const unsigned wb = __float_as_uint(w[j]);
                fw += hash_w((unsigned)v, (unsigned)u, wb);
                rw += hash_w((unsigned)u, (unsigned)v, wb);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        fs += __shfl_down_sync(0xffffffffu, fs, o);
        rs += __shfl_down_sync(0xffffffffu, rs, o);
        fw += __shfl_down_sync(0xffffffffu, fw, o);
        rw += __shfl_down_sync(0xffffffffu, rw, o);
    }
    bad = __any_sync(0xffffffffu, bad);
    uns = __any_sync(0xffffffffu, uns);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&c->fwd_s, fs);
        atomicAdd(&c->rev_s, rs);
        if (kWeights) {
            atomicAdd(&c->fwd_w, fw);
            atomicAdd(&c->rev_w, rw);
        }
        if (bad) atomicOr(&c->bad, 2);
        if (uns) atomicOr(&c->unsorted, 1);
    }
}

// Any CSR: bounds of every id, a warp per list.
__global__ void k_validate(const int2 *ranges, const int *nbrs, int n, long long nnz, GraphCheck *c)
{
    const int lane = threadIdx.x & 31;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long v = warp0; v < n; v += nwarps) {
        const int2 r = ranges[v];
        if (r.y <= r.x || r.x < 0 || (long long)r.y > nnz) continue;
        int local = 0;
        for (int j = r.x + lane; j < r.y; j += 32) {
            const int u = nbrs[j];
            local |= (u < 0 || u >= n);
        }
        if (__any_sync(0xffffffffu, local) && lane == 0) atomicOr(&c->bad, 2);
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
    dev_free(g->d_goff, 0);
    dev_free(g->d_vbase, 0);
    dev_free(g->d_last, 0);
    cudaStreamSynchronize(0);
    if (prev >= 0) cudaSetDevice(prev);
    delete g;
}

// Graph upload and validation.  The ranges go first and are checked; for a
// contiguous CSR the neighbour ids and weights then follow in chunks on a copy
// stream while a second stream checks each chunk that has arrived, so the
// checks hide under the transfer.
constexpr long long kUploadChunk = 1ll << 24;  // entries per chunk

mm_status upload_and_check(mm_graph *g, const int *ranges, const int *nbrs, const float *w,
                           cudaMemcpyKind kind)
{
    const int n = g->n;
    const long long nnz = g->nnz;
    GraphCheck *d_c = nullptr;
    MM_CUDA_TRY(dev_alloc((void **)&d_c, sizeof(GraphCheck), 0), "validation state");
    cudaError_t e = cudaMemsetAsync(d_c, 0, sizeof(GraphCheck), 0);
    if (e == cudaSuccess && n > 0) e = cudaMemcpyAsync(g->d_ranges, ranges, (size_t)n * sizeof(int2), kind, 0);
    if (e == cudaSuccess && n > 0) {
        k_check_ranges<<<grid_for(n, 256, 148 * 8), 256>>>(g->d_ranges, n, nnz, d_c);
        e = cudaGetLastError();
    }
    GraphCheck c = {};
    if (e == cudaSuccess) e = cudaMemcpy(&c, d_c, sizeof c, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && (c.bad & 1)) {
        dev_free(d_c, 0);
        set_error("mm_graph_create: a neighbour range lies outside [0, nnz)");
        return MM_ERR_GRAPH;
    }
    const bool contiguous = n > 0 && !c.noncontig;
    const bool have_w = w != nullptr;
    // Weighted graphs from host memory also get their preference windows here:
    // a chunk's check is followed by the windows of the vertices whose lists
    // end in it (host ranges say which), so they too hide under the transfer.
    bool windows = e == cudaSuccess && contiguous && nnz > 0 && have_w && kind == cudaMemcpyHostToDevice;
    if (windows && windows_begin(g, 0) != MM_OK) windows = false;
    if (e == cudaSuccess && contiguous && nnz > 0) {
        cudaStream_t cs = nullptr, ks = nullptr;
        cudaEvent_t ev = nullptr;
        e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ks, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        int va = 0;  // first vertex whose window is not built yet
        for (long long j0 = 0; e == cudaSuccess && j0 < nnz; j0 += kUploadChunk) {
            const long long j1 = j0 + kUploadChunk < nnz ? j0 + kUploadChunk : nnz;
            const size_t cnt = (size_t)(j1 - j0);
            e = cudaMemcpyAsync(g->d_nbrs + j0, nbrs + j0, cnt * sizeof(int), kind, cs);
            if (e == cudaSuccess && have_w) e = cudaMemcpyAsync(g->d_w + j0, w + j0, cnt * sizeof(float), kind, cs);
            if (e == cudaSuccess) e = cudaEventRecord(ev, cs);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(ks, ev, 0);
            if (e == cudaSuccess) {
                const int grid = grid_for((long long)cnt, kChk, 148 * 8);
                if (have_w) k_check_entries<true><<<grid, 256, 0, ks>>>(g->d_ranges, g->d_nbrs, g->d_w, n, j0, j1, d_c);
                else k_check_entries<false><<<grid, 256, 0, ks>>>(g->d_ranges, g->d_nbrs, g->d_w, n, j0, j1, d_c);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess && windows) {
                // vertices whose lists end at or before j1 (ends rise with v)
                int lo = va, hi = n;
                while (lo < hi) {
                    const int mid = lo + (hi - lo) / 2;
                    if ((long long)ranges[2 * (size_t)mid + 1] <= j1) lo = mid + 1;
                    else hi = mid;
                }
                const int vb = j1 == nnz ? n : lo;
                if (windows_range(g, va, vb, ks) != MM_OK) windows = false;
                va = vb;
            }
        }
        if (e == cudaSuccess && windows && windows_end(g, ks) != MM_OK) windows = false;
        // both streams are drained on every path: buffers may be freed next
        const cudaError_t eks = ks ? cudaStreamSynchronize(ks) : cudaSuccess;
        const cudaError_t ecs = cs ? cudaStreamSynchronize(cs) : cudaSuccess;
        if (e == cudaSuccess) e = eks != cudaSuccess ? eks : ecs;
        if (ev) cudaEventDestroy(ev);
        if (cs) cudaStreamDestroy(cs);
        if (ks) cudaStreamDestroy(ks);
    } else if (e == cudaSuccess) {
        if (nnz > 0) e = cudaMemcpy(g->d_nbrs, nbrs, (size_t)nnz * sizeof(int), kind);
        if (e == cudaSuccess && nnz > 0 && have_w) e = cudaMemcpy(g->d_w, w, (size_t)nnz * sizeof(float), kind);
        if (e == cudaSuccess && n > 0) {
            k_validate<<<grid_for((long long)n * 32, 256, 148 * 16), 256>>>(g->d_ranges, g->d_nbrs, n, nnz, d_c);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess && !have_w) {
        const size_t m = (size_t)(nnz > 0 ? nnz : 1);
        k_fill_one<<<grid_for((long long)m, 256, 148 * 8), 256>>>(g->d_w, (long long)m);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&c, d_c, sizeof c, cudaMemcpyDeviceToHost);
    dev_free(d_c, 0);
    if (!windows) windows_discard(g);  // built later, on demand, if the upload could not
    cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "graph upload and validation");
    if (c.bad & 2) {
        set_error("mm_graph_create: a neighbour id lies outside [0, n)");
        return MM_ERR_GRAPH;
    }
    g->has_weights = have_w;
    g->sym_struct = contiguous && !c.unsorted && c.fwd_s == c.rev_s;
    // unit weights are symmetric whenever the structure is
    g->sym_weights = g->sym_struct && (!have_w || c.fwd_w == c.rev_w);
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
    if (e == cudaSuccess) e = cudaMemsetAsync(g->d_nbrs + nnz, 0, (ne - (size_t)nnz) * sizeof(int), 0);
    if (e == cudaSuccess) e = cudaMemsetAsync(g->d_w + nnz, 0, (ne - (size_t)nnz) * sizeof(float), 0);
    // the non-blocking upload streams do not wait for the legacy stream: settle the pool first
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    mm_status s = MM_OK;
    if (e != cudaSuccess) s = cuda_fail(e, "graph allocation");
    if (s == MM_OK) s = upload_and_check(g, ranges, nbrs, w, kind);
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

// ---- batches of independent graphs ----
// vbase[v] = first vertex of v's graph (a warp per graph), then every entry
// must stay inside its vertex's graph: the union is disjoint.
// vbase[v]: the first vertex of v's graph; vend[v]: one past its last.
__global__ void k_batch_vbase(const int *goff, int ngraphs, int *vbase, int *vend)
{
    const int lane = threadIdx.x & 31;
    const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long gi = gwarp; gi < ngraphs; gi += nwarps) {
        const int lo = goff[gi], hi = goff[gi + 1];
        for (int v = lo + lane; v < hi; v += 32) {
            vbase[v] = lo;
            vend[v] = hi;
        }
    }
}

// Every entry of vertex v must name a vertex of v's own graph [vbase[v],
// vend[v]): a comparison per entry, a thread per vertex (neighbouring vertices'
// lists are neighbours in memory, so the pass streams), with no gather.
__global__ void k_batch_edges(const int2 *ranges, const int *nbrs, const int *vbase, const int *vend, int n, int *bad)
{
    int cross = 0;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const int2 r = ranges[v];
        const int lo = vbase[v], hi = vend[v];
        for (int j = r.x; j < r.y; ++j) {
            const int u = __ldg(nbrs + j);
            cross |= u < lo || u >= hi;
        }
    }
    if (__any_sync(0xffffffffu, cross) && (threadIdx.x & 31) == 0) atomicOr(bad, 1);
}

// ---- measurement: random-gather ceiling ----
//
// The round kernel's scans are bound by random single-sector reads (colour
// gathers, window and key loads), not by streaming bandwidth.  This probe
// times the device's rate for them: every thread reads a coalesced stream of
// random indices and gathers one byte per index from a table.
__global__ void k_probe_indices(int *idx, long long m, int range, unsigned long long seed)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
        unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ull + seed;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        idx[i] = (int)((z >> 32) % (unsigned long long)range);
    }
}

__global__ void k_probe_gather(const int *__restrict__ idx, long long m, const uint8_t *table, unsigned *sink)
{
    unsigned acc = 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += 4 * stride) {
        int j[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) j[k] = i + k * stride < m ? __ldcs(idx + i + k * stride) : 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) acc += table[j[k]];
    }
    if (acc == 0xffffffffu) sink[0] = acc;  // keeps the gathers live
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

MM_API mm_status mm_graph_copy_out(const mm_graph *g, int *ranges, int *neighbours, float *weights)
{
    if (!g) {
        set_error("mm_graph_copy_out: null graph");
        return MM_ERR_ARG;
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != g->device) MM_CUDA_TRY(cudaSetDevice(g->device), "set device");
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && ranges && g->n > 0)
        e = cudaMemcpy(ranges, g->d_ranges, sizeof(int2) * (size_t)g->n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && neighbours && g->nnz > 0)
        e = cudaMemcpy(neighbours, g->d_nbrs, sizeof(int) * (size_t)g->nnz, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && weights && g->nnz > 0)
        e = cudaMemcpy(weights, g->d_w, sizeof(float) * (size_t)g->nnz, cudaMemcpyDeviceToHost);
    if (prev >= 0 && prev != g->device) cudaSetDevice(prev);
    if (e != cudaSuccess) return cuda_fail(e, "mm_graph_copy_out");
    return MM_OK;
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
    if (path == MM_PATH_PULL) {
        if (g->ngraphs > 0) {
            set_error("mm_match_ex: the reference-structured path matches single graphs only");
            return MM_ERR_UNSUPPORTED;
        }
        return pull_match(g, type, barrier, seeds, nseeds, d_match_out, rounds_out, nullptr, 0, st);
    }
    if (path == MM_PATH_AUTO || path == MM_PATH_PUSH)
        return push_match(g, type, barrier, seeds, nseeds, d_match_out, rounds_out, nullptr, 0, st);
    set_error("mm_match_ex: unknown path");
    return MM_ERR_ARG;
}

MM_API mm_status mm_match_drawn(mm_graph *g, int type, uint32_t barrier, uint32_t (*draw)(void *), void *ctx,
                                int *d_match_out, int *rounds_out, void *stream)
{
    if (!draw) {
        set_error("mm_match_drawn: draw is null");
        return MM_ERR_ARG;
    }
    const uint32_t unused = 0;
    mm_status s = check_match_args(g, type, &unused, 1, d_match_out, rounds_out);
    if (s != MM_OK) return s;
    if (g->ngraphs > 0) {
        set_error("mm_match_drawn: matches single graphs only");
        return MM_ERR_UNSUPPORTED;
    }
    DeviceGuard guard(g->device);
    return pull_match(g, type, barrier, nullptr, 0, d_match_out, rounds_out, nullptr, 0, (cudaStream_t)stream, draw,
                      ctx);
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
    if (path == MM_PATH_PULL) {
        if (g->ngraphs > 0) {
            set_error("mm_match_stats: the reference-structured path matches single graphs only");
            return MM_ERR_UNSUPPORTED;
        }
        return pull_match(g, type, barrier, seeds, nseeds, d_match_out, rounds_out, stats, stats_rounds,
                          (cudaStream_t)stream);
    }
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

MM_API mm_status mm_match_policy(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                                 const float *mlp, float level, int *d_match_out, int *rounds_out, float *d_trace,
                                 int trace_rounds, void *stream)
{
    mm_status s = check_match_args(g, type, seeds, nseeds, d_match_out, rounds_out);
    if (s != MM_OK) return s;
    if (!mlp) {
        set_error("mm_match_policy: no policy weights");
        return MM_ERR_ARG;
    }
    if (trace_rounds < 0 || trace_rounds > mm::kMaxRounds) {
        set_error("mm_match_policy: trace_rounds must be in [0, 255]");
        return MM_ERR_ARG;
    }
    DeviceGuard guard(g->device);
    return push_match_policy(g, type, barrier, seeds, nseeds, mlp, level, d_match_out, rounds_out, d_trace,
                             trace_rounds, (cudaStream_t)stream);
}

MM_API mm_status mm_graph_set_batch(mm_graph *g, int ngraphs, const int *offsets)
{
    if (!g || ngraphs < 1 || !offsets) {
        set_error("mm_graph_set_batch: bad argument");
        return MM_ERR_ARG;
    }
    if (offsets[0] != 0 || offsets[ngraphs] != g->n) {
        set_error("mm_graph_set_batch: offsets must run from 0 to n");
        return MM_ERR_ARG;
    }
    for (int i = 0; i < ngraphs; ++i)
        if (offsets[i + 1] < offsets[i]) {
            set_error("mm_graph_set_batch: offsets must not decrease");
            return MM_ERR_ARG;
        }
    DeviceGuard guard(g->device);
    int *goff = nullptr, *vbase = nullptr, *vend = nullptr, *bad = nullptr;
    uint8_t *last = nullptr;
    const size_t nv = (size_t)(g->n > 0 ? g->n : 1);
    cudaError_t e = dev_alloc((void **)&goff, sizeof(int) * ((size_t)ngraphs + 1), 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&vbase, sizeof(int) * nv, 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&vend, sizeof(int) * nv, 0);  // for the check only
    if (e == cudaSuccess) e = dev_alloc((void **)&last, nv, 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&bad, sizeof(int), 0);
    if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int), 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(goff, offsets, sizeof(int) * ((size_t)ngraphs + 1), cudaMemcpyHostToDevice, 0);
    if (e == cudaSuccess) {
        k_batch_vbase<<<grid_for((long long)ngraphs * 32, 256, 148 * 8), 256>>>(goff, ngraphs, vbase, vend);
        if (g->n > 0)
            k_batch_edges<<<grid_for((long long)g->n, 256, 148 * 16), 256>>>(g->d_ranges, g->d_nbrs, vbase, vend,
                                                                           g->n, bad);
        e = cudaGetLastError();
    }
    int hbad = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost);
    dev_free(bad, 0);
    dev_free(vend, 0);
    if (e != cudaSuccess || hbad) {
        dev_free(goff, 0);
        dev_free(vbase, 0);
        dev_free(last, 0);
        cudaStreamSynchronize(0);
        if (e != cudaSuccess) return cuda_fail(e, "mm_graph_set_batch");
        set_error("mm_graph_set_batch: an edge joins two graphs of the batch");
        return MM_ERR_GRAPH;
    }
    dev_free(g->d_goff, 0);
    dev_free(g->d_vbase, 0);
    dev_free(g->d_last, 0);
    g->d_goff = goff;
    g->d_vbase = vbase;
    g->d_last = last;
    g->ngraphs = ngraphs;
    MM_CUDA_TRY(cudaStreamSynchronize(0), "mm_graph_set_batch");
    return MM_OK;
}

MM_API mm_status mm_match_batch(mm_graph *g, int type, uint32_t barrier, const uint32_t *seeds, int nseeds,
                                int *d_match_out, int *rounds_out, void *stream)
{
    if (g && g->ngraphs < 1) {
        set_error("mm_match_batch: the graph is not a batch (mm_graph_set_batch)");
        return MM_ERR_ARG;
    }
    int overall = 0;
    mm_status s = check_match_args(g, type, seeds, nseeds, d_match_out, rounds_out ? &overall : nullptr);
    if (s != MM_OK) return s;
    DeviceGuard guard(g->device);
    cudaStream_t st = (cudaStream_t)stream;
    s = push_match(g, type, barrier, seeds, nseeds, d_match_out, &overall, nullptr, 0, st);
    if (s == MM_OK) s = push_batch_rounds(g, type, rounds_out, st);
    return s;
}

MM_API const char *mm_last_error(void) { return g_last_error.c_str(); }

MM_API const char *mm_version(void) { return "mmatch 0.1 (sm_100a)"; }

MM_API mm_status mm_graph_tune(mm_graph *g, int key, int value)
{
    if (!g) {
        set_error("mm_graph_tune: null graph");
        return MM_ERR_ARG;
    }
    switch (key) {
    case MM_TUNE_FINISH_DIV:
        if (value < -1 || value == 1 || value > 1 << 20) break;
        g->opt_fin_div = value;
        return MM_OK;
    case MM_TUNE_BLOCKS_PER_SM:
        if (value < 0 || value > 64) break;
        g->opt_blocks_per_sm = value;
        return MM_OK;
    default:
        set_error("mm_graph_tune: unknown key");
        return MM_ERR_ARG;
    }
    set_error("mm_graph_tune: value out of range");
    return MM_ERR_ARG;
}

MM_API mm_status mm_debug(int key, long long value, long long *out)
{
    long long prev = 0;
    switch (key) {
    case MM_DEBUG_SPIN_LIMIT:
        prev = g_dbg_spin_limit.exchange(value < 0 ? 0 : value);
        break;
    case MM_DEBUG_SKIP_BARRIER:
        prev = g_dbg_skip_mark.exchange(value < 0 ? -1 : (int)value);
        break;
    case MM_DEBUG_ALLOC_LIMIT:
        prev = g_dbg_alloc_limit.exchange(value < 0 ? -1 : value);
        break;
    case MM_DEBUG_POOL_USED: {
        int device = -1;
        cudaMemPool_t pool = nullptr;
        MM_CUDA_TRY(cudaGetDevice(&device), "mm_debug: device");
        MM_CUDA_TRY(device_pool(device, &pool), "mm_debug: pool");
        MM_CUDA_TRY(cudaDeviceSynchronize(), "mm_debug: synchronise");
        uint64_t used = 0;
        MM_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used), "mm_debug: pool use");
        prev = (long long)used;
        break;
    }
    default:
        set_error("mm_debug: unknown key");
        return MM_ERR_ARG;
    }
    if (out) *out = prev;
    return MM_OK;
}

MM_API mm_status mm_probe_gather_rate(int device, long long table_bytes, double *gathers_per_s)
{
    if (!gathers_per_s || table_bytes < 1 || table_bytes > (1ll << 30)) {
        set_error("mm_probe_gather_rate: table_bytes must be in [1, 2^30] and the output non-null");
        return MM_ERR_ARG;
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (device >= 0) MM_CUDA_TRY(cudaSetDevice(device), "set device");
    const long long m = 1ll << 27;  // indices (512 MB, more than L2 holds)
    int *idx = nullptr;
    uint8_t *table = nullptr;
    unsigned *sink = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = dev_alloc((void **)&idx, sizeof(int) * (size_t)m, 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&table, (size_t)table_bytes, 0);
    if (e == cudaSuccess) e = dev_alloc((void **)&sink, sizeof(unsigned), 0);
    if (e == cudaSuccess) e = cudaMemsetAsync(table, 1, (size_t)table_bytes, 0);
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    int sms = 148;
    if (e == cudaSuccess) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        k_probe_indices<<<sms * 8, 256>>>(idx, m, (int)(table_bytes < (1ll << 31) ? table_bytes : (1ll << 31) - 1), 12345);
        e = cudaGetLastError();
    }
    float best = 1e30f;
    for (int rep = 0; e == cudaSuccess && rep < 4; ++rep) {
        cudaEventRecord(a, 0);
        k_probe_gather<<<sms * 8, 256>>>(idx, m, table, sink);
        cudaEventRecord(b, 0);
        e = cudaEventSynchronize(b);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        if (e == cudaSuccess && ms < best) best = ms;
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    dev_free(idx, 0);
    dev_free(table, 0);
    dev_free(sink, 0);
    cudaStreamSynchronize(0);
    if (prev >= 0 && device >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) return cuda_fail(e, "gather probe");
    *gathers_per_s = (double)m / (best * 1e-3);
    return MM_OK;
}

