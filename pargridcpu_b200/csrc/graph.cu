// Device residency: copies a host graph to the device and builds the
// node-major, slot-encoded CSR the kernels read (layout in device.h).
#include <cub/cub.cuh>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "device.h"

namespace fc {

static thread_local std::string g_last_err;

void set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
    char b[512];
    snprintf(b, sizeof(b), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    g_last_err = b;
}
const char* last_cuda_error() { return g_last_err.c_str(); }

bool cuda_available() {
    static int have = -1;
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if (have < 0) {
        int n = 0;
        have = (cudaGetDeviceCount(&n) == cudaSuccess && n > 0) ? 1 : 0;
        cudaGetLastError();
    }
    return have == 1;
}

// deg0[v*L + l] and the row length of every node, from per-layer offsets.
__global__ void k_degrees(const uint32_t* __restrict__ off, uint32_t n, uint32_t L,
                          uint32_t* __restrict__ deg0, uint32_t* __restrict__ rowlen) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        uint32_t sum = 0;
        for (uint32_t l = 0; l < L; l++) {
            const uint32_t* o = off + (uint64_t)l * (n + 1);
            uint32_t d = (uint32_t)(o[v + 1] - o[v]);
            deg0[(uint64_t)v * L + l] = d;
            sum += d;
        }
        rowlen[v] = sum;
    }
}

// One warp per node: copy its L layer rows into its node-major range as
// slots; the rows longer than ORDER_MIN_ROW are left to the ordering kernels.
__global__ void k_scatter(const uint32_t* __restrict__ off, const uint32_t* __restrict__ adj_in,
                          const uint32_t* __restrict__ node_ptr, uint32_t n, uint32_t L,
                          uint32_t* __restrict__ adj_out) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
        uint32_t dst = node_ptr[v];
        if (node_ptr[v + 1] - dst > ORDER_MIN_ROW) continue;  // written ordered (k_order_scatter)
        for (uint32_t l = 0; l < L; l++) {
            const uint32_t* o = off + (uint64_t)l * (n + 1);
            uint64_t b = o[v], e = o[v + 1];
            for (uint64_t j = b + lane; j < e; j += 32) adj_out[dst + (j - b)] = adj_in[j] * L + l;
            dst += (uint32_t)(e - b);
        }
    }
}

// The same for layers [l0, l1) only: a row's layer l starts after its
// layers below l (their degrees from deg0).  The upload scatters each group
// of layers as soon as its part of the input has arrived.
__global__ void k_scatter_layers(const uint32_t* __restrict__ off, const uint32_t* __restrict__ adj_in,
                                 const uint32_t* __restrict__ node_ptr,
                                 const uint32_t* __restrict__ deg0, uint32_t n, uint32_t L,
                                 uint32_t l0, uint32_t l1, uint32_t* __restrict__ adj_out) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
        uint32_t dst = node_ptr[v];
        if (node_ptr[v + 1] - dst > ORDER_MIN_ROW) continue;  // written ordered (k_order_scatter)
        for (uint32_t l = 0; l < l0; l++) dst += deg0[(uint64_t)v * L + l];
        for (uint32_t l = l0; l < l1; l++) {
            const uint32_t* o = off + (uint64_t)l * (n + 1);
            uint64_t b = o[v], e = o[v + 1];
            for (uint64_t j = b + lane; j < e; j += 32) adj_out[dst + (j - b)] = adj_in[j] * L + l;
            dst += (uint32_t)(e - b);
        }
    }
}

// ---- ordering of long rows by bound bucket (layout in device.h) ----------
// Each row longer than ORDER_MIN_ROW is cut into tiles of ORDER_TILE
// entries.  A tile's bucket histogram goes to hist at the row's base
// (first tile * BUCKETS) + (BUCKETS-1-b) * tiles + tile, so one exclusive scan
// over all rows lists, per row, the buckets highest first and each bucket's
// tiles in order: the scan minus its value at the row's base is where a
// tile's first entry of bucket b goes.  Entries keep their order within a
// bucket (a stable counting sort), so the layout is deterministic.
constexpr uint32_t ORDER_TILE = 1024;

// the bound of every node and, per row, whether it is ordered and its tiles
__global__ void k_order_flags(const uint32_t* __restrict__ deg0, const uint32_t* __restrict__ rowlen,
                              uint32_t n, uint32_t L, uint32_t* __restrict__ ub,
                              uint32_t* __restrict__ fbig, uint32_t* __restrict__ ftiles) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += gridDim.x * blockDim.x) {
        if (v == n) {
            fbig[n] = 0;
            ftiles[n] = 0;
            continue;
        }
        uint32_t m = 0;
        for (uint32_t l = 0; l < L; l++) m = max(m, deg0[(uint64_t)v * L + l]);
        ub[v] = m;
        const uint32_t len = rowlen[v];
        const bool big = len > ORDER_MIN_ROW;
        fbig[v] = big ? 1u : 0u;
        ftiles[v] = big ? (len + ORDER_TILE - 1) / ORDER_TILE : 0u;
    }
}

// big_id of every node; the node of every ordered row and of every tile
__global__ void k_order_index(const uint32_t* __restrict__ fbig, const uint32_t* __restrict__ bscan,
                              const uint32_t* __restrict__ tscan, uint32_t n,
                              uint32_t* __restrict__ big_id, uint32_t* __restrict__ big_v,
                              uint32_t* __restrict__ tile_row) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        if (!fbig[v]) {
            big_id[v] = NO_BIG_ROW;
            continue;
        }
        const uint32_t id = bscan[v];
        big_id[v] = id;
        big_v[id] = v;
        for (uint32_t t = tscan[v]; t < tscan[v + 1]; t++) tile_row[t] = v;
    }
}

// The entries of tile i of node v's row (row positions [i*ORDER_TILE, ...)),
// read from the per-layer input CSR: f(valid, lane's u, l) is called by the
// whole warp for 32 consecutive positions at a time, in row order; a call
// never spans two layers.
template <class F>
__device__ __forceinline__ void for_tile_entries(const uint32_t* __restrict__ off,
                                                 const uint32_t* __restrict__ adj_in,
                                                 const uint32_t* __restrict__ deg0, uint32_t n,
                                                 uint32_t L, uint32_t v, uint32_t len, uint32_t i,
                                                 F&& f) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t p0 = i * ORDER_TILE;
    const uint32_t p1 = min(len, p0 + ORDER_TILE);
    uint32_t s = 0;  // row position of layer l's first entry
    for (uint32_t l = 0; l < L && s < p1; l++) {
        const uint32_t d = deg0[(uint64_t)v * L + l];
        const uint32_t a = max(s, p0), b = min(s + d, p1);
        if (a < b) {
            const uint64_t ob = (uint64_t)off[(uint64_t)l * (n + 1) + v] - s;
            for (uint32_t p = a; p < b; p += 32) {
                const bool valid = p + lane < b;
                const uint32_t u = valid ? adj_in[ob + p + lane] : 0u;
                f(valid, u, l);
            }
        }
        s += d;
    }
}

// One warp per tile: its bucket histogram.
__global__ void k_order_hist(const uint32_t* __restrict__ off, const uint32_t* __restrict__ adj_in,
                             const uint32_t* __restrict__ deg0, const uint32_t* __restrict__ node_ptr,
                             uint32_t n, uint32_t L, const uint32_t* __restrict__ ub,
                             const uint32_t* __restrict__ tile_row, const uint32_t* __restrict__ tscan,
                             uint32_t ntiles, uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[8][BUCKETS];  // 256 threads
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += warps) {
        const uint32_t v = tile_row[t];
        const uint32_t t0 = tscan[v], nt = tscan[v + 1] - t0, i = t - t0;
        h[w][lane] = 0;
        h[w][lane + 32] = 0;
        __syncwarp();
        for_tile_entries(off, adj_in, deg0, n, L, v, node_ptr[v + 1] - node_ptr[v], i,
                         [&](bool valid, uint32_t u, uint32_t) {
                             if (valid) atomicAdd(&h[w][bucket_of(ub[u])], 1u);
                         });
        __syncwarp();
        const uint64_t base = (uint64_t)t0 * BUCKETS;
        for (uint32_t b = lane; b < BUCKETS; b += 32)
            hist[base + (uint64_t)(BUCKETS - 1 - b) * nt + i] = h[w][b];
        __syncwarp();
    }
}

// Per ordered row r and bucket b: entries of bucket >= b.
__global__ void k_order_ptab(const uint32_t* __restrict__ big_v, const uint32_t* __restrict__ tscan,
                             const uint32_t* __restrict__ G, uint32_t nbig, uint32_t* __restrict__ ptab) {
    const uint64_t total = (uint64_t)nbig * BUCKETS;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < total;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)(x / BUCKETS), b = (uint32_t)(x % BUCKETS);
        const uint32_t v = big_v[r];
        const uint32_t t0 = tscan[v], nt = tscan[v + 1] - t0;
        const uint64_t base = (uint64_t)t0 * BUCKETS;
        ptab[x] = G[base + (uint64_t)(BUCKETS - b) * nt] - G[base];
    }
}

// One warp per tile: its entries as slots to their ordered places in the
// row, ranked in row order within each bucket.
__global__ void k_order_scatter(const uint32_t* __restrict__ off, const uint32_t* __restrict__ adj_in,
                                const uint32_t* __restrict__ deg0, const uint32_t* __restrict__ node_ptr,
                                uint32_t n, uint32_t L, const uint32_t* __restrict__ ub,
                                const uint32_t* __restrict__ tile_row, const uint32_t* __restrict__ tscan,
                                const uint32_t* __restrict__ G, uint32_t ntiles,
                                uint32_t* __restrict__ adj) {
    __shared__ uint32_t cur[8][BUCKETS];  // 256 threads
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += warps) {
        const uint32_t v = tile_row[t];
        const uint32_t t0 = tscan[v], nt = tscan[v + 1] - t0, i = t - t0;
        const uint64_t base = (uint64_t)t0 * BUCKETS;
        const uint32_t g0 = G[base];
        for (uint32_t b = lane; b < BUCKETS; b += 32)
            cur[w][b] = G[base + (uint64_t)(BUCKETS - 1 - b) * nt + i] - g0;
        __syncwarp();
        const uint32_t rs = node_ptr[v];
        for_tile_entries(off, adj_in, deg0, n, L, v, node_ptr[v + 1] - rs, i,
                         [&](bool valid, uint32_t u, uint32_t l) {
                             const uint32_t mask = __ballot_sync(0xffffffffu, valid);
                             if (valid) {
                                 const uint32_t b = bucket_of(ub[u]);
                                 const uint32_t peers = __match_any_sync(mask, b);
                                 const uint32_t rank = __popc(peers & lt);
                                 adj[rs + cur[w][b] + rank] = u * L + l;
                                 __syncwarp(mask);
                                 if (rank == 0) cur[w][b] += __popc(peers);
                             }
                             __syncwarp();
                         });
        __syncwarp();
    }
}

__global__ void k_max(const uint32_t* __restrict__ a, uint64_t len, uint32_t* out) {
    uint32_t m = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len;
         i += (uint64_t)gridDim.x * blockDim.x)
        m = max(m, a[i]);
    m = __reduce_max_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

fc_status dev_alloc(void** p, size_t bytes, cudaStream_t s) {
    static std::mutex mu;
    static bool pool_set[64] = {};
    int dev = 0;
    FC_CUDA_TRY(cudaGetDevice(&dev));
    {
        std::lock_guard<std::mutex> lk(mu);
        if (dev < 64 && !pool_set[dev]) {
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
                uint64_t keep = ~0ull;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            }
            cudaGetLastError();
            pool_set[dev] = true;
        }
    }
    FC_CUDA_TRY(cudaMallocAsync(p, bytes ? bytes : 16, s));
    count_alloc();
    return FC_OK;
}

void dev_free(void* p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

// ---- host <-> device copies through a thread's pinned staging buffer ------
// A copy to or from pageable host memory goes through the driver's own
// staging, which copies from every thread share: a server lane's small
// read-back would wait behind another lane's read-back that waits for that
// lane's long kernel.  A thread that installs a pinned staging buffer (the
// server lanes) copies through it in pieces instead; other threads copy
// directly.

static thread_local Staging* t_staging = nullptr;

void set_thread_staging(Staging* st) { t_staging = st; }

fc_status to_host(void* h, const void* d, size_t bytes, cudaStream_t s) {
    if (!bytes) return FC_OK;
    Staging* st = t_staging;
    if (!st || !st->p) {
        FC_CUDA_TRY(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s));
        FC_CUDA_TRY(cudaStreamSynchronize(s));
        return FC_OK;
    }
    for (size_t off = 0; off < bytes; off += st->cap) {
        const size_t c = bytes - off < st->cap ? bytes - off : st->cap;
        FC_CUDA_TRY(cudaMemcpyAsync(st->p, (const char*)d + off, c, cudaMemcpyDeviceToHost, s));
        FC_CUDA_TRY(cudaStreamSynchronize(s));
        memcpy((char*)h + off, st->p, c);
    }
    return FC_OK;
}

fc_status to_device(void* d, const void* h, size_t bytes, cudaStream_t s) {
    if (!bytes) return FC_OK;
    Staging* st = t_staging;
    if (!st || !st->p) {
        FC_CUDA_TRY(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s));
        return FC_OK;
    }
    for (size_t off = 0; off < bytes; off += st->cap) {
        const size_t c = bytes - off < st->cap ? bytes - off : st->cap;
        memcpy(st->p, (const char*)h + off, c);
        FC_CUDA_TRY(cudaMemcpyAsync((char*)d + off, st->p, c, cudaMemcpyHostToDevice, s));
        FC_CUDA_TRY(cudaStreamSynchronize(s));  // before the buffer is written again
    }
    return FC_OK;
}

fc_status ensure_ws(DeviceGraph* d, size_t bytes, cudaStream_t s) {
    if (d->ws_bytes >= bytes) return FC_OK;
    dev_free(d->ws, s);
    d->ws = nullptr;
    d->ws_bytes = 0;
    size_t b = bytes + bytes / 8;
    FC_TRY(dev_alloc(&d->ws, b, s));
    d->ws_bytes = b;
    return FC_OK;
}

static int num_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

// Stream-ordered temporaries of one call, returned when it ends (on every path).
struct TempBufs {
    cudaStream_t s;
    void* p[12] = {};
    int k = 0;
    explicit TempBufs(cudaStream_t st) : s(st) {}
    ~TempBufs() {
        for (int i = 0; i < k; i++) cudaFreeAsync(p[i], s);
    }
    template <class T>
    cudaError_t alloc(T** out, size_t bytes) {
        *out = nullptr;
        if (k == 12) return cudaErrorMemoryAllocation;
        cudaError_t e = cudaMallocAsync((void**)out, bytes, s);
        if (e == cudaSuccess) {
            p[k++] = *out;
            count_alloc();
        }
        return e;
    }
};

// Writes the rows longer than ORDER_MIN_ROW, ordered by bound bucket, from
// the per-layer input CSR (off, adj_in), and builds big_id and ptab
// (device.h).
static fc_status order_rows(DeviceGraph* d, const uint32_t* rowlen, const uint32_t* off,
                            const uint32_t* adj_in, cudaStream_t s) {
    const uint32_t n = d->n, L = d->L;
    const int blocks = num_sms() * 8;
    TempBufs tb(s);
    uint32_t *ub, *fbig, *ftiles, *bscan, *tscan;
    FC_CUDA_TRY(tb.alloc(&ub, (uint64_t)n * 4 + 4));
    FC_CUDA_TRY(tb.alloc(&fbig, ((uint64_t)n + 1) * 4));
    FC_CUDA_TRY(tb.alloc(&ftiles, ((uint64_t)n + 1) * 4));
    FC_CUDA_TRY(tb.alloc(&bscan, ((uint64_t)n + 1) * 4));
    FC_CUDA_TRY(tb.alloc(&tscan, ((uint64_t)n + 1) * 4));
    k_order_flags<<<blocks, 256, 0, s>>>(d->deg0, rowlen, n, L, ub, fbig, ftiles);
    count_launch();
    FC_CUDA_TRY(cudaGetLastError());
    size_t tmp_bytes = 0;
    FC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, fbig, bscan, n + 1, s));
    void* tmp;
    FC_CUDA_TRY(tb.alloc(&tmp, tmp_bytes + 16));
    FC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, fbig, bscan, n + 1, s));
    FC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, ftiles, tscan, n + 1, s));
    uint32_t nbig = 0, ntiles = 0;
    FC_TRY(to_host(&nbig, bscan + n, 4, s));
    FC_TRY(to_host(&ntiles, tscan + n, 4, s));
    if (!nbig) return FC_OK;
    FC_TRY(dev_alloc((void**)&d->big_id, (uint64_t)n * 4 + 4, s));
    FC_TRY(dev_alloc((void**)&d->ptab, (uint64_t)nbig * BUCKETS * 4, s));
    d->nbig = nbig;
    d->bytes += (uint64_t)n * 4 + (uint64_t)nbig * BUCKETS * 4;
    const uint64_t hwords = (uint64_t)ntiles * BUCKETS + 1;
    if (hwords >= (1ull << 31)) return FC_ERR_TOO_LARGE;
    uint32_t *big_v, *tile_row, *hist, *G;
    FC_CUDA_TRY(tb.alloc(&big_v, (uint64_t)nbig * 4));
    FC_CUDA_TRY(tb.alloc(&tile_row, (uint64_t)ntiles * 4));
    FC_CUDA_TRY(tb.alloc(&hist, hwords * 4));
    FC_CUDA_TRY(tb.alloc(&G, hwords * 4));
    k_order_index<<<blocks, 256, 0, s>>>(fbig, bscan, tscan, n, d->big_id, big_v, tile_row);
    FC_CUDA_TRY(cudaGetLastError());
    FC_CUDA_TRY(cudaMemsetAsync(hist + hwords - 1, 0, 4, s));
    k_order_hist<<<blocks, 256, 0, s>>>(off, adj_in, d->deg0, d->node_ptr, n, L, ub, tile_row, tscan,
                                        ntiles, hist);
    FC_CUDA_TRY(cudaGetLastError());
    size_t tmp2 = 0;
    FC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp2, hist, G, (int)hwords, s));
    if (tmp2 > tmp_bytes) FC_CUDA_TRY(tb.alloc(&tmp, tmp2 + 16));
    FC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp2, hist, G, (int)hwords, s));
    k_order_ptab<<<blocks, 256, 0, s>>>(big_v, tscan, G, nbig, d->ptab);
    FC_CUDA_TRY(cudaGetLastError());
    k_order_scatter<<<blocks, 256, 0, s>>>(off, adj_in, d->deg0, d->node_ptr, n, L, ub, tile_row,
                                           tscan, G, ntiles, d->adj);
    count_launch(4);
    FC_CUDA_TRY(cudaGetLastError());
    return FC_OK;
}

// Library-owned streams, one of each kind per device (made once): the copy
// stream of the upload pipeline, and the stream a released graph's memory is
// freed on.
enum SideStream { SIDE_COPY = 0, SIDE_RELEASE = 1 };

static cudaStream_t side_stream(SideStream kind) {
    static std::mutex mu;
    static cudaStream_t cs[2][64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    cudaStream_t& st = cs[kind][dev];
    if (!st) {
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            st = nullptr;
        } else {
            count_alloc();
        }
    }
    return st;
}

static cudaStream_t upload_copy_stream() { return side_stream(SIDE_COPY); }
cudaStream_t library_copy_stream() { return side_stream(SIDE_COPY); }

// Groups of layers (at most MAX_GROUPS, about equal in entries) whose input
// adjacency is copied on the copy stream, one cudaMemcpyAsync and one event
// per group; `ev[i]` marks group i's arrival.
struct UploadPipe {
    static constexpr uint32_t MAX_GROUPS = 8;
    cudaStream_t cs = nullptr;
    cudaEvent_t start = nullptr;
    cudaEvent_t ev[MAX_GROUPS] = {};
    uint32_t l0[MAX_GROUPS + 1] = {};
    uint32_t groups = 0;
    ~UploadPipe() {
        if (start) cudaEventDestroy(start);
        for (uint32_t i = 0; i < groups; i++)
            if (ev[i]) cudaEventDestroy(ev[i]);
    }
    // the groups, or 0 when the pipeline cannot be set up (one copy then)
    uint32_t plan(const fc_graph* g, cudaStream_t s) {
        const char* e = getenv("FC_UPLOAD_PIPE");  // 0: one copy, no pipeline
        if (e && *e == '0') return 0;
        cs = upload_copy_stream();
        if (!cs || cs == s) return 0;
        const uint32_t L = g->L, n = g->n;
        const uint64_t total = g->total_entries();
        uint32_t k = 0;
        l0[0] = 0;
        for (uint32_t l = 0; l < L && k < MAX_GROUPS; l++) {
            // close a group once it holds its share of the entries
            const uint64_t upto = g->off[(uint64_t)l * (n + 1) + n];
            const bool last = l + 1 == L;
            if (last || upto * MAX_GROUPS >= total * (k + 1)) l0[++k] = l + 1;
        }
        if (k == 0) return 0;
        l0[k] = L;  // the last group takes any layers left
        if (cudaEventCreateWithFlags(&start, cudaEventDisableTiming) != cudaSuccess) return 0;
        for (uint32_t i = 0; i < k; i++)
            if (cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) {
                groups = i;
                cudaGetLastError();
                return 0;
            }
        count_alloc(k + 1);
        groups = k;
        return k;
    }
    // the copies: after the buffers allocated on s exist
    fc_status copy(const fc_graph* g, uint32_t* d_in, cudaStream_t s) {
        const uint32_t n = g->n;
        FC_CUDA_TRY(cudaEventRecord(start, s));
        FC_CUDA_TRY(cudaStreamWaitEvent(cs, start, 0));
        for (uint32_t i = 0; i < groups; i++) {
            const uint64_t b = g->off[(uint64_t)l0[i] * (n + 1)];
            const uint64_t e = g->off[(uint64_t)(l0[i + 1] - 1) * (n + 1) + n];
            if (e > b)
                FC_CUDA_TRY(cudaMemcpyAsync(d_in + b, g->adj.p + b, (e - b) * 4,
                                            cudaMemcpyHostToDevice, cs));
            FC_CUDA_TRY(cudaEventRecord(ev[i], cs));
        }
        return FC_OK;
    }
};

fc_status upload(fc_graph* g, cudaStream_t s) {
    if (!cuda_available()) return FC_ERR_NO_DEVICE;
    if (g->dev) return FC_OK;
    uint32_t n = g->n, L = g->L;
    uint64_t entries = g->total_entries();
    if ((uint64_t)n * L >= (1ull << 32) || entries >= (1ull << 32)) return FC_ERR_TOO_LARGE;
    DeviceGraph* d = new DeviceGraph();
    FC_CUDA_TRY(cudaGetDevice(&d->device));
    d->n = n;
    d->L = L;
    d->entries = entries;
    d->home = s;
    g->dev = d;
    uint64_t noff = (uint64_t)L * (n + 1);
    uint32_t* d_off = nullptr;
    uint32_t* d_in = nullptr;
    uint32_t* rowlen = nullptr;
    uint32_t* d_max = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    FC_CUDA_TRY(cudaMallocAsync(&d_off, noff * 4 + 4, s));
    FC_CUDA_TRY(cudaMallocAsync(&d_in, entries * 4 + 4, s));
    FC_CUDA_TRY(cudaMallocAsync(&rowlen, (uint64_t)n * 4 + 4, s));
    FC_CUDA_TRY(cudaMallocAsync(&d_max, 8, s));
    count_alloc(4);
    FC_TRY(dev_alloc((void**)&d->node_ptr, ((uint64_t)n + 1) * 4, s));
    FC_TRY(dev_alloc((void**)&d->adj, entries * 4 + 4, s));
    FC_TRY(dev_alloc((void**)&d->deg0, (uint64_t)n * L * 4 + 4, s));
    FC_TRY(dev_alloc((void**)&d->table, (uint64_t)n * L * 4 + 4, s));
    d->bytes = ((uint64_t)n + 1) * 4 + entries * 4 + 2ull * n * L * 4;
    // The adjacency goes over in groups of layers on a copy stream while this
    // stream copies the offsets and builds the degrees and row pointers; each
    // group is scattered into the node-major rows once it has arrived.
    UploadPipe pipe;
    const uint32_t ngroups = entries && n ? pipe.plan(g, s) : 0u;
    if (noff) FC_CUDA_TRY(cudaMemcpyAsync(d_off, g->off.p, noff * 4, cudaMemcpyHostToDevice, s));
    if (ngroups) {
        FC_TRY(pipe.copy(g, d_in, s));
    } else if (entries) {
        FC_CUDA_TRY(cudaMemcpyAsync(d_in, g->adj.p, entries * 4, cudaMemcpyHostToDevice, s));
    }
    FC_CUDA_TRY(cudaMemsetAsync(d_max, 0, 8, s));
    int blocks = num_sms() * 8;
    if (n) {
        k_degrees<<<blocks, 256, 0, s>>>(d_off, n, L, d->deg0, rowlen);
        FC_CUDA_TRY(cudaGetLastError());
        FC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, rowlen, d->node_ptr, n + 1, s));
        FC_CUDA_TRY(cudaMallocAsync(&tmp, tmp_bytes + 16, s));
        count_alloc();
        // rowlen has n entries; entry n of the scan input must be 0
        FC_CUDA_TRY(cudaMemsetAsync(rowlen + n, 0, 4, s));
        FC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, rowlen, d->node_ptr, n + 1, s));
        k_max<<<blocks, 256, 0, s>>>(d->deg0, (uint64_t)n * L, d_max);
        k_max<<<blocks, 256, 0, s>>>(rowlen, n, d_max + 1);
        count_launch(2);
        if (ngroups) {
            for (uint32_t i = 0; i < ngroups; i++) {
                FC_CUDA_TRY(cudaStreamWaitEvent(s, pipe.ev[i], 0));
                k_scatter_layers<<<blocks, 256, 0, s>>>(d_off, d_in, d->node_ptr, d->deg0, n, L,
                                                        pipe.l0[i], pipe.l0[i + 1], d->adj);
                count_launch();
            }
        } else {
            k_scatter<<<blocks, 256, 0, s>>>(d_off, d_in, d->node_ptr, n, L, d->adj);
            count_launch();
        }
        FC_CUDA_TRY(cudaGetLastError());
        FC_TRY(order_rows(d, rowlen, d_off, d_in, s));
    }
    uint32_t mx[2] = {0, 0};
    FC_TRY(to_host(mx, d_max, 8, s));
    if (tmp) FC_CUDA_TRY(cudaFreeAsync(tmp, s));
    FC_CUDA_TRY(cudaFreeAsync(d_off, s));
    FC_CUDA_TRY(cudaFreeAsync(d_in, s));
    FC_CUDA_TRY(cudaFreeAsync(rowlen, s));
    FC_CUDA_TRY(cudaFreeAsync(d_max, s));
    FC_CUDA_TRY(cudaStreamSynchronize(s));
    d->home = nullptr;
    d->max_deg = mx[0];
    d->max_row = mx[1];
    return FC_OK;
}

void release_device(fc_graph* g, bool wait_home) {
    DeviceGraph* d = g->dev;
    if (!d) return;
    residency_forget(g);
    int cur = -1;
    cudaGetDevice(&cur);
    if (d->device >= 0 && d->device != cur) cudaSetDevice(d->device);
    // the last call's work is done before its memory returns to the pool:
    // a call that left work in flight recorded its stream; one that finished
    // with a synchronize did not (that stream may already be destroyed)
    if (wait_home && d->home) cudaStreamSynchronize(d->home);
    cudaGetLastError();
    // The frees go on the library's release stream (the legacy stream when
    // it cannot be made), which outlives any caller stream, and that stream
    // is synchronized: the pool hands memory freed on one stream to an
    // allocation on another only once the free is known to be complete, so
    // an upload right after a release reuses the blocks instead of growing
    // the pool (which cost up to 30 ms in a step).
    cudaStream_t rs = side_stream(SIDE_RELEASE);
    free_densest_state(d, rs);
    free_cell_index(d, rs);
    dev_free(d->node_ptr, rs);
    dev_free(d->adj, rs);
    dev_free(d->deg0, rs);
    dev_free(d->big_id, rs);
    dev_free(d->ptab, rs);
    dev_free(d->table, rs);
    dev_free(d->ws, rs);
    cudaStreamSynchronize(rs);
    cudaGetLastError();
    if (cur >= 0 && d->device != cur) cudaSetDevice(cur);
    delete d;
    g->dev = nullptr;
}

uint64_t device_bytes(const fc_graph* g) {
    if (!g->dev) return 0;
    return g->dev->bytes + g->dev->ws_bytes;
}

// Kernels load on first use unless loaded before, and a load may wait for
// the kernels already running on the device: a server lane's first batch of
// a new kind would wait for another lane's batch.  This loads every kernel
// of the library (the scan of the CSR build by running it once on a few
// words) on the current device, once.
void preload_kernels() {
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lk(mu);
    if (done[dev]) return;
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, k_degrees);
    cudaFuncGetAttributes(&a, k_scatter);
    cudaFuncGetAttributes(&a, k_scatter_layers);
    cudaFuncGetAttributes(&a, k_max);
    cudaFuncGetAttributes(&a, k_order_flags);
    cudaFuncGetAttributes(&a, k_order_index);
    cudaFuncGetAttributes(&a, k_order_hist);
    cudaFuncGetAttributes(&a, k_order_ptab);
    cudaFuncGetAttributes(&a, k_order_scatter);
    peel_preload();
    densest_preload();
    uint32_t* buf = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    if (cudaMalloc(&buf, 64) == cudaSuccess &&
        cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, buf, buf + 8, 8, (cudaStream_t)0) ==
            cudaSuccess &&
        cudaMalloc(&tmp, tmp_bytes + 16) == cudaSuccess) {
        count_alloc(2);
        cudaMemset(buf, 0, 64);
        cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, buf, buf + 8, 8, (cudaStream_t)0);
        cudaDeviceSynchronize();
    }
    if (tmp) cudaFree(tmp);
    if (buf) cudaFree(buf);
    cudaGetLastError();
    done[dev] = true;
}

}  // namespace fc
