// Device residency: copies a host graph to the device and builds the
// node-major, slot-encoded CSR the kernels read (layout in device.h).
#include <cub/cub.cuh>

#include <cstdio>
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
__global__ void k_degrees(const uint64_t* __restrict__ off, uint32_t n, uint32_t L,
                          uint32_t* __restrict__ deg0, uint32_t* __restrict__ rowlen) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        uint32_t sum = 0;
        for (uint32_t l = 0; l < L; l++) {
            const uint64_t* o = off + (uint64_t)l * (n + 1);
            uint32_t d = (uint32_t)(o[v + 1] - o[v]);
            deg0[(uint64_t)v * L + l] = d;
            sum += d;
        }
        rowlen[v] = sum;
    }
}

// One warp per node: copy its L layer rows into its node-major range as slots.
__global__ void k_scatter(const uint64_t* __restrict__ off, const uint32_t* __restrict__ adj_in,
                          const uint32_t* __restrict__ node_ptr, uint32_t n, uint32_t L,
                          uint32_t* __restrict__ adj_out) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
        uint32_t dst = node_ptr[v];
        for (uint32_t l = 0; l < L; l++) {
            const uint64_t* o = off + (uint64_t)l * (n + 1);
            uint64_t b = o[v], e = o[v + 1];
            for (uint64_t j = b + lane; j < e; j += 32) adj_out[dst + (j - b)] = adj_in[j] * L + l;
            dst += (uint32_t)(e - b);
        }
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
    uint64_t* d_off = nullptr;
    uint32_t* d_in = nullptr;
    uint32_t* rowlen = nullptr;
    uint32_t* d_max = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    FC_CUDA_TRY(cudaMallocAsync(&d_off, noff * 8 + 8, s));
    FC_CUDA_TRY(cudaMallocAsync(&d_in, entries * 4 + 4, s));
    FC_CUDA_TRY(cudaMallocAsync(&rowlen, (uint64_t)n * 4 + 4, s));
    FC_CUDA_TRY(cudaMallocAsync(&d_max, 8, s));
    FC_TRY(dev_alloc((void**)&d->node_ptr, ((uint64_t)n + 1) * 4, s));
    FC_TRY(dev_alloc((void**)&d->adj, entries * 4 + 4, s));
    FC_TRY(dev_alloc((void**)&d->deg0, (uint64_t)n * L * 4 + 4, s));
    FC_TRY(dev_alloc((void**)&d->table, (uint64_t)n * L * 4 + 4, s));
    d->bytes = ((uint64_t)n + 1) * 4 + entries * 4 + 2ull * n * L * 4;
    if (noff) FC_CUDA_TRY(cudaMemcpyAsync(d_off, g->off.p, noff * 8, cudaMemcpyHostToDevice, s));
    if (entries) FC_CUDA_TRY(cudaMemcpyAsync(d_in, g->adj.p, entries * 4, cudaMemcpyHostToDevice, s));
    FC_CUDA_TRY(cudaMemsetAsync(d_max, 0, 8, s));
    int blocks = num_sms() * 8;
    if (n) {
        k_degrees<<<blocks, 256, 0, s>>>(d_off, n, L, d->deg0, rowlen);
        FC_CUDA_TRY(cudaGetLastError());
        FC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, rowlen, d->node_ptr, n + 1, s));
        FC_CUDA_TRY(cudaMallocAsync(&tmp, tmp_bytes + 16, s));
        // rowlen has n entries; entry n of the scan input must be 0
        FC_CUDA_TRY(cudaMemsetAsync(rowlen + n, 0, 4, s));
        FC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, rowlen, d->node_ptr, n + 1, s));
        k_scatter<<<blocks, 256, 0, s>>>(d_off, d_in, d->node_ptr, n, L, d->adj);
        FC_CUDA_TRY(cudaGetLastError());
        k_max<<<blocks, 256, 0, s>>>(d->deg0, (uint64_t)n * L, d_max);
        k_max<<<blocks, 256, 0, s>>>(rowlen, n, d_max + 1);
        count_launch(4);
        FC_CUDA_TRY(cudaGetLastError());
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
    // the last call's work is done before its memory returns to the pool;
    // the frees go on the legacy stream, which outlives any caller stream
    // a call that left work in flight recorded its stream; one that finished
    // with a synchronize did not (that stream may already be destroyed)
    if (wait_home && d->home) cudaStreamSynchronize(d->home);
    cudaGetLastError();
    free_densest_state(d);
    dev_free(d->node_ptr, 0);
    dev_free(d->adj, 0);
    dev_free(d->deg0, 0);
    dev_free(d->table, 0);
    dev_free(d->ws, 0);
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
    cudaFuncGetAttributes(&a, k_max);
    peel_preload();
    densest_preload();
    uint32_t* buf = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    if (cudaMalloc(&buf, 64) == cudaSuccess &&
        cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, buf, buf + 8, 8, (cudaStream_t)0) ==
            cudaSuccess &&
        cudaMalloc(&tmp, tmp_bytes + 16) == cudaSuccess) {
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
