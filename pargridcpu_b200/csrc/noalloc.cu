// fc_coreindex_fixed_scratch: the core-index peel for callers that cannot
// allocate device memory.
//
// Some callers must not call cudaMalloc (or anything that does): an
// application whose memory manager reserved the whole device up front and
// hands out nothing more, or a latency-bound loop that cannot afford a device
// allocation, which may synchronise the device and stall every stream.  This
// entry point takes the graph and the output table in device memory the
// caller already owns and runs the same peel kernel as fc_coreindex with its
// scratch carved from one fixed array in this file, FC_FIXED_SCRATCH_BYTES
// (64 MiB), which every GPU that loads this module holds until the process
// exits.  It allocates nothing itself.
//
// Set-up: the first call on a device looks the array's device address up
// with that device current (cudaGetSymbolAddress); make that first call before
// any stream capture.  All calls share the one array and it keeps the last
// call's contents: each call clears what must start empty (queues, control
// block) before its kernel runs, and calls that overlap on the GPU -- on two
// streams, or from two host threads -- race on it.
//
// The caller's CSR is checked before the peel reads it: node_ptr must start
// at 0, never decrease and end at `entries`, and every slot must name one of
// the n*L degree counters.  Those are the properties the peel's indexing
// rests on; a violation ends the call with FC_ERR_INVALID.  The check's flag
// is the last word of the array, outside the peel's scratch.
#include <mutex>

#include "device.h"

namespace fc {

constexpr size_t FIXED_SCRATCH_BYTES = 64ull << 20;
// the peel's part; the last 256 bytes hold the input check's flag
constexpr size_t PEEL_SCRATCH_BYTES = FIXED_SCRATCH_BYTES - 256;

// The scratch itself.  In host code this name is a host-side stand-in, not a
// device address: kernels are given the address from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_fixed_scratch[FIXED_SCRATCH_BYTES];

static std::mutex g_fixed_mu;
static void* g_fixed_addr[64];  // per device

// Device address of the fixed scratch on the current device (looked up once).
static fc_status fixed_scratch(void** out) {
    int dev = 0;
    FC_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return FC_ERR_DEVICE;
    std::lock_guard<std::mutex> lk(g_fixed_mu);
    if (!g_fixed_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_fixed_scratch);
        if (e != cudaSuccess || !p) {
            set_last_cuda_error(e, "cudaGetSymbolAddress(g_fixed_scratch)", __FILE__, __LINE__);
            return FC_ERR_DEVICE;
        }
        g_fixed_addr[dev] = p;
    }
    *out = g_fixed_addr[dev];
    return FC_OK;
}

// Bounded input check (grid-stride, no waits): sets *bad when node_ptr does
// not start at 0, decreases or does not end at `entries`, or a slot is not
// below nL.
__global__ void k_check_csr(const uint32_t* __restrict__ node_ptr, uint32_t n,
                            const uint32_t* __restrict__ adj, uint64_t entries, uint64_t nL,
                            uint32_t* __restrict__ bad) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint32_t b = 0;
    if (t == 0 && (node_ptr[0] != 0 || node_ptr[n] != entries)) b = 1;
    for (uint64_t v = t; v < n; v += stride)
        if (node_ptr[v + 1] < node_ptr[v]) b = 1;
    for (uint64_t e = t; e < entries; e += stride)
        if (adj[e] >= nL) b = 1;
    if (__any_sync(0xffffffffu, b) && (threadIdx.x & 31) == 0) atomicOr(bad, 1u);
}

}  // namespace fc

using namespace fc;

extern "C" fc_status fc_coreindex_fixed_scratch(uint32_t n, uint32_t n_layers, uint64_t entries,
                                                const uint32_t* node_ptr, const uint32_t* adj,
                                                const uint32_t* deg0, uint32_t* table,
                                                void* stream) {
    if (!cuda_available()) return FC_ERR_NO_DEVICE;
    if (n == 0 || n_layers == 0) return FC_OK;
    if (!node_ptr || !deg0 || !table || (entries && !adj)) return FC_ERR_INVALID;
    if ((uint64_t)n * n_layers >= (1ull << 32) || entries >= (1ull << 32)) return FC_ERR_TOO_LARGE;
    // the most columns per launch whose scratch fits the fixed array; a graph
    // whose single column does not fit is rejected before any device work
    uint32_t cols = n_layers;
    while (cols > 0 && peel_ws_bytes(n, n_layers, entries, cols) > PEEL_SCRATCH_BYTES) cols--;
    if (cols == 0) return FC_ERR_TOO_LARGE;
    void* ws = nullptr;
    FC_TRY(fixed_scratch(&ws));
    cudaStream_t s = (cudaStream_t)stream;
    {
        uint32_t* bad = (uint32_t*)((char*)ws + PEEL_SCRATCH_BYTES);
        FC_CUDA_TRY(cudaMemsetAsync(bad, 0, 4, s));
        int dev = 0, sms = 0;
        FC_CUDA_TRY(cudaGetDevice(&dev));
        FC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        k_check_csr<<<sms * 4, 256, 0, s>>>(node_ptr, n, adj, entries, (uint64_t)n * n_layers, bad);
        count_launch();
        FC_CUDA_TRY(cudaGetLastError());
        uint32_t flag = 0;
        FC_TRY(to_host(&flag, bad, 4, s));
        if (flag) return FC_ERR_INVALID;
    }
    // core <= largest degree <= n - 1 bounds the level count
    PeelGraph g{n, n_layers, entries, node_ptr, adj, deg0, n + 1};
    for (uint32_t c0 = 0; c0 < n_layers; c0 += cols) {
        const uint32_t nc = n_layers - c0 < cols ? n_layers - c0 : cols;
        PeelStats st;
        FC_TRY(peel_run(g, c0, nc, table, ws, PEEL_SCRATCH_BYTES, s, &st, false, false));
    }
    return FC_OK;
}
