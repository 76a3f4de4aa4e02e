// Device-side layout shared by the kernels.
//
// A graph on the device is node-major:
//   node_ptr[v] .. node_ptr[v+1]   all of v's adjacency, layer 0 first
//   adj[e] = u * L + l              a "slot": neighbour u in layer l; it is
//                                   also the index of deg[u][l] in an n*L
//                                   degree table, so one 4-byte load per edge
//                                   names both the neighbour and the counter
//                                   to decrement
//   deg0[v * L + l] = |N_l(v)|      the full per-layer degrees
// Core tables are lambda-major: table[(lambda-1) * n + v].
//
// Rows longer than ORDER_MIN_ROW entries are ordered by bound bucket,
// highest first: the bound of neighbour u is its largest layer degree, which
// is at least core_lambda(u) for every lambda, so at level K every entry
// whose bound is below K names a removed node.  For such a row,
// ptab[big_id[v] * BUCKETS + b] counts its entries of bucket >= b, and a
// removal at level K needs only the chunks covering the first
// ptab[.. + bucket_of(K)] entries.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "fc_internal.h"

namespace fc {

// Division by a run-time constant d >= 1 for 32-bit x by multiply and shifts
// (Granlund & Montgomery, "Division by invariant integers using
// multiplication", 1994, round-up variant):
//   l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1,
//   q = (t + ((x - t) >> min(l,1))) >> max(l-1,0), t = umulhi(m, x).
struct FastDiv {
    uint32_t d, m, s1, s2;
    void init(uint32_t dd) {
        d = dd;
        uint32_t l = 0;
        while ((1ull << l) < dd) l++;
        m = (uint32_t)((((1ull << 32) * ((1ull << l) - dd)) / dd) + 1);
        s1 = l < 1 ? l : 1;
        s2 = l > 1 ? l - 1 : 0;
    }
    __host__ __device__ __forceinline__ uint32_t div(uint32_t x) const {
#ifdef __CUDA_ARCH__
        uint32_t t = __umulhi(x, m);
#else
        uint32_t t = (uint32_t)(((uint64_t)x * m) >> 32);
#endif
        return (t + ((x - t) >> s1)) >> s2;
    }
};

// Bound buckets: 0..15 hold the values 0..15, buckets 16..63 eight per
// octave from 16 (lower ends 16 * 2^(i/8), rounded down); bucket 63 is
// unbounded above.
constexpr uint32_t BUCKETS = 64;
constexpr uint32_t ORDER_MIN_ROW = 256;
constexpr uint32_t NO_BIG_ROW = 0xFFFFFFFFu;
__host__ __device__ __forceinline__ uint32_t bucket_lo(uint32_t b) {
    if (b < 16) return b;
    const uint32_t t = b - 16;
    // 256 * 2^(i/8), i = 0..7, rounded down
    const uint32_t f = t & 7;
    const uint32_t frac = f == 0 ? 256u : f == 1 ? 279u : f == 2 ? 304u : f == 3 ? 331u
                        : f == 4 ? 362u : f == 5 ? 394u : f == 6 ? 430u : 469u;
    return ((16u << (t >> 3)) * frac) >> 8;
}
// the bucket holding value x: the largest b with bucket_lo(b) <= x
__host__ __device__ __forceinline__ uint32_t bucket_of(uint32_t x) {
    if (x < 16) return x;
    uint32_t lo = 16, hi = BUCKETS - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (bucket_lo(mid) <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

struct DeviceGraph {
    int device = -1;
    uint32_t n = 0, L = 0;
    uint64_t entries = 0;      // directed adjacency entries over all layers
    uint32_t max_deg = 0;      // largest single-layer degree
    uint32_t max_row = 0;      // largest node adjacency over all layers
    uint32_t* node_ptr = nullptr;  // n + 1
    uint32_t* adj = nullptr;       // entries (slots)
    uint32_t* deg0 = nullptr;      // n * L
    // ordered long rows: big_id[v] (NO_BIG_ROW for other rows), BUCKETS counts each
    uint32_t* big_id = nullptr;    // n
    uint32_t* ptab = nullptr;      // nbig * BUCKETS
    uint32_t nbig = 0;
    // resident results
    uint32_t* table = nullptr;     // L * n, lambda-major
    bool table_valid = false;
    // when the table is not all valid: columns [cols_lo, cols_hi) are
    // (fc_coreindex_range); an empty range when none
    uint32_t cols_lo = 0, cols_hi = 0;
    std::vector<uint32_t> kmax;    // per lambda, max core (host copy)
    // densest state for the resident table (histograms, cell records)
    void* dens = nullptr;
    // the cell index of the resident table (cellindex.cu)
    void* cidx = nullptr;
    // reusable scratch
    void* ws = nullptr;
    size_t ws_bytes = 0;
    uint64_t bytes = 0;            // CSR + table
    fc_stats stats{};              // diagnostics of the last computations
    cudaStream_t home = nullptr;   // stream that may still run work on it (nullptr: none)
};

// Device memory from the device's stream-ordered pool, which keeps freed
// memory for reuse (release threshold raised once per device), so that
// dropping and re-uploading a graph does not return to the driver.
fc_status dev_alloc(void** p, size_t bytes, cudaStream_t s);
void dev_free(void* p, cudaStream_t s);

// A pinned host buffer a thread copies through (set_thread_staging); the
// server lanes install one so that their copies do not queue behind other
// threads' copies to pageable memory.
struct Staging {
    void* p = nullptr;
    size_t cap = 0;
};
void set_thread_staging(Staging* st);
// device -> host, waits for the copy; host -> device, waits only when staged
fc_status to_host(void* h, const void* d, size_t bytes, cudaStream_t s);
fc_status to_device(void* d, const void* h, size_t bytes, cudaStream_t s);
// the library's copy stream of the current device (made once; null when it
// cannot be made)
cudaStream_t library_copy_stream();

// kernels launched by this library (fc_launch_count)
void count_launch(uint32_t k = 1);

// scratch owned by a DeviceGraph, grown on demand
fc_status ensure_ws(DeviceGraph* d, size_t bytes, cudaStream_t s);
// the frees go on stream s, with the graph's work finished
void free_densest_state(DeviceGraph* d, cudaStream_t s = 0);
void invalidate_densest(DeviceGraph* d);
// cellindex.cu: the resident cell index goes with the table it was built from
void free_cell_index(DeviceGraph* d, cudaStream_t s = 0);
void invalidate_cell_index(DeviceGraph* d);

// peel.cu
struct PeelStats {
    uint32_t levels = 0, subrounds = 0, err = 0;
    double ms = 0;  // CUDA-event time of the launch
    double phase_ms[3] = {0, 0, 0};  // scan, expand, recompute (device timer)
};
fc_status peel_columns(DeviceGraph* d, uint32_t col0, uint32_t ncols, cudaStream_t s,
                       PeelStats* st);
uint32_t peel_columns_per_group(const DeviceGraph* d);

// A device-resident graph in the kernels' layout, whoever owns the memory.
struct PeelGraph {
    uint32_t n, L;
    uint64_t entries;
    const uint32_t* node_ptr;
    const uint32_t* adj;
    const uint32_t* deg0;
    uint32_t max_level;  // bound on the level count (largest degree + 1, or n + 1)
    // ordered long rows (both null when the rows are in any order)
    const uint32_t* big_id = nullptr;
    const uint32_t* ptab = nullptr;
};
// scratch bytes one peel launch over `ncols` columns needs
uint64_t peel_ws_bytes(uint32_t n, uint32_t L, uint64_t entries, uint32_t ncols);
// columns [col0, col0 + ncols) of `table` (lambda-major), scratch in `ws`;
// allocates nothing unless `instrument` (events; a trace when FC_PEEL_TRACE)
// or `endgame` (the last levels in one block per column; a temporary buffer
// when the survivors' subgraphs outgrow the spent queues)
fc_status peel_run(const PeelGraph& g, uint32_t col0, uint32_t ncols, uint32_t* table, void* ws,
                   size_t ws_bytes, cudaStream_t s, PeelStats* st, bool instrument, bool endgame);

// One segment of a batched launch: columns [col0, col0 + ncols) of graph g,
// written to table (lambda-major, L*n).
struct PeelSegSpec {
    PeelGraph g;
    uint32_t col0, ncols;
    uint32_t* table;
};
uint64_t peel_batch_ws_bytes(const std::vector<PeelSegSpec>& specs);
// All segments in one persistent launch (threads per block and the longest row
// queued as one item: 0 = defaults).  With *use_graph set the launch is
// captured in a CUDA graph; on return *use_graph says whether it was.  The grid
// covers at most max_sms SMs (0 = all), so that launches on other streams can
// run beside it.
fc_status peel_batch(const std::vector<PeelSegSpec>& specs, void* ws, size_t ws_bytes,
                     cudaStream_t s, PeelStats* st, uint32_t threads, uint32_t small_row,
                     bool* use_graph, uint32_t max_sms = 0);

// last CUDA error text, for diagnostics
const char* last_cuda_error();

}  // namespace fc
