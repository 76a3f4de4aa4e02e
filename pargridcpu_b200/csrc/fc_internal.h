// Internal declarations of libfirmcore: host graph, device layout, kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "firmcore.h"

namespace fc {

// ---------------------------------------------------------------------------
// Host graph (the reference's MultilayerGraph after LoadFromFile/SetGraphOrder)
//
// Layers are stored in logical order (layer i = the reference's GetGraph(i) =
// graph_layers[order[i]]), each as a CSR over internal ids with ascending,
// de-duplicated neighbour rows -- the content of Graph::adj_lst_buf without the
// inline degree word.
// ---------------------------------------------------------------------------

// Page-locked when a CUDA device is present (so uploads run at full copy
// bandwidth), ordinary heap memory otherwise.
template <class T>
struct HostBuf {
    T* p = nullptr;
    size_t n = 0;
    bool pinned = false;
    HostBuf() = default;
    HostBuf(const HostBuf&) = delete;
    HostBuf& operator=(const HostBuf&) = delete;
    ~HostBuf() { reset(); }
    bool alloc(size_t count);
    void reset();
    T& operator[](size_t i) { return p[i]; }
    const T& operator[](size_t i) const { return p[i]; }
};

struct DeviceGraph;  // device-resident CSR and results (graph.cu)

}  // namespace fc

struct fc_graph {
    uint32_t n = 0, L = 0;
    std::vector<uint32_t> order;   // -o permutation (file layer index of logical layer i)
    std::vector<uint64_t> id2vtx;  // internal id -> raw id
    // L*(n+1) absolute indices into adj, 32-bit: a graph holds fewer than
    // 2^32 adjacency entries (FC_ERR_TOO_LARGE at load), and the upload
    // copies half the bytes of 64-bit offsets
    fc::HostBuf<uint32_t> off;
    fc::HostBuf<uint32_t> adj;     // all layers' rows, layer after layer
    uint64_t total_entries() const { return L ? off[(uint64_t)L * (n + 1) - 1] : 0; }
    uint64_t layer_m(uint32_t l) const {
        const uint32_t* o = off.p + (uint64_t)l * (n + 1);
        return o[n] - o[0];
    }
    fc::DeviceGraph* dev = nullptr;
};

namespace fc {

// ---- loader (loader.cpp) ----------------------------------------------------
fc_status load_dir(const std::string& dir, int order, bool write_vtx_map, fc_graph* g);
fc_status build_from_pairs(uint32_t L, const uint64_t* m, const uint32_t* pairs, fc_graph* g);
fc_status build_from_adjbuf(uint32_t n, uint32_t L, const uint32_t* const* bufs, const uint64_t* m,
                            fc_graph* g);
void apply_order(int order, fc_graph* g);

// ---- device (graph.cu / peel.cu / densest.cu) --------------------------------
bool cuda_available();
fc_status upload(fc_graph* g, cudaStream_t s);
// frees g's device copy; waits for g's last stream first unless the caller
// knows that its work is complete
void release_device(fc_graph* g, bool wait_home = true);
uint64_t device_bytes(const fc_graph* g);
fc_status coreindex(fc_graph* g, uint32_t* out, bool out_on_device, cudaStream_t s);
fc_status coreindex_densest(fc_graph* g, uint32_t* table, const double* betas, uint32_t nb,
                            fc_densest_result* res, cudaStream_t s);
// after_maxima (optional) runs once the per-column maxima are on the host,
// before the histogram kernels: the table is complete and the stream idle
fc_status densest(fc_graph* g, const double* betas, uint32_t nb, fc_densest_result* res,
                  cudaStream_t s, const std::function<fc_status()>* after_maxima = nullptr);
fc_status densest_members(fc_graph* g, const fc_densest_result* r, uint32_t* nodes,
                          uint32_t* layers, cudaStream_t s);
fc_status cells(fc_graph* g, double beta, fc_cell* out, uint32_t cap, uint32_t* count,
                cudaStream_t s);
fc_status cell_members(fc_graph* g, uint32_t k, uint32_t lmd, uint32_t* nodes, uint32_t cap,
                       uint32_t* count, cudaStream_t s);
// every cell as a prefix of one order per column (fc_cell_index), many cells
// at once (fc_cells_members), the MLCD membership test (fc_mlcd_query)
fc_status cell_index(fc_graph* g, uint32_t* order, uint64_t* col_off, uint32_t* sizes,
                     uint64_t sizes_cap, uint64_t* sizes_count, cudaStream_t s);
fc_status cells_members(fc_graph* g, const uint32_t* ks, const uint32_t* lmds, uint32_t nq,
                        bool by_index, uint64_t* offsets, uint32_t* nodes, uint64_t cap,
                        cudaStream_t s);
fc_status mlcd_query(const uint32_t* cores, uint32_t n, uint32_t P, const uint32_t* ks,
                     const uint32_t* lmds, uint32_t nq, uint64_t* offsets, uint32_t* nodes,
                     uint64_t cap, cudaStream_t s);
// fc_probe_atomics (probe.cu)
fc_status probe_atomics(uint64_t bytes, uint64_t ops, double* rate, cudaStream_t s);
// lambda columns [lo, hi), 0-based (fc_coreindex_range / fc_cells_range)
fc_status coreindex_range(fc_graph* g, uint32_t lo, uint32_t hi, uint32_t* out, bool out_on_device,
                          cudaStream_t s);
fc_status cells_range(fc_graph* g, uint32_t lo, uint32_t hi, double beta, fc_cell* out, uint32_t cap,
                      uint32_t* count, cudaStream_t s);
fc_status batch_run(fc_graph* const* gs, uint32_t count, double beta, uint32_t* const* tables,
                    fc_densest_result* res, const fc_batch_options* opt, fc_batch_report* rep,
                    cudaStream_t s);
// The peel of every graph (all its columns) in persistent launches covering
// at most max_sms SMs (0 = all) on stream s, uploading graphs as needed;
// each graph's table is valid on the device afterwards.  rep may be NULL.
fc_status batch_peel(fc_graph* const* gs, uint32_t count, const fc_batch_options* opt,
                     uint32_t max_sms, fc_batch_report* rep, cudaStream_t s);
// the peel scratch batch_peel allocates for these graphs (one launch group)
uint64_t batch_peel_ws_bytes(fc_graph* const* gs, uint32_t count);
// one graph, one lambda column per launch (the plain form); table valid
// after; adds to the three counters
fc_status batch_plain_one(fc_graph* g, cudaStream_t s, double* peel_ms, uint32_t* launches,
                          uint32_t* levels);
// a graph's device copy is going away: servers drop it from their records
void residency_forget(fc_graph* g);
// device or pinned-host allocations, streams and events this library created
// (fc_alloc_count)
void count_alloc(uint32_t k = 1);
// loads every kernel of the library on the current device now (once)
void preload_kernels();
void peel_preload();
void densest_preload();

}  // namespace fc

#define FC_CUDA_TRY(expr)                                                   \
    do {                                                                    \
        cudaError_t e_ = (expr);                                            \
        if (e_ != cudaSuccess) {                                            \
            fc::set_last_cuda_error(e_, #expr, __FILE__, __LINE__);         \
            return e_ == cudaErrorMemoryAllocation ? FC_ERR_OOM : FC_ERR_DEVICE; \
        }                                                                   \
    } while (0)

#define FC_TRY(expr)                      \
    do {                                  \
        fc_status s_ = (expr);            \
        if (s_ != FC_OK) return s_;       \
    } while (0)

namespace fc {
void set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line);
}
