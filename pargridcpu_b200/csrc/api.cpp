// extern "C" entry points of libfirmcore.so (declared in include/firmcore.h)
// and the table driver that runs the peel over column groups.
#include <atomic>
#include <cstring>
#include <new>
#include <string>

#include "device.h"

namespace fc {

static std::atomic<uint64_t> g_launches{0};
void count_launch(uint32_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
static std::atomic<uint64_t> g_allocs{0};
void count_alloc(uint32_t k) { g_allocs.fetch_add(k, std::memory_order_relaxed); }

// The peel of columns [lo, hi) in launches of up to peel_columns_per_group
// columns each, with the launches' statistics.
static fc_status peel_range(DeviceGraph* d, uint32_t lo, uint32_t hi, cudaStream_t s) {
    invalidate_densest(d);
    d->stats.peel_ms = 0;
    d->stats.peel_launches = d->stats.levels = d->stats.subrounds = 0;
    for (int i = 0; i < 3; i++) d->stats.phase_ms[i] = 0;
    if (!d->n || lo >= hi) return FC_OK;
    const uint32_t per = peel_columns_per_group(d);
    d->stats.columns_per_launch = per;
    for (uint32_t c0 = lo; c0 < hi; c0 += per) {
        const uint32_t nc = hi - c0 < per ? hi - c0 : per;
        PeelStats st;
        FC_TRY(peel_columns(d, c0, nc, s, &st));
        d->stats.peel_ms += st.ms;
        d->stats.peel_launches++;
        d->stats.levels += st.levels;
        d->stats.subrounds += st.subrounds;
        for (int i = 0; i < 3; i++) d->stats.phase_ms[i] += st.phase_ms[i];
    }
    return FC_OK;
}

fc_status coreindex(fc_graph* g, uint32_t* out, bool out_on_device, cudaStream_t s) {
    FC_TRY(upload(g, s));
    DeviceGraph* d = g->dev;
    d->home = s;
    if (!d->table_valid) {
        d->cols_lo = d->cols_hi = 0;
        FC_TRY(peel_range(d, 0, d->L, s));
        d->table_valid = true;
    }
    if (out) {
        uint64_t bytes = (uint64_t)d->n * d->L * 4;
        if (bytes) {
            if (out_on_device)
                FC_CUDA_TRY(cudaMemcpyAsync(out, d->table, bytes, cudaMemcpyDeviceToDevice, s));
            else
                FC_TRY(to_host(out, d->table, bytes, s));
        }
    }
    // every peel launch ended with a synchronize; only a device-to-device
    // copy of the table may still be in flight
    if (!out || !out_on_device) d->home = nullptr;
    return FC_OK;
}

// The table into `table` (host memory) and the densest search for `betas`:
// when the buffer is pinned, its copy runs on the library's copy stream while
// the densest kernels run on s -- issued once the densest search has read its
// per-column maxima back, so that its few small reads do not queue behind
// the table on the copy engines; otherwise the copy comes first.  Results as
// coreindex + densest.
fc_status coreindex_densest(fc_graph* g, uint32_t* table, const double* betas, uint32_t nb,
                            fc_densest_result* res, cudaStream_t s) {
    FC_TRY(coreindex(g, nullptr, false, s));
    DeviceGraph* d = g->dev;
    const uint64_t bytes = (uint64_t)d->n * d->L * 4;
    struct Events {  // destroyed on every return
        cudaEvent_t peeled = nullptr, copied = nullptr;
        ~Events() {
            if (peeled) cudaEventDestroy(peeled);
            if (copied) cudaEventDestroy(copied);
        }
    } ev;
    bool overlap = false, issued = false;
    cudaStream_t cs = nullptr;
    if (table && bytes) {
        cudaPointerAttributes a{};
        const bool pinned = cudaPointerGetAttributes(&a, table) == cudaSuccess &&
                            a.type == cudaMemoryTypeHost;
        cudaGetLastError();  // pageable memory is not an error
        cs = pinned ? library_copy_stream() : nullptr;
        if (cs && cs != s &&
            cudaEventCreateWithFlags(&ev.peeled, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&ev.copied, cudaEventDisableTiming) == cudaSuccess) {
            count_alloc(2);
            overlap = true;
        } else {
            cudaGetLastError();
            FC_TRY(to_host(table, d->table, bytes, s));
        }
    }
    const std::function<fc_status()> issue = [&]() -> fc_status {
        if (issued) return FC_OK;
        issued = true;
        FC_CUDA_TRY(cudaEventRecord(ev.peeled, s));
        FC_CUDA_TRY(cudaStreamWaitEvent(cs, ev.peeled, 0));
        FC_CUDA_TRY(cudaMemcpyAsync(table, d->table, bytes, cudaMemcpyDeviceToHost, cs));
        FC_CUDA_TRY(cudaEventRecord(ev.copied, cs));
        return FC_OK;
    };
    fc_status rc = densest(g, betas, nb, res, s, overlap ? &issue : nullptr);
    if (overlap) {
        // the histogram was already resident (the hook did not run), or the
        // densest search failed before it
        const fc_status rc2 = issue();
        if (rc == FC_OK) rc = rc2;
        if (rc2 == FC_OK) FC_CUDA_TRY(cudaEventSynchronize(ev.copied));
    }
    return rc;
}

// Columns [lo, hi) of the table (0-based); out (may be NULL) receives them,
// (hi - lo) rows of n.  Peels only those columns unless the whole table, or
// a range covering them, is already resident.
fc_status coreindex_range(fc_graph* g, uint32_t lo, uint32_t hi, uint32_t* out, bool out_on_device,
                          cudaStream_t s) {
    if (lo >= hi || hi > g->L) return FC_ERR_INVALID;
    FC_TRY(upload(g, s));
    DeviceGraph* d = g->dev;
    d->home = s;
    if (!d->table_valid && !(d->cols_lo <= lo && hi <= d->cols_hi)) {
        d->cols_lo = d->cols_hi = 0;
        FC_TRY(peel_range(d, lo, hi, s));
        d->cols_lo = lo;
        d->cols_hi = hi;
    }
    const uint64_t bytes = (uint64_t)d->n * (hi - lo) * 4;
    if (out && bytes) {
        const uint32_t* src = d->table + (uint64_t)lo * d->n;
        if (out_on_device)
            FC_CUDA_TRY(cudaMemcpyAsync(out, src, bytes, cudaMemcpyDeviceToDevice, s));
        else
            FC_TRY(to_host(out, src, bytes, s));
    }
    if (!out || !out_on_device) d->home = nullptr;
    return FC_OK;
}

}  // namespace fc

using namespace fc;

static fc_graph* new_graph() { return new (std::nothrow) fc_graph(); }

extern "C" {

const char* fc_status_string(fc_status s) {
    switch (s) {
        case FC_OK: return "ok";
        case FC_ERR_IO: return "i/o error";
        case FC_ERR_PARSE: return "malformed input";
        case FC_ERR_OOM: return "out of memory";
        case FC_ERR_BUDGET: return "over the device-memory budget";
        case FC_ERR_DEVICE: return "CUDA error";
        case FC_ERR_ITER_LIMIT: return "device loop or wait bound reached";
        case FC_ERR_INVALID: return "invalid argument";
        case FC_ERR_TOO_LARGE: return "graph exceeds the 32-bit index limits";
        case FC_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

int fc_abi_version(void) { return FC_ABI_VERSION; }

fc_status fc_graph_load_dir(const char* dir, int order, int write_vtx_map, fc_graph** out) {
    if (!dir || !out) return FC_ERR_INVALID;
    fc_graph* g = new_graph();
    if (!g) return FC_ERR_OOM;
    std::string d(dir);
    if (!d.empty() && d.back() != '/') d.push_back('/');
    fc_status s = load_dir(d, order, write_vtx_map != 0, g);
    if (s != FC_OK) {
        delete g;
        return s;
    }
    *out = g;
    return FC_OK;
}

fc_status fc_graph_from_pairs(uint32_t n_layers, const uint64_t* m, const uint32_t* pairs,
                              fc_graph** out) {
    if (!out || (n_layers && !m)) return FC_ERR_INVALID;
    uint64_t total = 0;
    for (uint32_t l = 0; l < n_layers; l++) total += m[l];
    if (total && !pairs) return FC_ERR_INVALID;
    fc_graph* g = new_graph();
    if (!g) return FC_ERR_OOM;
    fc_status s = build_from_pairs(n_layers, m, pairs, g);
    if (s != FC_OK) {
        delete g;
        return s;
    }
    *out = g;
    return FC_OK;
}

fc_status fc_graph_from_adjbuf(uint32_t n, uint32_t n_layers, const uint32_t* const* bufs,
                               const uint64_t* m, fc_graph** out) {
    if (!out || (n_layers && (!bufs || !m))) return FC_ERR_INVALID;
    fc_graph* g = new_graph();
    if (!g) return FC_ERR_OOM;
    fc_status s = build_from_adjbuf(n, n_layers, bufs, m, g);
    if (s != FC_OK) {
        delete g;
        return s;
    }
    *out = g;
    return FC_OK;
}

void fc_graph_free(fc_graph* g) {
    if (!g) return;
    release_device(g);
    delete g;
}

uint32_t fc_graph_n(const fc_graph* g) { return g ? g->n : 0; }
uint32_t fc_graph_layers(const fc_graph* g) { return g ? g->L : 0; }
uint64_t fc_graph_layer_m(const fc_graph* g, uint32_t l) {
    return (g && l < g->L) ? g->layer_m(l) : 0;
}

fc_status fc_graph_id2vtx(const fc_graph* g, uint64_t* out) {
    if (!g || (!out && g->n)) return FC_ERR_INVALID;
    if (g->n) memcpy(out, g->id2vtx.data(), (size_t)g->n * 8);
    return FC_OK;
}

fc_status fc_graph_order(const fc_graph* g, uint32_t* out) {
    if (!g || (!out && g->L)) return FC_ERR_INVALID;
    if (g->L) memcpy(out, g->order.data(), (size_t)g->L * 4);
    return FC_OK;
}

fc_status fc_graph_csr(const fc_graph* g, uint64_t* off, uint32_t* adj) {
    if (!g) return FC_ERR_INVALID;
    uint64_t no = (uint64_t)g->L * (g->n + 1);
    if (off)
        for (uint64_t i = 0; i < no; i++) off[i] = g->off.p[i];
    uint64_t na = g->total_entries();
    if (adj && na) memcpy(adj, g->adj.p, na * 4);
    return FC_OK;
}

fc_status fc_graph_upload(fc_graph* g, void* stream) {
    if (!g) return FC_ERR_INVALID;
    return upload(g, (cudaStream_t)stream);
}

fc_status fc_graph_release_device(fc_graph* g) {
    if (!g) return FC_ERR_INVALID;
    release_device(g);
    return FC_OK;
}

fc_status fc_graph_reset_results(fc_graph* g) {
    if (!g) return FC_ERR_INVALID;
    if (g->dev) {
        g->dev->table_valid = false;
        g->dev->cols_lo = g->dev->cols_hi = 0;
        invalidate_densest(g->dev);
    }
    return FC_OK;
}

uint64_t fc_graph_device_bytes(const fc_graph* g) { return g ? device_bytes(g) : 0; }

fc_status fc_coreindex(fc_graph* g, uint32_t* out, int out_on_device, void* stream) {
    if (!g) return FC_ERR_INVALID;
    return coreindex(g, out, out_on_device != 0, (cudaStream_t)stream);
}

fc_status fc_coreindex_densest(fc_graph* g, uint32_t* table, const double* betas,
                               uint32_t n_betas, fc_densest_result* res, void* stream) {
    if (!g || (n_betas && (!betas || !res))) return FC_ERR_INVALID;
    if (!g->n || !g->L) {
        FC_TRY(fc_coreindex(g, table, 0, stream));
        return fc_densest(g, betas, n_betas, res, stream);
    }
    return coreindex_densest(g, table, betas, n_betas, res, (cudaStream_t)stream);
}

fc_status fc_densest(fc_graph* g, const double* betas, uint32_t n_betas, fc_densest_result* res,
                     void* stream) {
    if (!g || (n_betas && (!betas || !res))) return FC_ERR_INVALID;
    if (!g->n || !g->L) {
        for (uint32_t b = 0; b < n_betas; b++) {
            memset(&res[b], 0, sizeof(res[b]));
            res[b].beta = betas[b];
        }
        return cuda_available() ? FC_OK : FC_ERR_NO_DEVICE;
    }
    return densest(g, betas, n_betas, res, (cudaStream_t)stream);
}

fc_status fc_densest_members(fc_graph* g, const fc_densest_result* res, uint32_t* nodes,
                             uint32_t* layers, void* stream) {
    if (!g || !res) return FC_ERR_INVALID;
    return densest_members(g, res, nodes, layers, (cudaStream_t)stream);
}

fc_status fc_cell_members(fc_graph* g, uint32_t k, uint32_t lmd, uint32_t* nodes, uint32_t cap,
                          uint32_t* count, void* stream) {
    if (!g) return FC_ERR_INVALID;
    if (!cuda_available()) return FC_ERR_NO_DEVICE;
    if (lmd < 1 || lmd > g->L) return FC_ERR_INVALID;
    if (!g->n) {
        if (count) *count = 0;
        return FC_OK;
    }
    return cell_members(g, k, lmd, nodes, cap, count, (cudaStream_t)stream);
}

fc_status fc_coreindex_range(fc_graph* g, uint32_t lmd_lo, uint32_t lmd_hi, uint32_t* out,
                             int out_on_device, void* stream) {
    if (!g || lmd_lo < 1 || lmd_lo >= lmd_hi || lmd_hi > g->L + 1) return FC_ERR_INVALID;
    if (!cuda_available()) return FC_ERR_NO_DEVICE;
    if (!g->n) return FC_OK;
    return coreindex_range(g, lmd_lo - 1, lmd_hi - 1, out, out_on_device != 0,
                           (cudaStream_t)stream);
}

fc_status fc_cells_range(fc_graph* g, uint32_t lmd_lo, uint32_t lmd_hi, double beta,
                         fc_cell* cells_out, uint32_t cap, uint32_t* count, void* stream) {
    if (!g || lmd_lo < 1 || lmd_lo >= lmd_hi || lmd_hi > g->L + 1) return FC_ERR_INVALID;
    if (!cuda_available()) return FC_ERR_NO_DEVICE;
    if (!g->n) {
        if (count) *count = 0;
        return FC_OK;
    }
    return cells_range(g, lmd_lo - 1, lmd_hi - 1, beta, cells_out, cap, count,
                       (cudaStream_t)stream);
}

fc_status fc_cells(fc_graph* g, double beta, fc_cell* cells_out, uint32_t cap, uint32_t* count,
                   void* stream) {
    if (!g) return FC_ERR_INVALID;
    if (!g->n || !g->L) {
        if (count) *count = 0;
        return cuda_available() ? FC_OK : FC_ERR_NO_DEVICE;
    }
    return cells(g, beta, cells_out, cap, count, (cudaStream_t)stream);
}

fc_status fc_cell_index(fc_graph* g, uint32_t* order, uint64_t* col_off, uint32_t* sizes,
                        uint64_t sizes_cap, uint64_t* sizes_count, void* stream) {
    if (!g) return FC_ERR_INVALID;
    if (!cuda_available()) return FC_ERR_NO_DEVICE;
    if (!g->n || !g->L) {
        if (col_off)
            for (uint32_t l = 0; l <= g->L; l++) col_off[l] = 0;
        if (sizes_count) *sizes_count = 0;
        return FC_OK;
    }
    return cell_index(g, order, col_off, sizes, sizes_cap, sizes_count, (cudaStream_t)stream);
}

fc_status fc_cells_members(fc_graph* g, const uint32_t* ks, const uint32_t* lmds, uint32_t nq,
                           int by_index, uint64_t* offsets, uint32_t* nodes, uint64_t cap,
                           void* stream) {
    if (!g || (nq && (!ks || !lmds))) return FC_ERR_INVALID;
    if (!cuda_available()) return FC_ERR_NO_DEVICE;
    for (uint32_t q = 0; q < nq; q++)
        if (lmds[q] < 1 || lmds[q] > g->L) return FC_ERR_INVALID;
    if (!g->n) {
        if (offsets)
            for (uint32_t q = 0; q <= nq; q++) offsets[q] = 0;
        return FC_OK;
    }
    return cells_members(g, ks, lmds, nq, by_index != 0, offsets, nodes, cap,
                         (cudaStream_t)stream);
}

fc_status fc_mlcd_query(const uint32_t* cores, uint32_t n, uint32_t P, const uint32_t* ks,
                        const uint32_t* lmds, uint32_t nq, uint64_t* offsets, uint32_t* nodes,
                        uint64_t cap, void* stream) {
    if ((n && P && !cores) || (nq && (!ks || !lmds))) return FC_ERR_INVALID;
    if (!cuda_available()) return FC_ERR_NO_DEVICE;
    if ((uint64_t)n * P >= (1ull << 40)) return FC_ERR_TOO_LARGE;
    return mlcd_query(cores, n, P, ks, lmds, nq, offsets, nodes, cap, (cudaStream_t)stream);
}

fc_status fc_graph_stats(const fc_graph* g, fc_stats* out) {
    if (!g || !out) return FC_ERR_INVALID;
    *out = g->dev ? g->dev->stats : fc_stats{};
    return FC_OK;
}

uint64_t fc_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }
uint64_t fc_alloc_count(void) { return g_allocs.load(std::memory_order_relaxed); }

fc_status fc_probe_atomics(uint64_t bytes, uint64_t ops, double* gatomics_per_s, void* stream) {
    if (!gatomics_per_s || !ops) return FC_ERR_INVALID;
    if (!cuda_available()) return FC_ERR_NO_DEVICE;
    return probe_atomics(bytes, ops, gatomics_per_s, (cudaStream_t)stream);
}

fc_status fc_batch_run(fc_graph* const* graphs, uint32_t count, double beta,
                       uint32_t* const* tables, fc_densest_result* res,
                       const fc_batch_options* opt, fc_batch_report* report, void* stream) {
    if (count && !graphs) return FC_ERR_INVALID;
    for (uint32_t i = 0; i < count; i++)
        if (!graphs[i]) return FC_ERR_INVALID;
    return batch_run(graphs, count, beta, tables, res, opt, report, (cudaStream_t)stream);
}

}  // extern "C"
