// Batched decomposition of many graphs (fc_batch_run).
//
// Batched form: every graph is one segment of a single persistent peel launch
// (all its lambda columns; graphs whose scratch would not fit one launch are
// spread over a few launches), optionally captured in a CUDA graph; then the
// densest search per graph.  The block size and the hub threshold (longest
// row queued as one work item) are chosen by an autotuner that times the
// candidates on a sample of the batch and remembers the winner per batch
// shape.  Results do not depend on either, so tuning never changes an output.
//
// Plain form (the baseline): one graph after another, one lambda column per
// launch -- "a single launch per lambda".
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "device.h"

namespace fc {

static uint32_t env_u32b(const char* name, uint32_t dflt) {
    const char* s = getenv(name);
    return s && *s ? (uint32_t)strtoul(s, nullptr, 10) : dflt;
}

// FC_DEBUG=1: one stderr line per step of a batched run
static bool debug_on() {
    static int v = -1;
    if (v < 0) v = env_u32b("FC_DEBUG", 0) ? 1 : 0;
    return v == 1;
}
#define BATCH_TRACE(...)                          \
    do {                                          \
        if (debug_on()) {                         \
            fprintf(stderr, "batch: " __VA_ARGS__); \
            fputc('\n', stderr);                  \
            fflush(stderr);                       \
        }                                         \
    } while (0)

// The densest searches of a batch run on DENSE_WORKERS host threads, each
// with its own stream and pinned staging buffer: one graph's search is a few
// small kernels separated by host round trips, so the graphs' searches
// overlap on the device.  The pool is per device and process-wide; batches
// from several callers take turns on it.
static constexpr uint32_t DENSE_WORKERS = 8;
struct DenseWorker {
    cudaStream_t s = nullptr;
    Staging stage;
};
static std::mutex g_dw_mu, g_dw_run_mu;
static std::map<int, std::vector<DenseWorker>> g_dw;

static std::vector<DenseWorker>* dense_workers() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lk(g_dw_mu);
    std::vector<DenseWorker>& v = g_dw[dev];
    if (v.empty()) {
        v.resize(DENSE_WORKERS);
        for (DenseWorker& w : v) {
            if (cudaStreamCreateWithFlags(&w.s, cudaStreamNonBlocking) != cudaSuccess) w.s = nullptr;
            count_alloc(2);  // the stream and the staging buffer
            if (cudaHostAlloc(&w.stage.p, 1u << 20, cudaHostAllocDefault) == cudaSuccess)
                w.stage.cap = 1u << 20;
            else
                w.stage.p = nullptr;
        }
        cudaGetLastError();
    }
    for (const DenseWorker& w : v)
        if (!w.s) return nullptr;
    return &v;
}

static fc_status densest_all(fc_graph* const* gs, uint32_t count, double beta,
                             fc_densest_result* res, cudaStream_t s, double* ms) {
    *ms = 0;
    if (!res) return FC_OK;
    std::vector<uint32_t> todo;
    for (uint32_t i = 0; i < count; i++) {
        if (gs[i]->n && gs[i]->L) {
            todo.push_back(i);
        } else {
            res[i] = fc_densest_result{};
            res[i].beta = beta;
        }
    }
    std::vector<DenseWorker>* pool = todo.size() >= 4 ? dense_workers() : nullptr;
    if (!pool) {  // a few graphs: one after another on the caller's stream
        for (uint32_t i : todo) {
            BATCH_TRACE("densest graph %u (n %u, L %u)", i, gs[i]->n, gs[i]->L);
            FC_TRY(densest(gs[i], &beta, 1, res + i, s));
            *ms += gs[i]->dev->stats.densest_ms;
        }
        return FC_OK;
    }
    std::lock_guard<std::mutex> lk(g_dw_run_mu);
    int dev = 0;
    cudaGetDevice(&dev);
    const uint32_t nw = (uint32_t)std::min<size_t>(pool->size(), todo.size());
    std::vector<fc_status> rc(nw, FC_OK);
    std::vector<double> wms(nw, 0.0);
    std::vector<std::thread> th;
    for (uint32_t w = 0; w < nw; w++) {
        th.emplace_back([&, w] {
            cudaSetDevice(dev);
            DenseWorker& me = (*pool)[w];
            set_thread_staging(me.stage.p ? &me.stage : nullptr);
            for (size_t k = w; k < todo.size() && rc[w] == FC_OK; k += nw) {
                fc_graph* g = gs[todo[k]];
                rc[w] = densest(g, &beta, 1, res + todo[k], me.s);
                if (rc[w] == FC_OK) wms[w] += g->dev->stats.densest_ms;
            }
            set_thread_staging(nullptr);
        });
    }
    for (auto& t : th) t.join();
    for (uint32_t w = 0; w < nw; w++) {
        FC_TRY(rc[w]);
        *ms += wms[w];
    }
    return FC_OK;
}

static fc_status copy_tables(fc_graph* const* gs, uint32_t count, uint32_t* const* tables,
                             cudaStream_t s) {
    if (!tables) return FC_OK;
    for (uint32_t i = 0; i < count; i++) {
        fc_graph* g = gs[i];
        const uint64_t bytes = (uint64_t)g->n * g->L * 4;
        if (tables[i] && bytes)
            FC_TRY(to_host(tables[i], g->dev->table, bytes, s));
    }
    FC_CUDA_TRY(cudaStreamSynchronize(s));
    return FC_OK;
}

// ---- plain: one lambda column per launch -------------------------------------

static fc_status batch_plain(fc_graph* const* gs, uint32_t count, double beta,
                             uint32_t* const* tables, fc_densest_result* res,
                             fc_batch_report* rep, cudaStream_t s) {
    double peel_ms = 0;
    uint32_t launches = 0, levels = 0;
    for (uint32_t i = 0; i < count; i++)
        FC_TRY(batch_plain_one(gs[i], s, &peel_ms, &launches, &levels));
    double dms = 0;
    const auto t_dense = std::chrono::steady_clock::now();
    FC_TRY(densest_all(gs, count, beta, res, s, &dms));
    dms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_dense)
              .count();
    FC_TRY(copy_tables(gs, count, tables, s));
    if (rep) {
        rep->peel_ms = peel_ms;
        rep->densest_ms = dms;
        rep->peel_launches = launches;
        rep->levels = levels;
        rep->used_cuda_graph = 0;
    }
    return FC_OK;
}

// ---- batched: segments in persistent launches --------------------------------

struct TuneKey {
    uint32_t count, maxL, max_sms;
    uint64_t entries_mb;
    bool operator<(const TuneKey& o) const {
        return std::tie(count, maxL, max_sms, entries_mb) <
               std::tie(o.count, o.maxL, o.max_sms, o.entries_mb);
    }
};
static std::mutex g_tune_mu;
static std::map<TuneKey, std::pair<uint32_t, uint32_t>> g_tuned;  // -> (threads, small_row)

// Launch groups: consecutive graphs whose peel scratch stays within the
// budget (FC_BATCH_WS_MB, default 32 GiB) share one launch.
static void plan_groups(const std::vector<PeelSegSpec>& specs, uint64_t budget,
                        std::vector<std::pair<size_t, size_t>>* groups) {
    size_t i = 0;
    while (i < specs.size()) {
        size_t e = i + 1;
        while (e < specs.size()) {
            std::vector<PeelSegSpec> trial(specs.begin() + i, specs.begin() + e + 1);
            if (peel_batch_ws_bytes(trial) > budget) break;
            e++;
        }
        groups->push_back({i, e});
        i = e;
    }
}

static fc_status run_groups(const std::vector<PeelSegSpec>& specs,
                            const std::vector<std::pair<size_t, size_t>>& groups, void* ws,
                            uint64_t ws_bytes, cudaStream_t s, uint32_t threads, uint32_t small_row,
                            bool want_graph, uint32_t max_sms, double* ms, uint32_t* levels,
                            bool* graphed) {
    *ms = 0;
    *levels = 0;
    *graphed = want_graph;
    for (const auto& gr : groups) {
        std::vector<PeelSegSpec> part(specs.begin() + gr.first, specs.begin() + gr.second);
        PeelStats st;
        bool g = want_graph;
        BATCH_TRACE("peel graphs [%zu, %zu) threads %u small_row %u graph %d", gr.first,
                    gr.second, threads, small_row, (int)g);
        FC_TRY(peel_batch(part, ws, ws_bytes, s, &st, threads, small_row, &g, max_sms));
        BATCH_TRACE("  done: %.3f ms, %u levels, cuda graph %d", st.ms, st.levels, (int)g);
        *graphed = *graphed && g;
        *ms += st.ms;
        *levels += st.levels;
    }
    return FC_OK;
}

uint64_t batch_peel_ws_bytes(fc_graph* const* gs, uint32_t count) {
    std::vector<PeelSegSpec> specs;
    for (uint32_t i = 0; i < count; i++) {
        const fc_graph* g = gs[i];
        if (!g->n || !g->L) continue;
        PeelSegSpec sp{};
        sp.g.n = g->n;
        sp.g.L = g->L;
        sp.g.entries = g->total_entries();
        sp.ncols = g->L;
        specs.push_back(sp);
    }
    return specs.empty() ? 0 : peel_batch_ws_bytes(specs);
}

fc_status batch_peel(fc_graph* const* gs, uint32_t count, const fc_batch_options* opt,
                     uint32_t max_sms, fc_batch_report* rep, cudaStream_t s) {
    std::vector<PeelSegSpec> specs;
    uint32_t maxL = 1;
    uint64_t entries = 0;
    for (uint32_t i = 0; i < count; i++) {
        fc_graph* g = gs[i];
        FC_TRY(upload(g, s));
        DeviceGraph* d = g->dev;
        d->home = s;
        invalidate_densest(d);
        if (d->n && d->L) {
            PeelSegSpec sp;
            sp.g = PeelGraph{d->n, d->L, d->entries, d->node_ptr, d->adj, d->deg0, d->max_deg + 1,
                             d->big_id, d->ptab};
            sp.col0 = 0;
            sp.ncols = d->L;
            sp.table = d->table;
            specs.push_back(sp);
            maxL = std::max(maxL, d->L);
            entries += (uint64_t)d->entries * d->L;
        }
    }
    const uint64_t budget = (uint64_t)env_u32b("FC_BATCH_WS_MB", 32768) << 20;
    std::vector<std::pair<size_t, size_t>> groups;
    plan_groups(specs, budget, &groups);
    uint64_t ws_bytes = 0;
    for (const auto& gr : groups) {
        std::vector<PeelSegSpec> part(specs.begin() + gr.first, specs.begin() + gr.second);
        ws_bytes = std::max(ws_bytes, peel_batch_ws_bytes(part));
    }
    BATCH_TRACE("%u graphs uploaded, %zu segments, %zu launch groups, workspace %llu bytes", count,
                specs.size(), groups.size(), (unsigned long long)ws_bytes);
    void* ws = nullptr;
    if (!specs.empty()) FC_TRY(dev_alloc(&ws, ws_bytes, s));
    const bool want_graph = opt ? opt->use_cuda_graph != 0 : true;
    uint32_t threads = opt ? opt->block_threads : 0;
    uint32_t small_row = opt ? opt->hub_threshold : 0;
    bool tuned_now = false;
    fc_status rc = FC_OK;
    if (!specs.empty() && (!threads || !small_row)) {
        TuneKey key{count, maxL, max_sms, entries >> 20};
        std::pair<uint32_t, uint32_t> best{0, 0};
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto it = g_tuned.find(key);
            if (it != g_tuned.end()) best = it->second;
        }
        if (!best.first) {
            // candidates timed on a sample: every k-th graph, up to 32 of them
            std::vector<PeelSegSpec> sample;
            const size_t step = std::max<size_t>(1, specs.size() / 32);
            for (size_t i = 0; i < specs.size(); i += step) sample.push_back(specs[i]);
            std::vector<std::pair<size_t, size_t>> sg;
            plan_groups(sample, ws_bytes, &sg);
            double best_ms = 1e300;
            for (uint32_t th : {512u, 1024u})
                for (uint32_t sr : {16u, 32u, 64u}) {
                    double ms;
                    uint32_t lv;
                    bool gr;
                    rc = run_groups(sample, sg, ws, ws_bytes, s, th, sr, false, max_sms, &ms, &lv,
                                    &gr);
                    if (rc != FC_OK) break;
                    if (ms < best_ms) {
                        best_ms = ms;
                        best = {th, sr};
                    }
                }
            if (rc == FC_OK) {
                std::lock_guard<std::mutex> lk(g_tune_mu);
                g_tuned[key] = best;
                tuned_now = true;
            }
        }
        if (!threads) threads = best.first;
        if (!small_row) small_row = best.second;
    }
    double peel_ms = 0;
    uint32_t levels = 0;
    bool graphed = false;
    if (rc == FC_OK && !specs.empty())
        rc = run_groups(specs, groups, ws, ws_bytes, s, threads, small_row, want_graph, max_sms,
                        &peel_ms, &levels, &graphed);
    if (ws) dev_free(ws, s);
    FC_TRY(rc);
    for (uint32_t i = 0; i < count; i++) gs[i]->dev->table_valid = true;
    if (rep) {
        rep->peel_ms = peel_ms;
        rep->peel_launches = (uint32_t)groups.size();
        rep->block_threads = threads;
        rep->hub_threshold = small_row;
        rep->levels = levels;
        rep->used_cuda_graph = graphed ? 1 : 0;
        rep->autotuned = tuned_now ? 1 : 0;
    }
    return FC_OK;
}

static fc_status batch_persistent(fc_graph* const* gs, uint32_t count, double beta,
                                  uint32_t* const* tables, fc_densest_result* res,
                                  const fc_batch_options* opt, fc_batch_report* rep,
                                  cudaStream_t s) {
    FC_TRY(batch_peel(gs, count, opt, 0, rep, s));
    double dms = 0;
    const auto t_dense = std::chrono::steady_clock::now();
    FC_TRY(densest_all(gs, count, beta, res, s, &dms));
    dms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_dense)
              .count();
    FC_TRY(copy_tables(gs, count, tables, s));
    if (rep) rep->densest_ms = dms;
    return FC_OK;
}

fc_status batch_plain_one(fc_graph* g, cudaStream_t s, double* peel_ms, uint32_t* launches,
                          uint32_t* levels) {
    FC_TRY(upload(g, s));
    DeviceGraph* d = g->dev;
    d->home = s;
    invalidate_densest(d);
    for (uint32_t c = 0; c < d->L && d->n; c++) {
        PeelStats st;
        FC_TRY(peel_columns(d, c, 1, s, &st));
        *peel_ms += st.ms;
        *launches += 1;
        *levels += st.levels;
    }
    d->table_valid = true;
    return FC_OK;
}

fc_status batch_run(fc_graph* const* gs, uint32_t count, double beta, uint32_t* const* tables,
                    fc_densest_result* res, const fc_batch_options* opt, fc_batch_report* rep,
                    cudaStream_t s) {
    if (!cuda_available()) return FC_ERR_NO_DEVICE;
    if (rep) *rep = fc_batch_report{};
    const fc_status rc = opt && opt->plain
                             ? batch_plain(gs, count, beta, tables, res, rep, s)
                             : batch_persistent(gs, count, beta, tables, res, opt, rep, s);
    // nothing of these graphs is left in flight on s afterwards
    const cudaError_t e = cudaStreamSynchronize(s);
    for (uint32_t i = 0; i < count; i++)
        if (gs[i]->dev) gs[i]->dev->home = nullptr;
    if (rc != FC_OK) return rc;
    FC_CUDA_TRY(e);
    return FC_OK;
}

}  // namespace fc
