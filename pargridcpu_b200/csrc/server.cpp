// Continuous-batching request loop (fc_server_*).
//
// Requests (a graph + beta) wait in one FIFO.  The server runs `lanes` lane
// threads, each with its own stream; a lane that is free takes, at once,
// every pending request that fits -- the admission tests below -- and runs
// them as one batch: one persistent peel launch over all their graphs (one
// segment per distinct graph, every lambda column), then the densest search
// of each request, then the table copies.  Requests that arrive while a
// batch is on the device wait for the next free lane, so new work joins as
// soon as a lane, SMs and memory free up.  Each batch's peel grid covers the
// SMs it claimed (form_batch): a heavy request runs alone on three quarters
// of them while light batches run on the rest, so the two overlap on the
// device and light requests never queue behind a heavy one.
//
// Admission: a request is taken while the device bytes of everything
// admitted -- the device copies of resident graphs plus the scratch of the
// running batches -- stay within the budget.  Graphs stay resident after
// their requests complete (they are often asked again); when memory is
// short, resident graphs that no running batch uses are released, least
// recently used first.  A graph runs on one lane at a time (its table lives
// with its device copy), so a request whose graph is running elsewhere waits.
// A request that alone would exceed the budget fails with FC_ERR_BUDGET.
//
// The plain form (options.plain) is the one-at-a-time baseline: one lane, one
// request per batch, one lambda column per launch.
//
// Every result equals fc_coreindex + fc_densest on the graph alone: the
// table is the unique core index, whatever the batch, and the densest search
// reads only the graph's own table.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <set>
#include <thread>
#include <unordered_map>
#include <vector>

#include "device.h"

using Clock = std::chrono::steady_clock;

namespace fc {

// ---- residency: device copies kept by servers ------------------------------
// Each server keeps its own least-recently-used list of the graphs whose
// device copies it holds, and its budget counts only those.  The index of
// all lists is process-wide, so that release_device (a graph freed by its
// owner, or released by any server) removes the graph from whichever list
// holds it.  A graph is on one list at a time: the last server to use it.

struct Residency {
    std::list<fc_graph*> lru;  // front = most recently used
    uint64_t bytes = 0;
};

struct ResEntry {
    Residency* owner;
    uint64_t bytes;
    std::list<fc_graph*>::iterator pos;
};

static std::mutex g_res_mu;
static std::unordered_map<fc_graph*, ResEntry> g_res;

static void res_unlink(std::unordered_map<fc_graph*, ResEntry>::iterator it) {  // under g_res_mu
    it->second.owner->bytes -= it->second.bytes;
    it->second.owner->lru.erase(it->second.pos);
    g_res.erase(it);
}

void residency_forget(fc_graph* g) {
    std::lock_guard<std::mutex> lk(g_res_mu);
    auto it = g_res.find(g);
    if (it != g_res.end()) res_unlink(it);
}

static void residency_touch(Residency* r, fc_graph* g, uint64_t bytes) {
    std::lock_guard<std::mutex> lk(g_res_mu);
    auto it = g_res.find(g);
    if (it != g_res.end()) res_unlink(it);
    r->lru.push_front(g);
    g_res[g] = ResEntry{r, bytes, r->lru.begin()};
    r->bytes += bytes;
}

static bool residency_has(Residency* r, fc_graph* g) {
    std::lock_guard<std::mutex> lk(g_res_mu);
    auto it = g_res.find(g);
    return it != g_res.end() && it->second.owner == r;
}

static uint64_t residency_bytes(Residency* r) {
    std::lock_guard<std::mutex> lk(g_res_mu);
    return r->bytes;
}

// The server forgets its copies (they stay on the device with their graphs).
static void residency_drop(Residency* r) {
    std::lock_guard<std::mutex> lk(g_res_mu);
    while (!r->lru.empty()) res_unlink(g_res.find(r->lru.front()));
}

// Graphs of r not in `keep`, least recently used first, until their bytes
// reach `need` (all of them when they do not).
static std::vector<std::pair<fc_graph*, uint64_t>> residency_victims(
    Residency* r, const std::set<fc_graph*>& keep, uint64_t need) {
    std::lock_guard<std::mutex> lk(g_res_mu);
    std::vector<std::pair<fc_graph*, uint64_t>> out;
    uint64_t got = 0;
    for (auto it = r->lru.rbegin(); it != r->lru.rend() && got < need; ++it) {
        if (keep.count(*it)) continue;
        const uint64_t b = g_res[*it].bytes;
        out.push_back({*it, b});
        got += b;
    }
    return out;
}

// Device bytes of a graph's resident copy: CSR, degrees, table, the
// ordered rows' index (at most one per ORDER_MIN_ROW + 1 entries) and the
// densest search's per-graph state (an estimate: transposed table, the
// histograms and cell records).
static uint64_t graph_bytes(const fc_graph* g) {
    const uint64_t n = g->n, L = g->L, e = g->total_entries();
    const uint64_t order = 4 * n + (e / (ORDER_MIN_ROW + 1) + 1) * BUCKETS * 4;
    return 4 * (n + 1) + 4 * e + 8 * n * L + 4 * n * L + order + (16ull << 20);
}

}  // namespace fc

namespace {

struct Request {
    uint64_t ticket = 0;
    fc_graph* g = nullptr;
    double beta = 1.0;
    uint32_t* table = nullptr;
    fc_densest_result* res = nullptr;
    Clock::time_point t_submit;
    fc_status status = FC_OK;
    double latency_ms = 0.0;
    bool done = false;
};

}  // namespace

struct fc_server {
    // options
    uint64_t budget = 0;
    uint32_t max_inflight = 0, lanes = 0, max_batch_graphs = 0;
    uint32_t sms = 0, heavy_sms = 0, min_light_sms = 0;  // the device's SMs and the shares
    uint64_t heavy_visits = 0;
    size_t backlog_requests = 8;  // pending requests from which everything batches
    Clock::time_point last_backlog = Clock::now() - std::chrono::hours(1);
    bool plain = false;
    fc_batch_options bopt{};

    fc::Residency res;  // device copies this server keeps

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> pending;
    std::map<uint64_t, Request*> all;
    uint64_t next_ticket = 1;
    std::set<fc_graph*> running_graphs;  // graphs of the batches on the device
    uint64_t running_bytes = 0;          // their scratch and not yet resident copies
    uint32_t running_requests = 0;
    uint32_t free_sms = 0;               // SMs no running peel grid claims
    bool heavy_running = false;
    bool stop = false;
    std::vector<std::thread> threads;

    // statistics (under mu)
    fc_server_stats st{};
    uint32_t running_lanes = 0;
    Clock::time_point t_mark = Clock::now();

    void clock_advance() {
        const Clock::time_point now = Clock::now();
        const double dt = std::chrono::duration<double, std::milli>(now - t_mark).count();
        if (running_lanes >= 1) st.busy_ms += dt;
        if (running_lanes >= 2) st.overlap_ms += dt;
        t_mark = now;
    }

    void finish(Request* r, fc_status status) {  // under mu
        r->status = status;
        r->latency_ms =
            std::chrono::duration<double, std::milli>(Clock::now() - r->t_submit).count();
        r->done = true;
        st.requests_done++;
    }

    // Edge visits of a request (every lambda column visits every entry).
    bool is_heavy(const Request* r) const {
        return !plain && r->g->total_entries() * (uint64_t)r->g->L >= heavy_visits;
    }

    // Memory admission of the graph of r, not yet in the batch (under mu):
    // 0 = admitted (`used` and the batch's `reserve` grow), 1 = can never fit
    // (r finished with FC_ERR_BUDGET), 2 = no room now.  Graphs released to
    // make room are released here, under the lock, so that no other lane can
    // take one of them meanwhile; their last work has completed (every batch
    // ends with a stream synchronize), so the release does not wait.
    int admit(Request* r, uint64_t* used, const std::set<fc_graph*>& taken, uint64_t* reserve) {
        fc_graph* g = r->g;
        const uint64_t gb = fc::graph_bytes(g);
        const uint64_t wb = plain ? fc::peel_ws_bytes(g->n, g->L, g->total_entries(), 1)
                                  : fc::batch_peel_ws_bytes(&g, 1);
        if (gb + wb > budget) {
            finish(r, FC_ERR_BUDGET);
            cv_done.notify_all();
            return 1;
        }
        const uint64_t need = (fc::residency_has(&res, g) ? 0 : gb) + wb;
        if (*used + need > budget) {
            // release resident graphs that nothing running or taken uses
            std::set<fc_graph*> keep(running_graphs);
            keep.insert(taken.begin(), taken.end());
            keep.insert(g);
            auto victims = fc::residency_victims(&res, keep, *used + need - budget);
            uint64_t freed = 0;
            for (auto& v : victims) freed += v.second;
            if (*used + need > budget + freed) return 2;
            for (auto& v : victims) fc::release_device(v.first, false);
            *used -= freed;
            st.evictions += victims.size();
        }
        *used += need;
        *reserve += need;
        return 0;
    }

    struct Plan {
        std::vector<Request*> reqs;
        std::vector<fc_graph*> graphs;
        uint64_t reserve = 0;  // bytes: scratch and copies not yet resident
        uint32_t sms = 0;      // SMs the peel grid may cover (0 = all)
        bool heavy = false;
    };

    // Takes the requests of the next batch out of `pending` (under mu).
    //   * While few requests wait (fewer than backlog_requests, and not so
    //     for the last second either), a heavy request
    //     (heavy_visits or more) runs alone -- with the other pending
    //     requests of its graph -- on heavy_sms SMs, one at a time, in arrival
    //     order among heavy requests: its latency is most of the tail.  Light
    //     batches then leave a waiting heavy request its SMs, taking only
    //     what is free beyond them, so it waits at most for the batches
    //     already running.
    //   * With a backlog, every request batches in arrival order: a batch
    //     of many graphs shares its level loop, which is what keeps up with
    //     the load.
    //   * Every other batch takes at most half of the SMs (and at least a
    //     quarter, which a running heavy request leaves), so that two
    //     batches, their uploads and densest searches overlap on the device.
    // The grids of concurrent batches never claim more SMs than the device
    // has, so every persistent grid is resident as soon as it launches.
    void form_batch(Plan* p) {
        uint64_t used = fc::residency_bytes(&res) + running_bytes;
        std::set<fc_graph*> taken;
        Request* waiting_heavy = nullptr;
        const Clock::time_point now = Clock::now();
        if (pending.size() >= backlog_requests) last_backlog = now;
        const bool backlog = now - last_backlog < std::chrono::milliseconds(1000);
        if (!plain && !heavy_running && !backlog) {
            for (auto it = pending.begin(); it != pending.end(); ++it)
                if (is_heavy(*it) && !running_graphs.count((*it)->g)) {
                    waiting_heavy = *it;
                    break;
                }
        }
        if (waiting_heavy && free_sms >= heavy_sms &&
            running_requests < max_inflight) {
            Request* h = waiting_heavy;
            const int a = admit(h, &used, taken, &p->reserve);
            if (a == 1) {
                pending.erase(std::find(pending.begin(), pending.end(), h));
                return;  // rejected; the lane looks again
            }
            if (a == 0) {
                for (auto it = pending.begin(); it != pending.end();) {
                    if ((*it)->g == h->g) {
                        p->reqs.push_back(*it);
                        it = pending.erase(it);
                    } else {
                        ++it;
                    }
                }
                p->graphs.push_back(h->g);
                p->sms = heavy_sms;
                p->heavy = true;
                return;
            }
        }
        uint32_t cap = std::min(free_sms, std::max(min_light_sms, sms / 2));
        if (!plain) {
            if (waiting_heavy) cap = free_sms > heavy_sms ? std::min(cap, free_sms - heavy_sms) : 0;
            if (cap < min_light_sms) return;
        }
        for (auto it = pending.begin(); it != pending.end();) {
            Request* r = *it;
            // running on another lane, or a heavy request that runs alone later
            if (running_graphs.count(r->g) || (!backlog && is_heavy(r))) {
                ++it;
                continue;
            }
            if (taken.count(r->g)) {  // shares the peel of a graph already taken
                if (plain) break;
                p->reqs.push_back(r);
                it = pending.erase(it);
                continue;
            }
            if (p->graphs.size() >= max_batch_graphs ||
                running_requests + p->reqs.size() >= max_inflight)
                break;
            const int a = admit(r, &used, taken, &p->reserve);
            if (a == 1) {
                it = pending.erase(it);
                continue;
            }
            if (a == 2) break;  // wait for memory, in order
            taken.insert(r->g);
            p->graphs.push_back(r->g);
            p->reqs.push_back(r);
            it = pending.erase(it);
            if (plain) break;
        }
        p->sms = plain ? 0 : cap;
    }

    // The device work of one batch on the lane's stream.
    fc_status run_batch(cudaStream_t s, const Plan& p) {
        const std::vector<Request*>& batch = p.reqs;
        const std::vector<fc_graph*>& graphs = p.graphs;
        for (fc_graph* g : graphs) {
            const bool had = g->dev != nullptr;
            FC_TRY(fc::upload(g, s));
            if (!had) {
                std::lock_guard<std::mutex> lk(mu);
                st.uploads++;
            }
        }
        if (plain) {
            double ms = 0;
            uint32_t launches = 0, levels = 0;
            FC_TRY(fc::batch_plain_one(graphs[0], s, &ms, &launches, &levels));
        } else {
            FC_TRY(fc::batch_peel(graphs.data(), (uint32_t)graphs.size(), &bopt, p.sms, nullptr, s));
        }
        // densest: every request's beta, one pass per graph
        for (fc_graph* g : graphs) {
            std::vector<double> betas;
            std::vector<Request*> rs;
            for (Request* r : batch)
                if (r->g == g && r->res) {
                    betas.push_back(r->beta);
                    rs.push_back(r);
                }
            if (betas.empty()) continue;
            std::vector<fc_densest_result> out(betas.size());
            if (g->n && g->L) {
                FC_TRY(fc::densest(g, betas.data(), (uint32_t)betas.size(), out.data(), s));
            } else {
                for (size_t i = 0; i < out.size(); i++) {
                    out[i] = fc_densest_result{};
                    out[i].beta = betas[i];
                }
            }
            for (size_t i = 0; i < rs.size(); i++) *rs[i]->res = out[i];
        }
        for (Request* r : batch) {
            const uint64_t bytes = (uint64_t)r->g->n * r->g->L * 4;
            if (r->table && bytes)
                FC_TRY(fc::to_host(r->table, r->g->dev->table, bytes, s));
        }
        FC_CUDA_TRY(cudaStreamSynchronize(s));
        return FC_OK;
    }

    void lane_loop() {
        cudaStream_t s = nullptr;
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        fc::count_alloc(2);  // the stream and the staging buffer
        // this lane's copies go through its own pinned buffer
        fc::Staging stage;
        if (cudaHostAlloc(&stage.p, 16u << 20, cudaHostAllocDefault) == cudaSuccess)
            stage.cap = 16u << 20;
        else
            stage.p = nullptr;
        cudaGetLastError();
        fc::set_thread_staging(&stage);
        for (;;) {
            Plan p;
            {
                std::unique_lock<std::mutex> lk(mu);
                for (;;) {
                    if (stop && pending.empty()) break;
                    if (!pending.empty()) {
                        form_batch(&p);
                        if (!p.reqs.empty()) break;
                    }
                    // nothing to take now: wait for an arrival or a completion
                    cv_work.wait_for(lk, std::chrono::milliseconds(100));
                }
                if (p.reqs.empty()) break;  // stopped and nothing pending
                for (fc_graph* g : p.graphs) running_graphs.insert(g);
                running_bytes += p.reserve;
                running_requests += (uint32_t)p.reqs.size();
                if (!plain) free_sms -= p.sms;
                if (p.heavy) {
                    heavy_running = true;
                    st.heavy_batches++;
                }
                st.peak_bytes = std::max(st.peak_bytes, fc::residency_bytes(&res) + running_bytes);
                clock_advance();
                running_lanes++;
                st.batches++;
                st.graphs_peeled += p.graphs.size();
                st.max_batch = std::max<uint32_t>(st.max_batch, (uint32_t)p.reqs.size());
            }
            const fc_status rc = run_batch(s, p);
            if (rc != FC_OK) cudaStreamSynchronize(s);  // what was enqueued has finished
            // nothing is left in flight on the lane's stream, which goes away
            // with the server while the graphs may live on
            for (fc_graph* g : p.graphs) {
                if (!g->dev) continue;
                g->dev->home = nullptr;
                fc::residency_touch(&res, g, fc::graph_bytes(g));
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                clock_advance();
                running_lanes--;
                for (fc_graph* g : p.graphs) running_graphs.erase(g);
                running_bytes -= p.reserve;
                running_requests -= (uint32_t)p.reqs.size();
                if (!plain) free_sms += p.sms;
                if (p.heavy) heavy_running = false;
                for (Request* r : p.reqs) finish(r, rc);
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
        fc::set_thread_staging(nullptr);
        if (stage.p) cudaFreeHost(stage.p);
        if (s) cudaStreamDestroy(s);
    }
};

extern "C" {

fc_status fc_server_create(const fc_server_options* opt, fc_server** out) {
    if (!out) return FC_ERR_INVALID;
    *out = nullptr;
    if (!fc::cuda_available()) return FC_ERR_NO_DEVICE;
    fc_server* s = new fc_server();
    s->budget = (opt && opt->hbm_budget_bytes) ? opt->hbm_budget_bytes : 150ull * 1000 * 1000 * 1000;
    s->max_inflight = (opt && opt->max_inflight) ? opt->max_inflight : 256;
    s->plain = opt && opt->plain;
    s->lanes = s->plain ? 1 : ((opt && opt->lanes) ? opt->lanes : 2);
    s->max_batch_graphs = s->plain ? 1 : ((opt && opt->max_batch_graphs) ? opt->max_batch_graphs : 64);
    // every kernel loaded now: a kernel's first load may wait for kernels
    // running on other lanes
    fc::preload_kernels();
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    s->sms = s->free_sms = (uint32_t)(nsm > 0 ? nsm : 148);
    s->min_light_sms = std::max(1u, s->sms / 4);
    s->heavy_sms = s->sms - s->min_light_sms;
    s->heavy_visits = (opt && opt->heavy_visits) ? opt->heavy_visits : 1000000000ull;
    // fixed launch shape: serving does not stop to autotune every new mix
    s->bopt.block_threads = (opt && opt->block_threads) ? opt->block_threads : 1024;
    s->bopt.hub_threshold = (opt && opt->hub_threshold) ? opt->hub_threshold : 64;
    s->bopt.use_cuda_graph = 0;
    s->st.lanes = s->lanes;
    for (uint32_t i = 0; i < s->lanes; i++) s->threads.emplace_back([s] { s->lane_loop(); });
    *out = s;
    return FC_OK;
}

fc_status fc_server_submit(fc_server* s, fc_graph* g, double beta, uint32_t* table,
                           fc_densest_result* res, uint64_t* ticket) {
    if (!s || !g) return FC_ERR_INVALID;
    Request* r = new Request();
    r->g = g;
    r->beta = beta;
    r->table = table;
    r->res = res;
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            delete r;
            return FC_ERR_INVALID;
        }
        r->ticket = s->next_ticket++;
        s->all[r->ticket] = r;
        s->pending.push_back(r);
    }
    if (ticket) *ticket = r->ticket;
    s->cv_work.notify_all();
    return FC_OK;
}

fc_status fc_server_wait(fc_server* s, uint64_t ticket, int64_t timeout_ms, fc_status* status,
                         double* latency_ms) {
    if (!s) return FC_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return FC_ERR_INVALID;
    Request* r = it->second;
    auto pred = [&] { return r->done; };
    if (timeout_ms < 0) s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred))
        return FC_ERR_ITER_LIMIT;
    if (status) *status = r->status;
    if (latency_ms) *latency_ms = r->latency_ms;
    s->all.erase(it);
    delete r;
    return FC_OK;
}

fc_status fc_server_query(fc_server* s, fc_server_stats* out) {
    if (!s || !out) return FC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    s->clock_advance();
    *out = s->st;
    out->resident_bytes = fc::residency_bytes(&s->res);
    return FC_OK;
}

fc_status fc_server_destroy(fc_server* s) {
    if (!s) return FC_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->threads) t.join();
    fc::residency_drop(&s->res);
    for (auto& kv : s->all) delete kv.second;
    delete s;
    return FC_OK;
}

}  // extern "C"
