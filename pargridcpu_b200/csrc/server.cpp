// Request loop: admits decomposition + densest requests by device-memory
// footprint and in-flight slots, runs them, and completes each independently.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "fc_internal.h"

namespace {

struct Request {
    uint64_t ticket;
    fc_graph* g;
    double beta;
    uint32_t* table;
    fc_densest_result* res;
    uint64_t footprint;
    std::chrono::steady_clock::time_point t_submit;
    fc_status status = FC_OK;
    double latency_ms = 0.0;
    bool done = false;
};

// Device bytes a request holds while it runs: CSR, table, peel scratch for
// one column group and the densest histograms (an upper estimate).
uint64_t footprint(const fc_graph* g) {
    uint64_t n = g->n, L = g->L, e = g->total_entries();
    uint64_t csr = 4 * (n + 1) + 4 * e + 4 * n * L;
    uint64_t table = 8 * n * L;
    uint64_t peel = 4 * (n * L * L + 8 * n * L);
    return csr + table + peel + (64ull << 20);
}

}  // namespace

struct fc_server {
    uint64_t budget;
    uint32_t max_inflight;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::map<uint64_t, Request*> all;
    uint64_t next_ticket = 1;
    uint64_t inflight_bytes = 0;
    uint32_t inflight = 0;
    bool stop = false;
    std::vector<std::thread> workers;
    std::mutex gpu_mu;  // one decomposition on the device at a time

    void worker() {
        cudaStream_t s = nullptr;
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        for (;;) {
            Request* r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] {
                    if (stop) return true;
                    if (queue.empty()) return false;
                    Request* h = queue.front();
                    return inflight < max_inflight &&
                           (inflight == 0 || inflight_bytes + h->footprint <= budget);
                });
                if (stop && queue.empty()) break;
                if (queue.empty()) continue;
                r = queue.front();
                queue.pop_front();
                inflight++;
                inflight_bytes += r->footprint;
            }
            fc_status st = FC_OK;
            if (r->footprint > budget) st = FC_ERR_BUDGET;
            if (st == FC_OK) st = fc::upload(r->g, s);
            if (st == FC_OK) {
                std::lock_guard<std::mutex> g(gpu_mu);
                st = fc::coreindex(r->g, r->table, false, s);
                if (st == FC_OK && r->res) {
                    if (r->g->n && r->g->L) st = fc::densest(r->g, &r->beta, 1, r->res, s);
                    else {
                        memset(r->res, 0, sizeof(*r->res));
                        r->res->beta = r->beta;
                    }
                }
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                r->status = st;
                r->latency_ms = std::chrono::duration<double, std::milli>(
                                    std::chrono::steady_clock::now() - r->t_submit)
                                    .count();
                r->done = true;
                inflight--;
                inflight_bytes -= r->footprint;
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
        if (s) cudaStreamDestroy(s);
    }
};

extern "C" {

fc_status fc_server_create(const fc_server_options* opt, fc_server** out) {
    if (!out) return FC_ERR_INVALID;
    if (!fc::cuda_available()) return FC_ERR_NO_DEVICE;
    fc_server* s = new fc_server();
    s->budget = (opt && opt->hbm_budget_bytes) ? opt->hbm_budget_bytes : 150ull * 1000 * 1000 * 1000;
    s->max_inflight = (opt && opt->max_inflight) ? opt->max_inflight : 16;
    for (uint32_t i = 0; i < s->max_inflight; i++) s->workers.emplace_back([s] { s->worker(); });
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
    r->footprint = footprint(g);
    r->t_submit = std::chrono::steady_clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->ticket = s->next_ticket++;
        s->all[r->ticket] = r;
        s->queue.push_back(r);
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

fc_status fc_server_destroy(fc_server* s) {
    if (!s) return FC_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto& kv : s->all) delete kv.second;
    delete s;
    return FC_OK;
}

}  // extern "C"
