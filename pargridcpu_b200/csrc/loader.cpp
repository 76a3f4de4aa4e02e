// Host loader: the reference's MultilayerGraph::LoadFromFile semantics
// (Graph/MultilayerGraph.cpp:47-166) and Graph::BuildFromEdgeLst's CSR
// (Graph/Graph.cpp:17-50), producing fc_graph's host CSR.
#include <algorithm>
#include <atomic>
#include <thread>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "fc_internal.h"

namespace fc {

template <class T>
bool HostBuf<T>::alloc(size_t count) {
    reset();
    size_t bytes = (count ? count : 1) * sizeof(T);
    if (cuda_available() && cudaMallocHost((void**)&p, bytes) == cudaSuccess) {
        pinned = true;
        count_alloc();
    } else {
        cudaGetLastError();
        p = (T*)malloc(bytes);
        pinned = false;
    }
    n = count;
    return p != nullptr;
}

template <class T>
void HostBuf<T>::reset() {
    if (p) {
        if (pinned) cudaFreeHost(p);
        else free(p);
    }
    p = nullptr;
    n = 0;
    pinned = false;
}

template struct HostBuf<uint64_t>;
template struct HostBuf<uint32_t>;

namespace {

// Open-addressing map raw id -> internal id; ids are handed out in order of
// first sight (MultilayerGraph.cpp:127-143: u is looked up before v).
struct IdMap {
    // open addressing, one 8-byte slot per entry: key in the high half, id + 1
    // in the low half (0: empty), so a probe touches one cache line
    std::vector<uint64_t> tab;
    uint64_t mask = 0, size = 0;
    std::vector<uint64_t>* id2vtx;
    explicit IdMap(std::vector<uint64_t>* out) : id2vtx(out) { rehash(1 << 16); }
    static uint64_t h(uint32_t x) {
        uint64_t z = (uint64_t)x * 0x9E3779B97F4A7C15ull;
        return z ^ (z >> 29);
    }
    void rehash(uint64_t cap) {
        std::vector<uint64_t> t2(cap, 0);
        const uint64_t m2 = cap - 1;
        for (uint64_t s : tab) {
            if (!s) continue;
            uint64_t j = h((uint32_t)(s >> 32)) & m2;
            while (t2[j]) j = (j + 1) & m2;
            t2[j] = s;
        }
        tab.swap(t2);
        mask = m2;
    }
    // the lookup of x is about to come: bring its first slot in
    void prefetch(uint32_t x) const { __builtin_prefetch(tab.data() + (h(x) & mask)); }
    uint32_t get(uint32_t x) {
        uint64_t j = h(x) & mask;
        for (uint64_t s; (s = tab[j]) != 0; j = (j + 1) & mask)
            if ((uint32_t)(s >> 32) == x) return (uint32_t)s - 1;
        const uint32_t id = (uint32_t)size++;
        tab[j] = ((uint64_t)x << 32) | ((uint64_t)id + 1);
        id2vtx->push_back(x);
        if (size * 2 > mask) rehash((mask + 1) * 2);
        return id;
    }
};

bool read_file(const std::string& path, std::vector<char>& buf) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return false;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    buf.resize(sz > 0 ? (size_t)sz : 0);
    size_t got = sz > 0 ? fread(buf.data(), 1, (size_t)sz, f) : 0;
    fclose(f);
    return got == buf.size();
}

// The layer-file loop of MultilayerGraph::LoadLayer (:122-156):
//     while (in.peek() != EOF) { in >> u >> v; if (u != v) keep(u, v); }
// with `uint u, v` and C++11 stream rules: an extraction that finds only
// whitespace before the end leaves its variable unchanged and fails the
// stream; one that finds no digit stores 0 and fails; an out-of-range value
// stores UINT_MAX and fails; a leading '-' negates modulo 2^32; reading the
// last digit sets end-of-file.  Once failed or at end, peek() is EOF.  A pair
// read before either variable was ever assigned is undefined in the
// reference and is dropped here.
struct PairParser {
    const char* p;
    const char* e;
    bool fail = false, eof = false;
    static bool ws(char c) {
        return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
    }
    // returns true when val was assigned
    bool extract(uint32_t& val) {
        if (fail || eof) {
            fail = true;
            return false;
        }
        while (p < e && ws(*p)) p++;
        if (p >= e) {
            eof = fail = true;
            return false;
        }
        bool neg = false;
        if (*p == '+' || *p == '-') {
            neg = *p == '-';
            p++;
        }
        const char* s = p;
        uint64_t mag = 0;
        bool over = false;
        while (p < e && *p >= '0' && *p <= '9') {
            if (!over) {
                mag = mag * 10 + (uint64_t)(*p - '0');
                if (mag > 0xFFFFFFFFull) over = true;
            }
            p++;
        }
        if (p >= e) eof = true;
        if (p == s) {
            fail = true;
            val = 0;
            return true;
        }
        if (over) {
            fail = true;
            val = 0xFFFFFFFFu;
            return true;
        }
        val = neg ? (uint32_t)(0u - (uint32_t)mag) : (uint32_t)mag;
        return true;
    }
};

void parse_pairs(const std::vector<char>& text, std::vector<uint32_t>& out) {
    PairParser ps{text.data(), text.data() + text.size()};
    uint32_t u = 0, v = 0;
    bool have_u = false, have_v = false;
    out.clear();
    out.reserve(text.size() / 6);
    while (!(ps.fail || ps.eof || ps.p >= ps.e)) {
        if (ps.extract(u)) have_u = true;
        if (ps.extract(v)) have_v = true;
        if (have_u && have_v && u != v) {
            out.push_back(u);
            out.push_back(v);
        }
    }
}

// Per-layer CSR from remapped directed pairs: rows ascending, duplicates
// dropped (Graph.cpp:27-47).  Counting sort by source, then each row sorted.
// C: the count type, 32-bit when the layer's entries fit (half the bytes of
// the two randomly written count arrays)
// f(lo, hi) over node ranges [lo, hi) of about equal entry counts (by the
// row prefix `cnt`), on `threads` host threads.
template <class C, class F>
void for_node_ranges(uint32_t n, const std::vector<C>& cnt, unsigned threads, F f) {
    if (threads <= 1 || n < 4096) {
        f(0u, n);
        return;
    }
    const uint64_t total = cnt[n];
    std::vector<uint32_t> cut(threads + 1, n);
    cut[0] = 0;
    for (unsigned t = 1; t < threads; t++) {
        const uint64_t want = total * t / threads;  // first row starting at or after it
        cut[t] = (uint32_t)(std::lower_bound(cnt.begin(), cnt.begin() + n, (C)want) - cnt.begin());
        if (cut[t] < cut[t - 1]) cut[t] = cut[t - 1];
    }
    std::vector<std::thread> th;
    for (unsigned t = 0; t < threads; t++) th.emplace_back([&, t] { f(cut[t], cut[t + 1]); });
    for (auto& x : th) x.join();
}

template <class C>
void build_layer_t(uint32_t n, const std::vector<uint32_t>& dir_pairs, std::vector<uint64_t>& off,
                   std::vector<uint32_t>& adj, unsigned threads) {
    uint64_t m = dir_pairs.size() / 2;
    std::vector<C> cnt((size_t)n + 1, 0);
    for (uint64_t i = 0; i < m; i++) cnt[dir_pairs[2 * i] + 1]++;
    for (uint32_t v = 0; v < n; v++) cnt[v + 1] += cnt[v];
    std::vector<uint32_t> tgt(m);
    std::vector<C> pos(cnt.begin(), cnt.end() - 1);
    for (uint64_t i = 0; i < m; i++) tgt[pos[dir_pairs[2 * i]]++] = dir_pairs[2 * i + 1];
    std::vector<C>().swap(pos);
    // each row sorted in place with its distinct neighbours moved to its
    // front (the reference's sort + dedupe, Graph.cpp:17-50), then the
    // distinct ones copied out: both passes over node ranges in parallel
    std::vector<uint32_t> uniq(n);
    for_node_ranges(n, cnt, threads, [&](uint32_t lo, uint32_t hi) {
        for (uint32_t v = lo; v < hi; v++) {
            uint32_t* b = tgt.data() + cnt[v];
            uint32_t* e = tgt.data() + cnt[v + 1];
            std::sort(b, e);
            uint32_t* w = b;
            for (uint32_t* q = b; q < e; q++)
                if (q == b || *q != q[-1]) *w++ = *q;
            uniq[v] = (uint32_t)(w - b);
        }
    });
    off.assign((size_t)n + 1, 0);
    for (uint32_t v = 0; v < n; v++) off[v + 1] = off[v] + uniq[v];
    adj.resize(off[n]);
    for_node_ranges(n, cnt, threads, [&](uint32_t lo, uint32_t hi) {
        for (uint32_t v = lo; v < hi; v++)
            if (uniq[v]) memcpy(adj.data() + off[v], tgt.data() + cnt[v], uniq[v] * 4ull);
    });
}

void build_layer(uint32_t n, const std::vector<uint32_t>& dir_pairs, std::vector<uint64_t>& off,
                 std::vector<uint32_t>& adj, unsigned threads) {
    if (dir_pairs.size() / 2 < (1ull << 32)) build_layer_t<uint32_t>(n, dir_pairs, off, adj, threads);
    else build_layer_t<uint64_t>(n, dir_pairs, off, adj, threads);
}

// f(l) for every layer l, on up to one host thread per core (layers are
// independent once their ids are assigned).
template <class F>
void for_each_layer(uint32_t L, F f) {
    unsigned hw = std::thread::hardware_concurrency();
    const uint32_t nt = std::min<uint32_t>(L, hw ? hw : 4);
    if (nt <= 1) {
        for (uint32_t l = 0; l < L; l++) f(l);
        return;
    }
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> th;
    for (uint32_t t = 0; t < nt; t++)
        th.emplace_back([&] {
            for (uint32_t l; (l = next.fetch_add(1)) < L;) f(l);
        });
    for (auto& t : th) t.join();
}

fc_status finish(uint32_t n, uint32_t L, std::vector<std::vector<uint32_t>>& dir_pairs, fc_graph* g) {
    g->n = n;
    g->L = L;
    g->order.resize(L);
    for (uint32_t i = 0; i < L; i++) g->order[i] = i;
    std::vector<std::vector<uint64_t>> offs(L);
    std::vector<std::vector<uint32_t>> adjs(L);
    // layers in parallel; the cores beyond L help inside each layer
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned per_layer = L && hw > L ? hw / L : 1u;
    for_each_layer(L, [&](uint32_t l) {
        build_layer(n, dir_pairs[l], offs[l], adjs[l], per_layer);
        std::vector<uint32_t>().swap(dir_pairs[l]);
    });
    std::vector<uint64_t> base(L + 1, 0);
    for (uint32_t l = 0; l < L; l++) base[l + 1] = base[l] + adjs[l].size();
    if (base[L] >= (1ull << 32)) return FC_ERR_TOO_LARGE;  // 32-bit offsets
    if (!g->off.alloc((uint64_t)L * (n + 1)) || !g->adj.alloc(base[L])) return FC_ERR_OOM;
    for_each_layer(L, [&](uint32_t l) {
        uint32_t* o = g->off.p + (uint64_t)l * (n + 1);
        for (uint32_t v = 0; v <= n; v++) o[v] = (uint32_t)(base[l] + offs[l][v]);
        if (!adjs[l].empty()) memcpy(g->adj.p + base[l], adjs[l].data(), adjs[l].size() * 4);
        std::vector<uint32_t>().swap(adjs[l]);
    });
    return FC_OK;
}

}  // namespace

fc_status build_from_pairs(uint32_t L, const uint64_t* m, const uint32_t* pairs, fc_graph* g) {
    IdMap map(&g->id2vtx);
    std::vector<std::vector<uint32_t>> dir(L);
    const uint32_t* p = pairs;
    for (uint32_t l = 0; l < L; l++) {
        dir[l].reserve(2 * m[l] * 2);
        for (uint64_t i = 0; i < m[l]; i++, p += 2) {
            if (i + 8 < m[l]) {  // the slots 8 pairs ahead
                map.prefetch(p[16]);
                map.prefetch(p[17]);
            }
            uint32_t u = p[0], v = p[1];
            if (u == v) continue;  // MultilayerGraph.cpp:126
            uint32_t a = map.get(u), b = map.get(v);
            dir[l].push_back(a);
            dir[l].push_back(b);
            dir[l].push_back(b);
            dir[l].push_back(a);
        }
    }
    return finish((uint32_t)map.size, L, dir, g);
}

fc_status load_dir(const std::string& dir, int order, bool write_vtx_map, fc_graph* g) {
    // mlg.conf: one layer file name per non-empty line (GetGraphFile, :47-63);
    // lines are split on '\n' only, as std::getline does.
    std::vector<char> conf;
    if (!read_file(dir + "mlg.conf", conf)) return FC_ERR_IO;
    std::vector<std::string> files;
    std::string line;
    for (size_t i = 0; i <= conf.size(); i++) {
        if (i == conf.size() || conf[i] == '\n') {
            if (!line.empty()) files.push_back(line);
            line.clear();
        } else {
            line.push_back(conf[i]);
        }
    }
    uint32_t L = (uint32_t)files.size();
    // read and parse the layer files in parallel; ids are then handed out in
    // one pass in file order, as the reference's sequential load does
    std::vector<std::vector<uint32_t>> raw(L);
    std::vector<char> io_ok(L, 0);
    for_each_layer(L, [&](uint32_t l) {
        std::vector<char> text;
        if (!read_file(dir + files[l], text)) return;
        parse_pairs(text, raw[l]);
        io_ok[l] = 1;
    });
    for (uint32_t l = 0; l < L; l++)
        if (!io_ok[l]) return FC_ERR_IO;
    IdMap map(&g->id2vtx);
    std::vector<std::vector<uint32_t>> dir_pairs(L);
    for (uint32_t l = 0; l < L; l++) {
        auto& d = dir_pairs[l];
        d.reserve(raw[l].size() * 2);
        const size_t nr = raw[l].size();
        for (size_t i = 0; i < nr; i += 2) {
            // the table outgrows the caches: fetch the slots 16 ids ahead
            if (i + 16 < nr) {
                map.prefetch(raw[l][i + 16]);
                map.prefetch(raw[l][i + 17]);
            }
            uint32_t a = map.get(raw[l][i]), b = map.get(raw[l][i + 1]);
            d.push_back(a);
            d.push_back(b);
            d.push_back(b);
            d.push_back(a);
        }
        std::vector<uint32_t>().swap(raw[l]);
    }
    if (write_vtx_map) {
        // `u uid` per new id, in assignment order (MultilayerGraph.cpp:131,139)
        FILE* f = fopen((dir + "__vtx_map.txt").c_str(), "wb");
        if (!f) return FC_ERR_IO;
        std::string out;
        out.reserve(g->id2vtx.size() * 22);
        char b[48];
        // decimal digits of x, written backwards from e; returns the start
        auto digits = [](uint64_t x, char* e) {
            do {
                *--e = (char)('0' + x % 10);
                x /= 10;
            } while (x);
            return e;
        };
        for (size_t i = 0; i < g->id2vtx.size(); i++) {
            char* e = b + sizeof(b);
            *--e = '\n';
            e = digits(i, e);
            *--e = ' ';
            e = digits((uint32_t)g->id2vtx[i], e);
            out.append(e, (size_t)(b + sizeof(b) - e));
        }
        bool ok = fwrite(out.data(), 1, out.size(), f) == out.size();
        ok = (fclose(f) == 0) && ok;
        if (!ok) return FC_ERR_IO;
    }
    FC_TRY(finish((uint32_t)map.size, L, dir_pairs, g));
    apply_order(order, g);
    return FC_OK;
}

fc_status build_from_adjbuf(uint32_t n, uint32_t L, const uint32_t* const* bufs, const uint64_t* m,
                            fc_graph* g) {
    g->n = n;
    g->L = L;
    g->order.resize(L);
    g->id2vtx.resize(n);
    for (uint32_t v = 0; v < n; v++) g->id2vtx[v] = v;
    for (uint32_t i = 0; i < L; i++) g->order[i] = i;
    uint64_t total = 0;
    for (uint32_t l = 0; l < L; l++) total += m[l];
    if (total >= (1ull << 32)) return FC_ERR_TOO_LARGE;  // 32-bit offsets
    if (!g->off.alloc((uint64_t)L * (n + 1)) || !g->adj.alloc(total)) return FC_ERR_OOM;
    uint64_t base = 0;
    for (uint32_t l = 0; l < L; l++) {
        const uint32_t* b = bufs[l];
        uint32_t* o = g->off.p + (uint64_t)l * (n + 1);
        uint64_t r = 0, w = base;
        for (uint32_t v = 0; v < n; v++) {
            o[v] = (uint32_t)w;
            uint32_t d = b[r++];
            if (w + d > base + m[l]) return FC_ERR_PARSE;
            for (uint32_t j = 0; j < d; j++) {
                uint32_t u = b[r++];
                if (u >= n || u == v || (j && u <= g->adj[w - 1])) return FC_ERR_PARSE;
                g->adj[w++] = u;
            }
        }
        if (w != base + m[l]) return FC_ERR_PARSE;
        o[n] = (uint32_t)w;
        base = w;
    }
    return FC_OK;
}

// SetGraphOrder (MultilayerGraph.cpp:9-45): 1/2 sort layers by
// (float)(m>>1)/(float)n ascending/descending, 3/4 by m; the same std::sort
// calls on the same input give the same permutation.
void apply_order(int o, fc_graph* g) {
    uint32_t L = g->L, n = g->n;
    if (o == 0 || L == 0) return;
    std::vector<uint32_t> ord(L);
    for (uint32_t i = 0; i < L; i++) ord[i] = i;
    std::vector<uint32_t> ms(L);
    for (uint32_t i = 0; i < L; i++) ms[i] = (uint32_t)g->layer_m(i);
    if (o == 1 || o == 2) {
        std::vector<float> density(L);
        for (uint32_t i = 0; i < L; i++) density[i] = (float)(ms[i] >> 1) / (float)n;
        if (o == 1)
            std::sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return density[a] < density[b]; });
        else
            std::sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return density[a] > density[b]; });
    } else if (o == 3 || o == 4) {
        if (o == 3)
            std::sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return ms[a] < ms[b]; });
        else
            std::sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return ms[a] > ms[b]; });
    } else {
        return;
    }
    HostBuf<uint32_t> off2;
    HostBuf<uint32_t> adj2;
    uint64_t total = g->total_entries();
    if (!off2.alloc((uint64_t)L * (n + 1)) || !adj2.alloc(total)) return;
    uint64_t base = 0;
    for (uint32_t i = 0; i < L; i++) {
        const uint32_t* src = g->off.p + (uint64_t)ord[i] * (n + 1);
        uint32_t* dst = off2.p + (uint64_t)i * (n + 1);
        uint64_t len = src[n] - src[0];
        for (uint32_t v = 0; v <= n; v++) dst[v] = (uint32_t)(base + (src[v] - src[0]));
        if (len) memcpy(adj2.p + base, g->adj.p + src[0], len * 4);
        base += len;
    }
    std::swap(g->off.p, off2.p);
    std::swap(g->off.pinned, off2.pinned);
    std::swap(g->adj.p, adj2.p);
    std::swap(g->adj.pinned, adj2.pinned);
    std::vector<uint32_t> composed(L);
    for (uint32_t i = 0; i < L; i++) composed[i] = g->order[ord[i]];
    g->order = composed;
}

}  // namespace fc
