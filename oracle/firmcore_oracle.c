/* Test infrastructure, not product code: the CPU oracle (see
 * firmcore_oracle.h).  Every function below restates one piece of the
 * reference (kouteisang/ParGridCPU) and cites the lines it follows.  Plain C,
 * single thread, no SIMD, no -ffast-math: the floating-point expressions are
 * evaluated in the same types and order as the reference's.
 */
#include "firmcore_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct oracle_graph {
    uint32_t n, L;
    uint64_t* off;     /* L*(n+1): row v of layer l is adj[off[l*(n+1)+v] .. off[l*(n+1)+v+1]) */
    uint32_t* adj;
    uint64_t* id2vtx;  /* n entries */
};

/* ---- id remap: open-addressing hash, key = raw id, value = internal id ---- */
typedef struct {
    uint64_t cap;
    uint32_t* key;
    uint32_t* val;
    uint8_t* used;
} idmap;

static int idmap_init(idmap* m, uint64_t cap) {
    m->cap = 16;
    while (m->cap < cap * 2) m->cap <<= 1;
    m->key = (uint32_t*)malloc(m->cap * 4);
    m->val = (uint32_t*)malloc(m->cap * 4);
    m->used = (uint8_t*)calloc(m->cap, 1);
    return m->key && m->val && m->used ? 0 : -1;
}
static void idmap_free(idmap* m) { free(m->key); free(m->val); free(m->used); }
static uint64_t hash32(uint32_t x) {
    uint64_t h = (uint64_t)x * 0x9E3779B97F4A7C15ull;
    return h ^ (h >> 29);
}
/* Returns the internal id of raw id x, assigning the next id on first sight
 * (MultilayerGraph.cpp:127-143: lookup u, then v; new ids are num_of_vtx++). */
static uint32_t idmap_get(idmap* m, uint32_t x, uint32_t* next, uint64_t* id2vtx) {
    uint64_t i = hash32(x) & (m->cap - 1);
    while (m->used[i]) {
        if (m->key[i] == x) return m->val[i];
        i = (i + 1) & (m->cap - 1);
    }
    m->used[i] = 1;
    m->key[i] = x;
    m->val[i] = *next;
    id2vtx[*next] = x;
    return (*next)++;
}

/* LSD radix sort of 64-bit keys (s << 32 | t): the same order as the
 * reference's std::sort on edge{s,t} (Graph.h:17-19, Graph.cpp:27). */
static void radix_sort_u64(uint64_t* a, uint64_t* tmp, uint64_t len) {
    for (int pass = 0; pass < 4; pass++) {
        uint64_t cnt[65537];
        memset(cnt, 0, sizeof(cnt));
        int sh = 16 * pass;
        for (uint64_t i = 0; i < len; i++) cnt[((a[i] >> sh) & 0xFFFF) + 1]++;
        for (int b = 0; b < 65536; b++) cnt[b + 1] += cnt[b];
        for (uint64_t i = 0; i < len; i++) tmp[cnt[(a[i] >> sh) & 0xFFFF]++] = a[i];
        memcpy(a, tmp, len * 8);
    }
}

int oracle_graph_from_pairs(uint32_t L, const uint64_t* m, const uint32_t* pairs,
                            oracle_graph** out) {
    uint64_t total = 0;
    for (uint32_t l = 0; l < L; l++) total += m[l];
    oracle_graph* g = (oracle_graph*)calloc(1, sizeof(*g));
    idmap map;
    if (!g || idmap_init(&map, 2 * total + 16)) return -1;
    uint64_t* id2vtx = (uint64_t*)malloc((2 * total + 1) * 8);
    uint64_t** keys = (uint64_t**)calloc(L ? L : 1, sizeof(uint64_t*));
    uint64_t* nkeys = (uint64_t*)calloc(L ? L : 1, 8);
    uint32_t next = 0;
    const uint32_t* p = pairs;
    /* LoadLayer, MultilayerGraph.cpp:104-166: drop self-loops (:126), remap
     * u then v, push (u,v) and (v,u) (:154-155). */
    for (uint32_t l = 0; l < L; l++) {
        keys[l] = (uint64_t*)malloc((2 * m[l] + 1) * 8);
        uint64_t ne = 0;
        for (uint64_t i = 0; i < m[l]; i++, p += 2) {
            uint32_t u = p[0], v = p[1];
            if (u == v) continue;
            uint32_t uid = idmap_get(&map, u, &next, id2vtx);
            uint32_t vid = idmap_get(&map, v, &next, id2vtx);
            keys[l][ne++] = ((uint64_t)uid << 32) | vid;
            keys[l][ne++] = ((uint64_t)vid << 32) | uid;
        }
        nkeys[l] = ne;
    }
    idmap_free(&map);
    uint32_t n = next; /* MultilayerGraph.cpp:95, n = |vtx2id| */
    g->n = n;
    g->L = L;
    g->id2vtx = (uint64_t*)malloc(((uint64_t)n + 1) * 8);
    memcpy(g->id2vtx, id2vtx, (uint64_t)n * 8);
    free(id2vtx);
    g->off = (uint64_t*)calloc((uint64_t)L * (n + 1) + 1, 8);
    uint64_t adj_total = 0;
    for (uint32_t l = 0; l < L; l++) adj_total += nkeys[l];
    g->adj = (uint32_t*)malloc((adj_total + 1) * 4);
    /* BuildFromEdgeLst, Graph.cpp:17-50: sort, then drop repeated (s,t). */
    uint64_t pos = 0;
    for (uint32_t l = 0; l < L; l++) {
        uint64_t ne = nkeys[l];
        uint64_t* tmp = (uint64_t*)malloc((ne + 1) * 8);
        radix_sort_u64(keys[l], tmp, ne);
        free(tmp);
        uint64_t* off = g->off + (uint64_t)l * (n + 1);
        uint64_t i = 0;
        for (uint32_t v = 0; v < n; v++) {
            off[v] = pos;
            while (i < ne && (uint32_t)(keys[l][i] >> 32) == v) {
                if (!(i > 0 && keys[l][i] == keys[l][i - 1])) g->adj[pos++] = (uint32_t)keys[l][i];
                i++;
            }
        }
        off[n] = pos;
        free(keys[l]);
    }
    free(keys);
    free(nkeys);
    *out = g;
    return 0;
}

void oracle_graph_free(oracle_graph* g) {
    if (!g) return;
    free(g->off);
    free(g->adj);
    free(g->id2vtx);
    free(g);
}
uint32_t oracle_n(const oracle_graph* g) { return g->n; }
uint32_t oracle_layers(const oracle_graph* g) { return g->L; }
uint64_t oracle_layer_m(const oracle_graph* g, uint32_t l) {
    const uint64_t* off = g->off + (uint64_t)l * (g->n + 1);
    return off[g->n] - off[0];
}
void oracle_id2vtx(const oracle_graph* g, uint64_t* out) { memcpy(out, g->id2vtx, (uint64_t)g->n * 8); }
void oracle_csr(const oracle_graph* g, uint64_t* off, uint32_t* adj) {
    uint64_t no = (uint64_t)g->L * (g->n + 1);
    memcpy(off, g->off, no * 8);
    uint64_t na = g->L ? g->off[no - 1] : 0;
    memcpy(adj, g->adj, na * 4);
}

static inline uint32_t layer_deg(const oracle_graph* g, uint32_t l, uint32_t v) {
    const uint64_t* off = g->off + (uint64_t)l * (g->n + 1);
    return (uint32_t)(off[v + 1] - off[v]);
}

/* findLmdthLargest, CoreIndex.cpp:46-58: the lmd-th largest of a node's L
 * degrees -- copy, sort descending, take [lmd-1]. */
static int cmp_u32_desc(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x > y ? -1 : (x < y);
}
static uint32_t lmd_th_largest(const uint32_t* d, uint32_t lmd, uint32_t L, uint32_t* scratch) {
    memcpy(scratch, d, L * 4);
    if (L <= 32) {
        for (uint32_t i = 1; i < L; i++) {
            uint32_t x = scratch[i], j = i;
            while (j > 0 && scratch[j - 1] < x) { scratch[j] = scratch[j - 1]; j--; }
            scratch[j] = x;
        }
    } else {
        qsort(scratch, L, 4, cmp_u32_desc);
    }
    return scratch[lmd - 1];
}

/* get_index2, CoreIndex.cpp:62-109, for one lambda.  Buckets B[0..n] hold
 * nodes by their current Top-lambda i_v; nodes are popped in increasing k;
 * a popped node fixes i_v = k and decrements its not-yet-popped neighbours'
 * layer degrees (:86-96; neighbours with i_v <= k are skipped, :90); a
 * neighbour whose degree drops from exactly i_v gets its Top-lambda recomputed
 * and is re-bucketed at max(i_v, k) (:92-102).  The std::set buckets are
 * restated as doubly linked lists; the order nodes leave one bucket does not
 * change the result, the core index being unique. */
static void coreindex_one(const oracle_graph* g, uint32_t lmd, uint32_t* deg /* n*L */,
                          uint32_t* iv /* n, out */) {
    uint32_t n = g->n, L = g->L;
    uint32_t* head = (uint32_t*)malloc(((uint64_t)n + 1) * 4);
    uint32_t* nxt = (uint32_t*)malloc((uint64_t)n * 4 + 4);
    uint32_t* prv = (uint32_t*)malloc((uint64_t)n * 4 + 4);
    uint32_t* scratch = (uint32_t*)malloc((uint64_t)L * 4 + 4);
    uint32_t* touched = (uint32_t*)malloc((uint64_t)n * 4 + 4);
    uint8_t* mark = (uint8_t*)calloc(n + 1, 1);
    const uint32_t NIL = 0xFFFFFFFFu;
    for (uint32_t k = 0; k <= n; k++) head[k] = NIL;
#define B_INSERT(b, v) do { nxt[v] = head[b]; prv[v] = NIL; if (head[b] != NIL) prv[head[b]] = v; head[b] = v; } while (0)
#define B_ERASE(b, v) do { if (prv[v] != NIL) nxt[prv[v]] = nxt[v]; else head[b] = nxt[v]; if (nxt[v] != NIL) prv[nxt[v]] = prv[v]; } while (0)
    uint32_t* bucket_of = (uint32_t*)malloc((uint64_t)n * 4 + 4);
    for (uint32_t v = 0; v < n; v++) {
        iv[v] = lmd_th_largest(deg + (uint64_t)v * L, lmd, L, scratch);
        bucket_of[v] = iv[v];
        B_INSERT(iv[v], v);
    }
    for (uint32_t k = 0; k <= n; k++) {
        while (head[k] != NIL) {
            uint32_t vv = head[k];
            B_ERASE(k, vv);
            bucket_of[vv] = NIL;
            iv[vv] = k;
            uint32_t nt = 0;
            for (uint32_t l = 0; l < L; l++) {
                const uint64_t* off = g->off + (uint64_t)l * (n + 1);
                for (uint64_t e = off[vv]; e < off[vv + 1]; e++) {
                    uint32_t u = g->adj[e];
                    if (iv[u] <= k) continue;
                    uint32_t* d = deg + (uint64_t)u * L + l;
                    *d -= 1;
                    if (*d + 1 == iv[u] && !mark[u]) { mark[u] = 1; touched[nt++] = u; }
                }
            }
            for (uint32_t i = 0; i < nt; i++) {
                uint32_t u = touched[i];
                mark[u] = 0;
                B_ERASE(bucket_of[u], u);
                iv[u] = lmd_th_largest(deg + (uint64_t)u * L, lmd, L, scratch);
                uint32_t b = iv[u] > k ? iv[u] : k;
                bucket_of[u] = b;
                B_INSERT(b, u);
            }
        }
    }
#undef B_INSERT
#undef B_ERASE
    free(head); free(nxt); free(prv); free(scratch); free(touched); free(mark); free(bucket_of);
}

/* CoreIndex::Execute, CoreIndex.cpp:168-213: per lambda a fresh degree table
 * degs[v][l] = |N_l(v)| (:189-197), then get_index2. */
int oracle_coreindex(const oracle_graph* g, uint32_t* table) {
    uint32_t n = g->n, L = g->L;
    if (!n) return 0;
    uint32_t* deg = (uint32_t*)malloc((uint64_t)n * L * 4);
    if (!deg) return -1;
    for (uint32_t lmd = 1; lmd <= L; lmd++) {
        for (uint32_t v = 0; v < n; v++)
            for (uint32_t l = 0; l < L; l++) deg[(uint64_t)v * L + l] = layer_deg(g, l, v);
        coreindex_one(g, lmd, deg, table + (uint64_t)(lmd - 1) * n);
    }
    free(deg);
    return 0;
}

typedef struct { uint32_t id; double degree; } layer_degree;

static int cmp_layer_desc(const void* a, const void* b) {
    double x = ((const layer_degree*)a)->degree, y = ((const layer_degree*)b)->degree;
    if (x > y) return -1;
    if (x < y) return 1;
    uint32_t i = ((const layer_degree*)a)->id, j = ((const layer_degree*)b)->id;
    return i < j ? -1 : (i > j);
}

/* The WDS block of FCPathLevelLeft::constructCore, Core/FCPathLevelLeft.cpp:57-99,
 * for one cell with |C| = length and e2[l] = sum over v in C of deg_C(v,l):
 *   degree_l = e2_l*1.0f/2            float arithmetic, stored as double (:66)
 *   sort layers by degree descending  (:72)
 *   for l = 1..L: d = degree_(l)*1.0f / length * 1.0 * pow(l, beta)   (:81-82)
 *                 if d >= best: best = d, lstar = l   (best starts at 0.0, :85-90)
 * Ties keep the larger l.  ld receives the sorted layers (ties by layer id). */
static double cell_density(const uint32_t* e2, uint32_t L, uint32_t length, const double* powl,
                           layer_degree* ld, uint32_t* lstar) {
    for (uint32_t l = 0; l < L; l++) {
        uint32_t num_edge = e2[l];
        float f = num_edge * 1.0f / 2;
        ld[l].id = l;
        ld[l].degree = f;
    }
    qsort(ld, L, sizeof(layer_degree), cmp_layer_desc);
    double best = 0.0;
    *lstar = 0;
    for (uint32_t l = 0; l < L; l++) {
        double mad = (ld[l].degree * 1.0f) / (length) * 1.0;
        double d = mad * powl[l];
        if (d >= best) {
            best = d;
            *lstar = l + 1;
        }
    }
    return best;
}

/* WdsList: per-cell densities over the fcgrid tree built by
 * FCPathLevelLeft::Execute, then FCTree::WeightDenestSubgraph
 * (Core/FCTree.cpp:69-82) over the tree in preorder -- node, left child
 * (k+1), right child (lambda+1) -- which is lambda-major, k ascending.  The
 * running maximum is a float (main.cpp:406) compared as
 * `node->layer_density >= maximum_density` (FCTree.cpp:73), so a later cell
 * wins ties and near-ties within float rounding.
 *
 * e2_l of every cell comes from the core table: C_{k,lambda} is
 * {v : core_lambda(v) >= k}, and deg_C(v,l) is v's layer-l neighbours inside
 * it.  Cells are walked from the largest k down, adding the nodes with
 * core == k each time (uint32 sums, wrapping like the reference's `uint
 * num_edge`). */
int oracle_densest(const oracle_graph* g, const uint32_t* table, double beta,
                   oracle_densest_result* res, oracle_cell* cells, uint32_t cells_cap,
                   uint32_t* nodes, uint32_t* layers) {
    uint32_t n = g->n, L = g->L;
    memset(res, 0, sizeof(*res));
    if (!n || !L) return 0;
    double* powl = (double*)malloc(L * sizeof(double));
    for (uint32_t l = 0; l < L; l++) powl[l] = pow((l + 1), beta);
    uint32_t* e2 = (uint32_t*)malloc(L * 4);
    layer_degree* ld = (layer_degree*)malloc(L * sizeof(layer_degree));
    uint32_t* order = (uint32_t*)malloc((uint64_t)n * 4);
    float maxd = 0.0f;
    uint32_t ncell = 0;
    /* per-lambda cell records, then emitted in k-ascending order */
    oracle_cell* col = (oracle_cell*)malloc(((uint64_t)n + 2) * sizeof(oracle_cell));
    int found = 0;
    for (uint32_t lmd = 1; lmd <= L; lmd++) {
        const uint32_t* core = table + (uint64_t)(lmd - 1) * n;
        uint32_t kmax = 0;
        for (uint32_t v = 0; v < n; v++) if (core[v] > kmax) kmax = core[v];
        if (kmax == 0) break; /* C_{1,lambda} empty: the spine ends (PathSerial :217-228) */
        /* counting sort of nodes by core descending */
        uint32_t* cnt = (uint32_t*)calloc(kmax + 2, 4);
        for (uint32_t v = 0; v < n; v++) cnt[kmax - core[v] + 1]++;
        for (uint32_t b = 0; b <= kmax; b++) cnt[b + 1] += cnt[b];
        for (uint32_t v = 0; v < n; v++) order[cnt[kmax - core[v]]++] = v;
        free(cnt);
        memset(e2, 0, L * 4);
        uint32_t length = 0, idx = 0;
        for (uint32_t k = kmax; k >= 1; k--) {
            while (idx < n && core[order[idx]] == k) {
                uint32_t v = order[idx++];
                length++;
                for (uint32_t l = 0; l < L; l++) {
                    const uint64_t* off = g->off + (uint64_t)l * (n + 1);
                    for (uint64_t e = off[v]; e < off[v + 1]; e++) {
                        uint32_t cu = core[g->adj[e]];
                        if (cu > k) e2[l] += 2;      /* both directions enter C now */
                        else if (cu == k) e2[l] += 1; /* the other direction is added with u */
                    }
                }
            }
            oracle_cell* c = &col[k];
            c->k = k;
            c->lmd = lmd;
            c->length = length;
            c->density = cell_density(e2, L, length, powl, ld, &c->lstar);
        }
        for (uint32_t k = 1; k <= kmax; k++) {
            oracle_cell* c = &col[k];
            if (cells && ncell < cells_cap) cells[ncell] = *c;
            ncell++;
            if (c->density >= maxd) {
                maxd = (float)c->density;
                res->density = c->density;
                res->k = c->k;
                res->lmd = c->lmd;
                res->length = c->length;
                res->lstar = c->lstar;
                found = 1;
            }
        }
    }
    res->max_density_f = maxd;
    res->n_cells = ncell;
    if (found && (nodes || layers)) {
        const uint32_t* core = table + (uint64_t)(res->lmd - 1) * n;
        uint32_t j = 0;
        memset(e2, 0, L * 4);
        for (uint32_t v = 0; v < n; v++) {
            if (core[v] < res->k) continue;
            if (nodes) nodes[j] = v;
            j++;
            for (uint32_t l = 0; l < L; l++) {
                const uint64_t* off = g->off + (uint64_t)l * (n + 1);
                for (uint64_t e = off[v]; e < off[v + 1]; e++) e2[l] += core[g->adj[e]] >= res->k;
            }
        }
        if (layers) {
            uint32_t ls;
            cell_density(e2, L, j, powl, ld, &ls);
            /* the first lstar layers of the descending order; for beta >= 0
             * lstar never splits a tie, so this is {l : e_l >= e_(lstar)} */
            uint32_t* pick = (uint32_t*)malloc(L * 4);
            for (uint32_t i = 0; i < res->lstar; i++) pick[i] = ld[i].id;
            /* ascending layer ids */
            for (uint32_t i = 1; i < res->lstar; i++) {
                uint32_t x = pick[i], q = i;
                while (q > 0 && pick[q - 1] > x) { pick[q] = pick[q - 1]; q--; }
                pick[q] = x;
            }
            memcpy(layers, pick, res->lstar * 4);
            free(pick);
        }
    }
    free(powl); free(e2); free(ld); free(order); free(col);
    return 0;
}

/* ---- query-time methods (Util/CoreIndexTime.h, Util/CheckMLCDTime.h) ---- */

/* getResCore, Util/CoreIndexTime.h:8-40: for each listed k of each lambda,
 * every (key, val) of the column with val >= k, in the file's order. */
uint64_t oracle_cells_scan(const uint32_t* table, uint32_t n, uint32_t L, const uint32_t* ks,
                           const uint32_t* lmds, uint32_t nq, uint64_t* offsets, uint32_t* nodes) {
    uint64_t at = 0;
    for (uint32_t q = 0; q < nq; q++) {
        offsets[q] = at;
        if (lmds[q] < 1 || lmds[q] > L) continue;
        const uint32_t* col = table + (uint64_t)(lmds[q] - 1) * n;
        for (uint32_t v = 0; v < n; v++)
            if (col[v] >= ks[q]) {
                if (nodes) nodes[at] = v;
                at++;
            }
    }
    offsets[nq] = at;
    return at;
}

/* main.cpp:567-572 sorts each column's (value, key) pairs by value; then
 * getResCoreOffline, Util/CoreIndexTime.h:43-59, takes lower_bound(k) and
 * everything after it.  A counting sort (stable) stands in for std::sort. */
uint64_t oracle_cells_sorted(const uint32_t* table, uint32_t n, uint32_t L, const uint32_t* ks,
                             const uint32_t* lmds, uint32_t nq, uint64_t* offsets,
                             uint32_t* nodes) {
    uint64_t at = 0;
    uint32_t* sorted = (uint32_t*)malloc(((size_t)n + 1) * 4);
    for (uint32_t q = 0; q < nq; q++) {
        offsets[q] = at;
        if (lmds[q] < 1 || lmds[q] > L || !sorted) continue;
        const uint32_t* col = table + (uint64_t)(lmds[q] - 1) * n;
        uint32_t kmax = 0;
        for (uint32_t v = 0; v < n; v++)
            if (col[v] > kmax) kmax = col[v];
        uint64_t* start = (uint64_t*)calloc((size_t)kmax + 2, 8);
        if (!start) continue;
        for (uint32_t v = 0; v < n; v++) start[col[v] + 1]++;
        for (uint32_t c = 1; c <= kmax + 1; c++) start[c] += start[c - 1];
        for (uint32_t v = 0; v < n; v++) sorted[start[col[v]]++] = v;
        /* start[c] is now the end of value c's run: lower_bound(k) = end of k-1's */
        const uint64_t lb = ks[q] == 0 ? 0 : (ks[q] - 1 <= kmax ? start[ks[q] - 1] : n);
        for (uint64_t i = lb; i < n; i++) {
            if (nodes) nodes[at] = sorted[i];
            at++;
        }
        free(start);
    }
    free(sorted);
    offsets[nq] = at;
    return at;
}

/* checktime, Util/CheckMLCDTime.h:9-42, node-major as there: for node i and
 * query j, t counts the values >= k and f is set once t >= lmd after a
 * match; node i joins query j's list when f. */
uint64_t oracle_mlcd_query(const uint32_t* cores, uint32_t n, uint32_t P, const uint32_t* ks,
                           const uint32_t* lmds, uint32_t nq, uint64_t* offsets,
                           uint32_t* nodes) {
    uint64_t* cnt = (uint64_t*)calloc((size_t)nq + 1, 8);
    uint8_t* hit = (uint8_t*)malloc((size_t)n * (nq ? nq : 1));
    uint64_t total = 0;
    if (!cnt || !hit) {
        free(cnt);
        free(hit);
        return 0;
    }
    for (uint32_t i = 0; i < n; i++) {
        for (uint32_t j = 0; j < nq; j++) {
            const uint32_t k = ks[j], lmd = lmds[j];
            int f = 0;
            uint32_t t = 0;
            for (uint32_t p = 0; p < P; p++) {
                if (cores[(uint64_t)i * P + p] >= k) {
                    t++;
                    if (t >= lmd) {
                        f = 1;
                        break;
                    }
                }
            }
            hit[(uint64_t)i * nq + j] = (uint8_t)f;
            cnt[j] += (uint64_t)f;
        }
    }
    for (uint32_t j = 0; j < nq; j++) {
        offsets[j] = total;
        total += cnt[j];
    }
    offsets[nq] = total;
    if (nodes)
        for (uint32_t j = 0; j < nq; j++) {
            uint64_t at = offsets[j];
            for (uint32_t i = 0; i < n; i++)
                if (hit[(uint64_t)i * nq + j]) nodes[at++] = i;
        }
    free(cnt);
    free(hit);
    return total;
}
