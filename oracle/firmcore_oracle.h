/* Test infrastructure, not product code: the CPU oracle.
 *
 * A plain-C restatement of the reference's hot path (kouteisang/ParGridCPU),
 * used only by the tests and by the benchmark's CPU-baseline leg as the
 * checker.  Nothing in the product links or calls it.
 *
 * Pinned against the reference itself: tests/golden/ holds outputs of the
 * reference's own code (compiled from its sources by oracle/Makefile and run
 * through oracle/ref_harness.cpp) for seeded inputs, and the oracle must
 * reproduce every one of them bit for bit.
 */
#ifndef FIRMCORE_ORACLE_H
#define FIRMCORE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_graph oracle_graph;

typedef struct oracle_cell {
    uint32_t k, lmd, length; /* cell (k, lambda) and |C_{k,lambda}| */
    uint32_t lstar;          /* number of selected layers (num_select_layer) */
    double density;          /* per-cell best density (layer_density) */
} oracle_cell;

typedef struct oracle_densest {
    float max_density_f;  /* the float running maximum main.cpp prints */
    double density;       /* FP64 density of the winning cell */
    uint32_t k, lmd, length, lstar;
    uint32_t n_cells;
} oracle_densest_result;

/* Build a graph from raw (u,v) pairs per layer, in file order, applying the
 * reference loader's semantics.  pairs is the concatenation of every layer's
 * interleaved u,v values; m[l] is the number of pairs of layer l. */
int oracle_graph_from_pairs(uint32_t n_layers, const uint64_t* m, const uint32_t* pairs,
                            oracle_graph** out);
void oracle_graph_free(oracle_graph* g);
uint32_t oracle_n(const oracle_graph* g);
uint32_t oracle_layers(const oracle_graph* g);
/* directed entry count of layer l after dedupe (the reference's Graph::m) */
uint64_t oracle_layer_m(const oracle_graph* g, uint32_t l);
void oracle_id2vtx(const oracle_graph* g, uint64_t* out);
/* per-layer CSR in the reference's row form: off[l*(n+1) + v], adj[...] */
void oracle_csr(const oracle_graph* g, uint64_t* off, uint32_t* adj);

/* core_lambda(v) for lambda = 1..L into table[(lambda-1)*n + v]. */
int oracle_coreindex(const oracle_graph* g, uint32_t* table);

/* Densest search over every non-empty cell.  cells (may be NULL) receives the
 * per-cell records in the reference's preorder (lambda-major, k ascending);
 * cells_cap bounds it.  nodes (may be NULL, n entries) receives the winner's
 * node set ascending, layers (may be NULL, L entries) its layer set. */
int oracle_densest(const oracle_graph* g, const uint32_t* table, double beta,
                   oracle_densest_result* res, oracle_cell* cells, uint32_t cells_cap,
                   uint32_t* nodes, uint32_t* layers);

/* getResCore (Util/CoreIndexTime.h:8-40): query q is the cell (ks[q], lmds[q]);
 * its answer is every node v whose core_lmd(v) >= k, in ascending ids (the
 * order of the core file the reference scans).  offsets (nq+1) receives each
 * answer's start and the total; nodes (may be NULL) the ids.  Returns the total. */
uint64_t oracle_cells_scan(const uint32_t* table, uint32_t n, uint32_t L, const uint32_t* ks,
                           const uint32_t* lmds, uint32_t nq, uint64_t* offsets, uint32_t* nodes);

/* getResCoreOffline with main.cpp:567-572 (Util/CoreIndexTime.h:43-59): the
 * column's (core, v) pairs sorted by core, then every pair from the first
 * with core >= k (lower_bound) to the end.  The sort here is stable, so a
 * query's nodes come by ascending core and ascending ids within a core (the
 * reference's std::sort leaves ties in any order: compare as sets).  Same
 * outputs as oracle_cells_scan. */
uint64_t oracle_cells_sorted(const uint32_t* table, uint32_t n, uint32_t L, const uint32_t* ks,
                             const uint32_t* lmds, uint32_t nq, uint64_t* offsets,
                             uint32_t* nodes);

/* checktime (Util/CheckMLCDTime.h:9-42): node i answers query (ks[q], lmds[q])
 * when, counting its values cores[i*P + p] >= k in p order, the count
 * reaches lmd (tested only after a match).  Answers in ascending ids. */
uint64_t oracle_mlcd_query(const uint32_t* cores, uint32_t n, uint32_t P, const uint32_t* ks,
                           const uint32_t* lmds, uint32_t nq, uint64_t* offsets,
                           uint32_t* nodes);

#ifdef __cplusplus
}
#endif
#endif
