/* firmcore.h -- C ABI of the B200 FirmCore engine (libfirmcore.so).
 *
 * FirmCore decomposition of a multilayer graph: L layers over one node set,
 * each layer an undirected simple graph.  The (k,lambda)-FirmCore C_{k,l} is
 * the largest node set in which every node has at least lambda layers with
 * degree >= k inside the set; core_lambda(v) = max{k : v in C_{k,lambda}}
 * (0 when no such k).  The engine computes the full fcgrid table core_lambda(v)
 * for lambda = 1..L and every node, and the densest-subgraph search over every
 * non-empty cell, on one NVIDIA B200 (sm_100a).
 *
 * Conventions
 *   - Plain C types only.  `stream` arguments are cudaStream_t passed as
 *     void* (NULL = the legacy default stream).
 *   - Node ids are the reference loader's internal ids: 0..n-1 in order of
 *     first appearance (layer by layer in file order, u before v); fc_graph_id2vtx
 *     maps them back to the ids in the input.
 *   - Tables are lambda-major: out[(lambda-1)*n + v] = core_lambda(v).
 *   - Caller allocates every output buffer; the library owns the graph handle
 *     and all device memory behind it; every handle is freed explicitly.
 *   - Every entry point returns fc_status; nothing aborts the process.  There
 *     is no CPU fallback: with no usable CUDA device the compute entry points
 *     return FC_ERR_NO_DEVICE.
 *   - Calls on different handles are independent and may run concurrently
 *     from different host threads; calls on one handle must not overlap.
 */
#ifndef FIRMCORE_H
#define FIRMCORE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FC_ABI_VERSION 1

typedef enum fc_status {
    FC_OK = 0,
    FC_ERR_IO = 1,          /* a file could not be read or written */
    FC_ERR_PARSE = 2,       /* malformed input */
    FC_ERR_OOM = 3,         /* host or device allocation failed */
    FC_ERR_BUDGET = 4,      /* request larger than the device-memory budget */
    FC_ERR_DEVICE = 5,      /* a CUDA call failed */
    FC_ERR_ITER_LIMIT = 6,  /* a device loop or wait hit its bound */
    FC_ERR_INVALID = 7,     /* bad argument or call order */
    FC_ERR_TOO_LARGE = 8,   /* graph exceeds the 32-bit index limits below */
    FC_ERR_NO_DEVICE = 9    /* no CUDA device */
} fc_status;

/* Opaque multilayer graph: host CSR, and device CSR once uploaded. */
typedef struct fc_graph fc_graph;

/* Result of the densest-subgraph search for one beta. */
typedef struct fc_densest_result {
    double beta;
    double density;        /* FP64 density of the winning cell (its layer_density) */
    float max_density_f;   /* the float running maximum the reference prints */
    uint32_t k, lmd;       /* winning cell (0, 0 when the graph has no edges) */
    uint32_t length;       /* |C_{k,lmd}| */
    uint32_t lstar;        /* number of selected layers */
    uint32_t n_cells;      /* non-empty cells searched */
} fc_densest_result;

/* One non-empty fcgrid cell with its best density. */
typedef struct fc_cell {
    uint32_t k, lmd, length, lstar;
    double density;
} fc_cell;

const char* fc_status_string(fc_status s);
int fc_abi_version(void);

/* ---- loading -------------------------------------------------------------
 * Replaces MultilayerGraph::LoadFromFile + SetGraphOrder
 * (Graph/MultilayerGraph.cpp:65-102, 9-45; Graph/MultilayerGraph.h:26-28) and
 * Graph::BuildFromEdgeLst (Graph/Graph.cpp:17-50).  `dir` holds mlg.conf (one
 * layer file name per non-empty line) and the layer files of `u v` lines.
 * Same parse, self-loop and duplicate removal, and first-seen id remap as the
 * reference.  With write_vtx_map != 0 the map is written to dir/__vtx_map.txt
 * as the reference does (`u uid` lines).  `order` is the -o layer order
 * (0 keep, 1/2 density ascending/descending, 3/4 edge count ascending/
 * descending); it permutes the layers, which changes no result. */
fc_status fc_graph_load_dir(const char* dir, int order, int write_vtx_map, fc_graph** out);

/* Same semantics from raw pairs in memory: pairs holds every layer's
 * interleaved (u,v) raw ids, layer after layer; m[l] pairs in layer l. */
fc_status fc_graph_from_pairs(uint32_t n_layers, const uint64_t* m, const uint32_t* pairs,
                              fc_graph** out);

/* From the reference's in-memory form (Graph::adj_lst_buf, Graph/Graph.cpp:
 * 20-47): for each layer l, adj_lst_buf[l] holds n rows [deg, nbr_1..nbr_deg]
 * (internal ids, neighbours ascending, no duplicates), n + m[l] entries where
 * m[l] is the layer's directed entry count (Graph::m). */
fc_status fc_graph_from_adjbuf(uint32_t n, uint32_t n_layers, const uint32_t* const* adj_lst_buf,
                               const uint64_t* m, fc_graph** out);

void fc_graph_free(fc_graph* g);
uint32_t fc_graph_n(const fc_graph* g);
uint32_t fc_graph_layers(const fc_graph* g);
/* directed entry count of layer l (the reference's Graph::getM) */
uint64_t fc_graph_layer_m(const fc_graph* g, uint32_t l);
/* original id of every internal id (MultilayerGraph::LoadId2VtxMap) */
fc_status fc_graph_id2vtx(const fc_graph* g, uint64_t* out);
/* layer order after -o (MultilayerGraph::GetOrder) */
fc_status fc_graph_order(const fc_graph* g, uint32_t* out);
/* per-layer CSR, layer by layer in the current order:
 * off[l*(n+1) + v] .. off[l*(n+1) + v + 1] index adj (internal ids). */
fc_status fc_graph_csr(const fc_graph* g, uint64_t* off, uint32_t* adj);

/* ---- device residency ----------------------------------------------------
 * Copies the graph to the device and builds the node-major CSR the kernels
 * read.  Called implicitly by the compute entry points; explicit calls let a
 * caller time or overlap the upload.  Limits: n*L < 2^32 and total directed
 * entries < 2^32 (FC_ERR_TOO_LARGE otherwise). */
fc_status fc_graph_upload(fc_graph* g, void* stream);
fc_status fc_graph_release_device(fc_graph* g);
/* drop the resident core table and densest state but keep the device CSR:
 * the next compute call recomputes them */
fc_status fc_graph_reset_results(fc_graph* g);
/* bytes of device memory the graph holds now (CSR + resident results) */
uint64_t fc_graph_device_bytes(const fc_graph* g);

/* ---- core index ----------------------------------------------------------
 * The full fcgrid table.  Replaces the table-producing methods behind -m
 * ParGrid / ParGridPlus / CoreIndex / ParCoreIndex: FCSyncLeft::Execute and
 * ExecuteMix (CoreParallel/FCSyncLeft.h:18,34), CoreIndex::Execute and
 * ExecuteParallel (CoreIndexParallel/CoreIndex.h:15-17).  All four compute
 * the same table; the reference keeps it in trees or drops it, this call
 * returns it.  out: L*n uint32, host memory when out_on_device == 0 (the call
 * then returns after the copy), device memory otherwise (the call is then
 * asynchronous on `stream`).  The table stays resident for fc_densest. */
fc_status fc_coreindex(fc_graph* g, uint32_t* out, int out_on_device, void* stream);

/* ---- densest subgraph ----------------------------------------------------
 * Replaces FCPathLevelLeft::Execute(mg, tree, true, beta) + FCTree::
 * WeightDenestSubgraph (Core/FCPathLevelLeft.h:14, Core/FCTree.h:66) as used
 * by -m WdsList (main.cpp:402-424).  Every non-empty cell C_{k,lmd} is scored
 * (e_(l)/|C|) * l^beta over its layers sorted by edge count, the best l per
 * cell is kept, and the cells are compared in the reference's order with its
 * float running maximum.  Runs fc_coreindex first when the table is not
 * resident.  One result per beta. */
fc_status fc_densest(fc_graph* g, const double* betas, uint32_t n_betas, fc_densest_result* res,
                     void* stream);
/* The core table into `table` (host memory, L*n words, as fc_coreindex with
 * out_on_device = 0; may be NULL) and the densest results for `betas` (as
 * fc_densest) in one call -- a -m ParGrid run and a -m WdsList run of the
 * reference (main.cpp:229-239, 402-424) on one graph.  When `table` is pinned
 * host memory its copy runs on the library's copy stream while the densest
 * kernels run on `stream`; otherwise the copy comes first.  Returns when both
 * are complete. */
fc_status fc_coreindex_densest(fc_graph* g, uint32_t* table, const double* betas,
                               uint32_t n_betas, fc_densest_result* res, void* stream);
/* Node set (ascending internal ids, res->length entries) and layer set
 * (ascending layer indices, res->lstar entries) of a result from fc_densest
 * on the same graph.  Either pointer may be NULL. */
fc_status fc_densest_members(fc_graph* g, const fc_densest_result* res, uint32_t* nodes,
                             uint32_t* layers, void* stream);
/* ---- one graph split by lambda range --------------------------------------
 * The lambda columns of a graph are independent given the graph, so a
 * graph's fcgrid can be split over processes or GPUs by lambda range: each
 * computes its columns lmd_lo .. lmd_hi-1 (1 <= lmd_lo < lmd_hi <= L+1) and
 * their cells, and the cells of all ranges, folded in the reference's order
 * with its float running maximum (FCTree::WeightDenestSubgraph,
 * Core/FCTree.cpp:69-82), give the whole graph's densest result
 * (pargridcpu_b200/shard.py, merge_cells).  The reference computes every
 * column in one process; these have no direct counterpart there. */
/* out[(lambda - lmd_lo)*n + v] = core_lambda(v) for the range; only its
 * columns are peeled unless the whole table (or a covering range) is
 * resident.  out may be NULL; out_on_device as for fc_coreindex. */
fc_status fc_coreindex_range(fc_graph* g, uint32_t lmd_lo, uint32_t lmd_hi, uint32_t* out,
                             int out_on_device, void* stream);
/* The range's non-empty cells with their best density for `beta`, lambda-major
 * and k ascending, as fc_cells gives them for the whole graph.  Writes
 * min(cap, count) cells; *count receives the total. */
fc_status fc_cells_range(fc_graph* g, uint32_t lmd_lo, uint32_t lmd_hi, double beta,
                         fc_cell* cells, uint32_t cap, uint32_t* count, void* stream);

/* Node set of any cell, C_{k,lambda} = {v : core_lambda(v) >= k}, in
 * ascending internal ids: the query of `-m kpe -k K -lmd L` (main.cpp:
 * 197-225) that FCTree::saveCoreToLocal writes out (Core/FCTree.cpp:138-153).
 * Writes min(cap, count) ids; *count receives |C|.  k = 0 gives every node;
 * lmd must be in 1..L.  Runs fc_coreindex first when the table is not
 * resident. */
fc_status fc_cell_members(fc_graph* g, uint32_t k, uint32_t lmd, uint32_t* nodes, uint32_t cap,
                          uint32_t* count, void* stream);
/* Every non-empty cell with its best density for `beta`, in the reference's
 * order (lambda-major, k ascending), as its fcgrid trees hold them
 * (coreNode / coreNodeP: k, lmd, length, layer_density, num_select_layer).
 * Writes min(cap, count) cells; *count receives the total. */
fc_status fc_cells(fc_graph* g, double beta, fc_cell* cells, uint32_t cap, uint32_t* count,
                   void* stream);

/* ---- every cell at once --------------------------------------------------
 * The compact form of all cells (the B200 counterpart of -m CoreMem /
 * PathMem, main.cpp:331-362: FCSyncMem::constructCoreSync, CoreParallel/
 * FCSyncMem.cpp:10-54, and FCPathMem::constructCore, Core/FCPathMem.cpp:9-59,
 * which keep per cell the nodes it loses against its parent).  Cells of one
 * column are nested, so one order per column holds every cell as a prefix:
 *   order[(lambda-1)*n + i]  column lambda's nodes by descending core_lambda,
 *                            ascending ids within one core value (L*n words);
 *   col_off[lambda-1]        where column lambda's sizes start (L+1 words);
 *   sizes[col_off[lambda-1] + k] = |C_{k,lambda}|, k = 0 .. kmax_lambda + 1
 *                            (the last is 0).
 * C_{k,lambda} is order[(lambda-1)*n .. (lambda-1)*n + sizes[col_off[lambda-1]
 * + k]), and the nodes with core_lambda = k exactly are the block between the
 * prefixes of k+1 and k.  *sizes_count receives the number of size words
 * (col_off[L]); sizes receives min(sizes_cap, *sizes_count) of them.  Any
 * output pointer may be NULL (call once with order = sizes = NULL to learn
 * the size).  All outputs are host memory.  Runs fc_coreindex first when the
 * table is not resident; the index stays resident with the table. */
fc_status fc_cell_index(fc_graph* g, uint32_t* order, uint64_t* col_off, uint32_t* sizes,
                        uint64_t sizes_cap, uint64_t* sizes_count, void* stream);

/* Many cells at once: query q is the cell (ks[q], lmds[q]), lmds[q] in 1..L.
 * The query lists of -m CoreIndexTimeOnline / CoreIndexTimeOffline
 * (main.cpp:493-582): getResCore scans each query's column for the nodes
 * with core >= k (Util/CoreIndexTime.h:8-40), getResCoreOffline takes them
 * from a core-sorted copy by lower_bound (:43-59).  by_index = 0 answers the
 * first way, each cell in ascending ids; by_index = 1 the second, each cell
 * as its prefix of the fc_cell_index order (building the index first when it
 * is not resident).  offsets (host, nq+1 words) receives the start of every
 * query's nodes and the total; nodes (host) receives min(cap, total) ids.
 * The reference's own loop loads only lambda = 1's core file, so its answers
 * for other lambdas are empty; here every query is answered. */
fc_status fc_cells_members(fc_graph* g, const uint32_t* ks, const uint32_t* lmds, uint32_t nq,
                           int by_index, uint64_t* offsets, uint32_t* nodes, uint64_t cap,
                           void* stream);

/* The membership test of -m MLCDTime (checktime, Util/CheckMLCDTime.h:9-42,
 * main.cpp:453-491) over per-node coreness vectors: cores (host) holds n rows
 * of P values, node v's row at v*P.  Node v answers query (ks[q], lmds[q])
 * when at least max(lmds[q], 1) of its P values are >= ks[q] (unsigned
 * comparisons, as the reference's `uint k` against its values).  offsets and
 * nodes as for fc_cells_members, ascending ids.  Needs no graph. */
fc_status fc_mlcd_query(const uint32_t* cores, uint32_t n, uint32_t P, const uint32_t* ks,
                        const uint32_t* lmds, uint32_t nq, uint64_t* offsets, uint32_t* nodes,
                        uint64_t cap, void* stream);

/* ---- batch ---------------------------------------------------------------
 * Many graphs at once: all (graph, lambda) columns in one persistent kernel
 * launch whose warps pull work items from device queues (captured in a CUDA
 * graph when use_cuda_graph is set), then the densest search for `beta` on
 * every graph.  tables[i] (host, may be NULL) receives graph i's L*n table,
 * res[i] (may be NULL) its densest result.  The equivalent of running the
 * reference once per graph; every result is identical to fc_coreindex +
 * fc_densest on the graph alone.  With `plain` set it runs the baseline
 * instead: one graph and one lambda column per launch, one after another. */
typedef struct fc_batch_options {
    uint32_t block_threads;    /* 512 or 1024 threads per block; 0 = autotuned */
    uint32_t hub_threshold;    /* longest row queued as one work item (longer rows are
                                  split in 256-entry pieces); 0 = autotuned */
    int use_cuda_graph;        /* capture the batched launch in a CUDA graph */
    int plain;                 /* 1 = the one-column-per-launch baseline */
} fc_batch_options;

/* What a batch run did (any pointer field may be ignored). */
typedef struct fc_batch_report {
    double peel_ms;            /* device time of the peel launch(es), CUDA events */
    double densest_ms;         /* time of the densest searches (they overlap on streams) */
    uint32_t peel_launches;
    uint32_t block_threads;    /* the configuration used */
    uint32_t hub_threshold;
    uint32_t levels;
    int used_cuda_graph;
    int autotuned;             /* 1 when this call measured the candidates */
} fc_batch_report;

fc_status fc_batch_run(fc_graph* const* graphs, uint32_t count, double beta,
                       uint32_t* const* tables, fc_densest_result* res,
                       const fc_batch_options* opt, fc_batch_report* report, void* stream);

/* ---- serving -------------------------------------------------------------
 * A continuous-batching request loop.  Requests (a graph + beta) queue in
 * arrival order; each of `lanes` lanes (a host thread and a stream) that is
 * free takes every pending request that fits and runs them as one batch --
 * one persistent peel launch over their graphs, then their densest searches
 * -- so requests that arrive while batches are on the device join the next
 * batch as a lane, SMs and memory free up.  A heavy request (heavy_visits
 * edge visits or more) runs alone on three quarters of the SMs, one at a
 * time, while light batches share the rest, so its work overlaps on the
 * device with the light requests that arrive meanwhile.  A request is
 * admitted while the device bytes of resident graphs plus running batches
 * stay within the budget; graphs stay resident between requests and the
 * least recently used ones that no batch is using are released when memory
 * is short.  Each result is identical to fc_coreindex + fc_densest on the
 * graph alone.  The plain form (one lane, one request at a time, one lambda
 * column per launch) is the baseline it is measured against.
 * A graph handed to a server must not be used by other calls, nor freed,
 * while any request of it is pending; afterwards the server may release its
 * device copy at any time (fc_graph_free is always safe once its requests
 * have completed). */
typedef struct fc_server fc_server;

typedef struct fc_server_options {
    uint64_t hbm_budget_bytes;  /* admission budget (0 = 150 GB) */
    uint32_t max_inflight;      /* requests on the device at once (0 = 256) */
    uint32_t lanes;             /* batches on the device at once (0 = 2) */
    uint32_t max_batch_graphs;  /* distinct graphs in one batch (0 = 64) */
    uint32_t block_threads;     /* peel launch shape (0 = 1024 threads, */
    uint32_t hub_threshold;     /*   rows of more than 64 entries split) */
    int plain;                  /* 1 = the one-at-a-time baseline */
    uint64_t heavy_visits;      /* entries x L at which a request runs alone (0 = 1e9) */
} fc_server_options;

/* Counters since fc_server_create. */
typedef struct fc_server_stats {
    uint64_t requests_done;
    uint64_t batches;
    uint64_t heavy_batches;     /* batches of one heavy request */
    uint64_t graphs_peeled;     /* distinct graphs over all batches */
    uint64_t uploads;           /* device copies made */
    uint64_t evictions;         /* resident copies released for room */
    uint64_t resident_bytes;    /* device copies this server keeps now */
    uint64_t peak_bytes;        /* most bytes admitted at once */
    double busy_ms;             /* time with a batch running */
    double overlap_ms;          /* time with two or more batches running */
    uint32_t max_batch;         /* most requests in one batch */
    uint32_t lanes;
} fc_server_stats;

fc_status fc_server_create(const fc_server_options* opt, fc_server** out);
/* Enqueue a request.  table (host, L*n, may be NULL) and res (may be NULL)
 * are filled on completion.  *ticket identifies it. */
fc_status fc_server_submit(fc_server* s, fc_graph* g, double beta, uint32_t* table,
                           fc_densest_result* res, uint64_t* ticket);
/* Wait up to timeout_ms (negative = forever) for a ticket; FC_ERR_ITER_LIMIT
 * on timeout.  *status receives the request's own status (FC_ERR_BUDGET for a
 * request that alone exceeds the budget); *latency_ms its time from submit to
 * completion. */
fc_status fc_server_wait(fc_server* s, uint64_t ticket, int64_t timeout_ms, fc_status* status,
                         double* latency_ms);
fc_status fc_server_query(fc_server* s, fc_server_stats* out);
/* Completes every pending request, then stops the lanes. */
fc_status fc_server_destroy(fc_server* s);

/* ---- core index without device allocation --------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory -- an application whose memory manager has reserved the whole
 * device, or a latency-bound loop that cannot take the stall a device
 * allocation may cause -- this computes the same table as fc_coreindex from a
 * graph already in device memory the caller owns, with its scratch carved
 * from one fixed 64 MiB device array that every GPU loading the library keeps
 * until the process exits.  It allocates nothing.
 *   Inputs (device): node_ptr[n+1] and adj[entries] -- node-major rows, each
 *   entry the slot u*L + l (neighbour u in layer l), v's layers in order --
 *   and deg0[n*L] = |N_l(v)| at v*L + l.  Output (device): table[L*n],
 *   lambda-major.  The call returns when the table is complete.
 * Preconditions, as the graph's own CSR satisfies them: node_ptr[0] = 0,
 * node_ptr non-decreasing, node_ptr[n] = entries, every slot < n*L, and the
 * graph undirected (each entry u*L + l in v's row matched by v*L + l in u's
 * row) with deg0[u*L + l] the number of entries u*L + l.  The first three
 * and the slot bound are checked on the device before the peel runs (a
 * violation returns FC_ERR_INVALID with nothing else done); the others
 * decide only the values of the table.
 * A graph whose one column needs more than the array's scratch (about
 * 4*n*L + 36*n + entries/16 bytes) is rejected with FC_ERR_TOO_LARGE before
 * any device work.  A call cannot be captured in a CUDA graph: it reads the
 * run's status back on the host (a copy and a stream synchronization) before
 * it returns.  All calls share the one array per device, so
 * calls that overlap on the GPU -- on two streams, or from two host threads
 * -- race, and the caller must serialize them; each call clears the parts
 * that must start empty. */
fc_status fc_coreindex_fixed_scratch(uint32_t n, uint32_t n_layers, uint64_t entries,
                                     const uint32_t* node_ptr, const uint32_t* adj,
                                     const uint32_t* deg0, uint32_t* table, void* stream);

/* ---- diagnostics ---------------------------------------------------------
 * Timings of the last fc_coreindex / fc_densest on a graph, taken with CUDA
 * events recorded around the kernels on the stream they ran on, and the
 * number of kernels this library has launched in the process. */
typedef struct fc_stats {
    double peel_ms;          /* peel kernels of the last table computation */
    double densest_ms;       /* histogram + scoring kernels of the last fc_densest */
    uint32_t peel_launches;  /* peel launches (one per column group) */
    uint32_t levels;         /* peel levels, summed over column groups */
    uint32_t subrounds;      /* peel sub-rounds, summed over column groups */
    uint32_t columns_per_launch;
    double phase_ms[3];      /* peel time in level scans, expansions, recomputes */
} fc_stats;

fc_status fc_graph_stats(const fc_graph* g, fc_stats* out);
uint64_t fc_launch_count(void);
/* Device and pinned-host allocations, streams and events this library has
 * created in the process (a call that allocates nothing leaves it unchanged). */
uint64_t fc_alloc_count(void);

/* The atomic-throughput denominator of the peel's roofline (no counterpart
 * in the reference): `ops` 4-byte atomic subtractions whose old value is
 * returned, as the peel's degree decrements are, at pseudo-random word
 * addresses of a device buffer of at most `bytes` bytes (a power-of-two word
 * count; at least 4 KiB), timed with CUDA events on `stream` after one
 * warm-up launch.  *gatomics_per_s receives the rate in 1e9 atomics/s.  The
 * buffer is allocated and freed by the call. */
fc_status fc_probe_atomics(uint64_t bytes, uint64_t ops, double* gatomics_per_s, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FIRMCORE_H */
