// The fcgrid peel: core_lambda(v) for groups of lambda columns of one or many
// graphs, in one persistent cooperative kernel with the level loop inside.
//
// A launch covers segments; a segment is one graph's group of columns (lambda
// = col0+c+1 for c < ncols).  Segments are laid end to end in one index space
// x, so one launch peels many graphs at once and they share the level loop.
// Edges never cross graphs: a queued node resolves its segment once and all
// its visits stay inside it.  All columns advance together, level by level,
// K = 0, 1, 2, ...:
//
//   SCAN(K)   every alive x counts its layers with degree >= K+1 inside the
//             alive set, cnt[x].  cnt < lambda means Top-lambda(x) <= K: x is
//             removed at level K (core = K).  The others keep cnt.
//   DRAIN(K)  removed nodes are expanded from device work queues: each
//             adjacency slot (u,l) of a removed x decrements deg[u][l] of an
//             alive u; a decrement from exactly K+1 to K lowers cnt[u], and the
//             decrement that takes cnt[u] from lambda to lambda-1 removes u at
//             level K too -- ParGrid's own trigger (CoreParallel/
//             FCSyncLeft.cpp:99-103).  Each of those crossings happens exactly
//             once, so every node is queued once.  Removals cascade through
//             the queues without any barrier; the level ends when no queued
//             item is left unprocessed (the processed-items count reaches the
//             reserved-items count).
//
// This computes the same table as the reference's get_index2 bucket peel
// (CoreIndexParallel/CoreIndex.cpp:62-109) and ParGrid's per-cell PeelSync:
// core_lambda is the unique fixpoint, whatever the removal order.
//
// Long rows (more than `small_row` entries, 64 by default; the batch
// autotuner picks it) are queued as CHUNK-entry items so that hubs spread over
// many warps.  SCAN and DRAIN are separated by a grid
// barrier whose last arriving block runs the serial "leader" step (level
// change, counter resets).  Every wait -- barrier or queue -- is bounded by a
// timeout after which the kernel records an error and winds down; the level
// count is bounded by the largest degree.
#include <cooperative_groups.h>

#include <cstdio>
#include <cstdlib>

#include "device.h"

namespace cg = cooperative_groups;

namespace fc {

// PH_INIT is 0 so that a zeroed control block starts a run
enum : uint32_t { PH_INIT = 0, PH_SCAN = 1, PH_DRAIN = 2, PH_DONE = 3 };
// ERR_DEADLINE: the whole run took longer than its deadline (a bound on
// every loop, including ones that keep making progress); ERR_ITEM: a dequeued
// item named no node of the launch (recorded and skipped, never expanded).
enum : uint32_t {
    ERR_NONE = 0, ERR_BARRIER = 1, ERR_LIMIT = 2, ERR_QUEUE = 3, ERR_DEADLINE = 4, ERR_ITEM = 5
};
constexpr uint32_t UNSET = 0xFFFFFFFFu;
constexpr unsigned long long EMPTY = ~0ull;
constexpr uint32_t EMPTY32 = 0xFFFFFFFFu;

// Work queues, per level parity q and kind s (0: nodes with short rows, one
// u32 item each; 1: CHUNK-entry pieces of long rows, u64 items x | chunk<<32).
enum : uint32_t { QS = 0, QC = 1 };

// rows longer than the job's small_row entries are expanded as CHUNK-entry
// work items
constexpr uint32_t SMALL_ROW_DEFAULT = 64;
constexpr uint32_t CHUNK = 256;

// A counter alone on its 128-byte line: the queue counters are hit by atomics
// and polls from every SM, and must not share a line with each other.
struct alignas(128) Hot {
    uint32_t v;
};

struct PeelCtl {
    uint32_t bar_count, bar_gen, err, phase;
    uint32_t level, alive_cur, q_cur, stopped;  // stopped: left the rest to the endgame
    uint32_t prev_tail[2];       // per kind: items the previous level's queues held
    uint32_t alive_cnt[2];
    uint32_t levels, items;
    uint32_t alive0[2];  // of alive_cnt, the pairs of the launch's first column
    uint64_t t_last;      // globaltimer at the last barrier
    uint64_t t_start;     // globaltimer at the first barrier
    uint64_t ph_ns[4];    // time per phase kind: scan, drain
    uint32_t bad_item, bad_where, err_level, pad3;  // what ERR_ITEM saw; level of the error
    Hot tail[2][2];       // [q][s] items reserved
    Hot head[2][2];       // [q][s] items claimed
    Hot processed[2][2];  // [q][s] items fully processed
    // endgame (one block per column): survivors, subgraph entries, levels run
    uint32_t eg_cnt[64], eg_tot[64], eg_levels[64];
    uint32_t eg_err, eg_nbig, eg_pad[2];  // eg_nbig: long rows listed for k_eg_fill_big
    uint64_t eg_base[64];  // first entry of each column's subgraph
};

// One segment: a graph's group of columns, as the kernel reads it.
struct SegP {
    uint32_t xbase;            // first x of the segment
    uint32_t n, L, col0;
    FastDiv divL, divN;
    uint64_t nL;               // n * L
    const uint32_t* node_ptr;
    const uint32_t* adj;
    const uint32_t* deg0;
    uint32_t* deg;             // ncols * n * L, degrees inside the alive set
    uint32_t* t;               // table + col0 * n: UNSET while alive, then the core
    const uint32_t* big_id;    // ordered long rows (device.h), or null
    const uint32_t* ptab;
    uint32_t ncols, pad;
};

struct PeelJob {
    SegP seg0;                     // the only segment when the launch has one
    const SegP* segs;              // nseg segments (device), when more than one
    const uint32_t* seg_xbase;     // nseg + 1 (device): segment starts, then nx
    uint32_t nseg, nx;
    uint32_t* cnt;                 // nx: layers with degree >= level+1, kept for alive x
    uint32_t* alive[2];            // each nx
    uint32_t* bits;                // (nx + 31) / 32: bit x set while x is not removed
    uint32_t* qs[2];               // short-row node items, EMPTY32 when unwritten
    unsigned long long* qc[2];     // chunk items, EMPTY when unwritten
    uint32_t qs_cap, qc_cap;
    PeelCtl* ctl;
    uint32_t max_level;
    uint32_t idle_polls;  // empty polls after which a warp other than warp 0 parks
    uint32_t small_row;   // longest row queued as one item; longer rows go in chunks
    uint64_t timeout_ns;  // longest wait without progress
    uint64_t deadline_ns; // longest whole run
    // optional per-level trace: [level][scan|drain] = {ns, items, alive}
    unsigned long long* trace;
    uint32_t trace_levels;
    uint32_t max_sms;     // host side: SMs the grid may cover (0 = every SM)
    // stop after a level's DRAIN once at most this many (column, node) pairs
    // are alive, for the endgame to finish (0: run to the end)
    uint32_t stop_alive;
};

// ---- memory-model helpers -------------------------------------------------

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t atom_add_acq_rel(uint32_t* p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// data written by other SMs during the kernel is read through L2 only
__device__ __forceinline__ uint32_t ld_l2(const uint32_t* p) { return __ldcg(p); }
__device__ __forceinline__ uint64_t ld_l2_64(const uint64_t* p) {
    return __ldcg((const unsigned long long*)p);
}

// The alive bitmap: one bit per x, cleared once when x is removed.  It is
// small enough to stay in L2, so the "is the neighbour still alive" test of
// every visit is an L2 hit rather than a DRAM read of cnt.
__device__ __forceinline__ uint32_t is_alive(const PeelJob& j, uint32_t x) {
    return (ld_l2(j.bits + (x >> 5)) >> (x & 31)) & 1u;
}
__device__ __forceinline__ void clear_alive(const PeelJob& j, uint32_t x) {
    atomicAnd(j.bits + (x >> 5), ~(1u << (x & 31)));
}

// ---- segments ---------------------------------------------------------------

template <bool MULTI>
__device__ __forceinline__ uint32_t seg_of(const PeelJob& j, uint32_t x) {
    if (!MULTI) return 0;
    uint32_t lo = 0, hi = j.nseg;  // seg_xbase[lo] <= x < seg_xbase[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(j.seg_xbase + mid) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <bool MULTI>
__device__ __forceinline__ SegP seg_load(const PeelJob& j, uint32_t s) {
    if (!MULTI) return j.seg0;
    SegP g;
    const SegP* p = j.segs + s;
    g.xbase = __ldg(&p->xbase);
    g.n = __ldg(&p->n);
    g.L = __ldg(&p->L);
    g.col0 = __ldg(&p->col0);
    g.divL.d = __ldg(&p->divL.d);
    g.divL.m = __ldg(&p->divL.m);
    g.divL.s1 = __ldg(&p->divL.s1);
    g.divL.s2 = __ldg(&p->divL.s2);
    g.divN.d = __ldg(&p->divN.d);
    g.divN.m = __ldg(&p->divN.m);
    g.divN.s1 = __ldg(&p->divN.s1);
    g.divN.s2 = __ldg(&p->divN.s2);
    g.nL = __ldg((const unsigned long long*)&p->nL);
    g.node_ptr = (const uint32_t*)__ldg((const unsigned long long*)&p->node_ptr);
    g.adj = (const uint32_t*)__ldg((const unsigned long long*)&p->adj);
    g.deg0 = (const uint32_t*)__ldg((const unsigned long long*)&p->deg0);
    g.deg = (uint32_t*)__ldg((const unsigned long long*)&p->deg);
    g.t = (uint32_t*)__ldg((const unsigned long long*)&p->t);
    g.big_id = (const uint32_t*)__ldg((const unsigned long long*)&p->big_id);
    g.ptab = (const uint32_t*)__ldg((const unsigned long long*)&p->ptab);
    g.ncols = __ldg(&p->ncols);
    return g;
}

// ---- leader step: phase transitions (one thread, all blocks parked) -------

// The serial step between phases, run by the last block to arrive at a
// grid barrier while all others wait.  Every field it reads is loaded in one
// round of independent L2 loads and every result stored once: the step is on
// the critical path of every level, twice.
__device__ void leader_step(PeelCtl* c, const PeelJob& j) {
    const uint64_t now = global_ns();
    const uint32_t phase = ld_l2(&c->phase), q = ld_l2(&c->q_cur), level = ld_l2(&c->level);
    uint32_t ac = ld_l2(&c->alive_cur);
    uint32_t err = ld_l2(&c->err);
    const uint32_t levels = ld_l2(&c->levels), items = ld_l2(&c->items);
    const uint64_t t_last = ld_l2_64(&c->t_last), t_start0 = ld_l2_64(&c->t_start);
    const uint32_t kind = phase == PH_DRAIN ? 1 : 0;
    const uint64_t ph = ld_l2_64(&c->ph_ns[kind]);
    const uint32_t t00 = ld_l2(&c->tail[0][QS].v), t01 = ld_l2(&c->tail[0][QC].v);
    const uint32_t t10 = ld_l2(&c->tail[1][QS].v), t11 = ld_l2(&c->tail[1][QC].v);
    const uint32_t ac0 = ld_l2(&c->alive_cnt[0]), ac1 = ld_l2(&c->alive_cnt[1]);
    const uint32_t first_col = ld_l2(&c->alive0[ac & 1u]);
    const uint32_t ts = q ? t10 : t00, tc = q ? t11 : t01;  // this level's reservations
    if (t_last) __stcg((unsigned long long*)&c->ph_ns[kind], ph + (now - t_last));
    if (j.trace && t_last && level < j.trace_levels && phase != PH_INIT) {
        unsigned long long* r = j.trace + 3ull * (2ull * level + kind);
        r[0] = now - t_last;
        r[1] = ts + tc;
        r[2] = (ac ^ (kind == 0 ? 1u : 0u)) ? ac1 : ac0;
    }
    __stcg((unsigned long long*)&c->t_last, now);
    // the run's deadline, checked at every phase change after the first
    uint32_t next = PH_DONE;
    if (phase == PH_INIT) __stcg((unsigned long long*)&c->t_start, now);
    else if (now - t_start0 > j.deadline_ns) err = ERR_DEADLINE;
    bool advance = false;
    if (!err) {
        switch (phase) {
            case PH_INIT:  // degree tables copied: the first scan follows
                next = PH_SCAN;
                break;
            case PH_SCAN:  // the scan wrote the other alive list
                ac ^= 1;
                __stcg(&c->alive_cur, ac);
                if (ts + tc > 0) next = PH_DRAIN;
                else if ((ac ? ac1 : ac0) == 0) next = PH_DONE;
                else advance = true;
                break;
            case PH_DRAIN:
                __stcg(&c->items, items + ts + tc);
                if ((ac ? ac1 : ac0) == 0) {
                    next = PH_DONE;
                } else if (j.stop_alive && first_col <= j.stop_alive) {
                    // every removal up to this level is done: the survivors
                    // are the nodes whose core exceeds it.  The launch's
                    // first column holds the most (core_(lmd+1) <= core_lmd),
                    // so no column has more than stop_alive
                    __stcg(&c->stopped, 1u);
                    next = PH_DONE;
                } else {
                    advance = true;
                }
                break;
            default:
                next = PH_DONE;
        }
    }
    if (advance) {
        // the queues of this level are done: the other parity becomes current
        __stcg(&c->prev_tail[QS], ts);
        __stcg(&c->prev_tail[QC], tc);
        __stcg(&c->q_cur, q ^ 1);
        for (uint32_t s = 0; s < 2; s++) {
            __stcg(&c->tail[q ^ 1][s].v, 0u);
            __stcg(&c->head[q ^ 1][s].v, 0u);
            __stcg(&c->processed[q ^ 1][s].v, 0u);
        }
        __stcg(&c->level, level + 1);
        __stcg(&c->levels, levels + 1);
        __stcg(&c->alive_cnt[ac ^ 1], 0u);
        __stcg(&c->alive0[ac ^ 1], 0u);
        next = PH_SCAN;
        if (level + 1 > j.max_level) err = ERR_LIMIT;
    }
    if (err) {
        __stcg(&c->err, err);
        __stcg(&c->err_level, advance ? level + 1 : level);
        next = PH_DONE;
    }
    __stcg(&c->phase, next);
}

// Grid barrier with a bounded wait.  Returns false once any block has
// recorded an error.
__device__ bool grid_barrier(const PeelJob& j) {
    PeelCtl* c = j.ctl;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t gen = ld_acquire(&c->bar_gen);
        __threadfence();
        uint32_t arrived = atom_add_acq_rel(&c->bar_count, 1);
        if (arrived == gridDim.x - 1) {
            // the release store of the new generation orders every store of
            // the step before it
            c->bar_count = 0;
            leader_step(c, j);
            st_release(&c->bar_gen, gen + 1);
        } else {
            uint64_t t0 = global_ns();
            uint32_t ns = 32;
            while (ld_acquire(&c->bar_gen) == gen) {
                __nanosleep(ns);
                if (ns < 256) ns <<= 1;
                if (global_ns() - t0 > j.timeout_ns) {
                    atomicExch(&c->err, ERR_BARRIER);
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ld_acquire(&c->err) == ERR_NONE;
}

// ---- queues -----------------------------------------------------------------

// A node removed at level k is queued as one short item when its row has at
// most small_row entries, else as chunk items; returns the chunk count (0 for
// a short row).  An ordered row (device.h) needs only the chunks covering its
// entries of bucket >= bucket_of(k): every later entry names a neighbour whose
// bound is below k, removed at an earlier level.  At least one chunk is
// queued, so that every removal of a long row is one or more chunk items.
__device__ __forceinline__ uint32_t chunks_of(const SegP& g, uint32_t v, uint32_t small_row,
                                              uint32_t k) {
    // the three loads are independent: one round trip
    const uint32_t id = g.big_id ? __ldg(g.big_id + v) : NO_BIG_ROW;
    const uint32_t len = __ldg(g.node_ptr + v + 1) - __ldg(g.node_ptr + v);
    if (len <= small_row) return 0u;
    uint32_t need = len;
    if (id != NO_BIG_ROW) need = min(len, __ldg(g.ptab + (uint64_t)id * BUCKETS + bucket_of(k)));
    return need ? (need + CHUNK - 1) / CHUNK : 1u;
}

__device__ __forceinline__ void write_short(const PeelJob& j, uint32_t q, uint32_t idx, uint32_t x) {
    if (idx < j.qs_cap)
        asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(j.qs[q] + idx), "r"(x) : "memory");
    else
        atomicExch(&j.ctl->err, ERR_QUEUE);
}

// Chunk items c_begin .. c_end-1 of x at queue slots first, first+1, ...
// The high word of chunk item c of a row queued as nch chunks at level k.
// From level 16 on (where the ordered rows' pruning acts) a row of 2 .. 32767
// chunks is visited strided: chunk c takes the 8-entry groups c, c + nch,
// c + 2 nch, ... (one group per lane), so that the front of an ordered row --
// the neighbours that may still be alive -- is spread over all of its chunks
// rather than loading its first one.  Otherwise chunk c is the CHUNK entries
// from c * CHUNK.  Either way the row's first 256 * nch entries (clipped to
// the row) are visited once each.
constexpr uint32_t STRIDED = 0x80000000u;
__device__ __forceinline__ uint32_t chunk_word(uint32_t c, uint32_t nch, uint32_t k) {
    return (k >= 16 && nch > 1 && nch < 32768) ? (STRIDED | (nch << 16) | c) : c;
}

__device__ __forceinline__ void write_chunks(const PeelJob& j, uint32_t q, uint32_t first,
                                             uint32_t x, uint32_t c_begin, uint32_t c_end,
                                             uint32_t k) {
    for (uint32_t c = c_begin; c < c_end; c++) {
        const uint32_t idx = first + (c - c_begin);
        if (idx < j.qc_cap) {
            const unsigned long long it =
                (unsigned long long)x | ((unsigned long long)chunk_word(c, c_end, k) << 32);
            asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(j.qc[q] + idx), "l"(it)
                         : "memory");
        } else {
            atomicExch(&j.ctl->err, ERR_QUEUE);
        }
    }
}

// Warp-wide inclusive scan.
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const uint32_t lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= (uint32_t)o) v += y;
    }
    return v;
}

// Count of the L values row[0..L) that are >= thr, by a group of G lanes (G 1
// or 32; all 32 lanes of the warp call this together, each group with its own
// row and L).  Every lane of a group returns the group's count.
template <int G>
__device__ __forceinline__ uint32_t group_count_ge(const uint32_t* row, uint32_t L, uint32_t thr,
                                                   bool live) {
    uint32_t cnt = 0;
    if (G == 1) {  // one lane per node: its L loads are independent
        if (live) {
#pragma unroll 8
            for (uint32_t li = 0; li < L; li++) cnt += ld_l2(row + li) >= thr;
        }
        return cnt;
    }
    const uint32_t gl = (threadIdx.x & 31) & (G - 1);
    if (live)
        for (uint32_t li = gl; li < L; li += G) cnt += ld_l2(row + li) >= thr;
#pragma unroll
    for (int off = G / 2; off >= 1; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
    return cnt;
}

// A removed node that the warp which removed it expands next itself instead
// of queueing it -- its whole row when short, its first chunk when long (the
// other chunks are queued): a removal cascade then takes no queue round trip
// per step along the warp's own chain, while the warp's other removals go to
// the queues for the other warps.  Warp-uniform.  Such an item is never
// reserved, so it never counts as processed; the warp must not flush its
// processed counts while it holds one (the level could otherwise end first).
struct Local {
    uint32_t x;      // launch index, EMPTY32 when none
    uint32_t chunk;  // n > 0: x's first chunk of n; 0: x's whole short row
};

// Queues the nodes this warp's lanes removed (rem[i]: launch index yg[i],
// nch[i] chunk items or one short item when 0), with one reservation per
// queue for the whole warp -- except one, kept in `loc` when it is empty.
// my_s / my_c are the lane's short / chunk item counts.  All 32 lanes call it
// together.
template <int N>
__device__ __forceinline__ void enqueue_removed(const PeelJob& j, uint32_t q, uint32_t k,
                                                const bool (&rem)[N], const uint32_t (&yg)[N],
                                                const uint32_t (&nch)[N], uint32_t my_s,
                                                uint32_t my_c, Local& loc) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t any = __ballot_sync(0xffffffffu, (my_s | my_c) != 0);
    if (!any) return;
    int keep = -1;  // on the lane that gives up an entry: that entry
    if (loc.x == EMPTY32) {
        const uint32_t src = __ffs(any) - 1;
        uint32_t px = 0, pn = 0;
        if (lane == src) {
#pragma unroll
            for (int i = 0; i < N; i++)
                if (keep < 0 && rem[i]) {
                    keep = i;
                    px = yg[i];
                    pn = nch[i];
                }
            if (pn == 0) my_s -= 1;
            else my_c -= 1;  // its first chunk stays with the warp
        }
        loc.x = __shfl_sync(0xffffffffu, px, src);
        loc.chunk = __shfl_sync(0xffffffffu, pn, src);
    }
    if (!__any_sync(0xffffffffu, (my_s | my_c) != 0)) return;
    const uint32_t is = warp_incl_scan(my_s);
    const uint32_t ic = warp_incl_scan(my_c);
    uint32_t bs = 0, bc = 0;
    if (lane == 31) {
        if (is) bs = atomicAdd(&j.ctl->tail[q][QS].v, is);
        if (ic) bc = atomicAdd(&j.ctl->tail[q][QC].v, ic);
    }
    bs = __shfl_sync(0xffffffffu, bs, 31) + is - my_s;
    bc = __shfl_sync(0xffffffffu, bc, 31) + ic - my_c;
#pragma unroll
    for (int i = 0; i < N; i++) {
        if (rem[i]) {
            const bool kept = i == keep;
            if (nch[i] == 0) {
                if (!kept) write_short(j, q, bs++, yg[i]);
            } else {
                const uint32_t c0 = kept ? 1u : 0u;
                write_chunks(j, q, bc, yg[i], c0, nch[i], k);
                bc += nch[i] - c0;
            }
        }
    }
}

// Up to four removed-neighbour slots per lane at once (loads first, then the
// atomics) so each lane keeps several memory operations in flight.  Entry i is
// slot slot[i] of column col[i] of segment seg[i] (entries of different nodes:
// the short-row path).  All 32 lanes call it together.
//
// An entry is skipped when its neighbour is already removed (alive bit
// clear).  A neighbour removed concurrently may still take a decrement; that
// is harmless: its degrees are never read again, and its count is already
// below lambda, so the count crossing that queues a node cannot recur.
template <bool MULTI>
__device__ __forceinline__ void visit4(const PeelJob& j, const uint32_t (&seg)[4],
                                       const uint32_t (&col)[4], const uint32_t (&slot)[4],
                                       const bool (&ok)[4], uint32_t k, uint32_t q, Local& loc) {
    uint32_t yl[4], yg[4], cy[4], old[4], lmd[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const SegP g = seg_load<MULTI>(j, seg[i]);
        yl[i] = col[i] * g.n + g.divL.div(slot[i]);  // within the segment
        yg[i] = g.xbase + yl[i];                      // in the launch
        lmd[i] = g.col0 + col[i] + 1;
        cy[i] = ok[i] ? is_alive(j, yg[i]) : 0u;
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        old[i] = 0u;
        if (cy[i]) {
            const SegP g = seg_load<MULTI>(j, seg[i]);
            old[i] = atomicSub(g.deg + (uint64_t)col[i] * g.nL + slot[i], 1u);
        }
    }
    bool rem[4];
    uint32_t nch[4], my_s = 0, my_c = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        rem[i] = false;
        if (cy[i] && old[i] == k + 1) rem[i] = atomicSub(j.cnt + yg[i], 1u) == lmd[i];
        nch[i] = 0;
        if (rem[i]) {
            const SegP g = seg_load<MULTI>(j, seg[i]);
            clear_alive(j, yg[i]);
            g.t[yl[i]] = k;
            nch[i] = chunks_of(g, yl[i] - col[i] * g.n, j.small_row, k);
            my_s += nch[i] == 0;
            my_c += nch[i];
        }
    }
    enqueue_removed<4>(j, q, k, rem, yg, nch, my_s, my_c, loc);
}

// The same for N entries per lane that all belong to one node (a chunk of a
// long row): the segment and column are shared, so they are loaded once and
// each lane can keep more entries in flight.
template <int N>
__device__ __forceinline__ void visit_node(const PeelJob& j, const SegP& g, uint32_t col,
                                           const uint32_t (&slot)[N], const bool (&ok)[N],
                                           uint32_t k, uint32_t q, Local& loc) {
    const uint32_t lmd = g.col0 + col + 1;
    const uint32_t cb = col * g.n;
    uint32_t* const deg = g.deg + (uint64_t)col * g.nL;
    uint32_t yg[N], cy[N], old[N];
#pragma unroll
    for (int i = 0; i < N; i++) {
        yg[i] = g.xbase + cb + g.divL.div(slot[i]);
        cy[i] = ok[i] ? is_alive(j, yg[i]) : 0u;
    }
#pragma unroll
    for (int i = 0; i < N; i++) old[i] = cy[i] ? atomicSub(deg + slot[i], 1u) : 0u;
    bool rem[N];
    uint32_t nch[N], my_s = 0, my_c = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        rem[i] = false;
        if (cy[i] && old[i] == k + 1) rem[i] = atomicSub(j.cnt + yg[i], 1u) == lmd;
        nch[i] = 0;
        if (rem[i]) {
            const uint32_t yl = yg[i] - g.xbase;
            clear_alive(j, yg[i]);
            g.t[yl] = k;
            nch[i] = chunks_of(g, yl - cb, j.small_row, k);
            my_s += nch[i] == 0;
            my_c += nch[i];
        }
    }
    enqueue_removed<N>(j, q, k, rem, yg, nch, my_s, my_c, loc);
}

// ---- phases ---------------------------------------------------------------

// SCAN(K) over `cnt_nodes` alive entries taken from `src` (or 0..nx-1 when
// src is null, the first level): removed nodes get t = K and are queued,
// the rest keep their count and move to `out`.  Survivors and queue items of
// a block are reserved with one atomic each per block iteration (the
// counters are shared by the whole grid).
// NPT nodes per group of G lanes and block iteration: with one-lane nodes and
// enough of them for every block, four (their loads all in flight together,
// and a quarter of the block barriers and reservations per node).  The kept
// pairs of the launch's first column are counted beside the total.
template <int G, bool MULTI, int NPT>
__device__ __forceinline__ void scan_nodes_n(const PeelJob& j, const uint32_t* src,
                                             uint32_t cnt_nodes, uint32_t k, uint32_t q,
                                             uint32_t* out, uint32_t* out_cnt, uint32_t* out_cnt0) {
    __shared__ uint32_t s_keep[32], s_short[32], s_chunk[32], s_kbase, s_sbase, s_cbase;
    __shared__ uint32_t s_keep0[32];  // kept pairs of the first column, per warp
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t nwarps = blockDim.x >> 5;
    const uint32_t per_pass = blockDim.x / G;
    const uint32_t per_block = per_pass * NPT;
    for (uint32_t base = blockIdx.x * per_block; base < cnt_nodes; base += gridDim.x * per_block) {
        uint32_t xs[NPT], nchs[NPT], tk = 0, tsh = 0, tch = 0, tk0 = 0;
        bool keeps[NPT], shorts[NPT];
#pragma unroll
        for (int i = 0; i < NPT; i++) {
            const uint32_t idx = base + i * per_pass + threadIdx.x / G;
            bool live = idx < cnt_nodes;
            const uint32_t x = live ? (src ? ld_l2(src + idx) : idx) : 0;
            if (live && src && !is_alive(j, x)) live = false;  // removed in the last drain
            const SegP g = seg_load<MULTI>(j, seg_of<MULTI>(j, x));
            const uint32_t xl = x - g.xbase;
            const uint32_t c = g.divN.div(xl);
            const uint32_t v = xl - c * g.n;
            const uint32_t cnt = group_count_ge<G>(g.deg + (uint64_t)c * g.nL + (uint64_t)v * g.L,
                                                   g.L, k + 1, live);
            const bool lead = live && (lane & (G - 1)) == 0;
            const bool remove = lead && cnt < g.col0 + c + 1;
            const bool keep = lead && !remove;
            const uint32_t nch = remove ? chunks_of(g, v, j.small_row, k) : 0u;
            const bool ns = remove && nch == 0;
            if (remove) {
                clear_alive(j, x);
                g.t[xl] = k;
            } else if (keep) {
                j.cnt[x] = cnt;
                if (!src) g.t[xl] = UNSET;
            }
            xs[i] = x;
            nchs[i] = nch;
            keeps[i] = keep;
            shorts[i] = ns;
            tk += keep;
            tk0 += keep && c == 0 && (!MULTI || g.xbase == 0);
            tsh += ns;
            tch += nch;
        }
        const uint32_t kin = warp_incl_scan(tk);
        const uint32_t sin = warp_incl_scan(tsh);
        const uint32_t cin = warp_incl_scan(tch);
        const uint32_t k0w = __reduce_add_sync(0xffffffffu, tk0);
        if (lane == 31) {
            s_keep[warp] = kin;
            s_short[warp] = sin;
            s_chunk[warp] = cin;
            s_keep0[warp] = k0w;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t kt = 0, st = 0, ct = 0, k0t = 0;
            for (uint32_t w = 0; w < nwarps; w++) {
                uint32_t a = s_keep[w], b = s_short[w], d = s_chunk[w];
                s_keep[w] = kt;
                s_short[w] = st;
                s_chunk[w] = ct;
                kt += a;
                st += b;
                ct += d;
                k0t += s_keep0[w];
            }
            if (k0t) atomicAdd(out_cnt0, k0t);
            s_kbase = kt ? atomicAdd(out_cnt, kt) : 0u;
            s_sbase = st ? atomicAdd(&j.ctl->tail[q][QS].v, st) : 0u;
            s_cbase = ct ? atomicAdd(&j.ctl->tail[q][QC].v, ct) : 0u;
        }
        __syncthreads();
        uint32_t kp = s_kbase + s_keep[warp] + kin - tk;
        uint32_t sp = s_sbase + s_short[warp] + sin - tsh;
        uint32_t cp = s_cbase + s_chunk[warp] + cin - tch;
#pragma unroll
        for (int i = 0; i < NPT; i++) {
            if (keeps[i]) out[kp++] = xs[i];
            if (shorts[i]) write_short(j, q, sp++, xs[i]);
            if (nchs[i]) {
                write_chunks(j, q, cp, xs[i], 0, nchs[i], k);
                cp += nchs[i];
            }
        }
        __syncthreads();
    }
}

template <int G, bool MULTI>
__device__ __forceinline__ void scan_nodes(const PeelJob& j, const uint32_t* src, uint32_t cnt_nodes,
                                           uint32_t k, uint32_t q, uint32_t* out,
                                           uint32_t* out_cnt, uint32_t* out_cnt0) {
    // grid-uniform choice (every block sees the same count)
    if (G == 1 && (uint64_t)cnt_nodes >= 4ull * gridDim.x * blockDim.x)
        scan_nodes_n<G, MULTI, 4>(j, src, cnt_nodes, k, q, out, out_cnt, out_cnt0);
    else
        scan_nodes_n<G, MULTI, 1>(j, src, cnt_nodes, k, q, out, out_cnt, out_cnt0);
}

// Every column of every segment starts from the full degrees.
template <bool MULTI>
__device__ __forceinline__ void phase_init(const PeelJob& j) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    for (uint32_t s = 0; s < j.nseg; s++) {
        const SegP g = seg_load<MULTI>(j, s);
        for (uint64_t i = tid; i < g.nL; i += stride) {
            const uint32_t d0 = __ldg(g.deg0 + i);
            for (uint32_t c = 0; c < g.ncols; c++) g.deg[(uint64_t)c * g.nL + i] = d0;
        }
    }
}

template <int G, bool MULTI>
__device__ __forceinline__ void phase_scan(const PeelJob& j, bool first) {
    const PeelCtl* c = j.ctl;
    const uint32_t k = ld_l2(&c->level);
    const uint32_t q = ld_l2(&c->q_cur);
    // the other parity's queues held the previous level's items: blank them
    const uint32_t ps = min(ld_l2(&c->prev_tail[QS]), j.qs_cap);
    const uint32_t pc = min(ld_l2(&c->prev_tail[QC]), j.qc_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ps; i += gridDim.x * blockDim.x)
        j.qs[q ^ 1][i] = EMPTY32;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pc; i += gridDim.x * blockDim.x)
        j.qc[q ^ 1][i] = EMPTY;
    if (first) {
        scan_nodes<G, MULTI>(j, nullptr, j.nx, k, q, j.alive[1], &j.ctl->alive_cnt[1],
                             &j.ctl->alive0[1]);
    } else {
        const uint32_t a = ld_l2(&c->alive_cur);
        scan_nodes<G, MULTI>(j, j.alive[a], ld_l2(&c->alive_cnt[a]), k, q, j.alive[a ^ 1],
                             &j.ctl->alive_cnt[a ^ 1], &j.ctl->alive0[a ^ 1]);
    }
}

// The level is complete once every reserved item has been processed.  All
// four counters only grow, so reading the processed counts first and finding
// their sum equal to the reserved sum proves the two were equal at the time
// of the first read.
__device__ __forceinline__ bool level_done(PeelCtl* c, uint32_t q) {
    const uint32_t p = ld_acquire(&c->processed[q][QS].v) + ld_acquire(&c->processed[q][QC].v);
    const uint32_t t = ld_acquire(&c->tail[q][QS].v) + ld_acquire(&c->tail[q][QC].v);
    return p == t;
}

// Warp-uniform decision while waiting (lane 0 decides): 0 keep waiting, 1 the
// level is done, 2 an error was recorded or this warp made no progress for
// the timeout.
__device__ __forceinline__ bool past_deadline(const PeelJob& j, uint64_t now) {
    return now - ld_l2_64(&j.ctl->t_start) > j.deadline_ns;
}

__device__ __forceinline__ uint32_t wait_check(const PeelJob& j, uint32_t q, uint64_t t0) {
    uint32_t r = 0;
    if ((threadIdx.x & 31) == 0) {
        const uint64_t now = global_ns();
        if (level_done(j.ctl, q)) {
            r = 1;
        } else if (now - t0 > j.timeout_ns || ld_l2(&j.ctl->err) != ERR_NONE) {
            atomicCAS(&j.ctl->err, ERR_NONE, ERR_BARRIER);
            r = 2;
        } else if (past_deadline(j, now)) {
            atomicCAS(&j.ctl->err, ERR_NONE, ERR_DEADLINE);
            r = 2;
        }
    }
    return __shfl_sync(0xffffffffu, r, 0);
}

// A dequeued item that names no node of the launch: the first one is
// recorded and the run ends with ERR_ITEM; the item itself is skipped.
__device__ __noinline__ void record_bad(const PeelJob& j, uint32_t item, uint32_t where) {
    if (atomicCAS(&j.ctl->err, ERR_NONE, ERR_ITEM) == ERR_NONE) {
        j.ctl->bad_item = item;
        j.ctl->bad_where = where;
    }
}

// Adds this warp's processed-item counts (ps short, pc chunk items; warp
// uniform) to the grid-wide ones and clears them.  The items the warp queued
// while processing them were reserved (tail raised, by returning atomics)
// before the fence, so the sums of level_done cannot meet early.  Counts are
// flushed in batches -- the fence is the expensive part -- and always before
// the warp polls for the end of the level, so they only ever lag.
__device__ __forceinline__ void flush_processed(PeelCtl* c, uint32_t q, uint32_t& ps,
                                                uint32_t& pc) {
    if ((ps | pc) == 0) return;
    __syncwarp();
    if ((threadIdx.x & 31) == 0) {
        __threadfence();
        if (ps) atomicAdd(&c->processed[q][QS].v, ps);
        if (pc) atomicAdd(&c->processed[q][QC].v, pc);
    }
    ps = 0;
    pc = 0;
}

// Short rows of the lanes with `ready` set (at most small_row entries each),
// flattened over the warp's lanes; the owner of entry q is found by binary
// search over the warp's exclusive scan of row lengths.
template <bool MULTI>
__device__ __forceinline__ void expand_short(const PeelJob& j, uint32_t k, uint32_t q, uint32_t x,
                                             bool ready, Local& loc) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t s = seg_of<MULTI>(j, x);
    const SegP g = seg_load<MULTI>(j, s);
    const uint32_t xl = x - g.xbase;
    const uint32_t col = g.divN.div(xl);
    const uint32_t v = xl - col * g.n;
    uint32_t b = 0, len = 0;
    const uint32_t* adj = g.adj;
    if (ready) {
        b = __ldg(g.node_ptr + v);
        len = __ldg(g.node_ptr + v + 1) - b;
        if (len > j.small_row) {  // long rows are never queued as short items
            record_bad(j, x, 1);
            len = 0;
        }
    }
    const uint32_t incl = warp_incl_scan(len);
    const uint32_t excl = incl - len;
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    for (uint32_t jb = 0; jb < total; jb += 128) {
        uint32_t segs[4], cols[4], slot[4];
        bool ok[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint32_t qq = jb + 32 * i + lane;
            uint32_t own = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                uint32_t cand = own + step;
                uint32_t ex = __shfl_sync(0xffffffffu, excl, cand & 31);
                if (cand < 32 && ex <= qq) own = cand;
            }
            const uint32_t ob = __shfl_sync(0xffffffffu, b, own);
            const uint32_t oe = __shfl_sync(0xffffffffu, excl, own);
            cols[i] = __shfl_sync(0xffffffffu, col, own);
            segs[i] = MULTI ? __shfl_sync(0xffffffffu, s, own) : 0u;
            const uint32_t* oadj = MULTI ? (const uint32_t*)__shfl_sync(
                                               0xffffffffu, (unsigned long long)adj, own)
                                         : adj;
            ok[i] = qq < total;
            slot[i] = ok[i] ? __ldg(oadj + ob + (qq - oe)) : 0u;
        }
        visit4<MULTI>(j, segs, cols, slot, ok, k, q, loc);
    }
}

// One chunk of a long row (chunk_word), by the whole warp (CHUNK / 32
// entries per lane).
template <bool MULTI>
__device__ __forceinline__ void expand_chunk(const PeelJob& j, uint32_t k, uint32_t q,
                                             unsigned long long it, Local& loc) {
    constexpr int PER_LANE = CHUNK / 32;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t x = (uint32_t)it, w = (uint32_t)(it >> 32);
    const SegP g = seg_load<MULTI>(j, seg_of<MULTI>(j, x));
    const uint32_t xl = x - g.xbase;
    const uint32_t col = g.divN.div(xl);
    const uint32_t v = xl - col * g.n;
    const uint32_t rb = __ldg(g.node_ptr + v), re = __ldg(g.node_ptr + v + 1);
    const uint32_t len = re - rb, full = (len + CHUNK - 1) / CHUNK;
    const bool strided = (w & STRIDED) != 0;
    const uint32_t nch = strided ? (w >> 16) & 0x7FFFu : 0u;
    const uint32_t ch = strided ? (w & 0xFFFFu) : w;
    if (strided ? (ch >= nch || nch > full) : ch >= full) {  // no such chunk of the row
        if (lane == 0) record_bad(j, x, 2);
        return;
    }
    // row offset of this lane's first entry and the step between its entries;
    // offsets stay below 256 * full, under 2^24 when strided
    const uint32_t o0 = strided ? 8u * (ch + lane * nch) : ch * CHUNK + lane;
    const uint32_t step = strided ? 1u : 32u;
    uint32_t slot[PER_LANE];
    bool ok[PER_LANE];
#pragma unroll
    for (int i = 0; i < PER_LANE; i++) {
        const uint32_t o = o0 + step * i;
        ok[i] = o < len && (strided || o < (ch + 1) * CHUNK);
        slot[i] = ok[i] ? __ldg(g.adj + rb + o) : 0u;
    }
    visit_node<PER_LANE>(j, g, col, slot, ok, k, q, loc);
}

// Per-block drain state in shared memory: `done` is set when the level is
// over (or the run failed), `wake` is bumped by warp 0 whenever it sees more
// unclaimed queue items than it takes itself.
struct DrainBlock {
    uint32_t done, wake;
};

// An idle warp holding no claim parks on its block's shared state instead of
// polling the grid-wide queue counters: it resumes claiming when warp 0 sees
// unclaimed work, and leaves DRAIN when the level is over.  Returns true to
// leave.  Bounded by the run's deadline.
__device__ __forceinline__ bool park(const PeelJob& j, volatile DrainBlock* sb) {
    uint32_t r = 0;
    if ((threadIdx.x & 31) == 0) {
        const uint32_t w0 = sb->wake;
        for (uint32_t spins = 1;; spins++) {
            if (sb->done) {
                r = 1;
                break;
            }
            if (sb->wake != w0) break;
            __nanosleep(256);
            if ((spins & 255) == 0 &&
                (past_deadline(j, global_ns()) || ld_l2(&j.ctl->err) != ERR_NONE)) {
                atomicCAS(&j.ctl->err, ERR_NONE, ERR_DEADLINE);
                sb->done = 1;
                r = 1;
                break;
            }
        }
    }
    return __shfl_sync(0xffffffffu, r, 0) != 0;
}

// DRAIN(K): each warp holds at most one chunk claim (one item) and one
// short-row claim (32 slots, one per lane) at a time, polls both, and works
// on whatever is ready; it stops once no queued item is left unprocessed.  A
// claim may run past the reserved items when warps race for the last ones;
// such a slot is either filled by a later removal or abandoned when the level
// completes -- meanwhile the warp keeps serving the other queue.
template <bool MULTI>
__device__ __forceinline__ void phase_drain(const PeelJob& j, volatile DrainBlock* sb) {
    PeelCtl* c = j.ctl;
    const uint32_t k = ld_l2(&c->level);
    const uint32_t q = ld_l2(&c->q_cur);
    const uint32_t lane = threadIdx.x & 31;
    const bool warp0 = (threadIdx.x >> 5) == 0;
    constexpr uint32_t NONE = 0xFFFFFFFFu;
    uint64_t t0 = global_ns();  // last progress of this warp
    uint32_t ns = 32;
    uint32_t cidx = NONE;       // held chunk slot (warp-uniform)
    uint32_t sidx = NONE;       // this lane's held short slot
    uint32_t idle = 0;          // consecutive polls without work
    uint32_t busy = 0;          // polls with work (lane 0's count)
    uint32_t pend_s = 0, pend_c = 0;  // processed items not yet flushed
    Local loc{EMPTY32, 0};            // a removal this warp expands itself next
    for (;;) {
        bool progress = false;
        if (loc.x != EMPTY32) {
            // the warp's own removal first: the next step of its cascade
            const Local cur = loc;
            loc.x = EMPTY32;
            if (cur.chunk)
                expand_chunk<MULTI>(j, k, q,
                                    (unsigned long long)cur.x |
                                        ((unsigned long long)chunk_word(0, cur.chunk, k) << 32),
                                    loc);
            else expand_short<MULTI>(j, k, q, lane == 0 ? cur.x : 0u, lane == 0, loc);
            progress = true;
            goto done_work;
        }
        {
        // new claims, decided by lane 0
        uint32_t want = 0, cb = NONE, sbase = NONE;
        const bool hold_s = __any_sync(0xffffffffu, sidx != NONE);
        if (lane == 0) {
            const uint32_t tc = ld_l2(&c->tail[q][QC].v), hc = ld_l2(&c->head[q][QC].v);
            const uint32_t ts = ld_l2(&c->tail[q][QS].v), hs = ld_l2(&c->head[q][QS].v);
            if (cidx == NONE && tc > hc) {
                cb = atomicAdd(&c->head[q][QC].v, 1u);
                want |= 1;
            }
            if (!hold_s && ts > hs) {
                sbase = atomicAdd(&c->head[q][QS].v, 32u);
                want |= 2;
            }
            // more unclaimed items than this warp takes: wake the parked warps
            if (warp0 && (tc > hc + 1 || ts > hs + 32)) sb->wake = sb->wake + 1;
        }
        want = __shfl_sync(0xffffffffu, want, 0);
        if (want & 1) cidx = __shfl_sync(0xffffffffu, cb, 0);
        if (want & 2) sidx = __shfl_sync(0xffffffffu, sbase, 0) + lane;
        // a ready chunk item
        if (cidx != NONE) {
            unsigned long long it = EMPTY;
            if (lane == 0 && cidx < j.qc_cap) it = ld_relaxed64(j.qc[q] + cidx);
            it = __shfl_sync(0xffffffffu, it, 0);
            if (it != EMPTY) {
                if ((uint32_t)it < j.nx) expand_chunk<MULTI>(j, k, q, it, loc);
                else if (lane == 0) record_bad(j, (uint32_t)it, 3);
                pend_c += 1;
                cidx = NONE;
                progress = true;
            }
        }
        // the ready short items among this warp's slots
        {
            uint32_t x = EMPTY32;
            if (sidx != NONE && sidx < j.qs_cap) x = __ldcg(j.qs[q] + sidx);
            const bool ready = x != EMPTY32;
            const bool bad = ready && x >= j.nx;
            if (bad) record_bad(j, x, 4);
            const uint32_t rmask = __ballot_sync(0xffffffffu, ready);
            if (rmask) {
                expand_short<MULTI>(j, k, q, ready && !bad ? x : 0u, ready && !bad, loc);
                if (ready) sidx = NONE;
                pend_s += (uint32_t)__popc(rmask);
                progress = true;
            }
        }
        }
    done_work:
        if (progress) {
            // never while a kept removal is pending: its parent must not count
            // as processed before the removal's row is visited
            if (pend_s + pend_c >= 16 && loc.x == EMPTY32) flush_processed(c, q, pend_s, pend_c);
            t0 = global_ns();
            ns = 32;
            idle = 0;
            // a warp that keeps finding work still ends by the run's deadline
            uint32_t stop = 0;
            if (lane == 0 && ((++busy & 63) == 0) &&
                (past_deadline(j, t0) || ld_l2(&c->err) != ERR_NONE)) {
                atomicCAS(&c->err, ERR_NONE, ERR_DEADLINE);
                sb->done = 1;
                stop = 1;
            }
            if (__shfl_sync(0xffffffffu, stop, 0)) return;
        } else {
            // nothing ready: done when every reserved item is processed (any
            // slots still held were overclaims), else wait a little.  Warp 0
            // keeps polling the grid-wide counters for the whole level; the
            // other warps, once idle for a while and holding no claim, park
            // on the block's shared state so that idle warps do not flood the
            // counters with polls.
            flush_processed(c, q, pend_s, pend_c);
            if (wait_check(j, q, t0)) {
                if (lane == 0) sb->done = 1;
                return;
            }
            if (!warp0 && ++idle >= j.idle_polls && cidx == NONE &&
                !__any_sync(0xffffffffu, sidx != NONE)) {
                if (park(j, sb)) return;
                idle = 0;
                ns = 32;
                t0 = global_ns();
                continue;
            }
            __nanosleep(ns);
            if (ns < 512) ns <<= 1;
        }
    }
}

// T threads per block, 1024 threads resident per SM (512 x 2 or 1024 x 1):
// at most 64 registers a thread.  (Three 512-thread blocks per SM at 40
// registers, with spills, measured slower: c4 batch 682 -> 814 ms.)
template <int G, int T, bool MULTI, int BPS = 1024 / T>
__global__ void __launch_bounds__(T, BPS) k_peel(PeelJob j) {
    __shared__ DrainBlock s_drain;
    phase_init<MULTI>(j);
    if (!grid_barrier(j)) return;
    phase_scan<G, MULTI>(j, true);
    if (!grid_barrier(j)) return;
    for (;;) {
        const uint32_t ph = ld_l2(&j.ctl->phase);
        if (ph == PH_DRAIN) {
            if (threadIdx.x == 0) s_drain = DrainBlock{0u, 0u};
            __syncthreads();
            phase_drain<MULTI>(j, &s_drain);
        } else if (ph == PH_SCAN) {
            phase_scan<G, MULTI>(j, false);
        } else {
            return;
        }
        if (!grid_barrier(j)) return;
    }
}

// ---- host ---------------------------------------------------------------------

static uint32_t env_u32(const char* name, uint32_t dflt) {
    const char* s = getenv(name);
    return s && *s ? (uint32_t)strtoul(s, nullptr, 10) : dflt;
}

uint32_t peel_columns_per_group(const DeviceGraph* d) {
    // every column needs an n*L degree table plus ~8 words per node; keep the
    // group's working set within a budget (FC_PEEL_GROUP_MB, default 4 GiB)
    uint64_t per_col = ((uint64_t)d->n * d->L + 8ull * d->n) * 4 + d->entries / 8;
    uint64_t budget = (uint64_t)env_u32("FC_PEEL_GROUP_MB", 4096) << 20;
    uint64_t cols = per_col ? budget / per_col : d->L;
    uint32_t want = env_u32("FC_PEEL_GROUP_COLS", 0);
    if (want) cols = want;
    if (cols < 1) cols = 1;
    if (cols > d->L) cols = d->L;
    // the (column, node) index must stay below 2^32
    while (cols > 1 && (uint64_t)cols * d->n >= (1ull << 32)) cols--;
    return (uint32_t)cols;
}

template <int G, int T, bool MULTI, int BPS = 1024 / T>
static fc_status launch_t(PeelJob& j, cudaStream_t s) {
    int dev = 0, sms = 0, occ = 0;
    FC_CUDA_TRY(cudaGetDevice(&dev));
    FC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    FC_CUDA_TRY(
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_peel<G, T, MULTI, BPS>, T, 0));
    if (occ < 1) return FC_ERR_DEVICE;
    uint32_t want_occ = env_u32("FC_PEEL_BLOCKS_PER_SM", BPS);
    if (want_occ >= 1 && (int)want_occ < occ) occ = (int)want_occ;
    if (j.max_sms && (int)j.max_sms < sms) sms = (int)j.max_sms;
    dim3 grid(sms * occ), block(T);
    void* args[] = {&j};
    FC_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_peel<G, T, MULTI, BPS>, grid, block, args, 0,
                                            s));
    return FC_OK;
}

template <int G, bool MULTI>
static fc_status launch_g(PeelJob& j, uint32_t threads, cudaStream_t s) {
    if (threads == 1024) return launch_t<G, 1024, MULTI>(j, s);
    return launch_t<G, 512, MULTI>(j, s);
}

// Lanes per node in SCAN: one when every segment has at most 32 layers (its L
// loads are independent), else a group of 32.
template <bool MULTI>
static fc_status launch(PeelJob& j, uint32_t maxL, uint32_t threads, cudaStream_t s) {
    if (maxL <= 32) return launch_g<1, MULTI>(j, threads, s);
    return launch_g<32, MULTI>(j, threads, s);
}

static uint32_t default_threads() { return env_u32("FC_PEEL_THREADS", 1024) == 512 ? 512 : 1024; }

// Queue capacities: a level removes each node at most once; short rows take
// one qs item, long rows at most entries/CHUNK + 1 qc items.
static void queue_caps(uint64_t nx, uint64_t col_entries, uint64_t* qs_cap, uint64_t* qc_cap) {
    *qs_cap = nx + 64;
    *qc_cap = nx + (col_entries + CHUNK - 1) / CHUNK + 64;
}

static uint64_t shared_ws_bytes(uint64_t nx, uint64_t col_entries) {
    uint64_t qs_cap, qc_cap;
    queue_caps(nx, col_entries, &qs_cap, &qc_cap);
    // qc0 qc1 (u64) | qs0 qs1 | bits | cnt alive0 alive1 | control block (256-aligned)
    return 4 * (4 * qc_cap + 2 * qs_cap + (nx + 31) / 32 + 3 * nx) + sizeof(PeelCtl) + 256;
}

uint64_t peel_ws_bytes(uint32_t n, uint32_t L, uint64_t entries, uint32_t ncols) {
    const uint64_t nx = (uint64_t)ncols * n;
    return shared_ws_bytes(nx, (uint64_t)ncols * entries) + 4ull * ncols * n * L + 256;
}

// Lays the shared part of the workspace out at `w` (queues, counts, lists,
// control block) and sets the job's pointers; returns the first free byte.
static char* carve_shared(PeelJob& j, char* w, char* end, uint64_t nx, uint64_t col_entries,
                          cudaStream_t s, fc_status* rc) {
    uint64_t qs_cap, qc_cap;
    queue_caps(nx, col_entries, &qs_cap, &qc_cap);
    *rc = FC_OK;
    if (qc_cap >= (1ull << 32) || qs_cap >= (1ull << 32) || nx >= (1ull << 32)) {
        *rc = FC_ERR_TOO_LARGE;
        return w;
    }
    uint32_t* p = (uint32_t*)w;
    j.qc[0] = (unsigned long long*)p;
    p += 2 * qc_cap;
    j.qc[1] = (unsigned long long*)p;
    p += 2 * qc_cap;
    j.qs[0] = p;
    p += qs_cap;
    j.qs[1] = p;
    p += qs_cap;
    j.bits = p;
    p += (nx + 31) / 32;
    j.qc_cap = (uint32_t)qc_cap;
    j.qs_cap = (uint32_t)qs_cap;
    j.nx = (uint32_t)nx;
    j.cnt = p;
    p += nx;
    j.alive[0] = p;
    p += nx;
    j.alive[1] = p;
    p += nx;
    j.ctl = (PeelCtl*)(((uintptr_t)p + 255) & ~(uintptr_t)255);
    char* next = (char*)(j.ctl + 1);
    if (next > end) {  // layout check
        *rc = FC_ERR_INVALID;
        return w;
    }
    return next;  // the queues and the control block are cleared by reset_job
}

// Launches the prepared job and reads its control block back.
// Every queue slot starts EMPTY and every x alive (qc, qs and the bitmap are
// contiguous); the control block starts all zero, which is phase INIT.
static fc_status reset_job(const PeelJob& j, cudaStream_t s) {
    const uint64_t words = 4ull * j.qc_cap + 2ull * j.qs_cap + (j.nx + 31ull) / 32;
    FC_CUDA_TRY(cudaMemsetAsync(j.qc[0], 0xFF, words * 4, s));
    FC_CUDA_TRY(cudaMemsetAsync(j.ctl, 0, sizeof(PeelCtl), s));
    return FC_OK;
}

template <bool MULTI>
static fc_status run_job(PeelJob& j, uint32_t maxL, uint32_t threads, cudaStream_t s,
                         PeelStats* st, bool instrument, uint32_t col0, uint32_t ncols,
                         bool* use_graph = nullptr, PeelCtl* ctl_out = nullptr) {
    j.idle_polls = env_u32("FC_PEEL_IDLE_POLLS", 2);
    if (!j.small_row) j.small_row = env_u32("FC_PEEL_SMALL_ROW", SMALL_ROW_DEFAULT);
    j.timeout_ns = (uint64_t)env_u32("FC_BARRIER_TIMEOUT_MS", 10000) * 1000000ull;
    j.deadline_ns = (uint64_t)env_u32("FC_PEEL_DEADLINE_MS", 60000) * 1000000ull;
    j.trace = nullptr;
    j.trace_levels = 0;
    const bool tracing = instrument && env_u32("FC_PEEL_TRACE", 0) != 0;
    if (tracing) {
        j.trace_levels = j.max_level + 2;
        FC_TRY(dev_alloc((void**)&j.trace, 6ull * 8 * j.trace_levels, s));
        FC_CUDA_TRY(cudaMemsetAsync(j.trace, 0, 6ull * 8 * j.trace_levels, s));
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (instrument) {
        FC_CUDA_TRY(cudaEventCreate(&e0));
        FC_CUDA_TRY(cudaEventCreate(&e1));
        count_alloc(2);
    }
    // the run: clear the queues and the control block, then the launch --
    // captured as one CUDA graph when asked (and when the driver captures a
    // cooperative launch), else issued directly
    bool graphed = false;
    if (use_graph && *use_graph) {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        bool ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            fc_status r1 = reset_job(j, s);
            fc_status r2 = r1 == FC_OK ? launch<MULTI>(j, maxL, threads, s) : r1;
            ok = cudaStreamEndCapture(s, &graph) == cudaSuccess && r2 == FC_OK;
        }
        if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
        if (ok) {
            if (instrument) FC_CUDA_TRY(cudaEventRecord(e0, s));
            ok = cudaGraphLaunch(exec, s) == cudaSuccess;
            graphed = ok;
        }
        cudaGetLastError();  // a refused capture falls back to direct launches
        if (graph && !graphed) cudaGraphDestroy(graph);
        if (exec && !graphed) cudaGraphExecDestroy(exec);
        if (graphed) {
            if (instrument) FC_CUDA_TRY(cudaEventRecord(e1, s));
            FC_CUDA_TRY(cudaStreamSynchronize(s));
            cudaGraphExecDestroy(exec);
            cudaGraphDestroy(graph);
        }
    }
    if (!graphed) {
        if (instrument) FC_CUDA_TRY(cudaEventRecord(e0, s));
        FC_TRY(reset_job(j, s));
        FC_TRY(launch<MULTI>(j, maxL, threads, s));
        if (instrument) FC_CUDA_TRY(cudaEventRecord(e1, s));
    }
    if (use_graph) *use_graph = graphed;
    count_launch();
    PeelCtl out;
    FC_TRY(to_host(&out, j.ctl, sizeof(out), s));
    if (ctl_out) *ctl_out = out;
    float ms = 0;
    if (instrument) {
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    if (st) {
        st->ms = ms;
        st->levels = out.levels;
        st->subrounds = out.items;
        st->err = out.err;
        st->phase_ms[0] = out.ph_ns[0] * 1e-6;
        st->phase_ms[1] = out.ph_ns[1] * 1e-6;
        st->phase_ms[2] = 0;
    }
    if (tracing) {
        // one line per level: level, scan us, drain us, queue items, alive
        std::vector<unsigned long long> tr(6ull * j.trace_levels);
        cudaMemcpy(tr.data(), j.trace, tr.size() * 8, cudaMemcpyDeviceToHost);
        dev_free(j.trace, s);
        for (uint32_t l = 0; l < j.trace_levels; l++) {
            const unsigned long long* r = tr.data() + 6ull * l;
            if (r[0] || r[3])
                fprintf(stderr, "peel-trace cols %u+%u level %u scan_us %.1f drain_us %.1f items %llu alive %llu\n",
                        col0, ncols, l, r[0] * 1e-3, r[3] * 1e-3, r[4] ? r[4] : r[1], r[2]);
        }
    }
    if (out.err) {
        if (env_u32("FC_DEBUG", 0))
            fprintf(stderr, "peel: error %u at level %u of %u (bad item %u, check %u), %u segments\n",
                    out.err, out.err_level, j.max_level, out.bad_item, out.bad_where, j.nseg);
        return FC_ERR_ITER_LIMIT;
    }
    return FC_OK;
}

// ---- endgame: each column's last levels inside one block --------------------
//
// Near the end of a peel the grid-wide levels cost their barriers, not their
// work.  After level K the nodes still alive are exactly those whose core
// exceeds K, and for k > K the (k, lambda)-cores of the graph are those of the
// subgraph they induce.  So k_peel stops once few nodes are alive
// (stop_alive), each column's survivors are given local ids and their
// subgraph is compacted (k_eg_index, k_eg_scan, k_eg_fill), and one block per
// column runs the remaining levels on it (k_endgame) with the same rules:
// degrees, counts, alive flags, lists and queue in shared memory, rounds
// separated by __syncthreads instead of grid barriers.  Every loop is bounded
// (levels by the level cap, rounds by the survivors); no block waits on
// another.

constexpr uint32_t EG_THREADS = 1024;
constexpr uint32_t EG_MAX_COLS = 64;
constexpr uint32_t EG_SMEM = 220u * 1024u;  // dynamic shared memory of k_endgame
constexpr uint32_t EG_FILL_SPLIT = 4096;    // longer rows are filled by a whole block

// shared bytes per survivor: degrees (L halves), count (a half), alive flag,
// two alive lists and the queue (16-bit local ids)
static uint32_t eg_node_bytes(uint32_t L) { return 2 * L + 9; }
// survivors one column's block can hold (0: the endgame is off for this L)
static uint32_t eg_capacity(uint32_t L) {
    const uint64_t fixed = 8ull * EG_THREADS + 256;  // batch prefixes and row starts + alignment
    uint64_t cap = (EG_SMEM - fixed) / eg_node_bytes(L);
    if (cap > 65535) cap = 65535;
    return cap >= 1024 ? (uint32_t)cap : 0u;
}

// Local ids of the survivors, per column; their subgraph row lengths are
// the alive-neighbour degrees the peel maintained.
__global__ void k_eg_index(const uint32_t* __restrict__ alive, uint32_t nalive,
                           const uint32_t* __restrict__ bits, FastDiv divN, uint32_t n, uint32_t L,
                           const uint32_t* __restrict__ deg, uint32_t cap,
                           uint32_t* __restrict__ map, uint32_t* __restrict__ ecnt,
                           uint32_t* __restrict__ l2g, uint32_t* __restrict__ rowlen) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nalive;
         i += gridDim.x * blockDim.x) {
        const uint32_t x = alive[i];
        if (!((bits[x >> 5] >> (x & 31)) & 1u)) continue;
        const uint32_t c = divN.div(x), v = x - c * n;
        const uint32_t lid = atomicAdd(ecnt + c, 1u);
        if (lid >= cap) continue;  // the host sees the count and fails the run
        map[x] = lid;
        l2g[(uint64_t)c * cap + lid] = v;
        const uint32_t* d = deg + (uint64_t)c * n * L + (uint64_t)v * L;
        uint32_t sum = 0;
        for (uint32_t l = 0; l < L; l++) sum += d[l];
        rowlen[(uint64_t)c * (cap + 1) + lid] = sum;
    }
}

// Block-wide exclusive scan of the 1024 threads' values; returns the total.
__device__ __forceinline__ uint32_t eg_block_scan(uint32_t v, uint32_t* excl, uint32_t* s_warp) {
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t in = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, in, d);
        if (lane >= (uint32_t)d) in += t;
    }
    __syncthreads();
    if (lane == 31) s_warp[w] = in;
    __syncthreads();
    if (w == 0) {
        uint32_t x = s_warp[lane];
        uint32_t y = x;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, y, d);
            if (lane >= (uint32_t)d) y += t;
        }
        s_warp[lane] = y - x;  // exclusive
        if (lane == 31) s_warp[32] = y;
    }
    __syncthreads();
    *excl = s_warp[w] + in - v;
    const uint32_t total = s_warp[32];
    __syncthreads();
    return total;
}

// One block per column: row offsets of its subgraph (exclusive scan of the
// row lengths, m + 1 values) and its entry count.
__global__ void __launch_bounds__(EG_THREADS) k_eg_scan(const uint32_t* __restrict__ rowlen,
                                                        uint32_t* __restrict__ rowptr, uint32_t cap,
                                                        const uint32_t* __restrict__ ecnt,
                                                        uint32_t* __restrict__ etot,
                                                        uint32_t* __restrict__ nbig) {
    __shared__ uint32_t s_warp[33];
    const uint32_t c = blockIdx.x;
    if (c == 0 && threadIdx.x == 0) *nbig = 0;  // k_eg_fill lists the long rows
    const uint32_t m = min(ecnt[c], cap);
    const uint32_t* in = rowlen + (uint64_t)c * (cap + 1);
    uint32_t* out = rowptr + (uint64_t)c * (cap + 1);
    const uint32_t per = (m + EG_THREADS - 1) / EG_THREADS;
    const uint32_t b = threadIdx.x * per, e = min(m, b + per);
    uint32_t sum = 0;
    for (uint32_t i = b; i < e; i++) sum += in[i];
    uint32_t base;
    const uint32_t total = eg_block_scan(sum, &base, s_warp);
    for (uint32_t i = b; i < e; i++) {
        out[i] = base;
        base += in[i];
    }
    if (threadIdx.x == 0) {
        out[m] = total;
        etot[c] = total;
    }
}

// The part of survivor v's row that can name survivors: an ordered row is read
// only as far as its entries of bucket >= bucket_of(K+1), the rest name nodes
// whose bound, hence core, is at most K.
__device__ __forceinline__ uint32_t eg_need(const uint32_t* __restrict__ node_ptr,
                                            const uint32_t* __restrict__ big_id,
                                            const uint32_t* __restrict__ ptab, uint32_t v,
                                            uint32_t k1, uint32_t* rb) {
    *rb = node_ptr[v];
    const uint32_t len = node_ptr[v + 1] - *rb;
    uint32_t need = len;
    if (big_id && len > ORDER_MIN_ROW) {
        const uint32_t id = big_id[v];
        if (id != NO_BIG_ROW) need = min(len, ptab[(uint64_t)id * BUCKETS + bucket_of(k1)]);
    }
    return need;
}

// One warp per survivor whose row part is at most EG_FILL_SPLIT entries: its
// subgraph row, the alive neighbours in row order, as local slots lid * L + l.
// Rows whose alive-neighbour count differs from the degrees the peel kept
// flag an error.  A longer row's node is appended to `list` (capacity lcap,
// count *nbig) for k_eg_fill_big.
__global__ void k_eg_fill(const uint32_t* __restrict__ alive, uint32_t nalive,
                          const uint32_t* __restrict__ bits, FastDiv divN, FastDiv divL, uint32_t n,
                          uint32_t L, const uint32_t* __restrict__ node_ptr,
                          const uint32_t* __restrict__ adj, const uint32_t* __restrict__ big_id,
                          const uint32_t* __restrict__ ptab, uint32_t k1,
                          const uint32_t* __restrict__ map, uint32_t cap,
                          const uint32_t* __restrict__ rowptr, const uint64_t* __restrict__ base,
                          uint32_t* __restrict__ H, uint32_t* __restrict__ err,
                          uint32_t* __restrict__ list, uint32_t lcap, uint32_t* __restrict__ nbig) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nalive; i += warps) {
        const uint32_t x = alive[i];
        if (!((bits[x >> 5] >> (x & 31)) & 1u)) continue;
        const uint32_t c = divN.div(x), v = x - c * n;
        const uint32_t lid = map[x];
        if (lid >= cap) continue;
        const uint32_t* rp = rowptr + (uint64_t)c * (cap + 1);
        const uint32_t o0 = rp[lid], want = rp[lid + 1] - o0;
        uint32_t* dst = H + base[c] + o0;
        uint32_t rb;
        const uint32_t need = eg_need(node_ptr, big_id, ptab, v, k1, &rb);
        if (need > EG_FILL_SPLIT) {  // k_eg_fill_big
            if (lane == 0) {
                const uint32_t pos = atomicAdd(nbig, 1u);
                if (pos < lcap) list[pos] = x;
                else atomicExch(err, 1u);
            }
            continue;
        }
        uint32_t got = 0;
        for (uint32_t p0 = 0; p0 < need; p0 += 32) {
            const uint32_t p = p0 + lane;
            uint32_t u = 0, l = 0;
            bool al = false;
            if (p < need) {
                const uint32_t slot = adj[rb + p];
                u = divL.div(slot);
                l = slot - u * L;
                const uint32_t y = c * n + u;
                al = (bits[y >> 5] >> (y & 31)) & 1u;
            }
            const uint32_t mk = __ballot_sync(0xffffffffu, al);
            if (al) {
                const uint32_t pos = got + __popc(mk & lt);
                if (pos < want) dst[pos] = map[c * n + u] * L + l;
            }
            got += __popc(mk);
        }
        if (lane == 0 && got != want) atomicExch(err, 1u);
    }
}

// One block per survivor whose row part exceeds EG_FILL_SPLIT entries (the
// nodes k_eg_fill listed), in tiles of 4 * EG_THREADS entries: each thread
// counts its four, a block scan places them (thread-major within a tile;
// deterministic, whatever the list's order).
__global__ void __launch_bounds__(EG_THREADS) k_eg_fill_big(
    const uint32_t* __restrict__ bits, FastDiv divN, FastDiv divL, uint32_t n, uint32_t L,
    const uint32_t* __restrict__ node_ptr,
    const uint32_t* __restrict__ adj, const uint32_t* __restrict__ big_id,
    const uint32_t* __restrict__ ptab, uint32_t k1, const uint32_t* __restrict__ map, uint32_t cap,
    const uint32_t* __restrict__ rowptr, const uint64_t* __restrict__ base,
    uint32_t* __restrict__ H, uint32_t* __restrict__ err, const uint32_t* __restrict__ list,
    uint32_t lcap, const uint32_t* __restrict__ nbig) {
    __shared__ uint32_t s_warp[33];
    const uint32_t nl = min(*nbig, lcap);
    for (uint32_t i = blockIdx.x; i < nl; i += gridDim.x) {
        const uint32_t x = list[i];
        const uint32_t c = divN.div(x), v = x - c * n;
        const uint32_t lid = map[x];
        if (lid >= cap) continue;
        uint32_t rb;
        const uint32_t need = eg_need(node_ptr, big_id, ptab, v, k1, &rb);
        const uint32_t* rp = rowptr + (uint64_t)c * (cap + 1);
        const uint32_t o0 = rp[lid], want = rp[lid + 1] - o0;
        uint32_t* dst = H + base[c] + o0;
        uint32_t got = 0;
        for (uint32_t p0 = 0; p0 < need; p0 += 4 * EG_THREADS) {
            uint32_t val[4], cnt = 0;
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const uint32_t p = p0 + r * EG_THREADS + threadIdx.x;
                val[r] = UNSET;
                if (p < need) {
                    const uint32_t slot = adj[rb + p];
                    const uint32_t u = divL.div(slot), l = slot - u * L;
                    const uint32_t y = c * n + u;
                    if ((bits[y >> 5] >> (y & 31)) & 1u) {
                        val[r] = map[y] * L + l;
                        cnt++;
                    }
                }
            }
            uint32_t off;
            const uint32_t total = eg_block_scan(cnt, &off, s_warp);
#pragma unroll
            for (int r = 0; r < 4; r++)
                if (val[r] != UNSET) {
                    const uint32_t pos = got + off++;
                    if (pos < want) dst[pos] = val[r];
                }
            got += total;
        }
        if (threadIdx.x == 0 && got != want) atomicExch(err, 1u);
    }
}

__device__ __forceinline__ uint32_t eg_get16(const uint32_t* w, uint32_t i) {
    return (w[i >> 1] >> ((i & 1) * 16)) & 0xFFFFu;
}
// decrements half i of w; returns its old value.  A half is only decremented
// while it is at least 1 (every decrement stands for a neighbour it counts),
// so no borrow reaches the other half.
__device__ __forceinline__ uint32_t eg_dec16(uint32_t* w, uint32_t i) {
    const uint32_t sh = (i & 1) * 16;
    return (atomicSub(w + (i >> 1), 1u << sh) >> sh) & 0xFFFFu;
}

// One block per column: the levels k0, k0+1, ... of the column's subgraph
// until no survivor is left (or the level cap, an error).
// Optional endgame trace (FC_PEEL_TRACE): per column and level, the level's
// start time (globaltimer ns), its rounds, the nodes it removed and the row
// entries it expanded.
// The cluster kernel adds, from its first block's first thread, the SM cycles
// of each level's phases: the scan round up to its cluster barrier, the
// rounds' row-offset loads and scans, their entry expansions, and their waits
// at the cluster barrier.
constexpr uint32_t EG_TRACE_LEVELS = 2048;
constexpr uint32_t EG_TR_W = 8;  // words per record
__device__ __forceinline__ unsigned long long* eg_tr(unsigned long long* tr, uint32_t c,
                                                     uint32_t lv) {
    return (tr && lv < EG_TRACE_LEVELS) ? tr + EG_TR_W * ((uint64_t)c * EG_TRACE_LEVELS + lv)
                                        : nullptr;
}

__global__ void __launch_bounds__(EG_THREADS) k_endgame(
    uint32_t cap, const uint32_t* __restrict__ ecnt, const uint32_t* __restrict__ rowptr,
    const uint64_t* __restrict__ base, const uint32_t* __restrict__ H,
    const uint32_t* __restrict__ l2g, const uint32_t* __restrict__ deg, uint32_t n, uint32_t L,
    FastDiv divL, uint32_t* __restrict__ t, uint32_t col0, uint32_t k0, uint32_t max_level,
    uint32_t* __restrict__ levels, uint32_t* __restrict__ err, unsigned long long* __restrict__ tr,
    uint32_t whole) {
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint32_t s_warp[33];
    __shared__ uint32_t s_nalive, s_next, s_tail;
    const uint32_t c = blockIdx.x;
    // whole: every column peels the whole graph from its first level -- the
    // graph's own rows, slots and initial degrees, local ids = node ids
    // (n = cap nodes); otherwise the column's compacted survivor subgraph
    const uint32_t m = whole ? cap : min(ecnt[c], cap);
    if (m == 0) return;
    const uint32_t lmd = col0 + c + 1;
    const uint32_t* rp = whole ? rowptr : rowptr + (uint64_t)c * (cap + 1);
    const uint32_t* Hc = whole ? H : H + base[c];
    const uint32_t* g_of = whole ? nullptr : l2g + (uint64_t)c * cap;
    uint32_t* tc = t + (uint64_t)c * n;
    // shared layout: degrees | counts | batch prefixes | batch row starts |
    // alive | lists | queue
    uint32_t* dw = sm;                                   // (m * L + 1) / 2 words
    uint32_t* cw = dw + ((uint64_t)m * L + 1) / 2;       // (m + 1) / 2 words
    uint32_t* pre = cw + (m + 1) / 2;                    // EG_THREADS words
    uint32_t* rs = pre + EG_THREADS;                     // EG_THREADS words
    uint8_t* alive = (uint8_t*)(rs + EG_THREADS);        // m bytes
    uint16_t* list0 = (uint16_t*)(((uintptr_t)(alive + m) + 3) & ~(uintptr_t)3);
    uint16_t* list1 = list0 + m;
    uint16_t* queue = list1 + m;
    for (uint32_t i = threadIdx.x; i < ((uint64_t)m * L + 1) / 2; i += blockDim.x) dw[i] = 0;
    for (uint32_t i = threadIdx.x; i < (m + 1) / 2; i += blockDim.x) cw[i] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < m * L; i += blockDim.x) {
        const uint32_t lid = i / L, l = i - lid * L;
        const uint32_t d = whole ? deg[(uint64_t)lid * L + l]
                                 : deg[(uint64_t)c * n * L + (uint64_t)g_of[lid] * L + l];
        atomicOr(dw + (i >> 1), (d & 0xFFFFu) << ((i & 1) * 16));
    }
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
        alive[i] = 1;
        list0[i] = (uint16_t)i;
    }
    if (threadIdx.x == 0) s_nalive = m;
    __syncthreads();
    uint16_t* cur = list0;
    uint16_t* nxt = list1;
    uint32_t k = k0;
    for (;;) {
        const uint32_t na = s_nalive;
        if (na == 0) break;
        if (k > max_level) {
            if (threadIdx.x == 0) atomicExch(err, 2u);
            break;
        }
        __syncthreads();
        unsigned long long* const trl = threadIdx.x == 0 ? eg_tr(tr, c, k - k0) : nullptr;
        unsigned long long tr_entries = 0, tr_rounds = 0;
        if (threadIdx.x == 0) {
            s_next = 0;
            s_tail = 0;
            if (trl) trl[0] = global_ns();
        }
        __syncthreads();
        // SCAN(k)
        for (uint32_t i = threadIdx.x; i < na; i += blockDim.x) {
            const uint32_t x = cur[i];
            if (!alive[x]) continue;
            uint32_t cnt = 0;
            for (uint32_t l = 0; l < L; l++) cnt += eg_get16(dw, x * L + l) >= k + 1;
            if (cnt < lmd) {
                alive[x] = 0;
                tc[whole ? x : g_of[x]] = k;
                queue[atomicAdd(&s_tail, 1u)] = (uint16_t)x;
            } else {
                atomicOr(cw + (x >> 1), cnt << ((x & 1) * 16));  // the half was 0
                nxt[atomicAdd(&s_next, 1u)] = (uint16_t)x;
            }
        }
        __syncthreads();
        // DRAIN(k): rounds over the queue, each round's rows flattened over
        // the block in batches of EG_THREADS items
        uint32_t qb = 0;
        for (uint32_t round = 0; round <= m; round++) {
            const uint32_t qe = s_tail;
            __syncthreads();
            if (qb >= qe) break;
            tr_rounds++;
            for (uint32_t b0 = qb; b0 < qe; b0 += EG_THREADS) {
                const uint32_t nb = min(EG_THREADS, qe - b0);
                uint32_t len = 0, start = 0;
                if (threadIdx.x < nb) {
                    const uint32_t x = queue[b0 + threadIdx.x];
                    start = rp[x];
                    len = rp[x + 1] - start;
                }
                uint32_t ex;
                const uint32_t total = eg_block_scan(len, &ex, s_warp);
                tr_entries += total;
                pre[threadIdx.x] = ex;
                rs[threadIdx.x] = start;
                __syncthreads();
                // four entries per thread at a time, their loads first
                uint32_t lo0 = 0;  // this thread's entries only move forward
                for (uint32_t e0 = threadIdx.x; e0 < total; e0 += 4 * blockDim.x) {
                    uint32_t slot[4];
#pragma unroll
                    for (int r = 0; r < 4; r++) {
                        const uint32_t e = e0 + r * blockDim.x;
                        slot[r] = UNSET;
                        if (e < total) {
                            uint32_t lo = lo0, hi = nb - 1;  // last item whose prefix is <= e
                            while (lo < hi) {
                                const uint32_t mid = (lo + hi + 1) >> 1;
                                if (pre[mid] <= e) lo = mid;
                                else hi = mid - 1;
                            }
                            lo0 = lo;
                            slot[r] = Hc[rs[lo] + (e - pre[lo])];
                        }
                    }
#pragma unroll
                    for (int r = 0; r < 4; r++) {
                        if (slot[r] == UNSET) continue;
                        const uint32_t u = divL.div(slot[r]);
                        if (u >= m || !alive[u]) continue;
                        const uint32_t old = eg_dec16(dw, slot[r]);
                        if (old == k + 1 && eg_dec16(cw, u) == lmd) {
                            alive[u] = 0;
                            tc[whole ? u : g_of[u]] = k;
                            queue[atomicAdd(&s_tail, 1u)] = (uint16_t)u;
                        }
                    }
                }
                __syncthreads();
            }
            qb = qe;
        }
        if (trl) {
            trl[1] = tr_rounds;
            trl[2] = s_tail;
            trl[3] = tr_entries;
        }
        // counts are rebuilt by the next SCAN: clear the kept ones
        for (uint32_t i = threadIdx.x; i < (m + 1) / 2; i += blockDim.x) cw[i] = 0;
        if (threadIdx.x == 0) s_nalive = s_next;
        uint16_t* tmp = cur;
        cur = nxt;
        nxt = tmp;
        k++;
        __syncthreads();
    }
    if (threadIdx.x == 0) levels[c] = k - k0;
}

// ---- the endgame on a thread-block cluster per column --------------------------
//
// The same levels as k_endgame, with a column's survivors spread over the CS
// blocks of one cluster (CS a power of two, at most 16): survivor i lives on
// block i % CS, at index i / CS of that block's degrees, count, alive flag
// and lists, and every block reaches the others' shared memory directly
// (distributed shared memory).  A level is a SCAN round, in which each block
// scans its own survivors, then DRAIN rounds: in each, every block expands
// the rows of its own nodes queued in the round before and its slice of
// every long row on block 0's list.  A removal its threads cause goes to
// that list when the node's row is long, else to one of the block's local
// halves, whose rows the block expands at once in further local iterations
// (separated by block barriers) until its threads cause no removal; only a
// removal that finds the local half full is queued on the removed node's
// owner for the next round.  Rounds are separated by cluster barriers.
// Block 0 holds, per round (three of them in rotation), the cluster-wide
// counts of nodes queued and of nodes a scan kept, and the long-row list;
// every block reads them right after the round's barrier, so all blocks take
// the same decisions.  The queue of round r+1 is the other half of a
// two-half queue, so a block never reads a slot another block may still be
// writing.  Every loop is bounded as in k_endgame, and no block leaves while
// another may still reach its shared memory.
constexpr uint32_t EGC_MAX = 16;
// The count half of a node that is not kept in the current level: decrements
// of a removed node's count (at most L, one per layer degree passing k + 1)
// leave it far above any lmd, and never borrow (L is at most 96 here: a
// block holds at least 1024 survivors at 2L + 11 shared bytes each, beside
// its fixed arrays; for larger L the cluster endgame is not used).
constexpr uint32_t EGC_DEAD = 0x8000u;
constexpr uint32_t EGC_DEAD2 = 0x80008000u;
// A kept node's count half is its count (bits 0-13) and, in bit 14, whether
// its row is long; a removed node's never matches lmd in bits 0-13.
constexpr uint32_t EGC_BIG = 0x4000u;
constexpr uint32_t EGC_CNT = 0x3FFFu;
// Long rows listed in one round, per cluster (more are expanded like short
// rows, by the block that found them removed or by their owners)
constexpr uint32_t EGC_BIG_MAX = 256;
// Capacity of each of a block's two local halves: rows found removed by the
// block's own threads, expanded by the block before the round ends
constexpr uint32_t EGC_LQ = 2048;
// set in block 0's count of a round by a block whose local iterations ran out
constexpr uint32_t EGC_FAIL = 0x80000000u;

// Block 0's counters of round rho + 1 (pushes, kept nodes) and its long-row
// list of round rho + 2 start empty; called at the start of round rho, when
// every block has read what they held three rounds before.
__device__ __forceinline__ void egc_reset(uint32_t* cnt, uint32_t* kept, uint32_t* bign,
                                          uint32_t rho) {
    cnt[(rho + 1) % 3] = 0;
    kept[(rho + 1) % 3] = 0;
    bign[(rho + 2) % 3] = 0;
}

// adds the calling threads of a warp to a (remote) counter with one atomic
__device__ __forceinline__ void egc_count(uint32_t* p) {
    const uint32_t am = __activemask();
    if ((threadIdx.x & 31) == (uint32_t)(__ffs(am) - 1)) atomicAdd(p, (uint32_t)__popc(am));
}

// Block-wide exclusive scan of 32 warps' values with one barrier: each warp
// scans the warp totals itself.  Two calls need a barrier between them.
__device__ __forceinline__ uint32_t egc_block_scan(uint32_t v, uint32_t* excl, uint32_t* s_warp) {
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t in = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, in, d);
        if (lane >= (uint32_t)d) in += t;
    }
    if (lane == 31) s_warp[w] = in;
    __syncthreads();
    const uint32_t x = s_warp[lane];
    uint32_t y = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, y, d);
        if (lane >= (uint32_t)d) y += t;
    }
    *excl = __shfl_sync(0xffffffffu, y - x, w) + in - v;
    return __shfl_sync(0xffffffffu, y, 31);
}

// appends column-local node u to block 0's list of long rows for a round
__device__ __forceinline__ bool egc_push_big(uint32_t* big, uint32_t* bign, uint32_t slot,
                                             uint32_t u) {
    const uint32_t pos = atomicAdd(bign + slot, 1u);
    if (pos >= EGC_BIG_MAX) return false;
    big[slot * EGC_BIG_MAX + pos] = u;
    return true;
}

__device__ __forceinline__ uint32_t egc_dec16(uint32_t* w, uint32_t i) {
    const uint32_t sh = (i & 1) * 16;
    return (atomicSub(w + (i >> 1), 1u << sh) >> sh) & 0xFFFFu;
}

// shared bytes per survivor a block owns: degrees (L halves), count (a half),
// alive flag, two lists and two queue halves (16-bit indices); besides them
// the batch prefixes and row starts and the two local halves
static uint32_t egc_node_bytes(uint32_t L) { return 2 * L + 11; }
static uint32_t egc_block_capacity(uint32_t L) {
    const uint64_t fixed = 8ull * EG_THREADS + 4ull * EGC_LQ + 256;
    uint64_t cap = (EG_SMEM - fixed) / egc_node_bytes(L);
    if (cap > 65535) cap = 65535;
    return cap >= 1024 ? (uint32_t)cap : 0u;
}
static uint64_t egc_smem_bytes(uint32_t mo, uint32_t L) {
    return 4ull * (((uint64_t)mo * L + 1) / 2 + (mo + 1) / 2 + 2ull * EG_THREADS) + mo + 4 +
           8ull * mo + 4ull * EGC_LQ + 16;
}

__global__ void __launch_bounds__(EG_THREADS) k_endgame_cl(
    uint32_t cap, const uint32_t* __restrict__ ecnt, const uint32_t* __restrict__ rowptr,
    const uint64_t* __restrict__ base, const uint32_t* __restrict__ H,
    const uint32_t* __restrict__ l2g, const uint32_t* __restrict__ deg, uint32_t n, uint32_t L,
    FastDiv divL, uint32_t* __restrict__ t, uint32_t col0, uint32_t k0, uint32_t max_level,
    uint32_t* __restrict__ levels, uint32_t* __restrict__ err, unsigned long long* __restrict__ tr,
    uint32_t split, uint32_t whole, uint32_t lq_cap) {
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint32_t s_warp[33];
    __shared__ uint32_t s_next, s_tail[2], s_lt[2];
    // FC_PEEL_TRACE counters of a level, kept by thread 0: entries, cluster
    // rounds, removals counted in block 0, local iterations, local removals,
    // the four phases' cycles, and three timestamps
    __shared__ unsigned long long s_tq[12];
    __shared__ uint32_t s_cnt[3], s_kept[3];  // block 0's are the cluster's
    __shared__ uint32_t s_big[3][EGC_BIG_MAX], s_bign[3];  // block 0's are the cluster's
    cg::cluster_group cl = cg::this_cluster();
    const uint32_t CS = cl.num_blocks();
    const uint32_t r = cl.block_rank();
    const uint32_t lg = 31 - __clz(CS);  // CS = 1 << lg
    const uint32_t c = blockIdx.x / CS;
    // whole: every column peels the whole graph from its first level (the
    // graph's own rows, slots and initial degrees; local ids = node ids)
    const uint32_t m = whole ? cap : min(ecnt[c], cap);
    if (m == 0) return;  // the whole cluster leaves, before any barrier
    const uint32_t lmd = col0 + c + 1;
    const uint32_t mo_max = (m + CS - 1) / CS;               // the same layout on every block
    const uint32_t mo = r < m ? (m - r + CS - 1) / CS : 0u;  // survivors r, r + CS, ...
    const uint32_t* rp = whole ? rowptr : rowptr + (uint64_t)c * (cap + 1);
    const uint32_t* Hc = whole ? H : H + base[c];
    const uint32_t* g_of = whole ? nullptr : l2g + (uint64_t)c * cap;
    uint32_t* tc = t + (uint64_t)c * n;
    uint32_t* dw = sm;                                       // (mo_max * L + 1) / 2 words
    uint32_t* cw = dw + ((uint64_t)mo_max * L + 1) / 2;      // (mo_max + 1) / 2 words
    uint32_t* pre = cw + (mo_max + 1) / 2;                   // EG_THREADS words
    uint32_t* rs = pre + EG_THREADS;                         // EG_THREADS words
    uint8_t* alive = (uint8_t*)(rs + EG_THREADS);            // mo_max bytes
    uint16_t* list0 = (uint16_t*)(((uintptr_t)(alive + mo_max) + 3) & ~(uintptr_t)3);
    uint16_t* list1 = list0 + mo_max;
    uint16_t* qh[2] = {list1 + mo_max, list1 + 2 * mo_max};  // the two queue halves
    uint16_t* lq[2] = {list1 + 3 * mo_max, list1 + 3 * mo_max + EGC_LQ};  // the local halves
    for (uint32_t i = threadIdx.x; i < ((uint64_t)mo_max * L + 1) / 2; i += blockDim.x) dw[i] = 0;
    for (uint32_t i = threadIdx.x; i < (mo_max + 1) / 2; i += blockDim.x) cw[i] = EGC_DEAD2;
    if (threadIdx.x < 3) {
        s_cnt[threadIdx.x] = 0;
        s_kept[threadIdx.x] = 0;
        s_bign[threadIdx.x] = 0;
    }
    if (threadIdx.x == 0) s_tail[0] = s_tail[1] = s_lt[0] = s_lt[1] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < mo * L; i += blockDim.x) {
        const uint32_t idx = i / L, l = i - idx * L;
        const uint32_t u = (idx << lg) + r;
        const uint32_t d = whole ? deg[(uint64_t)u * L + l]
                                 : deg[(uint64_t)c * n * L + (uint64_t)g_of[u] * L + l];
        atomicOr(dw + (i >> 1), (d & 0xFFFFu) << ((i & 1) * 16));
    }
    // alive: 1, or 2 for a node whose row is longer than split (expanded by
    // every block of the cluster, a slice each)
    for (uint32_t i = threadIdx.x; i < mo; i += blockDim.x) {
        const uint32_t u = (i << lg) + r;
        alive[i] = split && rp[u + 1] - rp[u] > split ? 2 : 1;
        list0[i] = (uint16_t)i;
    }
    uint32_t* const r0_cnt = cl.map_shared_rank(s_cnt, 0);
    uint32_t* const r0_kept = cl.map_shared_rank(s_kept, 0);
    uint32_t* const r0_big = cl.map_shared_rank(&s_big[0][0], 0);
    uint32_t* const r0_bign = cl.map_shared_rank(s_bign, 0);
    cl.sync();  // every block initialised before any reaches another
    uint16_t* cur = list0;
    uint16_t* nxt = list1;
    uint32_t na = mo, k = k0, rho = 0;
    bool failed = false;
    const bool tq = tr && threadIdx.x == 0;
    for (;;) {
        if (k > max_level) {  // k is the same on every block
            failed = true;
            break;
        }
        // SCAN round rho: removals queue locally in half (rho + 1) & 1
        const uint32_t qn = (rho + 1) & 1;
        if (tq) {
            for (int q = 0; q < 11; q++) s_tq[q] = 0;
            s_tq[11] = clock64();
            if (r == 0) {
                unsigned long long* const trl = eg_tr(tr, c, k - k0);
                if (trl) trl[0] = global_ns();
            }
        }
        if (threadIdx.x == 0) {
            s_next = 0;
            s_tail[0] = s_tail[1] = 0;  // no block queues remotely during a scan round
            if (r == 0) egc_reset(s_cnt, s_kept, s_bign, rho);
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < na; i += blockDim.x) {
            const uint32_t x = cur[i];
            const uint32_t ax = alive[x];
            if (!ax) continue;
            uint32_t cnt = 0;
            for (uint32_t l = 0; l < L; l++) cnt += eg_get16(dw, x * L + l) >= k + 1;
            if (cnt < lmd) {
                alive[x] = 0;
                tc[whole ? (x << lg) + r : g_of[(x << lg) + r]] = k;
                if (!(ax == 2 && egc_push_big(r0_big, r0_bign, (rho + 1) % 3, (x << lg) + r)))
                    qh[qn][atomicAdd(&s_tail[qn], 1u)] = (uint16_t)x;
                egc_count(r0_cnt + rho % 3);
            } else {
                // EGC_DEAD -> cnt, with the long-row flag
                const uint32_t v = cnt | (ax == 2 ? EGC_BIG : 0u);
                atomicSub(cw + (x >> 1), (EGC_DEAD - v) << ((x & 1) * 16));
                nxt[atomicAdd(&s_next, 1u)] = (uint16_t)x;
                egc_count(r0_kept + rho % 3);
            }
        }
        cl.sync();  // every block's counts are in block 0, every queue is final
        const uint32_t kept = r0_kept[rho % 3];
        const uint32_t scanned = r0_cnt[rho % 3];
        uint32_t nbig = min(r0_bign[(rho + 1) % 3], EGC_BIG_MAX);  // the next round's long rows
        if (tq) s_tq[5] = clock64() - s_tq[11];
        // with no survivor left in the column the rows of this scan's
        // removals name no node that could still change
        uint32_t pushes = kept ? scanned : 0u;
        if (tq) s_tq[2] = scanned;
        rho++;
        // DRAIN rounds while the last round queued anything for the cluster
        // (bounded: every node is queued at most once per level)
        for (uint32_t round = 0; pushes && round <= m; round++) {
            const uint32_t qc = rho & 1, qp = (rho + 1) & 1;
            const uint32_t* const bl = r0_big + (rho % 3) * EGC_BIG_MAX;
            if (threadIdx.x == 0 && r == 0) egc_reset(s_cnt, s_kept, s_bign, rho);
            if (tq) {
                s_tq[1]++;
                s_tq[9] = clock64();
            }
            // Local iterations: the first expands this block's queued rows and
            // its slice of every long row, each later one the rows that the
            // block's own threads found removed in the one before (of any
            // owner), until they find none.  A row found removed goes to the
            // cluster's list when it is long, else to the local half while it
            // has room, else to its owner's queue; the list and the queues are
            // expanded in the next round (block 0 holds their counts).
            uint32_t lcnt = 0;
            bool ldone = false;
            for (uint32_t li = 0; li <= m; li++) {
                const uint32_t hw = (li + 1) & 1;  // the local half this iteration fills
                const uint32_t qe = li ? lcnt : s_tail[qc];
                const uint32_t items = li ? lcnt : qe + nbig;
                const uint16_t* const lr = lq[li & 1];  // read by iterations >= 1
                if (tq) s_tq[3]++;
                for (uint32_t b0 = 0; b0 < items; b0 += EG_THREADS) {
                    if (b0) __syncthreads();  // the last batch's pre and rs are read
                    const uint32_t nb = min(EG_THREADS, items - b0);
                    uint32_t len = 0, start = 0;
                    const uint32_t it = b0 + threadIdx.x;
                    if (it < qe) {
                        const uint32_t lid =
                            li ? (uint32_t)lr[it] : ((uint32_t)qh[qc][it] << lg) + r;
                        start = rp[lid];
                        len = rp[lid + 1] - start;
                        tc[whole ? lid : g_of[lid]] = k;  // again for a scan removal: the same value
                    } else if (it < items) {
                        const uint32_t u = bl[it - qe];
                        const uint32_t s0 = rp[u], l0 = rp[u + 1] - s0;
                        const uint32_t e0 = (uint32_t)((uint64_t)l0 * r / CS);
                        start = s0 + e0;
                        len = (uint32_t)((uint64_t)l0 * (r + 1) / CS) - e0;
                        if ((u & (CS - 1)) == r) tc[whole ? u : g_of[u]] = k;  // its owner
                    }
                    uint32_t ex;
                    const uint32_t total = egc_block_scan(len, &ex, s_warp);
                    // every thread has read the half's length (before the
                    // scan's barrier): it takes a later iteration's (round's)
                    if (b0 == 0 && threadIdx.x == 0) {
                        if (li) s_lt[li & 1] = 0;
                        else s_tail[qc] = 0;
                    }
                    if (tq) s_tq[0] += total;
                    pre[threadIdx.x] = ex;
                    rs[threadIdx.x] = start;
                    __syncthreads();
                    if (tq) {
                        s_tq[10] = clock64();
                        s_tq[6] += s_tq[10] - s_tq[9];
                    }
                    uint32_t lo0 = 0;
                    for (uint32_t e0 = threadIdx.x; e0 < total; e0 += 4 * blockDim.x) {
                        uint32_t slot[4];
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            const uint32_t e = e0 + q * blockDim.x;
                            slot[q] = UNSET;
                            if (e < total) {
                                uint32_t lo = lo0, hi = nb - 1;
                                while (lo < hi) {
                                    const uint32_t mid = (lo + hi + 1) >> 1;
                                    if (pre[mid] <= e) lo = mid;
                                    else hi = mid - 1;
                                }
                                lo0 = lo;
                                slot[q] = Hc[rs[lo] + (e - pre[lo])];
                            }
                        }
                        // the degree decrements first, independent of one
                        // another; removed neighbours are decremented too (a
                        // half counts the alive neighbours, so it never drops
                        // below 0), and their count halves, EGC_DEAD less at
                        // most L crossings, never equal lmd
                        uint32_t ow[4], ui[4], old[4];
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            old[q] = 0;  // never k + 1
                            ow[q] = ui[q] = 0;
                            if (slot[q] == UNSET) continue;
                            const uint32_t u = divL.div(slot[q]);
                            if (u >= m) continue;
                            const uint32_t l = slot[q] - u * L;
                            ow[q] = u & (CS - 1);
                            ui[q] = u >> lg;
                            old[q] = egc_dec16(cl.map_shared_rank(dw, ow[q]), ui[q] * L + l);
                        }
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            if (old[q] != k + 1) continue;
                            const uint32_t oc = egc_dec16(cl.map_shared_rank(cw, ow[q]), ui[q]);
                            if ((oc & EGC_CNT) != lmd) continue;
                            // removed: its row is expanded by this block, by
                            // its owner or, when long, by every block (the
                            // table entry is written then)
                            cl.map_shared_rank(alive, ow[q])[ui[q]] = 0;
                            const uint32_t u2 = (ui[q] << lg) | ow[q];
                            // (the list's own count tells the cluster)
                            if ((oc & EGC_BIG) && egc_push_big(r0_big, r0_bign, (rho + 1) % 3, u2))
                                continue;
                            const uint32_t pos = lq_cap ? atomicAdd(&s_lt[hw], 1u) : 0u;
                            if (pos < lq_cap) {
                                lq[hw][pos] = (uint16_t)u2;
                            } else {
                                uint32_t* const t_ow = cl.map_shared_rank(s_tail, ow[q]);
                                const uint32_t p2 = atomicAdd(t_ow + qp, 1u);
                                cl.map_shared_rank(qh[qp], ow[q])[p2] = (uint16_t)ui[q];
                                egc_count(r0_cnt + rho % 3);
                            }
                        }
                    }
                    if (tq) {
                        s_tq[9] = clock64();
                        s_tq[7] += s_tq[9] - s_tq[10];
                    }
                }
                if (!lq_cap) {  // no local halves: the round ends here
                    ldone = true;
                    break;
                }
                __syncthreads();  // this iteration's local pushes are in place
                lcnt = min(s_lt[hw], lq_cap);
                if (lcnt == 0) {
                    ldone = true;
                    break;
                }
                if (tq) s_tq[4] += lcnt;
            }
            // (cannot happen: every node is found removed at most once a level)
            if (!ldone && threadIdx.x == 0) atomicOr(r0_cnt + rho % 3, EGC_FAIL);
            cl.sync();  // every push is counted in block 0 and queued
            const uint32_t cnt = r0_cnt[rho % 3];
            nbig = min(r0_bign[(rho + 1) % 3], EGC_BIG_MAX);
            pushes = (cnt & ~EGC_FAIL) + nbig;
            if (cnt & EGC_FAIL) {  // the same on every block
                pushes = 1;
                break;
            }
            if (tq) {
                s_tq[8] += clock64() - s_tq[9];
                s_tq[2] += pushes;
            }
            rho++;
        }
        if (pushes) {  // the round bound ended the level with rows unexpanded
            failed = true;  // (the cluster-wide count: every block breaks)
            break;
        }
        unsigned long long* const trl = tq ? eg_tr(tr, c, k - k0) : nullptr;
        if (trl) {
            if (r == 0) {
                trl[1] = s_tq[1] | s_tq[3] << 32;  // cluster rounds, block 0's iterations
                for (int q = 0; q < 4; q++) trl[4 + q] = s_tq[5 + q];
            }
            // every block's removals and rows
            atomicAdd(trl + 2, r == 0 ? s_tq[2] + s_tq[4] : s_tq[4]);
            atomicAdd(trl + 3, s_tq[0]);
        }
        // counts are rebuilt by the next scan: every half back to EGC_DEAD
        for (uint32_t i = threadIdx.x; i < (mo_max + 1) / 2; i += blockDim.x) cw[i] = EGC_DEAD2;
        na = s_next;
        uint16_t* tmp = cur;
        cur = nxt;
        nxt = tmp;
        k++;
        __syncthreads();
        if (kept == 0) break;  // the cluster-wide count: the same on every block
    }
    if (failed && r == 0 && threadIdx.x == 0) atomicExch(err, 2u);
    if (r == 0 && threadIdx.x == 0) levels[c] = k - k0;
    cl.sync();  // no block leaves while another may still reach its shared memory
}

static SegP make_seg(const PeelGraph& g, uint32_t col0, uint32_t ncols, uint32_t* table,
                     uint32_t* deg, uint32_t xbase) {
    SegP p{};
    p.xbase = xbase;
    p.n = g.n;
    p.L = g.L;
    p.col0 = col0;
    p.divL.init(g.L);
    p.divN.init(g.n);
    p.nL = (uint64_t)g.n * g.L;
    p.node_ptr = g.node_ptr;
    p.adj = g.adj;
    p.deg0 = g.deg0;
    p.deg = deg;
    p.t = table + (uint64_t)col0 * g.n;
    p.big_id = g.big_id;
    p.ptab = g.ptab;
    p.ncols = ncols;
    return p;
}

static int peel_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

// The endgame after a k_peel launch that stopped (see k_endgame): the
// survivors' subgraphs are built in buffers the peel no longer needs (its
// count array holds the local ids, the other alive list the local-to-global
// map, the node queues the row offsets and the chunk queues the entries, or
// a temporary buffer when they do not fit), then one block per column.
// Blocks per column in the endgame: FC_PEEL_EG_CLUSTER (1, 2, 4, 8 or 16;
// default 16), lowered until the device can run such a cluster of k_endgame_cl
// blocks with the largest shared memory they may take; 1 is the one-block
// k_endgame.  Decided once per device.
static uint32_t eg_cluster_size() {
    static int cached[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 1;
    if (cached[dev]) return (uint32_t)cached[dev];
    uint32_t want = env_u32("FC_PEEL_EG_CLUSTER", 16);
    uint32_t cs = 1;
    while (cs * 2 <= want && cs * 2 <= EGC_MAX) cs *= 2;
    if (cs > 1 &&
        (cudaFuncSetAttribute(k_endgame_cl, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)EG_SMEM) != cudaSuccess ||
         cudaFuncSetAttribute(k_endgame_cl, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
             cudaSuccess))
        cs = 1;
    for (; cs > 1; cs /= 2) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(cs);
        cfg.blockDim = dim3(EG_THREADS);
        cfg.dynamicSmemBytes = EG_SMEM;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, k_endgame_cl, &cfg) == cudaSuccess &&
            nclusters >= 1)
            break;
    }
    cudaGetLastError();
    cached[dev] = (int)cs;
    return cs;
}

// Rows longer than this are expanded by every block of the cluster, a slice
// each, in the round after their node's removal, instead of by one block:
// FC_PEEL_EG_SPLIT (entries; 0 = never).  2048 measured best with local
// iterations (shorter rows then cascade inside a block; longer ones would
// leave one block with the dense core's ~6,400-entry rows).
static uint32_t eg_split() {
    static const uint32_t v = env_u32("FC_PEEL_EG_SPLIT", 2048);
    return v;
}
// FC_PEEL_EG_LOCAL=0: every row found removed waits for the next cluster
// round (no local iterations)
static uint32_t eg_local_cap() {
    static const uint32_t v = env_u32("FC_PEEL_EG_LOCAL", 1) ? EGC_LQ : 0u;
    return v;
}

// survivors one column's endgame can hold with cs blocks (0: off for this L)
// FC_PEEL_EG_CAP lowers it (the endgame then starts later)
static uint32_t eg_column_capacity(uint32_t L, uint32_t cs) {
    // Degrees are 16-bit halves, and a survivor's degree in a layer is below
    // its column's survivor count: at most 65,536 survivors keep them exact.
    // (Where the endgame starts moves c3's peel stage by less than 1 %.)
    uint32_t cap = cs > 1 ? cs * egc_block_capacity(L) : eg_capacity(L);
    if (cap > 65536u) cap = 65536u;
    const uint32_t want = env_u32("FC_PEEL_EG_CAP", 0);
    return want && want < cap ? want : cap;
}

static fc_status endgame_run(const PeelJob& j, const PeelGraph& g, const PeelCtl& out, uint32_t col0,
                             uint32_t ncols, uint32_t cap, uint32_t cs, cudaStream_t s,
                             PeelStats* st, bool instrument) {
    const uint32_t K = out.level, ac = out.alive_cur & 1u;
    const uint32_t nalive = out.alive_cnt[ac];
    const uint32_t capE = cap < g.n ? cap : g.n;
    if (ncols > EG_MAX_COLS || (uint64_t)ncols * capE > j.nx ||
        (uint64_t)ncols * (capE + 1) > j.qs_cap)
        return FC_ERR_INVALID;
    PeelCtl* c = j.ctl;
    const uint32_t* alive = j.alive[ac];
    uint32_t* map = j.cnt;
    uint32_t* l2g = j.alive[ac ^ 1];
    uint32_t* rowlen = j.qs[1];
    uint32_t* rowptr = j.qs[0];
    const uint32_t* deg = j.seg0.deg;
    struct Events {  // destroyed on every return
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ~Events() {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } ev;
    if (instrument) {
        FC_CUDA_TRY(cudaEventCreate(&ev.e0));
        FC_CUDA_TRY(cudaEventCreate(&ev.e1));
        count_alloc(2);
        FC_CUDA_TRY(cudaEventRecord(ev.e0, s));
    }
    // FC_PEEL_TRACE: per-level records of the endgame kernels, printed after
    unsigned long long* etr = nullptr;
    struct TraceBuf {
        unsigned long long* p = nullptr;
        cudaStream_t s;
        ~TraceBuf() { dev_free(p, s); }
    } etr_own{nullptr, s};
    if (instrument && env_u32("FC_PEEL_TRACE", 0)) {
        const uint64_t bytes = 8ull * EG_TR_W * ncols * EG_TRACE_LEVELS;
        FC_TRY(dev_alloc((void**)&etr_own.p, bytes, s));
        FC_CUDA_TRY(cudaMemsetAsync(etr_own.p, 0, bytes, s));
        etr = etr_own.p;
    }
    FastDiv divN, divL;
    divN.init(g.n);
    divL.init(g.L);
    const int blocks = peel_sms() * 8;
    k_eg_index<<<blocks, 256, 0, s>>>(alive, nalive, j.bits, divN, g.n, g.L, deg, capE, map,
                                      c->eg_cnt, l2g, rowlen);
    FC_CUDA_TRY(cudaGetLastError());
    uint32_t cnts[EG_MAX_COLS], tots[EG_MAX_COLS];
    FC_TRY(to_host(cnts, c->eg_cnt, 4ull * ncols, s));
    uint32_t mmax = 0;
    for (uint32_t i = 0; i < ncols; i++) {
        if (cnts[i] > capE) return FC_ERR_DEVICE;  // more survivors than the stop rule allows
        mmax = cnts[i] > mmax ? cnts[i] : mmax;
    }
    k_eg_scan<<<ncols, EG_THREADS, 0, s>>>(rowlen, rowptr, capE, c->eg_cnt, c->eg_tot,
                                           &c->eg_nbig);
    FC_CUDA_TRY(cudaGetLastError());
    FC_TRY(to_host(tots, c->eg_tot, 4ull * ncols, s));
    uint64_t bases[EG_MAX_COLS], total = 0;
    for (uint32_t i = 0; i < ncols; i++) {
        bases[i] = total;
        total += tots[i];
    }
    uint32_t* H = (uint32_t*)j.qc[0];  // both parities' chunk queues: 4 * qc_cap words
    uint32_t* temp = nullptr;
    if (total > 4ull * j.qc_cap) {
        FC_TRY(dev_alloc((void**)&temp, total * 4 + 4, s));
        H = temp;
    }
    fc_status rc = to_device(c->eg_base, bases, 8ull * ncols, s);
    if (rc == FC_OK) {
        // the long rows' list takes the row lengths' buffer (spent after
        // k_eg_scan; its capacity exceeds the survivors)
        uint32_t* const big_list = rowlen;
        k_eg_fill<<<blocks, 256, 0, s>>>(alive, nalive, j.bits, divN, divL, g.n, g.L, g.node_ptr,
                                         g.adj, g.big_id, g.ptab, K + 1, map, capE, rowptr,
                                         c->eg_base, H, &c->eg_err, big_list, j.qs_cap,
                                         &c->eg_nbig);
        k_eg_fill_big<<<peel_sms() * 2, EG_THREADS, 0, s>>>(
            j.bits, divN, divL, g.n, g.L, g.node_ptr, g.adj, g.big_id, g.ptab, K + 1, map, capE, rowptr,
            c->eg_base, H, &c->eg_err, big_list, j.qs_cap, &c->eg_nbig);
        static const cudaError_t attr_rc = cudaFuncSetAttribute(
            k_endgame, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)EG_SMEM);
        if (cs > 1) {
            // a cluster of cs blocks per column (k_endgame_cl)
            const uint32_t mo = (mmax + cs - 1) / cs;
            const uint64_t smem = egc_smem_bytes(mo, g.L);
            if (smem > EG_SMEM || mo > 65535) {
                rc = FC_ERR_DEVICE;
            } else {
                cudaLaunchConfig_t cfg = {};
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeClusterDimension;
                at[0].val.clusterDim.x = cs;
                at[0].val.clusterDim.y = 1;
                at[0].val.clusterDim.z = 1;
                cfg.gridDim = dim3(ncols * cs);
                cfg.blockDim = dim3(EG_THREADS);
                cfg.dynamicSmemBytes = (size_t)smem;
                cfg.stream = s;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                const cudaError_t le = cudaLaunchKernelEx(
                    &cfg, k_endgame_cl, capE, (const uint32_t*)c->eg_cnt, (const uint32_t*)rowptr,
                    (const uint64_t*)c->eg_base, (const uint32_t*)H, (const uint32_t*)l2g, deg, g.n,
                    g.L, divL, j.seg0.t, col0, K + 1, j.max_level, c->eg_levels, &c->eg_err,
                    etr, eg_split(), 0u, eg_local_cap());
                count_launch(5);
                if (le != cudaSuccess) {
                    set_last_cuda_error(le, "k_endgame_cl", __FILE__, __LINE__);
                    rc = FC_ERR_DEVICE;
                }
            }
        } else {
        const uint64_t smem =
            4ull * (((uint64_t)mmax * g.L + 1) / 2 + (mmax + 1) / 2 + 2ull * EG_THREADS) + mmax + 4 +
            6ull * mmax + 16;
        if (attr_rc != cudaSuccess || smem > EG_SMEM) {
            rc = FC_ERR_DEVICE;
        } else {
            k_endgame<<<ncols, EG_THREADS, (size_t)smem, s>>>(
                capE, c->eg_cnt, rowptr, c->eg_base, H, l2g, deg, g.n, g.L, divL, j.seg0.t, col0,
                K + 1, j.max_level, c->eg_levels, &c->eg_err, etr, 0u);
            count_launch(5);
            const cudaError_t le = cudaGetLastError();
            if (le != cudaSuccess) {
                set_last_cuda_error(le, "k_endgame", __FILE__, __LINE__);
                rc = FC_ERR_DEVICE;
            }
        }
        }
    }
    uint32_t tail[EG_MAX_COLS + 1];  // eg_levels then eg_err
    if (rc == FC_OK) rc = to_host(tail, c->eg_levels, 4ull * (EG_MAX_COLS + 1), s);
    if (temp) dev_free(temp, s);
    if (instrument) {
        float ms = 0;
        cudaEventRecord(ev.e1, s);
        cudaEventSynchronize(ev.e1);
        cudaEventElapsedTime(&ms, ev.e0, ev.e1);
        if (st) st->ms += ms;
    }
    FC_TRY(rc);
    if (etr) {
        // one line per column and level: us, rounds, removals, row entries
        std::vector<unsigned long long> tr((uint64_t)EG_TR_W * ncols * EG_TRACE_LEVELS);
        FC_TRY(to_host(tr.data(), etr, tr.size() * 8, s));
        fprintf(stderr, "eg-trace start level %u, %u blocks per column, survivors", K + 1, cs);
        for (uint32_t i = 0; i < ncols; i++) fprintf(stderr, " %u", cnts[i]);
        uint32_t nbig = 0;
        FC_TRY(to_host(&nbig, &c->eg_nbig, 4, s));
        fprintf(stderr, ", entries %llu, rows filled by a block %u\n", (unsigned long long)total,
                nbig);
        for (uint32_t i = 0; i < ncols; i++)
            for (uint32_t lv = 0; lv + 1 < EG_TRACE_LEVELS; lv++) {
                const unsigned long long* r =
                    tr.data() + (uint64_t)EG_TR_W * (i * EG_TRACE_LEVELS + lv);
                if (!r[0]) break;
                const unsigned long long nx = r[EG_TR_W] ? r[EG_TR_W] : r[0];
                fprintf(stderr,
                        "eg-trace col %u level %u us %.1f rounds %llu local %llu items %llu"
                        " entries %llu cycles scan %llu rows %llu expand %llu sync %llu\n",
                        col0 + i, K + 1 + lv, (nx - r[0]) * 1e-3, r[1] & 0xFFFFFFFFull,
                        r[1] >> 32, r[2], r[3], r[4], r[5], r[6], r[7]);
            }
    }
    if (tail[EG_MAX_COLS]) return tail[EG_MAX_COLS] == 2 ? FC_ERR_ITER_LIMIT : FC_ERR_DEVICE;
    if (st) {
        uint32_t lv = 0;
        for (uint32_t i = 0; i < ncols; i++) lv = tail[i] > lv ? tail[i] : lv;
        st->levels += lv;
    }
    return FC_OK;
}

// A graph whose nodes fit one block's shared memory (or one cluster's, up to
// 65,536 nodes): every column peels the whole graph as the endgame from level
// 0, on the graph's own rows (no grid-wide levels, no compaction), one block
// (cluster) per column.
static uint32_t eg_whole_capacity(uint32_t L) {
    const uint64_t fixed = 8ull * EG_THREADS + 256;
    const uint64_t cap = (EG_SMEM - fixed) / eg_node_bytes(L);
    return cap > 65535 ? 65535u : (uint32_t)cap;
}

static fc_status whole_run(const PeelJob& j, const PeelGraph& g, uint32_t col0, uint32_t ncols,
                           uint32_t cs, cudaStream_t s, PeelStats* st, bool instrument) {
    const uint32_t n = g.n, L = g.L;
    const uint32_t mo = (n + cs - 1) / cs;
    const uint64_t smem =
        cs > 1 ? egc_smem_bytes(mo, L)
               : 4ull * (((uint64_t)n * L + 1) / 2 + (n + 1) / 2 + 2ull * EG_THREADS) + n + 4 +
                     6ull * n + 16;
    static const cudaError_t attr_rc = cudaFuncSetAttribute(
        k_endgame, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)EG_SMEM);
    if (attr_rc != cudaSuccess || smem > EG_SMEM || mo > 65535) return FC_ERR_DEVICE;
    struct Events {  // destroyed on every return
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ~Events() {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } ev;
    if (instrument) {
        FC_CUDA_TRY(cudaEventCreate(&ev.e0));
        FC_CUDA_TRY(cudaEventCreate(&ev.e1));
        count_alloc(2);
        FC_CUDA_TRY(cudaEventRecord(ev.e0, s));
    }
    // the levels of each column in the count array (nx >= ncols words)
    FC_CUDA_TRY(cudaMemsetAsync(&j.ctl->eg_err, 0, 4, s));
    FC_CUDA_TRY(cudaMemsetAsync(j.cnt, 0, 4ull * ncols, s));
    FastDiv divL;
    divL.init(L);
    cudaError_t le = cudaSuccess;
    if (cs > 1) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(ncols * cs);
        cfg.blockDim = dim3(EG_THREADS);
        cfg.dynamicSmemBytes = (size_t)smem;
        cfg.stream = s;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        le = cudaLaunchKernelEx(&cfg, k_endgame_cl, n, (const uint32_t*)nullptr, g.node_ptr,
                                (const uint64_t*)nullptr, g.adj, (const uint32_t*)nullptr,
                                g.deg0, n, L, divL, j.seg0.t, col0, 0u, j.max_level, j.cnt,
                                &j.ctl->eg_err, (unsigned long long*)nullptr, eg_split(), 1u,
                                eg_local_cap());
    } else {
        k_endgame<<<ncols, EG_THREADS, (size_t)smem, s>>>(
            n, nullptr, g.node_ptr, nullptr, g.adj, nullptr, g.deg0, n, L, divL, j.seg0.t, col0,
            0u, j.max_level, j.cnt, &j.ctl->eg_err, nullptr, 1u);
        le = cudaGetLastError();
    }
    count_launch();
    if (le != cudaSuccess) {
        set_last_cuda_error(le, "k_endgame", __FILE__, __LINE__);
        return FC_ERR_DEVICE;
    }
    std::vector<uint32_t> lv(ncols);
    uint32_t err = 0;
    FC_TRY(to_host(lv.data(), j.cnt, 4ull * ncols, s));
    FC_TRY(to_host(&err, &j.ctl->eg_err, 4, s));
    if (instrument) {
        float ms = 0;
        cudaEventRecord(ev.e1, s);
        cudaEventSynchronize(ev.e1);
        cudaEventElapsedTime(&ms, ev.e0, ev.e1);
        if (st) st->ms += ms;
    }
    if (err) return err == 2 ? FC_ERR_ITER_LIMIT : FC_ERR_DEVICE;
    if (st) {
        uint32_t m = 0;
        for (uint32_t x : lv) m = x > m ? x : m;
        st->levels += m;
    }
    return FC_OK;
}

fc_status peel_run(const PeelGraph& g, uint32_t col0, uint32_t ncols, uint32_t* table, void* ws,
                   size_t ws_bytes, cudaStream_t s, PeelStats* st, bool instrument, bool endgame) {
    const uint64_t nx = (uint64_t)ncols * g.n;
    if (peel_ws_bytes(g.n, g.L, g.entries, ncols) > ws_bytes) return FC_ERR_INVALID;
    PeelJob j{};
    char* w = (char*)ws;
    char* end = w + ws_bytes;
    uint32_t* deg = (uint32_t*)w;  // ncols * n * L at the start
    w += 4ull * ncols * g.n * g.L;
    // the chunk queues hold 8-byte items: start them on a 256-byte boundary
    w = (char*)(((uintptr_t)w + 255) & ~(uintptr_t)255);
    fc_status rc;
    carve_shared(j, w, end, nx, (uint64_t)ncols * g.entries, s, &rc);
    FC_TRY(rc);
    j.seg0 = make_seg(g, col0, ncols, table, deg, 0);
    j.segs = nullptr;
    j.seg_xbase = nullptr;
    j.nseg = 1;
    j.max_level = g.max_level;
    if (endgame && g.n && env_u32("FC_PEEL_ENDGAME", 1) && env_u32("FC_PEEL_WHOLE", 1)) {
        if (g.n <= eg_whole_capacity(g.L)) return whole_run(j, g, col0, ncols, 1, s, st, instrument);
        const uint32_t wcs = eg_cluster_size();
        if (wcs > 1 && g.n <= eg_column_capacity(g.L, wcs))
            return whole_run(j, g, col0, ncols, wcs, s, st, instrument);
    }
    const bool eg = endgame && ncols <= EG_MAX_COLS && env_u32("FC_PEEL_ENDGAME", 1);
    const uint32_t cs = eg ? eg_cluster_size() : 1u;
    const uint32_t cap = eg ? eg_column_capacity(g.L, cs) : 0u;
    j.stop_alive = cap;
    PeelCtl out;
    FC_TRY(run_job<false>(j, g.L, default_threads(), s, st, instrument, col0, ncols, nullptr, &out));
    if (!out.stopped) return FC_OK;
    return endgame_run(j, g, out, col0, ncols, cap, cs, s, st, instrument);
}

uint64_t peel_batch_ws_bytes(const std::vector<PeelSegSpec>& specs) {
    uint64_t nx = 0, ent = 0, deg = 0;
    for (const auto& sp : specs) {
        nx += (uint64_t)sp.ncols * sp.g.n;
        ent += (uint64_t)sp.ncols * sp.g.entries;
        deg += 4ull * sp.ncols * sp.g.n * sp.g.L;
    }
    const uint64_t nseg = specs.size();
    const uint64_t seg_bytes = (nseg * sizeof(SegP) + 4 * (nseg + 1) + 511) & ~511ull;
    return shared_ws_bytes(nx, ent) + deg + seg_bytes + 256;
}

fc_status peel_batch(const std::vector<PeelSegSpec>& specs, void* ws, size_t ws_bytes,
                     cudaStream_t s, PeelStats* st, uint32_t threads, uint32_t small_row,
                     bool* use_graph, uint32_t max_sms) {
    if (specs.empty()) return FC_OK;
    if (peel_batch_ws_bytes(specs) > ws_bytes) return FC_ERR_INVALID;
    char* w = (char*)ws;
    char* end = w + ws_bytes;
    // segment table and bases first (kept 256-byte aligned), then the degree
    // tables, then the shared lists
    const uint32_t nseg = (uint32_t)specs.size();
    std::vector<SegP> host(nseg);
    std::vector<uint32_t> xb(nseg + 1);
    uint64_t nx = 0, ent = 0;
    uint32_t maxL = 1, max_level = 1;
    SegP* dsegs = (SegP*)w;
    uint32_t* dxb = (uint32_t*)(w + nseg * sizeof(SegP));
    w += (nseg * sizeof(SegP) + 4 * (nseg + 1) + 511) & ~511ull;
    for (uint32_t i = 0; i < nseg; i++) {
        const PeelSegSpec& sp = specs[i];
        if (nx >= (1ull << 32)) return FC_ERR_TOO_LARGE;
        uint32_t* deg = (uint32_t*)w;
        w += 4ull * sp.ncols * sp.g.n * sp.g.L;
        host[i] = make_seg(sp.g, sp.col0, sp.ncols, sp.table, deg, (uint32_t)nx);
        xb[i] = (uint32_t)nx;
        nx += (uint64_t)sp.ncols * sp.g.n;
        ent += (uint64_t)sp.ncols * sp.g.entries;
        maxL = sp.g.L > maxL ? sp.g.L : maxL;
        max_level = sp.g.max_level > max_level ? sp.g.max_level : max_level;
    }
    if (nx >= (1ull << 32)) return FC_ERR_TOO_LARGE;
    xb[nseg] = (uint32_t)nx;
    w = (char*)(((uintptr_t)w + 255) & ~(uintptr_t)255);
    PeelJob j{};
    fc_status rc;
    carve_shared(j, w, end, nx, ent, s, &rc);
    FC_TRY(rc);
    FC_TRY(to_device(dsegs, host.data(), nseg * sizeof(SegP), s));
    FC_TRY(to_device(dxb, xb.data(), 4 * (nseg + 1), s));
    j.seg0 = host[0];
    j.segs = dsegs;
    j.seg_xbase = dxb;
    j.nseg = nseg;
    j.max_level = max_level;
    j.small_row = small_row;
    j.max_sms = max_sms;
    if (!threads) threads = default_threads();
    // the segment table must be on the device before a captured launch runs
    if (use_graph && *use_graph) FC_CUDA_TRY(cudaStreamSynchronize(s));
    if (nseg == 1) {
        j.segs = nullptr;
        return run_job<false>(j, maxL, threads, s, st, true, specs[0].col0, specs[0].ncols,
                              use_graph);
    }
    return run_job<true>(j, maxL, threads, s, st, true, 0, 0, use_graph);
}

void peel_preload() {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, k_peel<1, 512, false>);
    cudaFuncGetAttributes(&a, k_peel<1, 512, true>);
    cudaFuncGetAttributes(&a, k_peel<1, 1024, false>);
    cudaFuncGetAttributes(&a, k_peel<1, 1024, true>);
    cudaFuncGetAttributes(&a, k_peel<32, 512, false>);
    cudaFuncGetAttributes(&a, k_peel<32, 512, true>);
    cudaFuncGetAttributes(&a, k_peel<32, 1024, false>);
    cudaFuncGetAttributes(&a, k_peel<32, 1024, true>);
    cudaFuncGetAttributes(&a, k_eg_index);
    cudaFuncGetAttributes(&a, k_eg_scan);
    cudaFuncGetAttributes(&a, k_eg_fill);
    cudaFuncGetAttributes(&a, k_eg_fill_big);
    cudaFuncGetAttributes(&a, k_endgame);
    cudaGetLastError();
}

fc_status peel_columns(DeviceGraph* d, uint32_t col0, uint32_t ncols, cudaStream_t s,
                       PeelStats* st) {
    const uint64_t bytes = peel_ws_bytes(d->n, d->L, d->entries, ncols);
    FC_TRY(ensure_ws(d, bytes, s));
    PeelGraph g{d->n, d->L, d->entries, d->node_ptr, d->adj, d->deg0, d->max_deg + 1, d->big_id, d->ptab};
    return peel_run(g, col0, ncols, d->table, d->ws, d->ws_bytes, s, st, true, true);
}

}  // namespace fc
