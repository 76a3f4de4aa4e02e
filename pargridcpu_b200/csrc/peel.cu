// The fcgrid peel: core_lambda(v) for a group of lambda columns of one graph,
// in one persistent cooperative kernel with the level loop inside.
//
// Per column lambda (all columns of the group advance together, level by
// level) the kernel runs the bucket peel of the reference's get_index2
// (CoreIndexParallel/CoreIndex.cpp:62-109) level-synchronously:
//
//   t[x]    x = (column, node).  While the node is alive, t is its exact
//           Top-lambda -- the lambda-th largest of its L layer degrees inside
//           the alive set; once removed, t is its core index.
//   level k: the frontier is every alive x with t[x] == k.  Removing x
//           decrements deg[u][l] for each alive neighbour slot (u,l); a
//           decrement that takes deg from exactly t[u] to t[u]-1 is the only
//           way Top-lambda can fall (the lazy trigger of CoreIndex.cpp:92), so
//           u is marked dirty; dirty nodes get Top-lambda recomputed, and
//           those now <= k join the next frontier of the same level.
//   The sub-round EXPAND -> RECOMPUTE repeats until the frontier is empty,
//   then the next level is the smallest t still alive.
//
// Phases are separated by a grid barrier whose last arriving block runs the
// small serial "leader" step (counter resets, level changes).  Every barrier
// wait is bounded: a block that waits longer than the timeout records an
// error and the kernel winds down; level and sub-round counts are bounded by
// n*columns and the largest degree.
#include <cooperative_groups.h>
#include <cooperative_groups/scan.h>

#include <cstdio>
#include <cstdlib>

#include "device.h"

namespace cg = cooperative_groups;

namespace fc {

enum : uint32_t { PH_EXPAND = 1, PH_RECOMPUTE = 2, PH_SCAN = 3, PH_DONE = 4 };
enum : uint32_t { ERR_NONE = 0, ERR_BARRIER = 1, ERR_LIMIT = 2 };

struct PeelCtl {
    uint32_t bar_count, bar_gen, err, phase;
    uint32_t level, front_cur, alive_cur, dirty_cnt;
    uint32_t front_cnt[2], chunk_cnt[2], alive_cnt[2];
    uint32_t next_min, levels, subrounds, pad;
    uint64_t t_last;      // globaltimer at the last barrier
    uint64_t ph_ns[4];    // time spent per phase kind (scan/init, expand, recompute)
};

// rows longer than SMALL_ROW entries are expanded as CHUNK-entry work items
constexpr uint32_t SMALL_ROW = 32;
constexpr uint32_t CHUNK = 128;

struct PeelJob {
    uint32_t n, L, col0, ncols;
    uint64_t nL;  // n * L
    FastDiv divL, divN;
    const uint32_t* node_ptr;
    const uint32_t* adj;
    const uint32_t* deg0;
    uint32_t* deg;       // ncols * n * L
    uint32_t* t;         // table + col0 * n: ncols * n
    uint32_t* alive[2];  // each ncols * n
    uint32_t* front[2];  // rows of at most SMALL_ROW entries
    uint64_t* chunks[2]; // (x | chunk << 32) items of longer rows
    uint32_t* dirty;
    uint32_t* dflag;     // ncols * n
    PeelCtl* ctl;
    uint32_t max_level;
    uint32_t max_subrounds;
    uint32_t upper_bits;  // bits of the largest layer degree
    uint64_t timeout_ns;
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
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// data written by other SMs during the kernel is read through L2 only
__device__ __forceinline__ uint32_t ld_l2(const uint32_t* p) { return __ldcg(p); }

// ---- leader step: phase transitions (one thread, all blocks parked) -------

__device__ void leader_step(volatile PeelCtl* c, const PeelJob& j) {
    auto end_level = [&]() {
        if (c->next_min == 0xFFFFFFFFu) {
            c->phase = PH_DONE;
            return;
        }
        c->level = c->next_min;
        c->next_min = 0xFFFFFFFFu;
        c->alive_cnt[c->alive_cur ^ 1] = 0;
        c->levels++;
        c->phase = PH_SCAN;
        if (c->level > j.max_level) {
            c->err = ERR_LIMIT;
            c->phase = PH_DONE;
        }
    };
    {
        uint64_t now = global_ns();
        uint32_t kind = c->phase == PH_EXPAND ? 1 : (c->phase == PH_RECOMPUTE ? 2 : 0);
        if (c->t_last) c->ph_ns[kind] += now - c->t_last;
        c->t_last = now;
    }
    switch (c->phase) {
        case PH_SCAN:  // also the state after INIT
            c->alive_cur ^= 1;
            if (c->front_cnt[c->front_cur] + c->chunk_cnt[c->front_cur] > 0) {
                c->phase = PH_EXPAND;
                c->dirty_cnt = 0;
            } else {
                end_level();
            }
            break;
        case PH_EXPAND:
            c->phase = PH_RECOMPUTE;
            c->front_cnt[c->front_cur ^ 1] = 0;
            c->chunk_cnt[c->front_cur ^ 1] = 0;
            break;
        case PH_RECOMPUTE:
            c->dirty_cnt = 0;
            c->front_cur ^= 1;
            c->subrounds++;
            if (c->subrounds > j.max_subrounds) {
                c->err = ERR_LIMIT;
                c->phase = PH_DONE;
            } else if (c->front_cnt[c->front_cur] + c->chunk_cnt[c->front_cur] > 0) {
                c->phase = PH_EXPAND;
            } else {
                end_level();
            }
            break;
        default:
            c->phase = PH_DONE;
    }
    if (c->err) c->phase = PH_DONE;
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
            c->bar_count = 0;
            __threadfence();
            leader_step(c, j);
            __threadfence();
            st_release(&c->bar_gen, gen + 1);
        } else {
            uint64_t t0 = global_ns();
            uint32_t ns = 32;
            while (ld_acquire(&c->bar_gen) == gen) {
                __nanosleep(ns);
                if (ns < 512) ns <<= 1;
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

// ---- warp helpers -----------------------------------------------------------

// Append `val` to list/counter from the lanes that call it together.
__device__ __forceinline__ void push(uint32_t* list, uint32_t* cnt, uint32_t val) {
    cg::coalesced_group g = cg::coalesced_threads();
    uint32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(cnt, g.size());
    base = g.shfl(base, 0);
    list[base + g.thread_rank()] = val;
}

// Lambda-th largest of L values v[0..L) by a group of G lanes (G a power of
// two; all 32 lanes of the warp call this together, each group with its own
// row and lambda).  Radix select from bit `bits-1` down: the answer is the
// largest x with #{v >= x} >= lambda.  `bits` must be warp-uniform and cover
// the answer.  Rows with lmd == 0 are idle lanes (result unused).
template <int G>
__device__ __forceinline__ uint32_t group_topl(const uint32_t* row, uint32_t L, uint32_t lmd,
                                               uint32_t bits, bool live_row, bool l2) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t gl = lane & (G - 1);
    constexpr int MAXV = 16;
    uint32_t vals[MAXV];
    const uint32_t nv = (L + G - 1) / G;
    const bool inreg = nv <= MAXV;
    if (inreg) {
#pragma unroll
        for (int i = 0; i < MAXV; i++) {
            uint32_t li = gl + (uint32_t)i * G;
            vals[i] = (live_row && (uint32_t)i < nv && li < L) ? (l2 ? ld_l2(row + li) : row[li]) : 0u;
        }
    }
    uint32_t res = 0;
    for (int b = (int)bits - 1; b >= 0; b--) {
        uint32_t cand = res | (1u << b);
        uint32_t cnt = 0;
        if (inreg) {
#pragma unroll
            for (int i = 0; i < MAXV; i++) cnt += vals[i] >= cand;
        } else if (live_row) {
            for (uint32_t li = gl; li < L; li += G) cnt += (l2 ? ld_l2(row + li) : row[li]) >= cand;
        }
#pragma unroll
        for (int off = G / 2; off >= 1; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
        if (cnt >= lmd) res = cand;
    }
    return res;
}

__device__ __forceinline__ uint32_t row_len(const PeelJob& j, uint32_t v) {
    return __ldg(j.node_ptr + v + 1) - __ldg(j.node_ptr + v);
}

// A removed node joins the next expansion: short rows as one item, longer
// rows as ceil(len / CHUNK) chunk items so that no warp walks a long row alone.
__device__ __forceinline__ void push_frontier(const PeelJob& j, uint32_t f, uint32_t x) {
    uint32_t v = x - j.divN.div(x) * j.n;
    uint32_t len = row_len(j, v);
    if (len <= SMALL_ROW) {
        push(j.front[f], &j.ctl->front_cnt[f], x);
        return;
    }
    uint32_t nch = (len + CHUNK - 1) / CHUNK;
    cg::coalesced_group g = cg::coalesced_threads();
    uint32_t incl = cg::inclusive_scan(g, nch);
    uint32_t base = 0;
    if (g.thread_rank() == g.size() - 1) base = atomicAdd(&j.ctl->chunk_cnt[f], incl);
    base = g.shfl(base, g.size() - 1);
    uint64_t* out = j.chunks[f] + base + (incl - nch);
    for (uint32_t c = 0; c < nch; c++) out[c] = (uint64_t)x | ((uint64_t)c << 32);
}

// Up to four removed-neighbour slots per lane at once (loads first, then the
// atomics), so each lane keeps several memory operations in flight: decrement
// deg[u][l] and mark u dirty when the decrement took it from exactly t[u].
__device__ __forceinline__ void visit4(const PeelJob& j, const uint32_t (&col)[4],
                                       const uint32_t (&slot)[4], const bool (&ok)[4], uint32_t k) {
    uint32_t y[4], tu[4], old[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        y[i] = col[i] * j.n + j.divL.div(slot[i]);
        tu[i] = ok[i] ? ld_l2(j.t + y[i]) : 0u;
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
        old[i] = (ok[i] && tu[i] > k) ? atomicSub(j.deg + (uint64_t)col[i] * j.nL + slot[i], 1u) : 0u;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if (ok[i] && tu[i] > k && old[i] == tu[i]) {
            if (atomicExch(j.dflag + y[i], 1u) == 0u) push(j.dirty, &j.ctl->dirty_cnt, y[i]);
        }
    }
}

// Block-wide minimum into *dst (one atomic per block).
__device__ __forceinline__ void block_min_to(uint32_t v, uint32_t* dst) {
    __shared__ uint32_t smin;
    if (threadIdx.x == 0) smin = 0xFFFFFFFFu;
    __syncthreads();
    v = __reduce_min_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0 && v != 0xFFFFFFFFu) atomicMin(&smin, v);
    __syncthreads();
    if (threadIdx.x == 0 && smin != 0xFFFFFFFFu) atomicMin(dst, smin);
}

// ---- phases ---------------------------------------------------------------

template <int G>
__device__ void phase_init(const PeelJob& j) {
    // degree tables: every column starts from the full degrees
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < j.nL; i += stride) {
        const uint32_t d0 = __ldg(j.deg0 + i);
        for (uint32_t c = 0; c < j.ncols; c++) j.deg[(uint64_t)c * j.nL + i] = d0;
    }
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < (uint64_t)j.ncols * j.n;
         i += stride)
        j.dflag[i] = 0;
    // Top-lambda of every (column, node); level 0 split into frontier / alive
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t per_warp = 32 / G;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nx = j.ncols * j.n;
    uint32_t lmin = 0xFFFFFFFFu;
    for (uint32_t base = gw * per_warp; base < nx; base += nw * per_warp) {
        uint32_t x = base + lane / G;
        bool live = x < nx;
        uint32_t c = live ? j.divN.div(x) : 0;
        uint32_t v = x - c * j.n;
        uint32_t lmd = j.col0 + c + 1;
        uint32_t tv = group_topl<G>(j.deg0 + (uint64_t)v * j.L, j.L, live ? lmd : 0, j.upper_bits,
                                    live, false);
        if (live && (lane & (G - 1)) == 0) {
            j.t[x] = tv;
            if (tv == 0) push_frontier(j, 0, x);
            else {
                push(j.alive[1], &j.ctl->alive_cnt[1], x);
                lmin = min(lmin, tv);
            }
        }
    }
    block_min_to(lmin, &j.ctl->next_min);
}

__device__ void phase_expand(const PeelJob& j) {
    const PeelCtl* c = j.ctl;
    const uint32_t f = ld_l2(&c->front_cur);
    const uint32_t fsize = ld_l2(&c->front_cnt[f]);
    const uint32_t csize = ld_l2(&c->chunk_cnt[f]);
    const uint32_t k = ld_l2(&c->level);
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t* F = j.front[f];
    // long rows: CHUNK-entry items, one per warp, four slots per lane
    for (uint32_t ci = gw; ci < csize; ci += nw) {
        const uint64_t it = __ldcg(reinterpret_cast<const unsigned long long*>(j.chunks[f]) + ci);
        const uint32_t x = (uint32_t)it, ch = (uint32_t)(it >> 32);
        const uint32_t col = j.divN.div(x);
        const uint32_t v = x - col * j.n;
        const uint32_t b = __ldg(j.node_ptr + v) + ch * CHUNK;
        const uint32_t e = min(__ldg(j.node_ptr + v + 1), b + CHUNK);
        for (uint32_t q0 = b; q0 < e; q0 += 128) {
            uint32_t cols[4], slot[4];
            bool ok[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                uint32_t q = q0 + lane + 32 * i;
                ok[i] = q < e;
                slot[i] = ok[i] ? __ldg(j.adj + q) : 0u;
                cols[i] = col;
            }
            visit4(j, cols, slot, ok, k);
        }
    }
    // short rows: 32 frontier nodes per warp, their adjacency (at most 1024
    // entries) flattened over the lanes; the owner of entry q is found by
    // binary search over the warp's exclusive scan of row lengths
    for (uint32_t base = gw * 32; base < fsize; base += nw * 32) {
        uint32_t i = base + lane;
        uint32_t x = i < fsize ? ld_l2(F + i) : 0;
        uint32_t col = j.divN.div(x);
        uint32_t v = x - col * j.n;
        uint32_t b = 0, len = 0;
        if (i < fsize) {
            b = __ldg(j.node_ptr + v);
            len = __ldg(j.node_ptr + v + 1) - b;
        }
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += y;
        }
        uint32_t excl = incl - len;
        uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        for (uint32_t jb = 0; jb < total; jb += 128) {
            uint32_t cols[4], slot[4];
            bool ok[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t q = jb + 32 * i + lane;
                uint32_t own = 0;
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    uint32_t cand = own + step;
                    uint32_t ex = __shfl_sync(0xffffffffu, excl, cand & 31);
                    if (cand < 32 && ex <= q) own = cand;
                }
                const uint32_t ob = __shfl_sync(0xffffffffu, b, own);
                const uint32_t oe = __shfl_sync(0xffffffffu, excl, own);
                cols[i] = __shfl_sync(0xffffffffu, col, own);
                ok[i] = q < total;
                slot[i] = ok[i] ? __ldg(j.adj + ob + (q - oe)) : 0u;
            }
            visit4(j, cols, slot, ok, k);
        }
    }
}

template <int G>
__device__ void phase_recompute(const PeelJob& j) {
    const PeelCtl* c = j.ctl;
    const uint32_t dsize = ld_l2(&c->dirty_cnt);
    const uint32_t k = ld_l2(&c->level);
    const uint32_t fout = ld_l2(&c->front_cur) ^ 1;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t per_warp = 32 / G;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    uint32_t lmin = 0xFFFFFFFFu;
    for (uint32_t base = gw * per_warp; base < dsize; base += nw * per_warp) {
        uint32_t idx = base + lane / G;
        bool live = idx < dsize;
        uint32_t y = live ? ld_l2(j.dirty + idx) : 0;
        uint32_t col = j.divN.div(y);
        uint32_t u = y - col * j.n;
        uint32_t upper = live ? ld_l2(j.t + y) : 0;
        uint32_t bits = upper ? 32 - __clz(upper) : 0;
        bits = __reduce_max_sync(0xffffffffu, bits);
        uint32_t nt = group_topl<G>(j.deg + (uint64_t)col * j.nL + (uint64_t)u * j.L, j.L,
                                    live ? j.col0 + col + 1 : 0, bits, live, true);
        if (live && (lane & (G - 1)) == 0) {
            j.dflag[y] = 0;
            if (nt <= k) {
                j.t[y] = k;
                push_frontier(j, fout, y);
            } else {
                j.t[y] = nt;
                lmin = min(lmin, nt);
            }
        }
    }
    block_min_to(lmin, &j.ctl->next_min);
}

__device__ void phase_scan(const PeelJob& j) {
    const PeelCtl* c = j.ctl;
    const uint32_t a = ld_l2(&c->alive_cur);
    const uint32_t asize = ld_l2(&c->alive_cnt[a]);
    const uint32_t k = ld_l2(&c->level);
    const uint32_t f = ld_l2(&c->front_cur);
    const uint32_t* A = j.alive[a];
    uint32_t* out = j.alive[a ^ 1];
    uint32_t lmin = 0xFFFFFFFFu;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < asize; i += gridDim.x * blockDim.x) {
        uint32_t x = ld_l2(A + i);
        uint32_t tx = ld_l2(j.t + x);
        if (tx == k) push_frontier(j, f, x);
        else if (tx > k) {
            push(out, &j.ctl->alive_cnt[a ^ 1], x);
            lmin = min(lmin, tx);
        }
    }
    block_min_to(lmin, &j.ctl->next_min);
}

template <int G>
__global__ void __launch_bounds__(512) k_peel(PeelJob j) {
    phase_init<G>(j);
    if (!grid_barrier(j)) return;
    for (;;) {
        const uint32_t ph = ld_l2(&j.ctl->phase);
        if (ph == PH_EXPAND) phase_expand(j);
        else if (ph == PH_RECOMPUTE) phase_recompute<G>(j);
        else if (ph == PH_SCAN) phase_scan(j);
        else return;
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
    // group's working set within a budget (FC_PEEL_GROUP_BYTES, default 4 GiB)
    uint64_t per_col = ((uint64_t)d->n * d->L + 8ull * d->n) * 4;
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

template <int G>
static fc_status launch(PeelJob& j, cudaStream_t s) {
    int dev = 0, sms = 0, occ = 0;
    FC_CUDA_TRY(cudaGetDevice(&dev));
    FC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int threads = 512;
    FC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_peel<G>, threads, 0));
    if (occ < 1) return FC_ERR_DEVICE;
    uint32_t want_occ = env_u32("FC_PEEL_BLOCKS_PER_SM", 2);
    if ((int)want_occ < occ) occ = (int)want_occ;
    dim3 grid(sms * occ), block(threads);
    void* args[] = {&j};
    FC_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_peel<G>, grid, block, args, 0, s));
    return FC_OK;
}

fc_status peel_columns(DeviceGraph* d, uint32_t col0, uint32_t ncols, cudaStream_t s,
                       PeelStats* st) {
    const uint32_t n = d->n, L = d->L;
    const uint64_t nx = (uint64_t)ncols * n;
    const uint64_t nL = (uint64_t)n * L;
    // workspace: chunk0 chunk1 (uint64) | deg | alive0 alive1 front0 front1
    // dirty dflag | ctl.  A sub-round's chunk items number at most one per
    // removed node plus entries / CHUNK per column.
    const uint64_t nchunk = nx + ((uint64_t)ncols * d->entries + CHUNK - 1) / CHUNK + 1;
    size_t words = 4 * nchunk + (size_t)(ncols * nL) + 6 * nx + 256;
    FC_TRY(ensure_ws(d, words * 4));
    uint32_t* w = (uint32_t*)d->ws;
    PeelJob j;
    j.chunks[0] = (uint64_t*)w;
    w += 2 * nchunk;
    j.chunks[1] = (uint64_t*)w;
    w += 2 * nchunk;
    j.n = n;
    j.L = L;
    j.col0 = col0;
    j.ncols = ncols;
    j.nL = nL;
    j.divL.init(L);
    j.divN.init(n);
    j.node_ptr = d->node_ptr;
    j.adj = d->adj;
    j.deg0 = d->deg0;
    j.deg = w;
    w += ncols * nL;
    j.t = d->table + (uint64_t)col0 * n;
    j.alive[0] = w; w += nx;
    j.alive[1] = w; w += nx;
    j.front[0] = w; w += nx;
    j.front[1] = w; w += nx;
    j.dirty = w; w += nx;
    j.dflag = w; w += nx;
    j.ctl = (PeelCtl*)(((uintptr_t)w + 255) & ~(uintptr_t)255);
    j.max_level = d->max_deg + 1;
    j.max_subrounds = (uint32_t)std::min<uint64_t>(0xFFFFFFF0ull, nx + d->max_deg + 16);
    uint32_t bits = 0;
    while (bits < 32 && (d->max_deg >> bits)) bits++;
    j.upper_bits = bits;
    j.timeout_ns = (uint64_t)env_u32("FC_BARRIER_TIMEOUT_MS", 4000) * 1000000ull;
    PeelCtl init{};
    init.phase = PH_SCAN;  // INIT behaves as a scan into alive[1]
    init.alive_cur = 0;
    init.next_min = 0xFFFFFFFFu;
    FC_CUDA_TRY(cudaMemcpyAsync(j.ctl, &init, sizeof(init), cudaMemcpyHostToDevice, s));
    cudaEvent_t e0, e1;
    FC_CUDA_TRY(cudaEventCreate(&e0));
    FC_CUDA_TRY(cudaEventCreate(&e1));
    FC_CUDA_TRY(cudaEventRecord(e0, s));
    fc_status rc;
    if (L <= 1) rc = launch<1>(j, s);
    else if (L <= 2) rc = launch<2>(j, s);
    else if (L <= 4) rc = launch<4>(j, s);
    else if (L <= 8) rc = launch<8>(j, s);
    else if (L <= 16) rc = launch<16>(j, s);
    else rc = launch<32>(j, s);
    FC_TRY(rc);
    count_launch();
    FC_CUDA_TRY(cudaEventRecord(e1, s));
    PeelCtl out{};
    FC_CUDA_TRY(cudaMemcpyAsync(&out, j.ctl, sizeof(out), cudaMemcpyDeviceToHost, s));
    FC_CUDA_TRY(cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) {
        st->ms = ms;
        st->levels = out.levels;
        st->subrounds = out.subrounds;
        st->err = out.err;
        for (int i = 0; i < 3; i++) st->phase_ms[i] = out.ph_ns[i] * 1e-6;
    }
    if (out.err) return FC_ERR_ITER_LIMIT;
    return FC_OK;
}

}  // namespace fc
