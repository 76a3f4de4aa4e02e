// Every fcgrid cell as a prefix of one order per column, and many cells
// answered at once.
//
// The cells of one lambda column are nested: C_{k+1,lambda} is a subset of
// C_{k,lambda}.  So one order of the column's nodes by descending core_lambda
// holds every cell of the column as a prefix -- C_{k,lambda} is its first
// |C_{k,lambda}| nodes -- and the nodes a cell loses against the next one
// (core_lambda = k exactly) are one contiguous block of it.  That block is
// what the reference's memory-lean methods keep per cell as the difference to
// the parent cell (FCSyncMem::constructCoreSync, CoreParallel/
// FCSyncMem.cpp:10-54; FCPathMem::constructCore, Core/FCPathMem.cpp:9-59), so
// the order plus the cell sizes (n*L + sum over lambda of (kmax_lambda + 2)
// words) is the compact form of every cell at once.
//
// Layout (the "cell index"):
//   order[(lambda-1)*n + i]      column lambda's nodes, core descending, ids
//                                ascending within one core value
//   sizes[off[lambda-1] + k]     |C_{k,lambda}| for k = 0 .. kmax_lambda + 1
//                                (the last is 0)
// Built on the device from the resident table: per-column maxima and
// histograms, a reverse scan per column, and one stable radix sort of the
// keys (column, kmax - core) carrying the node ids.
//
// Batched queries (the query lists of -m CoreIndexTimeOnline / Offline,
// main.cpp:493-582; getResCore / getResCoreOffline, Util/CoreIndexTime.h:
// 8-59): either every cell's prefix of the index is gathered, or every
// cell's column is scanned for the nodes with core >= k, in ascending ids
// (count per tile, one scan, ordered write).  The scan form also answers the
// MLCD membership test of -m MLCDTime (checktime, Util/CheckMLCDTime.h:
// 9-42) on per-node coreness vectors.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "device.h"

namespace fc {

struct CellIndex {
    uint32_t* order = nullptr;     // L*n (device)
    std::vector<uint64_t> off;     // L+1 (host): column starts in sizes
    std::vector<uint32_t> sizes;   // host copy of the cell sizes
    bool valid = false;
};

void free_cell_index(DeviceGraph* d, cudaStream_t s) {
    CellIndex* c = (CellIndex*)d->cidx;
    if (!c) return;
    dev_free(c->order, s);
    delete c;
    d->cidx = nullptr;
}

void invalidate_cell_index(DeviceGraph* d) {
    CellIndex* c = (CellIndex*)d->cidx;
    if (c) c->valid = false;
}

// ---- kernels ------------------------------------------------------------------

// per-column maxima; grid.y = column
__global__ void k_ci_colmax(const uint32_t* __restrict__ table, uint32_t n,
                            uint32_t* __restrict__ kmax) {
    const uint32_t* col = table + (uint64_t)blockIdx.y * n;
    uint32_t m = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        m = max(m, col[v]);
    m = __reduce_max_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(kmax + blockIdx.y, m);
}

// per-column histogram of core values into sizes[off[col] + core];
// shared-memory bins when they fit
constexpr uint32_t CI_SH_BINS = 12288;
__global__ void k_ci_hist(const uint32_t* __restrict__ table, uint32_t n,
                          const uint64_t* __restrict__ off, uint32_t* __restrict__ sizes) {
    __shared__ uint32_t sh[CI_SH_BINS];
    const uint32_t col = blockIdx.y;
    const uint64_t base = off[col];
    const uint32_t bins = (uint32_t)(off[col + 1] - base);  // kmax + 2
    const bool use_sh = bins <= CI_SH_BINS;
    if (use_sh)
        for (uint32_t i = threadIdx.x; i < bins; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const uint32_t* c = table + (uint64_t)col * n;
    uint32_t* out = sizes + base;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t k = c[v];
        if (use_sh) atomicAdd(sh + k, 1u);
        else atomicAdd(out + k, 1u);
    }
    __syncthreads();
    if (use_sh)
        for (uint32_t i = threadIdx.x; i < bins; i += blockDim.x)
            if (sh[i]) atomicAdd(out + i, sh[i]);
}

// counts -> suffix sums, one 1024-thread block per column, top bin first:
// sizes[k] = sum of counts[j] for j >= k
__global__ void __launch_bounds__(1024) k_ci_suffix(const uint64_t* __restrict__ off,
                                                    uint32_t* __restrict__ sizes) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_carry;
    const uint64_t base = off[blockIdx.x];
    const uint32_t bins = (uint32_t)(off[blockIdx.x + 1] - base);
    uint32_t* s = sizes + base;
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    // tiles of 1024 bins from the top; within a tile, bin (top - t) for thread t
    for (uint32_t top = bins; top > 0; top = top > 1024 ? top - 1024 : 0) {
        const uint32_t t = threadIdx.x;
        const bool has = t < top;
        const uint32_t idx = has ? top - 1 - t : 0;
        uint32_t v = has ? s[idx] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (lane == 31) s_warp[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t y = s_warp[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t z = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= (uint32_t)o) y += z;
            }
            s_warp[lane] = y;  // inclusive over warps
        }
        __syncthreads();
        const uint32_t carry = s_carry;
        const uint32_t incl = x + (w ? s_warp[w - 1] : 0u) + carry;
        if (has) s[idx] = incl;
        __syncthreads();
        if (threadIdx.x == 1023) s_carry = incl;
        __syncthreads();
    }
}

// sort keys (column, kmax_all - core) and the node ids they carry
template <class K>
__global__ void k_ci_keys(const uint32_t* __restrict__ table, uint32_t n, uint32_t L,
                          uint32_t kmax_all, uint32_t kbits, K* __restrict__ keys,
                          uint32_t* __restrict__ ids) {
    const uint64_t total = (uint64_t)n * L;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t col = (uint32_t)(i / n), v = (uint32_t)(i - (uint64_t)col * n);
        keys[i] = ((K)col << kbits) | (K)(kmax_all - table[i]);
        ids[i] = v;
    }
}

// ---- batched queries ---------------------------------------------------------

// Node v answers query q of a core table: core_{col[q]+1}(v) >= k[q].
struct TablePred {
    const uint32_t* table;
    uint32_t n;
    const uint32_t* qk;
    const uint32_t* qcol;
    __device__ __forceinline__ bool operator()(uint32_t q, uint32_t v) const {
        return __ldg(table + (uint64_t)__ldg(qcol + q) * n + v) >= __ldg(qk + q);
    }
};

// Node v answers MLCD query q when at least need[q] of its P values are
// >= k[q] (checktime: the count must reach max(lmd, 1), since the reference
// tests it only after a match).
struct MlcdPred {
    const uint32_t* cores;
    uint32_t P;
    const uint32_t* qk;
    const uint32_t* qneed;
    __device__ __forceinline__ bool operator()(uint32_t q, uint32_t v) const {
        const uint32_t* r = cores + (uint64_t)v * P;
        const uint32_t k = __ldg(qk + q), need = __ldg(qneed + q);
        uint32_t c = 0;
        for (uint32_t p = 0; p < P && c < need; p++) c += __ldg(r + p) >= k;
        return c >= need;
    }
};

constexpr uint32_t Q_THREADS = 256;
constexpr uint32_t Q_TILE = 4096;  // nodes per (query, tile) block

// matches per (query, tile): cnt[q * ntiles + tile]
template <class P>
__global__ void __launch_bounds__(Q_THREADS) k_q_count(P pred, uint32_t n, uint32_t ntiles,
                                                       unsigned long long* __restrict__ cnt) {
    __shared__ uint32_t s_w[Q_THREADS / 32];
    const uint32_t q = blockIdx.y, tile = blockIdx.x;
    const uint32_t v0 = tile * Q_TILE, v1 = min(n, v0 + Q_TILE);
    uint32_t c = 0;
    for (uint32_t v = v0 + threadIdx.x; v < v1; v += Q_THREADS) c += pred(q, v) ? 1u : 0u;
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (uint32_t i = 0; i < Q_THREADS / 32; i++) t += s_w[i];
        cnt[(uint64_t)q * ntiles + tile] = t;
    }
}

// the matches of each (query, tile) in ascending ids at their scanned place
template <class P>
__global__ void __launch_bounds__(Q_THREADS) k_q_write(P pred, uint32_t n, uint32_t ntiles,
                                                       const unsigned long long* __restrict__ pos,
                                                       uint32_t* __restrict__ out, uint64_t cap) {
    __shared__ uint32_t s_w[Q_THREADS / 32];
    const uint32_t q = blockIdx.y, tile = blockIdx.x;
    const uint32_t v0 = tile * Q_TILE, v1 = min(n, v0 + Q_TILE);
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint64_t at = pos[(uint64_t)q * ntiles + tile];
    for (uint32_t b = v0; b < v1; b += Q_THREADS) {
        const uint32_t v = b + threadIdx.x;
        const bool hit = v < v1 && pred(q, v);
        const uint32_t m = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) s_w[w] = __popc(m);
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (uint32_t i = 0; i < Q_THREADS / 32; i++) {
            const uint32_t c = s_w[i];
            if (i < w) before += c;
            total += c;
        }
        if (hit) {
            const uint64_t o = at + before + __popc(m & ((1u << lane) - 1u));
            if (o < cap) out[o] = v;
        }
        at += total;
        __syncthreads();
    }
}

// offsets[q] = pos[q * ntiles], offsets[nq] = the total
__global__ void k_q_offsets(const unsigned long long* __restrict__ pos,
                            const unsigned long long* __restrict__ cnt, uint32_t nq,
                            uint32_t ntiles, unsigned long long* __restrict__ offsets) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < nq) offsets[q] = pos[(uint64_t)q * ntiles];
    if (q == nq) {
        const uint64_t last = (uint64_t)nq * ntiles - 1;
        offsets[nq] = nq ? pos[last] + cnt[last] : 0ull;
    }
}

// out[offsets[q] + i] = order[col[q] * n + i] for i < offsets[q+1] - offsets[q]
__global__ void k_q_gather(const uint32_t* __restrict__ order, uint32_t n,
                           const uint32_t* __restrict__ qcol,
                           const unsigned long long* __restrict__ offsets, uint32_t nq,
                           uint32_t* __restrict__ out, uint64_t cap) {
    const uint64_t total = offsets[nq];
    const uint64_t lim = total < cap ? total : cap;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < lim;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nq;  // offsets[lo] <= i < offsets[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (offsets[mid] <= i) lo = mid;
            else hi = mid;
        }
        out[i] = order[(uint64_t)qcol[lo] * n + (i - offsets[lo])];
    }
}

// ---- host ---------------------------------------------------------------------

static int sms() {
    int dev = 0, s = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev);
    return s > 0 ? s : 1;
}

// A device buffer freed on every return path (stream-ordered).
struct DevBuf {
    void* p = nullptr;
    cudaStream_t s;
    explicit DevBuf(cudaStream_t st) : s(st) {}
    ~DevBuf() { dev_free(p, s); }
    fc_status alloc(size_t bytes) { return dev_alloc(&p, bytes ? bytes : 16, s); }
    template <class T>
    T* as() const { return (T*)p; }
};

template <class K>
static fc_status sort_columns(const uint32_t* table, uint32_t n, uint32_t L, uint32_t kmax_all,
                              uint32_t kbits, uint32_t* order, cudaStream_t s) {
    const uint64_t total = (uint64_t)n * L;
    int cbits = 0;
    while ((1ull << cbits) < L) cbits++;
    DevBuf kin(s), kout(s), vin(s), tmp(s);
    FC_TRY(kin.alloc(total * sizeof(K)));
    FC_TRY(kout.alloc(total * sizeof(K)));
    FC_TRY(vin.alloc(total * 4));
    const int grid = std::max(1, std::min<int>(sms() * 8, (int)((total + 255) / 256)));
    k_ci_keys<K><<<grid, 256, 0, s>>>(table, n, L, kmax_all, kbits, kin.as<K>(), vin.as<uint32_t>());
    count_launch();
    FC_CUDA_TRY(cudaGetLastError());
    size_t tb = 0;
    const int end_bit = (int)kbits + cbits;
    FC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, kin.as<K>(), kout.as<K>(),
                                                vin.as<uint32_t>(), order, total, 0,
                                                std::max(end_bit, 1), s));
    FC_TRY(tmp.alloc(tb));
    FC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp.p, tb, kin.as<K>(), kout.as<K>(),
                                                vin.as<uint32_t>(), order, total, 0,
                                                std::max(end_bit, 1), s));
    count_launch();
    return FC_OK;
}

// The cell index of the resident table, built once per table.
static fc_status build_cell_index(fc_graph* g, cudaStream_t s) {
    FC_TRY(coreindex(g, nullptr, false, s));
    DeviceGraph* d = g->dev;
    d->home = s;
    CellIndex* c = (CellIndex*)d->cidx;
    if (c && c->valid) return FC_OK;
    if (!c) {
        c = new CellIndex();
        d->cidx = c;
    }
    const uint32_t n = d->n, L = d->L;
    // per-column maxima
    DevBuf kmx(s);
    FC_TRY(kmx.alloc((uint64_t)L * 4));
    FC_CUDA_TRY(cudaMemsetAsync(kmx.p, 0, (uint64_t)L * 4, s));
    dim3 mg(std::max(1u, std::min(64u, (n + 255) / 256)), L);
    k_ci_colmax<<<mg, 256, 0, s>>>(d->table, n, kmx.as<uint32_t>());
    count_launch();
    FC_CUDA_TRY(cudaGetLastError());
    std::vector<uint32_t> kmax(L);
    FC_TRY(to_host(kmax.data(), kmx.p, (uint64_t)L * 4, s));
    uint32_t kmax_all = 0;
    for (uint32_t l = 0; l < L; l++) {
        if (kmax[l] > d->max_deg) return FC_ERR_DEVICE;  // not a valid core table
        kmax_all = std::max(kmax_all, kmax[l]);
    }
    c->off.assign(L + 1, 0);
    for (uint32_t l = 0; l < L; l++) c->off[l + 1] = c->off[l] + kmax[l] + 2;
    const uint64_t nsizes = c->off[L];
    // sizes: histogram, then suffix sums
    DevBuf doff(s), dsz(s);
    FC_TRY(doff.alloc((L + 1) * 8ull));
    FC_TRY(dsz.alloc(nsizes * 4));
    FC_TRY(to_device(doff.p, c->off.data(), (L + 1) * 8ull, s));
    FC_CUDA_TRY(cudaMemsetAsync(dsz.p, 0, nsizes * 4, s));
    dim3 hg(std::max(1u, std::min(32u, (n + 255) / 256)), L);
    k_ci_hist<<<hg, 256, 0, s>>>(d->table, n, doff.as<uint64_t>(), dsz.as<uint32_t>());
    k_ci_suffix<<<L, 1024, 0, s>>>(doff.as<uint64_t>(), dsz.as<uint32_t>());
    count_launch(2);
    FC_CUDA_TRY(cudaGetLastError());
    // the order: one stable sort of (column, kmax_all - core)
    if (!c->order) FC_TRY(dev_alloc((void**)&c->order, (uint64_t)n * L * 4 + 4, s));
    uint32_t kbits = 0;
    while ((1ull << kbits) <= kmax_all) kbits++;
    int cbits = 0;
    while ((1ull << cbits) < L) cbits++;
    if (kbits + cbits <= 32)
        FC_TRY(sort_columns<uint32_t>(d->table, n, L, kmax_all, kbits, c->order, s));
    else
        FC_TRY(sort_columns<unsigned long long>(d->table, n, L, kmax_all, kbits, c->order, s));
    c->sizes.resize(nsizes);
    FC_TRY(to_host(c->sizes.data(), dsz.p, nsizes * 4, s));
    c->valid = true;
    return FC_OK;
}

fc_status cell_index(fc_graph* g, uint32_t* order, uint64_t* col_off, uint32_t* sizes,
                     uint64_t sizes_cap, uint64_t* sizes_count, cudaStream_t s) {
    FC_TRY(build_cell_index(g, s));
    DeviceGraph* d = g->dev;
    CellIndex* c = (CellIndex*)d->cidx;
    if (col_off) std::copy(c->off.begin(), c->off.end(), col_off);
    if (sizes_count) *sizes_count = c->off[d->L];
    if (sizes)
        std::copy(c->sizes.begin(), c->sizes.begin() + std::min<uint64_t>(sizes_cap, c->sizes.size()),
                  sizes);
    if (order && d->n) FC_TRY(to_host(order, c->order, (uint64_t)d->n * d->L * 4, s));
    d->home = nullptr;
    return FC_OK;
}

// Shared tail of the scan-form queries: count, scan, offsets, write, copy.
template <class P>
static fc_status scan_queries(const P& pred, uint32_t n, uint32_t nq, uint64_t* offsets,
                              uint32_t* nodes, uint64_t cap, cudaStream_t s) {
    const uint32_t ntiles = std::max(1u, (n + Q_TILE - 1) / Q_TILE);
    const uint64_t cells = (uint64_t)nq * ntiles;
    DevBuf cnt(s), pos(s), offs(s), tmp(s), out(s);
    FC_TRY(cnt.alloc(cells * 8));
    FC_TRY(pos.alloc(cells * 8));
    FC_TRY(offs.alloc((nq + 1) * 8ull));
    dim3 grid(ntiles, nq);
    k_q_count<P><<<grid, Q_THREADS, 0, s>>>(pred, n, ntiles, cnt.as<unsigned long long>());
    count_launch();
    FC_CUDA_TRY(cudaGetLastError());
    size_t tb = 0;
    FC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.as<unsigned long long>(),
                                              pos.as<unsigned long long>(), cells, s));
    FC_TRY(tmp.alloc(tb));
    FC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.as<unsigned long long>(),
                                              pos.as<unsigned long long>(), cells, s));
    k_q_offsets<<<(nq + 256) / 256, 256, 0, s>>>(pos.as<unsigned long long>(),
                                                 cnt.as<unsigned long long>(), nq, ntiles,
                                                 offs.as<unsigned long long>());
    count_launch(2);
    FC_CUDA_TRY(cudaGetLastError());
    std::vector<uint64_t> ho(nq + 1);
    FC_TRY(to_host(ho.data(), offs.p, (nq + 1) * 8ull, s));
    if (offsets) std::copy(ho.begin(), ho.end(), offsets);
    const uint64_t want = std::min<uint64_t>(ho[nq], cap);
    if (nodes && want) {
        FC_TRY(out.alloc(want * 4));
        k_q_write<P><<<grid, Q_THREADS, 0, s>>>(pred, n, ntiles, pos.as<unsigned long long>(),
                                                out.as<uint32_t>(), want);
        count_launch();
        FC_CUDA_TRY(cudaGetLastError());
        FC_TRY(to_host(nodes, out.p, want * 4, s));
    }
    return FC_OK;
}

fc_status cells_members(fc_graph* g, const uint32_t* ks, const uint32_t* lmds, uint32_t nq,
                        bool by_index, uint64_t* offsets, uint32_t* nodes, uint64_t cap,
                        cudaStream_t s) {
    for (uint32_t q = 0; q < nq; q++)
        if (lmds[q] < 1 || lmds[q] > g->L) return FC_ERR_INVALID;
    if (!nq) {
        if (offsets) offsets[0] = 0;
        return cuda_available() ? FC_OK : FC_ERR_NO_DEVICE;
    }
    if (by_index) FC_TRY(build_cell_index(g, s));
    else FC_TRY(coreindex(g, nullptr, false, s));
    DeviceGraph* d = g->dev;
    d->home = s;
    const uint32_t n = d->n;
    std::vector<uint32_t> qcol(nq);
    for (uint32_t q = 0; q < nq; q++) qcol[q] = lmds[q] - 1;
    DevBuf dq(s);
    FC_TRY(dq.alloc(nq * 8ull));
    uint32_t* d_k = dq.as<uint32_t>();
    uint32_t* d_col = d_k + nq;
    FC_TRY(to_device(d_k, ks, nq * 4ull, s));
    FC_TRY(to_device(d_col, qcol.data(), nq * 4ull, s));
    if (!by_index) {
        const TablePred pred{d->table, n, d_k, d_col};
        FC_TRY(scan_queries(pred, n, nq, offsets, nodes, cap, s));
        d->home = nullptr;
        return FC_OK;
    }
    // the index: each query's cell is a prefix of its column's order
    CellIndex* c = (CellIndex*)d->cidx;
    std::vector<uint64_t> ho(nq + 1, 0);
    for (uint32_t q = 0; q < nq; q++) {
        const uint64_t b = c->off[qcol[q]], e = c->off[qcol[q] + 1];
        const uint64_t len = ks[q] < e - b ? c->sizes[b + ks[q]] : 0;  // k > kmax + 1: empty
        ho[q + 1] = ho[q] + len;
    }
    if (offsets) std::copy(ho.begin(), ho.end(), offsets);
    const uint64_t want = std::min<uint64_t>(ho[nq], cap);
    if (nodes && want) {
        DevBuf doffs(s), out(s);
        FC_TRY(doffs.alloc((nq + 1) * 8ull));
        FC_TRY(out.alloc(want * 4));
        FC_TRY(to_device(doffs.p, ho.data(), (nq + 1) * 8ull, s));
        const int grid = std::max(1, std::min<int>(sms() * 8, (int)((want + 255) / 256)));
        k_q_gather<<<grid, 256, 0, s>>>(c->order, n, d_col, doffs.as<unsigned long long>(), nq,
                                        out.as<uint32_t>(), want);
        count_launch();
        FC_CUDA_TRY(cudaGetLastError());
        FC_TRY(to_host(nodes, out.p, want * 4, s));
    }
    d->home = nullptr;
    return FC_OK;
}

fc_status mlcd_query(const uint32_t* cores, uint32_t n, uint32_t P, const uint32_t* ks,
                     const uint32_t* lmds, uint32_t nq, uint64_t* offsets, uint32_t* nodes,
                     uint64_t cap, cudaStream_t s) {
    if (!n || !P || !nq) {
        if (offsets)
            for (uint32_t q = 0; q <= nq; q++) offsets[q] = 0;
        return FC_OK;
    }
    DevBuf dc(s), dq(s);
    FC_TRY(dc.alloc((uint64_t)n * P * 4));
    FC_TRY(dq.alloc(nq * 8ull));
    std::vector<uint32_t> need(nq);
    for (uint32_t q = 0; q < nq; q++) need[q] = lmds[q] ? lmds[q] : 1u;
    uint32_t* d_k = dq.as<uint32_t>();
    uint32_t* d_need = d_k + nq;
    FC_TRY(to_device(dc.p, cores, (uint64_t)n * P * 4, s));
    FC_TRY(to_device(d_k, ks, nq * 4ull, s));
    FC_TRY(to_device(d_need, need.data(), nq * 4ull, s));
    const MlcdPred pred{dc.as<uint32_t>(), P, d_k, d_need};
    return scan_queries(pred, n, nq, offsets, nodes, cap, s);
}

}  // namespace fc
