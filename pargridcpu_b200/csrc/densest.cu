// Densest-subgraph search over every non-empty fcgrid cell, from the core
// table, in one pass over the edges per group of lambda columns.
//
// A directed entry (v -> u, layer l) lies inside C_{k,lambda} iff
// min(core_lambda(v), core_lambda(u)) >= k.  So one histogram per lambda,
//     H[lambda][l][key] = #{entries (v,u,l) : min(core_lambda(v), core_lambda(u)) = key},
// gives by suffix sums over key every cell's
//     e2_l(k,lambda) = sum over v in C_{k,lambda} of deg_C(v,l)
// -- the `num_edge` the reference accumulates per cell (Core/FCPathLevelLeft.cpp:
// 60-64) -- and the node histogram gives |C_{k,lambda}|.  Each cell is then
// scored with the reference's expression (:66-90):
//     degree_l = (float)e2_l * 1.0f / 2;  sorted descending;
//     d_l = degree_(l) * 1.0f / |C| * 1.0 * pow(l, beta)   (FP64)
// keeping the best l (ties to the larger l), and the cells are folded in the
// reference's tree preorder (lambda-major, k ascending) with its float running
// maximum (Core/FCTree.cpp:69-82, main.cpp:406).  pow(l, beta) comes from the
// host's libm, as in the reference; every other step is IEEE FP32/FP64
// arithmetic in the same order, so densities are bit-identical.
#include <thrust/iterator/counting_iterator.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "device.h"

namespace fc {

struct DensState {
    uint32_t L = 0;
    std::vector<uint32_t> kmax;        // per lambda (index lambda-1)
    std::vector<uint64_t> hbase;       // per lambda: offset of H[lambda] (L*(kmax+1) words)
    std::vector<uint64_t> nbase;       // per lambda: offset of the node histogram
    std::vector<uint64_t> cbase;       // per lambda: first cell index
    uint64_t hwords = 0, nwords = 0, ncells = 0;
    uint32_t* H = nullptr;             // hwords: edge histogram -> suffix sums e2
    uint32_t* N = nullptr;             // nwords: node histogram -> suffix sums |C|
    uint32_t* coreT = nullptr;         // n*L node-major copy of the table
    uint64_t* d_hbase = nullptr;       // device copies of the bases (L each)
    uint64_t* d_nbase = nullptr;
    uint32_t* d_kmax = nullptr;
    fc_cell* cells = nullptr;          // ncells
    double* powl = nullptr;            // L
    fc_densest_result* d_res = nullptr;
    uint32_t* cell_lk = nullptr;       // 2 * ncells: lambda index, then k, per cell
    std::vector<uint32_t> cell_host;
    uint64_t H_cap = 0, N_cap = 0, cells_cap = 0, cell_lk_cap = 0, hbase_cap = 0, nbase_cap = 0;
    bool hist_valid = false;
    uint32_t lo = 0, hi = 0;           // the lambda columns (0-based) the histograms cover
};

template <class T>
static fc_status grow(T*& p, uint64_t& cap, uint64_t need, cudaStream_t st) {
    if (p && cap >= need) return FC_OK;
    dev_free(p, st);
    p = nullptr;
    cap = 0;
    uint64_t c = need + need / 4 + 16;
    FC_TRY(dev_alloc((void**)&p, c * sizeof(T), st));
    cap = c;
    return FC_OK;
}

void free_densest_state(DeviceGraph* d, cudaStream_t st) {
    DensState* s = (DensState*)d->dens;
    if (!s) return;
    // called with the graph's work finished (release_device waits for it, or
    // its caller knows that it has completed)
    for (void* p : {(void*)s->H, (void*)s->N, (void*)s->coreT, (void*)s->d_hbase,
                    (void*)s->d_nbase, (void*)s->d_kmax, (void*)s->cells, (void*)s->powl,
                    (void*)s->d_res, (void*)s->cell_lk})
        dev_free(p, st);
    delete s;
    d->dens = nullptr;
}

// ---- kernels -------------------------------------------------------------

__global__ void k_colmax(const uint32_t* __restrict__ table, uint32_t n, uint32_t L,
                         uint32_t* __restrict__ kmax) {
    // grid.y = lambda
    const uint32_t lam = blockIdx.y;
    const uint32_t* col = table + (uint64_t)lam * n;
    uint32_t m = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        m = max(m, col[v]);
    m = __reduce_max_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(kmax + lam, m);
}

// L < 32: one node per thread; each of its L loads is coalesced across the
// warp, and its values are stored as one row (a 16-byte store for L = 4)
__global__ void k_transpose_rows(const uint32_t* __restrict__ table, uint32_t n, uint32_t L,
                                 uint32_t* __restrict__ coreT) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        if (L == 4) {
            const uint4 q = make_uint4(table[v], table[(uint64_t)n + v], table[2ull * n + v],
                                       table[3ull * n + v]);
            *(uint4*)(coreT + 4ull * v) = q;
        } else {
            for (uint32_t l = 0; l < L; l++) coreT[(uint64_t)v * L + l] = table[(uint64_t)l * n + v];
        }
    }
}

__global__ void k_transpose(const uint32_t* __restrict__ table, uint32_t n, uint32_t L,
                            uint32_t* __restrict__ coreT) {
    // 32x32 tiles through shared memory
    __shared__ uint32_t tile[32][33];
    const uint32_t v0 = blockIdx.x * 32, l0 = blockIdx.y * 32;
    for (uint32_t r = threadIdx.y; r < 32; r += blockDim.y) {
        uint32_t l = l0 + r, v = v0 + threadIdx.x;
        if (l < L && v < n) tile[r][threadIdx.x] = table[(uint64_t)l * n + v];
    }
    __syncthreads();
    for (uint32_t r = threadIdx.y; r < 32; r += blockDim.y) {
        uint32_t v = v0 + r, l = l0 + threadIdx.x;
        if (l < L && v < n) coreT[(uint64_t)v * L + l] = tile[threadIdx.x][r];
    }
}

__global__ void k_node_hist(const uint32_t* __restrict__ table, uint32_t n,
                            const uint64_t* __restrict__ nbase, const uint32_t* __restrict__ kmax,
                            uint32_t* __restrict__ N) {
    extern __shared__ uint32_t sh[];
    const uint32_t lam = blockIdx.y;
    const uint32_t bins = kmax[lam] + 1;
    const bool use_sh = bins <= 12288;
    if (use_sh)
        for (uint32_t i = threadIdx.x; i < bins; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const uint32_t* col = table + (uint64_t)lam * n;
    uint32_t* out = N + nbase[lam];
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        uint32_t c = col[v];
        if (use_sh) atomicAdd(sh + c, 1u);
        else atomicAdd(out + c, 1u);
    }
    __syncthreads();
    if (use_sh)
        for (uint32_t i = threadIdx.x; i < bins; i += blockDim.x)
            if (sh[i]) atomicAdd(out + i, sh[i]);
}

// Edge histogram for lambda columns [lam0, lam0 + nl).  Each warp takes a
// contiguous slice of the entry array, 32 consecutive entries at a time (one
// per lane), and tracks each lane's source node by advancing along node_ptr.
// Bins live in shared memory when they fit (`sh_ok`), else in global memory.
// The entry (v, u, l) adds one to bin (l, min(core(v), core(u))) per column.
// The adjacency is symmetric (every (v, u, l) has its (u, v, l), in the same
// bin), so only the entry with u > v is visited and adds two; a self-loop
// (u = v, one entry) adds one.  The histogram is the same.
// sh_mode: 0 the bins in global memory, 1 in shared memory as 32-bit words,
// 2 in shared memory as 16-bit halves (a block's counts then stay below
// 65,536: the host chooses it only when 2 x its entries per block do).
__device__ __forceinline__ void edge_bin_add(uint32_t* sh, uint32_t* H, int sh_mode, uint32_t soff,
                                             uint64_t hbase, uint32_t l, uint32_t km1,
                                             uint32_t key, uint32_t cnt) {
    if (sh_mode == 2) {
        const uint32_t b = soff + l * km1 + key;
        atomicAdd(sh + (b >> 1), cnt << ((b & 1) * 16));
    } else if (sh_mode == 1) atomicAdd(sh + soff + l * km1 + key, cnt);
    else atomicAdd(H + hbase + (uint64_t)l * km1 + key, cnt);
}

// How a node's core values for the group's columns are read: one column at a
// time (EH_SCALAR); the group is four columns starting at a multiple of four
// with L a multiple of four, so a node's four values are one aligned 16-byte
// load, kept across its row (EH_V4); or the group starts at a multiple of four
// with L a multiple of four, any number of columns: four at a time, up to
// sixteen loads issued before their values are used (EH_QUAD).
enum : int { EH_SCALAR = 0, EH_V4 = 1, EH_QUAD = 2 };

template <int MODE>
__global__ void k_edge_hist(const uint32_t* __restrict__ node_ptr, const uint32_t* __restrict__ adj,
                            uint32_t n, uint32_t L, uint64_t entries, FastDiv divL,
                            const uint32_t* __restrict__ coreT, uint32_t lam0, uint32_t nl,
                            const uint64_t* __restrict__ hbase, const uint32_t* __restrict__ kmax,
                            uint32_t* __restrict__ H, uint32_t sh_words, int sh_ok) {
    // sh_ok: the shared-memory mode of edge_bin_add (0, 1 or 2); sh_words:
    // the 32-bit words the block clears
    constexpr bool V4 = MODE == EH_V4;
    extern __shared__ uint32_t sh[];
    __shared__ uint32_t soff[64];  // per column in the group: offset into sh
    __shared__ uint32_t skm1[64];  // kmax + 1
    __shared__ uint64_t shb[64];   // the column's base in H
    if (threadIdx.x == 0) {
        uint32_t o = 0;
        for (uint32_t i = 0; i < nl; i++) {
            soff[i] = o;
            skm1[i] = kmax[lam0 + i] + 1;
            shb[i] = hbase[lam0 + i];
            o += L * skm1[i];
        }
    }
    if (sh_ok)
        for (uint32_t i = threadIdx.x; i < sh_words; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t per = (entries + nwarps - 1) / nwarps;
    const uint64_t e0 = gw * per, e1 = min(entries, e0 + per);
    if (e0 < e1) {  // warp-uniform
        // source node of this lane's first entry: last v with node_ptr[v] <= e
        uint32_t lo = 0, hi = n;  // node_ptr[lo] <= e < node_ptr[hi]
        if (e0 + lane < e1) {
            while (hi - lo > 1) {
                uint32_t mid = (lo + hi) >> 1;
                if (node_ptr[mid] <= e0 + lane) lo = mid;
                else hi = mid;
            }
        }
        uint32_t v = lo;
        uint32_t next_row = node_ptr[v + 1];
        uint4 A = V4 ? *(const uint4*)(coreT + (uint64_t)v * L + lam0) : make_uint4(0, 0, 0, 0);
        for (uint64_t b0 = e0; b0 < e1; b0 += 32) {
            const uint64_t e = b0 + lane;
            uint32_t u = 0, l = 0, w = 0;  // w: what the entry adds (0, 1 or 2)
            if (e < e1) {
                if (next_row <= e) {
                    do v++;
                    while (node_ptr[v + 1] <= e);
                    next_row = node_ptr[v + 1];
                    if (V4) A = *(const uint4*)(coreT + (uint64_t)v * L + lam0);
                }
                const uint32_t slot = adj[e];
                u = divL.div(slot);
                l = slot - u * L;
                w = u > v ? 2u : u == v ? 1u : 0u;
            }
            if (MODE == EH_QUAD) {
                if (w) {
                    const uint32_t* av = coreT + (uint64_t)v * L + lam0;
                    const uint32_t* bu = coreT + (uint64_t)u * L + lam0;
                    const uint32_t nq = nl >> 2;
                    for (uint32_t q0 = 0; q0 < nq; q0 += 4) {
                        uint4 qa[4], qb[4];
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            qa[j] = qb[j] = make_uint4(0, 0, 0, 0);
                            if (q0 + j < nq) {
                                qa[j] = *(const uint4*)(av + 4 * (q0 + j));
                                qb[j] = *(const uint4*)(bu + 4 * (q0 + j));
                            }
                        }
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            const uint32_t i = 4 * (q0 + j);
                            const uint32_t ka[4] = {qa[j].x, qa[j].y, qa[j].z, qa[j].w};
                            const uint32_t kb[4] = {qb[j].x, qb[j].y, qb[j].z, qb[j].w};
#pragma unroll
                            for (int c = 0; c < 4; c++) {
                                const uint32_t key = min(ka[c], kb[c]);  // 0 past nq
                                if (key)
                                    edge_bin_add(sh, H, sh_ok, soff[i + c], shb[i + c], l,
                                                 skm1[i + c], key, w);
                            }
                        }
                    }
                    for (uint32_t i = nq * 4; i < nl; i++) {
                        const uint32_t a = av[i];
                        const uint32_t key = a ? min(a, bu[i]) : 0u;
                        if (key) edge_bin_add(sh, H, sh_ok, soff[i], shb[i], l, skm1[i], key, w);
                    }
                }
            } else {
                uint4 B = make_uint4(0, 0, 0, 0);
                if (V4 && w && (A.x | A.y | A.z | A.w))
                    B = *(const uint4*)(coreT + (uint64_t)u * L + lam0);
                for (uint32_t i = 0; i < nl; i++) {
                    uint32_t a = 0, b = 0;
                    if (V4) {
                        a = i == 0 ? A.x : i == 1 ? A.y : i == 2 ? A.z : A.w;
                        b = i == 0 ? B.x : i == 1 ? B.y : i == 2 ? B.z : B.w;
                    } else if (w) {
                        a = coreT[(uint64_t)v * L + lam0 + i];
                        if (a) b = coreT[(uint64_t)u * L + lam0 + i];
                    }
                    const uint32_t key = w ? min(a, b) : 0u;
                    if (key) edge_bin_add(sh, H, sh_ok, soff[i], shb[i], l, skm1[i], key, w);
                }
            }
        }
    }
    __syncthreads();
    if (sh_ok == 1) {
        for (uint32_t i = 0; i < nl; i++) {
            const uint32_t words = L * skm1[i];
            uint32_t* g = H + shb[i];
            for (uint32_t w = threadIdx.x; w < words; w += blockDim.x)
                if (sh[soff[i] + w]) atomicAdd(g + w, sh[soff[i] + w]);
        }
    } else if (sh_ok == 2) {
        for (uint32_t i = 0; i < nl; i++) {
            const uint32_t bins = L * skm1[i];
            uint32_t* g = H + shb[i];
            for (uint32_t w = threadIdx.x; w < bins; w += blockDim.x) {
                const uint32_t b = soff[i] + w;
                const uint32_t v = (sh[b >> 1] >> ((b & 1) * 16)) & 0xFFFFu;
                if (v) atomicAdd(g + w, v);
            }
        }
    }
}

// Suffix sums over key, per (lambda, layer) row of H and per lambda of N.
// uint32 arithmetic wraps exactly as the reference's `uint num_edge`.
__global__ void k_suffix(uint32_t L, const uint64_t* __restrict__ hbase,
                         const uint64_t* __restrict__ nbase, const uint32_t* __restrict__ kmax,
                         uint32_t* __restrict__ H, uint32_t* __restrict__ N) {
    const uint32_t lam = blockIdx.x;
    const uint32_t km1 = kmax[lam] + 1;
    for (uint32_t l = threadIdx.x; l <= L; l += blockDim.x) {
        uint32_t* row = l < L ? H + hbase[lam] + (uint64_t)l * km1 : N + nbase[lam];
        uint32_t acc = 0;
        for (int64_t k = (int64_t)km1 - 1; k >= 0; k--) {
            acc += row[k];
            row[k] = acc;
        }
    }
}

// One block per cell (lambda, k), k >= 1: sort the cell's L layer counts
// descending (bitonic sort in shared memory), evaluate every l, keep the best.
__global__ void k_cells(uint32_t L, uint32_t P /* pow2 >= L */, const uint64_t* __restrict__ hbase,
                        const uint64_t* __restrict__ nbase, const uint32_t* __restrict__ kmax,
                        const uint32_t* __restrict__ H, const uint32_t* __restrict__ N,
                        const double* __restrict__ powl, const uint32_t* __restrict__ cell_lam,
                        const uint32_t* __restrict__ cell_k, fc_cell* __restrict__ cells) {
    extern __shared__ uint32_t sv[];  // P values
    __shared__ double bestd[32];
    __shared__ uint32_t bestl[32];
    const uint32_t ci = blockIdx.x;
    const uint32_t lam = cell_lam[ci], k = cell_k[ci];
    const uint32_t km1 = kmax[lam] + 1;
    const uint32_t len = N[nbase[lam] + k];
    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x)
        sv[i] = i < L ? H[hbase[lam] + (uint64_t)i * km1 + k] : 0u;
    __syncthreads();
    // bitonic sort, descending
    for (uint32_t size = 2; size <= P; size <<= 1) {
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
                uint32_t p = i ^ stride;
                if (p > i) {
                    bool desc = (i & size) == 0;
                    uint32_t a = sv[i], b = sv[p];
                    if (desc ? (a < b) : (a > b)) {
                        sv[i] = b;
                        sv[p] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    double my_d = -1.0;
    uint32_t my_l = 0;
    for (uint32_t i = threadIdx.x; i < L; i += blockDim.x) {
        float f = __uint2float_rn(sv[i]) * 1.0f / 2;
        double degree = (double)f;
        double mad = (degree * 1.0f) / (double)len * 1.0;
        double d = mad * powl[i];
        if (d >= my_d) {  // later i in this thread's sequence wins ties
            my_d = d;
            my_l = i + 1;
        }
    }
    // block argmax, ties to the larger l
    for (int o = 16; o >= 1; o >>= 1) {
        double od = __shfl_down_sync(0xffffffffu, my_d, o);
        uint32_t ol = __shfl_down_sync(0xffffffffu, my_l, o);
        if (od > my_d || (od == my_d && ol > my_l)) {
            my_d = od;
            my_l = ol;
        }
    }
    const uint32_t w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        bestd[w] = my_d;
        bestl[w] = my_l;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double bd = -1.0;
        uint32_t bl = 0;
        for (uint32_t i = 0; i < (blockDim.x + 31) / 32; i++)
            if (bestd[i] > bd || (bestd[i] == bd && bestl[i] > bl)) {
                bd = bestd[i];
                bl = bestl[i];
            }
        // the reference starts from 0.0 and keeps l on `d >= best`
        fc_cell c;
        c.k = k;
        c.lmd = lam + 1;
        c.length = len;
        c.lstar = bl;
        c.density = bd < 0.0 ? 0.0 : bd;
        cells[ci] = c;
    }
}

// The reference's preorder fold with a float running maximum.
// One block: the cells' densities are staged in shared memory, FOLD_CHUNK at a
// time by all threads, and thread 0 folds them in order (the float running
// maximum is order-dependent, so the fold itself stays sequential).
constexpr uint32_t FOLD_CHUNK = 2048;
__global__ void k_fold(const fc_cell* __restrict__ cells, uint64_t ncells, double beta,
                       fc_densest_result* out) {
    __shared__ double sd[FOLD_CHUNK];
    __shared__ float s_maxd;
    __shared__ uint64_t s_win;  // winning cell, or ~0 for none
    if (threadIdx.x == 0) {
        s_maxd = 0.0f;
        s_win = ~0ull;
    }
    for (uint64_t c0 = 0; c0 < ncells; c0 += FOLD_CHUNK) {
        const uint32_t m = ncells - c0 < FOLD_CHUNK ? (uint32_t)(ncells - c0) : FOLD_CHUNK;
        __syncthreads();  // the last chunk is folded
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) sd[i] = cells[c0 + i].density;
        __syncthreads();
        if (threadIdx.x == 0) {
            float maxd = s_maxd;
            uint64_t win = s_win;
            for (uint32_t i = 0; i < m; i++)
                if (sd[i] >= (double)maxd) {
                    maxd = (float)sd[i];
                    win = c0 + i;
                }
            s_maxd = maxd;
            s_win = win;
        }
    }
    if (threadIdx.x == 0) {
        fc_densest_result r;
        r.beta = beta;
        r.density = 0.0;
        r.k = r.lmd = r.length = r.lstar = 0;
        if (s_win != ~0ull) {
            const fc_cell c = cells[s_win];
            r.density = c.density;
            r.k = c.k;
            r.lmd = c.lmd;
            r.length = c.length;
            r.lstar = c.lstar;
        }
        r.max_density_f = s_maxd;
        r.n_cells = (uint32_t)ncells;
        *out = r;
    }
}

// ---- host --------------------------------------------------------------------

static int sm_count() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// Histograms for the resident table (beta-independent), over the lambda
// columns [lo, hi): the other columns count as empty (kmax 0, no cells), and
// no kernel reads them, since they may not have been computed.
static fc_status build_hist(DeviceGraph* d, cudaStream_t st, uint32_t lo, uint32_t hi,
                            const std::function<fc_status()>* after_maxima = nullptr) {
    DensState* s = (DensState*)d->dens;
    if (s && s->hist_valid && s->lo == lo && s->hi == hi) return FC_OK;
    if (!s) {
        s = new DensState();
        d->dens = s;
    }
    const uint32_t n = d->n, L = d->L;
    s->L = L;
    // per-lambda maxima
    if (!s->d_kmax) FC_TRY(dev_alloc((void**)&s->d_kmax, (L + 1) * 4, st));
    FC_CUDA_TRY(cudaMemsetAsync(s->d_kmax, 0, (L + 1) * 4, st));
    // blocks per column: enough to fill the SMs, at least 2048 nodes each
    const uint32_t per_col = std::max<uint32_t>(
        1u, std::min<uint32_t>((n + 2047) / 2048,
                               8u * (uint32_t)sm_count() / std::max<uint32_t>(1u, hi - lo)));
    dim3 g(per_col, hi - lo);
    k_colmax<<<g, 256, 0, st>>>(d->table + (uint64_t)lo * n, n, L, s->d_kmax + lo);
    count_launch();
    FC_CUDA_TRY(cudaGetLastError());
    s->kmax.assign(L, 0);
    FC_TRY(to_host(s->kmax.data(), s->d_kmax, L * 4, st));
    if (after_maxima) FC_TRY((*after_maxima)());
    d->kmax = s->kmax;
    for (uint32_t l = 0; l < L; l++)
        if (s->kmax[l] > d->max_deg) return FC_ERR_DEVICE;  // not a valid core table
    s->hbase.assign(L, 0);
    s->nbase.assign(L, 0);
    s->cbase.assign(L, 0);
    uint64_t hw = 0, nw = 0, nc = 0;
    for (uint32_t l = 0; l < L; l++) {
        s->hbase[l] = hw;
        s->nbase[l] = nw;
        s->cbase[l] = nc;
        hw += (uint64_t)L * (s->kmax[l] + 1);
        nw += s->kmax[l] + 1;
        nc += s->kmax[l];
    }
    // grow-only buffers: a recomputation of the same graph allocates nothing
    s->hwords = hw;
    s->nwords = nw;
    s->ncells = nc;
    FC_TRY(grow(s->H, s->H_cap, hw + 1, st));
    FC_TRY(grow(s->N, s->N_cap, nw + 1, st));
    FC_TRY(grow(s->cells, s->cells_cap, nc + 1, st));
    FC_TRY(grow(s->cell_lk, s->cell_lk_cap, 2 * nc + 2, st));
    FC_TRY(grow(s->d_hbase, s->hbase_cap, L + 1, st));
    FC_TRY(grow(s->d_nbase, s->nbase_cap, L + 1, st));
    if (!s->coreT) FC_TRY(dev_alloc((void**)&s->coreT, (uint64_t)n * L * 4 + 4, st));
    FC_TRY(to_device(s->d_hbase, s->hbase.data(), L * 8, st));
    FC_TRY(to_device(s->d_nbase, s->nbase.data(), L * 8, st));
    // cell list (lambda index, k) in the reference's order, for k_cells
    s->cell_host.resize(2 * nc + 2);
    {
        uint64_t i = 0;
        for (uint32_t l = 0; l < L; l++)
            for (uint32_t k = 1; k <= s->kmax[l]; k++, i++) {
                s->cell_host[i] = l;
                s->cell_host[nc + i] = k;
            }
    }
    if (nc)
        FC_TRY(to_device(s->cell_lk, s->cell_host.data(), 2 * nc * 4, st));
    FC_CUDA_TRY(cudaMemsetAsync(s->H, 0, hw * 4 + 4, st));
    FC_CUDA_TRY(cudaMemsetAsync(s->N, 0, nw * 4 + 4, st));
    if (n && L) {
        if (L < 32) {
            const uint32_t tb =
                std::max<uint32_t>(1u, std::min<uint32_t>((n + 255) / 256, 8u * sm_count()));
            k_transpose_rows<<<tb, 256, 0, st>>>(d->table, n, L, s->coreT);
        } else {
            dim3 tg((n + 31) / 32, (L + 31) / 32);
            k_transpose<<<tg, dim3(32, 8), 0, st>>>(d->table, n, L, s->coreT);
        }
        FC_CUDA_TRY(cudaGetLastError());
        dim3 ng(per_col, hi - lo);
        k_node_hist<<<ng, 256, 12288 * 4, st>>>(d->table + (uint64_t)lo * n, n, s->d_nbase + lo,
                                               s->d_kmax + lo, s->N);
        count_launch(2);
        FC_CUDA_TRY(cudaGetLastError());
        // lambda groups whose bins fit the shared-memory budget
        const uint32_t SH_WORDS = 48 * 1024;  // 192 KB
        // once per process (thread-safe static initialisation)
        static const cudaError_t attr_rc = cudaFuncSetAttribute(
            k_edge_hist<EH_SCALAR>, cudaFuncAttributeMaxDynamicSharedMemorySize, SH_WORDS * 4);
        static const cudaError_t attr_rc4 = cudaFuncSetAttribute(
            k_edge_hist<EH_V4>, cudaFuncAttributeMaxDynamicSharedMemorySize, SH_WORDS * 4);
        static const cudaError_t attr_rcq = cudaFuncSetAttribute(
            k_edge_hist<EH_QUAD>, cudaFuncAttributeMaxDynamicSharedMemorySize, SH_WORDS * 4);
        FC_CUDA_TRY(attr_rc);
        FC_CUDA_TRY(attr_rc4);
        FC_CUDA_TRY(attr_rcq);
        FastDiv divL;
        divL.init(L);
        // about 16K entries per block, at most one block per SM: a block
        // clears and flushes all of its group's bins, which small graphs
        // should not pay on every SM (and graphs searched on other streams
        // get the SMs this one leaves)
        const uint64_t want = (d->entries + 16383) / 16384;
        const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>(sm_count(), want));
        // 16-bit bins when no block can count 65,536 in one bin (each entry
        // adds at most 2; a block's warps take at most 32 entries more than
        // an even share): twice the columns per pass over the entries
        const bool half = 2 * ((d->entries + blocks - 1) / blocks + 32) < 65536;
        const uint32_t budget = half ? 2 * SH_WORDS : SH_WORDS;  // bins
        uint32_t lam = lo;
        while (lam < hi) {
            uint32_t words = 0, nl = 0;  // words: bins of the group
            while (lam + nl < hi && nl < 64) {
                uint32_t w = L * (s->kmax[lam + nl] + 1);
                if (nl > 0 && words + w > budget) break;
                words += w;
                nl++;
            }
            // with L a multiple of four, groups of a multiple of four columns
            // keep the next group 16-byte aligned for quad loads
            if (L % 4 == 0 && lam % 4 == 0 && nl > 4 && lam + nl < hi && nl % 4) {
                nl &= ~3u;
                words = 0;
                for (uint32_t i = 0; i < nl; i++) words += L * (s->kmax[lam + i] + 1);
            }
            const int sh_ok = words > budget ? 0 : half ? 2 : 1;
            if (sh_ok == 2) words = (words + 1) / 2;  // the 32-bit words cleared
            size_t shb = sh_ok ? (size_t)words * 4 : 0;
            if (d->entries) {
                const bool aligned = L % 4 == 0 && lam % 4 == 0;
                if (aligned && nl == 4)
                    k_edge_hist<EH_V4><<<blocks, 1024, shb, st>>>(
                        d->node_ptr, d->adj, n, L, d->entries, divL, s->coreT, lam, nl, s->d_hbase,
                        s->d_kmax, s->H, words, sh_ok);
                else if (aligned && nl > 4)
                    k_edge_hist<EH_QUAD><<<blocks, 1024, shb, st>>>(
                        d->node_ptr, d->adj, n, L, d->entries, divL, s->coreT, lam, nl, s->d_hbase,
                        s->d_kmax, s->H, words, sh_ok);
                else
                    k_edge_hist<EH_SCALAR><<<blocks, 1024, shb, st>>>(
                        d->node_ptr, d->adj, n, L, d->entries, divL, s->coreT, lam, nl, s->d_hbase,
                        s->d_kmax, s->H, words, sh_ok);
                count_launch();
            }
            FC_CUDA_TRY(cudaGetLastError());
            lam += nl;
        }
        k_suffix<<<L, 128, 0, st>>>(L, s->d_hbase, s->d_nbase, s->d_kmax, s->H, s->N);
        count_launch();
        FC_CUDA_TRY(cudaGetLastError());
    }
    s->hist_valid = true;
    s->lo = lo;
    s->hi = hi;
    return FC_OK;
}

static fc_status score_cells(DeviceGraph* d, double beta, cudaStream_t st) {
    DensState* s = (DensState*)d->dens;
    const uint32_t L = d->L;
    if (!s->powl) FC_TRY(dev_alloc((void**)&s->powl, L * 8 + 8, st));
    std::vector<double> pw(L);
    for (uint32_t l = 0; l < L; l++) pw[l] = pow((double)(l + 1), beta);  // pow((l+1), beta)
    FC_TRY(to_device(s->powl, pw.data(), L * 8, st));
    if (!s->ncells) return FC_OK;
    uint32_t P = 1;
    while (P < L) P <<= 1;
    uint32_t threads = P < 32 ? 32 : (P > 1024 ? 1024 : P);
    size_t shb = (size_t)P * 4;
    if (shb > 48 * 1024) FC_CUDA_TRY(cudaFuncSetAttribute(k_cells, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shb));
    k_cells<<<(uint32_t)s->ncells, threads, shb, st>>>(L, P, s->d_hbase, s->d_nbase, s->d_kmax, s->H,
                                                      s->N, s->powl, s->cell_lk,
                                                      s->cell_lk + s->ncells, s->cells);
    count_launch();
    FC_CUDA_TRY(cudaGetLastError());
    return FC_OK;
}

fc_status densest(fc_graph* g, const double* betas, uint32_t nb, fc_densest_result* res,
                  cudaStream_t st, const std::function<fc_status()>* after_maxima) {
    FC_TRY(coreindex(g, nullptr, false, st));
    DeviceGraph* d = g->dev;
    struct Events {  // destroyed on every return
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ~Events() {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } ev;
    FC_CUDA_TRY(cudaEventCreate(&ev.e0));
    FC_CUDA_TRY(cudaEventCreate(&ev.e1));
    count_alloc(2);
    cudaEvent_t e0 = ev.e0, e1 = ev.e1;
    FC_CUDA_TRY(cudaEventRecord(e0, st));
    FC_TRY(build_hist(d, st, 0, d->L, after_maxima));
    DensState* s = (DensState*)d->dens;
    if (!s->d_res) FC_TRY(dev_alloc((void**)&s->d_res, sizeof(fc_densest_result), st));
    for (uint32_t b = 0; b < nb; b++) {
        FC_TRY(score_cells(d, betas[b], st));
        k_fold<<<1, 256, 0, st>>>(s->cells, s->ncells, betas[b], s->d_res);
        count_launch();
        FC_CUDA_TRY(cudaGetLastError());
        FC_TRY(to_host(res + b, s->d_res, sizeof(fc_densest_result), st));
    }
    FC_CUDA_TRY(cudaEventRecord(e1, st));
    FC_CUDA_TRY(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    d->stats.densest_ms = ms;
    return FC_OK;
}

fc_status cells(fc_graph* g, double beta, fc_cell* out, uint32_t cap, uint32_t* count,
                cudaStream_t st) {
    FC_TRY(coreindex(g, nullptr, false, st));
    DeviceGraph* d = g->dev;
    FC_TRY(build_hist(d, st, 0, d->L));
    DensState* s = (DensState*)d->dens;
    FC_TRY(score_cells(d, beta, st));
    uint64_t nc = s->ncells;
    if (count) *count = (uint32_t)nc;
    uint64_t w = nc < cap ? nc : cap;
    if (w && out) FC_TRY(to_host(out, s->cells, w * sizeof(fc_cell), st));
    FC_CUDA_TRY(cudaStreamSynchronize(st));
    return FC_OK;
}

// The cells of the lambda columns [lo, hi) (0-based), computing those
// columns first when they are not resident.
fc_status cells_range(fc_graph* g, uint32_t lo, uint32_t hi, double beta, fc_cell* out, uint32_t cap,
                      uint32_t* count, cudaStream_t st) {
    FC_TRY(coreindex_range(g, lo, hi, nullptr, false, st));
    DeviceGraph* d = g->dev;
    FC_TRY(build_hist(d, st, lo, hi));
    DensState* s = (DensState*)d->dens;
    FC_TRY(score_cells(d, beta, st));
    const uint64_t nc = s->ncells;
    if (count) *count = (uint32_t)nc;
    const uint64_t w = nc < cap ? nc : cap;
    if (w && out) FC_TRY(to_host(out, s->cells, w * sizeof(fc_cell), st));
    FC_CUDA_TRY(cudaStreamSynchronize(st));
    d->home = nullptr;
    return FC_OK;
}

fc_status densest_members(fc_graph* g, const fc_densest_result* r, uint32_t* nodes,
                          uint32_t* layers, cudaStream_t st) {
    if (!r || r->k == 0) return FC_OK;
    FC_TRY(coreindex(g, nullptr, false, st));
    DeviceGraph* d = g->dev;
    FC_TRY(build_hist(d, st, 0, d->L));
    DensState* s = (DensState*)d->dens;
    const uint32_t n = d->n, L = d->L, lam = r->lmd - 1;
    if (r->lmd < 1 || r->lmd > L || r->k > s->kmax[lam]) return FC_ERR_INVALID;
    if (nodes) {
        std::vector<uint32_t> col(n);
        FC_TRY(to_host(col.data(), d->table + (uint64_t)lam * n, (uint64_t)n * 4, st));
        uint32_t j = 0;
        for (uint32_t v = 0; v < n; v++)
            if (col[v] >= r->k) nodes[j++] = v;
    }
    if (layers) {
        // the cell's layer counts; the first lstar of the descending order
        // (ties by layer index) -- for beta >= 0 lstar never splits a tie
        const uint32_t km1 = s->kmax[lam] + 1;
        std::vector<uint32_t> e(L);
        for (uint32_t l = 0; l < L; l++)
            FC_TRY(to_host(&e[l], s->H + s->hbase[lam] + (uint64_t)l * km1 + r->k, 4, st));
        std::vector<uint32_t> idx(L);
        for (uint32_t l = 0; l < L; l++) idx[l] = l;
        std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return e[a] > e[b]; });
        std::vector<uint32_t> pick(idx.begin(), idx.begin() + r->lstar);
        std::sort(pick.begin(), pick.end());
        for (uint32_t i = 0; i < r->lstar; i++) layers[i] = pick[i];
    }
    return FC_OK;
}

void invalidate_densest(DeviceGraph* d) {
    invalidate_cell_index(d);
    DensState* s = (DensState*)d->dens;
    if (s) s->hist_valid = false;
}

// C_{k,lambda} = {v : core_lambda(v) >= k} in ascending ids, by an
// order-preserving stream compaction of the lambda column on the device (the
// query of -m kpe -k -lmd, main.cpp:197-225 and FCTree::saveCoreToLocal,
// Core/FCTree.cpp:138-153).
struct InCell {
    const uint32_t* col;
    uint32_t k;
    __host__ __device__ __forceinline__ bool operator()(uint32_t v) const { return col[v] >= k; }
};

fc_status cell_members(fc_graph* g, uint32_t k, uint32_t lmd, uint32_t* nodes, uint32_t cap,
                       uint32_t* count, cudaStream_t st) {
    if (lmd < 1 || lmd > g->L) return FC_ERR_INVALID;
    FC_TRY(coreindex(g, nullptr, false, st));
    DeviceGraph* d = g->dev;
    const uint32_t n = d->n;
    uint32_t* out = nullptr;
    uint32_t* num = nullptr;
    void* tmp = nullptr;
    size_t tb = 0;
    const InCell pred{d->table + (uint64_t)(lmd - 1) * n, k};
    thrust::counting_iterator<uint32_t> ids(0);
    FC_CUDA_TRY(cub::DeviceSelect::If(nullptr, tb, ids, out, num, (int)n, pred, st));
    fc_status rc = dev_alloc((void**)&out, (uint64_t)n * 4 + 4, st);
    if (rc == FC_OK) rc = dev_alloc((void**)&num, 8, st);
    if (rc == FC_OK) rc = dev_alloc(&tmp, tb + 16, st);
    uint32_t total = 0;
    if (rc == FC_OK) {
        const cudaError_t e = cub::DeviceSelect::If(tmp, tb, ids, out, num, (int)n, pred, st);
        count_launch(1);
        if (e != cudaSuccess) {
            set_last_cuda_error(e, "DeviceSelect::If", __FILE__, __LINE__);
            rc = FC_ERR_DEVICE;
        }
    }
    if (rc == FC_OK) rc = to_host(&total, num, 4, st);
    if (rc == FC_OK && nodes && total)
        rc = to_host(nodes, out, (size_t)std::min(total, cap) * 4, st);
    dev_free(tmp, st);
    dev_free(num, st);
    dev_free(out, st);
    if (count) *count = total;
    return rc;
}

void densest_preload() {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, k_colmax);
    cudaFuncGetAttributes(&a, k_transpose);
    cudaFuncGetAttributes(&a, k_transpose_rows);
    cudaFuncGetAttributes(&a, k_node_hist);
    cudaFuncGetAttributes(&a, k_edge_hist<EH_SCALAR>);
    cudaFuncGetAttributes(&a, k_edge_hist<EH_V4>);
    cudaFuncGetAttributes(&a, k_edge_hist<EH_QUAD>);
    cudaFuncGetAttributes(&a, k_suffix);
    cudaFuncGetAttributes(&a, k_cells);
    cudaFuncGetAttributes(&a, k_fold);
    cudaGetLastError();
}

}  // namespace fc
