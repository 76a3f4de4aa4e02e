// Device probe for the roofline's atomic denominator: the rate at which the
// GPU completes 4-byte atomic subtractions whose old value is returned (the
// form the peel's degree decrements take), at pseudo-random word addresses of
// a buffer that fits the L2 cache or does not.
#include <algorithm>

#include "device.h"

namespace fc {

// splitmix-style mixing of (thread, step) into a word index
__device__ __forceinline__ uint32_t probe_hash(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return (uint32_t)(x ^ (x >> 31));
}

// Each thread issues `per_thread` atomics, 8 independent ones in flight.
__global__ void __launch_bounds__(256) k_probe_atomics(uint32_t* __restrict__ buf, uint32_t mask,
                                                       uint32_t per_thread,
                                                       uint32_t* __restrict__ sink) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint32_t acc = 0;
    for (uint32_t i = 0; i < per_thread; i += 8) {
        uint32_t a[8];
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = probe_hash((t << 32) | (i + j)) & mask;
#pragma unroll
        for (int j = 0; j < 8; j++) acc += atomicSub(buf + a[j], 1u);
    }
    if (acc == 0x5A5A5A5Au) *sink = acc;  // keeps the returned values live
}

fc_status probe_atomics(uint64_t bytes, uint64_t ops, double* rate, cudaStream_t s) {
    // the largest power-of-two word count that fits `bytes` (every index is
    // masked into it)
    uint64_t words = 1;
    while (words * 2 * 4 <= bytes && words < (1ull << 31)) words <<= 1;
    if (words < 1024) return FC_ERR_INVALID;
    int dev = 0, sms = 0;
    FC_CUDA_TRY(cudaGetDevice(&dev));
    FC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const uint32_t blocks = (uint32_t)sms * 8, threads = 256;
    const uint64_t nthreads = (uint64_t)blocks * threads;
    uint32_t per = (uint32_t)std::max<uint64_t>(8, (ops + nthreads - 1) / nthreads);
    per = (per + 7) / 8 * 8;
    uint32_t* buf = nullptr;
    FC_TRY(dev_alloc((void**)&buf, words * 4 + 64, s));
    FC_CUDA_TRY(cudaMemsetAsync(buf, 0, words * 4 + 64, s));
    cudaEvent_t e0, e1;
    FC_CUDA_TRY(cudaEventCreate(&e0));
    FC_CUDA_TRY(cudaEventCreate(&e1));
    count_alloc(2);
    uint32_t* sink = buf + words;
    k_probe_atomics<<<blocks, threads, 0, s>>>(buf, (uint32_t)(words - 1), 8, sink);  // warm
    cudaEventRecord(e0, s);
    k_probe_atomics<<<blocks, threads, 0, s>>>(buf, (uint32_t)(words - 1), per, sink);
    cudaEventRecord(e1, s);
    count_launch(2);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    dev_free(buf, s);
    FC_CUDA_TRY(err);
    *rate = ms > 0 ? (double)nthreads * per / (ms * 1e-3) / 1e9 : 0.0;
    return FC_OK;
}

}  // namespace fc
