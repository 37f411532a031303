// Device-wide exclusive prefix sum over uint32 counts (three launches: block sums, one-CTA
// scan of the block sums, block-local scan plus offset). Used to build CSR offsets.
#pragma once
#include "common.cuh"

namespace xkb {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;                       // items per thread
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t * warp_tot, uint32_t & total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) { uint32_t y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0)
    {
        uint32_t t = lane < nwarps ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) { uint32_t y = __shfl_up_sync(0xffffffffu, t, o); if (lane >= o) t += y; }
        if (lane < nwarps) warp_tot[lane] = t;
    }
    __syncthreads();
    total = warp_tot[nwarps - 1];
    const uint32_t before = warp ? warp_tot[warp - 1] : 0;
    __syncthreads();
    return before + x - v;
}

__global__ void scan_block_sums(const uint32_t * __restrict__ in, size_t n, uint32_t * __restrict__ sums)
{
    __shared__ uint32_t wt[32];
    const size_t base = (size_t) blockIdx.x * SCAN_TILE + (size_t) threadIdx.x * SCAN_ITEMS;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) if (base + k < n) s += in[base + k];
    uint32_t total;
    block_exclusive_scan(s, wt, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// single CTA: exclusive scan of nblocks sums in place (loops over chunks of SCAN_THREADS)
__global__ void scan_sums_inplace(uint32_t * sums, size_t nblocks)
{
    __shared__ uint32_t wt[32];
    uint32_t carry = 0;
    for (size_t base = 0; base < nblocks; base += SCAN_THREADS)
    {
        const size_t i = base + threadIdx.x;
        const uint32_t v = i < nblocks ? sums[i] : 0;
        uint32_t total;
        const uint32_t ex = block_exclusive_scan(v, wt, total);
        if (i < nblocks) sums[i] = carry + ex;
        carry += total;
    }
}

__global__ void scan_finish(const uint32_t * __restrict__ in, size_t n, const uint32_t * __restrict__ sums,
                            uint32_t * __restrict__ out, uint32_t * __restrict__ grand_total)
{
    __shared__ uint32_t wt[32];
    const size_t base = (size_t) blockIdx.x * SCAN_TILE + (size_t) threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS], s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) { v[k] = base + k < n ? in[base + k] : 0; s += v[k]; }
    uint32_t total;
    uint32_t run = sums[blockIdx.x] + block_exclusive_scan(s, wt, total);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) { if (base + k < n) out[base + k] = run; run += v[k]; }
    if (grand_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) *grand_total = run;
}

// out[i] = sum(in[0..i)), out may alias in; *grand_total (device) = sum of all. `tmp` holds
// ceil(n / SCAN_TILE) uint32.
static inline int device_exclusive_scan(const uint32_t * in, uint32_t * out, size_t n, uint32_t * tmp,
                                        uint32_t * grand_total, cudaStream_t st)
{
    if (n == 0) return XKB_OK;
    const size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    scan_block_sums<<<(unsigned) nb, SCAN_THREADS, 0, st>>>(in, n, tmp);
    scan_sums_inplace<<<1, SCAN_THREADS, 0, st>>>(tmp, nb);
    scan_finish<<<(unsigned) nb, SCAN_THREADS, 0, st>>>(in, n, tmp, out, grand_total);
    XKB_CUDA_TRY(cudaGetLastError());
    return XKB_OK;
}

} // namespace xkb
