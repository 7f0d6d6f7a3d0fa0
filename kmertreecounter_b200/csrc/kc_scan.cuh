// Device-wide exclusive scan used by the batch pipeline (line index per
// tile, per-tile first-occurrence offsets).  Three launches: per-block
// totals, one block scanning those totals, per-block rescan with its offset.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace kc {

constexpr int SCAN_BLOCK = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__device__ __forceinline__ uint64_t block_exclusive_scan_u64(uint64_t v, uint64_t* smem_warp, uint64_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = lane < nwarps ? smem_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nwarps) smem_warp[lane] = w;
    }
    __syncthreads();
    const uint64_t r = (warp ? smem_warp[warp - 1] : 0) + x - v;
    if (total) *total = smem_warp[nwarps - 1];
    __syncthreads();
    return r;
}

template <class TI>
__global__ void __launch_bounds__(SCAN_BLOCK) scan_reduce(const TI* __restrict__ in, uint64_t n,
                                                          uint64_t* __restrict__ sums) {
    __shared__ uint64_t sw[32];
    const uint64_t b0 = (uint64_t)blockIdx.x * SCAN_TILE;
    uint64_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        const uint64_t idx = b0 + (uint64_t)threadIdx.x * SCAN_ITEMS + i;
        if (idx < n) s += (uint64_t)in[idx];
    }
    uint64_t total;
    block_exclusive_scan_u64(s, sw, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// One block: sums[0..nb) -> exclusive prefix + base; *total_out = base + sum.
static __global__ void __launch_bounds__(SCAN_BLOCK) scan_sums(uint64_t* __restrict__ sums, uint64_t nb, uint64_t base,
                                                        uint64_t* __restrict__ total_out) {
    __shared__ uint64_t sw[32];
    uint64_t carry = base;
    for (uint64_t c = 0; c < nb; c += SCAN_BLOCK) {
        const uint64_t idx = c + threadIdx.x;
        const uint64_t v = idx < nb ? sums[idx] : 0;
        uint64_t tot;
        const uint64_t ex = block_exclusive_scan_u64(v, sw, &tot);
        if (idx < nb) sums[idx] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && total_out) *total_out = carry;
}

template <class TI, class TO>
__global__ void __launch_bounds__(SCAN_BLOCK) scan_apply(const TI* __restrict__ in, uint64_t n,
                                                         const uint64_t* __restrict__ sums, TO* __restrict__ out) {
    __shared__ uint64_t sw[32];
    const uint64_t b0 = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
    uint64_t v[SCAN_ITEMS];
    uint64_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        v[i] = (b0 + i < n) ? (uint64_t)in[b0 + i] : 0;
        s += v[i];
    }
    uint64_t run = sums[blockIdx.x] + block_exclusive_scan_u64(s, sw, nullptr);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        if (b0 + i < n) out[b0 + i] = (TO)run;
        run += v[i];
    }
}

}  // namespace kc
