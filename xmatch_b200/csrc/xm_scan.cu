// xm_scan.cu -- exclusive prefix sum of uint32 counts (zone histograms, tile
// counts).  Three passes: per-tile totals, one block scanning the totals with
// a running carry, per-tile scan plus the tile's offset.  out[n] receives the
// grand total, so a zone histogram of length n becomes the zone offset array
// with the end sentinel (the zone begin/end of Sorter.cu:156-165).
#include "xm_internal.h"

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;  // 4096

// Exclusive scan of one value per thread across the block; returns the
// block total through *total.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t *total)
{
    __shared__ uint32_t warp_sums[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kThreads / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kThreads / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    uint32_t before = (warp > 0 ? warp_sums[warp - 1] : 0) + x - v;
    *total = warp_sums[kThreads / 32 - 1];
    __syncthreads();
    return before;
}

__global__ void scan_tile_sums(const uint32_t *__restrict__ in, size_t n, uint32_t *__restrict__ sums)
{
    size_t base = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * kItems;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k)
        if (base + k < n) s += in[base + k];
    uint32_t total;
    block_exclusive(s, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// Single block: exclusive scan of the tile totals in place, total to sums[nb].
__global__ void scan_sums_single(uint32_t *sums, size_t nb)
{
    uint32_t carry = 0;
    for (size_t start = 0; start < nb; start += kTile) {
        size_t base = start + (size_t)threadIdx.x * kItems;
        uint32_t v[kItems];
        uint32_t s = 0;
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            v[k] = base + k < nb ? sums[base + k] : 0;
            s += v[k];
        }
        uint32_t total;
        uint32_t run = carry + block_exclusive(s, &total);
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            if (base + k < nb) sums[base + k] = run;
            run += v[k];
        }
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[nb] = carry;
}

__global__ void scan_tile_apply(const uint32_t *__restrict__ in, size_t n,
                                const uint32_t *__restrict__ sums, uint32_t *__restrict__ out)
{
    size_t base = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * kItems;
    uint32_t v[kItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    uint32_t total;
    uint32_t run = sums[blockIdx.x] + block_exclusive(s, &total);
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = sums[gridDim.x];
}

}  // namespace

size_t xm_scan_tmp_bytes(size_t n)
{
    size_t nb = (n + kTile - 1) / kTile;
    return (nb + 1) * sizeof(uint32_t);
}

cudaError_t xm_scan_exclusive_u32(const uint32_t *in, uint32_t *out, size_t n, void *tmp,
                                  cudaStream_t s)
{
    if (n == 0) return cudaMemsetAsync(out, 0, sizeof(uint32_t), s);
    size_t nb = (n + kTile - 1) / kTile;
    uint32_t *sums = (uint32_t *)tmp;
    scan_tile_sums<<<(unsigned)nb, kThreads, 0, s>>>(in, n, sums);
    scan_sums_single<<<1, kThreads, 0, s>>>(sums, nb);
    scan_tile_apply<<<(unsigned)nb, kThreads, 0, s>>>(in, n, sums, out);
    return cudaGetLastError();
}
