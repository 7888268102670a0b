// Exclusive prefix sum of a uint32 array on the device (three passes: tile
// sums, scan of the tile sums in one CTA, tile scans with the offsets).
// Integer arithmetic: the result does not depend on the schedule.
#include <cuda_runtime.h>

#include <algorithm>

#include "cam_internal.h"

namespace cam {
namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t *warp_sums, uint32_t *total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += o;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const uint32_t ws = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0u;
        uint32_t wi = ws;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, wi, off);
            if (lane >= off) wi += o;
        }
        if (lane < (int)(blockDim.x >> 5)) warp_sums[lane] = wi - ws;
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    return warp_sums[wid] + incl - v;
}

__global__ void __launch_bounds__(kScanThreads) tile_sum_kernel(const uint32_t *__restrict__ in, int64_t n,
                                                                uint32_t *__restrict__ sums)
{
    __shared__ uint32_t red[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const int64_t idx = base + (int64_t)threadIdx.x * kScanItems + i;
        if (idx < n) s += in[idx];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kScanThreads / 32; ++w) t += red[w];
        sums[blockIdx.x] = t;
    }
}

// Exclusive scan of the tile sums (one CTA, any count); sums[ntiles] = total.
__global__ void __launch_bounds__(kScanThreads) tile_offsets_kernel(uint32_t *__restrict__ sums, int ntiles)
{
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t tot;
    uint32_t carry = 0;
    for (int base = 0; base < ntiles; base += kScanThreads) {
        const int idx = base + threadIdx.x;
        const uint32_t v = idx < ntiles ? sums[idx] : 0u;
        const uint32_t ex = block_exclusive(v, warp_sums, &tot);
        if (idx < ntiles) sums[idx] = carry + ex;
        __syncthreads();
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[ntiles] = carry;
}

__global__ void __launch_bounds__(kScanThreads) tile_scan_kernel(uint32_t *__restrict__ data, int64_t n,
                                                                 const uint32_t *__restrict__ offsets)
{
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t tot;
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < n ? data[base + i] : 0u;
        s += v[i];
    }
    uint32_t run = offsets[blockIdx.x] + block_exclusive(s, warp_sums, &tot);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) data[base + i] = run;
        run += v[i];
    }
}

}  // namespace

// In place; `total` (device, may be null) receives the sum of all inputs.
void exclusive_scan_u32(cam_ctx *ctx, uint32_t *data, int64_t n, uint32_t *total)
{
    const int64_t ntiles = std::max<int64_t>(1, (n + kScanTile - 1) / kScanTile);
    CAM_REQUIRE(ntiles < (1ll << 31), CAM_E_UNSUPPORTED, "scan too large");
    auto *sums = static_cast<uint32_t *>(scratch(ctx, "scan.sums", (ntiles + 1) * sizeof(uint32_t)));
    CAM_LAUNCH(ctx, tile_sum_kernel, (unsigned)ntiles, kScanThreads, 0, data, n, sums);
    CAM_LAUNCH(ctx, tile_offsets_kernel, 1, kScanThreads, 0, sums, (int)ntiles);
    CAM_LAUNCH(ctx, tile_scan_kernel, (unsigned)ntiles, kScanThreads, 0, data, n, sums);
    if (total)
        CAM_CUDA_TRY(cudaMemcpyAsync(total, sums + ntiles, sizeof(uint32_t), cudaMemcpyDeviceToDevice, ctx->stream));
}

}  // namespace cam
