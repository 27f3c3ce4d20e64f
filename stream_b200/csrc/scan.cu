#include "scan.cuh"

namespace sb {
namespace {

constexpr int kTile = 4096;
constexpr int kBlock = 256;
constexpr int kItems = kTile / kBlock;

__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* s) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) s[w] = v;
    __syncthreads();
    uint32_t t = 0;
    if (threadIdx.x < 32) {
        t = threadIdx.x < (kBlock / 32) ? s[threadIdx.x] : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    return t;  // valid in thread 0
}

__global__ void __launch_bounds__(kBlock) k_tile_sums(const uint32_t* __restrict__ in, uint32_t n,
                                                      uint32_t* __restrict__ partial) {
    __shared__ uint32_t s[32];
    const uint32_t base = blockIdx.x * kTile;
    uint32_t v = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const uint32_t idx = base + i * kBlock + threadIdx.x;
        if (idx < n) v += in[idx];
    }
    v = block_sum(v, s);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
}

// Exclusive scan of the tile sums in place (single block, any count).
__global__ void __launch_bounds__(1024) k_scan_partials(uint32_t* partial, uint32_t m) {
    __shared__ uint32_t s[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < m; base += 1024) {
        const uint32_t idx = base + threadIdx.x;
        const uint32_t v = idx < m ? partial[idx] : 0u;
        uint32_t x = v;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t t = s[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            s[lane] = t;
        }
        __syncthreads();
        const uint32_t incl = x + (w ? s[w - 1] : 0u);
        const uint32_t c = carry;
        if (idx < m) partial[idx] = c + incl - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry = c + incl;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kBlock) k_tile_scan(const uint32_t* __restrict__ in, uint32_t n,
                                                      const uint32_t* __restrict__ partial, uint32_t* __restrict__ out) {
    __shared__ uint32_t s[32];
    const uint32_t base = blockIdx.x * kTile + threadIdx.x * kItems;
    uint32_t v[kItems];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const uint32_t idx = base + i;
        v[i] = idx < n ? in[idx] : 0u;
        sum += v[i];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t t = lane < kBlock / 32 ? s[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        s[lane] = t;
    }
    __syncthreads();
    uint32_t run = partial[blockIdx.x] + (w ? s[w - 1] : 0u) + x - sum;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const uint32_t idx = base + i;
        run += v[i];
        if (idx < n) out[idx + 1] = run;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[0] = 0u;
}

}  // namespace

void exclusive_scan_u32(ScanPlan& plan, const uint32_t* in, uint32_t* out, uint32_t n, cudaStream_t stream) {
    const uint32_t tiles = n == 0 ? 1 : (n + kTile - 1) / kTile;
    plan.partial.ensure(tiles);
    k_tile_sums<<<tiles, kBlock, 0, stream>>>(in, n, plan.partial.ptr);
    SB_LAUNCH_CHECK();
    k_scan_partials<<<1, 1024, 0, stream>>>(plan.partial.ptr, tiles);
    SB_LAUNCH_CHECK();
    k_tile_scan<<<tiles, kBlock, 0, stream>>>(in, n, plan.partial.ptr, out);
    SB_LAUNCH_CHECK();
}

}  // namespace sb
