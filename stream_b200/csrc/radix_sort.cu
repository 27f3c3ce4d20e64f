// Onesweep LSD radix sort for (u64 key, u32 value) pairs on sm_100a.
#include "radix_sort.cuh"

namespace sb {
namespace {

constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagIncl = 2u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1u;
constexpr uint32_t kSpinLimit = 1u << 22;

// Look-back words carry their flag and their count in one 32-bit word and
// publish nothing else, so relaxed GPU-scope accesses suffice: a reader sees
// either the old word or the whole new one.  (Release/acquire fences cost
// 12% of the pass at 64M keys.)
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Histogram of every digit position, one pass over the keys.
__global__ void __launch_bounds__(256) k_hist(const uint64_t* __restrict__ keys, uint32_t n, int passes,
                                              uint32_t* __restrict__ hist) {
    __shared__ uint32_t s[kSortMaxPasses * 256];
    for (int i = threadIdx.x; i < kSortMaxPasses * 256; i += blockDim.x) s[i] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        radix_hist_add(s, keys[i], passes);
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x)
        if (s[i]) atomicAdd(&hist[i], s[i]);
}

// Block-wide exclusive scan of one value per thread (256 threads).
__device__ __forceinline__ uint32_t block_excl_scan256(uint32_t v, uint32_t* s_warp, uint32_t* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t t = lane < 8 ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < 8) s_warp[8 + lane] = t;  // inclusive warp totals
    }
    __syncthreads();
    const uint32_t warp_excl = w ? s_warp[8 + w - 1] : 0u;
    if (total) *total = s_warp[8 + 7];
    return warp_excl + x - v;
}

// Per-pass exclusive digit offsets from the counts (one block per pass).
__global__ void __launch_bounds__(256) k_hist_scan(uint32_t* hist) {
    __shared__ uint32_t s_warp[16];
    uint32_t* h = hist + blockIdx.x * 256;
    const uint32_t c = h[threadIdx.x];
    const uint32_t e = block_excl_scan256(c, s_warp, nullptr);
    h[threadIdx.x] = e;
}

struct __align__(16) SortSmem {
    uint64_t keys[kSortTile];            // 32 KiB: the tile's keys in (digit, input order) order
    uint32_t vals[kSortTile];            // 16 KiB: their values
    uint32_t warp_hist[8][256];          // per-warp digit counts, then offsets
    uint32_t local_start[256];
    uint32_t global_base[256];
    uint32_t scan_tmp[16];
    uint32_t tile_id;
};

// One pass: keys and values of a 4096-key tile are loaded together up front,
// ranked per warp (digit peers from eight bit ballots), the tile's global
// digit offsets come from the decoupled look-back, both are staged in shared
// memory in (digit, input order) order and written out in digit runs.  3
// resident blocks per SM (register cap 85, 58 KiB of shared memory each) keep
// enough tiles in flight to hide the look-back and load latencies.
__global__ void __launch_bounds__(kSortBlock, 3) k_onesweep(const uint64_t* __restrict__ kin,
                                                            const uint32_t* __restrict__ vin,
                                                            uint64_t* __restrict__ kout,
                                                            uint32_t* __restrict__ vout, uint32_t n,
                                                            int shift, const uint32_t* __restrict__ digit_off,
                                                            uint32_t* lookback, uint32_t* tile_ctr,
                                                            uint32_t* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem& S = *reinterpret_cast<SortSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;

    if (tid == 0) S.tile_id = atomicAdd(tile_ctr, 1u);
    for (int i = tid; i < 8 * 256; i += kSortBlock) (&S.warp_hist[0][0])[i] = 0u;
    __syncthreads();
    const uint32_t tile = S.tile_id;
    const uint32_t base = tile * kSortTile;
    const uint32_t wbase = base + (uint32_t)w * 32u * kSortItems;

    uint64_t k[kSortItems];
    uint32_t v[kSortItems];
    uint32_t rank[kSortItems];
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        k[i] = idx < n ? kin[idx] : 0ull;
        v[i] = idx < n ? vin[idx] : 0u;
    }
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = (uint32_t)(k[i] >> shift) & 0xffu;
        uint32_t peers = __ballot_sync(0xffffffffu, valid);  // lanes with the same digit, bit by bit
#pragma unroll
        for (int bit = 0; bit < 8; ++bit) {
            const uint32_t ones = __ballot_sync(0xffffffffu, (d >> bit) & 1u);
            peers &= ((d >> bit) & 1u) ? ones : ~ones;
        }
        const int leader = __ffs(peers) - 1;
        uint32_t old = 0;
        if (valid && lane == leader) {
            old = S.warp_hist[w][d];
            S.warp_hist[w][d] = old + __popc(peers);
        }
        old = __shfl_sync(0xffffffffu, old, leader);
        rank[i] = old + __popc(peers & lt);
        __syncwarp();
    }
    __syncthreads();

    // Thread tid owns digit tid: warp offsets within the tile and tile total.
    uint32_t tile_count = 0;
#pragma unroll
    for (int ww = 0; ww < 8; ++ww) {
        const uint32_t c = S.warp_hist[ww][tid];
        S.warp_hist[ww][tid] = tile_count;
        tile_count += c;
    }
    uint32_t* lb = lookback + (size_t)tile * 256 + tid;
    if (tile == 0) st_relaxed(lb, kFlagIncl | tile_count);
    else st_relaxed(lb, kFlagAgg | tile_count);

    const uint32_t lstart = block_excl_scan256(tile_count, S.scan_tmp, nullptr);
    S.local_start[tid] = lstart;

    uint32_t excl = 0;
    if (tile > 0) {
        int j = (int)tile - 1;
        uint32_t spins = 0;
        while (j >= 0) {
            const uint32_t wv = ld_relaxed(lookback + (size_t)j * 256 + tid);
            const uint32_t flag = wv & ~kValMask;
            if (flag == 0u) {
                if (++spins > kSpinLimit) {
                    atomicOr(status, ST_LOOKBACK_TIMEOUT);
                    break;
                }
                __nanosleep(20);
                continue;
            }
            excl += wv & kValMask;
            if (flag == kFlagIncl) break;
            --j;
        }
        st_relaxed(lb, kFlagIncl | ((excl + tile_count) & kValMask));
    }
    S.global_base[tid] = digit_off[tid] + excl - lstart;
    __syncthreads();

    // Stage keys and values in (digit, input order) order.
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        if (idx < n) {
            const uint32_t d = (uint32_t)(k[i] >> shift) & 0xffu;
            const uint32_t pos = S.local_start[d] + S.warp_hist[w][d] + rank[i];
            S.keys[pos] = k[i];
            S.vals[pos] = v[i];
        }
    }
    __syncthreads();
    const uint32_t tile_n = (n - base) < (uint32_t)kSortTile ? (n - base) : (uint32_t)kSortTile;
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        const uint32_t s = tid + i * kSortBlock;
        if (s < tile_n) {
            const uint64_t key = S.keys[s];
            const uint32_t dst = S.global_base[(uint32_t)(key >> shift) & 0xffu] + s;
            kout[dst] = key;
            vout[dst] = S.vals[s];
        }
    }
}

}  // namespace

void RadixSortPlan::prepare(uint32_t n, int bits) {
    passes = (bits + 7) / 8;
    if (passes & 1) ++passes;  // even pass count: the result lands in the input buffers
    if (passes > kSortMaxPasses) passes = kSortMaxPasses;
    tiles = (n + kSortTile - 1) / kSortTile;
    if (tiles == 0) tiles = 1;
    keys_alt.ensure(n);
    vals_alt.ensure(n);
    hist.ensure((size_t)passes * 256);
    lookback.ensure((size_t)passes * tiles * 256);
    tile_ctr.ensure(passes);
}

void radix_sort_pairs(RadixSortPlan& plan, uint64_t* keys, uint32_t* vals, uint32_t n, int bits,
                      bool hist_ready, uint32_t* d_status, cudaStream_t stream) {
    if (n >= (1u << 30)) throw std::invalid_argument("radix_sort_pairs: n must be < 2^30");
    if (n <= 1) return;
    if (plan.tiles != (n + kSortTile - 1) / kSortTile || plan.keys_alt.cap < n) plan.prepare(n, bits);
    const int passes = plan.passes;
    SB_CUDA(cudaMemsetAsync(plan.lookback.ptr, 0, sizeof(uint32_t) * (size_t)passes * plan.tiles * 256, stream));
    SB_CUDA(cudaMemsetAsync(plan.tile_ctr.ptr, 0, sizeof(uint32_t) * passes, stream));
    if (!hist_ready) {
        SB_CUDA(cudaMemsetAsync(plan.hist.ptr, 0, sizeof(uint32_t) * passes * 256, stream));
        int grid = grid_for(n, 256 * 16);
        if (grid > 4 * kNumSMs) grid = 4 * kNumSMs;
        k_hist<<<grid, 256, 0, stream>>>(keys, n, passes, plan.hist.ptr);
        SB_LAUNCH_CHECK();
    }
    k_hist_scan<<<passes, 256, 0, stream>>>(plan.hist.ptr);
    SB_LAUNCH_CHECK();
    static std::atomic<uint64_t> attr_set{0};  // one bit per device
    const size_t smem = sizeof(SortSmem);
    if (once_per_device(attr_set))
        SB_CUDA(cudaFuncSetAttribute(k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    uint64_t *ka = keys, *kb = plan.keys_alt.ptr;
    uint32_t *va = vals, *vb = plan.vals_alt.ptr;
    for (int p = 0; p < passes; ++p) {
        k_onesweep<<<plan.tiles, kSortBlock, smem, stream>>>(
            ka, va, kb, vb, n, 8 * p, plan.hist.ptr + p * 256, plan.lookback.ptr + (size_t)p * plan.tiles * 256,
            plan.tile_ctr.ptr + p, d_status);
        SB_LAUNCH_CHECK();
        std::swap(ka, kb);
        std::swap(va, vb);
    }
}

}  // namespace sb
