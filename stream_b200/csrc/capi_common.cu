// Library-wide extern "C" entry points.
#include <algorithm>
#include <atomic>

#include "capi_common.cuh"
#include "stream_b200.h"

namespace sb {
std::string& last_error_text() {
    thread_local std::string s;
    return s;
}
namespace {
__global__ void k_nonfinite(const float* __restrict__ v, size_t m, uint32_t* bad) {
    uint32_t b = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
        b |= (__float_as_uint(v[i]) & 0x7f800000u) == 0x7f800000u;  // exponent bits all set
    if (__any_sync(0xffffffffu, b) && (threadIdx.x & 31) == 0) atomicOr(bad, 1u);
}
}  // namespace

bool any_nonfinite(const float* d, size_t m, uint32_t* flag, uint32_t* pinned, cudaStream_t s) {
    SB_CUDA(cudaMemsetAsync(flag, 0, sizeof(uint32_t), s));
    if (m) {
        const size_t blocks = std::min<size_t>((m + 255) / 256, (size_t)kNumSMs * 8);
        k_nonfinite<<<(unsigned)blocks, 256, 0, s>>>(d, m, flag);
        SB_LAUNCH_CHECK();
    }
    SB_CUDA(cudaMemcpyAsync(pinned, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    return *pinned != 0;
}

static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(uint32_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
}  // namespace sb

extern "C" {

// Message of the last failure seen by this thread at the C boundary ("" if none).
SB_EXPORT const char* stream_b200_last_error(void) { return sb::last_error_text().c_str(); }

// 1 when a CUDA device of compute capability 10.0 is visible, 0 otherwise.
SB_EXPORT int stream_b200_device_ok(void) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return 0; }
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) { cudaGetLastError(); return 0; }
    return (p.major == 10 && p.minor == 0) ? 1 : 0;
}

// Kernel launches issued by this library since load (all handles, all threads).
SB_EXPORT unsigned long long stream_b200_launch_count(void) { return sb::g_launches.load(); }

}  // extern "C"
