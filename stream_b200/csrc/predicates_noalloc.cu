// Conflict-predicate batch for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a host program that hands this library
// only the device buffers it already owns and forbids new allocations (a fixed
// memory budget, or a pool it manages itself), or a plugin loaded into such a
// host.  For them this file offers the star kernel's exact conflict decision
// (the same three stages as stream_b200_conflict_batch) on device arrays the
// caller provides, with the exact stage's scratch in a fixed file-scope device
// array instead of a per-call allocation.
//
// Limits and sharing: at most kNoAllocMaxQuintuples quintuples per call
// (larger batches are rejected; split them).  The scratch array (3.3 MiB) is
// created in every GPU that loads this library and kept until the process
// exits.  All calls share it, and it keeps the previous call's contents: the
// status word that must start at zero is cleared on every call, and calls
// whose work overlaps on the GPU (for example from two streams at once) race
// on the scratch and must not be issued.  The call waits for its own work
// (it copies the status word back and synchronises the stream) before it
// returns.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address (cudaGetSymbolAddress) and caches it for the
// process; make that first call before any stream capture.  The cached address
// belongs to the device's primary context: after cudaDeviceReset on a device,
// this entry point must not be called again on it in the same process.
#include <mutex>

#include "capi_common.cuh"
#include "predicates.cuh"
#include "stream_b200.h"

namespace {

constexpr uint32_t kNoAllocMaxQuintuples = 256;

__device__ __align__(256) float g_noalloc_scratch[kNoAllocMaxQuintuples * sb::pred::kInsphereScratchFloats];
__device__ __align__(256) uint32_t g_noalloc_status[4];

// Device addresses of the two arrays, per device (host code may not use the
// symbols themselves as addresses).
struct NoAllocSlots {
    float* scratch = nullptr;
    uint32_t* status = nullptr;
};
constexpr int kMaxDevices = 64;
NoAllocSlots g_slots[kMaxDevices];
std::mutex g_slots_mu;

// Set-up, once per device, with that device current.
int slots_for_current_device(NoAllocSlots& out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        sb::last_error_text() = "conflict_batch_noalloc: no usable current device";
        return (int)sb::ST_CUDA_ERROR;
    }
    std::lock_guard<std::mutex> lk(g_slots_mu);
    NoAllocSlots& s = g_slots[dev];
    if (!s.scratch) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            sb::last_error_text() = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e);
            cudaGetLastError();
            return (int)sb::ST_CUDA_ERROR;
        }
        void* q = nullptr;
        e = cudaGetSymbolAddress(&q, g_noalloc_status);
        if (e != cudaSuccess) {
            sb::last_error_text() = std::string("cudaGetSymbolAddress(status): ") + cudaGetErrorString(e);
            cudaGetLastError();
            return (int)sb::ST_CUDA_ERROR;
        }
        s.scratch = static_cast<float*>(p);
        s.status = static_cast<uint32_t*>(q);
    }
    out = s;
    return 0;
}

__global__ void __launch_bounds__(64) k_conflict_batch_noalloc(uint32_t m, const float* __restrict__ pts,
                                                               const uint32_t* __restrict__ ids, float* __restrict__ out,
                                                               float* scratch, uint32_t* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    float3 p[5];
    uint32_t id[5];
    for (int k = 0; k < 5; ++k) {
        p[k] = make_float3(pts[15 * (size_t)i + 3 * k], pts[15 * (size_t)i + 3 * k + 1], pts[15 * (size_t)i + 3 * k + 2]);
        id[k] = ids[5 * (size_t)i + k];
    }
    uint32_t st = 0, nex = 0;
    bool need;
    out[i] = sb::pred::conflict_det(p, id, scratch + (size_t)i * sb::pred::kInsphereScratchFloats, need, st, nex);
    if (st) atomicOr(status, st);
}

}  // namespace

extern "C" {

// See stream_b200.h.  d_pts (m x 5 x 3 floats), d_ids (m x 5) and d_out (m)
// are device arrays owned by the caller; stream may be NULL (default stream).
SB_EXPORT int stream_b200_conflict_batch_noalloc(uint32_t m, const float* d_pts, const uint32_t* d_ids, float* d_out,
                                                 void* stream) {
    if (m == 0) return 0;
    if (m > kNoAllocMaxQuintuples) {
        sb::last_error_text() = "conflict_batch_noalloc: at most 256 quintuples per call";
        return (int)sb::ST_BAD_INPUT;
    }
    if (!d_pts || !d_ids || !d_out) {
        sb::last_error_text() = "conflict_batch_noalloc: null device array";
        return (int)sb::ST_BAD_INPUT;
    }
    NoAllocSlots s;
    if (int rc = slots_for_current_device(s)) return rc;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(s.status, 0, sizeof(uint32_t), cs);
    if (e == cudaSuccess) {
        k_conflict_batch_noalloc<<<(m + 63) / 64, 64, 0, cs>>>(m, d_pts, d_ids, d_out, s.scratch, s.status);
        e = cudaGetLastError();
    }
    uint32_t st = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&st, s.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    if (e != cudaSuccess) {
        sb::last_error_text() = std::string("conflict_batch_noalloc: ") + cudaGetErrorString(e);
        return (int)sb::ST_CUDA_ERROR;
    }
    sb::count_launch();
    return (int)st;
}

}  // extern "C"
