// Shared infrastructure of the stream_b200 CUDA library (sm_100a only).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace sb {

// Status bits recorded by kernels in a device word and surfaced through the
// C ABI (*_get_status).  Bounded device loops set a bit and return instead of
// spinning or faulting.
enum StatusBits : uint32_t {
    ST_OK = 0,
    ST_STACK_OVERFLOW = 1u << 0,   // BVH traversal stack exhausted
    ST_WALK_CAP = 1u << 1,         // cavity boundary walk reached its 100-step cap (reference behaviour)
    ST_BROKEN_CYCLE = 1u << 2,     // cavity boundary cycle not closed
    ST_TET_CAP = 1u << 3,          // local tet list overflow
    ST_EXACT_OVERFLOW = 1u << 4,   // exact-arithmetic expansion longer than its buffer
    ST_LOOKBACK_TIMEOUT = 1u << 5, // decoupled look-back gave up waiting (sort/scan)
    ST_TRUNCATED = 1u << 6,        // some star had more than 124 candidate neighbours
    ST_BAD_INPUT = 1u << 7,        // invalid argument (rejected on the host; non-finite device input flagged)
    ST_CUDA_ERROR = 1u << 8,       // a CUDA runtime call failed
    ST_INCOMPLETE = 1u << 9,       // a 2D Delaunay star still unverified after Mesh2D_insert_iterative
};

struct CudaError : std::runtime_error {
    explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};

inline void check(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        char buf[512];
        snprintf(buf, sizeof buf, "%s failed at %s:%d: %s", what, file, line, cudaGetErrorString(e));
        throw CudaError(buf);
    }
}
// Host-side count of kernel launches issued by the library (every launch site
// is followed by SB_LAUNCH_CHECK).
void count_launch();
void count_launches(uint32_t k);
#define SB_CUDA(x) ::sb::check((x), #x, __FILE__, __LINE__)
#define SB_LAUNCH_CHECK() (::sb::count_launch(), ::sb::check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__))

// Growable device buffer; contents are not preserved across growth.
template <typename T>
struct DeviceBuffer {
    T* ptr = nullptr;
    size_t cap = 0;   // elements
    size_t size = 0;  // elements in use

    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { release(); }

    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = size = 0;
    }
    // Ensure room for n elements (n may be 0).  Growth keeps 25% slack so
    // that sizes creeping up from call to call (a remesh per step) do not
    // reallocate (cudaFree synchronises the device) every time.
    T* ensure(size_t n) {
        if (n > cap) {
            const size_t grown = cap ? cap + cap / 4 : 0;
            release();
            size_t want = n < 16 ? 16 : (n > grown ? n : grown);
            SB_CUDA(cudaMalloc(&ptr, want * sizeof(T)));
            cap = want;
        }
        size = n;
        return ptr;
    }
    T* data() const { return ptr; }
};

// Pinned host scratch for small device->host reads.
struct PinnedWords {
    uint32_t* h = nullptr;
    PinnedWords() { SB_CUDA(cudaMallocHost(&h, 64 * sizeof(uint32_t))); }
    ~PinnedWords() { if (h) cudaFreeHost(h); }
    PinnedWords(const PinnedWords&) = delete;
    PinnedWords& operator=(const PinnedWords&) = delete;
};

// True the first time it is called for the current device with this flag
// word (per-device set-up such as cudaFuncSetAttribute, which is a property of
// each device's context); also true when the device cannot be determined.
inline bool once_per_device(std::atomic<uint64_t>& done) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return true;
    }
    const uint64_t bit = 1ull << dev;
    return (done.fetch_or(bit) & bit) == 0;
}

// True when none of the m floats is an infinity or a NaN (exponent field all
// ones): an integer scan the host compiler vectorises.
// True when any of the m device floats d is infinite or NaN: one pass on the
// GPU over the data where it already is (a host loop costs about 10 ms per
// 80 MB).  *flag is a device word (cleared here), *pinned a page-locked host
// word for the result; waits for the stream.
bool any_nonfinite(const float* d, size_t m, uint32_t* flag, uint32_t* pinned, cudaStream_t s);

constexpr int kNumSMs = 148;  // B200

// Bottom-up tree passes (a node's second arriving child combines both
// subtrees): the arrival counter is bumped with one acquire-release atomic,
// whose release half publishes this thread's stores of its child (box,
// ranges, parent) and whose acquire half makes the sibling's stores visible
// before they are read -- no separate fences (two fence.sc per level cost
// 20-24% of the fit and Apetrei passes).
__device__ __forceinline__ uint32_t atom_or_acq_rel(uint32_t* p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.or.b32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ uint32_t atom_add_acq_rel(uint32_t* p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

inline int grid_for(size_t n, int block) {
    size_t g = (n + block - 1) / block;
    return (int)(g == 0 ? 1 : g);
}

}  // namespace sb
