// ibp_common.cuh -- shared plumbing of the B200 IBP engine: error reporting, word helpers,
// workspace carving and launch geometry.  Everything here is internal to libibp_b200.so.
#pragma once

#include <nvtx3/nvToolsExt.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "ibp_b200.h"

namespace ibp200 {

// ------------------------------------------------------------------ errors
void set_error(const char *fmt, ...);
void clear_error();
extern bool g_debug;
extern std::atomic<unsigned long long> g_launches;  // engine kernels launched so far

// Optional CUDA events around row-fetch kernel launches (benchmark profiling hook):
// profile_begin returns a slot (or -1 when profiling is off or full), profile_end closes it.
// NVTX range around an entry point (visible in Nsight timelines; near-free without a tool).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};
#define IBP_RANGE(name) ::ibp200::NvtxRange ibp_nvtx_range_(name)

int profile_begin(cudaStream_t st);
int fetch_dedup_mode();  // ibp_set_fetch_dedup: 0 auto, 1 sort, 2 hash
int repeat_wait_polls();  // ibp_set_repeat_wait_limit
void profile_end(int slot, cudaStream_t st);

#define IBP_DPRINTF(...)                       \
    do {                                       \
        if (::ibp200::g_debug) printf(__VA_ARGS__); \
    } while (0)

#define IBP_ARG(cond, ...)                          \
    do {                                            \
        if (!(cond)) {                              \
            ::ibp200::set_error(__VA_ARGS__);       \
            return IBP_ERR_ARGUMENT;                \
        }                                           \
    } while (0)

#define IBP_CUDA(expr)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (expr);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            ::ibp200::set_error("%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, \
                                __LINE__);                                              \
            return IBP_ERR_CUDA;                                                        \
        }                                                                               \
    } while (0)

#define IBP_LAUNCHED(name)                                                              \
    do {                                                                                \
        ::ibp200::g_launches.fetch_add(1, std::memory_order_relaxed);                   \
        cudaError_t e_ = cudaGetLastError();                                            \
        if (e_ != cudaSuccess) {                                                        \
            ::ibp200::set_error("launch of %s failed: %s", name, cudaGetErrorString(e_)); \
            return IBP_ERR_CUDA;                                                        \
        }                                                                               \
    } while (0)

#define IBP_RET(expr)                      \
    do {                                   \
        ibp_status s_ = (expr);            \
        if (s_ != IBP_OK) return s_;       \
    } while (0)

// ------------------------------------------------------------------ sizes
constexpr size_t kAlign = 256;          // every workspace carve starts 256-byte aligned
constexpr size_t kStatusBytes = 256;    // head of every workspace: device status word(s)
constexpr int32_t kStatusBadIndex = 1;    // bit 0: an index was out of range
constexpr int32_t kStatusCorruptRow = 2;  // bit 1: a row's bitmap does not fit its mask
constexpr int32_t kStatusBadTable = 4;    // bit 2: request counts disagree with a stated total
constexpr int32_t kStatusWaitTimeout = 8;  // bit 3: a repeat gave up waiting for its first row

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Carves 256-byte aligned sub-buffers out of a caller workspace.
struct Carver {
    char *base;
    size_t used;
    size_t cap;
    template <typename T>
    T *take(size_t count) {
        size_t off = align_up(used, kAlign);
        used = off + count * sizeof(T);
        return (used <= cap && base) ? reinterpret_cast<T *>(base + off) : nullptr;
    }
};

// Size accounting twin of Carver.
struct Sizer {
    size_t used = 0;
    template <typename T>
    void take(size_t count) { used = align_up(used, kAlign) + count * sizeof(T); }
    size_t total() const { return align_up(used, kAlign); }
};

// Programmatic dependent launch.  A kernel launched by launch_dependent() may start while the
// kernel before it on the stream is still running: it may read only inputs of the call and
// its own shared memory until grid_dep_wait() returns, which happens once that kernel has
// completed and its writes are visible (at once for a kernel launched normally).
// grid_dep_release() lets the next such kernel start; a kernel calls it after its own wait,
// so that the kernel after it never starts before the one before it has completed.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_release() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_dependent(void (*kern)(KArgs...), unsigned grid, unsigned block,
                                    size_t smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
    if (e == cudaErrorNotSupported) {
        // no programmatic launches here: an ordinary launch (the waits then return at once)
        (void)cudaGetLastError();
        cfg.numAttrs = 0;
        e = cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
    }
    return e;
}

int device_sm_count();        // SMs of the current device (cached per device)
int device_max_smem_optin();  // opt-in shared memory per block (cached per device)
// Resident blocks per SM (at least 1) of a kernel launched with `threads` and `smem` bytes of
// dynamic shared memory on the current device, after raising the kernel's dynamic
// shared-memory limit to `smem` when needed; cached per device, kernel and shape.
ibp_status kernel_blocks_per_sm(const void *kern, int threads, size_t smem, int *per_sm);

// ------------------------------------------------------------------ word helpers
template <typename U>
struct WordBits { static constexpr int value = 8 * sizeof(U); };

template <typename U>
__device__ __forceinline__ int popc_w(U x) {
    if constexpr (sizeof(U) == 8)
        return __popcll((unsigned long long)x);
    else
        return __popc((unsigned)x);
}

template <typename U>
__device__ __forceinline__ int clz_w(U x) {
    if constexpr (sizeof(U) == 8)
        return __clzll((long long)x);
    else if constexpr (sizeof(U) == 4)
        return __clz((int)x);
    else
        return __clz((int)(unsigned)x) - (32 - 8 * (int)sizeof(U));
}

// Bytes of the per-row compressed-word bitmap (one bit per word, padded to whole words):
// include/compress/ibp_compress_dev.cuh:12-15.
__host__ __device__ inline int64_t meta_bytes(int64_t v, int wb) {
    return ((v + 7) / 8 + wb - 1) / wb * wb;
}

// Compressed row bytes from the saved-bit count s: include/misc/ibp_misc_dev.cuh:19-46.
// The row is stored compressed only when this is strictly below v * wb.
__host__ __device__ inline int64_t compressed_bytes(int64_t v, int wb, uint64_t s) {
    const int64_t vb = v * wb;
    int64_t data = vb - (int64_t)(s / 8);
    data = (data + wb - 1) / wb * wb;
    int64_t sz = meta_bytes(v, wb) + data;
    return sz < vb ? sz : vb;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// Sum over the lanes of aligned groups of G lanes (G a power of two <= 32).
template <int G, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace ibp200
