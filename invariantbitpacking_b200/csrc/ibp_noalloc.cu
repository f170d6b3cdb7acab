// ibp_noalloc.cu -- decompress_fetch for callers that cannot allocate device memory.
//
// Every other entry point asks the caller for device scratch (the *_workspace_size()
// functions).  Some callers cannot provide it: a host framework that owns all device memory
// and offers no allocation hook, an embedding that runs under an allocator policy which
// forbids cudaMalloc on the request path, or code that must not make the implicit device
// synchronisation a cudaMalloc/cudaFree can cause.  ibp_decompress_fetch_noalloc serves them
// from a scratch array that this library reserves statically in device memory.
//
// The scratch is the file-scope array below (IBP_NOALLOC_SCRATCH_BYTES, 4 MiB); every device
// that loads the library keeps it until the process exits.  Host code must not pass the
// array's name to a kernel (on the host it names a host-side stand-in, not device memory):
// the first call in each CUDA context looks up the array's device address with
// cudaGetSymbolAddress, with that context's device current, and caches it with the context's
// unique id; a later call in another context of the device (after cudaDeviceReset, say, when
// the module is loaded again and the array may move) looks it up again.  That first call
// should therefore come before any stream capture on that device.  All calls share the one
// array, which keeps whatever the last call left in it; the fetch path rewrites every byte it
// reads (status word, column tables, sort buffers) before use, so nothing is carried over
// between calls.  Calls whose GPU work overlaps -- on different streams or from different
// threads -- race on the array and must be serialised by the caller.  The status word of the
// last call is the array's first 4 bytes (ibp_decompress_fetch_noalloc_status).
#include <cuda.h>  // driver types for cuCtxGetCurrent / cuCtxGetId (no libcuda link)

#include <mutex>

#include "ibp_internal.cuh"

namespace ibp200 {

constexpr size_t kNoAllocScratchBytes = IBP_NOALLOC_SCRATCH_BYTES;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Unique id of the calling thread's current CUDA context (0 when none is current or the
// driver does not provide the query).  Ids are never reused within a process, so a cached
// address tagged with one cannot outlive its context unnoticed.
static unsigned long long current_context_id() {
    typedef CUresult (*GetCurrent)(CUcontext *);
    typedef CUresult (*GetId)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void **)&get_current, cudaEnableDefault,
                                    &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
            get_current = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", (void **)&get_id, cudaEnableDefault, &q) !=
                cudaSuccess || q != cudaDriverEntryPointSuccess)
            get_id = nullptr;
        cudaGetLastError();
    });
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the static scratch in the current device's context.
static ibp_status noalloc_scratch(void **out) {
    constexpr int kMaxDevices = 64;
    struct Entry {
        unsigned long long ctx;
        void *addr;
    };
    static std::mutex mu;
    static Entry cache[kMaxDevices] = {};
    int dev = 0;
    IBP_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("decompress_fetch_noalloc: device %d is beyond the %d this library tracks", dev,
                  kMaxDevices);
        return IBP_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> g(mu);
    const unsigned long long ctx = current_context_id();
    if (!cache[dev].addr || ctx == 0 || ctx != cache[dev].ctx) {
        void *p = nullptr;
        // also makes the device's primary context current on this thread if it was not
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error("decompress_fetch_noalloc: cudaGetSymbolAddress of the static scratch "
                      "failed: %s", cudaGetErrorString(e));
            return IBP_ERR_CUDA;
        }
        cache[dev].addr = p;
        cache[dev].ctx = current_context_id();  // 0 (no id available): look up every call
    }
    *out = cache[dev].addr;
    return IBP_OK;
}

}  // namespace ibp200

using namespace ibp200;

extern "C" {

ibp_status ibp_decompress_fetch_noalloc(const void *comp, int64_t num_vecs, int64_t vec_size,
                                        int word_bytes, const void *mask, const void *bitval,
                                        const int32_t *bitmask, const int64_t *index,
                                        int64_t num_index, int32_t comp_len, void *out,
                                        ibp_stream_t stream) {
    clear_error();
    if (word_bytes != 4 && word_bytes != 8) {
        set_error("decompress_fetch_noalloc: Input tensor must be 4-byte or 8-byte datatype");
        return IBP_ERR_ARGUMENT;
    }
    if (num_vecs < 0 || vec_size < 0) {
        set_error("decompress_fetch_noalloc: negative shape (%lld x %lld)", (long long)num_vecs,
                  (long long)vec_size);
        return IBP_ERR_ARGUMENT;
    }
    const size_t need = decompress_workspace(num_index, vec_size, word_bytes, num_index >= 0);
    if (need > kNoAllocScratchBytes) {
        set_error("decompress_fetch_noalloc: this call needs %zu bytes of scratch but the static "
                  "scratch holds %zu (fewer index entries or shorter rows fit; "
                  "ibp_decompress_fetch takes caller scratch of any size)",
                  need, kNoAllocScratchBytes);
        return IBP_ERR_WORKSPACE;
    }
    void *scratch = nullptr;
    IBP_RET(noalloc_scratch(&scratch));
    return ibp_decompress_fetch(comp, num_vecs, vec_size, word_bytes, mask, bitval, bitmask, index,
                                num_index, comp_len, out, -1, -1, -1, scratch,
                                kNoAllocScratchBytes, stream);
}

ibp_status ibp_decompress_fetch_noalloc_status(int32_t *status, ibp_stream_t stream) {
    clear_error();
    IBP_ARG(status, "decompress_fetch_noalloc_status: null pointer");
    void *scratch = nullptr;
    IBP_RET(noalloc_scratch(&scratch));
    return ibp_read_status(scratch, status, stream);
}

}  // extern "C"
