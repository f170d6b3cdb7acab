// ibp_noalloc.cu -- decompress_fetch for callers that cannot allocate device memory.
//
// Every other entry point asks the caller for device scratch (the *_workspace_size()
// functions).  Some callers cannot provide it: a host framework that owns all device memory
// and offers no allocation hook, an embedding that runs under an allocator policy which
// forbids cudaMalloc on the request path, or code that must not make the implicit device
// synchronisation a cudaMalloc/cudaFree can cause.  ibp_decompress_fetch_noalloc serves them
// from a scratch array that this library reserves statically in device memory.
//
// The scratch is the file-scope array below (kNoAllocScratchBytes, 4 MiB); every device that
// loads the library keeps it until the process exits.  Host code must not pass the array's
// name to a kernel (on the host it names a host-side stand-in, not device memory): the first
// call on each device looks up the array's device address with cudaGetSymbolAddress, with
// that device current, and caches it.  That first call should therefore come before any
// stream capture on that device.  All calls share the one array, which keeps whatever the
// last call left in it; the fetch path rewrites every byte it reads (status word, column
// tables, sort buffers) before use, so nothing is carried over between calls.  Calls whose
// GPU work overlaps -- on different streams or from different threads -- race on the array
// and must be serialised by the caller.
#include <mutex>

#include "ibp_internal.cuh"

namespace ibp200 {

constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static ibp_status noalloc_scratch(void **out) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static void *addr[kMaxDevices] = {};
    int dev = 0;
    IBP_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("decompress_fetch_noalloc: device %d is beyond the %d this library tracks", dev,
                  kMaxDevices);
        return IBP_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> g(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error("decompress_fetch_noalloc: cudaGetSymbolAddress of the static scratch "
                      "failed: %s", cudaGetErrorString(e));
            return IBP_ERR_CUDA;
        }
        addr[dev] = p;
    }
    *out = addr[dev];
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

}  // extern "C"
