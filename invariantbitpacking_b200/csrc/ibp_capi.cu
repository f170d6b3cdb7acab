// ibp_capi.cu -- the extern "C" boundary of libibp_b200.so (declared in include/ibp_b200.h):
// argument checks, word-size dispatch, workspace sizing and error reporting.  Every entry
// point replaces one function of the reference extension `ibp_cuda`
// (src/ibp_api.cu:124-135); none allocates device memory or calls exit().
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "ibp_codec.cuh"
#include "ibp_internal.cuh"

namespace ibp200 {

static thread_local std::string g_err;
bool g_debug = false;
std::atomic<unsigned long long> g_launches{0};

struct Profiler {
    std::mutex mu;
    int cap = 0, used = 0;
    std::vector<cudaEvent_t> ev;  // 2 per slot
};
static Profiler &profiler() {
    static Profiler p;
    return p;
}

static std::atomic<int> g_dedup_mode{0};
int fetch_dedup_mode() { return g_dedup_mode.load(std::memory_order_relaxed); }

constexpr int kDefaultRepeatWaitPolls = 1 << 20;  // ~0.25 s of polls 0.25 us apart
static std::atomic<int> g_repeat_wait_polls{kDefaultRepeatWaitPolls};
int repeat_wait_polls() { return g_repeat_wait_polls.load(std::memory_order_relaxed); }

int profile_begin(cudaStream_t st) {
    Profiler &p = profiler();
    std::lock_guard<std::mutex> g(p.mu);
    if (p.used >= p.cap) return -1;
    const int slot = p.used++;
    cudaEventRecord(p.ev[2 * slot], st);
    return slot;
}

void profile_end(int slot, cudaStream_t st) {
    if (slot < 0) return;
    Profiler &p = profiler();
    std::lock_guard<std::mutex> g(p.mu);
    cudaEventRecord(p.ev[2 * slot + 1], st);
}

void set_error(const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    IBP_DPRINTF("[ibp] error: %s\n", buf);
}

void clear_error() { g_err.clear(); }

struct DevInfo {
    int sms = 0;
    int smem_optin = 0;
};

static DevInfo &dev_info() {
    static std::mutex mu;
    static std::vector<DevInfo> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> g(mu);
    if ((int)cache.size() <= dev) cache.resize(dev + 1);
    DevInfo &d = cache[dev];
    if (d.sms == 0) {
        cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (d.sms <= 0) d.sms = 148;
        if (d.smem_optin <= 0) d.smem_optin = 48 * 1024;
    }
    return d;
}

int device_sm_count() { return dev_info().sms; }
int device_max_smem_optin() { return dev_info().smem_optin; }

// Per device and kernel: the dynamic shared-memory limit set so far, and the resident blocks
// per SM of each launch shape asked for (a per-call fetch of a few thousand rows spends
// microseconds of host time on these queries otherwise).
ibp_status kernel_blocks_per_sm(const void *kern, int threads, size_t smem, int *per_sm) {
    struct Shape {
        int dev;
        const void *kern;
        int threads;
        size_t smem;
        int per_sm;
    };
    struct Limit {
        int dev;
        const void *kern;
        size_t smem;
    };
    static std::mutex mu;
    static std::vector<Shape> shapes;
    static std::vector<Limit> limits;
    int dev = 0;
    IBP_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(mu);
    for (const Shape &s : shapes)
        if (s.dev == dev && s.kern == kern && s.threads == threads && s.smem == smem) {
            *per_sm = s.per_sm;
            return IBP_OK;
        }
    Limit *lim = nullptr;
    for (Limit &l : limits)
        if (l.dev == dev && l.kern == kern) lim = &l;
    if (!lim) {
        limits.push_back({dev, kern, 48 * 1024});
        lim = &limits.back();
    }
    if (smem > lim->smem) {
        IBP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        lim->smem = smem;
    }
    int n = 0;
    IBP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem));
    if (n < 1) n = 1;
    shapes.push_back({dev, kern, threads, smem, n});
    *per_sm = n;
    return IBP_OK;
}

static bool on_host(const void *p) {
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged;
}

// Device memory, managed memory or page-locked (registered/mapped) host memory: what a kernel
// may dereference.  Pageable host memory is rejected before any launch.
static bool gpu_accessible(const void *p) {
    if (!p) return true;
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return pa.type != cudaMemoryTypeUnregistered;
}

#define IBP_ACCESSIBLE(ptr, what, name)                                                        \
    IBP_ARG(gpu_accessible(ptr), "%s: %s must be device memory or pinned host memory", what, \
            name)

static ibp_status check_rows(const void *p, int64_t n, int64_t v, int wb, bool codec,
                             const char *what) {
    IBP_ARG(n >= 0 && v >= 0, "%s: negative shape (%lld x %lld)", what, (long long)n,
            (long long)v);
    if (codec)
        IBP_ARG(wb == 4 || wb == 8, "%s: Input tensor must be 4-byte or 8-byte datatype", what);
    else
        IBP_ARG(wb == 1 || wb == 2 || wb == 4 || wb == 8,
                "%s: Input tensor must be 1, 2, 4, or 8-byte datatype", what);
    IBP_ARG(p != nullptr || n * v == 0, "%s: null dataset pointer", what);
    if (n * v > 0) IBP_ACCESSIBLE(p, what, "the dataset");
    return IBP_OK;
}

size_t compress_inplace_workspace(int64_t nidx, int64_t v, int wb, bool has_index) {
    Sizer s;
    s.take<char>(kStatusBytes);
    s.take<char>(wb == 8 ? tables_bytes<uint64_t>(v) : tables_bytes<uint32_t>(v));
    if (has_index) s.take<char>((size_t)(nidx * v * wb));
    return s.total();
}

template <typename U>
static ibp_status compress_inplace_t(U *data, int64_t n, int64_t v, const U *mask,
                                     const U *bitval, const int64_t *index, int64_t nidx,
                                     bool has_index, int32_t *bitmask, void *ws, size_t ws_bytes,
                                     cudaStream_t st) {
    const int64_t nrows = has_index ? nidx : n;
    const size_t need = compress_inplace_workspace(nidx, v, sizeof(U), has_index);
    if (!ws || ws_bytes < need) {
        set_error("compress_inplace: workspace of %zu bytes is below the required %zu", ws_bytes,
                  need);
        return IBP_ERR_WORKSPACE;
    }
    Carver c{(char *)ws, 0, ws_bytes};
    int32_t *status = c.take<int32_t>(kStatusBytes / 4);
    ColTables<U> t = carve_tables<U>(c, v);
    IBP_CUDA(cudaMemsetAsync(status, 0, sizeof(int32_t), st));
    if (v > 0) IBP_RET(build_tables<U>(mask, bitval, v, t, st));
    if (has_index) {
        // every source row is read before any row is overwritten
        U *stage = c.take<U>((size_t)(nidx * v));
        IBP_RET(gather_rows_impl<U>(data, n, v, index, nidx, stage, status, st));
        return compress_rows_impl<U>(stage, nidx, v, t, nullptr, nidx, data, false, bitmask,
                                     status, st);
    }
    return compress_rows_impl<U>(data, n, v, t, nullptr, nrows, data, true, bitmask, status, st);
}

}  // namespace ibp200

using namespace ibp200;

extern "C" {

const char *ibp_last_error(void) { return g_err.c_str(); }

int ibp_abi_version(void) { return 1; }

void ibp_set_debug(int on) { g_debug = on != 0; }

ibp_status ibp_set_fetch_dedup(int32_t mode) {
    clear_error();
    IBP_ARG(mode >= 0 && mode <= 2, "set_fetch_dedup: mode must be 0 (auto), 1 (sort) or 2 (hash)");
    g_dedup_mode.store(mode);
    return IBP_OK;
}

ibp_status ibp_set_repeat_wait_limit(int32_t polls) {
    clear_error();
    IBP_ARG(polls >= -1, "set_repeat_wait_limit: polls must be >= 0, or -1 for the default");
    g_repeat_wait_polls.store(polls < 0 ? kDefaultRepeatWaitPolls : polls);
    return IBP_OK;
}

ibp_status ibp_profile_enable(int32_t capacity) {
    clear_error();
    Profiler &p = profiler();
    std::lock_guard<std::mutex> g(p.mu);
    IBP_ARG(capacity >= 0 && capacity <= (1 << 20), "profile_enable: bad capacity %d", capacity);
    while ((int)p.ev.size() < 2 * capacity) {
        cudaEvent_t e;
        IBP_CUDA(cudaEventCreate(&e));
        p.ev.push_back(e);
    }
    p.cap = capacity;
    p.used = 0;
    return IBP_OK;
}

int32_t ibp_profile_take(float *ms, int32_t capacity) {
    Profiler &p = profiler();
    std::lock_guard<std::mutex> g(p.mu);
    const int n = p.used < capacity ? p.used : capacity;
    for (int i = 0; i < n; ++i) {
        ms[i] = -1.0f;
        if (cudaEventSynchronize(p.ev[2 * i + 1]) == cudaSuccess)
            cudaEventElapsedTime(&ms[i], p.ev[2 * i], p.ev[2 * i + 1]);
    }
    cudaGetLastError();
    p.used = 0;
    p.cap = 0;
    return n;
}

unsigned long long ibp_kernel_launch_count(void) { return g_launches.load(); }

ibp_status ibp_read_status(const void *workspace, int32_t *status, ibp_stream_t stream) {
    clear_error();
    IBP_ARG(workspace && status, "ibp_read_status: null pointer");
    IBP_CUDA(cudaMemcpyAsync(status, workspace, sizeof(int32_t), cudaMemcpyDeviceToHost,
                             (cudaStream_t)stream));
    IBP_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return IBP_OK;
}

// ------------------------------------------------------------------ preprocess
size_t ibp_preprocess_workspace_size(int64_t num_vecs, int64_t vec_size, int word_bytes,
                                     float threshold) {
    return preprocess_workspace(num_vecs, vec_size, word_bytes, threshold, false);
}

ibp_status ibp_preprocess(const void *dataset, int64_t num_vecs, int64_t vec_size,
                          int word_bytes, float threshold, void *mask, void *bitval,
                          void *workspace, size_t workspace_bytes, ibp_stream_t stream) {
    clear_error();
    IBP_RANGE("ibp_preprocess");
    IBP_RET(check_rows(dataset, num_vecs, vec_size, word_bytes, false, "preprocess"));
    IBP_ARG((mask && bitval) || vec_size == 0, "preprocess: null mask/bitval");
    IBP_ACCESSIBLE(mask, "preprocess", "mask");
    IBP_ACCESSIBLE(bitval, "preprocess", "bitval");
    cudaStream_t st = (cudaStream_t)stream;
    const bool host = num_vecs * vec_size > 0 && on_host(dataset);
    switch (word_bytes) {
    case 1:
        return preprocess_impl<uint8_t>((const uint8_t *)dataset, num_vecs, vec_size, threshold,
                                        (uint8_t *)mask, (uint8_t *)bitval, workspace,
                                        workspace_bytes, host, st);
    case 2:
        return preprocess_impl<uint16_t>((const uint16_t *)dataset, num_vecs, vec_size, threshold,
                                         (uint16_t *)mask, (uint16_t *)bitval, workspace,
                                         workspace_bytes, host, st);
    case 4:
        return preprocess_impl<uint32_t>((const uint32_t *)dataset, num_vecs, vec_size, threshold,
                                         (uint32_t *)mask, (uint32_t *)bitval, workspace,
                                         workspace_bytes, host, st);
    default:
        return preprocess_impl<uint64_t>((const uint64_t *)dataset, num_vecs, vec_size, threshold,
                                         (uint64_t *)mask, (uint64_t *)bitval, workspace,
                                         workspace_bytes, host, st);
    }
}

// ------------------------------------------------------------------ preprocess_kmeans
size_t ibp_preprocess_kmeans_workspace_size(int64_t num_vecs, int64_t vec_size,
                                            int word_bytes, int32_t num_clusters) {
    return kmeans_workspace(num_vecs, vec_size, word_bytes, num_clusters);
}

ibp_status ibp_preprocess_kmeans(const void *dataset, int64_t num_vecs, int64_t vec_size,
                                 int word_bytes, int32_t num_clusters,
                                 const int64_t *init_rows, void *masks, void *bitvals,
                                 int32_t *clusters, void *workspace, size_t workspace_bytes,
                                 ibp_stream_t stream) {
    clear_error();
    IBP_RANGE("ibp_preprocess_kmeans");
    IBP_RET(check_rows(dataset, num_vecs, vec_size, word_bytes, true, "preprocess_kmeans"));
    IBP_ARG(num_clusters > 0, "preprocess_kmeans: num_clusters must be positive");
    IBP_ARG(masks && bitvals && (clusters || num_vecs == 0), "preprocess_kmeans: null output");
    IBP_ACCESSIBLE(masks, "preprocess_kmeans", "masks");
    IBP_ACCESSIBLE(bitvals, "preprocess_kmeans", "bitvals");
    IBP_ACCESSIBLE(clusters, "preprocess_kmeans", "clusters");
    std::vector<int64_t> init;
    const int64_t seeded = std::min<int64_t>(num_clusters, num_vecs);
    if (init_rows) {
        init.assign(init_rows, init_rows + seeded);
    } else {
        // include/preproc/ibp_preproc_host.cuh:176-188: std::random_shuffle over 0..n-1
        std::vector<int> indices((size_t)num_vecs);
        for (int64_t i = 0; i < num_vecs; ++i) indices[(size_t)i] = (int)i;
#pragma GCC diagnostic push
#pragma GCC diagnostic ignored "-Wdeprecated-declarations"
        std::random_shuffle(indices.begin(), indices.end());
#pragma GCC diagnostic pop
        init.resize((size_t)seeded);
        for (int64_t i = 0; i < seeded; ++i) init[(size_t)i] = indices[(size_t)i];
    }
    for (int64_t i = 1; i < seeded; ++i)
        IBP_ARG(init[i] >= 0 && init[i] < num_vecs, "preprocess_kmeans: seed row %lld out of range",
                (long long)init[i]);
    if (init.empty()) init.push_back(0);
    cudaStream_t st = (cudaStream_t)stream;
    if (word_bytes == 4)
        return kmeans_impl<uint32_t>((const uint32_t *)dataset, num_vecs, vec_size, num_clusters,
                                     init.data(), (uint32_t *)masks, (uint32_t *)bitvals,
                                     clusters, workspace, workspace_bytes, st);
    return kmeans_impl<uint64_t>((const uint64_t *)dataset, num_vecs, vec_size, num_clusters,
                                 init.data(), (uint64_t *)masks, (uint64_t *)bitvals, clusters,
                                 workspace, workspace_bytes, st);
}

// ------------------------------------------------------------------ get_compress_size
ibp_status ibp_get_compress_size(const void *dataset, int64_t num_vecs, int64_t vec_size,
                                 int word_bytes, const void *mask, const void *bitval,
                                 const int64_t *index, int64_t num_index, int64_t *sizes,
                                 int64_t *total, ibp_stream_t stream) {
    clear_error();
    IBP_RANGE("ibp_get_compress_size");
    IBP_RET(check_rows(dataset, num_vecs, vec_size, word_bytes, false, "get_compress_size"));
    if (num_index < 0) index = nullptr;
    const int64_t nrows = num_index >= 0 ? num_index : num_vecs;
    IBP_ARG(num_index <= 0 || index, "get_compress_size: null index array");
    IBP_ARG((mask && bitval) || vec_size == 0, "get_compress_size: null mask/bitval");
    IBP_ARG(sizes || nrows == 0, "get_compress_size: null sizes");
    IBP_ACCESSIBLE(mask, "get_compress_size", "mask");
    IBP_ACCESSIBLE(bitval, "get_compress_size", "bitval");
    IBP_ACCESSIBLE(index, "get_compress_size", "the index array");
    IBP_ACCESSIBLE(sizes, "get_compress_size", "sizes");
    IBP_ACCESSIBLE(total, "get_compress_size", "total");
    cudaStream_t st = (cudaStream_t)stream;
    // rows with an out-of-range index get size 0 (there is no workspace for a status word)
    int32_t *dummy = nullptr;
    switch (word_bytes) {
    case 1:
        return compress_size_impl<uint8_t>((const uint8_t *)dataset, num_vecs, vec_size,
                                           (const uint8_t *)mask, (const uint8_t *)bitval, index,
                                           nrows, sizes, total, dummy, st);
    case 2:
        return compress_size_impl<uint16_t>((const uint16_t *)dataset, num_vecs, vec_size,
                                            (const uint16_t *)mask, (const uint16_t *)bitval,
                                            index, nrows, sizes, total, dummy, st);
    case 4:
        return compress_size_impl<uint32_t>((const uint32_t *)dataset, num_vecs, vec_size,
                                            (const uint32_t *)mask, (const uint32_t *)bitval,
                                            index, nrows, sizes, total, dummy, st);
    default:
        return compress_size_impl<uint64_t>((const uint64_t *)dataset, num_vecs, vec_size,
                                            (const uint64_t *)mask, (const uint64_t *)bitval,
                                            index, nrows, sizes, total, dummy, st);
    }
}

// ------------------------------------------------------------------ compress_inplace
size_t ibp_compress_inplace_workspace_size(int64_t num_index, int64_t vec_size, int word_bytes,
                                           int has_index) {
    return compress_inplace_workspace(num_index, vec_size, word_bytes, has_index != 0);
}

ibp_status ibp_compress_inplace(void *dataset, int64_t num_vecs, int64_t vec_size,
                                int word_bytes, const void *mask, const void *bitval,
                                const int64_t *index, int64_t num_index, int32_t *bitmask,
                                void *workspace, size_t workspace_bytes, ibp_stream_t stream) {
    clear_error();
    IBP_RANGE("ibp_compress_inplace");
    IBP_RET(check_rows(dataset, num_vecs, vec_size, word_bytes, true, "compress_inplace"));
    if (num_index < 0) index = nullptr;
    const bool has_index = num_index >= 0;
    const int64_t nrows = has_index ? num_index : num_vecs;
    IBP_ARG(num_index <= 0 || index, "compress_inplace: null index array");
    IBP_ARG(!has_index || num_index <= num_vecs,
            "compress_inplace: %lld indexed rows do not fit a dataset of %lld rows",
            (long long)num_index, (long long)num_vecs);
    IBP_ARG((mask && bitval) || vec_size == 0, "compress_inplace: null mask/bitval");
    IBP_ARG(bitmask || nrows == 0, "compress_inplace: null bitmask");
    IBP_ACCESSIBLE(mask, "compress_inplace", "mask");
    IBP_ACCESSIBLE(bitval, "compress_inplace", "bitval");
    IBP_ACCESSIBLE(index, "compress_inplace", "the index array");
    IBP_ACCESSIBLE(bitmask, "compress_inplace", "bitmask");
    cudaStream_t st = (cudaStream_t)stream;
    if (word_bytes == 4)
        return compress_inplace_t<uint32_t>((uint32_t *)dataset, num_vecs, vec_size,
                                            (const uint32_t *)mask, (const uint32_t *)bitval,
                                            index, num_index, has_index, bitmask, workspace,
                                            workspace_bytes, st);
    return compress_inplace_t<uint64_t>((uint64_t *)dataset, num_vecs, vec_size,
                                        (const uint64_t *)mask, (const uint64_t *)bitval, index,
                                        num_index, has_index, bitmask, workspace,
                                        workspace_bytes, st);
}

// ------------------------------------------------------------------ compress_condensed
size_t ibp_condensed_offsets_workspace_size(int64_t nrows) {
    return inclusive_offsets_workspace(nrows);
}

ibp_status ibp_condensed_offsets(int64_t *sizes_to_offsets, int64_t nrows, int64_t *total,
                                 void *workspace, size_t workspace_bytes, ibp_stream_t stream) {
    clear_error();
    IBP_RANGE("ibp_condensed_offsets");
    IBP_ARG(nrows >= 0, "condensed_offsets: negative row count");
    IBP_ARG(sizes_to_offsets || nrows == 0, "condensed_offsets: null sizes");
    return inclusive_offsets_impl(sizes_to_offsets, nrows, total, workspace, workspace_bytes,
                                  (cudaStream_t)stream);
}

size_t ibp_compress_condensed_workspace_size(int64_t vec_size, int word_bytes) {
    return kStatusBytes + (word_bytes == 8 ? tables_bytes<uint64_t>(vec_size)
                                           : tables_bytes<uint32_t>(vec_size));
}

ibp_status ibp_compress_condensed(const void *dataset, int64_t num_vecs, int64_t vec_size,
                                  int word_bytes, const void *mask, const void *bitval,
                                  const int64_t *index, int64_t num_index,
                                  const int64_t *offsets, void *out, void *workspace,
                                  size_t workspace_bytes, ibp_stream_t stream) {
    clear_error();
    IBP_RANGE("ibp_compress_condensed");
    IBP_RET(check_rows(dataset, num_vecs, vec_size, word_bytes, true, "compress_condensed"));
    if (num_index < 0) index = nullptr;
    const int64_t nrows = num_index >= 0 ? num_index : num_vecs;
    IBP_ARG(num_index <= 0 || index, "compress_condensed: null index array");
    IBP_ARG((offsets && out) || nrows == 0, "compress_condensed: null offsets/out");
    IBP_ACCESSIBLE(mask, "compress_condensed", "mask");
    IBP_ACCESSIBLE(bitval, "compress_condensed", "bitval");
    IBP_ACCESSIBLE(index, "compress_condensed", "the index array");
    IBP_ACCESSIBLE(offsets, "compress_condensed", "offsets");
    IBP_ACCESSIBLE(out, "compress_condensed", "the output");
    const size_t need = ibp_compress_condensed_workspace_size(vec_size, word_bytes);
    if (!workspace || workspace_bytes < need) {
        set_error("compress_condensed: workspace of %zu bytes is below the required %zu",
                  workspace_bytes, need);
        return IBP_ERR_WORKSPACE;
    }
    cudaStream_t st = (cudaStream_t)stream;
    Carver c{(char *)workspace, 0, workspace_bytes};
    int32_t *status = c.take<int32_t>(kStatusBytes / 4);
    IBP_CUDA(cudaMemsetAsync(status, 0, sizeof(int32_t), st));
    if (word_bytes == 4) {
        ColTables<uint32_t> t = carve_tables<uint32_t>(c, vec_size);
        if (vec_size > 0)
            IBP_RET(build_tables<uint32_t>((const uint32_t *)mask, (const uint32_t *)bitval,
                                           vec_size, t, st));
        return compress_condensed_rows<uint32_t>((const uint32_t *)dataset, num_vecs, vec_size,
                                                 t, index, nrows, offsets, (uint32_t *)out,
                                                 status, st);
    }
    ColTables<uint64_t> t = carve_tables<uint64_t>(c, vec_size);
    if (vec_size > 0)
        IBP_RET(build_tables<uint64_t>((const uint64_t *)mask, (const uint64_t *)bitval,
                                       vec_size, t, st));
    return compress_condensed_rows<uint64_t>((const uint64_t *)dataset, num_vecs, vec_size, t,
                                             index, nrows, offsets, (uint64_t *)out, status, st);
}

// ------------------------------------------------------------------ decompress_fetch
size_t ibp_decompress_fetch_workspace_size(int64_t num_index, int64_t vec_size, int word_bytes,
                                           int has_index) {
    return decompress_workspace(num_index, vec_size, word_bytes, has_index != 0);
}

ibp_status ibp_decompress_fetch(const void *comp, int64_t num_vecs, int64_t vec_size,
                                int word_bytes, const void *mask, const void *bitval,
                                const int32_t *bitmask, const int64_t *index,
                                int64_t num_index, int32_t comp_len, void *out, int32_t nblks,
                                int32_t nthreads, int32_t impl, void *workspace,
                                size_t workspace_bytes, ibp_stream_t stream) {
    clear_error();
    IBP_RANGE("ibp_decompress_fetch");
    IBP_RET(check_rows(comp, num_vecs, vec_size, word_bytes, true, "decompress_fetch"));
    if (num_index < 0) index = nullptr;
    const int64_t nrows = num_index >= 0 ? num_index : num_vecs;
    IBP_ARG(num_index <= 0 || index, "decompress_fetch: null index array");
    IBP_ARG(out || nrows * vec_size == 0, "decompress_fetch: null output");
    if (impl != -1 && impl != 0 && impl != 1 && impl != 2 && impl != 5) {
        set_error("decompress_fetch: impl %d is not provided (3/4 are the reference's "
                  "upper-bound stand-ins, not decompressors)", impl);
        return IBP_ERR_UNSUPPORTED;
    }
    IBP_ARG(impl == 2 || (mask && bitval && bitmask) || nrows * vec_size == 0,
            "decompress_fetch: null mask/bitval/bitmask");
    IBP_ACCESSIBLE(mask, "decompress_fetch", "mask");
    IBP_ACCESSIBLE(bitval, "decompress_fetch", "bitval");
    IBP_ACCESSIBLE(bitmask, "decompress_fetch", "bitmask");
    IBP_ACCESSIBLE(index, "decompress_fetch", "the index array");
    IBP_ACCESSIBLE(out, "decompress_fetch", "the output");
    cudaStream_t st = (cudaStream_t)stream;
    if (word_bytes == 4)
        return decompress_impl<uint32_t>((const uint32_t *)comp, num_vecs, vec_size,
                                         (const uint32_t *)mask, (const uint32_t *)bitval,
                                         bitmask, index, num_index, num_index >= 0, comp_len,
                                         (uint32_t *)out,
                                         nblks, nthreads, impl, workspace, workspace_bytes, st);
    return decompress_impl<uint64_t>((const uint64_t *)comp, num_vecs, vec_size,
                                     (const uint64_t *)mask, (const uint64_t *)bitval, bitmask,
                                     index, num_index, num_index >= 0, comp_len,
                                     (uint64_t *)out, nblks,
                                     nthreads, impl, workspace, workspace_bytes, st);
}

ibp_status ibp_read_rows_probe(const void *base, int64_t stride_bytes, const int64_t *rows,
                               int64_t num_rows, int32_t read_bytes, void *workspace,
                               size_t workspace_bytes, ibp_stream_t stream) {
    clear_error();
    IBP_ARG(base && (rows || num_rows == 0), "read_rows_probe: null argument");
    IBP_ARG(num_rows >= 0, "read_rows_probe: negative row count");
    IBP_ARG(read_bytes > 0 && read_bytes <= 1024, "read_rows_probe: read_bytes must be 1..1024");
    IBP_ARG(stride_bytes >= read_bytes && stride_bytes % 16 == 0 && ((uintptr_t)base & 15) == 0,
            "read_rows_probe: rows must be 16-byte aligned and at least read_bytes apart");
    IBP_ACCESSIBLE(rows, "read_rows_probe", "the row list");
    return read_rows_probe(base, stride_bytes, rows, num_rows, read_bytes, workspace,
                           workspace_bytes, (cudaStream_t)stream);
}

// ------------------------------------------------------------------ condensed fetch
ibp_status ibp_decompress_fetch_condensed(const void *comp, int64_t comp_words,
                                          const int64_t *offsets, int64_t num_vecs,
                                          int64_t vec_size, int word_bytes,
                                          const void *mask, const void *bitval,
                                          const int64_t *index, int64_t num_index, void *out,
                                          void *workspace, size_t workspace_bytes,
                                          ibp_stream_t stream) {
    clear_error();
    IBP_RANGE("ibp_decompress_fetch_condensed");
    IBP_ARG(num_vecs >= 0 && vec_size >= 0 && comp_words >= 0,
            "decompress_fetch_condensed: negative shape");
    IBP_ARG(word_bytes == 4 || word_bytes == 8,
            "decompress_fetch_condensed: Input tensor must be 4-byte or 8-byte datatype");
    if (num_index < 0) index = nullptr;
    const int64_t nrows = num_index >= 0 ? num_index : num_vecs;
    const bool work = nrows * vec_size > 0;
    IBP_ARG(!work || (comp && offsets && mask && bitval),
            "decompress_fetch_condensed: null rows/offsets/mask/bitval");
    IBP_ARG(num_index <= 0 || index, "decompress_fetch_condensed: null index array");
    IBP_ARG(out || !work, "decompress_fetch_condensed: null output");
    if (work) {
        IBP_ACCESSIBLE(comp, "decompress_fetch_condensed", "the condensed rows");
        IBP_ACCESSIBLE(offsets, "decompress_fetch_condensed", "the offsets");
        IBP_ACCESSIBLE(mask, "decompress_fetch_condensed", "mask");
        IBP_ACCESSIBLE(bitval, "decompress_fetch_condensed", "bitval");
        IBP_ACCESSIBLE(index, "decompress_fetch_condensed", "the index array");
        IBP_ACCESSIBLE(out, "decompress_fetch_condensed", "the output");
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (word_bytes == 4)
        return decompress_impl<uint32_t>((const uint32_t *)comp, num_vecs, vec_size,
                                         (const uint32_t *)mask, (const uint32_t *)bitval,
                                         nullptr, index, num_index, num_index >= 0, -1,
                                         (uint32_t *)out, -1, -1, -1, workspace,
                                         workspace_bytes, st, offsets, comp_words * 4);
    return decompress_impl<uint64_t>((const uint64_t *)comp, num_vecs, vec_size,
                                     (const uint64_t *)mask, (const uint64_t *)bitval, nullptr,
                                     index, num_index, num_index >= 0, -1, (uint64_t *)out, -1,
                                     -1, -1, workspace, workspace_bytes, st, offsets,
                                     comp_words * 8);
}

}  // extern "C"
