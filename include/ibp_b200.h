/*
 * ibp_b200.h -- C ABI of the B200-native Invariant Bit Packing engine (libibp_b200.so).
 *
 * Plain pointers and sizes only.  Every entry point replaces one function of the
 * reference's PyTorch extension `ibp_cuda` (src/ibp_api.cu:124-135); the comment on
 * each gives the reference file:line it replaces.  A foreign-function binding
 * (ctypes, cgo, JNI, N-API) binds these symbols directly.
 *
 * Conventions
 *  - dataset rows: `num_vecs` rows of `vec_size` words of `word_bytes` bytes, row stride
 *    vec_size words, in device memory or in pinned (page-locked, mapped) host memory;
 *    kernels read host rows zero-copy over PCIe.
 *  - mask / bitval: `vec_size` words (k-means: num_clusters x vec_size), device memory.
 *  - bitmask: int32 words, bit (i % 32) of word i / 32 set when row i is stored compressed.
 *  - index arrays: int64, device memory, `num_index` entries; num_index < 0 means "no
 *    index" (rows 0..num_vecs-1, the pointer is ignored).  An index outside [0, num_vecs) is
 *    not read: the row is skipped and bit 0 of the call's device status word is set
 *    (ibp_read_status).
 *  - `workspace`: caller-owned device scratch of at least the size the matching
 *    *_workspace_size() returns (may be NULL when that size is 0).  No entry point
 *    allocates device memory, so every call can be captured in a CUDA graph except
 *    ibp_preprocess_kmeans with init_rows == NULL (host shuffle) and the condensed
 *    compressor's size query (which the caller synchronises on).
 *  - `stream`: a cudaStream_t (NULL = legacy default stream).  All work is enqueued on
 *    it; no entry point synchronises the host unless stated.
 *  - return value: IBP_OK or an error code; ibp_last_error() gives a message (per thread).
 *    Nothing ever calls exit().
 */
#ifndef IBP_B200_H
#define IBP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *ibp_stream_t; /* same type as cudaStream_t */

typedef enum {
    IBP_OK = 0,
    IBP_ERR_ARGUMENT = 1,   /* invalid sizes, word size, pointers */
    IBP_ERR_WORKSPACE = 2,  /* workspace missing or smaller than *_workspace_size() */
    IBP_ERR_CUDA = 3,       /* a CUDA runtime call or launch failed */
    IBP_ERR_UNSUPPORTED = 4 /* option the engine does not provide */
} ibp_status;

/* Message describing the last error returned on this thread ("" if none). */
const char *ibp_last_error(void);

/* ABI version of this header (bumped on any signature change). */
int ibp_abi_version(void);

/* Debug prints to stdout; replaces print_debug (src/ibp_api.cu:7-12). */
void ibp_set_debug(int on);

/* How decompress_fetch (and its condensed and no-alloc forms) finds the repeated rows of an
 * index array, process-wide: 0 = auto (hash table for compressed rows, fixed-stride or
 * condensed, in device memory, or in host memory when the index has fewer than a quarter as
 * many entries as the set has rows; else sort), 1 = always sort (rows then fetched in row
 * order), 2 = always hash (repeats are then copied inside the fetch for host rows).  Dense
 * host batches whose rows repeat a lot (skewed, e.g. Zipf) are faster with 2; dense batches
 * with few repeats are faster sorted.  No counterpart in the reference (it always sorts). */
ibp_status ibp_set_fetch_dedup(int32_t mode);

/* How long a repeated index of a hashed host-row fetch waits for the row of its first
 * occurrence, which another warp of the same fetch decodes, process-wide: at most `polls`
 * polls about 0.25 us apart (default 2^20, restored by -1).  A repeat that stops waiting
 * decodes its own row from the source instead (one more read of that row) and sets bit 3 of
 * the status word, so the output is the same whatever the limit; 0 makes every such repeat
 * take that path at once, which tests use to exercise it.  No counterpart in the reference
 * (it sorts and copies repeats after the fetch). */
ibp_status ibp_set_repeat_wait_limit(int32_t polls);

/* Profiling hooks (benchmarks): after ibp_profile_enable(cap), the next `cap` row-fetch
 * kernel launches (decompress_fetch, any thread) are bracketed by CUDA events on their
 * stream.  ibp_profile_take waits for them, writes their durations in milliseconds to ms[]
 * (at most `capacity` entries), returns how many, and turns profiling off. */
ibp_status ibp_profile_enable(int32_t capacity);
int32_t ibp_profile_take(float *ms, int32_t capacity);

/* Number of engine kernels this process has launched so far (all threads). */
unsigned long long ibp_kernel_launch_count(void);

/* Device status word of the last call that used `workspace`: bit 0 = an index was out of
 * range; bit 1 = a row marked compressed has a bitmap whose stream would not fit the row
 * (the bitmask/mask do not belong to the data), and its output row was left untouched;
 * bit 2 = a sorted batch's request counts did not add up to its stated total_rows;
 * bit 3 = a repeated index gave up waiting for the row of its first occurrence
 * (ibp_set_repeat_wait_limit) and decoded its own row from the source instead: its output
 * row is correct, the bit only reports the extra read.
 * Enqueues a copy on `stream` and waits for it (blocking). */
ibp_status ibp_read_status(const void *workspace, int32_t *status, ibp_stream_t stream);

/* ---------------------------------------------------------------- preprocess
 * Replaces preprocess (src/preprocess.cu:17-76; include/preproc/ibp_preproc_host.cuh:23-115).
 * threshold < 0: sweep 0.7f..1.0f in float32 steps of 0.05 and keep the first threshold
 * with the most saved bits; otherwise use `threshold`.  mask/bitval (vec_size words each)
 * are fully written: zero when no threshold saves any bit.  word_bytes in {1,2,4,8}.
 * Non-blocking (the reference blocks): the selection runs on the device.  A host-resident
 * dataset is copied into the workspace during the census (so the second pass reads HBM)
 * when workspace_bytes >= ibp_preprocess_workspace_size(...) + num_vecs*vec_size*word_bytes
 * rounded up to 256. */
size_t ibp_preprocess_workspace_size(int64_t num_vecs, int64_t vec_size, int word_bytes,
                                     float threshold);
ibp_status ibp_preprocess(const void *dataset, int64_t num_vecs, int64_t vec_size,
                          int word_bytes, float threshold, void *mask, void *bitval,
                          void *workspace, size_t workspace_bytes, ibp_stream_t stream);

/* ---------------------------------------------------------------- preprocess_kmeans
 * Replaces preprocess_kmeans (src/preprocess.cu:88-139; ibp_preproc_host.cuh:118-284).
 * word_bytes in {4,8}.  Centroid 0 is row 0 and centroid i (1 <= i < min(C, num_vecs)) is
 * row init_rows[i] (a host array of min(C, num_vecs) entries; entry 0 is ignored).  With
 * init_rows == NULL the rows come from std::random_shuffle over 0..num_vecs-1, as in the
 * reference (process rand() state; blocking).  10 assignment/update rounds, then per-
 * cluster masks at threshold 1.0f (the value the reference's sweep leaves behind; its
 * `threshold` argument has no effect).  Ties between centroids go to the highest id.
 * masks/bitvals: num_clusters x vec_size words; clusters: num_vecs int32 (device or
 * pinned host memory). */
size_t ibp_preprocess_kmeans_workspace_size(int64_t num_vecs, int64_t vec_size,
                                            int word_bytes, int32_t num_clusters);
ibp_status ibp_preprocess_kmeans(const void *dataset, int64_t num_vecs, int64_t vec_size,
                                 int word_bytes, int32_t num_clusters,
                                 const int64_t *init_rows, void *masks, void *bitvals,
                                 int32_t *clusters, void *workspace, size_t workspace_bytes,
                                 ibp_stream_t stream);

/* ---------------------------------------------------------------- get_compress_size
 * Replaces get_compress_size (src/compress.cu:25-174; include/misc/ibp_misc_dev.cuh:19-46).
 * sizes[i] = compressed bytes of row index[i] (or row i when num_index < 0, then
 * num_vecs rows are sized); a row whose index is out of range gets
 * size 0.  `total` (nullable, device memory) is incremented by the sum of sizes.
 * word_bytes in {1,2,4,8}.  sizes: device or pinned host memory. */
ibp_status ibp_get_compress_size(const void *dataset, int64_t num_vecs, int64_t vec_size,
                                 int word_bytes, const void *mask, const void *bitval,
                                 const int64_t *index, int64_t num_index, int64_t *sizes,
                                 int64_t *total, ibp_stream_t stream);

/* ---------------------------------------------------------------- compress_inplace
 * Replaces compress_inplace (src/compress.cu:176-236; include/compress/ibp_compress_host.cuh:7-27).
 * Row i (i < nrows, nrows = num_index >= 0 ? num_index : num_vecs) becomes the compressed form of
 * source row index[i] (or i), zero padded to vec_size words, when that is strictly smaller;
 * otherwise the raw source row.  bitmask ((nrows+31)/32 int32, device) is fully written.
 * With an index, every source row is read before any row is written (the reference races
 * there); that needs nrows*vec_size*word_bytes bytes of workspace.  word_bytes in {4,8}. */
size_t ibp_compress_inplace_workspace_size(int64_t num_index, int64_t vec_size, int word_bytes,
                                           int has_index);
ibp_status ibp_compress_inplace(void *dataset, int64_t num_vecs, int64_t vec_size,
                                int word_bytes, const void *mask, const void *bitval,
                                const int64_t *index, int64_t num_index, int32_t *bitmask,
                                void *workspace, size_t workspace_bytes, ibp_stream_t stream);

/* ---------------------------------------------------------------- compress_condensed
 * Replaces compress_condensed (src/compress.cu:238-313; ibp_compress_kernel.cuh:58-94).
 * Step 1: ibp_condensed_offsets turns sizes (from ibp_get_compress_size, device memory)
 * into inclusive byte offsets in place and writes the total to *total (device memory).
 * Step 2: the caller allocates total bytes (zeroed) and calls ibp_compress_condensed,
 * which writes row i's compressed form (or raw row) at byte offset offsets[i-1]
 * (0 for row 0).  word_bytes in {4,8}. */
size_t ibp_condensed_offsets_workspace_size(int64_t nrows);
ibp_status ibp_condensed_offsets(int64_t *sizes_to_offsets, int64_t nrows, int64_t *total,
                                 void *workspace, size_t workspace_bytes, ibp_stream_t stream);
size_t ibp_compress_condensed_workspace_size(int64_t vec_size, int word_bytes);
ibp_status ibp_compress_condensed(const void *dataset, int64_t num_vecs, int64_t vec_size,
                                  int word_bytes, const void *mask, const void *bitval,
                                  const int64_t *index, int64_t num_index,
                                  const int64_t *offsets, void *out, void *workspace,
                                  size_t workspace_bytes, ibp_stream_t stream);

/* ---------------------------------------------------------------- decompress_fetch
 * Replaces decompress_fetch (src/decompress.cu:10-156; include/decompress/).
 * out row k (k < nrows, nrows = num_index >= 0 ? num_index : num_vecs) = decompressed row index[k]
 * (or k) of `comp`, the fixed-stride in-place-compressed rows (device or pinned host;
 * pinned host rows are read zero-copy).  out: nrows x vec_size words in device or pinned
 * host memory.  comp_len (words, <= 0: vec_size) is the caller's average compressed row
 * length, a tuning hint only.  nblks / nthreads / impl follow the reference knobs:
 * impl -1 auto, 0/1/5 decompress (the engine picks its own kernel shape), 2 = plain
 * uncompressed gather of the stored rows (the reference's baseline); other values are
 * IBP_ERR_UNSUPPORTED.  nblks/nthreads <= 0 pick defaults.  word_bytes in {4,8}.
 * With an index, rows are fetched in sorted order and each distinct row is read once;
 * repeats are copied on the device. */
size_t ibp_decompress_fetch_workspace_size(int64_t num_index, int64_t vec_size, int word_bytes,
                                           int has_index);
ibp_status ibp_decompress_fetch(const void *comp, int64_t num_vecs, int64_t vec_size,
                                int word_bytes, const void *mask, const void *bitval,
                                const int32_t *bitmask, const int64_t *index,
                                int64_t num_index, int32_t comp_len, void *out, int32_t nblks,
                                int32_t nthreads, int32_t impl, void *workspace,
                                size_t workspace_bytes, ibp_stream_t stream);

/* Measurement aid, no counterpart in the reference: reads the first read_bytes (1..1024,
 * rounded up to 16-byte blocks) of each listed row -- row r at base + r * stride_bytes, rows
 * 16-byte aligned -- the way the row-fetch kernel does (a warp keeps 4 rows in flight, the
 * same grid shape) and decodes nothing.  Its time, taken with the profiling hooks, is the
 * ceiling of the fetch kernel's access pattern on this link or memory.  Each row is read
 * entirely inside [base + r * stride_bytes, + read_bytes rounded up to 16), so the caller
 * must own those bytes.  Workspace: 256 bytes of device memory. */
ibp_status ibp_read_rows_probe(const void *base, int64_t stride_bytes, const int64_t *rows,
                               int64_t num_rows, int32_t read_bytes, void *workspace,
                               size_t workspace_bytes, ibp_stream_t stream);

/* ---------------------------------------------------------------- condensed fetch
 * No counterpart in the reference, which writes the condensed layout (compress_condensed,
 * src/compress.cu:238-313) but has no decompressor for it.  out row k = decompressed row
 * index[k] (or k when num_index < 0) of `comp` (comp_words words), the condensed rows: row i
 * occupies bytes
 * [offsets[i-1], offsets[i]) (offsets[-1] = 0), i.e. the inclusive byte offsets that
 * ibp_condensed_offsets produced; a row whose length is vec_size words is stored raw, any
 * shorter one is compressed.  Each row is read once with its exact length (no fixed stride,
 * no length guess).  offsets: num_vecs entries, device memory (pinned host works, slowly).
 * Out-of-range indices set bit 0 of the status word; offsets that cannot describe a row of
 * `comp` or a bitmap whose stream overruns its row set bit 1; those output rows are left
 * untouched, and no read leaves the 16-byte blocks that hold `comp`.
 * Workspace: ibp_decompress_fetch_workspace_size(num_index, vec_size, word_bytes,
 * num_index >= 0). */
ibp_status ibp_decompress_fetch_condensed(const void *comp, int64_t comp_words,
                                          const int64_t *offsets, int64_t num_vecs,
                                          int64_t vec_size, int word_bytes,
                                          const void *mask, const void *bitval,
                                          const int64_t *index, int64_t num_index, void *out,
                                          void *workspace, size_t workspace_bytes,
                                          ibp_stream_t stream);

/* ---------------------------------------------------------------- batched multi-set fetch
 * No single counterpart in the reference, which fetches one tensor set per decompress_fetch
 * call (src/decompress.cu:10-156) and whose callers issue one call per table or tensor.  Here
 * one launch serves many requests -- (set, row list, output) -- across sets with different
 * row lengths, masks and compression ratios:
 *   1. describe the sets (same word size) and register them once: the registry is a device
 *      buffer the caller owns (ibp_sets_registry_size bytes) holding every set's descriptor
 *      and per-column tables; it stays valid as long as the sets' buffers do.  Registration
 *      blocks until the registry is written.
 *   2. put up to max_requests ibp_request records and their count in DEVICE memory and call
 *      ibp_batch_fetch.  It reads both on the device, so a CUDA graph that captured the call
 *      can be replayed after the caller rewrites the records (e.g. with a copy node).
 * Out-of-range rows or set ids set bit 0 of the status word (first 4 bytes of the workspace).
 * Rows are fetched as listed (no de-duplication inside a request; ibp_batch_fetch_sorted
 * below de-duplicates). */
typedef struct {
    const void *comp;       /* compressed rows, device or pinned host memory */
    int64_t num_vecs;
    int64_t vec_size;       /* words per row */
    const void *mask;       /* vec_size words, device memory */
    const void *bitval;     /* vec_size words, device memory */
    const int32_t *bitmask; /* (num_vecs+31)/32 words, device memory */
    int32_t comp_len;       /* average compressed row length in words (hint); <= 0: none */
    int32_t reserved;
} ibp_set_desc;

typedef struct {
    int32_t set;            /* registered set */
    int32_t reserved;
    const int64_t *index;   /* `count` row numbers (device); NULL: rows first .. first+count-1 */
    int64_t first;
    int64_t count;
    void *out;              /* count x vec_size words, device or pinned host memory */
} ibp_request;

size_t ibp_sets_registry_size(const ibp_set_desc *sets, int32_t nsets, int word_bytes);
ibp_status ibp_sets_register(const ibp_set_desc *sets, int32_t nsets, int word_bytes,
                             void *registry, size_t registry_bytes, ibp_stream_t stream);
size_t ibp_batch_fetch_workspace_size(void);
ibp_status ibp_batch_fetch(const void *registry, const ibp_request *requests,
                           const int32_t *num_requests, int32_t max_requests, void *workspace,
                           size_t workspace_bytes, ibp_stream_t stream);
/* Times the batch on every candidate launch shape (threads per block {128, 256} x rows in
 * flight per warp {1, 2, 4} x blocks per SM {all, 2, 1}), keeps the fastest for this
 * registry's (word size, longest row, compression-ratio bucket, residency) for the rest of
 * the process, and writes it to chosen[0..3] (threads, rows in flight, blocks per SM, index).
 * Blocking; runs the batch ~55 times. */
ibp_status ibp_batch_autotune(const void *registry, const ibp_request *requests,
                              const int32_t *num_requests, int32_t max_requests,
                              void *workspace, size_t workspace_bytes, int32_t *chosen,
                              ibp_stream_t stream);
/* De-duplicating batch: like ibp_batch_fetch, but each request's rows are radix-sorted on the
 * device first, so a row listed several times in one request crosses the bus once and is
 * copied into its other output rows, and the fetch walks each set in row order (the per-call
 * path of ibp_decompress_fetch does the same).  num_requests (1..8192) and total_rows (the sum
 * of the requests' counts, < 2^31) are host values, so a graph that captured the call serves
 * batches of exactly that shape only.  `requests` is device memory.  If the device counts
 * disagree with total_rows, bit 2 of the status word is set and only positions below the
 * smaller total are fetched.  Workspace: ibp_batch_fetch_sorted_workspace_size(max rows,
 * max requests) bytes; the status word is its first 4 bytes. */
size_t ibp_batch_fetch_sorted_workspace_size(int64_t max_total_rows, int32_t max_requests);
ibp_status ibp_batch_fetch_sorted(const void *registry, const ibp_request *requests,
                                  int32_t num_requests, int64_t total_rows, void *workspace,
                                  size_t workspace_bytes, ibp_stream_t stream);

/* De-duplicating batch without a sort: like ibp_batch_fetch_sorted (num_requests and total_rows
 * host values, requests in device memory, bit 2 of the status word when the device counts
 * disagree with total_rows), but each (set, row) of the batch is claimed in a hash table
 * inside the fetch kernel, so a row listed several times -- in one request or across requests
 * of the same set -- crosses the bus once, and its other output rows are copied on the device
 * as soon as its first copy is written (the per-call ibp_decompress_fetch does the same for
 * sparse host batches).  Each set gets row slots of its own length, so short rows keep
 * several reads in flight per warp beside long ones.  Rows are fetched in request order, not
 * row order.  Workspace: ibp_batch_fetch_hashed_workspace_size(max rows) bytes (32 per row);
 * the status word is its first 4 bytes.  A repeat that waits too long for its row's first
 * copy decodes its own (ibp_set_repeat_wait_limit). */
size_t ibp_batch_fetch_hashed_workspace_size(int64_t max_total_rows);
ibp_status ibp_batch_fetch_hashed(const void *registry, const ibp_request *requests,
                                  int32_t num_requests, int64_t total_rows, void *workspace,
                                  size_t workspace_bytes, ibp_stream_t stream);

/* ---------------------------------------------------------------- serving
 * No counterpart in the reference (its callers issue one decompress_fetch per lookup).  A
 * continuous-batching server over a registry: clients submit requests from any thread; a
 * scheduler thread admits them in arrival order whenever their output fits the caller's
 * device arena, packs all admitted requests into one de-duplicating batched launch
 * (ibp_batch_fetch_hashed, or ibp_batch_fetch_sorted after ibp_server_set_dedup(srv, 1); a
 * batch holds at most max(index_capacity, 2^20) rows, and a single range request above that
 * is fetched as listed), and keeps up to max_inflight
 * launches on the GPU, so requests arriving meanwhile join the next launch.  Buffers (index
 * staging rings of index_capacity entries, request tables, the sort workspace, a stream) are
 * allocated at creation only.  Timestamps are host steady-clock microseconds. */
typedef struct ibp_server ibp_server;
ibp_status ibp_server_create(const void *registry, const ibp_set_desc *sets, int32_t nsets,
                             int word_bytes, void *out_arena, size_t arena_bytes,
                             int64_t index_capacity, int32_t max_batch, int32_t max_inflight,
                             ibp_server **out);
/* rows == NULL: rows first .. first+count-1; else `count` host row numbers (copied before
 * returning).  IBP_ERR_WORKSPACE: index staging full (retry) or output larger than the arena. */
ibp_status ibp_server_submit(ibp_server *srv, int32_t set, const int64_t *rows, int64_t first,
                             int64_t count, int64_t *id);
/* Wait for a request (timeout_ms < 0: forever); *out = its output rows in the arena,
 * times[0..2] = submitted, admitted, done.  IBP_ERR_UNSUPPORTED on timeout. */
ibp_status ibp_server_wait(ibp_server *srv, int64_t id, int32_t timeout_ms, void **out,
                           double *times);
/* Withdraw a request still queued (not yet admitted): it is not fetched, and waiting for it
 * afterwards reports an unknown request.  IBP_ERR_UNSUPPORTED once it is admitted. */
ibp_status ibp_server_cancel(ibp_server *srv, int64_t id);
/* Give a finished request's output rows back to the arena. */
ibp_status ibp_server_release(ibp_server *srv, int64_t id);
/* Admission limits of one batch: at most max_rows rows (no more than the batch workspace's
 * max(index_capacity, 2^20)) and max_bytes output bytes, both counted after the batch's
 * first request, which is always admitted.  <= 0 keeps the current value.  Defaults: the
 * workspace's rows and 128 MiB.  When requests queue up faster than the link drains them,
 * the byte limit rises to the queued output bytes divided by max_inflight, so a backlog is
 * served by fewer, larger launches (which also share the rows that queued requests of one
 * set have in common).  Smaller batches finish early requests of a burst sooner (lower
 * p50); larger ones amortise per-launch cost.  Index spans and request tables are copied to
 * the device on a second stream, overlapping the previous batch's kernel. */
ibp_status ibp_server_set_batch_limits(ibp_server *srv, int64_t max_rows, int64_t max_bytes);
/* How later batches de-duplicate: 0 = hash claims inside the fetch (default), 1 = radix sort
 * (rows then fetched in row order). */
ibp_status ibp_server_set_dedup(ibp_server *srv, int32_t mode);
/* stats[0..3] = batches launched, rows done, output bytes done, requests pending. */
ibp_status ibp_server_stats(ibp_server *srv, int64_t *stats);
/* Stop the scheduler after the in-flight batches finish and free the server's buffers. */
ibp_status ibp_server_destroy(ibp_server *srv);

/* ---------------------------------------------------------------- decompress_fetch, no allocation
 * No counterpart in the reference.  For callers that cannot allocate device memory at all
 * (a host framework that owns every device byte and offers no allocation hook, an allocator
 * policy that forbids cudaMalloc on the request path, code that must not risk the implicit
 * device synchronisation of cudaMalloc/cudaFree).  Same arguments and results as
 * ibp_decompress_fetch without nblks/nthreads/impl/workspace; its scratch is a static
 * IBP_NOALLOC_SCRATCH_BYTES (4 MiB) device array that the library reserves on every device
 * that loads it, until the process exits.  A call fits exactly when
 *     ibp_decompress_fetch_workspace_size(num_index, vec_size, word_bytes, num_index >= 0)
 *         <= IBP_NOALLOC_SCRATCH_BYTES
 * (about 40-48 bytes per index entry plus the column tables: ~90k entries of 64-word int64
 * rows); a call that does not fit returns IBP_ERR_WORKSPACE before launching anything.  The
 * first call in a CUDA context looks the array's device address up (cudaGetSymbolAddress,
 * with that device current): make that first call before any stream capture on the device.
 * All calls share the array, and calls whose GPU work overlaps (other streams, other
 * threads) race on it: serialise them.  Nothing is allocated or freed. */
#define IBP_NOALLOC_SCRATCH_BYTES 4194304
ibp_status ibp_decompress_fetch_noalloc(const void *comp, int64_t num_vecs, int64_t vec_size,
                                        int word_bytes, const void *mask, const void *bitval,
                                        const int32_t *bitmask, const int64_t *index,
                                        int64_t num_index, int32_t comp_len, void *out,
                                        ibp_stream_t stream);
/* Device status word of the last ibp_decompress_fetch_noalloc call on the current device
 * (the same bits as ibp_read_status: out-of-range index, corrupt row, ...).  It is the
 * first word of the shared static scratch, so read it before the next no-alloc call on the
 * device.  Enqueues a copy on `stream` and waits for it (blocking). */
ibp_status ibp_decompress_fetch_noalloc_status(int32_t *status, ibp_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* IBP_B200_H */
