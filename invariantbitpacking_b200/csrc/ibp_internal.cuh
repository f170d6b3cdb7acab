// ibp_internal.cuh -- declarations shared between the kernel files and the C ABI layer.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "ibp_codec.cuh"
#include "ibp_common.cuh"

namespace ibp200 {

constexpr int kMaxThresholds = 8;

struct ThrList {
    int count;
    float v[kMaxThresholds];
};

ThrList sweep_thresholds(float threshold);

// ---- preprocess (ibp_preprocess.cu)
size_t preprocess_workspace(int64_t n, int64_t v, int wb, float threshold, bool staged);
template <typename U>
ibp_status preprocess_impl(const U *data, int64_t n, int64_t v, float threshold, U *mask,
                           U *bitval, void *ws, size_t ws_bytes, bool data_on_host,
                           cudaStream_t st);

// ---- sizes and packing (ibp_compress.cu)
template <typename U>
ibp_status compress_size_impl(const U *data, int64_t n, int64_t v, const U *mask,
                              const U *bitval, const int64_t *idx, int64_t nrows,
                              int64_t *sizes, int64_t *total, int32_t *status,
                              cudaStream_t st);
template <typename U>
ibp_status compress_rows_impl(const U *src, int64_t n, int64_t v, ColTables<U> t,
                              const int64_t *idx, int64_t nrows, U *out, bool out_is_src,
                              int32_t *bitmask, int32_t *status, cudaStream_t st);
template <typename U>
ibp_status gather_rows_impl(const U *src, int64_t n, int64_t v, const int64_t *idx,
                            int64_t nrows, U *out, int32_t *status, cudaStream_t st);
template <typename U>
ibp_status compress_condensed_rows(const U *src, int64_t n, int64_t v, ColTables<U> t,
                                   const int64_t *idx, int64_t nrows, const int64_t *offsets,
                                   U *out, int32_t *status, cudaStream_t st);
ibp_status inclusive_offsets_impl(int64_t *sizes, int64_t nrows, int64_t *total, void *ws,
                                  size_t ws_bytes, cudaStream_t st);
size_t inclusive_offsets_workspace(int64_t nrows);

// ---- decompress (ibp_decompress.cu)
size_t decompress_workspace(int64_t nidx, int64_t v, int wb, bool has_index);
template <typename U>
ibp_status decompress_impl(const U *comp, int64_t n, int64_t v, const U *mask,
                           const U *bitval, const int32_t *bitmask, const int64_t *idx,
                           int64_t nidx, bool has_index, int comp_len, U *out, int nblks,
                           int nthreads, int impl, void *ws, size_t ws_bytes, cudaStream_t st,
                           const int64_t *offsets = nullptr, int64_t comp_bytes = 0);

ibp_status read_rows_probe(const void *base, int64_t stride_bytes, const int64_t *rows,
                           int64_t nrows, int32_t read_bytes, void *ws, size_t ws_bytes,
                           cudaStream_t st);

// ---- k-means (ibp_kmeans.cu)
size_t kmeans_workspace(int64_t n, int64_t v, int wb, int c);
template <typename U>
ibp_status kmeans_impl(const U *data, int64_t n, int64_t v, int c, const int64_t *init_rows,
                       U *masks, U *bitvals, int32_t *clusters, void *ws, size_t ws_bytes,
                       cudaStream_t st);

}  // namespace ibp200
