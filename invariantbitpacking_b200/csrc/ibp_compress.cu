// ibp_compress.cu -- per-row compressed size, in-place bit packing and the condensed layout.
// Replaces include/misc/ibp_misc_{dev,kernels}.cuh (size check), include/compress/*.cuh
// (packer and its launchers) and the size/offset glue of src/compress.cu.
//
// B200 design
//  * sizes: G lanes per row (G = 8/16/32 by row length), a branch-free popc sum and
//    a shuffle reduction; no shared-memory atomics (the reference uses one 256-thread
//    block per row with smem atomics).
//  * packing: one warp per row.  The row is staged in shared memory once (so in-place
//    compression of a pinned host row reads it over PCIe once), every lane gathers its
//    word's non-invariant bits with the Hacker's Delight move masks, a warp prefix sum
//    gives bit offsets, and bits are ORed into a shared-memory copy of the output row
//    (32-bit shared atomics, at most 3 per word).  The finished row goes back with one
//    coalesced pass; an incompressible row compressed in place is not written at all.
//    No global workspace is cudaMalloc'd or freed per call (the reference does both and
//    thereby blocks the host).
#include <cub/device/device_scan.cuh>

#include "ibp_codec.cuh"
#include "ibp_internal.cuh"

namespace ibp200 {

// ------------------------------------------------------------------ sizes
template <typename U, int G>
__global__ void __launch_bounds__(256)
compress_size_kernel(const U *__restrict__ data, int64_t n, int64_t v,
                     const U *__restrict__ mask, const U *__restrict__ bitval,
                     const int64_t *__restrict__ idx, int64_t nrows,
                     int64_t *__restrict__ sizes, unsigned long long *__restrict__ total,
                     int32_t *__restrict__ status) {
    // groups of G lanes; the row loop advances a whole warp at a time so every lane
    // reaches the shuffles of every iteration
    constexpr int RPW = 32 / G;
    const int sub = threadIdx.x & (G - 1);
    const int gin = (threadIdx.x & 31) / G;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long acc = 0;
    for (int64_t wbase = warp * RPW; wbase < nrows; wbase += nwarps * RPW) {
        const int64_t i = wbase + gin;
        const bool live = i < nrows;
        const int64_t r = live ? (idx ? idx[i] : i) : 0;
        const bool ok = live && r >= 0 && r < n;
        uint32_t s = 0;
        if (ok) {
            const U *row = data + r * v;
            for (int64_t j = sub; j < v; j += G) {
                const U m = __ldg(&mask[j]);
                if ((U)(row[j] & m) == __ldg(&bitval[j])) s += popc_w(m);
            }
        }
        s = group_sum<G>(s);
        if (sub == 0 && live) {
            if (ok) {
                const int64_t sz = compressed_bytes(v, (int)sizeof(U), s);
                sizes[i] = sz;
                acc += (unsigned long long)sz;
            } else {
                sizes[i] = 0;
                if (status) atomicOr(status, kStatusBadIndex);
            }
        }
    }
    if (total) {
        acc = group_sum<32>(acc);
        if ((threadIdx.x & 31) == 0 && acc) atomicAdd(total, acc);
    }
}

template <typename U, int G>
static ibp_status launch_sizes(const U *data, int64_t n, int64_t v, const U *mask,
                               const U *bitval, const int64_t *idx, int64_t nrows,
                               int64_t *sizes, int64_t *total, int32_t *status,
                               cudaStream_t st) {
    const int rows_per_block = 256 / G;
    int64_t blocks = (nrows + rows_per_block - 1) / rows_per_block;
    const int64_t cap = (int64_t)device_sm_count() * 8;
    if (blocks > cap) blocks = cap;
    compress_size_kernel<U, G><<<(unsigned)blocks, 256, 0, st>>>(
        data, n, v, mask, bitval, idx, nrows, sizes, (unsigned long long *)total, status);
    IBP_LAUNCHED("compress_size_kernel");
    return IBP_OK;
}

template <typename U>
ibp_status compress_size_impl(const U *data, int64_t n, int64_t v, const U *mask,
                              const U *bitval, const int64_t *idx, int64_t nrows,
                              int64_t *sizes, int64_t *total, int32_t *status,
                              cudaStream_t st) {
    if (nrows <= 0) return IBP_OK;
    if (v >= 32) return launch_sizes<U, 32>(data, n, v, mask, bitval, idx, nrows, sizes, total, status, st);
    if (v >= 16) return launch_sizes<U, 16>(data, n, v, mask, bitval, idx, nrows, sizes, total, status, st);
    return launch_sizes<U, 8>(data, n, v, mask, bitval, idx, nrows, sizes, total, status, st);
}

// ------------------------------------------------------------------ packing
// Packs row `in` (v words in shared memory) into `out_units` (shared, zeroed, v words +
// pad) with a warp.  Returns nothing; bitmap + stream land in out_units.
template <typename U>
__device__ __forceinline__ void pack_row_warp(const U *in, int64_t v, ColTables<U> t,
                                              uint32_t *out_units) {
    constexpr int W = 8 * sizeof(U);
    const int lane = threadIdx.x & 31;
    const int64_t mw = meta_bytes(v, (int)sizeof(U)) / (int64_t)sizeof(U);
    const int64_t stream0 = mw * W;  // stream bit 0 in row bits
    int64_t base = 0;
    for (int64_t c0 = 0; c0 < v; c0 += 32) {
        const int64_t j = c0 + lane;
        bool cj = false;
        int L = 0;
        uint64_t val = 0;
        if (j < v) {
            const U x = in[j];
            const U m = __ldg(&t.mask[j]);
            cj = (U)(x & m) == __ldg(&t.bitval[j]);
            if (cj) {
                L = __ldg(&t.nb[j]);
                val = (uint64_t)gather_bits<U>(x, (U)~m, t.mv + j, (int)v);
            } else {
                L = W;
                val = (uint64_t)x;
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, cj);
        if (lane == 0) out_units[c0 >> 5] = bal;  // bitmap unit (j/32), LSB-first
        // exclusive prefix of L across the warp
        int incl = L;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int64_t off = base + incl - L;
        put_bits<U>(out_units, stream0 + off, val, L);
        base += __shfl_sync(0xffffffffu, incl, 31);
    }
}

template <typename U>
struct PackArgs {
    const U *src;
    int64_t n, v;
    ColTables<U> t;
    const int64_t *idx;
    int64_t nrows;
    U *out;             // fixed-stride output rows (nullptr for condensed)
    U *cond;            // condensed output base (word aligned offsets)
    const int64_t *offsets;
    bool in_place;      // out rows alias src rows one to one
    int32_t *bitmask;
    int32_t *status;
    int64_t row_words;  // smem words per staged row buffer
};

template <typename U>
__global__ void __launch_bounds__(256) pack_rows_kernel(PackArgs<U> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    U *in = reinterpret_cast<U *>(smem) + (int64_t)wib * 2 * a.row_words;
    U *outw = in + a.row_words;
    uint32_t *out_units = reinterpret_cast<uint32_t *>(outw);
    const int64_t v = a.v;
    const int64_t vb = v * (int64_t)sizeof(U);
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < a.nrows; i += nwarps) {
        const int64_t r = a.idx ? a.idx[i] : i;
        if (r < 0 || r >= a.n) {
            if (lane == 0) atomicOr(a.status, kStatusBadIndex);
            continue;
        }
        const U *srow = a.src + r * v;
        warp_copy<U>(in, srow, v);
        __syncwarp();
        uint32_t s = 0;
        for (int64_t j = lane; j < v; j += 32) {
            const U m = __ldg(&a.t.mask[j]);
            if ((U)(in[j] & m) == __ldg(&a.t.bitval[j])) s += popc_w(m);
        }
        s = __reduce_add_sync(0xffffffffu, s);
        const int64_t size = compressed_bytes(v, (int)sizeof(U), s);
        const bool comp = size < vb;
        if (comp) {
            for (int64_t k = lane; k < a.row_words; k += 32) outw[k] = 0;
            __syncwarp();
            pack_row_warp<U>(in, v, a.t, out_units);
            __syncwarp();
        }
        if (a.out) {
            U *orow = a.out + i * v;
            if (comp)
                warp_copy<U>(orow, outw, v);
            else if (!a.in_place)
                warp_copy<U>(orow, in, v);
            if (lane == 0 && comp) atomicOr(&a.bitmask[i >> 5], (int32_t)(1u << (i & 31)));
        } else {
            const int64_t start = i ? a.offsets[i - 1] : 0;
            U *orow = reinterpret_cast<U *>(reinterpret_cast<char *>(a.cond) + start);
            if (comp)
                warp_copy<U>(orow, outw, size / (int64_t)sizeof(U));
            else
                warp_copy<U>(orow, in, v);
        }
        __syncwarp();
    }
}

template <typename U>
static int pack_warps_per_block(int64_t row_words, size_t &smem) {
    const size_t per_warp = 2 * (size_t)row_words * sizeof(U);
    const size_t budget = 96 * 1024;
    int w = (int)(budget / per_warp);
    if (w > 8) w = 8;
    if (w < 1) w = 1;
    smem = per_warp * w;
    return w;
}

template <typename U>
static ibp_status launch_pack(PackArgs<U> a, cudaStream_t st) {
    if (a.nrows <= 0) return IBP_OK;
    a.row_words = (int64_t)align_up((size_t)a.v + 4, 4);
    size_t smem = 0;
    const int wpb = pack_warps_per_block<U>(a.row_words, smem);
    const int maxs = device_max_smem_optin();
    if ((int64_t)smem > maxs) {
        set_error("rows of %lld words do not fit the packer's shared-memory staging",
                  (long long)a.v);
        return IBP_ERR_UNSUPPORTED;
    }
    auto kern = pack_rows_kernel<U>;
    int per_sm = 0;
    IBP_RET(kernel_blocks_per_sm((const void *)kern, wpb * 32, smem, &per_sm));
    int64_t blocks = (a.nrows + wpb - 1) / wpb;
    const int64_t cap = (int64_t)device_sm_count() * per_sm;
    if (blocks > cap) blocks = cap;
    kern<<<(unsigned)blocks, wpb * 32, smem, st>>>(a);
    IBP_LAUNCHED("pack_rows_kernel");
    return IBP_OK;
}

template <typename U>
ibp_status compress_rows_impl(const U *src, int64_t n, int64_t v, ColTables<U> t,
                              const int64_t *idx, int64_t nrows, U *out, bool out_is_src,
                              int32_t *bitmask, int32_t *status, cudaStream_t st) {
    if (nrows > 0) IBP_CUDA(cudaMemsetAsync(bitmask, 0, sizeof(int32_t) * ((nrows + 31) / 32), st));
    PackArgs<U> a{};
    a.src = src;
    a.n = n;
    a.v = v;
    a.t = t;
    a.idx = idx;
    a.nrows = nrows;
    a.out = out;
    a.in_place = out_is_src && idx == nullptr;
    a.bitmask = bitmask;
    a.status = status;
    return launch_pack<U>(a, st);
}

template <typename U>
ibp_status compress_condensed_rows(const U *src, int64_t n, int64_t v, ColTables<U> t,
                                   const int64_t *idx, int64_t nrows, const int64_t *offsets,
                                   U *out, int32_t *status, cudaStream_t st) {
    PackArgs<U> a{};
    a.src = src;
    a.n = n;
    a.v = v;
    a.t = t;
    a.idx = idx;
    a.nrows = nrows;
    a.cond = out;
    a.offsets = offsets;
    a.status = status;
    return launch_pack<U>(a, st);
}

// ------------------------------------------------------------------ gather (staging)
template <typename U>
__global__ void gather_rows_kernel(const U *__restrict__ src, int64_t n, int64_t v,
                                   const int64_t *__restrict__ idx, int64_t nrows,
                                   U *__restrict__ out, int32_t *__restrict__ status) {
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < nrows; i += nwarps) {
        const int64_t r = idx[i];
        if (r < 0 || r >= n) {
            if ((threadIdx.x & 31) == 0) atomicOr(status, kStatusBadIndex);
            continue;
        }
        warp_copy<U>(out + i * v, src + r * v, v);
    }
}

template <typename U>
ibp_status gather_rows_impl(const U *src, int64_t n, int64_t v, const int64_t *idx,
                            int64_t nrows, U *out, int32_t *status, cudaStream_t st) {
    if (nrows <= 0) return IBP_OK;
    int64_t blocks = (nrows + 7) / 8;
    const int64_t cap = (int64_t)device_sm_count() * 8;
    if (blocks > cap) blocks = cap;
    gather_rows_kernel<U><<<(unsigned)blocks, 256, 0, st>>>(src, n, v, idx, nrows, out, status);
    IBP_LAUNCHED("gather_rows_kernel");
    return IBP_OK;
}

// ------------------------------------------------------------------ offsets
size_t inclusive_offsets_workspace(int64_t nrows) {
    size_t temp = 0;
    cub::DeviceScan::InclusiveSum(nullptr, temp, (int64_t *)nullptr, (int64_t *)nullptr,
                                  (int)(nrows > 0 ? nrows : 1));
    return kStatusBytes + align_up(temp, kAlign);
}

__global__ void copy_last_kernel(const int64_t *offsets, int64_t nrows, int64_t *total) {
    *total = nrows > 0 ? offsets[nrows - 1] : 0;
}

ibp_status inclusive_offsets_impl(int64_t *sizes, int64_t nrows, int64_t *total, void *ws,
                                  size_t ws_bytes, cudaStream_t st) {
    if (nrows > 0x7fffffffLL) {
        set_error("condensed offsets: more than 2^31-1 rows");
        return IBP_ERR_UNSUPPORTED;
    }
    if (nrows > 0) {
        size_t temp = 0;
        IBP_CUDA(cub::DeviceScan::InclusiveSum(nullptr, temp, sizes, sizes, (int)nrows, st));
        if (!ws || ws_bytes < kStatusBytes + temp) {
            set_error("condensed offsets: workspace of %zu bytes is below %zu", ws_bytes,
                      kStatusBytes + temp);
            return IBP_ERR_WORKSPACE;
        }
        IBP_CUDA(cub::DeviceScan::InclusiveSum((char *)ws + kStatusBytes, temp, sizes, sizes,
                                               (int)nrows, st));
    }
    if (total) {
        copy_last_kernel<<<1, 1, 0, st>>>(sizes, nrows, total);
        IBP_LAUNCHED("copy_last_kernel");
    }
    return IBP_OK;
}

#define IBP_INST(U)                                                                          \
    template ibp_status compress_size_impl<U>(const U *, int64_t, int64_t, const U *, const U *, \
                                              const int64_t *, int64_t, int64_t *, int64_t *,  \
                                              int32_t *, cudaStream_t);
IBP_INST(uint8_t)
IBP_INST(uint16_t)
IBP_INST(uint32_t)
IBP_INST(uint64_t)
#undef IBP_INST

#define IBP_INST(U)                                                                            \
    template ibp_status compress_rows_impl<U>(const U *, int64_t, int64_t, ColTables<U>,       \
                                              const int64_t *, int64_t, U *, bool, int32_t *,  \
                                              int32_t *, cudaStream_t);                        \
    template ibp_status compress_condensed_rows<U>(const U *, int64_t, int64_t, ColTables<U>,  \
                                                   const int64_t *, int64_t, const int64_t *,  \
                                                   U *, int32_t *, cudaStream_t);              \
    template ibp_status gather_rows_impl<U>(const U *, int64_t, int64_t, const int64_t *,      \
                                            int64_t, U *, int32_t *, cudaStream_t);
IBP_INST(uint32_t)
IBP_INST(uint64_t)
#undef IBP_INST

}  // namespace ibp200
