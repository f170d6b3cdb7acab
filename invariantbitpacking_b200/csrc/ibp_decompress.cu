// ibp_decompress.cu -- decompress_fetch: gather + unpack of fixed-stride compressed rows
// (replaces src/decompress.cu:10-156 and include/decompress/*.cuh).
//
// B200 design
//  * one warp per fetched row; rows come from pinned host memory (zero-copy over PCIe)
//    or HBM.  The warp first reads the row's bitmap (Mw words), sums the stream length
//    from the per-column bit counts, then reads exactly the stream words it needs with
//    16-byte loads into a shared-memory slot -- no speculative over-read, no ring buffer.
//  * decode: lane j of a 32-word chunk takes its bit length, a warp prefix sum gives its
//    stream offset, a funnel read pulls its bits and the Hacker's Delight scatter places
//    them at the non-invariant positions (constant log2(W) steps, no per-run loop);
//    the warp writes 32 consecutive output words per chunk (coalesced).
//  * index arrays: rows are fetched in sorted index order (cub radix sort on only the
//    bits the row count needs) so concurrent warps read neighbouring host pages, and every
//    distinct row crosses PCIe once: repeats are filled by a device-side row copy after
//    the unpack (Zipf-distributed mini-batches repeat hot rows many times).
//  * no allocation, no host synchronisation: everything lives in the caller's workspace
//    and is enqueued on the caller's stream.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "ibp_codec.cuh"
#include "ibp_internal.cuh"

namespace ibp200 {

template <typename U>
struct FetchArgs {
    const U *comp;
    int64_t n, v, mw;
    ColTables<U> t;
    const int32_t *bitmask;
    const int64_t *keys;  // source rows in processing order (nullptr: row k)
    const int64_t *pos;   // output row of each processed row (nullptr: k)
    int64_t nrows;
    bool dedup;           // skip a row equal to the previous key (filled by the copy pass)
    bool raw_only;        // impl 2: plain gather of the stored rows, no decoding
    U *out;
    int32_t *status;
    int64_t slot_words;   // shared-memory words per warp
    int64_t first_words;  // words of the first read of a compressed row
};

template <typename U>
__device__ __forceinline__ void decode_row_warp(const U *__restrict__ buf, int64_t v,
                                                int64_t mw, const ColTables<U> &t,
                                                U *__restrict__ orow) {
    constexpr int W = 8 * sizeof(U);
    const int lane = threadIdx.x & 31;
    const uint32_t *units = reinterpret_cast<const uint32_t *>(buf);
    const U *stream = buf + mw;
    int64_t base = 0;
    for (int64_t c0 = 0; c0 < v; c0 += 32) {
        const int64_t j = c0 + lane;
        const bool in = j < v;
        const bool cj = in && ((units[j >> 5] >> (j & 31)) & 1u);
        const int L = in ? (cj ? (int)__ldg(&t.nb[j]) : W) : 0;
        int incl = L;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (in) {
            const U y = get_bits<U>(stream, base + incl - L, L);
            U x = y;
            if (cj) {
                const U m = __ldg(&t.mask[j]);
                x = (U)(__ldg(&t.bitval[j]) | scatter_bits<U>(y, (U)~m, t.mv + j, (int)v));
            }
            orow[j] = x;
        }
        base += __shfl_sync(0xffffffffu, incl, 31);
    }
}

// Warp copy of row words [w0, w1) from global (host-mapped or device) memory into the same
// word positions of a shared-memory slot: 16-byte loads when the row is 16-byte aligned
// (whole aligned blocks; a block straddling w0 rewrites words already loaded with the same
// values), word loads otherwise.
template <typename U>
__device__ __forceinline__ void load_words(U *__restrict__ buf, const U *__restrict__ row,
                                           int64_t w0, int64_t w1) {
    const int lane = threadIdx.x & 31;
    if ((((uintptr_t)row) & 15) == 0) {
        constexpr int per16 = 16 / sizeof(U);
        const uint4 *r4 = reinterpret_cast<const uint4 *>(row);
        uint4 *b4 = reinterpret_cast<uint4 *>(buf);
        for (int64_t q = w0 / per16 + lane; q < (w1 + per16 - 1) / per16; q += 32) b4[q] = r4[q];
    } else {
        for (int64_t w = w0 + lane; w < w1; w += 32) buf[w] = row[w];
    }
}

template <typename U>
__global__ void __launch_bounds__(256) fetch_rows_kernel(FetchArgs<U> a) {
    constexpr int W = 8 * sizeof(U);
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    U *buf = reinterpret_cast<U *>(smem) + (int64_t)(threadIdx.x >> 5) * a.slot_words;
    const int64_t v = a.v;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t k = warp; k < a.nrows; k += nwarps) {
        const int64_t r = a.keys ? a.keys[k] : k;
        if (a.dedup && k > 0 && a.keys[k - 1] == r) continue;
        if (r < 0 || r >= a.n) {
            if (lane == 0) atomicOr(a.status, kStatusBadIndex);
            continue;
        }
        const int64_t d = a.pos ? a.pos[k] : k;
        const U *row = a.comp + r * v;
        U *orow = a.out + d * v;
        const bool packed = !a.raw_only && ((__ldg(&a.bitmask[r >> 5]) >> (r & 31)) & 1);
        if (!packed) {
            warp_copy<U>(orow, row, v);
            continue;
        }
        // first read: words [0, first) -- the bitmap plus as much of the stream as the
        // caller's average-length hint predicts, in one request per row
        const int64_t first = a.first_words;
        load_words<U>(buf, row, 0, first);
        __syncwarp();
        const uint32_t *units = reinterpret_cast<const uint32_t *>(buf);
        uint32_t bits = 0;
        for (int64_t j = lane; j < v; j += 32)
            bits += ((units[j >> 5] >> (j & 31)) & 1u) ? (uint32_t)__ldg(&a.t.nb[j]) : (uint32_t)W;
        bits = __reduce_add_sync(0xffffffffu, bits);
        const int64_t end = a.mw + (bits + W - 1) / W;  // exact compressed words of the row
        // second read, only for rows longer than the hint
        if (end > first) load_words<U>(buf, row, first, end);
        // words past the stream read as zero (get_bits looks one word ahead; the loaded
        // value there never reaches an output bit, zeroing keeps the slot deterministic)
        __syncwarp();
        if (lane < 2) buf[end + lane] = 0;
        __syncwarp();
        decode_row_warp<U>(buf, v, a.mw, a.t, orow);
        __syncwarp();
    }
}

// Repeats of a row in the sorted index: copy the first occurrence's output row.
template <typename U>
__global__ void __launch_bounds__(256)
fill_repeats_kernel(const int64_t *__restrict__ keys, const int64_t *__restrict__ pos,
                    const int64_t *__restrict__ head, int64_t nrows, int64_t n, int64_t v,
                    U *__restrict__ out) {
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t k = warp; k < nrows; k += nwarps) {
        const int64_t h = head[k];
        if (h == k) continue;
        const int64_t r = keys[k];
        if (r < 0 || r >= n) continue;
        warp_copy<U>(out + pos[k] * v, out + pos[h] * v, v);
    }
}

// head_cand[k] = k where a run of equal keys starts, else 0 (max-scanned into head[]).
__global__ void run_heads_kernel(const int64_t *__restrict__ keys, int64_t nrows,
                                 int64_t *__restrict__ cand, int64_t *__restrict__ iota) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nrows;
         k += (int64_t)gridDim.x * blockDim.x) {
        if (cand) cand[k] = (k == 0 || keys[k] != keys[k - 1]) ? k : 0;
        if (iota) iota[k] = k;
    }
}

struct MaxOp {
    __device__ __forceinline__ int64_t operator()(int64_t a, int64_t b) const {
        return a > b ? a : b;
    }
};

static int sort_end_bit(int64_t n) {
    int b = 1;
    while (b < 63 && ((int64_t)1 << b) < n) ++b;
    return b;
}

struct SortPlan {
    size_t sort_temp = 0, scan_temp = 0;
};

static SortPlan sort_plan(int64_t nidx, int64_t n) {
    SortPlan p;
    const int ni = (int)(nidx > 0 ? nidx : 1);
    cub::DeviceRadixSort::SortPairs(nullptr, p.sort_temp, (const int64_t *)nullptr,
                                    (int64_t *)nullptr, (const int64_t *)nullptr,
                                    (int64_t *)nullptr, ni, 0, sort_end_bit(n));
    cub::DeviceScan::InclusiveScan(nullptr, p.scan_temp, (const int64_t *)nullptr,
                                   (int64_t *)nullptr, MaxOp(), ni);
    return p;
}

size_t decompress_workspace(int64_t nidx, int64_t v, int wb, bool has_index) {
    Sizer s;
    s.take<char>(kStatusBytes);
    s.take<char>(wb == 8 ? tables_bytes<uint64_t>(v) : tables_bytes<uint32_t>(v));
    if (has_index && nidx > 0) {
        // sized for any row count: the sort uses at most 63 key bits
        SortPlan p = sort_plan(nidx, (int64_t)1 << 62);
        s.take<int64_t>(nidx);  // iota
        s.take<int64_t>(nidx);  // sorted keys
        s.take<int64_t>(nidx);  // positions
        s.take<int64_t>(nidx);  // head candidates / heads
        s.take<char>(p.sort_temp > p.scan_temp ? p.sort_temp : p.scan_temp);
    }
    return s.total();
}

template <typename U>
static ibp_status launch_fetch(FetchArgs<U> a, int nblks, int nthreads, cudaStream_t st) {
    if (a.nrows <= 0) return IBP_OK;
    a.slot_words = (int64_t)align_up((size_t)a.v + 4, 16 / sizeof(U));
    const size_t per_warp = (size_t)a.slot_words * sizeof(U);
    int threads = nthreads > 0 ? nthreads : 256;
    threads = threads < 32 ? 32 : (threads > 256 ? 256 : threads / 32 * 32);
    size_t smem = per_warp * (threads / 32);
    const int maxs = device_max_smem_optin();
    while ((int64_t)smem > maxs && threads > 32) {
        threads -= 32;
        smem = per_warp * (threads / 32);
    }
    if ((int64_t)smem > maxs) {
        set_error("rows of %lld words do not fit the fetch kernel's shared-memory slot",
                  (long long)a.v);
        return IBP_ERR_UNSUPPORTED;
    }
    auto kern = fetch_rows_kernel<U>;
    IBP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int64_t blocks = nblks;
    if (blocks <= 0) {
        int per_sm = 0;
        IBP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
        if (per_sm < 1) per_sm = 1;
        blocks = (int64_t)device_sm_count() * per_sm;
        const int64_t need = (a.nrows + threads / 32 - 1) / (threads / 32);
        if (blocks > need) blocks = need;
    }
    const int slot = profile_begin(st);
    kern<<<(unsigned)blocks, threads, smem, st>>>(a);
    IBP_LAUNCHED("fetch_rows_kernel");
    profile_end(slot, st);
    return IBP_OK;
}

template <typename U>
ibp_status decompress_impl(const U *comp, int64_t n, int64_t v, const U *mask,
                           const U *bitval, const int32_t *bitmask, const int64_t *idx,
                           int64_t nidx, bool has_index, int comp_len, U *out, int nblks,
                           int nthreads, int impl, void *ws, size_t ws_bytes, cudaStream_t st) {
    const int wb = sizeof(U);
    const int64_t nrows = has_index ? nidx : n;
    const size_t need = decompress_workspace(nidx, v, wb, has_index);
    if (!ws || ws_bytes < need) {
        set_error("decompress_fetch: workspace of %zu bytes is below the required %zu",
                  ws_bytes, need);
        return IBP_ERR_WORKSPACE;
    }
    Carver c{(char *)ws, 0, ws_bytes};
    int32_t *status = c.take<int32_t>(kStatusBytes / sizeof(int32_t));
    ColTables<U> t = carve_tables<U>(c, v);
    IBP_CUDA(cudaMemsetAsync(status, 0, sizeof(int32_t), st));
    if (nrows <= 0 || v <= 0) return IBP_OK;
    if (impl != 2) IBP_RET(build_tables<U>(mask, bitval, v, t, st));

    FetchArgs<U> a{};
    a.comp = comp;
    a.n = n;
    a.v = v;
    a.mw = meta_bytes(v, wb) / wb;
    a.t = t;
    a.bitmask = bitmask;
    a.nrows = nrows;
    a.raw_only = impl == 2;
    a.out = out;
    a.status = status;
    // first read of a compressed row: the hint (average compressed words) plus one word,
    // rounded up to whole 32-byte sectors; without a hint, the first 128 bytes
    {
        const int64_t sector = 32 / wb;
        int64_t want = (comp_len > 0 && comp_len < v) ? (int64_t)comp_len + 1 : 128 / wb;
        if (want < a.mw + 1) want = a.mw + 1;
        want = (want + sector - 1) / sector * sector;
        a.first_words = want < v ? want : v;
    }
    if (!has_index) return launch_fetch<U>(a, nblks, nthreads, st);

    if (nidx > 0x7fffffffLL) {
        set_error("decompress_fetch: index arrays above 2^31-1 entries are not supported");
        return IBP_ERR_UNSUPPORTED;
    }
    SortPlan p = sort_plan(nidx, (int64_t)1 << 62);
    int64_t *iota = c.take<int64_t>(nidx);
    int64_t *keys = c.take<int64_t>(nidx);
    int64_t *pos = c.take<int64_t>(nidx);
    int64_t *head = c.take<int64_t>(nidx);
    void *temp = c.take<char>(p.sort_temp > p.scan_temp ? p.sort_temp : p.scan_temp);
    size_t temp_bytes = p.sort_temp > p.scan_temp ? p.sort_temp : p.scan_temp;
    const int ni = (int)nidx;
    int blocks = (int)((nidx + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    run_heads_kernel<<<blocks, 256, 0, st>>>(keys, nidx, nullptr, iota);
    IBP_LAUNCHED("run_heads_kernel(iota)");
    size_t tb = temp_bytes;
    IBP_CUDA(cub::DeviceRadixSort::SortPairs(temp, tb, idx, keys, iota, pos, ni, 0,
                                             sort_end_bit(n), st));
    run_heads_kernel<<<blocks, 256, 0, st>>>(keys, nidx, head, nullptr);
    IBP_LAUNCHED("run_heads_kernel(heads)");
    tb = temp_bytes;
    IBP_CUDA(cub::DeviceScan::InclusiveScan(temp, tb, head, head, MaxOp(), ni, st));
    a.keys = keys;
    a.pos = pos;
    a.dedup = true;
    IBP_RET(launch_fetch<U>(a, nblks, nthreads, st));
    int64_t fb = (nidx + 7) / 8;
    const int64_t cap = (int64_t)device_sm_count() * 8;
    if (fb > cap) fb = cap;
    fill_repeats_kernel<U><<<(unsigned)fb, 256, 0, st>>>(keys, pos, head, nidx, n, v, out);
    IBP_LAUNCHED("fill_repeats_kernel");
    return IBP_OK;
}

template ibp_status decompress_impl<uint32_t>(const uint32_t *, int64_t, int64_t,
                                              const uint32_t *, const uint32_t *,
                                              const int32_t *, const int64_t *, int64_t, bool,
                                              int, uint32_t *, int, int, int, void *, size_t,
                                              cudaStream_t);
template ibp_status decompress_impl<uint64_t>(const uint64_t *, int64_t, int64_t,
                                              const uint64_t *, const uint64_t *,
                                              const int32_t *, const int64_t *, int64_t, bool,
                                              int, uint64_t *, int, int, int, void *, size_t,
                                              cudaStream_t);

}  // namespace ibp200
