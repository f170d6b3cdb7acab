// ibp_decompress.cu -- decompress_fetch: gather + unpack of fixed-stride compressed rows
// (replaces src/decompress.cu:10-156 and include/decompress/).
//
// B200 design
//  * rows come from pinned host memory (zero-copy over PCIe) or HBM.  A warp takes a chunk
//    of 32 consecutive (sorted) positions from a global work counter, loads their keys,
//    output positions and bitmask bits lane-parallel (one round trip for 32 rows), and then
//    loads the first read of up to kRowsInFlight distinct rows into registers (16-byte loads,
//    all rows before any store) and parks them in shared-memory slots, so several PCIe
//    round trips overlap per warp.
//  * the first read of a compressed row is sized by the caller's average-length hint
//    (comp_len), rounded to whole 32-byte sectors: one request per row when the hint holds;
//    the bitmap then gives the exact length and a second read fetches any remainder.
//  * decode: lane j of a 32-word chunk takes its bit length, a warp prefix sum gives its
//    stream offset, a funnel read pulls its bits and the Hacker's Delight scatter places
//    them at the non-invariant positions (log2(W) branch-free steps).  For rows of up to 64
//    words the per-column tables (mask, bitval, kept bits, move masks) live in registers,
//    loaded once per warp; longer rows read them through the L1 cache.
//  * index arrays: rows are fetched in sorted index order (cub radix sort on only the bits
//    the row count needs) so concurrent warps read neighbouring host pages, and each
//    distinct row crosses PCIe once; repeats are filled afterwards by a copy kernel that
//    reads each source row once per 32 positions (Zipf mini-batches repeat hot rows a lot).
//  * no allocation, no host synchronisation: everything lives in the caller's workspace
//    and is enqueued on the caller's stream.
#include <cub/device/device_radix_sort.cuh>

#include "ibp_codec.cuh"
#include "ibp_internal.cuh"

namespace ibp200 {

constexpr int kFetchThreads = 256;  // 8 warps per block
constexpr int kRowsInFlight = 4;    // first reads a warp keeps outstanding

template <typename U>
struct FetchArgs {
    const U *comp;
    int64_t n, v, mw;
    ColTables<U> t;
    const int32_t *bitmask;
    const int64_t *keys;  // source rows in processing order (nullptr: position k is row k)
    const int64_t *pos;   // output row of each position (nullptr: k)
    int64_t nrows;
    bool dedup;           // positions whose key equals the previous one are left to the fill
    bool raw_only;        // impl 2: plain gather of the stored rows, no decoding
    U *out;
    int32_t *status;
    unsigned long long *work;  // chunk counter, zero at launch
    int64_t slot_words;   // shared-memory words per row slot
    int64_t first_words;  // words of the first read of a compressed row
    int slots;            // row slots per warp (<= kRowsInFlight)
};

// Copy row words [w0, w1) into the same positions of a shared slot: 16-byte loads when the
// row is 16-byte aligned (whole aligned blocks; a block straddling w0 rewrites words already
// present with the same values), word loads otherwise.
template <typename U>
__device__ __forceinline__ void issue_words(U *__restrict__ slot, const U *__restrict__ row,
                                            int64_t w0, int64_t w1) {
    const int lane = threadIdx.x & 31;
    if ((((uintptr_t)row) & 15) == 0) {
        constexpr int per16 = 16 / sizeof(U);
        const uint4 *r4 = reinterpret_cast<const uint4 *>(row);
        uint4 *b4 = reinterpret_cast<uint4 *>(slot);
        for (int64_t q = w0 / per16 + lane; q < (w1 + per16 - 1) / per16; q += 32) b4[q] = r4[q];
    } else {
        for (int64_t w = w0 + lane; w < w1; w += 32) slot[w] = row[w];
    }
}

// ------------------------------------------------------------------ column tables
// Tables of the columns j = lane + 32*c, c < NC, held in registers (NC = 1 or 2), or read
// through L1 from the workspace copy (NC = 0, any row length).
template <typename U, int NC>
struct LaneTables {
    static constexpr int LW = LogW<U>::value;
    U m[NC > 0 ? NC : 1], bv[NC > 0 ? NC : 1], mv[NC > 0 ? NC : 1][LW];
    int nb[NC > 0 ? NC : 1];

    __device__ __forceinline__ void load(const ColTables<U> &t, int64_t v) {
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int64_t j = lane + 32 * c;
            const bool in = j < v;
            m[c] = in ? t.mask[j] : (U)0;
            bv[c] = in ? t.bitval[j] : (U)0;
            nb[c] = in ? (int)t.nb[j] : 0;
#pragma unroll
            for (int i = 0; i < LW; ++i) mv[c][i] = in ? t.mv[i * v + j] : (U)0;
        }
    }
};

template <typename U>
__device__ __forceinline__ U scatter_regs(U y, U sel, const U *mv) {
    constexpr int LW = LogW<U>::value;
#pragma unroll
    for (int i = LW - 1; i >= 0; --i) {
        const U t = (U)(y << (1 << i));
        y = (U)((y & ~mv[i]) | (t & mv[i]));
    }
    return (U)(y & sel);
}

// Decode one compressed row from its shared-memory slot (bitmap at word 0, stream at word
// mw, zero words after the stream) into the output row.
template <typename U, int NC>
__device__ __forceinline__ void decode_row(const U *__restrict__ buf, int64_t v, int64_t mw,
                                           const ColTables<U> &t, const LaneTables<U, NC> &lt,
                                           U *__restrict__ orow) {
    constexpr int W = 8 * sizeof(U);
    const int lane = threadIdx.x & 31;
    const uint32_t *units = reinterpret_cast<const uint32_t *>(buf);
    const U *stream = buf + mw;
    int64_t base = 0;
    auto chunk = [&](int64_t c0, U m, U bv, int nbits, const U *mv, int stride) {
        const int64_t j = c0 + lane;
        const bool in = j < v;
        const bool cj = in && ((units[j >> 5] >> (j & 31)) & 1u);
        const int L = in ? (cj ? nbits : W) : 0;
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
                if (stride == 0)
                    x = (U)(bv | scatter_regs<U>(y, (U)~m, mv));
                else
                    x = (U)(bv | scatter_bits<U>(y, (U)~m, mv, stride));
            }
            orow[j] = x;
        }
        base += __shfl_sync(0xffffffffu, incl, 31);
    };
    if constexpr (NC > 0) {
#pragma unroll
        for (int c = 0; c < NC; ++c)
            if (32 * c < v) chunk(32 * c, lt.m[c], lt.bv[c], lt.nb[c], lt.mv[c], 0);
    } else {
        for (int64_t c0 = 0; c0 < v; c0 += 32) {
            const int64_t j = c0 + lane;
            const bool in = j < v;
            chunk(c0, in ? __ldg(&t.mask[j]) : (U)0, in ? __ldg(&t.bitval[j]) : (U)0,
                  in ? (int)__ldg(&t.nb[j]) : 0, t.mv + (in ? j : 0), (int)v);
        }
    }
}

// Exact compressed words of the row whose bitmap is in the slot (bitmap + stream).
template <typename U, int NC>
__device__ __forceinline__ int64_t row_words(const U *__restrict__ buf, int64_t v, int64_t mw,
                                             const ColTables<U> &t,
                                             const LaneTables<U, NC> &lt) {
    constexpr int W = 8 * sizeof(U);
    const int lane = threadIdx.x & 31;
    const uint32_t *units = reinterpret_cast<const uint32_t *>(buf);
    uint32_t bits = 0;
    if constexpr (NC > 0) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int64_t j = lane + 32 * c;
            if (j < v) bits += ((units[j >> 5] >> (j & 31)) & 1u) ? (uint32_t)lt.nb[c] : (uint32_t)W;
        }
    } else {
        for (int64_t j = lane; j < v; j += 32)
            bits += ((units[j >> 5] >> (j & 31)) & 1u) ? (uint32_t)__ldg(&t.nb[j]) : (uint32_t)W;
    }
    bits = __reduce_add_sync(0xffffffffu, bits);
    return mw + (bits + W - 1) / W;
}

// ------------------------------------------------------------------ fetch kernel
template <typename U, int NC>
__global__ void __launch_bounds__(kFetchThreads) fetch_rows_kernel(FetchArgs<U> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    U *slots = reinterpret_cast<U *>(smem) + (int64_t)(threadIdx.x >> 5) * a.slots * a.slot_words;
    const int64_t v = a.v;
    LaneTables<U, NC> lt;
    if (!a.raw_only) lt.load(a.t, v);
    for (;;) {
        unsigned long long chunk = 0;
        if (lane == 0) chunk = atomicAdd(a.work, 1ull);
        chunk = __shfl_sync(0xffffffffu, chunk, 0);
        const int64_t k0 = (int64_t)chunk * 32;
        if (k0 >= a.nrows) break;
        // lane-parallel metadata of the chunk's 32 positions
        const int64_t k = k0 + lane;
        const bool valid = k < a.nrows;
        const int64_t key = valid ? (a.keys ? a.keys[k] : k) : -1;
        bool head = valid;
        if (a.dedup) {
            int64_t prev = __shfl_up_sync(0xffffffffu, key, 1);
            if (lane == 0) prev = k0 > 0 ? a.keys[k0 - 1] : key - 1;
            head = valid && key != prev;
        }
        const bool bad = head && (key < 0 || key >= a.n);
        if (bad) atomicOr(a.status, kStatusBadIndex);
        head = head && !bad;
        const int64_t dst = head ? (a.pos ? a.pos[k] : k) : 0;
        const bool packed =
            head && !a.raw_only && ((__ldg(&a.bitmask[key >> 5]) >> (key & 31)) & 1);
        unsigned hm = __ballot_sync(0xffffffffu, head);
        while (hm) {
            // up to `slots` heads: issue all their first reads, then decode them in turn
            int lid[kRowsInFlight];
            int cnt = 0;
#pragma unroll
            for (int s = 0; s < kRowsInFlight; ++s) {
                lid[s] = 0;
                if (s < a.slots && hm) {
                    lid[s] = __ffs(hm) - 1;
                    hm &= hm - 1;
                    ++cnt;
                }
            }
            // first reads of the group's compressed rows: every lane's 16-byte pieces of all
            // rows are loaded into registers before any is stored, so the rows' PCIe round
            // trips overlap; rows that are not 16-byte aligned or longer than 1 KiB take a
            // plain loop
            {
                constexpr int per16 = 16 / sizeof(U);
                const int64_t nq = (a.first_words + per16 - 1) / per16;
                uint4 stage[kRowsInFlight][2];
                bool fast[kRowsInFlight];
#pragma unroll
                for (int s = 0; s < kRowsInFlight; ++s) {
                    fast[s] = false;
                    if (s < cnt) {
                        const int64_t r = __shfl_sync(0xffffffffu, key, lid[s]);
                        const bool pk = __shfl_sync(0xffffffffu, (int)packed, lid[s]);
                        const U *row = a.comp + r * v;
                        fast[s] = pk && ((((uintptr_t)row) & 15) == 0) && nq <= 64;
                        if (fast[s]) {
                            const uint4 *r4 = reinterpret_cast<const uint4 *>(row);
                            if (lane < nq) stage[s][0] = r4[lane];
                            if (lane + 32 < nq) stage[s][1] = r4[lane + 32];
                        } else if (pk) {
                            issue_words<U>(slots + s * a.slot_words, row, 0, a.first_words);
                        }
                    }
                }
#pragma unroll
                for (int s = 0; s < kRowsInFlight; ++s) {
                    if (fast[s]) {
                        uint4 *b4 = reinterpret_cast<uint4 *>(slots + s * a.slot_words);
                        if (lane < nq) b4[lane] = stage[s][0];
                        if (lane + 32 < nq) b4[lane + 32] = stage[s][1];
                    }
                }
            }
            __syncwarp();
#pragma unroll
            for (int s = 0; s < kRowsInFlight; ++s) {
                if (s < cnt) {
                    const int64_t r = __shfl_sync(0xffffffffu, key, lid[s]);
                    const int64_t d = __shfl_sync(0xffffffffu, dst, lid[s]);
                    const bool pk = __shfl_sync(0xffffffffu, (int)packed, lid[s]);
                    const U *row = a.comp + r * v;
                    U *orow = a.out + d * v;
                    if (!pk) {
                        warp_copy<U>(orow, row, v);
                        continue;
                    }
                    U *buf = slots + s * a.slot_words;
                    const int64_t end = row_words<U, NC>(buf, v, a.mw, a.t, lt);
                    if (end >= v) {
                        // a bitmap claiming a stream as long as the raw row cannot come from
                        // this mask: report it and leave the output row alone
                        if (lane == 0) atomicOr(a.status, kStatusCorruptRow);
                        continue;
                    }
                    if (end > a.first_words) {  // longer than the hint: fetch the rest
                        issue_words<U>(buf, row, a.first_words, end);
                    }
                    __syncwarp();
                    // words past the stream read as zero (get_bits looks one word ahead;
                    // the value there never reaches an output bit)
                    if (lane < 2) buf[end + lane] = 0;
                    __syncwarp();
                    decode_row<U, NC>(buf, v, a.mw, a.t, lt, orow);
                    __syncwarp();
                }
            }
        }
    }
}

// ------------------------------------------------------------------ repeats
// First position of `target` in the sorted keys[0..hi] (keys[hi] == target): a 32-way
// search, one probe per lane per round.
__device__ __forceinline__ int64_t first_occurrence(const int64_t *__restrict__ keys, int64_t hi,
                                                    int64_t target) {
    const int lane = threadIdx.x & 31;
    int64_t lo = 0;  // invariant: keys[lo - 1] < target (or lo == 0), keys[hi] == target
    while (lo < hi) {
        const int64_t step = (hi - lo + 31) / 32;
        int64_t p = lo + (int64_t)lane * step;
        if (p > hi) p = hi;
        const unsigned less = __ballot_sync(0xffffffffu, keys[p] < target);
        const int cnt = __popc(less);
        if (cnt == 0) break;
        const int64_t plast = lo + (int64_t)(cnt - 1) * step;
        if (cnt < 32) {
            const int64_t pnext = lo + (int64_t)cnt * step;
            if (pnext < hi) hi = pnext;
        }
        lo = plast + 1;
    }
    return lo;
}

// Every position whose key repeats the previous one gets a copy of the output row decoded
// for the first position of its run.  A warp takes 32 positions; each distinct source row
// is read once and written to all of its positions in the chunk.
template <typename U>
__global__ void __launch_bounds__(256)
fill_repeats_kernel(const int64_t *__restrict__ keys, const int64_t *__restrict__ pos,
                    int64_t nrows, int64_t n, int64_t v, U *__restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const bool vec = (((uintptr_t)out) & 15) == 0 && ((v * (int64_t)sizeof(U)) & 15) == 0;
    for (int64_t k0 = warp * 32; k0 < nrows; k0 += nwarps * 32) {
        const int64_t k = k0 + lane;
        const bool valid = k < nrows;
        const int64_t key = valid ? keys[k] : -1;
        int64_t prev = __shfl_up_sync(0xffffffffu, key, 1);
        if (lane == 0) prev = k0 > 0 ? keys[k0 - 1] : key - 1;
        const bool head = valid && key != prev;
        const unsigned hb = __ballot_sync(0xffffffffu, head);
        if (__ballot_sync(0xffffffffu, valid && !head) == 0) continue;
        // run start of the chunk's first position when its run began in an earlier chunk
        int64_t h0 = k0;
        if (!(hb & 1u)) h0 = first_occurrence(keys, k0, __shfl_sync(0xffffffffu, key, 0));
        const unsigned below = hb & (lane == 31 ? 0xffffffffu : ((2u << lane) - 1u));
        const int64_t h = below ? k0 + (31 - __clz(below)) : h0;
        const bool dup = valid && !head && key >= 0 && key < n;
        const int64_t d = dup ? pos[k] : 0;
        unsigned dm = __ballot_sync(0xffffffffu, dup);
        while (dm) {
            const int64_t hs = __shfl_sync(0xffffffffu, h, __ffs(dm) - 1);
            const unsigned same = __ballot_sync(0xffffffffu, dup && h == hs) & dm;
            dm &= ~same;
            const U *src = out + pos[hs] * v;
            if (vec) {
                const int64_t n16 = v * (int64_t)sizeof(U) / 16;
                for (int64_t q0 = 0; q0 < n16; q0 += 32) {
                    const int64_t q = q0 + lane;
                    uint4 x = make_uint4(0, 0, 0, 0);
                    if (q < n16) x = reinterpret_cast<const uint4 *>(src)[q];
                    unsigned m = same;
                    while (m) {
                        const int j = __ffs(m) - 1;
                        m &= m - 1;
                        const int64_t dj = __shfl_sync(0xffffffffu, d, j);
                        if (q < n16) reinterpret_cast<uint4 *>(out + dj * v)[q] = x;
                    }
                }
            } else {
                for (int64_t w0 = 0; w0 < v; w0 += 32) {
                    const int64_t w = w0 + lane;
                    const U x = w < v ? src[w] : (U)0;
                    unsigned m = same;
                    while (m) {
                        const int j = __ffs(m) - 1;
                        m &= m - 1;
                        const int64_t dj = __shfl_sync(0xffffffffu, d, j);
                        if (w < v) out[dj * v + w] = x;
                    }
                }
            }
        }
    }
}

// Sort inputs: positions 0..nrows-1, and the keys with every out-of-range index replaced by
// n, so that the radix sort over the bits of n orders all keys exactly (the fetch kernel
// then flags the n's as bad indices, and they form one run at the end).
__global__ void sort_inputs_kernel(const int64_t *__restrict__ idx, int64_t nrows, int64_t n,
                                   int64_t *__restrict__ keys_in, int64_t *__restrict__ iota) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nrows;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = idx[k];
        keys_in[k] = (r >= 0 && r < n) ? r : n;
        iota[k] = k;
    }
}

// Key bits the sort needs for values 0..n.
static int sort_end_bit(int64_t n) {
    int b = 1;
    while (b < 63 && ((int64_t)1 << b) <= n) ++b;
    return b;
}

static size_t sort_temp_bytes(int64_t nidx) {
    size_t temp = 0;
    const int ni = (int)(nidx > 0 ? nidx : 1);
    // sized for any row count: the sort uses at most 63 key bits
    cub::DeviceRadixSort::SortPairs(nullptr, temp, (const int64_t *)nullptr, (int64_t *)nullptr,
                                    (const int64_t *)nullptr, (int64_t *)nullptr, ni, 0, 63);
    return temp;
}

size_t decompress_workspace(int64_t nidx, int64_t v, int wb, bool has_index) {
    Sizer s;
    s.take<char>(kStatusBytes);
    s.take<char>(wb == 8 ? tables_bytes<uint64_t>(v) : tables_bytes<uint32_t>(v));
    if (has_index && nidx > 0) {
        s.take<int64_t>(nidx);  // iota
        s.take<int64_t>(nidx);  // sanitised keys
        s.take<int64_t>(nidx);  // sorted keys
        s.take<int64_t>(nidx);  // positions
        s.take<char>(sort_temp_bytes(nidx));
    }
    return s.total();
}

template <typename U, int NC>
static ibp_status launch_fetch_nc(FetchArgs<U> a, int nblks, int nthreads, cudaStream_t st) {
    const size_t slot_bytes = (size_t)a.slot_words * sizeof(U);
    int threads = nthreads > 0 ? nthreads : kFetchThreads;
    threads = threads < 32 ? 32 : (threads > kFetchThreads ? kFetchThreads : threads / 32 * 32);
    const int maxs = device_max_smem_optin();
    // row slots per warp: up to kRowsInFlight within ~96 KB per block; long rows get fewer
    // slots and then fewer warps
    int slots = kRowsInFlight;
    while (slots > 1 && slot_bytes * slots * (threads / 32) > 96 * 1024) --slots;
    while (threads > 32 && slot_bytes * slots * (threads / 32) > (size_t)maxs) threads -= 32;
    const size_t smem = slot_bytes * slots * (threads / 32);
    if ((int64_t)smem > maxs) {
        set_error("rows of %lld words do not fit the fetch kernel's shared-memory slot",
                  (long long)a.v);
        return IBP_ERR_UNSUPPORTED;
    }
    a.slots = slots;
    auto kern = fetch_rows_kernel<U, NC>;
    IBP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int64_t blocks = nblks;
    if (blocks <= 0) {
        int per_sm = 0;
        IBP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
        if (per_sm < 1) per_sm = 1;
        blocks = (int64_t)device_sm_count() * per_sm;
    }
    const int64_t chunks = (a.nrows + 31) / 32;
    const int64_t need = (chunks + threads / 32 - 1) / (threads / 32);
    if (blocks > need) blocks = need;
    const int slot = profile_begin(st);
    kern<<<(unsigned)blocks, threads, smem, st>>>(a);
    IBP_LAUNCHED("fetch_rows_kernel");
    profile_end(slot, st);
    return IBP_OK;
}

template <typename U>
static ibp_status launch_fetch(FetchArgs<U> a, int nblks, int nthreads, cudaStream_t st) {
    if (a.nrows <= 0) return IBP_OK;
    a.slot_words = (int64_t)align_up((size_t)a.v + 2, 16 / sizeof(U));
    if (a.raw_only || a.v > 64) return launch_fetch_nc<U, 0>(a, nblks, nthreads, st);
    if (a.v > 32) return launch_fetch_nc<U, 2>(a, nblks, nthreads, st);
    return launch_fetch_nc<U, 1>(a, nblks, nthreads, st);
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
    // status word (offset 0) and the fetch work counter (offset 64)
    IBP_CUDA(cudaMemsetAsync(status, 0, 128, st));
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
    a.work = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(status) + 64);
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
    int64_t *iota = c.take<int64_t>(nidx);
    int64_t *keys_in = c.take<int64_t>(nidx);
    int64_t *keys = c.take<int64_t>(nidx);
    int64_t *pos = c.take<int64_t>(nidx);
    size_t temp_bytes = sort_temp_bytes(nidx);
    void *temp = c.take<char>(temp_bytes);
    int blocks = (int)((nidx + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    sort_inputs_kernel<<<blocks, 256, 0, st>>>(idx, nidx, n, keys_in, iota);
    IBP_LAUNCHED("sort_inputs_kernel");
    IBP_CUDA(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys, iota, pos,
                                             (int)nidx, 0, sort_end_bit(n), st));
    a.keys = keys;
    a.pos = pos;
    a.dedup = true;
    IBP_RET(launch_fetch<U>(a, nblks, nthreads, st));
    int64_t fb = (nidx + 255) / 256;
    const int64_t cap = (int64_t)device_sm_count() * 8;
    if (fb > cap) fb = cap;
    fill_repeats_kernel<U><<<(unsigned)fb, 256, 0, st>>>(keys, pos, nidx, n, v, out);
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
