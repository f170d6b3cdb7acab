// ibp_decompress.cu -- decompress_fetch: gather + unpack of fixed-stride compressed rows
// (replaces src/decompress.cu:10-156 and include/decompress/).
//
// B200 design
//  * rows come from pinned host memory (zero-copy over PCIe) or HBM.  A warp takes a chunk
//    of consecutive positions from a global work counter (up to its row slots for host
//    rows, so the rows the grid has in flight stay close together; 32 for HBM rows; fewer
//    towards the end of the work so the last chunks finish together), loads their keys,
//    output positions and bitmask bits lane-parallel, and then loads the first read of up
//    to kRowsInFlight distinct rows into registers (16-byte loads, all rows before any
//    store) and parks them in shared-memory slots, so several PCIe round trips overlap per
//    warp; the rows that need more than their first read get their tails the same way.
//  * the first read of a compressed row is the caller's average-length hint (comp_len)
//    rounded up to whole 32-byte sectors: one round trip per row when the hint holds.
//    Rows longer than 256 words get slots for twice the hint only; a row that outgrows its
//    slot decodes straight from its source.
//  * decode: lane j of a 32-word chunk takes its bit length, a warp prefix sum gives its
//    stream offset, a funnel read pulls its bits and the Hacker's Delight scatter places
//    them at the non-invariant positions (log2(W) branch-free steps).  For rows of up to 64
//    words the per-column tables (mask, bitval, kept bits, move masks) live in registers,
//    loaded once per warp; longer rows read them through the L1 cache, four chunks at a
//    time, and place the bits of columns that keep at most 4 directly from the mask.
//  * index arrays: each distinct row crosses the link once.  Dense batches of host rows (a
//    quarter of the rows or more) and raw gathers are fetched in sorted index order (cub
//    radix sort on only the bits the row count needs) so concurrent warps read neighbouring
//    host pages.  Compressed rows (fixed-stride or condensed) in HBM, and sparse batches of
//    them in host memory, where order gains little, claim rows in an open-addressing hash
//    table instead: inside the fetch for host rows (hidden behind PCIe), in a claim pass
//    that lists the distinct rows for HBM rows.  Repeats (Zipf mini-batches repeat hot
//    rows a lot) copy their first occurrence's output row: inside the fetch for host rows,
//    once that row is published in the table (so the copies overlap the PCIe reads), and
//    in a copy kernel afterwards for the other modes.
//  * no allocation, no host synchronisation: everything lives in the caller's workspace
//    and is enqueued on the caller's stream.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>

#include "ibp_codec.cuh"
#include "ibp_fetch.cuh"
#include "ibp_internal.cuh"

namespace ibp200 {

constexpr int kFetchThreads = 256;  // 8 warps per block

template <typename U>
struct FetchArgs {
    RowSet<U> s;
    const int64_t *keys;  // source rows in processing order (nullptr: position k is row k)
    const int64_t *pos;   // output row of each position (nullptr: k)
    int64_t nrows;
    bool dedup;           // positions whose key equals the previous one are left to the fill
    bool raw_only;        // impl 2: plain gather of the stored rows, no decoding
    U *out;
    int32_t *status;
    unsigned long long *work;  // chunk counter, zero at launch
    int64_t slot_words;   // shared-memory words per row slot
    int slots;            // row slots per warp (<= kRowsInFlight)
    int upos;             // positions per chunk the grid was sized for (unit_positions)
    int gmax;             // largest chunk a warp takes (positions); 0: its row slots
    bool async_rows;      // rows in device memory: first reads as asynchronous copies
    bool device_rows;     // rows in device memory
    ClaimTable claims;    // in-fetch claims (keys == nullptr: none); repeats are copied
                          // inside the fetch
    const int64_t *list;  // positions to fetch (claimed heads), or nullptr: all positions
    const unsigned long long *list_len;  // entries of `list` (device)
};

// ------------------------------------------------------------------ hashed dedup
// (row_hash, hash_claim_slot and the in-fetch claim helpers are in ibp_fetch.cuh)
constexpr uint64_t kRecordPacked = 1ull << 63;  // head record: the row is stored compressed

// Claim pass of a hashed fetch: every position claims its row; the positions that win are
// appended to `heads` (one atomic per block and pass, so the list's counter is not a hot
// spot), and the fetch kernel then walks distinct rows only, 32 to a chunk.  Out-of-range
// rows are flagged here and never claimed.  256 threads per block, P positions each.
// bitmask != nullptr: each listed head is a record of two words, its position (bit 63 set
// when the row is stored compressed) and its row, so that a fetch reads one 16-byte record
// per row instead of a position, then the index entry it points to, then the bitmask word.
// P positions per thread and pass: 2 when one position per thread would need more than one
// wave of resident blocks (fewer block-wide rounds), else 1 (more blocks for small batches).
template <int P>
__global__ void __launch_bounds__(256)
claim_heads_kernel(const int64_t *__restrict__ idx, int64_t nidx, int64_t n, int64_t *hkeys,
                   int64_t *hpos, int64_t hslots, int64_t *__restrict__ heads,
                   unsigned long long *nheads, int32_t *status,
                   const int32_t *__restrict__ bitmask) {
    const bool records = bitmask != nullptr;
    __shared__ unsigned counts[8];
    __shared__ unsigned long long block_base;
    // the block's own table of the rows its 256 x P positions hold (empty: ~0), so that a hot
    // row of a skewed batch is claimed once per block: every claim of one row reads the same
    // global slot, which one L2 slice serves
    constexpr int kBlockSlots = 512 * P;
    __shared__ unsigned long long btab[kBlockSlots];
    for (int i = threadIdx.x; i < kBlockSlots; i += 256) btab[i] = ~0ull;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    for (int64_t b0 = (int64_t)blockIdx.x * 256 * P; b0 < nidx;
         b0 += (int64_t)gridDim.x * 256 * P) {
        int64_t k[P], key[P];
        bool ok[P], head[P];
        int32_t bmw[P];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            k[p] = b0 + p * 256 + threadIdx.x;
            key[p] = k[p] < nidx ? idx[k[p]] : 0;
        }
        // the table and status words are cleared by the kernel before this one
        grid_dep_wait();
        grid_dep_release();
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const bool bad = k[p] < nidx && (key[p] < 0 || key[p] >= n);
            if (bad) atomicOr(status, kStatusBadIndex);
            ok[p] = k[p] < nidx && !bad;
        }
#pragma unroll
        for (int p = 0; p < P; ++p) {
            // the row's bitmask word, loaded before the claim so that the latencies overlap
            bmw[p] = records && ok[p] ? __ldg(&bitmask[key[p] >> 5]) : 0;
        }
        unsigned hm[P];
        unsigned total = 0;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            // one claim per distinct row of the warp (the lowest lane holding it)
            const unsigned same = __match_any_sync(0xffffffffu, ok[p] ? key[p] : (int64_t)-1);
            bool lead = ok[p] && (__ffs(same) - 1) == lane;
            if (lead) {
                uint32_t h = (uint32_t)row_hash(key[p], kBlockSlots);
                for (int probe = 0; probe < kBlockSlots; ++probe) {
                    const unsigned long long old =
                        atomicCAS(&btab[h], ~0ull, (unsigned long long)key[p]);
                    if (old == ~0ull) break;  // the block's first position of this row
                    if (old == (unsigned long long)key[p]) {
                        lead = false;
                        break;
                    }
                    h = (h + 1) & (kBlockSlots - 1);
                }
            }
            head[p] = false;
            if (lead) {
                const int64_t slot = hash_claim_slot(hkeys, hslots, key[p], head[p]);
                if (head[p]) hpos[slot] = k[p];
            }
            hm[p] = __ballot_sync(0xffffffffu, head[p]);
            total += __popc(hm[p]);
        }
        if (lane == 0) counts[wid] = total;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned run = 0;
            for (int w = 0; w < 8; ++w) {
                const unsigned c = counts[w];
                counts[w] = run;
                run += c;
            }
            block_base = run ? atomicAdd(nheads, (unsigned long long)run) : 0ull;
        }
        __syncthreads();
        unsigned long long at = block_base + counts[wid];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const unsigned long long my = at + __popc(hm[p] & below);
            if (head[p] && !records) heads[my] = k[p];
            if (head[p] && records) {
                const bool packed = (bmw[p] >> (key[p] & 31)) & 1;
                reinterpret_cast<longlong2 *>(heads)[my] = make_longlong2(
                    packed ? (int64_t)((uint64_t)k[p] | kRecordPacked) : k[p], key[p]);
            }
            at += __popc(hm[p]);
        }
        for (int i = threadIdx.x; i < kBlockSlots; i += 256) btab[i] = ~0ull;
        __syncthreads();  // counts, block_base and btab are rewritten by the next pass
    }
}

// Repeats of a hashed fetch whose claims came from claim_heads_kernel: each position whose
// row another position claimed copies that position's output row (copy_rows, four rows at
// a time per warp).  The rows it copies were written by the fetch kernel before it, so they
// are read through L1: the hot rows of a skewed batch then leave L2 once per SM rather than
// once per copy (one L2 slice holds each 128-byte line of a row, and a Zipf(1.1) batch of
// 400k positions over 2.4M rows copies its hottest row ~48k times); the claim table,
// written by the claim pass, is read the same way.
constexpr int kFillThreads = 256;

__device__ __forceinline__ int64_t hash_find(const int64_t *__restrict__ keys,
                                             const int64_t *__restrict__ pos, int64_t slots,
                                             int64_t key) {
    uint64_t h = row_hash(key, slots);
    for (int64_t probe = 0; probe < slots; ++probe) {
        const int64_t kk = __ldg(&keys[h]);
        if (kk == key) return __ldg(&pos[h]);
        if (kk == -1) return -1;
        h = h + 1 == (uint64_t)slots ? 0 : h + 1;
    }
    return -1;
}

template <typename U>
__global__ void __launch_bounds__(kFillThreads)
fill_hashed_kernel(const int64_t *__restrict__ idx, int64_t nrows, int64_t n,
                   const int64_t *__restrict__ hkeys, const int64_t *__restrict__ hpos,
                   int64_t hslots, U *__restrict__ out, int64_t v) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const bool vec_rows = ((v * (int64_t)sizeof(U)) & 15) == 0 && (((uintptr_t)out) & 15) == 0;
    for (int64_t k0 = warp * 32; k0 < nrows; k0 += nwarps * 32) {
        const int64_t k = k0 + lane;
        const int64_t key = k < nrows ? idx[k] : -1;
        int64_t hp = -1;
        if (key >= 0 && key < n) hp = hash_find(hkeys, hpos, hslots, key);
        const bool rep = hp >= 0 && hp != k;
        // the first occurrences' rows are written by the kernel before this one
        grid_dep_wait();
        copy_rows<U, true>(__ballot_sync(0xffffffffu, rep), out + (rep ? hp : 0) * v,
                           out + (rep ? k : 0) * v, v, vec_rows);
    }
}

// One wave of resident blocks, each warp striding over chunks of 32 positions.
template <typename U>
static ibp_status launch_fill_hashed(const int64_t *idx, int64_t nidx, int64_t n,
                                     const int64_t *hkeys, const int64_t *hpos, int64_t slots,
                                     U *out, int64_t v, cudaStream_t st) {
    auto kern = fill_hashed_kernel<U>;
    int per_sm = 0;
    IBP_RET(kernel_blocks_per_sm((const void *)kern, kFillThreads, 0, &per_sm));
    const int64_t fb = std::min<int64_t>((nidx + kFillThreads - 1) / kFillThreads,
                                         (int64_t)device_sm_count() * per_sm);
    IBP_CUDA(launch_dependent(kern, (unsigned)fb, kFillThreads, 0, st, idx, nidx, n, hkeys, hpos,
                              slots, out, v));
    IBP_LAUNCHED("fill_hashed_kernel");
    return IBP_OK;
}

// ------------------------------------------------------------------ fetch kernel
// EXACT: condensed rows (byte ranges from a.s.offsets) instead of fixed-stride rows.
// ASYNC: fixed-stride rows in device memory, first reads double-buffered (fetch_heads_async;
// each warp owns two sets of a.slots slots).
// RAW: rows stored raw may be staged with the first reads (rows of at most 1 KiB).
template <typename U, int NC, bool EXACT, bool ASYNC, bool RAW>
__global__ void __launch_bounds__(kFetchThreads, 2) fetch_rows_kernel(FetchArgs<U> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    // tables, counters, claim table and sorted keys come from the kernels before this one
    grid_dep_wait();
    constexpr bool kClaims = !ASYNC;  // in-fetch claims: host rows (fixed-stride or condensed)
    const int lane = threadIdx.x & 31;
    U *slots = reinterpret_cast<U *>(smem) +
               (int64_t)(threadIdx.x >> 5) * a.slots * (ASYNC ? 2 : 1) * a.slot_words;
    // in-fetch claims: 64 words per warp after all the row slots
    int64_t *claim = reinterpret_cast<int64_t *>(
                         reinterpret_cast<U *>(smem) + (int64_t)(blockDim.x >> 5) * a.slots *
                                                           (ASYNC ? 2 : 1) * a.slot_words) +
                     (threadIdx.x >> 5) * 64;
    LaneTables<U, NC> lt;
    if (!a.raw_only) lt.load(a.s.t, a.s.v);
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const int64_t nrows = a.list ? (int64_t)*a.list_len : a.nrows;
    int64_t seen = 0;  // positions handed out when this warp last took a chunk
    for (;;) {
        // guided self-scheduling: 32-position chunks while much work remains, shrinking to
        // 4 towards the end (fewer when the fetch is small enough to give every warp less),
        // so that the grid's last chunks (each a chain of dependent reads) finish close
        // together
        const int g = (int)min((int64_t)a.gmax,
                               max((int64_t)min(min(4, a.gmax), a.upos),
                                   (nrows - seen) / (2 * nwarps)));
        unsigned long long c = 0;
        if (lane == 0) c = atomicAdd(a.work, (unsigned long long)g);
        const int64_t p0 = (int64_t)__shfl_sync(0xffffffffu, c, 0);
        if (p0 >= nrows) break;
        seen = p0 + g;
        // lane-parallel metadata of the chunk's positions (list entries: claimed heads)
        const bool valid = lane < g && p0 + lane < nrows;
        const int64_t k = a.list ? (valid ? a.list[p0 + lane] : 0) : p0 + lane;
        const int64_t k0 = p0;
        const int64_t key = valid ? (a.keys ? a.keys[k] : k) : -1;
        bool head = valid;
        if (a.dedup) {
            int64_t prev = __shfl_up_sync(0xffffffffu, key, 1);
            if (lane == 0) prev = k0 > 0 ? a.keys[k0 - 1] : key - 1;
            head = valid && key != prev;
        }
        const bool bad = head && (key < 0 || key >= a.s.n);
        if (bad) atomicOr(a.status, kStatusBadIndex);
        head = head && !bad;
        // in-fetch claims: one claim per distinct row of the chunk; the other lanes of that
        // row, and the lanes whose row was claimed earlier, are repeats
        const bool claims = kClaims && a.claims.keys;
        bool rep = false;
        const bool out_row = head;  // lanes with an output row (heads before claiming)
        U *orow = a.out + (out_row ? (a.pos ? a.pos[k] : k) : 0) * a.s.v;
        if (claims) rep = claim_chunk(a.claims, claim, key, head, orow);
        // pass 0 fetches the chunk's claimed (or, without claims, all) rows; pass 1, which
        // only in-fetch claims need, fetches the rows of repeats that gave up waiting for
        // their first occurrence, from their source like any other row
        bool fetch_lane = head;
        for (int pass = 0;; ++pass) {
            if constexpr (EXACT) {
                fetch_heads_exact<U, NC>(a.s, lt, slots, a.slots, a.slot_words, key, orow,
                                         fetch_lane, a.status);
            } else {
                const bool packed = fetch_lane && !a.raw_only &&
                                    ((__ldg(&a.s.bitmask[key >> 5]) >> (key & 31)) & 1);
                if constexpr (ASYNC)
                    fetch_heads_async<U, NC>(a.s, lt, slots, a.slots, a.slot_words, key, orow,
                                             fetch_lane, packed, a.status);
                else
                    fetch_heads<U, NC, RAW>(a.s, lt, slots, a.slots, a.slot_words, key, orow,
                                       fetch_lane, packed, a.status);
            }
            if (!claims || pass > 0) break;
            fetch_lane = settle_chunk<U>(a.claims, claim, rep, a.s.v, a.status);
            if (!__any_sync(0xffffffffu, fetch_lane)) break;
        }
    }
}

// ------------------------------------------------------------------ HBM rows of <= 64 words
// Rows in device memory are not bound by a link but by the instructions around the decode,
// so this kernel keeps per-row bookkeeping to a minimum: a warp takes a chunk of listed rows
// from a work counter (the claim pass's head records -- position with the row's
// stored-compressed flag, and row -- or rows p, p+1, ... of an unindexed fetch; 4 to 32 rows
// at a time by the batch's size), parks their keys and output rows in shared memory, and
// copies groups of G whole rows (one 16-byte cp.async per lane and row; rows must be 16-byte
// aligned) into one of two shared buffers while it decodes the previous group from the
// other.  A group whose words are all compressible (the usual case: a good mask leaves few
// words whole) takes its stream offsets from a table made once per warp; otherwise its prefix
// sums are issued together.  The row's stream length falls out of the offsets (no separate
// length pass, no tail reads), and stream offsets are 32-bit.
//
// Stream reads: stream_bits_ending (ibp_codec.cuh), a word read as the W stream bits that end
// where its bits end.
// `full[32 * c + lane]`: the inclusive prefix over the lanes of chunk c of the kept bits of
// every column (the stream offsets of a row whose words are all compressible).
template <typename U, int NC, int G>
__device__ __forceinline__ void hbm_decode_group(const U *__restrict__ buf, int sw, int r0,
                                                 int rows, unsigned okm, unsigned pm, int v,
                                                 int mw, const LaneTables<U, NC> &lt,
                                                 const uint32_t *full, U *const *mout,
                                                 int32_t *status) {
    constexpr int W = 8 * sizeof(U);
    const int lane = threadIdx.x & 31;
    uint32_t incl[G][NC];
    unsigned cjm = 0;  // bit q * NC + c: this lane's column of chunk c in row q is compressible
    bool mixed = false;  // a packed row of the group has a word stored whole
#pragma unroll
    for (int q = 0; q < G; ++q) {
        const int r = r0 + q;
        const bool pk = r < rows && ((pm >> r) & 1);
        const uint32_t *units = reinterpret_cast<const uint32_t *>(buf + q * sw);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const bool in = 32 * c + lane < v;
            const bool cj = pk && in && ((units[c] >> lane) & 1u);
            cjm |= (unsigned)cj << (q * NC + c);
            mixed |= pk && in && !cj;
            incl[q][c] = pk ? full[c * 32 + lane] : 0u;
        }
    }
    if (__any_sync(0xffffffffu, mixed)) {
        // some word of the group is stored whole: offsets from a prefix sum per row and chunk
#pragma unroll
        for (int q = 0; q < G; ++q) {
            const bool pk = r0 + q < rows && ((pm >> (r0 + q)) & 1);
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const bool in = 32 * c + lane < v;
                const bool cj = (cjm >> (q * NC + c)) & 1u;
                incl[q][c] = (pk && in) ? (cj ? (uint32_t)lt.nb[c] : (uint32_t)W) : 0u;
            }
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
            for (int q = 0; q < G; ++q) {
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, incl[q][c], off);
                    if (lane >= off) incl[q][c] += y;
                }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < G; ++q) {
        const int r = r0 + q;
        if (r >= rows || !((okm >> r) & 1)) continue;
        U *o = mout[r];
        const U *row = buf + q * sw;
        if (!((pm >> r) & 1)) {  // stored raw
#pragma unroll
            for (int c = 0; c < NC; ++c)
                if (32 * c + lane < v) o[32 * c + lane] = row[32 * c + lane];
            continue;
        }
        const uint32_t t0 = __shfl_sync(0xffffffffu, incl[q][0], 31);
        uint32_t tot = t0;
        if (NC > 1) tot += __shfl_sync(0xffffffffu, incl[q][NC - 1], 31);
        if (mw + (int)((tot + W - 1) / W) >= v) {
            // a bitmap claiming a stream as long as the raw row cannot come from this mask:
            // report it and leave the output row alone
            if (lane == 0) atomicOr(status, kStatusCorruptRow);
            continue;
        }
        const U *stream = row + mw;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int j = 32 * c + lane;
            if (j < v) {
                const bool cj = (cjm >> (q * NC + c)) & 1u;
                const U y = stream_bits_ending<U>(stream, (int32_t)((c ? t0 : 0u) + incl[q][c]));
                o[j] = cj ? (U)(lt.bv[c] | scatter_regs<U>(y, (U)~lt.m[c], lt.mv[c])) : y;
            }
        }
    }
}

// Shared memory of hbm_rows_kernel per warp: keys, output rows and stored-compressed flags
// of its (up to) 32 rows, the stream offsets of an all-compressible row (up to 64 words),
// then two buffers of G row slots.
constexpr size_t kHbmWarpMetaBytes = 512 + 128 + 256;

template <typename U, int NC, int G>
__global__ void __launch_bounds__(256, 4) hbm_rows_kernel(FetchArgs<U> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int per16 = 16 / sizeof(U);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char *meta = smem + warp * kHbmWarpMetaBytes;
    int64_t *mkey = reinterpret_cast<int64_t *>(meta);
    U **mout = reinterpret_cast<U **>(mkey + 32);
    int32_t *mpk = reinterpret_cast<int32_t *>(meta + 512);
    const int sw = (int)a.slot_words;
    U *bufs = reinterpret_cast<U *>(smem + (blockDim.x >> 5) * kHbmWarpMetaBytes) +
              (int64_t)warp * 2 * G * sw;
    // the column tables, the claim pass's list, the work counter and the status words come
    // from the kernels before this one
    grid_dep_wait();
    grid_dep_release();
    LaneTables<U, NC> lt;
    lt.load(a.s.t, a.s.v);
    const int v = (int)a.s.v, mw = (int)a.s.mw;
    // stream offsets (inclusive) of a row whose words are all compressible, lane-major
    uint32_t *full = reinterpret_cast<uint32_t *>(meta + 640);
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        uint32_t f = 32 * c + lane < v ? (uint32_t)lt.nb[c] : 0u;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, f, off);
            if (lane >= off) f += y;
        }
        full[c * 32 + lane] = f;
    }
    __syncwarp();
    const int nq16 = v / per16;  // 16-byte blocks of a row (<= 32)
    const int64_t nrows = a.list ? (int64_t)*a.list_len : a.nrows;
    // chunks of 32 rows (double-buffered groups) when every warp gets several of them, of
    // 8 (two groups) when every warp gets two, otherwise one group per chunk, so that the
    // rows spread over all warps (each chunk costs an atomic on the one work counter)
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const int chunk = nrows >= 4 * 32 * nwarps ? 32 : (nrows >= 16 * nwarps ? 8 : G);
    const unsigned below = (1u << lane) - 1u;
    // a warp's first chunk is its own (warp w takes chunk w); later ones come from the work
    // counter, so the grid's warps do not all queue on the counter at the start
    const int64_t gwarp = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
    for (bool first = true;; first = false) {
        int64_t p0;
        if (first) {
            p0 = gwarp * chunk;
        } else {
            unsigned long long c0 = 0;
            if (lane == 0) c0 = atomicAdd(a.work, (unsigned long long)chunk);
            p0 = (int64_t)__shfl_sync(0xffffffffu, c0, 0) + nwarps * chunk;
        }
        if (p0 >= nrows) break;
        const int avail = (int)min((int64_t)chunk, nrows - p0);
        const bool valid = lane < avail;
        int64_t k = p0 + lane, key = k;
        int packed = 0;
        if (valid && a.list) {  // a head record of the claim pass: position and row
            const longlong2 r = reinterpret_cast<const longlong2 *>(a.list)[p0 + lane];
            k = (int64_t)((uint64_t)r.x & ~kRecordPacked);
            key = r.y;
            packed = r.x < 0;
        }
        const bool bad = valid && (key < 0 || key >= a.s.n);
        if (bad) atomicOr(a.status, kStatusBadIndex);
        const bool ok = valid && !bad;
        if (ok && !a.list) packed = (__ldg(&a.s.bitmask[key >> 5]) >> (key & 31)) & 1;
        // the chunk's rows, packed to the front of its metadata
        const unsigned fm = __ballot_sync(0xffffffffu, ok);
        const int rows = __popc(fm);
        if (ok) {
            const int slot = __popc(fm & below);
            mkey[slot] = key;
            mout[slot] = a.out + k * (int64_t)v;
            mpk[slot] = packed;
        }
        __syncwarp();
        const unsigned okm = rows == 32 ? 0xffffffffu : ((1u << rows) - 1u);
        const unsigned pm = __ballot_sync(0xffffffffu, lane < rows && mpk[lane]);
        const int ng = (rows + G - 1) / G;
        // groups of G whole rows: the next group is copied into the other buffer while this
        // one decodes
        auto issue = [&](int g) {
            U *buf = bufs + (g & 1) * G * sw;
#pragma unroll
            for (int q = 0; q < G; ++q) {
                const int r = g * G + q;
                if (r < rows && lane < nq16)
                    cp_async16(buf + q * sw + lane * per16, a.s.comp + mkey[r] * v + lane * per16);
            }
            cp_async_commit();
        };
        if (ng > 0) issue(0);
        for (int g = 0; g < ng; ++g) {
            if (g + 1 < ng) {
                issue(g + 1);
                cp_async_wait_one();
            } else {
                cp_async_wait_all();
            }
            __syncwarp();
            hbm_decode_group<U, NC, G>(bufs + (g & 1) * G * sw, sw, g * G, rows, okm, pm, v, mw,
                                       lt, full, mout, a.status);
            __syncwarp();
        }
    }
}

// Device rows of at most 64 words, each 16-byte aligned, fetched whole by hbm_rows_kernel
// (not the sorted mode, whose positions repeat keys, nor raw gathers or condensed rows).
template <typename U>
static bool hbm_rows_fit(const FetchArgs<U> &a) {
    return a.device_rows && !a.raw_only && !a.dedup && !a.pos && !a.s.offsets &&
           !a.claims.keys && (!a.keys || a.list) && a.s.v <= 64 &&
           (a.s.v * (int64_t)sizeof(U)) % 16 == 0 && (((uintptr_t)a.s.comp) & 15) == 0;
}

template <typename U, int NC>
static ibp_status launch_hbm_nc(FetchArgs<U> a, cudaStream_t st) {
    // groups of 4 rows: measured faster than 8 (37 against 39 us for the 79k distinct rows of
    // a 400k-row graph-feature batch), with half the shared memory
    constexpr int G = 4;
    constexpr int threads = 256;
    a.slot_words = (int64_t)align_up((size_t)a.s.v + 2, 16 / sizeof(U));
    const size_t smem =
        (size_t)(threads / 32) * (kHbmWarpMetaBytes + 2 * G * a.slot_words * sizeof(U));
    auto kern = hbm_rows_kernel<U, NC, G>;
    int per_sm = 0;
    IBP_RET(kernel_blocks_per_sm((const void *)kern, threads, smem, &per_sm));
    int64_t blocks = (int64_t)device_sm_count() * per_sm;
    const int64_t need = (a.nrows + (int64_t)G * (threads / 32) - 1) / ((int64_t)G * (threads / 32));
    if (!a.list && blocks > need) blocks = need;
    const int slot = profile_begin(st);
    IBP_CUDA(launch_dependent(kern, (unsigned)blocks, threads, smem, st, a));
    IBP_LAUNCHED("hbm_rows_kernel");
    profile_end(slot, st);
    return IBP_OK;
}

// ------------------------------------------------------------------ repeats
// Output rows of the per-call fetch: position k goes to row pos[k] of `out`.
template <typename U>
struct CallRows {
    U *out;
    const int64_t *pos;
    int64_t v, n;
    __device__ __forceinline__ bool valid(int64_t key) const { return key >= 0 && key < n; }
    __device__ __forceinline__ U *row(int64_t k, int64_t) const { return out + pos[k] * v; }
    __device__ __forceinline__ int64_t words(int64_t) const { return v; }
};

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

// Slots of the hashed dedup table for nidx positions (load factor at most one half).
static int64_t hash_slots(int64_t nidx) { return std::max<int64_t>(64, (2 * nidx + 63) / 64 * 64); }

size_t decompress_workspace(int64_t nidx, int64_t v, int wb, bool has_index) {
    Sizer s;
    s.take<char>(kStatusBytes);
    s.take<char>(wb == 8 ? tables_bytes<uint64_t>(v) : tables_bytes<uint32_t>(v));
    if (has_index && nidx > 0) {
        // either the sort's arrays or the hash table, whichever the call picks
        Sizer srt;
        srt.take<int64_t>(nidx);  // iota
        srt.take<int64_t>(nidx);  // sanitised keys
        srt.take<int64_t>(nidx);  // sorted keys
        srt.take<int64_t>(nidx);  // positions
        srt.take<char>(sort_temp_bytes(nidx));
        Sizer hsh;
        hsh.take<int64_t>(hash_slots(nidx));
        hsh.take<int64_t>(hash_slots(nidx));
        hsh.take<int64_t>(2 * nidx);  // claimed heads (records of two words)
        s.take<char>(std::max(srt.total(), hsh.total()));
    }
    return s.total();
}

template <typename U, int NC, bool EXACT, bool ASYNC>
static ibp_status launch_fetch_nc(FetchArgs<U> a, int nblks, int nthreads, cudaStream_t st) {
    // a warp's slots: one set, or two for the double-buffered reads of device rows
    const size_t slot_bytes = (size_t)a.slot_words * sizeof(U) * (ASYNC ? 2 : 1);
    int threads = nthreads > 0 ? nthreads : kFetchThreads;
    threads = threads < 32 ? 32 : (threads > kFetchThreads ? kFetchThreads : threads / 32 * 32);
    const int maxs = device_max_smem_optin();
    // row slots per warp: up to kRowsInFlight within ~96 KB per block; long rows get fewer
    // slots and then fewer warps
    // (plus 512 bytes per warp for the in-fetch claims' slots and positions)
    const size_t warp_extra = a.claims.keys ? 64 * sizeof(int64_t) : 0;
    auto smem_of = [&](int s, int t) { return (slot_bytes * s + warp_extra) * (t / 32); };
    int slots = kRowsInFlight;
    while (slots > 1 && smem_of(slots, threads) > 96 * 1024) --slots;
    while (threads > 32 && smem_of(slots, threads) > (size_t)maxs) threads -= 32;
    const size_t smem = smem_of(slots, threads);
    if ((int64_t)smem > maxs) {
        set_error("rows of %lld words do not fit the fetch kernel's shared-memory slot",
                  (long long)a.s.v);
        return IBP_ERR_UNSUPPORTED;
    }
    a.slots = slots;
    // raw rows of over 1 KiB are never staged with the first reads: their kernel goes without
    // that code and its registers (whole-set fetches of 16 KiB rows at 97% invariant bits:
    // 2.85 -> 2.36 ms); rows of up to 1 KiB keep it
    auto kern = (EXACT || ASYNC || a.s.v * (int64_t)sizeof(U) <= 1024)
                    ? fetch_rows_kernel<U, NC, EXACT, ASYNC, true>
                    : fetch_rows_kernel<U, NC, EXACT, ASYNC, false>;
    int per_sm = 0;
    IBP_RET(kernel_blocks_per_sm((const void *)kern, threads, smem, &per_sm));
    int64_t blocks = nblks > 0 ? nblks : (int64_t)device_sm_count() * per_sm;
    a.upos = unit_positions(a.nrows, blocks * (threads / 32));
    // host rows: a warp takes no more positions than it has row slots, so the rows the
    // whole grid has in flight stay close together in host memory; HBM rows: 32
    if (a.gmax <= 0) a.gmax = a.slots;
    const int64_t chunks = (a.nrows + a.upos - 1) / a.upos;
    const int64_t need = (chunks + threads / 32 - 1) / (threads / 32);
    if (blocks > need) blocks = need;
    const int slot = profile_begin(st);
    IBP_CUDA(launch_dependent(kern, (unsigned)blocks, threads, smem, st, a));
    IBP_LAUNCHED("fetch_rows_kernel");
    profile_end(slot, st);
    return IBP_OK;
}

template <typename U, bool EXACT, bool ASYNC>
static ibp_status launch_fetch_x(FetchArgs<U> a, int nblks, int nthreads, cudaStream_t st) {
    if (a.raw_only || a.s.v > 64)
        return launch_fetch_nc<U, 0, EXACT, ASYNC>(a, nblks, nthreads, st);
    if (a.s.v > 32) return launch_fetch_nc<U, 2, EXACT, ASYNC>(a, nblks, nthreads, st);
    return launch_fetch_nc<U, 1, EXACT, ASYNC>(a, nblks, nthreads, st);
}

template <typename U>
static ibp_status launch_fetch(FetchArgs<U> a, int nblks, int nthreads, cudaStream_t st) {
    if (a.nrows <= 0) return IBP_OK;
    constexpr int per16 = 16 / sizeof(U);
    if (a.s.offsets) {
        // a condensed row starts at any word: room for the blocks around it and the padding
        a.slot_words = (int64_t)align_up((size_t)a.s.v + 2 * per16 + 2, per16);
        return launch_fetch_x<U, true, false>(a, nblks, nthreads, st);
    }
    if (a.raw_only) {
        a.slot_words = per16;  // raw rows are copied straight to the output
    } else if (a.s.v > 256) {
        // long rows: slots for rows up to twice the first read (the average length when the
        // caller gives a hint); longer rows decode from their source.  Smaller slots leave
        // room for more warps per SM and for the column tables in L1.
        const int64_t cap = std::max<int64_t>(2 * a.s.first_words, 256);
        a.slot_words = (int64_t)align_up((size_t)std::min<int64_t>(a.s.v, cap) + 2, per16);
    } else {
        a.slot_words = (int64_t)align_up((size_t)a.s.v + 2, per16);
    }
    if (hbm_rows_fit(a))
        return a.s.v > 32 ? launch_hbm_nc<U, 2>(a, st) : launch_hbm_nc<U, 1>(a, st);
    if (a.async_rows && !a.raw_only) return launch_fetch_x<U, false, true>(a, nblks, nthreads, st);
    return launch_fetch_x<U, false, false>(a, nblks, nthreads, st);
}

// The first kernel of a fetch call, in place of two memsets and the table build (a per-call
// fetch of a few thousand rows is as long as a handful of launches): clears the status word
// and the counters (the first 192 bytes of the workspace), builds the column tables unless
// the call only gathers raw rows, and marks `fill_pairs` 16-byte entries of the claim table
// empty (all ones).
template <typename U>
__global__ void __launch_bounds__(256)
prep_fetch_kernel(int32_t *status, const U *__restrict__ mask, const U *__restrict__ bitval,
                  int64_t v, ColTables<U> t, bool tables, longlong2 *fill, int64_t fill_pairs) {
    grid_dep_release();  // the claim pass may load its positions meanwhile
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nthr = (int64_t)gridDim.x * blockDim.x;
    if (tid < 48) status[tid] = 0;
    if (tables)
        for (int64_t j = tid; j < v; j += nthr) build_table_column<U>(mask, bitval, v, t, j);
    for (int64_t i = tid; i < fill_pairs; i += nthr) fill[i] = make_longlong2(-1, -1);
}

template <typename U>
static ibp_status launch_prep(int32_t *status, const U *mask, const U *bitval, int64_t v,
                              const ColTables<U> &t, bool tables, int64_t *fill, int64_t fill_words,
                              cudaStream_t st) {
    const int64_t pairs = fill_words / 2;  // claim tables have an even number of words
    int64_t blocks = std::max<int64_t>(tables ? (v + 255) / 256 : 1, (pairs + 1023) / 1024);
    blocks = std::min<int64_t>(std::max<int64_t>(blocks, 1), (int64_t)device_sm_count() * 8);
    prep_fetch_kernel<U><<<(unsigned)blocks, 256, 0, st>>>(
        status, mask, bitval, v, t, tables, reinterpret_cast<longlong2 *>(fill), pairs);
    IBP_LAUNCHED("prep_fetch_kernel");
    return IBP_OK;
}

template <typename U>
ibp_status decompress_impl(const U *comp, int64_t n, int64_t v, const U *mask,
                           const U *bitval, const int32_t *bitmask, const int64_t *idx,
                           int64_t nidx, bool has_index, int comp_len, U *out, int nblks,
                           int nthreads, int impl, void *ws, size_t ws_bytes, cudaStream_t st,
                           const int64_t *offsets, int64_t comp_bytes) {
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
    // status word (offset 0), the fetch work counter (offset 64), the claimed-head count of a
    // hashed fetch (offset 128): cleared by the call's first kernel (prep_fetch_kernel)
    if (nrows <= 0 || v <= 0) {
        IBP_CUDA(cudaMemsetAsync(status, 0, 192, st));
        return IBP_OK;
    }
    const bool tables = impl != 2;

    bool on_device = false;
    {
        cudaPointerAttributes pa{};
        if (cudaPointerGetAttributes(&pa, comp) == cudaSuccess)
            on_device = pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged;
        else
            cudaGetLastError();
    }
    FetchArgs<U> a{};
    a.gmax = on_device ? 32 : 0;
    // HBM rows of 256 bytes and up: first reads double-buffered, and rows of up to 64 words
    // decoded a group at a time (256-byte rows: 75 -> 61 us for 100k rows; smaller rows
    // decode too quickly for the extra bookkeeping to pay)
    a.async_rows = on_device && v * (int64_t)sizeof(U) >= 256;
    a.device_rows = on_device;
    a.s.comp = comp;
    a.s.n = n;
    a.s.v = v;
    a.s.mw = meta_bytes(v, wb) / wb;
    a.s.t = t;
    a.s.bitmask = bitmask;
    a.s.offsets = offsets;
    a.s.comp_bytes = comp_bytes;
    a.s.first_words = first_read_words(v, a.s.mw, wb, comp_len);
    a.nrows = nrows;
    a.raw_only = impl == 2;
    a.out = out;
    a.status = status;
    a.work = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(status) + 64);
    if (!has_index) {
        IBP_RET(launch_prep<U>(status, mask, bitval, v, t, tables, nullptr, 0, st));
        return launch_fetch<U>(a, nblks, nthreads, st);
    }

    if (nidx > 0x7fffffffLL) {
        IBP_CUDA(cudaMemsetAsync(status, 0, 192, st));
        set_error("decompress_fetch: index arrays above 2^31-1 entries are not supported");
        return IBP_ERR_UNSUPPORTED;
    }
    const int mode = fetch_dedup_mode();
    if (mode == 2 || (mode == 0 && impl != 2 && (on_device || 4 * nidx < n))) {
        // compressed rows (fixed-stride or condensed) in HBM, or a sparse batch of them in
        // host memory: claim rows in a hash table instead of sorting (HBM does not care about
        // row order, and far-apart host rows gain little from it).  Dense host batches keep
        // the sort: reading their rows in order pays when few of them repeat (uniform batches
        // of a quarter to all of the set: 3-10% faster sorted), though skewed dense batches
        // are faster hashed (mode 2); raw gathers gain nothing from claims.
        const int64_t slots = hash_slots(nidx);
        int64_t *hkeys = c.take<int64_t>(slots);
        int64_t *hpos = c.take<int64_t>(slots);
        int64_t *heads = c.take<int64_t>(2 * nidx);
        // keys -1 (empty); positions -1 (unpublished) for the in-fetch claims (a claim pass
        // writes the position of each slot it claims); hpos follows hkeys directly (slots is
        // a multiple of 64 words)
        IBP_RET(launch_prep<U>(status, mask, bitval, v, t, tables, hkeys,
                               on_device ? slots : (int64_t)(hpos + slots - hkeys), st));
        a.keys = idx;
        if (on_device) {
            // HBM rows: claim in a pass of its own, so the fetch walks distinct rows only, 32
            // to a chunk (the fetch is latency-bound here and chunks of repeats cost it)
            auto *nheads =
                reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(status) + 128);
            const int64_t wave = (int64_t)device_sm_count() * 8;  // resident 256-thread blocks
            const bool two = nidx > 256 * wave;
            const int64_t cb = std::min<int64_t>((nidx + (two ? 511 : 255)) / (two ? 512 : 256),
                                                 wave);
            a.list = heads;
            a.list_len = nheads;
            // the HBM-row kernel reads head records (position and stored-compressed flag, row)
            const int32_t *records = hbm_rows_fit(a) ? bitmask : nullptr;
            IBP_CUDA(launch_dependent(two ? claim_heads_kernel<2> : claim_heads_kernel<1>,
                                      (unsigned)cb, 256, 0, st, idx, nidx, n, hkeys, hpos, slots,
                                      heads, nheads, status, records));
            IBP_LAUNCHED("claim_heads_kernel");
        } else {
            // host rows: claims and repeat copies happen inside the fetch, hidden behind its
            // PCIe reads
            a.claims = ClaimTable{hkeys, hpos, slots, repeat_wait_polls()};
            return launch_fetch<U>(a, nblks, nthreads, st);
        }
        IBP_RET(launch_fetch<U>(a, nblks, nthreads, st));
        return launch_fill_hashed<U>(idx, nidx, n, hkeys, hpos, slots, out, v, st);
    }
    IBP_RET(launch_prep<U>(status, mask, bitval, v, t, tables, nullptr, 0, st));
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
    fill_repeats_kernel<U, CallRows<U>><<<(unsigned)fb, 256, 0, st>>>(keys, nidx,
                                                                       CallRows<U>{out, pos, v, n});
    IBP_LAUNCHED("fill_repeats_kernel");
    return IBP_OK;
}

// ------------------------------------------------------------------ access-pattern probe
// Reads the first `nq` 16-byte blocks of each listed row the way fetch_heads does (a warp
// takes kRowsInFlight rows from a work counter, all their loads before any is consumed) and
// decodes nothing, so its time is what the fetch kernel's reads alone cost on this link.
__global__ void __launch_bounds__(kFetchThreads, 2)
read_rows_probe_kernel(const uint4 *__restrict__ base, int64_t stride16,
                       const int64_t *__restrict__ rows, int64_t nrows, int nq,
                       unsigned long long *work, int32_t *sink) {
    const int lane = threadIdx.x & 31;
    uint32_t acc = 0;
    for (;;) {
        unsigned long long c = 0;
        if (lane == 0) c = atomicAdd(work, (unsigned long long)kRowsInFlight);
        const int64_t p0 = (int64_t)__shfl_sync(0xffffffffu, c, 0);
        if (p0 >= nrows) break;
        uint4 st[kRowsInFlight][2];
#pragma unroll
        for (int q = 0; q < kRowsInFlight; ++q) {
            if (p0 + q < nrows) {
                const uint4 *r = base + rows[p0 + q] * stride16;
                if (lane < nq) st[q][0] = r[lane];
                if (lane + 32 < nq) st[q][1] = r[lane + 32];
            }
        }
#pragma unroll
        for (int q = 0; q < kRowsInFlight; ++q) {
            if (p0 + q < nrows) {
                if (lane < nq) acc ^= st[q][0].x ^ st[q][0].w;
                if (lane + 32 < nq) acc ^= st[q][1].y;
            }
        }
    }
    if (acc == 0x9E3779B9u) atomicAdd(sink, 1);  // keeps the loads; practically never taken
}

ibp_status read_rows_probe(const void *base, int64_t stride_bytes, const int64_t *rows,
                           int64_t nrows, int32_t read_bytes, void *ws, size_t ws_bytes,
                           cudaStream_t st) {
    if (!ws || ws_bytes < kStatusBytes) {
        set_error("read_rows_probe: workspace of %zu bytes is below the required %zu", ws_bytes,
                  kStatusBytes);
        return IBP_ERR_WORKSPACE;
    }
    if (nrows <= 0) return IBP_OK;
    int32_t *sink = reinterpret_cast<int32_t *>(ws);
    auto *work = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(ws) + 64);
    IBP_CUDA(cudaMemsetAsync(ws, 0, 128, st));
    const int nq = (read_bytes + 15) / 16;
    int per_sm = 0;
    IBP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, read_rows_probe_kernel,
                                                           kFetchThreads, 0));
    if (per_sm < 1) per_sm = 1;
    if (per_sm > 2) per_sm = 2;  // the fetch kernel's residency
    const int slot = profile_begin(st);
    read_rows_probe_kernel<<<device_sm_count() * per_sm, kFetchThreads, 0, st>>>(
        reinterpret_cast<const uint4 *>(base), stride_bytes / 16, rows, nrows, nq, work, sink);
    IBP_LAUNCHED("read_rows_probe_kernel");
    profile_end(slot, st);
    return IBP_OK;
}

template ibp_status decompress_impl<uint32_t>(const uint32_t *, int64_t, int64_t,
                                              const uint32_t *, const uint32_t *,
                                              const int32_t *, const int64_t *, int64_t, bool,
                                              int, uint32_t *, int, int, int, void *, size_t,
                                              cudaStream_t, const int64_t *, int64_t);
template ibp_status decompress_impl<uint64_t>(const uint64_t *, int64_t, int64_t,
                                              const uint64_t *, const uint64_t *,
                                              const int32_t *, const int64_t *, int64_t, bool,
                                              int, uint64_t *, int, int, int, void *, size_t,
                                              cudaStream_t, const int64_t *, int64_t);

}  // namespace ibp200
