// ibp_fetch.cuh -- device code shared by the per-call fetch (ibp_decompress.cu) and the
// batched multi-set fetch (ibp_batch.cu): row reads into shared-memory slots, the
// per-column tables a lane keeps, the row decoder, and the processing of one chunk's
// distinct rows with several first reads in flight per warp.
#pragma once

#include "ibp_codec.cuh"
#include "ibp_common.cuh"

namespace ibp200 {

constexpr int kRowsInFlight = 4;  // first reads a warp keeps outstanding

// Positions a warp takes per unit of work: 32 (lane-parallel metadata over the full warp)
// unless the fetch has too few rows to give every warp of the grid a unit; then fewer, down
// to 1, so a small fetch spreads over more warps and SMs (each warp's rows form a chain of
// dependent reads, a few microseconds each over PCIe, and an SM keeps a limited number of
// host reads in flight).
__host__ __device__ __forceinline__ int unit_positions(int64_t rows, int64_t warps) {
    int u = 32;
    while (u > 1 && (int64_t)(u / 2) * warps >= rows) u >>= 1;
    return u;
}

// One tensor set as the fetch kernels see it.
template <typename U>
struct RowSet {
    const U *comp;          // fixed-stride compressed rows (device or pinned host)
    int64_t n, v, mw;       // rows, words per row, bitmap words
    int64_t first_words;    // words of the first read of a compressed row
    ColTables<U> t;         // per-column tables (device)
    const int32_t *bitmask; // compressed-row bits (device)
    const int64_t *offsets; // condensed rows: inclusive end byte of each row (else nullptr)
    int64_t comp_bytes;     // condensed rows: bytes of `comp`
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
// mw, zero words after the stream) into the output row.  Lane j of a 32-word chunk takes
// its bit length (kept bits when compressible, W otherwise) and its stream offset, pulls its
// bits with a funnel read and scatters them to the column's non-invariant positions; a warp
// prefix sum per chunk of 32 columns gives the offsets.  Rows of up to 64 words use the
// lane's register tables, one chunk after the other; longer rows take their chunks four at
// a time with the prefix sums interleaved, so different chunks' shuffle chains overlap.
template <typename U, int NC>
__device__ __forceinline__ void decode_row(const U *__restrict__ buf, int64_t v, int64_t mw,
                                           const ColTables<U> &t, const LaneTables<U, NC> &lt,
                                           U *__restrict__ orow) {
    constexpr int W = 8 * sizeof(U);
    const int lane = threadIdx.x & 31;
    const uint32_t *units = reinterpret_cast<const uint32_t *>(buf);
    const U *stream = buf + mw;
    if constexpr (NC > 0) {
        int64_t base = 0;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            if (32 * c >= v) break;
            const int64_t j = 32 * c + lane;
            const bool in = j < v;
            const bool cj = in && ((units[j >> 5] >> (j & 31)) & 1u);
            const int L = in ? (cj ? lt.nb[c] : W) : 0;
            int incl = L;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (in) {
                const U y = get_bits<U>(stream, base + incl - L, L);
                orow[j] = cj ? (U)(lt.bv[c] | scatter_regs<U>(y, (U)~lt.m[c], lt.mv[c])) : y;
            }
            base += __shfl_sync(0xffffffffu, incl, 31);
        }
    } else {
        // four chunks of 32 columns at a time; bit offsets relative to the stream word that
        // holds the group's first bit, so they stay 32-bit however long the row
        constexpr int G = 4;
        constexpr int LW = LogW<U>::value;
        int64_t base = 0;  // stream bits of the row's earlier groups
        for (int64_t g0 = 0; g0 < v; g0 += 32 * G) {
            U m[G], bv[G];
            bool in[G], cj[G];
            int incl[G];
            int maxnb = 0;  // most bits any column of the group keeps
#pragma unroll
            for (int c = 0; c < G; ++c) {
                const int64_t j = g0 + 32 * c + lane;
                in[c] = j < v;
                m[c] = in[c] ? __ldg(&t.mask[j]) : (U)0;
                bv[c] = in[c] ? __ldg(&t.bitval[j]) : (U)0;
                const int nb = in[c] ? (int)__ldg(&t.nb[j]) : 0;
                maxnb = max(maxnb, nb);
                cj[c] = in[c] && ((units[j >> 5] >> (j & 31)) & 1u);
                incl[c] = in[c] ? (cj[c] ? nb : W) : 0;
            }
            maxnb = __reduce_max_sync(0xffffffffu, maxnb);
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
                for (int c = 0; c < G; ++c) {
                    const int y = __shfl_up_sync(0xffffffffu, incl[c], o);
                    if (lane >= o) incl[c] += y;
                }
            }
            const U *gs = stream + (base >> LW);
            const int32_t off0 = (int32_t)(base & (W - 1));
            int32_t off = off0;
            if (maxnb <= 4) {
                // highly invariant columns: place each kept bit from the mask directly (at
                // most 4 steps, no move-mask loads)
#pragma unroll
                for (int c = 0; c < G; ++c) {
                    const int64_t j = g0 + 32 * c + lane;
                    if (in[c]) {
                        const U y = stream_bits_ending<U>(gs, off + incl[c]);
                        U x = y;
                        if (cj[c]) {
                            U sel = (U)~m[c], r = 0;
#pragma unroll
                            for (int i = 0; i < 4; ++i) {  // nb <= 4: sel is empty after
                                const U low = (U)(sel & (U)(~sel + 1));
                                r |= ((y >> i) & 1) ? low : (U)0;
                                sel &= (U)(sel - 1);
                            }
                            x = (U)(bv[c] | r);
                        }
                        orow[j] = x;
                    }
                    off += __shfl_sync(0xffffffffu, incl[c], 31);
                }
            } else {
#pragma unroll
                for (int c = 0; c < G; ++c) {
                    const int64_t j = g0 + 32 * c + lane;
                    if (in[c]) {
                        const U y = stream_bits_ending<U>(gs, off + incl[c]);
                        orow[j] = cj[c] ? (U)(bv[c] | scatter_bits<U>(y, (U)~m[c], t.mv + j, (int)v))
                                        : y;
                    }
                    off += __shfl_sync(0xffffffffu, incl[c], 31);
                }
            }
            base += off - off0;
        }
    }
}

// decode_row for up to kRowsInFlight rows of at most 64 words at once (rows in slots
// `slots + q * slot_words` for the q set in `qm`, outputs `o[q]`): the prefix sums of every
// row's chunks are issued together, so their shuffle chains overlap instead of following
// one another, then each row's bits are placed as in decode_row.
template <typename U, int NC>
__device__ __forceinline__ void decode_rows_multi(const U *__restrict__ slots,
                                                  int64_t slot_words, unsigned qm, int64_t v,
                                                  int64_t mw, const LaneTables<U, NC> &lt,
                                                  U *const *o) {
    static_assert(NC > 0, "register tables only");
    constexpr int W = 8 * sizeof(U);
    constexpr int Q = kRowsInFlight;
    const int lane = threadIdx.x & 31;
    int incl[Q][NC];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const uint32_t *units = reinterpret_cast<const uint32_t *>(slots + q * slot_words);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int64_t j = 32 * c + lane;
            const bool in = ((qm >> q) & 1) && j < v;
            const bool cj = in && ((units[j >> 5] >> (j & 31)) & 1u);
            incl[q][c] = in ? (cj ? lt.nb[c] : W) : 0;
        }
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const int y = __shfl_up_sync(0xffffffffu, incl[q][c], off);
                if (lane >= off) incl[q][c] += y;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (!((qm >> q) & 1)) continue;
        const U *buf = slots + q * slot_words;
        const uint32_t *units = reinterpret_cast<const uint32_t *>(buf);
        const U *stream = buf + mw;
        int64_t base = 0;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            if (32 * c >= v) break;
            const int64_t j = 32 * c + lane;
            const bool in = j < v;
            const bool cj = in && ((units[j >> 5] >> (j & 31)) & 1u);
            const int L = in ? (cj ? lt.nb[c] : W) : 0;
            if (in) {
                const U y = get_bits<U>(stream, base + incl[q][c] - L, L);
                o[q][j] = cj ? (U)(lt.bv[c] | scatter_regs<U>(y, (U)~lt.m[c], lt.mv[c])) : y;
            }
            base += __shfl_sync(0xffffffffu, incl[q][c], 31);
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


// Second half of a group of rows whose first reads are in their slots (slot q at
// slots + q * slot_words for the rows of lanes lid[0..cnt)): exact lengths from the
// bitmaps, the rest of every row that needs more than its first read (all issued before any
// is waited for: 16-byte blocks in registers, at most 32 per row; longer tails and
// unaligned rows take the plain loop), then the decode (or copy, for rows stored raw).
// A row stored raw (not packed) is copied to its output from its slot when the caller staged
// it there whole (raw_staged), else straight from its source.
template <typename U>
__device__ __forceinline__ void copy_raw_row(U *o, const U *slot, const U *src, int64_t v,
                                             bool raw_staged) {
    if (raw_staged) {
        const int lane = threadIdx.x & 31;
        if ((((uintptr_t)o) & 15) == 0) {
            const int64_t n16 = v * (int64_t)sizeof(U) / 16;
            for (int64_t k = lane; k < n16; k += 32)
                reinterpret_cast<uint4 *>(o)[k] = reinterpret_cast<const uint4 *>(slot)[k];
        } else {
            for (int64_t k = lane; k < v; k += 32) o[k] = slot[k];
        }
    } else {
        warp_copy<U>(o, src, v);
    }
}

template <typename U, int NC, bool MULTI = false>
__device__ __forceinline__ void finish_rows(const RowSet<U> &s, const LaneTables<U, NC> &lt,
                                            U *__restrict__ slots, int64_t slot_words,
                                            const int *lid, int cnt, int64_t key, U *orow,
                                            bool packed, int32_t *status,
                                            bool raw_staged = false) {
    const int lane = threadIdx.x & 31;
    const int64_t v = s.v;
    int64_t end[kRowsInFlight];
    {
        constexpr int per16 = 16 / sizeof(U);
        uint4 tail[kRowsInFlight];
        int64_t tb0[kRowsInFlight], tb1[kRowsInFlight];
#pragma unroll
        for (int q = 0; q < kRowsInFlight; ++q) {
            end[q] = -1;
            tb0[q] = tb1[q] = 0;
            if (q < cnt && __shfl_sync(0xffffffffu, (int)packed, lid[q])) {
                const int64_t r = __shfl_sync(0xffffffffu, key, lid[q]);
                const U *row = s.comp + r * v;
                U *buf = slots + q * slot_words;
                end[q] = row_words<U, NC>(buf, v, s.mw, s.t, lt);
                // a row too long for its slot is decoded straight from its source below
                if (end[q] < v && end[q] > s.first_words && end[q] + 2 <= slot_words) {
                    const int64_t b0 = s.first_words / per16;
                    const int64_t b1 = (end[q] + per16 - 1) / per16;
                    if ((((uintptr_t)row) & 15) == 0 && b1 - b0 <= 32) {
                        tb0[q] = b0;
                        tb1[q] = b1;
                        if (b0 + lane < b1)
                            tail[q] = reinterpret_cast<const uint4 *>(row)[b0 + lane];
                    } else {
                        issue_words<U>(buf, row, s.first_words, end[q]);
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kRowsInFlight; ++q)
            if (tb0[q] + lane < tb1[q])
                reinterpret_cast<uint4 *>(slots + q * slot_words)[tb0[q] + lane] = tail[q];
    }
    __syncwarp();
    if constexpr (MULTI && NC > 0) {
        // rows of at most 64 words: copies and corrupt rows first, then every row of the
        // group that decodes from its slot, all at once
        U *o[kRowsInFlight];
        unsigned qm = 0;
#pragma unroll
        for (int q = 0; q < kRowsInFlight; ++q) {
            o[q] = nullptr;
            if (q < cnt) {
                const int64_t r = __shfl_sync(0xffffffffu, key, lid[q]);
                o[q] = reinterpret_cast<U *>(
                    __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(orow), lid[q]));
                if (end[q] < 0) {
                    copy_raw_row<U>(o[q], slots + q * slot_words, s.comp + r * v, v, raw_staged);
                } else if (end[q] >= v) {
                    if (lane == 0) atomicOr(status, kStatusCorruptRow);
                } else if (end[q] + 2 > slot_words) {  // not with slots of v + 2 words
                    decode_row<U, NC>(s.comp + r * v, v, s.mw, s.t, lt, o[q]);
                    __syncwarp();
                } else {
                    if (lane < 2) slots[q * slot_words + end[q] + lane] = 0;
                    qm |= 1u << q;
                }
            }
        }
        __syncwarp();
        if (qm) decode_rows_multi<U, NC>(slots, slot_words, qm, v, s.mw, lt, o);
        __syncwarp();
    } else {
#pragma unroll
        for (int q = 0; q < kRowsInFlight; ++q) {
            if (q < cnt) {
                const int64_t r = __shfl_sync(0xffffffffu, key, lid[q]);
                U *o = reinterpret_cast<U *>(
                    __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(orow), lid[q]));
                if (end[q] < 0) {
                    copy_raw_row<U>(o, slots + q * slot_words, s.comp + r * v, v, raw_staged);
                    continue;
                }
                if (end[q] >= v) {
                    // a bitmap claiming a stream as long as the raw row cannot come from this
                    // mask: report it and leave the output row alone
                    if (lane == 0) atomicOr(status, kStatusCorruptRow);
                    continue;
                }
                if (end[q] + 2 > slot_words) {
                    // longer than the slot (slots are sized for rows near the average length
                    // when rows are long): decode from the source row, whose words after the
                    // stream are its zero padding
                    decode_row<U, NC>(s.comp + r * v, v, s.mw, s.t, lt, o);
                    __syncwarp();
                    continue;
                }
                U *buf = slots + q * slot_words;
                // words past the stream read as zero (get_bits looks one word ahead; the
                // value there never reaches an output bit)
                if (lane < 2) buf[end[q] + lane] = 0;
                __syncwarp();
                decode_row<U, NC>(buf, v, s.mw, s.t, lt, o);
                __syncwarp();
            }
        }
    }
}

// Fetch and decode (or copy, when not packed) the rows of the lanes whose `head` is set:
// groups of up to `nslots` rows have their first reads, and then the rest of the rows that
// need it, loaded into registers together (16-byte loads, all rows before any store), so
// their PCIe or HBM round trips overlap; rows that are not 16-byte aligned, whose first
// read exceeds 1 KiB or whose tail exceeds 512 bytes take a plain loop.
// `orow` is each lane's output row.
// kRawStage: rows stored raw may be staged with the first reads (see below); instantiated
// false where no raw row can be (rows over 1 KiB), which frees the registers it takes.
template <typename U, int NC, bool kRawStage = true>
__device__ __forceinline__ void fetch_heads(const RowSet<U> &s, const LaneTables<U, NC> &lt,
                                            U *__restrict__ slots, int nslots,
                                            int64_t slot_words, int64_t key, U *orow,
                                            bool head, bool packed, int32_t *status) {
    constexpr int per16 = 16 / sizeof(U);
    const int lane = threadIdx.x & 31;
    const int64_t v = s.v;
    // rows stored raw are read whole into their slot together with the other rows' first
    // reads when they fit it and the register staging, so copying them out costs no round
    // trip of its own
    const int64_t nq_raw = v / per16;
    const bool raw_staged = kRawStage && (v % per16) == 0 && v + 2 <= slot_words &&
                            nq_raw <= 64 && (((uintptr_t)s.comp) & 15) == 0;
    unsigned hm = __ballot_sync(0xffffffffu, head);
    while (hm) {
        int lid[kRowsInFlight];
        int cnt = 0;
#pragma unroll
        for (int q = 0; q < kRowsInFlight; ++q) {
            lid[q] = 0;
            if (q < nslots && hm) {
                lid[q] = __ffs(hm) - 1;
                hm &= hm - 1;
                ++cnt;
            }
        }
        {
            const int64_t nq = (s.first_words + per16 - 1) / per16;
            uint4 stage[kRowsInFlight][2];
            unsigned fastm = 0, rawm = 0;  // bit q: staged in registers; row q stored raw
#pragma unroll
            for (int q = 0; q < kRowsInFlight; ++q) {
                if (q < cnt) {
                    const int64_t r = __shfl_sync(0xffffffffu, key, lid[q]);
                    const bool pk = __shfl_sync(0xffffffffu, (int)packed, lid[q]);
                    const U *row = s.comp + r * v;
                    const int64_t n = pk ? nq : nq_raw;
                    const bool fast = (pk || raw_staged) && ((((uintptr_t)row) & 15) == 0) &&
                                      n <= 64;
                    fastm |= (unsigned)fast << q;
                    rawm |= (unsigned)!pk << q;
                    if (fast) {
                        const uint4 *r4 = reinterpret_cast<const uint4 *>(row);
                        if (lane < n) stage[q][0] = r4[lane];
                        if (lane + 32 < n) stage[q][1] = r4[lane + 32];
                    } else if (pk) {
                        issue_words<U>(slots + q * slot_words, row, 0, s.first_words);
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < kRowsInFlight; ++q) {
                if ((fastm >> q) & 1) {
                    const int64_t n = ((rawm >> q) & 1) ? nq_raw : nq;
                    uint4 *b4 = reinterpret_cast<uint4 *>(slots + q * slot_words);
                    if (lane < n) b4[lane] = stage[q][0];
                    if (lane + 32 < n) b4[lane + 32] = stage[q][1];
                }
            }
        }
        __syncwarp();
        finish_rows<U, NC>(s, lt, slots, slot_words, lid, cnt, key, orow, packed, status,
                           raw_staged);
    }
}

// The next up-to-`nslots` head lanes of `hm` (removed from it), in lane order.
__device__ __forceinline__ int pick_rows(unsigned &hm, int nslots, int *lid) {
    int cnt = 0;
#pragma unroll
    for (int q = 0; q < kRowsInFlight; ++q) {
        lid[q] = 0;
        if (q < nslots && hm) {
            lid[q] = __ffs(hm) - 1;
            hm &= hm - 1;
            ++cnt;
        }
    }
    return cnt;
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// fetch_heads for rows in device memory: the first reads of the next group of rows are
// issued as asynchronous copies into a second set of slots while the current group is
// decoded, so a warp's HBM round trips overlap its decode instead of following it (the
// warp owns 2 x nslots slots).  Not used for host rows: asynchronous copies from host
// memory are slow on this part.
template <typename U, int NC>
__device__ __forceinline__ void fetch_heads_async(const RowSet<U> &s, const LaneTables<U, NC> &lt,
                                                  U *__restrict__ slots, int nslots,
                                                  int64_t slot_words, int64_t key, U *orow,
                                                  bool head, bool packed, int32_t *status) {
    constexpr int per16 = 16 / sizeof(U);
    const int lane = threadIdx.x & 31;
    const int64_t v = s.v;
    const int64_t nq = (s.first_words + per16 - 1) / per16;
    auto issue = [&](const int *lid, int cnt, U *base) {
        for (int q = 0; q < cnt; ++q) {
            const int64_t r = __shfl_sync(0xffffffffu, key, lid[q]);
            const bool pk = __shfl_sync(0xffffffffu, (int)packed, lid[q]);
            if (!pk) continue;
            const U *row = s.comp + r * v;
            U *buf = base + q * slot_words;
            if ((((uintptr_t)row) & 15) == 0) {
                for (int64_t b = lane; b < nq; b += 32)
                    cp_async16(reinterpret_cast<uint4 *>(buf) + b,
                               reinterpret_cast<const uint4 *>(row) + b);
            } else {
                issue_words<U>(buf, row, 0, s.first_words);
            }
        }
        cp_async_commit();
    };
    unsigned hm = __ballot_sync(0xffffffffu, head);
    int lid[kRowsInFlight], nlid[kRowsInFlight];
    int cnt = pick_rows(hm, nslots, lid);
    int cur = 0;
    if (cnt) issue(lid, cnt, slots);
    while (cnt) {
        const int ncnt = pick_rows(hm, nslots, nlid);
        U *nbase = slots + (int64_t)(cur ^ 1) * nslots * slot_words;
        if (ncnt) {
            issue(nlid, ncnt, nbase);
            cp_async_wait_one();  // the current group's copies are done
        } else {
            cp_async_wait_all();
        }
        __syncwarp();
        finish_rows<U, NC, true>(s, lt, slots + (int64_t)cur * nslots * slot_words, slot_words,
                                 lid, cnt, key, orow, packed, status);
        __syncwarp();
#pragma unroll
        for (int q = 0; q < kRowsInFlight; ++q) lid[q] = nlid[q];
        cnt = ncnt;
        cur ^= 1;
    }
}

// Condensed rows (byte ranges known from the offsets): each head lane's row is read exactly,
// its 16-byte blocks (at most 64 per row staged in registers, longer rows by a plain loop)
// loaded for up to `nslots` rows before any is stored, so one round trip serves a row.  A
// row whose stored length is the raw length is copied; any other is decoded, after checking
// that its bitmap's stream fits the stored length.  Ranges that cannot be a row (negative,
// decreasing, past the end of `comp`, longer than raw, not whole words) are flagged as
// corrupt and skipped, so no read leaves the 16-byte blocks of `comp`.
template <typename U, int NC>
__device__ __forceinline__ void fetch_heads_exact(const RowSet<U> &s, const LaneTables<U, NC> &lt,
                                                  U *__restrict__ slots, int nslots,
                                                  int64_t slot_words, int64_t key, U *orow,
                                                  bool head, int32_t *status) {
    const int lane = threadIdx.x & 31;
    const int64_t v = s.v;
    const int64_t raw_bytes = v * (int64_t)sizeof(U);
    int64_t b0 = 0, b1 = 0;
    if (head) {
        b0 = key > 0 ? s.offsets[key - 1] : 0;
        b1 = s.offsets[key];
        if (b0 < 0 || b1 < b0 || b1 > s.comp_bytes || b1 - b0 > raw_bytes ||
            ((b0 | b1) % (int64_t)sizeof(U)) != 0) {
            atomicOr(status, kStatusCorruptRow);
            head = false;
        }
    }
    const char *base = reinterpret_cast<const char *>(s.comp);
    unsigned hm = __ballot_sync(0xffffffffu, head);
    while (hm) {
        int lid[kRowsInFlight];
        int cnt = 0;
#pragma unroll
        for (int q = 0; q < kRowsInFlight; ++q) {
            lid[q] = 0;
            if (q < nslots && hm) {
                lid[q] = __ffs(hm) - 1;
                hm &= hm - 1;
                ++cnt;
            }
        }
        int woff[kRowsInFlight];
        {
            uint4 stage[kRowsInFlight][2];
            int64_t nblk[kRowsInFlight];
#pragma unroll
            for (int q = 0; q < kRowsInFlight; ++q) {
                nblk[q] = 0;
                woff[q] = 0;
                if (q < cnt) {
                    const int64_t lo = __shfl_sync(0xffffffffu, b0, lid[q]);
                    const int64_t hi = __shfl_sync(0xffffffffu, b1, lid[q]);
                    const uintptr_t a0 = (uintptr_t)(base + lo) & ~(uintptr_t)15;
                    const uintptr_t a1 = ((uintptr_t)(base + hi) + 15) & ~(uintptr_t)15;
                    woff[q] = (int)(((uintptr_t)(base + lo) - a0) / sizeof(U));
                    const uint4 *src = reinterpret_cast<const uint4 *>(a0);
                    const int64_t nb = (int64_t)((a1 - a0) >> 4);
                    if (nb <= 64) {
                        nblk[q] = nb;
                        if (lane < nb) stage[q][0] = src[lane];
                        if (lane + 32 < nb) stage[q][1] = src[lane + 32];
                    } else {
                        uint4 *dst = reinterpret_cast<uint4 *>(slots + q * slot_words);
                        for (int64_t k = lane; k < nb; k += 32) dst[k] = src[k];
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < kRowsInFlight; ++q) {
                uint4 *dst = reinterpret_cast<uint4 *>(slots + q * slot_words);
                if (lane < nblk[q]) dst[lane] = stage[q][0];
                if (lane + 32 < nblk[q]) dst[lane + 32] = stage[q][1];
            }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < kRowsInFlight; ++q) {
            if (q < cnt) {
                U *o = reinterpret_cast<U *>(
                    __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(orow), lid[q]));
                const int64_t len = (__shfl_sync(0xffffffffu, b1, lid[q]) -
                                     __shfl_sync(0xffffffffu, b0, lid[q])) / (int64_t)sizeof(U);
                U *buf = slots + q * slot_words + woff[q];
                if (len == v) {
                    for (int64_t j = lane; j < v; j += 32) o[j] = buf[j];
                    __syncwarp();
                    continue;
                }
                const int64_t end = row_words<U, NC>(buf, v, s.mw, s.t, lt);
                if (end > len) {
                    if (lane == 0) atomicOr(status, kStatusCorruptRow);
                    continue;
                }
                if (lane < 2) buf[end + lane] = 0;
                __syncwarp();
                decode_row<U, NC>(buf, v, s.mw, s.t, lt, o);
                __syncwarp();
            }
        }
    }
}

// ------------------------------------------------------------------ hashed dedup
// The first position to claim a row in an open-addressing table fetches it; later ones are
// repeats.  Tables have at least twice as many slots as positions, so linear probing ends
// quickly.
__device__ __forceinline__ uint64_t row_hash(int64_t key, int64_t slots) {
    return __umul64hi((uint64_t)key * 0x9E3779B97F4A7C15ull, (uint64_t)slots);
}

// The table slot holding `key` after this call: claimed by it (`won`) or by an earlier one;
// -1 when the table is full (it never is: it has twice as many slots as positions).
__device__ __forceinline__ int64_t hash_claim_slot(int64_t *keys, int64_t slots, int64_t key,
                                                   bool &won) {
    won = false;
    uint64_t h = row_hash(key, slots);
    for (int64_t probe = 0; probe < slots; ++probe) {
        // a plain read first: a row already claimed (hot rows of a skewed batch) costs no
        // atomic, so repeats do not queue on one address
        const int64_t cur = *reinterpret_cast<volatile int64_t *>(keys + h);
        if (cur == key) return (int64_t)h;
        if (cur == -1) {
            const unsigned long long old = atomicCAS(
                reinterpret_cast<unsigned long long *>(keys + h), ~0ull, (unsigned long long)key);
            if (old == ~0ull) {
                won = true;
                return (int64_t)h;
            }
            if ((int64_t)old == key) return (int64_t)h;
        }
        h = h + 1 == (uint64_t)slots ? 0 : h + 1;
    }
    return -1;
}

__device__ __forceinline__ int64_t load_acquire(const int64_t *p) {
    int64_t x;
    asm volatile("ld.acquire.gpu.global.s64 %0, [%1];" : "=l"(x) : "l"(p) : "memory");
    return x;
}

__device__ __forceinline__ void store_release(int64_t *p, int64_t x) {
    asm volatile("st.release.gpu.global.s64 [%0], %1;" ::"l"(p), "l"(x) : "memory");
}

// Copy rows src -> dst for the lanes of `dm` (each lane's src/dst), four rows at a time: all
// four rows' loads before any store (16-byte moves when the rows are aligned), so the loads'
// latencies overlap.  Sources are read through L2 (other SMs may have just written them),
// or, with kCached (sources written by an earlier kernel and not written during this one),
// through the SM's L1 as well, so that a hot row copied by many warps of an SM is read from
// L2 once per SM instead of once per copy; the copies are then written as streaming stores
// (evicted from L2 first), which keeps the sources in L2 (fill of a 400k-row batch's
// repeats: 39.0 -> 36.5 us).
template <typename U, bool kCached = false>
__device__ __forceinline__ void copy_rows(unsigned dm, const U *src_row, U *dst_row, int64_t v,
                                          bool vec_rows) {
    constexpr int R = 4;
    const int lane = threadIdx.x & 31;
    while (dm) {
        const U *src[R];
        U *dst[R];
        int cnt = 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            src[r] = src_row;
            dst[r] = dst_row;
            if (dm) {
                const int j = __ffs(dm) - 1;
                dm &= dm - 1;
                src[r] = reinterpret_cast<const U *>(__shfl_sync(
                    0xffffffffu, reinterpret_cast<unsigned long long>(src_row), j));
                dst[r] = reinterpret_cast<U *>(__shfl_sync(
                    0xffffffffu, reinterpret_cast<unsigned long long>(dst_row), j));
                cnt = r + 1;
            }
        }
        if (vec_rows) {
            const int64_t n16 = v * (int64_t)sizeof(U) / 16;
            for (int64_t q = lane; q < n16; q += 32) {
                uint4 t[R];
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r < cnt)
                        t[r] = kCached ? __ldg(reinterpret_cast<const uint4 *>(src[r]) + q)
                                       : __ldcg(reinterpret_cast<const uint4 *>(src[r]) + q);
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r < cnt) {
                        if (kCached)
                            __stcs(reinterpret_cast<uint4 *>(dst[r]) + q, t[r]);
                        else
                            reinterpret_cast<uint4 *>(dst[r])[q] = t[r];
                    }
            }
        } else {
            for (int64_t q = lane; q < v; q += 32) {
                U t[R];
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r < cnt) t[r] = kCached ? __ldg(src[r] + q) : __ldcg(src[r] + q);
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r < cnt) {
                        if (kCached)
                            __stcs(dst[r] + q, t[r]);
                        else
                            dst[r][q] = t[r];
                    }
            }
        }
    }
}

// ------------------------------------------------------------------ in-fetch claims
// A fetch kernel over host rows de-duplicates inside itself: each chunk of positions claims
// its distinct rows in a hash table before fetching them (claim_chunk), and once the chunk's
// claimed rows are written, publishes their output rows in the table and copies every repeat
// from the output row of its row's first claim (settle_chunk), so the copies overlap the
// other warps' host reads.  A warp waits only after publishing all of its own claims, so
// every row waited on belongs to a warp that is still fetching and waits on nothing; the
// wait is bounded all the same, and a repeat that stops waiting fetches its own row.
constexpr int64_t kRowDone = 1ll << 62;  // a published table entry: output row address | this

struct ClaimTable {
    int64_t *keys;   // row keys (-1 = empty slot)
    int64_t *rows;   // output row address of each slot's claim, | kRowDone once written (-1 before)
    int64_t slots;
    int wait_polls;  // polls (~0.25 us apart) a repeat makes for its row
};

// One claim per distinct key of the chunk (its lowest `head` lane).  On return `head` is set
// for the lanes that fetch their row (they claimed it); the result is true for repeats
// (their key was claimed by another lane or an earlier chunk).  Each lane parks its table slot
// (| kRowDone when it claimed) and its output row address in `park` (64 words of shared
// memory per warp) until the chunk is settled, which keeps them out of the fetch's registers.
__device__ __forceinline__ bool claim_chunk(const ClaimTable &c, int64_t *park, int64_t key,
                                            bool &head, const void *orow) {
    const int lane = threadIdx.x & 31;
    const unsigned same = __match_any_sync(0xffffffffu, head ? key : (int64_t)-1);
    const int first = __ffs(same) - 1;
    bool won = false;
    int64_t slot = -1;
    if (head && first == lane) slot = hash_claim_slot(c.keys, c.slots, key, won);
    slot = __shfl_sync(0xffffffffu, slot, first);
    const bool rep = head && !won && slot >= 0;
    // a lane whose claim found the table full (a caller that understated the batch) fetches
    // its row without a claim
    head = won || (head && slot < 0);
    park[lane] = won ? slot | kRowDone : (rep ? slot : -1);
    park[32 + lane] = (int64_t)reinterpret_cast<uintptr_t>(orow);
    return rep;
}

// After the chunk's claimed rows are written: publish them (every lane's stores are ordered
// before the release by the warp barrier), then copy each repeat once its row is published.
// Returns true for the repeats that gave up waiting (status bit 3); they fetch their own row.
template <typename U>
__device__ __forceinline__ bool settle_chunk(const ClaimTable &c, const int64_t *park, bool rep,
                                             int64_t v, int32_t *status) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    const int64_t cw = park[lane];
    U *const dst = reinterpret_cast<U *>(static_cast<uintptr_t>(park[32 + lane]));
    const int64_t slot = cw & ~kRowDone;
    if (cw >= 0 && (cw & kRowDone))
        store_release(c.rows + slot, (int64_t)reinterpret_cast<uintptr_t>(dst) | kRowDone);
    if (!__any_sync(0xffffffffu, rep)) return false;
    // once any wait has given up, later ones make a single check (lane 0 reads the status
    // word, so that every lane has the same bound)
    int limit = 0;
    if (lane == 0)
        limit = (*reinterpret_cast<volatile int32_t *>(status) & kStatusWaitTimeout)
                    ? min(1, c.wait_polls)
                    : c.wait_polls;
    limit = __shfl_sync(0xffffffffu, limit, 0);
    const U *src = nullptr;
    for (int it = 0; it < limit; ++it) {
        if (rep && !src) {
            const int64_t hv = load_acquire(c.rows + slot);
            if (hv >= 0 && (hv & kRowDone))
                src = reinterpret_cast<const U *>(static_cast<uintptr_t>(hv & ~kRowDone));
        }
        if (__all_sync(0xffffffffu, !rep || src)) break;
        if (it + 1 < limit) __nanosleep(256);
    }
    const bool go = rep && src;
    const bool vec = ((v * (int64_t)sizeof(U)) & 15) == 0 &&
                     __all_sync(0xffffffffu, !go || (((reinterpret_cast<uintptr_t>(src) |
                                                        reinterpret_cast<uintptr_t>(dst)) & 15) == 0));
    copy_rows<U>(__ballot_sync(0xffffffffu, go), go ? src : dst, dst, v, vec);
    const bool lost = rep && !src;
    if (lost) atomicOr(status, kStatusWaitTimeout);
    return lost;
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

// Every position whose (sorted) key repeats the previous one gets a copy of the output row
// decoded for the first position of its run.  A warp takes 32 positions; each distinct
// source row is read once and written to all of its positions in the chunk.  `Rows` maps a
// position and its key to its output row (valid(key), row(k, key), words(key)).
template <typename U, typename Rows>
__global__ void __launch_bounds__(256)
fill_repeats_kernel(const int64_t *__restrict__ keys, int64_t nrows, Rows rows) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
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
        const bool dup = valid && !head && rows.valid(key);
        U *d = dup ? rows.row(k, key) : nullptr;
        unsigned dm = __ballot_sync(0xffffffffu, dup);
        while (dm) {
            const int leader = __ffs(dm) - 1;
            const int64_t hs = __shfl_sync(0xffffffffu, h, leader);
            const int64_t ks = __shfl_sync(0xffffffffu, key, leader);
            const unsigned same = __ballot_sync(0xffffffffu, dup && h == hs) & dm;
            dm &= ~same;
            const U *src = rows.row(hs, ks);
            const int64_t v = rows.words(ks);
            const bool aligned = (((uintptr_t)d) & 15) == 0;
            const bool vec = (((uintptr_t)src) & 15) == 0 && ((v * (int64_t)sizeof(U)) & 15) == 0 &&
                             (__ballot_sync(0xffffffffu, (same >> lane & 1u) && !aligned) == 0);
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
                        U *dj = reinterpret_cast<U *>(
                            __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(d), j));
                        if (q < n16) reinterpret_cast<uint4 *>(dj)[q] = x;
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
                        U *dj = reinterpret_cast<U *>(
                            __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(d), j));
                        if (w < v) dj[w] = x;
                    }
                }
            }
        }
    }
}

// Words of the first read of a compressed row: the caller's average-length hint rounded up
// to whole 32-byte sectors (a row of exactly the hint's length, e.g. one full 128-byte line,
// costs one request); without a hint, the first 128 bytes.
inline int64_t first_read_words(int64_t v, int64_t mw, int wb, int comp_len) {
    const int64_t sector = 32 / wb;
    int64_t want = (comp_len > 0 && comp_len < v) ? (int64_t)comp_len : 128 / wb;
    if (want < mw + 1) want = mw + 1;
    want = (want + sector - 1) / sector * sector;
    return want < v ? want : v;
}

}  // namespace ibp200
