// ibp_codec.cuh -- device building blocks of the compressed row format.
//
// Row format (include/compress/ibp_compress_dev.cuh:7-97, restated):
//   words [0, Mw): bitmap, bit j (LSB-first in 32-bit units) = word j is compressible,
//                  Mw = ceil(ceil(v/8) / wb) words;
//   from word Mw : an MSB-first bit stream; word j contributes its non-invariant bits
//                  (the bits where mask_j is 0, highest first) when compressible, else
//                  all W bits;
//   then zeros up to v words.
//
// Bit gather/scatter (x -> bits of x under `sel`, packed right; and the inverse) uses the
// parallel-suffix method of H. S. Warren, "Hacker's Delight", 2nd ed., sections 7-4
// (compress) and 7-5 (expand): log2(W) steps, each moving bits right by 2^i under a
// per-column "move" mask.  The move masks depend only on the column's mask, so they are
// built once per call (build_tables_kernel) and every word then costs log2(W) branch-free
// steps instead of a data-dependent loop over mask runs.
#pragma once

#include "ibp_common.cuh"

namespace ibp200 {

template <typename U>
struct LogW { static constexpr int value = sizeof(U) == 8 ? 6 : 5; };

// Per-column decode/encode tables, structure-of-arrays in a workspace buffer.
template <typename U>
struct ColTables {
    U *mask;       // [v]
    U *bitval;     // [v]
    U *mv;         // [LogW][v] move masks of sel = ~mask
    uint8_t *nb;   // [v] bits a compressible word keeps = W - popc(mask)
};

template <typename U>
size_t tables_bytes(int64_t v) {
    return align_up((size_t)v * sizeof(U), kAlign) * (2 + LogW<U>::value) +
           align_up((size_t)v, kAlign);
}

template <typename U>
ColTables<U> carve_tables(Carver &c, int64_t v) {
    ColTables<U> t;
    t.mask = c.take<U>(v);
    t.bitval = c.take<U>(v);
    t.mv = c.take<U>((size_t)v * LogW<U>::value);
    t.nb = c.take<uint8_t>(v);
    return t;
}

// Shifts that are well defined for every amount in [0, W].
template <typename U>
__device__ __forceinline__ U shl_w(U x, int s) {
    return s >= (int)(8 * sizeof(U)) ? (U)0 : (U)(x << s);
}
template <typename U>
__device__ __forceinline__ U shr_w(U x, int s) {
    return s >= (int)(8 * sizeof(U)) ? (U)0 : (U)(x >> s);
}

// Move masks for gathering/scattering the bits of `sel` (Hacker's Delight 7-4 / 7-5).
template <typename U>
__device__ __forceinline__ void move_masks(U sel, U *mv, int stride) {
    constexpr int LW = LogW<U>::value;
    U m = sel;
    U mk = (U)(~m << 1);
#pragma unroll
    for (int i = 0; i < LW; ++i) {
        U mp = (U)(mk ^ (mk << 1));
#pragma unroll
        for (int k = 1; k < LW; ++k) mp = (U)(mp ^ (mp << (1 << k)));
        const U v = (U)(mp & m);
        mv[i * stride] = v;
        m = (U)((m ^ v) | (v >> (1 << i)));
        mk = (U)(mk & ~mp);
    }
}

// bits of x at the set positions of sel, packed to the right (pext)
template <typename U>
__device__ __forceinline__ U gather_bits(U x, U sel, const U *mv, int stride) {
    constexpr int LW = LogW<U>::value;
    x &= sel;
#pragma unroll
    for (int i = 0; i < LW; ++i) {
        const U v = mv[i * stride];
        const U t = (U)(x & v);
        x = (U)((x ^ t) | (t >> (1 << i)));
    }
    return x;
}

// inverse of gather_bits: the low bits of y placed at the set positions of sel (pdep)
template <typename U>
__device__ __forceinline__ U scatter_bits(U y, U sel, const U *mv, int stride) {
    constexpr int LW = LogW<U>::value;
#pragma unroll
    for (int i = LW - 1; i >= 0; --i) {
        const U v = mv[i * stride];
        const U t = (U)(y << (1 << i));
        y = (U)((y & ~v) | (t & v));
    }
    return (U)(y & sel);
}

// Column j of the tables.
template <typename U>
__device__ __forceinline__ void build_table_column(const U *__restrict__ mask,
                                                   const U *__restrict__ bitval, int64_t v,
                                                   const ColTables<U> &t, int64_t j) {
    const U m = mask[j];
    t.mask[j] = m;
    t.bitval[j] = bitval[j];
    t.nb[j] = (uint8_t)(8 * sizeof(U) - popc_w(m));
    move_masks<U>((U)~m, t.mv + j, (int)v);
}

template <typename U>
__global__ void build_tables_kernel(const U *__restrict__ mask, const U *__restrict__ bitval,
                                    int64_t v, ColTables<U> t) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < v;
         j += (int64_t)gridDim.x * blockDim.x)
        build_table_column<U>(mask, bitval, v, t, j);
}

template <typename U>
inline ibp_status build_tables(const U *mask, const U *bitval, int64_t v, ColTables<U> t,
                               cudaStream_t st) {
    if (v <= 0) return IBP_OK;
    int blocks = (int)((v + 255) / 256);
    if (blocks > 1024) blocks = 1024;
    build_tables_kernel<U><<<blocks, 256, 0, st>>>(mask, bitval, v, t);
    IBP_LAUNCHED("build_tables_kernel");
    return IBP_OK;
}

// ---- MSB-first stream access on 32-bit units.  Stream bit s of a W-bit word stream
// lives in 32-bit unit s/32 of the stream when W == 32, and in unit (s/32) ^ 1 when
// W == 64 (the high half of a little-endian 64-bit word comes second in memory).
template <typename U>
__device__ __forceinline__ int unit_slot(int64_t q) {
    return sizeof(U) == 8 ? (int)(q ^ 1) : (int)q;
}

// OR the L (0..64) low bits of val into the stream at bit offset s (shared memory units).
template <typename U>
__device__ __forceinline__ void put_bits(uint32_t *units, int64_t s, uint64_t val, int L) {
    if (L <= 0) return;
    const int64_t q = s >> 5;
    const int off = (int)(s & 31);
    // left-align the L bits in 64 bits
    const uint64_t a = (L >= 64) ? val : (val << (64 - L));
    // unit q takes the top (32 - off) bits of a
    atomicOr(&units[unit_slot<U>(q)], (uint32_t)(a >> (32 + off)));
    const int used = 32 - off;
    if (L > used) {
        const uint64_t b = a << used;  // used in [1, 32]
        atomicOr(&units[unit_slot<U>(q + 1)], (uint32_t)(b >> 32));
        if (L > used + 32) atomicOr(&units[unit_slot<U>(q + 2)], (uint32_t)(b & 0xffffffffu));
    }
}

// Read L (0..W) bits at stream offset s from W-bit words (MSB-first); needs word s/W + 1.
template <typename U>
__device__ __forceinline__ U get_bits(const U *words, int64_t s, int L) {
    constexpr int W = 8 * sizeof(U);
    const int64_t q = s / W;
    const int r = (int)(s % W);
    const U hi = words[q], lo = words[q + 1];
    const U win = r == 0 ? hi : (U)((hi << r) | (lo >> (W - r)));
    return shr_w<U>(win, W - L);
}

// The W stream bits that end at stream bit e (e >= 1) of `words`, right-aligned: the word
// whose bits end there, with whatever precedes them above.  Read from 32-bit units with two
// funnel shifts (stream unit t is memory unit t ^ 1 for 64-bit words, whose high half comes
// second in memory, and unit t for 32-bit words).  A compressible word's L kept bits come out
// in the low bits; its scatter never moves the bits above them to a kept position (each kept
// position takes exactly one of the low L bits), so they need no masking, and neither the
// kept-bit count nor a variable shift enters the read.  For e < W the window starts before
// `words`, in the W bits before it, which the caller's buffer holds (a row's bitmap, or the
// stream's earlier words).
template <typename U>
__device__ __forceinline__ U stream_bits_ending(const U *words, int32_t e) {
    const uint32_t *u = reinterpret_cast<const uint32_t *>(words);
    const int32_t s = e - 8 * (int32_t)sizeof(U);
    const int32_t t = s >> 5;  // may be -2 or -1
    const uint32_t r = (uint32_t)s & 31u;
    if constexpr (sizeof(U) == 8) {
        const uint32_t a = u[t ^ 1], b = u[(t + 1) ^ 1], c = u[(t + 2) ^ 1];
        return ((uint64_t)__funnelshift_l(b, a, r) << 32) | __funnelshift_l(c, b, r);
    } else {
        return __funnelshift_l(u[t + 1], u[t], r);
    }
}

// Copy `words` W-bit words between global buffers with a warp; 16-byte accesses when both
// sides are 16-byte aligned.
template <typename U>
__device__ __forceinline__ void warp_copy(U *__restrict__ dst, const U *__restrict__ src,
                                          int64_t words) {
    const int lane = threadIdx.x & 31;
    const int64_t bytes = words * (int64_t)sizeof(U);
    if ((((uintptr_t)dst | (uintptr_t)src) & 15) == 0) {
        const int64_t n16 = bytes >> 4;
        const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
        uint4 *d4 = reinterpret_cast<uint4 *>(dst);
        for (int64_t k = lane; k < n16; k += 32) d4[k] = s4[k];
        for (int64_t k = (n16 << 4) / (int64_t)sizeof(U) + lane; k < words; k += 32) dst[k] = src[k];
    } else {
        for (int64_t k = lane; k < words; k += 32) dst[k] = src[k];
    }
}

}  // namespace ibp200
