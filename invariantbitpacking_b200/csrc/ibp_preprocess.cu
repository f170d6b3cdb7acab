// ibp_preprocess.cu -- invariant-bit census, per-threshold masks, fused saved-bit check and
// on-device threshold selection (replaces include/preproc/ibp_preproc_host.cuh:23-115 and
// include/preproc/ibp_preproc_kernels.cuh:7-77).
//
// B200 design
//  * census: each thread owns one word column and keeps 8 bit-sliced vertical counters
//    (a ripple-carry adder in registers, 16 logic ops per word) that it flushes into
//    per-thread shared-memory counters every 255 rows; one global atomic per
//    (column, bit) per block at the end.  Reads are coalesced 32-word row slices.
//    A host-resident dataset is optionally staged into HBM during this pass so the
//    second pass reads HBM instead of PCIe.
//  * all sweep thresholds are checked in ONE pass over the data (the reference makes one
//    PCIe pass and one host round trip per threshold) and the winning mask is selected
//    by a one-block kernel, so preprocess never blocks the host.
#include "ibp_common.cuh"
#include "ibp_internal.cuh"

namespace ibp200 {

constexpr int kCensusThreads = 256;
constexpr int kCensusDepth = 8;  // bit-sliced counter levels: flush every 255 rows

template <typename U>
using Reg = typename std::conditional<(sizeof(U) < 4), uint32_t, U>::type;

// counts[col * W + b] += number of rows whose word `col` has bit b set.
// Block (bx, tile) covers columns [tile*cpb, tile*cpb + cpb) and rows bx*R + r_local + k*gx*R.
template <typename U>
__global__ void __launch_bounds__(kCensusThreads)
census_kernel(const U *__restrict__ data, int64_t n, int64_t v, int cpb, int R,
              uint32_t *__restrict__ counts, U *__restrict__ stage) {
    constexpr int W = WordBits<U>::value;
    extern __shared__ uint32_t sc[];  // [W][kCensusThreads]
    const int t = threadIdx.x;
    const int c_local = t % cpb, r_local = t / cpb;
    const int64_t col = (int64_t)blockIdx.y * cpb + c_local;
    const bool active = (r_local < R) && (col < v);
    for (int b = 0; b < W; ++b) sc[b * kCensusThreads + t] = 0;

    Reg<U> s[kCensusDepth];
#pragma unroll
    for (int d = 0; d < kCensusDepth; ++d) s[d] = 0;

    auto flush = [&]() {
#pragma unroll
        for (int b = 0; b < W; ++b) {
            uint32_t c = 0;
#pragma unroll
            for (int d = 0; d < kCensusDepth; ++d) c |= (uint32_t)((s[d] >> b) & 1u) << d;
            sc[b * kCensusThreads + t] += c;
        }
#pragma unroll
        for (int d = 0; d < kCensusDepth; ++d) s[d] = 0;
    };
    auto add = [&](Reg<U> x) {
#pragma unroll
        for (int d = 0; d < kCensusDepth; ++d) {
            Reg<U> carry = s[d] & x;
            s[d] ^= x;
            x = carry;
        }
    };

    if (active) {
        const int64_t rstride = (int64_t)gridDim.x * R;
        int64_t r = (int64_t)blockIdx.x * R + r_local;
        int pending = 0;
        constexpr int UNR = 4;
        for (; r + (UNR - 1) * rstride < n; r += UNR * rstride) {
            U x[UNR];
#pragma unroll
            for (int u = 0; u < UNR; ++u) x[u] = data[(r + u * rstride) * v + col];
#pragma unroll
            for (int u = 0; u < UNR; ++u) {
                if (stage) stage[(r + u * rstride) * v + col] = x[u];
                add((Reg<U>)x[u]);
            }
            pending += UNR;
            if (pending > 255 - UNR) {
                flush();
                pending = 0;
            }
        }
        for (; r < n; r += rstride) {
            U x = data[r * v + col];
            if (stage) stage[r * v + col] = x;
            add((Reg<U>)x);
            if (++pending == 255) {
                flush();
                pending = 0;
            }
        }
        flush();
    }
    __syncthreads();
    // reduce the R row slots of each column, one global atomic per (column, bit)
    if (r_local == 0 && col < v) {
        for (int b = 0; b < W; ++b) {
            uint32_t tot = 0;
            for (int k = 0; k < R; ++k) tot += sc[b * kCensusThreads + t + k * cpb];
            if (tot) atomicAdd(&counts[col * W + b], tot);
        }
    }
}

// One mask/bitval pair per threshold: include/preproc/ibp_preproc_kernels.cuh:33-51.
// `count > thr * N` is a float32 product and compare, `count < (1 - thr) * N` float64.
template <typename U>
__global__ void masks_from_counts_kernel(const uint32_t *__restrict__ counts, int64_t n,
                                         int64_t v, ThrList thr, U *__restrict__ masks,
                                         U *__restrict__ bitvals) {
    constexpr int W = WordBits<U>::value;
    const int64_t total = v * thr.count;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int ti = (int)(e / v);
        const int64_t j = e % v;
        const float t = thr.v[ti];
        const float lim1 = __fmul_rn(t, (float)(unsigned long long)n);
        const double lim0 = __dmul_rn(1.0 - (double)t, (double)(unsigned long long)n);
        uint64_t m = 0, val = 0;
        for (int b = 0; b < W; ++b) {
            const int32_t c = (int32_t)counts[j * W + b];
            if ((float)c > lim1) {
                val |= 1ull << b;
                m |= 1ull << b;
            } else if ((double)c < lim0) {
                m |= 1ull << b;
            }
        }
        masks[e] = (U)m;
        bitvals[e] = (U)val;
    }
}

// saved[t] += sum over rows of max(0, S_t(row) - v), S_t = sum of popc(mask_t[j]) over the
// words with (x & mask_t[j]) == bitval_t[j]: include/preproc/ibp_preproc_kernels.cuh:53-77,
// for every threshold of the sweep in one pass.  One warp per row.
template <typename U>
__global__ void __launch_bounds__(256)
check_saved_kernel(const U *__restrict__ data, int64_t n, int64_t v, int nthr,
                   const U *__restrict__ masks, const U *__restrict__ bitvals,
                   unsigned long long *__restrict__ saved) {
    __shared__ unsigned long long blk[kMaxThresholds];
    if (threadIdx.x < kMaxThresholds) blk[threadIdx.x] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long acc[kMaxThresholds];
#pragma unroll
    for (int t = 0; t < kMaxThresholds; ++t) acc[t] = 0;
    for (int64_t r = warp; r < n; r += nwarps) {
        uint32_t s[kMaxThresholds];
#pragma unroll
        for (int t = 0; t < kMaxThresholds; ++t) s[t] = 0;
        const U *row = data + r * v;
        for (int64_t j = lane; j < v; j += 32) {
            const U x = row[j];
#pragma unroll
            for (int t = 0; t < kMaxThresholds; ++t) {
                if (t < nthr) {
                    const U m = __ldg(&masks[t * v + j]);
                    if ((U)(x & m) == __ldg(&bitvals[t * v + j])) s[t] += popc_w(m);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < kMaxThresholds; ++t) {
            if (t < nthr) {
                const uint32_t tot = __reduce_add_sync(0xffffffffu, s[t]);
                if (tot > (uint64_t)v) acc[t] += tot - (uint64_t)v;
            }
        }
    }
    if (lane == 0) {
#pragma unroll
        for (int t = 0; t < kMaxThresholds; ++t)
            if (t < nthr && acc[t]) atomicAdd(&blk[t], acc[t]);
    }
    __syncthreads();
    if (threadIdx.x < nthr && blk[threadIdx.x]) atomicAdd(&saved[threadIdx.x], blk[threadIdx.x]);
}

// First threshold with strictly more saved bits than every earlier one (and > 0) wins;
// its mask/bitval go to the outputs, which are zero when none saves anything
// (include/preproc/ibp_preproc_host.cuh:91-99, src/preprocess.cu:46-47).
template <typename U>
__global__ void select_mask_kernel(const unsigned long long *__restrict__ saved, int nthr,
                                   int64_t v, const U *__restrict__ masks,
                                   const U *__restrict__ bitvals, U *__restrict__ mask_out,
                                   U *__restrict__ bitval_out, int32_t *__restrict__ selected) {
    int sel = -1;
    double best = 0.0;
    for (int t = 0; t < nthr; ++t) {
        if ((double)saved[t] > best) {
            best = (double)saved[t];
            sel = t;
        }
    }
    if (threadIdx.x == 0 && blockIdx.x == 0 && selected) *selected = sel;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < v;
         j += (int64_t)gridDim.x * blockDim.x) {
        mask_out[j] = sel >= 0 ? masks[sel * v + j] : (U)0;
        bitval_out[j] = sel >= 0 ? bitvals[sel * v + j] : (U)0;
    }
}

ThrList sweep_thresholds(float threshold) {
    // include/preproc/ibp_preproc_host.cuh:61-67: float loop variable, `+= 0.05` in double
    ThrList l{};
    l.count = 0;
    const float lo = threshold < 0 ? (float)0.7 : threshold;
    const float hi = threshold < 0 ? (float)1.0 : threshold;
    for (float t = lo; t <= hi && l.count < kMaxThresholds; t = (float)((double)t + 0.05))
        l.v[l.count++] = t;
    return l;
}

static void census_geometry(int64_t n, int64_t v, int &cpb, int &R, dim3 &grid) {
    cpb = (int)(v < kCensusThreads ? v : kCensusThreads);
    R = kCensusThreads / cpb;
    const int64_t tiles = (v + cpb - 1) / cpb;
    const int sms = device_sm_count();
    int64_t gx = (n + (int64_t)R * 512 - 1) / ((int64_t)R * 512);
    int64_t cap = (int64_t)sms * 8 / tiles;
    if (cap < 1) cap = 1;
    if (gx > cap) gx = cap;
    if (gx < 1) gx = 1;
    grid = dim3((unsigned)gx, (unsigned)tiles);
}

size_t preprocess_workspace(int64_t n, int64_t v, int wb, float threshold, bool staged) {
    Sizer s;
    s.take<char>(kStatusBytes);
    const ThrList l = sweep_thresholds(threshold);
    s.take<uint32_t>((size_t)(v * 8 * wb));              // counts
    s.take<char>((size_t)(l.count > 0 ? l.count : 1) * v * wb);  // masks
    s.take<char>((size_t)(l.count > 0 ? l.count : 1) * v * wb);  // bitvals
    s.take<unsigned long long>(kMaxThresholds);          // saved bits
    s.take<int32_t>(4);                                  // selected step
    if (staged) s.take<char>((size_t)(n * v * wb));
    return s.total();
}

template <typename U>
ibp_status preprocess_impl(const U *data, int64_t n, int64_t v, float threshold, U *mask,
                           U *bitval, void *ws, size_t ws_bytes, bool data_on_host,
                           cudaStream_t st) {
    const int wb = sizeof(U);
    const ThrList thr = sweep_thresholds(threshold);
    Carver c{(char *)ws, 0, ws_bytes};
    c.take<char>(kStatusBytes);
    uint32_t *counts = c.take<uint32_t>((size_t)(v * 8 * wb));
    U *masks = c.take<U>((size_t)(thr.count > 0 ? thr.count : 1) * v);
    U *bitvals = c.take<U>((size_t)(thr.count > 0 ? thr.count : 1) * v);
    unsigned long long *saved = c.take<unsigned long long>(kMaxThresholds);
    int32_t *selected = c.take<int32_t>(4);
    if (!selected) {
        set_error("preprocess: workspace of %zu bytes is below the required %zu", ws_bytes,
                  preprocess_workspace(n, v, wb, threshold, false));
        return IBP_ERR_WORKSPACE;
    }
    U *stage = nullptr;
    if (data_on_host && thr.count > 0) stage = c.take<U>((size_t)(n * v));  // null if it does not fit
    IBP_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * v * 8 * wb, st));
    IBP_CUDA(cudaMemsetAsync(saved, 0, sizeof(unsigned long long) * kMaxThresholds, st));
    if (n > 0 && v > 0) {
        int cpb, R;
        dim3 grid;
        census_geometry(n, v, cpb, R, grid);
        const size_t smem = sizeof(uint32_t) * 8 * wb * kCensusThreads;
        auto kern = census_kernel<U>;
        if (smem > 48 * 1024)
            IBP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        kern<<<grid, kCensusThreads, smem, st>>>(data, n, v, cpb, R, counts, stage);
        IBP_LAUNCHED("census_kernel");
    }
    if (thr.count > 0 && v > 0) {
        const int64_t tot = v * thr.count;
        const int blocks = (int)((tot + 255) / 256 < 4096 ? (tot + 255) / 256 : 4096);
        masks_from_counts_kernel<U><<<blocks, 256, 0, st>>>(counts, n, v, thr, masks, bitvals);
        IBP_LAUNCHED("masks_from_counts_kernel");
        if (n > 0) {
            const int sms = device_sm_count();
            int64_t blocks2 = (n + 7) / 8;
            if (blocks2 > (int64_t)sms * 8) blocks2 = (int64_t)sms * 8;
            check_saved_kernel<U><<<(unsigned)blocks2, 256, 0, st>>>(
                stage ? stage : data, n, v, thr.count, masks, bitvals, saved);
            IBP_LAUNCHED("check_saved_kernel");
        }
    }
    if (v > 0) {
        const int blocks = (int)((v + 255) / 256 < 1024 ? (v + 255) / 256 : 1024);
        select_mask_kernel<U><<<blocks, 256, 0, st>>>(saved, thr.count, v, masks, bitvals, mask,
                                                      bitval, selected);
        IBP_LAUNCHED("select_mask_kernel");
    }
    return IBP_OK;
}

template ibp_status preprocess_impl<uint8_t>(const uint8_t *, int64_t, int64_t, float, uint8_t *,
                                             uint8_t *, void *, size_t, bool, cudaStream_t);
template ibp_status preprocess_impl<uint16_t>(const uint16_t *, int64_t, int64_t, float,
                                              uint16_t *, uint16_t *, void *, size_t, bool,
                                              cudaStream_t);
template ibp_status preprocess_impl<uint32_t>(const uint32_t *, int64_t, int64_t, float,
                                              uint32_t *, uint32_t *, void *, size_t, bool,
                                              cudaStream_t);
template ibp_status preprocess_impl<uint64_t>(const uint64_t *, int64_t, int64_t, float,
                                              uint64_t *, uint64_t *, void *, size_t, bool,
                                              cudaStream_t);

}  // namespace ibp200
