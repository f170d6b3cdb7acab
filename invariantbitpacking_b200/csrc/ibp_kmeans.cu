// ibp_kmeans.cu -- bitwise k-means preprocessing (replaces
// include/preproc/ibp_preproc_host.cuh:118-284 and include/preproc/ibp_preproc_kmeans.cuh).
//
// B200 design
//  * a host-resident table is copied to HBM once by the copy engine (when the caller's
//    workspace has room) and all ten rounds read HBM; the reference re-reads pinned host
//    memory over PCIe in every round.
//  * assignment: one warp per row, centroids in shared memory, warp-reduced Hamming
//    distances; ties go to the highest centroid id (a deterministic choice among the
//    reference's racy outcomes, see include/preproc/ibp_preproc_kmeans.cuh:139-146).
//  * update: per-(cluster, word, bit) set counts.  A warp takes 32 rows (lane = row),
//    forms one membership ballot per cluster and one ballot per bit, and adds
//    popc(bit ballot & membership) into per-block shared-memory counters (lane = cluster:
//    one shared atomic per (cluster, bit) per 32 rows, no bank conflicts); the reference
//    issues one global atomic per set bit.
//  * the counts of the last round are exactly those of the final assignment, so the
//    final masks need no extra pass over the data.
#include <algorithm>
#include <vector>

#include "ibp_common.cuh"
#include "ibp_internal.cuh"

namespace ibp200 {

constexpr int kKmRounds = 10;  // include/preproc/ibp_preproc_host.cuh:191

template <typename U>
__global__ void seed_centroids_kernel(const U *__restrict__ data, int64_t n, int64_t v,
                                      const int64_t *__restrict__ init, int c,
                                      U *__restrict__ cent, int32_t *__restrict__ status) {
    const int64_t seeded = (int64_t)c < n ? (int64_t)c : n;
    const int64_t total = (int64_t)c * v;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / v, k = e % v;
        U x = 0;
        if (i < seeded) {
            const int64_t r = i == 0 ? 0 : init[i];
            if (r >= 0 && r < n)
                x = data[r * v + k];
            else if (k == 0)
                atomicOr(status, kStatusBadIndex);
        }
        cent[e] = x;
    }
}

// clusters[i] = argmin_j popcount(row_i ^ centroid_j), highest j on ties.
template <typename U>
__global__ void __launch_bounds__(256)
assign_kernel(const U *__restrict__ data, int64_t n, int64_t v, const U *__restrict__ cent_g,
              int c, bool cent_in_smem, int32_t *__restrict__ clusters) {
    extern __shared__ __align__(16) unsigned char smem[];
    U *cent_s = reinterpret_cast<U *>(smem);
    if (cent_in_smem) {
        for (int64_t e = threadIdx.x; e < (int64_t)c * v; e += blockDim.x) cent_s[e] = cent_g[e];
        __syncthreads();
    }
    const U *cent = cent_in_smem ? cent_s : cent_g;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < n; i += nwarps) {
        const U *row = data + i * v;
        int best = 0;
        uint32_t bestd = 0xffffffffu;
        for (int j = 0; j < c; ++j) {
            uint32_t d = 0;
            for (int64_t k = lane; k < v; k += 32) d += popc_w((U)(row[k] ^ cent[(int64_t)j * v + k]));
            d = __reduce_add_sync(0xffffffffu, d);
            if (d <= bestd) {
                bestd = d;
                best = j;
            }
        }
        if (lane == 0) clusters[i] = best;
    }
}

// bits[(cl*v + k)*W + b] += rows of cluster cl with bit b of word k set.
// Block (bx, tile) covers words [tile*kt, tile*kt + kt); shared counters [C][kt*W + 1].
template <typename U>
__global__ void __launch_bounds__(256)
cluster_bits_kernel(const U *__restrict__ data, int64_t n, int64_t v,
                    const int32_t *__restrict__ clusters, int c, int kt,
                    uint32_t *__restrict__ bits) {
    constexpr int W = 8 * sizeof(U);
    extern __shared__ uint32_t sc[];
    const int stride = kt * W + 1;
    const int64_t k0 = (int64_t)blockIdx.y * kt;
    const int kn = (int)((v - k0) < kt ? (v - k0) : kt);
    for (int e = threadIdx.x; e < c * stride; e += blockDim.x) sc[e] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t g = warp; g * 32 < n; g += nwarps) {
        const int64_t r = g * 32 + lane;
        const bool live = r < n;
        const int cl = live ? clusters[r] : -1;
        for (int cb = 0; cb < c; cb += 32) {
            uint32_t mine = 0;
            const int lim = (c - cb) < 32 ? (c - cb) : 32;
            for (int q = 0; q < lim; ++q) {
                const uint32_t m = __ballot_sync(0xffffffffu, cl == cb + q);
                if (lane == q) mine = m;
            }
            if (__ballot_sync(0xffffffffu, mine != 0) == 0) continue;
            uint32_t *myc = sc + (int64_t)(cb + lane) * stride;
            for (int kk = 0; kk < kn; ++kk) {
                const U x = live ? data[r * v + k0 + kk] : (U)0;
#pragma unroll 8
                for (int b = 0; b < W; ++b) {
                    const uint32_t bm = __ballot_sync(0xffffffffu, (x >> b) & 1);
                    // the block's warps share these counters: shared-memory atomics
                    if (lane < lim && (bm & mine)) atomicAdd(&myc[kk * W + b], __popc(bm & mine));
                }
            }
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < c * kt * W; e += blockDim.x) {
        const int cl = e / (kt * W), rem = e % (kt * W);
        const int kk = rem / W, b = rem % W;
        if (kk < kn) {
            const uint32_t val = sc[cl * stride + rem];
            if (val) atomicAdd(&bits[(cl * v + k0 + kk) * W + b], val);
        }
    }
}

// cnt[cl] = members of cluster cl
__global__ void cluster_sizes_kernel(const int32_t *__restrict__ clusters, int64_t n, int c,
                                     uint32_t *__restrict__ cnt) {
    extern __shared__ uint32_t hist[];
    for (int e = threadIdx.x; e < c; e += blockDim.x) hist[e] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int cl = clusters[i];
        if (cl >= 0 && cl < c) atomicAdd(&hist[cl], 1u);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < c; e += blockDim.x)
        if (hist[e]) atomicAdd(&cnt[e], hist[e]);
}

// Majority centroids with the reference's per-lane OR accumulation
// (include/preproc/ibp_preproc_kmeans.cuh:219-236): bit set when count > size/2 (int div).
template <typename U>
__global__ void majority_kernel(const uint32_t *__restrict__ bits, const uint32_t *__restrict__ cnt,
                                int64_t v, int c, U *__restrict__ cent) {
    constexpr int W = 8 * sizeof(U);
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (tid >= (int64_t)c * 32) return;
    const int cl = (int)(tid / 32), lane = (int)(tid % 32);
    const uint32_t half = (uint32_t)((int32_t)cnt[cl] / 2);
    uint64_t acc = 0;
    for (int64_t id = lane; id < v; id += 32) {
        const uint32_t *bb = bits + ((int64_t)cl * v + id) * W;
        for (int b = 0; b < W; ++b)
            if ((int32_t)bb[b] > (int32_t)half) acc |= 1ull << b;
        cent[(int64_t)cl * v + id] = (U)acc;
    }
}

// Per-cluster masks (include/preproc/ibp_preproc_kmeans.cuh:238-297): counts accumulate in
// float32 there (saturating at 2^24); `>= thr*count` in float32, `<= (1-thr)*count` in
// float64; an empty cluster yields all-ones mask and bitval.
template <typename U>
__global__ void cluster_masks_kernel(const uint32_t *__restrict__ bits,
                                     const uint32_t *__restrict__ cnt, int64_t v, int c,
                                     float thr, U *__restrict__ masks, U *__restrict__ bitvals) {
    constexpr int W = 8 * sizeof(U);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)c * v;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int cl = (int)(e / v);
        const int32_t count = (int32_t)cnt[cl];
        const float lim1 = __fmul_rn(thr, (float)count);
        const double lim0 = __dmul_rn(1.0 - (double)thr, (double)count);
        const uint32_t *bb = bits + e * W;
        uint64_t m = 0, val = 0;
        for (int b = 0; b < W; ++b) {
            const uint32_t bs = bb[b];
            const float bsf = bs > 16777216u ? 16777216.0f : (float)bs;
            if (bsf >= lim1) {
                val |= 1ull << b;
                m |= 1ull << b;
            } else if ((double)bsf <= lim0) {
                m |= 1ull << b;
            }
        }
        masks[e] = (U)m;
        bitvals[e] = (U)val;
    }
}

size_t kmeans_workspace(int64_t n, int64_t v, int wb, int c) {
    Sizer s;
    s.take<char>(kStatusBytes);
    s.take<int64_t>((size_t)c);                     // seed rows
    s.take<char>((size_t)c * v * wb);               // centroids
    s.take<uint32_t>((size_t)c * v * 8 * wb);       // bit counts
    s.take<uint32_t>((size_t)c);                    // cluster sizes
    s.take<int32_t>((size_t)n);                     // assignments
    return s.total();
}

static int kt_for(int64_t v, int c, int W, size_t &smem) {
    const size_t budget = 96 * 1024;
    int64_t kt = (int64_t)(budget / ((size_t)c * W * 4 + 4));
    if (kt > v) kt = v;
    if (kt < 1) kt = 1;
    smem = (size_t)c * ((size_t)kt * W + 1) * 4;
    return (int)kt;
}

template <typename U>
ibp_status kmeans_impl(const U *data, int64_t n, int64_t v, int c, const int64_t *init_rows,
                       U *masks, U *bitvals, int32_t *clusters, void *ws, size_t ws_bytes,
                       cudaStream_t st) {
    constexpr int W = 8 * sizeof(U);
    const int wb = sizeof(U);
    Carver cv{(char *)ws, 0, ws_bytes};
    int32_t *status = cv.take<int32_t>(kStatusBytes / 4);
    int64_t *seed = cv.take<int64_t>((size_t)c);
    U *cent = cv.take<U>((size_t)c * v);
    uint32_t *bits = cv.take<uint32_t>((size_t)c * v * W);
    uint32_t *cnt = cv.take<uint32_t>((size_t)c);
    int32_t *assign = cv.take<int32_t>((size_t)n);
    if (!assign) {
        set_error("preprocess_kmeans: workspace of %zu bytes is below the required %zu",
                  ws_bytes, kmeans_workspace(n, v, wb, c));
        return IBP_ERR_WORKSPACE;
    }
    // optional HBM copy of a host-resident table (room left in the workspace)
    U *stage = cv.take<U>((size_t)(n * v));
    IBP_CUDA(cudaMemsetAsync(status, 0, sizeof(int32_t), st));
    const U *rows = data;
    if (stage && n > 0) {
        cudaPointerAttributes pa{};
        if (cudaPointerGetAttributes(&pa, data) == cudaSuccess && pa.type != cudaMemoryTypeDevice &&
            pa.type != cudaMemoryTypeManaged) {
            IBP_CUDA(cudaMemcpyAsync(stage, data, (size_t)(n * v) * wb, cudaMemcpyDefault, st));
            rows = stage;
        }
        cudaGetLastError();
    }
    const int64_t seeded = (int64_t)c < n ? (int64_t)c : n;
    std::vector<int64_t> h(c > 0 ? c : 1, 0);
    for (int64_t i = 1; i < seeded; ++i) h[i] = init_rows[i];
    IBP_CUDA(cudaMemcpyAsync(seed, h.data(), sizeof(int64_t) * c, cudaMemcpyHostToDevice, st));
    const int sms = device_sm_count();
    {
        int64_t tot = (int64_t)c * v;
        int blocks = (int)std::min<int64_t>((tot + 255) / 256, 1024);
        seed_centroids_kernel<U><<<blocks, 256, 0, st>>>(rows, n, v, seed, c, cent, status);
        IBP_LAUNCHED("seed_centroids_kernel");
    }
    IBP_CUDA(cudaMemsetAsync(assign, 0, sizeof(int32_t) * n, st));
    if (n == 0) {
        IBP_CUDA(cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * c, st));
        IBP_CUDA(cudaMemsetAsync(bits, 0, sizeof(uint32_t) * c * v * W, st));
    }
    const size_t cent_bytes = (size_t)c * v * wb;
    const bool cent_smem = cent_bytes <= 64 * 1024;
    auto akern = assign_kernel<U>;
    if (cent_smem && cent_bytes > 48 * 1024)
        IBP_CUDA(cudaFuncSetAttribute(akern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cent_bytes));
    size_t bsmem = 0;
    const int kt = kt_for(v, c, W, bsmem);
    auto bkern = cluster_bits_kernel<U>;
    if (bsmem > 48 * 1024)
        IBP_CUDA(cudaFuncSetAttribute(bkern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsmem));
    const int64_t tiles = (v + kt - 1) / kt;
    int64_t gx = (n + 255) / 256;
    const int64_t capx = std::max<int64_t>(1, (int64_t)sms * 2 / tiles);
    if (gx > capx) gx = capx;
    if (gx < 1) gx = 1;
    int64_t ablocks = std::min<int64_t>((n + 7) / 8, (int64_t)sms * 8);
    if (ablocks < 1) ablocks = 1;
    for (int it = 0; it < kKmRounds && n > 0; ++it) {
        akern<<<(unsigned)ablocks, 256, cent_smem ? cent_bytes : 0, st>>>(rows, n, v, cent, c,
                                                                          cent_smem, assign);
        IBP_LAUNCHED("assign_kernel");
        IBP_CUDA(cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * c, st));
        IBP_CUDA(cudaMemsetAsync(bits, 0, sizeof(uint32_t) * c * v * W, st));
        bkern<<<dim3((unsigned)gx, (unsigned)tiles), 256, bsmem, st>>>(rows, n, v, assign, c,
                                                                        kt, bits);
        IBP_LAUNCHED("cluster_bits_kernel");
        cluster_sizes_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, sms * 4), 256,
                               sizeof(uint32_t) * c, st>>>(assign, n, c, cnt);
        IBP_LAUNCHED("cluster_sizes_kernel");
        majority_kernel<U><<<(c * 32 + 255) / 256, 256, 0, st>>>(bits, cnt, v, c, cent);
        IBP_LAUNCHED("majority_kernel");
    }
    if (n > 0)
        IBP_CUDA(cudaMemcpyAsync(clusters, assign, sizeof(int32_t) * n, cudaMemcpyDefault, st));
    // the reference's final sweep leaves the masks of its last step, thr = 1.0f
    const ThrList sweep = sweep_thresholds(-1.0f);
    const float last = sweep.v[sweep.count - 1];
    if (c > 0 && v > 0) {
        int blocks = (int)std::min<int64_t>(((int64_t)c * v + 255) / 256, 1024);
        cluster_masks_kernel<U><<<blocks, 256, 0, st>>>(bits, cnt, v, c, last, masks, bitvals);
        IBP_LAUNCHED("cluster_masks_kernel");
    }
    return IBP_OK;
}

template ibp_status kmeans_impl<uint32_t>(const uint32_t *, int64_t, int64_t, int,
                                          const int64_t *, uint32_t *, uint32_t *, int32_t *,
                                          void *, size_t, cudaStream_t);
template ibp_status kmeans_impl<uint64_t>(const uint64_t *, int64_t, int64_t, int,
                                          const int64_t *, uint64_t *, uint64_t *, int32_t *,
                                          void *, size_t, cudaStream_t);

}  // namespace ibp200
