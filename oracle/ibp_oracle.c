/*
 * ibp_oracle.c -- CPU restatement of the reference Invariant Bit Packing codec.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product.  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs load it.
 *
 * Each function states the reference file:line whose behaviour it follows
 * (paths relative to the reference repository root).  Device-side
 * implementation details that do not change results (shared-memory rings,
 * cp.async staging, warp scans) are not restated; the arithmetic is:
 *   - GPU 32-bit float product thr*N vs (float)count, and the float64
 *     (1.0-thr)*N vs (double)count of create_mask;
 *   - the float32 sweep t = (float)((double)t + 0.05) from 0.7f to 1.0f;
 *   - the byte-size formula and "strictly smaller" rule of the size check;
 *   - the MSB-first bit stream, LSB-first bitmap and zero padding of the
 *     compressed row.
 */
#include "ibp_oracle.h"

#include <omp.h>
#include <stdlib.h>
#include <string.h>

static int g_threads = 0;
void orc_set_threads(int t) { g_threads = t; }
int orc_get_threads(void) { return g_threads > 0 ? g_threads : omp_get_max_threads(); }
#define NT orc_get_threads()

static inline uint64_t wmask(int W) { return W >= 64 ? ~0ull : ((1ull << W) - 1ull); }

static inline uint64_t ldw(const void *p, int64_t i, int wb) {
    switch (wb) {
    case 1: return ((const uint8_t *)p)[i];
    case 2: return ((const uint16_t *)p)[i];
    case 4: return ((const uint32_t *)p)[i];
    default: return ((const uint64_t *)p)[i];
    }
}

static inline void stw(void *p, int64_t i, int wb, uint64_t x) {
    switch (wb) {
    case 1: ((uint8_t *)p)[i] = (uint8_t)x; break;
    case 2: ((uint16_t *)p)[i] = (uint16_t)x; break;
    case 4: ((uint32_t *)p)[i] = (uint32_t)x; break;
    default: ((uint64_t *)p)[i] = x; break;
    }
}

static inline int popc(uint64_t x) { return __builtin_popcountll(x); }

/* ---------------------------------------------------------------- preprocess */

/* include/preproc/ibp_preproc_kernels.cuh:7-31 (count_bit_kernel) */
void orc_count_bits(const void *data, int64_t n, int64_t v, int wb, uint32_t *counts) {
    const int W = 8 * wb;
    const int64_t nc = v * W;
    memset(counts, 0, sizeof(uint32_t) * nc);
    int nt = NT;
    uint32_t *loc = (uint32_t *)calloc((size_t)nt * nc, sizeof(uint32_t));
#pragma omp parallel num_threads(nt)
    {
        int t = omp_get_thread_num();
        uint32_t *c = loc + (size_t)t * nc;
#pragma omp for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            for (int64_t j = 0; j < v; ++j) {
                uint64_t x = ldw(data, i * v + j, wb);
                uint32_t *cj = c + j * W;
                while (x) {
                    int b = __builtin_ctzll(x);
                    cj[b]++;
                    x &= x - 1;
                }
            }
        }
    }
    for (int t = 0; t < nt; ++t)
        for (int64_t k = 0; k < nc; ++k) counts[k] += loc[(size_t)t * nc + k];
    free(loc);
}

/* include/preproc/ibp_preproc_kernels.cuh:33-51 (create_mask).
 * `count > threshold * num_vecs` is a float32 product and compare;
 * `count < (1.0 - threshold) * num_vecs` is evaluated in float64. */
void orc_create_mask(const uint32_t *counts, int64_t n, int64_t v, int wb, float thr,
                     void *mask, void *bitval) {
    const int W = 8 * wb;
    volatile float lim1 = thr * (float)(uint64_t)n;
    volatile double lim0 = (1.0 - (double)thr) * (double)(uint64_t)n;
    for (int64_t j = 0; j < v; ++j) {
        uint64_t m = 0, val = 0;
        for (int b = 0; b < W; ++b) {
            int32_t c = (int32_t)counts[j * W + b];
            if ((float)c > lim1) {
                val |= 1ull << b;
                m |= 1ull << b;
            } else if ((double)c < lim0) {
                m |= 1ull << b;
            }
        }
        stw(mask, j, wb, m);
        stw(bitval, j, wb, val);
    }
}

/* include/preproc/ibp_preproc_kernels.cuh:53-77 (check_feats): a row only counts
 * when its saved bits exceed vec_size (one metadata bit per word). */
uint64_t orc_check_feats(const void *data, int64_t n, int64_t v, int wb,
                         const void *mask, const void *bitval) {
    uint64_t tot = 0;
#pragma omp parallel for schedule(static) reduction(+ : tot) num_threads(NT)
    for (int64_t i = 0; i < n; ++i) {
        uint64_t s = 0;
        for (int64_t j = 0; j < v; ++j) {
            uint64_t m = ldw(mask, j, wb), b = ldw(bitval, j, wb);
            if ((ldw(data, i * v + j, wb) & m) == b) s += (uint64_t)popc(m);
        }
        if (s > (uint64_t)v) tot += s - (uint64_t)v;
    }
    return tot;
}

/* include/preproc/ibp_preproc_host.cuh:23-115 (preproc_data): one census, then for each
 * threshold of the float32 sweep a mask and its saved-bit count; the first threshold with
 * strictly more saved bits than every earlier one wins; nothing is written if none saves. */
int orc_preprocess(const void *data, int64_t n, int64_t v, int wb, float thr, void *mask,
                   void *bitval, uint64_t *saved_per_step, float *thr_per_step, int *num_steps) {
    const int W = 8 * wb;
    uint32_t *counts = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(v * W));
    void *m = malloc((size_t)(v * wb)), *b = malloc((size_t)(v * wb));
    orc_count_bits(data, n, v, wb, counts);
    float min_t = thr < 0 ? (float)0.7 : thr;
    float max_t = thr < 0 ? (float)1.0 : thr;
    double max_saved = 0;
    int sel = -1, step = 0;
    for (float t = min_t; t <= max_t; t = (float)((double)t + 0.05)) {
        orc_create_mask(counts, n, v, wb, t, m, b);
        uint64_t saved = orc_check_feats(data, n, v, wb, m, b);
        if (saved_per_step) saved_per_step[step] = saved;
        if (thr_per_step) thr_per_step[step] = t;
        if ((double)saved > max_saved) {
            memcpy(mask, m, (size_t)(v * wb));
            memcpy(bitval, b, (size_t)(v * wb));
            max_saved = (double)saved;
            sel = step;
        }
        step++;
    }
    if (num_steps) *num_steps = step;
    free(counts);
    free(m);
    free(b);
    return sel;
}

/* ---------------------------------------------------------------- sizes */

static inline int64_t roundup(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

static inline int64_t meta_bytes(int64_t v, int wb) { return roundup((v + 7) / 8, wb); }

/* include/misc/ibp_misc_dev.cuh:19-46 (check_compress_size_blk) and :61-91 (warp form) */
static inline int64_t row_size(const void *row, int64_t v, int wb, const void *mask,
                               const void *bitval) {
    uint64_t s = 0;
    for (int64_t j = 0; j < v; ++j) {
        uint64_t m = ldw(mask, j, wb);
        if ((ldw(row, j, wb) & m) == ldw(bitval, j, wb)) s += (uint64_t)popc(m);
    }
    const int64_t vb = v * wb;
    int64_t data = roundup(vb - (int64_t)(s / 8), wb);
    int64_t sz = meta_bytes(v, wb) + data;
    return sz < vb ? sz : vb;
}

void orc_compress_size(const void *data, int64_t n, int64_t v, int wb, const void *mask,
                       const void *bitval, const int64_t *idx, int64_t nout, int64_t *sizes) {
    (void)n;
#pragma omp parallel for schedule(static) num_threads(NT)
    for (int64_t i = 0; i < nout; ++i) {
        int64_t r = idx ? idx[i] : i;
        sizes[i] = row_size((const char *)data + r * v * wb, v, wb, mask, bitval);
    }
}

/* ---------------------------------------------------------------- bit packing */

/* Runs of set bits of `sel` (W bits), lowest first: position and length. */
typedef struct {
    int n;
    uint8_t pos[33], len[33];
} runs_t;

static void make_runs(uint64_t sel, int W, runs_t *r) {
    r->n = 0;
    int b = 0;
    while (b < W) {
        if ((sel >> b) & 1ull) {
            int s = b;
            while (b < W && ((sel >> b) & 1ull)) b++;
            r->pos[r->n] = (uint8_t)s;
            r->len[r->n] = (uint8_t)(b - s);
            r->n++;
        } else {
            b++;
        }
    }
}

/* bits of x at the selected positions, packed to the right in order */
static inline uint64_t pext_runs(uint64_t x, const runs_t *r) {
    uint64_t res = 0;
    int s = 0;
    for (int k = 0; k < r->n; ++k) {
        res |= ((x >> r->pos[k]) & wmask(r->len[k])) << s;
        s += r->len[k];
    }
    return res;
}

/* inverse: low bits of y scattered to the selected positions in order */
static inline uint64_t pdep_runs(uint64_t y, const runs_t *r) {
    uint64_t res = 0;
    int s = 0;
    for (int k = 0; k < r->n; ++k) {
        res |= ((y >> s) & wmask(r->len[k])) << r->pos[k];
        s += r->len[k];
    }
    return res;
}

/* Stream bit s lives in word (base + s/W) at bit W-1-(s%W): MSB-first
 * (include/compress/ibp_compress_dev.cuh:74-92). */
static inline void put_bits(void *row, int64_t base, int wb, int64_t *pos, uint64_t val, int nbits) {
    const int W = 8 * wb;
    while (nbits > 0) {
        int off = (int)(*pos % W), room = W - off;
        int take = nbits < room ? nbits : room;
        uint64_t chunk = (val >> (nbits - take)) & wmask(take);
        int64_t w = base + *pos / W;
        stw(row, w, wb, ldw(row, w, wb) | (chunk << (room - take)));
        *pos += take;
        nbits -= take;
    }
}

static inline uint64_t get_bits(const void *row, int64_t base, int wb, int64_t *pos, int nbits) {
    const int W = 8 * wb;
    uint64_t val = 0;
    while (nbits > 0) {
        int off = (int)(*pos % W), room = W - off;
        int take = nbits < room ? nbits : room;
        uint64_t word = ldw(row, base + *pos / W, wb);
        uint64_t chunk = (word >> (room - take)) & wmask(take);
        val = (take >= 64) ? chunk : ((val << take) | chunk);
        *pos += take;
        nbits -= take;
    }
    return val;
}

/* include/compress/ibp_compress_dev.cuh:7-97 (compress_and_write): bitmap of
 * compressible words, then per word either its non-invariant bits or all W bits. */
static void pack_row(const void *src, int64_t v, int wb, const void *mask, const void *bitval,
                     const runs_t *runs, void *dst) {
    const int W = 8 * wb;
    const int64_t mw = meta_bytes(v, wb) / wb;
    int64_t pos = 0;
    for (int64_t j = 0; j < v; ++j) {
        uint64_t x = ldw(src, j, wb), m = ldw(mask, j, wb);
        if ((x & m) == ldw(bitval, j, wb)) {
            stw(dst, j / W, wb, ldw(dst, j / W, wb) | (1ull << (j % W)));
            put_bits(dst, mw, wb, &pos, pext_runs(x, &runs[j]), W - popc(m));
        } else {
            put_bits(dst, mw, wb, &pos, x, W);
        }
    }
}

static runs_t *make_all_runs(int64_t v, int wb, const void *mask) {
    const int W = 8 * wb;
    runs_t *runs = (runs_t *)malloc(sizeof(runs_t) * (size_t)(v > 0 ? v : 1));
    for (int64_t j = 0; j < v; ++j) make_runs(~ldw(mask, j, wb) & wmask(W), W, &runs[j]);
    return runs;
}

/* include/compress/ibp_compress_kernel.cuh:9-56 (compress_inplace_kernel) */
void orc_compress(const void *src, int64_t n, int64_t v, int wb, const void *mask,
                  const void *bitval, const int64_t *idx, int64_t nout, void *out,
                  int32_t *bitmask) {
    (void)n;
    runs_t *runs = make_all_runs(v, wb, mask);
    const int64_t vb = v * wb;
    memset(bitmask, 0, sizeof(int32_t) * (size_t)((nout + 31) / 32));
#pragma omp parallel for schedule(static) num_threads(NT)
    for (int64_t i = 0; i < nout; ++i) {
        int64_t r = idx ? idx[i] : i;
        const char *s = (const char *)src + r * vb;
        char *d = (char *)out + i * vb;
        if (row_size(s, v, wb, mask, bitval) < vb) {
            memset(d, 0, (size_t)vb);
            pack_row(s, v, wb, mask, bitval, runs, d);
#pragma omp atomic
            bitmask[i / 32] |= (int32_t)(1u << (i % 32));
        } else {
            memcpy(d, s, (size_t)vb);
        }
    }
    free(runs);
}

/* include/compress/ibp_compress_kernel.cuh:58-94 (compress_condensed_kernel) */
void orc_compress_condensed(const void *src, int64_t n, int64_t v, int wb, const void *mask,
                            const void *bitval, const int64_t *idx, int64_t nout,
                            const int64_t *offsets, void *out) {
    (void)n;
    runs_t *runs = make_all_runs(v, wb, mask);
    const int64_t vb = v * wb;
#pragma omp parallel for schedule(static) num_threads(NT)
    for (int64_t i = 0; i < nout; ++i) {
        int64_t r = idx ? idx[i] : i;
        int64_t start = i ? offsets[i - 1] : 0;
        int64_t size = offsets[i] - start;
        const char *s = (const char *)src + r * vb;
        char *d = (char *)out + start;
        if (size != vb)
            pack_row(s, v, wb, mask, bitval, runs, d);
        else
            memcpy(d, s, (size_t)vb);
    }
    free(runs);
}

/* include/decompress/ibp_decompress_kernel.cuh:17-105 + ibp_decompress_dev.cuh:279-336:
 * compressed word = bitval | its stream bits placed at the mask-0 positions (MSB first);
 * other words take W stream bits; rows whose bitmask bit is clear are copied. */
void orc_decompress(const void *comp, int64_t n, int64_t v, int wb, const void *mask,
                    const void *bitval, const int32_t *bitmask, const int64_t *idx, int64_t nout,
                    void *out) {
    (void)n;
    const int W = 8 * wb;
    const int64_t vb = v * wb;
    const int64_t mw = meta_bytes(v, wb) / wb;
    runs_t *runs = make_all_runs(v, wb, mask);
#pragma omp parallel for schedule(static) num_threads(NT)
    for (int64_t k = 0; k < nout; ++k) {
        int64_t r = idx ? idx[k] : k;
        const char *s = (const char *)comp + r * vb;
        char *d = (char *)out + k * vb;
        if (!((uint32_t)bitmask[r / 32] & (1u << (r % 32)))) {
            memcpy(d, s, (size_t)vb);
            continue;
        }
        int64_t pos = 0;
        for (int64_t j = 0; j < v; ++j) {
            uint64_t x;
            if ((ldw(s, j / W, wb) >> (j % W)) & 1ull) {
                uint64_t m = ldw(mask, j, wb);
                uint64_t y = get_bits(s, mw, wb, &pos, W - popc(m));
                x = ldw(bitval, j, wb) | pdep_runs(y, &runs[j]);
            } else {
                x = get_bits(s, mw, wb, &pos, W);
            }
            stw(d, j, wb, x);
        }
    }
    free(runs);
}

/* ---------------------------------------------------------------- k-means */

/* include/preproc/ibp_preproc_kmeans.cuh:105-150 (cluster_vecs).  The reference lets the
 * last atomicExch of a tied minimum win; later rounds of its centroid loop overwrite earlier
 * ones, so the highest tied id is always a possible reference outcome. */
void orc_kmeans_assign(const void *data, int64_t n, int64_t v, int wb, const void *centroids,
                       int c, int32_t *clusters) {
#pragma omp parallel for schedule(static) num_threads(NT)
    for (int64_t i = 0; i < n; ++i) {
        int best = 0;
        int64_t bestd = -1;
        for (int j = 0; j < c; ++j) {
            int64_t d = 0;
            for (int64_t k = 0; k < v; ++k)
                d += popc(ldw(data, i * v + k, wb) ^ ldw(centroids, (int64_t)j * v + k, wb));
            if (bestd < 0 || d <= bestd) {
                bestd = d;
                best = j;
            }
        }
        clusters[i] = best;
    }
}

/* include/preproc/ibp_preproc_kmeans.cuh:195-236 (compute_new_centroids, construct_bitmasks):
 * bit b of centroid word id is set when more than count/2 (integer division) members have it;
 * the reference's accumulator is not reset between the words lane, lane+32, ... of a lane,
 * so word id is the OR over those words up to id. */
void orc_kmeans_update(const void *data, int64_t n, int64_t v, int wb, const int32_t *clusters,
                       int c, void *centroids) {
    const int W = 8 * wb;
    int64_t *cnt = (int64_t *)calloc((size_t)c, sizeof(int64_t));
    int64_t *bits = (int64_t *)calloc((size_t)c * v * W, sizeof(int64_t));
    for (int64_t i = 0; i < n; ++i) {
        int cl = clusters[i];
        cnt[cl]++;
        for (int64_t k = 0; k < v; ++k) {
            uint64_t x = ldw(data, i * v + k, wb);
            int64_t *bk = bits + ((int64_t)cl * v + k) * W;
            while (x) {
                bk[__builtin_ctzll(x)]++;
                x &= x - 1;
            }
        }
    }
    for (int cl = 0; cl < c; ++cl) {
        int32_t half = (int32_t)cnt[cl] / 2;
        for (int lane = 0; lane < 32; ++lane) {
            uint64_t acc = 0;
            for (int64_t id = lane; id < v; id += 32) {
                for (int b = 0; b < W; ++b)
                    if (bits[((int64_t)cl * v + id) * W + b] > half) acc |= 1ull << b;
                stw(centroids, (int64_t)cl * v + id, wb, acc);
            }
        }
    }
    free(cnt);
    free(bits);
}

/* include/preproc/ibp_preproc_kmeans.cuh:238-297 (create_mask_many): per-cluster counts are
 * accumulated in float32 (saturating at 2^24); `>= thr*count` in float32, `<= (1-thr)*count`
 * in float64; an empty cluster gets all-ones mask and bitval. */
void orc_kmeans_masks(const void *data, int64_t n, int64_t v, int wb, const int32_t *clusters,
                      int c, float thr, void *masks, void *bitvals) {
    const int W = 8 * wb;
    int64_t *cnt = (int64_t *)calloc((size_t)c, sizeof(int64_t));
    int64_t *bits = (int64_t *)calloc((size_t)c * v * W, sizeof(int64_t));
    for (int64_t i = 0; i < n; ++i) {
        int cl = clusters[i];
        cnt[cl]++;
        for (int64_t k = 0; k < v; ++k) {
            uint64_t x = ldw(data, i * v + k, wb);
            int64_t *bk = bits + ((int64_t)cl * v + k) * W;
            while (x) {
                bk[__builtin_ctzll(x)]++;
                x &= x - 1;
            }
        }
    }
    for (int cl = 0; cl < c; ++cl) {
        int32_t count = (int32_t)cnt[cl];
        volatile float lim1 = thr * (float)count;
        volatile double lim0 = (1.0 - (double)thr) * (double)count;
        for (int64_t id = 0; id < v; ++id) {
            uint64_t m = 0, val = 0;
            for (int b = 0; b < W; ++b) {
                int64_t bs = bits[((int64_t)cl * v + id) * W + b];
                float bsf = bs > 16777216 ? 16777216.0f : (float)bs;
                if (bsf >= lim1) {
                    val |= 1ull << b;
                    m |= 1ull << b;
                } else if ((double)bsf <= lim0) {
                    m |= 1ull << b;
                }
            }
            stw(masks, (int64_t)cl * v + id, wb, m);
            stw(bitvals, (int64_t)cl * v + id, wb, val);
        }
    }
    free(cnt);
    free(bits);
}

/* include/preproc/ibp_preproc_host.cuh:118-284 (preproc_kmeans): seed, 10 rounds of
 * assign + update, then masks; the float32 sweep 0.7..1.0 rewrites every mask each step
 * and keeps none, so the result is the mask of its last step, thr = 1.0f. */
void orc_preprocess_kmeans(const void *data, int64_t n, int64_t v, int wb, int c,
                           const int64_t *init, void *masks, void *bitvals, int32_t *clusters) {
    void *cent = calloc((size_t)c * v, (size_t)wb);
    int64_t seeded = c < n ? c : n;
    if (seeded > 0) memcpy(cent, data, (size_t)(v * wb));
    for (int64_t i = 1; i < seeded; ++i)
        memcpy((char *)cent + i * v * wb, (const char *)data + init[i] * v * wb, (size_t)(v * wb));
    memset(clusters, 0, sizeof(int32_t) * (size_t)n);
    for (int it = 0; it < 10; ++it) {
        orc_kmeans_assign(data, n, v, wb, cent, c, clusters);
        orc_kmeans_update(data, n, v, wb, clusters, c, cent);
    }
    float last = 0.7f;
    for (float t = 0.7f; t <= 1.0f; t = (float)((double)t + 0.05)) last = t;
    orc_kmeans_masks(data, n, v, wb, clusters, c, last, masks, bitvals);
    free(cent);
}
