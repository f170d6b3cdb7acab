/*
 * ibp_oracle.h -- CPU restatement of the reference Invariant Bit Packing codec.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product (tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg);
 * the product never links, loads or calls it.
 *
 * Words are W = 8*wb bits (wb in {1,2,4,8}), stored little-endian, rows of
 * v words at a fixed stride of v words.  All functions are deterministic and
 * thread-parallel (OpenMP) where the reference is data-parallel.
 *
 * Parity pinning: tests/golden/ holds vectors dumped by the reference
 * extension itself (built from its sources for sm_100a by oracle/build_ref.py
 * and run by tests/golden/make_golden.py); tests/test_oracle_golden.py
 * checks every function here against them.
 */
#ifndef IBP_ORACLE_H
#define IBP_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* include/preproc/ibp_preproc_kernels.cuh:7-31 -- counts[j*W+b] = #rows with bit b of word j set */
void orc_count_bits(const void *data, int64_t n, int64_t v, int wb, uint32_t *counts);

/* include/preproc/ibp_preproc_kernels.cuh:33-51 -- mask/bitval from counts at one threshold */
void orc_create_mask(const uint32_t *counts, int64_t n, int64_t v, int wb, float thr,
                     void *mask, void *bitval);

/* include/preproc/ibp_preproc_kernels.cuh:53-77 -- sum over rows of max(0, saved_bits - v) */
uint64_t orc_check_feats(const void *data, int64_t n, int64_t v, int wb,
                         const void *mask, const void *bitval);

/* include/preproc/ibp_preproc_host.cuh:23-115 -- census + threshold sweep (thr < 0: 0.7..1.0).
 * mask/bitval must be zeroed by the caller (src/preprocess.cu:46-47).
 * Returns the index of the selected sweep step, or -1 if none saved bits. */
int orc_preprocess(const void *data, int64_t n, int64_t v, int wb, float thr,
                   void *mask, void *bitval, uint64_t *saved_per_step, float *thr_per_step,
                   int *num_steps);

/* include/misc/ibp_misc_dev.cuh:19-46 -- compressed bytes of row (idx ? idx[i] : i) */
void orc_compress_size(const void *data, int64_t n, int64_t v, int wb, const void *mask,
                       const void *bitval, const int64_t *idx, int64_t nout, int64_t *sizes);

/* include/compress/ibp_compress_kernel.cuh:9-56 + ibp_compress_dev.cuh:7-97 -- out row i =
 * compressed(src row idx[i]) zero padded to v words, or raw; bitmask[(nout+31)/32] bit i = compressed.
 * out must not alias src. */
void orc_compress(const void *src, int64_t n, int64_t v, int wb, const void *mask,
                  const void *bitval, const int64_t *idx, int64_t nout, void *out,
                  int32_t *bitmask);

/* include/compress/ibp_compress_kernel.cuh:58-94 -- condensed layout at byte offsets
 * (inclusive scan of sizes); out holds sum(sizes) bytes, zeroed by the caller. */
void orc_compress_condensed(const void *src, int64_t n, int64_t v, int wb, const void *mask,
                            const void *bitval, const int64_t *idx, int64_t nout,
                            const int64_t *offsets, void *out);

/* include/decompress/ibp_decompress_dev.cuh:131-340 -- out row k = decompress(comp row idx[k]) */
void orc_decompress(const void *comp, int64_t n, int64_t v, int wb, const void *mask,
                    const void *bitval, const int32_t *bitmask, const int64_t *idx, int64_t nout,
                    void *out);

/* include/preproc/ibp_preproc_kmeans.cuh:105-150 -- Hamming-nearest centroid per row.
 * Ties go to the highest centroid id (always one of the reference's possible outcomes). */
void orc_kmeans_assign(const void *data, int64_t n, int64_t v, int wb, const void *centroids,
                       int c, int32_t *clusters);

/* include/preproc/ibp_preproc_kmeans.cuh:195-236 -- majority-bit centroids, with the
 * reference's per-lane OR accumulation across words lane, lane+32, ... */
void orc_kmeans_update(const void *data, int64_t n, int64_t v, int wb, const int32_t *clusters,
                       int c, void *centroids);

/* include/preproc/ibp_preproc_kmeans.cuh:238-297 -- per-cluster mask/bitval at threshold */
void orc_kmeans_masks(const void *data, int64_t n, int64_t v, int wb, const int32_t *clusters,
                      int c, float thr, void *masks, void *bitvals);

/* include/preproc/ibp_preproc_host.cuh:118-284 -- full k-means preprocess.  init[i] (i in
 * 1..min(c,n)-1) is the row that seeds centroid i; centroid 0 is row 0. */
void orc_preprocess_kmeans(const void *data, int64_t n, int64_t v, int wb, int c,
                           const int64_t *init, void *masks, void *bitvals, int32_t *clusters);

/* The reference's seeding: std::random_shuffle over 0..n-1 (process rand() state). */
void orc_random_shuffle_init(int64_t n, int c, int64_t *init, int reseed);

/* threads used by the parallel loops (0 = OpenMP default) */
void orc_set_threads(int t);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
