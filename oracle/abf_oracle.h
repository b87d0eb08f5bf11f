/*
 * abf_oracle.h -- CPU oracle for the Boolean-filtering hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker: tests/, the
 * smoke() entry point and bench.py's CPU-baseline leg load it; the product
 * library (libadabool.so) never links it and no product path calls it.
 *
 * Two kinds of restatement of the reference (yxr620/AdaBool):
 *   1. the match-set semantics: a scalar k-way merge over sorted unique
 *      lists, equal to ComputeGroundTruth (test/adsfilter_q_all.cu:196-208,
 *      test/adsfilter_batch.cu:173-190) and the bitmap -> ids loop
 *      CollectIdsFromBitmap (test/adsfilter_batch.cu:82-97);
 *   2. the reference's own index and kernels: its mixed-container builder
 *      (src/AdaBool/inverted_list.h:90-148,348-470) and what its list-union
 *      and bitmap-probe kernels compute from it
 *      (src/AdaBool/inverted_list.cu.h:61-94,
 *       src/AdaBool/load_balance_transformer.cu.h:16-91,
 *       src/AdaBool/key_transformer.cu.h:11-331).
 * Both are pinned against the reference itself: the builder against the
 * reference's BuildFrom compiled from its sources (oracle/ref_build.cpp),
 * the match sets against the reference's ComputeGroundTruth
 * (oracle/ref_cpu.cu), through the fixtures in tests/golden/.
 */
#ifndef ABF_ORACLE_H_
#define ABF_ORACLE_H_
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Sorted unique union of the lists of terms q[0..nq) (terms >= n_terms and
 * repeated terms are ignored); lists are CSR (offsets[n_terms+1], ads) and
 * each list sorted ascending and unique. Writes at most cap ids to out and
 * returns the full count. Heap-based k-way merge. */
uint64_t orc_kway_union(const uint64_t* offsets, const uint32_t* ads, uint32_t n_terms, const uint32_t* q,
                        uint32_t nq, uint32_t* out, uint64_t cap);

/* Same set from unsorted COO pairs by a linear scan, the reference's
 * ComputeGroundTruth semantics; out sorted ascending. */
uint64_t orc_scan_union(const uint32_t* terms, const uint32_t* ads, uint64_t nnz, const uint32_t* q, uint32_t nq,
                        uint32_t* out, uint64_t cap);

/* Sets bit id of a uint32 bitmap (word id>>5, bit id&31) for every id. */
void orc_ids_to_bitmap(const uint32_t* ids, uint64_t n, uint32_t* words, uint64_t n_words);

/* Ascending ids of set bits below ncols of a byte bitmap
 * (CollectIdsFromBitmap, test/adsfilter_batch.cu:82-97). Returns count. */
uint64_t orc_collect_ids(const uint8_t* bitmap, uint64_t bitmap_bytes, uint64_t ncols, uint32_t* out, uint64_t cap);

/* CPU baseline: k-way merge of every query of a batch on n_threads host
 * threads; counts[q] gets each query's match count. Returns the total. */
uint64_t orc_cpu_batch(const uint64_t* offsets, const uint32_t* ads, uint32_t n_terms, const uint64_t* q_off,
                       const uint32_t* q_terms, uint32_t n_queries, int n_threads, uint64_t* counts);
/* The same, also writing two checksums of each query's ascending id list
 * ids[0..n): sums[2q] = sum of ids[i], sums[2q+1] = sum of ids[i] * i, both
 * mod 2^64 (the second depends on the order). */
uint64_t orc_cpu_batch_sums(const uint64_t* offsets, const uint32_t* ads, uint32_t n_terms, const uint64_t* q_off,
                            const uint32_t* q_terms, uint32_t n_queries, int n_threads, uint64_t* counts,
                            uint64_t* sums);

/* ---------------- the reference's mixed-container index ---------------- */
enum { ORC_ARRAY1 = 0, ORC_ARRAY4, ORC_ARRAY8, ORC_ARRAY16, ORC_ARRAY32, ORC_BITSET, ORC_NTYPES };
enum { ORC_F_KEY_SEG = 0, ORC_F_HEADERS, ORC_F_KEYS, ORC_F_ARRAYS, ORC_F_POS_SEG, ORC_F_BLK_SEG, ORC_F_KEY_BUF };

typedef struct orc_mixed orc_mixed;

/* From COO pairs in any order, duplicates kept (as the reference does). */
orc_mixed* orc_mixed_build_coo(const uint32_t* terms, const uint32_t* ads, uint64_t nnz, int block_step);
/* From CSR with every list sorted ascending (duplicates allowed). */
orc_mixed* orc_mixed_build_csr(const uint64_t* offsets, const uint32_t* ads, uint32_t n_terms, int block_step);
void orc_mixed_free(orc_mixed* m);
/* Pointer and element count of one array (element size: 1 byte for
 * ARRAYS and KEY_BUF, 4 bytes otherwise). */
int orc_mixed_array(const orc_mixed* m, int type, int field, const void** ptr, uint64_t* len);

/* What the reference's list-union kernels OR into res (n_words words) for
 * the given keys. */
void orc_mixed_union(const orc_mixed* m, const uint32_t* keys, uint64_t n_keys, uint32_t* res, uint64_t n_words);
/* What the reference's bitmap-probe kernels OR into res for a byte bitmap
 * of query terms (bit t of byte t/8), decoding keys through the per-block
 * key metadata. */
void orc_mixed_probe(const orc_mixed* m, const uint8_t* qbm, uint64_t qbm_bytes, uint32_t* res, uint64_t n_words);

#ifdef __cplusplus
}
#endif
#endif
