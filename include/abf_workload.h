/*
 * abf_workload.h -- seeded synthetic filter matrices and query sets.
 *
 * The reference measures on the AdsFilter dataset, which is not
 * distributed with it (dataset/README.md). These generators stand in for
 * it with the shapes the benchmark configurations name: Zipf list lengths,
 * uniform sorted unique ad ids per list, queries of distinct terms drawn
 * with probability proportional to list length. Everything is a pure
 * function of the seed, independent of the thread count.
 *
 * The reference ships generators of its own (src/AdaBool/data_utility.hpp:13-250)
 * that its tests never call; these are new and follow the stated
 * distributions instead.
 */
#ifndef ABF_WORKLOAD_H_
#define ABF_WORKLOAD_H_

#include <stdint.h>
#include "adabool.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct abf_gen_lists_params {
    uint32_t n_terms;
    uint32_t n_ads;
    uint64_t nnz_target;   /* expected total postings */
    double zipf_s;         /* list length of rank r ~ C * r^-s */
    uint32_t max_len;      /* lengths clipped to [1, max_len]; C rescaled after clipping */
    uint64_t seed;
    int n_threads;         /* <= 0: all cores */
} abf_gen_lists_params;

/* Target length of every term (n_terms entries). Ranks are mapped to term
 * ids by a seeded permutation. */
abf_status abf_gen_target_lengths(const abf_gen_lists_params* p, uint32_t* h_len_out);

/* Pass 1: CSR offsets (n_terms + 1) of the lists. Each list is a
 * Bernoulli(len/n_ads) draw over the ad range (at least one posting), so
 * realised lengths scatter around the targets. */
abf_status abf_gen_lists_offsets(const abf_gen_lists_params* p, uint64_t* h_offsets_out);

/* Pass 2: the ads (offsets[n_terms] entries), sorted and unique per list. */
abf_status abf_gen_lists_fill(const abf_gen_lists_params* p, const uint64_t* h_offsets,
                              uint32_t* h_ads_out);

enum {
    ABF_QCOUNT_UNIFORM = 0,   /* term count uniform in [lo, hi] */
    ABF_QCOUNT_LOGNORMAL = 1  /* round(median * exp(sigma * N(0,1))) clipped to [lo, hi] */
};

typedef struct abf_gen_queries_params {
    uint32_t n_queries;
    int count_kind;        /* ABF_QCOUNT_* */
    double median, sigma;  /* lognormal parameters */
    uint32_t lo, hi;       /* count bounds */
    uint64_t seed;
    int n_threads;
} abf_gen_queries_params;

/* Pass 1: offsets (n_queries + 1) of the query term lists. Counts are also
 * capped at the number of non-empty terms. */
abf_status abf_gen_queries_offsets(const abf_gen_queries_params* p, const uint32_t* h_list_len,
                                   uint32_t n_terms, uint64_t* h_offsets_out);

/* Pass 2: distinct terms per query, drawn with probability proportional to
 * h_list_len, in draw order. */
abf_status abf_gen_queries_fill(const abf_gen_queries_params* p, const uint32_t* h_list_len,
                                uint32_t n_terms, const uint64_t* h_offsets,
                                uint32_t* h_terms_out);

#ifdef __cplusplus
}
#endif
#endif /* ABF_WORKLOAD_H_ */
