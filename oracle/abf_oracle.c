/*
 * abf_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; see abf_oracle.h).
 *
 * Plain C99 + pthreads, scalar code, no dependence on libadabool.
 */
#include "abf_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* k-way merge (binary min-heap of list cursors)                        */
/* ------------------------------------------------------------------ */
typedef struct {
    const uint32_t* p;
    const uint32_t* e;
} cursor;

static void sift_down(cursor* h, uint32_t n, uint32_t i) {
    for (;;) {
        uint32_t l = 2 * i + 1, r = l + 1, m = i;
        if (l < n && *h[l].p < *h[m].p) m = l;
        if (r < n && *h[r].p < *h[m].p) m = r;
        if (m == i) return;
        cursor t = h[i];
        h[i] = h[m];
        h[m] = t;
        i = m;
    }
}

static int cmp_u32(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x < y ? -1 : x > y;
}

/* ComputeGroundTruth (test/adsfilter_q_all.cu:196-208) takes the set of
 * ads of every pair whose term is in the query set; over per-term sorted
 * unique lists that is the merge of the query's distinct lists. */
uint64_t orc_kway_union(const uint64_t* offsets, const uint32_t* ads, uint32_t n_terms, const uint32_t* q,
                        uint32_t nq, uint32_t* out, uint64_t cap) {
    uint32_t* tq = (uint32_t*)malloc(sizeof(uint32_t) * (nq ? nq : 1));
    uint32_t k = 0;
    for (uint32_t i = 0; i < nq; ++i)
        if (q[i] < n_terms) tq[k++] = q[i];
    qsort(tq, k, sizeof(uint32_t), cmp_u32);
    cursor* h = (cursor*)malloc(sizeof(cursor) * (k ? k : 1));
    uint32_t n = 0;
    for (uint32_t i = 0; i < k; ++i) {
        if (i && tq[i] == tq[i - 1]) continue; /* repeated query term */
        uint64_t b = offsets[tq[i]], e = offsets[tq[i] + 1];
        if (b < e) {
            h[n].p = ads + b;
            h[n].e = ads + e;
            ++n;
        }
    }
    for (uint32_t i = n / 2; i-- > 0;) sift_down(h, n, i);
    uint64_t cnt = 0;
    int have = 0;
    uint32_t last = 0;
    while (n) {
        uint32_t v = *h[0].p;
        if (!have || v != last) {
            if (cnt < cap) out[cnt] = v;
            ++cnt;
            last = v;
            have = 1;
        }
        if (++h[0].p == h[0].e) h[0] = h[--n];
        if (n) sift_down(h, n, 0);
    }
    free(h);
    free(tq);
    return cnt;
}

uint64_t orc_scan_union(const uint32_t* terms, const uint32_t* ads, uint64_t nnz, const uint32_t* q, uint32_t nq,
                        uint32_t* out, uint64_t cap) {
    uint32_t* tq = (uint32_t*)malloc(sizeof(uint32_t) * (nq ? nq : 1));
    memcpy(tq, q, sizeof(uint32_t) * nq);
    qsort(tq, nq, sizeof(uint32_t), cmp_u32);
    uint64_t m = 0;
    uint32_t* tmp = (uint32_t*)malloc(sizeof(uint32_t) * (nnz ? nnz : 1));
    for (uint64_t i = 0; i < nnz; ++i)
        if (bsearch(&terms[i], tq, nq, sizeof(uint32_t), cmp_u32)) tmp[m++] = ads[i];
    qsort(tmp, m, sizeof(uint32_t), cmp_u32);
    uint64_t cnt = 0;
    for (uint64_t i = 0; i < m; ++i) {
        if (i && tmp[i] == tmp[i - 1]) continue;
        if (cnt < cap) out[cnt] = tmp[i];
        ++cnt;
    }
    free(tmp);
    free(tq);
    return cnt;
}

void orc_ids_to_bitmap(const uint32_t* ids, uint64_t n, uint32_t* words, uint64_t n_words) {
    for (uint64_t i = 0; i < n; ++i)
        if ((ids[i] >> 5) < n_words) words[ids[i] >> 5] |= 1u << (ids[i] & 31u);
}

uint64_t orc_collect_ids(const uint8_t* bitmap, uint64_t bitmap_bytes, uint64_t ncols, uint32_t* out, uint64_t cap) {
    uint64_t total_bits = bitmap_bytes * 8 < ncols ? bitmap_bytes * 8 : ncols;
    uint64_t cnt = 0;
    for (uint64_t byte = 0; byte < (total_bits + 7) / 8; ++byte) {
        uint8_t v = bitmap[byte];
        while (v) {
            unsigned lsb = (unsigned)__builtin_ctz((unsigned)v);
            uint64_t id = byte * 8 + lsb;
            if (id < ncols) {
                if (cnt < cap) out[cnt] = (uint32_t)id;
                ++cnt;
            }
            v &= (uint8_t)(v - 1);
        }
    }
    return cnt;
}

/* ------------------------------------------------------------------ */
/* CPU baseline: queries spread over host threads                       */
/* ------------------------------------------------------------------ */
typedef struct {
    const uint64_t* offsets;
    const uint32_t* ads;
    uint32_t n_terms;
    const uint64_t* q_off;
    const uint32_t* q_terms;
    uint32_t n_queries;
    uint64_t* counts;
    uint64_t* sums; /* optional: 2 per query (see orc_cpu_batch_sums) */
    uint64_t next; /* shared query cursor */
    pthread_mutex_t mu;
    uint64_t buf_cap;
} batch_job;

static void* batch_worker(void* arg) {
    batch_job* j = (batch_job*)arg;
    uint32_t* buf = (uint32_t*)malloc(sizeof(uint32_t) * (j->buf_cap ? j->buf_cap : 1));
    for (;;) {
        pthread_mutex_lock(&j->mu);
        uint64_t q = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (q >= j->n_queries) break;
        uint64_t b = j->q_off[q], e = j->q_off[q + 1];
        uint64_t n = orc_kway_union(j->offsets, j->ads, j->n_terms, j->q_terms + b, (uint32_t)(e - b), buf,
                                    j->buf_cap);
        j->counts[q] = n;
        if (j->sums) {
            uint64_t s1 = 0, s2 = 0;
            for (uint64_t i = 0; i < n && i < j->buf_cap; ++i) {
                s1 += buf[i];
                s2 += (uint64_t)buf[i] * i;
            }
            j->sums[2 * q] = s1;
            j->sums[2 * q + 1] = s2;
        }
    }
    free(buf);
    return NULL;
}

uint64_t orc_cpu_batch(const uint64_t* offsets, const uint32_t* ads, uint32_t n_terms, const uint64_t* q_off,
                       const uint32_t* q_terms, uint32_t n_queries, int n_threads, uint64_t* counts) {
    return orc_cpu_batch_sums(offsets, ads, n_terms, q_off, q_terms, n_queries, n_threads, counts, NULL);
}

uint64_t orc_cpu_batch_sums(const uint64_t* offsets, const uint32_t* ads, uint32_t n_terms, const uint64_t* q_off,
                            const uint32_t* q_terms, uint32_t n_queries, int n_threads, uint64_t* counts,
                            uint64_t* sums) {
    batch_job j;
    j.offsets = offsets;
    j.ads = ads;
    j.n_terms = n_terms;
    j.q_off = q_off;
    j.q_terms = q_terms;
    j.n_queries = n_queries;
    j.counts = counts;
    j.sums = sums;
    j.next = 0;
    j.buf_cap = 0;
    /* the match set is written out (sorted ids), bounded by the sum of the
     * query's list lengths */
    for (uint32_t q = 0; q < n_queries; ++q) {
        uint64_t s = 0;
        for (uint64_t i = q_off[q]; i < q_off[q + 1]; ++i)
            if (q_terms[i] < n_terms) s += offsets[q_terms[i] + 1] - offsets[q_terms[i]];
        if (s > j.buf_cap) j.buf_cap = s;
    }
    pthread_mutex_init(&j.mu, NULL);
    if (n_threads < 1) n_threads = 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)n_threads);
    for (int i = 0; i < n_threads; ++i) pthread_create(&th[i], NULL, batch_worker, &j);
    for (int i = 0; i < n_threads; ++i) pthread_join(th[i], NULL);
    free(th);
    pthread_mutex_destroy(&j.mu);
    uint64_t tot = 0;
    for (uint32_t q = 0; q < n_queries; ++q) tot += counts[q];
    return tot;
}

/* ------------------------------------------------------------------ */
/* restatement of the reference's mixed-container index                 */
/* ------------------------------------------------------------------ */
/* Growable arrays */
typedef struct {
    uint8_t* p;
    uint64_t n, cap;
} vec_u8;
typedef struct {
    uint32_t* p;
    uint64_t n, cap;
} vec_u32;

static void v8_push(vec_u8* v, uint8_t x) {
    if (v->n == v->cap) {
        v->cap = v->cap ? v->cap * 2 : 64;
        v->p = (uint8_t*)realloc(v->p, v->cap);
    }
    v->p[v->n++] = x;
}
static void v32_push(vec_u32* v, uint32_t x) {
    if (v->n == v->cap) {
        v->cap = v->cap ? v->cap * 2 : 64;
        v->p = (uint32_t*)realloc(v->p, v->cap * 4);
    }
    v->p[v->n++] = x;
}

struct orc_mixed {
    int block_step;
    vec_u32 key_seg[ORC_NTYPES], headers[ORC_NTYPES], keys[ORC_NTYPES];
    vec_u8 arrays[ORC_NTYPES];
    vec_u32 pos_seg[ORC_NTYPES], blk_seg[ORC_NTYPES];
    vec_u8 key_buf[ORC_NTYPES];
};

/* payload bytes per record: ARRAY1 none, ARRAYn n, BITSET 32
 * (src/AdaBool/inverted_list.h:425-458) */
static const int kArrayLen[ORC_NTYPES] = {0, 4, 8, 16, 32, 32};

static int type_of(uint64_t bucket_size) {
    if (bucket_size <= 1) return ORC_ARRAY1;
    if (bucket_size <= 5) return ORC_ARRAY4;
    if (bucket_size <= 9) return ORC_ARRAY8;
    if (bucket_size <= 17) return ORC_ARRAY16;
    if (bucket_size <= 33) return ORC_ARRAY32;
    return ORC_BITSET;
}

/* GroupKeys for one term whose ads are sorted ascending: buckets by the
 * high 24 bits, each bucket's low bytes (sorted, duplicates kept) go to the
 * container its size selects (src/AdaBool/inverted_list.h:402-468). */
static void add_term(orc_mixed* m, uint32_t key, const uint32_t* a, uint64_t n) {
    uint32_t cnt[ORC_NTYPES] = {0, 0, 0, 0, 0, 0};
    uint64_t i = 0;
    while (i < n) {
        uint32_t hi = a[i] & 0xffffff00u;
        uint64_t j = i;
        while (j < n && (a[j] & 0xffffff00u) == hi) ++j;
        uint64_t size = j - i;
        int t = type_of(size);
        ++cnt[t];
        v32_push(&m->keys[t], key);
        if (t == ORC_BITSET) {
            uint8_t bits[32];
            memset(bits, 0, sizeof(bits));
            for (uint64_t k = i; k < j; ++k) {
                uint8_t b = (uint8_t)(a[k] & 0xffu);
                bits[b / 8] |= (uint8_t)(1u << (b % 8));
            }
            v32_push(&m->headers[t], hi);
            for (int k = 0; k < 32; ++k) v8_push(&m->arrays[t], bits[k]);
        } else {
            v32_push(&m->headers[t], hi | (a[i] & 0xffu));
            for (int k = 0; k < kArrayLen[t]; ++k)
                v8_push(&m->arrays[t], (uint64_t)(k + 1) < size ? (uint8_t)(a[i + 1 + k] & 0xffu) : 0);
        }
        i = j;
    }
    for (int t = 0; t < ORC_NTYPES; ++t) {
        vec_u32* s = &m->key_seg[t];
        while (s->n <= key) v32_push(s, s->p[s->n - 1]);
        v32_push(s, s->p[s->n - 1] + cnt[t]);
    }
}

/* ComputeKeyBlockMeta (src/AdaBool/inverted_list.h:90-148) */
static void block_meta(orc_mixed* m, int t) {
    const uint32_t* keys = m->keys[t].p;
    uint64_t len = m->keys[t].n;
    int step = m->block_step;
    if (len == 0) return;
    vec_u32* bs = &m->blk_seg[t];
    vec_u32* ps = &m->pos_seg[t];
    vec_u8* kb = &m->key_buf[t];
    for (uint64_t i = 0; i < len; i += (uint64_t)step) v32_push(bs, keys[i]);
    v32_push(bs, keys[len - 1]);
    v32_push(ps, 0);
    for (uint64_t i = 0; i + 1 < bs->n; ++i) {
        uint32_t span = bs->p[i + 1] - bs->p[i];
        uint64_t num = len - i * (uint64_t)step < (uint64_t)step ? len - i * (uint64_t)step : (uint64_t)step;
        int kbytes = span < 256u ? 1 : (span < 65536u ? 2 : 4);
        v32_push(ps, ps->p[ps->n - 1] + (uint32_t)(num * (uint64_t)kbytes));
        const uint32_t* ks = keys + i * (uint64_t)step;
        for (uint64_t k = 0; k < num; ++k) {
            uint32_t off = ks[k] - bs->p[i];
            for (int b = 0; b < kbytes; ++b) v8_push(kb, (uint8_t)(off >> (8 * b)));
        }
        for (uint64_t k = num; k < (uint64_t)step; ++k)
            for (int b = 0; b < kbytes; ++b) v8_push(kb, 0);
    }
}

static orc_mixed* mixed_new(int block_step) {
    orc_mixed* m = (orc_mixed*)calloc(1, sizeof(orc_mixed));
    m->block_step = block_step > 0 ? block_step : 256;
    for (int t = 0; t < ORC_NTYPES; ++t) v32_push(&m->key_seg[t], 0);
    return m;
}

static void mixed_finish(orc_mixed* m) {
    for (int t = 0; t < ORC_NTYPES; ++t) block_meta(m, t);
}

orc_mixed* orc_mixed_build_csr(const uint64_t* offsets, const uint32_t* ads, uint32_t n_terms, int block_step) {
    orc_mixed* m = mixed_new(block_step);
    for (uint32_t k = 0; k < n_terms; ++k)
        if (offsets[k + 1] > offsets[k]) add_term(m, k, ads + offsets[k], offsets[k + 1] - offsets[k]);
    mixed_finish(m);
    return m;
}

static int cmp_u64(const void* a, const void* b) {
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : x > y;
}

orc_mixed* orc_mixed_build_coo(const uint32_t* terms, const uint32_t* ads, uint64_t nnz, int block_step) {
    uint64_t* kv = (uint64_t*)malloc(sizeof(uint64_t) * (nnz ? nnz : 1));
    for (uint64_t i = 0; i < nnz; ++i) kv[i] = ((uint64_t)terms[i] << 32) | ads[i];
    qsort(kv, nnz, sizeof(uint64_t), cmp_u64);
    uint32_t* a = (uint32_t*)malloc(sizeof(uint32_t) * (nnz ? nnz : 1));
    for (uint64_t i = 0; i < nnz; ++i) a[i] = (uint32_t)kv[i];
    orc_mixed* m = mixed_new(block_step);
    uint64_t i = 0;
    while (i < nnz) {
        uint32_t key = (uint32_t)(kv[i] >> 32);
        uint64_t j = i;
        while (j < nnz && (uint32_t)(kv[j] >> 32) == key) ++j;
        add_term(m, key, a + i, j - i);
        i = j;
    }
    mixed_finish(m);
    free(a);
    free(kv);
    return m;
}

void orc_mixed_free(orc_mixed* m) {
    if (!m) return;
    for (int t = 0; t < ORC_NTYPES; ++t) {
        free(m->key_seg[t].p);
        free(m->headers[t].p);
        free(m->keys[t].p);
        free(m->arrays[t].p);
        free(m->pos_seg[t].p);
        free(m->blk_seg[t].p);
        free(m->key_buf[t].p);
    }
    free(m);
}

int orc_mixed_array(const orc_mixed* m, int t, int f, const void** p, uint64_t* len) {
    if (!m || t < 0 || t >= ORC_NTYPES) return -1;
    switch (f) {
        case ORC_F_KEY_SEG: *p = m->key_seg[t].p; *len = m->key_seg[t].n; break;
        case ORC_F_HEADERS: *p = m->headers[t].p; *len = m->headers[t].n; break;
        case ORC_F_KEYS: *p = m->keys[t].p; *len = m->keys[t].n; break;
        case ORC_F_ARRAYS: *p = m->arrays[t].p; *len = t == ORC_ARRAY1 ? 0 : m->arrays[t].n; break;
        case ORC_F_POS_SEG: *p = m->pos_seg[t].p; *len = m->pos_seg[t].n; break;
        case ORC_F_BLK_SEG: *p = m->blk_seg[t].p; *len = m->blk_seg[t].n; break;
        case ORC_F_KEY_BUF: *p = m->key_buf[t].p; *len = m->key_buf[t].n; break;
        default: return -1;
    }
    return 0;
}

static void set_bit(uint32_t* res, uint64_t n_words, uint32_t v) {
    if ((v >> 5) < n_words) res[v >> 5] |= 1u << (v & 31u);
}

/* One record, as ProcessArrayFunctor (src/AdaBool/inverted_list.cu.h:61-94)
 * and the BITSET loop (src/AdaBool/load_balance_transformer.cu.h:62-91)
 * decode it: the header, then kMinNum payload bytes unconditionally, then
 * payload bytes up to the first zero. */
static void process_record(const orc_mixed* m, int t, uint64_t idx, uint32_t* res, uint64_t n_words) {
    static const int kMinNum[ORC_NTYPES] = {0, 1, 5, 9, 17, 0};
    uint32_t header = m->headers[t].p[idx];
    if (t == ORC_BITSET) {
        const uint8_t* bits = m->arrays[t].p + idx * 32;
        for (int j = 0; j < 8; ++j) {
            uint32_t w = (uint32_t)bits[4 * j] | ((uint32_t)bits[4 * j + 1] << 8) | ((uint32_t)bits[4 * j + 2] << 16) |
                         ((uint32_t)bits[4 * j + 3] << 24);
            uint32_t v = header | (uint32_t)(j * 32);
            if ((v >> 5) < n_words) res[v >> 5] |= w;
        }
        return;
    }
    set_bit(res, n_words, header);
    if (t == ORC_ARRAY1) return;
    uint32_t h = header & 0xffffff00u;
    const uint8_t* ls = m->arrays[t].p + idx * (uint64_t)kArrayLen[t];
    for (int i = 0; i < kMinNum[t]; ++i) set_bit(res, n_words, h | ls[i]);
    for (int i = kMinNum[t]; i < kArrayLen[t]; ++i) {
        if (!ls[i]) return;
        set_bit(res, n_words, h | ls[i]);
    }
}

/* ivf_list::Prepare(keys) takes keys below key_segments.len - 1
 * (src/AdaBool/inverted_list.h:491-505); the union kernels then decode
 * every record of those segments. */
void orc_mixed_union(const orc_mixed* m, const uint32_t* keys, uint64_t n_keys, uint32_t* res, uint64_t n_words) {
    for (uint64_t q = 0; q < n_keys; ++q) {
        uint32_t key = keys[q];
        for (int t = 0; t < ORC_NTYPES; ++t) {
            const vec_u32* s = &m->key_seg[t];
            if ((uint64_t)key + 1 >= s->n) continue;
            for (uint64_t idx = s->p[key]; idx < s->p[key + 1]; ++idx) process_record(m, t, idx, res, n_words);
        }
    }
}

/* The probe kernels decode each record's key from the per-block key
 * offsets (ForBPKeyIdxs, src/AdaBool/key_transformer.cu.h:11-44): block i
 * starts at key blk_seg[i], its offsets are 1, 2 or 4 bytes wide by the
 * span to the next block start, stored at pos_seg[i]. */
void orc_mixed_probe(const orc_mixed* m, const uint8_t* qbm, uint64_t qbm_bytes, uint32_t* res, uint64_t n_words) {
    for (int t = 0; t < ORC_NTYPES; ++t) {
        uint64_t len = m->keys[t].n;
        if (len == 0) continue;
        const vec_u32* bs = &m->blk_seg[t];
        for (uint64_t i = 0; i + 1 < bs->n; ++i) {
            uint32_t kbeg = bs->p[i], span = bs->p[i + 1] - bs->p[i];
            int kbytes = span < 256u ? 1 : (span < 65536u ? 2 : 4);
            const uint8_t* kb = m->key_buf[t].p + m->pos_seg[t].p[i];
            for (int k = 0; k < m->block_step; ++k) {
                uint64_t idx = i * (uint64_t)m->block_step + (uint64_t)k;
                if (idx >= len) break;
                uint32_t off = 0;
                for (int b = 0; b < kbytes; ++b) off |= (uint32_t)kb[k * kbytes + b] << (8 * b);
                uint32_t key = kbeg + off;
                if ((uint64_t)(key >> 3) >= qbm_bytes) continue;
                if (qbm[key >> 3] & (1u << (key & 7u))) process_record(m, t, idx, res, n_words);
            }
        }
    }
}
