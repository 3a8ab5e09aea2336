/*
 * mgv_oracle.c -- CPU oracle (test infrastructure; see mgv_oracle.h).
 *
 * Restates the reference's CPU loops in plain C:
 *   select predicate      src/operators/select3.cuh:10-23  (x <= bound, signed)
 *   stable select         src/main9.cu:48-52               (stable_select_cpu)
 *   select + SUM          src/main9.cu:56-61               (sum_select_cpu)
 *   murmur finaliser      src/operators/hashjoin.cu:4-11, src/main8.cu:75-82
 *   chained hash join     src/main8.cu:84-103              (sum_hashjoin_select_cpu)
 *   probe semantics       src/operators/hashjoin.cu:134-182 (all duplicates count)
 *   split / partition     src/operators/split.cu:49-118    (generalised to 2^bits ways)
 * and extends them with int64 SUM/COUNT, payloads, GROUP BY and the
 * select -> join -> group-by query, which the reference does not have.
 */
#include "mgv_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "../multigpu-vector_b200/csrc/mgv_gen.h"

/* ---------------------------------------------------------------------- */
/* generators                                                             */
/* ---------------------------------------------------------------------- */

void or_gen_uniform(int32_t *out, uint64_t n, uint64_t seed, uint32_t stream,
                    int64_t lo, uint64_t range) {
    for (uint64_t i = 0; i < n; ++i) out[i] = mgv_gen_uniform(seed, stream, i, lo, range);
}

void or_gen_perm(int32_t *out, uint64_t n, uint64_t seed) {
    for (uint64_t i = 0; i < n; ++i) out[i] = (int32_t)mgv_gen_perm(seed, n, i);
}

uint64_t or_gen_probe_keys(int32_t *out, uint64_t n, uint64_t seed, uint64_t build_seed,
                           uint64_t nbuild, uint32_t hit_num, int64_t miss_lo,
                           uint64_t miss_range) {
    uint64_t hits = 0;
    for (uint64_t i = 0; i < n; ++i) {
        int h = 0;
        out[i] = mgv_gen_probe_key(seed, build_seed, nbuild, hit_num, miss_lo, miss_range, i, &h);
        hits += (uint64_t)h;
    }
    return hits;
}

/* cdf[g] = floor(2^32 * H(g+1) / H(G)) with H the generalised harmonic
 * number of order s; the last entry is 2^32 so every 32-bit draw lands. */
void or_zipf_cdf(uint64_t *cdf, uint32_t G, double s) {
    double total = 0.0;
    for (uint32_t g = 1; g <= G; ++g) total += (s == 1.0) ? 1.0 / (double)g : 1.0 / __builtin_pow((double)g, s);
    double acc = 0.0;
    for (uint32_t g = 1; g <= G; ++g) {
        acc += (s == 1.0) ? 1.0 / (double)g : 1.0 / __builtin_pow((double)g, s);
        double v = acc / total * 4294967296.0;
        uint64_t c = (v >= 4294967296.0) ? 4294967296ull : (uint64_t)v;
        cdf[g - 1] = c;
    }
    cdf[G - 1] = 4294967296ull;
}

void or_gen_zipf(int32_t *out, uint64_t n, uint64_t seed, uint32_t stream,
                 const uint64_t *cdf, uint32_t G) {
    for (uint64_t i = 0; i < n; ++i) out[i] = mgv_gen_zipf(seed, stream, i, cdf, G);
}

/* ---------------------------------------------------------------------- */
/* hash + select                                                          */
/* ---------------------------------------------------------------------- */

/* MurmurHash3 32-bit finaliser, as hashMurmur in src/operators/hashjoin.cu:4-11. */
uint32_t or_hash_murmur(uint32_t x) {
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

/* Stable select of rows with a[i] <= bound (src/main9.cu:48-52). */
size_t or_select_rows(const int32_t *a, size_t n, int32_t bound, int32_t *out) {
    size_t k = 0;
    for (size_t i = 0; i < n; ++i)
        if (a[i] <= bound) out[k++] = a[i];
    return k;
}

/* COUNT and int64 SUM of v over rows with f <= bound.  The reference sums
 * the selected column itself into a wrapping int32 (src/main9.cu:56-61);
 * with v == NULL this sums f, and the low 32 bits equal the reference. */
void or_select_agg(const int32_t *f, const int32_t *v, size_t n, int32_t bound,
                   int64_t *count, int64_t *sum) {
    int64_t c = 0, s = 0;
    const int32_t *val = v ? v : f;
    for (size_t i = 0; i < n; ++i)
        if (f[i] <= bound) { ++c; s += val[i]; }
    *count = c;
    *sum = s;
}

typedef struct select_job {
    const int32_t *f, *v;
    uint64_t lo, hi;
    int32_t bound;
    int64_t count, sum;
} select_job;

static void *select_worker(void *arg) {
    select_job *j = (select_job *)arg;
    or_select_agg(j->f + j->lo, j->v ? j->v + j->lo : NULL, j->hi - j->lo, j->bound, &j->count, &j->sum);
    return NULL;
}

/* The same split over `threads` host threads. */
void or_select_agg_mt(const int32_t *f, const int32_t *v, size_t n, int32_t bound, int threads,
                      int64_t *count, int64_t *sum) {
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t tid[256];
    select_job jobs[256];
    for (int i = 0; i < threads; ++i) {
        jobs[i].f = f;
        jobs[i].v = v;
        jobs[i].bound = bound;
        jobs[i].lo = n * (uint64_t)i / (uint64_t)threads;
        jobs[i].hi = n * (uint64_t)(i + 1) / (uint64_t)threads;
        pthread_create(&tid[i], NULL, select_worker, &jobs[i]);
    }
    int64_t c = 0, s = 0;
    for (int i = 0; i < threads; ++i) {
        pthread_join(tid[i], NULL);
        c += jobs[i].count;
        s += jobs[i].sum;
    }
    *count = c;
    *sum = s;
}

/* ---------------------------------------------------------------------- */
/* chained hash join (src/main8.cu:84-103)                                */
/* ---------------------------------------------------------------------- */

/* Build: rows inserted in index order at the head of their bucket chain,
 * bucket = murmur(key) & (2^L - 1), L = ceil(log2(n)) (at least 1).  With
 * use_filter the build keeps only rows with key <= bound, as the reference's
 * CPU join does (src/main8.cu:87). */
int or_chain_build(or_chain_table *t, const int32_t *keys, const int32_t *pay,
                   uint64_t n, int use_filter, int32_t bound) {
    uint32_t L = mgv_bits_for(n ? n : 1);
    if (L < 1) L = 1;
    t->log_size = L;
    t->head = (int32_t *)malloc(sizeof(int32_t) << L);
    t->next = (int32_t *)malloc(sizeof(int32_t) * (n ? n : 1));
    if (!t->head || !t->next) return -1;
    memset(t->head, 0xff, sizeof(int32_t) << L);
    t->keys = keys;
    t->pay = pay;
    t->n = n;
    uint32_t mask = (1u << L) - 1u;
    for (uint64_t j = 0; j < n; ++j) {
        t->next[j] = -1;
        if (use_filter && !(keys[j] <= bound)) continue;
        uint32_t b = or_hash_murmur((uint32_t)keys[j]) & mask;
        t->next[j] = t->head[b];
        t->head[b] = (int32_t)j;
    }
    return 0;
}

void or_chain_free(or_chain_table *t) {
    free(t->head);
    free(t->next);
    t->head = t->next = NULL;
}

uint64_t or_chain_matches(const or_chain_table *t, int32_t key) {
    uint32_t mask = (1u << t->log_size) - 1u;
    uint64_t m = 0;
    for (int32_t c = t->head[or_hash_murmur((uint32_t)key) & mask]; c >= 0; c = t->next[c])
        m += (t->keys[c] == key);
    return m;
}

/* Probe: every build row with an equal key is a match (duplicates all
 * count, src/operators/hashjoin.cu:148-162).  SUM adds the build payload
 * and/or the probe payload of every match. */
void or_chain_probe_agg(const or_chain_table *t, const int32_t *pkeys,
                        const int32_t *ppay, uint64_t m, int add_build_pay,
                        int add_probe_pay, int64_t *count, int64_t *sum) {
    uint32_t mask = (1u << t->log_size) - 1u;
    int64_t c = 0, s = 0;
    for (uint64_t i = 0; i < m; ++i) {
        int32_t k = pkeys[i];
        for (int32_t cur = t->head[or_hash_murmur((uint32_t)k) & mask]; cur >= 0; cur = t->next[cur]) {
            if (t->keys[cur] == k) {
                ++c;
                if (add_build_pay && t->pay) s += t->pay[cur];
                if (add_probe_pay && ppay) s += ppay[i];
            }
        }
    }
    *count = c;
    *sum = s;
}

typedef struct probe_job {
    const or_chain_table *t;
    const int32_t *pkeys, *ppay;
    uint64_t lo, hi;
    int64_t count, sum;
} probe_job;

static void *probe_worker(void *arg) {
    probe_job *j = (probe_job *)arg;
    or_chain_probe_agg(j->t, j->pkeys + j->lo, j->ppay ? j->ppay + j->lo : NULL,
                       j->hi - j->lo, 1, 1, &j->count, &j->sum);
    return NULL;
}

/* The same probe split over `threads` host threads (read-only table). */
void or_chain_probe_agg_mt(const or_chain_table *t, const int32_t *pkeys,
                           const int32_t *ppay, uint64_t m, int threads,
                           int64_t *count, int64_t *sum) {
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t tid[256];
    probe_job jobs[256];
    for (int i = 0; i < threads; ++i) {
        jobs[i].t = t;
        jobs[i].pkeys = pkeys;
        jobs[i].ppay = ppay;
        jobs[i].lo = m * (uint64_t)i / (uint64_t)threads;
        jobs[i].hi = m * (uint64_t)(i + 1) / (uint64_t)threads;
        jobs[i].count = jobs[i].sum = 0;
        pthread_create(&tid[i], NULL, probe_worker, &jobs[i]);
    }
    int64_t c = 0, s = 0;
    for (int i = 0; i < threads; ++i) {
        pthread_join(tid[i], NULL);
        c += jobs[i].count;
        s += jobs[i].sum;
    }
    *count = c;
    *sum = s;
}

/* Emit (key, build payload, probe payload) for every match; returns the
 * number of matches (rows beyond cap are counted but not written). */
uint64_t or_chain_probe_emit(const or_chain_table *t, const int32_t *pkeys,
                             const int32_t *ppay, uint64_t m, int32_t *out,
                             uint64_t cap) {
    uint32_t mask = (1u << t->log_size) - 1u;
    uint64_t k = 0;
    for (uint64_t i = 0; i < m; ++i) {
        int32_t key = pkeys[i];
        for (int32_t cur = t->head[or_hash_murmur((uint32_t)key) & mask]; cur >= 0; cur = t->next[cur]) {
            if (t->keys[cur] == key) {
                if (k < cap) {
                    out[3 * k + 0] = key;
                    out[3 * k + 1] = t->pay ? t->pay[cur] : 0;
                    out[3 * k + 2] = ppay ? ppay[i] : 0;
                }
                ++k;
            }
        }
    }
    return k;
}

/* ---------------------------------------------------------------------- */
/* radix partition (src/operators/split.cu:49-118, 2 ways -> 2^bits ways)  */
/* ---------------------------------------------------------------------- */

/* Destination = (key >> shift) & (2^bits - 1).  Writes a stable
 * partition-major copy of keys (and payloads) and the histogram. */
void or_partition(const int32_t *keys, uint64_t n, uint32_t bits, uint32_t shift,
                  uint64_t *hist, int32_t *out_keys, const int32_t *pay,
                  int32_t *out_pay) {
    uint32_t P = 1u << bits, mask = P - 1u;
    uint64_t *off = (uint64_t *)calloc(P, sizeof(uint64_t));
    memset(hist, 0, sizeof(uint64_t) * P);
    for (uint64_t i = 0; i < n; ++i) hist[((uint32_t)keys[i] >> shift) & mask]++;
    uint64_t acc = 0;
    for (uint32_t p = 0; p < P; ++p) { off[p] = acc; acc += hist[p]; }
    if (out_keys) {
        for (uint64_t i = 0; i < n; ++i) {
            uint32_t p = ((uint32_t)keys[i] >> shift) & mask;
            uint64_t o = off[p]++;
            out_keys[o] = keys[i];
            if (out_pay && pay) out_pay[o] = pay[i];
        }
    }
    free(off);
}

/* ---------------------------------------------------------------------- */
/* group-by (no reference counterpart; the reference has a global SUM only, */
/* src/operators/aggregation.cu:5-66)                                      */
/* ---------------------------------------------------------------------- */

typedef struct gb_map {
    int32_t *key;
    int64_t *sum, *cnt;
    uint8_t *used;
    uint64_t cap, size;
} gb_map;

static int gb_init(gb_map *m, uint64_t cap) {
    m->cap = cap;
    m->size = 0;
    m->key = (int32_t *)malloc(sizeof(int32_t) * cap);
    m->sum = (int64_t *)calloc(cap, sizeof(int64_t));
    m->cnt = (int64_t *)calloc(cap, sizeof(int64_t));
    m->used = (uint8_t *)calloc(cap, 1);
    return (m->key && m->sum && m->cnt && m->used) ? 0 : -1;
}

static void gb_free(gb_map *m) {
    free(m->key); free(m->sum); free(m->cnt); free(m->used);
}

static void gb_add(gb_map *m, int32_t g, int64_t v, int64_t c);

static void gb_grow(gb_map *m) {
    gb_map n;
    gb_init(&n, m->cap * 2);
    for (uint64_t i = 0; i < m->cap; ++i)
        if (m->used[i]) gb_add(&n, m->key[i], m->sum[i], m->cnt[i]);
    gb_free(m);
    *m = n;
}

static void gb_add(gb_map *m, int32_t g, int64_t v, int64_t c) {
    if ((m->size + 1) * 2 > m->cap) gb_grow(m);
    uint64_t i = or_hash_murmur((uint32_t)g) & (m->cap - 1);
    while (m->used[i] && m->key[i] != g) i = (i + 1) & (m->cap - 1);
    if (!m->used[i]) { m->used[i] = 1; m->key[i] = g; m->size++; }
    m->sum[i] += v;
    m->cnt[i] += c;
}

static int cmp_group(const void *a, const void *b) {
    int32_t x = ((const or_group_row *)a)->group, y = ((const or_group_row *)b)->group;
    return (x > y) - (x < y);
}

/* SUM(value * mult) and COUNT(mult) per group, sorted by group key.
 * mult_or_null == NULL means multiplicity 1 for every row; rows with
 * multiplicity 0 create no group.  Returns the number of groups. */
uint64_t or_groupby(const int32_t *groups, const int32_t *values, const int32_t *mult_or_null,
                    uint64_t n, or_group_row *out, uint64_t cap) {
    gb_map m;
    gb_init(&m, 1024);
    for (uint64_t i = 0; i < n; ++i) {
        int64_t mu = mult_or_null ? mult_or_null[i] : 1;
        if (mu == 0) continue;
        gb_add(&m, groups[i], (int64_t)(values ? values[i] : 0) * mu, mu);
    }
    uint64_t k = 0;
    or_group_row *tmp = (or_group_row *)malloc(sizeof(or_group_row) * (m.size ? m.size : 1));
    for (uint64_t i = 0; i < m.cap; ++i)
        if (m.used[i]) {
            tmp[k].group = m.key[i];
            tmp[k].pad = 0;
            tmp[k].sum = m.sum[i];
            tmp[k].count = m.cnt[i];
            ++k;
        }
    qsort(tmp, k, sizeof(or_group_row), cmp_group);
    for (uint64_t i = 0; i < k && i < cap; ++i) out[i] = tmp[i];
    free(tmp);
    gb_free(&m);
    return k;
}

/* ---------------------------------------------------------------------- */
/* select -> hash join -> group-by query                                  */
/* ---------------------------------------------------------------------- */

/* For every probe row with filter <= bound, each build row with an equal
 * key contributes one output tuple; the tuples are grouped by the probe's
 * group column into int64 SUM(value) and COUNT.  The radix partition that
 * precedes the build on the GPU does not change this result. */
typedef struct query_job {
    const or_query *q;
    const or_chain_table *t;
    int32_t *mult;
    uint64_t lo, hi;
    int64_t count, sum;
} query_job;

/* The select + probe of rows [lo, hi): each row's match multiplicity. */
static void *query_probe(void *arg) {
    query_job *j = (query_job *)arg;
    const or_query *q = j->q;
    int64_t tc = 0, ts = 0;
    for (uint64_t i = j->lo; i < j->hi; ++i) {
        j->mult[i] = 0;
        if (q->probe_filter[i] <= q->filter_bound) {
            uint64_t mu = or_chain_matches(j->t, q->probe_key[i]);
            j->mult[i] = (int32_t)mu;
            tc += (int64_t)mu;
            ts += (int64_t)mu * q->probe_value[i];
        }
    }
    j->count = tc;
    j->sum = ts;
    return NULL;
}

/* The query with its select + probe phase split over `threads` host
 * threads (the table is read-only); build and group-by stay on one. */
uint64_t or_run_query_mt(const or_query *q, or_group_row *out, uint64_t cap,
                         int64_t *total_count, int64_t *total_sum, int threads) {
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    or_chain_table t;
    or_chain_build(&t, q->build_keys, NULL, q->build_rows, 0, 0);
    int32_t *mult = (int32_t *)malloc(sizeof(int32_t) * (q->probe_rows ? q->probe_rows : 1));
    pthread_t tid[256];
    query_job jobs[256];
    for (int i = 0; i < threads; ++i) {
        jobs[i].q = q;
        jobs[i].t = &t;
        jobs[i].mult = mult;
        jobs[i].lo = q->probe_rows * (uint64_t)i / (uint64_t)threads;
        jobs[i].hi = q->probe_rows * (uint64_t)(i + 1) / (uint64_t)threads;
        if (threads == 1) query_probe(&jobs[i]);
        else pthread_create(&tid[i], NULL, query_probe, &jobs[i]);
    }
    int64_t tc = 0, ts = 0;
    for (int i = 0; i < threads; ++i) {
        if (threads > 1) pthread_join(tid[i], NULL);
        tc += jobs[i].count;
        ts += jobs[i].sum;
    }
    uint64_t g = or_groupby(q->probe_group, q->probe_value, mult, q->probe_rows, out, cap);
    free(mult);
    or_chain_free(&t);
    if (total_count) *total_count = tc;
    if (total_sum) *total_sum = ts;
    return g;
}

uint64_t or_run_query(const or_query *q, or_group_row *out, uint64_t cap,
                      int64_t *total_count, int64_t *total_sum) {
    return or_run_query_mt(q, out, cap, total_count, total_sum, 1);
}
