/*
 * mgv_oracle.h -- CPU oracle for the vector-at-a-time operator pipeline.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load this library, and only as the checker or
 * as the timed CPU baseline; the product (libmgv) never links or calls it.
 *
 * It restates, in plain C, the reference's own CPU loops and the semantics of
 * its device operators, extended to the outputs the benchmarks ask for
 * (int64 SUM/COUNT, payload sums, hash GROUP BY, the join match multiset and
 * a radix partition).  Every function names the reference file:line it
 * follows.  The restatement is pinned against the reference's own CPU
 * functions compiled from its sources (oracle/build_ref.sh -> oracle/_ref)
 * and against the committed golden fixtures in tests/golden/.
 */
#ifndef MGV_ORACLE_H_
#define MGV_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- generators (same counter-based streams as the GPU side) ---------- */
void or_gen_uniform(int32_t *out, uint64_t n, uint64_t seed, uint32_t stream,
                    int64_t lo, uint64_t range);
void or_gen_perm(int32_t *out, uint64_t n, uint64_t seed);
uint64_t or_gen_probe_keys(int32_t *out, uint64_t n, uint64_t seed, uint64_t build_seed,
                           uint64_t nbuild, uint32_t hit_num, int64_t miss_lo,
                           uint64_t miss_range);
void or_zipf_cdf(uint64_t *cdf, uint32_t G, double s);
void or_gen_zipf(int32_t *out, uint64_t n, uint64_t seed, uint32_t stream,
                 const uint64_t *cdf, uint32_t G);

/* ---- hash ------------------------------------------------------------- */
uint32_t or_hash_murmur(uint32_t x);

/* ---- select ----------------------------------------------------------- */
size_t or_select_rows(const int32_t *a, size_t n, int32_t bound, int32_t *out);
void or_select_agg(const int32_t *f, const int32_t *v, size_t n, int32_t bound,
                   int64_t *count, int64_t *sum);
void or_select_agg_mt(const int32_t *f, const int32_t *v, size_t n, int32_t bound, int threads,
                      int64_t *count, int64_t *sum);

/* ---- chained hash join ------------------------------------------------ */
typedef struct or_chain_table {
    int32_t *head;      /* 2^log_size bucket heads, -1 = empty            */
    int32_t *next;      /* per build row: next row in chain, -1 = end     */
    const int32_t *keys;
    const int32_t *pay; /* may be NULL (payload 0)                        */
    uint64_t n;
    uint32_t log_size;
} or_chain_table;

int  or_chain_build(or_chain_table *t, const int32_t *keys, const int32_t *pay,
                    uint64_t n, int use_filter, int32_t bound);
void or_chain_free(or_chain_table *t);
void or_chain_probe_agg(const or_chain_table *t, const int32_t *pkeys,
                        const int32_t *ppay, uint64_t m, int add_build_pay,
                        int add_probe_pay, int64_t *count, int64_t *sum);
void or_chain_probe_agg_mt(const or_chain_table *t, const int32_t *pkeys,
                           const int32_t *ppay, uint64_t m, int threads,
                           int64_t *count, int64_t *sum);
uint64_t or_chain_probe_emit(const or_chain_table *t, const int32_t *pkeys,
                             const int32_t *ppay, uint64_t m, int32_t *out,
                             uint64_t cap);
uint64_t or_chain_matches(const or_chain_table *t, int32_t key);

/* ---- radix partition -------------------------------------------------- */
void or_partition(const int32_t *keys, uint64_t n, uint32_t bits, uint32_t shift,
                  uint64_t *hist, int32_t *out_keys, const int32_t *pay,
                  int32_t *out_pay);

/* ---- group-by --------------------------------------------------------- */
typedef struct or_group_row {
    int32_t group;
    int32_t pad;
    int64_t sum;
    int64_t count;
} or_group_row;

uint64_t or_groupby(const int32_t *groups, const int32_t *values, const int32_t *mult_or_null,
                    uint64_t n, or_group_row *out, uint64_t cap);

/* ---- full select -> join -> group-by query ---------------------------- */
typedef struct or_query {
    const int32_t *build_keys; uint64_t build_rows;
    const int32_t *probe_key, *probe_filter, *probe_group, *probe_value;
    uint64_t probe_rows;
    int32_t filter_bound;
} or_query;

uint64_t or_run_query(const or_query *q, or_group_row *out, uint64_t cap,
                      int64_t *total_count, int64_t *total_sum);
/* The same with the select + probe phase on `threads` host threads. */
uint64_t or_run_query_mt(const or_query *q, or_group_row *out, uint64_t cap,
                         int64_t *total_count, int64_t *total_sum, int threads);

#ifdef __cplusplus
}
#endif

#endif /* MGV_ORACLE_H_ */
