/*
 * CPU oracle for the oblivious operator path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithms, used by tests/, by
 * __graft_entry__.smoke() as the checker, and by bench.py's cpu_baseline and
 * `--impl reference` legs as the timed CPU path.  The product (velodb_b200)
 * never links or calls this library.
 *
 * Each function cites the reference file:line it restates (paths are relative
 * to the reference project root).  The ORCompact restatement is pinned
 * bit-exact against liboblivious o_compact compiled from the reference sources
 * (oracle/Makefile -> oracle/_ref/liboblivious.so); the bitonic restatement is
 * pinned against std-sort results and the reference's ORDER BY known answers.
 */
#ifndef VELO_ORACLE_H
#define VELO_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* DataTypeId values, reference include/data/data_type.hpp:12-26. */
enum {
    ORC_BOOLEAN = 1,
    ORC_TINYINT = 2,
    ORC_SMALLINT = 3,
    ORC_INTEGER = 4,
    ORC_BIGINT = 5,
    ORC_FLOAT = 6,
    ORC_DOUBLE = 7,
    ORC_VARCHAR = 8,
    ORC_DATE = 10
};

/* nextPow2, reference include/cuda/helper.hpp:50-62. */
size_t orc_next_pow2(size_t x);

/* Multi-column bitonic sort in the reference's network order and comparator,
 * reference include/cuda/sort.cuh:11-118.  Columns have capacity n_padded;
 * rows [n, n_padded) are filled with max/lowest per column; indices receives
 * the permutation (int64).  Returns 0, or -1 on an unsupported type. */
int orc_bitonic_sort_cols(int n_cols, void* const* cols, const int* types, const uint8_t* ascending,
                          size_t n, size_t n_padded, int64_t* indices);

/* Same network over (u64 key, u32 payload) rows compared lexicographically,
 * rows [n, n_padded) padded with (UINT64_MAX, UINT32_MAX); OpenMP across
 * n_threads (<= 0: all).  This is the timed CPU port of the sort. */
void orc_bitonic_kp(uint64_t* keys, uint32_t* pay, size_t n, size_t n_padded, int n_threads);

/* Same network over records of n_words u64 words (SoA, words[w][i]), compared
 * lexicographically on the first n_key_words words after AND-ing word w with
 * masks[w]; rows [n, n_padded) are filled with pad[w]. */
void orc_bitonic_records(uint64_t* const* words, int n_words, int n_key_words, const uint64_t* masks,
                         const uint64_t* pad, size_t n, size_t n_padded, int n_threads);

/* ORCompact (Goodrich's order-preserving compaction network as implemented by
 * liboblivious), reference obliviator/operator_1/third_party/liboblivious/
 * algorithms.c:116-213.  data is n elements of elem_size bytes; marks[i] != 0
 * marks element i; marks travel with their elements.  Returns the count. */
size_t orc_ocompact(uint8_t* data, size_t n, size_t elem_size, uint8_t* marks);

/* Stable scatter: out_idx[i] = rank of row i among marked rows for marked
 * rows (other entries untouched), as reference include/cuda/scatter.cuh:16-81
 * produces within one block; returns the count. */
size_t orc_scatter_stable(const uint8_t* mask, size_t n, int32_t* out_idx);

/* Oblivious group-by over key-sorted rows: forward segmented sum, backward
 * propagation, head flags, compaction of heads -- the single-thread path of
 * reference obliviator/operator_2/enclave/scalable_oblivious_join.c:222-245,
 * with int64 sums over n_vals value columns (vals row-major n x n_vals).
 * Writes one (key, sums) row per group in key order; returns the group count. */
size_t orc_groupby_sorted(const uint64_t* keys, const int64_t* vals, size_t n, int n_vals, uint64_t* out_keys,
                          int64_t* out_sums);

/* Filter + group-by over the synthetic lineitem-like fact table:
 * predicate  lo[c] <= col_c <= hi[c] for c in {shipdate, disc, qty},
 * group key  (flag1, flag2), sums (count, qty, price, price*(100-disc),
 * price*(100-disc)*(100+tax)), exact int64.  Steps: predicate -> stable
 * compaction -> bitonic sort by key -> segmented sum -> compaction of group
 * heads.  out_keys[g] = flag1 << 8 | flag2; out_sums is g x 5 row-major.
 * Returns the group count (at most max_groups are written). */
size_t orc_filter_groupby(size_t n, const int32_t* qty, const int64_t* price, const int32_t* disc,
                          const int32_t* tax, const int32_t* shipdate, const uint8_t* flag1, const uint8_t* flag2,
                          int32_t ship_lo, int32_t ship_hi, int32_t disc_lo, int32_t disc_hi, int32_t qty_lo,
                          int32_t qty_hi, size_t max_groups, uint64_t* out_keys, int64_t* out_sums, int n_threads);

/* PK-FK join + group-by + top-k: dim (key, date), fact (fk, price); join rows
 * with date < date_hi on the dim side and price < price_hi on the fact side;
 * group joined rows by fk summing price; return the k groups with the largest
 * sum (ties: smaller fk first).  Steps follow the union -> sort by (key, tag)
 * -> forward fill -> compaction -> group-by -> sort (sum desc, fk asc) order.
 * Writes up to k (fk, sum, count) triples; returns the number of joined groups. */
size_t orc_join_groupby_topk(size_t n_dim, const int32_t* dim_key, const int32_t* dim_date, size_t n_fact,
                             const int32_t* fact_fk, const int64_t* fact_price, int32_t date_hi, int64_t price_hi,
                             size_t k, int32_t* out_fk, int64_t* out_sum, int64_t* out_cnt, int n_threads);

/* Sort-merge inner equi-join with the reference's output, reference
 * include/cuda/sort_merge_join.cuh:63-199: both sides (rows with mask != 0;
 * NULL = all) sorted by (key, row id), merged, and every run of equal keys
 * written as its cross product, left row major.  Writes up to cap pairs of
 * (left row id, right row id) in (key, left row id, right row id) order and
 * returns the total pair count. */
size_t orc_smj_pairs(const int64_t* lkeys, const uint8_t* lmask, size_t nl, const int64_t* rkeys,
                     const uint8_t* rmask, size_t nr, int64_t* out_l, int64_t* out_r, size_t cap);

/* ------------------------------------------------------------------------ */
/* Oblivious CPU pipelines (oracle_obl.c): the timed CPU baseline.  The same  */
/* steps as the device pipelines, with no data-dependent branch, address or  */
/* size: network sorts over all next_pow2(n) rows, ORCompact, segmented      */
/* sums with masked slot adds.  OpenMP over n_threads (<= 0: all).           */
/* ------------------------------------------------------------------------ */

/* Bitonic network (reference order, strict exchanges) over np 16-byte
 * records {w0, w1}, ascending on (w0 & m0, w1 & m1); np a power of two. */
void orc_obl_sort_rec2(void* recs, size_t np, uint64_t m0, uint64_t m1, int n_threads);

/* ORCompact (liboblivious compact_offset, algorithms.c:118-153) of np
 * 16-byte records; a record is marked when bit `bit` of word `word`, XOR
 * inv, is 1.  np a power of two.  Returns the number of marked records. */
size_t orc_obl_compact_rec2(void* recs, size_t np, int word, int bit, int inv, int n_threads);

/* orc_filter_groupby's result (same contract) from the oblivious steps:
 * predicate -> ORCompact of all next_pow2(n) rows -> network sort of all of
 * them on the group key -> segmented sums into max_groups ranked slots. */
size_t orc_obl_filter_groupby(size_t n, const int32_t* qty, const int64_t* price, const int32_t* disc,
                              const int32_t* tax, const int32_t* shipdate, const uint8_t* flag1,
                              const uint8_t* flag2, int32_t ship_lo, int32_t ship_hi, int32_t disc_lo,
                              int32_t disc_hi, int32_t qty_lo, int32_t qty_hi, size_t max_groups,
                              uint64_t* out_keys, int64_t* out_sums, int n_threads);

/* orc_join_groupby_topk's result (same contract) from the oblivious steps:
 * union -> network sort on (key, tag) -> forward fill -> ORCompact of the
 * joined rows -> segmented sums -> ORCompact of the group records -> network
 * sort of next_pow2(n_dim) group records on (sum desc, fk asc).  Keys must be
 * below INT32_MAX (the pad key). */
size_t orc_obl_join_groupby_topk(size_t n_dim, const int32_t* dim_key, const int32_t* dim_date, size_t n_fact,
                                 const int32_t* fact_fk, const int64_t* fact_price, int32_t date_hi,
                                 int64_t price_hi, size_t k, int32_t* out_fk, int64_t* out_sum, int64_t* out_cnt,
                                 int n_threads);

#ifdef __cplusplus
}
#endif

#endif
