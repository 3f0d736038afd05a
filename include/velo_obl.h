/*
 * velo_obl.h -- C ABI of the B200 (sm_100a) oblivious operator library.
 *
 * Plain pointers and sizes only.  Every `d_*` pointer is device memory owned
 * by the caller; `stream` is a cudaStream_t passed as void* (NULL = the
 * legacy default stream).  Entry points enqueue work on the stream and return
 * without synchronising unless stated otherwise.  All kernels are
 * data-oblivious: for two inputs of the same public size they issue the same
 * launches, the same global/shared memory addresses and the same branches.
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the reference project root).  Sizes are public: outputs are padded to
 * public bounds instead of revealing true cardinalities, except where a
 * function documents that it returns a count (as the reference operators do).
 */
#ifndef VELO_OBL_H
#define VELO_OBL_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* status codes (replace the reference's VELODB_THROW / CHECKED_CALL_THROW,  */
/* include/cuda/helper.hpp:26-48)                                           */
/* ------------------------------------------------------------------------ */
typedef int32_t velo_status;
#define VELO_OK 0
#define VELO_EINVAL (-1)    /* bad argument (size, alignment, capacity, type) */
#define VELO_ENOMEM (-2)    /* scratch / arena too small */
#define VELO_ECUDA (-3)     /* a CUDA runtime call failed; see velo_last_error */
#define VELO_ETIMEDOUT (-4) /* a bounded wait ran out (host or device side) */
#define VELO_EOVERFLOW (-5) /* a public bound was exceeded by the data */
#define VELO_ESTATE (-6)    /* call not valid in the current state */
#define VELO_ENOTSUP (-7)   /* type or configuration not supported */

/* Column types, numerically equal to DataTypeId
 * (include/data/data_type.hpp:12-26; device types per
 * include/data/type_traits.hpp:10-19). */
typedef enum velo_type {
    VELO_BOOLEAN = 1,  /* uint8_t */
    VELO_TINYINT = 2,  /* int8_t */
    VELO_SMALLINT = 3, /* int16_t */
    VELO_INTEGER = 4,  /* int32_t */
    VELO_BIGINT = 5,   /* int64_t */
    VELO_FLOAT = 6,    /* float */
    VELO_DOUBLE = 7,   /* double */
    VELO_VARCHAR = 8,  /* size_t ordinal */
    VELO_DATE = 10     /* uint32_t */
} velo_type;

/* Tile configuration of the network kernels: tile = 2^tile_log2 rows per CTA
 * (11..13), threads = 256/512/1024.  NULL = defaults (velo_osort_kp and
 * velo_ocompact_kpm: 2048-row tiles of 256 threads up to 2^18 rows, 4096-row
 * tiles of 256 threads above). */
typedef struct velo_tune {
    uint32_t tile_log2;
    uint32_t threads;
} velo_tune;

/* nextPow2 (include/cuda/helper.hpp:50-62). */
size_t velo_next_pow2(size_t x);

/* Text of the last error raised on this host thread ("" if none). */
const char* velo_last_error_text(void);

/*
 * Stage timing for profilers (off by default; process-wide switch).  While it
 * is on, the multi-stage pipelines (velo_filter_groupby,
 * velo_join_groupby_topk) record a CUDA event on their stream before and
 * after each stage and synchronize that stream before returning; the stage
 * durations of the calling thread's last such call are then read with
 * velo_last_stage_times (ms, in stage order; returns how many were written).
 *   velo_filter_groupby:    pack, compact, sort, aggregate
 *   velo_join_groupby_topk: pack, sort, fill, compact, aggregate, top-k
 * No reference counterpart: a measurement hook of this implementation.
 */
void velo_set_stage_timing(int on);
int velo_last_stage_times(float* ms, int capacity);

/*
 * Pass timing for profilers (off by default; process-wide switch).  While it
 * is on, every network pass (bitonic tile sort, fused global levels, in-tile
 * merge, ORCompact tile and global passes) is bracketed by CUDA events on its
 * stream, and each call that launches passes synchronizes that stream before
 * returning and appends one velo_pass_time per pass to the calling thread's
 * list (at most 1024 entries; velo_set_pass_timing and velo_pass_times_clear
 * empty it).  kind: 0 tile sort, 1 in-tile merge, 2 global levels, 3 ORCompact
 * tile pass, 4 ORCompact global levels; row_bytes: bytes of one row the pass
 * reads and writes.  The events keep consecutive passes from overlapping, so
 * the figures are per-pass durations, not the pipelined whole.
 * No reference counterpart: a measurement hook of this implementation.
 */
typedef struct velo_pass_time {
    uint32_t kind;
    uint32_t log_n;
    uint32_t row_bytes;
    float ms;
} velo_pass_time;
void velo_set_pass_timing(int on);
/* Tune: run the in-tile merge passes of 4096-row sorts (key-payload rows and
 * two- or three-word records) as one persistent CTA per SM that prefetches
 * the next tile with bulk copies into a second shared-memory buffer while
 * the current tile's levels run (0 = off, the default).  Same network, same
 * results.  No reference counterpart. */
void velo_set_merge_pipeline(int on);
/* Tune: load the rows of each in-tile merge and fused global pass of sorts
 * in 4096-row tiles (key-payload rows, two- or three-word records) with one
 * 3-D tensor-map copy per word array into shared memory instead of
 * per-thread loads (0 = off, the default).  Same grid, same network, same
 * results.  The tensor maps cover the calling GPU's own arrays.  No
 * reference counterpart. */
void velo_set_tensor_tile_loads(int on);
/* Status of the tensor-map pass kernels on the current device since the
 * first of them ran (synchronizes with the device): 0 none, 1 a tile copy
 * did not complete in time, 2 / 3 a shared-memory destination / tensor map
 * off its required alignment (the CTA then skipped its rows); -1 if it
 * cannot be read.  No reference counterpart. */
int velo_tensor_tile_status(void);
void velo_pass_times_clear(void);
int velo_last_pass_times(velo_pass_time* out, int capacity);

/* ------------------------------------------------------------------------ */
/* Bitonic network sort                                                     */
/* ------------------------------------------------------------------------ */

/* Oblivious bitonic sort of (u64 key, u32 payload) rows, ascending on
 * (key, payload).  Replaces OP_SORT / executeBitonicSort
 * (include/cuda/sort.cuh:70-118, include/cuda/commands.hpp:68-76) for two
 * sort columns: same network (k ascending, j descending, partner i^j,
 * direction (i&k)==0), same exchange rule (swap iff strictly out of order),
 * so the output is identical to the reference network's.  Buffers hold
 * capacity >= velo_next_pow2(n) rows; rows [n, next_pow2(n)) are filled with
 * the sentinel (UINT64_MAX, UINT32_MAX) and sort last. */
velo_status velo_osort_kp(uint64_t* d_keys, uint32_t* d_payload, size_t n, size_t capacity, const velo_tune* tune,
                          void* stream);

/* Multi-column sort with the reference OP_SORT contract
 * (include/cuda/sort.cuh:70-118, src/operator/sort_operator.cpp:52-79):
 * up to 8 sort columns of any velo_type, per-column ascending flags, columns
 * sorted in place over capacity >= next_pow2(n) rows padded with
 * max()/lowest(), and d_indices (int64, capacity rows) receiving the
 * permutation.  Columns are encoded into order-preserving unsigned keys and
 * sorted by the same network, so ties resolve exactly as in the reference
 * (floating-point -0.0/+0.0 are ordered by bit pattern; NaN is unsupported).
 * d_scratch: velo_sort_scratch_bytes() bytes. */
velo_status velo_sort_columns(void* const* d_cols, const uint32_t* types, const uint8_t* ascending, uint32_t n_cols,
                              size_t n, size_t capacity, int64_t* d_indices, void* d_scratch, size_t scratch_bytes,
                              void* stream);
size_t velo_sort_scratch_bytes(const uint32_t* types, uint32_t n_cols, size_t n);

/* Oblivious bitonic sort of records of n_words u64 words (SoA: d_words[w]
 * points at word w of every row; 1..3 words), ordered on word 0 AND-ed with
 * key_mask; the other words ride along.  Rows [n, next_pow2(n)) are filled
 * with all-ones words (they sort last).  flags: VELO_SORT_STRICT keeps the
 * reference's tie rule (include/cuda/sort.cuh:31-40: equal keys are never
 * exchanged), so the arrangement of equal keys is exactly the reference
 * network's; without it equal keys may be exchanged in descending merges
 * (one comparison per exchange), for consumers that aggregate over ties.
 * This is the row-record form the operators use for ORDER BY and group-by
 * inputs whose payload is packed next to the key. */
#define VELO_SORT_STRICT 1u
velo_status velo_osort_records(uint64_t* const* d_words, uint32_t n_words, uint64_t key_mask, size_t n,
                               size_t capacity, uint32_t flags, const velo_tune* tune, void* stream);

/* ------------------------------------------------------------------------ */
/* ORCompact (order-preserving oblivious compaction)                        */
/* ------------------------------------------------------------------------ */

/* Oblivious compaction of (u64 key, u32 payload, u8 mark) rows: marked rows
 * move to the front in their original order, unmarked rows follow.  The
 * routing network is ORCompact as in liboblivious
 * (obliviator/operator_1/third_party/liboblivious/algorithms.c:116-213),
 * run over the next_pow2(n) padded rows; it replaces the non-oblivious
 * OP_SCATTER + OP_GATHER pair (include/cuda/scatter.cuh:16-81,
 * include/cuda/gather.cuh:28-45, src/operator/filter_compaction_operator.cpp:65-184).
 * *d_count (u64, device) receives the number of marked rows.
 * d_scratch: velo_compact_scratch_bytes(capacity) bytes of device memory. */
velo_status velo_ocompact_kpm(uint64_t* d_keys, uint32_t* d_payload, uint8_t* d_marks, size_t n, size_t capacity,
                              uint64_t* d_count, void* d_scratch, size_t scratch_bytes, const velo_tune* tune,
                              void* stream);
size_t velo_compact_scratch_bytes(size_t capacity, const velo_tune* tune);

/* Same compaction as velo_ocompact_kpm (same output; 8192-row tiles of 512
 * threads, which keep the fixed scratch small), for callers that cannot allocate device memory -- an engine whose HBM is
 * owned by its own pool allocator, a latency-critical path that cannot take
 * cudaMalloc's implicit device synchronisation, a plugin host without an
 * allocation hook.  It takes no scratch argument and allocates nothing: its
 * scratch is a fixed array of 262,400 B (256 KiB + 256 B) in the library's
 * device memory, held on every GPU that loads the library until the process
 * exits.  Limit: n up to 2^28 rows (larger n returns VELO_EINVAL).  The first
 * call on a device looks up the array's device address (cudaGetSymbolAddress)
 * and keeps it; make that first call before any stream capture, and do not
 * reset the device (cudaDeviceReset) after it.  All calls share the array: calls that overlap
 * on the GPU race and must be serialised by the caller.  Every call rewrites
 * the array before reading it, so results never depend on earlier calls.
 * This entry point has no counterpart in the reference. */
velo_status velo_ocompact_kpm_noalloc(uint64_t* d_keys, uint32_t* d_payload, uint8_t* d_marks, size_t n,
                                      size_t capacity, uint64_t* d_count, void* stream);

/* ------------------------------------------------------------------------ */
/* Column operators of the reference command set (same semantics, including  */
/* the reference's data-dependent addresses) -- for drop-in compatibility    */
/* ------------------------------------------------------------------------ */

/* OP_PERMUTE: out[i] = in[idx[i]], i < n (include/cuda/permute.cuh:24-40). */
velo_status velo_permute(void* d_out, const void* d_in, const int64_t* d_indices, size_t n, uint32_t type,
                         void* stream);
/* OP_SCATTER: for rows with mask != 0, out_idx[i] = rank among kept rows
 * (the order one block of include/cuda/scatter.cuh:16-81 produces; the
 * reference's block order is nondeterministic); *d_count = kept rows. */
size_t velo_scatter_scratch_bytes(size_t n);
velo_status velo_scatter(const uint8_t* d_mask, size_t n, int32_t* d_out_indices, uint64_t* d_count, void* d_scratch,
                         size_t scratch_bytes, void* stream);
/* OP_GATHER: out[idx[i]] = in[i] where mask (NULL = all)
 * (include/cuda/gather.cuh:28-45). */
velo_status velo_gather(void* d_out, const void* d_in, const int32_t* d_indices, const uint8_t* d_mask, size_t n,
                        uint32_t type, void* stream);
/* OP_COMPARE_EQ: out[i] = (l[i] == r[i]); BOOLEAN and VARCHAR give all zeros
 * and DATE compares as int32, as include/cuda/compare.cuh:25-91 does. */
velo_status velo_compare_eq(const void* d_left, const void* d_right, uint8_t* d_out_mask, size_t n, uint32_t type,
                            void* stream);
/* OP_COMPOSE_POSITION_MAP: new[i] = old[sigma[i]]
 * (include/cuda/oblivious_shuffle.cuh:10-21). */
velo_status velo_compose_position_map(const uint32_t* d_old, const uint32_t* d_sigma, uint32_t* d_new, size_t n,
                                      void* stream);
/* OP_ENRICH_POSITIONS: pos[i] = map[rid[i]] (oblivious_shuffle.cuh:23-34).
 * velo_ogather_u64 is the oblivious form. */
velo_status velo_enrich_positions(const uint32_t* d_record_ids, const uint32_t* d_map, uint32_t* d_out, size_t n,
                                  void* stream);

/* ------------------------------------------------------------------------ */
/* Device memory and streams (for host code above the ABI)                   */
/* ------------------------------------------------------------------------ */

enum { VELO_COPY_H2D = 1, VELO_COPY_D2H = 2, VELO_COPY_D2D = 3 };
/* Stream-ordered allocation (cudaMallocAsync); VELO_ENOMEM when the device is
 * full.  bytes == 0 gives NULL. */
velo_status velo_device_alloc(size_t bytes, void* stream, void** out);
velo_status velo_device_free(void* p, void* stream);
/* Stream-ordered copy; kind is VELO_COPY_*. */
velo_status velo_copy(void* dst, const void* src, size_t bytes, uint32_t kind, void* stream);
velo_status velo_memset(void* dst, int value, size_t bytes, void* stream);
velo_status velo_stream_sync(void* stream);

/* ------------------------------------------------------------------------ */
/* Address-trace recording (obliviousness tests)                            */
/* ------------------------------------------------------------------------ */

/* Only the test build libvelo_obl_trace.so (compiled with VELO_TRACE)
 * records; the product library returns VELO_ENOTSUP and velo_trace_enabled
 * 0.  Between begin and end, every instrumented global load/store folds
 * (site, address) into a hash chain per logical thread (slots of them) and
 * every instrumented kernel logs (kernel id, grid, block, dynamic smem).  No
 * reference counterpart. */
int velo_trace_enabled(void);
velo_status velo_trace_begin(uint64_t slots, uint64_t launch_capacity);
velo_status velo_trace_end(uint64_t* chain_digest, uint64_t* touched, uint64_t* launches, uint64_t launch_capacity,
                           uint64_t* n_launches);

/* ------------------------------------------------------------------------ */
/* Column helpers of the operator layer                                     */
/* ------------------------------------------------------------------------ */

/* d_mask[i] = (lo <= col[i] <= hi), or AND-ed into d_mask when combine != 0:
 * the conjunctive range predicates SeqScanOperator pushes down
 * (src/operator/seq_scan_operator.cpp:38-45), evaluated on the device.
 * Integer, BOOLEAN and DATE columns; one pass, every row read. */
velo_status velo_range_mask(const void* d_col, uint32_t type, size_t n, int64_t lo, int64_t hi, uint8_t* d_mask,
                            uint32_t combine, void* stream);
/* d_out[i] = the integer, BOOLEAN or DATE value col[i] as int64 (operands of
 * SUM in velo_ogroupby). */
velo_status velo_widen_i64(const void* d_col, uint32_t type, size_t n, int64_t* d_out, void* stream);
/* d_out[i] = start + i (the $_rowid column of a scan). */
velo_status velo_iota_i64(int64_t* d_out, size_t n, int64_t start, void* stream);
/* Oblivious in-place compaction of n_cols typed columns (and their validity
 * bytes, d_valid[c] may be NULL) by d_mask: the rows with mask != 0 move to
 * [0, *d_count) in input order.  ORCompact over next_pow2(n) rows, two columns
 * per network run; the exchanges depend only on n.  Replaces OP_SCATTER +
 * OP_GATHER of FilterCompactionOperator
 * (src/operator/filter_compaction_operator.cpp:65-184), whose scatter
 * addresses follow the data. */
size_t velo_ocompact_columns_scratch_bytes(size_t n);
velo_status velo_ocompact_columns(void* const* d_cols, const uint32_t* types, uint8_t* const* d_valid,
                                  uint32_t n_cols, const uint8_t* d_mask, size_t n, uint64_t* d_count,
                                  void* d_scratch, size_t scratch_bytes, void* stream);

/* Oblivious typed gather of one column with validity (materialization):
 * out[j] = col[rowid[j]] and out_valid[j] = valid[rowid[j]] for 0 <= rowid[j]
 * < table_n, else 0 / not valid.  Built on velo_ogather_u64 (one sort-based
 * gather, two for 8-byte types when out_valid is wanted); the addresses
 * depend only on table_n and n. */
size_t velo_ogather_column_scratch_bytes(size_t table_n, size_t n);
velo_status velo_ogather_column(const void* d_table_col, uint32_t type, const uint8_t* d_table_valid,
                                size_t table_n, const int64_t* d_rowids, size_t n, void* d_out,
                                uint8_t* d_out_valid, void* d_scratch, size_t scratch_bytes, void* stream);

/* Oblivious GROUP BY key with SUM / COUNT: one or two aggregates a call
 * (n_sums int64 columns summed mod 2^64, plus COUNT when with_count; n_sums +
 * with_count is 1 or 2).  Rows with mask == 0 (NULL = all rows) are left out.
 * Keys: VELO_INTEGER or VELO_BIGINT, every value of either.  Writes the first
 * group_bound groups in key order -- d_out_keys[j], d_out_sums[s][j],
 * d_out_counts[j] -- and zeros past the number of groups; d_counts (2 u64) =
 * (groups, 0).  Sort, segmented sums and ORCompact of one record per group;
 * every address depends only on n, group_bound and the key type.  The reference engine declares an
 * aggregate plan node (include/planner/abstract_plan_node.hpp:31) without an
 * operator; the algorithm is obliviator/operator_2/enclave/
 * scalable_oblivious_join.c:105-262. */
size_t velo_ogroupby_scratch_bytes(size_t n);
velo_status velo_ogroupby(const void* d_keys, uint32_t key_type, const int64_t* const* d_sums, uint32_t n_sums,
                          uint32_t with_count, const uint8_t* d_mask, size_t n, size_t group_bound,
                          int64_t* d_out_keys, int64_t* const* d_out_sums, int64_t* d_out_counts,
                          uint64_t* d_counts, void* d_scratch, size_t scratch_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* Oblivious shuffle, gather and PK-FK join                                 */
/* ------------------------------------------------------------------------ */

/* Oblivious re-shuffle of a position map on the device: map <- map o sigma
 * with sigma the permutation that sorts the keys Philox4x32-10(i, counter,
 * key) (Salmon et al., SC'11), applied by the bitonic network.  Replaces the
 * host Fisher-Yates draw plus H2D copy of sigma plus the data-dependent
 * compose (src/data/oblivious_table.cpp:170-202). */
size_t velo_oshuffle_scratch_bytes(size_t n);
velo_status velo_oshuffle_position_map(uint32_t* d_map, size_t n, uint64_t key, uint64_t counter, void* d_scratch,
                                       size_t scratch_bytes, void* stream);

/* Oblivious gather out[j] = table[rid[j]] (0 when rid >= table_n): union of
 * table rows and requests, bitonic sort on (row, tag), forward fill, bitonic
 * sort back to request order.  Replaces the data-dependent reads of
 * OP_ENRICH_POSITIONS and of oblivious materialization
 * (src/operator/materialization_operator.cpp:362-517, whose gather runs on the
 * CPU with dummy reads); duplicate requests are served without dummies. */
size_t velo_ogather_scratch_bytes(size_t table_n, size_t n_req);
velo_status velo_ogather_u64(const uint64_t* d_table, size_t table_n, const uint32_t* d_rids, size_t n_req,
                             uint64_t* d_out, void* d_scratch, size_t scratch_bytes, void* stream);

/* Oblivious PK-FK equi-join producing the reference join operators' output
 * (pairs of build-side and probe-side row ids, as OP_SORT_MERGE_JOIN_WRITE
 * and OP_HASH_JOIN_WRITE produce: include/cuda/sort_merge_join.cuh:141-199,
 * include/cuda/hash_join.cuh:170-254), for a build side with unique keys.
 * Rows with mask == 0 (NULL = all valid) do not join.  Output is padded to
 * the public bound probe_n: rows [0, count) hold the pairs in key order,
 * the rest -1.  d_counts: 2 u64 = (pairs, build rows whose key repeats an
 * earlier build key -- nonzero means the build side was not a key).
 * key_type: VELO_INTEGER or VELO_BIGINT. */
size_t velo_ojoin_scratch_bytes(size_t build_n, size_t probe_n);
velo_status velo_ojoin_pkfk(const void* d_build_keys, const uint8_t* d_build_mask, size_t build_n,
                            const void* d_probe_keys, const uint8_t* d_probe_mask, size_t probe_n, uint32_t key_type,
                            int64_t* d_out_build_rowid, int64_t* d_out_probe_rowid, uint64_t* d_counts,
                            void* d_scratch, size_t scratch_bytes, void* stream);

/* Oblivious many-to-many equi-join: every pair (build row b, probe row p)
 * with key_b == key_p and both rows valid (mask != 0; NULL = all valid), the
 * output of the reference's sort-merge join (the cross product of every run
 * of equal keys, include/cuda/sort_merge_join.cuh:63-199, sized from the true
 * pair count in src/operator/sort_merge_join_operator.cpp:114-148), padded to
 * the public bound max_pairs.  Rows [0, min(pairs, max_pairs)) of the two
 * outputs hold the pairs in (key, probe row id, build row id) order, the rest
 * -1.  d_counts: 2 u64 = (pairs, 1 if pairs > max_pairs else 0); a caller
 * that must not lose pairs re-runs with max_pairs >= pairs, which reveals the
 * pair count as the reference does.  Every launch and address depends only on
 * build_n, probe_n and max_pairs (all below 2^31).  key_type: VELO_INTEGER or
 * VELO_BIGINT.  d_scratch: velo_ojoin_mn_scratch_bytes() bytes. */
size_t velo_ojoin_mn_scratch_bytes(size_t build_n, size_t probe_n, size_t max_pairs);
velo_status velo_ojoin_mn(const void* d_build_keys, const uint8_t* d_build_mask, size_t build_n,
                          const void* d_probe_keys, const uint8_t* d_probe_mask, size_t probe_n, uint32_t key_type,
                          size_t max_pairs, int64_t* d_out_build_rowid, int64_t* d_out_probe_rowid,
                          uint64_t* d_counts, void* d_scratch, size_t scratch_bytes, void* stream);

/* Oblivious bin-padded hash join, the HashJoinOperator's algorithm
 * (replaces the chained hash table of include/cuda/hash_join.cuh:28-254 and
 * src/operator/hash_join_operator.cpp:88-393): both sides are hashed into
 * bins by a keyed Philox4x32-10 hash (hash_seed) and every bin is padded to a
 * public capacity derived from build_n and probe_n, so bin occupancy never
 * shows; each bin compares every probe slot with every build slot.  For a
 * build side with unique keys (the PK-FK case) rows [0, pairs) of the outputs
 * (probe_n rows) hold (build row id, probe row id) pairs in (bin, probe row
 * id) order, the rest -1.  Rows with mask == 0 (NULL = all valid) do not join.
 * d_counts: 3 u64 = (pairs, probe rows with more than one partner -- a
 * repeated build key --, real rows that did not fit their bin).  When either
 * of the last two is nonzero the pairs are incomplete: join with
 * velo_ojoin_mn instead (HashJoinOperator does).  key_type: VELO_INTEGER or
 * VELO_BIGINT.  d_scratch: velo_ohash_join_scratch_bytes() bytes. */
size_t velo_ohash_join_scratch_bytes(size_t build_n, size_t probe_n);
velo_status velo_ohash_join(const void* d_build_keys, const uint8_t* d_build_mask, size_t build_n,
                            const void* d_probe_keys, const uint8_t* d_probe_mask, size_t probe_n, uint32_t key_type,
                            uint64_t hash_seed, int64_t* d_out_build_rowid, int64_t* d_out_probe_rowid,
                            uint64_t* d_counts, void* d_scratch, size_t scratch_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* Batched form: one persistent launch for many independent commands        */
/* ------------------------------------------------------------------------ */

/* One command of a batch: an oblivious sort (as velo_osort_kp) or an
 * ORCompact (as velo_ocompact_kpm) of caller-owned device buffers. */
#define VELO_ITEM_SORT_KP 1u
#define VELO_ITEM_COMPACT_KPM 2u
typedef struct velo_batch_item {
    uint32_t kind; /* VELO_ITEM_SORT_KP or VELO_ITEM_COMPACT_KPM */
    uint32_t pad_;
    uint64_t* d_keys;
    uint32_t* d_payload;
    uint8_t* d_marks;  /* compaction only */
    size_t n;
    size_t capacity;   /* >= next_pow2(n) rows */
    uint64_t* d_count; /* compaction only: receives the number of marked rows */
} velo_batch_item;

typedef struct velo_batch velo_batch;

/* Plans a batch: every command becomes a list of passes over tiles; all
 * commands' (pass, tile) items are interleaved and run by one persistent
 * kernel whose CTAs claim items in order and wait (bounded) only for the
 * previous pass of the same command.  Replaces the reference's one-command-
 * at-a-time persistent grid (src/cuda/persistent_kernel.cu:76-124,
 * src/cuda/task_manager.cu:26-78).  Results are identical to running each
 * command through velo_osort_kp / velo_ocompact_kpm with the same tune
 * (NULL: 4096-row tiles of 256 threads).
 * Allocates the batch's device plan (cudaMalloc) here, never at launch. */
velo_status velo_batch_create(const velo_batch_item* items, size_t n_items, const velo_tune* tune,
                              velo_batch** out);
/* Enqueues the whole batch on `stream`: a counter reset and ONE kernel
 * launch, so the call can be captured into a CUDA graph and replayed. */
velo_status velo_batch_launch(velo_batch* batch, void* stream);
/* Synchronises `stream` and returns VELO_ETIMEDOUT if a device-side wait of
 * the last launch ran out of time (the kernel never spins unbounded). */
velo_status velo_batch_status(velo_batch* batch, void* stream);
void velo_batch_destroy(velo_batch* batch);
/* Limit of every device-side wait of the batch (default 2 s). */
velo_status velo_batch_set_timeout(velo_batch* batch, uint64_t timeout_ns);
/* Failure injection for tests: makes the first wait of command `item` wait
 * for a completion count that is never reached, so it runs into the time
 * limit; the launch still terminates and velo_batch_status reports
 * VELO_ETIMEDOUT (the command's output is then undefined). */
velo_status velo_batch_inject_unmet_wait(velo_batch* batch, uint32_t item);
/* Autotuner: times the batch for every tile configuration of the search
 * space (tiles 2^11, 2^12, 2^13 x 256, 512, 1024 threads; `reps` timed
 * launches each), writes the fastest to *best and the per-configuration
 * milliseconds to ms_out[9] (may be NULL).  Runs on the live buffers: the
 * networks are data-oblivious, so the timing does not depend on the data;
 * re-running keeps every sort's output and every compaction's marked prefix
 * and count (the unmarked tail of a compaction is re-routed). */
velo_status velo_batch_autotune(const velo_batch_item* items, size_t n_items, uint32_t reps, velo_tune* best,
                                float* ms_out, void* stream);

/* ------------------------------------------------------------------------ */
/* Filter + group-by (oblivious)                                            */
/* ------------------------------------------------------------------------ */

/* Columns of a lineitem-shaped fact table (device pointers, n rows each). */
typedef struct velo_lineitem {
    const int32_t* qty;      /* quantity */
    const int64_t* price;    /* extended price, cents */
    const int32_t* disc;     /* discount, percent */
    const int32_t* tax;      /* tax, percent */
    const int32_t* shipdate; /* ship date, days */
    const uint8_t* flag1;    /* first group column */
    const uint8_t* flag2;    /* second group column */
} velo_lineitem;

/* Conjunctive range predicate lo <= col <= hi on shipdate, disc and qty. */
typedef struct velo_lineitem_pred {
    int32_t ship_lo, ship_hi;
    int32_t disc_lo, disc_hi;
    int32_t qty_lo, qty_hi;
} velo_lineitem_pred;

/* flags: sort only next_pow2(filtered count) rows after compaction, reading
 * the count back to the host first (the reference FilterCompactionOperator
 * reveals it, src/operator/filter_compaction_operator.cpp:171-178).  Without
 * this flag the whole pipeline is oblivious and never synchronises. */
#define VELO_REVEAL_COUNT 1u

/* Oblivious filter + GROUP BY (flag1, flag2) with exact int64 sums:
 * predicate and record packing on the GPU (replacing the CPU predicate of
 * src/operator/seq_scan_operator.cpp:38-45), ORCompact of passing rows
 * (replacing src/operator/filter_compaction_operator.cpp:65-184), bitonic
 * sort on the group key, segmented sums
 * (obliviator/operator_2/enclave/scalable_oblivious_join.c:221-262, int64
 * instead of float), output padded to the public bound group_bound (1..16).
 * d_out: group_bound rows x 6 int64 = (flag1 << 8 | flag2, count, sum qty,
 * sum price, sum price*(100-disc), sum price*(100-disc)*(100+tax)) in key
 * order, unused rows zero.  d_counts: 2 u64 = (rows passing the filter,
 * number of groups; more groups than group_bound means the bound was too
 * small and only the first group_bound are written). */
size_t velo_filter_groupby_scratch_bytes(size_t n, uint32_t group_bound);
velo_status velo_filter_groupby(const velo_lineitem* cols, size_t n, const velo_lineitem_pred* pred,
                                uint32_t group_bound, uint32_t flags, int64_t* d_out, uint64_t* d_counts,
                                void* d_scratch, size_t scratch_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* PK-FK join + group-by + top-k (oblivious)                                */
/* ------------------------------------------------------------------------ */

typedef struct velo_join_tables {
    const int32_t* dim_key;    /* unique keys of the dimension table */
    const int32_t* dim_date;   /* dimension attribute filtered by date_hi */
    size_t n_dim;
    const int32_t* fact_fk;    /* foreign keys into dim_key */
    const int64_t* fact_price; /* fact attribute, cents; summed per fk */
    size_t n_fact;
} velo_join_tables;

typedef struct velo_join_pred {
    int32_t date_hi;  /* dimension rows with dim_date < date_hi join */
    int32_t pad_;
    int64_t price_hi; /* fact rows with fact_price < price_hi join */
} velo_join_pred;

/* Oblivious PK-FK join, GROUP BY fk with SUM(price) and COUNT, then the k
 * groups with the largest sums (ties: smaller fk first).  Replaces the
 * reference's sort-merge join kernels and operator
 * (include/cuda/sort_merge_join.cuh:63-199,
 * src/operator/sort_merge_join_operator.cpp:27-257) with union -> bitonic
 * sort on (key, tag) -> forward fill -> ORCompact -> segmented sums ->
 * bitonic top-k network on (sum desc, fk asc) (each group-by tile keeps its
 * best max(16, next_pow2(k)) groups, then rounds over candidate blocks).
 * k is 1..1024.  d_out: k rows x 3 int64 = (fk, sum price, count), unused
 * rows zero.  d_counts: 2 u64 = (joined fact rows, groups). */
size_t velo_join_groupby_topk_scratch_bytes(size_t n_dim, size_t n_fact);
velo_status velo_join_groupby_topk(const velo_join_tables* tables, const velo_join_pred* pred, uint32_t k,
                                   int64_t* d_out, uint64_t* d_counts, void* d_scratch, size_t scratch_bytes,
                                   void* stream);

/* ------------------------------------------------------------------------ */
/* Command queue: the boundary the reference's TaskManager /                */
/* CommandQueueController expose (include/cuda/task_manager.hpp:12-30,      */
/* include/cuda/commands.hpp:16-201, src/cuda/commands.cpp:47-91)           */
/* ------------------------------------------------------------------------ */

/* Opcodes: the reference's OpCode values for the operators it has, new
 * values for the oblivious operators. */
typedef enum velo_opcode {
    VELO_OP_NOP = 0,
    VELO_OP_SCATTER = 1,
    VELO_OP_GATHER = 2,
    VELO_OP_SORT = 3, /* multi-column sort, reference contract (velo_sort_columns) */
    VELO_OP_PERMUTE = 4,
    VELO_OP_COMPARE_EQ = 10,
    VELO_OP_COMPOSE_POSITION_MAP = 11,
    VELO_OP_ENRICH_POSITIONS = 12,
    VELO_OP_OSORT_KP = 0x100,
    VELO_OP_OCOMPACT_KPM = 0x101,
    VELO_OP_OSORT_RECORDS = 0x102,
    VELO_OP_OJOIN_PKFK = 0x103,
    VELO_OP_OGATHER = 0x104,
    VELO_OP_OSHUFFLE = 0x105,
    VELO_OP_FILTER_GROUPBY = 0x106,
    VELO_OP_JOIN_GROUPBY_TOPK = 0x107,
    VELO_OP_OJOIN_MN = 0x108,
    VELO_OP_OHASH_JOIN = 0x109
} velo_opcode;

/* A command: device pointers and public sizes only (the same arguments as
 * the direct entry point of each opcode; scratch buffers are caller-owned). */
typedef struct velo_cmd {
    uint32_t opcode;
    uint32_t flags;
    union {
        struct { void* d_out; const void* d_in; const int64_t* d_indices; size_t n; uint32_t type; } permute;
        struct { const uint8_t* d_mask; size_t n; int32_t* d_out_indices; uint64_t* d_count; void* d_scratch;
                 size_t scratch_bytes; } scatter;
        struct { void* d_out; const void* d_in; const int32_t* d_indices; const uint8_t* d_mask; size_t n;
                 uint32_t type; } gather;
        struct { void* const* d_cols; const uint32_t* types; const uint8_t* ascending; uint32_t n_cols; size_t n;
                 size_t capacity; int64_t* d_indices; void* d_scratch; size_t scratch_bytes; } sort;
        struct { const void* d_left; const void* d_right; uint8_t* d_out_mask; size_t n; uint32_t type; } compare_eq;
        struct { const uint32_t* d_old; const uint32_t* d_sigma; uint32_t* d_new; size_t n; } compose;
        struct { const uint32_t* d_record_ids; const uint32_t* d_map; uint32_t* d_out; size_t n; } enrich;
        struct { uint64_t* d_keys; uint32_t* d_payload; size_t n; size_t capacity; } osort_kp;
        struct { uint64_t* d_keys; uint32_t* d_payload; uint8_t* d_marks; size_t n; size_t capacity;
                 uint64_t* d_count; void* d_scratch; size_t scratch_bytes; } ocompact_kpm;
        struct { uint64_t* const* d_words; uint32_t n_words; uint64_t key_mask; size_t n; size_t capacity; }
            osort_records;
        struct { const void* d_build_keys; const uint8_t* d_build_mask; size_t build_n; const void* d_probe_keys;
                 const uint8_t* d_probe_mask; size_t probe_n; uint32_t key_type; int64_t* d_out_build_rowid;
                 int64_t* d_out_probe_rowid; uint64_t* d_counts; void* d_scratch; size_t scratch_bytes; } ojoin;
        struct { const void* d_build_keys; const uint8_t* d_build_mask; size_t build_n; const void* d_probe_keys;
                 const uint8_t* d_probe_mask; size_t probe_n; uint32_t key_type; size_t max_pairs;
                 int64_t* d_out_build_rowid; int64_t* d_out_probe_rowid; uint64_t* d_counts; void* d_scratch;
                 size_t scratch_bytes; } ojoin_mn;
        struct { const void* d_build_keys; const uint8_t* d_build_mask; size_t build_n; const void* d_probe_keys;
                 const uint8_t* d_probe_mask; size_t probe_n; uint32_t key_type; uint64_t hash_seed;
                 int64_t* d_out_build_rowid; int64_t* d_out_probe_rowid; uint64_t* d_counts; void* d_scratch;
                 size_t scratch_bytes; } ohash;
        struct { const uint64_t* d_table; size_t table_n; const uint32_t* d_rids; size_t n_req; uint64_t* d_out;
                 void* d_scratch; size_t scratch_bytes; } ogather;
        struct { uint32_t* d_map; size_t n; uint64_t key; uint64_t counter; void* d_scratch; size_t scratch_bytes; }
            oshuffle;
        struct { const velo_lineitem* cols; size_t n; const velo_lineitem_pred* pred; uint32_t group_bound;
                 int64_t* d_out; uint64_t* d_counts; void* d_scratch; size_t scratch_bytes; } filter_groupby;
        struct { const velo_join_tables* tables; const velo_join_pred* pred; uint32_t k; int64_t* d_out;
                 uint64_t* d_counts; void* d_scratch; size_t scratch_bytes; } join_topk;
    } args;
} velo_cmd;

typedef struct velo_ctx velo_ctx;

/* velo_config.flags */
#define VELO_QUEUE_PERSISTENT 1u /* commands run on a persistent device-side consumer */

/* velo_cmd.flags: with VELO_QUEUE_PERSISTENT, the command need not wait for
 * the commands submitted before it (it may run beside them) */
#define VELO_CMD_UNORDERED 0x100u

typedef struct velo_config {
    int32_t device;          /* CUDA device ordinal */
    uint32_t queue_capacity; /* tickets in flight before submit waits (0 = 1024) */
    uint32_t flags;          /* VELO_QUEUE_PERSISTENT or 0 */
    uint32_t idle_us;        /* persistent consumer: idle time before it exits (0 = 1000 us) */
} velo_config;

/* Creates a context on `device` (replaces TaskManager::start,
 * src/cuda/task_manager.cu:26-78).
 *
 * Default: a non-blocking stream and a ring of completion events; each
 * command is dispatched to its kernels on the stream; nothing runs while the
 * queue is empty.
 *
 * VELO_QUEUE_PERSISTENT: like the reference, a persistent kernel consumes
 * the commands from a host-mapped ring (src/cuda/persistent_kernel.cu:76-124),
 * but every command is planned on the host into a job of tile-sized work
 * items, and several jobs run at once: the consumer's CTAs claim items of
 * all published jobs in publication order, each item waiting (bounded) only
 * for the earlier steps of its own job.  Commands keep submission order
 * unless they carry VELO_CMD_UNORDERED; a velo_batch_submit batch runs
 * unordered among itself.  The consumer exits after idle_us without work and
 * is relaunched by the next submission or wait; while it runs it holds the
 * SMs, so work on other streams shares the GPU with it.  The queue is not
 * ordered after work on other streams: a command's inputs (and buffers that
 * other streams fill) must be complete before it is submitted.  Opcodes:
 * NOP, PERMUTE, SCATTER, GATHER, COMPARE_EQ, COMPOSE_POSITION_MAP,
 * ENRICH_POSITIONS, OSORT_KP, OCOMPACT_KPM, OSHUFFLE, OJOIN_PKFK, OGATHER,
 * FILTER_GROUPBY, JOIN_GROUPBY_TOPK; the others return VELO_ENOTSUP. */
velo_status velo_init(const velo_config* config, velo_ctx** out);
/* Waits up to timeout_ms for outstanding commands, then releases the
 * context.  Never resets the device (the reference calls cudaDeviceReset on
 * timeout, src/cuda/task_manager.cu:110-119).  VELO_ETIMEDOUT if commands
 * were still running (the context is released anyway). */
velo_status velo_shutdown(velo_ctx* ctx, uint32_t timeout_ms);
/* Enqueues one command; *ticket identifies its completion.  Thread-safe
 * (the reference's push is single-producer, src/cuda/commands.cpp:47-67). */
velo_status velo_submit(velo_ctx* ctx, const velo_cmd* cmd, uint64_t* ticket);
/* Enqueues n commands.  Stream queue: the VELO_OP_OSORT_KP /
 * VELO_OP_OCOMPACT_KPM commands among them run as ONE persistent batched
 * launch (velo_batch_*), the others in order after it, and tickets[i]
 * completes with the whole submission.  Persistent queue: every command is a
 * job of its own, the batch's jobs run beside each other after the commands
 * submitted before the batch, and tickets[i] completes with command i. */
velo_status velo_batch_submit(velo_ctx* ctx, const velo_cmd* cmds, size_t n, uint64_t* tickets);
/* Waits for a ticket, at most timeout_ns (VELO_ETIMEDOUT instead of
 * spinning forever, cf. src/cuda/commands.cpp:69-91). */
velo_status velo_wait(velo_ctx* ctx, uint64_t ticket, uint64_t timeout_ns);
/* Copies the context's last error text into buf (always NUL-terminated). */
velo_status velo_last_error(velo_ctx* ctx, char* buf, size_t len);
/* The context's stream (a cudaStream_t) for callers that interleave their
 * own work. */
void* velo_ctx_stream(velo_ctx* ctx);
/* sizeof(velo_cmd), for bindings that lay out command arrays themselves. */
size_t velo_cmd_size(void);
/* Launches of a persistent context's consumer kernel so far (the first one
 * and every relaunch after an idle exit); 0 for a stream context.  No
 * reference counterpart (the reference's kernel never exits). */
uint64_t velo_ctx_launches(velo_ctx* ctx);

/* ------------------------------------------------------------------------ */
/* Serving layer: continuous admission of queries over resident tables      */
/* ------------------------------------------------------------------------ */

/* Device-resident tables the server's queries read (owned by the caller,
 * resident for the server's lifetime). */
typedef struct velo_served_tables {
    velo_lineitem fact;         /* lineitem-shaped columns of the fact table */
    const int64_t* fact_fk;     /* fact -> dimension key */
    const int32_t* fact_fk32;   /* the same keys as int32 (two-way join query) */
    size_t fact_n;
    const int64_t* dim_key;     /* unique dimension keys */
    const int32_t* dim_key32;   /* the same keys as int32 */
    const int32_t* dim_date;
    size_t dim_n;
    const int64_t* fact2_fk;    /* second fact table -> fact row id */
    const int64_t* fact2_price;
    size_t fact2_n;
} velo_served_tables;

/* Query shapes: filter + group-by over a fact slice (config-1 shape);
 * dimension slice JOIN fact slice + group-by + top-10 (config-2 shape);
 * three-way chain dimension <- fact <- second fact, returning the number of
 * joined rows and the sum of the second fact table's price. */
#define VELO_Q_FILTER_GROUPBY 1u
#define VELO_Q_JOIN_TOPK 2u
#define VELO_Q_JOIN3 3u

typedef struct velo_query {
    uint32_t shape;
    uint32_t pad_;
    size_t offset, n;         /* fact slice (public size) */
    size_t dim_offset, dim_n; /* dimension slice (joins) */
    size_t f2_offset, f2_n;   /* second fact slice (VELO_Q_JOIN3) */
    velo_lineitem_pred pred;  /* VELO_Q_FILTER_GROUPBY */
    velo_join_pred jpred;     /* joins */
} velo_query;

typedef struct velo_query_result {
    uint64_t qid;
    int32_t status;
    uint32_t shape;
    double submit_ms, start_ms, end_ms; /* host clock, ms since server start */
    int64_t out[96]; /* FILTER_GROUPBY: 8 x 6 as velo_filter_groupby; JOIN_TOPK: 10 x 3 as
                        velo_join_groupby_topk; JOIN3: out[0] = sum of second-fact price */
    uint64_t counts[2];
} velo_query_result;

/* velo_server_config.flags */
#define VELO_SERVE_PERSISTENT 1u /* queries run as jobs of one persistent command queue */

typedef struct velo_server_config {
    int32_t device;
    uint32_t slots;            /* queries on the device at once (one stream or job each), 1..64 */
    uint64_t hbm_budget_bytes; /* arena for all in-flight queries' scratch, allocated once */
    uint32_t flags;            /* VELO_SERVE_PERSISTENT or 0 (per-slot streams) */
    uint32_t idle_us;          /* persistent queue: idle time before its consumer exits (0 = 1000 us) */
} velo_server_config;

typedef struct velo_server_stats_t {
    uint64_t admitted, completed, pending, peak_inflight, arena_bytes, peak_arena_bytes;
} velo_server_stats_t;

typedef struct velo_server velo_server;

/* Starts the request loop.  Queries are admitted in arrival order whenever a
 * slot is free and their scratch fits in the budget; admitted queries run
 * concurrently on their own streams, or with VELO_SERVE_PERSISTENT as jobs
 * of one persistent command queue (see velo_init), whose consumer runs the
 * work items of every admitted query as they become ready and copies each
 * result straight into host memory.  With slots = 1 the server runs one
 * query at a time (the plain path). */
velo_status velo_server_create(const velo_server_config* cfg, const velo_served_tables* tables, velo_server** out);
/* Thread-safe; returns immediately with the query id. */
velo_status velo_server_submit(velo_server* srv, const velo_query* q, uint64_t* qid);
/* Waits (bounded) for a query and collects its result (once per query). */
velo_status velo_server_wait(velo_server* srv, uint64_t qid, uint64_t timeout_ns, velo_query_result* out);
velo_status velo_server_stats(velo_server* srv, velo_server_stats_t* out);
/* Drains (bounded) and stops the loop; VELO_ETIMEDOUT leaves it running. */
velo_status velo_server_destroy(velo_server* srv, uint32_t timeout_ms);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* VELO_OBL_H */
