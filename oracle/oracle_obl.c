/*
 * Oblivious CPU pipelines -- TEST INFRASTRUCTURE ONLY (the timed CPU
 * baseline).  Only bench.py's CPU legs and tests/ load this code; the
 * product never does.
 *
 * These are the CPU counterparts of the device pipelines, step for step and
 * with no data-dependent branch, address or size:
 *   - the bitonic network of the reference sort (include/cuda/sort.cuh:70-118:
 *     k ascending, j descending, partner i ^ j, direction (i & k) == 0), run
 *     over all next_pow2(n) rows.  Levels with j below a cache block are run
 *     block by block: every compare-exchange still sees the same operands as
 *     in the stage-by-stage order, because such levels never cross a block;
 *   - ORCompact as liboblivious computes it
 *     (obliviator/operator_1/third_party/liboblivious/algorithms.c:116-153),
 *     with the left-half mark counts read from one prefix count of the input
 *     marks (a half's elements are only permuted within it before the count
 *     is used) and the two halves of each level run as parallel tasks;
 *   - the segmented group sums of
 *     obliviator/operator_2/enclave/scalable_oblivious_join.c:221-262 as a
 *     chunked segmented scan, each group total added into the output slot of
 *     its rank by masked adds over every slot.
 * Records are 16-byte (two u64 words) structures so that a compare-exchange
 * moves one cache-friendly record.  All threads: OpenMP over n_threads.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    uint64_t w[2];
} rec2;

static int obl_threads(int n_threads)
{
#ifdef _OPENMP
    return n_threads > 0 ? n_threads : omp_get_max_threads();
#else
    (void)n_threads;
    return 1;
#endif
}

static size_t obl_next_pow2(size_t x)
{
    size_t p = 1;
    while (p < x)
        p <<= 1;
    return p;
}

/* ------------------------------------------------------------------------ */
/* bitonic network over 16-byte records                                      */
/* ------------------------------------------------------------------------ */

/* 1 if (a.w0 & m0, a.w1 & m1) > (b.w0 & m0, b.w1 & m1) lexicographically */
static inline uint64_t rec_gt(const rec2* a, const rec2* b, uint64_t m0, uint64_t m1)
{
    const uint64_t a0 = a->w[0] & m0, b0 = b->w[0] & m0, a1 = a->w[1] & m1, b1 = b->w[1] & m1;
    return (uint64_t)((a0 > b0) | ((a0 == b0) & (a1 > b1)));
}

/* strict compare-exchange (no exchange of equal keys, sort.cuh:31-40) */
static inline void rec_cx(rec2* r, size_t i, size_t l, int asc, uint64_t m0, uint64_t m1)
{
    const uint64_t gt = rec_gt(&r[i], &r[l], m0, m1), lt = rec_gt(&r[l], &r[i], m0, m1);
    const uint64_t sw = asc ? gt : lt;
    const uint64_t m = (uint64_t)0 - sw;
    const uint64_t d0 = (r[i].w[0] ^ r[l].w[0]) & m, d1 = (r[i].w[1] ^ r[l].w[1]) & m;
    r[i].w[0] ^= d0;
    r[l].w[0] ^= d0;
    r[i].w[1] ^= d1;
    r[l].w[1] ^= d1;
}

static inline size_t pair_lo(size_t q, size_t j, int jb)
{
    return ((q >> jb) << (jb + 1)) | (q & (j - 1));
}

static inline int log2_exact(size_t x)
{
    int l = 0;
    while (((size_t)1 << l) < x)
        l++;
    return l;
}

/* levels j = jtop .. 1 of phase k inside block [b, b + B) */
static void block_levels(rec2* r, size_t b, size_t B, size_t k, size_t jtop, uint64_t m0, uint64_t m1)
{
    for (size_t j = jtop; j > 0; j >>= 1) {
        const int jb = log2_exact(j);
        for (size_t q = 0; q < B / 2; q++) {
            const size_t i = b + pair_lo(q, j, jb);
            rec_cx(r, i, i | j, (i & k) == 0, m0, m1);
        }
    }
}

#define OBL_BLOCK ((size_t)1 << 14) /* 16 Ki records = 256 KB: stays in L2 */

void orc_obl_sort_rec2(void* recs, size_t np, uint64_t m0, uint64_t m1, int n_threads)
{
    rec2* r = (rec2*)recs;
    if (np < 2)
        return;
    const size_t B = np < OBL_BLOCK ? np : OBL_BLOCK;
    const int nt = obl_threads(n_threads);
#pragma omp parallel num_threads(nt)
    {
        /* phases k <= B: whole phases inside each block */
#pragma omp for schedule(static)
        for (size_t b = 0; b < np; b += B)
            for (size_t k = 2; k <= B; k <<= 1)
                block_levels(r, b, B, k, k >> 1, m0, m1);
        for (size_t k = 2 * B; k <= np; k <<= 1) {
            for (size_t j = k >> 1; j >= B; j >>= 1) {
                const int jb = log2_exact(j);
#pragma omp for schedule(static)
                for (size_t q = 0; q < np / 2; q++) {
                    const size_t i = pair_lo(q, j, jb);
                    rec_cx(r, i, i | j, (i & k) == 0, m0, m1);
                }
            }
#pragma omp for schedule(static)
            for (size_t b = 0; b < np; b += B)
                block_levels(r, b, B, k, B >> 1, m0, m1);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* ORCompact over 16-byte records, mark = bit `bit` of word `word` (xor inv)  */
/* ------------------------------------------------------------------------ */

typedef struct {
    rec2* r;
    const uint32_t* pre; /* pre[i] = marks among input rows [0, i) */
} oc2;

static inline void rec_swap_if(rec2* a, rec2* b, uint64_t cond)
{
    const uint64_t m = (uint64_t)0 - cond;
    const uint64_t d0 = (a->w[0] ^ b->w[0]) & m, d1 = (a->w[1] ^ b->w[1]) & m;
    a->w[0] ^= d0;
    b->w[0] ^= d0;
    a->w[1] ^= d1;
    b->w[1] ^= d1;
}

#define OC_TASK_MIN ((size_t)1 << 15)

/* compact_offset (algorithms.c:118-153) on rows [start, start + n) */
static void oc2_offset(const oc2* c, size_t start, size_t n, size_t offset, int word, int bit, int inv)
{
    if (n < 2)
        return;
    rec2* r = c->r;
    if (n == 2) {
        const uint64_t l = ((r[start].w[word] >> bit) & 1) ^ (uint64_t)inv;
        const uint64_t rr = ((r[start + 1].w[word] >> bit) & 1) ^ (uint64_t)inv;
        rec_swap_if(&r[start], &r[start + 1], (uint64_t)(((!l) & rr) != (offset % 2 == 1)));
        return;
    }
    const size_t half = n / 2;
    const size_t lm = (size_t)(c->pre[start + half] - c->pre[start]);
    if (half >= OC_TASK_MIN) {
#pragma omp task
        oc2_offset(c, start, half, offset % half, word, bit, inv);
#pragma omp task
        oc2_offset(c, start + half, half, (offset + lm) % half, word, bit, inv);
#pragma omp taskwait
    } else {
        oc2_offset(c, start, half, offset % half, word, bit, inv);
        oc2_offset(c, start + half, half, (offset + lm) % half, word, bit, inv);
    }
    const uint64_t s = ((offset % half) + lm >= half) != (offset >= half);
    const size_t thr = (offset + lm) % half;
    if (half >= OC_TASK_MIN) {
#pragma omp taskloop grainsize(8192)
        for (size_t i = 0; i < half; i++)
            rec_swap_if(&r[start + i], &r[start + i + half], s != (uint64_t)(i >= thr));
    } else {
        for (size_t i = 0; i < half; i++)
            rec_swap_if(&r[start + i], &r[start + i + half], s != (uint64_t)(i >= thr));
    }
}

/* exclusive prefix count of the marks of rows [0, np) into pre[0..np] */
static uint64_t mark_prefix(const rec2* r, size_t np, int word, int bit, int inv, uint32_t* pre, int nt)
{
    const int chunks = nt * 4;
    uint32_t* part = (uint32_t*)calloc((size_t)chunks + 1, sizeof(uint32_t));
    const size_t csz = (np + (size_t)chunks - 1) / (size_t)chunks;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int c = 0; c < chunks; c++) {
        uint32_t s = 0;
        const size_t e = (size_t)(c + 1) * csz < np ? (size_t)(c + 1) * csz : np;
        for (size_t i = (size_t)c * csz; i < e; i++)
            s += (uint32_t)(((r[i].w[word] >> bit) & 1) ^ (uint64_t)inv);
        part[c + 1] = s;
    }
    for (int c = 0; c < chunks; c++)
        part[c + 1] += part[c];
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int c = 0; c < chunks; c++) {
        uint32_t s = part[c];
        const size_t e = (size_t)(c + 1) * csz < np ? (size_t)(c + 1) * csz : np;
        for (size_t i = (size_t)c * csz; i < e; i++) {
            pre[i] = s;
            s += (uint32_t)(((r[i].w[word] >> bit) & 1) ^ (uint64_t)inv);
        }
    }
    pre[np] = part[chunks];
    const uint64_t total = part[chunks];
    free(part);
    return total;
}

size_t orc_obl_compact_rec2(void* recs, size_t np, int word, int bit, int inv, int n_threads)
{
    rec2* r = (rec2*)recs;
    const int nt = obl_threads(n_threads);
    uint32_t* pre = (uint32_t*)malloc((np + 1) * sizeof(uint32_t));
    const size_t count = (size_t)mark_prefix(r, np, word, bit, inv, pre, nt);
    oc2 c = { r, pre };
#pragma omp parallel num_threads(nt)
#pragma omp single
    oc2_offset(&c, 0, np, 0, word, bit, inv);
    free(pre);
    return count;
}

/* ------------------------------------------------------------------------ */
/* chunked segmented sums over key runs, group totals into ranked slots      */
/* ------------------------------------------------------------------------ */

#define SEG_MAXV 5

/* key, validity and values of row i */
typedef void (*seg_row_fn)(const rec2* r, size_t i, uint64_t* key, uint64_t* valid, int64_t* v, const void* prm);

typedef struct {
    uint64_t head_key, tail_key;
    int64_t tail_run[SEG_MAXV]; /* sums of the chunk's trailing key run */
    uint64_t uniform;           /* the chunk is one key run */
    uint64_t tails;             /* valid groups ending inside the chunk */
} seg_chunk;

/* For each valid group (run of equal keys whose last row is valid), in key
 * order, out_keys[rank] = key and out_vals[rank * V + v] = the run's sums, for
 * ranks < slots; other slots stay zero.  Every row adds into every slot.
 * Returns the number of groups. */
static size_t seg_groups(const rec2* r, size_t np, int V, seg_row_fn row, const void* prm, size_t slots,
                         uint64_t* out_keys, int64_t* out_vals, int nt)
{
    const int chunks = nt * 4;
    const size_t csz = (np + (size_t)chunks - 1) / (size_t)chunks;
    seg_chunk* ch = (seg_chunk*)calloc((size_t)chunks, sizeof(seg_chunk));
    int64_t* carry = (int64_t*)calloc((size_t)chunks * SEG_MAXV, sizeof(int64_t));
    uint64_t* rank0 = (uint64_t*)calloc((size_t)chunks, sizeof(uint64_t));
    uint64_t* tkeys = (uint64_t*)calloc((size_t)chunks * slots, sizeof(uint64_t));
    int64_t* tvals = (int64_t*)calloc((size_t)chunks * slots * (size_t)V, sizeof(int64_t));
    /* A: per chunk, its trailing run and the groups ending inside it */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int c = 0; c < chunks; c++) {
        const size_t b = (size_t)c * csz, e = b + csz < np ? b + csz : np;
        int64_t run[SEG_MAXV] = { 0 };
        uint64_t prev = 0, tails = 0, uniform = 1, k = 0, ok = 0;
        for (size_t i = b; i < e; i++) {
            int64_t v[SEG_MAXV];
            row(r, i, &k, &ok, v, prm);
            const uint64_t starts = (i == b) | (k != prev);
            uniform &= (i == b) | (k == prev);
            for (int x = 0; x < V; x++)
                run[x] = (starts ? 0 : run[x]) + v[x];
            if (i + 1 < e) {
                uint64_t kn, okn;
                int64_t vn[SEG_MAXV];
                row(r, i + 1, &kn, &okn, vn, prm);
                tails += (kn != k) & ok;
            }
            if (i == b)
                ch[c].head_key = k;
            prev = k;
        }
        ch[c].tail_key = prev;
        ch[c].uniform = uniform;
        ch[c].tails = tails;
        for (int x = 0; x < V; x++)
            ch[c].tail_run[x] = run[x];
        /* the chunk's last row ends a group when the next chunk starts
         * another key; decided in B */
        (void)ok;
    }
    /* B: carries between chunks and the first group rank of each chunk */
    {
        int64_t cur[SEG_MAXV] = { 0 };
        uint64_t rank = 0;
        for (int c = 0; c < chunks; c++) {
            const size_t b = (size_t)c * csz;
            if (b >= np)
                break;
            for (int x = 0; x < V; x++)
                carry[(size_t)c * SEG_MAXV + x] = (c > 0 && ch[c - 1].tail_key == ch[c].head_key) ? cur[x] : 0;
            rank0[c] = rank;
            /* trailing run of this chunk including what flows into it */
            for (int x = 0; x < V; x++)
                cur[x] = ch[c].tail_run[x] + (ch[c].uniform ? carry[(size_t)c * SEG_MAXV + x] : 0);
            /* does the last row of this chunk end a valid group? */
            const size_t e = b + csz < np ? b + csz : np;
            uint64_t k, ok;
            int64_t v[SEG_MAXV];
            row(r, e - 1, &k, &ok, v, prm);
            const uint64_t next_head = (c + 1 < chunks && e < np) ? ch[c + 1].head_key : ~k;
            rank += ch[c].tails + ((next_head != k) & ok);
        }
        (void)cur;
    }
    /* C: in-chunk scan with the carry; masked adds of group totals into slots */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int c = 0; c < chunks; c++) {
        const size_t b = (size_t)c * csz, e = b + csz < np ? b + csz : np;
        if (b >= np)
            continue;
        int64_t run[SEG_MAXV];
        for (int x = 0; x < V; x++)
            run[x] = carry[(size_t)c * SEG_MAXV + x];
        uint64_t rank = rank0[c], prev = ch[c].head_key;
        uint64_t* sk = tkeys + (size_t)c * slots;
        int64_t* sv = tvals + (size_t)c * slots * (size_t)V;
        for (size_t i = b; i < e; i++) {
            uint64_t k, ok, kn, okn;
            int64_t v[SEG_MAXV], vn[SEG_MAXV];
            row(r, i, &k, &ok, v, prm);
            const uint64_t starts = (i != b) & (k != prev);
            for (int x = 0; x < V; x++)
                run[x] = (starts ? 0 : run[x]) + v[x];
            const int has_next = i + 1 < np;
            row(r, has_next ? i + 1 : i, &kn, &okn, vn, prm);
            const uint64_t tail = ((!has_next) | (kn != k)) & ok;
            for (size_t s = 0; s < slots; s++) {
                const uint64_t m = (uint64_t)0 - (tail & (rank == s));
                sk[s] |= k & m;
                for (int x = 0; x < V; x++)
                    sv[s * (size_t)V + (size_t)x] += run[x] & (int64_t)m;
            }
            rank += tail;
            prev = k;
        }
    }
    /* D: slot sums over chunks */
    memset(out_keys, 0, slots * sizeof(uint64_t));
    memset(out_vals, 0, slots * (size_t)V * sizeof(int64_t));
    for (int c = 0; c < chunks; c++)
        for (size_t s = 0; s < slots; s++) {
            out_keys[s] |= tkeys[(size_t)c * slots + s];
            for (int x = 0; x < V; x++)
                out_vals[s * (size_t)V + (size_t)x] += tvals[((size_t)c * slots + s) * (size_t)V + (size_t)x];
        }
    size_t groups = 0;
    {
        /* total group count: the rank after the last chunk */
        uint64_t rank = 0;
        for (int c = 0; c < chunks; c++) {
            const size_t b = (size_t)c * csz;
            if (b >= np)
                break;
            const size_t e = b + csz < np ? b + csz : np;
            uint64_t k, ok;
            int64_t v[SEG_MAXV];
            row(r, e - 1, &k, &ok, v, prm);
            const uint64_t next_head = (c + 1 < chunks && e < np) ? ch[c + 1].head_key : ~k;
            rank += ch[c].tails + ((next_head != k) & ok);
        }
        groups = (size_t)rank;
    }
    free(ch);
    free(carry);
    free(rank0);
    free(tkeys);
    free(tvals);
    return groups;
}

/* ------------------------------------------------------------------------ */
/* filter + group-by                                                         */
/* ------------------------------------------------------------------------ */

/* record: w0 = [63] row fails the predicate | [40..47] flag1 | [32..39] flag2
 *         | [16..31] qty | [8..15] disc | [0..7] tax;  w1 = price */
#define FG_FAIL (1ull << 63)
#define FG_KEY_MASK 0xFFFFFFFF00000000ull

static void fg_row(const rec2* r, size_t i, uint64_t* key, uint64_t* valid, int64_t* v, const void* prm)
{
    (void)prm;
    const uint64_t w0 = r[i].w[0];
    const uint64_t ok = (w0 >> 63) ^ 1;
    const int64_t m = (int64_t)((uint64_t)0 - ok);
    const int64_t qty = (int64_t)((w0 >> 16) & 0xFFFF), disc = (int64_t)((w0 >> 8) & 0xFF),
                  tax = (int64_t)(w0 & 0xFF), price = (int64_t)r[i].w[1];
    const int64_t dp = price * (100 - disc);
    *key = w0 >> 32;
    *valid = ok;
    v[0] = 1 & m;
    v[1] = qty & m;
    v[2] = price & m;
    v[3] = dp & m;
    v[4] = (dp * (100 + tax)) & m;
}

size_t orc_obl_filter_groupby(size_t n, const int32_t* qty, const int64_t* price, const int32_t* disc,
                              const int32_t* tax, const int32_t* shipdate, const uint8_t* flag1,
                              const uint8_t* flag2, int32_t ship_lo, int32_t ship_hi, int32_t disc_lo,
                              int32_t disc_hi, int32_t qty_lo, int32_t qty_hi, size_t max_groups,
                              uint64_t* out_keys, int64_t* out_sums, int n_threads)
{
    const int nt = obl_threads(n_threads);
    const size_t np = obl_next_pow2(n ? n : 1);
    rec2* r = (rec2*)malloc(np * sizeof(rec2));
    /* predicate + pack; pads fail the predicate */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (size_t i = 0; i < np; i++) {
        if (i < n) {
            const uint64_t ok = (uint64_t)((shipdate[i] >= ship_lo) & (shipdate[i] <= ship_hi) & (disc[i] >= disc_lo)
                                           & (disc[i] <= disc_hi) & (qty[i] >= qty_lo) & (qty[i] <= qty_hi));
            r[i].w[0] = ((ok ^ 1) << 63) | ((uint64_t)flag1[i] << 40) | ((uint64_t)flag2[i] << 32)
                | ((uint64_t)(uint16_t)qty[i] << 16) | ((uint64_t)(uint8_t)disc[i] << 8) | (uint64_t)(uint8_t)tax[i];
            r[i].w[1] = (uint64_t)price[i];
        } else {
            r[i].w[0] = ~0ull;
            r[i].w[1] = ~0ull;
        }
    }
    /* oblivious compaction of the passing rows (mark = bit 63 clear) */
    orc_obl_compact_rec2(r, np, 0, 63, 1, nt);
    /* network sort of all next_pow2(n) rows on (fail, flag1, flag2) */
    orc_obl_sort_rec2(r, np, FG_KEY_MASK, 0, nt);
    /* segmented sums, group totals into max_groups slots */
    uint64_t* keys = (uint64_t*)malloc((max_groups ? max_groups : 1) * sizeof(uint64_t));
    const size_t g = seg_groups(r, np, 5, fg_row, NULL, max_groups, keys, out_sums, nt);
    for (size_t s = 0; s < max_groups; s++)
        out_keys[s] = ((keys[s] >> 8) & 0xFF) << 8 | (keys[s] & 0xFF);
    free(keys);
    free(r);
    return g;
}

/* ------------------------------------------------------------------------ */
/* PK-FK join + group-by + top-k                                             */
/* ------------------------------------------------------------------------ */

/* union record: w0 = [32..63] key ^ sign | [31] tag (0 dim, 1 fact)
 *               | [30] passes its side's filter | [29] joined;  w1 = price */
#define JN_TAG (1ull << 31)
#define JN_OK (1ull << 30)
#define JN_JOINED (1ull << 29)

static void jn_row(const rec2* r, size_t i, uint64_t* key, uint64_t* valid, int64_t* v, const void* prm)
{
    (void)prm;
    const uint64_t w0 = r[i].w[0];
    const uint64_t ok = (w0 >> 29) & 1;
    const int64_t m = (int64_t)((uint64_t)0 - ok);
    /* rows that did not join form runs of their own (validity is part of the
     * run key), so a left-over row after the joined ones never extends the
     * last group */
    *key = (w0 >> 32) | ((ok ^ 1) << 32);
    *valid = ok;
    v[0] = (int64_t)r[i].w[1] & m;
    v[1] = 1 & m;
}

/* group record: w0 = [63] not a group | [32..62] count | [0..31] key;
 * w1 = sum */

size_t orc_obl_join_groupby_topk(size_t n_dim, const int32_t* dim_key, const int32_t* dim_date, size_t n_fact,
                                 const int32_t* fact_fk, const int64_t* fact_price, int32_t date_hi,
                                 int64_t price_hi, size_t k, int32_t* out_fk, int64_t* out_sum, int64_t* out_cnt,
                                 int n_threads)
{
    const int nt = obl_threads(n_threads);
    const size_t n = n_dim + n_fact;
    const size_t np = obl_next_pow2(n ? n : 1);
    rec2* r = (rec2*)malloc(np * sizeof(rec2));
#pragma omp parallel for num_threads(nt) schedule(static)
    for (size_t i = 0; i < np; i++) {
        if (i < n_dim) {
            const uint64_t key = (uint32_t)dim_key[i] ^ 0x80000000u;
            r[i].w[0] = (key << 32) | ((uint64_t)(dim_date[i] < date_hi) << 30);
            r[i].w[1] = 0;
        } else if (i < n) {
            const size_t j = i - n_dim;
            const uint64_t key = (uint32_t)fact_fk[j] ^ 0x80000000u;
            r[i].w[0] = (key << 32) | JN_TAG | ((uint64_t)(fact_price[j] < price_hi) << 30);
            r[i].w[1] = (uint64_t)fact_price[j];
        } else {
            r[i].w[0] = ~0ull & ~JN_JOINED;
            r[i].w[1] = ~0ull;
        }
    }
    /* sort on (key, tag): each key's dimension row first */
    orc_obl_sort_rec2(r, np, 0xFFFFFFFF80000000ull, 0, nt);
    /* forward fill of the last dimension row's (key, filter) into the fact
     * rows: a chunked scan; joined = fact & fact ok & same key & dim ok */
    {
        const int chunks = nt * 4;
        const size_t csz = (np + (size_t)chunks - 1) / (size_t)chunks;
        uint64_t* last = (uint64_t*)malloc((size_t)chunks * sizeof(uint64_t)); /* last dim row's w0, or ~0 */
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int c = 0; c < chunks; c++) {
            const size_t b = (size_t)c * csz, e = b + csz < np ? b + csz : np;
            uint64_t cur = ~0ull;
            for (size_t i = b; i < e; i++) {
                const uint64_t dim = ((r[i].w[0] & JN_TAG) == 0) & (i < n);
                cur = dim ? r[i].w[0] : cur;
            }
            last[c] = cur;
        }
        uint64_t run = ~0ull;
        for (int c = 0; c < chunks; c++) {
            const uint64_t here = last[c];
            last[c] = run;
            run = here != ~0ull ? here : run;
        }
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int c = 0; c < chunks; c++) {
            const size_t b = (size_t)c * csz, e = b + csz < np ? b + csz : np;
            uint64_t cur = last[c];
            for (size_t i = b; i < e; i++) {
                const uint64_t w0 = r[i].w[0];
                const uint64_t dim = ((w0 & JN_TAG) == 0) & (i < n);
                cur = dim ? w0 : cur;
                const uint64_t joined = (!dim) & (i < n) & ((w0 >> 30) & 1) & ((cur >> 30) & 1)
                    & ((cur >> 32) == (w0 >> 32)) & (cur != ~0ull);
                r[i].w[0] = w0 | (joined << 29);
            }
        }
        free(last);
    }
    /* oblivious compaction of the joined fact rows (still in key order) */
    orc_obl_compact_rec2(r, np, 0, 29, 0, nt);
    /* segmented sums per fk; every row writes a group record, marked on the
     * last row of each valid run; ORCompact moves the groups to the front */
    rec2* g = (rec2*)malloc(np * sizeof(rec2));
    {
        const int chunks = nt * 4;
        const size_t csz = (np + (size_t)chunks - 1) / (size_t)chunks;
        /* reuse the slot machinery with zero slots for the carries only */
        seg_chunk* ch = (seg_chunk*)calloc((size_t)chunks, sizeof(seg_chunk));
        int64_t* carry = (int64_t*)calloc((size_t)chunks * 2, sizeof(int64_t));
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int c = 0; c < chunks; c++) {
            const size_t b = (size_t)c * csz, e = b + csz < np ? b + csz : np;
            int64_t run0 = 0, run1 = 0;
            uint64_t prev = 0, uniform = 1;
            for (size_t i = b; i < e; i++) {
                uint64_t kk, ok;
                int64_t v[SEG_MAXV];
                jn_row(r, i, &kk, &ok, v, NULL);
                const uint64_t starts = (i == b) | (kk != prev);
                uniform &= (i == b) | (kk == prev);
                run0 = (starts ? 0 : run0) + v[0];
                run1 = (starts ? 0 : run1) + v[1];
                if (i == b)
                    ch[c].head_key = kk;
                prev = kk;
            }
            ch[c].tail_key = prev;
            ch[c].uniform = uniform;
            ch[c].tail_run[0] = run0;
            ch[c].tail_run[1] = run1;
        }
        int64_t cur0 = 0, cur1 = 0;
        for (int c = 0; c < chunks; c++) {
            const int link = c > 0 && ch[c - 1].tail_key == ch[c].head_key;
            carry[c * 2 + 0] = link ? cur0 : 0;
            carry[c * 2 + 1] = link ? cur1 : 0;
            cur0 = ch[c].tail_run[0] + (ch[c].uniform ? carry[c * 2 + 0] : 0);
            cur1 = ch[c].tail_run[1] + (ch[c].uniform ? carry[c * 2 + 1] : 0);
        }
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int c = 0; c < chunks; c++) {
            const size_t b = (size_t)c * csz, e = b + csz < np ? b + csz : np;
            int64_t run0 = carry[c * 2 + 0], run1 = carry[c * 2 + 1];
            uint64_t prev = ch[c].head_key;
            for (size_t i = b; i < e; i++) {
                uint64_t kk, ok, kn, okn;
                int64_t v[SEG_MAXV], vn[SEG_MAXV];
                jn_row(r, i, &kk, &ok, v, NULL);
                const uint64_t starts = (i != b) & (kk != prev);
                run0 = (starts ? 0 : run0) + v[0];
                run1 = (starts ? 0 : run1) + v[1];
                const int has_next = i + 1 < np;
                jn_row(r, has_next ? i + 1 : i, &kn, &okn, vn, NULL);
                const uint64_t tail = ((!has_next) | (kn != kk)) & ok;
                g[i].w[0] = ((tail ^ 1) << 63) | (((uint64_t)run1 & 0x7FFFFFFF) << 32) | (kk & 0xFFFFFFFF);
                g[i].w[1] = (uint64_t)run0;
                prev = kk;
            }
        }
        free(ch);
        free(carry);
    }
    const size_t groups = orc_obl_compact_rec2(g, np, 0, 63, 1, nt);
    /* top-k: network sort of the first next_pow2(n_dim) group records on
     * (not a group, sum descending, fk ascending) */
    const size_t dp = obl_next_pow2(n_dim ? n_dim : 1) < np ? obl_next_pow2(n_dim ? n_dim : 1) : np;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (size_t i = 0; i < dp; i++) {
        const uint64_t w0 = g[i].w[0], sum = g[i].w[1];
        const uint64_t notg = w0 >> 63;
        g[i].w[0] = (notg << 63) | (~sum & 0x7FFFFFFFFFFFFFFFull);
        g[i].w[1] = ((w0 & 0xFFFFFFFF) << 32) | ((w0 >> 32) & 0x7FFFFFFF);
    }
    orc_obl_sort_rec2(g, dp, ~0ull, 0xFFFFFFFF00000000ull, nt);
    for (size_t i = 0; i < k; i++) {
        const size_t j = i < dp ? i : dp - 1;
        const uint64_t ok = (i < groups) & (i < dp);
        out_fk[i] = ok ? (int32_t)((uint32_t)(g[j].w[1] >> 32) ^ 0x80000000u) : 0;
        out_sum[i] = ok ? (int64_t)(~g[j].w[0] & 0x7FFFFFFFFFFFFFFFull) : 0;
        out_cnt[i] = ok ? (int64_t)(g[j].w[1] & 0xFFFFFFFF) : 0;
    }
    free(g);
    free(r);
    return groups;
}
