/*
 * CPU oracle for the oblivious operator path -- TEST INFRASTRUCTURE ONLY.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load this
 * library; the product never does.  See oracle.h for the contract of each
 * function and the reference file:line it restates.
 */
#include "oracle.h"

#include <float.h>
#include <limits.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static int pick_threads(int n_threads)
{
#ifdef _OPENMP
    return n_threads > 0 ? n_threads : omp_get_max_threads();
#else
    (void)n_threads;
    return 1;
#endif
}

/* reference include/cuda/helper.hpp:50-62 */
size_t orc_next_pow2(size_t x)
{
    if (x <= 1)
        return 1;
    x--;
    x |= x >> 1;
    x |= x >> 2;
    x |= x >> 4;
    x |= x >> 8;
    x |= x >> 16;
    x |= x >> 32;
    return x + 1;
}

/* ------------------------------------------------------------------------ */
/* Generic multi-column bitonic sort: reference include/cuda/sort.cuh:11-118 */
/* ------------------------------------------------------------------------ */

#define ORC_CMP(T)                                                                                                     \
    {                                                                                                                  \
        const T* d = (const T*)p;                                                                                      \
        T a = d[i], b = d[j];                                                                                          \
        if (a == b)                                                                                                    \
            return 0;                                                                                                  \
        return (a < b) ? -1 : 1;                                                                                       \
    }

/* compareSingle, sort.cuh:11-29: equal -> 0, less -> -1, otherwise 1 (a NaN
 * operand therefore compares as "greater", exactly as the reference). */
static int cmp_single(const void* p, int type, size_t i, size_t j)
{
    switch (type) {
    case ORC_BOOLEAN:
        ORC_CMP(uint8_t)
    case ORC_TINYINT:
        ORC_CMP(int8_t)
    case ORC_SMALLINT:
        ORC_CMP(int16_t)
    case ORC_INTEGER:
        ORC_CMP(int32_t)
    case ORC_BIGINT:
        ORC_CMP(int64_t)
    case ORC_FLOAT:
        ORC_CMP(float)
    case ORC_DOUBLE:
        ORC_CMP(double)
    case ORC_VARCHAR:
        ORC_CMP(uint64_t)
    case ORC_DATE:
        ORC_CMP(uint32_t)
    default:
        return 0;
    }
}

static size_t type_size(int type)
{
    switch (type) {
    case ORC_BOOLEAN:
    case ORC_TINYINT:
        return 1;
    case ORC_SMALLINT:
        return 2;
    case ORC_INTEGER:
    case ORC_FLOAT:
    case ORC_DATE:
        return 4;
    case ORC_BIGINT:
    case ORC_DOUBLE:
    case ORC_VARCHAR:
        return 8;
    default:
        return 0;
    }
}

/* Pad value: numeric_limits<DT>::max() for ascending, lowest() for
 * descending columns (sort.cuh:79-100). */
static void fill_pad(void* p, int type, int asc, size_t i)
{
    switch (type) {
    case ORC_BOOLEAN:
        ((uint8_t*)p)[i] = asc ? UINT8_MAX : 0;
        break;
    case ORC_TINYINT:
        ((int8_t*)p)[i] = asc ? INT8_MAX : INT8_MIN;
        break;
    case ORC_SMALLINT:
        ((int16_t*)p)[i] = asc ? INT16_MAX : INT16_MIN;
        break;
    case ORC_INTEGER:
        ((int32_t*)p)[i] = asc ? INT32_MAX : INT32_MIN;
        break;
    case ORC_BIGINT:
        ((int64_t*)p)[i] = asc ? INT64_MAX : INT64_MIN;
        break;
    case ORC_FLOAT:
        ((float*)p)[i] = asc ? FLT_MAX : -FLT_MAX;
        break;
    case ORC_DOUBLE:
        ((double*)p)[i] = asc ? DBL_MAX : -DBL_MAX;
        break;
    case ORC_VARCHAR:
        ((uint64_t*)p)[i] = asc ? UINT64_MAX : 0;
        break;
    case ORC_DATE:
        ((uint32_t*)p)[i] = asc ? UINT32_MAX : 0;
        break;
    default:
        break;
    }
}

static void swap_bytes(void* p, size_t sz, size_t i, size_t j)
{
    uint8_t* a = (uint8_t*)p + i * sz;
    uint8_t* b = (uint8_t*)p + j * sz;
    for (size_t t = 0; t < sz; t++) {
        uint8_t x = a[t];
        a[t] = b[t];
        b[t] = x;
    }
}

int orc_bitonic_sort_cols(int n_cols, void* const* cols, const int* types, const uint8_t* ascending, size_t n,
                          size_t n_padded, int64_t* indices)
{
    for (int c = 0; c < n_cols; c++)
        if (type_size(types[c]) == 0)
            return -1;
    /* sort.cuh:79-100: indices and padding */
    for (size_t i = 0; i < n_padded; i++) {
        indices[i] = (int64_t)i;
        if (i >= n)
            for (int c = 0; c < n_cols; c++)
                fill_pad(cols[c], types[c], ascending[c], i);
    }
    /* sort.cuh:104-117: (k, j) stage loops; swap iff needSwap (sort.cuh:31-40) */
    for (size_t k = 2; k <= n_padded; k <<= 1) {
        for (size_t j = k >> 1; j > 0; j >>= 1) {
            for (size_t i = 0; i < n_padded; i++) {
                size_t ixj = i ^ j;
                if (i < ixj) {
                    int asc = ((i & k) == 0);
                    int swap = 0;
                    for (int c = 0; c < n_cols; c++) {
                        int cmp = cmp_single(cols[c], types[c], i, ixj);
                        if (cmp != 0) {
                            swap = (asc ^ (ascending[c] != 0)) ? (cmp < 0) : (cmp > 0);
                            break;
                        }
                    }
                    if (swap) {
                        int64_t t = indices[i];
                        indices[i] = indices[ixj];
                        indices[ixj] = t;
                        for (int c = 0; c < n_cols; c++)
                            swap_bytes(cols[c], type_size(types[c]), i, ixj);
                    }
                }
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Specialised network ports (same stage order, branchless exchanges)        */
/* ------------------------------------------------------------------------ */

static inline int ilog2_sz(size_t x)
{
    int l = -1;
    while (x) {
        l++;
        x >>= 1;
    }
    return l;
}

void orc_bitonic_kp(uint64_t* keys, uint32_t* pay, size_t n, size_t n_padded, int n_threads)
{
    for (size_t i = n; i < n_padded; i++) {
        keys[i] = UINT64_MAX;
        pay[i] = UINT32_MAX;
    }
    if (n_padded < 2)
        return;
    const size_t half = n_padded / 2;
    const int nt = pick_threads(n_threads);
#pragma omp parallel num_threads(nt) if (n_padded >= 4096)
    for (size_t k = 2; k <= n_padded; k <<= 1) {
        for (size_t j = k >> 1; j > 0; j >>= 1) {
            const int jb = ilog2_sz(j);
#pragma omp for schedule(static)
            for (size_t q = 0; q < half; q++) {
                /* q-th pair of the stage: insert a zero at bit jb */
                size_t i = ((q >> jb) << (jb + 1)) | (q & (j - 1));
                size_t l = i | j;
                uint64_t ka = keys[i], kb = keys[l];
                uint32_t pa = pay[i], pb = pay[l];
                int gt = (ka > kb) | ((ka == kb) & (pa > pb));
                int lt = (ka < kb) | ((ka == kb) & (pa < pb));
                int sw = ((i & k) == 0) ? gt : lt;
                uint64_t mk = (uint64_t)0 - (uint64_t)sw;
                uint32_t mp = (uint32_t)0 - (uint32_t)sw;
                uint64_t dk = (ka ^ kb) & mk;
                uint32_t dp = (pa ^ pb) & mp;
                keys[i] = ka ^ dk;
                keys[l] = kb ^ dk;
                pay[i] = pa ^ dp;
                pay[l] = pb ^ dp;
            }
        }
    }
}

void orc_bitonic_records(uint64_t* const* words, int n_words, int n_key_words, const uint64_t* masks,
                         const uint64_t* pad, size_t n, size_t n_padded, int n_threads)
{
    for (size_t i = n; i < n_padded; i++)
        for (int w = 0; w < n_words; w++)
            words[w][i] = pad[w];
    if (n_padded < 2)
        return;
    const size_t half = n_padded / 2;
    const int nt = pick_threads(n_threads);
#pragma omp parallel num_threads(nt) if (n_padded >= 4096)
    for (size_t k = 2; k <= n_padded; k <<= 1) {
        for (size_t j = k >> 1; j > 0; j >>= 1) {
            const int jb = ilog2_sz(j);
#pragma omp for schedule(static)
            for (size_t q = 0; q < half; q++) {
                size_t i = ((q >> jb) << (jb + 1)) | (q & (j - 1));
                size_t l = i | j;
                int cmp = 0;
                for (int w = 0; w < n_key_words && cmp == 0; w++) {
                    uint64_t a = words[w][i] & masks[w], b = words[w][l] & masks[w];
                    cmp = (a > b) - (a < b);
                }
                int sw = ((i & k) == 0) ? (cmp > 0) : (cmp < 0);
                uint64_t m = (uint64_t)0 - (uint64_t)sw;
                for (int w = 0; w < n_words; w++) {
                    uint64_t a = words[w][i], b = words[w][l];
                    uint64_t d = (a ^ b) & m;
                    words[w][i] = a ^ d;
                    words[w][l] = b ^ d;
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* ORCompact: liboblivious algorithms.c:116-213                              */
/* ------------------------------------------------------------------------ */

struct oc_ctx {
    uint8_t* data;
    size_t esz;
    uint8_t* marks;
};

/* o_memswap semantics: swap the two elements (and their marks) iff cond. */
static inline void oc_swap(struct oc_ctx* c, size_t a, size_t b, int cond)
{
    uint8_t m = (uint8_t)(0 - (cond != 0));
    uint8_t* pa = c->data + a * c->esz;
    uint8_t* pb = c->data + b * c->esz;
    for (size_t t = 0; t < c->esz; t++) {
        uint8_t d = (pa[t] ^ pb[t]) & m;
        pa[t] ^= d;
        pb[t] ^= d;
    }
    uint8_t d = (c->marks[a] ^ c->marks[b]) & m;
    c->marks[a] ^= d;
    c->marks[b] ^= d;
}

static inline int oc_marked(const struct oc_ctx* c, size_t i)
{
    return c->marks[i] != 0;
}

/* compact_offset, algorithms.c:118-153 */
static void oc_compact_offset(struct oc_ctx* c, size_t start, size_t n, size_t offset)
{
    if (n < 2)
        return;
    if (n == 2) {
        int l = oc_marked(c, start), r = oc_marked(c, start + 1);
        oc_swap(c, start, start + 1, ((!l) & r) != (offset % 2 == 1));
        return;
    }
    size_t half = n / 2;
    size_t left_marked = 0;
    for (size_t i = 0; i < half; i++)
        left_marked += (size_t)oc_marked(c, start + i);
    oc_compact_offset(c, start, half, offset % half);
    oc_compact_offset(c, start + half, half, (offset + left_marked) % half);
    int s = ((offset % half) + left_marked >= half) != (offset >= half);
    for (size_t i = 0; i < half; i++)
        oc_swap(c, start + i, start + i + half, s != (i >= (offset + left_marked) % half));
}

/* o_compact_generate_swaps, algorithms.c:155-181 */
static void oc_generate(struct oc_ctx* c, size_t n)
{
    if (n < 2)
        return;
    size_t right = (size_t)1 << ilog2_sz(n);
    size_t left = n - right;
    size_t left_marked = 0;
    for (size_t i = 0; i < left; i++)
        left_marked += (size_t)oc_marked(c, i);
    oc_generate(c, left);
    oc_compact_offset(c, left, right, (right - left + left_marked) % right);
    for (size_t i = 0; i < left; i++)
        oc_swap(c, i, i + right, i >= left_marked);
}

size_t orc_ocompact(uint8_t* data, size_t n, size_t elem_size, uint8_t* marks)
{
    size_t count = 0;
    for (size_t i = 0; i < n; i++)
        count += (marks[i] != 0);
    struct oc_ctx c = { data, elem_size, marks };
    oc_generate(&c, n);
    return count;
}

/* ------------------------------------------------------------------------ */
/* Stable scatter (reference scatter.cuh:16-81 with one block's ordering)    */
/* ------------------------------------------------------------------------ */

size_t orc_scatter_stable(const uint8_t* mask, size_t n, int32_t* out_idx)
{
    size_t cnt = 0;
    for (size_t i = 0; i < n; i++)
        if (mask[i])
            out_idx[i] = (int32_t)cnt++;
    return cnt;
}

/* ------------------------------------------------------------------------ */
/* Group-by: scalable_oblivious_join.c:221-232 (sums) and :262 (compaction)  */
/* ------------------------------------------------------------------------ */

size_t orc_groupby_sorted(const uint64_t* keys, const int64_t* vals, size_t n, int n_vals, uint64_t* out_keys,
                          int64_t* out_sums)
{
    if (n == 0)
        return 0;
    int64_t* sum = (int64_t*)malloc(n * (size_t)n_vals * sizeof(int64_t));
    uint8_t* cb = (uint8_t*)malloc(n);
    for (int v = 0; v < n_vals; v++)
        sum[v] = vals[v];
    cb[0] = 1;
    for (size_t i = 1; i < n; i++) {
        int cond = keys[i] == keys[i - 1];
        for (int v = 0; v < n_vals; v++)
            sum[i * n_vals + v] = cond * sum[(i - 1) * n_vals + v] + vals[i * n_vals + v];
        cb[i] = !cond;
    }
    for (size_t ii = n - 1; ii-- > 0;) {
        int cond = keys[ii] == keys[ii + 1];
        for (int v = 0; v < n_vals; v++)
            sum[ii * n_vals + v] = cond * sum[(ii + 1) * n_vals + v] + (!cond) * sum[ii * n_vals + v];
    }
    size_t g = 0;
    for (size_t i = 0; i < n; i++) {
        if (cb[i]) {
            out_keys[g] = keys[i];
            for (int v = 0; v < n_vals; v++)
                out_sums[g * n_vals + v] = sum[i * n_vals + v];
            g++;
        }
    }
    free(sum);
    free(cb);
    return g;
}

/* ------------------------------------------------------------------------ */
/* Pipelines                                                                 */
/* ------------------------------------------------------------------------ */

size_t orc_filter_groupby(size_t n, const int32_t* qty, const int64_t* price, const int32_t* disc,
                          const int32_t* tax, const int32_t* shipdate, const uint8_t* flag1, const uint8_t* flag2,
                          int32_t ship_lo, int32_t ship_hi, int32_t disc_lo, int32_t disc_hi, int32_t qty_lo,
                          int32_t qty_hi, size_t max_groups, uint64_t* out_keys, int64_t* out_sums, int n_threads)
{
    /* predicate -> mask, then stable compaction of the kept row ids */
    uint8_t* mask = (uint8_t*)malloc(n ? n : 1);
    for (size_t i = 0; i < n; i++)
        mask[i] = (shipdate[i] >= ship_lo) & (shipdate[i] <= ship_hi) & (disc[i] >= disc_lo) & (disc[i] <= disc_hi)
            & (qty[i] >= qty_lo) & (qty[i] <= qty_hi);
    int32_t* idx = (int32_t*)malloc((n ? n : 1) * sizeof(int32_t));
    size_t cnt = orc_scatter_stable(mask, n, idx);
    uint32_t* kept = (uint32_t*)malloc((cnt ? cnt : 1) * sizeof(uint32_t));
    for (size_t i = 0; i < n; i++)
        if (mask[i])
            kept[idx[i]] = (uint32_t)i;
    /* bitonic sort of (group key, row id) by group key */
    size_t np = orc_next_pow2(cnt);
    uint64_t* w0 = (uint64_t*)malloc(np * sizeof(uint64_t));
    uint64_t* w1 = (uint64_t*)malloc(np * sizeof(uint64_t));
    for (size_t r = 0; r < cnt; r++) {
        uint32_t i = kept[r];
        w0[r] = ((uint64_t)flag1[i] << 8) | flag2[i];
        w1[r] = i;
    }
    uint64_t* words[2] = { w0, w1 };
    uint64_t masks[1] = { UINT64_MAX };
    uint64_t pad[2] = { UINT64_MAX, UINT64_MAX };
    orc_bitonic_records(words, 2, 1, masks, pad, cnt, np, n_threads);
    int64_t* vals = (int64_t*)malloc((cnt ? cnt : 1) * 5 * sizeof(int64_t));
    for (size_t r = 0; r < cnt; r++) {
        size_t i = (size_t)w1[r];
        int64_t p = price[i];
        int64_t dp = p * (100 - disc[i]);
        vals[r * 5 + 0] = 1;
        vals[r * 5 + 1] = qty[i];
        vals[r * 5 + 2] = p;
        vals[r * 5 + 3] = dp;
        vals[r * 5 + 4] = dp * (100 + tax[i]);
    }
    uint64_t* gk = (uint64_t*)malloc((cnt ? cnt : 1) * sizeof(uint64_t));
    int64_t* gs = (int64_t*)malloc((cnt ? cnt : 1) * 5 * sizeof(int64_t));
    size_t g = orc_groupby_sorted(w0, vals, cnt, 5, gk, gs);
    for (size_t r = 0; r < g && r < max_groups; r++) {
        out_keys[r] = gk[r];
        memcpy(out_sums + r * 5, gs + r * 5, 5 * sizeof(int64_t));
    }
    free(mask);
    free(idx);
    free(kept);
    free(w0);
    free(w1);
    free(vals);
    free(gk);
    free(gs);
    return g;
}

size_t orc_join_groupby_topk(size_t n_dim, const int32_t* dim_key, const int32_t* dim_date, size_t n_fact,
                             const int32_t* fact_fk, const int64_t* fact_price, int32_t date_hi, int64_t price_hi,
                             size_t k, int32_t* out_fk, int64_t* out_sum, int64_t* out_cnt, int n_threads)
{
    /* union rows: w0 = [key ^ sign : 32][tag : 1][valid : 1][0 : 30], w1 = price */
    size_t n = n_dim + n_fact;
    size_t np = orc_next_pow2(n);
    uint64_t* w0 = (uint64_t*)malloc(np * sizeof(uint64_t));
    uint64_t* w1 = (uint64_t*)malloc(np * sizeof(uint64_t));
    for (size_t i = 0; i < n_dim; i++) {
        uint64_t key = (uint32_t)dim_key[i] ^ 0x80000000u;
        w0[i] = (key << 32) | ((uint64_t)(dim_date[i] < date_hi) << 30);
        w1[i] = 0;
    }
    for (size_t j = 0; j < n_fact; j++) {
        uint64_t key = (uint32_t)fact_fk[j] ^ 0x80000000u;
        w0[n_dim + j] = (key << 32) | (1ull << 31) | ((uint64_t)(fact_price[j] < price_hi) << 30);
        w1[n_dim + j] = (uint64_t)fact_price[j];
    }
    uint64_t* words[2] = { w0, w1 };
    uint64_t masks[1] = { 0xFFFFFFFF80000000ull };
    uint64_t pad[2] = { UINT64_MAX, UINT64_MAX };
    orc_bitonic_records(words, 2, 1, masks, pad, n, np, n_threads);
    /* forward fill of the dimension side's validity, then stable compaction
     * of the joined fact rows (still in key order) */
    uint64_t* jk = (uint64_t*)malloc((n_fact ? n_fact : 1) * sizeof(uint64_t));
    int64_t* jv = (int64_t*)malloc((n_fact ? n_fact : 1) * 2 * sizeof(int64_t));
    size_t nj = 0;
    uint64_t cur_key = UINT64_MAX;
    int cur_valid = 0;
    for (size_t i = 0; i < n; i++) {
        uint64_t key = w0[i] >> 32;
        int tag = (int)((w0[i] >> 31) & 1);
        int valid = (int)((w0[i] >> 30) & 1);
        if (!tag) {
            cur_key = key;
            cur_valid = valid;
        } else if (key == cur_key && cur_valid && valid) {
            jk[nj] = key;
            jv[nj * 2 + 0] = (int64_t)w1[i];
            jv[nj * 2 + 1] = 1;
            nj++;
        }
    }
    /* group-by fk (input already in fk order) */
    uint64_t* gk = (uint64_t*)malloc((nj ? nj : 1) * sizeof(uint64_t));
    int64_t* gs = (int64_t*)malloc((nj ? nj : 1) * 2 * sizeof(int64_t));
    size_t g = orc_groupby_sorted(jk, jv, nj, 2, gk, gs);
    /* sort groups by (sum desc, fk asc): w0 = ~(sum ^ sign), w1 = key, w2 = count */
    size_t gp = orc_next_pow2(g);
    uint64_t* s0 = (uint64_t*)malloc(gp * sizeof(uint64_t));
    uint64_t* s1 = (uint64_t*)malloc(gp * sizeof(uint64_t));
    uint64_t* s2 = (uint64_t*)malloc(gp * sizeof(uint64_t));
    for (size_t r = 0; r < g; r++) {
        s0[r] = ~((uint64_t)gs[r * 2] ^ 0x8000000000000000ull);
        s1[r] = gk[r];
        s2[r] = (uint64_t)gs[r * 2 + 1];
    }
    uint64_t* sw[3] = { s0, s1, s2 };
    uint64_t m2[2] = { UINT64_MAX, UINT64_MAX };
    uint64_t p3[3] = { UINT64_MAX, UINT64_MAX, UINT64_MAX };
    orc_bitonic_records(sw, 3, 2, m2, p3, g, gp, n_threads);
    for (size_t r = 0; r < k && r < g; r++) {
        out_fk[r] = (int32_t)((uint32_t)s1[r] ^ 0x80000000u);
        out_sum[r] = (int64_t)(~s0[r] ^ 0x8000000000000000ull);
        out_cnt[r] = (int64_t)s2[r];
    }
    free(w0);
    free(w1);
    free(jk);
    free(jv);
    free(gk);
    free(gs);
    free(s0);
    free(s1);
    free(s2);
    return g;
}

/* ------------------------------------------------------------------------ */
/* Sort-merge equi-join: reference include/cuda/sort_merge_join.cuh:63-199    */
/* ------------------------------------------------------------------------ */

typedef struct {
    int64_t key;
    int64_t rowid;
} orc_kr;

static int kr_cmp(const void* a, const void* b)
{
    const orc_kr* x = (const orc_kr*)a;
    const orc_kr* y = (const orc_kr*)b;
    if (x->key != y->key)
        return x->key < y->key ? -1 : 1;
    return (x->rowid > y->rowid) - (x->rowid < y->rowid);
}

static size_t kr_side(const int64_t* keys, const uint8_t* mask, size_t n, orc_kr** out)
{
    orc_kr* s = (orc_kr*)malloc((n ? n : 1) * sizeof(orc_kr));
    size_t m = 0;
    for (size_t i = 0; i < n; i++)
        if (!mask || mask[i]) {
            s[m].key = keys[i];
            s[m].rowid = (int64_t)i;
            m++;
        }
    qsort(s, m, sizeof(orc_kr), kr_cmp);
    *out = s;
    return m;
}

size_t orc_smj_pairs(const int64_t* lkeys, const uint8_t* lmask, size_t nl, const int64_t* rkeys,
                     const uint8_t* rmask, size_t nr, int64_t* out_l, int64_t* out_r, size_t cap)
{
    orc_kr *L, *R;
    const size_t ln = kr_side(lkeys, lmask, nl, &L);
    const size_t rn = kr_side(rkeys, rmask, nr, &R);
    /* mergeBlockCount (:61-101) with one block over the whole left side, then
     * writeJoinResults (:136-150): left-major, right-minor per key block */
    size_t l = 0, r = 0, total = 0;
    while (l < ln && r < rn) {
        if (L[l].key < R[r].key) {
            l++;
        } else if (L[l].key > R[r].key) {
            r++;
        } else {
            const int64_t key = L[l].key;
            const size_t l0 = l, r0 = r;
            while (l < ln && L[l].key == key)
                l++;
            while (r < rn && R[r].key == key)
                r++;
            for (size_t a = l0; a < l; a++)
                for (size_t b = r0; b < r; b++) {
                    if (total < cap) {
                        out_l[total] = L[a].rowid;
                        out_r[total] = R[b].rowid;
                    }
                    total++;
                }
        }
    }
    free(L);
    free(R);
    return total;
}
