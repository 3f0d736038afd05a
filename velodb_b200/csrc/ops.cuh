// Device bodies of the column operators (reference command set and the
// oblivious union-sort operators), written for any CTA index: the plain path
// runs them as kernels over a grid (ops.cu), the persistent command queue as
// work items (dq_kernel.cu).
#pragma once

#include "union.cuh"

namespace velo {

// exclusive scan of the tile carries; one CTA, rounds of blockDim.x
// consecutive tiles chained through the running carry; wsm: 33 entries of
// shared memory
__device__ __forceinline__ void fill_scan_body(const FillCarry* tile_last, int ntiles, FillCarry* carry,
                                               FillCarry* wsm)
{
    FillCarry run { 0, 0, 0, 0 };
    for (int base = 0; base < ntiles; base += blockDim.x) {
        const int t = base + (int)threadIdx.x;
        FillCarry x { 0, 0, 0, 0 };
        if (t < ntiles) {
            VELO_TRACE_AT(TS_FILL, tile_last + t);
            x = tile_last[t];
        }
        const FillCarry ex = block_fill_scan_excl(x, wsm);
        if (t < ntiles)
            carry[t] = fill_combine(run, ex);
        run = fill_combine(run, wsm[32]);
    }
}

// grid stride over n elements for CTA `blk` of `nblk`
#define VELO_BLK_STRIDE(i, n, blk, nblk)                                                                               \
    for (size_t i = (size_t)(blk) * blockDim.x + threadIdx.x; VELO_GRID_COND(i, (n));                                \
         i += (size_t)(nblk) * blockDim.x)

// ---------------------------------------------------------------------------
// compat operators (include/cuda/permute.cuh:24-40, gather.cuh:28-45,
// scatter.cuh:16-81, compare.cuh:25-91, oblivious_shuffle.cuh:10-34)
// ---------------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ void permute_body(T* out, const T* in, const int64_t* idx, size_t n, size_t blk, size_t nblk)
{
    VELO_BLK_STRIDE(i, n, blk, nblk)
    out[i] = in[idx[i]];
}

template <typename T>
__device__ __forceinline__ void gather_body(T* out, const T* in, const int32_t* idx, const uint8_t* mask, size_t n, size_t blk, size_t nblk)
{
    VELO_BLK_STRIDE(i, n, blk, nblk)
    {
        if (mask == nullptr || mask[i] != 0)
            out[idx[i]] = in[i];
    }
}

template <typename T>
__device__ __forceinline__ void compare_eq_body(const T* l, const T* r, uint8_t* out, size_t n, size_t blk, size_t nblk)
{
    VELO_BLK_STRIDE(i, n, blk, nblk)
    out[i] = (l[i] == r[i]) ? 1 : 0;
}

__device__ __forceinline__ void fill_u8_body(uint8_t* out, uint8_t v, size_t n, size_t blk, size_t nblk)
{
    VELO_BLK_STRIDE(i, n, blk, nblk)
    out[i] = v;
}

__device__ __forceinline__ void compose_body(const uint32_t* old_map, const uint32_t* sigma, uint32_t* new_map, size_t n, size_t blk, size_t nblk)
{
    VELO_BLK_STRIDE(i, n, blk, nblk)
    new_map[i] = old_map[sigma[i]];
}

// stable scatter: per-tile kept counts, their scan, then ranks
constexpr int SC_LT = 11;
// tile `blk` of 2^SC_LT rows; tmp: 33 words of shared memory
__device__ __forceinline__ void scatter_count_tile(const uint8_t* mask, size_t n, uint32_t* counts, size_t blk,
                                                   uint32_t* tmp)
{
    const size_t base = blk << SC_LT;
    uint32_t c = 0;
    for (int i = threadIdx.x; i < (1 << SC_LT); i += blockDim.x) {
        const size_t g = base + i;
        c += (g < n && mask[g] != 0) ? 1u : 0u;
    }
    uint32_t total;
    block_exclusive_scan(c, tmp, &total);
    if (threadIdx.x == 0)
        counts[blk] = total;
}

// tile `blk` (256 threads); tmp: 33 words of shared memory
__device__ __forceinline__ void scatter_write_tile(const uint8_t* mask, size_t n, const uint32_t* prefix,
                                                   int32_t* out_idx, size_t blk, uint32_t* tmp)
{
    // each thread owns 8 consecutive rows of the 2048-row tile
    const size_t base = (blk << SC_LT) + (size_t)threadIdx.x * 8;
    uint32_t m[8], c = 0;
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const size_t g = base + r;
        m[r] = (g < n && mask[g] != 0) ? 1u : 0u;
        c += m[r];
    }
    uint32_t total;
    uint32_t rank = prefix[blk] + block_exclusive_scan(c, tmp, &total);
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const size_t g = base + r;
        if (m[r])
            out_idx[g] = (int32_t)rank;
        rank += m[r];
    }
}

__device__ __forceinline__ void shuffle_pack_body(const uint32_t* map, size_t n, size_t np, uint64_t counter,
                                                  uint64_t key, uint64_t* k, uint32_t* p, size_t blk, size_t nblk)
{
    VELO_BLK_STRIDE(i, np, blk, nblk)
    {
        k[i] = i < n ? philox_u64(i, counter, key) : ~0ull;
        p[i] = i < n ? map[i] : ~0u;
    }
}

__device__ __forceinline__ void copy_u32_body(uint32_t* dst, const uint32_t* src, size_t n, size_t blk, size_t nblk)
{
    VELO_BLK_STRIDE(i, n, blk, nblk)
    dst[i] = src[i];
}

// ---------------------------------------------------------------------------
// oblivious gather: out[j] = table[rid[j]]
// union row layout (3 words):
//   table row i : w0 = i << 32 | tag 0      w1 = table[i]   w2 = 0
//   request j   : w0 = rid << 32 | tag 1    w1 = 0          w2 = j
// sort 1 on (index, tag); fill gives each request the value of its table
// row; the requests' w0 becomes (0, j), every other row (1, ...); sort 2 on
// w0 puts the requests first in request order.
// ---------------------------------------------------------------------------

struct GatherFill {
    __device__ __forceinline__ static FillCarry src(uint64_t a, uint64_t b, uint64_t)
    {
        const bool table = ((a >> 31) & 1ull) == 0 && a != ~0ull;
        return FillCarry { a >> 32, b, table ? 1u : 0u, 1u };
    }
    __device__ __forceinline__ static bool dup(uint64_t, uint64_t, uint64_t, const FillCarry&) { return false; }
    __device__ __forceinline__ static void apply(uint64_t& a, uint64_t& b, uint64_t& c, const FillCarry& last)
    {
        const bool req = ((a >> 31) & 1ull) == 1 && a != ~0ull;
        const bool hit = req & (last.has != 0) & (last.key == (a >> 32));
        b = req ? (hit ? last.val : 0ull) : b;
        a = req ? (c & 0xFFFFFFFFull) : (1ull << 63);
    }
};

__device__ __forceinline__ void ogather_pack_body(const uint64_t* table, size_t tn, const uint32_t* rids, size_t rn,
                                                  size_t rows, uint64_t* w0, uint64_t* w1, uint64_t* w2, size_t blk,
                                                  size_t nblk)
{
    VELO_BLK_STRIDE(g, rows, blk, nblk)
    {
        uint64_t a = ~0ull, b = ~0ull, c = ~0ull;
        if (g < tn) {
            a = (uint64_t)g << 32;
            b = table[g];
            c = 0;
        } else if (g < tn + rn) {
            const size_t j = g - tn;
            a = ((uint64_t)rids[j] << 32) | (1ull << 31);
            b = 0;
            c = j;
        }
        w0[g] = a;
        w1[g] = b;
        w2[g] = c;
    }
}

__device__ __forceinline__ void ogather_out_body(const uint64_t* w1, size_t rn, uint64_t* out, size_t blk, size_t nblk)
{
    VELO_BLK_STRIDE(j, rn, blk, nblk)
    out[j] = w1[j];
}

// ---------------------------------------------------------------------------
// oblivious PK-FK join producing rowid pairs
// union row layout (3 words):
//   w0 = key (order-preserving u64)
//   w1 = [63] tag (0 build, 1 probe) | [62] row valid | [61] joined | [60:0] rowid
//   w2 = build rowid of a joined probe row
// ---------------------------------------------------------------------------

constexpr uint64_t OJ_TAG = 1ull << 63, OJ_VALID = 1ull << 62, OJ_JOINED = 1ull << 61;
constexpr uint64_t OJ_ROWID = (1ull << 61) - 1;

struct JoinFill {
    __device__ __forceinline__ static bool is_pad(uint64_t a, uint64_t b) { return a == ~0ull && b == ~0ull; }
    __device__ __forceinline__ static FillCarry src(uint64_t a, uint64_t b, uint64_t)
    {
        const bool build = (b & OJ_TAG) == 0 && !is_pad(a, b);
        return FillCarry { a, b & OJ_ROWID, build ? 1u : 0u, (b & OJ_VALID) ? 1u : 0u };
    }
    // a build row whose key equals the preceding build row's key
    __device__ __forceinline__ static bool dup(uint64_t a, uint64_t b, uint64_t, const FillCarry& last)
    {
        const bool build = (b & OJ_TAG) == 0 && !is_pad(a, b);
        return build & (last.has != 0) & (last.key == a);
    }
    __device__ __forceinline__ static void apply(uint64_t& a, uint64_t& b, uint64_t& c, const FillCarry& last)
    {
        const bool probe = (b & OJ_TAG) != 0 && !is_pad(a, b);
        const bool joined = probe & ((b & OJ_VALID) != 0) & (last.has != 0) & (last.valid != 0) & (last.key == a);
        b = (b & ~OJ_JOINED) | (joined ? OJ_JOINED : 0ull);
        c = joined ? last.val : ~0ull;
    }
};

__device__ __forceinline__ void ojoin_pack_body(const void* bk, const uint8_t* bm, size_t bn, const void* pk,
                                                const uint8_t* pm, size_t pn, int key64, size_t rows, uint64_t* w0,
                                                uint64_t* w1, uint64_t* w2, size_t blk, size_t nblk)
{
    VELO_BLK_STRIDE(g, rows, blk, nblk)
    {
        uint64_t a = ~0ull, b = ~0ull, c = ~0ull;
        if (g < bn + pn) {
            const bool build = g < bn;
            const size_t j = build ? g : g - bn;
            const void* keys = build ? bk : pk;
            const uint8_t* mask = build ? bm : pm;
            const uint64_t key = key64 ? ((uint64_t) static_cast<const int64_t*>(keys)[j] ^ 0x8000000000000000ull)
                                       : (uint64_t)((uint32_t) static_cast<const int32_t*>(keys)[j] ^ 0x80000000u);
            const bool valid = mask == nullptr || mask[j] != 0;
            a = key;
            b = (build ? 0ull : OJ_TAG) | (valid ? OJ_VALID : 0ull) | ((uint64_t)j & OJ_ROWID);
            c = ~0ull;
        }
        w0[g] = a;
        w1[g] = b;
        w2[g] = c;
    }
}

__device__ __forceinline__ void ojoin_out_body(const uint64_t* w1, const uint64_t* w2, size_t pn, int64_t* ob,
                                               int64_t* op, size_t blk, size_t nblk)
{
    VELO_BLK_STRIDE(i, pn, blk, nblk)
    {
        const uint64_t b = w1[i];
        const bool j = (b & OJ_JOINED) != 0 && b != ~0ull;
        ob[i] = j ? (int64_t)w2[i] : -1;
        op[i] = j ? (int64_t)(b & OJ_ROWID) : -1;
    }
}

// (build, probe) counts of a PK-FK join: joined probe rows, repeated build keys
__device__ __forceinline__ void join_counts_body(const uint64_t* n_joined, const unsigned long long* dups,
                                                 uint64_t* d_counts)
{
    d_counts[0] = *n_joined;
    d_counts[1] = *dups;
}

// ---- small column steps of the served three-way join chain -----------------

// m[i] = lo <= c[i] <= hi
template <class T>
__device__ __forceinline__ void range_mask_body(const T* c, size_t n, T lo, T hi, uint8_t* m, size_t blk, size_t nblk)
{
    VELO_BLK_STRIDE(i, n, blk, nblk)
    m[i] = (c[i] >= lo) & (c[i] <= hi);
}

// rowid of a joined row -> (global key = rowid + offset, mask); -1 -> invalid
__device__ __forceinline__ void rowid_keys_body(const int64_t* rowid, size_t n, int64_t offset, int64_t* key,
                                                uint8_t* m, size_t blk, size_t nblk)
{
    VELO_BLK_STRIDE(i, n, blk, nblk)
    {
        const int64_t r = rowid[i];
        key[i] = r >= 0 ? r + offset : -1;
        m[i] = r >= 0;
    }
}

// probe rowid -> u32 request id, -1 -> `missing` (an id past the table)
__device__ __forceinline__ void rowid_rids_body(const int64_t* rowid, size_t n, uint32_t missing, uint32_t* rid,
                                                size_t blk, size_t nblk)
{
    VELO_BLK_STRIDE(i, n, blk, nblk)
    {
        const int64_t r = rowid[i];
        rid[i] = r >= 0 ? (uint32_t)r : missing;
    }
}

// *out += the sum of CTA `blk`'s share of v (one add per CTA at a fixed
// address); s: 32 words of shared memory
__device__ __forceinline__ void sum_u64_body(const uint64_t* v, size_t n, unsigned long long* out, size_t blk,
                                             size_t nblk, unsigned long long* s)
{
    unsigned long long acc = 0;
    VELO_BLK_STRIDE(i, n, blk, nblk)
    acc += v[i];
    for (int o = 16; o > 0; o >>= 1)
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0)
        s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++)
            t += s[w];
        atomicAdd(out, t);
    }
    __syncthreads();
}

} // namespace velo
