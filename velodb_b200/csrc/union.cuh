// Building blocks of the union-sort operators (oblivious gather, joins):
// the forward fill over a key-sorted record array and the scratch layout of
// a union of 3-word records.  Included by the translation units that
// implement those operators.
#pragma once

#include "net_impl.cuh"

namespace velo {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), counter-based PRF used
// to draw the shuffle keys on the device
// ---------------------------------------------------------------------------

__host__ __device__ __forceinline__ void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo)
{
    const uint64_t p = (uint64_t)a * b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

__host__ __device__ __forceinline__ uint64_t philox_u64(uint64_t idx, uint64_t counter, uint64_t key)
{
    uint32_t c0 = (uint32_t)idx, c1 = (uint32_t)(idx >> 32), c2 = (uint32_t)counter, c3 = (uint32_t)(counter >> 32);
    uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
    for (int r = 0; r < 10; r++) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c0, hi0, lo0);
        mulhilo32(0xCD9E8D57u, c2, hi1, lo1);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return ((uint64_t)c1 << 32) | c0;
}

// ---------------------------------------------------------------------------
// forward fill over a key-sorted record array: every row receives the
// (key, value) of the last "source" row at or before it (segmented scan in
// three passes; addresses never depend on the data)
// ---------------------------------------------------------------------------

struct FillCarry {
    uint64_t key;
    uint64_t val;
    uint32_t has;
    uint32_t valid;
};

__device__ __forceinline__ FillCarry fill_combine(const FillCarry& l, const FillCarry& r)
{
    return r.has ? r : l;
}

constexpr int FL_TS = 2048, FL_THREADS = 256, FL_RPT = FL_TS / FL_THREADS;

__device__ __forceinline__ FillCarry fill_shfl(const FillCarry& c, int d, bool up)
{
    FillCarry r;
    const uint32_t hv = c.has | (c.valid << 1);
    const uint32_t x = up ? __shfl_up_sync(0xFFFFFFFFu, hv, d) : __shfl_xor_sync(0xFFFFFFFFu, hv, d);
    r.key = up ? __shfl_up_sync(0xFFFFFFFFu, c.key, d) : __shfl_xor_sync(0xFFFFFFFFu, c.key, d);
    r.val = up ? __shfl_up_sync(0xFFFFFFFFu, c.val, d) : __shfl_xor_sync(0xFFFFFFFFu, c.val, d);
    r.has = x & 1u;
    r.valid = (x >> 1) & 1u;
    return r;
}

// block-wide exclusive "last source row" scan (warp shuffles, then one
// shared-memory round over the warp totals); wsm holds 33 entries, the
// block total is left in wsm[32]
__device__ __forceinline__ FillCarry block_fill_scan_excl(const FillCarry& mine, FillCarry* wsm)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const FillCarry zero { 0, 0, 0, 0 };
    FillCarry inc = mine;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const FillCarry y = fill_shfl(inc, off, true);
        if (lane >= off)
            inc = fill_combine(y, inc);
    }
    __syncthreads(); // wsm may still be read by a previous call
    if (lane == 31)
        wsm[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        FillCarry z = lane < nw ? wsm[lane] : zero;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const FillCarry y = fill_shfl(z, off, true);
            if (lane >= off)
                z = fill_combine(y, z);
        }
        FillCarry ez = fill_shfl(z, 1, true);
        if (lane == 0)
            ez = zero;
        __syncwarp();
        if (lane < nw)
            wsm[lane] = ez;
        if (lane == nw - 1)
            wsm[32] = z;
    }
    __syncthreads();
    FillCarry ex = fill_shfl(inc, 1, true);
    if (lane == 0)
        ex = zero;
    return fill_combine(wsm[warp], ex);
}

// Src: static FillCarry src(w0, w1, w2) -- has = row is a source
//      static void apply(uint64_t& w0, uint64_t& w1, uint64_t& w2, const FillCarry& last)
// the last source row of fill tile `blk` (FL_THREADS threads); sm, idx:
// FL_THREADS / 32 entries of shared memory each
template <class F>
__device__ __forceinline__ void fill_sum_tile(const uint64_t* w0, const uint64_t* w1, const uint64_t* w2,
                                              FillCarry* tile_last, size_t blk, FillCarry* sm, int* idx)
{
    const size_t base = blk * FL_TS;
    FillCarry c { 0, 0, 0, 0 };
    int last = -1;
    for (int i = threadIdx.x; i < FL_TS; i += FL_THREADS) {
        const size_t g = base + i;
        VELO_TRACE_AT(TS_FILL, w0 + g);
        const FillCarry d = F::src(w0[g], w1[g], w2[g]);
        c = fill_combine(c, d);
        last = d.has ? i : last;
    }
    // the source row with the largest index: warp shuffles, then warp 0
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const FillCarry oc = fill_shfl(c, off, false);
        const int oi = __shfl_xor_sync(0xFFFFFFFFu, last, off);
        const bool take = oi > last;
        c = take ? oc : c;
        last = take ? oi : last;
    }
    if ((threadIdx.x & 31) == 0) {
        sm[threadIdx.x >> 5] = c;
        idx[threadIdx.x >> 5] = last;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        FillCarry b = sm[0];
        int bi = idx[0];
        for (int w = 1; w < FL_THREADS / 32; w++) {
            const bool take = idx[w] > bi;
            b = take ? sm[w] : b;
            bi = take ? idx[w] : bi;
        }
        VELO_TRACE_AT(TS_FILL, tile_last + blk);
        tile_last[blk] = b;
    }
}

// fill of tile `blk` from its carry; wsm: 33 entries, tmp: 33 words of shared
// memory
template <class F>
__device__ __forceinline__ void fill_apply_tile(uint64_t* w0, uint64_t* w1, uint64_t* w2, const FillCarry* carry,
                                                unsigned long long* d_stat, size_t blk, FillCarry* wsm, uint32_t* tmp)
{
    const size_t base = blk * FL_TS + (size_t)threadIdx.x * FL_RPT;
    uint64_t a[FL_RPT], b[FL_RPT], c[FL_RPT];
    FillCarry mine { 0, 0, 0, 0 };
#pragma unroll
    for (int r = 0; r < FL_RPT; r++) {
        VELO_TRACE_AT(TS_FILL, w0 + base + r);
        a[r] = w0[base + r];
        b[r] = w1[base + r];
        c[r] = w2[base + r];
        mine = fill_combine(mine, F::src(a[r], b[r], c[r]));
    }
    FillCarry run = fill_combine(carry[blk], block_fill_scan_excl(mine, wsm));
    uint32_t stat = 0;
#pragma unroll
    for (int r = 0; r < FL_RPT; r++) {
        stat += F::dup(a[r], b[r], c[r], run) ? 1u : 0u;
        run = fill_combine(run, F::src(a[r], b[r], c[r]));
        F::apply(a[r], b[r], c[r], run);
        VELO_TRACE_AT(TS_FILL, w0 + base + r);
        w0[base + r] = a[r];
        w1[base + r] = b[r];
        w2[base + r] = c[r];
    }
    // one counter update per CTA at a fixed address
    uint32_t total;
    block_exclusive_scan(stat, tmp, &total);
    if (threadIdx.x == 0 && d_stat)
        atomicAdd(d_stat, (unsigned long long)total);
}

template <class F>
__global__ void __launch_bounds__(FL_THREADS) k_fill_sum(const uint64_t* w0, const uint64_t* w1, const uint64_t* w2,
                                                         FillCarry* tile_last)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_fill_sum"));
    __shared__ FillCarry sm[FL_THREADS / 32];
    __shared__ int idx[FL_THREADS / 32];
    fill_sum_tile<F>(w0, w1, w2, tile_last, blockIdx.x, sm, idx);
}

// exclusive scan of the tile carries (one CTA of 1024 threads), defined in
// ops.cu
__global__ void k_fill_scan(const FillCarry* tile_last, int ntiles, FillCarry* carry);

template <class F>
__global__ void __launch_bounds__(FL_THREADS) k_fill_apply(uint64_t* w0, uint64_t* w1, uint64_t* w2,
                                                           const FillCarry* carry, unsigned long long* d_stat)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_fill_apply"));
    __shared__ FillCarry wsm[33];
    __shared__ uint32_t tmp[33];
    fill_apply_tile<F>(w0, w1, w2, carry, d_stat, blockIdx.x, wsm, tmp);
}

template <class F>
static velo_status run_fill(uint64_t* w0, uint64_t* w1, uint64_t* w2, size_t rows, FillCarry* tl, FillCarry* carry,
                            unsigned long long* d_stat, cudaStream_t st)
{
    const int nt = (int)(rows / FL_TS);
    k_fill_sum<F><<<nt, FL_THREADS, 0, st>>>(w0, w1, w2, tl);
    k_fill_scan<<<1, 1024, 0, st>>>(tl, nt, carry);
    k_fill_apply<F><<<nt, FL_THREADS, 0, st>>>(w0, w1, w2, carry, d_stat);
    VELO_CUDA_TRY(cudaGetLastError(), "fill launch");
    return VELO_OK;
}

using Rec3 = RowRec<3, 1, false>;
using Rec3K2 = RowRec<3, 2, false>;
constexpr int OP_LT = 12; // 4096-row tiles (CTA shape per record width: Tile12)
// up to 8 fused global levels: the 16 contiguous rows a segment keeps of
// each 8-byte word array fill a 128-byte line
constexpr int OP_LMAX = OP_LT - 4 < 8 ? OP_LT - 4 : 8;

// scratch of the union-sort operators: 3 words x rows + fill carries + compaction
inline size_t union_rows(size_t n)
{
    size_t r = next_pow2(n);
    const size_t floor_rows = (size_t)1 << OP_LT;
    return r < floor_rows ? floor_rows : r;
}

struct UnionScratch {
    uint64_t* w[3];
    FillCarry* tl;
    FillCarry* carry;
    uint32_t* counts;
    uint32_t* prefix;
    uint64_t* n_marked;
    unsigned long long* stat;
    size_t bytes;
};

inline UnionScratch union_layout(char* base, size_t rows)
{
    UnionScratch s {};
    size_t off = 0;
    auto take = [&](size_t b) {
        char* p = base ? base + off : nullptr;
        off += align_up(b, 256);
        return p;
    };
    for (int i = 0; i < 3; i++)
        s.w[i] = reinterpret_cast<uint64_t*>(take(rows * 8));
    // tile counts sized for 2^(OP_LT-1)-row tiles: the persistent command
    // queue compacts three-word records in 2048-row tiles
    const size_t nft = rows / FL_TS, nct = rows >> (OP_LT - 1);
    s.tl = reinterpret_cast<FillCarry*>(take(nft * sizeof(FillCarry)));
    s.carry = reinterpret_cast<FillCarry*>(take(nft * sizeof(FillCarry)));
    s.counts = reinterpret_cast<uint32_t*>(take(nct * 4));
    s.prefix = reinterpret_cast<uint32_t*>(take((nct + 1) * 4));
    s.n_marked = reinterpret_cast<uint64_t*>(take(8));
    s.stat = reinterpret_cast<unsigned long long*>(take(8));
    s.bytes = off;
    return s;
}

// Run counts over a key-sorted array (the scans of the joins): summary of a
// range of rows = first/last key, counted rows in it, counted rows in its
// trailing key run, whether it is one key run
struct RunSum {
    uint64_t first_key, last_key;
    uint64_t nb, tail_nb;
    uint32_t uniform, has;
};

// a then b (a the earlier range); associative
__device__ __forceinline__ RunSum run_combine(const RunSum& a, const RunSum& b)
{
    if (!a.has)
        return b;
    if (!b.has)
        return a;
    const bool join = a.last_key == b.first_key;
    RunSum r;
    r.first_key = a.first_key;
    r.last_key = b.last_key;
    r.nb = a.nb + b.nb;
    r.tail_nb = b.tail_nb + ((b.uniform && join) ? a.tail_nb : 0ull);
    r.uniform = (a.uniform && b.uniform && join) ? 1u : 0u;
    r.has = 1u;
    return r;
}

__device__ __forceinline__ RunSum run_row(uint64_t key, uint64_t counted)
{
    return RunSum { key, key, counted, counted, 1u, 1u };
}

// block-wide exclusive scan of RunSum (shared-memory Hillis-Steele over the
// threads' summaries); the block total is returned in *total
__device__ __forceinline__ RunSum run_block_scan_excl(const RunSum& mine, RunSum* sm, RunSum* total)
{
    const int t = threadIdx.x, n = blockDim.x;
    RunSum x = mine;
    for (int off = 1; off < n; off <<= 1) {
        __syncthreads();
        sm[t] = x;
        __syncthreads();
        if (t >= off)
            x = run_combine(sm[t - off], x);
    }
    __syncthreads();
    sm[t] = x;
    __syncthreads();
    *total = sm[n - 1];
    RunSum ex {};
    if (t > 0)
        ex = sm[t - 1];
    __syncthreads();
    return ex;
}

// exclusive scan of run summaries of tiles (one CTA of 1024 threads),
// defined in joins.cu
__global__ void k_run_scan(const RunSum* tiles, int ntiles, RunSum* carry);

} // namespace velo
