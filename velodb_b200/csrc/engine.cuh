// Tile engine for the oblivious networks (bitonic sort, ORCompact) on sm_100a.
//
// A CTA of NT = 2^LOG_NT threads owns a tile of T = 2^t rows (t = LOG_NT +
// LOG_E); every thread keeps E = 2^LOG_E rows in registers.  Which local row
// index a register holds is given by a *layout* s: register e of thread tid
// holds local row
//
//     l = (tid & (2^s - 1)) | (e << s) | ((tid >> s) << (s + LOG_E)),
//
// i.e. the E registers cover local bits [s, s + LOG_E).  A network level whose
// partner bit lies in that window is a register-local compare-exchange; other
// levels first re-layout the tile through shared memory ("transpose", one smem
// write + read of the tile).  Global loads/stores use a layout with s >= 5 so
// the 32 lanes of a warp touch 32 consecutive rows (fully coalesced).
//
// Every network step is data-independent: the same loads, stores and smem
// accesses happen for any data of the same public size, and exchanges are
// selects, never branches on data.
#pragma once

#include <cstddef>
#include <cstdint>

#include "velo_obl.h"

namespace velo {

// ---------------------------------------------------------------------------
// row types: SoA columns in global memory, SoA arrays in shared memory
// ---------------------------------------------------------------------------

template <class T>
__device__ __forceinline__ T sel(bool c, T a, T b)
{
    return c ? a : b;
}

// (u64 key, u32 payload), ordered lexicographically on both (plain sort rows).
struct RowKP {
    uint64_t k;
    uint32_t p;
    struct Cols {
        uint64_t* k;
        uint32_t* p;
    };
    static constexpr int SMEM_BYTES = 12;
    static constexpr bool FULL_KEY = true;
    __device__ __forceinline__ static RowKP load(const Cols& c, size_t g) { return RowKP { c.k[g], c.p[g] }; }
    __device__ __forceinline__ static void store(const Cols& c, size_t g, const RowKP& r)
    {
        c.k[g] = r.k;
        c.p[g] = r.p;
    }
    __device__ __forceinline__ static RowKP pad(const Cols&) { return RowKP { ~0ull, ~0u }; }
    __device__ __forceinline__ static void sstore(char* sm, int T, int i, const RowKP& r)
    {
        reinterpret_cast<uint64_t*>(sm)[i] = r.k;
        reinterpret_cast<uint32_t*>(sm + 8 * T)[i] = r.p;
    }
    __device__ __forceinline__ static RowKP sload(const char* sm, int T, int i)
    {
        return RowKP { reinterpret_cast<const uint64_t*>(sm)[i], reinterpret_cast<const uint32_t*>(sm + 8 * T)[i] };
    }
    // a > b in the row order
    __device__ __forceinline__ static bool gt(const RowKP& a, const RowKP& b, const Cols&)
    {
        return (a.k > b.k) | ((a.k == b.k) & (a.p > b.p));
    }
    __device__ __forceinline__ static RowKP select(bool c, const RowKP& a, const RowKP& b)
    {
        return RowKP { sel(c, a.k, b.k), sel(c, a.p, b.p) };
    }
    __device__ __forceinline__ static bool marked(const RowKP&) { return false; }
};

// (u64 key, u32 payload, u8 mark): compaction rows; the order compares
// (key, payload) so the same rows can also be sorted.
struct RowKPM {
    uint64_t k;
    uint32_t p;
    uint32_t m;
    struct Cols {
        uint64_t* k;
        uint32_t* p;
        uint8_t* m;
    };
    static constexpr int SMEM_BYTES = 13;
    static constexpr bool FULL_KEY = false;
    __device__ __forceinline__ static RowKPM load(const Cols& c, size_t g)
    {
        return RowKPM { c.k[g], c.p[g], (uint32_t)c.m[g] };
    }
    __device__ __forceinline__ static void store(const Cols& c, size_t g, const RowKPM& r)
    {
        c.k[g] = r.k;
        c.p[g] = r.p;
        c.m[g] = (uint8_t)r.m;
    }
    __device__ __forceinline__ static RowKPM pad(const Cols&) { return RowKPM { ~0ull, ~0u, 0u }; }
    __device__ __forceinline__ static void sstore(char* sm, int T, int i, const RowKPM& r)
    {
        reinterpret_cast<uint64_t*>(sm)[i] = r.k;
        reinterpret_cast<uint32_t*>(sm + 8 * T)[i] = r.p;
        reinterpret_cast<uint8_t*>(sm + 12 * T)[i] = (uint8_t)r.m;
    }
    __device__ __forceinline__ static RowKPM sload(const char* sm, int T, int i)
    {
        return RowKPM { reinterpret_cast<const uint64_t*>(sm)[i], reinterpret_cast<const uint32_t*>(sm + 8 * T)[i],
                        (uint32_t) reinterpret_cast<const uint8_t*>(sm + 12 * T)[i] };
    }
    __device__ __forceinline__ static bool gt(const RowKPM& a, const RowKPM& b, const Cols&)
    {
        return (a.k > b.k) | ((a.k == b.k) & (a.p > b.p));
    }
    __device__ __forceinline__ static RowKPM select(bool c, const RowKPM& a, const RowKPM& b)
    {
        return RowKPM { sel(c, a.k, b.k), sel(c, a.p, b.p), sel(c, a.m, b.m) };
    }
    __device__ __forceinline__ static bool marked(const RowKPM& r) { return r.m != 0; }
};

// W u64 words per row (SoA).  Ordered lexicographically on the first KW words,
// each AND-ed with a mask; the mark (for compaction) is bit `mark_bit` of word
// 0, inverted when mark_inv is set (so an "invalid" flag can sort last).
template <int W, int KW>
struct RowRec {
    uint64_t w[W];
    struct Cols {
        uint64_t* w[W];
        uint64_t mask[KW];
        uint64_t pad[W];
        int mark_bit;
        int mark_inv;
    };
    static constexpr int SMEM_BYTES = 8 * W;
    static constexpr bool FULL_KEY = false;
    __device__ __forceinline__ static RowRec load(const Cols& c, size_t g)
    {
        RowRec r;
#pragma unroll
        for (int i = 0; i < W; i++)
            r.w[i] = c.w[i][g];
        return r;
    }
    __device__ __forceinline__ static void store(const Cols& c, size_t g, const RowRec& r)
    {
#pragma unroll
        for (int i = 0; i < W; i++)
            c.w[i][g] = r.w[i];
    }
    __device__ __forceinline__ static RowRec pad(const Cols& c)
    {
        RowRec r;
#pragma unroll
        for (int i = 0; i < W; i++)
            r.w[i] = c.pad[i];
        return r;
    }
    __device__ __forceinline__ static void sstore(char* sm, int T, int i, const RowRec& r)
    {
#pragma unroll
        for (int x = 0; x < W; x++)
            reinterpret_cast<uint64_t*>(sm + (size_t)8 * T * x)[i] = r.w[x];
    }
    __device__ __forceinline__ static RowRec sload(const char* sm, int T, int i)
    {
        RowRec r;
#pragma unroll
        for (int x = 0; x < W; x++)
            r.w[x] = reinterpret_cast<const uint64_t*>(sm + (size_t)8 * T * x)[i];
        return r;
    }
    __device__ __forceinline__ static bool gt(const RowRec& a, const RowRec& b, const Cols& c)
    {
        bool res = false, eq = true;
#pragma unroll
        for (int x = 0; x < KW; x++) {
            uint64_t aa = a.w[x] & c.mask[x], bb = b.w[x] & c.mask[x];
            res = res | (eq & (aa > bb));
            eq = eq & (aa == bb);
        }
        return res;
    }
    __device__ __forceinline__ static RowRec select(bool cnd, const RowRec& a, const RowRec& b)
    {
        RowRec r;
#pragma unroll
        for (int x = 0; x < W; x++)
            r.w[x] = sel(cnd, a.w[x], b.w[x]);
        return r;
    }
    __device__ __forceinline__ static bool marked_c(const RowRec& r, const Cols& c)
    {
        return (((r.w[0] >> c.mark_bit) & 1ull) != 0) != (c.mark_inv != 0);
    }
};

template <class R>
struct MarkOf {
    __device__ __forceinline__ static bool get(const R& r, const typename R::Cols&) { return R::marked(r); }
};
template <int W, int KW>
struct MarkOf<RowRec<W, KW>> {
    __device__ __forceinline__ static bool get(const RowRec<W, KW>& r, const typename RowRec<W, KW>::Cols& c)
    {
        return RowRec<W, KW>::marked_c(r, c);
    }
};

// ---------------------------------------------------------------------------
// layouts
// ---------------------------------------------------------------------------

template <int LOG_NT, int LOG_E>
struct Tile {
    static constexpr int NT = 1 << LOG_NT;
    static constexpr int E = 1 << LOG_E;
    static constexpr int LOG_T = LOG_NT + LOG_E;
    static constexpr int T = 1 << LOG_T;
    static_assert(LOG_NT >= 5, "at least one warp per CTA");

    __device__ __forceinline__ static int local(int s, int e, int tid)
    {
        return (tid & ((1 << s) - 1)) | (e << s) | ((tid >> s) << (s + LOG_E));
    }
    // bank-spreading swizzle: XOR bits 5..9 into bits 0..4 (a bijection on
    // every aligned group of 1024 rows, so it stays inside the tile)
    __device__ __forceinline__ static int swz(int l) { return l ^ ((l >> 5) & 31); }

    template <class R>
    __device__ __forceinline__ static void transpose(R (&v)[E], int s_from, int s_to, char* sm)
    {
        const int tid = threadIdx.x;
        __syncthreads();
#pragma unroll
        for (int e = 0; e < E; e++)
            R::sstore(sm, T, swz(local(s_from, e, tid)), v[e]);
        __syncthreads();
#pragma unroll
        for (int e = 0; e < E; e++)
            v[e] = R::sload(sm, T, swz(local(s_to, e, tid)));
    }
};

// window start that covers bit p, going down (bitonic) or up (ORCompact)
__device__ __forceinline__ int window_down(int p, int log_e, int log_t)
{
    int s = p - log_e + 1;
    s = s < 0 ? 0 : s;
    return s > log_t - log_e ? log_t - log_e : s;
}
__device__ __forceinline__ int window_up(int p, int log_e, int log_t)
{
    int s = p;
    return s > log_t - log_e ? log_t - log_e : s;
}

} // namespace velo
