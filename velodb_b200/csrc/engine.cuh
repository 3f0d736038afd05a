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
// Global loads use ld.global.cg (cached in L2 only): within one persistent
// launch a pass reads rows that other SMs wrote in the previous pass, so the
// non-coherent L1 must not serve them.
//
// Every network step is data-independent: the same loads, stores and smem
// accesses happen for any data of the same public size, and exchanges are
// selects, never branches on data.
#pragma once

#include <cstddef>
#include <cstdint>

#include "trace.cuh"
#include "velo_obl.h"

namespace velo {

// ---------------------------------------------------------------------------
// multi-limb unsigned comparison: 0xFFFFFFFF if x > y else 0, from the borrow
// of y - x (limb 0 least significant); one carry chain, no branches
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t gt_mask2(uint32_t x0, uint32_t x1, uint32_t y0, uint32_t y1)
{
    uint32_t r;
    asm("{\n\t.reg .u32 t;\n\t"
        "sub.cc.u32 t, %1, %3;\n\t"
        "subc.cc.u32 t, %2, %4;\n\t"
        "subc.u32 %0, 0, 0;\n\t}"
        : "=r"(r)
        : "r"(y0), "r"(y1), "r"(x0), "r"(x1));
    return r;
}

__device__ __forceinline__ uint32_t gt_mask3(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t y0, uint32_t y1,
                                             uint32_t y2)
{
    uint32_t r;
    asm("{\n\t.reg .u32 t;\n\t"
        "sub.cc.u32 t, %1, %4;\n\t"
        "subc.cc.u32 t, %2, %5;\n\t"
        "subc.cc.u32 t, %3, %6;\n\t"
        "subc.u32 %0, 0, 0;\n\t}"
        : "=r"(r)
        : "r"(y0), "r"(y1), "r"(y2), "r"(x0), "r"(x1), "r"(x2));
    return r;
}

__device__ __forceinline__ uint32_t gt_mask4(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3, uint32_t y0,
                                             uint32_t y1, uint32_t y2, uint32_t y3)
{
    uint32_t r;
    asm("{\n\t.reg .u32 t;\n\t"
        "sub.cc.u32 t, %1, %5;\n\t"
        "subc.cc.u32 t, %2, %6;\n\t"
        "subc.cc.u32 t, %3, %7;\n\t"
        "subc.cc.u32 t, %4, %8;\n\t"
        "subc.u32 %0, 0, 0;\n\t}"
        : "=r"(r)
        : "r"(y0), "r"(y1), "r"(y2), "r"(y3), "r"(x0), "r"(x1), "r"(x2), "r"(x3));
    return r;
}

__device__ __forceinline__ uint32_t lo32(uint64_t x) { return (uint32_t)x; }
__device__ __forceinline__ uint32_t hi32(uint64_t x) { return (uint32_t)(x >> 32); }

// 0xFFFFFFFF if the KW-word key x (word 0 most significant) exceeds y
template <int KW>
__device__ __forceinline__ uint32_t key_gt_mask(const uint64_t* x, const uint64_t* y)
{
    if constexpr (KW == 1) {
        return gt_mask2(lo32(x[0]), hi32(x[0]), lo32(y[0]), hi32(y[0]));
    } else if constexpr (KW == 2) {
        return gt_mask4(lo32(x[1]), hi32(x[1]), lo32(x[0]), hi32(x[0]), lo32(y[1]), hi32(y[1]), lo32(y[0]), hi32(y[0]));
    } else {
        // lexicographic from the most significant word
        bool res = false, eq = true;
#pragma unroll
        for (int i = 0; i < KW; i++) {
            res = res | (eq & (x[i] > y[i]));
            eq = eq & (x[i] == y[i]);
        }
        return res ? 0xFFFFFFFFu : 0u;
    }
}

// ---------------------------------------------------------------------------
// row types: SoA columns in global memory, SoA arrays in shared memory.
//
// swap_pred(a, b, desc) is the compare-exchange decision for the pair
// (a at the lower index, b): ascending swaps iff a > b, descending iff a < b.
// STRICT types follow the reference exactly on ties (include/cuda/sort.cuh:
// 31-40: no swap when equal).  Non-strict types are used where the
// arrangement of equal keys is invisible to the consumer (every field is
// compared, or the consumer aggregates over ties); they decide both
// directions with one comparison, swapping equal keys when descending,
// which still sorts.
// ---------------------------------------------------------------------------

template <class T>
__device__ __forceinline__ T sel(bool c, T a, T b)
{
    return c ? a : b;
}

// exchange a and b when x (selects, no branch)
__device__ __forceinline__ void xsel(bool x, uint32_t& a, uint32_t& b)
{
    const uint32_t na = x ? b : a, nb = x ? a : b;
    a = na;
    b = nb;
}

__device__ __forceinline__ void xsel(bool x, uint64_t& a, uint64_t& b)
{
    const uint64_t na = x ? b : a, nb = x ? a : b;
    a = na;
    b = nb;
}

// The same exchange on the integer multiply-add (FMA) pipe: with s = 1 to
// swap (mm = -s), d = b - a, a' = a + d*s, b' = b + d*mm, all mod 2^32.  The
// in-tile levels are bound by the integer ALU pipe (two selects a register);
// doing part of each row's registers here lets both pipes work.  `neg` is -1
// known only at run time, so the subtraction stays a multiply-add too.
struct MadSwap {
    uint32_t s, mm, neg;
    __device__ __forceinline__ explicit MadSwap(bool x)
    {
        neg = (uint32_t)(-(int)(blockDim.x != 0u));
        // an opaque copy: knowing mm is 0 or -1, the compiler would turn the
        // multiply-adds back into selects on the ALU pipe
        const uint32_t m0 = x ? 0xFFFFFFFFu : 0u;
        asm("mov.b32 %0, %1;" : "=r"(mm) : "r"(m0));
        s = mm * neg;
    }
    __device__ __forceinline__ void operator()(uint32_t& a, uint32_t& b) const
    {
        const uint32_t d = a * neg + b;
        a = d * s + a;
        b = d * mm + b;
    }
    __device__ __forceinline__ void operator()(uint64_t& a, uint64_t& b) const
    {
        uint32_t al = lo32(a), ah = hi32(a), bl = lo32(b), bh = hi32(b);
        (*this)(al, bl);
        (*this)(ah, bh);
        a = ((uint64_t)ah << 32) | al;
        b = ((uint64_t)bh << 32) | bl;
    }
};

// how a RowRec compares its key
enum KeyMode : int {
    KEY_MASKED = 0, // words 0..KW-1, each AND-ed with Cols::mask (runtime)
    KEY_FULL = 1,   // words 0..KW-1 as they are
    KEY_HI32 = 2,   // the high 32 bits of word 0 only (KW == 1)
};

// (u64 key, u32 payload), ordered lexicographically on both (plain sort rows).
// Every field is compared, so the sorted output is unique.  Registers hold
// the key as two 32-bit halves so exchanges never repack 64-bit values.
struct RowKP {
    uint32_t kl, kh, p;
    struct Cols {
        uint64_t* k;
        uint32_t* p;
    };
    static constexpr int SMEM_BYTES = 16; // one 16-byte slot per row (kl, kh, p, unused)
    static constexpr int SWZ_BITS = 3;
    __device__ __forceinline__ static RowKP load(const Cols& c, size_t g)
    {
        VELO_TRACE_AT(TS_ROW_LOAD, c.k + g);
        const uint64_t k = __ldcg(c.k + g);
        return RowKP { lo32(k), hi32(k), __ldcg(c.p + g) };
    }
    __device__ __forceinline__ static void store(const Cols& c, size_t g, const RowKP& r)
    {
        VELO_TRACE_AT(TS_ROW_STORE, c.k + g);
        c.k[g] = ((uint64_t)r.kh << 32) | r.kl;
        c.p[g] = r.p;
    }
    __device__ __forceinline__ static RowKP pad(const Cols&) { return RowKP { ~0u, ~0u, ~0u }; }
    __device__ __forceinline__ static void sstore(char* sm, int, int i, const RowKP& r)
    {
        reinterpret_cast<uint4*>(sm)[i] = make_uint4(r.kl, r.kh, r.p, 0u);
    }
    // the same at byte offset `b` = slot * SLOT_BYTES
    static constexpr int SLOT_BYTES = 16;
    __device__ __forceinline__ static void sstore_b(char* sm, int, uint32_t b, const RowKP& r)
    {
        *reinterpret_cast<uint4*>(sm + b) = make_uint4(r.kl, r.kh, r.p, 0u);
    }
    __device__ __forceinline__ static RowKP sload_b(const char* sm, int, uint32_t b)
    {
        const uint4 x = *reinterpret_cast<const uint4*>(sm + b);
        return RowKP { x.x, x.y, x.z };
    }
    __device__ __forceinline__ static RowKP sload(const char* sm, int, int i)
    {
        const uint4 x = reinterpret_cast<const uint4*>(sm)[i];
        return RowKP { x.x, x.y, x.z };
    }
    __device__ __forceinline__ static bool swap_pred(const RowKP& a, const RowKP& b, bool desc, const Cols&)
    {
        return (gt_mask3(a.p, a.kl, a.kh, b.p, b.kl, b.kh) != 0u) != desc;
    }
    // exchange a and b when x, in place: key halves on the multiply-add
    // pipe, payload by selects
    __device__ __forceinline__ static void cswap(RowKP& a, RowKP& b, bool x)
    {
        const MadSwap m(x);
        m(a.kl, b.kl);
        m(a.kh, b.kh);
        xsel(x, a.p, b.p);
    }
    __device__ __forceinline__ static bool marked(const RowKP&) { return false; }
};

// (u64 key, u32 payload, u8 mark): compaction rows; ordered on (key, payload)
// with the mark carried, strictly.
struct RowKPM {
    uint32_t kl, kh, p, m;
    struct Cols {
        uint64_t* k;
        uint32_t* p;
        uint8_t* m;
    };
    static constexpr int SMEM_BYTES = 16; // one 16-byte slot per row (kl, kh, p, m)
    static constexpr int SWZ_BITS = 3;
    __device__ __forceinline__ static RowKPM load(const Cols& c, size_t g)
    {
        VELO_TRACE_AT(TS_ROW_LOAD, c.k + g);
        const uint64_t k = __ldcg(c.k + g);
        return RowKPM { lo32(k), hi32(k), __ldcg(c.p + g), (uint32_t)__ldcg(c.m + g) };
    }
    __device__ __forceinline__ static void store(const Cols& c, size_t g, const RowKPM& r)
    {
        VELO_TRACE_AT(TS_ROW_STORE, c.k + g);
        c.k[g] = ((uint64_t)r.kh << 32) | r.kl;
        c.p[g] = r.p;
        c.m[g] = (uint8_t)r.m;
    }
    __device__ __forceinline__ static RowKPM pad(const Cols&) { return RowKPM { ~0u, ~0u, ~0u, 0u }; }
    __device__ __forceinline__ static void sstore(char* sm, int, int i, const RowKPM& r)
    {
        reinterpret_cast<uint4*>(sm)[i] = make_uint4(r.kl, r.kh, r.p, r.m);
    }
    static constexpr int SLOT_BYTES = 16;
    __device__ __forceinline__ static void sstore_b(char* sm, int, uint32_t b, const RowKPM& r)
    {
        *reinterpret_cast<uint4*>(sm + b) = make_uint4(r.kl, r.kh, r.p, r.m);
    }
    __device__ __forceinline__ static RowKPM sload_b(const char* sm, int, uint32_t b)
    {
        const uint4 x = *reinterpret_cast<const uint4*>(sm + b);
        return RowKPM { x.x, x.y, x.z, x.w };
    }
    __device__ __forceinline__ static RowKPM sload(const char* sm, int, int i)
    {
        const uint4 x = reinterpret_cast<const uint4*>(sm)[i];
        return RowKPM { x.x, x.y, x.z, x.w };
    }
    __device__ __forceinline__ static bool swap_pred(const RowKPM& a, const RowKPM& b, bool desc, const Cols&)
    {
        const uint32_t gt = gt_mask3(a.p, a.kl, a.kh, b.p, b.kl, b.kh);
        const uint32_t lt = gt_mask3(b.p, b.kl, b.kh, a.p, a.kl, a.kh);
        return (desc ? lt : gt) != 0u;
    }
    __device__ __forceinline__ static void cswap(RowKPM& a, RowKPM& b, bool x)
    {
        const MadSwap mad(x);
        mad(a.kl, b.kl);
        mad(a.kh, b.kh);
        mad(a.p, b.p);
        xsel(x, a.m, b.m);
    }
    __device__ __forceinline__ static bool marked(const RowKPM& r) { return r.m != 0; }
};

// W u64 words per row (SoA).  Ordered lexicographically on the first KW words
// as KM says (masked, whole, or the high half of word 0); the mark (for
// compaction) is bit `mark_bit` of word `mark_word`, inverted when mark_inv is
// set (so an "invalid" flag can sort last).
template <int W, int KW, bool STRICT = true, int KM = KEY_MASKED>
struct RowRec {
    static_assert(KM != KEY_HI32 || KW == 1, "a 32-bit key lives in word 0");
    static constexpr int WORDS = W;
    static constexpr int KEY_WORDS = KW;
    uint64_t w[W];
    struct Cols {
        uint64_t* w[W];
        uint64_t mask[KW];
        uint64_t pad[W];
        int mark_bit;
        int mark_inv;
        int mark_word; // word holding the mark bit (0 unless set)
    };
    // smem: words 0 and 1 share a 16-byte slot (W >= 2), word 2 (W == 3) is a
    // separate 8-byte array; W == 1 uses 8-byte slots
    static constexpr int SMEM_BYTES = 8 * W + (W == 3 ? 0 : 0);
    static constexpr int SWZ_BITS = W == 1 ? 4 : 3;
    __device__ __forceinline__ static RowRec load(const Cols& c, size_t g)
    {
        VELO_TRACE_AT(TS_ROW_LOAD, c.w[0] + g);
        RowRec r;
#pragma unroll
        for (int i = 0; i < W; i++)
            r.w[i] = __ldcg(c.w[i] + g);
        return r;
    }
    __device__ __forceinline__ static void store(const Cols& c, size_t g, const RowRec& r)
    {
        VELO_TRACE_AT(TS_ROW_STORE, c.w[0] + g);
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
    // slot at byte offset b = slot * SLOT_BYTES (words past the second in
    // 8-byte arrays at b / 2)
    static constexpr int SLOT_BYTES = W == 1 ? 8 : 16;
    __device__ __forceinline__ static void sstore_b(char* sm, int T, uint32_t b, const RowRec& r)
    {
        if constexpr (W == 1) {
            *reinterpret_cast<uint64_t*>(sm + b) = r.w[0];
        } else {
            *reinterpret_cast<ulonglong2*>(sm + b) = make_ulonglong2(r.w[0], r.w[1]);
#pragma unroll
            for (int x = 2; x < W; x++)
                *reinterpret_cast<uint64_t*>(sm + (size_t)16 * T + (size_t)8 * T * (x - 2) + (b >> 1)) = r.w[x];
        }
    }
    __device__ __forceinline__ static RowRec sload_b(const char* sm, int T, uint32_t b)
    {
        RowRec r;
        if constexpr (W == 1) {
            r.w[0] = *reinterpret_cast<const uint64_t*>(sm + b);
        } else {
            const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(sm + b);
            r.w[0] = x.x;
            r.w[1] = x.y;
#pragma unroll
            for (int y = 2; y < W; y++)
                r.w[y] = *reinterpret_cast<const uint64_t*>(sm + (size_t)16 * T + (size_t)8 * T * (y - 2) + (b >> 1));
        }
        return r;
    }
    __device__ __forceinline__ static void sstore(char* sm, int T, int i, const RowRec& r)
    {
        if constexpr (W == 1) {
            reinterpret_cast<uint64_t*>(sm)[i] = r.w[0];
        } else {
            reinterpret_cast<ulonglong2*>(sm)[i] = make_ulonglong2(r.w[0], r.w[1]);
#pragma unroll
            for (int x = 2; x < W; x++)
                reinterpret_cast<uint64_t*>(sm + (size_t)16 * T + (size_t)8 * T * (x - 2))[i] = r.w[x];
        }
    }
    __device__ __forceinline__ static RowRec sload(const char* sm, int T, int i)
    {
        RowRec r;
        if constexpr (W == 1) {
            r.w[0] = reinterpret_cast<const uint64_t*>(sm)[i];
        } else {
            const ulonglong2 x = reinterpret_cast<const ulonglong2*>(sm)[i];
            r.w[0] = x.x;
            r.w[1] = x.y;
#pragma unroll
            for (int y = 2; y < W; y++)
                r.w[y] = reinterpret_cast<const uint64_t*>(sm + (size_t)16 * T + (size_t)8 * T * (y - 2))[i];
        }
        return r;
    }
    // about half of the registers on the multiply-add pipe, the rest by
    // selects (W = 1: the high half only)
    __device__ __forceinline__ static void cswap(RowRec& a, RowRec& b, bool x)
    {
        const MadSwap mad(x);
        if constexpr (W == 1) {
            uint32_t al = lo32(a.w[0]), ah = hi32(a.w[0]), bl = lo32(b.w[0]), bh = hi32(b.w[0]);
            xsel(x, al, bl);
            mad(ah, bh);
            a.w[0] = ((uint64_t)ah << 32) | al;
            b.w[0] = ((uint64_t)bh << 32) | bl;
        } else {
#pragma unroll
            for (int i = 0; i < W; i++) {
                if (2 * i < W)
                    mad(a.w[i], b.w[i]);
                else
                    xsel(x, a.w[i], b.w[i]);
            }
        }
    }
    // the same exchange with one more 32-bit half on the multiply-add pipe
    // (two-word records compared on a whole word: three of four halves);
    // levels alternate between the two forms so that the ALU pipe, which
    // also carries the 64-bit compare, and the multiply-add pipe stay about
    // even (join union sort 1.92 -> 1.87 ms; no change with a 32-bit key)
    __device__ __forceinline__ static void cswap_fma(RowRec& a, RowRec& b, bool x)
    {
        if constexpr (W == 2 && KM != KEY_HI32) {
            const MadSwap mad(x);
            mad(a.w[0], b.w[0]);
            uint32_t al = lo32(a.w[1]), ah = hi32(a.w[1]), bl = lo32(b.w[1]), bh = hi32(b.w[1]);
            mad(al, bl);
            xsel(x, ah, bh);
            a.w[1] = ((uint64_t)ah << 32) | al;
            b.w[1] = ((uint64_t)bh << 32) | bl;
        } else {
            cswap(a, b, x);
        }
    }
    __device__ __forceinline__ static bool swap_pred(const RowRec& a, const RowRec& b, bool desc, const Cols& c)
    {
        if constexpr (KM == KEY_HI32) {
            const uint32_t x = hi32(a.w[0]), y = hi32(b.w[0]);
            if constexpr (STRICT)
                return desc ? (x < y) : (x > y);
            else
                return (x > y) != desc;
        }
        uint64_t ka[KW], kb[KW];
#pragma unroll
        for (int x = 0; x < KW; x++) {
            ka[x] = KM == KEY_FULL ? a.w[x] : (a.w[x] & c.mask[x]);
            kb[x] = KM == KEY_FULL ? b.w[x] : (b.w[x] & c.mask[x]);
        }
        if constexpr (STRICT) {
            const uint32_t gt = key_gt_mask<KW>(ka, kb);
            const uint32_t lt = key_gt_mask<KW>(kb, ka);
            return (desc ? lt : gt) != 0u;
        } else {
            return (key_gt_mask<KW>(ka, kb) != 0u) != desc;
        }
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
        // AND with a per-word mask rather than selecting the word: a select
        // chain over the words is turned into a dynamically indexed load, which
        // sends the whole register tile to local memory
        const uint64_t bit = 1ull << c.mark_bit;
        uint64_t w = 0;
#pragma unroll
        for (int x = 0; x < W; x++)
            w |= r.w[x] & (c.mark_word == x ? bit : 0ull);
        return (w != 0) != (c.mark_inv != 0);
    }
};

// compare-exchange form of a level: ALT = 1 takes a record's cswap_fma where
// it has one
template <class R, int ALT>
struct Cswap {
    __device__ __forceinline__ static void run(R& a, R& b, bool x) { R::cswap(a, b, x); }
};
template <int W, int KW, bool S, int KM>
struct Cswap<RowRec<W, KW, S, KM>, 1> {
    __device__ __forceinline__ static void run(RowRec<W, KW, S, KM>& a, RowRec<W, KW, S, KM>& b, bool x)
    {
        RowRec<W, KW, S, KM>::cswap_fma(a, b, x);
    }
};

template <class R>
struct MarkOf {
    __device__ __forceinline__ static bool get(const R& r, const typename R::Cols&) { return R::marked(r); }
};
template <int W, int KW, bool S, int KM>
struct MarkOf<RowRec<W, KW, S, KM>> {
    __device__ __forceinline__ static bool get(const RowRec<W, KW, S, KM>& r,
                                               const typename RowRec<W, KW, S, KM>::Cols& c)
    {
        return RowRec<W, KW, S, KM>::marked_c(r, c);
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

    // bank-spreading swizzle of smem slots: XOR SWZ bits taken above the
    // register window into the low bits, so the lanes of one shared-memory
    // phase (8 lanes for 16-byte slots, 16 for 8-byte slots) hit distinct
    // banks in every layout.  The source bits are never modified, so it is a
    // bijection on the tile; it is linear over XOR, so
    // swz(a | b) = swz(a) ^ swz(b) for disjoint a, b.
    template <int SWZ>
    __host__ __device__ __forceinline__ static constexpr int swz(int l)
    {
        return l ^ ((l >> (LOG_E > SWZ ? LOG_E : SWZ)) & ((1 << SWZ) - 1));
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
