// Pass kernels of the two oblivious networks on top of the tile engine.
//
// Bitonic sort of Np = 2^logN rows with tile T = 2^LT (reference network
// order, include/cuda/sort.cuh:104-117):
//   SORT_TILE          phases k = 2..min(T, Np) entirely inside each tile
//   SORT_GLOBAL(K,b,L) L consecutive levels j = 2^b .. 2^(b-L+1) (all >= T)
//                      of phase k = 2^K, fused: each CTA holds 2^L strided
//                      row groups x 2^(LT-L) consecutive rows
//   SORT_MERGE(K)      levels j = T/2 .. 1 of phase k = 2^K inside each tile
// ORCompact over Np rows (liboblivious algorithms.c:116-213, evaluated level
// by level; block offsets come from a prefix count of the marks):
//   COMPACT_TILE       levels with block size 2 .. T inside each tile
//   COMPACT_GLOBAL     L consecutive levels with block sizes > T, fused
#pragma once

#include <type_traits>

#include "engine.cuh"

namespace velo {

enum PassKind : int {
    P_SORT_TILE = 0,
    P_SORT_MERGE = 1,
    P_SORT_GLOBAL = 2,
    P_COMPACT_TILE = 3,
    P_COMPACT_GLOBAL = 4,
};

struct NetGeom {
    size_t n;  // real rows (public)
    int logN;  // log2 of the padded size
    int pad_;
};

struct NetPass {
    int kind;
    int K;    // sort phase (log2 k) / highest tile level for *_TILE passes
    int b_hi; // GLOBAL: highest global bit of the fused levels
    int L;    // GLOBAL: number of fused levels
};

// mark of the row stored at global index g (count pass)
template <class R>
struct MarkAt;
template <>
struct MarkAt<RowKP> {
    __device__ __forceinline__ static bool get(const RowKP::Cols&, size_t) { return false; }
};
template <>
struct MarkAt<RowKPM> {
    __device__ __forceinline__ static bool get(const RowKPM::Cols& c, size_t g)
    {
        VELO_TRACE_AT(TS_MARK_LOAD, c.m + g);
        return __ldcg(c.m + g) != 0;
    }
};
template <int W, int KW, bool S, int KM>
struct MarkAt<RowRec<W, KW, S, KM>> {
    __device__ __forceinline__ static bool get(const typename RowRec<W, KW, S, KM>::Cols& c, size_t g)
    {
        // select the column pointer with constant indices (indexing the
        // parameter array with mark_word copies it to local memory)
        const uint64_t* col = c.w[0];
#pragma unroll
        for (int x = 1; x < W; x++)
            col = c.mark_word == x ? c.w[x] : col;
        VELO_TRACE_AT(TS_MARK_LOAD, col + g);
        return (((__ldcg(col + g) >> c.mark_bit) & 1ull) != 0) != (c.mark_inv != 0);
    }
};

// exclusive scan of one u32 per thread across the CTA; tmp holds >= 33 u32
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t* tmp, uint32_t* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        inc += (lane >= o) ? y : 0u;
    }
    __syncthreads();
    if (lane == 31)
        tmp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? tmp[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            wi += (lane >= o) ? y : 0u;
        }
        if (lane < nw)
            tmp[lane] = wi - w;
        if (lane == 31)
            tmp[32] = wi;
    }
    __syncthreads();
    uint32_t r = tmp[warp] + inc - x;
    *total = tmp[32];
    return r;
}

// compile-time loops over register bits: f(integral_constant<Q>) for
// Q = HI down to 0, or 0 up to HI
template <int Q>
struct QDown {
    template <class F>
    __device__ __forceinline__ static void run(F& f)
    {
        f(std::integral_constant<int, Q> {});
        QDown<Q - 1>::run(f);
    }
};
template <>
struct QDown<-1> {
    template <class F>
    __device__ __forceinline__ static void run(F&)
    {
    }
};
template <int Q, int HI>
struct QUp {
    template <class F>
    __device__ __forceinline__ static void run(F& f)
    {
        f(std::integral_constant<int, Q> {});
        QUp<Q + 1, HI>::run(f);
    }
};
template <int HI>
struct QUp<HI, HI> {
    template <class F>
    __device__ __forceinline__ static void run(F&)
    {
    }
};

template <class R, int LOG_NT, int LOG_E>
struct Net {
    using TL = Tile<LOG_NT, LOG_E>;
    using Cols = typename R::Cols;
    static constexpr int E = TL::E;
    static constexpr int LT = TL::LOG_T;
    static constexpr int T = TL::T;
    static constexpr int S0 = LT - LOG_E; // load/store layout (lanes <-> rows 0..31)

    static constexpr size_t smem_rows() { return ((size_t)T * R::SMEM_BYTES + 15) & ~(size_t)15; }
    static constexpr size_t smem_bytes_sort() { return smem_rows(); }
    // the tile prefix array holds one pad word after every 16 (ppos)
    static constexpr size_t smem_bytes_compact() { return smem_rows() + (size_t)(T + T / 16) * 4 + 33 * 4; }

    // slot of tile prefix entry l: one pad word every 16 entries, so that a
    // warp reading entries 16 apart (the block starts of the lowest levels
    // in layout 0) hits 32 different banks instead of 2
    __device__ __forceinline__ static int ppos(int l) { return l + (l >> 4); }

    // thread part of the local row index in layout s
    __device__ __forceinline__ static int tidpart(int s)
    {
        const int tid = threadIdx.x;
        return (tid & ((1 << s) - 1)) | ((tid >> s) << (s + LOG_E));
    }

    static constexpr int SWZ = R::SWZ_BITS;

    // smem slots of the E registers in layout s: swz(tp | e<<s) =
    // swz(tp) ^ swz(e<<s), and swz(e<<s) is the XOR of the basis values
    // swz(1 << (s+j)) over the set bits j of e (one XOR per register)
    __device__ __forceinline__ static void slots(int s, int (&slot)[E])
    {
        int basis[LOG_E > 0 ? LOG_E : 1];
#pragma unroll
        for (int j = 0; j < LOG_E; j++)
            basis[j] = TL::template swz<SWZ>(1 << (s + j));
        slot[0] = TL::template swz<SWZ>(tidpart(s));
#pragma unroll
        for (int e = 1; e < E; e++) {
            const int low = e & (-e); // lowest set bit of e
            const int j = low == 1 ? 0 : low == 2 ? 1 : low == 4 ? 2 : low == 8 ? 3 : 4;
            slot[e] = slot[e & (e - 1)] ^ basis[j];
        }
    }

    // Transposes with the layout as a compile-time value (CT): the code for
    // layout S is picked at run time among 0 .. LT - LOG_E by a compare chain,
    // and each register's slot is the thread's base XOR a constant, instead
    // of a per-register XOR chain over run-time basis values.  Used by the
    // in-tile sort kernel, where transposes are a third of the ALU work.
    template <int S>
    __device__ __forceinline__ static int ct_base()
    {
        const int tp = (int)(threadIdx.x & ((1u << S) - 1)) | (int)((threadIdx.x >> S) << (S + LOG_E));
        return TL::template swz<SWZ>(tp);
    }
    // BOFF: XOR on byte offsets, (base ^ c) * SZ == (base * SZ) ^ (c * SZ),
    // so no multiply per register; the three-CTA forms (at most 85
    // registers) keep slot indices, measured faster there
    template <bool BOFF, int S = 0>
    __device__ __forceinline__ static void store_ct(const R (&v)[E], int s, char* sm)
    {
        if constexpr (S <= LT - LOG_E) {
            if (s == S) {
                if constexpr (BOFF) {
                    const uint32_t bb = (uint32_t)ct_base<S>() * R::SLOT_BYTES;
#pragma unroll
                    for (int e = 0; e < E; e++)
                        R::sstore_b(sm, T, bb ^ (uint32_t)(TL::template swz<SWZ>(e << S) * R::SLOT_BYTES), v[e]);
                } else {
                    const int base = ct_base<S>();
#pragma unroll
                    for (int e = 0; e < E; e++)
                        R::sstore(sm, T, base ^ TL::template swz<SWZ>(e << S), v[e]);
                }
            } else {
                store_ct<BOFF, S + 1>(v, s, sm);
            }
        }
    }
    template <bool BOFF, int S = 0>
    __device__ __forceinline__ static void load_ct(R (&v)[E], int s, const char* sm)
    {
        if constexpr (S <= LT - LOG_E) {
            if (s == S) {
                if constexpr (BOFF) {
                    const uint32_t bb = (uint32_t)ct_base<S>() * R::SLOT_BYTES;
#pragma unroll
                    for (int e = 0; e < E; e++)
                        v[e] = R::sload_b(sm, T, bb ^ (uint32_t)(TL::template swz<SWZ>(e << S) * R::SLOT_BYTES));
                } else {
                    const int base = ct_base<S>();
#pragma unroll
                    for (int e = 0; e < E; e++)
                        v[e] = R::sload(sm, T, base ^ TL::template swz<SWZ>(e << S));
                }
            } else {
                load_ct<BOFF, S + 1>(v, s, sm);
            }
        }
    }

    // re-layout the tile from layout `from` to layout `to` through smem
    template <bool CT = false, bool BOFF = true>
    __device__ __forceinline__ static void transpose(R (&v)[E], int from, int to, char* sm)
    {
        if constexpr (CT) {
            __syncthreads();
            store_ct<BOFF>(v, from, sm);
            __syncthreads();
            load_ct<BOFF>(v, to, sm);
            return;
        }
        int slot[E];
        __syncthreads();
        slots(from, slot);
#pragma unroll
        for (int e = 0; e < E; e++)
            R::sstore(sm, T, slot[e], v[e]);
        __syncthreads();
        slots(to, slot);
#pragma unroll
        for (int e = 0; e < E; e++)
            v[e] = R::sload(sm, T, slot[e]);
    }

    // ---- bitonic compare-exchange on register bit Q -----------------------
    // The direction of a pair is bit K of its local index (phase k = 2^K).
    // It is one mask `dm` for all of a thread's pairs unless K falls inside
    // the register window (only for phases k < 2^LOG_E), where pair e is
    // descending iff bit `dbit` of e is set.
    template <int Q, bool PER_E>
    __device__ __forceinline__ static void bitonic_level(R (&v)[E], const Cols& c, bool dm, uint32_t dpat)
    {
#pragma unroll
        for (int e = 0; e < E; e++) {
            if (e & (1 << Q))
                continue;
            const int e2 = e | (1 << Q);
            bool d = dm;
            if constexpr (PER_E)
                d = (dpat & (1u << e)) != 0u;
            Cswap<R, Q & 1>::run(v[e], v[e2], R::swap_pred(v[e], v[e2], d, c));
        }
    }

    // levels on local bits b_hi down to b_lo, all inside the window of layout s
    __device__ __forceinline__ static void bitonic_window(R (&v)[E], const Cols& c, int s, int b_hi, int b_lo, int K,
                                                          bool dconst, bool asc_c)
    {
        const bool per_e = !dconst && K >= s && K < s + LOG_E;
        const bool dm = dconst ? !asc_c : (((tidpart(s) >> K) & 1) != 0);
        // per-register directions: bit e set iff bit K-s of e is set
        const int kb = K - s;
        const uint32_t dpat = !per_e ? 0u
            : kb == 0               ? 0xAAAAAAAAu
            : kb == 1               ? 0xCCCCCCCCu
            : kb == 2               ? 0xF0F0F0F0u
            : kb == 3               ? 0xFF00FF00u
                                    : 0xFFFF0000u;
        static_assert(LOG_E <= 5, "direction patterns cover 32 registers");
        if (b_hi >= s + LOG_E - 1 && b_lo <= s) {
            // the whole window: straight-line levels, no per-level branch
            // (a branch per level makes every join re-home the row registers)
            if (per_e) {
                auto f = [&](auto qc) { bitonic_level<decltype(qc)::value, true>(v, c, dm, dpat); };
                QDown<LOG_E - 1>::run(f);
            } else {
                auto f = [&](auto qc) { bitonic_level<decltype(qc)::value, false>(v, c, dm, dpat); };
                QDown<LOG_E - 1>::run(f);
            }
            return;
        }
        auto f = [&](auto qc) {
            constexpr int Q = decltype(qc)::value;
            const int b = s + Q;
            if (b <= b_hi && b >= b_lo) {
                if (per_e)
                    bitonic_level<Q, true>(v, c, dm, dpat);
                else
                    bitonic_level<Q, false>(v, c, dm, dpat);
            }
        };
        QDown<LOG_E - 1>::run(f);
    }

    // ---- ORCompact exchange (tile-local level, block size 2^(b+1)) --------
    // Pair (l, l + 2^b) inside block S; the block's offset is P[S] mod 2^(b+1)
    // and its left-half mark count is P[S + 2^b] - P[S] (P = exclusive prefix
    // of the original marks; block counts are invariant under the
    // permutations of lower levels).  Level b is register bit Q of layout s
    // (b = s + Q): the registers whose bits above Q agree lie in one block, so
    // each of the thread's E >> (Q + 1) blocks is looked up once and its
    // 2^Q pairs share the offset, the count and the threshold.
    template <int Q>
    __device__ __forceinline__ static void compact_level_tile(R (&v)[E], const Cols& c, int s, int b, uint32_t p_tile,
                                                              const uint32_t* pre)
    {
        const int tp = tidpart(s);
        const uint32_t half = 1u << b;
        const int tblk = tp & ~(int)(2 * half - 1); // the thread's bits above b
        const uint32_t ti = (uint32_t)tp & (half - 1u); // its bits below b (all below s)
        constexpr int NB = E >> (Q + 1);
#pragma unroll
        for (int hb = 0; hb < NB; hb++) {
            const int blk = tblk | (hb << (b + 1));
            const uint32_t pb = pre[ppos(blk)];
            const uint32_t ps = p_tile + pb;
            if (b == 0) {
                // compact_offset, n == 2 (algorithms.c:123-128): one pair a block
                const int e = hb << 1, e2 = e | 1;
                const bool ml = MarkOf<R>::get(v[e], c), mr = MarkOf<R>::get(v[e2], c);
                R::cswap(v[e], v[e2], ((!ml) & mr) != ((ps & 1u) == 1u));
            } else {
                // compact_offset, n > 2 (algorithms.c:130-152)
                const uint32_t left = pre[ppos(blk + (int)half)] - pb;
                const uint32_t off = ps & (2 * half - 1);
                const bool sb = (((off & (half - 1)) + left) >= half) != (off >= half);
                const uint32_t thr = (off + left) & (half - 1);
#pragma unroll
                for (int lo = 0; lo < (1 << Q); lo++) {
                    const int e = (hb << (Q + 1)) | lo, e2 = e | (1 << Q);
                    const uint32_t i = ti | ((uint32_t)lo << s);
                    R::cswap(v[e], v[e2], sb != (i >= thr));
                }
            }
        }
    }

    // `gpre[m]` holds P at the tile whose bits b_lo..b_hi are m (the CTA's
    // other tile bits fixed, its bits below b_lo zero): every block start and
    // block middle of a global level is such a tile boundary.  Global level b
    // is register bit Q of layout s, so as in the tile levels the thread's
    // E >> (Q + 1) blocks are looked up once each.
    template <int Q>
    __device__ __forceinline__ static void compact_level_global(R (&v)[E], const Cols& c, int s, int b,
                                                                const uint32_t* gpre, int C, int b_lo,
                                                                size_t cta_bits, int L)
    {
        // 32-bit index arithmetic: row indices are below 2^MAX_LOGN = 2^31,
        // so g, 2 * half - 1 and (off + left) all fit
        const uint32_t tp = (uint32_t)tidpart(s);
        const uint32_t half = 1u << b;
        const uint32_t bm = 2u * half - 1u;
        const uint32_t mmask = (1u << L) - 1u;
        const uint32_t cb = (uint32_t)cta_bits;
        const uint32_t cm = (1u << C) - 1u;
        constexpr int NB = E >> (Q + 1);
#pragma unroll
        for (int hb = 0; hb < NB; hb++) {
            // the block of the block's first pair
            const uint32_t l0 = tp | ((uint32_t)(hb << (Q + 1)) << s);
            const uint32_t g0 = (l0 & cm) | ((l0 >> C) << b_lo) | cb;
            const uint32_t mb = ((g0 & ~bm) >> b_lo) & mmask;
            const uint32_t ps = gpre[mb];
            const uint32_t left = gpre[mb | (1u << (b - b_lo))] - ps;
            const uint32_t off = ps & bm;
            const bool sb = (((off & (half - 1u)) + left) >= half) != (off >= half);
            const uint32_t thr = (off + left) & (half - 1u);
#pragma unroll
            for (int lo = 0; lo < (1 << Q); lo++) {
                const int e = (hb << (Q + 1)) | lo, e2 = e | (1 << Q);
                const uint32_t l = tp | ((uint32_t)e << s);
                const uint32_t g = (l & cm) | ((l >> C) << b_lo) | cb;
                R::cswap(v[e], v[e2], sb != ((g & bm) >= thr));
            }
        }
    }

    // ---- one pass over one tile (CTA `cta`) --------------------------------
    // SORT = true compiles only the bitonic pass kinds, false only ORCompact.
    // PK: the pass kinds this instantiation handles (a separate kernel each,
    // so that each gets its own register allocation)
    // ST (not void): the pass's rows are already in shared memory in local
    // row order, staged by a tensor-map tile load; ST::read(sm, T, l) reads
    // row l (merge and fused global passes only)
    // PK_MERGE: the in-tile merges alone (no tile-sort code)
    enum : int { PK_ANY = 0, PK_LOCAL = 1, PK_GLOBAL = 2, PK_MERGE = 3 };
    template <bool SORT, int PK = PK_ANY, bool WIDE = false, class ST = void>
    __device__ static void run(const Cols& c, const NetGeom& g, const NetPass& p, const uint32_t* tile_prefix,
                               int cta, char* sm)
    {
        constexpr bool CT = SORT && (PK == PK_LOCAL || PK == PK_MERGE);
        constexpr bool BOFF = !WIDE;
        const size_t Np = (size_t)1 << g.logN;
        const bool is_global = PK == PK_GLOBAL ? true
            : PK == PK_LOCAL || PK == PK_MERGE ? false
                                               : (p.kind == P_SORT_GLOBAL) || (p.kind == P_COMPACT_GLOBAL);
        int C = LT, b_lo = 0;
        size_t cta_bits = (size_t)cta << LT;
        if (is_global) {
            C = LT - p.L;
            b_lo = p.b_hi - p.L + 1;
            const int lo_bits = b_lo - C;
            cta_bits = ((size_t)(cta & ((1 << lo_bits) - 1)) << C) | ((size_t)(cta >> lo_bits) << (p.b_hi + 1));
        }
        auto gidx = [&](int l) -> size_t {
            if (!is_global)
                return cta_bits | (size_t)l;
            return (size_t)(l & ((1 << C) - 1)) | ((size_t)(l >> C) << b_lo) | cta_bits;
        };
        const int smin = is_global ? (C < S0 ? C : S0) : 0;

        R v[E];
        int s = (p.kind == P_COMPACT_GLOBAL) ? smin : S0;
        const bool first = (p.kind == P_SORT_TILE) || (p.kind == P_COMPACT_TILE);
        if constexpr (!std::is_void_v<ST>) {
            // the first transpose's barrier ends these reads before the
            // staged tile is overwritten
            const int tp = tidpart(s);
#pragma unroll
            for (int e = 0; e < E; e++)
                v[e] = ST::read(sm, T, tp | (e << s));
        } else {
            const int tp = tidpart(s);
#pragma unroll
            for (int e = 0; e < E; e++) {
                const size_t gi = gidx(tp | (e << s));
                if (first)
                    v[e] = (gi < g.n) ? R::load(c, gi) : R::pad(c);
                else
                    v[e] = R::load(c, gi);
            }
        }

        if constexpr (SORT) {
            if (PK != PK_GLOBAL && PK != PK_MERGE && p.kind == P_SORT_TILE) {
                for (int K = 1; K <= p.K; K++) {
                    const bool dconst = K >= LT;
                    const bool asc_c = ((cta_bits >> K) & 1) == 0;
                    int b = K - 1;
                    while (b >= 0) {
                        if (b < s || b >= s + LOG_E) {
                            const int ns = window_down(b, LOG_E, LT);
                            transpose<CT, BOFF>(v, s, ns, sm);
                            s = ns;
                        }
                        bitonic_window(v, c, s, b, s, K, dconst, asc_c);
                        b = s - 1;
                    }
                }
            } else {
                // MERGE: bits LT-1..0; GLOBAL: local bits C+L-1..C (the L fused
                // global levels); the direction is fixed for the tile
                const bool merge = PK == PK_MERGE || (PK != PK_GLOBAL && p.kind == P_SORT_MERGE);
                const bool asc_c = (((merge ? cta_bits : gidx(0)) >> p.K) & 1) == 0;
                const int top = merge ? LT - 1 : C + p.L - 1;
                const int bottom = merge ? 0 : C;
                int b = top;
                while (b >= bottom) {
                    if (b < s || b >= s + LOG_E) {
                        int ns = window_down(b, LOG_E, LT);
                        ns = ns < smin ? smin : ns;
                        transpose<CT, BOFF>(v, s, ns, sm);
                        s = ns;
                    }
                    const int lo = s > bottom ? s : bottom;
                    bitonic_window(v, c, s, b, lo, p.K, true, asc_c);
                    b = lo - 1;
                }
            }
        } else {
            if (PK == PK_LOCAL || (PK != PK_GLOBAL && p.kind == P_COMPACT_TILE)) {
                // prefix of the original marks over the tile, in local-index order
                uint32_t* pre = reinterpret_cast<uint32_t*>(sm + smem_rows());
                uint32_t* tmp = pre + T + T / 16;
                transpose<CT, BOFF>(v, s, 0, sm);
                s = 0;
                uint32_t cnt = 0, m[E];
#pragma unroll
                for (int e = 0; e < E; e++) {
                    m[e] = cnt;
                    cnt += MarkOf<R>::get(v[e], c) ? 1u : 0u;
                }
                uint32_t total;
                const uint32_t base = block_exclusive_scan(cnt, tmp, &total);
                const int tp0 = tidpart(0);
#pragma unroll
                for (int e = 0; e < E; e++)
                    pre[ppos(tp0 | e)] = base + m[e];
                __syncthreads();
                VELO_TRACE_AT(TS_TILE_PREFIX, tile_prefix + cta);
                const uint32_t p_tile = __ldcg(tile_prefix + cta);
                int b = 0;
                while (b < p.K) {
                    if (b < s || b >= s + LOG_E) {
                        const int ns = window_up(b, LOG_E, LT);
                        transpose<CT, BOFF>(v, s, ns, sm);
                        s = ns;
                    }
                    const int hi = (s + LOG_E - 1 < p.K - 1) ? s + LOG_E - 1 : p.K - 1;
                    if (b <= s && hi == s + LOG_E - 1) {
                        auto f = [&](auto qc) {
                            constexpr int Q = decltype(qc)::value;
                            compact_level_tile<Q>(v, c, s, s + Q, p_tile, pre);
                        };
                        QUp<0, LOG_E>::run(f);
                    } else {
                        auto f = [&](auto qc) {
                            constexpr int Q = decltype(qc)::value;
                            const int bb = s + Q;
                            if (bb >= b && bb <= hi)
                                compact_level_tile<Q>(v, c, s, bb, p_tile, pre);
                        };
                        QUp<0, LOG_E>::run(f);
                    }
                    b = hi + 1;
                }
            } else { // P_COMPACT_GLOBAL: local bits C..C+L-1 bottom-up
                uint32_t* gpre = reinterpret_cast<uint32_t*>(sm + smem_rows());
                {
                    const int lo_bits = b_lo - C;
                    const size_t t_hi = ((size_t)(cta >> lo_bits)) << (p.b_hi + 1 - LT);
                    for (int m = threadIdx.x; m < (1 << p.L); m += TL::NT) {
                        VELO_TRACE_AT(TS_TILE_PREFIX, tile_prefix + (t_hi | ((size_t)m << (b_lo - LT))));
                        gpre[m] = __ldcg(tile_prefix + (t_hi | ((size_t)m << (b_lo - LT))));
                    }
                    __syncthreads();
                }
                int lb = C;
                const int top = C + p.L - 1;
                while (lb <= top) {
                    if (lb < s || lb >= s + LOG_E) {
                        int ns = window_up(lb, LOG_E, LT);
                        ns = ns < smin ? smin : ns;
                        transpose<CT, BOFF>(v, s, ns, sm);
                        s = ns;
                    }
                    const int hi = (s + LOG_E - 1 < top) ? s + LOG_E - 1 : top;
                    if (lb <= s && hi == s + LOG_E - 1) {
                        auto f = [&](auto qc) {
                            constexpr int Q = decltype(qc)::value;
                            compact_level_global<Q>(v, c, s, b_lo + (s + Q - C), gpre, C, b_lo, cta_bits, p.L);
                        };
                        QUp<0, LOG_E>::run(f);
                    } else {
                        auto f = [&](auto qc) {
                            constexpr int Q = decltype(qc)::value;
                            const int lp = s + Q;
                            if (lp >= lb && lp <= hi)
                                compact_level_global<Q>(v, c, s, b_lo + (lp - C), gpre, C, b_lo, cta_bits, p.L);
                        };
                        QUp<0, LOG_E>::run(f);
                    }
                    lb = hi + 1;
                }
            }
        }

        // stores need 32 consecutive rows a warp, or (global passes) the
        // layout the rows were loaded in: there the lanes cover whole
        // 2^C-row segments, which are whole lines of every word array
        if (s < 5 && !(is_global && s == smin)) {
            transpose<CT, BOFF>(v, s, S0, sm);
            s = S0;
        }
        {
            const int tp = tidpart(s);
#pragma unroll
            for (int e = 0; e < E; e++) {
                const size_t gi = gidx(tp | (e << s));
                if (gi < Np)
                    R::store(c, gi, v[e]);
            }
        }
    }
};

// mark count of each tile (rows >= n count as unmarked)
template <class R>
__device__ __forceinline__ void count_tile(const typename R::Cols& c, size_t n, int LT, int cta, uint32_t* counts,
                                           uint32_t* tmp)
{
    const size_t base = (size_t)cta << LT;
    const int T = 1 << LT;
    uint32_t cnt = 0;
    // U loads a thread in flight before any is summed
    constexpr int U = 8;
    for (int i0 = threadIdx.x; i0 < T; i0 += U * (int)blockDim.x) {
        bool m[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int i = i0 + u * (int)blockDim.x;
            m[u] = false;
            if (i < T) {
                const size_t gi = base + i;
                const bool in = gi < n;
                const size_t gs = in ? gi : 0; // every row index is public: read row 0 for pads
                m[u] = in & MarkAt<R>::get(c, gs);
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++)
            cnt += m[u] ? 1u : 0u;
    }
    uint32_t total;
    block_exclusive_scan(cnt, tmp, &total);
    if (threadIdx.x == 0) {
        VELO_TRACE_AT(TS_TILE_COUNT, counts + cta);
        counts[cta] = total;
    }
}

// exclusive scan of the tile counts into prefix[0..ntiles]; one CTA
__device__ __forceinline__ void scan_tiles(const uint32_t* counts, int ntiles, uint32_t* prefix, uint64_t* d_count,
                                           uint32_t* tmp)
{
    uint32_t carry = 0;
    for (int base = 0; base < ntiles; base += blockDim.x) {
        const int i = base + threadIdx.x;
        if (i < ntiles)
            VELO_TRACE_AT(TS_SCAN, counts + i);
        const uint32_t x = i < ntiles ? __ldcg(counts + i) : 0u;
        uint32_t total;
        const uint32_t ex = block_exclusive_scan(x, tmp, &total);
        if (i < ntiles)
            prefix[i] = carry + ex;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        prefix[ntiles] = carry;
        if (d_count)
            *d_count = carry;
    }
}

} // namespace velo
